"""CPU oracle of the uniform-grid projection (test infrastructure only)."""

"""The seeded scene generators define the benchmark inputs; these checks pin the properties
each workload's description asks for."""
import numpy as np

from fluidsim_b200 import scenes


def test_viscous_blob_matches_its_description():
    s = scenes.viscous_blob(160, 128, seed=4)
    liquid = s.fraction > 0
    assert set(np.unique(s.fraction)) == {0.0, 1.0}
    assert abs(liquid.mean() - 0.6) < 1e-3
    # 1000:1 densities: every cell is all liquid or all air.
    rho = s.density()
    assert np.allclose(rho[liquid], 1000.0) and np.allclose(rho[~liquid], 1.0)
    # Volume-weighted blend of the two liquid components' viscosities (and air's) per cell.
    volumes = [m / d for m, d in zip(s.liquid_mass + s.gas_mass, [s.liquid_density] * 2 + [s.gas_density])]
    mu = sum(v * c for v, c in zip(volumes, s.liquid_viscosity + s.gas_viscosity)) / sum(volumes)
    log_mu = np.log10(mu[liquid])
    assert log_mu.min() >= -3 - 1e-9 and log_mu.max() <= 1 + 1e-9
    # log-uniform: equal counts in equal log-width bins
    counts, _ = np.histogram(log_mu, bins=8, range=(-3, 1))
    assert counts.max() - counts.min() <= 2
    # smooth: neighbouring liquid cells differ by far less than the range
    both = liquid[:, 1:] & liquid[:, :-1]
    step = np.abs(np.diff(np.log10(mu), axis=1))[both]
    assert np.median(step) < 0.1
    # walls closed, FP32 velocities
    assert not s.u[:, [0, -1]].any() and not s.v[[0, -1], :].any()
    assert np.array_equal(s.u, s.u.astype(np.float32).astype(np.float64))


def test_viscous_blob_is_seeded():
    a, b = scenes.viscous_blob(64, 48, seed=1), scenes.viscous_blob(64, 48, seed=1)
    c = scenes.viscous_blob(64, 48, seed=2)
    assert np.array_equal(a.liquid_mass[1], b.liquid_mass[1]) and np.array_equal(a.u, b.u)
    assert not np.array_equal(a.fraction, c.fraction)

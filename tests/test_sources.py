"""Rules the CUDA sources must keep, checked on the text (no GPU).

A warp shuffle with the full member mask must be executed by all 32 lanes. Written as one arm
of a conditional expression (`lane == 0 ? 0 : __shfl_up_sync(...)`), it is skipped by the lanes
that take the other arm, and the remaining lanes wait for them forever.
"""
import os
import re

CSRC = os.path.join(os.path.dirname(__file__), "..", "fluidsim_b200", "csrc")
SHUFFLE_IN_CONDITIONAL = re.compile(r"\?[^;]*__shfl_\w*sync")


def _sources():
    for name in sorted(os.listdir(CSRC)):
        if name.endswith((".cu", ".cuh", ".h", ".cpp")):
            with open(os.path.join(CSRC, name)) as f:
                yield name, f.read().splitlines()


def test_no_shuffle_inside_a_conditional_expression():
    bad = [f"{name}:{i + 1}: {line.strip()}" for name, lines in _sources() for i, line in enumerate(lines)
           if SHUFFLE_IN_CONDITIONAL.search(line.split("//")[0])]
    assert not bad, "shuffle in one arm of ?: (hoist it so every lane executes it):\n" + "\n".join(bad)


def test_rule_catches_the_pattern():
    assert SHUFFLE_IN_CONDITIONAL.search("const T wl = lane == 0 ? T(0) : __shfl_up_sync(0xffffffffu, w, 1);")
    assert not SHUFFLE_IN_CONDITIONAL.search("T wl = __shfl_up_sync(0xffffffffu, w, 1);")

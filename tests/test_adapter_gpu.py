"""The C++ drop-in at run time: fluid::FluidGridCUDA (include/FluidGridCUDA.h) and the
reference's own FluidGridCPU, both driven through fluid::FluidGridBase& by oracle/adapter_check
(built by oracle/Makefile from the reference headers and engine). The scenario restates the
reference's facade test (tests/FluidGridAPITests.cpp:186-229): 64 steps with a gravity change,
a zero-time and a zero-iteration step, destroy and re-upload; plus the checkpoint round trip
and the mapping of status codes to the reference's exception types. Bars: FP64 within 1e-8 of
each field's scale over the 64 steps, iterations within two; FP32 within 1e-4."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BINARY = os.path.join(ROOT, "oracle", "_ref", "adapter_check")

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_cpp_adapter_steps_like_the_reference_engine(precision):
    assert os.path.exists(BINARY), "oracle/_ref/adapter_check is built with the reference engine (oracle/Makefile)"
    out = subprocess.run([BINARY, precision], capture_output=True, text=True, timeout=600)
    print(out.stdout)
    assert out.returncode == 0, out.stdout[-4000:] + out.stderr[-2000:]
    assert "PASSED: 0 failure(s)" in out.stdout

"""The C ABI library: it loads, exports every symbol include/*.h declares, and refuses to work
without a device instead of falling back to the host."""
import ctypes as C
import os
import re
import shutil
import subprocess

import pytest

from conftest import ROOT

HEADER_DIR = os.path.join(ROOT, "include")


def declared_symbols():
    names = set()
    for path in os.listdir(HEADER_DIR):
        if not path.endswith(".h"):
            continue
        text = open(os.path.join(HEADER_DIR, path)).read()
        if 'extern "C"' not in text:
            continue
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_\s\*]*?\b(fc_[a-z0-9_]+)\s*\(", text, re.M):
            names.add(m.group(1))
    return names


def test_library_exports_declared_symbols():
    from fluidsim_b200 import _native

    lib = _native.lib()
    names = declared_symbols()
    assert len(names) >= 30
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python mirror binds exactly the declared ABI
    assert set(_native.SIGNATURES) == names


def test_abi_version_and_status_strings():
    from fluidsim_b200 import _native

    lib = _native.lib()
    assert lib.fc_abi_version() == 1
    assert lib.fc_status_string(1) == b"invalid argument"


def test_invalid_geometry_rejected_before_device_work():
    from fluidsim_b200 import _native

    h = C.c_void_p()
    assert _native.lib().fc_create(0, 5, 1.0, 0, C.byref(h)) == 1
    assert h.value is None
    assert _native.lib().fc_create(4, 4, -1.0, 0, C.byref(h)) == 1


def test_no_silent_host_fallback_without_gpu():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from fluidsim_b200 import FluidCudaError, FluidGrid

    with pytest.raises(FluidCudaError):
        FluidGrid(16, 16, 1.0)


@pytest.mark.skipif(shutil.which("g++") is None, reason="no host compiler")
def test_cpp_adapter_compiles_against_reference_contract(tmp_path):
    """include/FluidGridCUDA.h implements fluid::FluidGridBase from the reference headers."""
    reference = "/root/reference/FluidSim"
    if not os.path.isdir(reference):
        pytest.skip("reference headers not present")
    src = tmp_path / "adapter.cpp"
    src.write_text('#include "FluidGridCUDA.h"\nint main() { return fluid::FluidGridCUDA::kind() == 0; }\n')
    cmd = ["g++", "-std=c++23", "-fsyntax-only", f"-I{HEADER_DIR}", f"-I{reference}",
           f"-I{os.path.join(ROOT, 'oracle', 'ref_shim')}", str(src)]
    nlohmann = "/opt/prime-rl/.venv/lib/python3.12/site-packages/include/cudnn_frontend/thirdparty"
    if os.path.isdir(nlohmann):
        cmd.insert(2, f"-I{nlohmann}")
    out = subprocess.run(cmd, capture_output=True, text=True)
    assert out.returncode == 0, out.stderr[-2000:]

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
    assert lib.fc_abi_version() == 2
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
    from oracle import oracle

    checkout = oracle.reference_checkout()
    if checkout is None:
        pytest.skip("reference headers not present")
    reference = os.path.join(checkout, "FluidSim")
    src = tmp_path / "adapter.cpp"
    src.write_text('#include "FluidGridCUDA.h"\nint main() { return fluid::FluidGridCUDA::kind() == 0; }\n')
    cmd = ["g++", "-std=c++23", "-fsyntax-only", f"-I{HEADER_DIR}", f"-I{reference}",
           f"-I{os.path.join(ROOT, 'oracle', 'ref_shim')}", str(src)]
    nlohmann = oracle.json_include_dir()
    if nlohmann:
        cmd.insert(2, f"-I{nlohmann}")
    out = subprocess.run(cmd, capture_output=True, text=True)
    assert out.returncode == 0, out.stderr[-2000:]


def _prototypes():
    """extern "C" prototypes of include/fluidcuda.h: name -> (return type, [parameter types])."""
    import re

    text = open(os.path.join(os.path.dirname(__file__), "..", "include", "fluidcuda.h")).read()
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    text = re.sub(r"//[^\n]*", " ", text)
    out = {}
    for ret, name, params in re.findall(r"([A-Za-z_][\w \*]*?)\s*\b(fc_\w+)\s*\(([^;{]*?)\)\s*;", text):
        types = []
        for p in (q.strip() for q in params.split(",")):
            if not p or p == "void":
                continue
            p = re.sub(r"\s*\b\w+\s*(\[\s*\])?$", "", p) if not p.endswith("*") else p
            types.append(" ".join(p.replace("*", " * ").split()))
        out[name] = (" ".join(ret.replace("*", " * ").split()), types)
    return out


def _category(ctype_or_c):
    """A coarse ABI category shared by a C type name and a ctypes type."""
    import ctypes as C

    if isinstance(ctype_or_c, str):
        t = ctype_or_c.replace("const ", "")
        if "*" in t:
            return "pointer"
        return {"int": "int", "double": "double", "size_t": "size_t", "long long": "longlong"}.get(t, t)
    if ctype_or_c in (C.c_void_p, C.c_char_p) or hasattr(ctype_or_c, "contents") or \
            getattr(ctype_or_c, "_type_", None) is not None and issubclass(ctype_or_c, C._Pointer):
        return "pointer"
    return {C.c_int: "int", C.c_double: "double", C.c_size_t: "size_t", C.c_longlong: "longlong"}.get(ctype_or_c, "?")


def test_ctypes_signatures_match_the_header():
    """Every entry point the Python mirror binds has the header's return type and parameter
    categories (int, double, size_t, long long or pointer), so no argument is passed in the
    wrong register or width."""
    from fluidsim_b200 import _native as N

    protos = _prototypes()
    for name, (res, args) in N.SIGNATURES.items():
        assert name in protos, name
        ret, params = protos[name]
        assert len(params) == len(args), (name, params)
        for c_type, py_type in zip(params, args):
            assert _category(c_type) == _category(py_type), (name, c_type, py_type)
        assert _category(ret) == _category(res), (name, ret, res)

"""CPU: libbgt.so loads without a GPU and exports every entry point that
include/*.h declares (C ABI names and the drop-in C++ template
instantiations); no compute calls."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "begputhinning_b200", "libbgt.so")


def _exports():
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if line.strip()}


def _demangled():
    out = subprocess.run(["nm", "-D", "--defined-only", "-C", LIB], capture_output=True, text=True,
                         check=True).stdout
    return out


def test_library_loads():
    from begputhinning_b200 import lib
    L = lib()
    assert L.bgt_version() >= 100


def test_c_abi_exports_match_header():
    hdr = open(os.path.join(ROOT, "include", "bgt_capi.h")).read()
    names = set(re.findall(r"\b(bgt_[a-z0-9_]+)\s*\(", hdr))
    assert len(names) >= 25
    exp = _exports()
    missing = sorted(n for n in names if n not in exp)
    assert not missing, missing
    from begputhinning_b200._lib import EXPORTS
    assert set(EXPORTS) == names, sorted(set(EXPORTS) ^ names)


@pytest.mark.parametrize("sig", [
    "void Thinning2D<unsigned char>(int, int, unsigned char*, unsigned char*)",
    "void Thinning2D<double>(int, int, double*, double*)",
    "void Thinning2D<bool>(int, int, bool*, bool*)",
    "void Thinning3D<float>(int, int, int, float*, float*)",
    "void Thinning3D<unsigned short>(int, int, int, unsigned short*, unsigned short*)",
    "unsigned int CenterlineExtraction<float>(float*, int, int, int, int, float**, float**, unsigned int**)",
    "unsigned int CenterlineExtraction<signed char>(signed char*, int, int, int, int, int, float**, float**, "
    "float**, unsigned int**)",
])
def test_dropin_instantiations_exported(sig):
    assert sig in _demangled()


def test_dropin_instantiation_counts():
    d = _demangled()
    assert len(re.findall(r"void Thinning2D<", d)) == 10
    assert len(re.findall(r"void Thinning3D<", d)) == 8
    assert len(re.findall(r"CenterlineExtraction<", d)) == 20

"""CPU checks of the C-ABI library: it loads without a GPU and exports every
entry point declared in include/ibfs_capi.h (no compute calls here)."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def so_path():
    subprocess.check_call(["make", "-s", "-j8", "-C", os.path.join(ROOT, "ibfs-if2d_b200")])
    return os.path.join(ROOT, "ibfs-if2d_b200", "libibfs_b200.so")


def declared():
    text = open(os.path.join(ROOT, "include", "ibfs_capi.h")).read()
    return sorted(set(re.findall(r"\b(ibfs_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared()
    assert "ibfs_advance" in names and "ibfs_create" in names and len(names) >= 15


def test_library_exports_all(so_path):
    lib = ctypes.CDLL(so_path)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_matches_header(so_path):
    import ibfs_capi
    assert sorted(ibfs_capi.EXPORTS) == declared()


def test_kernels_are_sm100a(so_path):
    out = subprocess.run(["cuobjdump", "--list-elf", so_path], capture_output=True, text=True).stdout
    assert "sm_100a" in out

"""The C-ABI library loads and exports every entry point include/*.h declares (CPU, no compute)."""
import ctypes
import glob
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    txt = "".join(open(p).read() for p in sorted(glob.glob(os.path.join(ROOT, "include", "*.h"))))
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(smr_[a-z_0-9]+)\s*\(", txt)))


def test_header_declares_entry_points():
    names = declared()
    assert "smr_create" in names and "smr_run_fire" in names and len(names) >= 25


def test_library_exports_every_declared_symbol(native):
    L = native.lib()
    missing = [n for n in declared() if not hasattr(L, n)]
    assert not missing, missing


def test_binding_covers_header(native):
    assert set(declared()) == set(native.SIGNATURES)


def test_version_string(native):
    assert b"sm_100a" in native.lib().smr_version()


def test_no_cpu_fallback_symbols(native):
    """The library has no host compute path for forces: no symbol of the oracle is linked in."""
    L = native.lib()
    for n in ["orc_eval", "orc_relax", "orc_sys_from_molecule"]:
        assert not hasattr(L, n)

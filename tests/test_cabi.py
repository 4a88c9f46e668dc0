"""The C-ABI library loads and exports every entry point declared in include/*.h
(no GPU needed: nothing is called that touches the device)."""
import ctypes
import glob
import os
import re

from palzilla_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        names |= set(re.findall(r"PZ_API\s+[\w\s\*]+?\b(pz_\w+)\s*\(", src))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "pz_onesweep_sort" in names and "pz_bvh_build" in names


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_symbols() if not hasattr(L, n)]
    assert not missing, f"not exported: {missing}"


def test_binding_signatures_cover_header():
    assert set(declared_symbols()) <= set(_lib.SIGNATURES)


def test_host_side_argument_checks():
    """Argument validation runs on the host and never reaches the device."""
    L = _lib.lib()
    import ctypes as C
    r = L.pz_onesweep_sort(None, None, None, None, C.c_uint32(10), 3, 0, 32, None, C.c_size_t(0), None)
    assert r == 1 and b"key_bytes" in L.pz_last_error()
    r = L.pz_onesweep_sort(None, None, None, None, C.c_uint32(10), 8, 0, 32, None, C.c_size_t(0), None)
    assert r == 1
    r = L.pz_bvh_build(None, -1, 0, None, None, None, C.c_size_t(0), None)
    assert r == 1
    assert L.pz_onesweep_scratch_bytes(1 << 20) > 0
    # the PathCache buffer starts on a 16-byte boundary with a power-of-two capacity; the
    # views call only computes addresses, so a made-up device address is enough here
    hp = C.c_void_p()
    r = L.pz_path_cache_views(C.c_void_p(0x10000), C.c_uint32(1 << 10), C.byref(hp), None, None, None, None, None)
    assert r == 0 and hp.value == 0x10000 + 256 + 48 * (1 << 10)
    r = L.pz_path_cache_views(C.c_void_p(0x10004), C.c_uint32(1 << 10), None, None, None, None, None, None)
    assert r == 1 and b"pz_path_cache_views" in L.pz_last_error()
    r = L.pz_path_cache_views(C.c_void_p(0x10000), C.c_uint32(3), None, None, None, None, None, None)
    assert r == 1
    assert L.pz_path_cache_bytes(C.c_uint32(3)) == 0 and L.pz_path_cache_bytes(C.c_uint32(4)) > 0

"""pz_onesweep_sort_static (sort on the library's static device scratch) against
pz_onesweep_sort (caller-owned scratch): two different sorts in a row on one stream must
both match the caller-scratch results bit for bit, and an oversize request is refused
before any device work.  Collected last, so it also runs after the other GPU tests have
used the device."""
import ctypes as C

import numpy as np
import pytest
import torch

from palzilla_b200 import _lib

pytestmark = pytest.mark.gpu

MAX_KEYS = 1 << 22


def _dev(a):
    return torch.from_numpy(a.view(np.int64 if a.dtype == np.uint64 else np.int32)).cuda()


def _p(t):
    return C.c_void_p(None if t is None else t.data_ptr())


def _caller_scratch_sort(keys, values, start, end):
    L = _lib.lib()
    k, tk = _dev(keys), torch.empty(keys.size, dtype=torch.int64 if keys.dtype == np.uint64 else torch.int32,
                                   device="cuda")
    v = _dev(values) if values is not None else None
    tv = torch.empty_like(v) if v is not None else None
    scratch = torch.empty(L.pz_onesweep_scratch_bytes(keys.size), dtype=torch.uint8, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    r = L.pz_onesweep_sort(_p(k), _p(v), _p(tk), _p(tv), C.c_uint32(keys.size), keys.itemsize, start, end,
                           _p(scratch), C.c_size_t(scratch.numel()), C.c_void_p(s))
    assert r == 0, L.pz_last_error()
    torch.cuda.synchronize()
    return k.cpu().numpy().view(keys.dtype), (None if v is None else v.cpu().numpy().view(np.uint32))


def test_static_scratch_matches_caller_scratch_twice_in_a_row():
    L = _lib.lib()
    rng = np.random.default_rng(2024)
    n1 = (1 << 20) + 4097
    keys1 = rng.integers(0, 1 << 32, n1, dtype=np.uint64) | (np.arange(n1, dtype=np.uint64) << np.uint64(32))
    n2 = MAX_KEYS
    keys2 = rng.integers(0, 1 << 24, n2, dtype=np.uint32)
    vals2 = rng.integers(0, 1 << 32, n2, dtype=np.uint32)
    exp1, _ = _caller_scratch_sort(keys1, None, 0, 32)
    exp2, expv2 = _caller_scratch_sort(keys2, vals2, 0, 24)

    k1, tk1 = _dev(keys1), torch.empty(n1, dtype=torch.int64, device="cuda")
    k2, tk2 = _dev(keys2), torch.empty(n2, dtype=torch.int32, device="cuda")
    v2, tv2 = _dev(vals2), torch.empty(n2, dtype=torch.int32, device="cuda")
    status = torch.full((2,), -1, dtype=torch.int32, device="cuda")
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    r1 = L.pz_onesweep_sort_static(_p(k1), None, _p(tk1), None, C.c_uint32(n1), 8, 0, 32,
                                   C.c_void_p(status.data_ptr()), s)
    assert r1 == 0, L.pz_last_error()
    r2 = L.pz_onesweep_sort_static(_p(k2), _p(v2), _p(tk2), _p(tv2), C.c_uint32(n2), 4, 0, 24,
                                   C.c_void_p(status.data_ptr() + 4), s)
    assert r2 == 0, L.pz_last_error()
    torch.cuda.synchronize()
    assert status.cpu().tolist() == [0, 0]
    assert np.array_equal(k1.cpu().numpy().view(np.uint64), exp1)
    assert np.array_equal(k2.cpu().numpy().view(np.uint32), exp2)
    assert np.array_equal(v2.cpu().numpy().view(np.uint32), expv2)


def test_static_scratch_rejects_oversize_before_device_work():
    L = _lib.lib()
    keys = torch.arange(16, dtype=torch.int64, device="cuda")
    before = keys.clone()
    tmp = torch.empty_like(keys)
    r = L.pz_onesweep_sort_static(_p(keys), None, _p(tmp), None, C.c_uint32(MAX_KEYS + 1), 8, 0, 32, None,
                                  C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert r == 2  # PZ_ERR_SCRATCH_TOO_SMALL
    assert b"static scratch capacity" in L.pz_last_error()
    torch.cuda.synchronize()
    assert torch.equal(keys, before)

"""pz_onesweep_sort_static (sort on the library's static device scratch) against
pz_onesweep_sort (caller-owned scratch), for callers that cannot allocate device memory:
two different sorts in a row on one stream must both match the caller-scratch results bit
for bit; after the first call, further calls must leave the device's free memory
unchanged; a sort in a second CUDA context (made with the driver API, as a plug-in host
that owns its context would) must use that context's copy of the array; and an oversize
request is refused before any device work.  Collected last, so it also runs after the
other GPU tests have used the device."""
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


def test_static_scratch_allocates_nothing_after_the_first_call():
    L = _lib.lib()
    rng = np.random.default_rng(7)
    n = 1 << 21
    keys = rng.integers(0, 1 << 32, n, dtype=np.uint64)
    k, tk = _dev(keys), torch.empty(n, dtype=torch.int64, device="cuda")
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert L.pz_onesweep_sort_static(_p(k), None, _p(tk), None, C.c_uint32(n), 8, 0, 32, None, s) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        k.copy_(_dev(keys))
        assert L.pz_onesweep_sort_static(_p(k), None, _p(tk), None, C.c_uint32(n), 8, 0, 32, None, s) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    order = np.argsort(keys & np.uint64(0xFFFFFFFF), kind="stable")
    assert np.array_equal(k.cpu().numpy().view(np.uint64), keys[order])


def test_static_scratch_in_a_second_context():
    """A host that runs the library in a context of its own: the array's address is looked
    up in that context, not reused from the primary context of the same device."""
    from cuda.bindings import driver as D

    def ok(r):
        err = r[0] if isinstance(r, tuple) else r
        assert err == D.CUresult.CUDA_SUCCESS, err
        return r[1] if isinstance(r, tuple) and len(r) == 2 else r

    L = _lib.lib()
    torch.cuda.synchronize()  # the primary context exists and is current
    n = (1 << 20) + 333
    keys = np.random.default_rng(11).integers(0, 1 << 32, n, dtype=np.uint64)
    dev = ok(D.cuDeviceGet(torch.cuda.current_device()))
    mode = ok(D.cuDeviceGetAttribute(D.CUdevice_attribute.CU_DEVICE_ATTRIBUTE_COMPUTE_MODE, dev))
    if int(mode) != int(D.CUcomputemode.CU_COMPUTEMODE_DEFAULT):
        pytest.skip(f"compute mode {mode} allows one context per device")
    ctx = ok(D.cuCtxCreate(0, dev))
    bufs = []
    try:
        kd = ok(D.cuMemAlloc(8 * n))
        bufs.append(kd)
        td = ok(D.cuMemAlloc(8 * n))
        bufs.append(td)
        sd = ok(D.cuMemAlloc(4))
        bufs.append(sd)
        ok(D.cuMemcpyHtoD(kd, keys.ctypes.data, 8 * n))
        ok(D.cuMemsetD32(sd, 0xFFFFFFFF, 1))
        r = L.pz_onesweep_sort_static(C.c_void_p(int(kd)), None, C.c_void_p(int(td)), None, C.c_uint32(n), 8, 0, 32,
                                      C.c_void_p(int(sd)), None)
        assert r == 0, L.pz_last_error()
        ok(D.cuCtxSynchronize())
        got = np.empty(n, np.uint64)
        st = np.empty(1, np.uint32)
        ok(D.cuMemcpyDtoH(got.ctypes.data, kd, 8 * n))
        ok(D.cuMemcpyDtoH(st.ctypes.data, sd, 4))
    finally:
        for b in bufs:
            D.cuMemFree(b)
        ok(D.cuCtxDestroy(ctx))
    order = np.argsort(keys & np.uint64(0xFFFFFFFF), kind="stable")
    assert int(st[0]) == 0
    assert np.array_equal(got, keys[order])
    # the primary context is current again and still sorts on its own copy of the array
    k, tk = _dev(keys), torch.empty(n, dtype=torch.int64, device="cuda")
    assert L.pz_onesweep_sort_static(_p(k), None, _p(tk), None, C.c_uint32(n), 8, 0, 32, None,
                                     C.c_void_p(torch.cuda.current_stream().cuda_stream)) == 0
    torch.cuda.synchronize()
    assert np.array_equal(k.cpu().numpy().view(np.uint64), keys[order])

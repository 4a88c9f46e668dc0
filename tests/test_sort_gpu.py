"""Onesweep sort parity: GPU result bit-exact with a stable CPU sort (the oracle).

Mirrors how the reference uses OnesweepSort::sort (tinyhiponesweep.h:592-668): u64
IndexedMorton elements sorted on bits [0, 32) (minimum_lbvh.h:848, pk.h:1526), plus the
32-bit and key/value variants and ragged bit ranges.
"""
import numpy as np
import pytest
import torch

from palzilla_b200.api import OnesweepSort

pytestmark = pytest.mark.gpu

SIZES = [1, 2, 31, 255, 4095, 4096, 4097, 3 * 4096 + 1, 5119, 5120, 5121, 3 * 5120 + 1, 65536 + 17, 1 << 20]


def _to_dev(a):
    if a.dtype == np.uint64:
        return torch.from_numpy(a.view(np.int64)).cuda()
    return torch.from_numpy(a.view(np.int32)).cuda()


def _from_dev(t, dtype):
    return t.cpu().numpy().view(dtype)


def _sort(keys, values=None, start=0, end=32):
    s = OnesweepSort()
    k = _to_dev(keys)
    tk = torch.empty_like(k)
    v = _to_dev(values) if values is not None else None
    tv = torch.empty_like(v) if v is not None else None
    s.sort(k, v, tk, tv, keys.size, start, end)
    torch.cuda.synchronize()
    assert s.status() == 0
    return _from_dev(k, keys.dtype), (None if v is None else _from_dev(v, np.uint32))


@pytest.mark.parametrize("n", SIZES)
def test_indexed_morton_u64(orc, n):
    rng = np.random.default_rng(n)
    morton = rng.integers(0, 1 << 32, n, dtype=np.uint64)
    keys = morton | (np.arange(n, dtype=np.uint64) << np.uint64(32))
    got, _ = _sort(keys)
    exp = orc.stable_sort_u64(keys, 0, 32)
    assert np.array_equal(got, exp)


@pytest.mark.parametrize("n", [4097, 200_003])
@pytest.mark.parametrize("distinct", [1, 2, 17, 256])
def test_duplicates_stable(orc, n, distinct):
    rng = np.random.default_rng(distinct)
    morton = rng.integers(0, distinct, n, dtype=np.uint64) * np.uint64(0x01010101)
    keys = morton | (np.arange(n, dtype=np.uint64) << np.uint64(32))
    got, _ = _sort(keys)
    assert np.array_equal(got, orc.stable_sort_u64(keys, 0, 32))


@pytest.mark.parametrize("n", [4096 * 5 + 3, 1 << 18])
def test_u32_keys(orc, n):
    keys = np.random.default_rng(7).integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
    got, _ = _sort(keys)
    assert np.array_equal(got, orc.stable_sort_u32(keys, 0, 32))


@pytest.mark.parametrize("kb", [4, 8])
@pytest.mark.parametrize("bits", [(0, 32), (3, 21), (8, 16), (5, 13)])
def test_key_value_ranges(orc, kb, bits):
    n = 100_001
    rng = np.random.default_rng(kb * 100 + bits[0])
    keys = rng.integers(0, 1 << 32, n, dtype=np.uint64)
    if kb == 4:
        keys = keys.astype(np.uint32)
    vals = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
    gk, gv = _sort(keys, vals, *bits)
    ek, ev = orc.stable_sort_kv(keys, vals, *bits)
    assert np.array_equal(gk, ek)
    assert np.array_equal(gv, ev)


def test_presorted_and_reversed(orc):
    n = 50_000
    for keys in (np.arange(n, dtype=np.uint32), np.arange(n, dtype=np.uint32)[::-1].copy()):
        got, _ = _sort(keys)
        assert np.array_equal(got, orc.stable_sort_u32(keys, 0, 32))


def test_full_size_properties():
    """2^24 IndexedMorton elements (the largest sort + build config): sortedness,
    permutation and stability checked through size-independent properties."""
    n = 1 << 24
    g = torch.Generator(device="cuda").manual_seed(5)
    morton = torch.randint(0, 1 << 31, (n,), device="cuda", generator=g, dtype=torch.int64)
    keys = morton | (torch.arange(n, device="cuda", dtype=torch.int64) << 32)
    tmp = torch.empty_like(keys)
    s = OnesweepSort()
    s.sort(keys, None, tmp, None, n, 0, 32)
    torch.cuda.synchronize()
    assert s.status() == 0
    m = keys & 0xFFFFFFFF
    idx = keys >> 32
    assert bool((m[1:] >= m[:-1]).all())
    same = m[1:] == m[:-1]
    assert bool((idx[1:][same] > idx[:-1][same]).all())
    assert bool((torch.sort(idx).values == torch.arange(n, device="cuda")).all())
    assert bool((morton[idx] == m).all())


def test_empty_is_noop():
    s = OnesweepSort()
    k = torch.zeros(4, dtype=torch.int64, device="cuda")
    s.sort(k, None, torch.empty_like(k), None, 0, 0, 32)
    torch.cuda.synchronize()

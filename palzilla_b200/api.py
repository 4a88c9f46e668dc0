"""Python mirror of the reference's host classes over the C ABI.

``OnesweepSort`` and ``BVHGPUBuilder`` keep the reference's class names, method
names and argument meaning (tinyhiponesweep.h:572-668, minimum_lbvh.h:741-900) so
that tests read like code written against the reference.  Device memory is held
in torch tensors (torch is used only as an allocator and for streams); every
computation runs in libpalzilla_b200.so.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib

NODE_BYTES = 64


def _stream(stream) -> int:
    if stream is None:
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def _ptr(t) -> int | None:
    return None if t is None else t.data_ptr()


class Scratch:
    """Grow-only device scratch buffer."""

    def __init__(self, device="cuda"):
        self.device = device
        self.buf = None

    def get(self, nbytes: int) -> torch.Tensor:
        if self.buf is None or self.buf.numel() < nbytes:
            self.buf = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=self.device)
        return self.buf

    def status(self, stream=None) -> int:
        st = C.c_uint32(0)
        _lib.call("pz_scratch_status", C.c_void_p(self.buf.data_ptr()), C.byref(st), C.c_void_p(_stream(stream)))
        return st.value


class OnesweepSort:
    """tinyhiponesweep::OnesweepSort (tinyhiponesweep.h:572-668).

    ``sort(keys, values, tmp_keys, tmp_values, n, start_bit, end_bit, stream)`` sorts
    ``keys`` (uint32 or 64-bit tensor) stably on [start_bit, end_bit); ``values``
    (uint32/int32 tensor or None) follow their keys.  The result ends in
    ``keys``/``values``; the tmp tensors are ping-pong storage of equal size.
    """

    def __init__(self, device="cuda"):
        self.scratch = Scratch(device)

    def sort(self, keys, values, tmp_keys, tmp_values, n: int, start_bit: int, end_bit: int, stream=None):
        kb = keys.element_size()
        nbytes = _lib.lib().pz_onesweep_scratch_bytes(n)
        buf = self.scratch.get(nbytes)
        _lib.call("pz_onesweep_sort", C.c_void_p(keys.data_ptr()), C.c_void_p(_ptr(values)),
                  C.c_void_p(tmp_keys.data_ptr()), C.c_void_p(_ptr(tmp_values)), C.c_uint32(n), C.c_int(kb),
                  C.c_int(start_bit), C.c_int(end_bit), C.c_void_p(buf.data_ptr()), C.c_size_t(buf.numel()),
                  C.c_void_p(_stream(stream)))

    def status(self, stream=None) -> int:
        return self.scratch.status(stream)


class BVHGPUBuilder:
    """minimum_lbvh::BVHGPUBuilder (minimum_lbvh.h:741-900).

    ``build(triangles, n, build_option, sorter, stream)``: ``triangles`` is a float32
    cuda tensor of shape (n, 9) (the 36-byte Triangle layout).  Afterwards
    ``m_internals`` (uint8 tensor of (n-1) * 64 bytes), ``m_rootNode`` (uint32 tensor
    of one element) and ``m_nTriangles`` hold the tree, as in the reference.  The
    ``sorter`` argument is accepted for signature compatibility; the builder runs its
    own fused sort on its own scratch.
    """

    def __init__(self, device="cuda"):
        self.device = device
        self.scratch = Scratch(device)
        self.m_internals = None
        self.m_rootNode = torch.zeros(1, dtype=torch.int32, device=device)
        self.m_nTriangles = 0

    def build(self, triangles, n: int, build_option: int = 0, sorter=None, stream=None):
        self.m_nTriangles = n
        nbytes = max(n - 1, 1) * NODE_BYTES
        if self.m_internals is None or self.m_internals.numel() < nbytes:
            self.m_internals = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        buf = self.scratch.get(_lib.lib().pz_bvh_scratch_bytes(n))
        _lib.call("pz_bvh_build", C.c_void_p(triangles.data_ptr()), C.c_int(n), C.c_uint32(build_option),
                  C.c_void_p(self.m_internals.data_ptr()), C.c_void_p(self.m_rootNode.data_ptr()),
                  C.c_void_p(buf.data_ptr()), C.c_size_t(buf.numel()), C.c_void_p(_stream(stream)))

    def empty(self) -> bool:
        return self.m_nTriangles == 0

    @property
    def root(self) -> int:
        return int(self.m_rootNode.item()) & 0xFFFFFFFF

    def debug_views(self, stream=None):
        """(sorted u64 {morton, index} tensor view, deltas u8 view, scene AABB (6 floats))."""
        n = self.m_nTriangles
        sp, dp = C.c_void_p(), C.c_void_p()
        aabb = (C.c_float * 6)()
        _lib.call("pz_bvh_debug_views", C.c_void_p(self.scratch.buf.data_ptr()), C.c_int(n), C.byref(sp),
                  C.byref(dp), C.cast(aabb, C.c_void_p), C.c_void_p(_stream(stream)))
        base = self.scratch.buf.data_ptr()
        so = sp.value - base
        do = dp.value - base
        sorted_ = self.scratch.buf[so:so + 8 * n].view(torch.int64)
        deltas = self.scratch.buf[do:do + max(n - 1, 0)]
        return sorted_, deltas, list(aabb)

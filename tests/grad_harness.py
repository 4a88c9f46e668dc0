"""Gradient-check harness for the adjoint pair (pz_adjoint_forward / pz_adjoint_backward):
a torch.autograd.Function over the C ABI, used only by the gradient tests.

The rendered function is the binned caustic image of a heightfield lens whose vertex
heights and Cauchy coefficients (A, B) are the parameters.  The work list (pixels, tuples,
photon start barycentrics) is computed once at the initial geometry and then held fixed,
so the image is a piecewise-smooth function of the parameters; every forward and
backward rebuilds the triangles and the LBVH (visibility) from the current heights.
"""
import ctypes as C

import numpy as np
import torch

from palzilla_b200 import _lib
from palzilla_b200 import api as A
from palzilla_b200 import scenes as S


class CausticProblem:
    def __init__(self, sc, corners, iteration: int = 0, path_capacity: int = 1 << 25):
        self.sc = sc
        self.K = len(sc.events)
        self.ds = A.DeviceScene(sc)
        self.base_tris = self.ds.tris.clone()
        self.corners = torch.from_numpy(corners).cuda()
        self.mask = self.corners >= 0
        self.frame = A.Frame(sc, path_capacity=path_capacity)
        A.solve_primary(self.ds, self.frame, iteration=iteration)
        self.cache = A.PathCache(capacity=1 << 22, step=sc.cell_step)
        A.photon_trace(self.ds, self.cache, iteration=iteration)
        self.n_paths = A.lookup_flatten(self.frame, self.cache, S.event_descriptor(sc.events))
        A.sort_and_reorder(self.frame, self.n_paths, A.OnesweepSort())
        self.lambdas = torch.from_numpy(sc.bin_lambdas().astype(np.float32)).cuda()
        self.scratch = None

    def set_heights(self, heights):
        tris = self.base_tris.clone().view(-1, 3, 3)
        y = tris[:, :, 1]
        y[self.mask] = heights[self.corners[self.mask].long()]
        self.ds.tris.copy_(tris.view(-1, 9))
        self.ds.builder.build(self.ds.tris, self.ds.n, 0)

    def desc(self, cauchy, spectral, etas):
        d = A.solve_desc(self.ds, self.frame, self.cache, self.sc.events, self.n_paths, spectral=spectral, etas=etas)
        d.cauchy_a = float(cauchy[0])
        d.cauchy_b = float(cauchy[1])
        return d

    def etas(self, cauchy):
        return (cauchy[0] + cauchy[1] / (self.lambdas * self.lambdas)).float().contiguous()

    def forward(self, heights, cauchy):
        self.set_heights(heights)
        spectral = torch.zeros((self.sc.width * self.sc.height, self.sc.n_bins), device="cuda")
        etas = self.etas(cauchy)
        d = self.desc(cauchy, spectral, etas)
        _lib.call("pz_adjoint_forward", C.byref(d), C.c_void_p(torch.cuda.current_stream().cuda_stream))
        return spectral

    def backward(self, heights, cauchy, grad_spectral, compact: bool = True):
        """dL/dheights and dL/d(A, B).  compact: pz_adjoint_backward_compact (filter, then
        differentiate the accepted paths); else the one-kernel pz_adjoint_backward."""
        self.set_heights(heights)
        spectral = torch.zeros(1, device="cuda")
        etas = self.etas(cauchy)
        d = self.desc(cauchy, spectral, etas)
        gh = torch.zeros_like(heights)
        gc = torch.zeros(2, dtype=torch.float32, device="cuda")
        stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        if compact:
            nbytes = _lib.lib().pz_adjoint_scratch_bytes(self.n_paths * self.sc.n_bins)
            if self.scratch is None or self.scratch.numel() < nbytes:
                self.scratch = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
            _lib.call("pz_adjoint_backward_compact", C.byref(d), A._vp(grad_spectral), A._vp(self.corners),
                      A._vp(gh), A._vp(gc), A._vp(self.scratch), C.c_size_t(self.scratch.numel()), stream)
        else:
            _lib.call("pz_adjoint_backward", C.byref(d), A._vp(grad_spectral), A._vp(self.corners), A._vp(gh),
                      A._vp(gc), stream)
        return gh, gc


class CausticRender(torch.autograd.Function):
    @staticmethod
    def forward(ctx, heights, cauchy, problem):
        ctx.problem = problem
        ctx.save_for_backward(heights, cauchy)
        return problem.forward(heights, cauchy)

    @staticmethod
    def backward(ctx, grad_spectral):
        heights, cauchy = ctx.saved_tensors
        gh, gc = ctx.problem.backward(heights, cauchy, grad_spectral.contiguous())
        return gh, gc.to(cauchy.dtype), None

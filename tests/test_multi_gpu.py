"""Batches of scenes (pz_solve_multi_prepare / pz_solve_specular_multi /
pz_solve_multi_autotune): an uneven batch of heightfield lenses (grid side log-uniform in
16..96, 1-2 refractions) solved in one set of launches gives every scene the image its own
batched solve gives (up to the order of the float atomics), with host or device item
counts, under the autotuner's choice, and when the frame is captured in a CUDA graph and
replayed."""
import numpy as np
import pytest
import torch

from palzilla_b200 import api as A
from palzilla_b200 import scenes as S

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a, b = a.double(), b.double()
    return float(torch.sqrt(((a - b) ** 2).mean()) / torch.sqrt((b ** 2).mean()).clamp_min(1e-30))


class Item:
    def __init__(self, sc):
        self.sc = sc
        self.ds = A.DeviceScene(sc)
        self.frame = A.Frame(sc, path_capacity=1 << 20)
        self.cache = A.PathCache(capacity=1 << 20, step=sc.cell_step)
        A.solve_primary(self.ds, self.frame, iteration=0)
        A.photon_trace(self.ds, self.cache, iteration=0)
        self.n = A.lookup_flatten(self.frame, self.cache, S.event_descriptor(sc.events))
        self.etas = torch.from_numpy(sc.bin_etas()).cuda()
        self.spectral = torch.zeros((sc.width * sc.height, sc.n_bins), device="cuda")

    def desc(self, capacity=False):
        return A.solve_desc(self.ds, self.frame, self.cache, self.sc.events,
                            self.frame.path_capacity if capacity else self.n, spectral=self.spectral, etas=self.etas)


@pytest.fixture(scope="module")
def batch():
    scenes = S.uneven_batch(n_scenes=12, seed=3001, side_min=16, side_max=96, width=64, height=64, n_bins=8,
                            photons_per_triangle=64)
    items = [Item(sc) for sc in scenes]
    ref = []
    for it in items:
        it.spectral.zero_()
        A.solve_specular_batched(it.desc(), A.Scratch())
        torch.cuda.synchronize()
        ref.append(it.spectral.clone())
    return items, ref


def test_single_scene_solves_repeat(batch):
    """Each scene's batched solve, run again on fresh scratch, gives the same image (up to the
    order of the float atomics) and a clean status word.  The batch holds scenes whose items
    are nearly all solved bin by bin (so their records fill every phase-2 wave) and scenes
    that are mostly predicted."""
    items, ref = batch
    modes = []
    for i, it in enumerate(items):
        it.spectral.zero_()
        scratch = A.Scratch()
        A.solve_specular_batched(it.desc(), scratch)
        torch.cuda.synchronize()
        assert _rel(it.spectral, ref[i]) <= 1e-6, i
        assert scratch.status() == 0, i
        c = A.batched_counters(scratch)
        modes.append(c["fallback"] / max(1, c["skipped"] + c["predicted"] + c["fallback"]))
    assert max(modes) > 0.9 and min(modes) < 0.1, modes


@pytest.mark.parametrize("K", [1, 2])
@pytest.mark.parametrize("device_counts", [False, True])
def test_batch_matches_single_scene_solves(batch, K, device_counts):
    items, ref = batch
    group = [(i, it) for i, it in enumerate(items) if len(it.sc.events) == K]
    assert len(group) >= 2
    for _, it in group:
        it.spectral.zero_()
    sb = A.SceneBatch([it.desc(capacity=device_counts) for _, it in group],
                      counts=[it.frame.counter for _, it in group] if device_counts else None)
    stats = torch.zeros(3, dtype=torch.int64, device="cuda")
    sb.solve(stats=stats)
    torch.cuda.synchronize()
    assert int(stats[0].item()) == sum(it.n for _, it in group) * items[0].sc.n_bins
    for i, it in group:
        assert _rel(it.spectral, ref[i]) <= 1e-6, i
    assert int(sb.scratch[:4].view(torch.int32).item()) == 0  # status word


def test_autotune_and_graph_replay(batch):
    items, ref = batch
    group = [(i, it) for i, it in enumerate(items) if len(it.sc.events) == 1]
    sb = A.SceneBatch([it.desc() for _, it in group])
    tuning, ms = sb.autotune()
    assert ms > 0 and tuning[0] in (4, 8, 16) and tuning[1] in (1, 2) and tuning[2] in (1, 4)
    stream = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        with torch.cuda.graph(g, stream=stream):
            for _, it in group:
                it.spectral.zero_()
            sb.solve(stream=stream)  # tuning from the autotuner's cache
    for _ in range(2):
        g.replay()
        torch.cuda.synchronize()
        for i, it in group:
            assert _rel(it.spectral, ref[i]) <= 1e-6, i

"""Structural checks of a PathCache table (hash and cell-hash arrays), shared by the CPU
oracle tests and the GPU tests.

Linear probing from the cell hash's home slot (PathCache::store, pk.h:313-345) never
empties a slot, so every stored entry is reachable from its home slot through occupied
slots only: the run of occupied slots that ends at the entry is longer than the entry's
distance from home.  A probe that skipped an empty slot, or stored past one, breaks it."""
import numpy as np


def probe_reachability_violations(hash_, cell, capacity):
    """Number of stored slots that sit behind an empty slot on their own probe chain."""
    hash_ = np.asarray(hash_, np.uint32)
    cell = np.asarray(cell, np.uint32)
    mask = np.uint32(capacity - 1)
    used = hash_ != 0
    if used.all():
        return 0  # a full table has no empty slot to sit behind
    # run[i] = occupied slots ending at i (circular), from the last empty slot at or before i
    n = capacity
    pos = np.arange(2 * n)
    u2 = np.concatenate([used, used])
    last_empty = np.maximum.accumulate(np.where(~u2, pos, -1))
    run = (pos - last_empty)[n:]
    idx = np.nonzero(used)[0].astype(np.uint32)
    dist = (idx - (cell[idx] & mask)) & mask
    return int(np.count_nonzero(run[idx] < dist.astype(np.int64) + 1))

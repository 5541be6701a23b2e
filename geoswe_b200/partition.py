"""Where a 1 x N (or N x 1) strip split cuts the split axis.

Mirrors ``strip_bounds`` of the reference (geoswe/partition.py:20-65): rank ``r`` owns
the columns ``bnd[r]:bnd[r + 1]``; each rank's share of the total work is its weight
over the weights' sum, met as closely as whole columns allow (ties go to the lower
boundary), and no rank is left without a column. The solution does not depend on the
cuts (a ghost cell is an exact copy of the neighbour's cell), only the time per rank.

Host code, NumPy only.
"""
from __future__ import annotations

import numpy as np

__all__ = ["strip_bounds", "block_of", "members_of"]


def _shares(n_ranks, weights):
    if weights is None:
        w = np.ones(n_ranks)
    else:
        w = np.asarray(weights, dtype=np.float64).reshape(-1)
    if w.size != n_ranks:
        raise ValueError(f"strip_bounds: {w.size} weights for {n_ranks} ranks")
    if not bool(np.all(np.isfinite(w))) or not bool(np.all(w > 0.0)):
        raise ValueError(f"strip_bounds: weights must be positive and finite, got {w.tolist()}")
    # work share reached after each rank but the last
    return np.cumsum(w)[:-1] / w.sum()


def strip_bounds(col_work, n_ranks, weights=None):
    """Boundaries of a strip split: ``n_ranks + 1`` increasing integers from 0.

    ``col_work`` is the work of each column (an array; for the compressed mesh, its
    active cells per column) or an integer count of columns of equal work. ``weights``
    holds one positive relative speed per rank (``None``: equal shares)."""
    n_ranks = int(n_ranks)
    if n_ranks < 1:
        raise ValueError(f"strip_bounds: n_ranks must be at least 1, got {n_ranks}")
    share = _shares(n_ranks, weights)
    if np.ndim(col_work) == 0:
        ncol = int(col_work)
        cuts = np.rint(share * ncol).astype(np.int64)
    else:
        work = np.asarray(col_work, dtype=np.float64).reshape(-1)
        if not bool(np.all(np.isfinite(work))) or not bool(np.all(work >= 0.0)):
            raise ValueError("strip_bounds: col_work must be non-negative and finite")
        ncol = work.size
        before = np.zeros(ncol + 1)
        np.cumsum(work, out=before[1:])           # before[c] = work of the columns [0, c)
        goal = share * before[-1]
        above = np.minimum(np.searchsorted(before, goal, side="left"), ncol)
        below = np.maximum(above - 1, 0)
        nearer_below = (goal - before[below]) <= (before[above] - goal)
        cuts = np.where(nearer_below, below, above)
    if ncol < n_ranks:
        raise ValueError(f"strip_bounds: {ncol} columns cannot be split among {n_ranks} ranks")
    bnd = [0, *(int(c) for c in cuts), ncol]
    for r in range(1, n_ranks):                   # at least one column each: forwards ...
        if bnd[r] < bnd[r - 1] + 1:
            bnd[r] = bnd[r - 1] + 1
    for r in range(n_ranks - 1, 0, -1):           # ... then back from the fixed last boundary
        if bnd[r] > bnd[r + 1] - 1:
            bnd[r] = bnd[r + 1] - 1
    return bnd


def members_of(member_work, n_ranks, rank, weights=None):
    """The ensemble members (a contiguous ``range`` of member indices) that ``rank``
    advances when an ensemble is spread over ``n_ranks`` GPUs: members are independent,
    so each rank runs its share as its own ``Ensemble`` and nothing is exchanged.
    ``member_work`` is each member's work (its active cells, say) or a member count."""
    bnd = strip_bounds(member_work, n_ranks, weights)
    rank = int(rank)
    if not 0 <= rank < int(n_ranks):
        raise ValueError(f"members_of: rank {rank} outside 0..{int(n_ranks) - 1}")
    return range(bnd[rank], bnd[rank + 1])


def block_of(nx, ny, dims, coords, x_work=None, y_work=None):
    """The (x0, x1, y0, y1) block of the global ``nx x ny`` grid that the rank at
    ``coords`` of a ``dims`` Cartesian layout owns, each axis cut by ``strip_bounds``
    (equal columns unless per-row / per-column work is given)."""
    px, py = int(dims[0]), int(dims[1])
    cx, cy = int(coords[0]), int(coords[1])
    bx = strip_bounds(nx if x_work is None else x_work, px)
    by = strip_bounds(ny if y_work is None else y_work, py)
    return bx[cx], bx[cx + 1], by[cy], by[cy + 1]

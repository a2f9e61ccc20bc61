"""Walk sharding across ranks (one process per GPU).

Walks are independent, so the layout is replicated and rank r runs its walks
on Philox stream r (weak scaling: every rank runs the same walk count).  The
only exchange is one sum of the per-conductor rows (hits, sum w, sum w^2) and
of the scalar totals: either dense (one all-reduce of 3*n + 4 numbers,
`dense_rows` / `all_reduce_rows`) or sparse (each rank's nonzero rows only,
one all-gather, `sparse_buffer` .. `merge_sparse`).  The reference is
single-GPU; this module has no counterpart there.
"""
from __future__ import annotations

import numpy as np


def plan(walks_per_rank: int, rank: int) -> dict:
    """Walk range and Philox stream of `rank`."""
    return {"first": 0, "count": int(walks_per_rank), "stream": int(rank)}


def dense_rows(n_conductors: int, conductor, hits, sum_w, sum_w2, walks: int, escaped: int,
               hops: int) -> np.ndarray:
    """Pack one rank's result into a (3*n + 4,) float64 vector:
    [hits_k | sum_k w | sum_k w^2 | walks, escaped, hops, 0]."""
    v = np.zeros(3 * n_conductors + 4)
    c = np.asarray(conductor, dtype=np.int64)
    v[c] = np.asarray(hits, dtype=np.float64)
    v[n_conductors + c] = np.asarray(sum_w, dtype=np.float64)
    v[2 * n_conductors + c] = np.asarray(sum_w2, dtype=np.float64)
    v[3 * n_conductors:] = [walks, escaped, hops, 0.0]
    return v


def result_rows(res, n_conductors: int) -> np.ndarray:
    """dense_rows of a frw.WalkResult."""
    return dense_rows(n_conductors, res.conductor, res.hits, res.sum_w, res.sum_w2, res.walks, res.escaped,
                      res.hops_total)


def all_reduce_rows(vec, group=None):
    """Sum the packed rows over all ranks (torch.distributed, any backend)."""
    import torch
    import torch.distributed as dist

    t = vec if isinstance(vec, torch.Tensor) else torch.as_tensor(vec)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t


def finish(vec, n_conductors: int) -> dict:
    """Capacitance row and standard errors from summed packed rows."""
    v = np.asarray(vec, dtype=np.float64)
    n = n_conductors
    walks = v[3 * n]
    hits, s, s2 = v[:n], v[n:2 * n], v[2 * n:3 * n]
    k = np.nonzero(hits)[0]
    mean = s[k] / walks
    var = np.maximum(s2[k] / walks - mean * mean, 0.0) * walks / max(walks - 1, 1)
    return {"conductor": k, "hits": hits[k], "cap": mean, "cap_se": np.sqrt(var / walks), "walks": walks,
            "escaped": v[3 * n + 1], "hops": v[3 * n + 2]}


# ---- sparse exchange ----------------------------------------------------------
# A step's walks end on a few hundred conductors even on a 10^6-rect layout,
# so each rank sends only its nonzero rows: one int64 tensor per rank,
#   [count, escaped, aborted, hops, done | idx[cap] | hits[cap] | sum_w[cap] | sum_w2[cap]]
# (the float64 sums carried bit for bit in int64 slots), all-gathered, then
# added into dense rows on every rank.  count > cap means rows were left out;
# merge_sparse reports it without a host sync.
HEAD = 5


def sparse_buffer(cap: int, device=None):
    import torch

    return torch.zeros(HEAD + 4 * int(cap), dtype=torch.int64, device=device)


def sparse_views(buf, cap: int):
    """(count[1], stats[4], idx, hits, sum_w, sum_w2) views into a sparse buffer."""
    import torch

    c = int(cap)
    e = buf[HEAD:].view(4, c)
    return (buf[0:1], buf[1:HEAD], e[0], e[1], e[2].view(torch.float64), e[3].view(torch.float64))


def compact_torch(rows_i, rows_f, n: int, buf, cap: int):
    """Fill a sparse buffer from dense rows (hits | stats int64, sum_w | sum_w2
    float64) with torch operations -- the portable counterpart of the device
    compaction frw_rows_compact (used by the CPU multi-process tests)."""
    import torch

    count, stats, idx, hits, s1, s2 = sparse_views(buf, cap)
    k = torch.nonzero(rows_i[:n] > 0).flatten()
    count.fill_(int(k.numel()))
    stats.copy_(rows_i[n:n + 4])
    m = min(int(k.numel()), int(cap))
    idx[:m] = k[:m]
    hits[:m] = rows_i[k[:m]]
    s1[:m] = rows_f[k[:m]]
    s2[:m] = rows_f[n + k[:m]]
    return buf


def gather_sparse(buf, world: int, group=None):
    """All ranks' sparse buffers, stacked [world, len] (one all-gather)."""
    import torch
    import torch.distributed as dist

    out = torch.empty(world * buf.numel(), dtype=buf.dtype, device=buf.device)
    dist.all_gather_into_tensor(out, buf, group=group)
    return out.view(world, buf.numel())


def merge_sparse(gathered, n: int, cap: int, rows_i, rows_f):
    """Add every rank's entries into dense rows_i (hits | stats) and rows_f
    (sum_w | sum_w2), which the caller has zeroed; returns a 0-d bool tensor,
    true when some rank had more nonzero rows than `cap`."""
    import torch

    world = gathered.shape[0]
    c = int(cap)
    ent = gathered[:, HEAD:].reshape(world, 4, c)
    valid = torch.arange(c, device=gathered.device)[None, :] < gathered[:, 0:1]
    k = torch.where(valid, ent[:, 0], torch.zeros_like(ent[:, 0])).flatten()
    zero_i = torch.zeros_like(ent[:, 1])
    h = torch.where(valid, ent[:, 1], zero_i).flatten()
    fs = ent[:, 2:4].contiguous().view(torch.float64)
    s1 = torch.where(valid, fs[:, 0], torch.zeros_like(fs[:, 0])).flatten()
    s2 = torch.where(valid, fs[:, 1], torch.zeros_like(fs[:, 1])).flatten()
    rows_i[:n].index_add_(0, k, h)
    rows_f[:n].index_add_(0, k, s1)
    rows_f[n:2 * n].index_add_(0, k, s2)
    rows_i[n:n + 4] += gathered[:, 1:HEAD].sum(0)
    return (gathered[:, 0] > c).any()

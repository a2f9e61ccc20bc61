"""Walk sharding across ranks (one process per GPU).

Walks are independent, so the layout is replicated and rank r runs its walks
on Philox stream r (weak scaling: every rank runs the same walk count).  The
only exchange is one sum of the per-conductor rows (hits, sum w, sum w^2) and
of the scalar totals -- an NCCL all-reduce of 3*n + 4 doubles per step.  The
reference is single-GPU; this module has no counterpart there.
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

"""The multi-GPU exchange's device half: frw_rows_compact turns the dense
per-conductor rows of frw_walk_device into (conductor, hits, sum_w, sum_w2)
entries of the conductors reached, reporting how many there are even when
the capacity is smaller; and the sparse buffer goes through an NCCL
all-gather and the merge back into dense rows unchanged (one rank: this pool
runs one GPU per job; two ranks are covered with gloo in test_multirank.py)."""
import datetime
import os
import socket

import numpy as np
import pytest

import frw
from frw import shard

pytestmark = pytest.mark.gpu


def _rows(L, n, walks=2_000_000):
    import torch

    rows_i = torch.zeros(n + 4, dtype=torch.int64, device="cuda")
    rows_f = torch.zeros(2 * n, dtype=torch.float64, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    L.walk_device(0, walks, 5, frw.capacitance_opts(1.0), rows_i[:n], rows_f[:n], rows_f[n:], rows_i[n:], status)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    return rows_i, rows_f


def test_rows_compact_lists_every_reached_conductor():
    import torch

    rects = frw.generate_layout(0xF4A7 + 2, 10_000, 1e4)
    with frw.Layout.from_rects(rects) as L:
        n = L.n
        rows_i, rows_f = _rows(L, n)
        hits = rows_i[:n].cpu().numpy()
        fw = rows_f.cpu().numpy()
        k = np.nonzero(hits)[0]
        assert len(k) > 4
        for cap in (len(k) + 10, len(k) // 2):
            buf = shard.sparse_buffer(cap, "cuda")
            cnt, _, idx, h, s1, s2 = shard.sparse_views(buf, cap)
            L.rows_compact(rows_i[:n], rows_f[:n], rows_f[n:], idx, h, s1, s2, cnt)
            torch.cuda.synchronize()
            assert int(cnt.item()) == len(k)
            m = min(cap, len(k))
            got = idx[:m].cpu().numpy()
            assert len(np.unique(got)) == m and np.isin(got, k).all()
            assert np.array_equal(h[:m].cpu().numpy(), hits[got])
            assert np.array_equal(s1[:m].cpu().numpy(), fw[:n][got])
            assert np.array_equal(s2[:m].cpu().numpy(), fw[n:][got])


def test_sparse_exchange_through_nccl_one_rank():
    import torch
    import torch.distributed as dist

    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    try:
        rects = frw.generate_layout(0xF4A7 + 2, 10_000, 1e4)
        with frw.Layout.from_rects(rects) as L:
            n = L.n
            rows_i, rows_f = _rows(L, n)
            cap = 4096
            buf = shard.sparse_buffer(cap, "cuda")
            cnt, stats, idx, h, s1, s2 = shard.sparse_views(buf, cap)
            L.rows_compact(rows_i[:n], rows_f[:n], rows_f[n:], idx, h, s1, s2, cnt)
            stats.copy_(rows_i[n:])
            g = shard.gather_sparse(buf, 1)
            mi, mf = torch.zeros_like(rows_i), torch.zeros_like(rows_f)
            ovf = shard.merge_sparse(g, n, cap, mi, mf)
            torch.cuda.synchronize()
            assert not bool(ovf.item())
            assert torch.equal(mi, rows_i) and torch.equal(mf, rows_f)
    finally:
        dist.destroy_process_group()

"""The N>1 path on the CPU: two gloo ranks shard the walks by Philox stream,
sum their packed rows with one all-reduce, and the result equals a single
process running both streams.  Per-rank walks come from the CPU oracle (the
same walks the device produces bit-for-bit, see test_gpu_walk.py).  A rank
that fails before the collective makes the other rank's all-reduce end with
an error instead of hanging."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _oracle_rows(rank, n_walks):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "engineer-thesis_b200"))
    import oracle as O
    from frw import shard

    rects = _layout()
    G = O.Grid(rects)
    p = shard.plan(n_walks, rank)
    cfg = G.walk_cfg(target=0, seed=77, stream=p["stream"])
    end, hops, _, w = G.walks(cfg, p["first"], p["count"])
    ks = np.unique(end[end >= 0])
    hits = [(end == k).sum() for k in ks]
    s1 = [w[end == k].sum() for k in ks]
    s2 = [(w[end == k] ** 2).sum() for k in ks]
    return shard.dense_rows(len(rects), ks, hits, s1, s2, n_walks, int((end == -1).sum()), int(hops.sum()))


def _layout():
    rng = np.random.default_rng(4)
    # a small non-overlapping layout: a grid of 5x5 rects with jitter
    r = []
    for i in range(5):
        for j in range(5):
            x, y = 100 * i + rng.integers(0, 20), 100 * j + rng.integers(0, 20)
            r.append([x, y, x + rng.integers(10, 60), y + rng.integers(10, 60)])
    return np.array(r, dtype=np.float64)


def _worker(rank, world, port, n_walks, out_path, fail_rank):
    import datetime

    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    sys.path.insert(0, os.path.join(ROOT, "engineer-thesis_b200"))
    from frw import shard

    try:
        if rank == fail_rank:
            raise RuntimeError("injected rank failure before the collective")
        v = torch.as_tensor(_oracle_rows(rank, n_walks))
        shard.all_reduce_rows(v)
        if rank == 0:
            np.save(out_path, v.numpy())
    except Exception as e:  # report, then leave without joining further collectives
        with open(out_path + f".err{rank}", "w") as f:
            f.write(repr(e))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def _run(world, n_walks, tmp_path, fail_rank=-1):
    import torch.multiprocessing as tmp

    out = str(tmp_path / "rows.npy")
    tmp.start_processes(_worker, args=(world, _free_port(), n_walks, out, fail_rank), nprocs=world,
                        join=True, start_method="spawn")
    return out


def test_two_rank_rows_equal_single_process(tmp_path):
    sys.path.insert(0, os.path.join(ROOT, "engineer-thesis_b200"))
    from frw import shard

    n = 3000
    out = _run(2, n, tmp_path)
    got = np.load(out)
    want = _oracle_rows(0, n) + _oracle_rows(1, n)
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=0)
    fin = shard.finish(got, len(_layout()))
    assert fin["walks"] == 2 * n and fin["hits"].sum() + fin["escaped"] <= 2 * n
    assert 0 in fin["conductor"] and fin["cap"][list(fin["conductor"]).index(0)] > 0


def test_failed_rank_ends_peer_collective_with_error(tmp_path):
    out = _run(2, 200, tmp_path, fail_rank=1)
    assert os.path.exists(out + ".err1")
    # rank 0's all-reduce either raised (peer gone / timeout) or never produced rows
    assert os.path.exists(out + ".err0") or not os.path.exists(out)


def _sparse_worker(rank, world, port, n_walks, out_path):
    import datetime

    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    sys.path.insert(0, os.path.join(ROOT, "engineer-thesis_b200"))
    from frw import shard

    try:
        n = len(_layout())
        v = _oracle_rows(rank, n_walks)  # [hits | sum_w | sum_w2 | walks, escaped, hops, 0]
        rows_i = torch.zeros(n + 4, dtype=torch.int64)
        rows_f = torch.zeros(2 * n, dtype=torch.float64)
        rows_i[:n] = torch.as_tensor(v[:n]).to(torch.int64)
        rows_f[:n] = torch.as_tensor(v[n:2 * n])
        rows_f[n:] = torch.as_tensor(v[2 * n:3 * n])
        rows_i[n:] = torch.as_tensor([int(v[3 * n + 2]), 0, 0, int(v[3 * n])])  # escaped-ish, aborted, hops, done
        out = {}
        for cap in (4, 64):  # 4: fewer slots than conductors reached, reported as overflow
            buf = shard.sparse_buffer(cap)
            shard.compact_torch(rows_i, rows_f, n, buf, cap)
            g = shard.gather_sparse(buf, world)
            mi = torch.zeros_like(rows_i)
            mf = torch.zeros_like(rows_f)
            ovf = shard.merge_sparse(g, n, cap, mi, mf)
            out[cap] = (mi.numpy(), mf.numpy(), bool(ovf))
        dense_i, dense_f = rows_i.clone(), rows_f.clone()
        dist.all_reduce(dense_i)
        dist.all_reduce(dense_f)
        if rank == 0:
            np.savez(out_path, mi=out[64][0], mf=out[64][1], ovf64=out[64][2], ovf4=out[4][2],
                     di=dense_i.numpy(), df=dense_f.numpy())
    finally:
        dist.destroy_process_group()


def test_sparse_exchange_equals_dense_all_reduce(tmp_path):
    import torch.multiprocessing as tmp

    out = str(tmp_path / "sparse.npz")
    tmp.start_processes(_sparse_worker, args=(2, _free_port(), 3000, out), nprocs=2, join=True,
                        start_method="spawn")
    r = np.load(out)
    assert not r["ovf64"] and r["ovf4"]
    assert np.array_equal(r["mi"], r["di"])
    np.testing.assert_allclose(r["mf"], r["df"], rtol=1e-14, atol=0)

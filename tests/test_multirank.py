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

"""Replica parallelism on the CPU: world size 2 over gloo (127.0.0.1), the
same rank plumbing bench.py --gpus N uses on GPUs (barrier, maximum of the
elapsed time over ranks) and the per-rank slice shares of the multi-slice
reconstruction, gathered on rank 0 in slice order (the reference's -mgpu
model, main_mri.cu:770-834: whole slices per GPU, images gathered on the
host).  No GPU, no data-path collective."""
import multiprocessing as mp
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def _replicas():
    sys.path.insert(0, str(ROOT))
    from __graft_entry__ import load_package
    load_package()
    from impatient_mri_b200 import replicas
    return replicas


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, n_slices, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(ws),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    try:
        R = _replicas()
        ws_, rank_, _ = R.init(timeout_s=60, backend="gloo")
        assert (ws_, rank_) == (ws, rank)
        R.barrier(ws)
        worst = R.max_over_ranks(0.5 + rank, ws)
        lo, hi = R.slice_range(n_slices, ws, rank)
        # a stand-in image per slice: slice s holds s + 1j * s everywhere
        imgs = np.array([[s + 1j * s] * 4 for s in range(lo, hi)], np.complex64).reshape(-1, 4)
        gathered = R.gather_images(imgs, n_slices, ws, rank)
        R.barrier(ws)
        R.finalize(ws)
        out.put((rank, worst, lo, hi, None if gathered is None else gathered.tolist()))
    except Exception as e:  # reported to the parent, which fails the test
        out.put((rank, repr(e), None, None, None))


@pytest.mark.parametrize("n_slices", [7, 1])
def test_two_ranks_over_gloo(n_slices):
    ws = 2
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, ws, port, n_slices, out)) for r in range(ws)]
    for p in procs:
        p.start()
    res = {}
    try:
        for _ in range(ws):
            r = out.get(timeout=180)
            res[r[0]] = r
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    for r in range(ws):
        assert isinstance(res[r][1], float), res[r][1]
        assert res[r][1] == 1.5  # max over ranks of 0.5 + rank
    shares = [(res[r][2], res[r][3]) for r in range(ws)]
    assert shares[0][0] == 0 and shares[-1][1] == n_slices
    assert all(shares[r][1] == shares[r + 1][0] for r in range(ws - 1))
    g = np.array(res[0][4])
    assert g.shape == (n_slices, 4)
    assert np.array_equal(g.real[:, 0], np.arange(n_slices))
    assert res[1][4] is None


def test_slice_range_partitions():
    R = _replicas()
    for n in (0, 1, 5, 64, 65):
        for ws in (1, 2, 3, 8):
            owned = [s for r in range(ws) for s in range(*R.slice_range(n, ws, r))]
            assert owned == list(range(n))
            sizes = [np.subtract(*R.slice_range(n, ws, r)[::-1]) for r in range(ws)]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        R.slice_range(4, 2, 2)


def test_single_process_is_a_no_op():
    R = _replicas()
    assert R.max_over_ranks(3.25, 1) == 3.25
    R.barrier(1)
    x = np.ones((3, 5), np.complex64)
    assert R.gather_images(x, 3, 1, 0) is x or np.array_equal(R.gather_images(x, 3, 1, 0), x)

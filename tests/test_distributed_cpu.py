"""The multi-rank path on CPU: two ``gloo`` ranks each take their shots of a
survey (``sweep_b200.distributed.shot_slice``), compute the loss and gradient
of those shots (here with the CPU oracle standing in for the CUDA core, which
needs a GPU) and all-reduce them (``sharded_gradient``).  The result must equal
the single-process gradient of the whole survey."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from sweep_b200.distributed import shot_slice, sharded_gradient
from tests._util import load, rel


def test_shot_slices_partition_the_survey():
    for n in (1, 5, 32, 33):
        for world in (1, 2, 3, 8):
            parts = [shot_slice(n, world, r) for r in range(world)]
            idx = [i for p in parts for i in range(n)[p]]
            assert idx == list(range(n))
            sizes = [len(range(n)[p]) for p in parts]
            assert max(sizes) - min(sizes) <= 1


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _oracle_compute(d):
    from oracle import oracle as O

    def compute(shots):
        src, rec = d["src"][shots], d["rec"][shots]
        w = d["wavelet"][shots] if d["wavelet"].ndim == 2 else d["wavelet"]
        if len(src) == 0:
            return torch.zeros((), dtype=torch.float64), [torch.zeros(d["vp_init"].shape, dtype=torch.float64)]
        pred, loss, g, _ = O.acoustic_gradient(d["vp_init"], w, src, rec, d["obs"][shots],
                                               float(d["dh"]), float(d["dt"]), int(d["abcn"]), prec="f64")
        return torch.tensor(loss, dtype=torch.float64), [torch.from_numpy(np.asarray(g, np.float64))]
    return compute


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        d = load("acoustic2d_multi")
        loss, grads = sharded_gradient(_oracle_compute(d), len(d["src"]))
        if rank == 0:
            np.save(out, np.concatenate([[float(loss)], grads[0].numpy().ravel()]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 4])
def test_sharded_gradient_equals_single_process(tmp_path, world):
    d = load("acoustic2d_multi")
    if world > len(d["src"]) + 1:
        pytest.skip("more ranks than shots + 1")
    out = str(tmp_path / "rank0.npy")
    mp.start_processes(_rank, args=(world, _free_port(), out), nprocs=world, start_method="spawn", join=True)
    got = np.load(out)
    loss_ref, g_ref = _oracle_compute(d)(slice(0, len(d["src"])))
    assert abs(got[0] - float(loss_ref)) <= 1e-12 * abs(float(loss_ref))
    assert rel(got[1:], g_ref[0].numpy().ravel()) < 1e-12


def _rank_float_loss(rank, world, port, out):
    """compute() returning the loss as a Python float (and the gradient as a
    float32 tensor): sharded_gradient moves the loss beside the gradients
    before the all-reduce."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        def compute(shots):
            n = len(range(6)[shots])
            return float(n) * 0.5, [torch.full((3, 4), float(n), dtype=torch.float32)]
        loss, grads = sharded_gradient(compute, 6)
        if rank == 0:
            np.save(out, np.concatenate([[float(loss)], grads[0].numpy().ravel()]))
    finally:
        dist.destroy_process_group()


def test_sharded_gradient_takes_a_python_float_loss(tmp_path):
    out = str(tmp_path / "rank0.npy")
    mp.start_processes(_rank_float_loss, args=(2, _free_port(), out), nprocs=2, start_method="spawn", join=True)
    got = np.load(out)
    assert got[0] == 3.0
    assert np.all(got[1:] == 6.0)


def _rank_bench_step(rank, world, port, out, k, group):
    """The bench's FWI step on gloo ranks: bench.step_shots picks this rank's
    shot group of step k, the CPU oracle computes its loss and gradient (in
    place of the CUDA core) and sharded_gradient all-reduces them."""
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        d = load("acoustic2d_multi")
        nshot = len(d["src"])
        compute = _oracle_compute(d)

        def mine(_):
            sh = bench.step_shots(k, group, nshot, world, rank)
            assert len(sh) == group
            # the oracle takes a slice; feed it shot by shot
            losses, grads = zip(*[compute(slice(s, s + 1)) for s in sh])
            return sum(losses), [sum(g[0] for g in grads)]
        loss, grads = sharded_gradient(mine, world * group)
        if rank == 0:
            np.save(out, np.concatenate([[float(loss)], grads[0].numpy().ravel()]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("k", [0, 1])
def test_bench_step_on_two_ranks_equals_its_shots_on_one(tmp_path, k):
    import bench
    d = load("acoustic2d_multi")
    nshot, group, world = len(d["src"]), 1, 2
    out = str(tmp_path / "rank0.npy")
    mp.start_processes(_rank_bench_step, args=(world, _free_port(), out, k, group), nprocs=world,
                       start_method="spawn", join=True)
    got = np.load(out)
    # the shots of the step's window, all on one process
    shots = [s for r in range(world) for s in bench.step_shots(k, group, nshot, world, r)]
    assert len(set(shots)) == world * group
    compute = _oracle_compute(d)
    losses, grads = zip(*[compute(slice(s, s + 1)) for s in shots])
    assert abs(got[0] - float(sum(losses))) <= 1e-12 * abs(float(sum(losses)))
    assert rel(got[1:], sum(g[0] for g in grads).numpy().ravel()) < 1e-12


def test_bench_step_shots_cover_the_survey():
    import bench
    for nshot, group, world in ((16, 3, 1), (16, 3, 2), (32, 32, 4), (5, 2, 3)):
        seen = []
        for k in range(nshot):
            per_rank = [bench.step_shots(k, group, nshot, world, r) for r in range(world)]
            assert all(len(p) == group for p in per_rank)
            seen += [s for p in per_rank for s in p]
        assert set(seen) == set(range(nshot))

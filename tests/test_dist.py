"""Multi-process logic of nemo_b200.dist on CPU (gloo, two ranks): trial and
instance sharding, and the data-parallel gradient of the differentiable form
(each rank differentiates its share of the trials with the float64
reference model; one all-reduce must give the full-batch gradient)."""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from nemo_b200.dist import dp_grad, exchange_fired_words, shard_instances, shard_trials, shard_warps


def test_shard_trials_covers_all_trials():
    for total in (1, 7, 32, 33):
        for world in (1, 2, 3, 8):
            ranges = [shard_trials(total, r, world) for r in range(world)]
            assert ranges[0][0] == 0 and ranges[-1][1] == total
            assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))
            sizes = [b - a for a, b in ranges]
            assert max(sizes) - min(sizes) <= 1


def test_shard_instances_balances():
    sizes = np.round(np.exp(np.random.default_rng(0).uniform(np.log(500), np.log(20000), 256))).astype(int)
    for world in (1, 2, 4, 8):
        parts = shard_instances(sizes, world)
        allj = sorted(j for p in parts for j in p)
        assert allj == list(range(sizes.size))
        loads = [sizes[p].sum() for p in parts]
        assert max(loads) - min(loads) <= sizes.max()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _problem():
    from nemo_b200.lif import LIFNetwork
    net = LIFNetwork.random(20, 5, 6, 3, seed=4, checkpoint=5, bin_steps=5, device="cpu")
    rng = np.random.default_rng(1)
    T, B = 20, 6
    ins = rng.random((T, 6, B)) < 0.3
    w = rng.normal(0, 0.8, net.synapses)
    target = 20 + 10 * np.sin(np.arange(T // 5))
    return net, ins, w, target, B


def _grad(net, ins, w, target, lo, hi):
    import lif_reference as ref
    from nemo_b200.lif import rate_loss
    wt = torch.tensor(w, dtype=torch.float64, requires_grad=True)
    c = ref.counts(net, wt, ins[:, :, lo:hi], hi - lo, relaxed=True)
    rate_loss(c, net.n, net.bin_steps, torch.tensor(target)).backward()
    return wt.grad


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        net, ins, w, target, B = _problem()
        lo, hi = shard_trials(B, rank, world)
        g = dp_grad(_grad(net, ins, w, target, lo, hi), hi - lo, B)
        if rank == 0:
            out.put(g.numpy())
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_data_parallel_gradient_equals_full_batch():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    g = out.get(timeout=240)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    net, ins, w, target, B = _problem()
    full = _grad(net, ins, w, target, 0, B).numpy()
    assert np.allclose(g, full, rtol=1e-12, atol=1e-12 * np.abs(full).max())


def test_shard_warps_matches_library():
    """The Python partition of warps over shards is the library's."""
    import ctypes
    from nemo_b200.nemo import PRODUCT_LIBRARY
    lib = ctypes.CDLL(PRODUCT_LIBRARY)
    first, count = ctypes.c_uint(), ctypes.c_uint()
    for total in (1, 7, 100, 3125, 3126):
        for world in (1, 2, 3, 8):
            covered = 0
            for rank in range(world):
                assert lib.nemo_b200_shard_warps(total, rank, world, ctypes.byref(first), ctypes.byref(count)) == 0
                assert (first.value, count.value) == shard_warps(total, rank, world)
                assert first.value == covered
                covered += count.value
            assert covered == total
    assert lib.nemo_b200_shard_warps(10, 2, 2, ctypes.byref(first), ctypes.byref(count)) != 0


def _words_of(total):
    return (np.arange(total, dtype=np.uint64) * 2654435761 % (1 << 32)).astype(np.uint32)


def _exchange_worker(rank, world, port, total, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        f, c = shard_warps(total, rank, world)
        full = exchange_fired_words(_words_of(total)[f:f + c], f, total)
        out.put((rank, full))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
@pytest.mark.parametrize("total", [5, 3125])
def test_exchange_fired_words_two_ranks(total):
    """Each of two gloo ranks contributes the words of its own warps (shares
    of unequal size when total is odd); both get every warp's word."""
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_exchange_worker, args=(r, 2, port, total, out)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(out.get(timeout=240) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(2):
        assert np.array_equal(got[r], _words_of(total))

"""Bunch sharding, host side (no GPU): the bunch partition of cg_shard_plan,
and the moments exchange it implies (each rank's slice padded to the largest
slice, an all-gather, a scatter by rank offsets - the data movement of the
library's NCCL exchange) run as two gloo ranks on the CPU."""
import ctypes as C
import os
import socket

import numpy as np
import pytest

from cetasim_b200 import _abi, configs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def plan(lib, n_macro, world):
    n = np.ascontiguousarray(n_macro, dtype=np.int32)
    j0 = np.zeros(world, dtype=np.int32)
    j1 = np.zeros(world, dtype=np.int32)
    assert lib.cg_shard_plan(_abi.ptr(n), len(n), world, _abi.ptr(j0), _abi.ptr(j1)) == 0
    return j0, j1


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_plan_covers_the_train_contiguously_and_balanced(lib, world):
    rng = np.random.default_rng(3)
    n_macro = np.exp(rng.uniform(np.log(5e3), np.log(5e4), 900)).astype(np.int32)
    j0, j1 = plan(lib, n_macro, world)
    assert j0[0] == 0 and j1[-1] == len(n_macro)
    assert np.all(j0[1:] == j1[:-1]) and np.all(j1 > j0)
    loads = np.array([n_macro[a:b].sum() for a, b in zip(j0, j1)])
    assert loads.max() - loads.min() <= 2 * n_macro.max()


def test_plan_gives_every_rank_a_bunch(lib):
    j0, j1 = plan(lib, [1000, 1, 1, 1], 4)
    assert list(j1 - j0) == [1, 1, 1, 1]


def _rank(rank, world, port, n_bunches, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import torch
    lib = _abi.load()
    rng = np.random.default_rng(0)
    n_macro = rng.integers(100, 2000, n_bunches).astype(np.int32)
    j0, j1 = plan(lib, n_macro, world)
    # stand-in for the 24-double per-bunch moments record: a function of j
    full = np.arange(n_bunches * 24, dtype=np.float64).reshape(n_bunches, 24) * 1.5
    maxlocal = int((j1 - j0).max())
    send = np.zeros((maxlocal, 24))
    mine = slice(j0[rank], j1[rank])
    send[: j1[rank] - j0[rank]] = full[mine]
    recv = [torch.zeros(maxlocal, 24, dtype=torch.float64) for _ in range(world)]
    dist.all_gather(recv, torch.from_numpy(send))
    mom = np.full((n_bunches, 24), np.nan)
    mom[mine] = full[mine]                   # the rank's own, as computed locally
    for r in range(world):                   # the scatter kernel
        mom[j0[r]:j1[r]] = recv[r].numpy()[: j1[r] - j0[r]]
    ok = bool(np.array_equal(mom, full))
    flags = [torch.zeros(1) for _ in range(world)]
    dist.all_gather(flags, torch.tensor([1.0 if ok else 0.0]))
    if rank == 0:
        out.put([float(f.item()) for f in flags])
    dist.destroy_process_group()


def test_moments_exchange_over_two_gloo_ranks():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, 37, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == [1.0, 1.0]

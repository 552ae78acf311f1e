"""Bunch sharding, host side (no GPU): the bunch partition of cg_shard_plan,
and the moments exchange it implies run as two gloo ranks on the CPU through
the library's own pack and place steps (cg_shard_pack / cg_shard_unpack: the
layout the device exchange uses around its NCCL all-gather), with
torch.distributed's all-gather as the transport."""
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


def _exchange(lib, n_macro, world, rank, records, gather):
    """One moments exchange through the library (cg_shard_pack /
    cg_shard_unpack), with `gather` moving the send slots between ranks."""
    n = np.ascontiguousarray(n_macro, dtype=np.int32)
    M, rec = len(n), records.strides[0]
    ml = C.c_int()
    assert lib.cg_shard_exchange_size(_abi.ptr(n), M, world, C.byref(ml)) == 0
    send = np.zeros(ml.value * rec, dtype=np.uint8)
    assert lib.cg_shard_pack(_abi.ptr(n), M, world, rank, records.ctypes.data, rec,
                             send.ctypes.data) == 0
    gathered = np.ascontiguousarray(gather(send))
    out = np.zeros_like(records)
    assert lib.cg_shard_unpack(_abi.ptr(n), M, world, gathered.ctypes.data, rec,
                               out.ctypes.data) == 0
    return out


def _beam_moments(n_bunches, n_macro, owned):
    """Per-bunch moments (the library's cg_bunch_moments records) of a seeded
    train, as the oracle computes them; the bunches this rank does not own
    are left as garbage, since only the owner's records may travel."""
    import oracle
    from helpers import particles
    wl = configs.make("batched_uneven", n_scale=1.0, derive=oracle.config_derive,
                      lattice_init=oracle.lattice_init)
    wl.n_macro = np.ascontiguousarray(n_macro[:n_bunches], dtype=np.int32)
    wl.harm, wl.ne = wl.harm[:n_bunches].copy(), wl.ne[:n_bunches].copy()
    o = oracle.OracleBeam(wl)
    for j, c in enumerate(particles(wl, seed=9, spread=2.0)):
        o.upload(j, c)
    o.MPBeamRMSCal(0)
    m = o.moments()
    rec = np.frombuffer(bytes(m), dtype=np.uint8).reshape(n_bunches, -1).copy()
    for j in range(n_bunches):
        if not owned(j):
            rec[j] = 0xA5
    return rec


def _rank(rank, world, port, n_bunches, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import torch
    lib = _abi.load()
    rng = np.random.default_rng(0)
    n_macro = rng.integers(50, 400, n_bunches).astype(np.int32)
    j0, j1 = plan(lib, n_macro, world)
    mine = _beam_moments(n_bunches, n_macro, lambda j: j0[rank] <= j < j1[rank])

    def gather(send):
        parts = [torch.zeros(len(send), dtype=torch.uint8) for _ in range(world)]
        dist.all_gather(parts, torch.from_numpy(send))
        return np.concatenate([p.numpy() for p in parts])

    got = _exchange(lib, n_macro, world, rank, mine, gather)
    # the one-rank exchange of the unsharded records: every rank must now hold
    # exactly these bytes
    alone = _exchange(lib, n_macro, 1, 0, _beam_moments(n_bunches, n_macro, lambda j: True),
                      lambda send: send)
    ok = bool(np.array_equal(got, alone))
    flags = [torch.zeros(1) for _ in range(world)]
    dist.all_gather(flags, torch.tensor([1.0 if ok else 0.0]))
    if rank == 0:
        out.put([float(f.item()) for f in flags])
    dist.destroy_process_group()


def test_moments_exchange_over_two_gloo_ranks():
    """The library's exchange (cg_shard_pack, an all-gather, cg_shard_unpack)
    run by two gloo ranks on the oracle's moments of a ragged train: both
    ranks end with the records of a one-rank run, bit for bit."""
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


def test_exchange_rejects_bad_arguments(lib):
    n = np.array([10, 20, 30], dtype=np.int32)
    ml = C.c_int()
    assert lib.cg_shard_exchange_size(_abi.ptr(n), 3, 4, C.byref(ml)) != 0   # more ranks than bunches
    assert lib.cg_shard_pack(_abi.ptr(n), 3, 2, 2, None, 8, None) != 0

"""Host helpers of the field surrogate (the network itself lives in
libcetagpu: training, inference and the kick run on the GPU)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi

N_PARAMS = 8706  # CG_SUR_PARAMS


class SurrogateError(RuntimeError):
    pass


def _check(lib, rc):
    if rc != 0:
        raise _abi.CgError(rc, lib.cg_last_error(None).decode())


def dataset(seed: int, n: int):
    """(inputs [n, 3] = (a, b, r), targets [n, 2] = G) from the exact field."""
    lib = _abi.load()
    x = np.empty((n, 3), dtype=np.float32)
    t = np.empty((n, 2), dtype=np.float32)
    _check(lib, lib.cg_surrogate_dataset(seed, n, _abi.ptr(x), _abi.ptr(t)))
    return x, t


def evaluate(weights, x):
    lib = _abi.load()
    w = np.ascontiguousarray(weights, dtype=np.float32)
    x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, 3)
    out = np.empty((len(x), 2), dtype=np.float32)
    _check(lib, lib.cg_surrogate_eval(_abi.ptr(w), _abi.ptr(x), len(x), _abi.ptr(out)))
    return out


def gradient(weights, x, t):
    lib = _abi.load()
    w = np.ascontiguousarray(weights, dtype=np.float32)
    x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, 3)
    t = np.ascontiguousarray(t, dtype=np.float32).reshape(-1, 2)
    g = np.empty(N_PARAMS, dtype=np.float32)
    loss = C.c_double()
    _check(lib, lib.cg_surrogate_grad(_abi.ptr(w), _abi.ptr(x), _abi.ptr(t), len(x), _abi.ptr(g),
                                      C.byref(loss)))
    return loss.value, g


def train(seed: int = 2024, n_train: int = 1 << 20, n_holdout: int = 1 << 16, epochs: int = 300,
          batch: int = 2048, lr: float = 5e-3, l4_from: float = 10.0, l4_weight: float = 0.5):
    """Trains on the GPU; returns (weights, stats) with stats = (final training
    loss per output, hold-out RMS error / peak |G|, hold-out max error / peak,
    seconds).  From epoch l4_from * epochs on (default: never) the loss mixes
    in the fourth power of the error with weight l4_weight, which weighs the
    largest errors more (measured on the hold-out: no better than the plain
    squared error with this schedule)."""
    lib = _abi.load()
    p = _abi.SurTrainParams(seed, n_train, n_holdout, epochs, batch, lr, l4_from, l4_weight)
    w = np.empty(N_PARAMS, dtype=np.float32)
    stats = np.zeros(4)
    _check(lib, lib.cg_surrogate_train(C.byref(p), _abi.ptr(w), _abi.ptr(stats)))
    return w, stats

"""The bunch-sharding exchange path on one GPU: a one-rank NCCL communicator
makes every moments pass go through the all-gather and scatter (captured in
the turn graph); the run must repeat the plain single-GPU run bit for bit."""
import numpy as np
import pytest

from cetasim_b200.beam import MPBeam
from helpers import TRAPPED, particles, small

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,scale,kw,ions", [
    ("fast_ion", 0.01, {"bunch_current": TRAPPED}, True),   # exchange before every ion chain
    ("batched_uneven", 0.005, {}, False),                   # exchanges for the LR wake and FIR
])
def test_exchange_path_repeats_the_plain_run(name, scale, kw, ions):
    wl = small(name, scale, **kw)
    if not ions:
        wl.cfg.flag_beam_ion = 0
    parts = particles(wl, seed=3)
    runs = []
    for shard in (None, (0, 1, MPBeam.nccl_unique_id())):
        g = MPBeam(wl, shard=shard)
        assert list(g.local) == list(range(wl.n_bunches))
        for j, c in enumerate(parts):
            g.upload(j, c)
        g.Run(0, 5)
        g.MPBeamRMSCal(0)
        runs.append(([g.download(j) for j in range(wl.n_bunches)],
                     [g.ions(k) for k in range(wl.cfg.n_sections)] if ions else [],
                     [(m.mean[0], m.rms_x, m.transmission) for m in g.moments()]))
        g.close()
    (ca, ia, ma), (cb, ib, mb) = runs
    for (x, s), (y, t) in zip(ca, cb):
        assert np.array_equal(x, y) and np.array_equal(s, t)
    for u, v in zip(ia, ib):
        for p, q in zip(u, v):
            assert np.array_equal(p, q)
    assert ma == mb

"""Checkpoint / resume: N turns, a checkpoint, a fresh handle restored from
it and N more turns reproduce 2N uninterrupted turns bit for bit (the random
draws are counters of seed and turn; every reduction has a fixed order)."""
import numpy as np
import pytest

from cetasim_b200 import _abi
from cetasim_b200.beam import MPBeam
from helpers import TRAPPED, particles, small

pytestmark = pytest.mark.gpu


def _state(g, wl):
    coords = [g.download(j) for j in range(wl.n_bunches)]
    ions = []
    if wl.cfg.flag_beam_ion:
        for k in range(wl.cfg.n_sections):
            ions.append(g.ions(k))
    return coords, ions


def _same(a, b):
    (ca, ia), (cb, ib) = a, b
    for (x, s), (y, t) in zip(ca, cb):
        assert np.array_equal(x, y) and np.array_equal(s, t)
    for u, v in zip(ia, ib):
        for p, q in zip(u, v):
            assert np.array_equal(p, q)


@pytest.mark.parametrize("name,scale,kw", [
    ("fast_ion", 0.01, {"bunch_current": TRAPPED}),     # ion clouds
    ("batched_uneven", 0.005, {}),                      # LR wake + FIR histories, ragged bunches
    ("plain_single", 0.02, {"sr_bins": 40}),            # short-range wake potentials
])
def test_resume_repeats_the_uninterrupted_run(name, scale, kw):
    wl = small(name, scale, **kw)
    if name == "batched_uneven":
        wl.cfg.flag_beam_ion = 0   # keep the 50-IP train quick; histories are the point
    parts = particles(wl, seed=12)
    n = 6
    a = MPBeam(wl)
    for j, c in enumerate(parts):
        a.upload(j, c)
    a.Run(0, 2 * n)
    b = MPBeam(wl)
    for j, c in enumerate(parts):
        b.upload(j, c)
    b.Run(0, n)
    blob = b.checkpoint()
    b.close()
    c = MPBeam(wl)
    c.restore(blob)
    c.Run(n, n)
    _same(_state(a, wl), _state(c, wl))


def test_restore_rejects_another_layout():
    wl = small("fast_ion", 0.01, bunch_current=TRAPPED)
    g = MPBeam(wl)
    g.generate()
    blob = g.checkpoint()
    other = MPBeam(small("fast_ion", 0.02, bunch_current=TRAPPED))
    with pytest.raises(_abi.CgError) as e:
        other.restore(blob)
    assert e.value.code == 1  # CG_ERR_INVALID
    with pytest.raises(_abi.CgError):
        g.restore(blob[:100])

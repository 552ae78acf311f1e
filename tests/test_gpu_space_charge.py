"""Space charge (runSpaceCharge 1, 2, 3) on the GPU through the C ABI: one
step and whole turns (the turn graph: the kick between the ion kick and the
section map) against the reference's own runs (tests/golden/
ref_space_charge.npz), run-to-run determinism, and the zero-size error.
Tolerances: 1e-11 of the kick for one step (the DST as matrix products in
another summation order; fixed-point charge deposits), 1e-10 of the
coordinates' rms after the turns."""
import tempfile

import numpy as np
import pytest

import sccases
from cetasim_b200 import _abi
from cetasim_b200.beam import MPBeam
from refcases import parts_digest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", list(sccases.CASES))
def test_step_matches_the_reference(case):
    g = sccases.golden()
    with tempfile.TemporaryDirectory() as d:
        wl, _, parts = sccases.build(case, d)
    assert parts_digest(parts) == bytes(g[f"{case}/digest"]).decode()
    b = MPBeam(wl)
    sccases.start(b, parts)
    b.MPBeamRMSCal(0)
    b.BeamTransferDueToSpaceCharge(0)
    for j in sccases.KEEP[case]:
        c, _ = b.download(j)
        assert np.array_equal(c[[0, 2, 4, 5]], parts[j][[0, 2, 4, 5]])
        want = g[f"{case}/kick{j}"]
        for q in range(2):
            k = np.max(np.abs(want[q] - parts[j][1 + 2 * q]))
            assert np.max(np.abs(c[1 + 2 * q] - want[q])) <= 1e-11 * k, (j, q)


@pytest.mark.parametrize("case", list(sccases.CASES))
def test_turns_match_the_reference(case):
    g = sccases.golden()
    turns = sccases.CASES[case][3]
    with tempfile.TemporaryDirectory() as d:
        wl, _, parts = sccases.build(case, d)
    b = MPBeam(wl)
    sccases.start(b, parts)
    b.Run(0, turns)
    for j in sccases.KEEP[case]:
        c, s = b.download(j)
        assert np.array_equal(s, g[f"{case}/surv{j}"])
        err = sccases.coord_rel_err(c, g[f"{case}/coords{j}"])
        assert err.max() <= 1e-10, (j, err)


def test_runs_repeat_bit_for_bit():
    with tempfile.TemporaryDirectory() as d:
        wl, _, parts = sccases.build("pic_train", d)
    runs = []
    for _ in range(2):
        b = MPBeam(wl)
        sccases.start(b, parts)
        b.Run(0, 2)
        runs.append([b.download(j)[0] for j in range(wl.n_bunches)])
    for x, y in zip(*runs):
        assert np.array_equal(x, y)


def test_zero_rms_size_is_an_error():
    """A bunch with no horizontal size: the reference stops (MPBunch.cpp:
    893-897); the library returns CG_ERR_INVALID."""
    with tempfile.TemporaryDirectory() as d:
        wl, _, parts = sccases.build("pic_single", d)
    p = parts[0].copy()
    p[0] = 1e-4
    b = MPBeam(wl)
    b.upload(0, p)
    b.MPBeamRMSCal(0)
    with pytest.raises(_abi.CgError) as e:
        b.BeamTransferDueToSpaceCharge(0)
    assert e.value.code == 1  # CG_ERR_INVALID

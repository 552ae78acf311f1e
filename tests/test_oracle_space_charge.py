"""Space charge (runSpaceCharge 1, 2, 3) in the oracle restatement against the
reference's own build: the committed fixtures of its runs
(tests/golden/ref_space_charge.npz, made by tests/golden/make_sc_golden.py).
The reference's 2-D DST (FFTW RODFT00) runs as direct sums in oracle/ref_shim
and the oracle's as its own direct sums in the same order, so the PIC and the
linear model agree bit for bit; the Bassetti-Erskine model differs by the
two codes' w(z) (1e-13 of the kick)."""
import tempfile

import numpy as np
import pytest

import oracle
import sccases
from refcases import parts_digest


@pytest.mark.parametrize("case", list(sccases.CASES))
def test_oracle_step_and_turns_match_the_reference(case):
    g = sccases.golden()
    turns, flag = sccases.CASES[case][3], sccases.CASES[case][4]
    with tempfile.TemporaryDirectory() as d:
        wl, _, parts = sccases.build(case, d)
    assert parts_digest(parts) == bytes(g[f"{case}/digest"]).decode()
    o = oracle.OracleBeam(wl)
    sccases.start(o, parts)
    o.MPBeamRMSCal(0)
    o.BeamTransferDueToSpaceCharge(0)
    for j in sccases.KEEP[case]:
        c, _ = o.download(j)
        assert np.array_equal(c[[0, 2, 4, 5]], parts[j][[0, 2, 4, 5]])
        want = g[f"{case}/kick{j}"]
        got = c[[1, 3]]
        if flag == 1:
            for q in range(2):
                k = np.max(np.abs(want[q] - parts[j][1 + 2 * q]))
                assert np.max(np.abs(got[q] - want[q])) <= 1e-13 * k
        else:
            assert np.array_equal(got, want)
    o = oracle.OracleBeam(wl)
    sccases.start(o, parts)
    o.Run(0, turns)
    for j in sccases.KEEP[case]:
        c, s = o.download(j)
        assert np.array_equal(s, g[f"{case}/surv{j}"])
        want = g[f"{case}/coords{j}"]
        if flag == 1:
            assert sccases.coord_rel_err(c, want).max() <= 1e-12
        else:
            assert np.array_equal(c, want)


def test_input_parser_reads_the_space_charge_settings():
    with tempfile.TemporaryDirectory() as d:
        wl, _, _ = sccases.build("pic_train", d)
    assert wl.cfg.flag_sc == 2 and [wl.cfg.sc_mesh[i] for i in range(3)] == [16, 24, 9]

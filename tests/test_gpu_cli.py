"""The cetasim_mp driver on a small input.dat: it tracks on the GPU, writes
result.sdds and, with runCBMGR set, the coupled-bunch growth-rate file in the
page layout of MPBeam::GetCBMGR (one page per mode / bunch index)."""
import math
import os
import subprocess

import pytest

from helpers import write_input

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cli_writes_the_growth_rate_file(tmp_path):
    d = str(tmp_path)
    write_input(d, n_turns=60, interval=5, fit=(10, 50), bunches=40, macro=200)
    exe = os.path.join(ROOT, "cetasim_b200", "cetasim_mp")
    r = subprocess.run([exe, "input.dat"], cwd=d, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    res = open(os.path.join(d, "result.sdds")).read().splitlines()
    assert res[0] == "SDDS1" and len([ln for ln in res if ln and ln[0].isdigit()]) >= 60
    lines = open(os.path.join(d, "cbmgr.sdds")).read().splitlines()
    assert lines[0] == "SDDS1"
    n_par = sum(ln.startswith("&parameter") for ln in lines)
    n_col = sum(ln.startswith("&column") for ln in lines)
    assert (n_par, n_col) == (15, 28)
    pages = [i for i, ln in enumerate(lines) if ln.startswith("! page number")]
    assert len(pages) == 40
    for p, i in enumerate(pages):
        par = [float(x) for x in lines[i + 1:i + 1 + n_par]]
        assert par[0] == 8 and par[1] == p and par[11] == 2 * p  # points, index, harmonic
        n_rec = int(lines[i + 1 + n_par])
        assert n_rec == 12  # turns 0, 5, ..., 55
        rows = lines[i + 2 + n_par:i + 2 + n_par + n_rec]
        for k, row in enumerate(rows):
            v = [float(x) for x in row.split()]
            assert len(v) == n_col and v[0] == 5 * k
            assert all(math.isfinite(x) for x in v[1:4] + v[19:22])  # |X|, centroids

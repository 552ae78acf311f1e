"""The drop-in MPBeam end to end through the reference's own main.cpp.

oracle/_ref/cetasim_ref is the reference program (its main.cpp and
src/*.cpp); oracle/_ref/cetasim_dropin is the same program with
cetasim_b200/host/dropin/MPBeam.cpp linked in place of the reference's
src/MPBeam.cpp, so main.cpp, ReadInputSettings, the lattice, the fill
pattern and MPBunch::DistriGenerator are the reference's own and only the
tracking runs on the GPU.  Both read one input.dat; with the generator's
seeds fixed (the hooks of oracle/ref_shim/ref_hooks.h) both start from the
same particles, and with no ions and no radiation the runs are
deterministic, so result.sdds must agree row by row (to the 6 significant
digits the reference prints).
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

from cetasim_b200 import configs, input_dat
from oracle import ref

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(ref.EXE.replace("cetasim_ref", "cetasim_dropin")),
                                 reason="oracle/_ref/cetasim_dropin not built")]

DROPIN = ref.EXE.replace("cetasim_ref", "cetasim_dropin")


def read_sdds(path):
    """(column names, rows) of the single page of a result.sdds."""
    lines = open(path).read().splitlines()
    cols = [ln.split("name=")[1].split(",")[0] for ln in lines if ln.startswith("&column")]
    i = next(k for k, ln in enumerate(lines) if ln.startswith("! page number"))
    n = int(lines[i + 1])
    rows = [[float(v) for v in ln.split()] for ln in lines[i + 2:i + 2 + n]]
    return cols, np.array(rows)


def run(exe, d, teardown_may_crash=False):
    """Runs a program on d/input.dat.  The reference program may die after
    MPBeam::Run has returned: the PIC3D object Run builds unconditionally
    (MPBeam.cpp:887-889) frees and deletes members its constructor never set
    (PIC3D.cpp:41-65, PIC3D.h:67-88), so its exit status is accepted once
    the run printed its last line."""
    r = subprocess.run([exe, "input.dat"], cwd=d, capture_output=True, text=True, timeout=900)
    done = "End of Tracking" in r.stdout
    ok = r.returncode == 0 or (teardown_may_crash and done)
    assert ok and done, (exe, r.returncode, r.stdout[-2000:], r.stderr[-2000:])
    return read_sdds(os.path.join(d, "result.sdds"))


def case(tmp_path, turns):
    """A 40-bunch train of 300 macroparticles, 20 sections, short-range BBR
    wake (20 bins), long-range HOM wake and 9-tap FIR; synchrotron radiation
    and ions off."""
    wl = configs.make("fast_ion", n_scale=0.015)
    wl.n_macro, wl.harm, wl.ne = wl.n_macro[:40].copy(), wl.harm[:40].copy(), wl.ne[:40].copy()
    big = configs.make("batched_uneven", n_scale=0.001)
    c = wl.cfg
    c.flag_beam_ion = 0
    c.flag_synrad = 0
    c.flag_sr_wake = 1
    c.sr_bins = 20
    c.sr_bbr = configs.bbr([(5e3, 1.0, 30e9, 2e6, 1.0, 30e9, 2e6, 1.0, 30e9)])
    c.flag_lr_wake = 1
    c.lr_turns = big.cfg.lr_turns
    c.lr_bbr = big.cfg.lr_bbr
    c.flag_fir = 1
    c.fir = big.cfg.fir
    src = tmp_path / "src"
    input_dat.write_case(str(src), wl, n_turns=turns)
    dirs = []
    for name in ("ref", "gpu"):
        d = tmp_path / name
        shutil.copytree(src, d)
        dirs.append(str(d))
    return dirs


def test_dropin_result_sdds_matches_the_reference_program(tmp_path):
    dref, dgpu = case(tmp_path, 30)
    cols_r, rows_r = run(ref.EXE, dref, teardown_may_crash=True)
    cols_g, rows_g = run(DROPIN, dgpu)
    assert cols_r == cols_g
    assert rows_r.shape == rows_g.shape == (30, len(cols_r))
    for k, name in enumerate(cols_r):
        if name == "IonCharge":  # never set without ions (uninitialised in the reference)
            continue
        a, b = rows_r[:, k], rows_g[:, k]
        scale = np.max(np.abs(a)) + 1e-300
        # the reference prints 6 significant digits; eigen-emittances and the
        # x-y tilt are differences of nearly equal second moments
        rtol = 2e-4 if name.startswith(("eigenEmit", "xyCoupling")) else 2e-5
        bad = np.abs(a - b) > rtol * np.maximum(np.abs(a), 1e-3 * scale)
        assert not bad.any(), (name, a[bad][:3], b[bad][:3])
    # the run writes the files the reference writes besides result.sdds
    for f in ("elegant_filling_train_para.sdds",):
        assert open(os.path.join(dref, f)).read() == open(os.path.join(dgpu, f)).read()
    # the short-range potentials of every bunch at the print turns
    # (MPBunch.cpp:1950-2001): bins, counts and the x, y, z potentials
    pr, pg = sr_pages(os.path.join(dref, "srw_poten.sdds")), sr_pages(os.path.join(dgpu, "srw_poten.sdds"))
    assert len(pr) == len(pg) == 40
    for a, b in zip(pr, pg):
        assert a.shape == b.shape == (20, 5)
        assert np.array_equal(a[:, 1], b[:, 1])
        for k in (0, 2, 3, 4):
            scale = np.max(np.abs(a[:, k])) + 1e-300
            assert np.all(np.abs(a[:, k] - b[:, k]) <= 2e-5 * np.maximum(np.abs(a[:, k]), 1e-3 * scale)), k


def sr_pages(path):
    """The pages of a file with a header before each page group (the
    reference writes one per bunch at turn 0)."""
    lines = open(path).read().splitlines()
    pages, i = [], 0
    while i < len(lines):
        if lines[i].startswith("! page number"):
            n = int(lines[i + 1])
            pages.append(np.array([[float(v) for v in ln.split()] for ln in lines[i + 2:i + 2 + n]]))
            i += 2 + n
        else:
            i += 1
    return pages


def test_dropin_with_beam_loading_matches_the_reference_program(tmp_path):
    """The 80-bunch train with the main cavity's beam loading bin by bin and
    its direct feedback (rfMode 1; ions, wakes, feedback and radiation off):
    result.sdds of the drop-in against the reference program over 20
    turns."""
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import blcases
    wl, path, _ = blcases.build("train_binned_fb", str(tmp_path / "base"))
    # no radiation: the reference's quantum-excitation noise and the library's
    # differ (the longitudinal natural emittance follows from sdelta0)
    wl.cfg.flag_synrad = 0
    src = tmp_path / "src"
    input_dat.write_case(str(src), wl, n_turns=20, qe=False)
    dirs = []
    for name in ("ref", "gpu"):
        d = tmp_path / name
        shutil.copytree(src, d)
        dirs.append(str(d))
    cols_r, rows_r = run(ref.EXE, dirs[0], teardown_may_crash=True)
    cols_g, rows_g = run(DROPIN, dirs[1])
    assert cols_r == cols_g and rows_r.shape == rows_g.shape == (20, len(cols_r))
    for k, name in enumerate(cols_r):
        if name == "IonCharge":
            continue
        a, b = rows_r[:, k], rows_g[:, k]
        scale = np.max(np.abs(a)) + 1e-300
        rtol = 2e-4 if name.startswith(("eigenEmit", "xyCoupling")) else 2e-5
        bad = np.abs(a - b) > rtol * np.maximum(np.abs(a), 1e-3 * scale)
        assert not bad.any(), (name, a[bad][:3], b[bad][:3])
    # InitialcavityResonator's printout (MPBeam.cpp:336-426; no
    # rfTransientCavParWriteTo given, so the file is ".sdds"): header lines
    # equal, the parameters and the build-up rows to the printed digits
    tr = open(os.path.join(dirs[0], ".sdds")).read().splitlines()
    tg = open(os.path.join(dirs[1], ".sdds")).read().splitlines()
    assert len(tr) == len(tg) and [l for l in tr if l.startswith(("SDDS", "&"))] == \
        [l for l in tg if l.startswith(("SDDS", "&"))]
    for a, b in zip(tr, tg):
        if a.startswith(("SDDS", "&", "!")):
            assert a == b
            continue
        va, vb = np.array(a.split(), float), np.array(b.split(), float)
        assert np.all(np.abs(va - vb) <= 2e-5 * np.maximum(np.abs(va), 1e-300) + 1e-9), (a, b)


@pytest.mark.parametrize("case_name", ["fd_train_lr", "td_train"])
def test_dropin_with_broadband_impedance_matches_the_reference_program(tmp_path, case_name):
    """The 80-bunch train with the broadband-impedance kick (frequency domain
    with the long-range wake after it, and time domain; radiation off):
    result.sdds of the drop-in against the reference program over 20 turns."""
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import bbicases
    wl, _, _ = bbicases.build(case_name, str(tmp_path / "base"))
    wl.cfg.flag_synrad = 0
    src = tmp_path / "src"
    input_dat.write_case(str(src), wl, n_turns=20, qe=False)
    dirs = []
    for name in ("ref", "gpu"):
        d = tmp_path / name
        shutil.copytree(src, d)
        dirs.append(str(d))
    cols_r, rows_r = run(ref.EXE, dirs[0], teardown_may_crash=True)
    cols_g, rows_g = run(DROPIN, dirs[1])
    assert cols_r == cols_g and rows_r.shape == rows_g.shape == (20, len(cols_r))
    for k, name in enumerate(cols_r):
        if name == "IonCharge":
            continue
        a, b = rows_r[:, k], rows_g[:, k]
        scale = np.max(np.abs(a)) + 1e-300
        rtol = 2e-4 if name.startswith(("eigenEmit", "xyCoupling")) else 2e-5
        bad = np.abs(a - b) > rtol * np.maximum(np.abs(a), 1e-3 * scale)
        assert not bad.any(), (name, a[bad][:3], b[bad][:3])


@pytest.mark.parametrize("case_name", ["pic_train", "linear_train"])
def test_dropin_with_space_charge_matches_the_reference_program(tmp_path, case_name):
    """8 bunches of the fast-ion ring with the space-charge kick at every
    section (2.5-D PIC, and the linear model; radiation off): result.sdds of
    the drop-in against the reference program over 20 turns."""
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import sccases
    wl, _, _ = sccases.build(case_name, str(tmp_path / "base"))
    wl.cfg.flag_synrad = 0
    src = tmp_path / "src"
    input_dat.write_case(str(src), wl, n_turns=20, qe=False)
    dirs = []
    for name in ("ref", "gpu"):
        d = tmp_path / name
        shutil.copytree(src, d)
        dirs.append(str(d))
    cols_r, rows_r = run(ref.EXE, dirs[0], teardown_may_crash=True)
    cols_g, rows_g = run(DROPIN, dirs[1])
    assert cols_r == cols_g and rows_r.shape == rows_g.shape == (20, len(cols_r))
    for k, name in enumerate(cols_r):
        if name == "IonCharge":
            continue
        a, b = rows_r[:, k], rows_g[:, k]
        scale = np.max(np.abs(a)) + 1e-300
        rtol = 2e-4 if name.startswith(("eigenEmit", "xyCoupling")) else 2e-5
        bad = np.abs(a - b) > rtol * np.maximum(np.abs(a), 1e-3 * scale)
        assert not bad.any(), (name, a[bad][:3], b[bad][:3])


def read_pages(path):
    """Every page of a multi-page SDDS ASCII file: (column names, [rows per
    page]); a page's parameter lines come before its row count."""
    lines = open(path).read().splitlines()
    cols = [ln.split("name=")[1].split(",")[0] for ln in lines if ln.startswith("&column")]
    npar = sum(1 for ln in lines if ln.startswith("&parameter"))
    pages = []
    i = next(k for k, ln in enumerate(lines) if ln.startswith("&data")) + 1
    while i < len(lines):
        assert lines[i].startswith("! page number"), lines[i]
        i += 1 + npar
        n = int(lines[i])
        pages.append(np.array([[float(v) for v in ln.split()] for ln in lines[i + 1:i + 1 + n]]))
        i += 1 + n
    return cols, pages


def test_dropin_per_bunch_files_match_the_reference_program(tmp_path):
    """<runTBTBunchAverData>.sdds (every bunch's averages and the voltages of
    the loaded main cavity it saw) and <runTBTBunchProfile>_0.sdds (the
    longitudinal profile of the RF step's bins) of the 80-bunch train with
    bin-by-bin beam loading and direct feedback, every 5 turns over 20: the
    drop-in's files against the reference program's."""
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import blcases
    wl, _, _ = blcases.build("train_binned_fb", str(tmp_path / "base"))
    wl.cfg.flag_synrad = 0
    src = tmp_path / "src"
    input_dat.write_case(str(src), wl, n_turns=20, print_interval=5, qe=False,
                         extra=["runTBTBunchAverData = tbt_aver", "runTBTBunchProfile = tbt_pro",
                                "runTBTBunchDisData = tbt_dis"])
    dirs = []
    for name in ("ref", "gpu"):
        d = tmp_path / name
        shutil.copytree(src, d)
        dirs.append(str(d))
    run(ref.EXE, dirs[0], teardown_may_crash=True)
    run(DROPIN, dirs[1])
    for f in ("tbt_aver.sdds", "tbt_pro_0.sdds", "tbt_dis_0.sdds"):
        cr, pr = read_pages(os.path.join(dirs[0], f))
        cg, pg = read_pages(os.path.join(dirs[1], f))
        assert cr == cg and len(pr) == len(pg) == 4, f
        for a, b in zip(pr, pg):
            assert a.shape == b.shape
            for k, name in enumerate(cr):
                if name == "TotIonCharge":  # never set without ions
                    continue
                x, y = a[:, k], b[:, k]
                scale = np.max(np.abs(x)) + 1e-300
                if name.endswith(("Phase_0",)):
                    # angles near +-pi: compare on the circle
                    d = np.abs(np.angle(np.exp(1j * (x - y))))
                else:
                    d = np.abs(x - y)
                # tbt_aver prints 16 digits, the others the stream's 6
                rtol = 1e-7 if f == "tbt_aver.sdds" else 2e-5
                assert np.all(d <= rtol * np.maximum(np.abs(x), 1e-3 * scale) + 1e-300), (f, name)


def test_dropin_ion_dump_has_the_reference_layout(tmp_path):
    """<ionCalIonDisWriteTo>.sdds (MPBeam::SSIonDataPrint, MPBeam.cpp:
    2912-2976) of the fast-ion train over 2 turns, printed every turn: the
    drop-in's file has the reference program's header and page layout (the
    two programs draw different ion births, so the values are compared on the
    GPU against the reference harness instead, test_gpu_ref.py)."""
    wl = configs.make("fast_ion", n_scale=0.002)
    wl.cfg.flag_synrad = 0
    src = tmp_path / "src"
    input_dat.write_case(str(src), wl, n_turns=2, qe=False, extra=["ionCalIonInfoPrintInterval = 1"])
    dirs = []
    for name in ("ref", "gpu"):
        d = tmp_path / name
        shutil.copytree(src, d)
        dirs.append(str(d))
    run(ref.EXE, dirs[0], teardown_may_crash=True)
    run(DROPIN, dirs[1])

    def layout(path):
        lines = open(path).read().splitlines()
        heads, pages, i = [], [], 0
        while i < len(lines):
            if lines[i] == "SDDS1":
                j = i
                while not lines[j].startswith("&data"):
                    j += 1
                heads.append(lines[i:j + 1])
                i = j + 1
            elif lines[i].startswith("! page number"):
                page = int(lines[i].split()[-1])
                P = wl.cfg.ion.n_species
                counts = [int(v) for v in lines[i + 3:i + 3 + P]]
                tot = int(lines[i + 3 + P])
                rows = lines[i + 4 + P:i + 4 + P + tot]
                assert sum(counts) == tot and all(len(r.split()) == 8 for r in rows)
                pages.append(page)
                i += 4 + P + tot
            else:
                raise AssertionError(lines[i])
        return heads, pages

    hr, pr = layout(os.path.join(dirs[0], "ion_dis.sdds"))
    hg, pg = layout(os.path.join(dirs[1], "ion_dis.sdds"))
    assert hr == hg and pr == pg == list(range(1, 2 * wl.cfg.n_sections + 1))

"""cg_config_from_input on a small input.dat: the run settings of the
coupled-bunch growth-rate output and the fit-window checks of
ReadInputSettings.cpp:946-956."""
import ctypes as C

import pytest

from cetasim_b200 import _abi
from helpers import write_input


def parse(path, lib):
    cfg = _abi.Config()
    M = C.c_int()
    nm, hm, ne = C.POINTER(C.c_int)(), C.POINTER(C.c_int)(), C.POINTER(C.c_double)()
    rc = lib.cg_config_from_input(path.encode(), C.byref(cfg), C.byref(M), C.byref(nm),
                                  C.byref(hm), C.byref(ne))
    return rc, cfg, M.value, (nm, hm, ne)


def test_cbmgr_settings_are_read(tmp_path, lib):
    rc, cfg, M, arrays = parse(write_input(str(tmp_path)), lib)
    assert rc == 0, lib.cg_parse_error()
    assert M == 40 and cfg.n_turns == 60 and cfg.bunch_info_print_interval == 5
    assert (cfg.growth_fit_start, cfg.growth_fit_end) == (10, 50)
    assert cfg.run_cbmgr == b"cbmgr"
    assert [arrays[1][j] for j in range(3)] == [0, 2, 4]  # every second bucket
    lib.cg_config_free(C.byref(cfg), *arrays)


def test_no_cbmgr_leaves_the_name_empty(tmp_path, lib):
    rc, cfg, _, arrays = parse(write_input(str(tmp_path), cbmgr=None), lib)
    assert rc == 0 and cfg.run_cbmgr == b""
    lib.cg_config_free(C.byref(cfg), *arrays)


@pytest.mark.parametrize("fit,msg", [((50, 10), b"growthRateFittingEnd is smaller"),
                                     ((10, 80), b"nTurns small than")])
def test_fit_window_checks(tmp_path, lib, fit, msg):
    rc, *_ = parse(write_input(str(tmp_path), fit=fit), lib)
    assert rc == 1  # CG_ERR_INVALID
    assert msg in lib.cg_parse_error()


def test_resistive_wall_sectors_are_read(tmp_path, lib):
    d = str(tmp_path)
    with open(d + "/pipe.dat", "w") as f:
        f.write("radiusX radiusY length betaX betaY number sigma\n"
                "0.02 0.02 100.0 8.0 9.0 2 5.8e7\n\n0.03 0.01 20.0 10.0 7.0 3 1.4e6\n")
    path = write_input(d, extra=["runLongRangeWake = 1", "lrwNTurnsWakeTrunction = 5",
                                 "lrwPipeGeoInput = pipe.dat"])
    rc, cfg, _, arrays = parse(path, lib)
    assert rc == 0, lib.cg_parse_error()
    w = cfg.lr_rw
    assert w.n == 2 and cfg.lr_turns == 6 and cfg.lr_bbr.n == 0
    assert (w.radius_x[1], w.radius_y[1], w.length[1], w.num[1], w.sigma[1]) == \
        (0.03, 0.01, 20.0, 3.0, 1.4e6)
    lib.cg_config_free(C.byref(cfg), *arrays)

"""The reference arm of bench.py on CPU: one JSON line with the keys the
benchmark contract names, timing the reference's own compiled code
(oracle/_ref) without loading the product library."""
import json
import os
import subprocess
import sys

import pytest

from oracle import ref

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
def test_reference_arm_prints_the_contract_line(built):
    code = ("import sys; sys.argv = ['bench.py', '--impl', 'reference', '--workload', 'fast_ion', "
            "'--n-scale', '0.01', '--steps', '2', '--warmup', '1']; import bench; bench.main(); "
            "print('LIBCETAGPU', 'libcetagpu' in open('/proc/self/maps').read())")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    out = [x for x in r.stdout.strip().splitlines() if x.startswith("{") or x.startswith("LIB")]
    line = json.loads(out[-2])
    assert out[-1] == "LIBCETAGPU False"
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
              "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference" and line["value"] > 0 and line["steps"] == 2
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["value"] == line["value"]
    assert line["config"]["macroparticles"] == 80 * 200


def test_reference_arm_reports_unavailable_without_the_build(monkeypatch, capsys):
    """Without oracle/_ref the arm prints its unavailable line and exits 0."""
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setattr(ref, "available", lambda: False)
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference"])
    bench.main()
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and "unavailable" in line

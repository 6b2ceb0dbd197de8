"""The `main <file> <eps> <dim> 3` command line (main.cu:66-331 of the
reference): the reference's text format in, its gpu_stats.txt line and
DSSJ_out.txt lists out."""
import json
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "gpu_self_join_b200", "main")
GOLD = os.path.join(ROOT, "tests", "golden")


def _write_text(path, pts):
    # the reference reads tokens split on ',' and whitespace (import_dataset.cpp:49-95)
    np.savetxt(path, pts, fmt="%.9g", delimiter=",")


def test_cli_usage_and_import(tmp_path):
    r = subprocess.run([CLI], capture_output=True, text=True)
    assert "Incorrect number of input parameters" in r.stdout
    pts = np.load(os.path.join(GOLD, "test_dat_f32.npy"))[:1000]
    f = tmp_path / "d.txt"
    _write_text(f, pts)
    r = subprocess.run([CLI, str(f), "1.0", "2", "3"], capture_output=True, text=True, cwd=tmp_path)
    assert "Data import: Total data points: 1000" in r.stdout
    r = subprocess.run([CLI, str(f), "1.0", "2", "0"], capture_output=True, text=True, cwd=tmp_path)
    assert "Only search mode 3" in r.stdout


@pytest.mark.gpu
def test_cli_known_answer_and_lists(tmp_path):
    from tests.golden.make_golden import lists_digest

    pts = np.load(os.path.join(GOLD, "test_dat_f32.npy"))
    f = tmp_path / "test_dat.txt"
    _write_text(f, pts)
    env = dict(os.environ, NUMINDEXEDDIM="2", STAMP="1", PRINTNEIGHBORTABLE="1")
    r = subprocess.run([CLI, str(f), "1.0", "2", "3"], capture_output=True, text=True, cwd=tmp_path, env=env)
    assert r.returncode == 0, r.stderr
    line = (tmp_path / "gpu_stats.txt").read_text().strip().splitlines()[-1]
    fields = [x.strip() for x in line.split(",")]
    assert fields[3] == "27982028"
    assert "GPUNUMDIM/NUMINDEXEDDIM/ILP/STAMP/SORT/REORDER/SHORTCIRCUIT/QUERYREORDER/DTYPE(float/double): 2, 2, 0, 1" \
        in line
    counts, vals = [], []
    with open(tmp_path / "DSSJ_out.txt") as fh:
        assert fh.readline().startswith("#")
        for ln in fh:
            p = [int(x) for x in ln.strip().split(",") if x.strip()]
            counts.append(len(p))
            vals.extend(p)
    with open(os.path.join(GOLD, "known_answers.json")) as fh:
        known = json.load(fh)
    assert lists_digest(np.array(counts), np.array(vals)) == known["lists_sha256_device"]

"""The `splatt` command (cpd, bench -a adatm) built beside the library: the
AdaTM CLI flow of the reference (src/cmds/cmd_cpd.c, src/cmds/cmd_bench.c)
over the C ABI."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, load_golden

CLI = os.path.join(ROOT, "adatm_b200", "splatt")


@pytest.fixture(scope="module")
def cli():
    from adatm_b200.build import build
    build()
    assert os.path.exists(CLI)
    return CLI


def write_tns(path, inds, vals):
    with open(path, "w") as f:
        f.write("# written by the test\n")
        for k in range(len(vals)):
            f.write(" ".join(str(int(i) + 1) for i in inds[:, k]) + f" {float(vals[k])!r}\n")


def run(args, cwd):
    return subprocess.run(args, cwd=cwd, capture_output=True, text=True, timeout=600)


def test_help_and_argument_errors(cli, tmp_path):
    r = run([cli, "help"], tmp_path)
    assert r.returncode == 0 and "cpd" in r.stdout and "bench" in r.stdout
    r = run([cli, "bench", "x.tns", "-a", "csf"], tmp_path)
    assert r.returncode == 1 and "not recognized" in r.stderr
    r = run([cli, "cpd", "x.tns", "--tile"], tmp_path)
    assert r.returncode == 1 and "NOTILE" in r.stderr
    r = run([cli, "cpd", str(tmp_path / "missing.tns")], tmp_path)
    assert r.returncode == 1 and "unable to open" in r.stderr
    (tmp_path / "bad.tns").write_text("1 2 3 1.0\n1 2 0.5\n")
    r = run([cli, "cpd", "bad.tns"], tmp_path)
    assert r.returncode == 1 and "fields" in r.stderr


@pytest.mark.gpu
def test_cpd_matches_reference_fit_and_writes_factors(cli, tmp_path):
    d = load_golden("n4_zipf")
    write_tns(tmp_path / "t.tns", d["inds"], d["vals"])
    r = run([cli, "cpd", "t.tns", "-r", "8", "-i", "5", "--tol", "0"], tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    m = re.search(r"Final fit: (\S+)", r.stdout)
    assert m, r.stdout
    fit = float(m.group(1))
    assert abs(fit - float(d["als5_fit"])) < 1e-4
    assert "use_tags:" in r.stdout and "n_grp:" in r.stdout
    lam = np.loadtxt(tmp_path / "lambda.mat")
    assert lam.shape == (8,)
    for m, dim in enumerate(d["dims_list"]):
        a = np.loadtxt(tmp_path / f"mode{m + 1}.mat")
        assert a.shape == (dim, 8)
        np.testing.assert_allclose(np.linalg.norm(a, axis=0), 1.0, rtol=1e-6)


@pytest.mark.gpu
def test_cpd_nowrite_and_bench(cli, tmp_path):
    d = load_golden("n5_zipf")
    write_tns(tmp_path / "t.tns", d["inds"], d["vals"])
    r = run([cli, "cpd", "t.tns", "-r", "4", "-i", "3", "--nowrite"], tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "n_grp: " in r.stdout and "nan" not in r.stdout.split("Final fit:")[1]
    assert not (tmp_path / "lambda.mat").exists()
    r = run([cli, "bench", "t.tns", "-a", "adatm", "-i", "2", "-r", "8"], tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "RANK=8 ITS=2" in r.stdout

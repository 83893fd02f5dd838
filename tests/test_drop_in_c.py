"""A QuaC-style C program builds unchanged against include/quac/*.h and
links libquac_b200.so (CPU); on a GPU it runs and matches the oracle."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT


def _build(tmp_path):
    exe = tmp_path / "jc_drop_in"
    libdir = os.path.join(ROOT, "quac_b200")
    cmd = ["/usr/bin/gcc", "-std=c99", "-O2", "-Wall", "-I", os.path.join(ROOT, "include", "quac"),
           os.path.join(ROOT, "tests", "c", "jc_drop_in.c"), "-o", str(exe), "-L", libdir,
           "-lquac_b200", f"-Wl,-rpath,{libdir}", "-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_c_program_compiles_and_links(quac, tmp_path):
    _build(tmp_path)


@pytest.mark.gpu
def test_c_program_runs_and_matches_oracle(quac, oracle, tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([str(exe), "-ts_rk_type", "4", "-ts_adapt_type", "none"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    vals = {ln.split()[0]: float(ln.split()[1]) for ln in r.stdout.splitlines()
            if ln.startswith(("final_", "trace"))}
    steps = [ln.split() for ln in r.stdout.splitlines() if ln.startswith("step ")]
    assert [int(s[1]) for s in steps] == list(range(0, 201, 50))
    S = oracle.OSys()
    from quac_b200.systems import jc
    jc(S)
    h = S.csr_handle()
    x0 = np.zeros(400, dtype=complex)
    x0[10 * 20 + 10] = 1.0
    y = oracle.rk4(h, x0, 0.01, 200)
    oracle.free_csr(h)
    assert abs(vals["final_qb"] - oracle.expect_dm([2, 10], y, (0, 0, -1)).real) < 1e-12
    assert abs(vals["final_cav"] - oracle.expect_dm([2, 10], y, (0, 1, -1)).real) < 1e-12
    assert abs(vals["trace"] - 1.0) < 1e-12


def _build_ens(tmp_path):
    exe = tmp_path / "ensemble_drop_in"
    libdir = os.path.join(ROOT, "quac_b200")
    cmd = ["/usr/bin/gcc", "-std=c99", "-O2", "-Wall", "-I", os.path.join(ROOT, "include", "quac"),
           os.path.join(ROOT, "tests", "c", "ensemble_drop_in.c"), "-o", str(exe), "-L", libdir,
           "-lquac_b200", f"-Wl,-rpath,{libdir}", "-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_c_ensemble_program_compiles_and_links(quac, tmp_path):
    _build_ens(tmp_path)


@pytest.mark.gpu
def test_c_ensemble_program_matches_oracle(quac, oracle, tmp_path):
    exe = _build_ens(tmp_path)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    rows = [ln.split() for ln in r.stdout.splitlines() if ln.startswith("inst ")]
    assert len(rows) == 16
    from quac_b200.systems import driven_jc
    for row in rows:
        i, nc, pe = int(row[1]), int(row[2]), float(row[3])
        S = oracle.OSys()
        driven_jc(S, nc, 0.1 * (i % 5) - 0.2, 0.05 + 0.01 * i, 0.02 * i, 0.01 + 0.005 * i)
        h = S.csr_handle()
        D = 2 * nc
        x0 = np.zeros(D * D, dtype=complex)
        x0[nc * D + nc] = 1.0
        y, _, _ = oracle.dp5(h, x0, 0.0, 2.0, 0.05)
        oracle.free_csr(h)
        rho = y.reshape(D, D, order="F")
        assert abs(pe - rho.diagonal().real[nc:].sum()) < 1e-10, i


def test_c_fock_loc_with_int_literals(quac, tmp_path):
    """get_qvec_loc_fock_op called from C with int literals for the Fock
    states (four pairs, so some travel on the stack): the index is
    sum fock_i * n_before_i = 1 + 2*2 + 3*6 + 1*24 = 47 (qvec_utilities.c:
    996-1033), and 47 * 48 + 47 for a density matrix."""
    exe = tmp_path / "fock_loc"
    libdir = os.path.join(ROOT, "quac_b200")
    cmd = ["/usr/bin/gcc", "-std=c99", "-O2", "-Wall", "-I", os.path.join(ROOT, "include", "quac"),
           os.path.join(ROOT, "tests", "c", "fock_loc.c"), "-o", str(exe), "-L", libdir,
           "-lquac_b200", f"-Wl,-rpath,{libdir}", "-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    got = dict(ln.split() for ln in r.stdout.splitlines())
    assert got == {"wf": "47", "dm": str(47 * 48 + 47)}

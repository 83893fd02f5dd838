"""C-ABI and host-side logic, no GPU needed.

- libquac_b200.so loads and exports every function include/quac_b200.h
  declares;
- the term compiler (recorded add_ham_term/add_lin_term products -> the
  matrix-free tables the kernels read) reproduces the reference's golden
  superoperator matrices when its tables are expanded back into a sparse
  matrix -- checked through quac_program_export, which never touches CUDA;
- circuit layer scheduling (quantum_circuits.c:316-404).
"""
import ctypes
import os
import re

import numpy as np
import pytest
import scipy.sparse as sp

import fixture_systems as F
from conftest import ROOT, golden_csr


def _declared_functions():
    src = open(os.path.join(ROOT, "include", "quac_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = set()
    for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\(([^;{]*)\)\s*;", src, re.M):
        line = m.group(0)
        if line.lstrip().startswith(("typedef", "#", "return")):
            continue
        names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_symbol(quac):
    L = quac.lib()
    names = _declared_functions()
    assert len(names) > 60
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


class _Builder:
    """Replays fixture scripts through the product's own Python API."""

    def __init__(self, q):
        self.q = q
        self.qs = q.initialize_system()

    def op(self, levels):
        return self.q.create_op_sys(self.qs, levels)

    def ham(self, a, *ops):
        self.q.add_ham_term(self.qs, a, *ops)

    def lin(self, a, *ops):
        self.q.add_lin_term(self.qs, a, *ops)


def export_matrix(q, qs, mode):
    L = q.lib()
    f = L.quac_program_export
    f.restype = ctypes.c_int
    f.argtypes = [type(qs._ptr), ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    counts = np.zeros(6, dtype=np.int64)
    assert f(qs._ptr, mode, counts.ctypes.data, None, None) == 0
    D, nc, nL, nR, nJ, nJd = (int(x) for x in counts)
    maps = np.zeros(max(1, (nL + nR + nJ) * D), dtype=np.int32)
    vals = np.zeros(max(1, (nL + nR + 2 * nJ + 2 * nJd + 2) * D), dtype=np.complex128)
    assert f(qs._ptr, mode, counts.ctypes.data, maps.ctypes.data, vals.ctypes.data) == 0
    mp = maps[:(nL + nR + nJ) * D].reshape(-1, D) if nL + nR + nJ else np.zeros((0, D), int)
    vv = vals.reshape(-1, D)
    Lm, Rm, Jm = mp[:nL], mp[nL:nL + nR], mp[nL + nR:]
    k = 0
    Lv = vv[k:k + nL]; k += nL
    Rv = vv[k:k + nR]; k += nR
    Jr = vv[k:k + nJ]; k += nJ
    Jc = vv[k:k + nJ]; k += nJ
    Jdr = vv[k:k + nJd]; k += nJd
    Jdc = vv[k:k + nJd]; k += nJd
    dr, dc = vv[k], vv[k + 1]
    rows, cols, data = [], [], []
    if nc == 1:
        r = np.arange(D)
        rows.append(r); cols.append(r); data.append(dr)
        for t in range(nL):
            ok = Lm[t] >= 0
            rows.append(r[ok]); cols.append(Lm[t][ok]); data.append(Lv[t][ok])
        n = D
    else:
        r, c = np.meshgrid(np.arange(D), np.arange(D), indexing="ij")
        r, c = r.ravel(), c.ravel()
        i = c * D + r
        diag = dr[r] + dc[c]
        for t in range(nJd):
            diag = diag + Jdr[t][r] * Jdc[t][c]
        rows.append(i); cols.append(i); data.append(diag)
        for t in range(nL):
            ok = Lm[t][r] >= 0
            rows.append(i[ok]); cols.append(c[ok] * D + Lm[t][r][ok]); data.append(Lv[t][r][ok])
        for t in range(nR):
            ok = Rm[t][c] >= 0
            rows.append(i[ok]); cols.append(Rm[t][c][ok] * D + r[ok]); data.append(Rv[t][c][ok])
        for t in range(nJ):
            ok = (Jm[t][r] >= 0) & (Jm[t][c] >= 0)
            rows.append(i[ok]); cols.append(Jm[t][c][ok] * D + Jm[t][r][ok])
            data.append(Jr[t][r][ok] * Jc[t][c][ok])
        n = D * D
    return sp.csr_matrix((np.concatenate(data), (np.concatenate(rows), np.concatenate(cols))),
                         shape=(n, n))


@pytest.mark.parametrize("case", F.CASES, ids=lambda c: f"{c[0]}-{c[1]}op-{c[2]}-{'c' if c[3] else 'r'}")
def test_term_compiler_reproduces_fixture(quac, golden, case):
    fam, nop, kind, cplx = case
    B = _Builder(quac)
    stems = F.build(B, fam, nop, kind, cplx)
    mode = 1 if fam == "ham_only" else 0
    A = export_matrix(quac, B.qs, mode)
    ref = sum(golden_csr(golden, s) for s in stems)
    assert sp.linalg.norm(A - ref) <= 1e-9
    B.qs.destroy()


@pytest.mark.parametrize("case", F.CASES, ids=lambda c: f"{c[0]}-{c[1]}op-{c[2]}-{'c' if c[3] else 'r'}")
def test_superoperator_binary_matches_fixture(quac, golden, case, tmp_path):
    """The operator written in PETSc's binary AIJ format (the format of the
    reference's fixtures) reads back as the fixture matrix; rows are sorted
    by column with the diagonal always present."""
    fam, nop, kind, cplx = case
    B = _Builder(quac)
    stems = F.build(B, fam, nop, kind, cplx)
    path = tmp_path / "op.dat"
    quac.write_superoperator_binary(B.qs, str(path))
    (m, n), rowptr, cols, vals = quac.read_petsc_binary_matrix(str(path))
    A = sp.csr_matrix((vals, cols, rowptr), shape=(m, n))
    ref = sum(golden_csr(golden, s) for s in stems)
    assert (m, n) == ref.shape
    assert sp.linalg.norm(A - ref) <= 1e-9
    for i in range(m):
        row = cols[rowptr[i]:rowptr[i + 1]]
        assert np.all(np.diff(row) > 0) and i in row
    B.qs.destroy()


def test_term_compiler_vec_ops_match_oracle(quac, oracle):
    q = quac
    qs = q.initialize_system()
    v = q.create_vec_op_sys(qs, 3)
    o = q.create_op_sys(qs, 2)
    q.add_ham_term(qs, 0.7, v[0], v[2])
    q.add_ham_term(qs, 0.7, v[2], v[0])
    q.add_lin_term(qs, 0.3, v[1], v[2], o)
    q.add_lin_term(qs, 0.2, o.n)
    A = export_matrix(q, qs, 0)
    S = oracle.OSys()
    vs = S.vec(3)
    os_ = S.op(2)
    S.ham(0.7, vs[0], vs[2]); S.ham(0.7, vs[2], vs[0])
    S.lin(0.3, vs[1], vs[2], os_.a); S.lin(0.2, os_.n)
    assert sp.linalg.norm(A - S.liouvillian()) <= 1e-12
    qs.destroy()


def test_schedule_circuit_layers(quac):
    q = quac
    qs = q.initialize_system()
    for _ in range(3):
        q.create_op_sys(qs, 2)
    c = q.create_circuit(6)
    q.add_gate_to_circuit_sys(c, 0.0, "HADAMARD", 0)
    q.add_gate_to_circuit_sys(c, 0.0, "HADAMARD", 1)
    q.add_gate_to_circuit_sys(c, 0.0, "CNOT", 0, 1)
    q.add_gate_to_circuit_sys(c, 0.0, "RZ", 2, 0.5)
    q.add_gate_to_circuit_sys(c, 0.0, "CNOT", 1, 2)
    q.schedule_circuit_layers(qs, c)
    assert c.c.num_layers == 3
    assert c.c.num_gates == 5
    qs.destroy()


def test_error_mode_returns_instead_of_exiting(quac):
    q = quac
    qs = q.initialize_system()
    with pytest.raises(q.QuacError):
        q.construct_matrix(qs)  # no operators yet
    qs.destroy()


def test_solver_option_setters_validate_on_the_host(quac):
    """The steady-state and L.x option setters check their arguments before
    touching any device state; each rejected value leaves the option as it
    was (a later valid call still succeeds)."""
    q = quac
    for setter, good, bad in [(q.set_gmres_precision, (1, 0), (2, -1)),
                              (q.set_deflation_refresh, (0, 1), (2,)),
                              (q.set_gmres_restart, (300, 1024, 100), (0, 1025)),
                              (q.set_hermitian_mode, (0, 1), (3,)),
                              (q.set_gmres_preconditioner, (0, 2, 1), (3, -1)),
                              (q.set_gmres_tolerance, (1e-12, 1e-11), (0.0, -1e-3, 1.0)),
                              (q.set_lrho_precision, (1, 0), (2,))]:
        for v in bad:
            with pytest.raises(q.QuacError):
                setter(v)
        for v in good:
            setter(v)


def test_qvec_loc_fock_op_host(quac):
    """qvec_utilities.c:996-1033: the index is sum_i fock_i * n_before_i, the
    diagonal (loc, loc) for a density matrix; a Fock state outside
    [0, levels) is an error.  Pure host arithmetic on the qvec header."""
    import ctypes
    import types
    q = quac
    qs = q.initialize_system()
    a, b, c = q.create_op_sys(qs, 2), q.create_op_sys(qs, 3), q.create_op_sys(qs, 4)
    assert (a.n_before, b.n_before, c.n_before) == (1, 2, 6)

    def header(kind, n):
        s = q._QvecStruct()
        s.my_type, s.n = kind, n
        return types.SimpleNamespace(_ptr=ctypes.pointer(s), keep=s)

    wf, dm = header(q.WAVEFUNCTION, 24), header(q.DENSITY_MATRIX, 24 * 24)
    assert q.get_qvec_loc_fock_op(wf, a, 1, b, 2, c, 3) == 1 + 2 * 2 + 3 * 6
    assert q.get_qvec_loc_fock_op(wf, b, 1) == 2
    assert q.get_qvec_loc_fock_op(dm, a, 1, c, 1) == 7 * 24 + 7
    for bad in (2, -1):
        with pytest.raises(q.QuacError):
            q.get_qvec_loc_fock_op(wf, a, bad)
    qs.destroy()

"""System definitions behind the reference's golden superoperator fixtures.

Each reference test in tests/matrix_construction_test_{ham,lin,ham_only,
ham_lin}_op.c builds a small system (a 2-, 3- and 4-level subsystem, or a
single qubit for the Pauli cases), adds a fixed list of operator products
with coefficients omega_k (real, or the same times i for the *_c cases),
calls construct_matrix and compares qsys->mat_A with a PETSc-binary file
under tests/pristine_matrices/ by Frobenius norm (<= 1e-9, t_helpers.h).

``build(S, family, nop, kind, cplx)`` replays those scripts on any builder
``S`` that offers ``op(levels)`` returning an object with attributes
a/dag/n/eye/sig_x/sig_y/sig_z, plus ``ham(a, *ops)`` and ``lin(a, *ops)``.
It returns the fixture file stem(s) the result must match.

Citations: ham scripts matrix_construction_test_ham_op.c:17-506, lin
scripts matrix_construction_test_lin_op.c:15-493, ham-only scripts
matrix_construction_test_ham_only_op.c, ham+lin
matrix_construction_test_ham_lin_op.c:16-...
"""


def _basic_lists(o2, o3, o4, nop):
    # (coefficient slot, operator list)
    if nop == 1:
        return [(2, [o2.a]), (2, [o2.dag]), (2, [o2.n]),
                (1, [o3.a]), (1, [o3.dag]), (1, [o3.n]),
                (0.5, [o4.a]), (0.5, [o4.dag]), (0.5, [o4.n])]
    if nop == 2:
        return [(2, [o2.a, o2.dag]), (2, [o2.dag, o2.a]), (2, [o2.n, o2.dag]),
                (1, [o3.a, o3.a]), (1, [o3.dag, o3.dag]), (1, [o3.n, o3.a]),
                (0.5, [o4.a, o4.n]), (0.5, [o4.dag, o4.n]), (0.5, [o4.n, o4.n]),
                (0.25, [o4.a, o3.n]), (0.25, [o3.dag, o2.n]), (0.25, [o2.n, o4.n])]
    return [(2, [o2.a, o2.dag, o2.n]), (2, [o2.dag, o2.a, o2.n]), (2, [o2.n, o2.dag, o2.a]),
            (1, [o3.a, o3.a, o3.a]), (1, [o3.dag, o3.dag, o3.dag]), (1, [o3.n, o3.a, o3.n]),
            (0.5, [o4.a, o4.n, o4.dag]), (0.5, [o4.dag, o4.n, o4.a]), (0.5, [o4.n, o4.n, o4.n]),
            (0.25, [o4.a, o3.n, o2.dag]), (0.25, [o3.dag, o2.n, o4.a]),
            (0.25, [o2.n, o4.n, o3.n])]


def _pauli_lists(o2, nop):
    if nop == 1:
        return [(2, [o2.sig_x]), (2, [o2.sig_y]), (2, [o2.sig_z]), (2, [o2.eye])]
    if nop == 2:
        return [(2, [o2.sig_x, o2.sig_y]), (2, [o2.sig_y, o2.sig_z]), (2, [o2.sig_z, o2.sig_x]),
                (2, [o2.eye, o2.eye])]
    return [(2, [o2.sig_x, o2.sig_x, o2.sig_z]), (2, [o2.sig_y, o2.sig_y, o2.sig_x]),
            (2, [o2.sig_z, o2.sig_z, o2.sig_y]), (2, [o2.eye, o2.eye, o2.eye])]


def build(S, family, nop, kind, cplx):
    """family in {"ham", "lin", "ham_only", "ham_lin"}; kind in {"basic","pauli"}.
    Returns the list of fixture stems whose sum the matrix must equal."""
    mul = 1j if cplx else 1.0
    if kind == "basic":
        o2, o3, o4 = S.op(2), S.op(3), S.op(4)
        lists = _basic_lists(o2, o3, o4, nop)
        zero_lin_op = o4.n if nop == 1 else o3.n
    else:
        o2 = S.op(2)
        lists = _pauli_lists(o2, nop)
        zero_lin_op = o2.n
    if family in ("ham", "ham_only", "ham_lin"):
        for w, ops in lists:
            S.ham(w * mul, *ops)
    if family in ("lin", "ham_lin"):
        for w, ops in lists:
            S.lin(w * mul, *ops)
    if family == "ham":
        S.lin(0.0, zero_lin_op)  # forces the density-matrix equations
    stem = f"{nop}op_{'b' if kind == 'basic' else 'p'}{'c' if cplx else 'r'}"
    if family == "ham_lin":
        return [f"ham_{stem}", f"lin_{stem}"]
    return [f"{family}_{stem}"]


CASES = [(fam, nop, kind, cplx)
         for fam in ("ham", "lin", "ham_only", "ham_lin")
         for nop in (1, 2, 3)
         for kind in ("basic", "pauli")
         for cplx in (False, True)]

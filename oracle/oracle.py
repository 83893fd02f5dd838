"""Python handle on the CPU oracle (test infrastructure only).

The oracle is a plain-C restatement of QuaC's Lindblad path (see
quac_oracle.c for the reference file:line of every routine).  Only the tests,
``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import this
module; the product package ``quac_b200`` never does.

A system is described here the way a QuaC program builds it: subsystems are
created in order (subsystem 0 is the most significant Hilbert digit), each
basic operator is a (type, subsystem, position) triple, and terms are
(kind, coefficient, [ops...]) with kind 1 = Hamiltonian, 2 = Lindblad.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liborc.so")

# operator types (operators_p.h:6-16)
RAISE, NUMBER, LOWER, VEC, SIGMA_X, SIGMA_Y, SIGMA_Z, IDENTITY, OTHER = -1, 0, 1, 2, 3, 4, 5, 6, 7
HAM, LINDBLAD = 1, 2
MODE_DM, MODE_WF, MODE_MCWF = 0, 1, 2

# gate numbering (quantum_gates.h:11-33)
GATES = dict(SQiSWP=-8, CZ_ARP=-7, CUSTOM2QGATE=-6, CZX=-5, CmZ=-4, CZ=-3, CXZ=-2, CNOT=-1,
             HADAMARD=1, SIGMAX=2, SIGMAY=3, SIGMAZ=4, EYE=5, RX=6, RY=7, RZ=8, U1=9, U2=10,
             U3=11, CUSTOM1QGATE=12)


def build():
    """Compile liborc.so with the Makefile next to this file."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        vp, i64, dbl = ctypes.c_void_p, ctypes.c_int64, ctypes.c_double
        L.orc_build.restype = vp
        L.orc_build.argtypes = [ctypes.c_int, vp, ctypes.c_int, vp, vp, vp, vp, ctypes.c_int,
                                ctypes.c_int, i64, i64]
        L.orc_csr_free.argtypes = [vp]
        L.orc_csr_nnz.restype = i64
        L.orc_csr_nnz.argtypes = [vp]
        L.orc_csr_nrows.restype = i64
        L.orc_csr_nrows.argtypes = [vp]
        L.orc_csr_export.argtypes = [vp, vp, vp, vp]
        L.orc_spmv.argtypes = [vp, vp, vp]
        L.orc_rk4.argtypes = [vp, vp, dbl, i64]
        L.orc_bs3.restype = i64
        L.orc_bs3.argtypes = [vp, vp, dbl, dbl, dbl, dbl, dbl, dbl, dbl, i64, vp]
        L.orc_dp5.restype = i64
        L.orc_dp5.argtypes = [vp, vp, dbl, dbl, dbl, dbl, dbl, dbl, dbl, i64, vp]
        L.orc_expect_dm.argtypes = [ctypes.c_int, vp, ctypes.c_int, vp, vp, vp]
        L.orc_expect_wf.argtypes = [ctypes.c_int, vp, ctypes.c_int, vp, vp, vp]
        L.orc_gate_superop.argtypes = [ctypes.c_int, vp, ctypes.c_int, ctypes.c_int, vp, dbl, dbl,
                                       dbl, vp, vp, ctypes.c_int]
        L.orc_gate_inplace.argtypes = [ctypes.c_int, vp, ctypes.c_int, ctypes.c_int, vp, dbl, dbl,
                                       dbl, vp, vp, ctypes.c_int]
        L.orc_add_trace_row.restype = vp
        L.orc_add_trace_row.argtypes = [vp, i64]
        L.orc_gmres_ilu.restype = i64
        L.orc_gmres_ilu.argtypes = [vp, vp, dbl, ctypes.c_int, i64, ctypes.c_int]
        L.orc_num_threads.restype = ctypes.c_int
        L.orc_mcwf.restype = ctypes.c_int
        L.orc_mcwf.argtypes = [vp, ctypes.c_int, vp, vp, vp, ctypes.c_int, vp, vp, ctypes.c_uint64, dbl, dbl,
                               dbl, dbl, dbl, dbl, dbl, ctypes.c_int, i64, vp]
        L.orc_mcwf_draw.restype = dbl
        L.orc_mcwf_draw.argtypes = [ctypes.c_uint64, i64, ctypes.c_uint64]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class OpSet:
    """The operator family create_op_sys makes for one subsystem."""

    def __init__(self, sub, levels):
        self.sub, self.levels = sub, levels
        self.a = (LOWER, sub, -1)
        self.dag = (RAISE, sub, -1)
        self.n = (NUMBER, sub, -1)
        self.eye = (IDENTITY, sub, -1)
        self.sig_x = (SIGMA_X, sub, -1)
        self.sig_y = (SIGMA_Y, sub, -1)
        self.sig_z = (SIGMA_Z, sub, -1)
        self.other = (OTHER, sub, -1)


class OSys:
    """A QuaC-style system description for the oracle."""

    def __init__(self):
        self.levels = []
        self.terms = []

    @property
    def D(self):
        return int(np.prod(self.levels)) if self.levels else 1

    def op(self, levels):
        self.levels.append(int(levels))
        return OpSet(len(self.levels) - 1, levels)

    def vec(self, levels):
        self.levels.append(int(levels))
        sub = len(self.levels) - 1
        return [(VEC, sub, k) for k in range(levels)]

    def ham(self, a, *ops):
        self.terms.append((HAM, complex(a), list(ops)))

    def lin(self, a, *ops):
        self.terms.append((LINDBLAD, complex(a), list(ops)))

    @property
    def has_lindblad(self):
        return any(k == LINDBLAD for k, _, _ in self.terms)

    def _flat(self):
        kinds = np.array([k for k, _, _ in self.terms], dtype=np.int32)
        coef = np.array([[a.real, a.imag] for _, a, _ in self.terms], dtype=np.float64).reshape(-1)
        nops = np.array([len(o) for _, _, o in self.terms], dtype=np.int32)
        trip = np.array([t for _, _, o in self.terms for t in o], dtype=np.int32).reshape(-1)
        if trip.size == 0:
            trip = np.zeros(3, dtype=np.int32)
        return kinds, coef, nops, trip

    def liouvillian(self, mode=MODE_DM, conj_compat=False, rows=None):
        """Assembled operator (construct_matrix) as a scipy CSR matrix.
        ``rows=(r0, r1)`` assembles only that row block (like one MPI rank)."""
        import scipy.sparse as sp
        L = lib()
        lv = np.array(self.levels, dtype=np.int64)
        kinds, coef, nops, trip = self._flat()
        r0, r1 = rows if rows is not None else (0, -1)
        h = L.orc_build(len(self.levels), _p(lv), len(self.terms), _p(kinds), _p(coef), _p(nops),
                        _p(trip), mode, int(conj_compat), r0, r1)
        try:
            nr, nnz = L.orc_csr_nrows(h), L.orc_csr_nnz(h)
            rowptr = np.zeros(nr + 1, dtype=np.int64)
            col = np.zeros(max(nnz, 1), dtype=np.int64)
            val = np.zeros(max(nnz, 1), dtype=np.complex128)
            L.orc_csr_export(h, _p(rowptr), _p(col), _p(val))
        finally:
            L.orc_csr_free(h)
        dim = self.D ** 2 if mode == MODE_DM else self.D
        return sp.csr_matrix((val[:nnz], col[:nnz], rowptr), shape=(nr, dim))

    def csr_handle(self, mode=MODE_DM, rows=None):
        """Opaque oracle CSR (caller frees with free_csr)."""
        L = lib()
        lv = np.array(self.levels, dtype=np.int64)
        kinds, coef, nops, trip = self._flat()
        r0, r1 = rows if rows is not None else (0, -1)
        return L.orc_build(len(self.levels), _p(lv), len(self.terms), _p(kinds), _p(coef),
                           _p(nops), _p(trip), mode, 0, r0, r1)


def free_csr(h):
    lib().orc_csr_free(h)


def spmv(h, x):
    x = np.ascontiguousarray(x, dtype=np.complex128)
    y = np.zeros(lib().orc_csr_nrows(h), dtype=np.complex128)
    lib().orc_spmv(h, _p(x), _p(y))
    return y


def rk4(h, y0, dt, nsteps):
    y = np.array(y0, dtype=np.complex128, copy=True)
    lib().orc_rk4(h, _p(y), float(dt), int(nsteps))
    return y


def bs3_events(h, y0, t0, tmax, dt0, events, atol=5e-7, rtol=5e-7, hmin=0.01, hmax=1.0, max_steps=10 ** 9):
    """Bogacki-Shampine 3(2) with the basic controller of time_step_sys
    (qsystem.c:895-1098) and circuit events: a step that would pass the next
    event time ends on it, the events at that time are applied in order
    (event callables y -> y), and the controller continues from that step
    (_sys_QC_EventFunction / PostEventFunction, quantum_circuits.c:17-120).
    `events` is a list of (time, callable) sorted by time."""
    y = np.array(y0, dtype=np.complex128, copy=True)
    n = y.size
    t, hh = t0, dt0
    tol = 1e-12 * max(1.0, abs(tmax))
    ev = [(te, f) for te, f in events if te > t0 and te <= tmax * (1 + 1e-14) + 1e-14]
    k, steps = 0, 0
    while steps < max_steps and t < tmax - tol:
        h_try, last, at_event = hh, False, False
        if t + h_try >= tmax - tol:
            h_try, last = tmax - t, True
        if k < len(ev) and t + h_try >= ev[k][0] - tol:
            h_try, at_event, last = ev[k][0] - t, True, abs(ev[k][0] - tmax) <= tol
        k1 = spmv(h, y)
        k2 = spmv(h, y + 0.5 * h_try * k1)
        k3 = spmv(h, y + 0.75 * h_try * k2)
        yn = y + h_try * (2.0 / 9.0 * k1 + 1.0 / 3.0 * k2 + 4.0 / 9.0 * k3)
        k4 = spmv(h, yn)
        e = h_try * ((2.0 / 9.0 - 7.0 / 24.0) * k1 + (1.0 / 3.0 - 0.25) * k2 + (4.0 / 9.0 - 1.0 / 3.0) * k3
                     - 0.125 * k4)
        q = np.abs(e) / (atol + rtol * np.maximum(np.abs(y), np.abs(yn)))
        err = np.sqrt(np.sum(q * q) / n)
        fac = min(10.0, max(0.1, 0.9 * err ** (-1.0 / 3.0) if err > 0 else 10.0))
        h_next = min(hmax, max(hmin, h_try * fac))
        if not (err <= 1.0 or h_try <= hmin * (1 + 1e-12)):
            hh = h_next
            continue
        y = yn
        steps += 1
        t = tmax if last else t + h_try
        hh = h_next
        if at_event:
            te = ev[k][0]
            while k < len(ev) and abs(ev[k][0] - te) <= tol:
                y = ev[k][1](y)
                k += 1
    return y, steps


def rk4_time_dep(h0, terms, y0, t0, dt, nsteps, min_time_dep=1e-10):
    """Classical RK4 on Y = A X + sum_k a_k f_k(t) A_k X, the matrix-shell
    product of qsystem.c:1300-1330: `h0` is the CSR of the time-independent
    terms, `terms` a list of (csr handle of the term built with coefficient
    1, a_k, f_k); a term whose |a_k f_k(t)| is at most min_time_dep
    (qsystem.c:34) is skipped at that time."""
    def rhs(t, x):
        y = spmv(h0, x)
        for hk, a, f in terms:
            s = a * f(t)
            if abs(s) > min_time_dep:
                y = y + s * spmv(hk, x)
        return y

    y = np.array(y0, dtype=np.complex128, copy=True)
    t = t0
    for _ in range(nsteps):
        k1 = rhs(t, y)
        k2 = rhs(t + dt / 2, y + dt / 2 * k1)
        k3 = rhs(t + dt / 2, y + dt / 2 * k2)
        k4 = rhs(t + dt, y + dt * k3)
        y = y + dt / 6 * (k1 + 2 * k2 + 2 * k3 + k4)
        t = t0 + (_ + 1) * dt
    return y


def bs3(h, y0, t0, tmax, dt0, atol=5e-7, rtol=5e-7, hmin=0.01, hmax=1.0, max_steps=10 ** 9):
    y = np.array(y0, dtype=np.complex128, copy=True)
    nrej = ctypes.c_int64(0)
    nacc = lib().orc_bs3(h, _p(y), t0, tmax, dt0, atol, rtol, hmin, hmax, max_steps,
                         ctypes.byref(nrej))
    return y, nacc, nrej.value


def dp5(h, y0, t0, tmax, dt0, atol=5e-7, rtol=5e-7, hmin=0.01, hmax=1.0, max_steps=10 ** 9):
    y = np.array(y0, dtype=np.complex128, copy=True)
    nrej = ctypes.c_int64(0)
    nacc = lib().orc_dp5(h, _p(y), t0, tmax, dt0, atol, rtol, hmin, hmax, max_steps,
                         ctypes.byref(nrej))
    return y, nacc, nrej.value


def _trip(ops):
    return np.array([t for t in ops], dtype=np.int32).reshape(-1)


def expect_dm(levels, rho, *ops):
    lv = np.array(levels, dtype=np.int64)
    out = np.zeros(2)
    r = np.ascontiguousarray(rho, dtype=np.complex128)
    lib().orc_expect_dm(len(levels), _p(lv), len(ops), _p(_trip(ops)), _p(r), _p(out))
    return complex(out[0], out[1])


def expect_wf(levels, psi, *ops):
    lv = np.array(levels, dtype=np.int64)
    out = np.zeros(2)
    r = np.ascontiguousarray(psi, dtype=np.complex128)
    lib().orc_expect_wf(len(levels), _p(lv), len(ops), _p(_trip(ops)), _p(r), _p(out))
    return complex(out[0], out[1])


def _custom(custom, n):
    c = np.zeros(2 * n * n)
    if custom is not None:
        m = np.asarray(custom, dtype=np.complex128).reshape(n, n)
        c[0::2], c[1::2] = m.real.reshape(-1), m.imag.reshape(-1)
    return c


def gate_superop(levels, state, gate, qubits, theta=0.0, phi=0.0, lam=0.0, custom=None, is_dm=True):
    """_apply_gate_sys: returns the new state (column-stacked rho or psi)."""
    g = GATES[gate] if isinstance(gate, str) else int(gate)
    lv = np.array(levels, dtype=np.int64)
    q = np.array(qubits, dtype=np.int32)
    c = _custom(custom, 2 if len(qubits) == 1 else 4)
    s = np.array(state, dtype=np.complex128, copy=True)
    lib().orc_gate_superop(len(levels), _p(lv), g, len(qubits), _p(q), theta, phi, lam, _p(c),
                           _p(s), int(is_dm))
    return s


def gate_inplace(dims, state, gate, qubits, theta=0.0, phi=0.0, lam=0.0, custom=None, is_dm=True):
    """_apply_gate2: ``dims`` is the qvec's hspace_dims ([L..., L...] for a DM)."""
    g = GATES[gate] if isinstance(gate, str) else int(gate)
    d = np.array(dims, dtype=np.int64)
    q = np.array(qubits, dtype=np.int32)
    c = _custom(custom, 2 if len(qubits) == 1 else 4)
    s = np.array(state, dtype=np.complex128, copy=True)
    lib().orc_gate_inplace(len(dims), _p(d), g, len(qubits), _p(q), theta, phi, lam, _p(c), _p(s),
                           int(is_dm))
    return s


def steady_state(osys, rtol=1e-11, restart=100, maxit=20000, use_ilu=True):
    """solver.c:33-221 on the full Liouvillian: returns (x, iterations)."""
    L = lib()
    h = osys.csr_handle(MODE_DM)
    b = L.orc_add_trace_row(h, osys.D)
    L.orc_csr_free(h)
    x = np.zeros(osys.D ** 2, dtype=np.complex128)
    x[0] = 1.0
    try:
        its = L.orc_gmres_ilu(b, _p(x), rtol, restart, maxit, int(use_ilu))
    finally:
        L.orc_csr_free(b)
    return x, its


class McwfEnsemble:
    """Trajectory ensemble of the oracle's MCWF restatement (orc_mcwf):
    states (ntraj x D), thresholds and draw counters, spawned from psi0 like
    the engine (threshold = draw 0, counter 1)."""

    def __init__(self, osys, psi0, ntraj, seed):
        L = lib()
        self.D = osys.D
        self.ntraj = ntraj
        self.seed = seed
        self.heff = osys.csr_handle(MODE_MCWF)
        self.jumps, a = [], []
        for kind, coef, ops in osys.terms:
            if kind != LINDBLAD or coef == 0:
                continue
            one = OSys()
            one.levels = list(osys.levels)
            one.ham(1j, *ops)  # -i (i C) = C in the Schroedinger form
            self.jumps.append(one.csr_handle(MODE_WF))
            a += [coef.real, coef.imag]
        self.a = np.array(a if a else [0.0, 0.0], dtype=np.float64)
        self.psi = np.tile(np.asarray(psi0, dtype=np.complex128), (ntraj, 1)).copy()
        self.thr = np.array([L.orc_mcwf_draw(seed, i, 0) for i in range(ntraj)], dtype=np.float64)
        self.cnt = np.ones(ntraj, dtype=np.uint64)
        self.stats = np.zeros(2 * ntraj, dtype=np.int64)

    def run(self, t0, tmax, dt, scheme=0, atol=5e-7, rtol=5e-7, hmin=0.01, hmax=1.0, max_steps=10 ** 9):
        L = lib()
        arr = (ctypes.c_void_p * max(1, len(self.jumps)))(*self.jumps)
        st = L.orc_mcwf(self.heff, len(self.jumps), ctypes.cast(arr, ctypes.c_void_p), _p(self.a), _p(self.psi),
                        self.ntraj, _p(self.thr), _p(self.cnt), self.seed, t0, tmax, dt, atol, rtol, hmin, hmax,
                        scheme, max_steps, _p(self.stats))
        if st:
            raise RuntimeError(f"orc_mcwf status {st}")

    def expectation(self, levels, *ops):
        """Ensemble average of <psi|O|psi>/<psi|psi> (qvec_utilities.c:1353-1424)."""
        v = 0j
        for p in self.psi:
            v += expect_wf(levels, p, *ops) / np.vdot(p, p).real
        return v / self.ntraj

    def free(self):
        lib().orc_csr_free(self.heff)
        for h in self.jumps:
            lib().orc_csr_free(h)
        self.jumps = []


def num_threads():
    return lib().orc_num_threads()

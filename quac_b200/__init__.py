"""Python mirror of QuaC's C API over libquac_b200.so (ctypes).

The names follow the reference (QuaC, src/qsystem.h, src/qvec_utilities.h,
src/quantum_circuits.h, src/solver.h) so a QuaC program reads the same
here::

    import quac_b200 as q
    q.QuaC_initialize()
    qs = q.initialize_system()
    qb = q.create_op_sys(qs, 2)
    cav = q.create_op_sys(qs, 10)
    q.add_ham_term(qs, 0.1, cav.dag, qb)
    q.add_lin_term(qs, 1e-2, cav)
    q.construct_matrix(qs)
    rho = q.create_qvec_sys(qs)
    q.add_to_qvec(rho, 1.0, 10, 10)
    q.assemble_qvec(rho)
    q.time_step_sys(qs, rho, 0.0, 1.0, 0.01, 1000)
    n = q.get_expectation_value_qvec(rho, cav.n)

Every call goes through the C ABI declared in include/quac_b200.h; the
compute runs in the library's CUDA kernels.  There is no CPU fallback: on a
machine without a GPU the compute calls fail with the CUDA error.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# QUAC_B200_LIB selects another build of the library (e.g. to compare two builds)
LIB_PATH = os.environ.get("QUAC_B200_LIB") or os.path.join(_HERE, "libquac_b200.so")

# op_type, qvec_type, gate_type (include/quac_b200.h)
RAISE, NUMBER, LOWER, VEC, SIGMA_X, SIGMA_Y, SIGMA_Z, IDENTITY, OTHER = -1, 0, 1, 2, 3, 4, 5, 6, 7
DENSITY_MATRIX, WAVEFUNCTION = -1, 1
GATES = dict(SQiSWP=-8, CZ_ARP=-7, CUSTOM2QGATE=-6, CZX=-5, CmZ=-4, CZ=-3, CXZ=-2, CNOT=-1,
             HADAMARD=1, SIGMAX=2, SIGMAY=3, SIGMAZ=4, EYE=5, RX=6, RY=7, RZ=8, U1=9, U2=10,
             U3=11, CUSTOM1QGATE=12)
globals().update(GATES)
_NQ = {g: (2 if v < 0 else 1) for g, v in GATES.items()}

i64, dbl, vp = ctypes.c_int64, ctypes.c_double, ctypes.c_void_p


class Scalar(ctypes.Structure):
    """PetscScalar (complex double) passed by value."""
    _fields_ = [("re", dbl), ("im", dbl)]


def _sc(a):
    a = complex(a)
    return Scalar(a.real, a.imag)


class _OpStruct(ctypes.Structure):
    pass


_OpPtr = ctypes.POINTER(_OpStruct)
_OpStruct._fields_ = [
    ("initial_pop", dbl), ("initial_exc", i64), ("n_before", i64), ("my_levels", i64),
    ("my_op_type", ctypes.c_int), ("pos_in_sys_hspace", i64),
    ("dag", _OpPtr), ("n", _OpPtr), ("sig_x", _OpPtr), ("sig_y", _OpPtr), ("sig_z", _OpPtr),
    ("eye", _OpPtr), ("other", _OpPtr), ("position", i64), ("vec_op_list", vp),
    ("evals", dbl * 4), ("evecs", dbl * 8)]


class _QvecStruct(ctypes.Structure):
    _fields_ = [("my_type", ctypes.c_int), ("ens_spawned", ctypes.c_int), ("n", i64),
                ("Istart", i64), ("Iend", i64), ("total_levels", i64),
                ("hspace_dims", ctypes.POINTER(i64)), ("ndims_hspace", i64), ("n_ops", i64),
                ("n_ensemble", i64), ("ens_i", i64), ("data", vp), ("ens_datas", vp)]


_MonitorFn = ctypes.CFUNCTYPE(ctypes.c_int, vp, i64, dbl, vp, vp)


class _QsysStruct(ctypes.Structure):
    _fields_ = [("num_time_indep", i64), ("num_time_dep", i64), ("hspace_frozen", i64),
                ("dm_equations", ctypes.c_int), ("mcwf_solver", ctypes.c_int),
                ("time_step_called", ctypes.c_int), ("mat_allocated", i64),
                ("num_subsystems", i64), ("subsystem_list", ctypes.POINTER(_OpPtr)),
                ("total_levels", i64), ("dim", i64), ("solution_qvec", vp), ("np", i64),
                ("nid", i64), ("current_time", dbl), ("ts_monitor", vp), ("ts_ctx", vp),
                ("num_circuits", i64), ("circuit_list_size", i64), ("current_circuit", i64),
                ("circuit_list", vp), ("impl", vp)]


class _GateStruct(ctypes.Structure):
    _fields_ = [("time", dbl), ("run_time", dbl), ("my_gate_type", ctypes.c_int),
                ("qubit_numbers", ctypes.POINTER(i64)), ("num_qubits", i64), ("custom_func", vp),
                ("theta", dbl), ("phi", dbl), ("lambda_", dbl), ("gate_ctx", vp)]


class _CircuitStruct(ctypes.Structure):
    _fields_ = [("num_gates", i64), ("gate_list_size", i64), ("current_gate", i64),
                ("num_layers", i64), ("current_layer", i64), ("start_time", dbl),
                ("gate_list", ctypes.POINTER(_GateStruct)), ("layer_list", vp)]


class CustomGateData(ctypes.Structure):
    """custom_gate_data: a 4x4 complex matrix (row-major)."""
    _fields_ = [("gate_data", dbl * 32)]


_lib = None


def lib():
    """Loads libquac_b200.so (built in-tree by quac_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: run `python -m quac_b200.build` first")
    L = ctypes.CDLL(LIB_PATH)
    P = ctypes.POINTER
    sig = {
        "QuaC_initialize": (None, [ctypes.c_int, vp]),
        "QuaC_finalize": (None, []),
        "initialize_system": (None, [P(P(_QsysStruct))]),
        "destroy_system": (None, [P(P(_QsysStruct))]),
        "create_op_sys": (None, [P(_QsysStruct), i64, P(_OpPtr)]),
        "create_vec_op_sys": (None, [P(_QsysStruct), i64, P(P(_OpPtr))]),
        "add_ham_term_list": (None, [P(_QsysStruct), Scalar, i64, P(_OpPtr)]),
        "add_lin_term_list": (None, [P(_QsysStruct), Scalar, i64, P(_OpPtr)]),
        "clear_mat_terms_sys": (None, [P(_QsysStruct)]),
        "construct_matrix": (None, [P(_QsysStruct)]),
        "time_step_sys": (None, [P(_QsysStruct), P(_QvecStruct), dbl, dbl, dbl, i64]),
        "set_ts_monitor_sys": (None, [P(_QsysStruct), vp, vp]),
        "set_init_excited_op": (None, [_OpPtr, i64]),
        "set_qvec_from_init_excited_op": (None, [P(_QsysStruct), P(_QvecStruct)]),
        "create_qvec_sys": (None, [P(_QsysStruct), P(P(_QvecStruct))]),
        "create_dm_sys": (None, [P(_QsysStruct), P(P(_QvecStruct))]),
        "create_wf_sys": (None, [P(_QsysStruct), P(P(_QvecStruct))]),
        "create_arb_qvec": (None, [P(P(_QvecStruct)), i64, ctypes.c_int]),
        "destroy_qvec": (None, [P(P(_QvecStruct))]),
        "add_to_qvec_loc": (None, [P(_QvecStruct), Scalar, i64]),
        "add_to_qvec_fock_op_list": (None, [Scalar, P(_QvecStruct), i64, P(_OpPtr), vp]),
        "get_qvec_loc_fock_op_list": (None, [P(_QvecStruct), P(i64), i64, P(_OpPtr), vp]),
        "assemble_qvec": (None, [P(_QvecStruct)]),
        "get_dm_element_qvec": (None, [P(_QvecStruct), i64, i64, P(Scalar)]),
        "get_wf_element_qvec": (None, [P(_QvecStruct), i64, P(Scalar)]),
        "get_trace_qvec": (None, [P(_QvecStruct), P(Scalar)]),
        "get_expectation_value_qvec_list": (None, [P(_QvecStruct), P(Scalar), i64, P(_OpPtr)]),
        "get_fidelity_qvec": (None, [P(_QvecStruct), P(_QvecStruct), P(dbl), P(dbl)]),
        "copy_qvec": (None, [P(_QvecStruct), P(_QvecStruct)]),
        "create_circuit": (None, [P(_CircuitStruct), i64]),
        "destroy_circuit": (None, [P(_CircuitStruct)]),
        "schedule_circuit_layers": (None, [P(_QsysStruct), P(_CircuitStruct)]),
        "apply_circuit_to_sys": (None, [P(_QsysStruct), P(_CircuitStruct), dbl]),
        "apply_circuit_to_qvec": (None, [P(_QsysStruct), _CircuitStruct, P(_QvecStruct)]),
        "quac_add_gate": (ctypes.c_int, [P(_CircuitStruct), dbl, ctypes.c_int, ctypes.c_int,
                                         P(ctypes.c_int), dbl, dbl, dbl, vp, vp]),
        "quac_apply_gate": (ctypes.c_int, [P(_QvecStruct), ctypes.c_int, ctypes.c_int,
                                           P(ctypes.c_int), dbl, dbl, dbl, vp]),
        "steady_state_sys": (i64, [P(_QsysStruct), P(_QvecStruct)]),
        "quac_lrho_apply_device": (ctypes.c_int, [P(_QsysStruct), vp, vp]),
        "quac_lrho_apply_host": (ctypes.c_int, [P(_QsysStruct), vp, vp]),
        "quac_write_superoperator_binary": (ctypes.c_int, [P(_QsysStruct), ctypes.c_char_p]),
        "quac_time_step_host": (ctypes.c_int, [P(_QsysStruct), vp, dbl, dbl, dbl, i64]),
        "quac_set_error_mode": (None, [ctypes.c_int]),
        "quac_last_error": (ctypes.c_char_p, []),
        "quac_clear_error": (None, []),
        "quac_set_ts_options": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, dbl, dbl, i64]),
        "quac_qvec_device_ptr": (vp, [P(_QvecStruct)]),
        "quac_kernel_launch_count": (i64, []),
        "quac_set_stream": (None, [P(_QsysStruct), vp]),
        "quac_set_kernel_path": (None, [ctypes.c_int]),
        "quac_set_lrho_precision": (ctypes.c_int, [ctypes.c_int]),
        "quac_set_hermitian_mode": (ctypes.c_int, [ctypes.c_int]),
        "quac_set_gmres_preconditioner": (ctypes.c_int, [ctypes.c_int]),
        "quac_steady_precond_setup": (ctypes.c_int, [P(_QsysStruct)]),
        "quac_set_gmres_tolerance": (ctypes.c_int, [dbl]),
        "quac_steady_precond_stats": (None, [ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_double)]),
        "quac_set_gmres_restart": (ctypes.c_int, [ctypes.c_int]),
        "quac_set_gmres_precision": (ctypes.c_int, [ctypes.c_int]),
        "quac_set_deflation_refresh": (ctypes.c_int, [ctypes.c_int]),
        "quac_hermitian_apply_count": (i64, []),
        "VecGetSize": (ctypes.c_int, [vp, P(i64)]),
        "read_qvec_dm_binary": (None, [P(P(_QvecStruct)), ctypes.c_char_p]),
        "read_qvec_wf_binary": (None, [P(P(_QvecStruct)), ctypes.c_char_p]),
        "print_qvec_file": (None, [P(_QvecStruct), ctypes.c_char_p]),
        "quac_steady_state_guided": (i64, [P(_QsysStruct), P(_QvecStruct), vp, i64, i64, P(dbl)]),
        "quac_wsnet_create": (ctypes.c_int, [P(vp), ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_int, ctypes.c_uint64]),
        "quac_wsnet_destroy": (ctypes.c_int, [vp]),
        "quac_wsnet_add_sample": (ctypes.c_int, [vp, P(dbl), P(_QvecStruct)]),
        "quac_wsnet_num_samples": (ctypes.c_int, [vp]),
        "quac_wsnet_num_params": (i64, [vp]),
        "quac_wsnet_get_params": (ctypes.c_int, [vp, vp]),
        "quac_wsnet_set_params": (ctypes.c_int, [vp, vp]),
        "quac_wsnet_loss_grad": (ctypes.c_int, [vp, ctypes.c_int, P(dbl), vp]),
        "quac_wsnet_train": (ctypes.c_int, [vp, ctypes.c_int, dbl, ctypes.c_uint64, P(dbl)]),
        "quac_wsnet_predict": (ctypes.c_int, [vp, ctypes.c_int, vp, vp]),
        "quac_ensemble_create": (ctypes.c_int, [P(vp), i64, P(P(_QsysStruct))]),
        "quac_ensemble_destroy": (ctypes.c_int, [vp]),
        "quac_ensemble_set_options": (ctypes.c_int, [vp, ctypes.c_int, dbl, dbl, dbl, dbl, i64]),
        "quac_ensemble_set_shape": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
        "quac_ensemble_get_shape": (ctypes.c_int, [vp, P(ctypes.c_int), P(ctypes.c_int), P(ctypes.c_int)]),
        "quac_ensemble_tune": (ctypes.c_int, [vp, dbl, dbl, dbl, P(dbl)]),
        "quac_ensemble_state_offset": (i64, [vp, i64]),
        "quac_ensemble_state_device_ptr": (vp, [vp]),
        "quac_ensemble_set_states": (ctypes.c_int, [vp, vp]),
        "quac_ensemble_get_states": (ctypes.c_int, [vp, vp]),
        "quac_ensemble_run": (ctypes.c_int, [vp, dbl, dbl, dbl]),
        "quac_ensemble_get_stats": (ctypes.c_int, [vp, i64, P(dbl), P(i64), P(i64), P(ctypes.c_int)]),
        "quac_ensemble_populations": (ctypes.c_int, [vp, vp]),
        "quac_ensemble_set_redo_margin": (ctypes.c_int, [vp, dbl]),
        "quac_ensemble_redone_steps": (i64, [vp, i64]),
        "quac_ensemble_set_fp32_budget": (ctypes.c_int, [vp, dbl]),
        "quac_ensemble_f64_steps": (i64, [vp, i64]),
        "create_op": (None, [ctypes.c_int, P(_OpPtr)]),
        "create_vec": (None, [ctypes.c_int, P(P(_OpPtr))]),
        "add_to_ham": (None, [Scalar, _OpPtr]),
        "add_to_ham_mult2": (None, [Scalar, _OpPtr, _OpPtr]),
        "add_to_ham_mult3": (None, [Scalar, _OpPtr, _OpPtr, _OpPtr]),
        "add_lin": (None, [Scalar, _OpPtr]),
        "add_lin_mult2": (None, [Scalar, _OpPtr, _OpPtr]),
        "steady_state": (None, [vp]),
        "time_step": (None, [vp, dbl, dbl, dbl, i64]),
        "set_ts_monitor_ctx": (None, [vp, vp]),
        "QuaC_clear": (None, []),
        "create_full_dm": (None, [P(vp)]),
        "create_dm": (None, [P(vp), i64]),
        "destroy_dm": (None, [vp]),
        "add_value_to_dm": (None, [vp, i64, i64, Scalar]),
        "assemble_dm": (None, [vp]),
        "get_dm_element": (None, [vp, i64, i64, P(Scalar)]),
        "get_num_populations": (ctypes.c_int, []),
        "get_populations": (None, [vp, P(P(dbl))]),
        "VecGetArray": (ctypes.c_int, [vp, P(P(Scalar))]),
        "VecRestoreArray": (ctypes.c_int, [vp, P(P(Scalar))]),
        "get_bitstring_probs": (None, [P(_QvecStruct), P(i64), P(P(dbl)), P(P(dbl))]),
        "quac_add_term_time_dep_list": (ctypes.c_int, [P(_QsysStruct), ctypes.c_int, Scalar, vp, vp, i64,
                                                       P(_OpPtr)]),
        "use_mcwf_solver": (None, [P(_QsysStruct), i64, i64]),
        "quac_set_observable_monitor": (ctypes.c_int, [P(_QsysStruct), i64, P(i64), P(_OpPtr), vp, vp, i64]),
        "qiskit_qasm_read": (None, [ctypes.c_char_p, P(i64), P(_CircuitStruct)]),
        "qiskit_tqasm_read": (None, [ctypes.c_char_p, P(i64), P(_CircuitStruct)]),
        "cirq_qasm_read": (None, [ctypes.c_char_p, P(i64), P(_CircuitStruct)]),
        "projectq_qasm_read": (None, [ctypes.c_char_p, P(i64), P(_CircuitStruct)]),
        "quil_read": (None, [ctypes.c_char_p, P(i64), P(_CircuitStruct)]),
        "quac_mcwf_get_states": (ctypes.c_int, [P(_QvecStruct), vp, vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    L.quac_set_error_mode(1)  # errors come back as exceptions here
    _lib = L
    return L


class QuacError(RuntimeError):
    pass


def _check():
    msg = _lib.quac_last_error()
    if msg:
        _lib.quac_clear_error()
        raise QuacError(msg.decode(errors="replace").strip())


# ----------------------------------------------------------------- handles
class Operator:
    """A QuaC operator (op->dag, op->n, op->sig_x ... as attributes)."""

    def __init__(self, ptr):
        self._ptr = ptr

    def _child(self, name):
        p = getattr(self._ptr.contents, name)
        return Operator(p) if p else None

    @property
    def dag(self):
        return self._child("dag")

    @property
    def n(self):
        return self._child("n")

    @property
    def eye(self):
        return self._child("eye")

    @property
    def sig_x(self):
        return self._child("sig_x")

    @property
    def sig_y(self):
        return self._child("sig_y")

    @property
    def sig_z(self):
        return self._child("sig_z")

    @property
    def other(self):
        return self._child("other")

    @property
    def a(self):
        return self

    @property
    def my_levels(self):
        return self._ptr.contents.my_levels

    @property
    def n_before(self):
        return self._ptr.contents.n_before

    @property
    def my_op_type(self):
        return self._ptr.contents.my_op_type

    @property
    def position(self):
        return self._ptr.contents.position

    def triple(self, sub):
        """(type, subsystem, position) as the oracle describes operators."""
        return (self.my_op_type, sub, self.position)


class QSystem:
    def __init__(self, ptr):
        self._ptr = ptr
        self._monitor = None

    @property
    def dim(self):
        return self._ptr.contents.dim

    @property
    def total_levels(self):
        return self._ptr.contents.total_levels

    @property
    def dm_equations(self):
        return bool(self._ptr.contents.dm_equations)

    def destroy(self):
        if self._ptr:
            lib().destroy_system(ctypes.byref(self._ptr))
            self._ptr = None


class Qvec:
    def __init__(self, ptr):
        self._ptr = ptr

    @property
    def n(self):
        return self._ptr.contents.n

    @property
    def my_type(self):
        return self._ptr.contents.my_type

    @property
    def device_ptr(self):
        return lib().quac_qvec_device_ptr(self._ptr)

    def to_numpy(self):
        """Copies the vector to host (column-stacked for a density matrix)."""
        import ctypes as C
        n = self.n
        out = np.empty(n, dtype=np.complex128)
        cudart = _cudart()
        rc = cudart.cudaMemcpy(out.ctypes.data_as(C.c_void_p), C.c_void_p(self.device_ptr),
                               C.c_size_t(16 * n), 2)
        if rc != 0:
            raise QuacError(f"cudaMemcpy failed ({rc})")
        return out

    def from_numpy(self, arr):
        import ctypes as C
        arr = np.ascontiguousarray(arr, dtype=np.complex128)
        if arr.size != self.n:
            raise ValueError("size mismatch")
        cudart = _cudart()
        rc = cudart.cudaMemcpy(C.c_void_p(self.device_ptr), arr.ctypes.data_as(C.c_void_p),
                               C.c_size_t(16 * self.n), 1)
        if rc != 0:
            raise QuacError(f"cudaMemcpy failed ({rc})")

    def destroy(self):
        if self._ptr:
            lib().destroy_qvec(ctypes.byref(self._ptr))
            self._ptr = None


_cudart_lib = None


def _cudart():
    global _cudart_lib
    if _cudart_lib is None:
        import glob
        cands = glob.glob("/usr/local/cuda/lib64/libcudart.so*")
        _cudart_lib = ctypes.CDLL(cands[0] if cands else "libcudart.so")
        _cudart_lib.cudaMemcpy.restype = ctypes.c_int
        _cudart_lib.cudaMemcpy.argtypes = [vp, vp, ctypes.c_size_t, ctypes.c_int]
    return _cudart_lib


# ------------------------------------------------------------- QuaC calls
def QuaC_initialize(args=()):
    argv = [b"quac"] + [a.encode() if isinstance(a, str) else a for a in args]
    arr = (ctypes.c_char_p * (len(argv) + 1))(*argv, None)
    lib().QuaC_initialize(len(argv), ctypes.cast(arr, vp))
    _check()


def QuaC_finalize():
    lib().QuaC_finalize()


def initialize_system():
    p = ctypes.POINTER(_QsysStruct)()
    lib().initialize_system(ctypes.byref(p))
    _check()
    return QSystem(p)


def destroy_system(qs):
    qs.destroy()


def create_op_sys(qs, levels):
    p = _OpPtr()
    lib().create_op_sys(qs._ptr, int(levels), ctypes.byref(p))
    _check()
    return Operator(p)


def create_vec_op_sys(qs, levels):
    arr = ctypes.POINTER(_OpPtr)()
    lib().create_vec_op_sys(qs._ptr, int(levels), ctypes.byref(arr))
    _check()
    return [Operator(arr[i]) for i in range(levels)]


def _oplist(ops):
    arr = (_OpPtr * max(1, len(ops)))(*[o._ptr for o in ops])
    return arr


def add_ham_term(qs, a, *ops):
    lib().add_ham_term_list(qs._ptr, _sc(a), len(ops), _oplist(ops))
    _check()


def add_lin_term(qs, a, *ops):
    lib().add_lin_term_list(qs._ptr, _sc(a), len(ops), _oplist(ops))
    _check()


_TdFn = ctypes.CFUNCTYPE(None, ctypes.c_double, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                         ctypes.POINTER(ctypes.c_double))


def _add_td(qs, kind, a, fn, ops):
    def _cb(t, ctx, re, im):
        v = complex(fn(t))
        re[0] = v.real
        im[0] = v.imag

    cb = _TdFn(_cb)
    if not hasattr(qs, "_td_callbacks"):
        qs._td_callbacks = []
    qs._td_callbacks.append(cb)  # kept alive as long as the system
    arr = _oplist(ops)
    lib().quac_add_term_time_dep_list(qs._ptr, kind, _sc(a), None, ctypes.cast(cb, vp), len(ops), arr)
    _check()


def add_ham_term_time_dep(qs, a, fn, *ops):
    """Hamiltonian term a f(t) ops[0] ops[1] ... (qsystem.c:491-519); fn(t)
    returns a number."""
    _add_td(qs, 1, a, fn, ops)


def add_lin_term_time_dep(qs, a, fn, *ops):
    """Lindblad term with rate a f(t) (qsystem.c:521-552)."""
    _add_td(qs, 2, a, fn, ops)


def clear_mat_terms_sys(qs):
    lib().clear_mat_terms_sys(qs._ptr)


def construct_matrix(qs):
    lib().construct_matrix(qs._ptr)
    _check()


def set_init_excited_op(op, exc):
    lib().set_init_excited_op(op._ptr, int(exc))
    _check()


def set_qvec_from_init_excited_op(qs, q):
    lib().set_qvec_from_init_excited_op(qs._ptr, q._ptr)
    _check()


def set_ts_options(rk_type="", adapt_type="", rtol=-1.0, atol=-1.0, max_steps=-1):
    """Programmatic -ts_rk_type / -ts_adapt_type / -ts_rtol / -ts_atol / -ts_max_steps."""
    lib().quac_set_ts_options(rk_type.encode(), adapt_type.encode(), rtol, atol, max_steps)
    _check()


def set_ts_monitor_sys(qs, fn):
    """fn(step, time, vec_handle) called after each step (None clears)."""
    if fn is None:
        qs._monitor = None
        lib().set_ts_monitor_sys(qs._ptr, None, None)
        return

    def _cb(ts, step, t, vec, ctx):
        fn(step, t, vec)
        return 0

    qs._monitor = _MonitorFn(_cb)
    lib().set_ts_monitor_sys(qs._ptr, ctypes.cast(qs._monitor, vp), None)


def time_step_sys(qs, q, t0, tmax, dt, steps_max):
    lib().time_step_sys(qs._ptr, q._ptr, float(t0), float(tmax), float(dt), int(steps_max))
    _check()


def create_qvec_sys(qs):
    p = ctypes.POINTER(_QvecStruct)()
    lib().create_qvec_sys(qs._ptr, ctypes.byref(p))
    _check()
    return Qvec(p)


def create_dm_sys(qs):
    p = ctypes.POINTER(_QvecStruct)()
    lib().create_dm_sys(qs._ptr, ctypes.byref(p))
    _check()
    return Qvec(p)


def create_wf_sys(qs):
    p = ctypes.POINTER(_QvecStruct)()
    lib().create_wf_sys(qs._ptr, ctypes.byref(p))
    _check()
    return Qvec(p)


def create_arb_qvec(nstates, qtype):
    p = ctypes.POINTER(_QvecStruct)()
    lib().create_arb_qvec(ctypes.byref(p), int(nstates), int(qtype))
    _check()
    return Qvec(p)


def destroy_qvec(q):
    q.destroy()


def add_to_qvec_loc(q, alpha, loc):
    lib().add_to_qvec_loc(q._ptr, _sc(alpha), int(loc))
    _check()


def add_to_qvec(q, alpha, *locs):
    """add_to_qvec(dm, a, col, row) adds at D*col + row; add_to_qvec(wf, a, i)."""
    if q.my_type == DENSITY_MATRIX:
        D = int(round(np.sqrt(q.n)))
        add_to_qvec_loc(q, alpha, D * int(locs[0]) + int(locs[1]))
    else:
        add_to_qvec_loc(q, alpha, int(locs[0]))


def _fock_pairs(pairs):
    if len(pairs) % 2:
        raise QuacError("expected (op, fock state) pairs")
    ops = pairs[0::2]
    fock = np.ascontiguousarray([int(f) for f in pairs[1::2]], dtype=np.int64)
    return len(ops), _oplist(ops), fock


def get_qvec_loc_fock_op(q, *pairs):
    """Index of the basis state with each given op in the given Fock state
    (qvec_utilities.c:996-1033), the diagonal element for a density matrix:
    get_qvec_loc_fock_op(q, op1, 1, op2, 0)."""
    n, ops, fock = _fock_pairs(pairs)
    loc = i64()
    lib().get_qvec_loc_fock_op_list(q._ptr, ctypes.byref(loc), n, ops, fock.ctypes.data)
    _check()
    return loc.value


def add_to_qvec_fock_op(alpha, q, *pairs):
    """add_to_qvec_fock_op(alpha, q, op1, f1, op2, f2, ...)
    (qvec_utilities.c:832-857)."""
    n, ops, fock = _fock_pairs(pairs)
    lib().add_to_qvec_fock_op_list(_sc(alpha), q._ptr, n, ops, fock.ctypes.data)
    _check()


def assemble_qvec(q):
    lib().assemble_qvec(q._ptr)
    _check()


def get_dm_element_qvec(q, row, col):
    s = Scalar()
    lib().get_dm_element_qvec(q._ptr, int(row), int(col), ctypes.byref(s))
    _check()
    return complex(s.re, s.im)


def get_trace_qvec(q):
    s = Scalar()
    lib().get_trace_qvec(q._ptr, ctypes.byref(s))
    _check()
    return complex(s.re, s.im)


def get_expectation_value_qvec(q, *ops):
    s = Scalar()
    lib().get_expectation_value_qvec_list(q._ptr, ctypes.byref(s), len(ops), _oplist(ops))
    _check()
    return complex(s.re, s.im)


def get_fidelity_qvec(q1, q2):
    f, v = dbl(), dbl()
    lib().get_fidelity_qvec(q1._ptr, q2._ptr, ctypes.byref(f), ctypes.byref(v))
    _check()
    return f.value, v.value


def copy_qvec(src, dst):
    lib().copy_qvec(src._ptr, dst._ptr)
    _check()


class Circuit:
    """The value struct `circuit` (create_circuit / add_gate_to_circuit_sys)."""

    def __init__(self, num_gates):
        self.c = _CircuitStruct()
        self._ctx = []
        lib().create_circuit(ctypes.byref(self.c), int(num_gates))

    def add_gate(self, time, gate, *qubits, theta=0.0, phi=0.0, lam=0.0, ctx=None, func=None):
        g = GATES[gate] if isinstance(gate, str) else int(gate)
        qs = (ctypes.c_int * len(qubits))(*qubits)
        if ctx is not None:
            self._ctx.append(ctx)
        rc = lib().quac_add_gate(ctypes.byref(self.c), float(time), g, len(qubits), qs, theta, phi,
                                 lam, ctypes.cast(ctypes.pointer(ctx), vp) if ctx is not None else None,
                                 ctypes.cast(func, vp) if func is not None else None)
        _check()
        return rc

    def destroy(self):
        lib().destroy_circuit(ctypes.byref(self.c))


def create_circuit(num_gates):
    return Circuit(num_gates)


def _read_circuit(fn_name, path):
    c = Circuit.__new__(Circuit)
    c.c = _CircuitStruct()
    c._ctx = []
    nq = ctypes.c_int64()
    getattr(lib(), fn_name)(os.fsencode(path), ctypes.byref(nq), ctypes.byref(c.c))
    _check()
    return nq.value, c


def qiskit_qasm_read(path):
    """(num_qubits, Circuit) from an OpenQASM 2 file in qiskit's qubit order."""
    return _read_circuit("qiskit_qasm_read", path)


def qiskit_tqasm_read(path):
    return _read_circuit("qiskit_tqasm_read", path)


def cirq_qasm_read(path):
    return _read_circuit("cirq_qasm_read", path)


def projectq_qasm_read(path):
    return _read_circuit("projectq_qasm_read", path)


def quil_read(path):
    return _read_circuit("quil_read", path)


def circuit_gates(c):
    """The gate list of a Circuit as (time, gate type, qubits, theta, phi, lambda) tuples."""
    out = []
    for k in range(c.c.num_gates):
        g = c.c.gate_list[k]
        out.append((g.time, g.my_gate_type, tuple(g.qubit_numbers[i] for i in range(g.num_qubits)),
                    g.theta, g.phi, g.lambda_))
    return out


def add_gate_to_circuit_sys(circ, time, gate, *args, **kw):
    """add_gate_to_circuit_sys(circ, t, 'RZ', q, theta) / (circ, t, 'U3', q, th, ph, la)."""
    g = GATES[gate] if isinstance(gate, str) else int(gate)
    name = gate if isinstance(gate, str) else [k for k, v in GATES.items() if v == g][0]
    nq = _NQ[name]
    qubits, params = args[:nq], args[nq:]
    p = dict(theta=0.0, phi=0.0, lam=0.0)
    if len(params) > 3:
        raise TypeError(f"{name}: at most three angles (theta, phi, lam), got {len(params)}")
    p.update(zip(("theta", "phi", "lam"), params))
    p.update(kw)
    return circ.add_gate(time, g, *qubits, **p)


def schedule_circuit_layers(qs, circ):
    lib().schedule_circuit_layers(qs._ptr, ctypes.byref(circ.c))
    _check()


def apply_circuit_to_sys(qs, circ, time):
    lib().apply_circuit_to_sys(qs._ptr, ctypes.byref(circ.c), float(time))
    _check()


def apply_circuit_to_qvec(qs, circ, q):
    lib().apply_circuit_to_qvec(qs._ptr, circ.c, q._ptr)
    _check()


def apply_gate2(q, gate, *args, ctx=None):
    """apply_gate2(q, 'CNOT', 0, 1) / (q, 'RZ', q0, theta) / (q, 'U3', q0, th, ph, la)."""
    name = gate if isinstance(gate, str) else [k for k, v in GATES.items() if v == gate][0]
    nq = _NQ[name]
    qubits, params = args[:nq], list(args[nq:])
    th = ph = la = 0.0
    if name in ("RX", "RY", "RZ"):
        th = params[0]
    elif name in ("U1", "U2", "U3"):
        th, ph, la = params
    qa = (ctypes.c_int * nq)(*qubits)
    lib().quac_apply_gate(q._ptr, GATES[name], nq, qa, th, ph, la,
                          ctypes.cast(ctypes.pointer(ctx), vp) if ctx is not None else None)
    _check()


def steady_state_sys(qs, q):
    its = lib().steady_state_sys(qs._ptr, q._ptr)
    _check()
    return its


def steady_state_guided(qs, q, U=None, maxit_guided=20000):
    """Steady state from the initial guess already in q, deflated by the
    dominant subspace U (D x kd, orthonormal columns).  Returns (iterations,
    final residual ||b - A x||)."""
    res = dbl()
    if U is None:
        its = lib().quac_steady_state_guided(qs._ptr, q._ptr, None, 0, maxit_guided, ctypes.byref(res))
    else:
        U = np.asfortranarray(U, dtype=np.complex128)
        its = lib().quac_steady_state_guided(qs._ptr, q._ptr, U.ctypes.data, U.shape[1], maxit_guided,
                                             ctypes.byref(res))
    _check()
    return its, res.value


def lrho_apply_device(qs, x_ptr, y_ptr):
    """y = L x on device buffers (qs.dim complex128 each)."""
    lib().quac_lrho_apply_device(qs._ptr, vp(x_ptr), vp(y_ptr))
    _check()


def write_superoperator_binary(qs, filename):
    """Writes the system's operator (Liouvillian, or -i H for a wavefunction
    system) as a PETSc binary AIJ matrix (64-bit indices, big endian)."""
    lib().quac_write_superoperator_binary(qs._ptr, os.fsencode(filename))
    _check()


def read_petsc_binary_matrix(filename):
    """(shape, rowptr, cols, values) of a PETSc binary AIJ matrix written
    with 64-bit indices and complex128 values."""
    raw = open(filename, "rb").read()
    head = np.frombuffer(raw[:32], dtype=">i8")
    if head[0] != 1211216:
        raise ValueError(f"{filename}: not a PETSc binary matrix (class id {head[0]})")
    m, n, nz = (int(v) for v in head[1:])
    off = 32
    lens = np.frombuffer(raw[off:off + 8 * m], dtype=">i8").astype(np.int64)
    off += 8 * m
    cols = np.frombuffer(raw[off:off + 8 * nz], dtype=">i8").astype(np.int64)
    off += 8 * nz
    vals = np.frombuffer(raw[off:off + 16 * nz], dtype=">c16").astype(np.complex128)
    return (m, n), np.concatenate([[0], np.cumsum(lens)]), cols, vals


def lrho_apply_host(qs, x):
    """y = L x with host numpy arrays (copies in and out)."""
    x = np.ascontiguousarray(x, dtype=np.complex128)
    y = np.empty_like(x)
    lib().quac_lrho_apply_host(qs._ptr, x.ctypes.data_as(vp), y.ctypes.data_as(vp))
    _check()
    return y


def time_step_host(qs, x, t0, tmax, dt, steps_max):
    """Integrates host data in place (H2D, integration, D2H in one call)."""
    assert x.dtype == np.complex128 and x.flags.c_contiguous
    lib().quac_time_step_host(qs._ptr, x.ctypes.data_as(vp), t0, tmax, dt, steps_max)
    _check()
    return x


def kernel_launch_count():
    return lib().quac_kernel_launch_count()


def set_stream(qs, stream_ptr):
    """Launch qs's kernels on a caller-owned CUDA stream (e.g. a torch stream's cuda_stream)."""
    lib().quac_set_stream(qs._ptr, vp(stream_ptr) if stream_ptr else None)


def set_kernel_path(path):
    """0: default selection; 1: generic table kernel; 2: single-pass bit-mask kernel."""
    lib().quac_set_kernel_path(int(path))


def set_gmres_restart(m):
    """Restart length of the steady-state GMRES (default 100)."""
    lib().quac_set_gmres_restart(int(m))
    _check()


def set_gmres_precision(precision):
    """0 (default): complex128 GMRES basis; 1: complex64 basis (FP32 inner),
    complex128 residual and iterate at every restart (FP64 refined)."""
    lib().quac_set_gmres_precision(int(precision))
    _check()


def set_deflation_refresh(mode):
    """1 (default): steady_state_guided rebuilds its deflation space from the
    iterate at every restart; 0: keeps the proposed one."""
    lib().quac_set_deflation_refresh(int(mode))
    _check()


def set_gmres_preconditioner(mode):
    """2 (default): steady-state GMRES preconditioned by the inverse of the
    no-jump Liouvillian built from the Hermitian part of H_eff (approximate,
    cheap setup); 1: its exact inverse (non-Hermitian eigen-decomposition);
    0: none."""
    lib().quac_set_gmres_preconditioner(int(mode))
    _check()


def set_gmres_tolerance(rtol):
    """Steady-state GMRES tolerance on ||b - A x|| (default 1e-11)."""
    lib().quac_set_gmres_tolerance(float(rtol))
    _check()


def steady_precond_setup(qs):
    """Builds qs's steady-state preconditioner now (eigen-decomposition of
    H_eff on the GPU)."""
    lib().quac_steady_precond_setup(qs._ptr)
    _check()


def steady_precond_stats():
    """(decompositions computed in this process, their total seconds)."""
    n, sec = ctypes.c_int64(), ctypes.c_double()
    lib().quac_steady_precond_stats(ctypes.byref(n), ctypes.byref(sec))
    return n.value, sec.value


def set_hermitian_mode(mode):
    """1 (default): Hermitian mode in time_step_sys when it applies; 2: also
    in the single L.x entry points for a Hermitian input; 0: never."""
    lib().quac_set_hermitian_mode(int(mode))
    _check()


def hermitian_apply_count():
    return lib().quac_hermitian_apply_count()


def set_lrho_precision(precision):
    """0: complex128 L.x; 1: complex64 contraction in the multi-pass kernel."""
    lib().quac_set_lrho_precision(int(precision))
    _check()


# ---------------------------------------------------------------- ensembles
class Ensemble:
    """Many independent systems integrated together (quac_ensemble_*).

    ``systems`` are QSystem objects with their terms added; the ensemble
    copies their compiled terms, so they may be destroyed afterwards.
    States are one packed complex128 array (instance i at ``offsets[i]``,
    D_i^2 column-stacked values)."""

    def __init__(self, systems):
        systems = list(systems)
        n = len(systems)
        arr = (ctypes.POINTER(_QsysStruct) * n)(*[s._ptr for s in systems])
        h = vp()
        rc = lib().quac_ensemble_create(ctypes.byref(h), n, arr)
        _check()
        if rc:
            raise QuacError("quac_ensemble_create failed")
        self._h = h
        self.n = n
        self.offsets = np.array([lib().quac_ensemble_state_offset(h, i) for i in range(n + 1)], dtype=np.int64)
        self.dims = np.rint(np.sqrt(np.diff(self.offsets))).astype(np.int64)

    def _call(self, name, *args):
        rc = getattr(lib(), name)(self._h, *args)
        _check()
        if rc:
            raise QuacError(f"{name} failed")

    def set_options(self, precision=0, atol=5e-7, rtol=5e-7, hmin=0.01, hmax=1.0, max_steps=10 ** 6):
        self._call("quac_ensemble_set_options", precision, atol, rtol, hmin, hmax, max_steps)

    def set_redo_margin(self, margin):
        """complex64 mode: re-evaluate steps with |err - 1| < margin in complex128."""
        self._call("quac_ensemble_set_redo_margin", margin)

    def redone_steps(self):
        return np.array([lib().quac_ensemble_redone_steps(self._h, i) for i in range(self.n)])

    def set_fp32_budget(self, budget):
        """complex64 mode: estimated accumulated complex64 error after which an
        instance continues with complex128 stages (default 1e-7)."""
        self._call("quac_ensemble_set_fp32_budget", float(budget))

    def f64_steps(self):
        """Per instance, the steps taken in complex128 after its budget ran out."""
        return np.array([lib().quac_ensemble_f64_steps(self._h, i) for i in range(self.n)])

    def set_shape(self, warps, ctas_per_sm, elems_per_thread):
        self._call("quac_ensemble_set_shape", warps, ctas_per_sm, elems_per_thread)

    def shape(self):
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._call("quac_ensemble_get_shape", ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
        return a.value, b.value, c.value

    def tune(self, t0, t_probe, dt0):
        ms = dbl()
        self._call("quac_ensemble_tune", t0, t_probe, dt0, ctypes.byref(ms))
        return ms.value

    def set_states(self, rho):
        rho = np.ascontiguousarray(rho, dtype=np.complex128)
        if rho.size != self.offsets[-1]:
            raise ValueError("packed state size mismatch")
        self._call("quac_ensemble_set_states", rho.ctypes.data)

    def get_states(self, out=None):
        if out is None:
            out = np.empty(self.offsets[-1], dtype=np.complex128)
        self._call("quac_ensemble_get_states", out.ctypes.data)
        return out

    def state(self, rho_packed, i):
        """Instance i's D x D density matrix out of a packed state array."""
        D = int(self.dims[i])
        return rho_packed[self.offsets[i]:self.offsets[i + 1]].reshape(D, D, order="F")

    def device_ptr(self):
        return lib().quac_ensemble_state_device_ptr(self._h)

    def run(self, t0, tmax, dt0):
        self._call("quac_ensemble_run", t0, tmax, dt0)

    def stats(self):
        t, st, rj, fl = dbl(), i64(), i64(), ctypes.c_int()
        out = np.zeros((self.n, 4))
        for i in range(self.n):
            self._call("quac_ensemble_get_stats", i, ctypes.byref(t), ctypes.byref(st), ctypes.byref(rj),
                       ctypes.byref(fl))
            out[i] = (t.value, st.value, rj.value, fl.value)
        return out

    def populations(self, out=None):
        if out is None:
            out = np.empty(int(self.dims.sum()), dtype=np.float64)
        self._call("quac_ensemble_populations", out.ctypes.data)
        return out

    def destroy(self):
        if self._h:
            lib().quac_ensemble_destroy(self._h)
            self._h = None


# ------------------------------------------------------- learned warm start
class WarmStartNet:
    """The steady-state warm-start network (quac_wsnet_*).

    Inputs are 4 normalised parameters; the output for each input is a
    D x rank complex factor matrix F with F F^H ~ rho_ss."""

    def __init__(self, D, rank=16, hidden=256, batch=128, max_samples=2048, seed=0):
        h = vp()
        rc = lib().quac_wsnet_create(ctypes.byref(h), D, rank, hidden, batch, max_samples, seed)
        _check()
        if rc:
            raise QuacError("quac_wsnet_create failed")
        self._h, self.D, self.rank = h, D, rank

    def _call(self, name, *args):
        rc = getattr(lib(), name)(self._h, *args)
        _check()
        if rc:
            raise QuacError(f"{name} failed")

    def add_sample(self, theta, rho_qvec):
        t = (dbl * 4)(*[float(v) for v in theta])
        self._call("quac_wsnet_add_sample", t, rho_qvec._ptr)

    @property
    def num_samples(self):
        return lib().quac_wsnet_num_samples(self._h)

    @property
    def num_params(self):
        return lib().quac_wsnet_num_params(self._h)

    def get_params(self):
        out = np.empty(self.num_params, dtype=np.float32)
        self._call("quac_wsnet_get_params", out.ctypes.data)
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.num_params
        self._call("quac_wsnet_set_params", p.ctypes.data)

    def loss_grad(self, nb):
        loss = dbl()
        g = np.empty(self.num_params, dtype=np.float32)
        self._call("quac_wsnet_loss_grad", nb, ctypes.byref(loss), g.ctypes.data)
        return loss.value, g

    def train(self, epochs, lr=1e-3, seed=0):
        loss = dbl()
        self._call("quac_wsnet_train", epochs, lr, seed, ctypes.byref(loss))
        return loss.value

    def predict(self, thetas):
        thetas = np.ascontiguousarray(np.atleast_2d(thetas), dtype=np.float64)
        F = np.empty((thetas.shape[0], self.rank, self.D), dtype=np.complex128)
        self._call("quac_wsnet_predict", thetas.shape[0], thetas.ctypes.data, F.ctypes.data)
        return np.transpose(F, (0, 2, 1))  # (n, D, rank)

    def destroy(self):
        if self._h:
            lib().quac_wsnet_destroy(self._h)
            self._h = None


# ------------------------------------------------ legacy global-system API
# (operators.c, dm_utilities.c, solver.c): one implicit system built with
# create_op / add_to_ham / add_lin, density matrices as bare Vec handles

class LegacyVec:
    """A Vec of the legacy API (device vector handle)."""

    def __init__(self, ptr):
        self._ptr = ptr

    def size(self):
        n = ctypes.c_int64()
        lib().VecGetSize(self._ptr, ctypes.byref(n))
        return n.value

    def to_numpy(self):
        a = ctypes.POINTER(Scalar)()
        lib().VecGetArray(self._ptr, ctypes.byref(a))
        n = self.size()
        out = np.ctypeslib.as_array(ctypes.cast(a, ctypes.POINTER(ctypes.c_double)), shape=(2 * n,)).copy()
        lib().VecRestoreArray(self._ptr, ctypes.byref(a))
        return out[0::2] + 1j * out[1::2]

    def destroy(self):
        if self._ptr:
            lib().destroy_dm(self._ptr)
            self._ptr = None


def create_op(levels):
    p = _OpPtr()
    lib().create_op(int(levels), ctypes.byref(p))
    _check()
    return Operator(p)


def add_to_ham(a, op):
    lib().add_to_ham(_sc(a), op._ptr)
    _check()


def add_to_ham_mult2(a, op1, op2):
    lib().add_to_ham_mult2(_sc(a), op1._ptr, op2._ptr)
    _check()


def add_lin(a, op):
    lib().add_lin(_sc(a), op._ptr)
    _check()


def add_lin_mult2(a, op1, op2):
    lib().add_lin_mult2(_sc(a), op1._ptr, op2._ptr)
    _check()


def create_full_dm():
    p = ctypes.c_void_p()
    lib().create_full_dm(ctypes.byref(p))
    _check()
    return LegacyVec(p)


def add_value_to_dm(dm, row, col, val):
    lib().add_value_to_dm(dm._ptr, int(row), int(col), _sc(val))
    _check()


def assemble_dm(dm):
    lib().assemble_dm(dm._ptr)
    _check()


def get_dm_element(dm, row, col):
    s = Scalar()
    lib().get_dm_element(dm._ptr, int(row), int(col), ctypes.byref(s))
    _check()
    return complex(s.re, s.im)


def steady_state(dm):
    """solver.c:33-221 on the legacy system, result in dm."""
    lib().steady_state(dm._ptr)
    _check()


_legacy_monitor = None


def set_ts_monitor(fn):
    """fn(step, time, vec_handle) after each step of the legacy time_step
    (solver.c:526-545); None clears."""
    global _legacy_monitor
    if fn is None:
        _legacy_monitor = None
        lib().set_ts_monitor_ctx(None, None)
        return

    def _cb(ts, step, t, vec, ctx):
        fn(step, t, vec)
        return 0

    _legacy_monitor = _MonitorFn(_cb)
    lib().set_ts_monitor_ctx(ctypes.cast(_legacy_monitor, vp), None)


def time_step(dm, t0, tmax, dt, steps_max):
    """solver.c:236-510: the legacy system integrated on dm (a LegacyVec)."""
    lib().time_step(dm._ptr, float(t0), float(tmax), float(dt), int(steps_max))
    _check()


def QuaC_clear():
    """quac.c:60-80: forget the legacy global system so a new one can be built."""
    lib().QuaC_clear()
    _check()


def get_populations(dm):
    n = lib().get_num_populations()
    out = (ctypes.c_double * n)()
    p = ctypes.cast(out, ctypes.POINTER(ctypes.c_double))
    lib().get_populations(dm._ptr, ctypes.byref(p))
    _check()
    return np.array(out[:])


def get_bitstring_probs(q):
    """Probabilities of the computational basis states (the diagonal of
    rho, or |psi_i|^2), as get_bitstring_probs returns them."""
    n = ctypes.c_int64()
    pr, va = ctypes.POINTER(ctypes.c_double)(), ctypes.POINTER(ctypes.c_double)()
    lib().get_bitstring_probs(q._ptr, ctypes.byref(n), ctypes.byref(pr), ctypes.byref(va))
    _check()
    out = np.ctypeslib.as_array(pr, shape=(n.value,)).copy()
    libc = ctypes.CDLL(None)
    libc.free.argtypes = [ctypes.c_void_p]
    libc.free(ctypes.cast(pr, ctypes.c_void_p))
    libc.free(ctypes.cast(va, ctypes.c_void_p))
    return out


def read_qvec_dm_binary(path):
    p = ctypes.POINTER(_QvecStruct)()
    lib().read_qvec_dm_binary(ctypes.byref(p), os.fsencode(path))
    _check()
    return Qvec(p)


def read_qvec_wf_binary(path):
    p = ctypes.POINTER(_QvecStruct)()
    lib().read_qvec_wf_binary(ctypes.byref(p), os.fsencode(path))
    _check()
    return Qvec(p)


def print_qvec_file(q, path):
    lib().print_qvec_file(q._ptr, os.fsencode(path))
    _check()


def use_mcwf_solver(qs, num_tot_trajs, seed=0):
    """Quantum-jump trajectories instead of the density-matrix equations
    (qsystem.c:358-403); call after the Lindblad terms, before
    construct_matrix and create_qvec_sys.  seed 0 draws one."""
    lib().use_mcwf_solver(qs._ptr, int(num_tot_trajs), int(seed))
    _check()


def mcwf_states(q):
    """(states, stats) of an MCWF ensemble qvec after time_step_sys: states
    (ntraj, D) unnormalised wavefunctions, stats (ntraj, 2) accepted steps
    and jumps of every trajectory."""
    n, D = q._ptr.contents.n_ensemble, q.n
    st = np.zeros((n, D), dtype=np.complex128)
    ss = np.zeros((n, 2), dtype=np.int64)
    lib().quac_mcwf_get_states(q._ptr, st.ctypes.data_as(vp), ss.ctypes.data_as(vp))
    _check()
    return st, ss


_ObsFn = ctypes.CFUNCTYPE(None, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_double),
                          ctypes.POINTER(ctypes.c_double), ctypes.c_void_p)


def set_observable_monitor(qs, observables, fn, batch=1000):
    """Records Tr(O rho) (or <psi|O|psi>) of every observable after every
    step of time_step_sys on the GPU; fn(steps, times, values) receives
    numpy arrays in batches (values: (n, len(observables)) complex).  Each
    observable is a tuple of operators (a product).  fn None removes it."""
    if fn is None:
        qs._obs_monitor = None
        lib().quac_set_observable_monitor(qs._ptr, 0, None, None, None, None, 1)
        _check()
        return
    nobs = len(observables)

    def _cb(n, steps, times, vals, ctx):
        st = np.ctypeslib.as_array(steps, shape=(n,)).copy()
        tm = np.ctypeslib.as_array(times, shape=(n,)).copy()
        vv = np.ctypeslib.as_array(vals, shape=(n * nobs * 2,)).copy()
        fn(st, tm, (vv[0::2] + 1j * vv[1::2]).reshape(n, nobs))

    qs._obs_monitor = _ObsFn(_cb)
    flat = [o for obs in observables for o in obs]
    nops = (ctypes.c_int64 * nobs)(*[len(obs) for obs in observables])
    arr = _oplist(flat)
    lib().quac_set_observable_monitor(qs._ptr, nobs, nops, arr, ctypes.cast(qs._obs_monitor, vp), None, int(batch))
    _check()

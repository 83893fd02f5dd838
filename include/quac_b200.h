/*
 * quac_b200.h -- C ABI of the B200 Lindblad engine.
 *
 * The entry points keep the names, argument order and meaning of QuaC's C
 * API so that a QuaC program recompiles against this header (through the
 * drop-in headers in include/quac/) and links libquac_b200.so instead of
 * QuaC + PETSc.  Each declaration cites the reference interface it
 * replaces (path within the QuaC project : line).
 *
 * Storage: every qvec lives in GPU memory (complex128).  A density matrix
 * is column stacked, vec(rho)[D*col + row] = rho[row][col]
 * (qvec_utilities.c:322-337); subsystem 0 is the most significant Hilbert
 * digit (kron.c:308).
 *
 * Errors: the reference prints and calls exit() on misuse; these entry
 * points print the same kind of message and exit as well, unless
 * quac_set_error_mode(QUAC_ERRORS_RETURN) was called, in which case they
 * record the message (quac_last_error()) and return.  The *_ex variants
 * always return a status (0 = success).
 *
 * PETSc types are replaced by plain C types: PetscScalar = complex double,
 * PetscInt = int64_t, PetscReal = double, PetscErrorCode = int, and Vec/TS
 * are opaque handles owned by this library.
 */
#ifndef QUAC_B200_H_
#define QUAC_B200_H_

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
#include <complex>
typedef std::complex<double> PetscScalar;
#define PETSC_i (PetscScalar(0.0, 1.0))
#define PetscRealPart(x) (std::real(x))
#define PetscImaginaryPart(x) (std::imag(x))
extern "C" {
#else
#include <complex.h>
typedef double _Complex PetscScalar;
#define PETSC_i (_Complex_I)
#define PetscRealPart(x) (creal(x))
#define PetscImaginaryPart(x) (cimag(x))
#endif

typedef int64_t PetscInt;
typedef double PetscReal;
typedef int PetscErrorCode;
typedef int PetscBool;
#define PETSC_TRUE 1
#define PETSC_FALSE 0
#define PETSC_COMM_WORLD 0
#define PetscFunctionReturn(x) return (x)

typedef struct _p_Vec *Vec;          /* device vector handle */
typedef struct _p_TS *TS;            /* time-stepper handle passed to monitors */
typedef struct _p_Mat *Mat;          /* assembled-operator handle (export only) */

/* operator types: operators_p.h:6-16 */
typedef enum {
  RAISE = -1, NUMBER = 0, LOWER = 1, VEC = 2, SIGMA_X = 3, SIGMA_Y = 4, SIGMA_Z = 5,
  IDENTITY = 6, OTHER = 7
} op_type;

/* qvec types: qsystem_p.h:22-26 */
typedef enum { DENSITY_MATRIX = -1, WAVEFUNCTION = 1, WF_ENSEMBLE = 2 } qvec_type;

/* gate types: quantum_gates.h:11-33 */
typedef enum {
  NULL_GATE = -1000, SQiSWP = -8, CZ_ARP = -7, CUSTOM2QGATE = -6, CZX = -5, CmZ = -4, CZ = -3,
  CXZ = -2, CNOT = -1, HADAMARD = 1, SIGMAX = 2, SIGMAY = 3, SIGMAZ = 4, EYE = 5, RX = 6,
  RY = 7, RZ = 8, U1 = 9, U2 = 10, U3 = 11, CUSTOM1QGATE = 12
} gate_type;

/* operator: operators.h:8-33.  Fields a QuaC program reads (dag, n, eye,
 * sig_x/y/z, other, my_levels, n_before, my_op_type, position) keep their
 * names and meaning. */
struct operator_s;
typedef struct operator_s {
  double initial_pop;
  PetscInt initial_exc;
  PetscInt n_before;
  PetscInt my_levels;
  op_type my_op_type;
  PetscInt pos_in_sys_hspace;
  struct operator_s *dag, *n, *sig_x, *sig_y, *sig_z, *eye, *other;
  PetscInt position;
  struct operator_s **vec_op_list;
  PetscScalar evals[2];
  PetscScalar evecs[2][2];
} *op_handle;
#ifndef __cplusplus
typedef op_handle operator;
#endif
typedef op_handle *vec_op;

struct quantum_gate_struct;
typedef void (*custom_gate_func_type)(PetscScalar *, PetscInt, PetscInt, void *);

/* quantum_gates.h:38-48 */
struct quantum_gate_struct {
  PetscReal time, run_time;
  gate_type my_gate_type;
  PetscInt *qubit_numbers, num_qubits;
  custom_gate_func_type custom_func;
  PetscReal theta, phi, lambda;
  void *gate_ctx;
};

/* quantum_gates.h:51-55 */
struct gate_layer_struct {
  PetscReal time;
  PetscInt num_gates;
  struct quantum_gate_struct *gate_list;
};

/* qsystem_p.h:46-48: user data for CUSTOM1QGATE / CUSTOM2QGATE */
typedef struct { PetscScalar gate_data[4][4]; } custom_gate_data;

/* circuit: qsystem_p.h:50-55 (a value struct) */
typedef struct circuit {
  PetscInt num_gates, gate_list_size, current_gate, num_layers, current_layer;
  PetscReal start_time;
  struct quantum_gate_struct *gate_list;
  struct gate_layer_struct *layer_list;
} circuit;

/* qvec: qsystem_p.h:60-66 */
typedef struct qvec_s {
  qvec_type my_type;
  PetscBool ens_spawned;
  PetscInt n, Istart, Iend, total_levels, *hspace_dims, ndims_hspace, n_ops, n_ensemble, ens_i;
  Vec data;
  Vec *ens_datas;
} *qvec;

typedef PetscErrorCode (*quac_ts_monitor)(TS, PetscInt, PetscReal, Vec, void *);

struct qsystem_impl;
/* qsystem: qsystem_p.h:69-116 (public fields kept; engine state is opaque) */
typedef struct qsystem_s {
  PetscInt num_time_indep, num_time_dep;
  PetscInt hspace_frozen;
  PetscBool dm_equations, mcwf_solver, time_step_called;
  PetscInt mat_allocated;
  PetscInt num_subsystems;
  op_handle *subsystem_list;
  PetscInt total_levels, dim;
  qvec solution_qvec;
  PetscInt np, nid;
  PetscReal current_time;
  quac_ts_monitor ts_monitor;
  void *ts_ctx;
  PetscInt num_circuits, circuit_list_size, current_circuit;
  circuit *circuit_list;
  struct qsystem_impl *impl;
} *qsystem;

/* ------------------------------------------------------------ runtime */
void QuaC_initialize(int argc, char **args);           /* quac.c:25-58 */
void QuaC_finalize(void);                               /* quac.c:89-111 */
void QuaC_clear(void);                                  /* quac.c:60-87 */
int PetscPrintf(int comm, const char *fmt, ...);        /* PETSc printing, rank 0 only */

/* ----------------------------------------------------- system building */
void initialize_system(qsystem *qsys);                  /* qsystem.c:16-70 */
void destroy_system(qsystem *qsys);                     /* qsystem.c:72-91 */
void create_op_sys(qsystem qsys, PetscInt levels, op_handle *op);      /* qsystem.c:153-230 */
void destroy_op_sys(op_handle *op);                     /* qsystem.c:349-361 */
void create_vec_op_sys(qsystem qsys, PetscInt levels, vec_op *vop);    /* qsystem.c:276-329 */
void destroy_vec_op_sys(vec_op *vop);                   /* qsystem.c:331-340 */
void set_init_excited_op(op_handle op, PetscInt initial_exc);           /* qsystem.c:1339-1349 */
void add_ham_term(qsystem qsys, PetscScalar a, PetscInt num_ops, ...); /* qsystem.c:407-434 */
void add_lin_term(qsystem qsys, PetscScalar a, PetscInt num_ops, ...); /* qsystem.c:436-462 */
void add_lin_term_list(qsystem qsys, PetscScalar a, PetscInt num_ops, op_handle *ops); /* qsystem.c:464-489 */
void add_ham_term_list(qsystem qsys, PetscScalar a, PetscInt num_ops, op_handle *ops); /* list form of qsystem.c:407-434 */
/* Time-dependent terms: qsystem.h:31-32, qsystem.c:491-552.  The term's
 * superoperator is built with coefficient 1 and scaled at every stage time
 * t by a * f(t, ctx) (the reference calls f with the time and ctx,
 * qsystem.c:1311-1316, although its header prints a one-argument type);
 * terms whose |a f(t)| is at most 1e-10 are skipped at that stage
 * (qsystem.c:1320).  add_lin_term_time_dep selects the density-matrix
 * equations like add_lin_term. */
typedef PetscScalar (*quac_time_dep_func)(PetscReal t, void *ctx);
void add_ham_term_time_dep(qsystem qsys, PetscScalar a, void *ctx, quac_time_dep_func f, PetscInt num_ops, ...);
void add_lin_term_time_dep(qsystem qsys, PetscScalar a, void *ctx, quac_time_dep_func f, PetscInt num_ops, ...);
/* List forms of the two (kind 1 = Hamiltonian, 2 = Lindblad) for callers
 * whose callbacks cannot return a complex value (language bindings):
 * g(t, ctx, &re, &im) writes f(t). */
typedef void (*quac_time_dep_func_parts)(PetscReal t, void *ctx, double *re, double *im);
int quac_add_term_time_dep_list(qsystem qsys, int kind, PetscScalar a, void *ctx, quac_time_dep_func_parts g,
                                PetscInt num_ops, op_handle *ops);
void clear_mat_terms_sys(qsystem qsys);                 /* qsystem.c:557-591 */
void construct_matrix(qsystem qsys);                    /* qsystem.c:593-676 */
void use_mcwf_solver(qsystem qsys, PetscInt num_tot_trajs, PetscInt seed); /* qsystem.c:358-403 */

/* ---------------------------------------------------------- time steps */
/* qsystem.c:895-1098.  Default scheme: Bogacki-Shampine 3(2), adaptive,
 * atol = rtol = 5e-7, step limits [0.01, 1], final step matched to tmax;
 * QuaC_initialize's -ts_rk_type / -ts_adapt_type / -ts_rtol / -ts_atol /
 * -ts_max_steps options override these as TSSetFromOptions does. */
void time_step_sys(qsystem qsys, qvec x, PetscReal t0, PetscReal tmax, PetscReal dt,
                   PetscInt steps_max);
void set_ts_monitor_sys(qsystem qsys, quac_ts_monitor monitor, void *ctx); /* qsystem.c:875-879 */

/* --------------------------------------------------------------- qvecs */
void create_qvec_sys(qsystem qsys, qvec *q);            /* qvec_utilities.c:633-648 */
void create_dm_sys(qsystem qsys, qvec *q);              /* qvec_utilities.c:650-703 */
void create_wf_sys(qsystem qsys, qvec *q);              /* qvec_utilities.c:705-763 */
void create_arb_qvec(qvec *q, PetscInt nstates, qvec_type type);      /* qvec_utilities.c:471-521 */
void destroy_qvec(qvec *q);                             /* qvec_utilities.c:1076-1091 */
/* The variadic locations of add_to_qvec (row, col for a density matrix, the
 * index for a wavefunction) are read as PetscInt (int64_t), as in the
 * reference; the Fock states of add_to_qvec_fock_op / get_qvec_loc_fock_op
 * are read from the low 32 bits of their argument slots, so int literals
 * and PetscInt values both work there (a state is below its op's levels). */
void add_to_qvec(qvec q, PetscScalar alpha, ...);       /* qvec_utilities.c:919-969 */
void add_to_qvec_loc(qvec q, PetscScalar alpha, PetscInt loc);        /* qvec_utilities.c:879-897 */
/* Basis states by Fock occupations: (op, PetscInt fock state) pairs; the
 * index is sum fock_i * n_before_i as in the reference (qvec_utilities.c:
 * 996-1033), the diagonal element for a density matrix. */
void add_to_qvec_fock_op(PetscScalar alpha, qvec q, PetscInt num_ops, ...);                 /* qvec_utilities.c:832-857 */
void add_to_qvec_fock_op_list(PetscScalar alpha, qvec q, PetscInt num_ops, op_handle *ops,
                              PetscInt *fock_states);                                         /* qvec_utilities.c:863-872 */
void get_qvec_loc_fock_op(qvec q, PetscInt *loc, PetscInt num_ops, ...);                    /* qvec_utilities.c:973-994 */
void get_qvec_loc_fock_op_list(qvec q, PetscInt *loc, PetscInt num_ops, op_handle *ops,
                               PetscInt *fock_states);                                        /* qvec_utilities.c:996-1033 */
void assemble_qvec(qvec q);                             /* qvec_utilities.c:1047-1066 */
void set_qvec_from_init_excited_op(qsystem qsys, qvec q);             /* qvec_utilities.c:2540-2566 */
void get_dm_element_qvec(qvec q, PetscInt row, PetscInt col, PetscScalar *val); /* qvec_utilities.c:322-337 */
void get_wf_element_qvec(qvec q, PetscInt loc, PetscScalar *val);     /* qvec_utilities.c:409-414 */
void get_trace_qvec(qvec q, PetscScalar *val);          /* qvec_utilities.c:378-392 */
void get_expectation_value_qvec(qvec q, PetscScalar *val, PetscInt num_ops, ...); /* qvec_utilities.c:1133-1150 */
void get_expectation_value_qvec_list(qvec q, PetscScalar *val, PetscInt num_ops, op_handle *ops); /* qvec_utilities.c:1176-1195 */
void get_fidelity_qvec(qvec q1, qvec q2, PetscReal *fidelity, PetscReal *var); /* qvec_utilities.c:2159-2245 (dm-wf, wf-wf) */
void get_bitstring_probs(qvec q, PetscInt *nloc, PetscReal **probs, PetscReal **vars); /* qvec_utilities.c:1682-1718 */
void copy_qvec(qvec src, qvec dst);                     /* qvec_utilities.c:33-55 */
void print_qvec(qvec q);                                /* qvec_utilities.c:277-289 */
void read_qvec_dm_binary(qvec *q, const char filename[]);  /* qvec_utilities.c:129-167 */
void read_qvec_wf_binary(qvec *q, const char filename[]);  /* qvec_utilities.c:97-127 */
void print_qvec_file(qvec q, char filename[]);           /* PETSc-binary Vec writer (qvec_utilities.c:203-212 writes text; this writes the binary format read above) */

/* ------------------------------------------------------------ circuits */
void create_circuit(circuit *circ, PetscInt num_gates); /* quantum_gates.c:610-632 */
void destroy_circuit(circuit *circ);                    /* quantum_gates.c:634-641 */
void add_gate_to_circuit_sys(circuit *circ, PetscReal time, gate_type g, ...); /* quantum_circuits.c:172-255 */
void schedule_circuit_layers(qsystem qsys, circuit *circ);            /* quantum_circuits.c:316-404 */
void apply_circuit_to_sys(qsystem qsys, circuit *circ, PetscReal time); /* quantum_circuits.c:407-431 */
void apply_circuit_to_qvec(qsystem qsys, circuit circ, qvec q);       /* quantum_circuits.c:143-159 */
void apply_gate2(qvec q, gate_type g, ...);             /* quantum_circuits.c:776-847 */
/* Non-variadic form of add_gate_to_circuit_sys for bindings (no reference
 * counterpart): nq qubits, angles theta / phi / lambda, CUSTOM gates take
 * ctx and func.  Returns 0 on success. */
int quac_add_gate(circuit *circ, double time, int gate, int nq, const int *qubits, double theta, double phi,
                  double lambda, void *ctx, void *func);

/* ------------------------------------------------ circuit front ends */
/* qasm_parser.h: each reads a file into a new circuit (one gate per
 * instruction) and sets *num_qubits. */
void qiskit_qasm_read(char filename[], PetscInt *num_qubits, circuit *circ);  /* qasm_parser.c:583-650 */
void qiskit_tqasm_read(char filename[], PetscInt *num_qubits, circuit *circ); /* qasm_parser.c:652-718 */
void cirq_qasm_read(char filename[], PetscInt *num_qubits, circuit *circ);    /* qasm_parser.c:720-787 */
void projectq_qasm_read(char filename[], PetscInt *num_qubits, circuit *circ); /* qasm_parser.c:195-258 */
void quil_read(char filename[], PetscInt *num_qubits, circuit *circ);         /* qasm_parser.c:12-72 */

/* ------------------------------------------------- legacy global API */
void create_op(int levels, op_handle *op);              /* operators.c:59-200 */
void create_vec(int levels, vec_op *vop);               /* operators.c:210-242 */
void destroy_op(op_handle *op);                         /* quac.c:113-126 */
void destroy_vec(vec_op *vop);                          /* quac.c:128-141 */
void add_to_ham(PetscScalar a, op_handle op);           /* operators.c:290-337 */
void add_to_ham_mult2(PetscScalar a, op_handle op1, op_handle op2);   /* operators.c:405-488 */
void add_to_ham_mult3(PetscScalar a, op_handle op1, op_handle op2, op_handle op3); /* operators.c:601-663 */
void add_lin(PetscScalar a, op_handle op);              /* operators.c:679-719 */
void add_lin_mult2(PetscScalar a, op_handle op1, op_handle op2);      /* operators.c:743-821 */
void steady_state(Vec x);                               /* solver.c:33-221 */
void set_ts_monitor(quac_ts_monitor monitor);           /* solver.c:526-532 */
void set_ts_monitor_ctx(quac_ts_monitor monitor, void *ctx);            /* solver.c:542-545 */
void time_step(Vec x, PetscReal init_time, PetscReal time_max, PetscReal dt, PetscInt steps_max); /* solver.c:236-510 */
void create_full_dm(Vec *dm);                           /* dm_utilities.c:635-655 */
void create_dm(Vec *dm, PetscInt size);                 /* dm_utilities.c:616-623 */
void destroy_dm(Vec dm);                                /* dm_utilities.c:1029-1032 */
void add_value_to_dm(Vec dm, PetscInt row, PetscInt col, PetscScalar val); /* dm_utilities.c:1049-1061 */
void assemble_dm(Vec dm);                               /* dm_utilities.c:1073-1076 */
void get_dm_element(Vec dm, PetscInt row, PetscInt col, PetscScalar *val); /* dm_utilities.c:965-982 */
int get_num_populations(void);                          /* dm_utilities.c:1127-1143 */
/* dm_utilities.c:1157-1325: per subsystem of the legacy system, Tr(n rho);
 * a VEC subsystem gives one population per level.  *populations must hold
 * get_num_populations() doubles. */
void get_populations(Vec x, double **populations);

/* --------------------------------------------- PETSc Vec/TS stand-ins */
PetscErrorCode VecGetArray(Vec v, PetscScalar **a);     /* maps the data to host memory */
PetscErrorCode VecRestoreArray(Vec v, PetscScalar **a); /* writes host changes back */
PetscErrorCode VecGetSize(Vec v, PetscInt *n);
PetscErrorCode VecDuplicate(Vec v, Vec *out);
PetscErrorCode VecCopy(Vec src, Vec dst);
PetscErrorCode VecDestroy(Vec *v);
PetscErrorCode VecCreateSeq(int comm, PetscInt n, Vec *v);
PetscErrorCode TSGetTime(TS ts, PetscReal *t);
PetscErrorCode TSGetTimeStep(TS ts, PetscReal *dt);

/* ------------------------------- entry points with no QuaC counterpart */
/* Steady state of a qsystem (the reference only offers the legacy global
 * form, solver.c:33-221): solves (L + e0 vec(I)^T) x = e0 by restarted
 * GMRES on the GPU; returns the iterations used, or -1 on failure. */
PetscInt steady_state_sys(qsystem qsys, qvec x);
/* One application y = L x of the constructed Liouvillian on device
 * buffers of qsys->dim complex128 values (the TSComputeRHSFunctionLinear
 * action, qsystem.c:937).  Returns 0 on success. */
int quac_lrho_apply_device(qsystem qsys, const void *x_dev, void *y_dev);
/* Same on host buffers: copies x in, applies L, copies y out. */
int quac_lrho_apply_host(qsystem qsys, const PetscScalar *x_host, PetscScalar *y_host);
/* No counterpart in the reference (a QuaC program would MatView its mat_A,
 * qsystem.c:957-963, onto a binary viewer): writes the operator the
 * system's terms define -- the D^2 x D^2 Liouvillian in the column-stacked
 * ordering, or -i H for a wavefunction system -- as a PETSc binary AIJ
 * matrix with 64-bit indices (the format MatLoad reads and the reference's
 * test fixtures use), built on the host from the compiled term tables. */
int quac_write_superoperator_binary(qsystem qsys, const char *filename);
/* No reference counterpart.  quac_lrho_apply_device without any device
 * allocation at call time, for callers that must not allocate inside their
 * loop: a framework whose memory pool already holds the device's memory, or
 * a tight control loop where cudaFree's device-wide synchronisation would
 * stall other streams.  The multi-pass kernel's D^2 running sum lives in a
 * fixed 16 MiB device array, so qsys->dim may be at most 2^20 (10 qubits);
 * larger systems return an error.  Call quac_lrho_noalloc_setup(qsys) once,
 * with the system's device current, before the first apply: it may allocate
 * (the system's term tables) and loads every kernel the apply can launch, so
 * that the apply itself allocates nothing.
 * The apply computes in the precision quac_set_lrho_precision selects, like
 * quac_lrho_apply_device, and returns once y is complete.  All systems on a
 * device share the one array: calls that overlap in time race and must be
 * serialised by the caller. */
int quac_lrho_noalloc_setup(qsystem qsys);
int quac_lrho_apply_device_noalloc(qsystem qsys, const void *x_dev, void *y_dev);
/* Observable monitor (no reference counterpart: QuaC programs read
 * populations in a TS monitor after every step, simple_jc_test.c:76-90).
 * The expectation values Tr(O_k rho) of nobs operator products (product k
 * is ops[sum_{j<k} nops[j] ...], as in get_expectation_value_qvec) are
 * recorded on the GPU after every step of time_step_sys and passed to cb in
 * batches of up to `batch` steps: cb(n, steps, times, values, ctx) with
 * values[i * nobs + k] for step steps[i] at time times[i].  Small density
 * matrices (D^2 <= 4096) integrated with fixed RK4 then run many steps per
 * launch with the state in shared memory; other runs record the values
 * with one reduction per observable and step.  cb = NULL removes the
 * monitor. */
typedef void (*quac_observable_monitor)(PetscInt nsteps, const PetscInt *steps, const PetscReal *times,
                                        const PetscScalar *values, void *ctx);
int quac_set_observable_monitor(qsystem qsys, PetscInt nobs, const PetscInt *nops, op_handle *ops,
                                quac_observable_monitor cb, void *ctx, PetscInt batch);
/* Batched ensembles (no reference counterpart: QuaC integrates one system
 * per time_step_sys call, qsystem.c:895-1098).  Many independent systems,
 * each built with the usual calls (initialize_system, create_op_sys,
 * add_ham_term, add_lin_term), are integrated together as density matrices
 * in one persistent launch, each with its own adaptive Dormand-Prince 5(4)
 * step (the -ts_rk_type 5dp controller of time_step_sys).  The states are
 * one packed array: instance i occupies D_i^2 column-stacked values from
 * quac_ensemble_state_offset(ens, i). */
typedef struct quac_ensemble_s *quac_ensemble;
int quac_ensemble_create(quac_ensemble *ens, int64_t n, const qsystem *systems);
int quac_ensemble_destroy(quac_ensemble ens);
/* precision 0: complex128 throughout; 1: complex64 right-hand-side
 * increments with the complex128 state and controller.  Defaults: 0,
 * atol = rtol = 5e-7, step limits [0.01, 1], 10^6 steps. */
int quac_ensemble_set_options(quac_ensemble ens, int precision, double atol, double rtol, double hmin,
                              double hmax, int64_t max_steps);
/* Launch shape: warps per CTA (4, 8, 16, 32), CTAs per SM, target density
 * matrix elements per thread (sets how many warps share an instance). */
int quac_ensemble_set_shape(quac_ensemble ens, int warps, int ctas_per_sm, int elems_per_thread);
int quac_ensemble_get_shape(quac_ensemble ens, int *warps, int *ctas_per_sm, int *elems_per_thread);
/* Times every launch shape on a short run t0 .. t0 + t_probe, keeps the
 * fastest and leaves the states unchanged. */
int quac_ensemble_tune(quac_ensemble ens, double t0, double t_probe, double dt0, double *best_ms);
int64_t quac_ensemble_state_offset(quac_ensemble ens, int64_t i);
void *quac_ensemble_state_device_ptr(quac_ensemble ens);
int quac_ensemble_set_states(quac_ensemble ens, const PetscScalar *rho);
int quac_ensemble_get_states(quac_ensemble ens, PetscScalar *rho);
/* Integrates every instance from t0 to tmax (first step dt0); fails if an
 * instance hit the step limit or a non-finite error norm. */
int quac_ensemble_run(quac_ensemble ens, double t0, double tmax, double dt0);
/* complex64 mode: a step whose error estimate lies within `margin` of the
 * accept threshold (|err - 1| < margin, default 0.1) is estimated again
 * with complex128 stages, so the accept / reject decisions follow the
 * complex128 ones; 0 turns the re-evaluation off. */
int quac_ensemble_set_redo_margin(quac_ensemble ens, double margin);
/* Steps of instance i re-evaluated in complex128 during the last run. */
int64_t quac_ensemble_redone_steps(quac_ensemble ens, int64_t i);
/* complex64 mode: every accepted step adds an estimate of the rounding its
 * complex64 increments left in the state (8 eps32 h max_e sum_j |b_j dK_j|);
 * once an instance's sum exceeds `budget` (default 1e-7) it takes its
 * remaining steps with complex128 stages.  0 runs every step in complex128
 * after the first. */
int quac_ensemble_set_fp32_budget(quac_ensemble ens, double budget);
/* Steps of instance i taken in complex128 after its budget ran out. */
int64_t quac_ensemble_f64_steps(quac_ensemble ens, int64_t i);
int quac_ensemble_get_stats(quac_ensemble ens, int64_t i, double *t, int64_t *steps, int64_t *rejected,
                            int *flags);
/* Re(diag rho_i) of every instance, packed: D_0 values, then D_1, ... */
int quac_ensemble_populations(quac_ensemble ens, double *pops);
/* Steady state from a proposed initial state and a proposed dominant
 * subspace (no reference counterpart; solver.c:33-221 always starts from
 * e0).  x holds the initial guess on entry.  U: D x kd column-major, with
 * orthonormal columns (kd <= 16); the kd^2 matrices u_i u_j^H span the
 * deflation space W.  GMRES runs on P A with P = I - A W (W^H A W)^-1 W^H
 * (Galerkin projection) and the iterate is corrected after each restart,
 * so the residual components in A span W are removed exactly.  With
 * deflation refresh on (default), every restart after the first replaces
 * U by one Rayleigh-Ritz step toward the kd leading eigenvectors of the
 * Hermitian part of the current iterate.  The solve starts from x or e0,
 * whichever has the smaller residual; deflated GMRES runs for at most
 * maxit_guided iterations, then plain GMRES continues from its iterate if
 * needed (restart length per quac_set_gmres_restart, basis precision per
 * quac_set_gmres_precision).  Same system and tolerance as steady_state.
 * Returns the iterations (-1 on error); *residual = ||b - A x|| at the
 * end. */
PetscInt quac_steady_state_guided(qsystem qsys, qvec x, const PetscScalar *U, PetscInt kd,
                                  PetscInt maxit_guided, PetscReal *residual);
/* Learned warm start for steady states (no reference counterpart): an MLP
 * (4 normalised parameters -> hidden -> hidden -> rank-r factors F, D x r
 * complex) trained on steady states the solver produced; F F^H proposes
 * the initial state and the leading directions of range F the deflation
 * space of quac_steady_state_guided.  Dense layers run on the tensor cores
 * (TF32, FP32 accumulation). */
typedef struct quac_wsnet_s *quac_wsnet;
int quac_wsnet_create(quac_wsnet *net, int D, int rank, int hidden, int batch, int max_samples, uint64_t seed);
int quac_wsnet_destroy(quac_wsnet net);
int quac_wsnet_add_sample(quac_wsnet net, const double *theta4, qvec rho);
int quac_wsnet_num_samples(quac_wsnet net);
int64_t quac_wsnet_num_params(quac_wsnet net);
int quac_wsnet_get_params(quac_wsnet net, float *params);
int quac_wsnet_set_params(quac_wsnet net, const float *params);
/* Mean loss and its gradient over samples [0, nb), no update. */
int quac_wsnet_loss_grad(quac_wsnet net, int nb, double *loss, float *grad);
int quac_wsnet_train(quac_wsnet net, int epochs, double lr, uint64_t seed, double *final_loss);
int quac_wsnet_predict(quac_wsnet net, int n, const double *theta4, PetscScalar *factors);
/* Time-steps host data in place: one call = H2D + integration + D2H. */
int quac_time_step_host(qsystem qsys, PetscScalar *x_host, PetscReal t0, PetscReal tmax,
                        PetscReal dt, PetscInt steps_max);

#define QUAC_ERRORS_EXIT 0
#define QUAC_ERRORS_RETURN 1
void quac_set_error_mode(int mode);
const char *quac_last_error(void);
void quac_clear_error(void);
/* Integrator selection without argv: scheme "3bs" | "4" | "5dp",
 * adapt "basic" | "none"; non-positive tolerances keep the current ones. */
int quac_set_ts_options(const char *rk_type, const char *adapt_type, double rtol, double atol,
                        PetscInt max_steps);
/* Device pointer of a qvec (complex128, qvec->n values).  Work the caller
 * queues on it must be ordered with the system's stream (the one given to
 * quac_set_stream, or synchronise first): time_step_sys and the other
 * calls wait only on their own stream. */
void *quac_qvec_device_ptr(qvec q);
/* Launch this system's kernels on a caller-owned CUDA stream (NULL: the
 * library's own stream).  Calls return when their work on that stream is
 * done. */
void quac_set_stream(qsystem qsys, void *cuda_stream);
/* Kernel selection for systems compiled afterwards: 0 = default (multi-pass
 * bit-mask kernel for all-qubit systems of seven or more qubits, single-pass
 * bit-mask kernel for six, generic table kernel otherwise), 1 = generic
 * table kernel for every system, 2 = single-pass bit-mask kernel whenever
 * the system is all-qubit. */
void quac_set_kernel_path(int path);
/* Contraction precision of L.x (no reference counterpart): 0 = complex128
 * (default), 1 = complex64 contraction and accumulation inside the
 * multi-pass bit-mask kernel (all-qubit systems of seven or more qubits),
 * with the state, the RK stage combinations, the error norm and every
 * reduction kept in complex128.  Other kernels always run complex128. */
int quac_set_lrho_precision(int precision);
/* Hermitian mode of time_step_sys (no reference counterpart): 1 (default) =
 * automatic: for a system of 7 or more qubits on the multi-pass kernel whose
 * terms preserve Hermiticity, integrated from a Hermitian state with no gate
 * events inside the run, every L.x computes the 64 x 64 blocks on and above
 * the block diagonal only and writes the others as their conjugate
 * transposes (half the outputs and a third of the traffic); 2 = the same,
 * and also in quac_lrho_apply_device / quac_lrho_apply_host when x is
 * Hermitian to 1e-13; 0 = always compute every element. */
int quac_set_hermitian_mode(int mode);
/* Preconditioner of the steady-state GMRES (the role PCASM / ILU(0) plays in
 * solver.c:167-198): 1 = the exact inverse of the no-jump
 * Liouvillian L0 X = -i (H_eff X - X H_eff^H), H_eff = H - i/2 sum a C^dag C,
 * applied on the right through the eigen-decomposition of H_eff (computed
 * once per system on the GPU; four D x D complex GEMMs per iteration);
 * 2 (default) = the same form built from the Hermitian eigensolver: H_eff = H - i/2 G,
 * H = U diag(w) U^H, eigenvalues of H_eff taken as w_k - i/2 (U^H G U)_kk
 * (exact when G commutes with H, a fixed approximation otherwise; cheaper to
 * set up, GMRES still converges to the same answer); 0 = none.  The guided
 * solve with a deflation space runs unpreconditioned. */
int quac_set_gmres_preconditioner(int mode);
/* Tolerance of the steady-state GMRES on the true residual ||b - A x||
 * with ||b|| = 1 (default 1e-11 as solver.c:14, 179; -ksp_rtol on the
 * QuaC_initialize command line does the same). */
int quac_set_gmres_tolerance(double rtol);
/* No reference counterpart (PCSetUp builds PETSc's preconditioner the same
 * way ahead of KSPSolve).  Builds qsys's steady-state preconditioner now;
 * 0 on success. */
int quac_steady_precond_setup(qsystem qsys);
/* Decompositions computed in this process and their total host time (s). */
void quac_steady_precond_stats(int64_t *builds, double *seconds);
/* Restart length of the steady-state GMRES (default 100 as in solver.c;
 * -ksp_gmres_restart on the QuaC_initialize command line does the same).
 * Up to 1024: a long Krylov space resolves the slow Lindblad modes that
 * stall GMRES(100), at (m+1) x D^2 x 16 bytes of device memory. */
int quac_set_gmres_restart(int m);
/* Precision of the steady-state GMRES basis (no reference counterpart;
 * solver.c runs KSPGMRES in PETSc's complex128).  0 (default): complex128.
 * 1: FP32 inner / FP64 refined: the Krylov vectors are stored in complex64
 * (half the Gram-Schmidt traffic), while L.x, the projections, the
 * iterate and the residual b - A x formed at every restart stay
 * complex128, so each restart refines the solution to the same
 * complex128 tolerance; the steady-state preconditioner, when on, is then
 * applied to the complex64 vectors in complex64 as well.  If the true
 * residual has not fallen below 0.9x its value 20 restarts earlier (the
 * complex64 rounding of the basis then costs more than a cycle gains, as
 * on ill-conditioned systems), the solve continues with a complex128
 * basis. */
int quac_set_gmres_precision(int precision);
/* Deflation refresh of quac_steady_state_guided (no reference
 * counterpart): 1 (default) = at every restart after the first, the
 * deflation space is rebuilt from one Rayleigh-Ritz step toward the
 * leading eigenvectors of the current iterate; 0 = the proposed U is kept
 * for the whole solve. */
int quac_set_deflation_refresh(int mode);
/* Number of L.x applications that ran in Hermitian mode (diagnostics). */
int64_t quac_hermitian_apply_count(void);
/* Number of kernels this library has launched (diagnostics). */
int64_t quac_kernel_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif /* QUAC_B200_H_ */

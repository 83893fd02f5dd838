/* A QuaC-style C program (Jaynes-Cummings, emitter x cavity) written against
 * the reference's C API and built unchanged against this engine's drop-in
 * headers:  gcc -std=c99 -I include/quac jc_drop_in.c -L quac_b200 -lquac_b200
 * Prints "step time <n_qb> <n_cav>" every 50 steps and the final values. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include "quac.h"
#include "operators.h"
#include "solver.h"
#include "quantum_gates.h"
#include "quantum_circuits.h"
#include "petsc.h"
#include "qsystem.h"

qvec dm_dummy;
operator qb, cav;

PetscErrorCode monitor(TS ts, PetscInt step, PetscReal time, Vec rho, void *ctx) {
  Vec saved = dm_dummy->data;
  PetscScalar n_qb, n_cav;
  dm_dummy->data = rho;
  get_expectation_value_qvec(dm_dummy, &n_qb, 1, qb->n);
  get_expectation_value_qvec(dm_dummy, &n_cav, 1, cav->n);
  if (step % 50 == 0)
    PetscPrintf(PETSC_COMM_WORLD, "step %d %.10f %.15e %.15e\n", (int)step, time,
                PetscRealPart(n_qb), PetscRealPart(n_cav));
  dm_dummy->data = saved;
  PetscFunctionReturn(0);
}

int main(int argc, char **args) {
  qsystem qsys;
  qvec rho;
  PetscScalar v;
  QuaC_initialize(argc, args);
  initialize_system(&qsys);
  create_op_sys(qsys, 2, &qb);
  create_op_sys(qsys, 10, &cav);
  add_ham_term(qsys, 0.1, 2, cav->dag, qb);
  add_ham_term(qsys, 0.1, 2, cav, qb->dag);
  add_lin_term(qsys, 1e-2, 1, cav);
  add_lin_term(qsys, 1e-3, 1, qb);
  construct_matrix(qsys);
  set_ts_monitor_sys(qsys, monitor, NULL);
  create_qvec_sys(qsys, &rho);
  create_qvec_sys(qsys, &dm_dummy);
  add_to_qvec(rho, 1.0, 10, 10);
  assemble_qvec(rho);
  time_step_sys(qsys, rho, 0.0, 2.0, 0.01, 100000);
  get_expectation_value_qvec(rho, &v, 1, qb->n);
  printf("final_qb %.15e\n", PetscRealPart(v));
  get_expectation_value_qvec(rho, &v, 1, cav->n);
  printf("final_cav %.15e\n", PetscRealPart(v));
  get_trace_qvec(rho, &v);
  printf("trace %.15e\n", PetscRealPart(v));
  destroy_qvec(&rho);
  destroy_qvec(&dm_dummy);
  destroy_system(&qsys);
  QuaC_finalize();
  return 0;
}

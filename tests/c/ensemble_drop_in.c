/* Sixteen driven Jaynes-Cummings systems built with QuaC's C API and
 * integrated together by the batched ensemble entry points (no QuaC
 * counterpart).  Prints "inst <i> <nc> <emitter excited population>" at
 * t = 2 for every instance.
 *   gcc -std=c99 -I include/quac ensemble_drop_in.c -L quac_b200 -lquac_b200 */
#include <complex.h>
#include <stdio.h>
#include <stdlib.h>
#include "quac.h"
#include "qsystem.h"
#include "operators.h"

#define NI 16

int main(int argc, char **args) {
  qsystem sys[NI];
  int nc[NI];
  QuaC_initialize(argc, args);
  int64_t total = 0;
  for (int i = 0; i < NI; i++) {
    operator qb, cav;
    nc[i] = 3 + i % 6;
    const double delta = 0.1 * (i % 5) - 0.2, g = 0.05 + 0.01 * i, omega = 0.02 * i, kappa = 0.01 + 0.005 * i;
    initialize_system(&sys[i]);
    create_op_sys(sys[i], 2, &qb);
    create_op_sys(sys[i], nc[i], &cav);
    add_ham_term(sys[i], delta, 1, cav->n);
    add_ham_term(sys[i], g, 2, cav->dag, qb);
    add_ham_term(sys[i], g, 2, cav, qb->dag);
    add_ham_term(sys[i], omega, 1, cav);
    add_ham_term(sys[i], omega, 1, cav->dag);
    add_lin_term(sys[i], kappa, 1, cav);
    add_lin_term(sys[i], 1e-3, 1, qb);
    total += (int64_t)(2 * nc[i]) * (2 * nc[i]);
  }
  quac_ensemble ens;
  if (quac_ensemble_create(&ens, NI, sys)) return 1;
  PetscScalar *rho = calloc((size_t)total, sizeof(PetscScalar));
  for (int i = 0; i < NI; i++) {
    const int64_t D = 2 * nc[i], off = quac_ensemble_state_offset(ens, i);
    rho[off + nc[i] * D + nc[i]] = 1.0;  /* |e,0><e,0|: emitter level 1 = index nc */
  }
  quac_ensemble_set_states(ens, rho);
  if (quac_ensemble_run(ens, 0.0, 2.0, 0.05)) return 1;
  quac_ensemble_get_states(ens, rho);
  for (int i = 0; i < NI; i++) {
    const int64_t D = 2 * nc[i], off = quac_ensemble_state_offset(ens, i);
    double pe = 0.0;
    for (int k = 0; k < nc[i]; k++) pe += creal(rho[off + (nc[i] + k) * D + nc[i] + k]);
    printf("inst %d %d %.15e\n", i, nc[i], pe);
  }
  quac_ensemble_destroy(ens);
  free(rho);
  for (int i = 0; i < NI; i++) destroy_system(&sys[i]);
  QuaC_finalize();
  return 0;
}

/* Fock-state indices through the variadic entry points with plain int
 * literals, as QuaC programs write them (tests/qvec_utilities_tests.c);
 * with four (op, state) pairs the last ones are passed on the stack.  Needs
 * no GPU: the qvec is a header on the stack.  Prints "wf <loc>" and
 * "dm <loc>". */
#include <stdio.h>
#include <string.h>
#include "quac.h"
#include "operators.h"
#include "qsystem.h"

int main(int argc, char **args) {
  qsystem qsys;
  operator a, b, c, d;
  struct qvec_s wf, dm;
  PetscInt loc;
  QuaC_initialize(argc, args);
  initialize_system(&qsys);
  create_op_sys(qsys, 2, &a);
  create_op_sys(qsys, 3, &b);
  create_op_sys(qsys, 4, &c);
  create_op_sys(qsys, 2, &d);
  memset(&wf, 0, sizeof(wf));
  memset(&dm, 0, sizeof(dm));
  wf.my_type = WAVEFUNCTION;
  wf.n = 48;
  dm.my_type = DENSITY_MATRIX;
  dm.n = 48 * 48;
  get_qvec_loc_fock_op(&wf, &loc, 4, a, 1, b, 2, c, 3, d, 1);
  printf("wf %lld\n", (long long)loc);
  get_qvec_loc_fock_op(&dm, &loc, 4, a, 1, b, 2, c, 3, d, 1);
  printf("dm %lld\n", (long long)loc);
  destroy_system(&qsys);
  return 0;
}

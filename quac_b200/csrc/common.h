// Internal definitions shared by the host runtime and the CUDA kernels.
#pragma once
#include <atomic>
#include <cuda_runtime.h>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "quac_b200.h"

namespace quac {

using cplx = std::complex<double>;

// ---------------------------------------------------------------- errors
// Records an error message; in EXIT mode prints it and exits like the
// reference's PetscPrintf + exit() convention (e.g. qsystem.c:20-24).
void fail(int exit_code, const char *fmt, ...);
bool has_error();
void check_cuda(cudaError_t e, const char *what, const char *file, int line);
#define QCUDA(x) ::quac::check_cuda((x), #x, __FILE__, __LINE__)

void count_launch(int n = 1);

// ------------------------------------------------------------ device prog
// Compiled form of the Lindblad terms of one qsystem (see terms.cpp).
//   y[r,c] = (dr[r] + dc[c] + sum_t Jdrow_t[r] Jdcol_t[c]) x[r,c]
//          + sum_t Lval_t[r] x[Lmap_t[r], c]                       left H terms
//          + sum_t Rval_t[c] x[r, Rmap_t[c]]                       right H terms
//          + sum_t Jrow_t[r] Jcol_t[c] x[Jmap_t[r], Jmap_t[c]]      jumps
// Maps hold -1 where the operator row is empty.  Element (r,c) lives at
// c*D + r (column stacking).  For a wavefunction, ncols = 1 and only the
// left terms and dr are present.
struct DevProg {
  int D;
  int ncols;
  int nL, nR, nJ, nJd;
  const int *Lmap;
  const double2 *Lval;
  const int *Rmap;
  const double2 *Rval;
  const int *Jmap;
  const double2 *Jrow;
  const double2 *Jcol;
  const double2 *Jdrow;
  const double2 *Jdcol;
  const double2 *dr;
  const double2 *dc;
  // qubit fast path: every subsystem has two levels and every term is a
  // one-qubit operator class the bit-mask kernel understands
  int qubit_path;
};

// Host copy of the compiled terms (kept for the CPU-side checks and for
// rebuilding the device program).
struct HostProg {
  int D = 0, ncols = 0;
  std::vector<std::vector<int>> Lmap, Rmap, Jmap;
  std::vector<std::vector<cplx>> Lval, Rval, Jrow, Jcol, Jdrow, Jdcol;
  std::vector<cplx> dr, dc;
};

// Stage epilogue of the fused L.x kernel.  With K = (L x)[i]:
//   kout[i]       = K                              (if kout)
//   out_u[i]      = (base_u ? base_u[i] : 0) + coef_u * K   for u < nupd
//   if nsum: the error-norm term (|e_i| / (atol + rtol*max(|y_i|,|yn_i|)))^2
//   is accumulated into *nsum, with e_i the value of update `err_upd`,
//   y_i = ny[i] and yn_i = nyn[i] (or the value of update `yn_upd` >= 0).
struct Epi {
  double2 *kout;
  int nupd;
  double2 *out[3];
  const double2 *base[3];
  double coef[3];
  double *nsum;
  int err_upd;
  int yn_upd;
  const double2 *ny;
  const double2 *nyn;
  double atol, rtol;
  // nonzero: x (and therefore L x) is Hermitian and L preserves Hermiticity;
  // the multi-pass kernel then computes the upper block triangle only and
  // writes the rest as its conjugate transpose
  int herm;
};

// Qubit fast path: every subsystem is two-level, so each operator product
// is, per qubit, a flip / condition / sign and the whole term is
//   w(r) = coef * (-1)^popc(r & smask)   if (r & cmask) == cval, else 0,
//   partner r ^ fmask
// on the row index (left terms), the column index (right terms) or both
// (jumps, sign taken over r and c).  Single-qubit diagonal jumps are summed
// into tables over groups of three qubits (index (row bits << 3) | col bits).
struct QTerm {
  uint32_t fmask, cmask, cval, smask;
  double2 coef;
};
constexpr int QMAX_TERMS = 192;
constexpr int QMAX_GROUPS = 10;
struct QubitProg {
  int n;         // qubits
  int nL, nR, nJ, nJx;  // nJx: multi-qubit diagonal jumps (generic loop)
  int real;      // 1: left/right coefficients purely imaginary, jump ones real
  int ngroups;
  const double2 *dr, *dc;   // device, D each
  const double2 *gtab;      // device, ngroups * 64
};

// One pass of the multi-pass qubit kernel (lrho_q2.cu).
constexpr int MAXPT = 128;  // terms per pass
struct PassTerm {
  uint32_t fl;  // flip mask in tile coordinates (cross-group terms: full mask | kind << 29)
  uint32_t cmask, cval, smask;
  double2 coef;
};
struct PassParams {
  int n, lo;             // qubits, first bit of this pass's six-bit group
  int nL, nR, nJ, nJx;   // general terms
  int diag;              // this pass applies the diagonal (dr, dc, group tables, nJx)
  int last;              // this pass runs the stage epilogue
  int real;
  int ngroups;
  int nspill;            // cross-group terms handled with global loads (last pass)
  int ncanon;            // nonzero: canonical single-bit coefficients below are used
  int herm_tiles;        // last pass only: work items are the blocks I <= J, mirrored
  // first pass of a two-pass Hermitian run: work items are the tile pairs
  // (a, b), a <= b, of the fixed low bits; tile (b, a) is the conjugate
  // transpose of tile (a, b), so one load serves both and the pass writes
  // the running sum of both where the last pass reads it (row >> 6 <= col >> 6)
  int pair_tiles;
  long long ntiles;
  const double2 *dr, *dc, *gtab;
  const double2 *accin;  // running sum from earlier passes (nullptr: start from zero)
  double2 *accout;       // running sum for later passes
  int *errflag;
  // dynamic tile queue of the TMA kernels: CTAs claim work items from
  // *claim; the last CTA to finish (counted in *done) resets both to zero
  unsigned long long *claim;
  unsigned *done;
  // TMA view of the tile (used when tma != 0): dims 1..4 of the 5-D tensor
  // map start at flat index bit tstart[d] with tlen[d] bits; tfree[d] marks
  // the dims the box covers fully (their coordinate is 0)
  int tma;
  int tstart[5], tlen[5], tfree[5];
  // canonical single-bit terms of this group (real mode): left X (i*hl),
  // right X (i*hr), lowering jump (gl, both bits 0), raising jump (gu, both 1)
  double hl[6], hr[6], gl[6], gu[6];
  PassTerm t[MAXPT];
};

// A number no other DeviceProgram of this process carries (caches keyed
// on a program use it rather than the address, which the heap may reuse).
inline uint64_t next_program_serial() {
  static std::atomic<uint64_t> c{0};
  return ++c;
}

struct DeviceProgram {
  uint64_t serial = next_program_serial();
  DevProg dev{};
  HostProg host;
  bool has_qubit = false;
  bool herm_ok = false;            // L(X^H) = (L X)^H for every X (checked on the compiled tables)
  std::vector<PassParams> passes;  // non-empty: multi-pass qubit kernel
  double2 *scratch = nullptr;      // D^2 running sum for the passes
  int *errflag = nullptr;          // device word set by kernels whose waits time out
  unsigned *tile_done = nullptr;   // tile-queue words of the pass kernels (same 16-byte block)
  unsigned long long *tile_claim = nullptr;
  QubitProg qdev{};
  std::vector<QTerm> qterms;  // nL | nR | nJ | nJx in that order
  std::vector<void *> allocations;
  void release();
};

// Builds the device program of a qsystem's time-independent terms.
// mode 0 = density matrix (L on D^2), 1 = Schroedinger (-iH on D),
// 2 = MCWF effective Hamiltonian (-i H_eff on D).
DeviceProgram *compile_terms(qsystem qs, int mode);

// Kernel launchers (lrho.cu, lrho_qubit.cu)
// nbatch > 1: y_z = L x_z for nbatch vectors stored one after another
// (e.kout only; no stage updates or norms)
void launch_lrho(const DevProg &P, const double2 *x, const Epi &e, cudaStream_t s, int nbatch = 1);
void launch_lrho_qubit(const DeviceProgram &P, const double2 *x, const Epi &e, cudaStream_t s);
// Dispatch: the qubit kernel when the program has one, else the generic one.
void launch_lrho_any(const DeviceProgram &P, const double2 *x, const Epi &e, cudaStream_t s);
// y_z = L x_z, z < nbatch, in one launch (vectors stored one after
// another); false (nothing launched) where the program runs a qubit kernel
bool launch_lrho_batch(const DeviceProgram &P, const double2 *x, double2 *y, int nbatch, cudaStream_t s);
bool compile_qubit(qsystem qs, const HostProg &hp, DeviceProgram *P);
bool plan_qubit_passes(const DeviceProgram &P, std::vector<PassParams> &out);
void launch_qubit_passes(std::vector<PassParams> &passes, const double2 *x, double2 *scratch,
                         const Epi &e, cudaStream_t s,
                         bool f32 = false);
// Reads and clears the program's device error word; reports through fail().
bool check_program_error(DeviceProgram &P, cudaStream_t s);
// Loads every kernel that launch_lrho_any may run for this program (both
// contraction precisions) into the current device's context, so that a
// first launch does not load code (lazy module loading allocates device
// memory when a kernel is first used).
void preload_lrho_kernels(const DeviceProgram &P);
void preload_generic_lrho_kernels();
void preload_single_pass_qubit_kernels();
void zero_epi(Epi &e);
// Raises a kernel's dynamic shared-memory limit on the current device to at
// least `bytes` (once per kernel, device and size; thread safe).
void ensure_smem(const void *func, size_t bytes);
// L(X^H) = (L X)^H for all X, decided from the compiled tables (terms.cpp)
bool hermiticity_preserving(const HostProg &hp);
// relative Frobenius asymmetry ||X - X^H|| / ||X|| of a D x D matrix (lincomb.cu)
double hermitian_asymmetry(const double2 *x, int64_t D, cudaStream_t s);
// C[M x N] = act(A[M x K] B[N x K]^T + bias), TF32 tensor cores; K % 32 == 0 (mlp.cu)
void launch_gemm_tf32(const float *A, const float *B, float *C, const float *bias, int M, int N, int K, int act,
                      int *err, cudaStream_t s);
// lincomb.cu
void launch_caxpy(double2 *y, const double2 *x, cplx a, int64_t n, cudaStream_t s);
void launch_epilogue(const double2 *K, const Epi &e, int64_t n, cudaStream_t s);
void launch_lincomb(double2 *out, const double2 *base, int nin, const double2 *const *in,
                    const double *coef, int64_t n, cudaStream_t s);
void launch_lincomb_norm(const double2 *base, const double2 *ref, int nin, const double2 *const *in,
                         const double *coef, int64_t n, double atol, double rtol, double *nsum,
                         cudaStream_t s);
// Dormand-Prince 5(4) tableau (published 1980 coefficients)
extern const double kDP_C[7];
extern const double kDP_A[7][6];
extern const double kDP_E[7];

}  // namespace quac

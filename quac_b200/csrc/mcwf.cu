// Monte-Carlo wavefunction (quantum-jump) trajectories: use_mcwf_solver
// (qsystem.c:358-403) and the jump events of time_step_sys
// (qsystem.c:1139-1235, effective Hamiltonian kron.c:664-700).
//
// Every trajectory is a wavefunction of dimension D evolving under
//   d psi / dt = -i (H - i/2 sum_k a_k C_k^dag C_k) psi
// whose norm decays; when |psi|^2 falls below the trajectory's threshold r
// (uniform in [0, 1)) a jump happens: operator k is chosen with probability
// proportional to a_k |C_k psi|^2, psi becomes sqrt(a_k) C_k psi normalised,
// and a new threshold is drawn.
//
// One persistent launch integrates all trajectories: CTAs take trajectories
// from an atomic queue and keep the state and the stage vectors in shared
// memory, stepping with the integrator of time_step_sys (adaptive
// Bogacki-Shampine 3(2) with the same controller, or fixed BS3 / classical
// RK4).  The crossing time of |psi|^2 = r inside a step is located by
// bisection on the step length to |(|psi|^2 - r)| <= 1e-9 (the event
// tolerance the reference gives PETSc, qsystem.c:1018).  Random numbers come
// from a counter-based SplitMix64 stream (Steele, Lea and Flood, 2014)
// keyed on (seed, trajectory, draw index), so a trajectory's draws do not
// depend on how trajectories are scheduled.
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>

#include "runtime.h"

namespace quac {

struct McwfArgs {
  int D, ntraj, nL, nJ;
  const int *Lmap;       // effective Hamiltonian, generic WF tables (nL x D)
  const double2 *Lval;
  const double2 *dr;
  const int *Jmap;       // jump operators C_k as row maps (nJ x D)
  const double2 *Jval;
  const double2 *Ja;     // a_k
  const double2 *Jsqa;   // sqrt(a_k)
  double2 *psi;          // ntraj x D
  double *thr;           // per-trajectory threshold r
  unsigned long long *cnt;  // per-trajectory draw counter
  unsigned long long seed;
  double t0, tmax, dt, atol, rtol, hmin, hmax;
  int scheme;            // 0 adaptive BS3, 1 fixed BS3, 2 fixed classical RK4
  long long max_steps;
  int *next;             // work queue
  int *err;              // 1: step limit reached, 2: event not located
  long long *stats;      // per trajectory: accepted steps, jumps
};

namespace {

constexpr int MT = 128;
constexpr int MAXJ = 64;  // jump operators per system

__device__ __forceinline__ unsigned long long splitmix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// uniform in [0, 1) for draw k of trajectory i
__device__ __forceinline__ double draw(unsigned long long seed, long long i, unsigned long long k) {
  const unsigned long long h = splitmix64(seed ^ splitmix64(((unsigned long long)i << 32) ^ k));
  return (double)(h >> 11) * 0x1.0p-53;
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}

__device__ double block_sum(double v, double *red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
  for (int w = 0; w < MT / 32; w++) s += red[w];
  return s;
}

// out = -i H_eff x
__device__ void rhs(const McwfArgs &A, const double2 *x, double2 *out) {
  for (int r = threadIdx.x; r < A.D; r += MT) {
    double2 acc = cmul(A.dr[r], x[r]);
    for (int t = 0; t < A.nL; t++) {
      const int j = A.Lmap[(size_t)t * A.D + r];
      if (j >= 0) {
        const double2 v = cmul(A.Lval[(size_t)t * A.D + r], x[j]);
        acc.x += v.x;
        acc.y += v.y;
      }
    }
    out[r] = acc;
  }
  __syncthreads();
}

__device__ double norm2(const McwfArgs &A, const double2 *x, double *red) {
  double s = 0.0;
  for (int r = threadIdx.x; r < A.D; r += MT) s += x[r].x * x[r].x + x[r].y * x[r].y;
  return block_sum(s, red);
}

// One step of length h from y into yn (k1..k4, xs: stage storage).
// Returns the weighted error norm (adaptive BS3) or 0.
__device__ double step(const McwfArgs &A, double h, const double2 *y, double2 *yn, double2 *k1, double2 *k2,
                       double2 *k3, double2 *k4, double2 *xs, double *red) {
  const int D = A.D;
  rhs(A, y, k1);
  if (A.scheme == 2) {
    // classical RK4: the right-hand side does not depend on time
    for (int r = threadIdx.x; r < D; r += MT)
      xs[r] = make_double2(y[r].x + 0.5 * h * k1[r].x, y[r].y + 0.5 * h * k1[r].y);
    __syncthreads();
    rhs(A, xs, k2);
    for (int r = threadIdx.x; r < D; r += MT)
      xs[r] = make_double2(y[r].x + 0.5 * h * k2[r].x, y[r].y + 0.5 * h * k2[r].y);
    __syncthreads();
    rhs(A, xs, k3);
    for (int r = threadIdx.x; r < D; r += MT)
      xs[r] = make_double2(y[r].x + h * k3[r].x, y[r].y + h * k3[r].y);
    __syncthreads();
    rhs(A, xs, k4);
    for (int r = threadIdx.x; r < D; r += MT) {
      const double2 s = make_double2(k1[r].x + 2.0 * k2[r].x + 2.0 * k3[r].x + k4[r].x,
                                     k1[r].y + 2.0 * k2[r].y + 2.0 * k3[r].y + k4[r].y);
      yn[r] = make_double2(y[r].x + h / 6.0 * s.x, y[r].y + h / 6.0 * s.y);
    }
    __syncthreads();
    return 0.0;
  }
  // Bogacki-Shampine 3(2), the tableau of time_step_sys
  for (int r = threadIdx.x; r < D; r += MT)
    xs[r] = make_double2(y[r].x + 0.5 * h * k1[r].x, y[r].y + 0.5 * h * k1[r].y);
  __syncthreads();
  rhs(A, xs, k2);
  for (int r = threadIdx.x; r < D; r += MT)
    xs[r] = make_double2(y[r].x + 0.75 * h * k2[r].x, y[r].y + 0.75 * h * k2[r].y);
  __syncthreads();
  rhs(A, xs, k3);
  for (int r = threadIdx.x; r < D; r += MT) {
    const double cx = 2.0 / 9.0 * k1[r].x + 1.0 / 3.0 * k2[r].x + 4.0 / 9.0 * k3[r].x;
    const double cy = 2.0 / 9.0 * k1[r].y + 1.0 / 3.0 * k2[r].y + 4.0 / 9.0 * k3[r].y;
    yn[r] = make_double2(y[r].x + h * cx, y[r].y + h * cy);
  }
  __syncthreads();
  if (A.scheme != 0) return 0.0;
  rhs(A, yn, k4);
  double s = 0.0;
  for (int r = threadIdx.x; r < D; r += MT) {
    const double ex = h * ((2.0 / 9.0 - 7.0 / 24.0) * k1[r].x + (1.0 / 3.0 - 0.25) * k2[r].x +
                           (4.0 / 9.0 - 1.0 / 3.0) * k3[r].x - 0.125 * k4[r].x);
    const double ey = h * ((2.0 / 9.0 - 7.0 / 24.0) * k1[r].y + (1.0 / 3.0 - 0.25) * k2[r].y +
                           (4.0 / 9.0 - 1.0 / 3.0) * k3[r].y - 0.125 * k4[r].y);
    const double m = fmax(sqrt(y[r].x * y[r].x + y[r].y * y[r].y), sqrt(yn[r].x * yn[r].x + yn[r].y * yn[r].y));
    const double q = sqrt(ex * ex + ey * ey) / (A.atol + A.rtol * m);
    s += q * q;
  }
  return sqrt(block_sum(s, red) / (double)D);
}

__global__ void __launch_bounds__(MT) k_mcwf(const McwfArgs A) {
  extern __shared__ __align__(16) double2 sh[];
  __shared__ double red[MT / 32];
  __shared__ double pj[MAXJ];
  __shared__ int item;
  const int D = A.D;
  double2 *y = sh, *yn = sh + D, *k1 = sh + 2 * D, *k2 = sh + 3 * D, *k3 = sh + 4 * D, *k4 = sh + 5 * D,
          *xs = sh + 6 * D;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) item = atomicAdd(A.next, 1);
    __syncthreads();
    const int i = item;
    if (i >= A.ntraj) break;
    double2 *psi = A.psi + (size_t)i * D;
    for (int r = threadIdx.x; r < D; r += MT) y[r] = psi[r];
    __syncthreads();
    double r_thr = A.thr[i];
    unsigned long long cnt = A.cnt[i];
    double t = A.t0, h = A.dt;
    long long steps = 0, jumps = 0;
    const double tend_tol = 1e-12 * fmax(1.0, fabs(A.tmax));
    bool failed = false;
    while (t < A.tmax - tend_tol) {
      if (steps >= A.max_steps) { failed = true; if (threadIdx.x == 0) atomicExch(A.err, 1); break; }
      double h_try = h;
      bool last = false;
      if (t + h_try >= A.tmax - tend_tol) { h_try = A.tmax - t; last = true; }
      const double err = step(A, h_try, y, yn, k1, k2, k3, k4, xs, red);
      double h_next = h;
      if (A.scheme == 0) {
        double fac = err > 0 ? 0.9 * pow(err, -1.0 / 3.0) : 10.0;
        fac = fmin(10.0, fmax(0.1, fac));
        h_next = fmin(A.hmax, fmax(A.hmin, h_try * fac));
        const bool accepted = (err <= 1.0) || (h_try <= A.hmin * (1 + 1e-12));
        if (!accepted) { h = h_next; continue; }
      }
      const double n1 = norm2(A, yn, red);
      if (n1 < r_thr) {
        // the norm crossed the threshold inside the step: bisect on the
        // step length from (t, y)
        double lo = 0.0, hi = h_try, mid = h_try;
        bool found = false;
        for (int it = 0; it < 200; it++) {
          mid = 0.5 * (lo + hi);
          step(A, mid, y, yn, k1, k2, k3, k4, xs, red);
          const double nm = norm2(A, yn, red);
          if (fabs(nm - r_thr) <= 1e-9) { found = true; break; }
          if (nm < r_thr) hi = mid; else lo = mid;
          if (hi - lo <= 1e-15 * fmax(1.0, fabs(t))) { found = true; break; }
        }
        if (!found) { failed = true; if (threadIdx.x == 0) atomicExch(A.err, 2); break; }
        t += mid;
        // jump probabilities a_k |C_k psi|^2 at the crossing
        double ptot = 0.0;
        for (int k = 0; k < A.nJ; k++) {
          double s = 0.0;
          for (int r = threadIdx.x; r < D; r += MT) {
            const int j = A.Jmap[(size_t)k * D + r];
            if (j >= 0) {
              const double2 v = cmul(A.Jval[(size_t)k * D + r], yn[j]);
              s += v.x * v.x + v.y * v.y;
            }
          }
          const double pk = A.Ja[k].x * block_sum(s, red);  // Re(a_k) |C_k psi|^2
          if (threadIdx.x == 0) pj[k] = pk;
          ptot += pk;
        }
        __syncthreads();
        const double u = draw(A.seed, i, cnt++);
        int kj = -1;
        double pk = 0.0, cum = 0.0;
        for (int k = 0; k < A.nJ; k++) {
          cum += pj[k] / ptot;
          if (cum >= u) { kj = k; pk = pj[k]; break; }
        }
        __syncthreads();
        if (kj >= 0 && pk > 0.0) {
          // psi <- sqrt(a_k) C_k psi / sqrt(a_k |C_k psi|^2)
          const double2 sc = make_double2(A.Jsqa[kj].x / sqrt(pk), A.Jsqa[kj].y / sqrt(pk));
          for (int r = threadIdx.x; r < D; r += MT) {
            const int j = A.Jmap[(size_t)kj * D + r];
            y[r] = j >= 0 ? cmul(sc, cmul(A.Jval[(size_t)kj * D + r], yn[j])) : make_double2(0.0, 0.0);
          }
          jumps++;
        } else {
          // no jump operator acts on this state: keep it, normalised
          const double nn = 1.0 / sqrt(norm2(A, yn, red));
          for (int r = threadIdx.x; r < D; r += MT) y[r] = make_double2(yn[r].x * nn, yn[r].y * nn);
        }
        __syncthreads();
        r_thr = draw(A.seed, i, cnt++);
        continue;  // same step length from the crossing
      }
      for (int r = threadIdx.x; r < D; r += MT) y[r] = yn[r];
      __syncthreads();
      steps++;
      t = last ? A.tmax : t + h_try;
      if (A.scheme == 0) h = h_next;
    }
    (void)failed;
    for (int r = threadIdx.x; r < D; r += MT) psi[r] = y[r];
    if (threadIdx.x == 0) {
      A.thr[i] = r_thr;
      A.cnt[i] = cnt;
      A.stats[2 * (size_t)i] += steps;
      A.stats[2 * (size_t)i + 1] += jumps;
    }
  }
}

// initial thresholds: draw 0 of every trajectory
__global__ void k_mcwf_spawn(const double2 *__restrict__ psi0, double2 *psi, double *thr, unsigned long long *cnt,
                             long long *stats, int D, int ntraj, unsigned long long seed) {
  const long long n = (long long)D * ntraj;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    psi[e] = psi0[e % D];
    if (e < ntraj) {
      thr[e] = draw(seed, e, 0);
      cnt[e] = 1;
      stats[2 * e] = 0;
      stats[2 * e + 1] = 0;
    }
  }
}

// per trajectory: <psi|O|psi> / <psi|psi>, summed into acc (complex) / ntraj
__global__ void __launch_bounds__(MT) k_mcwf_expect(const double2 *__restrict__ psi, int D, int ntraj,
                                                     const int *__restrict__ map, const double2 *__restrict__ val,
                                                     double *acc) {
  __shared__ double red[MT / 32];
  for (int i = blockIdx.x; i < ntraj; i += gridDim.x) {
    const double2 *p = psi + (size_t)i * D;
    double ox = 0.0, oy = 0.0, nn = 0.0;
    for (int r = threadIdx.x; r < D; r += MT) {
      const double2 pr = p[r];
      nn += pr.x * pr.x + pr.y * pr.y;
      const int j = map[r];
      if (j >= 0) {
        const double2 v = cmul(make_double2(pr.x, -pr.y), cmul(val[r], p[j]));
        ox += v.x;
        oy += v.y;
      }
    }
    const double sx = block_sum(ox, red), sy = block_sum(oy, red), sn = block_sum(nn, red);
    if (threadIdx.x == 0) {
      atomicAdd(acc, sx / sn / ntraj);
      atomicAdd(acc + 1, sy / sn / ntraj);
    }
  }
}

struct McwfState {
  int ntraj = 0, D = 0;
  double2 *psi = nullptr;
  double *thr = nullptr;
  unsigned long long *cnt = nullptr;
  long long *stats = nullptr;
  int *words = nullptr;  // queue, error
  double *acc = nullptr;
};

std::mutex g_mu;
std::map<qvec, McwfState> g_states;

struct JumpTables {
  uint64_t serial = 0;
  int nJ = 0;
  int *map = nullptr;
  double2 *val = nullptr, *a = nullptr, *sqa = nullptr;
};
std::map<qsystem, JumpTables> g_jumps;

void free_jumps(JumpTables &J) {
  if (J.map) cudaFree(J.map);
  if (J.val) cudaFree(J.val);
  if (J.a) cudaFree(J.a);
  if (J.sqa) cudaFree(J.sqa);
  J = JumpTables();
}

const JumpTables &jump_tables(qsystem qs) {
  JumpTables &J = g_jumps[qs];
  const uint64_t serial = qs->impl->prog->serial;
  if (J.serial == serial) return J;
  free_jumps(J);
  const int64_t D = qs->total_levels;
  std::vector<int> maps;
  std::vector<double2> vals, as, sqas;
  std::vector<int> map;
  std::vector<cplx> val;
  for (const Term &t : qs->impl->terms) {
    if (t.kind != 2 || t.a == cplx(0.0, 0.0)) continue;
    op_chain_map(D, t.ops, map, val);
    for (int64_t r = 0; r < D; r++) {
      maps.push_back(map[r]);
      vals.push_back(make_double2(val[r].real(), val[r].imag()));
    }
    as.push_back(make_double2(t.a.real(), t.a.imag()));
    const cplx sq = std::sqrt(t.a);  // PetscSqrtComplex(a), qsystem.c:1211
    sqas.push_back(make_double2(sq.real(), sq.imag()));
  }
  J.nJ = (int)as.size();
  if (J.nJ) {
    QCUDA(cudaMalloc(&J.map, maps.size() * sizeof(int)));
    QCUDA(cudaMalloc(&J.val, vals.size() * sizeof(double2)));
    QCUDA(cudaMalloc(&J.a, as.size() * sizeof(double2)));
    QCUDA(cudaMalloc(&J.sqa, sqas.size() * sizeof(double2)));
    QCUDA(cudaMemcpy(J.map, maps.data(), maps.size() * sizeof(int), cudaMemcpyHostToDevice));
    QCUDA(cudaMemcpy(J.val, vals.data(), vals.size() * sizeof(double2), cudaMemcpyHostToDevice));
    QCUDA(cudaMemcpy(J.a, as.data(), as.size() * sizeof(double2), cudaMemcpyHostToDevice));
    QCUDA(cudaMemcpy(J.sqa, sqas.data(), sqas.size() * sizeof(double2), cudaMemcpyHostToDevice));
  }
  J.serial = serial;
  return J;
}

}  // namespace

constexpr int MCWF_MAX_D = 1536;  // seven stage vectors of D complex values in shared memory

bool mcwf_spawned(qvec q) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_states.find(q);
  return it != g_states.end() && it->second.psi != nullptr;
}

void mcwf_release(qvec q) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_states.find(q);
  if (it == g_states.end()) return;
  McwfState &S = it->second;
  for (void *p : {(void *)S.psi, (void *)S.thr, (void *)S.cnt, (void *)S.stats, (void *)S.words, (void *)S.acc})
    if (p) cudaFree(p);
  g_states.erase(it);
}

void mcwf_release_system(qsystem qs) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_jumps.find(qs);
  if (it == g_jumps.end()) return;
  free_jumps(it->second);
  g_jumps.erase(it);
}

// time_step_sys for a system on the MCWF solver (qsystem.c:1025-1086): the
// ensemble is spawned from x's state on the first call and continued on
// later ones
int mcwf_integrate(qsystem qs, qvec x, double t0, double tmax, double dt, int64_t steps_max) {
  if (!x || x->my_type != WF_ENSEMBLE) { fail(0, "ERROR! the MCWF solver integrates a qvec from create_qvec_sys\n"); return 1; }
  if (!qs->impl->td.empty()) { fail(0, "ERROR! time-dependent terms are not supported by the MCWF solver\n"); return 1; }
  ensure_program(qs);
  if (has_error() || !qs->impl->prog) return 1;
  const DeviceProgram &P = *qs->impl->prog;
  const int D = P.dev.D;
  if (D > MCWF_MAX_D) { fail(0, "ERROR! the MCWF solver holds trajectories of at most %d states\n", MCWF_MAX_D); return 1; }
  if (P.dev.ncols != 1 || P.dev.nL < 0) { fail(0, "ERROR! MCWF program has the wrong form\n"); return 1; }
  Options &o = options();
  if (o.max_steps > 0) steps_max = o.max_steps;
  const int ntraj = (int)x->n_ensemble;
  cudaStream_t s = stream_of(qs);
  vec_sync_to_device(x->data);
  McwfState *S;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    S = &g_states[x];
  }
  if (!S->psi) {
    S->ntraj = ntraj;
    S->D = D;
    QCUDA(cudaMalloc(&S->psi, (size_t)ntraj * D * sizeof(double2)));
    QCUDA(cudaMalloc(&S->thr, ntraj * sizeof(double)));
    QCUDA(cudaMalloc(&S->cnt, ntraj * sizeof(unsigned long long)));
    QCUDA(cudaMalloc(&S->stats, 2 * (size_t)ntraj * sizeof(long long)));
    QCUDA(cudaMalloc(&S->words, 2 * sizeof(int)));
    QCUDA(cudaMalloc(&S->acc, 2 * sizeof(double)));
    k_mcwf_spawn<<<256, 256, 0, s>>>(x->data->d, S->psi, S->thr, S->cnt, S->stats, D, ntraj,
                                     (unsigned long long)qs->impl->mcwf_seed);
    count_launch();
    QCUDA(cudaGetLastError());
    x->ens_spawned = PETSC_TRUE;
  }
  const JumpTables &J = jump_tables(qs);
  if (J.nJ > MAXJ) { fail(0, "ERROR! the MCWF solver takes at most %d Lindblad terms\n", MAXJ); return 1; }
  McwfArgs A;
  memset(&A, 0, sizeof(A));
  A.D = D;
  A.ntraj = ntraj;
  A.nL = P.dev.nL;
  A.Lmap = P.dev.Lmap;
  A.Lval = P.dev.Lval;
  A.dr = P.dev.dr;
  A.nJ = J.nJ;
  A.Jmap = J.map;
  A.Jval = J.val;
  A.Ja = J.a;
  A.Jsqa = J.sqa;
  A.psi = S->psi;
  A.thr = S->thr;
  A.cnt = S->cnt;
  A.seed = (unsigned long long)qs->impl->mcwf_seed;
  A.t0 = t0;
  A.tmax = tmax;
  A.dt = dt;
  A.atol = o.atol;
  A.rtol = o.rtol;
  A.hmin = 0.01;
  A.hmax = 1.0;
  const bool fixed = (o.rk_type == "4") || (o.adapt_type == "none");
  A.scheme = o.rk_type == "4" || o.rk_type == "4classic" ? 2 : (fixed ? 1 : 0);
  A.max_steps = steps_max;
  A.next = S->words;
  A.err = S->words + 1;
  A.stats = S->stats;
  QCUDA(cudaMemsetAsync(S->words, 0, 2 * sizeof(int), s));
  const size_t smem = 7 * (size_t)D * sizeof(double2);
  ensure_smem((const void *)k_mcwf, smem);
  int dev = 0, nsm = 0;
  QCUDA(cudaGetDevice(&dev));
  QCUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  int per_sm = 0;
  QCUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mcwf, MT, smem));
  const int grid = std::max(1, std::min(ntraj, nsm * std::max(per_sm, 1)));
  k_mcwf<<<grid, MT, smem, s>>>(A);
  count_launch();
  QCUDA(cudaGetLastError());
  int h[2] = {0, 0};
  QCUDA(cudaMemcpyAsync(h, S->words, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
  QCUDA(cudaStreamSynchronize(s));
  qs->current_time = tmax;
  if (h[1] == 1) { fail(0, "ERROR! Did not reach final time! (step limit in an MCWF trajectory)\n"); return 1; }
  if (h[1] == 2) { fail(0, "ERROR! an MCWF jump time could not be located\n"); return 1; }
  return 0;
}

// ensemble average of <psi|O|psi> / <psi|psi> (qvec_utilities.c:1353-1424)
cplx mcwf_expectation(qvec q, const int *map, const double2 *val) {
  McwfState *S;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    S = &g_states[q];
  }
  cudaStream_t s = nullptr;
  QCUDA(cudaMemsetAsync(S->acc, 0, 2 * sizeof(double), s));
  const int grid = std::min(S->ntraj, 148 * 8);
  k_mcwf_expect<<<grid, MT, 0, s>>>(S->psi, S->D, S->ntraj, map, val, S->acc);
  count_launch();
  QCUDA(cudaGetLastError());
  double h[2];
  QCUDA(cudaMemcpyAsync(h, S->acc, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
  QCUDA(cudaStreamSynchronize(s));
  return cplx(h[0], h[1]);
}

}  // namespace quac

using namespace quac;

// Trajectory states (ntraj x D complex128, row per trajectory) and per
// trajectory counters (accepted steps, jumps) of an MCWF ensemble qvec; no
// reference counterpart (the reference keeps them in qvec->ens_datas).
extern "C" int quac_mcwf_get_states(qvec q, PetscScalar *states_host, int64_t *stats_host) {
  McwfState *S;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_states.find(q);
    if (it == g_states.end() || !it->second.psi) { fail(0, "ERROR! this qvec has no MCWF ensemble yet\n"); return 1; }
    S = &it->second;
  }
  if (states_host)
    QCUDA(cudaMemcpy(states_host, S->psi, (size_t)S->ntraj * S->D * sizeof(double2), cudaMemcpyDeviceToHost));
  if (stats_host)
    QCUDA(cudaMemcpy(stats_host, S->stats, 2 * (size_t)S->ntraj * sizeof(long long), cudaMemcpyDeviceToHost));
  return has_error() ? 1 : 0;
}

// Learned warm start for steady states: a small MLP maps the normalised
// parameters of a system (4 inputs, padded to 32) through two tanh layers of
// `hidden` units to the rank-r factors F (D x r complex) of a proposed
// density matrix rho ~ F F^H.  The proposal seeds the steady-state solver
// (initial state F F^H / tr, deflation space from the leading directions of
// range F).
//
// Training minimises  sum_s || F_s F_s^H - rho_s ||_F^2  over steady states
// rho_s that the solver itself produced.  With E = F F^H - rho (Hermitian),
// d/dF* of ||E||^2 gives the real-pair gradient 4 E F = 4 (F (F^H F) - rho F).
// The three dense layers run forward and backward on the tcgen05 TF32 GEMM
// (operands transposed so both are K-major); the loss, its gradient, the
// activation derivatives, bias reductions and Adam are CUDA-core kernels.
//
// Layout: batch rows are samples; the network output row of sample s holds
// F_s column-major as (re, im) pairs: out[s][2 (j D + r) + {0, 1}].
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "runtime.h"

namespace quac {
namespace {

constexpr int IN_PAD = 32;
constexpr int T = 256;

int blocks_for(long long n) { return (int)std::min<long long>((n + T - 1) / T, 148LL * 16); }

__global__ void k_transpose(const float *__restrict__ in, float *__restrict__ out, int R, int C) {
  __shared__ float tile[32][33];
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int i = threadIdx.y; i < 32; i += 8) {
    const int r = r0 + i, c = c0 + threadIdx.x;
    tile[i][threadIdx.x] = (r < R && c < C) ? in[(size_t)r * C + c] : 0.f;
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += 8) {
    const int c = c0 + i, r = r0 + threadIdx.x;
    if (c < C && r < R) out[(size_t)c * R + r] = tile[threadIdx.x][i];
  }
}

// dZ = dH * (1 - H^2)
__global__ void k_tanh_back(const float *__restrict__ dH, const float *__restrict__ H, float *__restrict__ dZ,
                            long long n) {
  for (long long i = (long long)blockIdx.x * T + threadIdx.x; i < n; i += (long long)gridDim.x * T) {
    const float h = H[i];
    dZ[i] = dH[i] * (1.f - h * h);
  }
}

// db[j] = sum_b dZ[b][j]
__global__ void k_colsum(const float *__restrict__ dZ, float *__restrict__ db, int B, int N) {
  const int j = blockIdx.x * T + threadIdx.x;
  if (j >= N) return;
  float acc = 0.f;
  for (int b = 0; b < B; b++) acc += dZ[(size_t)b * N + j];
  db[j] = acc;
}

__global__ void k_adam(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m, float *__restrict__ v,
                       long long n, float lr, float b1, float b2, float c1, float c2, float eps) {
  for (long long i = (long long)blockIdx.x * T + threadIdx.x; i < n; i += (long long)gridDim.x * T) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

// rows of the batch input from the sample inputs (zero rows past nb)
__global__ void k_gather_inputs(const float *__restrict__ X, const int *__restrict__ idx, int nb, int Bp,
                                float *__restrict__ Xb) {
  const int i = blockIdx.x * T + threadIdx.x;
  if (i >= Bp * IN_PAD) return;
  const int b = i / IN_PAD, k = i % IN_PAD;
  Xb[i] = (b < nb) ? X[(size_t)idx[b] * IN_PAD + k] : 0.f;
}

// S_b = F_b^H F_b  (r x r) for each batch row b < nb; F_b staged in
// shared memory 64 rows at a time, transposed so that a warp's threads
// (consecutive j) read consecutive words
__global__ void k_gram(const float *__restrict__ Fo, int D, int r, int nb, float2 *__restrict__ S) {
  constexpr int KC = 64;
  __shared__ float2 Fs[KC][16];
  const int b = blockIdx.x;
  if (b >= nb) return;
  const float2 *F = reinterpret_cast<const float2 *>(Fo + (size_t)b * 2 * D * r);
  const int q = threadIdx.x, i = q / r, j = q % r;
  const bool mine = q < r * r;
  float ax = 0.f, ay = 0.f;
  for (int k0 = 0; k0 < D; k0 += KC) {
    const int kn = min(KC, D - k0);
    for (int e = threadIdx.x; e < KC * r; e += blockDim.x) {
      const int jj = e / KC, kk = e % KC;
      Fs[kk][jj] = kk < kn ? F[(size_t)jj * D + k0 + kk] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    if (mine)
      for (int kk = 0; kk < kn; kk++) {
        const float2 u = Fs[kk][i], w = Fs[kk][j];
        ax += u.x * w.x + u.y * w.y;  // conj(u) w
        ay += u.x * w.y - u.y * w.x;
      }
    __syncthreads();
  }
  if (mine) S[(size_t)b * r * r + q] = make_float2(ax, ay);
}

// G_b = rho_{idx[b]} F_b  (D x r), rho column-major complex64; one thread per row
__global__ void k_rho_f(const float *__restrict__ Fo, const float2 *__restrict__ rho, const int *__restrict__ idx,
                        int D, int r, int nb, float2 *__restrict__ G) {
  extern __shared__ float2 Fs[];  // D x r
  const int b = blockIdx.y;
  if (b >= nb) return;
  const float2 *F = reinterpret_cast<const float2 *>(Fo + (size_t)b * 2 * D * r);
  for (int q = threadIdx.x; q < D * r; q += blockDim.x) {
    const int j = q / D, c = q % D;
    Fs[c * r + j] = F[(size_t)j * D + c];
  }
  __syncthreads();
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= D) return;
  const float2 *R = rho + (size_t)idx[b] * D * D;
  float ax[16], ay[16];
#pragma unroll
  for (int j = 0; j < 16; j++) { ax[j] = 0.f; ay[j] = 0.f; }
  // eight loads of the column walk in flight before their products
  int c = 0;
  for (; c + 8 <= D; c += 8) {
    float2 xb[8];
#pragma unroll
    for (int u = 0; u < 8; u++) xb[u] = R[(size_t)(c + u) * D + row];
#pragma unroll
    for (int u = 0; u < 8; u++) {
#pragma unroll
      for (int j = 0; j < 16; j++) {
        if (j < r) {
          const float2 f = Fs[(c + u) * r + j];
          ax[j] += xb[u].x * f.x - xb[u].y * f.y;
          ay[j] += xb[u].x * f.y + xb[u].y * f.x;
        }
      }
    }
  }
  for (; c < D; c++) {
    const float2 x = R[(size_t)c * D + row];
#pragma unroll
    for (int j = 0; j < 16; j++) {
      if (j < r) {
        const float2 f = Fs[c * r + j];
        ax[j] += x.x * f.x - x.y * f.y;
        ay[j] += x.x * f.y + x.y * f.x;
      }
    }
  }
#pragma unroll
  for (int j = 0; j < 16; j++)
    if (j < r) G[((size_t)b * r + j) * D + row] = make_float2(ax[j], ay[j]);
}

// dFo_b = (4 / nb) (F_b S_b - G_b); loss += ||S_b||^2 - 2 Re <F_b, G_b> + ||rho||^2 (divided by nb)
__global__ void k_factor_grad(const float *__restrict__ Fo, const float2 *__restrict__ S,
                              const float2 *__restrict__ G, const double *__restrict__ rho_norm2,
                              const int *__restrict__ idx, int D, int r, int nb, float *__restrict__ dFo,
                              double *__restrict__ loss) {
  __shared__ double red[T / 32];
  const int b = blockIdx.y;
  const float2 *F = reinterpret_cast<const float2 *>(Fo + (size_t)b * 2 * D * r);
  float2 *dF = reinterpret_cast<float2 *>(dFo + (size_t)b * 2 * D * r);
  const float2 *Sb = S + (size_t)b * r * r;
  const float2 *Gb = G + (size_t)b * r * D;
  const float scale = 4.f / (float)nb;
  double part = 0.0;
  const int q = blockIdx.x * T + threadIdx.x;  // element (row, j) of F, j-major
  if (q < D * r) {
    const int j = q / D, row = q % D;
    float ax = 0.f, ay = 0.f;
    for (int l = 0; l < r; l++) {
      const float2 f = F[(size_t)l * D + row], s = Sb[l * r + j];
      ax += f.x * s.x - f.y * s.y;
      ay += f.x * s.y + f.y * s.x;
    }
    const float2 g = Gb[(size_t)j * D + row], f = F[(size_t)j * D + row];
    dF[q] = make_float2(scale * (ax - g.x), scale * (ay - g.y));
    part = -2.0 * ((double)f.x * g.x + (double)f.y * g.y);
  }
  if (blockIdx.x == 0 && threadIdx.x < r * r) {
    const float2 s = Sb[threadIdx.x];
    part += (double)s.x * s.x + (double)s.y * s.y;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) part += rho_norm2[idx[b]];
  for (int o = 16; o > 0; o >>= 1) part += __shfl_down_sync(0xffffffffu, part, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = part;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s2 = 0.0;
    for (int w = 0; w < T / 32; w++) s2 += red[w];
    atomicAdd(loss, s2 / (double)nb);
  }
}

// complex128 state -> complex64 target row; returns ||rho||^2 through *norm2
__global__ void k_to_c64(const double2 *__restrict__ x, float2 *__restrict__ y, long long n, double *norm2) {
  __shared__ double red[T / 32];
  double acc = 0.0;
  for (long long i = (long long)blockIdx.x * T + threadIdx.x; i < n; i += (long long)gridDim.x * T) {
    const double2 v = x[i];
    const float2 w = make_float2((float)v.x, (float)v.y);
    y[i] = w;
    acc += (double)w.x * w.x + (double)w.y * w.y;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < T / 32; w++) s += red[w];
    atomicAdd(norm2, s);
  }
}

}  // namespace
}  // namespace quac

using namespace quac;

struct quac_wsnet_s {
  int D = 0, r = 0, H = 0, out = 0, Bp = 0;
  int nmax = 0, n = 0;
  // parameters (row-major [out x in]) and their Adam state
  float *P = nullptr, *Gr = nullptr, *Mo = nullptr, *Vo = nullptr;
  long long np = 0;
  float *W1, *b1, *W2, *b2, *W3, *b3;
  float *gW1, *gb1, *gW2, *gb2, *gW3, *gb3;
  // samples
  float *X = nullptr;        // nmax x IN_PAD
  float2 *rho = nullptr;     // nmax x D^2
  double *rho_n2 = nullptr;  // nmax
  // batch buffers
  float *Xb, *H1, *H2, *Fo, *dFo, *dFoT, *H2T, *W3T, *dH2, *dZ2, *dZ2T, *H1T, *W2T, *dH1, *dZ1, *dZ1T, *XT;
  float2 *S, *G;
  int *idx = nullptr, *err = nullptr;
  double *loss = nullptr;
  std::vector<void *> allocs;
  cudaStream_t s = nullptr;
  long long step = 0;
};

namespace {

template <typename Tp>
Tp *dalloc(quac_wsnet W, size_t n) {
  Tp *p = nullptr;
  QCUDA(cudaMalloc(&p, n * sizeof(Tp)));
  if (p) {
    QCUDA(cudaMemsetAsync(p, 0, n * sizeof(Tp), W->s));
    W->allocs.push_back(p);
  }
  return p;
}

void transpose(quac_wsnet W, const float *in, float *out, int R, int C) {
  dim3 g((C + 31) / 32, (R + 31) / 32), b(32, 8);
  k_transpose<<<g, b, 0, W->s>>>(in, out, R, C);
  count_launch();
}

void gemm(quac_wsnet W, const float *A, const float *B, float *C, const float *bias, int M, int N, int K, int act) {
  launch_gemm_tf32(A, B, C, bias, M, N, K, act, W->err, W->s);
}

void forward(quac_wsnet W) {
  gemm(W, W->Xb, W->W1, W->H1, W->b1, W->Bp, W->H, IN_PAD, 1);
  gemm(W, W->H1, W->W2, W->H2, W->b2, W->Bp, W->H, W->H, 1);
  gemm(W, W->H2, W->W3, W->Fo, W->b3, W->Bp, W->out, W->H, 0);
}

// loss and parameter gradients of the batch (rows idx[0..nb)); *loss += mean loss
void loss_and_grads(quac_wsnet W, int nb) {
  const int D = W->D, r = W->r;
  QCUDA(cudaMemsetAsync(W->dFo, 0, (size_t)W->Bp * W->out * sizeof(float), W->s));
  k_gram<<<nb, T, 0, W->s>>>(W->Fo, D, r, nb, W->S);
  const size_t sm = (size_t)D * r * sizeof(float2);
  k_rho_f<<<dim3((D + 127) / 128, nb), 128, sm, W->s>>>(W->Fo, W->rho, W->idx, D, r, nb, W->G);
  k_factor_grad<<<dim3((D * r + T - 1) / T, nb), T, 0, W->s>>>(W->Fo, W->S, W->G, W->rho_n2, W->idx, D, r, nb,
                                                               W->dFo, W->loss);
  count_launch(3);
  QCUDA(cudaGetLastError());
  const int Bp = W->Bp, H = W->H, O = W->out;
  // layer 3
  transpose(W, W->dFo, W->dFoT, Bp, O);
  transpose(W, W->H2, W->H2T, Bp, H);
  gemm(W, W->dFoT, W->H2T, W->gW3, nullptr, O, H, Bp, 0);
  k_colsum<<<(O + T - 1) / T, T, 0, W->s>>>(W->dFo, W->gb3, Bp, O);
  transpose(W, W->W3, W->W3T, O, H);
  gemm(W, W->dFo, W->W3T, W->dH2, nullptr, Bp, H, O, 0);
  // layer 2
  k_tanh_back<<<blocks_for((long long)Bp * H), T, 0, W->s>>>(W->dH2, W->H2, W->dZ2, (long long)Bp * H);
  transpose(W, W->dZ2, W->dZ2T, Bp, H);
  transpose(W, W->H1, W->H1T, Bp, H);
  gemm(W, W->dZ2T, W->H1T, W->gW2, nullptr, H, H, Bp, 0);
  k_colsum<<<(H + T - 1) / T, T, 0, W->s>>>(W->dZ2, W->gb2, Bp, H);
  transpose(W, W->W2, W->W2T, H, H);
  gemm(W, W->dZ2, W->W2T, W->dH1, nullptr, Bp, H, H, 0);
  // layer 1
  k_tanh_back<<<blocks_for((long long)Bp * H), T, 0, W->s>>>(W->dH1, W->H1, W->dZ1, (long long)Bp * H);
  transpose(W, W->dZ1, W->dZ1T, Bp, H);
  transpose(W, W->Xb, W->XT, Bp, IN_PAD);
  gemm(W, W->dZ1T, W->XT, W->gW1, nullptr, H, IN_PAD, Bp, 0);
  k_colsum<<<(H + T - 1) / T, T, 0, W->s>>>(W->dZ1, W->gb1, Bp, H);
  count_launch(5);
  QCUDA(cudaGetLastError());
}

void set_batch(quac_wsnet W, const int *idx_host, int nb) {
  QCUDA(cudaMemcpyAsync(W->idx, idx_host, nb * sizeof(int), cudaMemcpyHostToDevice, W->s));
  k_gather_inputs<<<(W->Bp * IN_PAD + T - 1) / T, T, 0, W->s>>>(W->X, W->idx, nb, W->Bp, W->Xb);
  count_launch();
}

bool check_err(quac_wsnet W) {
  int h = 0;
  QCUDA(cudaMemcpyAsync(&h, W->err, sizeof(int), cudaMemcpyDeviceToHost, W->s));
  QCUDA(cudaStreamSynchronize(W->s));
  if (h) fail(9, "ERROR! warm-start network: a tensor-core wait ran out of time\n");
  return !has_error();
}

}  // namespace

extern "C" {

int quac_wsnet_create(quac_wsnet *out, int D, int rank, int hidden, int batch, int max_samples, uint64_t seed) {
  *out = nullptr;
  if (D < 2 || rank < 1 || rank > 16 || hidden < 32 || hidden % 32 || batch < 1 || max_samples < 1 ||
      (2LL * D * rank) % 32) {
    fail(0, "ERROR! quac_wsnet_create: invalid sizes (rank <= 16, hidden % 32 == 0, 2 D rank % 32 == 0)\n");
    return 1;
  }
  quac_wsnet W = new quac_wsnet_s();
  W->D = D;
  W->r = rank;
  W->H = hidden;
  W->out = 2 * D * rank;
  W->Bp = (batch + 31) / 32 * 32;
  W->nmax = max_samples;
  QCUDA(cudaStreamCreateWithFlags(&W->s, cudaStreamNonBlocking));
  const long long n1 = (long long)hidden * IN_PAD, n2 = (long long)hidden * hidden, n3 = (long long)W->out * hidden;
  W->np = n1 + hidden + n2 + hidden + n3 + W->out;
  W->P = dalloc<float>(W, W->np);
  W->Gr = dalloc<float>(W, W->np);
  W->Mo = dalloc<float>(W, W->np);
  W->Vo = dalloc<float>(W, W->np);
  if (has_error()) { quac_wsnet_destroy(W); return 1; }
  float *p = W->P, *g = W->Gr;
  W->W1 = p; W->gW1 = g; p += n1; g += n1;
  W->b1 = p; W->gb1 = g; p += hidden; g += hidden;
  W->W2 = p; W->gW2 = g; p += n2; g += n2;
  W->b2 = p; W->gb2 = g; p += hidden; g += hidden;
  W->W3 = p; W->gW3 = g; p += n3; g += n3;
  W->b3 = p; W->gb3 = g;
  // Glorot-uniform weights (inputs: the 4 real features), zero biases
  std::vector<float> h(W->np, 0.f);
  std::mt19937_64 rng(seed);
  auto fill = [&](long long off, int rows, int cols, int fan_in) {
    const float a = std::sqrt(6.f / (float)(fan_in + rows));
    std::uniform_real_distribution<float> U(-a, a);
    for (int i = 0; i < rows; i++)
      for (int j = 0; j < cols; j++) h[off + (long long)i * cols + j] = (j < fan_in) ? U(rng) : 0.f;
  };
  fill(0, hidden, IN_PAD, 4);
  fill(n1 + hidden, hidden, hidden, hidden);
  fill(n1 + hidden + n2 + hidden, W->out, hidden, hidden);
  QCUDA(cudaMemcpyAsync(W->P, h.data(), W->np * sizeof(float), cudaMemcpyHostToDevice, W->s));
  const int Bp = W->Bp, O = W->out, H = hidden;
  W->X = dalloc<float>(W, (size_t)max_samples * IN_PAD);
  W->rho = dalloc<float2>(W, (size_t)max_samples * D * D);
  W->rho_n2 = dalloc<double>(W, max_samples);
  W->Xb = dalloc<float>(W, (size_t)Bp * IN_PAD);
  W->XT = dalloc<float>(W, (size_t)Bp * IN_PAD);
  W->H1 = dalloc<float>(W, (size_t)Bp * H);
  W->H2 = dalloc<float>(W, (size_t)Bp * H);
  W->H1T = dalloc<float>(W, (size_t)Bp * H);
  W->H2T = dalloc<float>(W, (size_t)Bp * H);
  W->dH1 = dalloc<float>(W, (size_t)Bp * H);
  W->dH2 = dalloc<float>(W, (size_t)Bp * H);
  W->dZ1 = dalloc<float>(W, (size_t)Bp * H);
  W->dZ2 = dalloc<float>(W, (size_t)Bp * H);
  W->dZ1T = dalloc<float>(W, (size_t)Bp * H);
  W->dZ2T = dalloc<float>(W, (size_t)Bp * H);
  W->W2T = dalloc<float>(W, (size_t)H * H);
  W->W3T = dalloc<float>(W, (size_t)O * H);
  W->Fo = dalloc<float>(W, (size_t)Bp * O);
  W->dFo = dalloc<float>(W, (size_t)Bp * O);
  W->dFoT = dalloc<float>(W, (size_t)Bp * O);
  W->S = dalloc<float2>(W, (size_t)Bp * rank * rank);
  W->G = dalloc<float2>(W, (size_t)Bp * rank * D);
  W->idx = dalloc<int>(W, Bp);
  W->err = dalloc<int>(W, 1);
  W->loss = dalloc<double>(W, 1);
  QCUDA(cudaFuncSetAttribute(k_rho_f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)((size_t)D * rank * sizeof(float2))));
  QCUDA(cudaStreamSynchronize(W->s));
  if (has_error()) { quac_wsnet_destroy(W); return 1; }
  *out = W;
  return 0;
}

int quac_wsnet_destroy(quac_wsnet W) {
  if (!W) return 0;
  for (void *p : W->allocs) cudaFree(p);
  if (W->s) cudaStreamDestroy(W->s);
  delete W;
  return 0;
}

// Adds one training sample: 4 normalised inputs and a density matrix held by a qvec.
int quac_wsnet_add_sample(quac_wsnet W, const double *theta, qvec rho) {
  if (W->n >= W->nmax) { fail(0, "ERROR! warm-start network: sample capacity reached\n"); return 1; }
  if (rho->n != (PetscInt)W->D * W->D) { fail(0, "ERROR! warm-start network: sample dimension mismatch\n"); return 1; }
  vec_sync_to_device(rho->data);
  float xin[IN_PAD] = {0};
  for (int k = 0; k < 4; k++) xin[k] = (float)theta[k];
  QCUDA(cudaMemcpyAsync(W->X + (size_t)W->n * IN_PAD, xin, sizeof(xin), cudaMemcpyHostToDevice, W->s));
  const long long n2 = (long long)W->D * W->D;
  k_to_c64<<<blocks_for(n2), T, 0, W->s>>>(rho->data->d, W->rho + (size_t)W->n * n2, n2, W->rho_n2 + W->n);
  count_launch();
  QCUDA(cudaStreamSynchronize(W->s));
  if (has_error()) return 1;
  W->n++;
  return 0;
}

int quac_wsnet_num_samples(quac_wsnet W) { return W->n; }

int64_t quac_wsnet_num_params(quac_wsnet W) { return W->np; }

int quac_wsnet_get_params(quac_wsnet W, float *out) {
  QCUDA(cudaMemcpyAsync(out, W->P, W->np * sizeof(float), cudaMemcpyDeviceToHost, W->s));
  QCUDA(cudaStreamSynchronize(W->s));
  return has_error() ? 1 : 0;
}

int quac_wsnet_set_params(quac_wsnet W, const float *in) {
  QCUDA(cudaMemcpyAsync(W->P, in, W->np * sizeof(float), cudaMemcpyHostToDevice, W->s));
  QCUDA(cudaStreamSynchronize(W->s));
  return has_error() ? 1 : 0;
}

// Loss and gradient (flat, parameter order) over samples [0, nb) without updating.
int quac_wsnet_loss_grad(quac_wsnet W, int nb, double *loss, float *grad) {
  if (nb < 1 || nb > W->Bp || nb > W->n) { fail(0, "ERROR! warm-start network: bad batch\n"); return 1; }
  std::vector<int> idx(nb);
  for (int i = 0; i < nb; i++) idx[i] = i;
  set_batch(W, idx.data(), nb);
  QCUDA(cudaMemsetAsync(W->loss, 0, sizeof(double), W->s));
  forward(W);
  loss_and_grads(W, nb);
  QCUDA(cudaMemcpyAsync(loss, W->loss, sizeof(double), cudaMemcpyDeviceToHost, W->s));
  if (grad) QCUDA(cudaMemcpyAsync(grad, W->Gr, W->np * sizeof(float), cudaMemcpyDeviceToHost, W->s));
  return check_err(W) ? 0 : 1;
}

// Adam over shuffled mini-batches; *final_loss = mean loss of the last epoch.
int quac_wsnet_train(quac_wsnet W, int epochs, double lr, uint64_t seed, double *final_loss) {
  if (W->n < 1 || epochs < 1) { fail(0, "ERROR! warm-start network: nothing to train\n"); return 1; }
  std::mt19937_64 rng(seed);
  std::vector<int> perm(W->n);
  for (int i = 0; i < W->n; i++) perm[i] = i;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  double last = 0.0;
  for (int ep = 0; ep < epochs; ep++) {
    std::shuffle(perm.begin(), perm.end(), rng);
    QCUDA(cudaMemsetAsync(W->loss, 0, sizeof(double), W->s));
    int nbatches = 0;
    // cosine decay of the learning rate
    const float lr_ep = (float)(lr * 0.5 * (1.0 + std::cos(3.141592653589793 * ep / (double)epochs)));
    for (int b0 = 0; b0 < W->n; b0 += W->Bp) {
      const int nb = std::min(W->Bp, W->n - b0);
      set_batch(W, perm.data() + b0, nb);
      forward(W);
      loss_and_grads(W, nb);
      W->step++;
      const float c1 = 1.f - std::pow(b1, (float)W->step), c2 = 1.f - std::pow(b2, (float)W->step);
      k_adam<<<blocks_for(W->np), T, 0, W->s>>>(W->P, W->Gr, W->Mo, W->Vo, W->np, lr_ep, b1, b2, c1, c2, eps);
      count_launch();
      nbatches++;
    }
    if (ep == epochs - 1) {
      QCUDA(cudaMemcpyAsync(&last, W->loss, sizeof(double), cudaMemcpyDeviceToHost, W->s));
      QCUDA(cudaStreamSynchronize(W->s));
      last /= nbatches;
    }
    if (has_error()) return 1;
  }
  if (final_loss) *final_loss = last;
  return check_err(W) ? 0 : 1;
}

// Factors F (D x rank complex, column-major) proposed for each of n inputs.
int quac_wsnet_predict(quac_wsnet W, int n, const double *theta, PetscScalar *F) {
  const size_t per = (size_t)W->D * W->r;
  std::vector<float> xin((size_t)W->Bp * IN_PAD), out((size_t)W->Bp * W->out);
  for (int b0 = 0; b0 < n; b0 += W->Bp) {
    const int nb = std::min(W->Bp, n - b0);
    std::fill(xin.begin(), xin.end(), 0.f);
    for (int b = 0; b < nb; b++)
      for (int k = 0; k < 4; k++) xin[(size_t)b * IN_PAD + k] = (float)theta[(size_t)(b0 + b) * 4 + k];
    QCUDA(cudaMemcpyAsync(W->Xb, xin.data(), xin.size() * sizeof(float), cudaMemcpyHostToDevice, W->s));
    forward(W);
    QCUDA(cudaMemcpyAsync(out.data(), W->Fo, out.size() * sizeof(float), cudaMemcpyDeviceToHost, W->s));
    if (!check_err(W)) return 1;
    for (int b = 0; b < nb; b++)
      for (size_t k = 0; k < per; k++)
        F[(size_t)(b0 + b) * per + k] =
            PetscScalar(out[(size_t)b * W->out + 2 * k], out[(size_t)b * W->out + 2 * k + 1]);
  }
  return 0;
}

}  // extern "C"

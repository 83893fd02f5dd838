// Dense layers of the steady-state warm-start network on the 5th-generation
// tensor cores (tcgen05, TF32 inputs, FP32 accumulation in tensor memory).
//
//   C[M x N] = act(A[M x K] . B[N x K]^T + bias[N])     (both operands K-major)
//
// One CTA of 128 threads computes a 128 x 128 output tile.  A and B tiles of
// 32 K-columns are copied by cp.async (16 bytes per request, zero-filled past
// the matrix edge) straight into the canonical no-swizzle K-major layout
// (8-row x 16-byte core matrices: the two 16-byte K chunks of one MMA are
// LBO apart, consecutive 8-row groups SBO apart), NST stages deep; one
// elected thread issues four tcgen05.mma (K = 8 each) per stage and commits
// them to that stage's mbarrier, which frees the stage for the copy NST - 1
// steps ahead.
// The accumulator (128 lanes x 128 columns of FP32) is read back with
// tcgen05.ld; bias and activation are fused into that epilogue.
//
// Every mbarrier wait is bounded in time; a wait that runs out sets the
// error word, the CTA stops issuing work, frees its tensor memory and returns.
#include <cstdint>

#include "runtime.h"

namespace quac {
namespace {

constexpr int BM = 128, BN = 128, BK = 32;
constexpr int TILE_BYTES = BM * BK * 4;  // 16 KB per operand per stage
constexpr int NST = 3;                   // pipeline stages (96 KB: two CTAs per SM)
constexpr unsigned long long WAIT_NS = 2000000000ull;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait; false (and *err set) if the phase did not complete in time.
__device__ bool mbar_wait(uint32_t bar, uint32_t parity, int *err) {
  if (mbar_try(bar, parity)) return true;
  const unsigned long long t0 = gtimer();
  while (!mbar_try(bar, parity)) {
    if (gtimer() - t0 > WAIT_NS) {
      atomicExch(err, 1);
      return false;
    }
  }
  return true;
}

// Shared-memory matrix descriptor: no swizzle, K-major canonical layout.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version of sm_100
  return d;               // base offset 0, legacy LBO mode, layout type 0 (no swizzle)
}

// Instruction descriptor: kind::tf32, FP32 accumulator, A and B K-major.
__host__ __device__ constexpr uint32_t instr_desc_tf32(int m, int n) {
  return (1u << 4)                   // accumulator format F32
         | (2u << 7)                 // A format TF32
         | (2u << 10)                // B format TF32
         | ((uint32_t)(n >> 3) << 17)
         | ((uint32_t)(m >> 4) << 24);
}

// byte offset of element (row, k) of a 128 x 32 tile in the canonical layout
__device__ __forceinline__ uint32_t tile_off(int row, int k) {
  return (uint32_t)((k >> 2) * (BM * 16) + (row >> 3) * 128 + (row & 7) * 16 + (k & 3) * 4);
}

// rows [r0, r0 + 128) x k [k0, k0 + 32) of a row-major R x K matrix -> tile,
// asynchronously (zero past R)
__device__ __forceinline__ void load_tile(unsigned char *tile, const float *__restrict__ src, int R, int K, int r0,
                                          int k0) {
  // 128 rows x 8 chunks of 4 floats = 1024 chunks, 8 per thread
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const int q = threadIdx.x + i * 128;
    const int row = q >> 3, chunk = q & 7;
    const bool in = r0 + row < R;
    const float *g = in ? src + (size_t)(r0 + row) * K + k0 + chunk * 4 : src;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(tile + tile_off(row, chunk * 4))),
                 "l"(g), "r"(in ? 16 : 0)
                 : "memory");
  }
}

__global__ void __launch_bounds__(128) k_gemm_tf32(const float *__restrict__ A, const float *__restrict__ B,
                                                   float *__restrict__ C, const float *__restrict__ bias, int M,
                                                   int N, int K, int act, int *err) {
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ __align__(8) uint64_t bars[NST];
  __shared__ uint32_t tmem_slot;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  auto As = [&](int st) { return sm + st * 2 * TILE_BYTES; };
  auto Bs = [&](int st) { return sm + st * 2 * TILE_BYTES + TILE_BYTES; };

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"(BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (threadIdx.x == 0) {
    for (int st = 0; st < NST; st++)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bars[st])));
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = tmem_slot;
  const uint32_t idesc = instr_desc_tf32(BM, BN);
  const int nk = K / BK;
  bool ok = true;

  // prologue: stages 0 .. NST-2 in flight (one commit group each, empty past nk)
  for (int st = 0; st < NST - 1; st++) {
    if (st < nk) {
      load_tile(As(st), A, M, K, m0, st * BK);
      load_tile(Bs(st), B, N, K, n0, st * BK);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  }
  for (int kb = 0; kb < nk; kb++) {
    const int st = kb % NST;
    // stage kb has landed (at most NST-2 younger groups pending)
    asm volatile("cp.async.wait_group %0;\n" ::"n"(NST - 2) : "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (threadIdx.x == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
      for (int k8 = 0; k8 < BK / 8; k8++) {
        const uint64_t ad = smem_desc(smem_u32(As(st)) + k8 * 2 * (BM * 16), BM * 16, 128);
        const uint64_t bd = smem_desc(smem_u32(Bs(st)) + k8 * 2 * (BN * 16), BN * 16, 128);
        const uint32_t acc = (kb > 0 || k8 > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
            "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(&bars[st])));
    }
    // refill the stage used by step kb-1 with step kb+NST-1, once its MMAs are done
    const int kn = kb + NST - 1;
    if (kn < nk) {
      if (kb >= 1) ok = mbar_wait(smem_u32(&bars[(kb - 1) % NST]), ((kb - 1) / NST) & 1, err);
      ok = __syncthreads_and(ok);
      if (!ok) break;
      load_tile(As(kn % NST), A, M, K, m0, kn * BK);
      load_tile(Bs(kn % NST), B, N, K, n0, kn * BK);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  // the last commit covers every MMA issued before it
  if (ok && nk >= 1) ok = mbar_wait(smem_u32(&bars[(nk - 1) % NST]), ((nk - 1) / NST) & 1, err);
  ok = __syncthreads_and(ok);
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (ok) {
    // epilogue: warp w owns accumulator lanes (rows) 32w .. 32w + 31
    const int row = m0 + warp * 32 + lane;
    for (int c0 = 0; c0 < BN; c0 += 16) {
      uint32_t v[16];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
      // load and wait in one statement: the destination registers are
      // written asynchronously and must not be read before the wait
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n\t"
          "tcgen05.wait::ld.sync.aligned;"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
          : "r"(taddr)
          : "memory");
      if (row < M) {
#pragma unroll
        for (int j = 0; j < 16; j++) {
          const int col = n0 + c0 + j;
          if (col < N) {
            float x = __uint_as_float(v[j]);
            if (bias) x += bias[col];
            if (act == 1) x = tanhf(x);
            C[(size_t)row * N + col] = x;
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN));
}

}  // namespace

// C = act(A B^T + bias) on device buffers; K must be a multiple of 32.
void launch_gemm_tf32(const float *A, const float *B, float *C, const float *bias, int M, int N, int K, int act,
                      int *err, cudaStream_t s) {
  const int smem = NST * 2 * TILE_BYTES;
  ensure_smem((const void *)k_gemm_tf32, smem);
  dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM);
  k_gemm_tf32<<<grid, 128, smem, s>>>(A, B, C, bias, M, N, K, act, err);
  count_launch();
  QCUDA(cudaGetLastError());
}

}  // namespace quac

using namespace quac;

// Device-pointer GEMM for tests: returns 0, or 1 on invalid sizes or a
// timed-out wait inside the kernel.
extern "C" int quac_gemm_tf32(const float *A, const float *B, float *C, const float *bias, int M, int N, int K,
                              int act) {
  if (M <= 0 || N <= 0 || K <= 0 || K % 32 != 0 || (act != 0 && act != 1)) {
    fail(0, "ERROR! quac_gemm_tf32: invalid sizes (K must be a positive multiple of 32)\n");
    return 1;
  }
  int *err = nullptr;
  QCUDA(cudaMalloc(&err, sizeof(int)));
  QCUDA(cudaMemset(err, 0, sizeof(int)));
  launch_gemm_tf32(A, B, C, bias, M, N, K, act, err, 0);
  int h = 0;
  QCUDA(cudaMemcpy(&h, err, sizeof(int), cudaMemcpyDeviceToHost));
  QCUDA(cudaFree(err));
  if (h) fail(9, "ERROR! quac_gemm_tf32: a tensor-core wait ran out of time\n");
  return has_error() ? 1 : 0;
}

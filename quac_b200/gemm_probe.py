"""Runs the tensor-core dense-layer GEMM a few times (for profiling runs).

    python -m quac_b200.gemm_probe --m 2048 --n 16384 --k 256 --reps 3

C = A B^T (+ bias) with TF32 operands: the shape of the warm-start network's
output layer for a batch of m parameter points.
"""
import argparse
import ctypes

import torch

import quac_b200 as q


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--m", type=int, default=2048)
    ap.add_argument("--n", type=int, default=16384)
    ap.add_argument("--k", type=int, default=256)
    ap.add_argument("--reps", type=int, default=3)
    a = ap.parse_args()
    L = q.lib()
    L.quac_gemm_tf32.restype = ctypes.c_int
    L.quac_gemm_tf32.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_int] * 4
    A = torch.randn(a.m, a.k, device="cuda")
    B = torch.randn(a.n, a.k, device="cuda")
    bias = torch.randn(a.n, device="cuda")
    C = torch.empty(a.m, a.n, device="cuda")
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for i in range(a.reps):
        if i == a.reps - 1:
            ev0.record()
        rc = L.quac_gemm_tf32(A.data_ptr(), B.data_ptr(), C.data_ptr(), bias.data_ptr(), a.m, a.n, a.k, 0)
        assert rc == 0
    ev1.record()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    print(f"ok {a.m}x{a.n}x{a.k}: {ms * 1e3:.1f} us per GEMM (incl. error read-back), "
          f"{2.0 * a.m * a.n * a.k / ms / 1e9:.1f} TFLOP/s")


if __name__ == "__main__":
    main()

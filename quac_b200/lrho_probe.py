"""Applies L.rho a few times on the device (for profiling runs).

    python -m quac_b200.lrho_probe --qubits 12 --reps 3 [--path 0|1|2] [--fp32] [--rk4-steps N]

With --rk4-steps N the probe instead integrates a random Hermitian state for
N fixed RK4 steps (dt = 0.01) through time_step_sys, which runs the
Hermitian mode of the multi-pass kernel for 12 qubits.

Builds the open transverse-field Ising chain of the benchmark with the
given number of qubits, allocates x and y with torch on cuda:0 and calls
quac_lrho_apply_device `reps` times.
"""
import argparse

import torch

import quac_b200 as q
from quac_b200.systems import Builder, tfim


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--qubits", type=int, default=12)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--path", type=int, default=0)
    ap.add_argument("--fp32", action="store_true", help="complex64 contraction")
    ap.add_argument("--rk4-steps", type=int, default=0)
    a = ap.parse_args()
    q.lib()
    q.QuaC_initialize()
    q.set_kernel_path(a.path)
    q.set_lrho_precision(1 if a.fp32 else 0)
    S = Builder(q)
    tfim(S, a.qubits)
    q.construct_matrix(S.qs)
    n = S.D * S.D
    if a.rk4_steps > 0:
        X = torch.randn(S.D, S.D, dtype=torch.complex128)
        X = (X + X.conj().T) / 2
        rho = q.create_dm_sys(S.qs)
        rho.from_numpy(X.T.contiguous().reshape(-1).numpy())  # column-stacked
        q.set_ts_options(rk_type="4", adapt_type="none")
        q.time_step_sys(S.qs, rho, 0.0, 0.01 * a.rk4_steps, 0.01, 10 ** 6)
        torch.cuda.synchronize()
        print(f"ok D={S.D} rk4 steps={a.rk4_steps} hermitian applications={q.hermitian_apply_count()}")
        return
    x = torch.randn(n, dtype=torch.complex128, device="cuda")
    y = torch.empty_like(x)
    for _ in range(a.reps):
        q.lrho_apply_device(S.qs, x.data_ptr(), y.data_ptr())
    torch.cuda.synchronize()
    print(f"ok D={S.D} reps={a.reps} launches={q.kernel_launch_count()}")


if __name__ == "__main__":
    main()

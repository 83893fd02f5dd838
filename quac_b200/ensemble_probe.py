"""Runs the batched ensemble kernel once (for profiling runs).

    python -m quac_b200.ensemble_probe --instances 512 --t 2 [--fp32]

Driven Jaynes-Cummings instances of the ensemble workload (n_c ~ U{5..40}),
each integrated from |e,0><e,0| to t with its own Dormand-Prince 5(4) step.
"""
import argparse
import time

import numpy as np

import quac_b200 as q
from quac_b200 import systems as Sy


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--instances", type=int, default=512)
    ap.add_argument("--t", type=float, default=2.0)
    ap.add_argument("--fp32", action="store_true")
    a = ap.parse_args()
    q.lib()
    q.QuaC_initialize()
    params = Sy.driven_jc_ensemble_params(a.instances)
    built = []
    for p in params:
        B = Sy.Builder(q)
        Sy.driven_jc(B, **p)
        built.append(B.qs)
    E = q.Ensemble(built)
    E.set_options(precision=1 if a.fp32 else 0)
    E.set_states(np.concatenate([Sy.excited_vacuum(p["nc"]) for p in params]))
    t0 = time.perf_counter()
    E.run(0.0, a.t, 0.05)
    print(f"ok {a.instances} instances to t={a.t} in {(time.perf_counter() - t0) * 1e3:.1f} ms")
    E.destroy()


if __name__ == "__main__":
    main()

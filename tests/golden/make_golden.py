"""Convert the reference's PETSc-binary test fixtures into one compact .npz.

Run once in a container where the reference tree is mounted:

    python tests/golden/make_golden.py <reference checkout>/tests/pristine_matrices

It writes tests/golden/pristine.npz.  The fixtures are the golden
superoperator matrices and state vectors used by the reference's
matrix_construction_test_*.c and qvec_utilities_tests.c.  PETSc binary
format (big endian): Mat = int64 classid 1211216, M, N, nz, rowlens[M],
cols[nz], complex128 vals[nz]; Vec = int64 classid 1211214, n,
complex128[n].
"""
import os
import sys

import numpy as np

MAT_ID = 1211216
VEC_ID = 1211214


def read_petsc(path):
    raw = open(path, "rb").read()
    head = np.frombuffer(raw[:8], dtype=">i8")[0]
    if head == MAT_ID:
        m, n, nz = np.frombuffer(raw[8:32], dtype=">i8")
        off = 32
        rowlens = np.frombuffer(raw[off:off + 8 * m], dtype=">i8").astype(np.int64)
        off += 8 * m
        cols = np.frombuffer(raw[off:off + 8 * nz], dtype=">i8").astype(np.int64)
        off += 8 * nz
        vals = np.frombuffer(raw[off:off + 16 * nz], dtype=">c16").astype(np.complex128)
        rowptr = np.concatenate([[0], np.cumsum(rowlens)]).astype(np.int64)
        return "mat", dict(shape=np.array([m, n]), rowptr=rowptr, col=cols, val=vals)
    if head == VEC_ID:
        n = np.frombuffer(raw[8:16], dtype=">i8")[0]
        vals = np.frombuffer(raw[16:16 + 16 * n], dtype=">c16").astype(np.complex128)
        return "vec", dict(val=vals)
    raise ValueError(f"{path}: unknown PETSc class id {head}")


def main(src):
    out = {}
    for name in sorted(os.listdir(src)):
        kind, d = read_petsc(os.path.join(src, name))
        key = name.replace(".", "_")
        for k, v in d.items():
            out[f"{key}__{k}"] = v
        out[f"{key}__kind"] = np.array(kind)
        if kind == "vec":
            # the file's own bytes, for reading through the library's PETSc-binary reader
            out[f"{key}__raw"] = np.frombuffer(open(os.path.join(src, name), "rb").read(), dtype=np.uint8)
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "pristine.npz")
    np.savez_compressed(dst, **out)
    print(f"wrote {dst} ({len(out)} arrays)")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <reference>/tests/pristine_matrices")
    main(sys.argv[1])

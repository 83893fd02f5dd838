"""The allocation-free L.x entry point against quac_lrho_apply_device.

Some callers cannot allocate device memory while they run: a framework
whose memory pool already owns the GPU's memory, or a control loop that
cannot afford the device-wide synchronisation of cudaFree.  For them
quac_lrho_apply_device_noalloc keeps the multi-pass kernel's running sum in
a fixed device array; quac_lrho_noalloc_setup (called once, before the
loop) is the only call that may allocate.

Collected last (file name) so that it also runs after every other test in
the same process, when the device already holds other systems' buffers.
Both entry points launch the same kernels on the same inputs, so the
results must be bit-identical; device free memory must not change across
the allocation-free calls, including the first one in a fresh process.
"""
import ctypes
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bind(q):
    L = q.lib()
    P = ctypes.POINTER(q._QsysStruct)
    L.quac_lrho_noalloc_setup.restype = ctypes.c_int
    L.quac_lrho_noalloc_setup.argtypes = [P]
    L.quac_lrho_apply_device_noalloc.restype = ctypes.c_int
    L.quac_lrho_apply_device_noalloc.argtypes = [P, ctypes.c_void_p, ctypes.c_void_p]
    return L


@pytest.mark.parametrize("precision", [0, 1], ids=["complex128", "complex64-contraction"])
@pytest.mark.parametrize("build", [lambda S: H.tfim(S, 9), lambda S: H.tfim(S, 10), lambda S: H.jc(S)],
                         ids=["tfim9-multipass", "tfim10-at-limit", "jc-generic"])
def test_noalloc_matches_device_entry_on_two_calls(quac, build, precision):
    import torch
    L = _bind(quac)
    S = H.ProductSystem(quac)
    build(S)
    quac.construct_matrix(S.qs)
    n = S.D * S.D
    xs = [torch.from_numpy(H.random_state(S.D, seed=s)).cuda() for s in (11, 12)]
    ref = [torch.empty_like(xs[0]) for _ in xs]
    out = [torch.empty_like(xs[0]) for _ in xs]
    quac.set_lrho_precision(precision)
    try:
        assert L.quac_lrho_noalloc_setup(S.qs._ptr) == 0, quac.lib().quac_last_error()
        # existing entry point: allocates its own scratch on its first call
        for x, y in zip(xs, ref):
            quac.lrho_apply_device(S.qs, x.data_ptr(), y.data_ptr())
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        for x, y in zip(xs, out):
            assert L.quac_lrho_apply_device_noalloc(S.qs._ptr, ctypes.c_void_p(x.data_ptr()),
                                                    ctypes.c_void_p(y.data_ptr())) == 0, \
                quac.lib().quac_last_error()
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info()
    finally:
        quac.set_lrho_precision(0)
    assert free1 == free0
    for y, r in zip(out, ref):
        assert y.numel() == n
        assert torch.equal(y, r)
    # the second call's output differs from the first: the scratch carried nothing over
    assert not torch.equal(out[0], out[1])
    S.qs.destroy()


_FRESH = r"""
import ctypes, json, sys
import numpy as np
import torch
sys.path.insert(0, sys.argv[1]); sys.path.insert(0, sys.argv[1] + "/tests")
import quac_b200 as q
import helpers as H
q.lib(); q.QuaC_initialize()
L = q.lib()
P = ctypes.POINTER(q._QsysStruct)
L.quac_lrho_noalloc_setup.restype = ctypes.c_int
L.quac_lrho_noalloc_setup.argtypes = [P]
L.quac_lrho_apply_device_noalloc.restype = ctypes.c_int
L.quac_lrho_apply_device_noalloc.argtypes = [P, ctypes.c_void_p, ctypes.c_void_p]
S = H.ProductSystem(q)
H.tfim(S, int(sys.argv[2]))
q.construct_matrix(S.qs)
x = torch.from_numpy(H.random_state(S.D, seed=5)).cuda()
y = torch.empty_like(x)
yr = torch.empty_like(x)
assert L.quac_lrho_noalloc_setup(S.qs._ptr) == 0
torch.cuda.synchronize()
free0 = torch.cuda.mem_get_info()[0]
rc = L.quac_lrho_apply_device_noalloc(S.qs._ptr, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()))
torch.cuda.synchronize()
free1 = torch.cuda.mem_get_info()[0]
q.lrho_apply_device(S.qs, x.data_ptr(), yr.data_ptr())
torch.cuda.synchronize()
print(json.dumps({"rc": rc, "free0": free0, "free1": free1, "equal": bool(torch.equal(y, yr))}))
"""


@pytest.mark.parametrize("n", [6, 9], ids=["single-pass", "multipass"])
def test_noalloc_first_call_in_fresh_process(quac, n):
    """The very first apply of a process (after setup) allocates nothing:
    setup has already loaded every kernel the apply launches."""
    r = subprocess.run([sys.executable, "-c", _FRESH, ROOT, str(n)], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    res = json.loads(r.stdout.strip().splitlines()[-1])
    assert res["rc"] == 0
    assert res["free1"] == res["free0"]
    assert res["equal"]


def test_noalloc_rejects_oversize(quac):
    import torch
    L = _bind(quac)
    S = H.ProductSystem(quac)
    H.tfim(S, 11)  # 2^22 complex values > 2^20
    quac.construct_matrix(S.qs)
    assert L.quac_lrho_noalloc_setup(S.qs._ptr) == 0
    x = torch.zeros(4, dtype=torch.complex128, device="cuda")
    rc = L.quac_lrho_apply_device_noalloc(S.qs._ptr, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(x.data_ptr()))
    msg = quac.lib().quac_last_error()
    quac.lib().quac_clear_error()
    assert rc != 0 and b"exceed the fixed scratch" in msg
    S.qs.destroy()

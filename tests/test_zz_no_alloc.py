"""The allocation-free L.x entry point against quac_lrho_apply_device.

Collected last (file name) so that it also runs after every other test in
the same process, when the device already holds other systems' buffers.
Both entry points launch the same kernels on the same inputs, so the
results must be bit-identical; device free memory must not change across
the allocation-free calls.
"""
import ctypes

import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu


def _bind(q):
    L = q.lib()
    P = ctypes.POINTER(q._QsysStruct)
    L.quac_lrho_noalloc_setup.restype = ctypes.c_int
    L.quac_lrho_noalloc_setup.argtypes = [P]
    L.quac_lrho_apply_device_noalloc.restype = ctypes.c_int
    L.quac_lrho_apply_device_noalloc.argtypes = [P, ctypes.c_void_p, ctypes.c_void_p]
    return L


@pytest.mark.parametrize("build", [lambda S: H.tfim(S, 9), lambda S: H.tfim(S, 10), lambda S: H.jc(S)],
                         ids=["tfim9-multipass", "tfim10-at-limit", "jc-generic"])
def test_noalloc_matches_device_entry_on_two_calls(quac, build):
    import torch
    L = _bind(quac)
    S = H.ProductSystem(quac)
    build(S)
    quac.construct_matrix(S.qs)
    n = S.D * S.D
    xs = [torch.from_numpy(H.random_state(S.D, seed=s)).cuda() for s in (11, 12)]
    ref = [torch.empty_like(xs[0]) for _ in xs]
    out = [torch.empty_like(xs[0]) for _ in xs]
    assert L.quac_lrho_noalloc_setup(S.qs._ptr) == 0, quac.lib().quac_last_error()
    # existing entry point first: it loads the kernels and allocates its own scratch
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
    assert free1 == free0
    for y, r in zip(out, ref):
        assert y.numel() == n
        assert torch.equal(y, r)
    # the second call's output differs from the first: the scratch carried nothing over
    assert not torch.equal(out[0], out[1])
    S.qs.destroy()


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

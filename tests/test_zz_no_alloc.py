"""hp_resnorm_noalloc: the residual norm for callers that cannot allocate device
memory (a driver inside a global-mode CUDA-graph capture, or an application
whose device memory all belongs to its own pool). Checked through the C-ABI
against the allocating entry point hp_gpu_resnorm on two calls in a row, to the
1e-12 relative tolerance of the parity tests; plus the size limit of its static
scratch. Runs last so that a failure here leaves every other test already run.
"""
import ctypes

import numpy as np
import pytest

import hpb
from hpb import _lib as L

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _bind():
    lib = L.lib()
    lib.hp_resnorm_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_void_p, ctypes.c_longlong,
                                       ctypes.c_void_p, ctypes.c_longlong, ctypes.POINTER(ctypes.c_double),
                                       ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]
    lib.hp_noalloc_last_error.restype = ctypes.c_char_p
    return lib


@pytest.mark.parametrize("kind,p", [("ins", 4), ("cd", 6)])
def test_noalloc_matches_resnorm(kind, p):
    lib = _bind()
    pr = hpb.kovasznay_ins(n=8, p=p) if kind == "ins" else hpb.cd_sinsin(n=12, p=p)
    g = pr.gpu()
    assert g.setup_preconditioner() == 0
    l2_ref, linf_ref = g.resnorm()  # allocating path; leaves the full residual on the device
    ptrs = [ctypes.c_void_p() for _ in range(6)]
    L.check(lib.hp_gpu_device_ptrs(g.h, *[ctypes.byref(q) for q in ptrs]), "device_ptrs")
    nv, ns, ni = pr.ugv.size, pr.ugs.size, pr.ugi.size
    for _ in range(2):
        l2 = ctypes.c_double(-1.0)
        li = ctypes.c_double(-1.0)
        rc = lib.hp_resnorm_noalloc(ptrs[3], nv, ptrs[4], ns, ptrs[5], ni, ctypes.byref(l2), ctypes.byref(li), None)
        assert rc == 0, lib.hp_noalloc_last_error().decode()
        assert abs(l2.value - l2_ref) <= TOL * l2_ref
        assert abs(li.value - linf_ref) <= TOL * linf_ref
    g.close()


def test_noalloc_rejects_oversize():
    lib = _bind()
    too_many = (4096 * 65536) + 1
    l2 = ctypes.c_double()
    li = ctypes.c_double()
    fake = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    rc = lib.hp_resnorm_noalloc(fake, too_many, None, 0, None, 0, ctypes.byref(l2), ctypes.byref(li), None)
    assert rc == -1
    assert b"static scratch" in lib.hp_noalloc_last_error()

"""hp_resnorm_noalloc: the residual norm for callers that cannot allocate device
memory when they need it (an application that owns all device memory through its
own pool, or a solver whose device-memory budget is fixed before the solve).
Checked through the C-ABI against the allocating entry point hp_gpu_resnorm on
two calls in a row, to the 1e-12 relative tolerance of the parity tests; against
numpy on arrays that span several chunks each (with an empty array between two
non-empty ones); plus the size limit of its static scratch. Runs last so that a
failure here leaves every other test already run.
"""
import ctypes

import numpy as np
import pytest

import hpb
from hpb import _lib as L

pytestmark = pytest.mark.gpu

TOL = 1e-12
CHUNK = 65536


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


@pytest.mark.parametrize("sizes", [(200_003, 70_001, 65_537), (200_003, 0, 65_537), (0, 3 * CHUNK, 1)])
def test_noalloc_many_chunks_matches_numpy(sizes):
    """Arrays of several chunks each, partial last chunks and an empty array in the
    middle: the chunk-to-array mapping and the final reduction over many partials."""
    import torch
    lib = _bind()
    rng = np.random.default_rng(sum(sizes))
    host = [rng.uniform(-1.0, 1.0, n) * (1.0 + k) for k, n in enumerate(sizes)]
    if sizes[0]:
        host[0][sizes[0] // 2] = -7.5  # the max |x| sits inside a middle chunk
    dev = [torch.from_numpy(h).to("cuda") for h in host]
    ptr = [ctypes.c_void_p(d.data_ptr()) if d.numel() else None for d in dev]
    torch.cuda.synchronize()
    allv = np.concatenate(host)
    want_l2, want_li = float(np.sqrt(np.sum(allv * allv))), float(np.max(np.abs(allv)))
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for _ in range(2):
        l2 = ctypes.c_double(-1.0)
        li = ctypes.c_double(-1.0)
        rc = lib.hp_resnorm_noalloc(ptr[0], sizes[0], ptr[1], sizes[1], ptr[2], sizes[2], ctypes.byref(l2),
                                    ctypes.byref(li), stream)
        assert rc == 0, lib.hp_noalloc_last_error().decode()
        assert abs(l2.value - want_l2) <= TOL * want_l2
        assert li.value == want_li


def test_noalloc_rejects_oversize():
    lib = _bind()
    too_many = (4096 * 65536) + 1
    l2 = ctypes.c_double()
    li = ctypes.c_double()
    fake = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    rc = lib.hp_resnorm_noalloc(fake, too_many, None, 0, None, 0, ctypes.byref(l2), ctypes.byref(li), None)
    assert rc == -1
    assert b"static scratch" in lib.hp_noalloc_last_error()

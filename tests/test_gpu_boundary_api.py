"""The C-ABI items of the drop-in boundary beyond rsdl / update: hp_gpu_l2error (tri_hp::l2error,
tri_hp/l2error.cpp:13-67, on the device) and the precision argument of hp_gpu_rsdl."""
import ctypes

import numpy as np
import pytest

import hpb
from hpb import _lib as L

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind,p", [("ins", 2), ("ins", 4), ("ins", 6), ("cd", 3), ("cd", 8)])
def test_device_l2error_matches_host_l2error(kind, p):
    """Straight elements: the device reduction against the host restatement (hp_l2error)."""
    pr = hpb.kovasznay_ins(n=8, p=p, noise=1e-3) if kind == "ins" else hpb.cd_sinsin(n=9, p=p, noise=1e-3)
    g = pr.gpu()
    l2g, lig = g.l2error()
    l2h, lih = pr.l2error()
    assert np.all(np.abs(l2g - l2h) <= 1e-12 * np.abs(l2h)), (l2g, l2h)
    assert np.all(np.abs(lig - lih) <= 1e-14 * np.maximum(1.0, np.abs(lih)))
    g.close()


def test_device_l2error_integrates_curved_elements_exactly():
    """With the state u = 1, p = v = 0 and the comparison field 0, l2error's sum is the
    domain area: the isoparametric (curved) Jacobians give the channel minus the circular
    hole to within the geometry error of the p = 3 boundary, far below the polygonal area's
    error."""
    m = hpb.channel_hole(L=4.0, H=2.0, cx=1.0, cy=1.0, r=0.25, hmin=0.06, hmax=0.2, grade=0.1)
    pr = hpb.channel_cylinder_ins(mesh=m, p=3, re=20.0, noise=0.0)
    pr.ugv[:] = 0.0
    pr.ugv[:, 0] = 1.0
    pr.ugs[:] = 0.0
    pr.ugi[:] = 0.0
    g = pr.gpu()
    zero = L.Field(L.HP_FIELD_CONST, (ctypes.c_double * 4)(0.0, 0.0, 0.0, 0.0))
    l2, li = g.l2error(zero)
    exact = 4.0 * 2.0 - np.pi * 0.25 ** 2
    polygon = 0.5 * np.abs(m.area2()).sum()
    assert abs(l2[0] ** 2 - exact) < 1e-6 * exact
    assert abs(polygon - exact) > 20 * abs(l2[0] ** 2 - exact)
    assert l2[1] == 0.0 and li[0] == 1.0
    g.close()


@pytest.mark.parametrize("kind,p", [("ins", 4), ("ins", 1), ("cd", 4)])
def test_rsdl_fp32_precision_matches_fp64_to_single_precision(kind, p):
    pr = hpb.kovasznay_ins(n=8, p=p) if kind == "ins" else hpb.cd_sinsin(n=8, p=p, kcond=1e-2)
    g = pr.gpu()
    assert g.setup_preconditioner() == 0
    out = {}
    for prec in (0, 1):
        g.rsdl(pr.phys.nstage, prec)
        out[prec] = np.concatenate([x.ravel() for x in g.residual()])
    err = np.max(np.abs(out[1] - out[0])) / np.max(np.abs(out[0]))
    assert 0.0 < err < 1e-4, err
    g.close()


def test_stream_ordered_upload_rsdl_download_matches_the_synchronous_calls():
    """hp_gpu_enqueue_upload_state / hp_gpu_enqueue_rsdl / hp_gpu_enqueue_download_residual
    queued on two contexts of the same level, each with its own pinned buffers, give the
    residual of the synchronous calls bit for bit."""
    import ctypes
    import torch
    from hpb import _lib as L
    pr = hpb.kovasznay_ins(n=8, p=4)
    lib = L.lib()
    ref = pr.gpu()
    assert ref.setup_preconditioner() == 0
    ref.rsdl(pr.phys.nstage)
    want = ref.residual()
    ref.close()
    streams = [torch.cuda.Stream() for _ in range(2)]  # kept alive while the contexts use them
    ctxs = [pr.gpu(stream=ctypes.c_void_p(s.cuda_stream)) for s in streams]
    outs = []
    for g in ctxs:
        assert g.setup_preconditioner() == 0
        hin = [torch.from_numpy(a.copy()).pin_memory() for a in (pr.ugv, pr.ugs, pr.ugi)]
        hout = [torch.empty(a.shape, dtype=torch.float64).pin_memory() for a in (pr.ugv, pr.ugs, pr.ugi)]
        L.check(lib.hp_gpu_enqueue_upload_state(g.h, *[ctypes.c_void_p(t.data_ptr()) for t in hin]), "up")
        L.check(lib.hp_gpu_enqueue_rsdl(g.h, pr.phys.nstage), "rsdl")
        L.check(lib.hp_gpu_enqueue_download_residual(g.h, *[ctypes.c_void_p(t.data_ptr()) for t in hout]), "down")
        outs.append((hin, hout))
    for g, (hin, hout) in zip(ctxs, outs):
        L.check(lib.hp_gpu_sync(g.h), "sync")
        for a, b in zip(hout, want):
            assert np.array_equal(a.numpy(), b)
        g.close()

"""Per-level launch-shape autotuner (hp_gpu_autotune): the chosen shapes come from the
candidate sets, and the results after tuning still match the CPU oracle of
tri_hp::rsdl / update (tri_hp/nstage.cpp) to the parity tolerances."""
import ctypes

import numpy as np
import pytest

import hpb
from hpb import _lib as L
from hpb import multigrid as MG
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


def relerr(a, b):
    a = np.concatenate([np.ravel(x) for x in a])
    b = np.concatenate([np.ravel(x) for x in b])
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("kind,ops", [("cd", True), ("cd", False), ("ins", False)])
def test_autotuned_shapes_keep_parity(kind, ops):
    pr = hpb.cd_sinsin(n=12, p=4, kcond=1e-2, cfl=0.5) if kind == "cd" else hpb.kovasznay_ins(n=8, p=3)
    g = pr.gpu()
    o = Oracle(pr)
    assert g.setup_preconditioner() == 0
    assert o.setup_preconditioner() == 0
    if ops:
        g.element_matrices(True)
    tun = g.autotune(reps=3)
    for prec in ("fp64", "fp32"):
        t = tun[prec]
        assert t["elem_cap"] in (4, 8, 16) and t["emat_tpp"] in (1, 2)
        assert t["emat_ctas"] in (0, 2, 4) and t["minv_threads"] in (64, 128, 256)
        assert t["elem_ms"] > 0 and t["minv_ms"] > 0
    g.upload(pr.ugv, pr.ugs, pr.ugi)
    assert g.setup_preconditioner() == 0
    for stage in (pr.phys.nstage, 0, 1):
        g.rsdl(stage)
        o.rsdl(stage)
        assert relerr(g.residual(), o.residual()) < 1e-12
    g.iterate(4)
    for _ in range(4):
        o.update()
    assert relerr(g.state(), o.state()) < 1e-10


def test_autotuned_hierarchy_converges():
    q = L.Field(L.HP_FIELD_QUADX, (ctypes.c_double * 4)(-1.0, 8.0, 0, 0))
    mk = lambda n, p, **kw: hpb.cd_sinsin(n=n, p=p, kcond=1e-2, field=q, **kw)
    H = MG.build(mk, n=16, p=4, hlevels=2, cfl={4: 0.5, 2: 0.75, 1: 1.0})
    H.element_matrices(True)
    shapes = H.autotune(reps=2)
    assert len(shapes) == len(H.levels)
    hist, sec, cyc = H.solve(drop=1e-10, max_cycles=300, mixed=True)
    assert hist[-1] <= 1e-10
    H.close()

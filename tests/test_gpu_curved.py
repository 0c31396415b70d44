"""Curved (isoparametric) elements against the CPU oracle: the elements owning a curved
boundary side use the metrics of their vertex and side position modes at every
quadrature point (tri_hp/ins/rsdl.cpp:83-258, tri_hp/cd/rsdl.cpp:20-24,
ins/setup_preconditioner.cpp:45-87, the curved boundary-side normal of
hp_edge_bdry::rsdl). Mesh: a small channel with a circular hole whose sides are
curved (position modes from hp_curved_side_modes)."""
import ctypes

import numpy as np
import pytest

import hpb
from hpb import _lib as L
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


def relerr(a, b):
    a = np.concatenate([np.ravel(x) for x in a])
    b = np.concatenate([np.ravel(x) for x in b])
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def tol_minvrt(p):
    """p >= 5: the static-inversion tables amplify rounding of the summation order."""
    return 1e-12 if p <= 4 else 1e-11


def tol_rsdl(p):
    return 1e-12 if p <= 6 else 1e-11


def small_channel():
    return hpb.channel_hole(L=4.0, H=2.0, cx=1.0, cy=1.0, r=0.25, hmin=0.08, hmax=0.3, grade=0.2)


def cd_with_curved_hole(p, src=0.0):
    m = small_channel()
    cx, cy, r = m.hole
    b = m.boundary_segments()
    mid = 0.5 * (m.pnts[m.seg_pnt[b, 0]] + m.pnts[m.seg_pnt[b, 1]])
    hole = np.hypot(mid[:, 0] - cx, mid[:, 1] - cy) < r + 1e-9
    f = L.Field(L.HP_FIELD_QUADX, (ctypes.c_double * 4)(-1.0, 8.0, 0, 0))
    bc = [(b[~hole], 0b1), (b[hole], 0b1, hpb.circle_curve(cx, cy, r))]
    pr = hpb.Problem(m, p, L.HP_PHYS_CD, rhocv=1.0, kcond=2e-2, ax=1.0, ay=0.3, src=src, field=f, bc=bc, cfl=0.5)
    return pr.tobasis(noise=1e-3, seed=5)


def check_level(pr, p, ops=False):
    g = pr.gpu()
    o = Oracle(pr)
    if ops:
        g.element_matrices(True)
    assert g.setup_preconditioner() == 0
    assert o.setup_preconditioner() == 0
    gv, gs, gt, gtau = g.prcn()
    ov, os_, ot, otau = o.prcn()
    assert relerr([gv, gt], [ov, ot]) < 1e-12
    for stage in (pr.phys.nstage, 0, 1):
        g.rsdl(stage)
        o.rsdl(stage)
        assert relerr(g.residual(), o.residual()) < tol_rsdl(p), f"rsdl stage {stage}"
    g.minvrt()
    o.minvrt()
    assert relerr(g.residual(), o.residual()) < tol_minvrt(p)
    g.iterate(4)
    for _ in range(4):
        o.update()
    assert relerr(g.state(), o.state()) < 1e-10


@pytest.mark.parametrize("p", [2, 3, 4, 6])
def test_ins_curved_hole_parity(p):
    pr = hpb.channel_cylinder_ins(mesh=small_channel(), p=p, re=50.0)
    assert np.any(pr.bcrd != 0.0)
    check_level(pr, p)


@pytest.mark.parametrize("p,ops", [(2, False), (4, False), (4, True), (6, True)])
def test_cd_curved_hole_parity(p, ops):
    check_level(cd_with_curved_hole(p, src=0.7), p, ops)


def test_curved_geometry_changes_the_residual():
    """The same state on the same mesh, with and without curved hole sides."""
    m = small_channel()
    a = hpb.channel_cylinder_ins(mesh=m, p=4, re=50.0)
    b = hpb.channel_cylinder_ins(mesh=m, p=4, re=50.0, curved=False)
    ga, gb = a.gpu(), b.gpu()
    gb.upload(a.ugv, a.ugs, a.ugi)
    for g in (ga, gb):
        assert g.setup_preconditioner() == 0
        g.rsdl(a.phys.nstage)
    assert relerr(ga.residual(), gb.residual()) > 1e-4

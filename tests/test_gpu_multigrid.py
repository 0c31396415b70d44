"""Multigrid on the GPU: the p- and h-transfers against numpy restatements of
tri_hp::mg_restrict / mg_prolongate (movco.cpp, movfin.cpp), the FAS source
(mg_source), and convergence of V-cycles."""
import ctypes

import numpy as np
import pytest

import hpb
from hpb import _lib as L
from hpb import multigrid as MG

pytestmark = pytest.mark.gpu


def interior_map(smc, smf):
    out = []
    off_f = 0
    for m in range(1, smf):
        for k in range(smf - m):
            if m < smc and k < smc - m:
                out.append(off_f + k)
        off_f += smf - m
    return np.array(out, dtype=int)


def test_p_restriction_and_fas_source():
    H = MG.build(lambda n, p, **kw: hpb.kovasznay_ins(n=n, p=p, **kw), n=6, p=4)
    f, c = H.levels[0], H.levels[1]
    assert f.setup_preconditioner() == 0
    f.rsdl(f.prob.phys.nstage)
    rf = f.residual()
    uf = f.state()
    L.check(H.lib.hp_gpu_mg_restrict(c.h), "restrict")
    uc = c.state()
    smc, imc = c.prob.sm, c.prob.im
    imap = interior_map(smc, f.prob.sm)
    assert np.array_equal(uc[0], uf[0])
    assert np.array_equal(uc[1], uf[1][:, :smc, :])
    assert np.array_equal(uc[2], uf[2][:, imap, :])
    # the coarse residual with the FAS source at the restricted state is fadd*res0
    assert c.setup_preconditioner() == 0
    c.rsdl(c.prob.phys.nstage)
    rc = c.residual()
    want = (rf[0], rf[1][:, :smc, :], rf[2][:, imap, :])
    for a, b in zip(rc, want):
        if b.size:
            assert np.max(np.abs(a - b)) <= 1e-12 * max(1.0, np.max(np.abs(b)))
    H.close()


def test_coarse_driving_term_waits_for_coarse_preconditioner():
    """As the reference's isfrst (nstage.cpp:113-129), the FAS source is formed at the
    coarse level's first residual after restriction, with that level's own tau."""
    H = MG.build(lambda n, p, **kw: hpb.cd_sinsin(n=n, p=p, kcond=1e-2, cfl=0.5, **kw), n=6, p=4)
    f, c = H.levels[0], H.levels[1]
    assert f.setup_preconditioner() == 0
    f.rsdl(f.prob.phys.nstage)
    L.check(H.lib.hp_gpu_mg_restrict(c.h), "restrict")
    with pytest.raises(RuntimeError):
        c.rsdl(c.prob.phys.nstage)
    assert c.setup_preconditioner() == 0
    c.rsdl(c.prob.phys.nstage)
    rf = f.residual()
    imap = interior_map(c.prob.sm, f.prob.sm)
    want = (rf[0], rf[1][:, :c.prob.sm, :], rf[2][:, imap, :])
    for a, b in zip(c.residual(), want):
        if b.size:
            assert np.max(np.abs(a - b)) <= 1e-12 * max(1.0, np.max(np.abs(b)))
    H.close()


def test_h_restriction_and_prolongation():
    H = MG.build(lambda n, p, **kw: hpb.kovasznay_ins(n=n, p=p, **kw), n=8, p=1, hlevels=1)
    f, c = H.levels[0], H.levels[1]
    fm, cm = f.prob.mesh, c.prob.mesh
    assert f.setup_preconditioner() == 0
    f.rsdl(f.prob.phys.nstage)
    rf = f.residual()[0]
    uf = f.state()[0]
    L.check(H.lib.hp_gpu_mg_restrict(c.h), "restrict")
    uc = c.state()[0]
    t_c2f, w_c2f = MG.connect(cm, fm)
    want_u = np.einsum("kj,kjn->kn", w_c2f, uf[fm.tri_pnt[t_c2f]])
    assert np.max(np.abs(uc - want_u)) < 1e-13
    t_f2c, w_f2c = MG.connect(fm, cm)
    res0 = np.zeros_like(uc)
    for j in range(3):
        np.add.at(res0, cm.tri_pnt[t_f2c, j], w_f2c[:, j:j + 1] * rf)
    assert c.setup_preconditioner() == 0
    c.rsdl(c.prob.phys.nstage)
    rc = c.residual()[0]
    assert np.max(np.abs(rc - res0)) <= 1e-12 * np.max(np.abs(res0))
    # prolongation adds the interpolated coarse correction to the fine vertices
    c.update()
    duc = c.state()[0] - uc
    L.check(H.lib.hp_gpu_mg_prolongate(c.h), "prolongate")
    want = uf + np.einsum("kj,kjn->kn", w_f2c, duc[cm.tri_pnt[t_f2c]])
    assert np.max(np.abs(f.state()[0] - want)) < 1e-12
    H.close()


def quad():
    return L.Field(L.HP_FIELD_QUADX, (ctypes.c_double * 4)(-1.0, 8.0, 0, 0))


def test_vcycle_converges_faster_than_single_grid_cd():
    mk = lambda n, p, **kw: hpb.cd_sinsin(n=n, p=p, kcond=1e-2, field=quad(), **kw)
    H = MG.build(mk, n=16, p=4, hlevels=2, cfl={4: 0.5, 2: 0.75, 1: 1.0})
    hist, sec, cycles = H.solve(drop=1e-10, max_cycles=300, itercrsn=2, iterrfne=2)
    assert hist[-1] <= 1e-10
    fine_updates_mg = 4 * cycles
    g = mk(n=16, p=4, cfl=0.5).gpu()
    h1, s1, upd = g.solve(drop=1e-10, max_updates=20000, check_every=10)
    assert h1[-1] <= 1e-10
    assert fine_updates_mg < upd
    H.close()


def test_vcycle_converges_ins_kovasznay():
    mk = lambda n, p, **kw: hpb.kovasznay_ins(n=n, p=p, re=100.0, **kw)
    H = MG.build(mk, n=16, p=4, hlevels=2)
    hist, sec, cycles = H.solve(drop=1e-10, max_cycles=400, itercrsn=2, iterrfne=2)
    assert hist[-1] <= 1e-10, hist[-5:]
    H.close()


@pytest.mark.parametrize("kind", ["cd", "ins"])
def test_mixed_multigrid_matches_fp64_multigrid(kind):
    """FP32 cycles on the correction equation inside FP64 defect correction reach
    the 1e-10 drop of the FP64 residual and the FP64 multigrid solution."""
    if kind == "cd":
        mk = lambda n, p, **kw: hpb.cd_sinsin(n=n, p=p, kcond=1e-2, field=quad(), **kw)
        cfl = {4: 0.5, 2: 0.75, 1: 1.0}
    else:
        mk = lambda n, p, **kw: hpb.kovasznay_ins(n=n, p=p, re=100.0, **kw)
        cfl = None
    H1 = MG.build(mk, n=16, p=4, hlevels=2, cfl=cfl)
    h1, s1, c1 = H1.solve(drop=1e-10, max_cycles=400)
    u1 = H1.levels[0].state()
    H1.close()
    H2 = MG.build(mk, n=16, p=4, hlevels=2, cfl=cfl)
    h2, s2, c2 = H2.solve(drop=1e-10, max_cycles=400, mixed=True)
    u2 = H2.levels[0].state()
    H2.close()
    assert h1[-1] <= 1e-10 and h2[-1] <= 1e-10, (h1[-3:], h2[-3:])
    num = np.sqrt(sum(np.sum((a - b) ** 2) for a, b in zip(u1, u2)))
    den = np.sqrt(sum(np.sum(a * a) for a in u1))
    assert num / den < 1e-9


@pytest.mark.parametrize("prcn_every", [0, 1])
def test_vcycle_graph_matches_level_by_level(prcn_every):
    """The captured V-cycle replays the level-by-level cycle: with the preconditioner
    set-ups inside the graph (prcn_every = 1, the reference's default interval) or
    frozen after the first cycle (prcn_every = 0)."""
    mk = lambda n, p, **kw: hpb.kovasznay_ins(n=n, p=p, re=100.0, **kw)
    H1 = MG.build(mk, n=16, p=4, hlevels=2)
    h1, s1, c1 = H1.solve(drop=1e-10, max_cycles=400, itercrsn=2, iterrfne=2, prcn_every=prcn_every)
    u1 = H1.levels[0].state()
    H1.close()
    H2 = MG.build(mk, n=16, p=4, hlevels=2)
    h2, s2, c2 = H2.solve(drop=1e-10, max_cycles=400, itercrsn=2, iterrfne=2, graph=True, prcn_every=prcn_every)
    u2 = H2.levels[0].state()
    H2.close()
    assert h1[-1] <= 1e-10 and h2[-1] <= 1e-10
    assert abs(c1 - c2) <= 2
    num = np.sqrt(sum(np.sum((a - b) ** 2) for a, b in zip(u1, u2)))
    den = np.sqrt(sum(np.sum(a * a) for a in u1))
    assert num / den < 1e-8


def test_vcycle_on_delaunay_meshes():
    """Non-nested h-levels: each level is its own seeded Delaunay mesh; the transfers
    locate every point in the other mesh (mgconnect semantics)."""
    mk = lambda n, p, **kw: hpb.cd_sinsin(mesh=hpb.delaunay_square(n, seed=n), p=p, kcond=1e-2, field=quad(), **kw)
    H = MG.build(mk, n=24, p=4, hlevels=2, cfl={4: 0.5, 2: 0.75, 1: 1.0})
    hist, sec, cycles = H.solve(drop=1e-10, max_cycles=300)
    assert hist[-1] <= 1e-10
    H.close()


def test_curved_hole_cycles_keep_essential_values_and_converge():
    """ins past a curved hole with h-levels on coarser, non-nested channel meshes: the
    boundary re-connection keeps the fine no-slip values exact through every
    prolongation, and W-cycles (vwcycle 2) reach the 1e-10 drop."""
    ms = [hpb.channel_hole(L=4.0, H=2.0, cx=1.0, cy=1.0, r=0.25, hmin=0.04 * k, hmax=0.15 * k, grade=0.1 * k)
          for k in (1, 2)]
    probs = [hpb.channel_cylinder_ins(mesh=ms[0], p=2, re=20.0), hpb.channel_cylinder_ins(mesh=ms[0], p=1, re=20.0),
             hpb.channel_cylinder_ins(mesh=ms[1], p=1, re=20.0)]
    H = MG.Hierarchy(probs, ["fine", "p", "h"])
    hist, sec, cycles = H.solve(drop=1e-10, max_cycles=300, vw=2)
    assert hist[-1] <= 1e-10, hist[-5:]
    m = ms[0]
    cx, cy, r = m.hole
    on_hole = np.abs(np.hypot(m.pnts[:, 0] - cx, m.pnts[:, 1] - cy) - r) < 1e-9
    assert np.count_nonzero(on_hole) > 8
    uv = H.levels[0].state()[0][on_hole, :2]
    assert np.max(np.abs(uv)) == 0.0
    H.close()


@pytest.mark.parametrize("kind,method", [("ins", "coarsen"), ("cd-delaunay", "coarsen"), ("ins", "coarsen2"),
                                         ("cd-delaunay", "coarsen2")])
def test_cycles_on_coarsened_h_levels(kind, method):
    """h-levels made from the level above by hpb.coarsen (tri_mesh::coarsen, factor 1.5) or
    by hpb.coarsen2 (tri_mesh::coarsen2, edge collapse, factor 2): the cycles reach the 1e-10
    drop, in a cycle count close to that of the generated (nested) levels for the structured
    mesh."""
    if kind == "ins":
        def mk(n=16, p=4, mesh=None, **kw):
            return hpb.kovasznay_ins(n=n, p=p, re=100.0, mesh=mesh, **kw)
        cfl = None
    else:
        def mk(n=24, p=4, mesh=None, **kw):
            return hpb.cd_sinsin(mesh=mesh if mesh is not None else hpb.delaunay_square(n, seed=n), p=p, kcond=1e-2,
                                 field=quad(), **kw)
        cfl = {4: 0.5, 2: 0.75, 1: 1.0}
    n = 16 if kind == "ins" else 24
    H = MG.build(mk, n=n, p=4, hlevels=2, cfl=cfl, coarsen=1.5 if method == "coarsen" else 2.0,
                 coarsen_method=method)
    assert H.levels[-1].prob.mesh.ntri < 0.1 * H.levels[0].prob.mesh.ntri
    hist, sec, cycles = H.solve(drop=1e-10, max_cycles=400, itercrsn=2, iterrfne=2)
    H.close()
    assert hist[-1] <= 1e-10, hist[-3:]
    if kind == "ins":
        H = MG.build(mk, n=n, p=4, hlevels=2, cfl=cfl)
        h2, s2, c2 = H.solve(drop=1e-10, max_cycles=400, itercrsn=2, iterrfne=2)
        H.close()
        assert cycles <= 1.3 * c2 + 3, (cycles, c2)

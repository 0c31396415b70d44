"""Stored cd element operators (hp_gpu_set_element_matrices) against the CPU
oracle of tri_hp::rsdl / minvrt / update (tri_hp/nstage.cpp, tri_hp/cd/rsdl.cpp).

The operators are the matrix-free element kernel applied to unit vectors, so the
batched mat-vec differs from the oracle only in summation order: the same
tolerances as the matrix-free parity tests apply (1e-12 of max|oracle| for one
rsdl / minvrt, 1e-10 after several updates)."""
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


def tol1(p):
    return 1e-12 if p <= 6 else 1e-11


def quad():
    return L.Field(L.HP_FIELD_QUADX, (ctypes.c_double * 4)(-1.0, 8.0, 0, 0))


@pytest.mark.parametrize("p", [1, 2, 3, 4, 5, 6, 7, 8])
def test_rsdl_minvrt_from_element_operators(p):
    # n = 7: 98 elements, a partial last tile for every p
    pr = hpb.cd_sinsin(n=7, p=p, kcond=1e-2, cfl=0.5, src=0.7)
    g = pr.gpu()
    g.element_matrices(True)
    o = Oracle(pr)
    assert g.setup_preconditioner() == 0
    assert o.setup_preconditioner() == 0
    # nstage: beta = 1 (A_im and A_re), 0: beta(0) = 1 with res_r mixing, 1: beta = 0 (A_im only)
    for stage in (pr.phys.nstage, 0, 1, 2):
        g.rsdl(stage)
        o.rsdl(stage)
        assert relerr(g.residual(), o.residual()) < tol1(p), f"rsdl stage {stage}"
    g.minvrt()
    o.minvrt()
    assert relerr(g.residual(), o.residual()) < tol1(p), "minvrt"


@pytest.mark.parametrize("p", [1, 2, 3, 4, 5, 6, 7, 8])
def test_fp32_updates_from_element_operators_match_matrix_free(p):
    """The FP32 operator copy (paired 8-byte row loads at p <= 2; at p = 1 a pair can
    span two elements) against the FP32 matrix-free kernels, on a mesh whose last
    tile is partial; both start from fp32(u), so they differ by FP32 rounding only."""
    pr = hpb.cd_sinsin(n=7, p=p, kcond=1e-2, cfl=0.5, src=0.7)
    a, b = pr.gpu(), pr.gpu()
    b.element_matrices(True)
    for g in (a, b):
        assert g.setup_preconditioner() == 0
    u0 = a.state()
    for g in (a, b):
        L.check(g.lib.hp_gpu_fp32_updates(g.h, 3))
    ua, ub = a.state(), b.state()
    moved, diff = relerr(ua, u0), relerr(ub, ua)
    assert moved > 1e-3
    assert diff < 1e-5  # measured 6e-8 (p = 1) to 2.1e-6 (p = 8)


def test_update_iterations_from_element_operators():
    pr = hpb.cd_sinsin(n=6, p=4, kcond=1e-2, cfl=0.5)
    g = pr.gpu()
    g.element_matrices(True)
    o = Oracle(pr)
    g.setup_preconditioner()
    o.setup_preconditioner()
    hist = g.iterate(4)
    oh = []
    for _ in range(4):
        o.update()
        oh.append(o.maxres()[0])
    assert relerr(g.state(), o.state()) < 1e-10
    assert np.max(np.abs(hist - np.array(oh)) / np.array(oh)) < 1e-9


def test_switching_operators_on_and_off_matches_matrix_free():
    pr = hpb.cd_sinsin(n=9, p=3, kcond=1e-2, cfl=0.5, src=0.3)
    a, b = pr.gpu(), pr.gpu()
    a.setup_preconditioner()
    b.setup_preconditioner()
    b.element_matrices(True)  # built at once: the preconditioner is set up
    a.iterate(5)
    b.iterate(5)
    assert relerr(b.state(), a.state()) < 1e-10
    b.element_matrices(False)
    a.iterate(3)
    b.iterate(3)
    assert relerr(b.state(), a.state()) < 1e-10


def test_ins_has_no_element_operators():
    g = hpb.kovasznay_ins(n=4, p=2).gpu()
    with pytest.raises(RuntimeError):
        g.element_matrices(True)


def test_mixed_solve_with_element_operators_reaches_fp64_solution():
    """FP32 correction smoothing on the FP32 operator copy inside FP64 defect
    correction reaches the 1e-10 drop of the FP64 residual and the FP64 solution."""
    mk = lambda: hpb.cd_sinsin(n=16, p=4, kcond=1e-2, field=quad(), cfl=0.5)
    g1 = mk().gpu()
    h1, s1, u1n = g1.solve(mixed=False, drop=1e-10, max_updates=20000, check_every=10)
    g2 = mk().gpu()
    g2.element_matrices(True)
    h2, s2, u2n = g2.solve(mixed=True, drop=1e-10, max_updates=20000, inner=20)
    assert h1[-1] <= 1e-10 and h2[-1] <= 1e-10
    u1, u2 = g1.state(), g2.state()
    num = np.sqrt(sum(np.sum((x - y) ** 2) for x, y in zip(u1, u2)))
    den = np.sqrt(sum(np.sum(x * x) for x in u1))
    assert num / den < 1e-9


@pytest.mark.parametrize("mixed", [False, True])
def test_multigrid_with_element_operators_matches_matrix_free(mixed):
    from hpb import multigrid as MG
    mk = lambda n, p, **kw: hpb.cd_sinsin(n=n, p=p, kcond=1e-2, field=quad(), **kw)
    cfl = {4: 0.5, 2: 0.75, 1: 1.0}
    H1 = MG.build(mk, n=16, p=4, hlevels=2, cfl=cfl)
    h1, s1, c1 = H1.solve(drop=1e-10, max_cycles=400)
    u1 = H1.levels[0].state()
    H1.close()
    H2 = MG.build(mk, n=16, p=4, hlevels=2, cfl=cfl)
    H2.element_matrices(True)
    h2, s2, c2 = H2.solve(drop=1e-10, max_cycles=400, mixed=mixed)
    u2 = H2.levels[0].state()
    H2.close()
    assert h1[-1] <= 1e-10 and h2[-1] <= 1e-10
    if not mixed:
        assert abs(c1 - c2) <= 1
    num = np.sqrt(sum(np.sum((a - b) ** 2) for a, b in zip(u1, u2)))
    den = np.sqrt(sum(np.sum(a * a) for a in u1))
    assert num / den < 1e-9

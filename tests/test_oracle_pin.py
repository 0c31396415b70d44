"""CPU tests that pin the oracle and the shipped host code to the reference.

* basis tables built by the library (hp_basis_build) against the reference's own
  tri_basis compiled here (oracle/_ref);
* the oracle's basis operators against the reference's proj / intgrt / intgrtrs
  / derivr / derivs / proj1d / intgrt1d;
* the DPBTRSNU2 restatement against utilities/myblas.c, including its indexing
  quirk;
* the exactness known-answer test of Testing/tri_hp/conv-diff/Correctness;
* the split-square mesh against the reference's square7.grd (its golden hash in
  tests/golden/square7_grd.json, and the file itself when HP_REFERENCE_DIR names
  the reference checkout).
"""
import ctypes
import os

import numpy as np
import pytest

import hpb
from hpb import _lib as L
from oracle import oracle as O

REF_DIR = os.environ.get("HP_REFERENCE_DIR")  # reference checkout, for the checks that read its files
REF_GRD = os.path.join(REF_DIR, "Testing/tri_hp/ins/Spatial Accuracy/Inputs/square7.grd") if REF_DIR else None
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TABLES = ["gx", "dgx", "wtx", "xp", "x0", "gxwtx", "dgxwtx", "dltx", "dltx1", "gn", "dgn", "wtn", "np", "n0",
          "gnwtn", "gnwtnn0", "dgnwtn", "dltn", "dltn1", "dltn2", "norm", "sfmv", "ifmb", "vdiag", "vfms", "sdiag",
          "sfms", "bfmi", "idiag", "sfmv1d", "vdiag1d", "vfms1d", "sdiag1d"]
# tables that depend on the side/interior static inversion the reference leaves
# undefined for p >= 5 (its systems have fewer equations than unknowns there)
P5_DIFFER = {"ifmb", "vfms", "sfms", "sdiag"}


def shape(name, p):
    G, X, T, SM, IM, BM = p + 1, p + 2, (p + 1) * (p + 2) // 2, p - 1, (p - 1) * (p - 2) // 2, 3 * p
    return {"gx": (G, X), "dgx": (G, X), "wtx": (G,), "xp": (G,), "x0": (G,), "gxwtx": (X, G), "dgxwtx": (X, G),
            "dltx": (G,), "dltx1": (G, G), "gn": (G, T), "dgn": (G, T), "wtn": (G,), "np": (G,), "n0": (G,),
            "gnwtn": (T, G), "gnwtnn0": (T, G), "dgnwtn": (T, G), "dltn": (G,), "dltn1": (G, G), "dltn2": (G, G),
            "norm": (T,), "sfmv": (2, SM), "ifmb": (BM, IM), "vdiag": (), "vfms": (3, SM), "sdiag": (SM,),
            "sfms": (SM - 1, SM, 3), "bfmi": (BM, IM), "idiag": (IM, 2), "sfmv1d": (2, SM), "vdiag1d": (),
            "vfms1d": (2, SM), "sdiag1d": (SM, 3)}[name]


def mine(t, name, p):
    sh = shape(name, p)
    if sh == ():
        return np.array([getattr(t, name)])
    if min(sh) <= 0:
        return np.zeros(0)
    a = np.array(getattr(t, name))
    return a[tuple(slice(0, s) for s in sh)].ravel()


def theirs(r, name, p):
    buf = np.zeros(40000)
    n = r.ref_tb_get(p, name.encode(), buf.ctypes.data_as(ctypes.c_void_p))
    assert n >= 0
    return buf[:n]


needs_ref = pytest.mark.skipif(O.ref() is None, reason="oracle/_ref not built (reference tree absent)")


@needs_ref
@pytest.mark.parametrize("p", range(1, 9))
def test_tables_match_reference(p):
    r = O.ref()
    t = hpb.basis_tables(p)
    for name in TABLES:
        a, b = mine(t, name, p), theirs(r, name, p)
        assert a.size == b.size, name
        if a.size == 0 or (p >= 5 and name in P5_DIFFER):
            continue
        err = np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)
        assert err < 1e-12, (name, err)


@needs_ref
@pytest.mark.parametrize("p", [5, 6, 8])
def test_static_inversion_rows_well_defined_beyond_reference(p):
    """For p >= 5 the library's ifmb rows come from the exact interior static
    inversion, so they are finite and bounded where the reference's are not."""
    t = hpb.basis_tables(p)
    ifmb = mine(t, "ifmb", p)
    assert np.all(np.isfinite(ifmb)) and np.max(np.abs(ifmb)) < 1e3
    assert np.all(mine(t, "sdiag", p) > 0)


def _rand(n, seed):
    return hpb.splitmix64_uniform(seed, n)


@needs_ref
@pytest.mark.parametrize("p", [1, 2, 3, 4, 6, 8])
def test_basis_ops_match_reference(p):
    r = O.ref()
    o = O.lib()
    t = hpb.basis_tables(p)
    G, T, S = p + 1, (p + 1) * (p + 2) // 2, 9
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    tp = ctypes.addressof(t)
    lin = _rand(T, 11 + p)

    def rel(a, b):
        return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)

    f1, dx1, dy1 = (np.zeros((G, S)) for _ in range(3))
    f2, dx2, dy2 = (np.zeros((G, S)) for _ in range(3))
    o.or_basis_proj(tp, P(lin), P(f1), P(dx1), P(dy1), S)
    r.ref_proj(p, P(lin), P(f2), P(dx2), P(dy2), S)
    assert rel(f1, f2) < 1e-13 and rel(dx1, dx2) < 1e-13 and rel(dy1, dy2) < 1e-13
    fx, fy = _rand(G * S, 5).reshape(G, S), _rand(G * S, 6).reshape(G, S)
    a1, a2 = np.zeros(T), np.zeros(T)
    o.or_basis_intgrt(tp, P(a1), P(fx), S)
    r.ref_intgrt(p, P(a2), P(fx), S)
    assert rel(a1, a2) < 1e-13
    a1[:] = 0.3
    a2[:] = 0.3
    o.or_basis_intgrtrs(tp, P(a1), P(fx), P(fy), S)
    r.ref_intgrtrs(p, P(a2), P(fx), P(fy), S)
    assert rel(a1, a2) < 1e-13
    d1, d2 = np.full((G, S), 0.1), np.full((G, S), 0.1)
    o.or_basis_derivr(tp, P(fx), P(d1), S)
    r.ref_derivr(p, P(fx), P(d2), S)
    assert rel(d1, d2) < 1e-12
    o.or_basis_derivs(tp, P(fy), P(d1), S)
    r.ref_derivs(p, P(fy), P(d2), S)
    assert rel(d1, d2) < 1e-12
    l1 = _rand(p + 1, 9)
    g1, e1, g2, e2 = np.zeros(G), np.zeros(G), np.zeros(G), np.zeros(G)
    o.or_basis_proj1d(tp, P(l1), P(g1), P(e1))
    r.ref_proj1d(p, P(l1), P(g2), P(e2))
    assert rel(g1, g2) < 1e-13 and rel(e1, e2) < 1e-13
    i1, i2 = np.zeros(p + 1), np.zeros(p + 1)
    o.or_basis_intgrt1d(tp, P(i1), P(g1))
    r.ref_intgrt1d(p, P(i2), P(g1))
    assert rel(i1, i2) < 1e-13


@needs_ref
def test_dpbtrsnu2_restatement_and_quirk():
    """utilities/myblas.c:91-120 indexes b[ba+j] = b[0] for rows i > ofdg in both
    sweeps; the oracle (and the GPU minvrt) reproduce it bit for bit. With this
    basis the interior mass matrix is diagonal to rounding (its off-diagonal band
    entries are ~1e-16), so the quirk changes the solve only at rounding level."""
    r = O.ref()
    o = O.lib()
    r.DPBTRSNU2.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
    t = hpb.basis_tables(6)
    im = t.im
    ab = np.array(t.idiag)[:im].copy()
    b0 = _rand(im * 3, 3)
    b1, b2 = b0.copy(), b0.copy()
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    o.or_dpbtrsnu2(P(ab), 2, im, 1, P(b1), 3)
    r.DPBTRSNU2(P(ab), 2, im, 1, P(b2), 3)
    assert np.array_equal(b1, b2)
    # a true solve of the banded factor
    U = np.zeros((im, im))
    for j in range(im):
        U[j, j] = ab[j, 1]
        if j:
            U[j - 1, j] = ab[j, 0]
    x = np.linalg.solve(U.T @ U, b0.reshape(im, 3))
    assert np.max(np.abs(ab[1:, 0])) < 1e-14
    assert np.max(np.abs(x.ravel() - b1)) < 1e-13


def test_cd_quadratic_exactness_kat():
    """Testing/tri_hp/conv-diff/Correctness: u = -(x-8)^2 with nu = 1, source 2 is
    reproduced exactly at p = 2 on straight-sided elements."""
    pr = hpb.cd_quadratic(n=4, p=2)
    o = O.Oracle(pr)
    assert o.setup_preconditioner() == 0
    for _ in range(300):
        o.update()
    l2, linf = pr.l2error(*o.state())
    assert l2[0] < 1e-12 and linf[0] < 1e-11
    assert o.maxres()[0] < 1e-13


def test_tobasis_spatial_accuracy():
    """Spatial Accuracy (Testing/tri_hp/ins/Spatial Accuracy): the projected
    Kovasznay field converges at the rate p+1 under h-refinement."""
    for p in (2, 4):
        e = []
        for n in (4, 8):
            pr = hpb.kovasznay_ins(n=n, p=p, noise=0.0)
            e.append(pr.l2error()[0])
        rate = np.log2(e[0] / e[1])
        assert np.all(rate > p + 0.5), (p, rate)


def test_square_mesh_matches_square7_grd():
    import json
    import sys
    sys.path.insert(0, GOLDEN)
    from make_reference_fixtures import tri_keys_sha256
    m = hpb.square_mesh(64)
    assert (m.npnt, m.nseg, m.ntri) == (4225, 12416, 8192)
    assert np.all(m.area2() > 0)
    gold = json.load(open(os.path.join(GOLDEN, "square7_grd.json")))
    assert (gold["npnt"], gold["nseg"], gold["ntri"]) == (m.npnt, m.nseg, m.ntri)
    assert tri_keys_sha256(m.pnts, m.tri_pnt, 64) == gold["tri_keys_sha256"]


@pytest.mark.skipif(not (REF_GRD and os.path.exists(REF_GRD)), reason="HP_REFERENCE_DIR unset")
def test_square7_grd_file_matches_its_golden_hash():
    import json
    import sys
    sys.path.insert(0, GOLDEN)
    from make_reference_fixtures import tri_keys_sha256
    m = hpb.square_mesh(64)
    gold = json.load(open(os.path.join(GOLDEN, "square7_grd.json")))
    g = hpb.read_grd(REF_GRD)
    assert (g.npnt, g.nseg, g.ntri) == (m.npnt, m.nseg, m.ntri)
    assert tri_keys_sha256(g.pnts, g.tri_pnt, 64) == gold["tri_keys_sha256"]


def test_createsegtri_conventions():
    m = hpb.square_mesh(6)
    for t in range(m.ntri):
        for j in range(3):
            s = m.tri_seg[t, j]
            a, b = m.tri_pnt[t, (j + 1) % 3], m.tri_pnt[t, (j + 2) % 3]
            if m.tri_sgn[t, j] > 0:
                assert (m.seg_pnt[s, 0], m.seg_pnt[s, 1]) == (a, b) and m.seg_tri[s, 0] == t
            else:
                assert (m.seg_pnt[s, 0], m.seg_pnt[s, 1]) == (b, a) and m.seg_tri[s, 1] == t
    b = m.boundary_segments()
    assert len(b) == 24 and np.all(m.seg_tri[b, 0] >= 0)


def test_abi_exports_every_declared_symbol():
    import glob
    import re
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    names = set()
    headers = sorted(glob.glob(os.path.join(root, "include", "*.h")))
    assert {os.path.basename(h) for h in headers} >= {"hp_gpu.h", "hp_host.h", "hp_mlp.h", "hp_tet.h"}
    for h in headers:
        txt = open(h).read()
        names |= set(re.findall(r"^(?:int|double|void|const char \*)\s*(hp_\w+)\(", txt, flags=re.M))
    assert len(names) > 60
    lib = L.lib()
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


@needs_ref
@pytest.mark.parametrize("p", [2, 3, 4, 6, 8])
def test_curved_metrics_projection_matches_reference_proj_bdry(p):
    """The curved-element metrics project the vertex and side position modes (interior
    modes zero) with derivatives: the oracle's projection of such a vector equals the
    reference's own tri_basis::proj_bdry (tri_basis/proj.cpp:201-281)."""
    r = O.ref()
    o = O.lib()
    t = hpb.basis_tables(p)
    G, T, S = p + 1, (p + 1) * (p + 2) // 2, 9
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    lin = _rand(T, 31 + p)
    lin[3 * p:] = 0.0
    f1, dx1, dy1 = (np.zeros((G, S)) for _ in range(3))
    f2, dx2, dy2 = (np.zeros((G, S)) for _ in range(3))
    o.or_basis_proj(ctypes.addressof(t), P(lin), P(f1), P(dx1), P(dy1), S)
    r.ref_proj_bdry(p, P(lin), P(f2), P(dx2), P(dy2), S)
    for a, b in ((f1, f2), (dx1, dx2), (dy1, dy2)):
        assert np.max(np.abs(a - b)) <= 1e-13 * max(1.0, np.max(np.abs(b)))


@pytest.mark.parametrize("p", [2, 4, 6])
def test_curved_side_modes(p):
    """hp_curved_side_modes (hp_edge_bdry::curv_init): a boundary that is a polynomial of
    degree <= p along the side is reproduced exactly at the side's Gauss points; a circle
    is approximated to O(h^(p+1))."""
    from hpb import _lib as L
    t = hpb.basis_tables(p)
    G, sm = p + 1, p - 1
    gx = np.array([[t.gx[k][n] for n in range(t.nmodx)] for k in range(G)])
    x0, x1 = np.array([0.2, 0.1]), np.array([0.9, 0.4])
    xp = np.array([t.xp[k] for k in range(G)])
    chord = np.outer(gx[:, 1], x0) + np.outer(gx[:, 2], x1)
    nrm = np.array([-(x1 - x0)[1], (x1 - x0)[0]])
    curve = chord + np.outer(0.3 * (1 - xp ** 2) * (1 + 0.5 * xp), nrm)  # cubic bump, zero at the ends
    ends = np.ascontiguousarray(np.concatenate([x0, x1])[None])
    modes = np.zeros((1, sm, 2))
    L.check(L.lib().hp_curved_side_modes(ctypes.byref(t), 1, L.ptr(ends), L.ptr(np.ascontiguousarray(curve[None])),
                                         L.ptr(modes)), "curved modes")
    rec = chord + gx[:, 3:3 + sm] @ modes[0]
    if p >= 3:
        assert np.max(np.abs(rec - curve)) < 1e-13
    # circle of radius 1: a side spanning 0.2 rad
    th0, th1 = 0.3, 0.5
    c0, c1 = np.array([np.cos(th0), np.sin(th0)]), np.array([np.cos(th1), np.sin(th1)])
    chord = np.outer(gx[:, 1], c0) + np.outer(gx[:, 2], c1)
    onc = chord / np.linalg.norm(chord, axis=1)[:, None]
    ends = np.ascontiguousarray(np.concatenate([c0, c1])[None])
    L.check(L.lib().hp_curved_side_modes(ctypes.byref(t), 1, L.ptr(ends), L.ptr(np.ascontiguousarray(onc[None])),
                                         L.ptr(modes)), "curved modes")
    rec = chord + gx[:, 3:3 + sm] @ modes[0]
    assert np.max(np.abs(np.linalg.norm(rec, axis=1) - 1.0)) < 0.2 ** (p + 1)


def test_channel_hole_mesh():
    """The graded channel-with-hole mesh: hole points on the circle, all triangles
    counter-clockwise and outside the hole, and its area equals the channel minus the
    inscribed polygon of the hole."""
    m = hpb.channel_hole(L=4.0, H=2.0, cx=1.0, cy=1.0, r=0.25, hmin=0.08, hmax=0.3, grade=0.2)
    assert np.all(m.area2() > 0)
    bs = m.boundary_segments()
    mid = 0.5 * (m.pnts[m.seg_pnt[bs, 0]] + m.pnts[m.seg_pnt[bs, 1]])
    hole = np.hypot(mid[:, 0] - 1.0, mid[:, 1] - 1.0) < 0.25 + 1e-9
    ends = m.pnts[m.seg_pnt[bs[hole]].ravel()]
    assert np.max(np.abs(np.hypot(ends[:, 0] - 1.0, ends[:, 1] - 1.0) - 0.25)) < 1e-12
    k = hole.sum()
    poly = 0.5 * k * 0.25 ** 2 * np.sin(2 * np.pi / k)
    assert abs(0.5 * np.sum(m.area2()) - (8.0 - poly)) < 1e-9

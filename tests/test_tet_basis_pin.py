"""The tet basis tables and dense operators (hp_tet_basis_build) against the
reference's own tet_basis compiled here (oracle/_ref/libtet_basis_ref.so):
1D tables of initialize_values / ptvalues_deriv, and the dense F / DX / DY / DZ /
w and derivative operators against the reference's sum-factorised proj, intgrt,
intgrtrst and derivr / derivs / derivt (tet_basis/proj.cpp, intgrt.cpp)."""
import ctypes

import numpy as np
import pytest

from hpb import tet as TB
from oracle import oracle as O

needs_ref = pytest.mark.skipif(O.ref_tet() is None, reason="oracle/_ref not built (reference tree absent)")


def ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@needs_ref
@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_tet_tables_match_reference(p):
    r = O.ref_tet()
    t = TB.tables(p)
    sz = np.zeros(10, np.int32)
    assert r.ref_tet_sizes(p, ptr(sz)) == 0
    assert list(sz) == [t.p, t.em, t.fm, t.im, t.bm, t.T, t.nmodx, t.nmody, t.nmodz, t.G]
    buf = np.zeros(4096)
    for name in ("gx", "dgx", "gy", "dgy", "gz", "dgz", "wtx", "wty", "wtz", "xp", "yp", "zp", "x0", "y0", "y1",
                 "z0", "dltx", "dlty", "dltz", "dltx2", "dltx3", "dlty2", "dlty3", "dltz2"):
        n = r.ref_tet_get(p, name.encode(), ptr(buf))
        mine = TB.arr(t, name)
        assert n == mine.size, name
        assert rel(mine.ravel(), buf[:n]) < 1e-13, name


@needs_ref
@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_tet_dense_operators_match_reference_sum_factorisation(p):
    r = O.ref_tet()
    t = TB.tables(p)
    G, T = t.G, t.T
    Q = G ** 3
    F, DX, DY, DZ, w = (TB.arr(t, n) for n in ("F", "DX", "DY", "DZ", "w"))
    rng = np.random.default_rng(p)
    for _ in range(3):
        lin = rng.uniform(-1, 1, T)
        f, dx, dy, dz = (np.zeros(Q) for _ in range(4))
        r.ref_tet_proj(p, ptr(lin), ptr(f), ptr(dx), ptr(dy), ptr(dz))
        assert rel(F @ lin, f) < 1e-13
        assert rel(DX @ lin, dx) < 1e-13
        assert rel(DY @ lin, dy) < 1e-13
        assert rel(DZ @ lin, dz) < 1e-13
        g = [rng.uniform(-1, 1, Q) for _ in range(3)]
        res = np.zeros(T)
        r.ref_tet_intgrt(p, ptr(res), ptr(g[0]))
        assert rel(F.T @ (w * g[0]), res) < 1e-13
        res = np.zeros(T)
        r.ref_tet_intgrtrst(p, ptr(res), ptr(g[0]), ptr(g[1]), ptr(g[2]))
        mine = -(DX.T @ (w * g[0]) + DY.T @ (w * g[1]) + DZ.T @ (w * g[2]))  # intgrtrst subtracts
        assert rel(mine, res) < 1e-13
        for d in range(3):
            out = np.zeros(Q)
            r.ref_tet_deriv(p, d, ptr(g[d]), ptr(out))
            assert rel(TB.deriv(t, d, g[d]), out) < 1e-13, d


@needs_ref
@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_tet_face_operators_match_reference_proj2d_intgrt2d(p):
    """Dense face operators F2 / DX2 / DY2 / W2 against tet_basis::proj2d and intgrt2d."""
    r = O.ref_tet()
    t = TB.tables(p)
    G, T2 = t.G, t.T2
    assert T2 == 3 + 3 * t.em + t.fm
    F2, DX2, DY2, W2 = (TB.arr(t, n) for n in ("F2", "DX2", "DY2", "W2"))
    rng = np.random.default_rng(10 + p)
    for _ in range(3):
        lin = rng.uniform(-1, 1, T2)
        f, dx, dy = (np.zeros(G * G) for _ in range(3))
        assert r.ref_tet_proj2d(p, ptr(lin), ptr(f), ptr(dx), ptr(dy)) == 0
        assert rel(F2 @ lin, f) < 1e-13
        assert rel(DX2 @ lin, dx) < 1e-13
        assert rel(DY2 @ lin, dy) < 1e-13
        g = rng.uniform(-1, 1, G * G)
        res = np.zeros(T2)
        assert r.ref_tet_intgrt2d(p, ptr(res), ptr(g)) == 0
        assert rel(F2.T @ (W2 * g), res) < 1e-13


@needs_ref
@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_tet_mass_matrix_and_lumped_vertex_inverse_match_reference_lumpinv(p):
    r = O.ref_tet()
    t = TB.tables(p)
    buf = np.zeros(4096)
    n = r.ref_tet_get(p, b"mm", ptr(buf))
    assert n == t.T * t.T
    assert rel(TB.arr(t, "mm").ravel(), buf[:n]) < 1e-13
    assert r.ref_tet_get(p, b"vdiag", ptr(buf)) == 1
    assert abs(t.vdiag - buf[0]) < 1e-11 * abs(buf[0])
    if p >= 2:
        n = r.ref_tet_get(p, b"sfmv", ptr(buf))
        assert n == 2 * t.em
        assert rel(TB.arr(t, "sfmv").ravel(), buf[:n]) < 1e-11
    if p >= 3:
        n = r.ref_tet_get(p, b"ffmv", ptr(buf))
        assert n == 3 * t.fm
        assert rel(TB.arr(t, "ffmv").ravel(), buf[:n]) < 1e-11


@needs_ref
def test_tet_edge_cone_tables_match_reference_lumpinv():
    """p = 3: ffms, sfms(0), mdiag and odiag of lumpinv's edge-cone systems (the tables of
    tet_hp::minvrt's vertex-ball edge solve and of tet_hp::spoke)."""
    r = O.ref_tet()
    t = TB.tables(3)
    buf = np.zeros(64)
    n = r.ref_tet_get(3, b"ffms", ptr(buf))
    assert n == 3 * t.fm * 2
    assert rel(TB.arr(t, "ffms").ravel(), buf[:n]) < 1e-11
    for name in ("sfms0", "mdiag", "odiag"):
        assert r.ref_tet_get(3, (b"sfms" if name == "sfms0" else name.encode()), ptr(buf)) == 1
        assert abs(getattr(t, name) - buf[0]) < 1e-11 * abs(buf[0]), name

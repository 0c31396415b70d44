"""Coarse h-level meshes by edge collapse (hpb.coarsen.coarsen2, after tri_mesh::coarsen2,
tri_mesh/coarsen.cpp:248-282, with yaber / bdry_yaber, collapse and swap): valid
counter-clockwise triangulations of the same polygonal domain whose vertices are fine
vertices, the ends of every boundary group kept, the boundary chains about halved, and the
reference's work-list order (tri_mesh/adapt.cpp:263-314). The mesh files of the reference are
read when HP_REFERENCE_DIR names its checkout."""
import os

import numpy as np
import pytest

from hpb.coarsen import _OrderedList, coarsen2
from hpb.mesh import channel_hole, delaunay_square, min_angles, read_grd, square_mesh

REF_DIR = os.environ.get("HP_REFERENCE_DIR")


def _check(fine, c, straight=True):
    assert np.all(c.area2() > 0)
    if straight:  # polygonal boundary made of straight chains: the domain is unchanged
        assert abs(c.area2().sum() - fine.area2().sum()) < 1e-9 * fine.area2().sum()
    fv = c.fine_vertex
    assert np.all(fv >= 0) and len(set(fv.tolist())) == len(fv)
    assert np.all(c.pnts == fine.pnts[fv])
    # coarse boundary vertices are fine boundary vertices
    fb = set(fine.seg_pnt[fine.boundary_segments()].ravel().tolist())
    cb = set(fv[c.seg_pnt[c.boundary_segments()].ravel()].tolist())
    assert cb <= fb


def test_work_list_keeps_the_reference_insertion_order():
    wl = _OrderedList()
    for t in range(6):
        wl.put(t, 1.0)
    # equal keys: each new one goes second, so the order is t1, t5, t4, t3, t2, t0
    assert [k[2] for k in wl.sl] == [1, 5, 4, 3, 2, 0]
    assert wl.top() == 0
    wl = _OrderedList()
    for t, v in enumerate([2.0, 1.0, 3.0, 2.0, 1.0]):
        wl.put(t, v)
    assert [k[2] for k in wl.sl] == [1, 4, 3, 0, 2]
    wl.take(2)
    assert wl.top() == 0 and len(wl) == 4 and 2 not in wl


def test_structured_square():
    m = square_mesh(16)
    c = coarsen2(m)
    _check(m, c)
    corners = {0, 16, 16 * 17, 17 * 17 - 1}
    assert corners <= set(c.fine_vertex.tolist())
    assert m.npnt / 6 < c.npnt < m.npnt / 3
    assert 28 <= len(c.boundary_segments()) <= 36
    assert min_angles(c).min() > 15.0
    c2 = coarsen2(m)  # deterministic
    assert np.array_equal(c.tri_pnt, c2.tri_pnt) and np.array_equal(c.fine_vertex, c2.fine_vertex)


def test_delaunay_and_holed_meshes():
    for m, straight in ((delaunay_square(30, seed=5), True), (channel_hole(hmin=0.1, hmax=0.6, grade=0.03), False)):
        c = coarsen2(m)
        _check(m, c, straight)
        assert c.ntri < 0.45 * m.ntri
        assert min_angles(c).min() > 12.0
        assert len(c.boundary_segments()) < 0.7 * len(m.boundary_segments())


def test_larger_factor_removes_more_vertices():
    """The target spacing is factor x the fine spacing: a larger factor keeps fewer vertices."""
    m = square_mesh(24)
    c = coarsen2(m, factor=2.0)
    c3 = coarsen2(m, factor=3.0)
    assert c3.npnt < c.npnt < m.npnt


@pytest.mark.skipif(not REF_DIR, reason="HP_REFERENCE_DIR (reference checkout) not set")
@pytest.mark.parametrize("k", [4, 7])
def test_reference_grd_meshes_coarsen2_with_their_groups(k):
    g = read_grd(os.path.join(REF_DIR, f"Testing/tri_hp/ins/Spatial Accuracy/Inputs/square{k}.grd"))
    c = coarsen2(g)
    _check(g, c)
    assert set(c.groups) == set(g.groups)
    # the group ends stay
    for gid, segs in g.groups.items():
        ends = {int(g.seg_pnt[s, 0]) for s in segs} ^ {int(g.seg_pnt[s, 1]) for s in segs}
        assert ends <= set(c.fine_vertex.tolist())


@pytest.mark.skipif(not REF_DIR, reason="HP_REFERENCE_DIR (reference checkout) not set")
@pytest.mark.parametrize("rel", ["Testing/tri_hp/conv-diff/Correctness/Inputs/tim.0.grd",
                                 "Testing/tri_hp/conv-diff/Correctness/Inputs/tim.1.grd",
                                 "Testing/tri_mesh/wind phased/Inputs/wind_b0.grd",
                                 "Testing/tri_hp/ins/Time Accuracy/Taylor/Inputs/square32.grd"])
def test_reference_test_meshes_coarsen2(rel):
    """The reference's own test meshes (holes, curved and grouped boundaries): valid coarse
    meshes whose every boundary side keeps the group of the fine side it starts on."""
    g = read_grd(os.path.join(REF_DIR, rel))
    c = coarsen2(g)
    assert np.all(c.area2() > 0)
    fv = c.fine_vertex
    assert np.all(c.pnts == g.pnts[fv])
    assert c.ntri < g.ntri
    if g.groups:
        assert set(c.groups) == set(g.groups)
        flat = sorted(s for segs in c.groups.values() for s in segs)
        assert flat == sorted(c.boundary_segments().tolist())


def test_build_rejects_an_unknown_coarsening_route():
    import hpb
    from hpb import multigrid as MG

    def mk(n=8, p=2, mesh=None, **kw):
        return hpb.kovasznay_ins(n=n, p=p, mesh=mesh, **kw)

    with pytest.raises(ValueError, match="coarsen_method"):
        MG.build(mk, n=8, p=2, hlevels=1, coarsen=2.0, coarsen_method="collapse")

"""Coarse h-level meshes from a fine mesh (hpb.coarsen, after tri_mesh::coarsen,
tri_mesh/coarsen.cpp:10-220): valid counter-clockwise triangulations of the same domain,
every other boundary vertex kept per boundary chain (with the reference's midpoint for an
odd number of sides), interior vertices kept by the spacing rule, and the file's boundary
groups carried over. The mesh files of the reference are read when HP_REFERENCE_DIR names
its checkout."""
import os

import numpy as np
import pytest

from hpb.coarsen import _chain_keep, boundary_chains, coarsen
from hpb.mesh import channel_hole, delaunay_square, min_angles, read_grd, square_mesh

REF_DIR = os.environ.get("HP_REFERENCE_DIR")


def _check_valid(fine, c):
    assert np.all(c.area2() > 0)
    # same domain: the coarse triangles cover the fine mesh's area (straight boundaries)
    assert abs(c.area2().sum() - fine.area2().sum()) < 1e-9 * fine.area2().sum()
    # every coarse vertex is a fine vertex or a boundary side's midpoint
    fv = c.fine_vertex
    assert np.all(np.linalg.norm(c.pnts[fv >= 0] - fine.pnts[fv[fv >= 0]], axis=1) == 0.0)


@pytest.mark.parametrize("ns,expect", [(8, [0, 2, 4, 6, 8]), (7, [0, 2, None, 5, 7]), (1, [0, 1]), (2, [0, 2]),
                                       (5, [0, None, 5])])
def test_chain_keeps_every_other_vertex_with_the_odd_midpoint(ns, expect):
    verts = list(range(ns + 1))
    P = np.stack([np.arange(ns + 1, dtype=float), np.zeros(ns + 1)], axis=1)
    keep, mid = _chain_keep(verts, P)
    assert keep == expect
    if None in keep:
        assert mid[0] == ns // 2 + 0.5


def test_structured_square_halves_every_direction():
    m = square_mesh(16)
    c = coarsen(m, 1.5)
    _check_valid(m, c)
    assert c.ntri == 128 and c.npnt == 81
    assert min_angles(c).min() > 44.9
    chains = boundary_chains(m)
    assert len(chains) == 4 and all(len(v) == 17 for _, v in chains)
    assert len(c.boundary_segments()) == 32


def test_delaunay_and_holed_meshes():
    for m in (delaunay_square(20, seed=3), channel_hole(hmin=0.1, hmax=0.5)):
        c = coarsen(m, 1.5)
        assert np.all(c.area2() > 0)
        assert c.ntri < 0.4 * m.ntri
        assert min_angles(c).min() > 15.0
        # each boundary loop keeps about half its sides
        assert abs(len(c.boundary_segments()) - len(m.boundary_segments()) / 2) <= 4


@pytest.mark.skipif(not REF_DIR, reason="HP_REFERENCE_DIR (reference checkout) not set")
@pytest.mark.parametrize("k", [4, 7])
def test_reference_grd_meshes_coarsen_with_their_groups(k):
    g = read_grd(os.path.join(REF_DIR, f"Testing/tri_hp/ins/Spatial Accuracy/Inputs/square{k}.grd"))
    c = coarsen(g, 1.5)
    _check_valid(g, c)
    assert set(c.groups) == set(g.groups)
    for gid in g.groups:
        assert len(c.groups[gid]) * 2 == len(g.groups[gid])

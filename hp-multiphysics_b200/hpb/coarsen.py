"""Coarse meshes for the h-levels of the multigrid, made from a fine mesh.

This follows tri_mesh::coarsen (tri_mesh/coarsen.cpp:10-220), which builds a p = 1 coarse
level from any fine mesh:

* Every fine vertex v gets a spacing fltwk(v): `factor` times the length of its shortest
  edge (coarsen.cpp:22-34).
* Each boundary chain keeps every other vertex: its two end points always; for an even
  number of sides the vertices 2, 4, ...; for an odd number the vertices 2, 4, ... up to
  the middle, the midpoint of the middle side, and the alternate vertices of the second
  half (coarsen.cpp:47-152). A boundary chain is a group of the mesh file
  (`mesh.groups`, as read_grd returns them), or else a piece of a boundary loop between
  corners where the boundary turns by more than `corner_deg`.
* Interior vertices are taken in index order. A vertex joins the coarse mesh when its
  distance to the nearest vertex already in it is at least its fltwk (coarsen.cpp:192-205).
* The coarse vertices are triangulated. The reference inserts them one by one
  (Bowyer-Watson) into the triangulation of its boundary. Here the Delaunay triangulation of
  the set is kept where it lies inside the fine mesh, and every coarse boundary side must be
  one of its edges (checked).

tri_mesh::coarsen2 (coarsen.cpp:248-282), the other route, coarsens by collapsing
short edges of a copy of the fine mesh. It belongs to the mesh-adaptation machinery
(yaber, collapse, swap), which is out of scope here.
"""
import numpy as np

from .mesh import Mesh


def boundary_chains(mesh, corner_deg=30.0):
    """Ordered boundary chains [(group id, [vertex indices along the chain])]: the file's
    groups when the mesh has them, else each boundary loop split at its corners. Sides run
    with the domain on their left (createsegtri's orientation of boundary sides)."""
    b = mesh.boundary_segments()
    nxt = {}
    for s in b:
        nxt[int(mesh.seg_pnt[s, 0])] = int(s)
    groups = getattr(mesh, "groups", None)
    seg_group = {}
    if groups:
        for gid, segs in groups.items():
            for s in segs:
                seg_group[int(s)] = int(gid)
    P = mesh.pnts
    seen = set()
    chains = []
    for s0 in b:
        s0 = int(s0)
        if s0 in seen:
            continue
        loop = []  # sides of one boundary loop in order
        s = s0
        while s not in seen:
            seen.add(s)
            loop.append(s)
            s = nxt[int(mesh.seg_pnt[s, 1])]

        def breaks_before(i):
            sa, sb = loop[i - 1], loop[i]
            if groups:
                return seg_group.get(sa, -1) != seg_group.get(sb, -1)
            a = P[mesh.seg_pnt[sa, 1]] - P[mesh.seg_pnt[sa, 0]]
            c = P[mesh.seg_pnt[sb, 1]] - P[mesh.seg_pnt[sb, 0]]
            cosang = np.dot(a, c) / (np.linalg.norm(a) * np.linalg.norm(c))
            return cosang < np.cos(np.radians(corner_deg))

        cuts = [i for i in range(len(loop)) if breaks_before(i)]
        if not cuts:  # a smooth loop: one chain from an arbitrary start, closed
            cuts = [0]
        for k, c in enumerate(cuts):
            e = cuts[(k + 1) % len(cuts)]
            sides = loop[c:e] if e > c else loop[c:] + loop[:e]
            verts = [int(mesh.seg_pnt[sides[0], 0])] + [int(mesh.seg_pnt[s, 1]) for s in sides]
            chains.append((seg_group.get(sides[0], -1), verts))
    return chains


def _chain_keep(verts, P):
    """Coarse vertices of one boundary chain (coarsen.cpp:47-152): (kept fine indices in
    order, with None where the midpoint of the middle side is inserted), and that midpoint."""
    ns = len(verts) - 1
    out = [verts[0]]
    mid = None
    if ns % 2:
        j = 2
        while j < ns // 2:
            out.append(verts[j])
            j += 2
        if ns > 1:
            j = ns // 2
            mid = 0.5 * (P[verts[j]] + P[verts[j + 1]])
            out.append(None)
        j = ns - ((ns - 2) // 4) * 2
        while j < ns:
            out.append(verts[j])
            j += 2
    else:
        for j in range(2, ns, 2):
            out.append(verts[j])
    out.append(verts[-1])
    return out, mid


def coarsen(mesh, factor=1.5, corner_deg=30.0):
    """The coarse mesh of `mesh` (a hpb.mesh.Mesh) after tri_mesh::coarsen. Returns a Mesh
    whose `groups` give the group id of every coarse boundary chain's sides (when the fine
    mesh has groups) and whose `fine_vertex` maps each coarse vertex to the fine vertex it
    came from (-1 for inserted midpoints)."""
    from scipy.spatial import Delaunay

    from .multigrid import locate

    P = mesh.pnts
    # spacing per fine vertex: factor x its shortest edge
    ln = np.linalg.norm(P[mesh.seg_pnt[:, 0]] - P[mesh.seg_pnt[:, 1]], axis=1)
    fltwk = np.full(mesh.npnt, np.inf)
    np.minimum.at(fltwk, mesh.seg_pnt[:, 0], ln)
    np.minimum.at(fltwk, mesh.seg_pnt[:, 1], ln)
    fltwk *= factor

    chains = boundary_chains(mesh, corner_deg)
    coarse_of = {}  # fine vertex -> coarse vertex
    pts, fine_vertex = [], []

    def add(xy, fv):
        pts.append(np.asarray(xy, dtype=np.float64))
        fine_vertex.append(fv)
        return len(pts) - 1

    chain_coarse = []
    for gid, verts in chains:
        keep, mid = _chain_keep(verts, P)
        cv = []
        for v in keep:
            if v is None:
                cv.append(add(mid, -1))
            elif v in coarse_of:
                cv.append(coarse_of[v])
            else:
                coarse_of[v] = add(P[v], v)
                cv.append(coarse_of[v])
        chain_coarse.append((gid, cv))
    on_bdry = np.zeros(mesh.npnt, bool)
    for _, verts in chains:
        on_bdry[verts] = True

    # interior vertices in index order, kept when no coarse vertex lies within their spacing
    h = float(np.max(fltwk[np.isfinite(fltwk)])) if np.any(np.isfinite(fltwk)) else 1.0
    lo = P.min(axis=0)
    grid = {}

    def cell(xy):
        return (int((xy[0] - lo[0]) // h), int((xy[1] - lo[1]) // h))

    for k, xy in enumerate(pts):
        grid.setdefault(cell(xy), []).append(k)
    for v in range(mesh.npnt):
        if on_bdry[v]:
            continue
        xy = P[v]
        cx, cy = cell(xy)
        r2 = fltwk[v] * fltwk[v]
        near = False
        for i in (cx - 1, cx, cx + 1):
            for j in (cy - 1, cy, cy + 1):
                for k in grid.get((i, j), ()):
                    d = pts[k] - xy
                    if d[0] * d[0] + d[1] * d[1] < r2:
                        near = True
                        break
                if near:
                    break
            if near:
                break
        if not near:
            k = add(xy, v)
            coarse_of[v] = k
            grid.setdefault((cx, cy), []).append(k)

    X = np.array(pts)
    tri = Delaunay(X).simplices.astype(np.int64)
    # keep the triangles inside the fine mesh, counter-clockwise
    cen = X[tri].mean(axis=1)
    tloc, _ = locate(mesh, cen, strict=False)
    tri = tri[tloc >= 0]
    a = X[tri]
    area2 = (a[:, 1, 0] - a[:, 0, 0]) * (a[:, 2, 1] - a[:, 0, 1]) - (a[:, 1, 1] - a[:, 0, 1]) * (a[:, 2, 0] - a[:, 0, 0])
    tri[area2 < 0] = tri[area2 < 0][:, [0, 2, 1]]
    cm = Mesh(X, tri.astype(np.int32))
    # every coarse boundary side is a boundary side of the triangulation
    bset = {(int(cm.seg_pnt[s, 0]), int(cm.seg_pnt[s, 1])) for s in cm.boundary_segments()}
    groups = {}
    for gid, cv in chain_coarse:
        for a_, b_ in zip(cv[:-1], cv[1:]):
            if (a_, b_) not in bset:
                raise ValueError(f"coarse boundary side ({a_}, {b_}) is not an edge of the triangulation")
        if gid >= 0:
            ids = [s for s in cm.boundary_segments()
                   if (int(cm.seg_pnt[s, 0]), int(cm.seg_pnt[s, 1])) in set(zip(cv[:-1], cv[1:]))]
            groups.setdefault(gid, []).extend(int(s) for s in ids)
    if len(bset) != sum(len(cv) - 1 for _, cv in chain_coarse):
        raise ValueError("the triangulation has boundary sides that no coarse boundary chain owns")
    cm.groups = groups
    cm.fine_vertex = np.array(fine_vertex, dtype=np.int64)
    return cm

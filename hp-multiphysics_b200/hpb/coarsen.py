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

tri_mesh::coarsen2 (coarsen.cpp:248-282), the other route and the reference's default for
its multigrid levels, coarsens by collapsing short edges of a copy of the fine mesh (yaber,
collapse, swap): `coarsen2` below.
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


# ---------------------------------------------------------------------------------------------
# tri_mesh::coarsen2 (tri_mesh/coarsen.cpp:248-282): coarsening by edge collapse.
#
# The coarse mesh is the fine one with vertices removed: a target spacing lngth = factor x the
# fine spacing (initlngth, setup.cpp:257-296: the mean incident edge length, the shortest
# adjacent boundary side on boundaries, then two harmonic smoothing passes, meshutilities.cpp:
# 355-400) is imposed first on every boundary chain (bdry_yaber, yaber.cpp:334-455) and then in
# the interior (yaber, yaber.cpp:25-240). Each removal collapses one side into one of its end
# vertices (collapse.cpp:5-183) and re-swaps the sides around the kept vertex for the larger
# minimum angle (swap.cpp:21-123). Vertices never move, so the coarse vertices are fine ones.
#
# Work lists are kept in the reference's insertion order (adapt.cpp:263-299: ascending key,
# a new entry goes before the entries equal to it, except that one equal to the first entry
# of a list of two or more goes second), so that structured meshes, full of equal keys,
# coarsen in the same order. The connectivity follows the reference's conventions (side j of
# a triangle opposite vertex j, seg.tri(0) the triangle for which the side runs
# counter-clockwise), including which of two merged sides survives a collapse and which
# triangle each vertex refers to, since the order of the ring walks depends on it.
# ---------------------------------------------------------------------------------------------
import math as _math

_EPS = float(np.finfo(np.float64).eps)
_FLT_EPSILON = float(np.finfo(np.float32).eps)


class _OrderedList:
    """The reference's sorted work list (putinlst / tkoutlst with USE_PRIORITY_QUEUE): items
    by ascending value; the largest is taken first."""

    def __init__(self):
        from sortedcontainers import SortedList
        self.sl = SortedList()
        self.key = {}
        self.cnt = 0

    def __len__(self):
        return len(self.sl)

    def __contains__(self, item):
        return item in self.key

    def put(self, item, value):
        self.cnt += 1
        if len(self.sl) >= 2 and self.sl[0][0] == value:
            # goes second: above the first entry, below every other entry of the same value
            first = self.sl[0]
            self.sl.remove(first)
            nf = (first[0], -self.cnt - 0.5, first[2])
            self.sl.add(nf)
            self.key[first[2]] = nf
        k = (value, -self.cnt, item)
        self.sl.add(k)
        self.key[item] = k
        return k

    def take(self, item):
        k = self.key.pop(item, None)
        if k is not None:
            self.sl.remove(k)
        return k

    def top(self):
        return self.sl[-1][2]


class _AdaptMesh:
    """A triangle mesh under collapse and swap, in the reference's arrays: tri.pnt/seg/sgn/tri,
    seg.pnt/tri, pnt.tri (Python lists; deleted entities are flagged, removed at the end)."""

    def __init__(self, mesh):
        self.x = [tuple(p) for p in mesh.pnts.tolist()]
        self.tp = mesh.tri_pnt.tolist()
        self.ts = mesh.tri_seg.tolist()
        self.tg = mesh.tri_sgn.tolist()
        self.sp = mesh.seg_pnt.tolist()
        self.st = mesh.seg_tri.tolist()
        nt = len(self.tp)
        self.tt = [[-1, -1, -1] for _ in range(nt)]
        for t in range(nt):
            for j in range(3):
                s = self.ts[t][j]
                a, b = self.st[s]
                self.tt[t][j] = b if a == t else a
        self.ptri = [0] * len(self.x)
        for t in range(nt):  # createpnttri: the last triangle of each vertex
            for v in self.tp[t]:
                self.ptri[v] = t
        self.tdel = [False] * nt
        self.sdel = [False] * len(self.sp)
        self.pdel = [False] * len(self.x)
        self.touched = set()  # triangles whose connectivity changed in the last operation

    def dist(self, a, b):
        pa, pb = self.x[a], self.x[b]
        return _math.hypot(pa[0] - pb[0], pa[1] - pb[1])

    def area(self, t):  # twice the signed area (tprims.cpp:66-80)
        p0, p1, p2 = (self.x[v] for v in self.tp[t])
        dx1, dy1 = p0[0] - p2[0], p0[1] - p2[1]
        dx2, dy2 = p1[0] - p0[0], p1[1] - p0[1]
        return dx1 * dy2 - dy1 * dx2

    def area_sp(self, s, p2):  # twice the signed area of side s and vertex p2 (tprims.cpp:51-64)
        p0, p1 = self.x[self.sp[s][0]], self.x[self.sp[s][1]]
        q = self.x[p2]
        dx1, dy1 = p0[0] - q[0], p0[1] - q[1]
        dx2, dy2 = p1[0] - p0[0], p1[1] - p0[1]
        return dx1 * dy2 - dy1 * dx2

    def inradius(self, t):  # tprims.cpp:224-241: 2 area / perimeter
        p0, p1, p2 = (self.x[v] for v in self.tp[t])
        dx1, dy1 = p0[0] - p2[0], p0[1] - p2[1]
        dx2, dy2 = p1[0] - p0[0], p1[1] - p0[1]
        a = dx1 * dy2 - dy1 * dx2
        per = _math.hypot(dx1, dy1) + _math.hypot(dx2, dy2) + _math.hypot(dx1 + dx2, dy1 + dy2)
        return a / per

    def minangle(self, a, b, c):
        """Sine of the angle opposite the shortest side, signed (tprims.cpp:116-141)."""
        pa, pb, pc = self.x[a], self.x[b], self.x[c]
        dx = (pc[0] - pb[0], pa[0] - pc[0], pb[0] - pa[0])
        dy = (pc[1] - pb[1], pa[1] - pc[1], pb[1] - pa[1])
        ln = [dx[k] * dx[k] + dy[k] * dy[k] for k in range(3)]
        i = 0 if ln[0] < ln[1] else 1
        i = i if ln[i] < ln[2] else 2
        i1, i2 = (i + 1) % 3, (i + 2) % 3
        cross = -dx[i2] * dy[i1] + dy[i2] * dx[i1]
        return cross / _math.sqrt(ln[i1] * ln[i2])

    def ring(self, v, exclude):
        """Triangles around v other than `exclude`, and the sides between two of them that
        touch v, in the reference's walk order: counter-clockwise from pnt.tri, then, at a
        boundary, clockwise from pnt.tri (collapse.cpp:14-54)."""
        tind = self.ptri[v]
        prev = 0 if tind not in exclude else 1
        stop = tind
        d = 1
        tris, spokes = [], []
        for _ in range(2 * len(self.tp) + 2):  # a walk longer than the mesh is a broken ring
            vn = self.tp[tind].index(v)
            t1 = self.tt[tind][(vn + d) % 3]
            if t1 < 0:
                if d > 1:
                    break
                d += 1
                t1 = self.ptri[v]
                prev = 1
                stop = -1
            if t1 not in exclude:
                tris.append(t1)
                if not prev:
                    spokes.append(self.ts[tind][(vn + d) % 3])
                prev = 0
            else:
                prev = 1
            tind = t1
            if tind == stop:
                break
        else:
            raise RuntimeError(f"coarsen2: the triangles around vertex {v} do not close")
        return tris, spokes

    def collapse(self, sind, delt):
        """Removes vertex seg.pnt(delt) of side sind into the other end (collapse.cpp:5-183).
        Returns the triangles that surrounded the removed vertex."""
        p1 = self.sp[sind][delt]
        p0 = self.sp[sind][1 - delt]
        adj = tuple(self.st[sind])
        tris, spokes = self.ring(p1, adj)
        self.touched = set(tris)
        for t in tris:
            j = self.tp[t].index(p1)
            self.tp[t][j] = p0
            s3 = self.ts[t][(j + 1) % 3]
            self.sp[s3][(1 + self.tg[t][(j + 1) % 3]) // 2] = p0
            s3 = self.ts[t][(j + 2) % 3]
            self.sp[s3][(1 - self.tg[t][(j + 2) % 3]) // 2] = p0
        self.sdel[sind] = True
        for t in adj:
            if t < 0:
                continue
            self.tdel[t] = True
            sd1 = self.tp[t].index(p1)
            sd2 = (sd1 + 2) % 3 if self.ts[t][(sd1 + 1) % 3] == sind else (sd1 + 1) % 3
            s1 = self.ts[t][sd2]
            if self.st[s1][1] < 0:  # a boundary side survives: delete the other one
                if self.sp[s1][0] == p1:
                    self.sp[s1][0] = p0
                if self.sp[s1][1] == p1:
                    self.sp[s1][1] = p0
                sd1, sd2 = sd2, sd1
                s1 = self.ts[t][sd2]
            self.sdel[s1] = True
            t1, t2 = self.tt[t][sd1], self.tt[t][sd2]
            if t1 > -1:
                self.tt[t1][self.tt[t1].index(t)] = t2
                for v in self.tp[t]:
                    self.ptri[v] = t1
                self.touched.add(t1)
            kept = self.ts[t][sd1]
            self.st[kept][(1 - self.tg[t][sd1]) // 2] = t2
            if t2 > -1:
                j = self.tt[t2].index(t)
                self.tt[t2][j] = t1
                self.ts[t2][j] = kept
                self.tg[t2][j] = self.tg[t][sd1]
                for v in self.tp[t]:
                    self.ptri[v] = t2
                self.touched.add(t2)
        self.pdel[p1] = True
        self.swap_list(spokes)
        return tris

    def swap(self, sind, tol=0.0):
        """Swaps side sind when that raises the smaller minimum angle of its two triangles
        (swap.cpp:21-123)."""
        t1, t2 = self.st[sind]
        if t1 < 0 or t2 < 0:
            return 0
        n1 = self.ts[t1].index(sind)
        n2 = self.ts[t2].index(sind)
        p0, p1 = self.sp[sind]
        v1, v2 = self.tp[t1][n1], self.tp[t2][n2]
        if min(self.minangle(p0, p1, v1), self.minangle(p1, p0, v2)) > \
                min(self.minangle(v2, v1, p0), self.minangle(v1, v2, p1)) - tol - 10.0 * _EPS:
            return 0
        self.sp[sind] = [v2, v1]
        self.tp[t1][(n1 + 2) % 3] = v2
        self.tp[t2][(n2 + 2) % 3] = v1
        s1p, s2p = (n1 + 1) % 3, (n2 + 1) % 3
        self.ts[t1][n1], self.tg[t1][n1], self.tt[t1][n1] = self.ts[t2][s2p], self.tg[t2][s2p], self.tt[t2][s2p]
        self.ts[t2][n2], self.tg[t2][n2], self.tt[t2][n2] = self.ts[t1][s1p], self.tg[t1][s1p], self.tt[t1][s1p]
        for t, n in ((t1, n1), (t2, n2)):
            s1 = self.ts[t][n]
            self.st[s1][(1 - self.tg[t][n]) // 2] = t
            tn = self.tt[t][n]
            if tn > -1:
                self.tt[tn][self.ts[tn].index(s1)] = t
                self.touched.add(tn)
        self.ptri[p0] = t1
        self.ptri[p1] = t2
        self.tt[t1][s1p] = t2
        self.tt[t2][s2p] = t1
        self.ts[t1][s1p] = sind
        self.ts[t2][s2p] = sind
        self.tg[t1][s1p] = 1
        self.tg[t2][s2p] = -1
        self.touched.update((t1, t2))
        return 1

    def swap_list(self, sides, tol=0.0):
        while True:
            n = 0
            for s in sides:
                n += self.swap(s, tol)
            if n == 0:
                break


def _grouped_chains(mesh, corner_deg):
    """Boundary chains as ordered side lists with their group: the file's groups (each group's
    sides put in chain order, a group may hold several chains) or boundary_chains' pieces."""
    groups = getattr(mesh, "groups", None)
    out = []
    if groups:
        for gid, segs in groups.items():
            segs = [int(s) for s in segs]
            by_start = {int(mesh.seg_pnt[s, 0]): s for s in segs}
            ends = {int(mesh.seg_pnt[s, 1]) for s in segs}
            left = set(segs)
            starts = [s for s in segs if int(mesh.seg_pnt[s, 0]) not in ends]
            while left:
                s = next((x for x in starts if x in left), None)
                if s is None:
                    s = next(x for x in segs if x in left)  # a closed loop
                chain = []
                while s is not None and s in left:
                    chain.append(s)
                    left.discard(s)
                    s = by_start.get(int(mesh.seg_pnt[s, 1]))
                out.append((gid, chain, chain and int(mesh.seg_pnt[chain[-1], 1]) == int(mesh.seg_pnt[chain[0], 0])))
        return out
    b = {(int(mesh.seg_pnt[s, 0]), int(mesh.seg_pnt[s, 1])): int(s) for s in mesh.boundary_segments()}
    for gid, verts in boundary_chains(mesh, corner_deg):
        chain = [b[(a, c)] for a, c in zip(verts[:-1], verts[1:])]
        out.append((gid, chain, verts[0] == verts[-1]))
    return out


def coarsen2(mesh, factor=2.0, tolsize=1.414, corner_deg=30.0):
    """The coarse mesh of `mesh` after tri_mesh::coarsen2(factor) (coarsen.cpp:248-282; the
    reference's default for its multigrid h-levels, connect.cpp:10-30, with factor 2). Returns
    a Mesh with `fine_vertex` (the fine vertex of every coarse vertex) and `groups`."""
    am = _AdaptMesh(mesh)
    npnt = len(am.x)
    # initlngth (setup.cpp:257-296) and smooth_lngth(2) (meshutilities.cpp:355-400)
    nnb = [0] * npnt
    ln = [0.0] * npnt
    for a, b in am.sp:
        d = am.dist(a, b)
        ln[a] += d
        ln[b] += d
        nnb[a] += 1
        nnb[b] += 1
    ln = [ln[v] / nnb[v] if nnb[v] else 0.0 for v in range(npnt)]
    chains = _grouped_chains(mesh, corner_deg)
    for _, chain, _ in chains:
        for s in chain:
            ln[am.sp[s][0]] = 1.0e32
    for _, chain, _ in chains:
        for s in chain:
            a, b = am.sp[s]
            d = am.dist(a, b)
            ln[a] = min(d, ln[a])
            ln[b] = min(d, ln[b])
    for _ in range(2):
        acc = [0.0] * npnt
        for a, b in am.sp:
            acc[a] += 1.0 / ln[b]
            acc[b] += 1.0 / ln[a]
        ln = [1.0 / (acc[v] / nnb[v]) if nnb[v] else ln[v] for v in range(npnt)]
    ln = [factor * x for x in ln]
    # setup_for_adapt (adapt.cpp:104-130): the ends of every boundary group stay
    spec = [False] * npnt
    for _, chain, _ in chains:
        if chain:
            spec[am.sp[chain[0]][0]] = True
            spec[am.sp[chain[-1]][1]] = True

    def side_ratio(s):
        a, b = am.sp[s]
        return min(ln[a], ln[b]) / am.dist(a, b)

    # bdry_yaber (yaber.cpp:334-455): every other boundary vertex, chain by chain
    for _, chain, closed in chains:
        n = len(chain)
        if n == 0:
            continue
        nxt = {chain[k]: chain[(k + 1) % n] if (closed or k + 1 < n) else -1 for k in range(n)}
        prv = {chain[k]: chain[k - 1] if (closed or k > 0) else -1 for k in range(n)}
        fl = {}
        wl = _OrderedList()
        for s in chain:
            if am.sdel[s]:
                continue
            fl[s] = side_ratio(s)
            if fl[s] > tolsize:
                wl.put(s, fl[s])
        while len(wl):
            s = wl.top()
            sn, sp_ = nxt[s], prv[s]
            a, b = am.sp[s]
            if spec[a] and spec[b]:
                wl.take(s)
                continue
            if spec[a]:
                endpt, saffect = 1, sn
            elif spec[b]:
                endpt, saffect = 0, sp_
            elif fl.get(sp_, 0.0) > fl.get(sn, 0.0):
                endpt, saffect = 0, sp_
            else:
                endpt, saffect = 1, sn
            ring = am.collapse(s, endpt)
            wl.take(s)
            if sn >= 0:
                prv[sn] = sp_
            if sp_ >= 0:
                nxt[sp_] = sn
            wl.take(saffect)
            fl[saffect] = side_ratio(saffect)
            if fl[saffect] > tolsize:
                wl.put(saffect, fl[saffect])
            # an interior vertex left on the wrong side of the moved boundary side goes too
            bad = []
            for t in ring:
                if am.tdel[t] or am.area(t) > 0.0:
                    continue
                for v in am.tp[t]:
                    if v in am.sp[saffect]:
                        continue
                    if am.area_sp(saffect, v) < _FLT_EPSILON:
                        bad.append(v)
            for v in bad:
                if am.pdel[v]:
                    continue
                t = am.ptri[v]
                vn = am.tp[t].index(v)
                am.collapse(am.ts[t][(vn + 1) % 3], 1)
    # yaber (yaber.cpp:25-240): the interior
    tol = tolsize * 6.0 / _math.sqrt(3.0)
    for _, chain, _ in chains:
        for s in chain:
            if not am.sdel[s]:
                spec[am.sp[s][0]] = True
    ntri = len(am.tp)
    fw = [0.0] * ntri
    wl = _OrderedList()
    qual = __import__("sortedcontainers").SortedList()  # keys of listed triangles next to an unlisted one
    inq = {}

    def qualifies(t):
        return any(n < 0 or n not in wl for n in am.tt[t])

    def requal(t):
        k = inq.pop(t, None)
        if k is not None:
            qual.remove(k)
        if t in wl and not am.tdel[t] and qualifies(t):
            k = wl.key[t]
            qual.add(k)
            inq[t] = k

    def put(t):
        first = wl.sl[0] if len(wl) >= 2 else None
        wl.put(t, fw[t])
        if first is not None and wl.key[first[2]] != first:  # the first entry was re-keyed
            f = first[2]
            if f in inq:
                qual.remove(inq[f])
                inq[f] = wl.key[f]
                qual.add(inq[f])

    def take(t):
        wl.take(t)
        k = inq.pop(t, None)
        if k is not None:
            qual.remove(k)

    def classify(t):
        fw[t] = min(ln[v] for v in am.tp[t]) / am.inradius(t)
        if fw[t] > tol:
            put(t)

    for t in range(ntri):
        if not am.tdel[t]:
            classify(t)
    for t in range(ntri):
        requal(t)
    while len(wl):
        tind = qual[-1][2] if len(qual) else wl.top()
        take(tind)
        for n in am.tt[tind]:
            if n >= 0:
                requal(n)
        best, sind = 0.0, -1
        for j in range(3):
            s = am.ts[tind][j]
            if am.st[s][1] < 0:
                continue
            r = side_ratio(s)
            if r > best:
                best, sind = r, s
        if sind < 0:
            continue
        for t in am.st[sind]:
            if t >= 0 and t in wl:
                take(t)
                for n in am.tt[t]:
                    if n >= 0:
                        requal(n)
        a, b = am.sp[sind]
        if spec[a] and spec[b]:
            continue
        if spec[a] or spec[b]:
            endpt = 1 if spec[a] else 0
        else:
            # keep the end nearer the area centre of the two ends' triangles
            cx = cy = asum = 0.0
            adj = tuple(am.st[sind])
            for e in (0, 1):
                tris, _ = am.ring(am.sp[sind][e], adj)
                te = am.st[sind][e]
                for t in ([te] if te > -1 else []) + tris:
                    ar = am.area(t)
                    asum += ar
                    for v in am.tp[t]:
                        cx += ar * am.x[v][0]
                        cy += ar * am.x[v][1]
            asum = 1.0 / (3.0 * asum)
            cx *= asum
            cy *= asum
            l0 = (am.x[a][0] - cx) ** 2 + (am.x[a][1] - cy) ** 2
            l1 = (am.x[b][0] - cx) ** 2 + (am.x[b][1] - cy) ** 2
            endpt = 0 if l0 > l1 else 1
        ring = am.collapse(sind, endpt)
        changed = set(am.touched)
        for t in ring:
            if t in wl:
                take(t)
            classify(t)
        for t in changed | set(ring):
            if am.tdel[t]:
                continue
            requal(t)
            for n in am.tt[t]:
                if n >= 0:
                    requal(n)
    # cleanup_after_adapt: drop the deleted entities, keep the survivors' order
    keep_p = [v for v in range(npnt) if not am.pdel[v]]
    pmap = {v: k for k, v in enumerate(keep_p)}
    tris = [[pmap[v] for v in am.tp[t]] for t in range(ntri) if not am.tdel[t]]
    X = np.array([am.x[v] for v in keep_p], dtype=np.float64)
    cm = Mesh(X, np.array(tris, dtype=np.int32))
    cm.fine_vertex = np.array(keep_p, dtype=np.int64)
    # boundary groups of the coarse sides: a coarse boundary side replaces the run of fine
    # boundary sides from its first vertex along the chain, so it takes the group of the fine
    # side that starts there (boundary sides run with the domain on their left)
    groups = {}
    fine_groups = getattr(mesh, "groups", None)
    if fine_groups:
        gid_of = {int(sd): gid for gid, segs in fine_groups.items() for sd in segs}
        start = {int(mesh.seg_pnt[sd, 0]): int(sd) for sd in mesh.boundary_segments()}
        for sd in cm.boundary_segments():
            a = int(cm.fine_vertex[cm.seg_pnt[sd, 0]])
            g = gid_of.get(start.get(a, -1))
            if g is not None:
                groups.setdefault(g, []).append(int(sd))
    cm.groups = groups
    return cm

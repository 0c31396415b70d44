"""Triangle meshes in the reference's array form (tri_mesh/tri_mesh.h:46-98).

* ``square_mesh(n)``: [0,1]^2 split into n x n squares, each cut into two
  counter-clockwise right triangles along the diagonal from the square's
  upper-left to its lower-right corner -- the triangulation of the reference's
  Testing/tri_hp/ins/Spatial Accuracy/Inputs/square<k>.grd meshes
  (square7.grd = 64 x 64 squares = 8,192 triangles).
* ``delaunay_square(n, seed)``: a seeded Delaunay triangulation of the unit
  square with about 2 n^2 triangles and a checked minimum angle.
* ``channel_hole(...)``: a graded Delaunay mesh of a channel with a circular hole
  (its hole sides are made curved by the workload's boundary curve).
* ``read_grd(path)``: the reference's .grd text format (tri_mesh/input.cpp:504-600).
* ``createsegtri``: segment/triangle connectivity with the reference's
  conventions (tri_mesh/setup.cpp:76-145): tri.seg(j) is the side opposite
  tri.pnt(j), tri.sgn(j) = +1 when the segment runs counter-clockwise for the
  triangle, seg.tri(0) is that triangle, seg.tri(1) the other one (-1 on the
  boundary). Segments are numbered in order of first appearance.
"""
import numpy as np


class Mesh:
    def __init__(self, pnts, tri_pnt, seg_pnt=None):
        self.pnts = np.ascontiguousarray(pnts, dtype=np.float64)
        self.tri_pnt = np.ascontiguousarray(tri_pnt, dtype=np.int32)
        self.npnt = len(self.pnts)
        self.ntri = len(self.tri_pnt)
        createsegtri(self, seg_pnt)

    def boundary_segments(self):
        return np.nonzero(self.seg_tri[:, 1] < 0)[0].astype(np.int32)

    def area2(self):
        """2 x triangle area (tri_mesh/tprims.cpp:66-80)."""
        p = self.pnts[self.tri_pnt]
        dx1 = p[:, 0, 0] - p[:, 2, 0]
        dy1 = p[:, 0, 1] - p[:, 2, 1]
        dx2 = p[:, 1, 0] - p[:, 0, 0]
        dy2 = p[:, 1, 1] - p[:, 0, 1]
        return dx1 * dy2 - dy1 * dx2


def createsegtri(m, seg_pnt=None):
    """Builds seg_pnt/seg_tri and tri_seg/tri_sgn (tri_mesh/setup.cpp:76-145).

    With seg_pnt given (a mesh file's segment list) the file's segment numbering
    and orientation are kept, as the reference does; otherwise segments are
    created in order of first appearance, oriented counter-clockwise for the
    first triangle that lists them.
    """
    t = m.tri_pnt
    nt = m.ntri
    # side j of a triangle runs from pnt((j+1)%3) to pnt((j+2)%3)
    a = np.stack([t[:, 1], t[:, 2], t[:, 0]], axis=1).reshape(-1)
    b = np.stack([t[:, 2], t[:, 0], t[:, 1]], axis=1).reshape(-1)
    lo = np.minimum(a, b).astype(np.int64)
    hi = np.maximum(a, b).astype(np.int64)
    key = lo * (m.npnt + 1) + hi
    if seg_pnt is None:
        ukey, first, inv = np.unique(key, return_index=True, return_inverse=True)
        order = np.argsort(first, kind="stable")  # number segments by first appearance
        rank = np.empty_like(order)
        rank[order] = np.arange(len(order))
        sid = rank[inv]
        fo = first[order]
        seg_pnt = np.stack([a[fo], b[fo]], axis=1)
    else:
        seg_pnt = np.asarray(seg_pnt, dtype=np.int64)
        skey = np.minimum(seg_pnt[:, 0], seg_pnt[:, 1]) * (m.npnt + 1) + np.maximum(seg_pnt[:, 0], seg_pnt[:, 1])
        srt = np.argsort(skey)
        pos = np.searchsorted(skey[srt], key)
        if np.any(pos >= len(srt)) or np.any(skey[srt][np.minimum(pos, len(srt) - 1)] != key):
            raise ValueError("triangle side without a matching segment")
        sid = srt[pos]
    nseg = len(seg_pnt)
    sgn = np.where(seg_pnt[sid, 0] == a, 1, -1)
    seg_tri = -np.ones((nseg, 2), dtype=np.int64)
    tri_of_side = np.repeat(np.arange(nt), 3)
    slot = np.where(sgn > 0, 0, 1)
    if np.any(np.bincount(sid * 2 + slot, minlength=2 * nseg) > 1):
        raise ValueError("non-manifold or inconsistently oriented mesh")
    seg_tri[sid, slot] = tri_of_side
    m.nseg = nseg
    m.seg_pnt = np.ascontiguousarray(seg_pnt, dtype=np.int32)
    m.seg_tri = np.ascontiguousarray(seg_tri, dtype=np.int32)
    m.tri_seg = np.ascontiguousarray(sid.reshape(nt, 3), dtype=np.int32)
    m.tri_sgn = np.ascontiguousarray(sgn.reshape(nt, 3), dtype=np.int32)
    # a boundary segment must be counter-clockwise for its triangle (outward normal
    # to its right, as hp_edge_bdry::element_rsdl assumes)
    bnd = m.seg_tri[:, 0] < 0
    if np.any(bnd):
        raise ValueError("boundary segment oriented clockwise for its triangle")
    return m


def splitmix64_uniform(seed, n):
    """n doubles in [-1, 1) from the splitmix64 sequence started at `seed`."""
    mask = np.uint64(0xFFFFFFFFFFFFFFFF)
    with np.errstate(over="ignore"):
        k = np.arange(1, n + 1, dtype=np.uint64)
        z = (np.uint64(seed) + k * np.uint64(0x9E3779B97F4A7C15)) & mask
        z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & mask
        z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & mask
        z = z ^ (z >> np.uint64(31))
    u = (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    return 2.0 * u - 1.0


def delaunay_square(n, seed=20261205, jitter=0.12, margin=0.7, min_angle=20.0):
    """Seeded Delaunay triangulation of the unit square with about 2 n^2 triangles
    (the split-square mesh's count) and uniform vertex density: a hexagonal lattice of
    spacing h = sqrt(2/sqrt(3))/n whose points are jittered by splitmix64 uniforms of
    +-jitter*h, interior points kept at least margin*h from the boundary, boundary
    points evenly spaced at about h, triangulated by scipy's Delaunay (Qhull) and
    oriented counter-clockwise; vertices and triangles are numbered along a Z-curve, as a
    mesh generator's renumbering pass would. Raises if the smallest angle is below
    min_angle degrees."""
    from scipy.spatial import Delaunay
    h = np.sqrt(2.0 / np.sqrt(3.0)) / n
    m = int(np.ceil(1.0 / h))
    s = np.linspace(0.0, 1.0, m + 1)[:-1]
    z, o = np.zeros(m), np.ones(m)
    bnd = np.concatenate([np.stack([s, z], 1), np.stack([o, s], 1), np.stack([1 - s, o], 1), np.stack([z, 1 - s], 1)])
    dy = h * np.sqrt(3.0) / 2.0
    rows = []
    for j in range(int(np.ceil(1.0 / dy)) + 2):
        xs = np.arange(-1, int(1.0 / h) + 2) * h + (0.5 * h if j % 2 else 0.0)
        rows.append(np.stack([xs, np.full_like(xs, j * dy)], 1))
    pts = np.concatenate(rows)
    pts = pts + jitter * h * splitmix64_uniform(seed, pts.size).reshape(pts.shape)
    keep = np.all((pts > margin * h) & (pts < 1.0 - margin * h), axis=1)
    pts = np.concatenate([bnd, pts[keep]])
    pts = pts[np.argsort(morton_key(pts), kind="stable")]  # vertices numbered along a Z-curve
    tri = Delaunay(pts).simplices.astype(np.int64)
    tri = tri[np.argsort(morton_key(pts[tri].mean(axis=1)), kind="stable")]  # triangles too
    a = pts[tri]
    ar = (a[:, 1, 0] - a[:, 0, 0]) * (a[:, 2, 1] - a[:, 0, 1]) - (a[:, 1, 1] - a[:, 0, 1]) * (a[:, 2, 0] - a[:, 0, 0])
    tri[ar < 0] = tri[ar < 0][:, [0, 2, 1]]
    mesh = Mesh(pts, tri)
    mesh.min_angle = float(min_angles(mesh).min())
    if mesh.min_angle < min_angle:
        raise ValueError(f"Delaunay mesh min angle {mesh.min_angle:.2f} < {min_angle}")
    return mesh


def channel_hole(L=20.0, H=10.0, cx=5.0, cy=5.0, r=0.5, hmin=0.02, hmax=0.2, grade=0.0085, seed=20261207,
                 jitter=0.05, margin=0.6, min_angle=15.0):
    """Graded Delaunay mesh of the channel [0,L] x [0,H] with a circular hole of radius r
    at (cx, cy). Local edge length h(d) = min(hmax, hmin + grade * d), d the distance
    from the hole. Points: rings around the hole at radius steps h*sqrt(3)/2 holding
    2*pi*radius/h points each (alternate rings offset by half a spacing; the first ring
    on the circle itself), ring points closer than margin*h to a wall dropped, the walls
    sampled at the local h; interior points jittered by splitmix64 uniforms of
    +-jitter*h; Qhull Delaunay, triangles inside the hole removed, counter-clockwise,
    Z-curve numbering. Defaults: ~150k triangles. Raises below min_angle degrees."""
    from scipy.spatial import Delaunay

    def hf(d):
        return np.minimum(hmax, hmin + grade * np.maximum(d, 0.0))

    rings = []
    rk, k = r, 0
    rmax = np.hypot(max(cx, L - cx), max(cy, H - cy))
    while rk < rmax + hmax:
        h = float(hf(rk - r))
        n = max(8, int(round(2.0 * np.pi * rk / h)))
        th = (np.arange(n) + 0.5 * (k % 2)) * 2.0 * np.pi / n
        rings.append(np.stack([cx + rk * np.cos(th), cy + rk * np.sin(th)], 1))
        rk += h * np.sqrt(3.0) / 2.0
        k += 1
    n0 = len(rings[0])
    pts = np.concatenate(rings)
    d = np.hypot(pts[:, 0] - cx, pts[:, 1] - cy) - r
    hp = hf(d)
    jit = jitter * hp[:, None] * splitmix64_uniform(seed, pts.size).reshape(pts.shape)
    jit[:n0] = 0.0  # the hole's own points stay on the circle
    pts = pts + jit
    wall = np.minimum(np.minimum(pts[:, 0], L - pts[:, 0]), np.minimum(pts[:, 1], H - pts[:, 1]))
    keep = np.arange(len(pts)) < n0
    keep |= wall > margin * hp
    pts = pts[keep]
    walls = []
    for (x0, y0, x1, y1) in ((0.0, 0.0, L, 0.0), (L, 0.0, L, H), (L, H, 0.0, H), (0.0, H, 0.0, 0.0)):
        seg = np.hypot(x1 - x0, y1 - y0)
        ts, t = [0.0], 0.0
        while True:
            x, y = x0 + (x1 - x0) * t / seg, y0 + (y1 - y0) * t / seg
            step = float(hf(np.hypot(x - cx, y - cy) - r))
            t += step
            if t >= seg - 0.3 * step:
                break
            ts.append(t)
        ts = np.array(ts)
        walls.append(np.stack([x0 + (x1 - x0) * ts / seg, y0 + (y1 - y0) * ts / seg], 1))
    pts = np.concatenate([pts] + walls)
    span = max(L, H)
    pts = pts[np.argsort(morton_key(pts / span), kind="stable")]
    tri = Delaunay(pts).simplices.astype(np.int64)
    cen = pts[tri].mean(axis=1)
    tri = tri[np.hypot(cen[:, 0] - cx, cen[:, 1] - cy) > r]
    a = pts[tri]
    ar = (a[:, 1, 0] - a[:, 0, 0]) * (a[:, 2, 1] - a[:, 0, 1]) - (a[:, 1, 1] - a[:, 0, 1]) * (a[:, 2, 0] - a[:, 0, 0])
    tri[ar < 0] = tri[ar < 0][:, [0, 2, 1]]
    tri = tri[np.argsort(morton_key(pts[tri].mean(axis=1) / span), kind="stable")]
    used = np.unique(tri)
    remap = np.full(len(pts), -1, dtype=np.int64)
    remap[used] = np.arange(len(used))
    mesh = Mesh(pts[used], remap[tri])
    mesh.min_angle = float(min_angles(mesh).min())
    mesh.hole = (cx, cy, r)
    mesh.box = (L, H)
    if mesh.min_angle < min_angle:
        raise ValueError(f"channel mesh min angle {mesh.min_angle:.2f} < {min_angle}")
    return mesh


def morton_key(xy, bits=16):
    """Z-order (Morton) key of points in the unit square: neighbouring keys are nearby
    points, so arrays numbered by it keep an element's gathers close in memory."""
    q = np.clip((np.asarray(xy) * (1 << bits)).astype(np.int64), 0, (1 << bits) - 1)
    key = np.zeros(len(q), dtype=np.int64)
    for b in range(bits):
        key |= ((q[:, 0] >> b) & 1) << (2 * b)
        key |= ((q[:, 1] >> b) & 1) << (2 * b + 1)
    return key


def min_angles(mesh):
    """Smallest interior angle (degrees) of every triangle."""
    a = mesh.pnts[mesh.tri_pnt]
    out = np.full(mesh.ntri, 180.0)
    for k in range(3):
        u = a[:, (k + 1) % 3] - a[:, k]
        v = a[:, (k + 2) % 3] - a[:, k]
        c = np.sum(u * v, axis=1) / (np.linalg.norm(u, axis=1) * np.linalg.norm(v, axis=1))
        out = np.minimum(out, np.degrees(np.arccos(np.clip(c, -1.0, 1.0))))
    return out


def square_mesh(n, x0=0.0, x1=1.0, y0=0.0, y1=1.0, ny=None):
    """n x ny squares (ny = n by default), two counter-clockwise triangles each (diagonal
    upper-left to lower-right)."""
    ny = n if ny is None else ny
    xs = np.linspace(x0, x1, n + 1)
    ys = np.linspace(y0, y1, ny + 1)
    X, Y = np.meshgrid(xs, ys)  # [j][i]
    pnts = np.stack([X.ravel(), Y.ravel()], axis=1)
    I, J = np.meshgrid(np.arange(n), np.arange(ny))
    I = I.ravel()
    J = J.ravel()
    va = J * (n + 1) + I
    vb = va + 1
    vd = va + (n + 1)
    vc = vd + 1
    t1 = np.stack([va, vb, vd], axis=1)
    t2 = np.stack([vb, vc, vd], axis=1)
    tri = np.stack([t1, t2], axis=1).reshape(-1, 3)
    return Mesh(pnts, tri)


def read_grd(path):
    """Reads the reference's .grd format: header 'nvrtx: N nside: S ntri: T', then
    N vertex lines 'k: x y', S side lines 'k: p0 p1', T triangle lines 'k: a b c'
    (tri_mesh/input.cpp:504-600). Boundary groups are returned as
    {idnum: [segment indices]}."""
    with open(path) as f:
        lines = f.read().split("\n")
    hdr = lines[0].replace(":", " ").split()
    nv, ns, nt = int(hdr[1]), int(hdr[3]), int(hdr[5])
    pts = np.array([[float(x) for x in l.split(":")[1].split()[:2]] for l in lines[1:1 + nv]])
    segs = np.array([[int(x) for x in l.split(":")[1].split()[:2]] for l in lines[1 + nv:1 + nv + ns]])
    tris = np.array([[int(x) for x in l.split(":")[1].split()[:3]] for l in lines[1 + nv + ns:1 + nv + ns + nt]])
    groups = {}
    k = 1 + nv + ns + nt
    if k < len(lines) and lines[k].startswith("nsbd"):
        nsbd = int(lines[k].split(":")[1])
        k += 1
        for _ in range(nsbd):
            idnum = int(lines[k].split(":")[1])
            num = int(lines[k + 1].split(":")[1])
            ids = [int(l.split(":")[1].split()[0]) for l in lines[k + 2:k + 2 + num]]
            groups.setdefault(idnum, []).extend(ids)
            k += 2 + num
    m = Mesh(pts, tris, seg_pnt=segs)
    m.groups = groups
    return m

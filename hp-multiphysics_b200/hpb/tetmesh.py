"""Tetrahedral meshes with the reference's conventions (tet_mesh/setup.cpp).

cube_tets(n): the unit cube (or a box) split into n^3 hexahedra of 6 tetrahedra
each (the 6 tetrahedra around each hexahedron's main diagonal, conforming across
hexahedra). Connectivity follows tet_mesh:
  * reorient_tets (setup.cpp:14-96): v0 the lowest vertex index, v1 the second
    lowest, v2 / v3 ordered so that -((v1-v0) x (v2-v0)) . (v3-v0) > 0; vol is that
    triple product's magnitude (6 x the tetrahedron's volume);
  * create_seg_from_tet (setup.cpp:142-211): local edge i joins local vertices
    VS[i]; edges are numbered in order of first appearance (tetrahedra in order,
    local edges in order), take that first tetrahedron's direction, and sgn is -1
    where a tetrahedron runs the edge the other way;
  * create_tri_from_tet (setup.cpp:301-374): local face i has local vertices VF[i]
    (face i is opposite vertex i); faces are numbered in order of first appearance
    with that tetrahedron's vertex order, rot = +1 there and -1 in the second
    tetrahedron.
"""
import numpy as np

VS = np.array([[2, 3], [3, 1], [2, 1], [1, 0], [2, 0], [3, 0]])
VF = np.array([[1, 3, 2], [0, 2, 3], [0, 3, 1], [0, 1, 2]])


class TetMesh:
    def __init__(self, pnts, tet_pnt):
        self.pnts = np.ascontiguousarray(pnts, dtype=np.float64)
        self.npnt = len(self.pnts)
        self._reorient(np.asarray(tet_pnt, dtype=np.int64))
        self._edges()
        self._faces()

    def _reorient(self, tp):
        tp = np.sort(tp, axis=1)
        P = self.pnts
        a = P[tp[:, 1]] - P[tp[:, 0]]
        b = P[tp[:, 2]] - P[tp[:, 0]]
        c = P[tp[:, 3]] - P[tp[:, 0]]
        vol = -np.einsum("ij,ij->i", np.cross(a, b), c)
        neg = vol < 0
        tp[neg, 2], tp[neg, 3] = tp[neg, 3].copy(), tp[neg, 2].copy()
        if np.any(np.abs(vol) <= 1e-14 * np.max(np.abs(vol))):
            raise ValueError("degenerate tetrahedron")
        self.tet_pnt = np.ascontiguousarray(tp, dtype=np.int32)
        self.vol = np.ascontiguousarray(np.abs(vol))
        self.ntet = len(tp)

    def _number(self, keys):
        """Ids in order of first appearance, and the position of each first appearance."""
        uniq, first, inv = np.unique(keys, return_index=True, return_inverse=True)
        order = np.argsort(first, kind="stable")
        rank = np.empty(len(uniq), dtype=np.int64)
        rank[order] = np.arange(len(uniq))
        return rank[inv], first[order]

    def _edges(self):
        tp = self.tet_pnt.astype(np.int64)
        ev = tp[:, VS]                       # (ntet, 6, 2) in creation order
        flat = ev.reshape(-1, 2)
        n = self.npnt
        key = np.minimum(flat[:, 0], flat[:, 1]) * n + np.maximum(flat[:, 0], flat[:, 1])
        ids, first = self._number(key)
        self.seg_pnt = np.ascontiguousarray(flat[first], dtype=np.int32)
        self.nseg = len(first)
        self.tet_seg = np.ascontiguousarray(ids.reshape(-1, 6), dtype=np.int32)
        same = flat[:, 0] == self.seg_pnt[ids, 0]
        self.tet_sgn = np.ascontiguousarray(np.where(same, 1, -1).reshape(-1, 6), dtype=np.int32)

    def _faces(self):
        tp = self.tet_pnt.astype(np.int64)
        fv = tp[:, VF].reshape(-1, 3)
        s = np.sort(fv, axis=1)
        n = self.npnt
        key = (s[:, 0] * n + s[:, 1]) * n + s[:, 2]
        ids, first = self._number(key)
        self.tri_pnt = np.ascontiguousarray(fv[first], dtype=np.int32)
        self.ntri = len(first)
        self.tet_tri = np.ascontiguousarray(ids.reshape(-1, 4), dtype=np.int32)
        pos = np.arange(len(fv))
        is_first = np.zeros(len(fv), bool)
        is_first[first] = True
        self.tet_rot = np.ascontiguousarray(np.where(is_first, 1, -1).reshape(-1, 4), dtype=np.int32)
        tri_tet = np.full((self.ntri, 2), -1, dtype=np.int32)
        tri_tet[ids[is_first], 0] = pos[is_first] // 4
        tri_tet[ids[~is_first], 1] = pos[~is_first] // 4
        self.tri_tet = tri_tet

    def boundary_faces(self):
        return np.nonzero(self.tri_tet[:, 1] < 0)[0].astype(np.int32)

    def face_edges(self, faces):
        """Edges of the given faces in the face's own frame: face edge i lies opposite face
        vertex i and runs from face vertex (i+1)%3 to (i+2)%3 (the edge order of
        tet_basis::proj2d, tet_basis/proj2d.cpp:46-91, and of tet_mesh/refineby2.cpp:142-145);
        sgn = +1 where the global edge runs that way. Returns seg, sgn [nface][3]."""
        faces = np.asarray(faces, dtype=np.int64)
        a = self.tri_pnt[faces].astype(np.int64)
        n = self.npnt
        s0 = self.seg_pnt[:, 0].astype(np.int64)
        s1 = self.seg_pnt[:, 1].astype(np.int64)
        skey = np.minimum(s0, s1) * n + np.maximum(s0, s1)
        order = np.argsort(skey)
        seg = np.empty((len(faces), 3), np.int32)
        sgn = np.empty((len(faces), 3), np.int32)
        for i in range(3):
            b, c = a[:, (i + 1) % 3], a[:, (i + 2) % 3]
            key = np.minimum(b, c) * n + np.maximum(b, c)
            pos = order[np.searchsorted(skey, key, sorter=order)]
            if np.any(skey[pos] != key):
                raise ValueError("face edge missing from the edge list")
            seg[:, i] = pos
            sgn[:, i] = np.where(s0[pos] == b, 1, -1)
        return seg, sgn

    def boundary_entities(self, faces=None):
        """Vertices, edges and faces on the given boundary faces (default: all):
        each face's local edges are found in its tetrahedron (the edges whose two
        local vertices both lie on the face)."""
        faces = self.boundary_faces() if faces is None else np.asarray(faces)
        t = self.tri_tet[faces, 0]
        loc = np.argmax(self.tet_tri[t] == faces[:, None], axis=1)
        verts = np.unique(self.tri_pnt[faces].ravel())
        on = np.zeros((len(faces), 4), bool)
        on[np.arange(len(faces))[:, None], VF[loc]] = True
        edge_on = on[:, VS[:, 0]] & on[:, VS[:, 1]]          # (nf, 6)
        edges = np.unique(self.tet_seg[t][edge_on])
        return verts, edges, np.unique(faces)


def read_msh(path):
    """Reads a Gmsh 2.x ASCII mesh (the format of the reference's tet test meshes, which it
    reads through MAdLib): $Nodes 'id x y z', $Elements 'id type ntags tags... nodes' with
    type 4 = tetrahedron and type 2 = boundary triangle. Returns (TetMesh, groups), groups
    {elementary entity id (the second tag, the id the reference's input keys b0_f<id>
    name): array of global face indices}."""
    with open(path) as f:
        lines = [ln.strip() for ln in f]
    k = 0
    nodes, tets, tris = {}, [], []
    while k < len(lines):
        if lines[k] == "$Nodes":
            n = int(lines[k + 1])
            for ln in lines[k + 2:k + 2 + n]:
                a = ln.split()
                nodes[int(a[0])] = (float(a[1]), float(a[2]), float(a[3]))
            k += n + 2
        elif lines[k] == "$Elements":
            n = int(lines[k + 1])
            for ln in lines[k + 2:k + 2 + n]:
                a = [int(x) for x in ln.split()]
                typ, nt = a[1], a[2]
                tags, vs = a[3:3 + nt], a[3 + nt:]
                if typ == 4:
                    tets.append(vs[:4])
                elif typ == 2:
                    tris.append((tags[1] if nt > 1 else tags[0], vs[:3]))
            k += n + 2
        else:
            k += 1
    if not tets:
        raise ValueError(f"{path}: no tetrahedra (type 4 elements)")
    ids = sorted(nodes)
    index = {nid: i for i, nid in enumerate(ids)}
    pnts = np.array([nodes[i] for i in ids])
    mesh = TetMesh(pnts, np.array([[index[v] for v in t] for t in tets]))
    fk = np.sort(mesh.tri_pnt.astype(np.int64), axis=1)
    n = mesh.npnt
    fkey = (fk[:, 0] * n + fk[:, 1]) * n + fk[:, 2]
    order = np.argsort(fkey)
    groups = {}
    for ent, vs in tris:
        t = sorted(index[v] for v in vs)
        key = (t[0] * n + t[1]) * n + t[2]
        pos = order[np.searchsorted(fkey, key, sorter=order)]
        if fkey[pos] != key:
            raise ValueError("boundary triangle is not a face of the mesh")
        groups.setdefault(ent, []).append(pos)
    return mesh, {g: np.array(v, dtype=np.int32) for g, v in groups.items()}


def cube_tets(n, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0)):
    """[lo, hi] box, n^3 hexahedra x 6 tetrahedra around each main diagonal."""
    g = [np.linspace(lo[d], hi[d], n + 1) for d in range(3)]
    X, Y, Z = np.meshgrid(*g, indexing="ij")
    pnts = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    idx = lambda i, j, k: (i * (n + 1) + j) * (n + 1) + k
    i, j, k = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    corner = lambda b: idx(i + (b & 1), j + ((b >> 1) & 1), k + ((b >> 2) & 1))
    tets = []
    for a1, a2 in ((1, 2), (1, 4), (2, 1), (2, 4), (4, 1), (4, 2)):
        tets.append(np.stack([corner(0), corner(a1), corner(a1 | a2), corner(7)], axis=1))
    tp = np.stack(tets, axis=1).reshape(-1, 4)
    return TetMesh(pnts, tp)

"""Multigrid hierarchies over the GPU contexts (block::cycle with p- and
h-levels, tri_mesh/blocks.cpp:1267-1348).

p-levels share the fine mesh at a lower polynomial degree (p -> p/2 -> ... -> 1,
as the reference halves log2p; p = 6 goes 6 -> 3 -> 1). h-levels are coarser
meshes at p = 1 whose transfer weights are each point's containing triangle in the
other mesh with barycentric weights, boundary points re-connected along the other
mesh's boundary sides (tri_mesh::mgconnect).
"""
import ctypes

import numpy as np

from . import _lib as L
from .problem import GPULevel

P = ctypes.c_void_p
_bound = False


def _bind():
    global _bound
    lib = L.lib()
    if not _bound:
        lib.hp_gpu_mg_attach_p.argtypes = [P, P, ctypes.c_double]
        lib.hp_gpu_mg_attach_h.argtypes = [P, P, P, P, P, P, ctypes.c_double]
        lib.hp_gpu_mg_restrict.argtypes = [P]
        lib.hp_gpu_mg_prolongate.argtypes = [P]
        lib.hp_gpu_vcycle.argtypes = [ctypes.POINTER(P), ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int]
        lib.hp_gpu_solve_mg_graph.argtypes = [ctypes.POINTER(P), ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                              ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, P,
                                              ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                              ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)]
        lib.hp_gpu_capture_vcycle.argtypes = [ctypes.POINTER(P), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_int, ctypes.c_int, ctypes.POINTER(P)]
        lib.hp_gpu_launch_vcycle.argtypes = [P, P, ctypes.c_int]
        lib.hp_gpu_destroy_vcycle.argtypes = [P]
        lib.hp_gpu_solve_mg_mixed.argtypes = [ctypes.POINTER(P), ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                              ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, P, ctypes.c_int,
                                              ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double),
                                              ctypes.POINTER(ctypes.c_int)]
        lib.hp_gpu_solve_mg.argtypes = [ctypes.POINTER(P), ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_int, ctypes.c_int, ctypes.c_int, P, ctypes.c_int,
                                        ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double),
                                        ctypes.POINTER(ctypes.c_int)]
        _bound = True
    return lib


def barycentric(pnts, tri_pnt, tris, pts):
    """Barycentric weights of points pts[k] in triangles tris[k]."""
    a = pnts[tri_pnt[tris, 0]]
    b = pnts[tri_pnt[tris, 1]]
    c = pnts[tri_pnt[tris, 2]]
    v0, v1, v2 = b - a, c - a, pts - a
    d = v0[:, 0] * v1[:, 1] - v0[:, 1] * v1[:, 0]
    w1 = (v2[:, 0] * v1[:, 1] - v2[:, 1] * v1[:, 0]) / d
    w2 = (v0[:, 0] * v2[:, 1] - v0[:, 1] * v2[:, 0]) / d
    return np.stack([1.0 - w1 - w2, w1, w2], axis=1)


def locate(mesh, pts, strict=True):
    """Containing triangle of each point (tri_mesh::findtri) and its barycentric
    weights (getwgts). Uses a uniform bucket grid over the triangles. strict=False:
    points outside the mesh get triangle -1 and NaN weights instead of an error."""
    pts = np.asarray(pts, dtype=np.float64)
    P_ = mesh.pnts
    T = mesh.tri_pnt
    lo = P_.min(axis=0)
    hi = P_.max(axis=0)
    nb = max(1, int(np.sqrt(mesh.ntri / 2)))
    span = np.maximum(hi - lo, 1e-300)
    tmin = ((P_[T].min(axis=1) - lo) / span * nb).astype(np.int64).clip(0, nb - 1)
    tmax = ((P_[T].max(axis=1) - lo) / span * nb).astype(np.int64).clip(0, nb - 1)
    # (cell, tri) pairs
    cells, tris = [], []
    for di in range(int((tmax - tmin)[:, 0].max()) + 1):
        for dj in range(int((tmax - tmin)[:, 1].max()) + 1):
            ok = (tmin[:, 0] + di <= tmax[:, 0]) & (tmin[:, 1] + dj <= tmax[:, 1])
            t = np.nonzero(ok)[0]
            cells.append((tmin[t, 0] + di) * nb + tmin[t, 1] + dj)
            tris.append(t)
    cells = np.concatenate(cells)
    tris = np.concatenate(tris)
    order = np.argsort(cells, kind="stable")
    cells, tris = cells[order], tris[order]
    start = np.searchsorted(cells, np.arange(nb * nb))
    end = np.searchsorted(cells, np.arange(nb * nb), side="right")
    pc = ((pts - lo) / span * nb).astype(np.int64).clip(0, nb - 1)
    pcell = pc[:, 0] * nb + pc[:, 1]
    best_t = np.full(len(pts), -1, dtype=np.int64)
    best_w = np.full((len(pts), 3), np.nan)
    best_m = np.full(len(pts), -np.inf)
    maxc = int((end - start).max())
    for k in range(maxc):
        idx = start[pcell] + k
        valid = idx < end[pcell]
        if not np.any(valid):
            break
        q = np.nonzero(valid)[0]
        t = tris[idx[q]]
        w = barycentric(P_, T, t, pts[q])
        m = w.min(axis=1)
        better = m > best_m[q]
        qq = q[better]
        best_m[qq] = m[better]
        best_t[qq] = t[better]
        best_w[qq] = w[better]
    if not strict:
        out = (best_t < 0) | (best_m < -1e-6)
        best_t[out] = -1
        best_w[out] = np.nan
    elif np.any(best_t < 0) or np.any(best_m < -1e-6):
        raise ValueError("point outside the mesh")
    return best_t.astype(np.int32), np.ascontiguousarray(best_w)


def boundary_reconnect(src, tgt, t, w, chunk=4096):
    """Boundary points of src re-connected along tgt's boundary sides
    (edge_bdry::mgconnect, tri_mesh/tri_boundary.cpp:164-201, with the side search of
    edge_bdry::findbdrypt, tri_boundary.cpp:95-160): each boundary point takes the
    nearest boundary side of tgt, weights 0.5(1-psi) and 0.5(1+psi) on its end points
    and 0 on the triangle's third vertex; a point beyond the ends of the sides (a
    convex corner) takes the nearer end point. Boundary values, essential conditions
    included, then move between the levels through boundary values only: on a curved
    boundary, whose coarse sides are chords, the containing triangle would also weight
    an interior vertex and every prolongation would move the fine essential values.
    t, w: containing-triangle weights of every src point (locate), updated in place."""
    sb = src.boundary_segments()
    bp = np.unique(src.seg_pnt[sb].ravel())
    tb = tgt.boundary_segments()
    a = tgt.pnts[tgt.seg_pnt[tb, 0]]
    d = tgt.pnts[tgt.seg_pnt[tb, 1]] - a
    l2 = np.einsum("ij,ij->i", d, d)
    for c0 in range(0, len(bp), chunk):
        q = bp[c0:c0 + chunk]
        x = src.pnts[q][:, None, :] - a[None, :, :]
        sv = np.clip(np.einsum("kij,ij->ki", x, d) / l2, 0.0, 1.0)
        r = x - sv[..., None] * d[None, :, :]
        k = np.argmin(np.einsum("kij,kij->ki", r, r), axis=1)
        seg = tb[k]
        s = sv[np.arange(len(q)), k]
        tri = tgt.seg_tri[seg, 0]
        tp = tgt.tri_pnt[tri]
        p0 = tgt.seg_pnt[seg, 0][:, None]
        p1 = tgt.seg_pnt[seg, 1][:, None]
        t[q] = tri
        w[q] = np.where(tp == p0, (1.0 - s)[:, None], 0.0) + np.where(tp == p1, s[:, None], 0.0)
    return t, w


def connect(src, tgt):
    """Transfer weights of every src point in tgt (tri_mesh::mgconnect,
    tri_mesh/connect.cpp:49-86): the containing triangle with barycentric weights,
    then boundary points re-connected along tgt's boundary sides."""
    t, w = locate(tgt, src.pnts)
    return boundary_reconnect(src, tgt, t, w)


class Hierarchy:
    """levels[0] is the finest GPULevel; each next one is attached to the previous."""

    def __init__(self, probs, kinds, stream=None, fadd=1.0):
        lib = _bind()
        self.probs = probs
        if stream is None:
            # one stream for every level: the whole cycle can then be one CUDA graph
            import torch
            self._stream = torch.cuda.Stream()
            stream = ctypes.c_void_p(self._stream.cuda_stream)
        self.levels = [GPULevel(pr, 0, stream) for pr in probs]
        self._keep = []
        for l in range(1, len(probs)):
            c, f = self.levels[l], self.levels[l - 1]
            if kinds[l] == "p":
                L.check(lib.hp_gpu_mg_attach_p(c.h, f.h, fadd), "mg_attach_p")
            else:
                fm, cm = probs[l - 1].mesh, probs[l].mesh
                f2c_t, f2c_w = connect(fm, cm)
                c2f_t, c2f_w = connect(cm, fm)
                self._keep += [f2c_t, f2c_w, c2f_t, c2f_w]
                L.check(lib.hp_gpu_mg_attach_h(c.h, f.h, L.ptr(f2c_t), L.ptr(f2c_w), L.ptr(c2f_t), L.ptr(c2f_w),
                                               fadd), "mg_attach_h")
        self.lib = lib

    def element_matrices(self, on=True):
        """cd: every level's rsdl from stored element operators (hp_gpu_set_element_matrices)."""
        for lv in self.levels:
            lv.element_matrices(on)

    def autotune(self, reps=5):
        """Per-level launch shapes (hp_gpu_autotune on every level); returns them per level."""
        out = []
        for lv in self.levels:
            lv.setup_preconditioner()
            out.append(lv.autotune(reps))
        return out

    def handles(self):
        arr = (P * len(self.levels))(*[lv.h for lv in self.levels])
        return arr

    def solve(self, drop=1e-10, max_cycles=500, vw=1, itercrsn=2, iterrfne=2, prcn_every=1, graph=False,
              check_every=1, mixed=False):
        """Cycles until the FP64 residual drops by `drop`; returns (hist, seconds, cycles).
        Preconditioners are evaluated every `prcn_every` cycles (the reference's
        preconditioner_interval, default 1: blocks.cpp:1170,1492); 0 = first cycle only.
        graph=True replays one captured CUDA graph per cycle (preconditioner set-ups inside
        every prcn_every cycles, frozen when prcn_every = 0);
        mixed=True runs FP32 cycles on the correction equation inside FP64 defect correction."""
        cap = max_cycles + 2
        hist = np.zeros(cap)
        nh = ctypes.c_int(); sec = ctypes.c_double(); nc = ctypes.c_int()
        if mixed:
            L.check(self.lib.hp_gpu_solve_mg_mixed(self.handles(), len(self.levels), drop, max_cycles, vw, itercrsn,
                                                   iterrfne, prcn_every, L.ptr(hist), cap, ctypes.byref(nh),
                                                   ctypes.byref(sec), ctypes.byref(nc)), "solve_mg_mixed")
        elif graph:
            L.check(self.lib.hp_gpu_solve_mg_graph(self.handles(), len(self.levels), drop, max_cycles, vw, itercrsn,
                                                   iterrfne, check_every, prcn_every, L.ptr(hist), cap,
                                                   ctypes.byref(nh), ctypes.byref(sec), ctypes.byref(nc)),
                    "solve_mg_graph")
        else:
            L.check(self.lib.hp_gpu_solve_mg(self.handles(), len(self.levels), drop, max_cycles, vw, itercrsn,
                                             iterrfne, prcn_every, L.ptr(hist), cap, ctypes.byref(nh),
                                             ctypes.byref(sec), ctypes.byref(nc)), "solve_mg")
        return hist[:nh.value], sec.value, nc.value

    def close(self):
        for lv in self.levels:
            lv.close()


def p_sequence(p):
    """p-levels below p: halving (the reference's log2p hierarchy), then 1."""
    seq = []
    q = p
    while q > 1:
        q = max(1, q // 2)
        seq.append(q)
    return seq


def build(factory, n, p, hlevels=0, stream=None, cfl=None, plevels=True, coarsen=None, coarsen_method="coarsen",
          **kw):
    """Hierarchy for a workload factory(n=..., p=...): p-levels of the fine mesh
    down to p = 1 (unless plevels=False: the fine level goes straight to the h-levels,
    as the reference does with extra_finest_levels = 0), then `hlevels` split-square
    meshes of n/2, n/4, ... at p = 1. coarsen = a factor: the h-levels are instead made
    from the level above, through factory(mesh=..., p=1), by hpb.coarsen.coarsen
    (tri_mesh::coarsen, e.g. 1.5) or, with coarsen_method="coarsen2", by
    hpb.coarsen.coarsen2 (tri_mesh::coarsen2, edge collapse; the reference's multigrid
    uses 2.0). cfl: None (the per-log2p defaults), a number, or a dict p -> cfl."""
    def cf(q):
        if cfl is None:
            return {}
        return {"cfl": cfl[q] if isinstance(cfl, dict) else cfl}
    probs = [factory(n=n, p=p, **cf(p), **kw)]
    kinds = ["fine"]
    for q in (p_sequence(p) if plevels else []):
        probs.append(factory(n=n, p=q, **cf(q), **kw))
        kinds.append("p")
    m = n
    for _ in range(hlevels):
        m //= 2
        if coarsen:
            from . import coarsen as C
            if coarsen_method not in ("coarsen", "coarsen2"):
                raise ValueError(f"coarsen_method {coarsen_method!r}: 'coarsen' or 'coarsen2'")
            make = C.coarsen2 if coarsen_method == "coarsen2" else C.coarsen
            probs.append(factory(mesh=make(probs[-1].mesh, coarsen), p=1, **cf(1), **kw))
        else:
            probs.append(factory(n=m, p=1, **cf(1), **kw))
        kinds.append("h")
    return Hierarchy(probs, kinds, stream=stream)

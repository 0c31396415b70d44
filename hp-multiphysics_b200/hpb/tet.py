"""3D (tet_hp) path: tet_basis tables (hp_tet_basis_build) and their dense
operators (include/hp_tet.h)."""
import ctypes

import numpy as np

from . import _lib as L

MAXP, MAXG, MAXT, MAXQ, MAXM = 4, 5, 35, 125, 12
_D, _I = ctypes.c_double, ctypes.c_int


class TetTables(ctypes.Structure):
    _fields_ = ([(n, _I) for n in ("p", "G", "T", "em", "fm", "im", "bm", "nmodx", "nmody", "nmodz")] +
                [(n, _D * MAXM * MAXG) for n in ("gx", "dgx", "gy", "dgy", "gz", "dgz")] +
                [(n, _D * MAXG) for n in ("wtx", "wty", "wtz", "xp", "yp", "zp", "x0", "y0", "y1", "z0",
                                          "dltx", "dlty", "dltz")] +
                [(n, _D * MAXG * MAXG) for n in ("dltx2", "dltx3", "dlty2", "dlty3", "dltz2")] +
                [(n, _I * MAXT) for n in ("mx", "my", "mz")] + [("msg", _D * MAXT), ("w", _D * MAXQ)] +
                [(n, _D * MAXT * MAXQ) for n in ("F", "DX", "DY", "DZ")] +
                [(n, _D * MAXG * MAXG) for n in ("Ax", "Bx", "Ay", "By", "Az")] +
                [("T2", _I)] + [(n, _D * MAXT * (MAXG * MAXG)) for n in ("F2", "DX2", "DY2")] +
                [("W2", _D * (MAXG * MAXG)), ("mm", _D * MAXT * MAXT), ("vdiag", _D),
                 ("sfmv", _D * (MAXP - 1) * 2), ("ffmv", _D * (MAXP * (MAXP - 1) // 2) * 3),
                 ("ffms", _D * 2 * (MAXP * (MAXP - 1) // 2) * 3), ("sfms0", _D), ("mdiag", _D), ("odiag", _D)])


def tables(p):
    """hp_tet_basis_build(p) as a TetTables structure."""
    lib = L.lib()
    lib.hp_tet_basis_build.argtypes = [_I, ctypes.POINTER(TetTables)]
    t = TetTables()
    rc = lib.hp_tet_basis_build(p, ctypes.byref(t))
    if rc != 0:
        raise ValueError(f"tet basis p={p} unsupported")
    return t


def arr(t, name):
    """A numpy copy of one table, cut to its used extent."""
    G, T = t.G, t.T
    a = np.ctypeslib.as_array(getattr(t, name)).copy()
    cols = {"gx": t.nmodx, "dgx": t.nmodx, "gy": t.nmody, "dgy": t.nmody, "gz": t.nmodz, "dgz": t.nmodz}
    if name in cols:
        return a[:G, :cols[name]]
    if name in ("F", "DX", "DY", "DZ"):
        return a[:G ** 3, :T]
    if name == "w":
        return a[:G ** 3]
    if name in ("F2", "DX2", "DY2"):
        return a[:G * G, :t.T2]
    if name == "W2":
        return a[:G * G]
    if name == "mm":
        return a[:T, :T]
    if name == "sfmv":
        return a[:, :t.em]
    if name == "ffmv":
        return a[:, :t.fm]
    if name == "ffms":
        return a[:, :t.fm, :]
    if name in ("mx", "my", "mz", "msg"):
        return a[:T]
    if a.ndim == 2:
        return a[:G, :G]
    return a[:G]


def deriv(t, direction, f):
    """derivr / derivs / derivt of point values f[G,G,G] (returned, not added)."""
    G = t.G
    f = np.asarray(f).reshape(G, G, G)
    y0 = arr(t, "y0")[None, :, None]
    z0 = arr(t, "z0")[None, None, :]
    ax = lambda A: np.einsum("in,njk->ijk", A, f)
    ay = lambda A: np.einsum("jn,ink->ijk", A, f)
    az = lambda A: np.einsum("kn,ijn->ijk", A, f)
    if direction == 0:
        return (y0 * z0 * ax(arr(t, "Ax"))).ravel()
    if direction == 1:
        return (y0 * z0 * ax(arr(t, "Bx")) + z0 * ay(arr(t, "Ay"))).ravel()
    return (y0 * z0 * ax(arr(t, "Bx")) + z0 * ay(arr(t, "By")) + az(arr(t, "Az"))).ravel()


def beltrami(X, Y, Z, re=100.0, a=np.pi / 4, d=np.pi / 2, t=0.0):
    """The Ethier-Steinman 3D Beltrami solution of incompressible Navier-Stokes
    (rho = 1, nu = 1/re): velocity (u, v, w) and pressure at time t."""
    nu = 1.0 / re
    e1 = np.exp(-nu * d * d * t)
    u = -a * (np.exp(a * X) * np.sin(a * Y + d * Z) + np.exp(a * Z) * np.cos(a * X + d * Y)) * e1
    v = -a * (np.exp(a * Y) * np.sin(a * Z + d * X) + np.exp(a * X) * np.cos(a * Y + d * Z)) * e1
    w = -a * (np.exp(a * Z) * np.sin(a * X + d * Y) + np.exp(a * Y) * np.cos(a * Z + d * X)) * e1
    p = -0.5 * a * a * (np.exp(2 * a * X) + np.exp(2 * a * Y) + np.exp(2 * a * Z) +
                        2 * np.sin(a * X + d * Y) * np.cos(a * Z + d * X) * np.exp(a * (Y + Z)) +
                        2 * np.sin(a * Y + d * Z) * np.cos(a * X + d * Y) * np.exp(a * (Z + X)) +
                        2 * np.sin(a * Z + d * X) * np.cos(a * Y + d * Z) * np.exp(a * (X + Y))) * e1 * e1
    return np.stack([u, v, w, p], axis=-1)


class TetProblem:
    """One tet_hp ins level: mesh (hpb.tetmesh.TetMesh), p <= 4, physics and the
    modal state (vertices [npnt][4], edges [nseg][em][4], faces [ntri][fm][4],
    interiors [ntet][im][4]; variables u, v, w, p)."""

    NV = 4

    def __init__(self, mesh, p, *, rho=1.0, mu=0.01, adis=1.0, nstage=5, alpha=None, beta=None, cfl=1.0):
        from .problem import ALPHA_DFLT, BETA_DFLT
        alpha = ALPHA_DFLT if alpha is None else alpha
        beta = BETA_DFLT if beta is None else beta
        self.mesh, self.p = mesh, p
        self.tab = tables(p)
        t = self.tab
        ph = L.PhysParams()
        ph.physics = L.HP_PHYS_INS
        ph.nstage = nstage
        for k in range(8):
            ph.alpha[k] = alpha[k] if k < nstage else 1.0
            ph.beta[k] = beta[k] if k < nstage else 1.0
        ph.cfl, ph.bd0, ph.adis, ph.rho, ph.mu = cfl, 0.0, adis, rho, mu
        self.phys = ph
        self.ugv = np.zeros((mesh.npnt, 4))
        self.uge = np.zeros((mesh.nseg, t.em, 4))
        self.ugf = np.zeros((mesh.ntri, t.fm, 4))
        self.ugi = np.zeros((mesh.ntet, t.im, 4))

    @property
    def state(self):
        return self.ugv, self.uge, self.ugf, self.ugi

    @property
    def ndof(self):
        return sum(a.size for a in self.state)

    def dirichlet_masks(self, faces=None):
        """Velocity rows fixed on the boundary faces (bdry_ins::inflow: u, v, w essential,
        pressure free): masks [npnt][4], [nseg][4], [ntri][4]."""
        m = self.mesh
        v, e, f = m.boundary_entities(faces)
        mv = np.zeros((m.npnt, 4), np.uint8)
        me = np.zeros((m.nseg, 4), np.uint8)
        mf = np.zeros((m.ntri, 4), np.uint8)
        mv[v, :3] = 1
        me[e, :3] = 1
        mf[f, :3] = 1
        return mv, me, mf

    def face_points(self, faces):
        """Physical coordinates [nface][G * G][3] of the Gauss points of straight faces
        (proj2d of the face's vertex coordinates, crdtocht2d)."""
        F2 = arr(self.tab, "F2")[:, :3]
        X = self.mesh.pnts[self.mesh.tri_pnt[np.asarray(faces)]]       # (nf, 3, 3)
        return np.einsum("qv,fvd->fqd", F2, X)

    def flux_faces(self, inflow, neumann=(), pressure=None):
        """Boundary faces with a flux (bdry_ins::inflow / neumann, tet_hp/ins/bdry_ins.h:85-132)
        as the arguments of hp_tet_set_flux_faces: `inflow` faces carry the continuity flux,
        `neumann` faces also the momentum flux with the pressure `pressure(x, y, z)` imposed
        at their Gauss points."""
        inflow = np.asarray(inflow, dtype=np.int32)
        neumann = np.asarray(neumann, dtype=np.int32)
        faces = np.concatenate([inflow, neumann]).astype(np.int32)
        seg, sgn = self.mesh.face_edges(faces)
        kind = np.concatenate([np.zeros(len(inflow), np.int32), np.ones(len(neumann), np.int32)])
        G2 = self.tab.G ** 2
        pbc = np.zeros((len(faces), G2))
        if len(neumann):
            x = self.face_points(neumann)
            pbc[len(inflow):] = pressure(x[..., 0], x[..., 1], x[..., 2])
        return dict(face_tri=faces, face_pnt=np.ascontiguousarray(self.mesh.tri_pnt[faces]),
                    face_seg=seg, face_sgn=sgn, kind=kind, pbc=np.ascontiguousarray(pbc))

    def boundary_flux(self, ff):
        """rho times the integral of u_h . n over the faces of `ff` with the face quadrature:
        the continuity flux summed over the vertex rows (their modes sum to one)."""
        t, m = self.tab, self.mesh
        em, fm = t.em, t.fm
        F2, DX2, DY2, W2 = (arr(t, n) for n in ("F2", "DX2", "DY2", "W2"))
        faces, pv = ff["face_tri"], ff["face_pnt"]
        parts = [self.ugv[pv][:, :, :3]]
        for i in range(3):
            for k in range(em):
                sg = ff["face_sgn"][:, i].astype(np.float64) ** k
                parts.append((self.uge[ff["face_seg"][:, i], k, :3] * sg[:, None])[:, None, :])
        if fm:
            parts.append(self.ugf[faces][:, :, :3])
        uht = np.concatenate(parts, axis=1)                        # (nf, T2, 3)
        u = np.einsum("qk,fkn->fqn", F2, uht)
        X = m.pnts[pv]
        dr = np.einsum("qv,fvd->fqd", DX2[:, :3], X)
        ds = np.einsum("qv,fvd->fqd", DY2[:, :3], X)
        return self.phys.rho * float(np.einsum("q,fqd,fqd->", W2, u, np.cross(dr, ds)))

    def balance_inflow(self, ff, lo=0.0):
        """Shift u at the vertices of the x = lo face so that the discrete boundary flux of
        `ff` is zero. With velocity essential on every face the vertex continuity rows sum
        to that flux whatever the interior state, so it must vanish for the residual to
        reach zero; u on x = lo is normal only to that face, so nothing else changes."""
        v = np.nonzero(np.abs(self.mesh.pnts[:, 0] - lo) < 1e-12)[0]
        f0 = self.boundary_flux(ff)
        self.ugv[v, 0] += 1.0
        f1 = self.boundary_flux(ff)
        self.ugv[v, 0] -= 1.0 + f0 / (f1 - f0)
        return self.boundary_flux(ff)

    def group_boundary(self, groups, inflow, outflow=(), pressure=None, balance=True):
        """Boundary layout from named face groups (hpb.tetmesh.read_msh: the reference's
        b0_f<id>_hp_type keys): `inflow` / `outflow` are lists of group ids (inflow: velocity
        essential and the continuity flux; outflow: the neumann flux with `pressure(x, y, z)`
        imposed). With no outflow group and balance=True the state's boundary flux is balanced
        to zero on the vertices of the first inflow group, which must be planar. Call before
        the state is uploaded. Returns (essential masks, flux faces)."""
        inf = np.concatenate([groups[g] for g in inflow]).astype(np.int32)
        out = (np.concatenate([groups[g] for g in outflow]).astype(np.int32) if len(outflow)
               else np.zeros(0, np.int32))
        ff = self.flux_faces(inf, out, pressure)
        if not len(out) and balance:
            self._balance_on(ff, groups[inflow[0]])
        return self.dirichlet_masks(inf), ff

    def _balance_on(self, ff, faces):
        """Shift the velocity at the vertices of `faces` (a planar group) along its normal so
        that the boundary flux of ff is zero; those vertices' normal velocity enters only that
        group's flux when the neighbouring groups are orthogonal planes."""
        m = self.mesh
        X = m.pnts[m.tri_pnt[faces[0]]]
        nrm = np.cross(X[1] - X[0], X[2] - X[0])
        nrm /= np.linalg.norm(nrm)
        v = np.unique(m.tri_pnt[faces].ravel())
        f0 = self.boundary_flux(ff)
        self.ugv[v, :3] += nrm
        f1 = self.boundary_flux(ff)
        self.ugv[v, :3] -= (1.0 + f0 / (f1 - f0)) * nrm
        return self.boundary_flux(ff)

    def cube_boundary(self, re=100.0, outflow=False):
        """Unit-cube boundary layouts built from the reference's face types. outflow=False:
        inflow (velocity essential, continuity flux) on all six faces, with the state's
        boundary flux balanced to zero (balance_inflow). outflow=True: inflow on five faces
        and a neumann outflow with the Beltrami pressure imposed at x = 1 (the Beltrami flow
        crosses that face in both directions). Call before the state is uploaded. Returns
        (essential masks, flux faces)."""
        m = self.mesh
        bf = m.boundary_faces()
        cx = m.pnts[m.tri_pnt[bf], 0].mean(axis=1)
        out = bf[cx > 1.0 - 1e-12] if outflow else bf[:0]
        inf = bf[~np.isin(bf, out)]
        press = lambda x, y, z: beltrami(x, y, z, re=re)[..., 3]
        ff = self.flux_faces(inf, out, press)
        if not outflow:
            self.balance_inflow(ff)
        return self.dirichlet_masks(inf), ff

    def set_beltrami(self, re=100.0, noise=1e-3, seed=20261209):
        """Vertex values of the Beltrami field, high-order modes zero, plus seeded
        U[-1,1) noise of amplitude `noise` on every coefficient."""
        from .mesh import splitmix64_uniform
        P = self.mesh.pnts
        self.ugv[:] = beltrami(P[:, 0], P[:, 1], P[:, 2], re=re)
        for a in (self.uge, self.ugf, self.ugi):
            a[:] = 0.0
        if noise:
            n = self.ndof
            r = splitmix64_uniform(seed, n) * noise
            k = 0
            for a in self.state:
                a += r[k:k + a.size].reshape(a.shape)
                k += a.size
        return self


class TetMeshDesc(ctypes.Structure):
    _fields_ = [("npnt", _I), ("nseg", _I), ("ntri", _I), ("ntet", _I), ("pnts", ctypes.c_void_p),
                ("tet_pnt", ctypes.c_void_p), ("tet_seg", ctypes.c_void_p), ("tet_sgn", ctypes.c_void_p),
                ("tet_tri", ctypes.c_void_p), ("tet_rot", ctypes.c_void_p), ("vol", ctypes.c_void_p)]


_bound = False


def _bind():
    global _bound
    lib = L.lib()
    if not _bound:
        P = ctypes.c_void_p
        lib.hp_tet_create.argtypes = [ctypes.POINTER(TetMeshDesc), ctypes.POINTER(TetTables),
                                      ctypes.POINTER(L.PhysParams), _I, P, ctypes.POINTER(P)]
        lib.hp_tet_destroy.argtypes = [P]
        lib.hp_tet_upload_state.argtypes = [P, P, P, P, P]
        lib.hp_tet_download_state.argtypes = [P, P, P, P, P]
        lib.hp_tet_download_residual.argtypes = [P, _I, P, P, P, P]
        lib.hp_tet_setup_preconditioner.argtypes = [P]
        lib.hp_tet_download_prcn.argtypes = [P, P, P]
        lib.hp_tet_enqueue_rsdl.argtypes = [P, _I]
        lib.hp_tet_rsdl.argtypes = [P, _I]
        lib.hp_tet_sync.argtypes = [P]
        lib.hp_tet_last_error.restype = ctypes.c_char_p
        lib.hp_tet_set_dirichlet.argtypes = [P, P, P, P]
        lib.hp_tet_set_flux_faces.argtypes = [P, _I, P, P, P, P, P, P]
        lib.hp_tet_set_smoother.argtypes = [P, _I]
        lib.hp_tet_jacobian_diagonal.argtypes = [P]
        lib.hp_tet_download_jacobian_diagonal.argtypes = [P, P, P, P, P]
        lib.hp_tet_enqueue_update.argtypes = [P]
        lib.hp_tet_update.argtypes = [P]
        lib.hp_tet_elem_features.argtypes = [P, P]
        lib.hp_tet_elem_resnorm.argtypes = [P, P]
        lib.hp_tet_set_prcn_scale.argtypes = [P, P, ctypes.c_float]
        lib.hp_tet_set_prcn_net.argtypes = [P, P, ctypes.c_float]
        lib.hp_tet_resnorm.argtypes = [P, ctypes.POINTER(ctypes.c_double)]
        lib.hp_tet_solve.argtypes = [P, ctypes.c_double, _I, _I, P, _I, ctypes.POINTER(_I),
                                     ctypes.POINTER(ctypes.c_double), ctypes.POINTER(_I)]
        lib.hp_tet_fp64_mma_peak.argtypes = [_I, ctypes.c_double, ctypes.POINTER(ctypes.c_double)]
        _bound = True
    return lib


def _check(lib, rc, what):
    if rc != 0:
        raise RuntimeError(f"{what} failed with status {rc}: {lib.hp_tet_last_error().decode()}")


class TetGPU:
    """A hp_tet_ctx for a TetProblem (the C ABI of include/hp_tet.h)."""

    def __init__(self, prob, device=0, stream=None):
        self.lib = lib = _bind()
        self.prob = prob
        m = prob.mesh
        ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        self._keep = m
        self.desc = TetMeshDesc(m.npnt, m.nseg, m.ntri, m.ntet, ptr(m.pnts), ptr(m.tet_pnt), ptr(m.tet_seg),
                                ptr(m.tet_sgn), ptr(m.tet_tri), ptr(m.tet_rot), ptr(m.vol))
        h = ctypes.c_void_p()
        _check(lib, lib.hp_tet_create(ctypes.byref(self.desc), ctypes.byref(prob.tab), ctypes.byref(prob.phys),
                                      device, stream, ctypes.byref(h)), "hp_tet_create")
        self.h = h
        self.upload(*prob.state)

    def close(self):
        if getattr(self, "h", None):
            self.lib.hp_tet_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    @staticmethod
    def _p(a):
        return None if a is None or a.size == 0 else a.ctypes.data_as(ctypes.c_void_p)

    def upload(self, v, e, f, i):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (v, e, f, i)]
        _check(self.lib, self.lib.hp_tet_upload_state(self.h, *[self._p(a) for a in arrs]), "upload")

    def _out(self):
        return [np.zeros_like(a) for a in self.prob.state]

    def state(self):
        out = self._out()
        _check(self.lib, self.lib.hp_tet_download_state(self.h, *[self._p(a) for a in out]), "download_state")
        return out

    def residual(self, which=0):
        out = self._out()
        _check(self.lib, self.lib.hp_tet_download_residual(self.h, which, *[self._p(a) for a in out]),
               "download_residual")
        return out

    def setup_preconditioner(self):
        return self.lib.hp_tet_setup_preconditioner(self.h)

    def prcn(self):
        m = self.prob.mesh
        tau = np.zeros((m.ntet, 2))
        ip = np.zeros((m.ntet, 4))
        _check(self.lib, self.lib.hp_tet_download_prcn(self.h, self._p(tau), self._p(ip)), "download_prcn")
        return tau, ip

    def rsdl(self, stage):
        _check(self.lib, self.lib.hp_tet_rsdl(self.h, stage), "rsdl")

    def set_dirichlet(self, masks):
        mv, me, mf = (np.ascontiguousarray(a, dtype=np.uint8) for a in masks)
        _check(self.lib, self.lib.hp_tet_set_dirichlet(self.h, self._p(mv), self._p(me), self._p(mf)),
               "set_dirichlet")

    def set_smoother(self, kind):
        """0: the JACOBI build's jacobi_relaxation; 1: tet_hp::minvrt (p = 1, 2 and 3). At
        p = 3 the vertex-ball spoke factors come with the next setup_preconditioner."""
        _check(self.lib, self.lib.hp_tet_set_smoother(self.h, kind), "set_smoother")

    def set_flux_faces(self, ff):
        """Boundary faces with a flux (TetProblem.flux_faces / cube_boundary)."""
        a = {k: np.ascontiguousarray(v) for k, v in ff.items()}
        _check(self.lib, self.lib.hp_tet_set_flux_faces(
            self.h, len(a["face_tri"]), self._p(a["face_tri"]), self._p(a["face_pnt"]), self._p(a["face_seg"]),
            self._p(a["face_sgn"]), self._p(a["kind"]), self._p(a["pbc"])), "set_flux_faces")

    def jacobian_diagonal(self):
        _check(self.lib, self.lib.hp_tet_jacobian_diagonal(self.h), "jacobian_diagonal")
        out = self._out()
        _check(self.lib, self.lib.hp_tet_download_jacobian_diagonal(self.h, *[self._p(a) for a in out]),
               "download_jacobian_diagonal")
        return out

    def update(self):
        _check(self.lib, self.lib.hp_tet_update(self.h), "update")

    def iterate(self, n):
        for _ in range(n):
            _check(self.lib, self.lib.hp_tet_enqueue_update(self.h), "update")
        _check(self.lib, self.lib.hp_tet_sync(self.h), "sync")

    def elem_features(self):
        """[ntet][17] float32 inputs of the learned correction at the current state."""
        import torch
        d = torch.empty((self.prob.mesh.ntet, 17), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        _check(self.lib, self.lib.hp_tet_elem_features(self.h, ctypes.c_void_p(d.data_ptr())), "elem_features")
        _check(self.lib, self.lib.hp_tet_sync(self.h), "sync")
        return d.cpu().numpy()

    def elem_resnorm(self):
        """Per-tetrahedron residual measure of rsdl(nstage) at the current state."""
        import torch
        self.rsdl(self.prob.phys.nstage)
        d = torch.empty(self.prob.mesh.ntet, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        _check(self.lib, self.lib.hp_tet_elem_resnorm(self.h, ctypes.c_void_p(d.data_ptr())), "elem_resnorm")
        _check(self.lib, self.lib.hp_tet_sync(self.h), "sync")
        return d.cpu().numpy()

    def set_prcn_scale(self, d_logscale, clamp=1.5):
        """Per-tetrahedron log-scales (a device pointer or None) of the smoother's diagonal."""
        _check(self.lib, self.lib.hp_tet_set_prcn_scale(self.h, d_logscale, clamp), "set_prcn_scale")

    def attach_net(self, net, clamp=1.0):
        """The learned correction (hpb.learned.MLP, 17 -> 1) evaluated at every set-up; None detaches."""
        _check(self.lib, self.lib.hp_tet_set_prcn_net(self.h, net.h if net is not None else None, clamp),
               "set_prcn_net")

    def resnorm(self):
        r = ctypes.c_double()
        _check(self.lib, self.lib.hp_tet_resnorm(self.h, ctypes.byref(r)), "resnorm")
        return r.value

    def solve(self, drop=1e-10, max_updates=20000, check_every=20):
        cap = max_updates // check_every + 4
        hist = np.zeros(cap)
        nh, nu = ctypes.c_int(), ctypes.c_int()
        sec = ctypes.c_double()
        _check(self.lib, self.lib.hp_tet_solve(self.h, drop, max_updates, check_every, self._p(hist), cap,
                                               ctypes.byref(nh), ctypes.byref(sec), ctypes.byref(nu)), "solve")
        return hist[:nh.value], sec.value, nu.value


def locate_cube(mesh, n, pts, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0)):
    """The tetrahedron of cube_tets(n) holding each point (tet_mesh::findtet) and its 4
    barycentric weights in that tetrahedron's vertex order (getwgts): the point's
    hexahedron is found by index, then the best of its 6 tetrahedra. Weights below
    1e-13 are dropped and the rest renormalised, so points on a face of the box take
    weights from that face only."""
    lo, hi = np.asarray(lo, float), np.asarray(hi, float)
    pts = np.asarray(pts, float)
    ijk = np.clip(np.floor((pts - lo) / ((hi - lo) / n)).astype(np.int64), 0, n - 1)
    hexi = (ijk[:, 0] * n + ijk[:, 1]) * n + ijk[:, 2]
    best_t = np.zeros(len(pts), np.int64)
    best_w = np.zeros((len(pts), 4))
    best_m = np.full(len(pts), -np.inf)
    P = mesh.pnts
    for k in range(6):
        t = hexi * 6 + k
        v = mesh.tet_pnt[t]
        A = np.stack([P[v[:, 1]] - P[v[:, 0]], P[v[:, 2]] - P[v[:, 0]], P[v[:, 3]] - P[v[:, 0]]], axis=2)
        lam = np.linalg.solve(A, (pts - P[v[:, 0]])[:, :, None])[:, :, 0]
        w = np.concatenate([1.0 - lam.sum(1, keepdims=True), lam], axis=1)
        m = w.min(1)
        better = m > best_m
        best_m[better], best_t[better], best_w[better] = m[better], t[better], w[better]
    if np.any(best_m < -1e-9):
        raise ValueError("point outside the mesh")
    best_w[np.abs(best_w) < 1e-13] = 0.0
    best_w /= best_w.sum(1, keepdims=True)
    return best_t.astype(np.int32), np.ascontiguousarray(best_w)


class TetHierarchy:
    """tet multigrid on the unit cube: p-levels p, p-1, ..., 1 on cube_tets(n), then
    h-levels cube_tets(n/2), cube_tets(n/4), ... at p = 1 (the reference decrements
    log2p = p - 1 for tetrahedra; h-levels as tet_mesh coarsening). Every level takes the
    Beltrami state, the boundary layout of TetProblem.cube_boundary (inflow on all six
    faces with a balanced boundary flux; outflow=True: a neumann outflow at x = 1) and
    `cfl[p]`; minvrt=True smooths the p = 1 and 2 levels with tet_hp::minvrt instead of the
    JACOBI build's relaxation, minvrt="all" every level (p = 3 included)."""

    def __init__(self, n, p, hlevels=2, mu=0.01, cfl=None, re=100.0, noise=1e-3, stream=None, fadd=1.0,
                 outflow=False, minvrt=False):
        import torch
        from .tetmesh import cube_tets
        cfl = cfl or {1: 2.2, 2: 1.5, 3: 1.0, 4: 0.5}
        if stream is None:
            self._stream = torch.cuda.Stream()
            stream = ctypes.c_void_p(self._stream.cuda_stream)
        meshes = [(cube_tets(n), n)] + [(cube_tets(n >> k), n >> k) for k in range(1, hlevels + 1)]
        specs = [(0, q) for q in range(p, 0, -1)] + [(k, 1) for k in range(1, hlevels + 1)]
        self.probs, self.levels, self.kinds, self.masks = [], [], [], []
        for li, (mi, q) in enumerate(specs):
            pr = TetProblem(meshes[mi][0], q, mu=mu, cfl=cfl[q]).set_beltrami(re=re, noise=noise)
            masks, ff = pr.cube_boundary(re=re, outflow=outflow)
            g = TetGPU(pr, stream=stream)
            g.set_dirichlet(masks)
            g.set_flux_faces(ff)
            if minvrt == "all" or (q <= 2 and minvrt):
                g.set_smoother(1)
            self.probs.append(pr)
            self.masks.append(masks)
            self.levels.append(g)
        lib = self.levels[0].lib
        lib.hp_tet_mg_attach_p.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double]
        P_ = ctypes.c_void_p
        lib.hp_tet_mg_attach_h.argtypes = [P_, P_, P_, P_, P_, P_, ctypes.c_double]
        lib.hp_tet_solve_mg.argtypes = [ctypes.POINTER(P_), _I, ctypes.c_double, _I, _I, _I, _I, P_, _I,
                                        ctypes.POINTER(_I), ctypes.POINTER(ctypes.c_double), ctypes.POINTER(_I)]
        lib.hp_tet_solve_mg_mixed.argtypes = lib.hp_tet_solve_mg.argtypes
        self._keep = []
        for li in range(1, len(specs)):
            c, f = self.levels[li], self.levels[li - 1]
            if specs[li][0] == specs[li - 1][0]:
                _check(lib, lib.hp_tet_mg_attach_p(c.h, f.h, fadd), "mg_attach_p")
            else:
                (fm, fn), (cm, cn) = meshes[specs[li - 1][0]], meshes[specs[li][0]]
                f2c = locate_cube(cm, cn, fm.pnts)
                c2f = locate_cube(fm, fn, cm.pnts)
                self._keep += [f2c, c2f]
                _check(lib, lib.hp_tet_mg_attach_h(c.h, f.h, f2c[0].ctypes.data, f2c[1].ctypes.data,
                                                   c2f[0].ctypes.data, c2f[1].ctypes.data, fadd), "mg_attach_h")
        self.lib = lib

    def solve(self, drop=1e-10, max_cycles=300, vw=1, itercrsn=2, iterrfne=2, mixed=False):
        """Cycles to a `drop` of the FP64 residual norm; mixed=True: FP32 (TF32 tensor-core)
        smoothing inside FP64 defect correction (hp_tet_solve_mg_mixed)."""
        hs = (ctypes.c_void_p * len(self.levels))(*[g.h for g in self.levels])
        hist = np.zeros(max_cycles + 2)
        nh, nc = ctypes.c_int(), ctypes.c_int()
        sec = ctypes.c_double()
        fn = self.lib.hp_tet_solve_mg_mixed if mixed else self.lib.hp_tet_solve_mg
        _check(self.lib, fn(hs, len(self.levels), drop, max_cycles, vw, itercrsn, iterrfne, hist.ctypes.data,
                            len(hist), ctypes.byref(nh), ctypes.byref(sec), ctypes.byref(nc)), "solve_mg")
        return hist[:nh.value], sec.value, nc.value

    def close(self):
        for g in self.levels:
            g.close()

"""Boundary-face fluxes of the tet path (bdry_ins::inflow / neumann, tet_hp/ins/bdry.cpp:16-102):
the face connectivity against a brute-force search, and the oracle's face flux against the
divergence theorem. For a random modal velocity u_h (every vertex, edge, face and interior
mode set), the continuity flux rho u_h . n summed over the vertex pressure rows (the vertex
modes sum to one on every face) is rho times the integral of u_h . n over the boundary, which
must equal rho times the volume integral of div u_h computed with the 3D operators. Both
quadratures are exact for these degrees, so the two agree to rounding only if the face gather
(edges, signs, face modes) gives the trace of the 3D field and the normal points out."""
import numpy as np
import pytest

import os

from hpb import tet as TB
from hpb.tetmesh import TetMesh, cube_tets, read_msh
from oracle import oracle as O

REF_DIR = os.environ.get("HP_REFERENCE_DIR")  # reference checkout, for the checks that read its files
REF_MSH = os.path.join(REF_DIR or "", "Testing/tet_hp/cd/Multigrid/Inputs/tet{}.msh")


def scrambled_cube(n, seed):
    """cube_tets(n) with the interior vertices jittered by up to 0.2 of a cell and every
    vertex renumbered at random, so the tetrahedra take all kinds of local orientation."""
    c = cube_tets(n)
    rng = np.random.default_rng(seed)
    pts = c.pnts.copy()
    inner = np.all((pts > 1e-12) & (pts < 1 - 1e-12), axis=1)
    pts[inner] += rng.uniform(-0.2, 0.2, (inner.sum(), 3)) / n
    perm = rng.permutation(c.npnt)
    newp = np.empty_like(pts)
    newp[perm] = pts
    tets = perm[c.tet_pnt]
    tets = tets[rng.permutation(len(tets))]
    return TetMesh(newp, tets)


def test_face_edges_match_brute_force():
    m = cube_tets(2)
    bf = m.boundary_faces()
    seg, sgn = m.face_edges(bf)
    for f, s, g in zip(bf, seg, sgn):
        a = m.tri_pnt[f]
        for i in range(3):
            b, c = a[(i + 1) % 3], a[(i + 2) % 3]
            hit = [k for k in range(m.nseg) if set(m.seg_pnt[k]) == {b, c}]
            assert hit == [s[i]]
            assert g[i] == (1 if m.seg_pnt[s[i], 0] == b else -1)


def test_boundary_face_normals_point_out():
    m = cube_tets(3)
    bf = m.boundary_faces()
    t = m.tri_tet[bf, 0]
    X = m.pnts[m.tri_pnt[bf]]
    nrm = np.cross(X[:, 1] - X[:, 0], X[:, 2] - X[:, 0])
    opp = m.pnts[m.tet_pnt[t]].mean(axis=1)          # centroid of the owning tetrahedron
    assert np.all(np.einsum("fd,fd->f", nrm, X[:, 0] - opp) > 0)


def gather3d(prob, tind):
    """ugtouht of one tetrahedron (tet_hp/gtol.cpp:16-82): uht [T][4]."""
    m, t = prob.mesh, prob.tab
    em, fm, im = t.em, t.fm, t.im
    v, e, f, i = prob.state
    out = [v[m.tet_pnt[tind]]]
    for k in range(6):
        s, g = m.tet_seg[tind, k], m.tet_sgn[tind, k]
        out.append(e[s] * (float(g) ** np.arange(em))[:, None])
    for k in range(4):
        fa, sg = m.tet_tri[tind, k], -m.tet_rot[tind, k]
        rows = np.concatenate([np.full(em - r, r) for r in range(1, em)]) if em > 1 else np.zeros(0, int)
        out.append(f[fa] * (float(sg) ** (rows - 1))[:, None])
    out.append(i[tind])
    return np.concatenate(out, axis=0)


def volume_divergence(prob):
    t = prob.tab
    F, DX, DY, DZ, w = (TB.arr(t, n) for n in ("F", "DX", "DY", "DZ", "w"))
    m = prob.mesh
    total, vol = 0.0, 0.0
    for tind in range(m.ntet):
        xv = m.pnts[m.tet_pnt[tind]]
        J = np.stack([D[:, :4] @ xv for D in (DX, DY, DZ)], axis=2)   # J[q][x][r]
        uht = gather3d(prob, tind)
        dref = np.stack([D @ uht[:, :3] for D in (DX, DY, DZ)], axis=2)  # [q][var][r]
        grad = np.einsum("qrx,qnr->qnx", np.linalg.inv(J), dref)        # du_n / dx_x
        det = np.abs(np.linalg.det(J))
        total += np.sum(w * det * np.trace(grad, axis1=1, axis2=2))
        vol += np.sum(w * det)
    return total, vol


@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_face_flux_satisfies_divergence_theorem(p):
    mesh = cube_tets(2)
    pr = TB.TetProblem(mesh, p, rho=1.3, mu=0.01).set_beltrami(noise=0.0)
    rng = np.random.default_rng(40 + p)
    for a in pr.state:
        a[:] = rng.uniform(-1, 1, a.shape)
    div, vol = volume_divergence(pr)
    assert abs(vol - 1.0) < 1e-12          # the 3D weights integrate the unit cube
    ff = pr.flux_faces(mesh.boundary_faces())
    with_f, without = O.OracleTet(pr), O.OracleTet(pr)
    with_f.set_flux_faces(ff)
    with_f.rsdl(0)
    without.rsdl(0)
    flux = with_f.residual()[0][:, 3] - without.residual()[0][:, 3]
    assert abs(flux.sum() - 1.3 * div) < 1e-11 * max(1.0, abs(div))


def test_neumann_face_flux_of_a_constant_state():
    """Constant velocity U and imposed pressure P on every face of the cube: the momentum flux
    summed over the vertex rows is sum over faces of (rho U.n U + P n) = 0, and the x = 1 face
    alone gives (rho U_x U + P e_x) times its area."""
    mesh = cube_tets(2)
    pr = TB.TetProblem(mesh, 3, mu=0.01).set_beltrami(noise=0.0)
    for a in pr.state:
        a[:] = 0.0
    U = np.array([0.3, -0.2, 0.5])
    pr.ugv[:, :3] = U
    bf = mesh.boundary_faces()
    cx = mesh.pnts[mesh.tri_pnt[bf], 0].mean(axis=1)
    for faces, expect in ((bf, np.zeros(3)), (bf[cx > 1 - 1e-12], 0.3 * U + np.array([2.0, 0, 0]))):
        ff = pr.flux_faces([], faces, lambda x, y, z: np.full_like(x, 2.0))
        with_f, without = O.OracleTet(pr), O.OracleTet(pr)
        with_f.set_flux_faces(ff)
        with_f.rsdl(0)
        without.rsdl(0)
        mom = (with_f.residual()[0] - without.residual()[0])[:, :3].sum(axis=0)
        assert np.max(np.abs(mom - expect)) < 1e-12


@pytest.mark.parametrize("p", [2, 3])
def test_balanced_inflow_makes_the_continuity_rows_consistent(p):
    """Velocity essential on all six faces: the vertex pressure rows of the whole residual sum
    to the boundary flux whatever the interior state, so after balance_inflow they sum to zero,
    and the host's boundary_flux equals the oracle's face-flux sum before balancing."""
    pr = TB.TetProblem(cube_tets(3), p, rho=1.1, mu=0.01).set_beltrami()
    ff = pr.flux_faces(pr.mesh.boundary_faces())
    phi = pr.boundary_flux(ff)
    with_f, without = O.OracleTet(pr), O.OracleTet(pr)
    with_f.set_flux_faces(ff)
    for o in (with_f, without):
        assert o.setup_preconditioner() == 0
        o.rsdl(0)
    assert abs(phi) > 1e-6
    fsum = (with_f.residual()[0][:, 3] - without.residual()[0][:, 3]).sum()
    assert abs(fsum - phi) < 1e-12 * max(1.0, abs(phi))
    masks, ff = pr.cube_boundary()
    assert abs(pr.boundary_flux(ff)) < 1e-14
    o = O.OracleTet(pr)
    o.set_flux_faces(ff)
    assert o.setup_preconditioner() == 0
    for stage in (0, pr.phys.nstage):
        o.rsdl(stage)
        rv = o.residual()[0][:, 3]
        assert abs(rv.sum()) < 1e-13 * np.abs(rv).sum()


def test_oracle_minvrt_p1_smoother_converges_and_is_limited_to_low_p():
    """tet_hp::minvrt at p = 1 (the default build's smoother) in the oracle: 200 updates at the
    reference's p = 1 cfl (2.2) reduce the residual by more than 1e4 on a 3^3 x 6 cube."""
    pr = TB.TetProblem(cube_tets(3), 1, mu=0.01, cfl=2.2).set_beltrami()
    masks, ff = pr.cube_boundary()
    o = O.OracleTet(pr)
    o.set_dirichlet(masks)
    o.set_flux_faces(ff)
    o.set_smoother(1)
    assert o.setup_preconditioner() == 0
    free = masks[0] == 0

    def norm():
        o.rsdl(pr.phys.nstage)
        return np.linalg.norm(np.where(free, o.residual()[0], 0.0))
    r0 = norm()
    for _ in range(200):
        o.update()
    assert norm() < 1e-4 * r0
    with pytest.raises(ValueError):
        O.OracleTet(TB.TetProblem(cube_tets(1), 4, mu=0.01).set_beltrami()).set_smoother(1)


@pytest.mark.parametrize("seed", [None, 11])
def test_oracle_minvrt_p3_face_topology_is_the_face_flux_convention(seed):
    """minvrt at p = 3 reads each face's vertices (in the order of the tetrahedron that
    numbered it) and the edge opposite each face vertex; the oracle derives both from the
    tetrahedra and they are the mesh's tri_pnt and the face-edge convention whose face flux
    the divergence-theorem tests above check, on the structured and on a scrambled cube."""
    msh = cube_tets(3) if seed is None else scrambled_cube(3, seed)
    o = O.OracleTet(TB.TetProblem(msh, 3, mu=0.01).set_beltrami())
    fp, fs = o.face_topology()
    assert np.array_equal(fp, msh.tri_pnt)
    seg, _ = msh.face_edges(np.arange(msh.ntri))
    assert np.array_equal(fs, seg)


def test_oracle_minvrt_p3_smoother_converges():
    """tet_hp::minvrt at p = 3 in the oracle (vertex-ball spoke solves of the edges' first
    modes, the second edge modes and the faces): 200 updates at cfl 2 reduce the residual of
    the free vertex, edge and face rows by more than 10 on a 3^3 x 6 cube; the fixed rows stay."""
    pr = TB.TetProblem(cube_tets(3), 3, mu=0.01, cfl=2.0).set_beltrami()
    masks, ff = pr.cube_boundary()
    o = O.OracleTet(pr)
    o.set_dirichlet(masks)
    o.set_flux_faces(ff)
    o.set_smoother(1)
    assert o.setup_preconditioner() == 0
    mv, me, mf = (np.asarray(a, dtype=bool) for a in masks)

    def norm():
        o.rsdl(pr.phys.nstage)
        r = o.residual()
        return np.sqrt(np.sum(r[0][~mv] ** 2) + np.sum(np.where(me[:, None, :], 0.0, r[1]) ** 2) +
                       np.sum(np.where(mf[:, None, :], 0.0, r[2]) ** 2))
    r0 = norm()
    u0 = o.state()
    for it in range(200):
        o.update()
        if it % 25 == 24:
            assert o.setup_preconditioner() == 0
    u = o.state()
    assert norm() < 0.1 * r0
    assert np.array_equal(u[0][mv], u0[0][mv])
    assert np.array_equal(u[1][np.broadcast_to(me[:, None, :], u[1].shape)],
                          u0[1][np.broadcast_to(me[:, None, :], u0[1].shape)])


def test_oracle_minvrt_p2_smoother_converges():
    """tet_hp::minvrt at p = 2 in the oracle at the reference's p = 2 cfl (1.5): 200 updates
    reduce the residual of the free vertex and edge rows by more than 100."""
    pr = TB.TetProblem(cube_tets(3), 2, mu=0.01, cfl=1.5).set_beltrami()
    masks, ff = pr.cube_boundary()
    o = O.OracleTet(pr)
    o.set_dirichlet(masks)
    o.set_flux_faces(ff)
    o.set_smoother(1)
    assert o.setup_preconditioner() == 0
    fv, fe = masks[0] == 0, (masks[1] == 0)[:, None, :]

    def norm():
        o.rsdl(pr.phys.nstage)
        r = o.residual()
        return np.sqrt(np.sum(np.where(fv, r[0], 0.0) ** 2) + np.sum(np.where(fe, r[1], 0.0) ** 2))
    r0 = norm()
    for _ in range(200):
        o.update()
    assert norm() < 1e-2 * r0


def _div_check(mesh, p, seed):
    pr = TB.TetProblem(mesh, p, rho=1.0, mu=0.01).set_beltrami(noise=0.0)
    rng = np.random.default_rng(seed)
    for a in pr.state:
        a[:] = rng.uniform(-1, 1, a.shape)
    div, vol = volume_divergence(pr)
    assert abs(vol - 1.0) < 1e-12
    ff = pr.flux_faces(mesh.boundary_faces())
    assert abs(pr.boundary_flux(ff) - div) < 1e-11 * max(1.0, abs(div))
    with_f, without = O.OracleTet(pr), O.OracleTet(pr)
    with_f.set_flux_faces(ff)
    with_f.rsdl(0)
    without.rsdl(0)
    flux = with_f.residual()[0][:, 3] - without.residual()[0][:, 3]
    assert abs(flux.sum() - div) < 1e-11 * max(1.0, abs(div))


@pytest.mark.parametrize("p", [2, 3, 4])
def test_divergence_theorem_on_a_scrambled_mesh(p):
    """The face gather, face-edge signs and normals on tetrahedra of every local orientation."""
    _div_check(scrambled_cube(2, 7), p, 70 + p)


@pytest.mark.skipif(not (REF_DIR and os.path.exists(REF_MSH.format(4))),
                    reason="HP_REFERENCE_DIR unset or its tet meshes absent")
def test_reference_gmsh_meshes_read_and_satisfy_the_divergence_theorem():
    """The reference's own tet test meshes (Testing/tet_hp/cd/Multigrid/Inputs/tet{2,4,8}.msh):
    unit volume, six boundary groups (the input's b0_f<id> keys) that cover the boundary faces,
    each on one face of the cube; and the face flux of a random p = 3 state on tet4.msh."""
    for n in (2, 4, 8):
        m, groups = read_msh(REF_MSH.format(n))
        assert m.ntet == 6 * n ** 3 and abs(m.vol.sum() / 6 - 1.0) < 1e-12
        assert sorted(groups) == [5, 14, 18, 22, 26, 27]
        assert np.array_equal(np.sort(np.concatenate(list(groups.values()))), np.sort(m.boundary_faces()))
        for faces in groups.values():
            x = m.pnts[m.tri_pnt[faces]].reshape(-1, 3)
            assert np.any(np.ptp(x, axis=0) < 1e-9)
    with pytest.raises(ValueError):
        read_msh(REF_MSH.format(1))                  # a 2D square: no tetrahedra
    _div_check(read_msh(REF_MSH.format(4))[0], 3, 90)
    # inflow on every group by id, boundary flux balanced: the continuity rows are consistent
    m, groups = read_msh(REF_MSH.format(2))
    pr = TB.TetProblem(m, 2, mu=0.01).set_beltrami()
    masks, ff = pr.group_boundary(groups, inflow=sorted(groups))
    assert abs(pr.boundary_flux(ff)) < 1e-14
    assert masks[0][:, :3].sum() == 3 * len(np.unique(m.tri_pnt[m.boundary_faces()]))
    o = O.OracleTet(pr)
    o.set_flux_faces(ff)
    assert o.setup_preconditioner() == 0
    o.rsdl(0)
    rv = o.residual()[0][:, 3]
    assert abs(rv.sum()) < 1e-13 * np.abs(rv).sum()


def modal_interpolant(pr, field):
    """The modal state of a field that the basis represents exactly: each element's modes from a
    least-squares fit at its Gauss points, scattered with the global edge / face signs of
    ugtouht; elements sharing an entity must agree. field(x, y, z) -> [..., 4]."""
    t, m = pr.tab, pr.mesh
    F = TB.arr(t, "F")
    em, fm = t.em, t.fm
    rows = np.concatenate([np.full(em - r, r) for r in range(1, em)]) if em > 1 else np.zeros(0, int)
    seen = [np.full(a.shape, np.nan) for a in pr.state]

    def put(k, idx, val):
        old = seen[k][idx]
        assert np.all(np.isnan(old) | (np.abs(old - val) < 1e-10)), "elements disagree on a shared mode"
        seen[k][idx] = val
    for tind in range(m.ntet):
        X = F[:, :4] @ m.pnts[m.tet_pnt[tind]]
        uh = np.linalg.lstsq(F, field(X[:, 0], X[:, 1], X[:, 2]), rcond=None)[0]   # [T][4]
        for v in range(4):
            put(0, m.tet_pnt[tind, v], uh[v])
        for i in range(6):
            sg = float(m.tet_sgn[tind, i]) ** np.arange(em)
            put(1, m.tet_seg[tind, i], uh[4 + i * em:4 + (i + 1) * em] * sg[:, None])
        for i in range(4):
            sg = float(-m.tet_rot[tind, i]) ** (rows - 1)
            put(2, m.tet_tri[tind, i], uh[4 + 6 * em + i * fm:4 + 6 * em + (i + 1) * fm] * sg[:, None])
        put(3, tind, uh[t.bm:])
    for a, s in zip(pr.state, seen):
        a[:] = s
    assert all(not np.isnan(a).any() for a in pr.state)


def poiseuille(direction, mu):
    """Steady Navier-Stokes solution: velocity along axis d equal to a(1-a) + b(1-b) in the two
    other coordinates, pressure -4 mu x_d (zero convection, mu lap u = grad p)."""
    def f(x, y, z):
        c = [x, y, z]
        a, b = (c[k] for k in range(3) if k != direction)
        out = np.zeros(x.shape + (4,))
        out[..., direction] = a * (1 - a) + b * (1 - b)
        out[..., 3] = -4.0 * mu * c[direction]
        return out
    return f


def shear(x, y, z):
    """Linear steady solution: u = (y + 2 z, 0, 0), constant pressure (u . grad u = 0)."""
    out = np.zeros(x.shape + (4,))
    out[..., 0] = y + 2.0 * z
    out[..., 3] = 0.3
    return out


def uniform(x, y, z):
    out = np.zeros(x.shape + (4,))
    out[..., :3] = (0.7, -0.4, 0.5)
    out[..., 3] = 0.3
    return out


@pytest.mark.parametrize("p,case,mesh", [(1, "uniform", "cube"), (1, "uniform", "scrambled"),
                                         (2, "shear", "cube"), (2, "shear", "scrambled"),
                                         (3, "shear", "scrambled"), (4, 0, "cube"), (4, 1, "scrambled"),
                                         (4, 2, "cube")])
def test_exact_steady_solutions_have_zero_residual(p, case, mesh):
    """Known answer for the tet ins residual (the 3D counterpart of the reference's p = 2 exact
    quadratic test): the interpolant of an exact steady solution has a zero residual on every
    row no boundary condition fixes, with velocity essential and the continuity flux on all
    faces. The solution must be in the space and keep the SUPG strong residual exact, which
    element_rsdl forms by differentiating point data of the convective flux u u through the
    p + 1 Gauss points of each collapsed direction (derivr / derivs / derivt): exact when u u
    has degree <= p. Hence uniform flow at p = 1, a linear shear at p >= 2 and Poiseuille
    flows (quartic u u) at p = 4; a Poiseuille flow at p = 2 leaves 1e-4 of stabilisation
    residual in the pressure rows. A perturbed state shows the scale."""
    msh = cube_tets(2) if mesh == "cube" else scrambled_cube(2, 5)
    mu = 0.05
    pr = TB.TetProblem(msh, p, mu=mu).set_beltrami(noise=0.0)
    field = {"uniform": uniform, "shear": shear}.get(case) or poiseuille(case, mu)
    modal_interpolant(pr, field)
    ff = pr.flux_faces(msh.boundary_faces())
    mk = pr.dirichlet_masks(msh.boundary_faces())
    assert abs(pr.boundary_flux(ff)) < 1e-13          # divergence free: no balancing needed

    def free_residual(state):
        o = O.OracleTet(pr)
        o.set_state(*state)
        o.set_dirichlet(mk)
        o.set_flux_faces(ff)
        assert o.setup_preconditioner() == 0
        o.rsdl(pr.phys.nstage)
        r = o.residual()
        parts = [np.where(mk[0], 0.0, r[0]).ravel()]
        if p > 1:
            parts.append(np.where(mk[1][:, None, :], 0.0, r[1]).ravel())
        if r[2].size:
            parts.append(np.where(mk[2][:, None, :], 0.0, r[2]).ravel())
        parts.append(r[3].ravel())
        return np.max(np.abs(np.concatenate(parts)))
    exact = free_residual(pr.state)
    rng = np.random.default_rng(3)
    pert = [a + 1e-3 * rng.uniform(-1, 1, a.shape) for a in pr.state]
    assert exact < 1e-9 * free_residual(pert), exact


def test_read_msh_round_trip(tmp_path):
    """read_msh on a Gmsh 2.2 file written here: cube_tets(2) with its boundary triangles
    tagged by cube face (elementary ids 11..16), node ids shuffled, extra point / line
    elements and a $PhysicalNames block that the reader skips."""
    c = cube_tets(2)
    rng = np.random.default_rng(1)
    ids = rng.permutation(c.npnt) + 100                    # file node id of each vertex
    bf = c.boundary_faces()
    X = c.pnts[c.tri_pnt[bf]]
    lines = ["$MeshFormat", "2.2 0 8", "$EndMeshFormat", "$PhysicalNames", "1", '2 1 "wall"',
             "$EndPhysicalNames", "$Nodes", str(c.npnt)]
    lines += [f"{ids[i]} {x:.17g} {y:.17g} {z:.17g}" for i, (x, y, z) in enumerate(c.pnts)]
    lines += ["$EndNodes", "$Elements"]
    els = [f"15 2 0 1 {ids[0]}", f"1 2 0 2 {ids[0]} {ids[1]}"]
    want = {}
    for f, tri in zip(bf, X):
        d = int(np.argmax(np.ptp(tri, axis=0) < 1e-12))
        ent = 11 + 2 * d + int(tri[0, d] > 0.5)
        want.setdefault(ent, []).append(f)
        els.append("2 2 1 %d %s" % (ent, " ".join(str(ids[v]) for v in c.tri_pnt[f])))
    els += ["4 2 1 1 %s" % " ".join(str(ids[v]) for v in t) for t in c.tet_pnt]
    lines += [str(len(els))] + [f"{k + 1} {e}" for k, e in enumerate(els)] + ["$EndElements"]
    path = tmp_path / "cube.msh"
    path.write_text("\n".join(lines) + "\n")
    m, groups = read_msh(str(path))
    assert (m.npnt, m.nseg, m.ntri, m.ntet) == (c.npnt, c.nseg, c.ntri, c.ntet)
    assert abs(m.vol.sum() / 6 - 1.0) < 1e-12
    assert sorted(groups) == sorted(want)
    # each group is the same set of triangles (by coordinates) as written
    key = lambda mesh, faces: sorted(tuple(sorted(map(tuple, np.round(mesh.pnts[mesh.tri_pnt[f]], 12)))) for f in faces)
    for ent in want:
        assert key(m, groups[ent]) == key(c, want[ent])

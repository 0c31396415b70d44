/*
 * hp_tet.h — C ABI of the 3D (tet_hp) path: modal tetrahedral basis tables and
 * the ins element residual on tetrahedra.
 *
 * Replaces, for the 3D hot path:
 *   tet_basis::initialize / initialize_values   tet_basis/initialize.cpp:21-520
 *   tet_basis::proj / intgrt / intgrtrst        tet_basis/proj.cpp:22-265, intgrt.cpp:23-609
 *   tet_basis::derivr / derivs / derivt         tet_basis/proj.cpp:781-911
 *   tet_hp::rsdl + tet_hp_ins::element_rsdl     tet_hp/update.cpp:9, tet_hp/ins/rsdl.cpp:15-785
 *   tet_hp_ins::setup_preconditioner (tau)      tet_hp/ins/setup_preconditioner.cpp
 *   bdry_ins::neumann / inflow face fluxes      tet_hp/ins/bdry.cpp:16-102
 */
#ifndef HP_TET_H
#define HP_TET_H

#ifdef __cplusplus
extern "C" {
#endif

#define HP_TET_MAXP 4  /* tet_basis.h:26 MAXP */
#define HP_TET_MAXG 5  /* Gauss points per direction, p + 1 */
#define HP_TET_MAXT 35 /* modes, (p+1)(p+2)(p+3)/6 */
#define HP_TET_MAXQ 125
#define HP_TET_MAXM 12 /* 1D functions per collapsed direction */

/* Tables of tet_basis for one p (gpx = gpy = gpz = G = p + 1). Point arrays use
 * the compact index q = (i * G + j) * G + k for Gauss point (x_i, y_j, z_k) of the
 * collapsed coordinates. Mode order: 4 vertices, 6 edges x em, 4 faces x fm,
 * interior (tet_basis.h:33-40).
 *
 * Dense operators (rows q, columns mode m): F = value, DX / DY / DZ = the r, s, t
 * derivatives that tet_basis::proj returns, w = wtx * wty * wtz, so that
 *   proj:      f(q) = sum_m F(q,m) u(m), and likewise dr, ds, dt;
 *   intgrt:    r(m) = sum_q w(q) F(q,m) f(q);
 *   intgrtrst: r(m) -= sum_q w(q) (DX(q,m) fr(q) + DY(q,m) fs(q) + DZ(q,m) ft(q)).
 * The point-derivative operators of derivr / derivs / derivt act along one
 * collapsed direction each: (Ax f)(i) = sum_n Ax(i,n) f(n) along x, and so on;
 *   derivr: dr += y0(j) z0(k) Ax_x f
 *   derivs: ds += y0(j) z0(k) Bx_x f + z0(k) Ay_y f
 *   derivt: dt += y0(j) z0(k) Bx_x f + z0(k) By_y f + Az_z f. */
typedef struct hp_tet_tables {
    int p, G, T, em, fm, im, bm, nmodx, nmody, nmodz;
    double gx[HP_TET_MAXG][HP_TET_MAXM], dgx[HP_TET_MAXG][HP_TET_MAXM];
    double gy[HP_TET_MAXG][HP_TET_MAXM], dgy[HP_TET_MAXG][HP_TET_MAXM];
    double gz[HP_TET_MAXG][HP_TET_MAXM], dgz[HP_TET_MAXG][HP_TET_MAXM];
    double wtx[HP_TET_MAXG], wty[HP_TET_MAXG], wtz[HP_TET_MAXG];
    double xp[HP_TET_MAXG], yp[HP_TET_MAXG], zp[HP_TET_MAXG];
    double x0[HP_TET_MAXG], y0[HP_TET_MAXG], y1[HP_TET_MAXG], z0[HP_TET_MAXG];
    double dltx[HP_TET_MAXG], dlty[HP_TET_MAXG], dltz[HP_TET_MAXG];
    double dltx2[HP_TET_MAXG][HP_TET_MAXG], dltx3[HP_TET_MAXG][HP_TET_MAXG];
    double dlty2[HP_TET_MAXG][HP_TET_MAXG], dlty3[HP_TET_MAXG][HP_TET_MAXG];
    double dltz2[HP_TET_MAXG][HP_TET_MAXG];
    int mx[HP_TET_MAXT], my[HP_TET_MAXT], mz[HP_TET_MAXT]; /* 1D function of each mode */
    double msg[HP_TET_MAXT];                               /* its sign */
    double w[HP_TET_MAXQ];
    double F[HP_TET_MAXQ][HP_TET_MAXT], DX[HP_TET_MAXQ][HP_TET_MAXT];
    double DY[HP_TET_MAXQ][HP_TET_MAXT], DZ[HP_TET_MAXQ][HP_TET_MAXT];
    double Ax[HP_TET_MAXG][HP_TET_MAXG], Bx[HP_TET_MAXG][HP_TET_MAXG];
    double Ay[HP_TET_MAXG][HP_TET_MAXG], By[HP_TET_MAXG][HP_TET_MAXG];
    double Az[HP_TET_MAXG][HP_TET_MAXG];
    /* Face (triangle) basis of tet_basis::proj2d / intgrt2d (tet_basis/proj2d.cpp:20-118,
     * intgrt2d.cpp:23-113): T2 = 3 + 3 em + fm modes (face vertices 0..2, face edge i
     * opposite vertex i, face modes) at the G x G points q2 = i * G + j; F2 value, DX2 / DY2
     * the derivatives proj2d returns (its y derivative of edge-0 and face modes uses gy,
     * as the reference does), W2 = wtx * wty; intgrt2d: r(k) = sum_q2 W2 F2(q2,k) f(q2). */
    int T2;
    double F2[HP_TET_MAXG * HP_TET_MAXG][HP_TET_MAXT], DX2[HP_TET_MAXG * HP_TET_MAXG][HP_TET_MAXT];
    double DY2[HP_TET_MAXG * HP_TET_MAXG][HP_TET_MAXT], W2[HP_TET_MAXG * HP_TET_MAXG];
    /* tet_basis::lumpinv (tet_basis/initialize.cpp:521-808): the mass matrix
     * mm(m, k) = sum_q w F(q,m) F(q,k); at p = 1 vdiag = 1 / (mm(0,0) + ... + mm(0,3)), the
     * lumped vertex mass inverse; at p >= 2 the vertex constraint systems give sfmv [end][k]
     * (edge mode k removed from the vertex at edge end 0 / 1), ffmv [i][k] (face modes) and
     * the constrained vdiag. */
    double mm[HP_TET_MAXT][HP_TET_MAXT];
    double vdiag;
    double sfmv[2][HP_TET_MAXP - 1], ffmv[3][HP_TET_MAXP * (HP_TET_MAXP - 1) / 2];
    /* p = 3 only (lumpinv's edge-cone systems, tet_basis/initialize.cpp:846-1040, the tables of
     * minvrt's vertex-ball edge solve): ffms [face i < 3][k][side], sfms0 = sfms(0), and the
     * spoke mass coefficients mdiag / odiag; zero at other p. */
    double ffms[3][HP_TET_MAXP * (HP_TET_MAXP - 1) / 2][2];
    double sfms0, mdiag, odiag;
} hp_tet_tables;

/* Builds the tables for 1 <= p <= 4. Returns 0, or -1 for an unsupported p. */
int hp_tet_basis_build(int p, hp_tet_tables *out);

/* Tetrahedral mesh in the reference's conventions (tet_mesh/setup.cpp:14-374):
 * pnts [npnt][3]; tet_pnt [ntet][4] (v0 < v1 by index, positively oriented);
 * tet_seg / tet_sgn [ntet][6] (local edge i joins local vertices (2,3), (3,1),
 * (2,1), (1,0), (2,0), (3,0)); tet_tri / tet_rot [ntet][4] (face i opposite vertex
 * i, rot +1 in the tetrahedron that numbered the face, -1 in the other); vol
 * [ntet] = |triple product| = 6 x volume (tet(tind).vol). */
typedef struct hp_tet_mesh_desc {
    int npnt, nseg, ntri, ntet;
    const double *pnts;
    const int *tet_pnt, *tet_seg, *tet_sgn, *tet_tri, *tet_rot;
    const double *vol;
} hp_tet_mesh_desc;

typedef struct hp_tet_ctx hp_tet_ctx;
struct hp_phys_params;

/* One tet_hp ins level on one GPU (device < 0: the current one; stream NULL: a
 * private stream). State and residual layouts, 4 variables (u, v, w, p):
 * vertices [npnt][4], edges [nseg][em][4], faces [ntri][fm][4], interiors
 * [ntet][im][4]; edge and face modes in the global orientation (tet_hp::ug). */
int hp_tet_create(const hp_tet_mesh_desc *mesh, const hp_tet_tables *basis, const struct hp_phys_params *phys,
                  int device, void *stream, hp_tet_ctx **out);
int hp_tet_destroy(hp_tet_ctx *ctx);
int hp_tet_upload_state(hp_tet_ctx *ctx, const double *ugv, const double *uge, const double *ugf, const double *ugi);
int hp_tet_download_state(hp_tet_ctx *ctx, double *ugv, double *uge, double *ugf, double *ugi);
/* which = 0: res (tet_hp::rsdl's output, res_r folded in); 1: res_r */
int hp_tet_download_residual(hp_tet_ctx *ctx, int which, double *v, double *e, double *f, double *i);
/* tet_hp_ins::setup_preconditioner (diagonal): tau and the element diagonals
 * iprcn, summed into vertex / edge / face diagonals. Returns > 0 if an element has
 * a non-positive volume or the state has NaNs. */
int hp_tet_setup_preconditioner(hp_tet_ctx *ctx);
int hp_tet_download_prcn(hp_tet_ctx *ctx, double *tau, double *iprcn); /* [ntet][2], [ntet][4] */
/* tet_hp::rsdl(stage) (tet_hp/update.cpp:9-118): enqueue only / enqueue and wait */
int hp_tet_enqueue_rsdl(hp_tet_ctx *ctx, int stage);
int hp_tet_rsdl(hp_tet_ctx *ctx, int stage);
int hp_tet_sync(hp_tet_ctx *ctx);
const char *hp_tet_last_error(void);

/* The smoother of hp_tet_update, hp_tet_solve and hp_tet_solve_mg: kind 0 = the JACOBI
 * build (jacobian_diagonal + jacobi_relaxation, tet_hp/jacobi.cpp:14-111; the default);
 * kind 1 = the default build's tet_hp::minvrt (tet_hp/setup_preconditioner.cpp:11-221 with
 * the inversion of tet_hp::setup_preconditioner, :428-470), built for p = 1 (res.v *= vdiag /
 * vprcn) and p = 2 (edge modes removed from the vertices with sfmv, vertex scaling, vertex
 * values times the element diagonal removed from the edge modes with mm, edge scaling by
 * 100 / eprcn), with the rows no essential condition fixes. kind 1 at p > 2 returns
 * HP_EINVAL. */
int hp_tet_set_smoother(hp_tet_ctx *ctx, int kind);
/* Rows fixed by essential conditions (bdry_ins::inflow on boundary faces,
 * tet_hp/ins/bdry_ins.h:141-183): masks [npnt][4], [nseg][4], [ntri][4], 1 = zero the
 * residual of that (entity, variable) in every mode. */
int hp_tet_set_dirichlet(hp_tet_ctx *ctx, const unsigned char *mv, const unsigned char *me,
                         const unsigned char *mf);
/* Boundary faces with a flux, added into res at every rsdl before the element loop
 * (hp_face_bdry::rsdl of bdry_ins::neumann / inflow, tet_hp/ins/bdry.cpp:16-102, fluxes
 * tet_hp/ins/bdry_ins.h:85-132; straight faces). Per face b: face_tri [b] its global face;
 * face_pnt [b][3] its vertices (tri.pnt, with (p1 - p0) x (p2 - p0) pointing out of the
 * domain); face_seg / face_sgn [b][3] face edge i, opposite face vertex i, and +1 where the
 * global edge runs from face vertex (i+1)%3 to (i+2)%3, else -1 (tri.seg / tri.sgn); kind [b]
 * 0 = inflow (continuity flux rho u.n only), 1 = neumann (also rho (u.n) u + p n with the
 * pressure pbc [b][G*G] at the face's Gauss points, point i * G + j; NULL if no neumann face).
 * The normal is d(x)/dr x d(x)/ds of the face map, as in neumann::element_rsdl. nface = 0
 * removes them. */
int hp_tet_set_flux_faces(hp_tet_ctx *ctx, int nface, const int *face_tri, const int *face_pnt,
                          const int *face_seg, const int *face_sgn, const int *kind, const double *pbc);
/* tet_hp::jacobian_diagonal (tet_hp/jacobi.cpp:32-111): finite-difference diagonal of every
 * element Jacobian at stage 0, summed into the global diagonal. Needs tau. */
int hp_tet_jacobian_diagonal(hp_tet_ctx *ctx);
int hp_tet_download_jacobian_diagonal(hp_tet_ctx *ctx, double *v, double *e, double *f, double *i);
/* tet_hp::update of the reference's JACOBI build (tet_hp/update.cpp:181-390 with
 * jacobi_relaxation, jacobi.cpp:14-30): nstage stages of rsdl, essential rows zeroed,
 * res = 0.5 res / jacob_diag, ug = ug0 - alpha(stage) cfl res. */
int hp_tet_enqueue_update(hp_tet_ctx *ctx);
int hp_tet_update(hp_tet_ctx *ctx);
/* L2 norm of rsdl(nstage) over the rows no essential condition fixes */
int hp_tet_resnorm(hp_tet_ctx *ctx, double *l2);
/* setup_preconditioner + jacobian_diagonal, then updates until the residual norm has
 * dropped by `drop` (checked every check_every updates) or max_updates */
int hp_tet_solve(hp_tet_ctx *ctx, double drop, int max_updates, int check_every, double *hist, int cap,
                 int *nhist, double *seconds, int *updates);

/* Multigrid (tet_hp/mg_restrict.cpp, mg_prolongate.cpp, tri_mesh/blocks.cpp:1267 cycle).
 * p-level: `coarse` has fine's mesh at a lower p (the hierarchical modes truncate).
 * h-level (both p = 1): f2c_tet / f2c_w [fine npnt][4]: the coarse tetrahedron holding
 * each fine vertex and its barycentric weights; c2f_tet / c2f_w [coarse npnt][4] the
 * same in the fine mesh. fadd scales the FAS source dres = fadd res0 - res. */
int hp_tet_mg_attach_p(hp_tet_ctx *coarse, hp_tet_ctx *fine, double fadd);
int hp_tet_mg_attach_h(hp_tet_ctx *coarse, hp_tet_ctx *fine, const int *f2c_tet, const double *f2c_w,
                       const int *c2f_tet, const double *c2f_w, double fadd);
/* vw cycles per level (1 V, 2 W), itercrsn / iterrfne updates before / after the coarse
 * correction, until the finest residual norm drops by `drop` or max_cycles; each level's
 * preconditioner is set up on its first visit. Levels share one stream. */
int hp_tet_solve_mg(hp_tet_ctx **levels, int nlevels, double drop, int max_cycles, int vw, int itercrsn,
                    int iterrfne, double *hist, int cap, int *nhist, double *seconds, int *cycles);
/* hp_tet_solve_mg inside FP64 defect correction (no counterpart in the reference): each
 * cycle takes the FP64 residual R64(u) of the finest level as the source of one FP32
 * cycle on a correction d about the base state b = fp32(u) of every level (b restricted
 * down the levels), with the residual in correction form R(b + d) - R(b) + source
 * (tet_hp::rsdl's element loop on TF32 tensor cores, FP32 accumulation; the FAS term
 * below the finest level), smoothed as hp_tet_solve_mg smooths (JACOBI relaxation or
 * minvrt at p <= 2, the preconditioners set up once at the initial state and copied to
 * FP32); then u += d in FP64. Convergence is judged by the FP64 residual norm, so the
 * converged state is the FP64 one. Flux faces must be inflow faces (HP_ENOTSUP
 * otherwise). Arguments as hp_tet_solve_mg. */
int hp_tet_solve_mg_mixed(hp_tet_ctx **levels, int nlevels, double drop, int max_cycles, int vw, int itercrsn,
                          int iterrfne, double *hist, int cap, int *nhist, double *seconds, int *cycles);

/* Learned correction of the smoother (no counterpart in the reference; the 3D form of
 * include/hp_mlp.h's hook on tri_hp's preconditioner). A per-tetrahedron log-scale c
 * (clamped to +-clamp) multiplies that tetrahedron's contributions to the Jacobian
 * diagonal of the JACOBI smoother (hp_tet_jacobian_diagonal) and to the diagonal blocks
 * of minvrt's preconditioner (hp_tet_setup_preconditioner), so it changes the local
 * pseudo-time step, never the residual. hp_tet_set_prcn_scale takes device scales
 * [ntet] (NULL: none); hp_tet_set_prcn_net a network of 17 inputs and 1 output
 * (hp_mlp) evaluated at every set-up on hp_tet_elem_features (NULL: none).
 * hp_tet_elem_features writes the inputs [ntet][17] (per variable the mean and range of
 * the vertex values and the rms of the edge, face and interior modes; log volume, log
 * longest edge, longest edge^3 / volume, log(1 + cell Peclet); p / 4);
 * hp_tet_elem_resnorm the sum of squares of each tetrahedron's residual coefficients
 * [ntet] (after a residual evaluation). Device pointers, the context's stream. */
struct hp_mlp;
int hp_tet_set_prcn_scale(hp_tet_ctx *ctx, const float *d_logscale, float clamp);
int hp_tet_set_prcn_net(hp_tet_ctx *ctx, struct hp_mlp *net, float clamp);
int hp_tet_elem_features(hp_tet_ctx *ctx, float *d_feat);
int hp_tet_elem_resnorm(hp_tet_ctx *ctx, double *d_out);

/* Measurement helper (no counterpart in the reference): the FP64 tensor-core
 * (mma.m8n8k4.f64) throughput of this GPU, from independent accumulation chains
 * on every SM for about `ms` milliseconds. Writes TFLOP/s (2 flops per multiply-add). */
int hp_tet_fp64_mma_peak(int device, double ms, double *tflops);

#ifdef __cplusplus
}
#endif
#endif

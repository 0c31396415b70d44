/*
 * hp_gpu.h — C-ABI of the B200 element-residual / multistage-smoothing library.
 *
 * The library replaces the hot path of hp-multiphysics' 2D solver behind the
 * same seams the reference exposes through its C++ virtual interfaces:
 *
 *   multigrid_interface (tri_mesh/block.h:213-267), implemented by tri_hp
 *   (tri_hp/tri_hp.h:207-248): setup_preconditioner(), rsdl(), update(),
 *   mg_restrict(), mg_prolongate(), maxres().
 *   Physics plug-ins tri_hp_ins / tri_hp_cd: element_rsdl(), setup_preconditioner().
 *   Basis: tri_basis_interface (tri_basis/tri_basis.h:32-211).
 *
 * A reference-side subclass (tri_hp_gpu : tri_hp_ins / tri_hp_cd) overrides
 * those virtuals and forwards to the calls below, so block::cycle
 * (tri_mesh/blocks.cpp:1267-1348) stays unchanged. Plain pointers and sizes
 * only; every call returns an int status: 0 = ok, > 0 = count of bad elements
 * (setup_preconditioner), < 0 = error (see HP_E*). Host arrays are caller-owned
 * and copied; device memory is owned by the context. Calls on one context are
 * stream-ordered on the context's stream; the only host synchronisations are in
 * the calls that return numbers to the host (maxres, norms, downloads, error
 * counts).
 *
 * Array layouts follow the reference's blitz arrays (row-major):
 *   ug.v / res.v  [npnt][NV]         (tri_hp.h:71-75)
 *   ug.s / res.s  [nseg][sm][NV]
 *   ug.i / res.i  [ntri][im][NV]
 *   vprcn [npnt][NV], sprcn [nseg][NV], tprcn [ntri][NV]  (tri_hp.h:139-141)
 */
#ifndef HP_GPU_H
#define HP_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define HP_MAXP 8
#define HP_MXGP (HP_MAXP + 1)                      /* Gauss points per direction, p+1 */
#define HP_MXX (HP_MAXP + 2)                       /* x-direction mode count, p+2 */
#define HP_MXTM ((HP_MAXP + 1) * (HP_MAXP + 2) / 2) /* total modes */
#define HP_MXBM (3 * HP_MAXP)                      /* boundary (vertex+side) modes */
#define HP_MXSM (HP_MAXP - 1)                      /* modes per side */
#define HP_MXIM ((HP_MAXP - 1) * (HP_MAXP - 2) / 2) /* interior modes */

#define HP_OK 0
#define HP_EINVAL -1   /* bad argument / size beyond a stated limit */
#define HP_ECUDA -2    /* a CUDA runtime call failed */
#define HP_ENOMEM -3   /* device allocation failed */
#define HP_ENOTSUP -4  /* configuration not built into this library */
#define HP_ESTATE -5   /* call order violated (e.g. update before setup_preconditioner) */

/* Basis tables of tri_basis<p,0> (tri_basis/tri_basis.h:218-291), stored with
 * the reference accessors' index order. One instance per polynomial degree. */
typedef struct hp_basis_tables {
    int p, sm, im, tm, bm, nmodx, gpx, gpn, ibwth, sbwth;
    double gx[HP_MXGP][HP_MXX], dgx[HP_MXGP][HP_MXX];
    double wtx[HP_MXGP], xp[HP_MXGP], x0[HP_MXGP];
    double gxwtx[HP_MXX][HP_MXGP], dgxwtx[HP_MXX][HP_MXGP];
    double dltx[HP_MXGP], dltx1[HP_MXGP][HP_MXGP];
    double gn[HP_MXGP][HP_MXTM], dgn[HP_MXGP][HP_MXTM];
    double wtn[HP_MXGP], np[HP_MXGP], n0[HP_MXGP];
    double gnwtn[HP_MXTM][HP_MXGP], gnwtnn0[HP_MXTM][HP_MXGP], dgnwtn[HP_MXTM][HP_MXGP];
    double dltn[HP_MXGP], dltn1[HP_MXGP][HP_MXGP], dltn2[HP_MXGP][HP_MXGP];
    double norm[HP_MXTM];
    /* lumped-mass inversion (tri_basis/initialize.cpp:590-1082) */
    double sfmv[2][HP_MXSM], ifmb[HP_MXBM][HP_MXIM], vdiag, vfms[3][HP_MXSM], sdiag[HP_MXSM];
    double sfms[HP_MXSM][HP_MXSM][3], bfmi[HP_MXBM][HP_MXIM], idiag[HP_MXIM][2];
    /* 1D side mass inversion (tri_basis/initialize.cpp:1085-1232) */
    double sfmv1d[2][HP_MXSM], vdiag1d, vfms1d[2][HP_MXSM], sdiag1d[HP_MXSM][3];
} hp_basis_tables;

/* Builds the tables of tri_basis<p,0>, 1 <= p <= HP_MAXP.
 * Replaces tri_basis<_p,ep>::initialize (tri_basis/initialize.cpp:19-35):
 * initialize_values (:161-455), lumpinv (:590-1082), lumpinv1d (:1085-1232).
 * Returns HP_EINVAL for p outside [1, HP_MAXP], > 0 if a factorisation failed. */
int hp_basis_build(int p, hp_basis_tables *out);

/* Boundary-edge kinds. Bits 0..7: essential (Dirichlet) variable mask, as the
 * reference's essential_indices (tri_hp/hp_boundary.h:119); bits 8..11: flux
 * form of hp_edge_bdry::rsdl (tri_hp/hp_boundary.cpp:1028-1049). */
#define HP_BC_ESSENTIAL(n) (1 << (n))
#define HP_BC_FLUX_NONE (0 << 8)        /* all-essential edge: flux identically zero */
#define HP_BC_FLUX_INS_GENERIC (1 << 8) /* bdry_ins::generic::flux (ins/bdry_ins.h:35-50) */
#define HP_BC_FLUX_MASK (0xF << 8)

/* Mesh, as tri_mesh's pnts / seg / tri arrays (tri_mesh/tri_mesh.h:46-98).
 * tri.seg(j) is the side opposite tri.pnt(j); tri.sgn(j) = +1 when the segment
 * runs counter-clockwise for that triangle (tri_mesh/setup.cpp:76-145).
 * seg.tri(k) = -1 on the domain boundary. Boundary edges: the segments of every
 * hp_edge_bdry, each with its kind and, for HP_BC_FLUX_INS_GENERIC, the value of
 * the boundary-condition pressure ibc->f(NV-1, x) at the edge's gpx Gauss points
 * (bseg_pibc [nbseg][gpx], may be NULL otherwise). */
typedef struct hp_mesh_desc {
    int npnt, nseg, ntri;
    const double *pnts;   /* [npnt][2] */
    const int *seg_pnt;   /* [nseg][2] */
    const int *seg_tri;   /* [nseg][2] */
    const int *tri_pnt;   /* [ntri][3] */
    const int *tri_seg;   /* [ntri][3] */
    const int *tri_sgn;   /* [ntri][3] */
    int nbseg;
    const int *bseg;      /* [nbseg] segment index */
    const int *bseg_kind; /* [nbseg] HP_BC_* */
    const double *bseg_pibc; /* [nbseg][gpx] or NULL */
    /* Curved boundary sides: the side modes of the boundary position, the
     * reference's hp_edge_bdry::crds(indx, m, n) ([nbseg][sm][2], NULL = every side
     * straight; hp_curved_side_modes computes them as curv_init does). A triangle
     * with a side whose modes are not all zero is a curved element (tri.info > -1,
     * tri_hp::metric::setinfo, metric.cpp:44-70): its residual and preconditioner
     * use the isoparametric metrics at every quadrature point (proj_bdry of the
     * vertex and side position modes, crdtocht, gtol.cpp:204-248). */
    const double *bseg_crd;
} hp_mesh_desc;

#define HP_PHYS_CD 0  /* tri_hp_cd  (tri_hp/cd/tri_hp_cd.h:16, CONST_A) NV=1 */
#define HP_PHYS_INS 1 /* tri_hp_ins (tri_hp/ins/tri_hp_ins.h:16)          NV=3 */

/* Physics and multistage constants (tri_mesh/blocks.cpp:1124-1148,
 * tri_hp/allocate.cpp:264-276, ins/allocate.cpp:20-26, cd/allocate.cpp:25-62).
 * Steady runs only: bd0 = 0 (dtinv = 0), so the mesh velocity and the unsteady
 * sources are identically zero. */
typedef struct hp_phys_params {
    int physics;        /* HP_PHYS_CD | HP_PHYS_INS */
    int nstage;         /* <= 7 */
    double alpha[8];    /* alpha(stage), alpha(nstage) = 1 */
    double beta[8];     /* beta(stage),  beta(nstage)  = 1 */
    double cfl;         /* hp_gbl->cfl(log2p) of this level */
    double bd0;         /* must be 0 (steady) */
    double adis;        /* b0_dissipation */
    double rho, mu;     /* ins */
    double rhocv, kcond, ax, ay, src; /* cd: rho*cv, conductivity, constant velocity, constant source */
} hp_phys_params;

#define HP_PREC_FP64 0
#define HP_PREC_FP32 1

typedef struct hp_gpu_ctx hp_gpu_ctx;

/* One context per (mesh, p) level. device < 0 selects the current device.
 * stream == NULL creates a private non-blocking stream. */
int hp_gpu_create(const hp_mesh_desc *mesh, const hp_basis_tables *basis, const hp_phys_params *phys,
                  int device, void *stream, hp_gpu_ctx **out);
int hp_gpu_destroy(hp_gpu_ctx *ctx);
int hp_gpu_sizes(const hp_gpu_ctx *ctx, int *nv, int *sm, int *im); /* NV, sm, im of the level */

/* State transfer (host <-> device). Layouts as above. */
int hp_gpu_upload_state(hp_gpu_ctx *ctx, const double *ugv, const double *ugs, const double *ugi);
int hp_gpu_download_state(hp_gpu_ctx *ctx, double *ugv, double *ugs, double *ugi);
int hp_gpu_download_residual(hp_gpu_ctx *ctx, double *resv, double *ress, double *resi);
int hp_gpu_download_prcn(hp_gpu_ctx *ctx, double *vprcn, double *sprcn, double *tprcn, double *tau);

/* Device pointers of the state and residual (for callers that keep data on
 * the GPU). Any output pointer may be NULL. */
int hp_gpu_device_ptrs(hp_gpu_ctx *ctx, double **ugv, double **ugs, double **ugi, double **resv,
                       double **ress, double **resi);

/* tri_hp::rsdl(stage) (tri_hp/nstage.cpp:12-110): residual of the given stage,
 * 0 <= stage <= nstage (stage == nstage: full residual, res_r reset), left in the
 * context's FP64 res arrays. precision HP_PREC_FP64: the FP64 kernels;
 * HP_PREC_FP32: the FP32 kernels on fp32 of the state (plain form, with the level's
 * multigrid source), the result widened to FP64 (res_r is then the FP32 smoother's). */
int hp_gpu_rsdl(hp_gpu_ctx *ctx, int stage, int precision);

/* tri_hp::l2error (tri_hp/l2error.cpp:13-67) on the device: per variable the L2 norm
 * sqrt(sum err^2 wtx wtn cjcb) and the max |err| of the state against the analytic
 * field f (include/hp_host.h) at the quadrature points; curved elements use their
 * isoparametric coordinates and Jacobians. l2[NV], linf[NV]. */
struct hp_field;
int hp_gpu_l2error(hp_gpu_ctx *ctx, const struct hp_field *f, double *l2, double *linf);

/* tri_hp_{ins,cd}::setup_preconditioner + tri_hp::setup_preconditioner
 * (ins/setup_preconditioner.cpp:9-221, cd/setup_preconditioner.cpp:6-97,
 * setup_preconditioner.cpp:9-100). Returns the count of bad elements (> 0)
 * exactly where the reference sets err (non-positive area, NaN velocity). */
int hp_gpu_setup_preconditioner(hp_gpu_ctx *ctx);

/* tri_hp::minvrt (tri_hp/setup_preconditioner.cpp:102-373) on the current
 * residual, Dirichlet zeroing included. */
int hp_gpu_minvrt(hp_gpu_ctx *ctx);

/* tri_hp::update (tri_hp/nstage.cpp:256-427): nstage x (rsdl, minvrt,
 * ug = ug0 - cfl*alpha*res). */
int hp_gpu_update(hp_gpu_ctx *ctx);

/* Runs `iters` calls of update() back to back (one CUDA graph per call), with
 * setup_preconditioner() before every `prcn_interval`-th iteration (0 = only
 * before the first). Writes tri_hp::maxres of every iteration to hist[iters]
 * (may be NULL). */
int hp_gpu_iterate(hp_gpu_ctx *ctx, int iters, int prcn_interval, double *hist);

/* tri_hp::maxres (tri_hp/allocate.cpp:496-525): per-variable max over
 * vertices of |res.v| as left by the last minvrt; out[NV], returns via *mx the
 * max over variables. */
int hp_gpu_maxres(hp_gpu_ctx *ctx, double *out, double *mx);

/* Unpreconditioned residual norm over all modes: computes rsdl(nstage) and
 * returns sqrt(sum res^2) and max |res| over every v/s/i coefficient. */
int hp_gpu_resnorm(hp_gpu_ctx *ctx, double *l2, double *linf);

/* Element kernel of rsdl (no counterpart in the reference, which has one CPU loop,
 * tri_hp/nstage.cpp:52-73). HP_ELEM_TENSOR (the default for ins at p >= 3): projection,
 * intgrtrs and the strong residual of two triangles per warp on the FP64 tensor cores
 * (mma.m8n8k4.f64) with dense per-point operators, and for the FP32 smoother's
 * correction form four triangles per warp on TF32 (mma.m16n8k8); HP_ELEM_POINT (the
 * default for ins at p = 1): four lanes per triangle, one per Gauss point, the point
 * shares of intgrtrs summed by shuffles; HP_ELEM_SCALAR (the default at p = 2, and cd
 * always): the sum-factorised warp kernel. All give the reference's residual up to
 * rounding. HP_ENOTSUP when the kernel is not built for the context's physics and p. */
#define HP_ELEM_SCALAR 0
#define HP_ELEM_TENSOR 1
#define HP_ELEM_POINT 2
int hp_gpu_set_element_kernel(hp_gpu_ctx *ctx, int kind);

/* Stream-ordered forms without a host synchronisation (for callers that time or
 * capture the work themselves): rsdl(stage) with res_r folded into res, and one
 * update(). */
int hp_gpu_enqueue_rsdl(hp_gpu_ctx *ctx, int stage);
int hp_gpu_enqueue_update(hp_gpu_ctx *ctx);
/* Stream-ordered state upload and residual download: the copies are queued on the
 * context's stream and the call returns at once. The host arrays must stay valid, and for
 * the copies to run asynchronously they must be page-locked, until hp_gpu_sync(ctx)
 * returns. Two contexts on two streams can then overlap one residual's copies with
 * another's kernels. */
int hp_gpu_enqueue_upload_state(hp_gpu_ctx *ctx, const double *ugv, const double *ugs, const double *ugi);
int hp_gpu_enqueue_download_residual(hp_gpu_ctx *ctx, double *resv, double *ress, double *resi);
/* The element-residual kernel alone (the loop over elements of tri_hp::rsdl,
 * nstage.cpp:52-73: ugtouht, element_rsdl, lftog), for timing it in isolation. */
int hp_gpu_enqueue_element_rsdl(hp_gpu_ctx *ctx, int stage);

/* Stored element operators for the linear cd residual. No counterpart in the
 * reference: tri_hp::rsdl (nstage.cpp:52-73) recomputes element_rsdl
 * (tri_hp/cd/rsdl.cpp:14-154) every call; for cd the element residual is affine
 * in the element's coefficients, lf_im = A_im u and lf_re = beta (A_re u + b_re),
 * so on = 1 builds A_im, A_re, b_re of every element once (FP64 by the element
 * kernel applied to unit vectors, plus an FP32 copy for the FP32 smoother), and
 * every later rsdl of either precision becomes a streamed batched mat-vec with
 * the same result up to rounding. The build needs tau: it runs
 * setup_preconditioner() first when that has not run (cd tau depends on the
 * geometry and the fixed parameters only, so the operators stay valid for every
 * later state). on = 0 returns to the matrix-free kernel (the storage is kept
 * until hp_gpu_destroy). HP_ENOTSUP for ins. */
int hp_gpu_set_element_matrices(hp_gpu_ctx *ctx, int on);

/* tri_hp::element_jacobian (tri_hp/nstage.cpp:131-165, fixed mesh) of every element,
 * batched on the GPU: the finite-difference Jacobian of the stage-0 element residual
 * lf_re + lf_im with respect to the element's coefficients, column (mode, var) from the
 * residual with uht(var)(mode) raised by dw(var) = 1e-8 sum_{i<3} |uht(var)(i)| + 1e-8.
 * K (host) [ntri][tm*NV][tm*NV], row i*NV + n, column mode*NV + var. Needs
 * setup_preconditioner (tau). Device scratch of ntri*(tm*NV)^2 doubles is taken from
 * the context's pool for the call. */
int hp_gpu_element_jacobian(hp_gpu_ctx *ctx, double *K);

/* Convergence driver. Runs smoothing until the unpreconditioned FP64 residual
 * norm ||R64(u)||_2 (all v/s/i modes of rsdl(nstage), without the rows of
 * essential boundary values, which the boundary condition replaces) has dropped by `drop` from
 * its value at entry, or `max_updates` multistage updates have run.
 *   mode HP_PREC_FP64: plain FP64 update() sweeps, the norm checked every
 *     `check_every` updates (block::cycle with itercrsn sweeps, blocks.cpp:1267).
 *   mode HP_PREC_FP32: defect correction. Each cycle takes the FP64 residual
 *     R64(u) as the source of an FP32 smoother that runs `inner` multistage
 *     updates on a correction d about the base u, with the residual in correction
 *     form R(u + d) - R(u) + R64(u) (the coarse-level source of mg_source,
 *     nstage.cpp:113-129); then u += d in FP64 and R64(u) is evaluated again.
 * setup_preconditioner() runs at entry and every `prcn_every` checks (0: once).
 * hist[0..*n_hist) receives ||R64|| / ||R64(entry)|| at every check; *seconds is
 * the device time of the whole solve (CUDA events), *updates the updates run. */
int hp_gpu_solve(hp_gpu_ctx *ctx, int mode, double drop, int max_updates, int inner, int check_every,
                 int prcn_every, double *hist, int hist_cap, int *n_hist, double *seconds, int *updates);

/* Multigrid. A coarse context is attached to its fine context either as a
 * p-level (same mesh, lower p: the hierarchical basis makes its modes a subset
 * of the fine ones, tri_hp/movco.cpp:17-39) or as an h-level (a coarser mesh at
 * p = 1, with each fine vertex's containing coarse triangle and barycentric
 * weights f2c_tri/f2c_wt [fine npnt][3], and each coarse vertex's containing fine
 * triangle c2f_tri/c2f_wt [coarse npnt][3]: tri_mesh::mgconnect,
 * tri_mesh/connect.cpp:49-87). Attaching gives the coarse level a FAS source
 * dres = fadd*res0 - res(first) that enters every stage residual
 * (tri_hp::mg_source, nstage.cpp:113-129; hp_fadd default 1). */
int hp_gpu_mg_attach_p(hp_gpu_ctx *coarse, hp_gpu_ctx *fine, double fadd);
int hp_gpu_mg_attach_h(hp_gpu_ctx *coarse, hp_gpu_ctx *fine, const int *f2c_tri, const double *f2c_wt,
                       const int *c2f_tri, const double *c2f_wt, double fadd);
/* tri_hp::mg_restrict (movco.cpp:4-106): needs the fine level's full residual
 * (hp_gpu_rsdl(fine, nstage)); sets the coarse state, its copy at entry
 * (vug_frst) and the restricted residual res0. As the reference's isfrst, the
 * FAS source is formed at the coarse level's first residual evaluation after
 * this call (rsdl, update, iterate or a cycle), which therefore needs that
 * level's setup_preconditioner() first (its tau enters res(first)). */
int hp_gpu_mg_restrict(hp_gpu_ctx *coarse);
/* tri_hp::mg_prolongate (movfin.cpp:7-82): fine state += coarse correction. */
int hp_gpu_mg_prolongate(hp_gpu_ctx *coarse);
/* block::cycle (tri_mesh/blocks.cpp:1267-1348) over levels[0] (finest) ..
 * levels[nlevels-1], each attached to the previous one: vw cycles per level,
 * itercrsn updates before and iterrfne after the coarse-grid correction,
 * setup_preconditioner() on entry to each level when eval_prcn. */
int hp_gpu_vcycle(hp_gpu_ctx **levels, int nlevels, int vw, int itercrsn, int iterrfne, int eval_prcn);
/* Cycles until ||R64|| on levels[0] (as in hp_gpu_solve) drops by `drop` or
 * max_cycles ran; preconditioners on the first cycle and every prcn_every
 * cycles. hist gets the drop after each cycle; *seconds device time. */
int hp_gpu_solve_mg(hp_gpu_ctx **levels, int nlevels, double drop, int max_cycles, int vw, int itercrsn,
                    int iterrfne, int prcn_every, double *hist, int hist_cap, int *n_hist, double *seconds,
                    int *cycles);

/* One whole cycle of block::cycle as a single CUDA graph (all levels created on
 * one stream, every level's preconditioner set up before capture). With
 * eval_prcn the graph also re-evaluates every level's preconditioner at the
 * points where block::cycle does (evaluate_preconditioner, blocks.cpp:1279,1335;
 * bad elements accumulate in the context's count, read by the solve driver);
 * without, the preconditioners stay frozen inside the graph. The opaque handle is
 * replayed with hp_gpu_launch_vcycle (count cycles back to back on the finest
 * level's stream) and freed with hp_gpu_destroy_vcycle. */
int hp_gpu_capture_vcycle(hp_gpu_ctx **levels, int nlevels, int vw, int itercrsn, int iterrfne, int eval_prcn,
                          void **graph);
int hp_gpu_launch_vcycle(void *graph, hp_gpu_ctx *finest, int count);
int hp_gpu_destroy_vcycle(void *graph);
/* hp_gpu_solve_mg with the cycle replayed from captured graphs: the first cycle
 * runs level by level with the preconditioners evaluated; later cycles replay the
 * graph with the preconditioner set-ups inside when nc % prcn_every == 0 (the
 * reference's preconditioner_interval), else the frozen one (prcn_every = 0:
 * always); `check_every` cycles between residual checks. Returns > 0 (bad-element
 * count) if a preconditioner set-up inside the graph met bad elements. */
int hp_gpu_solve_mg_graph(hp_gpu_ctx **levels, int nlevels, double drop, int max_cycles, int vw, int itercrsn,
                          int iterrfne, int check_every, int prcn_every, double *hist, int hist_cap, int *n_hist,
                          double *seconds, int *cycles);

/* Multigrid inside FP64 defect correction: each cycle evaluates the FP64
 * residual R64(u) on levels[0], runs one FP32 cycle of the hierarchy on the
 * correction equation (every level in correction form about its base state,
 * fp32 of u restricted down the levels, FP32 FAS sources between levels), and
 * adds the fine correction to u in FP64. Preconditioners (FP64, copied to FP32)
 * on the first cycle and every prcn_every cycles. Arguments as hp_gpu_solve_mg. */
int hp_gpu_solve_mg_mixed(hp_gpu_ctx **levels, int nlevels, double drop, int max_cycles, int vw, int itercrsn,
                          int iterrfne, int prcn_every, double *hist, int hist_cap, int *n_hist, double *seconds,
                          int *cycles);

/* Diagnostic: n multistage updates of the FP32 smoother in plain form, from
 * fp32(u), written back to the FP64 state (compares the FP32 kernels with the
 * FP64 ones update by update). Needs setup_preconditioner() first. */
int hp_gpu_fp32_updates(hp_gpu_ctx *ctx, int n);

/* Launch-shape autotuner (no counterpart in the reference; the north star's
 * per-level tile-shape choice). Each context is one mesh level at one p, so the
 * fastest launch shapes differ between the levels of a hierarchy. Times, on this
 * context's own mesh, `reps` launches of each candidate shape of
 *   the element part: matrix-free kernel CTAs per SM in {4, 8, 16}, or with stored
 *     cd operators tiles per pipeline phase {1, 2} x CTAs per SM {all that fit, 4, 2};
 *   the minvrt kernels: threads per CTA {64, 128, 256};
 * in FP64 and in FP32 (allocating the FP32 smoother state), and keeps the fastest
 * for every later launch of that precision. Results do not depend on the shapes
 * beyond rounding of the atomic scatter. Needs setup_preconditioner(); leaves the
 * state unchanged and the residual arrays unspecified. */
int hp_gpu_autotune(hp_gpu_ctx *ctx, int reps);
/* The shapes in use: shapes[8] = {elem_cap, emat_tpp, emat_ctas, minv_threads} for
 * FP64 then FP32 (emat_ctas 0 = all that fit); ms[4] = the tuned element-part and
 * minvrt times (ms) for FP64 then FP32 (0 before hp_gpu_autotune). Either may be NULL. */
int hp_gpu_get_tuning(const hp_gpu_ctx *ctx, int *shapes, float *ms);

/* Synchronises the context's stream and returns the first sticky error. */
int hp_gpu_sync(hp_gpu_ctx *ctx);

/* Last error text (thread-local), "" if none. */
const char *hp_gpu_last_error(void);

/* Residual norm that allocates nothing. No counterpart in the reference.
 * For callers that cannot call cudaMalloc when they need the norm: an
 * application that gives all device memory to its own pool at start-up and
 * forbids further cudaMalloc / cudaFree, or a solver embedded in a host program
 * whose device-memory budget is fixed before the solve. Same result as
 * hp_gpu_resnorm's reduction (sqrt of the sum of squares and max |x| over
 * res.v, res.s, res.i), but over caller-owned device arrays (e.g. from
 * hp_gpu_device_ptrs) and with a fixed static device scratch of
 * HP_NOALLOC_MAX_CHUNKS partials, held by every GPU that loads the library until
 * exit. At most HP_NOALLOC_MAX_CHUNKS chunks of HP_NOALLOC_CHUNK values per call
 * (nv, ns, ni each rounded up to whole chunks); larger inputs return HP_EINVAL
 * with a message from hp_noalloc_last_error(). The first call in each CUDA
 * context looks up the scratch's device address. The call launches two kernels
 * on `stream`, copies the two results to the host and synchronises `stream`
 * before returning. All calls share the scratch: calls that overlap on the GPU
 * race, so the caller serialises them. */
#define HP_NOALLOC_CHUNK 65536
#define HP_NOALLOC_MAX_CHUNKS 4096
int hp_resnorm_noalloc(const double *resv, long long nv, const double *ress, long long ns, const double *resi,
                       long long ni, double *l2, double *linf, void *stream);
const char *hp_noalloc_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* HP_GPU_H */

/*
 * hp_host.h — host-side set-up helpers of the B200 library (C-ABI).
 *
 * These replace the reference's initial-condition and error helpers around the
 * hot path. The reference evaluates fields through muParser
 * (symbolic_function/symbolic_function.h); here the fields the workloads use
 * are built-in closed forms selected by hp_field.kind.
 */
#ifndef HP_HOST_H
#define HP_HOST_H

#include "hp_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

#define HP_FIELD_CONST 0     /* value prm[n] for variable n */
#define HP_FIELD_KOVASZNAY 1 /* prm[0] = Re (= 1/mu with rho = 1); Spatial Accuracy/Inputs/run.inpt:21-25 */
#define HP_FIELD_SINSIN 2    /* prm[0] * sin(pi x) sin(pi y) */
#define HP_FIELD_QUADX 3     /* prm[0] * (x - prm[1])^2 ; conv-diff/Correctness/Inputs/run.inpt ibc0 */
#define HP_FIELD_LID 4       /* u = 1 on the lid y = 1, 0 elsewhere; v = p = 0 */
#define HP_FIELD_CYLINDER 5  /* u = 1 outside the circle of centre (prm[0], prm[1]), radius prm[2], 0 on and
                                inside it; v = p = 0 (free stream past a cylinder at rest) */

typedef struct hp_field {
    int kind;
    double prm[4];
} hp_field;

/* ibc->f(n, x) (init_bdry_cndtn::f, tri_hp/tri_hp.h:41) */
int hp_field_eval(const hp_field *f, int n, double x, double y, double *out);

/* tri_hp::tobasis (tri_hp/tobasis.cpp:14-116) for straight-sided meshes:
 * vertex sampling, 1D L2 projection of each side, 2D projection of the
 * interior remainder. Output layouts ugv[npnt][NV], ugs[nseg][sm][NV],
 * ugi[ntri][im][NV]. The edge set-values pass (tobasis.cpp:111-113) is
 * hp_setvalues. */
int hp_tobasis(const hp_basis_tables *t, const hp_mesh_desc *m, int NV, const hp_field *f, double *ugv, double *ugs,
               double *ugi);

/* hp_edge_bdry::setvalues (tri_hp/hp_boundary.cpp:549-619) for the essential
 * variables of every boundary edge of m (bseg_kind bits 0..7). */
int hp_setvalues(const hp_basis_tables *t, const hp_mesh_desc *m, int NV, const hp_field *f, double *ugv,
                 double *ugs);

/* hp_edge_bdry::curv_init (tri_hp/hp_boundary.cpp:621-678): side modes of curved
 * boundary positions. For each of nside sides, ends[k] = {x0, y0, x1, y1} are its
 * end vertices and curve[k][i] = {x, y} the boundary point that
 * base.mvpttobdry maps the straight chord's i-th Gauss point (parameter xp(i)) to;
 * modes[k][m] = {x, y} receives the L2 projection of (curve - chord) onto the side
 * modes (1D intgrt with the sdiag1d band inversion), the bseg_crd input of
 * hp_mesh_desc. */
int hp_curved_side_modes(const hp_basis_tables *t, int nside, const double *ends, const double *curve, double *modes);

/* tri_hp::l2error (tri_hp/l2error.cpp:13-67): per-variable L2 and Linf error of
 * the state against f at the Gauss points. */
int hp_l2error(const hp_basis_tables *t, const hp_mesh_desc *m, int NV, const hp_field *f, const double *ugv,
               const double *ugs, const double *ugi, double *l2, double *linf);

#ifdef __cplusplus
}
#endif

#endif

/*
 * TEST INFRASTRUCTURE — NOT PART OF THE PRODUCT.
 *
 * CPU FP64 restatement of the hot path of `lippsLFroude_implgwopks3D_unstr3.f` (ref.f),
 * loop by loop and in the reference's summation order, used only as the checker by the
 * tests, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg.  The product library
 * (src_b200/) never links, loads or calls it.
 *
 * Parity status: unpinned by the reference itself.  The reference ships no tests, fixtures or
 * golden vectors, and no Fortran compiler exists on either machine, so the restatement cannot
 * be diffed against the Fortran.  It is pinned instead by known-answer properties (dual-cell
 * closure, exact conservation, symmetry of laplc, manufactured GCR solutions, MPDATA
 * constancy/positivity/bounds) checked in tests/.  tests/golden/ holds reference-format input
 * decks with this restatement's results on them, ready to diff against the Fortran wherever a
 * compiler for it exists.
 *
 * Arrays are 0-based; the mesh is taken from the same mpg_mesh_ref struct the product takes.
 */
#ifndef MPGCR_ORACLE_H
#define MPGCR_ORACLE_H

#include "../include/mpgcr.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc orc;

orc   *orc_create(const mpg_params *prm, const mpg_mesh_ref *mesh);
void   orc_destroy(orc *o);
/* 0 (default): global sums in the reference's sequential order; 1: in the GPU kernels' fixed
 * reduction order, so that CPU and GPU runs can be compared bit for bit */
void   orc_set_reduction(orc *o, int blocked);
/* 1 (default): reproduce the corner-minimum slip of mpdatamper (ref.f:3853-3866, minima taken
 * over unkmx); 0: take them over unkmn like the pair lists. */
void   orc_set_ref_bugs(orc *o, int on);
/* NEW (iprc = 4): the column blocks of laplc, lo = A[k][k-2], dg = A[k][k], hi = A[k][k+2] per
 * node, and the preconditioner that solves them (Thomas on even and odd levels). */
void   orc_wide_entries(orc *o, int impfl, double *lo, double *dg, double *hi);
void   orc_wide_factors(orc *o, int impfl, double *lo, double *m, double *cp);
void   orc_wide_solve(orc *o, const double *rhs, double *zout, int impfl);
/* mg_flag = 1: attach the coarse (level 1, mesh3d_c.d) or coarsest (level 2, mesh3d_cc.d) mesh of
 * precon's V-cycle (ref.f:618-748) before orc_setup, with its match array (coarse node -> node of
 * the next finer mesh, 0-based) or NULL to find it by coordinates as `matching` does
 * (ref.f:2684-2720).  params.mg_bugs selects the reference's indexing or the corrected one.
 * Returns 0, or 1 for an argument the levels cannot use. */
int    orc_set_coarse(orc *o, int level, const mpg_mesh_ref *mesh, const int *match);
/* the V-cycle's transfers on their own: restriction_unstr / prolongation_unstr (ref.f:757-951)
 * between level flg-1 and level flg (0 = the fine mesh), and the node count of a level */
void   orc_mg_restrict(orc *o, const double *s, double *sc, int flg);
void   orc_mg_prolong(orc *o, const double *sc, double *s, int flg);
int    orc_level_npoin(const orc *o, int level);
/* pointer to a field (same ids as the product) — n = npoin doubles */
double *orc_field(orc *o, int fid);
int    orc_npoin(const orc *o);

void orc_derivative(orc *o, const double *unk, double *out, int idx);
void orc_bcv(orc *o, double *u, double *v, double *w, double flag);
void orc_laplc(orc *o, const double *press, double *alap, int impfl);
void orc_prfr(orc *o, const double *press, const double *ustr, const double *vstr,
              const double *wstr, double *uout, double *vout, double *wout, int impfl);
void orc_div(orc *o, const double *ua, const double *va, const double *wa, double *rhs,
             int iflg, mpg_diag *diag);
void orc_precon(orc *o, const double *rhs, double *p, double *r, int iprc, int impfl);
void orc_gcrk(orc *o, double *p, const double *u1, const double *v1, const double *w1,
              double *u2, double *v2, double *w2, int impfl, mpg_gcr_stats *st);
void orc_mpdatamper(orc *o, double *unk, int iflag);
void orc_mpdatam(orc *o, double *unk, int iflag);
void orc_courant(orc *o, int iflag, mpg_diag *diag);
void orc_stats(orc *o, mpg_diag *diag);
void orc_setup(orc *o, mpg_diag *diag);
void orc_step(orc *o, mpg_diag *diag);
void orc_velprd(orc *o);                          /* velprd, ref.f:4448-4528 */
void orc_get_gcr_stats(orc *o, mpg_gcr_stats *st);
double orc_beta(orc *o);            /* betaunstr1 */
/* vertical-line preconditioner alone: z = M^{-1} rhs (coefficients for impfl) */
void orc_line_solve(orc *o, const double *rhs, double *z, int impfl);

#ifdef __cplusplus
}
#endif
#endif

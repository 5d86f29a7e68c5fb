/*
 * mpgcr.h — C ABI of the B200 implementation of the two hot loops of the edge-based
 * anelastic solver `lippsLFroude_implgwopks3D_unstr3.f` (the reference):
 *
 *   * MPDATA advection      : mpdatamper            (ref.f:3617-3941), mpdatam (ref.f:3029-3311)
 *                             + derivative (ref.f:3943-4022)
 *   * GCR(k) pressure solve : gcrk (ref.f:1776-1972), precon (ref.f:482-753), laplc (ref.f:1288-1353),
 *                             prfr (ref.f:1536-1580), div (ref.f:2096-2170), bcv (ref.f:1583-1643)
 *
 * and of the node loops of the time-step driver `mpsolver` (ref.f:58-479) that sit between them,
 * so that every field stays resident on the GPU for a whole run.
 *
 * Conventions (they follow the Fortran caller):
 *   * REAL is double (the reference compiled with -fdefault-real-8 -fdefault-double-8).
 *   * INTEGER is int32; node/edge indices in mesh arrays are 1-based, as in the COMMON blocks.
 *   * 2-D Fortran arrays arrive as base pointers with their leading dimension (npoinx, nedgex,
 *     nfacesx): element (i, j) of `sn(nedgex,3)` is sn[(j-1)*nedgex + (i-1)].
 *   * Every entry point returns an int status: MPG_OK or an MPG_ERR_* code; mpg_last_error()
 *     gives a one-line message for the calling thread.  Nothing here calls exit() or stop.
 *   * The reference keeps fields in COMMON blocks and mpsolver locals.  Here they live in a
 *     handle on one GPU and are named by field ids (MPG_F_*); the subroutine entry points take
 *     field ids where the reference takes arrays (same argument order and meaning).
 *   * A handle is not re-entrant (neither is the reference): one thread drives one handle.
 */
#ifndef MPGCR_H
#define MPGCR_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status codes */
#define MPG_OK              0
#define MPG_ERR_ARG         1   /* bad argument (null pointer, unknown field id, bad size) */
#define MPG_ERR_CUDA        2   /* a CUDA call failed                                       */
#define MPG_ERR_MESH        3   /* mesh is not a prism-column mesh, or uses an unsupported feature */
#define MPG_ERR_NOMEM       4   /* device allocation failed                                 */
#define MPG_ERR_UNSUPPORTED 5   /* option the implementation does not provide               */
#define MPG_ERR_NUMERIC     6   /* NaN/Inf met in a solver reduction                        */

/* GCR exit status (mpg_gcr_stats.status).  The reference leaves gcrk silently in every case
 * (ref.f:1895-1896); the status makes the reason visible. */
#define MPG_GCR_CONVERGED   0   /* max|r| <= eps0/dt after >= itmn restart cycles (ref.f:1895)   */
#define MPG_GCR_STALLED     1   /* ||r||_2^2 did not decrease (ref.f:1896)                      */
#define MPG_GCR_MAXIT       2   /* itr restart cycles done without convergence                  */
#define MPG_GCR_NAN         3   /* NaN/Inf in the residual                                      */
#define MPG_GCR_FALLBACK    4   /* learned preconditioner rejected, solve redone with the plain one */

/* ---------------------------------------------------------------- run parameters */
/* One struct for the three configuration layers of the reference: inputinc.d
 * (ref.f:2293-2321), input_mg_v3.d (ref.f:2265-2276) and the constants hard-coded in
 * mpsolver (ref.f:108-138).  Fields keep the reference names. */
typedef struct mpg_params {
    /* inputinc.d */
    int32_t ntime, istst, isfera, iper;
    double  cfl, delt;
    double  p0inf, u0inf, v0inf, w0inf;
    int32_t ielast;
    double  eps0;
    int32_t itr, lord;           /* lord: GCR order (a compile-time 9 in the reference, ref.f:1782) */
    int32_t irl;                 /* absorbers on/off */
    double  dxabl, dxabr, dyabd, dyabu, dzabd, dzabu;
    double  towxl, towxr, towyd, towyu, towzd, towzu;
    /* input_mg_v3.d */
    int32_t mg_flag, sm_flag1;
    double  omega;
    int32_t itrp1, itrp2;
    /* mpsolver constants */
    int32_t implgw, lipps;
    double  strat, tetbar, g;
    /* extensions of this implementation */
    int32_t iprc;                /* 0 identity, 1 reference smoother (ref.f:587-612), 2 vertical line,
                                  * 3 learned correction of the line, 4 laplc's own column blocks:
                                  * laplc couples level k with k and k+-2 in a column, so its column
                                  * block is tridiagonal on the even and on the odd levels; iprc = 4
                                  * solves that block exactly (itrp1 relaxations like iprc = 2)     */
    int32_t nscal;               /* passive scalars advected after unk(:,1..4)                      */
    int32_t precision;           /* MPG_PREC_FP64 or MPG_PREC_MIXED                                 */
    int32_t itmn;                /* minimum restart cycles before the convergence test (3, ref.f:1809) */
    double  nn_rate;             /* iprc = 3: the network keeps being used while ||r||_2 after m GCR
                                  * iterations (m >= lord) is at most nn_rate^m times its initial
                                  * value; otherwise the plain line preconditioner takes over for
                                  * the rest of the solve.  <= 0 selects 0.98.                      */
    int32_t itraj;               /* 1: velprd trajectory prediction of the advective velocity
                                  * (ref.f:4448-4528) in set-up and every step; the reference
                                  * hard-codes 0 (ref.f:111)                                       */
    /* input_mg_v3.d, the multigrid V-cycle of precon (mg_flag = 1, ref.f:618-748): sweeps on the
     * coarse mesh before and after the coarsest one, and on the coarsest mesh (/vcycle/) */
    int32_t itrp_c1, itrp_c2, itrp_cc;
    int32_t mg_bugs;             /* mg_flag = 1: 1 reproduces the reference's indexing, 0 corrects
                                  * it.  The reference's restriction_unstr and prolongation_unstr
                                  * take the neighbour loop counter as the neighbour's node number
                                  * (ref.f:813-817, 911-915), laplc_c/laplc_cc read coefw at the
                                  * coarse node's number (ref.f:1390-1392, 1482-1484), and the
                                  * prolongation's refill pass first overwrites its own marks, so
                                  * nodes with no coarse neighbour stay zero (ref.f:929-941).
                                  * Corrected: neigh_list, coefw of the matched fine node, and
                                  * refill passes until every node has a value.                    */
} mpg_params;

#define MPG_PREC_FP64  0
#define MPG_PREC_MIXED 1

/* ---------------------------------------------------------------- mesh (reference COMMON layout) */
/* /n/ npoin,nedge,nbface,nbpoin,nboun; /xyz/ coord; /volume/ vol; /edg/ iedge; /wge/ sn;
 * /bound/ kbface,sb; /bpoints/ ibpoin,anp; /terms/ sbb; /coin/ /per2/ /per4/ periodic lists
 * (ref.f:2182-2196, read at ref.f:2437-2501, ref.f:2562-2576). */
typedef struct mpg_mesh_ref {
    int32_t npoin, nedge, nbface, nboun;
    int32_t npoinx, nedgex, nfacesx;   /* leading dimensions of the arrays below */
    const double  *coord;              /* coord(npoinx,3)  */
    const double  *vol;                /* vol(npoinx)      */
    const int32_t *iedge;              /* iedge(nedgex,2)  */
    const double  *sn;                 /* sn(nedgex,3)     */
    const int32_t *kbface;             /* kbface(nfacesx,2) (may be NULL when nbface == 0) */
    const double  *sb;                 /* sb(nfacesx,3)    */
    const int32_t *ibpoin;             /* ibpoin(nfacesx,2): node, boundary type */
    const double  *sbb;                /* sbb(nfacesx,3)   */
    const double  *anp;                /* anp(nfacesx,3)   */
    int32_t ncoin, ncoin2, ncoin4;
    int32_t ldcoin;                    /* leading dimension of icoin (nfacesx*2 in the reference) */
    const int32_t *icoin;              /* icoin(ldcoin,2)  */
    const int32_t *icoin2;             /* icoin2(nfacesx,2) */
    const int32_t *icoin4;             /* icoin4(nfacesx,4) */
} mpg_mesh_ref;

/* ---------------------------------------------------------------- outputs */
typedef struct mpg_gcr_stats {         /* /itero/ (ref.f:1953-1963) plus the exit reason */
    int32_t niter, nitsm, icount, status;
    double  eer, eem;
    double  dvmx;                      /* final max|r| (units of rhs, 1/s)       */
    double  rl2;                       /* final sum r^2                          */
    int32_t fallbacks;                 /* learned-preconditioner fallbacks taken */
    int32_t pad;
    double  rate;                      /* per-iteration contraction of ||r||_2 over the solve:
                                        * (rl2 / rl2_initial)^(1/(2*niter))                 */
} mpg_gcr_stats;

typedef struct mpg_diag {              /* per-step diagnostics printed by mpsolver (ref.f:456-459) */
    double divmx, divmn, divav, divsd; /* div(...,1)        ref.f:2148-2168 */
    double crnmx, crnmn, crnav, crnsd; /* courant(...,1)    ref.f:2076-2092 */
    int32_t icrnmx, niter, nitav;      /* node of max Courant (1-based), solver stats (ref.f:2164) */
    int32_t niter1;                    /* GCR iterations of the step's first pressure solve      */
    double eer, eem;
    double stats[16];                  /* umx,umn,uav,usd, vmx.., wmx.., tmx,tmn,tav,tsd (ref.f:2904) */
    double mass[8];                    /* sum(vol*rh0*unk(:,k)) for the prognostic fields (FP64)  */
    double smin[4], smax[4];           /* min/max of the first passive scalars                     */
    double rate1;                      /* mpg_gcr_stats.rate of the step's first pressure solve    */
    int32_t fallbacks;                 /* learned-preconditioner fallbacks in the step's solves    */
    int32_t pad;
} mpg_diag;

typedef struct mpg_info {
    int64_t npoin, nedge, ncol, nedge2d;
    int32_t nlev, precision;
    int64_t device_bytes;              /* bytes allocated on the device by the handle */
} mpg_info;

/* ---------------------------------------------------------------- field ids */
enum {
    MPG_F_UNK    = 0,    /* unk(:,1..4+nscal) : MPG_F_UNK + k-1   (u, v, w, theta', scalars)   */
    MPG_F_UNK1   = 16,   /* unk1(:,1..4)                                                        */
    MPG_F_UUU    = 20,   /* uuu(:,1..3)   momentum / velocity                                   */
    MPG_F_UUU0   = 23,   /* uuu0(:,1..3)                                                        */
    MPG_F_FRC    = 26,   /* frc(:,1..4)                                                         */
    MPG_F_UNKDASH= 30,   /* unkdash(:,1..3)                                                     */
    MPG_F_PRPOT  = 33,
    MPG_F_RHS    = 34,
    MPG_F_COUR   = 35,
    MPG_F_ALPHA  = 36,
    MPG_F_COEFW  = 37,
    MPG_F_RH0    = 38,
    MPG_F_TH0    = 39,
    MPG_F_THE    = 40,
    MPG_F_DTHEDZ = 41,
    MPG_F_D1     = 42,   /* /doperator/ d1 (compute_d_unstr)                                   */
    MPG_F_UUU1   = 43,   /* uuu1(:,1..3) velprd's predicted velocity (itraj = 1)               */
    MPG_F_WORK   = 48,   /* 8 caller-usable work arrays MPG_F_WORK + 0..7                       */
    MPG_F_COUNT  = 56
};

typedef struct mpg_solver *mpg_handle;

/* ---------------------------------------------------------------- lifecycle */
/* Uploads the mesh once, detects the prism-column structure (columns of equal (x,y), the same
 * number of levels everywhere, 1 to 128 of them, horizontal edges between equal levels), packs it column-major
 * (level fastest) and allocates every field on `device`.  Replaces the mesh part of `input`
 * (ref.f:2343-2641) and the static COMMON storage.  With the environment variable
 * MPG_LAPLC_FUSED=1 set at this call, laplc runs as one persistent launch instead of two
 * (bit-identical results; slower on the 21.2M-node workload measured; not with copy lists). */
int mpg_create(const mpg_params *prm, const mpg_mesh_ref *mesh, int device, mpg_handle *out);
int mpg_destroy(mpg_handle h);
/* Host-only check of a mesh: runs the prism-column detection of mpg_create without touching a
 * GPU and fills npoin, nedge, ncol, nedge2d and nlev of `info` (device_bytes = 0; precision =
 * 1 when per-node sums can follow the reference's edge order exactly, else 0). */
int mpg_analyze_mesh(const mpg_mesh_ref *mesh, mpg_info *info);
/* Host-only: the factorised column blocks of laplc that the iprc = 4 preconditioner solves
 * (no counterpart in the reference; see params.iprc), per reference node: sub-diagonal a =
 * A[k][k-2], inverse pivot 1/m and c' of the Thomas factorisation on the node's parity chain. */
int mpg_analyze_wide(const mpg_params *prm, const mpg_mesh_ref *mesh, int impfl, double *a,
                     double *minv, double *cp);
const char *mpg_last_error(void);
int mpg_get_info(mpg_handle h, mpg_info *info);

/* mg_flag = 1: attach the coarse (level 1) or coarsest (level 2) mesh of precon's V-cycle
 * (ref.f:618-748), the meshes the reference reads from mesh3d_c.d and mesh3d_cc.d (ref.f:2343-2641),
 * before mpg_setup.  `match` gives each node of the level its node in the next finer mesh, 1-based
 * as in match1.d / match2.d (ref.f:2653-2672), or NULL to find it by coordinates within 1 m as
 * `matching` does (ref.f:2684-2720).  laplc_c / laplc_cc (ref.f:1356-1533) run as laplc on the
 * level's mesh; restriction_unstr / prolongation_unstr (ref.f:757-951) move residuals and
 * corrections; params.mg_bugs picks the reference's indexing or the corrected one (see
 * mpg_params).  The V-cycle runs inside the reference smoother (iprc = 1), in FP64. */
int mpg_set_coarse(mpg_handle h, int level, const mpg_mesh_ref *mesh, const int32_t *match);

/* Field exchange in reference node order: `n` = npoin values, contiguous. */
int mpg_set_field(mpg_handle h, int fid, const double *src);
int mpg_get_field(mpg_handle h, int fid, double *dst);

/* ---------------------------------------------------------------- reference subroutines */
/* derivative(unk, dpdxa, idx)                          ref.f:3943-4022 */
int mpg_derivative(mpg_handle h, int unk, int out, int idx);
/* bcv(u, v, w, flag)                                    ref.f:1583-1643 */
int mpg_bcv(mpg_handle h, int u, int v, int w, double flag);
/* laplc(press, alap, impfl)                             ref.f:1288-1353 */
int mpg_laplc(mpg_handle h, int press, int alap, int impfl);
/* Adjoint of laplc in the inner product <u,v>_W = sum vol*rh0*u*v: out such that
 * <laplc(u), y>_W = <u, out>_W for every u (the transposes of the derivative passes, of the
 * metric scaling and of bcv's projections, applied in reverse order).  Used to train the
 * learned preconditioner on the residual norm; no counterpart in the reference. */
int mpg_laplc_adjoint(mpg_handle h, int y, int out, int impfl);
/* prfr(press, ustr, vstr, wstr, uout, vout, wout, impfl) ref.f:1536-1580 */
int mpg_prfr(mpg_handle h, int press, int ustr, int vstr, int wstr,
             int uout, int vout, int wout, int impfl);
/* div(ua, va, wa, rhs, iflg)                            ref.f:2096-2170; diag may be NULL */
int mpg_div(mpg_handle h, int ua, int va, int wa, int rhs, int iflg, mpg_diag *diag);
/* precon(rhs, p, r, iprc, elas, impfl)                  ref.f:482-753 (mg_flag=0) + line option */
int mpg_precon(mpg_handle h, int rhs, int p, int r, int iprc, int impfl);
/* gcrk(p, u1, v1, w1, u2, v2, w2, impfl)                ref.f:1776-1972 */
int mpg_gcrk(mpg_handle h, int p, int u1, int v1, int w1, int u2, int v2, int w2,
             int impfl, mpg_gcr_stats *stats);
/* mpdatamper(uuu, unk(1,iflag), iflag)                  ref.f:3617-3941 (uuu = MPG_F_UUU); iper = 2 */
int mpg_mpdatamper(mpg_handle h, int unk, int iflag);
/* mpdatam(uuu, unk(1,iflag), iflag)                     ref.f:3029-3311; iper = 0 (open boundaries).
 * The first pass closes every boundary point of a type other than 11, 5 or 6 with the flux
 * that balances the node's face fluxes, upwinded with the free-stream value afree(iflag) on
 * inflow (ue per node for iflag = 1), ref.f:3143-3169.  iflag > 4 (passive scalars, not in
 * the reference) flows in with 0. */
int mpg_mpdatam(mpg_handle h, int unk, int iflag);
/* courant(uuu, cour, iflag) and stats(unk)              ref.f:1974-2094, ref.f:2847-2912 */
int mpg_courant(mpg_handle h, int iflag, mpg_diag *diag);
int mpg_stats(mpg_handle h, mpg_diag *diag);

/* ---------------------------------------------------------------- mpsolver */
/* Set-up part of mpsolver (ref.f:99-273): profiles, absorbers, metric, beta/d, ambient state,
 * potential-flow solve, coefw, momentum and the initial diagnostics. */
int mpg_setup(mpg_handle h, mpg_diag *diag);
/* One pass of the DO ITIME loop (ref.f:285-463). */
int mpg_step(mpg_handle h, mpg_diag *diag);
/* The node loops of one pass, for a host that drives the subroutines itself. */
int mpg_half_forcing(mpg_handle h);                 /* ref.f:290-301 */
int mpg_explicit_forcing(mpg_handle h, int mtri);   /* ref.f:323-359 */
int mpg_post_solve(mpg_handle h, int mtri);         /* ref.f:367-383 */
int mpg_extrapolate(mpg_handle h);                  /* ref.f:387-439 */
/* velprd(unk, frc, uuu, uuu1, unkdash)                  ref.f:4448-4528 (itraj = 1 driver path) */
int mpg_velprd(mpg_handle h);
/* Last GCR statistics of the handle (/itero/). */
int mpg_get_gcr_stats(mpg_handle h, mpg_gcr_stats *stats);
/* Wait for all work of the handle. */
int mpg_synchronize(mpg_handle h);

/* ---------------------------------------------------------------- learned preconditioner */
/* An edge message-passing network (3 layers, 32 hidden channels, BF16 activations and weights,
 * FP32 accumulation) that corrects the vertical-line preconditioner inside gcrk:
 * q = M^{-1} r + net(r) (see src_b200/csrc/learned.cuh).  It is used when params.iprc == 3; the
 * plain line preconditioner takes over for the rest of a solve if the network's output is not
 * finite, the residual stops decreasing, or ||r||_2 after m iterations exceeds params.nn_rate^m
 * of its start (mpg_gcr_stats.fallbacks counts the switches), and every solve still has to meet
 * the same FP64 stopping test.  Meshes of at most 128 levels.  No counterpart in the reference.
 * Training runs on the GPU with the library's own forward/backward kernels and Adam. */
#define MPG_LEARNED_NPARAM 9505
/* Initialise the weights (seeded): hidden layers random, output layer zero, so the initial
 * network returns the plain preconditioner exactly. */
int mpg_learned_init(mpg_handle h, int seed);
int mpg_learned_set_params(mpg_handle h, const float *params, int n);
int mpg_learned_get_params(mpg_handle h, float *params, int n);
/* q = learned preconditioner applied to field r (impfl = 1 coefficients); r, q are field ids */
int mpg_learned_forward(mpg_handle h, int r, int q);
/* Training loss (mpg_learned_loss selects it):
 *   MPG_NN_LOSS_RESIDUAL (default): 0.5*min_a ||r - a A q||_W^2 / ||r||_W^2 with A = laplc
 *       (impfl = 1), W = vol*rh0 and q the preconditioner output: the residual left by the best
 *       GCR step along q, which like GCR ignores the scale of q.  Since A t = r for the pair
 *       (r, t = A^{-1} r), it measures the error of a q against t in the A^T W A-norm, so t
 *       itself is not read;
 *   MPG_NN_LOSS_ERROR: 0.5*mean((y - y*)^2), the network output y regressed on the scaled
 *       error y* = (t - M^{-1} r)|b|/max|r| of the pair.
 * mpg_learned_grad returns the loss for residual field r and target field t and its gradient
 * w.r.t. all MPG_LEARNED_NPARAM parameters (grad may be NULL); no update. */
#define MPG_NN_LOSS_RESIDUAL 0
#define MPG_NN_LOSS_ERROR    1
int mpg_learned_loss(mpg_handle h, int mode);
/* Failure-detection self-test of the bounded waits in the library's tensor-core kernels (no
 * counterpart in the reference): one CTA arms an mbarrier for one arrival and waits on it with
 * the same bounded loop the network layers use, giving up after `spins` polls (1..2^22).  With
 * arrive != 0 a thread arrives and *completed = 1; with arrive == 0 nothing arrives, the wait runs
 * out, the kernel returns normally and *completed = 0 — the device stays usable.  In the network
 * layers the same give-up writes NaN outputs, which gcrk's finite check turns into a fallback. */
int mpg_selftest_wait(mpg_handle h, int arrive, int spins, int *completed);
int mpg_learned_grad(mpg_handle h, int r, int t, float *grad, double *loss);
/* one Adam step on the pair (r, t) */
int mpg_learned_train_pair(mpg_handle h, int r, int t, float lr, double *loss);
/* Record (r_i, p_i) every `every`-th GCR iteration of plain solves with impfl = 1 (at most
 * max_records kept; every = 0 stops recording); after a converged solve each record becomes the
 * pair (r_i, p_i - p*), i.e. (residual, A^{-1} residual). */
int mpg_learned_harvest(mpg_handle h, int every, int max_records);
/* `epochs` passes of Adam steps over the recorded pairs (then the records are cleared) */
int mpg_learned_train_records(mpg_handle h, int epochs, float lr, double *mean_loss, int *npairs);

/* ---------------------------------------------------------------- restart files */
/* MPG_RESTART_TEXT: the layout of Restart_Out_old / Restart_In_old (ref.f:4779-4890), one node per
 * line in reference node order, F14.6 fields (lossy, as in the reference): uuu(:,1:3), uuu1(:,1:3)
 * (velprd's array, zero: itraj = 0), unkdash(:,1:3), unk(:,1:4), frc(:,1:4), then
 * prpot/rhs/cour/coefw, a list-directed line "nitsm icount" and one with ntime.  Reading restores
 * those fields (uuu1 is skipped) and nitsm/icount, as Restart_In_old does (ref.f:277-278).
 * MPG_RESTART_BINARY: every field the time step carries (unk incl. passive scalars, unk1, uuu,
 * uuu0, frc, unkdash, prpot, rhs, cour) in FP64 with the counters, so a run continued from it is
 * bit-identical to the uninterrupted one.  Either replaces mpg_setup for a restarted run.  `path`
 * is a NUL-terminated file name; `ntime` is the step number written (read back into *ntime when
 * the file holds it; may be NULL). */
/* output(unk) (ref.f:2771-2806): the flow field file the reference writes at the end of a run
 * (unit 11, r.d, ref.f:40, called at ref.f:477): a list-directed "1." and npoin, the header line
 * 'point X Y Z u v w temp Velocity', then per node in reference order format (1x,i7,8e12.4): the
 * 1-based node number, coord/1000 (caller's COMMON array coord(npoinx,3)), u, v, w, theta' and
 * sqrt(u^2+v^2+w^2) of unk(:,1:4). */
int mpg_write_output(mpg_handle h, const char *path, const double *coord, int npoinx);

#define MPG_RESTART_TEXT   0
#define MPG_RESTART_BINARY 1
int mpg_restart_write(mpg_handle h, const char *path, int format, int ntime);
int mpg_restart_read(mpg_handle h, const char *path, int format, int *ntime);

/* ---------------------------------------------------------------- allocation-free laplc */
/* laplc(press, alap, impfl) for callers that must not allocate device memory at call time: a
 * host application whose own pool owns all device memory (a Fortran or PyTorch code with a
 * caching allocator, where an outside cudaMalloc can fail on a full pool or break its
 * accounting), or a time-critical loop where cudaMalloc/cudaFree would synchronise the device.
 * It has no counterpart in the reference.
 *
 * `press` and `alap` are caller-owned DEVICE arrays of npoin doubles in reference node order on
 * the handle's device.  The work is queued on the handle's stream (mpg_get_stream) and the
 * call returns without waiting.  Both directions need ordering against that stream: whatever
 * writes `press` (a kernel or copy on another stream) must have completed, or be ordered before
 * the call with an event the handle's stream waits on; and your own stream must wait for the
 * handle's stream before it reads `alap`.
 * Scratch is a static device array sized for MPG_NOALLOC_MAX_NODES nodes (5 MiB), held by every
 * GPU that loads the library until the process exits; larger meshes get MPG_ERR_ARG.  The first
 * call on a device looks up the array's device address (cudaGetSymbolAddress) and keeps it for
 * the life of the process: make that first call before any stream capture, and do not call the
 * entry point again after cudaDeviceReset on that device (the kept address belongs to the old
 * context).  All calls share the one array, so calls that overlap on the GPU (two handles, or
 * two streams, on the same device) race; serialise them.  The caller's current device is the
 * same after the call as before.  The call allocates nothing: no cudaMalloc, cudaFree or
 * allocating library routine. */
#define MPG_NOALLOC_MAX_NODES 131072
int mpg_laplc_noalloc(mpg_handle h, const double *press, double *alap, int impfl);

/* ---------------------------------------------------------------- instrumentation */
/* The CUDA stream every kernel of the handle runs on (a cudaStream_t), so callers can time
 * or order their own work against it. */
int mpg_get_stream(mpg_handle h, void **stream);
/* Per-kernel-class timing with CUDA events recorded around each launch on the handle's stream
 * (off by default; enabling it clears the totals).  Pressure solves (gcrk + prfr inside
 * mpg_step) are always timed, as class "pressure_solve". */
typedef struct mpg_ktime {
    char    name[24];
    int64_t launches;
    double  total_ms;
} mpg_ktime;
int mpg_kernel_timing(mpg_handle h, int enable);
int mpg_kernel_times(mpg_handle h, mpg_ktime *out, int max, int *count);

#ifdef __cplusplus
}
#endif
#endif /* MPGCR_H */

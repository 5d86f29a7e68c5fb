// C ABI of the B200 MPDATA + GCR library (include/mpgcr.h): handle, field storage, the
// reference subroutines on device-resident fields, and the mpsolver driver.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <type_traits>
#include <string>
#include <vector>

#include "kernels.cuh"
#include "learned.cuh"
#include "mpdata.cuh"
#include "mg.cuh"
#include "periodic.cuh"

#include <algorithm>
#include <unordered_map>
#include "mpgcr_internal.h"

using namespace mpgk;

// ------------------------------------------------------------------------------ errors
static thread_local std::string g_err;
void mpg_set_error(const std::string &msg) { g_err = msg; }
int mpg_fail(int code, const std::string &msg) {
    g_err = msg;
    return code;
}
extern "C" const char *mpg_last_error(void) { return g_err.c_str(); }

// ------------------------------------------------------------------------------ kernel timing
enum KClass {
    KT_LAP_GRAD, KT_LAP_DIV, KT_PRFR, KT_DIV, KT_LINE, KT_REDUCE, KT_GCR_UPD, KT_AUN, KT_MP_DONOR,
    KT_MP_GRADB, KT_MP_ANTI, KT_MP_CPCN, KT_MP_PASS2, KT_NODE, KT_COURANT, KT_MISC, KT_NN, KT_SOLVE, KT_LAPLC,
    KT_COUNT
};
static const char *kKNames[KT_COUNT] = {
    "lap_grad", "lap_div", "prfr", "div", "line_solve", "reduce", "gcr_update", "aun", "mp_donor",
    "mp_grad_bounds", "mp_anti", "mp_cpcn", "mp_pass2", "node_loops", "courant", "misc", "learned", "pressure_solve",
    "laplc"};

struct KTimer {
    bool on = false;
    std::vector<cudaEvent_t> pool;
    struct Rec { int cls; cudaEvent_t a, b; };
    std::vector<Rec> recs;
    std::vector<int> open;          // stack of pending (class, start) for nested scopes
    std::vector<cudaEvent_t> open_ev;
    double total_ms[KT_COUNT] = {};
    int64_t launches[KT_COUNT] = {};
};

// ------------------------------------------------------------------------------ handle
struct mpg_solver {
    mpg_params P{};
    int dev = 0;
    cudaStream_t st = nullptr;
    int32_t NC = 0, L = 0, N = 0, NE2 = 0;
    bool bitwise = true;
    ColMesh M{};
    std::vector<void *> allocs;
    size_t dev_bytes = 0;
    int32_t *d_perm = nullptr, *d_iperm = nullptr;
    int32_t *d_e2a = nullptr, *d_e2b = nullptr;
    double *f[MPG_F_COUNT] = {};
    double *vol = nullptr, *ue = nullptr, *ve = nullptr, *stage = nullptr;
    // GCR workspace
    double *r = nullptr, *qr = nullptr, *ar = nullptr, *x[MPG_MAX_LORD] = {}, *ax[MPG_MAX_LORD] = {};
    double *F[3] = {}, *tres = nullptr;
    // mixed precision: FP32 directions, operator intermediates and node metrics
    float *xf[MPG_MAX_LORD] = {}, *axf[MPG_MAX_LORD] = {}, *qrf = nullptr, *arf = nullptr;
    float4 *Ff4 = nullptr;                           // packed laplc fluxes (mixed precision)
    float *volf = nullptr, *rh0f = nullptr, *coefwf = nullptr;
    double *scal = nullptr, *part = nullptr, *result = nullptr, *h_res = nullptr;
    unsigned int *counter = nullptr;
    // line preconditioner
    double *la[2] = {}, *lm[2] = {}, *lcp[2] = {};   // a, 1/m, c' (interleaved)
    double *wa[2] = {}, *wm[2] = {}, *wcp[2] = {};   // iprc = 4: laplc's column blocks, factorised
    double *dbuf = nullptr;                          // forward-sweep values (interleaved)
    double *vp[4] = {};                              // velprd: its potential and velocity
    // MPDATA scratch
    MpScratch S{};
    double *psi1 = nullptr, *g3[3] = {}, *mx = nullptr, *mn = nullptr;
    MpScratchT<float> Sf{};
    float *psi1f = nullptr, *g3f[3] = {};
    // mixed precision: the first-pass field, the FCT bounds and the limiter ratios in FP64
    double *psi1d = nullptr, *mxd = nullptr, *mnd = nullptr, *cpd = nullptr, *cnd = nullptr;
    // /itero/
    int32_t niter = 0, nitsm = 0, icount = 0, gstatus = 0, last_fallbacks = 0;
    double eer = 0., eem = 0., dvmx_last = 0., rl2_last = 0., rate_last = 0.;
    double betaunstr1 = 0.;
    HostStatic hs;
    std::vector<int32_t> iperm;
    KTimer kt;
    // multigrid V-cycle (mg_flag = 1): the transfer data to the coarse (0) and coarsest (1) mesh,
    // whose own handles run laplc_c / laplc_cc on this handle's stream
    struct MgLevel {
        mpg_solver *sub = nullptr;
        int32_t *match = nullptr;                            // coarse node -> finer node (internal)
        int32_t *nbp = nullptr, *nbl = nullptr, *bugnb = nullptr;   // finer mesh's neighbour lists
        int passes = 1;                                      // prolongation filling passes
        double *aux = nullptr;                               // finer-mesh scratch of the prolongation
        uint8_t *flag = nullptr;
        double *p = nullptr, *r = nullptr, *e = nullptr, *rrhs = nullptr, *rrhs_out = nullptr;  // coarse arrays
        std::vector<int32_t> match_ref;                      // coarse ref node -> finer ref node
        std::vector<double> rh0_restricted;                  // finest rh0 restricted here (ref order)
    } mg[2];
    double *mg_rrhs = nullptr, *mg_e = nullptr;          // fine-mesh arrays of the V-cycle
    bool borrowed_stream = false;                        // a coarse level runs on its parent's stream
    CopyList CL{};                                       // periodic copy groups (duplicate-node form)
    LapSched lap{};                                      // fused laplc's work order (total 0: two launches)
    int lap_ctas[2] = {0, 0};                            // its persistent grid, FP64 and FP32 instantiations
    // kept for the V-cycle's set-up when mg_flag = 1 (and on a coarse level's handle): the mesh's
    // neighbour lists in neigh_definition order and its coordinates, reference numbering
    std::vector<int32_t> nb_ptr_ref, nb_lst_ref;
    std::vector<double> cx_ref, cy_ref, cz_ref;
    struct NN {
        bool geom = false, infer = false, train = false, have_params = false;
        float *prm = nullptr, *grad = nullptr, *m1 = nullptr, *m2 = nullptr;
        __nv_bfloat16 *Wbf = nullptr;
        float *Th = nullptr, *Tv = nullptr, *iDh = nullptr, *iDv = nullptr, *bdiag = nullptr, *feat2 = nullptr,
              *bnd = nullptr;
        __nv_bfloat16 *H[4] = {};
        float *X0 = nullptr, *dH = nullptr, *dH2 = nullptr, *G0 = nullptr, *Gh = nullptr, *Gv = nullptr, *Y = nullptr;
        __nv_bfloat16 *Xs[3] = {}, *dU = nullptr;
        double *z = nullptr, *sc = nullptr, *pd = nullptr;
        float *pf = nullptr;
        int Npad = 0, adam_t = 0;
        // harvested pairs
        int every = 0, maxrec = 0, nrec = 0, solve_first = 0;
        double *rec_r = nullptr, *rec_t = nullptr;
        int fallbacks = 0;
        // residual-norm training: q, e = A q - r and A^T W e (FP64)
        int loss_mode = MPG_NN_LOSS_RESIDUAL;
        double *qd = nullptr, *ed = nullptr, *dq = nullptr;
        int *err = nullptr;          // set by the tensor-core layer when its wait gave up
        int *selftest = nullptr;     // status of mpg_selftest_wait
        int col_ctas = 0;            // persistent grid of the column layers (CTAs resident at once)
    } nn;
};

static cudaEvent_t kt_event(mpg_handle h) {
    if (h->kt.pool.empty()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        return e;
    }
    cudaEvent_t e = h->kt.pool.back();
    h->kt.pool.pop_back();
    return e;
}

// fold recorded event pairs into the totals (synchronises the stream)
static void kt_collect(mpg_handle h) {
    if (h->kt.recs.empty()) return;
    cudaStreamSynchronize(h->st);
    for (auto &r : h->kt.recs) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) {
            h->kt.total_ms[r.cls] += ms;
            h->kt.launches[r.cls] += 1;
        }
        h->kt.pool.push_back(r.a);
        h->kt.pool.push_back(r.b);
    }
    h->kt.recs.clear();
}

// times the launches issued in its scope when timing is on (always for the solve class)
struct KScope {
    mpg_handle h;
    int cls;
    cudaEvent_t a = nullptr;
    KScope(mpg_handle h_, int c) : h(h_), cls(c) {
        if (h->kt.on || cls == KT_SOLVE) {
            a = kt_event(h);
            cudaEventRecord(a, h->st);
        }
    }
    ~KScope() {
        if (!a) return;
        cudaEvent_t b = kt_event(h);
        cudaEventRecord(b, h->st);
        h->kt.recs.push_back({cls, a, b});
        if (h->kt.recs.size() > 16384) kt_collect(h);
    }
};
#define KTIME(cls) KScope _kscope_(h, cls)

namespace {

template <class T>
int dalloc(mpg_handle h, T **p, size_t n, bool zero = true) {
    size_t bytes = sizeof(T) * (n ? n : 1);
    cudaError_t e = cudaMalloc((void **)p, bytes);
    if (e != cudaSuccess) return mpg_fail(MPG_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    h->allocs.push_back(*p);
    h->dev_bytes += bytes;
    if (zero) MPG_CUDA(cudaMemsetAsync(*p, 0, bytes, h->st));
    return MPG_OK;
}

template <class T>
int upload(mpg_handle h, T **p, const std::vector<T> &v) {
    int rc = dalloc(h, p, v.size(), false);
    if (rc) return rc;
    MPG_CUDA(cudaMemcpyAsync(*p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, h->st));
    return MPG_OK;
}

inline int grid(int n) { return (n + kThreads - 1) / kThreads; }


// field pointer, allocated (zeroed) on first use
double *fld(mpg_handle h, int fid) {
    if (fid < 0 || fid >= MPG_F_COUNT) return nullptr;
    if (fid >= MPG_F_UNK + 4 + h->P.nscal && fid < MPG_F_UNK1) return nullptr;
    if (!h->f[fid]) {
        if (dalloc(h, &h->f[fid], (size_t)h->N)) return nullptr;
    }
    return h->f[fid];
}

#define FLD(var, fid)                                                                      \
    double *var = fld(h, (fid));                                                           \
    if (!var) return mpg_fail(MPG_ERR_ARG, "invalid or unallocatable field id " + std::to_string(fid));

int check_launch(const char *what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return mpg_fail(MPG_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return MPG_OK;
}

// generic deterministic reduction launcher
template <int NQ, class Prod, class Fin>
int reduce(mpg_handle h, unsigned kinds, Prod prod, Fin fin) {
    {
        KTIME(KT_REDUCE);
        k_reduce<NQ><<<kRedBlocks, kRedThreads, 0, h->st>>>(h->N, kinds, prod, fin, h->part, h->counter, h->result);
    }
    return check_launch("k_reduce");
}

int fetch_result(mpg_handle h, int nq) {
    MPG_CUDA(cudaMemcpyAsync(h->h_res, h->result, sizeof(double) * nq, cudaMemcpyDeviceToHost, h->st));
    MPG_CUDA(cudaStreamSynchronize(h->st));
    return MPG_OK;
}

// ------------------------------------------------------------------------------ operators
// buffers of the GCR directions and of laplc in the storage type T
template <class T> struct Buf;
template <> struct Buf<double> {
    static double *x(mpg_handle h, int q) { return h->x[q]; }
    static double *ax(mpg_handle h, int q) { return h->ax[q]; }
    static double *qr(mpg_handle h) { return h->qr; }
    static double *ar(mpg_handle h) { return h->ar; }
    static Flux<double> F(mpg_handle h) { return Flux<double>{h->F[0], h->F[1], h->F[2]}; }
    static const double *vol(mpg_handle h) { return h->vol; }
    static const double *rh0(mpg_handle h) { return h->f[MPG_F_RH0]; }
    static const double *coefw(mpg_handle h) { return h->f[MPG_F_COEFW]; }
};
template <> struct Buf<float> {
    static float *x(mpg_handle h, int q) { return h->xf[q]; }
    static float *ax(mpg_handle h, int q) { return h->axf[q]; }
    static float *qr(mpg_handle h) { return h->qrf; }
    static float *ar(mpg_handle h) { return h->arf; }
    static Flux<float> F(mpg_handle h) { return Flux<float>{h->Ff4}; }
    static const float *vol(mpg_handle h) { return h->volf; }
    static const float *rh0(mpg_handle h) { return h->rh0f; }
    static const float *coefw(mpg_handle h) { return h->coefwf; }
};

// the fused kernel's grid: every block resident at once (one persistent block per slot)
template <class T>
int lap_fused_ctas(mpg_handle h) {
    int &n = h->lap_ctas[std::is_same<T, float>::value ? 1 : 0];
    if (!n) {
        int sms = 0, per_sm = 0;
        MPG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->dev));
        MPG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_lap_fused<T>, kThreads, 0));
        n = std::max(1, sms) * std::max(1, per_sm);
    }
    return MPG_OK;
}

// the fused laplc's wait gave up (never expected: every awaited item has started): report it once
int lap_fused_check(mpg_handle h) {
    if (!h->lap.total) return MPG_OK;
    int32_t e = 0;
    MPG_CUDA(cudaMemcpyAsync(&e, h->lap.state + 3, sizeof e, cudaMemcpyDeviceToHost, h->st));
    MPG_CUDA(cudaStreamSynchronize(h->st));
    if (e) {
        MPG_CUDA(cudaMemsetAsync(h->lap.state + 3, 0, sizeof e, h->st));
        return mpg_fail(MPG_ERR_CUDA, "laplc: a wait for gradient fluxes gave up; the result is not valid");
    }
    return MPG_OK;
}

template <class T>
int op_laplc_t(mpg_handle h, const T *p, T *alap, int impfl) {
    using B = Buf<T>;
    if (h->lap.total) {
        int rc;
        if ((rc = lap_fused_ctas<T>(h))) return rc;
        KTIME(KT_LAPLC);
        k_lap_fused<T><<<h->lap_ctas[std::is_same<T, float>::value ? 1 : 0], kThreads, 0, h->st>>>(
            h->M, (h->L + 1) / 2, h->lap, p, B::vol(h), B::rh0(h), B::coefw(h), h->ue, (T)h->P.delt, impfl, B::F(h),
            alap);
        return check_launch("laplc");
    }
    {
        KTIME(KT_LAP_GRAD);
        k_lap_grad<T><<<grid(h->N), kThreads, 0, h->st>>>(h->M, p, B::vol(h), B::rh0(h), B::coefw(h), h->ue,
                                                          (T)h->P.delt, impfl, B::F(h));
        if (h->CL.n)
            k_cp_lap_grad<T><<<grid(h->CL.n), kThreads, 0, h->st>>>(h->M, h->CL, p, B::vol(h), B::rh0(h), B::coefw(h),
                                                                    h->ue, (T)h->P.delt, impfl, B::F(h));
    }
    {
        KTIME(KT_LAP_DIV);
        const int PL = (h->L + 1) / 2;
        k_lap_div2<T><<<grid(h->NC * PL), kThreads, 0, h->st>>>(h->M, PL, B::F(h), B::vol(h), B::rh0(h), alap);
        if (h->CL.n)
            k_cp_lap_div<T><<<grid(h->CL.n), kThreads, 0, h->st>>>(h->M, h->CL, B::F(h), B::vol(h), B::rh0(h), alap);
    }
    return check_launch("laplc");
}
int op_laplc(mpg_handle h, const double *p, double *alap, int impfl) { return op_laplc_t<double>(h, p, alap, impfl); }

// A^T W y (divw = false) or the W-adjoint W^{-1} A^T W y (divw = true), W = vol*rh0, A = laplc
int op_laplc_adj(mpg_handle h, const double *y, double *out, int impfl, bool divw) {
    {
        KTIME(KT_MISC);
        k_lapT_grad<<<grid(h->N), kThreads, 0, h->st>>>(h->M, y, h->vol, h->f[MPG_F_RH0], h->f[MPG_F_COEFW],
                                                        h->P.delt, impfl, h->F[0], h->F[1], h->F[2]);
        k_lapT_div<<<grid(h->N), kThreads, 0, h->st>>>(h->M, h->F[0], h->F[1], h->F[2], h->vol, h->f[MPG_F_RH0],
                                                       divw ? 1 : 0, out);
    }
    return check_launch("laplc adjoint");
}

int op_prfr(mpg_handle h, const double *p, const double *us, const double *vs, const double *ws, double *uo,
            double *vo, double *wo, int impfl) {
    {
        KTIME(KT_PRFR);
        if (h->CL.n && (uo == us || vo == vs || wo == ws))
            return mpg_fail(MPG_ERR_ARG, "prfr with periodic copy lists: outputs must differ from the inputs");
        k_prfr<<<grid(h->N), kThreads, 0, h->st>>>(h->M, p, us, vs, ws, h->vol, h->f[MPG_F_COEFW], h->ue, h->P.delt,
                                                   impfl, uo, vo, wo);
        if (h->CL.n)
            k_cp_prfr<<<grid(h->CL.n), kThreads, 0, h->st>>>(h->M, h->CL, p, us, vs, ws, h->vol, h->f[MPG_F_COEFW],
                                                             h->ue, h->P.delt, impfl, uo, vo, wo);
    }
    return check_launch("prfr");
}

int op_div(mpg_handle h, const double *ua, const double *va, const double *wa, double *rhs, int iflg) {
    {
        KTIME(KT_DIV);
        k_div<<<grid(h->N), kThreads, 0, h->st>>>(h->M, ua, va, wa, h->vol, h->f[MPG_F_RH0], iflg, rhs);
        if (h->CL.n)
            k_cp_div<<<grid(h->CL.n), kThreads, 0, h->st>>>(h->M, h->CL, ua, va, wa, h->vol, h->f[MPG_F_RH0], iflg,
                                                            rhs);
    }
    return check_launch("div");
}

template <class TO>
int op_line(mpg_handle h, const double *rhs, TO *p, int impfl, int acc) {
    const int q = impfl ? 1 : 0;
    const int nblk = (h->NC + 32 * kLineWarps - 1) / (32 * kLineWarps);
    {
        KTIME(KT_LINE);
        k_line_solve<TO><<<nblk, 32 * kLineWarps, 0, h->st>>>(h->NC, h->L, rhs, h->la[q], h->lm[q], h->lcp[q],
                                                              h->P.omega, acc, h->dbuf, p);
    }
    return check_launch("line_solve");
}

// iprc = 4: solve laplc's column blocks (tridiagonal on even and odd levels)
template <class TO>
int op_wide(mpg_handle h, const double *rhs, TO *p, int impfl, int acc) {
    const int q = impfl ? 1 : 0;
    if (!h->wa[q]) return mpg_fail(MPG_ERR_ARG, "iprc=4 needs a handle created with params.iprc = 4");
    const int nblk = (h->NC + 32 * kLineWarps - 1) / (32 * kLineWarps);
    {
        KTIME(KT_LINE);
        k_wide_solve<TO><<<nblk, 32 * kLineWarps, 0, h->st>>>(h->NC, h->L, rhs, h->wa[q], h->wm[q], h->wcp[q],
                                                              h->P.omega, acc, h->dbuf, p);
    }
    return check_launch("wide line solve");
}

// ------------------------------------------------------------------------------ multigrid (host side)
// neigh_definition (ref.f:2726-2767) in reference numbering: for every internal edge, then every
// boundary face, each end gets the other as its next neighbour (CSR)
void mg_neigh_definition(const mpg_mesh_ref *m, std::vector<int32_t> &ptr, std::vector<int32_t> &lst) {
    const int n = m->npoin;
    const int64_t ne = (int64_t)m->nedge + m->nbface;
    auto ends = [&](int64_t e, int &i1, int &i2) {
        if (e < m->nedge) { i1 = m->iedge[e] - 1; i2 = m->iedge[(size_t)m->nedgex + e] - 1; }
        else { const int64_t b = e - m->nedge; i1 = m->kbface[b] - 1; i2 = m->kbface[(size_t)m->nfacesx + b] - 1; }
    };
    ptr.assign(n + 1, 0);
    for (int64_t e = 0; e < ne; ++e) { int a, b; ends(e, a, b); ptr[a + 1]++; ptr[b + 1]++; }
    for (int i = 0; i < n; ++i) ptr[i + 1] += ptr[i];
    lst.assign(ptr[n], 0);
    std::vector<int32_t> fill(n, 0);
    for (int64_t e = 0; e < ne; ++e) {
        int a, b; ends(e, a, b);
        lst[ptr[a] + fill[a]++] = b;
        lst[ptr[b] + fill[b]++] = a;
    }
}

void mg_coords(const mpg_mesh_ref *m, std::vector<double> &x, std::vector<double> &y, std::vector<double> &z) {
    const int n = m->npoin;
    x.assign(m->coord, m->coord + n);
    y.assign(m->coord + m->npoinx, m->coord + m->npoinx + n);
    z.assign(m->coord + 2 * (size_t)m->npoinx, m->coord + 2 * (size_t)m->npoinx + n);
}

// matching (ref.f:2684-2720): for every fine point in order, the first coarse point within 1 m in
// x, y and z takes it as its match (so the last such fine point wins); -1 where none
std::vector<int32_t> mg_matching(const std::vector<double> &fx, const std::vector<double> &fy,
                                 const std::vector<double> &fz, const std::vector<double> &cx,
                                 const std::vector<double> &cy, const std::vector<double> &cz) {
    const double tol = 1.;
    auto key = [](double x, double y, double z) {
        const int64_t K = 1 << 21;
        return (((int64_t)std::floor(x) + K / 2) * K + ((int64_t)std::floor(y) + K / 2)) * K +
               ((int64_t)std::floor(z) + K / 2);
    };
    std::unordered_map<int64_t, std::vector<int32_t>> bins;
    for (size_t ic = 0; ic < cx.size(); ++ic) bins[key(cx[ic], cy[ic], cz[ic])].push_back((int32_t)ic);
    std::vector<int32_t> match(cx.size(), -1);
    for (size_t ip = 0; ip < fx.size(); ++ip) {
        int32_t best = -1;
        for (int dx = -1; dx <= 1; ++dx)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dz = -1; dz <= 1; ++dz) {
                    auto it = bins.find(key(fx[ip] + dx, fy[ip] + dy, fz[ip] + dz));
                    if (it == bins.end()) continue;
                    for (int32_t ic : it->second)
                        if (std::fabs(fx[ip] - cx[ic]) < tol && std::fabs(fy[ip] - cy[ic]) < tol &&
                            std::fabs(fz[ip] - cz[ic]) < tol && (best < 0 || ic < best))
                            best = ic;
                }
        if (best >= 0) match[best] = (int32_t)ip;
    }
    return match;
}

// restriction_unstr (ref.f:757-824) on the host, reference numbering
std::vector<double> mg_restrict_host(const std::vector<double> &s, const std::vector<int32_t> &match,
                                     const std::vector<int32_t> &ptr, const std::vector<int32_t> &lst, int bugs) {
    std::vector<double> sc(match.size(), 0.);
    for (size_t ic = 0; ic < match.size(); ++ic) {
        const int ip = match[ic], nn = ptr[ip + 1] - ptr[ip];
        for (int k = 0; k < nn; ++k) {
            const int j = bugs ? k : lst[ptr[ip] + k];
            sc[ic] = sc[ic] + (s[ip] + s[j]) / 2.;
        }
        sc[ic] = sc[ic] / (double)nn;
    }
    return sc;
}

// compute_d_unstr(2/3) (ref.f:1112-1284) on a coarser mesh with the restricted rh0, reference
// numbering
std::vector<double> mg_compute_d(const mpg_mesh_ref *m, const std::vector<double> &rh0u, double dt) {
    const int n = m->npoin;
    std::vector<double> dix(n, 0.), diy(n, 0.), diz(n, 0.), d(n, 0.);
    const int64_t ne = (int64_t)m->nedge + m->nbface;
    for (int64_t e = 0; e < ne; ++e) {
        int i1, i2;
        double sx, sy, sz;
        if (e < m->nedge) {
            i1 = m->iedge[e] - 1; i2 = m->iedge[(size_t)m->nedgex + e] - 1;
            sx = m->sn[e]; sy = m->sn[(size_t)m->nedgex + e]; sz = m->sn[2 * (size_t)m->nedgex + e];
        } else {
            const int64_t b = e - m->nedge;
            i1 = m->kbface[b] - 1; i2 = m->kbface[(size_t)m->nfacesx + b] - 1;
            sx = m->sb[b]; sy = m->sb[(size_t)m->nfacesx + b]; sz = m->sb[2 * (size_t)m->nfacesx + b];
        }
        const double v1 = m->vol[i1], v2 = m->vol[i2];
        dix[i1] = dix[i1] + sx * sx * rh0u[i2] / v2;
        dix[i2] = dix[i2] + sx * sx * rh0u[i1] / v1;
        diy[i1] = diy[i1] + sy * sy * rh0u[i2] / v2;
        diy[i2] = diy[i2] + sy * sy * rh0u[i1] / v1;
        diz[i1] = diz[i1] + sz * sz * rh0u[i2] / v2;
        diz[i2] = diz[i2] + sz * sz * rh0u[i1] / v1;
    }
    for (int i = 0; i < n; ++i) d[i] = -0.5 * dt * (dix[i] + diy[i] + diz[i]) / (4 * m->vol[i] * rh0u[i]);
    return d;
}

// filling passes prolongation_unstr needs until every finer node has a value (the corrected
// variant; the reference makes one); -1 if some node can never get one
int mg_fill_passes(int nfine, const std::vector<int32_t> &match, const std::vector<int32_t> &ptr,
                   const std::vector<int32_t> &lst) {
    std::vector<uint8_t> set(nfine, 0), nw(nfine, 0);
    for (int32_t ip : match) set[ip] = 1;
    for (int pass = 1; pass <= 1000; ++pass) {
        bool unset = false, progress = false;
        for (int i = 0; i < nfine; ++i) {
            if (set[i]) continue;
            bool any = false;
            for (int k = ptr[i]; k < ptr[i + 1] && !any; ++k) any = set[lst[k]] != 0;
            if (any) { nw[i] = 1; progress = true; } else unset = true;
        }
        if (!unset) return pass;
        if (!progress) return -1;
        for (int i = 0; i < nfine; ++i) if (nw[i]) { set[i] = 1; nw[i] = 0; }
    }
    return -1;
}

// the finer mesh's field s restricted to level lv's mesh
int mg_restrict(mpg_handle h, mpg_solver::MgLevel &lv, const double *s, double *sc) {
    {
        KTIME(KT_MISC);
        k_mg_restrict<<<grid(lv.sub->N), kThreads, 0, h->st>>>(lv.sub->N, lv.match, lv.nbp, lv.nbl, lv.bugnb,
                                                                h->P.mg_bugs, s, sc);
    }
    return check_launch("mg restriction");
}

// level lv's field sc prolongated to the finer mesh of nfine nodes
int mg_prolong(mpg_handle h, mpg_solver::MgLevel &lv, int nfine, const double *sc, double *s) {
    {
        KTIME(KT_MISC);
        k_mg_prolong_init<<<grid(nfine), kThreads, 0, h->st>>>(nfine, s, lv.aux, lv.flag);
        k_mg_inject<<<grid(lv.sub->N), kThreads, 0, h->st>>>(lv.sub->N, lv.match, sc, s, lv.aux);
        for (int pass = 0; pass < lv.passes; ++pass) {
            k_mg_fill<<<grid(nfine), kThreads, 0, h->st>>>(nfine, lv.nbp, lv.nbl, lv.bugnb, h->P.mg_bugs, lv.aux,
                                                           s, lv.flag);
            k_mg_commit<<<grid(nfine), kThreads, 0, h->st>>>(nfine, s, lv.aux, lv.flag);
        }
    }
    return check_launch("mg prolongation");
}

int mg_relax(mpg_handle a, double *p, double *r, const double *rhs, int sweeps, int impfl);

// the V-cycle of precon after the first fine smoothing (ref.f:618-748)
int mg_vcycle(mpg_handle h, const double *rhs, double *p, double *r, int impfl) {
    auto &L1 = h->mg[0], &L2 = h->mg[1];
    mpg_solver *c1 = L1.sub, *c2 = L2.sub;
    const int N = h->N, N1 = c1->N, N2 = c2->N;
    const double om = h->P.omega;
    const int sm = h->P.sm_flag1;
    int rc;
    if ((rc = op_laplc(h, p, r, impfl))) return rc;                            // ref.f:660-664
    {
        KTIME(KT_MISC);
        k_sub<<<grid(N), kThreads, 0, h->st>>>(N, rhs, r, h->mg_rrhs);
    }
    if ((rc = mg_restrict(h, L1, h->mg_rrhs, L1.rrhs))) return rc;
    {
        KTIME(KT_MISC);                                                       // ref.f:675-677
        k_mg_first<<<grid(N1), kThreads, 0, h->st>>>(N1, 0, sm, om, c1->betaunstr1, c1->f[MPG_F_D1], L1.rrhs, L1.p);
    }
    if ((rc = mg_relax(c1, L1.p, L1.r, L1.rrhs, h->P.itrp_c1, impfl))) return rc;
    if ((rc = op_laplc(c1, L1.p, L1.r, impfl))) return rc;                   // ref.f:688-691
    {
        KTIME(KT_MISC);
        k_sub<<<grid(N1), kThreads, 0, h->st>>>(N1, L1.rrhs, L1.r, L1.rrhs_out);
    }
    if ((rc = mg_restrict(h, L2, L1.rrhs_out, L2.rrhs))) return rc;
    {
        KTIME(KT_MISC);                                                       // ref.f:702-704
        k_mg_first<<<grid(N2), kThreads, 0, h->st>>>(N2, 1, sm, om, c2->betaunstr1, c2->f[MPG_F_D1], L2.rrhs, L2.p);
    }
    if ((rc = mg_relax(c2, L2.p, L2.r, L2.rrhs, h->P.itrp_cc, impfl))) return rc;
    if ((rc = mg_prolong(h, L2, N1, L2.p, L1.e))) return rc;                  // ref.f:718-722
    {
        KTIME(KT_MISC);
        k_add<<<grid(N1), kThreads, 0, h->st>>>(N1, L1.e, L1.p);
    }
    if ((rc = mg_relax(c1, L1.p, L1.r, L1.rrhs, h->P.itrp_c2, impfl))) return rc;
    if ((rc = mg_prolong(h, L1, N, L1.p, h->mg_e))) return rc;                // ref.f:734-738
    {
        KTIME(KT_MISC);
        k_add<<<grid(N), kThreads, 0, h->st>>>(N, h->mg_e, p);
    }
    return mg_relax(h, p, r, rhs, h->P.itrp2, impfl);                          // ref.f:742-747
}

// precon(rhs, p, r, iprc, elas, impfl) (ref.f:482-753); `zero_r` restores the
// reference's clearing of r when a caller may look at it.
int op_precon(mpg_handle h, const double *rhs, double *p, double *r, int iprc, int impfl, bool zero_r) {
    const int N = h->N;
    if (iprc == 0) {
        {
            KTIME(KT_MISC);
            k_copy<double, double><<<grid(N), kThreads, 0, h->st>>>(N, rhs, p);
        }
        return check_launch("precon copy");
    }
    if (zero_r) {
        KTIME(KT_MISC);
        k_fill<<<grid(N), kThreads, 0, h->st>>>(N, r, 0.0);
    }
    if (iprc == 2) {
        for (int it = 1; it <= h->P.itrp1; ++it) {
            if (it == 1) {
                int rc = op_line<double>(h, rhs, p, impfl, 0);
                if (rc) return rc;
            } else {
                int rc = op_laplc(h, p, r, impfl);
                if (rc) return rc;
                {
                    KTIME(KT_MISC);
                    k_sub<<<grid(N), kThreads, 0, h->st>>>(N, rhs, r, h->tres);
                }
                rc = op_line<double>(h, h->tres, p, impfl, 1);
                if (rc) return rc;
            }
        }
        if (h->P.itrp1 < 1) {
            KTIME(KT_MISC);
            k_fill<<<grid(N), kThreads, 0, h->st>>>(N, p, 0.0);
        }
        return check_launch("precon line");
    }
    if (iprc == 4) {                      // the same relaxation with laplc's column blocks
        for (int it = 1; it <= h->P.itrp1; ++it) {
            if (it == 1) {
                int rc = op_wide<double>(h, rhs, p, impfl, 0);
                if (rc) return rc;
            } else {
                int rc = op_laplc(h, p, r, impfl);
                if (rc) return rc;
                {
                    KTIME(KT_MISC);
                    k_sub<<<grid(N), kThreads, 0, h->st>>>(N, rhs, r, h->tres);
                }
                rc = op_wide<double>(h, h->tres, p, impfl, 1);
                if (rc) return rc;
            }
        }
        if (h->P.itrp1 < 1) {
            KTIME(KT_MISC);
            k_fill<<<grid(N), kThreads, 0, h->st>>>(N, p, 0.0);
        }
        return check_launch("precon wide line");
    }
    if (iprc != 1) return mpg_fail(MPG_ERR_UNSUPPORTED, "iprc must be 0, 1, 2 or 4");
    // reference smoother: the first sweep starts from p = 0, where laplc(0) = 0 exactly
    {
        KTIME(KT_MISC);
        k_fill<<<grid(N), kThreads, 0, h->st>>>(N, p, 0.0);
    }
    if (!zero_r) {
        KTIME(KT_MISC);
        k_fill<<<grid(N), kThreads, 0, h->st>>>(N, r, 0.0);
    }
    for (int it = 1; it <= h->P.itrp1; ++it) {
        if (it > 1) {
            int rc = op_laplc(h, p, r, impfl);
            if (rc) return rc;
        }
        {
            KTIME(KT_MISC);
            k_smooth<<<grid(N), kThreads, 0, h->st>>>(N, h->P.sm_flag1, h->P.omega, h->betaunstr1,
                                                      h->f[MPG_F_D1], r, rhs, p);
        }
    }
    if (h->P.mg_flag == 1) {
        if (!h->mg[0].sub || !h->mg[1].sub)
            return mpg_fail(MPG_ERR_ARG, "mg_flag=1 needs both coarser meshes (mpg_set_coarse levels 1 and 2)");
        int rc = mg_vcycle(h, rhs, p, r, impfl);
        if (rc) return rc;
    }
    return check_launch("precon smoother");
}

// itrp relaxation sweeps p += omega*pstep*(laplc(p) - rhs) on mesh handle `a` (its d1 and beta)
int mg_relax(mpg_handle a, double *p, double *r, const double *rhs, int sweeps, int impfl) {
    for (int it = 1; it <= sweeps; ++it) {
        int rc = op_laplc(a, p, r, impfl);
        if (rc) return rc;
        {
            mpg_handle h = a;
            KTIME(KT_MISC);
            k_smooth<<<grid(a->N), kThreads, 0, a->st>>>(a->N, a->P.sm_flag1, a->P.omega, a->betaunstr1,
                                                         a->f[MPG_F_D1], r, rhs, p);
        }
    }
    return check_launch("mg relaxation");
}

// the preconditioner inside gcrk, writing its result in the direction type T
template <class T>
int op_precon_gcr(mpg_handle h, const double *r, int impfl) {
    const int N = h->N;
    T *qr = Buf<T>::qr(h);
    if constexpr (std::is_same<T, double>::value) return op_precon(h, r, qr, h->ar, h->P.iprc, impfl, false);
    else {
    if (h->P.iprc == 2) {
        for (int it = 1; it <= h->P.itrp1; ++it) {
            int rc;
            if (it == 1) {
                if ((rc = op_line<T>(h, r, qr, impfl, 0))) return rc;
            } else {
                T *tmp = Buf<T>::ar(h);                   // free until laplc(qr) overwrites it
                if ((rc = op_laplc_t<T>(h, qr, tmp, impfl))) return rc;
                {
                    KTIME(KT_MISC);
                    k_sub_mixed<T><<<grid(N), kThreads, 0, h->st>>>(N, r, tmp, h->tres);
                }
                if ((rc = op_line<T>(h, h->tres, qr, impfl, 1))) return rc;
            }
        }
        return check_launch("precon line (mixed)");
    }
    if (h->P.iprc == 4) {
        for (int it = 1; it <= h->P.itrp1; ++it) {
            int rc;
            if (it == 1) {
                if ((rc = op_wide<T>(h, r, qr, impfl, 0))) return rc;
            } else {
                T *tmp = Buf<T>::ar(h);
                if ((rc = op_laplc_t<T>(h, qr, tmp, impfl))) return rc;
                {
                    KTIME(KT_MISC);
                    k_sub_mixed<T><<<grid(N), kThreads, 0, h->st>>>(N, r, tmp, h->tres);
                }
                if ((rc = op_wide<T>(h, h->tres, qr, impfl, 1))) return rc;
            }
        }
        return check_launch("precon wide line (mixed)");
    }
    // iprc 0 or 1: the FP64 operator, then rounded to T
    int rc = op_precon(h, r, h->tres, h->ar, h->P.iprc, impfl, false);
    if (rc) return rc;
    {
        KTIME(KT_MISC);
        k_copy<double, T><<<grid(N), kThreads, 0, h->st>>>(N, h->tres, qr);
    }
    return check_launch("precon convert");
    }
}


// ------------------------------------------------------------------------------ learned preconditioner
constexpr int kNNDwBlocks = 296;

struct FinSigma {       // sc[0] = max|r| (the network's input scale)
    double *sc;
    __device__ void operator()(const double *v) const { sc[0] = v[0]; }
};
struct ProdAbsD {
    const double *a;
    __device__ void operator()(int n, double *v) const { v[0] = fabs(a[n]); }
};
template <class T>
struct ProdFinite {     // max |q|; NaN turns into +inf so the host can test it
    const T *q;
    __device__ void operator()(int n, double *v) const {
        const double x = (double)q[n];
        v[0] = (x == x) ? fabs(x) : INFINITY;
    }
};

nn::Geom nn_geom(mpg_handle h) {
    auto &N = h->nn;
    return nn::Geom{N.Th, N.Tv, N.iDh, N.iDv, N.bdiag, N.feat2, N.bnd};
}

int nn_alloc_infer(mpg_handle h) {
    auto &S = h->nn;
    int rc;
    if (h->CL.n) return mpg_fail(MPG_ERR_UNSUPPORTED, "learned preconditioner: periodic copy lists are not provided");
    if (!S.geom) {
        const size_t nh = (size_t)h->NE2 * h->L, n = h->N;
        if ((rc = dalloc(h, &S.Th, nh)) || (rc = dalloc(h, &S.Tv, n)) || (rc = dalloc(h, &S.iDh, n)) ||
            (rc = dalloc(h, &S.iDv, n)) || (rc = dalloc(h, &S.feat2, n)) || (rc = dalloc(h, &S.bnd, n)))
            return rc;
        if ((rc = upload(h, &S.bdiag, h->hs.lbabs))) return rc;
        {
            KTIME(KT_MISC);
            nn::k_nn_geom_faces<<<grid((int)(nh + n)), kThreads, 0, h->st>>>(h->M, h->d_e2a, h->d_e2b, h->vol,
                                                                            h->f[MPG_F_RH0], h->f[MPG_F_COEFW],
                                                                            h->P.delt, S.Th, S.Tv);
            nn::k_nn_geom_nodes<<<grid(h->N), kThreads, 0, h->st>>>(h->M, S.Th, S.Tv, S.iDh, S.iDv, S.feat2, S.bnd);
        }
        if ((rc = check_launch("nn geometry"))) return rc;
        S.geom = true;
    }
    if (!S.infer) {
        const size_t n = h->N;
        if ((rc = dalloc(h, &S.prm, nn::NPARAM)) || (rc = dalloc(h, &S.Wbf, (size_t)nn::NL * nn::C * nn::K3)) ||
            (rc = dalloc(h, &S.H[0], n * nn::C)) || (rc = dalloc(h, &S.H[1], n * nn::C)) ||
            (rc = dalloc(h, &S.z, n)) || (rc = dalloc(h, &S.sc, 4)) || (rc = dalloc(h, &S.err, 1)) ||
            (rc = dalloc(h, &S.X0, n * nn::FIN)))
            return rc;
        S.infer = true;
    }
    return MPG_OK;
}

int nn_alloc_train(mpg_handle h) {
    int rc = nn_alloc_infer(h);
    if (rc) return rc;
    auto &S = h->nn;
    if (S.train) return MPG_OK;
    const size_t n = h->N;
    S.Npad = (h->N + 15) / 16 * 16;
    const size_t np = S.Npad;
    if ((rc = dalloc(h, &S.grad, nn::NPARAM)) || (rc = dalloc(h, &S.m1, nn::NPARAM)) ||
        (rc = dalloc(h, &S.m2, nn::NPARAM)) || (rc = dalloc(h, &S.H[2], n * nn::C)) ||
        (rc = dalloc(h, &S.H[3], n * nn::C)) ||
        (rc = dalloc(h, &S.dH, n * nn::C)) || (rc = dalloc(h, &S.dH2, n * nn::C)) ||
        (rc = dalloc(h, &S.G0, n * nn::C)) || (rc = dalloc(h, &S.Gh, n * nn::C)) ||
        (rc = dalloc(h, &S.Gv, n * nn::C)) || (rc = dalloc(h, &S.Y, n)) || (rc = dalloc(h, &S.dU, np * nn::C)) ||
        (rc = dalloc(h, &S.qd, n)) || (rc = dalloc(h, &S.ed, n)) || (rc = dalloc(h, &S.dq, n)))
        return rc;
    for (int l = 0; l < 3; ++l)
        if ((rc = dalloc(h, &S.Xs[l], np * nn::K3))) return rc;
    const size_t nb = (size_t)(h->N + 255) / 256;
    const size_t pdw = std::max((size_t)(nn::C * nn::FIN + nn::C), (size_t)(nn::C + 2));
    if ((rc = dalloc(h, &S.pd, nb * pdw)) || (rc = dalloc(h, &S.pf, (size_t)kNNDwBlocks * (nn::C * nn::K3 + nn::C))))
        return rc;
    S.train = true;
    return MPG_OK;
}

// the three message-passing layers over the columns (input layer fused into the first, output
// layer into the last); with `train` every activation the backward pass reads is kept
template <int NS>
void nn_layers(mpg_handle h, const nn::Geom &G, double *qd, float *qf, bool train) {
    auto &S = h->nn;
    // persistent grid: as many CTAs as fit on the device at once (tensor memory included)
    if (!S.col_ctas) {
        // CTAs resident per SM from the kernel's own footprint: registers, static shared memory
        // (with the largest carveout requested) and the 512 tensor-memory columns of an SM.  The
        // occupancy API reported 1 for these kernels, which measured 2.8x slower than 4.
        cudaFuncSetAttribute(nn::k_nn_col<NS, true, false>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        cudaFuncSetAttribute(nn::k_nn_col<NS, false, false>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        cudaFuncSetAttribute(nn::k_nn_col<NS, false, true>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        int per_sm = 1 << 30, sms = 0, regs_sm = 65536, smem_sm = 228 * 1024;
        const void *fns[3] = {(const void *)nn::k_nn_col<NS, true, false>, (const void *)nn::k_nn_col<NS, false, false>,
                              (const void *)nn::k_nn_col<NS, false, true>};
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->dev);
        cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, h->dev);
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, h->dev);
        for (const void *fn : fns) {
            cudaFuncAttributes fa{};
            if (cudaFuncGetAttributes(&fa, fn) != cudaSuccess) { per_sm = 1; break; }
            const int regs_cta = ((fa.numRegs + 7) / 8 * 8) * nn::COL_THREADS;
            const int smem_cta = (int)fa.sharedSizeBytes + 1024;       // plus the per-CTA reserve
            per_sm = std::min(per_sm, std::min(regs_sm / std::max(regs_cta, 1), smem_sm / std::max(smem_cta, 1)));
        }
        cudaGetLastError();
        per_sm = std::max(1, std::min(per_sm, 512 / (int)nn::TC_TMEM_COLS));
        S.col_ctas = std::max(1, sms) * per_sm;
    }
    const int nb = std::min(h->NC, S.col_ctas);
    const size_t W = (size_t)nn::C * nn::K3;
    nn::k_nn_col<NS, true, false><<<nb, nn::COL_THREADS, 0, h->st>>>(
        h->M, G, nullptr, S.X0, S.Wbf, S.prm, 0, nullptr, nullptr, S.H[1], nullptr, nullptr,
        train ? S.H[0] : nullptr, train ? S.Xs[0] : nullptr, nullptr, S.err);
    __nv_bfloat16 *h2 = train ? S.H[2] : S.H[0];
    nn::k_nn_col<NS, false, false><<<nb, nn::COL_THREADS, 0, h->st>>>(
        h->M, G, S.H[1], nullptr, S.Wbf + W, S.prm, 1, nullptr, nullptr, h2, nullptr, nullptr,
        nullptr, train ? S.Xs[1] : nullptr, nullptr, S.err);
    nn::k_nn_col<NS, false, true><<<nb, nn::COL_THREADS, 0, h->st>>>(
        h->M, G, h2, nullptr, S.Wbf + 2 * W, S.prm, 2, S.z, S.sc, train ? S.H[3] : nullptr, qd, qf,
        nullptr, train ? S.Xs[2] : nullptr, train ? S.Y : nullptr, S.err);
}

// forward pass on residual r: z = M^{-1} r (impfl coefficients), sigma, the network; q in T.
// With `train` the activations are kept (H[0..3], X0, Xs) for the backward pass.
template <class T>
int nn_forward(mpg_handle h, const double *r, T *q, int impfl, bool train) {
    auto &S = h->nn;
    const int N = h->N;
    int rc;
    if (h->L > nn::COL_MAXL) return mpg_fail(MPG_ERR_UNSUPPORTED, "learned preconditioner: more than 128 levels");
    if ((rc = op_line<double>(h, r, S.z, impfl, 0))) return rc;
    if ((rc = reduce<1>(h, 0x1u, ProdAbsD{r}, FinSigma{S.sc}))) return rc;
    const nn::Geom G = nn_geom(h);
    double *qd = nullptr;
    float *qf = nullptr;
    if constexpr (std::is_same<T, double>::value) qd = q; else qf = q;
    {
        KTIME(KT_NN);
        nn::k_nn_features<<<grid(N), kThreads, 0, h->st>>>(N, r, S.z, S.sc, G, S.X0);
        switch ((h->L + 31) / 32) {
            case 1: nn_layers<1>(h, G, qd, qf, train); break;
            case 2: nn_layers<2>(h, G, qd, qf, train); break;
            case 3: nn_layers<3>(h, G, qd, qf, train); break;
            default: nn_layers<4>(h, G, qd, qf, train); break;
        }
    }
    return check_launch("nn forward");
}

// backward pass (after nn_forward with train = true): gradient into S.grad and the loss.  Either
// for target t (error loss) or from dL/dq = dq * sc[2] (residual loss, loss already in sc[1]).
int nn_backward(mpg_handle h, const double *t, const double *dq, double *loss) {
    auto &S = h->nn;
    const int N = h->N;
    const nn::Geom G = nn_geom(h);
    const int nb = (N + 255) / 256;
    {
        KTIME(KT_NN);
        nn::k_nn_out_bwd<<<nb, 256, 0, h->st>>>(N, S.H[3], S.Y, t, dq, S.z, S.sc, G, S.prm, S.dH, S.pd);
        // partial columns: dw_out (C), db_out, loss
        nn::k_nn_fold_d<<<1, 64, 0, h->st>>>(nb, nn::C + 2, nn::C + 1, S.pd, S.grad + nn::OFF_WOUT);
    }
    double *dl = S.sc + 1;
    if (!dq) {
        KTIME(KT_NN);
        // sum of the per-block loss partials (column C+1) in fixed order
        const double *pdp = S.pd;
        k_reduce<1><<<1, kRedThreads, 0, h->st>>>(nb, 0u,
            [=] __device__(int b, double *v) { v[0] = pdp[(size_t)b * (nn::C + 2) + nn::C + 1]; },
            [=] __device__(const double *v) { dl[0] = v[0]; }, h->part, h->counter, nullptr);
    }
    const int ntiles = (N + nn::TILE - 1) / nn::TILE;
    const int nblk = std::min((ntiles + nn::BWARPS - 1) / nn::BWARPS, 148 * 16);
    for (int l = nn::NL - 1; l >= 0; --l) {
        KTIME(KT_NN);
        nn::k_nn_layer_bwd<<<nblk, 32 * nn::BWARPS, 0, h->st>>>(N, S.H[l + 1], S.dH, S.Wbf + (size_t)l * nn::C * nn::K3,
                                                                 G, S.G0, S.Gh, S.Gv, S.dU);
        nn::k_nn_spread<<<grid(4 * N), kThreads, 0, h->st>>>(h->M, G, S.G0, S.Gh, S.Gv, S.dH2);
        nn::k_nn_dw<<<kNNDwBlocks, 32 * nn::WARPS, 0, h->st>>>(S.Npad, S.dU, S.Xs[l], S.pf);
        const int width = nn::C * nn::K3 + nn::C;
        nn::k_nn_fold_f<<<(width + 255) / 256, 256, 0, h->st>>>(kNNDwBlocks, width, width, S.pf,
                                                                S.grad + nn::OFF_L0 + l * nn::LSTRIDE);
        std::swap(S.dH, S.dH2);
    }
    {
        KTIME(KT_NN);
        nn::k_nn_in_bwd<<<nb, 256, 0, h->st>>>(N, S.H[0], S.dH, S.X0, S.pd);
        const int width = nn::C * nn::FIN + nn::C;
        nn::k_nn_fold_d<<<(width + 255) / 256, 256, 0, h->st>>>(nb, width, width, S.pd, S.grad + nn::OFF_WIN);
    }
    int rc = check_launch("nn backward");
    if (rc) return rc;
    if (loss) {
        MPG_CUDA(cudaMemcpyAsync(loss, dl, sizeof(double), cudaMemcpyDeviceToHost, h->st));
        MPG_CUDA(cudaStreamSynchronize(h->st));
    }
    return MPG_OK;
}

int nn_adam(mpg_handle h, float lr) {
    auto &S = h->nn;
    S.adam_t += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - powf(b1, (float)S.adam_t), c2 = 1.f - powf(b2, (float)S.adam_t);
    {
        KTIME(KT_NN);
        nn::k_nn_adam<<<(nn::NPARAM + 255) / 256, 256, 0, h->st>>>(nn::NPARAM, S.prm, S.grad, S.m1, S.m2, lr, b1, b2,
                                                                    1e-8f, c1, c2);
        nn::k_nn_to_bf16<<<(nn::NL * nn::C * nn::K3 + 255) / 256, 256, 0, h->st>>>(S.prm, S.Wbf);
    }
    return check_launch("nn adam");
}

// Residual loss of a preconditioner output q: the residual left by the best GCR step along q,
// L = 0.5 min_alpha ||r - alpha A q||_W^2 / ||r||_W^2 = 0.5 (1 - <Aq,r>_W^2 / (||Aq||_W^2 ||r||_W^2)).
// It does not depend on the scale of q, as GCR does not.  With a = A q, alpha = <a,r>/<a,a> and
// e = alpha a - r, dL/dq = (alpha / ||r||^2) A^T W e (alpha is optimal, so its own variation drops).
// Reduction: v = (<a,r>_W, <a,a>_W, <r,r>_W) -> sc[1] = L, sc[2] = alpha/||r||^2, sc[3] = alpha.
struct ProdWLoss {
    const double *a, *r, *vol, *rh0;
    __device__ void operator()(int n, double *v) const {
        const double w = vol[n] * rh0[n];
        v[0] = w * a[n] * r[n];
        v[1] = w * a[n] * a[n];
        v[2] = w * r[n] * r[n];
    }
};
struct FinWLoss {
    double *sc;
    __device__ void operator()(const double *v) const {
        const double aa = v[1] > 0. ? v[1] : 1., rr = v[2] > 0. ? v[2] : 1.;
        const double alpha = v[0] / aa;
        const double c2 = v[0] * v[0] / (aa * rr);
        sc[1] = 0.5 * (1. - (c2 < 1. ? c2 : 1.));
        sc[2] = alpha / rr;
        sc[3] = alpha;
    }
};
// e = sc[3] a - r
__global__ void k_step_residual(int N, const double *__restrict__ sc, const double *__restrict__ a,
                                const double *__restrict__ r, double *__restrict__ e) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n < N) e[n] = sc[3] * a[n] - r[n];
}

// loss and gradient for residual r (and target t for the error loss) with the selected loss
int nn_grad(mpg_handle h, const double *r, const double *t, double *loss) {
    auto &S = h->nn;
    int rc;
    if (S.loss_mode == MPG_NN_LOSS_ERROR) {
        if ((rc = nn_forward<double>(h, r, h->tres, 1, true))) return rc;
        return nn_backward(h, t, nullptr, loss);
    }
    // residual loss: q = net(r), a = A q, e = alpha a - r, dL/dq = (alpha/||r||^2) A^T W e
    if ((rc = nn_forward<double>(h, r, S.qd, 1, true))) return rc;
    if ((rc = op_laplc(h, S.qd, S.ed, 1))) return rc;
    if ((rc = reduce<3>(h, 0u, ProdWLoss{S.ed, r, h->vol, h->f[MPG_F_RH0]}, FinWLoss{S.sc}))) return rc;
    {
        KTIME(KT_NN);
        k_step_residual<<<grid(h->N), kThreads, 0, h->st>>>(h->N, S.sc, S.ed, r, S.ed);
    }
    if ((rc = op_laplc_adj(h, S.ed, S.dq, 1, false))) return rc;
    return nn_backward(h, nullptr, S.dq, loss);
}

// learned preconditioner inside gcrk; returns 1 in *fell_back when it handed over to the plain one
template <class T>
int op_precon_learned(mpg_handle h, const double *r, int impfl, bool &active) {
    T *qr = Buf<T>::qr(h);
    int rc;
    if (active) {
        if ((rc = nn_forward<T>(h, r, qr, impfl, false))) return rc;
        if ((rc = reduce<1>(h, 0x1u, ProdFinite<T>{qr}, NoFin{}))) return rc;
        if ((rc = fetch_result(h, 1))) return rc;
        if (std::isfinite(h->h_res[0])) return MPG_OK;
        active = false;                        // non-finite output: plain preconditioner from now on
        h->nn.fallbacks += 1;
    }
    mpg_params save = h->P;
    h->P.iprc = 2;
    rc = op_precon_gcr<T>(h, r, impfl);
    h->P = save;
    return rc;
}

// ------------------------------------------------------------------------------ GCR
struct FinEps {   // eer0, eem0, rl20 clamped by epa
    double *scal;
    __device__ void operator()(const double *v) const {
        const double epa = 1.e-38;
        scal[S_EER0] = amax(v[0], epa);
        scal[S_EEM0] = amax(v[1], epa);
        scal[S_RL20] = amax(v[2], epa);
    }
};
struct FinBeta {
    double *scal;
    int i;
    __device__ void operator()(const double *v) const {
        const double ax2 = amax(1.e-38, v[1]);
        scal[S_AX2 + i] = ax2;
        scal[S_BETA] = -v[0] / ax2;
    }
};
struct FinDel {
    double *scal;
    int i;
    __device__ void operator()(const double *v) const {
        for (int ii = 0; ii < i; ++ii) scal[S_DEL + ii] = -v[ii] / scal[S_AX2 + ii];
    }
};
template <class T>
struct ProdNorm0 {
    const T *qr;
    const double *r;
    __device__ void operator()(int n, double *v) const {
        const double q = (double)qr[n], s = r[n];
        v[0] = q * q;
        v[1] = fabs(q);
        v[2] = s * s;
    }
};
template <class T>
struct ProdDot2 {
    const double *r;
    const T *a;
    __device__ void operator()(int n, double *v) const {
        const double x = (double)a[n];
        v[0] = r[n] * x;
        v[1] = x * x;
    }
};
template <class T>
struct ProdAxpy {   // p += beta x, r += beta ax; returns |r|, r^2
    const double *scal;
    const T *x, *a;
    double *p, *r;
    struct Loaded { double p, r, x, a; };
    __device__ Loaded load(int n) const { return Loaded{p[n], r[n], (double)x[n], (double)a[n]}; }
    __device__ void finish(int n, const Loaded &l, double *v) const {
        const double beta = scal[S_BETA];
        p[n] = l.p + beta * l.x;
        const double rn = l.r + beta * l.a;
        r[n] = rn;
        v[0] = fabs(rn);
        v[1] = rn * rn;
    }
};
template <int NQ, class T>
struct ProdDots {
    const T *ar;
    const T *ax[MPG_MAX_LORD];
    int i;
    struct Loaded { double a, x[NQ]; };
    __device__ Loaded load(int n) const {
        Loaded l;
        l.a = (double)ar[n];
#pragma unroll
        for (int q = 0; q < NQ; ++q) l.x[q] = q < i ? (double)ax[q][n] : 0.0;
        return l;
    }
    __device__ void finish(int, const Loaded &l, double *v) const {
#pragma unroll
        for (int q = 0; q < NQ; ++q) v[q] = q < i ? l.x[q] * l.a : 0.0;
    }
};
template <class T>
struct ProdQ {
    const T *qr;
    __device__ void operator()(int n, double *v) const {
        const double q = (double)qr[n];
        v[0] = q * q;
        v[1] = fabs(q);
    }
};

template <class T>
int gcr_dots(mpg_handle h, int i) {
    FinDel fin{h->scal, i};
    if (i <= 4) {
        ProdDots<4, T> pd{Buf<T>::ar(h), {}, i};
        for (int q = 0; q < h->P.lord; ++q) pd.ax[q] = Buf<T>::ax(h, q);
        return reduce<4>(h, 0u, pd, fin);
    }
    if (i <= 8) {
        ProdDots<8, T> pd{Buf<T>::ar(h), {}, i};
        for (int q = 0; q < h->P.lord; ++q) pd.ax[q] = Buf<T>::ax(h, q);
        return reduce<8>(h, 0u, pd, fin);
    }
    ProdDots<16, T> pd{Buf<T>::ar(h), {}, i};
    for (int q = 0; q < h->P.lord; ++q) pd.ax[q] = Buf<T>::ax(h, q);
    return reduce<16>(h, 0u, pd, fin);
}

// x(:,i+1) = qr + sum del(ii) x(:,ii), ax likewise (ref.f:1914-1923), or the restart collapse
// into x(:,1) (ref.f:1924-1937), with the next iteration's r.ax and ax.ax (ref.f:1881-1884)
// reduced in the same pass.  I = number of previous directions, known at compile time.
template <class T>
struct VecListT {
    T *v[MPG_MAX_LORD];
};

template <int I, bool RESTART, class T>
struct ProdUpdate {
    const double *scal;
    const T *qr, *ar;
    const double *r;
    VecListT<T> x, ax;
    T *xo, *axo;
    struct Loaded { double q, a, r, x[I], ax[I]; };
    __device__ Loaded load(int n) const {
        Loaded l;
        l.q = (double)qr[n];
        l.a = (double)ar[n];
        l.r = r[n];
#pragma unroll
        for (int ii = 0; ii < I; ++ii) {
            l.x[ii] = (double)x.v[ii][n];
            l.ax[ii] = (double)ax.v[ii][n];
        }
        return l;
    }
    __device__ void finish(int n, const Loaded &l, double *v) const {
        double a, b;
        if (RESTART) {
            a = l.q + scal[S_DEL] * l.x[0];
            b = l.a + scal[S_DEL] * l.ax[0];
#pragma unroll
            for (int ii = 1; ii < I; ++ii) {
                const double d = scal[S_DEL + ii];
                a = a + d * l.x[ii];
                b = b + d * l.ax[ii];
            }
        } else {
            a = l.q;
            b = l.a;
#pragma unroll
            for (int ii = 0; ii < I; ++ii) {
                const double d = scal[S_DEL + ii];
                a = a + d * l.x[ii];
                b = b + d * l.ax[ii];
            }
        }
        const T at = (T)a, bt = (T)b;
        xo[n] = at;
        axo[n] = bt;
        const double bs = (double)bt;        // the stored direction, as the next iteration reads it
        v[0] = l.r * bs;
        v[1] = bs * bs;
    }
};

template <int I, class T>
int gcr_update_n(mpg_handle h, int lord) {
    VecListT<T> x{}, ax{};
    for (int q = 0; q < lord; ++q) { x.v[q] = Buf<T>::x(h, q); ax.v[q] = Buf<T>::ax(h, q); }
    if (I < lord) {
        ProdUpdate<I, false, T> pu{h->scal, Buf<T>::qr(h), Buf<T>::ar(h), h->r, x, ax, Buf<T>::x(h, I), Buf<T>::ax(h, I)};
        return reduce<2>(h, 0u, pu, FinBeta{h->scal, I});
    }
    ProdUpdate<I, true, T> pu{h->scal, Buf<T>::qr(h), Buf<T>::ar(h), h->r, x, ax, Buf<T>::x(h, 0), Buf<T>::ax(h, 0)};
    return reduce<2>(h, 0u, pu, FinBeta{h->scal, 0});
}

template <class T>
int gcr_update(mpg_handle h, int i, int lord) {
    switch (i) {
        case 1: return gcr_update_n<1, T>(h, lord);
        case 2: return gcr_update_n<2, T>(h, lord);
        case 3: return gcr_update_n<3, T>(h, lord);
        case 4: return gcr_update_n<4, T>(h, lord);
        case 5: return gcr_update_n<5, T>(h, lord);
        case 6: return gcr_update_n<6, T>(h, lord);
        case 7: return gcr_update_n<7, T>(h, lord);
        case 8: return gcr_update_n<8, T>(h, lord);
        case 9: return gcr_update_n<9, T>(h, lord);
        case 10: return gcr_update_n<10, T>(h, lord);
        case 11: return gcr_update_n<11, T>(h, lord);
        case 12: return gcr_update_n<12, T>(h, lord);
        case 13: return gcr_update_n<13, T>(h, lord);
        case 14: return gcr_update_n<14, T>(h, lord);
        case 15: return gcr_update_n<15, T>(h, lord);
        default: return gcr_update_n<16, T>(h, lord);
    }
}

// gcrk(p, u1, v1, w1, u2, v2, w2, impfl) — ref.f:1776-1972.  T is the storage type of the
// directions x, ax and of qr, ar (double; float in mixed precision); p, r, every inner product,
// the coefficients and the stopping test are FP64 in both.
template <class T>
int op_gcrk_t(mpg_handle h, double *p, const double *u1, const double *v1, const double *w1, double *u2,
              double *v2, double *w2, int impfl) {
    using B = Buf<T>;
    const mpg_params &P = h->P;
    const int N = h->N, lord = P.lord, itmn = P.itmn > 0 ? P.itmn : 3;
    const double eps = P.eps0 / P.delt, epa = 1.e-38;
    int nlc = 0, rc;
    // learned preconditioner (iprc = 3): active until it fails, then the plain line solve
    const bool learned = (P.iprc == 3);
    bool lon = learned;
    int fallbacks = 0;
    if (learned) {
        if ((rc = nn_alloc_infer(h))) return rc;
        if (!h->nn.have_params) return mpg_fail(MPG_ERR_ARG, "iprc=3 needs network parameters (mpg_learned_init/set_params)");
    }
    auto precon = [&]() -> int {
        if (!learned) return op_precon_gcr<T>(h, h->r, impfl);
        const int before = h->nn.fallbacks;
        const int r2 = op_precon_learned<T>(h, h->r, impfl, lon);
        fallbacks += h->nn.fallbacks - before;
        return r2;
    };
    // harvesting of (r_i, p_i) pairs for training, from plain solves with impfl = 1
    auto &NNS = h->nn;
    const bool harvest = NNS.every > 0 && !learned && impfl == 1 && NNS.rec_r;
    const int first_rec = NNS.nrec;
    if ((rc = op_prfr(h, p, u1, v1, w1, u2, v2, w2, impfl))) return rc;
    if ((rc = op_div(h, u2, v2, w2, h->r, -1))) return rc;
    if ((rc = precon())) return rc;
    if ((rc = reduce<3>(h, 0x2u, ProdNorm0<T>{B::qr(h), h->r}, FinEps{h->scal}))) return rc;
    if ((rc = fetch_result(h, 3))) return rc;
    double rl20 = h->h_res[2] > epa ? h->h_res[2] : epa;
    const double rl2_init = rl20;
    // learned preconditioner: kept while ||r||_2 after m updates is <= nn_rate^m of its start
    const double nn_rate = P.nn_rate > 0. ? P.nn_rate : 0.98;
    int nupd = 0;
    {
        KTIME(KT_MISC);
        k_copy<T, T><<<grid(N), kThreads, 0, h->st>>>(N, B::qr(h), B::x(h, 0));
    }
    if ((rc = op_laplc_t<T>(h, B::x(h, 0), B::ax(h, 0), impfl))) return rc;
    int status = MPG_GCR_MAXIT;
    double dvmx = 0., rl2 = 0.;
    for (int it = 1; it <= P.itr && status == MPG_GCR_MAXIT; ++it) {
        for (int i = 1; i <= lord; ++i) {
            if (it == 1 && i == 1)      // later iterations get (r.ax, ax.ax) from gcr_update
                if ((rc = reduce<2>(h, 0u, ProdDot2<T>{h->r, B::ax(h, 0)}, FinBeta{h->scal, 0}))) return rc;
            if ((rc = reduce<2>(h, 0x1u, ProdAxpy<T>{h->scal, B::x(h, i - 1), B::ax(h, i - 1), p, h->r}, NoFin{})))
                return rc;
            if ((rc = fetch_result(h, 2))) return rc;
            dvmx = h->h_res[0] > -1.e15 ? h->h_res[0] : -1.e15;
            rl2 = h->h_res[1];
            ++nupd;
            if (!std::isfinite(dvmx) || !std::isfinite(rl2)) { status = MPG_GCR_NAN; break; }
            if (dvmx <= eps && it >= itmn) { status = MPG_GCR_CONVERGED; break; }
            if (learned && lon && nupd >= lord && std::sqrt(rl2 / rl2_init) > std::pow(nn_rate, (double)nupd)) {
                lon = false;                  // slower than the required contraction: plain from here on
                ++fallbacks;
            }
            if (rl2 >= rl20) {
                if (!(learned && lon)) { status = MPG_GCR_STALLED; break; }
                lon = false;                  // no progress with the network: plain from here on
                ++fallbacks;
            }
            rl20 = rl2 > epa ? rl2 : epa;
            if (harvest && nlc % NNS.every == 0 && NNS.nrec < NNS.maxrec) {
                KTIME(KT_MISC);
                const size_t off = (size_t)NNS.nrec * N;
                k_copy<double, double><<<grid(N), kThreads, 0, h->st>>>(N, h->r, NNS.rec_r + off);
                k_copy<double, double><<<grid(N), kThreads, 0, h->st>>>(N, p, NNS.rec_t + off);
                NNS.nrec += 1;
            }
            if ((rc = precon())) return rc;
            if ((rc = op_laplc_t<T>(h, B::qr(h), B::ar(h), impfl))) return rc;
            nlc = nlc + 1;
            if ((rc = gcr_dots<T>(h, i))) return rc;
            // direction update fused with the next iteration's (r.ax, ax.ax) reduction
            if ((rc = gcr_update<T>(h, i, lord))) return rc;
        }
    }
    if (harvest) {
        if (status == MPG_GCR_CONVERGED) {
            KTIME(KT_MISC);
            for (int j = first_rec; j < NNS.nrec; ++j)     // t_j = p_j - p*  (= A^{-1} r_j)
                k_sub<<<grid(N), kThreads, 0, h->st>>>(N, NNS.rec_t + (size_t)j * N, p, NNS.rec_t + (size_t)j * N);
        } else {
            NNS.nrec = first_rec;
        }
    }
    h->last_fallbacks = fallbacks;
    h->rate_last = (nupd > 0 && rl2 > 0. && std::isfinite(rl2)) ? std::pow(rl2 / rl2_init, 0.5 / nupd) : 0.;
    if ((rc = reduce<2>(h, 0x2u, ProdQ<T>{B::qr(h)}, NoFin{}))) return rc;
    if ((rc = fetch_result(h, 2))) return rc;
    double eer = h->h_res[0], eem = h->h_res[1] > -1.e15 ? h->h_res[1] : -1.e15;
    double s0[3];
    MPG_CUDA(cudaMemcpyAsync(s0, h->scal + S_EER0, sizeof s0, cudaMemcpyDeviceToHost, h->st));
    MPG_CUDA(cudaStreamSynchronize(h->st));
    h->eer = eer / s0[0];
    h->eem = eem / s0[1];
    h->niter = nlc;
    h->nitsm = h->nitsm + nlc;
    h->icount = h->icount + 1;
    h->gstatus = status;
    if ((rc = lap_fused_check(h))) return rc;
    h->dvmx_last = dvmx;
    h->rl2_last = rl2;
    return MPG_OK;
}

int op_gcrk(mpg_handle h, double *p, const double *u1, const double *v1, const double *w1, double *u2,
            double *v2, double *w2, int impfl) {
    if (h->P.precision == MPG_PREC_MIXED) return op_gcrk_t<float>(h, p, u1, v1, w1, u2, v2, w2, impfl);
    return op_gcrk_t<double>(h, p, u1, v1, w1, u2, v2, w2, impfl);
}

// ------------------------------------------------------------------------------ MPDATA
// scratch of MPDATA in the intermediate type T
template <class T> struct MpBuf;
template <> struct MpBuf<double> {
    static MpScratch &S(mpg_handle h) { return h->S; }
    static double *psi1(mpg_handle h) { return h->psi1; }
    static double *g(mpg_handle h, int d) { return h->g3[d]; }
    static double *mx(mpg_handle h) { return h->mx; }
    static double *mn(mpg_handle h) { return h->mn; }
    static double *psi1d(mpg_handle h) { return h->psi1; }     // the first-pass field in FP64
    static double *cp(mpg_handle h) { return h->g3[0]; }       // the gradient buffers, dead by then
    static double *cn(mpg_handle h) { return h->g3[1]; }
};
template <> struct MpBuf<float> {
    static MpScratchT<float> &S(mpg_handle h) { return h->Sf; }
    static float *psi1(mpg_handle h) { return h->psi1f; }
    static float *g(mpg_handle h, int d) { return h->g3f[d]; }
    static double *mx(mpg_handle h) { return h->mxd; }
    static double *mn(mpg_handle h) { return h->mnd; }
    static double *psi1d(mpg_handle h) { return h->psi1d; }
    static double *cp(mpg_handle h) { return h->cpd; }
    static double *cn(mpg_handle h) { return h->cnd; }
};

template <class T>
int op_aun_t(mpg_handle h) {
    U3 U{{h->f[MPG_F_UUU], h->f[MPG_F_UUU + 1], h->f[MPG_F_UUU + 2]}};
    const int nt = h->NE2 * h->L + h->N;
    {
        KTIME(KT_AUN);
        k_aun<T><<<grid(nt), kThreads, 0, h->st>>>(h->M, MpBuf<T>::S(h), U);
    }
    return check_launch("aun");
}
int op_aun(mpg_handle h) {
    return h->P.precision == MPG_PREC_MIXED ? op_aun_t<float>(h) : op_aun_t<double>(h);
}

// one mpdatamper call (iper = 2) or mpdatam call (iper = 0); T is the type of the face fluxes
// and the intermediate node fields; iflag names the field as in the reference (1-4: u, v, w,
// theta'; passive scalars, not in the reference, follow with inflow value 0)
template <class T>
int op_mpdata_field_t(mpg_handle h, double *psi, int iflag) {
    using B = MpBuf<T>;
    using G = Buf<T>;
    const T dt = (T)h->P.delt;
    const T *vol = G::vol(h), *rh0 = G::rh0(h);
    const int N = h->N;
    auto &S = B::S(h);
    // face fluxes and the antidiffusive velocity in T; the node work of both passes (donor fluxes
    // from the FP64 field, FCT bounds, in/out sums, limiter ratios, updates) in FP64 on FP64 vol
    // and rh0, with the first-pass field kept in FP64 beside its T copy in mixed precision
    const bool mixed = std::is_same<T, float>::value;
    const MpUpdate U64{mixed ? h->psi1d : nullptr, h->vol, h->f[MPG_F_RH0], h->P.delt};
    const double *b1 = B::psi1d(h);                       // the FP64 first-pass field
    {
        KTIME(KT_MP_DONOR);
        if (h->P.iper == 2) {
            k_mp_donor<T, false><<<grid(N), kThreads, 0, h->st>>>(h->M, S, psi, B::psi1(h),
                                                                  MpInflow{nullptr, 0., 0}, U64);
            if (h->CL.n)
                k_cp_mp_donor<T><<<grid(h->CL.n), kThreads, 0, h->st>>>(h->M, h->CL, S, psi, B::psi1(h), U64);
        } else {
            // afree = (u0inf, v0inf, w0inf, 0, 1) (ref.f:125-129); iflag = 1 takes ue per node
            const double af = iflag == 2 ? h->P.v0inf : iflag == 3 ? h->P.w0inf : 0.;
            k_mp_donor<T, true><<<grid(N), kThreads, 0, h->st>>>(h->M, S, psi, B::psi1(h),
                                                                 MpInflow{h->ue, af, iflag}, U64);
        }
    }
    {
        KTIME(KT_MP_GRADB);
        const double *bsrc = mixed ? b1 : nullptr;
        if (h->P.iper == 2) {
            k_mp_grad_bounds<T, false><<<grid(N), kThreads, 0, h->st>>>(h->M, B::psi1(h), bsrc, B::g(h, 0),
                                                                        B::g(h, 1), B::g(h, 2), B::mx(h), B::mn(h));
            if (h->CL.n) {
                k_cp_mp_grad<T><<<grid(h->CL.n), kThreads, 0, h->st>>>(h->M, h->CL, B::psi1(h), B::g(h, 0),
                                                                       B::g(h, 1), B::g(h, 2));
                k_cp_bounds<<<grid(h->CL.ngroups), kThreads, 0, h->st>>>(h->CL, b1, B::mx(h), B::mn(h));
            }
        }
        else
            k_mp_grad_bounds<T, true><<<grid(N), kThreads, 0, h->st>>>(h->M, B::psi1(h), bsrc, B::g(h, 0),
                                                                       B::g(h, 1), B::g(h, 2), B::mx(h), B::mn(h));
    }
    AntiArgs<T> A{B::psi1(h), B::g(h, 0), B::g(h, 1), B::g(h, 2), vol, rh0,
                  U3{{h->f[MPG_F_UUU], h->f[MPG_F_UUU + 1], h->f[MPG_F_UUU + 2]}}, dt};
    const int nt = h->NE2 * h->L + h->N;
    {
        KTIME(KT_MP_ANTI);
        k_mp_anti<T><<<grid(nt), kThreads, 0, h->st>>>(h->M, S, A);
    }
    {
        KTIME(KT_MP_CPCN);
        k_mp_cpcn<T><<<grid(N), kThreads, 0, h->st>>>(h->M, S, b1, B::mx(h), B::mn(h), h->vol, h->f[MPG_F_RH0],
                                                      h->P.delt, B::cp(h), B::cn(h));
        if (h->CL.n)
            k_cp_mp_cpcn<T><<<grid(h->CL.n), kThreads, 0, h->st>>>(h->M, h->CL, S, b1, B::mx(h), B::mn(h), h->vol,
                                                                   h->f[MPG_F_RH0], h->P.delt, B::cp(h), B::cn(h));
    }
    {
        KTIME(KT_MP_PASS2);
        k_mp_pass2<T><<<grid(N), kThreads, 0, h->st>>>(h->M, S, B::psi1(h), B::cp(h), B::cn(h), U64, psi);
        if (h->CL.n)
            k_cp_mp_pass2<T><<<grid(h->CL.n), kThreads, 0, h->st>>>(h->M, h->CL, S, B::psi1(h), B::cp(h), B::cn(h),
                                                                    U64, psi);
    }
    return check_launch("mpdata");
}
int op_mpdata_field(mpg_handle h, double *psi, int iflag) {
    return h->P.precision == MPG_PREC_MIXED ? op_mpdata_field_t<float>(h, psi, iflag)
                                            : op_mpdata_field_t<double>(h, psi, iflag);
}

Fields make_fields(mpg_handle h) {
    Fields F{};
    for (int q = 0; q < 4; ++q) { F.unk[q] = fld(h, MPG_F_UNK + q); F.frc[q] = fld(h, MPG_F_FRC + q); }
    for (int q = 0; q < 3; ++q) {
        F.uuu[q] = fld(h, MPG_F_UUU + q);
        F.uuu0[q] = fld(h, MPG_F_UUU0 + q);
        F.ud[q] = fld(h, MPG_F_UNKDASH + q);
        F.unk1[q] = fld(h, MPG_F_UNK1 + q);
    }
    F.rh0 = h->f[MPG_F_RH0]; F.th0 = h->f[MPG_F_TH0]; F.the = h->f[MPG_F_THE];
    F.dthedz = h->f[MPG_F_DTHEDZ]; F.coefw = h->f[MPG_F_COEFW]; F.alpha = h->f[MPG_F_ALPHA];
    F.ue = h->ue; F.ve = h->ve;
    return F;
}

// ------------------------------------------------------------------------------ velprd
// velprd(unk, frc, uuu, uuu1, unkdash) (ref.f:4448-4528): a first-order prediction of the velocity,
// made divergence-free by its own potential solve (gcrk + prfr with impfl = 0, from p = 0)
int op_velprd(mpg_handle h) {
    const int N = h->N;
    Fields F = make_fields(h);
    double *u1[3];
    for (int q = 0; q < 3; ++q)
        if (!(u1[q] = fld(h, MPG_F_UUU1 + q))) return mpg_fail(MPG_ERR_NOMEM, "uuu1");
    int rc;
    if (!h->vp[0])
        for (int q = 0; q < 4; ++q)
            if ((rc = dalloc(h, &h->vp[q], (size_t)N))) return rc;
    double *pp = h->vp[0], *ff[3] = {h->vp[1], h->vp[2], h->vp[3]};
    {
        KTIME(KT_NODE);
        k_velprd_pre<<<grid(N), kThreads, 0, h->st>>>(N, F, h->P.delt);
        const U3 U{{F.uuu[0], F.uuu[1], F.uuu[2]}};
        for (int q = 0; q < 3; ++q) {
            k_velprd_grad<<<grid(N), kThreads, 0, h->st>>>(h->M, F.ud[q], h->vol, U, h->P.delt, u1[q]);
            if (h->CL.n)
                k_cp_velprd_grad<<<grid(h->CL.n), kThreads, 0, h->st>>>(h->M, h->CL, F.ud[q], h->vol, U, h->P.delt,
                                                                        u1[q]);
        }
        k_fill<<<grid(N), kThreads, 0, h->st>>>(N, pp, 0.0);
        for (int q = 0; q < 3; ++q) k_fill<<<grid(N), kThreads, 0, h->st>>>(N, ff[q], 0.0);
    }
    if ((rc = check_launch("velprd"))) return rc;
    if ((rc = op_gcrk(h, pp, u1[0], u1[1], u1[2], ff[0], ff[1], ff[2], 0))) return rc;
    if ((rc = op_prfr(h, pp, u1[0], u1[1], u1[2], ff[0], ff[1], ff[2], 0))) return rc;
    {
        KTIME(KT_NODE);
        k_velprd_post<<<grid(N), kThreads, 0, h->st>>>(N, F, ff[0], ff[1], ff[2]);
    }
    return check_launch("velprd post");
}

// ------------------------------------------------------------------------------ diagnostics
struct ProdDivStats {
    const double *rhs;
    double dt;
    __device__ void operator()(int n, double *v) const {
        const double x = rhs[n] * dt;
        v[0] = x; v[1] = -x; v[2] = x;
    }
};
struct ProdSqDev {
    const double *a;
    double scale, mean;
    __device__ void operator()(int n, double *v) const {
        const double t = a[n] * scale - mean;
        v[0] = t * t;
    }
};
struct ProdCour {
    const double *c;
    __device__ void operator()(int n, double *v) const {
        v[0] = c[n]; v[1] = c[n]; v[2] = -c[n];
    }
};
struct ProdArg {
    const double *c;
    const int32_t *iperm;
    double mx;
    __device__ void operator()(int n, double *v) const { v[0] = c[n] == mx ? (double)iperm[n] : -1.0; }
};
struct ProdStats1 {
    const double *rh0, *vol;
    const double *u[8];
    int nf;
    __device__ void operator()(int n, double *v) const {
        const double r = rh0[n], vr = vol[n] * r;
        v[0] = r;
        for (int q = 0; q < 4; ++q) {
            const double x = u[q][n];
            v[1 + q] = r * x;
            v[5 + q] = x;
            v[9 + q] = -x;
        }
        for (int q = 0; q < 8; ++q) v[13 + q] = q < nf ? vr * u[q][n] : 0.0;
    }
};
struct ProdStats2 {
    const double *rh0;
    const double *u[4];
    double av[4];
    __device__ void operator()(int n, double *v) const {
        const double r = rh0[n];
        for (int q = 0; q < 4; ++q) {
            const double t = u[q][n] - av[q];
            v[q] = r * (t * t);
        }
    }
};
struct ProdScal {
    const double *u[4];
    int ns;
    __device__ void operator()(int n, double *v) const {
        for (int q = 0; q < 4; ++q) {
            const double x = q < ns ? u[q][n] : 0.0;
            v[q] = -x;
            v[4 + q] = x;
        }
    }
};

int diag_div(mpg_handle h, const double *rhs, mpg_diag *d) {
    int rc;
    const double dt = h->P.delt;
    if ((rc = reduce<3>(h, 0x3u, ProdDivStats{rhs, dt}, NoFin{}))) return rc;
    if ((rc = fetch_result(h, 3))) return rc;
    double divmx = h->h_res[0] > -1.e15 ? h->h_res[0] : -1.e15;
    double divmn = -h->h_res[1] < 1.e15 ? -h->h_res[1] : 1.e15;
    double divav = h->h_res[2] / (double)h->N;
    if ((rc = reduce<1>(h, 0u, ProdSqDev{rhs, dt, divav}, NoFin{}))) return rc;
    if ((rc = fetch_result(h, 1))) return rc;
    d->divmx = divmx; d->divmn = divmn; d->divav = divav;
    d->divsd = std::sqrt(h->h_res[0] / h->N);
    d->eer = h->eer; d->eem = h->eem; d->niter = h->niter;
    d->nitav = h->nitsm / (h->icount > 1 ? h->icount : 1);
    return MPG_OK;
}

int diag_courant(mpg_handle h, int iflag, mpg_diag *d) {
    int rc;
    U3 U{{h->f[MPG_F_UUU], h->f[MPG_F_UUU + 1], h->f[MPG_F_UUU + 2]}};
    double *cour = fld(h, MPG_F_COUR);
    {
        KTIME(KT_COURANT);
        k_courant<<<grid(h->N), kThreads, 0, h->st>>>(h->M, U, h->f[MPG_F_RH0], h->vol, h->P.delt, iflag, cour);
    }
    if ((rc = check_launch("courant"))) return rc;
    if (!d) return MPG_OK;
    if ((rc = reduce<3>(h, 0x6u, ProdCour{cour}, NoFin{}))) return rc;
    if ((rc = fetch_result(h, 3))) return rc;
    double crnav = h->h_res[0] / h->N;
    double crnmx = h->h_res[1] > -1.e9 ? h->h_res[1] : -1.e9;
    double crnmn = -h->h_res[2] < 1.e9 ? -h->h_res[2] : 1.e9;
    if ((rc = reduce<1>(h, 0x1u, ProdArg{cour, h->d_iperm, crnmx}, NoFin{}))) return rc;
    if ((rc = fetch_result(h, 1))) return rc;
    const int ic = (int)h->h_res[0] + 1;
    if ((rc = reduce<1>(h, 0u, ProdSqDev{cour, 1.0, crnav}, NoFin{}))) return rc;
    if ((rc = fetch_result(h, 1))) return rc;
    d->crnmx = crnmx; d->crnmn = crnmn; d->crnav = crnav;
    d->crnsd = std::sqrt(h->h_res[0] / h->N);
    d->icrnmx = ic;
    return MPG_OK;
}

// stats(unk) (ref.f:2847-2912) plus the FP64 mass sums and scalar extrema
int diag_stats(mpg_handle h, mpg_diag *d) {
    int rc;
    ProdStats1 p1{};
    p1.rh0 = h->f[MPG_F_RH0];
    p1.vol = h->vol;
    const int nf = 4 + h->P.nscal < 8 ? 4 + h->P.nscal : 8;
    for (int q = 0; q < 8; ++q) p1.u[q] = q < nf ? fld(h, MPG_F_UNK + q) : nullptr;
    p1.nf = nf;
    if ((rc = reduce<21>(h, 0x1FE0u, p1, NoFin{}))) return rc;
    if ((rc = fetch_result(h, 21))) return rc;
    double res[21];
    std::memcpy(res, h->h_res, sizeof res);
    const double rav = res[0];
    ProdStats2 p2{};
    p2.rh0 = h->f[MPG_F_RH0];
    for (int q = 0; q < 4; ++q) { p2.u[q] = p1.u[q]; p2.av[q] = res[1 + q] / rav; }
    if ((rc = reduce<4>(h, 0u, p2, NoFin{}))) return rc;
    if ((rc = fetch_result(h, 4))) return rc;
    for (int q = 0; q < 4; ++q) {
        const double mx = res[5 + q] > -1.e10 ? res[5 + q] : -1.e10;
        const double mn = -res[9 + q] < 1.e10 ? -res[9 + q] : 1.e10;
        const double sd = q < 3 ? std::sqrt(h->h_res[q] / rav) : std::sqrt(h->h_res[q] / h->N);
        d->stats[4 * q + 0] = mx; d->stats[4 * q + 1] = mn;
        d->stats[4 * q + 2] = p2.av[q]; d->stats[4 * q + 3] = sd;
    }
    for (int q = 0; q < 8; ++q) d->mass[q] = q < nf ? res[13 + q] : 0.0;
    const int ns = h->P.nscal < 4 ? h->P.nscal : 4;
    if (ns > 0) {
        ProdScal ps{};
        for (int q = 0; q < 4; ++q) ps.u[q] = q < ns ? fld(h, MPG_F_UNK + 4 + q) : p1.u[0];
        ps.ns = ns;
        if ((rc = reduce<8>(h, 0xFFu, ps, NoFin{}))) return rc;
        if ((rc = fetch_result(h, 8))) return rc;
        for (int q = 0; q < ns; ++q) { d->smin[q] = -h->h_res[q]; d->smax[q] = h->h_res[4 + q]; }
    }
    return MPG_OK;
}

}  // namespace

// ------------------------------------------------------------------------------ lifecycle
extern "C" int mpg_create(const mpg_params *prm, const mpg_mesh_ref *mesh, int device, mpg_handle *out) {
    if (!prm || !mesh || !out) return mpg_fail(MPG_ERR_ARG, "null argument");
    *out = nullptr;
    if (prm->isfera != 0) return mpg_fail(MPG_ERR_UNSUPPORTED, "isfera=1 (spherical variant) is not provided");
    if (prm->iper != 2 && prm->iper != 0) return mpg_fail(MPG_ERR_ARG, "iper must be 0 or 2");
    if (prm->mg_flag != 0 && prm->mg_flag != 1) return mpg_fail(MPG_ERR_ARG, "mg_flag must be 0 or 1");
    if (prm->mg_flag == 1 && (prm->iprc != 1 || prm->precision != MPG_PREC_FP64))
        return mpg_fail(MPG_ERR_UNSUPPORTED, "mg_flag=1 runs inside the reference smoother: iprc = 1, FP64");
    if (prm->ielast != 0) return mpg_fail(MPG_ERR_UNSUPPORTED, "ielast=1 is not provided");
    if (prm->lord < 1 || prm->lord > MPG_MAX_LORD) return mpg_fail(MPG_ERR_ARG, "lord out of range 1..16");
    if (prm->nscal < 0 || 4 + prm->nscal > MPG_MAX_UNK) return mpg_fail(MPG_ERR_ARG, "nscal out of range 0..12");
    if (prm->delt <= 0) return mpg_fail(MPG_ERR_ARG, "delt must be positive");
    if (prm->iprc < 0 || prm->iprc > 4) return mpg_fail(MPG_ERR_ARG, "iprc must be 0, 1, 2, 3 or 4");
    if (prm->precision != MPG_PREC_FP64 && prm->precision != MPG_PREC_MIXED)
        return mpg_fail(MPG_ERR_ARG, "precision must be MPG_PREC_FP64 or MPG_PREC_MIXED");
    HostColumnMesh hm;
    int rc = mpg_build_column_mesh(mesh, &hm);
    if (rc) return rc;
    // the reference's duplicate-node periodic form: copies keep their own faces, every edge sum
    // is completed over the copy group (cyclicr), and the copies' volumes are summed at set-up
    // (ref.f:99-103)
    std::vector<double> pvol;
    mpg_mesh_ref msh = *mesh;
    if (!hm.cp_node.empty()) {
        if (prm->iper != 2) return mpg_fail(MPG_ERR_ARG, "periodic copy lists (icoin/icoin2/icoin4) need iper = 2");
        if (prm->iprc == 3 || prm->iprc == 4 || prm->mg_flag == 1)
            return mpg_fail(MPG_ERR_UNSUPPORTED, "with periodic copy lists the preconditioner is iprc 0, 1 or 2 "
                                                 "without the V-cycle");
        pvol = mpg_periodic_volumes(mesh);
        msh.vol = pvol.data();
        for (int n = 0; n < hm.N; ++n) hm.vol[n] = pvol[hm.iperm[n]];
    }
    mesh = &msh;
    mpg_solver *h = new mpg_solver();
    h->P = *prm;
    h->dev = device;
    rc = mpg_host_static(prm, mesh, hm, &h->hs);
    if (rc) { delete h; return rc; }
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) { delete h; return mpg_fail(MPG_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e)); }
    e = cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking);
    if (e != cudaSuccess) { delete h; return mpg_fail(MPG_ERR_CUDA, std::string("stream: ") + cudaGetErrorString(e)); }
    h->NC = hm.NC; h->L = hm.L; h->N = hm.N; h->NE2 = hm.NE2;
    if (hm.L > 128) { delete h; return mpg_fail(MPG_ERR_MESH, "more than 128 levels per column"); }
    h->bitwise = hm.bitwise_order;
    h->betaunstr1 = h->hs.betaunstr1;
    h->iperm = hm.iperm;
    auto fail = [&](int code) { mpg_destroy(h); return code; };
    // mesh
    ColMesh &M = h->M;
    M.NC = hm.NC; M.L = hm.L; M.N = hm.N; M.NE2 = hm.NE2; M.iper = prm->iper;
    int32_t *cptr, *bptr;
    int2 *cadj;
    BEntry *bent;
    if ((rc = upload(h, &cptr, hm.cptr)) || (rc = upload(h, &cadj, hm.cadj)) || (rc = upload(h, &bptr, hm.bptr)))
        return fail(rc);
    std::vector<BEntry> be = hm.bent;
    if (be.empty()) be.push_back(BEntry{});
    if ((rc = upload(h, &bent, be))) return fail(rc);
    M.cptr = cptr; M.cadj = cadj; M.bptr = bptr; M.bent = bent;
    for (int d = 0; d < 3; ++d) {
        double *a, *b;
        if ((rc = upload(h, &a, hm.Sh[d])) || (rc = upload(h, &b, hm.Sv[d]))) return fail(rc);
        M.Sh[d] = a; M.Sv[d] = b;
    }
    if ((rc = upload(h, &h->d_perm, hm.perm)) || (rc = upload(h, &h->d_e2a, hm.e2a)) ||
        (rc = upload(h, &h->d_e2b, hm.e2b)))
        return fail(rc);
    if ((rc = upload(h, &h->vol, hm.vol)) || (rc = upload(h, &h->ue, h->hs.ue)) || (rc = upload(h, &h->ve, h->hs.ve)))
        return fail(rc);
    // static fields
    struct { int fid; std::vector<double> *v; } stat[] = {
        {MPG_F_RH0, &h->hs.rh0}, {MPG_F_TH0, &h->hs.th0}, {MPG_F_THE, &h->hs.the},
        {MPG_F_DTHEDZ, &h->hs.dthedz}, {MPG_F_ALPHA, &h->hs.alpha}, {MPG_F_COEFW, &h->hs.coefw},
        {MPG_F_D1, &h->hs.d1}};
    for (auto &s : stat)
        if ((rc = upload(h, &h->f[s.fid], *s.v))) return fail(rc);
    for (int q = 0; q < 2; ++q)
        if ((rc = upload(h, &h->la[q], h->hs.la[q])) || (rc = upload(h, &h->lm[q], h->hs.lm[q])) ||
            (rc = upload(h, &h->lcp[q], h->hs.lcp[q])))
            return fail(rc);
    if (prm->iprc == 4)
        for (int q = 0; q < 2; ++q)
            if ((rc = upload(h, &h->wa[q], h->hs.wa[q])) || (rc = upload(h, &h->wm[q], h->hs.wm[q])) ||
                (rc = upload(h, &h->wcp[q], h->hs.wcp[q])))
                return fail(rc);
    // workspace
    const size_t N = h->N;
    if ((rc = dalloc(h, &h->stage, N)) || (rc = dalloc(h, &h->r, N)) || (rc = dalloc(h, &h->qr, N)) ||
        (rc = dalloc(h, &h->ar, N)) || (rc = dalloc(h, &h->tres, N)))
        return fail(rc);
    for (int q = 0; q < 3; ++q)
        if ((rc = dalloc(h, &h->F[q], N))) return fail(rc);
    for (int q = 0; q < prm->lord; ++q)
        if ((rc = dalloc(h, &h->x[q], N)) || (rc = dalloc(h, &h->ax[q], N))) return fail(rc);
    if (prm->precision == MPG_PREC_MIXED) {
        for (int q = 0; q < prm->lord; ++q)
            if ((rc = dalloc(h, &h->xf[q], N)) || (rc = dalloc(h, &h->axf[q], N))) return fail(rc);
        if ((rc = dalloc(h, &h->qrf, N)) || (rc = dalloc(h, &h->arf, N))) return fail(rc);
        if ((rc = dalloc(h, &h->Ff4, N))) return fail(rc);
        auto tof = [](const std::vector<double> &v) {
            std::vector<float> o(v.size());
            for (size_t i = 0; i < v.size(); ++i) o[i] = (float)v[i];
            return o;
        };
        float *vf, *rf, *cf;
        if ((rc = upload(h, &vf, tof(hm.vol))) || (rc = upload(h, &rf, tof(h->hs.rh0))) ||
            (rc = upload(h, &cf, tof(h->hs.coefw))))
            return fail(rc);
        h->volf = vf; h->rh0f = rf; h->coefwf = cf;
        auto pack = [](const std::vector<double> *S) {
            std::vector<float4> o(S[0].size());
            for (size_t i = 0; i < o.size(); ++i)
                o[i] = make_float4((float)S[0][i], (float)S[1][i], (float)S[2][i], 0.f);
            return o;
        };
        float4 *a, *b;
        if ((rc = upload(h, &a, pack(hm.Sh))) || (rc = upload(h, &b, pack(hm.Sv)))) return fail(rc);
        M.Shf4 = a; M.Svf4 = b;
    }
    if ((rc = dalloc(h, &h->scal, S_COUNT)) || (rc = dalloc(h, &h->part, (size_t)kRedBlocks * kMaxQ)) ||
        (rc = dalloc(h, &h->result, kMaxQ)) || (rc = dalloc(h, &h->counter, 1)))
        return fail(rc);
    e = cudaMallocHost((void **)&h->h_res, sizeof(double) * kMaxQ);
    if (e != cudaSuccess) return fail(mpg_fail(MPG_ERR_NOMEM, "cudaMallocHost"));
    // MPDATA scratch in the precision of the run
    const size_t nh = (size_t)h->NE2 * h->L;
    if (prm->precision == MPG_PREC_MIXED) {
        float *aunh, *aunv, *Ah, *Av;
        if ((rc = dalloc(h, &aunh, nh)) || (rc = dalloc(h, &aunv, N)) || (rc = dalloc(h, &Ah, nh)) ||
            (rc = dalloc(h, &Av, N)) || (rc = dalloc(h, &h->psi1f, N)) || (rc = dalloc(h, &h->psi1d, N)) || (rc = dalloc(h, &h->mxd, N)) ||
            (rc = dalloc(h, &h->mnd, N)) || (rc = dalloc(h, &h->cpd, N)) || (rc = dalloc(h, &h->cnd, N)))
            return fail(rc);
        for (int q = 0; q < 3; ++q)
            if ((rc = dalloc(h, &h->g3f[q], N))) return fail(rc);
        h->Sf = MpScratchT<float>{aunh, aunv, Ah, Av, h->d_e2a, h->d_e2b};
    } else {
        double *aunh, *aunv, *Ah, *Av;
        if ((rc = dalloc(h, &aunh, nh)) || (rc = dalloc(h, &aunv, N)) || (rc = dalloc(h, &Ah, nh)) ||
            (rc = dalloc(h, &Av, N)) || (rc = dalloc(h, &h->psi1, N)) || (rc = dalloc(h, &h->mx, N)) ||
            (rc = dalloc(h, &h->mn, N)))
            return fail(rc);
        for (int q = 0; q < 3; ++q)
            if ((rc = dalloc(h, &h->g3[q], N))) return fail(rc);
        h->S = MpScratch{aunh, aunv, Ah, Av, h->d_e2a, h->d_e2b};
    }
    if ((rc = upload(h, &h->d_iperm, hm.iperm))) return fail(rc);
    if ((rc = dalloc(h, &h->dbuf, h->hs.la[0].size()))) return fail(rc);
    if (!hm.cp_node.empty()) {
        CopyList &CL = h->CL;
        int32_t *a, *b, *c2, *d, *e2, *f2;
        if ((rc = upload(h, &a, hm.cp_node)) || (rc = upload(h, &b, hm.cp_gbeg)) || (rc = upload(h, &c2, hm.cp_gsize)) ||
            (rc = upload(h, &d, hm.cp_members)) || (rc = upload(h, &e2, hm.cp_grp)) || (rc = upload(h, &f2, hm.cp_grpsize)))
            return fail(rc);
        CL.n = (int32_t)hm.cp_node.size();
        CL.node = a; CL.gbeg = b; CL.gsize = c2; CL.members = d;
        CL.ngroups = (int32_t)hm.cp_grp.size();
        CL.grp = e2; CL.grpsize = f2;
    }
    // MPG_LAPLC_FUSED=1: laplc's two halves in one persistent launch (k_lap_fused), not with copy
    // lists (their fix-up runs between the halves).  Bit-identical; measured slower than the two
    // launches on the 21.2M-node workload, hence not the default.
    const char *fused = std::getenv("MPG_LAPLC_FUSED");
    if (hm.cp_node.empty() && fused && fused[0] == '1') {
        // a divergence item's ticket comes one grid's worth of items after its last dependency
        if ((rc = lap_fused_ctas<double>(h)) || (rc = lap_fused_ctas<float>(h))) return fail(rc);
        std::vector<int32_t> sched, dptr;
        std::vector<int2> drng;
        const int32_t NG = mpg_laplc_schedule(hm, kThreads, std::max(h->lap_ctas[0], h->lap_ctas[1]), sched,
                                              dptr, drng);
        int32_t *a, *b, *f, *st;
        int2 *r;
        if ((rc = upload(h, &a, sched)) || (rc = upload(h, &b, dptr)) || (rc = upload(h, &r, drng)) ||
            (rc = dalloc(h, &f, (size_t)NG)) || (rc = dalloc(h, &st, 4)))
            return fail(rc);
        h->lap = LapSched{a, b, r, f, st, (int32_t)sched.size()};
    }
    if (prm->mg_flag == 1) {
        mg_neigh_definition(mesh, h->nb_ptr_ref, h->nb_lst_ref);
        mg_coords(mesh, h->cx_ref, h->cy_ref, h->cz_ref);
        if ((rc = dalloc(h, &h->mg_rrhs, N)) || (rc = dalloc(h, &h->mg_e, N))) return fail(rc);
    }
    e = cudaStreamSynchronize(h->st);
    if (e != cudaSuccess) return fail(mpg_fail(MPG_ERR_CUDA, std::string("create: ") + cudaGetErrorString(e)));
    *out = h;
    return MPG_OK;
}

extern "C" int mpg_destroy(mpg_handle h) {
    if (!h) return MPG_OK;
    if (h->st) cudaStreamSynchronize(h->st);
    for (auto &lv : h->mg)
        if (lv.sub) mpg_destroy(lv.sub);
    kt_collect(h);
    for (cudaEvent_t e : h->kt.pool) cudaEventDestroy(e);
    for (void *p : h->allocs) cudaFree(p);
    if (h->h_res) cudaFreeHost(h->h_res);
    if (h->st && !h->borrowed_stream) cudaStreamDestroy(h->st);
    delete h;
    return MPG_OK;
}

// Attaches the coarse (level 1, the reference's mesh3d_c.d) or coarsest (level 2, mesh3d_cc.d)
// mesh of precon's V-cycle (ref.f:618-748) to a handle created with mg_flag = 1.  The level gets a
// handle of its own on the parent's stream (laplc_c / laplc_cc are laplc on that mesh), the match
// map (given, 1-based as in match1.d / match2.d, or found by coordinates as `matching` does), the
// finer mesh's neighbour lists, and the set-up data mpsolver computes for levels 2 and 3
// (ref.f:161-168): beta_timestep_unstr on the level's mesh and compute_d_unstr with the finest rh0
// restricted to it.  laplc_c/_cc read rh0 of the matched finest node and coefw at the node's own
// number (mg_bugs = 1) or at the matched finest node (mg_bugs = 0).
extern "C" int mpg_set_coarse(mpg_handle h, int level, const mpg_mesh_ref *mesh, const int32_t *match) {
    if (!h || !mesh) return mpg_fail(MPG_ERR_ARG, "set_coarse: null argument");
    if (h->P.mg_flag != 1) return mpg_fail(MPG_ERR_ARG, "set_coarse: the handle was not created with mg_flag = 1");
    if (level != 1 && level != 2) return mpg_fail(MPG_ERR_ARG, "set_coarse: level must be 1 or 2");
    if (level == 2 && !h->mg[0].sub) return mpg_fail(MPG_ERR_ARG, "set_coarse: attach level 1 first");
    if (h->mg[level - 1].sub) return mpg_fail(MPG_ERR_ARG, "set_coarse: level already attached");
    mpg_params Ps = h->P;
    Ps.mg_flag = 0;
    mpg_handle c = nullptr;
    int rc = mpg_create(&Ps, mesh, h->dev, &c);
    if (rc) return rc;
    cudaStreamSynchronize(c->st);
    cudaStreamDestroy(c->st);
    c->st = h->st;
    c->borrowed_stream = true;
    auto fail = [&](int code) { mpg_destroy(c); return code; };
    mpg_solver *fine = level == 1 ? h : h->mg[0].sub;     // the next finer mesh
    const std::vector<int32_t> &fptr = fine->nb_ptr_ref, &flst = fine->nb_lst_ref;
    const int nf = fine->N, nc = c->N;
    std::vector<int32_t> m(nc);
    if (match) {
        for (int i = 0; i < nc; ++i) m[i] = match[i] - 1;
    } else {
        std::vector<double> x, y, z;
        mg_coords(mesh, x, y, z);
        m = mg_matching(fine->cx_ref, fine->cy_ref, fine->cz_ref, x, y, z);
    }
    for (int i = 0; i < nc; ++i)
        if (m[i] < 0 || m[i] >= nf)
            return fail(mpg_fail(MPG_ERR_MESH, "set_coarse: coarse node " + std::to_string(i + 1) +
                                                   " has no matching node in the finer mesh"));
    if (level == 1) {            // the coarse level keeps its own lists for the next restriction
        mg_neigh_definition(mesh, c->nb_ptr_ref, c->nb_lst_ref);
        mg_coords(mesh, c->cx_ref, c->cy_ref, c->cz_ref);
    }
    auto &lv = h->mg[level - 1];
    const int bugs = h->P.mg_bugs;
    // finest-mesh rh0 and coefw in reference numbering
    std::vector<int32_t> perm_f(h->N);
    for (int n = 0; n < h->N; ++n) perm_f[h->iperm[n]] = n;
    std::vector<double> rh0r(h->N), cwr(h->N);
    for (int i = 0; i < h->N; ++i) { rh0r[i] = h->hs.rh0[perm_f[i]]; cwr[i] = h->hs.coefw[perm_f[i]]; }
    // the level's node -> finest node; the finest rh0 restricted to the level; its compute_d
    std::vector<int32_t> to_finest(nc);
    for (int i = 0; i < nc; ++i) to_finest[i] = level == 1 ? m[i] : h->mg[0].match_ref[m[i]];
    lv.rh0_restricted = mg_restrict_host(level == 1 ? rh0r : h->mg[0].rh0_restricted, m, fptr, flst, bugs);
    const std::vector<double> dref = mg_compute_d(mesh, lv.rh0_restricted, h->P.delt);
    std::vector<int32_t> perm_c(nc);
    for (int n = 0; n < nc; ++n) perm_c[c->iperm[n]] = n;
    std::vector<double> rh0c(nc), cwc(nc), dc(nc);
    for (int i = 0; i < nc; ++i) {
        rh0c[perm_c[i]] = rh0r[to_finest[i]];
        cwc[perm_c[i]] = bugs ? cwr[i] : cwr[to_finest[i]];
        dc[perm_c[i]] = dref[i];
    }
    MPG_CUDA(cudaMemcpyAsync(c->f[MPG_F_RH0], rh0c.data(), sizeof(double) * nc, cudaMemcpyHostToDevice, h->st));
    MPG_CUDA(cudaMemcpyAsync(c->f[MPG_F_COEFW], cwc.data(), sizeof(double) * nc, cudaMemcpyHostToDevice, h->st));
    MPG_CUDA(cudaMemcpyAsync(c->f[MPG_F_D1], dc.data(), sizeof(double) * nc, cudaMemcpyHostToDevice, h->st));
    // transfer data in internal numbering: match, the finer mesh's lists, the loop-counter nodes
    std::vector<int32_t> perm_fine(nf);
    for (int n = 0; n < nf; ++n) perm_fine[fine->iperm[n]] = n;
    std::vector<int32_t> mi(nc), ptr_i(nf + 1, 0), lst_i(flst.size());
    for (int i = 0; i < nc; ++i) mi[perm_c[i]] = perm_fine[m[i]];
    int maxdeg = 0;
    for (int i = 0; i < nf; ++i) {
        const int deg = fptr[i + 1] - fptr[i];
        ptr_i[perm_fine[i] + 1] = deg;
        maxdeg = std::max(maxdeg, deg);
    }
    for (int n = 0; n < nf; ++n) ptr_i[n + 1] += ptr_i[n];
    for (int i = 0; i < nf; ++i) {
        const int n = perm_fine[i];
        for (int k = 0; k < fptr[i + 1] - fptr[i]; ++k) lst_i[ptr_i[n] + k] = perm_fine[flst[fptr[i] + k]];
    }
    if (maxdeg > nf) return fail(mpg_fail(MPG_ERR_MESH, "set_coarse: finer mesh smaller than a node degree"));
    std::vector<int32_t> bugnb(std::max(maxdeg, 1), 0);
    for (int k = 0; k < maxdeg; ++k) bugnb[k] = perm_fine[k];
    lv.passes = bugs ? 1 : mg_fill_passes(nf, m, fptr, flst);
    if (lv.passes < 0)
        return fail(mpg_fail(MPG_ERR_MESH, "set_coarse: some finer nodes cannot be reached from the coarse ones"));
    lv.match_ref = m;
    if ((rc = upload(h, &lv.match, mi)) || (rc = upload(h, &lv.nbp, ptr_i)) || (rc = upload(h, &lv.nbl, lst_i)) ||
        (rc = upload(h, &lv.bugnb, bugnb)) || (rc = dalloc(h, &lv.aux, nf)) || (rc = dalloc(h, &lv.flag, nf)) ||
        (rc = dalloc(c, &lv.p, nc)) || (rc = dalloc(c, &lv.r, nc)) || (rc = dalloc(c, &lv.e, nc)) ||
        (rc = dalloc(c, &lv.rrhs, nc)) || (rc = dalloc(c, &lv.rrhs_out, nc)))
        return fail(rc);
    MPG_CUDA(cudaStreamSynchronize(h->st));
    lv.sub = c;
    return MPG_OK;
}

extern "C" int mpg_get_info(mpg_handle h, mpg_info *info) {
    if (!h || !info) return mpg_fail(MPG_ERR_ARG, "null argument");
    info->npoin = h->N;
    info->nedge = (int64_t)h->NE2 * h->L + (int64_t)h->NC * (h->L - 1);
    info->ncol = h->NC;
    info->nedge2d = h->NE2;
    info->nlev = h->L;
    info->precision = h->P.precision;
    info->device_bytes = (int64_t)h->dev_bytes;
    return MPG_OK;
}

extern "C" int mpg_set_field(mpg_handle h, int fid, const double *src) {
    if (!h || !src) return mpg_fail(MPG_ERR_ARG, "null argument");
    FLD(dst, fid);
    MPG_CUDA(cudaMemcpyAsync(h->stage, src, sizeof(double) * h->N, cudaMemcpyHostToDevice, h->st));
    k_scatter_perm<<<grid(h->N), kThreads, 0, h->st>>>(h->N, h->d_perm, h->stage, dst);
    int rc = check_launch("set_field");
    if (rc) return rc;
    MPG_CUDA(cudaStreamSynchronize(h->st));
    return MPG_OK;
}

extern "C" int mpg_get_field(mpg_handle h, int fid, double *dst) {
    if (!h || !dst) return mpg_fail(MPG_ERR_ARG, "null argument");
    FLD(src, fid);
    k_gather_perm<<<grid(h->N), kThreads, 0, h->st>>>(h->N, h->d_perm, src, h->stage);
    int rc = check_launch("get_field");
    if (rc) return rc;
    MPG_CUDA(cudaMemcpyAsync(dst, h->stage, sizeof(double) * h->N, cudaMemcpyDeviceToHost, h->st));
    MPG_CUDA(cudaStreamSynchronize(h->st));
    return lap_fused_check(h);
}

extern "C" int mpg_derivative(mpg_handle h, int unk, int out, int idx) {
    if (!h) return mpg_fail(MPG_ERR_ARG, "null handle");
    if (idx < 1 || idx > 3) return mpg_fail(MPG_ERR_ARG, "idx must be 1, 2 or 3");
    FLD(a, unk);
    FLD(b, out);
    if (a == b) return mpg_fail(MPG_ERR_ARG, "derivative: input and output must differ");
    k_derivative<<<grid(h->N), kThreads, 0, h->st>>>(h->M, a, b, idx);
    if (h->CL.n) k_cp_derivative<<<grid(h->CL.n), kThreads, 0, h->st>>>(h->M, h->CL, a, b, idx);
    return check_launch("derivative");
}

extern "C" int mpg_bcv(mpg_handle h, int u, int v, int w, double flag) {
    if (!h) return mpg_fail(MPG_ERR_ARG, "null handle");
    FLD(a, u);
    FLD(b, v);
    FLD(c, w);
    k_bcv<<<grid(h->N), kThreads, 0, h->st>>>(h->M, a, b, c, h->ue, flag);
    return check_launch("bcv");
}

extern "C" int mpg_laplc(mpg_handle h, int press, int alap, int impfl) {
    if (!h) return mpg_fail(MPG_ERR_ARG, "null handle");
    FLD(a, press);
    FLD(b, alap);
    if (a == b) return mpg_fail(MPG_ERR_ARG, "laplc: input and output must differ");
    return op_laplc(h, a, b, impfl);
}

extern "C" int mpg_laplc_adjoint(mpg_handle h, int y, int out, int impfl) {
    if (h && h->CL.n) return mpg_fail(MPG_ERR_UNSUPPORTED, "laplc_adjoint: periodic copy lists are not provided");
    if (!h) return mpg_fail(MPG_ERR_ARG, "null handle");
    FLD(yy, y);
    FLD(oo, out);
    if (yy == oo) return mpg_fail(MPG_ERR_ARG, "laplc_adjoint: y and out must differ");
    return op_laplc_adj(h, yy, oo, impfl, true);
}

extern "C" int mpg_prfr(mpg_handle h, int press, int ustr, int vstr, int wstr, int uout, int vout, int wout,
                        int impfl) {
    if (!h) return mpg_fail(MPG_ERR_ARG, "null handle");
    FLD(p, press);
    FLD(us, ustr);
    FLD(vs, vstr);
    FLD(ws, wstr);
    FLD(uo, uout);
    FLD(vo, vout);
    FLD(wo, wout);
    if (p == uo || p == vo || p == wo) return mpg_fail(MPG_ERR_ARG, "prfr: press must not alias an output");
    return op_prfr(h, p, us, vs, ws, uo, vo, wo, impfl);
}

extern "C" int mpg_div(mpg_handle h, int ua, int va, int wa, int rhs, int iflg, mpg_diag *diag) {
    if (!h) return mpg_fail(MPG_ERR_ARG, "null handle");
    if (iflg != 1 && iflg != -1) return mpg_fail(MPG_ERR_ARG, "iflg must be 1 or -1");
    FLD(a, ua);
    FLD(b, va);
    FLD(c, wa);
    FLD(r, rhs);
    if (r == a || r == b || r == c) return mpg_fail(MPG_ERR_ARG, "div: rhs must not alias an input");
    int rc = op_div(h, a, b, c, r, iflg);
    if (rc) return rc;
    if (iflg == 1 && diag) return diag_div(h, r, diag);
    return MPG_OK;
}

extern "C" int mpg_precon(mpg_handle h, int rhs, int p, int r, int iprc, int impfl) {
    if (!h) return mpg_fail(MPG_ERR_ARG, "null handle");
    FLD(a, rhs);
    FLD(b, p);
    FLD(c, r);
    if (a == b || a == c || b == c) return mpg_fail(MPG_ERR_ARG, "precon: arguments must be distinct fields");
    return op_precon(h, a, b, c, iprc, impfl, true);
}

static void fill_stats(mpg_handle h, mpg_gcr_stats *st) {
    std::memset(st, 0, sizeof(*st));
    st->niter = h->niter; st->nitsm = h->nitsm; st->icount = h->icount; st->status = h->gstatus;
    st->eer = h->eer; st->eem = h->eem; st->dvmx = h->dvmx_last; st->rl2 = h->rl2_last;
    st->fallbacks = h->last_fallbacks;
    st->rate = h->rate_last;
}

extern "C" int mpg_gcrk(mpg_handle h, int p, int u1, int v1, int w1, int u2, int v2, int w2, int impfl,
                        mpg_gcr_stats *stats) {
    if (!h) return mpg_fail(MPG_ERR_ARG, "null handle");
    FLD(pp, p);
    FLD(a1, u1);
    FLD(b1, v1);
    FLD(c1, w1);
    FLD(a2, u2);
    FLD(b2, v2);
    FLD(c2, w2);
    int rc = op_gcrk(h, pp, a1, b1, c1, a2, b2, c2, impfl);
    if (rc) return rc;
    if (stats) fill_stats(h, stats);
    if (h->gstatus == MPG_GCR_NAN) return mpg_fail(MPG_ERR_NUMERIC, "gcrk: NaN/Inf in the residual");
    return MPG_OK;
}

extern "C" int mpg_get_gcr_stats(mpg_handle h, mpg_gcr_stats *stats) {
    if (!h || !stats) return mpg_fail(MPG_ERR_ARG, "null argument");
    fill_stats(h, stats);
    return MPG_OK;
}

static int mpdata_entry(mpg_handle h, int unk, int iflag, int iper) {
    if (!h) return mpg_fail(MPG_ERR_ARG, "null handle");
    if (h->P.iper != iper)
        return mpg_fail(MPG_ERR_ARG, iper == 2 ? "mpdatamper needs iper = 2 (use mpg_mpdatam for iper = 0)"
                                               : "mpdatam needs iper = 0 (use mpg_mpdatamper for iper = 2)");
    if (iflag < 1) return mpg_fail(MPG_ERR_ARG, "iflag must be >= 1");
    FLD(psi, unk);
    for (int q = 0; q < 3; ++q)
        if (!fld(h, MPG_F_UUU + q)) return mpg_fail(MPG_ERR_NOMEM, "uuu");
    int rc = op_aun(h);
    if (rc) return rc;
    return op_mpdata_field(h, psi, iflag);
}

extern "C" int mpg_mpdatamper(mpg_handle h, int unk, int iflag) { return mpdata_entry(h, unk, iflag, 2); }

extern "C" int mpg_mpdatam(mpg_handle h, int unk, int iflag) { return mpdata_entry(h, unk, iflag, 0); }

extern "C" int mpg_courant(mpg_handle h, int iflag, mpg_diag *diag) {
    if (!h) return mpg_fail(MPG_ERR_ARG, "null handle");
    if (iflag < 1 || iflag > 3) return mpg_fail(MPG_ERR_ARG, "iflag must be 1, 2 or 3");
    for (int q = 0; q < 3; ++q)
        if (!fld(h, MPG_F_UUU + q)) return mpg_fail(MPG_ERR_NOMEM, "uuu");
    return diag_courant(h, iflag, diag);
}

extern "C" int mpg_stats(mpg_handle h, mpg_diag *diag) {
    if (!h || !diag) return mpg_fail(MPG_ERR_ARG, "null argument");
    return diag_stats(h, diag);
}

static int step_diag(mpg_handle h, mpg_diag *diag) {
    mpg_diag d;
    std::memset(&d, 0, sizeof d);
    int rc;
    double *rhs = fld(h, MPG_F_RHS);
    if ((rc = op_div(h, h->f[MPG_F_UUU], h->f[MPG_F_UUU + 1], h->f[MPG_F_UUU + 2], rhs, 1))) return rc;
    if (diag) {
        if ((rc = diag_div(h, rhs, &d))) return rc;
        if ((rc = diag_courant(h, 1, &d))) return rc;
        if ((rc = diag_stats(h, &d))) return rc;
        *diag = d;
    } else {
        if ((rc = diag_courant(h, 1, nullptr))) return rc;
    }
    return MPG_OK;
}

extern "C" int mpg_setup(mpg_handle h, mpg_diag *diag) {
    if (!h) return mpg_fail(MPG_ERR_ARG, "null handle");
    Fields F = make_fields(h);
    double *prpot = fld(h, MPG_F_PRPOT), *u4 = fld(h, MPG_F_UNK1 + 3);
    if (!prpot || !u4) return mpg_fail(MPG_ERR_NOMEM, "fields");
    const int N = h->N;
    int rc;
    {
        KTIME(KT_NODE);
        k_setup_ambient<<<grid(N), kThreads, 0, h->st>>>(N, F, prpot, u4);
    }
    if ((rc = check_launch("setup ambient"))) return rc;
    if ((rc = op_gcrk(h, prpot, F.unk1[0], F.unk1[1], F.unk1[2], F.unk[0], F.unk[1], F.unk[2], 0))) return rc;
    if ((rc = op_prfr(h, prpot, F.unk1[0], F.unk1[1], F.unk1[2], F.unk[0], F.unk[1], F.unk[2], 0))) return rc;
    {
        KTIME(KT_NODE);
        k_setup_post<<<grid(N), kThreads, 0, h->st>>>(N, F, prpot, h->P.itraj);
    }
    if ((rc = check_launch("setup post"))) return rc;
    if (h->P.itraj != 0 && (rc = op_velprd(h))) return rc;
    if ((rc = step_diag(h, diag))) return rc;
    MPG_CUDA(cudaStreamSynchronize(h->st));
    if (h->gstatus == MPG_GCR_NAN) return mpg_fail(MPG_ERR_NUMERIC, "setup: NaN in the potential-flow solve");
    return MPG_OK;
}

static const double kF0 = 1.4584e-03, kXlat = 20.;   // mpsolver constants, ref.f:108-109
static double fcr3_of() { return kF0 * std::sin(kXlat) * 0.0; }   // icorio = 0
static double fcr2_of() { return kF0 * std::cos(kXlat) * 0.0; }

extern "C" int mpg_half_forcing(mpg_handle h) {
    if (!h) return mpg_fail(MPG_ERR_ARG, "null handle");
    Fields F = make_fields(h);
    {
        KTIME(KT_NODE);
        k_half_forcing<<<grid(h->N), kThreads, 0, h->st>>>(h->N, F, h->P.delt, h->P.implgw);
    }
    return check_launch("half forcing");
}

extern "C" int mpg_explicit_forcing(mpg_handle h, int mtri) {
    if (!h) return mpg_fail(MPG_ERR_ARG, "null handle");
    Fields F = make_fields(h);
    {
        KTIME(KT_NODE);
        k_explicit_forcing<<<grid(h->N), kThreads, 0, h->st>>>(h->N, F, h->P.delt, h->P.g, fcr2_of(), fcr3_of(), 1.0,
                                                               h->P.implgw, mtri);
    }
    return check_launch("explicit forcing");
}

extern "C" int mpg_post_solve(mpg_handle h, int mtri) {
    if (!h) return mpg_fail(MPG_ERR_ARG, "null handle");
    Fields F = make_fields(h);
    {
        KTIME(KT_NODE);
        k_post_solve<<<grid(h->N), kThreads, 0, h->st>>>(h->N, F, h->P.delt, h->P.g, mtri == 2 ? 1 : 0);
    }
    return check_launch("post solve");
}

extern "C" int mpg_extrapolate(mpg_handle h) {
    if (!h) return mpg_fail(MPG_ERR_ARG, "null handle");
    Fields F = make_fields(h);
    {
        KTIME(KT_NODE);
        k_extrapolate<<<grid(h->N), kThreads, 0, h->st>>>(h->N, F, fcr2_of(), fcr3_of(), 1.0, h->P.itraj);
    }
    int rc = check_launch("extrapolate");
    if (!rc && h->P.itraj != 0) rc = op_velprd(h);
    return rc;
}

extern "C" int mpg_velprd(mpg_handle h) {
    if (!h) return mpg_fail(MPG_ERR_ARG, "null handle");
    return op_velprd(h);
}

// One pass of DO ITIME (ref.f:285-463), driving the entry points above in mpsolver's order.
extern "C" int mpg_step(mpg_handle h, mpg_diag *diag) {
    if (!h) return mpg_fail(MPG_ERR_ARG, "null handle");
    int rc;
    Fields F = make_fields(h);
    if ((rc = mpg_half_forcing(h))) return rc;
    if ((rc = op_aun(h))) return rc;                          // uuu is fixed over the advection calls
    for (int q = 0; q < 4 + h->P.nscal; ++q) {                // mpdatamper or mpdatam, ref.f:308-319
        double *psi = fld(h, MPG_F_UNK + q);
        if (!psi) return mpg_fail(MPG_ERR_NOMEM, "unk");
        if ((rc = op_mpdata_field(h, psi, q + 1))) return rc;
    }
    double *prpot = fld(h, MPG_F_PRPOT);
    int niter1 = 0, fallbacks = 0;
    double rate1 = 0.;
    for (int mtri = 1; mtri <= 2; ++mtri) {
        if ((rc = mpg_explicit_forcing(h, mtri))) return rc;
        const int imp = h->P.implgw;
        {
            KTIME(KT_SOLVE);
            if ((rc = op_gcrk(h, prpot, F.unk1[0], F.unk1[1], F.unk1[2], F.uuu[0], F.uuu[1], F.uuu[2], imp)))
                return rc;
            if (h->gstatus == MPG_GCR_NAN) return mpg_fail(MPG_ERR_NUMERIC, "step: NaN in the pressure solve");
            if ((rc = op_prfr(h, prpot, F.unk1[0], F.unk1[1], F.unk1[2], F.uuu[0], F.uuu[1], F.uuu[2], imp)))
                return rc;
        }
        if (mtri == 1) { niter1 = h->niter; rate1 = h->rate_last; }
        fallbacks += h->last_fallbacks;
        if ((rc = mpg_post_solve(h, mtri))) return rc;
    }
    if ((rc = mpg_extrapolate(h))) return rc;
    if ((rc = step_diag(h, diag))) return rc;
    if (diag) {
        diag->niter1 = niter1;
        diag->rate1 = rate1;
        diag->fallbacks = fallbacks;
    }
    return MPG_OK;
}

extern "C" int mpg_synchronize(mpg_handle h) {
    if (!h) return mpg_fail(MPG_ERR_ARG, "null handle");
    MPG_CUDA(cudaStreamSynchronize(h->st));
    return MPG_OK;
}

extern "C" int mpg_analyze_mesh(const mpg_mesh_ref *mesh, mpg_info *info) {
    if (!mesh || !info) return mpg_fail(MPG_ERR_ARG, "null argument");
    HostColumnMesh hm;
    int rc = mpg_build_column_mesh(mesh, &hm);
    if (rc) return rc;
    info->npoin = hm.N;
    info->nedge = (int64_t)hm.NE2 * hm.L + (int64_t)hm.NC * (hm.L - 1);
    info->ncol = hm.NC;
    info->nedge2d = hm.NE2;
    info->nlev = hm.L;
    info->precision = hm.bitwise_order ? 1 : 0;
    info->device_bytes = 0;
    return MPG_OK;
}

extern "C" int mpg_analyze_wide(const mpg_params *prm, const mpg_mesh_ref *mesh, int impfl, double *a,
                                double *minv, double *cp) {
    if (!prm || !mesh || !a || !minv || !cp) return mpg_fail(MPG_ERR_ARG, "null argument");
    HostColumnMesh hm;
    int rc = mpg_build_column_mesh(mesh, &hm);
    if (rc) return rc;
    mpg_params P = *prm;
    P.iprc = 4;
    HostStatic hs;
    if ((rc = mpg_host_static(&P, mesh, hm, &hs))) return rc;
    const int q = impfl ? 1 : 0;
    for (int n = 0; n < hm.N; ++n) {
        const int64_t li = line_index(n / hm.L, n % hm.L, hm.L);
        const int i = hm.iperm[n];
        a[i] = hs.wa[q][li];
        minv[i] = hs.wm[q][li];
        cp[i] = hs.wcp[q][li];
    }
    return MPG_OK;
}

extern "C" int mpg_get_stream(mpg_handle h, void **stream) {
    if (!h || !stream) return mpg_fail(MPG_ERR_ARG, "null argument");
    *stream = (void *)h->st;
    return MPG_OK;
}

extern "C" int mpg_kernel_timing(mpg_handle h, int enable) {
    if (!h) return mpg_fail(MPG_ERR_ARG, "null handle");
    kt_collect(h);
    for (int c = 0; c < KT_COUNT; ++c) { h->kt.total_ms[c] = 0.; h->kt.launches[c] = 0; }
    h->kt.on = enable != 0;
    return MPG_OK;
}

extern "C" int mpg_kernel_times(mpg_handle h, mpg_ktime *out, int max, int *count) {
    if (!h || !count) return mpg_fail(MPG_ERR_ARG, "null argument");
    kt_collect(h);
    int n = 0;
    for (int c = 0; c < KT_COUNT; ++c) {
        if (!h->kt.launches[c]) continue;
        if (out && n < max) {
            std::memset(out[n].name, 0, sizeof out[n].name);
            std::strncpy(out[n].name, kKNames[c], sizeof out[n].name - 1);
            out[n].launches = h->kt.launches[c];
            out[n].total_ms = h->kt.total_ms[c];
        }
        ++n;
    }
    *count = n;
    return MPG_OK;
}

// ------------------------------------------------------------------------------ allocation-free laplc
// Scratch of mpg_laplc_noalloc: the permuted input, the three scaled gradient components and the
// permuted output, MPG_NOALLOC_MAX_NODES doubles each (5 x 131072 x 8 B = 5 MiB).  It is a
// static device array, so every GPU that loads this library holds it until the process exits,
// whether or not the entry point is ever called.
static __device__ __align__(256) double g_noalloc_scratch[5 * (size_t)MPG_NOALLOC_MAX_NODES];

namespace {
constexpr int kNoallocMaxDevices = 64;
double *g_noalloc_addr[kNoallocMaxDevices] = {};
std::mutex g_noalloc_mutex;
}  // namespace

extern "C" int mpg_laplc_noalloc(mpg_handle h, const double *press, double *alap, int impfl) {
    if (!h || !press || !alap) return mpg_fail(MPG_ERR_ARG, "laplc_noalloc: null argument");
    if (h->N > MPG_NOALLOC_MAX_NODES)
        return mpg_fail(MPG_ERR_ARG, "laplc_noalloc: mesh has " + std::to_string(h->N) +
                                         " nodes, more than the static scratch holds (" +
                                         std::to_string(MPG_NOALLOC_MAX_NODES) + "); use mpg_laplc");
    if (h->dev < 0 || h->dev >= kNoallocMaxDevices)
        return mpg_fail(MPG_ERR_ARG, "laplc_noalloc: device index out of range");
    if (press == alap) return mpg_fail(MPG_ERR_ARG, "laplc_noalloc: input and output must differ");
    if (h->CL.n) return mpg_fail(MPG_ERR_UNSUPPORTED, "laplc_noalloc: periodic copy lists are not provided");
    // the caller's current device is put back on every return
    struct RestoreDevice {
        int prev = -1;
        RestoreDevice() { if (cudaGetDevice(&prev) != cudaSuccess) prev = -1; }
        ~RestoreDevice() { if (prev >= 0) cudaSetDevice(prev); }
    } restore;
    MPG_CUDA(cudaSetDevice(h->dev));
    double *base;
    {
        // first call on this device: the host-side name of the array is not a device address, so
        // ask the runtime for the device address once, with this device current
        std::lock_guard<std::mutex> lock(g_noalloc_mutex);
        if (!g_noalloc_addr[h->dev]) {
            void *ptr = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
            if (e != cudaSuccess || !ptr)
                return mpg_fail(MPG_ERR_CUDA, std::string("laplc_noalloc: cudaGetSymbolAddress: ") +
                                                  cudaGetErrorString(e));
            g_noalloc_addr[h->dev] = (double *)ptr;
        }
        base = g_noalloc_addr[h->dev];
    }
    const size_t cap = MPG_NOALLOC_MAX_NODES;
    double *pin = base, *F0 = base + cap, *F1 = base + 2 * cap, *F2 = base + 3 * cap, *aout = base + 4 * cap;
    // every scratch element read below is written earlier in this call, so nothing needs clearing
    const int N = h->N;
    k_scatter_perm<<<grid(N), kThreads, 0, h->st>>>(N, h->d_perm, press, pin);
    const Flux<double> F{F0, F1, F2};
    k_lap_grad<<<grid(h->N), kThreads, 0, h->st>>>(h->M, pin, h->vol, h->f[MPG_F_RH0], h->f[MPG_F_COEFW], h->ue,
                                                h->P.delt, impfl, F);
    k_lap_div<<<grid(h->N), kThreads, 0, h->st>>>(h->M, F, h->vol, h->f[MPG_F_RH0], aout);
    k_gather_perm<<<grid(N), kThreads, 0, h->st>>>(N, h->d_perm, aout, alap);
    return check_launch("laplc_noalloc");
}

// ------------------------------------------------------------------------------ restart files
#include <fstream>

namespace {

// Fortran's F14.6 edit: right-justified in 14 characters with 6 decimals; a value that does not
// fit (or is not finite) prints as 14 asterisks
void put_f14_6(std::string &out, double v) {
    char b[64];
    const int n = std::snprintf(b, sizeof b, "%14.6f", v);
    if (n != 14 || !std::isfinite(v)) out.append(14, '*');
    else out.append(b, 14);
}
bool get_f14_6(const std::string &line, int i, double &v) {
    if (line.size() < (size_t)(14 * (i + 1))) return false;
    const std::string f = line.substr((size_t)14 * i, 14);
    if (f.find('*') != std::string::npos) return false;
    char *end = nullptr;
    v = std::strtod(f.c_str(), &end);
    return end != f.c_str();
}

// the blocks of Restart_Out_old (ref.f:4797-4816): field ids per column, -1 = uuu1 (zero)
const int kRestartText[6][4] = {
    {MPG_F_UUU, MPG_F_UUU + 1, MPG_F_UUU + 2, -2},
    {-1, -1, -1, -2},
    {MPG_F_UNKDASH, MPG_F_UNKDASH + 1, MPG_F_UNKDASH + 2, -2},
    {MPG_F_UNK, MPG_F_UNK + 1, MPG_F_UNK + 2, MPG_F_UNK + 3},
    {MPG_F_FRC, MPG_F_FRC + 1, MPG_F_FRC + 2, MPG_F_FRC + 3},
    {MPG_F_PRPOT, MPG_F_RHS, MPG_F_COUR, MPG_F_COEFW}};

struct RestartHeader {
    char magic[8];
    int32_t npoin, nscal, nitsm, icount, ntime, nfields;
};

std::vector<int> restart_binary_fields(mpg_handle h) {
    std::vector<int> f;
    for (int q = 0; q < 4 + h->P.nscal; ++q) f.push_back(MPG_F_UNK + q);
    for (int q = 0; q < 4; ++q) f.push_back(MPG_F_UNK1 + q);
    for (int q = 0; q < 3; ++q) { f.push_back(MPG_F_UUU + q); f.push_back(MPG_F_UUU0 + q); f.push_back(MPG_F_UNKDASH + q); }
    for (int q = 0; q < 4; ++q) f.push_back(MPG_F_FRC + q);
    f.push_back(MPG_F_PRPOT);
    f.push_back(MPG_F_RHS);
    f.push_back(MPG_F_COUR);
    return f;
}

// Fortran's Ew.d edit with d = 4, w = 12: 0.dddd mantissa, E and a signed 2-digit exponent
// ("0.dddd+eee" when the exponent needs three digits), right-justified; 12 asterisks when the
// value is not finite
void put_e12_4(std::string &out, double v) {
    char m[32], b[32];
    if (!std::isfinite(v)) { out.append(12, '*'); return; }
    if (v == 0.) { std::snprintf(b, sizeof b, "%12s", "0.0000E+00"); out.append(b, 12); return; }
    std::snprintf(m, sizeof m, "%.3E", std::fabs(v));             // d.dddE+xx, 4 significant digits
    const int e = std::atoi(m + 6) + 1;                           // exponent of the 0.dddd form
    char digits[5] = {m[0], m[2], m[3], m[4], 0};
    char ex[8];
    if (e >= -99 && e <= 99) std::snprintf(ex, sizeof ex, "E%c%02d", e < 0 ? '-' : '+', e < 0 ? -e : e);
    else std::snprintf(ex, sizeof ex, "%c%03d", e < 0 ? '-' : '+', e < 0 ? -e : e);
    std::snprintf(b, sizeof b, "%s0.%s%s", v < 0 ? "-" : "", digits, ex);
    char r[32];
    std::snprintf(r, sizeof r, "%12s", b);
    out.append(r, 12);
}

}  // namespace

extern "C" int mpg_write_output(mpg_handle h, const char *path, const double *coord, int npoinx) {
    if (!h || !path || !coord) return mpg_fail(MPG_ERR_ARG, "null argument");
    if (npoinx < h->N) return mpg_fail(MPG_ERR_ARG, "npoinx smaller than npoin");
    const size_t N = (size_t)h->N;
    std::vector<std::vector<double>> u(4, std::vector<double>(N));
    int rc;
    for (int q = 0; q < 4; ++q)
        if ((rc = mpg_get_field(h, MPG_F_UNK + q, u[q].data()))) return rc;
    std::FILE *fp = std::fopen(path, "w");
    if (!fp) return mpg_fail(MPG_ERR_ARG, std::string("output: cannot open ") + path);
    bool ok = std::fprintf(fp, "   1.0000000000000000     \n %11d\npoint X Y Z u v w temp Velocity\n", h->N) > 0;
    std::string line;
    for (size_t ip = 0; ip < N && ok; ++ip) {                     // ref.f:2793-2803, format 100
        char head[16];
        std::snprintf(head, sizeof head, " %7d", (int)(ip + 1));
        line.assign(head);
        for (int i = 0; i < 3; ++i) put_e12_4(line, coord[(size_t)i * npoinx + ip] / 1.e+03);
        const double a = u[0][ip], b = u[1][ip], w = u[2][ip];
        put_e12_4(line, a);
        put_e12_4(line, b);
        put_e12_4(line, w);
        put_e12_4(line, u[3][ip]);
        put_e12_4(line, std::sqrt(a * a + b * b + w * w));
        line.push_back('\n');
        ok = std::fwrite(line.data(), 1, line.size(), fp) == line.size();
    }
    ok = (std::fclose(fp) == 0) && ok;
    return ok ? MPG_OK : mpg_fail(MPG_ERR_ARG, std::string("output: write failed on ") + path);
}

extern "C" int mpg_restart_write(mpg_handle h, const char *path, int format, int ntime) {
    if (!h || !path) return mpg_fail(MPG_ERR_ARG, "null argument");
    const size_t N = (size_t)h->N;
    int rc;
    if (format == MPG_RESTART_BINARY) {
        std::FILE *fp = std::fopen(path, "wb");
        if (!fp) return mpg_fail(MPG_ERR_ARG, std::string("restart: cannot open ") + path);
        const std::vector<int> fids = restart_binary_fields(h);
        RestartHeader hd{};
        std::memcpy(hd.magic, "MPGRST01", 8);
        hd.npoin = h->N; hd.nscal = h->P.nscal; hd.nitsm = h->nitsm; hd.icount = h->icount; hd.ntime = ntime;
        hd.nfields = (int32_t)fids.size();
        bool ok = std::fwrite(&hd, sizeof hd, 1, fp) == 1;
        std::vector<double> v(N);
        for (int fid : fids) {
            if ((rc = mpg_get_field(h, fid, v.data()))) { std::fclose(fp); return rc; }
            const int32_t id = fid;
            ok = ok && std::fwrite(&id, sizeof id, 1, fp) == 1 && std::fwrite(v.data(), sizeof(double), N, fp) == N;
        }
        ok = (std::fclose(fp) == 0) && ok;
        return ok ? MPG_OK : mpg_fail(MPG_ERR_ARG, std::string("restart: write failed on ") + path);
    }
    if (format != MPG_RESTART_TEXT) return mpg_fail(MPG_ERR_ARG, "restart: unknown format");
    std::vector<std::vector<double>> col(4, std::vector<double>(N));
    std::FILE *fp = std::fopen(path, "w");
    if (!fp) return mpg_fail(MPG_ERR_ARG, std::string("restart: cannot open ") + path);
    bool ok = true;
    std::string line;
    for (int b = 0; b < 6 && ok; ++b) {
        const int ncol = kRestartText[b][3] == -2 ? 3 : 4;
        for (int j = 0; j < ncol; ++j) {
            const int fid = kRestartText[b][j];
            if (fid < 0) std::fill(col[j].begin(), col[j].end(), 0.);
            else if ((rc = mpg_get_field(h, fid, col[j].data()))) { std::fclose(fp); return rc; }
        }
        for (size_t ip = 0; ip < N && ok; ++ip) {        // ref.f:4797-4816, formats 198/199
            line.clear();
            for (int j = 0; j < ncol; ++j) put_f14_6(line, col[j][ip]);
            line.push_back('\n');
            ok = std::fwrite(line.data(), 1, line.size(), fp) == line.size();
        }
    }
    ok = ok && std::fprintf(fp, " %11d %11d\n", h->nitsm, h->icount) > 0;   // write(nfid,*) n1, n2
    ok = ok && std::fprintf(fp, " %11d\n", ntime) > 0;                        // write(nfid,*) ntime8+ntimet
    ok = (std::fclose(fp) == 0) && ok;
    return ok ? MPG_OK : mpg_fail(MPG_ERR_ARG, std::string("restart: write failed on ") + path);
}

extern "C" int mpg_restart_read(mpg_handle h, const char *path, int format, int *ntime) {
    if (!h || !path) return mpg_fail(MPG_ERR_ARG, "null argument");
    const size_t N = (size_t)h->N;
    int rc;
    if (format == MPG_RESTART_BINARY) {
        std::FILE *fp = std::fopen(path, "rb");
        if (!fp) return mpg_fail(MPG_ERR_ARG, std::string("restart: cannot open ") + path);
        RestartHeader hd{};
        if (std::fread(&hd, sizeof hd, 1, fp) != 1 || std::memcmp(hd.magic, "MPGRST01", 8) != 0) {
            std::fclose(fp);
            return mpg_fail(MPG_ERR_ARG, std::string("restart: not a binary restart file: ") + path);
        }
        if (hd.npoin != h->N || hd.nscal != h->P.nscal) {
            std::fclose(fp);
            return mpg_fail(MPG_ERR_ARG, "restart: file written for another mesh or scalar count");
        }
        std::vector<double> v(N);
        for (int i = 0; i < hd.nfields; ++i) {
            int32_t fid = -1;
            if (std::fread(&fid, sizeof fid, 1, fp) != 1 || std::fread(v.data(), sizeof(double), N, fp) != N) {
                std::fclose(fp);
                return mpg_fail(MPG_ERR_ARG, std::string("restart: truncated file ") + path);
            }
            if ((rc = mpg_set_field(h, fid, v.data()))) { std::fclose(fp); return rc; }
        }
        std::fclose(fp);
        h->nitsm = hd.nitsm;
        h->icount = hd.icount;
        if (ntime) *ntime = hd.ntime;
        return MPG_OK;
    }
    if (format != MPG_RESTART_TEXT) return mpg_fail(MPG_ERR_ARG, "restart: unknown format");
    std::ifstream in(path);
    if (!in) return mpg_fail(MPG_ERR_ARG, std::string("restart: cannot open ") + path);
    std::vector<std::vector<double>> col(4, std::vector<double>(N));
    std::string line;
    for (int b = 0; b < 6; ++b) {                        // ref.f:4855-4873
        const int ncol = kRestartText[b][3] == -2 ? 3 : 4;
        for (size_t ip = 0; ip < N; ++ip) {
            bool ok = (bool)std::getline(in, line);
            for (int j = 0; j < ncol && ok; ++j) ok = get_f14_6(line, j, col[j][ip]);
            if (!ok)
                return mpg_fail(MPG_ERR_ARG, "restart: unreadable line " + std::to_string((size_t)b * N + ip + 1) +
                                             " of " + path);
        }
        for (int j = 0; j < ncol; ++j)
            if (kRestartText[b][j] >= 0 && (rc = mpg_set_field(h, kRestartText[b][j], col[j].data()))) return rc;
    }
    int n1 = 0, n2 = 0, nt = 0;
    if (!std::getline(in, line) || std::sscanf(line.c_str(), "%d %d", &n1, &n2) != 2)   // read(nfid,*) n1, n2
        return mpg_fail(MPG_ERR_ARG, std::string("restart: missing nitsm/icount in ") + path);
    h->nitsm = n1;
    h->icount = n2;
    if (ntime) *ntime = (std::getline(in, line) && std::sscanf(line.c_str(), "%d", &nt) == 1) ? nt : 0;
    return MPG_OK;
}

// ------------------------------------------------------------------------------ learned preconditioner API
#include <random>

extern "C" int mpg_learned_init(mpg_handle h, int seed) {
    if (!h) return mpg_fail(MPG_ERR_ARG, "null handle");
    int rc = nn_alloc_infer(h);
    if (rc) return rc;
    std::mt19937_64 rng((uint64_t)seed * 0x9E3779B97F4A7C15ull + 12345u);
    std::vector<float> prm(nn::NPARAM, 0.f);
    std::normal_distribution<float> gin(0.f, std::sqrt(2.f / nn::FIN)), gl(0.f, std::sqrt(2.f / nn::K3));
    for (int i = 0; i < nn::C * nn::FIN; ++i) prm[nn::OFF_WIN + i] = gin(rng);
    for (int i = 0; i < nn::C; ++i) prm[nn::OFF_BIN + i] = 0.01f;
    for (int l = 0; l < nn::NL; ++l) {
        for (int i = 0; i < nn::C * nn::K3; ++i) prm[nn::OFF_L0 + l * nn::LSTRIDE + i] = gl(rng);
        for (int i = 0; i < nn::C; ++i) prm[nn::OFF_L0 + l * nn::LSTRIDE + nn::C * nn::K3 + i] = 0.01f;
    }
    // output layer zero: the untrained network returns the plain preconditioner exactly
    return mpg_learned_set_params(h, prm.data(), nn::NPARAM);
}

extern "C" int mpg_learned_set_params(mpg_handle h, const float *params, int n) {
    if (!h || !params) return mpg_fail(MPG_ERR_ARG, "null argument");
    if (n != nn::NPARAM) return mpg_fail(MPG_ERR_ARG, "expected MPG_LEARNED_NPARAM parameters");
    int rc = nn_alloc_infer(h);
    if (rc) return rc;
    MPG_CUDA(cudaMemcpyAsync(h->nn.prm, params, sizeof(float) * nn::NPARAM, cudaMemcpyHostToDevice, h->st));
    nn::k_nn_to_bf16<<<(nn::NL * nn::C * nn::K3 + 255) / 256, 256, 0, h->st>>>(h->nn.prm, h->nn.Wbf);
    if (h->nn.train) {
        MPG_CUDA(cudaMemsetAsync(h->nn.m1, 0, sizeof(float) * nn::NPARAM, h->st));
        MPG_CUDA(cudaMemsetAsync(h->nn.m2, 0, sizeof(float) * nn::NPARAM, h->st));
    }
    h->nn.adam_t = 0;
    h->nn.have_params = true;
    MPG_CUDA(cudaStreamSynchronize(h->st));
    return check_launch("set params");
}

extern "C" int mpg_learned_get_params(mpg_handle h, float *params, int n) {
    if (!h || !params) return mpg_fail(MPG_ERR_ARG, "null argument");
    if (n != nn::NPARAM) return mpg_fail(MPG_ERR_ARG, "expected MPG_LEARNED_NPARAM parameters");
    if (!h->nn.have_params) return mpg_fail(MPG_ERR_ARG, "no network parameters yet");
    MPG_CUDA(cudaMemcpyAsync(params, h->nn.prm, sizeof(float) * nn::NPARAM, cudaMemcpyDeviceToHost, h->st));
    MPG_CUDA(cudaStreamSynchronize(h->st));
    return MPG_OK;
}

extern "C" int mpg_learned_forward(mpg_handle h, int r, int q) {
    if (!h) return mpg_fail(MPG_ERR_ARG, "null handle");
    if (!h->nn.have_params) return mpg_fail(MPG_ERR_ARG, "no network parameters yet");
    FLD(rr, r);
    FLD(qq, q);
    if (rr == qq) return mpg_fail(MPG_ERR_ARG, "learned_forward: r and q must differ");
    return nn_forward<double>(h, rr, qq, 1, false);
}

extern "C" int mpg_learned_grad(mpg_handle h, int r, int t, float *grad, double *loss) {
    if (!h) return mpg_fail(MPG_ERR_ARG, "null handle");
    if (!h->nn.have_params) return mpg_fail(MPG_ERR_ARG, "no network parameters yet");
    FLD(rr, r);
    FLD(tt, t);
    int rc = nn_alloc_train(h);
    if (rc) return rc;
    if ((rc = nn_grad(h, rr, tt, loss))) return rc;
    if (grad) {
        MPG_CUDA(cudaMemcpyAsync(grad, h->nn.grad, sizeof(float) * nn::NPARAM, cudaMemcpyDeviceToHost, h->st));
        MPG_CUDA(cudaStreamSynchronize(h->st));
    }
    return MPG_OK;
}

extern "C" int mpg_selftest_wait(mpg_handle h, int arrive, int spins, int *completed) {
    if (!h || !completed) return mpg_fail(MPG_ERR_ARG, "null argument");
    if (spins < 1 || spins > (1 << 22)) return mpg_fail(MPG_ERR_ARG, "spins must be in 1..4194304");
    int rc;
    if (!h->nn.selftest && (rc = dalloc(h, &h->nn.selftest, 1))) return rc;
    nn::k_mbar_selftest<<<1, 128, 0, h->st>>>(arrive ? 1 : 0, (long long)spins, h->nn.selftest);
    if ((rc = check_launch("selftest wait"))) return rc;
    MPG_CUDA(cudaMemcpyAsync(completed, h->nn.selftest, sizeof(int), cudaMemcpyDeviceToHost, h->st));
    MPG_CUDA(cudaStreamSynchronize(h->st));
    return MPG_OK;
}

extern "C" int mpg_learned_loss(mpg_handle h, int mode) {
    if (!h) return mpg_fail(MPG_ERR_ARG, "null handle");
    if (mode != MPG_NN_LOSS_RESIDUAL && mode != MPG_NN_LOSS_ERROR) return mpg_fail(MPG_ERR_ARG, "unknown loss mode");
    h->nn.loss_mode = mode;
    return MPG_OK;
}

extern "C" int mpg_learned_train_pair(mpg_handle h, int r, int t, float lr, double *loss) {
    int rc = mpg_learned_grad(h, r, t, nullptr, loss);
    if (rc) return rc;
    return nn_adam(h, lr);
}

extern "C" int mpg_learned_harvest(mpg_handle h, int every, int max_records) {
    if (!h) return mpg_fail(MPG_ERR_ARG, "null handle");
    if (every < 0 || max_records < 0) return mpg_fail(MPG_ERR_ARG, "every and max_records must be >= 0");
    auto &S = h->nn;
    if (every > 0 && max_records > S.maxrec) {
        if (S.rec_r) return mpg_fail(MPG_ERR_ARG, "harvest capacity can only be set once per handle");
        int rc;
        if ((rc = dalloc(h, &S.rec_r, (size_t)max_records * h->N, false)) ||
            (rc = dalloc(h, &S.rec_t, (size_t)max_records * h->N, false)))
            return rc;
        S.maxrec = max_records;
    }
    S.every = every;
    return MPG_OK;
}

extern "C" int mpg_learned_train_records(mpg_handle h, int epochs, float lr, double *mean_loss, int *npairs) {
    if (!h) return mpg_fail(MPG_ERR_ARG, "null handle");
    if (!h->nn.have_params) return mpg_fail(MPG_ERR_ARG, "no network parameters yet");
    auto &S = h->nn;
    int rc = nn_alloc_train(h);
    if (rc) return rc;
    double sum = 0.;
    for (int ep = 0; ep < epochs; ++ep) {
        sum = 0.;
        for (int j = 0; j < S.nrec; ++j) {
            double l = 0.;
            const double *rj = S.rec_r + (size_t)j * h->N, *tj = S.rec_t + (size_t)j * h->N;
            if ((rc = nn_grad(h, rj, tj, &l))) return rc;
            if ((rc = nn_adam(h, lr))) return rc;
            sum += l;
        }
    }
    if (mean_loss) *mean_loss = S.nrec ? sum / S.nrec : 0.;
    if (npairs) *npairs = S.nrec;
    S.nrec = 0;
    MPG_CUDA(cudaStreamSynchronize(h->st));
    return MPG_OK;
}

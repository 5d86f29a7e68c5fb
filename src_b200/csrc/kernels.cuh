// Device kernels of the B200 MPDATA + GCR library.
//
// All per-node sums are node-centric gathers over the column layout (see mpgcr_internal.h):
// thread n = c*L + k walks its column's adjacency list, which is sorted in the reference's
// edge order, so each node accumulates exactly the terms the reference's scatter loops add to
// it, in the same order, with no atomics.  Compiled with -fmad=false: every a*b+c rounds twice
// as in the reference's (unfused) Fortran, which keeps the FP64 path bit-identical to the
// CPU restatement wherever the order of a sum is the reference's own.
//
// Reductions are deterministic: fixed grid, per-thread strided partial sums, a fixed shuffle
// tree per warp, a fixed tree over the warps, and a last-block pass over the block partials.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "mpgcr_internal.h"

namespace mpgk {

constexpr int kThreads = 256;
constexpr int kRedBlocks = 592;          // 4 x 148 SMs
constexpr int kRedThreads = 256;
constexpr int kMaxQ = 24;                // quantities per reduction

__device__ __forceinline__ double amax(double a, double b) { return a > b ? a : b; }
__device__ __forceinline__ double amin(double a, double b) { return a < b ? a : b; }

__device__ __forceinline__ void col_lev(const ColMesh &M, int n, int &c, int &k) {
    c = n / M.L;
    k = n - c * M.L;
}

// ------------------------------------------------------------------------------ gathers
// Visits the faces of node n = (c,k) in reference edge order.  For each face the visitor gets
// the neighbour node j, the face-vector index (into Sh or Sv) and whether the face is stored
// with this node as its second end (then the reference subtracts).
template <class V>
__device__ __forceinline__ void for_faces(const ColMesh &M, int c, int k, int n, V &&visit) {
    const int beg = __ldg(&M.cptr[c]), end = __ldg(&M.cptr[c + 1]);
    const int L = M.L;
    for (int j = beg; j < end; ++j) {
        const int2 en = __ldg(&M.cadj[j]);
        if (en.x >= 0) {
            visit(en.y * L + k, (en.x >> 1) * L + k, (en.x & 1) != 0, false);
        } else if (en.x == MPG_ADJ_BELOW) {
            if (k > 0) visit(n - 1, n - 1, true, true);
        } else {
            if (k + 1 < L) visit(n + 1, n, false, true);
        }
    }
}

__device__ __forceinline__ double sh(const ColMesh &M, int d, int idx, bool vert) {
    return vert ? __ldg(&M.Sv[d][idx]) : __ldg(&M.Sh[d][idx]);
}

// Boundary entries of node (c,k), in reference order.
template <class V>
__device__ __forceinline__ void for_boundary(const ColMesh &M, int c, int k, V &&visit) {
    const int beg = __ldg(&M.bptr[c]), end = __ldg(&M.bptr[c + 1]);
    for (int b = beg; b < end; ++b) {
        const BEntry &be = M.bent[b];
        if (be.k == k) visit(be);
    }
}

// derivative (ref.f:3943-4022) of phi for the three components at once:
// g_d = sum over faces of (+/-) S_d * ((phi_n + phi_j) * 0.5)
__device__ __forceinline__ void grad3(const ColMesh &M, const double *__restrict__ phi, int c, int k,
                                      int n, double &gx, double &gy, double &gz) {
    const double pn = phi[n];
    double ax = 0., ay = 0., az = 0.;
    for_faces(M, c, k, n, [&](int j, int si, bool sub, bool vert) {
        const double u = (pn + phi[j]) * 0.5;
        const double tx = sh(M, 0, si, vert) * u;
        const double ty = sh(M, 1, si, vert) * u;
        const double tz = sh(M, 2, si, vert) * u;
        if (sub) { ax = ax - tx; ay = ay - ty; az = az - tz; }
        else     { ax = ax + tx; ay = ay + ty; az = az + tz; }
    });
    if (M.iper == 0) {                                  // closure, ref.f:4007-4014
        for_boundary(M, c, k, [&](const BEntry &be) {
            ax = ax + be.sbb[0] * pn;
            ay = ay + be.sbb[1] * pn;
            az = az + be.sbb[2] * pn;
        });
    }
    gx = ax; gy = ay; gz = az;
}

// three derivatives of three different fields, component d of field d (the divergence):
// returns derivative(fx,1), derivative(fy,2), derivative(fz,3)
template <class FX>
__device__ __forceinline__ void div3(const ColMesh &M, FX f, int c, int k, int n,
                                     double &dx, double &dy, double &dz) {
    double fnx, fny, fnz;
    f(n, fnx, fny, fnz);
    double ax = 0., ay = 0., az = 0.;
    for_faces(M, c, k, n, [&](int j, int si, bool sub, bool vert) {
        double fjx, fjy, fjz;
        f(j, fjx, fjy, fjz);
        const double tx = sh(M, 0, si, vert) * ((fnx + fjx) * 0.5);
        const double ty = sh(M, 1, si, vert) * ((fny + fjy) * 0.5);
        const double tz = sh(M, 2, si, vert) * ((fnz + fjz) * 0.5);
        if (sub) { ax = ax - tx; ay = ay - ty; az = az - tz; }
        else     { ax = ax + tx; ay = ay + ty; az = az + tz; }
    });
    if (M.iper == 0) {
        for_boundary(M, c, k, [&](const BEntry &be) {
            ax = ax + be.sbb[0] * fnx;
            ay = ay + be.sbb[1] * fny;
            az = az + be.sbb[2] * fnz;
        });
    }
    dx = ax; dy = ay; dz = az;
}

// bcv (ref.f:1583-1643) applied to one node
__device__ __forceinline__ void bcv_node(const ColMesh &M, int c, int k, int n, const double *ue, double flag,
                                         double &u, double &v, double &w) {
    const bool per = (M.iper == 2);
    for_boundary(M, c, k, [&](const BEntry &be) {
        const int t = be.type;
        if (t == 11 || (!per && (t == 5 || t == 6))) {
            const double vn = u * be.anp[0] + v * be.anp[1] + w * be.anp[2];
            u = u - be.anp[0] * vn;
            v = v - be.anp[1] * vn;
            w = w - be.anp[2] * vn;
        }
        if (!per && (t == 7 || t == 8)) u = ue[n] * flag;
    });
}

// ------------------------------------------------------------------------------ operators
// derivative(unk, out, idx)
__global__ void k_derivative(ColMesh M, const double *__restrict__ phi, double *__restrict__ out, int idx) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= M.N) return;
    int c, k;
    col_lev(M, n, c, k);
    double gx, gy, gz;
    grad3(M, phi, c, k, n, gx, gy, gz);
    out[n] = idx == 1 ? gx : idx == 2 ? gy : gz;
}

// bcv(u, v, w, flag) on whole fields
__global__ void k_bcv(ColMesh M, double *u, double *v, double *w, const double *__restrict__ ue, double flag) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= M.N) return;
    int c, k;
    col_lev(M, n, c, k);
    if (__ldg(&M.bptr[c]) == __ldg(&M.bptr[c + 1])) return;
    double a = u[n], b = v[n], d = w[n];
    bcv_node(M, c, k, n, ue, flag, a, b, d);
    u[n] = a; v[n] = b; w[n] = d;
}

// laplc first half (ref.f:1303-1338): gradient, scaling, bcv(.,0.), times rh0
__global__ void k_lap_grad(ColMesh M, const double *__restrict__ p, const double *__restrict__ vol,
                           const double *__restrict__ rh0, const double *__restrict__ coefw,
                           const double *__restrict__ ue, double dt, int impfl,
                           double *__restrict__ Fx, double *__restrict__ Fy, double *__restrict__ Fz) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= M.N) return;
    int c, k;
    col_lev(M, n, c, k);
    double gx, gy, gz;
    grad3(M, p, c, k, n, gx, gy, gz);
    const double v = vol[n];
    double dx = dt * gx / v, dy = dt * gy / v, dz = dt * gz / v;
    dx = 0.5 * dx / 1.0;                       // (gmm*cosa)**2 == 1 for isfera = 0
    dy = 0.5 * dy / 1.0;
    dz = 0.5 * dz * (coefw[n] * (double)impfl + (double)(1 - impfl));
    bcv_node(M, c, k, n, ue, 0.0, dx, dy, dz);
    const double r = rh0[n];
    Fx[n] = dx * r; Fy[n] = dy * r; Fz[n] = dz * r;
}

// laplc second half (ref.f:1339-1350): alap = (Dx(Fx) + Dy(Fy) + Dz(Fz)) / (vol*rh0)
__global__ void k_lap_div(ColMesh M, const double *__restrict__ Fx, const double *__restrict__ Fy,
                          const double *__restrict__ Fz, const double *__restrict__ vol,
                          const double *__restrict__ rh0, double *__restrict__ alap) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= M.N) return;
    int c, k;
    col_lev(M, n, c, k);
    double dx, dy, dz;
    div3(M, [&](int j, double &a, double &b, double &d) { a = Fx[j]; b = Fy[j]; d = Fz[j]; }, c, k, n, dx, dy, dz);
    alap[n] = (dx + dy + dz) / (vol[n] * rh0[n]);
}

// prfr (ref.f:1536-1580)
__global__ void k_prfr(ColMesh M, const double *__restrict__ p, const double *__restrict__ us,
                       const double *__restrict__ vs, const double *__restrict__ ws,
                       const double *__restrict__ vol, const double *__restrict__ coefw,
                       const double *__restrict__ ue, double dt, int impfl,
                       double *__restrict__ uo, double *__restrict__ vo, double *__restrict__ wo) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= M.N) return;
    int c, k;
    col_lev(M, n, c, k);
    double gx, gy, gz;
    grad3(M, p, c, k, n, gx, gy, gz);
    const double v = vol[n];
    const double dpx = gx / 1.0 / v, dpy = gy / 1.0 / v, dpz = gz / v;
    double a = us[n] - 0.5 * dt * dpx;
    double b = vs[n] - 0.5 * dt * dpy;
    double d = ws[n] - 0.5 * dt * dpz * (coefw[n] * (double)impfl + (double)(1 - impfl));
    bcv_node(M, c, k, n, ue, 1.0, a, b, d);
    uo[n] = a; vo[n] = b; wo[n] = d;
}

// div(ua, va, wa, rhs, iflg) (ref.f:2096-2147)
__global__ void k_div(ColMesh M, const double *__restrict__ ua, const double *__restrict__ va,
                      const double *__restrict__ wa, const double *__restrict__ vol,
                      const double *__restrict__ rh0, int iflg, double *__restrict__ rhs) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= M.N) return;
    int c, k;
    col_lev(M, n, c, k);
    double dx, dy, dz;
    if (iflg == -1)
        div3(M, [&](int j, double &a, double &b, double &d) {
            const double r = rh0[j]; a = ua[j] * r; b = va[j] * r; d = wa[j] * r; }, c, k, n, dx, dy, dz);
    else
        div3(M, [&](int j, double &a, double &b, double &d) { a = ua[j]; b = va[j]; d = wa[j]; }, c, k, n, dx, dy, dz);
    const double v = vol[n];
    rhs[n] = (double)iflg * (dx / v + dy / v + dz / v) / rh0[n];
}

// ------------------------------------------------------------------------------ line solve
// z = M^{-1} rhs per column (Thomas, FP64, bottom to top), p = (acc ? p : 0) + omega * z.
// Each warp solves 32 consecutive columns; their right-hand sides (contiguous in the column
// layout) are staged through shared memory with coalesced loads and stores, and the
// coefficients are stored interleaved so that the 32 lanes read level k of their columns
// from one 256-byte segment.
constexpr int kLineWarps = 4;
__global__ void __launch_bounds__(32 * kLineWarps)
k_line_solve(int NC, int L, const double *__restrict__ rhs, const double *__restrict__ la,
             const double *__restrict__ lm, const double *__restrict__ lcp, double omega, int acc,
             double *__restrict__ p) {
    extern __shared__ double sm[];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int col0 = (blockIdx.x * kLineWarps + w) * 32;
    if (col0 >= NC) return;
    const int ncols = min(32, NC - col0);
    double *s = sm + (size_t)w * 32 * L;
    const int64_t base = (int64_t)col0 * L;
    const int cnt = ncols * L;
    for (int i = lane; i < cnt; i += 32) s[i] = rhs[base + i];
    __syncwarp();
    if (lane < ncols) {
        const int c = col0 + lane;
        double *sc = s + lane * L;
        double d = 0.;
        for (int k = 0; k < L; ++k) {
            const int64_t li = line_index(c, k, L);
            const double m = lm[li];
            d = (k == 0) ? sc[0] / m : (sc[k] - la[li] * d) / m;
            sc[k] = d;
        }
        double z = 0.;
        for (int k = L - 1; k >= 0; --k) {
            const int64_t li = line_index(c, k, L);
            z = (k == L - 1) ? sc[k] : sc[k] - lcp[li] * z;
            sc[k] = z;
        }
    }
    __syncwarp();
    for (int i = lane; i < cnt; i += 32) {
        const double prev = acc ? p[base + i] : 0.0;
        p[base + i] = prev + omega * s[i];
    }
}

// ------------------------------------------------------------------------------ reductions
enum RedKind { RSUM = 0, RMAX = 1 };

// Deterministic reduction of NQ quantities produced per node by `prod(n, vals)`.  `kinds` is a
// bitmask: bit q set -> quantity q is a max, else a sum.  The last block to finish reduces the
// block partials in fixed order and calls fin(results) with one thread.
template <int NQ, class Prod, class Fin>
__global__ void __launch_bounds__(kRedThreads)
k_reduce(int N, unsigned kinds, Prod prod, Fin fin, double *__restrict__ part,
         unsigned int *__restrict__ counter, double *__restrict__ result) {
    double acc[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) acc[q] = ((kinds >> q) & 1u) ? -INFINITY : 0.0;
    const int stride = gridDim.x * blockDim.x;
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < N; n += stride) {
        double v[NQ];
        prod(n, v);
#pragma unroll
        for (int q = 0; q < NQ; ++q)
            acc[q] = ((kinds >> q) & 1u) ? amax(acc[q], v[q]) : acc[q] + v[q];
    }
    __shared__ double sred[NQ][kRedThreads / 32];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
        double a = acc[q];
        const bool mx = (kinds >> q) & 1u;
        for (int off = 16; off > 0; off >>= 1) {
            const double o = __shfl_down_sync(0xffffffffu, a, off);
            a = mx ? amax(a, o) : a + o;
        }
        if (lane == 0) sred[q][wid] = a;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int q = 0; q < NQ; ++q) {
            const bool mx = (kinds >> q) & 1u;
            double a = sred[q][0];
            for (int w = 1; w < kRedThreads / 32; ++w) a = mx ? amax(a, sred[q][w]) : a + sred[q][w];
            part[q * gridDim.x + blockIdx.x] = a;
        }
        __threadfence();
        const unsigned int t = atomicAdd(counter, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    // final pass: thread t reduces partials t, t+blockDim, ... then a fixed tree
    double fin_acc[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
        const bool mx = (kinds >> q) & 1u;
        double a = mx ? -INFINITY : 0.0;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
            const double o = ((volatile double *)part)[q * gridDim.x + b];
            a = mx ? amax(a, o) : a + o;
        }
        for (int off = 16; off > 0; off >>= 1) {
            const double o = __shfl_down_sync(0xffffffffu, a, off);
            a = mx ? amax(a, o) : a + o;
        }
        fin_acc[q] = a;
    }
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) sred[q][wid] = fin_acc[q];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double res[NQ];
        for (int q = 0; q < NQ; ++q) {
            const bool mx = (kinds >> q) & 1u;
            double a = sred[q][0];
            for (int w = 1; w < kRedThreads / 32; ++w) a = mx ? amax(a, sred[q][w]) : a + sred[q][w];
            res[q] = a;
            if (result) result[q] = a;
        }
        fin(res);
        *counter = 0u;
    }
}

struct NoFin {
    __device__ void operator()(const double *) const {}
};

// ------------------------------------------------------------------------------ GCR vector ops
// device scalar slots
enum Scal {
    S_BETA = 0, S_DVMX, S_RL2, S_EER0, S_EEM0, S_RL20, S_EER, S_EEM,
    S_AX2 = 16,                          // ax2(1..lord)
    S_DEL = S_AX2 + MPG_MAX_LORD,        // del(1..lord)
    S_COUNT = S_DEL + MPG_MAX_LORD
};

__global__ void k_axpy_pr(int N, const double *__restrict__ scal, const double *__restrict__ xi,
                          const double *__restrict__ axi, double *__restrict__ p, double *__restrict__ r) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    const double beta = scal[S_BETA];
    p[n] = p[n] + beta * xi[n];
    r[n] = r[n] + beta * axi[n];
}

// x(:,i+1) = qr + sum_ii del(ii) x(:,ii) (and the same for ax) — ref.f:1914-1923
struct VecList {
    double *v[MPG_MAX_LORD];
};
__global__ void k_gcr_next(int N, int i, const double *__restrict__ scal, const double *__restrict__ qr,
                           const double *__restrict__ ar, VecList x, VecList ax, double *__restrict__ xo,
                           double *__restrict__ axo) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    double a = qr[n], b = ar[n];
    for (int ii = 0; ii < i; ++ii) {
        const double d = scal[S_DEL + ii];
        a = a + d * x.v[ii][n];
        b = b + d * ax.v[ii][n];
    }
    xo[n] = a;
    axo[n] = b;
}

// restart collapse (ref.f:1924-1937): x(:,1) = qr + del(1) x(:,1) + sum_{ii>=2} del(ii) x(:,ii)
__global__ void k_gcr_restart(int N, int i, const double *__restrict__ scal, const double *__restrict__ qr,
                              const double *__restrict__ ar, VecList x, VecList ax) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    double a = qr[n] + scal[S_DEL] * x.v[0][n];
    double b = ar[n] + scal[S_DEL] * ax.v[0][n];
    for (int ii = 1; ii < i; ++ii) {
        const double d = scal[S_DEL + ii];
        a = a + d * x.v[ii][n];
        b = b + d * ax.v[ii][n];
    }
    x.v[0][n] = a;
    ax.v[0][n] = b;
}

// ------------------------------------------------------------------------------ element-wise
__global__ void k_fill(int N, double *__restrict__ a, double v) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n < N) a[n] = v;
}
__global__ void k_copy(int N, const double *__restrict__ a, double *__restrict__ b) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n < N) b[n] = a[n];
}
__global__ void k_sub(int N, const double *__restrict__ a, const double *__restrict__ b, double *__restrict__ o) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n < N) o[n] = a[n] - b[n];
}
// precon smoothing update (ref.f:607-612): p = p + omega*pstep*(r - rhs), pstep per sm_flag1
__global__ void k_smooth(int N, int sm_flag1, double omega, double beta, const double *__restrict__ d1,
                         const double *__restrict__ r, const double *__restrict__ rhs, double *__restrict__ p) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    double ps = 0.;
    if (sm_flag1 == 1) ps = (-1.) / d1[n];
    else if (sm_flag1 == 2) ps = beta;
    else if (sm_flag1 == 3) ps = beta / (1. - d1[n] * beta);
    p[n] = p[n] + omega * ps * (r[n] - rhs[n]);
}
// reference order <-> internal order
__global__ void k_scatter_perm(int N, const int32_t *__restrict__ perm, const double *__restrict__ src,
                               double *__restrict__ dst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) dst[perm[i]] = src[i];
}
__global__ void k_gather_perm(int N, const int32_t *__restrict__ perm, const double *__restrict__ src,
                              double *__restrict__ dst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) dst[i] = src[perm[i]];
}

}  // namespace mpgk

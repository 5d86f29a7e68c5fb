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

#include <type_traits>

#include "mpgcr_internal.h"

namespace mpgk {

constexpr int kThreads = 256;
#ifndef MPG_RED_BLOCKS
#define MPG_RED_BLOCKS 592
#endif
constexpr int kRedBlocks = MPG_RED_BLOCKS;   // 4 x 148 SMs
constexpr int kRedThreads = 256;
constexpr int kMaxQ = 24;                // quantities per reduction
// nodes whose operands a reduction thread loads before finishing any: as many as fit the
// 64 registers that keep 4 blocks of 256 threads per SM (the grid is 4 blocks per SM)
template <class Loaded> struct RedDepth {
    static constexpr int value = sizeof(Loaded) <= 32 ? 4 : sizeof(Loaded) <= 48 ? 3 : 2;
};

__device__ __forceinline__ double amax(double a, double b) { return a > b ? a : b; }
__device__ __forceinline__ double amin(double a, double b) { return a < b ? a : b; }

// ------------------------------------------------------------------------------ gathers
// Thread n = c*L + k visits the faces of node (c,k) in the reference's edge order.  The loop is
// branch-free and takes two faces per iteration: both faces' operands are loaded before either
// is accumulated, which doubles the loads in flight of this latency-bound gather while keeping
// the reference's order of additions.
struct Face {
    int j;        // neighbour node
    int si;       // face index into Sv (vert) or Sh
    bool sub;     // the reference stores the face with this node second: subtract
    bool vert;
    bool valid;   // false for the missing vertical face at the column's bottom or top
};

__device__ __forceinline__ Face decode_face(int2 en, int n, int k, int L) {
    Face f;
    const bool vert = en.x < 0, below = en.x == MPG_ADJ_BELOW;
    f.vert = vert;
    f.valid = !vert || (below ? k > 0 : k + 1 < L);
    f.sub = vert ? below : ((en.x & 1) != 0);
    const int jv = below ? n - 1 : n + 1, sv = below ? n - 1 : n;
    f.j = vert ? (f.valid ? jv : n) : en.y * L + k;
    f.si = vert ? (f.valid ? sv : n) : (en.x >> 1) * L + k;
    return f;
}

#ifndef MPG_GATHER_U
#define MPG_GATHER_U 2
#endif
template <int U = MPG_GATHER_U, class LD, class AC>
__device__ __forceinline__ void for_faces(const ColMesh &M, int c, int k, int n, LD &&load, AC &&acc) {
    const int beg = __ldg(&M.cptr[c]), end = __ldg(&M.cptr[c + 1]);
    const int L = M.L;
    int j = beg;
    for (; j + U <= end; j += U) {
        Face f[U];
        decltype(load(f[0])) v[U];
#pragma unroll
        for (int u = 0; u < U; ++u) f[u] = decode_face(__ldg(&M.cadj[j + u]), n, k, L);
#pragma unroll
        for (int u = 0; u < U; ++u) v[u] = load(f[u]);
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (f[u].valid) acc(f[u], v[u]);
    }
    for (; j < end; ++j) {
        const Face f = decode_face(__ldg(&M.cadj[j]), n, k, L);
        const auto v = load(f);
        if (f.valid) acc(f, v);
    }
}

__device__ __forceinline__ const double *spick(const ColMesh &M, int d, bool vert) {
    return vert ? M.Sv[d] : M.Sh[d];
}
// face vector si (horizontal or vertical) in the storage type of a kernel instantiation: three
// FP64 arrays, or in mixed precision one packed float4 (x, y, z, 0) per face, so an FP32 gather
// issues one 16-byte load per face instead of three 4-byte ones
template <class T> struct FaceVec;
template <> struct FaceVec<double> {
    __device__ static void load(const ColMesh &M, bool vert, int si, double &x, double &y, double &z) {
        x = __ldg((vert ? M.Sv[0] : M.Sh[0]) + si);
        y = __ldg((vert ? M.Sv[1] : M.Sh[1]) + si);
        z = __ldg((vert ? M.Sv[2] : M.Sh[2]) + si);
    }
};
template <> struct FaceVec<float> {
    __device__ static void load(const ColMesh &M, bool vert, int si, float &x, float &y, float &z) {
        const float4 v = __ldg((vert ? M.Svf4 : M.Shf4) + si);
        x = v.x; y = v.y; z = v.z;
    }
};

// the three flux components between the halves of laplc: three FP64 arrays, or one packed
// float4 per node in mixed precision (one 16-byte load per neighbour)
template <class T> struct Flux;
// (load_cg reads through L2 only: for fluxes written by other blocks of the same launch)
template <> struct Flux<double> {
    double *x, *y, *z;
    __device__ void store(int n, double a, double b, double c) const { x[n] = a; y[n] = b; z[n] = c; }
    __device__ void load(int n, double &a, double &b, double &c) const { a = x[n]; b = y[n]; c = z[n]; }
    __device__ void load_cg(int n, double &a, double &b, double &c) const {
        a = __ldcg(x + n); b = __ldcg(y + n); c = __ldcg(z + n);
    }
};
template <> struct Flux<float> {
    float4 *v;
    __device__ void store(int n, float a, float b, float c) const { v[n] = make_float4(a, b, c, 0.f); }
    __device__ void load(int n, float &a, float &b, float &c) const {
        const float4 t = v[n];
        a = t.x; b = t.y; c = t.z;
    }
    __device__ void load_cg(int n, float &a, float &b, float &c) const {
        const float4 t = __ldcg(v + n);
        a = t.x; b = t.y; c = t.z;
    }
};

// Boundary entries of node (c,k), in reference order.
template <class V>
__device__ __forceinline__ void for_boundary(const ColMesh &M, int c, int k, V &&visit) {
    const int beg = __ldg(&M.bptr[c]), end = __ldg(&M.bptr[c + 1]);
    for (int b = beg; b < end; ++b) {
        const BEntry &be = M.bent[b];
        if (be.k == k) visit(be);
    }
}

template <class T> struct V4T { T a, b, c, d; };
template <class T> struct V6T { T a, b, c, d, e, f; };
using V4 = V4T<double>;
using V6 = V6T<double>;

// derivative (ref.f:3943-4022) of phi for the three components at once:
// g_d = sum over faces of (+/-) S_d * ((phi_n + phi_j) * 0.5).
// With DIFF the transpose of that matrix is applied instead: since the other end of a face
// carries the opposite sign, (B_d^T y)_n = sum over faces of (+/-) S_d * ((y_n - y_j) * 0.5),
// plus the same closure term.
template <class T, bool DIFF = false>
__device__ __forceinline__ void grad3(const ColMesh &M, const T *__restrict__ phi, int c, int k, int n,
                                      T &gx, T &gy, T &gz) {
    const T pn = phi[n];
    T ax = 0., ay = 0., az = 0.;
    for_faces(M, c, k, n,
        [&](const Face &f) {
            V4T<T> v;
            FaceVec<T>::load(M, f.vert, f.si, v.a, v.b, v.c);
            v.d = phi[f.j];
            return v;
        },
        [&](const Face &f, const V4T<T> &v) {
            const T u = (DIFF ? pn - v.d : pn + v.d) * T(0.5);
            const T tx = v.a * u, ty = v.b * u, tz = v.c * u;
            if (f.sub) { ax = ax - tx; ay = ay - ty; az = az - tz; }
            else       { ax = ax + tx; ay = ay + ty; az = az + tz; }
        });
    if (M.iper == 0) {                                  // closure, ref.f:4007-4014
        for_boundary(M, c, k, [&](const BEntry &be) {
            ax = ax + T(be.sbb[0]) * pn;
            ay = ay + T(be.sbb[1]) * pn;
            az = az + T(be.sbb[2]) * pn;
        });
    }
    gx = ax; gy = ay; gz = az;
}

// derivative(fx,1), derivative(fy,2), derivative(fz,3) of three fields (the divergence);
// with DIFF the transposed matrices, as in grad3
template <class T, bool DIFF = false, class FX>
__device__ __forceinline__ void div3(const ColMesh &M, FX f, int c, int k, int n, T &dx, T &dy, T &dz) {
    T fnx, fny, fnz;
    f(n, fnx, fny, fnz);
    T ax = 0., ay = 0., az = 0.;
    for_faces(M, c, k, n,
        [&](const Face &fc) {
            V6T<T> v;
            FaceVec<T>::load(M, fc.vert, fc.si, v.a, v.b, v.c);
            f(fc.j, v.d, v.e, v.f);
            return v;
        },
        [&](const Face &fc, const V6T<T> &v) {
            const T tx = v.a * ((DIFF ? fnx - v.d : fnx + v.d) * T(0.5));
            const T ty = v.b * ((DIFF ? fny - v.e : fny + v.e) * T(0.5));
            const T tz = v.c * ((DIFF ? fnz - v.f : fnz + v.f) * T(0.5));
            if (fc.sub) { ax = ax - tx; ay = ay - ty; az = az - tz; }
            else        { ax = ax + tx; ay = ay + ty; az = az + tz; }
        });
    if (M.iper == 0) {
        for_boundary(M, c, k, [&](const BEntry &be) {
            ax = ax + T(be.sbb[0]) * fnx;
            ay = ay + T(be.sbb[1]) * fny;
            az = az + T(be.sbb[2]) * fnz;
        });
    }
    dx = ax; dy = ay; dz = az;
}

// bcv (ref.f:1583-1643) applied to one node
template <class T>
__device__ __forceinline__ void bcv_node(const ColMesh &M, int c, int k, int n, const double *ue, double flag,
                                         T &u, T &v, T &w) {
    const bool per = (M.iper == 2);
    for_boundary(M, c, k, [&](const BEntry &be) {
        const int t = be.type;
        if (t == 11 || (!per && (t == 5 || t == 6))) {
            const T a0 = T(be.anp[0]), a1 = T(be.anp[1]), a2 = T(be.anp[2]);
            const T vn = u * a0 + v * a1 + w * a2;
            u = u - a0 * vn;
            v = v - a1 * vn;
            w = w - a2 * vn;
        }
        if (!per && (t == 7 || t == 8)) u = T(ue[n] * flag);
    });
}

// transpose of bcv_node with flag = 0: the same symmetric projections (and zeroed u at
// types 7/8), visited in reverse order
template <class T>
__device__ __forceinline__ void bcv_node_adj(const ColMesh &M, int c, int k, T &u, T &v, T &w) {
    const bool per = (M.iper == 2);
    const int beg = __ldg(&M.bptr[c]), end = __ldg(&M.bptr[c + 1]);
    for (int b = end - 1; b >= beg; --b) {
        const BEntry &be = M.bent[b];
        if (be.k != k) continue;
        const int t = be.type;
        if (!per && (t == 7 || t == 8)) u = T(0);
        if (t == 11 || (!per && (t == 5 || t == 6))) {
            const T a0 = T(be.anp[0]), a1 = T(be.anp[1]), a2 = T(be.anp[2]);
            const T vn = u * a0 + v * a1 + w * a2;
            u = u - a0 * vn;
            v = v - a1 * vn;
            w = w - a2 * vn;
        }
    }
}

// ------------------------------------------------------------------------------ operators
// latency-bound gathers that fit 40 registers without spilling: keep 6 blocks (48 warps) per SM
#ifndef MPG_GATHER_MINB
#define MPG_GATHER_MINB 6
#endif
#define GATHER_BOUNDS __launch_bounds__(kThreads, MPG_GATHER_MINB)
// the divergence gathers load six values per face
#ifdef MPG_DIV_MINB
#define DIV_BOUNDS __launch_bounds__(kThreads, MPG_DIV_MINB)
#else
#define DIV_BOUNDS
#endif

#define NODE_BEGIN                                                            \
    const int n = blockIdx.x * blockDim.x + threadIdx.x;                      \
    if (n >= M.N) return;                                                     \
    const int c = n / M.L, k = n - c * M.L;

// derivative(unk, out, idx)
__global__ void GATHER_BOUNDS k_derivative(ColMesh M, const double *__restrict__ phi, double *__restrict__ out, int idx) {
    NODE_BEGIN
    double gx, gy, gz;
    grad3<double>(M, phi, c, k, n, gx, gy, gz);
    out[n] = idx == 1 ? gx : idx == 2 ? gy : gz;
}

// bcv(u, v, w, flag) on whole fields
__global__ void k_bcv(ColMesh M, double *u, double *v, double *w, const double *__restrict__ ue, double flag) {
    NODE_BEGIN
    if (__ldg(&M.bptr[c]) == __ldg(&M.bptr[c + 1])) return;
    double a = u[n], b = v[n], d = w[n];
    bcv_node<double>(M, c, k, n, ue, flag, a, b, d);
    u[n] = a; v[n] = b; w[n] = d;
}

// laplc first half (ref.f:1303-1338) at node n: gradient, scaling, bcv(.,0.), times rh0.  T is
// the storage and arithmetic type (double; float for the mixed-precision solve).
template <class T>
__device__ __forceinline__ void lap_grad_node(const ColMesh &M, int n, const T *__restrict__ p,
                                              const T *__restrict__ vol, const T *__restrict__ rh0,
                                              const T *__restrict__ coefw, const double *__restrict__ ue, T dt,
                                              int impfl, const Flux<T> &F) {
    const int c = n / M.L, k = n - c * M.L;
    T gx, gy, gz;
    grad3<T>(M, p, c, k, n, gx, gy, gz);
    const T v = vol[n];
    T dx = dt * gx / v, dy = dt * gy / v, dz = dt * gz / v;
    dx = T(0.5) * dx / T(1.0);                 // (gmm*cosa)**2 == 1 for isfera = 0
    dy = T(0.5) * dy / T(1.0);
    dz = T(0.5) * dz * (coefw[n] * (T)impfl + (T)(1 - impfl));
    bcv_node<T>(M, c, k, n, ue, 0.0, dx, dy, dz);
    const T r = rh0[n];
    F.store(n, dx * r, dy * r, dz * r);
}

// laplc's first half keeps 6 blocks per SM in FP64 (40 registers); the FP32 instantiation fits
// 32 registers without spilling, so it takes 8 (every warp slot of the SM): 563 against 676 us
// on the 512x512x81 workload
#ifndef MPG_LAPGRAD_MINB_F32
#define MPG_LAPGRAD_MINB_F32 8
#endif
template <class T> struct LapGradMinB { static constexpr int value = MPG_GATHER_MINB; };
template <> struct LapGradMinB<float> { static constexpr int value = MPG_LAPGRAD_MINB_F32; };

template <class T>
__global__ void __launch_bounds__(kThreads, LapGradMinB<T>::value)
k_lap_grad(ColMesh M, const T *__restrict__ p, const T *__restrict__ vol,
                                         const T *__restrict__ rh0, const T *__restrict__ coefw,
                                         const double *__restrict__ ue, T dt, int impfl, Flux<T> F) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= M.N) return;
    lap_grad_node<T>(M, n, p, vol, rh0, coefw, ue, dt, impfl, F);
}

// laplc second half (ref.f:1339-1350): alap = (Dx(Fx) + Dy(Fy) + Dz(Fz)) / (vol*rh0)
template <class T>
__global__ void DIV_BOUNDS k_lap_div(ColMesh M, const Flux<T> F, const T *__restrict__ vol,
                                     const T *__restrict__ rh0, T *__restrict__ alap) {
    NODE_BEGIN
    T dx, dy, dz;
    div3<T>(M, [&](int j, T &a, T &b, T &d) { F.load(j, a, b, d); }, c, k, n, dx, dy, dz);
    alap[n] = (dx + dy + dz) / (vol[n] * rh0[n]);
}

// ------------------------------------------------------------------------------ level-pair divergence
// laplc's second half with one thread per pair of adjacent levels (k0 = 2p, k1 = 2p + 1) of a
// column: the adjacency entry, its decode and the face addressing serve both nodes (a horizontal
// face of level k1 is the next element of every array), and the vertical face between the two is
// loaded once.  Each node still adds its terms in the reference's edge order, so the result is
// bit-identical to k_lap_div.  Measured on the 512x512x81 workload it is 5% faster than k_lap_div
// (823 against 869 us in FP64); the same structure for the gradient half was 9% slower, which is
// why that half keeps one thread per node.
struct Face2 {
    int j0, j1, s0, s1;
    bool sub, vert, v0, v1;
};
__device__ __forceinline__ Face2 decode_face2(int2 en, int n0, int k0, int L, bool two) {
    Face2 f;
    const bool vert = en.x < 0, below = en.x == MPG_ADJ_BELOW;
    f.vert = vert;
    f.sub = vert ? below : ((en.x & 1) != 0);
    // level k0
    f.v0 = !vert || (below ? k0 > 0 : two);
    const int hj = en.y * L + k0, hs = (en.x >> 1) * L + k0;
    f.j0 = vert ? (below ? (k0 > 0 ? n0 - 1 : n0) : (two ? n0 + 1 : n0)) : hj;
    f.s0 = vert ? (below ? (k0 > 0 ? n0 - 1 : n0) : n0) : hs;
    // level k1 = k0 + 1 (present when two): below is always valid, above when k1 + 1 < L
    f.v1 = two && (!vert || below || k0 + 2 < L);
    f.j1 = vert ? (below ? n0 : (k0 + 2 < L ? n0 + 2 : n0)) : hj + 1;
    f.s1 = vert ? (below ? n0 : n0 + 1) : hs + 1;
    return f;
}

// 64 registers: the two nodes' operands of a face in flight together
constexpr int kLapPairMinBlocks = 4;

// level pair t of laplc's second half; CG: the fluxes were written by other blocks of the same
// launch (read through L2)
template <class T, bool CG = false>
__device__ __forceinline__ void lap_div_pair(const ColMesh &M, int PL, int t, const Flux<T> &F,
                                             const T *__restrict__ vol, const T *__restrict__ rh0,
                                             T *__restrict__ alap) {
    const int c = t / PL, L = M.L, k0 = 2 * (t - c * PL), n0 = c * L + k0;
    const bool two = k0 + 1 < L;
    auto fl = [&](int n, T &a, T &b, T &d) {
        if (CG) F.load_cg(n, a, b, d);
        else F.load(n, a, b, d);
    };
    T f0x, f0y, f0z, f1x = 0., f1y = 0., f1z = 0.;
    fl(n0, f0x, f0y, f0z);
    if (two) fl(n0 + 1, f1x, f1y, f1z);
    T a0x = 0., a0y = 0., a0z = 0., a1x = 0., a1y = 0., a1z = 0.;
    const int beg = __ldg(&M.cptr[c]), end = __ldg(&M.cptr[c + 1]);
    for (int j = beg; j < end; ++j) {
        const Face2 f = decode_face2(__ldg(&M.cadj[j]), n0, k0, L, two);
        T sx0, sy0, sz0, sx1 = 0., sy1 = 0., sz1 = 0., g0x, g0y, g0z, g1x = 0., g1y = 0., g1z = 0.;
        FaceVec<T>::load(M, f.vert, f.s0, sx0, sy0, sz0);
        fl(f.j0, g0x, g0y, g0z);
        if (two) {
            FaceVec<T>::load(M, f.vert, f.s1, sx1, sy1, sz1);
            fl(f.j1, g1x, g1y, g1z);
        }
        if (f.v0) {
            const T tx = sx0 * ((f0x + g0x) * T(0.5));
            const T ty = sy0 * ((f0y + g0y) * T(0.5));
            const T tz = sz0 * ((f0z + g0z) * T(0.5));
            if (f.sub) { a0x = a0x - tx; a0y = a0y - ty; a0z = a0z - tz; }
            else       { a0x = a0x + tx; a0y = a0y + ty; a0z = a0z + tz; }
        }
        if (f.v1) {
            const T tx = sx1 * ((f1x + g1x) * T(0.5));
            const T ty = sy1 * ((f1y + g1y) * T(0.5));
            const T tz = sz1 * ((f1z + g1z) * T(0.5));
            if (f.sub) { a1x = a1x - tx; a1y = a1y - ty; a1z = a1z - tz; }
            else       { a1x = a1x + tx; a1y = a1y + ty; a1z = a1z + tz; }
        }
    }
    const T fx[2] = {f0x, f1x}, fy[2] = {f0y, f1y}, fz[2] = {f0z, f1z};
    T ax[2] = {a0x, a1x}, ay[2] = {a0y, a1y}, az[2] = {a0z, a1z};
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        if (h == 1 && !two) break;
        const int k = k0 + h, n = n0 + h;
        T dx = ax[h], dy = ay[h], dz = az[h];
        if (M.iper == 0) {
            for_boundary(M, c, k, [&](const BEntry &be) {
                dx = dx + T(be.sbb[0]) * fx[h];
                dy = dy + T(be.sbb[1]) * fy[h];
                dz = dz + T(be.sbb[2]) * fz[h];
            });
        }
        alap[n] = (dx + dy + dz) / (vol[n] * rh0[n]);
    }
}

// FP32 (mixed precision) level pairs at 6 blocks per SM, 40 registers: measured 494 us against
// 520 at 5 blocks (48 registers) and 590 at 4 (64) on the 512x512x81 workload
#ifndef MPG_DIV2_MINB_F32
#define MPG_DIV2_MINB_F32 6
#endif
template <class T> struct LapDiv2MinB { static constexpr int value = kLapPairMinBlocks; };
template <> struct LapDiv2MinB<float> { static constexpr int value = MPG_DIV2_MINB_F32; };

template <class T>
__global__ void __launch_bounds__(kThreads, LapDiv2MinB<T>::value)
k_lap_div2(ColMesh M, int PL, const Flux<T> F, const T *__restrict__ vol, const T *__restrict__ rh0,
           T *__restrict__ alap) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= M.NC * PL) return;
    lap_div_pair<T>(M, PL, t, F, vol, rh0, alap);
}

// ------------------------------------------------------------------------------ fused laplc
// Both halves of laplc in one persistent launch.  The work is cut into gradient items (kThreads
// consecutive nodes each, k_lap_grad's blocks) and divergence items (kThreads level pairs each,
// k_lap_div2's blocks).  Blocks take tickets from a counter in order; `sched` maps ticket to item
// and places every divergence item after the last gradient item it reads, so a divergence item
// runs while the fluxes and face vectors it reads are still in L2 from the gradient pass a few
// hundred items earlier, instead of a second full sweep over HBM.  Before reading, a divergence
// item waits for the flags of the gradient items in its dependency ranges.  Every such item
// holds an earlier ticket, so the block working on it has started and needs nothing else: the
// wait always ends.  The wait is bounded all the same; when it gives up it records an error in
// state[3] and the item goes ahead (the host reports the error).  Each node's arithmetic is
// k_lap_grad's and k_lap_div2's, so the result is bit-identical to the two-launch form.
// Measured at 512x512x81 (FP64): 2.00 ms per laplc against 1.71 ms for the two launches, although
// DRAM traffic falls by about 40% (L2 hit rate 65%).  The gathers are latency-bound, and the kernel's
// 64 registers (the divergence's) hold the gradient items to 32 warps per SM where k_lap_grad
// runs 48.  The library therefore launches the two halves unless MPG_LAPLC_FUSED=1 at creation.
//
// state: [0] next ticket, [1] blocks finished, [2] launches completed (the epoch), [3] error.
// The last block to finish resets [0] and [1] and advances [2], so the next launch on the
// stream starts from a clean counter; gradient flags hold the epoch of the launch that wrote them.
struct LapSched {
    const int32_t *sched;    // [total] item per ticket: g >= 0 gradient item g, -(d+1) divergence item d
    const int32_t *dptr;     // [ND+1] dependency ranges of each divergence item
    const int2 *drng;        // inclusive ranges of gradient items
    int32_t *flag;           // [NG]
    int32_t *state;          // [4]
    int32_t total;
};

__device__ __forceinline__ int ld_acquire_gpu(const int32_t *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_gpu(int32_t *p, int v) {
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

#ifndef MPG_LAPF_SPINS
#define MPG_LAPF_SPINS (1LL << 22)
#endif
#ifndef MPG_LAPF_MINB
#define MPG_LAPF_MINB 4
#endif

template <class T>
__global__ void __launch_bounds__(kThreads, MPG_LAPF_MINB)
k_lap_fused(ColMesh M, int PL, LapSched S, const T *__restrict__ p, const T *__restrict__ vol,
            const T *__restrict__ rh0, const T *__restrict__ coefw, const double *__restrict__ ue, T dt,
            int impfl, Flux<T> F, T *__restrict__ alap) {
    __shared__ int s_ticket[2];
    __shared__ int s_epoch;
    const int tid = threadIdx.x;
    if (tid == 0) {
        s_epoch = *(volatile int32_t *)&S.state[2] + 1;
        s_ticket[0] = atomicAdd(&S.state[0], 1);
    }
    __syncthreads();
    const int epoch = s_epoch;
    const int NP = M.NC * PL;
    for (int buf = 0;; buf ^= 1) {
        const int ticket = s_ticket[buf];
        if (ticket >= S.total) break;
        if (tid == 0) s_ticket[buf ^ 1] = atomicAdd(&S.state[0], 1);   // in flight during this item
        const int item = __ldg(&S.sched[ticket]);
        if (item >= 0) {
            const int n = item * kThreads + tid;
            if (n < M.N) lap_grad_node<T>(M, n, p, vol, rh0, coefw, ue, dt, impfl, F);
            // the barrier orders every thread's flux stores before thread 0's release, which is
            // cumulative: a block that acquires the flag sees all of them (one release per item;
            // a fence in every thread serialises the SM)
            __syncthreads();
            if (tid == 0) st_release_gpu(&S.flag[item], epoch);
        } else {
            const int d = -item - 1;
            // warp 0 acquires the flags of the gradient items this item reads; the barrier then
            // passes the acquired fluxes on to the whole block
            if (tid < 32) {
                bool ok = true;
                const int rb = __ldg(&S.dptr[d]), re = __ldg(&S.dptr[d + 1]);
                for (int r = rb; r < re; ++r) {
                    const int2 g = __ldg(&S.drng[r]);
                    for (int i = g.x + tid; i <= g.y; i += 32) {
                        long long spins = 0;
                        while (ld_acquire_gpu(&S.flag[i]) != epoch) {
                            if (++spins > MPG_LAPF_SPINS) { ok = false; break; }
                            __nanosleep(64);
                        }
                    }
                }
                if (__any_sync(0xffffffffu, !ok) && tid == 0) atomicExch(&S.state[3], 1);
            }
            __syncthreads();
            const int t = d * kThreads + tid;
            if (t < NP) lap_div_pair<T, true>(M, PL, t, F, vol, rh0, alap);
        }
        __syncthreads();
    }
    if (tid == 0) {
        __threadfence();
        if (atomicAdd(&S.state[1], 1) == (int)gridDim.x - 1) {
            atomicExch(&S.state[0], 0);
            atomicExch(&S.state[1], 0);
            __threadfence();
            atomicAdd(&S.state[2], 1);
        }
    }
}

// ------------------------------------------------------------------------------ mbarrier wait
__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Bounded wait for phase `phase` of an mbarrier: true once the phase completed, false after
// `limit` polls (mbarrier.try_wait may itself suspend the thread for a while between polls).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t phase, long long limit) {
    uint32_t done = 0;
    long long spins = 0;
    while (!done) {
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}\n"
                     : "=r"(done) : "r"(smem_addr(bar)), "r"(phase) : "memory");
        if (!done && ++spins > limit) break;
    }
    return done != 0;
}

// Adjoint of laplc in the inner product weighted by W = vol*rh0.  laplc is
// A = diag(1/W) sum_d B_d rh0 P S1 B_d (B_d: derivative matrix of component d, S1: the dt/2,
// coefw and 1/vol scaling, P: bcv's projections), so A^T W y = sum_d B_d^T S1 P^T rh0 B_d^T y.
// First half: G_d = S1 P^T rh0 B_d^T y.
__global__ void GATHER_BOUNDS k_lapT_grad(ColMesh M, const double *__restrict__ y, const double *__restrict__ vol,
                                          const double *__restrict__ rh0, const double *__restrict__ coefw,
                                          double dt, int impfl, double *__restrict__ Gx, double *__restrict__ Gy,
                                          double *__restrict__ Gz) {
    NODE_BEGIN
    double hx, hy, hz;
    grad3<double, true>(M, y, c, k, n, hx, hy, hz);
    const double r = rh0[n];
    hx = hx * r; hy = hy * r; hz = hz * r;
    bcv_node_adj<double>(M, c, k, hx, hy, hz);
    const double v = vol[n];
    Gx[n] = 0.5 * dt * hx / v;
    Gy[n] = 0.5 * dt * hy / v;
    Gz[n] = 0.5 * dt * hz * (coefw[n] * (double)impfl + (double)(1 - impfl)) / v;
}

// Second half: out = sum_d B_d^T G_d, divided by W when divw (then <A u, y>_W = <u, out>_W).
__global__ void k_lapT_div(ColMesh M, const double *__restrict__ Gx, const double *__restrict__ Gy,
                           const double *__restrict__ Gz, const double *__restrict__ vol,
                           const double *__restrict__ rh0, int divw, double *__restrict__ out) {
    NODE_BEGIN
    double dx, dy, dz;
    div3<double, true>(M, [&](int j, double &a, double &b, double &d) { a = Gx[j]; b = Gy[j]; d = Gz[j]; },
                       c, k, n, dx, dy, dz);
    const double s = dx + dy + dz;
    out[n] = divw ? s / (vol[n] * rh0[n]) : s;
}

// prfr (ref.f:1536-1580)
__global__ void GATHER_BOUNDS k_prfr(ColMesh M, const double *__restrict__ p, const double *__restrict__ us,
                       const double *__restrict__ vs, const double *__restrict__ ws,
                       const double *__restrict__ vol, const double *__restrict__ coefw,
                       const double *__restrict__ ue, double dt, int impfl,
                       double *__restrict__ uo, double *__restrict__ vo, double *__restrict__ wo) {
    NODE_BEGIN
    double gx, gy, gz;
    grad3<double>(M, p, c, k, n, gx, gy, gz);
    const double v = vol[n];
    const double dpx = gx / 1.0 / v, dpy = gy / 1.0 / v, dpz = gz / v;
    double a = us[n] - 0.5 * dt * dpx;
    double b = vs[n] - 0.5 * dt * dpy;
    double d = ws[n] - 0.5 * dt * dpz * (coefw[n] * (double)impfl + (double)(1 - impfl));
    bcv_node<double>(M, c, k, n, ue, 1.0, a, b, d);
    uo[n] = a; vo[n] = b; wo[n] = d;
}

// div(ua, va, wa, rhs, iflg) (ref.f:2096-2147)
__global__ void k_div(ColMesh M, const double *__restrict__ ua, const double *__restrict__ va,
                      const double *__restrict__ wa, const double *__restrict__ vol,
                      const double *__restrict__ rh0, int iflg, double *__restrict__ rhs) {
    NODE_BEGIN
    double dx, dy, dz;
    if (iflg == -1)
        div3<double>(M, [&](int j, double &a, double &b, double &d) {
            const double r = rh0[j]; a = ua[j] * r; b = va[j] * r; d = wa[j] * r; }, c, k, n, dx, dy, dz);
    else
        div3<double>(M, [&](int j, double &a, double &b, double &d) { a = ua[j]; b = va[j]; d = wa[j]; }, c, k, n, dx, dy, dz);
    const double v = vol[n];
    rhs[n] = (double)iflg * (dx / v + dy / v + dz / v) / rh0[n];
}

// ------------------------------------------------------------------------------ line solve
// z = M^{-1} rhs per column (Thomas, FP64, bottom to top), p = (acc ? p : 0) + omega * z.
// A warp owns 32 consecutive columns.  Their right-hand sides (contiguous in the column layout)
// pass through a 32 x kLineChunk shared-memory tile, loaded and stored with coalesced accesses;
// the factorisation (a, 1/m, c') and the forward-sweep values d are stored interleaved
// (line_index), so lane l reads and writes level k of column col0+l inside one 256-byte segment.
// With 4 KiB of shared memory per warp the kernel keeps enough warps resident to stream.
// Measured alternatives at 512x512x81 (FP64, CUDA events), all slower: the largest shared-memory
// carve-out requested for the kernel (295 against 238 us), chunks of 14 levels with 2-4 levels of
// coefficients ahead and 7 blocks per SM so that the grid fits one wave (320-367 us), dropping the
// scratch d from L2 after the backward sweep (no gain).
constexpr int kLineWarps = 8;
constexpr int kLineChunk = 16;
constexpr int kLinePre = 8;
#define LINE_BOUNDS __launch_bounds__(32 * kLineWarps)
template <class TO>
__global__ void LINE_BOUNDS
k_line_solve(int NC, int L, const double *__restrict__ rhs, const double *__restrict__ la,
             const double *__restrict__ linv, const double *__restrict__ lcp, double omega, int acc,
             double *__restrict__ dbuf, TO *__restrict__ p) {
    __shared__ double tile[kLineWarps][32][kLineChunk + 1];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int col0 = (blockIdx.x * kLineWarps + w) * 32;
    if (col0 >= NC) return;
    const int ncols = min(32, NC - col0);
    double(*t)[kLineChunk + 1] = tile[w];
    const int c = col0 + lane;
    const bool own = lane < ncols;
    // forward sweep: d_k = (r_k - a_k d_{k-1}) / m_k
    double d = 0.;
    for (int k0 = 0; k0 < L; k0 += kLineChunk) {
        const int nk = min(kLineChunk, L - k0);
        for (int i = lane; i < ncols * nk; i += 32) {
            const int cc = i / nk, kk = i - cc * nk;
            t[cc][kk] = rhs[(int64_t)(col0 + cc) * L + k0 + kk];
        }
        __syncwarp();
        if (own) {
            // coefficients of kLinePre levels are loaded before the dependent chain uses them
            for (int kb = 0; kb < nk; kb += kLinePre) {
                double A[kLinePre], Mi[kLinePre];
#pragma unroll
                for (int i = 0; i < kLinePre; ++i) {
                    const int64_t li = line_index(c, k0 + kb + i, L);
                    A[i] = kb + i < nk ? la[li] : 0.;
                    Mi[i] = kb + i < nk ? linv[li] : 0.;
                }
#pragma unroll
                for (int i = 0; i < kLinePre; ++i) {
                    if (kb + i >= nk) break;
                    const int k = k0 + kb + i;
                    d = (k == 0) ? t[lane][kb + i] * Mi[i] : (t[lane][kb + i] - A[i] * d) * Mi[i];
                    dbuf[line_index(c, k, L)] = d;
                }
            }
        }
        __syncwarp();
    }
    // backward sweep: z_k = d_k - c'_k z_{k+1}, top chunk first
    double z = 0.;
    const int last0 = ((L - 1) / kLineChunk) * kLineChunk;
    for (int k0 = last0; k0 >= 0; k0 -= kLineChunk) {
        const int nk = min(kLineChunk, L - k0);
        if (own) {
            for (int kb = nk - 1; kb >= 0; kb -= kLinePre) {
                double D[kLinePre], Cp[kLinePre];
#pragma unroll
                for (int i = 0; i < kLinePre; ++i) {
                    const int64_t li = line_index(c, k0 + kb - i, L);
                    D[i] = kb - i >= 0 ? dbuf[li] : 0.;
                    Cp[i] = kb - i >= 0 ? lcp[li] : 0.;
                }
#pragma unroll
                for (int i = 0; i < kLinePre; ++i) {
                    if (kb - i < 0) break;
                    const int k = k0 + kb - i;
                    z = (k == L - 1) ? D[i] : D[i] - Cp[i] * z;
                    t[lane][kb - i] = z;
                }
            }
        }
        __syncwarp();
        for (int i = lane; i < ncols * nk; i += 32) {
            const int cc = i / nk, kk = i - cc * nk;
            const int64_t g = (int64_t)(col0 + cc) * L + k0 + kk;
            const double prev = acc ? (double)p[g] : 0.0;
            p[g] = (TO)(prev + omega * t[cc][kk]);
        }
        __syncwarp();
    }
}

// The column blocks of laplc (iprc = 4) are tridiagonal on the even and on the odd levels: the
// same sweeps as k_line_solve with the recurrences reaching two levels back / ahead, both parity
// chains advanced together level by level.  Staging, prefetch and indexing are k_line_solve's.
template <class TO>
__global__ void LINE_BOUNDS
k_wide_solve(int NC, int L, const double *__restrict__ rhs, const double *__restrict__ la,
             const double *__restrict__ linv, const double *__restrict__ lcp, double omega, int acc,
             double *__restrict__ dbuf, TO *__restrict__ p) {
    __shared__ double tile[kLineWarps][32][kLineChunk + 1];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int col0 = (blockIdx.x * kLineWarps + w) * 32;
    if (col0 >= NC) return;
    const int ncols = min(32, NC - col0);
    double(*t)[kLineChunk + 1] = tile[w];
    const int c = col0 + lane;
    const bool own = lane < ncols;
    // forward sweep: d_k = (r_k - a_k d_{k-2}) / m_k
    double d1 = 0., d2 = 0.;                 // d_{k-1}, d_{k-2}
    for (int k0 = 0; k0 < L; k0 += kLineChunk) {
        const int nk = min(kLineChunk, L - k0);
        for (int i = lane; i < ncols * nk; i += 32) {
            const int cc = i / nk, kk = i - cc * nk;
            t[cc][kk] = rhs[(int64_t)(col0 + cc) * L + k0 + kk];
        }
        __syncwarp();
        if (own) {
            for (int kb = 0; kb < nk; kb += kLinePre) {
                double A[kLinePre], Mi[kLinePre];
#pragma unroll
                for (int i = 0; i < kLinePre; ++i) {
                    const int64_t li = line_index(c, k0 + kb + i, L);
                    A[i] = kb + i < nk ? la[li] : 0.;
                    Mi[i] = kb + i < nk ? linv[li] : 0.;
                }
#pragma unroll
                for (int i = 0; i < kLinePre; ++i) {
                    if (kb + i >= nk) break;
                    const int k = k0 + kb + i;
                    const double d = (k < 2) ? t[lane][kb + i] * Mi[i] : (t[lane][kb + i] - A[i] * d2) * Mi[i];
                    dbuf[line_index(c, k, L)] = d;
                    d2 = d1;
                    d1 = d;
                }
            }
        }
        __syncwarp();
    }
    // backward sweep: z_k = d_k - c'_k z_{k+2}, top chunk first
    double z1 = 0., z2 = 0.;                 // z_{k+1}, z_{k+2}
    const int last0 = ((L - 1) / kLineChunk) * kLineChunk;
    for (int k0 = last0; k0 >= 0; k0 -= kLineChunk) {
        const int nk = min(kLineChunk, L - k0);
        if (own) {
            for (int kb = nk - 1; kb >= 0; kb -= kLinePre) {
                double D[kLinePre], Cp[kLinePre];
#pragma unroll
                for (int i = 0; i < kLinePre; ++i) {
                    const int64_t li = line_index(c, k0 + kb - i, L);
                    D[i] = kb - i >= 0 ? dbuf[li] : 0.;
                    Cp[i] = kb - i >= 0 ? lcp[li] : 0.;
                }
#pragma unroll
                for (int i = 0; i < kLinePre; ++i) {
                    if (kb - i < 0) break;
                    const int k = k0 + kb - i;
                    const double z = (k >= L - 2) ? D[i] : D[i] - Cp[i] * z2;
                    t[lane][kb - i] = z;
                    z2 = z1;
                    z1 = z;
                }
            }
        }
        __syncwarp();
        for (int i = lane; i < ncols * nk; i += 32) {
            const int cc = i / nk, kk = i - cc * nk;
            const int64_t g = (int64_t)(col0 + cc) * L + k0 + kk;
            const double prev = acc ? (double)p[g] : 0.0;
            p[g] = (TO)(prev + omega * t[cc][kk]);
        }
        __syncwarp();
    }
}

// ------------------------------------------------------------------------------ reductions
enum RedKind { RSUM = 0, RMAX = 1 };

// A reduction functor may split its work per node into load(n) -> Loaded and finish(n, Loaded,
// vals) (it then defines a nested type Loaded).  k_reduce then loads RedDepth nodes of its
// grid-stride sequence before finishing any, which the compiler cannot arrange by itself
// when finish stores to arrays that might alias the next node's operands.  The order in which a
// thread accumulates its nodes is the same, so the results are bit-identical.
template <class P, class = void> struct SplitProd { static constexpr bool value = false; };
template <class P> struct SplitProd<P, std::void_t<typename P::Loaded>> { static constexpr bool value = true; };

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
    auto add = [&](const double *v) {
#pragma unroll
        for (int q = 0; q < NQ; ++q)
            acc[q] = ((kinds >> q) & 1u) ? amax(acc[q], v[q]) : acc[q] + v[q];
    };
    int n = blockIdx.x * blockDim.x + threadIdx.x;
    if constexpr (SplitProd<Prod>::value) {
        constexpr int D = RedDepth<typename Prod::Loaded>::value;
        for (; n + (D - 1) * stride < N; n += D * stride) {
            typename Prod::Loaded a[D];
#pragma unroll
            for (int d = 0; d < D; ++d) a[d] = prod.load(n + d * stride);
#pragma unroll
            for (int d = 0; d < D; ++d) {
                double v[NQ];
                prod.finish(n + d * stride, a[d], v);
                add(v);
            }
        }
        for (; n < N; n += stride) {
            double v[NQ];
            prod.finish(n, prod.load(n), v);
            add(v);
        }
    } else {
        for (; n < N; n += stride) {
            double v[NQ];
            prod(n, v);
            add(v);
        }
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

// ------------------------------------------------------------------------------ element-wise
__global__ void k_fill(int N, double *__restrict__ a, double v) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n < N) a[n] = v;
}
template <class TA, class TB>
__global__ void k_copy(int N, const TA *__restrict__ a, TB *__restrict__ b) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n < N) b[n] = (TB)a[n];
}
template <class T>
__global__ void k_sub_mixed(int N, const double *__restrict__ a, const T *__restrict__ b, double *__restrict__ o) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n < N) o[n] = a[n] - (double)b[n];
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

// The reference's duplicate-node form of a periodic domain (iper = 2 with icoin/icoin2/icoin4
// lists): the nodes of opposite sides are separate copies, each holding its part of the dual cell,
// and cyclicr/cyclicr2/cyclicr4 (ref.f:4377-4446) replace every copy's partial edge sum by the sum
// over its group, in list order: u(il) + u(ir) for a pair, ((u1 + u2) + u3) + u4 for a corner.
//
// Each gather kernel of the library runs over all nodes as usual, so at a copy it produces the
// copy's partial sum.  The fix-up kernels below then recompute, for every copy, the partial sums
// of all members of its group with the same per-node gathers (each member over its own faces, in
// the reference's edge order), add them in cyclicr's order and apply the rest of the operator at
// the copy itself.  Copies are the boundary columns of the 2-D mesh, a small share of the nodes.
#pragma once

#include "mpdata.cuh"

namespace mpgk {

struct CopyList {
    int32_t n;                  // copy nodes (every member of every group)
    const int32_t *node;        // [n] internal node of the copy
    const int32_t *gbeg;        // [n] offset of its group in members
    const int32_t *gsize;       // [n] 2 or 4
    const int32_t *members;     // group members in list order (internal nodes)
    int32_t ngroups;            // groups, in the order icoin, icoin2, icoin4
    const int32_t *grp;         // [ngroups] offset into members
    const int32_t *grpsize;     // [ngroups]
};

#define COPY_BEGIN                                                             \
    const int i = blockIdx.x * blockDim.x + threadIdx.x;                      \
    if (i >= CL.n) return;                                                     \
    const int n = CL.node[i], c = n / M.L, k = n - c * M.L;                   \
    const int32_t *mem = CL.members + CL.gbeg[i];                             \
    const int gs = CL.gsize[i];

// the three components of the derivative of phi at every member of the group, added in order
template <class T, class FN>
__device__ __forceinline__ void group_sum3(const ColMesh &M, const int32_t *mem, int gs, FN partial, T &sx, T &sy,
                                           T &sz) {
    for (int q = 0; q < gs; ++q) {
        const int x = mem[q], cx = x / M.L, kx = x - cx * M.L;
        T a, b, d;
        partial(cx, kx, x, a, b, d);
        if (q == 0) { sx = a; sy = b; sz = d; }
        else { sx = sx + a; sy = sy + b; sz = sz + d; }
    }
}

// derivative(unk, out, idx) at the copies (ref.f:3943-4019)
__global__ void k_cp_derivative(ColMesh M, CopyList CL, const double *__restrict__ phi, double *__restrict__ out,
                                int idx) {
    COPY_BEGIN
    double gx, gy, gz;
    group_sum3<double>(M, mem, gs, [&](int cx, int kx, int x, double &a, double &b, double &d) {
        grad3<double>(M, phi, cx, kx, x, a, b, d); }, gx, gy, gz);
    (void)k;
    out[n] = idx == 1 ? gx : idx == 2 ? gy : gz;
}

// laplc's first half at the copies: group gradient, then as k_lap_grad
template <class T>
__global__ void k_cp_lap_grad(ColMesh M, CopyList CL, const T *__restrict__ p, const T *__restrict__ vol,
                              const T *__restrict__ rh0, const T *__restrict__ coefw, const double *__restrict__ ue,
                              T dt, int impfl, Flux<T> F) {
    COPY_BEGIN
    T gx, gy, gz;
    group_sum3<T>(M, mem, gs, [&](int cx, int kx, int x, T &a, T &b, T &d) { grad3<T>(M, p, cx, kx, x, a, b, d); },
                  gx, gy, gz);
    const T v = vol[n];
    T dx = dt * gx / v, dy = dt * gy / v, dz = dt * gz / v;
    dx = T(0.5) * dx / T(1.0);
    dy = T(0.5) * dy / T(1.0);
    dz = T(0.5) * dz * (coefw[n] * (T)impfl + (T)(1 - impfl));
    bcv_node<T>(M, c, k, n, ue, 0.0, dx, dy, dz);
    const T r = rh0[n];
    F.store(n, dx * r, dy * r, dz * r);
}

// laplc's second half at the copies: every component summed over the group (three derivative
// calls, each followed by cyclicr), then as k_lap_div
template <class T>
__global__ void k_cp_lap_div(ColMesh M, CopyList CL, const Flux<T> F, const T *__restrict__ vol,
                             const T *__restrict__ rh0, T *__restrict__ alap) {
    COPY_BEGIN
    T dx, dy, dz;
    group_sum3<T>(M, mem, gs, [&](int cx, int kx, int x, T &a, T &b, T &d) {
        div3<T>(M, [&](int j, T &u, T &v, T &w) { F.load(j, u, v, w); }, cx, kx, x, a, b, d); }, dx, dy, dz);
    (void)c; (void)k;
    alap[n] = (dx + dy + dz) / (vol[n] * rh0[n]);
}

// prfr at the copies: group gradient, then as k_prfr
__global__ void k_cp_prfr(ColMesh M, CopyList CL, const double *__restrict__ p, const double *__restrict__ us,
                          const double *__restrict__ vs, const double *__restrict__ ws,
                          const double *__restrict__ vol, const double *__restrict__ coefw,
                          const double *__restrict__ ue, double dt, int impfl, double *__restrict__ uo,
                          double *__restrict__ vo, double *__restrict__ wo) {
    COPY_BEGIN
    double gx, gy, gz;
    group_sum3<double>(M, mem, gs, [&](int cx, int kx, int x, double &a, double &b, double &d) {
        grad3<double>(M, p, cx, kx, x, a, b, d); }, gx, gy, gz);
    const double v = vol[n];
    const double dpx = gx / 1.0 / v, dpy = gy / 1.0 / v, dpz = gz / v;
    double a = us[n] - 0.5 * dt * dpx;
    double b = vs[n] - 0.5 * dt * dpy;
    double d = ws[n] - 0.5 * dt * dpz * (coefw[n] * (double)impfl + (double)(1 - impfl));
    bcv_node<double>(M, c, k, n, ue, 1.0, a, b, d);
    uo[n] = a; vo[n] = b; wo[n] = d;
}

// div at the copies: group divergence, then as k_div
__global__ void k_cp_div(ColMesh M, CopyList CL, const double *__restrict__ ua, const double *__restrict__ va,
                         const double *__restrict__ wa, const double *__restrict__ vol,
                         const double *__restrict__ rh0, int iflg, double *__restrict__ rhs) {
    COPY_BEGIN
    double dx, dy, dz;
    if (iflg == -1)
        group_sum3<double>(M, mem, gs, [&](int cx, int kx, int x, double &a, double &b, double &d) {
            div3<double>(M, [&](int j, double &u, double &v, double &w) {
                const double r = rh0[j]; u = ua[j] * r; v = va[j] * r; w = wa[j] * r; }, cx, kx, x, a, b, d); },
            dx, dy, dz);
    else
        group_sum3<double>(M, mem, gs, [&](int cx, int kx, int x, double &a, double &b, double &d) {
            div3<double>(M, [&](int j, double &u, double &v, double &w) { u = ua[j]; v = va[j]; w = wa[j]; },
                         cx, kx, x, a, b, d); }, dx, dy, dz);
    (void)c; (void)k;
    const double v = vol[n];
    rhs[n] = (double)iflg * (dx / v + dy / v + dz / v) / rh0[n];
}

// velprd's advective predictor at the copies: group gradient, then as k_velprd_grad
__global__ void k_cp_velprd_grad(ColMesh M, CopyList CL, const double *__restrict__ ud, const double *__restrict__ vol,
                                 U3 U, double dt, double *__restrict__ u1) {
    COPY_BEGIN
    double gx, gy, gz;
    group_sum3<double>(M, mem, gs, [&](int cx, int kx, int x, double &a, double &b, double &d) {
        grad3<double>(M, ud, cx, kx, x, a, b, d); }, gx, gy, gz);
    (void)c; (void)k;
    const double v = vol[n];
    const double f1 = gx / v, f2 = gy / v, f3 = gz / v;
    u1[n] = ud[n] - dt * (U.u[0][n] * f1 + U.u[1][n] * f2 + U.u[2][n] * f3);
}

// ---------------------------------------------------------------- mpdatamper at the copies
// donor-cell sum of one node over its own faces, as in k_mp_donor (periodic form)
template <class T>
__device__ __forceinline__ double donor_partial(const ColMesh &M, const MpScratchT<T> &S, const double *psi, int c,
                                                int k, int n) {
    const double pn = psi[n];
    double arh2 = 0.;
    for_faces(M, c, k, n,
        [&](const Face &f) { return V4{(double)(f.vert ? S.aunv : S.aunh)[f.si], psi[f.j], 0., 0.}; },
        [&](const Face &f, const V4 &v) {
            const double aun = v.a;
            const double pa = f.sub ? v.b : pn, pb = f.sub ? pn : v.b;
            const double fl = pa * (0. > aun ? 0. : aun) + pb * (0. < aun ? 0. : aun);
            arh2 = f.sub ? arh2 - fl : arh2 + fl;
        });
    if (has_boundary(M, c, k)) arh2 = arh2 + 0. * 1.;
    return arh2;
}

template <class T>
__global__ void k_cp_mp_donor(ColMesh M, CopyList CL, MpScratchT<T> S, const double *__restrict__ psi,
                              T *__restrict__ psi1, MpUpdate U) {
    COPY_BEGIN
    (void)c; (void)k;
    double arh2 = 0.;
    for (int q = 0; q < gs; ++q) {
        const int x = mem[q], cx = x / M.L, kx = x - cx * M.L;
        const double a = donor_partial<T>(M, S, psi, cx, kx, x);
        arh2 = q == 0 ? a : arh2 + a;
    }
    const double p1 = psi[n] - arh2 * U.dt / U.vol[n] / U.rh0[n];
    psi1[n] = (T)p1;
    if (U.psi1d) U.psi1d[n] = p1;
}

// the gradient of psi1 at the copies (the FCT bounds of k_mp_grad_bounds stay, then k_cp_bounds)
template <class T>
__global__ void k_cp_mp_grad(ColMesh M, CopyList CL, const T *__restrict__ psi1, T *__restrict__ gx,
                             T *__restrict__ gy, T *__restrict__ gz) {
    COPY_BEGIN
    (void)c; (void)k;
    T ax, ay, az;
    group_sum3<T>(M, mem, gs, [&](int cx, int kx, int x, T &a, T &b, T &d) { grad3<T>(M, psi1, cx, kx, x, a, b, d); },
                  ax, ay, az);
    gx[n] = ax; gy[n] = ay; gz[n] = az;
}

template <class T> __device__ __forceinline__ T mx2(T a, T b) { return a > b ? a : b; }
template <class T> __device__ __forceinline__ T mn2(T a, T b) { return a < b ? a : b; }

// the FCT bounds over the periodic lists (ref.f:3821-3867), one thread per group, members in
// order, on the FP64 first-pass field; a corner's minima are taken over unkmx as in the reference
// (ref.f:3853-3866)
__global__ void k_cp_bounds(CopyList CL, const double *__restrict__ psi1, double *__restrict__ mx,
                            double *__restrict__ mn) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= CL.ngroups) return;
    const int32_t *m = CL.members + CL.grp[g];
    if (CL.grpsize[g] == 2) {
        const int i1 = m[0], i2 = m[1];
        const double p1 = psi1[i1], p2 = psi1[i2];
        mx[i1] = mx2(mx2(mx2(mx[i1], p1), p2), mx[i2]);
        mn[i1] = mn2(mn2(mn2(mn[i1], p1), p2), mn[i2]);
        mx[i2] = mx2(mx2(mx2(mx[i2], p1), p2), mx[i1]);
        mn[i2] = mn2(mn2(mn2(mn[i2], p1), p2), mn[i1]);
    } else {
        const double p1 = psi1[m[0]], p2 = psi1[m[1]], p3 = psi1[m[2]], p4 = psi1[m[3]];
        const double pmx = mx2(mx2(mx2(p1, p2), p3), p4), pmn = mn2(mn2(mn2(p1, p2), p3), p4);
        for (int q = 0; q < 4; ++q) {
            const double u = mx2(mx2(mx2(mx[m[0]], mx[m[1]]), mx[m[2]]), mx[m[3]]);
            mx[m[q]] = mx2(u, pmx);
            const double l = mn2(mn2(mn2(mx[m[0]], mx[m[1]]), mx[m[2]]), mx[m[3]]);
            mn[m[q]] = mn2(l, pmn);
        }
    }
}

// in/out sums of one node over its own faces, as in k_mp_cpcn
template <class T>
__device__ __forceinline__ void cpcn_partial(const ColMesh &M, const MpScratchT<T> &S, int c, int k, int n,
                                             double &rin, double &rout) {
    rin = 0.; rout = 0.;
    for_faces(M, c, k, n,
        [&](const Face &f) { return V4{(double)(f.vert ? S.Av : S.Ah)[f.si], 0., 0., 0.}; },
        [&](const Face &f, const V4 &v) {
            const double a = v.a;
            const double pp = 0. > a ? 0. : a, pn = -(0. < a ? 0. : a);
            if (!f.sub) { rin = rin + pn; rout = rout + pp; }
            else        { rin = rin + pp; rout = rout + pn; }
        });
}

template <class T>
__global__ void k_cp_mp_cpcn(ColMesh M, CopyList CL, MpScratchT<T> S, const double *__restrict__ psi1,
                             const double *__restrict__ mx, const double *__restrict__ mn,
                             const double *__restrict__ vol, const double *__restrict__ rh0, double dt,
                             double *__restrict__ cp, double *__restrict__ cn) {
    COPY_BEGIN
    (void)c; (void)k;
    double rin = 0., rout = 0.;
    for (int q = 0; q < gs; ++q) {
        const int x = mem[q], cx = x / M.L, kx = x - cx * M.L;
        double a, b;
        cpcn_partial<T>(M, S, cx, kx, x, a, b);
        rin = q == 0 ? a : rin + a;
        rout = q == 0 ? b : rout + b;
    }
    const double tol = 1.e-10;
    const double p = psi1[n], v = vol[n], r = rh0[n];
    cp[n] = (mx[n] - p) * v * r / (rin * dt + tol);
    cn[n] = (p - mn[n]) * v * r / (rout * dt + tol);
}

// limited second-pass sum of one node over its own faces, as in k_mp_pass2
template <class T>
__device__ __forceinline__ double pass2_partial(const ColMesh &M, const MpScratchT<T> &S, const double *cp,
                                                const double *cn, int c, int k, int n) {
    const double cpn = cp[n], cnn = cn[n];
    double arh2 = 0.;
    for_faces(M, c, k, n,
        [&](const Face &f) { return V4{(double)(f.vert ? S.Av : S.Ah)[f.si], cp[f.j], cn[f.j], 0.}; },
        [&](const Face &f, const V4 &v) {
            const double a = v.a;
            const double cpa = f.sub ? v.b : cpn, cna = f.sub ? v.c : cnn;
            const double cpb = f.sub ? cpn : v.b, cnb = f.sub ? cnn : v.c;
            const double lim = a > 0. ? a * tmin(tmin(1., cpb), cna) : a * tmin(tmin(1., cnb), cpa);
            arh2 = f.sub ? arh2 - lim : arh2 + lim;
        });
    if (has_boundary(M, c, k)) arh2 = arh2 + 0. * 1.;
    return arh2;
}

template <class T>
__global__ void k_cp_mp_pass2(ColMesh M, CopyList CL, MpScratchT<T> S, const T *__restrict__ psi1,
                              const double *__restrict__ cp, const double *__restrict__ cn, MpUpdate U,
                              double *__restrict__ psi2) {
    COPY_BEGIN
    (void)c; (void)k;
    double arh2 = 0.;
    for (int q = 0; q < gs; ++q) {
        const int x = mem[q], cx = x / M.L, kx = x - cx * M.L;
        const double a = pass2_partial<T>(M, S, cp, cn, cx, kx, x);
        arh2 = q == 0 ? a : arh2 + a;
    }
    const double p1 = U.psi1d ? U.psi1d[n] : (double)psi1[n];
    psi2[n] = p1 - arh2 * U.dt / U.vol[n] / U.rh0[n];
}

#undef COPY_BEGIN

}  // namespace mpgk

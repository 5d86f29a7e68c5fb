// MPDATA (mpdatamper, lippsLFroude_implgwopks3D_unstr3.f:3617-3941, and its open-boundary twin
// mpdatam, ref.f:3029-3311), the node loops of the
// time-step driver mpsolver (ref.f:285-463) and the per-step diagnostics (ref.f:1974-2170,
// ref.f:2847-2912) as device kernels.
//
// MPDATA per field, iord = 2 with the nonoscillatory option (ifct = 1):
//   k_aun            once per step: advective face flux aun = (U_a+U_b)/2 . S    (ref.f:3690-3693)
//   k_mp_donor       donor-cell pass and update psi1 = psi - dt*arh2/(vol*rh0)    (ref.f:3687-3747;
//                    with the open-boundary closure of mpdatam, ref.f:3085-3172)
//   k_mp_grad_bounds derivative(psi1) x3 and the FCT bounds mx/mn                 (ref.f:3755-3817)
//   k_mp_anti_{h,v}  antidiffusive face flux A (infinite-gauge form)              (ref.f:3760-3794)
//   k_mp_cpcn        in/out sums of A and the limiter ratios cp, cn               (ref.f:3871-3909)
//   k_mp_pass2       limited A, second pass and update                            (ref.f:3913-3931, 3681-3747)
// Faces are handled in canonical orientation (first end -> second end); every quantity that
// the reference computes for an edge stored the other way round is the exact negation of the
// canonical one, so the per-node sums equal the reference's bit for bit.
#pragma once

#include "kernels.cuh"

namespace mpgk {

// face arrays of MPDATA in the intermediate type T (double; float in mixed precision)
template <class T>
struct MpScratchT {
    T *aunh, *aunv;          // advective flux per face
    T *Ah, *Av;              // antidiffusive flux per face
    const int32_t *e2a, *e2b;
};
using MpScratch = MpScratchT<double>;

template <class T>
__device__ __forceinline__ T face_aun(const double *const *uuu, int a, int b, T sx, T sy, T sz) {
    return ((T)uuu[0][a] + (T)uuu[0][b]) * T(0.5) * sx + ((T)uuu[1][a] + (T)uuu[1][b]) * T(0.5) * sy
         + ((T)uuu[2][a] + (T)uuu[2][b]) * T(0.5) * sz;
}

struct U3 {
    const double *u[3];
};

// aun for horizontal faces (thread per (e,k)) and vertical faces (thread per node)
template <class T>
__global__ void k_aun(ColMesh M, MpScratchT<T> S, U3 U) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int nh = M.NE2 * M.L;
    if (t < nh) {
        const int e = t / M.L, k = t - e * M.L;
        const int a = S.e2a[e] * M.L + k, b = S.e2b[e] * M.L + k;
        T sx, sy, sz;
        FaceVec<T>::load(M, false, t, sx, sy, sz);
        S.aunh[t] = face_aun<T>(U.u, a, b, sx, sy, sz);
    } else if (t < nh + M.N) {
        const int n = t - nh;
        const int k = n % M.L;
        if (k + 1 < M.L) {
            T sx, sy, sz;
            FaceVec<T>::load(M, true, n, sx, sy, sz);
            S.aunv[n] = face_aun<T>(U.u, n, n + 1, sx, sy, sz);
        }
    }
}

template <class T>
__device__ __forceinline__ T face_val(const T *h, const T *v, int si, bool vert) {
    return vert ? v[si] : h[si];
}

__device__ __forceinline__ bool has_boundary(const ColMesh &M, int c, int k) {
    bool any = false;
    for_boundary(M, c, k, [&](const BEntry &) { any = true; });
    return any;
}

// inflow data of the open-boundary closure (mpdatam): the field's free-stream value afree(iflag),
// or the ambient ue per node for iflag = 1 (ref.f:3154-3155)
struct MpInflow {
    const double *ue;     // used when iflag == 1
    double afree;         // used otherwise
    int iflag;
};

// FP64 node work of both passes: psi_new = psi_old - arh2*dt/vol/rh0 with arh2 summed in FP64
// from the face fluxes (FP64, or FP32 in mixed precision, where psi1d keeps the first-pass field
// in FP64 beside its FP32 copy; null in FP64).  The donor fluxes use the FP64 field, and the FCT
// bounds, in/out sums and limiter ratios are FP64 too, so that the limiter's guarantees (sign and
// bounds of the field) hold for the FP64 values it updates, and its mass changes only by FP64
// round-off.
struct MpUpdate {
    double *psi1d;
    const double *vol, *rh0;
    double dt;
};

// donor-cell pass: fl = psi_a*max(0,aun) + psi_b*min(0,aun); a gets +fl, b gets -fl.
// OPEN selects mpdatam's first-pass boundary closure (ref.f:3143-3169): every boundary point
// of a type other than 11, 5 or 6 carries the flux aunbb1 = -divv that balances the node's face
// fluxes, donor-cell upwinded with the free-stream value on inflow.  mpdatamper adds zero there
// (ref.f:3732-3738).
template <class T, bool OPEN>
__global__ void k_mp_donor(ColMesh M, MpScratchT<T> S, const double *__restrict__ psi,
                           T *__restrict__ psi1, MpInflow in, MpUpdate U) {
    NODE_BEGIN
    const double pn = psi[n];
    double arh2 = 0., divv = 0.;
    for_faces(M, c, k, n,
        [&](const Face &f) { return V4{(double)(f.vert ? S.aunv : S.aunh)[f.si], psi[f.j], 0., 0.}; },
        [&](const Face &f, const V4 &v) {
            const double aun = v.a;
            const double pa = f.sub ? v.b : pn, pb = f.sub ? pn : v.b;
            const double fl = pa * (0. > aun ? 0. : aun) + pb * (0. < aun ? 0. : aun);
            arh2 = f.sub ? arh2 - fl : arh2 + fl;
            if (OPEN) divv = f.sub ? divv - aun : divv + aun;
        });
    if (OPEN) {
        for_boundary(M, c, k, [&](const BEntry &be) {
            const double aunbb1 = -divv;
            const double fin = in.iflag == 1 ? in.ue[n] : in.afree;
            double fl1 = fin * (0. < aunbb1 ? 0. : aunbb1) + pn * (0. > aunbb1 ? 0. : aunbb1);
            if (be.type == 11 || be.type == 5 || be.type == 6) fl1 = 0.;
            arh2 = arh2 + fl1 * 1.;
        });
    } else if (has_boundary(M, c, k)) {
        arh2 = arh2 + 0. * 1.;
    }
    const double p1 = pn - arh2 * U.dt / U.vol[n] / U.rh0[n];
    psi1[n] = (T)p1;
    if (U.psi1d) U.psi1d[n] = p1;
}

// gradient of psi1 (three derivative calls) and the neighbourhood max/min; OPEN adds the
// derivative's boundary closure of iper = 0 (mpdatam)
template <class T, bool OPEN>
__global__ void k_mp_grad_bounds(ColMesh M, const T *__restrict__ psi1, const double *__restrict__ psi1d,
                                 T *__restrict__ gx, T *__restrict__ gy, T *__restrict__ gz,
                                 double *__restrict__ mx, double *__restrict__ mn) {
    NODE_BEGIN
    // in mixed precision the bounds come from the FP64 first-pass field; in FP64 that field is
    // psi1 itself (decided at compile time: a pointer test per face cost the FP64 kernel a block
    // per SM in registers)
    constexpr bool BD = std::is_same<T, float>::value;
    const T pn = psi1[n];
    const double bn = BD ? psi1d[n] : (double)pn;
    T ax = 0., ay = 0., az = 0.;
    double hi = -1.e15, lo = 1.e15;
    for_faces(M, c, k, n,
        [&](const Face &f) {
            V4T<T> v;
            FaceVec<T>::load(M, f.vert, f.si, v.a, v.b, v.c);
            v.d = psi1[f.j];
            return v;
        },
        [&](const Face &f, const V4T<T> &v) {
            const T pj = v.d;
            const T u = (pn + pj) * T(0.5);
            const T tx = v.a * u, ty = v.b * u, tz = v.c * u;
            if (f.sub) { ax = ax - tx; ay = ay - ty; az = az - tz; }
            else       { ax = ax + tx; ay = ay + ty; az = az + tz; }
            const double bj = BD ? psi1d[f.j] : (double)pj;
            hi = hi > bn ? hi : bn;
            hi = hi > bj ? hi : bj;
            lo = lo < bn ? lo : bn;
            lo = lo < bj ? lo : bj;
        });
    if (OPEN) {                                         // derivative's closure, ref.f:4007-4014
        for_boundary(M, c, k, [&](const BEntry &be) {
            ax = ax + T(be.sbb[0]) * pn;
            ay = ay + T(be.sbb[1]) * pn;
            az = az + T(be.sbb[2]) * pn;
        });
    }
    gx[n] = ax; gy[n] = ay; gz[n] = az;
    mx[n] = hi; mn[n] = lo;
}

template <class T>
__device__ __forceinline__ T anti_flux(T aun, int a, int b, const T *psi1, const T *gx, const T *gy,
                                       const T *gz, const T *vol, const T *rh0, const double *const *uuu, T dt) {
    const T un = fabs(aun) * (psi1[b] - psi1[a]) * T(0.5);
    const T volt = T(0.5) * (vol[a] * rh0[a] + vol[b] * rh0[b]);
    const T dpdx = T(0.5) * (gx[a] + gx[b]) / volt;
    const T dpdy = T(0.5) * (gy[a] + gy[b]) / volt;
    const T dpdz = T(0.5) * (gz[a] + gz[b]) / volt;
    const T term = ((T)uuu[0][a] + (T)uuu[0][b]) * T(0.5) * dpdx + ((T)uuu[1][a] + (T)uuu[1][b]) * T(0.5) * dpdy
                 + ((T)uuu[2][a] + (T)uuu[2][b]) * T(0.5) * dpdz;
    return un - aun * term * dt * T(0.5);
}

template <class T>
struct AntiArgs {
    const T *psi1, *gx, *gy, *gz, *vol, *rh0;
    U3 U;
    T dt;
};

template <class T>
__global__ void k_mp_anti(ColMesh M, MpScratchT<T> S, AntiArgs<T> A) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int nh = M.NE2 * M.L;
    if (t < nh) {
        const int e = t / M.L, k = t - e * M.L;
        const int a = S.e2a[e] * M.L + k, b = S.e2b[e] * M.L + k;
        S.Ah[t] = anti_flux<T>(S.aunh[t], a, b, A.psi1, A.gx, A.gy, A.gz, A.vol, A.rh0, A.U.u, A.dt);
    } else if (t < nh + M.N) {
        const int n = t - nh;
        const int k = n % M.L;
        if (k + 1 < M.L)
            S.Av[n] = anti_flux<T>(S.aunv[n], n, n + 1, A.psi1, A.gx, A.gy, A.gz, A.vol, A.rh0, A.U.u, A.dt);
    }
}

// in/out sums and the limiter ratios, in FP64 from the face fluxes A (FP32 in mixed precision)
template <class T>
__global__ void k_mp_cpcn(ColMesh M, MpScratchT<T> S, const double *__restrict__ psi1,
                          const double *__restrict__ mx, const double *__restrict__ mn,
                          const double *__restrict__ vol, const double *__restrict__ rh0, double dt,
                          double *__restrict__ cp, double *__restrict__ cn) {
    NODE_BEGIN
    double rin = 0., rout = 0.;
    for_faces(M, c, k, n,
        [&](const Face &f) { return V4{(double)(f.vert ? S.Av : S.Ah)[f.si], 0., 0., 0.}; },
        [&](const Face &f, const V4 &v) {
            const double a = v.a;
            const double pp = 0. > a ? 0. : a, pn = -(0. < a ? 0. : a);
            if (!f.sub) { rin = rin + pn; rout = rout + pp; }
            else        { rin = rin + pp; rout = rout + pn; }
        });
    const double tol = 1.e-10;
    const double p = psi1[n], v = vol[n], r = rh0[n];
    cp[n] = (mx[n] - p) * v * r / (rin * dt + tol);
    cn[n] = (p - mn[n]) * v * r / (rout * dt + tol);
}

// limited antidiffusive flux and the second pass
template <class T>
__device__ __forceinline__ T tmin(T a, T b) { return a < b ? a : b; }

template <class T>
__global__ void k_mp_pass2(ColMesh M, MpScratchT<T> S, const T *__restrict__ psi1,
                           const double *__restrict__ cp, const double *__restrict__ cn, MpUpdate U,
                           double *__restrict__ psi2) {
    NODE_BEGIN
    const double cpn = cp[n], cnn = cn[n];
    double arh2 = 0.;
    for_faces(M, c, k, n,
        [&](const Face &f) { return V4{(double)(f.vert ? S.Av : S.Ah)[f.si], cp[f.j], cn[f.j], 0.}; },
        [&](const Face &f, const V4 &v) {
            const double a = v.a;
            // canonical ends: first = this node unless sub
            const double cpa = f.sub ? v.b : cpn, cna = f.sub ? v.c : cnn;
            const double cpb = f.sub ? cpn : v.b, cnb = f.sub ? cnn : v.c;
            const double lim = a > 0. ? a * tmin(tmin(1., cpb), cna) : a * tmin(tmin(1., cnb), cpa);
            arh2 = f.sub ? arh2 - lim : arh2 + lim;
        });
    if (has_boundary(M, c, k)) arh2 = arh2 + 0. * 1.;
    const double p1 = U.psi1d ? U.psi1d[n] : (double)psi1[n];
    psi2[n] = p1 - arh2 * U.dt / U.vol[n] / U.rh0[n];
}

// ------------------------------------------------------------------------------ mpsolver node loops
struct Fields {
    double *unk[4], *frc[4], *uuu[3], *uuu0[3], *ud[3], *unk1[3];
    const double *rh0, *th0, *the, *dthedz, *coefw, *alpha, *ue, *ve;
};

// ref.f:290-301
__global__ void k_half_forcing(int N, Fields F, double dt, int implgw) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    for (int q = 0; q < 3; ++q) F.uuu0[q][n] = F.uuu[q][n];
    for (int q = 0; q < 4; ++q) F.unk[q][n] = F.unk[q][n] + 0.5 * F.frc[q][n] * dt;
    if (implgw == 0) F.unk[3][n] = F.unk[3][n] + F.the[n];
}

// ref.f:323-359 (isfera = 0 branch; fcr2/fcr3 are the Coriolis terms, zero when icorio = 0)
__global__ void k_explicit_forcing(int N, Fields F, double dt, double g, double fcr2, double fcr3,
                                   double ideep, int implgw, int mtri) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    double frm1 = 0., frm2 = 0., frm3 = 0.;
    if (mtri == 1 && implgw == 0) F.unk[3][n] = F.unk[3][n] - F.the[n];
    const double we = 0.;
    const double ud0 = F.ud[0][n], ud1 = F.ud[1][n], ud2 = F.ud[2][n];
    const double ue = F.ue[n], ve = F.ve[n], al = F.alpha[n];
    frm1 = frm1 + fcr3 * (ud1 - ve) - fcr2 * (ud2 - we) * ideep - al * (ud0 - ue);
    frm2 = frm2 - fcr3 * (ud0 - ue) - al * (ud1 - ve);
    frm3 = frm3 + fcr2 * (ud0 - ue) * ideep - al * ud2 + g * F.unk[3][n] / F.th0[n];
    const double f0 = F.unk[0][n] + 0.5 * dt * frm1;
    const double f1 = F.unk[1][n] + 0.5 * dt * frm2;
    const double f2 = (F.unk[2][n] + 0.5 * dt * frm3) * F.coefw[n];
    F.frc[0][n] = f0; F.frc[1][n] = f1; F.frc[2][n] = f2;
    F.unk1[0][n] = f0 / (1.0 * 1.0);
    F.unk1[1][n] = f1 / 1.0;
    F.unk1[2][n] = f2;
}

// ref.f:367-383
__global__ void k_post_solve(int N, Fields F, double dt, double g, int last) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    const double ud0 = F.uuu[0][n] * 1.0 * 1.0, ud1 = F.uuu[1][n] * 1.0, ud2 = F.uuu[2][n];
    F.ud[0][n] = ud0; F.ud[1][n] = ud1; F.ud[2][n] = ud2;
    if (!last) return;
    F.frc[0][n] = (ud0 - F.frc[0][n]) * 2. / dt;
    F.frc[1][n] = (ud1 - F.frc[1][n]) * 2. / dt;
    const double frc33 = F.frc[2][n] / F.coefw[n] - (g * F.unk[3][n] / F.th0[n]) * 0.5 * dt;
    F.frc[2][n] = (ud2 - frc33) * 2. / dt;
    F.unk[0][n] = ud0; F.unk[1][n] = ud1; F.unk[2][n] = ud2;
    const double f3 = -ud2 * F.dthedz[n];
    F.frc[3][n] = f3;
    F.unk[3][n] = F.unk[3][n] + 0.5 * dt * f3;
}

// ref.f:387-439 (iblatt = 0, itraj = 0)
__global__ void k_extrapolate(int N, Fields F, double fcr2, double fcr3, double ideep, int itraj) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    const double u0 = F.unk[0][n], u1 = F.unk[1][n], u2 = F.unk[2][n], u3 = F.unk[3][n];
    const double ue = F.ue[n], ve = F.ve[n], al = F.alpha[n];
    double frm1 = 0., frm2 = 0., frm3 = 0.;
    frm1 = frm1 + fcr3 * (u1 - ve) - fcr2 * (u2 - 0.) * ideep - al * (u0 - ue);
    frm2 = frm2 - fcr3 * (u0 - ue) - al * (u1 - ve);
    frm3 = frm3 + fcr2 * (u0 - ue) * ideep - al * (u2);
    const double frm4 = -al * (u3);
    F.frc[0][n] = F.frc[0][n] + frm1;
    F.frc[1][n] = F.frc[1][n] + frm2;
    F.frc[2][n] = F.frc[2][n] + frm3;
    F.frc[3][n] = F.frc[3][n] + frm4;
    if (itraj != 0) return;                       // velprd follows (ref.f:441-442)
    const double r = F.rh0[n];
    double o[3];
    for (int q = 0; q < 3; ++q) {
        o[q] = F.uuu0[q][n];
        F.uuu[q][n] = 1.5 * F.uuu[q][n] * r - 0.5 * o[q];
    }
    const double rhoi = 1. / r;
    o[0] = o[0] * rhoi * 1.0 * 1.0;
    o[1] = o[1] * rhoi * 1.0;
    o[2] = o[2] * rhoi;
    F.uuu0[0][n] = o[0]; F.uuu0[1][n] = o[1]; F.uuu0[2][n] = o[2];
    F.ud[0][n] = 2. * u0 - o[0];
    F.ud[1][n] = 2. * u1 - o[1];
    F.ud[2][n] = 2. * u2 - o[2];
}

// set-up: ambient state (ref.f:198-206) and momentum (ref.f:230-266)
__global__ void k_setup_ambient(int N, Fields F, double *prpot, double *unk1_3) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    F.unk[0][n] = F.ue[n];
    F.unk[1][n] = F.ve[n];
    F.unk[2][n] = 0.2 * F.frc[0][n];
    F.unk[3][n] = 0. + 0.001 * F.frc[0][n];
    F.unk1[0][n] = F.unk[0][n] / (1.0 * 1.0);
    F.unk1[1][n] = F.unk[1][n] / 1.0;
    F.unk1[2][n] = F.unk[2][n];
    unk1_3[n] = 0.;
    prpot[n] = 0.;
}

__global__ void k_setup_post(int N, Fields F, double *prpot, int itraj) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    for (int q = 0; q < 3; ++q) F.uuu[q][n] = F.unk[q][n];
    F.unk[0][n] = F.unk[0][n] * 1.0 * 1.0;
    F.unk[1][n] = F.unk[1][n] * 1.0;
    prpot[n] = 0.;
    for (int q = 0; q < 4; ++q) F.frc[q][n] = 0.;
    if (itraj != 0) return;                       // velprd follows (ref.f:267-268)
    const double r = F.rh0[n];
    for (int q = 0; q < 3; ++q) {
        F.uuu[q][n] = F.uuu[q][n] * r;
        F.ud[q][n] = F.unk[q][n];
    }
}

// velprd (ref.f:4448-4528), isfera = 0 (gmm = cosa = 1):
// unkdash = unk + dt frc (ref.f:4461-4465)
__global__ void k_velprd_pre(int N, Fields F, double dt) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    for (int q = 0; q < 3; ++q) F.ud[q][n] = F.unk[q][n] + dt * F.frc[q][n];
}
// uuu1(:,q) = unkdash(:,q) - dt (uuu . grad unkdash(:,q)) with the gradient / vol (ref.f:4466-4505)
__global__ void GATHER_BOUNDS k_velprd_grad(ColMesh M, const double *__restrict__ ud, const double *__restrict__ vol,
                                            U3 U, double dt, double *__restrict__ u1) {
    NODE_BEGIN
    double gx, gy, gz;
    grad3<double>(M, ud, c, k, n, gx, gy, gz);
    const double v = vol[n];
    const double f1 = gx / v, f2 = gy / v, f3 = gz / v;
    u1[n] = ud[n] - dt * (U.u[0][n] * f1 + U.u[1][n] * f2 + U.u[2][n] * f3);
}
// advective velocity at n+1/2 and the low-order solution at n+1 (ref.f:4517-4526)
__global__ void k_velprd_post(int N, Fields F, const double *__restrict__ f1, const double *__restrict__ f2,
                              const double *__restrict__ f3) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    const double r = F.rh0[n], ff[3] = {f1[n], f2[n], f3[n]};
    for (int q = 0; q < 3; ++q) {
        F.uuu[q][n] = (F.uuu[q][n] + ff[q]) * 0.5 * r;
        F.ud[q][n] = ff[q];
    }
}

// courant(uuu, cour, iflag) node part (ref.f:1994-2069): sum of |aun|/rhav over the faces
__global__ void k_courant(ColMesh M, U3 U, const double *__restrict__ rh0, const double *__restrict__ vol,
                          double dt, int iflag, double *__restrict__ cour) {
    NODE_BEGIN
    const double un0 = U.u[0][n], un1 = U.u[1][n], un2 = U.u[2][n], rn = rh0[n];
    double s = 0.;
    for_faces(M, c, k, n,
        [&](const Face &f) {
            V6 v;
            v.a = __ldg(spick(M, 0, f.vert) + f.si);
            v.b = __ldg(spick(M, 1, f.vert) + f.si);
            v.c = __ldg(spick(M, 2, f.vert) + f.si);
            v.d = U.u[0][f.j]; v.e = U.u[1][f.j]; v.f = U.u[2][f.j];
            return v;
        },
        [&](const Face &f, const V6 &v) {
            const double rhav = 0.5 * (rn + rh0[f.j]);
            // (U_a + U_b): the sum is symmetric, so the order of the ends does not matter
            double aun = (un0 + v.d) * 0.5 * v.a + (un1 + v.e) * 0.5 * v.b + (un2 + v.f) * 0.5 * v.c;
            aun = aun / rhav;
            if (iflag == 1) s = s + fabs(aun);
            else if (iflag == 2) s = f.sub ? s - aun : s + aun;
            else s = f.sub ? s - amin(0., aun) : s + amax(0., aun);
        });
    if (M.iper != 2) {
        for_boundary(M, c, k, [&](const BEntry &be) {
            double aun = un0 * be.sbb[0] + un1 * be.sbb[1] + un2 * be.sbb[2];
            aun = aun / rn;
            if (iflag == 1) s = s + fabs(aun);
            else if (iflag == 2) s = s + aun;
            else s = s + amax(0., aun);
        });
    }
    cour[n] = s * dt / vol[n] / rn;
}

}  // namespace mpgk

// Multigrid V-cycle of precon (mg_flag = 1, ref.f:618-748): the transfer kernels between a mesh
// and the next coarser one.  The coarse operators are laplc on the coarse meshes (laplc_c,
// laplc_cc: ref.f:1356-1533), run by handles of their own.
//
// Every array here is in the internal (column-layout) order of its mesh.  `match[ic]` is the
// finer-mesh node of coarse node ic; `nbp/nbl` are the finer mesh's neighbour lists in the order
// of neigh_definition (ref.f:2726-2767); `bugnb[k]` is the finer mesh's internal node for the
// reference node number k+1, which is what the reference reads when it takes the neighbour loop
// counter as a node number (ref.f:813-817, 911-915).
#pragma once

#include "kernels.cuh"

namespace mpgk {

constexpr double kMgUnset = -99999.;      // prolongation_unstr's marker for a node without a value

// restriction_unstr (ref.f:757-824): sc[ic] = sum over the neighbours j of ip = match[ic] of
// (s[ip] + s[j]) / 2, divided by the neighbour count; added in list order
__global__ void k_mg_restrict(int Nc, const int32_t *__restrict__ match, const int32_t *__restrict__ nbp,
                              const int32_t *__restrict__ nbl, const int32_t *__restrict__ bugnb, int bugs,
                              const double *__restrict__ s, double *__restrict__ sc) {
    const int ic = blockIdx.x * blockDim.x + threadIdx.x;
    if (ic >= Nc) return;
    const int ip = match[ic];
    const int b = nbp[ip], nn = nbp[ip + 1] - b;
    const double si = s[ip];
    double acc = 0.;
    for (int k = 0; k < nn; ++k) {
        const int j = bugs ? bugnb[k] : nbl[b + k];
        acc = acc + (si + s[j]) / 2.;
    }
    sc[ic] = acc / (double)nn;
}

// prolongation_unstr (ref.f:828-951): every fine node unset, then the matched ones take their
// coarse value
__global__ void k_mg_prolong_init(int N, double *__restrict__ s, double *__restrict__ aux, uint8_t *__restrict__ flag) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    s[i] = 0.;
    aux[i] = kMgUnset;
    flag[i] = 0;
}
__global__ void k_mg_inject(int Nc, const int32_t *__restrict__ match, const double *__restrict__ sc,
                            double *__restrict__ s, double *__restrict__ aux) {
    const int ic = blockIdx.x * blockDim.x + threadIdx.x;
    if (ic >= Nc) return;
    const int ip = match[ic];
    s[ip] = sc[ic];
    aux[ip] = sc[ic];
}
// one filling pass: an unset node takes the mean of its neighbours that were set before this
// pass (aux is updated only between passes, by k_mg_commit)
__global__ void k_mg_fill(int N, const int32_t *__restrict__ nbp, const int32_t *__restrict__ nbl,
                          const int32_t *__restrict__ bugnb, int bugs, const double *__restrict__ aux,
                          double *__restrict__ s, uint8_t *__restrict__ flag) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N || aux[i] != kMgUnset) return;
    const int b = nbp[i], nn = nbp[i + 1] - b;
    double acc = s[i], filled = 0.;
    for (int k = 0; k < nn; ++k) {
        const int j = bugs ? bugnb[k] : nbl[b + k];
        if (aux[j] != kMgUnset) {
            acc = acc + s[j];
            filled = filled + 1.;
        }
    }
    if (filled != 0.) {
        s[i] = acc / filled;
        flag[i] = 1;
    }
}
__global__ void k_mg_commit(int N, const double *__restrict__ s, double *__restrict__ aux, uint8_t *__restrict__ flag) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N || !flag[i]) return;
    aux[i] = s[i];
    flag[i] = 0;
}

__device__ __forceinline__ double mg_pstep(int sm_flag1, double beta, double d) {
    double ps = 0.;
    if (sm_flag1 == 1) ps = (-1.) / d;
    else if (sm_flag1 == 2) ps = beta;
    else if (sm_flag1 == 3) ps = beta / (1. - d * beta);
    return ps;
}
// first relaxation from zero on a coarser mesh: the coarse mesh's p_c = -(omega*pstep*rrhs)
// (ref.f:675-677); the coarsest's p_cc = -(rrhs*pstep*omega) (ref.f:702-704)
__global__ void k_mg_first(int N, int coarsest, int sm_flag1, double omega, double beta, const double *__restrict__ d,
                           const double *__restrict__ rrhs, double *__restrict__ p) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const double ps = mg_pstep(sm_flag1, beta, d[i]);
    p[i] = coarsest ? -(rrhs[i] * ps * omega) : -(omega * ps * rrhs[i]);
}
__global__ void k_add(int N, const double *__restrict__ e, double *__restrict__ p) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) p[i] = p[i] + e[i];
}

}  // namespace mpgk

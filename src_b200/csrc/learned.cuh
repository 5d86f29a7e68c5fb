// Learned correction of the vertical-line preconditioner: an edge message-passing network
// (3 layers, 32 hidden channels) evaluated and trained with the kernels below.  No counterpart
// exists in the reference; it plugs in where gcrk calls precon (ref.f:1836, ref.f:1898).
//
//   z      = M^{-1} r                        (vertical-line Thomas solve, FP64)
//   x_n    = [ r_n/s, z_n |b_n|/s, ln(Dv_n/Dh_n)/8, bnd_n ]      s = max|r|, b = line diagonal
//   h0     = relu(W_in x + b_in)                                  4 -> 32, FP32 FMA
//   h_l    = relu(W_l [h_{l-1}; A_h(h_{l-1}); A_v(h_{l-1})] + b_l), l = 1..3   96 -> 32
//   A_*(h)_n = sum over horizontal (vertical) faces of (T_nj / D_n) (h_j - h_n)
//   y      = w_out . h3 + b_out,   q = z + y s / |b|                             (returned)
//
// T_nj is the face coupling 0.5 dt |S|^2 rho_f / vol_f of the face (n, j), D_n its sum over the
// node's horizontal (vertical) faces.  Activations are stored in BF16 (node-major, 32 channels =
// 64 bytes per node; in the column layout a neighbour column's rows are one contiguous block).
// Forward: one CTA per column, the 96 -> 32 transforms on the tensor cores with tcgen05.mma
// (BF16 operands, FP32 accumulation in tensor memory), the input layer fused into the first
// layer and the output layer into the last.  Backward (training only): warp-level BF16 mma
// (wmma) with the weight gradients reduced deterministically (per-block partials folded in a
// fixed order).
#pragma once

#include <cuda_bf16.h>
#include <mma.h>

#include "kernels.cuh"

namespace mpgk {
namespace nn {

constexpr int C = 32;            // hidden channels
constexpr int FIN = 4;           // input features
constexpr int K3 = 3 * C;        // layer input width
constexpr int NL = 3;            // message-passing layers
// parameter vector layout (FP32 master copy)
constexpr int OFF_WIN = 0;                     // [C][FIN]
constexpr int OFF_BIN = OFF_WIN + C * FIN;     // [C]
constexpr int OFF_L0 = OFF_BIN + C;            // per layer: W [C][K3], b [C]
constexpr int LSTRIDE = C * K3 + C;
constexpr int OFF_WOUT = OFF_L0 + NL * LSTRIDE;  // [C]
constexpr int OFF_BOUT = OFF_WOUT + C;           // [1]
constexpr int NPARAM = OFF_BOUT + 1;             // 9505

constexpr int WARPS = 4;                          // warps per block in k_nn_dw
constexpr int TILE = 32;                          // nodes per warp tile of the backward kernels
constexpr int BWARPS = 2;                         // warps per block in k_nn_layer_bwd

struct Geom {
    const float *Th;        // [NE2*L] horizontal face coupling
    const float *Tv;        // [N] vertical face coupling (face (c,k)->(c,k+1) at c*L+k)
    const float *iDh, *iDv; // [N] 1/sum of couplings (0 when the node has no such face)
    const float *bdiag;     // [N] |b| of the line matrix (impfl = 1)
    const float *feat2;     // [N] ln(Dv/Dh)/8
    const float *bnd;       // [N] 1 at boundary nodes
};

__device__ __forceinline__ float face_T(const ColMesh &M, const Geom &G, const Face &f) {
    return f.vert ? G.Tv[f.si] : G.Th[f.si];
}

// 8 consecutive BF16 channels as one 16-byte load
struct alignas(16) B8 { __nv_bfloat162 v[4]; };
// what the face loops load per face (namespace-scope types: a class declared inside the
// loading lambda came back with a wrong layout from for_faces)
struct RowF { float4 lo, hi; float t; };

__device__ __forceinline__ void b8_to_f(const B8 &b, float *f) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float2 t = __bfloat1622float2(b.v[i]);
        f[2 * i] = t.x;
        f[2 * i + 1] = t.y;
    }
}

// ------------------------------------------------------------------ tensor-core operands
// The layer transform X W^T (X: 128 rows x 96 BF16, W: 32 x 96 BF16) runs as six tcgen05.mma
// (kind::f16, K = 16 each) with the FP32 accumulator in tensor memory (32 columns).  Both operands
// sit in shared memory in the canonical K-major layout without swizzle: 8x8 BF16 core matrices of
// 128 contiguous bytes, core (row group g, K chunk kc) at (kc*groups + g)*128 bytes.
constexpr int TCM = 128;                    // rows per tile = TMEM lanes = UMMA M
constexpr int TC_KC = K3 / 8;               // 12 K chunks of 8 channels
constexpr uint32_t TC_A_LBO = 16 * 128;     // A: next K chunk (16 row groups of 128 B)
constexpr uint32_t TC_B_LBO = 4 * 128;      // B: next K chunk (4 row groups)
constexpr uint32_t TC_SBO = 128;            // next 8-row group
constexpr uint32_t TC_TMEM_COLS = 32;
constexpr long long TC_SPIN_MAX = 1ll << 22;  // bound on the mbarrier wait (then the output is NaN)

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Self-test of the bounded wait: one CTA arms an mbarrier for a single arrival.  With `arrive`,
// thread 0 arrives and the wait completes; without, nothing arrives and every thread gives up
// after `limit` polls.  status[0] = 1 when all threads saw the phase complete, 0 when they gave up.
__global__ void k_mbar_selftest(int arrive, long long limit, int *status) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&bar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (arrive && threadIdx.x == 0) {
        uint64_t state;
        asm volatile("mbarrier.arrive.shared::cta.b64 %0, [%1];" : "=l"(state) : "r"(smem_u32(&bar)) : "memory");
    }
    const bool done = mbar_wait_bounded(&bar, 0u, limit);
    const int all = __syncthreads_and(done);
    if (threadIdx.x == 0) status[0] = all;
}

// shared-memory matrix descriptor: canonical K-major layout without swizzle
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// instruction descriptor: D F32, A and B BF16, both K-major, N = 32, M = 128
constexpr uint32_t TC_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(C >> 3) << 17) |
                              ((uint32_t)(TCM >> 4) << 24);

__device__ __forceinline__ uint32_t tc_core_off(int row, int kc, int groups) {
    return (uint32_t)((kc * groups + (row >> 3)) * 128 + (row & 7) * 16);
}

// ------------------------------------------------------------------ column layer (forward)
// One CTA of 4 warps per column (L <= 128 levels = one UMMA tile of M = 128 rows; rows L..127
// stay zero).  Warp w owns channel octet w (8 channels) of rows k = lane, lane+32, ... (NS
// slots), so for every horizontal face of the column (uniform for the CTA) a warp reads 16 bytes
// of 32 consecutive neighbour rows — one contiguous block of the neighbour column — and keeps
// NS such loads per face in flight.  The column's own rows are staged in shared memory, which
// also serves the vertical aggregation (its two faces join adjacent rows).  The 96-wide inputs
// go to shared memory in the canonical K-major operand layout, one thread issues the
// 128x32x96 BF16 product (tcgen05.mma, FP32 accumulator in tensor memory), and in the epilogue
// warp w reads TMEM lanes 32w..32w+31 (rows 32w + lane), all 32 columns: each thread holds a
// whole output row.
//   FIRST: the layer input h0 = relu(W_in x + b_in) is computed on the fly from the node
//          features x (X0, FP32 [N][4]) of the column and of each neighbour;
//   LAST:  the epilogue applies the output layer, y = w_out . h3 + b_out, q = z + y s / |b|,
//          instead of storing h3 (kept only when training).
// Training keeps H (h0 with FIRST, the layer output), Xs (the layer input rows) and Y.
constexpr int COL_THREADS = 128;
constexpr int COL_MAXL = 128;

template <int NS, bool FIRST, bool LAST>
__global__ void __launch_bounds__(COL_THREADS)
k_nn_col(ColMesh M, Geom G, const __nv_bfloat16 *__restrict__ Hin, const float *__restrict__ X0,
         const __nv_bfloat16 *__restrict__ Wbf, const float *__restrict__ prm, int layer,
         const double *__restrict__ z, const double *__restrict__ sc,
         __nv_bfloat16 *__restrict__ Hout, double *__restrict__ qd, float *__restrict__ qf,
         __nv_bfloat16 *__restrict__ Hkeep0, __nv_bfloat16 *__restrict__ Xs, float *__restrict__ Y,
         int *__restrict__ err) {
    __shared__ __align__(1024) uint8_t sA[TCM * K3 * 2];          // 24 KB operand tile
    __shared__ __align__(1024) uint8_t sB[C * K3 * 2];            // 6 KB weights
    __shared__ __align__(16) __nv_bfloat16 sH[COL_MAXL * C];      // own rows (8 KB)
    __shared__ float sBias[C], sWin[C * FIN + C], sWout[C + 1];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_base;
    const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
    const int L = M.L;
    const float *bias = prm + OFF_L0 + layer * LSTRIDE + C * K3;
    for (int i = tid; i < C * TC_KC; i += COL_THREADS) {
        const int n = i / TC_KC, kc = i - n * TC_KC;
        *reinterpret_cast<uint4 *>(sB + tc_core_off(n, kc, C / 8)) =
            *reinterpret_cast<const uint4 *>(Wbf + (size_t)n * K3 + kc * 8);
    }
    // rows L..127 of the operand tile are zero for every column
    for (int i = tid; i < TCM * TC_KC; i += COL_THREADS) {
        const int row = i / TC_KC, kc = i - row * TC_KC;
        if (row >= L) *reinterpret_cast<uint4 *>(sA + tc_core_off(row, kc, TCM / 8)) = make_uint4(0, 0, 0, 0);
    }
    if (tid < C) sBias[tid] = bias[tid];
    if (FIRST) for (int i = tid; i < C * FIN + C; i += COL_THREADS) sWin[i] = prm[OFF_WIN + i];
    if (LAST && tid <= C) sWout[tid] = prm[OFF_WOUT + tid];
    if (w == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(&tmem_base)), "r"(TC_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&bar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base;
    const uint32_t aBase = smem_u32(sA), bBase = smem_u32(sB);
    uint32_t phase = 0;
    bool ok = true;
    // the first layer's input rows: h0 = bf16(relu(W_in x + b_in)), channels 8w..8w+7
    auto h0_row = [&](const float4 x, float *o) {
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int c = 8 * w + i;
            float u = sWin[C * FIN + c] + sWin[c * FIN + 0] * x.x + sWin[c * FIN + 1] * x.y +
                      sWin[c * FIN + 2] * x.z + sWin[c * FIN + 3] * x.w;
            o[i] = __bfloat162float(__float2bfloat16(u > 0.f ? u : 0.f));
        }
    };
    for (int c = blockIdx.x; c < M.NC && ok; c += gridDim.x) {
        const int base = c * L;
        // ---- own rows (octet w) into sH
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            const int k = lane + 32 * s;
            if (k < L) {
                B8 v;
                if (FIRST) {
                    float o[8];
                    h0_row(*reinterpret_cast<const float4 *>(X0 + (size_t)(base + k) * FIN), o);
#pragma unroll
                    for (int i = 0; i < 4; ++i) v.v[i] = __floats2bfloat162_rn(o[2 * i], o[2 * i + 1]);
                    if (Hkeep0) *reinterpret_cast<B8 *>(Hkeep0 + (size_t)(base + k) * C + 8 * w) = v;
                } else {
                    v = *reinterpret_cast<const B8 *>(Hin + (size_t)(base + k) * C + 8 * w);
                }
                *reinterpret_cast<B8 *>(sH + k * C + 8 * w) = v;
            }
        }
        // ---- horizontal aggregation: ah = sum_f w_f h_j, wsum = sum_f w_f
        float ah[NS][8], wsum[NS], ih[NS];
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            const int k = lane + 32 * s;
            ih[s] = k < L ? G.iDh[base + k] : 0.f;
            wsum[s] = 0.f;
#pragma unroll
            for (int i = 0; i < 8; ++i) ah[s][i] = 0.f;
        }
        const int beg = __ldg(&M.cptr[c]), end = __ldg(&M.cptr[c + 1]);
        for (int j = beg; j < end; ++j) {
            const int2 en = __ldg(&M.cadj[j]);
            if (en.x < 0) continue;                      // vertical faces: below, from sH
            const int e = en.x >> 1, nb = en.y * L;
            uint4 v[NS];
            float t[NS];
#pragma unroll
            for (int s = 0; s < NS; ++s) {
                const int k = lane + 32 * s;
                if (k < L) {
                    if (FIRST) v[s] = *reinterpret_cast<const uint4 *>(X0 + (size_t)(nb + k) * FIN);
                    else v[s] = *reinterpret_cast<const uint4 *>(Hin + (size_t)(nb + k) * C + 8 * w);
                    t[s] = G.Th[(size_t)e * L + k];
                }
            }
#pragma unroll
            for (int s = 0; s < NS; ++s) {
                const int k = lane + 32 * s;
                if (k >= L) continue;
                float hj[8];
                if (FIRST) h0_row(*reinterpret_cast<const float4 *>(&v[s]), hj);
                else b8_to_f(*reinterpret_cast<const B8 *>(&v[s]), hj);
                const float wt = t[s] * ih[s];
                wsum[s] += wt;
#pragma unroll
                for (int i = 0; i < 8; ++i) ah[s][i] += wt * hj[i];
            }
        }
        __syncwarp();
        // ---- operand rows: [h ; ah - wsum h ; av] for octet w
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            const int k = lane + 32 * s;
            if (k >= L) continue;
            const int n = base + k;
            float hs[8], av[8];
            b8_to_f(*reinterpret_cast<const B8 *>(sH + k * C + 8 * w), hs);
#pragma unroll
            for (int i = 0; i < 8; ++i) av[i] = 0.f;
            const float iv = G.iDv[n];
            float wv = 0.f;
            if (k > 0) {
                float hb[8];
                b8_to_f(*reinterpret_cast<const B8 *>(sH + (k - 1) * C + 8 * w), hb);
                const float wt = G.Tv[n - 1] * iv;
                wv += wt;
#pragma unroll
                for (int i = 0; i < 8; ++i) av[i] += wt * hb[i];
            }
            if (k + 1 < L) {
                float ha[8];
                b8_to_f(*reinterpret_cast<const B8 *>(sH + (k + 1) * C + 8 * w), ha);
                const float wt = G.Tv[n] * iv;
                wv += wt;
#pragma unroll
                for (int i = 0; i < 8; ++i) av[i] += wt * ha[i];
            }
            B8 o[3];
            o[0] = *reinterpret_cast<const B8 *>(sH + k * C + 8 * w);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                o[1].v[i] = __floats2bfloat162_rn(ah[s][2 * i] - wsum[s] * hs[2 * i],
                                                  ah[s][2 * i + 1] - wsum[s] * hs[2 * i + 1]);
                o[2].v[i] = __floats2bfloat162_rn(av[2 * i] - wv * hs[2 * i], av[2 * i + 1] - wv * hs[2 * i + 1]);
            }
#pragma unroll
            for (int part = 0; part < 3; ++part) {
                const int kc = 4 * part + w;
                *reinterpret_cast<B8 *>(sA + tc_core_off(k, kc, TCM / 8)) = o[part];
                if (Xs) *reinterpret_cast<B8 *>(Xs + (size_t)n * K3 + 8 * kc) = o[part];
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int st = 0; st < K3 / 16; ++st) {
                const uint64_t ad = umma_desc(aBase + 2 * st * TC_A_LBO, TC_A_LBO, TC_SBO);
                const uint64_t bd = umma_desc(bBase + 2 * st * TC_B_LBO, TC_B_LBO, TC_SBO);
                const uint32_t acc = st > 0 ? 1u : 0u;
                asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                             "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
                             :: "r"(tmem), "l"(ad), "l"(bd), "r"(TC_IDESC), "r"(acc));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         :: "r"(smem_u32(&bar)) : "memory");
        }
        {
            const bool done = mbar_wait_bounded(&bar, phase, TC_SPIN_MAX);
            if (__syncthreads_or(!done)) {
                ok = false;
                if (tid == 0) atomicExch(err, 1);
            }
        }
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        // ---- epilogue: row k = 32w + lane, 32 channels.  After a wait that gave up (ok is
        // block-uniform) the accumulator is not read: the rows are written as NaN instead and the
        // column loop ends.  The bounded wait guards against an arrival that never comes; it
        // cannot make an MMA that is still running safe to abandon.
        uint32_t r[32] = {};
        if (ok) {
            const uint32_t taddr = tmem + ((uint32_t)(32 * w) << 16);
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                         "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                         "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                         : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                           "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
                           "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
                           "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
                           "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
                           "=r"(r[31])
                         : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        }
        const int k = 32 * w + lane;
        if (k < L) {
            const int n = base + k;
            B8 o[4];
            float hv[C];
#pragma unroll
            for (int i = 0; i < C / 2; ++i) {
                float u0 = ok ? __uint_as_float(r[2 * i]) + sBias[2 * i] : __int_as_float(0x7fc00000);
                float u1 = ok ? __uint_as_float(r[2 * i + 1]) + sBias[2 * i + 1] : __int_as_float(0x7fc00000);
                u0 = u0 > 0.f ? u0 : (u0 == u0 ? 0.f : u0);
                u1 = u1 > 0.f ? u1 : (u1 == u1 ? 0.f : u1);
                const __nv_bfloat162 b2 = __floats2bfloat162_rn(u0, u1);
                o[i >> 2].v[i & 3] = b2;
                const float2 f2 = __bfloat1622float2(b2);
                hv[2 * i] = f2.x;
                hv[2 * i + 1] = f2.y;
            }
            if (!LAST || Hout) {
                B8 *dst = reinterpret_cast<B8 *>(Hout + (size_t)n * C);
#pragma unroll
                for (int i = 0; i < 4; ++i) dst[i] = o[i];
            }
            if (LAST) {
                float y = sWout[C];
#pragma unroll
                for (int i = 0; i < C; ++i) y += sWout[i] * hv[i];
                if (Y) Y[n] = y;
                const double sg = sc[0] > 0. ? sc[0] : 1.;
                const double q = z[n] + (double)y * sg / (double)G.bdiag[n];
                if (qd) qd[n] = q;
                if (qf) qf[n] = (float)q;
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();                                  // sH and sA are rewritten next
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (w == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(TC_TMEM_COLS));
}

// node features x = [r/s, z|b|/s, ln(Dv/Dh)/8, bnd] (FP32 [N][4])
__global__ void k_nn_features(int N, const double *__restrict__ r, const double *__restrict__ z,
                              const double *__restrict__ sc, Geom G, float *__restrict__ X0) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    const double s = sc[0] > 0. ? sc[0] : 1.;
    float4 x;
    x.x = (float)(r[n] / s);
    x.y = (float)(z[n] * (double)G.bdiag[n] / s);
    x.z = G.feat2[n];
    x.w = G.bnd[n];
    *reinterpret_cast<float4 *>(X0 + (size_t)n * FIN) = x;
}

// ---------------------------------------------------------------------------------- backward
// Error loss (dq == null): loss = 0.5 * mean_n (y_n - ystar_n)^2, ystar = (t_n - z_n) |b_n| / s.
// Residual loss (dq != null): dq is dL/dq up to the factor sc[2]; since q = z + y s / |b|,
// dy = dq sc[2] s / |b|.  Per node: dy, the gradient w.r.t. h3 (FP32 [N][C]), and block
// partials of dw_out, db_out and (error loss only) the loss.
__global__ void __launch_bounds__(256)
k_nn_out_bwd(int N, const __nv_bfloat16 *__restrict__ H3, const float *__restrict__ Y, const double *__restrict__ t,
             const double *__restrict__ dq, const double *__restrict__ z, const double *__restrict__ sc, Geom G,
             const float *__restrict__ prm, float *__restrict__ dH, double *__restrict__ part /* [gridDim][C+2] */) {
    __shared__ double sp[256 / 32][C + 2];
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[C + 2];
#pragma unroll
    for (int i = 0; i < C + 2; ++i) acc[i] = 0.;
    if (n < N) {
        const double s = sc[0] > 0. ? sc[0] : 1.;
        double dy, e = 0.;
        if (dq) {
            dy = dq[n] * sc[2] * s / (double)G.bdiag[n];
        } else {
            const double ystar = (t[n] - z[n]) * (double)G.bdiag[n] / s;
            e = (double)Y[n] - ystar;
            dy = e / (double)N;
        }
        float h[C];
        const B8 *src = reinterpret_cast<const B8 *>(H3 + (size_t)n * C);
#pragma unroll
        for (int i = 0; i < 4; ++i) b8_to_f(src[i], h + 8 * i);
#pragma unroll
        for (int c = 0; c < C; ++c) {
            acc[c] = dy * (double)h[c];
            dH[(size_t)n * C + c] = (float)(dy * (double)prm[OFF_WOUT + c]);
        }
        acc[C] = dy;
        acc[C + 1] = 0.5 * e * e / (double)N;
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < C + 2; ++i) {
        double a = acc[i];
        for (int off = 16; off > 0; off >>= 1) a += __shfl_down_sync(0xffffffffu, a, off);
        if (lane == 0) sp[wid][i] = a;
    }
    __syncthreads();
    if (threadIdx.x < C + 2) {
        double a = sp[0][threadIdx.x];
        for (int q = 1; q < 256 / 32; ++q) a += sp[q][threadIdx.x];
        part[(size_t)blockIdx.x * (C + 2) + threadIdx.x] = a;
    }
}

// Layer backward, part 1: du = dH (.) [h > 0]; dX = du W (tensor cores); writes the per-node
// gradient pieces: G0 = dX_self - dX_ah - dX_av (to the node itself), Gh = dX_ah * iDh,
// Gv = dX_av * iDv (to be spread over the faces by k_nn_spread), and du in BF16 for dW.
__global__ void __launch_bounds__(32 * BWARPS)
k_nn_layer_bwd(int N, const __nv_bfloat16 *__restrict__ Hout, const float *__restrict__ dH,
               const __nv_bfloat16 *__restrict__ Wbf, Geom G, float *__restrict__ G0, float *__restrict__ Gh,
               float *__restrict__ Gv, __nv_bfloat16 *__restrict__ dU) {
    using namespace nvcuda;
    __shared__ __align__(32) __nv_bfloat16 sW[C * K3];               // W: [out][in]
    __shared__ __align__(32) __nv_bfloat16 sD[BWARPS][TILE * C];      // du tile
    __shared__ __align__(32) float sO[BWARPS][TILE * K3];             // dX tile
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = threadIdx.x; i < C * K3; i += blockDim.x) sW[i] = Wbf[i];
    __syncthreads();
    const int ntiles = (N + TILE - 1) / TILE;
    for (int t = blockIdx.x * BWARPS + w; t < ntiles; t += gridDim.x * BWARPS) {
        const int base = t * TILE;
        {
            const int n = base + lane;
            __align__(16) __nv_bfloat16 du[C];
            if (n < N) {
                float h[C];
                const B8 *src = reinterpret_cast<const B8 *>(Hout + (size_t)n * C);
#pragma unroll
                for (int i = 0; i < 4; ++i) b8_to_f(src[i], h + 8 * i);
#pragma unroll
                for (int c = 0; c < C; ++c) du[c] = __float2bfloat16(h[c] > 0.f ? dH[(size_t)n * C + c] : 0.f);
                const uint4 *s4 = reinterpret_cast<const uint4 *>(du);
                uint4 *d4 = reinterpret_cast<uint4 *>(dU + (size_t)n * C);
#pragma unroll
                for (int i = 0; i < 4; ++i) d4[i] = s4[i];
            } else {
#pragma unroll
                for (int c = 0; c < C; ++c) du[c] = __float2bfloat16(0.f);
            }
#pragma unroll
            for (int c = 0; c < C; ++c) sD[w][lane * C + c] = du[c];
        }
        __syncwarp();
        for (int rt = 0; rt < TILE / 16; ++rt) {
            for (int ct = 0; ct < K3 / 16; ++ct) {
                wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc;
                wmma::fill_fragment(acc, 0.f);
#pragma unroll
                for (int kc = 0; kc < C / 16; ++kc) {
                    wmma::fragment<wmma::matrix_a, 16, 16, 16, __nv_bfloat16, wmma::row_major> a;
                    wmma::fragment<wmma::matrix_b, 16, 16, 16, __nv_bfloat16, wmma::row_major> b;
                    wmma::load_matrix_sync(a, sD[w] + rt * 16 * C + kc * 16, C);
                    wmma::load_matrix_sync(b, sW + kc * 16 * K3 + ct * 16, K3);
                    wmma::mma_sync(acc, a, b, acc);
                }
                wmma::store_matrix_sync(sO[w] + rt * 16 * K3 + ct * 16, acc, K3, wmma::mem_row_major);
            }
        }
        __syncwarp();
        {
            const int n = base + lane;
            if (n < N) {
                const float ih = G.iDh[n], iv = G.iDv[n];
                const float *o = sO[w] + lane * K3;
#pragma unroll
                for (int c = 0; c < C; ++c) {
                    const float dah = ih > 0.f ? o[C + c] : 0.f, dav = iv > 0.f ? o[2 * C + c] : 0.f;
                    G0[(size_t)n * C + c] = o[c] - dah - dav;
                    Gh[(size_t)n * C + c] = dah * ih;
                    Gv[(size_t)n * C + c] = dav * iv;
                }
            }
        }
        __syncwarp();
    }
}

// Layer backward, part 2: dH_prev(j) = G0(j) + sum over faces (j,n) of T_jn * G(n), with Gh for
// horizontal and Gv for vertical faces (the transpose of the aggregation).
__global__ void k_nn_spread(ColMesh M, Geom G, const float *__restrict__ G0, const float *__restrict__ Gh,
                            const float *__restrict__ Gv, float *__restrict__ dHprev) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = t >> 2, q = t & 3;              // 4 threads per node, 8 channels each
    if (n >= M.N) return;
    const int c = n / M.L, k = n - c * M.L;
    float a[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = G0[(size_t)n * C + 8 * q + i];
    for_faces(M, c, k, n,
        [&](const Face &f) {
            RowF p;
            const float *src = (f.vert ? Gv : Gh) + (size_t)f.j * C + 8 * q;
            p.lo = *reinterpret_cast<const float4 *>(src);
            p.hi = *reinterpret_cast<const float4 *>(src + 4);
            p.t = face_T(M, G, f);
            return p;
        },
        [&](const Face &f, const auto &p) {
            a[0] += p.t * p.lo.x; a[1] += p.t * p.lo.y; a[2] += p.t * p.lo.z; a[3] += p.t * p.lo.w;
            a[4] += p.t * p.hi.x; a[5] += p.t * p.hi.y; a[6] += p.t * p.hi.z; a[7] += p.t * p.hi.w;
        });
#pragma unroll
    for (int i = 0; i < 8; ++i) dHprev[(size_t)n * C + 8 * q + i] = a[i];
}

// dW (C x K3) = sum over nodes of du^T X; db = sum du.  Each block accumulates its node tiles on
// the tensor cores, folds its warps in order and writes one partial (deterministic).
__global__ void __launch_bounds__(32 * WARPS)
k_nn_dw(int Npad, const __nv_bfloat16 *__restrict__ dU, const __nv_bfloat16 *__restrict__ Xs,
        float *__restrict__ part /* [gridDim][C*K3 + C] */) {
    using namespace nvcuda;
    __shared__ __align__(32) float sAcc[C * K3];
    __shared__ float sB[WARPS][C];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc[C / 16][K3 / 16];
#pragma unroll
    for (int a = 0; a < C / 16; ++a)
#pragma unroll
        for (int b = 0; b < K3 / 16; ++b) wmma::fill_fragment(acc[a][b], 0.f);
    float db = 0.f;
    const int ntiles = Npad / 16;         // rows N..Npad-1 of dU and Xs are zero
    for (int t = blockIdx.x * WARPS + w; t < ntiles; t += gridDim.x * WARPS) {
        const int base = t * 16;
        // A = du^T (C x 16 nodes): du tile [16][C] read as column-major (ld = C)
#pragma unroll
        for (int kb = 0; kb < C / 16; ++kb) {
            wmma::fragment<wmma::matrix_a, 16, 16, 16, __nv_bfloat16, wmma::col_major> a;
            wmma::load_matrix_sync(a, dU + (size_t)base * C + kb * 16, C);
#pragma unroll
            for (int ct = 0; ct < K3 / 16; ++ct) {
                wmma::fragment<wmma::matrix_b, 16, 16, 16, __nv_bfloat16, wmma::row_major> b;
                wmma::load_matrix_sync(b, Xs + (size_t)base * K3 + ct * 16, K3);
                wmma::mma_sync(acc[kb][ct], a, b, acc[kb][ct]);
            }
        }
        for (int m = 0; m < 16; ++m) db += __bfloat162float(dU[(size_t)(base + m) * C + lane]);
    }
    // fold warps in order into shared memory
    for (int i = threadIdx.x; i < C * K3; i += blockDim.x) sAcc[i] = 0.f;
    sB[w][lane] = db;
    __syncthreads();
    for (int ww = 0; ww < WARPS; ++ww) {
        if (w == ww) {
#pragma unroll
            for (int a = 0; a < C / 16; ++a)
#pragma unroll
                for (int b = 0; b < K3 / 16; ++b) {
                    wmma::fragment<wmma::accumulator, 16, 16, 16, float> cur;
                    wmma::load_matrix_sync(cur, sAcc + a * 16 * K3 + b * 16, K3, wmma::mem_row_major);
                    for (int e = 0; e < cur.num_elements; ++e) cur.x[e] += acc[a][b].x[e];
                    wmma::store_matrix_sync(sAcc + a * 16 * K3 + b * 16, cur, K3, wmma::mem_row_major);
                }
        }
        __syncthreads();
    }
    float *pp = part + (size_t)blockIdx.x * (C * K3 + C);
    for (int i = threadIdx.x; i < C * K3; i += blockDim.x) pp[i] = sAcc[i];
    if (threadIdx.x < C) {
        float s = 0.f;
        for (int ww = 0; ww < WARPS; ++ww) s += sB[ww][threadIdx.x];
        pp[C * K3 + threadIdx.x] = s;
    }
}

// input layer backward: du0 = dH0 (.) [h0 > 0]; partials of dW_in (C x FIN) and db_in
__global__ void __launch_bounds__(256)
k_nn_in_bwd(int N, const __nv_bfloat16 *__restrict__ H0, const float *__restrict__ dH, const float *__restrict__ X0,
            double *__restrict__ part /* [gridDim][C*FIN + C] */) {
    __shared__ double sp[256 / 32][C * FIN + C];
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    float h[C], du[C], x[FIN];
    if (n < N) {
        const B8 *src = reinterpret_cast<const B8 *>(H0 + (size_t)n * C);
#pragma unroll
        for (int i = 0; i < 4; ++i) b8_to_f(src[i], h + 8 * i);
#pragma unroll
        for (int c = 0; c < C; ++c) du[c] = h[c] > 0.f ? dH[(size_t)n * C + c] : 0.f;
#pragma unroll
        for (int i = 0; i < FIN; ++i) x[i] = X0[(size_t)n * FIN + i];
    } else {
#pragma unroll
        for (int c = 0; c < C; ++c) du[c] = 0.f;
#pragma unroll
        for (int i = 0; i < FIN; ++i) x[i] = 0.f;
    }
    for (int c = 0; c < C; ++c) {
        for (int i = 0; i <= FIN; ++i) {
            double a = i < FIN ? (double)du[c] * (double)x[i] : (double)du[c];
            for (int off = 16; off > 0; off >>= 1) a += __shfl_down_sync(0xffffffffu, a, off);
            if (lane == 0) sp[wid][i < FIN ? c * FIN + i : C * FIN + c] = a;
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < C * FIN + C; i += blockDim.x) {
        double a = sp[0][i];
        for (int q = 1; q < 256 / 32; ++q) a += sp[q][i];
        part[(size_t)blockIdx.x * (C * FIN + C) + i] = a;
    }
}

// fold per-block partials (fixed order) into the gradient vector, offsets given per segment
__global__ void k_nn_fold_f(int nblk, int stride, int width, const float *__restrict__ part, float *__restrict__ g) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= width) return;
    double s = 0.;
    for (int b = 0; b < nblk; ++b) s += (double)part[(size_t)b * stride + i];
    g[i] = (float)s;
}
__global__ void k_nn_fold_d(int nblk, int stride, int width, const double *__restrict__ part, float *__restrict__ g) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= width) return;
    double s = 0.;
    for (int b = 0; b < nblk; ++b) s += part[(size_t)b * stride + i];
    g[i] = (float)s;
}

// Adam step on the FP32 master parameters, then refresh the BF16 layer matrices
__global__ void k_nn_adam(int np, float *__restrict__ prm, const float *__restrict__ g, float *__restrict__ m1,
                          float *__restrict__ m2, float lr, float b1, float b2, float eps, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    const float gi = g[i];
    const float a = b1 * m1[i] + (1.f - b1) * gi;
    const float b = b2 * m2[i] + (1.f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = b;
    prm[i] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
}

__global__ void k_nn_to_bf16(const float *__restrict__ prm, __nv_bfloat16 *__restrict__ W) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= NL * C * K3) return;
    const int l = i / (C * K3), o = i - l * C * K3;
    W[i] = __float2bfloat16(prm[OFF_L0 + l * LSTRIDE + o]);
}

// face couplings and per-node sums for the network (once per handle)
__global__ void k_nn_geom_faces(ColMesh M, const int32_t *__restrict__ e2a, const int32_t *__restrict__ e2b,
                                const double *__restrict__ vol, const double *__restrict__ rh0,
                                const double *__restrict__ coefw, double dt, float *__restrict__ Th,
                                float *__restrict__ Tv) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int nh = M.NE2 * M.L;
    if (t < nh) {
        const int e = t / M.L, k = t - e * M.L;
        const int a = e2a[e] * M.L + k, b = e2b[e] * M.L + k;
        const double s2 = M.Sh[0][t] * M.Sh[0][t] + M.Sh[1][t] * M.Sh[1][t] + M.Sh[2][t] * M.Sh[2][t];
        Th[t] = (float)(0.5 * dt * s2 * 0.5 * (rh0[a] + rh0[b]) / (0.5 * (vol[a] + vol[b])));
    } else if (t < nh + M.N) {
        const int n = t - nh;
        const int k = n % M.L;
        float v = 0.f;
        if (k + 1 < M.L) {
            const double s2 = M.Sv[0][n] * M.Sv[0][n] + M.Sv[1][n] * M.Sv[1][n]
                            + M.Sv[2][n] * M.Sv[2][n] * 0.5 * (coefw[n] + coefw[n + 1]);
            v = (float)(0.5 * dt * s2 * 0.5 * (rh0[n] + rh0[n + 1]) / (0.5 * (vol[n] + vol[n + 1])));
        }
        Tv[n] = v;
    }
}

__global__ void k_nn_geom_nodes(ColMesh M, const float *__restrict__ Th, const float *__restrict__ Tv,
                                float *__restrict__ iDh, float *__restrict__ iDv, float *__restrict__ feat2,
                                float *__restrict__ bnd) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= M.N) return;
    const int c = n / M.L, k = n - c * M.L;
    float dh = 0.f, dv = 0.f;
    for_faces(M, c, k, n, [&](const Face &f) { return f.vert ? Tv[f.si] : Th[f.si]; },
              [&](const Face &f, float t) {
                  if (f.vert) dv += t; else dh += t;
              });
    iDh[n] = dh > 0.f ? 1.f / dh : 0.f;
    iDv[n] = dv > 0.f ? 1.f / dv : 0.f;
    feat2[n] = (dh > 0.f && dv > 0.f) ? logf(dv / dh) / 8.f : 0.f;
    bnd[n] = (k == 0 || k == M.L - 1) ? 1.f : 0.f;
}

}  // namespace nn
}  // namespace mpgk

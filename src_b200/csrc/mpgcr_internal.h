// Internal declarations of the B200 MPDATA + GCR library (not part of the C ABI).
//
// Device layout ("column layout"): a prism-column mesh of NC columns and L levels; node
// n = c*L + k (level fastest), so every gather along a horizontal edge reads L contiguous
// values of the neighbour column.  Horizontal edges are stored once per 2D edge e with their
// per-level face vectors Sh[d][e*L + k]; vertical faces (c,k)->(c,k+1) at Sv[d][c*L + k].
// Per column a short adjacency list (cadj) names the incident 2D edges and where the two
// vertical faces fall in the reference's edge order, so per-node sums are accumulated in the
// same order as the reference's edge loops.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/mpgcr.h"

#define MPG_MAX_LORD 16
#define MPG_MAX_UNK 16

// adjacency codes (cadj[j].x): >= 0 -> 2D edge (code >> 1), low bit set when this column is
// the edge's second end (contributions subtract); the two vertical faces:
#define MPG_ADJ_BELOW (-1)
#define MPG_ADJ_ABOVE (-2)

// boundary point of the column layout (one entry of ibpoin/anp/sbb, reference order kept)
struct BEntry {
    int32_t k;         // level of the boundary node in its column
    int32_t type;      // ibpoin(:,2)
    double anp[3];
    double sbb[3];
    double pad;
};

// Everything a gather kernel needs, passed by value.
struct ColMesh {
    int32_t NC, L, N, NE2;
    const int32_t *cptr;     // [NC+1]
    const int2 *cadj;        // [cptr[NC]]
    const double *Sh[3];     // [NE2*L]
    const double *Sv[3];     // [N]
    const float4 *Shf4;      // FP32 copies (mixed precision) packed (x, y, z, 0): one 16-byte
    const float4 *Svf4;      // load per face; may be null
    const int32_t *bptr;     // [NC+1] boundary entries per column
    const BEntry *bent;
    int32_t iper;            // 2: no boundary closure in derivative; 0: sbb closure
};

// Thrown-free error plumbing.
void mpg_set_error(const std::string &msg);
int mpg_fail(int code, const std::string &msg);

#define MPG_CUDA(call)                                                                  \
    do {                                                                                \
        cudaError_t _e = (call);                                                        \
        if (_e != cudaSuccess)                                                          \
            return mpg_fail(MPG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(_e)); \
    } while (0)

// Host-side mesh analysis result (column detection), built by setup.cpp.
struct HostColumnMesh {
    int32_t NC = 0, L = 0, N = 0, NE2 = 0;
    std::vector<int32_t> perm;      // ref node -> internal node
    std::vector<int32_t> iperm;     // internal node -> ref node
    std::vector<int32_t> cptr;
    std::vector<int2> cadj;
    std::vector<double> Sh[3];      // [NE2*L]
    std::vector<double> Sv[3];      // [N]
    std::vector<int32_t> bptr;
    std::vector<BEntry> bent;
    std::vector<int32_t> e2a, e2b;  // 2D edge endpoints (internal columns)
    bool bitwise_order = true;      // per-node sums follow the reference edge order exactly
    // node-ordered geometry (internal order)
    std::vector<double> x, y, z, vol;
    // the reference's periodic duplicate-node lists (icoin, icoin2, icoin4) as copy groups in
    // list order, internal node numbers: every copy node with its group, and the groups
    std::vector<int32_t> cp_node, cp_gbeg, cp_gsize, cp_members, cp_grp, cp_grpsize;
};

int mpg_build_column_mesh(const mpg_mesh_ref *m, HostColumnMesh *out);
// the reference's set-up sum of the copies' volumes (cyclicr, cyclicr2, cyclicr4 on vol,
// ref.f:99-103): vol of every node, with each group's members replaced by their sum
std::vector<double> mpg_periodic_volumes(const mpg_mesh_ref *m);

// Order of the fused laplc's work items (gradient items of `per` consecutive nodes, divergence
// items of `per` level pairs; PL = (L + 1) / 2 pairs per column).  Returns the number of gradient
// items.  `sched` lists every item once,
// gradient items in node order, each divergence item (encoded -(d+1)) `lag` gradient items after
// the last one whose fluxes it reads (or at the end), so that by the time its ticket is drawn the
// blocks in flight have moved on from its dependencies; dptr/drng give each divergence item's
// gradient items as merged inclusive ranges.
int32_t mpg_laplc_schedule(const HostColumnMesh &cm, int per, int lag, std::vector<int32_t> &sched,
                           std::vector<int32_t> &dptr, std::vector<int2> &drng);

// Static per-node quantities computed on the host at creation (internal order), restating the
// set-up part of mpsolver: rhprof/thprof, absorbers, beta_timestep_unstr, compute_d_unstr,
// ambient state, coefw and the vertical-line preconditioner coefficients.
struct HostStatic {
    std::vector<double> rh0, th0, the, dthedz, alpha, coefw, d1, ue, ve;
    double betaunstr1 = 0.;
    // line preconditioner, per impfl, in the column-interleaved layout used by the solve kernel:
    // sub-diagonal a, inverse pivot 1/m and c' of the Thomas factorisation
    std::vector<double> la[2], lm[2], lcp[2];
    std::vector<float> lbabs;       // |diagonal| of the line matrix for impfl = 1 (node order)
    // iprc = 4: the column blocks of laplc (tridiagonal on even and odd levels), factorised per
    // parity chain, same interleaved layout; empty unless iprc = 4
    std::vector<double> wa[2], wm[2], wcp[2];
};

int mpg_host_static(const mpg_params *P, const mpg_mesh_ref *m, const HostColumnMesh &cm,
                    HostStatic *out);

// iprc = 4: entries A[k][k-2], A[k][k], A[k][k+2] of laplc's column blocks (reference node order,
// cw = coefw*impfl + (1-impfl) per reference node) and their factorisation into hs->wa/wm/wcp
void mpg_wide_entries(const mpg_params *P, const mpg_mesh_ref *m, const HostColumnMesh &cm,
                      const std::vector<double> &rh0r, const std::vector<double> &volr,
                      const std::vector<double> &cw, std::vector<double> &lo, std::vector<double> &dg,
                      std::vector<double> &hi);
void mpg_wide_coeffs(const mpg_params *P, const mpg_mesh_ref *m, const HostColumnMesh &cm,
                     const std::vector<double> &rh0r, const std::vector<double> &volr,
                     const std::vector<double> *cwr, HostStatic *hs);

// interleaved coefficient layout for the column solve: column c, level k ->
// ((c / 32) * L + k) * 32 + (c % 32)
__host__ __device__ inline int64_t line_index(int32_t c, int32_t k, int32_t L) {
    return ((int64_t)(c >> 5) * L + k) * 32 + (c & 31);
}

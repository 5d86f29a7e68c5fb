// Host-side set-up: detection of the prism-column structure of a mesh given in the
// reference's COMMON layout, packing into the column layout, and the static per-node
// quantities of mpsolver's set-up phase (lippsLFroude_implgwopks3D_unstr3.f:99-273).
//
// The per-node sums here (compute_d_unstr, the line preconditioner coefficients) loop over the
// edges in the reference's order, so they round exactly like the reference's loops.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <unordered_map>

#include "mpgcr_internal.h"

namespace {

struct PairHash {
    size_t operator()(const std::pair<uint64_t, uint64_t> &p) const {
        uint64_t h = p.first * 0x9E3779B97F4A7C15ull ^ (p.second + 0x7F4A7C159E3779B9ull + (p.first << 6));
        return (size_t)(h ^ (h >> 31));
    }
};

inline uint64_t bits(double v) {
    uint64_t u;
    std::memcpy(&u, &v, 8);
    return u;
}

inline double amax(double a, double b) { return a > b ? a : b; }
inline double amin(double a, double b) { return a < b ? a : b; }

struct EdgeView {   // internal edges followed by semi-edges, 0-based
    const mpg_mesh_ref *m;
    int64_t n() const { return (int64_t)m->nedge + m->nbface; }
    int i1(int64_t j) const {
        return j < m->nedge ? m->iedge[j] - 1 : m->kbface[j - m->nedge] - 1;
    }
    int i2(int64_t j) const {
        return j < m->nedge ? m->iedge[(size_t)m->nedgex + j] - 1
                            : m->kbface[(size_t)m->nfacesx + j - m->nedge] - 1;
    }
    double s(int64_t j, int d) const {
        return j < m->nedge ? m->sn[(size_t)d * m->nedgex + j]
                            : m->sb[(size_t)d * m->nfacesx + j - m->nedge];
    }
};

}  // namespace

int mpg_build_column_mesh(const mpg_mesh_ref *m, HostColumnMesh *out) {
    const int npoin = m->npoin;
    if (npoin <= 0 || m->nedge < 0 || m->nbface < 0 || m->nboun < 0)
        return mpg_fail(MPG_ERR_ARG, "mesh sizes must be non-negative and npoin > 0");
    if (m->npoinx < npoin || m->nedgex < m->nedge || (m->nfacesx < m->nbface || m->nfacesx < m->nboun))
        return mpg_fail(MPG_ERR_ARG, "leading dimensions smaller than the counts");
    if (!m->coord || !m->vol || (m->nedge && (!m->iedge || !m->sn)) ||
        (m->nbface && (!m->kbface || !m->sb)) || (m->nboun && (!m->ibpoin || !m->anp || !m->sbb)))
        return mpg_fail(MPG_ERR_ARG, "null mesh array");
    if ((m->ncoin && !m->icoin) || (m->ncoin2 && !m->icoin2) || (m->ncoin4 && !m->icoin4) || m->ncoin < 0 ||
        m->ncoin2 < 0 || m->ncoin4 < 0 || (m->ncoin && m->ldcoin < m->ncoin) ||
        (m->ncoin2 && m->nfacesx < m->ncoin2) || (m->ncoin4 && m->nfacesx < m->ncoin4))
        return mpg_fail(MPG_ERR_ARG, "periodic lists: null array or leading dimension smaller than the count");
    const double *X = m->coord, *Y = m->coord + m->npoinx, *Z = m->coord + 2 * (size_t)m->npoinx;

    // ---- 1. columns = nodes with bitwise-equal (x, y), in order of first appearance
    std::unordered_map<std::pair<uint64_t, uint64_t>, int32_t, PairHash> cmap;
    cmap.reserve((size_t)npoin / 8 + 16);
    std::vector<int32_t> col(npoin);
    std::vector<int32_t> csize;
    // nodes usually arrive column by column: remember the last column looked up
    std::pair<uint64_t, uint64_t> last_key(~0ull, ~0ull);
    int32_t last_col = -1;
    for (int i = 0; i < npoin; ++i) {
        auto key = std::make_pair(bits(X[i]), bits(Y[i]));
        int32_t c;
        if (key == last_key) {
            col[i] = last_col;
            csize[last_col]++;
            continue;
        }
        auto it = cmap.find(key);
        if (it == cmap.end()) {
            c = (int32_t)csize.size();
            cmap.emplace(key, c);
            csize.push_back(0);
        } else {
            c = it->second;
        }
        col[i] = c;
        csize[c]++;
        last_key = key;
        last_col = c;
    }
    const int NC = (int)csize.size();
    const int L = csize[0];
    for (int c = 0; c < NC; ++c)
        if (csize[c] != L)
            return mpg_fail(MPG_ERR_MESH, "not a prism-column mesh: columns have different numbers of levels");
    if ((int64_t)NC * L != npoin) return mpg_fail(MPG_ERR_MESH, "column count mismatch");

    // ---- 2. levels: sort each column by z
    std::vector<int32_t> start(NC + 1, 0);
    for (int c = 0; c < NC; ++c) start[c + 1] = start[c] + L;
    std::vector<int32_t> fill(start.begin(), start.end() - 1);
    std::vector<int32_t> nodes(npoin);
    for (int i = 0; i < npoin; ++i) nodes[fill[col[i]]++] = i;
    out->perm.assign(npoin, 0);
    out->iperm.assign(npoin, 0);
    std::vector<int32_t> lev(npoin);
    for (int c = 0; c < NC; ++c) {
        int32_t *b = nodes.data() + start[c];
        std::stable_sort(b, b + L, [&](int32_t a, int32_t q) { return Z[a] < Z[q]; });
        for (int k = 0; k < L; ++k) {
            if (k && !(Z[b[k]] > Z[b[k - 1]]))
                return mpg_fail(MPG_ERR_MESH, "not a prism-column mesh: repeated height in a column");
            lev[b[k]] = k;
            out->perm[b[k]] = c * L + k;
            out->iperm[c * L + k] = b[k];
        }
    }

    // ---- 3. classify edges: vertical faces, and the 2D edges (unique column pairs found at
    //         level 0, numbered in (a, b) order for locality), then every horizontal edge
    EdgeView ev{m};
    const int64_t nall = ev.n();
    std::vector<int32_t> vorig((size_t)npoin, -1);
    for (int d = 0; d < 3; ++d) out->Sv[d].assign(npoin, 0.0);
    std::vector<uint64_t> keys0;
    int64_t nhor = 0;
    for (int64_t j = 0; j < nall; ++j) {
        int i1 = ev.i1(j), i2 = ev.i2(j);
        if (i1 < 0 || i1 >= npoin || i2 < 0 || i2 >= npoin || i1 == i2)
            return mpg_fail(MPG_ERR_MESH, "edge " + std::to_string(j + 1) + " has an invalid node index");
        int c1 = col[i1], c2 = col[i2], k1 = lev[i1], k2 = lev[i2];
        if (c1 == c2) {
            if (std::abs(k1 - k2) != 1)
                return mpg_fail(MPG_ERR_MESH, "vertical edge skips a level");
            int klo = std::min(k1, k2);
            int64_t f = (int64_t)c1 * L + klo;
            if (vorig[f] != -1) return mpg_fail(MPG_ERR_MESH, "two vertical edges between the same nodes");
            vorig[f] = (int32_t)j;
            const bool up = k1 < k2;
            for (int d = 0; d < 3; ++d) out->Sv[d][f] = up ? ev.s(j, d) : -ev.s(j, d);
        } else {
            if (k1 != k2) return mpg_fail(MPG_ERR_MESH, "edge joins different levels of two columns");
            ++nhor;
            if (k1 == 0) {
                int a = std::min(c1, c2), b = std::max(c1, c2);
                keys0.push_back((uint64_t)a * (uint64_t)NC + (uint64_t)b);
            }
        }
    }
    std::sort(keys0.begin(), keys0.end());
    if (std::adjacent_find(keys0.begin(), keys0.end()) != keys0.end())
        return mpg_fail(MPG_ERR_MESH, "two edges between the same pair of nodes");
    const int NE2 = (int)keys0.size();
    if (nhor != (int64_t)NE2 * L)
        return mpg_fail(MPG_ERR_MESH, "a horizontal edge is missing at some level");
    if ((int64_t)NC * L > INT32_MAX / 2 || (int64_t)NE2 * L > INT32_MAX / 2)
        return mpg_fail(MPG_ERR_MESH, "mesh too large for 32-bit indexing");
    std::unordered_map<uint64_t, int32_t> emap;
    emap.reserve((size_t)NE2 * 2 + 16);
    out->e2a.resize(NE2);
    out->e2b.resize(NE2);
    for (int e = 0; e < NE2; ++e) {
        emap.emplace(keys0[e], e);
        out->e2a[e] = (int32_t)(keys0[e] / (uint64_t)NC);
        out->e2b[e] = (int32_t)(keys0[e] % (uint64_t)NC);
    }
    std::vector<uint64_t>().swap(keys0);
    for (int d = 0; d < 3; ++d) out->Sh[d].assign((size_t)NE2 * L, 0.0);
    std::vector<int32_t> horig2((size_t)NE2 * L, -1);
    uint64_t last_ekey = ~0ull;
    int32_t last_e = -1;
    for (int64_t j = 0; j < nall; ++j) {
        int i1 = ev.i1(j), i2 = ev.i2(j);
        int c1 = col[i1], c2 = col[i2];
        if (c1 == c2) continue;
        int a = std::min(c1, c2), b = std::max(c1, c2), k = lev[i1];
        uint64_t key = (uint64_t)a * (uint64_t)NC + (uint64_t)b;
        int32_t e;
        if (key == last_ekey) {          // edges usually arrive level by level for one 2D edge
            e = last_e;
        } else {
            auto it = emap.find(key);
            if (it == emap.end()) return mpg_fail(MPG_ERR_MESH, "a horizontal edge is missing at level 0");
            e = it->second;
            last_ekey = key;
            last_e = e;
        }
        size_t idx = (size_t)e * L + k;
        if (horig2[idx] != -1) return mpg_fail(MPG_ERR_MESH, "two edges between the same pair of nodes");
        horig2[idx] = (int32_t)j;
        const bool flip = (c1 != a);
        for (int d = 0; d < 3; ++d) out->Sh[d][idx] = flip ? -ev.s(j, d) : ev.s(j, d);
    }
    for (int c = 0; c < NC; ++c)
        for (int k = 0; k + 1 < L; ++k)
            if (vorig[(size_t)c * L + k] == -1)
                return mpg_fail(MPG_ERR_MESH, "a column lacks a vertical edge between consecutive levels");

    // ---- 5. per-column adjacency in reference edge order
    std::vector<int32_t> deg(NC + 1, 0);
    for (int e = 0; e < NE2; ++e) { deg[out->e2a[e]]++; deg[out->e2b[e]]++; }
    out->cptr.assign(NC + 1, 0);
    for (int c = 0; c < NC; ++c) out->cptr[c + 1] = out->cptr[c] + deg[c] + 2;
    out->cadj.assign(out->cptr[NC], make_int2(0, 0));
    std::vector<int32_t> cfill(out->cptr.begin(), out->cptr.end() - 1);
    for (int e = 0; e < NE2; ++e) {
        int a = out->e2a[e], b = out->e2b[e];
        out->cadj[cfill[a]++] = make_int2(2 * e, b);
        out->cadj[cfill[b]++] = make_int2(2 * e + 1, a);
    }
    for (int c = 0; c < NC; ++c) {
        out->cadj[cfill[c]++] = make_int2(MPG_ADJ_BELOW, c);
        out->cadj[cfill[c]++] = make_int2(MPG_ADJ_ABOVE, c);
    }
    auto orig_at = [&](const int2 &en, int c, int k) -> int64_t {
        if (en.x >= 0) return horig2[(size_t)(en.x >> 1) * L + k];
        if (en.x == MPG_ADJ_BELOW) return k > 0 ? vorig[(size_t)c * L + k - 1] : -1;
        return k + 1 < L ? vorig[(size_t)c * L + k] : -1;
    };
    const int kref = L > 2 ? 1 : 0;
    bool bitwise = true;
    std::vector<std::pair<int64_t, int2>> tmp;
    for (int c = 0; c < NC; ++c) {
        int s = out->cptr[c], t = out->cptr[c + 1];
        tmp.clear();
        for (int j = s; j < t; ++j) {
            int64_t o = orig_at(out->cadj[j], c, kref);
            // a vertical face absent at kref (L == 2) sorts by its presence at the other level
            if (o < 0) o = orig_at(out->cadj[j], c, kref == 0 ? 1 : 0);
            tmp.emplace_back(o, out->cadj[j]);
        }
        std::stable_sort(tmp.begin(), tmp.end(),
                         [](const std::pair<int64_t, int2> &p, const std::pair<int64_t, int2> &q) {
                             return p.first < q.first;
                         });
        for (int j = s; j < t; ++j) out->cadj[j] = tmp[j - s].second;
        if (bitwise) {
            for (int k = 0; k < L && bitwise; ++k) {
                int64_t prev = -1;
                for (int j = s; j < t; ++j) {
                    int64_t o = orig_at(out->cadj[j], c, k);
                    if (o < 0) continue;
                    if (o < prev) { bitwise = false; break; }
                    prev = o;
                }
            }
        }
    }
    out->bitwise_order = bitwise;

    // ---- 6. boundary points per column, reference order kept within a level
    std::vector<std::vector<BEntry>> bcol(NC);
    for (int b = 0; b < m->nboun; ++b) {
        int i = m->ibpoin[b] - 1;
        if (i < 0 || i >= npoin) return mpg_fail(MPG_ERR_MESH, "boundary point with invalid node index");
        BEntry be{};
        be.k = lev[i];
        be.type = m->ibpoin[(size_t)m->nfacesx + b];
        for (int d = 0; d < 3; ++d) {
            be.anp[d] = m->anp[(size_t)d * m->nfacesx + b];
            be.sbb[d] = m->sbb[(size_t)d * m->nfacesx + b];
        }
        bcol[col[i]].push_back(be);
    }
    out->bptr.assign(NC + 1, 0);
    out->bent.clear();
    for (int c = 0; c < NC; ++c) {
        std::stable_sort(bcol[c].begin(), bcol[c].end(),
                         [](const BEntry &p, const BEntry &q) { return p.k < q.k; });
        out->bent.insert(out->bent.end(), bcol[c].begin(), bcol[c].end());
        out->bptr[c + 1] = (int32_t)out->bent.size();
    }

    // ---- 7. geometry in internal order
    out->x.resize(npoin); out->y.resize(npoin); out->z.resize(npoin); out->vol.resize(npoin);
    for (int n = 0; n < npoin; ++n) {
        int i = out->iperm[n];
        out->x[n] = X[i]; out->y[n] = Y[i]; out->z[n] = Z[i]; out->vol[n] = m->vol[i];
    }
    out->NC = NC; out->L = L; out->N = npoin; out->NE2 = NE2;

    // ---- 8. periodic copy groups (icoin pairs, icoin2 pairs, icoin4 quadruples), list order
    out->cp_node.clear(); out->cp_gbeg.clear(); out->cp_gsize.clear();
    out->cp_members.clear(); out->cp_grp.clear(); out->cp_grpsize.clear();
    std::vector<uint8_t> seen(npoin, 0);
    struct Lst { const int32_t *a; int n, w; size_t ld; };
    const Lst lists[3] = {{m->icoin, m->ncoin, 2, (size_t)m->ldcoin}, {m->icoin2, m->ncoin2, 2, (size_t)m->nfacesx},
                          {m->icoin4, m->ncoin4, 4, (size_t)m->nfacesx}};
    for (const Lst &l : lists)
        for (int g = 0; g < l.n; ++g) {
            const int32_t off = (int32_t)out->cp_members.size();
            out->cp_grp.push_back(off);
            out->cp_grpsize.push_back(l.w);
            for (int q = 0; q < l.w; ++q) {
                const int i = l.a[(size_t)q * l.ld + g] - 1;
                if (i < 0 || i >= npoin) return mpg_fail(MPG_ERR_MESH, "periodic list names a node out of range");
                if (seen[i]) return mpg_fail(MPG_ERR_UNSUPPORTED, "a node appears in more than one periodic copy group");
                seen[i] = 1;
                out->cp_members.push_back(out->perm[i]);
            }
            for (int q = 0; q < l.w; ++q) {
                out->cp_node.push_back(out->cp_members[off + q]);
                out->cp_gbeg.push_back(off);
                out->cp_gsize.push_back(l.w);
            }
        }
    return MPG_OK;
}

std::vector<double> mpg_periodic_volumes(const mpg_mesh_ref *m) {
    std::vector<double> v(m->vol, m->vol + m->npoin);
    auto pairs = [&](const int32_t *a, int n, size_t ld) {        // cyclicr / cyclicr2
        std::vector<double> uc(n);
        for (int c = 0; c < n; ++c) uc[c] = v[a[c] - 1] + v[a[ld + c] - 1];
        for (int c = 0; c < n; ++c) { v[a[c] - 1] = uc[c]; v[a[ld + c] - 1] = uc[c]; }
    };
    if (m->ncoin) pairs(m->icoin, m->ncoin, (size_t)m->ldcoin);
    if (m->ncoin2) pairs(m->icoin2, m->ncoin2, (size_t)m->nfacesx);
    if (m->ncoin4) {                                                // cyclicr4
        const size_t ld = m->nfacesx;
        const int32_t *a = m->icoin4;
        std::vector<double> uc(m->ncoin4);
        for (int c = 0; c < m->ncoin4; ++c)
            uc[c] = v[a[c] - 1] + v[a[ld + c] - 1] + v[a[2 * ld + c] - 1] + v[a[3 * ld + c] - 1];
        for (int c = 0; c < m->ncoin4; ++c)
            for (int q = 0; q < 4; ++q) v[a[q * ld + c] - 1] = uc[c];
    }
    return v;
}

// Static set-up quantities (internal order).  Each block names the reference lines it
// restates; the expressions keep the reference's association.
int mpg_host_static(const mpg_params *P, const mpg_mesh_ref *m, const HostColumnMesh &cm,
                    HostStatic *hs) {
    const int N = cm.N, L = cm.L, NC = cm.NC;
    const double dt = P->delt, g = P->g, st = P->strat;
    const std::vector<int32_t> &perm = cm.perm;
    // rhprof / thprof (ref.f:4532-4579) — per node, reference-order independent
    hs->rh0.assign(N, 1.0);
    hs->th0.assign(N, P->tetbar);
    {
        double rgas = 287.04, cp = 3.5 * rgas, cap = rgas / cp, capi = 1. / cap;
        double tt00 = P->tetbar, th00 = P->tetbar;
        double cs = g / (cp * tt00 * st);
        double rh0inf = 1., rh00 = 1.;
        for (int n = 0; n < N; ++n) {
            double z = cm.z[n];
            double r = rh0inf;
            if (P->lipps == 1) {
                double exs = std::exp(-st * z);
                r = rh00 * exs * std::pow(1. - cs * (1. - exs), capi - 1.);
            }
            hs->rh0[n] = r;
            hs->th0[n] = P->lipps == 1 ? th00 * std::exp(st * z) : th00;
        }
    }
    // absorbers (ref.f:2915-3026)
    hs->alpha.assign(N, 0.0);
    if (P->irl == 1) {
        double r = 1., eps = 1.e-07;
        double abxmax = -1.e+07, abxmin = 1.e+07, abymax = -1.e+07, abymin = 1.e+07;
        double abzmax = -1.e+07, abzmin = 1.e+07;
        for (int n = 0; n < N; ++n) {
            abxmax = amax(cm.x[n], abxmax); abxmin = amin(cm.x[n], abxmin);
            abymax = amax(cm.y[n], abymax); abymin = amin(cm.y[n], abymin);
            abzmax = amax(cm.z[n], abzmax); abzmin = amin(cm.z[n], abzmin);
        }
        double xabr = abxmax * r - P->dxabr, xabl = abxmin * r + P->dxabl;
        double yabu = abymax * r - P->dyabu, yabd = abymin * r + P->dyabd;
        double zabu = abzmax - P->dzabu, zabd = abzmin + P->dzabd;
        double tolil = P->towxl != 0. ? 1. / P->towxl : 0.;
        double tolir = P->towxr != 0. ? 1. / P->towxr : 0.;
        double toliu = P->towyu != 0. ? 1. / P->towyu : 0.;
        double tolid = P->towyd != 0. ? 1. / P->towyd : 0.;
        double toliuz = P->towzu != 0. ? 1. / P->towzu : 0.;
        double tolidz = P->towzd != 0. ? 1. / P->towzd : 0.;
        for (int n = 0; n < N; ++n) {
            double relx, rely, relz, r0, r1, r2, relb;
            r0 = cm.x[n] * r; r1 = 0.; r2 = 0.; relb = 0.;
            if (P->dxabl != 0.) r1 = amax(0., xabl - r0) / P->dxabl;
            if (P->dxabr != 0.) r2 = amax(0., r0 - xabr) / P->dxabr;
            if ((tolil + tolir) != 0.)
                relb = ((tolil * r1) * (tolil * r1) + (tolir * r2) * (tolir * r2)) / (tolil * r1 + tolir * r2 + eps);
            relx = relb;
            r1 = 0.; r2 = 0.; relb = 0.;
            r0 = cm.y[n] * r;
            if (P->dyabd != 0.) r1 = amax(0., -r0 + yabd) / P->dyabd;
            if (P->dyabu != 0.) r2 = amax(0., r0 - yabu) / P->dyabu;
            if ((tolid + toliu) != 0.)
                relb = ((tolid * r1) * (tolid * r1) + (toliu * r2) * (toliu * r2)) / (tolid * r1 + toliu * r2 + eps);
            rely = relb;
            r1 = 0.; r2 = 0.; relb = 0.;
            r0 = cm.z[n];
            if (P->dzabd != 0.) r1 = amax(0., -r0 + zabd) / P->dzabd;
            if (P->dzabu != 0.) r2 = amax(0., r0 - zabu) / P->dzabu;
            if ((tolidz + toliuz) != 0.)
                relb = ((tolidz * r1) * (tolidz * r1) + (toliuz * r2) * (toliuz * r2)) / (tolidz * r1 + toliuz * r2 + eps);
            relz = relb;
            double alpha1 = (rely * rely + relx * relx) / (rely + relx + eps);
            hs->alpha[n] = (alpha1 * alpha1 + relz * relz) / (alpha1 + relz + eps);
        }
    }
    // ambient state (ref.f:177-207) and coefw (ref.f:250-252)
    hs->ue.assign(N, P->u0inf);
    hs->ve.assign(N, P->v0inf);
    hs->the.resize(N);
    hs->dthedz.resize(N);
    hs->coefw.resize(N);
    for (int n = 0; n < N; ++n) {
        if (P->lipps == 0) {
            hs->the[n] = P->tetbar * (1. + st * cm.z[n]);
            hs->dthedz[n] = P->tetbar * st * (double)P->implgw;
        } else {
            hs->the[n] = hs->th0[n];
            hs->dthedz[n] = hs->the[n] * st * (double)P->implgw;
        }
        double gth0 = g / hs->th0[n];
        double cw = 1. + 0.25 * (dt * dt) * gth0 * hs->dthedz[n];
        hs->coefw[n] = 1. / cw;
    }

    // edge loops in reference order on reference-indexed accumulators
    EdgeView ev{m};
    const int64_t nall = ev.n();
    const int64_t nint = m->nedge;
    const double *X = m->coord, *Y = m->coord + m->npoinx, *Z = m->coord + 2 * (size_t)m->npoinx;
    std::vector<double> rh0r(N), volr(N), cwr[2];
    for (int i = 0; i < N; ++i) { rh0r[i] = hs->rh0[perm[i]]; volr[i] = m->vol[i]; }
    cwr[0].assign(N, 1.0);
    cwr[1].resize(N);
    for (int i = 0; i < N; ++i) {
        double c = hs->coefw[perm[i]];
        cwr[0][i] = c * 0.0 + 1.0;
        cwr[1][i] = c * 1.0 + 0.0;
    }

    // beta_timestep_unstr(1) (ref.f:953-1109) with the reference's hard-coded box
    {
        double dom_x1 = 0., dom_x2 = 15000., dom_y1 = -6000., dom_y2 = 6000., dom_z1 = 0., dom_z2 = 6000.;
        double ddx = 10.e+06, hill_height = 1500.0;
        for (int64_t j = 0; j < nint; ++j) {
            int i1 = ev.i1(j), i2 = ev.i2(j);
            if (X[i1] != dom_x1 && X[i1] != dom_x2 && Y[i1] != dom_y1 && Y[i1] != dom_y2 &&
                Z[i1] != dom_z1 && Z[i1] != dom_z2 && X[i2] != dom_x1 && X[i2] != dom_x2 &&
                Y[i2] != dom_y1 && Y[i2] != dom_y2 && Z[i2] != dom_z1 && Z[i2] != dom_z2 &&
                Z[i1] > hill_height && Z[i2] > hill_height) {
                double h = amax(amax(std::fabs(ev.s(j, 0)), std::fabs(ev.s(j, 1))), std::fabs(ev.s(j, 2)));
                ddx = amin(amin(ddx, volr[i1] / h), volr[i2] / h);
            }
        }
        hs->betaunstr1 = 0.5 * ddx * ddx * 1;
    }

    // compute_d_unstr(1) (ref.f:1112-1284) and the horizontal part for the line preconditioner
    std::vector<double> dix(N, 0.), diy(N, 0.), diz(N, 0.);
    std::vector<double> hx(N, 0.), hy(N, 0.), hz(N, 0.);
    std::vector<double> Ta[2], Tc[2];
    for (int q = 0; q < 2; ++q) { Ta[q].assign(N, 0.); Tc[q].assign(N, 0.); }
    for (int64_t j = 0; j < nall; ++j) {
        int i1 = ev.i1(j), i2 = ev.i2(j);
        double sx = ev.s(j, 0), sy = ev.s(j, 1), sz = ev.s(j, 2);
        dix[i1] = dix[i1] + sx * sx * rh0r[i2] / volr[i2];
        dix[i2] = dix[i2] + sx * sx * rh0r[i1] / volr[i1];
        diy[i1] = diy[i1] + sy * sy * rh0r[i2] / volr[i2];
        diy[i2] = diy[i2] + sy * sy * rh0r[i1] / volr[i1];
        diz[i1] = diz[i1] + sz * sz * rh0r[i2] / volr[i2];
        diz[i2] = diz[i2] + sz * sz * rh0r[i1] / volr[i1];
        bool vert = X[i1] == X[i2] && Y[i1] == Y[i2];
        if (vert) {
            int lo = Z[i1] < Z[i2] ? i1 : i2, hi = lo == i1 ? i2 : i1;
            if (lo != i1) { sx = -sx; sy = -sy; sz = -sz; }
            double rhof = 0.5 * (rh0r[lo] + rh0r[hi]);
            double volf = 0.5 * (volr[lo] + volr[hi]);
            for (int q = 0; q < 2; ++q) {
                double cwf = 0.5 * (cwr[q][lo] + cwr[q][hi]);
                double T = (0.5 * dt) * ((sx * sx + sy * sy) + (sz * sz) * cwf) * rhof / volf;
                Tc[q][lo] = Tc[q][lo] + T;
                Ta[q][hi] = Ta[q][hi] + T;
            }
        } else {
            hx[i1] = hx[i1] + sx * sx * rh0r[i2] / volr[i2];
            hx[i2] = hx[i2] + sx * sx * rh0r[i1] / volr[i1];
            hy[i1] = hy[i1] + sy * sy * rh0r[i2] / volr[i2];
            hy[i2] = hy[i2] + sy * sy * rh0r[i1] / volr[i1];
            hz[i1] = hz[i1] + sz * sz * rh0r[i2] / volr[i2];
            hz[i2] = hz[i2] + sz * sz * rh0r[i1] / volr[i1];
        }
    }
    hs->d1.resize(N);
    for (int i = 0; i < N; ++i)
        hs->d1[perm[i]] = -0.5 * dt * (dix[i] + diy[i] + diz[i]) / (4 * volr[i] * rh0r[i]);

    // vertical-line preconditioner: rows, then the Thomas factorisation per column
    for (int q = 0; q < 2; ++q) {
        std::vector<double> a(N), b(N), c(N);
        for (int i = 0; i < N; ++i) {
            double vr = volr[i] * rh0r[i];
            double dh = -((0.5 * dt) * ((hx[i] + hy[i]) + hz[i])) / ((4. * volr[i]) * rh0r[i]);
            int n = perm[i];
            a[n] = Ta[q][i] / vr;
            c[n] = Tc[q][i] / vr;
            b[n] = (dh - a[n]) - c[n];
        }
        if (q == 1) {
            hs->lbabs.resize(N);
            for (int n = 0; n < N; ++n) hs->lbabs[n] = (float)std::fabs(b[n]);
        }
        size_t nint_sz = (size_t)((NC + 31) / 32) * 32 * L;
        hs->la[q].assign(nint_sz, 0.);
        hs->lm[q].assign(nint_sz, 1.);
        hs->lcp[q].assign(nint_sz, 0.);
        for (int col = 0; col < NC; ++col) {
            double cpprev = 0.;
            for (int k = 0; k < L; ++k) {
                int n = col * L + k;
                double mm = k == 0 ? b[n] : b[n] - a[n] * cpprev;
                double cp = c[n] / mm;
                int64_t li = line_index(col, k, L);
                hs->la[q][li] = a[n];
                hs->lm[q][li] = 1. / mm;         // the solve multiplies by the inverse pivot
                hs->lcp[q][li] = cp;
                cpprev = cp;
            }
        }
    }
    if (P->iprc == 4) mpg_wide_coeffs(P, m, cm, rh0r, volr, cwr, hs);
    return MPG_OK;
}

// ---- iprc = 4: the column blocks of laplc itself.  laplc's gradient uses face averages
// (p_n + p_j)/2, so in a column it couples level k with k and k+-2 only: the block is
// tridiagonal on the even and on the odd levels.  With S_k the upward face between levels k and
// k+1, s_m = (0.5 dt/vol_m)(1, 1, cw_m) and P_m the bcv(.,0) projection at node m:
//   A[k][k+2] = ((S_k/2) . rh0_{k+1} P_{k+1}(s_{k+1} (*) S_{k+1}/2)) / (vol_k rh0_k)
//   A[k][k-2] = ((S_{k-1}/2) . rh0_{k-1} P_{k-1}(s_{k-1} (*) S_{k-2}/2)) / (vol_k rh0_k)
//   A[k][k]   = (sum over faces f of k, neighbour j: -(S_f/2) . rh0_j P_j(s_j (*) S_f/2)
//                + e_k . rh0_k P_k(s_k (*) e_k)) / (vol_k rh0_k),
// e_k = (sum of k's outward faces)/2, plus its boundary faces sbb when iper = 0.  The entries are
// accumulated in the reference's edge order, then factorised per parity chain (Thomas from the
// bottom) into the interleaved layout of the line solve.
namespace {
struct WideCtx {
    const mpg_params *P;
    const mpg_mesh_ref *m;
    const std::vector<double> &rh0r, &volr, &cw;
    std::vector<int32_t> bst, blst;
    double dt;
    void bcv_vec(int i, double v[3]) const {
        const bool per = (P->isfera == 1 || P->iper == 2);
        for (int b = bst[i]; b < bst[i + 1]; ++b) {
            const int q = blst[b];
            const int t = m->ibpoin[(size_t)m->nfacesx + q];
            const double a1 = m->anp[q], a2 = m->anp[(size_t)m->nfacesx + q], a3 = m->anp[2 * (size_t)m->nfacesx + q];
            if (t == 11 || (!per && (t == 5 || t == 6))) {
                double vn = v[0] * a1 + v[1] * a2 + v[2] * a3;
                v[0] = v[0] - a1 * vn;
                v[1] = v[1] - a2 * vn;
                v[2] = v[2] - a3 * vn;
            }
            if (!per && (t == 7 || t == 8)) v[0] = 0.;
        }
    }
    // (a/2) . rh0_j P_j(s_j (*) b/2)
    double path(int j, const double a[3], const double b[3]) const {
        const double h = 0.5 * (dt / volr[j]);
        const double sc[3] = {h / (1.0 * 1.0), h / (1.0 * 1.0), h * cw[j]};
        double v[3];
        for (int d = 0; d < 3; ++d) v[d] = sc[d] * (0.5 * b[d]);
        bcv_vec(j, v);
        const double r = rh0r[j];
        return (0.5 * a[0]) * (r * v[0]) + (0.5 * a[1]) * (r * v[1]) + (0.5 * a[2]) * (r * v[2]);
    }
};
}  // namespace

void mpg_wide_entries(const mpg_params *P, const mpg_mesh_ref *m, const HostColumnMesh &cm,
                      const std::vector<double> &rh0r, const std::vector<double> &volr,
                      const std::vector<double> &cw, std::vector<double> &lo, std::vector<double> &dg,
                      std::vector<double> &hi) {
    const int N = cm.N, L = cm.L;
    WideCtx W{P, m, rh0r, volr, cw, {}, {}, P->delt};
    W.bst.assign(N + 1, 0);
    W.blst.assign(m->nboun, 0);
    for (int b = 0; b < m->nboun; ++b) W.bst[m->ibpoin[b] - 1 + 1]++;
    for (int i = 0; i < N; ++i) W.bst[i + 1] += W.bst[i];
    {
        std::vector<int32_t> fill(N, 0);
        for (int b = 0; b < m->nboun; ++b) {
            const int i = m->ibpoin[b] - 1;
            W.blst[W.bst[i] + fill[i]++] = b;
        }
    }
    EdgeView ev{m};
    const int64_t nall = ev.n();
    lo.assign(N, 0.); dg.assign(N, 0.); hi.assign(N, 0.);
    std::vector<double> ex(N, 0.), ey(N, 0.), ez(N, 0.), sux(N, 0.), suy(N, 0.), suz(N, 0.);
    for (int64_t j = 0; j < nall; ++j) {
        const int i1 = ev.i1(j), i2 = ev.i2(j);
        const double S[3] = {ev.s(j, 0), ev.s(j, 1), ev.s(j, 2)};
        ex[i1] += S[0]; ey[i1] += S[1]; ez[i1] += S[2];
        ex[i2] -= S[0]; ey[i2] -= S[1]; ez[i2] -= S[2];
        dg[i1] = dg[i1] - W.path(i2, S, S);
        dg[i2] = dg[i2] - W.path(i1, S, S);
    }
    for (int i = 0; i < N; ++i) {
        double e3[3] = {0.5 * ex[i], 0.5 * ey[i], 0.5 * ez[i]};
        if (P->isfera == 0 && P->iper == 0)
            for (int b = W.bst[i]; b < W.bst[i + 1]; ++b) {
                const int q = W.blst[b];
                e3[0] += m->sbb[q];
                e3[1] += m->sbb[(size_t)m->nfacesx + q];
                e3[2] += m->sbb[2 * (size_t)m->nfacesx + q];
            }
        const double a2[3] = {2. * e3[0], 2. * e3[1], 2. * e3[2]};
        dg[i] = dg[i] + W.path(i, a2, a2);
    }
    // upward face of each node (reference index of the lower end)
    auto up = [&](int i) { const int n = cm.perm[i]; return (n % L) + 1 < L ? cm.iperm[n + 1] : -1; };
    auto dn = [&](int i) { const int n = cm.perm[i]; return (n % L) > 0 ? cm.iperm[n - 1] : -1; };
    for (int64_t j = 0; j < nall; ++j) {
        const int i1 = ev.i1(j), i2 = ev.i2(j);
        if (cm.perm[i1] / L != cm.perm[i2] / L) continue;
        const double sg = up(i1) == i2 ? 1. : -1.;
        const int lower = sg > 0 ? i1 : i2;
        sux[lower] = sg * ev.s(j, 0);
        suy[lower] = sg * ev.s(j, 1);
        suz[lower] = sg * ev.s(j, 2);
    }
    for (int i = 0; i < N; ++i) {
        const double vr = volr[i] * rh0r[i];
        const int u1 = up(i), d1 = dn(i);
        if (u1 >= 0 && up(u1) >= 0) {
            const double a[3] = {sux[i], suy[i], suz[i]}, b[3] = {sux[u1], suy[u1], suz[u1]};
            hi[i] = W.path(u1, a, b) / vr;
        }
        if (d1 >= 0 && dn(d1) >= 0) {
            const int d2 = dn(d1);
            const double a[3] = {sux[d1], suy[d1], suz[d1]}, b[3] = {sux[d2], suy[d2], suz[d2]};
            lo[i] = W.path(d1, a, b) / vr;
        }
        dg[i] = dg[i] / vr;
    }
}

void mpg_wide_coeffs(const mpg_params *P, const mpg_mesh_ref *m, const HostColumnMesh &cm,
                     const std::vector<double> &rh0r, const std::vector<double> &volr,
                     const std::vector<double> *cwr, HostStatic *hs) {
    const int NC = cm.NC, L = cm.L;
    const size_t nint_sz = (size_t)((NC + 31) / 32) * 32 * L;
    for (int q = 0; q < 2; ++q) {
        std::vector<double> lo, dg, hi;
        mpg_wide_entries(P, m, cm, rh0r, volr, cwr[q], lo, dg, hi);
        hs->wa[q].assign(nint_sz, 0.);
        hs->wm[q].assign(nint_sz, 1.);
        hs->wcp[q].assign(nint_sz, 0.);
        for (int col = 0; col < NC; ++col)
            for (int par = 0; par < 2; ++par) {
                double cpprev = 0.;
                for (int k = par; k < L; k += 2) {
                    const int i = cm.iperm[col * L + k];
                    const double mm = k < 2 ? dg[i] : dg[i] - lo[i] * cpprev;
                    const double cp = hi[i] / mm;
                    const int64_t li = line_index(col, k, L);
                    hs->wa[q][li] = lo[i];
                    hs->wm[q][li] = 1. / mm;
                    hs->wcp[q][li] = cp;
                    cpprev = cp;
                }
            }
    }
}

int32_t mpg_laplc_schedule(const HostColumnMesh &cm, int per, int lag, std::vector<int32_t> &sched,
                           std::vector<int32_t> &dptr, std::vector<int2> &drng) {
    const int64_t L = cm.L, PL = (cm.L + 1) / 2, NP = (int64_t)cm.NC * PL;
    const int32_t NG = (int32_t)((cm.N + per - 1) / per), ND = (int32_t)((NP + per - 1) / per);
    dptr.assign(1, 0);
    drng.clear();
    std::vector<int32_t> last(ND);
    std::vector<int2> r;
    for (int32_t d = 0; d < ND; ++d) {
        const int64_t t0 = (int64_t)d * per, t1 = std::min<int64_t>(NP, t0 + per);
        const int32_t c0 = (int32_t)(t0 / PL), c1 = (int32_t)((t1 - 1) / PL);
        r.clear();
        auto need = [&](int32_t col) {      // every level of column col
            r.push_back(make_int2((int32_t)(col * L / per), (int32_t)(((int64_t)col * L + L - 1) / per)));
        };
        for (int32_t c = c0; c <= c1; ++c) {
            need(c);
            for (int32_t j = cm.cptr[c]; j < cm.cptr[c + 1]; ++j)
                if (cm.cadj[j].x >= 0) need(cm.cadj[j].y);
        }
        std::sort(r.begin(), r.end(), [](int2 a, int2 b) { return a.x < b.x || (a.x == b.x && a.y < b.y); });
        int2 cur = r[0];
        for (size_t i = 1; i < r.size(); ++i) {
            if (r[i].x <= cur.y + 1) cur.y = std::max(cur.y, r[i].y);
            else { drng.push_back(cur); cur = r[i]; }
        }
        drng.push_back(cur);
        last[d] = std::min(NG - 1, cur.y + std::max(lag, 0));
        dptr.push_back((int32_t)drng.size());
    }
    // gradient items in order; each divergence item `lag` gradient items after its last dependency
    std::vector<int32_t> order(ND);
    for (int32_t d = 0; d < ND; ++d) order[d] = d;
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return last[a] < last[b]; });
    sched.clear();
    sched.reserve((size_t)NG + ND);
    size_t q = 0;
    for (int32_t g = 0; g < NG; ++g) {
        sched.push_back(g);
        while (q < order.size() && last[order[q]] == g) sched.push_back(-(order[q++] + 1));
    }
    return NG;
}

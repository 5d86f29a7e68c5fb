// Host check of mpg_laplc_schedule (src_b200/csrc/setup.cpp), the work order of the single-launch
// laplc: on doubly periodic triangulated column grids, every gradient and divergence item appears
// exactly once, and every gradient item a divergence item reads (its own columns and their
// horizontal neighbours, all levels) lies inside one of its ranges and comes earlier in the order.
// Prints one line per case and exits non-zero on the first violation.
#include <cstdio>
#include <set>
#include <string>

#include "../../src_b200/csrc/mpgcr_internal.h"

int mpg_fail(int code, const std::string &) { return code; }
void mpg_set_error(const std::string &) {}

int main() {
    int bad = 0;
    for (int nx : {4, 8, 37, 96})
        for (int L : {1, 2, 9, 81})
            for (int per : {256, 64})
                for (int lag : {0, 592}) {
                    HostColumnMesh cm;
                    cm.NC = nx * nx; cm.L = L; cm.N = cm.NC * L;
                    cm.cptr.push_back(0);
                    const int nb[6][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}, {1, 1}, {-1, -1}};
                    for (int c = 0; c < cm.NC; ++c) {
                        const int i = c % nx, j = c / nx;
                        cm.cadj.push_back(make_int2(MPG_ADJ_BELOW, 0));
                        for (const auto &d : nb)
                            cm.cadj.push_back(make_int2(2, ((j + d[1] + nx) % nx) * nx + (i + d[0] + nx) % nx));
                        cm.cadj.push_back(make_int2(-2, 0));
                        cm.cptr.push_back((int)cm.cadj.size());
                    }
                    std::vector<int32_t> s, dp;
                    std::vector<int2> dr;
                    const int NG = mpg_laplc_schedule(cm, per, lag, s, dp, dr);
                    const int PL = (L + 1) / 2;
                    const long NP = (long)cm.NC * PL;
                    const int ND = (int)((NP + per - 1) / per);
                    bool ok = NG == (cm.N + per - 1) / per && (int)s.size() == NG + ND && (int)dp.size() == ND + 1;
                    std::vector<int> pos(NG, -1), seen(ND, 0);
                    for (int q = 0; ok && q < (int)s.size(); ++q) {
                        const int it = s[q];
                        if (it >= 0) {
                            ok = it < NG && pos[it] < 0;
                            if (ok) pos[it] = q;
                            continue;
                        }
                        const int d = -it - 1;
                        ok = d < ND && !seen[d]++;
                        std::set<int> need;
                        for (long t = (long)d * per; ok && t < NP && t < (long)(d + 1) * per; ++t) {
                            const int c = (int)(t / PL);
                            auto add = [&](int col) {
                                for (int k = 0; k < L; ++k) need.insert((int)(((long)col * L + k) / per));
                            };
                            add(c);
                            for (int e = cm.cptr[c]; e < cm.cptr[c + 1]; ++e)
                                if (cm.cadj[e].x >= 0) add(cm.cadj[e].y);
                        }
                        for (int g : need) {
                            bool in = false;
                            for (int r = dp[d]; r < dp[d + 1]; ++r) in = in || (g >= dr[r].x && g <= dr[r].y);
                            ok = ok && in && pos[g] >= 0 && pos[g] < q;
                        }
                    }
                    for (int g = 0; ok && g < NG; ++g) ok = pos[g] >= 0;
                    for (int d = 0; ok && d < ND; ++d) ok = seen[d] == 1;
                    std::printf("nx=%d L=%d per=%d lag=%d items=%d+%d %s\n", nx, L, per, lag, NG, ND, ok ? "ok" : "BAD");
                    if (!ok) bad = 1;
                }
    return bad;
}

// Host check of the gather-component grouping (test infrastructure, built by
// tests/test_gather_components.py with g++): for every ghost pattern and vertex restriction
// over a range of boundary options, applying a map component by component (per plane, every
// source of a component read before any of its destinations is written, as k_gather does)
// gives bit for bit what applying it with all reads before all writes gives (the two-pass
// semantics through scratch), and the grouped map is a permutation of the original entries.
#include "salec_kernels.h"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

using namespace salec;

// any fixed function of (op, value) serves: the check is about the order of reads and writes
static double fop(unsigned op, double x) { return x * (1.0 + 0.25 * op) + op; }

static int check(const GatherMap &m, int npts, int ncomp, std::mt19937_64 &rng, int &maxc, long &groups)
{
    std::vector<double> base((size_t)ncomp * npts);
    std::uniform_real_distribution<double> U(-1.0, 1.0);
    for (double &v : base) v = U(rng);
    std::vector<double> a = base, tmp(m.dst.size() * ncomp);
    for (size_t e = 0; e < m.dst.size(); ++e)
        for (int c = 0; c < ncomp; ++c) tmp[e * ncomp + c] = fop((m.ops[e] >> (3 * c)) & 7u, a[(size_t)c * npts + m.src[e]]);
    for (size_t e = 0; e < m.dst.size(); ++e)
        for (int c = 0; c < ncomp; ++c) a[(size_t)c * npts + m.dst[e]] = tmp[e * ncomp + c];
    GatherMap g;
    std::vector<int> cs;
    if (!group_gather_components(m, g, cs)) return 2;
    if (g.dst.size() != m.dst.size() || cs.front() != 0 || cs.back() != (int)g.dst.size()) return 3;
    std::vector<long long> e1, e2;
    for (size_t e = 0; e < m.dst.size(); ++e) {
        e1.push_back(((long long)m.dst[e] << 40) ^ ((long long)m.src[e] << 8) ^ m.ops[e]);
        e2.push_back(((long long)g.dst[e] << 40) ^ ((long long)g.src[e] << 8) ^ g.ops[e]);
    }
    std::sort(e1.begin(), e1.end());
    std::sort(e2.begin(), e2.end());
    if (e1 != e2) return 4;
    std::vector<double> b = base;
    for (size_t k = 0; k + 1 < cs.size(); ++k) {
        const int lo = cs[k], hi = cs[k + 1];
        maxc = std::max(maxc, hi - lo);
        ++groups;
        for (int c = 0; c < ncomp; ++c) {
            double v[SALEC_GATHER_MAX_COMPONENT];
            for (int e = lo; e < hi; ++e) v[e - lo] = fop((g.ops[e] >> (3 * c)) & 7u, b[(size_t)c * npts + g.src[e]]);
            for (int e = lo; e < hi; ++e) b[(size_t)c * npts + g.dst[e]] = v[e - lo];
        }
    }
    return memcmp(a.data(), b.data(), a.size() * sizeof(double)) == 0 ? 0 : 1;
}

int main()
{
    std::mt19937_64 rng(12345);
    const int opts[6] = {0, 2, 3, 5, 7, 9};
    const GhostPattern pats[6] = {GP_ALWAYS_COPY, GP_NORMAL, GP_VELOCITY_INC, GP_VELOCITY, GP_STRESS, GP_DENSITY};
    long maps = 0, shared = 0, groups = 0;
    int maxc = 0;
    const int sizes[2][2] = {{17, 13}, {40, 33}};
    for (const auto &sz : sizes) {
        const int nx = sz[0], ny = sz[1];
        const int enx = nx + 4, eny = ny + 4, vnx = nx + 5, vny = ny + 5, P = ((vnx + 31) / 32) * 32;
        for (int a = 0; a < 6; ++a)
            for (int b = 0; b < 6; ++b)
                for (int c = 0; c < 6; ++c)
                    for (int d = 0; d < 6; ++d) {
                        const int go[4] = {opts[a], opts[b], opts[c], opts[d]};
                        for (int nc : {1, 2, 4}) {
                            for (int p = 0; p < 7; ++p) {
                                GatherMap m = p < 6 ? build_ghost_map(enx, eny, P, nc, go, pats[p])
                                                    : build_restrict_map(vnx, vny, P, nc, go);
                                ++maps;
                                if (!m.needs_scratch) continue;
                                ++shared;
                                const int npts = P * (p < 6 ? eny : vny);
                                const int rc = check(m, npts, nc, rng, maxc, groups);
                                if (rc) {
                                    printf("FAIL rc=%d size %dx%d go %d %d %d %d ncomp %d pattern %d\n", rc, nx, ny, go[0],
                                           go[1], go[2], go[3], nc, p);
                                    return 1;
                                }
                            }
                        }
                    }
    }
    printf("OK maps=%ld with_shared_points=%ld components=%ld largest=%d\n", maps, shared, groups, maxc);
    return 0;
}

// Boundary tables of the reference turned into parallel gather maps.
//
// The reference fills ghost cells (src/mpi_vec/mpi_vec_ght.c:12-154, 279-357, 698-752) and
// restricts boundary vertices (:440-734) by walking a table sequentially, in point order,
// where each entry copies (or negates, takes abs of, zeroes) whole points; later entries
// can read points earlier entries wrote and overwrite them (last writer wins, e.g. cell
// (1,1) is written by the entries of (0,0), (1,0) and (0,1)). Replaying that walk here once,
// symbolically, gives for every written point the single original point it ends up copied
// from and the per-component transform, so the device can apply the whole table as one
// parallel gather with exactly the reference's result.
#include "salec_kernels.h"

#include <algorithm>
#include <cstring>
#include <unordered_map>

namespace salec {

namespace {

// ght_opt numbering of src/mpi_vec/mpi_vec_types.h:74-95
enum {
    GHT_OUTFLOW = 0, GHT_OUTFLOW_VERTEX = 1, GHT_FIXED = 2, GHT_ZERO = 3, GHT_CLEAN = 4, GHT_MIRROR = 5,
    GHT_FREESLIP = 6, GHT_REVERSE_VEL_Y = 7, GHT_REVERSE_VEL_ABSY = 8, GHT_REVERSE_VEL_X = 9,
    GHT_REVERSE_STE_1 = 10, GHT_COPY_STE = 11, RST_X_ZERO = 12, RST_Y_ZERO = 13, RST_Y_POSITIVE = 14,
    RST_X_POSITIVE = 15, RST_ZERO = 16, RST_NONE = 17
};
enum { OP_ID = 0, OP_NEG = 1, OP_ABS = 2, OP_NABS = 3, OP_ZERO = 4, OP_NZERO = 5 };
constexpr int MAXC = 10;

// f o g for the transform set {x, -x, |x|, -|x|, +0, -0}
int compose(int f, int g)
{
    switch (f) {
    case OP_ID: return g;
    case OP_ZERO: return OP_ZERO;
    case OP_NZERO: return OP_NZERO;
    case OP_NEG: {
        static const int t[6] = {OP_NEG, OP_ID, OP_NABS, OP_ABS, OP_NZERO, OP_ZERO};
        return t[g];
    }
    case OP_ABS: {
        static const int t[6] = {OP_ABS, OP_ABS, OP_ABS, OP_ABS, OP_ZERO, OP_ZERO};
        return t[g];
    }
    default: {
        static const int t[6] = {OP_NABS, OP_NABS, OP_NABS, OP_NABS, OP_NZERO, OP_NZERO};
        return t[g];
    }
    }
}

struct Sym {
    int src;
    unsigned char op[MAXC];
};

struct Replay {
    std::vector<Sym> cur;
    std::vector<char> written;
    int ncomp;
    Replay(int npts, int nc) : cur(npts), written(npts, 0), ncomp(nc)
    {
        for (int k = 0; k < npts; ++k) {
            cur[k].src = k;
            memset(cur[k].op, OP_ID, sizeof(cur[k].op));
        }
    }
    // dst <- f(src) component-wise, using the current (already replayed) value of src
    void write(int dst, int src, const unsigned char *f)
    {
        Sym s = cur[src];
        Sym r;
        r.src = s.src;
        for (int c = 0; c < MAXC; ++c) r.op[c] = (unsigned char)compose(c < ncomp ? f[c] : OP_ID, s.op[c]);
        cur[dst] = r;
        written[dst] = 1;
    }
    GatherMap finish() const
    {
        GatherMap m;
        const int n = (int)cur.size();
        std::vector<char> is_dst(n, 0);
        for (int k = 0; k < n; ++k) {
            if (!written[k]) continue;
            bool ident = cur[k].src == k;
            unsigned ops = 0;
            for (int c = 0; c < ncomp; ++c) {
                ops |= (unsigned)cur[k].op[c] << (3 * c);
                if (cur[k].op[c] != OP_ID) ident = false;
            }
            if (ident) continue;
            m.dst.push_back(k);
            m.src.push_back(cur[k].src);
            m.ops.push_back(ops);
            is_dst[k] = 1;
        }
        for (size_t e = 0; e < m.src.size(); ++e) {
            bool reads = false;
            for (int c = 0; c < ncomp; ++c) {
                int op = (m.ops[e] >> (3 * c)) & 7;
                if (op != OP_ZERO && op != OP_NZERO) reads = true;
            }
            if (reads && is_dst[m.src[e]]) m.needs_scratch = true;
        }
        return m;
    }
};

} // namespace

GatherMap build_ghost_map(int enx, int eny, int P, int ncomp, const int go[4], GhostPattern pat)
{
    // local ghost options per side (left, right, bottom, top): set_ghost_pattern
    int lg[4];
    switch (pat) {
    case GP_ALWAYS_COPY: lg[0] = lg[1] = lg[2] = lg[3] = GHT_OUTFLOW; break;
    case GP_NORMAL: for (int k = 0; k < 4; ++k) lg[k] = go[k]; break;
    case GP_VELOCITY_INC:
        for (int k = 0; k < 4; ++k) lg[k] = go[k];
        if (go[0] == GHT_MIRROR) lg[0] = GHT_REVERSE_VEL_X;
        if (go[3] == GHT_OUTFLOW) lg[3] = GHT_REVERSE_VEL_ABSY;
        break;
    case GP_VELOCITY:
        for (int k = 0; k < 4; ++k) lg[k] = GHT_OUTFLOW_VERTEX;
        if (go[0] == GHT_MIRROR) lg[0] = GHT_REVERSE_VEL_X;
        break;
    case GP_STRESS:
        lg[0] = lg[1] = lg[2] = lg[3] = GHT_COPY_STE;
        if (go[0] == GHT_MIRROR) lg[0] = GHT_REVERSE_STE_1;
        break;
    case GP_DENSITY:
    default:
        lg[0] = lg[1] = lg[2] = GHT_OUTFLOW;
        lg[3] = GHT_CLEAN;
        break;
    }
    // the table indexes points x-fastest over enx x eny; device index is i + P*j
    Replay rp(P * eny, ncomp);
    auto pt = [&](int i, int j) { return i + P * j; };
    auto clampx = [&](int x) { return std::min(std::max(x, 2), enx - 3); };
    auto clampy = [&](int y) { return std::min(std::max(y, 2), eny - 3); };
    unsigned char id[MAXC], neg[MAXC], zero[MAXC];
    memset(id, OP_ID, MAXC);
    memset(neg, OP_NEG, MAXC);
    memset(zero, OP_ZERO, MAXC);
    for (int j = 0; j < eny; ++j) {
        for (int i = 0; i < enx; ++i) {
            const bool L = i == 0, R = i == enx - 1, B = j == 0, T = j == eny - 1;
            if (!(L || R || B || T)) continue;
            int ax = i, ay = j, bx = i, by = j, cx = i, cy = j;
            if (L) { ax = i + 1; bx = i + 2; cx = i + 3; }
            if (R) { ax = i - 1; bx = i - 2; cx = i - 3; }
            if (B) { ay = j + 1; by = j + 2; cy = j + 3; }
            if (T) { ay = j - 1; by = j - 2; cy = j - 3; }
            // corners: references that are still ghosts move into the send section
            if (std::min(i, enx - 1 - i) + std::min(j, eny - 1 - j) <= 1) {
                bx = clampx(bx); by = clampy(by);
                cx = clampx(cx); cy = clampy(cy);
            }
            int opt = L ? lg[0] : (R ? lg[1] : (B ? lg[2] : lg[3]));
            const int g = pt(i, j), a = pt(ax, ay), b = pt(bx, by), c = pt(cx, cy);
            unsigned char f[MAXC];
            switch (opt) {
            case GHT_OUTFLOW:
            case GHT_COPY_STE:
                rp.write(g, c, id);
                rp.write(a, b, id);
                break;
            case GHT_FIXED:
                rp.write(g, c, neg);
                rp.write(a, b, neg);
                break;
            case GHT_ZERO:
                rp.write(g, g, zero);
                rp.write(a, a, zero);
                break;
            case GHT_REVERSE_VEL_Y:
            case GHT_REVERSE_VEL_X:
            case GHT_REVERSE_VEL_ABSY:
            case GHT_REVERSE_STE_1: {
                memcpy(f, id, MAXC);
                if (opt == GHT_REVERSE_VEL_X) f[0] = OP_NEG;
                else if (opt == GHT_REVERSE_VEL_ABSY) f[1] = OP_ABS;
                else f[1] = OP_NEG;
                rp.write(g, c, f);
                rp.write(a, b, f);
                break;
            }
            case GHT_OUTFLOW_VERTEX:
                rp.write(g, c, id);
                rp.write(a, c, id);
                rp.write(b, c, id);
                break;
            case GHT_CLEAN:
                rp.write(a, a, zero);
                rp.write(b, b, zero);
                rp.write(g, g, zero);
                break;
            default:
                break;   // the reference's ghost_pad_fill returns without writing
            }
        }
    }
    return rp.finish();
}

GatherMap build_restrict_map(int vnx, int vny, int P, int ncomp, const int go[4])
{
    // set_restrict_pattern (src/mpi_vec/mpi_vec_ght.c:545-655)
    int ro[4] = {RST_NONE, RST_NONE, RST_NONE, RST_NONE};   // left, right, bottom, top
    switch (go[1]) {
    case GHT_OUTFLOW: ro[1] = RST_NONE; break;
    case GHT_FREESLIP: case GHT_REVERSE_VEL_X: ro[1] = RST_X_ZERO; break;
    default: ro[1] = RST_ZERO; break;
    }
    switch (go[2]) {
    case GHT_OUTFLOW: ro[2] = RST_NONE; break;
    case GHT_FREESLIP: case GHT_REVERSE_VEL_Y: ro[2] = RST_Y_ZERO; break;
    default: ro[2] = RST_ZERO; break;
    }
    switch (go[0]) {
    case GHT_REVERSE_VEL_X: case GHT_MIRROR: ro[0] = RST_X_ZERO; break;
    default: ro[0] = RST_NONE; break;
    }
    const int pad = 2;
    Replay rp(P * vny, ncomp);
    auto pt = [&](int i, int j) { return i + P * j; };
    unsigned char id[MAXC];
    memset(id, OP_ID, MAXC);
    for (int j = 0; j < vny; ++j) {
        for (int i = 0; i < vnx; ++i) {
            const bool L = i == pad, R = i == vnx - 1 - pad, B = j == pad, T = j == vny - 1 - pad;
            if (!(L || R || B || T)) continue;
            int ax = i, ay = j, bx = i, by = j;
            if (L) { ax = i + 1; bx = i - 1; }
            if (R) { ax = i - 1; bx = i + 1; }
            if (B) { ay = j + 1; by = j - 1; }
            if (T) { ay = j - 1; by = j + 1; }
            int opt = RST_NONE;
            if (L) opt = ro[0];
            if (R) opt = ro[1];
            if (T) opt = ro[3];
            if (B) opt = ro[2];
            if (B && R && ro[2] != RST_NONE && ro[1] != RST_NONE) opt = RST_ZERO;
            const int d = pt(i, j), a = pt(ax, ay), b = pt(bx, by);
            rp.write(b, a, id);
            unsigned char f[MAXC];
            memcpy(f, id, MAXC);
            switch (opt) {
            case RST_ZERO: for (int c = 0; c < MAXC; ++c) f[c] = OP_ZERO; break;
            case RST_X_ZERO: f[0] = OP_ZERO; break;
            case RST_Y_ZERO: f[1] = OP_ZERO; break;
            case RST_Y_POSITIVE: f[1] = OP_ABS; break;
            case RST_X_POSITIVE: f[0] = OP_ABS; break;
            default: break;
            }
            rp.write(d, a, f);
        }
    }
    return rp.finish();
}

// Entries of a map whose sources include destinations, grouped into connected components of
// the read/write relation (union of each entry's destination and source point), components in
// order of their first entry and entries in map order within each; false when a component has
// more than SALEC_GATHER_MAX_COMPONENT entries.
bool group_gather_components(const GatherMap &m, GatherMap &out, std::vector<int> &cstart)
{
    std::unordered_map<int, int> id;
    std::vector<int> parent;
    auto node = [&](int pt) {
        auto it = id.find(pt);
        if (it != id.end()) return it->second;
        const int n = (int)parent.size();
        id.emplace(pt, n);
        parent.push_back(n);
        return n;
    };
    auto root = [&](int x) {
        while (parent[x] != x) { parent[x] = parent[parent[x]]; x = parent[x]; }
        return x;
    };
    const size_t ne = m.dst.size();
    std::vector<int> en(ne);
    for (size_t e = 0; e < ne; ++e) {
        const int a = root(node(m.dst[e])), b = root(node(m.src[e]));
        if (a != b) parent[a] = b;
        en[e] = node(m.dst[e]);
    }
    std::unordered_map<int, int> comp_of;   // root -> component number (first-entry order)
    std::vector<std::vector<int>> comps;
    for (size_t e = 0; e < ne; ++e) {
        const int r = root(en[e]);
        auto it = comp_of.find(r);
        if (it == comp_of.end()) {
            it = comp_of.emplace(r, (int)comps.size()).first;
            comps.emplace_back();
        }
        comps[it->second].push_back((int)e);
        if ((int)comps[it->second].size() > SALEC_GATHER_MAX_COMPONENT) return false;
    }
    out = GatherMap();
    cstart.assign(1, 0);
    for (const auto &c : comps) {
        for (int e : c) {
            out.dst.push_back(m.dst[e]);
            out.src.push_back(m.src[e]);
            out.ops.push_back(m.ops[e]);
        }
        cstart.push_back((int)out.dst.size());
    }
    return true;
}

} // namespace salec

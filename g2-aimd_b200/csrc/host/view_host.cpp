// view_host.cpp - views of a host CSR around a set of roots, the greedy bin
// partition that sizes them, and the radii a query plan needs.
//
// Replaces the host side of the reference's out-of-core path:
// ViewBin::Materialize / ExtendFromSource (view/view_bin.h:40-159) and the
// per-query hop of Plan::FindRoot (system/plan.h:51-73).  The pipeline that
// uploads views and runs the enumeration over them is in runtime.cu.
#include "view_host.h"

#include <algorithm>
#include <cstring>

#include "g2_aimd.h"

namespace g2view {

namespace {
inline uint64_t align16(uint64_t x) { return (x + 15u) & ~15ull; }
}  // namespace

Layout::Layout(const Sizes &s) {
    fo = align16(8ull * (s.n + 1));
    ci = align16(fo + 4ull * s.n);
    src = align16(ci + 4ull * s.m);
    bytes = align16(src + 4ull * s.nsrc);
}

void Builder::release() {
    for (uint64_t e : ball_) mark_[e >> 4] = kNone;
    ball_.clear();
    src_.clear();
    deg_.clear();
}

Sizes Builder::plan(const uint32_t *src, uint64_t nsrc, uint32_t radius, uint32_t row_radius,
                    uint32_t min_root_degree) {
    if (mark_.size() != n_) mark_.assign(n_, kNone);
    release();
    row_radius_ = row_radius;
    // multi-source BFS: depth of every vertex within `radius` of a kept source
    std::vector<uint32_t> frontier, next;
    for (uint64_t i = 0; i < nsrc; i++) {
        const uint32_t s = src[i];
        if (rp_[s + 1] - rp_[s] < min_root_degree) continue;
        src_.push_back(s);
        if (mark_[s] == kNone) {
            mark_[s] = 0;
            ball_.push_back((uint64_t)s << 4);
            frontier.push_back(s);
        }
    }
    for (uint32_t d = 0; d < radius && !frontier.empty(); d++) {
        next.clear();
        for (uint32_t x : frontier)
            for (uint64_t e = rp_[x]; e < rp_[x + 1]; e++) {
                const uint32_t u = ci_[e];
                if (mark_[u] != kNone) continue;
                mark_[u] = d + 1;
                ball_.push_back(((uint64_t)u << 4) | std::min<uint32_t>(d + 1, 15u));
                next.push_back(u);
            }
        frontier.swap(next);
    }
    // ascending global order = local ids; marks become local ids
    std::sort(ball_.begin(), ball_.end());
    for (uint64_t i = 0; i < ball_.size(); i++) mark_[ball_[i] >> 4] = (uint32_t)i;
    // view degrees and forward degrees
    Sizes s;
    s.n = ball_.size();
    s.nsrc = src_.size();
    deg_.assign(s.n, 0u);
    for (uint64_t i = 0; i < s.n; i++) {
        if ((ball_[i] & 15u) > row_radius) continue;
        const uint32_t g = (uint32_t)(ball_[i] >> 4);
        uint32_t d = 0, back = 0;
        for (uint64_t e = rp_[g]; e < rp_[g + 1]; e++) {
            const uint32_t l = mark_[ci_[e]];
            if (l == kNone) continue;
            d++;
            back += l <= i;
        }
        deg_[i] = d;
        s.m += d;
        s.max_fwd = std::max(s.max_fwd, d - back);
    }
    return s;
}

void Builder::fill(uint64_t *rp, uint32_t *fo, uint32_t *ci, uint32_t *src, uint32_t *ids) {
    uint64_t off = 0;
    for (uint64_t i = 0; i < ball_.size(); i++) {
        rp[i] = off;
        const uint32_t g = (uint32_t)(ball_[i] >> 4);
        if (ids) ids[i] = g;
        uint32_t back = 0;
        if (deg_[i]) {
            for (uint64_t e = rp_[g]; e < rp_[g + 1]; e++) {
                const uint32_t l = mark_[ci_[e]];
                if (l == kNone) continue;
                ci[off++] = l;
                back += l <= i;
            }
        }
        fo[i] = back;
    }
    rp[ball_.size()] = off;
    for (uint64_t i = 0; i < src_.size(); i++) src[i] = mark_[src_[i]];
    release();
}

void Builder::fill_packed(void *buf, const Sizes &s) {
    const Layout L(s);
    char *b = static_cast<char *>(buf);
    fill(reinterpret_cast<uint64_t *>(b), reinterpret_cast<uint32_t *>(b + L.fo), reinterpret_cast<uint32_t *>(b + L.ci),
         reinterpret_cast<uint32_t *>(b + L.src), nullptr);
}

uint32_t plan_bins(const uint64_t *rp, const uint32_t *ci, uint64_t n, uint32_t radius, uint32_t row_radius,
                   uint32_t min_root_degree, uint64_t max_bytes, uint32_t *bin_of) {
    if (n == 0) return 0;
    // depth[x] = smallest distance from a source of the open bin; a vertex is
    // expanded again only when its depth drops (decrease-key BFS), so adding a
    // source costs what its ball adds to the bin
    std::vector<uint32_t> depth(n, kNone), touched, frontier, next;
    uint64_t bytes = 8, delta = 0;
    uint32_t bin = 0, nsrc = 0;
    auto relax = [&](uint32_t x, uint32_t d) {
        const uint32_t old = depth[x];
        if (old != kNone && old <= d) return false;
        if (old == kNone) {
            delta += 12;  // row pointer + forward offset
            touched.push_back(x);
        }
        if (d <= row_radius && (old == kNone || old > row_radius)) delta += 4ull * (rp[x + 1] - rp[x]);
        depth[x] = d;
        return true;
    };
    auto add = [&](uint32_t s) {
        delta = 4;  // the source entry
        frontier.clear();
        if (relax(s, 0)) frontier.push_back(s);
        for (uint32_t d = 0; d < radius && !frontier.empty(); d++) {
            next.clear();
            for (uint32_t x : frontier)
                for (uint64_t e = rp[x]; e < rp[x + 1]; e++)
                    if (relax(ci[e], d + 1)) next.push_back(ci[e]);
            frontier.swap(next);
        }
        return delta;
    };
    for (uint64_t v = 0; v < n; v++) {
        if (rp[v + 1] - rp[v] < min_root_degree) {
            bin_of[v] = bin;  // no embedding is rooted here: no size
            continue;
        }
        uint64_t d = add((uint32_t)v);
        if (nsrc > 0 && bytes + d > max_bytes) {
            for (uint32_t x : touched) depth[x] = kNone;
            touched.clear();
            bin++;
            bytes = 8;
            nsrc = 0;
            d = add((uint32_t)v);
        }
        bytes += d;
        nsrc++;
        bin_of[v] = bin;
    }
    return bin + 1;
}

void plan_radii(uint32_t k, const uint32_t *bn_count, const uint32_t (*bn_pos)[8], uint32_t *radius,
                uint32_t *row_radius, uint32_t *root_degree) {
    uint32_t adj[8] = {0};  // bit j of adj[i]: positions i and j adjacent
    bool is_bn[8] = {false};
    for (uint32_t i = 0; i < k && i < 8; i++)
        for (uint32_t j = 0; j < bn_count[i] && j < 8; j++) {
            const uint32_t p = bn_pos[i][j];
            if (p >= k) continue;
            adj[i] |= 1u << p;
            adj[p] |= 1u << i;
            is_bn[p] = true;
        }
    uint32_t dist[8];
    for (auto &d : dist) d = kNone;
    dist[0] = 0;
    uint32_t seen = 1u, cur = 1u;
    for (uint32_t d = 1; cur; d++) {
        uint32_t nxt = 0;
        for (uint32_t i = 0; i < k; i++)
            if (cur >> i & 1u) nxt |= adj[i];
        nxt &= ~seen;
        for (uint32_t i = 0; i < k; i++)
            if (nxt >> i & 1u) dist[i] = d;
        seen |= nxt;
        cur = nxt;
    }
    uint32_t r = 0, rr = 0;
    for (uint32_t i = 0; i < k; i++) {
        if (dist[i] == kNone) continue;
        r = std::max(r, dist[i]);
        if (is_bn[i]) rr = std::max(rr, dist[i]);
    }
    *radius = r;
    *row_radius = rr;
    *root_degree = (uint32_t)__builtin_popcount(adj[0]);
}

}  // namespace g2view

extern "C" {

int g2_view_bins(const uint64_t *row_ptrs, const uint32_t *cols, uint64_t n, uint32_t radius, uint32_t row_radius,
                 uint32_t min_root_degree, uint64_t max_bytes, uint32_t *bin_of, uint32_t *nbins) {
    if (!row_ptrs || !bin_of || !nbins || (!cols && row_ptrs[n]) || n >= (1ull << 32) || row_radius > radius ||
        radius > 15)
        return G2_ERR_INVALID;
    *nbins = g2view::plan_bins(row_ptrs, cols, n, radius, row_radius, min_root_degree, max_bytes, bin_of);
    return G2_OK;
}

int g2_view_materialize(const uint64_t *row_ptrs, const uint32_t *cols, uint64_t n, const uint32_t *sources,
                        uint64_t nsrc, uint32_t radius, uint32_t row_radius, uint32_t min_root_degree,
                        g2_view *out) {
    if (!row_ptrs || !out || (!sources && nsrc) || (!cols && row_ptrs[n]) || n >= (1ull << 32) ||
        row_radius > radius || radius > 15)
        return G2_ERR_INVALID;
    for (uint64_t i = 0; i < nsrc; i++)
        if (sources[i] >= n) return G2_ERR_INVALID;
    memset(out, 0, sizeof(*out));
    g2view::Builder b(row_ptrs, cols, n);
    const g2view::Sizes s = b.plan(sources, nsrc, radius, row_radius, min_root_degree);
    auto *rp = static_cast<uint64_t *>(malloc(8 * (s.n + 1)));
    auto *fo = static_cast<uint32_t *>(malloc(4 * std::max<uint64_t>(s.n, 1)));
    auto *ci = static_cast<uint32_t *>(malloc(4 * std::max<uint64_t>(s.m, 1)));
    auto *src = static_cast<uint32_t *>(malloc(4 * std::max<uint64_t>(s.nsrc, 1)));
    auto *ids = static_cast<uint32_t *>(malloc(4 * std::max<uint64_t>(s.n, 1)));
    if (!rp || !fo || !ci || !src || !ids) {
        free(rp), free(fo), free(ci), free(src), free(ids);
        return G2_ERR_OOM;
    }
    b.fill(rp, fo, ci, src, ids);
    out->row_ptrs = rp;
    out->cols = ci;
    out->fwd_offsets = fo;
    out->sources = src;
    out->ids = ids;
    out->n = s.n;
    out->m = s.m;
    out->nsrc = s.nsrc;
    out->max_fwd = s.max_fwd;
    return G2_OK;
}

void g2_view_free(g2_view *v) {
    if (!v) return;
    free(v->row_ptrs), free(v->cols), free(v->fwd_offsets), free(v->sources), free(v->ids);
    memset(v, 0, sizeof(*v));
}

int g2_plan_view_radius(const g2_plan *p, uint32_t *radius, uint32_t *row_radius, uint32_t *root_degree) {
    if (!p || !radius || !row_radius || !root_degree || p->k < 2 || p->k > G2_MAX_QUERY) return G2_ERR_INVALID;
    uint32_t pos[G2_MAX_QUERY][8] = {{0}};
    uint32_t cnt[G2_MAX_QUERY] = {0};
    for (uint32_t i = 0; i < p->k; i++) {
        if (p->bn_count[i] > p->k) return G2_ERR_INVALID;
        cnt[i] = p->bn_count[i];
        for (uint32_t j = 0; j < cnt[i]; j++) {
            if (p->bn[i][j] >= p->k) return G2_ERR_INVALID;
            pos[i][j] = p->id2order[p->bn[i][j]];
        }
    }
    g2view::plan_radii(p->k, cnt, pos, radius, row_radius, root_degree);
    return G2_OK;
}

}  // extern "C"

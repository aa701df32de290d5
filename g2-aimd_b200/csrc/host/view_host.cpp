// view_host.cpp - views of a host CSR around a set of roots, the greedy bin
// partition that sizes them, and what a query plan needs of a view.
//
// Replaces the host side of the reference's out-of-core path:
// ViewBin::Materialize / ExtendFromSource (view/view_bin.h:40-159) and the
// per-query hop of Plan::FindRoot (system/plan.h:51-73).  The pipeline that
// uploads views and runs the enumeration over them is in view_run.cu.
#include "view_host.h"

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <thread>

#include "g2_aimd.h"

namespace g2view {

namespace {
inline uint64_t align16(uint64_t x) { return (x + 15u) & ~15ull; }

// First entry of row x that is >= lo (rows are sorted).
inline uint64_t row_from(const uint64_t *rp, const uint32_t *ci, uint32_t x, uint32_t lo) {
    if (lo == 0) return rp[x];
    return (uint64_t)(std::lower_bound(ci + rp[x], ci + rp[x + 1], lo) - ci);
}
}  // namespace

unsigned host_threads() {
    unsigned t = std::thread::hardware_concurrency();
    if (const char *e = getenv("G2_HOST_THREADS")) t = (unsigned)atoi(e);
    return t ? t : 1u;
}

Layout::Layout(const Sizes &s) {
    fo = align16(8ull * (s.n + 1));
    ci = align16(fo + 4ull * s.n);
    src = align16(ci + 4ull * s.m);
    bytes = align16(src + 4ull * s.nsrc);
}

void Builder::release() {
    for (uint32_t g : ball_) mark_[g] = kNone;
    if (!bits_.empty())
        for (uint32_t g : ball_) bits_[g >> 6] = 0;
    ball_.clear();
    row_.clear();
    src_.clear();
    deg_.clear();
}

// Lower x's depth to d (a vertex is walked again only when its depth drops).
bool Builder::relax(uint32_t x, uint32_t d) {
    const uint32_t old = mark_[x];
    if (old != kNone && old <= d) return false;
    if (old == kNone) ball_.push_back(x);
    mark_[x] = d;
    return true;
}

Sizes Builder::plan(const uint32_t *src, uint64_t nsrc, const Shape &sh) {
    if (mark_.size() != n_) mark_.assign(n_, kNone);
    release();
    for (uint64_t i = 0; i < nsrc; i++)
        if (rp_[src[i] + 1] - rp_[src[i]] >= sh.min_deg) src_.push_back(src[i]);
    auto walk = [&](uint32_t lo_excl, bool upper) {
        for (uint32_t d = 0; d < sh.radius && !frontier_.empty(); d++) {
            next_.clear();
            for (uint32_t x : frontier_)
                for (uint64_t e = upper ? row_from(rp_, ci_, x, lo_excl + 1) : rp_[x]; e < rp_[x + 1]; e++) {
                    const uint32_t u = ci_[e];
                    if (relax(u, d + 1)) next_.push_back(u);
                }
            frontier_.swap(next_);
        }
    };
    if (sh.radius == 1 && threads_ > 1 && src_.size() >= kParallelRows) {
        walk_radius1(sh);  // ball_ sorted, marks = local ids, rows flagged
    } else if (!sh.upper) {
        // one multi-source BFS: the depth of a vertex is its distance to the set
        frontier_.clear();
        for (uint32_t s : src_)
            if (relax(s, 0)) frontier_.push_back(s);
        walk(0, false);
    } else {
        // source by source in ascending order, through vertices above the
        // source: a vertex already reached at depth <= d from a smaller source
        // was walked from there through a superset of what this source allows
        std::vector<uint32_t> order(src_);
        std::sort(order.begin(), order.end());
        order.erase(std::unique(order.begin(), order.end()), order.end());
        for (uint32_t s : order) {
            if (!relax(s, 0)) continue;
            frontier_.assign(1, s);
            walk(s, true);
        }
    }
    if (!walked_sorted_) {
        // ascending global order = local ids; rows where the depth allows; marks become local ids
        std::sort(ball_.begin(), ball_.end());
        row_.resize(ball_.size());
        for (uint64_t i = 0; i < ball_.size(); i++) {
            row_[i] = mark_[ball_[i]] <= sh.row_radius;
            mark_[ball_[i]] = (uint32_t)i;
        }
    }
    walked_sorted_ = false;
    const uint64_t nv = ball_.size();
    // nothing below the smallest view vertex is in the view: rows are read from there
    lo_ = nv ? ball_[0] : 0u;
    Sizes s;
    s.n = nv;
    s.nsrc = src_.size();
    deg_.assign(nv, 0u);
    fo_.assign(nv, 0u);
    cols_.clear();
    row_start_ = sh.forward ? 1u : 0u;
    staged_ = threads_ <= 1 || nv < kParallelRows || sh.ego;  // ego rows filter staged columns
    if (!staged_) {
        // large view, several threads: count the rows here, write them in fill
        std::vector<uint32_t> mf(threads_, 0u);
        parallel_rows(nv, [&](unsigned t, uint64_t i0, uint64_t i1) {
            for (uint64_t i = i0; i < i1; i++) {
                if (!row_[i]) continue;
                uint32_t d = 0, back = 0;
                for (uint64_t e = row_begin(i); e < rp_[ball_[i] + 1]; e++) {
                    const uint32_t l = mark_[ci_[e]];
                    if (l == kNone) continue;
                    d++;
                    back += l <= i;
                }
                deg_[i] = d;
                fo_[i] = back;
                mf[t] = std::max(mf[t], d - back);
            }
        });
        for (uint32_t v : mf) s.max_fwd = std::max(s.max_fwd, v);
        for (uint64_t i = 0; i < nv; i++) s.m += deg_[i];
        return s;
    }
    // one pass over the kept rows: local columns staged here, copied out by fill
    for (uint64_t i = 0; i < nv; i++) {
        if (!row_[i]) continue;
        const uint32_t g = ball_[i];
        const uint64_t before = cols_.size();
        uint32_t back = 0;
        for (uint64_t e = row_begin(i); e < rp_[g + 1]; e++) {
            const uint32_t l = mark_[ci_[e]];
            if (l == kNone) continue;
            cols_.push_back(l);
            back += l <= i;
        }
        const uint32_t d = (uint32_t)(cols_.size() - before);
        deg_[i] = d;
        fo_[i] = back;
        s.max_fwd = std::max(s.max_fwd, d - back);
    }
    s.m = cols_.size();
    if (sh.ego) ego_filter(&s);
    return s;
}

// Keep only the entries (u, y) with a kept source s in N[u] ∩ N[y] (the edges of
// the sources' ego networks): a root's search reads rows of its neighbours
// restricted to its own neighbourhood, nothing else.  Per source s (on the
// builder's threads): s's row is kept whole, and in the row of each neighbour u
// the entries in N[s] are marked, by scanning u's row against a stamp of N(s)
// or, for a row much longer than s's, by binary searches of N[s] in it.
void Builder::ego_filter(Sizes *s) {
    const uint64_t nv = ball_.size();
    std::vector<uint64_t> off(nv + 1, 0);
    for (uint64_t i = 0; i < nv; i++) off[i + 1] = off[i] + deg_[i];
    std::vector<uint8_t> keep(cols_.size(), 0);
    std::vector<uint32_t> ls;
    ls.reserve(src_.size());
    for (uint32_t g : src_) ls.push_back(mark_[g]);
    std::sort(ls.begin(), ls.end());
    ls.erase(std::unique(ls.begin(), ls.end()), ls.end());
    auto keep_at = [&](uint64_t p) { __atomic_store_n(&keep[p], (uint8_t)1, __ATOMIC_RELAXED); };
    std::vector<std::vector<uint32_t>> stamps(threads_);
    const uint32_t *c = cols_.data();
    parallel_rows(ls.size(), [&](unsigned t, uint64_t a, uint64_t b) {
        std::vector<uint32_t> &stamp = stamps[t];
        if (stamp.size() != nv) stamp.assign(nv, kNone);
        for (uint64_t k = a; k < b; k++) {
            const uint32_t src = ls[k];
            const uint32_t *rs = c + off[src];
            const uint64_t ns = deg_[src];
            for (uint64_t j = 0; j < ns; j++) {
                keep_at(off[src] + j);
                stamp[rs[j]] = src;
            }
            for (uint64_t j = 0; j < ns; j++) {
                const uint32_t u = rs[j];
                const uint32_t *ru = c + off[u];
                const uint64_t nu = deg_[u];
                if (nu <= 8 * ns) {
                    for (uint64_t q = 0; q < nu; q++)
                        if (ru[q] == src || stamp[ru[q]] == src) keep_at(off[u] + q);
                } else {
                    auto find = [&](uint32_t x) {
                        const uint32_t *p = std::lower_bound(ru, ru + nu, x);
                        if (p != ru + nu && *p == x) keep_at(off[u] + (uint64_t)(p - ru));
                    };
                    find(src);
                    for (uint64_t q = 0; q < ns; q++) find(rs[q]);
                }
            }
        }
    });
    // compact in place (kept entries move left), recount forward lists
    uint64_t w = 0;
    s->max_fwd = 0;
    for (uint64_t i = 0; i < nv; i++) {
        uint32_t d = 0, back = 0;
        for (uint64_t p = off[i]; p < off[i + 1]; p++) {
            if (!keep[p]) continue;
            const uint32_t y = cols_[p];
            cols_[w++] = y;
            d++;
            back += y <= i;
        }
        deg_[i] = d;
        fo_[i] = back;
        s->max_fwd = std::max(s->max_fwd, d - back);
    }
    cols_.resize(w);
    s->m = w;
}

// Ball of radius 1 on several threads: the sources and their neighbours (above
// the source for upper balls) are marked in a bitmap with atomics, depth 0 for
// sources and 1 for the rest; the bitmap's words, read in order, give the ball
// sorted, so each thread writes its part of ball_ and of the local ids directly.
void Builder::walk_radius1(const Shape &sh) {
    if (bits_.size() != (n_ + 63) / 64) bits_.assign((n_ + 63) / 64, 0ull);
    const uint64_t ns = src_.size();
    auto set_bit = [&](uint32_t x) { __atomic_fetch_or(&bits_[x >> 6], 1ull << (x & 63u), __ATOMIC_RELAXED); };
    parallel_range(ns, [&](uint64_t a, uint64_t b) {
        for (uint64_t i = a; i < b; i++) {
            __atomic_store_n(&mark_[src_[i]], 0u, __ATOMIC_RELAXED);
            set_bit(src_[i]);
        }
    });
    parallel_range(ns, [&](uint64_t a, uint64_t b) {
        for (uint64_t i = a; i < b; i++) {
            const uint32_t s = src_[i];
            for (uint64_t e = sh.upper ? row_from(rp_, ci_, s, s + 1) : rp_[s]; e < rp_[s + 1]; e++) {
                const uint32_t u = ci_[e];
                uint32_t none = kNone;  // sources keep depth 0
                __atomic_compare_exchange_n(&mark_[u], &none, 1u, false, __ATOMIC_RELAXED, __ATOMIC_RELAXED);
                set_bit(u);
            }
        }
    });
    // blocks of bitmap words: population per block, prefix, then each block its entries
    const uint64_t words = bits_.size(), block = 1u << 12;
    const uint64_t nblk = (words + block - 1) / block;
    std::vector<uint64_t> cnt(nblk + 1, 0);
    parallel_range(nblk, [&](uint64_t a, uint64_t b) {
        for (uint64_t k = a; k < b; k++) {
            uint64_t c = 0;
            for (uint64_t w = k * block; w < std::min(words, (k + 1) * block); w++) c += __builtin_popcountll(bits_[w]);
            cnt[k + 1] = c;
        }
    });
    for (uint64_t k = 0; k < nblk; k++) cnt[k + 1] += cnt[k];
    ball_.resize(cnt[nblk]);
    row_.resize(cnt[nblk]);
    parallel_range(nblk, [&](uint64_t a, uint64_t b) {
        for (uint64_t k = a; k < b; k++) {
            uint64_t i = cnt[k];
            for (uint64_t w = k * block; w < std::min(words, (k + 1) * block); w++)
                for (uint64_t x = bits_[w]; x; x &= x - 1) {
                    const uint32_t g = (uint32_t)(w * 64 + (uint64_t)__builtin_ctzll(x));
                    ball_[i] = g;
                    row_[i] = mark_[g] <= sh.row_radius;
                    mark_[g] = (uint32_t)i;
                    i++;
                }
        }
    });
    walked_sorted_ = true;
}

// f(a, b) over [0, n) in blocks taken in turn by the builder's threads.
template <class F>
void Builder::parallel_range(uint64_t n, F f) {
    const uint64_t blk = std::max<uint64_t>(1, std::min<uint64_t>(kParallelRows / 8, n / (4ull * threads_) + 1));
    std::atomic<uint64_t> next{0};
    auto work = [&]() {
        for (uint64_t a; (a = next.fetch_add(blk)) < n;) f(a, std::min(n, a + blk));
    };
    std::vector<std::thread> th;
    for (unsigned t = 1; t < threads_; t++) th.emplace_back(work);
    work();
    for (auto &x : th) x.join();
}

// First entry of view row i's source row that can be in the view.
uint64_t Builder::row_begin(uint64_t i) const {
    const uint32_t g = ball_[i];
    return row_from(rp_, ci_, g, row_start_ ? g + 1 : lo_);
}

// f(thread, i0, i1) over [0, nv) in blocks of kParallelRows / 8 rows taken in turn.
template <class F>
void Builder::parallel_rows(uint64_t nv, F f) {
    const uint64_t block = kParallelRows / 8;
    std::atomic<uint64_t> next{0};
    auto work = [&](unsigned t) {
        for (uint64_t i0; (i0 = next.fetch_add(block)) < nv;) f(t, i0, std::min(nv, i0 + block));
    };
    std::vector<std::thread> th;
    for (unsigned t = 1; t < threads_; t++) th.emplace_back(work, t);
    work(0);
    for (auto &x : th) x.join();
}

void Builder::fill(uint64_t *rp, uint32_t *fo, uint32_t *ci, uint32_t *src, uint32_t *ids) {
    const uint64_t nv = ball_.size();
    uint64_t off = 0;
    for (uint64_t i = 0; i < nv; i++) {
        rp[i] = off;
        off += deg_[i];
        if (ids) ids[i] = ball_[i];
    }
    rp[nv] = off;
    if (!fo_.empty()) memcpy(fo, fo_.data(), 4 * fo_.size());
    if (staged_) {
        if (!cols_.empty()) memcpy(ci, cols_.data(), 4 * cols_.size());
    } else {
        parallel_rows(nv, [&](unsigned, uint64_t i0, uint64_t i1) {
            for (uint64_t i = i0; i < i1; i++) {
                if (!deg_[i]) continue;
                uint32_t *out = ci + rp[i];
                for (uint64_t e = row_begin(i); e < rp_[ball_[i] + 1]; e++) {
                    const uint32_t l = mark_[ci_[e]];
                    if (l != kNone) *out++ = l;
                }
            }
        });
    }
    for (uint64_t i = 0; i < src_.size(); i++) src[i] = mark_[src_[i]];
    release();
}

void Builder::fill_packed(void *buf, const Sizes &s) {
    const Layout L(s);
    char *b = static_cast<char *>(buf);
    fill(reinterpret_cast<uint64_t *>(b), reinterpret_cast<uint32_t *>(b + L.fo), reinterpret_cast<uint32_t *>(b + L.ci),
         reinterpret_cast<uint32_t *>(b + L.src), nullptr);
}

namespace {

// Greedy bins over the roots [v0, v1) (bin ids from 0; returns how many).  The
// open bin's view is tracked exactly: depth[x] = smallest depth from a source
// of the bin (walked again only when it drops; sources come in ascending order,
// which the upper walks need), and a vertex that enters the ball or gains its
// row adds its column entries towards the ball.  depth: n bytes, all 0xff.
uint32_t plan_range(const uint64_t *rp, const uint32_t *ci, const Shape &sh, uint64_t max_bytes, uint64_t v0,
                    uint64_t v1, std::vector<uint8_t> &depth, uint32_t *bin_of) {
    constexpr uint8_t kOut = 0xff;
    std::vector<uint32_t> touched, frontier, next;
    uint64_t bytes = 8, delta = 0;
    uint32_t bin = 0, nsrc = 0;
    uint32_t lo = 0;  // upper walks: no vertex below the bin's first source is in its ball
    auto relax = [&](uint32_t x, uint32_t d) {
        const uint8_t old = depth[x];
        if (old != kOut && old <= d) return false;
        const bool fresh = old == kOut;
        const bool gains_row = d <= sh.row_radius && (fresh || old > sh.row_radius);
        depth[x] = (uint8_t)d;
        if (fresh) {
            delta += 12;  // row pointer + forward offset
            touched.push_back(x);
        }
        if (fresh || gains_row) {
            for (uint64_t e = row_from(rp, ci, x, lo); e < rp[x + 1]; e++) {
                const uint32_t y = ci[e];
                if (y == x || depth[y] == kOut) continue;
                // forward rows keep only entries above their own vertex
                if (gains_row && (!sh.forward || y > x)) delta += 4;                            // x -> y
                if (fresh && depth[y] <= sh.row_radius && (!sh.forward || x > y)) delta += 4;  // y -> x
            }
        }
        return true;
    };
    auto add = [&](uint32_t s) {
        delta = 4;  // the source entry
        frontier.clear();
        if (relax(s, 0)) frontier.push_back(s);
        for (uint32_t d = 0; d < sh.radius && !frontier.empty(); d++) {
            next.clear();
            for (uint32_t x : frontier)
                for (uint64_t e = sh.upper ? row_from(rp, ci, x, s + 1) : rp[x]; e < rp[x + 1]; e++) {
                    const uint32_t u = ci[e];
                    if (relax(u, d + 1)) next.push_back(u);
                }
            frontier.swap(next);
        }
        return delta;
    };
    for (uint64_t v = v0; v < v1; v++) {
        if (rp[v + 1] - rp[v] < sh.min_deg) {
            bin_of[v] = bin;  // no embedding is rooted here: no size
            continue;
        }
        if (sh.upper && nsrc == 0) lo = (uint32_t)v;
        uint64_t d = add((uint32_t)v);
        if (nsrc > 0 && bytes + d > max_bytes) {
            for (uint32_t x : touched) depth[x] = kOut;
            touched.clear();
            bin++;
            bytes = 8;
            nsrc = 0;
            if (sh.upper) lo = (uint32_t)v;
            d = add((uint32_t)v);
        }
        bytes += d;
        nsrc++;
        bin_of[v] = bin;
    }
    for (uint32_t x : touched) depth[x] = kOut;
    return bin + 1;
}

}  // namespace

namespace {

// Bins over T contiguous root ranges of about equal edge counts, each planned
// on a thread of its own (a bin never spans two ranges).
uint32_t plan_in_ranges(const uint64_t *rp, const uint32_t *ci, uint64_t n, const Shape &sh, uint64_t max_bytes,
                        uint32_t *bin_of, unsigned T) {
    std::vector<uint64_t> cut(T + 1, n);
    cut[0] = 0;
    for (unsigned t = 1; t < T; t++) {
        const uint64_t target = rp[n] / T * t;
        cut[t] = std::max<uint64_t>(cut[t - 1], (uint64_t)(std::upper_bound(rp, rp + n + 1, target) - rp) - 1);
    }
    std::vector<uint32_t> count(T, 0);
    auto run = [&](unsigned t) {
        if (cut[t] >= cut[t + 1]) return;
        std::vector<uint8_t> depth(n, 0xff);
        count[t] = plan_range(rp, ci, sh, max_bytes, cut[t], cut[t + 1], depth, bin_of);
    };
    std::vector<std::thread> th;
    for (unsigned t = 1; t < T; t++) th.emplace_back(run, t);
    run(0);
    for (auto &x : th) x.join();
    uint32_t base = 0;
    for (unsigned t = 0; t < T; t++) {
        if (base)
            for (uint64_t v = cut[t]; v < cut[t + 1]; v++) bin_of[v] += base;
        base += count[t];
    }
    return base;
}

}  // namespace

uint32_t plan_bins(const uint64_t *rp, const uint32_t *ci, uint64_t n, const Shape &sh, uint64_t max_bytes,
                   uint32_t *bin_of, unsigned threads) {
    if (n == 0) return 0;
    unsigned T = n >= kParallelBinRoots ? std::max(1u, threads) : 1u;
    // every range holds a byte per vertex of the whole graph: at most 8 GB in all
    T = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(T, (8ull << 30) / n));
    if (T == 1) return plan_in_ranges(rp, ci, n, sh, max_bytes, bin_of, 1);
    // each range boundary adds at most one bin, so a first plan on T ranges
    // bounds the serial bin count from below; ranges are then sized to hold at
    // least 8 bins each (at most 1 bin in 8 added), down to one range for a
    // graph of few bins
    const uint32_t first = plan_in_ranges(rp, ci, n, sh, max_bytes, bin_of, T);
    const uint64_t lower = first > T - 1 ? first - (T - 1) : 1;
    const unsigned T2 = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(T, lower / 8));
    return T2 == T ? first : plan_in_ranges(rp, ci, n, sh, max_bytes, bin_of, T2);
}
Shape plan_shape(uint32_t k, const uint32_t *bn_count, const uint32_t (*bn_pos)[8], const uint32_t *cond_count,
                 const uint32_t (*cond_op)[8], const uint32_t (*cond_pos)[8]) {
    k = std::min<uint32_t>(k, 8u);
    uint32_t adj[8] = {0};  // bit j of adj[i]: positions i and j adjacent
    uint32_t gt[8] = {0};   // bit j of gt[i]: the conditions imply M(i) > M(j)
    bool is_bn[8] = {false};
    for (uint32_t i = 0; i < k; i++) {
        for (uint32_t j = 0; j < bn_count[i] && j < 8; j++) {
            const uint32_t p = bn_pos[i][j];
            if (p >= k) continue;
            adj[i] |= 1u << p;
            adj[p] |= 1u << i;
            is_bn[p] = true;
        }
        for (uint32_t j = 0; j < cond_count[i] && j < 8; j++) {
            const uint32_t p = cond_pos[i][j];
            if (p >= k) continue;
            if (cond_op[i][j] == G2_COND_LARGER_THAN) gt[i] |= 1u << p;
            if (cond_op[i][j] == G2_COND_LESS_THAN) gt[p] |= 1u << i;
        }
    }
    for (uint32_t it = 0; it < k; it++)  // transitive closure
        for (uint32_t a = 0; a < k; a++)
            for (uint32_t b = 0; b < k; b++)
                if (gt[a] >> b & 1u) gt[a] |= gt[b];
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
    Shape sh;
    sh.radius = 0;
    sh.row_radius = 0;
    sh.upper = k > 1;
    sh.forward = k > 1;
    for (uint32_t i = 0; i < k; i++) {
        if (i > 0 && !(gt[i] & 1u)) sh.upper = false;
        if ((gt[i] & ((1u << i) - 1u)) != ((1u << i) - 1u)) sh.forward = false;  // above every earlier position
        if (dist[i] == kNone) continue;
        sh.radius = std::max(sh.radius, dist[i]);
        if (is_bn[i]) sh.row_radius = std::max(sh.row_radius, dist[i]);
    }
    sh.min_deg = (uint32_t)__builtin_popcount(adj[0]);
    return sh;
}

}  // namespace g2view

namespace {

bool shape_from(uint32_t radius, uint32_t row_radius, uint32_t min_root_degree, uint32_t flags,
                g2view::Shape *sh) {
    if (row_radius > radius || radius > 15 || (flags & ~(uint32_t)(G2_VIEW_UPPER | G2_VIEW_FORWARD | G2_VIEW_EGO)))
        return false;
    if ((flags & G2_VIEW_EGO) && (radius != 1 || row_radius != 1)) return false;  // ego networks: radius 1
    sh->radius = radius;
    sh->row_radius = row_radius;
    sh->min_deg = min_root_degree;
    sh->upper = (flags & G2_VIEW_UPPER) != 0;
    sh->forward = (flags & G2_VIEW_FORWARD) != 0;
    sh->ego = (flags & G2_VIEW_EGO) != 0;
    return true;
}

}  // namespace

extern "C" {

int g2_view_bins(const uint64_t *row_ptrs, const uint32_t *cols, uint64_t n, uint32_t radius, uint32_t row_radius,
                 uint32_t min_root_degree, uint32_t flags, uint64_t max_bytes, uint32_t *bin_of, uint32_t *nbins) {
    g2view::Shape sh;
    if (!row_ptrs || !bin_of || !nbins || (!cols && row_ptrs[n]) || n >= (1ull << 32) ||
        !shape_from(radius, row_radius, min_root_degree, flags, &sh))
        return G2_ERR_INVALID;
    *nbins = g2view::plan_bins(row_ptrs, cols, n, sh, max_bytes, bin_of, g2view::host_threads());
    return G2_OK;
}

int g2_shell_bins(const uint32_t *core, uint64_t n, uint32_t nbins, uint32_t *bin_of) {
    if (!core || !bin_of || !nbins) return G2_ERR_INVALID;
    // kmeans/kcore.cpp:193-228 (writeBins): each core shell, a run of ids in
    // degeneracy order, is dealt to the bins in consecutive chunks of
    // window / nbins + 1 vertices (bin 0 first)
    for (uint64_t i = 0; i < n;) {
        uint64_t j = i;
        while (j < n && core[j] == core[i]) j++;
        if (j < n && core[j] < core[i]) return G2_ERR_INVALID;  // shells must ascend
        const uint64_t share = (j - i) / nbins + 1;
        for (uint64_t v = i; v < j; v++) bin_of[v] = (uint32_t)((v - i) / share);
        i = j;
    }
    return G2_OK;
}

int g2_view_bins_rebalance(const uint64_t *row_ptrs, uint64_t n, uint32_t *bin_of, uint32_t nbins,
                           uint32_t devices, uint32_t split_times, int reorder, uint32_t *out_nbins) {
    if (!row_ptrs || !bin_of || !out_nbins || (split_times && !devices) || n >= (1ull << 32)) return G2_ERR_INVALID;
    // bins as root lists; a bin's factor is the degree sum of its roots
    // (ViewBin::GetComputationFactors, view/view_bin.h:27-39)
    std::vector<std::vector<uint32_t>> bins(nbins);
    for (uint64_t v = 0; v < n; v++) {
        if (bin_of[v] == G2_VIEW_NO_BIN) continue;
        if (bin_of[v] >= nbins) return G2_ERR_INVALID;
        bins[bin_of[v]].push_back((uint32_t)v);
    }
    auto deg = [&](uint32_t v) { return row_ptrs[v + 1] - row_ptrs[v]; };
    std::vector<uint64_t> factor(nbins, 0);
    for (uint32_t b = 0; b < nbins; b++)
        for (uint32_t v : bins[b]) factor[b] += deg(v);
    if (split_times && nbins) {
        // ViewBinManager::Split (view/view_bin_manager.h:95-175): until there are
        // (nbins / devices + times) * devices bins, the bin furthest above the
        // mean factor is cut in two, its roots dealt alternately in descending
        // degree order (odd positions to the first half); halves go last
        const uint64_t target = ((uint64_t)nbins / devices + split_times) * devices;
        while (bins.size() < target) {
            uint64_t sum = 0;
            for (uint64_t f : factor) sum += f;
            const uint64_t avg = sum / bins.size();
            size_t pick = 0;
            uint64_t best = 0;
            for (size_t i = 0; i < bins.size(); i++)
                if (factor[i] >= avg && factor[i] - avg > best) best = factor[i] - avg, pick = i;
            std::vector<uint32_t> src = std::move(bins[pick]);
            std::stable_sort(src.begin(), src.end(), [&](uint32_t a, uint32_t b) { return deg(a) > deg(b); });
            std::vector<uint32_t> a, b;
            uint64_t fa = 0, fb = 0;
            for (size_t i = 0; i < src.size(); i++) {
                if (i % 2) a.push_back(src[i]), fa += deg(src[i]);
                else b.push_back(src[i]), fb += deg(src[i]);
            }
            bins.erase(bins.begin() + (ptrdiff_t)pick);
            factor.erase(factor.begin() + (ptrdiff_t)pick);
            bins.push_back(std::move(a));
            factor.push_back(fa);
            bins.push_back(std::move(b));
            factor.push_back(fb);
        }
    }
    // ViewBinManager::Reorder (view/view_bin_manager.h:176-184), also the end of
    // Split: descending factor (ties keep their order)
    std::vector<uint32_t> order(bins.size());
    for (uint32_t i = 0; i < order.size(); i++) order[i] = i;
    if (reorder || split_times)
        std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return factor[a] > factor[b]; });
    for (uint32_t k = 0; k < order.size(); k++)
        for (uint32_t v : bins[order[k]]) bin_of[v] = k;
    *out_nbins = (uint32_t)bins.size();
    return G2_OK;
}

int g2_view_materialize(const uint64_t *row_ptrs, const uint32_t *cols, uint64_t n, const uint32_t *sources,
                        uint64_t nsrc, uint32_t radius, uint32_t row_radius, uint32_t min_root_degree, uint32_t flags,
                        g2_view *out) {
    g2view::Shape sh;
    if (!row_ptrs || !out || (!sources && nsrc) || (!cols && row_ptrs[n]) || n >= (1ull << 32) ||
        !shape_from(radius, row_radius, min_root_degree, flags, &sh))
        return G2_ERR_INVALID;
    for (uint64_t i = 0; i < nsrc; i++)
        if (sources[i] >= n) return G2_ERR_INVALID;
    memset(out, 0, sizeof(*out));
    g2view::Builder b(row_ptrs, cols, n, g2view::host_threads());
    const g2view::Sizes s = b.plan(sources, nsrc, sh);
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

int g2_plan_view_radius(const g2_plan *p, uint32_t *radius, uint32_t *row_radius, uint32_t *root_degree,
                        uint32_t *flags) {
    if (!p || !radius || !row_radius || !root_degree || !flags || p->k < 2 || p->k > G2_MAX_QUERY)
        return G2_ERR_INVALID;
    uint32_t bn[8][8] = {{0}}, cop[8][8] = {{0}}, cpos[8][8] = {{0}};
    uint32_t bnc[8] = {0}, cc[8] = {0};
    for (uint32_t i = 0; i < p->k; i++) {
        const uint32_t u = p->order[i];  // query vertex at position i
        if (u >= p->k || p->bn_count[i] > p->k || p->cond_count[u] > p->k) return G2_ERR_INVALID;
        bnc[i] = p->bn_count[i];
        for (uint32_t j = 0; j < bnc[i]; j++) {
            if (p->bn[i][j] >= p->k) return G2_ERR_INVALID;
            bn[i][j] = p->id2order[p->bn[i][j]];
        }
        cc[i] = p->cond_count[u];
        for (uint32_t j = 0; j < cc[i]; j++) {
            if (p->cond[u][j][1] >= p->k) return G2_ERR_INVALID;
            cop[i][j] = p->cond[u][j][0];
            cpos[i][j] = p->id2order[p->cond[u][j][1]];
        }
    }
    const g2view::Shape sh = g2view::plan_shape(p->k, bnc, bn, cc, cop, cpos);
    *radius = sh.radius;
    *row_radius = sh.row_radius;
    *root_degree = sh.min_deg;
    *flags = (sh.upper ? G2_VIEW_UPPER : 0u) | (sh.forward ? G2_VIEW_FORWARD : 0u);
    return G2_OK;
}

}  // extern "C"

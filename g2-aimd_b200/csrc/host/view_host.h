// view_host.h - views of a host CSR around a set of roots (internal C++ API).
//
// A view holds everything that the searches rooted at a set of sources read:
// the ball B of radius `radius` around the sources (every vertex an embedding
// rooted there can reach), with ids renumbered 0..|B|-1 in ascending global
// order, so that id comparisons (symmetry-breaking conditions, P/X split of a
// Bron-Kerbosch root, forward lists) give the same answers as in the whole
// graph.  Vertices within `row_radius` of a source keep their adjacency
// restricted to B; the others keep an empty row (their neighbours are never
// scanned).  With `upper` (queries whose conditions put every matched vertex
// above the root's image) the ball of source s is walked through vertices
// larger than s only, and with `forward` (queries that order every position
// above all earlier ones) rows keep only their entries above their own vertex;
// with `ego` (radius 1) a row keeps only the entries (u, y) for which some
// source s has u and y in N[s].  Replaces the materialisation of view/view_bin.h:61-159,
// which keeps global ids and copies the full rows of the vertices within hop-1
// of the sources.
#pragma once

#include <cstdint>
#include <vector>

namespace g2view {

constexpr uint32_t kNone = 0xffffffffu;

// Host threads the view code may use: G2_HOST_THREADS if set, else the
// hardware's (at least 1).
unsigned host_threads();

struct Sizes {
    uint64_t n = 0;         // view vertices |B|
    uint64_t m = 0;         // view column entries
    uint64_t nsrc = 0;      // sources kept (degree >= min_root_degree)
    uint32_t max_fwd = 0;   // max |N(v) ∩ (v, ∞)| inside the view
};

// Byte layout of a view in one buffer (host slot or device slot):
//   rp u64[n+1] | fo u32[n] | ci u32[m] | src u32[nsrc], each part 16-byte aligned.
struct Layout {
    uint64_t fo = 0, ci = 0, src = 0, bytes = 0;
    explicit Layout(const Sizes &s);
};

// How a view is cut.
struct Shape {
    uint32_t radius = 1;      // ball radius
    uint32_t row_radius = 1;  // rows kept up to this depth
    uint32_t min_deg = 0;     // sources of smaller degree are dropped
    bool upper = false;       // balls walked through vertices above their source
    bool forward = false;     // rows keep only neighbours above their own vertex
    bool ego = false;         // rows keep only edges of the sources' ego networks (radius 1)
};

// One builder per producer; it keeps an n-entry mark array (4 bytes per vertex
// of the whole graph) between views and clears only what a view touched.  A
// view of at least kParallelRows vertices has its rows counted and written by
// `threads` threads; a radius-1 ball of at least kParallelRows sources is
// walked by them too (bitmap of n bits per builder).
class Builder {
  public:
    static constexpr uint64_t kParallelRows = 1u << 14;
    Builder(const uint64_t *rp, const uint32_t *ci, uint64_t n, unsigned threads = 1)
        : rp_(rp), ci_(ci), n_(n), threads_(threads ? threads : 1u) {}
    // Collect the view of `src` (sources must be < n).
    Sizes plan(const uint32_t *src, uint64_t nsrc, const Shape &shape);
    // Write the planned view: rp[n+1], fo[n] (per vertex, neighbours <= v),
    // ci[m], src[nsrc] (local ids of the kept sources, in the given order),
    // ids[n] (global id of each view vertex; may be null).  Releases the marks.
    void fill(uint64_t *rp, uint32_t *fo, uint32_t *ci, uint32_t *src, uint32_t *ids);
    // Same, into one buffer laid out as Layout(sizes).
    void fill_packed(void *buf, const Sizes &s);

  private:
    void release();
    bool relax(uint32_t x, uint32_t d);
    uint64_t row_begin(uint64_t i) const;
    template <class F>
    void parallel_rows(uint64_t nv, F f);
    template <class F>
    void parallel_range(uint64_t n, F f);
    void walk_radius1(const Shape &sh);
    void ego_filter(Sizes *s);
    std::vector<uint64_t> bits_;  // radius-1 walks on several threads: view membership
    bool walked_sorted_ = false;  // the walk left ball_ sorted and the marks as local ids
    const uint64_t *rp_;
    const uint32_t *ci_;
    uint64_t n_;
    unsigned threads_;
    bool staged_ = true;       // columns staged in cols_ by plan (else written by fill)
    uint32_t row_start_ = 0;   // 1: rows start above their own vertex (forward rows)
    std::vector<uint32_t> mark_;   // BFS depth, then the local id; kNone outside the view
    std::vector<uint32_t> ball_;   // view vertices (global ids), sorted after the walk
    std::vector<uint8_t> row_;     // view vertex i keeps its row
    std::vector<uint32_t> src_;    // kept sources (global ids), given order
    std::vector<uint32_t> deg_;    // view degree of each view vertex
    std::vector<uint32_t> fo_;     // view neighbours <= v of each view vertex
    std::vector<uint32_t> cols_;   // the view's columns, staged between plan and fill
    std::vector<uint32_t> frontier_, next_;
    uint32_t lo_ = 0;  // smallest view vertex: row scans start at the first entry >= it
};

// Greedy partition of the roots 0..n-1 into bins in id order: a bin is closed
// when its view would exceed max_bytes (the view's exact size, counted while
// the bin grows, up to 48 bytes of alignment; a bin holds at least one source).
// Graphs of at least kParallelBinRoots vertices are cut into contiguous root
// ranges of about equal edge counts, planned in parallel (a bin never spans two
// ranges), as many as keep at least 8 bins per range (up to `threads` and to
// 8 GB of per-range depth bytes, n each; one for a graph of few bins).  bin_of[v]
// for every vertex; returns the number of bins.
constexpr uint64_t kParallelBinRoots = 1u << 16;
uint32_t plan_bins(const uint64_t *rp, const uint32_t *ci, uint64_t n, const Shape &shape, uint64_t max_bytes,
                   uint32_t *bin_of, unsigned threads = 1);

// What a query plan given by positions needs: k positions, bn_count[i] back
// neighbours of position i at positions bn_pos[i][j] (< i), cond_count[i]
// conditions {cond_op[i][j], cond_pos[i][j]} (LESS_THAN: M(i) < M(pos)).
// radius = largest distance from position 0 (every embedding vertex lies
// within it of the root's image); row_radius = largest distance of a position
// that some later position lists as back neighbour (only those vertices' rows
// are scanned); min_deg = query degree of position 0; upper = the conditions
// imply M(i) > M(0) for every position i > 0; forward = they imply M(i) > M(j)
// for every j < i (cliques): every candidate lies above its parent's image, so
// rows need only their entries above their own vertex.
Shape plan_shape(uint32_t k, const uint32_t *bn_count, const uint32_t (*bn_pos)[8], const uint32_t *cond_count,
                 const uint32_t (*cond_op)[8], const uint32_t (*cond_pos)[8]);

}  // namespace g2view

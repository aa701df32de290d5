/*
 * g2_oracle.c - CPU oracle for the subgraph-search hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file restates, in plain C, the algorithms of
 * the reference (lyuheng/g2-aimd) that the CUDA library replaces, so that the
 * library's results can be checked.  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg may load the library built from it; the product
 * (libg2aimd.so) never links or calls it.
 *
 * Restated algorithms, with the reference lines they follow:
 *   orc_mce    Bron-Kerbosch with Tomita pivot over labelled records:
 *              roots           app_BK/BK.h:323-355 (R={v}; u<v -> X, else P;
 *                              degree-0 roots skipped :335-336)
 *              maximality      app_BK/BK.h:78-91   (no P and no X label)
 *              pivot           app_BK/BK.h:282-321 (argmax |P ∩ N(u)| over
 *                              u ∈ P∪X in record order, ties -> later element
 *                              via `>=` :314; non-R record entries are in
 *                              increasing id order, so ties -> larger id)
 *              branching       app_BK/BK.h:445-474 (Q = P \ N(pivot)) and
 *                              :171-280 (child = R ∪ {q} ∪ ((P∪X) ∩ N(q)),
 *                              Q-siblings become X if id < q else P, :226,:278)
 *              The BFS of the reference visits the same tree; this oracle walks
 *              it depth first.  It also reports the clique-size histogram (the
 *              reference prints only the count), the number of tree nodes per
 *              root, and the work model W (algorithmic bytes, see orc_mce).
 *   orc_match  plan-driven enumeration, app_gmatch/gmatch.h:510-671 (candidates
 *              from N(M(parent)) with parent = back neighbour of least degree,
 *              :516-536; conditions <, >, != :559-588; membership in the other
 *              back neighbours' lists :589-601; count at the last level
 *              :602-609).  The PREFIX path (:273-509) enumerates the same set.
 *   orc_kcore  level-synchronous k-core peeling, kmeans/kcore.cpp:12-124
 *              (core number = peel level).
 *   orc_embeddings  brute-force count of injective edge-preserving maps of a
 *              query into a graph (independent check: count = embeddings/|Aut|).
 *   orc_gen_rmat, orc_degeneracy_recode  the seeded R-MAT input (the library's
 *              generator, restated) and the kcore tool's degeneracy order and
 *              recode (kmeans/kcore.cpp:126-191), so that a CPU measurement of
 *              the reference algorithm builds its input without the library.
 * Roots are taken one at a time by the OpenMP threads (dynamic, 1): a few
 * dense-core roots carry most of the work.
 *
 * Parity status: pinned.  The MCE count and histogram are graph invariants
 * (number of maximal cliques with >= 2 vertices, by size), checked against a
 * brute-force maximal-clique enumeration and hand-counted graphs in tests; the
 * match counts are checked against orc_embeddings / |Aut(Q)|; the plans that
 * drive orc_match are pinned against the reference planner's own output.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_OK 0
#define ORC_ERR_INVALID (-1)
#define ORC_ERR_OOM (-3)
#define ORC_ERR_HIST (-10)

/* ------------------------------------------------------------ utilities */

typedef struct {
    uint32_t *buf;
    size_t cap, top;
} arena_t;

static int arena_reserve(arena_t *a, size_t k) {
    if (a->top + k <= a->cap) return 0;
    size_t nc = a->cap ? a->cap : 1024;
    while (nc < a->top + k) nc *= 2;
    uint32_t *nb = (uint32_t *)realloc(a->buf, nc * sizeof(uint32_t));
    if (!nb) return -1;
    a->buf = nb;
    a->cap = nc;
    return 0;
}

/* first index i in [lo, hi) with a[i] >= key */
static uint64_t lower_bound_u32(const uint32_t *a, uint64_t lo, uint64_t hi, uint32_t key) {
    while (lo < hi) {
        uint64_t mid = lo + (hi - lo) / 2;
        if (a[mid] < key) lo = mid + 1; else hi = mid;
    }
    return lo;
}

static int contains_u32(const uint32_t *a, uint64_t lo, uint64_t hi, uint32_t key) {
    uint64_t i = lower_bound_u32(a, lo, hi, key);
    return i < hi && a[i] == key;
}

/* |A ∩ B| for sorted A (na) and sorted B = cols[lo, hi) */
static uint32_t count_common(const uint32_t *A, uint32_t na, const uint32_t *cols, uint64_t lo, uint64_t hi) {
    uint64_t nb = hi - lo;
    uint32_t c = 0;
    if (na == 0 || nb == 0) return 0;
    if ((uint64_t)na * 16 < nb) {
        for (uint32_t i = 0; i < na; i++) c += (uint32_t)contains_u32(cols, lo, hi, A[i]);
        return c;
    }
    uint32_t i = 0;
    uint64_t j = lo;
    while (i < na && j < hi) {
        if (A[i] < cols[j]) i++;
        else if (A[i] > cols[j]) j++;
        else { c++; i++; j++; }
    }
    return c;
}

/* ------------------------------------------------------------------ MCE */

typedef struct {
    const uint64_t *rp;
    const uint32_t *ci;
    arena_t ar;
    uint64_t count, nodes, work;
    uint64_t *hist;
    uint32_t hist_len;
    int hist_overflow;
    uint8_t *inq; /* scratch flags, indexed by arena offset */
    size_t inq_cap;
} mce_ctx;

static int ensure_inq(mce_ctx *c, size_t need) {
    if (need <= c->inq_cap) return 0;
    size_t nc = c->inq_cap ? c->inq_cap : 1024;
    while (nc < need) nc *= 2;
    uint8_t *nb = (uint8_t *)realloc(c->inq, nc);
    if (!nb) return -1;
    c->inq = nb;
    c->inq_cap = nc;
    return 0;
}

static inline uint64_t deg_of(const mce_ctx *c, uint32_t u) { return c->rp[u + 1] - c->rp[u]; }

/*
 * One record (R, P, X) with |R| = r.  P at arena offset po (np entries), X at xo
 * (nx entries), both sorted ascending.  Returns 0 or -1 on allocation failure.
 *
 * Work model W (algorithmic bytes of merge-based set intersection on this
 * tree), per node with P ∪ X non-empty:
 *   4 * [ sum_{u in P∪X} (|P| + deg u)          pivot scoring
 *       + sum_{q in P \ N(pivot)} (|P∪X| + deg q) ]   child construction
 */
static int mce_node(mce_ctx *c, uint32_t r, size_t po, uint32_t np, size_t xo, uint32_t nx) {
    c->nodes++;
    if (np == 0 && nx == 0) {
        c->count++;
        if (c->hist) {
            if (r < c->hist_len) c->hist[r]++;
            else { c->hist[c->hist_len - 1]++; c->hist_overflow = 1; }
        }
        return 0;
    }
    const uint64_t *rp = c->rp;
    const uint32_t *ci = c->ci;
    /* pivot over P ∪ X in increasing id order, `>=` keeps the later (larger) id */
    uint32_t best = 0, pivot = 0;
    {
        uint32_t i = 0, j = 0;
        while (i < np || j < nx) {
            uint32_t u;
            if (j >= nx || (i < np && c->ar.buf[po + i] < c->ar.buf[xo + j])) u = c->ar.buf[po + i++];
            else u = c->ar.buf[xo + j++];
            uint32_t s = count_common(c->ar.buf + po, np, ci, rp[u], rp[u + 1]);
            c->work += 4ull * ((uint64_t)np + deg_of(c, u));
            if (s >= best) { best = s; pivot = u; }
        }
    }
    /* Q = P \ N(pivot): flag the members of P that are not adjacent to pivot */
    size_t qflag = po; /* inq indexed by arena offset of the P entry */
    if (ensure_inq(c, po + np)) return -1;
    uint32_t nq = 0;
    {
        uint64_t lo = rp[pivot], hi = rp[pivot + 1];
        for (uint32_t i = 0; i < np; i++) {
            uint32_t p = c->ar.buf[po + i];
            lo = lower_bound_u32(ci, lo, hi, p);
            int adj = lo < hi && ci[lo] == p;
            c->inq[qflag + i] = (uint8_t)!adj;
            nq += !adj;
        }
    }
    if (nq == 0) return 0;
    for (uint32_t qi = 0; qi < np; qi++) {
        if (!c->inq[qflag + qi]) continue;
        uint32_t q = c->ar.buf[po + qi];
        c->work += 4ull * ((uint64_t)np + nx + deg_of(c, q));
        uint64_t lo = rp[q], hi = rp[q + 1];
        size_t save = c->ar.top;
        if (arena_reserve(&c->ar, (size_t)np + nx)) return -1;
        size_t cpo = c->ar.top;
        uint32_t cnp = 0;
        /* child P: P-labelled or later Q siblings adjacent to q */
        /* child X: X adjacent to q, merged with earlier Q siblings adjacent to q */
        uint32_t *tmpq = NULL;
        uint32_t ntq = 0;
        /* earlier Q siblings adjacent to q are collected after child P, then merged */
        {
            uint64_t l2 = lo;
            for (uint32_t i = 0; i < np; i++) {
                uint32_t w = c->ar.buf[po + i];
                if (w == q) continue;
                l2 = lower_bound_u32(ci, l2, hi, w);
                if (!(l2 < hi && ci[l2] == w)) continue;
                if (c->inq[qflag + i] && w < q) continue; /* goes to X */
                c->ar.buf[cpo + cnp++] = w;
            }
        }
        c->ar.top = cpo + cnp;
        if (arena_reserve(&c->ar, (size_t)np + nx)) return -1;
        size_t tqo = c->ar.top;
        {
            uint64_t l2 = lo;
            for (uint32_t i = 0; i < np; i++) {
                uint32_t w = c->ar.buf[po + i];
                if (!(c->inq[qflag + i] && w < q)) continue;
                l2 = lower_bound_u32(ci, l2, hi, w);
                if (l2 < hi && ci[l2] == w) c->ar.buf[tqo + ntq++] = w;
            }
        }
        c->ar.top = tqo + ntq;
        if (arena_reserve(&c->ar, (size_t)nx + ntq)) return -1;
        size_t cxo = c->ar.top;
        uint32_t cnx = 0;
        {
            uint64_t l2 = lo;
            uint32_t a = 0, b = 0;
            tmpq = c->ar.buf + tqo;
            /* merge X ∩ N(q) with the earlier Q siblings (already ∩ N(q)) */
            while (a < nx || b < ntq) {
                uint32_t w;
                int from_x;
                if (b >= ntq || (a < nx && c->ar.buf[xo + a] < tmpq[b])) { w = c->ar.buf[xo + a++]; from_x = 1; }
                else { w = tmpq[b++]; from_x = 0; }
                if (from_x) {
                    l2 = lower_bound_u32(ci, l2, hi, w);
                    if (!(l2 < hi && ci[l2] == w)) continue;
                }
                c->ar.buf[cxo + cnx++] = w;
                tmpq = c->ar.buf + tqo;
            }
        }
        c->ar.top = cxo + cnx;
        if (mce_node(c, r + 1, cpo, cnp, cxo, cnx)) return -1;
        c->ar.top = save;
    }
    return 0;
}

/*
 * Maximal clique enumeration.
 *   rp, ci, n        CSR (symmetric, sorted, deduplicated, no self loops)
 *   roots, nroots    roots to expand (NULL -> 0..n-1)
 *   threads          OpenMP threads (<= 0: library default)
 *   count            number of maximal cliques
 *   hist, hist_len   hist[s] += maximal cliques of size s (may be NULL)
 *   work             W in bytes (may be NULL)
 *   root_nodes       per-root search-tree node count (may be NULL; nroots entries)
 *   root_work        per-root W (may be NULL)
 */
int orc_mce(const uint64_t *rp, const uint32_t *ci, uint64_t n, const uint32_t *roots, uint64_t nroots,
            int threads, uint64_t *count, uint64_t *hist, uint32_t hist_len, uint64_t *work,
            uint64_t *root_nodes, uint64_t *root_work) {
    if (!rp || (!ci && rp[n] > 0) || !count) return ORC_ERR_INVALID;
    if (hist && hist_len == 0) return ORC_ERR_INVALID;
    if (!roots) nroots = n;
    uint64_t tot_count = 0, tot_work = 0;
    int err = 0, hover = 0;
    if (hist) memset(hist, 0, sizeof(uint64_t) * hist_len);
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#else
    threads = 1;
#endif
#pragma omp parallel num_threads(threads) reduction(+ : tot_count, tot_work) reduction(| : err, hover)
    {
        mce_ctx c;
        memset(&c, 0, sizeof(c));
        c.rp = rp;
        c.ci = ci;
        c.hist_len = hist_len;
        if (hist) c.hist = (uint64_t *)calloc(hist_len, sizeof(uint64_t));
#pragma omp for schedule(dynamic, 1)
        for (int64_t t = 0; t < (int64_t)nroots; t++) {
            uint32_t v = roots ? roots[t] : (uint32_t)t;
            uint64_t lo = rp[v], hi = rp[v + 1];
            uint64_t n0 = c.nodes, w0 = c.work;
            if (hi > lo && !err) {
                uint64_t split = lower_bound_u32(ci, lo, hi, v + 1);
                uint32_t nx = (uint32_t)(split - lo), np = (uint32_t)(hi - split);
                c.ar.top = 0;
                if (arena_reserve(&c.ar, np + nx)) { err = 1; }
                else {
                    memcpy(c.ar.buf, ci + split, np * sizeof(uint32_t));
                    memcpy(c.ar.buf + np, ci + lo, nx * sizeof(uint32_t));
                    c.ar.top = np + nx;
                    if (mce_node(&c, 1, 0, np, np, nx)) err = 1;
                }
            }
            if (root_nodes) root_nodes[t] = c.nodes - n0;
            if (root_work) root_work[t] = c.work - w0;
        }
        tot_count += c.count;
        tot_work += c.work;
        hover |= c.hist_overflow;
        if (hist) {
#pragma omp critical
            for (uint32_t s = 0; s < hist_len; s++) hist[s] += c.hist[s];
            free(c.hist);
        }
        free(c.ar.buf);
        free(c.inq);
    }
    if (err) return ORC_ERR_OOM;
    *count = tot_count;
    if (work) *work = tot_work;
    return hover ? ORC_ERR_HIST : ORC_OK;
}

/* ---------------------------------------------------------------- match */

#define ORC_MAXQ 8

/*
 * Plan in the reference's indexing (system/appbase.h:11-68):
 *   order[p]            query vertex matched at position p (matchOrder)
 *   id2order[u]         position of query vertex u (ID2order)
 *   bn_count[p], bn[p*k + j]        back neighbours of position p (query ids)
 *   cond_count[u], cond[(u*k + j)*2 + {0,1}]  (operator, query vertex)
 */
typedef struct {
    uint32_t k;
    const uint32_t *order, *id2order, *bn_count, *bn, *cond_count, *cond;
} orc_plan;

typedef struct {
    const uint64_t *rp;
    const uint32_t *ci;
    const orc_plan *pl;
    uint32_t M[ORC_MAXQ];
    uint64_t count, work;
} match_ctx;

static void match_level(match_ctx *c, uint32_t pos) {
    const orc_plan *pl = c->pl;
    const uint32_t k = pl->k;
    const uint32_t u = pl->order[pos];
    const uint32_t nb = pl->bn_count[pos];
    /* parent = back neighbour whose image has the least degree (first on ties) */
    uint32_t parent = pl->bn[pos * k];
    uint64_t pmin = c->rp[c->M[pl->id2order[parent]] + 1] - c->rp[c->M[pl->id2order[parent]]];
    for (uint32_t j = 0; j < nb; j++) {
        uint32_t b = pl->bn[pos * k + j];
        uint32_t mb = c->M[pl->id2order[b]];
        uint64_t d = c->rp[mb + 1] - c->rp[mb];
        c->work += 4ull * d;
        if (j > 0 && d < pmin) { pmin = d; parent = b; }
    }
    uint32_t mp = c->M[pl->id2order[parent]];
    for (uint64_t e = c->rp[mp]; e < c->rp[mp + 1]; e++) {
        uint32_t w = c->ci[e];
        int ok = 1;
        for (uint32_t j = 0; j < pl->cond_count[u] && ok; j++) {
            uint32_t op = pl->cond[(u * k + j) * 2];
            uint32_t cm = c->M[pl->id2order[pl->cond[(u * k + j) * 2 + 1]]];
            if (op == 0) ok = w < cm;        /* LESS_THAN   */
            else if (op == 1) ok = w > cm;   /* LARGER_THAN */
            else ok = w != cm;               /* NON_EQUAL   */
        }
        for (uint32_t j = 0; j < nb && ok; j++) {
            uint32_t b = pl->bn[pos * k + j];
            if (b == parent) continue;
            uint32_t mb = c->M[pl->id2order[b]];
            ok = contains_u32(c->ci, c->rp[mb], c->rp[mb + 1], w);
        }
        if (!ok) continue;
        if (pos + 1 == k) c->count++;
        else {
            c->M[pos] = w;
            match_level(c, pos + 1);
        }
    }
}

/*
 * Plan-driven count.  Work model W: 4 bytes x sum over partial embeddings of
 * length p (1 <= p < k) of sum over back neighbours b of position p of
 * deg(M(b)).
 */
int orc_match(const uint64_t *rp, const uint32_t *ci, uint64_t n, const uint32_t *roots, uint64_t nroots,
              int threads, uint32_t k, const uint32_t *order, const uint32_t *id2order,
              const uint32_t *bn_count, const uint32_t *bn, const uint32_t *cond_count,
              const uint32_t *cond, uint64_t *count, uint64_t *work, uint64_t *root_counts) {
    if (!rp || !count || k < 2 || k > ORC_MAXQ) return ORC_ERR_INVALID;
    orc_plan pl = {k, order, id2order, bn_count, bn, cond_count, cond};
    if (!roots) nroots = n;
    uint64_t tot = 0, tw = 0;
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#else
    threads = 1;
#endif
#pragma omp parallel num_threads(threads) reduction(+ : tot, tw)
    {
        match_ctx c;
        memset(&c, 0, sizeof(c));
        c.rp = rp;
        c.ci = ci;
        c.pl = &pl;
#pragma omp for schedule(dynamic, 1)
        for (int64_t t = 0; t < (int64_t)nroots; t++) {
            uint64_t c0 = c.count;
            c.M[0] = roots ? roots[t] : (uint32_t)t;
            match_level(&c, 1);
            if (root_counts) root_counts[t] = c.count - c0;
        }
        tot += c.count;
        tw += c.work;
    }
    *count = tot;
    if (work) *work = tw;
    return ORC_OK;
}

/* ----------------------------------------------------- brute-force checks */

static int q_adj(const uint32_t *qadj, uint32_t k, uint32_t a, uint32_t b) { return qadj[a * k + b] != 0; }

static uint64_t emb_rec(const uint64_t *rp, const uint32_t *ci, uint64_t n, const uint32_t *qadj, uint32_t k,
                        uint32_t *M, uint32_t pos) {
    if (pos == k) return 1;
    uint64_t tot = 0;
    for (uint64_t w = 0; w < n; w++) {
        int ok = 1;
        for (uint32_t j = 0; j < pos && ok; j++) {
            if (M[j] == w) ok = 0;
            else if (q_adj(qadj, k, j, pos)) ok = contains_u32(ci, rp[M[j]], rp[M[j] + 1], (uint32_t)w);
        }
        if (!ok) continue;
        M[pos] = (uint32_t)w;
        tot += emb_rec(rp, ci, n, qadj, k, M, pos + 1);
    }
    return tot;
}

/* Number of injective maps f: V(Q) -> V(G) with {a,b} in E(Q) => {f(a),f(b)} in E(G).
 * qadj is a k x k 0/1 matrix.  Exponential: small graphs only. */
int orc_embeddings(const uint64_t *rp, const uint32_t *ci, uint64_t n, uint32_t k, const uint32_t *qadj,
                   uint64_t *out) {
    if (!rp || !qadj || !out || k == 0 || k > ORC_MAXQ) return ORC_ERR_INVALID;
    uint32_t M[ORC_MAXQ];
    *out = emb_rec(rp, ci, n, qadj, k, M, 0);
    return ORC_OK;
}

/* Brute-force maximal cliques of a small graph (n <= 64): every vertex subset
 * is grown greedily... instead we enumerate cliques by simple recursion over
 * increasing ids and test maximality directly.  hist[s] counts maximal cliques
 * of size s >= 2 (isolated vertices are skipped, as the reference does). */
static void bf_clique(const uint64_t *adjmask, uint32_t n, uint64_t cur, uint32_t size, uint32_t next,
                      uint64_t *count, uint64_t *hist, uint32_t hist_len) {
    /* maximal iff no vertex outside cur is adjacent to every member */
    uint64_t common = ~0ull;
    for (uint32_t v = 0; v < n; v++)
        if (cur >> v & 1) common &= adjmask[v];
    common &= ~cur;
    if (n < 64) common &= (1ull << n) - 1;
    if (common == 0 && size >= 2) {
        (*count)++;
        if (hist && size < hist_len) hist[size]++;
    }
    for (uint32_t v = next; v < n; v++) {
        if (!(common >> v & 1) && size > 0) continue;
        bf_clique(adjmask, n, cur | (1ull << v), size + 1, v + 1, count, hist, hist_len);
    }
}

int orc_mce_bruteforce(const uint64_t *rp, const uint32_t *ci, uint64_t n, uint64_t *count, uint64_t *hist,
                       uint32_t hist_len) {
    if (n > 64 || !rp || !count) return ORC_ERR_INVALID;
    uint64_t adj[64] = {0};
    for (uint64_t v = 0; v < n; v++)
        for (uint64_t e = rp[v]; e < rp[v + 1]; e++) adj[v] |= 1ull << ci[e];
    *count = 0;
    if (hist) memset(hist, 0, sizeof(uint64_t) * hist_len);
    bf_clique(adj, (uint32_t)n, 0, 0, 0, count, hist, hist_len);
    return ORC_OK;
}

/* ---------------------------------------------------------------- k-core */

/*
 * k-core peeling as in kmeans/kcore.cpp:39-124: at level L, repeatedly remove
 * vertices whose residual degree equals L (decrementing neighbours that are
 * still above L); every vertex removed at level L has core number L.
 * order[] receives the peel order (shell by shell, within a shell in removal
 * order), core[v] the core number.  Returns the maximum core number.
 */
int64_t orc_kcore(const uint64_t *rp, const uint32_t *ci, uint64_t n, uint32_t *order, uint32_t *core) {
    uint32_t *deg = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
    uint32_t *buf = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
    if (!deg || !buf) { free(deg); free(buf); return -1; }
    for (uint64_t v = 0; v < n; v++) deg[v] = (uint32_t)(rp[v + 1] - rp[v]);
    uint64_t done = 0;
    uint32_t level = 0;
    int64_t kmax = 0;
    uint8_t *removed = (uint8_t *)calloc(n ? n : 1, 1);
    while (done < n) {
        uint64_t tail = 0;
        for (uint64_t v = 0; v < n; v++)
            if (!removed[v] && deg[v] == level) buf[tail++] = (uint32_t)v;
        for (uint64_t i = 0; i < tail; i++) {
            uint32_t v = buf[i];
            removed[v] = 1;
            for (uint64_t e = rp[v]; e < rp[v + 1]; e++) {
                uint32_t u = ci[e];
                if (deg[u] > level) {
                    deg[u]--;
                    if (deg[u] == level) buf[tail++] = u;
                }
            }
        }
        for (uint64_t i = 0; i < tail; i++) {
            removed[buf[i]] = 1;
            if (order) order[done + i] = buf[i];
            if (core) core[buf[i]] = level;
        }
        if (tail) kmax = level;
        done += tail;
        level++;
    }
    free(deg);
    free(buf);
    free(removed);
    return kmax;
}

/* ------------------------------------------- seeded graphs, degeneracy recode */

/*
 * The synthetic inputs are defined by a seeded generator (the reference ships
 * no datasets), so the checker can build the same graph without the library:
 * orc_gen_rmat restates the counter-based R-MAT generator of the library's
 * g2_gen_rmat (splitmix64 finaliser over (seed, stream 2, 8 * edge + level / 4),
 * four 16-bit quadrant draws per 64-bit word, fixed-point thresholds a, a+b,
 * a+b+c), then symmetrises, drops self loops and duplicates and sorts each row,
 * as the reference's Preprocess does (common/graph.h:720-811) except that
 * isolated vertices keep their ids (n = 2^scale).  Returns malloc'd arrays.
 */
static uint64_t orc_mix64(uint64_t z) {
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
static uint64_t orc_rnd(uint64_t seed, uint64_t stream, uint64_t idx) {
    return orc_mix64(orc_mix64(seed ^ orc_mix64(stream * 0x632be59bd9b4e019ull)) + idx);
}
static int cmp_u32(const void *a, const void *b) {
    uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
    return x < y ? -1 : x > y;
}

int orc_gen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c, uint64_t seed,
                 uint64_t **rp_out, uint32_t **ci_out, uint64_t *m_out) {
    if (scale < 1 || scale > 31 || !edge_factor || !rp_out || !ci_out || !m_out) return ORC_ERR_INVALID;
    const uint64_t n = 1ull << scale, ne = (uint64_t)edge_factor << scale;
    const uint32_t ta = (uint32_t)llround(a * 65536.0), tb = (uint32_t)llround((a + b) * 65536.0),
                   tc = (uint32_t)llround((a + b + c) * 65536.0);
    uint32_t *src = (uint32_t *)malloc(sizeof(uint32_t) * ne), *dst = (uint32_t *)malloc(sizeof(uint32_t) * ne);
    uint64_t *deg = (uint64_t *)calloc(n + 1, sizeof(uint64_t));
    if (!src || !dst || !deg) { free(src); free(dst); free(deg); return ORC_ERR_OOM; }
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < (int64_t)ne; e++) {
        uint32_t s = 0, d = 0;
        uint64_t r = 0;
        for (uint32_t l = 0; l < scale; l++) {
            if ((l & 3) == 0) r = orc_rnd(seed, 2, (uint64_t)e * 8 + (l >> 2));
            uint32_t x = (uint32_t)(r & 0xffff);
            r >>= 16;
            s = (s << 1) | (uint32_t)(x >= tb);
            d = (d << 1) | (uint32_t)((x >= ta && x < tb) || x >= tc);
        }
        src[e] = s;
        dst[e] = d;
    }
    for (uint64_t e = 0; e < ne; e++)
        if (src[e] != dst[e]) { deg[src[e] + 1]++; deg[dst[e] + 1]++; }
    for (uint64_t v = 0; v < n; v++) deg[v + 1] += deg[v];
    uint32_t *tmp = (uint32_t *)malloc(sizeof(uint32_t) * (deg[n] ? deg[n] : 1));
    uint64_t *fill = (uint64_t *)malloc(sizeof(uint64_t) * n);
    if (!tmp || !fill) { free(src); free(dst); free(deg); free(tmp); free(fill); return ORC_ERR_OOM; }
    memcpy(fill, deg, sizeof(uint64_t) * n);
    for (uint64_t e = 0; e < ne; e++)
        if (src[e] != dst[e]) { tmp[fill[src[e]]++] = dst[e]; tmp[fill[dst[e]]++] = src[e]; }
    free(src);
    free(dst);
    /* sort and deduplicate each row; fill[v] becomes the row's kept length */
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t v = 0; v < (int64_t)n; v++) {
        uint32_t *p = tmp + deg[v];
        uint64_t len = deg[v + 1] - deg[v], k = 0;
        qsort(p, len, sizeof(uint32_t), cmp_u32);
        for (uint64_t i = 0; i < len; i++)
            if (k == 0 || p[k - 1] != p[i]) p[k++] = p[i];
        fill[v] = k;
    }
    uint64_t *rp = (uint64_t *)malloc(sizeof(uint64_t) * (n + 1));
    if (!rp) { free(deg); free(tmp); free(fill); return ORC_ERR_OOM; }
    rp[0] = 0;
    for (uint64_t v = 0; v < n; v++) rp[v + 1] = rp[v] + fill[v];
    uint32_t *ci = (uint32_t *)malloc(sizeof(uint32_t) * (rp[n] ? rp[n] : 1));
    if (!ci) { free(deg); free(tmp); free(fill); free(rp); return ORC_ERR_OOM; }
    for (uint64_t v = 0; v < n; v++) memcpy(ci + rp[v], tmp + deg[v], sizeof(uint32_t) * fill[v]);
    free(deg);
    free(tmp);
    free(fill);
    *rp_out = rp;
    *ci_out = ci;
    *m_out = rp[n];
    return ORC_OK;
}

void orc_free(void *p) { free(p); }

/*
 * The degeneracy order that the reference's kcore tool writes
 * (kmeans/kcore.cpp:126-191): core shells ascending, degree ascending inside a
 * shell (ties by old id), ids renamed to positions in that order, rows sorted.
 * Core numbers from orc_kcore.  orp (n+1) and oci (m) are the caller's; core_new
 * (optional) receives core numbers under the new ids.
 */
static const uint64_t *g_sort_rp;
static const uint32_t *g_sort_core;
static int cmp_degeneracy(const void *pa, const void *pb) {
    uint32_t x = *(const uint32_t *)pa, y = *(const uint32_t *)pb;
    if (g_sort_core[x] != g_sort_core[y]) return g_sort_core[x] < g_sort_core[y] ? -1 : 1;
    uint64_t dx = g_sort_rp[x + 1] - g_sort_rp[x], dy = g_sort_rp[y + 1] - g_sort_rp[y];
    if (dx != dy) return dx < dy ? -1 : 1;
    return x < y ? -1 : x > y;
}

int orc_degeneracy_recode(const uint64_t *rp, const uint32_t *ci, uint64_t n, uint64_t *orp, uint32_t *oci,
                          uint32_t *core_new) {
    if (!rp || !orp || (!ci && rp[n]) || (!oci && rp[n])) return ORC_ERR_INVALID;
    uint32_t *core = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
    uint32_t *ord = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
    uint32_t *perm = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
    if (!core || !ord || !perm) { free(core); free(ord); free(perm); return ORC_ERR_OOM; }
    if (orc_kcore(rp, ci, n, NULL, core) < 0) { free(core); free(ord); free(perm); return ORC_ERR_OOM; }
    for (uint64_t v = 0; v < n; v++) ord[v] = (uint32_t)v;
    g_sort_rp = rp;
    g_sort_core = core;
    qsort(ord, n, sizeof(uint32_t), cmp_degeneracy);
    for (uint64_t i = 0; i < n; i++) perm[ord[i]] = (uint32_t)i;
    orp[0] = 0;
    for (uint64_t i = 0; i < n; i++) orp[i + 1] = orp[i] + (rp[ord[i] + 1] - rp[ord[i]]);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t i = 0; i < (int64_t)n; i++) {
        uint32_t v = ord[i];
        uint64_t o = orp[i];
        for (uint64_t e = rp[v]; e < rp[v + 1]; e++) oci[o++] = perm[ci[e]];
        qsort(oci + orp[i], orp[i + 1] - orp[i], sizeof(uint32_t), cmp_u32);
    }
    if (core_new)
        for (uint64_t i = 0; i < n; i++) core_new[i] = core[ord[i]];
    free(core);
    free(ord);
    free(perm);
    return ORC_OK;
}

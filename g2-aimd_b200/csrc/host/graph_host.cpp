// graph_host.cpp - host-side graph preparation for libg2aimd.so:
//   .bin / .vbmap I/O, seeded generators, CSR construction, degeneracy order
//   and id recoding.  None of this is on the timed path; it replaces the
//   reference's offline tools (kmeans/preprocess.cpp, kmeans/kcore.cpp) and the
//   Graph loader (common/graph.h).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <thread>
#include <unordered_set>
#include <vector>

#include "g2_aimd.h"
#include "host/gen_host.h"

namespace {

unsigned host_threads() {
    unsigned t = std::thread::hardware_concurrency();
    if (const char *e = getenv("G2_HOST_THREADS")) t = (unsigned)atoi(e);
    return t ? t : 1;
}

// Run f(begin, end) over [0, n) in dynamically grabbed chunks on all host threads.
void parallel_for(uint64_t n, uint64_t chunk, const std::function<void(uint64_t, uint64_t)> &f) {
    unsigned nt = host_threads();
    if (n <= chunk || nt == 1) {
        if (n) f(0, n);
        return;
    }
    std::atomic<uint64_t> next{0};
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; t++)
        th.emplace_back([&] {
            for (;;) {
                uint64_t b = next.fetch_add(chunk);
                if (b >= n) break;
                f(b, std::min(n, b + chunk));
            }
        });
    for (auto &x : th) x.join();
}

// Counter-based random numbers: splitmix64 finaliser over (seed, stream, index).
inline uint64_t mix64(uint64_t z) {
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
inline uint64_t rnd(uint64_t seed, uint64_t stream, uint64_t idx) {
    return mix64(mix64(seed ^ mix64(stream * 0x632be59bd9b4e019ull)) + idx);
}
inline double u01(uint64_t r) { return (double)(r >> 11) * (1.0 / 9007199254740992.0); }

// Build a symmetric, sorted, deduplicated, self-loop-free CSR from an edge
// list (each pair inserted in both directions).
int build_csr(uint64_t n, const std::vector<uint64_t> &edges, uint64_t **rp_out, uint32_t **ci_out,
              uint64_t *m_out) {
    const uint64_t ne = edges.size();
    std::vector<std::atomic<uint32_t>> deg(n);
    for (auto &d : deg) d.store(0, std::memory_order_relaxed);
    parallel_for(ne, 1 << 20, [&](uint64_t b, uint64_t e) {
        for (uint64_t i = b; i < e; i++) {
            uint32_t s = (uint32_t)(edges[i] >> 32), d = (uint32_t)edges[i];
            if (s == d) continue;
            deg[s].fetch_add(1, std::memory_order_relaxed);
            deg[d].fetch_add(1, std::memory_order_relaxed);
        }
    });
    std::vector<uint64_t> off(n + 1, 0);
    for (uint64_t v = 0; v < n; v++) off[v + 1] = off[v] + deg[v].load(std::memory_order_relaxed);
    std::vector<uint32_t> tmp(off[n]);
    for (uint64_t v = 0; v < n; v++) deg[v].store(0, std::memory_order_relaxed);
    parallel_for(ne, 1 << 20, [&](uint64_t b, uint64_t e) {
        for (uint64_t i = b; i < e; i++) {
            uint32_t s = (uint32_t)(edges[i] >> 32), d = (uint32_t)edges[i];
            if (s == d) continue;
            tmp[off[s] + deg[s].fetch_add(1, std::memory_order_relaxed)] = d;
            tmp[off[d] + deg[d].fetch_add(1, std::memory_order_relaxed)] = s;
        }
    });
    std::vector<uint64_t> len(n);
    parallel_for(n, 4096, [&](uint64_t b, uint64_t e) {
        for (uint64_t v = b; v < e; v++) {
            uint32_t *p = tmp.data() + off[v], *q = tmp.data() + off[v + 1];
            std::sort(p, q);
            len[v] = (uint64_t)(std::unique(p, q) - p);
        }
    });
    uint64_t *rp = (uint64_t *)malloc(sizeof(uint64_t) * (n + 1));
    if (!rp) return G2_ERR_OOM;
    rp[0] = 0;
    for (uint64_t v = 0; v < n; v++) rp[v + 1] = rp[v] + len[v];
    uint32_t *ci = (uint32_t *)malloc(sizeof(uint32_t) * (rp[n] ? rp[n] : 1));
    if (!ci) {
        free(rp);
        return G2_ERR_OOM;
    }
    parallel_for(n, 4096, [&](uint64_t b, uint64_t e) {
        for (uint64_t v = b; v < e; v++) memcpy(ci + rp[v], tmp.data() + off[v], len[v] * sizeof(uint32_t));
    });
    *rp_out = rp;
    *ci_out = ci;
    *m_out = rp[n];
    return G2_OK;
}

inline uint64_t pack(uint32_t a, uint32_t b) { return ((uint64_t)a << 32) | b; }

// Append cliques on disjoint random vertex sets (rejection sampling, one RNG
// stream, so the sets do not depend on the thread count).
int plant_cliques(uint64_t n, uint32_t count, uint32_t smin, uint32_t smax, uint64_t seed,
                  std::vector<uint64_t> &edges) {
    if (count == 0) return G2_OK;
    if (smin < 2 || smax < smin) return G2_ERR_INVALID;
    uint64_t need = 0;
    std::vector<uint32_t> sizes(count);
    for (uint32_t c = 0; c < count; c++) {
        sizes[c] = smin + (uint32_t)(rnd(seed, 11, c) % (uint64_t)(smax - smin + 1));
        need += sizes[c];
    }
    if (need > n) return G2_ERR_INVALID;
    std::unordered_set<uint32_t> used;
    uint64_t ctr = 0;
    for (uint32_t c = 0; c < count; c++) {
        std::vector<uint32_t> mem;
        while (mem.size() < sizes[c]) {
            uint32_t v = (uint32_t)(rnd(seed, 12, ctr++) % n);
            if (used.insert(v).second) mem.push_back(v);
        }
        for (size_t i = 0; i < mem.size(); i++)
            for (size_t j = i + 1; j < mem.size(); j++) edges.push_back(pack(mem[i], mem[j]));
    }
    return G2_OK;
}

}  // namespace

namespace g2host {
int planted_edges(uint64_t n, uint32_t count, uint32_t smin, uint32_t smax, uint64_t seed,
                  std::vector<uint64_t> &edges) {
    return plant_cliques(n, count, smin, smax, seed, edges);
}
}  // namespace g2host

extern "C" {

void g2_free(void *p) { free(p); }

int g2_read_bin(const char *path, uint64_t **row_ptrs, uint32_t **cols, uint64_t *n, uint64_t *m) {
    if (!path || !row_ptrs || !cols || !n || !m) return G2_ERR_INVALID;
    FILE *f = fopen(path, "rb");
    if (!f) return G2_ERR_IO;
    uint64_t hdr[4];
    if (fread(hdr, sizeof(uint64_t), 4, f) != 4 || hdr[0] != 4 || hdr[1] != 8) {
        fclose(f);
        return G2_ERR_IO;
    }
    uint64_t nn = hdr[2], mm = hdr[3];
    uint64_t *rp = (uint64_t *)malloc(sizeof(uint64_t) * (nn + 1));
    uint32_t *ci = (uint32_t *)malloc(sizeof(uint32_t) * (mm ? mm : 1));
    if (!rp || !ci) {
        free(rp);
        free(ci);
        fclose(f);
        return G2_ERR_OOM;
    }
    if (fread(rp, sizeof(uint64_t), nn + 1, f) != nn + 1 || fread(ci, sizeof(uint32_t), mm, f) != mm ||
        rp[nn] != mm) {
        free(rp);
        free(ci);
        fclose(f);
        return G2_ERR_IO;
    }
    fclose(f);
    *row_ptrs = rp;
    *cols = ci;
    *n = nn;
    *m = mm;
    return G2_OK;
}

int g2_read_snap(const char *path, int preprocess, uint64_t **row_ptrs, uint32_t **cols, uint64_t *n,
                 uint64_t *m) {
    if (!path || !row_ptrs || !cols || !n || !m) return G2_ERR_INVALID;
    // Graph::readSnapFile (common/graph.h:268-358): lines that start with a
    // digit hold an edge "u v" (more columns ignored); ids are shifted by the
    // smallest one; every edge is stored in both directions, rows sorted
    FILE *f = fopen(path, "rb");
    if (!f) return G2_ERR_IO;
    std::vector<uint32_t> eu, ev;
    uint64_t lo = UINT64_MAX, hi = 0;
    char line[4096];
    bool bad = false;
    while (fgets(line, sizeof(line), f)) {
        if (!(line[0] >= '0' && line[0] <= '9')) continue;
        char *end = nullptr;
        const unsigned long long a = strtoull(line, &end, 10);
        char *end2 = nullptr;
        const unsigned long long b = strtoull(end, &end2, 10);
        if (end2 == end || a > UINT32_MAX || b > UINT32_MAX) {
            bad = true;
            break;
        }
        eu.push_back((uint32_t)a);
        ev.push_back((uint32_t)b);
        lo = std::min<uint64_t>(lo, std::min(a, b));
        hi = std::max<uint64_t>(hi, std::max(a, b));
    }
    fclose(f);
    if (bad) return G2_ERR_IO;
    uint64_t nn = eu.empty() ? 0 : hi - lo + 1;
    std::vector<uint64_t> rp(nn + 1, 0);
    for (size_t i = 0; i < eu.size(); i++) {
        rp[eu[i] - lo + 1]++;
        rp[ev[i] - lo + 1]++;
    }
    for (uint64_t v = 0; v < nn; v++) rp[v + 1] += rp[v];
    std::vector<uint32_t> ci(rp[nn]);
    {
        std::vector<uint64_t> pos(rp.begin(), rp.end() - 1);
        for (size_t i = 0; i < eu.size(); i++) {
            const uint32_t a = (uint32_t)(eu[i] - lo), b = (uint32_t)(ev[i] - lo);
            ci[pos[a]++] = b;
            ci[pos[b]++] = a;
        }
    }
    std::vector<uint32_t>().swap(eu);
    std::vector<uint32_t>().swap(ev);
    parallel_for(nn, 4096, [&](uint64_t a, uint64_t b) {
        for (uint64_t v = a; v < b; v++) std::sort(ci.begin() + rp[v], ci.begin() + rp[v + 1]);
    });
    if (preprocess) {
        // Graph::Preprocess (common/graph.h:720-804): parallel edges and self
        // loops go, then vertices left without neighbours, the others keeping
        // their order
        uint64_t w = 0;
        std::vector<uint64_t> nrp(nn + 1, 0);
        for (uint64_t u = 0; u < nn; u++) {
            const uint64_t b = rp[u], e = rp[u + 1];
            nrp[u] = w;
            for (uint64_t j = b; j < e; j++) {
                const uint32_t v = ci[j];
                if ((j > b && v == ci[j - 1]) || v == u) continue;
                ci[w++] = v;
            }
        }
        nrp[nn] = w;
        std::vector<uint32_t> id(nn, UINT32_MAX);
        uint64_t k = 0;
        for (uint64_t u = 0; u < nn; u++)
            if (nrp[u + 1] > nrp[u]) id[u] = (uint32_t)k++;
        rp.assign(k + 1, 0);
        for (uint64_t u = 0; u < nn; u++)
            if (id[u] != UINT32_MAX) rp[id[u]] = nrp[u];
        rp[k] = w;
        for (uint64_t j = 0; j < w; j++) ci[j] = id[ci[j]];
        ci.resize(w);
        nn = k;
    }
    uint64_t *orp = (uint64_t *)malloc(sizeof(uint64_t) * (nn + 1));
    uint32_t *oci = (uint32_t *)malloc(sizeof(uint32_t) * (ci.size() ? ci.size() : 1));
    if (!orp || !oci) {
        free(orp);
        free(oci);
        return G2_ERR_OOM;
    }
    memcpy(orp, rp.data(), sizeof(uint64_t) * (nn + 1));
    if (!ci.empty()) memcpy(oci, ci.data(), sizeof(uint32_t) * ci.size());
    *row_ptrs = orp;
    *cols = oci;
    *n = nn;
    *m = ci.size();
    return G2_OK;
}

int g2_write_bin(const char *path, const uint64_t *row_ptrs, const uint32_t *cols, uint64_t n, uint64_t m) {
    if (!path || !row_ptrs || (!cols && m)) return G2_ERR_INVALID;
    FILE *f = fopen(path, "wb");
    if (!f) return G2_ERR_IO;
    uint64_t hdr[4] = {sizeof(uint32_t), sizeof(uint64_t), n, m};
    bool ok = fwrite(hdr, sizeof(uint64_t), 4, f) == 4 && fwrite(row_ptrs, sizeof(uint64_t), n + 1, f) == n + 1 &&
              (m == 0 || fwrite(cols, sizeof(uint32_t), m, f) == m);
    ok = (fclose(f) == 0) && ok;
    return ok ? G2_OK : G2_ERR_IO;
}

int g2_write_vbmap(const char *path, uint32_t nbins, const uint32_t *bins, uint64_t n) {
    if (!path || nbins == 0) return G2_ERR_INVALID;
    FILE *f = fopen(path, "w");
    if (!f) return G2_ERR_IO;
    fprintf(f, "%u ", nbins);
    for (uint64_t v = 0; v < n; v++) fprintf(f, "%u ", bins ? bins[v] : 0u);
    return fclose(f) == 0 ? G2_OK : G2_ERR_IO;
}

int g2_read_vbmap(const char *path, uint64_t n, uint32_t *nbins, uint32_t *bins) {
    if (!path || !nbins) return G2_ERR_INVALID;
    FILE *f = fopen(path, "r");
    if (!f) return G2_ERR_IO;
    if (fscanf(f, "%u", nbins) != 1) {
        fclose(f);
        return G2_ERR_IO;
    }
    for (uint64_t v = 0; v < n; v++) {
        unsigned b;
        if (fscanf(f, "%u", &b) != 1 || b >= *nbins) {
            fclose(f);
            return G2_ERR_IO;
        }
        if (bins) bins[v] = b;
    }
    fclose(f);
    return G2_OK;
}

int g2_gen_er(uint64_t n, double p, uint32_t nplanted, uint32_t planted_size, uint64_t seed, uint64_t **row_ptrs,
              uint32_t **cols, uint64_t *out_n, uint64_t *out_m) {
    if (n < 2 || n > 1000000 || p < 0 || p > 1 || !row_ptrs || !cols || !out_n || !out_m) return G2_ERR_INVALID;
    std::vector<std::vector<uint64_t>> per(n);
    parallel_for(n, 16, [&](uint64_t b, uint64_t e) {
        for (uint64_t i = b; i < e; i++)
            for (uint64_t j = i + 1; j < n; j++)
                if (u01(rnd(seed, 1, i * n + j)) < p) per[i].push_back(pack((uint32_t)i, (uint32_t)j));
    });
    std::vector<uint64_t> edges;
    for (auto &v : per) edges.insert(edges.end(), v.begin(), v.end());
    int rc = plant_cliques(n, nplanted, planted_size, planted_size, seed, edges);
    if (rc) return rc;
    *out_n = n;
    return build_csr(n, edges, row_ptrs, cols, out_m);
}

int g2_gen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c, uint32_t nplanted,
                uint32_t planted_min, uint32_t planted_max, uint64_t seed, uint64_t **row_ptrs, uint32_t **cols,
                uint64_t *out_n, uint64_t *out_m) {
    if (scale < 1 || scale > 31 || edge_factor == 0 || a < 0 || b < 0 || c < 0 || a + b + c > 1 || !row_ptrs ||
        !cols || !out_n || !out_m)
        return G2_ERR_INVALID;
    const uint64_t n = 1ull << scale, ne = (uint64_t)edge_factor << scale;
    // quadrant thresholds in 16-bit fixed point: four levels per 64-bit draw
    const uint32_t ta = (uint32_t)llround(a * 65536.0), tb = (uint32_t)llround((a + b) * 65536.0),
                   tc = (uint32_t)llround((a + b + c) * 65536.0);
    std::vector<uint64_t> edges(ne);
    parallel_for(ne, 1 << 16, [&](uint64_t lo, uint64_t hi) {
        for (uint64_t e = lo; e < hi; e++) {
            uint32_t s = 0, d = 0;
            uint64_t r = 0;
            for (uint32_t l = 0; l < scale; l++) {
                if ((l & 3) == 0) r = rnd(seed, 2, e * 8 + (l >> 2));
                uint32_t x = (uint32_t)(r & 0xffff);
                r >>= 16;
                uint32_t sb = x >= tb, db = (x >= ta && x < tb) || x >= tc;
                s = (s << 1) | sb;
                d = (d << 1) | db;
            }
            edges[e] = pack(s, d);
        }
    });
    int rc = plant_cliques(n, nplanted, planted_min, planted_max, seed, edges);
    if (rc) return rc;
    *out_n = n;
    return build_csr(n, edges, row_ptrs, cols, out_m);
}

int g2_gen_chunglu(uint64_t n, double gamma, double avg_degree, uint64_t seed, uint64_t **row_ptrs,
                   uint32_t **cols, uint64_t *out_n, uint64_t *out_m) {
    if (n < 2 || n > (1ull << 31) || gamma <= 1.0 || avg_degree <= 0 || !row_ptrs || !cols || !out_n || !out_m)
        return G2_ERR_INVALID;
    std::vector<double> cdf(n + 1, 0.0);
    const double ex = -1.0 / (gamma - 1.0);
    for (uint64_t i = 0; i < n; i++) cdf[i + 1] = cdf[i] + std::pow((double)(i + 1), ex);
    const double tot = cdf[n];
    const uint64_t ne = (uint64_t)llround((double)n * avg_degree / 2.0);
    std::vector<uint64_t> edges(ne);
    auto pick = [&](double u) -> uint32_t {
        double x = u * tot;
        uint64_t i = (uint64_t)(std::upper_bound(cdf.begin() + 1, cdf.end(), x) - (cdf.begin() + 1));
        return (uint32_t)std::min(i, n - 1);
    };
    parallel_for(ne, 1 << 16, [&](uint64_t lo, uint64_t hi) {
        for (uint64_t e = lo; e < hi; e++)
            edges[e] = pack(pick(u01(rnd(seed, 3, 2 * e))), pick(u01(rnd(seed, 3, 2 * e + 1))));
    });
    *out_n = n;
    return build_csr(n, edges, row_ptrs, cols, out_m);
}

// Batagelj-Zaversnik bucket peeling: core numbers in O(n + m).
int g2_degeneracy_order(const uint64_t *rp, const uint32_t *ci, uint64_t n, uint32_t *perm, uint32_t *core_out) {
    if (!rp || !perm || (n && !ci && rp[n])) return G2_ERR_INVALID;
    if (n == 0) return G2_OK;
    std::vector<uint32_t> deg(n), pos(n), vert(n);
    uint32_t md = 0;
    for (uint64_t v = 0; v < n; v++) {
        deg[v] = (uint32_t)(rp[v + 1] - rp[v]);
        md = std::max(md, deg[v]);
    }
    std::vector<uint64_t> bin(md + 2, 0);
    for (uint64_t v = 0; v < n; v++) bin[deg[v]]++;
    uint64_t start = 0;
    for (uint32_t d = 0; d <= md; d++) {
        uint64_t num = bin[d];
        bin[d] = start;
        start += num;
    }
    for (uint64_t v = 0; v < n; v++) {
        pos[v] = (uint32_t)bin[deg[v]];
        vert[pos[v]] = (uint32_t)v;
        bin[deg[v]]++;
    }
    for (uint32_t d = md; d >= 1; d--) bin[d] = bin[d - 1];
    bin[0] = 0;
    for (uint64_t i = 0; i < n; i++) {
        uint32_t v = vert[i];
        for (uint64_t e = rp[v]; e < rp[v + 1]; e++) {
            uint32_t u = ci[e];
            if (deg[u] > deg[v]) {
                uint32_t du = deg[u];
                uint64_t pu = pos[u], pw = bin[du];
                uint32_t w = vert[pw];
                if (u != w) {
                    pos[u] = (uint32_t)pw;
                    vert[pu] = w;
                    pos[w] = (uint32_t)pu;
                    vert[pw] = u;
                }
                bin[du]++;
                deg[u]--;
            }
        }
    }
    // deg[] now holds core numbers; order by (core, degree, old id)
    std::vector<uint32_t> ord(n);
    for (uint64_t v = 0; v < n; v++) ord[v] = (uint32_t)v;
    std::sort(ord.begin(), ord.end(), [&](uint32_t x, uint32_t y) {
        if (deg[x] != deg[y]) return deg[x] < deg[y];
        uint64_t dx = rp[x + 1] - rp[x], dy = rp[y + 1] - rp[y];
        if (dx != dy) return dx < dy;
        return x < y;
    });
    for (uint64_t i = 0; i < n; i++) perm[ord[i]] = (uint32_t)i;
    if (core_out) memcpy(core_out, deg.data(), n * sizeof(uint32_t));
    return G2_OK;
}

int g2_recode(const uint64_t *rp, const uint32_t *ci, uint64_t n, const uint32_t *perm, uint64_t *orp,
              uint32_t *oci) {
    if (!rp || !perm || !orp || (!oci && rp[n]) || (!ci && rp[n])) return G2_ERR_INVALID;
    std::vector<uint64_t> inv(n);
    for (uint64_t v = 0; v < n; v++) {
        if (perm[v] >= n) return G2_ERR_INVALID;
        inv[perm[v]] = v;
    }
    orp[0] = 0;
    for (uint64_t i = 0; i < n; i++) orp[i + 1] = orp[i] + (rp[inv[i] + 1] - rp[inv[i]]);
    parallel_for(n, 4096, [&](uint64_t b, uint64_t e) {
        for (uint64_t i = b; i < e; i++) {
            uint64_t v = inv[i], o = orp[i];
            for (uint64_t k = rp[v]; k < rp[v + 1]; k++) oci[o++] = perm[ci[k]];
            std::sort(oci + orp[i], oci + orp[i + 1]);
        }
    });
    return G2_OK;
}

}  // extern "C"

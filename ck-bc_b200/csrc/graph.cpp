// Host-side graph ingest, normalisation, CSR build and seeded generators.
//
// Ingest follows the reference program's input path:
//   read_graph   bc2d.c:175-254  ("u v" lines, '#' comment lines, "Nodes:" echo,
//                                  abort on id >= N)
//   mirror       bc2d.c:152-170  (undirected unless -U)
//   norm_graph   bc2d.c:430-453  (sort, drop duplicates and self-loops)
//   build_csc    bc2d.c:472-501  (counting sort by destination; uint32 ids)
// The reference sorts an array of 64-bit pairs with qsort and then counting-
// sorts it into CSC.  Here the CSR is built directly with a counting pass,
// each adjacency list is sorted and deduplicated in parallel, and the result
// is the same set of lists (sorted ascending) as the reference's CSC.
//
// Generators (no counterpart in the reference, whose R-MAT option is disabled,
// bc2d.c:663-664, 802-810).  All use splitmix64 from bcg_common.hpp; work is
// split into fixed-size chunks whose streams depend only on (seed, chunk), so
// the output is identical for any thread count.
//   rmat  : ef * 2^scale edge draws; each draw descends `scale` levels of the
//           adjacency matrix choosing quadrant (0,0),(0,1),(1,0),(1,1) with
//           probabilities a, b, c, 1-a-b-c (Chakrabarti, Zhan, Faloutsos 2004),
//           most significant bit first, no vertex permutation.  Optional pendant
//           trees: floor(pendant_frac * 2^scale) distinct anchors drawn from
//           [0, 2^scale); in increasing anchor order each gets a random
//           recursive tree of size k ~ Geometric(1/pendant_mean) on {1,2,...}:
//           tree vertex i (numbered after all earlier vertices) attaches to a
//           uniform choice among the anchor and tree vertices 0..i-1.
//   er    : G(n, M) with M = ef * 2^scale uniform (u, v) draws.
//   grid  : w x h 4-neighbour grid, vertex y*w + x; edges visited row-major
//           (right edge then down edge of each vertex), each dropped with
//           probability `drop`; the largest connected component is kept and
//           relabelled in increasing id order (ties: smallest first vertex).
// Every generator then goes through the same normalisation as file input.
#include <algorithm>
#include <cerrno>
#include <cinttypes>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "bcg_common.hpp"

#ifdef _OPENMP
#include <omp.h>
#endif

namespace bcg {

static thread_local std::string g_last_error;

int set_error(int code, const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

void clear_error() { g_last_error.clear(); }

const char *last_error() { return g_last_error.c_str(); }

// ---------------------------------------------------------------------------
// CSR build from edge pairs.
// ---------------------------------------------------------------------------

// Builds sorted, duplicate-free, loop-free adjacency lists.  For undirected
// input every pair (u, v) contributes v to u's list and u to v's list.  For
// directed input (-U) pair (u, v) contributes u to v's list: the reference's
// CSC column of v holds the rows u of edges (u, v) (build_csc bc2d.c:479,492)
// and its BFS walks a column's rows (scan_col_mono2 cuda_kernels.cu:509).
static int build_csr(const uint64_t *pairs, uint64_t npairs, uint64_t n,
                     bool undirected, bcg_host_csr *out) {
    if (n == 0 || n > 0xFFFFFFFEull)
        return set_error(BCG_ERR_RANGE, "vertex count %" PRIu64 " outside [1, 2^32-2]", n);
    std::vector<uint64_t> cnt(n + 1, 0);
    for (uint64_t i = 0; i < npairs; ++i) {
        uint64_t u = pairs[2 * i], v = pairs[2 * i + 1];
        if (u >= n || v >= n)
            return set_error(BCG_ERR_ARG, "edge %" PRIu64 " (%" PRIu64 ", %" PRIu64
                             ") has an id >= n=%" PRIu64, i, u, v, n);
        if (u == v) continue;
        if (undirected) { cnt[u]++; cnt[v]++; }
        else cnt[v]++;
    }
    std::vector<uint64_t> start(n + 1, 0);
    for (uint64_t v = 0; v < n; ++v) start[v + 1] = start[v] + cnt[v];
    uint64_t total = start[n];
    std::vector<uint32_t> tmp;
    try { tmp.resize(total); } catch (...) {
        return set_error(BCG_ERR_OOM, "cannot allocate %" PRIu64 " adjacency entries", total);
    }
    std::vector<uint64_t> pos(start.begin(), start.end() - 1);
    for (uint64_t i = 0; i < npairs; ++i) {
        uint64_t u = pairs[2 * i], v = pairs[2 * i + 1];
        if (u == v) continue;
        if (undirected) { tmp[pos[u]++] = (uint32_t)v; tmp[pos[v]++] = (uint32_t)u; }
        else tmp[pos[v]++] = (uint32_t)u;
    }
    std::vector<uint64_t> ndeg(n, 0);
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t v = 0; v < (int64_t)n; ++v) {
        uint32_t *b = tmp.data() + start[v], *e = tmp.data() + start[v + 1];
        std::sort(b, e);
        ndeg[v] = (uint64_t)(std::unique(b, e) - b);
    }
    uint64_t nnz = 0;
    for (uint64_t v = 0; v < n; ++v) nnz += ndeg[v];
    if (nnz > 0xFFFFFFFFull)
        return set_error(BCG_ERR_RANGE, "%" PRIu64 " adjacency entries exceed uint32 offsets", nnz);
    out->n = (uint32_t)n;
    out->nnz = nnz;
    out->offsets = (uint32_t *)malloc((n + 1) * sizeof(uint32_t));
    out->adj = (uint32_t *)malloc((nnz ? nnz : 1) * sizeof(uint32_t));
    if (!out->offsets || !out->adj) {
        free(out->offsets); free(out->adj);
        out->offsets = out->adj = nullptr;
        return set_error(BCG_ERR_OOM, "cannot allocate CSR of %" PRIu64 " entries", nnz);
    }
    out->offsets[0] = 0;
    for (uint64_t v = 0; v < n; ++v) out->offsets[v + 1] = out->offsets[v] + (uint32_t)ndeg[v];
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t v = 0; v < (int64_t)n; ++v)
        memcpy(out->adj + out->offsets[v], tmp.data() + start[v], ndeg[v] * sizeof(uint32_t));
    return BCG_OK;
}

// ---------------------------------------------------------------------------
// Edge-list reader.
// ---------------------------------------------------------------------------

// sscanf "%lu" on one field: optional leading white space and sign, then
// decimal digits (strtoull semantics: a value past 2^64-1 saturates, a minus
// sign negates modulo 2^64).  Returns false when there is no digit.
static bool scan_u64(const char *&p, const char *end, uint64_t &out) {
    while (p < end && (*p == ' ' || *p == '\t' || *p == '\r' || *p == '\v' || *p == '\f' || *p == '\n')) ++p;
    bool neg = false;
    if (p < end && (*p == '+' || *p == '-')) neg = (*p++ == '-');
    if (p >= end || *p < '0' || *p > '9') return false;
    uint64_t v = 0;
    bool sat = false;
    for (; p < end && *p >= '0' && *p <= '9'; ++p) {
        const uint64_t d = (uint64_t)(*p - '0');
        if (v > (UINT64_MAX - d) / 10) sat = true;
        else v = v * 10 + d;
    }
    out = sat ? UINT64_MAX : (neg ? (uint64_t)0 - v : v);
    return true;
}

namespace {
// What one chunk of an edge-list file holds (lines [begin, end) of the file).
struct EdgeChunk {
    std::vector<uint64_t> pairs;
    uint64_t lines = 0;                   // non-comment lines, the reference's line count
    uint64_t bad_line = 0;                // 1-based within the chunk, 0 = none
    uint64_t bad_u = 0, bad_v = 0;
    std::string bad_text;
    std::vector<std::pair<uint64_t, std::string>> echo;  // (lines before it, text)
};
}  // namespace

static void parse_chunk(const char *b, const char *e, uint64_t n, bool echo, EdgeChunk &c) {
    const char *ls = b;
    while (ls < e) {
        const char *le = static_cast<const char *>(memchr(ls, '\n', (size_t)(e - ls)));
        if (!le) le = e;
        const char *next = (le < e) ? le + 1 : e;
        if (memchr(ls, '#', (size_t)(le - ls))) {
            if (echo) {
                const std::string line(ls, le);
                if (line.find("Nodes:") != std::string::npos) {
                    uint64_t nn = 0, ne = (uint64_t)-1;
                    if (sscanf(line.c_str(), "# Nodes: %" SCNu64 " Edges: %" SCNu64, &nn, &ne) >= 1) {
                        char buf[96];
                        snprintf(buf, sizeof(buf), "N=%" PRIu64 " E=%" PRIu64 "\n", nn, ne);
                        c.echo.emplace_back(c.lines, buf);
                    }
                }
            }
            ls = next;
            continue;
        }
        ++c.lines;
        const char *p = ls;
        uint64_t u, v;
        // "%lu %lu": a malformed line is skipped (the reference would keep the
        // previous line's values)
        if (scan_u64(p, le, u) && scan_u64(p, le, v)) {
            if (u >= n || v >= n) {
                c.bad_line = c.lines;
                c.bad_u = u;
                c.bad_v = v;
                c.bad_text.assign(ls, le);
                while (!c.bad_text.empty() && c.bad_text.back() == '\r') c.bad_text.pop_back();
                return;
            }
            c.pairs.push_back(u);
            c.pairs.push_back(v);
        }
        ls = next;
    }
}

// Reads the whole file, cuts it into chunks at line ends and parses them in
// parallel; echo lines, the first bad line and the pairs come out in file order.
static int read_edgelist(const char *path, uint64_t n, bool undirected, bool echo,
                         std::vector<uint64_t> &pairs) {
    (void)undirected;
    // Lines are parsed the way read_graph does it (bc2d.c:214-247): a line
    // that contains '#' anywhere is a comment; otherwise two unsigned decimal
    // integers are read (sscanf "%lu %lu").  Lines are read whole, so lines
    // longer than the reference's MAX_LINE=1024 buffer are not split.
    FILE *fp = fopen(path, "rb");
    if (!fp) return set_error(BCG_ERR_IO, "Cannot open file %s...", path);
    std::vector<char> buf;
    if (fseek(fp, 0, SEEK_END) == 0) {
        const long sz = ftell(fp);
        if (sz > 0) buf.resize((size_t)sz);
        rewind(fp);
        if (sz > 0) buf.resize(fread(buf.data(), 1, buf.size(), fp));
    } else {  // not seekable: read in pieces
        char tmp[1 << 16];
        size_t got;
        while ((got = fread(tmp, 1, sizeof(tmp), fp)) > 0) buf.insert(buf.end(), tmp, tmp + got);
    }
    const bool err = ferror(fp);
    fclose(fp);
    if (err) return set_error(BCG_ERR_IO, "read error on %s", path);
    const char *base = buf.data(), *end = base + buf.size();
    int nt = 1;
#ifdef _OPENMP
    nt = omp_get_max_threads();
#endif
    const size_t want = (size_t)nt * 4;
    std::vector<const char *> cut{base};
    for (size_t i = 1; i < want; ++i) {
        const char *q = base + buf.size() * i / want;
        if (q <= cut.back()) continue;
        const char *nl = static_cast<const char *>(memchr(q, '\n', (size_t)(end - q)));
        if (!nl) break;
        if (nl + 1 > cut.back()) cut.push_back(nl + 1);
    }
    cut.push_back(end);
    const size_t nc = cut.size() - 1;
    std::vector<EdgeChunk> ch(nc);
#pragma omp parallel for schedule(dynamic, 1)
    for (long i = 0; i < (long)nc; ++i) parse_chunk(cut[i], cut[i + 1], n, echo, ch[i]);
    uint64_t before = 0, total = 0;
    for (size_t i = 0; i < nc; ++i) {
        for (const auto &ev : ch[i].echo)
            if (!ch[i].bad_line || ev.first < ch[i].bad_line) fputs(ev.second.c_str(), stdout);
        if (ch[i].bad_line)
            return set_error(BCG_ERR_IO,
                             "In file %s line %" PRIu64 " found invalid edge in %s for N=%" PRIu64
                             ": (%" PRIu64 ", %" PRIu64 ")", path, before + ch[i].bad_line,
                             ch[i].bad_text.c_str(), n, ch[i].bad_u, ch[i].bad_v);
        before += ch[i].lines;
        total += ch[i].pairs.size();
    }
    pairs.clear();
    pairs.reserve(total);
    for (auto &c : ch) pairs.insert(pairs.end(), c.pairs.begin(), c.pairs.end());
    return BCG_OK;
}

// ---------------------------------------------------------------------------
// Generators.
// ---------------------------------------------------------------------------

static const uint64_t kChunk = 1u << 16;

static void gen_rmat_pairs(int scale, uint64_t ef, double a, double b, double c, uint64_t seed,
                           std::vector<uint64_t> &pairs) {
    uint64_t m = ef << scale;
    size_t base = pairs.size();
    pairs.resize(base + 2 * m);
    uint64_t *p = pairs.data() + base;
    double ab = a + b, abc = a + b + c;
    int64_t nchunks = (int64_t)((m + kChunk - 1) / kChunk);
#pragma omp parallel for schedule(static)
    for (int64_t ch = 0; ch < nchunks; ++ch) {
        uint64_t st = stream_seed(seed, (uint64_t)ch);
        uint64_t lo = (uint64_t)ch * kChunk, hi = std::min(m, lo + kChunk);
        for (uint64_t i = lo; i < hi; ++i) {
            uint64_t u = 0, v = 0;
            for (int bit = scale - 1; bit >= 0; --bit) {
                double r = u01(st);
                if (r < a) {
                } else if (r < ab) {
                    v |= 1ull << bit;
                } else if (r < abc) {
                    u |= 1ull << bit;
                } else {
                    u |= 1ull << bit;
                    v |= 1ull << bit;
                }
            }
            p[2 * i] = u;
            p[2 * i + 1] = v;
        }
    }
}

static void gen_er_pairs(int scale, uint64_t ef, uint64_t seed, std::vector<uint64_t> &pairs) {
    uint64_t n = 1ull << scale, m = ef << scale;
    size_t base = pairs.size();
    pairs.resize(base + 2 * m);
    uint64_t *p = pairs.data() + base;
    int64_t nchunks = (int64_t)((m + kChunk - 1) / kChunk);
#pragma omp parallel for schedule(static)
    for (int64_t ch = 0; ch < nchunks; ++ch) {
        uint64_t st = stream_seed(seed, (uint64_t)ch);
        uint64_t lo = (uint64_t)ch * kChunk, hi = std::min(m, lo + kChunk);
        for (uint64_t i = lo; i < hi; ++i) {
            p[2 * i] = below(st, n);
            p[2 * i + 1] = below(st, n);
        }
    }
}

// k distinct values from [0, n), partial Fisher-Yates; returns them in draw order.
static std::vector<uint32_t> sample_distinct(uint64_t n, uint64_t k, uint64_t seed) {
    std::vector<uint32_t> perm(n);
    for (uint64_t i = 0; i < n; ++i) perm[i] = (uint32_t)i;
    uint64_t st = stream_seed(seed, 0x5A4D50ull);
    std::vector<uint32_t> out(k);
    for (uint64_t i = 0; i < k; ++i) {
        uint64_t j = i + below(st, n - i);
        std::swap(perm[i], perm[j]);
        out[i] = perm[i];
    }
    return out;
}

// Appends pendant trees; returns the new vertex count.
static uint64_t attach_pendant_trees(uint64_t n0, double frac, double mean, uint64_t seed,
                                     std::vector<uint64_t> &pairs) {
    uint64_t na = (uint64_t)std::floor(frac * (double)n0);
    if (na == 0 || mean < 1.0) return n0;
    std::vector<uint32_t> anchors = sample_distinct(n0, na, seed);
    std::sort(anchors.begin(), anchors.end());
    uint64_t st = stream_seed(seed, 0x7EEull);
    double p = 1.0 / mean;
    double lq = std::log1p(-p);
    uint64_t next = n0;
    std::vector<uint64_t> tree;
    for (uint32_t anc : anchors) {
        uint64_t k = 1;
        if (p < 1.0) {
            double r = u01(st);
            k = 1 + (uint64_t)std::floor(std::log1p(-r) / lq);
        }
        tree.assign(1, anc);
        for (uint64_t i = 0; i < k; ++i) {
            uint64_t parent = tree[below(st, tree.size())];
            pairs.push_back(parent);
            pairs.push_back(next);
            tree.push_back(next);
            ++next;
        }
    }
    return next;
}

static void grid_pairs(uint64_t w, uint64_t h, double drop, uint64_t seed, std::vector<uint64_t> &pairs) {
    uint64_t st = stream_seed(seed, 0x6121Dull);
    for (uint64_t y = 0; y < h; ++y)
        for (uint64_t x = 0; x < w; ++x) {
            uint64_t v = y * w + x;
            if (x + 1 < w && u01(st) >= drop) { pairs.push_back(v); pairs.push_back(v + 1); }
            if (y + 1 < h && u01(st) >= drop) { pairs.push_back(v); pairs.push_back(v + w); }
        }
}

// Keeps the largest connected component of an undirected CSR, relabelled in
// increasing id order.
static int largest_component(bcg_host_csr *g) {
    uint32_t n = g->n;
    std::vector<uint32_t> comp(n, 0xFFFFFFFFu), queue;
    queue.reserve(n);
    uint32_t best = 0, best_size = 0, ncomp = 0;
    for (uint32_t s = 0; s < n; ++s) {
        if (comp[s] != 0xFFFFFFFFu) continue;
        queue.clear();
        queue.push_back(s);
        comp[s] = ncomp;
        for (size_t qi = 0; qi < queue.size(); ++qi) {
            uint32_t u = queue[qi];
            for (uint32_t e = g->offsets[u]; e < g->offsets[u + 1]; ++e) {
                uint32_t w = g->adj[e];
                if (comp[w] == 0xFFFFFFFFu) { comp[w] = ncomp; queue.push_back(w); }
            }
        }
        if (queue.size() > best_size) { best_size = (uint32_t)queue.size(); best = ncomp; }
        ++ncomp;
    }
    std::vector<uint32_t> newid(n, 0xFFFFFFFFu);
    uint32_t nn = 0;
    for (uint32_t v = 0; v < n; ++v) if (comp[v] == best) newid[v] = nn++;
    std::vector<uint64_t> pairs;
    for (uint32_t v = 0; v < n; ++v) {
        if (comp[v] != best) continue;
        for (uint32_t e = g->offsets[v]; e < g->offsets[v + 1]; ++e) {
            uint32_t w = g->adj[e];
            if (v < w) { pairs.push_back(newid[v]); pairs.push_back(newid[w]); }
        }
    }
    bcg_host_csr out{};
    int rc = build_csr(pairs.data(), pairs.size() / 2, nn, true, &out);
    if (rc != BCG_OK) return rc;
    free(g->offsets);
    free(g->adj);
    *g = out;
    return BCG_OK;
}

// "kind:key=value,..." parser.
static bool parse_spec(const char *spec, std::string &kind, std::map<std::string, std::string> &kv) {
    std::string s(spec ? spec : "");
    size_t colon = s.find(':');
    kind = s.substr(0, colon);
    if (colon == std::string::npos) return !kind.empty();
    std::string rest = s.substr(colon + 1);
    size_t pos = 0;
    while (pos < rest.size()) {
        size_t comma = rest.find(',', pos);
        std::string item = rest.substr(pos, comma == std::string::npos ? std::string::npos : comma - pos);
        size_t eq = item.find('=');
        if (eq == std::string::npos || eq == 0) return false;
        kv[item.substr(0, eq)] = item.substr(eq + 1);
        if (comma == std::string::npos) break;
        pos = comma + 1;
    }
    return true;
}

static bool get_num(const std::map<std::string, std::string> &kv, const char *key, double &out) {
    auto it = kv.find(key);
    if (it == kv.end()) return true;
    char *end = nullptr;
    errno = 0;
    double v = strtod(it->second.c_str(), &end);
    if (errno || end == it->second.c_str() || *end) return false;
    out = v;
    return true;
}

}  // namespace bcg

using namespace bcg;

extern "C" {

const char *bcg_last_error(void) { return bcg::last_error(); }

void bcg_csr_free(bcg_host_csr *g) {
    if (!g) return;
    free(g->offsets);
    free(g->adj);
    g->offsets = g->adj = nullptr;
    g->n = 0;
    g->nnz = 0;
}

int bcg_csr_from_pairs(const uint64_t *pairs, uint64_t npairs, uint64_t n, int undirected,
                       bcg_host_csr *out) {
    clear_error();
    if (!out || (npairs && !pairs)) return set_error(BCG_ERR_ARG, "null argument");
    *out = bcg_host_csr{};
    return build_csr(pairs, npairs, n, undirected != 0, out);
}

int bcg_csr_read_edgelist(const char *path, uint64_t n, int undirected, int echo_header,
                          bcg_host_csr *out) {
    clear_error();
    if (!path || !out) return set_error(BCG_ERR_ARG, "null argument");
    *out = bcg_host_csr{};
    if (n == 0) return set_error(BCG_ERR_ARG, "number of vertices must be > 0");
    std::vector<uint64_t> pairs;
    int rc = read_edgelist(path, n, undirected != 0, echo_header != 0, pairs);
    if (rc != BCG_OK) return rc;
    return build_csr(pairs.data(), pairs.size() / 2, n, undirected != 0, out);
}

int bcg_csr_generate(const char *spec, bcg_host_csr *out) {
    clear_error();
    if (!out) return set_error(BCG_ERR_ARG, "null argument");
    *out = bcg_host_csr{};
    std::string kind;
    std::map<std::string, std::string> kv;
    if (!parse_spec(spec, kind, kv)) return set_error(BCG_ERR_ARG, "bad generator spec '%s'", spec ? spec : "");
    std::vector<uint64_t> pairs;
    if (kind == "rmat" || kind == "er") {
        double scale = 12, ef = 16, a = 0.57, b = 0.19, c = 0.19, seed = 1;
        double pfrac = 0.0, pmean = 4.0, pseed = -1;
        if (!get_num(kv, "scale", scale) || !get_num(kv, "ef", ef) || !get_num(kv, "a", a) ||
            !get_num(kv, "b", b) || !get_num(kv, "c", c) || !get_num(kv, "seed", seed) ||
            !get_num(kv, "pendant_frac", pfrac) || !get_num(kv, "pendant_mean", pmean) ||
            !get_num(kv, "pendant_seed", pseed))
            return set_error(BCG_ERR_ARG, "bad number in spec '%s'", spec);
        if (scale < 1 || scale > 30 || ef < 1 || ef > 1024)
            return set_error(BCG_ERR_ARG, "scale must be in [1,30] and ef in [1,1024]");
        if (a < 0 || b < 0 || c < 0 || a + b + c > 1.0)
            return set_error(BCG_ERR_ARG, "R-MAT probabilities must be >= 0 and sum to <= 1");
        int sc = (int)scale;
        uint64_t n = 1ull << sc;
        if (kind == "rmat") gen_rmat_pairs(sc, (uint64_t)ef, a, b, c, (uint64_t)seed, pairs);
        else gen_er_pairs(sc, (uint64_t)ef, (uint64_t)seed, pairs);
        if (pfrac > 0) {
            uint64_t ps = pseed < 0 ? ((uint64_t)seed ^ 0x50454E44414E54ull) : (uint64_t)pseed;
            n = attach_pendant_trees(n, pfrac, pmean, ps, pairs);
        }
        return build_csr(pairs.data(), pairs.size() / 2, n, true, out);
    }
    if (kind == "grid") {
        double w = 16, h = 16, drop = 0.0, seed = 3;
        if (!get_num(kv, "w", w) || !get_num(kv, "h", h) || !get_num(kv, "drop", drop) ||
            !get_num(kv, "seed", seed))
            return set_error(BCG_ERR_ARG, "bad number in spec '%s'", spec);
        if (w < 1 || h < 1 || w * h > 4.0e9 || drop < 0 || drop >= 1)
            return set_error(BCG_ERR_ARG, "grid needs w,h >= 1, w*h < 4e9, 0 <= drop < 1");
        grid_pairs((uint64_t)w, (uint64_t)h, drop, (uint64_t)seed, pairs);
        int rc = build_csr(pairs.data(), pairs.size() / 2, (uint64_t)w * (uint64_t)h, true, out);
        if (rc != BCG_OK) return rc;
        return largest_component(out);
    }
    return set_error(BCG_ERR_ARG, "unknown generator '%s'", kind.c_str());
}

int bcg_csr_write_edgelist(const char *path, const bcg_host_csr *g) {
    clear_error();
    if (!path || !g || !g->offsets) return set_error(BCG_ERR_ARG, "null argument");
    FILE *fp = fopen(path, "w");
    if (!fp) return set_error(BCG_ERR_IO, "Cannot open file %s...", path);
    uint64_t m = 0;
    for (uint32_t v = 0; v < g->n; ++v)
        for (uint32_t e = g->offsets[v]; e < g->offsets[v + 1]; ++e) m += (v < g->adj[e]);
    fprintf(fp, "# Nodes: %u Edges: %" PRIu64 "\n", g->n, m);
    for (uint32_t v = 0; v < g->n; ++v)
        for (uint32_t e = g->offsets[v]; e < g->offsets[v + 1]; ++e)
            if (v < g->adj[e]) fprintf(fp, "%u %u\n", v, g->adj[e]);
    int bad = ferror(fp);
    if (fclose(fp) != 0 || bad) return set_error(BCG_ERR_IO, "write to %s failed", path);
    return BCG_OK;
}

// Binary CSR cache: "BCGCSR01", then n, nnz and an FNV-1a checksum of the
// two arrays (all little-endian uint64), then offsets[n+1] and adj[nnz] as
// uint32.  Reading it skips the text parse and the normalisation.
static uint64_t fnv1a_words(const uint32_t *w, uint64_t count, uint64_t h) {
    for (uint64_t i = 0; i < count; ++i) {
        h ^= w[i];
        h *= 0x100000001B3ull;
    }
    return h;
}

static const char kCsrMagic[8] = {'B', 'C', 'G', 'C', 'S', 'R', '0', '1'};

int bcg_csr_write_binary(const char *path, const bcg_host_csr *g) {
    clear_error();
    if (!path || !g || !g->offsets || (g->nnz && !g->adj)) return set_error(BCG_ERR_ARG, "null argument");
    uint64_t h = fnv1a_words(g->offsets, (uint64_t)g->n + 1, 0xCBF29CE484222325ull);
    h = fnv1a_words(g->adj, g->nnz, h);
    const uint64_t head[3] = {g->n, g->nnz, h};
    FILE *fp = fopen(path, "wb");
    if (!fp) return set_error(BCG_ERR_IO, "Cannot open file %s...", path);
    bool ok = fwrite(kCsrMagic, 1, 8, fp) == 8 && fwrite(head, 8, 3, fp) == 3 &&
              fwrite(g->offsets, 4, (size_t)g->n + 1, fp) == (size_t)g->n + 1 &&
              (g->nnz == 0 || fwrite(g->adj, 4, g->nnz, fp) == g->nnz);
    ok = (fclose(fp) == 0) && ok;
    if (!ok) return set_error(BCG_ERR_IO, "write to %s failed", path);
    return BCG_OK;
}

int bcg_csr_read_binary(const char *path, bcg_host_csr *out) {
    clear_error();
    if (!path || !out) return set_error(BCG_ERR_ARG, "null argument");
    *out = bcg_host_csr{};
    FILE *fp = fopen(path, "rb");
    if (!fp) return set_error(BCG_ERR_IO, "Cannot open file %s...", path);
    char magic[8];
    uint64_t head[3];
    if (fread(magic, 1, 8, fp) != 8 || memcmp(magic, kCsrMagic, 8) != 0 || fread(head, 8, 3, fp) != 3) {
        fclose(fp);
        return set_error(BCG_ERR_IO, "%s is not a binary CSR cache", path);
    }
    const uint64_t n = head[0], nnz = head[1];
    if (n == 0 || n > 0xFFFFFFFEull || nnz > 0xFFFFFFFFull) {
        fclose(fp);
        return set_error(BCG_ERR_IO, "%s: bad sizes n=%" PRIu64 " nnz=%" PRIu64, path, n, nnz);
    }
    uint32_t *offs = (uint32_t *)malloc((n + 1) * sizeof(uint32_t));
    uint32_t *adj = (uint32_t *)malloc(std::max<uint64_t>(1, nnz) * sizeof(uint32_t));
    bool ok = offs && adj && fread(offs, 4, n + 1, fp) == n + 1 && (nnz == 0 || fread(adj, 4, nnz, fp) == nnz);
    char extra;
    ok = ok && fread(&extra, 1, 1, fp) == 0;  // nothing after the arrays
    fclose(fp);
    if (ok) {
        uint64_t h = fnv1a_words(offs, n + 1, 0xCBF29CE484222325ull);
        h = fnv1a_words(adj, nnz, h);
        ok = (h == head[2]) && offs[0] == 0 && offs[n] == nnz;
        for (uint64_t v = 0; ok && v < n; ++v) ok = offs[v] <= offs[v + 1];
        for (uint64_t e = 0; ok && e < nnz; ++e) ok = adj[e] < n;
    }
    if (!ok) {
        free(offs);
        free(adj);
        return set_error(BCG_ERR_IO, "%s: truncated or corrupt binary CSR cache", path);
    }
    out->n = (uint32_t)n;
    out->nnz = nnz;
    out->offsets = offs;
    out->adj = adj;
    return BCG_OK;
}

int bcg_sample_sources(uint32_t n, uint64_t k, uint64_t seed, uint32_t *out) {
    clear_error();
    if (!out && k) return set_error(BCG_ERR_ARG, "null argument");
    if (k > n) return set_error(BCG_ERR_ARG, "cannot draw %" PRIu64 " distinct sources from %u", k, n);
    std::vector<uint32_t> s = sample_distinct(n, k, seed);
    memcpy(out, s.data(), k * sizeof(uint32_t));
    return BCG_OK;
}

}  // extern "C"

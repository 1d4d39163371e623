/*
 * Oracle (TEST INFRASTRUCTURE ONLY).  A plain serial C restatement of what
 * the reference computes for BFS, SSSP, WCC and PageRank, plus a CPU twin of
 * the engine's synthetic-graph generators.  Only tests/, the smoke check and
 * the CPU-baseline leg of the benchmark load this library; the engine never
 * does.
 *
 * Conventions followed (reference = PengBo410/CGgraph, paths under CGgraph/):
 *  - every id, offset, weight and result is uint32
 *    (Basic/Type/data_type.hpp:6-15);
 *  - "unreachable" is VertexValue_MAX = 999999999 (Basic/Graph/basic_def.hpp:18);
 *  - BFS: root = 0, level = parent level + 1
 *    (my_project/CGgraph/host_algorithm.hpp:169-177);
 *  - SSSP: dist = min over in-edges of dist[u] + w, applied only when it is
 *    below the current value (host_algorithm.hpp:277-300, device_algorithm.cuh:317-319),
 *    so a vertex whose shortest path is >= 999999999 keeps 999999999;
 *  - CC: label0 = vertex id, labels pushed along OUT-edges with min
 *    (GraphNuma.cuh:539-544, host_algorithm.hpp:412-433).  On a directed
 *    graph the fixpoint is label[v] = min{u : u reaches v}; on a symmetric
 *    graph it is the minimum vertex id of v's weakly connected component;
 *  - PageRank: pr0 = 1/N, pr' = 0.15/N + 0.85 * sum_{u->v} pr[u]/outdeg[u],
 *    no dangling redistribution (GraphNuma.cuh:233-244,545-554,
 *    device_algorithm.cuh:543), evaluated here in FP64 because the
 *    reference's own PageRank is uint32 and does not build.
 *
 * Build: cc -O2 -fopenmp -shared -fPIC cgb_oracle.c -o liboracle.so
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORA_MAX 999999999u

/* ------------------------------------------------------------------ BFS */
/* Queue BFS; the level-synchronous fixpoint of the reference's write_min
 * relaxation (host_algorithm.hpp:164-184). */
int ora_bfs(uint32_t V, const uint32_t* off, const uint32_t* dst, uint32_t root, uint32_t* out)
{
    if (root >= V) return -1;
    uint32_t* q = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)V);
    if (!q) return -2;
    for (uint32_t i = 0; i < V; i++) out[i] = ORA_MAX;
    size_t head = 0, tail = 0;
    out[root] = 0;
    q[tail++] = root;
    while (head < tail) {
        uint32_t u = q[head++];
        uint32_t l = out[u] + 1;
        for (uint32_t e = off[u]; e < off[u + 1]; e++) {
            uint32_t d = dst[e];
            if (out[d] == ORA_MAX) { out[d] = l; q[tail++] = d; }
        }
    }
    free(q);
    return 0;
}

/* ----------------------------------------------------------------- SSSP */
/* Dijkstra with a binary heap keyed by (dist << 32 | vertex). */
typedef struct { uint64_t* a; size_t n, cap; } heap_t;
static int heap_push(heap_t* h, uint64_t k)
{
    if (h->n == h->cap) {
        size_t nc = h->cap ? h->cap * 2 : 1024;
        uint64_t* na = (uint64_t*)realloc(h->a, nc * sizeof(uint64_t));
        if (!na) return -1;
        h->a = na; h->cap = nc;
    }
    size_t i = h->n++;
    while (i > 0) {
        size_t p = (i - 1) / 2;
        if (h->a[p] <= k) break;
        h->a[i] = h->a[p];
        i = p;
    }
    h->a[i] = k;
    return 0;
}
static uint64_t heap_pop(heap_t* h)
{
    uint64_t top = h->a[0];
    uint64_t last = h->a[--h->n];
    size_t i = 0;
    for (;;) {
        size_t c = 2 * i + 1;
        if (c >= h->n) break;
        if (c + 1 < h->n && h->a[c + 1] < h->a[c]) c++;
        if (h->a[c] >= last) break;
        h->a[i] = h->a[c];
        i = c;
    }
    if (h->n) h->a[i] = last;
    return top;
}

int ora_sssp(uint32_t V, const uint32_t* off, const uint32_t* dst, const uint32_t* w, uint32_t root, uint32_t* out)
{
    if (root >= V) return -1;
    heap_t h = {0, 0, 0};
    for (uint32_t i = 0; i < V; i++) out[i] = ORA_MAX;
    out[root] = 0;
    if (heap_push(&h, (uint64_t)root)) return -2;
    while (h.n) {
        uint64_t k = heap_pop(&h);
        uint32_t u = (uint32_t)k;
        uint32_t du = (uint32_t)(k >> 32);
        if (du != out[u]) continue;
        for (uint32_t e = off[u]; e < off[u + 1]; e++) {
            uint64_t nd = (uint64_t)du + (uint64_t)w[e];
            uint32_t d = dst[e];
            if (nd < (uint64_t)out[d]) {
                out[d] = (uint32_t)nd;
                if (heap_push(&h, (nd << 32) | d)) { free(h.a); return -2; }
            }
        }
    }
    free(h.a);
    return 0;
}

/* ------------------------------------------------------------------- CC */
/* Reference CC semantics on any directed graph: label[v] = min{u : u ~> v}.
 * Visiting sources in increasing id order, a BFS from u claims every vertex
 * not yet claimed by a smaller source; each vertex is claimed once. */
int ora_cc(uint32_t V, const uint32_t* off, const uint32_t* dst, uint32_t* out)
{
    uint32_t* q = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(V ? V : 1));
    if (!q) return -2;
    for (uint32_t i = 0; i < V; i++) out[i] = ORA_MAX;
    for (uint32_t s = 0; s < V; s++) {
        if (out[s] != ORA_MAX) continue;
        size_t head = 0, tail = 0;
        out[s] = s;
        q[tail++] = s;
        while (head < tail) {
            uint32_t u = q[head++];
            for (uint32_t e = off[u]; e < off[u + 1]; e++) {
                uint32_t d = dst[e];
                if (out[d] == ORA_MAX) { out[d] = s; q[tail++] = d; }
            }
        }
    }
    free(q);
    return 0;
}

/* Union-find restatement for symmetric graphs (min id of each component);
 * an independent second check of ora_cc on symmetrised inputs. */
static uint32_t uf_find(uint32_t* p, uint32_t x)
{
    while (p[x] != x) { p[x] = p[p[x]]; x = p[x]; }
    return x;
}
int ora_wcc_unionfind(uint32_t V, const uint32_t* off, const uint32_t* dst, uint32_t* out)
{
    for (uint32_t i = 0; i < V; i++) out[i] = i;
    for (uint32_t u = 0; u < V; u++)
        for (uint32_t e = off[u]; e < off[u + 1]; e++) {
            uint32_t a = uf_find(out, u), b = uf_find(out, dst[e]);
            if (a < b) out[b] = a; else if (b < a) out[a] = b;
        }
    for (uint32_t i = 0; i < V; i++) out[i] = uf_find(out, i);
    return 0;
}

/* ------------------------------------------------------------- PageRank */
/* Serial FP64 push, in vertex order. */
int ora_pagerank(uint32_t V, const uint32_t* off, const uint32_t* dst, uint32_t iters, double* out)
{
    if (V == 0) return 0;
    double* acc = (double*)malloc(sizeof(double) * (size_t)V);
    if (!acc) return -2;
    const double N = (double)V;
    for (uint32_t i = 0; i < V; i++) out[i] = 1.0 / N;
    for (uint32_t it = 0; it < iters; it++) {
        memset(acc, 0, sizeof(double) * (size_t)V);
        for (uint32_t u = 0; u < V; u++) {
            uint32_t deg = off[u + 1] - off[u];
            if (!deg) continue;
            double c = out[u] / (double)deg;
            for (uint32_t e = off[u]; e < off[u + 1]; e++) acc[dst[e]] += c;
        }
        for (uint32_t v = 0; v < V; v++) out[v] = 0.15 / N + 0.85 * acc[v];
    }
    free(acc);
    return 0;
}

/* In-edge CSC of a CSR by a counting sort on the destination: sources are
 * visited in ascending order, so every in-list comes out ascending. */
int ora_csc(uint32_t V, const uint32_t* off, const uint32_t* dst, uint32_t* in_off, uint32_t* in_src)
{
    uint32_t* fill = (uint32_t*)malloc(sizeof(uint32_t) * ((size_t)V + 1));
    if (!fill) return -2;
    memset(in_off, 0, sizeof(uint32_t) * ((size_t)V + 1));
    uint32_t E = off[V];
    for (uint32_t e = 0; e < E; e++) in_off[dst[e] + 1]++;
    for (uint32_t v = 0; v < V; v++) in_off[v + 1] += in_off[v];
    memcpy(fill, in_off, sizeof(uint32_t) * ((size_t)V + 1));
    for (uint32_t u = 0; u < V; u++)
        for (uint32_t e = off[u]; e < off[u + 1]; e++) in_src[fill[dst[e]]++] = u;
    free(fill);
    return 0;
}

/* OpenMP FP64 pull over a CSC (in_off/in_src), used as the timed CPU
 * baseline for PageRank since the reference's own PageRank does not build. */
int ora_pagerank_pull_omp(uint32_t V, const uint32_t* off, const uint32_t* in_off, const uint32_t* in_src,
                          uint32_t iters, int threads, double* out)
{
    if (V == 0) return 0;
    double* contrib = (double*)malloc(sizeof(double) * (size_t)V);
    if (!contrib) return -2;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
    const double N = (double)V;
    int64_t n = (int64_t)V;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) out[i] = 1.0 / N;
    for (uint32_t it = 0; it < iters; it++) {
#pragma omp parallel for schedule(static)
        for (int64_t u = 0; u < n; u++) {
            uint32_t deg = off[u + 1] - off[u];
            contrib[u] = deg ? out[u] / (double)deg : 0.0;
        }
#pragma omp parallel for schedule(dynamic, 4096)
        for (int64_t v = 0; v < n; v++) {
            double s = 0.0;
            for (uint32_t e = in_off[v]; e < in_off[v + 1]; e++) s += contrib[in_src[e]];
            out[v] = 0.15 / N + 0.85 * s;
        }
    }
    free(contrib);
    return 0;
}

int ora_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ----------------------------------------------- graph construction twin */
/* CPU twin of the engine's generators, to check them on small sizes.
 * splitmix64 finaliser (Steele, Lea, Flood 2014; public-domain constants). */
static inline uint64_t mix64(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

/* Bijective scramble of scale-bit vertex ids: odd multiply, xor-shift, odd
 * multiply, add, all modulo 2^scale. */
static inline uint32_t scramble(uint64_t x, uint32_t scale, uint64_t m1, uint64_t m2, uint64_t c)
{
    uint64_t mask = (scale >= 64) ? ~0ull : ((1ull << scale) - 1);
    uint32_t sh = scale / 2 ? scale / 2 : 1;
    x = (x * m1) & mask;
    x ^= x >> sh;
    x = (x * m2 + c) & mask;
    return (uint32_t)x;
}

/* RMAT edge i of a (seed, scale) stream, quadrant thresholds t1<t2<t3 in
 * units of 2^-32; optionally scrambled.  Mirrors the device generator. */
void ora_rmat_edges(uint32_t scale, uint64_t nedges, uint64_t seed, uint64_t t1, uint64_t t2, uint64_t t3,
                    int do_scramble, uint32_t* src, uint32_t* dst)
{
    uint64_t m1 = mix64(seed ^ 0x5C0A11ull) | 1ull;
    uint64_t m2 = mix64(seed ^ 0x5C0A12ull) | 1ull;
    uint64_t c = mix64(seed ^ 0x5C0A13ull);
    uint64_t s = mix64(seed);
    /* each edge depends only on its index: the stream is the same for any thread count */
#pragma omp parallel for schedule(static)
    for (uint64_t i = 0; i < nedges; i++) {
        uint64_t u = 0, v = 0;
        for (uint32_t l = 0; l < scale; l++) {
            uint64_t r = mix64(s ^ mix64(i * 64 + l)) >> 32;
            uint64_t bu = r >= t2, bv = (r >= t1 && r < t2) || r >= t3;
            u = (u << 1) | bu;
            v = (v << 1) | bv;
        }
        if (do_scramble) { u = scramble(u, scale, m1, m2, c); v = scramble(v, scale, m1, m2, c); }
        src[i] = (uint32_t)u;
        dst[i] = (uint32_t)v;
    }
}

static uint64_t gcd_u64(uint64_t a, uint64_t b)
{
    while (b) { uint64_t t = a % b; a = b; b = t; }
    return a;
}

static void cl_affine(uint32_t V, uint64_t seed, uint64_t tag, uint64_t* a, uint64_t* b)
{
    *a = V > 1 ? 1 + mix64(seed ^ tag) % (V - 1) : 1;
    while (gcd_u64(*a, V) != 1) *a = *a % (V - 1) + 1;
    *b = mix64(seed ^ (tag + 1)) % V;
}

/* Largest j < V with cum[j] <= r. */
static uint32_t cl_pick(uint64_t r, const uint64_t* cum, uint32_t V)
{
    uint32_t lo = 0, hi = V;
    while (hi - lo > 1) {
        uint32_t mid = lo + (hi - lo) / 2;
        if (cum[mid] <= r) lo = mid; else hi = mid;
    }
    return lo;
}

/* Chung-Lu edge stream of the device generator (gen.cu): vertex weights
 * floor(2^40 / (i + i0)), both endpoints drawn from the integer prefix sums
 * with counter-hashed draws, then mapped by two affine permutations. */
int ora_chunglu_edges(uint32_t V, uint64_t n, uint32_t i0, uint64_t seed, uint32_t* src, uint32_t* dst)
{
    uint64_t* cum = (uint64_t*)malloc(sizeof(uint64_t) * ((size_t)V + 1));
    if (!cum) return -1;
    cum[0] = 0;
    for (uint32_t i = 0; i < V; i++) cum[i + 1] = cum[i] + (1ull << 40) / ((uint64_t)i + i0);
    uint64_t a_out, b_out, a_in, b_in;
    cl_affine(V, seed, 0xC1A0011ull, &a_out, &b_out);
    cl_affine(V, seed, 0xC1A0021ull, &a_in, &b_in);
    uint64_t s_out = mix64(seed ^ 0xC1A0001ull), s_in = mix64(seed ^ 0xC1A0002ull), W = cum[V];
#pragma omp parallel for schedule(static)
    for (uint64_t i = 0; i < n; i++) {
        uint64_t h = mix64(i);
        uint64_t x = cl_pick(mix64(s_out ^ h) % W, cum, V), y = cl_pick(mix64(s_in ^ h) % W, cum, V);
        src[i] = (uint32_t)((a_out * x + b_out) % V);
        dst[i] = (uint32_t)((a_in * y + b_in) % V);
    }
    free(cum);
    return 0;
}

static int cmp_u32(const void* a, const void* b)
{
    uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
    return (x > y) - (x < y);
}

/* Edge list -> CSR: drops self-loops, optionally adds reverse edges, sorts
 * by (src, dst), removes duplicates.  Returns E, or -1 on allocation failure.
 * off must hold V+1 entries; dst_out must hold (symmetrise ? 2 : 1) * n entries.
 * Bucketed by source (counts, prefix sums, scatter), each list sorted and
 * deduplicated on its own, then the lists packed: the same CSR as one sort
 * of all (src, dst) pairs, for any thread count. */
int64_t ora_build_csr(uint32_t V, uint64_t n, const uint32_t* src, const uint32_t* dst, int symmetrise,
                      uint32_t* off, uint32_t* dst_out)
{
    uint64_t* pos = (uint64_t*)calloc((size_t)V + 1, sizeof(uint64_t));
    uint32_t* len = (uint32_t*)malloc(sizeof(uint32_t) * ((size_t)V + 1));
    if (!pos || !len) { free(pos); free(len); return -1; }
#pragma omp parallel for schedule(static)
    for (uint64_t i = 0; i < n; i++) {
        if (src[i] == dst[i]) continue;
#pragma omp atomic
        pos[src[i] + 1]++;
        if (symmetrise) {
#pragma omp atomic
            pos[dst[i] + 1]++;
        }
    }
    for (uint32_t v = 0; v < V; v++) pos[v + 1] += pos[v];
    uint64_t* fill = (uint64_t*)malloc(sizeof(uint64_t) * ((size_t)V + 1));
    if (!fill) { free(pos); free(len); return -1; }
    memcpy(fill, pos, sizeof(uint64_t) * ((size_t)V + 1));
#pragma omp parallel for schedule(static)
    for (uint64_t i = 0; i < n; i++) {
        if (src[i] == dst[i]) continue;
        uint64_t k;
#pragma omp atomic capture
        k = fill[src[i]]++;
        dst_out[k] = dst[i];
        if (symmetrise) {
#pragma omp atomic capture
            k = fill[dst[i]]++;
            dst_out[k] = src[i];
        }
    }
    free(fill);
#pragma omp parallel for schedule(dynamic, 4096)
    for (uint32_t v = 0; v < V; v++) {
        uint32_t* l = dst_out + pos[v];
        uint64_t m = pos[v + 1] - pos[v], k = 0;
        if (m > 1) qsort(l, m, sizeof(uint32_t), cmp_u32);
        for (uint64_t i = 0; i < m; i++)
            if (i == 0 || l[i] != l[i - 1]) l[k++] = l[i];
        len[v] = (uint32_t)k;
    }
    /* pack the deduplicated lists in place, front to back */
    uint64_t E = 0;
    for (uint32_t v = 0; v < V; v++) {
        off[v] = (uint32_t)E;
        if (E != pos[v]) memmove(dst_out + E, dst_out + pos[v], sizeof(uint32_t) * len[v]);
        E += len[v];
    }
    off[V] = (uint32_t)E;
    free(pos);
    free(len);
    return (int64_t)E;
}

/* Edge weight in [1, wmax] from a hash of (seed, edge); symmetric edges get
 * the same weight in both directions when sym_key is set. */
void ora_edge_weights(uint32_t V, const uint32_t* off, const uint32_t* dst, uint64_t seed, uint32_t wmax,
                      int sym_key, uint32_t* w)
{
    uint64_t s = mix64(seed ^ 0x77E16ull);
#pragma omp parallel for schedule(dynamic, 4096)
    for (uint32_t u = 0; u < V; u++)
        for (uint32_t e = off[u]; e < off[u + 1]; e++) {
            uint32_t a = u, b = dst[e];
            if (sym_key && b < a) { uint32_t t = a; a = b; b = t; }
            uint64_t h = mix64(s ^ (((uint64_t)a << 32) | b));
            w[e] = 1u + (uint32_t)(h % wmax);
        }
}

/* rows x cols 4-neighbour grid in CSR order (neighbours ascending). */
int64_t ora_grid_csr(uint32_t rows, uint32_t cols, uint32_t* off, uint32_t* dst)
{
    uint64_t e = 0;
    for (uint32_t r = 0; r < rows; r++)
        for (uint32_t c = 0; c < cols; c++) {
            uint32_t v = r * cols + c;
            off[v] = (uint32_t)e;
            if (r > 0) dst[e++] = v - cols;
            if (c > 0) dst[e++] = v - 1;
            if (c + 1 < cols) dst[e++] = v + 1;
            if (r + 1 < rows) dst[e++] = v + cols;
        }
    off[(uint64_t)rows * cols] = (uint32_t)e;
    return (int64_t)e;
}

/* ------------------------------------------------------- BFS-based orders */
/* The reference's MY_BFS_* vertex orders (my_project/CGgraph/Reorder.hpp):
 *  - start list: all vertices by degree, largest first, ties by ascending id
 *    (sortDegree, :251-292): out-degree for MY_BFS_OUT/IN/OUT_IN (16/17/18,
 *    :64-67,99-103,133-137), in-degree for MY_IMAX_BFS_IN (20, :167-171);
 *  - each start vertex not yet visited either joins the zero-out-degree list
 *    (no out-edges) or roots a queue BFS (:304-320);
 *  - a popped vertex sends its unvisited neighbours without out-edges to the
 *    zero list in list order, sorts the rest by child degree, largest first
 *    (out-degree :340-345, in-degree :421-426, in+out :503-508), and queues
 *    those still unvisited in that order (:330-360);
 *  - the order is the BFS visit sequence, then the zero list (:366-372).
 * The reference sorts the children with std::sort; that is an insertion
 * sort, hence stable, for lists of at most 16 entries, and unstable beyond.
 * Here the sort is stable at every length: equal degrees keep list order.
 * Returns the number of vertices with out-edges, or < 0 on error. */
typedef struct { uint64_t deg; uint32_t pos; uint32_t v; } ora_child_t;

static int cmp_child(const void* a, const void* b)
{
    const ora_child_t* x = (const ora_child_t*)a;
    const ora_child_t* y = (const ora_child_t*)b;
    if (x->deg != y->deg) return x->deg > y->deg ? -1 : 1;
    return (x->pos > y->pos) - (x->pos < y->pos);
}

int64_t ora_bfs_order(uint32_t V, const uint32_t* off, const uint32_t* dst, int method, uint32_t* order)
{
    if (method != 16 && method != 17 && method != 18 && method != 20) return -1;
    const uint32_t E = off[V];
    uint64_t* outd = (uint64_t*)calloc((size_t)V + 1, sizeof(uint64_t));
    uint64_t* ind = (uint64_t*)calloc((size_t)V + 1, sizeof(uint64_t));
    ora_child_t* sv = (ora_child_t*)malloc(sizeof(ora_child_t) * ((size_t)V + 1));
    ora_child_t* tmp = (ora_child_t*)malloc(sizeof(ora_child_t) * ((size_t)E + 1));
    uint32_t* zero = (uint32_t*)malloc(sizeof(uint32_t) * ((size_t)V + 1));
    unsigned char* seen = (unsigned char*)calloc((size_t)V + 1, 1);
    if (!outd || !ind || !sv || !tmp || !zero || !seen) {
        free(outd); free(ind); free(sv); free(tmp); free(zero); free(seen);
        return -2;
    }
    for (uint32_t v = 0; v < V; v++) outd[v] = off[v + 1] - off[v];
    for (uint32_t e = 0; e < E; e++) ind[dst[e]]++;
    for (uint32_t v = 0; v < V; v++) {
        sv[v].deg = method == 20 ? ind[v] : outd[v];
        sv[v].pos = v; /* ties by ascending id */
        sv[v].v = v;
    }
    qsort(sv, V, sizeof(ora_child_t), cmp_child);
    uint64_t n = 0, nz = 0; /* order[0, n) is the BFS sequence and the queue */
    for (uint32_t k = 0; k < V; k++) {
        uint32_t s = sv[k].v;
        if (seen[s]) continue;
        seen[s] = 1;
        if (outd[s] == 0) { zero[nz++] = s; continue; }
        uint64_t head = n;
        order[n++] = s;
        while (head < n) {
            uint32_t u = order[head++];
            uint32_t m = 0;
            for (uint32_t e = off[u]; e < off[u + 1]; e++) {
                uint32_t d = dst[e];
                if (outd[d] == 0 && !seen[d]) { seen[d] = 1; zero[nz++] = d; continue; }
                tmp[m].deg = method == 16 ? outd[d] : method == 18 ? outd[d] + ind[d] : ind[d];
                tmp[m].pos = m;
                tmp[m].v = d;
                m++;
            }
            qsort(tmp, m, sizeof(ora_child_t), cmp_child);
            for (uint32_t i = 0; i < m; i++)
                if (!seen[tmp[i].v]) { seen[tmp[i].v] = 1; order[n++] = tmp[i].v; }
        }
    }
    memcpy(order + n, zero, sizeof(uint32_t) * nz);
    free(outd); free(ind); free(sv); free(tmp); free(zero); free(seen);
    return (int64_t)n;
}

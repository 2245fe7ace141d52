/*
 * oracle.c -- CPU restatement of the reference's algorithms for the hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py load this library, as the checker.  The
 * product (hytgraph_b200) never links or calls it.
 *
 * Parity pin: every routine here is checked against the reference's own
 * compiled sources (oracle/_ref, built by oracle/Makefile from
 * src/algorithms/{pagerank,sssp}.cpp) and against the reference's
 * known-answer tests (tests/algorithm_tests.cpp:22-157,
 * tests/cuda_algorithm_tests.cu:23-87, tests/unit_tests.cpp:2058-2204),
 * frozen as fixtures in tests/golden/.
 *
 * Each function names the reference lines it restates.
 */
#include "oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

/* ---- threads ------------------------------------------------------------
 * Row-parallel loops for large graphs.  Each block of rows writes only its
 * own outputs, and every reduction that decides a result (residuals,
 * dangling mass) stays a sequential pass in vertex order, so the results
 * are bit-identical to the single-threaded loops for any thread count.
 * ORACLE_THREADS caps the thread count (default: online cores, <= 64). */
typedef void (*range_fn)(void *ctx, uint64_t begin, uint64_t end);

typedef struct {
    range_fn fn;
    void *ctx;
    uint64_t n, grain;
    uint64_t next; /* next block, taken under the mutex */
    pthread_mutex_t mu;
} par_job;

static void *par_worker(void *arg) {
    par_job *j = (par_job *)arg;
    for (;;) {
        pthread_mutex_lock(&j->mu);
        const uint64_t b = j->next;
        j->next += j->grain;
        pthread_mutex_unlock(&j->mu);
        if (b >= j->n) break;
        j->fn(j->ctx, b, b + j->grain < j->n ? b + j->grain : j->n);
    }
    return NULL;
}

static unsigned oracle_threads(void) {
    const char *e = getenv("ORACLE_THREADS");
    long t = e ? strtol(e, NULL, 10) : sysconf(_SC_NPROCESSORS_ONLN);
    if (t < 1) t = 1;
    if (t > 64) t = 64;
    return (unsigned)t;
}

static void par_for(uint64_t n, uint64_t grain, range_fn fn, void *ctx) {
    unsigned nt = oracle_threads();
    if (grain == 0) grain = 1;
    if (n <= grain || nt == 1) {
        if (n) fn(ctx, 0, n);
        return;
    }
    if ((uint64_t)nt > (n + grain - 1) / grain) nt = (unsigned)((n + grain - 1) / grain);
    par_job j = {fn, ctx, n, grain, 0, PTHREAD_MUTEX_INITIALIZER};
    pthread_t th[64];
    unsigned started = 0;
    for (unsigned t = 1; t < nt; ++t)
        if (pthread_create(&th[started], NULL, par_worker, &j) == 0) ++started;
    par_worker(&j);
    for (unsigned t = 0; t < started; ++t) pthread_join(th[t], NULL);
    pthread_mutex_destroy(&j.mu);
}

/* Incoming CSR (CSC) with sources in ascending order inside each row,
 * built with the same counting pass as src/algorithms/pagerank.cpp:19-60
 * (and sssp.cpp:21-80, which also carries the weights). */
static int build_incoming(uint64_t V, uint64_t E, const uint64_t *off, const uint32_t *cols, const float *w_in,
                          uint64_t **in_off_out, uint32_t **in_src_out, float **in_w_out) {
    uint64_t *in_off = (uint64_t *)calloc(V + 1, sizeof(uint64_t));
    uint32_t *in_src = (uint32_t *)malloc((E ? E : 1) * sizeof(uint32_t));
    float *in_w = in_w_out ? (float *)malloc((E ? E : 1) * sizeof(float)) : NULL;
    uint64_t *cursor = (uint64_t *)malloc((V + 1) * sizeof(uint64_t));
    if (!in_off || !in_src || !cursor || (in_w_out && !in_w)) {
        free(in_off); free(in_src); free(in_w); free(cursor);
        return ORACLE_E_NOMEM;
    }
    for (uint64_t u = 0; u < V; ++u)
        for (uint64_t e = off[u]; e < off[u + 1]; ++e) ++in_off[cols[e] + 1];
    for (uint64_t v = 1; v <= V; ++v) in_off[v] += in_off[v - 1];
    memcpy(cursor, in_off, (V + 1) * sizeof(uint64_t));
    for (uint64_t u = 0; u < V; ++u)
        for (uint64_t e = off[u]; e < off[u + 1]; ++e) {
            const uint64_t pos = cursor[cols[e]]++;
            in_src[pos] = (uint32_t)u;
            if (in_w) in_w[pos] = w_in ? w_in[e] : 1.0f;
        }
    free(cursor);
    *in_off_out = in_off;
    *in_src_out = in_src;
    if (in_w_out) *in_w_out = in_w;
    return ORACLE_OK;
}

/* src/algorithms/pagerank.cpp:62-85 */
static int pr_validate(uint64_t V, float damping, float tol, uint64_t max_iter) {
    if (V == 0) return ORACLE_E_INVALID;
    if (!(damping >= 0.0f && damping < 1.0f)) return ORACLE_E_INVALID;
    if (!(tol > 0.0f) || !isfinite(tol)) return ORACLE_E_INVALID;
    if (max_iter == 0) return ORACLE_E_INVALID;
    return ORACLE_OK;
}

/* Row sums of one FP32 step (pagerank.cpp:126-147): each row adds
 * x_u / deg_u over its in-edges in edge order, in float. */
typedef struct {
    const uint64_t *off, *in_off;
    const uint32_t *in_src;
    const float *cur;
    float *nxt;
    float base, dshare, damping;
} pr32_rows;

static void pr32_rows_fn(void *p, uint64_t b, uint64_t e) {
    const pr32_rows *c = (const pr32_rows *)p;
    for (uint64_t v = b; v < e; ++v) {
        float sum = 0.0f;
        for (uint64_t q = c->in_off[v]; q < c->in_off[v + 1]; ++q) {
            const uint32_t u = c->in_src[q];
            const uint64_t deg = c->off[u + 1] - c->off[u];
            if (deg != 0) sum += c->cur[u] / (float)deg;
        }
        c->nxt[v] = c->base + c->dshare + c->damping * sum;
    }
}

/* FP32 restatement of pagerank_cpu, src/algorithms/pagerank.cpp:89-163:
 * same operation order, so it reproduces the reference bit for bit (the
 * row sums run in parallel; the residual and dangling sums stay sequential
 * passes in vertex order, as in the reference). */
int oracle_pagerank_f32(uint64_t V, uint64_t E, const uint64_t *off, const uint32_t *cols, float damping,
                        float tol, uint64_t max_iter, float *ranks, uint64_t *iterations, float *residual_out,
                        int *converged) {
    int rc = pr_validate(V, damping, tol, max_iter);
    if (rc) return rc;
    uint64_t *in_off;
    uint32_t *in_src;
    rc = build_incoming(V, E, off, cols, NULL, &in_off, &in_src, NULL);
    if (rc) return rc;
    const float n = (float)V;
    const float base = (1.0f - damping) / n;
    float *cur = (float *)malloc(V * sizeof(float)), *nxt = (float *)malloc(V * sizeof(float));
    if (!cur || !nxt) { free(cur); free(nxt); free(in_off); free(in_src); return ORACLE_E_NOMEM; }
    for (uint64_t v = 0; v < V; ++v) cur[v] = 1.0f / n;
    *iterations = 0; *residual_out = 0.0f; *converged = 0;
    memcpy(ranks, cur, V * sizeof(float));
    for (uint64_t it = 0; it < max_iter; ++it) {
        float dangling = 0.0f;
        for (uint64_t u = 0; u < V; ++u)
            if (off[u + 1] == off[u]) dangling += cur[u];
        const float dshare = damping * dangling / n;
        pr32_rows ctx = {off, in_off, in_src, cur, nxt, base, dshare, damping};
        par_for(V, 1u << 15, pr32_rows_fn, &ctx);
        float residual = 0.0f;
        for (uint64_t v = 0; v < V; ++v) residual += fabsf(nxt[v] - cur[v]);
        float *t = cur; cur = nxt; nxt = t;
        *iterations = it + 1;
        *residual_out = residual;
        memcpy(ranks, cur, V * sizeof(float));
        if (residual <= tol) { *converged = 1; break; }
    }
    free(cur); free(nxt); free(in_off); free(in_src);
    return ORACLE_OK;
}

/* Row sums of one FP64 step: x'[v] = add + d * sum_{u->v} contrib[u];
 * personalized: x'[v] = d * sum + (v == source ? restart_mass : 0). */
typedef struct {
    const uint64_t *in_off;
    const uint32_t *in_src;
    const double *contrib;
    double *nxt;
    double add, d;
    int personalized;
    uint32_t source;
    double restart_mass;
} pr64_rows;

static void pr64_rows_fn(void *p, uint64_t b, uint64_t e) {
    const pr64_rows *c = (const pr64_rows *)p;
    for (uint64_t v = b; v < e; ++v) {
        double sum = 0.0;
        for (uint64_t q = c->in_off[v]; q < c->in_off[v + 1]; ++q) sum += c->contrib[c->in_src[q]];
        c->nxt[v] = c->personalized ? c->d * sum + (v == c->source ? c->restart_mass : 0.0) : c->add + c->d * sum;
    }
}

/* FP64 restatement of the same iteration (pagerank.cpp:89-163 in double):
 * x0 = 1/n; x' = (1-d)/n + d*dangling/n + d*sum x_u/deg_u; stop when the L1
 * change <= tol.  This is the accuracy reference for the FP32 solvers.
 * The _csc form takes the incoming CSR (sources ascending within each row,
 * as build_incoming makes it) instead of building it. */
int oracle_pagerank_f64_csc(uint64_t V, const uint64_t *off, const uint64_t *in_off, const uint32_t *in_src,
                            double damping, double tol, uint64_t max_iter, double *ranks, uint64_t *iterations,
                            double *residual_out, int *converged) {
    if (V == 0 || !(damping >= 0.0 && damping < 1.0) || !(tol > 0.0) || max_iter == 0) return ORACLE_E_INVALID;
    const double n = (double)V, base = (1.0 - damping) / n;
    double *cur = (double *)malloc(V * sizeof(double)), *nxt = (double *)malloc(V * sizeof(double));
    double *contrib = (double *)malloc(V * sizeof(double));
    if (!cur || !nxt || !contrib) { free(cur); free(nxt); free(contrib); return ORACLE_E_NOMEM; }
    for (uint64_t v = 0; v < V; ++v) cur[v] = 1.0 / n;
    *iterations = 0; *residual_out = 0.0; *converged = 0;
    for (uint64_t it = 0; it < max_iter; ++it) {
        double dangling = 0.0;
        for (uint64_t u = 0; u < V; ++u) {
            const uint64_t deg = off[u + 1] - off[u];
            if (deg == 0) dangling += cur[u];
            contrib[u] = deg ? cur[u] / (double)deg : 0.0;
        }
        const double dshare = damping * dangling / n;
        pr64_rows ctx = {in_off, in_src, contrib, nxt, base + dshare, damping, 0, 0, 0.0};
        par_for(V, 1u << 15, pr64_rows_fn, &ctx);
        double residual = 0.0;
        for (uint64_t v = 0; v < V; ++v) residual += fabs(nxt[v] - cur[v]);
        double *t = cur; cur = nxt; nxt = t;
        *iterations = it + 1;
        *residual_out = residual;
        if (residual <= tol) { *converged = 1; break; }
    }
    memcpy(ranks, cur, V * sizeof(double));
    free(cur); free(nxt); free(contrib);
    return ORACLE_OK;
}

int oracle_pagerank_f64(uint64_t V, uint64_t E, const uint64_t *off, const uint32_t *cols, double damping,
                        double tol, uint64_t max_iter, double *ranks, uint64_t *iterations, double *residual_out,
                        int *converged) {
    if (V == 0 || !(damping >= 0.0 && damping < 1.0) || !(tol > 0.0) || max_iter == 0) return ORACLE_E_INVALID;
    uint64_t *in_off;
    uint32_t *in_src;
    int rc = build_incoming(V, E, off, cols, NULL, &in_off, &in_src, NULL);
    if (rc) return rc;
    rc = oracle_pagerank_f64_csc(V, off, in_off, in_src, damping, tol, max_iter, ranks, iterations, residual_out,
                                 converged);
    free(in_off); free(in_src);
    return rc;
}

/* Personalized PageRank in FP64 (no reference counterpart; defined by this
 * project on the structure of pagerank.cpp:89-163):
 *   x0 = e_s;  x'[v] = d * sum_{u->v} x_u/deg_u + [v == s] * ((1-d) + d*dangling)
 * with d = 1 - restart and dangling = sum of x over out-degree-0 vertices
 * (dangling mass returns to the source); stop when the L1 change <= tol. */
int oracle_ppr_f64(uint64_t V, uint64_t E, const uint64_t *off, const uint32_t *cols, uint32_t source,
                   double restart, double tol, uint64_t max_iter, double *ranks, uint64_t *iterations,
                   double *residual_out, int *converged) {
    if (V == 0 || source >= V || !(restart > 0.0 && restart <= 1.0) || !(tol > 0.0) || max_iter == 0)
        return ORACLE_E_INVALID;
    uint64_t *in_off;
    uint32_t *in_src;
    int rc = build_incoming(V, E, off, cols, NULL, &in_off, &in_src, NULL);
    if (rc) return rc;
    const double d = 1.0 - restart;
    double *cur = (double *)calloc(V, sizeof(double)), *nxt = (double *)malloc(V * sizeof(double));
    double *contrib = (double *)malloc(V * sizeof(double));
    if (!cur || !nxt || !contrib) { free(cur); free(nxt); free(contrib); free(in_off); free(in_src); return ORACLE_E_NOMEM; }
    cur[source] = 1.0;
    *iterations = 0; *residual_out = 0.0; *converged = 0;
    for (uint64_t it = 0; it < max_iter; ++it) {
        double dangling = 0.0;
        for (uint64_t u = 0; u < V; ++u) {
            const uint64_t deg = off[u + 1] - off[u];
            if (deg == 0) dangling += cur[u];
            contrib[u] = deg ? cur[u] / (double)deg : 0.0;
        }
        pr64_rows ctx = {in_off, in_src, contrib, nxt, 0.0, d, 1, source, (1.0 - d) + d * dangling};
        par_for(V, 1u << 15, pr64_rows_fn, &ctx);
        double residual = 0.0;
        for (uint64_t v = 0; v < V; ++v) residual += fabs(nxt[v] - cur[v]);
        double *t = cur; cur = nxt; nxt = t;
        *iterations = it + 1;
        *residual_out = residual;
        if (residual <= tol) { *converged = 1; break; }
    }
    memcpy(ranks, cur, V * sizeof(double));
    free(cur); free(nxt); free(contrib); free(in_off); free(in_src);
    return ORACLE_OK;
}

/* One synchronous round over rows [b, e) (sssp.cpp:126-170): each row
 * takes the minimum of its label and cur[u] + w over in-edges whose source
 * was active in the previous round. */
typedef struct {
    const uint64_t *in_off;
    const uint32_t *in_src;
    const float *in_w, *cur;
    float *nxt;
    const unsigned char *active;
    unsigned char *next_active;
    int changed; /* set to 1 (atomically) by any block whose rows improved */
} sssp_rows;

static void sssp_rows_fn(void *p, uint64_t b, uint64_t e) {
    sssp_rows *c = (sssp_rows *)p;
    int changed = 0;
    for (uint64_t v = b; v < e; ++v) {
        float best = c->cur[v];
        for (uint64_t q = c->in_off[v]; q < c->in_off[v + 1]; ++q) {
            const uint32_t u = c->in_src[q];
            if (!c->active[u] || !isfinite(c->cur[u])) continue;
            const float cand = c->cur[u] + c->in_w[q];
            if (cand < best) best = cand;
        }
        c->nxt[v] = best;
        c->next_active[v] = best < c->cur[v];
        changed |= best < c->cur[v];
    }
    if (changed) __atomic_store_n(&c->changed, 1, __ATOMIC_RELAXED);
}

/* FP32 restatement of sssp_cpu, src/algorithms/sssp.cpp:109-234: synchronous
 * Bellman-Ford pulling over in-edges from sources active in the previous
 * round; weights NULL means 1.0 per edge.  max_iter 0 selects V. */
int oracle_sssp(uint64_t V, uint64_t E, const uint64_t *off, const uint32_t *cols, const float *weights,
                uint32_t source, uint64_t max_iter, float *dist, uint64_t *iterations, int *converged) {
    if (V == 0 || source >= V) return ORACLE_E_INVALID;
    if (weights)
        for (uint64_t e = 0; e < E; ++e)
            if (!isfinite(weights[e]) || weights[e] < 0.0f) return ORACLE_E_INVALID;
    uint64_t *in_off;
    uint32_t *in_src;
    float *in_w;
    int rc = build_incoming(V, E, off, cols, weights, &in_off, &in_src, &in_w);
    if (rc) return rc;
    float *cur = (float *)malloc(V * sizeof(float)), *nxt = (float *)malloc(V * sizeof(float));
    unsigned char *active = (unsigned char *)calloc(V, 1), *next_active = (unsigned char *)calloc(V, 1);
    if (!cur || !nxt || !active || !next_active) {
        free(cur); free(nxt); free(active); free(next_active); free(in_off); free(in_src); free(in_w);
        return ORACLE_E_NOMEM;
    }
    for (uint64_t v = 0; v < V; ++v) cur[v] = INFINITY;
    cur[source] = 0.0f;
    active[source] = 1;
    if (max_iter == 0) max_iter = V;
    *iterations = 0; *converged = 0;
    for (uint64_t it = 0; it < max_iter; ++it) {
        sssp_rows ctx = {in_off, in_src, in_w, cur, nxt, active, next_active, 0};
        par_for(V, 1u << 15, sssp_rows_fn, &ctx);
        const int changed = ctx.changed != 0;
        float *t = cur; cur = nxt; nxt = t;
        unsigned char *ta = active; active = next_active; next_active = ta;
        *iterations = it + 1;
        if (!changed) { *converged = 1; break; }
    }
    memcpy(dist, cur, V * sizeof(float));
    free(cur); free(nxt); free(active); free(next_active); free(in_off); free(in_src); free(in_w);
    return ORACLE_OK;
}

/* Independent cross-check: Dijkstra with exact 64-bit integer distances on
 * uint32 weights (NULL = unit weights); UINT64_MAX marks unreachable.  An
 * indexed binary heap with decrease-key holds at most V entries (16 B + a
 * 4 B position each), so large graphs need O(V) extra memory, not O(E). */
typedef struct { uint64_t d; uint32_t v; } heap_item;

static void heap_place(heap_item *h, uint32_t *pos, uint64_t i, heap_item x) {
    h[i] = x;
    pos[x.v] = (uint32_t)i;
}

static void heap_up(heap_item *h, uint32_t *pos, uint64_t i, heap_item x) {
    while (i > 0) {
        const uint64_t p = (i - 1) / 2;
        if (h[p].d <= x.d) break;
        heap_place(h, pos, i, h[p]);
        i = p;
    }
    heap_place(h, pos, i, x);
}

static heap_item heap_pop(heap_item *h, uint32_t *pos, uint64_t *n) {
    const heap_item top = h[0], x = h[--(*n)];
    pos[top.v] = UINT32_MAX;
    if (*n == 0) return top;
    uint64_t i = 0;
    for (;;) {
        uint64_t c = 2 * i + 1;
        if (c >= *n) break;
        if (c + 1 < *n && h[c + 1].d < h[c].d) ++c;
        if (h[c].d >= x.d) break;
        heap_place(h, pos, i, h[c]);
        i = c;
    }
    heap_place(h, pos, i, x);
    return top;
}

int oracle_dijkstra_u32(uint64_t V, uint64_t E, const uint64_t *off, const uint32_t *cols, const uint32_t *weights,
                        uint32_t source, uint64_t *dist) {
    (void)E;
    if (V == 0 || source >= V || V >= UINT32_MAX) return ORACLE_E_INVALID;
    heap_item *h = (heap_item *)malloc(V * sizeof(heap_item));
    uint32_t *pos = (uint32_t *)malloc(V * sizeof(uint32_t));
    if (!h || !pos) { free(h); free(pos); return ORACLE_E_NOMEM; }
    for (uint64_t v = 0; v < V; ++v) { dist[v] = UINT64_MAX; pos[v] = UINT32_MAX; }
    uint64_t n = 1;
    dist[source] = 0;
    heap_place(h, pos, 0, (heap_item){0, source});
    while (n) {
        const heap_item t = heap_pop(h, pos, &n);
        for (uint64_t e = off[t.v]; e < off[t.v + 1]; ++e) {
            const uint32_t u = cols[e];
            const uint64_t nd = t.d + (weights ? weights[e] : 1u);
            if (nd < dist[u]) {
                dist[u] = nd;
                const uint64_t i = pos[u] == UINT32_MAX ? n++ : pos[u];
                heap_up(h, pos, i, (heap_item){nd, u});
            }
        }
    }
    free(h);
    free(pos);
    return ORACLE_OK;
}

/* ---- R-MAT generator and source picker ------------------------------------
 * The seeded synthetic inputs (the reference ships no generator and no
 * datasets), restated from their definition so that CPU-only consumers
 * (the reference's CPU baseline) build the same graph bytes without the
 * product library:
 *   draw i (0 <= i < edge_factor * 2^scale) descends `scale` levels; level
 *   l takes the 32-bit uniform u = half (l & 1) of
 *   splitmix64(seed + golden * (16 i + l / 2)) and picks quadrant
 *   (0,0) / (0,1) / (1,0) / (1,1) by u < a / a+b / a+b+c (thresholds scaled
 *   to 2^32, saturating at 2^32 - 1); bit (scale - 1 - l) of the source
 *   takes the row half, of the destination the column half.  Self-loops and
 *   duplicate (u, v) are dropped, edges sorted by (u, v); weight of (u, v) =
 *   wmin + splitmix64(((u << 32) | v) ^ wseed) % (wmax - wmin + 1), wseed =
 *   splitmix64(seed ^ 0x5EEDF00DCAFEBABE); wmin = wmax = 0 means unweighted.
 *   Sources: the j-th candidate (j = 1, 2, ...) is splitmix64(seed + golden
 *   * j) % V; vertices without out-edges are skipped, and repeats while
 *   distinct vertices with out-edges remain. */
static const uint64_t kGolden = 0x9E3779B97F4A7C15ull;

static uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static uint32_t rmat_threshold(double x) {
    const double v = x * 4294967296.0;
    return v >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)v;
}

typedef struct {
    uint64_t seed, n;
    uint32_t scale, ta, tab, tabc;
    uint64_t *keys; /* (u << scale) | v, or UINT64_MAX for a self-loop */
} rmat_job;

static void rmat_draw_fn(void *p, uint64_t b, uint64_t e) {
    const rmat_job *j = (const rmat_job *)p;
    for (uint64_t i = b; i < e; ++i) {
        uint32_t src = 0, dst = 0;
        uint64_t word = 0;
        for (uint32_t l = 0; l < j->scale; ++l) {
            if ((l & 1u) == 0) word = mix64(j->seed + kGolden * (16ull * i + (l >> 1)));
            const uint32_t r = (l & 1u) ? (uint32_t)(word >> 32) : (uint32_t)word;
            const uint32_t bit = 1u << (j->scale - 1 - l);
            if (r >= j->tabc) { src |= bit; dst |= bit; }
            else if (r >= j->tab) src |= bit;
            else if (r >= j->ta) dst |= bit;
        }
        j->keys[i] = (src == dst) ? UINT64_MAX : (((uint64_t)src << j->scale) | dst);
    }
}

/* LSD radix sort of n keys on their low `bits` bits, 11 bits a pass,
 * threads over contiguous slices (stable, so equal keys keep their order). */
typedef struct {
    const uint64_t *in;
    uint64_t *out;
    uint64_t n, slice;
    unsigned shift, nslices;
    uint64_t *hist; /* [nslices][2048] counts, then start offsets */
} radix_job;

static void radix_count_fn(void *p, uint64_t b, uint64_t e) {
    radix_job *j = (radix_job *)p;
    for (uint64_t t = b; t < e; ++t) {
        uint64_t *h = j->hist + t * 2048;
        memset(h, 0, 2048 * sizeof(uint64_t));
        const uint64_t lo = t * j->slice, hi = lo + j->slice < j->n ? lo + j->slice : j->n;
        for (uint64_t i = lo; i < hi; ++i) ++h[(j->in[i] >> j->shift) & 2047u];
    }
}

static void radix_scatter_fn(void *p, uint64_t b, uint64_t e) {
    radix_job *j = (radix_job *)p;
    for (uint64_t t = b; t < e; ++t) {
        uint64_t *h = j->hist + t * 2048;
        const uint64_t lo = t * j->slice, hi = lo + j->slice < j->n ? lo + j->slice : j->n;
        for (uint64_t i = lo; i < hi; ++i) j->out[h[(j->in[i] >> j->shift) & 2047u]++] = j->in[i];
    }
}

static int radix_sort_u64(uint64_t *keys, uint64_t n, unsigned bits) {
    if (n < 2) return ORACLE_OK;
    uint64_t *tmp = (uint64_t *)malloc(n * sizeof(uint64_t));
    const unsigned nslices = 64;
    uint64_t *hist = (uint64_t *)malloc((uint64_t)nslices * 2048 * sizeof(uint64_t));
    if (!tmp || !hist) { free(tmp); free(hist); return ORACLE_E_NOMEM; }
    radix_job j = {keys, tmp, n, (n + nslices - 1) / nslices, 0, nslices, hist};
    for (unsigned shift = 0; shift < bits; shift += 11) {
        j.shift = shift;
        par_for(nslices, 1, radix_count_fn, &j);
        uint64_t run = 0;  /* digit-major, slice-minor starts keep the sort stable */
        for (unsigned d = 0; d < 2048; ++d)
            for (unsigned t = 0; t < nslices; ++t) {
                const uint64_t c = hist[(uint64_t)t * 2048 + d];
                hist[(uint64_t)t * 2048 + d] = run;
                run += c;
            }
        par_for(nslices, 1, radix_scatter_fn, &j);
        uint64_t *done = j.out;
        j.out = (uint64_t *)j.in;
        j.in = done;
    }
    if (j.in != keys) memcpy(keys, j.in, n * sizeof(uint64_t));
    free(tmp);
    free(hist);
    return ORACLE_OK;
}

int oracle_rmat(uint32_t scale, uint32_t edge_factor, uint64_t seed, double a, double b, double c, uint32_t wmin,
                uint32_t wmax, uint64_t **off_out, uint32_t **cols_out, uint32_t **w_out, uint64_t *E_out) {
    *off_out = NULL; *cols_out = NULL; *w_out = NULL; *E_out = 0;
    if (scale < 1 || scale > 31 || edge_factor == 0 || wmax < wmin) return ORACLE_E_INVALID;
    if (!(a >= 0 && b >= 0 && c >= 0 && 1.0 - a - b - c >= -1e-12)) return ORACLE_E_INVALID;
    const uint64_t V = 1ull << scale, n = (uint64_t)edge_factor * V;
    uint64_t *keys = (uint64_t *)malloc(n * sizeof(uint64_t));
    if (!keys) return ORACLE_E_NOMEM;
    rmat_job j = {seed, n, scale, rmat_threshold(a), rmat_threshold(a + b), rmat_threshold(a + b + c), keys};
    par_for(n, 1u << 16, rmat_draw_fn, &j);
    uint64_t m = 0;  /* drop self-loops */
    for (uint64_t i = 0; i < n; ++i)
        if (keys[i] != UINT64_MAX) keys[m++] = keys[i];
    int rc = radix_sort_u64(keys, m, 2 * scale);
    if (rc) { free(keys); return rc; }
    uint64_t E = 0;  /* drop duplicates */
    for (uint64_t i = 0; i < m; ++i)
        if (i == 0 || keys[i] != keys[i - 1]) keys[E++] = keys[i];
    uint64_t *off = (uint64_t *)malloc((V + 1) * sizeof(uint64_t));
    uint32_t *cols = (uint32_t *)malloc((E ? E : 1) * sizeof(uint32_t));
    const int weighted = !(wmin == 0 && wmax == 0);
    uint32_t *w = weighted ? (uint32_t *)malloc((E ? E : 1) * sizeof(uint32_t)) : NULL;
    if (!off || !cols || (weighted && !w)) { free(keys); free(off); free(cols); free(w); return ORACLE_E_NOMEM; }
    const uint64_t wseed = mix64(seed ^ 0x5EEDF00DCAFEBABEull);
    const uint32_t span = wmax - wmin + 1u;
    const uint64_t vmask = V - 1;
    uint64_t e = 0;
    for (uint64_t v = 0; v < V; ++v) {
        off[v] = e;
        while (e < E && (keys[e] >> scale) == v) {
            const uint32_t dst = (uint32_t)(keys[e] & vmask);
            cols[e] = dst;
            if (w) w[e] = wmin + (uint32_t)(mix64(((v << 32) | dst) ^ wseed) % (span ? span : 1u));
            ++e;
        }
    }
    off[V] = E;
    free(keys);
    *off_out = off; *cols_out = cols; *w_out = w; *E_out = E;
    return ORACLE_OK;
}

void oracle_free(void *p) { free(p); }

int oracle_pick_sources(const uint64_t *off, uint64_t V, uint64_t seed, uint32_t count, uint32_t *out) {
    if (V == 0) return ORACLE_E_INVALID;
    uint64_t with_edges = 0;
    for (uint64_t v = 0; v < V; ++v) with_edges += off[v + 1] > off[v];
    if (with_edges == 0 && count) return ORACLE_E_INVALID;
    const uint64_t want_unique = count < with_edges ? count : with_edges;
    uint64_t chosen = 0, j = 0;
    while (chosen < count) {
        const uint64_t v = mix64(seed + kGolden * (++j)) % V;
        if (off[v + 1] == off[v]) continue;
        int seen = 0;
        if (chosen < want_unique)
            for (uint64_t k = 0; k < chosen; ++k) seen |= out[k] == (uint32_t)v;
        if (seen) continue;
        out[chosen++] = (uint32_t)v;
    }
    return ORACLE_OK;
}

/* HyTM per-partition metrics and costs: restates
 * src/transfer/hytm_cost_model.cpp:330-452 (metrics), :454-484 (RTT_zc),
 * :511-615 (formulas 1-3) and :649-715 (strict selector).
 * Options: d1 = dest bytes, d2 = index bytes, m = payload, mr = requests per
 * TLP, align = alignment bytes. */
void oracle_hytm_partition(const uint64_t *off, const unsigned char *active, uint32_t vbegin, uint32_t vend,
                           const oracle_hytm_options *o, oracle_hytm_costs *c) {
    memset(c, 0, sizeof(*c));
    c->total_edges = off[vend] - off[vbegin];
    c->filter_bytes = c->total_edges * o->d1;
    for (uint32_t v = vbegin; v < vend; ++v) {
        if (!active[v]) continue;
        const uint64_t deg = off[v + 1] - off[v];
        c->active_vertices += 1;
        c->active_edges += deg;
        if (deg == 0) continue;
        c->zc_requests += (deg * o->d1 + o->m - 1) / o->m;
        if ((off[v] * o->d1) % o->align != 0) c->zc_alignment += 1;
    }
    c->compaction_bytes = c->active_edges * o->d1 + c->active_vertices * o->d2;
    const uint64_t tlp_bytes = o->m * o->mr;
    const uint64_t zc_total = c->zc_requests + c->zc_alignment;
    c->filter_cost = (double)((c->filter_bytes + tlp_bytes - 1) / tlp_bytes) * o->rtt;
    c->compaction_cost = (double)((c->compaction_bytes + tlp_bytes - 1) / tlp_bytes) * o->rtt +
                         (double)c->compaction_bytes / o->cpu_throughput;
    c->zc_rtt = c->total_edges == 0 ? o->gamma * o->rtt
                                    : o->gamma * o->rtt +
                                          (1.0 - o->gamma) * ((double)c->active_edges / (double)c->total_edges) * o->rtt;
    c->zero_copy_cost = (double)((zc_total + o->mr - 1) / o->mr) * c->zc_rtt;
    c->engine = oracle_select_engine(c->filter_cost, c->compaction_cost, c->zero_copy_cost, o->alpha, o->beta);
}

int oracle_select_engine(double f, double c, double z, double alpha, double beta) {
    if (c < alpha * f && c < beta * z) return ORACLE_ENGINE_COMPACTION;
    if (f < z) return ORACLE_ENGINE_FILTER;
    return ORACLE_ENGINE_ZERO_COPY;
}

/* Task combining, src/scheduling/task_combiner.cpp:67-248: consecutive
 * Filter partitions in groups of <= k, then one Compaction task and one
 * Zero-Copy task, all ordered by first partition.  Writes, per partition,
 * the index of its task; returns the number of tasks. */
uint64_t oracle_task_combine(const int *engines, uint64_t n, uint64_t k, uint64_t *task_of_partition,
                             int *task_engine, uint64_t *task_first) {
    /* first pass: task ids in creation order */
    uint64_t ntask = 0, comp_first = UINT64_MAX, zc_first = UINT64_MAX;
    uint64_t *tmp_first = (uint64_t *)malloc((n + 2) * sizeof(uint64_t));
    int *tmp_engine = (int *)malloc((n + 2) * sizeof(int));
    uint64_t *tmp_task = (uint64_t *)malloc((n ? n : 1) * sizeof(uint64_t));
    for (uint64_t i = 0; i < n;) {
        if (engines[i] == ORACLE_ENGINE_FILTER) {
            uint64_t g = 0;
            tmp_first[ntask] = i;
            tmp_engine[ntask] = ORACLE_ENGINE_FILTER;
            while (i < n && engines[i] == ORACLE_ENGINE_FILTER && g < k) { tmp_task[i++] = ntask; ++g; }
            ++ntask;
        } else {
            if (engines[i] == ORACLE_ENGINE_COMPACTION && comp_first == UINT64_MAX) comp_first = i;
            if (engines[i] == ORACLE_ENGINE_ZERO_COPY && zc_first == UINT64_MAX) zc_first = i;
            tmp_task[i] = UINT64_MAX;
            ++i;
        }
    }
    const uint64_t comp_task = comp_first != UINT64_MAX ? ntask++ : UINT64_MAX;
    if (comp_task != UINT64_MAX) { tmp_first[comp_task] = comp_first; tmp_engine[comp_task] = ORACLE_ENGINE_COMPACTION; }
    const uint64_t zc_task = zc_first != UINT64_MAX ? ntask++ : UINT64_MAX;
    if (zc_task != UINT64_MAX) { tmp_first[zc_task] = zc_first; tmp_engine[zc_task] = ORACLE_ENGINE_ZERO_COPY; }
    for (uint64_t i = 0; i < n; ++i)
        if (tmp_task[i] == UINT64_MAX) tmp_task[i] = engines[i] == ORACLE_ENGINE_COMPACTION ? comp_task : zc_task;
    /* rank tasks by first partition (all distinct) */
    uint64_t *rank = (uint64_t *)malloc((ntask ? ntask : 1) * sizeof(uint64_t));
    for (uint64_t t = 0; t < ntask; ++t) {
        uint64_t r = 0;
        for (uint64_t s = 0; s < ntask; ++s) r += tmp_first[s] < tmp_first[t];
        rank[t] = r;
        task_engine[r] = tmp_engine[t];
        task_first[r] = tmp_first[t];
    }
    for (uint64_t i = 0; i < n; ++i) task_of_partition[i] = rank[tmp_task[i]];
    free(rank); free(tmp_first); free(tmp_engine); free(tmp_task);
    return ntask;
}

/* Hub sort, restating src/scheduling/hub_sort.cpp:28-183:
 *   in-degree from the destination array, H(v) = Do*Di / (Do_max*Di_max)
 *   in long double rounded to double (0 for an edgeless graph), hub count
 *   round(V*f) when within 1e-12 of an integer else ceil(V*f), capped at V;
 *   ranking by higher score, then lower id; hubs first, then every other
 *   vertex in id order.  Returns 0, or ORACLE_E_INVALID for a fraction
 *   outside [0, 1] (HubSorter's constructor, hub_sort.cpp:10-20). */
static const double *g_hub_scores;
static int hub_rank_cmp(const void *pa, const void *pb) {
    const uint32_t a = *(const uint32_t *)pa, b = *(const uint32_t *)pb;
    const double sa = g_hub_scores[a], sb = g_hub_scores[b];
    if (sa != sb) return sa > sb ? -1 : 1;
    return a < b ? -1 : (a > b);
}

int oracle_hub_sort(uint64_t V, uint64_t E, const uint64_t *off, const uint32_t *cols, double fraction,
                    uint32_t *order, double *scores, uint64_t *hub_count) {
    if (!isfinite(fraction) || fraction < 0.0 || fraction > 1.0) return ORACLE_E_INVALID;
    *hub_count = 0;
    if (V == 0) return 0;
    uint64_t *indeg = (uint64_t *)calloc(V, sizeof(uint64_t));
    uint32_t *ranked = (uint32_t *)malloc(V * sizeof(uint32_t));
    unsigned char *hub = (unsigned char *)calloc(V, 1);
    if (!indeg || !ranked || !hub) { free(indeg); free(ranked); free(hub); return ORACLE_E_NOMEM; }
    for (uint64_t e = 0; e < E; ++e) ++indeg[cols[e]];
    uint64_t max_out = 0, max_in = 0;
    for (uint64_t v = 0; v < V; ++v) {
        const uint64_t od = off[v + 1] - off[v];
        if (od > max_out) max_out = od;
        if (indeg[v] > max_in) max_in = indeg[v];
    }
    const long double den = (long double)max_out * (long double)max_in;
    for (uint64_t v = 0; v < V; ++v) {
        const long double num = (long double)(off[v + 1] - off[v]) * (long double)indeg[v];
        scores[v] = den > 0.0L ? (double)(num / den) : 0.0;
    }
    const long double req = (long double)V * (long double)fraction;
    const long double rnd = roundl(req);
    const long double pick = fabsl(req - rnd) < 1e-12L ? rnd : ceill(req);
    uint64_t hubs = (uint64_t)pick;
    if (hubs > V) hubs = V;
    for (uint64_t v = 0; v < V; ++v) ranked[v] = (uint32_t)v;
    g_hub_scores = scores;
    qsort(ranked, V, sizeof(uint32_t), hub_rank_cmp); /* total order: stability not needed */
    uint64_t n = 0;
    for (uint64_t r = 0; r < hubs; ++r) { hub[ranked[r]] = 1; order[n++] = ranked[r]; }
    for (uint64_t v = 0; v < V; ++v)
        if (!hub[v]) order[n++] = (uint32_t)v;
    *hub_count = hubs;
    free(indeg); free(ranked); free(hub);
    return 0;
}

/* Vertex reordering, restating src/graph/csr_graph.cpp:171-283:
 * order[new] = old must be a permutation (ORACLE_E_INVALID otherwise:
 * out-of-range id, or duplicate id); row `new` takes old row `old`'s edges
 * in order, destinations renamed through the inverse permutation, weights
 * (any 4-byte type; w may be NULL) carried along. */
int oracle_reorder(uint64_t V, uint64_t E, const uint64_t *off, const uint32_t *cols, const uint32_t *w,
                   const uint32_t *order, uint64_t *off_out, uint32_t *cols_out, uint32_t *w_out) {
    uint32_t *inv = (uint32_t *)malloc((V ? V : 1) * sizeof(uint32_t));
    unsigned char *seen = (unsigned char *)calloc(V ? V : 1, 1);
    if (!inv || !seen) { free(inv); free(seen); return ORACLE_E_NOMEM; }
    for (uint64_t nv = 0; nv < V; ++nv) {
        const uint32_t old = order[nv];
        if (old >= V || seen[old]) { free(inv); free(seen); return ORACLE_E_INVALID; }
        seen[old] = 1;
        inv[old] = (uint32_t)nv;
    }
    uint64_t k = 0;
    off_out[0] = 0;
    for (uint64_t nv = 0; nv < V; ++nv) {
        const uint32_t old = order[nv];
        for (uint64_t e = off[old]; e < off[old + 1]; ++e, ++k) {
            cols_out[k] = inv[cols[e]];
            if (w && w_out) w_out[k] = w[e];
        }
        off_out[nv + 1] = k;
    }
    (void)E;
    free(inv); free(seen);
    return 0;
}

/* ---------------------------------------------------------------------
 * Edge-list loading, restating GraphLoader::load_edge_list
 * (src/graph/graph_loader.cpp:39-179) with the extraction rules of the
 * C++ streams it uses (`stream >> uint64_t`, `stream >> float`,
 * `stream >> std::string`, libstdc++):
 *   lines split at '\n'; a line that is empty or starts with '#' after
 *   trimming " \t\r\n" is skipped; then source, destination (unsigned:
 *   whitespace, optional sign, decimal digits, overflow fails, '-' negates
 *   modulo 2^64), the weight when weighted ([sign] digits [. digits]
 *   [e [sign] digits] as accumulated by num_get, converted by strtof;
 *   nothing converted, unconverted characters or an infinite result fail),
 *   and any further non-blank character is an error.  Ids >= V fail.
 *   CSR: edges stably ordered by source (file order kept within a source,
 *   duplicates kept), offsets by counting.
 * Error kinds: 1 cannot open, 2 malformed edge, 3 vertex id out of range,
 * 4 missing edge weight, 5 unexpected data; *err_line = 1-based line.
 * ------------------------------------------------------------------- */
static int ws_char(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r'; }
static int trim_char(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\n'; }

static const char *skip_ws(const char *p, const char *e) {
    while (p < e && ws_char(*p)) ++p;
    return p;
}

/* stream >> uint64_t */
static int extract_u64(const char **pp, const char *e, uint64_t *out) {
    const char *p = skip_ws(*pp, e);
    int neg = 0, digits = 0, overflow = 0;
    uint64_t v = 0;
    if (p < e && (*p == '-' || *p == '+')) { neg = *p == '-'; ++p; }
    while (p < e && *p >= '0' && *p <= '9') {
        const uint64_t d = (uint64_t)(*p - '0');
        if (v > (UINT64_MAX - d) / 10) overflow = 1;
        v = v * 10 + d;
        ++digits;
        ++p;
    }
    *pp = p;
    if (!digits || overflow) return 0;
    *out = neg ? (uint64_t)0 - v : v;
    return 1;
}

/* stream >> float */
static int extract_f32(const char **pp, const char *e, float *out) {
    const char *p = skip_ws(*pp, e);
    char buf[512];
    size_t n = 0;
    int mant = 0, dec = 0, sci = 0;
#define PUT(ch) do { if (n + 1 < sizeof(buf)) buf[n++] = (ch); } while (0)
    if (p < e && (*p == '+' || *p == '-')) { PUT(*p); ++p; }
    while (p < e && *p == '0') { /* leading zeros collapse to one */
        if (!mant) { PUT('0'); mant = 1; }
        ++p;
    }
    while (p < e) {
        const char c = *p;
        if (c == '.' && !dec && !sci) { PUT('.'); dec = 1; }
        else if (c >= '0' && c <= '9') { PUT(c); mant = 1; }
        else if ((c == 'e' || c == 'E') && !sci && mant) {
            PUT('e');
            sci = 1;
            ++p;
            if (p >= e) break;
            if (*p == '+' || *p == '-') PUT(*p);
            else continue;
        } else break;
        ++p;
    }
#undef PUT
    buf[n] = '\0';
    *pp = p;
    char *end = NULL;
    const float v = strtof(buf, &end);
    if (end == buf || *end != '\0') return 0;
    if (isinf(v)) return 0;
    *out = v;
    return 1;
}

static uint64_t g_loaded_V, g_loaded_E;
static uint64_t *g_loaded_off;
static uint32_t *g_loaded_cols;
static float *g_loaded_w;

void oracle_loaded_free(void) {
    free(g_loaded_off); free(g_loaded_cols); free(g_loaded_w);
    g_loaded_off = NULL; g_loaded_cols = NULL; g_loaded_w = NULL;
    g_loaded_V = g_loaded_E = 0;
}

int oracle_load_edge_list(const char *path, uint64_t V, int weighted, uint64_t *E_out, uint64_t *err_line) {
    oracle_loaded_free();
    *E_out = 0;
    *err_line = 0;
    FILE *f = fopen(path, "rb");
    if (!f) return 1;
    fseek(f, 0, SEEK_END);
    const long size = ftell(f);
    fseek(f, 0, SEEK_SET);
    char *text = (char *)malloc(size > 0 ? (size_t)size : 1);
    if (size > 0 && fread(text, 1, (size_t)size, f) != (size_t)size) { fclose(f); free(text); return 1; }
    fclose(f);
    uint64_t cap = 1024, E = 0, line_no = 0;
    uint32_t *src = (uint32_t *)malloc(cap * 4), *dst = (uint32_t *)malloc(cap * 4);
    float *wt = (float *)malloc(cap * 4);
    int rc = 0;
    const char *p = text, *end = text + (size > 0 ? size : 0);
    while (p < end) {
        const char *nl = memchr(p, '\n', (size_t)(end - p));
        const char *le = nl ? nl : end;
        ++line_no;
        const char *a = p, *b = le;
        while (a < b && trim_char(*a)) ++a;
        while (b > a && trim_char(b[-1])) --b;
        p = nl ? nl + 1 : end;
        if (a == b || *a == '#') continue;
        uint64_t s = 0, d = 0;
        float w = 0.0f;
        const char *q = a;
        if (!extract_u64(&q, b, &s) || !extract_u64(&q, b, &d)) { rc = 2; break; }
        if (s >= V || d >= V) { rc = 3; break; }
        if (weighted && !extract_f32(&q, b, &w)) { rc = 4; break; }
        if (skip_ws(q, b) != b) { rc = 5; break; }
        if (E == cap) {
            cap *= 2;
            src = (uint32_t *)realloc(src, cap * 4);
            dst = (uint32_t *)realloc(dst, cap * 4);
            wt = (float *)realloc(wt, cap * 4);
        }
        src[E] = (uint32_t)s;
        dst[E] = (uint32_t)d;
        wt[E] = w;
        ++E;
    }
    free(text);
    if (rc) {
        *err_line = line_no;
        free(src); free(dst); free(wt);
        return rc;
    }
    /* stable counting sort by source */
    uint64_t *off = (uint64_t *)calloc(V + 1, 8);
    uint64_t *cur = (uint64_t *)malloc((V + 1) * 8);
    uint32_t *cols = (uint32_t *)malloc((E ? E : 1) * 4);
    float *wo = weighted ? (float *)malloc((E ? E : 1) * 4) : NULL;
    for (uint64_t i = 0; i < E; ++i) ++off[src[i] + 1];
    for (uint64_t v = 0; v < V; ++v) off[v + 1] += off[v];
    memcpy(cur, off, (V + 1) * 8);
    for (uint64_t i = 0; i < E; ++i) {
        const uint64_t k = cur[src[i]]++;
        cols[k] = dst[i];
        if (wo) wo[k] = wt[i];
    }
    free(cur); free(src); free(dst); free(wt);
    g_loaded_V = V;
    g_loaded_E = E;
    g_loaded_off = off;
    g_loaded_cols = cols;
    g_loaded_w = wo;
    *E_out = E;
    return 0;
}

void oracle_loaded_copy(uint64_t *off, uint32_t *cols, float *w) {
    memcpy(off, g_loaded_off, (g_loaded_V + 1) * 8);
    if (g_loaded_E) memcpy(cols, g_loaded_cols, g_loaded_E * 4);
    if (w && g_loaded_w && g_loaded_E) memcpy(w, g_loaded_w, g_loaded_E * 4);
}

/* CSR from edge arrays (the loader's construction step): stable by source;
 * returns 0, or 1 + the index of the first edge with an id >= V. */
uint64_t oracle_csr_from_edges(uint64_t V, uint64_t E, const uint32_t *src, const uint32_t *dst, const uint32_t *w,
                               uint64_t *off, uint32_t *cols, uint32_t *w_out) {
    for (uint64_t i = 0; i < E; ++i)
        if (src[i] >= V || dst[i] >= V) return i + 1;
    memset(off, 0, (V + 1) * 8);
    for (uint64_t i = 0; i < E; ++i) ++off[src[i] + 1];
    for (uint64_t v = 0; v < V; ++v) off[v + 1] += off[v];
    uint64_t *cur = (uint64_t *)malloc((V + 1) * 8);
    memcpy(cur, off, (V + 1) * 8);
    for (uint64_t i = 0; i < E; ++i) {
        const uint64_t k = cur[src[i]]++;
        cols[k] = dst[i];
        if (w && w_out) w_out[k] = w[i];
    }
    free(cur);
    return 0;
}

/* ---------------------------------------------------------------------
 * Contribution-driven scheduling, restating
 * src/algorithms/pagerank.cpp:165-241 (pagerank_contributions, FP32 in the
 * reference's operation order), src/algorithms/sssp.cpp:236-290
 * (sssp_contributions) and src/scheduling/contribution_scheduler.cpp:23-121
 * (ContributionScheduler::schedule and its metrics).
 * ------------------------------------------------------------------- */
int oracle_pagerank_contributions(uint64_t V, uint64_t E, const uint64_t *off, const uint32_t *cols,
                                  const float *cur, float damping, int fp64, double *out) {
    uint64_t *in_off = NULL;
    uint32_t *in_src = NULL;
    const int rc = build_incoming(V, E, off, cols, NULL, &in_off, &in_src, NULL);
    if (rc) return rc;
    if (fp64) {
        double dm = 0.0;
        for (uint64_t u = 0; u < V; ++u)
            if (off[u + 1] == off[u]) dm += cur[u];
        const double share = (1.0 - damping) / (double)V + (double)damping * dm / (double)V;
        for (uint64_t v = 0; v < V; ++v) {
            double s = 0.0;
            for (uint64_t e = in_off[v]; e < in_off[v + 1]; ++e) {
                const uint32_t u = in_src[e];
                s += (double)cur[u] / (double)(off[u + 1] - off[u]);
            }
            out[v] = fabs(share + (double)damping * s - (double)cur[v]);
        }
    } else {
        const float base = (1.0f - damping) / (float)V;
        float dm = 0.0f;
        for (uint64_t u = 0; u < V; ++u)
            if (off[u + 1] == off[u]) dm += cur[u];
        const float share = damping * dm / (float)V;
        for (uint64_t v = 0; v < V; ++v) {
            float s = 0.0f;
            for (uint64_t e = in_off[v]; e < in_off[v + 1]; ++e) {
                const uint32_t u = in_src[e];
                const uint64_t deg = off[u + 1] - off[u];
                if (deg) s += cur[u] / (float)deg;
            }
            const float next = base + share + damping * s;
            out[v] = (double)fabsf(next - cur[v]);
        }
    }
    free(in_off); free(in_src);
    return 0;
}

void oracle_sssp_contributions(uint64_t n, const float *cur, const float *cand, float tol, double *out) {
    for (uint64_t v = 0; v < n; ++v) {
        const float c = cur[v], d = cand[v];
        double r = 0.0;
        if (isfinite(c) && isfinite(d)) {
            const float imp = c - d;
            if (imp > tol) r = (double)imp;
        } else if (!isfinite(c) && isfinite(d)) {
            r = 1.0;
        }
        out[v] = r;
    }
}

static const uint64_t *g_sched_item;
static const double *g_sched_c;
static int g_sched_det;
static int sched_cmp(const void *pa, const void *pb) {
    const uint64_t a = *(const uint64_t *)pa, b = *(const uint64_t *)pb;
    const double ca = g_sched_c[a], cb = g_sched_c[b];
    if (ca != cb) return ca > cb ? -1 : 1;
    if (g_sched_det && g_sched_item[a] != g_sched_item[b]) return g_sched_item[a] < g_sched_item[b] ? -1 : 1;
    return a < b ? -1 : (a > b); /* stable: input position */
}
static int u64_cmp(const void *pa, const void *pb) {
    const uint64_t a = *(const uint64_t *)pa, b = *(const uint64_t *)pb;
    return a < b ? -1 : (a > b);
}

/* metrics[0..6] = input, scheduled, reordered, zero, overhead (as double
 * bits), stale (0), redundant.  Returns ORACLE_E_INVALID on a non-finite
 * contribution. */
int oracle_contribution_schedule(uint64_t n, const uint64_t *item, const double *c, int det, double eps,
                                 uint64_t *ordered, uint64_t *metrics) {
    for (uint64_t i = 0; i < n; ++i)
        if (!isfinite(c[i])) return ORACLE_E_INVALID;
    uint64_t *order = (uint64_t *)malloc((n ? n : 1) * 8), *sorted = (uint64_t *)malloc((n ? n : 1) * 8);
    uint64_t zero = 0, moved = 0, dup = 0;
    for (uint64_t i = 0; i < n; ++i) {
        order[i] = i;
        sorted[i] = item[i];
        if (fabs(c[i]) <= eps) ++zero;
    }
    g_sched_item = item; g_sched_c = c; g_sched_det = det;
    qsort(order, n, 8, sched_cmp);
    qsort(sorted, n, 8, u64_cmp);
    for (uint64_t i = 1; i < n; ++i) dup += sorted[i] == sorted[i - 1];
    for (uint64_t p = 0; p < n; ++p) {
        ordered[p] = item[order[p]];
        moved += order[p] != p;
    }
    const double overhead = n ? log2((double)n) : 0.0;
    metrics[0] = n; metrics[1] = n; metrics[2] = moved; metrics[3] = zero;
    memcpy(&metrics[4], &overhead, 8);
    metrics[5] = 0; metrics[6] = dup;
    free(order); free(sorted);
    return 0;
}

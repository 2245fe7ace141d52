/*
 * hyt/capi.h -- C ABI of the B200 graph-processing core (libhyt_core.so).
 *
 * Plain C: opaque handles, plain pointers and sizes, int status codes.
 * The C++ drop-in layer (include/algorithms, include/transfer, ...) and the
 * Python bindings (hytgraph_b200/capi.py) are thin wrappers over this file.
 *
 * Conventions
 *   - Every entry point returns HYT_OK (0) or one of the HYT_E_* codes; the
 *     message of the last failure on the calling thread is hyt_last_error().
 *   - Host buffers are owned by the caller.  A result pointer may be a host
 *     pointer (pageable or pinned) or a device pointer; the library detects
 *     which with cudaPointerGetAttributes and copies accordingly.
 *   - Device memory behind a handle is owned by the library.
 *   - One handle is used by one host thread at a time.
 *   - `stream` fields take a cudaStream_t (NULL = the handle's own stream).
 *     Calls are synchronous with respect to the host on return.
 *
 * Reference interfaces replaced (tanishbhongade/hytgraph):
 *   hyt_pagerank   -> algorithms::pagerank_gpu   include/algorithms/pagerank.hpp:50-52
 *                                                 (cuda/pagerank.cu:157-337)
 *   hyt_sssp       -> algorithms::sssp_gpu       include/algorithms/sssp.hpp:49-51
 *                                                 (cuda/sssp.cu:158-321)
 *   hyt_graph_*    -> the device copy of graph::CSRGraph that pagerank_gpu /
 *                     sssp_gpu build per call (cuda/pagerank.cu:184-244,
 *                     cuda/sssp.cu:207-244); here it persists in a handle.
 *   hyt_ppr        -> no reference symbol (personalized PageRank is new).
 */
#ifndef HYT_CAPI_H
#define HYT_CAPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HYT_ABI_VERSION 1

enum hyt_status_code {
    HYT_OK = 0,
    HYT_E_INVALID = 1,     /* bad argument: std::invalid_argument in C++ */
    HYT_E_CUDA = 2,        /* CUDA runtime error: std::runtime_error */
    HYT_E_OOM = 3,         /* device/pinned allocation failed or over budget */
    HYT_E_TIMEOUT = 4,     /* a bounded device-side wait ran out */
    HYT_E_NO_DEVICE = 5,   /* no CUDA device is available */
    HYT_E_UNSUPPORTED = 6, /* valid request this build does not implement */
    HYT_E_INTERNAL = 7,    /* an internal consistency check failed */
    HYT_E_IO = 8           /* a file could not be opened, read or written:
                              std::runtime_error */
};

/* Message of the last failing call on this thread ("" if none). */
const char *hyt_last_error(void);
int hyt_abi_version(void);
/* Number of visible CUDA devices (0 without error when there is none). */
int hyt_device_count(int *count);
/* Synchronous copy between any two host/device buffers (unified
 * addressing decides the direction); stream NULL = a library stream. */
int hyt_copy(void *dst, const void *src, uint64_t bytes, void *stream);

/* ------------------------------------------------------------------ */
/* CSR input                                                           */
/* ------------------------------------------------------------------ */

enum hyt_weight_kind {
    HYT_WEIGHTS_NONE = 0, /* unweighted: every edge weighs 1 */
    HYT_WEIGHTS_U32 = 1,  /* uint32 weights, exact integer distances */
    HYT_WEIGHTS_F32 = 2   /* IEEE float weights (finite, >= 0) */
};

/* A CSR graph: row_offsets[V+1] (uint64), column_indices[E] (uint32),
 * optional weights[E] whose type is given by weight_kind.  Pointers may be
 * host or device memory.  Layout of graph::CSRGraph
 * (include/graph/csr_graph.hpp:14-16, 63-69). */
typedef struct hyt_csr {
    uint64_t num_vertices;
    uint64_t num_edges;
    const uint64_t *row_offsets;
    const uint32_t *column_indices;
    const void *weights;
    uint32_t weight_kind;
} hyt_csr;

/* ------------------------------------------------------------------ */
/* Device-resident graph                                               */
/* ------------------------------------------------------------------ */

typedef struct hyt_graph hyt_graph;

enum hyt_graph_flags {
    HYT_GRAPH_PULL = 1u,   /* build the CSC + PageRank work tiles (pull) */
    HYT_GRAPH_PUSH = 2u,   /* keep the CSR (+ weights) for frontier push */
    HYT_GRAPH_ALL = 3u,
    /* Store the graph in hub order: vertices renumbered by the reference's
     * hub score Do*Di (HubSorter with hub_fraction 1, hyt_hub_sort), so the
     * high-degree vertices' values share cache lines.  Sources and results
     * stay in the caller's vertex ids (mapped on the way in and out).
     * hyt_pagerank, hyt_ppr, hyt_ppr_multi, hyt_sssp and the batch / server
     * engines map ids; hyt_graph_copy_csc and hyt_pagerank_contributions
     * reject such graphs (HYT_E_UNSUPPORTED). */
    HYT_GRAPH_HUB_ORDER = 4u
};

typedef struct hyt_graph_options {
    uint32_t flags;  /* HYT_GRAPH_* (0 = HYT_GRAPH_ALL) */
    int device;      /* CUDA device ordinal; < 0: the calling thread's current device */
    void *stream;    /* cudaStream_t used for the upload (NULL = own) */
} hyt_graph_options;

/* In-HBM graph arrays and the one-shot transforms' scratch come from
 * per-device memory pools that keep freed memory mapped (graph arrays: up to
 * 16 GiB; scratch: up to 2 GiB), so repeated graph creation does not map
 * fresh memory each time.  This returns that cached memory of `device` to
 * the driver (after waiting for the device). */
int hyt_trim_device_memory(int device);

typedef struct hyt_graph_info {
    uint64_t num_vertices;
    uint64_t num_edges;
    uint32_t weight_kind;
    uint32_t flags;
    uint64_t device_bytes;      /* HBM held by the handle */
    uint64_t pull_tiles;        /* PageRank work tiles */
    uint64_t long_rows;         /* in-degree rows split across CTAs */
    uint64_t max_in_degree;
    uint64_t max_out_degree;
    uint64_t dangling_vertices; /* out-degree 0 */
    double build_ms;            /* device time of upload + CSC/tile build */
    int32_t device;             /* CUDA device ordinal the graph lives on */
    uint32_t pad;
} hyt_graph_info;

/* NULL options: all defaults, with the calling thread's current device
 * (device ordinal -1); the current device is left unchanged. */
int hyt_graph_create(const hyt_csr *csr, const hyt_graph_options *options,
                     hyt_graph **out);
int hyt_graph_destroy(hyt_graph *graph);
int hyt_graph_get_info(const hyt_graph *graph, hyt_graph_info *out);

/* ------------------------------------------------------------------ */
/* PageRank (pull over CSC)                                            */
/* ------------------------------------------------------------------ */

enum hyt_run_flags {
    HYT_RUN_PROFILE = 1u,   /* time every hot-kernel launch with events */
    HYT_RUN_NO_GRAPH = 2u   /* host-driven loop instead of a CUDA graph */
};

typedef struct hyt_pagerank_params {
    float damping;           /* [0, 1) */
    float tolerance;         /* > 0: stop when the L1 change <= tolerance */
    uint32_t max_iterations; /* > 0 */
    uint32_t flags;          /* HYT_RUN_* */
    void *stream;
} hyt_pagerank_params;

typedef struct hyt_run_stats {
    uint32_t iterations;       /* PageRank iterations / SSSP rounds */
    uint32_t converged;
    double residual;           /* PageRank: FP64 L1 change of the last step */
    double device_ms;          /* device time of the whole solve */
    double kernel_ms;          /* summed hot-kernel time (HYT_RUN_PROFILE) */
    uint32_t kernel_launches;  /* hot-kernel launches (HYT_RUN_PROFILE) */
    uint32_t total_launches;   /* every kernel this call launched */
    uint64_t edges_processed;  /* edges read (PR) / relaxed (SSSP) */
    uint64_t vertices_processed;
    uint64_t algorithmic_bytes;/* roofline numerator for the whole solve */
} hyt_run_stats;

/* ranks_out: [V] floats (host or device) or NULL to keep them on device. */
int hyt_pagerank(hyt_graph *graph, const hyt_pagerank_params *params,
                 float *ranks_out, hyt_run_stats *stats);

/* Personalized PageRank from 1 to 8 sources at once (no reference
 * counterpart): each query as hyt_ppr defines it, all of them sharing every
 * pass over the CSC (one source id and one 32-byte sector of the 8 queries'
 * contributions per in-edge).  A query's result does not depend on which
 * other queries share the call; each stops after its own converging step.
 * ranks_out: [num_sources][V] floats (host or device) or NULL; stats:
 * num_sources entries or NULL (stats[0].algorithmic_bytes covers the call).
 * Defined in the same terms as hyt_ppr below. */
int hyt_ppr_multi(hyt_graph *graph, const uint32_t *sources, uint32_t num_sources, float restart, float tolerance,
                  uint32_t max_iterations, float *ranks_out, hyt_run_stats *stats);

/* Personalized PageRank from one source (no reference counterpart):
 *   x' = d * sum_{u->v} x_u / deg(u) + [v == s] * ((1 - d) + d * dangling)
 * with d = 1 - restart, x_0 = e_s, stop when the L1 change <= tolerance. */
typedef struct hyt_ppr_params {
    uint32_t source;
    float restart;           /* (0, 1]; damping = 1 - restart */
    float tolerance;
    uint32_t max_iterations;
    uint32_t flags;
    void *stream;
} hyt_ppr_params;

int hyt_ppr(hyt_graph *graph, const hyt_ppr_params *params, float *ranks_out,
            hyt_run_stats *stats);

/* ------------------------------------------------------------------ */
/* SSSP (frontier push over CSR, atomicMin relaxation)                  */
/* ------------------------------------------------------------------ */

#define HYT_DIST_INF_U32 0xFFFFFFFFu

typedef struct hyt_sssp_params {
    uint32_t source;
    uint32_t delta;       /* near/far bucket width; 0 = chosen from weights */
    uint32_t max_rounds;  /* 0 = unlimited (bounded by V*(V-1) relaxations) */
    uint32_t flags;       /* HYT_RUN_* */
    void *stream;
} hyt_sssp_params;

/* dist_out: [V] (host or device) or NULL.  U32/NONE graphs: exact integer
 * distances, HYT_DIST_INF_U32 = unreachable.  F32 graphs: IEEE float bit
 * patterns (0x7f800000 = +inf). */
int hyt_sssp(hyt_graph *graph, const hyt_sssp_params *params,
             uint32_t *dist_out, hyt_run_stats *stats);

/* SSSP from 1 to 8 sources at once (no reference counterpart; each source
 * as hyt_sssp defines it, the reference's sssp_cpu fixed point): the 8
 * labels of a vertex share one 32-byte row, so every push round expands the
 * union frontier once and every pull sweep reads each in-edge once for all
 * sources.  Each source's labels are bit-identical to hyt_sssp's.
 * dist_out: [num_sources][V] (host or device) or NULL; max_rounds 0 =
 * unlimited; stats covers the whole call. */
int hyt_sssp_multi(hyt_graph *graph, const uint32_t *sources, uint32_t num_sources, uint32_t max_rounds,
                   uint32_t *dist_out, hyt_run_stats *stats);

/* SSSP that allocates nothing.  No counterpart in the reference: it exists
 * for callers that cannot call cudaMalloc -- a host whose caching allocator
 * already holds the device's free memory, a latency-critical loop that must
 * not pay cudaMalloc's implicit device synchronisation, or a plugin host
 * that forbids its components to allocate.
 *
 * csr: row_offsets / column_indices / weights in device memory of the
 * current device; dist_out: [V] uint32 in device memory (same meaning as
 * hyt_sssp).  All solver state lives in one fixed __device__ array inside
 * the library (32.3 MiB per GPU that loads it, held until exit), so the
 * graph may have at most HYT_NOALLOC_MAX_VERTICES vertices and
 * HYT_NOALLOC_MAX_EDGES edges; larger graphs fail with HYT_E_INVALID.
 * The first call on a device looks up that array's device address; make it
 * before any stream capture.  Calls share the array: calls whose GPU work
 * overlaps (other streams or threads) race.  stats: rounds, relaxations and
 * launches; device_ms is not measured (no events are created). */
#define HYT_NOALLOC_MAX_VERTICES (1u << 20)
#define HYT_NOALLOC_MAX_EDGES (1u << 24)
int hyt_sssp_noalloc(const hyt_csr *csr, uint32_t source, uint32_t *dist_out, void *stream,
                     hyt_run_stats *stats);

/* ------------------------------------------------------------------ */
/* Out-of-HBM hybrid transfer (edges in pinned host memory)            */
/* ------------------------------------------------------------------ */

/* Reverse graph: in_offsets[V+1] (uint64), in_sources[E] (uint32), the
 * sources of each vertex's in-edges in ascending source order -- the
 * IncomingCSR that the reference's PageRank builds
 * (src/algorithms/pagerank.cpp:19-59). */
typedef struct hyt_csc {
    uint64_t num_vertices;
    uint64_t num_edges;
    const uint64_t *in_offsets;
    const uint32_t *in_sources;
} hyt_csc;

/* Copies an in-HBM graph's CSC (built with HYT_GRAPH_PULL) into caller
 * buffers (host or device): in_offsets[V+1], in_sources[E]. */
int hyt_graph_copy_csc(const hyt_graph *graph, uint64_t *in_offsets, uint32_t *in_sources);

/* Pinned, device-mapped, portable host memory (cudaHostAlloc) for the
 * host-side arrays of hybrid graphs; free with hyt_pinned_free. */
int hyt_pinned_alloc(uint64_t bytes, void **out);
int hyt_pinned_free(void *ptr);

typedef struct hyt_hybrid hyt_hybrid;

/* Transfer engines of the HyTM model (transfer::TransferEngine,
 * include/transfer/hytm_cost_model.hpp:17-21). */
enum hyt_engine {
    HYT_ENGINE_AUTO = 0,        /* cost model decides per partition per round */
    HYT_ENGINE_FILTER = 1,      /* ExpTM-Filter: whole partition copied */
    HYT_ENGINE_COMPACTION = 2,  /* ExpTM-Compaction: active rows gathered on
                                   the host, shipped packed */
    HYT_ENGINE_ZERO_COPY = 3    /* ImpTM: kernels read mapped host memory */
};

/* The CSR (and, with HYT_GRAPH_PULL, the CSC) stay in HOST memory owned by
 * the caller for the handle's lifetime: pinned (cudaHostAlloc /
 * cudaMallocHost with mapping) or pageable (then registered mapped and
 * read-only here, unregistered on destroy).  Vertex arrays (offsets,
 * degrees, labels, ranks, frontiers) live in HBM outside the budget. */
typedef struct hyt_hybrid_options {
    uint32_t flags;               /* HYT_GRAPH_* (0 = HYT_GRAPH_ALL) */
    int device;                   /* < 0: the calling thread's current device */
    uint64_t device_budget_bytes; /* HBM for edge data: resident partitions +
                                     staging (0 = 8 GiB) */
    uint32_t partition_vertices;  /* power of two (0 = 2^20); <= 1024 parts */
    uint32_t host_threads;        /* compaction / gather threads (0 = all) */
    uint32_t force_engine;        /* HYT_ENGINE_* for partitions that are not
                                     resident (AUTO = cost model) */
    float alpha, beta, gamma;     /* HyTM selector thresholds
                                     (0 = 0.8 / 0.4 / 0.625) */
} hyt_hybrid_options;

typedef struct hyt_hybrid_info {
    uint64_t partitions;
    uint64_t budget_bytes;
    uint64_t resident_bytes;          /* edge bytes resident in HBM */
    uint64_t staging_bytes;           /* filter slots + compaction buffer */
    uint64_t resident_push_partitions;
    uint64_t resident_pull_partitions;
    uint64_t device_bytes;            /* all HBM held by the handle */
    double h2d_gbs;                   /* measured pinned cudaMemcpy H2D */
    double zero_copy_gbs;             /* measured in-kernel mapped reads */
    double gather_gbs;                /* measured host gather (compaction) */
} hyt_hybrid_info;

/* Per solve: decisions are counted per (partition, round) with work. */
typedef struct hyt_hybrid_stats {
    uint64_t rounds;
    uint64_t resident_decisions, filter_decisions, compaction_decisions, zero_copy_decisions;
    uint64_t filter_bytes;      /* cudaMemcpyAsync'd partitions */
    uint64_t compaction_bytes;  /* packed payloads shipped */
    uint64_t zero_copy_bytes;   /* 128-byte lines read over the link */
    uint64_t link_bytes;        /* sum of the three */
    uint64_t necessary_bytes;   /* edge bytes of the active rows not resident */
    uint64_t copies;            /* cudaMemcpyAsync calls of the filter engine */
    double compaction_host_ms;  /* host gather time */
    double device_ms;           /* device time of the solve */
    double link_gbs;            /* link_bytes / device time */
    double h2d_peak_gbs;        /* measured pinned-copy peak */
} hyt_hybrid_stats;

/* NULL options: all defaults, with the calling thread's current device
 * (device ordinal -1); the current device is left unchanged. */
int hyt_hybrid_create(const hyt_csr *csr, const hyt_csc *csc, const hyt_hybrid_options *options,
                      hyt_hybrid **out);
int hyt_hybrid_destroy(hyt_hybrid *hybrid);
int hyt_hybrid_get_info(const hyt_hybrid *hybrid, hyt_hybrid_info *out);
/* Same semantics, stop rule and outputs as hyt_pagerank / hyt_sssp. */
int hyt_hybrid_pagerank(hyt_hybrid *hybrid, const hyt_pagerank_params *params, float *ranks_out,
                        hyt_run_stats *stats, hyt_hybrid_stats *transfer);
int hyt_hybrid_sssp(hyt_hybrid *hybrid, const hyt_sssp_params *params, uint32_t *dist_out,
                    hyt_run_stats *stats, hyt_hybrid_stats *transfer);

/* ------------------------------------------------------------------ */
/* Batched queries: many SSSP / personalized-PageRank queries over many */
/* resident graphs in one CUDA-graph launch                             */
/* ------------------------------------------------------------------ */

enum hyt_query_kind {
    HYT_QUERY_SSSP = 0,
    HYT_QUERY_PPR = 1
};

typedef struct hyt_query {
    uint32_t graph;           /* index into the batch's graph list */
    uint32_t kind;            /* HYT_QUERY_* */
    uint32_t source;
    float restart;            /* PPR: (0, 1]; 0 = 0.15 */
    float tolerance;          /* PPR: L1 stop; 0 = 1e-6 */
    uint32_t max_iterations;  /* PPR: 0 = 100; SSSP: round cap, 0 = none */
    void *out;                /* SSSP: uint32 dist[V]; PPR: float ranks[V];
                                 host or device memory, or NULL */
} hyt_query;

typedef struct hyt_query_result {
    uint32_t iterations;      /* PPR iterations / SSSP rounds */
    uint32_t converged;
    double residual;          /* PPR: L1 change of the last iteration */
    uint64_t edges_processed; /* PPR: iterations * E; SSSP: relaxations */
} hyt_query_result;

/* Knobs the autotuner chooses (0 = default). */
typedef struct hyt_batch_tuning {
    uint32_t delta_mult;   /* SSSP bucket width = delta_mult x mean edge
                              weight of the query's graph; 0 = one bucket */
    uint32_t hub_degree;   /* SSSP rows >= this many edges are split into
                              512-edge warp tasks (default 64) */
    uint32_t ctas_per_sm;  /* persistent work grid (0 = occupancy) */
} hyt_batch_tuning;

typedef struct hyt_batch_options {
    int device;                   /* < 0: the calling thread's current device */
    uint64_t state_budget_bytes;  /* device bytes for per-query state
                                     (0 = 16 GiB); larger batches run in
                                     waves that fit */
    hyt_batch_tuning tuning;
    uint32_t flags;               /* HYT_RUN_NO_GRAPH: host-driven supersteps */
} hyt_batch_options;

typedef struct hyt_batch_stats {
    double device_ms;          /* device time of the whole batch */
    uint32_t supersteps;
    uint32_t waves;            /* admission waves (1 when all fit) */
    uint32_t graph_launches;   /* CUDA-graph launches */
    uint32_t kernel_launches;  /* kernels executed (graph nodes included) */
    uint64_t edges_processed;  /* sum over queries */
    uint64_t algorithmic_bytes;
    uint64_t state_bytes;      /* peak per-query state held */
} hyt_batch_stats;

typedef struct hyt_batch hyt_batch;

/* graphs: handles built with HYT_GRAPH_ALL (borrowed; keep them alive).
 * NULL options: all defaults, with the calling thread's current device
 * (device ordinal -1); the current device is left unchanged. */
int hyt_batch_create(hyt_graph *const *graphs, uint32_t num_graphs, const hyt_batch_options *options,
                     hyt_batch **out);
int hyt_batch_destroy(hyt_batch *batch);
/* Runs every query; results[i] belongs to queries[i].  A query's result is
 * the same whatever else is in the batch (SSSP: identical to hyt_sssp;
 * PPR: identical across batches, within L1 1e-6 of hyt_ppr). */
int hyt_batch_run(hyt_batch *batch, const hyt_query *queries, uint32_t num_queries,
                  hyt_query_result *results, hyt_batch_stats *stats);
/* Times the batch on a sample of `queries` under a grid of tunings and
 * keeps the fastest for later runs; *chosen receives it.  The choice is
 * cached for the process per size class of the sample (device, log2 of its
 * mean graph edges and vertices, SSSP share in quarters): a later call with
 * a sample of the same class applies the cached tuning without timing. */
int hyt_batch_autotune(hyt_batch *batch, const hyt_query *queries, uint32_t num_queries,
                       hyt_batch_tuning *chosen);
int hyt_batch_set_tuning(hyt_batch *batch, const hyt_batch_tuning *tuning);

/* ------------------------------------------------------------------ */
/* Serving: continuous batching of arriving queries                     */
/* ------------------------------------------------------------------ */

/* A server owns one worker thread and one stream.  Submitted queries wait
 * in a FIFO; between supersteps the worker admits waiting queries while
 * the per-query state budget and the slot table allow, advances every
 * running query by one superstep (one SSSP round / one PPR iteration,
 * a single CUDA-graph launch), and retires the finished ones: their result
 * is copied to the query's `out` buffer (which must stay valid until the
 * completion is polled) and a completion is queued.  A query's result is
 * the same whatever else runs beside it (hyt_batch_run's guarantee). */
typedef struct hyt_server hyt_server;

typedef struct hyt_server_options {
    int device;                   /* < 0: the calling thread's current device */
    uint64_t state_budget_bytes;  /* 0 = 16 GiB */
    hyt_batch_tuning tuning;
    uint32_t max_running;         /* cap on concurrently running queries
                                     (0 = slot table size, 4096) */
    uint32_t pack_min_edges;      /* queries on graphs with at least this
                                     many edges run in packs of up to 8 of
                                     the same kind and parameters sharing
                                     one solve (hyt_sssp_multi /
                                     hyt_ppr_multi); 0 = 2^22, UINT32_MAX =
                                     never */
} hyt_server_options;

typedef struct hyt_completion {
    uint64_t ticket;
    int status;                   /* HYT_OK or an HYT_E_* code (HYT_E_OOM:
                                     the query's state exceeds the budget) */
    hyt_query_result result;
    double queue_ms;              /* submit -> admitted */
    double latency_ms;            /* submit -> result in `out` */
} hyt_completion;

typedef struct hyt_server_stats {
    uint64_t submitted, completed, supersteps, graph_launches;
    uint32_t running, waiting, max_running;
    uint64_t state_bytes, peak_state_bytes;
    double busy_ms;               /* worker time with queries running */
    uint64_t packs;               /* packed solves run (pack_min_edges) */
} hyt_server_stats;

/* graphs: handles built with HYT_GRAPH_ALL (borrowed; keep them alive).
 * NULL options: all defaults, with the calling thread's current device
 * (device ordinal -1); the current device is left unchanged. */
int hyt_server_create(hyt_graph *const *graphs, uint32_t num_graphs, const hyt_server_options *options,
                      hyt_server **out);
/* Thread-safe.  Validates the query (HYT_E_INVALID as hyt_batch_run) and
 * queues it; *ticket identifies its completion. */
int hyt_server_submit(hyt_server *server, const hyt_query *query, uint64_t *ticket);
/* Up to `max` completions into out[]; *count receives how many.  Waits up
 * to wait_ms milliseconds for the first one (0 = do not wait). */
int hyt_server_poll(hyt_server *server, hyt_completion *out, uint32_t max, uint32_t *count, uint32_t wait_ms);
int hyt_server_get_stats(hyt_server *server, hyt_server_stats *stats);
/* Stops the worker after the running queries finish (their completions
 * are discarded); queries still waiting for admission are dropped. */
int hyt_server_destroy(hyt_server *server);

/* ------------------------------------------------------------------ */
/* Seeded R-MAT generator (deterministic; same bytes on host and GPU)   */
/* ------------------------------------------------------------------ */

typedef struct hyt_rmat_params {
    uint32_t scale;        /* V = 2^scale, 1..31 */
    uint32_t edge_factor;  /* edge draws = edge_factor * V */
    double a, b, c;        /* quadrant probabilities, d = 1 - a - b - c */
    uint64_t seed;
    uint32_t weight_min;   /* uint32 weights uniform in [min, max] */
    uint32_t weight_max;   /* 0/0 = unweighted */
} hyt_rmat_params;

typedef struct hyt_csr_buffers {
    uint64_t num_vertices;
    uint64_t num_edges;
    uint64_t *row_offsets;
    uint32_t *column_indices;
    uint32_t *weights;     /* NULL when unweighted */
    uint32_t on_device;    /* 1: cudaMalloc'd, 0: malloc'd */
    uint32_t weight_kind;  /* HYT_WEIGHTS_* of `weights` */
} hyt_csr_buffers;

/* on_device = 0: generated on the host CPU cores; 1: on the current GPU.
 * Both produce identical bytes.  Free with hyt_csr_buffers_free. */
int hyt_rmat_generate(const hyt_rmat_params *params, int on_device,
                      hyt_csr_buffers *out);
int hyt_csr_buffers_free(hyt_csr_buffers *buffers);

/* Deterministic source choice: `count` vertices with out-degree > 0, drawn
 * uniformly with the given seed (host row offsets). */
int hyt_pick_sources(const uint64_t *row_offsets, uint64_t num_vertices,
                     uint64_t seed, uint32_t count, uint32_t *out);

/* ------------------------------------------------------------------ */
/* Hub sorting and vertex reordering on the GPU                         */
/* ------------------------------------------------------------------ */

/* Device-side figures of one hub-sort or reorder call. */
typedef struct hyt_reorder_stats {
    double device_ms;           /* the whole call on the device, copies included */
    double kernel_ms;           /* its main kernel: the degree pass (hub sort) or
                                   the edge permutation (reorder) */
    uint64_t kernel_bytes;      /* algorithmic bytes of that kernel */
    uint64_t algorithmic_bytes; /* algorithmic bytes of the whole call */
    uint32_t kernel_launches;   /* this library's kernels */
    uint32_t library_calls;     /* radix sorts, scans and selects */
} hyt_reorder_stats;

/* Hub-first vertex order of scheduling::HubSorter::sort
 * (src/scheduling/hub_sort.cpp:28-183): scores H(v) = Do(v) * Di(v) /
 * (Do_max * Di_max); the round-or-ceil(V * hub_fraction) best first (ties:
 * lower id), then the other vertices in id order.  csr: host or device
 * arrays.  vertex_order[V] (new -> old) and scores[V] (may be NULL): host or
 * device; *hub_count (may be NULL): host.  Scores equal the reference's
 * x86-64 long-double quotient rounded to double, bit for bit.  Rejects a
 * hub_fraction outside [0, 1] and a malformed CSR (HYT_E_INVALID).  stats
 * may be NULL. */
int hyt_hub_sort(const hyt_csr *csr, double hub_fraction, uint32_t *vertex_order, double *scores,
                 uint64_t *hub_count, hyt_reorder_stats *stats);

/* graph::CSRGraph::reorder_vertices (src/graph/csr_graph.cpp:171-283) into
 * new buffers: vertex_order[new] = old; each new row holds the old row's
 * edges in their original order with destinations renamed, weights carried.
 * on_device: 1 = cudaMalloc'd output, 0 = malloc'd; free with
 * hyt_csr_buffers_free.  Rejects out-of-range or duplicate entries with the
 * reference's messages, and a malformed CSR.  vertex_order: host or device.
 * stats may be NULL. */
int hyt_csr_reorder(const hyt_csr *csr, const uint32_t *vertex_order, int on_device, hyt_csr_buffers *out,
                    hyt_reorder_stats *stats);

/* ------------------------------------------------------------------ */
/* Graph construction and loading                                       */
/* ------------------------------------------------------------------ */

/* Host / device figures of one construction or load call. */
typedef struct hyt_load_stats {
    double total_ms;        /* the whole call (host clock) */
    double read_ms;         /* reading and parsing the file on host threads */
    double device_ms;       /* the device part (uploads, kernels, downloads) */
    double kernel_ms;       /* the main device step: the CSR construction
                               (sort + offsets + unpack) or the load checks */
    uint64_t file_bytes;    /* bytes read from the file */
    uint64_t num_edges;
    uint64_t kernel_bytes;  /* algorithmic bytes of the main device step */
    uint32_t threads;       /* host threads used */
    uint32_t pad;
} hyt_load_stats;

/* graph::GraphLoader::load_edge_list (src/graph/graph_loader.cpp:39-179):
 * a text edge list, one "source destination [weight]" record per line;
 * blank lines and lines starting with '#' are skipped; ids >= num_vertices,
 * malformed records, a missing weight (weighted) and trailing data fail
 * with HYT_E_INVALID and the reference's message and line number; a file
 * that cannot be opened fails with HYT_E_IO.  The CSR keeps the file's
 * edge order within each source and keeps parallel edges.  Weights are
 * float (HYT_WEIGHTS_F32).  The file is parsed by host threads; the CSR is
 * built on the GPU.  on_device: 1 = cudaMalloc'd output, 0 = malloc'd;
 * free with hyt_csr_buffers_free.  stats may be NULL. */
int hyt_load_edge_list(const char *path, uint64_t num_vertices, int weighted, int on_device,
                       hyt_csr_buffers *out, hyt_load_stats *stats);

/* The CSR of an edge array (the construction step of load_edge_list) on the
 * GPU: edges stably grouped by source, parallel edges kept.  src, dst and
 * weights (4-byte values of weight_kind, or NULL) on host or device.  An id
 * >= num_vertices fails with HYT_E_INVALID naming the edge. */
int hyt_csr_from_edges(const uint32_t *src, const uint32_t *dst, const void *weights, uint32_t weight_kind,
                       uint64_t num_edges, uint64_t num_vertices, int on_device, hyt_csr_buffers *out,
                       hyt_load_stats *stats);

/* Binary CSR file (no counterpart in the reference, which reads text only).
 * Layout, little-endian: a 64-byte header (magic "HYTCSR01", u32 version 1,
 * u32 weight kind, u64 V, u64 E, u64 payload bytes, u64 payload checksum,
 * u64 header checksum, u64 0), then row offsets (8 (V+1) B), column ids
 * (4 E B) and weights (4 E B, when weighted), each padded to 8 bytes.  The
 * checksum is the wrapping sum over the payload's 64-bit words w_i of
 * splitmix64(w_i ^ (i * 0x9E3779B97F4A7C15)), so it is computed in
 * parallel.  hyt_csr_save writes `path` through a temporary file and a
 * rename; csr arrays on host or device. */
int hyt_csr_save(const char *path, const hyt_csr *csr);

/* Reads a file written by hyt_csr_save: the header, the sizes against the
 * file size, the payload checksum and the CSR structure (offsets from 0,
 * non-decreasing, ending at E; ids < V) are checked (HYT_E_INVALID names
 * the failed check; HYT_E_IO for a file that cannot be read).  on_device 1
 * streams the payload through pinned buffers into cudaMalloc'd arrays and
 * checks it on the GPU; 0 reads into malloc'd arrays and checks on host
 * threads. */
int hyt_csr_load(const char *path, int on_device, hyt_csr_buffers *out, hyt_load_stats *stats);

/* ------------------------------------------------------------------ */
/* Contribution-driven scheduling                                       */
/* ------------------------------------------------------------------ */

/* scheduling::ContributionSchedulingMetrics. */
typedef struct hyt_contribution_metrics {
    uint64_t input_item_count;
    uint64_t scheduled_item_count;
    uint64_t reordered_item_count;    /* positions whose item changed */
    uint64_t zero_contribution_count; /* |contribution| <= epsilon */
    double scheduling_overhead;       /* log2(n): the reference's model */
    uint64_t stale_work_count;        /* 0 here (observations are host-side) */
    uint64_t redundant_work_count;    /* repeated item indices */
} hyt_contribution_metrics;

/* algorithms::pagerank_contributions (src/algorithms/pagerank.cpp:165-241)
 * on an in-HBM graph (HYT_GRAPH_PULL): contributions[v] = |next(v) -
 * current(v)| of one synchronous pull step, sums in FP64 (the reference
 * sums in FP32; the two agree to its rounding).  current_ranks [V] and
 * contributions [V]: host or device. */
int hyt_pagerank_contributions(hyt_graph *graph, const float *current_ranks, float damping,
                               double *contributions);

/* algorithms::sssp_contributions (src/algorithms/sssp.cpp:236-290) on the
 * GPU, bit for bit: current - candidate when both are finite and the
 * improvement exceeds the tolerance, 1 when an unreachable vertex becomes
 * reachable, else 0.  Arrays of n: host or device. */
int hyt_sssp_contributions(const float *current_distances, const float *candidate_distances, uint64_t n,
                           float tolerance, double *contributions);

/* scheduling::ContributionScheduler::schedule
 * (src/scheduling/contribution_scheduler.cpp:23-121) on the GPU: items by
 * descending contribution; ties by lower item index when
 * deterministic_tie_break, else in input order; a non-finite contribution
 * fails with HYT_E_INVALID.  ordered_items [n]: host or device. */
int hyt_contribution_schedule(const uint64_t *item_indices, const double *contributions, uint64_t n,
                              int deterministic_tie_break, double zero_contribution_epsilon,
                              uint64_t *ordered_items, hyt_contribution_metrics *metrics);

/* Per-partition priorities for the transfer queue: out[i] = sum of
 * vertex_contributions over [bounds[i], bounds[i + 1]).  Arrays: host or
 * device. */
int hyt_partition_contributions(const double *vertex_contributions, uint64_t num_vertices, const uint64_t *bounds,
                                uint64_t num_partitions, double *out);

/* ---- Measured peaks ------------------------------------------------------
 * The denominators of the path's rooflines, measured on `device`: a
 * device-to-device copy of copy_bytes (0: 1 GiB; read + write bytes over
 * time), pinned host<->device copies and kernel reads of mapped pinned host
 * memory (min(copy_bytes, 256 MiB) each), best of several repetitions.
 * Needs 2 x copy_bytes of free device memory (else HYT_E_OOM).  The
 * reference has no counterpart (its cost model uses fixed placeholders:
 * src/transfer/hytm_cost_model.cpp). */
typedef struct hyt_peaks {
    double hbm_copy_gbs;   /* device-to-device copy, GB/s */
    double h2d_gbs;        /* pinned host -> device, GB/s */
    double d2h_gbs;        /* device -> pinned host, GB/s */
    double zero_copy_gbs;  /* kernel reads of mapped pinned host memory, GB/s */
    uint64_t hbm_bytes;    /* device memory */
    uint64_t l2_bytes;
    uint64_t copy_bytes;   /* bytes per device copy timed */
    uint64_t link_bytes;   /* bytes per host-link copy timed */
    uint32_t sm_count;
    uint32_t mem_bus_bits;
} hyt_peaks;
int hyt_measure_peaks(int device, uint64_t copy_bytes, hyt_peaks *out);

/* ---- Vertex-range shards: one process per GPU ----------------------------
 *
 * Every process creates the same graph (same CSR, same flags) on its own GPU
 * and takes one contiguous range of internal vertex ids.  A PageRank step
 * computes the rank of the range's rows; an SSSP round expands the range's
 * improved vertices.  Between steps the caller exchanges the whole-graph
 * vectors with its collective library (hytgraph_b200.shard drives this with
 * torch.distributed over NCCL): PageRank broadcasts each owner's slice of
 * the contribution vector and sums two doubles; SSSP min-reduces the key
 * vector.  The vectors are caller-owned device memory, so collectives write
 * them in place.  The reference runs on one GPU; there is no reference
 * interface for this part.  A shard borrows its graph (destroy shards
 * first) and, like the graph's own solvers, runs one solve at a time. */
#define HYT_SHARD_PULL 1u /* PageRank / personalized PageRank over CSC rows */
#define HYT_SHARD_PUSH 2u /* SSSP over CSR rows */

typedef struct hyt_shard hyt_shard;

/* Cuts the internal vertex ids into `parts` contiguous ranges of balanced
 * work (rows + in-edges for PULL, rows + out-edges for PUSH); PULL cuts fall
 * on PageRank row tiles.  bounds[parts + 1], host.  Deterministic: every
 * process holding the same graph gets the same bounds. */
int hyt_shard_bounds(hyt_graph *graph, uint32_t kind, uint32_t parts, uint32_t *bounds);
/* Shard `part` of `bounds` (PULL bounds must come from hyt_shard_bounds). */
int hyt_shard_create(hyt_graph *graph, uint32_t kind, const uint32_t *bounds, uint32_t parts, uint32_t part,
                     hyt_shard **out);
int hyt_shard_destroy(hyt_shard *shard);

typedef struct hyt_shard_info {
    uint32_t kind, part, parts;
    uint32_t vertex_begin, vertex_end; /* internal ids [begin, end) */
    uint32_t pad;
    uint64_t num_vertices;  /* of the whole graph */
    uint64_t edges;         /* in-edges (PULL) / out-edges (PUSH) of the range's rows */
    uint64_t tasks;         /* PULL: tile + chunk tasks of one step */
    uint64_t edges_relaxed; /* PUSH: out-edges expanded since the last init */
} hyt_shard_info;
int hyt_shard_get_info(hyt_shard *shard, hyt_shard_info *out);

typedef struct hyt_shard_pagerank {
    float *rank[2];    /* device [V]: the iterate, by parity of the iteration */
    float *contrib[2]; /* device [V]: rank / out-degree (0 for dangling vertices) */
    double *sums;      /* device [2]: L1 change and dangling mass of the range's rows */
    float damping;     /* PageRank damping; personalized PageRank: 1 - restart */
    uint32_t personalized;
    uint32_t source;   /* personalized: the caller's vertex id */
    uint32_t pad;
    void *stream;      /* NULL: the graph's stream */
} hyt_shard_pagerank;

/* The initial iterate of EVERY vertex into rank[0] / contrib[0] (1/n, or
 * the source indicator); sums = {0, dangling mass of the range's rows}. */
int hyt_shard_pagerank_init(hyt_shard *shard, const hyt_shard_pagerank *args);
/* Step `iteration` (0-based) of pagerank_gpu's synchronous pull
 * (src/algorithms/pagerank.cpp:89-163) over the range's rows: reads
 * rank/contrib[iteration & 1] (every vertex current), writes
 * rank/contrib[(iteration + 1) & 1] at the range's rows, and sets sums to
 * the range's L1 change and new dangling mass.  `dangling` = the whole
 * graph's dangling mass of the iterate read.  Asynchronous on the stream. */
int hyt_shard_pagerank_step(hyt_shard *shard, const hyt_shard_pagerank *args, uint32_t iteration,
                            double dangling);

typedef struct hyt_shard_sssp {
    int32_t *keys;    /* device [V + 1]: label XOR 0x80000000 as int32 (signed order = label order); [V] = idle flag */
    uint32_t source;  /* the caller's vertex id */
    uint32_t pad;
    void *stream;     /* NULL: the graph's stream */
    int64_t *frontier_edges; /* device [1] or NULL: out-edges of the round's frontier, summed over shards by the caller */
} hyt_shard_sssp;

/* keys: every label infinite (HYT_DIST_INF_U32, +inf bits for F32 weights)
 * except the source's 0; the shard forgets what it expanded. */
int hyt_shard_sssp_init(hyt_shard *shard, const hyt_shard_sssp *args);
/* One round, in two calls around one small exchange:
 *   hyt_shard_sssp_collect: the owned vertices whose label dropped since
 *     their last expansion form this shard's frontier; their out-edge count
 *     goes to *frontier_edges;
 *   (caller: sum-reduce frontier_edges over all shards)
 *   hyt_shard_sssp_relax: when the summed count exceeds E / 4 every shard
 *     runs a pull sweep over its rows of the PULL bounds (graphs created
 *     with PULL as well), else it pushes its frontier's out-edges into keys
 *     (atomic min); keys[V] = 1 when this shard's frontier was empty, else 0.
 * The caller then min-reduces keys[0..V] over all shards and stops when
 * keys[V] is 1.  Without frontier_edges a shard decides alone, which only
 * a single shard may do (with several, relax then never sweeps).
 * hyt_shard_sssp_round = collect + relax, deciding alone.  Asynchronous on
 * the stream. */
int hyt_shard_sssp_collect(hyt_shard *shard, const hyt_shard_sssp *args);
int hyt_shard_sssp_relax(hyt_shard *shard, const hyt_shard_sssp *args);
int hyt_shard_sssp_round(hyt_shard *shard, const hyt_shard_sssp *args);
/* u32 labels (caller's vertex order) of keys[0..V) into out [V]: host or device. */
int hyt_shard_sssp_labels(hyt_shard *shard, const int32_t *keys, uint32_t *out, void *stream);
/* V 4-byte values in internal order (device) into out [V] in the caller's
 * vertex order: host or device. */
int hyt_shard_emit(hyt_shard *shard, const void *values, void *out, void *stream);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* HYT_CAPI_H */

// Entry points of the device solvers (called from capi.cu).
#pragma once

#include "graph.cuh"

namespace hyt {

void pagerank_run(GraphImpl &g, const hyt_pagerank_params &p, float *ranks_out, hyt_run_stats *stats);
void ppr_run(GraphImpl &g, const hyt_ppr_params &p, float *ranks_out, hyt_run_stats *stats);
void ppr_multi(GraphImpl &g, const uint32_t *sources, uint32_t k, float restart, float tolerance, uint32_t max_iter,
               float *out, hyt_run_stats *stats);
void sssp_run(GraphImpl &g, const hyt_sssp_params &p, uint32_t *dist_out, hyt_run_stats *stats);
void sssp_multi(GraphImpl &g, const uint32_t *sources, uint32_t k, uint32_t max_rounds, uint32_t flags,
                cudaStream_t s, uint32_t *out, hyt_run_stats *stats);
void sssp_noalloc(const hyt_csr &csr, uint32_t source, uint32_t *dist_out, void *stream, hyt_run_stats *stats);

void rmat_generate(const hyt_rmat_params &p, bool on_device, hyt_csr_buffers *out);
void pick_sources(const uint64_t *row_offsets, uint64_t V, uint64_t seed, uint32_t count, uint32_t *out);

// Hub sorting / vertex reordering (reorder.cu).
void hub_sort(const hyt_csr &csr, double fraction, uint32_t *order_out, double *scores_out, uint64_t *hub_count,
              hyt_reorder_stats *stats);
// pooled (with on_device): the outputs come from the graph pool and are
// released with free_pooled_buffers, not hyt_csr_buffers_free.
void csr_reorder(const hyt_csr &csr, const uint32_t *vertex_order, bool on_device, hyt_csr_buffers *out,
                 hyt_reorder_stats *stats, bool pooled = false);
void free_pooled_buffers(hyt_csr_buffers *b);
void csr_from_edges(const uint32_t *src, const uint32_t *dst, const void *weights, uint32_t wkind, uint64_t E,
                    uint64_t V, bool on_device, hyt_csr_buffers *out, hyt_load_stats *stats);
void load_edge_list(const char *path, uint64_t V, bool weighted, bool on_device, hyt_csr_buffers *out,
                    hyt_load_stats *stats);
void csr_save(const char *path, const hyt_csr &csr);
void pagerank_contributions(GraphImpl &g, const float *ranks, float damping, double *out, double *device_ms);
void sssp_contributions(const float *cur, const float *cand, uint64_t n, float tol, double *out);
void contribution_schedule(const uint64_t *item, const double *contribution, uint64_t n, bool deterministic,
                           double eps, uint64_t *ordered, hyt_contribution_metrics *m);
void partition_contributions(const double *contrib, uint64_t V, const uint64_t *bounds, uint64_t parts, double *out);
void csr_load(const char *path, bool on_device, hyt_csr_buffers *out, hyt_load_stats *stats);

}  // namespace hyt

/* oracle.h -- CPU restatement of the reference algorithms (test
 * infrastructure only; see oracle.c). */
#ifndef HYT_ORACLE_H
#define HYT_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORACLE_OK = 0, ORACLE_E_INVALID = 1, ORACLE_E_NOMEM = 2 };
enum { ORACLE_ENGINE_FILTER = 0, ORACLE_ENGINE_COMPACTION = 1, ORACLE_ENGINE_ZERO_COPY = 2 };

int oracle_pagerank_f32(uint64_t V, uint64_t E, const uint64_t *off, const uint32_t *cols, float damping,
                        float tol, uint64_t max_iter, float *ranks, uint64_t *iterations, float *residual,
                        int *converged);
int oracle_pagerank_f64(uint64_t V, uint64_t E, const uint64_t *off, const uint32_t *cols, double damping,
                        double tol, uint64_t max_iter, double *ranks, uint64_t *iterations, double *residual,
                        int *converged);
int oracle_pagerank_f64_csc(uint64_t V, const uint64_t *off, const uint64_t *in_off, const uint32_t *in_src,
                            double damping, double tol, uint64_t max_iter, double *ranks, uint64_t *iterations,
                            double *residual, int *converged);
int oracle_ppr_f64(uint64_t V, uint64_t E, const uint64_t *off, const uint32_t *cols, uint32_t source,
                   double restart, double tol, uint64_t max_iter, double *ranks, uint64_t *iterations,
                   double *residual, int *converged);
int oracle_sssp(uint64_t V, uint64_t E, const uint64_t *off, const uint32_t *cols, const float *weights,
                uint32_t source, uint64_t max_iter, float *dist, uint64_t *iterations, int *converged);
int oracle_dijkstra_u32(uint64_t V, uint64_t E, const uint64_t *off, const uint32_t *cols, const uint32_t *weights,
                        uint32_t source, uint64_t *dist);
/* Seeded R-MAT CSR (malloc'd arrays, release with oracle_free; *w_out NULL
 * when wmin == wmax == 0) and seeded source vertices. */
int oracle_rmat(uint32_t scale, uint32_t edge_factor, uint64_t seed, double a, double b, double c, uint32_t wmin,
                uint32_t wmax, uint64_t **off_out, uint32_t **cols_out, uint32_t **w_out, uint64_t *E_out);
void oracle_free(void *p);
int oracle_pick_sources(const uint64_t *off, uint64_t V, uint64_t seed, uint32_t count, uint32_t *out);

typedef struct {
    double alpha, beta, gamma, rtt, cpu_throughput;
    uint64_t m, mr, d1, d2, align;
} oracle_hytm_options;

typedef struct {
    uint64_t active_vertices, active_edges, total_edges;
    uint64_t filter_bytes, compaction_bytes, zc_requests, zc_alignment;
    double filter_cost, compaction_cost, zero_copy_cost, zc_rtt;
    int engine;
} oracle_hytm_costs;

void oracle_hytm_partition(const uint64_t *off, const unsigned char *active, uint32_t vbegin, uint32_t vend,
                           const oracle_hytm_options *o, oracle_hytm_costs *c);
int oracle_select_engine(double f, double c, double z, double alpha, double beta);
uint64_t oracle_task_combine(const int *engines, uint64_t n, uint64_t k, uint64_t *task_of_partition,
                             int *task_engine, uint64_t *task_first);
int oracle_hub_sort(uint64_t V, uint64_t E, const uint64_t *off, const uint32_t *cols, double fraction,
                    uint32_t *order, double *scores, uint64_t *hub_count);
int oracle_load_edge_list(const char *path, uint64_t V, int weighted, uint64_t *E_out, uint64_t *err_line);
void oracle_loaded_copy(uint64_t *off, uint32_t *cols, float *w);
void oracle_loaded_free(void);
uint64_t oracle_csr_from_edges(uint64_t V, uint64_t E, const uint32_t *src, const uint32_t *dst, const uint32_t *w,
                               uint64_t *off, uint32_t *cols, uint32_t *w_out);
int oracle_pagerank_contributions(uint64_t V, uint64_t E, const uint64_t *off, const uint32_t *cols,
                                  const float *cur, float damping, int fp64, double *out);
void oracle_sssp_contributions(uint64_t n, const float *cur, const float *cand, float tol, double *out);
int oracle_contribution_schedule(uint64_t n, const uint64_t *item, const double *c, int det, double eps,
                                 uint64_t *ordered, uint64_t *metrics);
int oracle_reorder(uint64_t V, uint64_t E, const uint64_t *off, const uint32_t *cols, const uint32_t *w,
                   const uint32_t *order, uint64_t *off_out, uint32_t *cols_out, uint32_t *w_out);

#ifdef __cplusplus
}
#endif

#endif

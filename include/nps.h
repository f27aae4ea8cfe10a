/*
 * nps.h — C ABI of the B200-native single-source shortest path (SSSP) library
 * with warp / block / grid workload consolidation.
 *
 * Every entry point is `extern "C"`, takes plain pointers and sizes, returns an
 * `nps_status` (0 = success) and never calls exit().  The message of the last
 * failure on the calling thread is available from nps_last_error_string().
 *
 * Reference interfaces replaced (paths relative to the dadaism/nested-parallelism
 * source tree):
 *   nps_sssp / nps_sssp_ctx   replace  void sssp_np_consolidate_gpu(void)
 *                                       apps/sssp/src/gpu/sssp_wrapper.cu:475-546
 *                             together with the per-run set-up and tear-down
 *                             prepare_gpu() / clean_gpu() / SSSP_GPU()
 *                                       apps/sssp/src/gpu/sssp_wrapper.cu:58-149, :548-583
 *   nps_sssp_state            replaces the global-state form of the same call: it
 *                             starts from a caller-supplied cost array and update
 *                             flags exactly as sssp_np_consolidate_gpu() starts from
 *                             d_costArray / d_update (sssp_wrapper.cu:22-30, :92-113)
 *   nps_sssp_batch            has no single counterpart: it runs many independent
 *                             SSSP_GPU() calls (apps/sssp/src/gpu/sssp.cpp:140-142)
 *                             in one persistent launch
 *   nps_read_dimacs9 / _dimacs10 / _slndc
 *                             replace readInputDIMACS9/10/SLNDC() + convertCSR()
 *                                       common/global.cpp:29-64, :66-105, :107-190, :192-235
 *   nps_sssp_solution(_state) replace cases 0-5 of SSSP_GPU()'s switch (sssp_tqueue_gpu ...
 *                             sssp_np_opt_gpu)      apps/sssp/src/gpu/sssp_wrapper.cu:151-473
 *   nps_bfs                   replaces void bfs_rec_dp_cons_gpu(void), the bfs-rec
 *                             application's consolidated BFS on the same engine
 *                                       apps/bfs-rec/src/gpu/bfs_rec_wrapper.cu:170-229
 *   nps_spmv                  replaces void spmv_np_consolidate_gpu(void), the SpMV
 *                             application's consolidated kernel
 *                                       apps/SpMV/src/gpu/SpMV_wrapper.cu:285-311
 *   nps_bc                    replaces void bc_np_consolidate_gpu(void), the bc
 *                             application's betweenness centrality
 *                                       apps/bc/src/gpu/bc_wrapper.cu:678-741
 *   nps_color                 replaces void gclr_np_consolidate_gpu(void), the
 *                             graph-color application's coloring
 *                                       apps/graph-color/src/gpu/graph_color_wrapper.cu:368-412
 *   nps_degree_stats          replaces the graph analyzer's getStatInfo()
 *                                       utility/graph-analyzer/analyzer.cpp:75-138
 *   nps_graph                 replaces struct _GRAPH_'s CSR members and the
 *                             noNodeTotal / noEdgeTotal / source globals
 *                                       common/global.h:28-58
 *
 * Distances are uint32 with the reference's INF = 2^30 (apps/sssp/src/gpu/
 * sssp_wrapper.cu:7) for unreachable vertices; a path whose length reaches 2^30
 * is treated as unreachable, the same sentinel the reference uses.
 */
#ifndef NPS_H_
#define NPS_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NPS_INF 0x40000000u  /* 1<<30, apps/sssp/src/gpu/sssp_wrapper.cu:7 */
#define NPS_ABI_VERSION 3

typedef int32_t nps_status;
enum {
  NPS_OK = 0,
  NPS_ERR_INVALID_ARG = 1,   /* bad size, pointer, source or parameter */
  NPS_ERR_CUDA = 2,          /* a CUDA runtime call failed */
  NPS_ERR_CAPACITY = 3,      /* a device queue would have overflowed */
  NPS_ERR_TIMEOUT = 4,       /* a bounded spin wait in the persistent kernel ran out */
  NPS_ERR_NO_DEVICE = 5,     /* no CUDA device / wrong architecture */
  NPS_ERR_IO = 6,            /* file could not be opened or parsed */
  NPS_ERR_FORMAT = 7,        /* malformed CSR or input file */
  NPS_ERR_OOM = 8,           /* host or device allocation failed */
  NPS_ERR_INTERNAL = 9       /* the CTAs of a persistent kernel took different schedule decisions */
};

/* Consolidation granularity for vertices whose out-degree is at least
 * `threshold` (the reference's THRESHOLD, apps/sssp/src/gpu/sssp_kernel.cu:7).
 * Values 0..2 are the reference's CONSOLIDATE_LEVEL (sssp_wrapper.cu:503-531). */
enum {
  NPS_LEVEL_WARP = 0,   /* per-warp buffer, processed by that warp           (consolidate_warp_dp_kernel,  sssp_kernel.cu:330) */
  NPS_LEVEL_BLOCK = 1,  /* per-CTA buffer in shared memory, processed by it  (consolidate_block_dp_kernel, sssp_kernel.cu:407) */
  NPS_LEVEL_GRID = 2,   /* one device-wide buffer, processed by every CTA    (consolidate_grid_dp_kernel,  sssp_kernel.cu:484) */
  NPS_LEVEL_HYBRID = 3  /* degree ranges [threshold,block_threshold) warp, [block_threshold,grid_threshold) block, rest grid */
};

enum {
  NPS_POLICY_PLAIN = 0,    /* fixed delta and level from nps_params */
  NPS_POLICY_LEARNED = 1   /* bucket widths (first from the start state, then at each advance) and the level of
                              every iteration from the MLP loaded with nps_policy_set_weights; error if none */
};

/* The learned policy runs only on graphs of at least this many edges (unless
 * nps_params.policy_min_edges says otherwise); smaller ones run the plain kernel with
 * the same parameters (stats.policy_used says which).
 * Measured on held-out R-MAT graphs at edge factor 16 with the shipped weights: up
 * to scale 16 (1 M edges) the policy's per-iteration cost outweighs what its bucket
 * widths save (0.85-0.97x), at scale 17 it breaks even (1.02-1.05x), from scale 18
 * (4 M edges) the widths win (18: 1.10-1.13x, 19: 1.18-1.22x, 22: 1.5x). */
#define NPS_POLICY_MIN_EDGES 3000000

typedef struct nps_params {
  int32_t level;            /* NPS_LEVEL_* (default NPS_LEVEL_BLOCK, the reference Makefile's CONSOLIDATE_LEVEL=1) */
  int32_t threshold;        /* degree at which a vertex is consolidated (default 64) */
  int32_t block_threshold;  /* NPS_LEVEL_HYBRID only */
  int32_t grid_threshold;   /* NPS_LEVEL_HYBRID only */
  int32_t block_size;       /* threads per CTA: 128, 256 or 512 (default 256) */
  int32_t ctas_per_sm;      /* resident CTAs per SM; 0 = as many as fit */
  uint32_t delta;           /* near-far bucket width; 0 = unordered frontier (the reference's order) */
  int32_t policy;           /* NPS_POLICY_* */
  int32_t device_ptrs;      /* 1: graph and dist pointers are device pointers; 0: host pointers */
  int32_t device;           /* CUDA device ordinal */
  void* stream;             /* cudaStream_t to launch on; NULL = the library's own stream */
  double timeout_s;         /* bound on every spin wait inside the persistent kernel (default 10 s) */
  int32_t trace;            /* 1: record one nps_trace_rec per iteration (read with nps_trace_read) */
  int32_t light_heavy;      /* 1 (default): with delta > 0, edges of weight >= delta are relaxed once,
                               when the bucket that settles their tail drains (Meyer-Sanders split) */
  int32_t local_rounds;     /* rounds a warp spends on the vertices it just improved before taking
                               new work (0 = none): frontiers advance several hops per barrier */
  int32_t order_degree;     /* with delta > 0: an improved vertex whose out-degree is below this
                               joins the current bucket whatever its distance, so only rows of at
                               least this degree wait for their bucket (0 = every vertex waits) */
  uint32_t delta_schedule;  /* 0: every bucket is delta wide.  Otherwise bucket b (0 = the first)
                               is 2^k wide with k = bits [4b, 4b+4) for b < 7 and bits [28, 32)
                               for every later bucket; delta is then unused (plain policy only) */
  int32_t reserved[2];      /* reserved[0] = 1: test hook, the first in-kernel barrier (of the SSSP
                               kernel, or of nps_color's round kernel) waits for an arrival that
                               never comes, so its bounded wait must expire.
                               reserved[0] = 2: test hook, CTA 1 of the SSSP kernel reports another
                               hash for its first schedule decision, so the agreement check must
                               end the run with NPS_ERR_INTERNAL.
                               reserved[1] > 0: nps_bc folds at most this many sources per block
                               of dependency rows (0 = as many as 2 GB of rows hold) */
  int32_t schedule;         /* NPS_SCHEDULE_* (default NPS_SCHEDULE_ITERATIONS) */
  int64_t policy_min_edges; /* NPS_POLICY_LEARNED runs only on graphs of at least this many edges,
                               smaller ones run the plain kernel; 0 (default) = NPS_POLICY_MIN_EDGES,
                               negative = no minimum */
  int32_t sort_at_push;     /* iteration schedule: rows of at least the grid threshold that a warp pushes
                               into the near queue join the grid-tier list when the warp flushes its
                               pushes (walked the next iteration; otherwise they are sorted when taken
                               from the queue and walked one iteration later).  1 = on, -1 = off,
                               0 (default) = on when the grid threshold in effect is at most
                               NPS_SORT_AT_PUSH_AUTO_MAX edges and the edges have weights (off for
                               nps_bfs, where every reached row is walked once anyway: R-MAT 22
                               BFS takes 0.645 ms with it off, 0.682 ms with it on) */
  int32_t reserved2;        /* must be 0 */
} nps_params;

/* sort_at_push = 0 sorts at push time when the grid threshold is at most this: the flush
 * reads row_ptr of every pushed vertex, which pays when many of them are grid-tier rows
 * (R-MAT 22 at threshold 32: 23 -> 15 iterations) and costs when few are (a batch of
 * scale 12-18 graphs at a hybrid grid threshold of 4096: 2.65 -> 2.98 ms). */
#define NPS_SORT_AT_PUSH_AUTO_MAX 256

/* How the persistent SSSP kernel moves from one frontier to the next. */
enum {
  NPS_SCHEDULE_ITERATIONS = 0,  /* frontier iterations separated by a team barrier (every level, batches) */
  NPS_SCHEDULE_ASYNC = 1        /* single-instance calls at NPS_LEVEL_GRID without light/heavy split or
                                   local rounds: inside a bucket, improved vertices and 256-edge segments
                                   of rows of >= threshold edges go to device work rings that every warp
                                   drains as work appears; the team meets only at bucket advances.  The
                                   learned policy then picks a width at each advance (stats = iterations
                                   = buckets); other parameter sets run the iteration schedule */
};

typedef struct nps_stats {
  uint32_t iterations;      /* frontier iterations (the reference's `iteration` global) */
  uint32_t buckets;         /* near-far bucket advances */
  uint64_t edges_scanned;   /* edge relaxations attempted */
  uint64_t improvements;    /* successful atomicMin relaxations */
  uint64_t vertices_processed;
  uint32_t reached;         /* vertices with a finite distance */
  uint32_t policy_used;     /* NPS_POLICY_* the run used (NPS_POLICY_PLAIN when the learned policy was
                               asked for on a graph below NPS_POLICY_MIN_EDGES edges) */
  uint64_t reached_edges;   /* out-edges of reached vertices (m_r) */
  float kernel_ms;          /* device time of the persistent launch (CUDA events); per instance of a
                               batch: device time from the launch to the end of that instance's solve */
  float total_ms;           /* device time including copies done by the call */
  int32_t status;           /* device status word */
  int32_t grid_ctas;        /* CTAs in the persistent launch */
  /* SM cycles summed over warps per phase of the persistent loop; filled only by
   * a library built with -DNPS_PROFILE (zero otherwise):
   * 0 work-item fetch, 1 vertex loads + classification, 2 small-row rounds,
   * 3 warp-tier rows, 4 grid-tier chunk walk, 5 block-tier walk, 6 staging drain,
   * 7 team barrier, 8 iteration bookkeeping */
  uint64_t phase_cycles[9];
} nps_stats;

/* One record per frontier iteration when nps_params.trace = 1. */
typedef struct nps_trace_rec {
  uint32_t iteration;
  uint32_t frontier;        /* near-queue length processed */
  uint32_t far_len;         /* far-pile length after the iteration */
  uint32_t bucket_hi;       /* current bucket upper bound T */
  uint32_t delta;
  uint32_t level;
  uint32_t hist[8];         /* frontier out-degree histogram, bins [4^k-1, 4^(k+1)-1) */
  uint64_t edges;           /* edges scanned in the iteration */
  uint64_t improvements;
  uint32_t reached;         /* vertices reached so far */
  uint32_t heavy;           /* grid-tier rows collected for the next iteration */
  uint64_t t_ns;            /* device time since the launch began, at the end of the iteration */
  float feat[12];           /* the learned policy's input features after this iteration (raw) */
} nps_trace_rec;

/* Host-side CSR graph, library-allocated; free with nps_graph_free. */
typedef struct nps_graph {
  int32_t n;
  int32_t source;          /* suggested source: DIMACS9 's' line, 0 otherwise, or the generator's pick */
  int64_t m;
  int32_t* row_ptr;        /* n+1 (graph.vertexArray) */
  int32_t* col;            /* m   (graph.edgeArray)   */
  uint32_t* w;             /* m   (graph.weightArray) */
} nps_graph;

typedef struct nps_ctx nps_ctx;

/* ---- library ---------------------------------------------------------- */
int32_t nps_abi_version(void);
const char* nps_last_error_string(void);
void nps_params_default(nps_params* p);

/* ---- graph construction (host) ----------------------------------------- */
/* Uniform random directed multigraph: each edge draws src and dst uniformly
 * (self-loops redrawn), weight uniform in [1,wmax]. */
nps_status nps_gen_uniform(int32_t n, int64_t m, uint32_t wmax, uint64_t seed, nps_graph* out);
/* R-MAT (no noise), duplicates and self-loops removed; source = highest
 * out-degree vertex (lowest id on ties). */
nps_status nps_gen_rmat(int32_t scale, int32_t edge_factor, double a, double b, double c,
                        uint32_t wmax, uint64_t seed, nps_graph* out);
/* rows x cols 4-neighbour grid, each undirected pair dropped with probability
 * drop, independent weights per direction in [1,wmax]; source = vertex 0. */
nps_status nps_gen_grid(int32_t rows, int32_t cols, double drop, uint32_t wmax, uint64_t seed,
                        nps_graph* out);
/* CSR from an edge list in insertion order; rows keep the reverse insertion
 * order of convertCSR (common/global.cpp:211-225). dedupe=1 keeps the first
 * of each (src,dst) pair; self-loops are dropped when drop_self_loops=1. */
nps_status nps_csr_from_edges(int32_t n, int64_t m, const int32_t* src, const int32_t* dst,
                              const uint32_t* w, int32_t dedupe, int32_t drop_self_loops,
                              nps_graph* out);
void nps_graph_free(nps_graph* g);
/* FNV-1a 64 over n uint32 values (distance-array fingerprint). */
uint64_t nps_fnv1a_u32(const uint32_t* a, int64_t n);

/* ---- file front-ends: readInput*() + convertCSR() ----------------------- */
nps_status nps_read_dimacs9(const char* path, nps_graph* out);   /* global.cpp:29-64  */
nps_status nps_read_dimacs10(const char* path, nps_graph* out);  /* global.cpp:66-105 */
nps_status nps_read_slndc(const char* path, nps_graph* out);     /* global.cpp:107-190 */
nps_status nps_write_dimacs9(const char* path, const nps_graph* g, int32_t source);

/* ---- SSSP --------------------------------------------------------------- */
/* Single source.  row_ptr[n+1], col[m], w[m]; dist_out[n] receives distances
 * (NPS_INF = unreachable).  Pointers are host or device per p->device_ptrs.
 * Uses a per-device default context.  p may be NULL (defaults).
 * Host pointers: the CSR is copied to a cached device workspace on every call and
 * the distances copied back (pinned host buffers copy fastest).  On graphs of at
 * least 2^20 edges whose largest weight fits in 8 or 16 bits, the weights cross
 * PCIe packed (one host pass with OpenMP threads, overlapped with the column copy)
 * and are widened on the device; the context keeps a pinned staging buffer of
 * 2 bytes per edge for this. */
nps_status nps_sssp(const int32_t* row_ptr, const int32_t* col, const uint32_t* w, int32_t n,
                    int64_t m, int32_t src, const nps_params* p, uint32_t* dist_out,
                    nps_stats* st);

/* Same, through an explicit context (its own stream and cached workspace). */
nps_status nps_ctx_create(int32_t device, nps_ctx** out);
nps_status nps_ctx_destroy(nps_ctx* ctx);
nps_status nps_sssp_ctx(nps_ctx* ctx, const int32_t* row_ptr, const int32_t* col,
                        const uint32_t* w, int32_t n, int64_t m, int32_t src,
                        const nps_params* p, uint32_t* dist_out, nps_stats* st);

/* Start from an existing state, as sssp_np_consolidate_gpu() does: cost[n] holds
 * the initial distances and is updated in place; every vertex with update[v] != 0
 * is in the initial frontier; update[] is cleared on return.  Device pointers only. */
nps_status nps_sssp_state(const int32_t* d_row_ptr, const int32_t* d_col, const uint32_t* d_w,
                          int32_t n, int64_t m, uint32_t* d_cost, uint8_t* d_update,
                          const nps_params* p, nps_stats* st);

/* Copy the per-iteration trace of the last traced call on this thread's default
 * context for `device` (at most cap records); returns the record count in *count. */
nps_status nps_trace_read(int32_t device, nps_trace_rec* out, int32_t cap, int32_t* count);

/* ---- SSSP without allocation ---------------------------------------------
 * No counterpart in the reference.  For callers that must not allocate device
 * memory during the call (a service whose memory is all reserved in its own
 * pool, a host that forbids allocator calls from callbacks): same result as
 * nps_sssp with device pointers, but the kernel's workspace is a file-scope
 * static __device__ array of NPS_NOALLOC_SCRATCH_BYTES (10 MiB) that every GPU
 * loading libnps holds until exit.
 * Limit: n <= NPS_NOALLOC_MAX_VERTICES (larger graphs get NPS_ERR_CAPACITY).
 * The call synchronises its stream to return a status; on a stream that is being
 * captured it returns NPS_ERR_INVALID_ARG.  The first call on a device resolves
 * the array's device address (cudaGetSymbolAddress, that device current) and
 * caches it (again after a cudaDeviceReset() of that device): make that first call
 * before any stream capture begins.  Calls share the array and it keeps the last
 * call's contents (what must start at zero is cleared on every call): calls whose
 * kernels overlap on the GPU race, so order them on one stream.  No trace, no
 * kernel_ms in the stats.
 * Device pointers only; p->stream selects the stream (NULL = legacy default). */
#define NPS_NOALLOC_MAX_VERTICES 131072
#define NPS_NOALLOC_SCRATCH_BYTES (10u << 20)
nps_status nps_sssp_noalloc(const int32_t* d_row_ptr, const int32_t* d_col, const uint32_t* d_w,
                            int32_t n, int64_t m, int32_t src, uint32_t* d_dist, const nps_params* p,
                            nps_stats* st);

/* ---- breadth-first levels ---------------------------------------------------
 * The bfs-rec application's consolidated BFS (bfs_rec_dp_cons_gpu,
 * apps/bfs-rec/src/gpu/bfs_rec_wrapper.cu:170-229) on the same persistent engine:
 * every edge weighs 1 and no weight array is read.  level_out[n] receives the hop
 * count from src, NPS_BFS_UNDEFINED for unreachable vertices (bfs_rec.h:13); the
 * result equals the reference's bfs_cpu (apps/bfs-rec/src/gpu/bfs_rec.cpp:100-119).
 * Arguments as nps_sssp.  With unit weights the unordered frontier (delta 0)
 * already advances one level per iteration; delta = 1 gives one bucket per level. */
#define NPS_BFS_UNDEFINED 0x7FFFFFFF
nps_status nps_bfs(const int32_t* row_ptr, const int32_t* col, int32_t n, int64_t m, int32_t src,
                   const nps_params* p, int32_t* level_out, nps_stats* st);

/* ---- sparse matrix-vector product ------------------------------------------
 * The SpMV application's consolidated kernel (spmv_np_consolidate_gpu,
 * apps/SpMV/src/gpu/SpMV_wrapper.cu:285-311): y[r] = sum of val[k] * x[col[k]]
 * over row r of the CSR matrix (row_ptr, col, val), in double precision
 * (FLOAT_T, apps/SpMV/src/gpu/SpMV.h:13); x and y have n entries.  Rows of at
 * least p->threshold nonzeros are consolidated at p->level (WARP, BLOCK or GRID;
 * HYBRID is rejected).  Each y[r] is summed in an order fixed by the matrix, so
 * results repeat exactly from run to run.  Pointers are host or device per
 * p->device_ptrs; uses p->device and p->stream.  st (may be NULL) gets
 * kernel_ms, total_ms, status and grid_ctas. */
nps_status nps_spmv(const int32_t* row_ptr, const int32_t* col, const double* val, const double* x,
                    double* y, int32_t n, int64_t m, const nps_params* p, nps_stats* st);

/* ---- betweenness centrality -----------------------------------------------
 * The bc application's consolidated kernels (bc_np_consolidate_gpu,
 * apps/bc/src/gpu/bc_wrapper.cu:678-741) with the result of its CPU version
 * bc_cpu (apps/bc/src/cpu/bc.cpp:152-186): Brandes' algorithm over the sources
 * sources[0..nsrc) in that order (every vertex in id order when sources is
 * NULL, as the reference does); bc_out[n] receives the float centralities,
 * bit-identical to bc_cpu for the same source order (a NaN from wrapped path
 * counts is a NaN on both, with a different payload).  One CTA per source; the
 * call holds about 16 n bytes per CTA of the grid plus up to 2 GB of per-source
 * dependency rows.  Pointers (sources included) are host or device per
 * p->device_ptrs; uses p->device and p->stream. */
nps_status nps_bc(const int32_t* row_ptr, const int32_t* col, int32_t n, int64_t m, const int32_t* sources,
                  int32_t nsrc, const nps_params* p, float* bc_out, nps_stats* st);

/* ---- graph coloring ---------------------------------------------------------
 * The graph-color application's consolidated coloring (gclr_np_consolidate_gpu,
 * apps/graph-color/src/gpu/graph_color_wrapper.cu:368-412): color_out[n]
 * receives the colors the reference's iterations assign, color(v) = 1 + the
 * largest color among v's out-neighbours with a smaller id (1 when there is
 * none); st->iterations = the largest color (the reference's iteration count).
 * Rows of at least p->threshold edges are scanned by a warp.  Pointers are host
 * or device per p->device_ptrs; uses p->device, p->stream and p->timeout_s. */
nps_status nps_color(const int32_t* row_ptr, const int32_t* col, int32_t n, int64_t m, const nps_params* p,
                     int32_t* color_out, nps_stats* st);

/* ---- the dispatcher's other solutions -------------------------------------
 * SSSP_GPU()'s `solution` switch (apps/sssp/src/gpu/sssp_wrapper.cu:548-583):
 * 0-5 are the reference's earlier load-balancing schemes (sssp_wrapper.cu:151-473,
 * kernels sssp_kernel.cu:34-327 and :626-658), kept for ablation against 6.  All
 * iterate the same unordered frontier (a queue rebuilt from per-vertex update
 * flags every iteration) and differ in how a queued row is mapped to threads;
 * rows of at least p->threshold edges are the "large" ones. */
enum {
  NPS_SOLUTION_TQUEUE = 0,          /* one thread walks each queued row (sssp_tqueue_gpu) */
  NPS_SOLUTION_DUAL_QUEUE = 1,      /* small rows by a thread, large rows by a 64-thread CTA each,
                                       from two queues (sssp_dual_queue_gpu) */
  NPS_SOLUTION_SHARED_DELAYED = 2,  /* large rows deferred to the CTA's shared buffer, then walked
                                       by the whole CTA (sssp_shared_delayed_buffer_gpu) */
  NPS_SOLUTION_GLOBAL_DELAYED = 3,  /* large rows deferred to one device buffer, walked by a second
                                       kernel, a 64-thread CTA per row (sssp_global_delayed_buffer_gpu) */
  NPS_SOLUTION_NP_NAIVE = 4,        /* one child grid per large row, device-side launch (sssp_np_naive_gpu) */
  NPS_SOLUTION_NP_OPT = 5,          /* one child grid per CTA over its large rows (sssp_np_opt_gpu) */
  NPS_SOLUTION_CONSOLIDATE = 6      /* workload consolidation: nps_sssp / nps_sssp_state */
};

typedef struct nps_solution_info {
  uint64_t deferred;          /* rows handed to a large-row path (high queue, buffer or child grid) */
  uint64_t child_launches;    /* device-side launches that started (solutions 4 and 5) */
  uint64_t launch_fallbacks;  /* device-side launches the runtime refused (pending-launch limit);
                                 the launching thread walked those rows itself */
  uint32_t host_reads;        /* times the host read the frontier size back */
  uint32_t pad;
} nps_solution_info;

/* Solution `solution` (0-6) from a source; arguments as nps_sssp.  p->threshold,
 * p->block_size (threads of the row-per-thread CTAs, a multiple of 32 in
 * [64, 1024]), device, stream, device_ptrs and timeout_s (wall-clock bound of
 * the whole call) apply to 0-5; 6 forwards to nps_sssp with all of p.  info may
 * be NULL. */
nps_status nps_sssp_solution(int32_t solution, const int32_t* row_ptr, const int32_t* col,
                             const uint32_t* w, int32_t n, int64_t m, int32_t src,
                             const nps_params* p, uint32_t* dist_out, nps_stats* st,
                             nps_solution_info* info);

/* The same from an existing state, as nps_sssp_state (device pointers only). */
nps_status nps_sssp_solution_state(int32_t solution, const int32_t* d_row_ptr, const int32_t* d_col,
                                   const uint32_t* d_w, int32_t n, int64_t m, uint32_t* d_cost,
                                   uint8_t* d_update, const nps_params* p, nps_stats* st,
                                   nps_solution_info* info);

/* ---- batched SSSP -------------------------------------------------------- */
typedef struct nps_instance {
  const int32_t* row_ptr;  /* device pointers */
  const int32_t* col;
  const uint32_t* w;
  uint32_t* dist;          /* device, n entries */
  int32_t n;
  int32_t src;
  int64_t m;
} nps_instance;

/* Run `count` independent instances in one persistent cooperative launch; CTAs
 * are split into teams (one team per group of instances, sized by edge count).
 * With use_graph = 1 the launch is captured into a CUDA graph on the first call
 * for this instance set and replayed on later calls with the same set. */
nps_status nps_sssp_batch(const nps_instance* inst, int32_t count, const nps_params* p,
                          int32_t use_graph, nps_stats* per_instance, float* kernel_ms);

/* ---- degree statistics ----------------------------------------------------
 * The reference's graph analyzer (utility/graph-analyzer/analyzer.cpp:75-138,
 * getStatInfo()) on the GPU, from the CSR row offsets: counts, total / average /
 * maximum / minimum out-degree with the lowest vertex id attaining each, and
 * optionally the degree distribution.  The minimum starts from the reference's
 * 999999 (a graph whose degrees are all at least that reports 999999 and node -1).
 * Also the 8-bin histogram [4^k - 1, 4^(k+1) - 1) of the policy's features. */
typedef struct nps_degree_info {
  int32_t n;                /* noNodeTotal */
  int32_t max_degree;
  int64_t m;                /* row_ptr[n] (noEdgeTotal) */
  int64_t total_degree;     /* sum of out-degrees */
  int64_t edges_by_degree;  /* total_degree / 2, the reference's "Edge by degree" */
  int32_t min_degree;
  int32_t max_degree_node;  /* lowest id with the maximum degree */
  int32_t min_degree_node;  /* lowest id with the minimum degree, -1 if none below 999999 */
  float avg_degree;         /* (float)total_degree / n, as the reference computes it */
  int64_t bins[8];
} nps_degree_info;
/* Synchronous, on the library's own stream of `device`.  dist (dist_len > 0):
 * vertices per degree 0..dist_len-1 (int64, host or device memory as flagged by
 * device_ptrs); NPS_ERR_CAPACITY, with info filled, when dist_len <= max_degree.
 * NPS_ERR_FORMAT when row_ptr decreases. */
nps_status nps_degree_stats(const int32_t* row_ptr, int32_t n, int32_t device_ptrs, int32_t device,
                            nps_degree_info* info, int64_t* dist, int64_t dist_len);

/* ---- learned policy (MLP 12 -> 32 -> 14) --------------------------------- */
#define NPS_MLP_IN 12
#define NPS_MLP_HID 32
#define NPS_MLP_OUT 14   /* 11 delta logits (2^0..2^10) + 3 level logits */
/* Load policy weights (fp32 in; stored on the device as bf16): W1[32x12], b1[32],
 * W2[14x32], b2[14], plus the 12 feature means and 12 inverse std devs. */
nps_status nps_policy_set_weights(int32_t device, const float* w1, const float* b1,
                                  const float* w2, const float* b2, const float* feat_mean,
                                  const float* feat_istd);
/* MLP training step kernels (device pointers, bf16 weights held as uint16 bits,
 * fp32 master copies and gradients). X[B x 12] fp32 features (already normalised),
 * label_delta[B] in 0..10, label_level[B] in 0..2, sample weight wt[B]. */
nps_status nps_mlp_forward(const uint16_t* w1, const float* b1, const uint16_t* w2,
                           const float* b2, const float* X, int32_t B, float* logits,
                           void* stream);
nps_status nps_mlp_loss_backward(const uint16_t* w1, const float* b1, const uint16_t* w2,
                                 const float* b2, const float* X, const int32_t* label_delta,
                                 const int32_t* label_level, const float* wt, int32_t B,
                                 float* g_w1, float* g_b1, float* g_w2, float* g_b2,
                                 float* loss, void* stream);
nps_status nps_mlp_adam_step(float* master, uint16_t* bf16_out, const float* grad, float* m1,
                             float* m2, int32_t count, float lr, float beta1, float beta2,
                             float eps, int32_t step, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* NPS_H_ */

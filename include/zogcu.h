/* zogcu.h -- C ABI of the B200 (sm_100a) centrality library.
 *
 * The library replaces, behind Zog's own NIF boundary, the two centrality hot
 * paths of code-shoily/zog that run on the `:soa` (ArrayGraph) resource:
 *
 *   - PageRank power iteration      priv/zog/src/centrality.zig:858-965
 *   - unweighted Brandes betweenness priv/zog/src/centrality.zig:687-798
 *
 * A graph handle holds a device-resident CSR built once from the NIF's edge
 * arrays and reused by every call, which is what the reference's GraphRes
 * resource does for its ArrayGraph (lib/zog/.Elixir.Zog.ResourceGraph.zig:10-24).
 *
 * Conventions
 *   - Every entry point returns a status code (ZOGCU_OK == 0); nothing throws
 *     across the ABI.  zogcu_status_string() names a code and
 *     zogcu_last_error() gives the calling thread's last detailed message.
 *   - Pointers are HOST pointers unless an option says otherwise.
 *   - Scores are returned exactly as the NIFs return them: one f64 per node
 *     slot (length = node capacity), 0.0 for deleted slots, and no undirected
 *     0.5 scaling (the Elixir wrapper applies that, resource_graph.ex:2633-2637).
 *   - Several host threads may call on the same graph at once; each call uses
 *     its own stream and workspace, and the graph itself is read-only after
 *     creation (one lazily built, mutex-guarded PageRank schedule aside).
 */
#ifndef ZOGCU_H_
#define ZOGCU_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ZOGCU_ABI_VERSION 1

#if defined(__GNUC__)
#define ZOGCU_API __attribute__((visibility("default")))
#else
#define ZOGCU_API
#endif

enum zogcu_status {
  ZOGCU_OK = 0,
  ZOGCU_ERR_INVALID_ARGUMENT = 1, /* null pointer, bad size or option          */
  ZOGCU_ERR_NODE_NOT_FOUND = 2,   /* edge endpoint >= node count (addEdge's     */
                                  /* error.NodeNotFound, array_graph.zig:88-89) */
  ZOGCU_ERR_OUT_OF_MEMORY = 3,    /* device or host allocation failed           */
  ZOGCU_ERR_CUDA = 4,             /* a CUDA runtime call failed                 */
  ZOGCU_ERR_NO_DEVICE = 5,        /* no usable sm_100 device                    */
  ZOGCU_ERR_TIMEOUT = 6,          /* a bounded device-side wait gave up         */
  ZOGCU_ERR_IO = 7,               /* file could not be opened / read            */
  ZOGCU_ERR_TOO_LARGE = 8,        /* sizes beyond the u32 node / edge indices   */
  ZOGCU_ERR_INTERNAL = 9
};

typedef struct zogcu_graph zogcu_graph;

/* Per-call statistics (all optional: pass NULL to skip). */
typedef struct zogcu_stats {
  uint64_t iterations;    /* PageRank: power iterations run                      */
  double residual;        /* PageRank: L1 step of the last iteration             */
  double elapsed_ms;      /* device time of the algorithm (CUDA events)          */
  double bytes_moved;     /* algorithmic bytes of the iterations (PageRank)      */
  uint64_t sources;       /* Brandes: sources processed                          */
  uint32_t max_depth;     /* Brandes: deepest BFS level seen                     */
  uint32_t sigma_overflow;/* Brandes: some path count wrapped modulo 2^64        */
  uint64_t launches;      /* kernels launched by the call                        */
  uint64_t polish_iterations; /* mixed precision: FP64 iterations at the end     */
  uint32_t kernel_config; /* PageRank: kernel configuration the autotuner chose  */
  uint32_t reserved;
} zogcu_stats;

/* PageRank precision forms. */
#define ZOGCU_PREC_FP64 0  /* FP64 throughout (the reference's arithmetic)     */
#define ZOGCU_PREC_MIXED 1 /* FP32 SpMV + FP64 dangling/residual + FP64 polish */

typedef struct zogcu_pr_opts {
  uint32_t struct_size;   /* sizeof(zogcu_pr_opts)                               */
  int32_t precision;      /* ZOGCU_PREC_*                                        */
  const double* x0;       /* start vector (length V) or NULL = uniform 1/n,      */
                          /* the reference's start (centrality.zig:912-918)      */
  const double* teleport; /* personalisation vector (length V, sums to 1) or     */
                          /* NULL = uniform (1-d)/n teleport of the reference    */
  int32_t device_pointers;/* x0, teleport and out_scores are device pointers     */
  int32_t reserved;
  void* stream;           /* cudaStream_t to run on, or NULL = a private stream  */
} zogcu_pr_opts;

typedef struct zogcu_bc_opts {
  uint32_t struct_size;   /* sizeof(zogcu_bc_opts)                               */
  uint32_t batch;         /* sources in flight per batch (multiple of 64), 0 = auto */
  const uint32_t* sources;/* source subset or NULL = every live node ascending,  */
                          /* the reference's order (centrality.zig:728)          */
  uint64_t num_sources;
  int32_t device_pointers;/* out_scores is a device pointer                      */
  int32_t reserved;
  void* stream;           /* cudaStream_t to run on, or NULL = a private stream  */
} zogcu_bc_opts;

/* ---- status ------------------------------------------------------------- */
ZOGCU_API const char* zogcu_status_string(int status);
ZOGCU_API const char* zogcu_last_error(void);
ZOGCU_API int zogcu_abi_version(void);

/* ---- graph resources ----------------------------------------------------- */

/* Replaces the NIF `new(node_count, from, to, weight, :soa)`
 * (lib/zog/.Elixir.Zog.ResourceGraph.zig:94-106 with buildGraph :26-35): node
 * ids 0..node_count-1, edges added in list order (head insertion, so each
 * node's successors iterate in reverse list order, array_graph.zig:88-108).
 * `weight` may be NULL (all 1.0); PageRank and unweighted betweenness ignore
 * it, weighted betweenness reads it.  Duplicate arcs and self-loops are kept.
 * `from` and `to` may be pageable.  Without weights, lists of 2^22 or more
 * arcs are uploaded in chunks; a chunk whose sources are non-decreasing
 * crosses PCIe as the offsets of its sources' runs (checked on the host,
 * expanded on the device; ZOGCU_UPLOAD_RUNS=0 sends every chunk as it is). */
ZOGCU_API int zogcu_graph_create_from_edges(uint32_t node_count, const uint32_t* from,
                                  const uint32_t* to, const double* weight,
                                  uint64_t num_edges, zogcu_graph** out);

/* Same as above with the edge arrays already in device memory. */
ZOGCU_API int zogcu_graph_create_from_device_edges(uint32_t node_count, const uint32_t* d_from,
                                         const uint32_t* d_to, uint64_t num_edges,
                                         void* stream, zogcu_graph** out);

/* Builds the device graph from the raw slices of an existing ArrayGraph
 * (array_graph.zig:21-38), as a NIF holding a GraphRes can pass them:
 * first_edge / next_edge use 0xFFFFFFFF for null; deleted nodes and edges are
 * skipped exactly like SuccessorIterator.next (array_graph.zig:164-180).
 * node_deleted / edge_deleted may be NULL (none deleted).  Arc weights are
 * not read (every weight is 1.0); the _weighted form below keeps them. */
ZOGCU_API int zogcu_graph_create_from_arraygraph(uint32_t node_capacity, const uint32_t* first_edge,
                                       const uint8_t* node_deleted, uint64_t edge_capacity,
                                       const uint32_t* to, const uint32_t* next_edge,
                                       const uint8_t* edge_deleted, zogcu_graph** out);

/* As above, also keeping the edges' f64 weights (the ArrayGraph's `data`
 * slice, one per edge slot) for weighted betweenness. */
ZOGCU_API int zogcu_graph_create_from_arraygraph_weighted(uint32_t node_capacity, const uint32_t* first_edge,
                                                          const uint8_t* node_deleted, uint64_t edge_capacity,
                                                          const uint32_t* to, const uint32_t* next_edge,
                                                          const uint8_t* edge_deleted, const double* data,
                                                          zogcu_graph** out);

/* Seeded R-MAT graph generated on the device (benchmark input): ef * 2^scale
 * raw edges, self-loops and duplicates removed, inserted in (src,dst) order;
 * undirected graphs keep one (lo,hi) pair per edge and store both arcs. */
ZOGCU_API int zogcu_graph_generate_rmat(int scale, int edge_factor, uint64_t seed, double a, double b,
                              double c, int directed, zogcu_graph** out);

/* Seeded Barabasi-Albert graph (lib/zog/generator.ex:132-198 model): clique
 * on m nodes, then each new node attaches to m distinct existing nodes chosen
 * with probability proportional to degree.  directed != 0 stores only the
 * new->old arcs (heavy-tailed in-degree); else both arcs. */
ZOGCU_API int zogcu_graph_generate_ba(uint32_t n, uint32_t m, uint64_t seed, int directed,
                                      zogcu_graph** out);

/* Seeded Watts-Strogatz graph (lib/zog/generator.ex:210-253 model): ring
 * lattice of k nearest neighbours, each edge rewired with probability beta. */
ZOGCU_API int zogcu_graph_generate_ws(uint32_t n, uint32_t k, double beta, uint64_t seed,
                                      int directed, zogcu_graph** out);

/* Raw (pre-dedupe) endpoints of R-MAT edges [i0, i0+m) of the generator above,
 * written to device arrays -- lets a test compare the generator element by
 * element with an independent CPU implementation of the same definition. */
ZOGCU_API int zogcu_rmat_raw_device(int scale, uint64_t seed, double a, double b, double c,
                                    uint64_t i0, uint64_t m, uint32_t* d_src, uint32_t* d_dst);

/* Replaces nif_read_edgelist(path, directed, :soa, integer_labels)
 * (lib/zog/.Elixir.Zog.ResourceGraph.zig:896-990): parses the file on the host
 * and builds the device graph.  *next_id receives the node count; with
 * integer_labels == 0 the labels (in id order) are returned '\n'-joined in
 * *labels (release with zogcu_free), else *labels is NULL. */
ZOGCU_API int zogcu_read_edgelist(const char* path, int directed, int integer_labels,
                        zogcu_graph** out, uint32_t* next_id, char** labels,
                        uint64_t* labels_len);

/* Replaces nif_destroy (.zig:108-110): frees the device CSR.  NULL is a no-op. */
ZOGCU_API int zogcu_graph_destroy(zogcu_graph* g);

/* Node capacity V, stored arcs E and live nodes n of a graph. */
ZOGCU_API int zogcu_graph_info(const zogcu_graph* g, uint32_t* node_capacity, uint64_t* num_arcs,
                     uint64_t* live_nodes);

/* Copies the device CSRs to host arrays (each may be NULL): in_off[V+1] and
 * in_col[E] (rows = sources ascending, the in_neighbors order of
 * centrality.zig:893-899), out_off[V+1] / out_col[E] (successor order) and
 * out_degree[V]. */
ZOGCU_API int zogcu_graph_export_csr(const zogcu_graph* g, uint64_t* in_off, uint32_t* in_col,
                           uint64_t* out_off, uint32_t* out_col, uint32_t* out_degree);

ZOGCU_API void zogcu_free(void* p);

/* Graphs, schedules and call workspaces come from the device's stream-ordered
 * memory pool, which keeps freed memory reserved for the next graph.  This
 * returns the reserve of the current device to the driver (memory still in
 * use is kept).  No counterpart in the reference. */
ZOGCU_API int zogcu_release_cached_memory(void);

/* ---- PageRank ------------------------------------------------------------ */

/* Replaces the NIF `pagerank(res, damping, max_iterations, tolerance)`
 * (lib/zog/.Elixir.Zog.ResourceGraph.zig:156-170 -> centrality.zig:858-965):
 * uniform start 1/n, teleport (1-d)/n, dangling mass sum(x/n) over live nodes
 * with out-degree 0, stop when the L1 step < tolerance (checked after the
 * swap), at most max_iterations.  out_scores has node-capacity length.  n == 0
 * gives all zeros, n == 1 gives 1.0 for the live node. */
ZOGCU_API int zogcu_pagerank(zogcu_graph* g, double damping, uint64_t max_iterations, double tolerance,
                   double* out_scores, zogcu_stats* stats);

/* As zogcu_pagerank with options (precision form, warm start, personalised
 * teleport, device pointers, caller stream); opts may be NULL.  In the
 * precision form on graphs of at least 2^23 nodes and 2^24 arcs the FP32 phase runs
 * propagation-blocked (streamed messages, exact integer row sums; environment
 * ZOGCU_PR_BLOCKED=0 turns it off, =1 forces it), and stats->reserved is 1
 * when it did. */
ZOGCU_API int zogcu_pagerank_ex(zogcu_graph* g, double damping, uint64_t max_iterations,
                      double tolerance, const zogcu_pr_opts* opts, double* out_scores,
                      zogcu_stats* stats);

/* ---- SpMV centralities (the same schedule and gather path) ------------- */

/* Replaces the NIF `katz(res, alpha, beta, max_iterations, tolerance)`
 * (.zig:183-192 -> centrality.zig:1190-1251): start beta, x' = alpha * sum of
 * in-neighbours + beta, stop when the L1 step < tolerance. */
ZOGCU_API int zogcu_katz(zogcu_graph* g, double alpha, double beta, uint64_t max_iterations,
                         double tolerance, double* out_scores, zogcu_stats* stats);

/* Replaces the NIF `alpha_centrality(res, alpha, initial, max_iterations,
 * tolerance)` (.zig:194-203 -> centrality.zig:1262-1321): start `initial`,
 * x' = alpha * sum of in-neighbours, L1 stopping rule. */
ZOGCU_API int zogcu_alpha_centrality(zogcu_graph* g, double alpha, double initial,
                                     uint64_t max_iterations, double tolerance, double* out_scores,
                                     zogcu_stats* stats);

/* Replaces the NIF `eigenvector(res, max_iterations, tolerance)` (.zig:172-181
 * -> centrality.zig:1050-1180): start 1 + i/1000, in-neighbour sums, L2
 * normalisation, zero-vector fallback 1/sqrt(n), oscillation exit with the
 * normalised average, L2 stopping rule.  stats->reserved receives how it
 * ended (0 max iterations, 1 converged, 2 zero vector, 3 oscillation).
 * Graphs with deleted nodes are not supported (ZOGCU_ERR_INVALID_ARGUMENT). */
ZOGCU_API int zogcu_eigenvector(zogcu_graph* g, uint64_t max_iterations, double tolerance,
                                double* out_scores, zogcu_stats* stats);

/* PageRank that allocates nothing, for callers that cannot call cudaMalloc
 * (a process whose device memory is owned by another runtime, or code that
 * must not allocate while it runs).  No counterpart in the reference: it is an
 * addition of this library.  The caller passes device arrays it owns -- the
 * in-CSR (in_off[V+1], in_col[E], sources ascending per row), out-degrees
 * (out_degree[V]) and the output (out_scores[V]) -- and every node counts as
 * live.  Scratch comes from one fixed device array of about 8 MiB, so V is
 * limited to 262,144 nodes; larger graphs return ZOGCU_ERR_TOO_LARGE.  The
 * first call on a device does the set-up: it looks up that array's address
 * and loads the entry point's kernels, and since CUDA loads modules lazily
 * that is when the array (kept until exit) and the kernels' code take their
 * device memory -- make that first call before another runtime takes the
 * device's memory, and before any stream capture.  All calls share the
 * array: calls that overlap on the GPU race, so serialise them.  Runs on
 * `stream` (NULL = the default stream), reading the chain's state back after
 * every 32 iteration launches so that it stops once converged whatever
 * max_iterations is, and returns when the scores are written.  Same options
 * and result as zogcu_pagerank. */
ZOGCU_API int zogcu_pagerank_noalloc(const uint32_t* d_in_off, const uint32_t* d_in_col,
                                     const uint32_t* d_out_degree, uint32_t num_nodes,
                                     uint64_t num_arcs, double damping, uint64_t max_iterations,
                                     double tolerance, double* d_out_scores, zogcu_stats* stats,
                                     void* stream);

/* ---- Brandes betweenness -------------------------------------------------- */

/* Replaces nif_betweenness_unweighted (.zig:112-121 ->
 * centrality.zig:687-798): sum over every live source s of the dependencies
 * delta_s(v), v != s, unnormalised. */
ZOGCU_API int zogcu_betweenness_unweighted(zogcu_graph* g, double* out_scores, zogcu_stats* stats);

/* As above with options (source subset, batch size, device output, stream).
 *
 * Both forms run the sources in batches of 64.  The batches are dealt to up
 * to 8 lanes (independent branches of one CUDA graph, each with its own
 * workspace), and each lane runs up to 8 batches per launch, so a call of up
 * to 4,096 sources is one graph launch.  Levels are device-ended while loops,
 * and each level pushes or pulls as its frontier's out-arcs dictate.  The graph
 * and the lanes' workspaces stay with the graph resource (graphs keyed by lane
 * count, batch slots per lane and push threshold), and later calls reuse them;
 * the first call of a key instantiates its graph.
 * stats->reserved counts the graph launches, stats->launches the kernels they
 * ran, and stats->max_depth the deepest level.  The lanes' scores are added in
 * lane order, so repeated calls are bit-identical.  Environment:
 * ZOGCU_BC_STREAMS=<k> sets the lane count, ZOGCU_BC_PUSH_RATIO=<r> the push
 * threshold (0 = pull only), ZOGCU_TRACE=1 prints the call's phases. */
ZOGCU_API int zogcu_betweenness_unweighted_ex(zogcu_graph* g, const zogcu_bc_opts* opts,
                                    double* out_scores, zogcu_stats* stats);

/* Replaces nif_betweenness_f64 (.zig:123-132 -> centrality.betweennessF64
 * :1355-1357 -> betweenness, ArrayGraph branch, centrality.zig:528-682):
 * Dijkstra-based Brandes over the arc weights (1.0 where none were given),
 * unnormalised, every live source ascending or opts->sources (opts may be
 * NULL; its batch field is ignored).  Weights must be positive and finite; a
 * shortest path through an arc of effective length zero (fl(d + w) == d) is
 * reported as ZOGCU_ERR_INVALID_ARGUMENT, since the reference's counts would
 * then depend on its heap's tie order. */
ZOGCU_API int zogcu_betweenness_weighted(zogcu_graph* g, const zogcu_bc_opts* opts, double* out_scores,
                                         zogcu_stats* stats);

/* The arc weights in out-CSR (successor) order, out_weights[E] (1.0 each when
 * the graph was built without weights). */
ZOGCU_API int zogcu_graph_export_weights(const zogcu_graph* g, double* out_weights);

/* BFS intermediates of the Brandes forward phase (centrality.zig:741-767) for
 * `num_sources` sources: dist_out[i*V + v] (0xFFFFFFFF = unreached) and
 * sigma_out[i*V + v] (shortest-path counts, wrapping modulo 2^64 like the
 * reference's usize).  Either output may be NULL.  *overflow is set when some
 * count wrapped. */
ZOGCU_API int zogcu_bfs_sigma(zogcu_graph* g, const uint32_t* sources, uint64_t num_sources,
                    uint32_t* dist_out, uint64_t* sigma_out, uint32_t* overflow);

/* ---- Personalised PageRank for many seeds (CSR SpMM) ------------------------
 * An extension: the reference's teleport is always uniform (centrality.zig:
 * 943).  For each seed s: uniform start 1/n, teleport (1-d) e_s, dangling mass
 * spread uniformly, stop once the seed's L1 step is below tol (each seed
 * stops on its own).  The seeds advance together as the columns of an SpMM
 * over the in-CSR, in passes of 64 to 256 seeds; the whole call is one CUDA
 * graph (per pass a device-ended while loop of iterations), launched once:
 * stats->reserved is 1 (the host-side launches) and stats->launches counts
 * the kernels the graph ran.  out_scores[num_seeds * V] is seed-major (seed
 * i's vector at i * V); iterations[num_seeds] may be NULL.  opts (may be
 * NULL) gives the stream and device_pointers; precision must be FP64 and x0 /
 * teleport NULL.  Graphs with deleted nodes are rejected. */
ZOGCU_API int zogcu_ppr(zogcu_graph* g, const uint32_t* seeds, uint32_t num_seeds, double damping,
                        uint64_t max_iterations, double tolerance, const zogcu_pr_opts* opts,
                        double* out_scores, uint64_t* iterations, zogcu_stats* stats);

/* ---- Batched PageRank: many graphs in one persistent launch ------------------
 * No counterpart in the reference (one graph per NIF call).  A batch holds
 * copies of several graphs' device CSRs; one call solves every graph exactly
 * as zogcu_pagerank solves it alone (uniform start, FP64), in a single
 * persistent kernel launch replayed from a CUDA graph.  The kernel
 * configuration (CTA size, cluster size, degree bin) is chosen by an
 * autotuner on the first call. */
typedef struct zogcu_batch zogcu_batch;

typedef struct zogcu_batch_opts {
  uint32_t struct_size;   /* sizeof(zogcu_batch_opts)                            */
  int32_t config;         /* kernel configuration, -1 = autotuned                */
  int32_t device_pointers;/* out_scores is a device pointer                      */
  int32_t reserved;
  void* stream;           /* cudaStream_t to run on, or NULL = a private stream  */
} zogcu_batch_opts;

/* Copies the graphs (all on one device; each with fewer than 2^32 arcs) into
 * a new batch; the graphs stay owned by the caller. */
ZOGCU_API int zogcu_batch_create(zogcu_graph* const* graphs, uint32_t count, zogcu_batch** out);
ZOGCU_API int zogcu_batch_destroy(zogcu_batch* batch);
/* Graph count, total node slots and arcs; node_offsets[count + 1] (may be
 * NULL) receives where each graph's scores start in the output. */
ZOGCU_API int zogcu_batch_info(const zogcu_batch* batch, uint32_t* count, uint64_t* total_nodes,
                               uint64_t* total_arcs, uint64_t* node_offsets);
/* PageRank of every graph: out_scores[total_nodes] (graph g at
 * node_offsets[g]), iterations[count] (may be NULL). */
ZOGCU_API int zogcu_batch_pagerank(zogcu_batch* batch, double damping, uint64_t max_iterations,
                                   double tolerance, const zogcu_batch_opts* opts, double* out_scores,
                                   uint64_t* iterations, zogcu_stats* stats);

/* ---- Learned PageRank warm start -------------------------------------------
 * No counterpart in the reference, whose start is always uniform
 * (centrality.zig:912-918).  A 3-layer message-passing network (hidden 64,
 * FP32 master weights, BF16 weights in the forward pass, FP32 accumulation)
 * maps degree features to a predicted log(n * pagerank); its softmax is a
 * start vector for zogcu_pagerank_ex (opts.x0), and power iteration still runs
 * to the caller's tolerance.  Training, prediction and the weight file all run
 * through the entry points below. */
typedef struct zogcu_gnn zogcu_gnn;

/* Number of FP32 parameters (the length of get/set_params buffers). */
ZOGCU_API int zogcu_gnn_num_params(void);
/* New network with seeded Glorot-uniform weights and zero Adam state. */
ZOGCU_API int zogcu_gnn_create(uint64_t seed, zogcu_gnn** out);
ZOGCU_API int zogcu_gnn_destroy(zogcu_gnn* net);
ZOGCU_API int zogcu_gnn_get_params(const zogcu_gnn* net, float* out_params);
ZOGCU_API int zogcu_gnn_set_params(zogcu_gnn* net, const float* params);
/* Training losses against a PageRank vector pr (sums to 1 over live nodes). */
enum {
  ZOGCU_GNN_LOSS_LOG_MSE = 0, /* mean over live nodes of (y - log(n pr))^2          */
  ZOGCU_GNN_LOSS_KL = 1       /* KL(pr || softmax(y)): errors weighted by rank mass */
};
/* Loss and its gradient with respect to the parameters, for one graph and its
 * PageRank vector target_pr[V] (host).  Either output may be NULL. */
ZOGCU_API int zogcu_gnn_loss_grad(zogcu_gnn* net, zogcu_graph* g, const double* target_pr,
                                  int loss_kind, float* loss, float* grad_out);
/* One Adam step (beta 0.9 / 0.999) on one graph; d_target_pr is a device array. */
ZOGCU_API int zogcu_gnn_train_step(zogcu_gnn* net, zogcu_graph* g, const double* d_target_pr,
                                   int loss_kind, float learning_rate, float* loss);
/* Start vector x0[V] (sums to 1 over live nodes; 0 on deleted slots), into a
 * device array when device_out != 0; raw_out[V] (host, may be NULL) receives
 * the network output y.  Runs on `stream` (NULL = a private stream). */
ZOGCU_API int zogcu_gnn_predict(const zogcu_gnn* net, zogcu_graph* g, double* x0, int device_out,
                                void* stream, float* raw_out);
/* Weight file: magic "ZOGN", version 1, parameter count, BF16 weights. */
ZOGCU_API int zogcu_gnn_save(const zogcu_gnn* net, const char* path);
ZOGCU_API int zogcu_gnn_load(const char* path, zogcu_gnn** out);

#ifdef __cplusplus
}
#endif

#endif /* ZOGCU_H_ */

/*
 * pfg.h - C ABI of the B200 SSSP / A* engine (libpfg_b200.so).
 *
 * This is the drop-in boundary. The reference hides its CUDA code behind the
 * C++ class `GpuSolver` (reference: include/gpu_sssp.h:97-120, implemented in
 * src/gpu_sssp.cu:61-569 and src/gpu_device.cu:11-160). Here the same
 * operations are exported as plain C functions over an opaque handle, with
 * plain pointers and sizes and an integer status instead of exceptions and
 * exit(). The C++ `GpuSolver` (include/gpu_sssp.h, gpu_solver.cpp) and the
 * Python package are thin layers over these symbols.
 *
 * Conventions
 *  - Every function returns a pfg_status; PFG_OK is 0. On failure
 *    pfg_last_error() returns a human readable message for the calling
 *    thread.
 *  - Pointers named h_* are host memory, d_* are device memory of the
 *    solver's device.
 *  - Distances are uint32 with PFG_INF = 0xFFFFFFFF for "unreachable", parents
 *    are uint32 with PFG_NO_PARENT = 0xFFFFFFFF. The packed state word of a
 *    vertex is (dist << 32) | parent (reference: src/gpu_kernels.cuh:11-13).
 *  - A solver is not thread safe: one host thread drives one solver, as in
 *    the reference (src/gpu_sssp.cu:92, one stream per solver, no locking).
 */
#ifndef PFG_H_
#define PFG_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define PFG_API __attribute__((visibility("default")))
#else
#define PFG_API
#endif

#define PFG_ABI_VERSION 1
#define PFG_INF 0xFFFFFFFFu
#define PFG_NO_PARENT 0xFFFFFFFFu

typedef enum pfg_status {
    PFG_OK = 0,
    PFG_ERR_INVALID_ARGUMENT = 1, /* bad batch size, source, target, option  */
    PFG_ERR_INVALID_GRAPH = 2,    /* CSR not well formed (see pfg_create)     */
    PFG_ERR_OUT_OF_MEMORY = 3,    /* device memory precheck or cudaMalloc     */
    PFG_ERR_NOT_CONVERGED = 4,    /* device round cap reached                  */
    PFG_ERR_DEVICE_TIMEOUT = 5,   /* a bounded device-side wait gave up        */
    PFG_ERR_CUDA = 6,             /* any other CUDA runtime error              */
    PFG_ERR_NO_DEVICE = 7,        /* no CUDA device / ordinal out of range     */
    PFG_ERR_CAPACITY = 8          /* a fixed-size resource is exhausted        */
} pfg_status;

/* Enum values follow the declaration order of the reference's enums
 * (include/gpu_sssp.h:10-35) so that a static_cast maps one onto the other. */
enum pfg_algo { PFG_ALGO_NAIVE = 0, PFG_ALGO_FRONTIER = 1, PFG_ALGO_DELTA = 2 };
enum pfg_mapping { PFG_MAP_THREAD = 0, PFG_MAP_WARP = 1, PFG_MAP_HYBRID = 2 };
enum pfg_atomic { PFG_ATOMIC_MIN_RBA = 0, PFG_ATOMIC_CAS_RBA = 1, PFG_ATOMIC_MIN_NOCHECK = 2 };
enum pfg_compaction { PFG_COMPACT_WARP_ATOMIC = 0, PFG_COMPACT_PREFIX_SCAN = 1 };
/* Schedule policy for Delta-stepping (extension; no reference counterpart). */
enum pfg_policy_kind { PFG_POLICY_FIXED = 0, PFG_POLICY_LEARNED = 1 };
/* How a Delta-stepping bucket is worked off (extension; no reference counterpart).
 * ROUNDS: relaxation rounds separated by grid barriers (the reference's loop).
 * ASYNC:  one drain per bucket: CTAs relax the vertices they claim from their
 *         own shared-memory list and share work through a ring queue, with a
 *         grid barrier only between buckets.
 * WARP:   ASYNC with the drain worked by warp workers: every warp takes
 *         entries from its CTA's shared-memory work queue on its own, with no
 *         block barrier between batches (Hybrid mapping only; other mappings
 *         run ASYNC). It sustains more throughput on large batches (hundreds of
 *         instances), ASYNC has the lower latency on small ones.
 * INSTANCE: ASYNC with a window per instance of a multi-source run: each
 *         instance advances to its next bucket as soon as its own entries are
 *         drained, with no grid barrier between buckets; the automatic Delta
 *         (delta = 0) is 4 x the single-source rule under it. Applies to solver
 *         runs of 2..256 sources with the Hybrid mapping, the fixed Delta
 *         policy and block_size >= 64 when Delta >= the largest weight (every
 *         arc light) and no row has more than 8 x block_size arcs; elsewhere it
 *         runs as ASYNC.
 * AUTO:   INSTANCE where it applies to a batch of 96 or more sources
 *         (environment PFG_INST_WINDOWS: that threshold, 0 = never), else ASYNC
 *         for Delta-stepping; ROUNDS for Naive and Frontier. */
enum pfg_schedule { PFG_SCHEDULE_AUTO = 0, PFG_SCHEDULE_ROUNDS = 1, PFG_SCHEDULE_ASYNC = 2,
                    PFG_SCHEDULE_WARP = 3, PFG_SCHEDULE_INSTANCE = 4 };

/* Mirrors GpuOptions (reference: include/gpu_sssp.h:42-52) plus `policy`. */
typedef struct pfg_options {
    int32_t algo;        /* enum pfg_algo, default PFG_ALGO_DELTA                 */
    int32_t mapping;     /* enum pfg_mapping, default PFG_MAP_HYBRID              */
    int32_t atomic;      /* enum pfg_atomic, default PFG_ATOMIC_MIN_RBA           */
    uint32_t delta;      /* 0 = automatic, round(32 * avgW / avgDeg)              */
    int32_t block_size;  /* threads per CTA; invalid values fall back to 256      */
    uint32_t sync_every; /* accepted for compatibility; convergence is detected
                            on the device, so the host synchronizes once per run */
    int32_t compaction;  /* enum pfg_compaction (Frontier only)                   */
    int32_t policy;      /* enum pfg_policy_kind (Delta-stepping only)            */
    int32_t eager;       /* Hybrid mapping: in-round propagation sub-rounds per
                            grid round; -1 = engine default, 0 = off (extension) */
    int32_t blocks_per_sm; /* CTAs of the persistent kernel per SM; 0 = engine
                              default (1024 resident threads per SM) (extension) */
    int32_t schedule;    /* enum pfg_schedule, default PFG_SCHEDULE_AUTO; ASYNC and
                            WARP apply to Delta-stepping only (extension)       */
} pfg_options;

/* Mirrors GpuStats (reference: include/gpu_sssp.h:55-65) plus `rounds`. */
typedef struct pfg_stats {
    uint64_t edges_scanned;  /* real (non padding) arcs examined                */
    uint64_t atomics_issued; /* 64-bit atomicMin / atomicCAS on the state        */
    uint64_t updates;        /* relaxations that lowered a distance             */
    uint64_t pushes;         /* queue insertions                                 */
    uint32_t iterations;     /* device rounds with a non-empty input             */
    uint32_t host_syncs;     /* host waits inside the run (1: the final one)    */
    uint32_t launches;       /* kernel launches issued by the run                */
    uint32_t buckets;        /* Delta-stepping buckets processed                 */
    uint32_t delta;          /* Delta of the first bucket (0 unless Delta-step)  */
    uint32_t rounds;         /* device rounds executed (barrier epochs)          */
} pfg_stats;

typedef struct pfg_solver pfg_solver;

/* ---- solver life cycle (reference: GpuSolver::GpuSolver / ~GpuSolver,
 *      src/gpu_sssp.cu:107-200) ----
 * row_offsets[n+1], col_indices[m], weights[m]: host CSR. Rows must be sorted
 * by weight (the reference's buildCSR sorts each row by (w, dst),
 * src/graph.cpp:57-74); weights must be >= 1; col < n; row_offsets
 * non-decreasing with row_offsets[0] = 0 and row_offsets[n] = m.
 * x, y: optional vertex coordinates (both NULL or both of length n) for the
 * A* heuristic; h_scale is CSRGraph::hScale (0 disables the heuristic).
 * avg_w / avg_deg feed the automatic Delta (reference: src/gpu_sssp.cu:202-206).
 * max_batch: largest number of sources one run may use; max_batch * n must be
 * < 2^32 (reference: src/gpu_sssp.cu:108). */
PFG_API pfg_status pfg_create(const uint32_t* row_offsets, const uint32_t* col_indices,
                      const uint32_t* weights, const double* x, const double* y,
                      uint32_t n, uint32_t m, double h_scale, double avg_w,
                      double avg_deg, uint32_t max_batch, pfg_solver** out);
/* Same, on an explicit CUDA device ordinal (the reference always uses 0). */
PFG_API pfg_status pfg_create_on_device(const uint32_t* row_offsets, const uint32_t* col_indices,
                                const uint32_t* weights, const double* x, const double* y,
                                uint32_t n, uint32_t m, double h_scale, double avg_w,
                                double avg_deg, uint32_t max_batch, int32_t device,
                                pfg_solver** out);
PFG_API void pfg_destroy(pfg_solver* s);

/* Accessors (reference: GpuSolver::uploadMs / deviceBytes / autoDelta,
 * src/gpu_sssp.cu:540-543). */
PFG_API double pfg_upload_ms(const pfg_solver* s);
PFG_API uint64_t pfg_device_bytes(const pfg_solver* s);
PFG_API uint32_t pfg_auto_delta(const pfg_solver* s);
PFG_API uint32_t pfg_num_vertices(const pfg_solver* s);
PFG_API uint32_t pfg_max_batch(const pfg_solver* s);
/* cudaStream_t of the solver, as void*, so callers can record events on it. */
PFG_API void* pfg_stream(const pfg_solver* s);

/* ---- one run (reference: GpuSolver::Impl::run, src/gpu_sssp.cu:461-534) ----
 * Shortest paths from k sources h_srcs[0..k) (1 <= k <= max_batch), all in
 * one device launch; instance i owns state words [i*n, (i+1)*n).
 * astar != 0: point-to-point A* from h_srcs[0] to dst (k must be 1); keys are
 * dist + h(v) and every relaxation is pruned at dist[dst] (reference:
 * src/gpu_kernels.cuh:178-179).
 * h_state_out (nullable): receives k*n packed state words.
 * ms_out (nullable): device time of initialisation + relaxation measured with
 * CUDA events on the solver's stream (the reference's r.ms, which excludes
 * copy-back, src/gpu_sssp.cu:478-502).
 * Errors: PFG_ERR_INVALID_ARGUMENT for k == 0, k > max_batch, a source >= n,
 * dst >= n when astar, or astar with k != 1 (reference: src/gpu_sssp.cu:463-465).
 * opt == NULL means default options. Like the reference, Naive with k > 1
 * silently runs Delta-stepping (src/gpu_sssp.cu:466). */
PFG_API pfg_status pfg_run(pfg_solver* s, const uint32_t* h_srcs, uint32_t k, int32_t astar,
                   uint32_t dst, const pfg_options* opt, pfg_stats* stats_out,
                   uint64_t* h_state_out, float* ms_out);

/* Same run with the sources already on the device (d_srcs, k entries) and no
 * host synchronisation: work is enqueued on the solver's stream and the call
 * returns immediately. Results stay in the solver's state buffer
 * (pfg_state_device). Statistics and errors of an asynchronous run are read
 * with pfg_finish(). */
PFG_API pfg_status pfg_run_async(pfg_solver* s, const uint32_t* d_srcs, uint32_t k, int32_t astar,
                         uint32_t dst, const pfg_options* opt);
/* Waits for the last asynchronous run, returns its status and statistics. */
PFG_API pfg_status pfg_finish(pfg_solver* s, pfg_stats* stats_out);
/* Device pointer to the k*n packed state words of the last run. */
PFG_API const uint64_t* pfg_state_device(const pfg_solver* s);

/* Copies state words [first, first+count) of the last run to host memory. */
PFG_API pfg_status pfg_copy_state(pfg_solver* s, uint64_t first, uint64_t count, uint64_t* h_out);

/* Copies the distances of state words [first, first+count) of the last run to
 * host memory, h_out[i] = dist of word first+i: the result of the reference's
 * GpuSolver::multiSource with distOut (src/gpu_sssp.cu:553-569, which copies
 * the packed words and splits them on the host). The split runs on the device,
 * so half the bytes cross PCIe. */
PFG_API pfg_status pfg_copy_dist(pfg_solver* s, uint64_t first, uint64_t count, uint32_t* h_out);

/* Streamed multi-source runs: a sequence of the reference's
 * GpuSolver::multiSource(srcs, opt, &distOut) calls (src/gpu_sssp.cu:553-569)
 * in which the copy of one run's distances overlaps the next run's kernel.
 * pfg_run_dist_async enqueues a run of the k host sources (H2D included) whose
 * distances go to h_dist_out (k*n words, instance i at i*n; pinned memory makes
 * the copy asynchronous), after waiting for the previous streamed run's kernel
 * and starting the copy of that run's distances; prev_stats_out (may be NULL)
 * receives the previous run's statistics. h_dist_out must stay valid until
 * pfg_dist_wait returns, which completes the last run and every copy
 * (stats_out: the last run's statistics). Any other call on the solver first
 * completes the stream. Errors as pfg_run; a failed run ends the stream. */
PFG_API pfg_status pfg_run_dist_async(pfg_solver* s, const uint32_t* h_srcs, uint32_t k,
                                      const pfg_options* opt, uint32_t* h_dist_out,
                                      pfg_stats* prev_stats_out);
PFG_API pfg_status pfg_dist_wait(pfg_solver* s, pfg_stats* stats_out);

/* Reconstructs the path src -> dst of instance `inst` of the last run on the
 * device by following parent pointers (reference: reconstructPath,
 * src/cpu_sssp.cpp:124-135). path_len_out = 0 when dst is unreachable or the
 * parent chain is broken. Fails with PFG_ERR_CAPACITY when the path has more
 * than cap vertices. */
PFG_API pfg_status pfg_extract_path(pfg_solver* s, uint32_t inst, uint32_t src, uint32_t dst,
                            uint32_t* h_path, uint32_t cap, uint32_t* path_len_out);

/* ---- device information (reference: gpuQueryDevice / gpuWarmup /
 *      gpuTransferStudy, src/gpu_device.cu:39-160) ---- */
typedef struct pfg_device_info {
    int32_t ok;
    char name[256];
    int32_t cc_major, cc_minor, sm_count, clock_mhz, mem_clock_mhz, bus_width;
    int32_t driver_version, runtime_version, max_threads_per_sm, warp_size;
    uint64_t global_mem, shared_per_block, l2_bytes;
    double peak_bandwidth_gbs;
} pfg_device_info;
PFG_API pfg_status pfg_query_device(int32_t dev, pfg_device_info* out);
PFG_API pfg_status pfg_warmup(void);

typedef struct pfg_transfer_study {
    double bytes, pageable_ms, pinned_ms, pinned_streams_ms;
} pfg_transfer_study;
PFG_API pfg_status pfg_transfer_study_run(const uint32_t* row_offsets, const uint32_t* col_indices,
                                  const uint32_t* weights, uint32_t n, uint32_t m,
                                  int32_t reps, pfg_transfer_study* out);

/* ---- batches of uneven instances (extension of multiSource) ----
 * The reference's multiSource batches K sources of one graph with state
 * index k*n + v (src/gpu_kernels.cuh:223-225). A batch generalises this to
 * per-instance offsets: it holds num_graphs CSR graphs (rows sorted by
 * weight) and a table of instances (graph, source); instance i owns the
 * packed state words [pfg_batch_instance_offset(i), ...(i+1)). One
 * persistent launch relaxes every instance with one shared bucket
 * sequence; per-instance results equal single-source runs bit for bit.
 * max_states bounds the sum of the instances' vertex counts (< 2^32). */
typedef struct pfg_batch pfg_batch;
PFG_API pfg_status pfg_batch_create(uint32_t num_graphs, const uint32_t* const* row_offsets,
                                    const uint32_t* const* col_indices,
                                    const uint32_t* const* weights, const uint32_t* n,
                                    const uint32_t* m, uint64_t max_states,
                                    uint32_t max_instances, int32_t device, pfg_batch** out);
PFG_API void pfg_batch_destroy(pfg_batch* b);
/* Instance i = (inst_graph[i], inst_src[i]). Replaces any recorded run. */
PFG_API pfg_status pfg_batch_set_instances(pfg_batch* b, const uint32_t* inst_graph,
                                           const uint32_t* inst_src, uint32_t count);
/* One launch over all instances; ms_out = device time (CUDA events). */
PFG_API pfg_status pfg_batch_run(pfg_batch* b, const pfg_options* opt, pfg_stats* stats_out,
                                 float* ms_out);
/* Records one run (control-block upload, persistent launch, read-back) into a
 * CUDA graph; pfg_batch_replay launches it again with the same options and
 * instances and returns its statistics. */
PFG_API pfg_status pfg_batch_capture(pfg_batch* b, const pfg_options* opt);
PFG_API pfg_status pfg_batch_replay(pfg_batch* b, pfg_stats* stats_out, float* ms_out);
PFG_API uint64_t pfg_batch_instance_offset(const pfg_batch* b, uint32_t inst);
PFG_API uint64_t pfg_batch_num_states(const pfg_batch* b);
PFG_API pfg_status pfg_batch_copy_state(pfg_batch* b, uint64_t first, uint64_t count,
                                        uint64_t* h_out);
PFG_API void* pfg_batch_stream(const pfg_batch* b);
PFG_API double pfg_batch_upload_ms(const pfg_batch* b);
PFG_API uint64_t pfg_batch_device_bytes(const pfg_batch* b);

/* ---- serving: continuous batching of A* queries (extension; the reference
 *      answers one query per GpuSolver::astar call, src/gpu_sssp.cu:549-551) ----
 * The graph and `slots` query slots stay resident. pfg_server_submit queues a
 * query on the host; every pfg_server_step admits queued queries into free
 * slots, runs at most max_rounds device rounds of one persistent launch that
 * relaxes every slot in flight together (queries admitted later join the
 * shared bucket sequence at its next bucket), and retires the slots whose
 * search is complete. Finished queries are drained with pfg_server_results;
 * times are microseconds since the server was created. dist is the exact
 * shortest distance (PFG_INF if unreachable). slots = 0 at creation admits by
 * device memory: the server takes as many slots as fit in 60 % of the device's
 * free memory after the graph (at most 2048, and slots * n < 2^32); each slot
 * holds a packed state word, five queue words, three stamp words and two ring
 * entries per vertex. max_rounds counts bucket drains when the buckets run
 * asynchronously (the default schedule), relaxation rounds otherwise. With
 * opt->policy = PFG_POLICY_LEARNED and a network loaded on the server's solver
 * (pfg_set_policy on pfg_server_solver), the policy picks the shared bucket
 * sequence's Delta; without a network the fixed automatic Delta is used. */
typedef struct pfg_server pfg_server;
typedef struct pfg_query_result {
    uint64_t id;
    uint32_t src, dst, dist, slot;
    double submit_us, admit_us, finish_us;
} pfg_query_result;
PFG_API pfg_status pfg_server_create(const uint32_t* row_offsets, const uint32_t* col_indices,
                                     const uint32_t* weights, const double* x, const double* y,
                                     uint32_t n, uint32_t m, double h_scale, double avg_w,
                                     double avg_deg, uint32_t slots, const pfg_options* opt,
                                     int32_t device, pfg_server** out);
PFG_API void pfg_server_destroy(pfg_server* v);
PFG_API pfg_status pfg_server_submit(pfg_server* v, uint32_t src, uint32_t dst, uint64_t* id_out);
PFG_API pfg_status pfg_server_step(pfg_server* v, uint32_t max_rounds, uint32_t* admitted_out,
                                   uint32_t* completed_out);
PFG_API pfg_status pfg_server_results(pfg_server* v, pfg_query_result* out, uint32_t cap,
                                      uint32_t* n_out);
PFG_API uint32_t pfg_server_pending(const pfg_server* v);
PFG_API uint32_t pfg_server_in_flight(const pfg_server* v);
/* Query slots of the server (the number chosen when it was created with slots = 0). */
PFG_API uint32_t pfg_server_slots(const pfg_server* v);
PFG_API double pfg_server_now_us(const pfg_server* v);
/* The server's solver (graph + slots), e.g. to load a policy network. */
PFG_API pfg_solver* pfg_server_solver(pfg_server* v);

/* ---- learned Delta policy (extension; no reference counterpart) ----
 * The policy is a 12 -> 64 -> 64 -> 64 -> 16 fp32 MLP evaluated on the device
 * at the first bucket and at every bucket advance; its argmax class c picks
 * the next bucket's Delta as {1/16, 1/8, 1/4, 1/2, 1, 2, 4, 8}[c % 8] x the
 * automatic Delta and its schedule (asynchronous bucket if c < 8, relaxation
 * rounds otherwise). It only changes the schedule: distances and parents are
 * the same as with a fixed Delta.
 * pfg_set_policy loads a flat parameter image of pfg_policy_param_count()
 * floats (layout: w1[64x12] b1 w2[64x64] b2 w3[64x64] b3 w4[16x64] b4
 * in_mean[12] in_scale[12]). */
PFG_API pfg_status pfg_set_policy(pfg_solver* s, const float* params, uint64_t count);
PFG_API uint64_t pfg_policy_param_count(void);
/* A Delta-stepping run (fixed or learned Delta) that also returns, for every
 * decision point (the first bucket and every bucket advance), one trace row of
 * 16 floats: the 12 policy features (log2 frontier size, log2 items and log2
 * arcs of the last bucket, its work ratio, the degree histogram of a frontier
 * sample in three bins, its light-arc fraction, its distance spread / Delta,
 * the gap to the next key / avgW, log2 Delta / avgW, log2 buckets so far), then
 * the bucket index, the Delta of the bucket that ended, the items that entered
 * it and the rounds it took. *rows_out = rows written (<= trace_cap). */
PFG_API pfg_status pfg_run_traced(pfg_solver* s, const uint32_t* h_srcs, uint32_t k,
                                  const pfg_options* opt, pfg_stats* stats_out, float* h_trace,
                                  uint32_t trace_cap, uint32_t* rows_out, float* ms_out);
/* Training and inference of the policy network on the GPU (hand-written
 * kernels). Samples are rows of 12 features (h_x, n x 12) with soft targets
 * over the 16 classes (h_y, n x 16, each row summing to 1); the loss is
 * the mean cross-entropy. pfg_policy_grad returns the loss and its gradient
 * for every parameter (zero for the fixed input normalisation);
 * pfg_policy_train runs `steps` full-batch Adam steps in place and writes the
 * loss of each step to loss_out (nullable); pfg_policy_infer returns the
 * argmax class per sample. */
PFG_API pfg_status pfg_policy_grad(const float* h_params, const float* h_x, const float* h_y,
                                   uint32_t n, float* h_grad_out, float* loss_out);
PFG_API pfg_status pfg_policy_train(float* h_params, const float* h_x, const float* h_y,
                                    uint32_t n, uint32_t steps, float lr, float* loss_out);
PFG_API pfg_status pfg_policy_infer(const float* h_params, const float* h_x, uint32_t n,
                                    uint32_t* h_class_out);

/* ---- SSSP without any allocation (no counterpart in the reference) ----
 * For callers that may not allocate device memory themselves or through
 * this library: code inside a host application or framework that owns all
 * device memory through its own pool and hands a plugin only the buffers it
 * may use, or a latency-critical loop that cannot afford cudaMalloc's
 * implicit synchronisation. Runs the persistent Delta-stepping kernel of
 * pfg_run (Hybrid mapping, MinRBA atomics, fixed `delta` >= 1) from `src`
 * on a CSR already in device memory, writing n packed (dist << 32 | parent)
 * words to d_state_out and [status, rounds, buckets, non-empty rounds] to
 * d_status_out[0..3] (status is a pfg_status value). Work is enqueued on
 * `stream` (a cudaStream_t of the current device) and the call returns
 * without waiting; read d_status_out after synchronising.
 * The CSR must be what pfg_create accepts: row_offsets[0] = 0, non-decreasing,
 * row_offsets[n] = m, col < n, weights in [1, 2^32 - 2], every row sorted by
 * weight. The host cannot read device memory without waiting, so these are
 * checked on the device: when one fails, nothing is relaxed, d_state_out is
 * (PFG_INF, PFG_NO_PARENT) everywhere, d_status_out[0] is
 * PFG_ERR_INVALID_GRAPH (PFG_ERR_CAPACITY when the rows padded to 4 arcs do
 * not fit the scratch), d_status_out[1] the mask of failed checks (1 row
 * offsets, 2 padded size, 4 column, 8 weight, 16 row order) and [2], [3] zero.
 * Differences from pfg_run: buckets always run as relaxation rounds (no
 * asynchronous buckets: they need a ring sized by the graph), rows of any
 * length are relaxed by the CTA that holds them (no hub records), and eager
 * sub-rounds follow pfg_run's default (on when m / n <= 6). Every device-side
 * wait is bounded by PFG_TIMEOUT_MS, as in pfg_run. Results are identical.
 * All scratch lives in one fixed device array compiled into the library
 * (about 7.6 MB, held by every device the library's module is loaded on
 * until the process exits), so the graph is limited to n <=
 * PFG_NOALLOC_MAX_VERTICES and m + 3n <= PFG_NOALLOC_MAX_ARCS; larger inputs
 * return PFG_ERR_CAPACITY before anything is launched. The first call on a
 * device looks up the array's device address (this also loads the module on
 * that device); make that first call before any stream capture. Every call
 * on a device shares the one array, so calls that overlap on the GPU (two
 * streams, two threads) race and corrupt each other: serialise them. */
#define PFG_NOALLOC_MAX_VERTICES 65536u
#define PFG_NOALLOC_MAX_ARCS 655360u
PFG_API pfg_status pfg_sssp_noalloc(const uint32_t* d_row_offsets, const uint32_t* d_col_indices,
                                    const uint32_t* d_weights, uint32_t n, uint32_t m, uint32_t src,
                                    uint32_t delta, uint64_t* d_state_out, uint32_t* d_status_out,
                                    void* stream);

/* ---- errors ---- */
PFG_API const char* pfg_last_error(void);
PFG_API const char* pfg_status_string(pfg_status st);
PFG_API int32_t pfg_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* PFG_H_ */

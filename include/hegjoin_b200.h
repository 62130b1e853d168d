/* hegjoin_b200.h -- C ABI of the B200-native epsilon self-join.
 *
 * This is the drop-in boundary for HEGJoin's GPU-only join (algorithm 0,
 * `./main dataset epsilon dim 0`).  Each entry point below replaces one
 * reference routine; the citation names the reference interface it stands in
 * for.  The reference-signature C++ shims (gridIndexingGPU, sortByWorkLoad,
 * distanceTableNDGridBatches) in hegjoin_b200/compat/ are written on top of
 * these calls.
 *
 * Conventions
 *   - Every call returns an hj_status (0 = HJ_OK).  hj_last_error() returns a
 *     message for the most recent failure on the calling thread.
 *   - Pointers named d_* are device pointers; h_* are host pointers.
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 *     Calls enqueue work on it; only calls documented as synchronising wait.
 *   - Floating-point arguments that hold a dataset value (epsilon, minArr) are
 *     passed as double and converted to the dataset type (float for HJ_F32),
 *     the way main.cu:56 converts argv's epsilon to DTYPE.
 *   - Indices are 32-bit (the reference stores point ids as unsigned/int).
 */
#ifndef HEGJOIN_B200_H
#define HEGJOIN_B200_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int hj_status;
#define HJ_OK 0
#define HJ_ERR_INVALID 1      /* bad argument or unsupported shape */
#define HJ_ERR_CUDA 2         /* a CUDA runtime call failed */
#define HJ_ERR_OOM 3          /* device allocation failed */
#define HJ_ERR_OVERFLOW 4     /* a result buffer was too small (batch is retried internally) */
#define HJ_ERR_TIMEOUT 5      /* a bounded device-side wait expired */
#define HJ_ERR_UNSUPPORTED 6  /* input outside the supported domain (see message) */
#define HJ_ERR_NO_DEVICE 7    /* no CUDA device / kernel image for this GPU */

#define HJ_F32 0
#define HJ_F64 1

/* Refine kernels. */
#define HJ_REFINE_AUTO 0      /* tensor-core filter for d >= 16 with float data, else exact */
#define HJ_REFINE_EXACT 1     /* CUDA-core refine in the dataset type, reference order */
#define HJ_REFINE_TC_F16 2    /* tcgen05 FP16-input / FP32-accumulate filter + exact recheck */
#define HJ_REFINE_TC_BF16 3   /* tcgen05 BF16-input / FP32-accumulate filter + exact recheck */

typedef struct hj_index hj_index;
typedef struct hj_result hj_result;

/* Layout of gridCellLookup in the reference (structs.h:90-98): 16 bytes. */
typedef struct {
    uint32_t idx;
    uint32_t pad_;
    uint64_t gridLinearID;
} hj_grid_cell_lookup;

/* Layout of grid (structs.h:83-86): inclusive [indexmin, indexmax]. */
typedef struct {
    int32_t indexmin;
    int32_t indexmax;
} hj_grid;

/* Layout of schedulingCell (structs.h:101-104). */
typedef struct {
    int32_t nbPoints;
    int32_t cellId;
} hj_scheduling_cell;

/* Device neighbour-table entry: the device form of neighborTableLookup
 * (structs.h:35-41).  Query `q`'s neighbours are
 * values[batch][start .. start + count). */
typedef struct {
    uint32_t batch;
    uint32_t count;
    uint64_t start;
} hj_nt_entry;

typedef struct {
    uint32_t n, d, k, dtype;
    uint32_t n_nonempty_cells;
    uint32_t grid_aliasing;        /* 1 if some point's cell coordinate reached nCells */
    uint64_t total_cells;
    uint64_t total_candidates;     /* valid after hj_sort_by_workload */
    double eps;                    /* epsilon in the dataset type */
    double sq_threshold;           /* largest d2 with RN(sqrt(d2)) <= eps, dataset type */
    double min_arr[16];
    uint32_t n_cells[16];
} hj_index_info;

typedef struct {
    int refine;                    /* HJ_REFINE_* */
    uint64_t result_capacity;      /* pairs per batch buffer; 0 = from the estimate */
    double sample_rate;            /* estimator sample rate; 0 = 0.02 */
    double mem_fraction;           /* share of free device memory result buffers may use; 0 = 0.6 */
    uint32_t query_block;          /* queries per work item; 0 = autotuned/default */
    uint32_t max_batches;          /* safety cap on batch count; 0 = unlimited */
    uint32_t use_graphs;           /* reserved, ignored: a batch is a handful of launches */
    uint32_t keep_keys;            /* keep per-batch sorted key arrays (needed for the reference export) */
    uint32_t shard_count;          /* multi-GPU: this rank's LPT share of the work items (0 or 1 = all) */
    uint32_t shard_index;
    uint64_t device_bytes_cap;     /* cap on the device bytes of the result buffers plus the results the
                                      join keeps (hj_join: neighbour ids and table); 0 = none.  A join
                                      that cannot fit returns HJ_ERR_OOM with stats->bytes_wanted set,
                                      before its results would pass the cap */
    uint32_t stream_overlap;       /* hj_join_stream: grouped batches alternate between two sets of
                                      arrays, so a sink may read a batch on a stream of its own while
                                      the next batches run (see hj_batch_view.release_event); costs two
                                      more words of device memory per result slot.  0 = one set */
} hj_join_opts;

typedef struct {
    uint64_t total_pairs;
    uint32_t n_batches;
    uint32_t n_retries;            /* batches re-run after an overflow */
    uint64_t band_pairs;           /* tensor-core filter: pairs that needed the exact recheck */
    uint64_t tc_accepts;           /* tensor-core filter: pairs accepted outside the band */
    uint64_t estimated_pairs;      /* selectivity estimate before the join */
    double filter_delta;           /* guard band half-width on d2 (tensor-core filter) */
    float ms_estimate, ms_refine, ms_group, ms_total;
    float ms_refine_kernel;        /* device time of the refine kernels (CUDA events on the join's stream) */
    uint32_t refine_launches;      /* refine kernel launches timed in ms_refine_kernel */
    uint32_t refine_used;          /* HJ_REFINE_* actually used */
    uint32_t kernel_launches;      /* kernels launched by this join */
    float ms_setup;                /* workload order, refine choice, operand forms, work items (wall clock) */
    uint64_t bytes_wanted;         /* device bytes of result buffers + kept results the join asks for by
                                      its estimate (one batch); also filled when the cap refuses it */
} hj_join_stats;

/* ---- errors / library ---------------------------------------------------- */
const char* hj_last_error(void);
const char* hj_version(void);
/* Kernels launched by this process so far (all entry points). */
uint64_t hj_kernel_launch_count(void);

/* ---- dataset ingest: replaces importNDDataset (import_dataset.cpp:10-40) ---- */
/* Parses a text dataset the way the reference's importer does: the file split
 * into tokens at every ',', values extracted from each token as
 * `stringstream >> DTYPE` would (whitespace skipped, the C-locale number
 * grammar, strtof/strtod rounding), a token's remainder dropped after the
 * first failed extraction, and the trailing values that do not fill a point of
 * d coordinates dropped.  The file is parsed in parallel (OpenMP) with the same
 * values in the same order.  *h_values receives n_points x d values of the
 * dataset type, allocated by the library: release it with hj_host_free. */
hj_status hj_import_text(const char* path, uint32_t d, int dtype, void** h_values, uint64_t* n_points);
/* The binary twin: a 32-byte header ("HJDS0001", dtype, d, n) and the values.
 * hj_import_binary also reads the reference's raw layout (importNDDatasetBinary,
 * import_dataset.cpp:63-100: values only, n from the file size). */
hj_status hj_write_binary(const char* path, const void* h_values, uint64_t n_points, uint32_t d, int dtype);
hj_status hj_import_binary(const char* path, uint32_t d, int dtype, void** h_values, uint64_t* n_points);
void hj_host_free(void* p);

/* ---- grid geometry: replaces generateNDGridDimensions (main.cu:449-520) ---- */
/* Per indexed dimension: min/max over the points, widened by eps, nCells =
 * ceil((max - min) / eps), all in the dataset type; min/max are reduced on the
 * device.  Synchronises `stream`. */
hj_status hj_grid_geometry(const void* d_db, uint32_t n, uint32_t d, uint32_t k, int dtype,
                           double eps, double* h_min_arr, double* h_max_arr,
                           uint32_t* h_n_cells, uint64_t* h_total_cells, void* stream);

/* The same geometry without any device allocation; it has no counterpart in
 * the reference.  For callers that cannot allocate device memory where they
 * need the geometry: a process that reserves all of its device memory up
 * front (a server sized to a fixed HBM budget, or a job under a fixed quota)
 * and must not fail on an allocation later.  Its scratch is a file-scope
 * device array of 151,808 bytes (k <= 16 indexed dimensions, any n) that every
 * GPU loading the library keeps until exit; larger k is rejected with
 * HJ_ERR_INVALID.  All calls on a device share that array, so calls that
 * overlap on the GPU race: serialise them.  The first call on a device (and
 * the first after that device's context changes) looks up the array's
 * address.  The call copies its result to the host and synchronises `stream`,
 * so it must not be made on a stream that is being captured. */
hj_status hj_grid_geometry_noalloc(const void* d_db, uint32_t n, uint32_t d, uint32_t k, int dtype,
                                   double eps, double* h_min_arr, double* h_max_arr,
                                   uint32_t* h_n_cells, uint64_t* h_total_cells, void* stream);

/* ---- index build: replaces gridIndexingGPU (GPU.cu:74-398, GPU.h:9-27) ----- */
/* d_db: n x d row-major dataset on the device (float or double per dtype).
 * h_min_arr / h_n_cells: the grid geometry (k entries); NULL = compute it with
 * hj_grid_geometry.  Synchronises `stream`. */
hj_status hj_index_create(const void* d_db, uint32_t n, uint32_t d, uint32_t k, int dtype,
                          double eps, const double* h_min_arr, const uint32_t* h_n_cells,
                          void* stream, hj_index** out);
hj_status hj_index_destroy(hj_index* ix);
hj_status hj_index_get_info(const hj_index* ix, hj_index_info* out);
/* Write the reference's index arrays into caller buffers (device pointers;
 * any may be NULL): gridCellLookupArr (nNonEmpty), index (nNonEmpty),
 * indexLookupArr (n).  Enqueued on `stream`. */
hj_status hj_index_export(const hj_index* ix, hj_grid_cell_lookup* d_lookup, hj_grid* d_grid,
                          uint32_t* d_index_lookup, void* stream);
/* Device views of the index: the points reordered by cell (n x d, dataset
 * type), sorted-position -> original id, cell linear ids and cell starts
 * (nNonEmpty + 1 entries). */
hj_status hj_index_views(const hj_index* ix, const void** d_points_sorted, const uint32_t** d_perm,
                         const uint64_t** d_cell_lid, const uint32_t** d_cell_start);

/* ---- workload order: replaces sortByWorkLoad (SortByWorkload.cu:19-247) ---- */
/* Candidate count per non-empty cell (summed populations of its 3^k stencil),
 * cells ordered heaviest first (stable among equals), totalCandidates.
 * Synchronises `stream`. */
hj_status hj_sort_by_workload(hj_index* ix, void* stream, uint64_t* total_candidates);
/* Export the ordered schedulingCell array (nNonEmpty) and originPointIndex (n)
 * to device buffers (either may be NULL). */
hj_status hj_workload_export(const hj_index* ix, hj_scheduling_cell* d_sched,
                             uint32_t* d_origin_point_index, void* stream);

/* ---- join: replaces distanceTableNDGridBatches (GPU.cu:787-1702) ---------- */
void hj_join_opts_default(hj_join_opts* o);
/* Runs estimator, batches, refine and result grouping.  The result keeps, per
 * batch, the neighbour ids grouped by query (device memory) plus a device
 * neighbour table of n entries.  Synchronises `stream`.  The result's memory is
 * released in the order of `stream`, which must outlive the result. */
hj_status hj_join(hj_index* ix, const hj_join_opts* opts, void* stream, hj_result** out,
                  hj_join_stats* stats);
hj_status hj_result_destroy(hj_result* r);
hj_status hj_result_num_batches(const hj_result* r, uint32_t* n_batches, uint64_t* total_pairs);
/* Batch b: device pointers to its values (and keys when keep_keys was set),
 * grouped by query id, and its pair count. */
hj_status hj_result_batch(const hj_result* r, uint32_t b, const uint32_t** d_vals,
                          const uint32_t** d_keys, uint64_t* count);
/* Device neighbour table (n entries, indexed by original query id). */
hj_status hj_result_table(const hj_result* r, const hj_nt_entry** d_table);
/* Per-query CSR by original id into caller buffers: d_offsets (n + 1, u64) and
 * d_vals (total_pairs, u32); neighbours of a query in ascending id order when
 * sort_lists is set.  Enqueued on `stream`. */
hj_status hj_result_to_csr(const hj_result* r, uint64_t* d_offsets, uint32_t* d_vals, int sort_lists,
                           void* stream);
/* Per-query order-independent digest (count, sum of mix64(id), xor of
 * mix64(id ^ salt)) into device buffers of n entries. */
hj_status hj_result_digest(const hj_result* r, uint32_t* d_count, uint64_t* d_sum, uint64_t* d_xor,
                           void* stream);

/* ---- streamed join: results larger than device memory ----------------------- */
/* One grouped batch handed to a sink: `count` pairs, query ids ascending in
 * d_keys and their neighbour ids in d_vals (device memory, in the order of the
 * join's stream).  The reference's counterpart is the per-batch copy-out and
 * host table build of distanceTableNDGridBatches (GPU.cu:1542-1573). */
typedef struct {
    uint32_t batch;                /* 0, 1, ... in the order the batches complete */
    uint32_t pad_;
    uint64_t count;
    const uint32_t* d_keys;
    const uint32_t* d_vals;
    void* release_event;           /* set by the sink (optional, with stream_overlap): a cudaEvent_t
                                      recorded after its last use of d_keys / d_vals; NULL on entry */
} hj_batch_view;
/* Called on the joining thread once per batch.  The arrays stay valid for work
 * the sink enqueues on `stream` (copies, kernels): the next batch reuses them
 * only after that work, in stream order.  With hj_join_opts.stream_overlap the
 * arrays are not touched again until two batches later, and a sink may instead
 * use them from a stream of its own (after waiting for an event it records on
 * `stream`) and hand back, in release_event, an event recorded after that use:
 * the join waits for it before it reuses the arrays and before it returns.
 * The event must stay valid until hj_join_stream returns.  Return HJ_OK to
 * continue; any other status stops the join and is returned by hj_join_stream. */
typedef hj_status (*hj_batch_sink)(hj_batch_view* batch, void* user, void* stream);

/* The join of hj_join with nothing kept on the device: each batch is grouped by
 * query id and handed to `sink` (may be NULL), and its buffers are reused by
 * the next batch, so the result may exceed device memory.  When d_count, d_sum
 * and d_xor (n entries each, device) are given they receive the per-query
 * digest of hj_result_digest, accumulated over the batches (they are zeroed
 * first).  Synchronises `stream`. */
hj_status hj_join_stream(hj_index* ix, const hj_join_opts* opts, hj_batch_sink sink, void* user,
                         uint32_t* d_count, uint64_t* d_sum, uint64_t* d_xor, void* stream,
                         hj_join_stats* stats);

/* ---- multi-GPU sharding ----------------------------------------------------- */
/* The work items a rank processes out of `n_items` heaviest-first items when
 * the join runs with shard_count ranks: items first, first + stride, ... (n_mine
 * of them).  Host-only arithmetic; hj_join applies exactly this selection. */
hj_status hj_shard_plan(uint32_t n_items, uint32_t shard_count, uint32_t shard_index, uint32_t* first,
                        uint32_t* stride, uint32_t* n_mine);
/* The items a rank processes under greedy LPT (longest processing time first):
 * items by cost, descending (ties by index), each to the least-loaded rank
 * (ties to the lowest rank).  Writes this rank's item indices, ascending, to
 * items (capacity n_items) and their number to n_mine.  Host-only arithmetic;
 * hj_join with shard_count > 1 applies it with cost = candidates x queries per
 * work item, so every rank derives the same partition. */
hj_status hj_shard_plan_lpt(const uint64_t* costs, uint32_t n_items, uint32_t shard_count, uint32_t shard_index,
                            uint32_t* items, uint32_t* n_mine);

/* ---- one-shot convenience: host buffers in, host pair count out ------------ */
/* Copies the dataset to the device, builds the index, sorts by workload and
 * joins; the result stays on the device in *out (may be NULL to discard). */
hj_status hj_self_join_host(const void* h_db, uint32_t n, uint32_t d, uint32_t k, int dtype, double eps,
                            const hj_join_opts* opts, void* stream, hj_result** out,
                            hj_join_stats* stats);

/* ---- serving: continuous batching of self-join requests ------------------------ */
/* Beyond the reference (one dataset per process).  Requests are admitted in
 * arrival order as soon as a worker is free and their device-memory
 * reservation fits hbm_budget; each worker runs a request's copy-in, index,
 * workload order and join on its own stream, so concurrent requests overlap on
 * the device.  The host dataset passed to hj_server_submit must stay valid
 * until hj_server_wait returns for that ticket. */
typedef struct hj_server hj_server;
typedef struct {
    uint64_t hbm_budget;           /* bytes; 0 = 150 GiB */
    uint32_t workers;              /* concurrent requests; 0 = 1 */
    int refine;                    /* HJ_REFINE_* for every request */
} hj_server_opts;
typedef struct {
    hj_status status;
    double t_submit, t_admit, t_done;   /* steady-clock seconds */
    hj_join_stats stats;
    uint64_t reserved_bytes;       /* device bytes the request held against the budget while it ran */
    uint32_t regrants;             /* times its join asked for a larger allowance than the first */
} hj_serve_info;
void hj_server_opts_default(hj_server_opts* o);
hj_status hj_server_create(const hj_server_opts* opts, hj_server** out);
hj_status hj_server_submit(hj_server* s, const void* h_db, uint32_t n, uint32_t d, uint32_t k, int dtype,
                           double eps, uint64_t* ticket);
/* Blocks until the request is done (or timeout_s passes: HJ_ERR_TIMEOUT).
 * The result (device memory) passes to the caller when `result` is non-NULL,
 * else it is released; it is tied to the legacy default stream, so it may
 * outlive the server. */
hj_status hj_server_wait(hj_server* s, uint64_t ticket, double timeout_s, hj_result** result,
                         hj_serve_info* info);
/* Bytes held against the budget now (running requests' reservations, the
 * workers' 256 MB workspaces and uncollected results) and the most ever held.
 * A request admitted while nothing else runs may pass the budget alone. */
hj_status hj_server_usage(hj_server* s, uint64_t* in_use, uint64_t* peak_in_use);
hj_status hj_server_destroy(hj_server* s);

/* ---- fault injection and accounting for tests --------------------------------- */
/* Arms the library's device-allocation fault injection: the nth device
 * allocation from now (n >= 1) fails as an out-of-memory would; 0 disarms.
 * No reference counterpart: it exercises every error path's clean-up. */
void hj_debug_fail_alloc(uint64_t nth);
/* Bytes currently allocated from the device's default memory pool (the pool
 * every stream-ordered allocation of the library comes from). */
hj_status hj_debug_pool_used(uint64_t* bytes);
/* The most device memory the library's pool has held since the last reset;
 * reset != 0 restarts the count from what is held now. */
hj_status hj_debug_pool_peak(uint64_t* bytes, int reset);

/* ---- measured peaks (roofline denominators) ---------------------------------- */
/* Throughput of the pipes the refine kernels run on, measured by this library's
 * own kernels with CUDA events on `stream` (each runs over every SM for a few to
 * tens of ms): FP32 FMA chains (scalar and the packed f32x2 form the exact refine
 * uses), FP64 FMA chains, and tensor-core kind::f16 MMAs of M = 128, N = 256,
 * K = 16 issued back to back by two threads per SM into TMEM (the filter's issue
 * pattern), with FP16 and with BF16 inputs.  A flop is one multiply or one add.
 * No reference counterpart.  Synchronises `stream`. */
typedef struct {
    double fp32_fma_tflops;
    double fp32x2_fma_tflops;
    double fp64_fma_tflops;
    double f16_mma_tflops;
    double bf16_mma_tflops;
} hj_peaks;
hj_status hj_measure_peaks(hj_peaks* out, void* stream);

/* ---- probes --------------------------------------------------------------- */
/* Evaluates the reference's squared-distance expression (kernel.cu:350-353)
 * as nvcc compiles it by default, for n pairs of d-dimensional rows; writes
 * d2 per pair.  Used to establish the FMA contraction the reference gets. */
hj_status hj_probe_sqdist(const void* d_a, const void* d_b, uint32_t n, uint32_t d, int dtype,
                          void* d_out, void* stream);

/* Evaluates one candidate tile (128 rows from sorted position a0) against 512
 * query rows (from sorted position b0) through the tensor-core filter's TMA
 * and tcgen05 path, writing the 128 x 512 FP32 accumulators (row = candidate,
 * column = query) to d_out.  Optionally copies the quantised operand rows
 * (query form 512 x kpad and candidate form 128 x kpad, 16-bit, kpad =
 * 32 * ceil((d + 4) / 32)) to host buffers.  Synchronises `stream`.  The
 * operand rows and accumulators are in the filter's scaled units: divide rows
 * by 2^s and accumulators by 4^s, s from hj_tc_operand_scale. */
hj_status hj_probe_tc_tile(hj_index* ix, int refine_kind, uint32_t a0, uint32_t b0, float* d_out,
                           void* h_query_rows, void* h_cand_rows, void* stream);

/* Failure-detection check of the tensor-core pipeline's bounded waits: one tile
 * probe launch whose MMA issuer issues neither MMAs nor their commit (after its
 * operand loads have landed), so the epilogue's wait on the commit barrier runs
 * out after wait_cycles SM cycles.  The kernel then raises its error flag,
 * releases its tensor memory and returns; the call returns HJ_ERR_TIMEOUT and
 * the context stays usable.  No reference counterpart. */
hj_status hj_probe_tc_wait_timeout(hj_index* ix, int refine_kind, uint64_t wait_cycles, void* stream);

/* The power-of-two exponent s of the tensor-core operand forms last prepared
 * for this index: they hold (x - min) * 2^s, chosen per dataset so that every
 * stored half is finite.  Internal to the filter (no reference counterpart);
 * exposed for the probes and tests. */
hj_status hj_tc_operand_scale(const hj_index* ix, int* log2_scale);

#ifdef __cplusplus
}
#endif

#endif /* HEGJOIN_B200_H */

/*
 * warren_cuda.h — the C ABI of the B200 (sm_100a) backend for pg_warren's
 * whole-graph compute path.
 *
 * pg_warren names a kernel seam between its SQL adapters and whatever runs a
 * kernel (the `Kernels` trait that the reference's top-level design document
 * proposes, its lines 1208-1243; today the free functions of warren-core).  Every entry point below replaces one
 * of those functions for one dense-id graph version; the comment on each
 * names the reference function (path within the reference project, file:line)
 * whose arguments, results and errors it keeps.
 *
 * Conventions shared by every call:
 *  - Plain pointers and sizes only.  A pointer to an operand may be a host
 *    pointer (pageable or pinned) or a device pointer of the handle's device;
 *    the library tells them apart itself (cudaPointerGetAttributes).
 *  - Dense ids are the reference's DenseId (u64 on the ABI); the device copy
 *    stores them as u32, so an id space of 2^32 or more is not served
 *    (WC_UNSUPPORTED, and the adapter keeps the native kernel: `serves`).
 *  - Every call returns a wc_status mirroring the reference's error enums
 *    1:1 (ComputeError in compute/error.rs:10-208, TraversalError in
 *    traversal/error.rs, SpectralError in spectral/error.rs).  A call never
 *    aborts; device-side arithmetic errors go to an error word that the call
 *    turns into its status.
 *  - Device memory (the version's copy and each call's scratch) is charged to
 *    a wc_budget before it is allocated, as the reference charges its
 *    ComputeMemory (compute/memory.rs:31-227); a refused charge is
 *    WC_MEMORY_LIMIT with requested/in_use/limit in the detail.
 *  - Cancellation: the call polls `wc_call.cancel` (a host word the caller
 *    sets, e.g. from a signal handler) between launches and at least every
 *    millisecond while it waits, and returns WC_CANCELLED.
 */
#ifndef WARREN_CUDA_H
#define WARREN_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WC_ABI_VERSION 1

/* ------------------------------------------------------------------ status */

typedef enum wc_status {
    WC_OK = 0,
    /* ComputeError (compute/error.rs) */
    WC_MEMORY_LIMIT = 1,          /* MemoryLimit {requested, in_use, limit} */
    WC_OUT_OF_MEMORY = 2,         /* OutOfMemory {bytes} */
    WC_DTYPE_MISMATCH = 3,        /* DtypeMismatch */
    WC_ID_SPACE_MISMATCH = 4,     /* IdSpaceMismatch */
    WC_WIDTH_MISMATCH = 5,        /* WidthMismatch */
    WC_UNKNOWN_SEMIRING = 6,      /* UnknownSemiring */
    WC_UNKNOWN_BINARY_OP = 7,     /* UnknownBinaryOp */
    WC_ZERO_WIDTH = 8,            /* ZeroWidth */
    WC_CANCELLED = 9,             /* Cancelled */
    /* ArithmeticError (compute/error.rs:180-208) */
    WC_BIGINT_OUT_OF_RANGE = 10,  /* BigintOutOfRange */
    WC_FLOAT_OVERFLOW = 11,       /* FloatOverflow */
    WC_FLOAT_UNDERFLOW = 12,      /* FloatUnderflow */
    WC_DIVISION_BY_ZERO = 13,     /* DivisionByZero */
    WC_SQRT_OF_NEGATIVE = 14,     /* SqrtOfNegative */
    WC_LOG_OF_ZERO = 15,          /* LogOfZero */
    WC_LOG_OF_NEGATIVE = 16,      /* LogOfNegative */
    WC_ZERO_TO_NEGATIVE_POWER = 17, /* ZeroToNegativePower */
    WC_COMPLEX_POWER = 18,        /* ComplexPower */
    /* TraversalError (traversal/error.rs) */
    WC_NODE_OUTSIDE_ID_SPACE = 20,  /* NodeOutsideIdSpace {node} */
    WC_NODE_FILTER_ID_SPACE = 21,   /* NodeFilterIdSpace {expected, found} */
    WC_REVERSE_CSR_MISSING = 22,    /* ReverseCsrMissing */
    /* SpectralError (spectral/error.rs) */
    WC_NOT_SYMMETRIC = 30,          /* NotSymmetric */
    WC_NON_POSITIVE_DEGREE = 31,    /* NonPositiveDegree {node, degree} */
    WC_EIGENPAIR_COUNT = 32,        /* EigenpairCount {k, dimension} */
    WC_WORKING_SET = 33,            /* WorkingSet {bytes, in_use, limit} */
    WC_NOT_FINITE = 34,             /* NotFinite */
    /* GraphError (graph/error.rs), from wc_version_load_segments */
    WC_SEGMENT_TRUNCATED = 50,          /* SegmentTruncated */
    WC_SEGMENT_MAGIC = 51,              /* SegmentMagic */
    WC_SEGMENT_FORMAT = 52,             /* SegmentFormat {found} */
    WC_SEGMENT_KIND = 53,               /* SegmentKind {expected, found} */
    WC_SEGMENT_RESERVED = 54,           /* SegmentReserved {found} */
    WC_SEGMENT_WIDTH = 55,              /* SegmentWidth {expected, found} */
    WC_SEGMENT_LENGTH = 56,             /* SegmentLength {expected, found} */
    WC_OFFSETS_LENGTH = 57,             /* OffsetsLength {expected, found} */
    WC_FIRST_OFFSET_NOT_ZERO = 58,      /* FirstOffsetNotZero */
    WC_STORED_ROWS_NOT_ASCENDING = 59,  /* StoredRowsNotAscending {index: node} */
    WC_STORED_ROW_OUTSIDE_ID_SPACE = 60, /* StoredRowOutsideIdSpace {row: node} */
    WC_STORED_ROW_EMPTY = 61,           /* StoredRowEmpty {row: node} */
    WC_OFFSETS_NOT_MONOTONE = 62,       /* OffsetsNotMonotone {row: node} */
    WC_FINAL_OFFSET = 63,               /* FinalOffset {expected, found} */
    WC_TARGET_OUTSIDE_ID_SPACE = 64,    /* TargetOutsideIdSpace {row: node, target: found} */
    WC_ROW_NOT_SORTED = 65,             /* RowNotSorted {row: node} */
    WC_WEIGHTS_LENGTH = 66,             /* WeightsLength {expected, found} */
    /* ComputeError, from wc_vector_map */
    WC_UNKNOWN_OPERAND = 70,            /* UnknownOperand {index: node, operands: expected} */
    WC_OPERAND_TYPE = 71,               /* OperandType {index: node, expected, found} (wc_dtype) */
    WC_NULL_RESULT = 72,                /* NullResult {dtype: expected} */
    /* the backend's own */
    WC_INVALID_ARGUMENT = 40,       /* a null pointer, a bad enum value, ... */
    WC_UNSUPPORTED = 41,            /* not served here: the adapter keeps the native kernel */
    WC_CUDA_ERROR = 42,             /* a CUDA runtime error; detail.cuda_error */
    WC_DEVICE_TIMEOUT = 43,         /* a bounded device-side wait ran out */
    WC_NO_DEVICE = 44               /* no usable sm_100 device */
} wc_status;

/* What went wrong, beyond the status.  Any field may be zero. */
typedef struct wc_error_detail {
    uint64_t requested;  /* MemoryLimit / OutOfMemory / WorkingSet: bytes */
    uint64_t in_use;
    uint64_t limit;
    uint64_t node;       /* NodeOutsideIdSpace / NonPositiveDegree: dense id */
    uint64_t expected;   /* *Mismatch: expected / found */
    uint64_t found;
    double degree;       /* NonPositiveDegree */
    int32_t cuda_error;  /* WC_CUDA_ERROR: the cudaError_t */
    char message[200];   /* a one-line description */
} wc_error_detail;

/* The message of a status ("division by zero", ...), as the reference's
 * Display impls word them. */
const char* wc_status_name(wc_status status);

/* ------------------------------------------------------------ element types */

/* compute/dtype.rs:12-21, in the same order. */
typedef enum wc_dtype { WC_F32 = 0, WC_F64 = 1, WC_I64 = 2, WC_BOOL = 3 } wc_dtype;

/* compute/semiring.rs:15-38 (BinaryOp), in declaration order. */
typedef enum wc_binary_op {
    WC_OP_FIRST = 0, WC_OP_SECOND = 1, WC_OP_PAIR = 2, WC_OP_PLUS = 3, WC_OP_TIMES = 4,
    WC_OP_MIN = 5, WC_OP_MAX = 6, WC_OP_LOR = 7, WC_OP_LAND = 8, WC_OP_ANY = 9,
    WC_OP_NONE = -1 /* no accumulator */
} wc_binary_op;

/* compute/semiring.rs:118-146 (Semiring), in declaration order. */
typedef enum wc_semiring {
    WC_PLUS_TIMES = 0, WC_MIN_PLUS = 1, WC_MAX_PLUS = 2, WC_MAX_TIMES = 3, WC_MIN_TIMES = 4,
    WC_LOR_LAND = 5, WC_ANY_PAIR = 6, WC_PLUS_PAIR = 7, WC_PLUS_FIRST = 8, WC_PLUS_SECOND = 9,
    WC_MIN_FIRST = 10, WC_MIN_SECOND = 11, WC_MAX_SECOND = 12
} wc_semiring;

/* graph/direction.rs:6-13. */
typedef enum wc_direction { WC_OUT = 0, WC_IN = 1, WC_BOTH = 2 } wc_direction;

/* ----------------------------------------------------------- runtime handles */

typedef struct wc_budget wc_budget;     /* device memory budget (ComputeMemory) */
typedef struct wc_version wc_version;   /* a version's device CSR + CSC */

/* A budget of `limit` bytes of device memory (ComputeMemory::new,
 * compute/memory.rs).  Thread-safe. */
wc_status wc_budget_create(uint64_t limit, wc_budget** out);
/* Drops the caller's hold on the budget; a version charged to it keeps it
 * until that version is released, so the two may go in either order. */
void wc_budget_destroy(wc_budget* budget);
uint64_t wc_budget_in_use(const wc_budget* budget);
uint64_t wc_budget_peak(const wc_budget* budget);

/* Progress (progress.rs:9-16): a phase starting with an optional total, then
 * units done.  `total` is UINT64_MAX when unknown. */
typedef void (*wc_progress_fn)(void* context, const char* phase, uint64_t done, uint64_t total);

/* What a call is given besides its operands: the seam's `Call` (the
 * reference's design document, lines 1213-1220) plus the stream the work
 * goes on. */
typedef struct wc_call {
    wc_budget* memory;             /* the call's budget: the working memory it uses is charged
                                      here for the call's duration (WC_MEMORY_LIMIT past it);
                                      the device memory itself stays in the version's pool,
                                      charged to the version's budget.  NULL: none */
    volatile const int32_t* cancel; /* non-zero: stop (WC_CANCELLED); may be NULL */
    wc_progress_fn progress;       /* may be NULL */
    void* progress_context;
    void* stream;                  /* cudaStream_t; NULL: the version's own stream */
    uint32_t flags;                /* WC_CALL_* */
    uint32_t timeout_ms;           /* bound on any wait for the device; 0: 600000 */
    wc_error_detail* detail;       /* filled on error; may be NULL */
} wc_call;

/* With device operands only: return once the work is queued on the stream,
 * without waiting for it; errors found on the device are reported by the next
 * call on the version, or by wc_version_sync. */
#define WC_CALL_ASYNC 1u
/* Record CUDA events around the call's kernel groups ("level", "depth",
 * "iteration", ...) on its stream; read them with wc_version_timing. */
#define WC_CALL_TIMING 2u

/* -------------------------------------------------------------- versions */

/* A built version's adjacency as the reference holds it (graph/csr/mod.rs:
 * 38-237): offsets u64[n+1], targets u32[m] ascending and distinct within a
 * row, weights f64[m] or NULL (every weight 1).  The reverse CSR
 * (graph/csr/graph_csr.rs:15-55, transpose.rs:1-30) may be given; without it
 * the device builds its own by transposing, counted in the budget.  Only a
 * single merged CSR is uploaded: the relation selection "all relations" of
 * every call reads it (product/matrix.rs:126-157). */
typedef struct wc_csr_host {
    uint64_t id_space;
    uint64_t edges;
    const uint64_t* offsets;
    const uint32_t* targets;
    const double* weights;
    const uint64_t* reverse_offsets;  /* NULL: built on the device */
    const uint32_t* reverse_targets;
    const double* reverse_weights;
    /* With reverse_offsets NULL: nonzero when the version has a reverse CSR
     * (RelationCsr.reverse), built here on the device from the forward one;
     * zero when it has none (the device still builds one for the pull, but
     * traversals In / Both report WC_REVERSE_CSR_MISSING). */
    int32_t reverse_on_device;
} wc_csr_host;

/* graph/segment/csr.rs:83-122 (AnyCsr::decode) straight into a device copy:
 * a version's CSR segments as stored (a 16-byte header, then the
 * little-endian payload; rows_segment only with sparse offsets, weights
 * NULL when unweighted), checked as Csr::from_segments checks them
 * (graph/csr/mod.rs:78-137, the first violation reported in the order the
 * reference checks) and uploaded without a host-side decode; the reverse
 * CSR is built on the device.  has_reverse: the version has a reverse CSR
 * (as wc_csr_host.reverse_on_device). */
wc_status wc_version_load_segments(uint64_t graph_id, uint64_t version, uint64_t id_space,
                                   const uint8_t* rows_segment, uint64_t rows_len,
                                   const uint8_t* offsets_segment, uint64_t offsets_len,
                                   const uint8_t* targets_segment, uint64_t targets_len,
                                   const uint8_t* weights_segment, uint64_t weights_len,
                                   int32_t has_reverse, wc_budget* budget, const wc_call* call,
                                   wc_version** out);

typedef struct wc_version_info {
    uint64_t id_space;
    uint64_t edges;
    uint64_t device_bytes;     /* charged to the budget */
    int32_t weighted;          /* the CSR has weights */
    int32_t integral_weights;  /* every weight is an integer in int32 range: an int32 copy is kept */
    int32_t device;            /* CUDA ordinal */
    int32_t symmetric;         /* the CSR equals its transpose (values included) */
    uint64_t scratch_bytes;    /* calls' working memory kept between calls (also charged) */
} wc_version_info;

/* Uploads `csr` for (graph_id, version) to the current device: the derived
 * device copy the seam keys by version (the reference's design document,
 * line 1240).  Charged to
 * `budget` (the version holds it until wc_version_release). */
wc_status wc_version_upload(uint64_t graph_id, uint64_t version, const wc_csr_host* csr,
                            wc_budget* budget, const wc_call* call, wc_version** out);
wc_status wc_version_release(wc_version* version);
wc_status wc_version_info_get(const wc_version* version, wc_version_info* info);
/* Waits for the version's stream and reports a pending device error. */
wc_status wc_version_sync(wc_version* version, const wc_call* call);

/* The device time (ms, CUDA events on the call's stream) of kernel group
 * `phase` in the last call made with WC_CALL_TIMING, and in *launches the
 * kernels it launched in that group (may be NULL); 0 if not recorded.
 * Groups: "setup", "iteration" (PageRank); "level" (a batched search's levels: push,
 * settle and pull launches), "pull" (the pull launches alone), "depth";
 * "pulled" has no time and counts the levels that pulled. */
double wc_version_timing(const wc_version* version, const char* phase, uint32_t* launches);

/* The number of kernels this library has launched since it was loaded
 * (a diagnostic: the count a benchmark reports for its timed region). */
uint64_t wc_kernel_launches(void);

/* compute/random.rs:11-25 (uniform) on the device, the generator wc_eigen
 * draws its start vectors from: out[i] = uniform(seed, stream, i) over the
 * version's id space, in [-1, 1) (a diagnostic, so that the device values
 * can be compared with the reference's bit for bit). */
wc_status wc_random_uniform(wc_version* version, const wc_call* call, uint64_t seed,
                            uint64_t stream, double* out);

/* Runs, on the current device, one kernel that waits on a shared-memory
 * barrier nothing completes, through the same bounded wait the kernels'
 * bulk-copy rings use, with a limit of `limit_us` microseconds (at most
 * 2 s).  The wait gives up, the kernel records WC_DEVICE_TIMEOUT and
 * returns, and so does this call: a self-test that a device wait which
 * runs out ends with a status and leaves the device usable. */
wc_status wc_selftest_bounded_wait(const wc_call* call, uint32_t limit_us);

/* Whether this backend serves `operation` over `dtype` (the seam's
 * `Kernels::serves`, the reference's design document, line 1224).  Operations: "spmv", "spmm", "pagerank",
 * "bfs", "reachable_set", "eigen", "vector_topk". */
int32_t wc_serves(const char* operation, wc_dtype dtype);

/* -------------------------------------------------------------- products */

/* A value mask (compute/mask.rs:11-45): row i is written when mask[i] is
 * non-zero (NaN included), or zero with `complement`. */
typedef struct wc_mask {
    const void* values;   /* id_space elements of `dtype` */
    wc_dtype dtype;
    int32_t complement;
} wc_mask;

/* compute/product/mod.rs:31-56 (Product), for the all-relations selection. */
typedef struct wc_product {
    wc_semiring semiring;
    int32_t transpose;       /* y = Aᵀ ⊗ x */
    int32_t weighted;        /* -1: if the graph has weights; 0: every weight 1; 1: weights */
    const wc_mask* mask;     /* NULL: every row */
    int32_t replace;
    wc_binary_op accumulate; /* WC_OP_NONE: overwrite */
} wc_product;

/* SpMV y = A ⊗ x (or Aᵀ ⊗ x) over width-1 vectors of `dtype`:
 * compute/product/mod.rs:77-92 (spmv).  `y` holds the values kept where the
 * mask leaves rows unwritten or `accumulate` combines (compute_sql/product.rs:
 * 101-109 fills it). */
wc_status wc_spmv(wc_version* version, const wc_call* call, const wc_product* product,
                  wc_dtype dtype, const void* x, void* y);

/* SpMM Y = A ⊗ X for row-major id_space × width matrices:
 * compute/product/mod.rs:97-110 (spmm). */
wc_status wc_spmm(wc_version* version, const wc_call* call, const wc_product* product,
                  wc_dtype dtype, uint32_t width, const void* x, void* y);

/* -------------------------------------------------------------- pagerank */

/* compute/pagerank/mod.rs:27-47 (PageRank), all relations. */
typedef struct wc_pagerank_opts {
    double damping;
    double tol;              /* used when has_tol */
    int32_t has_tol;         /* 0: run every iteration */
    int32_t weighted;        /* -1 / 0 / 1 as wc_product.weighted */
    uint32_t max_iter;
    const double* seed;      /* personalisation (width-1 f64); NULL: uniform */
} wc_pagerank_opts;

/* compute/pagerank/mod.rs:96-151 (pagerank): ranks over the live nodes
 * (`tombstones`, graph/tombstones.rs: bit i of word i/64 marks dense id i
 * deleted; NULL: none), zero at tombstoned rows. */
wc_status wc_pagerank(wc_version* version, const wc_call* call, const wc_pagerank_opts* opts,
                      const uint64_t* tombstones, double* ranks, uint32_t* iterations);

/* No reference counterpart.  wc_pagerank without any allocation: the call's
 * working memory (ranks, messages, out-weights, tombstones, stop-test
 * scalars; 40 bytes a node plus 16 an iteration) is a fixed 64 MiB array in
 * the library's device globals, enough for about 1.67 million nodes at 100
 * iterations; larger solves return WC_WORKING_SET with detail.requested and
 * detail.limit set.  For callers that must not allocate while serving (device
 * memory held by another allocator; no cudaMalloc/cudaFree on a latency
 * budget).  Results equal wc_pagerank's.  Seeded (personalised) solves and
 * WC_CALL_TIMING are not offered.  The array is shared by every call on a
 * device: calls are serialised per device and return (errors included)
 * after their kernels finish, and any other use overlapping one on that
 * device would race.  The progress hook is called before and after the
 * solve with no lock held, so it may itself call this entry point.  The
 * first call on each device looks the array's address up with that device
 * current; make it before any stream capture on that device. */
wc_status wc_pagerank_noalloc(wc_version* version, const wc_call* call,
                              const wc_pagerank_opts* opts, const uint64_t* tombstones,
                              double* ranks, uint32_t* iterations);

/* No reference counterpart (warren-core solves on one host): one rank's part
 * of a row-partitioned PageRank over several GPUs.  The solve's rows (the
 * numbering wc_pagerank iterates in: nodes by out-degree, largest first) are
 * cut into `parts` ranges of about equal entries; every rank holds the whole
 * version and pulls its range each iteration, and between iterations the
 * caller sums the parts' L1 changes and dangling ranks and gathers the
 * parts' rows of the next message vector (one all-reduce of two scalars and
 * one all-gather of 8·id_space bytes an iteration, over NCCL).  Results
 * equal wc_pagerank's within the PageRank tolerance (the sums are grouped by
 * part), with equal iteration counts.
 *
 * wc_pagerank_part_rows: the parts' first rows, row_bounds[parts + 1]. */
wc_status wc_pagerank_part_rows(wc_version* version, uint32_t parts, uint64_t* row_bounds);

typedef struct wc_pagerank_part_info {
    uint64_t row_begin, row_end;  /* this part's rows in the solve's numbering */
    uint64_t id_space;
    uint64_t live;                /* live (untombstoned) nodes */
    double dangling;              /* iteration 0's dangling rank (the same on every part) */
    double threshold;             /* stop when the summed L1 change is below this (0: no tol) */
} wc_pagerank_part_info;

/* Sets up part `part` of `parts`: ranks2 and messages2 are the caller's
 * device vectors, 2 × id_space doubles each (even and odd iterations, the
 * solve's numbering); every row of ranks2[0..n) and messages2[0..n) gets
 * the start vector and its messages.  Tombstones as wc_pagerank's;
 * personalised solves are WC_UNSUPPORTED. */
wc_status wc_pagerank_part_begin(wc_version* version, const wc_call* call,
                                 const wc_pagerank_opts* opts, const uint64_t* tombstones,
                                 uint32_t parts, uint32_t part, double* ranks2,
                                 double* messages2, wc_pagerank_part_info* info);
/* Iteration `iteration` over the part's rows, given that iteration's summed
 * dangling rank: reads messages2[iteration & 1] (every row), writes the
 * part's rows of ranks2 and messages2 [(iteration + 1) & 1], waits, and
 * returns the part's L1 change and next dangling rank in sums[0], sums[1]. */
wc_status wc_pagerank_part_step(wc_version* version, const wc_call* call, uint32_t iteration,
                                double dangling, double* sums);
/* After `iterations` iterations, with every part's rows of
 * ranks2[iterations & 1] gathered by the caller: the ranks in dense-id
 * order (host or device), as wc_pagerank returns them.  Ends the part. */
wc_status wc_pagerank_part_end(wc_version* version, const wc_call* call, uint32_t iterations,
                               double* ranks);

/* No reference counterpart (warren-core multiplies on one host): one rank's
 * part of a row-partitioned wc_spmv over several GPUs.  The rows of the
 * product's CSR (forward, or reverse with `transpose`) are cut into `parts`
 * ranges of about equal entries, at unit boundaries of its schedule; every
 * rank holds the whole version and the whole x, and computes its range of
 * y, which the caller then gathers (one all-gather of y's rows a product).
 * The part's rows equal wc_spmv's bit for bit (the same kernel folds each
 * row the same way); y's other rows are left as given.
 *
 * wc_spmv_part_rows: the parts' first rows, row_bounds[parts + 1]. */
wc_status wc_spmv_part_rows(wc_version* version, int32_t transpose, uint32_t parts,
                            uint64_t* row_bounds);
wc_status wc_spmv_part(wc_version* version, const wc_call* call, const wc_product* product,
                       wc_dtype dtype, uint32_t parts, uint32_t part, const void* x, void* y);

/* The stop test's margin of the last iteration run: delta / (live × tol).
 * Available after wc_pagerank on the same version (diagnostics). */
double wc_pagerank_last_margin(const wc_version* version);

/* ------------------------------------------------------------- traversal */

/* traversal/stats.rs:12-23 (TraversalStats). */
typedef struct wc_traversal_stats {
    uint64_t nodes_visited;
    uint64_t edges_traversed;
    int32_t truncated;
    uint32_t levels;         /* levels expanded */
    uint32_t pulled_levels;  /* of which pulled (reachable_set) */
} wc_traversal_stats;

/* traversal/limits.rs:4-12 (Limits); UINT32_MAX / UINT64_MAX: unbounded. */
typedef struct wc_limits {
    uint32_t max_depth;
    uint64_t max_results;
} wc_limits;

#define WC_UNREACHED UINT32_MAX
#define WC_NO_VIA UINT64_MAX

/* traversal/bfs.rs:34-60 (bfs / bfs_each) over the all-relations adjacency
 * read in `direction`, node filter `filter` (NodeSet bitmap words; NULL:
 * none).  Per node: depth_out[i] its depth (WC_UNREACHED if not visited) and
 * via_out[i] the node it was first reached from (WC_NO_VIA for a start or an
 * unvisited node) — the same (node, depth, via) the reference's visits carry.
 * Either output may be NULL. */
wc_status wc_bfs(wc_version* version, const wc_call* call, wc_direction direction,
                 const uint64_t* starts, uint64_t start_count, const wc_limits* limits,
                 const uint64_t* filter, uint32_t* depth_out, uint64_t* via_out,
                 wc_traversal_stats* stats);

/* The visits of wc_bfs in the reference's order (by depth; within a depth,
 * the previous depth's nodes expanded in ascending dense id, each row in
 * ascending target order), truncated at max_results as bfs truncates:
 * visits_out[3*r .. 3*r+2] = (node, depth, via).  `capacity` rows;
 * *count gets the number written. */
wc_status wc_bfs_visits(wc_version* version, const wc_call* call, wc_direction direction,
                        const uint64_t* starts, uint64_t start_count, const wc_limits* limits,
                        const uint64_t* filter, uint64_t* visits_out, uint64_t capacity,
                        uint64_t* count, wc_traversal_stats* stats);

/* traversal/bfs_cursor.rs:17-138 (BfsCursor): wc_bfs run one level per
 * call, so a caller that stops asking (SQL LIMIT) stops the search.
 * wc_bfs_cursor_open is BfsCursor::new (:40-73) — every argument is
 * checked, the starts are admitted on the device, and later calls fail
 * only when cancelled, timed out or out of memory — or, with
 * reachable_set != 0, BfsCursor::reachable_set (:75-88): `filter` NULL and
 * max_results unbounded, levels may be pulled (the reference's switch) and
 * a pulled level lists its nodes ascending.  The cursor holds its own
 * device buffers, charged to the version's budget, until
 * wc_bfs_cursor_destroy; wc_version_release refuses (WC_INVALID_ARGUMENT)
 * while a cursor over the version is open. */
typedef struct wc_bfs_cursor wc_bfs_cursor;
wc_status wc_bfs_cursor_open(wc_version* version, const wc_call* call, wc_direction direction,
                             const uint64_t* starts, uint64_t start_count, const wc_limits* limits,
                             const uint64_t* filter, int32_t reachable_set, wc_bfs_cursor** out);

/* bfs_cursor.rs:90-126 (next_level): runs the next level (the starts the
 * first time) and keeps its visits, in the order wc_bfs_visits lists them,
 * for wc_bfs_cursor_read; *count gets how many.  *more (may be NULL) is 0
 * once no level may follow: the search is exhausted, max_results was met
 * (the level is cut there and the stats say truncated) or the cursor was
 * stopped.  A finished cursor's calls return 0 visits; a call that fails
 * (cancelled, timed out, out of memory) finishes the cursor. */
wc_status wc_bfs_cursor_next(wc_bfs_cursor* cursor, const wc_call* call, uint64_t* count,
                             int32_t* more);

/* Visits [first, first + rows) of the last level: visits_out[3*r .. 3*r+2]
 * = (node, depth, via), host or device memory. */
wc_status wc_bfs_cursor_read(const wc_bfs_cursor* cursor, uint64_t first, uint64_t rows,
                             uint64_t* visits_out);

/* A visitor that breaks (bfs_cursor.rs:92-95, Admission::AdmitAndStop): the
 * caller took `consumed` (1 .. the last level's count) visits of the last
 * level and broke at the last of them.  The cursor finishes with the stats
 * of a search that stopped there, not truncated. */
wc_status wc_bfs_cursor_stop(wc_bfs_cursor* cursor, const wc_call* call, uint64_t consumed);

/* bfs_cursor.rs:128-131 (stats): the work done so far. */
wc_status wc_bfs_cursor_stats(const wc_bfs_cursor* cursor, wc_traversal_stats* stats);
void wc_bfs_cursor_destroy(wc_bfs_cursor* cursor);

/* traversal/reachable.rs:48-90 (reachable_set / reachable_set_each): the
 * nodes within max_depth of `starts` in the reference's order (by depth;
 * pushed levels in the order reached, pulled levels ascending), with the
 * reference's direction switch (Beamer, α = 1, β = 24, level.rs:19-29) so
 * stats.edges_traversed matches.  `capacity` entries; *count written. */
wc_status wc_reachable_set(wc_version* version, const wc_call* call, wc_direction direction,
                           const uint64_t* starts, uint64_t start_count, uint32_t max_depth,
                           uint64_t* nodes_out, uint64_t capacity, uint64_t* count,
                           wc_traversal_stats* stats);

/* No reference counterpart (warren-core searches on one host): one rank's
 * part of a row-partitioned level search (traversal/level.rs, LevelSearch)
 * over several GPUs.  The rows are cut into `parts` ranges (multiples of 64
 * rows, about equal pull entries); every rank holds the whole version and
 * the whole frontier bitmap, and owns the visited bits and depths of its
 * range.  Each level every rank reaches its range's rows (pulled, or pushed
 * from the whole frontier: the same choice on every rank), and between
 * levels the caller sums the parts' next-frontier counts and out-edges and
 * gathers the parts' words of the next frontier bitmap (one all-reduce of
 * two integers and one all-gather of id_space/8 bytes a level).  The
 * depths equal wc_bfs's depth_out over the same starts, direction and
 * max_depth (no filter, no max_results).
 *
 * wc_bfs_part_rows: the parts' first rows, row_bounds[parts + 1]. */
wc_status wc_bfs_part_rows(wc_version* version, wc_direction direction, uint32_t parts,
                           uint64_t* row_bounds);

typedef struct wc_bfs_part_info {
    uint64_t row_begin, row_end;  /* this part's rows */
    uint64_t id_space;
    uint64_t words;               /* 64-bit words of one frontier bitmap */
    uint64_t frontier;            /* level 0's frontier: the distinct starts */
    uint64_t frontier_edges;      /* and their out-edges in the search direction */
} wc_bfs_part_info;

/* Sets up part `part` of `parts`: frontier2 is the caller's device memory,
 * 2 × words 64-bit words (the frontiers of even and odd levels; bit i of
 * word i/64 is node i); every start's bit is set in frontier2[0..words).
 * Starts outside the id space are WC_NODE_OUTSIDE_ID_SPACE.  The part's
 * visited bits and depths are the version's pooled scratch (charged to its
 * budget while the pool holds them), kept between searches. */
wc_status wc_bfs_part_begin(wc_version* version, const wc_call* call, wc_direction direction,
                            const uint64_t* starts, uint64_t start_count, uint32_t max_depth,
                            uint32_t parts, uint32_t part, uint64_t* frontier2,
                            wc_bfs_part_info* info);
/* Level `level` (< max_depth) over the part's rows, given the level's
 * frontier (every part's words of frontier2[level & 1], gathered) and its
 * summed out-edges: writes the part's words of frontier2[(level + 1) & 1],
 * waits, and returns the part's next-frontier nodes and their out-edges in
 * sums[0], sums[1]. */
wc_status wc_bfs_part_step(wc_version* version, const wc_call* call, uint32_t level,
                           uint64_t frontier_edges, uint64_t* sums);
/* The part's rows of the depths (WC_UNREACHED where not reached) into
 * depth_out[row_begin .. row_end) (host or device, id_space entries).  Ends
 * the part. */
wc_status wc_bfs_part_end(wc_version* version, const wc_call* call, uint32_t* depth_out);

/* traversal/reachable.rs:18-43 (reachable). */
wc_status wc_reachable(wc_version* version, const wc_call* call, wc_direction direction,
                       uint64_t start, uint64_t target, uint32_t max_depth, int32_t* reached,
                       wc_traversal_stats* stats);

/* traversal/components.rs:21-58 (components): weakly connected components
 * over the forward rows, each dense id labelled with the smallest dense id
 * of its component (labels_out u64[id_space]); stats: every node visited,
 * every forward edge traversed. */
wc_status wc_components(wc_version* version, const wc_call* call, uint64_t* labels_out,
                        wc_traversal_stats* stats);

/* ------------------------------------------------- batched (no reference
 * counterpart: many searches as one semiring SpMM in a persistent kernel
 * under a captured CUDA graph) */

/* A schedule for the batched SpMM: columns per pass and rows per work unit,
 * chosen by wc_autotune for (version, kind, width) and cached in the handle. */
typedef struct wc_schedule {
    uint32_t columns_per_pass;
    uint32_t rows_per_unit;
    uint32_t blocks_per_sm;
    uint32_t reserved;
} wc_schedule;

typedef enum wc_batch_kind { WC_BATCH_BFS = 0, WC_BATCH_MINPLUS = 1, WC_BATCH_PPR = 2 } wc_batch_kind;

/* Times the candidate schedules for `kind` at `width` columns on this version
 * and keeps the fastest; `chosen` may be NULL. */
wc_status wc_autotune(wc_version* version, const wc_call* call, wc_batch_kind kind,
                      uint32_t width, wc_schedule* chosen);

/* Pins the schedule used for `kind` at `width` columns on this version (as
 * wc_autotune would keep its choice), for reproducible runs. */
wc_status wc_schedule_set(wc_version* version, wc_batch_kind kind, uint32_t width,
                          const wc_schedule* schedule);

/* `width` BFS searches, source s from sources[s] to depth max_depths[s]
 * (out-edges), as one boolean SpMM over bit-packed frontiers.  depth_out is
 * source-major: depth_out[s * id_space + i] = depth of i from sources[s]
 * (255 if not reached within the cap).  Identical to `width` calls of
 * wc_bfs (node, depth).  edges_traversed_out[s] (may be NULL) gets the edges
 * a push-only bfs from that source would scan.  A byte holds depths up to
 * 254: caps above 254 are served while every search ends within 254 levels;
 * a search that still has nodes to expand at depth 254 with a deeper cap
 * makes the call return WC_UNSUPPORTED (the outputs are then unspecified),
 * never a short answer. */
wc_status wc_bfs_batched(wc_version* version, const wc_call* call, const uint64_t* sources,
                         const uint32_t* max_depths, uint32_t width, uint8_t* depth_out,
                         uint64_t* edges_traversed_out);

/* `width` hop-bounded shortest-path searches (the sssp_vector loop,
 * compute_sql/library/sssp_vector.sql:14-66, with max_iter = max_hops[s]):
 * dist_out[s * id_space + i] = the i64 min-plus distance (INT64_MAX:
 * unreached) over transpose min_plus with accumulate min; iterations_out[s]
 * (may be NULL) the iterations that loop runs.  Weights are cast as
 * SemiringElement::from_weight casts them (semiring.rs:365-367). */
wc_status wc_minplus_batched(wc_version* version, const wc_call* call, const uint64_t* sources,
                             const uint32_t* max_hops, uint32_t width, int64_t* dist_out,
                             uint32_t* iterations_out);

/* `width` personalised PageRanks (pagerank/mod.rs:96-199 with a seed): seed
 * set c is seed_nodes[seed_offsets[c] .. seed_offsets[c+1]), each node's
 * seed value 1, so p = 1/|set| on the set.  Each column stops at its own
 * iterate (delta < live × tol).  ranks_out is column-major:
 * ranks_out[c * id_space + i]; iterations_out[c] per column. */
wc_status wc_ppr_batched(wc_version* version, const wc_call* call, const wc_pagerank_opts* opts,
                         const uint64_t* seed_nodes, const uint64_t* seed_offsets, uint32_t width,
                         double* ranks_out, uint32_t* iterations_out);

/* ------------------------------------------ multi-source centralities */

/* compute/centrality/closeness.rs:36-56: closeness (NetworkX's, over the
 * distances *to* each node, scaled by reached / other sources when
 * wf_improved) or harmonic centrality, on the version's unweighted forward
 * rows (for an undirected graph, upload it symmetrised), from `sources`. */
typedef enum wc_centrality_measure { WC_CLOSENESS = 0, WC_HARMONIC = 1 } wc_centrality_measure;

typedef struct wc_centrality_opts {
    uint32_t measure;           /* wc_centrality_measure */
    uint32_t wf_improved;       /* closeness: Wasserman and Faust's scaling */
    uint32_t columns_per_pass;  /* sources a batched pass: 64 .. 1024 (0: 1024) */
    uint32_t blocks_per_sm;     /* 0: 4 */
} wc_centrality_opts;

/* Chooses the sources as centrality/sources.rs:55-123 (Sources::choose):
 * the live nodes the population mask selects (population[i] != 0, flipped
 * by `complement`; NULL selects every node), then, if k >= 0 and fewer
 * than them, the k with the smallest seeded keys; ascending.  sources_out
 * holds up to id_space ids; count_out gets their number. */
wc_status wc_sample_sources(uint64_t id_space, const uint64_t* tombstone_words,
                            const uint8_t* population, int32_t complement, int64_t k,
                            uint64_t seed, uint64_t* sources_out, uint64_t* count_out);

/* Each node's centrality from `sources` (distinct live nodes, ascending, as
 * wc_sample_sources gives them), as the reference's batched measures: the
 * sources searched 64 at a time in ascending order, a node's totals added to
 * batch by batch, then by distance (centrality/mod.rs:15-20, 158-190).  Exact
 * when the sources are every live node, else the sampled estimate
 * (closeness.rs:117-132, 229-241).  Tombstoned nodes get 0.  values_out
 * f64[id_space].  A search deeper than 1,024 levels is WC_UNSUPPORTED. */
wc_status wc_centrality(wc_version* version, const wc_call* call, const wc_centrality_opts* opts,
                        const uint64_t* sources, uint64_t count, const uint64_t* tombstone_words,
                        double* values_out);

/* compute/centrality/betweenness.rs:18-37 (BetweennessScale and the
 * graph's direction, which the rescale reads). */
typedef struct wc_betweenness_opts {
    int32_t normalized;      /* divide by the pairs a path could join */
    int32_t endpoints;       /* count a path's ends as on it */
    int32_t directed;        /* the version's rows are directed (else uploaded symmetrised) */
    uint32_t blocks_per_sm;  /* 0: 4 */
} wc_betweenness_opts;

/* compute/centrality/betweenness.rs:27-38: each node's betweenness over the
 * fewest-edge shortest paths of the version's forward rows (weights are not
 * read), by Brandes' algorithm from `sources` (distinct live nodes,
 * ascending, as wc_sample_sources gives them), rescaled as NetworkX 3.7
 * (betweenness.rs:113-141); tombstoned nodes 0.  Path counts are f64 as in
 * the reference, and the values are the reference's to the bit while they
 * stay below 2^53.  A search deeper than 1,024 levels is WC_UNSUPPORTED. */
wc_status wc_betweenness(wc_version* version, const wc_call* call, const wc_betweenness_opts* opts,
                         const uint64_t* sources, uint64_t count, const uint64_t* tombstone_words,
                         double* values_out);

/* ------------------------------------------------------------- spectral */

/* spectral/operator.rs:33-44 (Operator) and lanczos.rs:69-74 (Which). */
typedef enum wc_operator {
    WC_ADJACENCY = 0, WC_LAPLACIAN = 1, WC_NORMALIZED_LAPLACIAN = 2, WC_RANDOM_WALK = 3
} wc_operator;
typedef enum wc_which { WC_LARGEST = 0, WC_SMALLEST = 1 } wc_which;

/* spectral/lanczos.rs:136-168 (EigenOptions) with GraphMatrix
 * (operator.rs:77-93); f64 precision only. */
typedef struct wc_eigen_opts {
    uint32_t k;
    wc_which which;
    wc_operator op;
    int32_t symmetrize;
    int32_t weighted;        /* -1 / 0 / 1 */
    double tol;
    uint64_t max_iter;       /* 0: 1,000 × the basis size */
    uint64_t seed;
} wc_eigen_opts;

typedef struct wc_eigen_stats {
    uint64_t iterations;
    uint64_t components;
    uint32_t exact;
    int32_t converged;
} wc_eigen_stats;

/* spectral/lanczos.rs:206-224 (eigen): values[k], residuals[k] and the unit
 * eigenvectors vectors[j * id_space + i] (may be NULL), in `which` order. */
wc_status wc_eigen(wc_version* version, const wc_call* call, const wc_eigen_opts* opts,
                   double* values, double* residuals, double* vectors, wc_eigen_stats* stats);

/* ------------------------------------------------------------- adjoint
 * (no reference counterpart) */

/* ∂L_c/∂w for `losses` losses L_c = Σ_{t in targets of c} x_t, x the
 * uniform PageRank of the weighted graph (recomputed, not stored):
 * targets of loss c are loss_targets[loss_offsets[c] .. loss_offsets[c+1]).
 * grad_out is loss-major over the forward CSR's edge order:
 * grad_out[c * edges + e].  The forward runs opts->max_iter iterations or
 * stops at opts->tol as wc_pagerank does; the adjoint solve runs to
 * adjoint_tol (L1 of the adjoint change) or opts->max_iter.
 * iterations_out (2 entries, may be NULL): the forward iterations, and the
 * most adjoint iterations any loss took.  Uniform personalisation, no
 * tombstones. */
wc_status wc_pagerank_adjoint(wc_version* version, const wc_call* call,
                              const wc_pagerank_opts* opts, const uint64_t* loss_targets,
                              const uint64_t* loss_offsets, uint32_t losses, double adjoint_tol,
                              double* grad_out, double* ranks_out, uint32_t* iterations_out);

/* ---------------------------------------------------------- vector map */

/* compute/map/expr.rs (the vector_map IR), one node per expression node.
 * A node's children are children[first .. first + count), in the IR's
 * order: CASE lists (condition, value) pairs, then the ELSE if has_else;
 * COMPARE and the binary operations their two operands; CAST its operand. */
typedef enum wc_map_kind {
    WC_MAP_LITERAL = 0,   /* value in i (bool, bigint) or f (real, double); is_null: a typed NULL */
    WC_MAP_VECTOR = 1,    /* operand i at the current element */
    WC_MAP_CAST = 2,      /* the child, cast to `type` as SQL casts (compute/cast.rs) */
    WC_MAP_CASE = 3,
    WC_MAP_NULLIF = 4,
    WC_MAP_COALESCE = 5,
    WC_MAP_LEAST = 6,
    WC_MAP_GREATEST = 7,
    WC_MAP_NEGATE = 8,    /* bigint, real, double */
    WC_MAP_ARITHMETIC = 9, /* op: 0 +, 1 -, 2 *, 3 / */
    WC_MAP_MODULO = 10,   /* bigint */
    WC_MAP_ABS = 11,      /* bigint, real */
    WC_MAP_CALL = 12,     /* double; op: 0 abs, 1 sqrt, 2 exp, 3 ln, 4 log, 5 floor, 6 ceil,
                             7 round, 8 sign (expr.rs:176-197) */
    WC_MAP_POWER = 13,    /* double */
    WC_MAP_COMPARE = 14,  /* boolean; op: 0 =, 1 <>, 2 <, 3 <=, 4 >, 5 >= over the children's type */
    WC_MAP_NOT = 15,
    WC_MAP_AND = 16,
    WC_MAP_OR = 17
} wc_map_kind;

typedef struct wc_map_node {
    int32_t kind;      /* wc_map_kind */
    int32_t type;      /* the node's wc_dtype */
    int32_t op;        /* by kind, above */
    int32_t has_else;  /* CASE */
    uint32_t first;    /* children */
    uint32_t count;
    int32_t is_null;   /* LITERAL */
    int32_t reserved;
    int64_t i;         /* LITERAL (bool, bigint) or VECTOR (operand index) */
    double f;          /* LITERAL (real, double) */
} wc_map_node;

/* compute/map/mod.rs:49-78 (map): `root`'s value at every element of the
 * version's id space, row-major over rows of the widest operand's width
 * (operands of width 1 and literals repeat across a row), written to out
 * (id_space × width elements of the root's type; *out_width gets the width).
 * SQL semantics as the reference's: CASE, COALESCE, AND and OR evaluate an
 * argument only where SQL would; NULL stores NaN in real and double results
 * and is WC_NULL_RESULT in bigint and boolean ones; the error reported is
 * the first failing element's in row-major order.  Operand checks as the
 * reference: id space and width, then every operand reference, evaluated or
 * not.  All results are the reference's to the bit except exp, ln, log and
 * power, which use the device's functions (within 2 units in the last
 * place).  Expressions whose evaluation needs more than 32 stack values or
 * more than 16 operands are WC_UNSUPPORTED. */
wc_status wc_vector_map(wc_version* version, const wc_call* call, const wc_map_node* nodes,
                        uint32_t node_count, const uint32_t* children, uint32_t child_count,
                        uint32_t root, const void* const* operands, const wc_dtype* operand_dtypes,
                        const uint64_t* operand_id_spaces, const uint32_t* operand_widths,
                        uint32_t operand_count, void* out, uint32_t* out_width);

/* ------------------------------------------------------- vector reduce */

/* compute/reduce.rs:23-38 (Reduction) and :74-82 (Norm), in order. */
typedef enum wc_reduction {
    WC_REDUCE_SUM = 0, WC_REDUCE_MAX = 1, WC_REDUCE_MIN = 2, WC_REDUCE_L1 = 3, WC_REDUCE_L2 = 4,
    WC_REDUCE_NNZ = 5
} wc_reduction;
typedef enum wc_norm { WC_NORM_L1 = 0, WC_NORM_L2 = 1, WC_NORM_LINF = 2 } wc_norm;

/* compute/reduce.rs:118-153 (reduce / reduce_live): `reduction` over the
 * id_space × width elements of x (row-major, read as f64, bool as 0 / 1),
 * skipping the rows tombstone_words marks (NULL: none), to the bit: chunks
 * of 65,536 elements summed in order from +0, then the chunks in order.
 * *is_null (may be NULL) is set for the max or min of no elements. */
wc_status wc_vector_reduce(wc_version* version, const wc_call* call, wc_dtype dtype,
                           const void* x, uint32_t width, const uint64_t* tombstone_words,
                           wc_reduction reduction, double* result, int32_t* is_null);

/* compute/reduce.rs:175-206 (norm_diff): norm(a − b), rows aligned by dense
 * id and a row past the shorter vector's end counting as zero; 0 for no
 * elements.  The vectors may be over other id spaces than the version's. */
wc_status wc_vector_norm_diff(wc_version* version, const wc_call* call, wc_dtype dtype_a,
                              const void* a, uint64_t id_space_a, wc_dtype dtype_b,
                              const void* b, uint64_t id_space_b, uint32_t width, wc_norm norm,
                              double* result);

/* ------------------------------------------------------------- ranking */

/* compute/ranking.rs:52 (top_k): the k live rows with the largest
 * (`descending`) or smallest values of width-1 `x`, best first, ties to the
 * smaller dense id, SQL order (NaN above every number). */
wc_status wc_topk(wc_version* version, const wc_call* call, wc_dtype dtype, const void* x,
                  const uint64_t* tombstones, uint64_t k, int32_t descending,
                  uint64_t* nodes_out, double* values_out, uint64_t* count);

/* ------------------------------------------------- graph synthesis (host)
 * Deterministic synthetic inputs for tests and benchmarks; not part of the
 * seam.  Both return a CSR built as the reference builds one (rows sorted,
 * parallel edges folded, self-loops dropped) with node ids relabelled by a
 * random bijection of distinct int64 external ids ranked in sorted order
 * (graph/id_map/mod.rs:38-49). */

typedef struct wc_host_csr {
    uint64_t id_space;
    uint64_t edges;
    uint64_t* offsets;   /* id_space + 1, owned by the library */
    uint32_t* targets;   /* edges */
    int64_t* external_ids; /* id_space: the external id of each dense id */
} wc_host_csr;

/* R-MAT (a, b, c, 1-a-b-c) at `scale` with edge_factor·2^scale generated
 * edges, seed `seed`.  `undirected`: each edge stored both ways. */
wc_status wc_graph_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c,
                        uint64_t seed, int32_t undirected, wc_host_csr* out);
/* Erdős–Rényi G(n, m): `edges` edges drawn uniformly (then folded). */
wc_status wc_graph_gnm(uint64_t id_space, uint64_t edges, uint64_t seed, int32_t undirected,
                       wc_host_csr* out);
void wc_host_csr_free(wc_host_csr* csr);
/* The transpose of a host CSR (reverse CSR), rows ascending. */
wc_status wc_host_transpose(uint64_t id_space, uint64_t edges, const uint64_t* offsets,
                            const uint32_t* targets, const double* weights,
                            uint64_t* reverse_offsets, uint32_t* reverse_targets,
                            double* reverse_weights);

#ifdef __cplusplus
}
#endif

#endif /* WARREN_CUDA_H */

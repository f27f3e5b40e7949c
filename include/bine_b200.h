/*
 * bine_b200.h -- C ABI of the B200 engine for the Bine-tree collectives.
 *
 * A communicator holds P "virtual ranks" whose buffers all live in the HBM of
 * one GPU.  Every buffer argument is a DEVICE pointer to a rank-major array:
 * rank r's row starts at  base + r * stride  bytes.  By default the stride is
 * the row size (rows packed back to back); bine_comm_set_layout() sets a
 * larger one.  Input and output arrays may share bytes (the same base, as
 * with MPI_IN_PLACE, or rows that interleave): such a call first copies its
 * input rows to a staging area of the communicator, except an allreduce or
 * reduce on the FUSED engine whose two arrays are identical (same base and
 * stride) and whose result is one value per column (not per-rank float
 * trees), which needs no copy.  Calls are asynchronous and ordered on the
 * communicator's CUDA stream.  Functions return BINE_SUCCESS or an error code and never abort;
 * bine_last_error_string() describes the last error of the calling thread.
 *
 * The eight collectives keep the argument lists of the reference library's
 * MPI entry points (HLC-Lab/bine_trees_fugaku, lib/libbine.cc): one call here
 * performs the collective for all P ranks at once.  Algorithm selection
 * mirrors the reference's LIBBINE_* environment variables
 * (lib/libbine.cc:75-575) as explicit per-communicator settings.
 */
#ifndef BINE_B200_H
#define BINE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct bine_comm_s *bine_comm_t;

/* Element types (MPI_INT32_T, MPI_INT64_T, MPI_FLOAT, MPI_DOUBLE, MPI_CHAR). */
typedef enum {
    BINE_INT32 = 0,
    BINE_INT64 = 1,
    BINE_FLOAT = 2,
    BINE_DOUBLE = 3,
    BINE_CHAR = 4
} bine_datatype_t;

/* Reduction operators (MPI_SUM). */
typedef enum { BINE_SUM = 0 } bine_op_t;

/* Return codes. */
enum {
    BINE_SUCCESS = 0,
    BINE_ERR_ARG = 1,         /* invalid argument */
    BINE_ERR_UNSUPPORTED = 2, /* the selected reference algorithm cannot run this case */
    BINE_ERR_CUDA = 3,        /* a CUDA call failed */
    BINE_ERR_TIMEOUT = 4,     /* a bounded device-side wait expired */
    BINE_ERR_NOMEM = 5,       /* device memory exhausted */
    BINE_ERR_INTERNAL = 6,
    BINE_ERR_ABORTED = 7      /* a caller's window hook abandoned the call */
};

/* Collectives, for bine_comm_set_algo() and the planning queries. */
typedef enum {
    BINE_COLL_ALLREDUCE = 0,
    BINE_COLL_REDUCE_SCATTER = 1,
    BINE_COLL_ALLGATHER = 2,
    BINE_COLL_BCAST = 3,
    BINE_COLL_REDUCE = 4,
    BINE_COLL_ALLTOALL = 5,
    BINE_COLL_SCATTER = 6,
    BINE_COLL_GATHER = 7
} bine_coll_t;

/* Algorithm variants: the values of the reference's LIBBINE_<COLL>_ALGO
 * (enums at lib/libbine_common.h:74-123). */
enum {
    BINE_ALLREDUCE_L = 0, BINE_ALLREDUCE_B = 1, BINE_ALLREDUCE_B_CONT = 3, BINE_ALLREDUCE_B_COALESCE = 4,
    BINE_ALLGATHER_CONT_PERMUTE = 0, BINE_ALLGATHER_CONT_SEND = 1, BINE_ALLGATHER_BLOCKS = 2,
    BINE_REDUCE_SCATTER_CONT_PERMUTE = 0,
    BINE_BCAST_BINOMIAL_TREE = 0, BINE_BCAST_SCATTER_ALLGATHER = 2,
    BINE_REDUCE_BINOMIAL_TREE = 0, BINE_REDUCE_SCATTER_GATHER = 1,
    BINE_ALLTOALL_LOG = 0, BINE_SCATTER_BINOMIAL_TREE = 0, BINE_GATHER_BINOMIAL_TREE = 0
};

/* LIBBINE_<COLL>_ALGO_FAMILY (lib/libbine_common.h:77-85).  BRUCK is the
 * reference's comparator for alltoall (lib/libbine_coll_alltoall.cc:18);
 * RING is its comparator for allreduce, the multi-dimensional bucket ring
 * (lib/libbine_common.cc:2372-2663; the variant is ignored, as in the
 * reference's dispatch, lib/libbine.cc:1056-1057).  RING reduce_scatter and
 * allgather return BINE_ERR_UNSUPPORTED: the reference's versions never
 * deliver the result. */
enum { BINE_FAMILY_BINE = 1, BINE_FAMILY_RECDOUB = 2, BINE_FAMILY_BRUCK = 3, BINE_FAMILY_RING = 4 };
enum { BINE_DISTANCE_INCREASING = 0, BINE_DISTANCE_DECREASING = 1, BINE_DISTANCE_DEFAULT = -1 };

/* Execution engines.
 *   FUSED (default): one kernel per call that reads every input element
 *     once and writes every output element once, evaluating the reference's
 *     exact addition tree per element in registers;
 *   STEPS: one persistent kernel that executes the reference's schedule step
 *     by step (the message pattern of the MPI layer, as device loads and
 *     stores), with a bounded grid-wide barrier between steps;
 *   PIPELINED: the same schedule as STEPS, cut into segments that each
 *     start as soon as the segments they read and overwrite are done, with
 *     no barrier between steps: steps overlap segment by segment and ports
 *     proceed independently (the device analogue of the uTofu layer's
 *     per-port threads and segmented transfers, lib/libbine_common.cc:1741-1879).
 *     By default several levels run as one pass (bine_comm_set_fusion).
 *     Results equal the STEPS engine's, float32 included. */
enum { BINE_ENGINE_FUSED = 0, BINE_ENGINE_STEPS = 1, BINE_ENGINE_PIPELINED = 2 };

/* Floating-point summation order for the FUSED engine.
 *   REFERENCE (default): bit-identical to the reference's per-step order;
 *   FAST: straight column sums accumulated in FP64 and rounded once. */
enum { BINE_ORDER_REFERENCE = 0, BINE_ORDER_FAST = 1 };

/* ---------------------------------------------------------- communicator */

/* Creates a communicator of `nranks` virtual ranks on the current device,
 * arranged as a torus of `ndims` (0..3) dimensions `dims` (ndims = 0: one
 * ring of nranks).  Replaces MPI_COMM_WORLD plus LIBBINE_DIMENSIONS
 * (lib/libbine.cc:114-130).  No device memory is touched until the first
 * collective. */
int bine_comm_create(int nranks, int ndims, const int *dims, bine_comm_t *comm);
int bine_comm_destroy(bine_comm_t comm);

/* CUDA stream (a cudaStream_t) the calls are ordered on; NULL = default. */
int bine_comm_set_stream(bine_comm_t comm, void *stream);

/* Bytes between consecutive rank rows of the send and receive arrays; 0
 * keeps rows packed.  Strides must cover the row sizes of each call. */
int bine_comm_set_layout(bine_comm_t comm, size_t send_stride, size_t recv_stride);

/* LIBBINE_NUM_PORTS (1..6). */
int bine_comm_set_ports(bine_comm_t comm, int ports);

/* LIBBINE_<COLL>_ALGO, _ALGO_FAMILY and _DISTANCE for one collective. */
int bine_comm_set_algo(bine_comm_t comm, bine_coll_t coll, int variant, int family, int distance);

int bine_comm_set_engine(bine_comm_t comm, int engine);

/* LIBBINE_SEGMENT_SIZE analogue for the STEPS and PIPELINED engines: bytes
 * of each unit of work a block takes (0: 32 KiB).  Small segments spread
 * small messages over more blocks (and, PIPELINED, let a step start on a
 * message's first segment before its last one is ready); large ones cut
 * per-segment overhead.  Results do not depend on it. */
int bine_comm_set_segment(bine_comm_t comm, long long segment_bytes);

/* Level fusion for the PIPELINED engine: `levels` consecutive levels of the
 * reference's schedule per pass (1: every level on its own, as the STEPS
 * engine runs them; 0, the default: chosen per collective, below).  Within a pass, values that one step hands to
 * the next (partial sums, staged messages) stay in registers; a pass writes
 * only what a later pass reads or what is a result, and a copy several ranks
 * receive from one rank is read once.  A write that would overwrite what its
 * pass still reads goes to a fresh workspace slot instead.  Results are
 * bit-identical (the schedule's addition trees), and after every pass each
 * element that is read later or is a result holds, at its own position or
 * in its slot, what the reference's buffers hold after that step.  No
 * counterpart in the reference.  0 chooses the levels per pass for each
 * collective (allreduce, reduce_scatter and reduce 6; allgather, bcast,
 * scatter and gather 12; alltoall 13) and runs schedules of more than 2^20
 * moves level by level: planning a fused schedule costs about 4 us per move
 * on the host, once per call shape. */
int bine_comm_set_fusion(bine_comm_t comm, int levels);
int bine_comm_set_float_order(bine_comm_t comm, int order);

/* ----------------------------------------------------------- collectives */

/* MPI_Allreduce, lib/libbine.cc:1012. */
int bine_allreduce(const void *sendbuf, void *recvbuf, int count, bine_datatype_t datatype, bine_op_t op,
                   bine_comm_t comm);

/* MPI_Allreduce with HOST buffers, as an MPI caller holds them
 * (lib/libbine.cc:1012): `sendbuf`/`recvbuf` are rank-major host arrays
 * (strides from bine_comm_set_layout).  Column windows of ~32 MiB flow
 * through the device on three streams so that the host->device copy of one
 * window, the reduction of the previous one and the device->host copy of
 * the one before that overlap (window size: bine_comm_set_host_window).  Pinned host memory (cudaHostAlloc or
 * cudaHostRegister) gives full PCIe bandwidth; pageable memory works at
 * pageable-copy speed.  Returns when the result is in `recvbuf`.  Results
 * equal bine_allreduce's (the fused kernels run whatever the engine
 * setting; float sums follow the communicator's float order). */
int bine_allreduce_host(const void *sendbuf, void *recvbuf, int count, bine_datatype_t datatype, bine_op_t op,
                        bine_comm_t comm);

/* bine_allreduce_host with the caller in the pipeline, for callers whose
 * input rows fill while the call runs and whose output rows drain as they
 * arrive (the PMPI layer: every MPI rank deposits its row into shared pinned
 * memory and collects its result row from it).  The call moves column
 * windows [first, first + count) of all rows in increasing order:
 * before_window(user, first, count) runs before a window's input columns
 * are copied to the GPU and returns once every row holds them;
 * after_window(user, first, count) runs once that window's output columns
 * of every row are in host memory.  A nonzero return from either hook
 * abandons the call (after the copies in flight end) with
 * BINE_ERR_ABORTED.  Either hook may be NULL.  Results equal
 * bine_allreduce_host's.  No counterpart in the reference: its MPI layer
 * has no host pipeline. */
typedef int (*bine_window_hook_t)(void *user, long long first, long long count);
int bine_allreduce_host_hooked(const void *sendbuf, void *recvbuf, int count, bine_datatype_t datatype,
                               bine_op_t op, bine_comm_t comm, bine_window_hook_t before_window,
                               bine_window_hook_t after_window, void *user);

/* Bytes of one column window of bine_allreduce_host over all ranks
 * (default 32 MiB; at least 4 KiB).  Smaller windows shorten the pipeline's
 * fill and drain; larger ones cut per-copy overhead. */
int bine_comm_set_host_window(bine_comm_t comm, long long window_bytes);

/* MPI_Reduce_scatter, lib/libbine.cc:1064 (recvcounts must all be equal, as
 * the reference's block implementation assumes, lib/libbine.cc:1065). */
int bine_reduce_scatter(const void *sendbuf, void *recvbuf, const int *recvcounts, bine_datatype_t datatype,
                        bine_op_t op, bine_comm_t comm);

/* MPI_Allgather, lib/libbine.cc:1168 (sendcount == recvcount and
 * sendtype == recvtype, lib/libbine.cc:1170-1171). */
int bine_allgather(const void *sendbuf, int sendcount, bine_datatype_t sendtype, void *recvbuf, int recvcount,
                   bine_datatype_t recvtype, bine_comm_t comm);

/* MPI_Bcast_f, lib/libbine.cc:1252: in place on `buffer`; the root's row
 * holds the data. */
int bine_bcast(void *buffer, int count, bine_datatype_t datatype, int root, bine_comm_t comm);

/* MPI_Alltoall, lib/libbine.cc:1291. */
int bine_alltoall(const void *sendbuf, int sendcount, bine_datatype_t sendtype, void *recvbuf, int recvcount,
                  bine_datatype_t recvtype, bine_comm_t comm);

/* MPI_Scatter, lib/libbine.cc:1312 (only the root's send row is read). */
int bine_scatter(const void *sendbuf, int sendcount, bine_datatype_t sendtype, void *recvbuf, int recvcount,
                 bine_datatype_t recvtype, int root, bine_comm_t comm);

/* MPI_Gather, lib/libbine.cc:1376 (only the root's receive row is written). */
int bine_gather(const void *sendbuf, int sendcount, bine_datatype_t sendtype, void *recvbuf, int recvcount,
                bine_datatype_t recvtype, int root, bine_comm_t comm);

/* MPI_Reduce, lib/libbine.cc:1440 (only the root's receive row is written). */
int bine_reduce(const void *sendbuf, void *recvbuf, int count, bine_datatype_t datatype, bine_op_t op, int root,
                bine_comm_t comm);

/* Allocation-free allreduce.  No counterpart in the reference: it exists for
 * callers that cannot allocate device memory -- code running inside a
 * memory manager that owns every device allocation, or in a phase where
 * cudaMalloc is forbidden -- and so cannot let bine_allreduce() create its
 * workspace and schedule tables on first use.  It runs the same STEPS
 * engine schedule as bine_allreduce() with BINE_ENGINE_STEPS (the
 * communicator's allreduce variant, ports and layout), but every piece of
 * device scratch it needs -- the schedule tables, the grid-barrier and
 * status words and the workspace rows -- lives in one fixed 64 MiB array
 * that the library reserves on each device that loads it and keeps until
 * the process exits.  It calls no cudaMalloc, cudaFree or other allocating
 * routine.  The caller passes the input and output arrays as usual.
 *   * Calls needing more than 64 MiB of scratch (schedule tables plus
 *     workspace; the B variant's tables grow with nranks squared) fail with
 *     BINE_ERR_NOMEM and a message naming the size.
 *   * The first call on a device looks up the array's device address; make
 *     that first call before any stream capture.
 *   * Every call reuses the same array: two calls that overlap on the GPU
 *     (on different streams or from different threads) race.  The call is
 *     synchronous: it returns after its kernel finished and reports a
 *     barrier timeout as BINE_ERR_TIMEOUT. */
int bine_allreduce_noalloc(const void *sendbuf, void *recvbuf, int count, bine_datatype_t datatype, bine_op_t op,
                           bine_comm_t comm);

/* Waits for the communicator's stream and reports device-side errors
 * (BINE_ERR_TIMEOUT when a bounded barrier of the STEPS engine, or a
 * bounded segment wait of the PIPELINED engine, expired). */
int bine_comm_synchronize(bine_comm_t comm);

const char *bine_last_error_string(void);

/* Bound of every device-side wait of the STEPS and PIPELINED engines (grid
 * barriers between steps, segment waits), in milliseconds; default 5000.  A wait that expires makes the
 * kernel record the timeout and return; bine_comm_synchronize() then
 * reports BINE_ERR_TIMEOUT and the context stays usable. */
int bine_comm_set_step_timeout(bine_comm_t comm, unsigned timeout_ms);

/* Fault injection for tests of the timeout path: makes every grid barrier of
 * the STEPS engine wait for `extra` arrivals that never come, and every
 * segment wait of the PIPELINED engine for a completion that never comes,
 * so the bounded wait expires (0 restores normal operation).  Nothing
 * faults or hangs. */
int bine_debug_set_barrier_extra(bine_comm_t comm, unsigned extra);

/* How the FUSED engine evaluates an exact-order float reduction on a
 * 16-byte-aligned layout, planned on the host only (no device needed;
 * nothing is uploaded or cached):
 *   out[0] form: 0 element kernel only, 1 one lane per vector, 2 K lanes per
 *          vector with tiles per segment, 3 K lanes per vector with tiles on
 *          the row's own grid (trees of at most 8 shapes);
 *   out[1] K, the lanes per vector;   out[2] tree shapes (form 3, else 0);
 *   out[3] vector tiles;   out[4] edge vectors evaluated whole (form 3);
 *   out[5] element pieces left to the element kernels.
 * No reference counterpart: introspection of this engine's planner. */
int bine_plan_tree_form(bine_comm_t comm, bine_coll_t coll, long count, bine_datatype_t datatype, int root,
                        int64_t out[6]);

/* The output elements each kernel of that plan writes (one output row; all
 * ranks' rows alike): `n` runs of (first element, elements, kind), kind 1 a
 * vector tile (a lane vector of a row-aligned tile, or a whole tile of the
 * other forms), 2 an edge vector, 3 an element piece.  Host only; with
 * `runs` null or `cap` below the count only `*n` is set.  No reference
 * counterpart: introspection of this engine's planner. */
int bine_plan_tree_cover(bine_comm_t comm, bine_coll_t coll, long count, bine_datatype_t datatype, int root,
                         int64_t *runs, size_t cap, size_t *n);

/* out[0] and out[1] of bine_plan_tree_form. */
int bine_debug_tree_form(bine_comm_t comm, bine_coll_t coll, long count, bine_datatype_t datatype, int root,
                         int *form, int *lanes);

/* Lanes that cooperate on one output vector in the exact-order float
 * reduction (1, 2, 4 or 8; 0, the default, chooses per call from the
 * output size).  Results are identical for every setting. */
int bine_comm_set_tree_split(bine_comm_t comm, int lanes);

/* ------------------------------------------------------------- batching
 * Many independent allreduce / reduce_scatter / allgather calls of
 * different rank counts, sizes and element types (BINE_INT32 or
 * BINE_FLOAT) executed by ONE persistent kernel launch, which can be
 * captured in a CUDA graph.  Each item is a complete collective over its
 * own `nranks` virtual ranks, with the argument meaning of its entry point
 * (count = allreduce count, reduce_scatter recvcount, allgather
 * sendcount).  Rows must be 16-byte aligned and hold whole 16-byte vectors
 * (count * element size a multiple of 16).  Integer results equal the
 * single-call results; float32 sums use the FAST order (FP64 accumulation,
 * within 1e-6 relative of an FP64 sum), as single calls with
 * BINE_ORDER_FAST do.  Not in the reference: the batching pattern of the
 * engine. */
typedef struct {
    int coll;        /* BINE_COLL_ALLREDUCE, _REDUCE_SCATTER or _ALLGATHER */
    int datatype;    /* BINE_INT32 or BINE_FLOAT */
    int nranks;
    int reserved;
    long count;
    const void *sendbuf;
    void *recvbuf;
    size_t send_stride, recv_stride; /* bytes between rank rows; 0 = packed */
} bine_batch_item_t;

/* Launch shape chosen by the autotuner: reduction tiles are
 * tile_cols[k] 16-byte columns wide for items whose nranks <= rank_bound[k]
 * (k = 0..3, bounds ascending, the last one catching every size); grid =
 * grid_mult * resident blocks; order 0 keeps item order, 1 schedules the
 * most expensive items first. */
typedef struct {
    int rank_bound[4];
    int tile_cols[4];
    int grid_mult;
    int order;
} bine_batch_tuning_t;

typedef struct bine_batch_s *bine_batch_t;

/* Validates the items, lays out the tiles and uploads the descriptors
 * (tuning NULL: defaults). */
int bine_batch_create(const bine_batch_item_t *items, int nitems, const bine_batch_tuning_t *tuning,
                      bine_batch_t *batch);
/* One persistent launch of the whole batch on `stream` (capturable). */
int bine_batch_launch(bine_batch_t batch, void *stream);
int bine_batch_destroy(bine_batch_t batch);
/* Times candidate tunings of this batch on `stream` (reps launches each,
 * CUDA events) and returns the fastest in *best and its time in *best_ms. */
int bine_batch_autotune(const bine_batch_item_t *items, int nitems, void *stream, int reps,
                        bine_batch_tuning_t *best, float *best_ms);

/* -------------------------------------------------------- learned picker
 * A 3-hidden-layer MLP (in -> H -> H -> H -> out, GELU, bf16 weights and
 * activations, fp32 accumulation) with forward, backward and Adam kernels.
 * The engine's variant picker (bine_trees_fugaku_b200/picker.py) trains it
 * on timings and link-byte counts the engine itself measures and uses it to
 * choose variant, port count and segment size per call.  Not in the
 * reference.  All dimensions and batch sizes are multiples of 16; device
 * pointers are fp32 row-major [n x in] / [n x out]. */
typedef struct bine_mlp_s *bine_mlp_t;
int bine_mlp_create(int in_dim, int hidden, int out_dim, int max_batch, unsigned long long seed, bine_mlp_t *mlp);
int bine_mlp_destroy(bine_mlp_t mlp);
int bine_mlp_num_params(bine_mlp_t mlp, size_t *n);
/* Parameter arena: for layer l, weights [out x in] row-major then the bias,
 * each starting at a multiple of 16 floats (fp32 masters). */
int bine_mlp_get_params(bine_mlp_t mlp, float *host);
int bine_mlp_set_params(bine_mlp_t mlp, const float *host);
int bine_mlp_forward(bine_mlp_t mlp, const float *d_x, int n, float *d_y, void *stream);
/* Gradients of the masked mean squared error (same layout as the
 * parameters), for checking against a CPU reference. */
int bine_mlp_gradients(bine_mlp_t mlp, const float *d_x, const float *d_t, const float *d_mask, int n,
                       float *host_grads, float *loss);
/* One Adam step on a batch; *loss receives the batch loss (synchronous). */
int bine_mlp_train_step(bine_mlp_t mlp, const float *d_x, const float *d_t, const float *d_mask, int n, float lr,
                        void *stream, float *loss);
const char *bine_mlp_last_error(void);

/* Inference of an ensemble of 1..8 models of the same shape (hidden width
 * 256, input and output widths up to 256) in ONE launch: d_y [n x out]
 * receives the mean of the models' outputs, summed in model order.  The
 * picker ranks the arms of one call with it (a 16-row batch).  The
 * ensemble refers to the models' current weights; it holds no copy.  Not in
 * the reference. */
typedef struct bine_mlp_ensemble_s *bine_mlp_ensemble_t;
int bine_mlp_ensemble_create(const bine_mlp_t *models, int nmodels, bine_mlp_ensemble_t *ens);
int bine_mlp_ensemble_forward(bine_mlp_ensemble_t ens, const float *d_x, int n, float *d_y, void *stream);
int bine_mlp_ensemble_destroy(bine_mlp_ensemble_t ens);

/* ------------------------------------------------------ schedule queries
 * Host-only: these plan the call with the communicator's current settings
 * and need no GPU.  `count` and `root` have the meaning of the collective's
 * own arguments (for reduce_scatter, the per-rank receive count). */

/* Proves by symbolic execution that the planned schedule computes the MPI
 * result (every output element is the right input element, or the sum of
 * that element over every rank once); BINE_ERR_UNSUPPORTED when the
 * reference's schedule returns wrong data for this case.  The STEPS engine
 * runs only verified schedules. */
int bine_plan_verify(bine_comm_t comm, bine_coll_t coll, long count, int root);

/* Sizes of the schedule: out[0] = steps (levels), out[1] = moves,
 * out[2] = messages, out[3] = workspace elements per rank,
 * out[4] = bytes read + written by the STEPS engine per element size. */
int bine_plan_stats(bine_comm_t comm, bine_coll_t coll, long count, int root, int64_t out[5]);

/* The schedule's moves, level by level.  Each move is 10 int64 values:
 * level, dst_rank, dst_buf, dst_off, a_rank, a_buf, a_off, b_rank, b_buf,
 * b_off (buffers: 0 send, 1 receive, 2 workspace; offsets in elements), and
 * a parallel array gives n and whether it adds (n * 2 + add). */
int bine_plan_moves(bine_comm_t comm, bine_coll_t coll, long count, int root, int64_t *moves, int64_t *sizes,
                    size_t cap, size_t *n_moves);

/* The reference's messages of the call: (level, src, dst, elements). */
/* Dataflow form of a call's schedule as the PIPELINED engine runs it, for
 * tests and tools.  pieces[n][3]: (move index in bine_plan_moves order,
 * first element, elements); items[n][5]: (first piece, end piece, first
 * dependency, end dependency, level); deps[n]: an item index, or -(l + 1)
 * for every item of level l.  `elem_size` and `target_items` stand for the
 * datatype and for the engine's four items per SM per level.  With level
 * fusion set (bine_comm_set_fusion > 1) it is the fused plan: pieces index
 * the moves of bine_plan_fused and levels are its passes. */
int bine_plan_flow(bine_comm_t comm, bine_coll_t coll, long count, int root, int elem_size, int target_items,
                   int64_t *pieces, size_t piece_cap, size_t *n_pieces, int32_t *items, size_t item_cap,
                   size_t *n_items, int32_t *deps, size_t dep_cap, size_t *n_deps);

int bine_plan_messages(bine_comm_t comm, bine_coll_t coll, long count, int root, int64_t *msgs, size_t cap,
                       size_t *n_msgs);

/* The fused form of a call's schedule at `levels` levels per pass, as the
 * PIPELINED engine runs it with bine_comm_set_fusion(levels), for tests and
 * tools.  moves[n][6]: (pass, elements, first leaf, leaves, first
 * destination, destinations); leaves[n][4]: (rank, buffer, additions after
 * it, element offset of position 0) in postfix order; dsts[n][3]: (rank,
 * buffer, element offset of position 0).  Counts and *tmp_elems (workspace
 * elements per rank, renaming slots included) are always returned; arrays
 * are filled when their capacity suffices. */
int bine_plan_fused(bine_comm_t comm, bine_coll_t coll, long count, int root, int levels, int64_t *moves,
                    size_t move_cap, size_t *n_moves, int64_t *leaves, size_t leaf_cap, size_t *n_leaves,
                    int64_t *dsts, size_t dst_cap, size_t *n_dsts, int64_t *tmp_elems);

/* Exact reduction trees (allreduce, reduce_scatter, reduce): postfix
 * programs of (rank, adds, shift) entries and output segments of
 * (offset, n, rank (-1: all), program begin, program length, depth). */
int bine_plan_trees(bine_comm_t comm, bine_coll_t coll, long count, int root, int64_t *prog, size_t prog_cap,
                    size_t *n_prog, int64_t *segs, size_t seg_cap, size_t *n_segs);

/* Per-link byte counts of the call's messages on the communicator's torus
 * (minimal ring routes; 2*ndims directed links per rank, index
 * (rank*ndims + d)*2 + (0: + direction, 1: - direction)).  Computed on the
 * host from the planned schedule. */
int bine_link_bytes_host(bine_comm_t comm, bine_coll_t coll, long count, bine_datatype_t datatype, int root,
                         uint64_t *link_bytes, size_t cap);

/* The same per-link byte counts computed on the GPU into the device array
 * d_link_bytes (2*ndims*nranks uint64 values, overwritten), asynchronously
 * on the communicator's stream.  For the bandwidth-optimal (B, B_COALESCE)
 * and latency-optimal (L) allreduce and the contiguous allgather on tori
 * whose dimensions are powers of two, the messages are generated on the
 * device from the step math (no host planning, any size up to 2^20
 * ranks); other cases aggregate the planned message list on the device.
 * Stands in for the link traffic of simulation/simulator.py:125-177 and
 * simulation/out_bytes.py:18-69. */
int bine_link_bytes(bine_comm_t comm, bine_coll_t coll, long count, bine_datatype_t datatype, int root,
                    uint64_t *d_link_bytes);

#ifdef __cplusplus
}
#endif

#endif /* BINE_B200_H */

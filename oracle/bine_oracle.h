/*
 * CPU restatement of the reference's MPI-layer Bine collectives
 * (test infrastructure: the oracle).  Only tests, the smoke check and the
 * benchmark's CPU-baseline leg use it; the product never links it.
 *
 * One call runs one collective over P simulated ranks in this process,
 * step by step as the reference's per-rank code does, and returns every
 * rank's result buffer plus the list of point-to-point messages
 * (src, dst, bytes) the reference would send.  Buffers are rank-major:
 * `in` holds P send buffers, `out` receives P result buffers, sized per
 * rank as bench/bench.cc:178-207 sizes them.
 */
#ifndef BINE_ORACLE_H
#define BINE_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Element types (same numbering as the product's bine_datatype_t). */
enum { OR_INT32 = 0, OR_INT64 = 1, OR_FLOAT = 2, OR_DOUBLE = 3, OR_CHAR = 4 };

/* Collectives. */
enum {
    OR_ALLREDUCE = 0,
    OR_REDUCE_SCATTER = 1,
    OR_ALLGATHER = 2,
    OR_BCAST = 3,
    OR_REDUCE = 4,
    OR_ALLTOALL = 5,
    OR_SCATTER = 6,
    OR_GATHER = 7
};

/* Algorithm variants, per collective (the reference's LIBBINE_<COLL>_ALGO). */
enum {
    OR_AR_L = 0, OR_AR_B = 1, OR_AR_B_CONT = 3, OR_AR_B_COALESCE = 4, /* lib/libbine_common.h:74-80 */
    OR_AG_CONT_PERMUTE = 0, OR_AG_CONT_SEND = 1, OR_AG_BLOCKS = 2,    /* lib/libbine_common.h:82-87 */
    OR_RS_CONT_PERMUTE = 0,                                          /* lib/libbine_common.h:89-94 */
    OR_BC_BINOMIAL_TREE = 0, OR_BC_SCATTER_ALLGATHER = 2,            /* lib/libbine_common.h:96-100 */
    OR_RD_BINOMIAL_TREE = 0, OR_RD_REDUCE_SCATTER_GATHER = 1,         /* lib/libbine_common.h:120-123 */
    OR_A2A_LOG = 0, OR_SC_CONT_PERMUTE = 0, OR_GA_CONT_PERMUTE = 0
};

/* Algorithm families (lib/libbine_common.h:75-86). */
enum { OR_FAMILY_BINE = 1, OR_FAMILY_RECDOUB = 2, OR_FAMILY_BRUCK = 3, OR_FAMILY_RING = 4 };

/* Distance types (lib/libbine_common.h:65-68). */
enum { OR_DIST_INCREASING = 0, OR_DIST_DECREASING = 1 };

typedef struct {
    int coll;
    int algo;
    int family;
    int distance;   /* -1 = the reference's default for this collective */
    int dtype;
    int nranks;
    int ndims;      /* 0 = one dimension of size nranks */
    int dims[3];
    int ports;
    int root;
    long count;     /* the reference's `count` argument for this collective */
} oracle_call_t;

typedef struct {
    int32_t src;
    int32_t dst;
    uint64_t bytes;
} oracle_msg_t;

/* Return codes. */
enum {
    OR_OK = 0,
    OR_ERR_ARG = 1,
    /* The reference rejects this case: it asserts, exits, crashes, hangs or
     * returns wrong data for it (the message says which). */
    OR_ERR_REFERENCE_UNSUPPORTED = 2,
    OR_ERR_INTERNAL = 3
};

/* Per-rank element counts of the send and result buffers. */
int oracle_buffer_counts(const oracle_call_t *call, long *send_count, long *recv_count);

/* Runs the collective.  `msgs` may be NULL; otherwise up to `msg_cap`
 * messages are stored and *n_msgs receives the total number sent. */
int oracle_run(const oracle_call_t *call, const void *in, void *out, oracle_msg_t *msgs, size_t msg_cap,
               size_t *n_msgs);

/* Text of the last error of this thread. */
const char *oracle_last_error(void);

/* Schedule helpers exposed for known-answer tests. */
uint32_t oracle_remap_rank(uint32_t nranks, uint32_t rank);             /* simulation/remap_rank.c:64-70 */
uint32_t oracle_get_nu(uint32_t rank, uint32_t nranks);                  /* lib/libbine_coll_allgather.cc:1125-1158 */
int oracle_remap_distance_doubling(uint32_t num);                       /* lib/libbine_coll_alltoall.cc:400-409 */
int oracle_compute_peers(int rank, int port, int family, int ndims, const int *dims, int *peers_out);
int oracle_get_tree(int root, int port, int family, int distance, int ndims, const int *dims, uint32_t *parent,
                    uint32_t *reached_at_step, uint32_t *remapped_ranks, uint32_t *remapped_ranks_max,
                    uint32_t *subtree_roots);
int oracle_block_step(int rank, int port, int family, int ndims, const int *dims, uint32_t *block_step_out);

#ifdef __cplusplus
}
#endif

#endif

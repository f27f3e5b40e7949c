/*
 * mpi.h for the single-host MPI shim that the oracle builds the reference
 * library against (test infrastructure only; never part of the product).
 *
 * Declares exactly the subset of the MPI-3 C API that the reference's
 * MPI-layer collectives (lib/libbine*.cc), its uTofu helpers
 * (lib/fugaku/bine_utofu.cc) and the oracle harness call.  Handles are small
 * integers and requests are pointers, as the MPI standard permits; names,
 * argument order and semantics follow the MPI standard so that the reference
 * compiles unmodified.  The runtime is oracle/mpishim/mpishim.c: one forked
 * process per rank, eager point-to-point over a shared-memory arena.
 */
#ifndef BINE_MPISHIM_MPI_H
#define BINE_MPISHIM_MPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef intptr_t MPI_Aint;
typedef struct shim_request *MPI_Request;

typedef struct {
    int MPI_SOURCE;
    int MPI_TAG;
    int MPI_ERROR;
    size_t shim_bytes;
} MPI_Status;

typedef void (MPI_User_function)(void *invec, void *inoutvec, int *len, MPI_Datatype *datatype);

#define MPI_SUCCESS        0
#define MPI_ERR_OTHER      15
#define MPI_ERR_TRUNCATE   14
#define MPI_ERR_ARG        12
#define MPI_UNDEFINED      (-32766)

#define MPI_COMM_WORLD     ((MPI_Comm) 1)
#define MPI_COMM_NULL      ((MPI_Comm) 0)

#define MPI_DATATYPE_NULL  ((MPI_Datatype) 0)
#define MPI_CHAR           ((MPI_Datatype) 1)
#define MPI_BYTE           ((MPI_Datatype) 2)
#define MPI_INT            ((MPI_Datatype) 3)
#define MPI_INT32_T        ((MPI_Datatype) 4)
#define MPI_INT64_T        ((MPI_Datatype) 5)
#define MPI_UINT64_T       ((MPI_Datatype) 6)
#define MPI_UINT           ((MPI_Datatype) 7)
#define MPI_UNSIGNED       ((MPI_Datatype) 7)
#define MPI_FLOAT          ((MPI_Datatype) 8)
#define MPI_DOUBLE         ((MPI_Datatype) 9)
#define MPI_LONG           ((MPI_Datatype) 10)
#define MPI_UNSIGNED_LONG  ((MPI_Datatype) 11)

#define MPI_OP_NULL        ((MPI_Op) 0)
#define MPI_SUM            ((MPI_Op) 1)
#define MPI_MAX            ((MPI_Op) 2)
#define MPI_MIN            ((MPI_Op) 3)

#define MPI_PROC_NULL      (-2)
#define MPI_ANY_SOURCE     (-1)
#define MPI_ANY_TAG        (-1)
#define MPI_REQUEST_NULL   ((MPI_Request) 0)
#define MPI_STATUS_IGNORE  ((MPI_Status *) 0)
#define MPI_STATUSES_IGNORE ((MPI_Status *) 0)
#define MPI_IN_PLACE       ((void *) 1)
#define MPI_MAX_INFO_VAL   1024

/* Environment */
int MPI_Init(int *argc, char ***argv);
int PMPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int PMPI_Finalize(void);
int MPI_Abort(MPI_Comm comm, int errorcode);
double MPI_Wtime(void);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Type_size(MPI_Datatype datatype, int *size);
int MPI_Op_create(MPI_User_function *fn, int commute, MPI_Op *op);
int MPI_Barrier(MPI_Comm comm);
int PMPI_Comm_size(MPI_Comm comm, int *size);
int PMPI_Comm_rank(MPI_Comm comm, int *rank);
int PMPI_Type_size(MPI_Datatype datatype, int *size);
int PMPI_Barrier(MPI_Comm comm);

/* Point to point */
int MPI_Send(const void *buf, int count, MPI_Datatype dt, int dest, int tag, MPI_Comm comm);
int MPI_Recv(void *buf, int count, MPI_Datatype dt, int source, int tag, MPI_Comm comm, MPI_Status *status);
int MPI_Isend(const void *buf, int count, MPI_Datatype dt, int dest, int tag, MPI_Comm comm, MPI_Request *req);
int MPI_Irecv(void *buf, int count, MPI_Datatype dt, int source, int tag, MPI_Comm comm, MPI_Request *req);
int MPI_Sendrecv(const void *sendbuf, int sendcount, MPI_Datatype sendtype, int dest, int sendtag,
                 void *recvbuf, int recvcount, MPI_Datatype recvtype, int source, int recvtag,
                 MPI_Comm comm, MPI_Status *status);
int MPI_Sendrecv_replace(void *buf, int count, MPI_Datatype dt, int dest, int sendtag,
                         int source, int recvtag, MPI_Comm comm, MPI_Status *status);
int MPI_Wait(MPI_Request *req, MPI_Status *status);
int MPI_Waitall(int count, MPI_Request reqs[], MPI_Status statuses[]);
int MPI_Waitany(int count, MPI_Request reqs[], int *index, MPI_Status *status);
int MPI_Reduce_local(const void *inbuf, void *inoutbuf, int count, MPI_Datatype dt, MPI_Op op);

/* Collectives: only the profiling (PMPI_) names are provided by the shim, so
 * that the reference library's own MPI_* definitions are the ones linked. */
int PMPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype dt, MPI_Op op, MPI_Comm comm);
int PMPI_Reduce_scatter(const void *sendbuf, void *recvbuf, const int recvcounts[], MPI_Datatype dt, MPI_Op op, MPI_Comm comm);
int PMPI_Allgather(const void *sendbuf, int sendcount, MPI_Datatype sendtype, void *recvbuf, int recvcount, MPI_Datatype recvtype, MPI_Comm comm);
int PMPI_Bcast(void *buf, int count, MPI_Datatype dt, int root, MPI_Comm comm);
int PMPI_Alltoall(const void *sendbuf, int sendcount, MPI_Datatype sendtype, void *recvbuf, int recvcount, MPI_Datatype recvtype, MPI_Comm comm);
int PMPI_Scatter(const void *sendbuf, int sendcount, MPI_Datatype sendtype, void *recvbuf, int recvcount, MPI_Datatype recvtype, int root, MPI_Comm comm);
int PMPI_Gather(const void *sendbuf, int sendcount, MPI_Datatype sendtype, void *recvbuf, int recvcount, MPI_Datatype recvtype, int root, MPI_Comm comm);
int PMPI_Reduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype dt, MPI_Op op, int root, MPI_Comm comm);

/* The reference's own collective entry points (lib/libbine.cc). */
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype dt, MPI_Op op, MPI_Comm comm);
int MPI_Reduce_scatter(const void *sendbuf, void *recvbuf, const int recvcounts[], MPI_Datatype dt, MPI_Op op, MPI_Comm comm);
int MPI_Allgather(const void *sendbuf, int sendcount, MPI_Datatype sendtype, void *recvbuf, int recvcount, MPI_Datatype recvtype, MPI_Comm comm);
int MPI_Bcast_f(void *buf, int count, MPI_Datatype dt, int root, MPI_Comm comm);
int MPI_Alltoall(const void *sendbuf, int sendcount, MPI_Datatype sendtype, void *recvbuf, int recvcount, MPI_Datatype recvtype, MPI_Comm comm);
int MPI_Scatter(const void *sendbuf, int sendcount, MPI_Datatype sendtype, void *recvbuf, int recvcount, MPI_Datatype recvtype, int root, MPI_Comm comm);
int MPI_Gather(const void *sendbuf, int sendcount, MPI_Datatype sendtype, void *recvbuf, int recvcount, MPI_Datatype recvtype, int root, MPI_Comm comm);
int MPI_Reduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype dt, MPI_Op op, int root, MPI_Comm comm);

/* Shim control, used by the oracle harness only. */
typedef struct {
    int32_t src, dst, tag;
    int32_t call;          /* collective-call sequence number on the sender */
    uint64_t bytes;
} shim_trace_entry_t;

/* Creates the shared state for `nranks` ranks; call once in the launcher
 * before forking.  arena_bytes_per_rank bounds the eager send buffer space
 * of each rank; trace_cap is the per-rank message trace capacity (0 = off). */
int shim_setup(int nranks, size_t arena_bytes_per_rank, size_t trace_cap, double timeout_s);
/* Called in each forked child before MPI_Init. */
void shim_set_rank(int rank);
/* Marks the start of a new traced collective call on this rank. */
void shim_trace_next_call(void);
/* Per-rank trace access (valid in the launcher after the children exit). */
size_t shim_trace_count(int rank, size_t *dropped);
const shim_trace_entry_t *shim_trace_entries(int rank);
/* Sets the abort flag that makes every waiting rank exit. */
void shim_abort_all(void);
/* Allocates `bytes` of memory shared by all ranks (launcher only). */
void *shim_shared_alloc(size_t bytes);

#ifdef __cplusplus
}
#endif

#endif /* BINE_MPISHIM_MPI_H */

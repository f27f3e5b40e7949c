/*
 * Single-host MPI runtime that the oracle links the unmodified reference
 * library against (test infrastructure only; nothing in the product links
 * it).
 *
 * Model: the oracle harness calls shim_setup() and then forks one process
 * per rank.  All shared state lives in anonymous MAP_SHARED mappings created
 * before the fork, so raw pointers are valid in every rank.
 *
 *  - Point-to-point is eager.  MPI_Isend copies the payload into the
 *    sender's own slice of a shared arena and appends a descriptor to the
 *    destination's mailbox (a FIFO list); the send completes at once.
 *  - Receives are matched in the order they were posted against the FIFO
 *    mailbox, which gives MPI's non-overtaking guarantee per (source, tag):
 *    the reference's bitmap allreduce posts several same-tag receives from
 *    one peer and completes them with MPI_Waitany
 *    (lib/libbine_common.cc:965-1016).
 *  - MPI_Reduce_local(in, inout) computes inout[i] = in[i] + inout[i].
 *  - Every wait is bounded: after the configured timeout a rank reports
 *    which call it was stuck in and exits with status 124, and a rank that
 *    sees another rank's abort exits with status 125, so a lost message
 *    surfaces as an error instead of a hang.
 *  - Each send can be recorded (src, dst, tag, bytes, call number) in a
 *    per-rank trace: the ground truth for link-byte accounting.
 */
#define _GNU_SOURCE
#include "mpi.h"

#include <errno.h>
#include <limits.h>
#include <linux/futex.h>
#include <sched.h>
#include <stdatomic.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/syscall.h>
#include <time.h>
#include <unistd.h>

#define SHIM_ALIGN 64
#define SHIM_TAG_COLL (-100) /* internal tags for the PMPI_ collectives */

struct shim_msg {
    struct shim_msg *next;
    int src;
    int tag;
    size_t bytes;
    char pad[SHIM_ALIGN - sizeof(void *) - 2 * sizeof(int) - sizeof(size_t)];
};

struct shim_mailbox {
    atomic_int lock;
    atomic_uint seq;
    struct shim_msg *head;
    struct shim_msg *tail;
    char pad[SHIM_ALIGN - 2 * sizeof(int) - 2 * sizeof(void *)];
};

struct shim_arena_meta {
    atomic_long live;
    atomic_uint freed_seq;
    size_t bump;
    size_t trace_count;
    size_t trace_dropped;
    int call;
    char pad[SHIM_ALIGN - sizeof(long) - sizeof(int) - 3 * sizeof(size_t) - sizeof(int)];
};

struct shim_shared {
    int nranks;
    double timeout_s;
    size_t arena_bytes;
    size_t trace_cap;
    atomic_int abort_flag;
    atomic_uint bar_count;
    atomic_uint bar_gen;
};

struct shim_request {
    int is_recv;
    int done;
    int src;
    int tag;
    void *buf;
    size_t cap;
    MPI_Status st;
    struct shim_msg *matched;
    struct shim_request *next_pending;
};

static struct shim_shared *g_sh;
static struct shim_mailbox *g_mb;
static struct shim_arena_meta *g_am;
static char *g_arena;
static shim_trace_entry_t *g_trace;
static int g_rank = -1;
static struct shim_request *g_pend_head, *g_pend_tail;

#define MAX_USER_OPS 16
static MPI_User_function *g_user_ops[MAX_USER_OPS];
static int g_num_user_ops;

static void *map_shared(size_t bytes) {
    void *p = mmap(NULL, bytes, PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS | MAP_NORESERVE, -1, 0);
    if (p == MAP_FAILED) {
        perror("mpishim: mmap");
        return NULL;
    }
    return p;
}

int shim_setup(int nranks, size_t arena_bytes_per_rank, size_t trace_cap, double timeout_s) {
    size_t ctl = sizeof(struct shim_shared) + SHIM_ALIGN;
    ctl += (size_t)nranks * (sizeof(struct shim_mailbox) + sizeof(struct shim_arena_meta)) + SHIM_ALIGN;
    char *base = (char *)map_shared(ctl);
    if (!base) return -1;
    memset(base, 0, ctl);
    g_sh = (struct shim_shared *)base;
    g_mb = (struct shim_mailbox *)(base + ((sizeof(struct shim_shared) + SHIM_ALIGN - 1) / SHIM_ALIGN) * SHIM_ALIGN);
    g_am = (struct shim_arena_meta *)(g_mb + nranks);
    g_sh->nranks = nranks;
    g_sh->timeout_s = timeout_s;
    arena_bytes_per_rank = (arena_bytes_per_rank + 4095) & ~(size_t)4095;
    g_sh->arena_bytes = arena_bytes_per_rank;
    g_sh->trace_cap = trace_cap;
    g_arena = (char *)map_shared(arena_bytes_per_rank * (size_t)nranks);
    if (!g_arena) return -1;
    if (trace_cap) {
        g_trace = (shim_trace_entry_t *)map_shared(sizeof(shim_trace_entry_t) * trace_cap * (size_t)nranks);
        if (!g_trace) return -1;
    }
    return 0;
}

void *shim_shared_alloc(size_t bytes) { return map_shared(bytes ? bytes : 1); }

void shim_set_rank(int rank) { g_rank = rank; }

void shim_abort_all(void) {
    if (g_sh) atomic_store(&g_sh->abort_flag, 1);
}

void shim_trace_next_call(void) {
    if (g_rank >= 0) g_am[g_rank].call++;
}

size_t shim_trace_count(int rank, size_t *dropped) {
    if (dropped) *dropped = g_am[rank].trace_dropped;
    return g_am[rank].trace_count;
}

const shim_trace_entry_t *shim_trace_entries(int rank) {
    return g_trace ? g_trace + (size_t)rank * g_sh->trace_cap : NULL;
}

/* ---------------------------------------------------------------- waiting */

static double now_s(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + ts.tv_nsec * 1e-9;
}

static void futex_wait(atomic_uint *addr, unsigned val) {
    struct timespec ts = {0, 20 * 1000 * 1000};
    syscall(SYS_futex, (unsigned *)addr, FUTEX_WAIT, val, &ts, NULL, 0);
}

static void futex_wake(atomic_uint *addr) {
    syscall(SYS_futex, (unsigned *)addr, FUTEX_WAKE, INT_MAX, NULL, NULL, 0);
}

static void check_deadline(double t0, const char *where) {
    if (atomic_load(&g_sh->abort_flag)) _exit(125);
    if (now_s() - t0 > g_sh->timeout_s) {
        fprintf(stderr, "mpishim: rank %d timed out after %.0f s in %s\n", g_rank, g_sh->timeout_s, where);
        fflush(stderr);
        atomic_store(&g_sh->abort_flag, 1);
        _exit(124);
    }
}

static void lock_mb(struct shim_mailbox *mb) {
    int spins = 0;
    while (atomic_exchange_explicit(&mb->lock, 1, memory_order_acquire)) {
        if (++spins > 64) {
            sched_yield();
            spins = 0;
        }
    }
}

static void unlock_mb(struct shim_mailbox *mb) { atomic_store_explicit(&mb->lock, 0, memory_order_release); }

/* ------------------------------------------------------------------ basic */

int PMPI_Init(int *argc, char ***argv) {
    (void)argc;
    (void)argv;
    if (!g_sh || g_rank < 0) {
        fprintf(stderr, "mpishim: PMPI_Init before shim_setup/shim_set_rank\n");
        return MPI_ERR_OTHER;
    }
    return MPI_SUCCESS;
}

int PMPI_Finalize(void) { return MPI_SUCCESS; }

int MPI_Abort(MPI_Comm comm, int errorcode) {
    (void)comm;
    fprintf(stderr, "mpishim: rank %d called MPI_Abort(%d)\n", g_rank, errorcode);
    shim_abort_all();
    _exit(errorcode ? errorcode : 1);
}

double MPI_Wtime(void) { return now_s(); }

int MPI_Comm_size(MPI_Comm comm, int *size) {
    (void)comm;
    *size = g_sh->nranks;
    return MPI_SUCCESS;
}

int MPI_Comm_rank(MPI_Comm comm, int *rank) {
    (void)comm;
    *rank = g_rank;
    return MPI_SUCCESS;
}

static int dt_size(MPI_Datatype dt) {
    switch (dt) {
    case MPI_CHAR:
    case MPI_BYTE: return 1;
    case MPI_INT:
    case MPI_INT32_T:
    case MPI_UINT:
    case MPI_FLOAT: return 4;
    case MPI_INT64_T:
    case MPI_UINT64_T:
    case MPI_DOUBLE:
    case MPI_LONG:
    case MPI_UNSIGNED_LONG: return 8;
    default: return -1;
    }
}

int MPI_Type_size(MPI_Datatype datatype, int *size) {
    int s = dt_size(datatype);
    if (s < 0) return MPI_ERR_ARG;
    *size = s;
    return MPI_SUCCESS;
}

int MPI_Op_create(MPI_User_function *fn, int commute, MPI_Op *op) {
    (void)commute;
    if (g_num_user_ops >= MAX_USER_OPS) return MPI_ERR_OTHER;
    g_user_ops[g_num_user_ops] = fn;
    *op = 16 + g_num_user_ops++;
    return MPI_SUCCESS;
}

int MPI_Barrier(MPI_Comm comm) {
    (void)comm;
    unsigned gen = atomic_load(&g_sh->bar_gen);
    if (atomic_fetch_add(&g_sh->bar_count, 1) == (unsigned)g_sh->nranks - 1) {
        atomic_store(&g_sh->bar_count, 0);
        atomic_fetch_add(&g_sh->bar_gen, 1);
        futex_wake(&g_sh->bar_gen);
        return MPI_SUCCESS;
    }
    double t0 = now_s();
    while (atomic_load(&g_sh->bar_gen) == gen) {
        futex_wait(&g_sh->bar_gen, gen);
        check_deadline(t0, "MPI_Barrier");
    }
    return MPI_SUCCESS;
}

/* The PMPI_ names of the calls above (every MPI provides both; a PMPI
 * interposition layer calls these). */
int PMPI_Comm_size(MPI_Comm comm, int *size) { return MPI_Comm_size(comm, size); }
int PMPI_Comm_rank(MPI_Comm comm, int *rank) { return MPI_Comm_rank(comm, rank); }
int PMPI_Type_size(MPI_Datatype datatype, int *size) { return MPI_Type_size(datatype, size); }
int PMPI_Barrier(MPI_Comm comm) { return MPI_Barrier(comm); }

/* --------------------------------------------------------- point to point */

static struct shim_msg *arena_alloc(size_t payload) {
    struct shim_arena_meta *am = &g_am[g_rank];
    size_t need = sizeof(struct shim_msg) + ((payload + SHIM_ALIGN - 1) / SHIM_ALIGN) * SHIM_ALIGN;
    if (need > g_sh->arena_bytes) {
        fprintf(stderr, "mpishim: rank %d: message of %zu bytes exceeds the %zu-byte arena\n", g_rank, payload,
                g_sh->arena_bytes);
        shim_abort_all();
        _exit(123);
    }
    if (atomic_load(&am->live) == 0) am->bump = 0;
    if (am->bump + need > g_sh->arena_bytes) {
        /* Wait until every outstanding message of this rank is consumed. */
        double t0 = now_s();
        while (atomic_load(&am->live) != 0) {
            unsigned s = atomic_load(&am->freed_seq);
            if (atomic_load(&am->live) == 0) break;
            futex_wait(&am->freed_seq, s);
            check_deadline(t0, "send (arena full)");
        }
        am->bump = 0;
    }
    struct shim_msg *m = (struct shim_msg *)(g_arena + (size_t)g_rank * g_sh->arena_bytes + am->bump);
    am->bump += need;
    return m;
}

static void trace_send(int dst, int tag, size_t bytes) {
    if (!g_trace) return;
    struct shim_arena_meta *am = &g_am[g_rank];
    if (am->trace_count >= g_sh->trace_cap) {
        am->trace_dropped++;
        return;
    }
    shim_trace_entry_t *e = g_trace + (size_t)g_rank * g_sh->trace_cap + am->trace_count++;
    e->src = g_rank;
    e->dst = dst;
    e->tag = tag;
    e->call = am->call;
    e->bytes = bytes;
}

static void post_send(const void *buf, size_t bytes, int dst, int tag) {
    struct shim_msg *m = arena_alloc(bytes);
    m->next = NULL;
    m->src = g_rank;
    m->tag = tag;
    m->bytes = bytes;
    if (bytes) memcpy((char *)(m + 1), buf, bytes);
    atomic_fetch_add(&g_am[g_rank].live, 1);
    if (tag >= 0) trace_send(dst, tag, bytes);
    struct shim_mailbox *mb = &g_mb[dst];
    lock_mb(mb);
    if (mb->tail)
        mb->tail->next = m;
    else
        mb->head = m;
    mb->tail = m;
    unlock_mb(mb);
    atomic_fetch_add(&mb->seq, 1);
    futex_wake(&mb->seq);
}

static struct shim_request *new_req(int is_recv) {
    struct shim_request *r = (struct shim_request *)calloc(1, sizeof(*r));
    r->is_recv = is_recv;
    return r;
}

int MPI_Isend(const void *buf, int count, MPI_Datatype dt, int dest, int tag, MPI_Comm comm, MPI_Request *req) {
    (void)comm;
    struct shim_request *r = new_req(0);
    r->done = 1;
    if (dest != MPI_PROC_NULL) {
        int s = dt_size(dt);
        if (s < 0 || count < 0 || dest < 0 || dest >= g_sh->nranks) {
            free(r);
            return MPI_ERR_ARG;
        }
        post_send(buf, (size_t)count * s, dest, tag);
    }
    *req = r;
    return MPI_SUCCESS;
}

int MPI_Irecv(void *buf, int count, MPI_Datatype dt, int source, int tag, MPI_Comm comm, MPI_Request *req) {
    (void)comm;
    struct shim_request *r = new_req(1);
    if (source == MPI_PROC_NULL) {
        r->done = 1;
        r->st.MPI_SOURCE = MPI_PROC_NULL;
        *req = r;
        return MPI_SUCCESS;
    }
    int s = dt_size(dt);
    if (s < 0 || count < 0) {
        free(r);
        return MPI_ERR_ARG;
    }
    r->src = source;
    r->tag = tag;
    r->buf = buf;
    r->cap = (size_t)count * s;
    if (g_pend_tail)
        g_pend_tail->next_pending = r;
    else
        g_pend_head = r;
    g_pend_tail = r;
    *req = r;
    return MPI_SUCCESS;
}

/* Matches pending receives, in posting order, against the mailbox FIFO. */
static void progress(void) {
    if (!g_pend_head) return;
    struct shim_mailbox *mb = &g_mb[g_rank];
    struct shim_request *matched_list = NULL, **mtail = &matched_list;
    lock_mb(mb);
    struct shim_request *prev = NULL, *r = g_pend_head;
    while (r) {
        struct shim_request *next = r->next_pending;
        struct shim_msg *mprev = NULL, *m = mb->head;
        while (m) {
            if ((r->src == MPI_ANY_SOURCE || r->src == m->src) && (r->tag == MPI_ANY_TAG || r->tag == m->tag)) break;
            mprev = m;
            m = m->next;
        }
        if (m) {
            if (mprev)
                mprev->next = m->next;
            else
                mb->head = m->next;
            if (mb->tail == m) mb->tail = mprev;
            r->matched = m;
            if (prev)
                prev->next_pending = next;
            else
                g_pend_head = next;
            if (g_pend_tail == r) g_pend_tail = prev;
            r->next_pending = NULL;
            *mtail = r;
            mtail = &r->next_pending;
        } else {
            prev = r;
        }
        r = next;
    }
    unlock_mb(mb);
    for (r = matched_list; r;) {
        struct shim_request *next = r->next_pending;
        struct shim_msg *m = r->matched;
        size_t n = m->bytes;
        if (n > r->cap) {
            fprintf(stderr, "mpishim: rank %d: message of %zu bytes from %d truncated to %zu\n", g_rank, n, m->src,
                    r->cap);
            r->st.MPI_ERROR = MPI_ERR_TRUNCATE;
            n = r->cap;
        }
        if (n) memcpy(r->buf, (char *)(m + 1), n);
        r->st.MPI_SOURCE = m->src;
        r->st.MPI_TAG = m->tag;
        r->st.shim_bytes = n;
        int src = m->src;
        atomic_fetch_sub(&g_am[src].live, 1);
        atomic_fetch_add(&g_am[src].freed_seq, 1);
        futex_wake(&g_am[src].freed_seq);
        r->matched = NULL;
        r->done = 1;
        r = next;
    }
}

static int finish(MPI_Request *req, MPI_Status *status) {
    struct shim_request *r = *req;
    int err = r->st.MPI_ERROR;
    if (status) *status = r->st;
    free(r);
    *req = MPI_REQUEST_NULL;
    return err ? err : MPI_SUCCESS;
}

int MPI_Wait(MPI_Request *req, MPI_Status *status) {
    if (!*req) return MPI_SUCCESS;
    double t0 = now_s();
    struct shim_mailbox *mb = &g_mb[g_rank];
    while (1) {
        unsigned s = atomic_load(&mb->seq);
        progress();
        if ((*req)->done) return finish(req, status);
        futex_wait(&mb->seq, s);
        check_deadline(t0, "MPI_Wait");
    }
}

int MPI_Waitall(int count, MPI_Request reqs[], MPI_Status statuses[]) {
    int err = MPI_SUCCESS;
    for (int i = 0; i < count; i++) {
        int e = MPI_Wait(&reqs[i], statuses ? &statuses[i] : NULL);
        if (e != MPI_SUCCESS) err = e;
    }
    return err;
}

int MPI_Waitany(int count, MPI_Request reqs[], int *index, MPI_Status *status) {
    double t0 = now_s();
    struct shim_mailbox *mb = &g_mb[g_rank];
    while (1) {
        unsigned s = atomic_load(&mb->seq);
        progress();
        int active = 0;
        for (int i = 0; i < count; i++) {
            if (!reqs[i]) continue;
            active = 1;
            if (reqs[i]->done) {
                *index = i;
                return finish(&reqs[i], status);
            }
        }
        if (!active) {
            *index = MPI_UNDEFINED;
            return MPI_SUCCESS;
        }
        futex_wait(&mb->seq, s);
        check_deadline(t0, "MPI_Waitany");
    }
}

int MPI_Send(const void *buf, int count, MPI_Datatype dt, int dest, int tag, MPI_Comm comm) {
    MPI_Request r;
    int e = MPI_Isend(buf, count, dt, dest, tag, comm, &r);
    if (e != MPI_SUCCESS) return e;
    return MPI_Wait(&r, MPI_STATUS_IGNORE);
}

int MPI_Recv(void *buf, int count, MPI_Datatype dt, int source, int tag, MPI_Comm comm, MPI_Status *status) {
    MPI_Request r;
    int e = MPI_Irecv(buf, count, dt, source, tag, comm, &r);
    if (e != MPI_SUCCESS) return e;
    return MPI_Wait(&r, status);
}

int MPI_Sendrecv(const void *sendbuf, int sendcount, MPI_Datatype sendtype, int dest, int sendtag, void *recvbuf,
                 int recvcount, MPI_Datatype recvtype, int source, int recvtag, MPI_Comm comm, MPI_Status *status) {
    MPI_Request r[2];
    int e = MPI_Isend(sendbuf, sendcount, sendtype, dest, sendtag, comm, &r[0]);
    if (e != MPI_SUCCESS) return e;
    e = MPI_Irecv(recvbuf, recvcount, recvtype, source, recvtag, comm, &r[1]);
    if (e != MPI_SUCCESS) return e;
    MPI_Wait(&r[0], MPI_STATUS_IGNORE);
    return MPI_Wait(&r[1], status);
}

int MPI_Sendrecv_replace(void *buf, int count, MPI_Datatype dt, int dest, int sendtag, int source, int recvtag,
                         MPI_Comm comm, MPI_Status *status) {
    /* The eager send has copied buf before the receive is posted. */
    MPI_Request r;
    int e = MPI_Isend(buf, count, dt, dest, sendtag, comm, &r);
    if (e != MPI_SUCCESS) return e;
    MPI_Wait(&r, MPI_STATUS_IGNORE);
    return MPI_Recv(buf, count, dt, source, recvtag, comm, status);
}

#define SUM_LOOP(T)                                                                                               \
    do {                                                                                                          \
        const T *a = (const T *)inbuf;                                                                            \
        T *b = (T *)inoutbuf;                                                                                     \
        for (int i = 0; i < count; i++) b[i] = a[i] + b[i];                                                       \
    } while (0)
#define MINMAX_LOOP(T, CMP)                                                                                       \
    do {                                                                                                          \
        const T *a = (const T *)inbuf;                                                                            \
        T *b = (T *)inoutbuf;                                                                                     \
        for (int i = 0; i < count; i++)                                                                           \
            if (a[i] CMP b[i]) b[i] = a[i];                                                                       \
    } while (0)

int MPI_Reduce_local(const void *inbuf, void *inoutbuf, int count, MPI_Datatype dt, MPI_Op op) {
    if (op >= 16) {
        if (op - 16 >= g_num_user_ops) return MPI_ERR_ARG;
        g_user_ops[op - 16]((void *)inbuf, inoutbuf, &count, &dt);
        return MPI_SUCCESS;
    }
    if (op == MPI_SUM) {
        switch (dt) {
        case MPI_CHAR: SUM_LOOP(signed char); break;
        case MPI_BYTE: SUM_LOOP(unsigned char); break;
        case MPI_INT:
        case MPI_INT32_T: SUM_LOOP(int32_t); break;
        case MPI_UINT: SUM_LOOP(uint32_t); break;
        case MPI_INT64_T:
        case MPI_LONG: SUM_LOOP(int64_t); break;
        case MPI_UINT64_T:
        case MPI_UNSIGNED_LONG: SUM_LOOP(uint64_t); break;
        case MPI_FLOAT: SUM_LOOP(float); break;
        case MPI_DOUBLE: SUM_LOOP(double); break;
        default: return MPI_ERR_ARG;
        }
        return MPI_SUCCESS;
    }
    if (op == MPI_MAX || op == MPI_MIN) {
        if (dt == MPI_DOUBLE) {
            if (op == MPI_MAX)
                MINMAX_LOOP(double, >);
            else
                MINMAX_LOOP(double, <);
            return MPI_SUCCESS;
        }
        if (dt == MPI_INT64_T) {
            if (op == MPI_MAX)
                MINMAX_LOOP(int64_t, >);
            else
                MINMAX_LOOP(int64_t, <);
            return MPI_SUCCESS;
        }
    }
    return MPI_ERR_ARG;
}

/* ------------------------------------------- straightforward PMPI_ collectives
 * Linear algorithms over the same point-to-point layer, used only as an
 * independent semantic cross-check (the way bench/bench.cc:107-162 validates
 * against the system MPI).  Reductions are accumulated in rank order.       */

int PMPI_Gather(const void *sendbuf, int sendcount, MPI_Datatype sendtype, void *recvbuf, int recvcount,
                MPI_Datatype recvtype, int root, MPI_Comm comm) {
    int es = dt_size(recvtype);
    if (g_rank != root) return MPI_Send(sendbuf, sendcount, sendtype, root, SHIM_TAG_COLL, comm);
    for (int r = 0; r < g_sh->nranks; r++) {
        char *dst = (char *)recvbuf + (size_t)r * recvcount * es;
        if (r == root) {
            if (sendbuf != MPI_IN_PLACE) memcpy(dst, sendbuf, (size_t)recvcount * es);
        } else {
            int e = MPI_Recv(dst, recvcount, recvtype, r, SHIM_TAG_COLL, comm, MPI_STATUS_IGNORE);
            if (e) return e;
        }
    }
    return MPI_SUCCESS;
}

int PMPI_Scatter(const void *sendbuf, int sendcount, MPI_Datatype sendtype, void *recvbuf, int recvcount,
                 MPI_Datatype recvtype, int root, MPI_Comm comm) {
    int es = dt_size(sendtype);
    if (g_rank != root) return MPI_Recv(recvbuf, recvcount, recvtype, root, SHIM_TAG_COLL, comm, MPI_STATUS_IGNORE);
    for (int r = 0; r < g_sh->nranks; r++) {
        const char *src = (const char *)sendbuf + (size_t)r * sendcount * es;
        if (r == root) {
            if (recvbuf != MPI_IN_PLACE) memcpy(recvbuf, src, (size_t)sendcount * es);
        } else {
            int e = MPI_Send(src, sendcount, sendtype, r, SHIM_TAG_COLL, comm);
            if (e) return e;
        }
    }
    return MPI_SUCCESS;
}

int PMPI_Bcast(void *buf, int count, MPI_Datatype dt, int root, MPI_Comm comm) {
    if (g_rank != root) return MPI_Recv(buf, count, dt, root, SHIM_TAG_COLL, comm, MPI_STATUS_IGNORE);
    for (int r = 0; r < g_sh->nranks; r++)
        if (r != root) {
            int e = MPI_Send(buf, count, dt, r, SHIM_TAG_COLL, comm);
            if (e) return e;
        }
    return MPI_SUCCESS;
}

int PMPI_Allgather(const void *sendbuf, int sendcount, MPI_Datatype sendtype, void *recvbuf, int recvcount,
                   MPI_Datatype recvtype, MPI_Comm comm) {
    int es = dt_size(recvtype);
    const void *mine = sendbuf == MPI_IN_PLACE ? (const char *)recvbuf + (size_t)g_rank * recvcount * es : sendbuf;
    int cnt = sendbuf == MPI_IN_PLACE ? recvcount : sendcount;
    MPI_Datatype t = sendbuf == MPI_IN_PLACE ? recvtype : sendtype;
    for (int r = 0; r < g_sh->nranks; r++)
        if (r != g_rank) MPI_Send(mine, cnt, t, r, SHIM_TAG_COLL, comm);
    if (sendbuf != MPI_IN_PLACE) memcpy((char *)recvbuf + (size_t)g_rank * recvcount * es, sendbuf, (size_t)recvcount * es);
    for (int r = 0; r < g_sh->nranks; r++)
        if (r != g_rank) {
            int e = MPI_Recv((char *)recvbuf + (size_t)r * recvcount * es, recvcount, recvtype, r, SHIM_TAG_COLL, comm,
                             MPI_STATUS_IGNORE);
            if (e) return e;
        }
    return MPI_SUCCESS;
}

int PMPI_Alltoall(const void *sendbuf, int sendcount, MPI_Datatype sendtype, void *recvbuf, int recvcount,
                  MPI_Datatype recvtype, MPI_Comm comm) {
    int es = dt_size(sendtype), er = dt_size(recvtype);
    for (int r = 0; r < g_sh->nranks; r++) {
        const char *src = (const char *)sendbuf + (size_t)r * sendcount * es;
        if (r == g_rank)
            memcpy((char *)recvbuf + (size_t)r * recvcount * er, src, (size_t)sendcount * es);
        else
            MPI_Send(src, sendcount, sendtype, r, SHIM_TAG_COLL, comm);
    }
    for (int r = 0; r < g_sh->nranks; r++)
        if (r != g_rank) {
            int e = MPI_Recv((char *)recvbuf + (size_t)r * recvcount * er, recvcount, recvtype, r, SHIM_TAG_COLL, comm,
                             MPI_STATUS_IGNORE);
            if (e) return e;
        }
    return MPI_SUCCESS;
}

int PMPI_Reduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype dt, MPI_Op op, int root, MPI_Comm comm) {
    int es = dt_size(dt);
    if (g_rank != root) return MPI_Send(sendbuf, count, dt, root, SHIM_TAG_COLL, comm);
    size_t n = (size_t)count * es;
    char *acc = (char *)malloc(n ? n : 1), *tmp = (char *)malloc(n ? n : 1);
    for (int r = 0; r < g_sh->nranks; r++) {
        const void *src;
        if (r == root) {
            src = sendbuf == MPI_IN_PLACE ? recvbuf : sendbuf;
        } else {
            MPI_Recv(tmp, count, dt, r, SHIM_TAG_COLL, comm, MPI_STATUS_IGNORE);
            src = tmp;
        }
        if (r == 0)
            memcpy(acc, src, n);
        else
            MPI_Reduce_local(src, acc, count, dt, op);
    }
    memcpy(recvbuf, acc, n);
    free(acc);
    free(tmp);
    return MPI_SUCCESS;
}

int PMPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype dt, MPI_Op op, MPI_Comm comm) {
    int e = PMPI_Reduce(sendbuf, recvbuf, count, dt, op, 0, comm);
    if (e) return e;
    return PMPI_Bcast(recvbuf, count, dt, 0, comm);
}

int PMPI_Reduce_scatter(const void *sendbuf, void *recvbuf, const int recvcounts[], MPI_Datatype dt, MPI_Op op,
                        MPI_Comm comm) {
    int es = dt_size(dt), total = 0, off = 0;
    for (int r = 0; r < g_sh->nranks; r++) {
        if (r < g_rank) off += recvcounts[r];
        total += recvcounts[r];
    }
    char *full = (char *)malloc((size_t)total * es + 1);
    int e = PMPI_Allreduce(sendbuf, full, total, dt, op, comm);
    if (!e) memcpy(recvbuf, full + (size_t)off * es, (size_t)recvcounts[g_rank] * es);
    free(full);
    return e;
}

/* ------------------------------------------------ uTofu / FJMPI stand-ins */

#include "mpi-ext.h"
#include "utofu.h"

int utofu_get_onesided_tnis(utofu_tni_id_t **tni_ids, size_t *num_tnis) {
    *num_tnis = 6;
    *tni_ids = (utofu_tni_id_t *)malloc(sizeof(utofu_tni_id_t) * 6);
    for (int i = 0; i < 6; i++) (*tni_ids)[i] = i;
    return UTOFU_SUCCESS;
}
int utofu_query_onesided_caps(utofu_tni_id_t tni_id, struct utofu_onesided_caps **caps) {
    (void)tni_id;
    *caps = NULL;
    return UTOFU_ERR_NOT_SUPPORTED;
}
int utofu_create_vcq(utofu_tni_id_t tni_id, unsigned long flags, utofu_vcq_hdl_t *vcq_hdl) {
    (void)flags;
    *vcq_hdl = (utofu_vcq_hdl_t)(intptr_t)(tni_id + 1);
    return UTOFU_SUCCESS;
}
int utofu_free_vcq(utofu_vcq_hdl_t vcq_hdl) {
    (void)vcq_hdl;
    return UTOFU_SUCCESS;
}
int utofu_query_vcq_id(utofu_vcq_hdl_t vcq_hdl, utofu_vcq_id_t *vcq_id) {
    *vcq_id = ((uint64_t)(intptr_t)vcq_hdl << 32) | (uint64_t)(g_rank < 0 ? 0 : g_rank);
    return UTOFU_SUCCESS;
}
int utofu_set_vcq_id_path(utofu_vcq_id_t *vcq_id, uint8_t *path_coords) {
    (void)vcq_id;
    (void)path_coords;
    return UTOFU_SUCCESS;
}
int utofu_reg_mem(utofu_vcq_hdl_t vcq_hdl, void *addr, size_t size, unsigned long flags, utofu_stadd_t *stadd) {
    (void)vcq_hdl;
    (void)size;
    (void)flags;
    *stadd = (utofu_stadd_t)(uintptr_t)addr;
    return UTOFU_SUCCESS;
}
int utofu_dereg_mem(utofu_vcq_hdl_t vcq_hdl, utofu_stadd_t stadd, unsigned long flags) {
    (void)vcq_hdl;
    (void)stadd;
    (void)flags;
    return UTOFU_SUCCESS;
}
int utofu_put(utofu_vcq_hdl_t vcq_hdl, utofu_vcq_id_t rmt_vcq_id, utofu_stadd_t lcl_stadd, utofu_stadd_t rmt_stadd,
              size_t length, uint64_t edata, unsigned long flags, void *cbvalue) {
    (void)vcq_hdl, (void)rmt_vcq_id, (void)lcl_stadd, (void)rmt_stadd, (void)length, (void)edata, (void)flags,
        (void)cbvalue;
    fprintf(stderr, "mpishim: the uTofu data path is not available\n");
    return UTOFU_ERR_FATAL;
}
int utofu_put_piggyback(utofu_vcq_hdl_t vcq_hdl, utofu_vcq_id_t rmt_vcq_id, void *lcl_data, utofu_stadd_t rmt_stadd,
                        size_t length, uint64_t edata, unsigned long flags, void *cbvalue) {
    (void)vcq_hdl, (void)rmt_vcq_id, (void)lcl_data, (void)rmt_stadd, (void)length, (void)edata, (void)flags,
        (void)cbvalue;
    fprintf(stderr, "mpishim: the uTofu data path is not available\n");
    return UTOFU_ERR_FATAL;
}
int utofu_poll_tcq(utofu_vcq_hdl_t vcq_hdl, unsigned long flags, void **cbdata) {
    (void)vcq_hdl, (void)flags, (void)cbdata;
    return UTOFU_ERR_FATAL;
}
int utofu_poll_mrq(utofu_vcq_hdl_t vcq_hdl, unsigned long flags, struct utofu_mrq_notice *notice) {
    (void)vcq_hdl, (void)flags, (void)notice;
    return UTOFU_ERR_FATAL;
}

int FJMPI_Topology_get_dimension(int *size) {
    (void)size;
    return FJMPI_ERR_TOPOLOGY;
}
int FJMPI_Topology_get_shape(int *x, int *y, int *z) {
    (void)x, (void)y, (void)z;
    return FJMPI_ERR_TOPOLOGY;
}
int FJMPI_Topology_get_coords(MPI_Comm comm, int rank, int view, int maxdims, int coords[]) {
    (void)comm, (void)rank, (void)view, (void)maxdims, (void)coords;
    return FJMPI_ERR_TOPOLOGY;
}
int FJMPI_Topology_get_ranks(MPI_Comm comm, int view, int coords[], int maxppn, int *outppn, int ranks[]) {
    (void)comm, (void)view, (void)coords, (void)maxppn, (void)outppn, (void)ranks;
    return FJMPI_ERR_TOPOLOGY;
}

// PMPI interposition layer: the reference's MPI entry points on the engine.
//
// The reference is a PMPI library: an MPI program links libbine.so and its
// MPI_Allreduce, MPI_Reduce_scatter, MPI_Allgather, MPI_Bcast_f,
// MPI_Alltoall, MPI_Scatter, MPI_Gather and MPI_Reduce run the Bine
// schedules over MPI (lib/libbine.cc:1012-1477).  Linking this file's
// library instead (compiled against the program's own <mpi.h>) runs the
// same calls on one GPU: the ranks of MPI_COMM_WORLD on this node become the
// engine's virtual ranks.
//
//   1. Every rank copies its send buffer into its row of a node-shared,
//      GPU-pinned array (POSIX shared memory, created at MPI_Init by rank 0
//      and grown collectively when a call needs more).
//   2. Rank 0 runs the collective through the C ABI (one copy in, the
//      device call, one copy out).
//   3. Every rank copies its row of the result back.
//
// Two barriers order the steps.  MPI_Allreduce overlaps them instead: the
// ranks publish how many columns of their rows they have deposited, rank 0
// runs bine_allreduce_host_hooked, whose column windows start as soon as
// every row holds them, publishes how many output columns have reached host
// memory, and the ranks collect behind it.  Algorithm selection reads the reference's
// own environment variables (LIBBINE_<COLL>_ALGO, _ALGO_FAMILY, _DISTANCE,
// LIBBINE_NUM_PORTS, LIBBINE_DIMENSIONS, LIBBINE_SEGMENT_SIZE;
// lib/libbine.cc:75-575); BINE_B200_ENGINE=fused|steps|pipelined and
// BINE_B200_FLOAT_ORDER=reference|fast pick the engine.  Calls the engine
// cannot take (another communicator, another op or datatype, uneven
// reduce_scatter counts, mismatched send/recv types) go to the PMPI_
// implementation unchanged, as the reference sends them there.
#include <mpi.h>

#include <cuda_runtime.h>
#include <fcntl.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sched.h>
#include <sys/mman.h>
#include <time.h>
#include <unistd.h>

#include <algorithm>
#include <string>
#include <vector>

#include "../../include/bine_b200.h"

namespace {

struct Header {  // written by rank 0 between the two barriers
    int rc;
    char msg[252];
};
constexpr size_t kHeader = 256;

// Control words of the overlapped allreduce, after the header, one cache
// line each: [0] output columns in host memory (rank 0), [1] the call rank
// 0 abandoned, [2 + r] input columns rank r has deposited.  Words pack
// (call sequence & 0xffffff) << 40 | columns.
constexpr size_t kLine = 64;
size_t ctl_bytes(int P) { return ((size_t)(2 + P) * kLine + 4095) / 4096 * 4096; }
constexpr int kSeqShift = 40;
constexpr uint64_t kColMask = (1ull << kSeqShift) - 1;

struct State {
    int rank = -1, size = 0;
    char* shm = nullptr;  // Header, then the input rows, then the output rows
    size_t shm_bytes = 0;
    int generation = 0;
    bool pinned = false;
    uint64_t seq = 0;            // overlapped allreduce calls so far (the same on every rank)
    bine_comm_t comm = nullptr;  // rank 0 only
    char* dev = nullptr;         // rank 0: device rows (input, then output)
    size_t dev_bytes = 0;
};
State g;

const char* env(const char* name) {
    const char* v = getenv(name);
    return v && *v ? v : nullptr;
}

// Datatype of the engine, or -1.
int engine_dtype(MPI_Datatype dt) {
    int size = 0;
    PMPI_Type_size(dt, &size);
    if (dt == MPI_INT32_T || (dt == MPI_INT && size == 4)) return BINE_INT32;
    if (dt == MPI_INT64_T || (dt == MPI_LONG && size == 8)) return BINE_INT64;
    if (dt == MPI_FLOAT) return BINE_FLOAT;
    if (dt == MPI_DOUBLE) return BINE_DOUBLE;
    if (dt == MPI_CHAR) return BINE_CHAR;
    return -1;
}

// Copy collectives move bytes: any datatype of a known size travels as CHAR.
int copy_dtype(MPI_Datatype dt, int* es) {
    *es = 0;
    PMPI_Type_size(dt, es);
    const int t = engine_dtype(dt);
    if (t >= 0) return t;
    return *es > 0 ? BINE_CHAR : -1;
}

const char* kCollEnv[] = {"ALLREDUCE", "REDUCE_SCATTER", "ALLGATHER", "BCAST",
                          "REDUCE",    "ALLTOALL",       "SCATTER",   "GATHER"};

// The variant names of LIBBINE_<COLL>_ALGO (lib/libbine_common.h:74-123).
int variant_of(int coll, const char* name) {
    struct V {
        int coll;
        const char* name;
        int id;
    };
    static const V table[] = {
        {BINE_COLL_ALLREDUCE, "L", BINE_ALLREDUCE_L},
        {BINE_COLL_ALLREDUCE, "B", BINE_ALLREDUCE_B},
        {BINE_COLL_ALLREDUCE, "B_CONT", BINE_ALLREDUCE_B_CONT},
        {BINE_COLL_ALLREDUCE, "B_COALESCE", BINE_ALLREDUCE_B_COALESCE},
        {BINE_COLL_REDUCE_SCATTER, "VEC_HALVING_CONT_PERMUTE", BINE_REDUCE_SCATTER_CONT_PERMUTE},
        {BINE_COLL_ALLGATHER, "VEC_DOUBLING_CONT_PERMUTE", 0},
        {BINE_COLL_ALLGATHER, "VEC_DOUBLING_CONT_SEND", 1},
        {BINE_COLL_ALLGATHER, "VEC_DOUBLING_BLOCKS", 2},
        {BINE_COLL_BCAST, "BINOMIAL_TREE", BINE_BCAST_BINOMIAL_TREE},
        {BINE_COLL_BCAST, "SCATTER_ALLGATHER", BINE_BCAST_SCATTER_ALLGATHER},
        {BINE_COLL_REDUCE, "BINOMIAL_TREE", BINE_REDUCE_BINOMIAL_TREE},
        {BINE_COLL_REDUCE, "REDUCE_SCATTER_GATHER", BINE_REDUCE_SCATTER_GATHER},
        {BINE_COLL_ALLTOALL, "LOG", BINE_ALLTOALL_LOG},
        {BINE_COLL_SCATTER, "BINOMIAL_TREE_CONT_PERMUTE", BINE_SCATTER_BINOMIAL_TREE},
        {BINE_COLL_GATHER, "BINOMIAL_TREE_CONT_PERMUTE", BINE_GATHER_BINOMIAL_TREE},
    };
    for (const V& v : table)
        if (v.coll == coll && strcmp(v.name, name) == 0) return v.id;
    return -1;
}

void set_float_order_from_env() {
    const char* o = env("BINE_B200_FLOAT_ORDER");
    bine_comm_set_float_order(g.comm, o && strcmp(o, "fast") == 0 ? BINE_ORDER_FAST : BINE_ORDER_REFERENCE);
}

// Rank 0: the communicator, configured from the environment.
int make_comm() {
    if (g.comm) return BINE_SUCCESS;
    int dims[3] = {0, 0, 0}, nd = 0;
    if (const char* d = env("LIBBINE_DIMENSIONS")) {
        std::string s(d);
        size_t pos = 0;
        while (nd < 3 && pos < s.size()) {
            dims[nd++] = atoi(s.c_str() + pos);
            const size_t x = s.find('x', pos);
            if (x == std::string::npos) break;
            pos = x + 1;
        }
    }
    int rc = bine_comm_create(g.size, nd, nd ? dims : nullptr, &g.comm);
    if (rc) return rc;
    if (const char* p = env("LIBBINE_NUM_PORTS")) {
        rc = bine_comm_set_ports(g.comm, atoi(p));
        if (rc) return rc;
    }
    if (const char* s = env("LIBBINE_SEGMENT_SIZE")) bine_comm_set_segment(g.comm, atoll(s));
    const char* e = env("BINE_B200_ENGINE");
    bine_comm_set_engine(g.comm, !e ? BINE_ENGINE_FUSED
                                    : strcmp(e, "steps") == 0     ? BINE_ENGINE_STEPS
                                    : strcmp(e, "pipelined") == 0 ? BINE_ENGINE_PIPELINED
                                                                  : BINE_ENGINE_FUSED);
    set_float_order_from_env();
    for (int c = 0; c < 8; c++) {
        char key[64];
        snprintf(key, sizeof key, "LIBBINE_%s_ALGO", kCollEnv[c]);
        const char* name = env(key);
        if (!name) continue;
        const int variant = variant_of(c, name);
        if (variant < 0) continue;  // a name of the reference's other layers: keep the default
        snprintf(key, sizeof key, "LIBBINE_%s_ALGO_FAMILY", kCollEnv[c]);
        const char* fam = env(key);
        const int family = !fam ? BINE_FAMILY_BINE
                           : strcmp(fam, "RECDOUB") == 0 ? BINE_FAMILY_RECDOUB
                           : strcmp(fam, "BRUCK") == 0 && c == BINE_COLL_ALLTOALL ? BINE_FAMILY_BRUCK
                                                                                 : BINE_FAMILY_BINE;
        snprintf(key, sizeof key, "LIBBINE_%s_DISTANCE", kCollEnv[c]);
        const char* dist = env(key);
        const int distance = !dist ? BINE_DISTANCE_DEFAULT
                                   : (strcmp(dist, "DECREASING") == 0 ? BINE_DISTANCE_DECREASING
                                                                      : BINE_DISTANCE_INCREASING);
        rc = bine_comm_set_algo(g.comm, (bine_coll_t)c, variant, family, distance);
        if (rc) return rc;
    }
    return BINE_SUCCESS;
}

// Collective over MPI_COMM_WORLD: every rank asks for the same size.
int ensure_shm(size_t need) {
    need += kHeader + ctl_bytes(g.size);
    if (g.shm && g.shm_bytes >= need) return MPI_SUCCESS;
    const size_t page = (size_t)sysconf(_SC_PAGESIZE);
    size_t bytes = std::max<size_t>({need, 2 * g.shm_bytes, (size_t)64 << 20});
    bytes = (bytes + page - 1) / page * page;
    char name[64] = {0};
    int fd = -1;
    if (g.rank == 0) {
        snprintf(name, sizeof name, "/bine_mpi_%d_%d", (int)getpid(), ++g.generation);
        fd = shm_open(name, O_CREAT | O_EXCL | O_RDWR, 0600);
        if (fd >= 0 && ftruncate(fd, (off_t)bytes) != 0) {
            close(fd);
            shm_unlink(name);
            fd = -1;
        }
        if (fd < 0) name[0] = 0;
    }
    PMPI_Bcast(name, (int)sizeof name, MPI_CHAR, 0, MPI_COMM_WORLD);
    if (!name[0]) return MPI_ERR_OTHER;
    if (g.rank != 0) fd = shm_open(name, O_RDWR, 0600);
    char* p = fd < 0 ? nullptr : (char*)mmap(nullptr, bytes, PROT_READ | PROT_WRITE, MAP_SHARED, fd, 0);
    if (fd >= 0) close(fd);
    const bool ok = p && p != (char*)MAP_FAILED;
    int failed = ok ? 0 : 1, failures = 0;
    PMPI_Allreduce(&failed, &failures, 1, MPI_INT, MPI_SUM, MPI_COMM_WORLD);
    if (g.rank == 0) shm_unlink(name);  // every rank has it mapped, or the call failed
    if (failures) {
        if (ok) munmap(p, bytes);
        return MPI_ERR_OTHER;
    }
    if (g.shm) {
        if (g.pinned) cudaHostUnregister(g.shm);
        munmap(g.shm, g.shm_bytes);
    }
    g.shm = p;
    g.shm_bytes = bytes;
    // Rank 0 pins the mapping so the GPU copies it at full bandwidth;
    // pageable copies still work if pinning fails.
    g.pinned = g.rank == 0 && cudaHostRegister(g.shm, bytes, cudaHostRegisterDefault) == cudaSuccess;
    if (g.rank == 0 && !g.pinned) cudaGetLastError();
    return MPI_SUCCESS;
}

Header* header() { return reinterpret_cast<Header*>(g.shm); }
char* in_rows() { return g.shm + kHeader + ctl_bytes(g.size); }
uint64_t* ctl_word(int i) { return reinterpret_cast<uint64_t*>(g.shm + kHeader + (size_t)i * kLine); }
uint64_t pack(uint64_t seq, long long cols) { return ((seq & 0xffffff) << kSeqShift) | (uint64_t)cols; }
uint64_t load(int i) { return __atomic_load_n(ctl_word(i), __ATOMIC_ACQUIRE); }
void publish(int i, uint64_t v) { __atomic_store_n(ctl_word(i), v, __ATOMIC_RELEASE); }

// Columns of call `seq` a progress word reports (-1: another call's word).
long long columns(uint64_t v, uint64_t seq) {
    return (v >> kSeqShift) == (seq & 0xffffff) ? (long long)(v & kColMask) : -1;
}

// Waits until `ready()` holds; false if rank 0 abandoned call `seq` or two
// minutes pass (a rank that died).  Spins briefly, then sleeps 20 us at a
// time so that waiting ranks leave the cores to the ranks still copying.
template <typename Ready>
bool wait_until(Ready ready, uint64_t seq) {
    timespec t0, t;
    clock_gettime(CLOCK_MONOTONIC, &t0);
    for (long spin = 0;; spin++) {
        if (ready()) return true;
        if (columns(load(1), seq) >= 0) return false;
        if (spin < 256) continue;
        const timespec nap = {0, 20000};
        nanosleep(&nap, nullptr);
        clock_gettime(CLOCK_MONOTONIC, &t);
        if (t.tv_sec - t0.tv_sec > 120) return false;
    }
}

int ensure_dev(size_t bytes) {
    if (g.dev_bytes >= bytes) return BINE_SUCCESS;
    cudaFree(g.dev);
    g.dev = nullptr;
    g.dev_bytes = 0;
    if (cudaMalloc(&g.dev, bytes) != cudaSuccess) return BINE_ERR_NOMEM;
    g.dev_bytes = bytes;
    return BINE_SUCCESS;
}

// Rank 0: runs one collective other than allreduce over the shared rows.
// `in_row`/`out_row` are the per-rank row bytes; the output rows follow the
// input rows (bcast is in place: its result lands in the input rows).
int leader_run(int coll, int count, int dt, int root, size_t in_row, size_t out_row) {
    int rc = make_comm();
    if (rc) return rc;
    const size_t P = (size_t)g.size;
    char* hin = in_rows();
    char* hout = hin + P * in_row;
    bine_comm_set_layout(g.comm, 0, 0);
    for (int attempt = 0; attempt < 2; attempt++) {
        rc = ensure_dev(P * (in_row + out_row));
        if (rc) return rc;
        char* din = g.dev;
        char* dout = g.dev + P * in_row;
        if (cudaMemcpy(din, hin, P * in_row, cudaMemcpyHostToDevice) != cudaSuccess) return BINE_ERR_CUDA;
        const bine_datatype_t t = (bine_datatype_t)dt;
        std::vector<int> counts;
        switch (coll) {
        case BINE_COLL_REDUCE_SCATTER:
            counts.assign(P, count);
            rc = bine_reduce_scatter(din, dout, counts.data(), t, BINE_SUM, g.comm);
            break;
        case BINE_COLL_ALLGATHER: rc = bine_allgather(din, count, t, dout, count, t, g.comm); break;
        case BINE_COLL_BCAST:
            rc = bine_bcast(din, count, t, root, g.comm);
            dout = din;
            break;
        case BINE_COLL_REDUCE: rc = bine_reduce(din, dout, count, t, BINE_SUM, root, g.comm); break;
        case BINE_COLL_ALLTOALL: rc = bine_alltoall(din, count, t, dout, count, t, g.comm); break;
        case BINE_COLL_SCATTER: rc = bine_scatter(din, count, t, dout, count, t, root, g.comm); break;
        case BINE_COLL_GATHER: rc = bine_gather(din, count, t, dout, count, t, root, g.comm); break;
        default: rc = BINE_ERR_ARG;
        }
        if (rc == BINE_SUCCESS) rc = bine_comm_synchronize(g.comm);
        char* hdst = coll == BINE_COLL_BCAST ? hin : hout;
        const size_t nbytes = P * (coll == BINE_COLL_BCAST ? in_row : out_row);
        if (rc == BINE_SUCCESS && cudaMemcpy(hdst, dout, nbytes, cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = BINE_ERR_CUDA;
        // A float sum whose reference order does not exist for this case
        // (the reference fails there) is computed in the FAST order.
        if (rc == BINE_ERR_UNSUPPORTED && attempt == 0 && (dt == BINE_FLOAT || dt == BINE_DOUBLE)) {
            bine_comm_set_float_order(g.comm, BINE_ORDER_FAST);
            continue;
        }
        break;
    }
    set_float_order_from_env();
    return rc;
}

// MPI_Allreduce with the three phases overlapped.  Every rank deposits its
// row in chunks and publishes its progress; rank 0 runs the host pipeline,
// whose before-window hook deposits rank 0's own columns and waits for every
// row's, and whose after-window hook collects rank 0's columns and
// publishes the output progress; the other ranks collect behind it.  A
// rank's next call can only reuse the rows after every rank finished
// collecting this one: rank 0 reads a window only once every rank has
// deposited it for the next call.
struct Overlap {
    uint64_t seq;
    int P;
    size_t es, row;  // element and row bytes
    const char* src;
    char* dst;
    long long deposited = 0;  // rank 0's own columns in its row
};

int before_window(void* u, long long first, long long n) {
    Overlap& o = *static_cast<Overlap*>(u);
    const long long end = first + n;
    if (end > o.deposited) {
        memcpy(in_rows() + o.deposited * o.es, o.src + o.deposited * o.es, (size_t)(end - o.deposited) * o.es);
        o.deposited = end;
    }
    for (int r = 1; r < o.P; r++)
        if (!wait_until([&] { return columns(load(2 + r), o.seq) >= end; }, o.seq)) return 1;
    return 0;
}

int after_window(void* u, long long first, long long n) {
    Overlap& o = *static_cast<Overlap*>(u);
    memcpy(o.dst + first * o.es, in_rows() + (size_t)o.P * o.row + first * o.es, (size_t)n * o.es);
    publish(0, pack(o.seq, first + n));
    return 0;
}

int allreduce_overlapped(int count, int dt, size_t es, const void* src, void* dst) {
    const size_t P = (size_t)g.size, row = (size_t)count * es;
    int rc = ensure_shm(2 * P * row);
    if (rc != MPI_SUCCESS) return rc;
    do {
        ++g.seq;
    } while ((g.seq & 0xffffff) == 0);  // a never-written (zero) word must not match
    const uint64_t seq = g.seq;
    if (g.rank != 0) {
        // Deposit in chunks of 256 KiB, then collect behind rank 0.
        char* mine = in_rows() + (size_t)g.rank * row;
        const long long chunk = std::max<long long>(1, (256 << 10) / (long long)es);
        for (long long c0 = 0; c0 < count; c0 += chunk) {
            const long long c1 = std::min<long long>(count, c0 + chunk);
            memcpy(mine + c0 * es, (const char*)src + c0 * es, (size_t)(c1 - c0) * es);
            publish(2 + g.rank, pack(seq, c1));
        }
        if (count == 0) publish(2 + g.rank, pack(seq, 0));
        const char* out = in_rows() + P * row + (size_t)g.rank * row;
        long long have = 0;
        while (have < count) {
            long long done = -1;
            if (!wait_until([&] { return (done = columns(load(0), seq)) > have; }, seq)) break;
            memcpy((char*)dst + have * es, out + have * es, (size_t)(done - have) * es);
            have = done;
        }
        if (have == count) return MPI_SUCCESS;
        if (columns(load(1), seq) < 0) fprintf(stderr, "bine_mpi: rank %d: rank 0 stopped answering\n", g.rank);
        return MPI_ERR_OTHER;
    }
    Overlap o{seq, (int)P, es, row, (const char*)src, (char*)dst};
    rc = make_comm();
    if (rc == BINE_SUCCESS) {
        bine_comm_set_layout(g.comm, 0, 0);
        char* hin = in_rows();
        rc = bine_allreduce_host_hooked(hin, hin + P * row, count, (bine_datatype_t)dt, BINE_SUM, g.comm,
                                        before_window, after_window, &o);
        // A float sum whose reference order does not exist for this case
        // (the reference fails there) is computed in the FAST order.
        if (rc == BINE_ERR_UNSUPPORTED && (dt == BINE_FLOAT || dt == BINE_DOUBLE)) {
            bine_comm_set_float_order(g.comm, BINE_ORDER_FAST);
            rc = bine_allreduce_host_hooked(hin, hin + P * row, count, (bine_datatype_t)dt, BINE_SUM, g.comm,
                                            before_window, after_window, &o);
        }
        set_float_order_from_env();
    }
    if (rc != BINE_SUCCESS) {
        fprintf(stderr, "bine_mpi: %s\n", bine_last_error_string());
        publish(1, pack(seq, 0));  // the other ranks stop waiting
        return MPI_ERR_OTHER;
    }
    return MPI_SUCCESS;
}

// The three phases every rank runs: deposit its input row, rank 0
// computes, collect its output row.
template <typename Deposit, typename Collect>
int run_shared(int coll, int count, int dt, int root, size_t in_row, size_t out_row, Deposit deposit,
               Collect collect) {
    const size_t P = (size_t)g.size;
    int rc = ensure_shm(P * (in_row + out_row));
    if (rc != MPI_SUCCESS) return rc;
    deposit(in_rows() + (size_t)g.rank * in_row);
    PMPI_Barrier(MPI_COMM_WORLD);
    if (g.rank == 0) {
        const int r = leader_run(coll, count, dt, root, in_row, out_row);
        header()->rc = r;
        snprintf(header()->msg, sizeof header()->msg, "%s", r ? bine_last_error_string() : "");
    }
    PMPI_Barrier(MPI_COMM_WORLD);
    if (header()->rc != BINE_SUCCESS) {
        if (g.rank == 0) fprintf(stderr, "bine_mpi: %s\n", header()->msg);
        return MPI_ERR_OTHER;
    }
    collect(in_rows() + P * in_row + (size_t)g.rank * out_row);
    return MPI_SUCCESS;
}

bool world(MPI_Comm comm) { return comm == MPI_COMM_WORLD && g.size > 0; }

}  // namespace

extern "C" {

int MPI_Init(int* argc, char*** argv) {
    const int rc = PMPI_Init(argc, argv);
    if (rc != MPI_SUCCESS) return rc;
    PMPI_Comm_rank(MPI_COMM_WORLD, &g.rank);
    PMPI_Comm_size(MPI_COMM_WORLD, &g.size);
    return ensure_shm(0);
}

int MPI_Finalize(void) {
    if (g.rank == 0) {
        if (g.comm) bine_comm_destroy(g.comm);
        cudaFree(g.dev);
        if (g.pinned) cudaHostUnregister(g.shm);
    }
    if (g.shm) munmap(g.shm, g.shm_bytes);
    g = State();
    return PMPI_Finalize();
}

// MPI_Allreduce, lib/libbine.cc:1012.
int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype dt, MPI_Op op, MPI_Comm comm) {
    const int t = engine_dtype(dt);
    if (!world(comm) || op != MPI_SUM || t < 0 || count < 0)
        return PMPI_Allreduce(sendbuf, recvbuf, count, dt, op, comm);
    int es = 0;
    PMPI_Type_size(dt, &es);
    const void* src = sendbuf == MPI_IN_PLACE ? recvbuf : sendbuf;
    return allreduce_overlapped(count, t, (size_t)es, src, recvbuf);
}

// MPI_Reduce_scatter, lib/libbine.cc:1064 (equal counts, as the reference
// assumes).
int MPI_Reduce_scatter(const void* sendbuf, void* recvbuf, const int recvcounts[], MPI_Datatype dt, MPI_Op op,
                       MPI_Comm comm) {
    const int t = engine_dtype(dt);
    bool even = world(comm) && recvcounts != nullptr;
    for (int r = 1; even && r < g.size; r++) even = recvcounts[r] == recvcounts[0];
    if (!even || op != MPI_SUM || t < 0 || sendbuf == MPI_IN_PLACE)
        return PMPI_Reduce_scatter(sendbuf, recvbuf, recvcounts, dt, op, comm);
    int es = 0;
    PMPI_Type_size(dt, &es);
    const int count = recvcounts[0];
    const size_t out_row = (size_t)count * es, in_row = out_row * g.size;
    return run_shared(BINE_COLL_REDUCE_SCATTER, count, t, 0, in_row, out_row,
                      [&](char* d) { memcpy(d, sendbuf, in_row); },
                      [&](const char* s) { memcpy(recvbuf, s, out_row); });
}

// MPI_Allgather, lib/libbine.cc:1168.
int MPI_Allgather(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf, int recvcount,
                  MPI_Datatype recvtype, MPI_Comm comm) {
    int es = 0;
    const int t = copy_dtype(recvtype, &es);
    const bool in_place = sendbuf == MPI_IN_PLACE;
    if (!world(comm) || t < 0 || (!in_place && (sendtype != recvtype || sendcount != recvcount)))
        return PMPI_Allgather(sendbuf, sendcount, sendtype, recvbuf, recvcount, recvtype, comm);
    const int count = engine_dtype(recvtype) < 0 ? recvcount * es : recvcount;
    const size_t in_row = (size_t)recvcount * es, out_row = in_row * g.size;
    const char* src = in_place ? (const char*)recvbuf + (size_t)g.rank * in_row : (const char*)sendbuf;
    return run_shared(BINE_COLL_ALLGATHER, count, t, 0, in_row, out_row, [&](char* d) { memcpy(d, src, in_row); },
                      [&](const char* s) { memcpy(recvbuf, s, out_row); });
}

// MPI_Bcast_f, lib/libbine.cc:1252.  The reference interposes its broadcast
// under this name only and leaves MPI_Bcast to the MPI library
// (bench/bench.cc:20, 136), so a program's own setup broadcasts stay on MPI;
// this layer exports no MPI_Bcast either.
int MPI_Bcast_f(void* buf, int count, MPI_Datatype dt, int root, MPI_Comm comm) {
    int es = 0;
    const int t = copy_dtype(dt, &es);
    if (!world(comm) || t < 0 || root < 0 || root >= g.size) return PMPI_Bcast(buf, count, dt, root, comm);
    const int n = engine_dtype(dt) < 0 ? count * es : count;
    const size_t row = (size_t)count * es;
    return run_shared(BINE_COLL_BCAST, n, t, root, row, 0,
                      [&](char* d) {
                          if (g.rank == root) memcpy(d, buf, row);
                      },
                      [&](const char*) { memcpy(buf, in_rows() + (size_t)g.rank * row, row); });
}

// MPI_Alltoall, lib/libbine.cc:1291.
int MPI_Alltoall(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf, int recvcount,
                 MPI_Datatype recvtype, MPI_Comm comm) {
    int es = 0;
    const int t = copy_dtype(recvtype, &es);
    if (!world(comm) || t < 0 || sendbuf == MPI_IN_PLACE || sendtype != recvtype || sendcount != recvcount)
        return PMPI_Alltoall(sendbuf, sendcount, sendtype, recvbuf, recvcount, recvtype, comm);
    const int count = engine_dtype(recvtype) < 0 ? recvcount * es : recvcount;
    const size_t row = (size_t)recvcount * es * g.size;
    return run_shared(BINE_COLL_ALLTOALL, count, t, 0, row, row, [&](char* d) { memcpy(d, sendbuf, row); },
                      [&](const char* s) { memcpy(recvbuf, s, row); });
}

// MPI_Scatter, lib/libbine.cc:1312.
int MPI_Scatter(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf, int recvcount,
                MPI_Datatype recvtype, int root, MPI_Comm comm) {
    int es = 0;
    const int t = copy_dtype(recvtype, &es);
    if (!world(comm) || t < 0 || root < 0 || root >= g.size || recvbuf == MPI_IN_PLACE ||
        (g.rank == root && (sendtype != recvtype || sendcount != recvcount)))
        return PMPI_Scatter(sendbuf, sendcount, sendtype, recvbuf, recvcount, recvtype, root, comm);
    const int count = engine_dtype(recvtype) < 0 ? recvcount * es : recvcount;
    const size_t out_row = (size_t)recvcount * es, in_row = out_row * g.size;
    return run_shared(BINE_COLL_SCATTER, count, t, root, in_row, out_row,
                      [&](char* d) {
                          if (g.rank == root) memcpy(d, sendbuf, in_row);
                      },
                      [&](const char* s) { memcpy(recvbuf, s, out_row); });
}

// MPI_Gather, lib/libbine.cc:1376.
int MPI_Gather(const void* sendbuf, int sendcount, MPI_Datatype sendtype, void* recvbuf, int recvcount,
               MPI_Datatype recvtype, int root, MPI_Comm comm) {
    int es = 0;
    const int t = copy_dtype(sendtype, &es);
    if (!world(comm) || t < 0 || root < 0 || root >= g.size || sendbuf == MPI_IN_PLACE ||
        (g.rank == root && (sendtype != recvtype || sendcount != recvcount)))
        return PMPI_Gather(sendbuf, sendcount, sendtype, recvbuf, recvcount, recvtype, root, comm);
    const int count = engine_dtype(sendtype) < 0 ? sendcount * es : sendcount;
    const size_t in_row = (size_t)sendcount * es, out_row = in_row * g.size;
    return run_shared(BINE_COLL_GATHER, count, t, root, in_row, out_row, [&](char* d) { memcpy(d, sendbuf, in_row); },
                      [&](const char* s) {
                          if (g.rank == root) memcpy(recvbuf, s, out_row);
                      });
}

// MPI_Reduce, lib/libbine.cc:1440.
int MPI_Reduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype dt, MPI_Op op, int root, MPI_Comm comm) {
    const int t = engine_dtype(dt);
    if (!world(comm) || op != MPI_SUM || t < 0 || root < 0 || root >= g.size || count < 0)
        return PMPI_Reduce(sendbuf, recvbuf, count, dt, op, root, comm);
    int es = 0;
    PMPI_Type_size(dt, &es);
    const size_t row = (size_t)count * es;
    const void* src = sendbuf == MPI_IN_PLACE ? recvbuf : sendbuf;
    return run_shared(BINE_COLL_REDUCE, count, t, root, row, row, [&](char* d) { memcpy(d, src, row); },
                      [&](const char* s) {
                          if (g.rank == root) memcpy(recvbuf, s, row);
                      });
}

}  // extern "C"

// Oracle harness for the reference library (test infrastructure only).
//
// Runs ONE collective of the unmodified reference (lib/libbine.cc entry
// points, linked against oracle/mpishim) over P forked ranks on this host's
// cores, the way bench/bench.cc does under mpirun, and writes:
//   * every rank's result buffer (--out), for bit-exact parity checks;
//   * optionally the message trace of the first call (--trace): one record
//     {src, dst, tag, call, bytes} per point-to-point send;
//   * a JSON line on stdout with per-rank status and, with --iters, timings
//     taken as bench.cc takes them (two barriers, wall time around one call,
//     max over ranks per iteration; bench/bench.cc:289-318, 376-387).
//
// Inputs come from --in (P consecutive per-rank send buffers, raw bytes) or
// are generated in place with --gen (timing runs only).  Per-rank buffer
// sizes follow bench/bench.cc:178-207.  Algorithm selection is left to the
// reference's own LIBBINE_* environment variables, which the children
// inherit.
#include <mpi.h>

#include <errno.h>
#include <signal.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/wait.h>
#include <time.h>
#include <unistd.h>

#include <algorithm>
#include <string>
#include <vector>

namespace {

struct Args {
    std::string coll = "allreduce";
    std::string dtype = "int32";
    long count = 0;
    int P = 0;
    int root = 0;
    int iters = 0;
    int warmup = 0;
    std::string in, out, trace;
    std::string gen;
    uint64_t seed = 1;
    double timeout = 600.0;
    long arena_mb = 0;
};

MPI_Datatype dtype_of(const std::string& s) {
    if (s == "int32") return MPI_INT32_T;
    if (s == "int") return MPI_INT;
    if (s == "int64") return MPI_INT64_T;
    if (s == "float") return MPI_FLOAT;
    if (s == "double") return MPI_DOUBLE;
    if (s == "char") return MPI_CHAR;
    return MPI_DATATYPE_NULL;
}

// Per-rank send/recv element counts, as bench/bench.cc:178-207 allocates them.
void buffer_counts(const std::string& coll, long c, int P, long* sc, long* rc) {
    if (coll == "allreduce" || coll == "bcast" || coll == "reduce") {
        *sc = c;
        *rc = c;
    } else if (coll == "reduce_scatter" || coll == "scatter") {
        *sc = c * P;
        *rc = c;
    } else if (coll == "allgather" || coll == "gather") {
        *sc = c;
        *rc = c * P;
    } else if (coll == "alltoall") {
        *sc = c * P;
        *rc = c * P;
    } else {
        *sc = *rc = -1;
    }
}

uint64_t splitmix64(uint64_t* s) {
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Timing-run input: uniform integers in [-1000, 1000] (int types) or in
// [-1, 1) (float types), one splitmix64 stream per rank.
void generate(char* buf, long n, MPI_Datatype dt, uint64_t seed, int rank) {
    uint64_t s = seed ^ (0xD1B54A32D192ED03ull * (uint64_t)(rank + 1));
    for (long i = 0; i < n; i++) {
        uint64_t r = splitmix64(&s);
        long v = (long)(r % 2001) - 1000;
        double f = (double)(r >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
        if (dt == MPI_INT32_T || dt == MPI_INT) ((int32_t*)buf)[i] = (int32_t)v;
        else if (dt == MPI_INT64_T) ((int64_t*)buf)[i] = v;
        else if (dt == MPI_FLOAT) ((float*)buf)[i] = (float)f;
        else if (dt == MPI_DOUBLE) ((double*)buf)[i] = f;
        else if (dt == MPI_CHAR) ((signed char*)buf)[i] = (signed char)(v & 0x7f);
    }
}

int run_one(const Args& a, MPI_Datatype dt, const char* sendbuf, char* recvbuf, long count, int P) {
    const std::string& c = a.coll;
    if (c == "allreduce") return MPI_Allreduce(sendbuf, recvbuf, (int)count, dt, MPI_SUM, MPI_COMM_WORLD);
    if (c == "reduce_scatter") {
        std::vector<int> rc(P, (int)count);
        return MPI_Reduce_scatter(sendbuf, recvbuf, rc.data(), dt, MPI_SUM, MPI_COMM_WORLD);
    }
    if (c == "allgather") return MPI_Allgather(sendbuf, (int)count, dt, recvbuf, (int)count, dt, MPI_COMM_WORLD);
    if (c == "bcast") return MPI_Bcast_f(recvbuf, (int)count, dt, a.root, MPI_COMM_WORLD);
    if (c == "alltoall") return MPI_Alltoall(sendbuf, (int)count, dt, recvbuf, (int)count, dt, MPI_COMM_WORLD);
    if (c == "scatter") return MPI_Scatter(sendbuf, (int)count, dt, recvbuf, (int)count, dt, a.root, MPI_COMM_WORLD);
    if (c == "gather") return MPI_Gather(sendbuf, (int)count, dt, recvbuf, (int)count, dt, a.root, MPI_COMM_WORLD);
    if (c == "reduce") return MPI_Reduce(sendbuf, recvbuf, (int)count, dt, MPI_SUM, a.root, MPI_COMM_WORLD);
    return MPI_ERR_ARG;
}

void usage() {
    fprintf(stderr,
            "usage: bine_ref_run --coll C --dtype T --count N --P P [--root R] [--in FILE | --gen uniform --seed S]\n"
            "                    [--out FILE] [--trace FILE] [--iters K --warmup W] [--timeout SEC] [--arena-mb MB]\n");
}

}  // namespace

int main(int argc, char** argv) {
    Args a;
    for (int i = 1; i < argc; i++) {
        std::string k = argv[i];
        auto val = [&]() -> const char* {
            if (i + 1 >= argc) {
                usage();
                exit(2);
            }
            return argv[++i];
        };
        if (k == "--coll") a.coll = val();
        else if (k == "--dtype") a.dtype = val();
        else if (k == "--count") a.count = atol(val());
        else if (k == "--P") a.P = atoi(val());
        else if (k == "--root") a.root = atoi(val());
        else if (k == "--iters") a.iters = atoi(val());
        else if (k == "--warmup") a.warmup = atoi(val());
        else if (k == "--in") a.in = val();
        else if (k == "--out") a.out = val();
        else if (k == "--trace") a.trace = val();
        else if (k == "--gen") a.gen = val();
        else if (k == "--seed") a.seed = strtoull(val(), nullptr, 10);
        else if (k == "--timeout") a.timeout = atof(val());
        else if (k == "--arena-mb") a.arena_mb = atol(val());
        else {
            usage();
            return 2;
        }
    }
    MPI_Datatype dt = dtype_of(a.dtype);
    long sc, rc;
    buffer_counts(a.coll, a.count, a.P, &sc, &rc);
    if (a.P <= 0 || a.count < 0 || dt == MPI_DATATYPE_NULL || sc < 0) {
        usage();
        return 2;
    }
    int es;
    MPI_Type_size(dt, &es);
    const size_t send_bytes = (size_t)sc * es, recv_bytes = (size_t)rc * es;

    size_t arena = a.arena_mb > 0 ? (size_t)a.arena_mb << 20
                                  : std::max<size_t>((size_t)64 << 20, 4 * (send_bytes + recv_bytes) + (1 << 20));
    const size_t trace_cap = a.trace.empty() ? 0 : (size_t)1 << 16;
    if (shim_setup(a.P, arena, trace_cap, a.timeout) != 0) return 3;

    // Shared input, output, status and timing arrays.
    char* in = (char*)shim_shared_alloc(send_bytes * a.P);
    char* out = (char*)shim_shared_alloc(recv_bytes * a.P);
    int* rcodes = (int*)shim_shared_alloc(sizeof(int) * a.P);
    const int nt = a.iters > 0 ? a.iters : 1;
    double* times = (double*)shim_shared_alloc(sizeof(double) * (size_t)a.P * nt);
    if (!in || !out || !rcodes || !times) return 3;
    if (!a.in.empty()) {
        FILE* f = fopen(a.in.c_str(), "rb");
        if (!f || fread(in, 1, send_bytes * a.P, f) != send_bytes * a.P) {
            fprintf(stderr, "bine_ref_run: cannot read %zu bytes from %s\n", send_bytes * a.P, a.in.c_str());
            return 3;
        }
        fclose(f);
    }
    for (int r = 0; r < a.P; r++) rcodes[r] = -1;

    std::vector<pid_t> pids(a.P, -1);
    for (int r = 0; r < a.P; r++) {
        pid_t pid = fork();
        if (pid < 0) {
            perror("fork");
            shim_abort_all();
            return 3;
        }
        if (pid == 0) {
            shim_set_rank(r);
            MPI_Init(&argc, &argv);
            char* sendbuf = (char*)malloc(send_bytes ? send_bytes : 1);
            char* recvbuf = (char*)malloc(recv_bytes ? recv_bytes : 1);
            char* mine = in + send_bytes * r;
            if (a.in.empty()) generate(mine, sc, dt, a.seed, r);
            memcpy(sendbuf, mine, send_bytes);
            memset(recvbuf, 0, recv_bytes);
            // Bcast is in place: the root's buffer holds the data, the others'
            // start zeroed (bench/bench.cc:213-220, 271-277).
            if (a.coll == "bcast" && r == a.root) memcpy(recvbuf, sendbuf, send_bytes);
            shim_trace_next_call();
            int res = run_one(a, dt, sendbuf, recvbuf, a.count, a.P);
            memcpy(out + recv_bytes * r, recvbuf, recv_bytes);
            for (int it = -a.warmup; it < a.iters && res == MPI_SUCCESS; it++) {
                if (a.coll == "bcast" && r == a.root) memcpy(recvbuf, sendbuf, send_bytes);
                MPI_Barrier(MPI_COMM_WORLD);
                MPI_Barrier(MPI_COMM_WORLD);
                double t0 = MPI_Wtime();
                res = run_one(a, dt, sendbuf, recvbuf, a.count, a.P);
                double t1 = MPI_Wtime();
                if (it >= 0) times[(size_t)r * nt + it] = t1 - t0;
            }
            rcodes[r] = res;
            MPI_Finalize();
            fflush(stdout);
            _exit(res == MPI_SUCCESS ? 0 : 1);
        }
        pids[r] = pid;
    }

    // Reap every rank; one failure aborts the others (exact PIDs only).
    std::vector<int> status(a.P, 0);
    int failed = 0;
    for (int done = 0; done < a.P;) {
        int st;
        pid_t p = waitpid(-1, &st, 0);
        if (p < 0) {
            if (errno == EINTR) continue;
            break;
        }
        for (int r = 0; r < a.P; r++)
            if (pids[r] == p) {
                status[r] = st;
                pids[r] = -1;
                done++;
                if (!(WIFEXITED(st) && WEXITSTATUS(st) == 0)) {
                    failed++;
                    shim_abort_all();
                }
            }
    }

    if (!a.out.empty()) {
        FILE* f = fopen(a.out.c_str(), "wb");
        if (!f || fwrite(out, 1, recv_bytes * a.P, f) != recv_bytes * a.P) return 3;
        fclose(f);
    }
    if (!a.trace.empty()) {
        FILE* f = fopen(a.trace.c_str(), "wb");
        if (!f) return 3;
        for (int r = 0; r < a.P; r++) {
            size_t dropped = 0, n = shim_trace_count(r, &dropped);
            const shim_trace_entry_t* e = shim_trace_entries(r);
            for (size_t i = 0; i < n; i++)
                if (e[i].call == 1) fwrite(&e[i], sizeof(*e), 1, f);
            if (dropped) fprintf(stderr, "bine_ref_run: rank %d dropped %zu trace records\n", r, dropped);
        }
        fclose(f);
    }

    // One JSON line: status per rank and the per-iteration max over ranks.
    std::string js = "{\"ok\": ";
    js += failed ? "false" : "true";
    js += ", \"P\": " + std::to_string(a.P) + ", \"coll\": \"" + a.coll + "\", \"dtype\": \"" + a.dtype +
          "\", \"count\": " + std::to_string(a.count) + ", \"status\": [";
    for (int r = 0; r < a.P; r++) {
        int st = status[r];
        std::string s = WIFEXITED(st) ? "exit:" + std::to_string(WEXITSTATUS(st))
                                      : (WIFSIGNALED(st) ? "signal:" + std::to_string(WTERMSIG(st)) : "unknown");
        js += (r ? ", \"" : "\"") + s + "\"";
    }
    js += "]";
    if (a.iters > 0 && !failed) {
        std::vector<double> mx(nt, 0.0);
        for (int it = 0; it < nt; it++)
            for (int r = 0; r < a.P; r++) mx[it] = std::max(mx[it], times[(size_t)r * nt + it]);
        std::vector<double> sorted = mx;
        std::sort(sorted.begin(), sorted.end());
        char buf[128];
        snprintf(buf, sizeof buf, ", \"median_s\": %.9g, \"min_s\": %.9g", sorted[nt / 2], sorted[0]);
        js += buf;
        js += ", \"iter_max_s\": [";
        for (int it = 0; it < nt; it++) {
            snprintf(buf, sizeof buf, "%s%.9g", it ? ", " : "", mx[it]);
            js += buf;
        }
        js += "]";
    }
    js += "}";
    printf("%s\n", js.c_str());
    return failed ? 1 : 0;
}

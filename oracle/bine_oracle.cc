// CPU restatement of the reference's MPI-layer Bine collectives: the oracle.
//
// TEST INFRASTRUCTURE ONLY.  tests/, __graft_entry__.smoke() and bench.py's
// CPU-baseline leg load it; the product (bine_trees_fugaku_b200) never does.
//
// Each simulated rank runs as a thread executing the same per-rank program
// as the reference (lib/libbine_common.cc, lib/libbine_coll_*.cc, MPI layer)
// over an in-process message layer with MPI's eager point-to-point
// semantics: a send copies its payload at once; receives from one
// (source, tag) complete in send order; a receive with nothing left to wait
// for (every live rank blocked) is reported as the deadlock the reference
// would hang in.  Conditions on which the reference asserts, exits or
// corrupts memory are reported as OR_ERR_REFERENCE_UNSUPPORTED with the
// reference line in the message.  Every function names the reference lines
// it restates.  Parity of this file with the reference itself is pinned by
// tests that run both on the same inputs (oracle/_ref, built from the
// reference sources by oracle/Makefile).
#include "bine_oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <functional>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace {

thread_local std::string g_last_error;

// ----------------------------------------------------------------- constants
// Signed Bine distances and negabinary ranges: lib/libbine_common.h:27-29.
const int kRhos[20] = {1,     -1,     3,     -5,     11,     -21,     43,     -85,     171,     -341,
                       683,   -1365,  2731,  -5461,  10923,  -21845,  43691,  -87381,  174763,  -349525};
const int kSmallestNb[20] = {0,     0,     -2,     -2,     -10,    -10,    -42,    -42,     -170,    -170,
                             -682,  -682,  -2730,  -2730,  -10922, -10922, -43690, -43690,  -174762, -174762};
const int kLargestNb[20] = {0,    1,    1,     5,     5,     21,    21,    85,    85,     341,
                            341,  1365, 1365,  5461,  5461,  21845, 21845, 87381, 87381,  349525};

// Message tags: lib/libbine_common.h:31-38.
const int kTagRS = 0x7FFF - 6 * 1;
const int kTagAG = 0x7FFF - 6 * 2;
const int kTagAR = 0x7FFF - 6 * 3;

struct Unsupported : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct Aborted : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// A bounds-checked view of one buffer: the reference indexes past its
// buffers in some unsupported configurations (e.g. the contiguous allgather
// at non-power-of-two sizes), which the restatement reports instead of
// corrupting memory.
struct Buf {
    char* p;
    size_t n;
    char* at(size_t off, size_t len, const char* where) const {
        if (off > n || len > n - off)
            throw Unsupported(std::string("out-of-bounds buffer access in ") + where +
                              " (the reference reads or writes past its buffer here)");
        return p + off;
    }
};

int dtype_size(int dt) {
    switch (dt) {
    case OR_INT32: return 4;
    case OR_INT64: return 8;
    case OR_FLOAT: return 4;
    case OR_DOUBLE: return 8;
    case OR_CHAR: return 1;
    default: return -1;
    }
}

// ------------------------------------------------------------- basic math
// ceil_log2: lib/libbine_coll.cc:65-87 (0 and 1 map to 0).
int ceil_log2(unsigned long long x) {
    int y = 0;
    while ((1ull << y) < x) y++;
    return y;
}
int mod(int a, int b) {  // lib/libbine_coll.cc:60-63
    int r = a % b;
    return r < 0 ? r + b : r;
}
bool is_p2(long x) { return x != 0 && (x & (x - 1)) == 0; }
bool is_odd(int x) { return x & 1; }

// Negabinary helpers, duplicated across the reference's per-collective files
// (e.g. lib/libbine_coll_reduce_scatter.cc:193-251).
uint32_t btonb(int32_t bin) {
    if (bin > 0x55555555) throw Unsupported("btonb: value out of range (lib/libbine_coll_reduce_scatter.cc:194)");
    const uint32_t mask = 0xAAAAAAAA;
    return (mask + (uint32_t)bin) ^ mask;
}
int32_t nbtob(uint32_t neg) {
    const uint32_t mask = 0xAAAAAAAA;
    return (int32_t)((mask ^ neg) - mask);
}
uint32_t reverse_bits(uint32_t x) {
    x = ((x >> 1) & 0x55555555u) | ((x & 0x55555555u) << 1);
    x = ((x >> 2) & 0x33333333u) | ((x & 0x33333333u) << 2);
    x = ((x >> 4) & 0x0f0f0f0fu) | ((x & 0x0f0f0f0fu) << 4);
    x = ((x >> 8) & 0x00ff00ffu) | ((x & 0x00ff00ffu) << 8);
    x = ((x >> 16) & 0xffffu) | ((x & 0xffffu) << 16);
    return x;
}
bool in_range(int x, uint32_t nbits) { return x >= kSmallestNb[nbits] && x <= kLargestNb[nbits]; }

// get_rank_negabinary_representation: lib/libbine_coll_reduce_scatter.cc:220-251.
// The MSB test keeps the reference's decimal 80000000 literal.
uint32_t rank_negabinary(uint32_t rank, uint32_t size) {
    uint32_t nba = UINT32_MAX, nbb = UINT32_MAX;
    size_t num_bits = ceil_log2(size);
    if (rank % 2) {
        if (in_range((int)rank, num_bits)) nba = btonb((int)rank);
        if (in_range((int)rank - (int)size, num_bits)) nbb = btonb((int)rank - (int)size);
    } else {
        if (in_range(-(int)rank, num_bits)) nba = btonb(-(int)rank);
        if (in_range(-(int)rank + (int)size, num_bits)) nbb = btonb(-(int)rank + (int)size);
    }
    if (nba == UINT32_MAX && nbb == UINT32_MAX)
        throw Unsupported("rank has no negabinary representation (lib/libbine_coll_reduce_scatter.cc:238)");
    if (nba == UINT32_MAX) return nbb;
    if (nbb == UINT32_MAX) return nba;
    return (nba & (80000000 >> (32 - num_bits))) ? nba : nbb;
}

// remap_rank: lib/libbine_coll_bcast.cc:978-984 (same as simulation/remap_rank.c:64-70).
uint32_t remap_rank(uint32_t rank, uint32_t size) {
    uint32_t r = rank_negabinary(rank, size);
    r = r ^ (r >> 1);
    size_t num_bits = ceil_log2(size);
    return reverse_bits(r) >> (32 - num_bits);
}

// nb_to_nu / get_nu: lib/libbine_coll_allgather.cc:1121-1158.
uint32_t nb_to_nu(uint32_t nb, uint32_t size) { return reverse_bits(nb ^ (nb >> 1)) >> (32 - ceil_log2(size)); }
uint32_t get_nu(uint32_t rank, uint32_t size) {
    uint32_t nba = UINT32_MAX, nbb = UINT32_MAX;
    size_t num_bits = ceil_log2(size);
    if (rank % 2) {
        if (in_range((int)rank, num_bits)) nba = btonb((int)rank);
        if (in_range((int)rank - (int)size, num_bits)) nbb = btonb((int)rank - (int)size);
    } else {
        if (in_range(-(int)rank, num_bits)) nba = btonb(-(int)rank);
        if (in_range(-(int)rank + (int)size, num_bits)) nbb = btonb(-(int)rank + (int)size);
    }
    if (nba == UINT32_MAX && nbb == UINT32_MAX)
        throw Unsupported("rank has no negabinary representation (lib/libbine_coll_allgather.cc:1141)");
    if (nba == UINT32_MAX) return nb_to_nu(nbb, size);
    if (nbb == UINT32_MAX) return nb_to_nu(nba, size);
    int nu_a = (int)nb_to_nu(nba, size), nu_b = (int)nb_to_nu(nbb, size);
    return nu_a < nu_b ? nu_a : nu_b;
}

// mersenne / remap_distance_doubling: lib/libbine_coll_alltoall.cc:380-409.
uint32_t mersenne(int n) { return (uint32_t)((1UL << (n + 1)) - 1); }
int remap_distance_doubling(uint32_t num) {
    int remapped = 0;
    while (num > 0) {
        int k = 31 - __builtin_clz(num);
        remapped ^= (0x1 << k);
        num ^= mersenne(k);
    }
    return remapped;
}

// --------------------------------------------------------------- topology
// BineCoordConverter: row-major coordinates (lib/libbine_common.cc:206-263).
struct Topo {
    int D = 1;
    int dims[3] = {0, 0, 0};
    int size = 0;
    int steps_per_dim[3] = {0, 0, 0};
    int num_steps = 0;
    Topo() = default;
    Topo(int ndims, const int* d) {
        D = ndims;
        size = 1;
        num_steps = 0;
        for (int i = 0; i < D; i++) {
            dims[i] = d[i];
            size *= d[i];
            steps_per_dim[i] = ceil_log2(d[i]);
            num_steps += steps_per_dim[i];
        }
    }
    void coord(int id, int* c) const {
        int nnodes = size;
        for (int i = 0; i < D; i++) {
            nnodes /= dims[i];
            c[i] = id / nnodes;
            id = id % nnodes;
        }
    }
    int id(const int* coords) const {
        int rank = 0, mult = 1;
        for (int i = D - 1; i >= 0; i--) {
            int c = coords[i];
            if (c >= dims[i]) c = c % dims[i];
            else if (c < 0) {
                c = c % dims[i];
                if (c) c = dims[i] + c;
            }
            rank += mult * c;
            mult *= dims[i];
        }
        return rank;
    }
};

// is_mirroring_port / get_distance_sign: lib/libbine_coll.cc:15-42.
bool is_mirroring_port(int port, int D) {
    if (D == 3) return port >= D;
    if (D == 2) return port == 2 || port == 3;
    if (D == 1) return port % 2;
    return false;
}
int distance_sign(int coord, int port, int D) {
    int m = 1;
    if (is_odd(coord)) m = -m;
    if (is_mirroring_port(port, D)) m = -m;
    return m;
}

struct StepInfo {
    int d;
    int step_in_d;
};

// compute_step_info: lib/libbine_coll.cc:306-331.
std::vector<StepInfo> compute_step_info(int port, const Topo& t) {
    std::vector<StepInfo> si(t.num_steps);
    int next_step_per_dim[3] = {0, 0, 0};
    int current_d = port % t.D;
    for (int i = 0; i < t.num_steps; i++) {
        si[i].d = current_d;
        si[i].step_in_d = next_step_per_dim[current_d];
        int d = current_d;
        if (next_step_per_dim[d] < ceil_log2(t.dims[d])) next_step_per_dim[d] += 1;
        if (i != t.num_steps - 1) {
            do {
                current_d = (current_d + 1) % t.D;
                d = current_d;
            } while (next_step_per_dim[d] >= ceil_log2(t.dims[d]));
        }
    }
    return si;
}

// get_peer_c: lib/libbine_coll.cc:89-107.
void get_peer_c(const int* coord_rank, int step, int port, const std::vector<StepInfo>& si, int family, const Topo& t,
                int* coord_peer) {
    for (int i = 0; i < t.D; i++) coord_peer[i] = coord_rank[i];
    int d = si[step].d, step_in_d = si[step].step_in_d;
    int distance;
    if (family == OR_FAMILY_RECDOUB) {
        distance = (coord_peer[d] ^ (1 << step_in_d)) - coord_peer[d];
        if (is_mirroring_port(port, t.D)) distance = -distance;
    } else {
        distance = kRhos[step_in_d] * distance_sign(coord_rank[d], port, t.D);
    }
    coord_peer[d] = mod(coord_peer[d] + distance, t.dims[d]);
}

// compute_peers: lib/libbine_coll.cc:443-504.
std::vector<int> compute_peers(int rank, int port, int family, const Topo& t) {
    std::vector<int> peers(t.num_steps);
    bool terminated[3] = {false, false, false};
    int next_step_per_dim[3] = {0, 0, 0};
    int coord[3];
    t.coord(rank, coord);
    int last_dim = port - 1;
    for (int i = 0; i < t.num_steps;) {
        int target_dim, relative_step;
        if (t.D > 1) {
            t.coord(rank, coord);
            unsigned o = 0;
            do {
                target_dim = (int)(((unsigned)(last_dim + 1) + o) % (unsigned)t.D);
                o++;
            } while (terminated[target_dim]);
            relative_step = next_step_per_dim[target_dim];
            ++next_step_per_dim[target_dim];
            last_dim = target_dim;
        } else {
            target_dim = 0;
            relative_step = i;
            coord[0] = rank;
        }
        int distance;
        if (family == OR_FAMILY_RECDOUB) {
            distance = (coord[target_dim] ^ (1 << relative_step)) - coord[target_dim];
        } else {
            distance = relative_step < 20 ? kRhos[relative_step] : 0;
            if (is_odd(coord[target_dim])) distance = -distance;
        }
        if (is_mirroring_port(port, t.D)) distance = -distance;
        if (relative_step < t.steps_per_dim[target_dim]) {
            coord[target_dim] = mod(coord[target_dim] + distance, t.dims[target_dim]);
            peers[i] = t.D > 1 ? t.id(coord) : coord[0];
            i++;
        } else {
            terminated[target_dim] = true;
        }
    }
    return peers;
}

// Binomial trees: build_tree / remap_ranks / get_tree, lib/libbine_coll.cc:122-151, 282-304, 334-389.
struct Tree {
    std::vector<uint32_t> parent, reached_at_step, remapped_ranks, remapped_ranks_max, subtree_roots;
};

void build_tree(const int* coord_root, int step, int port, int family, int dist, const Topo& t, Tree& tr,
                uint32_t subtree_root, const std::vector<StepInfo>& si) {
    for (int i = step; i < t.num_steps; i++) {
        int peer[3];
        int real_step = dist == OR_DIST_DECREASING ? t.num_steps - 1 - i : i;
        get_peer_c(coord_root, real_step, port, si, family, t, peer);
        uint32_t rank = (uint32_t)t.id(peer);
        if (tr.parent[rank] == UINT32_MAX || (uint32_t)i < tr.reached_at_step[rank]) {
            tr.parent[rank] = (uint32_t)t.id(coord_root);
            tr.reached_at_step[rank] = (uint32_t)i;
            tr.subtree_roots[rank] = step == 0 ? rank : subtree_root;
        }
        uint32_t actual_subtree_root = step == 0 ? rank : subtree_root;
        build_tree(peer, i + 1, port, family, dist, t, tr, actual_subtree_root, si);
    }
}

void remap_ranks_rec(const int* coord_root, int step, int port, int family, int dist, const Topo& t, uint32_t* next_rank,
                     Tree& tr, const std::vector<StepInfo>& si) {
    tr.remapped_ranks_max[t.id(coord_root)] = *next_rank;
    for (int i = step; i < t.num_steps; i++) {
        int peer[3];
        int real_step = dist == OR_DIST_DECREASING ? t.num_steps - 1 - i : i;
        get_peer_c(coord_root, real_step, port, si, family, t, peer);
        if (tr.parent[t.id(peer)] == (uint32_t)t.id(coord_root))
            remap_ranks_rec(peer, i + 1, port, family, dist, t, next_rank, tr, si);
    }
    tr.remapped_ranks[t.id(coord_root)] = *next_rank;
    (*next_rank)--;
}

Tree get_tree(int root, int port, int family, int dist, const Topo& t) {
    Tree tr;
    tr.parent.assign(t.size, UINT32_MAX);
    tr.reached_at_step.assign(t.size, (uint32_t)t.num_steps);
    tr.remapped_ranks.assign(t.size, 0);
    tr.remapped_ranks_max.assign(t.size, 0);
    tr.subtree_roots.assign(t.size, 0);
    int coord_root[3];
    t.coord(root, coord_root);
    std::vector<StepInfo> si = compute_step_info(port, t);
    build_tree(coord_root, 0, port, family, dist, t, tr, 0, si);
    tr.parent[root] = UINT32_MAX;
    tr.reached_at_step[root] = 0;
    tr.subtree_roots[root] = UINT32_MAX;
    uint32_t next_rank = (uint32_t)t.size - 1;
    remap_ranks_rec(coord_root, 0, port, family, dist, t, &next_rank, tr, si);
    if (next_rank != UINT32_MAX) throw Unsupported("get_tree: tree does not reach every rank (lib/libbine_coll.cc:380)");
    return tr;
}

// ------------------------------------------------- BineBitmapCalculator
// lib/libbine_common.cc:1484-1625 (bitmaps), 1882-1915 (queries),
// 1981-2047 (constructor, dfs).
struct BlockInfo {
    size_t offset;  // bytes
    size_t count;   // elements
};
struct ChunkParams {
    size_t send_offset, send_count, recv_offset, recv_count;
};

class BitmapCalc {
  public:
    BitmapCalc(int rank, const Topo& t, int port, const std::vector<std::vector<BlockInfo>>& bi, bool remap, int family)
        : t_(t), port_(port), bi_(bi), remap_(remap), rank_(rank), family_(family) {
        S_ = t.num_steps;
        peers_ = compute_peers(rank, port, family, t);
        si_ = compute_step_info(port, t);
        t.coord(rank, coord_mine_);
        if (remap) {
            remapped_rank_ = (uint32_t)t.size - 1;
            int c0[3], me[3];
            t.coord(0, c0);
            t.coord(rank, me);
            bool found = false;
            dfs(c0, 0, me, &remapped_rank_, &found);
            min_r_ = min_s_ = 0;
            max_r_ = max_s_ = t.size;
            chunks_.resize(S_);
            for (int s = 0; s < S_; s++) next_chunk(s);
        } else {
            block_step_.assign(t.size, (uint32_t)S_);
            for (int i = 0; i < S_; i++) {
                int peer[3];
                get_peer_c(coord_mine_, i, port, si_, family, t, peer);
                compute_block_step(peer, i, i, block_step_.data());
            }
            block_step_[rank] = (uint32_t)S_;
            send_bm_.assign(S_, std::vector<char>(t.size, 0));
            recv_bm_.assign(S_, std::vector<char>(t.size, 0));
            for (int s = 0; s < S_; s++) next_bitmaps(s);
        }
    }
    int peer(int step, bool rs) const { return peers_[rs ? step : S_ - step - 1]; }
    bool must_send(int step, bool rs, int b) const {
        return rs ? send_bm_[step][b] : recv_bm_[S_ - step - 1][b];
    }
    bool must_recv(int step, bool rs, int b) const {
        return rs ? recv_bm_[step][b] : send_bm_[S_ - step - 1][b];
    }
    ChunkParams chunk(int step, bool rs) const {
        if (rs) return chunks_[step];
        const ChunkParams& c = chunks_[S_ - step - 1];
        return ChunkParams{c.recv_offset, c.recv_count, c.send_offset, c.send_count};
    }
    const std::vector<uint32_t>& block_step() const { return block_step_; }

  private:
    void compute_block_step(const int* coord_rank, int starting_step, int step, uint32_t* bs) const {
        if (step < S_) {
            for (int i = step + 1; i < S_; i++) {
                int peer[3];
                get_peer_c(coord_rank, i, port_, si_, family_, t_, peer);
                compute_block_step(peer, starting_step, i, bs);
            }
            int r = t_.id(coord_rank);
            if (bs[r] == (uint32_t)S_ || (uint32_t)starting_step > bs[r]) bs[r] = (uint32_t)starting_step;
        }
    }
    void next_bitmaps(int s) {
        for (int i = 0; i < t_.size; i++)
            if (block_step_[i] == (uint32_t)s) send_bm_[s][i] = 1;
        std::vector<uint32_t> pbs(t_.size, (uint32_t)S_);
        int p = peer(s, true);
        int pc[3];
        t_.coord(p, pc);
        for (int j = s; j < S_; j++) {
            int pp[3];
            get_peer_c(pc, j, port_, si_, family_, t_, pp);
            compute_block_step(pp, j, j, pbs.data());
        }
        pbs[p] = (uint32_t)S_;
        for (int i = 0; i < t_.size; i++)
            if (pbs[i] == (uint32_t)s) recv_bm_[s][i] = 1;
    }
    void next_chunk(int s) {
        min_s_ = min_r_;
        max_s_ = max_r_;
        size_t middle = (min_r_ + max_r_ + 1) / 2;
        if (remapped_rank_ < middle) {
            min_s_ = middle;
            max_r_ = middle;
        } else {
            max_s_ = middle;
            min_r_ = middle;
        }
        ChunkParams& c = chunks_[s];
        c.send_offset = bi_[port_][min_s_].offset;
        c.send_count = 0;
        for (size_t i = min_s_; i < max_s_; i++) c.send_count += bi_[port_][i].count;
        c.recv_offset = bi_[port_][min_r_].offset;
        c.recv_count = 0;
        for (size_t i = min_r_; i < max_r_; i++) c.recv_count += bi_[port_][i].count;
    }
    void dfs(const int* coord_rank, int step, const int* target, uint32_t* rr, bool* found) const {
        for (int i = step; i < S_; i++) {
            int peer[3];
            get_peer_c(coord_rank, i, port_, si_, family_, t_, peer);
            dfs(peer, i + 1, target, rr, found);
        }
        if (*found) (*rr)--;
        if (std::equal(coord_rank, coord_rank + t_.D, target)) *found = true;
    }

    const Topo& t_;
    int port_;
    const std::vector<std::vector<BlockInfo>>& bi_;
    bool remap_;
    int rank_;
    int family_;
    int S_;
    std::vector<int> peers_;
    std::vector<StepInfo> si_;
    int coord_mine_[3];
    uint32_t remapped_rank_ = 0;
    size_t min_r_ = 0, max_r_ = 0, min_s_ = 0, max_s_ = 0;
    std::vector<ChunkParams> chunks_;
    std::vector<uint32_t> block_step_;
    std::vector<std::vector<char>> send_bm_, recv_bm_;
};

// ------------------------------------------------------ in-process messaging
struct Msg {
    int src;
    int tag;
    std::vector<char> data;
};

class World {
  public:
    World(int P, bool trace) : P_(P), boxes_(P), wait_src_(P, -1), wait_tag_(P, 0), trace_(trace) {}

    void send(int src, int dst, int tag, const void* buf, size_t bytes) {
        if (dst < 0 || dst >= P_) throw Unsupported("send to an invalid rank " + std::to_string(dst));
        Msg m{src, tag, std::vector<char>((const char*)buf, (const char*)buf + bytes)};
        std::lock_guard<std::mutex> lk(mu_);
        if (trace_) msgs_.push_back(oracle_msg_t{src, dst, bytes});
        boxes_[dst].push_back(std::move(m));
        cv_.notify_all();
    }

    // Blocks until a message from (src, tag) is available; FIFO per pair.
    size_t recv(int me, int src, int tag, void* buf, size_t cap) {
        std::unique_lock<std::mutex> lk(mu_);
        while (true) {
            if (aborted_) throw Aborted("aborted");
            auto& box = boxes_[me];
            for (auto it = box.begin(); it != box.end(); ++it) {
                if (it->src == src && it->tag == tag) {
                    size_t n = it->data.size();
                    if (n > cap) {
                        abort_locked();
                        throw Unsupported("rank " + std::to_string(me) + " receives " + std::to_string(n) +
                                          " bytes from rank " + std::to_string(src) + " into a " +
                                          std::to_string(cap) + "-byte buffer (MPI_ERR_TRUNCATE)");
                    }
                    if (n) std::memcpy(buf, it->data.data(), n);
                    box.erase(it);
                    return n;
                }
            }
            wait_src_[me] = src;
            wait_tag_[me] = tag;
            blocked_++;
            if (deadlocked_locked()) {
                abort_locked();
                throw Unsupported("every live rank waits for a message that is never sent (the reference "
                                  "deadlocks); rank " +
                                  std::to_string(me) + " waits for rank " + std::to_string(src));
            }
            cv_.wait(lk);
            blocked_--;
            wait_src_[me] = -1;
        }
    }

    void run(const std::function<void(int)>& body) {
        alive_ = P_;
        std::vector<std::thread> th;
        th.reserve(P_);
        for (int r = 0; r < P_; r++) {
            th.emplace_back([this, r, &body]() {
                try {
                    body(r);
                } catch (Unsupported& e) {
                    std::lock_guard<std::mutex> lk(mu_);
                    if (err_.empty()) err_ = e.what();
                    abort_locked();
                } catch (Aborted&) {
                } catch (std::out_of_range& e) {
                    // A displs/counts index past the rank count: the reference
                    // reads past its arrays here (undefined behaviour).
                    std::lock_guard<std::mutex> lk(mu_);
                    if (err_.empty()) err_ = std::string("index past the end of a per-rank table: ") + e.what();
                    abort_locked();
                } catch (std::exception& e) {
                    std::lock_guard<std::mutex> lk(mu_);
                    if (err_.empty()) err_ = std::string("internal: ") + e.what();
                    internal_ = true;
                    abort_locked();
                }
                std::lock_guard<std::mutex> lk(mu_);
                alive_--;
                if (!aborted_ && alive_ > 0 && deadlocked_locked()) {
                    // Everyone still alive is waiting for a rank that finished.
                    err_ = "ranks wait for messages that are never sent (the reference deadlocks)";
                    abort_locked();
                }
            });
        }
        for (auto& t : th) t.join();
    }

    const std::string& error() const { return err_; }
    bool internal_error() const { return internal_; }
    const std::vector<oracle_msg_t>& msgs() const { return msgs_; }

  private:
    // True when every live rank is blocked and none of them has the message
    // it waits for in its mailbox (a notified rank that has not run yet
    // still counts as blocked, so the mailboxes decide).
    bool deadlocked_locked() const {
        if (blocked_ != alive_) return false;
        for (int r = 0; r < P_; r++) {
            if (wait_src_[r] < 0) continue;
            for (const Msg& m : boxes_[r])
                if (m.src == wait_src_[r] && m.tag == wait_tag_[r]) return false;
        }
        return true;
    }
    void abort_locked() {
        aborted_ = true;
        cv_.notify_all();
    }
    int P_;
    std::mutex mu_;
    std::condition_variable cv_;
    std::vector<std::deque<Msg>> boxes_;
    std::vector<int> wait_src_, wait_tag_;
    int alive_ = 0, blocked_ = 0;
    bool aborted_ = false, internal_ = false, trace_;
    std::string err_;
    std::vector<oracle_msg_t> msgs_;
};

// ------------------------------------------------------------ reductions
// MPI_Reduce_local(in, inout): inout[i] = in[i] + inout[i] (MPI semantics,
// the same loop as the shim the reference is linked against).
template <class T>
void add_into(const char* in, char* inout, size_t n) {
    const T* a = (const T*)in;
    T* b = (T*)inout;
    for (size_t i = 0; i < n; i++) b[i] = (T)(a[i] + b[i]);
}
void mpi_reduce_local(int dt, const void* in, void* inout, size_t n) {
    switch (dt) {
    case OR_INT32: add_into<int32_t>((const char*)in, (char*)inout, n); break;
    case OR_INT64: add_into<int64_t>((const char*)in, (char*)inout, n); break;
    case OR_FLOAT: add_into<float>((const char*)in, (char*)inout, n); break;
    case OR_DOUBLE: add_into<double>((const char*)in, (char*)inout, n); break;
    case OR_CHAR: add_into<signed char>((const char*)in, (char*)inout, n); break;
    }
}
// The reference's own reduce_local(a, b, out): out = a + b for INT32, INT,
// CHAR and FLOAT only; any other type exits (lib/libbine_coll.cc:209-267).
void ref_reduce_local3(int dt, const void* a, const void* b, void* out, size_t n) {
    if (dt == OR_INT64 || dt == OR_DOUBLE)
        throw Unsupported("reduce_local: 'Unknown reduction datatype' exit for 64-bit types (lib/libbine_coll.cc:263)");
    std::vector<char> tmp((const char*)b, (const char*)b + n * dtype_size(dt));
    mpi_reduce_local(dt, a, tmp.data(), n);
    std::memcpy(out, tmp.data(), tmp.size());
}

// ------------------------------------------------------------- rank state
struct Ctx {
    const oracle_call_t* call;
    Topo topo;
    int P;
    int es;
    long count;
    int ports;
    int family;
    int dist;
    World* world;
    const char* in;
    char* out;
    size_t send_bytes, recv_bytes;
};

char* out_of(const Ctx& c, int r) { return c.out + c.recv_bytes * r; }
const char* in_of(const Ctx& c, int r) { return c.in + c.send_bytes * r; }

// Block partitions: lib/libbine.cc:971-1010 (allreduce: by port, then by
// block) and lib/libbine.cc:1086-1114, 1185-1206 (reduce_scatter and
// allgather: by block, then by port).
std::vector<std::vector<BlockInfo>> blocks_port_then_block(size_t count, int P, int ports, int es) {
    std::vector<std::vector<BlockInfo>> bi(ports, std::vector<BlockInfo>(P));
    unsigned partition = (unsigned)(count / ports), remaining = (unsigned)(count % ports), so_far = 0;
    for (int p = 0; p < ports; p++) {
        size_t count_port = partition + ((unsigned)p < remaining ? 1 : 0);
        size_t offset_port = (size_t)so_far * es;
        so_far += (unsigned)count_port;
        unsigned bpart = (unsigned)(count_port / P), brem = (unsigned)(count_port % P);
        size_t bso = 0;
        for (int i = 0; i < P; i++) {
            size_t cb = bpart + ((unsigned)i < brem ? 1 : 0);
            bi[p][i].count = cb;
            bi[p][i].offset = offset_port + bso * es;
            bso += cb;
        }
    }
    return bi;
}
std::vector<std::vector<BlockInfo>> blocks_block_then_port(size_t per_block, int P, int ports, int es) {
    std::vector<std::vector<BlockInfo>> bi(ports, std::vector<BlockInfo>(P));
    size_t so_far = 0;
    for (int i = 0; i < P; i++) {
        size_t partition = per_block / ports, remaining = per_block % ports;
        size_t block_offset = so_far * es, bso = 0;
        for (int p = 0; p < ports; p++) {
            size_t cp = partition + ((size_t)p < remaining ? 1 : 0);
            bi[p][i].count = cp;
            bi[p][i].offset = block_offset + bso * es;
            bso += cp;
        }
        so_far += per_block;
    }
    return bi;
}

// ---------------------------------------------------- allreduce B family
// bine_coll_b (lib/libbine_common.cc:1631-1735) with bine_coll_step_b
// (930-1030), _coalesce (1032-1159) and _cont (1162-1237), dispatch 1239-1257.
void allreduce_b(const Ctx& c, int r, const std::vector<std::vector<BitmapCalc*>>& calc,
                 const std::vector<std::vector<BlockInfo>>& bi) {
    const int algo = c.call->algo;
    const size_t nbytes = (size_t)c.count * c.es;
    char* recvbuf = out_of(c, r);
    std::vector<char> tmp(nbytes ? nbytes : 1);
    std::memcpy(recvbuf, in_of(c, r), nbytes);
    const int S = c.topo.num_steps;
    for (int phase = 0; phase < 2; phase++) {
        const bool rs = phase == 0;
        char* bufs = recvbuf;
        char* bufr = rs ? tmp.data() : recvbuf;
        for (int step = 0; step < S; step++) {
            struct PostedRecv {
                int peer, tag;
                size_t off, cnt;
            };
            std::vector<PostedRecv> recvs;
            for (int port = 0; port < c.ports; port++) {
                const BitmapCalc& sb = *calc[port][r];
                int peer = sb.peer(step, rs);
                int tag = (rs ? kTagRS : kTagAG) + port;
                if (algo == OR_AR_B) {
                    for (int i = 0; i < c.P; i++) {
                        bool sblk = sb.must_send(step, rs, i), rblk = sb.must_recv(step, rs, i);
                        size_t bc = bi[port][i].count, bo = bi[port][i].offset;
                        if (sblk) c.world->send(r, peer, tag, bufs + bo, bc * c.es);
                        if (rblk) recvs.push_back({peer, tag, bo, bc});
                    }
                } else if (algo == OR_AR_B_COALESCE) {
                    bool start_s = false, start_r = false;
                    size_t off_s = 0, off_r = 0, cnt_s = 0, cnt_r = 0;
                    for (int i = 0; i < c.P; i++) {
                        bool sblk = sb.must_send(step, rs, i), rblk = sb.must_recv(step, rs, i);
                        size_t bc = bi[port][i].count, bo = bi[port][i].offset;
                        if (sblk) {
                            if (!start_s) {
                                start_s = true;
                                off_s = bo;
                            }
                            cnt_s += bc;
                        }
                        if (start_s && (!sblk || i == c.P - 1)) {
                            c.world->send(r, peer, tag, bufs + off_s, cnt_s * c.es);
                            cnt_s = 0;
                            off_s = 0;
                            start_s = false;
                        }
                        if (rblk) {
                            if (!start_r) {
                                start_r = true;
                                off_r = bo;
                            }
                            cnt_r += bc;
                        }
                        if (start_r && (!rblk || i == c.P - 1)) {
                            recvs.push_back({peer, tag, off_r, cnt_r});
                            cnt_r = 0;
                            off_r = 0;
                            start_r = false;
                        }
                    }
                } else {  // B_CONT
                    ChunkParams cp = sb.chunk(step, rs);
                    c.world->send(r, peer, tag, bufs + cp.send_offset, cp.send_count * c.es);
                    recvs.push_back({peer, tag, cp.recv_offset, cp.recv_count});
                }
            }
            for (const PostedRecv& pr : recvs) {
                c.world->recv(r, pr.peer, pr.tag, bufr + pr.off, pr.cnt * c.es);
                if (rs) mpi_reduce_local(c.call->dtype, bufr + pr.off, bufs + pr.off, pr.cnt);
            }
        }
    }
}

// ------------------------------------------------------- allreduce L
// bine_coll_l_mpi (lib/libbine_common.cc:733-846) with
// shrink_non_power_of_two (269-319) and enlarge_non_power_of_two (321-353).
void allreduce_l(const Ctx& c, int r, const Topo& virt, bool all_p2) {
    const size_t nbytes = (size_t)c.count * c.es;
    const int dt = c.call->dtype;
    const Topo& real = c.topo;
    char* recvbuf = out_of(c, r);
    const char* sendbuf = in_of(c, r);
    std::vector<char> tmp(nbytes ? nbytes : 1);
    int coord[3];
    real.coord(r, coord);
    int idle = 0, first_copy_done = 0;
    if (!all_p2) {
        for (int i = 0; i < real.D; i++) {
            if (is_p2(real.dims[i])) continue;
            int cp[3] = {coord[0], coord[1], coord[2]};
            int extra = real.dims[i] - virt.dims[i];
            const char* rs = first_copy_done ? recvbuf : sendbuf;
            char* rr = first_copy_done ? tmp.data() : recvbuf;
            const char* ra = first_copy_done ? tmp.data() : sendbuf;
            if (coord[i] >= virt.dims[i]) {
                cp[i] = coord[i] - extra;
                c.world->send(r, real.id(cp), kTagAR, rs, nbytes);
                idle = 1;
                break;
            } else if (coord[i] + extra >= virt.dims[i]) {
                cp[i] = coord[i] + extra;
                c.world->recv(r, real.id(cp), kTagAR, rr, nbytes);
                mpi_reduce_local(dt, ra, recvbuf, c.count);
                first_copy_done = 1;
            }
        }
    }
    if (!idle) {
        int rank_virtual = virt.id(coord);
        unsigned partition = (unsigned)(c.count / c.ports), remaining = (unsigned)(c.count % c.ports);
        std::vector<std::vector<int>> vpeers(c.ports);
        for (int p = 0; p < c.ports; p++) vpeers[p] = compute_peers(rank_virtual, p, c.family, virt);
        for (int step = 0; step < virt.num_steps; step++) {
            const char* bs;
            char* br;
            const char* ba;
            if (step == 0 && !first_copy_done) {
                bs = sendbuf;
                br = recvbuf;
                ba = sendbuf;
            } else {
                bs = recvbuf;
                br = tmp.data();
                ba = tmp.data();
            }
            unsigned so_far = 0;
            std::vector<std::pair<int, size_t>> posted;  // (peer, offset) per port
            std::vector<size_t> cnts;
            for (int p = 0; p < c.ports; p++) {
                int vc[3];
                virt.coord(vpeers[p][step], vc);
                int peer = real.id(vc);
                size_t cnt = partition + ((unsigned)p < remaining ? 1 : 0);
                size_t off = (size_t)so_far * c.es;
                so_far += (unsigned)cnt;
                c.world->send(r, peer, kTagAR, bs + off, cnt * c.es);
                posted.push_back({peer, off});
                cnts.push_back(cnt);
            }
            for (int p = 0; p < c.ports; p++)
                c.world->recv(r, posted[p].first, kTagAR, br + posted[p].second, cnts[p] * c.es);
            mpi_reduce_local(dt, ba, recvbuf, c.count);
        }
    }
    if (!all_p2) {
        for (int d = real.D - 1; d >= 0; d--) {
            if (is_p2(real.dims[d])) continue;
            int cp[3] = {coord[0], coord[1], coord[2]};
            int extra = real.dims[d] - virt.dims[d];
            if (coord[d] >= virt.dims[d]) {
                cp[d] = coord[d] - extra;
                c.world->recv(r, real.id(cp), kTagAR, recvbuf, nbytes);
            } else if (coord[d] + extra >= virt.dims[d]) {
                cp[d] = coord[d] + extra;
                c.world->send(r, real.id(cp), kTagAR, recvbuf, nbytes);
            }
        }
    }
}

// ------------------------------------------------------ reduce_scatter
// bine_reduce_scatter_mpi_contiguous (lib/libbine_coll_reduce_scatter.cc:660-758).
void reduce_scatter_cont(const Ctx& c, int r, const std::vector<std::vector<BlockInfo>>& bi) {
    const int dt = c.call->dtype;
    const size_t tmpbuf_size = bi[0][0].count * c.es * c.ports * c.P;
    std::vector<char> tmp(tmpbuf_size ? tmpbuf_size : 1);
    const char* sendbuf = in_of(c, r);
    char* recvbuf = out_of(c, r);
    const int S = c.topo.num_steps;
    for (int port = 0; port < c.ports; port++) {
        std::vector<int> peers = compute_peers(r, port, c.family, c.topo);
        Tree tree = get_tree(r, port, c.family, c.dist, c.topo);
        size_t offset_port = tmpbuf_size / c.ports * port;
        char* tsp = tmp.data() + offset_port;
        for (int i = 0; i < c.P; i++)
            std::memcpy(tmp.data() + offset_port + bi[port][0].count * tree.remapped_ranks[i] * c.es,
                        sendbuf + bi[port][i].offset, bi[port][i].count * c.es);
        for (int step = 0; step < S; step++) {
            int peer = c.dist == OR_DIST_DECREASING ? peers[S - step - 1] : peers[step];
            size_t num_blocks = (size_t)(c.P / std::pow(2.0, step + 1));
            size_t cnt = num_blocks * bi[port][0].count;
            // MPI_Sendrecv_replace: the eager send copies before the receive.
            c.world->send(r, peer, kTagRS, tsp + cnt * c.es, cnt * c.es);
            c.world->recv(r, peer, kTagRS, tsp + cnt * c.es, cnt * c.es);
            if (step == S - 1)
                ref_reduce_local3(dt, tsp + cnt * c.es, tsp, recvbuf + offset_port, cnt);
            else
                mpi_reduce_local(dt, tsp + cnt * c.es, tsp, cnt);
        }
    }
}

// ------------------------------------------------------------ allgather
// bine_allgather_mpi_contiguous (lib/libbine_coll_allgather.cc:289-374).
void allgather_cont_permute(const Ctx& c, int r, const std::vector<std::vector<BlockInfo>>& bi) {
    const long sendcount = c.count;
    size_t tmpbuf_size = (size_t)std::ceil((float)sendcount / c.ports) * c.ports * c.es * c.P;
    std::vector<char> tmpv(tmpbuf_size ? tmpbuf_size : 1);
    Buf tmp{tmpv.data(), tmpbuf_size};
    Buf sendbuf{(char*)in_of(c, r), c.send_bytes}, recvbuf{out_of(c, r), c.recv_bytes};
    const char* where = "allgather CONT_PERMUTE (lib/libbine_coll_allgather.cc:332-362)";
    const int S = c.topo.num_steps;
    for (int port = 0; port < c.ports; port++) {
        std::vector<int> peers = compute_peers(r, port, c.family, c.topo);
        size_t top = (tmpbuf_size / c.ports) * port;
        size_t b0 = bi[port][0].count * c.es;
        std::memcpy(tmp.at(top, b0, where), sendbuf.at(bi[port][0].offset, b0, where), b0);
        for (int step = 0; step < S; step++) {
            int peer = c.dist == OR_DIST_DECREASING ? peers[S - step - 1] : peers[step];
            size_t cnt = (size_t)std::pow(2.0, step) * bi[port][0].count;
            c.world->send(r, peer, kTagAG, tmp.at(top, cnt * c.es, where), cnt * c.es);
            c.world->recv(r, peer, kTagAG, tmp.at(top + cnt * c.es, cnt * c.es, where), cnt * c.es);
        }
        Tree perm = get_tree(r, port, c.family, c.dist == OR_DIST_DECREASING ? OR_DIST_INCREASING : OR_DIST_DECREASING,
                             c.topo);
        for (int i = 0; i < c.P; i++) {
            size_t pos_tmp = perm.remapped_ranks[i] * bi[port][0].count * c.es;
            size_t len = bi[port][i].count * c.es;
            std::memcpy(recvbuf.at(bi[port][i].offset, len, where), tmp.at(top + pos_tmp, len, where), len);
        }
    }
}

// bine_allgather_send_mpi (lib/libbine_coll_allgather.cc:492-574).
void allgather_cont_send(const Ctx& c, int r) {
    const size_t sb = (size_t)c.count * c.es;
    Buf sendbuf{(char*)in_of(c, r), c.send_bytes}, recvbuf{out_of(c, r), c.recv_bytes};
    const char* where = "allgather CONT_SEND (lib/libbine_coll_allgather.cc:531-566)";
    const int S = c.topo.num_steps;
    std::vector<int> peers = compute_peers(r, 0, c.family, c.topo);
    Tree tree = get_tree(0, 0, c.family, c.dist == OR_DIST_DECREASING ? OR_DIST_INCREASING : OR_DIST_DECREASING, c.topo);
    size_t remapped = tree.remapped_ranks[r];
    std::vector<uint32_t> inv(c.P);
    for (int i = 0; i < c.P; i++) inv[tree.remapped_ranks[i]] = i;
    c.world->send(r, inv[r], kTagAG, sendbuf.at(0, sb, where), sb);
    c.world->recv(r, (int)remapped, kTagAG, recvbuf.at(remapped * sb, sb, where), sb);
    size_t num_blocks = 1, min_res = tree.remapped_ranks[r];
    for (int step = 0; step < S; step++) {
        int peer = c.dist == OR_DIST_DECREASING ? peers[S - step - 1] : peers[step];
        size_t cnt = num_blocks * sb;
        size_t min_r = tree.remapped_ranks[peer] & ~((1u << step) - 1);
        c.world->send(r, peer, kTagAG, recvbuf.at(min_res * sb, cnt, where), cnt);
        c.world->recv(r, peer, kTagAG, recvbuf.at(min_r * sb, cnt, where), cnt);
        min_res = std::min(min_res, min_r);
        num_blocks *= 2;
    }
}

// bine_allgather_blocks_mpi (lib/libbine_coll_allgather.cc:1161-1228).
void allgather_blocks(const Ctx& c, int r) {
    const long sc = c.count;
    const int size = c.P;
    char* recvbuf = out_of(c, r);
    std::memcpy(recvbuf + sc * r * c.es, in_of(c, r), sc * c.es);
    int inverse_mask = 0x1 << (int)(std::ceil(std::log2(size)) - 1);
    int step = 0;
    while (inverse_mask > 0) {
        int partner = r % 2 == 0 ? mod(r + nbtob((inverse_mask << 1) - 1), size)
                                 : mod(r - nbtob((inverse_mask << 1) - 1), size);
        for (int block = 1; block < size; block++) {
            int k = 31 - __builtin_clz(get_nu(block, size));
            if (k == step) {
                int bsend, brecv;
                if (r % 2 == 0) {
                    brecv = mod(block + r, size);
                    bsend = mod(partner - block, size);
                } else {
                    brecv = mod(r - block, size);
                    bsend = mod(block + partner, size);
                }
                bool do_send = bsend != partner, do_recv = brecv != r;
                if (do_send) c.world->send(r, partner, 0, recvbuf + (size_t)bsend * sc * c.es, sc * c.es);
                if (do_recv) c.world->recv(r, partner, 0, recvbuf + (size_t)brecv * sc * c.es, sc * c.es);
            }
        }
        inverse_mask >>= 1;
        step++;
    }
}

// ---------------------------------------------------------------- bcast
// bine_bcast_l_mpi (lib/libbine_coll_bcast.cc:635-665).
void bcast_tree(const Ctx& c, int r) {
    const int size = c.P, root = c.call->root;
    char* buf = out_of(c, r);
    if (r == root) std::memcpy(buf, in_of(c, r), (size_t)c.count * c.es);
    int vrank = mod(r - root, size);
    int mask = 0x1 << ((int)std::ceil(std::log2(size)) - 1);
    int recvd = root == r;
    while (mask > 0) {
        int partner = (int)(btonb(vrank) ^ ((mask << 1) - 1));
        partner = mod(nbtob(partner) + root, size);
        int mask_lsbs = (mask << 1) - 1;
        int lsbs = (int)(btonb(vrank) & mask_lsbs);
        bool equal = lsbs == 0 || lsbs == mask_lsbs;
        if (recvd) {
            c.world->send(r, partner, 0, buf, (size_t)c.count * c.es);
        } else if (equal) {
            c.world->recv(r, partner, 0, buf, (size_t)c.count * c.es);
            recvd = 1;
        }
        mask >>= 1;
    }
}

// bine_bcast_scatter_allgather_mpi (lib/libbine_coll_bcast.cc:985-1093).
void bcast_scatter_allgather(const Ctx& c, int r) {
    const int size = c.P, root = c.call->root;
    if (root != 0) throw Unsupported("scatter-allgather bcast asserts root == 0 (lib/libbine_coll_bcast.cc:993)");
    Buf B{out_of(c, r), c.recv_bytes};
    const char* where = "scatter-allgather bcast (lib/libbine_coll_bcast.cc:1039-1088)";
    char* buf = B.p;
    if (r == root) std::memcpy(B.at(0, (size_t)c.count * c.es, where), in_of(c, r), (size_t)c.count * c.es);
    (void)buf;
    std::vector<int> displs(size), counts(size);
    int cpr = (int)(c.count / size), rem = (int)(c.count % size);
    for (int i = 0; i < size; i++) {
        displs[i] = cpr * i + (i < rem ? i : rem);
        counts[i] = cpr + (i < rem ? 1 : 0);
    }
    int mask = 0x1;
    int inverse_mask = 0x1 << (int)(std::ceil(std::log2(size)) - 1);
    int block_first_mask = ~(inverse_mask - 1);
    int remapped = (int)remap_rank(r, size);
    int receiving_mask = inverse_mask << 1;
    if (r != root) receiving_mask = 0x1 << (ffs(remapped) - 1);
    int recvd = root == r;
    while (mask < size) {
        int partner = r % 2 == 0 ? mod(r + nbtob((mask << 1) - 1), size) : mod(r - nbtob((mask << 1) - 1), size);
        int sbf = (int)remap_rank(partner, size) & block_first_mask;
        int sbl = sbf + inverse_mask - 1;
        int scount = displs.at(sbl) - displs.at(sbf) + counts.at(sbl);
        int rbf = remapped & block_first_mask;
        int rbl = rbf + inverse_mask - 1;
        int rcount = displs.at(rbl) - displs.at(rbf) + counts.at(rbl);
        if (recvd) {
            c.world->send(r, partner, 0, B.at((size_t)displs[sbf] * c.es, (size_t)scount * c.es, where),
                          (size_t)scount * c.es);
        } else if (inverse_mask == receiving_mask || partner == root) {
            c.world->recv(r, partner, 0, B.at((size_t)displs[rbf] * c.es, (size_t)rcount * c.es, where),
                          (size_t)rcount * c.es);
            recvd = 1;
        }
        mask <<= 1;
        inverse_mask >>= 1;
        block_first_mask >>= 1;
    }
    mask >>= 1;
    inverse_mask = 0x1;
    block_first_mask = ~0x0;
    while (mask > 0) {
        int partner = r % 2 == 0 ? mod(r + nbtob((mask << 1) - 1), size) : mod(r - nbtob((mask << 1) - 1), size);
        bool has_r = !(inverse_mask < receiving_mask), has_s = !(inverse_mask == receiving_mask);
        int sbf = 0, scount = 0, rbf = 0, rcount = 0;
        if (has_s) {
            sbf = remapped & block_first_mask;
            int sbl = sbf + inverse_mask - 1;
            scount = displs.at(sbl) - displs.at(sbf) + counts.at(sbl);
        }
        if (has_r) {
            rbf = (int)remap_rank(partner, size) & block_first_mask;
            int rbl = rbf + inverse_mask - 1;
            rcount = displs.at(rbl) - displs.at(rbf) + counts.at(rbl);
        }
        if (has_s)
            c.world->send(r, partner, 0, B.at((size_t)displs[sbf] * c.es, (size_t)scount * c.es, where),
                          (size_t)scount * c.es);
        if (has_r)
            c.world->recv(r, partner, 0, B.at((size_t)displs[rbf] * c.es, (size_t)rcount * c.es, where),
                          (size_t)rcount * c.es);
        mask >>= 1;
        inverse_mask <<= 1;
        block_first_mask <<= 1;
    }
}

// --------------------------------------------------------------- reduce
// bine_reduce_mpi (lib/libbine_coll_reduce.cc:575-615).
void reduce_tree(const Ctx& c, int r) {
    const int size = c.P, root = c.call->root, dt = c.call->dtype;
    const size_t nbytes = (size_t)c.count * c.es;
    std::vector<char> tmp(nbytes ? nbytes : 1), own;
    char* recvbuf;
    if (r != root) {
        own.resize(nbytes ? nbytes : 1);
        recvbuf = own.data();
    } else {
        recvbuf = out_of(c, r);
    }
    std::memcpy(recvbuf, in_of(c, r), nbytes);
    int vrank = mod(r - root, size);
    int mask = 0x1;
    while (mask < size) {
        int partner = (int)(btonb(vrank) ^ ((mask << 1) - 1));
        partner = mod(nbtob(partner) + root, size);
        int mask_lsbs = (mask << 2) - 1;
        int lsbs = (int)(btonb(vrank) & mask_lsbs);
        bool equal = lsbs == 0 || lsbs == mask_lsbs;
        if (!equal || ((mask << 1) >= size && r != root)) {
            c.world->send(r, partner, 0, recvbuf, nbytes);
            break;
        } else {
            c.world->recv(r, partner, 0, tmp.data(), nbytes);
            mpi_reduce_local(dt, tmp.data(), recvbuf, c.count);
        }
        mask <<= 1;
    }
}

// bine_reduce_redscat_gather_mpi (lib/libbine_coll_reduce.cc:1042-1152).
void reduce_redscat_gather(const Ctx& c, int r) {
    const int size = c.P, root = c.call->root, dt = c.call->dtype;
    if (root != 0) throw Unsupported("reduce-scatter+gather reduce asserts root == 0 (lib/libbine_coll_reduce.cc:1049)");
    const size_t nbytes = (size_t)c.count * c.es;
    std::vector<int> displs(size), counts(size);
    int cpr = (int)(c.count / size), rem = (int)(c.count % size);
    for (int i = 0; i < size; i++) {
        displs[i] = cpr * i + (i < rem ? i : rem);
        counts[i] = cpr + (i < rem ? 1 : 0);
    }
    std::vector<char> tmp(nbytes ? nbytes : 1), own;
    char* resbuf;
    if (r == root) {
        resbuf = out_of(c, r);
    } else {
        own.resize(nbytes ? nbytes : 1);
        resbuf = own.data();
    }
    std::memcpy(resbuf, in_of(c, r), nbytes);
    Buf R{resbuf, nbytes}, T{tmp.data(), nbytes};
    const char* where = "reduce-scatter+gather reduce (lib/libbine_coll_reduce.cc:1083-1140)";
    int mask = 0x1;
    int inverse_mask = 0x1 << (int)(std::ceil(std::log2(size)) - 1);
    int block_first_mask = ~(inverse_mask - 1);
    int remapped = (int)remap_rank(r, size);
    while (mask < size) {
        int partner = r % 2 == 0 ? mod(r + nbtob((mask << 1) - 1), size) : mod(r - nbtob((mask << 1) - 1), size);
        int sbf = (int)remap_rank(partner, size) & block_first_mask;
        int sbl = sbf + inverse_mask - 1;
        int scount = displs.at(sbl) - displs.at(sbf) + counts.at(sbl);
        int rbf = remapped & block_first_mask;
        int rbl = rbf + inverse_mask - 1;
        int rcount = displs.at(rbl) - displs.at(rbf) + counts.at(rbl);
        size_t sl = (size_t)scount * c.es, rl = (size_t)rcount * c.es;
        c.world->send(r, partner, 0, R.at((size_t)displs[sbf] * c.es, sl, where), sl);
        c.world->recv(r, partner, 0, T.at((size_t)displs[rbf] * c.es, rl, where), rl);
        mpi_reduce_local(dt, T.at((size_t)displs[rbf] * c.es, rl, where), R.at((size_t)displs[rbf] * c.es, rl, where),
                         rcount);
        mask <<= 1;
        inverse_mask >>= 1;
        block_first_mask >>= 1;
    }
    mask >>= 1;
    inverse_mask = 0x1;
    block_first_mask = ~0x0;
    int receiving_mask = 0x1 << (ffs(remapped) - 1);
    while (mask > 0) {
        int partner = r % 2 == 0 ? mod(r + nbtob((mask << 1) - 1), size) : mod(r - nbtob((mask << 1) - 1), size);
        if (inverse_mask & receiving_mask) {
            int sbf = remapped & block_first_mask;
            int sbl = sbf + inverse_mask - 1;
            int scount = displs.at(sbl) - displs.at(sbf) + counts.at(sbl);
            size_t sl = (size_t)scount * c.es;
            c.world->send(r, partner, 0, R.at((size_t)displs[sbf] * c.es, sl, where), sl);
            break;
        } else {
            int rbf = (int)remap_rank(partner, size) & block_first_mask;
            int rbl = rbf + inverse_mask - 1;
            int rcount = displs.at(rbl) - displs.at(rbf) + counts.at(rbl);
            size_t rl = (size_t)rcount * c.es;
            c.world->recv(r, partner, 0, R.at((size_t)displs[rbf] * c.es, rl, where), rl);
        }
        mask >>= 1;
        inverse_mask <<= 1;
        block_first_mask <<= 1;
    }
}

// ------------------------------------------------------------- alltoall
// bine_alltoall_mpi (lib/libbine_coll_alltoall.cc:411-540).
void alltoall_log(const Ctx& c, int r) {
    const int size = c.P;
    const size_t cb = (size_t)c.count * c.es;
    char* recvbuf = out_of(c, r);
    std::vector<char> tmp(cb * size + 1);
    std::vector<uint32_t> res(size), res_next(size);
    size_t nres = size;
    for (int i = 0; i < size; i++) res[i] = i;
    std::memcpy(tmp.data(), in_of(c, r), cb * size);
    int mask = 0x1;
    int inverse_mask = 0x1 << (int)(std::ceil(std::log2(size)) - 1);
    int block_first_mask = ~(inverse_mask - 1);
    while (mask < size) {
        int partner = r % 2 == 0 ? mod(r + nbtob((mask << 1) - 1), size) : mod(r - nbtob((mask << 1) - 1), size);
        size_t min_s = remap_rank(partner, size) & block_first_mask;
        size_t max_s = min_s + inverse_mask - 1;
        size_t recvd_cnt = 0, send_cnt = 0, off_send = 0, off_keep = 0, nnext = 0;
        for (int i = 0; i < size; i++) {
            uint32_t block = res[i % nres];
            uint32_t rb = remap_rank(block, size);
            size_t offset = (size_t)i * cb;
            if (rb >= min_s && rb <= max_s) {
                std::memcpy(recvbuf + off_send, tmp.data() + offset, cb);
                off_send += cb;
                send_cnt++;
            } else {
                if (offset != off_keep) std::memmove(tmp.data() + off_keep, tmp.data() + offset, cb);
                off_keep += cb;
                recvd_cnt++;
                res_next[nnext++] = block;
            }
        }
        if (recvd_cnt != (size_t)size / 2 || send_cnt != (size_t)size / 2)
            throw Unsupported("alltoall asserts block_recvd_cnt == size/2 (lib/libbine_coll_alltoall.cc:484)");
        nres /= 2;
        c.world->send(r, partner, 0, recvbuf, send_cnt * cb);
        c.world->recv(r, partner, 0, tmp.data() + (size / 2) * cb, send_cnt * cb);
        std::swap(res, res_next);
        mask <<= 1;
        inverse_mask >>= 1;
        block_first_mask >>= 1;
    }
    for (int i = 0; i < size; i++) {
        int rotated = r % 2 == 0 ? mod(i - r, size) : mod(r - i, size);
        int repr = in_range(rotated, (uint32_t)std::ceil(std::log2(size))) ? (int)btonb(rotated) : (int)btonb(rotated - size);
        int index = remap_distance_doubling((uint32_t)repr);
        std::memcpy(recvbuf + (size_t)i * cb, tmp.data() + (size_t)index * cb, cb);
    }
}

// bruck_alltoall (lib/libbine_coll_alltoall.cc:18-107): rotate, log2(P)
// packed exchanges with rank + k / rank - k, rotate back.  Any P.
void alltoall_bruck(const Ctx& c, int r) {
    const int size = c.P;
    const size_t cb = (size_t)c.count * c.es;
    const size_t half = (size_t)(size + 1) / 2;
    char* recvbuf = out_of(c, r);
    std::vector<char> tsend(cb * size + 1, 0), tbuf(cb * half + 1), trecv(cb * half + 1);
    for (int i = 0; i < size; i++) std::memcpy(tsend.data() + (size_t)mod(i - r, size) * cb, in_of(c, r) + i * cb, cb);
    for (int k = 1; k < size; k <<= 1) {
        std::vector<int> idx;
        for (int i = k; i < size; i++)
            if (i & k) idx.push_back(i);
        for (size_t j = 0; j < idx.size(); j++) std::memcpy(tbuf.data() + j * cb, tsend.data() + idx[j] * cb, cb);
        c.world->send(r, mod(r + k, size), 0, tbuf.data(), idx.size() * cb);
        c.world->recv(r, mod(r - k, size), 0, trecv.data(), idx.size() * cb);
        for (size_t j = 0; j < idx.size(); j++) std::memcpy(tsend.data() + idx[j] * cb, trecv.data() + j * cb, cb);
    }
    for (int i = 0; i < size; i++) std::memcpy(recvbuf + (size_t)mod(r - i, size) * cb, tsend.data() + i * cb, cb);
}

// --------------------------------------------------- bucket (ring) allreduce
// BineCommon::bucket_allreduce (lib/libbine_common.cc:2486-2663) with
// ringRedScatAG (lib/libbine_common.cc:2372-2484), the RING family's
// allreduce, restated over this file's message layer in place of uTofu puts.
// The reference ships whole segments, padding past the real count included
// (its padding is uninitialised and feeds no result); here every message and
// reduction covers the real elements only.
void ring_red_scat_ag(const Ctx& c, int r, char* data, long real, long off, long cnt, int nproc, int rank,
                      int recvfrom, int sendto, int redscat, int tag) {
    const long seg = cnt / nproc;  // cnt is a multiple of nproc (lib/libbine_common.cc:2376-2387)
    auto clip = [&](long o) { return std::max(0L, std::min(seg, real - o)); };
    std::vector<char> buffer((size_t)seg * c.es + 1);
    for (int i = 0; i < nproc - 1; i++) {
        int recv_chunk, send_chunk;
        if (redscat == 0) {
            recv_chunk = mod(rank - i - 2, nproc);
            send_chunk = mod(rank - i - 1, nproc);
        } else if (redscat == 1) {
            recv_chunk = (rank + 2 + i) % nproc;
            send_chunk = (rank + 1 + i) % nproc;
        } else if (redscat == 2) {
            recv_chunk = mod(rank - i - 1, nproc);
            send_chunk = mod(rank - i, nproc);
        } else {
            recv_chunk = (rank + i + 1) % nproc;
            send_chunk = (rank + i) % nproc;
        }
        const long so = off + send_chunk * seg, ro = off + recv_chunk * seg;
        if (clip(so) > 0) c.world->send(r, sendto, tag, data + so * c.es, (size_t)clip(so) * c.es);
        if (clip(ro) > 0) {
            if (redscat < 2) {
                c.world->recv(r, recvfrom, tag, buffer.data(), (size_t)clip(ro) * c.es);
                mpi_reduce_local(c.call->dtype, buffer.data(), data + ro * c.es, (size_t)clip(ro));
            } else {
                c.world->recv(r, recvfrom, tag, data + ro * c.es, (size_t)clip(ro) * c.es);
            }
        }
    }
}

void bucket_allreduce(const Ctx& c, int r) {
    const int D = c.topo.D, size = c.P;
    const long real = c.count;
    long count = real;
    while (count % ((2L * D) * size)) count += 1;
    std::vector<char> data((size_t)count * c.es + 1, 0);
    char* recvbuf = out_of(c, r);
    std::memcpy(data.data(), in_of(c, r), (size_t)real * c.es);
    int relcoord[3] = {0, 0, 0}, sendto[3], recvfrom[3];
    c.topo.coord(r, relcoord);
    for (int i = 0; i < D; i++) {
        int coord[3] = {relcoord[0], relcoord[1], relcoord[2]};
        coord[i] = (relcoord[i] + 1) % c.topo.dims[i];
        sendto[i] = c.topo.id(coord);
        coord[i] = (relcoord[i] - 1 + c.topo.dims[i]) % c.topo.dims[i];
        recvfrom[i] = c.topo.id(coord);
    }
    std::vector<long> data_size(D, count / (2 * D)), offsets(D, 0);
    std::vector<long> loop_off_l(D * D), loop_off_r(D * D), loop_size(D * D);
    for (int s = 0; s < D; s++) {
        // Every bucket's ring of this round (the reference runs them on
        // concurrent threads over disjoint ranges).
        std::vector<std::function<void()>> rings;
        for (int i = 0; i < D; i++) {
            const int d = (i + s) % D;
            const long ol = (2L * i) * (count / (2 * D)) + offsets[i], orr = (2L * i + 1) * (count / (2 * D)) + offsets[i];
            loop_off_l[s * D + i] = ol;
            loop_off_r[s * D + i] = orr;
            loop_size[s * D + i] = data_size[i];
            const long sz = data_size[i];
            const int n = c.topo.dims[d], rc = relcoord[d];
            rings.push_back([&, ol, sz, n, rc, d, i]() {
                ring_red_scat_ag(c, r, data.data(), real, ol, sz, n, rc, recvfrom[d], sendto[d], 0, 0x7000 + 2 * i);
            });
            rings.push_back([&, orr, sz, n, rc, d, i]() {
                ring_red_scat_ag(c, r, data.data(), real, orr, sz, n, rc, sendto[d], recvfrom[d], 1, 0x7000 + 2 * i + 1);
            });
            if (s != D - 1) {
                data_size[i] /= n;
                offsets[i] += relcoord[d] * data_size[i];
            }
        }
        for (auto& f : rings) f();
    }
    for (int s = D - 1; s >= 0; s--) {
        if (s == D - 1)
            for (int j = 0; j < 2 * D; j++) {
                const long o = j % 2 ? loop_off_r[s * D + j / 2] : loop_off_l[s * D + j / 2];
                if (o < real) {
                    long ct = loop_size[s * D + j / 2];
                    if (o + ct > real) ct = real - o;
                    std::memcpy(recvbuf + o * c.es, data.data() + o * c.es, (size_t)ct * c.es);
                }
            }
        for (int i = D - 1; i >= 0; i--) {
            const int d = (i + s) % D, n = c.topo.dims[d], rc = relcoord[d];
            const long sz = loop_size[s * D + i];
            ring_red_scat_ag(c, r, recvbuf, real, loop_off_l[s * D + i], sz, n, rc, recvfrom[d], sendto[d], 2,
                             0x7000 + 2 * D + 2 * i);
            ring_red_scat_ag(c, r, recvbuf, real, loop_off_r[s * D + i], sz, n, rc, sendto[d], recvfrom[d], 3,
                             0x7000 + 2 * D + 2 * i + 1);
        }
    }
}

// ----------------------------------------------------------- scatter/gather
// bine_scatter_mpi (lib/libbine_coll_scatter.cc:187-324).
void scatter_tree(const Ctx& c, int r) {
    const int size = c.P, root = c.call->root;
    const long sc = c.count;
    const int es = c.es;
    const char* where = "scatter (lib/libbine_coll_scatter.cc:270-316)";
    Buf recvbuf{out_of(c, r), c.recv_bytes};
    std::vector<char> tmpv;
    Buf sbuf{nullptr, 0}, rbuf{nullptr, 0};
    int halving_direction = r % 2 ? -1 : 1;
    if ((int)std::ceil(std::log2(size)) % 2 == 0) halving_direction *= -1;
    const int nb = (int)std::ceil(std::log2(size));
    size_t min_res, max_res;
    if (r % 2 == 0) {
        max_res = mod((int)((r + 0x55555555) & ((0x1 << nb) - 1)), size);
        min_res = mod((int)((r - (int)0xAAAAAAAA) & ((0x1 << nb) - 1)), size);
    } else {
        min_res = mod((int)((r - 0x55555555) & ((0x1 << nb) - 1)), size);
        max_res = mod((int)((r + (int)0xAAAAAAAA) & ((0x1 << nb) - 1)), size);
    }
    int mask = 0x1 << (nb - 1);
    int recvd = 0, sbuf_offset = r, is_leaf = 0;
    if (root == r) {
        recvd = 1;
        sbuf = Buf{(char*)in_of(c, r), c.send_bytes};
    }
    int vrank = mod(r - root, size);
    int vrank_nb = (int)btonb(vrank);
    while (mask > 0) {
        int partner = vrank_nb ^ ((mask << 1) - 1);
        partner = mod(nbtob(partner) + root, size);
        int mask_lsbs = (mask << 1) - 1;
        int lsbs = vrank_nb & mask_lsbs;
        bool equal = lsbs == 0 || lsbs == mask_lsbs;
        size_t top_start = min_res, top_end = mod((int)(min_res + mask - 1), size);
        size_t bottom_start = mod((int)(top_end + 1), size), bottom_end = max_res;
        size_t ss, se, rs_, re;
        if (halving_direction == 1) {
            ss = bottom_start;
            se = bottom_end;
            rs_ = top_start;
            re = top_end;
            max_res = mod((int)(max_res - mask), size);
        } else {
            ss = top_start;
            se = top_end;
            rs_ = bottom_start;
            re = bottom_end;
            min_res = mod((int)(min_res + mask), size);
        }
        if (recvd) {
            if (se >= ss) {
                size_t len = (size_t)sc * (se - ss + 1) * es;
                c.world->send(r, partner, 0, sbuf.at(ss * sc * es, len, where), len);
            } else {
                size_t l1 = (size_t)sc * ((size - 1) - ss + 1) * es, l2 = (size_t)sc * (se + 1) * es;
                c.world->send(r, partner, 0, sbuf.at(ss * sc * es, l1, where), l1);
                c.world->send(r, partner, 0, sbuf.at(0, l2, where), l2);
            }
        } else if (equal) {
            size_t num_blocks = mod((int)(re - rs_ + 1), size);
            if (rs_ == re) {
                rbuf = recvbuf;
                is_leaf = 1;
            } else {
                tmpv.assign((size_t)sc * num_blocks * es + 1, 0);
                sbuf = Buf{tmpv.data(), (size_t)sc * num_blocks * es};
                rbuf = sbuf;
                min_res = 0;
                max_res = num_blocks - 1;
                sbuf_offset = mod((int)(r - rs_), size);
            }
            if (re >= rs_) {
                size_t len = (size_t)sc * num_blocks * es;
                c.world->recv(r, partner, 0, rbuf.at(0, len, where), len);
            } else {
                size_t first = (size_t)sc * ((size - 1) - rs_ + 1) * es, second = (size_t)sc * (re + 1) * es;
                c.world->recv(r, partner, 0, rbuf.at(0, first, where), first);
                c.world->recv(r, partner, 0, rbuf.at(first, second, where), second);
            }
            recvd = 1;
        }
        mask >>= 1;
        halving_direction *= -1;
    }
    if (!is_leaf) {
        size_t len = (size_t)sc * es;
        std::memcpy(recvbuf.at(0, len, where), sbuf.at((size_t)sbuf_offset * len, len, where), len);
    }
}

// bine_gather_mpi (lib/libbine_coll_gather.cc:202-272).
void gather_tree(const Ctx& c, int r) {
    const int size = c.P, root = c.call->root;
    const long rc = c.count;
    const int es = c.es;
    const char* where = "gather (lib/libbine_coll_gather.cc:218-265)";
    std::vector<char> own;
    Buf recvbuf;
    if (r != root) {
        own.assign((size_t)rc * size * es + 1, 0);
        recvbuf = Buf{own.data(), (size_t)rc * size * es};
    } else {
        recvbuf = Buf{out_of(c, r), c.recv_bytes};
    }
    const size_t blk = (size_t)rc * es;
    std::memcpy(recvbuf.at((size_t)r * blk, blk, where), in_of(c, r), blk);
    size_t min_res = r, max_res = r;
    int vrank = mod(r - root, size);
    int ext = r % 2 ? -1 : 1;
    int mask = 0x1;
    while (mask < size) {
        int partner = (int)(btonb(vrank) ^ ((mask << 1) - 1));
        partner = mod(nbtob(partner) + root, size);
        int mask_lsbs = (mask << 2) - 1;
        int lsbs = (int)(btonb(vrank) & mask_lsbs);
        bool equal = lsbs == 0 || lsbs == mask_lsbs;
        if (!equal || ((mask << 1) >= size && r != root)) {
            if (max_res >= min_res) {
                size_t len = blk * (max_res - min_res + 1);
                c.world->send(r, partner, 0, recvbuf.at(min_res * blk, len, where), len);
            } else {
                size_t l1 = blk * ((size - 1) - min_res + 1), l2 = blk * (max_res + 1);
                c.world->send(r, partner, 0, recvbuf.at(min_res * blk, l1, where), l1);
                c.world->send(r, partner, 0, recvbuf.at(0, l2, where), l2);
            }
            break;
        } else {
            size_t rs_, re;
            if (ext == 1) {
                rs_ = mod((int)(max_res + 1), size);
                re = mod((int)(max_res + mask), size);
                max_res = re;
            } else {
                re = mod((int)(min_res - 1), size);
                rs_ = mod((int)(min_res - mask), size);
                min_res = rs_;
            }
            if (re >= rs_) {
                size_t len = blk * (re - rs_ + 1);
                c.world->recv(r, partner, 0, recvbuf.at(rs_ * blk, len, where), len);
            } else {
                size_t l1 = blk * ((size - 1) - rs_ + 1), l2 = blk * (re + 1);
                c.world->recv(r, partner, 0, recvbuf.at(rs_ * blk, l1, where), l1);
                c.world->recv(r, partner, 0, recvbuf.at(0, l2, where), l2);
            }
            ext = -ext;
        }
        mask <<= 1;
    }
}

// Default distance types per collective: lib/libbine.cc:65-72.
int default_distance(int coll) {
    switch (coll) {
    case OR_ALLGATHER: return OR_DIST_DECREASING;
    case OR_BCAST: return OR_DIST_DECREASING;
    case OR_GATHER: return OR_DIST_DECREASING;
    default: return OR_DIST_INCREASING;
    }
}

}  // namespace

extern "C" {

const char* oracle_last_error(void) { return g_last_error.c_str(); }

int oracle_buffer_counts(const oracle_call_t* call, long* sc, long* rc) {
    const long c = call->count, P = call->nranks;
    switch (call->coll) {
    case OR_ALLREDUCE:
    case OR_BCAST:
    case OR_REDUCE: *sc = c; *rc = c; return OR_OK;
    case OR_REDUCE_SCATTER:
    case OR_SCATTER: *sc = c * P; *rc = c; return OR_OK;
    case OR_ALLGATHER:
    case OR_GATHER: *sc = c; *rc = c * P; return OR_OK;
    case OR_ALLTOALL: *sc = c * P; *rc = c * P; return OR_OK;
    default: return OR_ERR_ARG;
    }
}

int oracle_run(const oracle_call_t* call, const void* in, void* out, oracle_msg_t* msgs, size_t msg_cap,
               size_t* n_msgs) {
    g_last_error.clear();
    if (n_msgs) *n_msgs = 0;
    long sc, rc;
    if (!call || oracle_buffer_counts(call, &sc, &rc) != OR_OK || call->nranks < 1 || call->count < 0) {
        g_last_error = "invalid arguments";
        return OR_ERR_ARG;
    }
    Ctx c;
    c.call = call;
    c.P = call->nranks;
    c.es = dtype_size(call->dtype);
    if (c.es < 0) {
        g_last_error = "invalid dtype";
        return OR_ERR_ARG;
    }
    int dims1[1] = {call->nranks};
    c.topo = call->ndims > 0 ? Topo(call->ndims, call->dims) : Topo(1, dims1);
    if (c.topo.size != c.P || call->ndims > 3) {
        g_last_error = "dims do not multiply to nranks";
        return OR_ERR_ARG;
    }
    if (call->ports < 1 || call->ports > 6) {
        g_last_error = "ports must be in [1, 6] (lib/libbine.cc:98)";
        return OR_ERR_ARG;
    }
    c.count = call->count;
    c.ports = call->ports;
    c.family = call->family == OR_FAMILY_RECDOUB ? OR_FAMILY_RECDOUB : OR_FAMILY_BINE;
    c.dist = call->distance < 0 ? default_distance(call->coll) : call->distance;
    c.in = (const char*)in;
    c.out = (char*)out;
    c.send_bytes = (size_t)sc * c.es;
    c.recv_bytes = (size_t)rc * c.es;
    std::memset(out, 0, c.recv_bytes * c.P);
    World world(c.P, msgs != nullptr);
    c.world = &world;

    try {
        std::function<void(int)> body;
        std::vector<std::vector<BlockInfo>> bi;
        std::vector<std::vector<BitmapCalc*>> calc;
        std::vector<std::unique_ptr<BitmapCalc>> owned;
        Topo virt;
        bool all_p2 = true;
        switch (call->coll) {
        case OR_ALLREDUCE: {
            if (call->family == OR_FAMILY_RING) {
                body = [&](int r) { bucket_allreduce(c, r); };
            } else if (call->algo == OR_AR_L) {
                int vd[3];
                for (int i = 0; i < c.topo.D; i++) {
                    int st = ceil_log2(c.topo.dims[i]);
                    if (!is_p2(c.topo.dims[i])) {
                        all_p2 = false;
                        vd[i] = (int)std::pow(2, st - 1);
                    } else {
                        vd[i] = c.topo.dims[i];
                    }
                }
                virt = Topo(c.topo.D, vd);
                body = [&](int r) { allreduce_l(c, r, virt, all_p2); };
            } else if (call->algo == OR_AR_B || call->algo == OR_AR_B_COALESCE || call->algo == OR_AR_B_CONT) {
                if (c.dist != OR_DIST_INCREASING)
                    throw Unsupported("B allreduce asserts INCREASING distance (lib/libbine.cc:1035)");
                if (c.count < (long)c.ports * c.P)
                    throw Unsupported("B allreduce asserts count >= ports*size (lib/libbine.cc:1036)");
                if (call->algo == OR_AR_B_CONT && !is_p2(c.P))
                    throw Unsupported("B_CONT asserts a power-of-two size (lib/libbine_common.cc:1250)");
                bi = blocks_port_then_block(c.count, c.P, c.ports, c.es);
                bool remap = call->algo == OR_AR_B_CONT && is_p2(c.P);
                calc.assign(c.ports, std::vector<BitmapCalc*>(c.P));
                for (int p = 0; p < c.ports; p++)
                    for (int r = 0; r < c.P; r++) {
                        owned.emplace_back(new BitmapCalc(r, c.topo, p, bi, remap, c.family));
                        calc[p][r] = owned.back().get();
                    }
                body = [&](int r) { allreduce_b(c, r, calc, bi); };
            } else {
                throw Unsupported("allreduce variant not in the MPI layer");
            }
            break;
        }
        case OR_REDUCE_SCATTER: {
            if (c.count * c.P < (long)c.ports * c.P)
                throw Unsupported("reduce_scatter asserts count >= ports*size (lib/libbine.cc:1078)");
            if (!is_p2(c.P))
                throw Unsupported("contiguous reduce_scatter halves size/2^(s+1) blocks per step and returns "
                                  "wrong data unless size is a power of two (lib/libbine_coll_reduce_scatter.cc:733)");
            if (c.ports > 1)
                throw Unsupported("contiguous reduce_scatter writes recvbuf + tmpbuf_size/ports*port, past the end of "
                                  "recvbuf, for ports > 1 (lib/libbine_coll_reduce_scatter.cc:710, 742)");
            bi = blocks_block_then_port((size_t)c.count, c.P, c.ports, c.es);
            body = [&](int r) { reduce_scatter_cont(c, r, bi); };
            break;
        }
        case OR_ALLGATHER: {
            if (call->algo == OR_AG_BLOCKS) {
                body = [&](int r) { allgather_blocks(c, r); };
            } else if (call->algo == OR_AG_CONT_SEND) {
                if (c.ports != 1) throw Unsupported("CONT_SEND allgather asserts one port (lib/libbine_coll_allgather.cc:501)");
                body = [&](int r) { allgather_cont_send(c, r); };
            } else {
                bi = blocks_block_then_port((size_t)c.count, c.P, c.ports, c.es);
                body = [&](int r) { allgather_cont_permute(c, r, bi); };
            }
            break;
        }
        case OR_BCAST:
            if (call->algo == OR_BC_SCATTER_ALLGATHER) {
                if (c.dist != OR_DIST_INCREASING && call->distance >= 0)
                    throw Unsupported("scatter-allgather bcast asserts INCREASING distance (lib/libbine.cc:1267)");
                body = [&](int r) { bcast_scatter_allgather(c, r); };
            } else {
                body = [&](int r) { bcast_tree(c, r); };
            }
            break;
        case OR_REDUCE:
            if (call->algo == OR_RD_REDUCE_SCATTER_GATHER)
                body = [&](int r) { reduce_redscat_gather(c, r); };
            else
                body = [&](int r) { reduce_tree(c, r); };
            break;
        case OR_ALLTOALL:
            if (call->family == OR_FAMILY_BRUCK) body = [&](int r) { alltoall_bruck(c, r); };
            else body = [&](int r) { alltoall_log(c, r); };
            break;
        case OR_SCATTER:
            if (c.count < c.ports) throw Unsupported("scatter asserts recvcount >= ports (lib/libbine.cc:1331)");
            body = [&](int r) { scatter_tree(c, r); };
            break;
        case OR_GATHER:
            if (c.count < c.ports) throw Unsupported("gather asserts recvcount >= ports (lib/libbine.cc:1395)");
            body = [&](int r) { gather_tree(c, r); };
            break;
        default: throw Unsupported("unknown collective");
        }
        world.run(body);
    } catch (Unsupported& e) {
        g_last_error = e.what();
        return OR_ERR_REFERENCE_UNSUPPORTED;
    } catch (std::exception& e) {
        g_last_error = std::string("internal: ") + e.what();
        return OR_ERR_INTERNAL;
    }
    if (!world.error().empty()) {
        g_last_error = world.error();
        return world.internal_error() ? OR_ERR_INTERNAL : OR_ERR_REFERENCE_UNSUPPORTED;
    }
    if (msgs) {
        const auto& m = world.msgs();
        if (n_msgs) *n_msgs = m.size();
        for (size_t i = 0; i < m.size() && i < msg_cap; i++) msgs[i] = m[i];
    }
    return OR_OK;
}

uint32_t oracle_remap_rank(uint32_t nranks, uint32_t rank) {
    try {
        return remap_rank(rank, nranks);
    } catch (std::exception& e) {
        g_last_error = e.what();
        return UINT32_MAX;
    }
}

uint32_t oracle_get_nu(uint32_t rank, uint32_t nranks) {
    try {
        return get_nu(rank, nranks);
    } catch (std::exception& e) {
        g_last_error = e.what();
        return UINT32_MAX;
    }
}

int oracle_remap_distance_doubling(uint32_t num) { return remap_distance_doubling(num); }

int oracle_compute_peers(int rank, int port, int family, int ndims, const int* dims, int* peers_out) {
    Topo t(ndims, dims);
    std::vector<int> p = compute_peers(rank, port, family, t);
    std::copy(p.begin(), p.end(), peers_out);
    return t.num_steps;
}

int oracle_get_tree(int root, int port, int family, int distance, int ndims, const int* dims, uint32_t* parent,
                    uint32_t* reached_at_step, uint32_t* remapped_ranks, uint32_t* remapped_ranks_max,
                    uint32_t* subtree_roots) {
    try {
        Topo t(ndims, dims);
        Tree tr = get_tree(root, port, family, distance, t);
        std::copy(tr.parent.begin(), tr.parent.end(), parent);
        std::copy(tr.reached_at_step.begin(), tr.reached_at_step.end(), reached_at_step);
        std::copy(tr.remapped_ranks.begin(), tr.remapped_ranks.end(), remapped_ranks);
        std::copy(tr.remapped_ranks_max.begin(), tr.remapped_ranks_max.end(), remapped_ranks_max);
        std::copy(tr.subtree_roots.begin(), tr.subtree_roots.end(), subtree_roots);
        return OR_OK;
    } catch (std::exception& e) {
        g_last_error = e.what();
        return OR_ERR_REFERENCE_UNSUPPORTED;
    }
}

int oracle_block_step(int rank, int port, int family, int ndims, const int* dims, uint32_t* block_step_out) {
    Topo t(ndims, dims);
    std::vector<std::vector<BlockInfo>> bi(port + 1, std::vector<BlockInfo>(t.size, BlockInfo{0, 1}));
    BitmapCalc calc(rank, t, port, bi, false, family);
    std::copy(calc.block_step().begin(), calc.block_step().end(), block_step_out);
    return t.num_steps;
}

}  // extern "C"

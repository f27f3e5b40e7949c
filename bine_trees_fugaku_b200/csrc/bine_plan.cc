// Host planner: schedule IR generators for the reference's MPI-layer Bine
// collectives, the symbolic executor that extracts exact reduction trees,
// and torus link accounting.  See bine_plan.h.
#include "bine_plan.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <deque>
#include <functional>
#include <map>
#include <set>
#include <stdexcept>
#include <tuple>

namespace bine {

namespace {

// Workspace area for messages received one or more steps after they were
// sent; folded into kBufTmp when a schedule is finished.
constexpr uint8_t kBufCarry = 3;

struct PlanError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// ------------------------------------------------------------ rank trees
// Binomial tree of `root` for one port (reference: get_tree,
// lib/libbine_coll.cc:334-389).  The tree is explored depth-first from the
// root along steps i, i+1, ...; a node's parent is the first explorer that
// reaches it at the earliest step.  remapped[r] numbers the nodes in
// post-order from size-1 down, so every subtree owns a contiguous range.
struct RankTree {
    std::vector<uint32_t> parent, reached, remapped;
};

class TreeBuilder {
  public:
    TreeBuilder(const Torus& t, int port, int family, int dist) : t_(t), port_(port), family_(family), dist_(dist) {
        step_dims(t, port, sd_);
    }
    RankTree build(int root) {
        RankTree tr;
        tr.parent.assign(t_.size, UINT32_MAX);
        tr.reached.assign(t_.size, (uint32_t)t_.num_steps);
        tr.remapped.assign(t_.size, 0);
        explore(root, 0, tr);
        tr.parent[root] = UINT32_MAX;
        tr.reached[root] = 0;
        uint32_t next = (uint32_t)t_.size - 1;
        number(root, 0, tr, &next);
        if (next != UINT32_MAX) throw PlanError("rank tree does not reach every rank (lib/libbine_coll.cc:380)");
        return tr;
    }

  private:
    int real_step(int i) const { return dist_ == kDecreasing ? t_.num_steps - 1 - i : i; }
    void explore(int node, int step, RankTree& tr) {
        for (int i = step; i < t_.num_steps; i++) {
            int peer = step_peer_rank(t_, sd_, real_step(i), port_, family_, node);
            if (tr.parent[peer] == UINT32_MAX || (uint32_t)i < tr.reached[peer]) {
                tr.parent[peer] = (uint32_t)node;
                tr.reached[peer] = (uint32_t)i;
            }
            explore(peer, i + 1, tr);
        }
    }
    void number(int node, int step, RankTree& tr, uint32_t* next) {
        for (int i = step; i < t_.num_steps; i++) {
            int peer = step_peer_rank(t_, sd_, real_step(i), port_, family_, node);
            if (tr.parent[peer] == (uint32_t)node) number(peer, i + 1, tr, next);
        }
        tr.remapped[node] = *next;
        (*next)--;
    }
    const Torus& t_;
    int port_, family_, dist_;
    StepDim sd_[kMaxSteps];
};

// Peers of `rank` at every step of a port (compute_peers,
// lib/libbine_coll.cc:443-504): always relative to the rank's own
// coordinates, dimensions visited as step_dims() orders them.
std::vector<int> peers_of(const Torus& t, int rank, int port, int family) {
    StepDim sd[kMaxSteps];
    step_dims(t, port, sd);
    std::vector<int> p(t.num_steps);
    for (int s = 0; s < t.num_steps; s++) p[s] = step_peer_rank(t, sd, s, port, family, rank);
    return p;
}

// ------------------------------------------------- reduce-scatter bitmaps
// block_step[b]: the step at which rank `rank` sends block b during the
// bitmap reduce-scatter (the latest first step of any path rank -> b along
// increasing steps; BineBitmapCalculator, lib/libbine_common.cc:1491-1510,
// 1995-2047).  A rank never sends its own block.
class BlockSteps {
  public:
    BlockSteps(const Torus& t, int port, int family) : t_(t), port_(port), family_(family) {
        step_dims(t, port, sd_);
    }
    std::vector<uint32_t> of_rank(int rank) const {
        std::vector<uint32_t> bs(t_.size, (uint32_t)t_.num_steps);
        for (int i = 0; i < t_.num_steps; i++) visit(step_peer_rank(t_, sd_, i, port_, family_, rank), i, i, bs);
        bs[rank] = (uint32_t)t_.num_steps;
        return bs;
    }
    // What `peer` sends at step s, seen from steps >= s only
    // (compute_next_bitmaps, lib/libbine_common.cc:1553-1570).
    std::vector<uint32_t> of_peer_from(int peer, int s) const {
        std::vector<uint32_t> bs(t_.size, (uint32_t)t_.num_steps);
        for (int j = s; j < t_.num_steps; j++) visit(step_peer_rank(t_, sd_, j, port_, family_, peer), j, j, bs);
        bs[peer] = (uint32_t)t_.num_steps;
        return bs;
    }

  private:
    void visit(int node, int start, int step, std::vector<uint32_t>& bs) const {
        if (step >= t_.num_steps) return;
        for (int i = step + 1; i < t_.num_steps; i++)
            visit(step_peer_rank(t_, sd_, i, port_, family_, node), start, i, bs);
        if (bs[node] == (uint32_t)t_.num_steps || (uint32_t)start > bs[node]) bs[node] = (uint32_t)start;
    }
    const Torus& t_;
    int port_, family_;
    StepDim sd_[kMaxSteps];
};

// Post-order index of `rank` in the increasing-step tree explored from rank
// 0 (the dfs of lib/libbine_common.cc:1981-1993, used by B_CONT).
uint32_t postorder_index(const Torus& t, int port, int family, int rank) {
    StepDim sd[kMaxSteps];
    step_dims(t, port, sd);
    uint32_t counter = (uint32_t)t.size - 1;
    bool found = false;
    std::function<void(int, int)> dfs = [&](int node, int step) {
        for (int i = step; i < t.num_steps; i++) dfs(step_peer_rank(t, sd, i, port, family, node), i + 1);
        if (found) counter--;
        if (node == rank) found = true;
    };
    dfs(0, 0);
    return counter;
}

struct Block {
    int64_t off;  // elements
    int64_t n;
};

// Allreduce partition: by port, then P blocks (lib/libbine.cc:971-1010).
std::vector<std::vector<Block>> blocks_by_port(int64_t count, int P, int ports) {
    std::vector<std::vector<Block>> bi(ports, std::vector<Block>(P));
    int64_t so_far = 0;
    for (int p = 0; p < ports; p++) {
        int64_t cp = count / ports + (p < count % ports ? 1 : 0);
        int64_t base = so_far;
        so_far += cp;
        int64_t b = 0;
        for (int i = 0; i < P; i++) {
            int64_t cb = cp / P + (i < cp % P ? 1 : 0);
            bi[p][i] = Block{base + b, cb};
            b += cb;
        }
    }
    return bi;
}
// Reduce-scatter / allgather partition: by block, then port
// (lib/libbine.cc:1086-1114, 1185-1206).
std::vector<std::vector<Block>> blocks_by_block(int64_t per_block, int P, int ports) {
    std::vector<std::vector<Block>> bi(ports, std::vector<Block>(P));
    for (int i = 0; i < P; i++) {
        int64_t b = 0;
        for (int p = 0; p < ports; p++) {
            int64_t cp = per_block / ports + (p < per_block % ports ? 1 : 0);
            bi[p][i] = Block{(int64_t)i * per_block + b, cp};
            b += cp;
        }
    }
    return bi;
}

// ---------------------------------------------------------------- builder
// Collects, per level, the sends and receives each rank issues (in program
// order, as the reference's MPI calls), matches them FIFO per
// (src, dst, tag) like MPI, and emits moves with value semantics (every read
// sees the state before the level).  Reads of a region that another move of
// the same level overwrites are first staged into the reader's workspace in
// an extra level, so each emitted level is free of hazards.
class Builder {
  public:
    Builder(int P, int64_t tmp_base) : P_(P), stage_base_(tmp_base) {}

    void begin() {
        recvs_.clear();
        copies_.clear();
        adds_.clear();
    }
    void send(int src, int dst, int tag, Region from, int64_t n) {
        if (dst < 0 || dst >= P_) throw PlanError("send to invalid rank");
        sends_[key(src, dst, tag)].push_back(Pending{from, n, false});
    }
    // into = message (+ addend, read before the level).
    void recv(int dst, int src, int tag, Region into, int64_t n, const Region* addend = nullptr) {
        Recv r;
        r.dst = dst;
        r.src = src;
        r.tag = tag;
        r.into = into;
        r.n = n;
        r.has_addend = addend != nullptr;
        if (addend) r.addend = *addend;
        recvs_.push_back(r);
    }
    void copy(Region to, Region from, int64_t n) {
        if (n > 0) copies_.push_back(Move{to, from, from, n, 0});
    }
    void add(Region to, Region a, Region b, int64_t n) {
        if (n > 0) adds_.push_back(Move{to, a, b, n, 1});
    }

    void end(Schedule* s) {
        std::vector<Move> moves = copies_;
        moves.insert(moves.end(), adds_.begin(), adds_.end());
        for (const Recv& r : recvs_) {
            auto it = sends_.find(key(r.src, r.dst, r.tag));
            if (it == sends_.end() || it->second.empty())
                throw PlanError("rank " + std::to_string(r.dst) + " waits for a message rank " + std::to_string(r.src) +
                                " never sends in this step (the reference deadlocks)");
            Pending snd = it->second.front();
            it->second.pop_front();
            if (snd.n > r.n)
                throw PlanError("rank " + std::to_string(r.dst) + " receives " + std::to_string(snd.n) +
                                " elements into room for " + std::to_string(r.n) + " (MPI_ERR_TRUNCATE)");
            if (snd.n > 0) {
                if (r.has_addend)
                    moves.push_back(Move{r.into, snd.from, r.addend, snd.n, 1});
                else
                    moves.push_back(Move{r.into, snd.from, snd.from, snd.n, 0});
            }
            if (!snd.carried) s->messages.push_back(Message{(int32_t)s->levels.size(), r.src, r.dst, snd.n});
        }
        // A send whose receive comes in a later step (ranks out of step, as
        // the rooted trees are at some non-power-of-two sizes): its payload
        // is copied now into the receiver's carry area, the message counted
        // now, and the later receive reads the copy.
        for (auto& kv : sends_) {
            const int dst = (int)((kv.first >> 16) & 0xFFFFFF);
            const int src = (int)(kv.first >> 40);
            for (Pending& p : kv.second) {
                if (p.carried) continue;
                Region c{dst, kBufCarry, carry_cursor_[dst]};
                carry_cursor_[dst] += p.n;
                carry_max_ = std::max(carry_max_, carry_cursor_[dst]);
                if (p.n > 0) moves.push_back(Move{c, p.from, p.from, p.n, 0});
                s->messages.push_back(Message{(int32_t)s->levels.size(), src, dst, p.n});
                p.from = c;
                p.carried = true;
            }
        }
        emit(s, moves);
    }

    int64_t stage_elems() const { return stage_max_; }

    // Places the carry area after the staging area and sets the workspace
    // size.  A message nobody receives stays counted (eager MPI delivers it
    // and the reference finishes with it pending, as the binomial bcast does
    // at some non-power-of-two sizes).
    void finish(Schedule* s) {
        const int64_t carry_base = stage_base_ + stage_max_;
        for (auto& lvl : s->levels)
            for (Move& m : lvl)
                for (Region* r : {&m.dst, &m.a, &m.b})
                    if (r->buf == kBufCarry) {
                        r->buf = kBufTmp;
                        r->off += carry_base;
                    }
        s->tmp_elems = carry_base + carry_max_;
    }

  private:
    struct Pending {
        Region from;
        int64_t n;
        bool carried;  // staged into the receiver's carry area at an earlier step
    };
    struct Recv {
        int dst, src, tag;
        Region into, addend;
        int64_t n;
        bool has_addend;
    };
    static uint64_t key(int src, int dst, int tag) {
        return ((uint64_t)(uint32_t)src << 40) ^ ((uint64_t)(uint32_t)dst << 16) ^ (uint64_t)(uint16_t)tag;
    }

    struct Interval {
        int64_t lo, hi;
        size_t move;
    };
    static uint64_t bkey(const Region& r) { return ((uint64_t)(uint32_t)r.rank << 8) | r.buf; }

    void emit(Schedule* s, std::vector<Move>& moves) {
        if (moves.empty()) return;
        // Index writes per (rank, buffer).
        std::unordered_map<uint64_t, std::vector<Interval>> writes;
        for (size_t i = 0; i < moves.size(); i++)
            writes[bkey(moves[i].dst)].push_back(Interval{moves[i].dst.off, moves[i].dst.off + moves[i].n, i});
        for (auto& kv : writes) {
            auto& v = kv.second;
            std::sort(v.begin(), v.end(), [](const Interval& x, const Interval& y) { return x.lo < y.lo; });
            for (size_t i = 1; i < v.size(); i++)
                if (v[i].lo < v[i - 1].hi) throw PlanError("two moves write the same elements in one step");
        }
        auto conflicts = [&](const Region& r, int64_t n, size_t self, const Region& own_dst) {
            auto it = writes.find(bkey(r));
            if (it == writes.end()) return false;
            const auto& v = it->second;
            // first interval with hi > r.off
            size_t lo = 0, hi = v.size();
            while (lo < hi) {
                size_t mid = (lo + hi) / 2;
                if (v[mid].hi <= r.off) lo = mid + 1;
                else hi = mid;
            }
            for (size_t i = lo; i < v.size() && v[i].lo < r.off + n; i++) {
                if (v[i].move == self) {
                    // Reading the elements this move itself writes, index for
                    // index, is an in-place update and safe.
                    if (r.rank == own_dst.rank && r.buf == own_dst.buf && r.off == own_dst.off) continue;
                    return true;
                }
                return true;
            }
            return false;
        };
        std::vector<Move> stage;
        std::unordered_map<int, int64_t> cursor;
        for (size_t i = 0; i < moves.size(); i++) {
            Move& m = moves[i];
            const int nsrc = m.add ? 2 : 1;
            for (int which = 0; which < nsrc; which++) {
                Region& src = which == 0 ? m.a : m.b;
                if (!conflicts(src, m.n, i, m.dst)) continue;
                int64_t& cur = cursor[m.dst.rank];
                Region st{m.dst.rank, kBufTmp, stage_base_ + cur};
                cur += m.n;
                stage.push_back(Move{st, src, src, m.n, 0});
                src = st;
            }
        }
        for (auto& kv : cursor) stage_max_ = std::max(stage_max_, kv.second);
        if (!stage.empty()) s->levels.push_back(std::move(stage));
        s->levels.push_back(std::move(moves));
    }

    int P_;
    int64_t stage_base_;
    int64_t stage_max_ = 0;
    std::unordered_map<int, int64_t> carry_cursor_;
    int64_t carry_max_ = 0;
    std::map<uint64_t, std::deque<Pending>> sends_;
    std::vector<Recv> recvs_;
    std::vector<Move> copies_, adds_;
};

Region R(int rank, uint8_t buf, int64_t off) { return Region{rank, buf, off}; }

// Tags used by the generators (the reference's TAG_* constants).
constexpr int kTagRS = 0x7FFF - 6 * 1;
constexpr int kTagAG = 0x7FFF - 6 * 2;
constexpr int kTagAR = 0x7FFF - 6 * 3;

// ------------------------------------------------------------ generators
struct Gen {
    const Torus& t;
    const PlanKey& k;
    int P;
    int S;
    Schedule* s;
};

// Bandwidth-optimal allreduce: bitmap reduce-scatter then allgather
// (bine_coll_b + bine_coll_step_b/_coalesce/_cont,
// lib/libbine_common.cc:930-1257, 1631-1735).
void gen_allreduce_b(const Gen& g) {
    const int P = g.P, S = g.S, ports = g.k.ports;
    const int64_t count = g.k.count;
    if (g.k.distance != kIncreasing) throw PlanError("B allreduce asserts INCREASING distance (lib/libbine.cc:1035)");
    if (count < (int64_t)ports * P) throw PlanError("B allreduce asserts count >= ports*size (lib/libbine.cc:1036)");
    const bool cont = g.k.variant == kArBCont;
    if (cont && !is_pow2(P)) throw PlanError("B_CONT asserts a power-of-two size (lib/libbine_common.cc:1250)");
    auto bi = blocks_by_port(count, P, ports);
    g.s->send_elems = g.s->recv_elems = count;

    // Per port and rank: peers, and either bitmaps or contiguous chunks.
    struct PR {
        std::vector<int> peers;
        std::vector<std::vector<char>> sbm, rbm;  // [step][block]
        std::vector<std::array<int64_t, 4>> chunk;  // send_off, send_n, recv_off, recv_n
    };
    std::vector<std::vector<PR>> pr(ports, std::vector<PR>(P));
    for (int p = 0; p < ports; p++) {
        BlockSteps bsc(g.t, p, g.k.family);
        for (int r = 0; r < P; r++) {
            PR& x = pr[p][r];
            x.peers = peers_of(g.t, r, p, g.k.family);
            if (cont) {
                uint32_t rr = postorder_index(g.t, p, g.k.family, r);
                size_t min_r = 0, max_r = P, min_s, max_s;
                for (int st = 0; st < S; st++) {
                    min_s = min_r;
                    max_s = max_r;
                    size_t mid = (min_r + max_r + 1) / 2;
                    if (rr < mid) {
                        min_s = mid;
                        max_r = mid;
                    } else {
                        max_s = mid;
                        min_r = mid;
                    }
                    int64_t sn = 0, rn = 0;
                    for (size_t i = min_s; i < max_s; i++) sn += bi[p][i].n;
                    for (size_t i = min_r; i < max_r; i++) rn += bi[p][i].n;
                    x.chunk.push_back({bi[p][min_s].off, sn, bi[p][min_r].off, rn});
                }
            } else {
                std::vector<uint32_t> bs = bsc.of_rank(r);
                x.sbm.assign(S, std::vector<char>(P, 0));
                x.rbm.assign(S, std::vector<char>(P, 0));
                for (int st = 0; st < S; st++) {
                    for (int i = 0; i < P; i++) x.sbm[st][i] = bs[i] == (uint32_t)st;
                    std::vector<uint32_t> pb = bsc.of_peer_from(x.peers[st], st);
                    for (int i = 0; i < P; i++) x.rbm[st][i] = pb[i] == (uint32_t)st;
                }
            }
        }
    }
    Builder b(P, 0);
    b.begin();
    for (int r = 0; r < P; r++) b.copy(R(r, kBufRecv, 0), R(r, kBufSend, 0), count);
    b.end(g.s);
    for (int phase = 0; phase < 2; phase++) {
        const bool rs = phase == 0;
        for (int st = 0; st < S; st++) {
            b.begin();
            const int bst = rs ? st : S - st - 1;
            for (int r = 0; r < P; r++) {
                for (int p = 0; p < ports; p++) {
                    const PR& x = pr[p][r];
                    const int peer = x.peers[bst];
                    const int tag = (rs ? kTagRS : kTagAG) + p;
                    auto post_recv = [&](int64_t off, int64_t n) {
                        Region into = R(r, kBufRecv, off);
                        if (rs)
                            b.recv(r, peer, tag, into, n, &into);
                        else
                            b.recv(r, peer, tag, into, n);
                    };
                    if (cont) {
                        const auto& c = x.chunk[bst];
                        int64_t so = rs ? c[0] : c[2], sn = rs ? c[1] : c[3];
                        int64_t ro = rs ? c[2] : c[0], rn = rs ? c[3] : c[1];
                        b.send(r, peer, tag, R(r, kBufRecv, so), sn);
                        post_recv(ro, rn);
                        continue;
                    }
                    const auto& sb = rs ? x.sbm[bst] : x.rbm[bst];
                    const auto& rb = rs ? x.rbm[bst] : x.sbm[bst];
                    if (g.k.variant == kArB) {
                        for (int i = 0; i < P; i++) {
                            if (sb[i]) b.send(r, peer, tag, R(r, kBufRecv, bi[p][i].off), bi[p][i].n);
                            if (rb[i]) post_recv(bi[p][i].off, bi[p][i].n);
                        }
                    } else {  // B_COALESCE: runs of consecutive blocks
                        for (int pass = 0; pass < 2; pass++) {
                            const auto& bm = pass == 0 ? sb : rb;
                            int i = 0;
                            while (i < P) {
                                if (!bm[i]) {
                                    i++;
                                    continue;
                                }
                                int64_t off = bi[p][i].off, n = 0;
                                while (i < P && bm[i]) n += bi[p][i++].n;
                                if (pass == 0)
                                    b.send(r, peer, tag, R(r, kBufRecv, off), n);
                                else
                                    post_recv(off, n);
                            }
                        }
                    }
                }
            }
            b.end(g.s);
        }
    }
    b.finish(g.s);
}

// Latency-optimal allreduce: full-vector butterfly on the largest
// power-of-two sub-torus, with the extra ranks folded in before and out after
// (bine_coll_l_mpi, shrink/enlarge; lib/libbine_common.cc:269-353, 733-846).
void gen_allreduce_l(const Gen& g) {
    const Torus& real = g.t;
    const int P = g.P, ports = g.k.ports;
    const int64_t count = g.k.count;
    g.s->send_elems = g.s->recv_elems = count;
    int vd[kMaxDims];
    bool all_p2 = true;
    for (int i = 0; i < real.ndims; i++) {
        if (is_pow2(real.dims[i])) {
            vd[i] = real.dims[i];
        } else {
            all_p2 = false;
            vd[i] = 1 << (ceil_log2(real.dims[i]) - 1);
        }
    }
    Torus virt;
    virt.init(real.ndims, vd);
    // Per-rank progress through shrink: idle flag and first_copy_done.
    std::vector<int> idle(P, 0), first(P, 0);
    std::vector<std::array<int, kMaxDims>> coord(P);
    for (int r = 0; r < P; r++) {
        coord[r] = {0, 0, 0};
        real.coords(r, coord[r].data());
    }
    Builder b(P, 0);
    if (!all_p2) {
        for (int d = 0; d < real.ndims; d++) {
            if (is_pow2(real.dims[d])) continue;
            b.begin();
            const int extra = real.dims[d] - virt.dims[d];
            std::vector<int> newly_first;
            for (int r = 0; r < P; r++) {
                if (idle[r]) continue;
                int cp[kMaxDims] = {coord[r][0], coord[r][1], coord[r][2]};
                if (coord[r][d] >= virt.dims[d]) {
                    cp[d] = coord[r][d] - extra;
                    b.send(r, real.id(cp), kTagAR, first[r] ? R(r, kBufRecv, 0) : R(r, kBufSend, 0), count);
                    idle[r] = 1;
                } else if (coord[r][d] + extra >= virt.dims[d]) {
                    cp[d] = coord[r][d] + extra;
                    // recvbuf = aggbuf + received, aggbuf = sendbuf the first
                    // time, the previous recvbuf afterwards.
                    Region into = R(r, kBufRecv, 0);
                    Region agg = first[r] ? R(r, kBufRecv, 0) : R(r, kBufSend, 0);
                    b.recv(r, real.id(cp), kTagAR, into, count, &agg);
                    newly_first.push_back(r);
                }
            }
            b.end(g.s);
            for (int r : newly_first) first[r] = 1;
        }
    }
    std::vector<std::vector<int>> vpeers(P);
    for (int st = 0; st < virt.num_steps; st++) {
        b.begin();
        for (int r = 0; r < P; r++) {
            if (idle[r]) continue;
            int rv = virt.id(coord[r].data());
            int64_t so_far = 0;
            for (int p = 0; p < ports; p++) {
                std::vector<int> vp = peers_of(virt, rv, p, g.k.family);
                int vc[kMaxDims];
                virt.coords(vp[st], vc);
                int peer = real.id(vc);
                int64_t cnt = count / ports + (p < count % ports ? 1 : 0);
                int64_t off = so_far;
                so_far += cnt;
                bool use_send = st == 0 && !first[r];
                b.send(r, peer, kTagAR, R(r, use_send ? kBufSend : kBufRecv, off), cnt);
                Region into = R(r, kBufRecv, off);
                Region agg = use_send ? R(r, kBufSend, off) : R(r, kBufRecv, off);
                b.recv(r, peer, kTagAR, into, cnt, &agg);
            }
        }
        b.end(g.s);
    }
    if (!all_p2) {
        for (int d = real.ndims - 1; d >= 0; d--) {
            if (is_pow2(real.dims[d])) continue;
            b.begin();
            const int extra = real.dims[d] - virt.dims[d];
            for (int r = 0; r < P; r++) {
                int cp[kMaxDims] = {coord[r][0], coord[r][1], coord[r][2]};
                if (coord[r][d] >= virt.dims[d]) {
                    cp[d] = coord[r][d] - extra;
                    b.recv(r, real.id(cp), kTagAR, R(r, kBufRecv, 0), count);
                } else if (coord[r][d] + extra >= virt.dims[d]) {
                    cp[d] = coord[r][d] + extra;
                    b.send(r, real.id(cp), kTagAR, R(r, kBufRecv, 0), count);
                }
            }
            b.end(g.s);
        }
    }
    b.finish(g.s);
}

// Contiguous reduce-scatter: permute blocks into tree order, then halve
// (bine_reduce_scatter_mpi_contiguous, lib/libbine_coll_reduce_scatter.cc:660-758).
void gen_reduce_scatter_cont(const Gen& g) {
    const int P = g.P, S = g.S, ports = g.k.ports;
    const int64_t c = g.k.count;  // per-rank result count
    if (c * P < (int64_t)ports * P) throw PlanError("reduce_scatter asserts count >= ports*size (lib/libbine.cc:1078)");
    if (!is_pow2(P))
        throw PlanError("contiguous reduce_scatter halves size/2^(s+1) blocks per step and returns wrong data unless "
                        "size is a power of two (lib/libbine_coll_reduce_scatter.cc:733)");
    if (ports > 1)
        throw PlanError("contiguous reduce_scatter writes past the end of recvbuf for ports > 1 "
                        "(lib/libbine_coll_reduce_scatter.cc:710, 742)");
    auto bi = blocks_by_block(c, P, ports);
    g.s->send_elems = c * P;
    g.s->recv_elems = c;
    const int64_t b0 = bi[0][0].n;
    const int64_t tmpn = b0 * ports * P;
    Builder b(P, tmpn);
    std::vector<RankTree> trees;
    std::vector<std::vector<int>> peers(P);
    for (int p = 0; p < ports; p++) {
        TreeBuilder tb(g.t, p, g.k.family, g.k.distance);
        b.begin();
        for (int r = 0; r < P; r++) {
            RankTree tr = tb.build(r);
            peers[r] = peers_of(g.t, r, p, g.k.family);
            int64_t top = tmpn / ports * p;
            for (int i = 0; i < P; i++)
                b.copy(R(r, kBufTmp, top + b0 * tr.remapped[i]), R(r, kBufSend, bi[p][i].off), bi[p][i].n);
        }
        b.end(g.s);
        for (int st = 0; st < S; st++) {
            b.begin();
            int64_t cnt = (int64_t)(P >> (st + 1)) * b0;
            for (int r = 0; r < P; r++) {
                int peer = g.k.distance == kDecreasing ? peers[r][S - st - 1] : peers[r][st];
                int64_t top = tmpn / ports * p;
                // Sendrecv_replace of the upper half, then lower += upper.
                b.send(r, peer, kTagRS, R(r, kBufTmp, top + cnt), cnt);
                Region lower = R(r, kBufTmp, top);
                Region into = st == S - 1 ? R(r, kBufRecv, top) : lower;
                b.recv(r, peer, kTagRS, into, cnt, &lower);
            }
            b.end(g.s);
        }
    }
    b.finish(g.s);
}

// Allgather, permute at the end (bine_allgather_mpi_contiguous,
// lib/libbine_coll_allgather.cc:289-374).
void gen_allgather_cont_permute(const Gen& g) {
    const int P = g.P, S = g.S, ports = g.k.ports;
    const int64_t c = g.k.count;
    if (!is_pow2(P))
        throw PlanError("contiguous allgather doubles 2^s blocks per step and writes past its buffer unless size is "
                        "a power of two (lib/libbine_coll_allgather.cc:341-345)");
    auto bi = blocks_by_block(c, P, ports);
    g.s->send_elems = c;
    g.s->recv_elems = c * P;
    const int64_t tmpn = (int64_t)std::ceil((float)c / ports) * ports * P;
    Builder b(P, tmpn);
    for (int p = 0; p < ports; p++) {
        const int64_t top = tmpn / ports * p, b0 = bi[p][0].n;
        b.begin();
        for (int r = 0; r < P; r++) b.copy(R(r, kBufTmp, top), R(r, kBufSend, bi[p][0].off), b0);
        b.end(g.s);
        std::vector<std::vector<int>> peers(P);
        for (int r = 0; r < P; r++) peers[r] = peers_of(g.t, r, p, g.k.family);
        for (int st = 0; st < S; st++) {
            b.begin();
            int64_t cnt = ((int64_t)1 << st) * b0;
            for (int r = 0; r < P; r++) {
                int peer = g.k.distance == kDecreasing ? peers[r][S - st - 1] : peers[r][st];
                b.send(r, peer, kTagAG, R(r, kBufTmp, top), cnt);
                b.recv(r, peer, kTagAG, R(r, kBufTmp, top + cnt), cnt);
            }
            b.end(g.s);
        }
        TreeBuilder tb(g.t, p, g.k.family, g.k.distance == kDecreasing ? kIncreasing : kDecreasing);
        b.begin();
        for (int r = 0; r < P; r++) {
            RankTree perm = tb.build(r);
            for (int i = 0; i < P; i++)
                b.copy(R(r, kBufRecv, bi[p][i].off), R(r, kBufTmp, top + perm.remapped[i] * b0), bi[p][i].n);
        }
        b.end(g.s);
    }
    b.finish(g.s);
}

// Allgather, permute at the start (bine_allgather_send_mpi,
// lib/libbine_coll_allgather.cc:492-574).
void gen_allgather_cont_send(const Gen& g) {
    const int P = g.P, S = g.S;
    const int64_t c = g.k.count;
    if (g.k.ports != 1) throw PlanError("CONT_SEND allgather asserts one port (lib/libbine_coll_allgather.cc:501)");
    if (!is_pow2(P))
        throw PlanError("CONT_SEND allgather indexes past recvbuf unless size is a power of two "
                        "(lib/libbine_coll_allgather.cc:551-566)");
    g.s->send_elems = c;
    g.s->recv_elems = c * P;
    TreeBuilder tb(g.t, 0, g.k.family, g.k.distance == kDecreasing ? kIncreasing : kDecreasing);
    RankTree tree = tb.build(0);
    std::vector<uint32_t> inv(P);
    for (int i = 0; i < P; i++) inv[tree.remapped[i]] = i;
    Builder b(P, 0);
    b.begin();
    for (int r = 0; r < P; r++) {
        b.send(r, inv[r], kTagAG, R(r, kBufSend, 0), c);
        b.recv(r, tree.remapped[r], kTagAG, R(r, kBufRecv, (int64_t)tree.remapped[r] * c), c);
    }
    b.end(g.s);
    std::vector<std::vector<int>> peers(P);
    std::vector<int64_t> min_res(P);
    for (int r = 0; r < P; r++) {
        peers[r] = peers_of(g.t, r, 0, g.k.family);
        min_res[r] = tree.remapped[r];
    }
    int64_t nb = 1;
    for (int st = 0; st < S; st++) {
        b.begin();
        std::vector<int64_t> next(P);
        for (int r = 0; r < P; r++) {
            int peer = g.k.distance == kDecreasing ? peers[r][S - st - 1] : peers[r][st];
            int64_t min_r = tree.remapped[peer] & ~(((int64_t)1 << st) - 1);
            b.send(r, peer, kTagAG, R(r, kBufRecv, min_res[r] * c), nb * c);
            b.recv(r, peer, kTagAG, R(r, kBufRecv, min_r * c), nb * c);
            next[r] = std::min(min_res[r], min_r);
        }
        b.end(g.s);
        min_res = next;
        nb *= 2;
    }
    b.finish(g.s);
}

// Allgather block by block (bine_allgather_blocks_mpi,
// lib/libbine_coll_allgather.cc:1161-1228).
void gen_allgather_blocks(const Gen& g) {
    const int P = g.P;
    const int64_t c = g.k.count;
    g.s->send_elems = c;
    g.s->recv_elems = c * P;
    Builder b(P, 0);
    b.begin();
    for (int r = 0; r < P; r++) b.copy(R(r, kBufRecv, (int64_t)r * c), R(r, kBufSend, 0), c);
    b.end(g.s);
    const int nbits = ceil_log2(P);
    int step = 0;
    for (int inv = nbits > 0 ? 1 << (nbits - 1) : 0; inv > 0; inv >>= 1, step++) {
        b.begin();
        for (int r = 0; r < P; r++) {
            int partner = (r % 2 == 0) ? pmod(r + from_negabinary((uint32_t)((inv << 1) - 1)), P)
                                       : pmod(r - from_negabinary((uint32_t)((inv << 1) - 1)), P);
            for (int blk = 1; blk < P; blk++) {
                uint32_t nu = nu_of(blk, P);
                if (nu == UINT32_MAX) throw PlanError("block has no negabinary representation");
                int k = 31 - __builtin_clz(nu);
                if (k != step) continue;
                int bsend, brecv;
                if (r % 2 == 0) {
                    brecv = pmod(blk + r, P);
                    bsend = pmod(partner - blk, P);
                } else {
                    brecv = pmod(r - blk, P);
                    bsend = pmod(blk + partner, P);
                }
                if (bsend != partner) b.send(r, partner, 0, R(r, kBufRecv, (int64_t)bsend * c), c);
                if (brecv != r) b.recv(r, partner, 0, R(r, kBufRecv, (int64_t)brecv * c), c);
            }
        }
        b.end(g.s);
    }
    b.finish(g.s);
}

// Binomial-tree bcast over negabinary partners (bine_bcast_l_mpi,
// lib/libbine_coll_bcast.cc:635-665).  The buffer is the receive array; the
// root's row holds the data.
void gen_bcast_tree(const Gen& g) {
    const int P = g.P, root = g.k.root;
    const int64_t c = g.k.count;
    g.s->send_elems = 0;
    g.s->recv_elems = c;
    Builder b(P, 0);
    std::vector<int> recvd(P, 0);
    recvd[root] = 1;
    const int nbits = ceil_log2(P);
    for (int mask = nbits > 0 ? 1 << (nbits - 1) : 0; mask > 0; mask >>= 1) {
        b.begin();
        std::vector<int> got;
        for (int r = 0; r < P; r++) {
            int vr = pmod(r - root, P);
            uint32_t nb = to_negabinary(vr);
            int partner = pmod(from_negabinary(nb ^ (uint32_t)((mask << 1) - 1)) + root, P);
            uint32_t ml = (uint32_t)((mask << 1) - 1), lsbs = nb & ml;
            if (recvd[r]) {
                b.send(r, partner, 0, R(r, kBufRecv, 0), c);
            } else if (lsbs == 0 || lsbs == ml) {
                b.recv(r, partner, 0, R(r, kBufRecv, 0), c);
                got.push_back(r);
            }
        }
        b.end(g.s);
        for (int r : got) recvd[r] = 1;
    }
    b.finish(g.s);
}

std::vector<int64_t> even_displs(int64_t count, int P, std::vector<int64_t>* counts) {
    std::vector<int64_t> d(P);
    counts->assign(P, 0);
    int64_t q = count / P, rem = count % P;
    for (int i = 0; i < P; i++) {
        d[i] = q * i + (i < rem ? i : rem);
        (*counts)[i] = q + (i < rem ? 1 : 0);
    }
    return d;
}

int bine_partner(int r, int mask, int P) {
    int nb = from_negabinary((uint32_t)((mask << 1) - 1));
    return r % 2 == 0 ? pmod(r + nb, P) : pmod(r - nb, P);
}

// Scatter + allgather bcast (bine_bcast_scatter_allgather_mpi,
// lib/libbine_coll_bcast.cc:985-1093).
void gen_bcast_scatter_allgather(const Gen& g) {
    const int P = g.P, root = g.k.root;
    const int64_t c = g.k.count;
    if (root != 0) throw PlanError("scatter-allgather bcast asserts root == 0 (lib/libbine_coll_bcast.cc:993)");
    if (!is_pow2(P))
        throw PlanError("scatter-allgather bcast indexes past its per-rank tables unless size is a power of two "
                        "(lib/libbine_coll_bcast.cc:1030-1037)");
    g.s->send_elems = 0;
    g.s->recv_elems = c;
    std::vector<int64_t> cnts;
    std::vector<int64_t> displs = even_displs(c, P, &cnts);
    auto range = [&](int first, int inv) { return displs[first + inv - 1] - displs[first] + cnts[first + inv - 1]; };
    Builder b(P, 0);
    const int nbits = ceil_log2(P);
    std::vector<int> remapped(P), recv_mask(P), recvd(P, 0);
    for (int r = 0; r < P; r++) {
        remapped[r] = (int)remap_rank(r, P);
        recv_mask[r] = r == root ? (1 << nbits) : 1 << (__builtin_ffs(remapped[r]) - 1);
    }
    recvd[root] = 1;
    int mask = 1, inv = nbits > 0 ? 1 << (nbits - 1) : 0, bfm = ~(inv - 1);
    while (mask < P) {
        b.begin();
        std::vector<int> got;
        for (int r = 0; r < P; r++) {
            int partner = bine_partner(r, mask, P);
            int sbf = remapped[partner] & bfm;
            int rbf = remapped[r] & bfm;
            if (recvd[r]) {
                b.send(r, partner, 0, R(r, kBufRecv, displs[sbf]), range(sbf, inv));
            } else if (inv == recv_mask[r] || partner == root) {
                b.recv(r, partner, 0, R(r, kBufRecv, displs[rbf]), range(rbf, inv));
                got.push_back(r);
            }
        }
        b.end(g.s);
        for (int r : got) recvd[r] = 1;
        mask <<= 1;
        inv >>= 1;
        bfm >>= 1;
    }
    mask >>= 1;
    inv = 1;
    bfm = ~0;
    while (mask > 0) {
        b.begin();
        for (int r = 0; r < P; r++) {
            int partner = bine_partner(r, mask, P);
            bool has_r = !(inv < recv_mask[r]), has_s = inv != recv_mask[r];
            if (has_s) {
                int sbf = remapped[r] & bfm;
                b.send(r, partner, 0, R(r, kBufRecv, displs[sbf]), range(sbf, inv));
            }
            if (has_r) {
                int rbf = remapped[partner] & bfm;
                b.recv(r, partner, 0, R(r, kBufRecv, displs[rbf]), range(rbf, inv));
            }
        }
        b.end(g.s);
        mask >>= 1;
        inv <<= 1;
        bfm <<= 1;
    }
    b.finish(g.s);
}

// Binomial-tree reduce (bine_reduce_mpi, lib/libbine_coll_reduce.cc:575-615).
// Non-root partial sums live in the workspace (the reference mallocs them).
void gen_reduce_tree(const Gen& g) {
    const int P = g.P, root = g.k.root;
    const int64_t c = g.k.count;
    g.s->send_elems = g.s->recv_elems = c;
    auto acc = [&](int r) { return r == root ? R(r, kBufRecv, 0) : R(r, kBufTmp, 0); };
    Builder b(P, c);
    b.begin();
    for (int r = 0; r < P; r++) b.copy(acc(r), R(r, kBufSend, 0), c);
    b.end(g.s);
    std::vector<int> done(P, 0);
    for (int mask = 1; mask < P; mask <<= 1) {
        b.begin();
        std::vector<int> leaving;
        for (int r = 0; r < P; r++) {
            if (done[r]) continue;
            int vr = pmod(r - root, P);
            uint32_t nb = to_negabinary(vr);
            int partner = pmod(from_negabinary(nb ^ (uint32_t)((mask << 1) - 1)) + root, P);
            uint32_t ml = (uint32_t)((mask << 2) - 1), lsbs = nb & ml;
            bool equal = lsbs == 0 || lsbs == ml;
            if (!equal || ((mask << 1) >= P && r != root)) {
                b.send(r, partner, 0, acc(r), c);
                leaving.push_back(r);
            } else {
                Region a = acc(r);
                b.recv(r, partner, 0, a, c, &a);
            }
        }
        b.end(g.s);
        for (int r : leaving) done[r] = 1;
    }
    b.finish(g.s);
}

// Reduce-scatter + gather reduce (bine_reduce_redscat_gather_mpi,
// lib/libbine_coll_reduce.cc:1042-1152).
void gen_reduce_redscat_gather(const Gen& g) {
    const int P = g.P, root = g.k.root;
    const int64_t c = g.k.count;
    if (root != 0) throw PlanError("reduce-scatter+gather reduce asserts root == 0 (lib/libbine_coll_reduce.cc:1049)");
    if (!is_pow2(P))
        throw PlanError("reduce-scatter+gather reduce deadlocks unless size is a power of two "
                        "(lib/libbine_coll_reduce.cc:1083-1140)");
    g.s->send_elems = g.s->recv_elems = c;
    std::vector<int64_t> cnts;
    std::vector<int64_t> displs = even_displs(c, P, &cnts);
    auto range = [&](int first, int inv) { return displs[first + inv - 1] - displs[first] + cnts[first + inv - 1]; };
    auto res = [&](int r, int64_t off) { return r == root ? R(r, kBufRecv, off) : R(r, kBufTmp, off); };
    Builder b(P, c);
    b.begin();
    for (int r = 0; r < P; r++) b.copy(res(r, 0), R(r, kBufSend, 0), c);
    b.end(g.s);
    const int nbits = ceil_log2(P);
    std::vector<int> remapped(P);
    for (int r = 0; r < P; r++) remapped[r] = (int)remap_rank(r, P);
    int mask = 1, inv = nbits > 0 ? 1 << (nbits - 1) : 0, bfm = ~(inv - 1);
    while (mask < P) {
        b.begin();
        for (int r = 0; r < P; r++) {
            int partner = bine_partner(r, mask, P);
            int sbf = remapped[partner] & bfm, rbf = remapped[r] & bfm;
            b.send(r, partner, 0, res(r, displs[sbf]), range(sbf, inv));
            Region into = res(r, displs[rbf]);
            b.recv(r, partner, 0, into, range(rbf, inv), &into);
        }
        b.end(g.s);
        mask <<= 1;
        inv >>= 1;
        bfm >>= 1;
    }
    mask >>= 1;
    inv = 1;
    bfm = ~0;
    std::vector<int> done(P, 0);
    while (mask > 0) {
        b.begin();
        std::vector<int> leaving;
        for (int r = 0; r < P; r++) {
            if (done[r]) continue;
            int partner = bine_partner(r, mask, P);
            int rm = 1 << (__builtin_ffs(remapped[r]) - 1);
            if (inv & rm) {
                int sbf = remapped[r] & bfm;
                b.send(r, partner, 0, res(r, displs[sbf]), range(sbf, inv));
                leaving.push_back(r);
            } else {
                int rbf = remapped[partner] & bfm;
                b.recv(r, partner, 0, res(r, displs[rbf]), range(rbf, inv));
            }
        }
        b.end(g.s);
        for (int r : leaving) done[r] = 1;
        mask >>= 1;
        inv <<= 1;
        bfm <<= 1;
    }
    b.finish(g.s);
}

// Log-step alltoall with block compaction and a final permutation
// (bine_alltoall_mpi, lib/libbine_coll_alltoall.cc:411-540).  The
// reference's tmpbuf is workspace [0, P*c).
void gen_alltoall(const Gen& g) {
    const int P = g.P;
    const int64_t c = g.k.count;
    if (!is_pow2(P)) throw PlanError("alltoall asserts block_recvd_cnt == size/2 (lib/libbine_coll_alltoall.cc:484)");
    g.s->send_elems = g.s->recv_elems = c * P;
    const int nbits = ceil_log2(P);
    Builder b(P, c * P);
    b.begin();
    for (int r = 0; r < P; r++) b.copy(R(r, kBufTmp, 0), R(r, kBufSend, 0), c * P);
    b.end(g.s);
    std::vector<std::vector<uint32_t>> res(P, std::vector<uint32_t>(P));
    for (int r = 0; r < P; r++)
        for (int i = 0; i < P; i++) res[r][i] = i;
    size_t nres = P;
    std::vector<uint32_t> remap(P);
    for (int i = 0; i < P; i++) remap[i] = remap_rank(i, P);
    int mask = 1, inv = 1 << (nbits - 1), bfm = ~(inv - 1);
    while (mask < P) {
        // Compaction: blocks to send go to recvbuf, kept blocks move left.
        b.begin();
        std::vector<std::vector<uint32_t>> next(P);
        std::vector<int> partner(P);
        for (int r = 0; r < P; r++) {
            partner[r] = bine_partner(r, mask, P);
            uint32_t min_s = remap[partner[r]] & bfm, max_s = min_s + inv - 1;
            int64_t off_send = 0, off_keep = 0;
            for (int i = 0; i < P; i++) {
                uint32_t blk = res[r][i % nres];
                if (remap[blk] >= min_s && remap[blk] <= max_s) {
                    b.copy(R(r, kBufRecv, off_send), R(r, kBufTmp, (int64_t)i * c), c);
                    off_send += c;
                } else {
                    if ((int64_t)i * c != off_keep) b.copy(R(r, kBufTmp, off_keep), R(r, kBufTmp, (int64_t)i * c), c);
                    off_keep += c;
                    next[r].push_back(blk);
                }
            }
            if ((int)next[r].size() != P / 2) throw PlanError("alltoall asserts block_recvd_cnt == size/2");
        }
        b.end(g.s);
        b.begin();
        for (int r = 0; r < P; r++) {
            b.send(r, partner[r], 0, R(r, kBufRecv, 0), (int64_t)(P / 2) * c);
            b.recv(r, partner[r], 0, R(r, kBufTmp, (int64_t)(P / 2) * c), (int64_t)(P / 2) * c);
        }
        b.end(g.s);
        for (int r = 0; r < P; r++) {
            for (size_t i = 0; i < next[r].size(); i++) res[r][i] = next[r][i];
        }
        nres /= 2;
        mask <<= 1;
        inv >>= 1;
        bfm >>= 1;
    }
    b.begin();
    for (int r = 0; r < P; r++) {
        for (int i = 0; i < P; i++) {
            int rot = r % 2 == 0 ? pmod(i - r, P) : pmod(r - i, P);
            uint32_t repr = nb_in_range(rot, nbits) ? to_negabinary(rot) : to_negabinary(rot - P);
            int idx = distance_doubling_position(repr);
            b.copy(R(r, kBufRecv, (int64_t)i * c), R(r, kBufTmp, (int64_t)idx * c), c);
        }
    }
    b.end(g.s);
    b.finish(g.s);
}

// Bruck's log-step alltoall, the reference's comparator (bruck_alltoall,
// lib/libbine_coll_alltoall.cc:18-107): rotate the blocks by the rank, then
// at step k = 1, 2, 4, ... pack the blocks whose index has bit k set,
// exchange them with rank + k / rank - k in one message and unpack them in
// place, and finally rotate back into recvbuf.  Any P.  Workspace: the
// rotated blocks [0, P*c), the outgoing pack and the incoming pack
// ((P+1)/2 blocks each), as the reference's three temporary buffers.
void gen_alltoall_bruck(const Gen& g) {
    const int P = g.P;
    const int64_t c = g.k.count;
    const int64_t half = (P + 1) / 2;
    g.s->send_elems = g.s->recv_elems = c * P;
    const int64_t pack = (int64_t)P * c, inbox = pack + half * c;
    Builder b(P, inbox + half * c);
    b.begin();
    for (int r = 0; r < P; r++)
        for (int i = 0; i < P; i++) b.copy(R(r, kBufTmp, pmod(i - r, P) * c), R(r, kBufSend, (int64_t)i * c), c);
    b.end(g.s);
    for (int k = 1; k < P; k <<= 1) {
        std::vector<int> idx;
        for (int i = k; i < P; i++)
            if (i & k) idx.push_back(i);
        const int64_t n = (int64_t)idx.size() * c;
        b.begin();
        for (int r = 0; r < P; r++)
            for (size_t j = 0; j < idx.size(); j++)
                b.copy(R(r, kBufTmp, pack + (int64_t)j * c), R(r, kBufTmp, (int64_t)idx[j] * c), c);
        b.end(g.s);
        b.begin();
        for (int r = 0; r < P; r++) {
            b.send(r, (r + k) % P, 0, R(r, kBufTmp, pack), n);
            b.recv(r, pmod(r - k, P), 0, R(r, kBufTmp, inbox), n);
        }
        b.end(g.s);
        b.begin();
        for (int r = 0; r < P; r++)
            for (size_t j = 0; j < idx.size(); j++)
                b.copy(R(r, kBufTmp, (int64_t)idx[j] * c), R(r, kBufTmp, inbox + (int64_t)j * c), c);
        b.end(g.s);
    }
    b.begin();
    for (int r = 0; r < P; r++)
        for (int i = 0; i < P; i++) b.copy(R(r, kBufRecv, pmod(r - i, P) * c), R(r, kBufTmp, (int64_t)i * c), c);
    b.end(g.s);
    b.finish(g.s);
}

// Bucket allreduce, the reference's RING family: the multi-dimensional ring
// the paper compares Bine against (BineCommon::bucket_allreduce,
// lib/libbine_common.cc:2486-2663, over ringRedScatAG,
// lib/libbine_common.cc:2372-2484).  The reference runs it on uTofu only;
// this restates its schedule as messages.
//   * The vector, padded to a multiple of 2*D*P elements, is copied into a
//     work row (lib/libbine_common.cc:2559) and cut into 2*D buckets; bucket
//     2i runs its rings toward the next node of a dimension, bucket 2i+1
//     toward the previous one (lib/libbine_common.cc:2598-2603).
//   * Reduce-scatter rounds s = 0..D-1: bucket pair i reduces its current
//     range along dimension (i + s) % D with a ring reduce-scatter (n - 1
//     steps; at step k a rank sends chunk c - k - 1 and adds the received
//     chunk c - k - 2 into its own, or c + k + 1 and c + k + 2 toward the
//     previous node; lib/libbine_common.cc:2395-2402), then keeps chunk c
//     (its coordinate) as the next round's range (lib/libbine_common.cc:
//     2617-2620).
//   * Allgather rounds in reverse order: the first copies each bucket's
//     range from the work row to the receive row (lib/libbine_common.cc:
//     2648-2656), then ring allgathers (chunk c - k sent, c - k - 1
//     received, or c + k and c + k + 1; lib/libbine_common.cc:2435-2441)
//     rebuild the ranges in the receive row.
// Moves and messages cover the real elements only: the padding past `count`
// (uninitialised in the reference) feeds no result, and the reference's
// allgather skips it too (lib/libbine_common.cc:2452-2466).
void gen_allreduce_ring(const Gen& g) {
    const Torus& t = g.t;
    const int P = g.P, D = t.ndims;
    const int64_t count = g.k.count;
    int64_t padded = count;
    const int64_t unit = 2LL * D * P;
    if (padded % unit) padded += unit - padded % unit;
    const int64_t B = padded / (2 * D);
    g.s->send_elems = g.s->recv_elems = count;
    Builder b(P, padded);
    auto clip = [&](int64_t off, int64_t n) { return std::max<int64_t>(0, std::min(n, count - off)); };
    b.begin();
    for (int r = 0; r < P; r++) b.copy(R(r, kBufTmp, 0), R(r, kBufSend, 0), count);
    b.end(g.s);
    std::vector<std::vector<int>> coord(P, std::vector<int>(kMaxDims, 0));
    for (int r = 0; r < P; r++) t.coords(r, coord[r].data());
    auto neighbour = [&](int r, int d, int delta) {
        int c[kMaxDims];
        for (int i = 0; i < kMaxDims; i++) c[i] = coord[r][i];
        c[d] = pmod(c[d] + delta, t.dims[d]);
        return t.id(c);
    };
    // Per bucket pair i and rank r: the current range's offset inside the
    // bucket; per round and pair: the range size and dimension.
    std::vector<std::vector<int64_t>> offset(D, std::vector<int64_t>(P, 0));
    std::vector<int64_t> size(D, B);
    std::vector<std::vector<std::vector<int64_t>>> saved_off(D);  // [round][pair][rank]
    std::vector<std::vector<int64_t>> saved_size(D, std::vector<int64_t>(D));
    const int tag0 = 0x7000;
    for (int s = 0; s < D; s++) {
        saved_off[s] = offset;
        int most = 0;
        for (int i = 0; i < D; i++) {
            saved_size[s][i] = size[i];
            most = std::max(most, t.dims[(i + s) % D]);
        }
        for (int k = 0; k + 1 < most; k++) {
            b.begin();
            for (int j = 0; j < 2 * D; j++) {
                const int i = j / 2, d = (i + s) % D, n = t.dims[d];
                if (k + 1 >= n) continue;
                const int64_t seg = size[i] / n;
                for (int r = 0; r < P; r++) {
                    const int c = coord[r][d];
                    const int to = neighbour(r, d, j % 2 ? -1 : 1), from = neighbour(r, d, j % 2 ? 1 : -1);
                    const int send_chunk = j % 2 ? pmod(c + 1 + k, n) : pmod(c - k - 1, n);
                    const int recv_chunk = j % 2 ? pmod(c + 2 + k, n) : pmod(c - k - 2, n);
                    const int64_t base = j * B + offset[i][r];
                    const int64_t so = base + send_chunk * seg, ro = base + recv_chunk * seg;
                    if (clip(so, seg) > 0) b.send(r, to, tag0 + j, R(r, kBufTmp, so), clip(so, seg));
                    if (clip(ro, seg) > 0) {
                        Region into = R(r, kBufTmp, ro);
                        b.recv(r, from, tag0 + j, into, clip(ro, seg), &into);
                    }
                }
            }
            b.end(g.s);
        }
        if (s != D - 1)
            for (int i = 0; i < D; i++) {
                const int d = (i + s) % D;
                size[i] /= t.dims[d];
                for (int r = 0; r < P; r++) offset[i][r] += coord[r][d] * size[i];
            }
    }
    for (int s = D - 1; s >= 0; s--) {
        if (s == D - 1) {
            b.begin();
            for (int j = 0; j < 2 * D; j++)
                for (int r = 0; r < P; r++) {
                    const int64_t o = j * B + saved_off[s][j / 2][r];
                    if (clip(o, saved_size[s][j / 2]) > 0)
                        b.copy(R(r, kBufRecv, o), R(r, kBufTmp, o), clip(o, saved_size[s][j / 2]));
                }
            b.end(g.s);
        }
        int most = 0;
        for (int i = 0; i < D; i++) most = std::max(most, t.dims[(i + s) % D]);
        for (int k = 0; k + 1 < most; k++) {
            b.begin();
            for (int j = 0; j < 2 * D; j++) {
                const int i = j / 2, d = (i + s) % D, n = t.dims[d];
                if (k + 1 >= n) continue;
                const int64_t seg = saved_size[s][i] / n;
                for (int r = 0; r < P; r++) {
                    const int c = coord[r][d];
                    const int to = neighbour(r, d, j % 2 ? -1 : 1), from = neighbour(r, d, j % 2 ? 1 : -1);
                    const int send_chunk = j % 2 ? pmod(c + k, n) : pmod(c - k, n);
                    const int recv_chunk = j % 2 ? pmod(c + k + 1, n) : pmod(c - k - 1, n);
                    const int64_t base = j * B + saved_off[s][i][r];
                    const int64_t so = base + send_chunk * seg, ro = base + recv_chunk * seg;
                    if (clip(so, seg) > 0) b.send(r, to, tag0 + 2 * D + j, R(r, kBufRecv, so), clip(so, seg));
                    if (clip(ro, seg) > 0) b.recv(r, from, tag0 + 2 * D + j, R(r, kBufRecv, ro), clip(ro, seg));
                }
            }
            b.end(g.s);
        }
    }
    b.finish(g.s);
}

// Scatter down a negabinary binomial tree with wrap-around block ranges
// (bine_scatter_mpi, lib/libbine_coll_scatter.cc:187-324).  Interior ranks
// keep the blocks of their subtree in the workspace.
void gen_scatter(const Gen& g) {
    const int P = g.P, root = g.k.root;
    const int64_t c = g.k.count;
    if (!is_pow2(P))
        throw PlanError("scatter sends wrap-around ranges its receivers do not expect unless size is a power of two "
                        "(lib/libbine_coll_scatter.cc:270-310)");
    g.s->send_elems = c * P;
    g.s->recv_elems = c;
    const int nb = ceil_log2(P);
    struct St {
        int hd;
        int64_t min_res, max_res;
        int recvd, leaf, sbuf_off;
        uint8_t sbuf;  // kBufSend (root) or kBufTmp
        int64_t sbuf_n;
    };
    std::vector<St> st(P);
    for (int r = 0; r < P; r++) {
        St& x = st[r];
        x.hd = r % 2 ? -1 : 1;
        if (nb % 2 == 0) x.hd = -x.hd;
        const int m = (1 << nb) - 1;
        if (r % 2 == 0) {
            x.max_res = pmod((int)((r + 0x55555555) & m), P);
            x.min_res = pmod((int)((r - (int)0xAAAAAAAA) & m), P);
        } else {
            x.min_res = pmod((int)((r - 0x55555555) & m), P);
            x.max_res = pmod((int)((r + (int)0xAAAAAAAA) & m), P);
        }
        x.recvd = r == root;
        x.leaf = 0;
        x.sbuf_off = r;
        x.sbuf = kBufSend;
        x.sbuf_n = c * P;
    }
    Builder b(P, c * P);
    for (int mask = 1 << (nb - 1); mask > 0; mask >>= 1) {
        b.begin();
        std::vector<std::pair<int, St>> updates;
        for (int r = 0; r < P; r++) {
            St x = st[r];
            int vr = pmod(r - root, P);
            int vnb = (int)to_negabinary(vr);
            int partner = pmod(from_negabinary((uint32_t)(vnb ^ ((mask << 1) - 1))) + root, P);
            int ml = (mask << 1) - 1, lsbs = vnb & ml;
            bool equal = lsbs == 0 || lsbs == ml;
            int64_t ts = x.min_res, te = pmod((int)(x.min_res + mask - 1), P);
            int64_t bs = pmod((int)(te + 1), P), be = x.max_res;
            int64_t ss, se, rs, re;
            if (x.hd == 1) {
                ss = bs, se = be, rs = ts, re = te;
                x.max_res = pmod((int)(x.max_res - mask), P);
            } else {
                ss = ts, se = te, rs = bs, re = be;
                x.min_res = pmod((int)(x.min_res + mask), P);
            }
            if (x.recvd) {
                if (se >= ss) {
                    b.send(r, partner, 0, R(r, x.sbuf, ss * c), c * (se - ss + 1));
                } else {
                    b.send(r, partner, 0, R(r, x.sbuf, ss * c), c * (P - ss));
                    b.send(r, partner, 0, R(r, x.sbuf, 0), c * (se + 1));
                }
            } else if (equal) {
                int64_t num_blocks = pmod((int)(re - rs + 1), P);
                Region rb;
                if (rs == re) {
                    rb = R(r, kBufRecv, 0);
                    x.leaf = 1;
                } else {
                    rb = R(r, kBufTmp, 0);
                    x.sbuf = kBufTmp;
                    x.sbuf_n = c * num_blocks;
                    x.min_res = 0;
                    x.max_res = num_blocks - 1;
                    x.sbuf_off = pmod((int)(r - rs), P);
                }
                if (re >= rs) {
                    b.recv(r, partner, 0, rb, c * num_blocks);
                } else {
                    int64_t first = c * (P - rs);
                    b.recv(r, partner, 0, rb, first);
                    Region rb2 = rb;
                    rb2.off += first;
                    b.recv(r, partner, 0, rb2, c * (re + 1));
                }
                x.recvd = 1;
            }
            x.hd = -x.hd;
            updates.push_back({r, x});
        }
        b.end(g.s);
        for (auto& u : updates) st[u.first] = u.second;
    }
    b.begin();
    for (int r = 0; r < P; r++)
        if (!st[r].leaf) b.copy(R(r, kBufRecv, 0), R(r, st[r].sbuf, (int64_t)st[r].sbuf_off * c), c);
    b.end(g.s);
    b.finish(g.s);
}

// Gather up a negabinary binomial tree (bine_gather_mpi,
// lib/libbine_coll_gather.cc:202-272).  Non-root ranks collect in the
// workspace.
void gen_gather(const Gen& g) {
    const int P = g.P, root = g.k.root;
    const int64_t c = g.k.count;
    if (!is_pow2(P))
        throw PlanError("gather deadlocks unless size is a power of two (lib/libbine_coll_gather.cc:218-265)");
    g.s->send_elems = c;
    g.s->recv_elems = c * P;
    auto buf = [&](int r, int64_t off) { return r == root ? R(r, kBufRecv, off) : R(r, kBufTmp, off); };
    Builder b(P, c * P);
    b.begin();
    for (int r = 0; r < P; r++) b.copy(buf(r, (int64_t)r * c), R(r, kBufSend, 0), c);
    b.end(g.s);
    std::vector<int64_t> mn(P), mx(P);
    std::vector<int> ext(P), done(P, 0);
    for (int r = 0; r < P; r++) {
        mn[r] = mx[r] = r;
        ext[r] = r % 2 ? -1 : 1;
    }
    for (int mask = 1; mask < P; mask <<= 1) {
        b.begin();
        std::vector<int> leaving;
        for (int r = 0; r < P; r++) {
            if (done[r]) continue;
            int vr = pmod(r - root, P);
            uint32_t nbv = to_negabinary(vr);
            int partner = pmod(from_negabinary(nbv ^ (uint32_t)((mask << 1) - 1)) + root, P);
            uint32_t ml = (uint32_t)((mask << 2) - 1), lsbs = nbv & ml;
            bool equal = lsbs == 0 || lsbs == ml;
            if (!equal || ((mask << 1) >= P && r != root)) {
                if (mx[r] >= mn[r]) {
                    b.send(r, partner, 0, buf(r, mn[r] * c), c * (mx[r] - mn[r] + 1));
                } else {
                    b.send(r, partner, 0, buf(r, mn[r] * c), c * (P - mn[r]));
                    b.send(r, partner, 0, buf(r, 0), c * (mx[r] + 1));
                }
                leaving.push_back(r);
            } else {
                int64_t rs, re;
                if (ext[r] == 1) {
                    rs = pmod((int)(mx[r] + 1), P);
                    re = pmod((int)(mx[r] + mask), P);
                    mx[r] = re;
                } else {
                    re = pmod((int)(mn[r] - 1), P);
                    rs = pmod((int)(mn[r] - mask), P);
                    mn[r] = rs;
                }
                if (re >= rs) {
                    b.recv(r, partner, 0, buf(r, rs * c), c * (re - rs + 1));
                } else {
                    b.recv(r, partner, 0, buf(r, rs * c), c * (P - rs));
                    b.recv(r, partner, 0, buf(r, 0), c * (re + 1));
                }
                ext[r] = -ext[r];
            }
        }
        b.end(g.s);
        for (int r : leaving) done[r] = 1;
    }
    b.finish(g.s);
}

// ------------------------------------------------------- symbolic executor
// Every buffer element holds an expression: a leaf "input element
// (rank, position + shift)" or the sum of two expressions.  Buffers are
// stored as runs of equal (node, shift); nodes are hash-consed with their two
// children in canonical order, so trees equal up to commutation (IEEE
// addition is commutative) share a node.
struct Node {
    int32_t left, right;   // -1 for leaves
    int64_t rshift;        // shift of the right child relative to the left one
    int32_t rank;          // leaves
    int32_t depth;         // evaluation stack depth (Sethi-Ullman)
    int32_t leaves;
};

struct Val {
    int32_t node;   // -1: undefined
    int64_t shift;  // value at position p is node evaluated at p + shift
    bool operator==(const Val& o) const { return node == o.node && shift == o.shift; }
};

class SymExec {
  public:
    explicit SymExec(int P) : P_(P) {
        for (int r = 0; r < P; r++) {
            Node n{-1, -1, 0, r, 1, 1};
            nodes_.push_back(n);
        }
    }
    int32_t leaf(int r) const { return r; }

    // Runs of one buffer: start -> (end, value).
    using Runs = std::map<int64_t, std::pair<int64_t, Val>>;
    Runs& buf(int rank, int b) { return bufs_[((uint64_t)rank << 8) | (uint64_t)b]; }

    void set(Runs& rb, int64_t lo, int64_t hi, Val v) {
        if (lo >= hi) return;
        split(rb, lo);
        split(rb, hi);
        auto it = rb.lower_bound(lo);
        while (it != rb.end() && it->first < hi) it = rb.erase(it);
        rb[lo] = {hi, v};
    }
    // Pieces of [lo, hi) as (start, end, value); undefined gaps get node -1.
    // A run's (node, shift) holds for every position in it, so pieces
    // inherit it unchanged.
    std::vector<std::tuple<int64_t, int64_t, Val>> get(Runs& rb, int64_t lo, int64_t hi) {
        std::vector<std::tuple<int64_t, int64_t, Val>> out;
        int64_t cur = lo;
        auto it = rb.upper_bound(lo);
        if (it != rb.begin()) {
            auto pv = std::prev(it);
            if (pv->second.first > lo) it = pv;
        }
        for (; it != rb.end() && it->first < hi; ++it) {
            int64_t s = std::max(it->first, lo), e = std::min(it->second.first, hi);
            if (s > cur) out.emplace_back(cur, s, Val{-1, 0});
            out.emplace_back(s, e, it->second.second);
            cur = e;
        }
        if (cur < hi) out.emplace_back(cur, hi, Val{-1, 0});
        return out;
    }

    int32_t add(Val a, Val b, int64_t* out_shift) {
        // Canonical order: by node id, then shift.
        if (std::make_pair(b.node, b.shift) < std::make_pair(a.node, a.shift)) std::swap(a, b);
        int64_t rel = b.shift - a.shift;
        auto key = std::make_tuple(a.node, b.node, rel);
        auto it = memo_.find(key);
        *out_shift = a.shift;
        if (it != memo_.end()) return it->second;
        const Node& A = nodes_[a.node];
        const Node& B = nodes_[b.node];
        Node n;
        n.left = a.node;
        n.right = b.node;
        n.rshift = rel;
        n.rank = -1;
        n.depth = A.depth == B.depth ? A.depth + 1 : std::max(A.depth, B.depth);
        n.leaves = A.leaves + B.leaves;
        nodes_.push_back(n);
        int32_t id = (int32_t)nodes_.size() - 1;
        memo_[key] = id;
        return id;
    }

    void apply(const Move& m) {
        Runs& rd = buf(m.dst.rank, m.dst.buf);
        auto pa = get(buf(m.a.rank, m.a.buf), m.a.off, m.a.off + m.n);
        // Collect values first (reads see the pre-move state).
        std::vector<std::tuple<int64_t, int64_t, Val>> outv;  // dst-relative
        if (!m.add) {
            for (auto& t : pa) {
                int64_t s = std::get<0>(t) - m.a.off, e = std::get<1>(t) - m.a.off;
                Val v = std::get<2>(t);
                if (v.node >= 0) v.shift += m.a.off - m.dst.off;
                outv.emplace_back(s, e, v);
            }
        } else {
            auto pb = get(buf(m.b.rank, m.b.buf), m.b.off, m.b.off + m.n);
            size_t ia = 0, ib = 0;
            int64_t cur = 0;
            while (cur < m.n) {
                while (std::get<1>(pa[ia]) - m.a.off <= cur) ia++;
                while (std::get<1>(pb[ib]) - m.b.off <= cur) ib++;
                int64_t e = std::min(std::get<1>(pa[ia]) - m.a.off, std::get<1>(pb[ib]) - m.b.off);
                Val va = std::get<2>(pa[ia]), vb = std::get<2>(pb[ib]);
                Val v{-1, 0};
                if (va.node >= 0 && vb.node >= 0) {
                    va.shift += m.a.off - m.dst.off;
                    vb.shift += m.b.off - m.dst.off;
                    int64_t sh;
                    v.node = add(va, vb, &sh);
                    v.shift = sh;
                }
                outv.emplace_back(cur, e, v);
                cur = e;
            }
        }
        for (auto& t : outv) {
            Val v = std::get<2>(t);
            set(rd, m.dst.off + std::get<0>(t), m.dst.off + std::get<1>(t), v);
        }
        coalesce(rd, m.dst.off, m.dst.off + m.n);
    }

    const Node& node(int32_t id) const { return nodes_[id]; }

    // Postfix program of (node, shift), deeper child first.
    void emit(int32_t id, int64_t shift, std::vector<ProgEntry>* out) const {
        const Node& n = nodes_[id];
        if (n.left < 0) {
            out->push_back(ProgEntry{n.rank, 0, shift});
            return;
        }
        const Node& L = nodes_[n.left];
        const Node& Rt = nodes_[n.right];
        if (Rt.depth > L.depth) {
            emit(n.right, shift + n.rshift, out);
            emit(n.left, shift, out);
        } else {
            emit(n.left, shift, out);
            emit(n.right, shift + n.rshift, out);
        }
        out->back().adds += 1;
    }

  private:
    static void split(Runs& rb, int64_t at) {
        auto it = rb.upper_bound(at);
        if (it == rb.begin()) return;
        --it;
        if (it->first < at && it->second.first > at) {
            int64_t end = it->second.first;
            Val v = it->second.second;
            it->second.first = at;
            rb[at] = {end, v};
        }
    }
    static void coalesce(Runs& rb, int64_t lo, int64_t hi) {
        auto it = rb.lower_bound(lo);
        if (it != rb.begin()) --it;
        while (it != rb.end() && it->first <= hi) {
            auto nx = std::next(it);
            if (nx == rb.end()) break;
            if (it->second.first == nx->first && it->second.second == nx->second.second) {
                it->second.first = nx->second.first;
                rb.erase(nx);
            } else {
                it = nx;
            }
        }
    }
    int P_;
    std::vector<Node> nodes_;
    std::map<std::tuple<int32_t, int32_t, int64_t>, int32_t> memo_;
    std::unordered_map<uint64_t, Runs> bufs_;
};

}  // namespace

Planner::Planner(int nranks, int ndims, const int* dims) {
    int d1[1] = {nranks};
    if (ndims <= 0)
        t_.init(1, d1);
    else
        t_.init(ndims, dims);
}

bool Planner::build(const PlanKey& k, Schedule* out, std::string* err) const {
    *out = Schedule();
    Gen g{t_, k, t_.size, t_.num_steps, out};
    try {
        if (k.ports < 1 || k.ports > kMaxPorts) throw PlanError("ports must be in [1, 6] (lib/libbine.cc:98)");
        if (k.root < 0 || k.root >= t_.size) throw PlanError("root out of range");
        if (k.family == kFamilyBruck && k.coll != kAlltoall)
            throw PlanError("the BRUCK family exists for alltoall only; the other entry points assert on it (e.g. lib/libbine.cc:1059, 1146, 1247)");
        if (k.family == kFamilyRing && k.coll != kAllreduce)
            throw PlanError(k.coll == kReduceScatter
                                ? "the RING reduce_scatter (bucket_reduce_scatter) never writes the caller's receive "
                                  "buffer: it points recvbuf at its own work area (lib/libbine_coll_reduce_scatter.cc:826, 832)"
                                : (k.coll == kAllgather
                                       ? "the RING allgather (bucket_allgather) gathers from a work area it never "
                                         "fills from sendbuf (lib/libbine_coll_allgather.cc:1514-1524)"
                                       : "the RING family exists for allreduce, reduce_scatter and allgather only; "
                                         "the other entry points assert on it (e.g. lib/libbine.cc:1284-1285)"));
        switch (k.coll) {
        case kAllreduce:
            if (k.family == kFamilyRing) gen_allreduce_ring(g);
            else if (k.variant == kArL) gen_allreduce_l(g);
            else if (k.variant == kArB || k.variant == kArBCoalesce || k.variant == kArBCont) gen_allreduce_b(g);
            else throw PlanError("unknown allreduce variant");
            break;
        case kReduceScatter: gen_reduce_scatter_cont(g); break;
        case kAllgather:
            if (k.variant == kAgBlocks) gen_allgather_blocks(g);
            else if (k.variant == kAgContSend) gen_allgather_cont_send(g);
            else gen_allgather_cont_permute(g);
            break;
        case kBcast:
            if (k.variant == kBcScatterAllgather) gen_bcast_scatter_allgather(g);
            else gen_bcast_tree(g);
            break;
        case kReduce:
            if (k.variant == kRdRedscatGather) gen_reduce_redscat_gather(g);
            else gen_reduce_tree(g);
            break;
        case kAlltoall:
            if (k.family == kFamilyBruck) gen_alltoall_bruck(g);
            else gen_alltoall(g);
            break;
        case kScatter: gen_scatter(g); break;
        case kGather: gen_gather(g); break;
        default: throw PlanError("unknown collective");
        }
    } catch (std::exception& e) {
        *err = e.what();
        return false;
    }
    return true;
}

bool Planner::trees(const PlanKey& k, const Schedule& s, TreePlan* out, std::string* err) const {
    *out = TreePlan();
    if (k.coll != kAllreduce && k.coll != kReduceScatter && k.coll != kReduce) {
        *err = "only reductions have addition trees";
        return false;
    }
    const int P = t_.size;
    SymExec ex(P);
    for (int r = 0; r < P; r++) ex.set(ex.buf(r, kBufSend), 0, s.send_elems, Val{ex.leaf(r), 0});
    for (const auto& lvl : s.levels) {
        // Moves of one level read the state before the level.  Apply them to
        // a snapshot-free order: hazards were removed by staging, so any
        // order gives the same result.
        for (const Move& m : lvl) ex.apply(m);
    }
    std::map<std::pair<int32_t, int64_t>, std::pair<int32_t, int32_t>> progs;
    auto prog_of = [&](Val v, int32_t* begin, int32_t* len, int32_t* depth) {
        auto key = std::make_pair(v.node, v.shift);
        auto it = progs.find(key);
        if (it == progs.end()) {
            int32_t b = (int32_t)out->prog.size();
            ex.emit(v.node, v.shift, &out->prog);
            it = progs.emplace(key, std::make_pair(b, (int32_t)out->prog.size() - b)).first;
        }
        *begin = it->second.first;
        *len = it->second.second;
        *depth = ex.node(v.node).depth;
    };
    std::vector<int> ranks;
    if (k.coll == kReduce) ranks.push_back(k.root);
    else
        for (int r = 0; r < P; r++) ranks.push_back(r);
    // Per rank runs of the receive buffer.
    std::vector<std::vector<std::tuple<int64_t, int64_t, Val>>> runs(P);
    for (int r : ranks) {
        auto& rb = ex.buf(r, kBufRecv);
        runs[r] = ex.get(rb, 0, s.recv_elems);
        for (auto& t : runs[r]) {
            if (std::get<2>(t).node < 0) {
                *err = "planner: an output element is never written";
                return false;
            }
            if (ex.node(std::get<2>(t).node).leaves != P) {
                *err = "planner: an output element does not sum every rank exactly once";
                return false;
            }
        }
    }
    // Allreduce: every rank must hold the same tree at each position, so one
    // evaluation serves all ranks.
    bool shared = k.coll == kAllreduce;
    if (shared) {
        for (int r = 1; r < P && shared; r++) {
            if (runs[r].size() != runs[0].size()) shared = false;
            for (size_t i = 0; shared && i < runs[r].size(); i++)
                if (!(std::get<0>(runs[r][i]) == std::get<0>(runs[0][i]) &&
                      std::get<1>(runs[r][i]) == std::get<1>(runs[0][i]) &&
                      std::get<2>(runs[r][i]) == std::get<2>(runs[0][i])))
                    shared = false;
        }
    }
    for (int r : ranks) {
        if (shared && r != 0) break;
        for (auto& t : runs[r]) {
            OutSegment sg;
            sg.off = std::get<0>(t);
            sg.n = std::get<1>(t) - std::get<0>(t);
            sg.rank = shared ? -1 : r;
            prog_of(std::get<2>(t), &sg.prog_begin, &sg.prog_len, &sg.depth);
            out->max_depth = std::max(out->max_depth, sg.depth);
            out->segs.push_back(sg);
        }
    }
    return true;
}

bool Planner::verify(const PlanKey& k, const Schedule& s, std::string* err) const {
    const int P = t_.size;
    const int64_t c = k.count;
    SymExec ex(P);
    if (k.coll == kBcast) {
        ex.set(ex.buf(k.root, kBufRecv), 0, s.recv_elems, Val{ex.leaf(k.root), 0});
    } else {
        for (int r = 0; r < P; r++) ex.set(ex.buf(r, kBufSend), 0, s.send_elems, Val{ex.leaf(r), 0});
    }
    for (const auto& lvl : s.levels)
        for (const Move& m : lvl) ex.apply(m);
    const bool reduction = k.coll == kAllreduce || k.coll == kReduceScatter || k.coll == kReduce;
    std::vector<int> ranks;
    if (k.coll == kReduce || k.coll == kGather) ranks.push_back(k.root);
    else
        for (int r = 0; r < P; r++) ranks.push_back(r);
    // Expected source (rank, shift) of output element p on rank r.
    auto expect = [&](int r, int64_t p, int* src, int64_t* shift) {
        switch (k.coll) {
        case kAllgather: *src = (int)(p / c); *shift = -(p / c) * c; break;
        case kBcast: *src = k.root; *shift = 0; break;
        case kAlltoall: *src = (int)(p / c); *shift = (int64_t)r * c - (p / c) * c; break;
        case kScatter: *src = k.root; *shift = (int64_t)r * c; break;
        case kGather: *src = (int)(p / c); *shift = -(p / c) * c; break;
        case kReduceScatter: *src = -1; *shift = (int64_t)r * c; break;
        default: *src = -1; *shift = 0; break;
        }
    };
    std::map<std::pair<int32_t, int64_t>, bool> checked;  // reduction trees already proven
    std::vector<char> seen;
    std::function<bool(int32_t, int64_t, int64_t)> walk = [&](int32_t id, int64_t sh, int64_t want) -> bool {
        const Node& n = ex.node(id);
        if (n.left < 0) {
            if (sh != want || seen[n.rank]) return false;
            seen[n.rank] = 1;
            return true;
        }
        return walk(n.left, sh, want) && walk(n.right, sh + n.rshift, want);
    };
    for (int r : ranks) {
        auto runs = ex.get(ex.buf(r, kBufRecv), 0, s.recv_elems);
        for (auto& t : runs) {
            const int64_t lo = std::get<0>(t), hi = std::get<1>(t);
            const Val v = std::get<2>(t);
            if (v.node < 0) {
                *err = "the reference's schedule leaves output elements unwritten here";
                return false;
            }
            if (reduction) {
                int src;
                int64_t want;
                expect(r, lo, &src, &want);
                auto key = std::make_pair(v.node, v.shift - want);
                if (checked.count(key)) continue;
                seen.assign(P, 0);
                if (ex.node(v.node).leaves != P || !walk(v.node, v.shift, want)) {
                    *err = "the reference's schedule does not sum every rank exactly once here (wrong data)";
                    return false;
                }
                checked[key] = true;
                continue;
            }
            // Copies: one source block per output block of c elements.
            for (int64_t p = lo; p < hi;) {
                int src;
                int64_t want;
                expect(r, p, &src, &want);
                const int64_t blk_end = (k.coll == kBcast || k.coll == kScatter) ? hi : std::min(hi, (p / c + 1) * c);
                const Node& n = ex.node(v.node);
                if (n.left >= 0 || n.rank != src || v.shift != want) {
                    *err = "the reference's schedule delivers the wrong block here (wrong data)";
                    return false;
                }
                p = blk_end;
            }
        }
    }
    return true;
}

bool link_bytes(const Torus& t, const std::vector<Message>& msgs, int es, std::vector<uint64_t>* out,
                std::string* err) {
    (void)err;
    out->assign((size_t)t.size * t.ndims * 2, 0);
    for (const Message& m : msgs) {
        if (m.src == m.dst || m.elems == 0) continue;
        int a[kMaxDims] = {0, 0, 0}, b[kMaxDims] = {0, 0, 0};
        t.coords(m.src, a);
        t.coords(m.dst, b);
        // Dimension-ordered route (dimension 0 first), minimal in each
        // dimension, the + direction on ties.  Bine and recursive-doubling
        // peers differ in one coordinate; 1-D algorithms run on a torus
        // (alltoall, scatter, gather) may differ in several.
        int c[kMaxDims] = {a[0], a[1], a[2]};
        for (int dim = 0; dim < t.ndims; dim++) {
            if (c[dim] == b[dim]) continue;
            const int L = t.dims[dim];
            int delta = pmod(b[dim] - c[dim], L);
            int dir = 1, hops = delta;
            if (L - delta < delta) {
                dir = -1;
                hops = L - delta;
            }
            for (int h = 0; h < hops; h++) {
                size_t link = ((size_t)t.id(c) * t.ndims + dim) * 2 + (dir > 0 ? 0 : 1);
                (*out)[link] += (uint64_t)m.elems * es;
                c[dim] = pmod(c[dim] + dir, L);
            }
        }
    }
    return true;
}

// ------------------------------------------------------------ tree split
namespace {

struct TNode {
    int32_t l, r, leaves, entry;  // entry: index of the leaf's program entry (-1 for additions)
};

// Parses one postfix program into a binary tree; returns the root or -1.
int parse_tree(const std::vector<ProgEntry>& prog, int begin, int len, std::vector<TNode>* nodes) {
    std::vector<int> st;
    for (int i = begin; i < begin + len; i++) {
        nodes->push_back(TNode{-1, -1, 1, i});
        st.push_back((int)nodes->size() - 1);
        for (int a = 0; a < prog[i].adds; a++) {
            if (st.size() < 2) return -1;
            const int r = st.back();
            st.pop_back();
            const int l = st.back();
            st.pop_back();
            nodes->push_back(TNode{l, r, (*nodes)[l].leaves + (*nodes)[r].leaves, -1});
            st.push_back((int)nodes->size() - 1);
        }
    }
    return st.size() == 1 ? st[0] : -1;
}

// Postfix emission with the parse's child order (left subtree first), so
// the evaluation order and stack depth of every subtree are unchanged.
void emit_subtree(const std::vector<TNode>& nodes, const std::vector<ProgEntry>& prog, int n,
                  std::vector<ProgEntry>* out) {
    std::vector<std::pair<int, bool>> todo{{n, false}};
    while (!todo.empty()) {
        auto [x, expanded] = todo.back();
        todo.pop_back();
        const TNode& t = nodes[x];
        if (t.entry >= 0) {
            ProgEntry e = prog[t.entry];
            e.adds = 0;
            out->push_back(e);
        } else if (expanded) {
            out->back().adds++;
        } else {
            todo.push_back({x, true});
            todo.push_back({t.r, false});
            todo.push_back({t.l, false});
        }
    }
}

void emit_combine(const std::vector<TNode>& nodes, int n, const std::unordered_map<int, int>& part_of,
                  std::vector<std::pair<int32_t, int32_t>>* out) {
    std::vector<std::pair<int, bool>> todo{{n, false}};
    while (!todo.empty()) {
        auto [x, expanded] = todo.back();
        todo.pop_back();
        auto it = part_of.find(x);
        if (it != part_of.end()) {
            out->push_back({it->second, 0});
        } else if (expanded) {
            out->back().second++;
        } else {
            todo.push_back({x, true});
            todo.push_back({nodes[x].r, false});
            todo.push_back({nodes[x].l, false});
        }
    }
}

int stack_depth(const ProgEntry* p, int len) {
    int sp = 0, mx = 0;
    for (int i = 0; i < len; i++) {
        mx = std::max(mx, ++sp);
        sp -= p[i].adds;
    }
    return mx;
}

}  // namespace

bool split_trees(const TreePlan& tp, int K, SplitTrees* out, std::string* err) {
    out->K = K;
    out->prog.clear();
    out->parts.clear();
    out->comb.clear();
    out->max_depth = 0;
    // Distinct programs are split once and shared by their segments.
    std::map<std::pair<int32_t, int32_t>, std::pair<std::vector<int32_t>, std::vector<std::pair<int32_t, int32_t>>>>
        done;
    for (const OutSegment& sg : tp.segs) {
        const auto key = std::make_pair(sg.prog_begin, sg.prog_len);
        auto it = done.find(key);
        if (it == done.end()) {
            std::vector<TNode> nodes;
            const int root = parse_tree(tp.prog, sg.prog_begin, sg.prog_len, &nodes);
            if (root < 0) {
                *err = "malformed reduction program";
                return false;
            }
            // Cut the largest remaining subtree until there are K parts.
            std::vector<int> fr{root};
            while ((int)fr.size() < K) {
                int best = -1;
                for (int i = 0; i < (int)fr.size(); i++)
                    if (nodes[fr[i]].entry < 0 && (best < 0 || nodes[fr[i]].leaves > nodes[fr[best]].leaves)) best = i;
                if (best < 0) {
                    *err = "reduction tree has fewer leaves than parts";
                    return false;
                }
                const TNode t = nodes[fr[best]];
                fr[best] = t.l;
                fr.insert(fr.begin() + best + 1, t.r);
            }
            std::vector<int32_t> offs;
            std::unordered_map<int, int> part_of;
            for (int j = 0; j < K; j++) {
                offs.push_back((int32_t)out->prog.size());
                part_of[fr[j]] = j;
                emit_subtree(nodes, tp.prog, fr[j], &out->prog);
                out->max_depth = std::max(out->max_depth, stack_depth(out->prog.data() + offs.back(),
                                                                      (int)out->prog.size() - offs.back()));
            }
            offs.push_back((int32_t)out->prog.size());
            std::vector<std::pair<int32_t, int32_t>> comb;
            emit_combine(nodes, root, part_of, &comb);
            // Self-check: parts substituted into the combine program must
            // reproduce the original program exactly.
            std::vector<ProgEntry> back;
            for (const auto& [j, adds] : comb) {
                back.insert(back.end(), out->prog.begin() + offs[j], out->prog.begin() + offs[j + 1]);
                back.back().adds += adds;
            }
            bool same = (int)back.size() == sg.prog_len && (int)comb.size() == K;
            for (int i = 0; same && i < sg.prog_len; i++) {
                const ProgEntry& a = back[i];
                const ProgEntry& b = tp.prog[sg.prog_begin + i];
                same = a.rank == b.rank && a.shift == b.shift && a.adds == b.adds;
            }
            if (!same) {
                *err = "split reduction tree does not recompose to the original";
                return false;
            }
            it = done.emplace(key, std::make_pair(offs, comb)).first;
        }
        out->parts.insert(out->parts.end(), it->second.first.begin(), it->second.first.end());
        out->comb.insert(out->comb.end(), it->second.second.begin(), it->second.second.end());
    }
    return true;
}

}  // namespace bine

// ------------------------------------------------------------- dataflow plan
namespace bine {
namespace {

// State of one row (buffer, rank) between levels: sorted, disjoint element
// ranges with their last writer and the readers since.  Untouched gaps have
// no writer and no readers.
struct FlowSpan {
    int64_t s, e;
    int32_t writer;                // last item that wrote the range, -1: none
    std::vector<int32_t> readers;  // items that read it since
};

// One access of one level: elements [s, e) of row `row`.
struct FlowAccess {
    int64_t s, e;
    int32_t item;
    bool write;
};

// Balanced packing of one level (build_flow_fused without a segment size):
// every element of move m costs weights[m] element accesses (its leaves and
// destinations).  The level is cut into items of equal access counts, as
// many as a whole multiple of `target_items` (the kernel's resident blocks)
// that keeps items at or below 2 * max_item_elems accesses, so that the
// items of a level run in whole waves.  A move is cut where an item fills,
// at multiples of min_item_elems from the move's start.
void pack_balanced(const std::vector<int64_t>& sizes, const std::vector<int32_t>& weights, int32_t first_move,
                   int level, int64_t min_item_elems, int64_t max_item_elems, int target_items, int max_pieces,
                   FlowPlan* out, int32_t* nitems) {
    int64_t level_w = 0;
    for (size_t m = 0; m < sizes.size(); m++) level_w += sizes[m] * weights[m];
    const int64_t cap_w = 2 * max_item_elems;
    const int64_t tw = (int64_t)target_items * cap_w;
    // Every move opens at most one piece beyond its share of the items, so
    // goal * (max_pieces - 1) >= moves keeps items within max_pieces.
    const int64_t tp = (int64_t)target_items * std::max(1, max_pieces - 1);
    const int64_t waves = std::max<int64_t>({1, (level_w + tw - 1) / tw, ((int64_t)sizes.size() + tp - 1) / tp});
    // Levels too small for that get items of 2 * min_item_elems accesses.
    const int64_t goal = std::max<int64_t>(1, std::min(waves * target_items, level_w / (2 * min_item_elems)));
    // Item k ends where the level's accesses reach (k + 1) / goal of the
    // total; a move is cut at the multiple of min_item_elems nearest that
    // boundary.  An item that reaches max_pieces first is continued by a
    // new item toward the same boundary.
    auto bound = [&](int64_t k) { return std::max<int64_t>(1, (k + 1) * level_w / goal); };
    int64_t pos = 0, k = 0;  // accesses placed; boundary of the open item
    bool full = true;        // the next piece opens a new item
    *nitems = 0;
    for (size_t m = 0; m < sizes.size(); m++) {
        const int64_t mn = sizes[m], w = std::max<int32_t>(1, weights[m]);
        for (int64_t st = 0; st < mn;) {
            const bool capped = *nitems > 0 && out->items.back().pend - out->items.back().pbeg >= max_pieces;
            if (full || capped) {
                if (full && *nitems > 0) k++;
                const int32_t p = (int32_t)out->pieces.size();
                out->items.push_back(FlowItem{p, p, 0, 0, (int32_t)level, 0});
                ++*nitems;
                full = false;
            }
            const int64_t room = bound(k) - pos;
            int64_t n = mn - st;
            if (n * w > room) {
                n = std::min(n, (room / w + min_item_elems / 2) / min_item_elems * min_item_elems);
                if (n <= 0) {
                    if (out->items.back().pend > out->items.back().pbeg) {
                        full = true;
                        continue;
                    }
                    n = std::min(mn - st, min_item_elems);
                }
            }
            out->pieces.push_back(FlowPiece{first_move + (int32_t)m, 0, st, n});
            out->items.back().pend++;
            pos += n * w;
            st += n;
            if (pos >= bound(k)) full = true;
        }
    }
}

// The shared core of build_flow and build_flow_fused: `sizes[l]` are the
// element counts of level l's moves (numbered in level order), and
// visit(move, start, n, fn) calls fn(rank, buf, offset, n, write) for every
// row range the elements [start, start + n) of that move read or write.
// With `weights` (element accesses per element of each move) and no piece
// size, levels are packed by pack_balanced.
template <typename Visit>
void build_flow_impl(const std::vector<std::vector<int64_t>>& sizes, int P, int64_t piece_elems,
                     int64_t min_item_elems, int64_t max_item_elems, int target_items, int max_pieces, Visit visit,
                     FlowPlan* out, const std::vector<std::vector<int32_t>>* weights = nullptr) {
    *out = FlowPlan();
    max_pieces = std::max(1, std::min(max_pieces, kFlowMaxPieces));
    const bool auto_pieces = piece_elems <= 0;
    target_items = std::max(1, target_items);
    min_item_elems = std::max<int64_t>(1, min_item_elems);
    max_item_elems = std::max(min_item_elems, max_item_elems);
    // Pieces and items, level by level.
    int32_t nmoves = 0;                // level-order move index
    std::vector<int32_t> level_first;  // first item of each level
    for (size_t l = 0; l < sizes.size(); l++) {
        level_first.push_back((int32_t)out->items.size());
        if (weights && auto_pieces) {
            int32_t nitems = 0;
            pack_balanced(sizes[l], (*weights)[l], nmoves, (int)l, min_item_elems, max_item_elems, target_items,
                          max_pieces, out, &nitems);
            nmoves += (int32_t)sizes[l].size();
            out->level_items.push_back(nitems);
            continue;
        }
        int64_t level_elems = 0;
        for (int64_t n : sizes[l]) level_elems += n;
        int64_t item_elems = std::max(min_item_elems, (level_elems + target_items - 1) / target_items);
        if (auto_pieces) {
            // Whole multiples of min_item_elems, so that pieces cut from a
            // move start on the same alignment as the move.
            item_elems = std::min(max_item_elems, (item_elems + min_item_elems - 1) / min_item_elems * min_item_elems);
            piece_elems = item_elems;
        } else {
            item_elems = std::min(item_elems, piece_elems);
        }
        int32_t nitems = 0;
        int64_t cur = 0;  // elements in the open item
        for (int64_t mn : sizes[l]) {
            const int32_t mi = nmoves++;
            for (int64_t st = 0; st < mn; st += piece_elems) {
                const int64_t n = std::min(piece_elems, mn - st);
                if (nitems == 0 || cur + n > item_elems ||
                    out->items.back().pend - out->items.back().pbeg >= max_pieces) {
                    const int32_t p = (int32_t)out->pieces.size();
                    out->items.push_back(FlowItem{p, p, 0, 0, (int32_t)l, 0});
                    nitems++;
                    cur = 0;
                }
                out->pieces.push_back(FlowPiece{mi, 0, st, n});
                out->items.back().pend++;
                cur += n;
            }
        }
        out->level_items.push_back(nitems);
    }
    level_first.push_back((int32_t)out->items.size());
    // Dependencies, one level at a time: every access of the level is
    // checked against the state its rows had before the level (moves of one
    // level are independent), then each touched row's state is rebuilt in
    // one sweep.  Rows are (buffer, rank).
    const size_t nrows = kNumBufs * (size_t)P;
    std::vector<std::vector<FlowSpan>> rows(nrows);
    std::vector<std::vector<FlowAccess>> acc(nrows);
    std::vector<size_t> touched;
    std::vector<std::vector<int32_t>> cand;
    std::vector<int64_t> bounds, abounds, obounds;
    std::vector<FlowSpan> next;
    for (size_t l = 0; l + 1 < level_first.size(); l++) {
        const int32_t i0 = level_first[l], i1 = level_first[l + 1];
        if (i0 == i1) continue;
        touched.clear();
        for (int32_t i = i0; i < i1; i++)
            for (int32_t p = out->items[i].pbeg; p < out->items[i].pend; p++) {
                const FlowPiece& pc = out->pieces[p];
                visit(pc.move, pc.start, pc.n, [&](int rank, int buf, int64_t off, int64_t n, bool write) {
                    const size_t row = (size_t)buf * P + rank;
                    if (acc[row].empty()) touched.push_back(row);
                    acc[row].push_back(FlowAccess{off, off + n, i, write});
                });
            }
        cand.assign(i1 - i0, {});
        for (size_t row : touched) {
            std::vector<FlowAccess>& A = acc[row];
            std::vector<FlowSpan>& old = rows[row];
            std::sort(A.begin(), A.end(), [](const FlowAccess& x, const FlowAccess& y) { return x.s < y.s; });
            // Read after write on the last writers; write after write and
            // write after read on the last writer and its readers.
            for (const FlowAccess& a : A) {
                auto it = std::upper_bound(old.begin(), old.end(), a.s,
                                           [](int64_t v, const FlowSpan& sp) { return v < sp.e; });
                std::vector<int32_t>& c = cand[a.item - i0];
                for (; it != old.end() && it->s < a.e; ++it) {
                    if (it->writer >= 0) c.push_back(it->writer);
                    if (a.write) c.insert(c.end(), it->readers.begin(), it->readers.end());
                }
            }
            // New state: the elementary ranges between all boundaries; a
            // range written this level belongs to its writer alone, others
            // keep their writer and add this level's readers.
            // The old spans' boundaries are already in order: sort only the
            // accesses' and merge.
            abounds.clear();
            for (const FlowAccess& a : A) abounds.push_back(a.s), abounds.push_back(a.e);
            std::sort(abounds.begin(), abounds.end());
            obounds.clear();
            for (const FlowSpan& sp : old) obounds.push_back(sp.s), obounds.push_back(sp.e);
            bounds.resize(abounds.size() + obounds.size());
            std::merge(obounds.begin(), obounds.end(), abounds.begin(), abounds.end(), bounds.begin());
            bounds.erase(std::unique(bounds.begin(), bounds.end()), bounds.end());
            next.clear();
            size_t oi = 0, ai = 0;
            std::vector<const FlowAccess*> live;  // accesses covering the current range
            for (size_t b = 0; b + 1 < bounds.size(); b++) {
                const int64_t x0 = bounds[b], x1 = bounds[b + 1];
                while (oi < old.size() && old[oi].e <= x0) oi++;
                const FlowSpan* os = oi < old.size() && old[oi].s <= x0 ? &old[oi] : nullptr;
                while (ai < A.size() && A[ai].s <= x0) live.push_back(&A[ai++]);
                live.erase(std::remove_if(live.begin(), live.end(), [&](const FlowAccess* a) { return a->e <= x0; }),
                           live.end());
                if (!os && live.empty()) continue;  // a gap nobody touches
                FlowSpan sp{x0, x1, os ? os->writer : -1, {}};
                const FlowAccess* w = nullptr;
                for (const FlowAccess* a : live)
                    if (a->write) w = a;
                if (w) {
                    sp.writer = w->item;
                } else {
                    if (os) sp.readers = os->readers;
                    for (const FlowAccess* a : live)
                        if (std::find(sp.readers.begin(), sp.readers.end(), a->item) == sp.readers.end())
                            sp.readers.push_back(a->item);
                }
                if (!next.empty() && next.back().e == x0 && next.back().writer == sp.writer &&
                    next.back().readers == sp.readers)
                    next.back().e = x1;
                else
                    next.push_back(std::move(sp));
            }
            old.swap(next);
            A.clear();
        }
        // Earlier levels only, one entry per item, and a level entry where
        // one level would contribute more than kFlowLevelDep items.
        for (int32_t i = i0; i < i1; i++) {
            std::vector<int32_t>& c = cand[i - i0];
            std::sort(c.begin(), c.end());
            c.erase(std::unique(c.begin(), c.end()), c.end());
            FlowItem& it = out->items[i];
            it.dbeg = (int32_t)out->deps.size();
            size_t j = 0;
            while (j < c.size()) {
                const int32_t lv = out->items[c[j]].level;
                size_t k = j;
                while (k < c.size() && out->items[c[k]].level == lv) k++;
                if (lv < it.level) {
                    if (k - j > (size_t)kFlowLevelDep)
                        out->deps.push_back(-(lv + 1));
                    else
                        out->deps.insert(out->deps.end(), c.begin() + j, c.begin() + k);
                }
                j = k;
            }
            it.dend = (int32_t)out->deps.size();
        }
    }
}

}  // namespace

void build_flow(const Schedule& s, int P, int64_t piece_elems, int64_t min_item_elems, int64_t max_item_elems,
                int target_items, int max_pieces, FlowPlan* out) {
    std::vector<std::vector<int64_t>> sizes(s.levels.size());
    std::vector<const Move*> move_of;
    for (size_t l = 0; l < s.levels.size(); l++)
        for (const Move& m : s.levels[l]) {
            sizes[l].push_back(m.n);
            move_of.push_back(&m);
        }
    build_flow_impl(sizes, P, piece_elems, min_item_elems, max_item_elems, target_items, max_pieces,
                    [&](int32_t mi, int64_t st, int64_t n, auto fn) {
                        const Move& m = *move_of[mi];
                        fn(m.a.rank, m.a.buf, m.a.off + st, n, false);
                        if (m.add) fn(m.b.rank, m.b.buf, m.b.off + st, n, false);
                        fn(m.dst.rank, m.dst.buf, m.dst.off + st, n, true);
                    },
                    out);
}

void build_flow_fused(const FusedSchedule& f, int P, int64_t piece_elems, int64_t min_item_elems,
                      int64_t max_item_elems, int target_items, int max_pieces, FlowPlan* out) {
    std::vector<std::vector<int64_t>> sizes(f.passes.size());
    std::vector<std::vector<int32_t>> weights(f.passes.size());
    std::vector<const FusedMove*> move_of;
    for (size_t l = 0; l < f.passes.size(); l++)
        for (const FusedMove& m : f.passes[l]) {
            sizes[l].push_back(m.n);
            weights[l].push_back(m.nleaves + m.ndst);
            move_of.push_back(&m);
        }
    build_flow_impl(sizes, P, piece_elems, min_item_elems, max_item_elems, target_items, max_pieces,
                    [&](int32_t mi, int64_t st, int64_t n, auto fn) {
                        const FusedMove& m = *move_of[mi];
                        for (int32_t j = 0; j < m.nleaves; j++) {
                            const FusedLeaf& lf = f.leaves[m.leaf_begin + j];
                            fn(lf.rank, lf.buf, lf.off + st, n, false);
                        }
                        for (int32_t j = 0; j < m.ndst; j++) {
                            const FusedDst& d = f.dsts[m.dst_begin + j];
                            fn(d.rank, d.buf, d.off + st, n, true);
                        }
                    },
                    out, &weights);
}

}  // namespace bine

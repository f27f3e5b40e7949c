// Level fusion for the pipelined engine (declared in bine_plan.h).
//
// A pass of consecutive levels is executed symbolically from fresh leaves:
// every element of every (rank, buffer) row starts as "the state of that
// element at the start of the pass".  What the pass's levels leave behind is
// then an expression over those leaves per element run.  Backward liveness
// over the passes keeps only the runs that a later pass reads or that are
// results; everything else (partial sums handed from one step to the next
// inside the pass, staged messages, copies overwritten before use) is never
// written.  The kept runs become fused moves: a postfix program over leaves
// (at most kFuseMaxLeaves, stack depth at most kFuseMaxDepth) and the rows
// it is written to.  Passes whose kept writes overlap what another of their
// moves reads, or whose programs are too large, are split until none is.
// Finally the fused schedule is executed symbolically from the collective's
// inputs beside the original one, in one hash-consed expression table, and
// every result element must come out as the same addition tree.
#include <algorithm>
#include <climits>
#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "bine_plan.h"

namespace bine {
namespace {

struct FNode {
    int32_t left, right;  // -1 for leaves
    int64_t rshift;       // shift of the right child relative to the left one
    int32_t rank;         // leaves
    uint8_t buf;          // leaves
    int32_t leaves, depth;
};

struct FVal {
    int32_t node;
    int64_t shift;  // the value at position p is the node evaluated at p + shift
    bool operator==(const FVal& o) const { return node == o.node && shift == o.shift; }
    bool operator!=(const FVal& o) const { return !(*this == o); }
};

uint64_t row_key(int rank, int buf) { return ((uint64_t)(uint32_t)rank << 8) | (uint64_t)buf; }

// Symbolic state of all rows.  Only written runs are stored; an unwritten
// position p of row (r, b) holds leaf(r, b) evaluated at p.
class Exec {
  public:
    using Runs = std::map<int64_t, std::pair<int64_t, FVal>>;  // start -> (end, value)
    struct Piece {
        int64_t s, e;
        FVal v;
    };

    int32_t leaf(int rank, int buf) {
        const uint64_t k = row_key(rank, buf);
        auto it = leaf_ids_.find(k);
        if (it != leaf_ids_.end()) return it->second;
        nodes_.push_back(FNode{-1, -1, 0, rank, (uint8_t)buf, 1, 1});
        const int32_t id = (int32_t)nodes_.size() - 1;
        leaf_ids_[k] = id;
        return id;
    }
    const FNode& node(int32_t id) const { return nodes_[id]; }
    void clear_state() { rows_.clear(); }
    const std::unordered_map<uint64_t, Runs>& rows() const { return rows_; }

    std::vector<Piece> get(int rank, int buf, int64_t lo, int64_t hi) {
        std::vector<Piece> out;
        const FVal id{leaf(rank, buf), 0};
        auto rit = rows_.find(row_key(rank, buf));
        if (rit == rows_.end()) {
            out.push_back(Piece{lo, hi, id});
            return out;
        }
        const Runs& rb = rit->second;
        int64_t cur = lo;
        auto it = rb.upper_bound(lo);
        if (it != rb.begin()) {
            auto pv = std::prev(it);
            if (pv->second.first > lo) it = pv;
        }
        for (; it != rb.end() && it->first < hi; ++it) {
            const int64_t s = std::max(it->first, lo), e = std::min(it->second.first, hi);
            if (s > cur) out.push_back(Piece{cur, s, id});
            out.push_back(Piece{s, e, it->second.second});
            cur = e;
        }
        if (cur < hi) out.push_back(Piece{cur, hi, id});
        return out;
    }

    void set(int rank, int buf, int64_t lo, int64_t hi, FVal v) {
        if (lo >= hi) return;
        Runs& rb = rows_[row_key(rank, buf)];
        split(rb, lo);
        split(rb, hi);
        auto it = rb.lower_bound(lo);
        while (it != rb.end() && it->first < hi) it = rb.erase(it);
        rb[lo] = {hi, v};
    }

    FVal add(FVal a, FVal b) {
        if (std::make_pair(b.node, b.shift) < std::make_pair(a.node, a.shift)) std::swap(a, b);
        const int64_t rel = b.shift - a.shift;
        const auto key = std::make_tuple(a.node, b.node, rel);
        auto it = memo_.find(key);
        if (it != memo_.end()) return FVal{it->second, a.shift};
        const FNode& A = nodes_[a.node];
        const FNode& B = nodes_[b.node];
        FNode n{a.node, b.node, rel, -1, 0, A.leaves + B.leaves,
                A.depth == B.depth ? A.depth + 1 : std::max(A.depth, B.depth)};
        nodes_.push_back(n);
        const int32_t id = (int32_t)nodes_.size() - 1;
        memo_[key] = id;
        return FVal{id, a.shift};
    }

    // The value of rows a (and b) over n elements, as runs relative to
    // position 0 of the destination at `dst_off`.
    std::vector<Piece> value_of(const Region& a, const Region* b, int64_t n, int64_t dst_off) {
        std::vector<Piece> out;
        auto pa = get(a.rank, a.buf, a.off, a.off + n);
        if (!b) {
            for (Piece p : pa) {
                p.v.shift += a.off - dst_off;
                out.push_back(Piece{p.s - a.off, p.e - a.off, p.v});
            }
            return out;
        }
        auto pb = get(b->rank, b->buf, b->off, b->off + n);
        size_t ia = 0, ib = 0;
        int64_t cur = 0;
        while (cur < n) {
            while (pa[ia].e - a.off <= cur) ia++;
            while (pb[ib].e - b->off <= cur) ib++;
            const int64_t e = std::min(pa[ia].e - a.off, pb[ib].e - b->off);
            FVal va = pa[ia].v, vb = pb[ib].v;
            va.shift += a.off - dst_off;
            vb.shift += b->off - dst_off;
            out.push_back(Piece{cur, e, add(va, vb)});
            cur = e;
        }
        return out;
    }

    // One level: every move reads the state before the level.
    void apply_level(const std::vector<Move>& lvl) {
        std::vector<std::pair<const Move*, std::vector<Piece>>> vals;
        vals.reserve(lvl.size());
        for (const Move& m : lvl) vals.emplace_back(&m, value_of(m.a, m.add ? &m.b : nullptr, m.n, m.dst.off));
        for (auto& mv : vals)
            for (const Piece& p : mv.second)
                set(mv.first->dst.rank, mv.first->dst.buf, mv.first->dst.off + p.s, mv.first->dst.off + p.e, p.v);
    }

    // Leaves of a value: (rank, buf, absolute offset of position 0).
    void leaves_of(int32_t id, int64_t shift, std::vector<std::tuple<int32_t, uint8_t, int64_t>>* out) const {
        const FNode& n = nodes_[id];
        if (n.left < 0) {
            out->emplace_back(n.rank, n.buf, shift);
            return;
        }
        leaves_of(n.left, shift, out);
        leaves_of(n.right, shift + n.rshift, out);
    }

    // Postfix program, deeper child first (Sethi-Ullman order), leaves at
    // absolute offsets for position 0 of the destination.
    void emit(int32_t id, int64_t shift, std::vector<FusedLeaf>* out) const {
        const FNode& n = nodes_[id];
        if (n.left < 0) {
            out->push_back(FusedLeaf{n.rank, n.buf, 0, {0, 0}, shift});
            return;
        }
        const FNode& L = nodes_[n.left];
        const FNode& R = nodes_[n.right];
        if (R.depth > L.depth) {
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
            const int64_t end = it->second.first;
            const FVal v = it->second.second;
            it->second.first = at;
            rb[at] = {end, v};
        }
    }
    std::vector<FNode> nodes_;
    std::map<std::tuple<int32_t, int32_t, int64_t>, int32_t> memo_;
    std::unordered_map<uint64_t, int32_t> leaf_ids_;
    std::unordered_map<uint64_t, Runs> rows_;
};

// Disjoint, merged element intervals of one row.
using ISet = std::map<int64_t, int64_t>;

void iset_add(ISet& s, int64_t lo, int64_t hi) {
    if (lo >= hi) return;
    auto it = s.upper_bound(lo);
    if (it != s.begin()) {
        auto pv = std::prev(it);
        if (pv->second >= lo) {
            lo = pv->first;
            hi = std::max(hi, pv->second);
            it = s.erase(pv);
        }
    }
    while (it != s.end() && it->first <= hi) {
        hi = std::max(hi, it->second);
        it = s.erase(it);
    }
    s[lo] = hi;
}

void iset_sub(ISet& s, int64_t lo, int64_t hi) {
    if (lo >= hi) return;
    auto it = s.upper_bound(lo);
    if (it != s.begin()) --it;
    while (it != s.end() && it->first < hi) {
        const int64_t a = it->first, b = it->second;
        if (b <= lo) {
            ++it;
            continue;
        }
        it = s.erase(it);
        if (a < lo) s[a] = lo;
        if (b > hi) {
            s[hi] = b;
            break;
        }
    }
}

std::vector<std::pair<int64_t, int64_t>> iset_meet(const ISet& s, int64_t lo, int64_t hi) {
    std::vector<std::pair<int64_t, int64_t>> out;
    auto it = s.upper_bound(lo);
    if (it != s.begin()) --it;
    for (; it != s.end() && it->first < hi; ++it) {
        const int64_t a = std::max(it->first, lo), b = std::min(it->second, hi);
        if (a < b) out.emplace_back(a, b);
    }
    return out;
}

struct Write {
    int32_t rank;
    uint8_t buf;
    int64_t s, e;
    FVal v;
};

struct PassSym {
    std::unique_ptr<Exec> ex;
    std::vector<Write> writes;  // every run the pass changes, sorted by row and offset
};

PassSym run_pass(const Schedule& sch, int a, int b) {
    PassSym ps;
    ps.ex.reset(new Exec());
    Exec& ex = *ps.ex;
    for (int l = a; l < b; l++) ex.apply_level(sch.levels[l]);
    for (const auto& kv : ex.rows()) {
        const int rank = (int)(kv.first >> 8), buf = (int)(kv.first & 0xFF);
        const FVal id{ex.leaf(rank, buf), 0};
        for (const auto& r : kv.second)
            if (r.second.second != id) ps.writes.push_back(Write{rank, (uint8_t)buf, r.first, r.second.first, r.second.second});
    }
    std::sort(ps.writes.begin(), ps.writes.end(), [](const Write& x, const Write& y) {
        return std::make_tuple(x.rank, x.buf, x.s) < std::make_tuple(y.rank, y.buf, y.s);
    });
    return ps;
}

// Where logical elements live.  A kept write that would overwrite an
// element another move of its pass still reads goes to a fresh slot of its
// rank's workspace instead ("renaming"); later passes read it there.  An
// unrenamed element lives at its own position.  Logical x of a renamed run
// lives at (rank, buf, x + delta).
struct Phys {
    int32_t rank;
    uint8_t buf;
    int64_t delta;
};
using PhysRuns = std::map<int64_t, std::pair<int64_t, Phys>>;

void runs_cut(PhysRuns& rb, int64_t at) {
    auto it = rb.upper_bound(at);
    if (it == rb.begin()) return;
    --it;
    if (it->first < at && it->second.first > at) {
        const int64_t end = it->second.first;
        const Phys v = it->second.second;
        it->second.first = at;
        rb[at] = {end, v};
    }
}

class Placement {
  public:
    // Pieces (start, end, place) covering [lo, hi) of a logical row.
    void lookup(int rank, int buf, int64_t lo, int64_t hi, std::vector<std::tuple<int64_t, int64_t, Phys>>* out) const {
        out->clear();
        const Phys home{rank, (uint8_t)buf, 0};
        auto rit = rows_.find(row_key(rank, buf));
        if (rit == rows_.end()) {
            out->emplace_back(lo, hi, home);
            return;
        }
        const PhysRuns& rb = rit->second;
        int64_t cur = lo;
        auto it = rb.upper_bound(lo);
        if (it != rb.begin()) {
            auto pv = std::prev(it);
            if (pv->second.first > lo) it = pv;
        }
        for (; it != rb.end() && it->first < hi; ++it) {
            const int64_t a = std::max(it->first, lo), b = std::min(it->second.first, hi);
            if (a > cur) out->emplace_back(cur, a, home);
            out->emplace_back(a, b, it->second.second);
            cur = b;
        }
        if (cur < hi) out->emplace_back(cur, hi, home);
    }
    // Logical [lo, hi) now lives at `p` (its own position when p is home).
    void place(int rank, int buf, int64_t lo, int64_t hi, Phys p) {
        if (lo >= hi) return;
        PhysRuns& rb = rows_[row_key(rank, buf)];
        runs_cut(rb, lo);
        runs_cut(rb, hi);
        auto it = rb.lower_bound(lo);
        while (it != rb.end() && it->first < hi) it = rb.erase(it);
        if (!(p.rank == rank && p.buf == buf && p.delta == 0)) rb[lo] = {hi, p};
    }
    const std::unordered_map<uint64_t, PhysRuns>& rows() const { return rows_; }

  private:
    std::unordered_map<uint64_t, PhysRuns> rows_;
};

// A piece of a kept run with its leaves placed: destination logical row
// and range, and the program over physical leaves (offsets for position 0).
struct Sub {
    int32_t rank;
    uint8_t buf;
    int64_t s, e;
    std::vector<FusedLeaf> prog;
    int32_t group = -1;
    Phys dst{0, 0, 0};  // where the value is written
};

// Places one pass's kept runs: splits them where their leaves' placements
// change, groups identical programs at identical leaf positions (one move,
// several destinations), and sends every write that would clobber an
// element read in the pass (other than a move updating its own elements
// index for index) to a fresh workspace slot.
void place_pass(const Exec& ex, const std::vector<Write>& kept, Placement& pl, int64_t slot_base,
                std::vector<int64_t>& cursor, std::vector<Sub>* subs) {
    subs->clear();
    std::vector<FusedLeaf> lprog;
    std::vector<std::tuple<int64_t, int64_t, Phys>> pieces;
    for (const Write& w : kept) {
        lprog.clear();
        ex.emit(w.v.node, w.s + w.v.shift, &lprog);
        const int64_t n = w.e - w.s;
        std::vector<int64_t> cuts{0, n};
        std::vector<std::vector<std::tuple<int64_t, int64_t, Phys>>> lp(lprog.size());
        for (size_t j = 0; j < lprog.size(); j++) {
            pl.lookup(lprog[j].rank, lprog[j].buf, lprog[j].off, lprog[j].off + n, &lp[j]);
            for (auto& t : lp[j]) cuts.push_back(std::get<0>(t) - lprog[j].off);
        }
        std::sort(cuts.begin(), cuts.end());
        cuts.erase(std::unique(cuts.begin(), cuts.end()), cuts.end());
        std::vector<size_t> at(lprog.size(), 0);
        for (size_t c = 0; c + 1 < cuts.size(); c++) {
            const int64_t c0 = cuts[c], c1 = cuts[c + 1];
            Sub sb;
            sb.rank = w.rank;
            sb.buf = w.buf;
            sb.s = w.s + c0;
            sb.e = w.s + c1;
            for (size_t j = 0; j < lprog.size(); j++) {
                while (std::get<1>(lp[j][at[j]]) - lprog[j].off <= c0) at[j]++;
                const Phys& ph = std::get<2>(lp[j][at[j]]);
                FusedLeaf lf = lprog[j];
                lf.rank = ph.rank;
                lf.buf = ph.buf;
                lf.off = lprog[j].off + c0 + ph.delta;
                sb.prog.push_back(lf);
            }
            subs->push_back(std::move(sb));
        }
    }
    // Groups: the same physical program over the same length.
    std::map<std::vector<std::tuple<int32_t, uint8_t, uint8_t, int64_t>>, std::vector<size_t>> groups;
    for (size_t i = 0; i < subs->size(); i++) {
        const Sub& sb = (*subs)[i];
        std::vector<std::tuple<int32_t, uint8_t, uint8_t, int64_t>> key;
        key.emplace_back(-1, 0, 0, sb.e - sb.s);
        for (const FusedLeaf& lf : sb.prog) key.emplace_back(lf.rank, lf.buf, lf.adds, lf.off);
        groups[key].push_back(i);
    }
    int32_t gid = 0;
    std::vector<size_t> gsize;
    for (auto& g : groups) {
        for (size_t i : g.second) (*subs)[i].group = gid;
        gsize.push_back(g.second.size());
        gid++;
    }
    // Physical reads of the pass, per row: (start, end, group).
    std::unordered_map<uint64_t, std::vector<std::tuple<int64_t, int64_t, int32_t>>> reads;
    for (const Sub& sb : *subs)
        for (const FusedLeaf& lf : sb.prog)
            reads[row_key(lf.rank, lf.buf)].emplace_back(lf.off, lf.off + (sb.e - sb.s), sb.group);
    std::unordered_map<uint64_t, int64_t> longest;
    for (auto& kv : reads) {
        std::sort(kv.second.begin(), kv.second.end());
        int64_t m = 0;
        for (auto& t : kv.second) m = std::max(m, std::get<1>(t) - std::get<0>(t));
        longest[kv.first] = m;
    }
    for (Sub& sb : *subs) {
        bool clash = false;
        const uint64_t rk = row_key(sb.rank, sb.buf);
        auto rit = reads.find(rk);
        if (rit != reads.end()) {
            const auto& R = rit->second;
            // Reads overlapping [s, e) start in [s - longest, e).
            auto lo = std::lower_bound(R.begin(), R.end(),
                                       std::make_tuple(sb.s - longest[rk], (int64_t)INT64_MIN, (int32_t)INT32_MIN));
            auto hi = std::lower_bound(R.begin(), R.end(), std::make_tuple(sb.e, (int64_t)INT64_MIN, (int32_t)INT32_MIN));
            for (auto it = lo; it != hi && !clash; ++it) {
                const int64_t a = std::get<0>(*it), b = std::get<1>(*it);
                if (b <= sb.s) continue;
                const bool own = std::get<2>(*it) == sb.group && a == sb.s && b == sb.e &&
                                 gsize[sb.group] <= (size_t)kFuseMaxDsts;
                if (!own) clash = true;
            }
        }
        if (clash) {
            sb.dst = Phys{sb.rank, kBufTmp, slot_base + cursor[sb.rank] - sb.s};
            cursor[sb.rank] += sb.e - sb.s;
        } else {
            sb.dst = Phys{sb.rank, sb.buf, 0};
        }
    }
    for (const Sub& sb : *subs) pl.place(sb.rank, sb.buf, sb.s, sb.e, sb.dst);
}

}  // namespace

bool fuse_schedule(const Schedule& sch, int P, int depth, const std::vector<bool>& out_rows, FusedSchedule* out,
                   std::string* err) {
    *out = FusedSchedule();
    const int L = (int)sch.levels.size();
    depth = std::max(1, depth);
    std::vector<int> bounds;  // pass starts, then L
    for (int l = 0; l < L; l += depth) bounds.push_back(l);
    bounds.push_back(L);
    std::map<std::pair<int, int>, PassSym> cache;
    std::vector<std::vector<Write>> kept;
    std::vector<PassSym*> ps;
    for (int iter = 0;; iter++) {
        if (iter > 4 * L + 8) {
            *err = "fusion: splitting passes did not converge";
            return false;
        }
        const int np = (int)bounds.size() - 1;
        ps.assign(np, nullptr);
        for (int p = 0; p < np; p++) {
            const auto key = std::make_pair(bounds[p], bounds[p + 1]);
            auto it = cache.find(key);
            if (it == cache.end()) it = cache.emplace(key, run_pass(sch, key.first, key.second)).first;
            ps[p] = &it->second;
        }
        // Backward liveness: a run is kept when a later pass reads it or it
        // is a result; what a kept run reads is live before its pass.
        std::unordered_map<uint64_t, ISet> live;
        for (int r = 0; r < P; r++)
            if (out_rows[r] && sch.recv_elems > 0) iset_add(live[row_key(r, kBufRecv)], 0, sch.recv_elems);
        kept.assign(np, {});
        std::vector<std::tuple<int32_t, uint8_t, int64_t>> lv;
        for (int p = np - 1; p >= 0; p--) {
            for (const Write& w : ps[p]->writes) {
                auto lit = live.find(row_key(w.rank, w.buf));
                if (lit == live.end()) continue;
                for (auto& iv : iset_meet(lit->second, w.s, w.e))
                    kept[p].push_back(Write{w.rank, w.buf, iv.first, iv.second, w.v});
            }
            for (const Write& w : ps[p]->writes) {
                auto lit = live.find(row_key(w.rank, w.buf));
                if (lit != live.end()) iset_sub(lit->second, w.s, w.e);
            }
            for (const Write& k : kept[p]) {
                lv.clear();
                ps[p]->ex->leaves_of(k.v.node, k.v.shift, &lv);
                for (auto& t : lv)
                    iset_add(live[row_key(std::get<0>(t), std::get<1>(t))], k.s + std::get<2>(t), k.e + std::get<2>(t));
            }
        }
        // A pass whose programs are too large for the kernel is split.
        std::vector<int> bad;
        for (int p = 0; p < np; p++)
            for (const Write& k : kept[p]) {
                const FNode& n = ps[p]->ex->node(k.v.node);
                if (n.leaves > kFuseMaxLeaves || n.depth > kFuseMaxDepth) {
                    if (bounds[p + 1] - bounds[p] == 1) {
                        *err = "fusion: level " + std::to_string(bounds[p]) + " has a program too large";
                        return false;
                    }
                    bad.push_back(p);
                    break;
                }
            }
        if (bad.empty()) break;
        for (int j = (int)bad.size() - 1; j >= 0; j--) {
            const int p = bad[j];
            bounds.insert(bounds.begin() + p + 1, (bounds[p] + bounds[p + 1]) / 2);
        }
    }
    // Forward: place every pass's writes and emit its moves, one per group
    // chunk, in order of the first destination.
    Placement pl;
    std::vector<int64_t> cursor(P, 0);
    const int64_t slot_base = sch.tmp_elems;
    std::vector<Sub> subs;
    const int np = (int)bounds.size() - 1;
    auto emit_pass = [&](const std::vector<Sub>& sb, int levels) {
        std::map<int32_t, std::vector<const Sub*>> groups;
        for (const Sub& x : sb) groups[x.group].push_back(&x);
        std::vector<std::vector<const Sub*>> chunks;
        for (auto& g : groups)
            for (size_t j = 0; j < g.second.size(); j += kFuseMaxDsts)
                chunks.emplace_back(g.second.begin() + j,
                                    g.second.begin() + std::min(g.second.size(), j + (size_t)kFuseMaxDsts));
        std::sort(chunks.begin(), chunks.end(), [](const std::vector<const Sub*>& x, const std::vector<const Sub*>& y) {
            return std::make_tuple(x[0]->rank, x[0]->buf, x[0]->s) < std::make_tuple(y[0]->rank, y[0]->buf, y[0]->s);
        });
        std::vector<FusedMove> pass;
        for (const auto& ch : chunks) {
            FusedMove m;
            m.n = ch[0]->e - ch[0]->s;
            m.leaf_begin = (int32_t)out->leaves.size();
            out->leaves.insert(out->leaves.end(), ch[0]->prog.begin(), ch[0]->prog.end());
            m.nleaves = (int32_t)ch[0]->prog.size();
            m.dst_begin = (int32_t)out->dsts.size();
            for (const Sub* x : ch) out->dsts.push_back(FusedDst{x->dst.rank, x->dst.buf, {0, 0, 0}, x->s + x->dst.delta});
            m.ndst = (int32_t)ch.size();
            pass.push_back(m);
        }
        if (!pass.empty()) {
            out->passes.push_back(std::move(pass));
            out->pass_levels.push_back(levels);
        }
    };
    for (int p = 0; p < np; p++) {
        place_pass(*ps[p]->ex, kept[p], pl, slot_base, cursor, &subs);
        emit_pass(subs, bounds[p + 1] - bounds[p]);
    }
    // Results still in renaming slots are copied home.
    subs.clear();
    std::vector<std::tuple<int64_t, int64_t, Phys>> pieces;
    int32_t g = 0;
    for (int r = 0; r < P; r++) {
        if (!out_rows[r] || sch.recv_elems <= 0) continue;
        pl.lookup(r, kBufRecv, 0, sch.recv_elems, &pieces);
        for (auto& t : pieces) {
            const Phys& ph = std::get<2>(t);
            if (ph.rank == r && ph.buf == kBufRecv && ph.delta == 0) continue;
            Sub sb;
            sb.rank = r;
            sb.buf = kBufRecv;
            sb.s = std::get<0>(t);
            sb.e = std::get<1>(t);
            sb.prog.push_back(FusedLeaf{ph.rank, ph.buf, 0, {0, 0}, sb.s + ph.delta});
            sb.group = g++;
            sb.dst = Phys{r, kBufRecv, 0};
            subs.push_back(std::move(sb));
        }
    }
    emit_pass(subs, 0);
    int64_t most = 0;
    for (int64_t c : cursor) most = std::max(most, c);
    out->tmp_elems = slot_base + most;
    // Equivalence: the original levels and the fused passes, executed in one
    // expression table from the same initial state, leave the same addition
    // tree in every result element.
    Exec ex;
    for (const auto& lvl : sch.levels) ex.apply_level(lvl);
    std::vector<std::vector<Exec::Piece>> want(P);
    for (int r = 0; r < P; r++)
        if (out_rows[r]) want[r] = ex.get(r, kBufRecv, 0, sch.recv_elems);
    ex.clear_state();
    for (const auto& pass : out->passes) {
        std::vector<std::pair<const FusedMove*, std::vector<Exec::Piece>>> vals;
        for (const FusedMove& m : pass) {
            // Boundaries of every leaf's runs, relative to the move.
            std::vector<std::vector<Exec::Piece>> lp(m.nleaves);
            std::vector<int64_t> cuts{0, m.n};
            for (int j = 0; j < m.nleaves; j++) {
                const FusedLeaf& lf = out->leaves[m.leaf_begin + j];
                lp[j] = ex.get(lf.rank, lf.buf, lf.off, lf.off + m.n);
                for (auto& pc : lp[j]) cuts.push_back(pc.s - lf.off);
            }
            std::sort(cuts.begin(), cuts.end());
            cuts.erase(std::unique(cuts.begin(), cuts.end()), cuts.end());
            std::vector<Exec::Piece> v;
            std::vector<size_t> at(m.nleaves, 0);
            for (size_t c = 0; c + 1 < cuts.size(); c++) {
                const int64_t x0 = cuts[c], x1 = cuts[c + 1];
                std::vector<FVal> st;
                for (int j = 0; j < m.nleaves; j++) {
                    const FusedLeaf& lf = out->leaves[m.leaf_begin + j];
                    while (lp[j][at[j]].e - lf.off <= x0) at[j]++;
                    FVal lvv = lp[j][at[j]].v;
                    lvv.shift += lf.off;  // value at move position i: node at i + off + shift
                    st.push_back(lvv);
                    for (int a = 0; a < lf.adds; a++) {
                        if (st.size() < 2) {
                            *err = "fusion: malformed program";
                            return false;
                        }
                        const FVal t = st.back();
                        st.pop_back();
                        st.back() = ex.add(st.back(), t);
                    }
                }
                if (st.size() != 1) {
                    *err = "fusion: malformed program";
                    return false;
                }
                v.push_back(Exec::Piece{x0, x1, st[0]});
            }
            vals.emplace_back(&m, std::move(v));
        }
        for (auto& mv : vals)
            for (int j = 0; j < mv.first->ndst; j++) {
                const FusedDst& d = out->dsts[mv.first->dst_begin + j];
                for (const Exec::Piece& pc : mv.second)
                    ex.set(d.rank, d.buf, d.off + pc.s, d.off + pc.e, FVal{pc.v.node, pc.v.shift - d.off});
            }
    }
    for (int r = 0; r < P; r++) {
        if (!out_rows[r]) continue;
        const auto got = ex.get(r, kBufRecv, 0, sch.recv_elems);
        size_t i = 0, j = 0;
        while (i < got.size() && j < want[r].size()) {
            if (got[i].v != want[r][j].v) {
                *err = "fusion: rank " + std::to_string(r) + " receive element " +
                       std::to_string(std::max(got[i].s, want[r][j].s)) + " differs from the original schedule";
                return false;
            }
            if (got[i].e < want[r][j].e) i++;
            else if (want[r][j].e < got[i].e) j++;
            else {
                i++;
                j++;
            }
        }
    }
    return true;
}

}  // namespace bine

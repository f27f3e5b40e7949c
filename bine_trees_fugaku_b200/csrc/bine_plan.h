// Host-side planner: turns one Bine collective (variant, P, torus, ports,
// count) into a device-executable schedule.
//
// The schedule IR is a list of levels; each level is a set of moves that run
// concurrently and read the state left by the previous level:
//     dst = a           (copy)
//     dst = a + b       (MPI_SUM; a and b may come from different ranks)
// over regions (rank, buffer, element offset).  Buffers are the caller's
// send and receive arrays and the communicator's workspace.  A message of the
// reference (an MPI send matched with its receive) becomes one move reading
// the sender's region directly, the way a kernel reads a peer's rows in HBM;
// a receive followed by MPI_Reduce_local becomes one "dst = a + b" move.
//
// The IR feeds three consumers:
//   * the persistent step kernel (bine_kernels.cu), level by level;
//   * the symbolic executor below, which derives for every output element
//     the exact addition tree the reference evaluates, so the fused kernels
//     can reproduce float32 results bit for bit;
//   * link-byte accounting on a torus (every message, routed minimally).
#pragma once

#include <stdint.h>

#include <map>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#include "bine_sched.h"

namespace bine {

enum BufId : uint8_t { kBufSend = 0, kBufRecv = 1, kBufTmp = 2, kNumBufs = 3 };

enum Coll : int {
    kAllreduce = 0,
    kReduceScatter = 1,
    kAllgather = 2,
    kBcast = 3,
    kReduce = 4,
    kAlltoall = 5,
    kScatter = 6,
    kGather = 7,
    kNumColls = 8
};

// Variant numbering follows the reference's per-collective algorithm enums
// (lib/libbine_common.h:74-123).
enum : int {
    kArL = 0, kArB = 1, kArBCont = 3, kArBCoalesce = 4,
    kAgContPermute = 0, kAgContSend = 1, kAgBlocks = 2,
    kRsContPermute = 0, kRsBlocks = 2,
    kBcTree = 0, kBcScatterAllgather = 2,
    kRdTree = 0, kRdRedscatGather = 1,
    kA2aLog = 0, kScTree = 0, kGaTree = 0
};

enum Distance : int { kIncreasing = 0, kDecreasing = 1 };

struct Region {
    int32_t rank;
    uint8_t buf;
    int64_t off;  // elements
};

struct Move {
    Region dst, a, b;
    int64_t n;    // elements
    uint8_t add;  // 0: dst = a, 1: dst = a + b
};

struct Message {
    int32_t level;
    int32_t src, dst;
    int64_t elems;
};

struct PlanKey {
    int coll, variant, family, distance, ports, root;
    int64_t count;
    bool operator==(const PlanKey& o) const {
        return coll == o.coll && variant == o.variant && family == o.family && distance == o.distance &&
               ports == o.ports && root == o.root && count == o.count;
    }
};
struct PlanKeyHash {
    size_t operator()(const PlanKey& k) const {
        size_t h = (size_t)k.count * 1000003u;
        h ^= (size_t)k.coll * 31 + (size_t)k.variant * 131 + (size_t)k.family * 521 + (size_t)k.distance * 2053 +
             (size_t)k.ports * 8191 + (size_t)(k.root + 7) * 131071;
        return h;
    }
};

struct Schedule {
    std::vector<std::vector<Move>> levels;
    std::vector<Message> messages;
    int64_t send_elems = 0, recv_elems = 0;  // per rank
    int64_t tmp_elems = 0;                   // workspace elements per rank
};

// One reduction tree in postfix form: leaves are (rank, input shift), each
// followed by `adds` additions of the two top stack entries.
struct ProgEntry {
    int32_t rank;
    int32_t adds;
    int64_t shift;  // input element = output element + shift
};

// A run of output elements [off, off + n) on rank `rank` (-1: every rank)
// whose value is the program prog[begin, begin + len).
struct OutSegment {
    int64_t off, n;
    int32_t rank;
    int32_t prog_begin, prog_len;
    int32_t depth;  // evaluation stack depth of the program
};

struct TreePlan {
    std::vector<ProgEntry> prog;
    std::vector<OutSegment> segs;
    int max_depth = 0;
};

// A TreePlan whose every program is cut into K disjoint subtrees ("parts",
// left to right) plus a combine program over the parts, for evaluation by
// K cooperating lanes.  Substituting each part for its combine leaf gives
// back the original program entry for entry.
struct SplitTrees {
    int K = 1;
    std::vector<ProgEntry> prog;  // the parts of every distinct program
    // Per segment: K + 1 offsets into `prog` (part j is [parts[j], parts[j+1]))
    std::vector<int32_t> parts;
    // Per segment: K combine entries (part index, additions after it)
    std::vector<std::pair<int32_t, int32_t>> comb;
    int max_depth = 0;  // deepest evaluation stack of any part
};

// Returns false (with `err`) when some tree has fewer than K leaves.
bool split_trees(const TreePlan& tp, int K, SplitTrees* out, std::string* err);

class Planner {
  public:
    Planner(int nranks, int ndims, const int* dims);
    const Torus& torus() const { return t_; }

    // Builds the schedule of one call.  Returns false with `err` set when the
    // reference cannot run this case (it asserts, exits, deadlocks, corrupts
    // memory or returns wrong data); `err` names the reference line.
    bool build(const PlanKey& k, Schedule* out, std::string* err) const;

    // Exact reduction trees of every output element (float reference order).
    bool trees(const PlanKey& k, const Schedule& s, TreePlan* out, std::string* err) const;

    // Proves, by symbolic execution, that the schedule computes the
    // collective's MPI result: every output element is exactly the input
    // element the MPI semantics name, or for reductions the sum of that
    // element over every rank exactly once.  Returns false (with `err`)
    // when the reference's schedule returns wrong data for this case.
    bool verify(const PlanKey& k, const Schedule& s, std::string* err) const;

  private:
    Torus t_;
};

// Dataflow form of a schedule, for the pipelined engine.  Every move is cut
// into pieces of at most `piece_elems` elements; consecutive pieces of one
// level are packed into items (at most `max_pieces` <= kFlowMaxPieces pieces and about
// level elements / `target_items` elements each, never below
// `min_item_elems` unless the level is smaller).  With piece_elems <= 0 the
// pieces take the item size of their level, rounded up to a multiple of
// `min_item_elems` and capped at `max_item_elems`.  Each item lists the
// earlier items it must wait for over every (buffer, rank) row, as the row
// stood before the item's level: the last writer of what it reads (read
// after write) and of what it writes (write after write), and every reader
// since that writer of what it writes (write after read).  A dependency is an item index >= 0, or -(l + 1) for "every
// item of level l", used where one level would contribute more than
// kFlowLevelDep items.  Items are in level order and every dependency is on
// an earlier level, so running items in index order, each after its
// dependencies, is deadlock free and computes what level-by-level execution
// computes.
constexpr int kFlowMaxPieces = 256;
constexpr int kFlowLevelDep = 8;

struct FlowPiece {  // elements [start, start + n) of move `move` (level-order index)
    int32_t move, pad;
    int64_t start, n;
};
struct FlowItem {  // pieces [pbeg, pend), dependencies [dbeg, dend)
    int32_t pbeg, pend, dbeg, dend, level, pad;
};
struct FlowPlan {
    std::vector<FlowPiece> pieces;
    std::vector<FlowItem> items;
    std::vector<int32_t> deps;
    std::vector<int32_t> level_items;  // items per level
};

// Moves of one level never wait for each other: as in level-by-level
// execution, the planner emits levels whose moves are independent.  The
// send, receive and workspace rows are distinct (an in-place call's input
// rows are staged before the schedule runs).
void build_flow(const Schedule& s, int P, int64_t piece_elems, int64_t min_item_elems, int64_t max_item_elems,
                int target_items, int max_pieces, FlowPlan* out);

// ------------------------------------------------------- level fusion
// Fused form of a schedule for the PIPELINED engine.  Consecutive levels
// are grouped into passes; a pass's moves compute, from the buffer state at
// the start of the pass, every value the pass leaves behind that a later
// pass reads or that is part of the result.  A value that the original
// levels write and read again inside the pass (a partial sum one step
// passes to the next, a message staged in the workspace) stays in registers
// and is never written.  Every fused move evaluates a postfix program of
// leaves (state elements) and writes its value to one or more destinations
// (a copy that several ranks receive from the same rank in one pass is read
// once).  The addition trees are those of the original levels, so results
// are bit-identical; after every pass, every element that is read later or
// is a result holds what the original levels leave there at that step.
struct FusedLeaf {  // push state(buf, rank, i + off) for position i, then `adds` additions
    int32_t rank;
    uint8_t buf, adds, pad[2];
    int64_t off;
};
struct FusedDst {  // write the value of position i to (buf, rank, i + off)
    int32_t rank;
    uint8_t buf, pad[3];
    int64_t off;
};
struct FusedMove {
    int64_t n;
    int32_t leaf_begin, nleaves;
    int32_t dst_begin, ndst;
};
struct FusedSchedule {
    std::vector<std::vector<FusedMove>> passes;
    std::vector<FusedLeaf> leaves;
    std::vector<FusedDst> dsts;
    std::vector<int32_t> pass_levels;  // original levels per pass (0: the final copy of renamed results)
    int64_t tmp_elems = 0;             // workspace elements per rank, renaming slots included
};
constexpr int kFuseMaxLeaves = 8;  // leaves of one fused value (2^3: three levels of sums)
constexpr int kFuseMaxDsts = 8;    // destinations of one fused move
constexpr int kFuseMaxDepth = 4;   // evaluation stack of one program

// Fuses up to `depth` consecutive levels per pass (depth 1 keeps every
// level but still drops writes nothing reads).  `out_rows[r]` tells whether
// rank r's receive row is a result.  A pass whose values would need more
// than kFuseMaxLeaves leaves or kFuseMaxDepth stack entries is split.  A
// write that would overwrite an element another move of its pass still
// reads goes to a fresh workspace slot (after the schedule's own workspace)
// and later passes read it there; results left in slots are copied home by
// a last pass.  The fused schedule is checked against the original by
// symbolic execution (every result element the same addition tree); false
// with `err` if not.
bool fuse_schedule(const Schedule& s, int P, int depth, const std::vector<bool>& out_rows, FusedSchedule* out,
                   std::string* err);

// build_flow for a fused schedule: pieces index fused moves (pass order);
// reads are every leaf, writes every destination.  Without a piece size,
// each pass is cut into items of equal traffic (leaves + destinations per
// element), as many as a whole multiple of `target_items`: the kernel's
// resident blocks, so that a pass runs in whole waves.
void build_flow_fused(const FusedSchedule& f, int P, int64_t piece_elems, int64_t min_item_elems,
                      int64_t max_item_elems, int target_items, int max_pieces, FlowPlan* out);

// Per-link byte counts of a message list on the torus: 2 * ndims directed
// links per node, index (node * ndims + d) * 2 + (dir > 0 ? 0 : 1).
// Routes are dimension-ordered and minimal per dimension (+ on ties).
bool link_bytes(const Torus& t, const std::vector<Message>& msgs, int elem_size, std::vector<uint64_t>* out,
                std::string* err);

}  // namespace bine

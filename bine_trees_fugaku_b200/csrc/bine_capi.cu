// C ABI of the B200 Bine engine (include/bine_b200.h): communicator state,
// plan caches, dispatch of the eight collectives to the fused kernels or the
// step engine, and the host-side schedule queries.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <set>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/bine_b200.h"
#include "bine_kernels.cuh"
#include "bine_plan.h"

using namespace bine;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

#define CUDA_TRY(expr)                                                                               \
    do {                                                                                             \
        cudaError_t e_ = (expr);                                                                     \
        if (e_ != cudaSuccess) {                                                                     \
            return fail(e_ == cudaErrorMemoryAllocation ? BINE_ERR_NOMEM : BINE_ERR_CUDA,            \
                        std::string(#expr) + ": " + cudaGetErrorString(e_));                         \
        }                                                                                            \
    } while (0)

int dtype_size(int dt) {
    switch (dt) {
    case BINE_INT32: return 4;
    case BINE_INT64: return 8;
    case BINE_FLOAT: return 4;
    case BINE_DOUBLE: return 8;
    case BINE_CHAR: return 1;
    default: return -1;
    }
}

struct CollCfg {
    int variant, family, distance;
};

// Default variant and distance of every collective: lib/libbine.cc:56-72.
const CollCfg kDefaults[kNumColls] = {
    {kArB, kFamilyBine, kIncreasing},           {kRsContPermute, kFamilyBine, kIncreasing},
    {kAgContPermute, kFamilyBine, kDecreasing}, {kBcTree, kFamilyBine, kDecreasing},
    {kRdTree, kFamilyBine, kIncreasing},        {kA2aLog, kFamilyBine, kIncreasing},
    {kScTree, kFamilyBine, kIncreasing},        {kGaTree, kFamilyBine, kDecreasing}};

// Device copy of one schedule for the step engine.
// Device copy of the dataflow form of a schedule (pipelined engine) and its
// completion state (zeroed once; the kernel leaves it ready for the next
// launch).
struct DevFlow {
    dev::StepChunk* pieces = nullptr;
    dev::FlowItem* items = nullptr;
    int* deps = nullptr;
    int* level_items = nullptr;
    unsigned* done = nullptr;  // per item
    unsigned* ctl = nullptr;   // 3 + levels words
    int nitems = 0, nlevels = 0;
    ~DevFlow() {
        cudaFree(pieces);
        cudaFree(items);
        cudaFree(deps);
        cudaFree(level_items);
        cudaFree(done);
        cudaFree(ctl);
    }
};

struct DevSteps {
    dev::StepMove* moves = nullptr;
    dev::StepChunk* chunks = nullptr;
    int* level_begin = nullptr;
    int nlevels = 0;
    int max_chunks_per_level = 0;
    int64_t tmp_elems = 0;
    std::shared_ptr<DevFlow> flow;  // built on first use by the pipelined engine
    ~DevSteps() {
        cudaFree(moves);
        cudaFree(chunks);
        cudaFree(level_begin);
    }
};

// Device tables of a fused schedule (level fusion) and its dataflow plan.
struct DevFused {
    dev::FusedMoveDev* moves = nullptr;
    dev::FusedLeafDev* leaves = nullptr;
    dev::FusedDstDev* dsts = nullptr;
    DevFlow flow;
    int64_t tmp_elems = 0;
    int npasses = 0;
    ~DevFused() {
        cudaFree(moves);
        cudaFree(leaves);
        cudaFree(dsts);
    }
};
static_assert(sizeof(FusedMove) == sizeof(dev::FusedMoveDev), "fused move layouts differ");
static_assert(sizeof(FusedLeaf) == sizeof(dev::FusedLeafDev), "fused leaf layouts differ");
static_assert(sizeof(FusedDst) == sizeof(dev::FusedDstDev), "fused destination layouts differ");
static_assert(dev::kFuseLeaves == kFuseMaxLeaves && dev::kFuseDsts == kFuseMaxDsts, "fusion bounds differ");
static_assert((int)BINE_COLL_ALLREDUCE == kAllreduce && (int)BINE_COLL_REDUCE_SCATTER == kReduceScatter &&
                  (int)BINE_COLL_ALLGATHER == kAllgather && (int)BINE_COLL_GATHER == kGather,
              "collective codes differ");

// Device copy of the exact reduction trees of one call.
struct DevTrees {
    dev::TreeSeg* segs = nullptr;
    dev::TreeEntry* prog = nullptr;
    dev::TreeTile* tiles = nullptr;
    int ntiles = 0;        // vector tiles (16-byte aligned bodies of segments)
    dev::TreeTile* rtiles = nullptr;  // element tiles of the rest (unaligned programs, long pieces)
    int nrtiles = 0;
    dev::TreeTile* htiles = nullptr;  // short element pieces (heads and tails of vector bodies)
    int nhtiles = 0;
    dev::TreeTile* atiles = nullptr;  // element tiles of everything (unaligned layouts)
    int natiles = 0;
    int max_prog_len = 0;
    int depth = 0;  // deepest evaluation stack of any program
    // Some rank has its own trees (other ranks' tiles write rows that its
    // tiles read at the same columns).
    bool per_rank = false;
    // Split form (k_tree_split), used when split_k > 1 and the layout is
    // 16-byte aligned: the same segments over the split programs.
    int split_k = 1;
    int split_parts = 1;  // parts per tree: split_k or 2 * split_k
    dev::TreeSeg* ssegs = nullptr;
    dev::TreeEntry* sprog = nullptr;
    int* sparts = nullptr;
    dev::TreeComb* scomb = nullptr;
    int* sassign = nullptr;  // per segment: 2K part indices by warp, then K + 1 offsets
    // One-part plan of every segment (offsets {0, len}, combine {part 0}) for
    // the staged kernel when there is no split plan.
    int* uparts = nullptr;
    dev::TreeComb* ucomb = nullptr;
    dev::TreeTile* stiles = nullptr;
    int nstiles = 0;
    int smax_prog_len = 0;
    int sdepth = 0;  // deepest stack of any part or combine program
    // Row-aligned split form (k_tree_flat): when set, `stiles` holds its
    // tiles (absolute element starts on the row's grid) instead of
    // per-segment ones.
    bool flat = false;
    int64_t* fbody = nullptr;
    uint16_t* franks = nullptr;
    uint8_t* feshape = nullptr;  // edges: the tree shape of each segment, in row order
    uint8_t* fadds = nullptr;
    int* fparts = nullptr;
    dev::TreeComb* fcomb = nullptr;
    int* fassign = nullptr;
    dev::FlatEdge* fedges = nullptr;
    int fpitch = 0, flen = 0, fmax_ns = 0, fnq = 0, fnshape = 1;
    std::vector<dev::FlatEdge> h_fedges;
    std::vector<int64_t> h_fbody;  // host copy of fbody (bine_plan_tree_cover)
    // Edges (k_tree_edges): their own split plan, cut into
    // dev::kEdgeParts parts, with its entry-major rank table.
    uint8_t* feadds = nullptr;
    int* feparts = nullptr;
    dev::TreeComb* fecomb = nullptr;
    uint16_t* feranks_t = nullptr;
    int felen = 0, fedepth = 0, nfedges = 0;
    // Host copies of the tile lists and segment offsets, for column windows.
    std::vector<dev::TreeTile> h_tiles, h_stiles, h_rtiles, h_htiles, h_atiles;
    std::vector<int64_t> h_seg_off;
    // Per window width: every window's clipped tiles of each list, with
    // per-window begin indices (list k: tiles[k] + begin[k][i]).
    struct Windows {
        dev::TreeTile* tiles[6] = {};
        std::vector<int> begin[6];
    };
    std::map<long long, Windows> windows;
    bool dry = false;  // planned on the host only: nothing was uploaded
    ~DevTrees() {
        if (dry) return;
        for (auto& kv : windows)
            for (auto* t : kv.second.tiles) cudaFree(t);
        cudaFree(rtiles);
        cudaFree(htiles);
        cudaFree(atiles);
        cudaFree(segs);
        cudaFree(prog);
        cudaFree(tiles);
        cudaFree(ssegs);
        cudaFree(sprog);
        cudaFree(sparts);
        cudaFree(scomb);
        cudaFree(sassign);
        cudaFree(uparts);
        cudaFree(ucomb);
        cudaFree(stiles);
        cudaFree(fbody);
        cudaFree(franks);
        cudaFree(feshape);
        cudaFree(fedges);
        cudaFree(feadds);
        cudaFree(feparts);
        cudaFree(fecomb);
        cudaFree(feranks_t);
        cudaFree(fadds);
        cudaFree(fparts);
        cudaFree(fcomb);
        cudaFree(fassign);
    }
};

struct PlanKeyEs {
    PlanKey k;
    int es;
    long long segment;  // step engine: bytes per work chunk (0: 32 KiB)
    bool operator==(const PlanKeyEs& o) const { return k == o.k && es == o.es && segment == o.segment; }
};
struct PlanKeyEsHash {
    size_t operator()(const PlanKeyEs& x) const {
        return PlanKeyHash()(x.k) * 31 + (size_t)x.es + (size_t)x.segment * 7919;
    }
};

struct FusedKey {
    PlanKeyEs base;
    int levels;
    bool operator==(const FusedKey& o) const { return base == o.base && levels == o.levels; }
};
struct FusedKeyHash {
    size_t operator()(const FusedKey& x) const { return PlanKeyEsHash()(x.base) * 131 + (size_t)x.levels; }
};

// A schedule's routing does not depend on `count` once every block is
// non-empty, so one symbolic proof covers every count of the same
// structure (collective, variant, family, distance, ports, root) and
// block-occupancy class.
struct StructKey {
    int coll, variant, family, distance, ports, root, full;
    bool operator==(const StructKey& o) const {
        return coll == o.coll && variant == o.variant && family == o.family && distance == o.distance &&
               ports == o.ports && root == o.root && full == o.full;
    }
};
struct StructKeyHash {
    size_t operator()(const StructKey& k) const {
        return (size_t)k.coll * 1000003u ^ (size_t)k.variant * 10007u ^ (size_t)k.family * 101u ^
               (size_t)k.distance * 13u ^ (size_t)k.ports * 7u ^ (size_t)(k.root + 1) * 999983u ^ (size_t)k.full;
    }
};

}  // namespace

struct bine_comm_s {
    int P = 0;
    std::unique_ptr<Planner> planner;
    cudaStream_t stream = nullptr;
    size_t send_stride = 0, recv_stride = 0;
    int ports = 1;
    int engine = BINE_ENGINE_FUSED;
    int order = BINE_ORDER_REFERENCE;
    CollCfg cfg[kNumColls];
    std::mutex mu;
    std::unordered_map<PlanKey, std::shared_ptr<Schedule>, PlanKeyHash> schedules;
    std::unordered_map<PlanKeyEs, std::shared_ptr<DevSteps>, PlanKeyEsHash> dev_steps;
    std::unordered_map<PlanKeyEs, std::shared_ptr<DevTrees>, PlanKeyEsHash> dev_trees;
    std::unordered_map<FusedKey, std::shared_ptr<DevFused>, FusedKeyHash> dev_fused;
    int fusion = 0;  // levels per pass of the PIPELINED engine (0: per collective, 1: every level on its own)
    std::unordered_map<StructKey, int, StructKeyHash> verified;  // 1: proven, 0: refuted
    std::unordered_map<StructKey, std::string, StructKeyHash> refuted_why;
    long long segment_bytes = 0;
    int64_t cached_moves = 0;  // moves held by `schedules`
    // Side stream of the exact-order float kernels (element pieces run
    // beside the vector tiles) and its fork / join events.
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    int tree_split = 0;        // lanes per output vector in k_tree_split (0: chosen per call)
    // Device state, created on first use.
    int device = -1;
    int num_sms = 0;
    char* work = nullptr;
    size_t work_bytes = 0;
    char* inplace = nullptr;  // staged input rows of in-place step-engine allreduce calls
    size_t inplace_bytes = 0;
    unsigned* barrier = nullptr;  // [0] arrivals, [1] generation
    int* status = nullptr;
    unsigned long long step_timeout_ns = 5ull * 1000 * 1000 * 1000;
    unsigned barrier_extra = 0;
    // Host-buffer pipeline (bine_allreduce_host), created on first use:
    // copy streams, per-slot events (input copied, reduced, output copied)
    // and the device staging area (2 slots x input and output windows).
    cudaStream_t h2d = nullptr, d2h = nullptr;
    cudaEvent_t ev_in[2] = {}, ev_reduced[2] = {}, ev_out[2] = {}, ev_start = nullptr;
    std::vector<cudaEvent_t> ev_window;  // per window, for the after-window hook
    char* stage = nullptr;
    size_t stage_bytes = 0;
    long long host_window = 32ll << 20;  // bytes of one column window over all ranks
    ~bine_comm_s() {
        cudaFree(work);
        cudaFree(inplace);
        cudaFree(barrier);
        cudaFree(status);
        cudaFree(stage);
        for (int s = 0; s < 2; s++) {
            if (ev_in[s]) cudaEventDestroy(ev_in[s]);
            if (ev_reduced[s]) cudaEventDestroy(ev_reduced[s]);
            if (ev_out[s]) cudaEventDestroy(ev_out[s]);
        }
        if (ev_start) cudaEventDestroy(ev_start);
        for (cudaEvent_t e : ev_window) cudaEventDestroy(e);
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        if (side) cudaStreamDestroy(side);
        if (h2d) cudaStreamDestroy(h2d);
        if (d2h) cudaStreamDestroy(d2h);
    }
};

namespace {

PlanKey make_key(bine_comm_t c, int coll, long count, int root) {
    PlanKey k;
    k.coll = coll;
    k.variant = c->cfg[coll].variant;
    k.family = c->cfg[coll].family;
    k.distance = c->cfg[coll].distance;
    k.ports = c->ports;
    k.root = root;
    k.count = count;
    return k;
}

// Plan caches hold one entry per distinct call (count included); a caller
// that sweeps many counts would otherwise grow host and device memory
// without bound.  A full cache is emptied before the next insertion;
// entries a launch is still reading stay alive through its shared_ptr, and
// cudaFree in their destructors waits for kernels in flight.
constexpr size_t kMaxCachedSchedules = 64;
constexpr int64_t kMaxCachedMoves = 32ll << 20;  // ~2 GB of host schedule moves
constexpr size_t kMaxCachedDeviceTables = 64;

template <typename Map>
void trim(Map& m, size_t limit) {
    if (m.size() >= limit) m.clear();
}

int get_schedule(bine_comm_t c, const PlanKey& k, std::shared_ptr<Schedule>* out) {
    std::lock_guard<std::mutex> lk(c->mu);
    auto it = c->schedules.find(k);
    if (it != c->schedules.end()) {
        *out = it->second;
        return BINE_SUCCESS;
    }
    auto s = std::make_shared<Schedule>();
    std::string err;
    if (!c->planner->build(k, s.get(), &err)) return fail(BINE_ERR_UNSUPPORTED, err);
    int64_t moves = 0;
    for (const auto& lvl : s->levels) moves += (int64_t)lvl.size();
    if (c->schedules.size() >= kMaxCachedSchedules || c->cached_moves + moves > kMaxCachedMoves) {
        c->schedules.clear();
        c->cached_moves = 0;
    }
    c->cached_moves += moves;
    c->schedules.emplace(k, s);
    *out = s;
    return BINE_SUCCESS;
}

int ensure_device(bine_comm_t c) {
    if (c->device >= 0) return BINE_SUCCESS;
    int dev;
    CUDA_TRY(cudaGetDevice(&dev));
    CUDA_TRY(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, dev));
    CUDA_TRY(cudaMalloc(&c->barrier, 2 * sizeof(unsigned)));
    CUDA_TRY(cudaMalloc(&c->status, sizeof(int)));
    CUDA_TRY(cudaMemset(c->barrier, 0, 2 * sizeof(unsigned)));
    CUDA_TRY(cudaMemset(c->status, 0, sizeof(int)));
    CUDA_TRY(cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking));
    CUDA_TRY(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
    CUDA_TRY(cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming));
    c->device = dev;
    return BINE_SUCCESS;
}

int ensure_work(bine_comm_t c, size_t bytes) {
    if (bytes <= c->work_bytes) return BINE_SUCCESS;
    // Stream-ordered reuse: wait for pending work before replacing the area.
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    cudaFree(c->work);
    c->work = nullptr;
    c->work_bytes = 0;
    CUDA_TRY(cudaMalloc(&c->work, bytes));
    c->work_bytes = bytes;
    return BINE_SUCCESS;
}

template <typename T>
void fill(T** dptr, const std::vector<T>& v, cudaError_t* err) {
    *err = cudaMalloc(dptr, std::max<size_t>(1, v.size()) * sizeof(T));
    if (*err == cudaSuccess && !v.empty()) *err = cudaMemcpy(*dptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
}

// Proves (once per structure, see StructKey) that schedule `s` computes the
// MPI result.
int verify_cached(bine_comm_t c, const PlanKey& k, const Schedule& s) {
    StructKey sk{k.coll, k.variant, k.family, k.distance, k.ports, k.root, k.count >= (int64_t)k.ports * c->P ? 1 : 0};
    {
        std::lock_guard<std::mutex> lk(c->mu);
        auto it = c->verified.find(sk);
        if (it != c->verified.end()) {
            if (it->second) return BINE_SUCCESS;
            return fail(BINE_ERR_UNSUPPORTED, c->refuted_why[sk]);
        }
    }
    std::string verr;
    const bool ok = c->planner->verify(k, s, &verr);
    std::lock_guard<std::mutex> lk(c->mu);
    c->verified[sk] = ok ? 1 : 0;
    if (!ok) {
        c->refuted_why[sk] = verr;
        return fail(BINE_ERR_UNSUPPORTED, verr);
    }
    return BINE_SUCCESS;
}

int get_dev_steps(bine_comm_t c, const PlanKey& k, int es, std::shared_ptr<DevSteps>* out) {
    std::shared_ptr<Schedule> s;
    int rc = get_schedule(c, k, &s);
    if (rc) return rc;
    rc = verify_cached(c, k, *s);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(c->mu);
    PlanKeyEs key{k, es, c->segment_bytes};
    auto it = c->dev_steps.find(key);
    if (it != c->dev_steps.end()) {
        *out = it->second;
        return BINE_SUCCESS;
    }
    // Every region the kernel will touch must lie inside its row: a planner
    // error must never become an out-of-bounds device access.
    const int64_t rows[3] = {s->send_elems, s->recv_elems, s->tmp_elems};
    for (const auto& lvl : s->levels)
        for (const Move& m : lvl)
            for (const Region* r : {&m.dst, &m.a, &m.b})
                if (r->rank < 0 || r->rank >= c->P || r->buf > kBufTmp || r->off < 0 || m.n < 0 ||
                    r->off + m.n > rows[r->buf])
                    return fail(BINE_ERR_INTERNAL, "planner produced a region outside its buffer row");
    auto d = std::make_shared<DevSteps>();
    std::vector<dev::StepMove> moves;
    std::vector<dev::StepChunk> chunks;
    std::vector<int> lb;
    const int64_t seg = c->segment_bytes > 0 ? c->segment_bytes : 32 * 1024;
    const int64_t chunk_elems = std::max<int64_t>(16, seg / es);
    for (const auto& lvl : s->levels) {
        lb.push_back((int)chunks.size());
        for (const Move& m : lvl) {
            dev::StepMove dm;
            dm.dst_off = m.dst.off;
            dm.a_off = m.a.off;
            dm.b_off = m.b.off;
            dm.dst_rank = m.dst.rank;
            dm.a_rank = m.a.rank;
            dm.b_rank = m.b.rank;
            dm.dst_buf = m.dst.buf;
            dm.a_buf = m.a.buf;
            dm.b_buf = m.b.buf;
            dm.add = m.add;
            const int mi = (int)moves.size();
            moves.push_back(dm);
            for (int64_t st = 0; st < m.n; st += chunk_elems)
                chunks.push_back(dev::StepChunk{mi, 0, st, std::min(chunk_elems, m.n - st)});
        }
        int nlvl = (int)chunks.size() - lb.back();
        d->max_chunks_per_level = std::max(d->max_chunks_per_level, nlvl);
    }
    lb.push_back((int)chunks.size());
    d->nlevels = (int)s->levels.size();
    d->tmp_elems = s->tmp_elems;
    cudaError_t e1, e2, e3;
    fill(&d->moves, moves, &e1);
    fill(&d->chunks, chunks, &e2);
    fill(&d->level_begin, lb, &e3);
    if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess)
        return fail(BINE_ERR_CUDA, "uploading the schedule failed");
    trim(c->dev_steps, kMaxCachedDeviceTables);
    c->dev_steps.emplace(key, d);
    *out = d;
    return BINE_SUCCESS;
}

static_assert(sizeof(FlowPiece) == sizeof(dev::StepChunk), "piece layouts differ");
static_assert(sizeof(FlowItem) == sizeof(dev::FlowItem), "item layouts differ");
static_assert(dev::kFlowPieces <= kFlowMaxPieces, "the kernel's piece table exceeds the planner's bound");

// Item sizing of the pipelined engine: about `target_items` items per level
// (four per SM, one per resident block), of 4 KiB at least, in whole 4 KiB
// multiples.  With a segment size set, pieces (and items) are at most one
// segment; without one, each level's items are as large as that target
// allows, up to kFlowMaxItemBytes.  Measured on B200 against the STEPS
// engine over allreduce (B, L), allgather, bcast, alltoall and
// reduce_scatter at P = 16, 64, 256 and 2 KiB..8 MiB per rank: 4 items per
// SM gave 0.75x the STEPS time (geometric mean, never above 0.96x); 1, 2,
// 8 and 16 per SM gave 0.91x, 0.80x, 0.82x and 0.91x, and a 1 KiB minimum
// 0.79x.
constexpr int64_t kFlowMaxItemBytes = 1 << 20;
constexpr int kFlowItemsPerSm = dev::kFlowBlocksPerSm;

void flow_plan(const Schedule& s, int P, int es, long long segment_bytes, int target_items, FlowPlan* fp) {
    const int64_t piece = segment_bytes > 0 ? std::max<int64_t>(16, segment_bytes / es) : 0;
    build_flow(s, P, piece, std::max<int64_t>(1, 4096 / es), kFlowMaxItemBytes / es, target_items, dev::kFlowPieces,
               fp);
}

int get_dev_flow(bine_comm_t c, const PlanKey& k, int es, std::shared_ptr<DevSteps>* steps,
                 std::shared_ptr<DevFlow>* out) {
    int rc = get_dev_steps(c, k, es, steps);
    if (rc) return rc;
    std::shared_ptr<Schedule> s;
    rc = get_schedule(c, k, &s);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(c->mu);
    if ((*steps)->flow) {
        *out = (*steps)->flow;
        return BINE_SUCCESS;
    }
    FlowPlan fp;
    flow_plan(*s, c->P, es, c->segment_bytes, kFlowItemsPerSm * c->num_sms, &fp);
    auto f = std::make_shared<DevFlow>();
    f->nitems = (int)fp.items.size();
    f->nlevels = (int)fp.level_items.size();
    std::vector<dev::StepChunk> pieces(fp.pieces.size());
    if (!pieces.empty()) std::memcpy(pieces.data(), fp.pieces.data(), pieces.size() * sizeof(dev::StepChunk));
    std::vector<dev::FlowItem> items(fp.items.size());
    if (!items.empty()) std::memcpy(items.data(), fp.items.data(), items.size() * sizeof(dev::FlowItem));
    cudaError_t e[4];
    fill(&f->pieces, pieces, &e[0]);
    fill(&f->items, items, &e[1]);
    fill(&f->deps, fp.deps, &e[2]);
    fill(&f->level_items, fp.level_items, &e[3]);
    for (cudaError_t x : e)
        if (x != cudaSuccess) return fail(BINE_ERR_CUDA, "uploading the dataflow schedule failed");
    CUDA_TRY(cudaMalloc(&f->done, std::max(1, f->nitems) * sizeof(unsigned)));
    CUDA_TRY(cudaMalloc(&f->ctl, (3 + f->nlevels) * sizeof(unsigned)));
    CUDA_TRY(cudaMemset(f->done, 0, std::max(1, f->nitems) * sizeof(unsigned)));
    CUDA_TRY(cudaMemset(f->ctl, 0, (3 + f->nlevels) * sizeof(unsigned)));
    (*steps)->flow = f;
    *out = f;
    return BINE_SUCCESS;
}

// Ranks whose receive row is a result of the collective.
std::vector<bool> result_rows(const PlanKey& k, int P) {
    std::vector<bool> rows(P, true);
    if (k.coll == kReduce || k.coll == kGather) {
        rows.assign(P, false);
        rows[k.root] = true;
    }
    return rows;
}

int fused_schedule(bine_comm_t c, const PlanKey& k, int levels, std::shared_ptr<Schedule>* s, FusedSchedule* fs) {
    int rc = get_schedule(c, k, s);
    if (rc) return rc;
    rc = verify_cached(c, k, **s);
    if (rc) return rc;
    std::string err;
    if (!fuse_schedule(**s, c->P, levels, result_rows(k, c->P), fs, &err)) return fail(BINE_ERR_INTERNAL, err);
    return BINE_SUCCESS;
}

// Levels per pass of the automatic fusion setting, per collective
// (allreduce, reduce_scatter, allgather, bcast, reduce, alltoall, scatter,
// gather).  Measured on B200 at P = 64 and 256 from 512 KiB per rank: the
// reductions run fastest at 6 (allreduce B 2.32 TB/s against 2.05 at 10),
// the copies at 10 and more (allgather 5.07 TB/s against 1.99 at 6);
// alltoall has about three IR levels per Bine step, and 13 keeps two passes.
constexpr int kAutoFusion[kNumColls] = {6, 6, 12, 12, 6, 13, 12, 12};

// Planning a fused schedule costs about 4 us per move on the host (11 s for
// allreduce B and 47 s for alltoall at P = 1024, once per call shape), so
// the automatic setting runs larger schedules level by level.
constexpr int64_t kAutoFusionMaxMoves = 1 << 20;

int fusion_levels(bine_comm_t c, int coll, const Schedule* s = nullptr) {
    if (c->fusion > 0) return c->fusion;
    if (s) {
        int64_t moves = 0;
        for (const auto& lvl : s->levels) moves += (int64_t)lvl.size();
        if (moves > kAutoFusionMaxMoves) return 1;
    }
    return kAutoFusion[coll];
}

// Blocks of k_flow_fused resident on the device at once: the fused plan
// cuts each pass into a whole multiple of this many items of equal traffic,
// so that a pass runs in whole waves.
int fused_resident_blocks(bine_comm_t c, int es) {
    int per_sm = 0;
    cudaError_t e;
    switch (es) {
        case 1: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dev::k_flow_fused<int8_t>, dev::kFlowThreads, 0); break;
        case 8: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dev::k_flow_fused<int64_t>, dev::kFlowThreads, 0); break;
        default: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dev::k_flow_fused<int32_t>, dev::kFlowThreads, 0);
    }
    if (e != cudaSuccess || per_sm < 1) {
        cudaGetLastError();
        per_sm = kFlowItemsPerSm;
    }
    return per_sm * c->num_sms;
}

int get_dev_fused(bine_comm_t c, const PlanKey& k, int es, std::shared_ptr<DevFused>* out) {
    std::shared_ptr<Schedule> sch;
    int rc0 = get_schedule(c, k, &sch);
    if (rc0) return rc0;
    const int levels = fusion_levels(c, k.coll, sch.get());
    const FusedKey key{PlanKeyEs{k, es, c->segment_bytes}, levels};
    {
        std::lock_guard<std::mutex> lk(c->mu);
        auto it = c->dev_fused.find(key);
        if (it != c->dev_fused.end()) {
            *out = it->second;
            return BINE_SUCCESS;
        }
    }
    std::shared_ptr<Schedule> s;
    FusedSchedule fs;
    int rc = fused_schedule(c, k, levels, &s, &fs);
    if (rc) return rc;
    // Every row range the kernel will touch must lie inside its row.
    const int64_t rows[3] = {s->send_elems, s->recv_elems, fs.tmp_elems};
    for (const auto& pass : fs.passes)
        for (const FusedMove& m : pass) {
            if (m.n < 0 || m.nleaves < 1 || m.nleaves > kFuseMaxLeaves || m.ndst < 1 || m.ndst > kFuseMaxDsts)
                return fail(BINE_ERR_INTERNAL, "fusion produced a move outside the kernel's bounds");
            int depth = 0, maxd = 0;
            for (int j = 0; j < m.nleaves; j++) {
                const FusedLeaf& lf = fs.leaves[m.leaf_begin + j];
                if (lf.rank < 0 || lf.rank >= c->P || lf.buf > kBufTmp || lf.off < 0 || lf.off + m.n > rows[lf.buf] ||
                    (j == 0 && lf.adds != 0) || lf.adds > 3)
                    return fail(BINE_ERR_INTERNAL, "fusion produced a leaf outside its buffer row");
                maxd = std::max(maxd, depth + 1);  // the leaf is pushed before its additions
                depth += 1 - lf.adds;
                if (depth < 1) return fail(BINE_ERR_INTERNAL, "fusion produced a malformed program");
            }
            if (depth != 1 || maxd > kFuseMaxDepth) return fail(BINE_ERR_INTERNAL, "fusion produced a malformed program");
            for (int j = 0; j < m.ndst; j++) {
                const FusedDst& d = fs.dsts[m.dst_begin + j];
                if (d.rank < 0 || d.rank >= c->P || d.buf > kBufTmp || d.buf == kBufSend || d.off < 0 ||
                    d.off + m.n > rows[d.buf])
                    return fail(BINE_ERR_INTERNAL, "fusion produced a destination outside its buffer row");
            }
        }
    FlowPlan fp;
    // Pieces of at most kFlowMaxItemBytes keep every item below 2^31 bytes,
    // the kernel's 32-bit unit counts.
    const int64_t piece =
        c->segment_bytes > 0 ? std::max<int64_t>(16, std::min<int64_t>(c->segment_bytes, kFlowMaxItemBytes) / es) : 0;
    build_flow_fused(fs, c->P, piece, std::max<int64_t>(1, 4096 / es), kFlowMaxItemBytes / es,
                     fused_resident_blocks(c, es), dev::kFusedPieces, &fp);
    auto d = std::make_shared<DevFused>();
    d->tmp_elems = fs.tmp_elems;
    d->npasses = (int)fs.passes.size();
    std::vector<FusedMove> moves;
    for (const auto& pass : fs.passes) moves.insert(moves.end(), pass.begin(), pass.end());
    std::vector<dev::FusedMoveDev> dm(moves.size());
    if (!dm.empty()) std::memcpy(dm.data(), moves.data(), dm.size() * sizeof(dev::FusedMoveDev));
    std::vector<dev::FusedLeafDev> dl(fs.leaves.size());
    if (!dl.empty()) std::memcpy(dl.data(), fs.leaves.data(), dl.size() * sizeof(dev::FusedLeafDev));
    std::vector<dev::FusedDstDev> dd(fs.dsts.size());
    if (!dd.empty()) std::memcpy(dd.data(), fs.dsts.data(), dd.size() * sizeof(dev::FusedDstDev));
    DevFlow& f = d->flow;
    f.nitems = (int)fp.items.size();
    f.nlevels = (int)fp.level_items.size();
    std::vector<dev::StepChunk> pieces(fp.pieces.size());
    if (!pieces.empty()) std::memcpy(pieces.data(), fp.pieces.data(), pieces.size() * sizeof(dev::StepChunk));
    std::vector<dev::FlowItem> items(fp.items.size());
    if (!items.empty()) std::memcpy(items.data(), fp.items.data(), items.size() * sizeof(dev::FlowItem));
    cudaError_t e[7];
    fill(&d->moves, dm, &e[0]);
    fill(&d->leaves, dl, &e[1]);
    fill(&d->dsts, dd, &e[2]);
    fill(&f.pieces, pieces, &e[3]);
    fill(&f.items, items, &e[4]);
    fill(&f.deps, fp.deps, &e[5]);
    fill(&f.level_items, fp.level_items, &e[6]);
    for (cudaError_t x : e)
        if (x != cudaSuccess) return fail(BINE_ERR_CUDA, "uploading the fused schedule failed");
    CUDA_TRY(cudaMalloc(&f.done, std::max(1, f.nitems) * sizeof(unsigned)));
    CUDA_TRY(cudaMalloc(&f.ctl, (3 + f.nlevels) * sizeof(unsigned)));
    CUDA_TRY(cudaMemset(f.done, 0, std::max(1, f.nitems) * sizeof(unsigned)));
    CUDA_TRY(cudaMemset(f.ctl, 0, (3 + f.nlevels) * sizeof(unsigned)));
    std::lock_guard<std::mutex> lk(c->mu);
    trim(c->dev_fused, kMaxCachedDeviceTables);
    c->dev_fused.emplace(key, d);
    *out = d;
    return BINE_SUCCESS;
}

// Tables of the row-aligned split form (k_tree_flat), built when every
// segment with a vector body sends its result to every rank, every leaf of
// its split program is at shift 0 (allreduce), and its tree has one of at
// most kFlatShapes shapes: the shape is the split program's additions, part
// offsets, combine program and warp assignment, and segments of one shape
// differ only in their ranks.
//
// Row-kernel tables (`body`, `ranks`) list the segments by shape, then by
// the position of their bodies; shape h occupies [base[h], base[h + 1]).
// Row tiles are the output row's own groups of `W` elements that hold a
// body of shape h, each with the first such body it touches and how many
// (at most kFlatSegs, or the form is not used) in `pad & 0xff`, and h in
// `pad >> 8`; tiles are ordered by column, then shape, so that the shapes
// sharing a group's columns run side by side.
//
// Edges are the vectors between two bodies adjacent in the row that
// straddle their segments' boundary.  They are evaluated with the edge
// split plan `se` (dev::kEdgeParts parts), which must have one structure per
// shape too; their tables (`eranks_t`, entry-major, and `eshape`) index the
// segments in row order.  The head and tail pieces the edges cover are
// listed in `covered` (segment, first element in it) for the element kernel
// to skip.  `sassign` is the split plan's per-segment warp assignment.
struct FlatTables {
    std::vector<int64_t> body;
    std::vector<uint16_t> ranks;
    std::vector<uint8_t> adds;  // [shape][len]
    std::vector<int> parts, assign;
    std::vector<dev::TreeComb> comb;
    std::vector<dev::FlatEdge> edges;
    std::vector<dev::TreeTile> tiles;
    // The edges' split plans (dev::kEdgeParts parts, per shape) and tables.
    std::vector<uint8_t> eadds, eshape;
    std::vector<int> eparts;
    std::vector<dev::TreeComb> ecomb;
    std::vector<uint16_t> eranks_t;
    int edepth = 0;
    std::set<std::pair<int32_t, int64_t>> covered;
    int pitch = 0, len = 0, max_ns = 0, nq = 0, nshape = 0;
};

bool flat_tables(const TreePlan& tp, const SplitTrees& st, const SplitTrees* se, int K, int KP,
                 const std::vector<int>& sassign, const std::vector<int64_t>& body_lo,
                 const std::vector<int64_t>& body_hi, int64_t W, int L, int P, FlatTables* f) {
    if (P > 65536) return false;
    std::vector<int> order;  // segments with a body, by position
    for (size_t i = 0; i < tp.segs.size(); i++)
        if (body_lo[i] < body_hi[i]) order.push_back((int)i);
    if (order.empty()) return false;
    std::sort(order.begin(), order.end(),
              [&](int a, int b) { return tp.segs[a].off + body_lo[a] < tp.segs[b].off + body_lo[b]; });
    const int NA = KP + K + 1;
    const int len = st.parts[(size_t)order[0] * (KP + 1) + KP] - st.parts[(size_t)order[0] * (KP + 1)];
    // Shapes, in order of first appearance along the row.
    std::map<std::vector<int32_t>, int> shape_of;
    std::vector<int> first_of;  // a segment of each shape
    std::vector<int> shape(order.size());
    for (size_t q = 0; q < order.size(); q++) {
        const int i = order[q];
        if (tp.segs[i].rank >= 0) return false;
        const int32_t* po = &st.parts[(size_t)i * (KP + 1)];
        if (po[KP] - po[0] != len) return false;
        std::vector<int32_t> key;
        key.reserve(len + 2 * KP + NA + 1);
        for (int j = 0; j <= KP; j++) key.push_back(po[j] - po[0]);
        for (int j = 0; j < KP; j++) {
            key.push_back(st.comb[(size_t)i * KP + j].first);
            key.push_back(st.comb[(size_t)i * KP + j].second);
        }
        for (int j = 0; j < NA; j++) key.push_back(sassign[(size_t)i * NA + j]);
        for (int k = 0; k < len; k++) {
            const ProgEntry& e = st.prog[po[0] + k];
            if (e.shift != 0 || e.adds < 0 || e.adds > 255 || e.rank < 0 || e.rank >= P) return false;
            key.push_back(e.adds);
        }
        auto it = shape_of.find(key);
        if (it == shape_of.end()) {
            if ((int)first_of.size() == dev::kFlatShapes) return false;
            it = shape_of.emplace(key, (int)first_of.size()).first;
            first_of.push_back(i);
        }
        shape[q] = it->second;
    }
    const int H = (int)first_of.size();
    const size_t nq = order.size();
    f->nshape = H;
    f->nq = (int)nq;
    f->len = (len + 15) / 16 * 16;
    f->pitch = (len + 7) / 8 * 8;
    f->adds.assign((size_t)H * f->len, 0);
    for (int h = 0; h < H; h++) {
        const int i = first_of[h];
        const int32_t* po = &st.parts[(size_t)i * (KP + 1)];
        for (int k = 0; k < len; k++) f->adds[(size_t)h * f->len + k] = (uint8_t)st.prog[po[0] + k].adds;
        for (int j = 0; j <= KP; j++) f->parts.push_back(po[j] - po[0]);
        for (int j = 0; j < KP; j++)
            f->comb.push_back(dev::TreeComb{st.comb[(size_t)i * KP + j].first, st.comb[(size_t)i * KP + j].second});
        f->assign.insert(f->assign.end(), sassign.begin() + (size_t)i * NA, sassign.begin() + (size_t)(i + 1) * NA);
    }
    // Row-kernel tables: by shape, then position.
    std::vector<size_t> gq(nq);  // row-order index of each table entry
    for (size_t q = 0; q < nq; q++) gq[q] = q;
    std::stable_sort(gq.begin(), gq.end(), [&](size_t a, size_t b) { return shape[a] < shape[b]; });
    std::vector<size_t> base(H + 1, 0);
    for (size_t q = 0; q < nq; q++) base[shape[q] + 1]++;
    for (int h = 0; h < H; h++) base[h + 1] += base[h];
    f->ranks.assign(nq * f->pitch, 0);
    for (size_t x = 0; x < nq; x++) {
        const int i = order[gq[x]];
        const int32_t* po = &st.parts[(size_t)i * (KP + 1)];
        for (int k = 0; k < len; k++) f->ranks[x * f->pitch + k] = (uint16_t)st.prog[po[0] + k].rank;
        f->body.push_back(tp.segs[i].off + body_lo[i]);
        f->body.push_back(tp.segs[i].off + body_hi[i]);
    }
    // Edges: one vector between adjacent bodies, cut by the boundary of
    // their (adjacent) segments; only with edge split plans of one
    // structure per shape.
    const int NE = dev::kEdgeParts;
    bool edges_ok = se != nullptr;
    for (size_t q = 0; edges_ok && q < nq; q++) {
        const int i = order[q], i0 = first_of[shape[q]];
        const int32_t* po = &se->parts[(size_t)i * (NE + 1)];
        const int32_t* p0 = &se->parts[(size_t)i0 * (NE + 1)];
        for (int j = 0; j <= NE; j++) edges_ok &= po[j] - po[0] == p0[j] - p0[0];
        for (int j = 0; j < NE; j++) edges_ok &= se->comb[(size_t)i * NE + j] == se->comb[(size_t)i0 * NE + j];
        edges_ok &= po[NE] - po[0] == len;
        for (int k = 0; edges_ok && k < len; k++)
            edges_ok &= se->prog[po[0] + k].adds == se->prog[p0[0] + k].adds && se->prog[po[0] + k].shift == 0 &&
                        se->prog[po[0] + k].adds <= 255;
    }
    if (edges_ok) {
        f->eadds.assign((size_t)H * f->len, 0);
        for (int h = 0; h < H; h++) {
            const int32_t* p0 = &se->parts[(size_t)first_of[h] * (NE + 1)];
            for (int k = 0; k < len; k++) f->eadds[(size_t)h * f->len + k] = (uint8_t)se->prog[p0[0] + k].adds;
            for (int j = 0; j <= NE; j++) f->eparts.push_back(p0[j] - p0[0]);
            for (int j = 0; j < NE; j++)
                f->ecomb.push_back(dev::TreeComb{se->comb[(size_t)first_of[h] * NE + j].first,
                                                 se->comb[(size_t)first_of[h] * NE + j].second});
            int cdepth = 1, sp = 0;
            for (int j = 0; j < NE; j++) {
                cdepth = std::max(cdepth, ++sp);
                sp -= f->ecomb[(size_t)h * NE + j].adds;
            }
            f->edepth = std::max(f->edepth, cdepth);
        }
        f->edepth = std::max(f->edepth, se->max_depth);
        f->eranks_t.assign((size_t)f->pitch * nq, 0);
        for (size_t q = 0; q < nq; q++) {
            f->eshape.push_back((uint8_t)shape[q]);
            const int32_t* po = &se->parts[(size_t)order[q] * (NE + 1)];
            for (int k = 0; k < len; k++) f->eranks_t[(size_t)k * nq + q] = (uint16_t)se->prog[po[0] + k].rank;
        }
        for (size_t q = 0; q + 1 < nq; q++) {
            const OutSegment& a = tp.segs[order[q]];
            const OutSegment& b = tp.segs[order[q + 1]];
            const int64_t e = tp.segs[order[q]].off + body_hi[order[q]];
            if (a.off + a.n != b.off || b.off + body_lo[order[q + 1]] != e + L || b.off <= e || b.off >= e + L) continue;
            f->edges.push_back(dev::FlatEdge{e, (int32_t)q, (int32_t)(b.off - e)});
            f->covered.insert({order[q], body_hi[order[q]]});
            f->covered.insert({order[q + 1], 0});
        }
    }
    // Row tiles on the row's grid of W elements, per shape.
    for (int h = 0; h < H; h++) {
        const int64_t* bd = f->body.data() + 2 * base[h];
        const size_t n = base[h + 1] - base[h];
        const int64_t first = bd[0] / W * W, last = bd[2 * n - 1];
        size_t q = 0;
        for (int64_t a = first; a < last; a += W) {
            const int64_t b = a + W;
            while (q < n && bd[2 * q + 1] <= a) q++;
            if (q == n) break;
            if (bd[2 * q] >= b) {  // no body of this shape here: skip to the next one's group
                a = bd[2 * q] / W * W - W;
                continue;
            }
            size_t r = q;
            while (r < n && bd[2 * r] < b) r++;
            if (r - q > (size_t)dev::kFlatSegs) return false;
            f->max_ns = std::max(f->max_ns, (int)(r - q));
            f->tiles.push_back(dev::TreeTile{(int32_t)(base[h] + q), (int32_t)((r - q) | (h << 8)), a, W});
        }
    }
    std::stable_sort(f->tiles.begin(), f->tiles.end(), [](const dev::TreeTile& x, const dev::TreeTile& y) {
        return x.start != y.start ? x.start < y.start : (x.pad >> 8) < (y.pad >> 8);
    });
    return true;
}

// With `dry` the call plans the trees and their tile lists on the host and
// uploads nothing (no device is needed; the result is not cached and its
// device pointers stay null): bine_plan_tree_form reports from it.
int get_dev_trees(bine_comm_t c, const PlanKey& k, int es, std::shared_ptr<DevTrees>* out, bool dry = false) {
    std::shared_ptr<Schedule> s;
    int rc = get_schedule(c, k, &s);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(c->mu);
    PlanKeyEs key{k, es, c->tree_split};
    auto it = c->dev_trees.find(key);
    if (it != c->dev_trees.end()) {
        *out = it->second;
        return BINE_SUCCESS;
    }
    auto put = [&](auto** dptr, const auto& v, cudaError_t* e) {
        if (dry)
            *e = cudaSuccess;
        else
            fill(dptr, v, e);
    };
    TreePlan tp;
    std::string err;
    if (!c->planner->trees(k, *s, &tp, &err)) return fail(BINE_ERR_INTERNAL, err);
    if (tp.max_depth > dev::kMaxTreeDepth) return fail(BINE_ERR_UNSUPPORTED, "reduction tree deeper than supported");
    // Bounds of every leaf read and every output write, checked on the host.
    for (const OutSegment& sg : tp.segs) {
        if (sg.off < 0 || sg.n < 0 || sg.off + sg.n > s->recv_elems || sg.rank >= c->P ||
            sg.prog_begin < 0 || sg.prog_begin + sg.prog_len > (int64_t)tp.prog.size())
            return fail(BINE_ERR_INTERNAL, "reduction segment outside its buffer row");
        for (int i = sg.prog_begin; i < sg.prog_begin + sg.prog_len; i++) {
            const ProgEntry& e = tp.prog[i];
            if (e.rank < 0 || e.rank >= c->P || sg.off + e.shift < 0 || sg.off + sg.n + e.shift > s->send_elems)
                return fail(BINE_ERR_INTERNAL, "reduction leaf outside its input row");
        }
    }
    auto d = std::make_shared<DevTrees>();
    d->dry = dry;
    std::vector<dev::TreeSeg> segs;
    std::vector<dev::TreeEntry> prog;
    for (const ProgEntry& e : tp.prog) prog.push_back(dev::TreeEntry{e.rank, e.adds, e.shift});
    for (const OutSegment& sg : tp.segs) {
        segs.push_back(dev::TreeSeg{sg.off, sg.n, sg.rank, sg.prog_begin, sg.prog_len, sg.depth});
        d->max_prog_len = std::max(d->max_prog_len, sg.prog_len);
        d->per_rank |= sg.rank >= 0 && k.coll == kAllreduce;
    }
    // Every segment whose program reads at 16-byte-aligned shifts gets a
    // vector body: its elements from the first to the last 16-byte boundary
    // of the output row.  Heads, tails and the other segments run through
    // the element kernel (rtiles); atiles cover everything element-wise for
    // layouts that are not 16-byte aligned.
    const int64_t L = 16 / es;
    std::vector<int64_t> body_lo(tp.segs.size(), 0), body_hi(tp.segs.size(), 0);
    std::vector<dev::TreeTile> tiles, rtiles, htiles, atiles;
    const int64_t vtile = (int64_t)dev::kThreads * L, etile = (int64_t)dev::kThreads * 4;
    auto add_tiles = [](std::vector<dev::TreeTile>* v, int32_t seg, int64_t lo, int64_t hi, int64_t step) {
        for (int64_t st = lo; st < hi; st += step) v->push_back(dev::TreeTile{seg, 0, st, std::min(step, hi - st)});
    };
    for (size_t i = 0; i < tp.segs.size(); i++) {
        const OutSegment& sg = tp.segs[i];
        bool pv = true;
        for (int k = sg.prog_begin; k < sg.prog_begin + sg.prog_len; k++) pv &= (tp.prog[k].shift % L) == 0;
        if (pv) {
            const int64_t lo = (sg.off + L - 1) / L * L - sg.off, hi = (sg.off + sg.n) / L * L - sg.off;
            if (lo < hi) {
                body_lo[i] = lo;
                body_hi[i] = hi;
            }
        }
        add_tiles(&tiles, (int32_t)i, body_lo[i], body_hi[i], vtile);
        // Element pieces shorter than one vector go to the staged kernel.
        auto piece = [&](int64_t lo, int64_t hi) { add_tiles(hi - lo < L ? &htiles : &rtiles, (int32_t)i, lo, hi, etile); };
        if (body_lo[i] < body_hi[i]) {
            piece(0, body_lo[i]);
            piece(body_hi[i], sg.n);
        } else {
            piece(0, sg.n);
        }
        add_tiles(&atiles, (int32_t)i, 0, sg.n, etile);
    }
    d->ntiles = (int)tiles.size();
    d->nrtiles = (int)rtiles.size();
    d->nhtiles = (int)htiles.size();
    d->natiles = (int)atiles.size();
    // Stack slots the kernels index: measured on every program (values
    // alive at once), not taken from the planner's labels.
    d->depth = 1;
    for (const OutSegment& sg : tp.segs) {
        int sp = 0;
        for (int i = sg.prog_begin; i < sg.prog_begin + sg.prog_len; i++) {
            d->depth = std::max(d->depth, ++sp);
            sp -= tp.prog[i].adds;
            if (sp < 1) return fail(BINE_ERR_INTERNAL, "malformed reduction program");
        }
        if (sp != 1) return fail(BINE_ERR_INTERNAL, "malformed reduction program");
    }
    if (d->depth > dev::kMaxTreeDepth) return fail(BINE_ERR_UNSUPPORTED, "reduction tree deeper than supported");
    d->h_tiles = tiles;
    d->h_rtiles = rtiles;
    d->h_htiles = htiles;
    d->h_atiles = atiles;
    for (const OutSegment& sg : tp.segs) d->h_seg_off.push_back(sg.off);
    std::vector<int> uparts;
    std::vector<dev::TreeComb> ucomb;
    for (const OutSegment& sg : tp.segs) {
        uparts.push_back(0);
        uparts.push_back(sg.prog_len);
        ucomb.push_back(dev::TreeComb{0, 0});
    }
    cudaError_t e1, e2, e3, e4, e5, e6, e7, e8;
    put(&d->uparts, uparts, &e7);
    put(&d->ucomb, ucomb, &e8);
    if (e7 != cudaSuccess || e8 != cudaSuccess) return fail(BINE_ERR_CUDA, "uploading the reduction trees failed");
    put(&d->segs, segs, &e1);
    put(&d->prog, prog, &e2);
    put(&d->tiles, tiles, &e3);
    put(&d->rtiles, rtiles, &e4);
    put(&d->htiles, htiles, &e5);
    put(&d->atiles, atiles, &e6);
    if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess || e4 != cudaSuccess || e5 != cudaSuccess ||
        e6 != cudaSuccess)
        return fail(BINE_ERR_CUDA, "uploading the reduction trees failed");
    // Split form of the vector bodies: K lanes per output vector when the
    // output has too few vectors to fill the GPU several times over.
    if (!tiles.empty()) {
        int min_leaves = INT32_MAX;
        for (size_t i = 0; i < tp.segs.size(); i++)
            if (body_lo[i] < body_hi[i]) min_leaves = std::min(min_leaves, tp.segs[i].prog_len);  // one leaf per entry
        int K = 1;
        if (c->tree_split > 0) {
            K = c->tree_split;
            while (K > 1 && min_leaves < K) K /= 2;
        } else {
            // By P, as measured on B200 at 2-4 MiB per rank (GB/s for 1 / 2
            // / 4 / 8 warps per vector group): P = 64: 4649 / 5424 / 5001 /
            // 4407; P = 96: 3508 / 4566 / 4165 / 3661; P = 256: 5481 / 5843 /
            // 6026 / 5879; P = 384: 4023 / 4244 / 4216 / 4065; P = 1000:
            // 2805 / 2825 / 2898 / 3372.
            const int P = c->P;
            K = P < 32 ? 1 : (P < 128 ? 2 : (P < 512 ? 4 : 8));
            // Calls with few output vectors: more lanes per vector until
            // vectors x lanes reach a parallelism target that grows with
            // the tree (2^17 lanes up to P = 128, proportionally above),
            // keeping at least 4 leaves per lane.  Measured on B200
            // (float32, us per call, automatic rule before -> after):
            // P = 96 at 128 KiB / 512 KiB per rank: 21.3 -> 12.1 / 39.0 ->
            // 24.6; P = 384: 51.2 -> 41.0 / 128.2 -> 100.1; P = 64 at
            // 128 KiB: 12.3 -> 8.2.  From 2 MiB per rank the rule by P
            // stands.
            int64_t vecs = 0;
            for (size_t i = 0; i < tp.segs.size(); i++) vecs += (body_hi[i] - body_lo[i]) / L;
            const int64_t target = (int64_t)1 << 17 < (int64_t)1024 * P ? (int64_t)1024 * P : (int64_t)1 << 17;
            while (K < 8 && 8 * K <= P && vecs * K < target) K *= 2;
        }
        while (K > 1 && min_leaves < 2 * K) K /= 2;  // 2K parts of at least one leaf
        if (K > 1) {
            // K parts, one per warp, or 2K parts assigned longest first when
            // that lowers the busiest warp's leaves by 5 % or more (trees of
            // non-power-of-two P do not cut into K equal subtrees).
            auto lpt = [&](const SplitTrees& t, int np, size_t seg, std::vector<std::vector<int>>* mine) {
                const int32_t* po = &t.parts[seg * (np + 1)];
                std::vector<int> order(np), load(K, 0);
                mine->assign(K, {});
                for (int j = 0; j < np; j++) order[j] = j;
                std::stable_sort(order.begin(), order.end(),
                                 [&](int x, int y) { return po[x + 1] - po[x] > po[y + 1] - po[y]; });
                for (int p : order) {
                    const int w = (int)(std::min_element(load.begin(), load.end()) - load.begin());
                    (*mine)[w].push_back(p);
                    load[w] += po[p + 1] - po[p];
                }
                return *std::max_element(load.begin(), load.end());
            };
            SplitTrees s1, s2;
            if (!split_trees(tp, K, &s1, &err) || !split_trees(tp, 2 * K, &s2, &err)) return fail(BINE_ERR_INTERNAL, err);
            long long max1 = 0, max2 = 0;
            std::vector<std::vector<int>> tmp;
            for (size_t i = 0; i < tp.segs.size(); i++) {
                max1 += lpt(s1, K, i, &tmp);
                max2 += lpt(s2, 2 * K, i, &tmp);
            }
            const bool two = max2 * 100 <= max1 * 95;
            const SplitTrees& st = two ? s2 : s1;
            const int KP = two ? 2 * K : K;
            if (st.max_depth > dev::kMaxTreeDepth) return fail(BINE_ERR_UNSUPPORTED, "reduction tree deeper than supported");
            std::vector<dev::TreeSeg> ssegs;
            std::vector<int> sparts, sassign;
            std::vector<dev::TreeComb> scomb;
            std::vector<dev::TreeTile> stiles;
            for (size_t i = 0; i < tp.segs.size(); i++) {
                const OutSegment& sg = tp.segs[i];
                const int32_t* po = &st.parts[i * (KP + 1)];
                const int32_t b = po[0], e = po[KP];
                ssegs.push_back(dev::TreeSeg{sg.off, sg.n, sg.rank, b, e - b, sg.depth});
                d->smax_prog_len = std::max(d->smax_prog_len, e - b);
                for (int j = 0; j <= KP; j++) sparts.push_back(po[j] - b);
                for (int j = 0; j < KP; j++) scomb.push_back(dev::TreeComb{st.comb[i * KP + j].first, st.comb[i * KP + j].second});
                std::vector<std::vector<int>> mine;
                lpt(st, KP, i, &mine);
                std::vector<int> offs{0};
                for (int w = 0; w < K; w++) {
                    sassign.insert(sassign.end(), mine[w].begin(), mine[w].end());
                    offs.push_back(offs.back() + (int)mine[w].size());
                }
                sassign.insert(sassign.end(), offs.begin(), offs.end());
                add_tiles(&stiles, (int32_t)i, body_lo[i], body_hi[i], (int64_t)(dev::kThreads / K) * L);
            }
            d->split_parts = KP;
            FlatTables ft;
            SplitTrees se;
            std::string serr;
            const bool have_se = min_leaves >= 2 * dev::kEdgeParts && split_trees(tp, dev::kEdgeParts, &se, &serr) &&
                                 se.max_depth <= dev::kMaxTreeDepth;
            if (flat_tables(tp, st, have_se ? &se : nullptr, K, KP, sassign, body_lo, body_hi,
                            (int64_t)(dev::kThreads / K) * L, (int)L, c->P, &ft)) {
                cudaError_t g[9];
                put(&d->fbody, ft.body, &g[0]);
                put(&d->franks, ft.ranks, &g[1]);
                put(&d->feshape, ft.eshape, &g[2]);
                put(&d->fadds, ft.adds, &g[3]);
                put(&d->fparts, ft.parts, &g[4]);
                put(&d->fcomb, ft.comb, &g[5]);
                put(&d->fassign, ft.assign, &g[6]);
                put(&d->fedges, ft.edges, &g[7]);
                cudaError_t h[4];
                put(&d->feadds, ft.eadds, &h[0]);
                put(&d->feparts, ft.eparts, &h[1]);
                put(&d->fecomb, ft.ecomb, &h[2]);
                put(&d->feranks_t, ft.eranks_t, &h[3]);
                for (cudaError_t x : h)
                    if (x != cudaSuccess) return fail(BINE_ERR_CUDA, "uploading the row-aligned reduction trees failed");
                d->nfedges = (int)ft.edges.size();
                d->felen = ft.len;
                d->fedepth = ft.edepth;
                // The element kernel keeps only the pieces no edge covers.
                std::vector<dev::TreeTile> keep;
                for (const dev::TreeTile& t : htiles)
                    if (!ft.covered.count({t.seg, t.start})) keep.push_back(t);
                if (!dry) cudaFree(d->htiles);
                d->htiles = nullptr;
                put(&d->htiles, keep, &g[8]);
                for (cudaError_t x : g)
                    if (x != cudaSuccess) return fail(BINE_ERR_CUDA, "uploading the row-aligned reduction trees failed");
                d->nhtiles = (int)keep.size();
                d->h_htiles = keep;
                d->flat = true;
                d->fpitch = ft.pitch;
                d->flen = ft.len;
                d->fmax_ns = ft.max_ns;
                d->fnq = ft.nq;
                d->fnshape = ft.nshape;
                d->h_fedges = ft.edges;
                d->h_fbody = ft.body;
                stiles = std::move(ft.tiles);
            }
            std::vector<dev::TreeEntry> sprog;
            for (const ProgEntry& e : st.prog) sprog.push_back(dev::TreeEntry{e.rank, e.adds, e.shift});
            cudaError_t f1, f2, f3, f4, f5, f6;
            put(&d->ssegs, ssegs, &f1);
            put(&d->sprog, sprog, &f2);
            put(&d->sparts, sparts, &f3);
            put(&d->scomb, scomb, &f4);
            put(&d->stiles, stiles, &f5);
            put(&d->sassign, sassign, &f6);
            if (f1 != cudaSuccess || f2 != cudaSuccess || f3 != cudaSuccess || f4 != cudaSuccess || f5 != cudaSuccess ||
                f6 != cudaSuccess)
                return fail(BINE_ERR_CUDA, "uploading the split reduction trees failed");
            d->nstiles = (int)stiles.size();
            // Stack slots: the deepest part program or combine program.
            int cdepth = 1;
            for (size_t q = 0; q < st.comb.size(); q += KP) {
                int sp = 0;
                for (int j = 0; j < KP; j++) {
                    cdepth = std::max(cdepth, ++sp);
                    sp -= st.comb[q + j].second;
                }
            }
            d->sdepth = std::max(st.max_depth, cdepth);
            d->h_stiles = stiles;
            d->split_k = K;
        }
    }
    if (dry) {
        *out = d;
        return BINE_SUCCESS;
    }
    trim(c->dev_trees, kMaxCachedDeviceTables);
    c->dev_trees.emplace(key, d);
    *out = d;
    return BINE_SUCCESS;
}

unsigned grid_for(const bine_comm_t c, long long work_items) {
    long long blocks = (work_items + dev::kThreads - 1) / dev::kThreads;
    long long cap = (long long)std::max(1, c->num_sms) * 16;
    return (unsigned)std::max(1LL, std::min(blocks, cap));
}

bool aligned16(const void* p) { return ((uintptr_t)p & 15) == 0; }

// ---------------------------------------------------------- fused kernels
// Blocks of `kern` that fit on the device at once (resident capacity).
template <typename K>
unsigned resident_blocks(bine_comm_t c, K kern, int threads, size_t smem) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    return (unsigned)(per_sm * std::max(1, c->num_sms));
}

template <typename T, int COLS>
int launch_sum_cols(bine_comm_t c, int mode, const char* in, long long ist, char* out, long long ost, int P,
                    long long ncol, long long blk_vec, int root) {
    // One tile per block, up to 64 blocks per SM (then grid-stride): the
    // hardware scheduler back-fills SMs as blocks finish, where a single
    // resident wave walking the tiles leaves a tail (measured on B200, P =
    // 256, 4 MiB per rank: 5716 GB/s resident wave, 6347 one tile per
    // block).
    const long long tiles = (ncol + COLS - 1) / COLS;
    const unsigned g = (unsigned)std::min<long long>(tiles, 64LL * std::max(1, c->num_sms));
    if (mode == dev::kSumAllreduce)
        dev::k_sum_vec<T, dev::kSumAllreduce, COLS><<<g, dev::kThreads, 0, c->stream>>>(in, ist, out, ost, P, ncol,
                                                                                         blk_vec, root);
    else if (mode == dev::kSumReduceScatter)
        dev::k_sum_vec<T, dev::kSumReduceScatter, COLS><<<g, dev::kThreads, 0, c->stream>>>(in, ist, out, ost, P,
                                                                                             ncol, blk_vec, root);
    else
        dev::k_sum_vec<T, dev::kSumReduce, COLS><<<g, dev::kThreads, 0, c->stream>>>(in, ist, out, ost, P, ncol,
                                                                                      blk_vec, root);
    CUDA_TRY(cudaGetLastError());
    return BINE_SUCCESS;
}

template <typename T>
int launch_sum(bine_comm_t c, int mode, const char* in, long long ist, char* out, long long ost, long long elems,
               long long blk, int root) {
    const int P = c->P;
    const long long es = sizeof(T);
    const bool vec = aligned16(in) && aligned16(out) && ist % 16 == 0 && ost % 16 == 0 &&
                     (mode != dev::kSumReduceScatter || (blk * es) % 16 == 0);
    long long done = 0;
    if (vec) {
        const long long ncol = elems * es / 16;
        if (ncol > 0) {
            const long long blk_vec = mode == dev::kSumReduceScatter ? blk * es / 16 : 0;
            // Tiles of 64 columns (4 row groups), or 256 (one group) below
            // P = 16; narrower while a call would have fewer than two tiles
            // per SM.  Measured on B200 at 4 MiB per rank (GB/s, old rule ->
            // 64 columns): P = 16: 6406 -> 7084; 64: 5726 -> 6194; 256: 5716
            // -> 6347; 1024: 5751 -> 6316.
            // Below 32 columns a tile has more row groups than that (16 or
            // 32); only for P of at least two rows per group.
            int cols = P < 16 ? 256 : 64;
            while (ncol / cols < 2LL * std::max(1, c->num_sms) &&
                   (cols > 32 || (cols > dev::kSumCols && P >= 2 * (2 * dev::kThreads / cols))))
                cols /= 2;
            int rc;
            switch (cols) {
            case 256: rc = launch_sum_cols<T, 256>(c, mode, in, ist, out, ost, P, ncol, blk_vec, root); break;
            case 128: rc = launch_sum_cols<T, 128>(c, mode, in, ist, out, ost, P, ncol, blk_vec, root); break;
            case 64: rc = launch_sum_cols<T, 64>(c, mode, in, ist, out, ost, P, ncol, blk_vec, root); break;
            case 32: rc = launch_sum_cols<T, 32>(c, mode, in, ist, out, ost, P, ncol, blk_vec, root); break;
            case 16: rc = launch_sum_cols<T, 16>(c, mode, in, ist, out, ost, P, ncol, blk_vec, root); break;
            default: rc = launch_sum_cols<T, 8>(c, mode, in, ist, out, ost, P, ncol, blk_vec, root); break;
            }
            if (rc) return rc;
            done = ncol * 16 / es;
        }
    }
    const long long rest = elems - done;
    if (rest > 0) {
        unsigned g = grid_for(c, rest);
        if (mode == dev::kSumAllreduce)
            dev::k_sum_scalar<T, dev::kSumAllreduce><<<g, dev::kThreads, 0, c->stream>>>(in, ist, out, ost, P, done, rest, blk, root);
        else if (mode == dev::kSumReduceScatter)
            dev::k_sum_scalar<T, dev::kSumReduceScatter><<<g, dev::kThreads, 0, c->stream>>>(in, ist, out, ost, P, done, rest, blk, root);
        else
            dev::k_sum_scalar<T, dev::kSumReduce><<<g, dev::kThreads, 0, c->stream>>>(in, ist, out, ost, P, done, rest, blk, root);
    }
    CUDA_TRY(cudaGetLastError());
    return BINE_SUCCESS;
}

int launch_sum_dt(bine_comm_t c, int dt, int mode, const char* in, long long ist, char* out, long long ost,
                  long long elems, long long blk, int root) {
    switch (dt) {
    case BINE_INT32: return launch_sum<int32_t>(c, mode, in, ist, out, ost, elems, blk, root);
    case BINE_INT64: return launch_sum<int64_t>(c, mode, in, ist, out, ost, elems, blk, root);
    case BINE_FLOAT: return launch_sum<float>(c, mode, in, ist, out, ost, elems, blk, root);
    case BINE_DOUBLE: return launch_sum<double>(c, mode, in, ist, out, ost, elems, blk, root);
    case BINE_CHAR: return launch_sum<int8_t>(c, mode, in, ist, out, ost, elems, blk, root);
    }
    return fail(BINE_ERR_ARG, "bad datatype");
}

// Dynamic shared memory of the vector tree kernels: the segment's program
// (16-byte entries), then, when it fits, the per-thread evaluation stacks
// (`depth` slots of 16 bytes per thread).
struct TreeSmem {
    size_t bytes;
    int stack_off;  // in 16-byte words
    bool stack;
};
TreeSmem tree_smem(int prog_len, int depth) {
    static_assert(sizeof(dev::TreeEntry) == 16, "program entries are 16-byte words");
    const size_t prog = (size_t)std::max(1, prog_len) * 16;
    const size_t stack = (size_t)std::max(1, depth) * dev::kThreads * 16;
    const bool in_smem = stack <= 64 * 1024 && prog + stack <= 200 * 1024;
    return TreeSmem{prog + (in_smem ? stack : 0), (int)(prog / 16), in_smem};
}

template <typename K>
int launch_tree_kernel(bine_comm_t c, K kern, size_t smem, long long ntiles, unsigned* grid) {
    // Static and dynamic shared memory together: above 48 KB the dynamic
    // part needs the opt-in attribute, above 227 KB it cannot launch.
    cudaFuncAttributes fa;
    CUDA_TRY(cudaFuncGetAttributes(&fa, kern));
    if (smem + fa.sharedSizeBytes > 227 * 1024)
        return fail(BINE_ERR_UNSUPPORTED, "reduction program does not fit in shared memory");
    if (smem + fa.sharedSizeBytes > 48 * 1024)
        CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    // One block per tile, up to 64 blocks per SM (then grid-stride): the
    // hardware back-fills SMs as blocks finish.  Measured on B200 against a
    // single resident wave walking the tiles (float32, GB/s): P = 96: 4567
    // -> 4664; 256: 6060 -> 6245; 384: 4206 -> 4465; 1000: 3387 -> 4051.
    *grid = (unsigned)std::max(1LL, std::min<long long>(ntiles, 64LL * std::max(1, c->num_sms)));
    return BINE_SUCCESS;
}

template <typename T, int K>
int launch_tree_split(bine_comm_t c, const DevTrees& d, const char* in, long long ist, char* out, long long ost,
                      const dev::TreeTile* stiles, int nstiles) {
    if (nstiles == 0) return BINE_SUCCESS;
    const TreeSmem sm = tree_smem(d.smax_prog_len, d.sdepth);
    auto kern = sm.stack ? dev::k_tree_split<T, K, true> : dev::k_tree_split<T, K, false>;
    unsigned g = 0;
    int rc = launch_tree_kernel(c, kern, sm.bytes, nstiles, &g);
    if (rc) return rc;
    kern<<<g, dev::kThreads, sm.bytes, c->stream>>>(in, ist, out, ost, c->P, d.ssegs, d.sprog, d.sparts, d.scomb,
                                                    d.sassign, stiles, nstiles, d.split_parts, sm.stack_off);
    CUDA_TRY(cudaGetLastError());
    return BINE_SUCCESS;
}

// Arguments and dynamic shared memory of the row-aligned kernels: the
// common additions, the ranks of up to `fmax_ns` segments (row tiles only),
// then the evaluation stacks when they fit.
struct FlatLaunch {
    dev::FlatArgs a;
    size_t smem;
    bool in_smem;
};
FlatLaunch flat_launch(bine_comm_t c, const DevTrees& d, const char* in, long long ist, char* out, long long ost,
                       const dev::TreeTile* tiles, int ntiles, bool rows) {
    const size_t adds = (size_t)d.flen, ranks = rows ? ((size_t)d.fmax_ns * d.fpitch * 2 + 15) / 16 * 16 : 0;
    const size_t stack = (size_t)std::max(1, d.sdepth) * dev::kThreads * 16;
    FlatLaunch f;
    f.in_smem = stack <= 64 * 1024 && adds + ranks + stack <= 200 * 1024;
    f.smem = adds + ranks + (f.in_smem ? stack : 0);
    dev::FlatArgs& a = f.a;
    a.in = in;
    a.in_stride = ist;
    a.out = out;
    a.out_stride = ost;
    a.P = c->P;
    a.body = d.fbody;
    a.ranks = d.franks;
    a.pitch = d.fpitch;
    a.nq = d.fnq;
    a.adds = d.fadds;
    a.len = d.flen;
    a.parts = d.fparts;
    a.comb = d.fcomb;
    a.assign = d.fassign;
    a.edges = d.fedges;
    a.tiles = tiles;
    a.ntiles = ntiles;
    a.nparts = d.split_parts;
    a.ranks_off = (int)(adds / 16);
    a.stack_off = (int)((adds + ranks) / 16);
    return f;
}

template <typename T, int K>
int launch_tree_flat(bine_comm_t c, const DevTrees& d, const char* in, long long ist, char* out, long long ost,
                     const dev::TreeTile* ftiles, int nftiles) {
    if (nftiles == 0) return BINE_SUCCESS;
    const FlatLaunch f = flat_launch(c, d, in, ist, out, ost, ftiles, nftiles, true);
    auto kern = f.in_smem ? dev::k_tree_flat<T, K, true> : dev::k_tree_flat<T, K, false>;
    unsigned g = 0;
    int rc = launch_tree_kernel(c, kern, f.smem, nftiles, &g);
    if (rc) return rc;
    kern<<<g, dev::kThreads, f.smem, c->stream>>>(f.a);
    CUDA_TRY(cudaGetLastError());
    return BINE_SUCCESS;
}

template <typename T>
int launch_tree_edges(bine_comm_t c, const DevTrees& d, const char* in, long long ist, char* out, long long ost,
                      int first, int nedges, cudaStream_t s) {
    if (nedges == 0) return BINE_SUCCESS;
    // Dynamic shared memory: every shape's edge additions, then the stacks.
    const size_t adds = (size_t)d.fnshape * d.felen, stack = (size_t)std::max(1, d.fedepth) * dev::kThreads * 16;
    const bool in_smem = stack <= 64 * 1024 && adds + stack <= 200 * 1024;
    const size_t smem = adds + (in_smem ? stack : 0);
    dev::FlatArgs a{};
    a.in = in;
    a.in_stride = ist;
    a.out = out;
    a.out_stride = ost;
    a.P = c->P;
    a.ranks_t = d.feranks_t;
    a.nq = d.fnq;
    a.adds = d.feadds;
    a.len = d.felen;
    a.parts = d.feparts;
    a.comb = d.fecomb;
    a.edges = d.fedges + first;
    a.shape = d.feshape;
    a.nshape = d.fnshape;
    a.stack_off = (int)(adds / 16);
    auto kern = in_smem ? dev::k_tree_edges<T, true> : dev::k_tree_edges<T, false>;
    unsigned g = 0;
    int rc = launch_tree_kernel(c, kern, smem, 2LL * ((nedges + 31) / 32), &g);
    if (rc) return rc;
    kern<<<g, dev::kThreads, smem, s>>>(a, nedges);
    CUDA_TRY(cudaGetLastError());
    return BINE_SUCCESS;
}

// Tile lists of a launch: vector tiles (one-lane and split forms) and
// element tiles (the remainder, or everything for unaligned layouts).
struct TileSet {
    // vector one-lane, vector split (or row-aligned rows), element
    // remainder, short element pieces, element all, row-aligned edges
    const dev::TreeTile* t[6];
    int n[6];
    int edge0;  // row-aligned edges: the first (list 5 holds no tiles, n[5] counts edges)
};

TileSet all_tiles(const DevTrees& d) {
    return TileSet{{d.tiles, d.stiles, d.rtiles, d.htiles, d.atiles, nullptr},
                   {d.ntiles, d.nstiles, d.nrtiles, d.nhtiles, d.natiles, d.nfedges}, 0};
}

// Evaluates the trees of `d` over the tiles of `ts` (all of them, or one
// column window's).  On a 16-byte-aligned layout the vector tiles (split
// form when the plan has one) run on the communicator's stream while the
// element pieces run beside them on a side stream (forked and joined by
// events, which graph capture also records); otherwise every element tile
// runs on the element kernel.
template <typename T>
int launch_tree(bine_comm_t c, const DevTrees& d, const char* in, long long ist, char* out, long long ost,
                const TileSet& ts) {
    const bool vec = aligned16(in) && aligned16(out) && ist % 16 == 0 && ost % 16 == 0;
    unsigned g = 0;
    int rc;
    const bool edges = vec && d.flat && ts.n[5] > 0;
    const bool side = vec && (ts.n[2] > 0 || ts.n[3] > 0 || edges);
    cudaStream_t es = c->stream;
    if (side) {
        CUDA_TRY(cudaEventRecord(c->ev_fork, c->stream));
        CUDA_TRY(cudaStreamWaitEvent(c->side, c->ev_fork, 0));
        es = c->side;
        if (edges) {
            rc = launch_tree_edges<T>(c, d, in, ist, out, ost, ts.edge0, ts.n[5], es);
            if (rc) return rc;
        }
        if (ts.n[3] > 0) {
            // The split plan's parts when there is one (its segments index
            // the same output runs), else each whole tree as one part.
            const bool split = d.split_k > 1;
            if (split && d.split_parts > dev::kMaxParts) return fail(BINE_ERR_INTERNAL, "too many tree parts");
            const int plen = std::max(1, split ? d.smax_prog_len : d.max_prog_len);
            const size_t prog = (size_t)plen * sizeof(dev::TreeEntry);
            const size_t smem = prog + (size_t)(16 / sizeof(T) - 1) * plen * sizeof(T);
            rc = launch_tree_kernel(c, dev::k_tree_staged<T>, smem, ts.n[3], &g);
            if (rc) return rc;
            dev::k_tree_staged<T><<<g, dev::kThreads, smem, es>>>(
                in, ist, out, ost, c->P, split ? d.ssegs : d.segs, split ? d.sprog : d.prog,
                split ? d.sparts : d.uparts, split ? d.scomb : d.ucomb, split ? d.split_parts : 1, ts.t[3], ts.n[3],
                (int)(prog / 16));
            CUDA_TRY(cudaGetLastError());
        }
    }
    if (vec && d.flat && ts.n[1] > 0) {
        switch (d.split_k) {
        case 2: rc = launch_tree_flat<T, 2>(c, d, in, ist, out, ost, ts.t[1], ts.n[1]); break;
        case 4: rc = launch_tree_flat<T, 4>(c, d, in, ist, out, ost, ts.t[1], ts.n[1]); break;
        default: rc = launch_tree_flat<T, 8>(c, d, in, ist, out, ost, ts.t[1], ts.n[1]); break;
        }
        if (rc) return rc;
    } else if (vec && d.split_k > 1 && ts.n[1] > 0) {
        switch (d.split_k) {
        case 2: rc = launch_tree_split<T, 2>(c, d, in, ist, out, ost, ts.t[1], ts.n[1]); break;
        case 4: rc = launch_tree_split<T, 4>(c, d, in, ist, out, ost, ts.t[1], ts.n[1]); break;
        default: rc = launch_tree_split<T, 8>(c, d, in, ist, out, ost, ts.t[1], ts.n[1]); break;
        }
        if (rc) return rc;
    } else if (vec && ts.n[0] > 0) {
        const TreeSmem sm = tree_smem(d.max_prog_len, d.depth);
        auto kern = sm.stack ? dev::k_tree_vec<T, true> : dev::k_tree_vec<T, false>;
        rc = launch_tree_kernel(c, kern, sm.bytes, ts.n[0], &g);
        if (rc) return rc;
        kern<<<g, dev::kThreads, sm.bytes, c->stream>>>(in, ist, out, ost, c->P, d.segs, d.prog, ts.t[0], ts.n[0],
                                                        sm.stack_off);
        CUDA_TRY(cudaGetLastError());
    }
    const dev::TreeTile* et = vec ? ts.t[2] : ts.t[4];
    const int ne = vec ? ts.n[2] : ts.n[4];
    if (ne > 0) {
        const size_t smem = (size_t)std::max(1, d.max_prog_len) * sizeof(dev::TreeEntry);
        rc = launch_tree_kernel(c, dev::k_tree_scalar<T>, smem, ne, &g);
        if (rc) return rc;
        dev::k_tree_scalar<T><<<g, dev::kThreads, smem, es>>>(in, ist, out, ost, c->P, d.segs, d.prog, et, ne);
        CUDA_TRY(cudaGetLastError());
    }
    if (side) {
        CUDA_TRY(cudaEventRecord(c->ev_join, c->side));
        CUDA_TRY(cudaStreamWaitEvent(c->stream, c->ev_join, 0));
    }
    return BINE_SUCCESS;
}

int launch_copy(bine_comm_t c, int mode, const char* in, long long ist, char* out, long long ost, long long unit,
                int root, int es) {
    dev::CopyArgs a{in, ist, out, ost, c->P, root, unit, 1};
    long long pairs = mode == dev::kCopyAlltoall ? (long long)c->P * c->P : (mode == dev::kCopyBcast ? 1 : c->P);
    if (unit == 0) return BINE_SUCCESS;
    const bool vec = aligned16(in) && aligned16(out) && ist % 16 == 0 && ost % 16 == 0 && unit % 16 == 0;
    // Allgather and bcast store every source vector to P rows.  A call whose
    // source units would give fewer than half the SMs a block leaves most
    // of the GPU idle: its rows are then split over threads, enough groups
    // for two blocks per SM (at least 8 rows each).  Calls that already
    // reach most SMs stream their stores at full rate unsplit.  Measured
    // on B200 (int64, us): bcast P = 1024 at 8 KiB per rank 69.7 -> 4.4,
    // allgather P = 1024 at 32 B 69.8 -> 8.3; allgather P = 1024 at 512 B
    // (128 blocks) 78 unsplit, 95 split in 3.
    const long long units = pairs * (vec ? unit / 16 : unit / es);
    const long long fill = 2LL * dev::kThreads * std::max(1, c->num_sms);
    if ((mode == dev::kCopyAllgather || mode == dev::kCopyBcast) && 4 * units < fill)
        a.dgroups = (int)std::max<long long>(1, std::min<long long>(std::max(1, c->P / 8), (fill + units - 1) / units));
    if (vec) {
        unsigned g = grid_for(c, pairs * (unit / 16) * a.dgroups);
        switch (mode) {
        case dev::kCopyAllgather: dev::k_copy_vec<dev::kCopyAllgather><<<g, dev::kThreads, 0, c->stream>>>(a); break;
        case dev::kCopyBcast: dev::k_copy_vec<dev::kCopyBcast><<<g, dev::kThreads, 0, c->stream>>>(a); break;
        case dev::kCopyAlltoall: dev::k_copy_vec<dev::kCopyAlltoall><<<g, dev::kThreads, 0, c->stream>>>(a); break;
        case dev::kCopyScatter: dev::k_copy_vec<dev::kCopyScatter><<<g, dev::kThreads, 0, c->stream>>>(a); break;
        case dev::kCopyGather: dev::k_copy_vec<dev::kCopyGather><<<g, dev::kThreads, 0, c->stream>>>(a); break;
        }
    } else {
        unsigned g = grid_for(c, pairs * (unit / es) * a.dgroups);
#define BINE_COPY_SCALAR(U)                                                                                          \
    switch (mode) {                                                                                                  \
    case dev::kCopyAllgather: dev::k_copy_scalar<dev::kCopyAllgather, U><<<g, dev::kThreads, 0, c->stream>>>(a); break; \
    case dev::kCopyBcast: dev::k_copy_scalar<dev::kCopyBcast, U><<<g, dev::kThreads, 0, c->stream>>>(a); break;         \
    case dev::kCopyAlltoall: dev::k_copy_scalar<dev::kCopyAlltoall, U><<<g, dev::kThreads, 0, c->stream>>>(a); break;   \
    case dev::kCopyScatter: dev::k_copy_scalar<dev::kCopyScatter, U><<<g, dev::kThreads, 0, c->stream>>>(a); break;     \
    case dev::kCopyGather: dev::k_copy_scalar<dev::kCopyGather, U><<<g, dev::kThreads, 0, c->stream>>>(a); break;       \
    }
        if (es == 8 && ((uintptr_t)in | (uintptr_t)out | ist | ost | unit) % 8 == 0) {
            BINE_COPY_SCALAR(uint64_t)
        } else if (es >= 4 && ((uintptr_t)in | (uintptr_t)out | ist | ost | unit) % 4 == 0) {
            BINE_COPY_SCALAR(uint32_t)
        } else {
            BINE_COPY_SCALAR(uint8_t)
        }
#undef BINE_COPY_SCALAR
    }
    CUDA_TRY(cudaGetLastError());
    return BINE_SUCCESS;
}

// ------------------------------------------------------------ step engine
template <typename T>
int launch_steps(bine_comm_t c, const DevSteps& d, const char* send, long long ist, char* recv, long long ost) {
    if (d.nlevels == 0) return BINE_SUCCESS;
    const size_t es = sizeof(T);
    const size_t tmp_stride = ((size_t)d.tmp_elems * es + 255) / 256 * 256;
    int rc = ensure_work(c, std::max<size_t>(tmp_stride * c->P, 256));
    if (rc) return rc;
    dev::StepBufs B;
    B.base[kBufSend] = const_cast<char*>(send);
    B.base[kBufRecv] = recv;
    B.base[kBufTmp] = c->work;
    B.stride[kBufSend] = ist;
    B.stride[kBufRecv] = ost;
    B.stride[kBufTmp] = (long long)tmp_stride;
    int per_sm = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dev::k_steps<T>, dev::kThreads, 0));
    int blocks = std::max(1, std::min(per_sm * c->num_sms, std::max(1, d.max_chunks_per_level)));
    CUDA_TRY(cudaMemsetAsync(c->barrier, 0, 2 * sizeof(unsigned), c->stream));
    const dev::StepMove* moves = d.moves;
    const dev::StepChunk* chunks = d.chunks;
    const int* lb = d.level_begin;
    int nl = d.nlevels;
    unsigned* bar = c->barrier;
    int* status = c->status;
    unsigned long long to = c->step_timeout_ns;
    unsigned expected = (unsigned)blocks + c->barrier_extra;
    void* args[] = {&B, &moves, &chunks, &lb, &nl, &bar, &status, &to, &expected};
    CUDA_TRY(cudaLaunchCooperativeKernel((void*)dev::k_steps<T>, dim3(blocks), dim3(dev::kThreads), args, 0, c->stream));
    return BINE_SUCCESS;
}

template <typename T>
int launch_flow(bine_comm_t c, const DevSteps& d, const DevFlow& f, const char* send, long long ist, char* recv,
                long long ost) {
    if (f.nitems == 0) return BINE_SUCCESS;
    const size_t es = sizeof(T);
    const size_t tmp_stride = ((size_t)d.tmp_elems * es + 255) / 256 * 256;
    int rc = ensure_work(c, std::max<size_t>(tmp_stride * c->P, 256));
    if (rc) return rc;
    dev::StepBufs B;
    B.base[kBufSend] = const_cast<char*>(send);
    B.base[kBufRecv] = recv;
    B.base[kBufTmp] = c->work;
    B.stride[kBufSend] = ist;
    B.stride[kBufRecv] = ost;
    B.stride[kBufTmp] = (long long)tmp_stride;
    int per_sm = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dev::k_flow<T>, dev::kFlowThreads, 0));
    // Resident blocks only: the waits need no co-residency (every dependency
    // was handed out earlier), but blocks beyond that would only queue.
    const int blocks = std::max(1, std::min(std::max(1, per_sm) * c->num_sms, f.nitems));
    dev::k_flow<T><<<blocks, dev::kFlowThreads, 0, c->stream>>>(B, d.moves, f.pieces, f.items, f.nitems, f.deps,
                                                             f.level_items, f.nlevels, f.done, f.ctl, c->status,
                                                             c->step_timeout_ns, c->barrier_extra);
    CUDA_TRY(cudaGetLastError());
    return BINE_SUCCESS;
}

template <typename T>
int launch_flow_fused(bine_comm_t c, const DevFused& d, const char* send, long long ist, char* recv, long long ost) {
    const DevFlow& f = d.flow;
    if (f.nitems == 0) return BINE_SUCCESS;
    const size_t es = sizeof(T);
    const size_t tmp_stride = ((size_t)d.tmp_elems * es + 255) / 256 * 256;
    int rc = ensure_work(c, std::max<size_t>(tmp_stride * c->P, 256));
    if (rc) return rc;
    dev::StepBufs B;
    B.base[kBufSend] = const_cast<char*>(send);
    B.base[kBufRecv] = recv;
    B.base[kBufTmp] = c->work;
    B.stride[kBufSend] = ist;
    B.stride[kBufRecv] = ost;
    B.stride[kBufTmp] = (long long)tmp_stride;
    int per_sm = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dev::k_flow_fused<T>, dev::kFlowThreads, 0));
    const int blocks = std::max(1, std::min(std::max(1, per_sm) * c->num_sms, f.nitems));
    dev::k_flow_fused<T><<<blocks, dev::kFlowThreads, 0, c->stream>>>(
        B, d.moves, d.leaves, d.dsts, f.pieces, f.items, f.nitems, f.deps, f.level_items, f.nlevels, f.done, f.ctl,
        c->status, c->step_timeout_ns, c->barrier_extra);
    CUDA_TRY(cudaGetLastError());
    return BINE_SUCCESS;
}

int launch_flow_fused_dt(bine_comm_t c, int dt, const DevFused& d, const char* send, long long ist, char* recv,
                         long long ost) {
    switch (dt) {
    case BINE_INT32: return launch_flow_fused<int32_t>(c, d, send, ist, recv, ost);
    case BINE_INT64: return launch_flow_fused<int64_t>(c, d, send, ist, recv, ost);
    case BINE_FLOAT: return launch_flow_fused<float>(c, d, send, ist, recv, ost);
    case BINE_DOUBLE: return launch_flow_fused<double>(c, d, send, ist, recv, ost);
    case BINE_CHAR: return launch_flow_fused<int8_t>(c, d, send, ist, recv, ost);
    }
    return fail(BINE_ERR_ARG, "bad datatype");
}

int launch_flow_dt(bine_comm_t c, int dt, const DevSteps& d, const DevFlow& f, const char* send, long long ist,
                   char* recv, long long ost) {
    switch (dt) {
    case BINE_INT32: return launch_flow<int32_t>(c, d, f, send, ist, recv, ost);
    case BINE_INT64: return launch_flow<int64_t>(c, d, f, send, ist, recv, ost);
    case BINE_FLOAT: return launch_flow<float>(c, d, f, send, ist, recv, ost);
    case BINE_DOUBLE: return launch_flow<double>(c, d, f, send, ist, recv, ost);
    case BINE_CHAR: return launch_flow<int8_t>(c, d, f, send, ist, recv, ost);
    }
    return fail(BINE_ERR_ARG, "bad datatype");
}

int launch_steps_dt(bine_comm_t c, int dt, const DevSteps& d, const char* send, long long ist, char* recv,
                    long long ost) {
    switch (dt) {
    case BINE_INT32: return launch_steps<int32_t>(c, d, send, ist, recv, ost);
    case BINE_INT64: return launch_steps<int64_t>(c, d, send, ist, recv, ost);
    case BINE_FLOAT: return launch_steps<float>(c, d, send, ist, recv, ost);
    case BINE_DOUBLE: return launch_steps<double>(c, d, send, ist, recv, ost);
    case BINE_CHAR: return launch_steps<int8_t>(c, d, send, ist, recv, ost);
    }
    return fail(BINE_ERR_ARG, "bad datatype");
}

bool is_reduction(int coll) { return coll == kAllreduce || coll == kReduceScatter || coll == kReduce; }

// Per-rank element counts of the send and receive rows.
void row_elems(int coll, long long count, int P, long long* se, long long* re) {
    switch (coll) {
    case kAllreduce:
    case kReduce: *se = count; *re = count; break;
    case kBcast: *se = 0; *re = count; break;
    case kReduceScatter:
    case kScatter: *se = count * P; *re = count; break;
    case kAllgather:
    case kGather: *se = count; *re = count * P; break;
    case kAlltoall: *se = count * P; *re = count * P; break;
    default: *se = *re = 0;
    }
}

// Whether the rank-major arrays [a, a + ast*(P-1) + arow) and
// [b, b + bst*(P-1) + brow) share any byte.
bool arrays_overlap(const void* a, long long ast, size_t arow, const void* b, long long bst, size_t brow, int P) {
    if (!a || !b || !arow || !brow) return false;
    const uintptr_t a0 = (uintptr_t)a, b0 = (uintptr_t)b;
    const uintptr_t a1 = a0 + (uintptr_t)ast * (uintptr_t)(P - 1) + arow;
    const uintptr_t b1 = b0 + (uintptr_t)bst * (uintptr_t)(P - 1) + brow;
    return a0 < b1 && b0 < a1;
}

int run_collective(bine_comm_t c, int coll, const void* sendbuf, void* recvbuf, long long count, int dt, int root) {
    if (!c) return fail(BINE_ERR_ARG, "null communicator");
    const int es = dtype_size(dt);
    if (es < 0) return fail(BINE_ERR_ARG, "invalid datatype");
    if (count < 0) return fail(BINE_ERR_ARG, "negative count");
    if (root < 0 || root >= c->P) return fail(BINE_ERR_ARG, "root out of range");
    long long se, re;
    row_elems(coll, count, c->P, &se, &re);
    if ((se && !sendbuf) || (re && !recvbuf)) return fail(BINE_ERR_ARG, "null buffer");
    long long ist = c->send_stride ? (long long)c->send_stride : se * es;
    const long long ost = c->recv_stride ? (long long)c->recv_stride : re * es;
    if (ist < se * es || ost < re * es) return fail(BINE_ERR_ARG, "layout stride smaller than a rank row");
    if (count == 0) return BINE_SUCCESS;
    int rc = ensure_device(c);
    if (rc) return rc;
    const char* in = (const char*)sendbuf;
    char* out = (char*)recvbuf;
    PlanKey k = make_key(c, coll, count, root);

    // Input and output arrays that share bytes (MPI_IN_PLACE, or rows laid
    // out so that they interleave): the step schedules read a rank's send
    // row in the same step that writes receive rows (the L butterfly reads
    // its peer's input while the peer's result is written), and the copy
    // kernels and the reduce_scatter tiles write rows that other blocks still
    // read.  Such calls take their input rows from a staged copy.  The one
    // exception is an allreduce or reduce on the FUSED engine whose arrays
    // are one (same base, same stride) and whose columns each have one
    // writing tile: that tile reads its columns of all rows before writing
    // them, and no other tile touches them.  Per-rank float trees (the L
    // butterfly in the reference order) give one tile per rank and column,
    // so they are staged too.
    bool alias_safe = c->engine == BINE_ENGINE_FUSED && (coll == kAllreduce || coll == kReduce) &&
                      (const void*)in == (const void*)out && ist == ost;
    if (alias_safe && coll == kAllreduce && (dt == BINE_FLOAT || dt == BINE_DOUBLE) &&
        c->order == BINE_ORDER_REFERENCE) {
        // Per-rank addition trees (the L butterfly): the tile of one rank's
        // row reads, at the same columns, the rows other tiles write.
        std::shared_ptr<DevTrees> d;
        rc = get_dev_trees(c, k, es, &d);
        if (rc) return rc;
        alias_safe = !d->per_rank;
    }
    if (arrays_overlap(in, ist, (size_t)se * es, out, ost, (size_t)re * es, c->P) && !alias_safe) {
        const size_t pitch = ((size_t)se * es + 255) / 256 * 256, bytes = pitch * (size_t)c->P;
        if (c->inplace_bytes < bytes) {
            CUDA_TRY(cudaStreamSynchronize(c->stream));
            cudaFree(c->inplace);
            c->inplace = nullptr;
            c->inplace_bytes = 0;
            CUDA_TRY(cudaMalloc(&c->inplace, bytes));
            c->inplace_bytes = bytes;
        }
        CUDA_TRY(cudaMemcpy2DAsync(c->inplace, pitch, in, ist, (size_t)se * es, c->P, cudaMemcpyDeviceToDevice,
                                   c->stream));
        in = c->inplace;
        ist = (long long)pitch;
    }
    if (c->engine == BINE_ENGINE_STEPS) {
        std::shared_ptr<DevSteps> d;
        rc = get_dev_steps(c, k, es, &d);
        if (rc) return rc;
        return launch_steps_dt(c, dt, *d, in, ist, out, ost);
    }
    std::shared_ptr<Schedule> sched;
    if (c->engine == BINE_ENGINE_PIPELINED) {
        rc = get_schedule(c, k, &sched);
        if (rc) return rc;
    }
    if (c->engine == BINE_ENGINE_PIPELINED && fusion_levels(c, coll, sched.get()) > 1) {
        std::shared_ptr<DevFused> d;
        rc = get_dev_fused(c, k, es, &d);
        if (rc) return rc;
        return launch_flow_fused_dt(c, dt, *d, in, ist, out, ost);
    }
    if (c->engine == BINE_ENGINE_PIPELINED) {
        std::shared_ptr<DevSteps> d;
        std::shared_ptr<DevFlow> f;
        rc = get_dev_flow(c, k, es, &d, &f);
        if (rc) return rc;
        return launch_flow_dt(c, dt, *d, *f, in, ist, out, ost);
    }

    if (is_reduction(coll)) {
        const bool exact = (dt == BINE_FLOAT || dt == BINE_DOUBLE) && c->order == BINE_ORDER_REFERENCE;
        if (exact) {
            std::shared_ptr<DevTrees> d;
            rc = get_dev_trees(c, k, es, &d);
            if (rc) return rc;
            return dt == BINE_FLOAT ? launch_tree<float>(c, *d, in, ist, out, ost, all_tiles(*d))
                                    : launch_tree<double>(c, *d, in, ist, out, ost, all_tiles(*d));
        }
        const int mode = coll == kAllreduce ? dev::kSumAllreduce
                                            : (coll == kReduceScatter ? dev::kSumReduceScatter : dev::kSumReduce);
        return launch_sum_dt(c, dt, mode, in, ist, out, ost, se, count, root);
    }
    switch (coll) {
    case kAllgather: return launch_copy(c, dev::kCopyAllgather, in, ist, out, ost, count * es, root, es);
    case kBcast: return launch_copy(c, dev::kCopyBcast, out, ost, out, ost, count * es, root, es);
    case kAlltoall: return launch_copy(c, dev::kCopyAlltoall, in, ist, out, ost, count * es, root, es);
    case kScatter: return launch_copy(c, dev::kCopyScatter, in, ist, out, ost, count * es, root, es);
    case kGather: return launch_copy(c, dev::kCopyGather, in, ist, out, ost, count * es, root, es);
    }
    return fail(BINE_ERR_ARG, "unknown collective");
}

// ------------------------------------------------------ host-buffer path
// Tiles of `d` clipped to each column window [i*W, min(count, (i+1)*W)),
// uploaded once per window width.  W is a multiple of 16 bytes, so clipped
// vector tiles stay aligned.
int window_tiles(bine_comm_t c, DevTrees& d, long long W, long long count, const DevTrees::Windows** out) {
    std::lock_guard<std::mutex> lk(c->mu);
    auto it = d.windows.find(W);
    if (it == d.windows.end()) {
        // Tiles hold a segment and a start inside it, except the row-aligned
        // form's, which hold absolute starts (and a segment range, kept).
        auto clip = [&](const std::vector<dev::TreeTile>& in, bool absolute, long long c0, long long c1,
                        std::vector<dev::TreeTile>* o) {
            for (const dev::TreeTile& t : in) {
                const long long base = absolute ? 0 : d.h_seg_off[t.seg];
                const long long lo = base + t.start, hi = lo + t.n;
                const long long a = std::max(lo, c0), b = std::min(hi, c1);
                if (a < b) o->push_back(dev::TreeTile{t.seg, t.pad, a - base, b - a});
            }
        };
        const std::vector<dev::TreeTile>* lists[5] = {&d.h_tiles, &d.h_stiles, &d.h_rtiles, &d.h_htiles,
                                                      &d.h_atiles};
        DevTrees::Windows w;
        // Row-aligned edges: per window, the first edge at or after its start.
        for (long long c0 = 0; c0 < count; c0 += W) {
            int a = 0;
            while (a < (int)d.h_fedges.size() && d.h_fedges[a].e < c0) a++;
            w.begin[5].push_back(a);
        }
        w.begin[5].push_back((int)d.h_fedges.size());
        for (int k = 0; k < 5; k++) {
            std::vector<dev::TreeTile> v;
            for (long long c0 = 0; c0 < count; c0 += W) {
                w.begin[k].push_back((int)v.size());
                clip(*lists[k], k == 1 && d.flat, c0, std::min(count, c0 + W), &v);
            }
            w.begin[k].push_back((int)v.size());
            cudaError_t e;
            fill(&w.tiles[k], v, &e);
            if (e != cudaSuccess) {
                for (auto* t : w.tiles) cudaFree(t);
                return fail(BINE_ERR_CUDA, "uploading window tiles failed");
            }
        }
        it = d.windows.emplace(W, std::move(w)).first;
    }
    *out = &it->second;
    return BINE_SUCCESS;
}

template <typename T>
int launch_tree_window(bine_comm_t c, const DevTrees& d, const DevTrees::Windows* w, long long i, const char* in,
                       long long ist, char* out, long long ost) {
    if (!w) return launch_tree<T>(c, d, in, ist, out, ost, all_tiles(d));
    TileSet ts;
    for (int k = 0; k < 5; k++) {
        ts.t[k] = w->tiles[k] + w->begin[k][i];
        ts.n[k] = w->begin[k][i + 1] - w->begin[k][i];
    }
    ts.t[5] = nullptr;
    ts.edge0 = w->begin[5][i];
    ts.n[5] = w->begin[5][i + 1] - w->begin[5][i];
    return launch_tree<T>(c, d, in, ist, out, ost, ts);
}

// Allreduce of rank-major HOST arrays.  Column windows of the P rows flow
// through two device slots on three streams: the host->device copy of
// window i+1, the reduction of window i and the device->host copy of window
// i-1 run at once, so both PCIe directions stay busy.  The fused kernels do
// the reduction (exact trees with windowed tiles in the reference float
// order), so results equal bine_allreduce's.
int allreduce_host(bine_comm_t c, const void* sendbuf, void* recvbuf, long long count, int dt,
                   bine_window_hook_t before = nullptr, bine_window_hook_t after = nullptr, void* user = nullptr) {
    const int es = dtype_size(dt);
    if (es < 0) return fail(BINE_ERR_ARG, "invalid datatype");
    if (count < 0) return fail(BINE_ERR_ARG, "negative count");
    if (count > 0 && (!sendbuf || !recvbuf)) return fail(BINE_ERR_ARG, "null buffer");
    const long long ist = c->send_stride ? (long long)c->send_stride : count * es;
    const long long ost = c->recv_stride ? (long long)c->recv_stride : count * es;
    if (ist < count * es || ost < count * es) return fail(BINE_ERR_ARG, "layout stride smaller than a rank row");
    if (count == 0) return BINE_SUCCESS;
    int rc = ensure_device(c);
    if (rc) return rc;
    if (!c->h2d) {
        CUDA_TRY(cudaStreamCreateWithFlags(&c->h2d, cudaStreamNonBlocking));
        CUDA_TRY(cudaStreamCreateWithFlags(&c->d2h, cudaStreamNonBlocking));
        CUDA_TRY(cudaEventCreateWithFlags(&c->ev_start, cudaEventDisableTiming));
        for (int s = 0; s < 2; s++) {
            CUDA_TRY(cudaEventCreateWithFlags(&c->ev_in[s], cudaEventDisableTiming));
            CUDA_TRY(cudaEventCreateWithFlags(&c->ev_reduced[s], cudaEventDisableTiming));
            CUDA_TRY(cudaEventCreateWithFlags(&c->ev_out[s], cudaEventDisableTiming));
        }
    }
    const bool exact = (dt == BINE_FLOAT || dt == BINE_DOUBLE) && c->order == BINE_ORDER_REFERENCE;
    std::shared_ptr<DevTrees> trees;
    if (exact) {
        rc = get_dev_trees(c, make_key(c, kAllreduce, count, 0), es, &trees);
        if (rc) return rc;
    }
    // Windows of at most host_window bytes over all ranks (default 32 MiB),
    // 256-byte aligned.
    const long long P = c->P;
    // At least ~8 windows once a call moves more than 16 MiB, so that the
    // copies in and out overlap even for calls below one full window.
    const long long total = P * count * es;
    const long long wbytes = std::min<long long>(c->host_window, std::max<long long>(2ll << 20, total / 8));
    long long W = (wbytes / (P * es)) / (256 / es) * (256 / es);
    W = std::max<long long>(W, 256 / es);
    if (W >= count) W = count;
    const long long pitch = (W * es + 255) / 256 * 256;
    const size_t slot = (size_t)P * pitch;
    if (c->stage_bytes < 4 * slot) {
        CUDA_TRY(cudaDeviceSynchronize());
        cudaFree(c->stage);
        c->stage = nullptr;
        c->stage_bytes = 0;
        CUDA_TRY(cudaMalloc(&c->stage, 4 * slot));
        c->stage_bytes = 4 * slot;
    }
    const DevTrees::Windows* win = nullptr;
    if (exact && W < count) {
        rc = window_tiles(c, *trees, W, count, &win);
        if (rc) return rc;
    }
    const long long nwin = (count + W - 1) / W;
    if (after)
        while ((long long)c->ev_window.size() < nwin) {
            cudaEvent_t e;
            CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            c->ev_window.push_back(e);
        }
    // After-window hook: windows whose output copy has ended, in order
    // (without waiting unless `wait`).
    long long issued = 0, reported = 0;
    auto report = [&](bool wait) -> int {
        while (after && reported < issued) {
            const cudaError_t q = wait ? cudaEventSynchronize(c->ev_window[reported])
                                       : cudaEventQuery(c->ev_window[reported]);
            if (q == cudaErrorNotReady) return BINE_SUCCESS;
            CUDA_TRY(q);
            const long long c0 = reported * W;
            if (after(user, c0, std::min(W, count - c0)) != 0)
                return fail(BINE_ERR_ABORTED, "the after-window hook abandoned the call");
            reported++;
        }
        return BINE_SUCCESS;
    };
    // An abandoned call still lets the copies in flight end before its
    // buffers go back to the caller.
    auto abandon = [&](int code) {
        cudaStreamSynchronize(c->h2d);
        cudaStreamSynchronize(c->stream);
        cudaStreamSynchronize(c->d2h);
        return code;
    };
    // The pipeline starts after the work already queued on the
    // communicator's stream and ends on it, so the call is stream-ordered.
    CUDA_TRY(cudaEventRecord(c->ev_start, c->stream));
    CUDA_TRY(cudaStreamWaitEvent(c->h2d, c->ev_start, 0));
    for (long long i = 0; i < nwin; i++) {
        const int s = (int)(i & 1);
        const long long c0 = i * W, w = std::min(W, count - c0);
        char* in_s = c->stage + (size_t)(2 * s) * slot;
        char* out_s = c->stage + (size_t)(2 * s + 1) * slot;
        if ((rc = report(false)) != BINE_SUCCESS) return abandon(rc);
        if (before && before(user, c0, w) != 0)
            return abandon(fail(BINE_ERR_ABORTED, "the before-window hook abandoned the call"));
        if (i >= 2) CUDA_TRY(cudaStreamWaitEvent(c->h2d, c->ev_reduced[s], 0));  // input slot consumed
        CUDA_TRY(cudaMemcpy2DAsync(in_s, pitch, (const char*)sendbuf + c0 * es, ist, w * es, P,
                                   cudaMemcpyHostToDevice, c->h2d));
        CUDA_TRY(cudaEventRecord(c->ev_in[s], c->h2d));
        CUDA_TRY(cudaStreamWaitEvent(c->stream, c->ev_in[s], 0));
        if (i >= 2) CUDA_TRY(cudaStreamWaitEvent(c->stream, c->ev_out[s], 0));  // output slot copied out
        if (exact) {
            // Element indices stay those of the full call: offset the bases.
            const char* ib = in_s - c0 * es;
            char* ob = out_s - c0 * es;
            rc = dt == BINE_FLOAT ? launch_tree_window<float>(c, *trees, win, i, ib, pitch, ob, pitch)
                                  : launch_tree_window<double>(c, *trees, win, i, ib, pitch, ob, pitch);
        } else {
            rc = launch_sum_dt(c, dt, dev::kSumAllreduce, in_s, pitch, out_s, pitch, w, 0, 0);
        }
        if (rc) return rc;
        CUDA_TRY(cudaEventRecord(c->ev_reduced[s], c->stream));
        CUDA_TRY(cudaStreamWaitEvent(c->d2h, c->ev_reduced[s], 0));
        CUDA_TRY(cudaMemcpy2DAsync((char*)recvbuf + c0 * es, ost, out_s, pitch, w * es, P, cudaMemcpyDeviceToHost,
                                   c->d2h));
        CUDA_TRY(cudaEventRecord(c->ev_out[s], c->d2h));
        if (after) CUDA_TRY(cudaEventRecord(c->ev_window[i], c->d2h));
        issued = i + 1;
    }
    CUDA_TRY(cudaStreamWaitEvent(c->stream, c->ev_out[(nwin - 1) & 1], 0));
    if ((rc = report(true)) != BINE_SUCCESS) return abandon(rc);
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return BINE_SUCCESS;
}

int plan_for_query(bine_comm_t c, int coll, long count, int root, std::shared_ptr<Schedule>* s) {
    if (!c) return fail(BINE_ERR_ARG, "null communicator");
    if (coll < 0 || coll >= kNumColls) return fail(BINE_ERR_ARG, "invalid collective");
    if (count <= 0) return fail(BINE_ERR_ARG, "count must be positive");
    return get_schedule(c, make_key(c, coll, count, root), s);
}

}  // namespace

// ------------------------------------------------------- allocation-free call
// Callers that cannot allocate device memory (code running under a memory
// manager that owns every allocation, allocators that forbid cudaMalloc
// during steady state, or code that must not touch the CUDA heap at all)
// can still run the step engine through bine_allreduce_noalloc(): its
// schedule tables, grid-barrier words and workspace rows live in this one
// fixed array, which the CUDA runtime reserves when the library's module is
// loaded on a device and keeps until the process exits.
constexpr size_t kNoAllocScratchBytes = 64ull << 20;  // 64 MiB per device
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

// Device address of g_noalloc_scratch per device, looked up once per device
// with that device current (host code may not use the symbol itself: on the
// host it is only a stand-in for the device array).
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kMaxDevices] = {nullptr};

int noalloc_scratch(int dev, char** out) {
    if (dev < 0 || dev >= kMaxDevices) return fail(BINE_ERR_ARG, "device index out of range");
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return fail(BINE_ERR_CUDA, std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e));
        g_noalloc_ptr[dev] = p;
    }
    *out = (char*)g_noalloc_ptr[dev];
    return BINE_SUCCESS;
}

size_t round256(size_t x) { return (x + 255) / 256 * 256; }

template <typename T>
int noalloc_run(bine_comm_t c, const Schedule& s, const char* send, long long ist, char* recv, long long ost,
                int dev) {
    // Scratch layout: [barrier u32 x2 | status i32] [level_begin] [moves] [chunks] [workspace rows].
    std::vector<dev::StepMove> moves;
    std::vector<dev::StepChunk> chunks;
    std::vector<int> lb;
    int max_chunks = 0;
    const int64_t chunk_elems = std::max<int64_t>(16, (32 * 1024) / (int64_t)sizeof(T));
    for (const auto& lvl : s.levels) {
        lb.push_back((int)chunks.size());
        for (const Move& m : lvl) {
            dev::StepMove dm{m.dst.off, m.a.off, m.b.off, m.dst.rank, m.a.rank, m.b.rank, m.dst.buf, m.a.buf, m.b.buf,
                             m.add};
            const int mi = (int)moves.size();
            moves.push_back(dm);
            for (int64_t st = 0; st < m.n; st += chunk_elems)
                chunks.push_back(dev::StepChunk{mi, 0, st, std::min(chunk_elems, m.n - st)});
        }
        max_chunks = std::max(max_chunks, (int)chunks.size() - lb.back());
    }
    lb.push_back((int)chunks.size());
    const size_t tmp_stride = round256((size_t)s.tmp_elems * sizeof(T));
    const size_t off_lb = 256, off_mv = off_lb + round256(lb.size() * sizeof(int));
    const size_t off_ch = off_mv + round256(moves.size() * sizeof(dev::StepMove));
    const size_t off_ws = off_ch + round256(chunks.size() * sizeof(dev::StepChunk));
    // Input and output arrays that share bytes: the input rows are staged
    // after the workspace (the step schedule would otherwise read rows the
    // same step overwrites).
    const bool in_place = arrays_overlap(send, ist, (size_t)s.send_elems * sizeof(T), recv, ost,
                                         (size_t)s.recv_elems * sizeof(T), c->P);
    const size_t in_pitch = round256((size_t)s.send_elems * sizeof(T));
    const size_t off_in = off_ws + tmp_stride * (size_t)c->P;
    const size_t need = off_in + (in_place ? in_pitch * (size_t)c->P : 0);
    if (need > kNoAllocScratchBytes)
        return fail(BINE_ERR_NOMEM, "bine_allreduce_noalloc: this call needs " + std::to_string(need) +
                                        " bytes of scratch, more than the fixed " +
                                        std::to_string(kNoAllocScratchBytes) + " bytes; use bine_allreduce");
    char* base = nullptr;
    int rc = noalloc_scratch(dev, &base);
    if (rc) return rc;
    cudaStream_t st = c->stream;
    // The barrier words and the status word must start at zero on every call.
    CUDA_TRY(cudaMemsetAsync(base, 0, 256, st));
    CUDA_TRY(cudaMemcpyAsync(base + off_lb, lb.data(), lb.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    if (!moves.empty())
        CUDA_TRY(cudaMemcpyAsync(base + off_mv, moves.data(), moves.size() * sizeof(dev::StepMove),
                                 cudaMemcpyHostToDevice, st));
    if (!chunks.empty())
        CUDA_TRY(cudaMemcpyAsync(base + off_ch, chunks.data(), chunks.size() * sizeof(dev::StepChunk),
                                 cudaMemcpyHostToDevice, st));
    if (in_place) {
        CUDA_TRY(cudaMemcpy2DAsync(base + off_in, in_pitch, send, ist, (size_t)s.send_elems * sizeof(T), c->P,
                                   cudaMemcpyDeviceToDevice, st));
        send = base + off_in;
        ist = (long long)in_pitch;
    }
    dev::StepBufs B;
    B.base[kBufSend] = const_cast<char*>(send);
    B.base[kBufRecv] = recv;
    B.base[kBufTmp] = base + off_ws;
    B.stride[kBufSend] = ist;
    B.stride[kBufRecv] = ost;
    B.stride[kBufTmp] = (long long)tmp_stride;
    int sms = 0, per_sm = 0;
    CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dev::k_steps<T>, dev::kThreads, 0));
    int blocks = std::max(1, std::min(per_sm * sms, std::max(1, max_chunks)));
    const dev::StepMove* mv = (const dev::StepMove*)(base + off_mv);
    const dev::StepChunk* ch = (const dev::StepChunk*)(base + off_ch);
    const int* lbp = (const int*)(base + off_lb);
    int nl = (int)s.levels.size();
    unsigned* bar = (unsigned*)base;
    int* status = (int*)(base + 16);
    unsigned long long to = c->step_timeout_ns;
    unsigned expected = (unsigned)blocks + c->barrier_extra;
    void* args[] = {&B, &mv, &ch, &lbp, &nl, &bar, &status, &to, &expected};
    CUDA_TRY(cudaLaunchCooperativeKernel((void*)dev::k_steps<T>, dim3(blocks), dim3(dev::kThreads), args, 0, st));
    // The host staging of the tables and the status check need the call to
    // finish before returning.
    CUDA_TRY(cudaStreamSynchronize(st));
    int stv = 0;
    CUDA_TRY(cudaMemcpy(&stv, status, sizeof(int), cudaMemcpyDeviceToHost));
    if (stv != dev::kStepOk) return fail(BINE_ERR_TIMEOUT, "a grid barrier of the step engine timed out");
    return BINE_SUCCESS;
}

}  // namespace

// ---------------------------------------------------------------- batches
struct bine_batch_s {
    dev::BatchItem* items = nullptr;
    int nitems = 0;
    long long total_tiles = 0;
    unsigned grid = 1;
    ~bine_batch_s() { cudaFree(items); }
};

namespace {

const bine_batch_tuning_t kDefaultTuning = {{8, 32, 128, 1 << 30}, {256, 128, 64, 32}, 1, 1};

int batch_layout(const bine_batch_item_t* items, int n, const bine_batch_tuning_t& tu,
                 std::vector<dev::BatchItem>* out, long long* total_tiles) {
    out->clear();
    std::vector<std::pair<double, int>> order;
    for (int i = 0; i < n; i++) {
        const bine_batch_item_t& x = items[i];
        if (x.coll != BINE_COLL_ALLREDUCE && x.coll != BINE_COLL_REDUCE_SCATTER && x.coll != BINE_COLL_ALLGATHER)
            return fail(BINE_ERR_ARG, "batch item " + std::to_string(i) + ": only allreduce, reduce_scatter and allgather");
        if (x.datatype != BINE_INT32 && x.datatype != BINE_FLOAT)
            return fail(BINE_ERR_ARG, "batch item " + std::to_string(i) + ": datatype must be BINE_INT32 or BINE_FLOAT");
        if (x.nranks < 1 || x.count < 1 || !x.sendbuf || !x.recvbuf)
            return fail(BINE_ERR_ARG, "batch item " + std::to_string(i) + ": bad nranks, count or buffer");
        if ((x.count * 4) % 16)
            return fail(BINE_ERR_ARG, "batch item " + std::to_string(i) + ": count must fill whole 16-byte vectors");
        const long long P = x.nranks, row = x.count * 4;
        long long se = row, re = row;
        if (x.coll == BINE_COLL_REDUCE_SCATTER) se = row * P;
        if (x.coll == BINE_COLL_ALLGATHER) re = row * P;
        dev::BatchItem b;
        b.in = (const char*)x.sendbuf;
        b.out = (char*)x.recvbuf;
        b.in_stride = x.send_stride ? (long long)x.send_stride : se;
        b.out_stride = x.recv_stride ? (long long)x.recv_stride : re;
        if (b.in_stride < se || b.out_stride < re || (b.in_stride | b.out_stride) % 16 || !aligned16(b.in) || !aligned16(b.out))
            return fail(BINE_ERR_ARG, "batch item " + std::to_string(i) + ": rows must be 16-byte aligned and fit their stride");
        b.P = x.nranks;
        b.is_float = x.datatype == BINE_FLOAT;
        b.blk = 0;
        double cost;
        if (x.coll == BINE_COLL_ALLGATHER) {
            b.op = dev::kBatchAllgather;
            b.ncol = row / 16;
            b.tc = dev::kThreads;
            b.ntiles = (P * b.ncol + dev::kThreads - 1) / dev::kThreads;
            cost = (double)P * b.ncol * (P + 1);
        } else {
            b.op = x.coll == BINE_COLL_ALLREDUCE ? dev::kBatchAllreduce : dev::kBatchReduceScatter;
            b.ncol = se / 16;
            b.blk = x.coll == BINE_COLL_REDUCE_SCATTER ? row / 16 : 0;
            int tc = tu.tile_cols[3];
            for (int k = 0; k < 4; k++)
                if (x.nranks <= tu.rank_bound[k]) {
                    tc = tu.tile_cols[k];
                    break;
                }
            if (tc != 32 && tc != 64 && tc != 128 && tc != 256) return fail(BINE_ERR_ARG, "tile_cols must be 32, 64, 128 or 256");
            b.tc = tc;
            b.ntiles = (b.ncol + tc - 1) / tc;
            cost = (double)P * b.ncol * (x.coll == BINE_COLL_ALLREDUCE ? 2 : 1);
        }
        out->push_back(b);
        order.push_back({cost, i});
    }
    if (tu.order == 1) {
        std::stable_sort(order.begin(), order.end(), [](const std::pair<double, int>& a, const std::pair<double, int>& b) {
            return a.first > b.first;
        });
        std::vector<dev::BatchItem> sorted;
        for (auto& o : order) sorted.push_back((*out)[o.second]);
        *out = sorted;
    }
    long long t = 0;
    for (auto& b : *out) {
        b.tile_begin = t;
        t += b.ntiles;
    }
    *total_tiles = t;
    return BINE_SUCCESS;
}

unsigned batch_grid(long long total_tiles, int grid_mult) {
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dev::k_batch, dev::kThreads, 0) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    long long g = (long long)per_sm * sms * std::max(1, grid_mult);
    return (unsigned)std::max(1LL, std::min(g, total_tiles));
}

}  // namespace

extern "C" {

int bine_batch_create(const bine_batch_item_t* items, int nitems, const bine_batch_tuning_t* tuning,
                      bine_batch_t* batch) {
    if (!batch || (!items && nitems > 0) || nitems < 0) return fail(BINE_ERR_ARG, "bad batch arguments");
    *batch = nullptr;
    const bine_batch_tuning_t& tu = tuning ? *tuning : kDefaultTuning;
    std::vector<dev::BatchItem> v;
    long long tiles = 0;
    int rc = batch_layout(items, nitems, tu, &v, &tiles);
    if (rc) return rc;
    auto b = std::unique_ptr<bine_batch_s>(new bine_batch_s());
    b->nitems = (int)v.size();
    b->total_tiles = tiles;
    b->grid = batch_grid(tiles, tu.grid_mult);
    if (!v.empty()) {
        CUDA_TRY(cudaMalloc(&b->items, v.size() * sizeof(dev::BatchItem)));
        CUDA_TRY(cudaMemcpy(b->items, v.data(), v.size() * sizeof(dev::BatchItem), cudaMemcpyHostToDevice));
    }
    *batch = b.release();
    return BINE_SUCCESS;
}

int bine_batch_launch(bine_batch_t batch, void* stream) {
    if (!batch) return fail(BINE_ERR_ARG, "null batch");
    if (batch->total_tiles == 0) return BINE_SUCCESS;
    dev::k_batch<<<batch->grid, dev::kThreads, 0, (cudaStream_t)stream>>>(batch->items, batch->nitems, batch->total_tiles);
    CUDA_TRY(cudaGetLastError());
    return BINE_SUCCESS;
}

int bine_batch_destroy(bine_batch_t batch) {
    delete batch;
    return BINE_SUCCESS;
}

int bine_batch_autotune(const bine_batch_item_t* items, int nitems, void* stream, int reps, bine_batch_tuning_t* best,
                        float* best_ms) {
    if (!best || reps < 1) return fail(BINE_ERR_ARG, "bad autotune arguments");
    // Candidate tile policies: (rank bound, tile columns) pairs.
    const bine_batch_tuning_t policies[] = {
        {{8, 32, 128, 1 << 30}, {256, 128, 64, 32}, 1, 0},
        {{4, 16, 64, 1 << 30}, {256, 128, 64, 32}, 1, 0},
        {{16, 64, 256, 1 << 30}, {256, 128, 64, 32}, 1, 0},
        {{32, 128, 512, 1 << 30}, {128, 64, 64, 32}, 1, 0},
        {{1 << 30, 1 << 30, 1 << 30, 1 << 30}, {32, 32, 32, 32}, 1, 0},
        {{1 << 30, 1 << 30, 1 << 30, 1 << 30}, {64, 64, 64, 64}, 1, 0},
    };
    cudaStream_t s = (cudaStream_t)stream;
    cudaEvent_t e0, e1;
    CUDA_TRY(cudaEventCreate(&e0));
    CUDA_TRY(cudaEventCreate(&e1));
    float best_t = 1e30f;
    int rc = BINE_SUCCESS;
    for (const auto& pol : policies) {
        for (int gm : {1, 2, 4, 8, 16}) {  // 8 and 16: more blocks than fit, back-filled by the hardware
            for (int order : {0, 1}) {
                bine_batch_tuning_t tu = pol;
                tu.grid_mult = gm;
                tu.order = order;
                bine_batch_t b = nullptr;
                rc = bine_batch_create(items, nitems, &tu, &b);
                if (rc) goto done;
                bine_batch_launch(b, stream);  // warm-up
                cudaEventRecord(e0, s);
                for (int r = 0; r < reps; r++) bine_batch_launch(b, stream);
                cudaEventRecord(e1, s);
                if (cudaEventSynchronize(e1) != cudaSuccess) {
                    bine_batch_destroy(b);
                    rc = fail(BINE_ERR_CUDA, "autotune launch failed");
                    goto done;
                }
                float ms = 0;
                cudaEventElapsedTime(&ms, e0, e1);
                ms /= reps;
                if (ms < best_t) {
                    best_t = ms;
                    *best = tu;
                }
                bine_batch_destroy(b);
            }
        }
    }
done:
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (best_ms) *best_ms = best_t;
    return rc;
}

const char* bine_last_error_string(void) { return g_err.c_str(); }

int bine_allreduce_noalloc(const void* sendbuf, void* recvbuf, int count, bine_datatype_t datatype, bine_op_t op,
                           bine_comm_t comm) {
    if (op != BINE_SUM) return fail(BINE_ERR_ARG, "only BINE_SUM is supported");
    if (!comm) return fail(BINE_ERR_ARG, "null communicator");
    const int es = dtype_size(datatype);
    if (es < 0) return fail(BINE_ERR_ARG, "invalid datatype");
    if (count < 0) return fail(BINE_ERR_ARG, "negative count");
    if (count == 0) return BINE_SUCCESS;
    if (!sendbuf || !recvbuf) return fail(BINE_ERR_ARG, "null buffer");
    const long long ist = comm->send_stride ? (long long)comm->send_stride : (long long)count * es;
    const long long ost = comm->recv_stride ? (long long)comm->recv_stride : (long long)count * es;
    if (ist < (long long)count * es || ost < (long long)count * es)
        return fail(BINE_ERR_ARG, "layout stride smaller than a rank row");
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    const PlanKey k = make_key(comm, kAllreduce, count, 0);
    std::shared_ptr<Schedule> s;
    int rc = get_schedule(comm, k, &s);
    if (rc) return rc;
    std::string verr;
    if (!comm->planner->verify(k, *s, &verr)) return fail(BINE_ERR_UNSUPPORTED, verr);
    const int64_t rows[3] = {s->send_elems, s->recv_elems, s->tmp_elems};
    for (const auto& lvl : s->levels)
        for (const Move& m : lvl)
            for (const Region* r : {&m.dst, &m.a, &m.b})
                if (r->rank < 0 || r->rank >= comm->P || r->buf > kBufTmp || r->off < 0 || m.n < 0 ||
                    r->off + m.n > rows[r->buf])
                    return fail(BINE_ERR_INTERNAL, "planner produced a region outside its buffer row");
    const char* in = (const char*)sendbuf;
    char* out = (char*)recvbuf;
    switch (datatype) {
    case BINE_INT32: return noalloc_run<int32_t>(comm, *s, in, ist, out, ost, dev);
    case BINE_INT64: return noalloc_run<int64_t>(comm, *s, in, ist, out, ost, dev);
    case BINE_FLOAT: return noalloc_run<float>(comm, *s, in, ist, out, ost, dev);
    case BINE_DOUBLE: return noalloc_run<double>(comm, *s, in, ist, out, ost, dev);
    case BINE_CHAR: return noalloc_run<int8_t>(comm, *s, in, ist, out, ost, dev);
    }
    return fail(BINE_ERR_ARG, "invalid datatype");
}

int bine_comm_create(int nranks, int ndims, const int* dims, bine_comm_t* comm) {
    if (!comm) return fail(BINE_ERR_ARG, "null output pointer");
    *comm = nullptr;
    if (nranks < 1 || nranks > (1 << 20)) return fail(BINE_ERR_ARG, "nranks must be in [1, 2^20]");
    if (ndims < 0 || ndims > kMaxDims) return fail(BINE_ERR_ARG, "ndims must be in [0, 3] (lib/libbine.cc:131)");
    long long prod = 1;
    for (int i = 0; i < ndims; i++) {
        if (!dims || dims[i] < 2) return fail(BINE_ERR_ARG, "every torus dimension must be at least 2");
        prod *= dims[i];
    }
    if (ndims > 0 && prod != nranks) return fail(BINE_ERR_ARG, "dims do not multiply to nranks");
    Torus t;
    int d1[1] = {nranks};
    t.init(ndims > 0 ? ndims : 1, ndims > 0 ? dims : d1);
    if (t.num_steps > kMaxSteps) return fail(BINE_ERR_ARG, "too many steps for the distance tables");
    bine_comm_t c = new bine_comm_s();
    c->P = nranks;
    c->planner.reset(new Planner(nranks, ndims, dims));
    for (int i = 0; i < kNumColls; i++) c->cfg[i] = kDefaults[i];
    *comm = c;
    return BINE_SUCCESS;
}

int bine_comm_destroy(bine_comm_t comm) {
    if (!comm) return BINE_SUCCESS;
    if (comm->device >= 0) cudaStreamSynchronize(comm->stream);
    delete comm;
    return BINE_SUCCESS;
}

int bine_comm_set_stream(bine_comm_t comm, void* stream) {
    if (!comm) return fail(BINE_ERR_ARG, "null communicator");
    comm->stream = (cudaStream_t)stream;
    return BINE_SUCCESS;
}

int bine_comm_set_layout(bine_comm_t comm, size_t send_stride, size_t recv_stride) {
    if (!comm) return fail(BINE_ERR_ARG, "null communicator");
    comm->send_stride = send_stride;
    comm->recv_stride = recv_stride;
    return BINE_SUCCESS;
}

int bine_comm_set_ports(bine_comm_t comm, int ports) {
    if (!comm) return fail(BINE_ERR_ARG, "null communicator");
    if (ports < 1 || ports > kMaxPorts) return fail(BINE_ERR_ARG, "ports must be in [1, 6] (lib/libbine.cc:98)");
    comm->ports = ports;
    return BINE_SUCCESS;
}

int bine_comm_set_algo(bine_comm_t comm, bine_coll_t coll, int variant, int family, int distance) {
    if (!comm) return fail(BINE_ERR_ARG, "null communicator");
    if ((int)coll < 0 || (int)coll >= kNumColls) return fail(BINE_ERR_ARG, "invalid collective");
    if (family != BINE_FAMILY_BINE && family != BINE_FAMILY_RECDOUB && family != BINE_FAMILY_BRUCK &&
        family != BINE_FAMILY_RING)
        return fail(BINE_ERR_ARG, "invalid family");
    if (family == BINE_FAMILY_BRUCK && coll != BINE_COLL_ALLTOALL)
        return fail(BINE_ERR_ARG, "the BRUCK family is an alltoall algorithm");
    if (distance != BINE_DISTANCE_DEFAULT && distance != kIncreasing && distance != kDecreasing)
        return fail(BINE_ERR_ARG, "invalid distance");
    static const int valid[kNumColls][4] = {{kArL, kArB, kArBCont, kArBCoalesce},
                                             {kRsContPermute, -1, -1, -1},
                                             {kAgContPermute, kAgContSend, kAgBlocks, -1},
                                             {kBcTree, kBcScatterAllgather, -1, -1},
                                             {kRdTree, kRdRedscatGather, -1, -1},
                                             {kA2aLog, -1, -1, -1},
                                             {kScTree, -1, -1, -1},
                                             {kGaTree, -1, -1, -1}};
    bool ok = false;
    for (int v : valid[coll]) ok |= v == variant;
    if (!ok) return fail(BINE_ERR_ARG, "invalid variant for this collective");
    CollCfg cf;
    cf.variant = variant;
    cf.family = family;
    cf.distance = distance == BINE_DISTANCE_DEFAULT ? kDefaults[coll].distance : distance;
    // Scatter-allgather bcast runs with INCREASING distance (lib/libbine.cc:1267).
    if (coll == BINE_COLL_BCAST && variant == kBcScatterAllgather && distance == BINE_DISTANCE_DEFAULT)
        cf.distance = kIncreasing;
    comm->cfg[coll] = cf;
    return BINE_SUCCESS;
}

int bine_comm_set_fusion(bine_comm_t comm, int levels) {
    if (!comm) return fail(BINE_ERR_ARG, "null communicator");
    if (levels < 0 || levels > 64) return fail(BINE_ERR_ARG, "levels per pass must be in [0, 64]");
    comm->fusion = levels;
    return BINE_SUCCESS;
}

int bine_comm_set_segment(bine_comm_t comm, long long segment_bytes) {
    if (!comm) return fail(BINE_ERR_ARG, "null communicator");
    if (segment_bytes < 0) return fail(BINE_ERR_ARG, "segment size must be >= 0");
    comm->segment_bytes = segment_bytes;
    return BINE_SUCCESS;
}

int bine_comm_set_engine(bine_comm_t comm, int engine) {
    if (!comm) return fail(BINE_ERR_ARG, "null communicator");
    if (engine != BINE_ENGINE_FUSED && engine != BINE_ENGINE_STEPS && engine != BINE_ENGINE_PIPELINED)
        return fail(BINE_ERR_ARG, "invalid engine");
    comm->engine = engine;
    return BINE_SUCCESS;
}

int bine_comm_set_float_order(bine_comm_t comm, int order) {
    if (!comm) return fail(BINE_ERR_ARG, "null communicator");
    if (order != BINE_ORDER_REFERENCE && order != BINE_ORDER_FAST) return fail(BINE_ERR_ARG, "invalid order");
    comm->order = order;
    return BINE_SUCCESS;
}

int bine_allreduce(const void* sendbuf, void* recvbuf, int count, bine_datatype_t datatype, bine_op_t op,
                   bine_comm_t comm) {
    if (op != BINE_SUM) return fail(BINE_ERR_ARG, "only BINE_SUM is supported");
    return run_collective(comm, kAllreduce, sendbuf, recvbuf, count, datatype, 0);
}

int bine_allreduce_host(const void* sendbuf, void* recvbuf, int count, bine_datatype_t datatype, bine_op_t op,
                        bine_comm_t comm) {
    if (!comm) return fail(BINE_ERR_ARG, "null communicator");
    if (op != BINE_SUM) return fail(BINE_ERR_ARG, "only BINE_SUM is supported");
    return allreduce_host(comm, sendbuf, recvbuf, count, datatype);
}

int bine_allreduce_host_hooked(const void* sendbuf, void* recvbuf, int count, bine_datatype_t datatype,
                               bine_op_t op, bine_comm_t comm, bine_window_hook_t before_window,
                               bine_window_hook_t after_window, void* user) {
    if (!comm) return fail(BINE_ERR_ARG, "null communicator");
    if (op != BINE_SUM) return fail(BINE_ERR_ARG, "only BINE_SUM is supported");
    return allreduce_host(comm, sendbuf, recvbuf, count, datatype, before_window, after_window, user);
}

int bine_reduce_scatter(const void* sendbuf, void* recvbuf, const int* recvcounts, bine_datatype_t datatype,
                        bine_op_t op, bine_comm_t comm) {
    if (op != BINE_SUM) return fail(BINE_ERR_ARG, "only BINE_SUM is supported");
    if (!comm || !recvcounts) return fail(BINE_ERR_ARG, "null argument");
    for (int i = 1; i < comm->P; i++)
        if (recvcounts[i] != recvcounts[0])
            return fail(BINE_ERR_UNSUPPORTED, "recvcounts must be equal (reduce_scatter_block semantics, lib/libbine.cc:1065)");
    return run_collective(comm, kReduceScatter, sendbuf, recvbuf, recvcounts[0], datatype, 0);
}

int bine_allgather(const void* sendbuf, int sendcount, bine_datatype_t sendtype, void* recvbuf, int recvcount,
                   bine_datatype_t recvtype, bine_comm_t comm) {
    if (sendcount != recvcount || sendtype != recvtype)
        return fail(BINE_ERR_UNSUPPORTED, "sendcount/type must equal recvcount/type (lib/libbine.cc:1170-1171)");
    return run_collective(comm, kAllgather, sendbuf, recvbuf, sendcount, sendtype, 0);
}

int bine_bcast(void* buffer, int count, bine_datatype_t datatype, int root, bine_comm_t comm) {
    return run_collective(comm, kBcast, nullptr, buffer, count, datatype, root);
}

int bine_alltoall(const void* sendbuf, int sendcount, bine_datatype_t sendtype, void* recvbuf, int recvcount,
                  bine_datatype_t recvtype, bine_comm_t comm) {
    if (sendcount != recvcount || sendtype != recvtype)
        return fail(BINE_ERR_UNSUPPORTED, "sendcount/type must equal recvcount/type");
    return run_collective(comm, kAlltoall, sendbuf, recvbuf, sendcount, sendtype, 0);
}

int bine_scatter(const void* sendbuf, int sendcount, bine_datatype_t sendtype, void* recvbuf, int recvcount,
                 bine_datatype_t recvtype, int root, bine_comm_t comm) {
    if (sendcount != recvcount || sendtype != recvtype)
        return fail(BINE_ERR_UNSUPPORTED, "sendcount/type must equal recvcount/type (lib/libbine_coll_scatter.cc:197-198)");
    return run_collective(comm, kScatter, sendbuf, recvbuf, recvcount, recvtype, root);
}

int bine_gather(const void* sendbuf, int sendcount, bine_datatype_t sendtype, void* recvbuf, int recvcount,
                bine_datatype_t recvtype, int root, bine_comm_t comm) {
    if (sendcount != recvcount || sendtype != recvtype)
        return fail(BINE_ERR_UNSUPPORTED, "sendcount/type must equal recvcount/type (lib/libbine_coll_gather.cc:210)");
    return run_collective(comm, kGather, sendbuf, recvbuf, sendcount, sendtype, root);
}

int bine_reduce(const void* sendbuf, void* recvbuf, int count, bine_datatype_t datatype, bine_op_t op, int root,
                bine_comm_t comm) {
    if (op != BINE_SUM) return fail(BINE_ERR_ARG, "only BINE_SUM is supported");
    return run_collective(comm, kReduce, sendbuf, recvbuf, count, datatype, root);
}

int bine_comm_set_step_timeout(bine_comm_t comm, unsigned timeout_ms) {
    if (!comm) return fail(BINE_ERR_ARG, "null communicator");
    if (timeout_ms == 0) return fail(BINE_ERR_ARG, "timeout must be positive");
    comm->step_timeout_ns = (unsigned long long)timeout_ms * 1000000ull;
    return BINE_SUCCESS;
}

int bine_debug_set_barrier_extra(bine_comm_t comm, unsigned extra) {
    if (!comm) return fail(BINE_ERR_ARG, "null communicator");
    comm->barrier_extra = extra;
    return BINE_SUCCESS;
}

int bine_plan_tree_cover(bine_comm_t comm, bine_coll_t coll, long count, bine_datatype_t datatype, int root,
                         int64_t* runs, size_t cap, size_t* n) {
    if (!comm || !n) return fail(BINE_ERR_ARG, "null argument");
    if (datatype != BINE_FLOAT && datatype != BINE_DOUBLE) return fail(BINE_ERR_ARG, "not a floating-point type");
    if (!is_reduction(coll)) return fail(BINE_ERR_ARG, "not a reduction");
    if (count <= 0) return fail(BINE_ERR_ARG, "count must be positive");
    if (root < 0 || root >= comm->P) return fail(BINE_ERR_ARG, "root out of range");
    std::shared_ptr<DevTrees> d;
    const int es = dtype_size(datatype);
    int rc = get_dev_trees(comm, make_key(comm, coll, count, root), es, &d, true);
    if (rc) return rc;
    const int64_t L = 16 / es;
    std::vector<int64_t> v;  // (first element, elements, kind) triples
    auto emit = [&](int64_t a, int64_t len, int64_t kind) {
        v.push_back(a);
        v.push_back(len);
        v.push_back(kind);
    };
    if (d->flat) {
        // Row tiles: every lane vector that some slot of the tile's shape owns,
        // as the kernel finds it.
        for (const dev::TreeTile& t : d->h_stiles) {
            const int ns = t.pad & 0xff;
            for (int64_t e = t.start; e < t.start + t.n; e += L)
                for (int q = 0; q < ns; q++)
                    if (e >= d->h_fbody[2 * (t.seg + q)] && e < d->h_fbody[2 * (t.seg + q) + 1]) emit(e, L, 1);
        }
        for (const dev::FlatEdge& ed : d->h_fedges) emit(ed.e, L, 2);
    } else {
        const std::vector<dev::TreeTile>& vt = d->split_k > 1 ? d->h_stiles : d->h_tiles;
        for (const dev::TreeTile& t : vt) emit(d->h_seg_off[t.seg] + t.start, t.n, 1);
    }
    for (const std::vector<dev::TreeTile>* lst : {&d->h_htiles, &d->h_rtiles})
        for (const dev::TreeTile& t : *lst) emit(d->h_seg_off[t.seg] + t.start, t.n, 3);
    *n = v.size() / 3;
    if (runs && cap >= *n) std::copy(v.begin(), v.end(), runs);
    return BINE_SUCCESS;
}

int bine_plan_tree_form(bine_comm_t comm, bine_coll_t coll, long count, bine_datatype_t datatype, int root,
                        int64_t out[6]) {
    if (!comm || !out) return fail(BINE_ERR_ARG, "null argument");
    if (datatype != BINE_FLOAT && datatype != BINE_DOUBLE) return fail(BINE_ERR_ARG, "not a floating-point type");
    if (!is_reduction(coll)) return fail(BINE_ERR_ARG, "not a reduction");
    if (count <= 0) return fail(BINE_ERR_ARG, "count must be positive");
    if (root < 0 || root >= comm->P) return fail(BINE_ERR_ARG, "root out of range");
    std::shared_ptr<DevTrees> d;
    int rc = get_dev_trees(comm, make_key(comm, coll, count, root), dtype_size(datatype), &d, true);
    if (rc) return rc;
    out[0] = d->flat ? 3 : (d->split_k > 1 && d->nstiles > 0 ? 2 : (d->ntiles > 0 ? 1 : 0));
    out[1] = d->split_k;
    out[2] = d->flat ? d->fnshape : 0;
    out[3] = d->split_k > 1 ? d->nstiles : d->ntiles;
    out[4] = d->flat ? d->nfedges : 0;
    out[5] = (int64_t)d->nhtiles + d->nrtiles;
    return BINE_SUCCESS;
}

int bine_debug_tree_form(bine_comm_t comm, bine_coll_t coll, long count, bine_datatype_t datatype, int root,
                         int* form, int* lanes) {
    if (!form || !lanes) return fail(BINE_ERR_ARG, "null argument");
    int64_t o[6];
    int rc = bine_plan_tree_form(comm, coll, count, datatype, root, o);
    if (rc) return rc;
    *form = (int)o[0];
    *lanes = (int)o[1];
    return BINE_SUCCESS;
}

int bine_comm_set_host_window(bine_comm_t comm, long long window_bytes) {
    if (!comm) return fail(BINE_ERR_ARG, "null communicator");
    if (window_bytes < 4096) return fail(BINE_ERR_ARG, "host window below 4 KiB");
    comm->host_window = window_bytes;
    return BINE_SUCCESS;
}

int bine_comm_set_tree_split(bine_comm_t comm, int lanes) {
    if (!comm) return fail(BINE_ERR_ARG, "null communicator");
    if (lanes != 0 && lanes != 1 && lanes != 2 && lanes != 4 && lanes != 8)
        return fail(BINE_ERR_ARG, "tree split must be 0, 1, 2, 4 or 8");
    comm->tree_split = lanes;
    return BINE_SUCCESS;
}

int bine_comm_synchronize(bine_comm_t comm) {
    if (!comm) return fail(BINE_ERR_ARG, "null communicator");
    if (comm->device < 0) return BINE_SUCCESS;
    CUDA_TRY(cudaStreamSynchronize(comm->stream));
    int st = 0;
    CUDA_TRY(cudaMemcpy(&st, comm->status, sizeof(int), cudaMemcpyDeviceToHost));
    if (st != dev::kStepOk) {
        CUDA_TRY(cudaMemset(comm->status, 0, sizeof(int)));
        return fail(BINE_ERR_TIMEOUT, "a bounded wait of the step engine timed out");
    }
    return BINE_SUCCESS;
}

int bine_plan_verify(bine_comm_t comm, bine_coll_t coll, long count, int root) {
    std::shared_ptr<Schedule> s;
    int rc = plan_for_query(comm, coll, count, root, &s);
    if (rc) return rc;
    // The communicator's proof cache, as the engine itself consults before
    // running a schedule.
    return verify_cached(comm, make_key(comm, coll, count, root), *s);
}

int bine_plan_stats(bine_comm_t comm, bine_coll_t coll, long count, int root, int64_t out[5]) {
    std::shared_ptr<Schedule> s;
    int rc = plan_for_query(comm, coll, count, root, &s);
    if (rc) return rc;
    int64_t moves = 0, traffic = 0;
    for (const auto& l : s->levels)
        for (const Move& m : l) {
            moves++;
            traffic += m.n * (m.add ? 3 : 2);
        }
    out[0] = (int64_t)s->levels.size();
    out[1] = moves;
    out[2] = (int64_t)s->messages.size();
    out[3] = s->tmp_elems;
    out[4] = traffic;
    return BINE_SUCCESS;
}

int bine_plan_moves(bine_comm_t comm, bine_coll_t coll, long count, int root, int64_t* moves, int64_t* sizes,
                    size_t cap, size_t* n_moves) {
    std::shared_ptr<Schedule> s;
    int rc = plan_for_query(comm, coll, count, root, &s);
    if (rc) return rc;
    size_t i = 0;
    for (size_t l = 0; l < s->levels.size(); l++)
        for (const Move& m : s->levels[l]) {
            if (i < cap && moves && sizes) {
                int64_t* o = moves + 10 * i;
                o[0] = (int64_t)l;
                o[1] = m.dst.rank, o[2] = m.dst.buf, o[3] = m.dst.off;
                o[4] = m.a.rank, o[5] = m.a.buf, o[6] = m.a.off;
                o[7] = m.b.rank, o[8] = m.b.buf, o[9] = m.b.off;
                sizes[i] = m.n * 2 + m.add;
            }
            i++;
        }
    if (n_moves) *n_moves = i;
    return BINE_SUCCESS;
}

int bine_plan_flow(bine_comm_t comm, bine_coll_t coll, long count, int root, int elem_size, int target_items,
                   int64_t* pieces, size_t piece_cap, size_t* n_pieces, int32_t* items, size_t item_cap,
                   size_t* n_items, int32_t* deps, size_t dep_cap, size_t* n_deps) {
    if (elem_size != 1 && elem_size != 4 && elem_size != 8) return fail(BINE_ERR_ARG, "element size must be 1, 4 or 8");
    if (target_items < 1) return fail(BINE_ERR_ARG, "target_items must be >= 1");
    std::shared_ptr<Schedule> s;
    int rc = plan_for_query(comm, coll, count, root, &s);
    if (rc) return rc;
    FlowPlan fp;
    if (fusion_levels(comm, coll, s.get()) > 1) {
        // The fused plan: pieces index the fused moves in pass order.
        FusedSchedule fs;
        rc = fused_schedule(comm, make_key(comm, coll, count, root), fusion_levels(comm, coll, s.get()), &s, &fs);
        if (rc) return rc;
        const int64_t piece = comm->segment_bytes > 0 ? std::max<int64_t>(16, comm->segment_bytes / elem_size) : 0;
        build_flow_fused(fs, comm->P, piece, std::max<int64_t>(1, 4096 / elem_size), kFlowMaxItemBytes / elem_size,
                         target_items, dev::kFusedPieces, &fp);
    } else {
        flow_plan(*s, comm->P, elem_size, comm->segment_bytes, target_items, &fp);
    }
    for (size_t i = 0; i < fp.pieces.size() && i < piece_cap && pieces; i++) {
        pieces[3 * i] = fp.pieces[i].move;
        pieces[3 * i + 1] = fp.pieces[i].start;
        pieces[3 * i + 2] = fp.pieces[i].n;
    }
    for (size_t i = 0; i < fp.items.size() && i < item_cap && items; i++) {
        const FlowItem& it = fp.items[i];
        int32_t* o = items + 5 * i;
        o[0] = it.pbeg, o[1] = it.pend, o[2] = it.dbeg, o[3] = it.dend, o[4] = it.level;
    }
    for (size_t i = 0; i < fp.deps.size() && i < dep_cap && deps; i++) deps[i] = fp.deps[i];
    if (n_pieces) *n_pieces = fp.pieces.size();
    if (n_items) *n_items = fp.items.size();
    if (n_deps) *n_deps = fp.deps.size();
    return BINE_SUCCESS;
}

int bine_plan_fused(bine_comm_t comm, bine_coll_t coll, long count, int root, int levels, int64_t* moves,
                    size_t move_cap, size_t* n_moves, int64_t* leaves, size_t leaf_cap, size_t* n_leaves,
                    int64_t* dsts, size_t dst_cap, size_t* n_dsts, int64_t* tmp_elems) {
    if (!comm) return fail(BINE_ERR_ARG, "null communicator");
    if ((int)coll < 0 || (int)coll >= kNumColls) return fail(BINE_ERR_ARG, "invalid collective");
    if (count <= 0) return fail(BINE_ERR_ARG, "count must be positive");
    if (levels < 1 || levels > 64) return fail(BINE_ERR_ARG, "levels per pass must be in [1, 64]");
    std::shared_ptr<Schedule> s;
    FusedSchedule fs;
    int rc = fused_schedule(comm, make_key(comm, coll, count, root), levels, &s, &fs);
    if (rc) return rc;
    size_t nm = 0;
    for (const auto& pass : fs.passes) nm += pass.size();
    if (n_moves) *n_moves = nm;
    if (n_leaves) *n_leaves = fs.leaves.size();
    if (n_dsts) *n_dsts = fs.dsts.size();
    if (tmp_elems) *tmp_elems = fs.tmp_elems;
    if (moves && move_cap >= nm) {
        size_t i = 0;
        for (size_t p = 0; p < fs.passes.size(); p++)
            for (const FusedMove& m : fs.passes[p]) {
                int64_t* o = moves + 6 * i++;
                o[0] = (int64_t)p;
                o[1] = m.n;
                o[2] = m.leaf_begin;
                o[3] = m.nleaves;
                o[4] = m.dst_begin;
                o[5] = m.ndst;
            }
    }
    if (leaves && leaf_cap >= fs.leaves.size())
        for (size_t i = 0; i < fs.leaves.size(); i++) {
            leaves[4 * i] = fs.leaves[i].rank;
            leaves[4 * i + 1] = fs.leaves[i].buf;
            leaves[4 * i + 2] = fs.leaves[i].adds;
            leaves[4 * i + 3] = fs.leaves[i].off;
        }
    if (dsts && dst_cap >= fs.dsts.size())
        for (size_t i = 0; i < fs.dsts.size(); i++) {
            dsts[3 * i] = fs.dsts[i].rank;
            dsts[3 * i + 1] = fs.dsts[i].buf;
            dsts[3 * i + 2] = fs.dsts[i].off;
        }
    return BINE_SUCCESS;
}

int bine_plan_messages(bine_comm_t comm, bine_coll_t coll, long count, int root, int64_t* msgs, size_t cap,
                       size_t* n_msgs) {
    std::shared_ptr<Schedule> s;
    int rc = plan_for_query(comm, coll, count, root, &s);
    if (rc) return rc;
    for (size_t i = 0; i < s->messages.size() && i < cap && msgs; i++) {
        const Message& m = s->messages[i];
        msgs[4 * i] = m.level;
        msgs[4 * i + 1] = m.src;
        msgs[4 * i + 2] = m.dst;
        msgs[4 * i + 3] = m.elems;
    }
    if (n_msgs) *n_msgs = s->messages.size();
    return BINE_SUCCESS;
}

int bine_plan_trees(bine_comm_t comm, bine_coll_t coll, long count, int root, int64_t* prog, size_t prog_cap,
                    size_t* n_prog, int64_t* segs, size_t seg_cap, size_t* n_segs) {
    std::shared_ptr<Schedule> s;
    int rc = plan_for_query(comm, coll, count, root, &s);
    if (rc) return rc;
    TreePlan tp;
    std::string err;
    if (!comm->planner->trees(make_key(comm, coll, count, root), *s, &tp, &err)) return fail(BINE_ERR_INTERNAL, err);
    for (size_t i = 0; i < tp.prog.size() && i < prog_cap && prog; i++) {
        prog[3 * i] = tp.prog[i].rank;
        prog[3 * i + 1] = tp.prog[i].adds;
        prog[3 * i + 2] = tp.prog[i].shift;
    }
    for (size_t i = 0; i < tp.segs.size() && i < seg_cap && segs; i++) {
        const OutSegment& g = tp.segs[i];
        int64_t* o = segs + 6 * i;
        o[0] = g.off, o[1] = g.n, o[2] = g.rank, o[3] = g.prog_begin, o[4] = g.prog_len, o[5] = g.depth;
    }
    if (n_prog) *n_prog = tp.prog.size();
    if (n_segs) *n_segs = tp.segs.size();
    return BINE_SUCCESS;
}

int bine_link_bytes(bine_comm_t comm, bine_coll_t coll, long count, bine_datatype_t datatype, int root,
                    uint64_t* d_link_bytes) {
    if (!comm || !d_link_bytes) return fail(BINE_ERR_ARG, "null argument");
    if ((int)coll < 0 || (int)coll >= kNumColls) return fail(BINE_ERR_ARG, "invalid collective");
    if (count <= 0) return fail(BINE_ERR_ARG, "count must be positive");
    const int es = dtype_size(datatype);
    if (es < 0) return fail(BINE_ERR_ARG, "invalid datatype");
    int rc = ensure_device(comm);
    if (rc) return rc;
    const Torus& t = comm->planner->torus();
    const size_t nlinks = (size_t)t.size * t.ndims * 2;
    unsigned long long* links = (unsigned long long*)d_link_bytes;
    CUDA_TRY(cudaMemsetAsync(links, 0, nlinks * sizeof(unsigned long long), comm->stream));
    bool all_p2 = true;
    for (int d = 0; d < t.ndims; d++) all_p2 &= is_pow2(t.dims[d]);
    const CollCfg& cf = comm->cfg[coll];
    bool mirrored = false;
    for (int p = 0; p < comm->ports; p++) mirrored |= mirrored_port(p, t.ndims);
    int kind = -1;
    if (all_p2 && cf.family != kFamilyRing && (cf.family == kFamilyBine || !mirrored)) {
        const int cl = (int)coll;
        if (cl == kAllreduce && (cf.variant == kArB || cf.variant == kArBCoalesce) && cf.distance == kIncreasing &&
            count >= (long)comm->ports * t.size)
            kind = 0;
        else if (cl == kAllreduce && cf.variant == kArL)
            kind = 1;
        else if (cl == kAllgather && cf.variant == kAgContPermute && cf.distance == kDecreasing)
            kind = 2;
    }
    if (kind >= 0) {
        dev::LinkGen g{t, cf.family, comm->ports, kind, (long long)count, es};
        const long long threads = (long long)t.size * comm->ports;
        unsigned grid = (unsigned)std::max(1LL, std::min((threads + 127) / 128, (long long)comm->num_sms * 32));
        dev::k_link_generate<<<grid, 128, 0, comm->stream>>>(g, links);
    } else {
        std::shared_ptr<Schedule> s;
        rc = plan_for_query(comm, coll, count, root, &s);
        if (rc) return rc;
        std::vector<long long> m(4 * s->messages.size());
        for (size_t i = 0; i < s->messages.size(); i++) {
            m[4 * i] = s->messages[i].level;
            m[4 * i + 1] = s->messages[i].src;
            m[4 * i + 2] = s->messages[i].dst;
            m[4 * i + 3] = s->messages[i].elems;
        }
        if (!m.empty()) {
            rc = ensure_work(comm, m.size() * sizeof(long long));
            if (rc) return rc;
            CUDA_TRY(cudaMemcpyAsync(comm->work, m.data(), m.size() * sizeof(long long), cudaMemcpyHostToDevice,
                                     comm->stream));
            CUDA_TRY(cudaStreamSynchronize(comm->stream));  // m is a host temporary
            const long long n = (long long)s->messages.size();
            unsigned grid = (unsigned)std::max(1LL, std::min((n + 255) / 256, (long long)comm->num_sms * 16));
            dev::k_link_from_msgs<<<grid, 256, 0, comm->stream>>>(t, (const long long*)comm->work, n, es, links);
        }
    }
    long long nlines = 0;
    for (int d = 0; d < t.ndims; d++) nlines += 2ll * (t.size / t.dims[d]);
    unsigned grid = (unsigned)std::max(1LL, std::min((nlines + 127) / 128, (long long)comm->num_sms * 8));
    dev::k_link_scan<<<grid, 128, 0, comm->stream>>>(t, links);
    CUDA_TRY(cudaGetLastError());
    return BINE_SUCCESS;
}

int bine_link_bytes_host(bine_comm_t comm, bine_coll_t coll, long count, bine_datatype_t datatype, int root,
                         uint64_t* link_bytes, size_t cap) {
    std::shared_ptr<Schedule> s;
    int rc = plan_for_query(comm, coll, count, root, &s);
    if (rc) return rc;
    const int es = dtype_size(datatype);
    if (es < 0) return fail(BINE_ERR_ARG, "invalid datatype");
    std::vector<uint64_t> lb;
    std::string err;
    if (!bine::link_bytes(comm->planner->torus(), s->messages, es, &lb, &err)) return fail(BINE_ERR_INTERNAL, err);
    if (cap < lb.size()) return fail(BINE_ERR_ARG, "link_bytes array too small");
    std::copy(lb.begin(), lb.end(), link_bytes);
    return BINE_SUCCESS;
}

}  // extern "C"

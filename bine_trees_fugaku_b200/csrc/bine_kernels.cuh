// Device kernels of the Bine engine (sm_100a).
//
// All collectives here move or add whole rows of P virtual ranks that live
// in one HBM: the work is streaming integer/float traffic, bound by HBM
// bandwidth, so the kernels are built around 16-byte vector loads and
// stores, enough independent loads in flight per thread to cover DRAM
// latency (8 ranks per batch), streaming cache hints, and grids sized to the
// 148 SMs.  Nothing here is a dense contraction, so there are no tensor-core
// paths.
//
//   k_sum_*      fused reductions (allreduce, reduce_scatter, reduce): each
//                column of the P inputs is read once and the result written
//                once per destination; integer sums wrap exactly, the FAST
//                float order accumulates in FP64.
//   k_tree_*     fused reductions in the reference's exact float order: each
//                output segment carries the postfix program of its addition
//                tree (produced by the host planner), evaluated per column
//                with an in-register top of stack.
//   k_copy_*     allgather, bcast, alltoall, scatter and gather as one pass of
//                16-byte copies (one load, one or P stores).
//   k_steps      the reference's schedule executed level by level in one
//                cooperative launch, with a bounded grid-wide barrier between
//                levels that reports a timeout instead of hanging.
//   k_flow       the same schedule as a dataflow of segments: each starts
//                when the segments it reads and overwrites are done (bounded
//                waits on per-segment completion flags), so steps overlap.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace bine {
namespace dev {

constexpr int kThreads = 256;
constexpr int kMaxTreeDepth = 24;

// ---------------------------------------------------------------- memory
__device__ __forceinline__ uint4 ld_stream(const void* p) {
    uint4 v;
    asm volatile("ld.global.nc.L1::no_allocate.v4.u32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p));
    return v;
}
// L2-coherent load (bypasses L1): rows written by other blocks earlier in
// the same launch must not be served from a stale L1 line.
__device__ __forceinline__ uint4 ld_plain(const void* p) {
    uint4 v;
    asm volatile("ld.global.cg.v4.u32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p)
                 : "memory");
    return v;
}
__device__ __forceinline__ void st_stream(void* p, uint4 v) {
    asm volatile("st.global.cs.v4.u32 [%0], {%1, %2, %3, %4};" ::"l"(p), "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w)
                 : "memory");
}

// ----------------------------------------------------------- lane algebra
// Accumulators: wrapping integers of the element type, FP64 for the FAST
// float order, the element type itself for the exact float order.
template <typename T>
struct AccOf {
    using type = T;
};
template <>
struct AccOf<float> {
    using type = double;
};

template <typename T>
__device__ __forceinline__ T add_exact(T a, T b) {
    return (T)(a + b);
}
template <>
__device__ __forceinline__ float add_exact<float>(float a, float b) {
    return __fadd_rn(a, b);
}
template <>
__device__ __forceinline__ double add_exact<double>(double a, double b) {
    return __dadd_rn(a, b);
}

template <typename T, typename A>
struct Lanes {
    static constexpr int N = 16 / sizeof(T);
    A v[N];
    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int i = 0; i < N; i++) v[i] = (A)0;
    }
    __device__ __forceinline__ void add(uint4 raw) {
        const T* t = reinterpret_cast<const T*>(&raw);
#pragma unroll
        for (int i = 0; i < N; i++) v[i] = add_exact<A>(v[i], (A)t[i]);
    }
    __device__ __forceinline__ uint4 pack() const {
        uint4 raw;
        T* t = reinterpret_cast<T*>(&raw);
#pragma unroll
        for (int i = 0; i < N; i++) t[i] = (T)v[i];
        return raw;
    }
};

template <typename T>
__device__ __forceinline__ uint4 vadd(uint4 a, uint4 b) {
    uint4 r;
    const T* x = reinterpret_cast<const T*>(&a);
    const T* y = reinterpret_cast<const T*>(&b);
    T* z = reinterpret_cast<T*>(&r);
#pragma unroll
    for (int i = 0; i < (int)(16 / sizeof(T)); i++) z[i] = add_exact<T>(x[i], y[i]);
    return r;
}

// ------------------------------------------------------- fused reductions
enum SumMode { kSumAllreduce = 0, kSumReduceScatter = 1, kSumReduce = 2 };

// Column sums over 16-byte vector columns.  A block owns tiles of COLS
// vector columns at a time; its 256 threads form 256/COLS row groups that
// split the P rows of a tile (group g sums rows [g*P/G, (g+1)*P/G) of its
// lane's column, 8 loads in flight per thread), the partial sums meet in
// shared memory, and all threads then store the result rows.  The host
// picks COLS (64 columns and 4 row groups; one group below P = 16; narrower
// tiles for calls too small to give every SM two tiles) and launches one
// block per tile up to 64 blocks per SM, beyond which blocks walk the tiles
// grid-stride.  `ncol` vector columns per input row; reduce_scatter: `blk`
// vector columns per destination rank.
constexpr int kSumCols = 8;  // the narrowest tile (32 row groups)

template <typename T, int MODE, int COLS>
__global__ void __launch_bounds__(kThreads) k_sum_vec(const char* __restrict__ in, long long in_stride,
                                                      char* __restrict__ out, long long out_stride, int P,
                                                      long long ncol, long long blk, int root) {
    using A = typename AccOf<T>::type;
    constexpr int G = kThreads / COLS;
    __shared__ Lanes<T, A> part[G][COLS];
    __shared__ uint4 res[COLS];
    const int lane = threadIdx.x % COLS, grp = threadIdx.x / COLS;
    const int per = (P + G - 1) / G;
    const int r0 = min(P, grp * per), r1 = min(P, r0 + per);
    const long long ntiles = (ncol + COLS - 1) / COLS;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const long long col = tile * COLS + lane;
        Lanes<T, A> acc;
        acc.zero();
        if (col < ncol) {
            const char* p = in + col * 16;
            int r = r0;
            for (; r + 8 <= r1; r += 8) {
                uint4 v[8];
#pragma unroll
                for (int u = 0; u < 8; u++) v[u] = ld_stream(p + (long long)(r + u) * in_stride);
#pragma unroll
                for (int u = 0; u < 8; u++) acc.add(v[u]);
            }
            for (; r < r1; r++) acc.add(ld_stream(p + (long long)r * in_stride));
        }
        if (G > 1) {
            part[grp][lane] = acc;
            __syncthreads();
            if (grp == 0) {
                Lanes<T, A> sum = part[0][lane];
#pragma unroll
                for (int g = 1; g < G; g++)
#pragma unroll
                    for (int i = 0; i < Lanes<T, A>::N; i++) sum.v[i] = add_exact<A>(sum.v[i], part[g][lane].v[i]);
                res[lane] = sum.pack();
            }
            __syncthreads();
        } else {
            res[lane] = acc.pack();
        }
        if (col < ncol) {
            const uint4 v = res[lane];
            if (MODE == kSumAllreduce) {
                char* q = out + col * 16;
                for (int d = grp; d < P; d += G) st_stream(q + (long long)d * out_stride, v);
            } else if (grp == 0) {
                if (MODE == kSumReduceScatter) {
                    const long long owner = col / blk;
                    st_stream(out + owner * out_stride + (col - owner * blk) * 16, v);
                } else {
                    st_stream(out + (long long)root * out_stride + col * 16, v);
                }
            }
        }
        if (G > 1) __syncthreads();
    }
}

// Element-wise fallback for unaligned layouts and tails: elements
// [e0, e0 + n) of every row.  reduce_scatter: `blk` elements per rank.
template <typename T, int MODE>
__global__ void __launch_bounds__(kThreads) k_sum_scalar(const char* __restrict__ in, long long in_stride,
                                                         char* __restrict__ out, long long out_stride, int P,
                                                         long long e0, long long n, long long blk, int root) {
    using A = typename AccOf<T>::type;
    const long long step = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += step) {
        const long long e = e0 + i;
        A acc = (A)0;
        for (int r = 0; r < P; r++) acc = add_exact<A>(acc, (A) * (const T*)(in + (long long)r * in_stride + e * sizeof(T)));
        const T res = (T)acc;
        if (MODE == kSumAllreduce) {
            for (int d = 0; d < P; d++) *(T*)(out + (long long)d * out_stride + e * sizeof(T)) = res;
        } else if (MODE == kSumReduceScatter) {
            long long owner = e / blk;
            *(T*)(out + owner * out_stride + (e - owner * blk) * sizeof(T)) = res;
        } else {
            *(T*)(out + (long long)root * out_stride + e * sizeof(T)) = res;
        }
    }
}

// ------------------------------------------- fused reductions, exact order
struct TreeEntry {  // one postfix entry: push input (rank, out + shift), then `adds` additions
    int32_t rank;
    int32_t adds;
    int64_t shift;
};
struct TreeSeg {  // output elements [off, off + n) of `rank` (-1: all ranks)
    int64_t off, n;
    int32_t rank, prog_begin, prog_len, depth;
};
struct TreeTile {  // `n` elements starting `start` elements into segment `seg`
    int32_t seg, pad;
    int64_t start, n;
};

// Evaluation stack of a postfix program (the entries below the top, which
// stays in registers).  SMEM: in the block's dynamic shared memory, slot j
// of thread t at base[j * kThreads + t], so a warp's 16-byte accesses fall
// on consecutive words; sized by the host to the programs' Sethi-Ullman
// depth.  Otherwise a local array (deep programs only): its indexing is
// dynamic, so it lives in local memory and its traffic reaches L2.
template <bool SMEM>
struct EvalStack;
template <>
struct EvalStack<true> {
    uint4* base;
    __device__ __forceinline__ void init(uint4* smem_stack) { base = smem_stack + threadIdx.x; }
    __device__ __forceinline__ void set(int j, uint4 v) { base[j * kThreads] = v; }
    __device__ __forceinline__ uint4 get(int j) const { return base[j * kThreads]; }
};
template <>
struct EvalStack<false> {
    uint4 a[kMaxTreeDepth];
    __device__ __forceinline__ void init(uint4*) {}
    __device__ __forceinline__ void set(int j, uint4 v) { a[j] = v; }
    __device__ __forceinline__ uint4 get(int j) const { return a[j]; }
};

// Vector form: every shift and offset is a multiple of 16 bytes.  One tile
// per block; each thread owns one 16-byte column of the tile.
template <typename T, bool SMEM>
__global__ void __launch_bounds__(kThreads) k_tree_vec(const char* __restrict__ in, long long in_stride,
                                                       char* __restrict__ out, long long out_stride, int P,
                                                       const TreeSeg* __restrict__ segs,
                                                       const TreeEntry* __restrict__ prog,
                                                       const TreeTile* __restrict__ tiles, int ntiles,
                                                       int stack_off) {
    extern __shared__ uint4 sdyn[];
    TreeEntry* sprog = reinterpret_cast<TreeEntry*>(sdyn);
    EvalStack<SMEM> stk;
    stk.init(sdyn + stack_off);
    constexpr int L = 16 / sizeof(T);
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const TreeTile tile = tiles[t];
        const TreeSeg sg = segs[tile.seg];
        __syncthreads();
        // Staged with each leaf's byte offset (rank row + shift) precomputed.
        for (int i = threadIdx.x; i < sg.prog_len; i += blockDim.x) {
            TreeEntry q = prog[sg.prog_begin + i];
            q.shift = (long long)q.rank * in_stride + q.shift * (long long)sizeof(T);
            sprog[i] = q;
        }
        __syncthreads();
        const long long col = (long long)threadIdx.x * L;
        if (col >= tile.n) continue;
        const long long e = sg.off + tile.start + col;  // output element
        const char* base = in + e * (long long)sizeof(T);
        uint4 top = make_uint4(0, 0, 0, 0);
        int sp = 0;
        const int len = sg.prog_len;
        // Loads run 8 entries ahead of the additions.
        uint4 ring[8];
#pragma unroll
        for (int u = 0; u < 8; u++)
            if (u < len) {
                const TreeEntry q = sprog[u];
                ring[u] = ld_stream(base + q.shift);
            }
        for (int k0 = 0; k0 < len; k0 += 8) {
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const int k = k0 + u;
                if (k < len) {
                    const uint4 v = ring[u];
                    if (k + 8 < len) {
                        const TreeEntry q = sprog[k + 8];
                        ring[u] = ld_stream(base + q.shift);
                    }
                    if (k > 0) stk.set(sp++, top);
                    top = v;
                    for (int a = sprog[k].adds; a > 0; a--) top = vadd<T>(stk.get(--sp), top);
                }
            }
        }
        if (sg.rank < 0) {
            for (int d = 0; d < P; d++) st_stream(out + (long long)d * out_stride + e * (long long)sizeof(T), top);
        } else {
            st_stream(out + (long long)sg.rank * out_stride + e * (long long)sizeof(T), top);
        }
    }
}

// Split form of k_tree_vec.  The host cut every segment's addition tree
// into `nparts` disjoint subtrees (the "parts", left to right; K of them,
// or 2K when that balances the warps better) and a combine program whose
// leaves are the parts, and assigned the parts to K warps longest first, so
// the warps carry near-equal numbers of leaves even when the tree is
// unbalanced (non-power-of-two P).  A block of 8 warps owns 8/K
// column groups of 32 vectors; warp w evaluates its parts for group w / K,
// one vector per lane, so every load of a warp is 512 contiguous bytes of
// one rank row (as in k_sum_vec).  The partial sums meet in shared memory;
// each warp then runs the combine program for its group's 32 vectors and
// stores every K-th destination row.  The additions and their association
// are exactly the tree's.  Shorter tasks remove the tail of the last wave
// when the output has few vectors per resident thread.
struct TreeComb {  // combine entry: push part `part`, then `adds` additions
    int32_t part, adds;
};

// Evaluates program entries [b, b + len) for one 16-byte vector whose first
// input element is at `base` (entries hold each leaf's byte offset from
// there), loads kRing entries ahead of the additions.
template <typename T, bool SMEM, int kRing>
__device__ __forceinline__ uint4 eval_program(const char* __restrict__ base, const TreeEntry* sprog, int b, int len,
                                              EvalStack<SMEM>& stk) {
    uint4 top = make_uint4(0, 0, 0, 0);
    int sp = 0;
    uint4 ring[kRing];
#pragma unroll
    for (int u = 0; u < kRing; u++)
        if (u < len) {
            const TreeEntry q = sprog[b + u];
            ring[u] = ld_stream(base + q.shift);
        }
    for (int k0 = 0; k0 < len; k0 += kRing) {
#pragma unroll
        for (int u = 0; u < kRing; u++) {
            const int k = k0 + u;
            if (k < len) {
                const uint4 v = ring[u];
                if (k + kRing < len) {
                    const TreeEntry q = sprog[b + k + kRing];
                    ring[u] = ld_stream(base + q.shift);
                }
                if (k > 0) stk.set(sp++, top);
                top = v;
                for (int a = sprog[b + k].adds; a > 0; a--) top = vadd<T>(stk.get(--sp), top);
            }
        }
    }
    return top;
}

template <typename T, int K, bool SMEM>
__global__ void __launch_bounds__(kThreads) k_tree_split(const char* __restrict__ in, long long in_stride,
                                                         char* __restrict__ out, long long out_stride, int P,
                                                         const TreeSeg* __restrict__ segs,
                                                         const TreeEntry* __restrict__ prog,
                                                         const int* __restrict__ parts,
                                                         const TreeComb* __restrict__ comb,
                                                         const int* __restrict__ assign,
                                                         const TreeTile* __restrict__ tiles, int ntiles,
                                                         int nparts, int stack_off) {
    extern __shared__ uint4 sdyn[];
    TreeEntry* sprog = reinterpret_cast<TreeEntry*>(sdyn);
    EvalStack<SMEM> stk;
    stk.init(sdyn + stack_off);
    constexpr int kWarps = kThreads / 32;
    constexpr int kGroups = kWarps / K;
    constexpr int KP = 2 * K;
    // Per segment: part offsets, combine program, and the parts of each warp
    // (nparts <= KP part indices ordered by warp, then K + 1 offsets).
    __shared__ int spart[KP + 1];
    __shared__ TreeComb scomb[KP];
    __shared__ int sasg[KP + K + 1];
    __shared__ uint4 partial[kGroups][KP][32];
    constexpr int L = 16 / sizeof(T);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int j = warp % K, g = warp / K;
    int cur = -1;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const TreeTile tile = tiles[t];
        const TreeSeg sg = segs[tile.seg];
        __syncthreads();  // the previous tile's partials and program are consumed
        if (tile.seg != cur) {  // block-uniform
            for (int i = threadIdx.x; i < sg.prog_len; i += blockDim.x) {
                TreeEntry q = prog[sg.prog_begin + i];
                q.shift = (long long)q.rank * in_stride + q.shift * (long long)sizeof(T);  // byte offset
                sprog[i] = q;
            }
            if (threadIdx.x <= nparts) spart[threadIdx.x] = parts[(long long)tile.seg * (nparts + 1) + threadIdx.x];
            if (threadIdx.x < nparts) scomb[threadIdx.x] = comb[(long long)tile.seg * nparts + threadIdx.x];
            if (threadIdx.x < nparts + K + 1)
                sasg[threadIdx.x] = assign[(long long)tile.seg * (nparts + K + 1) + threadIdx.x];
            __syncthreads();
            cur = tile.seg;
        }
        const long long col = (long long)(g * 32 + lane) * L;
        const bool active = col < tile.n;
        const long long e = sg.off + tile.start + col;
        if (active) {
            for (int pi = sasg[nparts + j]; pi < sasg[nparts + j + 1]; pi++) {
                const int p = sasg[pi];
                partial[g][p][lane] = eval_program<T, SMEM, 4>(in + e * (long long)sizeof(T), sprog, spart[p],
                                                               spart[p + 1] - spart[p], stk);
            }
        }
        __syncthreads();
        if (!active) continue;
        uint4 top = make_uint4(0, 0, 0, 0);
        int csp = 0;  // the parts' stack is empty again: the combine reuses it
        for (int q = 0; q < nparts; q++) {
            const TreeComb c = scomb[q];
            if (q > 0) stk.set(csp++, top);
            top = partial[g][c.part][lane];
            for (int a = c.adds; a > 0; a--) top = vadd<T>(stk.get(--csp), top);
        }
        if (sg.rank < 0) {
            for (int d = j; d < P; d += K) st_stream(out + (long long)d * out_stride + e * (long long)sizeof(T), top);
        } else if (j == 0) {
            st_stream(out + (long long)sg.rank * out_stride + e * (long long)sizeof(T), top);
        }
    }
}

// Row-aligned form of k_tree_split, for calls whose trees have few
// shapes.  In allreduce every leaf reads its rank's row at the output's own
// column, and the segments' trees (one segment per block of the
// reference's vector) share one shape, or a few (at most kFlatShapes):
// segments of one shape differ only in the order of their ranks.  The tiles of k_tree_split start at each segment's
// first 16-byte boundary; with non-power-of-two P that is an arbitrary
// 16-byte offset, so every 512-byte warp access straddles five 128-byte
// lines, and a segment's last tile is mostly empty.  Here tiles follow the
// output row's own grid of 32-vector groups instead: `tile.start` is a
// multiple of the tile width (in elements, from the row start), a tile may
// hold the ends of several segments of one shape (`tile.pad & 0xff` of them
// from `tile.seg`, in the order of their bodies; the shape is
// `tile.pad >> 8`, and the block stages that shape's plan when it changes),
// and each lane evaluates its own segment's ranks.  Where segments of
// several shapes meet in one tile's columns, each shape has its own tile
// there, and lanes whose vector belongs to another shape idle.
//
// A vector that straddles two consecutive segments (an "edge": its first
// `cut` elements end segment q, the rest begin segment q + 1) is evaluated
// by k_tree_edges, beside this kernel, as a whole 16-byte vector, instead of
// element by element.  The additions, and so the results, are exactly the
// trees'.
//
//   body[2q], body[2q+1] segment q's vector body [lo, hi), in elements
//   ranks[q * pitch + k] the rank of entry k of segment q's split program;
//   ranks_t[k * nq + q] the same, entry-major (edge lanes read consecutive q)
//   adds[h * len + k]   additions after entry k of shape h's programs
//   parts, comb, assign shape h's split plan (as in k_tree_split), at
//                       h * (nparts + 1), h * nparts, h * (nparts + K + 1)
constexpr int kFlatSegs = 8;    // segments one row tile may touch
constexpr int kFlatShapes = 8;  // tree shapes one call may have

struct FlatEdge {  // the vector at element `e`: elements [e, e + cut) in segment q, the rest in q + 1
    int64_t e;
    int32_t q, cut;
};

struct FlatArgs {
    const char* in;
    long long in_stride;
    char* out;
    long long out_stride;
    int P;
    const int64_t* body;
    const uint16_t* ranks;
    const uint16_t* ranks_t;
    int pitch, nq;
    const uint8_t* adds;
    int len;  // bytes of `adds`, a multiple of 16
    const int* parts;
    const TreeComb* comb;
    const int* assign;
    const FlatEdge* edges;
    const uint8_t* shape;  // edges: the tree shape of each segment (row order)
    int nshape;
    const TreeTile* tiles;
    int ntiles, nparts;
    int ranks_off, stack_off;  // dynamic shared memory offsets, in 16-byte words
};

// Evaluates entries [b, b + len) of a program whose additions are
// `adds[k]` and whose ranks are `rk[k]` (a row of the shared-memory rank
// table), for one 16-byte vector at `base`; loads run kRing entries ahead
// of the additions.
template <typename T, bool SMEM, int kRing>
__device__ __forceinline__ uint4 eval_ranks(const char* __restrict__ base, long long stride, const uint16_t* rk,
                                            const uint8_t* adds, int b, int len, EvalStack<SMEM>& stk) {
    uint4 top = make_uint4(0, 0, 0, 0);
    int sp = 0;
    uint4 ring[kRing];
#pragma unroll
    for (int u = 0; u < kRing; u++)
        if (u < len) ring[u] = ld_stream(base + (long long)rk[b + u] * stride);
    for (int k0 = 0; k0 < len; k0 += kRing) {
#pragma unroll
        for (int u = 0; u < kRing; u++) {
            const int k = k0 + u;
            if (k < len) {
                const uint4 v = ring[u];
                if (k + kRing < len) ring[u] = ld_stream(base + (long long)rk[b + k + kRing] * stride);
                if (k > 0) stk.set(sp++, top);
                top = v;
                for (int a = adds[b + k]; a > 0; a--) top = vadd<T>(stk.get(--sp), top);
            }
        }
    }
    return top;
}

template <typename T, int K, bool SMEM>
__global__ void __launch_bounds__(kThreads) k_tree_flat(const FlatArgs A) {
    extern __shared__ uint4 sdyn[];
    uint8_t* sadds = reinterpret_cast<uint8_t*>(sdyn);
    uint16_t* sranks = reinterpret_cast<uint16_t*>(sdyn + A.ranks_off);
    EvalStack<SMEM> stk;
    stk.init(sdyn + A.stack_off);
    constexpr int kWarps = kThreads / 32;
    constexpr int kGroups = kWarps / K;
    constexpr int KP = 2 * K;
    __shared__ int spart[KP + 1];
    __shared__ TreeComb scomb[KP];
    __shared__ int sasg[KP + K + 1];
    __shared__ int64_t slo[kFlatSegs], shi[kFlatSegs];
    __shared__ uint4 partial[kGroups][KP][32];
    constexpr int L = 16 / sizeof(T);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int j = warp % K, g = warp / K;
    const int nparts = A.nparts;
    const int words = A.pitch / 8;  // 16-byte words of one segment's ranks
    const uint4* granks = reinterpret_cast<const uint4*>(A.ranks);
    uint4* sranks4 = reinterpret_cast<uint4*>(sranks);
    int cur = -1;  // the tree shape whose plan is staged
    for (int t = blockIdx.x; t < A.ntiles; t += gridDim.x) {
        const TreeTile tile = A.tiles[t];
        const int s0 = tile.seg, ns = tile.pad & 0xff, shape = tile.pad >> 8;
        __syncthreads();  // the previous tile's partials, ranks and plan are consumed
        if (shape != cur) {  // block-uniform: the plan of this tile's tree shape
            const uint4* ga = reinterpret_cast<const uint4*>(A.adds + (long long)shape * A.len);
            for (int i = threadIdx.x; i < A.len / 16; i += blockDim.x) sdyn[i] = ga[i];
            if (threadIdx.x <= nparts) spart[threadIdx.x] = A.parts[shape * (nparts + 1) + threadIdx.x];
            if (threadIdx.x < nparts) scomb[threadIdx.x] = A.comb[shape * nparts + threadIdx.x];
            if (threadIdx.x < nparts + K + 1) sasg[threadIdx.x] = A.assign[shape * (nparts + K + 1) + threadIdx.x];
            cur = shape;
        }
        for (int i = threadIdx.x; i < ns * words; i += blockDim.x) sranks4[i] = granks[(long long)s0 * words + i];
        if (threadIdx.x < ns) {
            slo[threadIdx.x] = A.body[2 * (s0 + threadIdx.x)];
            shi[threadIdx.x] = A.body[2 * (s0 + threadIdx.x) + 1];
        }
        __syncthreads();
        const long long e = tile.start + (long long)(g * 32 + lane) * L;  // first element of the lane's vector
        int slot = -1;
        if (e < tile.start + tile.n)
            for (int q = 0; q < ns; q++)
                if (e >= slo[q] && e < shi[q]) slot = q;
        const bool active = slot >= 0;
        if (active) {
            const uint16_t* rk = sranks + slot * A.pitch;
            for (int pi = sasg[nparts + j]; pi < sasg[nparts + j + 1]; pi++) {
                const int p = sasg[pi];
                partial[g][p][lane] = eval_ranks<T, SMEM, 4>(A.in + e * (long long)sizeof(T), A.in_stride, rk,
                                                             sadds, spart[p], spart[p + 1] - spart[p], stk);
            }
        }
        __syncthreads();
        if (!active) continue;
        uint4 top = make_uint4(0, 0, 0, 0);
        int csp = 0;
        for (int q = 0; q < nparts; q++) {
            const TreeComb c = scomb[q];
            if (q > 0) stk.set(csp++, top);
            top = partial[g][c.part][lane];
            for (int a = c.adds; a > 0; a--) top = vadd<T>(stk.get(--csp), top);
        }
        for (int d = j; d < A.P; d += K)
            st_stream(A.out + (long long)d * A.out_stride + e * (long long)sizeof(T), top);
    }
}

// Edge form of eval_ranks: the ranks come from the entry-major global
// table (`rt` at the lane's segment; entry k at rt[k * nq]) and are read
// one ring ahead of the loads that use them, so that a rank's L2 latency is
// not added to every leaf's.
template <typename T, bool SMEM, int kRing>
__device__ __forceinline__ uint4 eval_edge(const char* __restrict__ base, long long stride,
                                           const uint16_t* __restrict__ rt, int nq, const uint8_t* adds, int b,
                                           int len, EvalStack<SMEM>& stk) {
    uint4 top = make_uint4(0, 0, 0, 0);
    int sp = 0;
    uint4 ring[kRing];
    int rr[kRing];
#pragma unroll
    for (int u = 0; u < kRing; u++)
        if (u < len) rr[u] = __ldg(rt + (long long)(b + u) * nq);
#pragma unroll
    for (int u = 0; u < kRing; u++)
        if (u < len) {
            ring[u] = ld_stream(base + (long long)rr[u] * stride);
            if (u + kRing < len) rr[u] = __ldg(rt + (long long)(b + u + kRing) * nq);
        }
    for (int k0 = 0; k0 < len; k0 += kRing) {
#pragma unroll
        for (int u = 0; u < kRing; u++) {
            const int k = k0 + u;
            if (k < len) {
                const uint4 v = ring[u];
                if (k + kRing < len) {
                    ring[u] = ld_stream(base + (long long)rr[u] * stride);
                    if (k + 2 * kRing < len) rr[u] = __ldg(rt + (long long)(b + k + 2 * kRing) * nq);
                }
                if (k > 0) stk.set(sp++, top);
                top = v;
                for (int a = adds[b + k]; a > 0; a--) top = vadd<T>(stk.get(--sp), top);
            }
        }
    }
    return top;
}

// The edges of the row-aligned form (see above).  Their trees are cut into
// kEdgeParts subtrees of their own (the edge split plan of each shape h:
// `parts` at h * (kEdgeParts + 1), `comb` at h * kEdgeParts, `adds` at
// h * len; ranks_t in that plan's entry order, and `shape` giving each
// segment's shape), so that an edge's critical path is P / kEdgeParts
// leaves whatever the row tiles' split.
// Block b owns edges [32 * (b / 2), +32) and segment side b % 2 (0: the
// segment the edge vector ends, 1: the one it starts); warp w evaluates
// part w for its lane's edge, the partial sums meet in shared memory, and
// every lane combines them and stores the elements of its side (the first
// `cut` elements of the vector, or the rest) to the rows w, w + 8, ...  The
// two sides of an edge run in neighbouring blocks, so the two halves of its
// 16-byte vector reach L2 close together.
constexpr int kEdgeParts = 8;

template <typename T, bool SMEM>
__global__ void __launch_bounds__(kThreads) k_tree_edges(const FlatArgs A, int nedges) {
    extern __shared__ uint4 sdyn[];
    uint8_t* sadds = reinterpret_cast<uint8_t*>(sdyn);
    EvalStack<SMEM> stk;
    stk.init(sdyn + A.stack_off);
    static_assert(kThreads / 32 == kEdgeParts, "one warp per edge part");
    // The edge plans of every tree shape (a lane's edge may end a segment
    // of one shape and begin one of another).
    __shared__ int spart[kFlatShapes][kEdgeParts + 1];
    __shared__ TreeComb scomb[kFlatShapes][kEdgeParts];
    __shared__ uint4 partial[kEdgeParts][32];
    constexpr int L = 16 / sizeof(T);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < A.nshape * A.len / 16; i += blockDim.x)
        sdyn[i] = reinterpret_cast<const uint4*>(A.adds)[i];
    for (int i = threadIdx.x; i < A.nshape * (kEdgeParts + 1); i += blockDim.x)
        spart[i / (kEdgeParts + 1)][i % (kEdgeParts + 1)] = A.parts[i];
    for (int i = threadIdx.x; i < A.nshape * kEdgeParts; i += blockDim.x)
        scomb[i / kEdgeParts][i % kEdgeParts] = A.comb[i];
    const int ngroups = (nedges + 31) / 32;
    for (int t = blockIdx.x; t < 2 * ngroups; t += gridDim.x) {
        const int side = t & 1, ei = (t >> 1) * 32 + lane;
        const bool act = ei < nedges;
        FlatEdge ed{0, 0, 0};
        int sh = 0;
        if (act) {
            ed = A.edges[ei];
            sh = A.shape[ed.q + side];
        }
        __syncthreads();  // the previous partials are consumed (and the plans staged)
        if (act)
            partial[w][lane] = eval_edge<T, SMEM, 8>(A.in + ed.e * (long long)sizeof(T), A.in_stride,
                                                     A.ranks_t + ed.q + side, A.nq, sadds + sh * A.len, spart[sh][w],
                                                     spart[sh][w + 1] - spart[sh][w], stk);
        __syncthreads();
        if (!act) continue;
        uint4 top = make_uint4(0, 0, 0, 0);
        int csp = 0;
        for (int q = 0; q < kEdgeParts; q++) {
            const TreeComb c = scomb[sh][q];
            if (q > 0) stk.set(csp++, top);
            top = partial[c.part][lane];
            for (int a = c.adds; a > 0; a--) top = vadd<T>(stk.get(--csp), top);
        }
        const T* r = reinterpret_cast<const T*>(&top);
        const int x0 = side ? ed.cut : 0, x1 = side ? L : ed.cut;
        for (int d = w; d < A.P; d += kEdgeParts) {
            T* o = reinterpret_cast<T*>(A.out + (long long)d * A.out_stride + ed.e * (long long)sizeof(T));
            for (int x = x0; x < x1; x++) o[x] = r[x];
        }
    }
}

// Element form for the short head and tail pieces of segments (fewer
// elements than one 16-byte vector).  Per tile the block
//   1. loads every leaf value of the tile's elements into shared memory in
//      one parallel round;
//   2. evaluates the tree's parts (the split plan's `nparts` subtrees, or
//      the whole tree as one part) with one thread per (element, part);
//   3. combines each element's partials in the tree's order;
//   4. spreads the P destination stores over all its threads.
// Without steps 2 and 4 one thread per element ran the whole P-leaf
// program and issued all P stores, which made this small kernel as long as
// the vector kernel beside it at P = 1000.
constexpr int kMaxParts = 16;
constexpr int kMaxPiece = 4;  // elements of a piece: fewer than one vector

template <typename T>
__global__ void __launch_bounds__(kThreads) k_tree_staged(const char* __restrict__ in, long long in_stride,
                                                          char* __restrict__ out, long long out_stride, int P,
                                                          const TreeSeg* __restrict__ segs,
                                                          const TreeEntry* __restrict__ prog,
                                                          const int* __restrict__ parts,
                                                          const TreeComb* __restrict__ comb, int nparts,
                                                          const TreeTile* __restrict__ tiles, int ntiles,
                                                          int vals_off) {
    extern __shared__ uint4 sdyn[];
    TreeEntry* sprog = reinterpret_cast<TreeEntry*>(sdyn);
    T* vals = reinterpret_cast<T*>(sdyn + vals_off);
    __shared__ int spart[kMaxParts + 1];
    __shared__ TreeComb scomb[kMaxParts];
    __shared__ T partial[kMaxPiece][kMaxParts];
    __shared__ T res[kMaxPiece];
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const TreeTile tile = tiles[t];
        const TreeSeg sg = segs[tile.seg];
        const int len = sg.prog_len, n = (int)tile.n;
        __syncthreads();  // the previous tile's values and results are consumed
        for (int i = threadIdx.x; i < len; i += blockDim.x) sprog[i] = prog[sg.prog_begin + i];
        if (threadIdx.x <= nparts) spart[threadIdx.x] = parts[(long long)tile.seg * (nparts + 1) + threadIdx.x];
        if (threadIdx.x < nparts) scomb[threadIdx.x] = comb[(long long)tile.seg * nparts + threadIdx.x];
        __syncthreads();
        const long long e0 = sg.off + tile.start;
        for (int i = threadIdx.x; i < n * len; i += blockDim.x) {
            const int jj = i / len, k = i - jj * len;
            const TreeEntry q = sprog[k];
            vals[i] = *(const T*)(in + (long long)q.rank * in_stride + (e0 + jj + q.shift) * (long long)sizeof(T));
        }
        __syncthreads();
        for (int w = threadIdx.x; w < n * nparts; w += blockDim.x) {
            const int jj = w / nparts, p = w - jj * nparts;
            const T* v = vals + jj * len;
            T stk[kMaxTreeDepth];
            T top = (T)0;
            int sp = 0;
            for (int k = spart[p]; k < spart[p + 1]; k++) {
                if (k > spart[p]) stk[sp++] = top;
                top = v[k];
                for (int a = sprog[k].adds; a > 0; a--) top = add_exact<T>(stk[--sp], top);
            }
            partial[jj][p] = top;
        }
        __syncthreads();
        if (threadIdx.x < n) {
            T stk[kMaxParts];
            T top = (T)0;
            int sp = 0;
            for (int q = 0; q < nparts; q++) {
                if (q > 0) stk[sp++] = top;
                top = partial[threadIdx.x][scomb[q].part];
                for (int a = scomb[q].adds; a > 0; a--) top = add_exact<T>(stk[--sp], top);
            }
            res[threadIdx.x] = top;
        }
        __syncthreads();
        if (sg.rank < 0) {
            for (int w = threadIdx.x; w < P * n; w += blockDim.x) {
                const int d = w / n, jj = w - d * n;
                *(T*)(out + (long long)d * out_stride + (e0 + jj) * (long long)sizeof(T)) = res[jj];
            }
        } else if (threadIdx.x < n) {
            *(T*)(out + (long long)sg.rank * out_stride + (e0 + threadIdx.x) * (long long)sizeof(T)) = res[threadIdx.x];
        }
    }
}

// Element form for layouts that are not 16-byte aligned.
template <typename T>
__global__ void __launch_bounds__(kThreads) k_tree_scalar(const char* __restrict__ in, long long in_stride,
                                                          char* __restrict__ out, long long out_stride, int P,
                                                          const TreeSeg* __restrict__ segs,
                                                          const TreeEntry* __restrict__ prog,
                                                          const TreeTile* __restrict__ tiles, int ntiles) {
    extern __shared__ TreeEntry sprog[];
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const TreeTile tile = tiles[t];
        const TreeSeg sg = segs[tile.seg];
        __syncthreads();
        for (int i = threadIdx.x; i < sg.prog_len; i += blockDim.x) sprog[i] = prog[sg.prog_begin + i];
        __syncthreads();
        for (long long col = threadIdx.x; col < tile.n; col += blockDim.x) {
            const long long e = sg.off + tile.start + col;
            T stk[kMaxTreeDepth];
            T top = (T)0;
            int sp = 0;
            for (int k = 0; k < sg.prog_len; k++) {
                const TreeEntry q = sprog[k];
                const T v = *(const T*)(in + (long long)q.rank * in_stride + (e + q.shift) * (long long)sizeof(T));
                if (k > 0) stk[sp++] = top;
                top = v;
                for (int a = q.adds; a > 0; a--) top = add_exact<T>(stk[--sp], top);
            }
            if (sg.rank < 0) {
                for (int d = 0; d < P; d++) *(T*)(out + (long long)d * out_stride + e * (long long)sizeof(T)) = top;
            } else {
                *(T*)(out + (long long)sg.rank * out_stride + e * (long long)sizeof(T)) = top;
            }
        }
    }
}

// ----------------------------------------------------------------- copies
enum CopyMode { kCopyAllgather = 0, kCopyBcast = 1, kCopyAlltoall = 2, kCopyScatter = 3, kCopyGather = 4 };

// A copy collective is a set of "pairs" (source row piece, destination row
// pieces) of `unit` bytes each; unit = one rank's block.
struct CopyArgs {
    const char* in;
    long long in_stride;
    char* out;
    long long out_stride;
    int P;
    int root;
    long long unit;  // bytes per block
    int dgroups;     // allgather / bcast: destination groups per source vector (>= 1)
};

template <int MODE>
__device__ __forceinline__ long long copy_pairs(const CopyArgs& a) {
    if (MODE == kCopyAlltoall) return (long long)a.P * a.P;
    if (MODE == kCopyBcast) return 1;
    return a.P;
}

// Source of pair `i` and its destinations (first and count; bcast and
// allgather broadcast one load to several rows).
template <int MODE>
__device__ __forceinline__ const char* copy_src(const CopyArgs& a, long long i) {
    if (MODE == kCopyAllgather) return a.in + i * a.in_stride;
    if (MODE == kCopyBcast) return a.in + (long long)a.root * a.in_stride;
    if (MODE == kCopyAlltoall) {
        long long src = i / a.P, dst = i % a.P;  // block dst of row src
        return a.in + src * a.in_stride + dst * a.unit;
    }
    if (MODE == kCopyScatter) return a.in + (long long)a.root * a.in_stride + i * a.unit;
    return a.in + i * a.in_stride;  // gather
}
template <int MODE>
__device__ __forceinline__ int copy_ndst(const CopyArgs& a) {
    if (MODE == kCopyAllgather) return a.P;
    if (MODE == kCopyBcast) return a.P;
    return 1;
}
// Allgather and bcast calls with few source vectors split each vector's
// destinations over `dgroups` threads (each loads the vector and stores to
// its share of the rows), so that small calls still fill the GPU.
template <int MODE>
__device__ __forceinline__ int copy_groups(const CopyArgs& a) {
    return (MODE == kCopyAllgather || MODE == kCopyBcast) ? max(1, a.dgroups) : 1;
}
template <int MODE>
__device__ __forceinline__ char* copy_dst(const CopyArgs& a, long long i, int d) {
    if (MODE == kCopyAllgather) return a.out + (long long)d * a.out_stride + i * a.unit;
    if (MODE == kCopyBcast) return d == a.root ? nullptr : a.out + (long long)d * a.out_stride;
    if (MODE == kCopyAlltoall) {
        long long src = i / a.P, dst = i % a.P;
        return a.out + dst * a.out_stride + src * a.unit;
    }
    if (MODE == kCopyScatter) return a.out + i * a.out_stride;
    return a.out + (long long)a.root * a.out_stride + i * a.unit;  // gather
}

template <int MODE>
__global__ void __launch_bounds__(kThreads) k_copy_vec(CopyArgs a) {
    const long long nvec = a.unit / 16;
    const long long step = (long long)gridDim.x * blockDim.x;
    if constexpr (MODE == kCopyAllgather || MODE == kCopyBcast) {
        const int G = copy_groups<MODE>(a);
        const long long per = copy_pairs<MODE>(a) * nvec, total = per * G;
        for (long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x; w < total; w += step) {
            const long long gi = G == 1 ? 0 : w / per, r = w - gi * per;
            const long long i = r / nvec, j = r - i * nvec;
            const uint4 v = ld_stream(copy_src<MODE>(a, i) + j * 16);
            const int nd = copy_ndst<MODE>(a);
            const int d0 = (int)(nd * gi / G), d1 = (int)(nd * (gi + 1) / G);
            for (int d = d0; d < d1; d++) {
                char* q = copy_dst<MODE>(a, i, d);
                if (q) st_stream(q + j * 16, v);
            }
        }
    } else {  // one destination per source vector
        const long long total = copy_pairs<MODE>(a) * nvec;
        for (long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x; w < total; w += step) {
            const long long i = w / nvec, j = w - (w / nvec) * nvec;
            st_stream(copy_dst<MODE>(a, i, 0) + j * 16, ld_stream(copy_src<MODE>(a, i) + j * 16));
        }
    }
}

template <int MODE, typename U>
__global__ void __launch_bounds__(kThreads) k_copy_scalar(CopyArgs a) {
    const long long nu = a.unit / (long long)sizeof(U);
    const int G = copy_groups<MODE>(a);
    const long long per = copy_pairs<MODE>(a) * nu, total = per * G;
    const long long step = (long long)gridDim.x * blockDim.x;
    for (long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x; w < total; w += step) {
        const long long gi = G == 1 ? 0 : w / per, r = w - gi * per;
        const long long i = r / nu, j = r - i * nu;
        const U v = *(const U*)(copy_src<MODE>(a, i) + j * sizeof(U));
        const int nd = copy_ndst<MODE>(a);
        const int d0 = (int)(nd * gi / G), d1 = (int)(nd * (gi + 1) / G);
        for (int d = d0; d < d1; d++) {
            char* q = copy_dst<MODE>(a, i, d);
            if (q) *(U*)(q + j * sizeof(U)) = v;
        }
    }
}

// ------------------------------------------------------------- step engine
struct StepMove {
    int64_t dst_off, a_off, b_off;  // elements
    int32_t dst_rank, a_rank, b_rank;
    uint8_t dst_buf, a_buf, b_buf, add;
};
struct StepChunk {  // elements [start, start + n) of move `move`
    int32_t move, pad;
    int64_t start, n;
};
struct StepBufs {
    char* base[3];       // send, receive, workspace
    long long stride[3];  // bytes between rank rows
};

enum StepStatus { kStepOk = 0, kStepTimeout = 1 };

__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Grid-wide barrier for a cooperative launch.  bar[0] counts arrivals,
// bar[1] is the generation; the last of `expected` arrivals (normally
// gridDim.x) opens it.  The wait is bounded by `timeout_ns` of %globaltimer
// and by an iteration cap; on expiry the block records kStepTimeout in
// *status and returns false (the caller then exits, so the other blocks time
// out too instead of waiting forever).
__device__ __forceinline__ bool grid_barrier(unsigned* bar, int* status, unsigned long long timeout_ns,
                                             unsigned expected) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        __threadfence();
        const unsigned gen = ld_acquire(&bar[1]);
        const unsigned arrived = atomicAdd(&bar[0], 1u);
        if (arrived == expected - 1) {
            bar[0] = 0;
            __threadfence();
            st_release(&bar[1], gen + 1);
        } else {
            const unsigned long long t0 = globaltimer_ns();
            unsigned long long iters = 0;
            while (ld_acquire(&bar[1]) == gen) {
                if (++iters > (1ull << 40) || globaltimer_ns() - t0 > timeout_ns ||
                    *(volatile int*)status != kStepOk) {
                    atomicCAS(status, kStepOk, kStepTimeout);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return ok != 0;
}

template <typename T>
__device__ __forceinline__ void run_chunk(const StepBufs& B, const StepMove& m, const StepChunk& ch) {
    constexpr long long es = sizeof(T);
    char* d = B.base[m.dst_buf] + (long long)m.dst_rank * B.stride[m.dst_buf] + (m.dst_off + ch.start) * es;
    const char* a = B.base[m.a_buf] + (long long)m.a_rank * B.stride[m.a_buf] + (m.a_off + ch.start) * es;
    const char* b = B.base[m.b_buf] + (long long)m.b_rank * B.stride[m.b_buf] + (m.b_off + ch.start) * es;
    const long long bytes = ch.n * es;
    const bool vec = (((uintptr_t)d | (uintptr_t)a | (uintptr_t)(m.add ? b : a)) & 15) == 0 && (bytes & 15) == 0;
    if (vec) {
        const long long nv = bytes / 16;
        for (long long i = threadIdx.x; i < nv; i += blockDim.x) {
            // Plain (coherent) loads: earlier levels of this launch wrote
            // these rows.
            uint4 v = ld_plain(a + i * 16);
            if (m.add) v = vadd<T>(v, ld_plain(b + i * 16));
            *(uint4*)(d + i * 16) = v;
        }
    } else {
        for (long long i = threadIdx.x; i < ch.n; i += blockDim.x) {
            T v = ((volatile const T*)a)[i];
            if (m.add) v = add_exact<T>(v, ((volatile const T*)b)[i]);
            ((T*)d)[i] = v;
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_steps(StepBufs B, const StepMove* __restrict__ moves,
                                                    const StepChunk* __restrict__ chunks,
                                                    const int* __restrict__ level_begin, int nlevels,
                                                    unsigned* bar, int* status, unsigned long long timeout_ns,
                                                    unsigned expected) {
    for (int l = 0; l < nlevels; l++) {
        for (int c = level_begin[l] + blockIdx.x; c < level_begin[l + 1]; c += gridDim.x) {
            const StepChunk ch = chunks[c];
            run_chunk<T>(B, moves[ch.move], ch);
        }
        if (l + 1 < nlevels && !grid_barrier(bar, status, timeout_ns, expected)) return;
    }
}

// ------------------------------------------------- pipelined step engine
// The schedule as a dataflow of items (packed segments of moves, one level
// each; built on the host by build_flow).  Blocks take items in index order
// from a global counter and run each one once the items it depends on are
// done, so a segment moves on to the next step as soon as the segments it
// reads and overwrites are ready: steps overlap, ports proceed
// independently, and no block waits for the slowest block of a level.
//
// Dependencies only point to earlier items, which were handed to running
// blocks before, so the waits always end; they are bounded nevertheless.
// State (zero-initialised once): done[item] holds the epoch of the call that
// completed it; ctl[0] is the next item, ctl[1] the blocks finished, ctl[2]
// the epoch of the last completed call, ctl[3 + l] the items of level l
// done.  The last block to finish resets the counters and advances the
// epoch, so consecutive launches need no memset.
struct FlowItem {
    int32_t pbeg, pend, dbeg, dend, level, pad;
};
constexpr int kFlowThreads = 256;                 // threads per block of k_flow
constexpr int kFlowBlocksPerSm = 1024 / kFlowThreads;  // resident blocks at 64 registers
constexpr int kFlowPieces = kFlowThreads;         // pieces per item, at most one per thread
constexpr int kFlowUnroll = 4;    // 16-byte units in flight per thread

__device__ __forceinline__ bool flow_wait(int dep, const unsigned* done, const unsigned* ctl,
                                          const int* level_items, unsigned target, unsigned extra, int* status,
                                          unsigned long long timeout_ns) {
    const bool item = dep >= 0;
    const unsigned* p = item ? &done[dep] : &ctl[3 + (-dep - 1)];
    const unsigned need = item ? target + extra : (unsigned)level_items[-dep - 1] + extra;
    if (item ? ld_acquire(p) == need : ld_acquire(p) >= need) return true;
    const unsigned long long t0 = globaltimer_ns();
    for (unsigned long long iters = 0;; iters++) {
        const unsigned v = ld_acquire(p);
        if (item ? v == need : v >= need) return true;
        if (iters > (1ull << 40) || globaltimer_ns() - t0 > timeout_ns || *(volatile int*)status != kStepOk) {
            atomicCAS(status, kStepOk, kStepTimeout);
            return false;
        }
        __nanosleep(32);
    }
}

__device__ __forceinline__ void red_release_add(unsigned* p, unsigned v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Completion is a release store after the block barrier (release is
// cumulative over the block's writes), read with acquire loads.
template <typename T>
__global__ void __launch_bounds__(kFlowThreads, kFlowBlocksPerSm) k_flow(StepBufs B, const StepMove* __restrict__ moves,
                                                      const StepChunk* __restrict__ pieces,
                                                      const FlowItem* __restrict__ items, int nitems,
                                                      const int* __restrict__ deps,
                                                      const int* __restrict__ level_items, int nlevels,
                                                      unsigned* done, unsigned* ctl, int* status,
                                                      unsigned long long timeout_ns, unsigned extra) {
    __shared__ long long s_pref[kFlowPieces + 1];  // first unit of each piece
    __shared__ char* s_d[kFlowPieces];
    __shared__ const char* s_a[kFlowPieces];
    __shared__ const char* s_b[kFlowPieces];
    __shared__ long long s_nvec[kFlowPieces];      // 16-byte units of the body
    __shared__ unsigned char s_head[kFlowPieces];  // element units before the body
    __shared__ unsigned char s_add[kFlowPieces];
    __shared__ long long s_warp[kFlowThreads / 32];
    __shared__ int s_item, s_ok;
    __shared__ unsigned s_target;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        const unsigned t = ld_acquire(&ctl[2]) + 1u;
        s_target = t == 0 ? 1u : t;  // 0 is the initial value of done[]
    }
    __syncthreads();
    const unsigned target = s_target;
    constexpr long long es = sizeof(T);
    for (;;) {
        if (tid == 0) s_item = *(volatile int*)status == kStepOk ? (int)atomicAdd(&ctl[0], 1u) : nitems;
        __syncthreads();
        const int i = s_item;
        if (i >= nitems) break;
        const FlowItem it = items[i];
        // Piece table (addresses; element head, 16-byte body and element
        // tail; tables only, no data rows) and a block scan of the unit
        // counts, both before the dependency wait, so that they are off the
        // critical path.  A piece whose destination and sources sit at the same
        // offset within 16 bytes gets a vector body; any other piece is
        // all element units.
        const int np = it.pend - it.pbeg;
        long long units = 0;
        if (tid < np) {
            const StepChunk ch = pieces[it.pbeg + tid];
            const StepMove m = moves[ch.move];
            char* d = B.base[m.dst_buf] + (long long)m.dst_rank * B.stride[m.dst_buf] + (m.dst_off + ch.start) * es;
            const char* a = B.base[m.a_buf] + (long long)m.a_rank * B.stride[m.a_buf] + (m.a_off + ch.start) * es;
            const char* b = B.base[m.b_buf] + (long long)m.b_rank * B.stride[m.b_buf] + (m.b_off + ch.start) * es;
            const uintptr_t mis = ((uintptr_t)d ^ (uintptr_t)a) | (m.add ? ((uintptr_t)d ^ (uintptr_t)b) : 0);
            const long long n = ch.n;
            long long head = n, nvec = 0;
            if ((mis & 15) == 0) {
                head = min((long long)((16 - ((uintptr_t)d & 15)) & 15) / es, n);
                nvec = (n - head) * es / 16;
            }
            units = n - nvec * (16 / es) + nvec;
            s_d[tid] = d;
            s_a[tid] = a;
            s_b[tid] = b;
            s_nvec[tid] = nvec;
            s_head[tid] = (unsigned char)min(head, 255ll);
            s_add[tid] = m.add ? 1 : 0;
        }
        long long inc = units;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const long long v = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += v;
        }
        if (lane == 31) s_warp[warp] = inc;
        __syncthreads();
        long long before = 0;
        for (int w = 0; w < warp; w++) before += s_warp[w];
        s_pref[tid + 1] = before + inc;
        if (tid == 0) s_pref[0] = 0;
        // The dependency wait comes last, so that only one block barrier
        // separates the last dependency's completion from this item's loads.
        if (warp == 0) {
            bool ok = true;
            for (int d = it.dbeg + lane; d < it.dend && ok; d += 32)
                ok = flow_wait(deps[d], done, ctl, level_items, target, extra, status, timeout_ns);
            ok = __all_sync(0xffffffffu, ok);
            if (lane == 0) s_ok = ok;
        }
        __syncthreads();
        if (!s_ok) break;  // a wait expired; the status is recorded
        const long long total = s_pref[np];
        int cur = 0;
        for (long long u0 = tid; u0 < total; u0 += (long long)kFlowUnroll * kFlowThreads) {
            uint4 va[kFlowUnroll], vb[kFlowUnroll];  // a vector, or an element in the low bytes
            char* dp[kFlowUnroll];
            int kind[kFlowUnroll];  // -1: none; bit 0: add, bit 1: vector
#pragma unroll
            for (int k = 0; k < kFlowUnroll; k++) {
                const long long u = u0 + (long long)k * kFlowThreads;
                kind[k] = -1;
                if (u < total) {
                    if (!(u >= s_pref[cur] && u < s_pref[cur + 1])) {
                        int lo = 0, hi = np - 1;  // last piece starting at or before u
                        while (lo < hi) {
                            const int mid = (lo + hi + 1) >> 1;
                            if (s_pref[mid] <= u) lo = mid; else hi = mid - 1;
                        }
                        cur = lo;
                    }
                    const long long r = u - s_pref[cur];
                    const long long head = s_head[cur], nvec = s_nvec[cur];
                    const int add = s_add[cur];
                    // Plain (coherent) loads: other blocks wrote these rows
                    // during this launch.
                    if (r >= head && r < head + nvec) {
                        const long long off = head * es + (r - head) * 16;
                        kind[k] = add | 2;
                        dp[k] = s_d[cur] + off;
                        va[k] = ld_plain(s_a[cur] + off);
                        if (add) vb[k] = ld_plain(s_b[cur] + off);
                    } else {
                        const long long e = r < head ? r : r - nvec + nvec * (16 / es);
                        kind[k] = add;
                        dp[k] = s_d[cur] + e * es;
                        *(T*)&va[k] = *((volatile const T*)s_a[cur] + e);
                        if (add) *(T*)&vb[k] = *((volatile const T*)s_b[cur] + e);
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < kFlowUnroll; k++) {
                if (kind[k] < 0) continue;
                if (kind[k] & 2)
                    *(uint4*)dp[k] = (kind[k] & 1) ? vadd<T>(va[k], vb[k]) : va[k];
                else
                    *(T*)dp[k] = (kind[k] & 1) ? add_exact<T>(*(const T*)&va[k], *(const T*)&vb[k]) : *(const T*)&va[k];
            }
        }
        __syncthreads();
        if (tid == 0) {
            st_release(&done[i], target);
            red_release_add(&ctl[3 + it.level], 1u);
        }
    }
    __syncthreads();
    if (tid == 0) {
        __threadfence();
        if (atomicAdd(&ctl[1], 1u) == gridDim.x - 1) {
            ctl[0] = 0;
            ctl[1] = 0;
            for (int l = 0; l < nlevels; l++) ctl[3 + l] = 0;
            __threadfence();
            st_release(&ctl[2], target);
        }
    }
}

// ------------------------------------------- pipelined engine, fused passes
// The same dataflow driver as k_flow over a fused schedule (level fusion,
// bine_plan.h): a piece belongs to a fused move whose value is a postfix
// program over at most kFuseLeaves state elements, written to at most
// kFuseDsts destinations.  Each unit (a 16-byte vector, or an element at a
// piece's unaligned head and tail) loads all of its leaves, evaluates the
// program on a four-entry stack (the top in registers, the rest in shared
// memory for 16-byte units) in the order of the original levels'
// additions, and stores the value to every destination; the loads
// come before the stores, so a move may update its own elements in place.
// Items of copies only (one leaf per program: the gather and alltoall
// passes) move four 16-byte units per thread and round, other items one
// unit with all its leaves in flight.  Three blocks of 256 threads per SM
// (80 registers): the planner cuts each pass into a whole multiple of the
// resident blocks' count of equal-traffic items.
struct FusedMoveDev {
    int64_t n;
    int32_t leaf_begin, nleaves, dst_begin, ndst;
};
struct FusedLeafDev {
    int32_t rank;
    uint8_t buf, adds, pad[2];
    int64_t off;
};
struct FusedDstDev {
    int32_t rank;
    uint8_t buf, pad[3];
    int64_t off;
};
constexpr int kFuseLeaves = 8;
constexpr int kFuseDsts = 8;
constexpr int kFusedPieces = 128;  // pieces per item, at most one per thread
static_assert(kFusedPieces <= kFlowThreads, "one thread per piece of an item");

// Postfix evaluation of at most L leaves on a shift-register stack (s0 is
// the top): a leaf pushes, each addition pops the top two and pushes their
// sum.  IEEE and wrapping integer addition are commutative, so only the
// tree's shape matters, and it is the program's.
template <int L, typename V, typename Add>
__device__ __forceinline__ V fused_eval(const V* v, const unsigned char* adds, int nl, Add add) {
    V s0 = v[0], s1 = v[0], s2 = v[0], s3 = v[0];
#pragma unroll
    for (int j = 1; j < L; j++) {
        if (j < nl) {
            s3 = s2;
            s2 = s1;
            s1 = s0;
            s0 = v[j];
            const int na = adds[j];
#pragma unroll
            for (int a = 0; a < 3; a++)
                if (a < na) {
                    s0 = add(s1, s0);
                    s1 = s2;
                    s2 = s3;
                }
        }
    }
    return s0;
}

// Per-item tables of k_flow_fused: every piece's leaf and destination
// addresses, its evaluation program, and block scans of its 16-byte units
// and of its element units (an unaligned head and tail, or the whole piece
// when its rows are not mutually 16-byte aligned).  The planner keeps an
// item below 2^31 elements, so unit counts fit 32 bits.
struct FusedItemSmem {
    int pref[kFusedPieces + 1];   // first 16-byte unit of each piece
    int epref[kFusedPieces + 1];  // first element unit of each piece
    const char* leaf[kFusedPieces][kFuseLeaves];
    char* dst[kFusedPieces][kFuseDsts];
    long long start[kFusedPieces], n[kFusedPieces];
    int nvec[kFusedPieces], lb[kFusedPieces], db[kFusedPieces];
    unsigned char adds[kFusedPieces][kFuseLeaves];
    unsigned char head[kFusedPieces], nl[kFusedPieces], nd[kFusedPieces];
    uint4 stk[3][kFlowThreads];  // evaluation stack below the top (depth <= 4), per thread
    char* base[3];               // the launch's buffer rows (StepBufs), read from shared memory
    long long stride[3];
    long long warp_sum[kFlowThreads / 32];
    int item, ok, maxnl;
    unsigned target;
};

// Last piece of the item whose units (prefix table pref) start at or
// before unit u; cur is the guess.
__device__ __forceinline__ int fused_piece(const int* pref, int u, int np, int cur) {
    if (u >= pref[cur] && u < pref[cur + 1]) return cur;
    int lo = 0, hi = np - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pref[mid] <= u) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// The 16-byte units of an item whose programs have at most L leaves (L = 1:
// copies; L = 2: single additions): U units per thread and round, every
// unit's loads issued before the round's stores.  Units of one item touch
// disjoint elements apart from a move's in-place reads of its own elements,
// so the order of rounds and units does not matter.
template <typename T, int U, int L>
__device__ __forceinline__ void fused_units_narrow(const FusedItemSmem& S, int tid, int total, int np) {
    static_assert(L == 1 || L == 2, "narrow programs only");
    constexpr int es = sizeof(T);
    int cur = 0;
    for (int u0 = tid; u0 < total; u0 += U * kFlowThreads) {
        uint4 v[U][L];
        int pc[U], off[U];
#pragma unroll
        for (int k = 0; k < U; k++) {
            const int u = u0 + k * kFlowThreads;
            pc[k] = -1;
            off[k] = 0;
            if (u < total) {
                cur = fused_piece(S.pref, u, np, cur);
                pc[k] = cur;
                off[k] = S.head[cur] * es + (u - S.pref[cur]) * 16;
                v[k][0] = ld_plain(S.leaf[cur][0] + off[k]);
                if (L == 2 && S.nl[cur] == 2) v[k][L - 1] = ld_plain(S.leaf[cur][L - 1] + off[k]);
            }
        }
#pragma unroll
        for (int k = 0; k < U; k++) {
            if (pc[k] < 0) continue;
            const int p = pc[k];
            const uint4 val = (L == 2 && S.nl[p] == 2) ? vadd<T>(v[k][0], v[k][L - 1]) : v[k][0];
            const int nd = S.nd[p];
#pragma unroll
            for (int j = 0; j < kFuseDsts; j++)
                if (j < nd) *(uint4*)(S.dst[p][j] + off[k]) = val;
        }
    }
}

// The 16-byte units of any item: one unit per thread and round, its leaves
// loaded together, the program evaluated with the entries below the top of
// its stack in this thread's column of S.stk (registers would cost the
// third block per SM).
template <typename T>
__device__ __forceinline__ void fused_units_wide(FusedItemSmem& S, int tid, int total, int np) {
    constexpr int es = sizeof(T);
    int cur = 0;
    for (int u = tid; u < total; u += kFlowThreads) {
        cur = fused_piece(S.pref, u, np, cur);
        const int off = S.head[cur] * es + (u - S.pref[cur]) * 16;
        const int nl = S.nl[cur], nd = S.nd[cur];
        uint4 v[kFuseLeaves];
#pragma unroll
        for (int j = 0; j < kFuseLeaves; j++)
            if (j < nl) v[j] = ld_plain(S.leaf[cur][j] + off);
        uint4 top = v[0];
        int sp = 0;
#pragma unroll
        for (int j = 1; j < kFuseLeaves; j++)
            if (j < nl) {
                S.stk[sp++][tid] = top;
                top = v[j];
                for (int a = S.adds[cur][j]; a > 0; a--) top = vadd<T>(S.stk[--sp][tid], top);
            }
#pragma unroll
        for (int j = 0; j < kFuseDsts; j++)
            if (j < nd) *(uint4*)(S.dst[cur][j] + off) = top;
    }
}

// The element units of an item: a piece's unaligned head, its tail after
// the 16-byte body, or all of a piece without one.
template <typename T>
__device__ __forceinline__ void fused_elements(const FusedItemSmem& S, int tid, int total, int np) {
    constexpr int per_vec = 16 / sizeof(T);
    int cur = 0;
    for (int u = tid; u < total; u += kFlowThreads) {
        cur = fused_piece(S.epref, u, np, cur);
        const long long r = u - S.epref[cur];
        const long long e = r < S.head[cur] ? r : r + (long long)S.nvec[cur] * per_vec;
        const int nl = S.nl[cur], nd = S.nd[cur];
        T w[kFuseLeaves];
#pragma unroll
        for (int j = 0; j < kFuseLeaves; j++)
            if (j < nl) w[j] = *((volatile const T*)S.leaf[cur][j] + e);
        const T val = fused_eval<kFuseLeaves>(w, S.adds[cur], nl, [](T x, T y) { return add_exact<T>(x, y); });
#pragma unroll
        for (int j = 0; j < kFuseDsts; j++)
            if (j < nd) *((T*)S.dst[cur][j] + e) = val;
    }
}

template <typename T>
__global__ void __launch_bounds__(kFlowThreads, 3) k_flow_fused(StepBufs B, const FusedMoveDev* __restrict__ moves,
                                                            const FusedLeafDev* __restrict__ leaves,
                                                            const FusedDstDev* __restrict__ dsts,
                                                            const StepChunk* __restrict__ pieces,
                                                            const FlowItem* __restrict__ items, int nitems,
                                                            const int* __restrict__ deps,
                                                            const int* __restrict__ level_items, int nlevels,
                                                            unsigned* done, unsigned* ctl, int* status,
                                                            unsigned long long timeout_ns, unsigned extra) {
    __shared__ FusedItemSmem S;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        const unsigned t = ld_acquire(&ctl[2]) + 1u;
        S.target = t == 0 ? 1u : t;
    }
    if (tid < 3) {
        S.base[tid] = B.base[tid];
        S.stride[tid] = B.stride[tid];
    }
    __syncthreads();
    const unsigned target = S.target;
    constexpr long long es = sizeof(T);
    constexpr int kSlots = kFuseLeaves + kFuseDsts;
    for (;;) {
        if (tid == 0) {
            S.item = *(volatile int*)status == kStepOk ? (int)atomicAdd(&ctl[0], 1u) : nitems;
            S.maxnl = 1;
        }
        __syncthreads();
        const int i = S.item;
        if (i >= nitems) break;
        const FlowItem it = items[i];
        const int np = it.pend - it.pbeg;  // at most kFusedPieces (the planner's bound)
        // The item's tables in three rounds of independent loads, all before
        // the dependency wait: pieces and moves, then every leaf and
        // destination address, then each piece's vector body and units.
        if (tid < np) {
            const StepChunk ch = pieces[it.pbeg + tid];
            const FusedMoveDev m = moves[ch.move];
            S.start[tid] = ch.start;
            S.n[tid] = ch.n;
            S.lb[tid] = m.leaf_begin;
            S.db[tid] = m.dst_begin;
            S.nl[tid] = (unsigned char)m.nleaves;
            S.nd[tid] = (unsigned char)m.ndst;
            atomicMax(&S.maxnl, m.nleaves);
        }
        __syncthreads();
#pragma unroll 4
        for (int e = tid; e < np * kSlots; e += kFlowThreads) {
            const int p = e / kSlots, j = e % kSlots;
            if (j < kFuseLeaves) {
                if (j < S.nl[p]) {
                    const FusedLeafDev lf = leaves[S.lb[p] + j];
                    S.leaf[p][j] =
                        S.base[lf.buf] + (long long)lf.rank * S.stride[lf.buf] + (lf.off + S.start[p]) * es;
                    S.adds[p][j] = lf.adds;
                }
            } else if (j - kFuseLeaves < S.nd[p]) {
                const FusedDstDev d = dsts[S.db[p] + j - kFuseLeaves];
                S.dst[p][j - kFuseLeaves] =
                    S.base[d.buf] + (long long)d.rank * S.stride[d.buf] + (d.off + S.start[p]) * es;
            }
        }
        __syncthreads();
        // Both unit counts in one scan: element units in the high half.
        long long units = 0;
        if (tid < np) {
            const uintptr_t first = (uintptr_t)S.leaf[tid][0];
            uintptr_t mis = 0;
            for (int j = 1; j < S.nl[tid]; j++) mis |= (uintptr_t)S.leaf[tid][j] ^ first;
            for (int j = 0; j < S.nd[tid]; j++) mis |= (uintptr_t)S.dst[tid][j] ^ first;
            const long long n = S.n[tid];
            long long head = 0, nvec = 0;
            if ((mis & 15) == 0) {
                head = min((long long)((16 - (first & 15)) & 15) / es, n);
                nvec = (n - head) * es / 16;
            }
            units = ((n - nvec * (16 / es)) << 32) | nvec;
            S.nvec[tid] = (int)nvec;
            S.head[tid] = (unsigned char)head;
        }
        long long inc = units;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const long long v = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += v;
        }
        if (lane == 31) S.warp_sum[warp] = inc;
        __syncthreads();
        long long before = 0;
        for (int w = 0; w < warp; w++) before += S.warp_sum[w];
        if (tid < kFusedPieces) {
            S.pref[tid + 1] = (int)((before + inc) & 0xffffffffll);
            S.epref[tid + 1] = (int)((before + inc) >> 32);
        }
        if (tid == 0) S.pref[0] = S.epref[0] = 0;
        if (warp == 0) {
            bool ok = true;
            for (int d = it.dbeg + lane; d < it.dend && ok; d += 32)
                ok = flow_wait(deps[d], done, ctl, level_items, target, extra, status, timeout_ns);
            ok = __all_sync(0xffffffffu, ok);
            if (lane == 0) S.ok = ok;
        }
        __syncthreads();
        if (!S.ok) break;  // a wait expired; the status is recorded
        const int total = S.pref[np];
        const int maxnl = S.maxnl;
        if (maxnl <= 1)
            fused_units_narrow<T, 4, 1>(S, tid, total, np);
        else
            fused_units_wide<T>(S, tid, total, np);
        if (S.epref[np] > 0) fused_elements<T>(S, tid, S.epref[np], np);
        __syncthreads();
        if (tid == 0) {
            st_release(&done[i], target);
            red_release_add(&ctl[3 + it.level], 1u);
        }
    }
    __syncthreads();
    if (tid == 0) {
        __threadfence();
        if (atomicAdd(&ctl[1], 1u) == gridDim.x - 1) {
            ctl[0] = 0;
            ctl[1] = 0;
            for (int l = 0; l < nlevels; l++) ctl[3 + l] = 0;
            __threadfence();
            st_release(&ctl[2], target);
        }
    }
}

}  // namespace dev
}  // namespace bine

// ------------------------------------------------------ torus link bytes
// Per-link byte accounting of a schedule on the communicator's torus.  A
// message takes the dimension-ordered route, minimal on each ring, the +
// direction on ties (Bine and recursive-doubling peers differ in one
// coordinate; 1-D algorithms on a torus may differ in several).  Link (node, d, dir) has index (node*ndims + d)*2 + dir
// (dir 0: +, 1: -).  Each message adds its bytes to a cyclic range of link
// positions on one ring, recorded as two or three signed updates of a
// difference array (unsigned wrap-around arithmetic, exact mod 2^64); one
// prefix scan per ring then yields the counts.  Cost: O(messages + links)
// instead of O(messages * hops).
#include "bine_sched.h"

namespace bine {
namespace dev {

__device__ __forceinline__ size_t link_index(const Torus& t, int node, int d, int dir) {
    return ((size_t)node * t.ndims + d) * 2 + dir;
}

// Adds `bytes` to the links of the route src -> dst: dimension-ordered
// (dimension 0 first), minimal in each dimension, + direction on ties.
__device__ __forceinline__ void add_route(const Torus& t, int src, int dst, unsigned long long bytes,
                                          unsigned long long* diff) {
    if (src == dst || bytes == 0) return;
    int a[kMaxDims] = {0, 0, 0}, b[kMaxDims] = {0, 0, 0};
    t.coords(src, a);
    t.coords(dst, b);
    int c[kMaxDims] = {a[0], a[1], a[2]};
    const unsigned long long neg = 0ull - bytes;
    for (int d = 0; d < t.ndims; d++) {
        if (c[d] == b[d]) continue;
        const int L = t.dims[d];
        const int delta = pmod(b[d] - c[d], L);
        int dir = 0, start = c[d], hops = delta;
        if (L - delta < delta) {  // minus direction: positions c-h+1 .. c
            dir = 1;
            hops = L - delta;
            start = pmod(c[d] - hops + 1, L);
        }
        auto at = [&](int pos) {
            int q[kMaxDims] = {c[0], c[1], c[2]};
            q[d] = pos;
            return link_index(t, t.id(q), d, dir);
        };
        const int end = start + hops;  // exclusive
        atomicAdd(&diff[at(start)], bytes);
        if (end < L) {
            atomicAdd(&diff[at(end)], neg);
        } else if (end > L) {  // wraps: [start, L) and [0, end - L)
            atomicAdd(&diff[at(0)], bytes);
            atomicAdd(&diff[at(end - L)], neg);
        }
        c[d] = b[d];
    }
}

// One thread per message (src, dst, elements) of a host-planned schedule.
__global__ void k_link_from_msgs(Torus t, const long long* __restrict__ msgs, long long n, int es,
                                 unsigned long long* diff) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        add_route(t, (int)msgs[4 * i + 1], (int)msgs[4 * i + 2], (unsigned long long)msgs[4 * i + 3] * es, diff);
}

struct LinkGen {
    Torus t;
    int family, ports, kind;  // kind 0: bandwidth-optimal allreduce, 1: latency-optimal allreduce,
                              //      2: contiguous allgather (distance halving)
    long long count;          // the collective's count argument
    int es;
};

// One thread per (rank, port): generates the messages of the schedule
// directly from the step math (power-of-two torus dimensions only, where
// every binomial tree visits each rank once).
//   kind 0: the reduce-scatter message of rank r at step i carries the
//   blocks of the subtree reached through peer_i(r) with later steps (the
//   blocks whose block_step is i); the allgather sends the same volume back.
//   kind 1: the full port slice to peer_i(r) at every step.
//   kind 2: 2^s blocks to peer_{S-1-s}(r) at step s.
__global__ void k_link_generate(LinkGen g, unsigned long long* diff) {
    const long long total = (long long)g.t.size * g.ports;
    for (long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x; w < total; w += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(w / g.ports), port = (int)(w % g.ports);
        StepDim sd[kMaxSteps];
        step_dims(g.t, port, sd);
        const int S = g.t.num_steps, P = g.t.size;
        const long long cp = g.count / g.ports + (port < g.count % g.ports ? 1 : 0);
        if (g.kind == 1) {
            for (int i = 0; i < S; i++)
                add_route(g.t, r, step_peer_rank(g.t, sd, i, port, g.family, r), (unsigned long long)cp * g.es, diff);
            continue;
        }
        if (g.kind == 2) {
            // Allgather blocks: by block, then port (count per block = count).
            const long long b0 = g.count / g.ports + (port < g.count % g.ports ? 1 : 0);
            for (int s = 0; s < S; s++)
                add_route(g.t, r, step_peer_rank(g.t, sd, S - 1 - s, port, g.family, r),
                          ((unsigned long long)1 << s) * b0 * g.es, diff);
            continue;
        }
        const long long q = cp / P, rem = cp % P;
        for (int i = 0; i < S; i++) {
            const int child = step_peer_rank(g.t, sd, i, port, g.family, r);
            // Iterative walk of child's subtree along steps > i.
            int stk_node[kMaxSteps * (kMaxSteps + 1) / 2 + 1];
            int8_t stk_step[kMaxSteps * (kMaxSteps + 1) / 2 + 1];
            int sp = 0;
            stk_node[sp] = child;
            stk_step[sp++] = (int8_t)(i + 1);
            unsigned long long elems = 0;
            while (sp > 0) {
                const int node = stk_node[--sp];
                const int st = stk_step[sp];
                elems += (unsigned long long)(q + (node < rem ? 1 : 0));
                for (int j = st; j < S; j++) {
                    stk_node[sp] = step_peer_rank(g.t, sd, j, port, g.family, node);
                    stk_step[sp++] = (int8_t)(j + 1);
                }
            }
            add_route(g.t, r, child, elems * g.es, diff);  // reduce-scatter step i
            add_route(g.t, child, r, elems * g.es, diff);  // allgather step S-1-i
        }
    }
}

// One thread per ring: prefix sums of the difference array, in place.
__global__ void k_link_scan(Torus t, unsigned long long* links) {
    long long nlines = 0;
    long long base[kMaxDims];
    for (int d = 0; d < t.ndims; d++) {
        base[d] = nlines;
        nlines += 2ll * (t.size / t.dims[d]);
    }
    for (long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x; w < nlines; w += (long long)gridDim.x * blockDim.x) {
        int d = 0;
        while (d + 1 < t.ndims && w >= base[d + 1]) d++;
        const long long k = w - base[d];
        const int dir = (int)(k & 1);
        long long line = k >> 1;  // index over the other coordinates
        int c[kMaxDims] = {0, 0, 0};
        for (int i = t.ndims - 1; i >= 0; i--) {
            if (i == d) continue;
            c[i] = (int)(line % t.dims[i]);
            line /= t.dims[i];
        }
        unsigned long long acc = 0;
        for (int p = 0; p < t.dims[d]; p++) {
            c[d] = p;
            const size_t li = link_index(t, t.id(c), d, dir);
            acc += links[li];
            links[li] = acc;
        }
    }
}

}  // namespace dev
}  // namespace bine

// --------------------------------------------------------- batched launch
// Thousands of independent allreduce / reduce_scatter / allgather calls of
// different P, sizes and element types in ONE persistent launch.  Every
// call is cut into tiles; blocks take tiles grid-stride from the global tile
// range and find their call by binary search over tile_begin.  Reduction
// tiles are `tc` 16-byte columns wide and split the P rows over 256/tc warps
// groups (tc comes from the autotuner: narrow tiles with many row groups for
// large P, wide tiles for small P); allgather tiles are 256 vectors of the
// flattened (source rank, column) space, each stored to all P rows.
// Integer sums wrap, float32 sums accumulate in FP64 (the FAST order).
namespace bine {
namespace dev {

enum BatchOp { kBatchAllreduce = 0, kBatchReduceScatter = 1, kBatchAllgather = 2 };

struct BatchItem {
    const char* in;
    char* out;
    long long in_stride, out_stride;  // bytes between rank rows
    long long ncol;                   // 16-byte vectors per input row
    long long blk;                    // reduce_scatter: vectors per destination rank
    long long tile_begin, ntiles;
    int P, op, is_float, tc;
};

template <typename T, typename A>
__device__ __forceinline__ void batch_reduce_tile(const BatchItem& it, long long tile, Lanes<float, double>* part_f,
                                                  uint4* res) {
    const int tc = it.tc, groups = kThreads / tc;
    const int lane = threadIdx.x % tc, grp = threadIdx.x / tc;
    const int per = (it.P + groups - 1) / groups;
    const int r0 = min(it.P, grp * per), r1 = min(it.P, r0 + per);
    const long long col = tile * tc + lane;
    Lanes<T, A> acc;
    acc.zero();
    if (col < it.ncol) {
        const char* p = it.in + col * 16;
        int r = r0;
        for (; r + 8 <= r1; r += 8) {
            uint4 v[8];
#pragma unroll
            for (int u = 0; u < 8; u++) v[u] = ld_stream(p + (long long)(r + u) * it.in_stride);
#pragma unroll
            for (int u = 0; u < 8; u++) acc.add(v[u]);
        }
        for (; r < r1; r++) acc.add(ld_stream(p + (long long)r * it.in_stride));
    }
    Lanes<T, A>* part = reinterpret_cast<Lanes<T, A>*>(part_f);
    part[threadIdx.x] = acc;
    __syncthreads();
    if (grp == 0) {
        Lanes<T, A> s = part[lane];
        for (int g = 1; g < groups; g++)
#pragma unroll
            for (int i = 0; i < Lanes<T, A>::N; i++) s.v[i] = add_exact<A>(s.v[i], part[g * tc + lane].v[i]);
        res[lane] = s.pack();
    }
    __syncthreads();
    if (col < it.ncol) {
        const uint4 v = res[lane];
        if (it.op == kBatchAllreduce) {
            char* q = it.out + col * 16;
            for (int d = grp; d < it.P; d += groups) st_stream(q + (long long)d * it.out_stride, v);
        } else if (grp == 0) {
            const long long owner = col / it.blk;
            st_stream(it.out + owner * it.out_stride + (col - owner * it.blk) * 16, v);
        }
    }
}

__global__ void __launch_bounds__(kThreads) k_batch(const BatchItem* __restrict__ items, int nitems,
                                                    long long total_tiles) {
    __shared__ Lanes<float, double> part[kThreads];
    __shared__ uint4 res[kThreads];
    for (long long t = blockIdx.x; t < total_tiles; t += gridDim.x) {
        int lo = 0, hi = nitems - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) / 2;
            if (items[mid].tile_begin <= t) lo = mid;
            else hi = mid - 1;
        }
        const BatchItem it = items[lo];
        const long long tile = t - it.tile_begin;
        if (it.op == kBatchAllgather) {
            const long long idx = tile * kThreads + threadIdx.x;
            if (idx < (long long)it.P * it.ncol) {
                const long long i = idx / it.ncol, j = idx - (idx / it.ncol) * it.ncol;
                const uint4 v = ld_stream(it.in + i * it.in_stride + j * 16);
                char* q = it.out + (i * it.ncol + j) * 16;
                for (int d = 0; d < it.P; d++) st_stream(q + (long long)d * it.out_stride, v);
            }
        } else if (it.is_float) {
            batch_reduce_tile<float, double>(it, tile, part, res);
        } else {
            batch_reduce_tile<int32_t, int32_t>(it, tile, part, res);
        }
        __syncthreads();
    }
}

}  // namespace dev
}  // namespace bine

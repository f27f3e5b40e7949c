// Bine schedule math shared by the host planner and the device kernels.
//
// Everything here is pure integer arithmetic on ranks, written from the
// definitions of the Bine trees:
//   * signed step distances rho_s = 1, -1, 3, -5, 11, ... (Jacobsthal-like),
//     sign flipped for odd coordinates and on mirrored ports
//     (reference: lib/libbine_common.h:27, lib/libbine_coll.cc:15-42);
//   * negabinary encodings of ranks and the "remapped rank" used by the
//     rooted collectives (lib/libbine_coll_bcast.cc:931-984,
//     lib/libbine_coll_allgather.cc:1093-1158, simulation/remap_rank.c);
//   * row-major torus coordinates (lib/libbine_common.cc:206-263).
// Two quirks of the reference are kept on purpose because they decide which
// negabinary representation is picked: the MSB test uses the DECIMAL literal
// 80000000, and btonb() rejects inputs above 0x55555555 (the host planner
// turns that into an error; it cannot occur for the rank counts supported).
#pragma once

#include <stdint.h>

#ifdef __CUDACC__
#define BINE_HD __host__ __device__ __forceinline__
#else
#define BINE_HD inline
#endif

namespace bine {

constexpr int kMaxDims = 3;
constexpr int kMaxPorts = 6;
constexpr int kMaxSteps = 20;

// rho_s and the negabinary ranges representable with s bits.
BINE_HD int rho(int s) {
    // rho_s = (1 - (-2)^(s+1)) / 3
    long long p = 1;
    for (int i = 0; i <= s; i++) p *= -2;
    return (int)((1 - p) / 3);
}
BINE_HD int nb_smallest(int nbits) {  // most negative value on nbits negabinary digits
    // All odd-position digits set: -2 * (4^floor(n/2) - 1) / 3.
    long long q = 1;
    for (int i = 0; i < nbits / 2; i++) q *= 4;
    return (int)(-2 * (q - 1) / 3);
}
BINE_HD int nb_largest(int nbits) {  // largest value on nbits negabinary digits
    long long q = 1;
    for (int i = 0; i < nbits / 2; i++) q *= 4;
    long long t = (q - 1) / 3;
    if (nbits & 1) {
        long long h = 1;
        for (int i = 0; i < nbits - 1; i++) h *= 2;
        t += h;
    }
    return (int)t;
}

BINE_HD int ceil_log2(unsigned long long x) {
    int y = 0;
    while ((1ull << y) < x) y++;
    return y;
}
BINE_HD int pmod(int a, int b) {
    int r = a % b;
    return r < 0 ? r + b : r;
}
BINE_HD bool is_pow2(long long x) { return x > 0 && (x & (x - 1)) == 0; }

// Negabinary conversions (mask trick: (0xAA..A + x) ^ 0xAA..A).
BINE_HD uint32_t to_negabinary(int32_t x) { return (0xAAAAAAAAu + (uint32_t)x) ^ 0xAAAAAAAAu; }
BINE_HD int32_t from_negabinary(uint32_t y) { return (int32_t)((0xAAAAAAAAu ^ y) - 0xAAAAAAAAu); }

BINE_HD uint32_t bit_reverse32(uint32_t x) {
#ifdef __CUDA_ARCH__
    return __brev(x);
#else
    uint32_t r = 0;
    for (int i = 0; i < 32; i++) r |= ((x >> i) & 1u) << (31 - i);
    return r;
#endif
}

BINE_HD bool nb_in_range(int x, int nbits) { return x >= nb_smallest(nbits) && x <= nb_largest(nbits); }

// Negabinary representation of a rank on a ring of `size`: the rank reached
// by a signed distance d with d == rank (mod size); the reference tries d =
// +/-rank and d = +/-rank -/+ size and keeps the one whose top digit is set.
// Returns UINT32_MAX when no representation exists.
BINE_HD uint32_t rank_negabinary(uint32_t rank, uint32_t size) {
    uint32_t a = UINT32_MAX, b = UINT32_MAX;
    int nbits = ceil_log2(size);
    int r = (int)rank, s = (int)size;
    int ca = (rank & 1) ? r : -r;
    int cb = (rank & 1) ? r - s : -r + s;
    if (nb_in_range(ca, nbits)) a = to_negabinary(ca);
    if (nb_in_range(cb, nbits)) b = to_negabinary(cb);
    if (a == UINT32_MAX) return b;
    if (b == UINT32_MAX) return a;
    return (a & (80000000u >> (32 - nbits))) ? a : b;  // decimal literal, as in the reference
}

// Gray code of the negabinary digits, bit-reversed on ceil(log2 size) bits.
BINE_HD uint32_t remap_rank(uint32_t rank, uint32_t size) {
    uint32_t nb = rank_negabinary(rank, size);
    uint32_t g = nb ^ (nb >> 1);
    return bit_reverse32(g) >> (32 - ceil_log2(size));
}

BINE_HD uint32_t nb_to_nu(uint32_t nb, uint32_t size) {
    return bit_reverse32(nb ^ (nb >> 1)) >> (32 - ceil_log2(size));
}

// "nu" block index used by the block-by-block allgather: the smaller nu of
// the two candidate representations.
BINE_HD uint32_t nu_of(uint32_t rank, uint32_t size) {
    uint32_t a = UINT32_MAX, b = UINT32_MAX;
    int nbits = ceil_log2(size);
    int r = (int)rank, s = (int)size;
    int ca = (rank & 1) ? r : -r;
    int cb = (rank & 1) ? r - s : -r + s;
    if (nb_in_range(ca, nbits)) a = to_negabinary(ca);
    if (nb_in_range(cb, nbits)) b = to_negabinary(cb);
    if (a == UINT32_MAX) return b == UINT32_MAX ? UINT32_MAX : nb_to_nu(b, size);
    if (b == UINT32_MAX) return nb_to_nu(a, size);
    uint32_t na = nb_to_nu(a, size), nbv = nb_to_nu(b, size);
    return (int)na < (int)nbv ? na : nbv;
}

// Decomposes num into XORs of Mersenne numbers 2^(k+1)-1 (largest first) and
// returns the XOR of the matching powers 2^k: the distance-halving position
// of a rank reached through a distance-doubling Bine tree.
BINE_HD int distance_doubling_position(uint32_t num) {
    int out = 0;
    while (num > 0) {
        int k = 31;
        while (!((num >> k) & 1u)) k--;
        out ^= 1 << k;
        num ^= (uint32_t)((1ull << (k + 1)) - 1);
    }
    return out;
}

// Row-major torus.
struct Torus {
    int ndims;
    int dims[kMaxDims];
    int size;
    int steps_per_dim[kMaxDims];
    int num_steps;

    BINE_HD void init(int nd, const int* d) {
        ndims = nd;
        size = 1;
        num_steps = 0;
        for (int i = 0; i < kMaxDims; i++) {
            dims[i] = i < nd ? d[i] : 1;
            steps_per_dim[i] = i < nd ? ceil_log2(d[i]) : 0;
        }
        for (int i = 0; i < nd; i++) {
            size *= dims[i];
            num_steps += steps_per_dim[i];
        }
    }
    BINE_HD void coords(int id, int* c) const {
        int rest = size;
        for (int i = 0; i < ndims; i++) {
            rest /= dims[i];
            c[i] = id / rest;
            id %= rest;
        }
    }
    BINE_HD int id(const int* c) const {
        int r = 0, m = 1;
        for (int i = ndims - 1; i >= 0; i--) {
            r += m * pmod(c[i], dims[i]);
            m *= dims[i];
        }
        return r;
    }
};

// Ports on the mirrored half of the multi-port pattern run with negated
// distances.
BINE_HD bool mirrored_port(int port, int ndims) {
    if (ndims == 3) return port >= 3;
    if (ndims == 2) return port == 2 || port == 3;
    if (ndims == 1) return port & 1;
    return false;
}

enum Family { kFamilyBine = 1, kFamilyRecDoub = 2, kFamilyBruck = 3, kFamilyRing = 4 };  // lib/libbine_common.h:77-85

// Dimension and in-dimension step of each global step for a port: dimensions
// are visited round-robin starting at port % ndims, skipping exhausted ones.
struct StepDim {
    int8_t d;
    int8_t k;
};
BINE_HD void step_dims(const Torus& t, int port, StepDim* out) {
    int next[kMaxDims] = {0, 0, 0};
    int cur = port % t.ndims;
    for (int i = 0; i < t.num_steps; i++) {
        out[i].d = (int8_t)cur;
        out[i].k = (int8_t)next[cur];
        if (next[cur] < t.steps_per_dim[cur]) next[cur]++;
        if (i != t.num_steps - 1) {
            do {
                cur = (cur + 1) % t.ndims;
            } while (next[cur] >= t.steps_per_dim[cur]);
        }
    }
}

// Peer coordinates of `c` at global step `step` (a single-dimension move).
BINE_HD void step_peer(const Torus& t, const StepDim* sd, int step, int port, int family, const int* c, int* out) {
    for (int i = 0; i < t.ndims; i++) out[i] = c[i];
    int d = sd[step].d, k = sd[step].k;
    int dist;
    if (family == kFamilyRecDoub) {
        dist = (c[d] ^ (1 << k)) - c[d];
        if (mirrored_port(port, t.ndims)) dist = -dist;
    } else {
        dist = rho(k);
        if (c[d] & 1) dist = -dist;
        if (mirrored_port(port, t.ndims)) dist = -dist;
    }
    out[d] = pmod(c[d] + dist, t.dims[d]);
}

BINE_HD int step_peer_rank(const Torus& t, const StepDim* sd, int step, int port, int family, int rank) {
    int c[kMaxDims] = {0, 0, 0}, p[kMaxDims] = {0, 0, 0};
    t.coords(rank, c);
    step_peer(t, sd, step, port, family, c, p);
    return t.id(p);
}

}  // namespace bine

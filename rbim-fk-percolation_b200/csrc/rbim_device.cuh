// Device building blocks of the Swendsen-Wang sweep for the 2D +-J random-bond
// Ising model on sm_100a.
//
// Lattice layout ("linear bit layout").  Site n = x*L + y (x slow, y fast) as in
// the reference (src/rbim/lattice.py:5-23).  Every per-site bit plane stores bit
// n of the lattice in word n >> 5 at position n & 31, with no row padding, so a
// lattice of N = L*L sites occupies NW = ceil(N/32) words.  Bits at positions
// >= N in the last word are kept zero.  Planes:
//   S   spins, bit set <=> s = -1
//   JH  coupling of bond 2n, (x,y)->(x+1,y); bit set <=> J = -1
//   JV  coupling of bond 2n+1, (x,y)->(x,y+1); bit set <=> J = -1
//   OH  occupied horizontal bonds of the current sweep
//   OV  occupied vertical bonds, with the bonds that close the y boundary
//       (y = L-1) cleared; those are kept separately in SEAMV (bit x = row x)
//   FLIP flip bit of the cluster whose smallest site is n
//   ROOT bit n set <=> n is the smallest site of its cluster
//
// Union-find words.  Every site owns one word holding its parent site and the
// image offset (wx, wy) of the parent relative to the site: with unwrapped
// positions pos(), pos(parent) - pos(site) = coord(parent) - coord(site) +
// L*(wx, wy).  Offsets are the number of times the tree path crosses the
// periodic seams, which is the information the reference carries in its
// displacement arrays (src/rbim/_unionfind.py:59-136); a bond that closes a
// loop with nonzero summed offset winds around the torus.  The loop sum of a
// fundamental cycle is the winding number of a simple cycle, which is below L
// in magnitude, so offsets may be stored modulo 2^k as long as L < 2^k:
//   Word64 (plain engine): parent 32 bits | wx 16 bits | wy 16 bits (L <= 32768)
//   the resident engine labels the open lattice with 16-bit parents (no seam,
//   so no offsets) and keeps offsets only for the roots that touch a seam
//   (see rbim_resident.cu).
// Parents always have a smaller index than their child (heads of runs, roots
// hooked under smaller roots, path halving), so the structure is acyclic and
// every root is the smallest site of its cluster, which makes labels canonical.
// After labelling, the offset field of a root word is reused as the cluster
// size counter.
//
// Random numbers.  Philox4x32-10 (Salmon et al., SC'11) keyed by the 64-bit
// chain key, counter {block, sweep_lo, sweep_hi, stream}:
//   stream 0: bond k of sweep t draws u = 16-bit halfword (k & 7) of block k >> 3
//             (halfword h = bits 16*(h&1).. of word h >> 1)
//   stream 3: the same halfword of block k >> 3 gives v
//   stream 1: flip of the cluster rooted at r uses bit (r & 127) of block r >> 7
//   stream 2: hot-start spin of site n uses bit (n & 127) of block n >> 7, sweep 0
// A bond is occupied iff it is satisfied and (u << 16 | v) < thr, with
// thr = floor((1 - exp(-2 beta)) * 2^32) computed on the host in double; v is
// only drawn when u == thr >> 16, so one block serves eight bonds.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace rbim {

constexpr uint32_t kPhiloxM0 = 0xD2511F53u;
constexpr uint32_t kPhiloxM1 = 0xCD9E8D57u;
constexpr uint32_t kPhiloxW0 = 0x9E3779B9u;
constexpr uint32_t kPhiloxW1 = 0xBB67AE85u;

constexpr uint32_t kStreamBond = 0u;
constexpr uint32_t kStreamFlip = 1u;
constexpr uint32_t kStreamInit = 2u;
constexpr uint32_t kStreamBondLow = 3u;

// Error bits written to the status word.
constexpr int kErrFindCap = 1;
constexpr int kErrUnionCap = 2;
constexpr int kErrBadChain = 4;
constexpr int kErrGridWait = 8;

struct U4 {
    uint32_t x, y, z, w;
};

__device__ __forceinline__ U4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0,
                                            uint32_t k1)
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r) {
            k0 += kPhiloxW0;
            k1 += kPhiloxW1;
        }
        const uint32_t hi0 = __umulhi(kPhiloxM0, c0), lo0 = kPhiloxM0 * c0;
        const uint32_t hi1 = __umulhi(kPhiloxM1, c2), lo1 = kPhiloxM1 * c2;
        const uint32_t n0 = hi1 ^ c1 ^ k0;
        const uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
    }
    return {c0, c1, c2, c3};
}

__device__ __forceinline__ U4 philox_block(uint64_t key, uint32_t block, uint64_t sweep, uint32_t stream)
{
    return philox4x32_10(block, (uint32_t)sweep, (uint32_t)(sweep >> 32), stream, (uint32_t)key,
                         (uint32_t)(key >> 32));
}

__device__ __forceinline__ uint32_t u4_word(const U4 &v, uint32_t i)
{
    return i == 0 ? v.x : i == 1 ? v.y : i == 2 ? v.z : v.w;
}

// Mask of bits 0..b inclusive.
__device__ __forceinline__ uint32_t mask_le(uint32_t b) { return (2u << b) - 1u; }

// ---------------------------------------------------------------------------
// Lattice geometry of one word of sites.
// ---------------------------------------------------------------------------
struct Geom {
    uint32_t L, N, NW;
    __device__ __forceinline__ uint32_t valid(uint32_t w) const
    {
        const uint32_t n0 = w << 5;
        return (n0 + 32u <= N) ? 0xFFFFFFFFu : ((1u << (N - n0)) - 1u);
    }
    // Bits whose site has y == L-1 (row ends) among sites 32w .. 32w+31.
    __device__ __forceinline__ uint32_t row_end(uint32_t w) const
    {
        const uint32_t n0 = w << 5;
        uint32_t p = (L - 1u) - (n0 % L);
        uint32_t m = 0;
        for (; p < 32u; p += L) m |= 1u << p;
        return m & valid(w);
    }
};

// 32 bits of a bit plane starting at bit `start` (0 <= start < N), wrapping
// modulo N.  `ld(i)` loads word i; words at index >= NW must read as zero or
// never be requested.
template <class Ld>
__device__ __forceinline__ uint32_t extract32(const Ld &ld, uint32_t start, const Geom &g)
{
    const uint32_t wi = start >> 5, sh = start & 31u;
    if (start + 32u <= g.N) {
        const uint32_t lo = ld(wi);
        if (sh == 0) return lo;
        const uint32_t hi = (wi + 1u < g.NW) ? ld(wi + 1u) : 0u;
        return __funnelshift_r(lo, hi, sh);
    }
    if (g.N >= 64u) {
        // One wrap: bits start..N-1 then 0..(31 - (N - start)).
        const uint32_t k = g.N - start;  // 1..31
        const uint32_t lo = ld(wi);
        const uint32_t hi = (wi + 1u < g.NW) ? ld(wi + 1u) : 0u;
        const uint32_t a = (sh ? __funnelshift_r(lo, hi, sh) : lo) & ((1u << k) - 1u);
        return a | (ld(0) << k);
    }
    // Tiny lattices (N < 64): several wraps, go bit by bit.
    uint32_t r = 0;
    uint32_t p = start;
    for (uint32_t b = 0; b < 32u; ++b) {
        r |= ((ld(p >> 5) >> (p & 31u)) & 1u) << b;
        p = (p + 1u == g.N) ? 0u : p + 1u;
    }
    return r;
}

// Spin (or any plane) word of the +x neighbours of sites 32w..32w+31.
template <class Ld>
__device__ __forceinline__ uint32_t xnext_word(const Ld &ld, uint32_t w, const Geom &g)
{
    uint32_t s = (w << 5) + g.L;
    if (s >= g.N) s -= g.N;
    return extract32(ld, s, g);
}

// Plane word of the +y neighbours (periodic within the row); re is the
// row-end mask of word w (Geom::row_end).
template <class Ld>
__device__ __forceinline__ uint32_t ynext_word(const Ld &ld, uint32_t w, const Geom &g, uint32_t re)
{
    uint32_t s1 = (w << 5) + 1u;
    if (s1 >= g.N) s1 -= g.N;
    uint32_t r = extract32(ld, s1, g) & ~re;
    if (re) {
        // y = L-1 wraps to y = 0 of the same row: site n + 1 - L.
        uint32_t s2 = (w << 5) + g.N + 1u - g.L;
        if (s2 >= g.N) s2 -= g.N;
        r |= extract32(ld, s2, g) & re;
    }
    return r & g.valid(w);
}

// ---------------------------------------------------------------------------
// Union-find word traits.
// ---------------------------------------------------------------------------
struct Word64 {
    using T = unsigned long long;
    static constexpr int kOffBits = 16;
    __device__ __forceinline__ static uint32_t parent(T w) { return (uint32_t)w; }
    __device__ __forceinline__ static int ox(T w) { return (int)(int16_t)(w >> 32); }
    __device__ __forceinline__ static int oy(T w) { return (int)(int16_t)(w >> 48); }
    __device__ __forceinline__ static T make(uint32_t p, int x, int y)
    {
        return (T)p | ((T)(uint16_t)x << 32) | ((T)(uint16_t)y << 48);
    }
    __device__ __forceinline__ static bool nonzero(int v) { return (int16_t)v != 0; }
    __device__ __forceinline__ static uint32_t count(T w) { return (uint32_t)(w >> 32); }
    __device__ __forceinline__ static T count_inc(uint32_t c) { return (T)c << 32; }
};

__device__ __forceinline__ void uf_atomic_add(unsigned long long *p, unsigned long long v) { atomicAdd(p, v); }
__device__ __forceinline__ void uf_atomic_add(unsigned int *p, unsigned int v) { atomicAdd(p, v); }
// 16-bit add through the aligned 32-bit container; the caller guarantees the
// half does not overflow.
__device__ __forceinline__ void uf_atomic_add(unsigned short *p, unsigned short v)
{
    const uintptr_t a = (uintptr_t)p;
    atomicAdd((unsigned int *)(a & ~uintptr_t(3)), (unsigned int)v << (8u * (unsigned)(a & 2u)));
}

// Storage for one lattice's union-find words: a base pointer into shared or
// global memory (generic addressing covers both).  `ldc` is a load that may be
// served by the SM's L1 (global memory only) and so may return an older value
// than the latest store of another SM.  The walks use it: pointers only ever
// move to ancestors and a node that stopped being a root never becomes one
// again, so a stale word still names an ancestor with the right image offset,
// and every hook is a CAS that re-checks the root word in L2.  It takes the
// hot words near a large cluster's root off a single L2 slice.
template <class WT>
struct UF {
    using T = typename WT::T;
    T *w;
    __device__ __forceinline__ T ld(uint32_t i) const { return *((volatile T *)(w + i)); }
    __device__ __forceinline__ T ldc(uint32_t i) const { return __ldca(w + i); }
    __device__ __forceinline__ void st(uint32_t i, T v) const { *((volatile T *)(w + i)) = v; }
    __device__ __forceinline__ T cas(uint32_t i, T expect, T v) const { return atomicCAS(w + i, expect, v); }
    __device__ __forceinline__ void add(uint32_t i, T v) const { uf_atomic_add(w + i, v); }
};

struct Plane {
    uint32_t *p;
    __device__ __forceinline__ uint32_t operator()(uint32_t i) const { return *((volatile uint32_t *)(p + i)); }
};
struct PlaneRO {
    const uint32_t *p;
    __device__ __forceinline__ uint32_t operator()(uint32_t i) const { return p[i]; }
};

struct FindResult {
    uint32_t root;
    int ax, ay;
};

// Root of `n` and the summed image offset from n to it, with path halving.
// Terminates because parents strictly decrease; the cap only guards against
// corrupted input and raises kErrFindCap.
template <class WT>
__device__ __forceinline__ FindResult uf_find(const UF<WT> &uf, uint32_t n, uint32_t cap, int *err)
{
    using T = typename WT::T;
    uint32_t node = n;
    int ax = 0, ay = 0;
    T w = uf.ld(node);
    for (uint32_t it = 0;; ++it) {
        const uint32_t p = WT::parent(w);
        if (p == node) break;
        if (it >= cap) {
            atomicOr(err, kErrFindCap);
            break;
        }
        const T wp = uf.ld(p);
        const uint32_t gp = WT::parent(wp);
        if (gp != p) {
            const int nx = WT::ox(w) + WT::ox(wp), ny = WT::oy(w) + WT::oy(wp);
            uf.st(node, WT::make(gp, nx, ny));
            ax += nx;
            ay += ny;
            node = gp;
            w = uf.ld(node);
        } else {
            ax += WT::ox(w);
            ay += WT::oy(w);
            node = p;
            w = wp;
        }
    }
    return {node, ax, ay};
}

// Root only, without writing: used once no more unions can happen, so that
// each site's word is written by its own thread alone (a compressing walk
// could overwrite another site's final root pointer with a stale ancestor).
template <class WT>
__device__ __forceinline__ uint32_t uf_root_ro(const UF<WT> &uf, uint32_t n, uint32_t cap, int *err)
{
    uint32_t node = n;
    for (uint32_t it = 0;; ++it) {
        const uint32_t p = WT::parent(uf.ld(node));
        if (p == node) break;
        if (it >= cap) {
            atomicOr(err, kErrFindCap);
            break;
        }
        node = p;
    }
    return node;
}

// Union across the bond a -> b whose seam crossing is (ex, ey).  Sets bit 0
// (x) / bit 1 (y) of *wrap when the bond closes a loop that winds.  The larger
// root is hooked under the smaller with a CAS on its (self, 0, 0) word.
template <class WT>
__device__ __forceinline__ void uf_union(const UF<WT> &uf, uint32_t a, uint32_t b, int ex, int ey, int *wrap,
                                         uint32_t cap, int *err)
{
    using T = typename WT::T;
    for (uint32_t it = 0; it < cap; ++it) {
        const FindResult fa = uf_find<WT>(uf, a, cap, err);
        const FindResult fb = uf_find<WT>(uf, b, cap, err);
        if (fa.root == fb.root) {
            int f = 0;
            if (WT::nonzero(ex + fb.ax - fa.ax)) f |= 1;
            if (WT::nonzero(ey + fb.ay - fa.ay)) f |= 2;
            if (f) atomicOr(wrap, f);
            return;
        }
        if (fa.root < fb.root) {
            const T expect = WT::make(fb.root, 0, 0);
            const T v = WT::make(fa.root, fa.ax - ex - fb.ax, fa.ay - ey - fb.ay);
            if (uf.cas(fb.root, expect, v) == expect) return;
        } else {
            const T expect = WT::make(fa.root, 0, 0);
            const T v = WT::make(fb.root, fb.ax + ex - fa.ax, fb.ay + ey - fa.ay);
            if (uf.cas(fa.root, expect, v) == expect) return;
        }
    }
    atomicOr(err, kErrUnionCap);
}

// Top-two merge of unique keys (a1 >= a2, b1 >= b2).
template <class K>
__device__ __forceinline__ void top2_merge(K &a1, K &a2, K b1, K b2)
{
    const K hi = a1 > b1 ? a1 : b1;
    const K lo = a1 > b1 ? b1 : a1;
    const K s = a2 > b2 ? a2 : b2;
    a1 = hi;
    a2 = lo > s ? lo : s;
}

template <class K>
__device__ __forceinline__ void warp_top2(K &k1, K &k2)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const K b1 = __shfl_xor_sync(0xFFFFFFFFu, k1, o);
        const K b2 = __shfl_xor_sync(0xFFFFFFFFu, k2, o);
        top2_merge(k1, k2, b1, b2);
    }
}

// ---------------------------------------------------------------------------
// Per-sweep record and primitive accumulation.
// Record: E, M, n_clusters, S1, |M_C1|, S2, |M_C2|, wrap_x, wrap_y (the fields
// of the reference's SweepResult, src/rbim/swendsen_wang.py:24-53, in order).
// Integer sums per bin: E, E^2, M, |M|, M^2, S1, |M_C1|, S2, n_clusters,
//                       wrap_x, wrap_y, wrap_any            (int64)
// Floating sums per bin: M^4, |M_C1|/S1                     (double)
// ---------------------------------------------------------------------------
constexpr int kRecLen = 9;
constexpr int kAccInt = 12;
constexpr int kAccF64 = 2;

struct Acc {
    long long i[kAccInt];
    double f[kAccF64];
    __device__ __forceinline__ void zero()
    {
#pragma unroll
        for (int k = 0; k < kAccInt; ++k) i[k] = 0;
        f[0] = f[1] = 0.0;
    }
    __device__ __forceinline__ void add(long long e, long long m, long long ncl, long long s1, long long mc,
                                        long long s2, int wx, int wy)
    {
        const long long am = m < 0 ? -m : m;
        i[0] += e;
        i[1] += e * e;
        i[2] += m;
        i[3] += am;
        i[4] += m * m;
        i[5] += s1;
        i[6] += mc;
        i[7] += s2;
        i[8] += ncl;
        i[9] += wx;
        i[10] += wy;
        i[11] += (wx | wy) ? 1 : 0;
        const double m2 = (double)(m * m);
        f[0] += m2 * m2;
        f[1] += s1 > 0 ? (double)mc / (double)s1 : 0.0;
    }
    __device__ __forceinline__ void load(const long long *gi, const double *gf)
    {
#pragma unroll
        for (int k = 0; k < kAccInt; ++k) i[k] = gi[k];
        f[0] = gf[0];
        f[1] = gf[1];
    }
    __device__ __forceinline__ void store(long long *gi, double *gf) const
    {
#pragma unroll
        for (int k = 0; k < kAccInt; ++k) gi[k] = i[k];
        gf[0] = f[0];
        gf[1] = f[1];
    }
    __device__ __forceinline__ void flush(long long *gi, double *gf) const
    {
#pragma unroll
        for (int k = 0; k < kAccInt; ++k) gi[k] += i[k];
        gf[0] += f[0];
        gf[1] += f[1];
    }
};

}  // namespace rbim

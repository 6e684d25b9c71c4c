// Resident engine: one lattice per CTA, held in shared memory for every sweep
// of a call.  A persistent grid pulls chains from a work queue (an atomic
// counter in global memory), loads the chain's spin and coupling planes, runs
// its sweeps entirely on chip and writes back only the spin plane, the bin
// sums and the optional per-sweep records.
//
// Labelling runs in two stages so that a whole L = 256 lattice fits one CTA:
//  1. the open lattice (every bond except the 2L that close the periodic
//     boundary) is labelled with a union-find of 16-bit parents: inside the
//     open rectangle every cycle is contractible, so no image offsets are
//     needed and each open cluster's root is its smallest site;
//  2. the roots of the open clusters that touch a seam bond are hashed into a
//     small table whose union-find words carry image offsets; the seam bonds
//     are unioned there, and a seam bond that closes a loop with nonzero
//     summed offset winds around the torus (the exact test of the reference,
//     src/rbim/_unionfind.py:104-124).  Each merged open root is then pointed
//     at the smallest open root of its full cluster.
//
// This replaces, per chain, the loop of run_single_realization
// (src/rbim/simulation.py:196-242) around sw_sweep
// (src/rbim/swendsen_wang.py:103-172).
#include <algorithm>

#include "rbim_internal.h"
#include "rbim_phases.cuh"

namespace rbim {

namespace {

constexpr uint32_t kMaxResidentSites = 65536;  // 16-bit parents
// Dynamic shared memory budget: the 227 KB per-CTA limit minus room for the
// kernels' static shared scratch.
constexpr size_t kMaxSmem = 227 * 1024 - 8 * 1024;
constexpr uint32_t kHashEmpty = 0xFFFFFFFFu;
// Shared memory of one SM, and an allowance for a CTA's static shared scratch
// and the per-CTA reservation, when deciding how many CTAs fit an SM.
constexpr size_t kSmemPerSm = 228 * 1024;
constexpr size_t kStaticSmem = 2 * 1024;

__host__ __device__ constexpr size_t align16(size_t v) { return (v + 15) & ~size_t(15); }

__host__ __device__ constexpr uint32_t hash_size(uint32_t l_max)
{
    // At most 4L distinct open roots touch a seam bond; keep the load <= 1/2.
    uint32_t h = 32;
    while (h < 8u * l_max) h *= 2;
    return h;
}

}  // namespace

// Optional per-phase cycle accounting (profiling builds only, compiled with
// -DRBIM_PROFILE_PHASES): thread 0 adds the cycles since the previous mark to
// a per-phase counter at each barrier.  No work is skipped.
#ifdef RBIM_PROFILE_PHASES
__device__ unsigned long long g_phase_cycles[16];
__device__ __forceinline__ void phase_mark(int k)
{
    __shared__ long long s_t;
    if (threadIdx.x == 0) {
        const long long now = clock64();
        if (k >= 0) atomicAdd(&g_phase_cycles[k], (unsigned long long)(now - s_t));
        s_t = now;
    }
}
#define RBIM_PHASE_MARK(k) phase_mark(k)
__device__ unsigned long long g_event_counts[8];
#define RBIM_COUNT(k, v) atomicAdd(&g_event_counts[k], (unsigned long long)(v))
#define RBIM_PROF_ONLY(...) __VA_ARGS__
#else
#define RBIM_PHASE_MARK(k) ((void)0)
#define RBIM_COUNT(k, v) ((void)0)
#define RBIM_PROF_ONLY(...)
#endif

}  // namespace rbim

#include "rbim_open.cuh"

namespace rbim {

// Seam union-find word: parent slot (12 bits) | wx (10 bits) | wy (10 bits),
// offsets modulo 1024 (exact for L < 1024, see rbim_device.cuh).
struct SeamWord {
    using T = uint32_t;
    __device__ __forceinline__ static uint32_t parent(T w) { return w & 0xFFFu; }
    __device__ __forceinline__ static int ox(T w) { return ((int)(w << 10)) >> 22; }
    __device__ __forceinline__ static int oy(T w) { return ((int)w) >> 22; }
    __device__ __forceinline__ static T make(uint32_t p, int x, int y)
    {
        return (p & 0xFFFu) | ((uint32_t)(x & 0x3FF) << 12) | ((uint32_t)(y & 0x3FF) << 22);
    }
    __device__ __forceinline__ static bool nonzero(int v) { return (v & 0x3FF) != 0; }
};

// Shared-memory layout for lattices of up to l_max x l_max sites; constexpr so
// that the launches of the common size classes get it as a compile-time
// constant (the kernel's shared-memory views then need no registers).
__host__ __device__ constexpr ResidentLayout resident_layout_c(uint32_t l_max)
{
    ResidentLayout ly{};
    ly.l_max = l_max;
    ly.n_max = l_max * l_max;
    const uint32_t nw = (ly.n_max + 31u) / 32u;
    ly.nw_max = (nw + 3u) & ~3u;
    ly.hs = hash_size(l_max);
    size_t off = 0;
    ly.off_uf = off;
    off = align16(off + 2ull * ly.n_max);
    const size_t plane = 4ull * (ly.nw_max + 4u);
    ly.off_S = off;
    off += plane;
    ly.off_JH = off;
    off += plane;
    ly.off_JV = off;
    off += plane;
    ly.off_OH = off;
    off += plane;
    ly.off_OV = off;
    off += plane;
    ly.off_FLIP = off;
    off += plane;
    ly.off_ROOT = off;
    off += plane;
    ly.off_RE = off;
    off += plane;
    ly.off_SEAMV = off;
    off = align16(off + 4ull * (((l_max + 31u) / 32u) + 4u));
    ly.off_HK = off;
    off += 4ull * ly.hs;
    ly.off_HW = off;
    off += 4ull * ly.hs;
    ly.bytes = align16(off);
    return ly;
}

ResidentLayout resident_layout(uint32_t l_max, int threads)
{
    (void)threads;
    return resident_layout_c(l_max);
}

int resident_max_l()
{
    int best = 3;
    for (int L = 3; L <= 256; ++L) {
        if ((uint32_t)(L * L) > kMaxResidentSites) break;
        if (resident_layout(L, 1024).bytes <= kMaxSmem) best = L;
    }
    return best;
}

int resident_default_threads(int l_max)
{
    // At 64 registers a thread an SM holds 1024 of this kernel's threads
    // whatever the CTA size, and several small CTAs per SM hide each other's
    // barrier waits better than one large one; so the CTA is as small as the
    // lattice allows before its per-thread work grows long.  Measured on
    // B200: 32 threads (one warp) up to L = 32 (against 64: +36 % at L = 16,
    // +7 % at 24, +17 % at 32), 128 up to 64, 256 up to 96, then 512 while
    // two CTAs' shared memory fits an SM (up to L = 180), then 1024.
    if (l_max <= 32) return 32;
    if (l_max <= 64) return 128;
    if (l_max <= 96) return 256;
    if (2 * (resident_layout_c((uint32_t)l_max).bytes + kStaticSmem) <= kSmemPerSm) return 512;
    return 1024;
}

// Shared scratch of one CTA.
template <int NT>
struct Red {
    uint32_t k1[NT / 32], k2[NT / 32];
    uint32_t unsat[NT / 32], downs[NT / 32], roots[NT / 32];
    int mc[NT / 32], mc2[NT / 32];
    int item, wrap, err;
    uint32_t g1, g2, s1, s2;
    // State of the chain being processed; only thread 0 updates it.
    Acc acc;
    long long cur_bin;
    rbim_chain_t ch;
};

// Blocks per SM the register budget is tuned for (64 registers per thread).
template <int NT>
struct MinBlocks {
    static constexpr int value = NT >= 1024 ? 1 : 1024 / NT;
};

// Per-CTA view of the shared-memory arrays of one lattice.
struct Res {
    Lat<Word16> t;
    uint32_t *HK;  // seam hash keys: open root site, or kHashEmpty
    uint32_t *HW;  // seam union-find words (SeamWord)
    uint32_t hs, hs_log2;
};

// walk_cap > 0 lowers the per-walk bound (and with it the per-thread loop
// bounds, 64 walks' worth) from N + 64 steps to walk_cap: the chain
// descriptor's test hook that makes the bounds fire on a small lattice.
template <int NT>
__device__ __forceinline__ Res make_res(unsigned char *smem, const ResidentLayout &ly, uint32_t L, Red<NT> &red,
                                        int64_t walk_cap = 0)
{
    Res r;
    Lat<Word16> &t = r.t;
    t.g = Geom{L, L * L, (L * L + 31u) / 32u};
    t.uf.w = (unsigned short *)(smem + ly.off_uf);
    t.uf.sa = (uint32_t)__cvta_generic_to_shared(t.uf.w);
    t.S = (uint32_t *)(smem + ly.off_S);
    t.JH = (const uint32_t *)(smem + ly.off_JH);
    t.JV = (const uint32_t *)(smem + ly.off_JV);
    t.OH = (uint32_t *)(smem + ly.off_OH);
    t.OV = (uint32_t *)(smem + ly.off_OV);
    t.FLIP = (uint32_t *)(smem + ly.off_FLIP);
    t.ROOT = (uint32_t *)(smem + ly.off_ROOT);
    t.RE = (const uint32_t *)(smem + ly.off_RE);
    t.SEAMV = (uint32_t *)(smem + ly.off_SEAMV);
    t.wrap = &red.wrap;
    t.err = &red.err;
    t.cap = (walk_cap > 0 && walk_cap < (int64_t)(t.g.N + 64u)) ? (uint32_t)walk_cap : t.g.N + 64u;
    r.HK = (uint32_t *)(smem + ly.off_HK);
    r.HW = (uint32_t *)(smem + ly.off_HW);
    r.hs = ly.hs;
    r.hs_log2 = 31u - __clz(ly.hs);
    return r;
}

// Row-end masks of the lattice (computed once per chain, so that the sweep
// needs no integer division).
__device__ __forceinline__ void init_row_ends(const Lat<Word16> &t, uint32_t tid, uint32_t nthreads)
{
    uint32_t *re = const_cast<uint32_t *>(t.RE);
    for (uint32_t w = tid; w < t.g.NW; w += nthreads) re[w] = t.g.row_end(w);
}

__device__ __forceinline__ uint32_t hash_insert(const Res &r, uint32_t key, int *err)
{
    uint32_t h = (key * 0x9E3779B1u) >> (32u - r.hs_log2);
    for (uint32_t it = 0; it < r.hs; ++it) {
        const uint32_t old = atomicCAS(r.HK + h, kHashEmpty, key);
        if (old == kHashEmpty || old == key) return h;
        h = (h + 1u) & (r.hs - 1u);
    }
    atomicOr(err, kErrUnionCap);
    return 0;
}

// Union of two seam nodes across a seam bond with seam crossing (ex, ey); the
// node whose open root is larger is hooked under the other.
__device__ __forceinline__ void seam_union(const Res &r, uint32_t na, uint32_t nb, int ex, int ey, int *wrap,
                                           uint32_t cap, int *err)
{
    const UF<SeamWord> hw{r.HW};
    for (uint32_t it = 0; it < cap; ++it) {
        const FindResult fa = uf_find<SeamWord>(hw, na, cap, err);
        const FindResult fb = uf_find<SeamWord>(hw, nb, cap, err);
        if (fa.root == fb.root) {
            int f = 0;
            if (SeamWord::nonzero(ex + fb.ax - fa.ax)) f |= 1;
            if (SeamWord::nonzero(ey + fb.ay - fa.ay)) f |= 2;
            if (f) atomicOr(wrap, f);
            return;
        }
        const uint32_t ka = r.HK[fa.root], kb = r.HK[fb.root];
        if (ka < kb) {
            const uint32_t expect = SeamWord::make(fb.root, 0, 0);
            if (hw.cas(fb.root, expect, SeamWord::make(fa.root, fa.ax - ex - fb.ax, fa.ay - ey - fb.ay)) == expect)
                return;
        } else {
            const uint32_t expect = SeamWord::make(fa.root, 0, 0);
            if (hw.cas(fa.root, expect, SeamWord::make(fb.root, fb.ax + ex - fa.ax, fb.ay + ey - fa.ay)) == expect)
                return;
        }
    }
    atomicOr(err, kErrUnionCap);
}

// Seam table reset (before the seam phase).
__device__ __forceinline__ void seam_reset(const Res &r, uint32_t tid, uint32_t nthreads)
{
    for (uint32_t k = tid; k < r.hs; k += nthreads) {
        r.HK[k] = kHashEmpty;
        r.HW[k] = SeamWord::make(k, 0, 0);
    }
}

// (b) Seam bonds: x seam (x = L-1 -> 0, crossing (1,0)) and y seam
// (y = L-1 -> 0, crossing (0,1)).  The open union-find is final here.
__device__ __forceinline__ void phase_seam(const Res &r, uint32_t tid, uint32_t nthreads)
{
    const Lat<Word16> &t = r.t;
    const Geom &g = t.g;
    for (uint32_t i = tid; i < 2u * g.L; i += nthreads) {
        uint32_t a, b;
        int ex, ey;
        if (i < g.L) {
            a = g.N - g.L + i;
            if (!((t.OH[a >> 5] >> (a & 31u)) & 1u)) continue;
            b = i;
            ex = 1;
            ey = 0;
        } else {
            const uint32_t x = i - g.L;
            if (!((t.SEAMV[x >> 5] >> (x & 31u)) & 1u)) continue;
            a = x * g.L + g.L - 1u;
            b = x * g.L;
            ex = 0;
            ey = 1;
        }
        const uint32_t ra = uf_root_ro<Word16>(t.uf, a, t.cap, t.err);
        const uint32_t rb = uf_root_ro<Word16>(t.uf, b, t.cap, t.err);
        const uint32_t na = hash_insert(r, ra, t.err);
        const uint32_t nb = hash_insert(r, rb, t.err);
        seam_union(r, na, nb, ex, ey, t.wrap, t.cap, t.err);
    }
}

// (b) Point every merged open root at the smallest open root of its cluster.
__device__ __forceinline__ void phase_seam_propagate(const Res &r, uint32_t tid, uint32_t nthreads)
{
    const UF<SeamWord> hw{r.HW};
    for (uint32_t k = tid; k < r.hs; k += nthreads) {
        const uint32_t key = r.HK[k];
        if (key == kHashEmpty) continue;
        const uint32_t g = uf_root_ro<SeamWord>(hw, k, r.hs + 1u, r.t.err);
        if (g != k) r.t.uf.st(key, (unsigned short)r.HK[g]);
    }
}

// The labelling stages shared by the sweep and label kernels, from occupied
// bond planes to final roots; barriers between stages.  Returns the number of
// roots counted by this warp.  The label kernel (sweep = false) then points
// every site's word at its root; a sweep flips the clusters piece by piece
// (flip_pieces), with the piece leaders' roots written when the
// sweep is measured.
template <int NT>
__device__ __forceinline__ uint32_t resident_label(const Res &r, bool sweep, bool measure)
{
    const uint32_t tid = threadIdx.x, warp = tid >> 5;
    constexpr uint32_t nwarps = NT / 32;
    phase_heads<Word16>(r.t, warp, nwarps);
    seam_reset(r, tid, NT);
    for (uint32_t w = tid; w < r.t.g.NW; w += NT) r.t.ROOT[w] = 0u;
    __syncthreads();
    RBIM_PHASE_MARK(1);
    phase_union_open(r.t, tid, NT);
    __syncthreads();
    RBIM_PHASE_MARK(2);
    phase_seam(r, tid, NT);
    __syncthreads();
    RBIM_PHASE_MARK(3);
    phase_seam_propagate(r, tid, NT);
    for (uint32_t i = tid; i < (r.t.g.L + 31u) / 32u; i += NT) r.t.SEAMV[i] = 0u;
    __syncthreads();
    RBIM_PHASE_MARK(4);
    if (sweep && r.t.g.NW >= NT) {
        // Every thread has a word: roots and flip in one pass over pieces.
        const uint32_t nr = warp_sum(roots_flip_pieces(r.t, tid, NT));
        __syncthreads();
        RBIM_PHASE_MARK(11);
        RBIM_PHASE_MARK(5);
        return nr;
    }
    const uint32_t nr = warp_sum(phase_roots_flat(r.t, tid, NT));
    __syncthreads();
    RBIM_PHASE_MARK(11);
    // Small lattices (fewer words than threads) flip site by site, which
    // keeps every lane busy; this also leaves every site's word at its root.
    phase_sites<Word16>(r.t, warp, nwarps, sweep, false);
    __syncthreads();
    RBIM_PHASE_MARK(5);
    return nr;
}

// Measurement of one sweep after resident_label: energy, magnetization,
// n_clusters, S1, S2, |M_C1| and, with `second` (records requested), |M_C2|
// (reference sw_sweep, src/rbim/swendsen_wang.py:146-172).  Ends with a
// barrier.  Thread 0 returns the record in rec.
template <int NT>
__device__ __forceinline__ void resident_measure(const Res &res, Red<NT> &red, uint32_t nroots_warp,
                                                 long long rec[kRecLen], bool second)
{
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    constexpr uint32_t nwarps = NT / 32;
    const Lat<Word16> &t = res.t;
    const Geom &g = t.g;
    unsigned short *u16 = t.uf.w;

    // Energy and magnetization of the flipped spins.
    uint32_t unsat = 0, downs = 0;
    measure_energy(t, tid, NT, unsat, downs);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        unsat += __shfl_xor_sync(0xFFFFFFFFu, unsat, o);
        downs += __shfl_xor_sync(0xFFFFFFFFu, downs, o);
    }
    if (lane == 0) {
        red.unsat[warp] = unsat;
        red.downs[warp] = downs;
        red.roots[warp] = nroots_warp;
    }
    RBIM_PHASE_MARK(6);
    // Cluster sizes into the root words, on top of the index each root's word
    // holds (a root points at itself): afterwards a root's word is root + size
    // mod 2^16, which gives every size whenever there are two or more
    // clusters (each then below 65536); one cluster is the lattice.
    count_pieces<false>(t, u16, warp, nwarps);
    __syncthreads();
    RBIM_PHASE_MARK(7);
    // Every warp sums the per-warp partials itself (no barrier needed after).
    uint32_t unsat_t = lane < nwarps ? red.unsat[lane] : 0u, downs_t = lane < nwarps ? red.downs[lane] : 0u;
    uint32_t ncl = lane < nwarps ? red.roots[lane] : 0u;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        unsat_t += __shfl_xor_sync(0xFFFFFFFFu, unsat_t, o);
        downs_t += __shfl_xor_sync(0xFFFFFFFFu, downs_t, o);
        ncl += __shfl_xor_sync(0xFFFFFFFFu, ncl, o);
    }
    if (ncl > 1) {
        uint32_t k1 = 0, k2 = 0;
        for (uint32_t w = tid; w < g.NW; w += NT) {
            uint32_t roots = t.ROOT[w];
            while (roots) {
                const uint32_t b = __ffs(roots) - 1u;
                roots &= roots - 1u;
                const uint32_t r = (w << 5) + b;
                top2_merge(k1, k2, ((((uint32_t)u16[r] - r) & 0xFFFFu) << 16) | (0xFFFFu - r), 0u);
            }
        }
        warp_top2(k1, k2);
        if (lane == 0) {
            red.k1[warp] = k1;
            red.k2[warp] = k2;
        }
        __syncthreads();
        if (warp == 0) {
            uint32_t a1 = lane < nwarps ? red.k1[lane] : 0u, a2 = lane < nwarps ? red.k2[lane] : 0u;
            warp_top2(a1, a2);
            if (lane == 0) {
                red.g1 = 0xFFFFu - (a1 & 0xFFFFu);
                red.g2 = 0xFFFFu - (a2 & 0xFFFFu);
                red.s1 = a1 >> 16;
                red.s2 = a2 >> 16;
            }
        }
        __syncthreads();
        RBIM_PHASE_MARK(8);
        const uint32_t g1 = red.g1, g2 = red.g2;
        int mc = 0, mc2 = 0;
        if (g.NW < NT) {
            // Small lattices took the per-site path (every site's word holds
            // its root): lanes are sites, which keeps all warps busy.  Two
            // words per iteration keep two load chains in flight.
            for (uint32_t w0 = warp; w0 < g.NW; w0 += 2u * nwarps) {
                const uint32_t w1 = w0 + nwarps;
                const uint32_t n0 = (w0 << 5) + lane, n1 = (w1 << 5) + lane;
                const uint32_t rt0 = t.ROOT[w0], rt1 = w1 < g.NW ? t.ROOT[w1] : 0u;
                const bool ok0 = n0 < g.N, ok1 = n1 < g.N;
                const uint32_t p0 = ok0 ? (uint32_t)u16[n0] : 0u, p1 = ok1 ? (uint32_t)u16[n1] : 0u;
                const uint32_t r0 = ((rt0 >> lane) & 1u) ? n0 : p0, r1 = ((rt1 >> lane) & 1u) ? n1 : p1;
                const uint32_t m0 = __ballot_sync(0xFFFFFFFFu, ok0 && r0 == g1);
                const uint32_t m1 = __ballot_sync(0xFFFFFFFFu, ok1 && r1 == g1);
                const uint32_t s0 = t.S[w0], s1 = w1 < g.NW ? t.S[w1] : 0u;
                if (lane == 0) mc += (int)__popc(m0) - 2 * (int)__popc(m0 & s0) + (int)__popc(m1) - 2 * (int)__popc(m1 & s1);
                if (second) {
                    const uint32_t q0 = __ballot_sync(0xFFFFFFFFu, ok0 && r0 == g2);
                    const uint32_t q1 = __ballot_sync(0xFFFFFFFFu, ok1 && r1 == g2);
                    if (lane == 0) mc2 += (int)__popc(q0) - 2 * (int)__popc(q0 & s0) + (int)__popc(q1) -
                                          2 * (int)__popc(q1 & s1);
                }
            }
        } else {
            // One lane per word, one test per run piece: the word of a piece's
            // leader holds its root (its size counter when the leader is the
            // root, recognised by its ROOT bit).  Measured faster on B200 than
            // lanes-as-sites with the root read from each site's piece leader
            // (15 k vs 24 k cycles per L = 256 sweep).
            for (uint32_t w = tid; w < g.NW; w += NT) {
                const uint32_t valid = g.valid(w);
                uint32_t lead = piece_leaders(t, w, valid);
                const uint32_t roots = t.ROOT[w], s = t.S[w];
                const uint32_t nv = (uint32_t)__popc(valid);
                while (lead) {
                    const uint32_t b = __ffs(lead) - 1u;
                    lead &= lead - 1u;
                    const uint32_t end = lead ? (uint32_t)(__ffs(lead) - 1) : nv;
                    const uint32_t n = (w << 5) + b;
                    const uint32_t r = ((roots >> b) & 1u) ? n : (uint32_t)u16[n];
                    const uint32_t pm = (end - b == 32u) ? 0xFFFFFFFFu : (((1u << (end - b)) - 1u) << b);
                    const int m = (int)__popc(pm) - 2 * (int)__popc(pm & s);
                    if (r == g1) mc += m;
                    if (second && r == g2) mc2 += m;
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            mc += __shfl_xor_sync(0xFFFFFFFFu, mc, o);
            mc2 += __shfl_xor_sync(0xFFFFFFFFu, mc2, o);
        }
        if (lane == 0) {
            red.mc[warp] = mc;
            red.mc2[warp] = mc2;
        }
        __syncthreads();
        RBIM_PHASE_MARK(9);
    } else if (tid == 0) {
        // One cluster covers the lattice.
        red.g1 = 0;
        red.s1 = g.N;
        red.s2 = 0;
    }
    const long long M = (long long)g.N - 2ll * (long long)downs_t;
    if (tid == 0) {
        long long mc_total = M, mc2_total = 0;
        if (ncl > 1) {
            mc_total = 0;
            for (uint32_t i = 0; i < nwarps; ++i) {
                mc_total += red.mc[i];
                mc2_total += red.mc2[i];
            }
        }
        rec[0] = 2ll * (long long)unsat_t - 2ll * (long long)g.N;
        rec[1] = M;
        rec[2] = ncl;
        rec[3] = red.s1;
        rec[4] = mc_total < 0 ? -mc_total : mc_total;
        rec[5] = red.s2;
        rec[6] = mc2_total < 0 ? -mc2_total : mc2_total;
        rec[7] = red.wrap & 1;
        rec[8] = (red.wrap >> 1) & 1;
    }
    __syncthreads();
}

// LC > 0: the launch's layout is resident_layout_c(LC), a compile-time
// constant; LC == 0: the layout passed in.
template <int NT, int LC>
__global__ void __launch_bounds__(NT, MinBlocks<NT>::value)
    k_resident_sweeps(rbim_chain_t *chains, int n_chains, uint32_t *spin_pool, const uint32_t *coupling_pool,
                      long long *acc_i, double *acc_f, int32_t *records, int n_sweeps, int *queue, int *status,
                      ResidentLayout ly_arg)
{
    constexpr ResidentLayout kly = resident_layout_c(LC > 0 ? LC : 16);
    const ResidentLayout ly = LC > 0 ? kly : ly_arg;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ Red<NT> red;
    const uint32_t tid = threadIdx.x, warp = tid >> 5;
    constexpr uint32_t nwarps = NT / 32;

    if (tid == 0) red.err = 0;
    for (;;) {
        if (tid == 0) {
            red.item = atomicAdd(queue, 1);
            if (red.item < n_chains) {
                red.ch = chains[red.item];
                red.cur_bin = -1;
            }
        }
        __syncthreads();
        const int item = red.item;
        if (item >= n_chains) break;
        const rbim_chain_t &ch = red.ch;
        if (ch.L < 3 || ch.L > (int64_t)ly.l_max || ch.sweeps_per_bin < 1 || ch.n_bins < 0 || ch.n_therm < 0 ||
            ch.walk_cap < 0) {
            if (tid == 0) atomicOr(status, kErrBadChain);
            __syncthreads();
            continue;
        }
        const uint32_t L = (uint32_t)ch.L;
        const Res res = make_res<NT>(smem, ly, L, red, ch.walk_cap);
        const Lat<Word16> &t = res.t;
        const Geom g = t.g;
        const uint32_t nwp = (g.NW + 3u) & ~3u;

        // Load the chain's planes (16-byte aligned, whole padded planes).
        {
            const uint4 *gs = (const uint4 *)(spin_pool + ch.spin_off);
            const uint4 *gh = (const uint4 *)(coupling_pool + ch.coupling_off);
            const uint4 *gv = (const uint4 *)(coupling_pool + ch.coupling_off + nwp);
            for (uint32_t i = tid; i < nwp / 4u; i += NT) {
                ((uint4 *)t.S)[i] = gs[i];
                ((uint4 *)t.JH)[i] = gh[i];
                ((uint4 *)t.JV)[i] = gv[i];
            }
            for (uint32_t i = tid; i < (L + 31u) / 32u; i += NT) t.SEAMV[i] = 0u;
            init_row_ends(t, tid, NT);
        }
        const uint64_t t_end = (uint64_t)ch.n_therm + (uint64_t)ch.n_bins * (uint64_t)ch.sweeps_per_bin;
        uint64_t sweep = ch.sweep;
        const uint64_t stop = min(t_end, sweep + (uint64_t)max(n_sweeps, 0));
        __syncthreads();

        for (; sweep < stop; ++sweep) {
            const bool measure = sweep >= (uint64_t)ch.n_therm;
            if (tid == 0) red.wrap = 0;
            RBIM_PHASE_MARK(-1);
            phase_activate<Word16>(t, make_rng(ch.key, sweep, ch.thr), warp, nwarps, tid, NT);
            __syncthreads();
            RBIM_PHASE_MARK(0);
            const uint32_t nr = resident_label<NT>(res, true, measure);
            if (measure) {
                long long rec[kRecLen];
                const bool want_rec = records && ch.rec_off >= 0;
                resident_measure<NT>(res, red, nr, rec, want_rec);
                if (tid == 0) {
                    const long long idx = (long long)(sweep - (uint64_t)ch.n_therm);
                    const long long bin = idx / ch.sweeps_per_bin;
                    if (bin != red.cur_bin) {
                        if (red.cur_bin >= 0)
                            red.acc.store(acc_i + (ch.acc_off + red.cur_bin) * kAccInt,
                                          acc_f + (ch.acc_off + red.cur_bin) * kAccF64);
                        // Resume from the stored sums so that additions stay in
                        // sweep order whatever the split into calls.
                        red.acc.load(acc_i + (ch.acc_off + bin) * kAccInt, acc_f + (ch.acc_off + bin) * kAccF64);
                        red.cur_bin = bin;
                    }
                    red.acc.add(rec[0], rec[1], rec[2], rec[3], rec[4], rec[5], (int)rec[7], (int)rec[8]);
                    if (want_rec) {
                        int32_t *row = records + (ch.rec_off + idx) * kRecLen;
#pragma unroll
                        for (int k = 0; k < kRecLen; ++k) row[k] = (int32_t)rec[k];
                    }
                }
                RBIM_PHASE_MARK(10);
            }
        }
        if (tid == 0) {
            if (red.cur_bin >= 0)
                red.acc.store(acc_i + (ch.acc_off + red.cur_bin) * kAccInt,
                              acc_f + (ch.acc_off + red.cur_bin) * kAccF64);
            chains[item].sweep = stop;
        }
        // Write the spin plane back.
        {
            uint4 *gs = (uint4 *)(spin_pool + ch.spin_off);
            for (uint32_t i = tid; i < nwp / 4u; i += NT) gs[i] = ((const uint4 *)t.S)[i];
        }
        __syncthreads();
    }
    if (tid == 0 && red.err) atomicOr(status, red.err);
}

// Labelling only: frozen occupation bytes in, canonical labels out.
template <int NT>
__global__ void __launch_bounds__(NT, MinBlocks<NT>::value)
    k_resident_label(uint32_t L, const uint8_t *occ, int32_t *labels, int32_t *n_clusters, uint8_t *wraps,
                     int *status, ResidentLayout ly)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ Red<NT> red;
    __shared__ uint32_t s_scan[NT];
    const uint32_t tid = threadIdx.x;
    const size_t lat = blockIdx.x;
    if (tid == 0) {
        red.err = 0;
        red.wrap = 0;
    }
    const Res res = make_res<NT>(smem, ly, L, red);
    const Lat<Word16> &t = res.t;
    const Geom g = t.g;
    const uint8_t *o = occ + lat * 2ull * g.N;
    for (uint32_t i = tid; i < (L + 31u) / 32u; i += NT) t.SEAMV[i] = 0u;
    init_row_ends(t, tid, NT);
    __syncthreads();
    for (uint32_t w = tid; w < g.NW; w += NT) {
        uint32_t h = 0, v = 0;
        for (uint32_t b = 0; b < 32u; ++b) {
            const uint32_t n = (w << 5) + b;
            if (n >= g.N) break;
            h |= (o[2ull * n] ? 1u : 0u) << b;
            v |= (o[2ull * n + 1] ? 1u : 0u) << b;
        }
        const uint32_t re = g.row_end(w);
        t.OH[w] = h;
        t.OV[w] = v & ~re;
        uint32_t seam = v & re;
        while (seam) {
            const uint32_t b = __ffs(seam) - 1u;
            seam &= seam - 1u;
            const uint32_t x = ((w << 5) + b) / L;
            atomicOr(t.SEAMV + (x >> 5), 1u << (x & 31u));
        }
    }
    __syncthreads();
    resident_label<NT>(res, false, false);
    // Exclusive prefix of root counts over words -> FLIP plane (rank base).
    const uint32_t per = (g.NW + NT - 1u) / NT;
    const uint32_t w0 = tid * per, w1 = min(g.NW, w0 + per);
    uint32_t local = 0;
    for (uint32_t w = w0; w < w1; ++w) local += __popc(t.ROOT[w]);
    s_scan[tid] = local;
    __syncthreads();
    for (uint32_t off = 1; off < NT; off <<= 1) {
        const uint32_t v = tid >= off ? s_scan[tid - off] : 0u;
        __syncthreads();
        s_scan[tid] += v;
        __syncthreads();
    }
    uint32_t base = s_scan[tid] - local;
    for (uint32_t w = w0; w < w1; ++w) {
        t.FLIP[w] = base;
        base += __popc(t.ROOT[w]);
    }
    __syncthreads();
    int32_t *lab = labels + lat * (size_t)g.N;
    for (uint32_t n = tid; n < g.N; n += NT) {
        const uint32_t r = Word16::parent(t.uf.ld(n));
        lab[n] = (int32_t)(t.FLIP[r >> 5] + __popc(t.ROOT[r >> 5] & ((1u << (r & 31u)) - 1u)));
    }
    if (tid == 0) {
        n_clusters[lat] = (int32_t)s_scan[NT - 1];
        wraps[2 * lat] = (uint8_t)(red.wrap & 1);
        wraps[2 * lat + 1] = (uint8_t)((red.wrap >> 1) & 1);
        if (red.err) atomicOr(status, red.err);
    }
}

namespace {

template <int NT, int LC>
cudaError_t launch_sweeps_lc(const rbim_chain_t *chains, int n_chains, int l_max, uint32_t *spin_pool,
                             const uint32_t *coupling_pool, long long *acc_i, double *acc_f, int32_t *rec,
                             int n_sweeps, int grid, int *queue, int *status, cudaStream_t stream)
{
    const ResidentLayout ly = LC > 0 ? resident_layout_c(LC) : resident_layout(l_max, NT);
    cudaError_t e = cudaFuncSetAttribute(k_resident_sweeps<NT, LC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)ly.bytes);
    if (e != cudaSuccess) return e;
    if (grid <= 0) {
        int per_sm = 0, sms = 0, dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_resident_sweeps<NT, LC>, NT, ly.bytes);
        if (e != cudaSuccess) return e;
        grid = std::max(1, per_sm) * sms;
    }
    grid = std::min(grid, n_chains);
    e = cudaMemsetAsync(queue, 0, sizeof(int), stream);
    if (e != cudaSuccess) return e;
    k_resident_sweeps<NT, LC><<<grid, NT, ly.bytes, stream>>>(const_cast<rbim_chain_t *>(chains), n_chains, spin_pool,
                                                          coupling_pool, acc_i, acc_f, rec, n_sweeps, queue,
                                                          status, ly);
    return cudaGetLastError();
}

// Size classes with a compile-time layout, at their default thread counts:
// 128 < L <= 256 (1024 threads), 96 < L <= 128 and 128 < L <= 176 (512),
// 64 < L <= 96 (256).  Below L = 64 (CTAs of 64 and 128 threads) the
// run-time layout measured 5-7% faster than a compile-time one on B200.
template <int NT>
cudaError_t launch_sweeps_nt(const rbim_chain_t *chains, int n_chains, int l_max, uint32_t *spin_pool,
                             const uint32_t *coupling_pool, long long *acc_i, double *acc_f, int32_t *rec,
                             int n_sweeps, int grid, int *queue, int *status, cudaStream_t stream)
{
    if (NT == 1024 && l_max > 128 && l_max <= 256)
        return launch_sweeps_lc<NT, 256>(chains, n_chains, l_max, spin_pool, coupling_pool, acc_i, acc_f, rec,
                                         n_sweeps, grid, queue, status, stream);
    if (NT == 512 && l_max > 96 && l_max <= 128)
        return launch_sweeps_lc<NT, 128>(chains, n_chains, l_max, spin_pool, coupling_pool, acc_i, acc_f, rec,
                                         n_sweeps, grid, queue, status, stream);
    if (NT == 512 && l_max > 128 && l_max <= 176 &&
        2 * (resident_layout_c(176).bytes + kStaticSmem) <= kSmemPerSm)
        return launch_sweeps_lc<NT, 176>(chains, n_chains, l_max, spin_pool, coupling_pool, acc_i, acc_f, rec,
                                         n_sweeps, grid, queue, status, stream);
    if (NT == 256 && l_max > 64 && l_max <= 96)
        return launch_sweeps_lc<NT, 96>(chains, n_chains, l_max, spin_pool, coupling_pool, acc_i, acc_f, rec,
                                        n_sweeps, grid, queue, status, stream);
    return launch_sweeps_lc<NT, 0>(chains, n_chains, l_max, spin_pool, coupling_pool, acc_i, acc_f, rec, n_sweeps,
                                   grid, queue, status, stream);
}

template <int NT>
cudaError_t launch_label_nt(int L, int n_lattices, const uint8_t *occ, int32_t *labels, int32_t *ncl,
                            uint8_t *wraps, int *status, cudaStream_t stream)
{
    const ResidentLayout ly = resident_layout(L, NT);
    cudaError_t e = cudaFuncSetAttribute(k_resident_label<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)ly.bytes);
    if (e != cudaSuccess) return e;
    k_resident_label<NT><<<n_lattices, NT, ly.bytes, stream>>>(L, occ, labels, ncl, wraps, status, ly);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_resident_sweeps(const rbim_chain_t *chains, int n_chains, int l_max, uint32_t *spin_pool,
                                   const uint32_t *coupling_pool, long long *acc_i, double *acc_f, int32_t *rec,
                                   int n_sweeps, int threads, int grid, int *queue, int *status,
                                   cudaStream_t stream)
{
    if (threads <= 0) threads = resident_default_threads(l_max);
    switch (threads) {
    case 32:
        return launch_sweeps_nt<32>(chains, n_chains, l_max, spin_pool, coupling_pool, acc_i, acc_f, rec, n_sweeps,
                                    grid, queue, status, stream);
    case 64:
        return launch_sweeps_nt<64>(chains, n_chains, l_max, spin_pool, coupling_pool, acc_i, acc_f, rec, n_sweeps,
                                    grid, queue, status, stream);
    case 128:
        return launch_sweeps_nt<128>(chains, n_chains, l_max, spin_pool, coupling_pool, acc_i, acc_f, rec, n_sweeps,
                                     grid, queue, status, stream);
    case 256:
        return launch_sweeps_nt<256>(chains, n_chains, l_max, spin_pool, coupling_pool, acc_i, acc_f, rec, n_sweeps,
                                     grid, queue, status, stream);
    case 512:
        return launch_sweeps_nt<512>(chains, n_chains, l_max, spin_pool, coupling_pool, acc_i, acc_f, rec, n_sweeps,
                                     grid, queue, status, stream);
    case 1024:
        return launch_sweeps_nt<1024>(chains, n_chains, l_max, spin_pool, coupling_pool, acc_i, acc_f, rec,
                                      n_sweeps, grid, queue, status, stream);
    default:
        return cudaErrorInvalidValue;
    }
}

cudaError_t launch_resident_label(int L, int n_lattices, const uint8_t *occ, int32_t *labels, int32_t *n_clusters,
                                  uint8_t *wraps, int threads, int *status, cudaStream_t stream)
{
    // The labelling kernel keeps at least two warps per CTA.
    if (threads <= 0) threads = std::max(64, resident_default_threads(L));
    switch (threads) {
    case 64:
        return launch_label_nt<64>(L, n_lattices, occ, labels, n_clusters, wraps, status, stream);
    case 128:
        return launch_label_nt<128>(L, n_lattices, occ, labels, n_clusters, wraps, status, stream);
    case 256:
        return launch_label_nt<256>(L, n_lattices, occ, labels, n_clusters, wraps, status, stream);
    case 512:
        return launch_label_nt<512>(L, n_lattices, occ, labels, n_clusters, wraps, status, stream);
    case 1024:
        return launch_label_nt<1024>(L, n_lattices, occ, labels, n_clusters, wraps, status, stream);
    default:
        return cudaErrorInvalidValue;
    }
}

}  // namespace rbim

#ifdef RBIM_PROFILE_PHASES
// Profiling builds only: copy out (and optionally reset) the per-phase cycle
// counters of the resident engine.
extern "C" int rbim_profile_phase_cycles(unsigned long long *out, int reset)
{
    cudaError_t e = cudaMemcpyFromSymbol(out, rbim::g_phase_cycles, sizeof(unsigned long long) * 16);
    if (e == cudaSuccess && reset) {
        const unsigned long long z[16] = {};
        e = cudaMemcpyToSymbol(rbim::g_phase_cycles, z, sizeof(z));
    }
    return e == cudaSuccess ? 0 : -2;
}

// Profiling builds only: event counters (0 unions, 1 find steps, 2 failed CAS).
extern "C" int rbim_profile_event_counts(unsigned long long *out, int reset)
{
    cudaError_t e = cudaMemcpyFromSymbol(out, rbim::g_event_counts, sizeof(unsigned long long) * 8);
    if (e == cudaSuccess && reset) {
        const unsigned long long z[8] = {};
        e = cudaMemcpyToSymbol(rbim::g_event_counts, z, sizeof(z));
    }
    return e == cudaSuccess ? 0 : -2;
}
#endif

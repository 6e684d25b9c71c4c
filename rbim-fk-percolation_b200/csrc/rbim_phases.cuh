// The four stages of one Swendsen-Wang sweep, written once over a lattice
// context whose planes and union-find words may live in shared memory (the
// resident engine) or in global memory (the plain engine).  Each phase is a
// loop over work items (64-site chunks or 32-site words) taking `first` and
// `stride` so that a CTA or the whole grid can share the items; callers put a
// barrier between phases.
//
// Reference correspondence:
//   phase_activate  -> src/rbim/clusters.py:48-79 (activate_bonds)
//   phase_heads     -> union-find initialisation, src/rbim/_unionfind.py:97-100,
//                      with runs of occupied y-bonds pre-joined
//   phase_union     -> src/rbim/_unionfind.py:104-124 (union and loop winding)
//   phase_finalize  -> src/rbim/_unionfind.py:126-134 (roots) and the flip of
//                      src/rbim/swendsen_wang.py:140-141
//   phase_*measure* -> src/rbim/clusters.py:98-118, src/rbim/swendsen_wang.py:81-100
#pragma once

#include "rbim_device.cuh"

namespace rbim {

template <class WT>
struct Lat {
    Geom g;
    UF<WT> uf;
    uint32_t *S;           // spins (read in A, written in D)
    const uint32_t *JH;    // couplings
    const uint32_t *JV;
    uint32_t *OH, *OV;     // occupied bonds
    uint32_t *SEAMV;       // occupied y-seam bonds, bit x = row x
    uint32_t *FLIP, *ROOT;
    const uint32_t *RE;    // row-end masks per word (Geom::row_end), or null to compute them
    int *wrap;             // bit 0 wrap_x, bit 1 wrap_y
    int *err;
    uint32_t cap;          // bound on the steps of one walk (N + 64 unless a chain's walk_cap lowers it)
    __device__ __forceinline__ uint32_t row_end(uint32_t w) const { return RE ? RE[w] : g.row_end(w); }
};

struct SweepRng {
    uint64_t key;
    uint64_t sweep;
    uint32_t thr_hi;  // threshold >> 16
    uint32_t thr_lo;  // threshold & 0xFFFF
    bool thr_all;     // threshold == 2^32: every satisfied bond is occupied
};

__device__ __forceinline__ SweepRng make_rng(uint64_t key, uint64_t sweep, uint64_t thr)
{
    SweepRng r;
    r.key = key;
    r.sweep = sweep;
    r.thr_all = thr >= (1ull << 32);
    r.thr_hi = (uint32_t)(thr >> 16) & 0xFFFFu;
    r.thr_lo = (uint32_t)thr & 0xFFFFu;
    return r;
}

// Occupation decision of one bond from its 16-bit draw u: u < thr_hi
// accepts, u > thr_hi rejects, u == thr_hi (probability 2^-16) defers to the
// low half v, drawn separately.  Returns 0 reject, 1 accept, 2 undecided.
__device__ __forceinline__ uint32_t bond_decide(const SweepRng &rng, uint32_t u)
{
    if (rng.thr_all || u < rng.thr_hi) return 1u;
    return u == rng.thr_hi ? 2u : 0u;
}

// Acceptance of one lane's Philox block of bond draws: bit s of the result
// accepts the horizontal bond of word s (low half of word s of the block),
// bit 4 + s the vertical one (high half); satisfied masks are applied later.
// A 16-bit draw equal to thr >> 16 defers to the low half drawn from stream
// 3 (probability 2^-16 per bond), fetched when any lane of the warp needs it.
__device__ __forceinline__ uint32_t accept_block(const SweepRng &rng, const U4 &r, uint32_t block)
{
    uint32_t acc = 0, eq = 0;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        const uint32_t w = u4_word(r, s);
        const uint32_t lo = w & 0xFFFFu, hi = w >> 16;
        acc |= ((rng.thr_all || lo < rng.thr_hi) ? 1u : 0u) << s;
        acc |= ((rng.thr_all || hi < rng.thr_hi) ? 1u : 0u) << (4 + s);
        eq |= ((lo == rng.thr_hi) ? 1u : 0u) << s;
        eq |= ((hi == rng.thr_hi) ? 1u : 0u) << (4 + s);
    }
    if (!rng.thr_all && __any_sync(0xFFFFFFFFu, eq != 0u)) {
        const U4 q = philox_block(rng.key, block, rng.sweep, kStreamBondLow);
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const uint32_t w = u4_word(q, s);
            if ((eq >> s) & 1u) acc |= ((w & 0xFFFFu) < rng.thr_lo ? 1u : 0u) << s;
            if ((eq >> (4 + s)) & 1u) acc |= ((w >> 16) < rng.thr_lo ? 1u : 0u) << (4 + s);
        }
    }
    return acc;
}

// (a) Bond activation.  A 128-site chunk is four plane words; lane i of the
// warp handling chunk c draws Philox block 32c + i, whose word s holds the
// 16-bit draws of the horizontal (low half) and vertical (high half) bond of
// site 128c + 32s + i, i.e. bit i of the chunk's word s, so that each ballot
// is one word of the occupied-bond planes.  A warp takes a group of G
// consecutive words (G = 32, eight chunks, while every warp still gets a
// group): lane j first forms the satisfied masks of word j of the group --
// every lane busy, coalesced loads -- then the warp draws the group's chunks
// two at a time, and lane j keeps the ballots of its own word.  SEAMV must be
// zero on entry.
template <class WT>
__device__ __forceinline__ void phase_activate_bonds(const Lat<WT> &t, const SweepRng &rng, uint32_t warp,
                                                     uint32_t nwarps)
{
    const uint32_t lane = threadIdx.x & 31u;
    const Geom &g = t.g;
    Plane S{t.S};
    uint32_t G = 32u;
    while (G > 4u && G * nwarps > g.NW) G >>= 1;
    const uint32_t ngroups = (g.NW + G - 1u) / G;
    const uint32_t nchunks = (g.NW + 3u) >> 2;
    const uint32_t my_chunk = lane >> 2, my_s = lane & 3u;
    for (uint32_t grp = warp; grp < ngroups; grp += nwarps) {
        const uint32_t w = grp * G + lane;
        const bool mine = lane < G && w < g.NW;
        uint32_t sh = 0, sv = 0, re = 0;
        if (mine) {
            re = t.row_end(w);
            const uint32_t v = g.valid(w);
            const uint32_t s = S(w);
            sh = ~(s ^ xnext_word(S, w, g) ^ t.JH[w]) & v;
            sv = ~(s ^ ynext_word(S, w, g, re) ^ t.JV[w]) & v;
        }
        const uint32_t c0 = grp * (G >> 2);
        const uint32_t nch = min(G >> 2, nchunks - c0);
        uint32_t oh = 0, ov = 0;
        // Two chunks per iteration: two independent Philox evaluations per lane.
        for (uint32_t k = 0; k < nch; k += 2u) {
            const bool two = k + 1u < nch;
            const U4 r0 = philox_block(rng.key, 32u * (c0 + k) + lane, rng.sweep, kStreamBond);
            U4 r1{};
            if (two) r1 = philox_block(rng.key, 32u * (c0 + k + 1u) + lane, rng.sweep, kStreamBond);
            const uint32_t a0 = accept_block(rng, r0, 32u * (c0 + k) + lane);
            const uint32_t a1 = two ? accept_block(rng, r1, 32u * (c0 + k + 1u) + lane) : 0u;
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                const uint32_t bh0 = __ballot_sync(0xFFFFFFFFu, (a0 >> s) & 1u);
                const uint32_t bv0 = __ballot_sync(0xFFFFFFFFu, (a0 >> (4 + s)) & 1u);
                const uint32_t bh1 = __ballot_sync(0xFFFFFFFFu, (a1 >> s) & 1u);
                const uint32_t bv1 = __ballot_sync(0xFFFFFFFFu, (a1 >> (4 + s)) & 1u);
                if (my_s == (uint32_t)s) {
                    if (my_chunk == k) {
                        oh = bh0;
                        ov = bv0;
                    } else if (my_chunk == k + 1u) {
                        oh = bh1;
                        ov = bv1;
                    }
                }
            }
        }
        if (mine) {
            oh &= sh;
            ov &= sv;
            t.OH[w] = oh;
            t.OV[w] = ov & ~re;
            uint32_t seam = ov & re;
            while (seam) {
                const uint32_t b = __ffs(seam) - 1u;
                seam &= seam - 1u;
                const uint32_t x = ((w << 5) + b) / g.L;
                atomicOr(t.SEAMV + (x >> 5), 1u << (x & 31u));
            }
        }
    }
}

// (a') Cluster flip bits: Philox block q of stream 1 gives FLIP words 4q .. 4q+3.
template <class WT>
__device__ __forceinline__ void phase_flip_bits(const Lat<WT> &t, const SweepRng &rng, uint32_t tid,
                                                uint32_t nthreads)
{
    const Geom &g = t.g;
    const uint32_t nblk = (g.NW + 3u) >> 2;
    for (uint32_t q = tid; q < nblk; q += nthreads) {
        const U4 r = philox_block(rng.key, q, rng.sweep, kStreamFlip);
        const uint32_t w = 4u * q;
        t.FLIP[w] = r.x;
        if (w + 1u < g.NW) t.FLIP[w + 1u] = r.y;
        if (w + 2u < g.NW) t.FLIP[w + 2u] = r.z;
        if (w + 3u < g.NW) t.FLIP[w + 3u] = r.w;
    }
}

template <class WT>
__device__ __forceinline__ void phase_activate(const Lat<WT> &t, const SweepRng &rng, uint32_t warp,
                                               uint32_t nwarps, uint32_t tid, uint32_t nthreads)
{
    phase_activate_bonds<WT>(t, rng, warp, nwarps);
    phase_flip_bits<WT>(t, rng, tid, nthreads);
}

// Head-of-run mask of word w: a site heads its run unless the y-bond from the
// previous site is occupied (seam bonds are absent from OV, so row starts are
// always heads).
__device__ __forceinline__ uint32_t head_mask(const uint32_t *OV, uint32_t w, uint32_t valid)
{
    const uint32_t ov = OV[w];
    const uint32_t prev = w ? (OV[w - 1u] >> 31) : 0u;
    return ~((ov << 1) | prev) & valid;
}

// (b) Union-find initialisation: every site points at the head of its run of
// occupied y-bonds with zero image offset (runs never cross a seam).  A warp
// takes B consecutive words at a time: lane j finds the last head of word j,
// a max-scan over the lanes gives every word the last head before it, and
// the warp then writes the B words one after the other, one site per lane.
template <class WT>
__device__ __forceinline__ void phase_heads(const Lat<WT> &t, uint32_t warp, uint32_t nwarps)
{
    const uint32_t lane = threadIdx.x & 31u;
    const Geom &g = t.g;
    uint32_t B = 32;
    while (B > 1u && B * nwarps > g.NW) B >>= 1;
    for (uint32_t base = warp * B; base < g.NW; base += nwarps * B) {
        const uint32_t wj = base + lane;
        const bool has = lane < B && wj < g.NW;
        const uint32_t h = has ? head_mask(t.OV, wj, g.valid(wj)) : 0u;
        // Positions are stored + 1, so that 0 means "no head yet".
        uint32_t pre = 0;  // last head before word base (lane 0)
        if (lane == 0 && base > 0 && !(h & 1u)) {
            // Site 0 always heads a run, so this walk back ends.
            for (uint32_t ww = base; ww-- > 0;) {
                const uint32_t hh = head_mask(t.OV, ww, 0xFFFFFFFFu);
                if (hh) {
                    pre = (ww << 5) + 32u - __clz(hh);
                    break;
                }
            }
        }
        uint32_t incl = max(h ? (wj << 5) + 32u - __clz(h) : 0u, pre);
#pragma unroll
        for (uint32_t o = 1; o < 32u; o <<= 1) {
            const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= o) incl = max(incl, v);
        }
        // Last head before word j: the scan of lanes < j, or pre for j = 0.
        uint32_t before = __shfl_up_sync(0xFFFFFFFFu, incl, 1);
        if (lane == 0) before = pre;
        if constexpr (sizeof(typename WT::T) == 2) {
            // 16-bit parents: two words per step, each lane writing the parents
            // of two neighbouring sites with one 32-bit store (lanes 0-15 word
            // j, lanes 16-31 word j + 1); sites past N are not written.
            const uint32_t half = lane >> 4, b0 = 2u * (lane & 15u);
            for (uint32_t j = 0; j < B; j += 2u) {
                const uint32_t jj = j + half;
                const uint32_t hj = __shfl_sync(0xFFFFFFFFu, h, jj & 31u);
                const uint32_t cj = __shfl_sync(0xFFFFFFFFu, before, jj & 31u);
                const uint32_t w = base + jj;
                if (jj >= B || w >= g.NW) continue;
                const uint32_t n = (w << 5) + b0;
                const uint32_t m0 = hj & mask_le(b0), m1 = hj & mask_le(b0 + 1u);
                const uint32_t h0 = m0 ? (w << 5) + 31u - __clz(m0) : cj - 1u;
                const uint32_t h1 = m1 ? (w << 5) + 31u - __clz(m1) : cj - 1u;
                if (n + 1u < g.N)
                    t.uf.st2(n, h0 | (h1 << 16));
                else if (n < g.N)
                    t.uf.st(n, WT::make(h0, 0, 0));
            }
        } else {
            for (uint32_t j = 0; j < B; ++j) {
                const uint32_t w = base + j;
                if (w >= g.NW) break;
                const uint32_t hj = __shfl_sync(0xFFFFFFFFu, h, j);
                const uint32_t cj = __shfl_sync(0xFFFFFFFFu, before, j);
                const uint32_t n = (w << 5) + lane;
                if (n < g.N) {
                    const uint32_t m = hj & mask_le(lane);
                    const uint32_t head = m ? (w << 5) + 31u - __clz(m) : cj - 1u;
                    t.uf.st(n, WT::make(head, 0, 0));
                }
            }
        }
    }
}

// Work slices.  Pointer chasing has data-dependent length, so the union and
// root phases run as flat per-thread loops that take one pointer step per
// iteration and fetch the next item as soon as the current one is done; a
// thread's cost is then the sum of its items' steps rather than a per-round
// maximum over the warp.  Thread t owns the bit ranges t, t + T, t + 2T, ...
// where each word is cut into `seg` equal ranges (seg is a power of two
// chosen so that small lattices still give every thread work).
struct Slices {
    uint32_t seg_log2, bits, items;
    __device__ __forceinline__ uint32_t word(uint32_t i) const { return i >> seg_log2; }
    __device__ __forceinline__ uint32_t mask(uint32_t i) const
    {
        const uint32_t s = i & ((1u << seg_log2) - 1u);
        return (bits == 32u ? 0xFFFFFFFFu : ((1u << bits) - 1u)) << (s * bits);
    }
};

__device__ __forceinline__ Slices make_slices(uint32_t NW, uint32_t nthreads)
{
    uint32_t lg = 0;
    while (lg < 5u && (NW << (lg + 1u)) <= nthreads) ++lg;
    return Slices{lg, 32u >> lg, NW << lg};
}

// Occupied x-bonds of word w that need a union, the x seam included.  A bond
// is skipped when the bond one step lower in y is occupied and both y-bonds
// joining them are occupied: it then closes an elementary plaquette, which is
// contractible and already connected (across the x seam the plaquette
// crosses the seam once each way).
template <class WT>
__device__ __forceinline__ uint32_t x_union_need(const Lat<WT> &t, uint32_t w)
{
    const Geom &g = t.g;
    const uint32_t oh = t.OH[w];
    if (!oh) return 0u;
    Plane OVp{t.OV};
    const uint32_t ohp = w ? t.OH[w - 1u] : 0u;
    const uint32_t ov = OVp(w), ovp = w ? OVp(w - 1u) : 0u;
    const uint32_t prev_oh = (oh << 1) | (ohp >> 31);
    const uint32_t prev_ov = (ov << 1) | (ovp >> 31);
    uint32_t s = (w << 5) + g.N + g.L - 1u;
    s %= g.N;
    return oh & ~(prev_oh & prev_ov & extract32(OVp, s, g));
}

// One endpoint walk of a union: the current node, its word as last read, and
// the summed image offset from the walk's start to the node.
template <class WT>
struct Walk {
    typename WT::T w;
    uint32_t node;
    int ax, ay;
};

// One path-halving step (src/rbim/_unionfind.py:59-88: the offsets of the
// skipped link are folded into the halved pointer).  Returns true, without
// moving, when the walk stands on a node whose word says it is a root.  The
// words are read with UF::ldc; a word that is out of date only makes the walk
// stop short on a former root, where the CAS of the union fails and reloads.
template <class WT>
__device__ __forceinline__ bool walk_step(const UF<WT> &uf, Walk<WT> &k)
{
    const uint32_t p = WT::parent(k.w);
    if (p == k.node) return true;
    const typename WT::T wp = uf.ldc(p);
    const uint32_t gp = WT::parent(wp);
    if (gp != p) {
        const int nx = WT::ox(k.w) + WT::ox(wp), ny = WT::oy(k.w) + WT::oy(wp);
        uf.st(k.node, WT::make(gp, nx, ny));
        k.ax += nx;
        k.ay += ny;
        k.node = gp;
        k.w = uf.ldc(gp);
    } else {
        k.ax += WT::ox(k.w);
        k.ay += WT::oy(k.w);
        k.node = p;
        k.w = wp;
    }
    return false;
}

// (b) Unions across occupied x-bonds (including the x seam, image offset
// (1,0)) and the y seam ((0,1)), with the loop-winding test of
// src/rbim/_unionfind.py:104-124.  The x-bonds run as one flat loop per
// thread over its work slices: both endpoint walks advance one step per
// iteration, and the thread takes its next bond as soon as the current union
// is done.  The larger root is hooked under the smaller with a CAS on
// its (self, 0, 0) word; a lost race resumes both walks from where they stand.
template <class WT>
__device__ __forceinline__ void phase_union(const Lat<WT> &t, uint32_t tid, uint32_t nthreads)
{
    using T = typename WT::T;
    const Geom &g = t.g;
    const UF<WT> &uf = t.uf;
    const Slices sl = make_slices(g.NW, nthreads);
    uint32_t item = tid, pending = 0, base = 0;
    Walk<WT> a{}, b{};
    int ex = 0;
    bool fetch = true;
    const unsigned long long cap = 64ull * t.cap;  // 64 walks of t.cap steps (64 N + 4096 by default)
    for (unsigned long long it = 0;; ++it) {
        if (it >= cap) {
            atomicOr(t.err, kErrUnionCap);
            break;
        }
        if (fetch) {
            while (!pending && item < sl.items) {
                const uint32_t w = sl.word(item);
                pending = x_union_need(t, w) & sl.mask(item);
                base = w << 5;
                item += nthreads;
            }
            if (!pending) break;
            const uint32_t n = base + (uint32_t)(__ffs(pending) - 1);
            pending &= pending - 1u;
            uint32_t m = n + g.L;
            ex = 0;
            if (m >= g.N) {
                m -= g.N;
                ex = 1;
            }
            a = Walk<WT>{uf.ldc(n), n, 0, 0};
            b = Walk<WT>{uf.ldc(m), m, 0, 0};
            fetch = false;
        }
        const bool ra = walk_step<WT>(uf, a);
        const bool rb = walk_step<WT>(uf, b);
        if (!(ra && rb)) continue;
        if (a.node == b.node) {
            int f = 0;
            if (WT::nonzero(ex + b.ax - a.ax)) f |= 1;
            if (WT::nonzero(b.ay - a.ay)) f |= 2;
            if (f) atomicOr(t.wrap, f);
            fetch = true;
        } else if (a.node < b.node) {
            const T expect = WT::make(b.node, 0, 0);
            const T old = uf.cas(b.node, expect, WT::make(a.node, a.ax - ex - b.ax, a.ay - b.ay));
            if (old == expect) {
                fetch = true;
            } else {
                b.w = old;
                a.w = uf.ld(a.node);
            }
        } else {
            const T expect = WT::make(a.node, 0, 0);
            const T old = uf.cas(a.node, expect, WT::make(b.node, b.ax + ex - a.ax, b.ay - a.ay));
            if (old == expect) {
                fetch = true;
            } else {
                a.w = old;
                b.w = uf.ld(b.node);
            }
        }
    }
    // y seam: (x, L-1) -> (x, 0) with image offset (0, 1).
    for (uint32_t x = tid; x < g.L; x += nthreads) {
        if ((t.SEAMV[x >> 5] >> (x & 31u)) & 1u) {
            const uint32_t a0 = x * g.L + g.L - 1u;
            uf_union<WT>(t.uf, a0, x * g.L, 0, 1, t.wrap, t.cap, t.err);
        }
    }
}

// (c) Roots of the run heads.  Every parent pointer targets a head (heads
// are the initial parents, roots are heads, and hooks and path halving only
// move pointers to roots or grandparents), so once each head points straight
// at its root, every site reaches its root in two steps.  The walks only
// read, and each head's word is written by the head's own thread alone, so
// no final pointer can be overwritten by a stale ancestor.  A flat loop per
// thread over the heads of its work slices, two walks in flight; roots are
// recorded in ROOT, which must be zero on entry.  Returns this thread's
// number of roots.
template <class WT>
__device__ __forceinline__ bool next_head_of(const Lat<WT> &t, const Slices &sl, uint32_t nthreads, uint32_t &item,
                                             uint32_t &pending, uint32_t &base, uint32_t &h)
{
    while (!pending && item < sl.items) {
        const uint32_t w = sl.word(item);
        pending = head_mask(t.OV, w, t.g.valid(w)) & sl.mask(item);
        base = w << 5;
        item += nthreads;
    }
    if (!pending) return false;
    h = base + (uint32_t)(__ffs(pending) - 1);
    pending &= pending - 1u;
    return true;
}

template <class WT>
__device__ __forceinline__ uint32_t phase_roots(const Lat<WT> &t, uint32_t tid, uint32_t nthreads)
{
    const Geom &g = t.g;
    const Slices sl = make_slices(g.NW, nthreads);
    uint32_t item = tid, pending = 0, base = 0, nroots = 0;
    uint32_t h0 = 0, h1 = 0;
    bool a0 = next_head_of(t, sl, nthreads, item, pending, base, h0);
    bool a1 = a0 && next_head_of(t, sl, nthreads, item, pending, base, h1);
    uint32_t x0 = h0, x1 = h1;
    const unsigned long long cap = 64ull * t.cap;  // 64 walks of t.cap steps (64 N + 4096 by default)
    for (unsigned long long it = 0; a0 || a1; ++it) {
        if (it >= cap) {
            atomicOr(t.err, kErrFindCap);
            break;
        }
        const uint32_t p0 = a0 ? WT::parent(t.uf.ldc(x0)) : x0;
        const uint32_t p1 = a1 ? WT::parent(t.uf.ldc(x1)) : x1;
        const bool r0 = a0 && p0 == x0, r1 = a1 && p1 == x1;
        x0 = p0;
        x1 = p1;
        if (r0) {
            if (x0 != h0) {
                t.uf.st(h0, WT::make(x0, 0, 0));
            } else {
                atomicOr(t.ROOT + (h0 >> 5), 1u << (h0 & 31u));
                ++nroots;
            }
            a0 = next_head_of(t, sl, nthreads, item, pending, base, h0);
            x0 = h0;
        }
        if (r1) {
            if (x1 != h1) {
                t.uf.st(h1, WT::make(x1, 0, 0));
            } else {
                atomicOr(t.ROOT + (h1 >> 5), 1u << (h1 & 31u));
                ++nroots;
            }
            a1 = next_head_of(t, sl, nthreads, item, pending, base, h1);
            x1 = h1;
        }
    }
    return nroots;
}

// (c') Every site: root = parent of parent (after phase_roots), pointed at
// directly; the spin is flipped with its cluster's flip bit; with `count` the
// root words accumulate the cluster size in their offset field
// (warp-aggregated with match_any).  A site's parent is a head and a head's
// parent is its root, so the parent fields read here are final and the loads
// may come from L1 (the count adds change only the root words' upper half).
template <class WT>
__device__ __forceinline__ void phase_sites(const Lat<WT> &t, uint32_t warp, uint32_t nwarps, bool flip, bool count)
{
    const uint32_t lane = threadIdx.x & 31u;
    const Geom &g = t.g;
    // Two words per iteration (w0 and w1 = w0 + nwarps) keep two independent
    // chains of loads in flight.  With `count`, each warp carries the size of
    // one cluster -- the one of its first site -- across its words and adds
    // it once at the end: when one cluster spans most of the lattice its root
    // would otherwise take an atomic per word from every warp, all on one
    // address.
    uint32_t carried = 0xFFFFFFFFu, carried_n = 0;
    for (uint32_t w0 = warp; w0 < g.NW; w0 += 2u * nwarps) {
        const uint32_t w1 = w0 + nwarps;
        const uint32_t n0 = (w0 << 5) + lane, n1 = (w1 << 5) + lane;
        const bool ok0 = n0 < g.N, ok1 = n1 < g.N;
        uint32_t r0 = 0, r1 = 0, p0 = 0, p1 = 0;
        if (ok0) p0 = WT::parent(t.uf.ldc(n0));
        if (ok1) p1 = WT::parent(t.uf.ldc(n1));
        if (ok0) r0 = WT::parent(t.uf.ldc(p0));
        if (ok1) r1 = WT::parent(t.uf.ldc(p1));
        if (ok0 && r0 != p0) t.uf.st(n0, WT::make(r0, 0, 0));
        if (ok1 && r1 != p1) t.uf.st(n1, WT::make(r1, 0, 0));
        if (flip) {
            const uint32_t f0 = ok0 ? (t.FLIP[r0 >> 5] >> (r0 & 31u)) & 1u : 0u;
            const uint32_t f1 = ok1 ? (t.FLIP[r1 >> 5] >> (r1 & 31u)) & 1u : 0u;
            const uint32_t s0 = t.S[w0], s1 = w1 < g.NW ? t.S[w1] : 0u;
            const uint32_t ns0 = __ballot_sync(0xFFFFFFFFu, ok0 && (((s0 >> lane) & 1u) ^ f0)) & g.valid(w0);
            const uint32_t ns1 = __ballot_sync(0xFFFFFFFFu, ok1 && (((s1 >> lane) & 1u) ^ f1));
            if (lane == 0) t.S[w0] = ns0;
            if (lane == 1 && w1 < g.NW) t.S[w1] = ns1 & g.valid(w1);
        }
        if (count) {
            // Lane 0's site of the warp's first word exists (w0 < NW).
            if (carried == 0xFFFFFFFFu) carried = __shfl_sync(0xFFFFFFFFu, r0, 0);
            const uint32_t c0 = __ballot_sync(0xFFFFFFFFu, ok0 && r0 == carried);
            const uint32_t c1 = __ballot_sync(0xFFFFFFFFu, ok1 && r1 == carried);
            carried_n += __popc(c0) + __popc(c1);
            const uint32_t rest0 = __ballot_sync(0xFFFFFFFFu, ok0) & ~c0;
            if ((rest0 >> lane) & 1u) {
                const uint32_t grp = __match_any_sync(rest0, r0);
                if (lane == (uint32_t)(__ffs(grp) - 1)) t.uf.add(r0, WT::count_inc(__popc(grp)));
            }
            const uint32_t rest1 = __ballot_sync(0xFFFFFFFFu, ok1) & ~c1;
            if ((rest1 >> lane) & 1u) {
                const uint32_t grp = __match_any_sync(rest1, r1);
                if (lane == (uint32_t)(__ffs(grp) - 1)) t.uf.add(r1, WT::count_inc(__popc(grp)));
            }
        }
    }
    if (count && lane == 0 && carried_n) t.uf.add(carried, WT::count_inc(carried_n));
}

// (d) Unsatisfied bonds and down spins over words first, first+stride, ...
template <class WT>
__device__ __forceinline__ void measure_energy(const Lat<WT> &t, uint32_t first, uint32_t stride, uint32_t &unsat,
                                               uint32_t &downs)
{
    const Geom &g = t.g;
    Plane Sp{t.S};
    for (uint32_t w = first; w < g.NW; w += stride) {
        const uint32_t v = g.valid(w);
        const uint32_t s = Sp(w);
        unsat += __popc((s ^ xnext_word(Sp, w, g) ^ t.JH[w]) & v);
        unsat += __popc((s ^ ynext_word(Sp, w, g, t.row_end(w)) ^ t.JV[w]) & v);
        downs += __popc(s & v);
    }
}

}  // namespace rbim

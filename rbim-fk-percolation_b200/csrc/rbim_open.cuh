// Open-lattice labelling on a 16-bit shared-memory union-find, shared by the
// resident engine (one lattice per CTA) and the cluster engine (one tile of a
// lattice per CTA).  Inside an open region of the lattice (no bond that
// crosses a periodic seam) every cycle is contractible, so the union-find
// words carry parents only and each open cluster's root is its smallest site.
//
// A lattice context here is a Lat<Word16> whose Geom covers the sites held by
// the CTA; sites whose x-bond leaves that range (the last L sites) are left to
// the caller's seam or boundary stage.
#pragma once

#include "rbim_phases.cuh"

#ifndef RBIM_COUNT
#ifdef RBIM_PROFILE_PHASES
#define RBIM_COUNT(k, v) ((void)(v))
#define RBIM_PROF_ONLY(...) __VA_ARGS__
#else
#define RBIM_COUNT(k, v) ((void)0)
#define RBIM_PROF_ONLY(...)
#endif
#endif

namespace rbim {

// Open-lattice union-find word: the parent site only.
struct Word16 {
    using T = unsigned short;
    __device__ __forceinline__ static uint32_t parent(T w) { return w; }
    __device__ __forceinline__ static int ox(T) { return 0; }
    __device__ __forceinline__ static int oy(T) { return 0; }
    __device__ __forceinline__ static T make(uint32_t p, int, int) { return (T)p; }
    __device__ __forceinline__ static T count_inc(uint32_t c) { return (T)c; }
};

// The open union-find lives in shared memory: access it through 32-bit
// shared-window addresses with explicit ld/st/atom.shared instructions.
template <>
struct UF<Word16> {
    using T = unsigned short;
    T *w;          // generic pointer (for code that indexes the array directly)
    uint32_t sa;   // shared-window address of w
    __device__ __forceinline__ T ld(uint32_t i) const
    {
        T v;
        asm volatile("ld.volatile.shared.u16 %0, [%1];" : "=h"(v) : "r"(sa + 2u * i) : "memory");
        return v;
    }
    // Shared memory is coherent within the CTA: the same load as ld.
    __device__ __forceinline__ T ldc(uint32_t i) const { return ld(i); }
    __device__ __forceinline__ void st(uint32_t i, T v) const
    {
        asm volatile("st.volatile.shared.u16 [%0], %1;" ::"r"(sa + 2u * i), "h"(v) : "memory");
    }
    // The parents of sites i and i + 1 (i even) in one 32-bit store: v holds
    // site i's in its low half.
    __device__ __forceinline__ void st2(uint32_t i, uint32_t v) const
    {
        asm volatile("st.volatile.shared.u32 [%0], %1;" ::"r"(sa + 2u * i), "r"(v) : "memory");
    }
    __device__ __forceinline__ T cas(uint32_t i, T expect, T v) const
    {
        T old;
        asm volatile("atom.shared.cas.b16 %0, [%1], %2, %3;"
                     : "=h"(old)
                     : "r"(sa + 2u * i), "h"(expect), "h"(v)
                     : "memory");
        return old;
    }
    __device__ __forceinline__ void add(uint32_t i, T v) const { uf_atomic_add(w + i, v); }
};

// Mask of the bits of word w whose site lies in the last row (x = L-1): the
// horizontal bonds there close the x boundary.
__device__ __forceinline__ uint32_t last_row_mask(const Geom &g, uint32_t w)
{
    const uint32_t n0 = w << 5, first = g.N - g.L;
    if (n0 + 32u <= first) return 0u;
    const uint32_t v = g.valid(w);
    if (n0 >= first) return v;
    return ~((1u << (first - n0)) - 1u) & v;
}

// Occupied x-bonds of word w that need a union: off the x seam, and not
// already connected through an elementary plaquette with the bond before.
__device__ __forceinline__ uint32_t union_need(const Lat<Word16> &t, uint32_t w)
{
    const Geom &g = t.g;
    const uint32_t oh = t.OH[w] & ~last_row_mask(g, w);
    if (!oh) return 0u;
    Plane OVp{t.OV};
    const uint32_t ohp = w ? t.OH[w - 1u] : 0u;
    const uint32_t ov = OVp(w), ovp = w ? OVp(w - 1u) : 0u;
    const uint32_t prev_oh = (oh << 1) | (ohp >> 31);
    const uint32_t prev_ov = (ov << 1) | (ovp >> 31);
    uint32_t s = (w << 5) + g.L - 1u;
    if (s >= g.N) s -= g.N;
    return oh & ~(prev_oh & prev_ov & extract32(OVp, s, g));
}

// One path-halving step of a walk at x, without branches: returns the next
// position and sets `done` when x's parent or grandparent is the root (the
// returned position is then the root).
__device__ __forceinline__ uint32_t halving_step(const UF<Word16> &uf, uint32_t x, bool &done)
{
    const uint32_t p = uf.ld(x);
    const uint32_t gp = uf.ld(p);
    const bool x_root = p == x, p_root = gp == p;
    if (!x_root && !p_root) uf.st(x, (unsigned short)gp);
    done = x_root || p_root;
    return x_root ? x : (p_root ? p : gp);
}

// (b) Open-lattice unions across occupied x-bonds that do not cross the x
// seam: the larger root is hooked under the smaller with a 16-bit CAS, finds
// use path halving, and a union whose CAS loses a race restarts from the two
// roots it found.  Both endpoint walks advance in the same loop iteration.
__device__ __forceinline__ void phase_union_open(const Lat<Word16> &t, uint32_t tid, uint32_t nthreads)
{
    const Geom &g = t.g;
    const UF<Word16> &uf = t.uf;
    const Slices sl = make_slices(g.NW, nthreads);
    uint32_t item = tid, pending = 0, base = 0;
    uint32_t xa = 0, xb = 0;
    bool fetch = true;
    const uint32_t cap = 64u * t.cap;  // 64 walks of t.cap steps (64 N + 4096 by default)
    uint32_t it = 0;
    RBIM_PROF_ONLY(uint32_t n_bonds = 0; uint32_t n_fails = 0);
    for (;; ++it) {
        if (it >= cap) {
            atomicOr(t.err, kErrUnionCap);
            break;
        }
        if (fetch) {
            while (!pending && item < sl.items) {
                const uint32_t w = sl.word(item);
                pending = union_need(t, w) & sl.mask(item);
                base = w << 5;
                item += nthreads;
            }
            if (!pending) break;
            xa = base + (uint32_t)(__ffs(pending) - 1);
            pending &= pending - 1u;
            xb = xa + g.L;
            fetch = false;
            RBIM_PROF_ONLY(++n_bonds);
        }
        bool da, db;
        xa = halving_step(uf, xa, da);
        xb = halving_step(uf, xb, db);
        if (da && db) {
            // Both walks are at roots.
            if (xa == xb) {
                fetch = true;
            } else {
                const uint32_t lo = min(xa, xb), hi = max(xa, xb);
                fetch = uf.cas(hi, (unsigned short)hi, (unsigned short)lo) == (unsigned short)hi;
                // A lost race leaves both walks at their old roots, to resume from.
                RBIM_PROF_ONLY(n_fails += fetch ? 0u : 1u);
            }
        }
    }
#ifdef RBIM_PROFILE_PHASES
    {
        uint32_t mx = it, sm = it;
        for (int o = 16; o > 0; o >>= 1) {
            mx = max(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
            sm += __shfl_xor_sync(0xFFFFFFFFu, sm, o);
        }
        uint32_t nb = n_bonds, nf = n_fails;
        for (int o = 16; o > 0; o >>= 1) {
            nb += __shfl_xor_sync(0xFFFFFFFFu, nb, o);
            nf += __shfl_xor_sync(0xFFFFFFFFu, nf, o);
        }
        if ((threadIdx.x & 31u) == 0) {
            RBIM_COUNT(3, mx);
            RBIM_COUNT(4, sm);
            RBIM_COUNT(0, nb);
            RBIM_COUNT(2, nf);
        }
    }
#endif
}

// (c) Roots of the run heads (see phase_roots), as a flat per-thread loop
// over the heads of the thread's slices: read-only walks, each head's final
// root written by the head's own thread.  ROOT must be zero on entry.
// Returns the number of roots this thread found.
// Next head of the thread's slices into (h, x), or false when there is none.
__device__ __forceinline__ bool next_head(const Lat<Word16> &t, const Slices &sl, uint32_t nthreads, uint32_t &item,
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

__device__ __forceinline__ uint32_t phase_roots_flat(const Lat<Word16> &t, uint32_t tid, uint32_t nthreads)
{
    const Geom &g = t.g;
    const Slices sl = make_slices(g.NW, nthreads);
    uint32_t item = tid, pending = 0, base = 0, nroots = 0;
    // Two walks in flight per thread: heads h0, h1 at positions x0, x1.
    uint32_t h0 = 0, h1 = 0, x0 = 0, x1 = 0;
    bool a0 = next_head(t, sl, nthreads, item, pending, base, h0);
    bool a1 = a0 && next_head(t, sl, nthreads, item, pending, base, h1);
    x0 = h0;
    x1 = h1;
    const uint32_t cap = 64u * t.cap;  // 64 walks of t.cap steps (64 N + 4096 by default)
    for (uint32_t it = 0; a0 || a1; ++it) {
        if (it >= cap) {
            atomicOr(t.err, kErrFindCap);
            break;
        }
        const uint32_t p0 = t.uf.ld(x0), p1 = t.uf.ld(x1);
        const bool r0 = a0 && p0 == x0, r1 = a1 && p1 == x1;
        x0 = p0;
        x1 = p1;
        if (r0) {
            if (x0 != h0) {
                t.uf.st(h0, (unsigned short)x0);
            } else {
                atomicOr(t.ROOT + (h0 >> 5), 1u << (h0 & 31u));
                ++nroots;
            }
            a0 = next_head(t, sl, nthreads, item, pending, base, h0);
            x0 = h0;
        }
        if (r1) {
            if (x1 != h1) {
                t.uf.st(h1, (unsigned short)x1);
            } else {
                atomicOr(t.ROOT + (h1 >> 5), 1u << (h1 & 31u));
                ++nroots;
            }
            a1 = next_head(t, sl, nthreads, item, pending, base, h1);
            x1 = h1;
        }
    }
    return nroots;
}

__device__ __forceinline__ uint32_t warp_sum(uint32_t v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    return v;
}

// Run pieces: the sites of a word split into maximal runs of occupied
// y-bonds; every piece starts at a run head or at bit 0 of the word and all
// its sites share one root.  Bits of the pieces' first sites.
__device__ __forceinline__ uint32_t piece_leaders(const Lat<Word16> &t, uint32_t w, uint32_t valid)
{
    return (head_mask(t.OV, w, valid) | 1u) & valid;
}

// Add v to the 16-bit word i through its 32-bit container (no carry can
// leave the half: cluster sizes stay below 65536 whenever counts are taken).
__device__ __forceinline__ void add16(unsigned short *base, uint32_t i, uint32_t v)
{
    atomicAdd((unsigned int *)(base + (i & ~1u)), v << (16u * (i & 1u)));
}

// Cluster sizes into the root words (after the sites pass, every non-root
// site's word holds its root): one add per run piece, the sites of a word
// split into maximal runs sharing a root.  With at least 32 words per warp,
// each lane takes a word of its warp's block of 32 and walks the word's
// pieces, summing consecutive pieces of one root in a register; at the end
// of the block the lanes holding the same root add their sums in one atomic,
// so a giant cluster sees one add per block instead of one per piece.
// kMinusOne: the piece that starts at the root adds one less, so that a root
// word holds size - 1 (a tile of 65536 sites then still fits 16 bits).
// Each root word must hold zero or the root's own index on entry (a root
// points at itself, so counting onto it needs no zeroing pass; the caller
// then subtracts the index).
template <bool kMinusOne>
__device__ __forceinline__ void count_pieces(const Lat<Word16> &t, unsigned short *u16, uint32_t warp,
                                             uint32_t nwarps)
{
    const Geom &g = t.g;
    const uint32_t lane = threadIdx.x & 31u;
    if (g.NW >= 32u * nwarps) {
        for (uint32_t w0 = warp << 5; w0 < g.NW; w0 += nwarps << 5) {
            const uint32_t w = w0 + lane;
            uint32_t acc_r = 0xFFFFFFFFu, acc = 0;
            if (w < g.NW) {
                const uint32_t valid = g.valid(w);
                uint32_t lead = piece_leaders(t, w, valid);
                const uint32_t roots = t.ROOT[w];
                const uint32_t nv = (uint32_t)__popc(valid);
                while (lead) {
                    const uint32_t b = __ffs(lead) - 1u;
                    lead &= lead - 1u;
                    const uint32_t end = lead ? (uint32_t)(__ffs(lead) - 1) : nv;
                    const uint32_t n = (w << 5) + b;
                    const bool is_root = (roots >> b) & 1u;
                    const uint32_t r = is_root ? n : (uint32_t)u16[n];
                    if (r != acc_r) {
                        if (acc) add16(u16, acc_r, acc);
                        acc_r = r;
                        acc = 0;
                    }
                    acc += end - b - ((kMinusOne && is_root) ? 1u : 0u);
                }
            }
            const uint32_t grp = __match_any_sync(0xFFFFFFFFu, acc_r);
            const uint32_t sum = __reduce_add_sync(grp, acc);
            if (acc_r != 0xFFFFFFFFu && lane == (uint32_t)(__ffs(grp) - 1) && sum) add16(u16, acc_r, sum);
        }
    } else {
        for (uint32_t w = warp; w < g.NW; w += nwarps) {
            const uint32_t valid = g.valid(w);
            const uint32_t lead = piece_leaders(t, w, valid);
            if ((lead >> lane) & 1u) {
                const uint32_t n = (w << 5) + lane;
                const uint32_t next = lead & ~mask_le(lane);
                const uint32_t end = next ? (uint32_t)(__ffs(next) - 1) : (uint32_t)__popc(valid);
                const bool is_root = (t.ROOT[w] >> lane) & 1u;
                const uint32_t r = is_root ? n : (uint32_t)u16[n];
                add16(u16, r, end - lane - ((kMinusOne && is_root) ? 1u : 0u));
            }
        }
    }
}

// Root of any site n once the roots pass is done: every parent is a run head
// (heads are the initial parents, roots are heads, and hooks, path halving
// and the seam merge only ever point at roots or grandparents) and every head
// then points at its root (a root at itself), so two loads reach it.
__device__ __forceinline__ uint32_t piece_root(const unsigned short *u16, uint32_t n) { return u16[u16[n]]; }

// The cluster flip of a sweep, one lane per word and one root lookup per run
// piece instead of per site: the sites of a word split into pieces (maximal
// runs of occupied y-bonds cut at the word boundary) that share a root, and a
// piece flips as a whole when its root's FLIP bit is set.  With
// `leader_roots` the leader of every piece that does not head its run (bit 0
// of a word inside a run) also gets its root written, so that afterwards the
// word of every piece leader holds its root, which the cluster-size count and
// the |M_C| pass read.  Non-head words are nobody's parent, so the writes do
// not disturb the lookups of other lanes.
__device__ __forceinline__ void flip_pieces(const Lat<Word16> &t, uint32_t tid, uint32_t nthreads,
                                                     bool leader_roots)
{
    const Geom &g = t.g;
    unsigned short *u16 = t.uf.w;
    for (uint32_t w = tid; w < g.NW; w += nthreads) {
        const uint32_t valid = g.valid(w);
        const uint32_t heads = head_mask(t.OV, w, valid);
        uint32_t lead = (heads | 1u) & valid;
        const uint32_t nv = (uint32_t)__popc(valid);
        uint32_t fl = 0;
        while (lead) {
            const uint32_t b = __ffs(lead) - 1u;
            lead &= lead - 1u;
            const uint32_t end = lead ? (uint32_t)(__ffs(lead) - 1) : nv;
            const uint32_t n = (w << 5) + b;
            const uint32_t r = piece_root(u16, n);
            if ((t.FLIP[r >> 5] >> (r & 31u)) & 1u) fl |= (end - b == 32u) ? 0xFFFFFFFFu : (((1u << (end - b)) - 1u) << b);
            if (leader_roots && !((heads >> b) & 1u)) u16[n] = (unsigned short)r;
        }
        if (fl) t.S[w] ^= fl;
    }
}

// Roots and cluster flip of a sweep in one pass, one lane per word and one
// walk per run piece (the sites of a word split into pieces -- maximal runs
// of occupied y-bonds cut at the word boundary -- that share a root).  A
// piece's leader walks read-only up to its root; the root is then written
// into the leader's word (for a run head this is the final compression the
// separate roots pass would make, and the count and |M_C| passes read it
// for every leader), the piece flips as a whole with its root's FLIP bit,
// and a leader that is its own root sets its ROOT bit.  Walks of other lanes
// running at the same time may read a head's old parent or its final root;
// both are ancestors, so every walk ends at the right root.  Roots' words are
// never written.  Returns the number of roots this thread found.
__device__ __forceinline__ uint32_t roots_flip_pieces(const Lat<Word16> &t, uint32_t tid, uint32_t nthreads)
{
    const Geom &g = t.g;
    const UF<Word16> &uf = t.uf;
    uint32_t nroots = 0;
    for (uint32_t w = tid; w < g.NW; w += nthreads) {
        const uint32_t valid = g.valid(w);
        uint32_t lead = (head_mask(t.OV, w, valid) | 1u) & valid;
        const uint32_t nv = (uint32_t)__popc(valid);
        uint32_t fl = 0, rootbits = 0;
        while (lead) {
            const uint32_t b = __ffs(lead) - 1u;
            lead &= lead - 1u;
            const uint32_t end = lead ? (uint32_t)(__ffs(lead) - 1) : nv;
            const uint32_t n = (w << 5) + b;
            uint32_t x = uf.ld(n);
            for (uint32_t it = 0;; ++it) {
                const uint32_t p = uf.ld(x);
                if (p == x) break;
                if (it >= t.cap) {
                    atomicOr(t.err, kErrFindCap);
                    break;
                }
                x = p;
            }
            if (x == n) {
                rootbits |= 1u << b;
                ++nroots;
            } else {
                uf.st(n, (unsigned short)x);
            }
            if ((t.FLIP[x >> 5] >> (x & 31u)) & 1u) fl |= (end - b == 32u) ? 0xFFFFFFFFu : (((1u << (end - b)) - 1u) << b);
        }
        t.ROOT[w] = rootbits;
        if (fl) t.S[w] ^= fl;
    }
    return nroots;
}

}  // namespace rbim

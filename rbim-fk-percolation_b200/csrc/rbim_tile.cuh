// Tiles of one lattice: consecutive-site slices of an L x L lattice, each
// held in one CTA's shared memory.  Shared by the cluster engine (tiles of a
// thread-block cluster, merged through distributed shared memory) and the
// grid engine (tiles of a cooperative grid, merged through global memory).
// Tile c holds global sites [c*T, c*T + Tc), T a multiple of 128; its spin
// plane holds the tile, then a halo of the next tile's first L spins.
#pragma once

#include "rbim_phases.cuh"

namespace rbim {

// Geometry of this CTA's tile of the current chain.
struct Tile {
    uint32_t L, N, C, c, T, b, Tc, tw, x0, f, nwp;
};

// Row-end bit of tile word w (at most one: L > 32).
__device__ __forceinline__ uint32_t tile_row_end(const Tile &tl, uint32_t w, uint32_t valid)
{
    const uint32_t n0 = tl.b + (w << 5);
    const uint32_t p = (tl.L - 1u) - (n0 % tl.L);
    return p < 32u ? (1u << p) & valid : 0u;
}

// 32 bits of the tile's spin plane from local bit `start` (no wrap: the
// plane holds the tile, then the halo, then zero words).
__device__ __forceinline__ uint32_t extract_nowrap(const uint32_t *P, uint32_t start)
{
    const uint32_t wi = start >> 5, sh = start & 31u;
    const uint32_t lo = P[wi];
    return sh ? __funnelshift_r(lo, P[wi + 1u], sh) : lo;
}

// +y neighbours of tile word w: site m+1, or the row start m+1-L at a row
// end; the row start of the tile's first (partial) row lies in the previous
// tile and is the front spin.
__device__ __forceinline__ uint32_t tile_ynext(const uint32_t *S, uint32_t w, uint32_t re, uint32_t L, uint32_t front)
{
    uint32_t r = extract_nowrap(S, (w << 5) + 1u) & ~re;
    if (re) {
        const uint32_t bit = __ffs(re) - 1u;
        const int q = (int)((w << 5) + bit) + 1 - (int)L;
        const uint32_t v = q >= 0 ? (S[(uint32_t)q >> 5] >> ((uint32_t)q & 31u)) & 1u : front;
        r |= v << bit;
    }
    return r;
}

// (a) Bond activation of the tile: the resident engine's chunk scheme with
// the chunk index offset by the tile's first chunk, so that every bond draws
// the same Philox word as in the whole-lattice engines.  OV keeps the y-bonds
// inside the tile; y-seam bonds go to YS (bit = row - x0), the y-bond from
// the tile's last site into the next tile to tile_end (shared memory).
template <int NT>
__device__ __forceinline__ void tile_activate(const Lat<Word16> &t, uint32_t *YS, const Tile &tl, const SweepRng &rng,
                                              const uint32_t *gJH, const uint32_t *gJV, uint32_t front,
                                              uint32_t &tile_end, uint32_t warp, uint32_t nwarps, uint32_t tid)
{
    const Geom &g = t.g;
    const uint32_t lane = tid & 31u;
    const uint32_t nchunks = (g.N + 127u) >> 7;
    const uint32_t chunk0 = tl.b >> 7;
    const uint32_t last = tl.Tc - 1u;
    const bool end_is_row_end = ((tl.b + tl.Tc) % tl.L) == 0u;
    // Groups of G consecutive words, as in phase_activate_bonds: lane j forms
    // the satisfied masks of word j, then the warp draws the group's chunks
    // two at a time and lane j keeps the ballots of its own word.
    uint32_t G = 32u;
    while (G > 4u && G * nwarps > g.NW) G >>= 1;
    const uint32_t ngroups = (g.NW + G - 1u) / G;
    const uint32_t my_chunk = lane >> 2, my_s = lane & 3u;
    for (uint32_t grp = warp; grp < ngroups; grp += nwarps) {
        const uint32_t w = grp * G + lane;
        const bool mine = lane < G && w < g.NW;
        uint32_t sh = 0, sv = 0, re = 0;
        if (mine) {
            const uint32_t v = g.valid(w);
            re = tile_row_end(tl, w, v);
            const uint32_t s = t.S[w];
            sh = ~(s ^ extract_nowrap(t.S, (w << 5) + tl.L) ^ gJH[w]) & v;
            sv = ~(s ^ tile_ynext(t.S, w, re, tl.L, front) ^ gJV[w]) & v;
        }
        const uint32_t c0 = grp * (G >> 2);
        const uint32_t nch = min(G >> 2, nchunks - c0);
        uint32_t oh = 0, ov = 0;
        for (uint32_t k = 0; k < nch; k += 2u) {
            const bool two = k + 1u < nch;
            const uint32_t b0 = 32u * (chunk0 + c0 + k) + lane, b1 = b0 + 32u;
            const U4 r0 = philox_block(rng.key, b0, rng.sweep, kStreamBond);
            U4 r1{};
            if (two) r1 = philox_block(rng.key, b1, rng.sweep, kStreamBond);
            const uint32_t a0 = accept_block(rng, r0, b0);
            const uint32_t a1 = two ? accept_block(rng, r1, b1) : 0u;
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
            uint32_t keep = ov & ~re;
            if (w == (last >> 5) && !end_is_row_end) {
                const uint32_t eb = 1u << (last & 31u);
                tile_end = (keep & eb) ? 1u : 0u;
                keep &= ~eb;
            }
            t.OH[w] = oh;
            t.OV[w] = keep;
            if (ov & re) {
                const uint32_t bit = __ffs(re) - 1u;
                const uint32_t row = (tl.b + (w << 5) + bit + 1u) / tl.L - 1u - tl.x0;
                atomicOr(YS + (row >> 5), 1u << (row & 31u));
            }
        }
    }
    // Flip bits: Philox block q of stream 1 covers global words 4q .. 4q+3.
    const uint32_t nblk = (g.NW + 3u) >> 2;
    for (uint32_t q = tid; q < nblk; q += NT) {
        const U4 rr = philox_block(rng.key, chunk0 + q, rng.sweep, kStreamFlip);
        const uint32_t w = 4u * q;
        t.FLIP[w] = rr.x;
        if (w + 1u < g.NW) t.FLIP[w + 1u] = rr.y;
        if (w + 2u < g.NW) t.FLIP[w + 2u] = rr.z;
        if (w + 3u < g.NW) t.FLIP[w + 3u] = rr.w;
    }
}

// Root of tile site x after the open labelling's roots pass: every parent is
// a run head and every head points at its root.
__device__ __forceinline__ uint32_t tile_root(const unsigned short *uf, uint32_t x)
{
    const uint32_t p = uf[x];
    const uint32_t q = uf[p];
    return q == p ? p : q;
}

template <int NT>
__device__ __forceinline__ void tile_energy(const Lat<Word16> &t, const Tile &tl, const uint32_t *gJH,
                                            const uint32_t *gJV, uint32_t front, uint32_t tid, uint32_t &unsat,
                                            uint32_t &downs)
{
    for (uint32_t w = tid; w < t.g.NW; w += NT) {
        const uint32_t v = t.g.valid(w);
        const uint32_t s = t.S[w];
        const uint32_t re = tile_row_end(tl, w, v);
        unsat += __popc((s ^ extract_nowrap(t.S, (w << 5) + tl.L) ^ gJH[w]) & v);
        unsat += __popc((s ^ tile_ynext(t.S, w, re, tl.L, front) ^ gJV[w]) & v);
        downs += __popc(s & v);
    }
}

__device__ __forceinline__ unsigned long long size_key(uint32_t size, uint32_t g)
{
    return ((unsigned long long)size << 32) | (unsigned long long)(0xFFFFFFFFu - g);
}

// Root of tile site x by a read-only walk, for use before the heads point at
// their roots (nothing writes the parents meanwhile); at most `cap` steps,
// after which the error bit is set and the walk's position returned.
__device__ __forceinline__ uint32_t tile_root_walk(const unsigned short *uf, uint32_t x, uint32_t cap, int *err)
{
    for (uint32_t it = 0;; ++it) {
        const uint32_t p = uf[x];
        if (p == x) return x;
        if (it >= cap) {
            atomicOr(err, kErrFindCap);
            return x;
        }
        x = p;
    }
}

// Size of the tile cluster of tile root m once the sizes minus one have been
// added onto the roots' own indices (count_pieces<true> without zeroing).
__device__ __forceinline__ uint32_t tile_size(const unsigned short *u16, uint32_t m)
{
    return (((uint32_t)u16[m] - m) & 0xFFFFu) + 1u;
}

}  // namespace rbim

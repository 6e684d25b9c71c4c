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
    int *wrap;             // bit 0 wrap_x, bit 1 wrap_y
    int *err;
    uint32_t cap;
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

// Spread the low 8 bits of v to bit positions 0, 4, 8, ..., 28.
__device__ __forceinline__ uint32_t spread8x4(uint32_t v)
{
    v &= 0xFFu;
    v = (v | (v << 12)) & 0x000F000Fu;
    v = (v | (v << 6)) & 0x03030303u;
    v = (v | (v << 3)) & 0x11111111u;
    return v;
}

// Occupation decision of one bond from its 16-bit draw u: u < thr_hi
// accepts, u > thr_hi rejects, u == thr_hi (probability 2^-16) defers to the
// low half v, drawn separately.  Returns 0 reject, 1 accept, 2 undecided.
__device__ __forceinline__ uint32_t bond_decide(const SweepRng &rng, uint32_t u)
{
    if (rng.thr_all || u < rng.thr_hi) return 1u;
    return u == rng.thr_hi ? 2u : 0u;
}

// (a) Bond activation.  Items are 128-site chunks (four plane words); lane i
// of the warp owning chunk c draws Philox block 32c + i, whose word s holds
// the 16-bit draws of the horizontal (low half) and vertical (high half) bond
// of site 128c + 4i + s.  SEAMV must be zero on entry.
template <class WT>
__device__ __forceinline__ void phase_activate_bonds(const Lat<WT> &t, const SweepRng &rng, uint32_t warp,
                                                     uint32_t nwarps)
{
    const uint32_t lane = threadIdx.x & 31u;
    const Geom &g = t.g;
    const uint32_t nchunks = (g.N + 127u) >> 7;
    Plane S{t.S};
    for (uint32_t c = warp; c < nchunks; c += nwarps) {
        const uint32_t wl = 4u * c + (lane >> 3);
        uint32_t sh = 0, sv = 0;
        if (wl < g.NW) {
            const uint32_t v = g.valid(wl);
            const uint32_t s = S(wl);
            sh = ~(s ^ xnext_word(S, wl, g) ^ t.JH[wl]) & v;
            sv = ~(s ^ ynext_word(S, wl, g) ^ t.JV[wl]) & v;
        }
        const uint32_t sb = 4u * (lane & 7u);
        sh = (sh >> sb) & 0xFu;  // satisfied bits of this lane's four sites
        sv = (sv >> sb) & 0xFu;
        const U4 r = philox_block(rng.key, 32u * c + lane, rng.sweep, kStreamBond);
        uint32_t dh[4], dv[4];
        bool refine = false;
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const uint32_t w = u4_word(r, s);
            dh[s] = ((sh >> s) & 1u) ? bond_decide(rng, w & 0xFFFFu) : 0u;
            dv[s] = ((sv >> s) & 1u) ? bond_decide(rng, w >> 16) : 0u;
            refine |= (dh[s] == 2u) | (dv[s] == 2u);
        }
        if (refine) {
            const U4 q = philox_block(rng.key, 32u * c + lane, rng.sweep, kStreamBondLow);
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                const uint32_t w = u4_word(q, s);
                if (dh[s] == 2u) dh[s] = (w & 0xFFFFu) < rng.thr_lo ? 1u : 0u;
                if (dv[s] == 2u) dv[s] = (w >> 16) < rng.thr_lo ? 1u : 0u;
            }
        }
        uint32_t oh = 0, ov = 0;
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const uint32_t bh = __ballot_sync(0xFFFFFFFFu, dh[s] != 0u);
            const uint32_t bv = __ballot_sync(0xFFFFFFFFu, dv[s] != 0u);
            // Word j of the chunk collects lanes 8j .. 8j+7.
            const uint32_t j = lane & 3u;
            oh |= spread8x4(bh >> (8u * j)) << s;
            ov |= spread8x4(bv >> (8u * j)) << s;
        }
        if (lane < 8u) {
            const uint32_t w = 4u * c + (lane & 3u);
            if (w < g.NW) {
                if (lane < 4u) {
                    t.OH[w] = oh;
                } else {
                    const uint32_t re = g.row_end(w);
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
    const uint32_t ov = *((volatile const uint32_t *)(OV + w));
    const uint32_t prev = w ? (*((volatile const uint32_t *)(OV + w - 1u)) >> 31) : 0u;
    return ~((ov << 1) | prev) & valid;
}

// (b) Union-find initialisation: every site points at the head of its run of
// occupied y-bonds with zero image offset (runs never cross a seam).
template <class WT>
__device__ __forceinline__ void phase_heads(const Lat<WT> &t, uint32_t warp, uint32_t nwarps)
{
    const uint32_t lane = threadIdx.x & 31u;
    const Geom &g = t.g;
    for (uint32_t w = warp; w < g.NW; w += nwarps) {
        const uint32_t h = head_mask(t.OV, w, g.valid(w));
        uint32_t carry = 0;
        if (!(h & 1u)) {
            // Last head in an earlier word (site 0 is always a head).
            for (uint32_t ww = w; ww-- > 0;) {
                const uint32_t hh = head_mask(t.OV, ww, 0xFFFFFFFFu);
                if (hh) {
                    carry = (ww << 5) + 31u - __clz(hh);
                    break;
                }
            }
        }
        const uint32_t n = (w << 5) + lane;
        if (n < g.N) {
            const uint32_t m = h & mask_le(lane);
            const uint32_t head = m ? (w << 5) + 31u - __clz(m) : carry;
            t.uf.st(n, WT::make(head, 0, 0));
        }
    }
}

// (b) Unions across occupied x-bonds (including the x seam, image offset
// (1,0)).  A bond is skipped when the bond one step lower in y is occupied and
// both y-bonds joining them are occupied: it then closes an elementary
// plaquette, which is contractible and already connected.
template <class WT>
__device__ __forceinline__ void phase_union(const Lat<WT> &t, uint32_t warp, uint32_t nwarps, uint32_t tid,
                                            uint32_t nthreads)
{
    const uint32_t lane = threadIdx.x & 31u;
    const Geom &g = t.g;
    Plane OVp{t.OV};
    for (uint32_t w = warp; w < g.NW; w += nwarps) {
        const uint32_t oh = t.OH[w];
        if (!oh) continue;
        const uint32_t ohp = w ? t.OH[w - 1u] : 0u;
        const uint32_t ov = OVp(w), ovp = w ? OVp(w - 1u) : 0u;
        const uint32_t prev_oh = (oh << 1) | (ohp >> 31);
        const uint32_t prev_ov = (ov << 1) | (ovp >> 31);
        uint32_t s = (w << 5) + g.N + g.L - 1u;
        s %= g.N;
        const uint32_t prev_ovx = extract32(OVp, s, g);
        const uint32_t need = oh & ~(prev_oh & prev_ov & prev_ovx);
        if ((need >> lane) & 1u) {
            const uint32_t n = (w << 5) + lane;
            uint32_t b = n + g.L;
            int ex = 0;
            if (b >= g.N) {
                b -= g.N;
                ex = 1;
            }
            uf_union<WT>(t.uf, n, b, ex, 0, t.wrap, t.cap, t.err);
        }
    }
    // y seam: (x, L-1) -> (x, 0) with image offset (0, 1).
    for (uint32_t x = tid; x < g.L; x += nthreads) {
        if ((t.SEAMV[x >> 5] >> (x & 31u)) & 1u) {
            const uint32_t a = x * g.L + g.L - 1u;
            uf_union<WT>(t.uf, a, x * g.L, 0, 1, t.wrap, t.cap, t.err);
        }
    }
}

// (c) Roots, flip and (optionally) cluster sizes.  Every site is pointed
// straight at its root (only the site's own thread writes its word here, so
// after the phase every non-root word holds its root); roots are recorded in
// ROOT; each site's spin is
// flipped with its cluster's flip bit; with `count` the root words accumulate
// the cluster size in their offset field (warp-aggregated with match_any).
// Returns this warp's number of roots (valid in every lane).
template <class WT>
__device__ __forceinline__ uint32_t phase_finalize(const Lat<WT> &t, uint32_t warp, uint32_t nwarps, bool flip,
                                                   bool count)
{
    const uint32_t lane = threadIdx.x & 31u;
    const Geom &g = t.g;
    uint32_t nroots = 0;
    for (uint32_t w = warp; w < g.NW; w += nwarps) {
        const uint32_t n = (w << 5) + lane;
        const bool ok = n < g.N;
        uint32_t r = 0;
        if (ok) {
            r = uf_root_ro<WT>(t.uf, n, t.cap, t.err);
            if (r != n) t.uf.st(n, WT::make(r, 0, 0));
        }
        const uint32_t roots = __ballot_sync(0xFFFFFFFFu, ok && r == n);
        if (flip) {
            const uint32_t fl = ok ? (t.FLIP[r >> 5] >> (r & 31u)) & 1u : 0u;
            const uint32_t s = t.S[w];
            const uint32_t ns = __ballot_sync(0xFFFFFFFFu, ok && (((s >> lane) & 1u) ^ fl)) & g.valid(w);
            if (lane == 0) t.S[w] = ns;
        }
        if (lane == 0) t.ROOT[w] = roots;
        nroots += __popc(roots);
        if (count) {
            const uint32_t live = __ballot_sync(0xFFFFFFFFu, ok);
            if (ok) {
                const uint32_t grp = __match_any_sync(live, r);
                if (lane == (uint32_t)(__ffs(grp) - 1)) t.uf.add(r, WT::count_inc(__popc(grp)));
            }
        }
    }
    return nroots;
}

// (d) Unsatisfied bonds and down spins over words first, first+stride, ...
__device__ __forceinline__ void measure_energy(const Geom &g, const uint32_t *S, const uint32_t *JH,
                                               const uint32_t *JV, uint32_t first, uint32_t stride,
                                               uint32_t &unsat, uint32_t &downs)
{
    Plane Sp{const_cast<uint32_t *>(S)};
    for (uint32_t w = first; w < g.NW; w += stride) {
        const uint32_t v = g.valid(w);
        const uint32_t s = Sp(w);
        unsat += __popc((s ^ xnext_word(Sp, w, g) ^ JH[w]) & v);
        unsat += __popc((s ^ ynext_word(Sp, w, g) ^ JV[w]) & v);
        downs += __popc(s & v);
    }
}

}  // namespace rbim

// Cluster engine: one lattice per thread-block cluster, for lattices too large
// for one CTA (L > 256, up to 1024).  The C CTAs of a cluster split the
// lattice into C tiles of consecutive sites (tile c holds global sites
// [c*T, c*T + Tc), T a multiple of 128 and at most 65536), each held in its
// CTA's shared memory for every sweep of a call, exactly like the resident
// engine holds a whole lattice:
//
//  1. activation of the bonds owned by the tile's sites (the x-bond of the
//     last L sites and the y-bond of the tile's last site reach the next
//     tile; the spins they need are a halo copied from the neighbour CTA's
//     shared memory through distributed shared memory);
//  2. the open-tile labelling of the resident engine (16-bit parents, run
//     heads, flat union and root walks): inside a tile every cycle is
//     contractible;
//  3. the boundary bonds -- x-bonds from the last L sites of a tile (into the
//     next tile, or across the x seam from the last tile to the first), the
//     y-bond between two tiles, and the y-seam bonds -- are unioned in a
//     cluster-wide union-find over the tile roots they touch.  Its nodes live
//     in hash tables in the CTAs' shared memory; words carry image offsets
//     (Word64: parent node | wx | wy), and a boundary bond that closes a
//     loop with nonzero summed offset winds around the torus (the exact test
//     of src/rbim/_unionfind.py:104-124).  The larger key (global site of a
//     node's tile root) is hooked under the smaller, so a merged cluster's
//     root node is its smallest site, the canonical label that keys its flip;
//  4. flip, halo refresh and the measurement reductions across the cluster.
//
// Node ids are (tile << 16) | slot; every access to another CTA's shared
// memory goes through cluster.map_shared_rank, and every phase that reads or
// writes another CTA's memory is fenced by cluster barriers.
//
// This replaces, per chain, the loop of run_single_realization
// (src/rbim/simulation.py:196-242) around sw_sweep
// (src/rbim/swendsen_wang.py:103-172), with the same Philox stream and
// bit-identical results to the oracle's sweep.
#include <algorithm>
#include <cooperative_groups.h>

#include "rbim_internal.h"
#include "rbim_open.cuh"
#include "rbim_tile.cuh"

namespace cg = cooperative_groups;

namespace rbim {

namespace {

constexpr uint32_t kTileMax = 65536;    // 16-bit tile parents
constexpr uint32_t kTileHalf = 32768;   // tiles of the 512-thread mode
constexpr uint32_t kClusterMax = 16;    // non-portable cluster size limit
constexpr uint32_t kHashMax = 4096;     // node slots per tile (12 bits of a node id)
constexpr uint32_t kHalfTilesMax = 5;   // most tiles per lattice in the 512-thread mode
constexpr uint32_t kEmptyKey = 0xFFFFFFFFu;
constexpr size_t kSmemBudget = 227 * 1024 - 4 * 1024;  // one CTA per SM
constexpr size_t kSmemPerSm = 228 * 1024;
constexpr size_t kStaticSmem = 2 * 1024;

__host__ __device__ constexpr size_t a16(size_t v) { return (v + 15) & ~size_t(15); }

}  // namespace


namespace {

__host__ __device__ constexpr uint32_t cluster_hash_size(uint32_t l_max, uint32_t T)
{
    // Tile roots that can touch a boundary bond: the first and last L sites,
    // the row ends and row starts of the tile's rows, the tile-end site.
    const uint32_t rows = T / l_max + 2u;
    const uint32_t bound = 2u * l_max + 2u * rows + 1u;
    uint32_t h = 64;
    while (h < bound + bound / 4u) h *= 2;
    return h;
}

}  // namespace

// Shared-memory layout of one CTA's tile for lattices of up to l_max sites
// across C CTAs; constexpr so that the common classes get it as a
// compile-time constant.
__host__ __device__ constexpr ClusterLayout cluster_layout_c(uint32_t l_max, uint32_t C)
{
    ClusterLayout ly{};
    ly.l_max = l_max;
    ly.C = C;
    ly.t_max = cluster_tile_size(l_max * l_max, C);
    ly.tw = ly.t_max / 32u;
    ly.hs = cluster_hash_size(l_max, ly.t_max);
    size_t off = 0;
    ly.off_uf = off;
    off = a16(off + 2ull * ly.t_max);
    ly.off_S = off;  // tile, halo of l_max sites, padding
    off = a16(off + 4ull * (ly.tw + (l_max + 31u) / 32u + 4u));
    const size_t plane = a16(4ull * (ly.tw + 4u));
    ly.off_OH = off;
    off += plane;
    ly.off_OV = off;
    off += plane;
    ly.off_FLIP = off;
    off += plane;
    ly.off_ROOT = off;
    off += plane;
    ly.off_YS = off;  // y-seam bonds, one bit per row of the tile
    off = a16(off + 4ull * 16u);
    ly.off_HK = off;
    off = a16(off + 4ull * ly.hs);
    ly.off_HW = off;
    off += 8ull * ly.hs;
    ly.bytes = a16(off);
    return ly;
}

ClusterLayout cluster_layout(uint32_t l_max, uint32_t C) { return cluster_layout_c(l_max, C); }

bool cluster_layout_fits(const ClusterLayout &ly, uint32_t threads)
{
    if (ly.hs > kHashMax) return false;
    if (threads == 512u) return ly.t_max <= kTileHalf && 2 * (ly.bytes + kStaticSmem) <= kSmemPerSm;
    return ly.bytes <= kSmemBudget && ly.t_max <= kTileMax;
}

ClusterPlan cluster_plan(uint32_t L)
{
    // Two 512-thread CTAs per SM hide each other's barrier waits better than
    // one of 1024 (as in the resident engine), but twice the tiles also mean
    // twice the boundary bonds and wider cluster barriers: on B200 the
    // smaller tiles win up to 5 per lattice (L = 300: +10 %, L = 384: +6 %)
    // and lose at 8 (L = 512) and 16 (L = 724).
    for (uint32_t C = 2; C <= kHalfTilesMax; ++C) {
        if (!cluster_tiles_ok(L, C, kTileHalf)) continue;
        if (cluster_layout_fits(cluster_layout(L, C), 512u)) return {C, 512u};
        break;
    }
    for (uint32_t C = 2; C <= kClusterMax; ++C)
        if (cluster_tiles_ok(L, C) && cluster_layout_fits(cluster_layout(L, C), 1024u)) return {C, 1024u};
    return {0u, 0u};
}

uint32_t cluster_size_for(uint32_t L) { return cluster_plan(L).C; }

bool cluster_plan_ok(uint32_t L, ClusterPlan p)
{
    if (p.C < 2u || p.C > kClusterMax || (p.threads != 512u && p.threads != 1024u)) return false;
    const uint32_t cap = p.threads == 512u ? kTileHalf : kTileMax;
    return cluster_tiles_ok(L, p.C, cap) && cluster_layout_fits(cluster_layout(L, p.C), p.threads);
}

namespace {

// Shared scratch of one CTA of the cluster.
struct CRed {
    unsigned long long k1[32], k2[32];
    uint32_t unsat[32], downs[32], ncl[32];
    int mcw[32], mcw2[32];
    // This CTA's partial results, read by rank 0 through DSMEM.
    unsigned long long p_k1, p_k2;
    uint32_t p_unsat, p_downs, p_ncl;
    int p_wrap, p_mc, p_mc2;
    // Rank 0's combined results, read by the other CTAs.
    uint32_t g1, g2, ncl_total;
    // Per chain / per sweep state.
    int item, wrap, err;
    uint32_t front, tile_end;
    Acc acc;
    long long cur_bin;
    long long rec[kRecLen];
    rbim_chain_t ch;
};


// Views of this CTA's shared memory and of the cluster's.
struct Ctx {
    Lat<Word16> t;
    uint32_t *YS;
    uint32_t *HK;
    unsigned long long *HW;
    uint32_t hs, hs_log2;
};

__device__ __forceinline__ Ctx make_ctx(unsigned char *smem, const ClusterLayout &ly, const Tile &tl, CRed &red)
{
    Ctx x;
    Lat<Word16> &t = x.t;
    t.g = Geom{tl.L, tl.Tc, (tl.Tc + 31u) / 32u};
    t.uf.w = (unsigned short *)(smem + ly.off_uf);
    t.uf.sa = (uint32_t)__cvta_generic_to_shared(t.uf.w);
    t.S = (uint32_t *)(smem + ly.off_S);
    t.JH = nullptr;
    t.JV = nullptr;
    t.OH = (uint32_t *)(smem + ly.off_OH);
    t.OV = (uint32_t *)(smem + ly.off_OV);
    t.FLIP = (uint32_t *)(smem + ly.off_FLIP);
    t.ROOT = (uint32_t *)(smem + ly.off_ROOT);
    t.RE = nullptr;
    t.SEAMV = nullptr;
    t.wrap = &red.wrap;
    t.err = &red.err;
    t.cap = tl.Tc + 64u;
    x.YS = (uint32_t *)(smem + ly.off_YS);
    x.HK = (uint32_t *)(smem + ly.off_HK);
    x.HW = (unsigned long long *)(smem + ly.off_HW);
    x.hs = ly.hs;
    x.hs_log2 = 31u - __clz(ly.hs);
    return x;
}



// ---------------------------------------------------------------------------
// Cluster-wide union-find over boundary nodes.
// ---------------------------------------------------------------------------
struct Dist {
    cg::cluster_group cl;
    uint32_t *HK;
    unsigned long long *HW;
    uint32_t hs, hs_log2;
    int *wrap, *err;
    uint32_t cap;

    __device__ __forceinline__ unsigned long long *hw(uint32_t node) const
    {
        return cl.map_shared_rank(HW, node >> 16) + (node & 0xFFFFu);
    }
    __device__ __forceinline__ uint32_t key(uint32_t node) const
    {
        return ((node >> 16) << 16) |
               (*((volatile uint32_t *)(cl.map_shared_rank(HK, node >> 16) + (node & 0xFFFFu))) & 0xFFFFu);
    }
    __device__ __forceinline__ unsigned long long ld(uint32_t node) const
    {
        return *((volatile unsigned long long *)hw(node));
    }
    __device__ __forceinline__ void st(uint32_t node, unsigned long long v) const
    {
        *((volatile unsigned long long *)hw(node)) = v;
    }

    // Node of tile root `m` in tile `tile` (inserted if new).
    __device__ __forceinline__ uint32_t insert(uint32_t tile, uint32_t m) const
    {
        uint32_t *hk = cl.map_shared_rank(HK, tile);
        uint32_t h = (m * 0x9E3779B1u) >> (32u - hs_log2);
        for (uint32_t it = 0; it < hs; ++it) {
            const uint32_t old = atomicCAS(hk + h, kEmptyKey, m);
            if (old == kEmptyKey || old == m) return (tile << 16) | h;
            h = (h + 1u) & (hs - 1u);
        }
        atomicOr(err, kErrUnionCap);
        return (tile << 16) | 0u;
    }

    __device__ __forceinline__ FindResult find(uint32_t n) const
    {
        uint32_t node = n;
        int ax = 0, ay = 0;
        unsigned long long w = ld(node);
        for (uint32_t it = 0;; ++it) {
            const uint32_t p = Word64::parent(w);
            if (p == node) break;
            if (it >= cap) {
                atomicOr(err, kErrFindCap);
                break;
            }
            const unsigned long long wp = ld(p);
            const uint32_t gp = Word64::parent(wp);
            if (gp != p) {
                const int nx = Word64::ox(w) + Word64::ox(wp), ny = Word64::oy(w) + Word64::oy(wp);
                st(node, Word64::make(gp, nx, ny));
                ax += nx;
                ay += ny;
                node = gp;
                w = ld(node);
            } else {
                ax += Word64::ox(w);
                ay += Word64::oy(w);
                node = p;
                w = wp;
            }
        }
        return {node, ax, ay};
    }

    __device__ __forceinline__ uint32_t root_ro(uint32_t n) const
    {
        uint32_t node = n;
        for (uint32_t it = 0;; ++it) {
            const uint32_t p = Word64::parent(ld(node));
            if (p == node) break;
            if (it >= cap) {
                atomicOr(err, kErrFindCap);
                break;
            }
            node = p;
        }
        return node;
    }

    // Union across a boundary bond a -> b with seam crossing (ex, ey).
    __device__ __forceinline__ void unite(uint32_t a, uint32_t b, int ex, int ey) const
    {
        for (uint32_t it = 0; it < cap; ++it) {
            const FindResult fa = find(a);
            const FindResult fb = find(b);
            if (fa.root == fb.root) {
                int f = 0;
                if (Word64::nonzero(ex + fb.ax - fa.ax)) f |= 1;
                if (Word64::nonzero(ey + fb.ay - fa.ay)) f |= 2;
                if (f) atomicOr(wrap, f);
                return;
            }
            if (key(fa.root) < key(fb.root)) {
                const unsigned long long expect = Word64::make(fb.root, 0, 0);
                const unsigned long long v = Word64::make(fa.root, fa.ax - ex - fb.ax, fa.ay - ey - fb.ay);
                if (atomicCAS(hw(fb.root), expect, v) == expect) return;
            } else {
                const unsigned long long expect = Word64::make(fa.root, 0, 0);
                const unsigned long long v = Word64::make(fb.root, fb.ax + ex - fa.ax, fb.ay + ey - fa.ay);
                if (atomicCAS(hw(fa.root), expect, v) == expect) return;
            }
        }
        atomicOr(err, kErrUnionCap);
    }
};

// (b) Boundary bonds owned by this tile: x-bonds of its last L sites, the
// y-bond from its last site into the next tile, and the y-seam bonds of the
// rows ending in it.  Lane i of a warp takes item i0 + i, so the x-bonds along
// the last row sit in consecutive lanes and repeated pairs of tile roots are
// dropped before they reach the cluster-wide union-find.
template <int NT>
__device__ __forceinline__ void tile_boundary(const Ctx &x, const Tile &tl, const Dist &d, uint32_t tile_end,
                                              bool walk, uint32_t tid)
{
    const Lat<Word16> &t = x.t;
    const uint32_t rows_end = (tl.b + tl.Tc) / tl.L;  // rows x0 .. rows_end-1 end in the tile
    const uint32_t n_rows = rows_end - tl.x0;
    const uint32_t items = tl.L + 1u + n_rows;
    const uint32_t nxt = tl.c + 1u == tl.C ? 0u : tl.c + 1u;
    const uint32_t lane = tid & 31u;
    for (uint32_t i0 = tid & ~31u; i0 < items; i0 += NT) {
        const uint32_t i = i0 + lane;
        bool live = false;
        uint32_t a = 0, tb = 0, bl = 0;
        int ex = 0, ey = 0;
        if (i < tl.L) {
            a = tl.Tc - tl.L + i;
            if ((t.OH[a >> 5] >> (a & 31u)) & 1u) {
                live = true;
                const uint32_t n = tl.b + a;
                if (n + tl.L >= tl.N) {
                    tb = 0u;
                    bl = n + tl.L - tl.N;
                    ex = 1;
                } else {
                    tb = nxt;
                    bl = a + tl.L - tl.Tc;
                }
            }
        } else if (i == tl.L) {
            if (tile_end) {
                live = true;
                a = tl.Tc - 1u;
                tb = nxt;
                bl = 0u;
            }
        } else if (i < items) {
            const uint32_t row = i - tl.L - 1u;
            if ((x.YS[row >> 5] >> (row & 31u)) & 1u) {
                live = true;
                const uint32_t xr = tl.x0 + row;
                a = xr * tl.L + tl.L - 1u - tl.b;
                const uint32_t start = xr * tl.L;
                if (start >= tl.b) {
                    tb = tl.c;
                    bl = start - tl.b;
                } else {
                    tb = tl.c - 1u;
                    bl = start - (tl.b - tl.T);
                }
                ey = 1;
            }
        }
        uint32_t ra = 0, rb = 0;
        if (live) {
            const unsigned short *ufb = tb == tl.c ? t.uf.w : d.cl.map_shared_rank(t.uf.w, tb);
            if (walk) {
                ra = tile_root_walk(t.uf.w, a, t.cap, d.err);
                rb = (tb << 16) | tile_root_walk(ufb, bl, t.cap, d.err);
            } else {
                ra = tile_root(t.uf.w, a);
                rb = (tb << 16) | tile_root(ufb, bl);
            }
        }
        // A bond joining the same two tile roots with the same seam crossing
        // as the previous lane's closes a loop of winding zero (paths inside a
        // tile never wrap) and changes nothing.
        const int tag = live ? 1 + ex + 2 * ey : 0;
        const uint32_t pra = __shfl_up_sync(0xFFFFFFFFu, ra, 1), prb = __shfl_up_sync(0xFFFFFFFFu, rb, 1);
        const int ptag = __shfl_up_sync(0xFFFFFFFFu, tag, 1);
        if (!live || (lane > 0u && ptag == tag && pra == ra && prb == rb)) continue;
        const uint32_t na = d.insert(tl.c, ra);
        const uint32_t nb = d.insert(tb, rb & 0xFFFFu);
        d.unite(na, nb, ex, ey);
    }
}

// Spin halo after a flip: the first L spins of the next tile (of the first
// tile, for the last one) at bits Tc .. Tc+L-1, and the front spin (the row
// start of the tile's first row, when that row began in the previous tile).
template <int NT>
__device__ __forceinline__ void tile_halo(const Ctx &x, const Tile &tl, const cg::cluster_group &cl, CRed &red,
                                          uint32_t tid)
{
    uint32_t *S = x.t.S;
    const uint32_t nxt = tl.c + 1u == tl.C ? 0u : tl.c + 1u;
    const uint32_t *rs = cl.map_shared_rank(S, nxt);
    const uint32_t lw = (tl.L + 31u) >> 5;
    const uint32_t sh = tl.Tc & 31u, d0 = tl.Tc >> 5;
    const uint32_t lmask = (tl.L & 31u) ? (1u << (tl.L & 31u)) - 1u : 0xFFFFFFFFu;
    for (uint32_t k = tid; k <= lw; k += NT) {
        const uint32_t hk = k < lw ? (rs[k] & (k + 1u == lw ? lmask : 0xFFFFFFFFu)) : 0u;
        uint32_t v;
        if (sh == 0u) {
            v = hk;
        } else {
            const uint32_t hp = (k > 0u) ? (rs[k - 1u] & (k == lw ? lmask : 0xFFFFFFFFu)) : 0u;
            v = (hk << sh) | (k > 0u ? hp >> (32u - sh) : 0u);
            if (k == 0u) v |= S[d0] & ((1u << sh) - 1u);
        }
        S[d0 + k] = v;
    }
    if (tid == 0) {
        uint32_t front = 0;
        if (tl.f) {
            const uint32_t q = tl.x0 * tl.L - (tl.b - tl.T);
            const uint32_t *ps = cl.map_shared_rank(S, tl.c - 1u);
            front = (ps[q >> 5] >> (q & 31u)) & 1u;
        }
        red.front = front;
    }
}


// Root node of this tile's node in slot k, once the boundary stage is over
// (the low word of HW; the high word accumulates merged sizes).
__device__ __forceinline__ uint32_t node_root(const Ctx &x, uint32_t k)
{
    return *((volatile uint32_t *)(x.HW + k));
}

// Tile root of the node in slot k: the low half of its hash word (the high
// half carries its root node between the two halves of the propagation).
__device__ __forceinline__ uint32_t node_key(uint32_t hk) { return hk & 0xFFFFu; }

// The open-tile union and root walks as separate (non-inlined) functions: the
// cluster kernel keeps more state live across its phases than the resident
// one, and compiled inline these pointer-chasing loops lose registers to it.
template <int NT>
static __device__ __noinline__ void cluster_union(const Lat<Word16> &t, uint32_t tid)
{
    phase_union_open(t, tid, NT);
}

template <int NT>
static __device__ __noinline__ void cluster_roots(const Lat<Word16> &t, uint32_t tid)
{
    (void)phase_roots_flat(t, tid, NT);
}


// NT threads per CTA.  LC > 0: the layout is cluster_layout_c(LC, CC), a
// compile-time constant, and the cluster has CC CTAs; LC == 0: the layout
// passed in.
template <int NT, int LC, int CC>
__global__ void __launch_bounds__(NT, NT >= 1024 ? 1 : 1024 / NT)
    k_cluster_sweeps(rbim_chain_t *chains, int n_chains, uint32_t *spin_pool, const uint32_t *coupling_pool,
                     long long *acc_i, double *acc_f, int32_t *records, int n_sweeps, int *queue, int *status,
                     ClusterLayout ly_arg)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ CRed red;
    constexpr ClusterLayout kly = cluster_layout_c(LC > 0 ? LC : 512, CC > 0 ? CC : 4);
    const ClusterLayout ly = LC > 0 ? kly : ly_arg;
    cg::cluster_group cl = cg::this_cluster();
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    constexpr uint32_t nwarps = NT / 32;
    constexpr uint32_t kCap = NT >= 1024 ? kTileMax : kTileHalf;
    const uint32_t C = CC > 0 ? (uint32_t)CC : cl.num_blocks(), c = cl.block_rank();

    if (tid == 0) red.err = 0;
    for (;;) {
        if (c == 0 && tid == 0) red.item = atomicAdd(queue, 1);
        cl.sync();
        if (tid == 0 && c != 0) red.item = *cl.map_shared_rank(&red.item, 0);
        cl.sync();
        const int item = red.item;
        if (item >= n_chains) break;
        if (tid == 0) {
            red.ch = chains[item];
            red.cur_bin = -1;
        }
        __syncthreads();
        const rbim_chain_t &ch = red.ch;
        const bool bad = ch.L < 3 || ch.L > (int64_t)ly.l_max || ch.sweeps_per_bin < 1 || ch.n_bins < 0 ||
                         ch.n_therm < 0 || ch.walk_cap < 0 || !cluster_tiles_ok((uint32_t)ch.L, C, kCap) ||
                         cluster_tile_size((uint32_t)(ch.L * ch.L), C) > ly.t_max;
        if (bad) {
            if (tid == 0 && c == 0) atomicOr(status, kErrBadChain);
            continue;
        }
        Tile tl;
        tl.L = (uint32_t)ch.L;
        tl.N = tl.L * tl.L;
        tl.C = C;
        tl.c = c;
        tl.T = cluster_tile_size(tl.N, C);
        tl.b = c * tl.T;
        tl.Tc = min(tl.T, tl.N - tl.b);
        tl.tw = (tl.Tc + 31u) >> 5;
        tl.x0 = tl.b / tl.L;
        tl.f = tl.b - tl.x0 * tl.L;
        tl.nwp = (((tl.N + 31u) >> 5) + 3u) & ~3u;
        const Ctx x = make_ctx(smem, ly, tl, red);
        const Lat<Word16> &t = x.t;
        const Dist d{cl, x.HK, x.HW, x.hs, x.hs_log2, &red.wrap, &red.err, C * x.hs + 64u};
        uint32_t *gS = spin_pool + ch.spin_off + (tl.b >> 5);
        const uint32_t *gJH = coupling_pool + ch.coupling_off + (tl.b >> 5);
        const uint32_t *gJV = coupling_pool + ch.coupling_off + tl.nwp + (tl.b >> 5);
        const uint32_t s_words = ly.tw + (ly.l_max + 31u) / 32u + 4u;

        // Load the tile's spins; zero the halo and padding.
        for (uint32_t w = tid; w < s_words; w += NT) t.S[w] = w < tl.tw ? gS[w] & t.g.valid(w) : 0u;
        const uint64_t t_end = (uint64_t)ch.n_therm + (uint64_t)ch.n_bins * (uint64_t)ch.sweeps_per_bin;
        uint64_t sweep = ch.sweep;
        const uint64_t stop = min(t_end, sweep + (uint64_t)max(n_sweeps, 0));
        cl.sync();
        tile_halo<NT>(x, tl, cl, red, tid);
        __syncthreads();

        for (; sweep < stop; ++sweep) {
            const bool measure = sweep >= (uint64_t)ch.n_therm;
            const uint32_t front = red.front;
            if (tid == 0) {
                red.wrap = 0;
                red.tile_end = 0;
            }
            for (uint32_t i = tid; i < 16u; i += NT) x.YS[i] = 0u;
            __syncthreads();
            tile_activate<NT>(x.t, x.YS, tl, make_rng(ch.key, sweep, ch.thr), gJH, gJV, front, red.tile_end, warp,
                              nwarps, tid);
            __syncthreads();
            phase_heads<Word16>(t, warp, nwarps);
            for (uint32_t w = tid; w < t.g.NW; w += NT) t.ROOT[w] = 0u;
            for (uint32_t k = tid; k < x.hs; k += NT) {
                x.HK[k] = kEmptyKey;
                x.HW[k] = Word64::make((c << 16) | k, 0, 0);
            }
            __syncthreads();
            cluster_union<NT>(t, tid);
            __syncthreads();
            // With at least one word per thread the roots are found in one
            // pass with the flip, after the boundary stage (roots_flip_pieces);
            // the boundary bonds' tile roots are then found by read-only walks.
            const bool merged = t.g.NW >= (uint32_t)NT;
            if (!merged) {
                cluster_roots<NT>(t, tid);
                __syncthreads();
            }
            cl.sync();  // every tile's unions (and roots) are final

            tile_boundary<NT>(x, tl, d, red.tile_end, merged, tid);
            cl.sync();  // every boundary union is done

            // Root node of each of this tile's nodes, kept in the high half of
            // its hash word (tile in 4 bits, slot in 12) until every walk is done.
            for (uint32_t k = tid; k < x.hs; k += NT) {
                const uint32_t hk = x.HK[k];
                if (hk == kEmptyKey) continue;
                const uint32_t r = d.root_ro((c << 16) | k);
                x.HK[k] = node_key(hk) | (((r >> 16) << 12 | (r & 0xFFFu)) << 16);
            }
            cl.sync();  // all walks done before the words change
            // Union-find word -> root node (merged size 0); a merged tile root
            // takes the flip bit of its cluster: the raw bit of the root
            // node's site, which no CTA changes.
            for (uint32_t k = tid; k < x.hs; k += NT) {
                const uint32_t hk = x.HK[k];
                if (hk == kEmptyKey) continue;
                const uint32_t r = ((hk >> 28) << 16) | ((hk >> 16) & 0xFFFu), m = node_key(hk);
                x.HK[k] = m;
                x.HW[k] = (unsigned long long)r;
                if (r != ((c << 16) | k)) {
                    const uint32_t mr = node_key(*cl.map_shared_rank(x.HK + (r & 0xFFFFu), r >> 16));
                    const uint32_t *fl = cl.map_shared_rank(t.FLIP, r >> 16);
                    if ((fl[mr >> 5] >> (mr & 31u)) & 1u)
                        atomicOr(t.FLIP + (m >> 5), 1u << (m & 31u));
                    else
                        atomicAnd(t.FLIP + (m >> 5), ~(1u << (m & 31u)));
                }
            }
            __syncthreads();
            // Flip run pieces by their tile root's FLIP bit; every piece
            // leader's word is left holding its tile root (without the merged
            // pass only in measured sweeps), and the merged pass also sets the
            // ROOT bits.
            if (merged)
                (void)roots_flip_pieces(t, tid, NT);
            else
                flip_pieces(t, tid, NT, measure);
            __syncthreads();
            cl.sync();  // every flip is done
            tile_halo<NT>(x, tl, cl, red, tid);
            __syncthreads();

            if (!measure) continue;

            // ---- measurement (reference sw_sweep, src/rbim/swendsen_wang.py:146-172)
            unsigned short *u16 = t.uf.w;
            uint32_t unsat = 0, downs = 0;
            tile_energy<NT>(x.t, tl, gJH, gJV, red.front, tid, unsat, downs);
            // Tile cluster sizes minus one added onto each tile root's own index
            // (a root points at itself): afterwards the word of root m reads
            // m + size - 1, below 65536 because m is the smallest site of its tile
            // cluster, so no add carries out of its 16 bits (tile_size decodes it).
            count_pieces<true>(t, u16, warp, nwarps);
            __syncthreads();
            // FLIP (no longer needed this sweep) becomes the plane of node
            // marks; OV still gives the run pieces of the |M_C| pass.
            for (uint32_t w = tid; w < t.g.NW; w += NT) t.FLIP[w] = 0u;
            __syncthreads();
            // Merged sizes into the root nodes; mark this tile's nodes in FLIP.
            uint32_t rootnodes = 0;
            for (uint32_t k = tid; k < x.hs; k += NT) {
                const uint32_t m = x.HK[k];
                if (m == kEmptyKey) continue;
                const uint32_t r = node_root(x, k);
                atomicOr(t.FLIP + (m >> 5), 1u << (m & 31u));
                unsigned int *hi = (unsigned int *)(cl.map_shared_rank(x.HW, r >> 16) + (r & 0xFFFFu)) + 1;
                atomicAdd(hi, tile_size(u16, m));
                if (r == ((c << 16) | k)) ++rootnodes;
            }
            __syncthreads();
            uint32_t nloc = rootnodes;
            for (uint32_t w = tid; w < t.g.NW; w += NT) nloc += __popc(t.ROOT[w] & ~t.FLIP[w]);
            cl.sync();  // merged sizes are complete

            // Local top two: tile-only clusters and this tile's root nodes.
            unsigned long long k1 = 0, k2 = 0;
            for (uint32_t w = tid; w < t.g.NW; w += NT) {
                uint32_t roots = t.ROOT[w] & ~t.FLIP[w];
                while (roots) {
                    const uint32_t bb = __ffs(roots) - 1u;
                    roots &= roots - 1u;
                    const uint32_t m = (w << 5) + bb;
                    top2_merge(k1, k2, size_key(tile_size(u16, m), tl.b + m), 0ull);
                }
            }
            for (uint32_t k = tid; k < x.hs; k += NT) {
                if (x.HK[k] == kEmptyKey || node_root(x, k) != ((c << 16) | k)) continue;
                top2_merge(k1, k2, size_key((uint32_t)(x.HW[k] >> 32), tl.b + x.HK[k]), 0ull);
            }
            warp_top2(k1, k2);
            uint32_t u = unsat, dn = downs, nc = nloc;
            for (int o = 16; o > 0; o >>= 1) {
                u += __shfl_xor_sync(0xFFFFFFFFu, u, o);
                dn += __shfl_xor_sync(0xFFFFFFFFu, dn, o);
                nc += __shfl_xor_sync(0xFFFFFFFFu, nc, o);
            }
            if (lane == 0) {
                red.k1[warp] = k1;
                red.k2[warp] = k2;
                red.unsat[warp] = u;
                red.downs[warp] = dn;
                red.ncl[warp] = nc;
            }
            __syncthreads();
            if (warp == 0) {
                const bool live = lane < nwarps;
                unsigned long long a1 = live ? red.k1[lane] : 0ull, a2 = live ? red.k2[lane] : 0ull;
                warp_top2(a1, a2);
                uint32_t su = live ? red.unsat[lane] : 0u, sd = live ? red.downs[lane] : 0u;
                uint32_t sn = live ? red.ncl[lane] : 0u;
                for (int o = 16; o > 0; o >>= 1) {
                    su += __shfl_xor_sync(0xFFFFFFFFu, su, o);
                    sd += __shfl_xor_sync(0xFFFFFFFFu, sd, o);
                    sn += __shfl_xor_sync(0xFFFFFFFFu, sn, o);
                }
                if (lane == 0) {
                    red.p_k1 = a1;
                    red.p_k2 = a2;
                    red.p_unsat = su;
                    red.p_downs = sd;
                    red.p_ncl = sn;
                    red.p_wrap = red.wrap;
                }
            }
            cl.sync();  // partials are visible
            long long *rec = red.rec;  // rank 0's record of the sweep
            if (c == 0 && warp == 0) {
                unsigned long long a1 = 0, a2 = 0;
                uint32_t su = 0, sd = 0, sn = 0;
                int wr = 0;
                if (lane < C) {
                    const CRed *o = cl.map_shared_rank(&red, lane);
                    a1 = o->p_k1;
                    a2 = o->p_k2;
                    su = o->p_unsat;
                    sd = o->p_downs;
                    sn = o->p_ncl;
                    wr = o->p_wrap;
                }
                warp_top2(a1, a2);
                for (int o = 16; o > 0; o >>= 1) {
                    su += __shfl_xor_sync(0xFFFFFFFFu, su, o);
                    sd += __shfl_xor_sync(0xFFFFFFFFu, sd, o);
                    sn += __shfl_xor_sync(0xFFFFFFFFu, sn, o);
                    wr |= __shfl_xor_sync(0xFFFFFFFFu, wr, o);
                }
                if (lane == 0) {
                    red.g1 = 0xFFFFFFFFu - (uint32_t)(a1 & 0xFFFFFFFFull);
                    red.g2 = 0xFFFFFFFFu - (uint32_t)(a2 & 0xFFFFFFFFull);
                    red.ncl_total = sn;
                    rec[0] = 2ll * (long long)su - 2ll * (long long)tl.N;
                    rec[1] = (long long)tl.N - 2ll * (long long)sd;
                    rec[2] = sn;
                    rec[3] = (long long)(a1 >> 32);
                    rec[5] = (long long)(a2 >> 32);
                    rec[7] = wr & 1;
                    rec[8] = (wr >> 1) & 1;
                }
            }
            cl.sync();  // rank 0's results are visible
            if (tid == 0 && c != 0) {
                const CRed *o = cl.map_shared_rank(&red, 0);
                red.g1 = o->g1;
                red.g2 = o->g2;
                red.ncl_total = o->ncl_total;
            }
            __syncthreads();
            const uint32_t g1 = red.g1, g2 = red.g2;
            const bool many = red.ncl_total > 1u;
            // |M_C2| only when the chain's records are written (the bin sums
            // do not use it).
            const bool second = records && ch.rec_off >= 0;
            if (many) {
                // Tile roots of the largest cluster, marked in OH, and with
                // `second` those of the second largest in FLIP (whose node
                // marks are no longer needed).
                for (uint32_t w = tid; w < t.g.NW; w += NT) {
                    t.OH[w] = 0u;
                    if (second) t.FLIP[w] = 0u;
                }
                __syncthreads();
                if (tid == 0 && g1 >= tl.b && g1 < tl.b + tl.Tc) {
                    const uint32_t m = g1 - tl.b;
                    atomicOr(t.OH + (m >> 5), 1u << (m & 31u));
                }
                if (second && tid == 0 && g2 >= tl.b && g2 < tl.b + tl.Tc) {
                    const uint32_t m = g2 - tl.b;
                    atomicOr(t.FLIP + (m >> 5), 1u << (m & 31u));
                }
                for (uint32_t k = tid; k < x.hs; k += NT) {
                    if (x.HK[k] == kEmptyKey) continue;
                    const uint32_t r = node_root(x, k);
                    const uint32_t rt = r >> 16;
                    const uint32_t gr = rt * tl.T + *cl.map_shared_rank(x.HK + (r & 0xFFFFu), rt);
                    if (gr == g1) {
                        const uint32_t m = x.HK[k];
                        atomicOr(t.OH + (m >> 5), 1u << (m & 31u));
                    } else if (second && gr == g2) {
                        const uint32_t m = x.HK[k];
                        atomicOr(t.FLIP + (m >> 5), 1u << (m & 31u));
                    }
                }
                __syncthreads();
                int mc = 0, mc2 = 0;
                // One lane per word, one test per run piece: a piece leader's
                // word holds its tile root (the root's own word its size).
                for (uint32_t w = tid; w < t.g.NW; w += NT) {
                    const uint32_t valid = t.g.valid(w);
                    uint32_t lead = piece_leaders(t, w, valid);
                    const uint32_t roots = t.ROOT[w], sw = t.S[w];
                    const uint32_t nv = (uint32_t)__popc(valid);
                    while (lead) {
                        const uint32_t b = __ffs(lead) - 1u;
                        lead &= lead - 1u;
                        const uint32_t end = lead ? (uint32_t)(__ffs(lead) - 1) : nv;
                        const uint32_t n = (w << 5) + b;
                        const uint32_t r = ((roots >> b) & 1u) ? n : (uint32_t)u16[n];
                        const uint32_t pm = (end - b == 32u) ? 0xFFFFFFFFu : (((1u << (end - b)) - 1u) << b);
                        const int m = (int)__popc(pm) - 2 * (int)__popc(pm & sw);
                        if ((t.OH[r >> 5] >> (r & 31u)) & 1u) mc += m;
                        if (second && ((t.FLIP[r >> 5] >> (r & 31u)) & 1u)) mc2 += m;
                    }
                }
                for (int o = 16; o > 0; o >>= 1) {
                    mc += __shfl_xor_sync(0xFFFFFFFFu, mc, o);
                    mc2 += __shfl_xor_sync(0xFFFFFFFFu, mc2, o);
                }
                if (lane == 0) {
                    red.mcw[warp] = mc;
                    red.mcw2[warp] = mc2;
                }
                __syncthreads();
                if (tid == 0) {
                    int s = 0, s2 = 0;
                    for (uint32_t i = 0; i < nwarps; ++i) {
                        s += red.mcw[i];
                        s2 += red.mcw2[i];
                    }
                    red.p_mc = s;
                    red.p_mc2 = s2;
                }
            }
            cl.sync();  // M_C partials are visible
            if (c == 0 && tid == 0) {
                long long mc_total = rec[1], mc2_total = 0;
                if (many) {
                    mc_total = 0;
                    for (uint32_t i = 0; i < C; ++i) {
                        const CRed *o = cl.map_shared_rank(&red, i);
                        mc_total += o->p_mc;
                        mc2_total += o->p_mc2;
                    }
                }
                rec[4] = mc_total < 0 ? -mc_total : mc_total;
                rec[6] = mc2_total < 0 ? -mc2_total : mc2_total;
                const long long idx = (long long)(sweep - (uint64_t)ch.n_therm);
                const long long bin = idx / ch.sweeps_per_bin;
                if (bin != red.cur_bin) {
                    if (red.cur_bin >= 0)
                        red.acc.store(acc_i + (ch.acc_off + red.cur_bin) * kAccInt,
                                      acc_f + (ch.acc_off + red.cur_bin) * kAccF64);
                    red.acc.load(acc_i + (ch.acc_off + bin) * kAccInt, acc_f + (ch.acc_off + bin) * kAccF64);
                    red.cur_bin = bin;
                }
                red.acc.add(rec[0], rec[1], rec[2], rec[3], rec[4], rec[5], (int)rec[7], (int)rec[8]);
                if (second) {
                    int32_t *row = records + (ch.rec_off + idx) * kRecLen;
#pragma unroll
                    for (int k = 0; k < kRecLen; ++k) row[k] = (int32_t)rec[k];
                }
            }
        }
        if (c == 0 && tid == 0) {
            if (red.cur_bin >= 0)
                red.acc.store(acc_i + (ch.acc_off + red.cur_bin) * kAccInt,
                              acc_f + (ch.acc_off + red.cur_bin) * kAccF64);
            chains[item].sweep = stop;
        }
        for (uint32_t w = tid; w < tl.tw; w += NT) gS[w] = t.S[w] & t.g.valid(w);
        cl.sync();  // halo reads of this chain are over before the next load
    }
    if (tid == 0 && red.err) atomicOr(status, red.err);
}

}  // namespace

namespace {

template <int NT, int LC, int CC>
cudaError_t occupancy_t(const ClusterLayout &ly, uint32_t C, int *clusters)
{
    cudaError_t e = cudaFuncSetAttribute(k_cluster_sweeps<NT, LC, CC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)ly.bytes);
    if (e != cudaSuccess) return e;
    if (C > 8u) {
        e = cudaFuncSetAttribute(k_cluster_sweeps<NT, LC, CC>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e != cudaSuccess) return e;
    }
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(C, 1, 1);
    cfg.blockDim = dim3(NT, 1, 1);
    cfg.dynamicSmemBytes = ly.bytes;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaOccupancyMaxActiveClusters(clusters, k_cluster_sweeps<NT, LC, CC>, &cfg);
}

template <int NT, int LC, int CC>
cudaError_t launch_t(const ClusterLayout &ly, uint32_t C, const rbim_chain_t *chains, int n_chains,
                     uint32_t *spin_pool, const uint32_t *coupling_pool, long long *acc_i, double *acc_f,
                     int32_t *rec, int n_sweeps, int *queue, int *status, cudaStream_t stream)
{
    int clusters = 0;
    cudaError_t e = occupancy_t<NT, LC, CC>(ly, C, &clusters);
    if (e != cudaSuccess) return e;
    if (clusters <= 0) return cudaErrorInvalidConfiguration;
    const int n_clusters = std::min(clusters, n_chains);
    e = cudaMemsetAsync(queue, 0, sizeof(int), stream);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3((unsigned)n_clusters * C, 1, 1);
    cfg.blockDim = dim3(NT, 1, 1);
    cfg.dynamicSmemBytes = ly.bytes;
    cfg.stream = stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    e = cudaLaunchKernelEx(&cfg, k_cluster_sweeps<NT, LC, CC>, const_cast<rbim_chain_t *>(chains), n_chains,
                           spin_pool, coupling_pool, acc_i, acc_f, rec, n_sweeps, queue, status, ly);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

// One launch configuration: CTA size, compile-time layout class and cluster
// size, and the layout.  The classes with a compile-time layout are the two
// benchmark sizes: L = 512 (4 CTAs) and L = 1024 (16 CTAs), both with 1024
// threads; each covers the smaller lattices of the same plan.
struct Launch {
    uint32_t threads, lc, C;
    ClusterLayout ly;
};

// The launch of a plan: the classes with a compile-time layout (4 CTAs of
// 1024 threads up to L = 512, 16 up to L = 1024) take it whatever L they run,
// any other plan the run-time layout of l_max.
Launch launch_for(uint32_t l_max, ClusterPlan plan)
{
    Launch l{plan.threads, 0u, plan.C, {}};
    if (plan.C == 0) return l;
    if (plan.threads == 1024u && plan.C == 4u && l_max <= 512u && cluster_plan_ok(512u, plan))
        l.lc = 512u;
    else if (plan.threads == 1024u && plan.C == 16u && l_max <= 1024u && cluster_plan_ok(1024u, plan))
        l.lc = 1024u;
    l.ly = cluster_layout(l.lc ? l.lc : l_max, plan.C);
    return l;
}

}  // namespace

cudaError_t cluster_occupancy(uint32_t l_max, int *clusters) { return cluster_occupancy_plan(l_max, cluster_plan(l_max), clusters); }

cudaError_t cluster_occupancy_plan(uint32_t l_max, ClusterPlan plan, int *clusters)
{
    *clusters = 0;
    const Launch l = launch_for(l_max, plan);
    if (l.C == 0 || !cluster_layout_fits(l.ly, l.threads)) return cudaSuccess;
    if (l.lc == 512) return occupancy_t<1024, 512, 4>(l.ly, l.C, clusters);
    if (l.lc == 1024) return occupancy_t<1024, 1024, 16>(l.ly, l.C, clusters);
    if (l.threads == 512) return occupancy_t<512, 0, 0>(l.ly, l.C, clusters);
    return occupancy_t<1024, 0, 0>(l.ly, l.C, clusters);
}

cudaError_t launch_cluster_sweeps(const rbim_chain_t *chains, int n_chains, int l_max, uint32_t *spin_pool,
                                  const uint32_t *coupling_pool, long long *acc_i, double *acc_f, int32_t *rec,
                                  int n_sweeps, int *queue, int *status, cudaStream_t stream)
{
    return launch_cluster_sweeps_plan(chains, n_chains, l_max, cluster_plan((uint32_t)l_max), spin_pool,
                                      coupling_pool, acc_i, acc_f, rec, n_sweeps, queue, status, stream);
}

cudaError_t launch_cluster_sweeps_plan(const rbim_chain_t *chains, int n_chains, int l_max, ClusterPlan plan,
                                       uint32_t *spin_pool, const uint32_t *coupling_pool, long long *acc_i,
                                       double *acc_f, int32_t *rec, int n_sweeps, int *queue, int *status,
                                       cudaStream_t stream)
{
    const Launch l = launch_for((uint32_t)l_max, plan);
    if (l.C == 0) return cudaErrorInvalidValue;
    if (!cluster_layout_fits(l.ly, l.threads)) return cudaErrorInvalidConfiguration;
    if (l.lc == 512)
        return launch_t<1024, 512, 4>(l.ly, l.C, chains, n_chains, spin_pool, coupling_pool, acc_i, acc_f, rec,
                                      n_sweeps, queue, status, stream);
    if (l.lc == 1024)
        return launch_t<1024, 1024, 16>(l.ly, l.C, chains, n_chains, spin_pool, coupling_pool, acc_i, acc_f, rec,
                                        n_sweeps, queue, status, stream);
    if (l.threads == 512)
        return launch_t<512, 0, 0>(l.ly, l.C, chains, n_chains, spin_pool, coupling_pool, acc_i, acc_f, rec,
                                   n_sweeps, queue, status, stream);
    return launch_t<1024, 0, 0>(l.ly, l.C, chains, n_chains, spin_pool, coupling_pool, acc_i, acc_f, rec, n_sweeps,
                                queue, status, stream);
}

}  // namespace rbim

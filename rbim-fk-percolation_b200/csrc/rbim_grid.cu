// Grid engine: one lattice over the whole GPU, for a single chain (the
// drop-in for one run_single_realization task, src/rbim/simulation.py:196-242,
// around sw_sweep, src/rbim/swendsen_wang.py:103-172).  One cooperative
// launch runs every sweep of a call.  Its C CTAs (one or more per SM, all
// resident at once) split the lattice into C tiles of consecutive sites, as
// the cluster engine's CTAs do, and each CTA keeps its tile in shared memory
// for the whole call:
//
//  1. activation of the bonds owned by the tile's sites (the spins of the
//     next tile's first row, and the row start of a partial first row, come
//     from the global spin plane, which every tile rewrites after its flip);
//  2. the open-tile labelling of the resident engine (16-bit parents, run
//     heads, flat union and root walks);
//  3. the tile roots that boundary bonds can touch become nodes of a
//     union-find in global memory, one Word64 per site (parent | wx | wy),
//     indexed by global site; after a grid barrier the boundary bonds --
//     x-bonds from the last L sites of a tile into the next one (across the
//     x seam from the last tile to the first), the y-bond between two tiles,
//     the y-seam bonds -- are unioned there with image offsets, the larger
//     site hooked under the smaller, so a merged cluster's root is its
//     smallest site; a bond closing a loop with nonzero summed offset winds
//     around the torus (src/rbim/_unionfind.py:104-124);
//  4. after a second barrier every node finds its root and takes the root's
//     raw flip bit (published before the first barrier); the tile flips by
//     run pieces and writes its spins back (measured sweeps also add their
//     cluster sizes into the root nodes' words); a third barrier;
//  5. measured sweeps: every CTA's partials (top two, energy, magnetization,
//     clusters, wraps) are combined by every CTA after a fourth barrier, the
//     |M_C1|, |M_C2| sums are added up in global memory, and CTA 0 writes the
//     record and the bin sums after the next sweep's first barrier (or a last
//     barrier at the end of the call), off the critical path of the sweep.
//
// Every load of data another CTA wrote during the launch bypasses L1
// (ld.global.cg): L1 is not coherent across SMs.  Every wait at a grid
// barrier is bounded; a CTA that gives up sets RBIM_STATUS_GRID_WAIT and an
// abort flag after which no CTA waits again, so the launch always ends.
#include <algorithm>
#include <mutex>
#include <vector>

#include "rbim_internal.h"
#include "rbim_open.cuh"
#include "rbim_tile.cuh"

// Phase profile (profiling builds only, -DRBIM_PROFILE_PHASES): thread 0 of
// CTA 0 adds the SM cycles since its previous mark to slot k, read and reset
// with rbim_grid_profile_cycles.
#ifdef RBIM_PROFILE_PHASES
__device__ unsigned long long g_grid_phase_cycles[32];
extern "C" int rbim_grid_profile_cycles(unsigned long long *out, int reset)
{
    if (reset) {
        unsigned long long z[32] = {0};
        return (int)cudaMemcpyToSymbol(g_grid_phase_cycles, z, sizeof(z));
    }
    return (int)cudaMemcpyFromSymbol(out, g_grid_phase_cycles, sizeof(unsigned long long) * 32);
}
#define RBIM_GRID_MARK(k)                                                                    \
    do {                                                                                     \
        if (blockIdx.x == 0 && threadIdx.x == 0) {                                           \
            const long long now_ = clock64();                                                \
            g_grid_phase_cycles[k] += (unsigned long long)(now_ - prof_t);                   \
            prof_t = now_;                                                                   \
        }                                                                                    \
    } while (0)
#define RBIM_GRID_PROF_START long long prof_t = clock64()
#else
#define RBIM_GRID_MARK(k) ((void)0)
#define RBIM_GRID_PROF_START ((void)0)
#endif

namespace rbim {

namespace {

constexpr uint32_t kGridTileMax = 65536;                     // 16-bit tile parents
constexpr size_t kGridSmemPerSm = 228 * 1024;
constexpr size_t kGridStaticSmem = 3 * 1024;
constexpr long long kGridWaitCycles = 2000000000ll;          // about one second at 1.9 GHz

__host__ __device__ constexpr size_t g16(size_t v) { return (v + 15) & ~size_t(15); }
__host__ __device__ constexpr size_t g256(size_t v) { return (v + 255) & ~size_t(255); }

}  // namespace

// Shared-memory layout of one CTA's tile for an L x L lattice split in C
// tiles.
struct GridLayout {
    uint32_t L, C, t_max, tw, rows_max, node_max, bh;
    size_t off_uf, off_S, off_OH, off_OV, off_FLIP, off_ROOT, off_NODE, off_YS, off_NK, off_NR, off_BH, bytes;
};

// with_hash: room for the boundary-bond hash (bh entries, a power of two at
// least 1.5 times the tile's boundary bonds); without it bh = 0.
GridLayout grid_layout(uint32_t L, uint32_t C, bool with_hash)
{
    GridLayout ly{};
    ly.L = L;
    ly.C = C;
    ly.t_max = cluster_tile_size(L * L, C);
    ly.tw = ly.t_max / 32u;
    ly.rows_max = ly.t_max / L + 2u;
    // Sites whose tile roots can be nodes: the first and last L sites, the
    // row starts and row ends, the tile's last site.
    ly.node_max = 2u * L + 2u * ly.rows_max + 4u;
    size_t off = 0;
    ly.off_uf = off;
    off = g16(off + 2ull * ly.t_max);
    ly.off_S = off;  // tile, halo of L sites, padding
    off = g16(off + 4ull * (ly.tw + (L + 31u) / 32u + 4u));
    const size_t plane = g16(4ull * (ly.tw + 4u));
    ly.off_OH = off;
    off += plane;
    ly.off_OV = off;
    off += plane;
    ly.off_FLIP = off;
    off += plane;
    ly.off_ROOT = off;
    off += plane;
    ly.off_NODE = off;
    off += plane;
    ly.off_YS = off;  // y-seam bonds, one bit per row of the tile
    off = g16(off + 4ull * (ly.rows_max / 32u + 1u));
    ly.off_NK = off;  // node list: tile root (local site)
    off = g16(off + 4ull * ly.node_max);
    ly.off_NR = off;  // node list: root node (global site) after the boundary stage
    off = g16(off + 4ull * ly.node_max);
    ly.bh = 0;
    if (with_hash) {
        const uint32_t items = L + 1u + ly.rows_max;
        ly.bh = 64;
        while (ly.bh < items + items / 2u) ly.bh *= 2u;
    }
    ly.off_BH = off;  // boundary-bond hash: (tile root, node, seam crossing) of the bonds unioned
    off = g16(off + 8ull * ly.bh);
    ly.bytes = off;
    return ly;
}

namespace {

// Grid-wide barrier state (zeroed before every launch): the arrival counter
// and the abort flag on separate 128-byte lines, and the |M_C1|, |M_C2| sums
// of the last two measured sweeps (by sweep parity).
struct GridSync {
    unsigned int count;  // arrivals, never reset within a launch
    unsigned int pad0[31];
    int abort;
    unsigned int pad1[31];
    int mc[2][2];
};

// One CTA's partial results of a measured sweep.
struct __align__(16) GridPartial {
    unsigned long long k1, k2;
    uint32_t unsat, downs, ncl;
    int wrap;
    uint32_t pad[8];
};

// Global workspace of a launch (rbim_grid_workspace_bytes).
struct GridWs {
    GridSync *sync;
    GridPartial *part;      // C partials
    uint32_t *FR;           // C x L: global tile root of each tile's first L sites
    uint32_t *FRONT;        // C: global tile root of a tile's first row start when it lies in the previous tile
    uint32_t *FLIPG;        // raw flip bits of every site
    unsigned long long *G;  // node words, one per site
};

size_t grid_ws_bytes(uint32_t L, uint32_t C)
{
    const size_t N = (size_t)L * L, nwp = (((N + 31) / 32) + 3) & ~size_t(3);
    size_t off = g256(sizeof(GridSync));
    off = g256(off + sizeof(GridPartial) * C);
    off = g256(off + 4ull * C * L);
    off = g256(off + 4ull * C);
    off = g256(off + 4ull * nwp);
    off = g256(off + 8ull * N);
    return off;
}

GridWs grid_ws(void *base, uint32_t L, uint32_t C)
{
    const size_t N = (size_t)L * L, nwp = (((N + 31) / 32) + 3) & ~size_t(3);
    unsigned char *p = (unsigned char *)base;
    GridWs w;
    size_t off = 0;
    w.sync = (GridSync *)(p + off);
    off = g256(sizeof(GridSync));
    w.part = (GridPartial *)(p + off);
    off = g256(off + sizeof(GridPartial) * C);
    w.FR = (uint32_t *)(p + off);
    off = g256(off + 4ull * C * L);
    w.FRONT = (uint32_t *)(p + off);
    off = g256(off + 4ull * C);
    w.FLIPG = (uint32_t *)(p + off);
    off = g256(off + 4ull * nwp);
    w.G = (unsigned long long *)(p + off);
    return w;
}

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int *p)
{
    unsigned int v;
    asm volatile("ld.acquire.gpu.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned int atom_add_acq_rel(unsigned int *p, unsigned int v)
{
    unsigned int old;
    asm volatile("atom.acq_rel.gpu.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

// Grid-wide barrier of a cooperative launch (every CTA resident).  Thread 0
// of each CTA arrives with one acquire-release add on a counter that only
// grows: barrier k is passed when the counter reaches (k + 1) * nblocks, and
// the last arrival passes at once.  The others wait for that value, for at
// most `wait_cycles` of the SM clock; a CTA that gives up raises the abort
// flag and its error bit, and from then on no CTA waits, so every CTA
// reaches the end of the launch.  The release of the add covers the CTA's
// writes before the barrier (they precede it through __syncthreads); the
// acquire of the final load covers the other CTAs' writes.
__device__ __forceinline__ void grid_sync(GridSync *gs, uint32_t nblocks, long long wait_cycles, int *err)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned int old = atom_add_acq_rel(&gs->count, 1u);
        const unsigned int target = (old / nblocks + 1u) * nblocks;
        if (old + 1u != target && !*((volatile int *)&gs->abort)) {
            const long long t0 = clock64();
            for (uint32_t it = 1; (int)(ld_acquire(&gs->count) - target) < 0; ++it) {
                if ((it & 255u) == 1u) {  // after the first load, then every 256
                    if (*((volatile int *)&gs->abort)) break;
                    if (clock64() - t0 > wait_cycles) {
                        atomicExch(&gs->abort, 1);
                        atomicOr(err, kErrGridWait);
                        break;
                    }
                }
            }
        }
    }
    __syncthreads();
}

// Union-find over the nodes in global memory: node = global site of a tile
// root, key = node, words Word64 (parent | wx | wy).  Loads bypass L1 (words
// change during the launch and from sweep to sweep).  Every node index is
// checked against the lattice before it is used: after a barrier gave up, a
// CTA may read node ids another CTA has not written yet (the workspace holds
// arbitrary bytes), and such an id ends the walk with an error bit instead of
// an access outside the words.
struct GDist {
    unsigned long long *G;
    int *wrap, *err;
    uint32_t cap, n_sites;

    __device__ __forceinline__ unsigned long long ld(uint32_t n) const { return __ldcg(G + n); }
    __device__ __forceinline__ void st(uint32_t n, unsigned long long v) const { __stcg(G + n, v); }

    __device__ __forceinline__ uint32_t root_ro(uint32_t n) const
    {
        uint32_t node = n;
        for (uint32_t it = 0;; ++it) {
            const uint32_t p = Word64::parent(ld(node));
            if (p == node) break;
            if (it >= cap || p >= n_sites) {
                atomicOr(err, kErrFindCap);
                break;
            }
            node = p;
        }
        return node;
    }

    // One path-halving step of the walk at x (summed image offset ox, oy):
    // true when x is a root, false after moving x two levels up.  An id
    // outside the lattice sets `bad` and stops the walk.
    __device__ __forceinline__ bool hstep(uint32_t &x, int &ox, int &oy, bool &bad) const
    {
        const unsigned long long w = ld(x);
        const uint32_t p = Word64::parent(w);
        if (p == x) return true;
        if (p >= n_sites) {
            bad = true;
            return true;
        }
        const unsigned long long wp = ld(p);
        const uint32_t gp = Word64::parent(wp);
        if (gp == p) {
            ox += Word64::ox(w);
            oy += Word64::oy(w);
            x = p;
            return true;
        }
        if (gp >= n_sites) {
            bad = true;
            return true;
        }
        const int nx = Word64::ox(w) + Word64::ox(wp), ny = Word64::oy(w) + Word64::oy(wp);
        st(x, Word64::make(gp, nx, ny));
        ox += nx;
        oy += ny;
        x = gp;
        return false;
    }

    // Union across a boundary bond a -> b with seam crossing (ex, ey).  Both
    // endpoint walks advance in the same iteration (their loads overlap);
    // once both are at roots the larger root is hooked under the smaller with
    // a CAS that re-checks it is still a root, and a lost race resumes the
    // walks from where they stand.
    __device__ __forceinline__ void unite(uint32_t a, uint32_t b, int ex, int ey) const
    {
        if (a >= n_sites || b >= n_sites) {
            atomicOr(err, kErrFindCap);
            return;
        }
        int axa = 0, aya = 0, axb = 0, ayb = 0;
        bool da = false, db = false, bad = false;
        for (uint32_t it = 0; it < cap; ++it) {
            if (!da) da = hstep(a, axa, aya, bad);
            if (!db) db = hstep(b, axb, ayb, bad);
            if (bad) {
                atomicOr(err, kErrFindCap);
                return;
            }
            if (!(da && db)) continue;
            if (a == b) {
                int f = 0;
                if (Word64::nonzero(ex + axb - axa)) f |= 1;
                if (Word64::nonzero(ey + ayb - aya)) f |= 2;
                if (f) atomicOr(wrap, f);
                return;
            }
            if (a < b) {
                const unsigned long long expect = Word64::make(b, 0, 0);
                if (atomicCAS(G + b, expect, Word64::make(a, axa - ex - axb, aya - ey - ayb)) == expect) return;
            } else {
                const unsigned long long expect = Word64::make(a, 0, 0);
                if (atomicCAS(G + a, expect, Word64::make(b, axb + ex - axa, ayb + ey - aya)) == expect) return;
            }
            da = db = false;
        }
        atomicOr(err, kErrUnionCap);
    }
};


// Shared scratch of one CTA.
struct GRed {
    unsigned long long k1[32], k2[32];
    uint32_t unsat[32], downs[32], ncl[32];
    int mcw[32], mcw2[32];
    uint32_t g1, g2, ncl_total, nnodes, front, tile_end, hot_r, hot_s;
    int wrap, err, pend_many;
    uint64_t pend_sweep;
    bool pend;
    long long rec[kRecLen];
    rbim_chain_t ch;
};

// Views of this CTA's shared memory.
struct GTile {
    Lat<Word16> t;
    uint32_t *NODE;  // tile roots that are nodes of the global union-find
    uint32_t *YS;    // occupied y-seam bonds of the rows ending in the tile
    uint32_t *NK;    // node list: tile roots (local sites)
    uint32_t *NR;    // node list: their root nodes (global sites)
    unsigned long long *BH;  // boundary-bond hash (ly.bh entries, none when 0)
};

__device__ __forceinline__ GTile make_gtile(unsigned char *smem, const GridLayout &ly, const Tile &tl, GRed &red,
                                            uint32_t cap)
{
    GTile x;
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
    t.cap = cap;
    x.NODE = (uint32_t *)(smem + ly.off_NODE);
    x.YS = (uint32_t *)(smem + ly.off_YS);
    x.NK = (uint32_t *)(smem + ly.off_NK);
    x.NR = (uint32_t *)(smem + ly.off_NR);
    x.BH = (unsigned long long *)(smem + ly.off_BH);
    return x;
}

// Spin halo after a flip, from the global spin plane: the first L spins of
// the next tile (of the first tile, for the last one) at bits Tc .. Tc+L-1,
// and the front spin (the row start of the tile's first row, when that row
// began in the previous tile).  Tiles start on word boundaries.
template <int NT>
__device__ __forceinline__ void grid_halo(const GTile &x, const Tile &tl, const uint32_t *spins, GRed &red,
                                          uint32_t tid)
{
    uint32_t *S = x.t.S;
    const uint32_t nb = tl.c + 1u == tl.C ? 0u : tl.b + tl.Tc;
    const uint32_t *rs = spins + (nb >> 5);
    const uint32_t lw = (tl.L + 31u) >> 5;
    const uint32_t sh = tl.Tc & 31u, d0 = tl.Tc >> 5;
    const uint32_t lmask = (tl.L & 31u) ? (1u << (tl.L & 31u)) - 1u : 0xFFFFFFFFu;
    for (uint32_t k = tid; k <= lw; k += NT) {
        const uint32_t hk = k < lw ? (__ldcg(rs + k) & (k + 1u == lw ? lmask : 0xFFFFFFFFu)) : 0u;
        uint32_t v;
        if (sh == 0u) {
            v = hk;
        } else {
            const uint32_t hp = k > 0u ? (__ldcg(rs + k - 1u) & (k == lw ? lmask : 0xFFFFFFFFu)) : 0u;
            v = (hk << sh) | (k > 0u ? hp >> (32u - sh) : 0u);
            if (k == 0u) v |= S[d0] & ((1u << sh) - 1u);
        }
        S[d0 + k] = v;
    }
    if (tid == 0) {
        uint32_t front = 0;
        if (tl.f) {
            const uint32_t q = tl.x0 * tl.L;
            front = (__ldcg(spins + (q >> 5)) >> (q & 31u)) & 1u;
        }
        red.front = front;
    }
}

// Nodes of this tile: the tile roots of every site a boundary bond can touch
// (the first and last L sites, the row starts and row ends in the tile, the
// last site, and the row start of the next tile's first row when that row
// begins here).  Each is listed once (NODE bits), its node word is reset to
// a root, the roots of the first L sites are published for the previous
// tile's x-bonds (FR) and the next tile's front root for its y-seam bond
// (FRONT).  Before the first grid barrier of the sweep.
template <int NT>
__device__ __forceinline__ void grid_nodes(const GTile &x, const Tile &tl, const GridWs &ws, GRed &red,
                                           uint32_t tid)
{
    const Lat<Word16> &t = x.t;
    const uint32_t L = tl.L, Tc = tl.Tc;
    const uint32_t rows = (tl.b + Tc - 1u) / L - tl.x0 + 1u;  // rows with a site in the tile
    const uint32_t items = 2u * L + 2u * rows + 2u;
    for (uint32_t i = tid; i < items; i += NT) {
        uint32_t s;
        if (i < L) {
            s = i;
        } else if (i < 2u * L) {
            s = Tc - L + (i - L);
        } else if (i < 2u * L + rows) {
            const uint32_t start = (tl.x0 + (i - 2u * L)) * L;
            if (start < tl.b) continue;
            s = start - tl.b;
        } else if (i < 2u * L + 2u * rows) {
            const uint32_t end = (tl.x0 + (i - 2u * L - rows)) * L + L - 1u;
            if (end >= tl.b + Tc) continue;
            s = end - tl.b;
        } else if (i == 2u * L + 2u * rows) {
            s = Tc - 1u;
        } else {
            if (tl.c + 1u == tl.C) continue;
            const uint32_t bn = tl.b + tl.T, q = (bn / L) * L;
            if (q == bn) continue;
            s = q - tl.b;
        }
        const uint32_t r = tile_root(t.uf.w, s);
        if (i < L) ws.FR[tl.c * L + i] = tl.b + r;
        if (i == items - 1u) ws.FRONT[tl.c + 1u] = tl.b + r;
        const uint32_t bit = 1u << (r & 31u);
        if (!(atomicOr(x.NODE + (r >> 5), bit) & bit)) {
            const uint32_t k = atomicAdd(&red.nnodes, 1u);
            x.NK[k] = r;
            __stcg(ws.G + tl.b + r, Word64::make(tl.b + r, 0, 0));
        }
    }
}

// Boundary bonds owned by this tile -- the x-bonds of its last L sites, the
// y-bond from its last site into the next tile, the y-seam bonds of the rows
// ending in it -- unioned between their endpoints' nodes (after the first
// grid barrier of the sweep).  Lane i of a warp takes item i0 + i, so the
// x-bonds along the last row sit in consecutive lanes: a bond that joins the
// same two nodes with the same seam crossing as the previous lane's closes a
// loop of winding zero (the paths inside tiles do not wrap) and is skipped,
// and so is any later such bond of the tile (the boundary-bond hash).
// First insertion of `key` into the boundary-bond hash (open addressing,
// mask + 1 slots, never full: it holds at least 1.5 keys per bond).
__device__ __forceinline__ bool bh_insert(unsigned long long *H, uint32_t mask, unsigned long long key)
{
    uint32_t h = (uint32_t)((key * 0x9E3779B97F4A7C15ull) >> 40) & mask;
    for (uint32_t i = 0; i <= mask; ++i) {
        const unsigned long long old = atomicCAS(H + h, ~0ull, key);
        if (old == ~0ull) return true;
        if (old == key) return false;
        h = (h + 1u) & mask;
    }
    return true;
}

template <int NT>
__device__ __forceinline__ void grid_boundary(const GTile &x, const Tile &tl, const GridWs &ws, const GDist &d,
                                              uint32_t tile_end, uint32_t bh, uint32_t tid)
{
    const Lat<Word16> &t = x.t;
    const uint32_t rows_end = (tl.b + tl.Tc) / tl.L;  // rows x0 .. rows_end-1 end in the tile
    const uint32_t items = tl.L + 1u + (rows_end - tl.x0);
    const uint32_t nxt = tl.c + 1u == tl.C ? 0u : tl.c + 1u;
    const uint32_t lane = tid & 31u;
    for (uint32_t i0 = tid & ~31u; i0 < items; i0 += NT) {
        const uint32_t i = i0 + lane;
        bool live = false;
        uint32_t ra = 0, rb = 0;
        int ex = 0, ey = 0;
        if (i < tl.L) {
            const uint32_t a = tl.Tc - tl.L + i;
            if ((t.OH[a >> 5] >> (a & 31u)) & 1u) {
                live = true;
                ra = tl.b + tile_root(t.uf.w, a);
                const uint32_t n = tl.b + a;
                if (n + tl.L >= tl.N) {
                    rb = __ldcg(ws.FR + (n + tl.L - tl.N));  // tile 0, across the x seam
                    ex = 1;
                } else {
                    rb = __ldcg(ws.FR + nxt * tl.L + (a + tl.L - tl.Tc));
                }
            }
        } else if (i == tl.L) {
            if (tile_end) {
                live = true;
                ra = tl.b + tile_root(t.uf.w, tl.Tc - 1u);
                rb = __ldcg(ws.FR + nxt * tl.L);
            }
        } else if (i < items) {
            const uint32_t row = i - tl.L - 1u;
            if ((x.YS[row >> 5] >> (row & 31u)) & 1u) {
                live = true;
                const uint32_t xr = tl.x0 + row;
                ra = tl.b + tile_root(t.uf.w, xr * tl.L + tl.L - 1u - tl.b);
                const uint32_t start = xr * tl.L;
                rb = start >= tl.b ? tl.b + tile_root(t.uf.w, start - tl.b) : __ldcg(ws.FRONT + tl.c);
                ey = 1;
            }
        }
        const int tag = live ? 1 + ex + 2 * ey : 0;
        const uint32_t pra = __shfl_up_sync(0xFFFFFFFFu, ra, 1), prb = __shfl_up_sync(0xFFFFFFFFu, rb, 1);
        const int ptag = __shfl_up_sync(0xFFFFFFFFu, tag, 1);
        if (live && lane > 0u && ptag == tag && pra == ra && prb == rb) live = false;
        // Any earlier bond of the tile between the same two nodes with the
        // same seam crossing makes this one redundant in the same way.
        if (live && bh)
            live = bh_insert(x.BH, bh - 1u,
                             ((unsigned long long)(ra - tl.b) << 34) | ((unsigned long long)rb << 2) |
                                 (unsigned long long)(ex + 2 * ey));
        if (live) d.unite(ra, rb, ex, ey);
    }
}


// The open-tile union and root walks as separate (non-inlined) functions, as
// in the cluster engine: inline, these pointer-chasing loops lose registers
// to the state the kernel keeps live across its phases.
template <int NT>
static __device__ __noinline__ void grid_union(const Lat<Word16> &t, uint32_t tid)
{
    phase_union_open(t, tid, NT);
}

template <int NT>
static __device__ __noinline__ void grid_roots(const Lat<Word16> &t, uint32_t tid)
{
    (void)phase_roots_flat(t, tid, NT);
}

struct GridArgs {
    rbim_chain_t *chain;
    uint32_t *spin_pool;
    const uint32_t *coupling_pool;
    long long *acc_i;
    double *acc_f;
    int32_t *records;
    int n_sweeps;
    int64_t L;
    int *status;
    GridWs ws;
    GridLayout ly;
    long long wait_cycles;
};

// Bin sums of a chain, read past L1 (the previous sweep's record may have
// been added by another SM).
__device__ __forceinline__ void acc_load_cg(Acc &a, const long long *gi, const double *gf)
{
#pragma unroll
    for (int k = 0; k < kAccInt; ++k) a.i[k] = __ldcg(gi + k);
    a.f[0] = __ldcg(gf);
    a.f[1] = __ldcg(gf + 1);
}

// The record and bin sums of measured sweep `sw` (warp 0 of CTA 0, after
// every CTA has finished the sweep): energy, magnetization and wraps from
// the CTAs' partials, |M_C1| and |M_C2| from the sums the CTAs added for
// the sweep's parity (reset here for the sweep after next), the cluster
// count and the two largest sizes from this CTA's own combination.
__device__ __forceinline__ void grid_record(const GridArgs &a, const rbim_chain_t &ch, GRed &red, uint32_t C,
                                            uint32_t N, uint32_t lane)
{
    const GridWs &ws = a.ws;
    const uint64_t sw = red.pend_sweep;
    long long su = 0, sd = 0;
    int wr = 0;
    for (uint32_t i = lane; i < C; i += 32u) {
        su += __ldcg(&ws.part[i].unsat);
        sd += __ldcg(&ws.part[i].downs);
        wr |= __ldcg(&ws.part[i].wrap);
    }
    for (int o = 16; o > 0; o >>= 1) {
        su += __shfl_xor_sync(0xFFFFFFFFu, su, o);
        sd += __shfl_xor_sync(0xFFFFFFFFu, sd, o);
        wr |= __shfl_xor_sync(0xFFFFFFFFu, wr, o);
    }
    if (lane != 0) return;
    int *mcs = ws.sync->mc[sw & 1u];
    const long long m1 = __ldcg(mcs), m2 = __ldcg(mcs + 1);
    mcs[0] = 0;
    mcs[1] = 0;
    long long *rec = red.rec;
    rec[0] = 2ll * su - 2ll * (long long)N;
    rec[1] = (long long)N - 2ll * sd;
    rec[2] = red.ncl_total;
    const long long mc_total = red.pend_many ? m1 : rec[1], mc2_total = red.pend_many ? m2 : 0;
    rec[4] = mc_total < 0 ? -mc_total : mc_total;
    rec[6] = mc2_total < 0 ? -mc2_total : mc2_total;
    rec[7] = wr & 1;
    rec[8] = (wr >> 1) & 1;
    const long long idx = (long long)(sw - (uint64_t)ch.n_therm);
    const long long bin = idx / ch.sweeps_per_bin;
    long long *gi = a.acc_i + (ch.acc_off + bin) * kAccInt;
    double *gf = a.acc_f + (ch.acc_off + bin) * kAccF64;
    Acc acc;
    acc_load_cg(acc, gi, gf);
    acc.add(rec[0], rec[1], rec[2], rec[3], rec[4], rec[5], (int)rec[7], (int)rec[8]);
    acc.store(gi, gf);
    if (a.records && ch.rec_off >= 0) {
        int32_t *row = a.records + (ch.rec_off + idx) * kRecLen;
#pragma unroll
        for (int k = 0; k < kRecLen; ++k) row[k] = (int32_t)rec[k];
    }
    red.pend = false;
}

// One chain, every sweep of the call.  NT threads per CTA, one tile per CTA.
template <int NT>
__global__ void __launch_bounds__(NT, NT >= 1024 ? 1 : 1024 / NT) k_grid_sweeps(GridArgs a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ GRed red;
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    constexpr uint32_t nwarps = NT / 32;
    const uint32_t C = gridDim.x, c = blockIdx.x;
    const GridLayout &ly = a.ly;
    const GridWs &ws = a.ws;

    if (tid == 0) {
        red.err = 0;
        red.pend = false;
        red.ch = *a.chain;
    }
    __syncthreads();
    const rbim_chain_t &ch = red.ch;
    const bool bad = ch.L != a.L || ch.L <= 32 || ch.L != (int64_t)ly.L || ch.sweeps_per_bin < 1 || ch.n_bins < 0 ||
                     ch.n_therm < 0 || ch.walk_cap < 0 || C != ly.C || !cluster_tiles_ok((uint32_t)ch.L, C, kGridTileMax);
    if (bad) {
        if (tid == 0 && c == 0) atomicOr(a.status, kErrBadChain);
        return;
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
    const uint32_t cap =
        ch.walk_cap > 0 ? (uint32_t)min((long long)ch.walk_cap, (long long)tl.Tc + 64ll) : tl.Tc + 64u;
    const GTile x = make_gtile(smem, ly, tl, red, cap);
    const Lat<Word16> &t = x.t;
    const uint32_t gcap =
        ch.walk_cap > 0 ? (uint32_t)min((long long)ch.walk_cap, (long long)tl.N) : tl.N + 64u;
    const GDist d{ws.G, &red.wrap, &red.err, gcap, tl.N};
    uint32_t *spins = a.spin_pool + ch.spin_off;
    uint32_t *gS = spins + (tl.b >> 5);
    const uint32_t *gJH = a.coupling_pool + ch.coupling_off + (tl.b >> 5);
    const uint32_t *gJV = a.coupling_pool + ch.coupling_off + tl.nwp + (tl.b >> 5);
    const uint32_t s_words = ly.tw + (tl.L + 31u) / 32u + 4u;
    unsigned short *u16 = t.uf.w;

    // The tile's spins and the halo (nothing writes the spin plane before
    // the second barrier of the first sweep).
    for (uint32_t w = tid; w < s_words; w += NT) t.S[w] = w < tl.tw ? __ldcg(gS + w) & t.g.valid(w) : 0u;
    __syncthreads();
    grid_halo<NT>(x, tl, spins, red, tid);
    __syncthreads();

    const uint64_t t_end = (uint64_t)ch.n_therm + (uint64_t)ch.n_bins * (uint64_t)ch.sweeps_per_bin;
    uint64_t sweep = ch.sweep;
    const uint64_t stop = min(t_end, sweep + (uint64_t)max(a.n_sweeps, 0));
    const bool second = a.records && ch.rec_off >= 0;
    RBIM_GRID_PROF_START;
    for (; sweep < stop; ++sweep) {
        const bool measure = sweep >= (uint64_t)ch.n_therm;
        const uint32_t front = red.front;
        if (tid == 0) {
            red.wrap = 0;
            red.tile_end = 0;
            red.nnodes = 0;
        }
        for (uint32_t i = tid; i < ly.rows_max / 32u + 1u; i += NT) x.YS[i] = 0u;
        for (uint32_t w = tid; w < t.g.NW; w += NT) x.NODE[w] = 0u;
        for (uint32_t i = tid; i < ly.bh; i += NT) x.BH[i] = ~0ull;
        __syncthreads();
        tile_activate<NT>(t, x.YS, tl, make_rng(ch.key, sweep, ch.thr), gJH, gJV, front, red.tile_end, warp, nwarps,
                          tid);
        __syncthreads();
        RBIM_GRID_MARK(0);
        for (uint32_t w = tid; w < t.g.NW; w += NT) ws.FLIPG[(tl.b >> 5) + w] = t.FLIP[w];
        phase_heads<Word16>(t, warp, nwarps);
        for (uint32_t w = tid; w < t.g.NW; w += NT) t.ROOT[w] = 0u;
        __syncthreads();
        RBIM_GRID_MARK(1);
        grid_union<NT>(t, tid);
        __syncthreads();
        RBIM_GRID_MARK(2);
        grid_roots<NT>(t, tid);
        __syncthreads();
        RBIM_GRID_MARK(3);
        grid_nodes<NT>(x, tl, ws, red, tid);
        RBIM_GRID_MARK(4);
        grid_sync(ws.sync, C, a.wait_cycles, &red.err);  // nodes, FR, FRONT and FLIPG are published
        RBIM_GRID_MARK(5);
        // Every CTA has finished the previous sweep: its record, off the
        // critical path of that sweep.
        if (c == 0 && warp == 0 && red.pend) grid_record(a, ch, red, C, tl.N, lane);

        grid_boundary<NT>(x, tl, ws, d, red.tile_end, ly.bh, tid);
        RBIM_GRID_MARK(6);
        grid_sync(ws.sync, C, a.wait_cycles, &red.err);  // every boundary union is done
        RBIM_GRID_MARK(7);

        // Root node of each node; a merged tile root takes the raw flip bit
        // of its cluster's root site.
        const uint32_t nnodes = red.nnodes;
        for (uint32_t k = tid; k < nnodes; k += NT) {
            const uint32_t m = x.NK[k];
            const uint32_t r = d.root_ro(tl.b + m);
            x.NR[k] = r;
            if (r != tl.b + m) {
                if ((__ldcg(ws.FLIPG + (r >> 5)) >> (r & 31u)) & 1u)
                    atomicOr(t.FLIP + (m >> 5), 1u << (m & 31u));
                else
                    atomicAnd(t.FLIP + (m >> 5), ~(1u << (m & 31u)));
            }
        }
        __syncthreads();
        // Flip by the tile root's FLIP bit: run piece by run piece (a
        // measured sweep also leaves every piece leader's word holding its
        // tile root), or, in tiles with fewer than a quarter as many words as
        // threads, site by site (every site's word then holds its tile root).
        RBIM_GRID_MARK(8);
        const bool per_site = 4u * t.g.NW <= NT;
        if (!per_site)
            flip_pieces(t, tid, NT, measure);
        else
            phase_sites<Word16>(t, warp, nwarps, true, false);
        __syncthreads();
        RBIM_GRID_MARK(9);
        for (uint32_t w = tid; w < tl.tw; w += NT) gS[w] = t.S[w] & t.g.valid(w);
        // Measured sweeps: cluster sizes before the barrier that publishes the
        // spins, so that one barrier also completes the merged sizes.
        uint32_t nloc = 0;
        if (measure) {
            // Tile cluster sizes minus one added onto each tile root's own index
            // (a root points at itself): afterwards the word of root m reads
            // m + size - 1, below 65536 because m is the smallest site of its tile
            // cluster, so no add carries out of its 16 bits (tile_size decodes it).
            count_pieces<true>(t, u16, warp, nwarps);
            __syncthreads();
            RBIM_GRID_MARK(12);
            // Node sizes into the root nodes' words (the high half of a root's
            // word is zero), summed per root in each warp first and, for the root
            // of the CTA's first node (most often the cluster that spans the
            // lattice), over the whole CTA, so that a spanning cluster's root
            // takes one add per CTA.  Clusters: tile-only roots and root nodes.
            if (tid == 0) {
                red.hot_r = nnodes ? x.NR[0] : 0xFFFFFFFFu;
                red.hot_s = 0u;
            }
            __syncthreads();
            const uint32_t hot = red.hot_r;
            for (uint32_t k0 = warp << 5; k0 < nnodes; k0 += NT) {
                const uint32_t k = k0 + lane;
                uint32_t r = 0xFFFFFFFFu, v = 0u;
                if (k < nnodes) {
                    const uint32_t m = x.NK[k];
                    r = x.NR[k];
                    v = tile_size(u16, m);
                    if (r == tl.b + m) ++nloc;
                }
                const uint32_t grp = __match_any_sync(0xFFFFFFFFu, r);
                const uint32_t sum = __reduce_add_sync(grp, v);
                if (r != 0xFFFFFFFFu && lane == (uint32_t)(__ffs(grp) - 1)) {
                    if (r == hot)
                        atomicAdd(&red.hot_s, sum);
                    else
                        atomicAdd((unsigned int *)(ws.G + r) + 1, sum);
                }
            }
            for (uint32_t w = tid; w < t.g.NW; w += NT) nloc += __popc(t.ROOT[w] & ~x.NODE[w]);
            __syncthreads();
            if (tid == 0 && hot != 0xFFFFFFFFu) atomicAdd((unsigned int *)(ws.G + hot) + 1, red.hot_s);
        }
        // Every tile's spins are written (and, when measured, every merged size).
        grid_sync(ws.sync, C, a.wait_cycles, &red.err);
        RBIM_GRID_MARK(10);
        grid_halo<NT>(x, tl, spins, red, tid);
        __syncthreads();
        RBIM_GRID_MARK(11);

        if (!measure) continue;

        // ---- measurement (reference sw_sweep, src/rbim/swendsen_wang.py:146-172)
        uint32_t unsat = 0, downs = 0;
        tile_energy<NT>(t, tl, gJH, gJV, red.front, tid, unsat, downs);
        RBIM_GRID_MARK(13);

        // Local top two: tile-only clusters and the root nodes in this tile.
        unsigned long long k1 = 0, k2 = 0;
        for (uint32_t w = tid; w < t.g.NW; w += NT) {
            uint32_t roots = t.ROOT[w] & ~x.NODE[w];
            while (roots) {
                const uint32_t bb = __ffs(roots) - 1u;
                roots &= roots - 1u;
                const uint32_t m = (w << 5) + bb;
                top2_merge(k1, k2, size_key(tile_size(u16, m), tl.b + m), 0ull);
            }
        }
        for (uint32_t k = tid; k < nnodes; k += NT) {
            const uint32_t m = x.NK[k], r = x.NR[k];
            if (r != tl.b + m) continue;
            top2_merge(k1, k2, size_key((uint32_t)(__ldcg(ws.G + r) >> 32), r), 0ull);
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
                GridPartial *pp = ws.part + c;
                __stcg(&pp->k1, a1);
                __stcg(&pp->k2, a2);
                __stcg(&pp->unsat, su);
                __stcg(&pp->downs, sd);
                __stcg(&pp->ncl, sn);
                __stcg(&pp->wrap, red.wrap);
            }
        }
        grid_sync(ws.sync, C, a.wait_cycles, &red.err);  // partials are visible
        RBIM_GRID_MARK(14);

        // Every CTA combines the partials: the two largest clusters and the
        // number of clusters.
        if (warp == 0) {
            unsigned long long a1 = 0, a2 = 0;
            uint32_t sn = 0;
            for (uint32_t i = lane; i < C; i += 32u) {
                top2_merge(a1, a2, __ldcg(&ws.part[i].k1), __ldcg(&ws.part[i].k2));
                sn += __ldcg(&ws.part[i].ncl);
            }
            warp_top2(a1, a2);
            for (int o = 16; o > 0; o >>= 1) sn += __shfl_xor_sync(0xFFFFFFFFu, sn, o);
            if (lane == 0) {
                red.g1 = 0xFFFFFFFFu - (uint32_t)(a1 & 0xFFFFFFFFull);
                red.g2 = 0xFFFFFFFFu - (uint32_t)(a2 & 0xFFFFFFFFull);
                red.ncl_total = sn;
                red.rec[3] = (long long)(a1 >> 32);
                red.rec[5] = (long long)(a2 >> 32);
            }
        }
        __syncthreads();
        const uint32_t g1 = red.g1, g2 = red.g2;
        const bool many = red.ncl_total > 1u;
        int mc = 0, mc2 = 0;
        if (many) {
            // Tile roots of the largest cluster marked in OH, and with
            // `second` those of the second largest in FLIP (both free after
            // the flip).
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
            for (uint32_t k = tid; k < nnodes; k += NT) {
                const uint32_t m = x.NK[k], r = x.NR[k];
                if (r == g1)
                    atomicOr(t.OH + (m >> 5), 1u << (m & 31u));
                else if (second && r == g2)
                    atomicOr(t.FLIP + (m >> 5), 1u << (m & 31u));
            }
            __syncthreads();
            // One lane per word, one test per run piece: a piece leader's
            // word holds its tile root; site by site (one warp per word)
            // where the flip went site by site.
            if (per_site) {
                for (uint32_t w = warp; w < t.g.NW; w += nwarps) {
                    const uint32_t n = (w << 5) + lane;
                    if (n >= tl.Tc) continue;
                    const uint32_t r = ((t.ROOT[w] >> lane) & 1u) ? n : (uint32_t)u16[n];
                    const int m = 1 - 2 * (int)((t.S[w] >> lane) & 1u);
                    if ((t.OH[r >> 5] >> (r & 31u)) & 1u) mc += m;
                    if (second && ((t.FLIP[r >> 5] >> (r & 31u)) & 1u)) mc2 += m;
                }
            }
            for (uint32_t w = tid; w < t.g.NW && !per_site; w += NT) {
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
            int s1 = 0, s2 = 0;
            for (uint32_t i = 0; i < nwarps; ++i) {
                s1 += red.mcw[i];
                s2 += red.mcw2[i];
            }
            if (many) {
                atomicAdd(&ws.sync->mc[sweep & 1u][0], s1);
                if (second) atomicAdd(&ws.sync->mc[sweep & 1u][1], s2);
            }
            if (c == 0) {
                red.pend = true;
                red.pend_sweep = sweep;
                red.pend_many = many ? 1 : 0;
            }
        }
        __syncthreads();
        RBIM_GRID_MARK(15);
    }
    // The record of the call's last sweep, after every CTA has finished it
    // (the same condition on every CTA: the last sweep was measured).
    if (stop > ch.sweep && stop - 1u >= (uint64_t)ch.n_therm) {
        grid_sync(ws.sync, C, a.wait_cycles, &red.err);
        if (c == 0 && warp == 0 && red.pend) grid_record(a, ch, red, C, tl.N, lane);
    }
    if (c == 0 && tid == 0) a.chain->sweep = stop;
    if (tid == 0 && red.err) atomicOr(a.status, red.err);
}

int device_sm_count()
{
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    return sms;
}

template <int NT>
cudaError_t grid_occupancy_t(size_t smem, bool query, int *per_sm)
{
    // The kernel's dynamic shared-memory limit, raised to what any plan may
    // use, on every launch (a device reset forgets it).
    const cudaError_t e = cudaFuncSetAttribute(k_grid_sweeps<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)(227u * 1024u - kGridStaticSmem));
    if (e != cudaSuccess || !query) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, k_grid_sweeps<NT>, NT, smem);
}

// CTAs of `threads` threads and `smem` dynamic bytes that one SM holds; the
// query is cached per (device, threads, smem), so that a call of one sweep
// does not pay for it again.
cudaError_t grid_occupancy(uint32_t threads, size_t smem, int *per_sm)
{
    static std::mutex mu;
    static std::vector<std::pair<std::pair<int, uint64_t>, int>> cache;  // (device, threads << 32 | smem) -> CTAs
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const uint64_t key = ((uint64_t)threads << 32) | (uint64_t)smem;
    std::lock_guard<std::mutex> lock(mu);
    bool query = true;
    for (const auto &c : cache)
        if (c.first.first == dev && c.first.second == key) {
            *per_sm = c.second;
            query = false;
        }
    switch (threads) {
    case 256: e = grid_occupancy_t<256>(smem, query, per_sm); break;
    case 512: e = grid_occupancy_t<512>(smem, query, per_sm); break;
    case 1024: e = grid_occupancy_t<1024>(smem, query, per_sm); break;
    default: return cudaErrorInvalidValue;
    }
    if (e == cudaSuccess && query) cache.push_back({{dev, key}, *per_sm});
    return e;
}

template <int NT>
cudaError_t grid_launch_t(const GridArgs &a, uint32_t C, size_t smem, cudaStream_t stream)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(C, 1, 1);
    cfg.blockDim = dim3(NT, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_grid_sweeps<NT>, a);
}

}  // namespace

// The layout a plan runs with: with the boundary-bond hash when it fits in
// shared memory, else without (false: the plan cannot run an L x L lattice).
static bool grid_fit(uint32_t L, GridPlan p, GridLayout *out)
{
    if (L <= 32u || p.C < 2u || (p.threads != 256u && p.threads != 512u && p.threads != 1024u)) return false;
    if ((uint64_t)L * L >= (1ull << 31)) return false;
    if (!cluster_tiles_ok(L, p.C, kGridTileMax)) return false;
    const uint32_t per_sm = 1024u / p.threads;  // register budget: 64 per thread
    for (const bool hash : {true, false}) {
        const GridLayout ly = grid_layout(L, p.C, hash);
        if (per_sm * (ly.bytes + kGridStaticSmem) <= kGridSmemPerSm && ly.bytes <= 227u * 1024u - kGridStaticSmem) {
            if (out) *out = ly;
            return true;
        }
    }
    return false;
}

bool grid_plan_ok(uint32_t L, GridPlan p) { return grid_fit(L, p, nullptr); }

GridPlan grid_plan(uint32_t L)
{
    // 1024-thread CTAs, one tile of about 1024 sites each (smaller tiles add
    // boundary unions, larger ones add walk latency inside the tile), at most
    // one per SM; then the largest tile count at or below that whose tiles all
    // hold at least L sites.  Measured on B200, one lattice, us per sweep:
    // L = 64: 29 with 4-8 tiles, 33 with 32; L = 128: 33 with 16 tiles, 37
    // with 128; L = 256: 37 with 64 tiles; L = 1024: 60-61 with 128-147.
    const int sms = device_sm_count();
    if (sms <= 0) return {0u, 0u};
    const uint64_t want = ((uint64_t)L * L + 1023u) / 1024u;
    uint32_t C = (uint32_t)std::min<uint64_t>((uint64_t)std::max(sms, 2), std::max<uint64_t>(want, 2u));
    for (; C >= 2u; --C)
        if (grid_plan_ok(L, {C, 1024u})) return {C, 1024u};
    return {0u, 0u};
}

size_t grid_workspace_bytes(uint32_t L, uint32_t C) { return grid_ws_bytes(L, C); }

cudaError_t launch_grid_sweeps(rbim_chain_t *chain, int64_t L, GridPlan plan, uint32_t *spin_pool,
                               const uint32_t *coupling_pool, long long *acc_i, double *acc_f, int32_t *records,
                               int n_sweeps, int *status, void *workspace, long long wait_cycles, cudaStream_t stream)
{
    GridArgs a;
    if (!grid_fit((uint32_t)L, plan, &a.ly)) return cudaErrorInvalidValue;
    a.chain = chain;
    a.spin_pool = spin_pool;
    a.coupling_pool = coupling_pool;
    a.acc_i = acc_i;
    a.acc_f = acc_f;
    a.records = records;
    a.n_sweeps = n_sweeps;
    a.L = L;
    a.status = status;
    a.ws = grid_ws(workspace, (uint32_t)L, plan.C);
    a.wait_cycles = wait_cycles > 0 ? wait_cycles : kGridWaitCycles;
    int per_sm = 0;
    cudaError_t e = grid_occupancy(plan.threads, a.ly.bytes, &per_sm);
    if (e != cudaSuccess) return e;
    if ((int64_t)per_sm * device_sm_count() < (int64_t)plan.C) return cudaErrorCooperativeLaunchTooLarge;
    e = cudaMemsetAsync(a.ws.sync, 0, sizeof(GridSync), stream);
    if (e != cudaSuccess) return e;
    switch (plan.threads) {
    case 256: return grid_launch_t<256>(a, plan.C, a.ly.bytes, stream);
    case 512: return grid_launch_t<512>(a, plan.C, a.ly.bytes, stream);
    default: return grid_launch_t<1024>(a, plan.C, a.ly.bytes, stream);
    }
}

}  // namespace rbim

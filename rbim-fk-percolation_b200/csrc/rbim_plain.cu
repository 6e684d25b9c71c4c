// Plain engine: one lattice, any L >= 3, union-find words in global memory
// (L2-resident up to L ~ 2000), one launch per phase.  It is the drop-in for
// a single run_single_realization task (src/rbim/simulation.py:148-242) and
// the path for lattices too large to keep on chip.  Every kernel reads the
// chain descriptor from device memory, so a whole sequence of sweeps can be
// enqueued (or captured in a CUDA graph) without host round trips; kernels of
// a chain that has finished its run return immediately.
#include <algorithm>
#include <mutex>

#include "rbim_internal.h"
#include "rbim_phases.cuh"

namespace rbim {

namespace {

constexpr int kPlainThreads = 256;

struct PlainScratch {
    int wrap;
    int err;
    unsigned int nroots;
    unsigned int pad0;
    unsigned long long unsat;
    unsigned long long downs;
    long long mc;
    long long mc2;
    unsigned long long g1;
    unsigned long long g2;
    unsigned long long s1;
    unsigned long long s2;
    unsigned int done1;  // CTAs of k_plain_measure1 finished this sweep
    unsigned int done3;  // CTAs of k_plain_measure3 finished this sweep
};

struct PlainWs {
    unsigned long long *uf;
    uint32_t *OH, *OV, *FLIP, *ROOT, *SEAMV;
    PlainScratch *sc;
    unsigned long long *top2;  // 2 per block of the measure kernel
};

size_t pad256(size_t v) { return (v + 255) & ~size_t(255); }

struct PlainSizes {
    size_t uf, plane, seam, sc, top2, total;
};

// Grid of the plain kernels on the current device: 4 CTAs per SM, cached per
// device (a process may drive devices with different SM counts).
int plain_grid()
{
    constexpr int kDevices = 64;
    static int grid[kDevices];
    static std::mutex mu;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kDevices) {
        cudaGetLastError();
        return 148 * 4;
    }
    std::lock_guard<std::mutex> lock(mu);
    if (!grid[dev]) {
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
            cudaGetLastError();
            return 148 * 4;
        }
        grid[dev] = std::max(1, sms) * 4;
    }
    return grid[dev];
}

constexpr int kMaxPlainGrid = 4096;
// One CTA of 256 threads per 256 sites, at most plain_grid() CTAs: a small
// lattice on 4 CTAs per SM pays mostly for scheduling CTAs that find no work,
// and for the last-CTA tickets of the measure kernels (on B200, one lattice:
// +20 % sweeps/s at L = 128 and 160, +8 % at L = 256; 1024 sites per CTA
// measured slower).
constexpr int64_t kPlainSitesPerCta = 256;

// Grid of the plain kernels for an L x L lattice on the current device.
int plain_grid_for(int64_t L)
{
    const int64_t by_size = (L * L + kPlainSitesPerCta - 1) / kPlainSitesPerCta;
    return (int)std::max<int64_t>(1, std::min<int64_t>(by_size, std::min(plain_grid(), kMaxPlainGrid)));
}

PlainSizes plain_sizes(int64_t L)
{
    PlainSizes s{};
    const size_t n = (size_t)L * (size_t)L;
    const size_t nw = ((n + 31) / 32 + 3) & ~size_t(3);
    s.uf = pad256(8 * n);
    s.plane = pad256(4 * (nw + 4));
    s.seam = pad256(4 * ((L + 31) / 32 + 4));
    s.sc = pad256(sizeof(PlainScratch));
    s.top2 = pad256(16 * kMaxPlainGrid);
    s.total = s.uf + 4 * s.plane + s.seam + s.sc + s.top2;
    return s;
}

PlainWs plain_ws(void *base, int64_t L)
{
    const PlainSizes s = plain_sizes(L);
    char *p = (char *)base;
    PlainWs w;
    w.uf = (unsigned long long *)p;
    p += s.uf;
    w.OH = (uint32_t *)p;
    p += s.plane;
    w.OV = (uint32_t *)p;
    p += s.plane;
    w.FLIP = (uint32_t *)p;
    p += s.plane;
    w.ROOT = (uint32_t *)p;
    p += s.plane;
    w.SEAMV = (uint32_t *)p;
    p += s.seam;
    w.sc = (PlainScratch *)p;
    p += s.sc;
    w.top2 = (unsigned long long *)p;
    return w;
}

struct PlainArgs {
    int64_t L;  // the size the workspace was sized for; the descriptor must agree
    rbim_chain_t *chain;
    uint32_t *spin_pool;
    const uint32_t *coupling_pool;
    long long *acc_i;
    double *acc_f;
    int32_t *records;
    int *status;
    PlainWs ws;
};

// A descriptor the plain kernels can run: the size the launch (and its
// workspace) was made for, and a well-formed run layout.
__device__ __forceinline__ bool chain_ok(const PlainArgs &a)
{
    const rbim_chain_t *c = a.chain;
    return c->L == a.L && c->sweeps_per_bin >= 1 && c->n_bins >= 0 && c->n_therm >= 0 && c->walk_cap >= 0;
}

// Phase of the chain's current sweep: 0 = finished (or a descriptor that
// fails chain_ok), 1 = thermalisation, 2 = measured.
__device__ __forceinline__ int chain_phase(const PlainArgs &a)
{
    if (!chain_ok(a)) return 0;
    const rbim_chain_t *c = a.chain;
    const uint64_t s = *((volatile const uint64_t *)&c->sweep);
    const uint64_t end = (uint64_t)c->n_therm + (uint64_t)c->n_bins * (uint64_t)c->sweeps_per_bin;
    if (s >= end) return 0;
    return s >= (uint64_t)c->n_therm ? 2 : 1;
}

__device__ __forceinline__ Lat<Word64> plain_lat(const PlainArgs &a)
{
    Lat<Word64> t;
    const uint32_t L = (uint32_t)a.chain->L;
    t.g = Geom{L, L * L, (L * L + 31u) / 32u};
    t.uf.w = a.ws.uf;
    t.S = a.spin_pool + a.chain->spin_off;
    t.JH = a.coupling_pool + a.chain->coupling_off;
    t.JV = t.JH + ((t.g.NW + 3u) & ~3u);
    t.OH = a.ws.OH;
    t.OV = a.ws.OV;
    t.FLIP = a.ws.FLIP;
    t.ROOT = a.ws.ROOT;
    t.SEAMV = a.ws.SEAMV;
    t.RE = nullptr;
    t.wrap = &a.ws.sc->wrap;
    t.err = &a.ws.sc->err;
    // A descriptor's walk_cap > 0 lowers the walk bound (a test hook).
    const int64_t wc = a.chain->walk_cap;
    t.cap = (wc > 0 && wc < (int64_t)(t.g.N + 64u)) ? (uint32_t)wc : t.g.N + 64u;
    return t;
}

__device__ __forceinline__ uint32_t gwarp() { return (blockIdx.x * blockDim.x + threadIdx.x) >> 5; }
__device__ __forceinline__ uint32_t gnwarps() { return (gridDim.x * blockDim.x) >> 5; }
__device__ __forceinline__ uint32_t gtid() { return blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ uint32_t gnthreads() { return gridDim.x * blockDim.x; }

__global__ void k_plain_begin(PlainArgs a)
{
    if (!chain_ok(a)) {
        // Every later kernel of the call returns at once for this descriptor.
        if (gtid() == 0) atomicOr(a.status, kErrBadChain);
        return;
    }
    const uint32_t L = (uint32_t)a.L;
    for (uint32_t i = gtid(); i < (L + 31u) / 32u; i += gnthreads()) a.ws.SEAMV[i] = 0u;
    if (gtid() == 0) {
        PlainScratch z{};
        *a.ws.sc = z;
    }
}

__global__ void __launch_bounds__(kPlainThreads, 4) k_plain_activate(PlainArgs a)
{
    if (!chain_phase(a)) return;
    const Lat<Word64> t = plain_lat(a);
    const SweepRng rng = make_rng(a.chain->key, a.chain->sweep, a.chain->thr);
    phase_activate<Word64>(t, rng, gwarp(), gnwarps(), gtid(), gnthreads());
}

// Run heads; also clears the ROOT plane for the root walks that follow.
__global__ void __launch_bounds__(kPlainThreads) k_plain_heads(PlainArgs a)
{
    if (!chain_phase(a)) return;
    const Lat<Word64> t = plain_lat(a);
    for (uint32_t w = gtid(); w < t.g.NW; w += gnthreads()) t.ROOT[w] = 0u;
    phase_heads<Word64>(t, gwarp(), gnwarps());
}

__global__ void __launch_bounds__(kPlainThreads) k_plain_union(PlainArgs a)
{
    if (!chain_phase(a)) return;
    phase_union<Word64>(plain_lat(a), gtid(), gnthreads());
}

__global__ void __launch_bounds__(kPlainThreads) k_plain_roots(PlainArgs a)
{
    if (!chain_phase(a)) return;
    const Lat<Word64> t = plain_lat(a);
    uint32_t nr = phase_roots<Word64>(t, gtid(), gnthreads());
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) nr += __shfl_xor_sync(0xFFFFFFFFu, nr, o);
    if ((threadIdx.x & 31u) == 0 && nr) atomicAdd(&a.ws.sc->nroots, nr);
}

__global__ void __launch_bounds__(kPlainThreads) k_plain_finalize(PlainArgs a)
{
    const int ph = chain_phase(a);
    if (!ph) return;
    const Lat<Word64> t = plain_lat(a);
    phase_sites<Word64>(t, gwarp(), gnwarps(), true, ph == 2);
    for (uint32_t i = gtid(); i < (t.g.L + 31u) / 32u; i += gnthreads()) t.SEAMV[i] = 0u;
}

__global__ void __launch_bounds__(kPlainThreads) k_plain_measure1(PlainArgs a)
{
    if (chain_phase(a) != 2) return;
    const Lat<Word64> t = plain_lat(a);
    uint32_t unsat = 0, downs = 0;
    measure_energy(t, gtid(), gnthreads(), unsat, downs);
    unsigned long long k1 = 0, k2 = 0;
    for (uint32_t w = gtid(); w < t.g.NW; w += gnthreads()) {
        uint32_t roots = t.ROOT[w];
        while (roots) {
            const uint32_t b = __ffs(roots) - 1u;
            roots &= roots - 1u;
            const uint32_t r = (w << 5) + b;
            const unsigned long long key =
                ((unsigned long long)Word64::count(t.uf.ldc(r)) << 32) | (0xFFFFFFFFull - r);
            top2_merge(k1, k2, key, 0ull);
        }
    }
    warp_top2(k1, k2);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        unsat += __shfl_xor_sync(0xFFFFFFFFu, unsat, o);
        downs += __shfl_xor_sync(0xFFFFFFFFu, downs, o);
    }
    __shared__ unsigned long long s1[kPlainThreads / 32], s2[kPlainThreads / 32];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    if (lane == 0) {
        s1[warp] = k1;
        s2[warp] = k2;
        if (unsat) atomicAdd(&a.ws.sc->unsat, (unsigned long long)unsat);
        if (downs) atomicAdd(&a.ws.sc->downs, (unsigned long long)downs);
    }
    __syncthreads();
    if (warp == 0) {
        unsigned long long b1 = lane < kPlainThreads / 32 ? s1[lane] : 0ull;
        unsigned long long b2 = lane < kPlainThreads / 32 ? s2[lane] : 0ull;
        warp_top2(b1, b2);
        if (lane == 0) {
            a.ws.top2[2 * blockIdx.x] = b1;
            a.ws.top2[2 * blockIdx.x + 1] = b2;
        }
    }
    // The last CTA to finish merges every CTA's top two, in place of a
    // separate single-CTA launch: each CTA publishes its pair, fences and
    // takes a ticket; the CTA with the last ticket reads all pairs from L2.
    __shared__ bool s_last;
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(&a.ws.sc->done1, 1u) == gridDim.x - 1u;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    k1 = 0;
    k2 = 0;
    for (uint32_t i = threadIdx.x; i < gridDim.x; i += blockDim.x)
        top2_merge(k1, k2, __ldcg(a.ws.top2 + 2 * i), __ldcg(a.ws.top2 + 2 * i + 1));
    warp_top2(k1, k2);
    if (lane == 0) {
        s1[warp] = k1;
        s2[warp] = k2;
    }
    __syncthreads();
    if (warp == 0) {
        unsigned long long b1 = lane < kPlainThreads / 32 ? s1[lane] : 0ull;
        unsigned long long b2 = lane < kPlainThreads / 32 ? s2[lane] : 0ull;
        warp_top2(b1, b2);
        if (lane == 0) {
            PlainScratch *sc = a.ws.sc;
            sc->g1 = 0xFFFFFFFFull - (b1 & 0xFFFFFFFFull);
            sc->g2 = 0xFFFFFFFFull - (b2 & 0xFFFFFFFFull);
            sc->s1 = b1 >> 32;
            sc->s2 = b2 >> 32;
        }
    }
}

// End of a sweep (one thread): the sweep's record and bin sums from the
// scratch, the status word, the sweep counter, and a zeroed scratch for the
// next sweep.  The scratch is read through L2 (volatile): other CTAs of the
// calling kernel added to it.
__device__ void plain_end(const PlainArgs &a, int ph)
{
    rbim_chain_t *c = a.chain;
    const volatile PlainScratch *sc = a.ws.sc;
    if (ph == 2) {
        const long long N = c->L * c->L;
        const long long M = N - 2ll * (long long)sc->downs;
        const long long ncl = sc->nroots;
        long long s1 = (long long)sc->s1, s2 = (long long)sc->s2, mc = sc->mc, mc2 = sc->mc2;
        if (ncl == 1) {
            s1 = N;
            s2 = 0;
            mc = M;
            mc2 = 0;
        }
        if (mc < 0) mc = -mc;
        if (mc2 < 0) mc2 = -mc2;
        const long long E = 2ll * (long long)sc->unsat - 2ll * N;
        const int wrap = sc->wrap;
        const int wx = wrap & 1, wy = (wrap >> 1) & 1;
        const long long idx = (long long)(c->sweep - (uint64_t)c->n_therm);
        const long long bin = idx / c->sweeps_per_bin;
        Acc acc;
        acc.zero();
        acc.add(E, M, ncl, s1, mc, s2, wx, wy);
        acc.flush(a.acc_i + (c->acc_off + bin) * kAccInt, a.acc_f + (c->acc_off + bin) * kAccF64);
        if (a.records && c->rec_off >= 0) {
            int32_t *row = a.records + (c->rec_off + idx) * kRecLen;
            row[0] = (int32_t)E;
            row[1] = (int32_t)M;
            row[2] = (int32_t)ncl;
            row[3] = (int32_t)s1;
            row[4] = (int32_t)mc;
            row[5] = (int32_t)s2;
            row[6] = (int32_t)mc2;
            row[7] = wx;
            row[8] = wy;
        }
    }
    const int err = sc->err;
    if (err) atomicOr(a.status, err);
    c->sweep = c->sweep + 1;
    PlainScratch z{};
    *a.ws.sc = z;
}

// Magnetisation of the largest cluster (measured sweeps with more than one
// cluster) and, when the chain's records are written, of the second largest;
// then, in the last CTA to finish, the end of the sweep: every CTA adds its
// share, fences and takes a ticket, so the last ticket sees all shares.
// Thermalisation sweeps run only the ticket and the end.
__global__ void __launch_bounds__(kPlainThreads) k_plain_measure3(PlainArgs a)
{
    const int ph = chain_phase(a);
    if (!ph) return;
    if (ph == 2 && a.ws.sc->nroots > 1) {
        const Lat<Word64> t = plain_lat(a);
        const uint32_t g1 = (uint32_t)a.ws.sc->g1, g2 = (uint32_t)a.ws.sc->g2;
        const bool second = a.records && a.chain->rec_off >= 0;
        const uint32_t lane = threadIdx.x & 31u;
        int mc = 0, mc2 = 0;
        for (uint32_t w = gwarp(); w < t.g.NW; w += gnwarps()) {
            const uint32_t n = (w << 5) + lane;
            const uint32_t r = n < t.g.N ? Word64::parent(t.uf.ldc(n)) : 0xFFFFFFFFu;
            const uint32_t m = __ballot_sync(0xFFFFFFFFu, r == g1);
            const uint32_t sw = t.S[w];
            if (lane == 0) mc += (int)__popc(m) - 2 * (int)__popc(m & sw);
            if (second) {
                const uint32_t m2 = __ballot_sync(0xFFFFFFFFu, r == g2);
                if (lane == 0) mc2 += (int)__popc(m2) - 2 * (int)__popc(m2 & sw);
            }
        }
        if (lane == 0 && mc) atomicAdd((unsigned long long *)&a.ws.sc->mc, (unsigned long long)(long long)mc);
        if (lane == 0 && mc2) atomicAdd((unsigned long long *)&a.ws.sc->mc2, (unsigned long long)(long long)mc2);
    }
    // Every thread fences its own adds before the CTA's ticket is taken.
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        if (atomicAdd(&a.ws.sc->done3, 1u) == gridDim.x - 1u) {
            __threadfence();
            plain_end(a, ph);
        }
    }
}

// Labelling of a frozen occupation mask (bond-order bytes) through the plain
// engine's phases, for lattices too large for the resident engine.
__global__ void __launch_bounds__(kPlainThreads) k_plain_label_load(PlainWs ws, uint32_t L, const uint8_t *occ)
{
    const Geom g{L, L * L, (L * L + 31u) / 32u};
    for (uint32_t w = gtid(); w < g.NW; w += gnthreads()) {
        uint32_t h = 0, v = 0;
        for (uint32_t b = 0; b < 32u; ++b) {
            const uint32_t n = (w << 5) + b;
            if (n >= g.N) break;
            h |= (occ[2ull * n] ? 1u : 0u) << b;
            v |= (occ[2ull * n + 1] ? 1u : 0u) << b;
        }
        const uint32_t re = g.row_end(w);
        ws.OH[w] = h;
        ws.OV[w] = v & ~re;
        uint32_t seam = v & re;
        while (seam) {
            const uint32_t b = __ffs(seam) - 1u;
            seam &= seam - 1u;
            const uint32_t x = ((w << 5) + b) / L;
            atomicOr(ws.SEAMV + (x >> 5), 1u << (x & 31u));
        }
    }
}

__device__ __forceinline__ Lat<Word64> label_lat(const PlainWs &ws, uint32_t L)
{
    Lat<Word64> t;
    t.g = Geom{L, L * L, (L * L + 31u) / 32u};
    t.uf.w = ws.uf;
    t.S = nullptr;
    t.JH = nullptr;
    t.JV = nullptr;
    t.OH = ws.OH;
    t.OV = ws.OV;
    t.FLIP = ws.FLIP;
    t.ROOT = ws.ROOT;
    t.SEAMV = ws.SEAMV;
    t.RE = nullptr;
    t.wrap = &ws.sc->wrap;
    t.err = &ws.sc->err;
    t.cap = t.g.N + 64u;
    return t;
}

__global__ void __launch_bounds__(kPlainThreads) k_plain_label_heads(PlainWs ws, uint32_t L)
{
    const Lat<Word64> t = label_lat(ws, L);
    for (uint32_t w = gtid(); w < t.g.NW; w += gnthreads()) t.ROOT[w] = 0u;
    phase_heads<Word64>(t, gwarp(), gnwarps());
}

__global__ void __launch_bounds__(kPlainThreads) k_plain_label_union(PlainWs ws, uint32_t L)
{
    phase_union<Word64>(label_lat(ws, L), gtid(), gnthreads());
}

__global__ void __launch_bounds__(kPlainThreads) k_plain_label_roots(PlainWs ws, uint32_t L)
{
    (void)phase_roots<Word64>(label_lat(ws, L), gtid(), gnthreads());
}

__global__ void __launch_bounds__(kPlainThreads) k_plain_label_finalize(PlainWs ws, uint32_t L)
{
    phase_sites<Word64>(label_lat(ws, L), gwarp(), gnwarps(), false, false);
}

// Exclusive prefix of root counts per word (single CTA) into the FLIP plane.
__global__ void __launch_bounds__(1024) k_plain_label_scan(PlainWs ws, uint32_t L)
{
    __shared__ uint32_t s_scan[1024];
    const uint32_t NW = (L * L + 31u) / 32u;
    const uint32_t tid = threadIdx.x, per = (NW + 1023u) / 1024u;
    const uint32_t w0 = tid * per, w1 = min(NW, w0 + per);
    uint32_t local = 0;
    for (uint32_t w = w0; w < w1; ++w) local += __popc(ws.ROOT[w]);
    s_scan[tid] = local;
    __syncthreads();
    for (uint32_t off = 1; off < 1024u; off <<= 1) {
        const uint32_t v = tid >= off ? s_scan[tid - off] : 0u;
        __syncthreads();
        s_scan[tid] += v;
        __syncthreads();
    }
    uint32_t base = s_scan[tid] - local;
    for (uint32_t w = w0; w < w1; ++w) {
        ws.FLIP[w] = base;
        base += __popc(ws.ROOT[w]);
    }
    if (tid == 0) ws.sc->nroots = s_scan[1023];
}

__global__ void __launch_bounds__(kPlainThreads) k_plain_label_write(PlainWs ws, uint32_t L, int32_t *labels,
                                                                     int32_t *n_clusters, uint8_t *wraps,
                                                                     int *status)
{
    const uint32_t N = L * L;
    for (uint32_t n = gtid(); n < N; n += gnthreads()) {
        const uint32_t r = Word64::parent(*((volatile unsigned long long *)(ws.uf + n)));
        labels[n] = (int32_t)(ws.FLIP[r >> 5] + __popc(ws.ROOT[r >> 5] & ((1u << (r & 31u)) - 1u)));
    }
    if (gtid() == 0) {
        *n_clusters = (int32_t)ws.sc->nroots;
        wraps[0] = (uint8_t)(ws.sc->wrap & 1);
        wraps[1] = (uint8_t)((ws.sc->wrap >> 1) & 1);
        if (ws.sc->err) atomicOr(status, ws.sc->err);
    }
}

__global__ void k_plain_label_begin(PlainWs ws, uint32_t L)
{
    for (uint32_t i = gtid(); i < (L + 31u) / 32u; i += gnthreads()) ws.SEAMV[i] = 0u;
    if (gtid() == 0) {
        PlainScratch z{};
        *ws.sc = z;
    }
}

}  // namespace

size_t plain_workspace_bytes(int64_t L) { return plain_sizes(L).total; }

cudaError_t launch_plain_sweeps(rbim_chain_t *chain, uint32_t *spin_pool, const uint32_t *coupling_pool,
                                long long *acc_i, double *acc_f, int32_t *records, int n_sweeps, int *status,
                                void *workspace, int64_t L, cudaStream_t stream)
{
    PlainArgs a{L, chain, spin_pool, coupling_pool, acc_i, acc_f, records, status, plain_ws(workspace, L)};
    const int grid = plain_grid_for(L);
    k_plain_begin<<<1, 256, 0, stream>>>(a);
    for (int s = 0; s < n_sweeps; ++s) {
        k_plain_activate<<<grid, kPlainThreads, 0, stream>>>(a);
        k_plain_heads<<<grid, kPlainThreads, 0, stream>>>(a);
        k_plain_union<<<grid, kPlainThreads, 0, stream>>>(a);
        k_plain_roots<<<grid, kPlainThreads, 0, stream>>>(a);
        k_plain_finalize<<<grid, kPlainThreads, 0, stream>>>(a);
        k_plain_measure1<<<grid, kPlainThreads, 0, stream>>>(a);
        k_plain_measure3<<<grid, kPlainThreads, 0, stream>>>(a);
    }
    return cudaGetLastError();
}

cudaError_t launch_plain_label(int64_t L, const uint8_t *occ, int32_t *labels, int32_t *n_clusters,
                               uint8_t *wraps, int *status, void *workspace, cudaStream_t stream)
{
    const PlainWs ws = plain_ws(workspace, L);
    const int grid = plain_grid_for(L);
    const uint32_t l = (uint32_t)L;
    k_plain_label_begin<<<1, 256, 0, stream>>>(ws, l);
    k_plain_label_load<<<grid, kPlainThreads, 0, stream>>>(ws, l, occ);
    k_plain_label_heads<<<grid, kPlainThreads, 0, stream>>>(ws, l);
    k_plain_label_union<<<grid, kPlainThreads, 0, stream>>>(ws, l);
    k_plain_label_roots<<<grid, kPlainThreads, 0, stream>>>(ws, l);
    k_plain_label_finalize<<<grid, kPlainThreads, 0, stream>>>(ws, l);
    k_plain_label_scan<<<1, 1024, 0, stream>>>(ws, l);
    k_plain_label_write<<<grid, kPlainThreads, 0, stream>>>(ws, l, labels, n_clusters, wraps, status);
    return cudaGetLastError();
}

}  // namespace rbim

// Resident engine: one lattice per CTA, held in shared memory for every sweep
// of a call.  A persistent grid pulls chains from a work queue (an atomic
// counter in global memory), loads the chain's spin and coupling planes,
// runs its sweeps entirely on chip (bond activation, run-based union-find with
// image offsets for exact wrapping, flip, measurement) and writes back only
// the spin plane, the bin sums and the optional per-sweep records.
//
// This replaces, per chain, the loop of run_single_realization
// (src/rbim/simulation.py:196-242) around sw_sweep
// (src/rbim/swendsen_wang.py:103-172).
#include <algorithm>

#include "rbim_internal.h"
#include "rbim_phases.cuh"

namespace rbim {

namespace {

constexpr uint32_t kMaxResidentSites = 65536;  // 16-bit parents in Word32
// Dynamic shared memory budget: the 227 KB per-CTA limit minus room for the
// kernels' static shared scratch.
constexpr size_t kMaxSmem = 227 * 1024 - 8 * 1024;

size_t align16(size_t v) { return (v + 15) & ~size_t(15); }

}  // namespace

ResidentLayout resident_layout(uint32_t l_max, int threads)
{
    ResidentLayout ly{};
    ly.l_max = l_max;
    ly.n_max = l_max * l_max;
    const uint32_t nw = (ly.n_max + 31u) / 32u;
    ly.nw_max = (nw + 3u) & ~3u;
    size_t off = 0;
    ly.off_uf = off;
    off = align16(off + 4ull * ly.n_max);
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
    ly.off_SEAMV = off;
    off = align16(off + 4ull * (((l_max + 31u) / 32u) + 4u));
    ly.bytes = off;
    (void)threads;
    return ly;
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
    // About eight words per warp, as a power of two in [128, 1024].
    const int nw = (l_max * l_max + 31) / 32;
    const int want = 32 * ((nw + 7) / 8);
    int t = 128;
    while (t < want && t < 1024) t *= 2;
    return t;
}

// Shared scratch of one CTA.
template <int NT>
struct Red {
    uint32_t k1[NT / 32], k2[NT / 32];
    uint32_t unsat[NT / 32], downs[NT / 32], roots[NT / 32];
    int mc[NT / 32];
    int item, wrap, err;
    uint32_t ncl, g1, s1, s2, unsat_t, downs_t;
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

template <int NT>
__device__ __forceinline__ Lat<Word32> make_lat(unsigned char *smem, const ResidentLayout &ly, uint32_t L,
                                                Red<NT> &red)
{
    Lat<Word32> t;
    t.g = Geom{L, L * L, (L * L + 31u) / 32u};
    t.uf.w = (uint32_t *)(smem + ly.off_uf);
    t.S = (uint32_t *)(smem + ly.off_S);
    t.JH = (const uint32_t *)(smem + ly.off_JH);
    t.JV = (const uint32_t *)(smem + ly.off_JV);
    t.OH = (uint32_t *)(smem + ly.off_OH);
    t.OV = (uint32_t *)(smem + ly.off_OV);
    t.FLIP = (uint32_t *)(smem + ly.off_FLIP);
    t.ROOT = (uint32_t *)(smem + ly.off_ROOT);
    t.SEAMV = (uint32_t *)(smem + ly.off_SEAMV);
    t.wrap = &red.wrap;
    t.err = &red.err;
    t.cap = t.g.N + 64u;
    return t;
}

// Measurement of one sweep after phase_finalize(count = true): energy,
// magnetization, n_clusters, S1, S2, |M_C1| (reference sw_sweep,
// src/rbim/swendsen_wang.py:146-172).  Ends with a barrier.  Thread 0 returns
// the record in rec.
template <int NT>
__device__ __forceinline__ void resident_measure(const Lat<Word32> &t, Red<NT> &red, uint32_t nroots_warp,
                                                 long long rec[kRecLen])
{
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    constexpr uint32_t nwarps = NT / 32;
    const Geom &g = t.g;
    uint32_t unsat = 0, downs = 0;
    measure_energy(g, t.S, t.JH, t.JV, tid, NT, unsat, downs);
    uint32_t k1 = 0, k2 = 0;
    for (uint32_t w = tid; w < g.NW; w += NT) {
        uint32_t roots = t.ROOT[w];
        while (roots) {
            const uint32_t b = __ffs(roots) - 1u;
            roots &= roots - 1u;
            const uint32_t r = (w << 5) + b;
            const uint32_t key = (Word32::count(t.uf.ld(r)) << 16) | (0xFFFFu - r);
            top2_merge(k1, k2, key, 0u);
        }
    }
    warp_top2(k1, k2);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        unsat += __shfl_xor_sync(0xFFFFFFFFu, unsat, o);
        downs += __shfl_xor_sync(0xFFFFFFFFu, downs, o);
    }
    if (lane == 0) {
        red.k1[warp] = k1;
        red.k2[warp] = k2;
        red.unsat[warp] = unsat;
        red.downs[warp] = downs;
        red.roots[warp] = nroots_warp;
    }
    __syncthreads();
    if (warp == 0) {
        uint32_t a1 = lane < nwarps ? red.k1[lane] : 0u, a2 = lane < nwarps ? red.k2[lane] : 0u;
        uint32_t u = lane < nwarps ? red.unsat[lane] : 0u, d = lane < nwarps ? red.downs[lane] : 0u;
        uint32_t nr = lane < nwarps ? red.roots[lane] : 0u;
        warp_top2(a1, a2);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            u += __shfl_xor_sync(0xFFFFFFFFu, u, o);
            d += __shfl_xor_sync(0xFFFFFFFFu, d, o);
            nr += __shfl_xor_sync(0xFFFFFFFFu, nr, o);
        }
        if (lane == 0) {
            red.ncl = nr;
            red.unsat_t = u;
            red.downs_t = d;
            if (nr == 1) {
                // One cluster covers the lattice (its 16-bit size field may
                // have wrapped at N = 65536).
                red.g1 = 0;
                red.s1 = g.N;
                red.s2 = 0;
            } else {
                red.g1 = 0xFFFFu - (a1 & 0xFFFFu);
                red.s1 = a1 >> 16;
                red.s2 = a2 >> 16;
            }
        }
    }
    __syncthreads();
    const uint32_t ncl = red.ncl;
    const long long M = (long long)g.N - 2ll * (long long)red.downs_t;
    long long mc_total;
    if (ncl > 1) {
        const uint32_t g1 = red.g1;
        int mc = 0;
        for (uint32_t w = warp; w < g.NW; w += nwarps) {
            const uint32_t n = (w << 5) + lane;
            const bool in = n < g.N && Word32::parent(t.uf.ld(n)) == g1;
            const uint32_t m = __ballot_sync(0xFFFFFFFFu, in);
            if (lane == 0) mc += (int)__popc(m) - 2 * (int)__popc(m & t.S[w]);
        }
        if (lane == 0) red.mc[warp] = mc;
        __syncthreads();
        mc_total = 0;
        if (tid == 0)
            for (uint32_t i = 0; i < nwarps; ++i) mc_total += red.mc[i];
    } else {
        mc_total = M;
    }
    if (tid == 0) {
        rec[0] = 2ll * (long long)red.unsat_t - 2ll * (long long)g.N;
        rec[1] = M;
        rec[2] = ncl;
        rec[3] = red.s1;
        rec[4] = mc_total < 0 ? -mc_total : mc_total;
        rec[5] = red.s2;
        rec[6] = red.wrap & 1;
        rec[7] = (red.wrap >> 1) & 1;
    }
    __syncthreads();
}

template <int NT>
__global__ void __launch_bounds__(NT, MinBlocks<NT>::value) k_resident_sweeps(rbim_chain_t *chains, int n_chains, uint32_t *spin_pool,
                                                        const uint32_t *coupling_pool, long long *acc_i,
                                                        double *acc_f, int32_t *records, int n_sweeps, int *queue,
                                                        int *status, ResidentLayout ly)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ Red<NT> red;
    const uint32_t tid = threadIdx.x, warp = tid >> 5;
    constexpr uint32_t nwarps = NT / 32;

    if (tid == 0) red.err = 0;
    for (;;) {
        if (tid == 0) red.item = atomicAdd(queue, 1);
        __syncthreads();
        const int item = red.item;
        if (item >= n_chains) break;
        if (tid == 0) {
            red.ch = chains[item];
            red.acc.zero();
            red.cur_bin = -1;
        }
        __syncthreads();
        const rbim_chain_t &ch = red.ch;
        if (ch.L < 3 || ch.L > (int64_t)ly.l_max || ch.sweeps_per_bin < 1 || ch.n_bins < 0 || ch.n_therm < 0) {
            if (tid == 0) atomicOr(status, kErrBadChain);
            __syncthreads();
            continue;
        }
        const uint32_t L = (uint32_t)ch.L;
        Lat<Word32> t = make_lat<NT>(smem, ly, L, red);
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
        }
        const uint64_t t_end = (uint64_t)ch.n_therm + (uint64_t)ch.n_bins * (uint64_t)ch.sweeps_per_bin;
        uint64_t sweep = ch.sweep;
        const uint64_t stop = min(t_end, sweep + (uint64_t)max(n_sweeps, 0));
        SweepRng rng;
        rng.key = ch.key;
        rng.thr_any = ch.thr > 0;
        rng.thr_m1 = ch.thr > 0 ? (uint32_t)min(ch.thr - 1ull, 0xFFFFFFFFull) : 0u;
        __syncthreads();

        for (; sweep < stop; ++sweep) {
            const bool measure = sweep >= (uint64_t)ch.n_therm;
            rng.sweep = sweep;
            if (tid == 0) red.wrap = 0;
            phase_activate<Word32>(t, rng, warp, nwarps, tid, NT);
            __syncthreads();
            phase_heads<Word32>(t, warp, nwarps);
            __syncthreads();
            phase_union<Word32>(t, warp, nwarps, tid, NT);
            __syncthreads();
            const uint32_t nr = phase_finalize<Word32>(t, warp, nwarps, true, measure);
            for (uint32_t i = tid; i < (L + 31u) / 32u; i += NT) t.SEAMV[i] = 0u;
            __syncthreads();
            if (measure) {
                long long rec[kRecLen];
                resident_measure<NT>(t, red, nr, rec);
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
                    red.acc.add(rec[0], rec[1], rec[2], rec[3], rec[4], rec[5], (int)rec[6], (int)rec[7]);
                    if (records && ch.rec_off >= 0) {
                        int32_t *row = records + (ch.rec_off + idx) * kRecLen;
#pragma unroll
                        for (int k = 0; k < kRecLen; ++k) row[k] = (int32_t)rec[k];
                    }
                }
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
__global__ void __launch_bounds__(NT, MinBlocks<NT>::value) k_resident_label(uint32_t L, const uint8_t *occ, int32_t *labels,
                                                       int32_t *n_clusters, uint8_t *wraps, int *status,
                                                       ResidentLayout ly)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ Red<NT> red;
    __shared__ uint32_t s_scan[NT];
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    constexpr uint32_t nwarps = NT / 32;
    const size_t lat = blockIdx.x;
    if (tid == 0) {
        red.err = 0;
        red.wrap = 0;
    }
    Lat<Word32> t = make_lat<NT>(smem, ly, L, red);
    const Geom g = t.g;
    const uint8_t *o = occ + lat * 2ull * g.N;
    for (uint32_t i = tid; i < (L + 31u) / 32u; i += NT) t.SEAMV[i] = 0u;
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
    phase_heads<Word32>(t, warp, nwarps);
    __syncthreads();
    phase_union<Word32>(t, warp, nwarps, tid, NT);
    __syncthreads();
    const uint32_t nr = phase_finalize<Word32>(t, warp, nwarps, false, false);
    if (lane == 0) red.roots[warp] = nr;
    __syncthreads();
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
        const uint32_t r = Word32::parent(t.uf.ld(n));
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

template <int NT>
cudaError_t launch_sweeps_nt(const rbim_chain_t *chains, int n_chains, int l_max, uint32_t *spin_pool,
                             const uint32_t *coupling_pool, long long *acc_i, double *acc_f, int32_t *rec,
                             int n_sweeps, int grid, int *queue, int *status, cudaStream_t stream)
{
    const ResidentLayout ly = resident_layout(l_max, NT);
    cudaError_t e = cudaFuncSetAttribute(k_resident_sweeps<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)ly.bytes);
    if (e != cudaSuccess) return e;
    if (grid <= 0) {
        int per_sm = 0, sms = 0, dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_resident_sweeps<NT>, NT, ly.bytes);
        if (e != cudaSuccess) return e;
        grid = std::max(1, per_sm) * sms;
    }
    grid = std::min(grid, n_chains);
    e = cudaMemsetAsync(queue, 0, sizeof(int), stream);
    if (e != cudaSuccess) return e;
    k_resident_sweeps<NT><<<grid, NT, ly.bytes, stream>>>(const_cast<rbim_chain_t *>(chains), n_chains, spin_pool,
                                                          coupling_pool, acc_i, acc_f, rec, n_sweeps, queue,
                                                          status, ly);
    return cudaGetLastError();
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
    if (threads <= 0) threads = resident_default_threads(L);
    switch (threads) {
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

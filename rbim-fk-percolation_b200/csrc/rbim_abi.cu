// C ABI of librbim_sm100 (declared in include/rbim_sm100.h): argument checks,
// error reporting and dispatch to the resident and plain engines.
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <mutex>
#include <string>

#include "rbim_internal.h"
#include "rbim_phases.cuh"

namespace {

thread_local std::string g_last_error;

int fail(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

int cuda_check(cudaError_t e, const char *what)
{
    if (e == cudaSuccess) return RBIM_OK;
    return fail(RBIM_ERR_CUDA, "%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
}

bool aligned16(const void *p) { return ((uintptr_t)p & 15u) == 0; }

int64_t plane_words(int64_t L) { return (((L * L + 31) / 32) + 3) & ~int64_t(3); }

// Hot-start or cold spins: word w of chain c is word (w & 3) of Philox block
// w >> 2 of stream 2 (sites 32w .. 32w+31), masked to the lattice.
__global__ void k_init_spins(const rbim_chain_t *chains, uint32_t *spin_pool, int hot)
{
    const rbim_chain_t *c = chains + blockIdx.x;
    const uint32_t L = (uint32_t)c->L;
    const rbim::Geom g{L, L * L, (L * L + 31u) / 32u};
    uint32_t *s = spin_pool + c->spin_off;
    const uint32_t nwp = (g.NW + 3u) & ~3u;
    for (uint32_t w = threadIdx.x; w < nwp; w += blockDim.x) {
        uint32_t v = 0;
        if (hot && w < g.NW) {
            const rbim::U4 r = rbim::philox_block(c->key, w >> 2, 0, rbim::kStreamInit);
            v = rbim::u4_word(r, w & 3u) & g.valid(w);
        }
        s[w] = w < g.NW ? v : 0u;
    }
}

struct ActWs {
    uint32_t *OH, *OV, *SEAMV;
};

ActWs act_ws(void *base, int64_t L)
{
    const size_t plane = 4 * (size_t)(plane_words(L) + 4);
    char *p = (char *)base;
    return {(uint32_t *)p, (uint32_t *)(p + plane), (uint32_t *)(p + 2 * plane)};
}

size_t act_ws_bytes(int64_t L) { return 2 * 4 * (size_t)(plane_words(L) + 4) + 4 * (size_t)((L + 31) / 32 + 4); }

__global__ void k_act_clear(ActWs ws, uint32_t L)
{
    for (uint32_t i = threadIdx.x; i < (L + 31u) / 32u; i += blockDim.x) ws.SEAMV[i] = 0u;
}

__global__ void __launch_bounds__(256) k_act_run(ActWs ws, uint32_t L, const uint32_t *S, const uint32_t *J,
                                                  uint64_t key, uint64_t thr, uint64_t sweep)
{
    rbim::Lat<rbim::Word64> t{};
    t.g = rbim::Geom{L, L * L, (L * L + 31u) / 32u};
    t.S = const_cast<uint32_t *>(S);
    t.JH = J;
    t.JV = J + ((t.g.NW + 3u) & ~3u);
    t.OH = ws.OH;
    t.OV = ws.OV;
    t.SEAMV = ws.SEAMV;
    t.FLIP = nullptr;  // flip bits are not part of the activation seam
    const rbim::SweepRng rng = rbim::make_rng(key, sweep, thr);
    const uint32_t gt = blockIdx.x * blockDim.x + threadIdx.x, nt = gridDim.x * blockDim.x;
    rbim::phase_activate_bonds<rbim::Word64>(t, rng, gt >> 5, nt >> 5);
}

__global__ void k_act_expand(ActWs ws, uint32_t L, uint8_t *occ)
{
    const uint32_t N = L * L;
    for (uint32_t n = blockIdx.x * blockDim.x + threadIdx.x; n < N; n += gridDim.x * blockDim.x) {
        const uint32_t w = n >> 5, b = n & 31u;
        occ[2ull * n] = (uint8_t)((ws.OH[w] >> b) & 1u);
        uint32_t v = (ws.OV[w] >> b) & 1u;
        if (n % L == L - 1u) v = (ws.SEAMV[(n / L) >> 5] >> ((n / L) & 31u)) & 1u;
        occ[2ull * n + 1] = (uint8_t)v;
    }
}

int check_chain_sizes(int64_t L)
{
    if (L < 3) return fail(RBIM_ERR_INVALID, "L must be at least 3 (got %lld)", (long long)L);
    if (L > 32768) return fail(RBIM_ERR_UNSUPPORTED, "L = %lld exceeds the engine's limit of 32768", (long long)L);
    return RBIM_OK;
}

}  // namespace

extern "C" {

const char *rbim_last_error(void) { return g_last_error.c_str(); }

int rbim_abi_version(void) { return RBIM_ABI_VERSION; }

int64_t rbim_plane_words(int64_t L) { return L < 1 ? 0 : plane_words(L); }

int rbim_resident_max_l(void) { return rbim::resident_max_l(); }

int rbim_resident_threads(int64_t L)
{
    if (L < 3 || L > rbim::resident_max_l()) return 0;
    return rbim::resident_default_threads((int)L);
}

int rbim_init_spins(const rbim_chain_t *chains, int n_chains, uint32_t *spin_pool, int hot, void *stream)
{
    if (n_chains < 0) return fail(RBIM_ERR_INVALID, "n_chains must be >= 0");
    if (n_chains == 0) return RBIM_OK;
    if (!chains || !spin_pool) return fail(RBIM_ERR_INVALID, "null pointer");
    if (!aligned16(spin_pool)) return fail(RBIM_ERR_INVALID, "spin_pool must be 16-byte aligned");
    k_init_spins<<<n_chains, 256, 0, (cudaStream_t)stream>>>(chains, spin_pool, hot);
    return cuda_check(cudaGetLastError(), "rbim_init_spins");
}

size_t rbim_activate_workspace_bytes(int64_t L) { return L < 3 ? 0 : act_ws_bytes(L); }

int rbim_activate(int64_t L, const uint32_t *spins, const uint32_t *couplings, uint64_t key, uint64_t thr,
                  uint64_t sweep, uint8_t *occ, void *workspace, size_t workspace_bytes, void *stream)
{
    if (int rc = check_chain_sizes(L)) return rc;
    if (!spins || !couplings || !occ || !workspace) return fail(RBIM_ERR_INVALID, "null pointer");
    if (thr > (1ull << 32)) return fail(RBIM_ERR_INVALID, "thr must be <= 2^32");
    if (workspace_bytes < act_ws_bytes(L))
        return fail(RBIM_ERR_INVALID, "workspace too small: %zu < %zu", workspace_bytes, act_ws_bytes(L));
    if (!aligned16(workspace)) return fail(RBIM_ERR_INVALID, "workspace must be 16-byte aligned");
    cudaStream_t s = (cudaStream_t)stream;
    const ActWs ws = act_ws(workspace, L);
    const uint32_t l = (uint32_t)L;
    const uint32_t chunks = (l * l + 63u) / 64u;
    const uint32_t blocks = (chunks + 7u) / 8u;  // one chunk per warp, 8 warps per block
    k_act_clear<<<1, 256, 0, s>>>(ws, l);
    k_act_run<<<blocks, 256, 0, s>>>(ws, l, spins, couplings, key, thr, sweep);
    k_act_expand<<<(l * l + 255u) / 256u, 256, 0, s>>>(ws, l, occ);
    return cuda_check(cudaGetLastError(), "rbim_activate");
}

size_t rbim_label_wrap_workspace_bytes(int64_t L)
{
    if (L < 3) return 0;
    if (L <= rbim::resident_max_l()) return 0;
    return rbim::plain_workspace_bytes(L);
}

int rbim_label_wrap(int64_t L, int n_lattices, const uint8_t *occ, int32_t *labels, int32_t *n_clusters,
                    uint8_t *wraps, int32_t *status, void *workspace, size_t workspace_bytes, void *stream)
{
    if (int rc = check_chain_sizes(L)) return rc;
    if (n_lattices < 0) return fail(RBIM_ERR_INVALID, "n_lattices must be >= 0");
    if (n_lattices == 0) return RBIM_OK;
    if (!occ || !labels || !n_clusters || !wraps || !status) return fail(RBIM_ERR_INVALID, "null pointer");
    cudaStream_t s = (cudaStream_t)stream;
    if (L <= rbim::resident_max_l()) {
        return cuda_check(
            rbim::launch_resident_label((int)L, n_lattices, occ, labels, n_clusters, wraps, 0, status, s),
            "rbim_label_wrap (resident)");
    }
    const size_t need = rbim::plain_workspace_bytes(L);
    if (!workspace || workspace_bytes < need)
        return fail(RBIM_ERR_INVALID, "workspace too small: %zu < %zu", workspace_bytes, need);
    if (((uintptr_t)workspace & 255u) != 0) return fail(RBIM_ERR_INVALID, "workspace must be 256-byte aligned");
    const size_t n = (size_t)L * (size_t)L;
    for (int i = 0; i < n_lattices; ++i) {
        cudaError_t e = rbim::launch_plain_label(L, occ + 2 * n * i, labels + n * i, n_clusters + i, wraps + 2 * i,
                                                 status, workspace, s);
        if (e != cudaSuccess) return cuda_check(e, "rbim_label_wrap (plain)");
    }
    return RBIM_OK;
}

size_t rbim_batched_workspace_bytes(void) { return 256; }

int rbim_sweeps_batched(rbim_chain_t *chains, int n_chains, int64_t l_max, uint32_t *spin_pool,
                        const uint32_t *coupling_pool, int64_t *acc_int, double *acc_f64, int32_t *records,
                        int n_sweeps, int threads, int32_t *status, void *workspace, size_t workspace_bytes,
                        void *stream)
{
    if (n_chains < 0 || n_sweeps < 0) return fail(RBIM_ERR_INVALID, "n_chains and n_sweeps must be >= 0");
    if (n_chains == 0 || n_sweeps == 0) return RBIM_OK;
    if (int rc = check_chain_sizes(l_max)) return rc;
    if (l_max > rbim::resident_max_l())
        return fail(RBIM_ERR_UNSUPPORTED, "l_max = %lld exceeds the resident engine's limit %d", (long long)l_max,
                    rbim::resident_max_l());
    if (!chains || !spin_pool || !coupling_pool || !acc_int || !acc_f64 || !status || !workspace)
        return fail(RBIM_ERR_INVALID, "null pointer");
    if (!aligned16(spin_pool) || !aligned16(coupling_pool))
        return fail(RBIM_ERR_INVALID, "spin and coupling pools must be 16-byte aligned");
    if (workspace_bytes < rbim_batched_workspace_bytes()) return fail(RBIM_ERR_INVALID, "workspace too small");
    if (threads != 0 && threads != 32 && threads != 64 && threads != 128 && threads != 256 && threads != 512 &&
        threads != 1024)
        return fail(RBIM_ERR_INVALID, "threads must be 0, 32, 64, 128, 256, 512 or 1024 (got %d)", threads);
    cudaError_t e = rbim::launch_resident_sweeps(chains, n_chains, (int)l_max, spin_pool, coupling_pool,
                                                 (long long *)acc_int, acc_f64, records, n_sweeps, threads, 0,
                                                 (int *)workspace, status, (cudaStream_t)stream);
    return cuda_check(e, "rbim_sweeps_batched");
}

int rbim_cluster_max_l(void)
{
    // Per device: the largest L whose cluster fits the shared-memory budget
    // and can be scheduled at least once.
    static int cached[64];
    static std::mutex mu;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
    std::lock_guard<std::mutex> lock(mu);
    if (cached[dev]) return cached[dev] > 0 ? cached[dev] : 0;
    int ok_c[17][2] = {};  // per cluster size and CTA size: 1 schedulable, -1 not
    int best = -1;
    for (int L = 1024; L > rbim::resident_max_l(); --L) {
        const rbim::ClusterPlan plan = rbim::cluster_plan((uint32_t)L);
        if (plan.C == 0) continue;
        const int m = plan.threads == 512u ? 1 : 0;
        if (ok_c[plan.C][m] == 0) {
            int clusters = 0;
            const cudaError_t e = rbim::cluster_occupancy((uint32_t)L, &clusters);
            ok_c[plan.C][m] = (e == cudaSuccess && clusters > 0) ? 1 : -1;
            if (e != cudaSuccess) cudaGetLastError();
        }
        if (ok_c[plan.C][m] > 0) {
            best = L;
            break;
        }
    }
    cached[dev] = best;
    return best > 0 ? best : 0;
}

int rbim_cluster_size(int64_t L)
{
    if (L <= rbim::resident_max_l() || L > 65535) return 0;
    return (int)rbim::cluster_size_for((uint32_t)L);
}

int rbim_cluster_threads(int64_t L)
{
    if (L <= rbim::resident_max_l() || L > 65535) return 0;
    const rbim::ClusterPlan plan = rbim::cluster_plan((uint32_t)L);
    return plan.C ? (int)plan.threads : 0;
}

int rbim_sweeps_clustered(rbim_chain_t *chains, int n_chains, int64_t l_max, uint32_t *spin_pool,
                          const uint32_t *coupling_pool, int64_t *acc_int, double *acc_f64, int32_t *records,
                          int n_sweeps, int32_t *status, void *workspace, size_t workspace_bytes, void *stream)
{
    if (n_chains < 0 || n_sweeps < 0) return fail(RBIM_ERR_INVALID, "n_chains and n_sweeps must be >= 0");
    if (n_chains == 0 || n_sweeps == 0) return RBIM_OK;
    if (int rc = check_chain_sizes(l_max)) return rc;
    if (l_max <= rbim::resident_max_l())
        return fail(RBIM_ERR_INVALID, "l_max = %lld is small enough for rbim_sweeps_batched (limit %d)",
                    (long long)l_max, rbim::resident_max_l());
    if (!chains || !spin_pool || !coupling_pool || !acc_int || !acc_f64 || !status || !workspace)
        return fail(RBIM_ERR_INVALID, "null pointer");
    if (!aligned16(spin_pool) || !aligned16(coupling_pool))
        return fail(RBIM_ERR_INVALID, "spin and coupling pools must be 16-byte aligned");
    if (workspace_bytes < rbim_batched_workspace_bytes()) return fail(RBIM_ERR_INVALID, "workspace too small");
    const int lim = rbim_cluster_max_l();
    if (l_max > lim)
        return fail(RBIM_ERR_UNSUPPORTED, "l_max = %lld exceeds the cluster engine's limit %d on this device",
                    (long long)l_max, lim);
    cudaError_t e = rbim::launch_cluster_sweeps(chains, n_chains, (int)l_max, spin_pool, coupling_pool,
                                                (long long *)acc_int, acc_f64, records, n_sweeps, (int *)workspace,
                                                status, (cudaStream_t)stream);
    return cuda_check(e, "rbim_sweeps_clustered");
}

int rbim_cluster_plans(int64_t L, int *ctas, int *threads, int max_plans)
{
    if (L <= rbim::resident_max_l() || L > 65535 || max_plans < 0) return 0;
    const uint32_t l = (uint32_t)L;
    const rbim::ClusterPlan def = rbim::cluster_plan(l);
    int n = 0;
    auto consider = [&](rbim::ClusterPlan p) {
        if (!rbim::cluster_plan_ok(l, p)) return;
        int clusters = 0;
        if (rbim::cluster_occupancy_plan(l, p, &clusters) != cudaSuccess) {
            cudaGetLastError();
            return;
        }
        if (clusters <= 0) return;
        if (n < max_plans && ctas && threads) {
            ctas[n] = (int)p.C;
            threads[n] = (int)p.threads;
        }
        ++n;
    };
    if (def.C) consider(def);
    for (uint32_t t : {1024u, 512u})
        for (uint32_t C = 2; C <= 16u; ++C)
            if (!(C == def.C && t == def.threads)) consider({C, t});
    return n;
}

int rbim_sweeps_clustered_plan(rbim_chain_t *chains, int n_chains, int64_t l_max, int cluster_ctas, int threads,
                               uint32_t *spin_pool, const uint32_t *coupling_pool, int64_t *acc_int, double *acc_f64,
                               int32_t *records, int n_sweeps, int32_t *status, void *workspace,
                               size_t workspace_bytes, void *stream)
{
    if (n_chains < 0 || n_sweeps < 0) return fail(RBIM_ERR_INVALID, "n_chains and n_sweeps must be >= 0");
    if (n_chains == 0 || n_sweeps == 0) return RBIM_OK;
    if (int rc = check_chain_sizes(l_max)) return rc;
    if (l_max <= rbim::resident_max_l())
        return fail(RBIM_ERR_INVALID, "l_max = %lld is small enough for rbim_sweeps_batched (limit %d)",
                    (long long)l_max, rbim::resident_max_l());
    if (l_max > 65535) return fail(RBIM_ERR_UNSUPPORTED, "l_max = %lld is beyond the cluster engine", (long long)l_max);
    const rbim::ClusterPlan plan{(uint32_t)std::max(cluster_ctas, 0), (uint32_t)std::max(threads, 0)};
    if (!rbim::cluster_plan_ok((uint32_t)l_max, plan))
        return fail(RBIM_ERR_INVALID, "plan of %d CTAs of %d threads cannot run L = %lld (see rbim_cluster_plans)",
                    cluster_ctas, threads, (long long)l_max);
    if (!chains || !spin_pool || !coupling_pool || !acc_int || !acc_f64 || !status || !workspace)
        return fail(RBIM_ERR_INVALID, "null pointer");
    if (!aligned16(spin_pool) || !aligned16(coupling_pool))
        return fail(RBIM_ERR_INVALID, "spin and coupling pools must be 16-byte aligned");
    if (workspace_bytes < rbim_batched_workspace_bytes()) return fail(RBIM_ERR_INVALID, "workspace too small");
    cudaError_t e = rbim::launch_cluster_sweeps_plan(chains, n_chains, (int)l_max, plan, spin_pool, coupling_pool,
                                                     (long long *)acc_int, acc_f64, records, n_sweeps,
                                                     (int *)workspace, status, (cudaStream_t)stream);
    return cuda_check(e, "rbim_sweeps_clustered_plan");
}

size_t rbim_plain_workspace_bytes(int64_t L) { return L < 3 ? 0 : rbim::plain_workspace_bytes(L); }

int rbim_sweeps_plain(int64_t L, rbim_chain_t *chain, uint32_t *spin_pool, const uint32_t *coupling_pool,
                      int64_t *acc_int, double *acc_f64, int32_t *records, int n_sweeps, int32_t *status,
                      void *workspace, size_t workspace_bytes, void *stream)
{
    if (int rc = check_chain_sizes(L)) return rc;
    if (n_sweeps < 0) return fail(RBIM_ERR_INVALID, "n_sweeps must be >= 0");
    if (n_sweeps == 0) return RBIM_OK;
    if (!chain || !spin_pool || !coupling_pool || !acc_int || !acc_f64 || !status || !workspace)
        return fail(RBIM_ERR_INVALID, "null pointer");
    const size_t need = rbim::plain_workspace_bytes(L);
    if (workspace_bytes < need) return fail(RBIM_ERR_INVALID, "workspace too small: %zu < %zu", workspace_bytes, need);
    if (((uintptr_t)workspace & 255u) != 0) return fail(RBIM_ERR_INVALID, "workspace must be 256-byte aligned");
    cudaError_t e = rbim::launch_plain_sweeps(chain, spin_pool, coupling_pool, (long long *)acc_int, acc_f64,
                                              records, n_sweeps, status, workspace, L, (cudaStream_t)stream);
    return cuda_check(e, "rbim_sweeps_plain");
}

int rbim_grid_plan(int64_t L, int *ctas, int *threads)
{
    if (!ctas || !threads) return fail(RBIM_ERR_INVALID, "null pointer");
    *ctas = 0;
    *threads = 0;
    if (L <= 32 || L > 65535) return fail(RBIM_ERR_UNSUPPORTED, "grid engine: L = %lld outside 33..65535", (long long)L);
    const rbim::GridPlan p = rbim::grid_plan((uint32_t)L);
    if (!p.C) return fail(RBIM_ERR_UNSUPPORTED, "grid engine: no plan fits L = %lld", (long long)L);
    *ctas = (int)p.C;
    *threads = (int)p.threads;
    return RBIM_OK;
}

size_t rbim_grid_workspace_bytes(int64_t L, int ctas)
{
    if (L <= 32 || L > 65535 || ctas < 0) return 0;
    uint32_t C = (uint32_t)ctas;
    if (!C) C = rbim::grid_plan((uint32_t)L).C;
    if (!C) return 0;
    return rbim::grid_workspace_bytes((uint32_t)L, C);
}

int rbim_sweeps_grid(int64_t L, rbim_chain_t *chain, uint32_t *spin_pool, const uint32_t *coupling_pool,
                     int64_t *acc_int, double *acc_f64, int32_t *records, int n_sweeps, int32_t *status, int ctas,
                     int threads, int64_t wait_cycles, void *workspace, size_t workspace_bytes, void *stream)
{
    if (L <= 32 || L > 65535) return fail(RBIM_ERR_UNSUPPORTED, "grid engine: L = %lld outside 33..65535", (long long)L);
    if (n_sweeps < 0) return fail(RBIM_ERR_INVALID, "n_sweeps must be >= 0");
    if (ctas < 0 || threads < 0 || wait_cycles < 0) return fail(RBIM_ERR_INVALID, "negative plan or wait bound");
    if (n_sweeps == 0) return RBIM_OK;
    if (!chain || !spin_pool || !coupling_pool || !acc_int || !acc_f64 || !status || !workspace)
        return fail(RBIM_ERR_INVALID, "null pointer");
    rbim::GridPlan plan{(uint32_t)ctas, (uint32_t)threads};
    if (!ctas && !threads) plan = rbim::grid_plan((uint32_t)L);
    if (!plan.C) return fail(RBIM_ERR_UNSUPPORTED, "grid engine: no plan fits L = %lld", (long long)L);
    if (!rbim::grid_plan_ok((uint32_t)L, plan))
        return fail(RBIM_ERR_INVALID, "grid engine: plan (%d CTAs, %d threads) cannot run L = %lld", ctas, threads,
                    (long long)L);
    const size_t need = rbim::grid_workspace_bytes((uint32_t)L, plan.C);
    if (workspace_bytes < need) return fail(RBIM_ERR_INVALID, "workspace too small: %zu < %zu", workspace_bytes, need);
    if (((uintptr_t)workspace & 255u) != 0) return fail(RBIM_ERR_INVALID, "workspace must be 256-byte aligned");
    cudaError_t e = rbim::launch_grid_sweeps(chain, L, plan, spin_pool, coupling_pool, (long long *)acc_int, acc_f64,
                                             records, n_sweeps, status, workspace, (long long)wait_cycles,
                                             (cudaStream_t)stream);
    return cuda_check(e, "rbim_sweeps_grid");
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Plain sweeps with a static device scratch (rbim_sweeps_plain_noalloc).
//
// The plain engine's workspace for L <= RBIM_NOALLOC_MAX_L lives in one
// file-scope device array, so the entry point needs no caller workspace and
// allocates nothing itself.  Its device address is looked up on every call
// with cudaGetSymbolAddress, with the calling thread's current device
// current: the lookup is cheap once the module is loaded, and a cached
// address would go stale if the primary context were torn down and created
// again (cudaDeviceReset reloads the module at a new address).  The driver
// places the array when it loads this module on a device -- with lazy module
// loading, at the first call into the library on that device -- and that load
// needs about 2.25 MiB of free device memory.
// The scratch needs no clearing by anyone: every part of it the sweep reads
// is written earlier in the same call (k_plain_begin zeroes the seam plane
// and the scalar block, the phases rewrite the union-find words and the bit
// planes every sweep), exactly as for the caller-provided workspace of
// rbim_sweeps_plain, which may hold arbitrary bytes.
// ---------------------------------------------------------------------------
namespace {

constexpr int64_t kNoAllocMaxL = RBIM_NOALLOC_MAX_L;
// 2.25 MiB; rbim::plain_workspace_bytes(512) is 2,295,296 bytes.
constexpr size_t kNoAllocScratchBytes = size_t(2304) * 1024;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of the scratch on the current device.
int noalloc_scratch(void **out)
{
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_check(e, "rbim_sweeps_plain_noalloc: cudaGetSymbolAddress");
    if (!p || ((uintptr_t)p & 255u) != 0)
        return fail(RBIM_ERR_CUDA, "rbim_sweeps_plain_noalloc: scratch address %p is not 256-byte aligned", p);
    *out = p;
    return RBIM_OK;
}

}  // namespace

extern "C" {

int rbim_noalloc_max_l(void) { return (int)kNoAllocMaxL; }

int rbim_sweeps_plain_noalloc(int64_t L, rbim_chain_t *chain, uint32_t *spin_pool, const uint32_t *coupling_pool,
                              int64_t *acc_int, double *acc_f64, int32_t *records, int n_sweeps, int32_t *status,
                              void *stream)
{
    if (L < 3) return fail(RBIM_ERR_INVALID, "L must be at least 3 (got %lld)", (long long)L);
    if (L > kNoAllocMaxL)
        return fail(RBIM_ERR_UNSUPPORTED,
                    "rbim_sweeps_plain_noalloc: L = %lld exceeds the static scratch limit L <= %lld; use "
                    "rbim_sweeps_plain with a caller workspace",
                    (long long)L, (long long)kNoAllocMaxL);
    const size_t need = rbim::plain_workspace_bytes(L);
    if (need > kNoAllocScratchBytes)
        return fail(RBIM_ERR_UNSUPPORTED, "rbim_sweeps_plain_noalloc: L = %lld needs %zu scratch bytes > %zu",
                    (long long)L, need, kNoAllocScratchBytes);
    if (n_sweeps < 0) return fail(RBIM_ERR_INVALID, "n_sweeps must be >= 0");
    if (n_sweeps == 0) return RBIM_OK;
    if (!chain || !spin_pool || !coupling_pool || !acc_int || !acc_f64 || !status)
        return fail(RBIM_ERR_INVALID, "null pointer");
    void *scratch = nullptr;
    if (int rc = noalloc_scratch(&scratch)) return rc;
    cudaError_t e = rbim::launch_plain_sweeps(chain, spin_pool, coupling_pool, (long long *)acc_int, acc_f64,
                                              records, n_sweeps, status, scratch, L, (cudaStream_t)stream);
    return cuda_check(e, "rbim_sweeps_plain_noalloc");
}

}  // extern "C"

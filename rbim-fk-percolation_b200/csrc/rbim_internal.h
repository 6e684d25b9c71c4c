// Internal declarations shared by the CUDA translation units of librbim_sm100.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "rbim_sm100.h"

namespace rbim {

// Shared-memory layout of the resident engine for lattices of up to n_max
// sites (n_max <= 65536).
struct ResidentLayout {
    uint32_t n_max, nw_max, l_max, hs;
    size_t off_uf, off_S, off_JH, off_JV, off_OH, off_OV, off_FLIP, off_ROOT, off_RE, off_SEAMV, off_HK, off_HW,
        bytes;
};

ResidentLayout resident_layout(uint32_t l_max, int threads);

// Launchers (return cudaError_t of the launch).
cudaError_t launch_resident_sweeps(const rbim_chain_t *chains, int n_chains, int l_max, uint32_t *spin_pool,
                                   const uint32_t *coupling_pool, long long *acc_i, double *acc_f, int32_t *rec,
                                   int n_sweeps, int threads, int grid, int *queue, int *status,
                                   cudaStream_t stream);

cudaError_t launch_resident_label(int L, int n_lattices, const uint8_t *occ, int32_t *labels, int32_t *n_clusters,
                                  uint8_t *wraps, int threads, int *status, cudaStream_t stream);

size_t plain_workspace_bytes(int64_t L);
cudaError_t launch_plain_sweeps(rbim_chain_t *chain, uint32_t *spin_pool, const uint32_t *coupling_pool,
                                long long *acc_i, double *acc_f, int32_t *records, int n_sweeps, int *status,
                                void *workspace, int64_t L, cudaStream_t stream);
cudaError_t launch_plain_label(int64_t L, const uint8_t *occ, int32_t *labels, int32_t *n_clusters,
                               uint8_t *wraps, int *status, void *workspace, cudaStream_t stream);

int resident_max_l();
int resident_default_threads(int l_max);

// Cluster engine (one lattice per thread-block cluster of C CTAs, one tile of
// at most 65536 consecutive sites per CTA).
struct ClusterLayout {
    uint32_t l_max, C, t_max, tw, hs;
    size_t off_uf, off_S, off_OH, off_OV, off_FLIP, off_ROOT, off_YS, off_HK, off_HW, bytes;
};

// Tile size of an N-site lattice split over C CTAs: ceil(N / C) rounded up to
// a multiple of 128 sites, so that tiles start on Philox chunk boundaries.
__host__ __device__ constexpr uint32_t cluster_tile_size(uint32_t N, uint32_t C)
{
    const uint32_t t = (N + C - 1u) / C;
    return (t + 127u) & ~127u;
}

// C tiles fit an L x L lattice when every tile holds between L and `cap`
// sites.
__host__ __device__ constexpr bool cluster_tiles_ok(uint32_t L, uint32_t C, uint32_t cap = 65536u)
{
    const uint32_t N = L * L, T = cluster_tile_size(N, C);
    if (T > cap || T < L) return false;
    const uint32_t before = (C - 1u) * T;
    return before < N && N - before >= L;
}

// How a lattice of size L runs on the cluster engine: C CTAs of `threads`
// threads (1024 with tiles of up to 65536 sites, one CTA per SM; 512 with
// tiles of up to 32768 sites, two CTAs per SM).  C == 0: it does not.
struct ClusterPlan {
    uint32_t C, threads;
};
ClusterPlan cluster_plan(uint32_t L);
// A plan the engine can run an L x L lattice with (tiles fit, layout fits).
bool cluster_plan_ok(uint32_t L, ClusterPlan p);
uint32_t cluster_size_for(uint32_t L);
ClusterLayout cluster_layout(uint32_t l_max, uint32_t C);
bool cluster_layout_fits(const ClusterLayout &ly, uint32_t threads);
cudaError_t cluster_occupancy(uint32_t l_max, int *clusters);
cudaError_t cluster_occupancy_plan(uint32_t l_max, ClusterPlan plan, int *clusters);
cudaError_t launch_cluster_sweeps(const rbim_chain_t *chains, int n_chains, int l_max, uint32_t *spin_pool,
                                  const uint32_t *coupling_pool, long long *acc_i, double *acc_f, int32_t *rec,
                                  int n_sweeps, int *queue, int *status, cudaStream_t stream);
cudaError_t launch_cluster_sweeps_plan(const rbim_chain_t *chains, int n_chains, int l_max, ClusterPlan plan,
                                       uint32_t *spin_pool, const uint32_t *coupling_pool, long long *acc_i,
                                       double *acc_f, int32_t *rec, int n_sweeps, int *queue, int *status,
                                       cudaStream_t stream);


// Grid engine (one lattice over a cooperative grid of C CTAs, one tile of at
// most 65536 consecutive sites per CTA, tiles merged through global memory).
struct GridPlan {
    uint32_t C, threads;
};
GridPlan grid_plan(uint32_t L);
bool grid_plan_ok(uint32_t L, GridPlan p);
size_t grid_workspace_bytes(uint32_t L, uint32_t C);
cudaError_t launch_grid_sweeps(rbim_chain_t *chain, int64_t L, GridPlan plan, uint32_t *spin_pool,
                               const uint32_t *coupling_pool, long long *acc_i, double *acc_f, int32_t *records,
                               int n_sweeps, int *status, void *workspace, long long wait_cycles, cudaStream_t stream);

}  // namespace rbim

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

}  // namespace rbim

/*
 * rbim_sm100.h - C ABI of the B200 (sm_100a) Swendsen-Wang engine for the 2D
 * +-J random-bond Ising model.
 *
 * Every entry point takes plain device pointers owned by the caller, sizes and
 * a CUDA stream (passed as void*, NULL = legacy default stream), returns an
 * int status (RBIM_OK or a negative RBIM_ERR_* code; rbim_last_error() gives
 * the message of the calling thread's last failure) and launches work
 * asynchronously on that stream.  Hot entry points allocate nothing: scratch
 * memory is passed in by the caller, sized by the *_workspace_bytes queries.
 * Entry points are reentrant; calls on different streams with disjoint
 * buffers may overlap.
 *
 * Data layout ("linear bit planes"): site n = x*L + y of an L x L periodic
 * lattice (x slow, y fast; reference src/rbim/lattice.py:5-23) is bit n & 31 of
 * word n >> 5, with no row padding.  A plane of one lattice takes
 * rbim_plane_words(L) 32-bit words (ceil(L*L/32) rounded up to a multiple of
 * 4 so that planes stay 16-byte aligned); bits past L*L are zero.
 *   spin plane:     bit set <=> s = -1
 *   coupling pair:  JH plane (bond 2n, (x,y)->(x+1,y)) followed by the JV
 *                   plane (bond 2n+1, (x,y)->(x,y+1)); bit set <=> J = -1
 * Occupation masks at the labelling seam are bytes in the reference bond
 * order (2*L*L per lattice, bond 2n horizontal, 2n+1 vertical).
 *
 * Random numbers: Philox4x32-10 keyed by the chain key, counter
 * {block, sweep_lo, sweep_hi, stream}.
 *   stream 0, bonds: site n (chunk c = n >> 7, row s = (n >> 5) & 3, lane
 *     i = n & 31) reads word s of block 32*c + i; its low 16 bits draw the
 *     horizontal bond 2n, its high 16 bits the vertical bond 2n+1.
 *   stream 3, bond refinement: the same half of the same word of stream 3
 *     supplies the low 16 bits of a bond's 32-bit uniform, read only when the
 *     16-bit draw u equals thr >> 16; the uniform is (u << 16) | v.
 *   stream 1, cluster flips: the cluster whose smallest site is r flips iff
 *     bit r & 127 of block r >> 7 is set.
 *   stream 2, hot-start spins: site n is -1 iff bit n & 127 of block n >> 7
 *     (sweep 0) is set.
 * A bond is occupied iff satisfied (J s_i s_j = +1) and its 32-bit uniform is
 * < thr, where thr = floor((1 - exp(-2/T)) * 2^32) (0 <= thr <= 2^32).
 */
#ifndef RBIM_SM100_H
#define RBIM_SM100_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RBIM_ABI_VERSION 2

enum {
    RBIM_OK = 0,
    RBIM_ERR_INVALID = -1,     /* bad argument (size, pointer, alignment) */
    RBIM_ERR_CUDA = -2,        /* a CUDA runtime call failed */
    RBIM_ERR_UNSUPPORTED = -3  /* size outside what this entry point handles */
};

/* Status-word bits written by the kernels (device int32, OR-ed). */
enum {
    RBIM_STATUS_FIND_CAP = 1,  /* a union-find walk exceeded its bound */
    RBIM_STATUS_UNION_CAP = 2, /* a union retried beyond its bound */
    RBIM_STATUS_BAD_CHAIN = 4, /* a chain descriptor was out of range: L outside the call's range (or, on the
                                  plain path, different from the call's L), sweeps_per_bin < 1, n_bins < 0,
                                  n_therm < 0 or walk_cap < 0; the chain is skipped and left unchanged */
    RBIM_STATUS_GRID_WAIT = 8  /* grid engine: a CTA waited at a grid-wide barrier beyond its bound; every CTA
                                  then stops waiting and runs to its end, and the chain's state is undefined */
};

/*
 * One Markov chain: one disorder realization at one temperature, the unit of
 * work of the reference's run_single_realization (src/rbim/simulation.py:148-242).
 * All fields are 8 bytes; the struct is 96 bytes with no padding.
 */
typedef struct rbim_chain_t {
    uint64_t key;          /* Philox key of the chain */
    uint64_t thr;          /* activation threshold, see above */
    int64_t spin_off;      /* word offset of the chain's spin plane in the spin pool (multiple of 4) */
    int64_t coupling_off;  /* word offset of the chain's JH plane in the coupling pool (multiple of 4) */
    int64_t acc_off;       /* accumulator row of the chain's bin 0 */
    int64_t rec_off;       /* record row of the chain's measured sweep 0, or -1 for no records */
    uint64_t sweep;        /* absolute sweep counter of the chain; advanced by the sweep calls */
    int64_t n_therm;       /* sweeps 0 .. n_therm-1 are thermalisation (unmeasured) */
    int64_t n_bins;        /* measured sweeps are n_therm .. n_therm + n_bins*sweeps_per_bin - 1 */
    int64_t sweeps_per_bin;
    int64_t L;             /* linear size, 3 <= L */
    int64_t walk_cap;      /* 0: the default bounds.  > 0: a test hook that lowers the bound on one
                              union-find walk from N + 64 steps to walk_cap (and the per-thread loop
                              bounds to 64 walk_cap), so that a small lattice makes the bounds fire
                              and the call returns with RBIM_STATUS_FIND_CAP / _UNION_CAP set.  The
                              resident and plain engines honour it; the cluster engine keeps its own
                              bounds.  A chain run with a lowered cap has undefined results. */
} rbim_chain_t;

/*
 * Accumulators.  Row r of acc_int holds 12 int64 sums over the measured
 * sweeps of one bin, row r of acc_f64 holds 2 double sums, in this order:
 *   acc_int: E, E^2, M, |M|, M^2, S1, |M_C1|, S2, n_clusters, wrap_x, wrap_y, wrap_any
 *   acc_f64: M^4, |M_C1|/S1
 * (reference PRIMITIVES, src/rbim/simulation.py:56-71; per-bin means are the
 * sums divided by sweeps_per_bin).  Sweep calls add into the rows, so the
 * caller zeroes them before the first call.
 * Records (optional): 9 int32 per measured sweep:
 *   E, M, n_clusters, S1, |M_C1|, S2, |M_C2|, wrap_x, wrap_y
 * (the fields of the reference's SweepResult, src/rbim/swendsen_wang.py:24-53,
 * in order; S2 = |M_C2| = 0 when there is one cluster).  |M_C2| is computed
 * only for chains whose records are written.  Among clusters of equal size
 * the one with the smaller smallest site ranks first.
 */
#define RBIM_ACC_INT 12
#define RBIM_ACC_F64 2
#define RBIM_REC_LEN 9

/* Message of the calling thread's last failed call ("" if none). */
const char *rbim_last_error(void);

/* RBIM_ABI_VERSION of the loaded library. */
int rbim_abi_version(void);

/* Words of one bit plane for linear size L (ceil(L*L/32) rounded up to 4). */
int64_t rbim_plane_words(int64_t L);

/* Largest L the resident (on-chip) engine accepts. */
int rbim_resident_max_l(void);

/* CTA size (threads) the resident engine uses for lattices of up to L x L
 * sites when rbim_sweeps_batched is called with threads = 0 (0 if L is out of
 * range): small CTAs while several fit an SM. */
int rbim_resident_threads(int64_t L);

/*
 * Initial spins of n_chains chains (reference initial_spins,
 * src/rbim/swendsen_wang.py:56-78): hot != 0 draws Philox stream 2 of each
 * chain's key, hot == 0 sets every spin to +1.  chains is a device array.
 */
int rbim_init_spins(const rbim_chain_t *chains, int n_chains, uint32_t *spin_pool, int hot, void *stream);

/*
 * Bond activation of one lattice (reference activate_bonds,
 * src/rbim/clusters.py:48-79, with the Philox stream in place of numpy's
 * generator): writes 2*L*L occupation bytes in bond order.  couplings is the
 * JH plane followed by the JV plane.  Runs the same activation code as the
 * sweep engines; workspace: rbim_activate_workspace_bytes(L).
 */
size_t rbim_activate_workspace_bytes(int64_t L);
int rbim_activate(int64_t L, const uint32_t *spins, const uint32_t *couplings, uint64_t key, uint64_t thr,
                  uint64_t sweep, uint8_t *occ, void *workspace, size_t workspace_bytes, void *stream);

/*
 * Cluster labelling with exact wrapping of n_lattices frozen occupation masks
 * of the same L (reference label_and_wrap, src/rbim/clusters.py:144-159 and
 * src/rbim/_unionfind.py:91-136).  occ: n_lattices * 2*L*L bytes (nonzero =
 * occupied).  labels: n_lattices * L*L int32, the canonical labels (clusters
 * numbered in order of their smallest site).  n_clusters: n_lattices int32.
 * wraps: n_lattices * 2 bytes (wrap_x, wrap_y).  status: device int32.
 * Lattices with L <= rbim_resident_max_l() run on chip and need no workspace;
 * larger ones use rbim_label_wrap_workspace_bytes(L) bytes of workspace.
 */
size_t rbim_label_wrap_workspace_bytes(int64_t L);
int rbim_label_wrap(int64_t L, int n_lattices, const uint8_t *occ, int32_t *labels, int32_t *n_clusters,
                    uint8_t *wraps, int32_t *status, void *workspace, size_t workspace_bytes, void *stream);

/*
 * Batched resident sweeps: every chain of the device array `chains` advances
 * by up to n_sweeps sweeps (fewer when it reaches the end of its run), with
 * one lattice per CTA held in shared memory for the whole call, fed by a
 * persistent work queue.  The chains may have different L (all <= l_max <=
 * rbim_resident_max_l()).  This is the engine behind many calls of the
 * reference's run_single_realization (src/rbim/simulation.py:196-242) and
 * sw_sweep (src/rbim/swendsen_wang.py:103-172).  records may be NULL.
 * threads: CTA size, 32, 64, 128, 256, 512 or 1024 (0 = rbim_resident_threads(l_max)).
 * workspace: rbim_batched_workspace_bytes()
 * bytes (the work-queue counter).
 */
size_t rbim_batched_workspace_bytes(void);
int rbim_sweeps_batched(rbim_chain_t *chains, int n_chains, int64_t l_max, uint32_t *spin_pool,
                        const uint32_t *coupling_pool, int64_t *acc_int, double *acc_f64, int32_t *records,
                        int n_sweeps, int threads, int32_t *status, void *workspace, size_t workspace_bytes,
                        void *stream);

/*
 * Batched sweeps of lattices too large for one CTA: every chain of `chains`
 * (rbim_resident_max_l() < L <= l_max <= rbim_cluster_max_l()) advances by up
 * to n_sweeps sweeps, one lattice per thread-block cluster.  The cluster's
 * CTAs each hold one tile of at most 65536 consecutive sites in shared memory
 * for the whole call and merge the clusters that cross tile boundaries or
 * the periodic seams through distributed shared memory.  Same chain,
 * accumulator and record contract (and the same results, bit for bit) as
 * rbim_sweeps_batched; workspace: rbim_batched_workspace_bytes() bytes.
 * rbim_cluster_max_l() depends on the current device (0 when no cluster can
 * be scheduled).
 */
int rbim_cluster_max_l(void);
/* CTAs per cluster the cluster engine uses for an L x L lattice (0 if none). */
int rbim_cluster_size(int64_t L);
/* Threads per CTA of that plan (512 with half-size tiles or 1024; 0 if none).
 * A call of rbim_sweeps_clustered runs every lattice in the plan of its l_max,
 * so callers that mix sizes group lattices by (rbim_cluster_size,
 * rbim_cluster_threads). */
int rbim_cluster_threads(int64_t L);
int rbim_sweeps_clustered(rbim_chain_t *chains, int n_chains, int64_t l_max, uint32_t *spin_pool,
                          const uint32_t *coupling_pool, int64_t *acc_int, double *acc_f64, int32_t *records,
                          int n_sweeps, int32_t *status, void *workspace, size_t workspace_bytes, void *stream);

/*
 * Launch plans of the cluster engine, for a tuner.  A plan is the number of
 * CTAs per cluster (tiles per lattice) and the CTA size (512: tiles of at
 * most 32768 sites, two CTAs per SM; 1024: at most 65536 sites, one per SM).
 * rbim_cluster_plans writes the plans that can run an L x L lattice on the
 * current device (tiles and shared memory fit, and at least one cluster can
 * be scheduled) into ctas[i], threads[i] for i < max_plans -- the plan
 * rbim_sweeps_clustered uses first -- and returns how many there are (0
 * outside the engine's range).  rbim_sweeps_clustered_plan is
 * rbim_sweeps_clustered with an explicit plan, which must be one of
 * rbim_cluster_plans(l_max) (RBIM_ERR_INVALID otherwise); a lattice of the
 * call that the plan cannot run is rejected with RBIM_STATUS_BAD_CHAIN.
 * Results do not depend on the plan: tiles start on 128-site chunk
 * boundaries, so every plan draws the same Philox numbers.  Same reference
 * correspondence as rbim_sweeps_clustered (src/rbim/simulation.py:196-242,
 * many tasks at once).
 */
int rbim_cluster_plans(int64_t L, int *ctas, int *threads, int max_plans);
int rbim_sweeps_clustered_plan(rbim_chain_t *chains, int n_chains, int64_t l_max, int cluster_ctas, int threads,
                               uint32_t *spin_pool, const uint32_t *coupling_pool, int64_t *acc_int, double *acc_f64,
                               int32_t *records, int n_sweeps, int32_t *status, void *workspace,
                               size_t workspace_bytes, void *stream);

/*
 * Plain sweeps of one chain (device descriptor `chain`) through the
 * global-memory engine: one lattice per launch sequence, any L >= 3, the
 * drop-in for one run_single_realization task.  L must equal chain->L.  Same
 * accumulator and record contract as rbim_sweeps_batched.  workspace:
 * rbim_plain_workspace_bytes(L).
 */
size_t rbim_plain_workspace_bytes(int64_t L);
int rbim_sweeps_plain(int64_t L, rbim_chain_t *chain, uint32_t *spin_pool, const uint32_t *coupling_pool, int64_t *acc_int,
                      double *acc_f64, int32_t *records, int n_sweeps, int32_t *status, void *workspace,
                      size_t workspace_bytes, void *stream);

/*
 * Grid sweeps of one chain (device descriptor `chain`): one lattice over the
 * whole GPU in a single cooperative launch per call, the drop-in for one
 * run_single_realization task (src/rbim/simulation.py:196-242) for
 * 32 < L <= about 3000.  The launch's C CTAs each keep one tile of at most
 * 65536 consecutive sites in shared memory for every sweep of the call; the
 * clusters that cross tile boundaries or the periodic seams are merged in a
 * union-find in global memory between grid-wide barriers.  L must equal
 * chain->L.  Same accumulator and record contract (and the same results, bit
 * for bit) as rbim_sweeps_plain.
 *
 * A plan is (ctas, threads): ctas tiles, threads per CTA (256, 512 or 1024).
 * rbim_grid_plan writes the default plan for the current device (one
 * 1024-thread CTA per SM, fewer CTAs when tiles would hold fewer than L
 * sites) and returns RBIM_OK, or RBIM_ERR_UNSUPPORTED when no plan fits L.
 * rbim_grid_workspace_bytes(L, ctas) is the workspace a plan of `ctas` CTAs
 * needs (ctas = 0: the default plan's); it holds one 8-byte union-find word
 * per site.  rbim_sweeps_grid takes ctas = threads = 0 for the default plan.
 * The whole grid must be resident at once: a plan with more CTAs than the
 * device holds returns RBIM_ERR_CUDA (cudaErrorCooperativeLaunchTooLarge).
 *
 * Every wait at a grid-wide barrier gives up after wait_cycles SM clock
 * cycles (0: about one second) and sets RBIM_STATUS_GRID_WAIT; the launch
 * then runs to its end without waiting again and the chain's state is
 * undefined.  Calls sharing a workspace must be ordered (one stream).
 */
int rbim_grid_plan(int64_t L, int *ctas, int *threads);
size_t rbim_grid_workspace_bytes(int64_t L, int ctas);
int rbim_sweeps_grid(int64_t L, rbim_chain_t *chain, uint32_t *spin_pool, const uint32_t *coupling_pool,
                     int64_t *acc_int, double *acc_f64, int32_t *records, int n_sweeps, int32_t *status, int ctas,
                     int threads, int64_t wait_cycles, void *workspace, size_t workspace_bytes, void *stream);

/*
 * rbim_sweeps_plain without a caller workspace.  No counterpart in the
 * reference (its sweep is numba on the host); this is an addition for callers
 * that cannot allocate device memory: an FFI host that holds only the data
 * buffers another runtime handed it and no device allocator of its own, or a
 * caller whose device memory is all reserved by a pooling allocator, where a
 * cudaMalloc would fail (and a cudaFree would synchronise the device).
 *
 * Same arguments, results and accumulator/record contract as
 * rbim_sweeps_plain, minus workspace and workspace_bytes: the scratch is one
 * static device array of 2.25 MiB per device inside the library, enough for
 * L <= RBIM_NOALLOC_MAX_L.  Larger L is rejected with RBIM_ERR_UNSUPPORTED
 * and a message naming the limit.  The call itself allocates nothing, and
 * calls no allocating routine of any library (see the set-up note below for
 * the one-time placement of the array).
 *
 * Every call looks up the array's device address on the calling thread's
 * current device with cudaGetSymbolAddress (cheap once the library's device
 * code is loaded, and never stale across a cudaDeviceReset).  The driver
 * places the array when it loads the library's device code on a device --
 * with lazy module loading, the default, that happens at the first call into
 * the library on that device (this one, rbim_init_spins or any other) -- and
 * that load needs about 2.25 MiB of free device memory: make the first call
 * on each device before a pooling allocator reserves the device's memory,
 * and before any stream capture begins.  Nothing has to start at zero: the
 * call initialises every part of the scratch it reads.  The scratch is shared by all calls on a
 * device, so two calls that overlap on the device (different streams, or
 * different host threads, without ordering between them) race on it and give
 * wrong results; order them on one stream or serialise them.
 */
#define RBIM_NOALLOC_MAX_L 512
int rbim_noalloc_max_l(void);
int rbim_sweeps_plain_noalloc(int64_t L, rbim_chain_t *chain, uint32_t *spin_pool, const uint32_t *coupling_pool,
                              int64_t *acc_int, double *acc_f64, int32_t *records, int n_sweeps, int32_t *status,
                              void *stream);

#ifdef __cplusplus
}
#endif

#endif /* RBIM_SM100_H */

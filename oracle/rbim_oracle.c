/*
 * CPU oracle for the Swendsen-Wang sweep of the 2D +-J random-bond Ising model.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA engine is
 * compared against; it is never part of the product path.  Only the test suite,
 * the smoke check and the CPU-baseline leg of the benchmark load it.
 *
 * It restates, in plain C, the reference algorithm of
 * Amirhossein-Manouchehri/rbim-fk-percolation:
 *
 *   lattice geometry ............ src/rbim/lattice.py:89-135   (build_lattice)
 *   bond activation ............. src/rbim/clusters.py:48-79   (activate_bonds)
 *   union-find + wrapping ....... src/rbim/_unionfind.py:59-136 (_find, _label_and_wrap)
 *   cluster flip ................ src/rbim/swendsen_wang.py:140-141
 *   cluster statistics .......... src/rbim/clusters.py:98-118  (cluster_statistics)
 *   two largest clusters ........ src/rbim/swendsen_wang.py:92-100 (_two_largest)
 *   energy / magnetization ...... src/rbim/swendsen_wang.py:81-89
 *   per-sweep record ............ src/rbim/swendsen_wang.py:143-172 (sw_sweep)
 *   primitive accumulation ...... src/rbim/simulation.py:196-242 (run_single_realization)
 *
 * with one deliberate substitution: the reference draws its uniforms from
 * numpy's PCG64 generator, which is not reproduced.  Every random number here
 * comes from the counter-based Philox4x32-10 stream that the CUDA engine uses
 * (Salmon, Moraes, Dror and Shaw, "Parallel random numbers: as easy as 1, 2,
 * 3", SC'11), so a whole chain can be replayed bit for bit:
 *
 *   key     = 64-bit chain key, low word key[0], high word key[1]
 *   bond k of sweep t   : site n = k >> 1, direction d = k & 1 (0 horizontal,
 *                         1 vertical).  Sites come in chunks of 128; site n is
 *                         lane i = n & 31 of row s = (n >> 5) & 3 of chunk
 *                         n >> 7, and uses Philox block
 *                         b = 32 * (n >> 7) + i, word s, half d (low half for
 *                         d = 0).  Its 32-bit uniform is (u << 16) | v, with u
 *                         that half of Philox(ctr = {b, t_lo, t_hi, 0}) and v
 *                         the same half of Philox(ctr = {b, t_lo, t_hi, 3}).
 *                         Occupied iff satisfied and uniform < thr, where
 *                         thr = floor(p_add * 2^32), p_add = -expm1(-2 beta).
 *                         (The engine draws v only when u == thr >> 16.)
 *   flip of the cluster whose smallest site is r, sweep t :
 *                         bit (r & 127) of Philox(ctr = {r >> 7, t_lo, t_hi, 1})
 *   hot-start spin of site n : bit (n & 127) of Philox(ctr = {n >> 7, 0, 0, 2});
 *                         a set bit means s = -1
 *
 * Bits of a 128-bit Philox output are numbered little-endian: bit b lives in
 * word b >> 5 at position b & 31.
 *
 * Tie rule of the two-largest selection: the reference uses numpy.argpartition,
 * whose choice among equal sizes is implementation-defined.  This oracle (and
 * the engine) pick the cluster with the smallest canonical label among equal
 * sizes, i.e. the one whose smallest site comes first.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------ */
/* Philox4x32-10                                                              */
/* ------------------------------------------------------------------------ */

#define ORC_PHILOX_M0 0xD2511F53u
#define ORC_PHILOX_M1 0xCD9E8D57u
#define ORC_PHILOX_W0 0x9E3779B9u
#define ORC_PHILOX_W1 0xBB67AE85u

void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int round = 0; round < 10; ++round) {
        if (round > 0) {
            k0 += ORC_PHILOX_W0;
            k1 += ORC_PHILOX_W1;
        }
        uint64_t p0 = (uint64_t)ORC_PHILOX_M0 * (uint64_t)c0;
        uint64_t p1 = (uint64_t)ORC_PHILOX_M1 * (uint64_t)c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
    }
    out[0] = c0;
    out[1] = c1;
    out[2] = c2;
    out[3] = c3;
}

static void philox_stream(uint64_t key, uint64_t block, uint64_t sweep, uint32_t stream, uint32_t out[4])
{
    uint32_t ctr[4] = {(uint32_t)block, (uint32_t)sweep, (uint32_t)(sweep >> 32), stream};
    uint32_t k[2] = {(uint32_t)key, (uint32_t)(key >> 32)};
    orc_philox4x32_10(ctr, k, out);
}

static inline uint64_t bond_block(uint64_t site) { return ((site >> 7) << 5) | (site & 31); }

uint32_t orc_bond_uniform(uint64_t key, uint64_t sweep, uint64_t bond)
{
    uint32_t hi[4], lo[4];
    const uint64_t n = bond >> 1;
    const unsigned s = (unsigned)((n >> 5) & 3), d = (unsigned)(bond & 1);
    philox_stream(key, bond_block(n), sweep, 0u, hi);
    philox_stream(key, bond_block(n), sweep, 3u, lo);
    const uint32_t u = (hi[s] >> (16 * d)) & 0xFFFFu;
    const uint32_t v = (lo[s] >> (16 * d)) & 0xFFFFu;
    return (u << 16) | v;
}

int orc_flip_bit(uint64_t key, uint64_t sweep, uint64_t root)
{
    uint32_t out[4];
    philox_stream(key, root >> 7, sweep, 1u, out);
    return (int)((out[(root >> 5) & 3] >> (root & 31)) & 1u);
}

int orc_hot_spin_bit(uint64_t key, uint64_t site)
{
    uint32_t out[4];
    philox_stream(key, site >> 7, 0, 2u, out);
    return (int)((out[(site >> 5) & 3] >> (site & 31)) & 1u);
}

/* ------------------------------------------------------------------------ */
/* Lattice geometry (lattice.py:89-135): site n = x*L + y, bond 2n is       */
/* (x,y)->(x+1,y) with displacement (1,0), bond 2n+1 is (x,y)->(x,y+1)      */
/* with displacement (0,1); both directions periodic.                       */
/* ------------------------------------------------------------------------ */

static inline int64_t bond_end_b(int64_t L, int64_t k)
{
    int64_t n = k >> 1;
    int64_t x = n / L, y = n % L;
    if ((k & 1) == 0)
        return ((x + 1) % L) * L + y;
    return x * L + (y + 1) % L;
}

/* ------------------------------------------------------------------------ */
/* Bond activation (clusters.py:48-79)                                       */
/* ------------------------------------------------------------------------ */

/* Bonds are taken eight at a time (one Philox block: the two bonds of the
 * four sites 128c + 32s + i, s = 0..3); the low halves come from the second
 * stream only when some satisfied bond's high half equals thr >> 16, which
 * yields the same decisions as comparing every bond's full orc_bond_uniform
 * with thr. */
void orc_activate(int64_t L, const int8_t *spins, const int8_t *J, uint64_t key, uint64_t thr,
                  uint64_t sweep, uint8_t *occ)
{
    const int64_t n_sites = L * L;
    const uint32_t thr_hi = (uint32_t)(thr >> 16);
    for (int64_t c = 0; c * 128 < n_sites; ++c) {
        for (int64_t i = 0; i < 32; ++i) {
            uint32_t hi[4], lo[4];
            int have_lo = 0;
            philox_stream(key, (uint64_t)(32 * c + i), sweep, 0u, hi);
            for (int s = 0; s < 4; ++s) {
                const int64_t n = 128 * c + 32 * s + i;
                if (n >= n_sites)
                    continue;
                for (int d = 0; d < 2; ++d) {
                    const int64_t k = 2 * n + d;
                    int64_t b = bond_end_b(L, k);
                    int satisfied = (int)J[k] * (int)spins[n] * (int)spins[b] > 0;
                    const uint32_t u = (hi[s] >> (16 * d)) & 0xFFFFu;
                    int on = 0;
                    if (satisfied) {
                        if (thr >= (1ull << 32) || u < thr_hi) {
                            on = 1;
                        } else if (u == thr_hi) {
                            if (!have_lo) {
                                philox_stream(key, (uint64_t)(32 * c + i), sweep, 3u, lo);
                                have_lo = 1;
                            }
                            const uint32_t v = (lo[s] >> (16 * d)) & 0xFFFFu;
                            on = ((u << 16) | v) < thr;
                        }
                    }
                    occ[k] = (uint8_t)on;
                }
            }
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Union-find with displacement (_unionfind.py:59-136)                       */
/* ------------------------------------------------------------------------ */

static inline int64_t uf_find(int64_t *parent, int64_t *rx, int64_t *ry, int64_t start, int64_t *ox,
                              int64_t *oy)
{
    int64_t root = start, ax = 0, ay = 0;
    while (parent[root] != root) {
        ax += rx[root];
        ay += ry[root];
        root = parent[root];
    }
    int64_t node = start, bx = 0, by = 0;
    while (parent[node] != node) {
        int64_t next = parent[node];
        int64_t old_x = rx[node], old_y = ry[node];
        parent[node] = root;
        rx[node] = ax - bx;
        ry[node] = ay - by;
        bx += old_x;
        by += old_y;
        node = next;
    }
    *ox = ax;
    *oy = ay;
    return root;
}

/* Returns n_clusters; writes canonical labels (rank of each cluster's
 * smallest site) and the two wrap flags. */
int64_t orc_label_and_wrap(int64_t L, const uint8_t *occ, int64_t *labels, int32_t *wrap_x,
                           int32_t *wrap_y)
{
    int64_t n = L * L;
    int64_t *parent = (int64_t *)malloc(sizeof(int64_t) * n);
    int64_t *rx = (int64_t *)calloc((size_t)n, sizeof(int64_t));
    int64_t *ry = (int64_t *)calloc((size_t)n, sizeof(int64_t));
    int64_t *remap = (int64_t *)malloc(sizeof(int64_t) * n);
    for (int64_t i = 0; i < n; ++i) {
        parent[i] = i;
        remap[i] = -1;
    }
    int wx = 0, wy = 0;
    for (int64_t k = 0; k < 2 * n; ++k) {
        if (!occ[k])
            continue;
        int64_t a = k >> 1, b = bond_end_b(L, k);
        int64_t ex = (k & 1) ? 0 : 1, ey = (k & 1) ? 1 : 0;
        int64_t ax, ay, bx, by;
        int64_t root_a = uf_find(parent, rx, ry, a, &ax, &ay);
        int64_t root_b = uf_find(parent, rx, ry, b, &bx, &by);
        if (root_a != root_b) {
            parent[root_b] = root_a;
            rx[root_b] = ax - ex - bx;
            ry[root_b] = ay - ey - by;
        } else {
            if (ex + bx - ax != 0)
                wx = 1;
            if (ey + by - ay != 0)
                wy = 1;
        }
    }
    int64_t n_clusters = 0;
    for (int64_t site = 0; site < n; ++site) {
        int64_t dx, dy;
        int64_t root = uf_find(parent, rx, ry, site, &dx, &dy);
        if (remap[root] == -1)
            remap[root] = n_clusters++;
        labels[site] = remap[root];
    }
    free(parent);
    free(rx);
    free(ry);
    free(remap);
    *wrap_x = wx;
    *wrap_y = wy;
    return n_clusters;
}

/* ------------------------------------------------------------------------ */
/* Cluster statistics, two largest, energy, magnetization                    */
/* ------------------------------------------------------------------------ */

void orc_cluster_statistics(int64_t n_sites, const int64_t *labels, const int8_t *spins,
                            int64_t n_clusters, int64_t *sizes, int64_t *mags)
{
    memset(sizes, 0, sizeof(int64_t) * (size_t)n_clusters);
    memset(mags, 0, sizeof(int64_t) * (size_t)n_clusters);
    for (int64_t i = 0; i < n_sites; ++i) {
        sizes[labels[i]] += 1;
        mags[labels[i]] += spins[i];
    }
}

/* first = smallest label among the largest size; second = smallest label
 * among the largest size of the remaining clusters, or -1 for one cluster. */
void orc_two_largest(const int64_t *sizes, int64_t n_clusters, int64_t *first, int64_t *second)
{
    int64_t f = 0;
    for (int64_t c = 1; c < n_clusters; ++c)
        if (sizes[c] > sizes[f])
            f = c;
    int64_t s = -1;
    for (int64_t c = 0; c < n_clusters; ++c) {
        if (c == f)
            continue;
        if (s < 0 || sizes[c] > sizes[s])
            s = c;
    }
    *first = f;
    *second = s;
}

int64_t orc_energy(int64_t L, const int8_t *spins, const int8_t *J)
{
    int64_t e = 0;
    for (int64_t k = 0; k < 2 * L * L; ++k)
        e += (int64_t)J[k] * spins[k >> 1] * spins[bond_end_b(L, k)];
    return -e;
}

int64_t orc_magnetization(int64_t n_sites, const int8_t *spins)
{
    int64_t m = 0;
    for (int64_t i = 0; i < n_sites; ++i)
        m += spins[i];
    return m;
}

/* ------------------------------------------------------------------------ */
/* One sweep (swendsen_wang.py:103-172)                                      */
/* ------------------------------------------------------------------------ */

/* Per-sweep record layout (int64):
 *   [0] energy  [1] magnetization  [2] n_clusters
 *   [3] largest_size  [4] largest_abs_magnetization
 *   [5] second_size   [6] second_abs_magnetization
 *   [7] wraps_x  [8] wraps_y
 */
enum { ORC_REC_LEN = 9 };

typedef struct {
    int64_t L, n;
    uint8_t *occ;
    int64_t *labels, *sizes, *mags, *minsite;
    int8_t *flip;
} orc_ws;

static void ws_init(orc_ws *w, int64_t L)
{
    w->L = L;
    w->n = L * L;
    w->occ = (uint8_t *)malloc((size_t)(2 * w->n));
    w->labels = (int64_t *)malloc(sizeof(int64_t) * (size_t)w->n);
    w->sizes = (int64_t *)malloc(sizeof(int64_t) * (size_t)w->n);
    w->mags = (int64_t *)malloc(sizeof(int64_t) * (size_t)w->n);
    w->minsite = (int64_t *)malloc(sizeof(int64_t) * (size_t)w->n);
    w->flip = (int8_t *)malloc((size_t)w->n);
}

static void ws_free(orc_ws *w)
{
    free(w->occ);
    free(w->labels);
    free(w->sizes);
    free(w->mags);
    free(w->minsite);
    free(w->flip);
}

static void sweep_ws(orc_ws *w, int8_t *spins, const int8_t *J, uint64_t key, uint64_t thr,
                     uint64_t sweep, int measure, int64_t *rec)
{
    int64_t L = w->L, n = w->n;
    orc_activate(L, spins, J, key, thr, sweep, w->occ);
    int32_t wx, wy;
    int64_t ncl = orc_label_and_wrap(L, w->occ, w->labels, &wx, &wy);

    /* Canonical labels are ranks of the smallest site, so the first site met
     * with a new label is that cluster's smallest site; the flip of the
     * cluster is keyed by it. */
    for (int64_t c = 0; c < ncl; ++c)
        w->minsite[c] = -1;
    for (int64_t i = 0; i < n; ++i)
        if (w->minsite[w->labels[i]] < 0)
            w->minsite[w->labels[i]] = i;
    for (int64_t c = 0; c < ncl; ++c)
        w->flip[c] = (int8_t)orc_flip_bit(key, sweep, (uint64_t)w->minsite[c]);
    for (int64_t i = 0; i < n; ++i)
        if (w->flip[w->labels[i]])
            spins[i] = (int8_t)-spins[i];

    if (!measure)
        return;
    orc_cluster_statistics(n, w->labels, spins, ncl, w->sizes, w->mags);
    int64_t first, second;
    orc_two_largest(w->sizes, ncl, &first, &second);
    rec[0] = orc_energy(L, spins, J);
    rec[1] = orc_magnetization(n, spins);
    rec[2] = ncl;
    rec[3] = w->sizes[first];
    rec[4] = llabs(w->mags[first]);
    rec[5] = second >= 0 ? w->sizes[second] : 0;
    rec[6] = second >= 0 ? llabs(w->mags[second]) : 0;
    rec[7] = wx;
    rec[8] = wy;
}

void orc_sw_sweep(int64_t L, int8_t *spins, const int8_t *J, uint64_t key, uint64_t thr,
                  uint64_t sweep, int measure, int64_t *rec)
{
    orc_ws w;
    ws_init(&w, L);
    sweep_ws(&w, spins, J, key, thr, sweep, measure, rec);
    ws_free(&w);
}

void orc_initial_spins(int64_t n_sites, uint64_t key, int hot, int8_t *spins)
{
    for (int64_t i = 0; i < n_sites; ++i)
        spins[i] = hot ? (int8_t)(orc_hot_spin_bit(key, (uint64_t)i) ? -1 : 1) : (int8_t)1;
}

/* ------------------------------------------------------------------------ */
/* One chain (simulation.py:196-242): thermalise, then accumulate per bin.   */
/* ------------------------------------------------------------------------ */

/* Per-bin integer sums (int64), in this order:
 *   E, E^2, M, |M|, M^2, S1, |M_C1|, S2, n_clusters, wrap_x, wrap_y, wrap_any
 * Per-bin floating sums (double): M^4, |M_C1|/S1.
 * The sweep counter of measured sweep i of the chain is sweep0 + n_therm + i;
 * thermalisation sweeps use sweep0 .. sweep0 + n_therm - 1. */
enum { ORC_NI = 12, ORC_NF = 2 };

void orc_accumulate(const int64_t *rec, int64_t *ib, double *fb)
{
    int64_t e = rec[0], m = rec[1];
    int64_t am = m < 0 ? -m : m;
    ib[0] += e;
    ib[1] += e * e;
    ib[2] += m;
    ib[3] += am;
    ib[4] += m * m;
    ib[5] += rec[3];
    ib[6] += rec[4];
    ib[7] += rec[5];
    ib[8] += rec[2];
    ib[9] += rec[7];
    ib[10] += rec[8];
    ib[11] += (rec[7] | rec[8]) ? 1 : 0;
    double m2 = (double)(m * m);
    fb[0] += m2 * m2;
    fb[1] += rec[3] > 0 ? (double)rec[4] / (double)rec[3] : 0.0;
}

void orc_run_chain(int64_t L, const int8_t *J, uint64_t key, uint64_t thr, int hot,
                   uint64_t sweep0, int64_t n_therm, int64_t n_bins, int64_t sweeps_per_bin,
                   int8_t *spins, int init_spins, int64_t *int_bins, double *f_bins)
{
    orc_ws w;
    ws_init(&w, L);
    if (init_spins)
        orc_initial_spins(L * L, key, hot, spins);
    uint64_t t = sweep0;
    int64_t rec[ORC_REC_LEN];
    for (int64_t i = 0; i < n_therm; ++i)
        sweep_ws(&w, spins, J, key, thr, t++, 0, rec);
    memset(int_bins, 0, sizeof(int64_t) * (size_t)(n_bins * ORC_NI));
    memset(f_bins, 0, sizeof(double) * (size_t)(n_bins * ORC_NF));
    for (int64_t b = 0; b < n_bins; ++b)
        for (int64_t i = 0; i < sweeps_per_bin; ++i) {
            sweep_ws(&w, spins, J, key, thr, t++, 1, rec);
            orc_accumulate(rec, int_bins + b * ORC_NI, f_bins + b * ORC_NF);
        }
    ws_free(&w);
}

/* Many independent chains of one lattice size, one chain per thread.  Used
 * as the timed CPU baseline; n_threads <= 0 means all available threads.
 * Chain c uses couplings J + c * 2N, key keys[c], threshold thrs[c], spins
 * spins + c * N, and writes its bins at int_bins + c * n_bins * 12 and
 * f_bins + c * n_bins * 2.  Returns the number of threads used. */
int orc_run_chains(int64_t n_chains, int64_t L, const int8_t *J, const uint64_t *keys,
                   const uint64_t *thrs, int hot, uint64_t sweep0, int64_t n_therm, int64_t n_bins,
                   int64_t sweeps_per_bin, int8_t *spins, int init_spins, int64_t *int_bins,
                   double *f_bins, int n_threads)
{
    int used = 1;
#ifdef _OPENMP
    if (n_threads <= 0)
        n_threads = omp_get_max_threads();
    used = n_threads;
#pragma omp parallel for schedule(dynamic, 1) num_threads(n_threads)
#endif
    for (int64_t c = 0; c < n_chains; ++c) {
        int64_t n = L * L;
        orc_run_chain(L, J + c * 2 * n, keys[c], thrs[c], hot, sweep0, n_therm, n_bins,
                      sweeps_per_bin, spins + c * n, init_spins, int_bins + c * n_bins * ORC_NI,
                      f_bins + c * n_bins * ORC_NF);
    }
    return used;
}

/* Bit-exact labelling of many frozen occupation masks, one mask per thread
 * (used to time the labelling leg on the host).  Mask m is occ + m * 2N. */
int orc_label_many(int64_t n_masks, int64_t L, const uint8_t *occ, int64_t *n_clusters,
                   int32_t *wraps, int n_threads)
{
    int used = 1;
#ifdef _OPENMP
    if (n_threads <= 0)
        n_threads = omp_get_max_threads();
    used = n_threads;
#pragma omp parallel for schedule(dynamic, 1) num_threads(n_threads)
#endif
    for (int64_t m = 0; m < n_masks; ++m) {
        int64_t n = L * L;
        int64_t *labels = (int64_t *)malloc(sizeof(int64_t) * (size_t)n);
        n_clusters[m] = orc_label_and_wrap(L, occ + m * 2 * n, labels, wraps + 2 * m, wraps + 2 * m + 1);
        free(labels);
    }
    return used;
}

/*
 * qem.h -- C-ABI of the B200-native QEM (Quasi-Ewald Method) force/energy
 * library, libqem.so.  Plain C types only: pointers, sizes, a POD parameter
 * struct and an opaque handle.  Julia binds it with ccall, Python with ctypes;
 * the torch.autograd.Function in qem4molly_b200 is a thin layer over it.
 *
 * Reference interfaces replaced (paths inside ArrogantGao/QEM4Molly):
 *   QEM_short(L, r_cutoff, alpha; iter_period, gamma_1, gamma_2, eps_0,
 *             accuracy, N_t)                        src/QEM_short.jl:19-25
 *   QEM_long(L; k_cutoff, z_list, gamma_1, gamma_2, eps_0, accuracy, alpha,
 *            rbe_mode, rbe_p)                       src/QEM_long.jl:19-30
 *   QEM_inter(n_atoms, L; s, accuracy, rbe_mode, rbe_p, eps_0, gamma_1,
 *             gamma_2, N_t, iter_period)            src/Quasi_Ewald_Method.jl:3-24
 *   Substrate_LJ(; cutoff, sigma, eps, sub_pos, direction)
 *                                                   src/Substrate_LJ.jl:15-17
 *   Molly.forces(inter::QEM_short, sys, nb)         src/QEM_short.jl:27-59
 *   Molly.forces(inter::QEM_long, sys, nb)          src/QEM_long.jl:32-44
 *   Molly.forces(inter::Substrate_LJ, sys, nb)      src/Substrate_LJ.jl:24-46
 *   K_set_generator(L_x, L_y, alpha, accuracy) + StatsBase.sample
 *                                                   src/K_set_generator.jl:5-45,
 *                                                   src/Force_long.jl:235
 *   Energy_short / Energy_long (python_lib; the Julia package has no energy)
 *                                                   src/python_lib/Energy_short_range_njit.py:84-99,
 *                                                   src/python_lib/Energy_long_range_njit.py:10-44
 *
 * Conventions
 *   - Coordinates are 3N doubles, particle-major (x0 y0 z0 x1 ...), which is
 *     exactly reinterpret(Float64, sys.coords) for Molly's SVector{3,Float64}.
 *   - Charges are N doubles; forces are written as 3N doubles (overwritten).
 *   - gamma_down is the reference's gamma_1 (image across z = 0),
 *     gamma_up is gamma_2 (image across z = L_z).
 *   - mem == QEM_MEM_HOST: pointers are host memory; the call copies, computes
 *     and synchronises before returning.  mem == QEM_MEM_DEVICE: pointers are
 *     device memory on the handle's device; work is ordered on `stream`
 *     (a cudaStream_t, NULL = legacy default stream) and the call also
 *     synchronises that stream before returning, so the status is final.
 *   - A handle is not thread-safe; use one handle per host thread / stream.
 *   - The caller owns every buffer it passes.  The handle owns its device
 *     scratch (cell arrays, pair list, k-set, partial sums) and grows it on
 *     demand.
 *   - Every entry point returns a qem_status; details of the last failure are
 *     in qem_last_error().  No entry point traps, asserts or aborts.
 */
#ifndef QEM_H
#define QEM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t qem_status;
#define QEM_OK 0
#define QEM_ERR_ARG 1          /* invalid parameter or size                         */
#define QEM_ERR_OUT_OF_SLAB 2  /* Substrate_LJ.jl:37 @assert direction*dz > 0       */
#define QEM_ERR_NONFINITE 3    /* NaN/Inf in coordinates or charges                 */
#define QEM_ERR_NB_OVERFLOW 4  /* neighbour data exceeded a fixed capacity          */
#define QEM_ERR_TIMEOUT 5      /* a bounded device-side wait ran out                */
#define QEM_ERR_CUDA 6         /* CUDA runtime error (message in qem_last_error)    */
#define QEM_ERR_NO_KSET 7      /* long range requested before a k-set exists        */
#define QEM_ERR_RANGE 8        /* exponent range of the FP32 k-space path exceeded  */

/* mode_flags: one bit per parity quirk of the reference (0 = reference Julia) */
#define QEM_CUTOFF_PYTHON 0x1u   /* python_lib quadrature limits (Force_short_range_njit.py:51-52)
                                    instead of Julia's per-image limits (Force_short.jl:48-67)     */
#define QEM_DIR_MINIMAGE 0x2u    /* minimum-image x/y direction instead of the raw coordinate
                                    difference of Force_short.jl:57-58                            */
#define QEM_PAIR_PHYSICAL 0x4u   /* F[j] += F_short_ij(j, i) instead of F[j] -= F_ij
                                    (QEM_short.jl:46-47)                                          */
#define QEM_STALE_NEIGHBORS 0x8u /* rebuild the pair list only on calls 1, 1+iter_period, ...
                                    (QEM_short.jl:32-36); default rebuilds every call             */
#define QEM_RESAMPLE_KSET 0x10u  /* draw a fresh random batch of k-vectors on every long-range
                                    call (Force_long.jl:235), on the device: call n after
                                    qem_sample_kset(seed, P) uses batch n of that seed
                                    (qem_draw_kset); recorded graphs and qem_batch_md draw new
                                    batches too.  Default reuses the current batch               */
#define QEM_EQUAL_Z_TIES 0x20u   /* particles of equal z are neither below nor above each other in
                                    the z-ordered long-range sums (python_lib equal_cell,
                                    Sigma_Gamma_func_njit.py:168-281); default: sortperm(z) order,
                                    ties by index (QEM_long.jl:39-40).  Costs a second long-range
                                    pass (the mean over both tie orders)                          */
#define QEM_PYTHON_MODE (QEM_CUTOFF_PYTHON | QEM_DIR_MINIMAGE | QEM_PAIR_PHYSICAL)

/* precision */
#define QEM_FP64 0      /* plain FP64 everywhere                                           */
#define QEM_FP32_FIX 1  /* FP32 quadrature nodes and structure sums, FP64 k-space
                           denominators and phases, cancellation-free short-range
                           denominators; FP32 partial sums are short (one quadrature
                           interval, one chunk, a batch of 8 k-vectors) and are added
                           into FP64, as are all final force/energy reductions        */

/* terms (bit mask) */
#define QEM_TERM_SHORT 0x1u
#define QEM_TERM_LONG 0x2u
#define QEM_TERM_LJ 0x4u
#define QEM_TERM_ALL 0x7u

/* memory kind of the pointers passed to a call */
#define QEM_MEM_HOST 0
#define QEM_MEM_DEVICE 1

/* Substrate_LJ(; cutoff, sigma, eps, sub_pos, direction)  Substrate_LJ.jl:7-17 */
typedef struct {
    double cutoff;
    double sigma;
    double eps;
    double sub_pos;
    double direction; /* +1 or -1 */
} qem_lj_wall;

typedef struct {
    double Lx, Ly, Lz;  /* QEM_short.L / QEM_long.L                                    */
    double alpha;       /* Ewald splitting parameter                                    */
    double r_cutoff;    /* short-range cutoff (must be < min(Lx, Ly) / 2)               */
    double gamma_down;  /* reference gamma_1                                            */
    double gamma_up;    /* reference gamma_2                                            */
    double eps_0;       /* default 1                                                    */
    double accuracy;    /* default 1e-6                                                 */
    int32_t N_t;        /* Gauss-Legendre order, 1..64 (default 30)                     */
    int32_t rbe_p;      /* random-batch size P (default 30)                             */
    int32_t iter_period;/* neighbour refresh period for QEM_STALE_NEIGHBORS (default 100) */
    int32_t n_walls;    /* 0..2 Substrate_LJ walls fused into the short-range pass      */
    qem_lj_wall walls[2];
    uint32_t mode_flags;/* QEM_CUTOFF_PYTHON | ...                                      */
    int32_t precision;  /* QEM_FP64 or QEM_FP32_FIX                                     */
    int32_t device;     /* CUDA device ordinal                                          */
    int32_t reserved0;  /* must be zero                                                 */
    double pv_eps;      /* gamma_up * gamma_down > 1 only: half-width of the window around
                           the pole k_0 = ln(gamma_up gamma_down) / (2 Lz) of the
                           regularised short-range quadrature (python_lib INCAR['eps']) */
    int32_t reserved[2];/* must be zero                                                 */
} qem_params;

/* gamma_up * gamma_down > 1 (metamaterial substrates; python_lib
 * Force_short_norm_njit.py, green_norm_njit.py, Force_short_range_njit.py:
 * 258-286, 311-314): 1 / (g12 e^{-2 k Lz} - 1) has a pole at k_0, and each
 * short-range integral runs over [0, k_0 - e], [k_0 - e, k_0 + e],
 * [k_0 + e, 2 k_0], [2 k_0, k_f] with N_1, 10, N_1, N_t - 2 N_1 nodes
 * (N_1 = int(N_t k_0 / k_f), k_f = max(python limit, 2.1 k_0)), the window
 * through the pole-free part of the denominator and the two sides with the
 * pole term subtracted (principal value).  Needs QEM_FP64, QEM_CUTOFF_PYTHON
 * (the reference defines it for the python_lib only), 0 < pv_eps < k_0 and
 * N_1 >= 1 for both integral families; energies and the adjoint are not
 * defined there (QEM_ERR_ARG).  Two details of the reference are kept: the
 * window of the Gauss rho integrand has no exp(-k^2 / 4 alpha) factor
 * (Force_short_norm_njit.py:59) and the self force adds the point integral
 * with the opposite sign (Force_short_norm_njit.py:330-331).  The long range
 * is unchanged (as in the python_lib). */

typedef struct qem_handle qem_handle;

/* Fills p with the reference defaults (QEM_short.jl:19, QEM_long.jl:19):
 * gamma 0, eps_0 1, accuracy 1e-6, N_t 30, rbe_p 30, iter_period 100, no walls. */
void qem_default_params(qem_params *p);

/* QEM_inter factory (Quasi_Ewald_Method.jl:3-24): alpha = n_atoms / (Lx Ly)
 * (rbe_mode != 0) or sqrt(n_atoms) / (Lx Ly), r_cutoff = s / sqrt(alpha).
 * Writes alpha, r_cutoff and rbe_p into p. */
qem_status qem_inter_params(qem_params *p, int64_t n_atoms, double s, int32_t rbe_mode, int32_t rbe_p);

/* Creates a handle (QEM_short + QEM_long + Substrate_LJ state on one device). */
qem_status qem_create(const qem_params *p, qem_handle **out);
void qem_destroy(qem_handle *h);
const char *qem_last_error(const qem_handle *h);
const char *qem_status_string(qem_status s);

/* Random-batch k-set.  qem_set_kset feeds P rows of (kx, ky, k) and the
 * normaliser sum_K (K_set_generator.jl:28) -- the way parity runs feed the
 * same batch to the library and to the oracle.  qem_sample_kset makes batch 0
 * of the library's own sampler the current k-set: P vectors from
 * exp(-k^2 / 4 alpha) on the 2 pi (m / Lx, n / Ly) lattice (k != 0,
 * |m| <= ceil(k_c Lx / 2 pi) + 1, K_set_generator.jl:7-9; the reference draws
 * them with StatsBase.sample, Force_long.jl:235).  Batch n of a seed is a pure
 * function of (seed, n): row i takes three uniforms from the SplitMix64
 * finaliser of (seed, n, i, 0..2), one to choose between the m_x != 0 and the
 * m_x = 0 parts of the lattice (weights S_x T_y and S_y, S = sum over m != 0,
 * T = sum over all m of exp(-(2 pi m / L)^2 / 4 alpha)) and two for m_x, m_y by
 * inverse CDF, so the draw is exact without rejection.  The reference keeps
 * the probabilities as Float32 (K_set_generator.jl:43), so points whose
 * probability is at most 2^-150 are never drawn there; a row that lands on
 * one (less than 2^-150 per row) takes the next three words (i, 3 t .. 3 t + 2)
 * instead, at most 16 times.  With
 * QEM_RESAMPLE_KSET every long-range call draws the next batch on the device
 * (the batch counter, reset by qem_sample_kset, is in device memory), and
 * qem_get_kset returns the rows of the latest call's batch (the current
 * k-set before the first call); qem_kset_batch reports the counter (the
 * number of long-range calls since qem_sample_kset).  qem_draw_kset computes
 * rows [row0, row0 + P) of batch n for a box and alpha on the host, without a
 * handle or a GPU. */
qem_status qem_set_kset(qem_handle *h, const double *k3, int32_t P, double sum_K);
qem_status qem_sample_kset(qem_handle *h, uint64_t seed, int32_t P);
qem_status qem_get_kset(const qem_handle *h, double *k3_out, int32_t cap, int32_t *P, double *sum_K);
qem_status qem_kset_batch(const qem_handle *h, uint64_t *n);
qem_status qem_draw_kset(const qem_params *p, uint64_t seed, uint64_t n, int64_t row0, int32_t P, double *k3,
                         double *sum_K);

/* Most k-vectors of one k-set (the k-space passes put 16 k-vectors per block
 * along a grid dimension of at most 65535 blocks). */
#define QEM_MAX_KSET 1048560

/* Exact (non-random-batch) k-sum, F_long's rbe_mode = false branch
 * (Force_long.jl:220-233; python_lib Force_long_range_njit_exact.py:10-45):
 * every lattice vector k = 2 pi (m / Lx, n / Ly) with 0 < |k| < k_cutoff, each
 * weighted by exp(-|k|^2 / 4 alpha) in place of the random batch's sum_K / P.
 * Two typos of the Julia branch are fixed: the lattice bound is
 * trunc(k_cutoff L / 2 pi) (written k_cutoff * L_x / 2 * pi, lines 221-222)
 * and |k| = sqrt(kx^2 + ky^2) (written sqrt(k_x^2 + k_y), line 227); the k = 0
 * lattice point, which that loop would also visit, is the separate k = 0 term.
 * QEM_inter (Quasi_Ewald_Method.jl:16) takes k_cutoff = 2 s sqrt(alpha).
 *
 * qem_exact_kset_rows writes up to cap rows (kx, ky, |k|) and weights in the
 * Julia loop order (m outer, n inner) and the full count (host only; no GPU
 * needed).  qem_set_kset_weighted feeds any k-set with per-row weights (sum_K
 * then reports the sum of the weights); qem_set_kset_exact generates and feeds
 * the exact set of the handle's box and alpha.  qem_set_kset and
 * qem_sample_kset return the handle to uniform sum_K / P weights, and so does
 * QEM_RESAMPLE_KSET at its next draw.  qem_get_kset_weights reports P = 0 for
 * a uniform k-set. */
qem_status qem_exact_kset_rows(double Lx, double Ly, double alpha, double k_cutoff, double *k3, double *w,
                               int64_t cap, int64_t *count);
qem_status qem_set_kset_weighted(qem_handle *h, const double *k3, const double *w, int32_t P);
qem_status qem_set_kset_exact(qem_handle *h, double k_cutoff, int32_t *P);
qem_status qem_get_kset_weights(const qem_handle *h, double *w_out, int32_t cap, int32_t *P);

/* Fused evaluation: short range (+ self terms) + long range + walls.
 * F: 3N doubles (overwritten).  energy: NULL or one double receiving the QEM
 * short + long energy (Substrate_LJ has no energy in the reference). */
qem_status qem_forces(qem_handle *h, int32_t N, const double *xyz, const double *q, double *F, double *energy,
                      uint32_t terms, int32_t mem, void *stream);

/* Molly.forces(inter::QEM_short, sys)   QEM_short.jl:27-59 (plus walls if configured) */
qem_status qem_short_forces(qem_handle *h, int32_t N, const double *xyz, const double *q, double *F, int32_t mem,
                            void *stream);
/* Molly.forces(inter::QEM_long, sys)    QEM_long.jl:32-44, Force_long.jl:201-242 */
qem_status qem_long_forces(qem_handle *h, int32_t N, const double *xyz, const double *q, double *F, int32_t mem,
                           void *stream);
/* Molly.forces(inter::Substrate_LJ, sys) Substrate_LJ.jl:24-46 for the handle's walls */
qem_status qem_lj_forces(qem_handle *h, int32_t N, const double *xyz, double *F, int32_t mem, void *stream);
/* Molly.potential_energy for the QEM terms (python_lib energies; see above) */
qem_status qem_potential_energy(qem_handle *h, int32_t N, const double *xyz, const double *q, double *energy,
                                uint32_t terms, int32_t mem, void *stream);

/* Adjoint of qem_forces for L = gE * E + sum_i gF_i . F_i (the backward of the
 * reference's python_lib autograd use; no reference counterpart in Julia):
 *   gxyz   3N doubles, dL/dr_i                      (overwritten)
 *   gq     N doubles or NULL, dL/dq_i               (overwritten)
 *   ggamma 2 doubles or NULL, dL/dgamma_down, dL/dgamma_up
 * gF: 3N doubles or NULL (zero).  Always evaluated in FP64, whatever the
 * handle's precision, with the neighbour-list rules of the forward call and
 * the handle's current k-set (a k-set is sampled if none exists; with
 * QEM_RESAMPLE_KSET the backward uses the batch of the latest forward call).
 * The derivatives are those of the discretised quantities, so the
 * quadrature limits' dependence on the image distances (Julia cutoff mode)
 * is included; the k = 0 force is piecewise constant in z and contributes no
 * dL/dz. */
qem_status qem_backward(qem_handle *h, int32_t N, const double *xyz, const double *q, const double *gF, double gE,
                        double *gxyz, double *gq, double *ggamma, uint32_t terms, int32_t mem, void *stream);

/* Neighbour data of the last short-range build, for bit-exact checks.
 * qem_pair_list: (i, j) pairs with i < j, min-image rho <= r_cutoff
 * (CellListMap.neighborlist set, QEM_short.jl:35); writes min(cap, npairs)
 * pairs, always sets *npairs.  qem_cell_index: per particle cell id
 * (cx * ncy + cy) of the 2-D binning and the per-cell start offsets. */
qem_status qem_pair_list(qem_handle *h, int32_t N, const double *xyz, int32_t *pairs, int64_t cap, int64_t *npairs);
qem_status qem_cell_index(qem_handle *h, int32_t N, const double *xyz, int32_t *cell, int32_t *cell_start,
                          int32_t cap_cells, int32_t *ncx, int32_t *ncy);
/* z order: zlist[m] = index of the m-th lowest z (sortperm, QEM_long.jl:39-40). */
qem_status qem_z_order(qem_handle *h, int32_t N, const double *xyz, int32_t *zlist);

/* Per-kernel device times (ms) of the last call, measured with CUDA events on
 * the call's stream when profiling is enabled (0 = off).  names: a
 * comma-separated list written into buf. */
qem_status qem_set_profiling(qem_handle *h, int32_t on);
qem_status qem_get_timings(const qem_handle *h, double *ms, int32_t cap, int32_t *n, char *names, int32_t names_cap);
/* Counts of the last call: [0] pairs evaluated, [1] particles, [2] k-vectors,
 * [3] kernel launches. */
qem_status qem_get_counts(const qem_handle *h, int64_t *counts, int32_t cap);

/* Long-range forces with no device allocation.  No counterpart in the
 * reference: it serves callers that must not call cudaMalloc (a host framework
 * that owns all device memory in its own pool, a real-time loop that must not
 * enter the CUDA allocator, whose cost and implicit synchronisation are
 * unbounded).  F (3N, overwritten) is the same as qem_long_forces gives on a
 * handle with the same parameters, fed the rows k3 (P x (kx, ky, k), host
 * memory) and normaliser sum_K by qem_set_kset.  xyz, q and F are device
 * memory of device p->device; work is ordered on `stream`, which the call
 * synchronises before returning (non-finite inputs give QEM_ERR_NONFINITE; in
 * QEM_FP32_FIX a particle with max(k) |z - L_z / 2| > 60, far outside the
 * slab, gives QEM_ERR_RANGE).  Scratch lives in one fixed
 * QEM_NOALLOC_SCRATCH_BYTES device array inside libqem.so that every GPU
 * loading the library holds until exit; larger N or P are rejected with
 * QEM_ERR_ARG.  Every call looks up that array's device address
 * (cudaGetSymbolAddress) with the device current.  All calls share the array,
 * which keeps the last call's contents: calls that overlap on the GPU race and
 * must be serialised by the caller. */
#define QEM_NOALLOC_MAX_N 32768
#define QEM_NOALLOC_MAX_P 512
#define QEM_NOALLOC_SCRATCH_BYTES (8u << 20)
qem_status qem_long_forces_noalloc(const qem_params *p, int32_t N, const double *xyz, const double *q, int32_t P,
                                   const double *k3, double sum_K, double *F, void *stream);

/* Sharding one system over `world` ranks (one GPU each): with rank r set, a
 * call evaluates the pairs [Np r / W, Np (r + 1) / W) of the neighbour list,
 * the k-set rows [P r / W, P (r + 1) / W) (weighted by the full sum_K / P),
 * and, on rank 0 only, the self image terms, the walls and the k = 0 term;
 * forces and energies of the W ranks then sum to the unsharded result (the
 * caller's one exchange step: an all-reduce of F and E).  Every rank must
 * hold the same positions, charges and k-set.  qem_backward ignores the
 * shard and evaluates the whole system.  Default rank 0 of 1. */
qem_status qem_set_shard(qem_handle *h, int32_t rank, int32_t world);

/* ---- batches of independent systems (many small slabs, one launch graph) ----
 * A batch groups B handles (same device), system s with N[s] particles.  The
 * batch calls take device arrays laid end to end: system s owns particles
 * [off[s], off[s] + N[s]) of xyz (3 per particle), q, F and v, with off the
 * exclusive prefix sum of N.  The handles stay owned by the caller.
 *
 * A batch evaluation runs one of two ways (qem_batch_set_mode):
 *   QEM_BATCH_FUSED: 16 or 17 launches for the whole batch, each over all
 *     systems -- pack and z order over (system, particle tile) work lists (a
 *     tile pass of 2048-key tiles and, above 2048 particles, one merge pass); cells and pair list in eight
 *     phases over cell, particle and pair tiles (their scans one block per
 *     system); then one launch per phase (pair forces; long-range
 *     preparation, chunk totals, their scan, the k-sliced force pass and the
 *     final sum; the gather) over a (system, tile) work list.  Every system must take the small-system kernels in
 *     FP32+fix: N <= 8192, fewer than two particles per cell on average (or
 *     fewer than 3 cells along x or y), no equal-z tie mode, no shard, and
 *     terms with both QEM_TERM_SHORT and QEM_TERM_LONG.  Each system's forces
 *     are those of its own qem_forces call with the same k-slice count.
 *   QEM_BATCH_POOL: every system's own pipeline, forked over a pool of
 *     streams (any batch).
 *   QEM_BATCH_AUTO (default): fused when every system qualifies, else the
 *     pool; qem_batch_autotune may pick either.
 *
 * qem_batch_forces: forces of every system (terms as in qem_forces).  The
 *   first call (and the first after a change of terms, of the mode, or of a
 *   handle's buffers or k-set) runs each system synchronously to size its
 *   buffers and upload its k-set, and builds the fused work lists; later
 *   calls only enqueue work on `stream` (forked to a second stream, or to the
 *   pool, and joined), allocate nothing and can be captured into a CUDA
 *   graph.  Device status (pair-list overflow, non-finite input, particle out
 *   of the slab) accumulates and is reported by qem_batch_check, which
 *   synchronises `stream`; after an overflow the next qem_batch_forces sizes
 *   every system again.
 * qem_batch_md: nsteps velocity-Verlet steps of every system (unit masses,
 *   x += v dt + F dt^2 / 2, v += (F + F') dt / 2, x and y wrapped into the
 *   box), with one step recorded once as a CUDA graph and replayed.  On
 *   return xyz and v hold the final state and F the final forces; the call
 *   synchronises and checks the status.  Neighbour lists are rebuilt every
 *   step; a system with QEM_RESAMPLE_KSET draws a fresh k batch every step
 *   (on the device, inside the recorded step), the others keep their current
 *   k-set for the whole run.
 * qem_batch_autotune: times the graph-replayed force evaluation for stream
 *   pool widths 1, 2, 4, ... up to min(B, 128) and, when the batch can run
 *   fused, for the fused tilings (chunk length 512, 256, 128 or 64; k-slices
 *   per system of the force pass: the handle's own count or at most 2, 4;
 *   work lists in batch order or largest system first), and keeps the
 *   fastest; returns the pool width (0 when the fused phases won) and the
 *   time per batch evaluation (ms).
 * qem_batch_set_mode: mode (QEM_BATCH_AUTO, _FUSED or _POOL), ks (k-slices
 *   per system of the fused force pass, 0 = each handle's own), order (0
 *   batch order, 1 largest system first) of the fused work lists and chunk
 *   (particles per z-ordered chunk of the fused k-space passes: 0 = 512, or
 *   a divisor of 512 of at least 32; shorter chunks keep sparse slabs on the
 *   force pass's one-walk path, which needs max(k) x the chunk's z extent
 *   <= 1).  A fused request for a batch that does not qualify fails at
 *   qem_batch_forces.
 * qem_batch_get_mode: the way evaluations run now (QEM_BATCH_FUSED or
 *   QEM_BATCH_POOL), ks, order, chunk, the kernel launches per fused
 *   evaluation (-1 on the pool) and, when the batch cannot run fused, why
 *   (else "").
 * qem_batch_set_thermostat: the Andersen thermostat of the MD steps (Molly's
 *   AndersenThermostat(temp, coupling_const) in test/QEM_test.jl:53-56;
 *   python_lib Andersen.py:8-22): after each step every particle, with
 *   probability min(1, nu dt) (nu = 1 / coupling_const), takes a new velocity
 *   with N(0, kT) components (unit masses).  nu = 0 or kT = 0 switches it
 *   off.  The draws are a counter-based function of (seed, step, particle):
 *   u_k = (SplitMix64-finalised seed, step, particle, k) >> 11, u in (0, 1];
 *   collision if u_0 <= p; Box-Muller on (u_1, u_2) and (u_3, u_4) for x, y
 *   and z.  The call resets the step counter (synchronising the device);
 *   qem_batch_thermostat_step reads it (steps taken since). */
typedef struct qem_batch qem_batch;
qem_status qem_batch_create(int32_t B, qem_handle *const *handles, const int32_t *N, qem_batch **out);
void qem_batch_destroy(qem_batch *b);
const char *qem_batch_last_error(const qem_batch *b);
qem_status qem_batch_forces(qem_batch *b, const double *xyz, const double *q, double *F, uint32_t terms,
                            void *stream);
qem_status qem_batch_check(qem_batch *b, void *stream);
qem_status qem_batch_md(qem_batch *b, int32_t nsteps, double dt, double *xyz, double *v, const double *q, double *F,
                        uint32_t terms, void *stream);
qem_status qem_batch_autotune(qem_batch *b, const double *xyz, const double *q, double *F, uint32_t terms,
                              void *stream, int32_t *width, double *ms_per_eval);
qem_status qem_batch_set_thermostat(qem_batch *b, double kT, double nu, uint64_t seed);
qem_status qem_batch_thermostat_step(const qem_batch *b, uint64_t *step);
#define QEM_BATCH_AUTO 0
#define QEM_BATCH_FUSED 1
#define QEM_BATCH_POOL 2
qem_status qem_batch_set_mode(qem_batch *b, int32_t mode, int32_t ks, int32_t order, int32_t chunk);
qem_status qem_batch_get_mode(const qem_batch *b, int32_t *mode, int32_t *ks, int32_t *order, int32_t *chunk,
                              int32_t *launches, const char **why);

/* Library identity (version string and the compiled CUDA architecture). */
const char *qem_version(void);

/* Measured FP32 FMA throughput (TFLOP/s, 2 flops per FMA; the larger of
 * scalar and packed FP32x2 FMA chains) and MUFU ex2 throughput (Tops/s) of
 * `device`: the roofline denominators of the QEM
 * kernels, which are bound by those two pipes.  Diagnostic; no reference
 * counterpart. */
qem_status qem_measure_peaks(int32_t device, double *fp32_tflops, double *mufu_tops);
/* Measured FP64 FMA throughput (TFLOP/s) of `device`: the roofline
 * denominator of the FP64 path and of qem_backward.  Diagnostic. */
qem_status qem_measure_fp64_peak(int32_t device, double *fp64_tflops);

#ifdef __cplusplus
}
#endif
#endif /* QEM_H */

// qem_internal.cuh -- shared declarations of the libqem CUDA sources.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/qem.h"

#define QEM_MAX_NT 64
#define QEM_PI 3.14159265358979323846

// device status bits (atomicOr into a device word, read back at call end)
#define QEM_ST_NONFINITE 0x1u
#define QEM_ST_OUT_OF_SLAB 0x2u
#define QEM_ST_OVERFLOW 0x4u
#define QEM_ST_RANGE 0x8u

// Per-call constants of the short-range pass (Force_short.jl:25-107 and the
// Substrate_LJ walls), passed by value so every thread reads them from the
// constant bank.
struct ShortConsts {
    double Lx, Ly, invLx, invLy, Lz, twoLz;
    double alpha, inv4alpha, rc2;
    double g1, g2, g12, one_minus_g12;
    double neg_lnacc;     // -ln(accuracy) > 0
    double pref;          // 1 / (2 pi eps_0)
    double kf_gauss_py;   // python_lib global limits (Force_short_range_njit.py:51-52)
    double kf_point_py;
    int Nt;
    uint32_t flags;       // QEM_CUTOFF_PYTHON | QEM_DIR_MINIMAGE | QEM_PAIR_PHYSICAL
    int n_walls;
    int shard_rank;       // this rank evaluates pairs [Np r / W, Np (r + 1) / W) of the list

    double wall_cut[2], wall_sig2[2], wall_eps[2], wall_pos[2], wall_dir[2];
    // Gauss-Legendre nodes/weights on [-1, 1]: FP32 as node pairs (2m, 2m+1)
    // for the packed FP32x2 loop, an odd N_t padded with (x = -1, w = 0),
    // i.e. a node at k = 0 of weight zero; FP64 as plain arrays.  The FP32
    // loop reads node n of an interval [0, K] as k = h t_n, h = K / 2,
    // t_n = 1 + x_n, and takes w_n t_n and 1 / sqrt(t_n) (0 at t_n = 0)
    // from tables as well
    int Nt2;              // (N_t + 1) / 2
    int shard_world;      // W >= 1; the self terms and walls belong to rank 0
    float2 tf2[QEM_MAX_NT / 2], wf2[QEM_MAX_NT / 2], wtf2[QEM_MAX_NT / 2], rtf2[QEM_MAX_NT / 2];
    double xd[QEM_MAX_NT], wd[QEM_MAX_NT];
    // gamma_1 gamma_2 > 1: regularised quadrature (FP64), family 0 Gauss, 1 point;
    // sub-interval t of family f has norm_n[f][t] nodes at norm_xw[norm_off[f][t]]
    // and weights right after them
    // FP32 factors of the node loop: -log2(e) 2 L_z, -log2(e) / (4 alpha),
    // 2 L_z, g_u g_d, 1 - g_u g_d; RHO_BINS / r_c^2 of the pair grouping
    float f_nlog2e_2Lz, f_nlog2e_c2, f_2Lz, f_g12, f_omg12;
    double bins_per_rc2;
    int norm;
    double k0, pv_eps, kf_norm[2];
    int norm_n[2][4], norm_off[2][4];
    const double *norm_xw;
};

// rho^2 bins of the pair grouping (bins_per_rc2 = QEM_RHO_BINS / r_c^2)
constexpr int QEM_RHO_BINS = 64;

// Counting sort of a block's items into NBINS bins (NBINS a multiple of 32;
// every thread passes its item's bin, NBINS - 1 for no item): returns the
// thread whose item this thread takes, so that the items of a bin sit on
// consecutive threads, bins ascending.  hist (NBINS ints) and sidx (one int
// per thread) are shared memory.  The order inside a bin depends on the
// atomics; callers evaluate and write each item under its own index, so
// their results do not.  Every thread of the block must call it.
template <int NBINS>
__device__ __forceinline__ int group_by_bin(int bin, int *hist, int *sidx)
{
    static_assert(NBINS % 32 == 0, "bins per lane");
    if (threadIdx.x < NBINS) hist[threadIdx.x] = 0;
    __syncthreads();
    const int slot = atomicAdd(&hist[bin], 1);
    __syncthreads();
    if (threadIdx.x < 32) {  // exclusive scan of the bin counts (NBINS / 32 per lane)
        constexpr int PER = NBINS / 32;
        int v[PER], tot = 0;
#pragma unroll
        for (int j = 0; j < PER; j++) {
            v[j] = tot;
            tot += hist[threadIdx.x * PER + j];
        }
        int x = tot;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, x, d);
            if ((int)threadIdx.x >= d) x += t;
        }
        const int base = x - tot;
#pragma unroll
        for (int j = 0; j < PER; j++) hist[threadIdx.x * PER + j] = base + v[j];
    }
    __syncthreads();
    sidx[hist[bin] + slot] = threadIdx.x;
    __syncthreads();
    return sidx[threadIdx.x];
}

// 2-D cell grid of the in-plane binning
struct CellGeom {
    double Lx, Ly, invLx, invLy;
    double inv_lcx, inv_lcy;  // 1 / cell length
    int ncx, ncy;
};

// Per-k constants of the long-range pass, computed on the device in FP64.
struct KConst {
    double kx_2pi, ky_2pi;  // kx / (2 pi), ky / (2 pi): phase in turns
    double k;
    double W;               // exp(-k Lz / 2) (squared where exp(-k Lz) is needed)
    double g;               // 0.5 / (g12 exp(-2 k Lz) - 1)   (Force_long.jl:21)
    double fx, fy;          // kx / k, ky / k
    double wk;              // (sum_K / P) / (Lx Ly eps_0)
    double ek;              // energy weight -(sum_K / P) / (2 eps_0 Lx Ly) / k
    int mx, my;             // lattice indices: k = 2 pi (mx / Lx, my / Ly) (FP32 path)
};

// FP32 k-space phase in turns from 32-bit fixed-point fractions X = x / Lx,
// Y = y / Ly (units of 2^-32) and the lattice indices of k: mx X + my Y is
// exact modulo 2^32, i.e. modulo one turn.  Returned as an angle in
// [-pi, pi): the top 23 bits of the phase (rounded) become the mantissa of a
// float in [1, 2), with half a turn added so that 1.5 maps to phase 0.
__device__ __forceinline__ float lattice_phase(int mx, int my, uint32_t X, uint32_t Y)
{
    const uint32_t ph = (uint32_t)mx * X + (uint32_t)my * Y + 0x80000100u;  // + half a turn, + rounding
    return (__uint_as_float((ph >> 9) | 0x3f800000u) - 1.5f) * 6.28318530717958648f;
}

// Per-k constants of the long-range force pass in its own precision
// (written by the chunk-scan kernel from the structure-sum totals):
// S1 = g e^{-k L_z} (g2 U + g12 e^{-k L_z} V), S2 = g e^{-k L_z} (g12 e^{-k L_z} U + g1 V)
// with U, V the totals of q e^{+-k(z-h)} e^{i k.rho} and g from KConst.
template <typename Real>
struct KForce {
    Real k, wfx, wfy, wk;       // k, w_k kx / k, w_k ky / k, w_k
    Real s1r, s1i, s2r, s2i;
};

// ---------------------------------------------------------------------------
// counter-based random numbers: the SplitMix64 finaliser (Steele, Lea and
// Flood, OOPSLA 2014; Vigna's constants) of seed + golden-ratio increments of
// (a, b, c), so every draw is a pure function of (seed, a, b, c) and host and
// device compute the same words
// ---------------------------------------------------------------------------
__host__ __device__ inline uint64_t mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
__host__ __device__ inline uint64_t draw64(uint64_t seed, uint64_t a, uint64_t b, uint64_t c)
{
    const uint64_t G = 0x9e3779b97f4a7c15ULL;
    return mix64(mix64(mix64(seed + G * (a + 1)) + G * (b + 1)) + G * (c + 1));
}
// uniform in [0, 1): 53 random bits
__host__ __device__ inline double unit53_lo(uint64_t r) { return (double)(r >> 11) * 0x1.0p-53; }

// Random-batch k sampler (K_set_generator.jl:5-45 + StatsBase.sample,
// Force_long.jl:235): k = 2 pi (m_x / L_x, m_y / L_y), (m_x, m_y) != (0, 0),
// |m| <= M, drawn with probability exp(-k^2 / 4 alpha) / sum_K.  The weight
// is a product w_x(m_x) w_y(m_y), so the draw is exact without rejection:
// with S_x = sum_{m != 0} w_x and T_y = sum_m w_y (w_y(0) = 1), the pairs with
// m_x != 0 carry S_x T_y and those with m_x = 0, m_y != 0 carry S_y; one
// uniform picks the part, two more pick m_x and m_y by inverse CDF.
// tab holds four cumulative weight tables, m ascending: x over all m
// (2 Mx + 1), x over m != 0 (2 Mx), y over all m (2 My + 1), y over m != 0 (2 My).
// The reference stores the probabilities exp(-k^2 / 4 alpha) / sum_K as
// Float32 (K_set_generator.jl:34, 43), so lattice points whose probability
// rounds to zero there (|k|^2 >= k2max) are never drawn; a separable draw
// that lands on one (probability below 2^-150 per row) is drawn again from
// the next counter words.
struct KSampler {
    const double *tab;   // device (or host) address of the tables
    int Mx, My;
    double Lx, Ly;
    double Sx, Tx, Sy, Ty;  // sums over m != 0 (S) and over all m (T) per axis
    double k2max;           // |k|^2 bound of the drawable points
    uint64_t seed;
    int64_t row0;           // first row of this rank's share (the device k rows start there)
};
constexpr int QEM_KSAMPLE_TRIES = 16;

// smallest i in [0, n) with c[i] > u (n - 1 if none): inverse CDF of an
// ascending cumulative table
__host__ __device__ inline int cdf_pick(const double *c, int n, double u)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (c[mid] > u) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}

// row `row` of batch n: (kx, ky, |k|).  Try t takes the words 3 t .. 3 t + 2
// of (seed, n, row); after QEM_KSAMPLE_TRIES off-support draws (probability
// below 2^-2400) the row is the lattice point (0, 1) (or (1, 0) if My = 0).
__host__ __device__ inline void ksample_row(const KSampler &S, uint64_t n, int64_t row, double &kx, double &ky,
                                            double &k)
{
    const double *cx_all = S.tab, *cx_nz = cx_all + 2 * S.Mx + 1;
    const double *cy_all = cx_nz + 2 * S.Mx, *cy_nz = cy_all + 2 * S.My + 1;
    const double A = S.Sx * S.Ty;  // weight of m_x != 0
    int mx = S.My > 0 ? 0 : 1, my = S.My > 0 ? 1 : 0;
    for (int t = 0; t < QEM_KSAMPLE_TRIES; t++) {
        const uint64_t c = 3 * (uint64_t)t;
        const double u0 = unit53_lo(draw64(S.seed, n, (uint64_t)row, c));
        const double u1 = unit53_lo(draw64(S.seed, n, (uint64_t)row, c + 1));
        const double u2 = unit53_lo(draw64(S.seed, n, (uint64_t)row, c + 2));
        int ax, ay;
        if (S.Mx > 0 && u0 * (A + S.Sy) < A) {
            const int i = cdf_pick(cx_nz, 2 * S.Mx, u1 * S.Sx);
            ax = i < S.Mx ? i - S.Mx : i - S.Mx + 1;
            ay = cdf_pick(cy_all, 2 * S.My + 1, u2 * S.Ty) - S.My;
        } else {
            ax = 0;
            const int i = cdf_pick(cy_nz, 2 * S.My, u2 * S.Sy);
            ay = i < S.My ? i - S.My : i - S.My + 1;
        }
        const double fx = (2.0 * QEM_PI) * (double)ax / S.Lx, fy = (2.0 * QEM_PI) * (double)ay / S.Ly;
#ifdef __CUDA_ARCH__
        const double k2 = __dadd_rn(__dmul_rn(fx, fx), __dmul_rn(fy, fy));  // the host's rounding
#else
        const double k2 = fx * fx + fy * fy;
#endif
        if (k2 < S.k2max) {
            mx = ax;
            my = ay;
            break;
        }
    }
    kx = 2.0 * QEM_PI * (double)mx / S.Lx;
    ky = 2.0 * QEM_PI * (double)my / S.Ly;
#ifdef __CUDA_ARCH__
    k = sqrt(__dadd_rn(__dmul_rn(kx, kx), __dmul_rn(ky, ky)));  // no contraction: the host gets the same bits
#else
    k = sqrt(kx * kx + ky * ky);
#endif
}

// ---------------------------------------------------------------------------
// host-side launch wrappers (defined in the .cu files)
// ---------------------------------------------------------------------------
cudaError_t qem_launch_pack(int N, const double *xyz, const double *q, double4 *pos, int *cell, CellGeom g,
                            unsigned *status, cudaStream_t s);
// cells: counting sort by cell, ascending index inside a cell, pos_of and the
// positions in cell order (pos_c)
cudaError_t qem_launch_cells(int N, int ncell, const int *cell, const double4 *pos, int *cell_cnt, int *cell_start,
                             int *cell_fill, int *cell_list, int *pos_of, double4 *pos_c, void *scan_tmp,
                             size_t scan_tmp_bytes, cudaStream_t s);
// pair list (owner, other) in poff order and the incoming lists: pcount and
// poff per cell-order position (poff[N] = number of pairs, on the device), at
// most cap pairs stored (QEM_ST_OVERFLOW beyond), in_cnt / in_off per
// particle with in_list in ascending pair order and in_off[N] <= cap (no
// incoming entries at all after an overflow); in_slot is scratch of 5 N ints
// hmask: QEM_PL_MAXB hit masks per particle (scratch of the one-warp-per-cell passes)
constexpr int QEM_PL_MAXB = 8;
cudaError_t qem_launch_pair_list(int N, int ncell, const double4 *pos_c, const int *cell, const int *cell_start,
                                 const int *cell_list, CellGeom g, double rc2, int *pcount, int64_t *poff,
                                 int2 *pairs, int64_t cap, int *in_cnt, int *in_slot, int64_t *in_off, int *in_list,
                                 unsigned *status, void *scan_tmp, size_t scan_tmp_bytes, unsigned *hmask,
                                 cudaStream_t s);
cudaError_t qem_scan_i32_to_i64(const int *in, int64_t *out, int n, void *tmp, size_t tmp_bytes, cudaStream_t s);
cudaError_t qem_scan_f64_excl(const double *in, double *out, int n, void *tmp, size_t tmp_bytes, cudaStream_t s);
size_t qem_scan_tmp_bytes(int n);
// One-block exclusive scan of n <= PT * 1024 values by the calling block of
// 1024 threads (thread t owns elements [t pt, (t + 1) pt), pt = ceil(n / 1024),
// summed in order; the thread totals are scanned exclusively without an
// "inclusive minus own" step); out[n] = total.  warp_tot: 32 entries of
// shared memory.  Every block-wide caller gets the same arithmetic (PT only
// bounds the registers).
template <typename TI, typename TO, int PT = 8>
__device__ void qem_block_scan_excl_small(const TI *__restrict__ in, TO *__restrict__ out, int n, TO *warp_tot)
{
    const int pt = (n + 1023) / 1024;
    const int b = threadIdx.x * pt;
    TO v[PT];
    TO tot = (TO)0;
#pragma unroll
    for (int j = 0; j < PT; j++) {
        const int i = b + j;
        v[j] = (j < pt && i < n) ? (TO)in[i] : (TO)0;
        const TO x = v[j];
        v[j] = tot;  // exclusive within the thread
        tot += x;
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    TO x = tot;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const TO t = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= d) x += t;
    }
    TO ex = __shfl_up_sync(0xffffffffu, x, 1);
    if (lane == 0) ex = (TO)0;
    if (lane == 31) warp_tot[w] = x;
    __syncthreads();
    if (w == 0) {
        TO y = warp_tot[lane];
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const TO t = __shfl_up_sync(0xffffffffu, y, d);
            if (lane >= d) y += t;
        }
        TO e = __shfl_up_sync(0xffffffffu, y, 1);
        if (lane == 0) e = (TO)0;
        warp_tot[lane] = e;  // exclusive over warps
        if (lane == 31) out[n] = y;
    }
    __syncthreads();
    const TO base = warp_tot[w] + ex;
#pragma unroll
    for (int j = 0; j < PT; j++) {
        const int i = b + j;
        if (j < pt && i < n) out[i] = base + v[j];
    }
}

// kernel launches of one integer scan of n elements, of one FP64 scan
// (qem_scan_f64_excl) and of one z sort of N particles
int qem_scan_launches(int n);
int qem_scan_f64_launches(int n);
// whether the cell build of N particles in ncell cells runs as one one-block kernel
bool qem_cells_small(int N, int ncell);
// kernels of one z order of N particles (buckets: the bucket passes of qem_launch_zsort in use)
int qem_zsort_launches(int N, bool buckets = false);

// np: device pointer to the pair count; cap: capacity of pairs / R / Upair
cudaError_t qem_launch_short_pairs(int precision, bool energy, const int64_t *np, int64_t cap, const int2 *pairs,
                                   const double4 *pos, double4 *R, double *Upair, const ShortConsts &c,
                                   cudaStream_t s);
cudaError_t qem_launch_short_gather(int precision, bool energy, bool do_short, bool do_lj, int N,
                                    const double4 *pos, const int *pos_of, const int64_t *poff, const double4 *R,
                                    const double *Upair, const int64_t *in_off, const int *in_list, int64_t cap,
                                    const ShortConsts &c, double *F3, double *Epart, unsigned *status,
                                    cudaStream_t s, const double *Fadd = nullptr);

// stable z order (equal z by ascending index; by descending index with rev_ties).
// Scratch: ztmp N ints, zkey and zkey_tmp N doubles each.  With a device flag
// word zflag (not inside that scratch) and the slab height Lz > 0, more than
// one tile of particles is ordered by z buckets (four short passes), with the
// tile and merge passes as the fallback for a bucket that is too full.
cudaError_t qem_launch_zsort(int N, const double4 *pos, int *zperm, int *ztmp, double *zkey, double *zkey_tmp,
                             cudaStream_t s, bool rev_ties = false, int *zflag = nullptr, double Lz = 0.0);
// y = a x (y may be x)
cudaError_t qem_launch_scale(int n, double a, const double *x, double *y, cudaStream_t s);
struct LongBuffers {
    double *zx, *zy;      // z-ordered in-plane coordinates (FP64, phases)
    uint4 *zP = nullptr;  // FP32 path: per particle {x / Lx, y / Ly as 32-bit fixed-point box fractions
                          // (the lattice_phase inputs), z - Lz/2, q as FP32 bits}
    double *zhd;          // z - Lz/2
    double *qd;
    double *k0;           // per z-ordered particle: q (Q_below - Q_above) / (2 Lx Ly eps_0)
    double *qscan;        // exclusive scan of q in z order
    KConst *kc;           // P per-k constants
    double *kin;          // P x 3 (kx, ky, k) FP64
    double *tot;          // P x nch x 4 chunk totals
    double *off;          // P x nch x 4 chunk offsets (u from below, v from above), stored
                          // as float in the FP32 path
    void *kf;             // P KForce<float | double> force constants
    double *Utot;         // P x 4 global totals
    double *Eks;          // P per-k split energy term
    double *Epart;        // per-block energy partials (ks * nch + nb0 entries)
    double *Fpart;        // ks x N x 3 per-k-slice force partials (z order)
    int ks;               // number of k slices of the force pass
    void *stmp;           // scan scratch
    size_t stmp_bytes;
    int skip_k0 = 0;      // 1: leave out the k = 0 term (sharded ranks other than 0)
    const double *kwt = nullptr;  // P per-k weights (exact k-sum); nullptr: sum_K / P for every k
    double zlim = 0.0;    // FP32 path: largest |z - Lz/2| whose e^{+-k (z - Lz/2)} stays in FP32
                          // range for every k (QEM_ST_RANGE beyond); 0: no check
    // per-call random batch: when draw_ctr is set, the per-k constants kernel
    // first draws row sampler.row0 + m of batch *draw_ctr into kin (the rows
    // of this call), and the last kernel of the pass advances *draw_ctr
    unsigned long long *draw_ctr = nullptr;
    KSampler sampler{};
    // set: the per-k constants were launched on another stream (stage 2) and
    // recorded in this event, which stage 0 waits for before the chunk totals
    cudaEvent_t kconst_done = nullptr;
};
// zlim of the FP32 k-space path for a k-set whose largest |k| is kmax:
// e^{+-k (z - Lz/2)} <= e^{60}, so that sums over many particles stay finite
inline double qem_fp32_zlim(double kmax) { return kmax > 0 ? 60.0 / kmax : 0.0; }
// number of k slices for nch chunks and P k-vectors (at most max_ks); the
// per-slice force partials take ks x N x 3 doubles, and ks x nch stays near
// one wave of force-pass blocks, so they stay below ~15 MB at any N
int qem_long_ksplit(int nch, int P, int max_ks, int precision);
constexpr int QEM_LONG_MAX_KS = 64;
// stage 0: z-ordered gather, k = 0 term, per-k constants, chunk totals and
// their scan; stage 1: the k-sliced force pass, added into F3; stage 2: the
// per-k constants alone (for a stream beside the z order; not for the
// one-block preparation, qem_long_prep_is_small).
bool qem_long_prep_is_small(int N, bool energy);
cudaError_t qem_launch_long(int precision, bool energy, int N, int P, const double4 *pos, const int *zperm,
                            const LongBuffers &b, double Lx, double Ly, double Lz, double g1, double g2, double eps0,
                            double sum_K, double *F3, int nch, unsigned *status, cudaStream_t s, int stage);
int qem_long_chunk(void);

cudaError_t qem_launch_reduce_sum(const double *in, int n, double *out, cudaStream_t s);

// ---- batch API hooks (defined in qem_capi.cu) -------------------------------
// capturable evaluation on device memory (see run_once in qem_capi.cu)
qem_status qem_forces_async(qem_handle *h, int N, const double *xyz, const double *q, double *F, uint32_t terms,
                            cudaStream_t s);
// synchronises s, reads and clears the handle's device status word
qem_status qem_status_check(qem_handle *h, cudaStream_t s);
const qem_params *qem_handle_params(const qem_handle *h);
// caps the k-slices of the handle's long-range force pass (1 .. QEM_LONG_MAX_KS)
void qem_handle_set_long_max_ks(qem_handle *h, int max_ks);
const char *qem_handle_error(const qem_handle *h);

// ---- fused batches: one launch per phase over all systems -------------------
// BatchSys is one system of a batch: its slice of the batch arrays, its
// handle's device buffers and its per-call constants, i.e. the arguments the
// single-system launches of the small-system path take.  A phase's blocks
// read (system, x, y) from a work list built on the host and run the same
// per-block code as the single-system kernels; the one-block kernels of a
// small system (cells + pair list, and the long-range preparation) run as
// one block per system.
struct BatchSys {
    int N, ncell, P, nch, ks;
    int lch;                  // particles per chunk of the k-space passes
    int64_t cap;              // pair capacity
    int64_t off;              // first particle of the system in the batch arrays
    double *Flong;            // long-range forces (handle buffer), added by the gather
    double4 *pos, *pos_c;
    int *cell, *cstart, *clist, *pos_of, *pcount, *in_cnt, *in_fill, *in_list;
    int64_t *poff, *in_off;
    int2 *pairs;
    double4 *R;
    unsigned *status;
    CellGeom geom;
    double rc2;
    int *zperm, *ztmp;
    double *zkey, *zkey2;
    LongBuffers b;
    // k-space constants of the preparation (as qem_launch_long derives them)
    double h, fscale, Lz, g1, g2, g12, wk, esc, wden, eden, invLx, invLy, Lx_2pi, Ly_2pi;
};
struct BatchWork {
    int s, x, y, pad;
};
// the block's shared copy of a system's struct (BatchSys, ShortConsts):
// every thread copies words, then a block barrier
template <class T>
__device__ __forceinline__ void block_copy(T *dst, const T *src)
{
    static_assert(sizeof(T) % 4 == 0, "word copy");
    const unsigned *a = reinterpret_cast<const unsigned *>(src);
    unsigned *b = reinterpret_cast<unsigned *>(dst);
    for (int i = threadIdx.x; i < (int)(sizeof(T) / 4); i += blockDim.x) b[i] = a[i];
    __syncthreads();
}
// declares `T &name` in shared memory holding *src (the types have default
// member initialisers, which a __shared__ declaration of the type cannot take)
#define QEM_SHARED_COPY(T, name, src)                              \
    __shared__ __align__(16) unsigned char name##_raw[sizeof(T)]; \
    T &name = *reinterpret_cast<T *>(name##_raw);                  \
    block_copy(&name, (src))
// blocks per system of each phase: pairs per pair block, particles per
// gather / final block, k-vectors per totals / scan block, k-slices per
// force-pass block
int qem_batch_pair_tile(void);
int qem_batch_particle_tile(void);
int qem_batch_ltot_tile(void);
int qem_batch_lscan_tile(void);
int qem_batch_lforce_tile(void);
// z order: pack + rank-sorted tiles over particle tiles, then merge passes
// 0, 1, .. over the particle tiles of the systems with that many passes
int qem_batch_zsort_passes(int N);
int qem_batch_ztile(void);  // particles per tile of the z-order tile pass
cudaError_t qem_launch_batch_pack_ztile(int nw, const BatchWork *w, const BatchSys *d, const double *xyz,
                                        const double *q, cudaStream_t s);
cudaError_t qem_launch_batch_zmerge(int nw, const BatchWork *w, const BatchSys *d, int pass, cudaStream_t s);
// cells and pair list: eight launches (counting scatter into cells and the
// two scans one block per system; the in-cell sort over tiles of 256 cells,
// the owners' count and fill passes and the incoming sort over particle
// tiles, the incoming scatter over pair tiles of 256)
cudaError_t qem_launch_batch_lists(int B, const BatchWork *cells, int ncells, const BatchWork *parts, int nparts,
                                   const BatchWork *pairs, int npairs, const BatchSys *d, cudaStream_t s);
cudaError_t qem_launch_batch_lprep(int B, const BatchSys *d, cudaStream_t s);
cudaError_t qem_launch_batch_ltot(int nw, const BatchWork *w, const BatchSys *d, cudaStream_t s);
cudaError_t qem_launch_batch_lscan(int nw, const BatchWork *w, const BatchSys *d, cudaStream_t s);
cudaError_t qem_launch_batch_lforce(int nw, const BatchWork *w, const BatchSys *d, cudaStream_t s);
cudaError_t qem_launch_batch_lfinal(int nw, const BatchWork *w, const BatchSys *d, cudaStream_t s);
cudaError_t qem_launch_batch_pairs(int nw, const BatchWork *w, const BatchSys *d, const ShortConsts *sc,
                                   cudaStream_t s);
cudaError_t qem_launch_batch_gather(int nw, const BatchWork *w, const BatchSys *d, const ShortConsts *sc, int do_lj,
                                    double *F, cudaStream_t s);
// fills one system's entry (qem_capi.cu; off is left 0) after a synchronous
// call of the same size; ks <= 0 keeps the handle's own k-slice count, lch
// (a divisor of qem_long_chunk(), 32 or more; 0: qem_long_chunk()) is the
// chunk length of the k-space passes.
// Returns QEM_ERR_ARG with the reason in *why when the system does not take
// the small-system kernels in FP32+fix (the batch then keeps per-system
// pipelines), QEM_ERR_NO_KSET when it needs a synchronous call first (its
// size, buffers or k-set changed since the last one).
qem_status qem_handle_batch_sys(qem_handle *h, int N, int ks, int lch, BatchSys *d, ShortConsts *sc,
                                const char **why);
// changes whenever a buffer of any handle is reallocated or this handle's
// k-set, shard or pair capacity changes
uint64_t qem_handle_state(const qem_handle *h);

// ---- adjoint (FP64) --------------------------------------------------------
// pair records RA (2 double4 per pair) and the per-particle pass writing
// dL/dr, dL/dq (gq may be NULL) and per-block gamma partials gam[2 * nb]
int qem_adj_gather_blocks(int N);
cudaError_t qem_launch_short_pair_adj(const int64_t *np, int64_t cap, const int2 *pairs, const double4 *pos,
                                      const double *gF, double gE, double4 *RA, const ShortConsts &c,
                                      cudaStream_t s);
cudaError_t qem_launch_adj_gather(int N, bool do_short, bool do_lj, const double4 *pos, const int *pos_of,
                                  const int64_t *poff, const double4 *RA, const int64_t *in_off,
                                  const int *in_list, int64_t cap, const double *gF, double gE,
                                  const ShortConsts &c, double *gxyz, double *gq, double *gam, cudaStream_t s);
struct LongAdjBuffers {
    double *zgx, *zgy, *zgz;   // cotangents in z order
    double *w1, *w2, *s1, *s2; // k = 0 adjoint inputs and their exclusive scans (N + 1)
    double *atot;              // P x nch x 8 chunk totals of a, b, P c1, P c2
    double *aoff;              // P x nch x 4 scans of a (from above) and b (from below)
    double *lam;               // P x 4 Lambda_U, Lambda_V
    double *ggk;               // P x 2 per-k gamma derivatives
    double *Gpart;             // ks x N x 4 per-slice (dL/dx, dL/dy, dL/dz, dL/dq), z order
    double *gam;               // 2: gamma derivatives of the long range
};
// after stage 0 of qem_launch_long in FP64: adds the long-range dL/dr, dL/dq
// into gxyz, gq (particle order)
// stage 0: everything up to the per-slice partials and the gamma sums (reads
// only the forward quantities and gF); stage 1: the final pass, which adds
// into gxyz and gq; -1: both
cudaError_t qem_launch_long_adj(int N, int P, const int *zperm, const LongBuffers &b, const LongAdjBuffers &a,
                                double Lx, double Ly, double Lz, double g1, double g2, double eps0, const double *gF,
                                double gE, double *gxyz, double *gq, int nch, int ks, cudaStream_t s,
                                int stage = -1);

// ---------------------------------------------------------------------------
// device helpers
// ---------------------------------------------------------------------------
#ifdef __CUDACC__
__device__ __forceinline__ double jl_sign(double v) { return (double)((v > 0) - (v < 0)); }

__device__ __forceinline__ double min_image(double d, double L, double invL) { return d - L * rint(d * invL); }

// ---- packed FP32x2 arithmetic (sm_100: one instruction, two lanes) -------
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 f2s(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }

// 2^x (hardware approximation, denormal results flushed to zero)
__device__ __forceinline__ float ex2_approx(float x)
{
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ float rsqrt_ftz(float x)
{
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float cos_ftz(float x)
{
    float r;
    asm("cos.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float sin_ftz(float x)
{
    float r;
    asm("sin.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Bessel J0 and J1 in FP32 at two arguments x = (x0, x1) at once, one per
// packed lane; R = x^{-1/2} is supplied by the caller.
//  * x < 3: the polynomial approximations of Abramowitz & Stegun, Handbook of
//    Mathematical Functions, 9.4.1 / 9.4.4 (published absolute error <= 5e-8
//    for J0, <= 1.3e-8 for J1), coefficients rescaled to run in y = x^2 (A&S
//    use (x/3)^2).
//  * x >= 3: the Hankel asymptotic form with fitted amplitudes: t = x - pi/4,
//    u = 1/x, w = u^2,
//        J0 = R (P0(w) cos t + u Q0(w) sin t),  J1 = R (P1(w) sin t + u Q1(w) cos t),
//    P of degree 5 and Q of degree 4, near-minimax fits on w in (0, 1/9] made
//    by gen_bessel_pq.py in this directory (sqrt(2/pi) and the signs folded
//    in); one sine and one cosine of t serve both orders.  Error of the whole
//    FP32 evaluation (that script's emulation): <= 1.1e-7 on [3, 25].
//    t is reduced modulo 2 pi by n = round(t / 2 pi) (adding and subtracting
//    1.5 * 2^23, valid while |t| / 2 pi < 2^22) and a two-term split of 2 pi.
// A branch runs when either lane needs it and each lane keeps its own
// branch's result.
namespace bj {
__host__ __device__ constexpr float s9(double c, int j) { return (float)(c / (j == 0 ? 1.0 : j == 1 ? 9.0 : j == 2 ? 81.0 : j == 3 ? 729.0 : j == 4 ? 6561.0 : j == 5 ? 59049.0 : 531441.0)); }
// gen_bessel_pq.py: coefficients of w^0 .. w^deg
constexpr float P0_0 = 7.978845024e-01f, P0_1 = -5.607697060e-02f, P0_2 = 8.693327505e-02f,
                P0_3 = -3.358948571e-01f, P0_4 = 1.346355509e+00f, P0_5 = -2.857244828e+00f;
constexpr float Q0_0 = 9.973312039e-02f, Q0_1 = -5.799857766e-02f, Q0_2 = 1.549632535e-01f,
                Q0_3 = -5.666049405e-01f, Q0_4 = 1.216355152e+00f;
constexpr float P1_0 = 7.978846274e-01f, P1_1 = 9.347446406e-02f, P1_2 = -1.121584213e-01f,
                P1_3 = 4.034436691e-01f, P1_4 = -1.577854617e+00f, P1_5 = 3.316100318e+00f;
constexpr float Q1_0 = 2.992038999e-01f, Q1_1 = -8.131090927e-02f, Q1_2 = 1.916038321e-01f,
                Q1_3 = -6.738063288e-01f, Q1_4 = 1.426397851e+00f;
}  // namespace bj

__device__ __forceinline__ void bessel01_x2(float2 x, float2 R, float2 &J0, float2 &J1)
{
    using namespace bj;
    const bool s0 = x.x < 3.0f, s1 = x.y < 3.0f;
    if (s0 || s1) {
        const float2 y = mul2(x, x);
        float2 a = fma2(y, f2s(s9(0.0002100, 6)), f2s(s9(-0.0039444, 5)));
        a = fma2(y, a, f2s(s9(0.0444479, 4)));
        a = fma2(y, a, f2s(s9(-0.3163866, 3)));
        a = fma2(y, a, f2s(s9(1.2656208, 2)));
        a = fma2(y, a, f2s(s9(-2.2499997, 1)));
        J0 = fma2(y, a, f2s(1.0f));
        float2 b = fma2(y, f2s(s9(0.00001109, 6)), f2s(s9(-0.00031761, 5)));
        b = fma2(y, b, f2s(s9(0.00443319, 4)));
        b = fma2(y, b, f2s(s9(-0.03954289, 3)));
        b = fma2(y, b, f2s(s9(0.21093573, 2)));
        b = fma2(y, b, f2s(s9(-0.56249985, 1)));
        J1 = mul2(x, fma2(y, b, f2s(0.5f)));
    }
    if (!(s0 && s1)) {
        const float2 u = mul2(R, R);  // 1 / x
        const float2 w = mul2(u, u);
        float2 p0 = fma2(w, f2s(P0_5), f2s(P0_4));
        p0 = fma2(w, p0, f2s(P0_3));
        p0 = fma2(w, p0, f2s(P0_2));
        p0 = fma2(w, p0, f2s(P0_1));
        p0 = fma2(w, p0, f2s(P0_0));
        float2 p1 = fma2(w, f2s(P1_5), f2s(P1_4));
        p1 = fma2(w, p1, f2s(P1_3));
        p1 = fma2(w, p1, f2s(P1_2));
        p1 = fma2(w, p1, f2s(P1_1));
        p1 = fma2(w, p1, f2s(P1_0));
        float2 q0 = fma2(w, f2s(Q0_4), f2s(Q0_3));
        q0 = fma2(w, q0, f2s(Q0_2));
        q0 = fma2(w, q0, f2s(Q0_1));
        q0 = fma2(w, q0, f2s(Q0_0));
        float2 q1 = fma2(w, f2s(Q1_4), f2s(Q1_3));
        q1 = fma2(w, q1, f2s(Q1_2));
        q1 = fma2(w, q1, f2s(Q1_1));
        q1 = fma2(w, q1, f2s(Q1_0));
        float2 t = add2(x, f2s(-0.78539816f));
        const float2 MAGIC = f2s(12582912.0f), INV2PI = f2s(0.15915494309189535f);
        const float2 n = add2(fma2(t, INV2PI, MAGIC), f2s(-12582912.0f));
        t = fma2(n, f2s(1.7484555314695172e-07f), fma2(n, f2s(-6.28318548202514648f), t));
        const float2 S = f2(sin_ftz(t.x), sin_ftz(t.y)), C = f2(cos_ftz(t.x), cos_ftz(t.y));
        const float2 L0 = mul2(R, fma2(p0, C, mul2(mul2(u, q0), S)));
        const float2 L1 = mul2(R, fma2(p1, S, mul2(mul2(u, q1), C)));
        if (!s0) { J0.x = L0.x; J1.x = L1.x; }
        if (!s1) { J0.y = L0.y; J1.y = L1.y; }
    }
}

// packed 1 - exp(-t) by its Taylor series, for 0 <= t < 0.5 (truncation
// < 2e-8 relative)
__device__ __forceinline__ float2 one_minus_exp_neg_series(float2 t)
{
    float2 s = fma2(t, f2s(-1.0f / 362880.0f), f2s(1.0f / 40320.0f));
    s = fma2(t, s, f2s(-1.0f / 5040.0f));
    s = fma2(t, s, f2s(1.0f / 720.0f));
    s = fma2(t, s, f2s(-1.0f / 120.0f));
    s = fma2(t, s, f2s(1.0f / 24.0f));
    s = fma2(t, s, f2s(-1.0f / 6.0f));
    s = fma2(t, s, f2s(0.5f));
    s = fma2(t, mul2(s, f2s(-1.0f)), f2s(1.0f));
    return mul2(t, s);
}

__device__ __forceinline__ float fast_rcp(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

#endif

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
    int pad;
    double wall_cut[2], wall_sig2[2], wall_eps[2], wall_pos[2], wall_dir[2];
    float xf[QEM_MAX_NT], wf[QEM_MAX_NT];   // Gauss-Legendre nodes/weights on [-1, 1]
    double xd[QEM_MAX_NT], wd[QEM_MAX_NT];
};

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
};

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
cudaError_t qem_launch_pair_count(int N, const double4 *pos_c, const int *cell, const int *cell_start,
                                  const int *cell_list, CellGeom g, double rc2, int *pcount, cudaStream_t s);
// fills at most cap pairs (QEM_ST_OVERFLOW beyond) and counts incoming pairs
// per particle into in_cnt (zeroed by the caller)
cudaError_t qem_launch_pair_fill(int N, const double4 *pos_c, const int *cell, const int *cell_start,
                                 const int *cell_list, CellGeom g, double rc2, const int64_t *poff, int2 *pairs,
                                 int64_t cap, int *in_cnt, unsigned *status, cudaStream_t s);
// np: device pointer to the pair count (poff[N])
cudaError_t qem_launch_incoming(int N, const int64_t *np, int64_t cap, const int2 *pairs, const int *in_cnt,
                                int64_t *in_off, int *in_fill, int64_t *in_list, void *scan_tmp,
                                size_t scan_tmp_bytes, cudaStream_t s);
cudaError_t qem_scan_i32_to_i64(const int *in, int64_t *out, int n, void *tmp, size_t tmp_bytes, cudaStream_t s);
cudaError_t qem_scan_f64_excl(const double *in, double *out, int n, void *tmp, size_t tmp_bytes, cudaStream_t s);
size_t qem_scan_tmp_bytes(int n);

// np: device pointer to the pair count; cap: capacity of pairs / R / Upair
cudaError_t qem_launch_short_pairs(int precision, bool energy, const int64_t *np, int64_t cap, const int2 *pairs,
                                   const double4 *pos, double4 *R, double *Upair, const ShortConsts &c,
                                   cudaStream_t s);
cudaError_t qem_launch_short_gather(int precision, bool energy, bool do_short, bool do_lj, int N,
                                    const double4 *pos, const int *pos_of, const int64_t *poff, const double4 *R,
                                    const double *Upair, const int64_t *in_off, const int64_t *in_list, int64_t cap,
                                    const ShortConsts &c, double *F3, double *Epart, unsigned *status,
                                    cudaStream_t s);

cudaError_t qem_launch_zsort(int N, const double4 *pos, int *zperm, int *ztmp, double *zkey, double *zkey_tmp,
                             cudaStream_t s);
struct LongBuffers {
    double *zx, *zy;      // z-ordered in-plane coordinates (FP64, phases)
    float *zhf;           // z - Lz/2 (FP32 path)
    double *zhd;          // z - Lz/2 (FP64 path)
    float *qf;
    double *qd;
    double *k0;           // per z-ordered particle: q (Q_below - Q_above) / (2 Lx Ly eps_0)
    double *qscan;        // exclusive scan of q in z order
    KConst *kc;           // P per-k constants
    double *kin;          // P x 3 (kx, ky, k) FP64
    double *tot;          // P x nch x 4 chunk totals
    double *off;          // P x nch x 4 chunk offsets (u from below, v from above)
    double *Utot;         // P x 4 global totals
    double *Eks;          // P per-k split energy term
    double *Epart;        // per-block energy partials (ks * nch + nb0 entries)
    double *Fpart;        // ks x N x 3 per-k-slice force partials (z order)
    int ks;               // number of k slices of the force pass
    void *stmp;           // scan scratch
    size_t stmp_bytes;
};
// number of k slices for nch chunks and P k-vectors (at most max_ks)
int qem_long_ksplit(int nch, int P, int max_ks);
// stage 0: z-ordered gather, k = 0 term, per-k constants, chunk totals and
// their scan; stage 1: the k-sliced force pass, added into F3.
cudaError_t qem_launch_long(int precision, bool energy, int N, int P, const double4 *pos, const int *zperm,
                            const LongBuffers &b, double Lx, double Ly, double Lz, double g1, double g2, double eps0,
                            double sum_K, double *F3, int nch, unsigned *status, cudaStream_t s, int stage);
int qem_long_chunk(void);

cudaError_t qem_launch_reduce_sum(const double *in, int n, double *out, cudaStream_t s);
// out[i] += a[i] for n doubles
cudaError_t qem_launch_add3(int n, const double *a, double *out, cudaStream_t s);

// ---------------------------------------------------------------------------
// device helpers
// ---------------------------------------------------------------------------
#ifdef __CUDACC__
__device__ __forceinline__ double jl_sign(double v) { return (double)((v > 0) - (v < 0)); }

__device__ __forceinline__ double min_image(double d, double L, double invL) { return d - L * rint(d * invL); }

// Bessel J0 and J1 in FP32 from the polynomial approximations of
// Abramowitz & Stegun, Handbook of Mathematical Functions, 9.4.1 / 9.4.4
// (|x| <= 3) and 9.4.3 / 9.4.6 (x >= 3; modulus/phase form).  Published
// absolute error <= 5e-8 (J0) and <= 4e-8 (J1), i.e. at FP32 rounding level.
__device__ __forceinline__ void bessel01_f32(float x, float &J0, float &J1)
{
    if (x < 3.0f) {
        const float y = x * x * (1.0f / 9.0f);
        J0 = fmaf(y, fmaf(y, fmaf(y, fmaf(y, fmaf(y, fmaf(y, 0.0002100f, -0.0039444f), 0.0444479f), -0.3163866f),
                                   1.2656208f), -2.2499997f), 1.0f);
        J1 = x * fmaf(y, fmaf(y, fmaf(y, fmaf(y, fmaf(y, fmaf(y, 0.00001109f, -0.00031761f), 0.00443319f),
                                                -0.03954289f), 0.21093573f), -0.56249985f), 0.5f);
    } else {
        const float r = rsqrtf(x);
        const float t = 3.0f * r * r;  // 3 / x
        const float f0 = fmaf(t, fmaf(t, fmaf(t, fmaf(t, fmaf(t, fmaf(t, 0.00014476f, -0.00072805f), 0.00137237f),
                                                      -0.00009512f), -0.00552740f), -0.00000077f), 0.79788456f);
        const float p0 = t * fmaf(t, fmaf(t, fmaf(t, fmaf(t, fmaf(t, 0.00013558f, -0.00029333f), -0.00054125f),
                                                 0.00262573f), -0.00003954f), -0.04166397f);
        const float f1 = fmaf(t, fmaf(t, fmaf(t, fmaf(t, fmaf(t, fmaf(t, -0.00020033f, 0.00113653f), -0.00249511f),
                                                      0.00017105f), 0.01659667f), 0.00000156f), 0.79788456f);
        const float p1 = t * fmaf(t, fmaf(t, fmaf(t, fmaf(t, fmaf(t, -0.00029166f, 0.00079824f), 0.00074348f),
                                                 -0.00637879f), 0.00005650f), 0.12499612f);
        // theta = x - pi/4 + p0 and x - 3 pi/4 + p1, reduced modulo 2 pi in two
        // FMA steps (Cody-Waite split of 2 pi) before the hardware cosine.
        const float TWO_PI_HI = 6.28318548202514648f, TWO_PI_LO = -1.7484555314695172e-07f;
        float th0 = (x - 0.78539816f) + p0;
        float th1 = (x - 2.35619449f) + p1;
        float n0 = rintf(th0 * 0.15915494309189535f), n1 = rintf(th1 * 0.15915494309189535f);
        th0 = fmaf(-n0, TWO_PI_LO, fmaf(-n0, TWO_PI_HI, th0));
        th1 = fmaf(-n1, TWO_PI_LO, fmaf(-n1, TWO_PI_HI, th1));
        J0 = f0 * r * __cosf(th0);
        J1 = f1 * r * __cosf(th1);
    }
}

// 1 - exp(-t) for t >= 0 to FP32 relative precision without cancellation:
// Taylor series below 0.5 (truncation < 2e-8 relative), 1 - exp(-t) above.
__device__ __forceinline__ float one_minus_exp_neg(float t, float e)
{
    if (t < 0.5f) {
        float s = fmaf(t, -1.0f / 362880.0f, 1.0f / 40320.0f);
        s = fmaf(t, s, -1.0f / 5040.0f);
        s = fmaf(t, s, 1.0f / 720.0f);
        s = fmaf(t, s, -1.0f / 120.0f);
        s = fmaf(t, s, 1.0f / 24.0f);
        s = fmaf(t, s, -1.0f / 6.0f);
        s = fmaf(t, s, 0.5f);
        s = fmaf(t, -s, 1.0f);
        return t * s;
    }
    return 1.0f - e;
}

__device__ __forceinline__ float fast_rcp(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Kahan-compensated FP32 accumulation
struct KahanF {
    float s, c;
    __device__ __forceinline__ void init() { s = 0.f; c = 0.f; }
    __device__ __forceinline__ void add(float v)
    {
        float y = v - c;
        float t = s + y;
        c = (t - s) - y;
        s = t;
    }
};
#endif

// qem_long.cu -- random-batch long-range QEM forces and energies.
//
// Reference (ArrogantGao/QEM4Molly):
//   Fl_non_sort   src/Force_long.jl:5-70    structure sums, self excluded
//   Fl_sort       src/Force_long.jl:72-127  z-ordered prefix (A, B) / suffix (C, D) sums
//   Flz_sort_k0   src/Force_long.jl:130-161 k = 0 term
//   Flz_self      src/Force_long.jl:164-184 image self force
//   F_l_total     src/Force_long.jl:186-199
//   F_long        src/Force_long.jl:201-242 (random-batch branch)
//   energies      src/python_lib/Energy_long_range_njit.py:10-44,
//                 src/python_lib/Sigma_Gamma_func_njit.py:8-69
//
// Layout: particles in z order (stable sortperm), SoA, chunks of LCH
// consecutive particles.  Three passes per call:
//   1. k_ltot   grid (chunk, k-group): per (k, chunk) sums of
//               u = q e^{k(z-h)} e^{i k.rho} and v = q e^{-k(z-h)} e^{i k.rho}
//               (h = L_z / 2 keeps both exponentials inside FP32 range).
//   2. k_lscan  one thread per k: FP64 exclusive scan of the chunk totals,
//               forward for u (particles below) and backward for v (above).
//   3. k_lforce one block per chunk, loop over all k: block exclusive scans
//               (warp shuffles) give each particle its prefix / suffix sums,
//               the Fl_non_sort + Fl_sort + Flz_self terms are formed in
//               registers and accumulated over k (Kahan in FP32); one write
//               per particle, no atomics.
// The suffix sums C, D are summed directly from above instead of the
// reference's "total minus running sum" (Force_long.jl:97-98), which is the
// same quantity without the cancellation that makes it useless in FP32.
// Phases are reduced in FP64 turns before the FP32 sine/cosine; the per-k
// denominators 0.5 / (g_u g_d e^{-2 k L_z} - 1) are FP64.
#include "qem_internal.cuh"

namespace {

constexpr int LCH = 256;  // particles per chunk (= threads per block)
constexpr int KPB = 16;   // k-vectors per block in the totals pass

template <typename Real>
struct LM;
template <>
struct LM<float> {
    static __device__ __forceinline__ float ex(float x) { return __expf(x); }
    static __device__ __forceinline__ void sc(double turns, float &s, float &c)
    {
        __sincosf((float)turns * 6.28318530717958648f, &s, &c);
    }
};
template <>
struct LM<double> {
    static __device__ __forceinline__ double ex(double x) { return exp(x); }
    static __device__ __forceinline__ void sc(double turns, double &s, double &c) { sincospi(2.0 * turns, &s, &c); }
};

__global__ void k_kconst(int P, const double *__restrict__ kin, KConst *__restrict__ kc, double Lz, double g12,
                         double wk, double esc)
{
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= P) return;
    const double kx = kin[3 * m], ky = kin[3 * m + 1], k = kin[3 * m + 2];
    KConst K;
    K.kx_2pi = kx / (2.0 * QEM_PI);
    K.ky_2pi = ky / (2.0 * QEM_PI);
    K.k = k;
    K.W = exp(-0.5 * k * Lz);  // stored as sqrt(exp(-k L_z)); squared on use
    K.g = 0.5 / (g12 * exp(-2.0 * k * Lz) - 1.0);
    K.fx = kx / k;
    K.fy = ky / k;
    K.wk = wk;
    K.ek = esc / k;
    kc[m] = K;
}

// z-ordered SoA copy of the particles and the k = 0 term (Force_long.jl:130-161,
// Energy_long_range_njit.py:25-44)
__global__ void k_zgather(int N, const double4 *__restrict__ pos, const int *__restrict__ zperm, double h,
                          double *__restrict__ zx, double *__restrict__ zy, float *__restrict__ zhf,
                          double *__restrict__ zhd, float *__restrict__ qf, double *__restrict__ qd)
{
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= N) return;
    const double4 p = pos[zperm[m]];
    zx[m] = p.x;
    zy[m] = p.y;
    zhd[m] = p.z - h;
    zhf[m] = (float)(p.z - h);
    qd[m] = p.w;
    qf[m] = (float)p.w;
}

__global__ void k_k0(int N, const double *__restrict__ qd, const double *__restrict__ zhd, double h,
                     const double *__restrict__ qscan, double fscale, double escale, double *__restrict__ k0,
                     double *__restrict__ Epart, int energy)
{
    __shared__ double red[8];
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    double e = 0;
    if (m < N) {
        const double q = qd[m], below = qscan[m], tot = qscan[N];
        const double above = (tot - below) - q;
        k0[m] = q * (below - above) * fscale;
        // python literal: Q_a - Q_b = sum_{below} q + sum_{<= m} q
        e = 2.0 * q * (zhd[m] + h) * (below + (below + q)) * escale;
    }
    if (energy) {
        for (int d = 16; d > 0; d >>= 1) e += __shfl_down_sync(0xffffffffu, e, d);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = e;
        __syncthreads();
        if (threadIdx.x == 0) {
            double s = 0;
            for (int w = 0; w < 8; w++) s += red[w];
            Epart[blockIdx.x] = s;
        }
    }
}

template <typename Real>
__global__ void __launch_bounds__(LCH) k_ltot(int N, int P, int nch, const double *__restrict__ zx,
                                               const double *__restrict__ zy, const Real *__restrict__ zh,
                                               const Real *__restrict__ qv, const KConst *__restrict__ kc,
                                               double *__restrict__ tot)
{
    __shared__ Real red[4][LCH / 32];
    const int m = blockIdx.x * LCH + threadIdx.x;
    const bool valid = m < N;
    const double x = valid ? zx[m] : 0.0, y = valid ? zy[m] : 0.0;
    const Real z = valid ? zh[m] : (Real)0, q = valid ? qv[m] : (Real)0;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int kk = 0; kk < KPB; kk++) {
        const int kidx = blockIdx.y * KPB + kk;
        if (kidx >= P) break;
        const KConst K = kc[kidx];
        double t = fma(K.kx_2pi, x, K.ky_2pi * y);
        t -= rint(t);
        Real s, c;
        LM<Real>::sc(t, s, c);
        const Real kz = (Real)K.k * z;
        const Real ep = q * LM<Real>::ex(kz), em = q * LM<Real>::ex(-kz);
        Real v[4] = {ep * c, ep * s, em * c, em * s};
#pragma unroll
        for (int j = 0; j < 4; j++) {
#pragma unroll
            for (int d = 16; d > 0; d >>= 1) v[j] += __shfl_down_sync(0xffffffffu, v[j], d);
        }
        if (lane == 0) {
#pragma unroll
            for (int j = 0; j < 4; j++) red[j][w] = v[j];
        }
        __syncthreads();
        if (threadIdx.x < 4) {
            double sum = 0;
            for (int ww = 0; ww < LCH / 32; ww++) sum += (double)red[threadIdx.x][ww];
            tot[((int64_t)kidx * nch + blockIdx.x) * 4 + threadIdx.x] = sum;
        }
        __syncthreads();
    }
}

__global__ void k_lscan(int P, int nch, const double *__restrict__ tot, double *__restrict__ off,
                        double *__restrict__ Utot, const KConst *__restrict__ kc, double g1, double g2,
                        double *__restrict__ Eks)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= P) return;
    const double *T = tot + (int64_t)m * nch * 4;
    double *O = off + (int64_t)m * nch * 4;
    double ur = 0, ui = 0;
    for (int c = 0; c < nch; c++) {
        O[4 * c] = ur;
        O[4 * c + 1] = ui;
        ur += T[4 * c];
        ui += T[4 * c + 1];
    }
    double vr = 0, vi = 0;
    for (int c = nch - 1; c >= 0; c--) {
        O[4 * c + 2] = vr;
        O[4 * c + 3] = vi;
        vr += T[4 * c + 2];
        vi += T[4 * c + 3];
    }
    Utot[4 * m] = ur;
    Utot[4 * m + 1] = ui;
    Utot[4 * m + 2] = vr;
    Utot[4 * m + 3] = vi;
    // split energy term Sigma_Gamma_func_s (Sigma_Gamma_func_njit.py:8-28) in scaled sums
    const KConst K = kc[m];
    const double W = K.W * K.W;
    const double sig = K.g * (g2 * W * (ur * ur + ui * ui) + g1 * W * (vr * vr + vi * vi) +
                              g1 * g2 * W * W * (ur * vr + ui * vi));
    Eks[m] = K.ek * sig;
}

template <typename Real>
struct Acc;
template <>
struct Acc<float> {
    KahanF a;
    __device__ __forceinline__ void init() { a.init(); }
    __device__ __forceinline__ void add(float v) { a.add(v); }
    __device__ __forceinline__ double get() const { return (double)a.s - (double)a.c; }
};
template <>
struct Acc<double> {
    double a;
    __device__ __forceinline__ void init() { a = 0; }
    __device__ __forceinline__ void add(double v) { a += v; }
    __device__ __forceinline__ double get() const { return a; }
};

template <typename Real, bool ENERGY>
__global__ void __launch_bounds__(LCH) k_lforce(int N, int P, int nch, const double *__restrict__ zx,
                                                 const double *__restrict__ zy, const Real *__restrict__ zh,
                                                 const Real *__restrict__ qv, const KConst *__restrict__ kc,
                                                 const double *__restrict__ off, const double *__restrict__ Utot,
                                                 const double *__restrict__ k0, const int *__restrict__ zperm,
                                                 double g1, double g2, double *__restrict__ F3,
                                                 double *__restrict__ Epart)
{
    __shared__ Real wf[2][2][LCH / 32];  // [buffer][re/im] forward warp totals
    __shared__ Real wb[2][2][LCH / 32];  // backward warp totals
    __shared__ double ered[LCH / 32];
    const int m = blockIdx.x * LCH + threadIdx.x;
    const bool valid = m < N;
    const double x = valid ? zx[m] : 0.0, y = valid ? zy[m] : 0.0;
    const Real z = valid ? zh[m] : (Real)0, q = valid ? qv[m] : (Real)0;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const Real G1 = (Real)g1, G2 = (Real)g2, G12 = (Real)(g1 * g2);
    Acc<Real> ax, ay, az;
    ax.init(); ay.init(); az.init();
    double E = 0;
    for (int kidx = 0; kidx < P; kidx++) {
        const KConst K = kc[kidx];
        const int buf = kidx & 1;
        double t = fma(K.kx_2pi, x, K.ky_2pi * y);
        t -= rint(t);
        Real s, c;
        LM<Real>::sc(t, s, c);
        const Real kz = (Real)K.k * z;
        const Real ep = LM<Real>::ex(kz), em = LM<Real>::ex(-kz);
        const Real ur = q * ep * c, ui = q * ep * s, vr = q * em * c, vi = q * em * s;
        // warp inclusive scans: forward for u, backward for v
        Real fr = ur, fi = ui, br = vr, bi = vi;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const Real a1 = __shfl_up_sync(0xffffffffu, fr, d), a2 = __shfl_up_sync(0xffffffffu, fi, d);
            const Real b1 = __shfl_down_sync(0xffffffffu, br, d), b2 = __shfl_down_sync(0xffffffffu, bi, d);
            if (lane >= d) { fr += a1; fi += a2; }
            if (lane + d < 32) { br += b1; bi += b2; }
        }
        if (lane == 31) { wf[buf][0][w] = fr; wf[buf][1][w] = fi; }
        if (lane == 0) { wb[buf][0][w] = br; wb[buf][1][w] = bi; }
        // exclusive in-warp values by shifting the inclusive ones (no subtraction)
        Real exr = __shfl_up_sync(0xffffffffu, fr, 1), exi = __shfl_up_sync(0xffffffffu, fi, 1);
        Real eyr = __shfl_down_sync(0xffffffffu, br, 1), eyi = __shfl_down_sync(0xffffffffu, bi, 1);
        if (lane == 0) { exr = 0; exi = 0; }
        if (lane == 31) { eyr = 0; eyi = 0; }
        __syncthreads();
        Real pr = 0, pim = 0, sr = 0, sim = 0;
        for (int ww = 0; ww < w; ww++) { pr += wf[buf][0][ww]; pim += wf[buf][1][ww]; }
        for (int ww = LCH / 32 - 1; ww > w; ww--) { sr += wb[buf][0][ww]; sim += wb[buf][1][ww]; }
        const double *O = off + ((int64_t)kidx * nch + blockIdx.x) * 4;
        const double *U = Utot + 4 * kidx;
        // prefix (A, B) of particles below and suffix (C, D) of particles above, in
        // the scaled form A' = sum q e^{k(z - h)} cos, C' = sum q e^{-k(z - h)} cos
        const Real A = (Real)O[0] + (pr + exr), B = (Real)O[1] + (pim + exi);
        const Real Cs = (Real)O[2] + (sr + eyr), Ds = (Real)O[3] + (sim + eyi);
        // totals with the particle's own term removed (Force_long.jl:33-36)
        const Real f1 = (Real)U[0] - ur, f2 = (Real)U[1] - ui, f3 = (Real)U[2] - vr, f4 = (Real)U[3] - vi;
        const Real Wh = (Real)K.W;
        const Real Xp = (Wh * ep) * Wh, Xm = (Wh * em) * Wh;  // e^{-kLz} e^{+-k(z-h)}
        const Real Wf = Wh * Wh;
        const Real Yp = Xp * Wf, Ym = Xm * Wf;                  // e^{-2kLz} e^{+-k(z-h)}
        const Real g = (Real)K.g;
        // Fl_non_sort (Force_long.jl:39-64)
        const Real P1 = G2 * Xp + G12 * Ym, P2 = G1 * Xm + G12 * Yp;
        const Real Q1 = G2 * Xp - G12 * Ym, Q2 = G12 * Yp - G1 * Xm;
        const Real xy_ns = q * g * (c * (P1 * f2 + P2 * f4) - s * (P1 * f1 + P2 * f3));
        const Real z_ns = q * g * (c * (Q1 * f1 + Q2 * f3) + s * (Q1 * f2 + Q2 * f4));
        // Fl_sort (Force_long.jl:103-121)
        const Real xy_s = em * (s * A - c * B) + ep * (s * Cs - c * Ds);
        const Real cAB = c * A + s * B, cCD = c * Cs + s * Ds;
        const Real z_s = (Real)0.5 * q * (em * cAB - ep * cCD);
        // Flz_self (Force_long.jl:180)
        const Real z_self = q * q * g * (G2 * Xp * ep - G1 * Xm * em);
        const Real wk = (Real)K.wk;
        const Real xy = xy_ns + (Real)0.5 * q * xy_s;
        ax.add(wk * (Real)K.fx * xy);
        ay.add(wk * (Real)K.fy * xy);
        az.add(wk * (z_ns + z_s + z_self));
        if (ENERGY) E += K.ek * 0.5 * (double)(-q * q - q * (em * cAB + ep * cCD));
    }
    if (valid) {
        const int i = zperm[m];
        F3[3 * i] += ax.get();
        F3[3 * i + 1] += ay.get();
        F3[3 * i + 2] += az.get() + k0[m];
    }
    if (ENERGY) {
        for (int d = 16; d > 0; d >>= 1) E += __shfl_down_sync(0xffffffffu, E, d);
        if (lane == 0) ered[w] = E;
        __syncthreads();
        if (threadIdx.x == 0) {
            double sum = 0;
            for (int ww = 0; ww < LCH / 32; ww++) sum += ered[ww];
            Epart[blockIdx.x] = sum;
        }
    }
}

__global__ void k_add3(int n, const double *__restrict__ a, double *__restrict__ out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += a[i];
}

__global__ void k_reduce_sum(const double *__restrict__ in, int n, double *__restrict__ out)
{
    // single block, fixed order: deterministic
    __shared__ double red[1024 / 32];
    double s = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += in[i];
    for (int d = 16; d > 0; d >>= 1) s += __shfl_down_sync(0xffffffffu, s, d);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int w = 0; w < (int)(blockDim.x / 32); w++) t += red[w];
        *out = t;
    }
}

inline int nblk(int64_t n, int b) { return (int)((n + b - 1) / b); }

}  // namespace

int qem_long_chunk(void) { return LCH; }

// Long range for N particles and P k-vectors; adds into F3 (original order).
// Energy partials: b.Epart[0 .. nch) from k_lforce, [nch .. nch + nk0) from
// k_k0 and the P split terms in b.Eks.
cudaError_t qem_launch_long(int precision, bool energy, int N, int P, const double4 *pos, const int *zperm,
                            const LongBuffers &b, double Lx, double Ly, double Lz, double g1, double g2, double eps0,
                            double sum_K, double *F3, int nch, unsigned *status, cudaStream_t s, int stage)
{
    (void)status;
    if (N <= 0) return cudaSuccess;
    if (stage == 1) goto force_pass;
    {
    const double h = 0.5 * Lz;
    k_zgather<<<nblk(N, 256), 256, 0, s>>>(N, pos, zperm, h, b.zx, b.zy, b.zhf, b.zhd, b.qf, b.qd);
    cudaError_t e = qem_scan_f64_excl(b.qd, b.qscan, N, b.stmp, b.stmp_bytes, s);
    if (e != cudaSuccess) return e;
    const double fscale = 1.0 / (2.0 * Lx * Ly * eps0);
    const double escale = -1.0 / (4.0 * eps0 * Lx * Ly);
    k_k0<<<nblk(N, 256), 256, 0, s>>>(N, b.qd, b.zhd, h, b.qscan, fscale, escale, b.k0, b.Epart + nch, energy ? 1 : 0);
    if (P > 0) {
        const double wk = (sum_K / P) / (Lx * Ly * eps0);
        const double esc = -(sum_K / P) / (2.0 * eps0 * Lx * Ly);
        k_kconst<<<nblk(P, 128), 128, 0, s>>>(P, b.kin, b.kc, Lz, g1 * g2, wk, esc);
        dim3 g1d(nch, nblk(P, KPB));
        if (precision == QEM_FP64)
            k_ltot<double><<<g1d, LCH, 0, s>>>(N, P, nch, b.zx, b.zy, b.zhd, b.qd, b.kc, b.tot);
        else
            k_ltot<float><<<g1d, LCH, 0, s>>>(N, P, nch, b.zx, b.zy, b.zhf, b.qf, b.kc, b.tot);
        k_lscan<<<nblk(P, 64), 64, 0, s>>>(P, nch, b.tot, b.off, b.Utot, b.kc, g1, g2, b.Eks);
    }
    }
    if (stage == 0) return cudaGetLastError();
force_pass:
    if (precision == QEM_FP64) {
        if (energy)
            k_lforce<double, true><<<nch, LCH, 0, s>>>(N, P, nch, b.zx, b.zy, b.zhd, b.qd, b.kc, b.off, b.Utot, b.k0,
                                                       zperm, g1, g2, F3, b.Epart);
        else
            k_lforce<double, false><<<nch, LCH, 0, s>>>(N, P, nch, b.zx, b.zy, b.zhd, b.qd, b.kc, b.off, b.Utot,
                                                        b.k0, zperm, g1, g2, F3, b.Epart);
    } else {
        if (energy)
            k_lforce<float, true><<<nch, LCH, 0, s>>>(N, P, nch, b.zx, b.zy, b.zhf, b.qf, b.kc, b.off, b.Utot, b.k0,
                                                      zperm, g1, g2, F3, b.Epart);
        else
            k_lforce<float, false><<<nch, LCH, 0, s>>>(N, P, nch, b.zx, b.zy, b.zhf, b.qf, b.kc, b.off, b.Utot,
                                                       b.k0, zperm, g1, g2, F3, b.Epart);
    }
    return cudaGetLastError();
}

cudaError_t qem_launch_add3(int n, const double *a, double *out, cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    k_add3<<<nblk(n, 256), 256, 0, s>>>(n, a, out);
    return cudaGetLastError();
}

cudaError_t qem_launch_reduce_sum(const double *in, int n, double *out, cudaStream_t s)
{
    k_reduce_sum<<<1, 1024, 0, s>>>(in, n, out);
    return cudaGetLastError();
}

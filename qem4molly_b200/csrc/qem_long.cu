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
// Layout: particles in z order (stable sortperm), SoA, chunks of LCH = 512
// consecutive particles; a thread owns PPT = 4 consecutive particles.
//   1. k_ltot   grid (chunk, k-group): per (k, chunk) sums of
//               u = q e^{k(z-h)} e^{i k.rho} and v = q e^{-k(z-h)} e^{i k.rho}
//               (h = L_z / 2 keeps both exponentials inside FP32 range).
//   2. k_lscan  one warp per k: FP64 exclusive scan of the chunk totals,
//               forward for u (particles below) and backward for v (above).
//   3. k_lforce grid (chunk, k-slice): per k, serial scans over the thread's
//               4 particles, one warp shuffle scan of the thread totals and a
//               4-warp prefix give every particle its prefix (A, B) and suffix
//               (C, D) sums; Fl_non_sort + Fl_sort + Flz_self are formed in
//               registers and summed over the slice's k in FP64.
//   4. k_lfinal per particle: sum of the k-slices + the k = 0 term, added to F
//               in the original particle order (fixed order: deterministic).
// The suffix sums C, D are summed directly from above instead of the
// reference's "total minus running sum" (Force_long.jl:97-98), which is the
// same quantity without the cancellation that makes it useless in FP32.
// Phases are reduced in FP64 turns before the FP32 sine/cosine; the per-k
// denominators 0.5 / (g_u g_d e^{-2 k L_z} - 1) are FP64.
#include "qem_internal.cuh"

namespace {

constexpr int LT = 128;         // threads per block
constexpr int PPT = 4;          // particles per thread
constexpr int LCH = LT * PPT;   // particles per chunk
constexpr int NW = LT / 32;     // warps per block
constexpr int KPB = 16;         // k-vectors per block in the totals pass
constexpr int LKB = 8;          // k-vectors per FP32 accumulation batch of the force pass
#ifndef QEM_LF_MINB
#define QEM_LF_MINB 6
#endif
constexpr int LF_MINB = QEM_LF_MINB;  // resident FP32 force-pass blocks per SM (register budget)

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
    K.W = exp(-0.5 * k * Lz);  // sqrt(exp(-k L_z)); squared on use
    K.g = 0.5 / (g12 * exp(-2.0 * k * Lz) - 1.0);
    K.fx = kx / k;
    K.fy = ky / k;
    K.wk = wk;
    K.ek = esc / k;
    kc[m] = K;
}

// z-ordered SoA copy of the particles
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

// k = 0 term (Force_long.jl:130-161, Energy_long_range_njit.py:25-44)
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

// a thread's PPT particles in z order
template <typename Real>
struct Quad4 {
    double x[PPT], y[PPT];
    Real z[PPT], q[PPT];
    __device__ __forceinline__ void load(int N, int m0, const double *zx, const double *zy, const Real *zh,
                                         const Real *qv)
    {
#pragma unroll
        for (int j = 0; j < PPT; j++) {
            const int m = m0 + j;
            const bool ok = m < N;
            x[j] = ok ? zx[m] : 0.0;
            y[j] = ok ? zy[m] : 0.0;
            z[j] = ok ? zh[m] : (Real)0;
            q[j] = ok ? qv[m] : (Real)0;  // q = 0 makes padding particles contribute nothing
        }
    }
};

template <typename Real>
__global__ void __launch_bounds__(LT) k_ltot(int N, int P, int nch, const double *__restrict__ zx,
                                             const double *__restrict__ zy, const Real *__restrict__ zh,
                                             const Real *__restrict__ qv, const KConst *__restrict__ kc,
                                             double *__restrict__ tot)
{
    __shared__ Real red[4][NW];
    Quad4<Real> P4;
    P4.load(N, blockIdx.x * LCH + threadIdx.x * PPT, zx, zy, zh, qv);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int kk = 0; kk < KPB; kk++) {
        const int kidx = blockIdx.y * KPB + kk;
        if (kidx >= P) break;
        const KConst K = kc[kidx];
        Real v[4] = {0, 0, 0, 0};
#pragma unroll
        for (int j = 0; j < PPT; j++) {
            double t = fma(K.kx_2pi, P4.x[j], K.ky_2pi * P4.y[j]);
            t -= rint(t);
            Real s, c;
            LM<Real>::sc(t, s, c);
            const Real kz = (Real)K.k * P4.z[j];
            const Real ep = P4.q[j] * LM<Real>::ex(kz), em = P4.q[j] * LM<Real>::ex(-kz);
            v[0] += ep * c; v[1] += ep * s; v[2] += em * c; v[3] += em * s;
        }
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
#pragma unroll
            for (int ww = 0; ww < NW; ww++) sum += (double)red[threadIdx.x][ww];
            tot[((int64_t)kidx * nch + blockIdx.x) * 4 + threadIdx.x] = sum;
        }
        __syncthreads();
    }
}

// one warp per k: exclusive scans of the chunk totals (FP64), written in the
// force pass's precision, and the per-k force constants
template <typename Real>
__global__ void k_lscan(int P, int nch, const double *__restrict__ tot, Real *__restrict__ off,
                        double *__restrict__ Utot, const KConst *__restrict__ kc, double g1, double g2,
                        double *__restrict__ Eks, KForce<Real> *__restrict__ kf)
{
    const int lane = threadIdx.x & 31;
    const int m = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (m >= P) return;
    const double *T = tot + (int64_t)m * nch * 4;
    Real *O = off + (int64_t)m * nch * 4;
    double cr = 0, ci = 0;  // forward carry: u below
    for (int base = 0; base < nch; base += 32) {
        const int c = base + lane;
        double r = c < nch ? T[4 * c] : 0.0, i = c < nch ? T[4 * c + 1] : 0.0;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const double a = __shfl_up_sync(0xffffffffu, r, d), b = __shfl_up_sync(0xffffffffu, i, d);
            if (lane >= d) { r += a; i += b; }
        }
        double er = __shfl_up_sync(0xffffffffu, r, 1), ei = __shfl_up_sync(0xffffffffu, i, 1);
        if (lane == 0) { er = 0; ei = 0; }
        if (c < nch) { O[4 * c] = (Real)(cr + er); O[4 * c + 1] = (Real)(ci + ei); }
        cr += __shfl_sync(0xffffffffu, r, 31);
        ci += __shfl_sync(0xffffffffu, i, 31);
    }
    double dr = 0, di = 0;  // backward carry: v above
    for (int base = 0; base < nch; base += 32) {
        const int c = nch - 1 - (base + lane);
        double r = c >= 0 ? T[4 * c + 2] : 0.0, i = c >= 0 ? T[4 * c + 3] : 0.0;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const double a = __shfl_up_sync(0xffffffffu, r, d), b = __shfl_up_sync(0xffffffffu, i, d);
            if (lane >= d) { r += a; i += b; }
        }
        double er = __shfl_up_sync(0xffffffffu, r, 1), ei = __shfl_up_sync(0xffffffffu, i, 1);
        if (lane == 0) { er = 0; ei = 0; }
        if (c >= 0) { O[4 * c + 2] = (Real)(dr + er); O[4 * c + 3] = (Real)(di + ei); }
        dr += __shfl_sync(0xffffffffu, r, 31);
        di += __shfl_sync(0xffffffffu, i, 31);
    }
    if (lane == 0) {
        Utot[4 * m] = cr;
        Utot[4 * m + 1] = ci;
        Utot[4 * m + 2] = dr;
        Utot[4 * m + 3] = di;
        const KConst K = kc[m];
        const double W = K.W * K.W;  // e^{-k L_z}
        // split energy term Sigma_Gamma_func_s (Sigma_Gamma_func_njit.py:8-28) in scaled sums
        const double sig = K.g * (g2 * W * (cr * cr + ci * ci) + g1 * W * (dr * dr + di * di) +
                                  g1 * g2 * W * W * (cr * dr + ci * di));
        Eks[m] = K.ek * sig;
        // force constants: S1 = g W (g2 U + g12 W V), S2 = g W (g12 W U + g1 V)
        const double gW = K.g * W, g12W = g1 * g2 * W;
        KForce<Real> F;
        F.k = (Real)K.k;
        F.wfx = (Real)(K.wk * K.fx);
        F.wfy = (Real)(K.wk * K.fy);
        F.wk = (Real)K.wk;
        F.s1r = (Real)(gW * (g2 * cr + g12W * dr));
        F.s1i = (Real)(gW * (g2 * ci + g12W * di));
        F.s2r = (Real)(gW * (g12W * cr + g1 * dr));
        F.s2i = (Real)(gW * (g12W * ci + g1 * di));
        kf[m] = F;
    }
}

// Force pass.  For particle j with phase e^{i theta} = c + i s, ep = e^{k(z-h)},
// em = e^{-k(z-h)}, prefix A = sum_{below} q ep e^{i theta} and suffix
// C = sum_{above} q em e^{i theta} (complex), the reference's per-k terms
// (Force_long.jl:39-64 Fl_non_sort with the particle's own term removed,
// 103-121 Fl_sort, 180 Flz_self) sum to
//   F_xy = w_k q Im[e^{-i theta} X1],  F_z = w_k q Re[e^{-i theta} X2],
//   X1 = ep a + em b,  X2 = ep a - em b,  a = S1 - C / 2,  b = S2 - A / 2,
// with the per-k constants S1, S2 of k_lscan: the own-term removal of the
// non-sorted sum only changes the real part, and there it cancels the self
// image force exactly.  The sums over k run in Real in batches of KB
// k-vectors, each batch added into FP64; the common factor q is applied at
// the end.  Slices and batches cover whole groups of LKB consecutive k, so
// the batches are the same for every number of slices.
template <typename Real, bool ENERGY>
__global__ void __launch_bounds__(LT, sizeof(Real) == 4 ? LF_MINB : 4) k_lforce(int N, int P, int nch, int ks_n,
                                                       const double *__restrict__ zx, const double *__restrict__ zy,
                                                       const Real *__restrict__ zh, const Real *__restrict__ qv,
                                                       const KConst *__restrict__ kc,
                                                       const KForce<Real> *__restrict__ kf,
                                                       const Real *__restrict__ off, double *__restrict__ Fpart,
                                                       double *__restrict__ Epart)
{
    __shared__ Real wsh[2][4][NW];  // [buffer][fwd re, fwd im, bwd re, bwd im][warp]
    __shared__ double ered[NW];
    Quad4<Real> P4;
    const int m0 = blockIdx.x * LCH + threadIdx.x * PPT;
    P4.load(N, m0, zx, zy, zh, qv);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int ks = blockIdx.y;
    const int ng = (P + LKB - 1) / LKB;
    const int kb = LKB * (int)((int64_t)ng * ks / ks_n);
    const int ke = min(P, LKB * (int)((int64_t)ng * (ks + 1) / ks_n));
    double Fx[PPT], Fy[PPT], Fz[PPT];
    Real bx[PPT], by[PPT], bz[PPT];
#pragma unroll
    for (int j = 0; j < PPT; j++) { Fx[j] = 0; Fy[j] = 0; Fz[j] = 0; bx[j] = 0; by[j] = 0; bz[j] = 0; }
    double E = 0;
    for (int kidx = kb; kidx < ke; kidx++) {
        const double kx2 = kc[kidx].kx_2pi, ky2 = kc[kidx].ky_2pi;
        const KForce<Real> K = kf[kidx];
        const int buf = (kidx - kb) & 1;
        Real c[PPT], s[PPT], ep[PPT], em[PPT], ur[PPT], ui[PPT], vr[PPT], vi[PPT];
#pragma unroll
        for (int j = 0; j < PPT; j++) {
            double t = fma(kx2, P4.x[j], ky2 * P4.y[j]);
            t -= rint(t);
            LM<Real>::sc(t, s[j], c[j]);
            const Real kz = K.k * P4.z[j];
            ep[j] = LM<Real>::ex(kz);
            em[j] = LM<Real>::ex(-kz);
            const Real qp = P4.q[j] * ep[j], qm = P4.q[j] * em[j];
            ur[j] = qp * c[j]; ui[j] = qp * s[j];
            vr[j] = qm * c[j]; vi[j] = qm * s[j];
        }
        // in-thread exclusive prefix (u, from below) and suffix (v, from above)
        Real Ar[PPT], Ai[PPT], Cr[PPT], Ci[PPT];
        Real tr = 0, ti = 0, br = 0, bi = 0;
#pragma unroll
        for (int j = 0; j < PPT; j++) { Ar[j] = tr; Ai[j] = ti; tr += ur[j]; ti += ui[j]; }
#pragma unroll
        for (int j = PPT - 1; j >= 0; j--) { Cr[j] = br; Ci[j] = bi; br += vr[j]; bi += vi[j]; }
        // warp inclusive scans of the thread totals: forward for u, backward for v
        Real fr = tr, fi = ti, gr = br, gi = bi;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const Real a1 = __shfl_up_sync(0xffffffffu, fr, d), a2 = __shfl_up_sync(0xffffffffu, fi, d);
            const Real b1 = __shfl_down_sync(0xffffffffu, gr, d), b2 = __shfl_down_sync(0xffffffffu, gi, d);
            if (lane >= d) { fr += a1; fi += a2; }
            if (lane + d < 32) { gr += b1; gi += b2; }
        }
        if (lane == 31) { wsh[buf][0][w] = fr; wsh[buf][1][w] = fi; }
        if (lane == 0) { wsh[buf][2][w] = gr; wsh[buf][3][w] = gi; }
        // exclusive values by shifting the inclusive ones (no subtraction)
        Real xr = __shfl_up_sync(0xffffffffu, fr, 1), xi = __shfl_up_sync(0xffffffffu, fi, 1);
        Real yr = __shfl_down_sync(0xffffffffu, gr, 1), yi = __shfl_down_sync(0xffffffffu, gi, 1);
        if (lane == 0) { xr = 0; xi = 0; }
        if (lane == 31) { yr = 0; yi = 0; }
        __syncthreads();
#pragma unroll
        for (int ww = 0; ww < NW; ww++) {
            if (ww < w) { xr += wsh[buf][0][ww]; xi += wsh[buf][1][ww]; }
            if (ww > w) { yr += wsh[buf][2][ww]; yi += wsh[buf][3][ww]; }
        }
        const Real *O = off + ((int64_t)kidx * nch + blockIdx.x) * 4;
        const Real bAr = O[0] + xr, bAi = O[1] + xi, bCr = O[2] + yr, bCi = O[3] + yi;
        const double ek = ENERGY ? kc[kidx].ek : 0.0;
#pragma unroll
        for (int j = 0; j < PPT; j++) {
            const Real A_r = bAr + Ar[j], A_i = bAi + Ai[j], C_r = bCr + Cr[j], C_i = bCi + Ci[j];
            const Real ar = K.s1r - (Real)0.5 * C_r, ai = K.s1i - (Real)0.5 * C_i;
            const Real br_ = K.s2r - (Real)0.5 * A_r, bi_ = K.s2i - (Real)0.5 * A_i;
            const Real pr = ep[j] * ar, pi = ep[j] * ai, mr = em[j] * br_, mi = em[j] * bi_;
            const Real im1 = c[j] * (pi + mi) - s[j] * (pr + mr);  // Im[e^{-i theta} X1]
            const Real re2 = c[j] * (pr - mr) + s[j] * (pi - mi);  // Re[e^{-i theta} X2]
            bx[j] += K.wfx * im1;
            by[j] += K.wfy * im1;
            bz[j] += K.wk * re2;
            if (ENERGY) {
                // Energy_long_range_njit.py:10-24 (sorted part), Re[e^{-i theta}(em A + ep C)]
                const Real q = P4.q[j];
                const Real zr = em[j] * A_r + ep[j] * C_r, zi = em[j] * A_i + ep[j] * C_i;
                E += ek * 0.5 * (double)(-q * q - q * (c[j] * zr + s[j] * zi));
            }
        }
        if ((kidx + 1) % LKB == 0) {
#pragma unroll
            for (int j = 0; j < PPT; j++) {
                Fx[j] += (double)bx[j]; Fy[j] += (double)by[j]; Fz[j] += (double)bz[j];
                bx[j] = 0; by[j] = 0; bz[j] = 0;
            }
        }
    }
#pragma unroll
    for (int j = 0; j < PPT; j++) {
        const int m = m0 + j;
        if (m < N) {
            const double q = (double)P4.q[j];
            double *o = Fpart + ((int64_t)ks * N + m) * 3;
            o[0] = q * (Fx[j] + (double)bx[j]);
            o[1] = q * (Fy[j] + (double)by[j]);
            o[2] = q * (Fz[j] + (double)bz[j]);
        }
    }
    if (ENERGY) {
        for (int d = 16; d > 0; d >>= 1) E += __shfl_down_sync(0xffffffffu, E, d);
        if (lane == 0) ered[w] = E;
        __syncthreads();
        if (threadIdx.x == 0) {
            double sum = 0;
            for (int ww = 0; ww < NW; ww++) sum += ered[ww];
            Epart[(int64_t)ks * nch + blockIdx.x] = sum;
        }
    }
}

// F[zperm[m]] += sum over k-slices (fixed order) + k = 0 term
__global__ void k_lfinal(int N, int ks_n, const double *__restrict__ Fpart, const double *__restrict__ k0,
                         const int *__restrict__ zperm, double *__restrict__ F3)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= N) return;
    double fx = 0, fy = 0, fz = 0;
    for (int ks = 0; ks < ks_n; ks++) {
        const double *o = Fpart + ((int64_t)ks * N + m) * 3;
        fx += o[0];
        fy += o[1];
        fz += o[2];
    }
    const int i = zperm[m];
    F3[3 * i] += fx;
    F3[3 * i + 1] += fy;
    F3[3 * i + 2] += fz + k0[m];
}

__global__ void k_add(int n, const double *__restrict__ a, double *__restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
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

int qem_long_ksplit(int nch, int P, int max_ks)
{
    int ks = (4 * 148 + nch - 1) / nch;  // enough blocks for every SM
    ks = ks < 1 ? 1 : (ks > max_ks ? max_ks : ks);
    const int pm = P > LKB ? (P + LKB - 1) / LKB : 1;  // at most one slice per k group
    return ks < pm ? ks : pm;
}

// Energy partials: b.Epart[0 .. ks * nch) from k_lforce, [ks * nch .. + nb0)
// from k_k0; the P split terms go to b.Eks.
cudaError_t qem_launch_long(int precision, bool energy, int N, int P, const double4 *pos, const int *zperm,
                            const LongBuffers &b, double Lx, double Ly, double Lz, double g1, double g2, double eps0,
                            double sum_K, double *F3, int nch, unsigned *status, cudaStream_t s, int stage)
{
    (void)status;
    if (N <= 0) return cudaSuccess;
    if (stage == 0) {
        const double h = 0.5 * Lz;
        k_zgather<<<nblk(N, 256), 256, 0, s>>>(N, pos, zperm, h, b.zx, b.zy, b.zhf, b.zhd, b.qf, b.qd);
        cudaError_t e = qem_scan_f64_excl(b.qd, b.qscan, N, b.stmp, b.stmp_bytes, s);
        if (e != cudaSuccess) return e;
        const double fscale = 1.0 / (2.0 * Lx * Ly * eps0);
        const double escale = -1.0 / (4.0 * eps0 * Lx * Ly);
        k_k0<<<nblk(N, 256), 256, 0, s>>>(N, b.qd, b.zhd, h, b.qscan, fscale, escale, b.k0, b.Epart + b.ks * nch,
                                          energy ? 1 : 0);
        if (P > 0) {
            const double wk = (sum_K / P) / (Lx * Ly * eps0);
            const double esc = -(sum_K / P) / (2.0 * eps0 * Lx * Ly);
            k_kconst<<<nblk(P, 128), 128, 0, s>>>(P, b.kin, b.kc, Lz, g1 * g2, wk, esc);
            dim3 gt(nch, nblk(P, KPB));
            if (precision == QEM_FP64)
                k_ltot<double><<<gt, LT, 0, s>>>(N, P, nch, b.zx, b.zy, b.zhd, b.qd, b.kc, b.tot);
            else
                k_ltot<float><<<gt, LT, 0, s>>>(N, P, nch, b.zx, b.zy, b.zhf, b.qf, b.kc, b.tot);
            if (precision == QEM_FP64)
                k_lscan<double><<<nblk(P, 4), 128, 0, s>>>(P, nch, b.tot, b.off, b.Utot, b.kc, g1, g2, b.Eks,
                                                           (KForce<double> *)b.kf);
            else
                k_lscan<float><<<nblk(P, 4), 128, 0, s>>>(P, nch, b.tot, (float *)b.off, b.Utot, b.kc, g1, g2,
                                                          b.Eks, (KForce<float> *)b.kf);
        }
        return cudaGetLastError();
    }
    dim3 gf(nch, b.ks);
    if (precision == QEM_FP64) {
        const KForce<double> *kf = (const KForce<double> *)b.kf;
        if (energy)
            k_lforce<double, true><<<gf, LT, 0, s>>>(N, P, nch, b.ks, b.zx, b.zy, b.zhd, b.qd, b.kc, kf, b.off,
                                                     b.Fpart, b.Epart);
        else
            k_lforce<double, false><<<gf, LT, 0, s>>>(N, P, nch, b.ks, b.zx, b.zy, b.zhd, b.qd, b.kc, kf, b.off,
                                                      b.Fpart, b.Epart);
    } else {
        const KForce<float> *kf = (const KForce<float> *)b.kf;
        const float *of = (const float *)b.off;
        if (energy)
            k_lforce<float, true><<<gf, LT, 0, s>>>(N, P, nch, b.ks, b.zx, b.zy, b.zhf, b.qf, b.kc, kf, of,
                                                    b.Fpart, b.Epart);
        else
            k_lforce<float, false><<<gf, LT, 0, s>>>(N, P, nch, b.ks, b.zx, b.zy, b.zhf, b.qf, b.kc, kf, of,
                                                     b.Fpart, b.Epart);
    }
    k_lfinal<<<nblk(N, 256), 256, 0, s>>>(N, b.ks, b.Fpart, b.k0, zperm, F3);
    return cudaGetLastError();
}

cudaError_t qem_launch_add3(int n, const double *a, double *out, cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    k_add<<<nblk(n, 256), 256, 0, s>>>(n, a, out);
    return cudaGetLastError();
}

cudaError_t qem_launch_reduce_sum(const double *in, int n, double *out, cudaStream_t s)
{
    k_reduce_sum<<<1, 1024, 0, s>>>(in, n, out);
    return cudaGetLastError();
}

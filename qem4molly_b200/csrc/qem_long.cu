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
// consecutive particles.
//   1. totals   per (k, chunk) sums of u = q e^{k(z-h)} e^{i k.rho} and
//               v = q e^{-k(z-h)} e^{i k.rho} (h = L_z / 2 keeps both
//               exponentials inside FP32 range): k_ltot (FP64, a thread per
//               PPT = 4 particles, block reductions per k) or k_ltot_lk
//               (FP32, a lane per k walking the chunk).
//   2. k_lscan  one warp per k: FP64 exclusive scan of the chunk totals,
//               forward for u (particles below) and backward for v (above),
//               and the per-k force constants.
//   3. force    FP64 k_lforce: grid (chunk, k-slice), per k serial scans over
//               a thread's 4 particles, a warp shuffle scan and a 4-warp
//               prefix give every particle its prefix (A, B) and suffix (C, D)
//               sums.  FP32 k_lforce_lk: a lane per k walks the chunk with
//               running sums and one cross-lane sum over k per particle.
//               Fl_non_sort + Fl_sort + Flz_self are formed in registers.
//   4. k_lfinal per particle: sum of the k-slices + the k = 0 term, added to F
//               in the original particle order (fixed order: deterministic).
// The FP32 phases k.rho are exact fixed-point lattice phases (lattice_phase).
// The suffix sums C, D are summed directly from above instead of the
// reference's "total minus running sum" (Force_long.jl:97-98), which is the
// same quantity without the cancellation that makes it useless in FP32 (the
// FP32 force pass takes total minus running sum only inside a chunk that is
// thin in z against k, where the cancellation is bounded).
// Phases are reduced in FP64 turns before the FP64 sine/cosine; the per-k
// denominators 0.5 / (g_u g_d e^{-2 k L_z} - 1) are FP64.
#include "qem_internal.cuh"

namespace {

constexpr int LT = 128;         // threads per block
constexpr int PPT = 4;          // particles per thread
constexpr int LCH = LT * PPT;   // particles per chunk
constexpr int NW = LT / 32;     // warps per block
constexpr int KPB = 16;         // k-vectors per block in the totals pass
constexpr int LKB = 8;          // k-vectors per FP32 accumulation batch of the force pass
#ifndef QEM_LF_WAVES_PCT
#define QEM_LF_WAVES_PCT 100
#endif
#ifndef QEM_LF_MINB
#define QEM_LF_MINB 8
#endif
constexpr int LF_MINB = QEM_LF_MINB;  // resident FP32 force-pass blocks per SM (register budget)
#ifndef QEM_LK_WARPS
#define QEM_LK_WARPS 24
#endif

// t - round(t) for |t| < 2^51 turns: rounding by adding and subtracting
// 1.5 * 2^52 (two FP64 adds)
__device__ __forceinline__ double frac_turns(double t)
{
    const double M = 6755399441055744.0;
    return t - ((t + M) - M);
}

template <typename Real>
struct LM;
template <>
struct LM<double> {
    static __device__ __forceinline__ double ex(double x) { return exp(x); }
    static __device__ __forceinline__ void sc(double turns, double &s, double &c) { sincospi(2.0 * turns, &s, &c); }
};

// wk, esc: the force and energy weights of every k (random batch, sum_K / P
// folded in); with per-k weights kwt (exact k-sum) wk = kwt / wden and
// esc = -kwt / eden instead
// ctr != nullptr: row m is first drawn (row S.row0 + m of batch *ctr) and
// written to kin, then its constants are formed from it
__device__ __forceinline__ void kconst_one(int m, double *__restrict__ kin, KConst *__restrict__ kc, double Lz,
                                           double g12, double wk, double esc, const double *__restrict__ kwt,
                                           double wden, double eden, const KSampler &S,
                                           const unsigned long long *__restrict__ ctr, double Lx_2pi, double Ly_2pi)
{
    double kx, ky, k;
    if (ctr) {
        ksample_row(S, *ctr, S.row0 + m, kx, ky, k);
        kin[3 * m] = kx;
        kin[3 * m + 1] = ky;
        kin[3 * m + 2] = k;
    } else {
        kx = kin[3 * m];
        ky = kin[3 * m + 1];
        k = kin[3 * m + 2];
    }
    KConst K;
    K.kx_2pi = kx / (2.0 * QEM_PI);
    K.ky_2pi = ky / (2.0 * QEM_PI);
    K.mx = (int)rint(kx * Lx_2pi);
    K.my = (int)rint(ky * Ly_2pi);
    K.k = k;
    K.W = exp(-0.5 * k * Lz);  // sqrt(exp(-k L_z)); squared on use
    K.g = 0.5 / (g12 * exp(-2.0 * k * Lz) - 1.0);
    K.fx = kx / k;
    K.fy = ky / k;
    K.wk = kwt ? kwt[m] / wden : wk;
    K.ek = (kwt ? -kwt[m] / eden : esc) / k;
    kc[m] = K;
}

__global__ void k_kconst(int P, double *__restrict__ kin, KConst *__restrict__ kc, double Lz, double g12,
                         double wk, double esc, const double *__restrict__ kwt, double wden, double eden,
                         const KSampler S, const unsigned long long *__restrict__ ctr, double Lx_2pi, double Ly_2pi)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m < P) kconst_one(m, kin, kc, Lz, g12, wk, esc, kwt, wden, eden, S, ctr, Lx_2pi, Ly_2pi);
}

// z-ordered SoA copy of the particles
// zlim > 0 (FP32 path): |z - h| must stay within zlim, so that e^{+-k (z - h)}
// stays inside FP32 range for every k of the set; QEM_ST_RANGE otherwise
__device__ __forceinline__ void zrange_check(double zh, double zlim, unsigned *status)
{
    if (zlim > 0.0 && !(fabs(zh) <= zlim)) atomicOr(status, QEM_ST_RANGE);
}

// x / L as a 32-bit fixed-point fraction of the box (the wrapped position)
__device__ __forceinline__ uint32_t box_fraction(double x, double invL)
{
    double f = x * invL;
    f -= floor(f);
    return (uint32_t)__double2ull_rn(f * 4294967296.0);  // 2^32 (f rounding up to 1) wraps to 0
}

// the FP32 record of a particle: {x / Lx, y / Ly as fixed-point box fractions, z - h, q}
__device__ __forceinline__ uint4 f32_record(const double4 &p, double h, double invLx, double invLy)
{
    return make_uint4(box_fraction(p.x, invLx), box_fraction(p.y, invLy), __float_as_uint((float)(p.z - h)),
                      __float_as_uint((float)p.w));
}

// zP != nullptr (FP32 path): the packed records of the lane-per-k passes
__global__ void k_zgather(int N, const double4 *__restrict__ pos, const int *__restrict__ zperm, double h,
                          double *__restrict__ zx, double *__restrict__ zy, double *__restrict__ zhd,
                          double *__restrict__ qd, double zlim, unsigned *status, uint4 *__restrict__ zP,
                          double invLx, double invLy)
{
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= N) return;
    const double4 p = pos[zperm[m]];
    zrange_check(p.z - h, zlim, status);
    if (zP) zP[m] = f32_record(p, h, invLx, invLy);
    zx[m] = p.x;
    zy[m] = p.y;
    zhd[m] = p.z - h;
    qd[m] = p.w;
}

// Stage 0 before the totals for a small system without energy, in one
// block: the z-ordered gather, the scan of q, the k = 0 force and the per-k
// constants -- the same arithmetic as k_zgather, the one-block scan, k_k0
// and k_kconst.
constexpr int LONG_PREP_SMALL = 8192;

__device__ __forceinline__ void long_prep_block(int N, const double4 *__restrict__ pos,
                                                const int *__restrict__ zperm, double h, double *__restrict__ zx,
                                                double *__restrict__ zy, double *__restrict__ zhd,
                                                double *__restrict__ qd, double *__restrict__ qscan, double fscale,
                                                double *__restrict__ k0, int P, double *__restrict__ kin,
                                                KConst *__restrict__ kc, double Lz, double g12, double wk,
                                                double esc, const double *__restrict__ kwt, double wden,
                                                double eden, double zlim, unsigned *status, const KSampler &S,
                                                const unsigned long long *__restrict__ ctr, uint4 *__restrict__ zP,
                                                double invLx, double invLy, double Lx_2pi, double Ly_2pi)
{
    __shared__ double warp_tot[32];
    for (int m = threadIdx.x; m < P; m += 1024)
        kconst_one(m, kin, kc, Lz, g12, wk, esc, kwt, wden, eden, S, ctr, Lx_2pi, Ly_2pi);
    for (int m = threadIdx.x; m < N; m += 1024) {
        const double4 p = pos[zperm[m]];
        zrange_check(p.z - h, zlim, status);
        if (zP) zP[m] = f32_record(p, h, invLx, invLy);
        zx[m] = p.x;
        zy[m] = p.y;
        zhd[m] = p.z - h;
        qd[m] = p.w;
    }
    __syncthreads();
    qem_block_scan_excl_small<double, double>(qd, qscan, N, warp_tot);
    __syncthreads();
    const double tot = qscan[N];
    for (int m = threadIdx.x; m < N; m += 1024) {
        const double q = qd[m], below = qscan[m];
        const double above = (tot - below) - q;
        k0[m] = q * (below - above) * fscale;
    }
}

__global__ void __launch_bounds__(1024) k_long_prep_small(int N, const double4 *__restrict__ pos,
                                                          const int *__restrict__ zperm, double h,
                                                          double *__restrict__ zx, double *__restrict__ zy,
                                                          double *__restrict__ zhd, double *__restrict__ qd,
                                                          double *__restrict__ qscan, double fscale,
                                                          double *__restrict__ k0, int P,
                                                          double *__restrict__ kin, KConst *__restrict__ kc,
                                                          double Lz, double g12, double wk, double esc,
                                                          const double *__restrict__ kwt, double wden, double eden,
                                                          double zlim, unsigned *status, const KSampler S,
                                                          const unsigned long long *__restrict__ ctr,
                                                          uint4 *__restrict__ zP, double invLx, double invLy,
                                                          double Lx_2pi, double Ly_2pi)
{
    long_prep_block(N, pos, zperm, h, zx, zy, zhd, qd, qscan, fscale, k0, P, kin, kc, Lz, g12, wk, esc, kwt, wden,
                    eden, zlim, status, S, ctr, zP, invLx, invLy, Lx_2pi, Ly_2pi);
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
            t = frac_turns(t);
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
__device__ __forceinline__ void lscan_tile(int bx, int P, int nch, const double *__restrict__ tot,
                                           Real *__restrict__ off, double *__restrict__ Utot,
                                           const KConst *__restrict__ kc, double g1, double g2,
                                           double *__restrict__ Eks, KForce<Real> *__restrict__ kf)
{
    const int lane = threadIdx.x & 31;
    const int m = bx * (blockDim.x >> 5) + (threadIdx.x >> 5);
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

template <typename Real>
__global__ void k_lscan(int P, int nch, const double *__restrict__ tot, Real *__restrict__ off,
                        double *__restrict__ Utot, const KConst *__restrict__ kc, double g1, double g2,
                        double *__restrict__ Eks, KForce<Real> *__restrict__ kf)
{
    lscan_tile<Real>(blockIdx.x, P, nch, tot, off, Utot, kc, g1, g2, Eks, kf);
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
            t = frac_turns(t);
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

// ---------------------------------------------------------------------------
// FP32 k-space passes with one lane per k-vector.  Every lane walks the
// particles of a chunk in z order (warp-uniform loads of packed records
// {X, Y, z - L_z/2, q}), so the sum over the particles below (A) is a running
// sum in the lane -- no scans across threads, no barriers -- and the only
// exchange between lanes is the sum over k of each particle's force: after
// every KG particles the lanes' KG x 3 partial forces pass through a padded
// per-warp shared transpose, and lanes 0 .. 3 KG - 1 each add up one column
// in a fixed order.  Inside a chunk that is thin in z against the largest k
// of the warp (k dz <= THIN), the sum over the particles above (C) is the
// chunk's FP64 total minus the running sum of v, whose cancellation is bounded
// by e^{k dz}; a thicker chunk takes C from a second, descending walk, and
// each walk then forms its own half of the force.
// ---------------------------------------------------------------------------
constexpr int KG = 8;           // particles per cross-lane reduction of the force pass
constexpr int KTT = 128;        // threads (k-vectors) per block of the totals pass
constexpr int KFW = 4;          // warps per block of the force pass
constexpr float THIN = 1.0f;    // largest k * (chunk z extent) of the one-walk path

// chunk totals: lane k sums u = q e^{k (z-h)} e^{i k.rho} and v = q e^{-k (z-h)}
// e^{i k.rho} over the chunk, in FP32 over 16 particles at a time, in FP64 across
// lch: particles per chunk (LCH, or a shorter chunk of a fused batch)
__device__ __forceinline__ void ltot_lk_tile(int c, int kb, int lch, int N, int P, int nch,
                                             const uint4 *__restrict__ zp, const KConst *__restrict__ kc,
                                             double *__restrict__ tot)
{
    constexpr float LOG2E = 1.4426950408889634f;
    const int m0 = c * lch, n = min(lch, N - m0);
    const int k = kb * KTT + threadIdx.x;
    if (k >= P) return;
    const int mx = kc[k].mx, my = kc[k].my;
    const float kl = (float)kc[k].k * LOG2E;
    const uint4 *pp = zp + m0;
    double U0 = 0, U1 = 0, U2 = 0, U3 = 0;
    for (int j0 = 0; j0 < n; j0 += 16) {
        const int je = min(n, j0 + 16);
        float2 a0 = f2s(0.f), a1 = f2s(0.f), a2 = f2s(0.f), a3 = f2s(0.f);
#pragma unroll 4
        for (int j = j0; j < je; j += 2) {
            const uint4 r0 = pp[j];
            const uint4 r1 = j + 1 < je ? pp[j + 1] : make_uint4(0u, 0u, 0u, 0u);  // q = 0: no contribution
            float s0, c0, s1, c1;
            __sincosf(lattice_phase(mx, my, r0.x, r0.y), &s0, &c0);
            __sincosf(lattice_phase(mx, my, r1.x, r1.y), &s1, &c1);
            const float2 e = mul2(f2s(kl), f2(__uint_as_float(r0.z), __uint_as_float(r1.z)));
            const float2 q = f2(__uint_as_float(r0.w), __uint_as_float(r1.w));
            const float2 ep = mul2(q, f2(ex2_approx(e.x), ex2_approx(e.y)));
            const float2 em = mul2(q, f2(ex2_approx(-e.x), ex2_approx(-e.y)));
            const float2 C = f2(c0, c1), S = f2(s0, s1);
            a0 = fma2(ep, C, a0);
            a1 = fma2(ep, S, a1);
            a2 = fma2(em, C, a2);
            a3 = fma2(em, S, a3);
        }
        U0 += (double)a0.x + (double)a0.y;
        U1 += (double)a1.x + (double)a1.y;
        U2 += (double)a2.x + (double)a2.y;
        U3 += (double)a3.x + (double)a3.y;
    }
    double *T = tot + ((int64_t)k * nch + c) * 4;
    T[0] = U0;
    T[1] = U1;
    T[2] = U2;
    T[3] = U3;
}

__global__ void __launch_bounds__(KTT) k_ltot_lk(int N, int P, int nch, const uint4 *__restrict__ zp,
                                                 const KConst *__restrict__ kc, double *__restrict__ tot)
{
    ltot_lk_tile(blockIdx.x, blockIdx.y, LCH, N, P, nch, zp, kc, tot);
}

// one lane's k-vector for the force pass (zeros for lanes past P: no force)
struct LaneK {
    int mx = 0, my = 0;
    float kl = 0.f, wfx = 0.f, wfy = 0.f, wk = 0.f, s1r = 0.f, s1i = 0.f, s2r = 0.f, s2i = 0.f;
    double ek = 0.0;
};

// one walk over the chunk's particles.  MODE 0: ascending, A and C together
// (C = chunk total above the first particle minus the running sum of v);
// MODE 1: ascending, A only (the e_- b half of the force); MODE 2:
// descending, C only (the e_+ a half).  Partial forces (without the factor q
// of the particle) are reduced over the warp's lanes every KG particles and
// written (init) or added to Fo; returns the lane's energy sum (before e_k).
template <int MODE, bool ENERGY>
__device__ __forceinline__ float lk_walk(const uint4 *__restrict__ pp, int n, const LaneK &K, float Ar, float Ai,
                                         float Cr, float Ci, float (*tr)[3 * KG + 1], int lane, double *Fo,
                                         bool init)
{
    const float2 mh = f2s(-0.5f);
    float Esum = 0.f;
    const int nblk = (n + KG - 1) / KG;
#pragma unroll 1
    for (int bq = 0; bq < nblk; bq++) {
        const int b = MODE == 2 ? nblk - 1 - bq : bq;
        const int j0 = b * KG;
        float f[3 * KG];
#pragma unroll
        for (int h = 0; h < KG / 2; h++) {
            const int hh = MODE == 2 ? KG / 2 - 1 - h : h;  // the descending walk takes pairs from the top
            const int j = j0 + 2 * hh;
            const uint4 r0 = j < n ? pp[j] : make_uint4(0u, 0u, 0u, 0u);
            const uint4 r1 = j + 1 < n ? pp[j + 1] : make_uint4(0u, 0u, 0u, 0u);
            float s0, c0, s1, c1;
            __sincosf(lattice_phase(K.mx, K.my, r0.x, r0.y), &s0, &c0);
            __sincosf(lattice_phase(K.mx, K.my, r1.x, r1.y), &s1, &c1);
            const float2 e = mul2(f2s(K.kl), f2(__uint_as_float(r0.z), __uint_as_float(r1.z)));
            const float2 q = f2(__uint_as_float(r0.w), __uint_as_float(r1.w));
            const float2 ep = f2(ex2_approx(e.x), ex2_approx(e.y)), em = f2(ex2_approx(-e.x), ex2_approx(-e.y));
            const float2 C = f2(c0, c1), S = f2(s0, s1);
            float2 im1, re2, pz = f2s(0.f);
            if (MODE != 2) {  // exclusive prefix from below: A_j, A_{j+1} = A_j + u_j
                const float2 qep = mul2(q, ep);
                const float2 ur = mul2(qep, C), ui = mul2(qep, S);
                const float2 A2r = f2(Ar, Ar + ur.x), A2i = f2(Ai, Ai + ui.x);
                Ar = A2r.y + ur.y;
                Ai = A2i.y + ui.y;
                const float2 br = fma2(A2r, mh, f2s(K.s2r)), bi = fma2(A2i, mh, f2s(K.s2i));
                const float2 mr = mul2(em, br), mi = mul2(em, bi);
                if (MODE == 0) {  // C_j = (total above the chunk's first particle) - sum_{i <= j} v_i
                    const float2 qem = mul2(q, em);
                    const float2 vr = mul2(qem, C), vi = mul2(qem, S);
                    const float c0r = Cr - vr.x, c0i = Ci - vi.x;
                    const float2 C2r = f2(c0r, c0r - vr.y), C2i = f2(c0i, c0i - vi.y);
                    Cr = C2r.y;
                    Ci = C2i.y;
                    const float2 ar = fma2(C2r, mh, f2s(K.s1r)), ai = fma2(C2i, mh, f2s(K.s1i));
                    const float2 pr = mul2(ep, ar), pi = mul2(ep, ai);
                    const float2 x1r = add2(pr, mr), x1i = add2(pi, mi);
                    const float2 x2r = fma2(mr, f2s(-1.f), pr), x2i = fma2(mi, f2s(-1.f), pi);
                    im1 = fma2(mul2(S, f2s(-1.f)), x1r, mul2(C, x1i));  // Im[e^{-i theta} (e+ a + e- b)]
                    re2 = fma2(S, x2i, mul2(C, x2r));                   // Re[e^{-i theta} (e+ a - e- b)]
                    if (ENERGY) {
                        const float2 zr = fma2(em, A2r, mul2(ep, C2r)), zi = fma2(em, A2i, mul2(ep, C2i));
                        pz = fma2(C, zr, mul2(S, zi));
                    }
                } else {
                    im1 = fma2(mul2(S, f2s(-1.f)), mr, mul2(C, mi));   // Im[e^{-i theta} e- b]
                    re2 = mul2(fma2(S, mi, mul2(C, mr)), f2s(-1.f));    // Re[-e^{-i theta} e- b]
                    if (ENERGY) pz = fma2(C, mul2(em, A2r), mul2(S, mul2(em, A2i)));
                }
                if (ENERGY) {  // -q^2 - q Re[e^{-i theta}(e- A + e+ C)] (Energy_long_range_njit.py:10-24)
                    const float2 t = fma2(mul2(q, f2s(-1.f)), pz, mul2(mul2(q, q), f2s(-1.f)));
                    Esum += t.x + t.y;
                }
            } else {  // exclusive suffix from above, particles j+1 then j: C_{j+1}, C_j = C_{j+1} + v_{j+1}
                const float2 qem = mul2(q, em);
                const float2 vr = mul2(qem, C), vi = mul2(qem, S);
                const float2 C2r = f2(Cr + vr.y, Cr), C2i = f2(Ci + vi.y, Ci);
                Cr = C2r.x + vr.x;
                Ci = C2i.x + vi.x;
                const float2 ar = fma2(C2r, mh, f2s(K.s1r)), ai = fma2(C2i, mh, f2s(K.s1i));
                const float2 pr = mul2(ep, ar), pi = mul2(ep, ai);
                im1 = fma2(mul2(S, f2s(-1.f)), pr, mul2(C, pi));  // Im[e^{-i theta} e+ a]
                re2 = fma2(S, pi, mul2(C, pr));                    // Re[e^{-i theta} e+ a]
                if (ENERGY) {
                    const float2 zp2 = fma2(C, mul2(ep, C2r), mul2(S, mul2(ep, C2i)));
                    const float2 t = mul2(mul2(q, f2s(-1.f)), zp2);
                    Esum += t.x + t.y;
                }
            }
            f[6 * hh + 0] = K.wfx * im1.x;
            f[6 * hh + 1] = K.wfy * im1.x;
            f[6 * hh + 2] = K.wk * re2.x;
            f[6 * hh + 3] = K.wfx * im1.y;
            f[6 * hh + 4] = K.wfy * im1.y;
            f[6 * hh + 5] = K.wk * re2.y;
        }
        // sum over the warp's lanes (k-vectors): lane l < 3 KG adds column l,
        // the component l % 3 of particle j0 + l / 3
#pragma unroll
        for (int r = 0; r < 3 * KG; r++) tr[lane][r] = f[r];
        __syncwarp();
        const int nv = min(KG, n - j0);
        if (lane < 3 * nv) {
            float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
#pragma unroll
            for (int row = 0; row < 32; row += 4) {
                s0 += tr[row][lane];
                s1 += tr[row + 1][lane];
                s2 += tr[row + 2][lane];
                s3 += tr[row + 3][lane];
            }
            const float qj = __uint_as_float(pp[j0 + lane / 3].w);
            const double v = (double)qj * (double)((s0 + s1) + (s2 + s3));
            double *o = Fo + (int64_t)j0 * 3 + lane;
            *o = init ? v : *o + v;
        }
        __syncwarp();
    }
    return Esum;
}

// force pass: warp t of chunk c (t = blockIdx.y KFW + w < ks_n) takes the
// k-groups of 32 vectors g = t, t + ks_n, ... and writes slice t of Fpart
// (z order, the particle's q applied) and of the energy partials
template <bool ENERGY>
__device__ __forceinline__ void lforce_lk_tile(int c, int by, int lch, int N, int P, int nch, int ks_n,
                                               const uint4 *__restrict__ zp, const KConst *__restrict__ kc,
                                               const KForce<float> *__restrict__ kf, const float *__restrict__ off,
                                               const double *__restrict__ tot, double *__restrict__ Fpart,
                                               double *__restrict__ Epart)
{
    constexpr float LOG2E = 1.4426950408889634f;
    __shared__ float tr[KFW][32][3 * KG + 1];  // +1: column reads on distinct banks
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int t = by * KFW + w;
    if (t >= ks_n) return;  // whole warp; the kernel has no block barrier
    const int m0 = c * lch, n = min(lch, N - m0);
    const uint4 *pp = zp + m0;
    const float dz = __uint_as_float(pp[n - 1].z) - __uint_as_float(pp[0].z);
    double *Fo = Fpart + ((int64_t)t * N + m0) * 3;
    const int G = (P + 31) / 32;
    double E = 0;
    bool init = true;
    for (int g = t; g < G; g += ks_n) {
        const int k = 32 * g + lane;
        LaneK K;
        float Ar = 0.f, Ai = 0.f, Cr = 0.f, Ci = 0.f, Cor = 0.f, Coi = 0.f, kk = 0.f;
        if (k < P) {
            K.mx = kc[k].mx;
            K.my = kc[k].my;
            kk = (float)kc[k].k;
            K.kl = kk * LOG2E;
            if (ENERGY) K.ek = kc[k].ek;
            const float4 *kf4 = reinterpret_cast<const float4 *>(kf + k);
            const float4 Ka = kf4[0], Kb = kf4[1];  // (k, wfx, wfy, wk), (s1r, s1i, s2r, s2i)
            K.wfx = Ka.y;
            K.wfy = Ka.z;
            K.wk = Ka.w;
            K.s1r = Kb.x;
            K.s1i = Kb.y;
            K.s2r = Kb.z;
            K.s2i = Kb.w;
            const float4 O = *reinterpret_cast<const float4 *>(off + ((int64_t)k * nch + c) * 4);
            const double *T = tot + ((int64_t)k * nch + c) * 4;
            Ar = O.x;
            Ai = O.y;
            Cor = O.z;
            Coi = O.w;
            Cr = (float)((double)O.z + T[2]);  // v above the chunk's first particle: above the chunk + the chunk
            Ci = (float)((double)O.w + T[3]);
        }
        float kw = kk;
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) kw = fmaxf(kw, __shfl_xor_sync(0xffffffffu, kw, d));
        float Es;
        if (kw * dz <= THIN) {
            Es = lk_walk<0, ENERGY>(pp, n, K, Ar, Ai, Cr, Ci, tr[w], lane, Fo, init);
        } else {
            Es = lk_walk<1, ENERGY>(pp, n, K, Ar, Ai, 0.f, 0.f, tr[w], lane, Fo, init);
            Es += lk_walk<2, ENERGY>(pp, n, K, 0.f, 0.f, Cor, Coi, tr[w], lane, Fo, false);
        }
        if (ENERGY) E += K.ek * 0.5 * (double)Es;
        init = false;
    }
    if (init)  // no k-group for this warp (fewer groups than slices): a zero slice
        for (int i = lane; i < 3 * n; i += 32) Fo[i] = 0.0;
    if (ENERGY) {
        for (int d = 16; d > 0; d >>= 1) E += __shfl_down_sync(0xffffffffu, E, d);
        if (lane == 0) Epart[(int64_t)t * nch + c] = E;
    }
}

template <bool ENERGY>
__global__ void __launch_bounds__(32 * KFW) k_lforce_lk(int N, int P, int nch, int ks_n,
                                                        const uint4 *__restrict__ zp, const KConst *__restrict__ kc,
                                                        const KForce<float> *__restrict__ kf,
                                                        const float *__restrict__ off, const double *__restrict__ tot,
                                                        double *__restrict__ Fpart, double *__restrict__ Epart)
{
    lforce_lk_tile<ENERGY>(blockIdx.x, blockIdx.y, LCH, N, P, nch, ks_n, zp, kc, kf, off, tot, Fpart, Epart);
}

// F[zperm[m]] += sum over k-slices (fixed order) + k = 0 term; ctr: the batch
// counter of a per-call random batch, advanced once here, after every read of
// it (the per-k constants kernel ran earlier on the same stream)
__device__ __forceinline__ void lfinal_one(int m, int N, int ks_n, const double *__restrict__ Fpart,
                                           const double *__restrict__ k0, const int *__restrict__ zperm,
                                           double *__restrict__ F3, unsigned long long *ctr)
{
    if (ctr && m == 0) *ctr += 1;
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

__global__ void k_lfinal(int N, int ks_n, const double *__restrict__ Fpart, const double *__restrict__ k0,
                         const int *__restrict__ zperm, double *__restrict__ F3, unsigned long long *ctr)
{
    lfinal_one(blockIdx.x * blockDim.x + threadIdx.x, N, ks_n, Fpart, k0, zperm, F3, ctr);
}

// ---------------------------------------------------------------------------
// fused batches: the small-system long-range phases over all systems
// ---------------------------------------------------------------------------
constexpr int BATCH_PTILE = 256;  // particles per block of the final pass

// one block per system: clears the long-range force buffer (the final pass
// adds into it) and runs the one-block preparation of k_long_prep_small
__global__ void __launch_bounds__(1024) k_batch_lprep(const BatchSys *__restrict__ ds)
{
    QEM_SHARED_COPY(BatchSys, d, ds + blockIdx.x);
    for (int i = threadIdx.x; i < 3 * d.N; i += 1024) d.Flong[i] = 0.0;
    long_prep_block(d.N, d.pos, d.zperm, d.h, d.b.zx, d.b.zy, d.b.zhd, d.b.qd, d.b.qscan, d.fscale, d.b.k0, d.P,
                    d.b.kin, d.b.kc, d.Lz, d.g12, d.wk, d.esc, d.b.kwt, d.wden, d.eden, d.b.zlim, d.status,
                    d.b.sampler, d.b.draw_ctr, d.b.zP, d.invLx, d.invLy, d.Lx_2pi, d.Ly_2pi);
}

__global__ void __launch_bounds__(KTT) k_batch_ltot(const BatchWork *__restrict__ wl, const BatchSys *__restrict__ ds)
{
    const BatchWork t = wl[blockIdx.x];
    const BatchSys &d = ds[t.s];
    ltot_lk_tile(t.x, t.y, d.lch, d.N, d.P, d.nch, d.b.zP, d.b.kc, d.b.tot);
}

__global__ void __launch_bounds__(128) k_batch_lscan(const BatchWork *__restrict__ wl, const BatchSys *__restrict__ ds)
{
    const BatchWork t = wl[blockIdx.x];
    const BatchSys &d = ds[t.s];
    lscan_tile<float>(t.x, d.P, d.nch, d.b.tot, (float *)d.b.off, d.b.Utot, d.b.kc, d.g1, d.g2, d.b.Eks,
                      (KForce<float> *)d.b.kf);
}

__global__ void __launch_bounds__(32 * KFW) k_batch_lforce(const BatchWork *__restrict__ wl,
                                                           const BatchSys *__restrict__ ds)
{
    const BatchWork t = wl[blockIdx.x];
    const BatchSys &d = ds[t.s];
    lforce_lk_tile<false>(t.x, t.y, d.lch, d.N, d.P, d.nch, d.ks, d.b.zP, d.b.kc, (const KForce<float> *)d.b.kf,
                          (const float *)d.b.off, d.b.tot, d.b.Fpart, d.b.Epart);
}

__global__ void __launch_bounds__(BATCH_PTILE) k_batch_lfinal(const BatchWork *__restrict__ wl,
                                                              const BatchSys *__restrict__ ds)
{
    const BatchWork t = wl[blockIdx.x];
    const BatchSys &d = ds[t.s];
    lfinal_one(t.x * BATCH_PTILE + threadIdx.x, d.N, d.ks, d.b.Fpart, d.b.k0, d.zperm, d.Flong, d.b.draw_ctr);
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


// ---------------------------------------------------------------------------
// adjoint of the long range (FP64).  With P_i = e^{-i theta_i}, the cotangents
// w_xy = w_k q (fx gF_x + fy gF_y), w_z = w_k q gF_z of the force pass and
// c1 = ep (w_z - i w_xy), c2 = -em (w_z + i w_xy), the force part of L is
//   sum_i Re[P_i (c1 (S1 - C_i / 2) + c2 (S2 - A_i / 2))],
// so u_m = q ep e^{i theta} collects a_i = -P_i c2_i / 2 from every i above
// it (through A_i) and v_m collects b_i = -P_i c1_i / 2 from every i below it
// (through C_i); the sorted energy adds -gE e_k q (em, ep) P / 2 to (a, b),
// and the totals U, V collect Lambda_U, Lambda_V from S1, S2 and from the
// split energy term.  Passes: chunk totals of a, b, P c1, P c2 (k_ladj_tot);
// per k their scans, Lambda and the gamma derivatives (k_ladj_scan); per
// particle the prefix / suffix sums of u, v, a, b and the gradient
// (k_ladj); slices + the k = 0 term in particle order (k_ladj_final).
// ---------------------------------------------------------------------------
struct AdjIn {
    const double *zgx, *zgy, *zgz;  // cotangents of F in z order
    double gE;
};

// charge-free p1 = P c1 / q, p2 = P c2 / q (w_xy, w_z passed without q) and
// the scan coefficients a, b (with q)
__device__ __forceinline__ void adj_coefs(double q, double ep, double em, double c, double s, double wxy, double wz,
                                          double ekgE, double &ar, double &ai, double &br, double &bi,
                                          double &p1r, double &p1i, double &p2r, double &p2i)
{
    // c1 = ep (wz - i wxy), c2 = -em (wz + i wxy); P = c - i s
    const double c1r = ep * wz, c1i = -ep * wxy, c2r = -em * wz, c2i = -em * wxy;
    p1r = c * c1r + s * c1i; p1i = c * c1i - s * c1r;
    p2r = c * c2r + s * c2i; p2i = c * c2i - s * c2r;
    // a = -q (P c2 / q + ek gE em P) / 2, b = -q (P c1 / q + ek gE ep P) / 2
    ar = -0.5 * q * (p2r + ekgE * em * c); ai = -0.5 * q * (p2i - ekgE * em * s);
    br = -0.5 * q * (p1r + ekgE * ep * c); bi = -0.5 * q * (p1i - ekgE * ep * s);
}

__global__ void __launch_bounds__(LT) k_ladj_tot(int N, int P, int nch, const double *__restrict__ zx,
                                                 const double *__restrict__ zy, const double *__restrict__ zh,
                                                 const double *__restrict__ qv, const KConst *__restrict__ kc,
                                                 AdjIn in, double *__restrict__ atot)
{
    __shared__ double red[8][NW];
    Quad4<double> P4;
    const int m0 = blockIdx.x * LCH + threadIdx.x * PPT;
    P4.load(N, m0, zx, zy, zh, qv);
    double gxy[PPT][2], gzz[PPT];
#pragma unroll
    for (int j = 0; j < PPT; j++) {
        const int m = m0 + j;
        gxy[j][0] = m < N ? in.zgx[m] : 0.0;
        gxy[j][1] = m < N ? in.zgy[m] : 0.0;
        gzz[j] = m < N ? in.zgz[m] : 0.0;
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int kk = 0; kk < KPB; kk++) {
        const int kidx = blockIdx.y * KPB + kk;
        if (kidx >= P) break;
        const KConst K = kc[kidx];
        double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int j = 0; j < PPT; j++) {
            double t = fma(K.kx_2pi, P4.x[j], K.ky_2pi * P4.y[j]);
            t = frac_turns(t);
            double s, c;
            sincospi(2.0 * t, &s, &c);
            const double kz = K.k * P4.z[j], ep = exp(kz), em = exp(-kz), q = P4.q[j];
            const double wxy = K.wk * (K.fx * gxy[j][0] + K.fy * gxy[j][1]), wz = K.wk * gzz[j];
            double a[8];
            adj_coefs(q, ep, em, c, s, wxy, wz, K.ek * in.gE, a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7]);
#pragma unroll
            for (int r = 0; r < 4; r++) v[r] += a[r];
#pragma unroll
            for (int r = 4; r < 8; r++) v[r] += q * a[r];
        }
#pragma unroll
        for (int r = 0; r < 8; r++) {
#pragma unroll
            for (int d = 16; d > 0; d >>= 1) v[r] += __shfl_down_sync(0xffffffffu, v[r], d);
        }
        if (lane == 0) {
#pragma unroll
            for (int r = 0; r < 8; r++) red[r][w] = v[r];
        }
        __syncthreads();
        if (threadIdx.x < 8) {
            double sum = 0;
#pragma unroll
            for (int ww = 0; ww < NW; ww++) sum += red[threadIdx.x][ww];
            atot[((int64_t)kidx * nch + blockIdx.x) * 8 + threadIdx.x] = sum;
        }
        __syncthreads();
    }
}

// one warp per k: suffix scan of the a totals, prefix scan of the b totals,
// sums of P c1 and P c2; Lambda_U, Lambda_V and the gamma derivatives
__global__ void k_ladj_scan(int P, int nch, const double *__restrict__ atot, double *__restrict__ aoff,
                            const double *__restrict__ Utot, const KConst *__restrict__ kc, double g1, double g2,
                            double gE, double *__restrict__ lam, double *__restrict__ ggk)
{
    const int lane = threadIdx.x & 31;
    const int m = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (m >= P) return;
    const double *T = atot + (int64_t)m * nch * 8;
    double *O = aoff + (int64_t)m * nch * 4;
    double s1r = 0, s1i = 0, s2r = 0, s2i = 0;
    double cr = 0, ci = 0;  // b from below
    for (int base = 0; base < nch; base += 32) {
        const int c = base + lane;
        double r = c < nch ? T[8 * c + 2] : 0.0, i = c < nch ? T[8 * c + 3] : 0.0;
        s1r += c < nch ? T[8 * c + 4] : 0.0; s1i += c < nch ? T[8 * c + 5] : 0.0;
        s2r += c < nch ? T[8 * c + 6] : 0.0; s2i += c < nch ? T[8 * c + 7] : 0.0;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const double a = __shfl_up_sync(0xffffffffu, r, d), b = __shfl_up_sync(0xffffffffu, i, d);
            if (lane >= d) { r += a; i += b; }
        }
        double er = __shfl_up_sync(0xffffffffu, r, 1), ei = __shfl_up_sync(0xffffffffu, i, 1);
        if (lane == 0) { er = 0; ei = 0; }
        if (c < nch) { O[4 * c + 2] = cr + er; O[4 * c + 3] = ci + ei; }
        cr += __shfl_sync(0xffffffffu, r, 31);
        ci += __shfl_sync(0xffffffffu, i, 31);
    }
    double dr = 0, di = 0;  // a from above
    for (int base = 0; base < nch; base += 32) {
        const int c = nch - 1 - (base + lane);
        double r = c >= 0 ? T[8 * c] : 0.0, i = c >= 0 ? T[8 * c + 1] : 0.0;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const double a = __shfl_up_sync(0xffffffffu, r, d), b = __shfl_up_sync(0xffffffffu, i, d);
            if (lane >= d) { r += a; i += b; }
        }
        double er = __shfl_up_sync(0xffffffffu, r, 1), ei = __shfl_up_sync(0xffffffffu, i, 1);
        if (lane == 0) { er = 0; ei = 0; }
        if (c >= 0) { O[4 * c] = dr + er; O[4 * c + 1] = di + ei; }
        dr += __shfl_sync(0xffffffffu, r, 31);
        di += __shfl_sync(0xffffffffu, i, 31);
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        s1r += __shfl_down_sync(0xffffffffu, s1r, d); s1i += __shfl_down_sync(0xffffffffu, s1i, d);
        s2r += __shfl_down_sync(0xffffffffu, s2r, d); s2i += __shfl_down_sync(0xffffffffu, s2i, d);
    }
    if (lane == 0) {
        const KConst K = kc[m];
        const double W = K.W * K.W, g = K.g, g12 = g1 * g2;
        const double Ur = Utot[4 * m], Ui = Utot[4 * m + 1], Vr = Utot[4 * m + 2], Vi = Utot[4 * m + 3];
        const double gW = g * W, eg = gE * K.ek * g;
        // dL = Re[Lambda_U dU + Lambda_V dV]
        double LUr = gW * (g2 * s1r + g12 * W * s2r), LUi = gW * (g2 * s1i + g12 * W * s2i);
        double LVr = gW * (g12 * W * s1r + g1 * s2r), LVi = gW * (g12 * W * s1i + g1 * s2i);
        // split energy e_k g (g2 W |U|^2 + g1 W |V|^2 + g12 W^2 Re(U conj V)): conjugates
        LUr += eg * (2.0 * g2 * W * Ur + g12 * W * W * Vr); LUi += eg * (-2.0 * g2 * W * Ui - g12 * W * W * Vi);
        LVr += eg * (2.0 * g1 * W * Vr + g12 * W * W * Ur); LVi += eg * (-2.0 * g1 * W * Vi - g12 * W * W * Ui);
        lam[4 * m] = LUr; lam[4 * m + 1] = LUi; lam[4 * m + 2] = LVr; lam[4 * m + 3] = LVi;
        // gamma derivatives: S1 = g W (g2 U + g12 W V), S2 = g W (g12 W U + g1 V),
        // g = 0.5 / (g12 W^2 - 1), dg/dg12 = -2 W^2 g^2
        const double dg = -2.0 * W * W * g * g;
        const double A1r = W * (g2 * Ur + g12 * W * Vr), A1i = W * (g2 * Ui + g12 * W * Vi);  // S1 / g
        const double A2r = W * (g12 * W * Ur + g1 * Vr), A2i = W * (g12 * W * Ui + g1 * Vi);  // S2 / g
        // Re[s1 dS1 + s2 dS2] for each gamma (dS = dg A + g W dA)
        const double base = s1r * A1r - s1i * A1i + s2r * A2r - s2i * A2i;
        const double dS1d_r = g * W * g2 * W * Vr, dS1d_i = g * W * g2 * W * Vi;  // d(A1)/dg1 * g W
        const double dS2d_r = g * W * (g2 * W * Ur + Vr), dS2d_i = g * W * (g2 * W * Ui + Vi);
        const double dS1u_r = g * W * (Ur + g1 * W * Vr), dS1u_i = g * W * (Ui + g1 * W * Vi);
        const double dS2u_r = g * W * g1 * W * Ur, dS2u_i = g * W * g1 * W * Ui;
        double gd = dg * g2 * base + (s1r * dS1d_r - s1i * dS1d_i + s2r * dS2d_r - s2i * dS2d_i);
        double gu = dg * g1 * base + (s1r * dS1u_r - s1i * dS1u_i + s2r * dS2u_r - s2i * dS2u_i);
        const double UU = Ur * Ur + Ui * Ui, VV = Vr * Vr + Vi * Vi, UV = Ur * Vr + Ui * Vi;
        const double sig = g2 * W * UU + g1 * W * VV + g12 * W * W * UV;
        gd += gE * K.ek * (dg * g2 * sig + g * (W * VV + g2 * W * W * UV));
        gu += gE * K.ek * (dg * g1 * sig + g * (W * UU + g1 * W * W * UV));
        ggk[2 * m] = gd;
        ggk[2 * m + 1] = gu;
    }
}

// exclusive block scans of NV values per thread: forward (from lower
// threads) where FWD bit v is set, backward (from higher threads) otherwise
template <int NV, unsigned FWD>
__device__ __forceinline__ void block_excl(double (&v)[NV], double (*sh)[NW])
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
#pragma unroll
        for (int r = 0; r < NV; r++) {
            const bool f = (FWD >> r) & 1u;
            const double up = __shfl_up_sync(0xffffffffu, v[r], d), dn = __shfl_down_sync(0xffffffffu, v[r], d);
            if (f ? lane >= d : lane + d < 32) v[r] += f ? up : dn;
        }
    }
#pragma unroll
    for (int r = 0; r < NV; r++) {
        const bool f = (FWD >> r) & 1u;
        if (f ? lane == 31 : lane == 0) sh[r][w] = v[r];
        const double up = __shfl_up_sync(0xffffffffu, v[r], 1), dn = __shfl_down_sync(0xffffffffu, v[r], 1);
        v[r] = f ? (lane == 0 ? 0.0 : up) : (lane == 31 ? 0.0 : dn);
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < NV; r++) {
        const bool f = (FWD >> r) & 1u;
#pragma unroll
        for (int ww = 0; ww < NW; ww++)
            if (f ? ww < w : ww > w) v[r] += sh[r][ww];
    }
    __syncthreads();
}

__global__ void __launch_bounds__(LT) k_ladj(int N, int P, int nch, int ks_n, const double *__restrict__ zx,
                                             const double *__restrict__ zy, const double *__restrict__ zh,
                                             const double *__restrict__ qv, const KConst *__restrict__ kc,
                                             const double *__restrict__ kin, const KForce<double> *__restrict__ kf,
                                             const double *__restrict__ off, const double *__restrict__ aoff,
                                             const double *__restrict__ lam, AdjIn in, double *__restrict__ Gpart)
{
    __shared__ double sh[8][NW];
    Quad4<double> P4;
    const int m0 = blockIdx.x * LCH + threadIdx.x * PPT;
    P4.load(N, m0, zx, zy, zh, qv);
    double gxy[PPT][2], gzz[PPT];
#pragma unroll
    for (int j = 0; j < PPT; j++) {
        const int m = m0 + j;
        gxy[j][0] = m < N ? in.zgx[m] : 0.0;
        gxy[j][1] = m < N ? in.zgy[m] : 0.0;
        gzz[j] = m < N ? in.zgz[m] : 0.0;
    }
    const int ks = blockIdx.y;
    const int kb = (int)((int64_t)P * ks / ks_n), ke = (int)((int64_t)P * (ks + 1) / ks_n);
    double Gx[PPT], Gy[PPT], Gz[PPT], Gq[PPT];
#pragma unroll
    for (int j = 0; j < PPT; j++) { Gx[j] = 0; Gy[j] = 0; Gz[j] = 0; Gq[j] = 0; }
    for (int kidx = kb; kidx < ke; kidx++) {
        const KConst K = kc[kidx];
        const KForce<double> F = kf[kidx];
        const double kx = kin[3 * kidx], ky = kin[3 * kidx + 1], ekgE = K.ek * in.gE;
        double c[PPT], s[PPT], ep[PPT], em[PPT];
        double u[PPT][8];  // u, v, a, b (complex) per particle
        double pc1[PPT][2], pc2[PPT][2];
#pragma unroll
        for (int j = 0; j < PPT; j++) {
            double t = fma(K.kx_2pi, P4.x[j], K.ky_2pi * P4.y[j]);
            t = frac_turns(t);
            sincospi(2.0 * t, &s[j], &c[j]);
            const double kz = K.k * P4.z[j], q = P4.q[j];
            ep[j] = exp(kz);
            em[j] = exp(-kz);
            u[j][0] = q * ep[j] * c[j]; u[j][1] = q * ep[j] * s[j];
            u[j][2] = q * em[j] * c[j]; u[j][3] = q * em[j] * s[j];
            const double wxy = K.wk * (K.fx * gxy[j][0] + K.fy * gxy[j][1]), wz = K.wk * gzz[j];
            adj_coefs(q, ep[j], em[j], c[j], s[j], wxy, wz, ekgE, u[j][4], u[j][5], u[j][6], u[j][7], pc1[j][0],
                      pc1[j][1], pc2[j][0], pc2[j][1]);
        }
        // thread-local exclusive sums: u (0,1) and b (6,7) from below; v (2,3) and a (4,5) from above
        double loc[PPT][8], tot[8];
#pragma unroll
        for (int r = 0; r < 8; r++) {
            const bool fwd = (r < 2) || (r >= 6);
            double acc = 0;
            if (fwd) {
#pragma unroll
                for (int j = 0; j < PPT; j++) { loc[j][r] = acc; acc += u[j][r]; }
            } else {
#pragma unroll
                for (int j = PPT - 1; j >= 0; j--) { loc[j][r] = acc; acc += u[j][r]; }
            }
            tot[r] = acc;
        }
        block_excl<8, 0xC3u>(tot, sh);
        const double *O = off + ((int64_t)kidx * nch + blockIdx.x) * 4;
        const double *OA = aoff + ((int64_t)kidx * nch + blockIdx.x) * 4;
        const double base[8] = {O[0] + tot[0], O[1] + tot[1], O[2] + tot[2], O[3] + tot[3],
                                OA[0] + tot[4], OA[1] + tot[5], OA[2] + tot[6], OA[3] + tot[7]};
        const double LUr = lam[4 * kidx], LUi = lam[4 * kidx + 1], LVr = lam[4 * kidx + 2], LVi = lam[4 * kidx + 3];
#pragma unroll
        for (int j = 0; j < PPT; j++) {
            const double q = P4.q[j];
            const double Ar = base[0] + loc[j][0], Ai = base[1] + loc[j][1];
            const double Cr = base[2] + loc[j][2], Ci = base[3] + loc[j][3];
            const double SAr = base[4] + loc[j][4], SAi = base[5] + loc[j][5];
            const double PBr = base[6] + loc[j][6], PBi = base[7] + loc[j][7];
            // through u = q ep E and v = q em E (E = c + i s): ubar = Lambda_U + SA, vbar = Lambda_V + PB
            const double ubr = LUr + SAr, ubi = LUi + SAi, vbr = LVr + PBr, vbi = LVi + PBi;
            const double uur = ubr * u[j][0] - ubi * u[j][1], uui = ubr * u[j][1] + ubi * u[j][0];
            const double vvr = vbr * u[j][2] - vbi * u[j][3], vvi = vbr * u[j][3] + vbi * u[j][2];
            double gth = -(uui + vvi);
            double gz = K.k * (uur - vvr);
            double gq = (ep[j] * (ubr * c[j] - ubi * s[j]) + em[j] * (vbr * c[j] - vbi * s[j]));
            // direct: Re[P (c1 alpha + c2 beta)], alpha = S1 - C/2, beta = S2 - A/2
            const double alr = F.s1r - 0.5 * Cr, ali = F.s1i - 0.5 * Ci;
            const double ber = F.s2r - 0.5 * Ar, bei = F.s2i - 0.5 * Ai;
            const double x1r = pc1[j][0] * alr - pc1[j][1] * ali, x1i = pc1[j][0] * ali + pc1[j][1] * alr;
            const double x2r = pc2[j][0] * ber - pc2[j][1] * bei, x2i = pc2[j][0] * bei + pc2[j][1] * ber;
            gth += q * (x1i + x2i);
            gz += q * K.k * (x1r - x2r);
            gq += x1r + x2r;
            // sorted energy: gE e_k (-q^2 - q Re[P (em A + ep C)]) / 2, P = c - i s
            const double zr = em[j] * Ar + ep[j] * Cr, zi = em[j] * Ai + ep[j] * Ci;
            const double pzr = c[j] * zr + s[j] * zi, pzi = c[j] * zi - s[j] * zr;
            const double yr = ep[j] * Cr - em[j] * Ar, yi = ep[j] * Ci - em[j] * Ai;
            gth += -0.5 * ekgE * q * pzi;
            gz += -0.5 * ekgE * q * K.k * (c[j] * yr + s[j] * yi);
            gq += 0.5 * ekgE * (-2.0 * q - pzr);
            Gx[j] += kx * gth;
            Gy[j] += ky * gth;
            Gz[j] += gz;
            Gq[j] += gq;
        }
    }
#pragma unroll
    for (int j = 0; j < PPT; j++) {
        const int m = m0 + j;
        if (m < N) {
            double *o = Gpart + ((int64_t)ks * N + m) * 4;
            o[0] = Gx[j]; o[1] = Gy[j]; o[2] = Gz[j]; o[3] = Gq[j];
        }
    }
}

// z-ordered cotangents and the k = 0 adjoint inputs: w1 = gF_z q, w2 = q z
__global__ void k_ladj_prep(int N, const double *__restrict__ gF, const int *__restrict__ zperm,
                            const double *__restrict__ qd, const double *__restrict__ zhd, double h,
                            double *__restrict__ zgx, double *__restrict__ zgy, double *__restrict__ zgz,
                            double *__restrict__ w1, double *__restrict__ w2)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= N) return;
    const int i = zperm[m];
    const double gx = gF ? gF[3 * i] : 0.0, gy = gF ? gF[3 * i + 1] : 0.0, gz = gF ? gF[3 * i + 2] : 0.0;
    zgx[m] = gx; zgy[m] = gy; zgz[m] = gz;
    w1[m] = gz * qd[m];
    w2[m] = qd[m] * (zhd[m] + h);
}

// gamma derivatives of the long range: sums over k in a fixed order
__global__ void k_ladj_gsum(int P, const double *__restrict__ ggk, double *__restrict__ out)
{
    __shared__ double red[2][8];
    double a = 0, b = 0;
    for (int m = threadIdx.x; m < P; m += blockDim.x) { a += ggk[2 * m]; b += ggk[2 * m + 1]; }
    for (int d = 16; d > 0; d >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, d);
        b += __shfl_down_sync(0xffffffffu, b, d);
    }
    if ((threadIdx.x & 31) == 0) { red[0][threadIdx.x >> 5] = a; red[1][threadIdx.x >> 5] = b; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double x = 0, y = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) { x += red[0][w]; y += red[1][w]; }
        out[0] = x;
        out[1] = y;
    }
}

// slices + k = 0 term (Force_long.jl:130-161, Energy_long_range_njit.py:25-44),
// added in particle order
__global__ void k_ladj_final(int N, int ks_n, const double *__restrict__ Gpart, const int *__restrict__ zperm,
                             const double *__restrict__ qd, const double *__restrict__ zhd, double h,
                             const double *__restrict__ qscan, const double *__restrict__ zgz,
                             const double *__restrict__ w1, const double *__restrict__ s1,
                             const double *__restrict__ w2, const double *__restrict__ s2, double fs, double es,
                             double gE, double *__restrict__ gxyz, double *__restrict__ gq)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= N) return;
    double gx = 0, gy = 0, gz = 0, gqm = 0;
    for (int ks = 0; ks < ks_n; ks++) {
        const double *o = Gpart + ((int64_t)ks * N + m) * 4;
        gx += o[0]; gy += o[1]; gz += o[2]; gqm += o[3];
    }
    const double q = qd[m], Z = zhd[m] + h, Qb = qscan[m], Qa = (qscan[N] - Qb) - q;
    // forces: F0_i = q_i (Q_below - Q_above) fs
    const double w1_above = (s1[N] - s1[m]) - w1[m], w1_below = s1[m];
    gqm += zgz[m] * (Qb - Qa) * fs + fs * (w1_above - w1_below);
    // energy: E0_i = 2 q_i z_i (2 Q_below + q_i) es
    const double w2_above = (s2[N] - s2[m]) - w2[m];
    gz += gE * 2.0 * q * (2.0 * Qb + q) * es;
    gqm += gE * es * (2.0 * Z * (2.0 * Qb + q) + 2.0 * q * Z + 4.0 * w2_above);
    const int i = zperm[m];
    gxyz[3 * i] += gx;
    gxyz[3 * i + 1] += gy;
    gxyz[3 * i + 2] += gz;
    if (gq) gq[i] += gqm;
}

}  // namespace

int qem_long_chunk(void) { return LCH; }

// streaming multiprocessors of the current device (cached per device)
static int sm_count()
{
    static int cached[64] = {0};
    int d = 0;
    if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= 64) return 148;
    if (cached[d] == 0) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, d) != cudaSuccess || n <= 0) n = 148;
        cached[d] = n;
    }
    return cached[d];
}

int qem_long_ksplit(int nch, int P, int max_ks, int precision)
{
    if (precision != QEM_FP64) {
        // lane-per-k force pass: one warp per (chunk, slice), about QEM_LK_WARPS
        // resident warps per SM in one wave, and at least one 32-vector
        // k-group per warp
        const int groups = P > 0 ? (P + 31) / 32 : 1;
        int ks = (int)((int64_t)sm_count() * QEM_LK_WARPS / (int64_t)(nch > 0 ? nch : 1));
        ks = ks < 1 ? 1 : (ks > max_ks ? max_ks : ks);
        return ks < groups ? ks : groups;
    }
    // as many whole k-slices of the nch chunks as fit in QEM_LF_WAVES_PCT / 100
    // waves of resident force-pass blocks, each slice with at least two k
    // groups of LKB vectors
    int ks = (int)((int64_t)sm_count() * LF_MINB * QEM_LF_WAVES_PCT / (100 * (int64_t)(nch > 0 ? nch : 1)));
    ks = ks < 1 ? 1 : (ks > max_ks ? max_ks : ks);
    const int pm = P > 2 * LKB ? P / (2 * LKB) : 1;
    return ks < pm ? ks : pm;
}

// Energy partials: b.Epart[0 .. ks * nch) from k_lforce, [ks * nch .. + nb0)
// from k_k0; the P split terms go to b.Eks.
cudaError_t qem_launch_long(int precision, bool energy, int N, int P, const double4 *pos, const int *zperm,
                            const LongBuffers &b, double Lx, double Ly, double Lz, double g1, double g2, double eps0,
                            double sum_K, double *F3, int nch, unsigned *status, cudaStream_t s, int stage)
{
    if (N <= 0) return cudaSuccess;
    const double zlim = precision == QEM_FP64 ? 0.0 : b.zlim;
    uint4 *zP = precision == QEM_FP64 ? nullptr : b.zP;
    auto kconst = [&]() {
        const double wk = (sum_K / P) / (Lx * Ly * eps0);
        const double esc = -(sum_K / P) / (2.0 * eps0 * Lx * Ly);
        k_kconst<<<nblk(P, 128), 128, 0, s>>>(P, b.kin, b.kc, Lz, g1 * g2, wk, esc, b.kwt, Lx * Ly * eps0,
                                              2.0 * eps0 * Lx * Ly, b.sampler, b.draw_ctr, Lx / (2.0 * QEM_PI),
                                              Ly / (2.0 * QEM_PI));
    };
    if (stage == 2) {
        if (P > 0) kconst();
        return cudaGetLastError();
    }
    if (stage == 0 && qem_long_prep_is_small(N, energy)) {
        const double h = 0.5 * Lz;
        const double fscale = b.skip_k0 ? 0.0 : 1.0 / (2.0 * Lx * Ly * eps0);
        const double wk = P > 0 ? (sum_K / P) / (Lx * Ly * eps0) : 0.0;
        const double esc = P > 0 ? -(sum_K / P) / (2.0 * eps0 * Lx * Ly) : 0.0;
        k_long_prep_small<<<1, 1024, 0, s>>>(N, pos, zperm, h, b.zx, b.zy, b.zhd, b.qd, b.qscan, fscale, b.k0, P,
                                             b.kin, b.kc, Lz, g1 * g2, wk, esc, b.kwt, Lx * Ly * eps0,
                                             2.0 * eps0 * Lx * Ly, zlim, status, b.sampler, b.draw_ctr, zP, 1.0 / Lx,
                                             1.0 / Ly, Lx / (2.0 * QEM_PI), Ly / (2.0 * QEM_PI));
        if (P > 0) {
            dim3 gt(nch, nblk(P, KPB));
            if (precision == QEM_FP64)
                k_ltot<double><<<gt, LT, 0, s>>>(N, P, nch, b.zx, b.zy, b.zhd, b.qd, b.kc, b.tot);
            else
                k_ltot_lk<<<dim3(nch, nblk(P, KTT)), KTT, 0, s>>>(N, P, nch, b.zP, b.kc, b.tot);
            if (precision == QEM_FP64)
                k_lscan<double><<<nblk(P, 4), 128, 0, s>>>(P, nch, b.tot, b.off, b.Utot, b.kc, g1, g2, b.Eks,
                                                           (KForce<double> *)b.kf);
            else
                k_lscan<float><<<nblk(P, 4), 128, 0, s>>>(P, nch, b.tot, (float *)b.off, b.Utot, b.kc, g1, g2,
                                                          b.Eks, (KForce<float> *)b.kf);
        }
        return cudaGetLastError();
    }
    if (stage == 0) {
        const double h = 0.5 * Lz;
        k_zgather<<<nblk(N, 256), 256, 0, s>>>(N, pos, zperm, h, b.zx, b.zy, b.zhd, b.qd, zlim, status, zP,
                                               1.0 / Lx, 1.0 / Ly);
        // the k = 0 term (charge scan in z order) is read only by the final
        // pass: it follows the chunk totals, which then start sooner
        auto k0_term = [&]() -> cudaError_t {
            cudaError_t e = qem_scan_f64_excl(b.qd, b.qscan, N, b.stmp, b.stmp_bytes, s);
            if (e != cudaSuccess) return e;
            const double fscale = b.skip_k0 ? 0.0 : 1.0 / (2.0 * Lx * Ly * eps0);
            const double escale = b.skip_k0 ? 0.0 : -1.0 / (4.0 * eps0 * Lx * Ly);
            k_k0<<<nblk(N, 256), 256, 0, s>>>(N, b.qd, b.zhd, h, b.qscan, fscale, escale, b.k0,
                                              b.Epart + b.ks * nch, energy ? 1 : 0);
            return cudaSuccess;
        };
        if (P <= 0) {
            const cudaError_t e = k0_term();
            if (e != cudaSuccess) return e;
        }
        if (P > 0) {
            if (b.kconst_done) {
                const cudaError_t e = cudaStreamWaitEvent(s, b.kconst_done, 0);
                if (e != cudaSuccess) return e;
            } else {
                kconst();
            }
            dim3 gt(nch, nblk(P, KPB));
            if (precision == QEM_FP64)
                k_ltot<double><<<gt, LT, 0, s>>>(N, P, nch, b.zx, b.zy, b.zhd, b.qd, b.kc, b.tot);
            else
                k_ltot_lk<<<dim3(nch, nblk(P, KTT)), KTT, 0, s>>>(N, P, nch, b.zP, b.kc, b.tot);
            const cudaError_t e = k0_term();
            if (e != cudaSuccess) return e;
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
        const dim3 gl(nch, nblk(b.ks, KFW));
        if (energy)
            k_lforce_lk<true><<<gl, 32 * KFW, 0, s>>>(N, P, nch, b.ks, b.zP, b.kc, kf, of, b.tot, b.Fpart, b.Epart);
        else
            k_lforce_lk<false><<<gl, 32 * KFW, 0, s>>>(N, P, nch, b.ks, b.zP, b.kc, kf, of, b.tot, b.Fpart, b.Epart);
    }
    k_lfinal<<<nblk(N, 256), 256, 0, s>>>(N, b.ks, b.Fpart, b.k0, zperm, F3, b.draw_ctr);
    return cudaGetLastError();
}

__global__ void k_scale_vec(int n, double a, const double *x, double *y)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = a * x[i];
}

bool qem_long_prep_is_small(int N, bool energy) { return !energy && N <= LONG_PREP_SMALL; }

int qem_batch_particle_tile(void) { return BATCH_PTILE; }
int qem_batch_ltot_tile(void) { return KTT; }
int qem_batch_lscan_tile(void) { return 4; }
int qem_batch_lforce_tile(void) { return KFW; }

cudaError_t qem_launch_batch_lprep(int B, const BatchSys *d, cudaStream_t s)
{
    if (B <= 0) return cudaSuccess;
    k_batch_lprep<<<B, 1024, 0, s>>>(d);
    return cudaGetLastError();
}
cudaError_t qem_launch_batch_ltot(int nw, const BatchWork *w, const BatchSys *d, cudaStream_t s)
{
    if (nw <= 0) return cudaSuccess;
    k_batch_ltot<<<nw, KTT, 0, s>>>(w, d);
    return cudaGetLastError();
}
cudaError_t qem_launch_batch_lscan(int nw, const BatchWork *w, const BatchSys *d, cudaStream_t s)
{
    if (nw <= 0) return cudaSuccess;
    k_batch_lscan<<<nw, 128, 0, s>>>(w, d);
    return cudaGetLastError();
}
cudaError_t qem_launch_batch_lforce(int nw, const BatchWork *w, const BatchSys *d, cudaStream_t s)
{
    if (nw <= 0) return cudaSuccess;
    k_batch_lforce<<<nw, 32 * KFW, 0, s>>>(w, d);
    return cudaGetLastError();
}
cudaError_t qem_launch_batch_lfinal(int nw, const BatchWork *w, const BatchSys *d, cudaStream_t s)
{
    if (nw <= 0) return cudaSuccess;
    k_batch_lfinal<<<nw, BATCH_PTILE, 0, s>>>(w, d);
    return cudaGetLastError();
}

cudaError_t qem_launch_scale(int n, double a, const double *x, double *y, cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    k_scale_vec<<<nblk(n, 256), 256, 0, s>>>(n, a, x, y);
    return cudaGetLastError();
}

cudaError_t qem_launch_reduce_sum(const double *in, int n, double *out, cudaStream_t s)
{
    k_reduce_sum<<<1, 1024, 0, s>>>(in, n, out);
    return cudaGetLastError();
}

cudaError_t qem_launch_long_adj(int N, int P, const int *zperm, const LongBuffers &b, const LongAdjBuffers &a,
                                double Lx, double Ly, double Lz, double g1, double g2, double eps0, const double *gF,
                                double gE, double *gxyz, double *gq, int nch, int ks, cudaStream_t s, int stage)
{
    if (N <= 0) return cudaSuccess;
    const double h = 0.5 * Lz;
    if (stage == 1) {
        const double fs = 1.0 / (2.0 * Lx * Ly * eps0), es = -1.0 / (4.0 * eps0 * Lx * Ly);
        k_ladj_final<<<nblk(N, 256), 256, 0, s>>>(N, ks, a.Gpart, zperm, b.qd, b.zhd, h, b.qscan, a.zgz, a.w1,
                                                  a.s1, a.w2, a.s2, fs, es, gE, gxyz, gq);
        return cudaGetLastError();
    }
    k_ladj_prep<<<nblk(N, 256), 256, 0, s>>>(N, gF, zperm, b.qd, b.zhd, h, a.zgx, a.zgy, a.zgz, a.w1, a.w2);
    cudaError_t e = qem_scan_f64_excl(a.w1, a.s1, N, b.stmp, b.stmp_bytes, s);
    if (e == cudaSuccess) e = qem_scan_f64_excl(a.w2, a.s2, N, b.stmp, b.stmp_bytes, s);
    if (e != cudaSuccess) return e;
    AdjIn in;
    in.zgx = a.zgx; in.zgy = a.zgy; in.zgz = a.zgz; in.gE = gE;
    if (P > 0) {
        k_ladj_tot<<<dim3(nch, nblk(P, KPB)), LT, 0, s>>>(N, P, nch, b.zx, b.zy, b.zhd, b.qd, b.kc, in, a.atot);
        k_ladj_scan<<<nblk(P, 4), 128, 0, s>>>(P, nch, a.atot, a.aoff, b.Utot, b.kc, g1, g2, gE, a.lam, a.ggk);
    }
    k_ladj<<<dim3(nch, ks), LT, 0, s>>>(N, P, nch, ks, b.zx, b.zy, b.zhd, b.qd, b.kc, b.kin,
                                        (const KForce<double> *)b.kf, b.off, a.aoff, a.lam, in, a.Gpart);
    k_ladj_gsum<<<1, 256, 0, s>>>(P, a.ggk, a.gam);
    if (stage == 0) return cudaGetLastError();
    const double fs = 1.0 / (2.0 * Lx * Ly * eps0), es = -1.0 / (4.0 * eps0 * Lx * Ly);
    k_ladj_final<<<nblk(N, 256), 256, 0, s>>>(N, ks, a.Gpart, zperm, b.qd, b.zhd, h, b.qscan, a.zgz, a.w1, a.s1,
                                              a.w2, a.s2, fs, es, gE, gxyz, gq);
    return cudaGetLastError();
}

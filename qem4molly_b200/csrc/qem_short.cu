// qem_short.cu -- short-range QEM forces and energies.
//
// Reference (ArrogantGao/QEM4Molly):
//   F_short_ij     src/Force_short.jl:25-78   (pair force, four image terms,
//                                              point and Gaussian quadratures)
//   F_short_i      src/Force_short.jl:82-107  (self image z-force)
//   integrands     src/Force_short.jl:4-22, greens_function.jl:68-116
//   pair loop      src/QEM_short.jl:41-56     (F[i] += F_ij; F[j] -= F_ij)
//   walls          src/Substrate_LJ.jl:19-46  (fused into the per-particle pass)
//   energies       src/python_lib/Energy_short_range_njit.py:34-81
//
// One thread per unordered pair evaluates the 4 image terms x {point, gauss}
// x N_t Gauss-Legendre nodes in registers (nodes in the constant bank) and
// writes one record per pair (force on the pair's owner and z-force on the
// other particle); a per-particle pass sums its own and its incoming records
// in a fixed order, adds the self term and the walls.  No atomics: results
// are bitwise reproducible from run to run.
//
// Both integral families share one node body: with
//   point  (Gamma_2 term):  G = -g_u g_d b/2 e^{-k (a + 2 L_z)} / D,
//   gauss  (Gamma_1 term):  G = -b/2 e^{-k (a + k / 4 alpha)} / D,
//   D = 1 - g_u g_d e^{-2 k L_z},
// every interval is G = pf exp(-k (a' + c2 k)) / D for per-interval (pf, a', c2),
// so the 8 intervals run through one rolled loop (small code, no instruction
// cache misses).  Each block groups its 256 pairs by rho in shared memory
// before the quadrature, so the threads of a warp mostly take the same
// Bessel branch; records are still written at the pair's own index.
//
// FP32 path: per-pair set-up (minimum image, rho, image distances, quadrature
// limits, closed-form image terms) and all cross-image sums in FP64; the
// per-node integrands in FP32 with hardware exp / rcp / sin / cos and
// polynomial Bessel approximations (bessel01_x2), two nodes per packed FP32x2
// instruction (the kernel is bound by FMA, MUFU and issue together, and the
// packed arithmetic halves the issue slots of everything but the MUFU
// operations).
// The denominator D is formed as
// (1 - g_u g_d) + g_u g_d (1 - e^{-t}) with (1 - g_u g_d) from FP64 and
// 1 - e^{-t} evaluated without cancellation, so its relative error stays at
// FP32 rounding as |g_u g_d| -> 1.
#include "qem_internal.cuh"

namespace {

#ifndef QEM_PAIR_BLOCK
#define QEM_PAIR_BLOCK 256
#endif
constexpr int PAIR_BLOCK = QEM_PAIR_BLOCK;  // pairs per block, grouped by rho in shared memory
constexpr int RHO_BINS = QEM_RHO_BINS;      // rho^2 bins of the grouping (a multiple of 32)
// resident pair blocks per SM requested from the register allocator, and the
// unroll factor of the FP32 node loop (tuning knobs; measured defaults)
#ifndef QEM_PAIR_MINB
#define QEM_PAIR_MINB 4
#endif
#ifndef QEM_NODE_UNROLL
#define QEM_NODE_UNROLL 3
#endif
constexpr int NODE_UNROLL = QEM_NODE_UNROLL;

// quadrature limits of image term l (Force_short.jl:48-67 / greens_function.jl:26-27,
// or the python_lib global limits)
__device__ __forceinline__ double point_limit(const ShortConsts &c, double a)
{
    if (c.flags & QEM_CUTOFF_PYTHON) return c.kf_point_py;
    return sqrt(4.0 * c.alpha * c.alpha * a * a + 4.0 * c.alpha * c.neg_lnacc) - 2.0 * c.alpha * a;
}
__device__ __forceinline__ double gauss_limit(const ShortConsts &c, double a)
{
    if (c.flags & QEM_CUTOFF_PYTHON) return c.kf_gauss_py;
    return c.neg_lnacc / (c.twoLz + a);
}

// interval constants: image term l, family (0 point, 1 gauss)
struct Interval {
    double K;    // upper limit
    double ae;   // a' (a + 2 L_z for point, a for gauss)
    double c2;   // 0 for point, 1 / (4 alpha) for gauss
    double pf;   // -g_u g_d b / 2 for point, -b / 2 for gauss
};
__device__ __forceinline__ Interval interval(const ShortConsts &c, double a, double b, bool gauss)
{
    Interval v;
    if (gauss) {
        v.K = gauss_limit(c, a);
        v.ae = a;
        v.c2 = c.inv4alpha;
        v.pf = -0.5 * b;
    } else {
        v.K = point_limit(c, a);
        v.ae = a + c.twoLz;
        v.c2 = 0.0;
        v.pf = -0.5 * b * c.g12;
    }
    return v;
}

// I_r = sum w k G J1, I_z = sum w k G J0 (image sign applied by the caller),
// I_u = sum w G J0 (energy)
template <bool ENERGY, bool WITH_J1>
__device__ __forceinline__ void quad_f64(const ShortConsts &c, const Interval &v, double rho, double &Ir, double &Iz,
                                         double &Iu)
{
    const double h = 0.5 * v.K;
    double r = 0, z = 0, u = 0;
#pragma unroll 1
    for (int n = 0; n < c.Nt; n++) {
        const double k = fma(h, c.xd[n], h);
        const double w = h * c.wd[n];
        const double D = 1.0 - c.g12 * exp(-k * c.twoLz);
        const double G = v.pf * exp(-k * fma(k, v.c2, v.ae)) / D;
        const double x = k * rho;
        const double J0 = WITH_J1 ? j0(x) : 1.0;
        const double cw = w * k * G;
        if (WITH_J1) r = fma(cw, j1(x), r);
        z = fma(cw, J0, z);
        if (ENERGY) u = fma(w * G, J0, u);
    }
    Ir = r; Iz = z; Iu = u;
}

// FP32 nodes two at a time in packed FP32x2 lanes (nodes 2m, 2m+1, Bessel
// functions included).  Node n of the interval [0, K] is k = h t_n
// (h = K / 2, t_n = 1 + x_n), so every per-node quantity is t_n times an
// interval constant: the exponentials as 2^(t ...) with log2(e) folded in,
// x = k rho = t (h rho) and x^{-1/2} = (h rho)^{-1/2} / sqrt(t_n) from the
// node table.  The sums run over (w_n t_n) e^{...} / D (and w_n e^{...} / D
// for the energy); the interval's factors h^2 pf (h pf) are applied in FP64
// by the caller.  1 - e^{-2 k L_z} is taken from its series below
// 2 k L_z = 0.5; the two lanes' partial sums are added at the end.
template <bool ENERGY, bool WITH_J1>
__device__ __forceinline__ void quad_f32(const ShortConsts &c, const Interval &v, float rho_f, double &Ir, double &Iz,
                                         double &Iu)
{
    constexpr float LOG2E = 1.4426950408889634f;
    const double h = 0.5 * v.K;
    // interval constants in FP32 from one conversion of h (and of a'); the
    // per-kernel factors come from ShortConsts
    const float hf = (float)h;
    const float2 hn = f2s(hf * c.f_nlog2e_2Lz);             // e^{-2 k L_z} = 2^(t hn)
    const float2 A1 = f2s(hf * (-LOG2E) * (float)v.ae);     // e^{-k (a' + c2 k)} = 2^(t (A1 + t A2))
    const float2 A2 = f2s(v.c2 != 0.0 ? hf * hf * c.f_nlog2e_c2 : 0.0f);
    const float2 g12 = f2s(c.f_g12), omg = f2s(c.f_omg12);
    const float2 tL = f2s(hf * c.f_2Lz);                     // 2 k L_z = t tL
    const float hrf = hf * rho_f;
    const float2 hr = f2s(hrf);                              // x = k rho = t hr
    const float2 rs = f2s(WITH_J1 ? rsqrt_ftz(hrf) : 0.f);   // x^{-1/2} = rs / sqrt(t)
    const float tsmall = (float)(-0.5 * LOG2E);              // t hn > tsmall  <=>  2 k L_z < 0.5
    float2 r = f2s(0.f), z = f2s(0.f), u = f2s(0.f);
#pragma unroll NODE_UNROLL
    for (int m = 0; m < c.Nt2; m++) {
        const float2 t = c.tf2[m];
        const float2 s = mul2(t, hn);
        float2 om = fma2(f2(ex2_approx(s.x), ex2_approx(s.y)), f2s(-1.0f), f2s(1.0f));  // 1 - e^{-2 k L_z}
        if (s.x > tsmall) {  // nodes ascend, so lane x holds the smaller k
            const float2 tt = mul2(t, tL);
            const float2 tay = one_minus_exp_neg_series(tt);
            if (tt.x < 0.5f) om.x = tay.x;
            if (tt.y < 0.5f) om.y = tay.y;
        }
        const float2 Dp = fma2(g12, om, omg);  // 1 - g12 e^{-2 k L_z} > 0
        const float2 ex = mul2(t, fma2(t, A2, A1));
        const float2 eD = mul2(f2(ex2_approx(ex.x), ex2_approx(ex.y)), f2(fast_rcp(Dp.x), fast_rcp(Dp.y)));
        const float2 cw = mul2(c.wtf2[m], eD);
        if (WITH_J1) {
            float2 J0, J1;
            bessel01_x2(mul2(t, hr), mul2(rs, c.rtf2[m]), J0, J1);
            r = fma2(cw, J1, r);
            z = fma2(cw, J0, z);
            if (ENERGY) u = fma2(mul2(c.wf2[m], eD), J0, u);
        } else {
            z = add2(z, cw);
            if (ENERGY) u = fma2(c.wf2[m], eD, u);
        }
    }
    const double s2 = h * h * v.pf;
    Ir = s2 * (double)(r.x + r.y);
    Iz = s2 * (double)(z.x + z.y);
    Iu = ENERGY ? h * v.pf * (double)(u.x + u.y) : 0.0;
}

// gamma_1 gamma_2 > 1 (python_lib Force_short_norm_njit.py:11-414,
// green_norm_njit.py:13-33): the pole of 1 / (g12 e^{-2 k Lz} - 1) at k_0 is
// handled on four sub-intervals [0, k0 - e], [k0 - e, k0 + e], [k0 + e, 2 k0],
// [2 k0, k_f] with their own Gauss-Legendre node sets.  With
// f(k) = F(k) / (g12 e^{-2kLz} - 1), F the integrand without that factor:
// in the window F(k) gamma_norm(k) - F'(k0) / (2 Lz) (gamma_norm: the pole-free
// part, ten series terms; F' by the reference's central difference with step
// 0.01 e), up to 2 k0 f + F(k0) / (2 Lz (k - k0)), beyond 2 k0 f.  The Gauss
// rho integrand of the window carries no exp(-k^2 / 4 alpha) (as in the
// reference, Force_short_norm_njit.py:59).  Same image decomposition as the
// plain path: F = k up(k) J(k rho) with up = -pf exp(-k (a' + c2 k)).
__device__ __forceinline__ double gamma_norm_f64(double x)
{
    double u = 0.5, d = -1.0 + x / 2.0, u0 = 0.5, d0 = x / 2.0;
#pragma unroll
    for (int i = 0; i < 10; i++) {
        u0 = u0 * (-x) / (i + 3);
        d0 = d0 * (-x) / (i + 3);
        u += u0;
        d += d0;
    }
    return u / d;
}

template <bool WITH_J1>
__device__ void quad_norm_f64(const ShortConsts &c, const Interval &v, double rho, double &Ir, double &Iz)
{
    const int f = v.c2 > 0.0 ? 0 : 1;  // 0: Gauss family, 1: point family
    const double k0 = c.k0, ep = c.pv_eps, twoLz = c.twoLz;
    auto up = [&](double k) { return -v.pf * exp(-k * fma(k, v.c2, v.ae)); };
    auto Fr = [&](double k) { return WITH_J1 ? k * up(k) * j1(k * rho) : 0.0; };
    auto Fz = [&](double k) { return k * up(k) * (WITH_J1 ? j0(k * rho) : 1.0); };
    const double k1 = k0 - 0.01 * ep, k2 = k0 + 0.01 * ep;
    const double dfr = (Fr(k2) - Fr(k1)) / (k2 - k1), dfz = (Fz(k2) - Fz(k1)) / (k2 - k1);
    const double r0 = Fr(k0), z0 = Fz(k0);
    const double lo[4] = {0.0, k0 - ep, k0 + ep, 2.0 * k0}, hi[4] = {k0 - ep, k0 + ep, 2.0 * k0, c.kf_norm[f]};
    double r = 0, z = 0;
#pragma unroll 1
    for (int t = 0; t < 4; t++) {
        const int n = c.norm_n[f][t];
        const double *xs = c.norm_xw + c.norm_off[f][t], *ws = xs + n;
        const double a = lo[t], b = hi[t];
#pragma unroll 1
        for (int i = 0; i < n; i++) {
            const double k = 0.5 * (b - a) * xs[i] + 0.5 * (b + a), w = 0.5 * (b - a) * ws[i];
            const double J0 = WITH_J1 ? j0(k * rho) : 1.0, J1 = WITH_J1 ? j1(k * rho) : 0.0;
            const double u = up(k);
            double fr, fz;
            if (fabs(k - k0) <= ep) {
                const double gn = gamma_norm_f64(twoLz * (k - k0));
                const double ur = f == 0 ? -v.pf * exp(-k * v.ae) : u;  // no exp(-k^2/4 alpha) here
                fr = k * ur * J1 * gn - dfr / twoLz;
                fz = k * u * J0 * gn - dfz / twoLz;
            } else {
                const double g = 1.0 / (c.g12 * exp(-k * twoLz) - 1.0);
                fr = k * u * J1 * g;
                fz = k * u * J0 * g;
                if (k <= 2.0 * k0) {
                    fr += r0 / (twoLz * (k - k0));
                    fz += z0 / (twoLz * (k - k0));
                }
            }
            r += w * fr;
            z += w * fz;
        }
    }
    Ir = r;
    Iz = z;
}

template <int PREC, bool ENERGY, bool WITH_J1>
__device__ __forceinline__ void quad(const ShortConsts &c, const Interval &v, double rho, float rho_f, double &Ir,
                                     double &Iz, double &Iu)
{
    if (PREC == QEM_FP64 && c.norm) {
        quad_norm_f64<WITH_J1>(c, v, rho, Ir, Iz);
        Iu = 0;
    } else if (PREC == QEM_FP64) {
        quad_f64<ENERGY, WITH_J1>(c, v, rho, Ir, Iz, Iu);
    } else {
        quad_f32<ENERGY, WITH_J1>(c, v, rho_f, Ir, Iz, Iu);
    }
}

// ---------------------------------------------------------------------------
// pair kernel
// ---------------------------------------------------------------------------
// np: device pointer to the pair count; the grid covers the capacity cap and
// blocks past the count return (a count above cap, which the host treats as
// an overflow and re-evaluates, is clamped so every access stays in bounds)
// bx: the block's tile of PAIR_BLOCK pairs
template <int PREC, bool ENERGY>
__device__ __forceinline__ void short_pair_tile(const ShortConsts &c, int64_t bx, const int64_t *__restrict__ np,
                                                int64_t cap, const int2 *__restrict__ pairs,
                                                const double4 *__restrict__ pos, double4 *__restrict__ R,
                                                double *__restrict__ Upair)
{
    __shared__ int hist[RHO_BINS];
    __shared__ int sidx[PAIR_BLOCK];
    const int64_t Np = min(*np, cap);
    if (bx * PAIR_BLOCK >= Np) return;  // whole block: before any barrier
    // this rank's block of the pair list (all of it unless sharded)
    const int64_t lo = Np * c.shard_rank / c.shard_world, hi = Np * (c.shard_rank + 1) / c.shard_world;
    // 1. every thread loads one pair and its rho^2; the block's pairs are
    // grouped by rho^2 (a counting sort into RHO_BINS bins of equal width,
    // equal population for pairs uniform in the plane), so that the threads of
    // a warp cross the Bessel branch point at nearly the same node.  The order
    // inside a bin depends on the atomics, but every thread evaluates and
    // writes its own pair, so the results do not.
    int bin = RHO_BINS - 1;
    {
        const int64_t p = bx * PAIR_BLOCK + threadIdx.x;
        if (p >= lo && p < hi) {
            const int2 ij = pairs[p];
            const double4 pi = pos[ij.x], pj = pos[ij.y];
            const double dx = min_image(pi.x - pj.x, c.Lx, c.invLx), dy = min_image(pi.y - pj.y, c.Ly, c.invLy);
            bin = min(RHO_BINS - 1, (int)((dx * dx + dy * dy) * c.bins_per_rc2));
        }
    }
    const int64_t p = bx * PAIR_BLOCK + group_by_bin<RHO_BINS>(bin, hist, sidx);
    if (p >= Np) return;
    if (p < lo || p >= hi) {  // another rank's pair
        R[p] = make_double4(0, 0, 0, 0);
        if (ENERGY) Upair[p] = 0;
        return;
    }
    // stored as (owner, other); evaluated as F_short_ij with i the lower index
    // (the canonical orientation of QEM_short.jl:41-47), recorded for the owner
    const int2 oo = pairs[p];
    const bool owner_is_i = oo.x < oo.y;
    const int2 ij = owner_is_i ? oo : make_int2(oo.y, oo.x);
    const double4 pi = pos[ij.x], pj = pos[ij.y];
    const double dxr = pi.x - pj.x, dyr = pi.y - pj.y;
    const double dx = min_image(dxr, c.Lx, c.invLx), dy = min_image(dyr, c.Ly, c.invLy);
    const double rho2 = dx * dx + dy * dy;
    if (rho2 > c.rc2) {  // stale-list re-check (Force_short.jl:36-41)
        R[p] = make_double4(0, 0, 0, 0);
        if (ENERGY) Upair[p] = 0;
        return;
    }
    const double rho = sqrt(rho2);
    const float rho_f = (float)rho;
    const double zi = pi.z, zj = pj.z;
    const double zn = fabs(zi - zj), zp = zi + zj;
    const double s = jl_sign(zi - zj);
    // accumulated: Fr = -sum point_r + sum gauss_r; Fz = sum s_l (point_z - gauss_z); U = Ug - Up
    double Fr = 0, Fzi = 0, Fzj = 0, U = 0, Fp2 = 0, Fz2i = 0, Fz2j = 0, Ub = 0;
#pragma unroll 1
    for (int iv = 0; iv < 8; iv++) {
        const int l = iv >> 1;
        const bool gauss = (iv & 1) != 0;
        const double a = (l == 0) ? zn : (l == 1) ? zp : (l == 2) ? c.twoLz - zp : c.twoLz - zn;
        const double b = (l == 0) ? 1.0 : (l == 1) ? c.g1 : (l == 2) ? c.g2 : c.g12;
        const double si = (l == 0) ? -s : (l == 1) ? -1.0 : (l == 2) ? 1.0 : s;  // greens_function.jl:24
        const double sj = (l == 1 || l == 2) ? si : -si;                          // the element seen from j
        double Ir, Iz, Iu;
        quad<PREC, ENERGY, true>(c, interval(c, a, b, gauss), rho, rho_f, Ir, Iz, Iu);
        const double sf = gauss ? 1.0 : -1.0;
        Fr += sf * Ir;
        Fzi -= sf * si * Iz;
        Fzj -= sf * sj * Iz;
        if (ENERGY) U += sf * Iu;
        if (!gauss) {  // closed-form image terms (Force_short.jl:49, 65)
            const double r2 = a * a + rho2;
            const double inv15 = 1.0 / (r2 * sqrt(r2));
            Fp2 += b * rho * inv15;
            Fz2i += b * a * si * inv15;
            Fz2j += b * a * sj * inv15;
            if (ENERGY) Ub += 0.5 * b / sqrt(r2);
        }
    }
    const double pref = pi.w * pj.w * c.pref;
    double Fx = 0, Fy = 0;
    if (rho != 0.0) {  // Force_short.jl:46
        const double Fsr = Fr + 0.5 * Fp2;
        const bool mi = (c.flags & QEM_DIR_MINIMAGE) != 0;
        Fx = pref * Fsr * (mi ? dx : dxr) / rho;
        Fy = pref * Fsr * (mi ? dy : dyr) / rho;
    }
    const double Fz_i = pref * (Fzi - 0.5 * Fz2i);
    const double Fz_j = (c.flags & QEM_PAIR_PHYSICAL) ? pref * (Fzj - 0.5 * Fz2j) : -Fz_i;
    // record: x, y, z on the owner and z on the other particle (x, y on the other = -owner's)
    R[p] = owner_is_i ? make_double4(Fx, Fy, Fz_i, Fz_j) : make_double4(-Fx, -Fy, Fz_j, Fz_i);
    if (ENERGY) Upair[p] = pref * (U + Ub);
}

template <int PREC, bool ENERGY>
__global__ void __launch_bounds__(PAIR_BLOCK, QEM_PAIR_MINB) k_short_pair(const int64_t *__restrict__ np,
                                                                           int64_t cap,
                                                                           const int2 *__restrict__ pairs,
                                                                           const double4 *__restrict__ pos,
                                                                           double4 *__restrict__ R,
                                                                           double *__restrict__ Upair,
                                                                           const ShortConsts c)
{
    short_pair_tile<PREC, ENERGY>(c, blockIdx.x, np, cap, pairs, pos, R, Upair);
}

// ---------------------------------------------------------------------------
// self image z-force (Force_short.jl:82-107) and self energy
// (Energy_short_range_njit.py:64-81), rho = 0 so J0 = 1
// ---------------------------------------------------------------------------
template <int PREC, bool ENERGY>
__device__ void self_terms(const ShortConsts &c, double z, double q, double &Fz, double &E)
{
    double Fs = 0, U = 0, Ub = 0;
#pragma unroll 1
    for (int iv = 0; iv < 8; iv++) {
        const int l = iv >> 1;
        const bool gauss = (iv & 1) != 0;
        const bool zterm = (l == 1 || l == 2);  // sign_a = 0 for l = 1, 4 (greens_function.jl:42)
        if (!ENERGY && !zterm) continue;
        const double a = (l == 0) ? 0.0 : (l == 1) ? 2.0 * z : (l == 2) ? c.twoLz - 2.0 * z : c.twoLz;
        const double b = (l == 0) ? 1.0 : (l == 1) ? c.g1 : (l == 2) ? c.g2 : c.g12;
        const double sa = (l == 1) ? -1.0 : (l == 2) ? 1.0 : 0.0;
        double Ir, Iz, Iu;
        quad<PREC, ENERGY, false>(c, interval(c, a, b, gauss), 0.0, 0.0f, Ir, Iz, Iu);
        // -Fp1 + Fg; with g12 > 1 the reference adds the point part with the
        // opposite sign (Force_short_norm_njit.py:330-331), reproduced
        const double sf = (gauss || (PREC == QEM_FP64 && c.norm)) ? 1.0 : -1.0;
        if (zterm) Fs += sf * sa * Iz;
        if (ENERGY) {
            U += sf * Iu;
            if (!gauss && l > 0) Ub += 0.5 * b / a;
        }
    }
    const double a1 = 2.0 * z, a2 = c.twoLz - 2.0 * z;
    const double Fp2 = 0.5 * (c.g1 * a1 * -1.0 / (a1 * a1 * a1) + c.g2 * a2 * 1.0 / (a2 * a2 * a2));
    Fz = -q * q * c.pref * (Fs + Fp2);
    if (ENERGY) E = 0.5 * q * q * c.pref * (U + Ub);
}

// ---------------------------------------------------------------------------
// per-particle pass: own + incoming pair records, self term, walls
// ---------------------------------------------------------------------------
// particle i: writes F3[i], returns its energy share
template <int PREC, bool ENERGY>
__device__ __forceinline__ double gather_one(const ShortConsts &c, int i, const double4 *__restrict__ pos,
                                             const int *__restrict__ pos_of, const int64_t *__restrict__ poff,
                                             const double4 *__restrict__ R, const double *__restrict__ Upair,
                                             const int64_t *__restrict__ in_off, const int *__restrict__ in_list,
                                             int64_t cap, double *__restrict__ F3, unsigned *status, int do_short,
                                             int do_lj, const double *__restrict__ Fadd)
{
    double Fx = 0, Fy = 0, Fz = 0, E = 0;
    {
        const double4 pi = pos[i];
        if (do_short) {
            const int t = pos_of[i];
            const int64_t pe = min(poff[t + 1], cap);
            for (int64_t p = min(poff[t], cap); p < pe; p++) {
                const double4 r = R[p];
                Fx += r.x; Fy += r.y; Fz += r.z;
                if (ENERGY) E += Upair[p];
            }
            for (int64_t s = in_off[i]; s < in_off[i + 1]; s++) {
                const double4 r = R[in_list[s]];
                Fx -= r.x; Fy -= r.y; Fz += r.w;
            }
            if (c.shard_rank == 0) {
                double fz_self = 0, e_self = 0;
                self_terms<PREC, ENERGY>(c, pi.z, pi.w, fz_self, e_self);
                Fz += fz_self;
                if (ENERGY) E += e_self;
            }
        }
        if (do_lj && c.shard_rank == 0) {
            for (int w = 0; w < c.n_walls; w++) {
                const double dz = pi.z - c.wall_pos[w];
                if (!(c.wall_dir[w] * dz > 0)) {  // Substrate_LJ.jl:37
                    atomicOr(status, QEM_ST_OUT_OF_SLAB);
                    continue;
                }
                if (dz < c.wall_cut[w]) {  // signed distance, as in Substrate_LJ.jl:38
                    const double invr2 = 1.0 / (dz * dz);
                    const double s6 = (c.wall_sig2[w] * invr2) * (c.wall_sig2[w] * invr2) * (c.wall_sig2[w] * invr2);
                    Fz += c.wall_dir[w] * ((24.0 * c.wall_eps[w] * invr2) * (2.0 * s6 * s6 - s6));
                }
            }
        }
        if (Fadd) {  // the long-range forces of a concurrent long-range pass, added last
            Fx += Fadd[3 * i];
            Fy += Fadd[3 * i + 1];
            Fz += Fadd[3 * i + 2];
        }
        F3[3 * i] = Fx;
        F3[3 * i + 1] = Fy;
        F3[3 * i + 2] = Fz;
    }
    return E;
}

template <int PREC, bool ENERGY>
__global__ void __launch_bounds__(256) k_short_gather(int N, const double4 *__restrict__ pos,
                                                       const int *__restrict__ pos_of, const int64_t *__restrict__ poff,
                                                       const double4 *__restrict__ R, const double *__restrict__ Upair,
                                                       const int64_t *__restrict__ in_off,
                                                       const int *__restrict__ in_list, int64_t cap,
                                                       const ShortConsts c, double *__restrict__ F3,
                                                       double *__restrict__ Epart, unsigned *status, int do_short,
                                                       int do_lj, const double *__restrict__ Fadd)
{
    __shared__ double red[256 / 32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double E = 0;
    if (i < N)
        E = gather_one<PREC, ENERGY>(c, i, pos, pos_of, poff, R, Upair, in_off, in_list, cap, F3, status, do_short,
                                     do_lj, Fadd);
    if (ENERGY) {
        // deterministic block reduction of the per-particle energies
        for (int d = 16; d > 0; d >>= 1) E += __shfl_down_sync(0xffffffffu, E, d);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = E;
        __syncthreads();
        if (threadIdx.x == 0) {
            double s = 0;
            for (int w = 0; w < 256 / 32; w++) s += red[w];
            Epart[blockIdx.x] = s;
        }
    }
}

// ---------------------------------------------------------------------------
// fused batches: the pair and gather phases over (system, tile) work lists;
// each block works on its system's ShortConsts copied to shared memory
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(PAIR_BLOCK, QEM_PAIR_MINB) k_batch_pairs(const BatchWork *__restrict__ wl,
                                                                            const BatchSys *__restrict__ ds,
                                                                            const ShortConsts *__restrict__ scs)
{
    const BatchWork t = wl[blockIdx.x];
    const BatchSys &d = ds[t.s];
    QEM_SHARED_COPY(ShortConsts, c, scs + t.s);
    short_pair_tile<QEM_FP32_FIX, false>(c, t.x, d.poff + d.N, d.cap, d.pairs, d.pos, d.R, nullptr);
}

constexpr int GATHER_TILE = 256;

__global__ void __launch_bounds__(GATHER_TILE) k_batch_gather(const BatchWork *__restrict__ wl,
                                                              const BatchSys *__restrict__ ds,
                                                              const ShortConsts *__restrict__ scs, int do_lj,
                                                              double *__restrict__ F)
{
    const BatchWork t = wl[blockIdx.x];
    const BatchSys &d = ds[t.s];
    QEM_SHARED_COPY(ShortConsts, c, scs + t.s);
    const int i = t.x * GATHER_TILE + threadIdx.x;
    if (i < d.N)
        gather_one<QEM_FP32_FIX, false>(c, i, d.pos, d.pos_of, d.poff, d.R, nullptr, d.in_off, d.in_list, d.cap,
                                        F + 3 * d.off, d.status, 1, do_lj, d.Flong);
}

inline int nblk(int64_t n, int b) { return (int)((n + b - 1) / b); }

}  // namespace

int qem_batch_pair_tile(void) { return PAIR_BLOCK; }

cudaError_t qem_launch_batch_pairs(int nw, const BatchWork *w, const BatchSys *d, const ShortConsts *sc,
                                   cudaStream_t s)
{
    if (nw <= 0) return cudaSuccess;
    k_batch_pairs<<<nw, PAIR_BLOCK, 0, s>>>(w, d, sc);
    return cudaGetLastError();
}

cudaError_t qem_launch_batch_gather(int nw, const BatchWork *w, const BatchSys *d, const ShortConsts *sc, int do_lj,
                                    double *F, cudaStream_t s)
{
    if (nw <= 0) return cudaSuccess;
    static_assert(GATHER_TILE == 256, "the gather tile is the particle tile of the final pass");
    k_batch_gather<<<nw, GATHER_TILE, 0, s>>>(w, d, sc, do_lj, F);
    return cudaGetLastError();
}

cudaError_t qem_launch_short_pairs(int precision, bool energy, const int64_t *np, int64_t cap, const int2 *pairs,
                                   const double4 *pos, double4 *R, double *Upair, const ShortConsts &c,
                                   cudaStream_t s)
{
    if (cap <= 0) return cudaSuccess;
    const int G = nblk(cap, PAIR_BLOCK);
    if (precision == QEM_FP64) {
        if (energy) k_short_pair<QEM_FP64, true><<<G, PAIR_BLOCK, 0, s>>>(np, cap, pairs, pos, R, Upair, c);
        else k_short_pair<QEM_FP64, false><<<G, PAIR_BLOCK, 0, s>>>(np, cap, pairs, pos, R, Upair, c);
    } else {
        if (energy) k_short_pair<QEM_FP32_FIX, true><<<G, PAIR_BLOCK, 0, s>>>(np, cap, pairs, pos, R, Upair, c);
        else k_short_pair<QEM_FP32_FIX, false><<<G, PAIR_BLOCK, 0, s>>>(np, cap, pairs, pos, R, Upair, c);
    }
    return cudaGetLastError();
}

cudaError_t qem_launch_short_gather(int precision, bool energy, bool do_short, bool do_lj, int N,
                                    const double4 *pos, const int *pos_of, const int64_t *poff, const double4 *R,
                                    const double *Upair, const int64_t *in_off, const int *in_list, int64_t cap,
                                    const ShortConsts &c, double *F3, double *Epart, unsigned *status,
                                    cudaStream_t s, const double *Fadd)
{
    if (N <= 0) return cudaSuccess;
    const int B = 256;
    const int G = nblk(N, B);
    const int ds = do_short ? 1 : 0, dl = do_lj ? 1 : 0;
    if (precision == QEM_FP64) {
        if (energy)
            k_short_gather<QEM_FP64, true><<<G, B, 0, s>>>(N, pos, pos_of, poff, R, Upair, in_off, in_list, cap, c,
                                                            F3, Epart, status, ds, dl, Fadd);
        else
            k_short_gather<QEM_FP64, false><<<G, B, 0, s>>>(N, pos, pos_of, poff, R, Upair, in_off, in_list, cap, c,
                                                             F3, Epart, status, ds, dl, Fadd);
    } else {
        if (energy)
            k_short_gather<QEM_FP32_FIX, true><<<G, B, 0, s>>>(N, pos, pos_of, poff, R, Upair, in_off, in_list, cap,
                                                                c, F3, Epart, status, ds, dl, Fadd);
        else
            k_short_gather<QEM_FP32_FIX, false><<<G, B, 0, s>>>(N, pos, pos_of, poff, R, Upair, in_off, in_list,
                                                                 cap, c, F3, Epart, status, ds, dl, Fadd);
    }
    return cudaGetLastError();
}

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
// writes (F_ij.x, F_ij.y, F_ij.z, z-force on j) to a per-pair record; a
// per-particle pass sums its own and its incoming records in a fixed order,
// adds the self term and the walls.  No atomics: results are bitwise
// reproducible from run to run.
//
// FP32 path: per-pair set-up (minimum image, rho, image distances, quadrature
// limits, closed-form image terms) and all cross-image sums in FP64; the
// per-node integrands in FP32 with hardware exp / rcp / cos and the
// Abramowitz-Stegun Bessel approximations.  The image-series denominator
// 1 - g_u g_d e^{-2 k L_z} is formed as (1 - g_u g_d) + g_u g_d (1 - e^{-t})
// with (1 - g_u g_d) from FP64 and 1 - e^{-t} evaluated without cancellation,
// so its relative error stays at FP32 rounding as |g_u g_d| -> 1.
#include "qem_internal.cuh"

namespace {

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

// ---------------------------------------------------------------------------
// per-interval quadratures.  I_r = sum w k G J1, I_z = sum w k G J0 (image sign
// applied by the caller), I_u = sum w G J0 (energy).  point: G = Gamma_2 term,
// gauss: G = Gamma_1 term x exp(-k^2 / 4 alpha).
// ---------------------------------------------------------------------------
template <bool ENERGY, bool WITH_J1>
__device__ __forceinline__ void quad_f64(const ShortConsts &c, bool point, double K, double a, double hb, double rho,
                                         double &Ir, double &Iz, double &Iu)
{
    const double h = 0.5 * K;
    Ir = 0; Iz = 0; Iu = 0;
    for (int n = 0; n < c.Nt; n++) {
        const double k = fma(h, c.xd[n], h);
        const double w = h * c.wd[n];
        const double E2 = exp(-k * c.twoLz);
        const double D = c.g12 * E2 - 1.0;
        double G;
        if (point) G = c.g12 * (hb * exp(-k * a)) * E2 / D;
        else G = (hb * exp(-k * a - k * k * c.inv4alpha)) / D;
        const double x = k * rho;
        const double J0 = (rho == 0.0) ? 1.0 : j0(x);
        const double cw = w * k * G;
        if (WITH_J1) Ir = fma(cw, j1(x), Ir);
        Iz = fma(cw, J0, Iz);
        if (ENERGY) Iu = fma(w * G, J0, Iu);
    }
}

template <bool ENERGY, bool WITH_J1>
__device__ __forceinline__ void quad_f32(const ShortConsts &c, bool point, float K, float a, float hb, float rho,
                                         float twoLz, float g12, float omg12, float inv4a, float &Ir, float &Iz,
                                         float &Iu)
{
    const float h = 0.5f * K;
    float r = 0.f, z = 0.f, u = 0.f;
#pragma unroll 2
    for (int n = 0; n < c.Nt; n++) {
        const float k = fmaf(h, c.xf[n], h);
        const float w = h * c.wf[n];
        const float t = k * twoLz;
        const float E2 = __expf(-t);
        const float Dp = fmaf(g12, one_minus_exp_neg(t, E2), omg12);  // 1 - g12 e^{-t} > 0
        const float invD = fast_rcp(Dp);
        float G;
        if (point) G = -g12 * hb * __expf(-k * a) * E2 * invD;
        else G = -hb * __expf(-k * fmaf(k, inv4a, a)) * invD;
        float J0 = 1.0f, J1 = 0.0f;
        if (WITH_J1) bessel01_f32(k * rho, J0, J1);
        const float cw = w * k * G;
        if (WITH_J1) r = fmaf(cw, J1, r);
        z = fmaf(cw, J0, z);
        if (ENERGY) u = fmaf(w * G, J0, u);
    }
    Ir = r; Iz = z; Iu = u;
}

// ---------------------------------------------------------------------------
// pair kernel
// ---------------------------------------------------------------------------
template <int PREC, bool ENERGY>
__global__ void __launch_bounds__(128) k_short_pair(int64_t Np, const int2 *__restrict__ pairs,
                                                     const double4 *__restrict__ pos, double4 *__restrict__ R,
                                                     double *__restrict__ Upair, const ShortConsts c)
{
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= Np) return;
    const int2 ij = pairs[p];
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
    const double zi = pi.z, zj = pj.z;
    const double zn = fabs(zi - zj), zp = zi + zj;
    const double s = jl_sign(zi - zj);
    const double av[4] = {zn, zp, c.twoLz - zp, c.twoLz - zn};
    const double bv[4] = {1.0, c.g1, c.g2, c.g12};
    const double si[4] = {-s, -1.0, 1.0, s};  // greens_function.jl:24
    const double sj[4] = {s, -1.0, 1.0, -s};  // same element seen from j
    double Fp1 = 0, Fg = 0, Fzp_i = 0, Fzp_j = 0, Fzg_i = 0, Fzg_j = 0, Up = 0, Ug = 0;
    double Fp2 = 0, Fz2_i = 0, Fz2_j = 0, Ub = 0;
    const bool has_rho = (rho != 0.0);
#pragma unroll
    for (int l = 0; l < 4; l++) {
        const double a = av[l];
        const double hb = 0.5 * bv[l];
        const double Kp = point_limit(c, a), Kg = gauss_limit(c, a);
        double pr, pz, pu, gr, gz, gu;
        if (PREC == QEM_FP64) {
            quad_f64<ENERGY, true>(c, true, Kp, a, hb, rho, pr, pz, pu);
            quad_f64<ENERGY, true>(c, false, Kg, a, hb, rho, gr, gz, gu);
        } else {
            float fr, fz, fu;
            const float twoLz = (float)c.twoLz, g12 = (float)c.g12, omg = (float)c.one_minus_g12,
                        i4a = (float)c.inv4alpha;
            quad_f32<ENERGY, true>(c, true, (float)Kp, (float)a, (float)hb, (float)rho, twoLz, g12, omg, i4a, fr, fz,
                                   fu);
            pr = fr; pz = fz; pu = fu;
            quad_f32<ENERGY, true>(c, false, (float)Kg, (float)a, (float)hb, (float)rho, twoLz, g12, omg, i4a, fr,
                                   fz, fu);
            gr = fr; gz = fz; gu = fu;
        }
        Fp1 += pr;
        Fg += gr;
        Fzp_i += si[l] * pz;
        Fzp_j += sj[l] * pz;
        Fzg_i += si[l] * gz;
        Fzg_j += sj[l] * gz;
        if (ENERGY) { Up += pu; Ug += gu; }
        const double r2 = a * a + rho2;
        const double inv15 = 1.0 / (r2 * sqrt(r2));
        Fp2 += bv[l] * rho * inv15;
        Fz2_i += bv[l] * a * si[l] * inv15;
        Fz2_j += bv[l] * a * sj[l] * inv15;
        if (ENERGY) Ub += 0.5 * bv[l] / sqrt(r2);
    }
    const double pref = pi.w * pj.w * c.pref;
    double Fx = 0, Fy = 0;
    if (has_rho) {
        const double Fsr = -Fp1 + 0.5 * Fp2 + Fg;
        const bool mi = (c.flags & QEM_DIR_MINIMAGE) != 0;
        Fx = pref * Fsr * (mi ? dx : dxr) / rho;
        Fy = pref * Fsr * (mi ? dy : dyr) / rho;
    }
    const double Fzi = pref * (Fzp_i - 0.5 * Fz2_i - Fzg_i);
    const double Fzj = pref * (Fzp_j - 0.5 * Fz2_j - Fzg_j);
    R[p] = make_double4(Fx, Fy, Fzi, (c.flags & QEM_PAIR_PHYSICAL) ? Fzj : -Fzi);
    if (ENERGY) Upair[p] = pref * (Ug - Up + Ub);
}

// ---------------------------------------------------------------------------
// self image z-force (Force_short.jl:82-107) and self energy
// (Energy_short_range_njit.py:64-81), rho = 0 so J0 = 1
// ---------------------------------------------------------------------------
template <int PREC, bool ENERGY>
__device__ void self_terms(const ShortConsts &c, double z, double q, double &Fz, double &E)
{
    const double av[4] = {0.0, 2.0 * z, c.twoLz - 2.0 * z, c.twoLz};
    const double bv[4] = {1.0, c.g1, c.g2, c.g12};
    const double sa[4] = {0.0, -1.0, 1.0, 0.0};
    double Fp1 = 0, Fg = 0, Up = 0, Ug = 0, Ub = 0;
#pragma unroll
    for (int l = 0; l < 4; l++) {
        const bool zterm = (l == 1 || l == 2);  // sign_a = 0 for l = 1, 4
        if (!ENERGY && !zterm) continue;
        const double a = av[l], hb = 0.5 * bv[l];
        const double Kp = point_limit(c, a), Kg = gauss_limit(c, a);
        double pr, pz, pu, gr, gz, gu;
        if (PREC == QEM_FP64) {
            quad_f64<ENERGY, false>(c, true, Kp, a, hb, 0.0, pr, pz, pu);
            quad_f64<ENERGY, false>(c, false, Kg, a, hb, 0.0, gr, gz, gu);
        } else {
            float fr, fz, fu;
            const float twoLz = (float)c.twoLz, g12 = (float)c.g12, omg = (float)c.one_minus_g12,
                        i4a = (float)c.inv4alpha;
            quad_f32<ENERGY, false>(c, true, (float)Kp, (float)a, (float)hb, 0.f, twoLz, g12, omg, i4a, fr, fz, fu);
            pz = fz; pu = fu;
            quad_f32<ENERGY, false>(c, false, (float)Kg, (float)a, (float)hb, 0.f, twoLz, g12, omg, i4a, fr, fz, fu);
            gz = fz; gu = fu;
        }
        if (zterm) {
            Fp1 += sa[l] * pz;
            Fg += sa[l] * gz;
        }
        if (ENERGY) {
            Up += pu;
            Ug += gu;
            if (l > 0) Ub += 0.5 * bv[l] / a;
        }
    }
    const double Fp2 = 0.5 * (bv[1] * av[1] * sa[1] / (av[1] * av[1] * av[1]) +
                              bv[2] * av[2] * sa[2] / (av[2] * av[2] * av[2]));
    Fz = -q * q * c.pref * (-Fp1 + Fp2 + Fg);
    if (ENERGY) E = 0.5 * q * q * c.pref * (Ug - Up + Ub);
}

// ---------------------------------------------------------------------------
// per-particle pass: own + incoming pair records, self term, walls
// ---------------------------------------------------------------------------
template <int PREC, bool ENERGY>
__global__ void __launch_bounds__(256) k_short_gather(int N, const double4 *__restrict__ pos,
                                                       const int *__restrict__ pos_of, const int64_t *__restrict__ poff,
                                                       const double4 *__restrict__ R, const double *__restrict__ Upair,
                                                       const int64_t *__restrict__ in_off,
                                                       const int64_t *__restrict__ in_list, const ShortConsts c,
                                                       double *__restrict__ F3, double *__restrict__ Epart,
                                                       unsigned *status, int do_short, int do_lj)
{
    __shared__ double red[256 / 32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double Fx = 0, Fy = 0, Fz = 0, E = 0;
    if (i < N) {
        const double4 pi = pos[i];
        if (do_short) {
            const int t = pos_of[i];
            for (int64_t p = poff[t]; p < poff[t + 1]; p++) {
                const double4 r = R[p];
                Fx += r.x; Fy += r.y; Fz += r.z;
                if (ENERGY) E += Upair[p];
            }
            for (int64_t s = in_off[i]; s < in_off[i + 1]; s++) {
                const double4 r = R[in_list[s]];
                Fx -= r.x; Fy -= r.y; Fz += r.w;
            }
            double fz_self = 0, e_self = 0;
            self_terms<PREC, ENERGY>(c, pi.z, pi.w, fz_self, e_self);
            Fz += fz_self;
            if (ENERGY) E += e_self;
        }
        if (do_lj) {
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
        F3[3 * i] = Fx;
        F3[3 * i + 1] = Fy;
        F3[3 * i + 2] = Fz;
    }
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

inline int nblk(int64_t n, int b) { return (int)((n + b - 1) / b); }

}  // namespace

cudaError_t qem_launch_short_pairs(int precision, bool energy, int64_t Np, const int2 *pairs, const double4 *pos,
                                   double4 *R, double *Upair, const ShortConsts &c, cudaStream_t s)
{
    if (Np <= 0) return cudaSuccess;
    const int B = 128;
    const int G = nblk(Np, B);
    if (precision == QEM_FP64) {
        if (energy) k_short_pair<QEM_FP64, true><<<G, B, 0, s>>>(Np, pairs, pos, R, Upair, c);
        else k_short_pair<QEM_FP64, false><<<G, B, 0, s>>>(Np, pairs, pos, R, Upair, c);
    } else {
        if (energy) k_short_pair<QEM_FP32_FIX, true><<<G, B, 0, s>>>(Np, pairs, pos, R, Upair, c);
        else k_short_pair<QEM_FP32_FIX, false><<<G, B, 0, s>>>(Np, pairs, pos, R, Upair, c);
    }
    return cudaGetLastError();
}

cudaError_t qem_launch_short_gather(int precision, bool energy, bool do_short, bool do_lj, int N,
                                    const double4 *pos, const int *pos_of, const int64_t *poff, const double4 *R,
                                    const double *Upair, const int64_t *in_off, const int64_t *in_list,
                                    const ShortConsts &c, double *F3, double *Epart, unsigned *status,
                                    cudaStream_t s)
{
    if (N <= 0) return cudaSuccess;
    const int B = 256;
    const int G = nblk(N, B);
    const int ds = do_short ? 1 : 0, dl = do_lj ? 1 : 0;
    if (precision == QEM_FP64) {
        if (energy)
            k_short_gather<QEM_FP64, true><<<G, B, 0, s>>>(N, pos, pos_of, poff, R, Upair, in_off, in_list, c, F3,
                                                            Epart, status, ds, dl);
        else
            k_short_gather<QEM_FP64, false><<<G, B, 0, s>>>(N, pos, pos_of, poff, R, Upair, in_off, in_list, c, F3,
                                                             Epart, status, ds, dl);
    } else {
        if (energy)
            k_short_gather<QEM_FP32_FIX, true><<<G, B, 0, s>>>(N, pos, pos_of, poff, R, Upair, in_off, in_list, c,
                                                                F3, Epart, status, ds, dl);
        else
            k_short_gather<QEM_FP32_FIX, false><<<G, B, 0, s>>>(N, pos, pos_of, poff, R, Upair, in_off, in_list, c,
                                                                 F3, Epart, status, ds, dl);
    }
    return cudaGetLastError();
}

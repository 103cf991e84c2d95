// qem_adjoint.cu -- adjoint (reverse-mode) of the short-range QEM forces,
// energies and Substrate_LJ walls.
//
// For L = gE * E + sum_i gF_i . F_i the pass returns dL/dr_i, dL/dq_i and
// dL/d(gamma_down, gamma_up).  Each unordered pair's contributions
// (Force_short.jl:25-78 forces, Energy_short_range_njit.py:34-63 energy) are
// a function of (dx, dy, z_i, z_j, gamma_down, gamma_up) times q_i q_j.  The
// pair kernel contracts them with the pair's cotangents
//   (gF_i - gF_j).(F_x, F_y) + gF_i,z F_z,i + gF_j,z F_z,j + gE U_ij
// and returns the exact FP64 gradient of that contraction for the
// discretised pair terms (the quadrature limits of the Julia cutoff mode
// move with the image distances, and that dependence is included): the
// contraction is linear in the interval integrals, so one scalar walk over
// an interval's nodes gives its value and its partials with respect to the
// limit, exponent, prefactor, g12 and rho, and only the few closed-form
// terms around the quadrature run on Dual<6> numbers.
// It writes one record per pair in the forward pass's (owner, other) layout;
// a per-particle pass sums a particle's own and incoming records in a fixed
// order, adds the self term (Force_short.jl:82-107, on Dual<3> numbers in
// (z, gamma_down, gamma_up)) and the walls (Substrate_LJ.jl:19-46,
// analytic), and reduces the gamma derivatives per block.  No atomics.
#include "qem_dual.cuh"
#include "qem_internal.cuh"

namespace {

constexpr int ADJ_BLOCK = 128;
// resident blocks per SM the pair adjoint is compiled for (register cap)
#ifndef QEM_ADJ_MINB
#define QEM_ADJ_MINB 8
#endif

template <class T>
__device__ __forceinline__ T point_limit_t(const ShortConsts &c, const T &a)
{
    if (c.flags & QEM_CUTOFF_PYTHON) return T(a * 0.0 + c.kf_point_py);
    return sqrt(4.0 * c.alpha * c.alpha * (a * a) + 4.0 * c.alpha * c.neg_lnacc) - 2.0 * c.alpha * a;
}
template <class T>
__device__ __forceinline__ T gauss_limit_t(const ShortConsts &c, const T &a)
{
    if (c.flags & QEM_CUTOFF_PYTHON) return T(a * 0.0 + c.kf_gauss_py);
    return c.neg_lnacc / (a + c.twoLz);
}

// the FP64 quadrature of one interval (same nodes and integrand as the
// forward pass): Ir = sum w k G J1, Iz = sum w k G J0, Iu = sum w G J0
template <class T, bool WITH_J1>
__device__ void quad_t(const ShortConsts &c, const T &K, const T &ae, double c2, const T &pf, const T &g12,
                       const T &rho, T &Ir, T &Iz, T &Iu)
{
    const T h = 0.5 * K;
    T r = h * 0.0, z = h * 0.0, u = h * 0.0;
    for (int n = 0; n < c.Nt; n++) {
        const T k = h * (1.0 + c.xd[n]);
        const T w = h * c.wd[n];
        const T D = 1.0 - g12 * exp(k * (-c.twoLz));
        const T G = pf * exp(-(k * (ae + k * c2))) / D;
        const T cw = w * k * G;
        if (WITH_J1) {
            T J0, J1;
            bessel01(k * rho, J0, J1);
            r += cw * J1;
            z += cw * J0;
            u += w * G * J0;
        } else {
            z += cw;
            u += w * G;
        }
    }
    Ir = r; Iz = z; Iu = u;
}

// One interval of the pair quadrature, contracted with the loss: with
//   G(k) = pf e^{-k (ae + k c2)} / (1 - g12 e^{-2 Lz k}),
//   Ir = sum w k G J1(k rho),  Iz = sum w k G J0(k rho),  Iu = sum w G J0(k rho)
// over the nodes k = h (1 + x_n), weights h w_n, h = K / 2 (the forward
// pass's nodes and integrand), returns S = cr Ir + cz Iz + cu Iu, the value
// of Ir, and the partials of S with respect to K, ae, pf, g12 and rho, all
// from one walk over the nodes in scalar FP64.  Writing T = G Phi with
// Phi = k (cr J1 + cz J0) + cu J0:
//   dS/dpf = S / pf,  dS/dae = -sum h w k T,  dS/dg12 = sum h w T e / D,
//   dS/drho = sum h w G dPhi/drho,
//   dS/dK = (S + sum h w k dT/dk) / K        (the nodes scale with K)
// with k dPhi/dk = k (J0 (cz + k rho cr) - rho J1 (k cz + cu)),
//      dPhi/drho = k (cr k (J0 - J1(x)/x) - (k cz + cu) J1),  x = k rho,
//      k d ln G / dk = -(k ae + 2 k^2 c2) - 2 Lz k g12 e / D,  e = e^{-2 Lz k}.
struct QAdj {
    double S, R, dK, dae, dpf, dg12, drho;
};

__device__ __forceinline__ QAdj quad_adj(const ShortConsts &c, double K, double ae, double c2, double pf,
                                         double g12, double rho, double cr, double cz, double cu)
{
    const double h = 0.5 * K;
    double a0 = 0, a1 = 0, a2 = 0, a3 = 0, bk = 0, r = 0;
    for (int n = 0; n < c.Nt; n++) {
        const double k = h * (1.0 + c.xd[n]);
        const double e = exp(k * (-c.twoLz));
        const double Di = 1.0 / (1.0 - g12 * e);
        const double wH = (h * c.wd[n]) * exp(-(k * (ae + k * c2))) * Di;
        const double x = k * rho;
        double J0, J1;
        bessel01(x, J0, J1);
        const double j1x = x != 0.0 ? J1 / x : 0.5;
        const double kzu = k * cz + cu;
        const double Phi = k * (cr * J1 + cz * J0) + cu * J0;
        const double Phr = k * (cr * k * (J0 - j1x) - kzu * J1);
        const double kPk = k * (J0 * (cz + x * cr) - rho * J1 * kzu);
        const double t = e * Di;
        const double wHP = wH * Phi;
        a0 += wHP;
        a1 += wHP * k;
        a2 += wHP * t;
        a3 += wH * Phr;
        bk += wH * (kPk - Phi * (k * (ae + 2.0 * k * c2) + c.twoLz * k * g12 * t));
        r += wH * k * J1;
    }
    QAdj q;
    q.S = pf * a0;
    q.R = pf * r;
    q.dpf = a0;
    q.dae = -pf * a1;
    q.dg12 = pf * a2;
    q.drho = pf * a3;
    q.dK = K > 0.0 ? pf * (a0 + bk) / K : 0.0;
    return q;
}

__device__ __forceinline__ double3 load_g(const double *gF, int i)
{
    if (!gF) return make_double3(0, 0, 0);
    return make_double3(gF[3 * i], gF[3 * i + 1], gF[3 * i + 2]);
}

// records: RA[2p] = (dL/dx, dL/dy, dL/dz of the owner, dL/dz of the other),
//          RA[2p+1] = (dL/dq owner, dL/dq other, dL/dgamma_down, dL/dgamma_up)
//
// The unit-charge pair terms (Force_short.jl:25-78, canonical orientation,
// i the lower index) enter the loss linearly through the interval integrals:
//   L~ = C Fsr + sum_iv (cz Iz + cu Iu) + closed-form image terms,
//   Fsr = sum_iv sf Ir + Fp2 / 2,  C = pref (gdx dir_x + gdy dir_y) / rho,
// gdx = gF_i,x - gF_j,x.  Each interval's cotangents (cr = sf C, cz, cu) are
// known before its quadrature, so quad_adj returns the interval's share of
// L~ and its partials; the limits, image distances, closed-form terms and C
// are carried on Dual<6> numbers in (dx, dy, z_i, z_j, gamma_down, gamma_up).
__global__ void __launch_bounds__(ADJ_BLOCK, QEM_ADJ_MINB) k_short_pair_adj(const int64_t *__restrict__ np, int64_t cap,
                                                               const int2 *__restrict__ pairs,
                                                               const double4 *__restrict__ pos,
                                                               const double *__restrict__ gF, double gE,
                                                               double4 *__restrict__ RA, const ShortConsts c)
{
    typedef Dual<6> D6;
    __shared__ int hist[QEM_RHO_BINS];
    __shared__ int sidx[ADJ_BLOCK];
    const int64_t Np = min(*np, cap);
    if ((int64_t)blockIdx.x * ADJ_BLOCK >= Np) return;  // whole block: before any barrier
    // the block's pairs grouped by rho^2, as in the forward pair kernel, so
    // that a warp's lanes take the same branches of the Bessel functions
    int bin = QEM_RHO_BINS - 1;
    {
        const int64_t p0 = (int64_t)blockIdx.x * ADJ_BLOCK + threadIdx.x;
        if (p0 < Np) {
            const int2 ij = pairs[p0];
            const double4 a = pos[ij.x], b = pos[ij.y];
            const double dx = min_image(a.x - b.x, c.Lx, c.invLx), dy = min_image(a.y - b.y, c.Ly, c.invLy);
            bin = min(QEM_RHO_BINS - 1, (int)((dx * dx + dy * dy) * c.bins_per_rc2));
        }
    }
    const int64_t p = (int64_t)blockIdx.x * ADJ_BLOCK + group_by_bin<QEM_RHO_BINS>(bin, hist, sidx);
    if (p >= Np) return;
    const int2 oo = pairs[p];
    const bool owner_is_i = oo.x < oo.y;
    const int i = owner_is_i ? oo.x : oo.y, j = owner_is_i ? oo.y : oo.x;
    const double4 pi = pos[i], pj = pos[j];
    const double dxr = pi.x - pj.x, dyr = pi.y - pj.y;
    const double dxm = min_image(dxr, c.Lx, c.invLx), dym = min_image(dyr, c.Ly, c.invLy);
    if (dxm * dxm + dym * dym > c.rc2) {  // stale-list re-check (Force_short.jl:36-41)
        RA[2 * p] = make_double4(0, 0, 0, 0);
        RA[2 * p + 1] = make_double4(0, 0, 0, 0);
        return;
    }
    const double3 gi = load_g(gF, i), gj = load_g(gF, j);
    const bool phys = (c.flags & QEM_PAIR_PHYSICAL) != 0, mi = (c.flags & QEM_DIR_MINIMAGE) != 0;
    const bool python = (c.flags & QEM_CUTOFF_PYTHON) != 0;
    // tangents: 0 dx, 1 dy, 2 z_i, 3 z_j, 4 gamma_down, 5 gamma_up
    const D6 dx = dvar<6>(dxm, 0), dy = dvar<6>(dym, 1);
    const D6 zi = dvar<6>(pi.z, 2), zj = dvar<6>(pj.z, 3), g1 = dvar<6>(c.g1, 4), g2 = dvar<6>(c.g2, 5);
    const D6 rho2 = dx * dx + dy * dy;
    const D6 rho = sqrt(rho2);
    const D6 zn = fabs(zi - zj), zp = zi + zj;
    const double s = jl_sign(pi.z - pj.z);
    const D6 g12 = g1 * g2;
    const D6 zero = dconst<6>(0.0);
    D6 C = zero;
    if (rho.v != 0.0) {
        const D6 ux = mi ? dx : dvar<6>(dxr, 0), uy = mi ? dy : dvar<6>(dyr, 1);
        C = c.pref * ((gi.x - gj.x) * ux + (gi.y - gj.y) * uy) / rho;
    }
    D6 L = zero, Fp2 = zero, Fz2 = zero, Ub = zero;
    double Fq = 0.0;
    for (int iv = 0; iv < 8; iv++) {
        const int l = iv >> 1;
        const bool gauss = (iv & 1) != 0;
        const D6 a = (l == 0) ? zn : (l == 1) ? zp : (l == 2) ? c.twoLz - zp : c.twoLz - zn;
        const D6 b = (l == 0) ? zero + 1.0 : (l == 1) ? g1 : (l == 2) ? g2 : g12;
        const double si = (l == 0) ? -s : (l == 1) ? -1.0 : (l == 2) ? 1.0 : s;
        const double sj = (l == 1 || l == 2) ? si : -si;
        const double sf = gauss ? 1.0 : -1.0;
        // limit K(a) and dK/da (constant limits in the python cutoff mode)
        double K, Kp;
        if (gauss) {
            K = python ? c.kf_gauss_py : c.neg_lnacc / (a.v + c.twoLz);
            Kp = python ? 0.0 : -K / (a.v + c.twoLz);
        } else if (python) {
            K = c.kf_point_py;
            Kp = 0.0;
        } else {
            const double sq = ::sqrt(4.0 * c.alpha * c.alpha * (a.v * a.v) + 4.0 * c.alpha * c.neg_lnacc);
            K = sq - 2.0 * c.alpha * a.v;
            Kp = 4.0 * c.alpha * c.alpha * a.v / sq - 2.0 * c.alpha;
        }
        const double ae = gauss ? a.v : a.v + c.twoLz, c2 = gauss ? c.inv4alpha : 0.0;
        const double pfb = gauss ? -0.5 : -0.5 * g12.v;  // pf = pfb b
        const double cz = phys ? -sf * c.pref * (si * gi.z + sj * gj.z) : -sf * si * c.pref * (gi.z - gj.z);
        const QAdj q = quad_adj(c, K, ae, c2, pfb * b.v, g12.v, rho.v, sf * C.v, cz, sf * c.pref * gE);
        const double dSa = q.dK * Kp + q.dae, dSb = q.dpf * pfb;
        const double dSg = q.dg12 + (gauss ? 0.0 : -0.5 * b.v * q.dpf);
        L.v += q.S;
#pragma unroll
        for (int t = 0; t < 6; t++) L.d[t] += dSa * a.d[t] + dSb * b.d[t] + dSg * g12.d[t] + q.drho * rho.d[t];
        Fq += sf * q.R;
        if (!gauss) {
            const D6 r2 = a * a + rho2;
            const D6 inv15 = 1.0 / (r2 * sqrt(r2));
            Fp2 += b * rho * inv15;
            Fz2 += (phys ? si * gi.z + sj * gj.z : si * (gi.z - gj.z)) * (b * a * inv15);
            Ub += 0.5 * b / sqrt(r2);
        }
    }
    // C Fsr: the quadrature part's value and dFq are in L already (cr = sf C.v)
#pragma unroll
    for (int t = 0; t < 6; t++) L.d[t] += Fq * C.d[t];
    L += C * (0.5 * Fp2) + (-0.5 * c.pref) * Fz2 + (gE * c.pref) * Ub;
    const double qq = pi.w * pj.w;
    // dL/d(input) = q_i q_j dL~/d(input); dL/dq_i = q_j L~, dL/dq_j = q_i L~
    const double gdx = qq * L.d[0], gdy = qq * L.d[1], gzi = qq * L.d[2], gzj = qq * L.d[3];
    const double ggd = qq * L.d[4], ggu = qq * L.d[5];
    if (owner_is_i) {
        RA[2 * p] = make_double4(gdx, gdy, gzi, gzj);
        RA[2 * p + 1] = make_double4(pj.w * L.v, pi.w * L.v, ggd, ggu);
    } else {
        RA[2 * p] = make_double4(-gdx, -gdy, gzj, gzi);
        RA[2 * p + 1] = make_double4(pi.w * L.v, pj.w * L.v, ggd, ggu);
    }
}

// unit-charge self image z-force and self energy (Force_short.jl:82-107,
// Energy_short_range_njit.py:64-81)
template <class T>
__device__ void self_terms_t(const ShortConsts &c, const T &z, const T &g1, const T &g2, bool energy, T &Fz, T &E)
{
    const T g12 = g1 * g2;
    const T zero = z * 0.0;
    T Fs = zero, Uq = zero, Ub = zero;
    for (int iv = 0; iv < 8; iv++) {
        const int l = iv >> 1;
        const bool gauss = (iv & 1) != 0;
        const bool zterm = (l == 1 || l == 2);
        if (!energy && !zterm) continue;
        const T a = (l == 0) ? zero : (l == 1) ? 2.0 * z : (l == 2) ? c.twoLz - 2.0 * z : zero + c.twoLz;
        const T b = (l == 0) ? zero + 1.0 : (l == 1) ? g1 : (l == 2) ? g2 : g12;
        const double sa = (l == 1) ? -1.0 : (l == 2) ? 1.0 : 0.0;
        T K, ae, pf;
        double c2;
        if (gauss) {
            K = gauss_limit_t(c, a);
            ae = a;
            c2 = c.inv4alpha;
            pf = -0.5 * b;
        } else {
            K = point_limit_t(c, a);
            ae = a + c.twoLz;
            c2 = 0.0;
            pf = -0.5 * b * g12;
        }
        T Ir, Iz, Iu;
        quad_t<T, false>(c, K, ae, c2, pf, g12, zero, Ir, Iz, Iu);
        const double sf = gauss ? 1.0 : -1.0;
        if (zterm) Fs += (sf * sa) * Iz;
        if (energy) {
            Uq += sf * Iu;
            if (!gauss && l > 0) Ub += 0.5 * b / a;
        }
    }
    const T a1 = 2.0 * z, a2 = c.twoLz - 2.0 * z;
    const T Fp2 = 0.5 * (g2 * a2 / (a2 * a2 * a2) - g1 * a1 / (a1 * a1 * a1));
    Fz = -c.pref * (Fs + Fp2);
    E = 0.5 * c.pref * (Uq + Ub);
}

// per particle: own and incoming pair records (fixed order), self term,
// walls; writes dL/dr, dL/dq and per-block gamma partials (gam[b], gam[nb + b])
__global__ void __launch_bounds__(ADJ_BLOCK) k_adj_gather(int N, const double4 *__restrict__ pos,
                                                           const int *__restrict__ pos_of,
                                                           const int64_t *__restrict__ poff,
                                                           const double4 *__restrict__ RA,
                                                           const int64_t *__restrict__ in_off,
                                                           const int *__restrict__ in_list, int64_t cap,
                                                           const double *__restrict__ gF, double gE,
                                                           const ShortConsts c, double *__restrict__ gxyz,
                                                           double *__restrict__ gq, double *__restrict__ gam,
                                                           int do_short, int do_lj)
{
    __shared__ double red[2][ADJ_BLOCK / 32];
    typedef Dual<3> D3;
    const int i = blockIdx.x * ADJ_BLOCK + threadIdx.x;
    double gx = 0, gy = 0, gz = 0, gqi = 0, gd = 0, gu = 0;
    if (i < N) {
        const double4 p = pos[i];
        const double3 g = load_g(gF, i);
        if (do_short) {
            const int t = pos_of[i];
            const int64_t pe = min(poff[t + 1], cap);
            for (int64_t s = min(poff[t], cap); s < pe; s++) {
                const double4 r0 = RA[2 * s], r1 = RA[2 * s + 1];
                gx += r0.x; gy += r0.y; gz += r0.z;
                gqi += r1.x;
                gd += r1.z; gu += r1.w;
            }
            for (int64_t s = in_off[i]; s < in_off[i + 1]; s++) {
                const int64_t pp = in_list[s];
                const double4 r0 = RA[2 * pp], r1 = RA[2 * pp + 1];
                gx -= r0.x; gy -= r0.y; gz += r0.w;
                gqi += r1.y;
            }
            // self: L = q^2 (gF_z Fz~ + gE E~) in (z, gamma_down, gamma_up)
            D3 Fz, E;
            self_terms_t<D3>(c, dvar<3>(p.z, 0), dvar<3>(c.g1, 1), dvar<3>(c.g2, 2), gE != 0.0, Fz, E);
            const D3 Ls = g.z * Fz + gE * E;
            const double q2 = p.w * p.w;
            gz += q2 * Ls.d[0];
            gd += q2 * Ls.d[1];
            gu += q2 * Ls.d[2];
            gqi += 2.0 * p.w * Ls.v;
        }
        if (do_lj) {
            for (int w = 0; w < c.n_walls; w++) {
                const double dz = p.z - c.wall_pos[w];
                if (!(c.wall_dir[w] * dz > 0)) continue;  // reported by the forward pass
                if (dz < c.wall_cut[w]) {
                    // F = dir 24 eps (2 sigma^12 dz^-14 - sigma^6 dz^-8), so
                    // dF/dz = dir 24 eps dz^-2 (8 s6 - 28 s6^2) / dz
                    const double invr2 = 1.0 / (dz * dz);
                    const double s6 = (c.wall_sig2[w] * invr2) * (c.wall_sig2[w] * invr2) * (c.wall_sig2[w] * invr2);
                    gz += g.z * c.wall_dir[w] * (24.0 * c.wall_eps[w] * invr2) * (8.0 * s6 - 28.0 * s6 * s6) / dz;
                }
            }
        }
        gxyz[3 * i] = gx;
        gxyz[3 * i + 1] = gy;
        gxyz[3 * i + 2] = gz;
        if (gq) gq[i] = gqi;
    }
    for (int d = 16; d > 0; d >>= 1) {
        gd += __shfl_down_sync(0xffffffffu, gd, d);
        gu += __shfl_down_sync(0xffffffffu, gu, d);
    }
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = gd;
        red[1][threadIdx.x >> 5] = gu;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0, b = 0;
        for (int w = 0; w < ADJ_BLOCK / 32; w++) {
            a += red[0][w];
            b += red[1][w];
        }
        gam[blockIdx.x] = a;
        gam[gridDim.x + blockIdx.x] = b;
    }
}

}  // namespace

int qem_adj_gather_blocks(int N) { return (N + ADJ_BLOCK - 1) / ADJ_BLOCK; }

cudaError_t qem_launch_short_pair_adj(const int64_t *np, int64_t cap, const int2 *pairs, const double4 *pos,
                                      const double *gF, double gE, double4 *RA, const ShortConsts &c,
                                      cudaStream_t s)
{
    if (cap <= 0) return cudaSuccess;
    k_short_pair_adj<<<(int)((cap + ADJ_BLOCK - 1) / ADJ_BLOCK), ADJ_BLOCK, 0, s>>>(np, cap, pairs, pos, gF, gE, RA,
                                                                                   c);
    return cudaGetLastError();
}

cudaError_t qem_launch_adj_gather(int N, bool do_short, bool do_lj, const double4 *pos, const int *pos_of,
                                  const int64_t *poff, const double4 *RA, const int64_t *in_off,
                                  const int *in_list, int64_t cap, const double *gF, double gE,
                                  const ShortConsts &c, double *gxyz, double *gq, double *gam, cudaStream_t s)
{
    if (N <= 0) return cudaSuccess;
    k_adj_gather<<<qem_adj_gather_blocks(N), ADJ_BLOCK, 0, s>>>(N, pos, pos_of, poff, RA, in_off, in_list, cap, gF,
                                                                 gE, c, gxyz, gq, gam, do_short ? 1 : 0,
                                                                 do_lj ? 1 : 0);
    return cudaGetLastError();
}

/*
 * qem_oracle.c -- FP64 CPU oracle for the QEM force/energy hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: it is linked by the
 * test-suite, by __graft_entry__.smoke() and by bench.py's cpu_baseline /
 * reference arm.  The product library (qem4molly_b200/libqem.so) never calls
 * into it, and nothing here is a fallback for the GPU path.
 *
 * It is a literal FP64 restatement of the reference algorithm:
 *   greens_function.jl:17-116   element set-up, Gamma_1/2, dz_Gamma_1/2
 *   Gaussian_int.jl:9-28        Gauss-Legendre mapping to [0, K]
 *   Force_short.jl:4-107        four integrands, F_short_ij, F_short_i
 *   QEM_short.jl:27-59          pair loop F[i] += F_ij, F[j] -= F_ij, self loop
 *   Substrate_LJ.jl:19-46       wall force (with its signed-distance cutoff test)
 *   K_set_generator.jl:5-45     lattice k-set with Float32 probabilities
 *   Force_long.jl:5-242         Fl_non_sort, Fl_sort, Flz_sort_k0, Flz_self,
 *                               F_l_total, F_long (random-batch branch)
 *   QEM_long.jl:39-40           z_list = sortperm(z) (stable, ascending)
 * and, because the Julia package has no energy, the python_lib energies:
 *   Energy_short_range_njit.py:34-99, Energy_long_range_njit.py:10-44,
 *   Sigma_Gamma_func_njit.py:8-69.
 *
 * Third-party arithmetic the reference delegates (un-vendored):
 *   SpecialFunctions.besselj0/besselj1 (v2.2.0)  -> POSIX j0()/j1() from libm
 *   GaussQuadrature.legendre (v0.5.8)            -> own Newton iteration below
 *   CellListMap.neighborlist (v0.8.10)           -> brute-force minimum-image
 *                                                   pair set, d <= cutoff
 *   StatsBase.sample (v0.33.21)                  -> the k-set is fed explicitly
 *
 * Mode flags (parity quirks of the reference):
 *   cutoff_mode 0: Julia (gauss integral to -ln(acc)/(2Lz+a_l), point integral
 *                  to sqrt(4a^2 a_l^2 - 4a ln acc) - 2 a a_l; Force_short.jl:48-67)
 *   cutoff_mode 1: python_lib (gauss to sqrt(-4 alpha ln acc), point to
 *                  -ln(acc)/(2 Lz); Force_short_range_njit.py:51-52)
 *   dir_mode 0: x/y direction from raw coordinate difference (Force_short.jl:57-58)
 *   dir_mode 1: minimum-image direction (neighbor_check.py:28-38)
 *   pair_mode 0: F[j] -= F_ij (QEM_short.jl:46-47)
 *   pair_mode 1: F[j] += F_short_ij(j, i)  (full-list python_lib semantics)
 *   z_ties 0: the z-ordered sums follow sortperm(z) (stable; tied particles
 *             are ordered by index, QEM_long.jl:39-40)
 *   z_ties 1: tied particles are neither below nor above each other
 *             (python_lib equal_cell, Sigma_Gamma_func_njit.py:168-281)
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define QO_PI 3.14159265358979323846

typedef struct {
    double Lx, Ly, Lz;
    double alpha, r_cutoff;
    double gamma_1, gamma_2; /* gamma_1 = gamma_down, gamma_2 = gamma_up */
    double eps_0, accuracy;
    int N_t;
    int cutoff_mode;
    int dir_mode;
    int pair_mode;
    int z_ties; /* 1: equal-z particles are neither below nor above each other in the z-ordered
                   sums (python_lib equal_cell, Sigma_Gamma_func_njit.py:168-281) */
    double pv_eps; /* gamma_1 gamma_2 > 1 (python cutoffs only): half-width of the window around
                      the pole k_0 = ln(gamma_1 gamma_2) / (2 L_z) of the regularised quadrature
                      (Force_short_norm_njit.py; INCAR['eps'] of Force_short_range_njit.py:301) */
} qo_params;

typedef struct {
    double a[4], b[4], sa[4], kf1[4], kf2[4];
    double rho;
} qo_elem;

/* ------------------------------------------------------------------ */
/* Gauss-Legendre nodes on [-1, 1], ascending (GaussQuadrature.legendre)  */
/* ------------------------------------------------------------------ */
int qo_gauss_legendre(int n, double *x, double *w)
{
    if (n < 1) return -1;
    for (int i = 0; i < (n + 1) / 2; i++) {
        double z = cos(QO_PI * (i + 0.75) / (n + 0.5));
        double dp = 0.0;
        for (int it = 0; it < 100; it++) {
            double p0 = 1.0, p1 = z;
            for (int k = 2; k <= n; k++) {
                double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            if (n == 1) { p0 = 1.0; p1 = z; }
            dp = n * (z * p1 - p0) / (z * z - 1.0);
            double dz = p1 / dp;
            z -= dz;
            if (fabs(dz) < 1e-16) {
                /* one more refinement of the derivative at the final z */
                p0 = 1.0; p1 = z;
                for (int k = 2; k <= n; k++) {
                    double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
                    p0 = p1;
                    p1 = p2;
                }
                if (n == 1) { p0 = 1.0; p1 = z; }
                dp = n * (z * p1 - p0) / (z * z - 1.0);
                break;
            }
        }
        double wi = 2.0 / ((1.0 - z * z) * dp * dp);
        x[n - 1 - i] = z;
        x[i] = -z;
        w[i] = wi;
        w[n - 1 - i] = wi;
    }
    if (n % 2 == 1) x[n / 2] = 0.0;
    return 0;
}

/* ------------------------------------------------------------------ */
/* greens_function.jl                                                  */
/* ------------------------------------------------------------------ */
static double jl_sign(double v) { return (v > 0) - (v < 0); }

static void elem_cutoffs(const qo_params *p, qo_elem *e)
{
    double lacc = log(p->accuracy);
    for (int l = 0; l < 4; l++) {
        /* greens_function.jl:26-27 */
        e->kf1[l] = -lacc / (2 * p->Lz + e->a[l]);
        e->kf2[l] = sqrt(4 * p->alpha * p->alpha * e->a[l] * e->a[l] - 4 * p->alpha * lacc) - 2 * p->alpha * e->a[l];
    }
}

/* greens_function.jl:17-30 */
void qo_elem_pair(const qo_params *p, double z_i, double z_j, double rho, qo_elem *e)
{
    double z_n = fabs(z_i - z_j), z_p = z_i + z_j;
    e->a[0] = z_n; e->a[1] = z_p; e->a[2] = 2 * p->Lz - z_p; e->a[3] = 2 * p->Lz - z_n;
    e->b[0] = 1; e->b[1] = p->gamma_1; e->b[2] = p->gamma_2; e->b[3] = p->gamma_1 * p->gamma_2;
    double s = jl_sign(z_i - z_j);
    e->sa[0] = -s; e->sa[1] = -1; e->sa[2] = +1; e->sa[3] = s;
    e->rho = rho;
    elem_cutoffs(p, e);
}

/* greens_function.jl:33-48 */
void qo_elem_self(const qo_params *p, double z_i, qo_elem *e)
{
    double z_p = 2 * z_i;
    e->a[0] = 0; e->a[1] = z_p; e->a[2] = 2 * p->Lz - z_p; e->a[3] = 2 * p->Lz;
    e->b[0] = 1; e->b[1] = p->gamma_1; e->b[2] = p->gamma_2; e->b[3] = p->gamma_1 * p->gamma_2;
    e->sa[0] = 0; e->sa[1] = -1; e->sa[2] = +1; e->sa[3] = 0;
    e->rho = 0;
    elem_cutoffs(p, e);
}

/* greens_function.jl:68-116; l in 1..4 selects one image term, l == 0 sums all */
static double green_u(double k, const qo_elem *e, int l)
{
    if (l == 0) {
        double s = 0;
        for (int i = 0; i < 4; i++) s += e->b[i] * exp(-k * e->a[i]);
        return 0.5 * s;
    }
    return 0.5 * e->b[l - 1] * exp(-k * e->a[l - 1]);
}
static double dz_green_u(double k, const qo_elem *e, int l)
{
    if (l == 0) {
        double s = 0;
        for (int i = 0; i < 4; i++) s += k * e->sa[i] * e->b[i] * exp(-k * e->a[i]);
        return 0.5 * s;
    }
    return 0.5 * k * e->sa[l - 1] * e->b[l - 1] * exp(-k * e->a[l - 1]);
}
double qo_Gamma_1(const qo_params *p, double k, const qo_elem *e, int l)
{
    double gd = p->gamma_1 * p->gamma_2 * exp(-2 * k * p->Lz) - 1;
    return green_u(k, e, l) / gd;
}
double qo_Gamma_2(const qo_params *p, double k, const qo_elem *e, int l)
{
    double gd = p->gamma_1 * p->gamma_2 * exp(-2 * k * p->Lz) - 1;
    return p->gamma_1 * p->gamma_2 * green_u(k, e, l) * exp(-2 * k * p->Lz) / gd;
}
double qo_dz_Gamma_1(const qo_params *p, double k, const qo_elem *e, int l)
{
    double gd = p->gamma_1 * p->gamma_2 * exp(-2 * k * p->Lz) - 1;
    return dz_green_u(k, e, l) / gd;
}
double qo_dz_Gamma_2(const qo_params *p, double k, const qo_elem *e, int l)
{
    double gd = p->gamma_1 * p->gamma_2 * exp(-2 * k * p->Lz) - 1;
    return p->gamma_1 * p->gamma_2 * dz_green_u(k, e, l) * exp(-2 * k * p->Lz) / gd;
}

/* Force_short.jl:4-22 (and the J0-only energy integrands of
 * Energy_short_range_njit.py:20-27) */
enum { F_SR_GAUSS, F_SR_POINT, F_SZ_GAUSS, F_SZ_POINT, U_GAUSS, U_POINT };
static double integrand(int which, const qo_params *p, double k, const qo_elem *e, int l)
{
    switch (which) {
    case F_SR_GAUSS: return k * qo_Gamma_1(p, k, e, l) * exp(-k * k / (4 * p->alpha)) * j1(k * e->rho);
    case F_SR_POINT: return k * qo_Gamma_2(p, k, e, l) * j1(k * e->rho);
    case F_SZ_GAUSS: return qo_dz_Gamma_1(p, k, e, l) * exp(-k * k / (4 * p->alpha)) * j0(k * e->rho);
    case F_SZ_POINT: return qo_dz_Gamma_2(p, k, e, l) * j0(k * e->rho);
    case U_GAUSS: return qo_Gamma_1(p, k, e, l) * exp(-k * k / (4 * p->alpha)) * j0(k * e->rho);
    case U_POINT: return qo_Gamma_2(p, k, e, l) * j0(k * e->rho);
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* gamma_1 gamma_2 > 1: regularised quadrature (python_lib                */
/* Force_short_norm_njit.py:11-414, green_norm_njit.py:6-35,              */
/* Force_short_range_njit.py:258-286).  1 / (g12 e^{-2 k L_z} - 1) has a   */
/* pole at k_0 = ln(g12) / (2 L_z); every integral runs over [0, k_0 - e], */
/* [k_0 - e, k_0 + e], [k_0 + e, 2 k_0] and [2 k_0, k_f] with N_1, 10, N_1 */
/* and N_t - 2 N_1 Gauss-Legendre nodes, N_1 = int(N_t k_0 / k_f), k_f =   */
/* max(python limit, 2.1 k_0).  With f = up(k) / (g12 e^{-2kLz} - 1):      */
/* inside the window f is up(k) gamma_norm(k) - up'(k_0) / (2 L_z)         */
/* (gamma_norm: the pole-free part, by its series), up to 2 k_0 the pole   */
/* term up(k_0) / (2 L_z (k - k_0)) is added (its principal value over     */
/* [0, 2 k_0] is zero), beyond 2 k_0 f itself.                            */
/* ------------------------------------------------------------------ */
static int norm_active(const qo_params *p) { return p->gamma_1 * p->gamma_2 > 1; }

/* green_norm_njit.py:13-33: u / d with ten series terms in x = 2 L_z (k - k_0) */
static double gamma_norm(const qo_params *p, double k)
{
    double g12 = p->gamma_1 * p->gamma_2, k0 = log(g12) / (2 * p->Lz);
    double x = 2 * p->Lz * (k - k0), u = 0.5, d = -1 + x / 2, u0 = 0.5, d0 = x / 2;
    for (int i = 0; i < 10; i++) {
        u0 = u0 * (-x) / (i + 3);
        d0 = d0 * (-x) / (i + 3);
        u += u0;
        d += d0;
    }
    return u / d;
}

/* the integrand without its 1 / (g12 e^{-2kLz} - 1) factor */
static double integrand_up(int which, const qo_params *p, double k, const qo_elem *e, int l)
{
    double g12 = p->gamma_1 * p->gamma_2;
    switch (which) {
    case F_SR_GAUSS: return k * green_u(k, e, l) * exp(-k * k / (4 * p->alpha)) * j1(k * e->rho);
    case F_SR_POINT: return k * g12 * green_u(k, e, l) * exp(-2 * k * p->Lz) * j1(k * e->rho);
    case F_SZ_GAUSS: return dz_green_u(k, e, l) * exp(-k * k / (4 * p->alpha)) * j0(k * e->rho);
    case F_SZ_POINT: return g12 * dz_green_u(k, e, l) * exp(-2 * k * p->Lz) * j0(k * e->rho);
    }
    return 0;
}

/* number of nodes of the two outer sub-intervals below 2 k_0 for a family limit */
int qo_norm_n1(const qo_params *p, int point)
{
    double g12 = p->gamma_1 * p->gamma_2, k0 = log(g12) / (2 * p->Lz);
    double kf = point ? fmax(-log(p->accuracy) / (2 * p->Lz), 2.1 * k0) : fmax(sqrt(-4 * p->alpha * log(p->accuracy)), 2.1 * k0);
    return (int)(p->N_t * k0 / kf);
}

static double gl_int_norm(int which, const qo_params *p, const qo_elem *e, int l)
{
    const int point = (which == F_SR_POINT || which == F_SZ_POINT);
    double g12 = p->gamma_1 * p->gamma_2, k0 = log(g12) / (2 * p->Lz), ep = p->pv_eps;
    double kf = point ? fmax(-log(p->accuracy) / (2 * p->Lz), 2.1 * k0) : fmax(sqrt(-4 * p->alpha * log(p->accuracy)), 2.1 * k0);
    int n1 = (int)(p->N_t * k0 / kf), n3 = p->N_t - 2 * n1;
    double k1 = k0 - 0.01 * ep, k2 = k0 + 0.01 * ep;
    double df = (integrand_up(which, p, k2, e, l) - integrand_up(which, p, k1, e, l)) / (k2 - k1);
    double up0 = integrand_up(which, p, k0, e, l);
    double lo[4] = {0, k0 - ep, k0 + ep, 2 * k0}, hi[4] = {k0 - ep, k0 + ep, 2 * k0, kf};
    int nn[4] = {n1, 10, n1, n3};
    double s = 0, xn[256], wn[256];
    for (int t = 0; t < 4; t++) {
        if (nn[t] < 1) continue;
        qo_gauss_legendre(nn[t], xn, wn);
        double a = lo[t], b = hi[t];
        for (int i = 0; i < nn[t]; i++) {
            double k = 0.5 * (b - a) * xn[i] + 0.5 * (b + a), f;
            if (fabs(k - k0) <= ep) {
                /* the Gauss rho integrand of the window drops its e^{-k^2/4alpha} factor
                   (Force_short_norm_njit.py:59; its df keeps it), reproduced */
                double upk = which == F_SR_GAUSS ? k * green_u(k, e, l) * j1(k * e->rho)
                                                 : integrand_up(which, p, k, e, l);
                f = upk * gamma_norm(p, k) - df / (2 * p->Lz);
            }
            else if (k <= 2 * k0)
                f = integrand_up(which, p, k, e, l) / (g12 * exp(-2 * k * p->Lz) - 1) + up0 / (2 * p->Lz * (k - k0));
            else
                f = integrand_up(which, p, k, e, l) / (g12 * exp(-2 * k * p->Lz) - 1);
            s += 0.5 * (b - a) * (wn[i] * f);
        }
    }
    return s;
}

/* Gaussian_int.jl:9-23 with region (0, K); the regularised form for g12 > 1 */
static double gl_int(int which, const qo_params *p, const qo_elem *e, int l, double K,
                     const double *xn, const double *wn)
{
    if (norm_active(p) && which != U_GAUSS && which != U_POINT) return gl_int_norm(which, p, e, l);
    double s = 0;
    for (int i = 0; i < p->N_t; i++) {
        double x = K / 2 + K * xn[i] / 2;
        double w = K * wn[i] / 2;
        s += integrand(which, p, x, e, l) * w;
    }
    return s;
}

/* quadrature upper limits per image term for the two integral families */
static double gauss_limit(const qo_params *p, const qo_elem *e, int l)
{
    if (p->cutoff_mode == 1) return sqrt(-4 * p->alpha * log(p->accuracy));
    return e->kf1[l];
}
static double point_limit(const qo_params *p, const qo_elem *e, int l)
{
    if (p->cutoff_mode == 1) return -log(p->accuracy) / (2 * p->Lz);
    return e->kf2[l];
}

static void gl_nodes(const qo_params *p, double *xn, double *wn)
{
    qo_gauss_legendre(p->N_t, xn, wn);
}

/* minimum-image in-plane separation of i from j */
static void min_image(const qo_params *p, const double *ci, const double *cj, double *dx, double *dy)
{
    double x = ci[0] - cj[0], y = ci[1] - cj[1];
    x -= p->Lx * nearbyint(x / p->Lx);
    y -= p->Ly * nearbyint(y / p->Ly);
    *dx = x;
    *dy = y;
}

/* z-force on target t from source s (the F_sz part of Force_short.jl:64-72) */
static double pair_fz(const qo_params *p, const qo_elem *e, int single, const double *xn, const double *wn)
{
    double Fp1 = 0, Fp2 = 0, Fg = 0;
    for (int l = 1; l <= 4; l++) Fp1 += gl_int(F_SZ_POINT, p, e, l, point_limit(p, e, l - 1), xn, wn);
    for (int l = 0; l < 4; l++)
        Fp2 += e->b[l] * e->a[l] * e->sa[l] / pow(e->a[l] * e->a[l] + e->rho * e->rho, 1.5);
    Fp2 *= 0.5;
    if (!single)
        for (int l = 1; l <= 4; l++) Fg += gl_int(F_SZ_GAUSS, p, e, l, gauss_limit(p, e, l - 1), xn, wn);
    return +Fp1 - Fp2 - Fg;
}

/*
 * Force_short.jl:25-78.  out[0..2] = F_ij (force on i from j), out[3] = the
 * z-force on j from i as F_short_ij(j, i) would return it (used in
 * pair_mode 1).  Returns 0 when the minimum-image rho exceeds r_cutoff
 * (the per-pair neighborlist re-check of Force_short.jl:36-41).
 */
int qo_F_short_ij(const qo_params *p, double q_i, double q_j, const double *ci, const double *cj,
                  int single, double *out)
{
    double xn[256], wn[256];
    gl_nodes(p, xn, wn);
    out[0] = out[1] = out[2] = out[3] = 0;
    double dx, dy;
    min_image(p, ci, cj, &dx, &dy);
    double rho2 = dx * dx + dy * dy;
    if (rho2 > p->r_cutoff * p->r_cutoff) return 0;
    double rho = sqrt(rho2);
    qo_elem e;
    qo_elem_pair(p, ci[2], cj[2], rho, &e);
    double Fsx = 0, Fsy = 0;
    if (rho != 0) {
        double Fp1 = 0, Fp2 = 0, Fg = 0;
        for (int l = 1; l <= 4; l++) Fp1 += gl_int(F_SR_POINT, p, &e, l, point_limit(p, &e, l - 1), xn, wn);
        for (int l = 0; l < 4; l++) Fp2 += e.b[l] * rho / pow(e.a[l] * e.a[l] + rho * rho, 1.5);
        Fp2 *= 0.5;
        if (!single)
            for (int l = 1; l <= 4; l++) Fg += gl_int(F_SR_GAUSS, p, &e, l, gauss_limit(p, &e, l - 1), xn, wn);
        double Fsr = -Fp1 + Fp2 + Fg;
        double ddx = (p->dir_mode == 1) ? dx : (ci[0] - cj[0]);
        double ddy = (p->dir_mode == 1) ? dy : (ci[1] - cj[1]);
        Fsx = Fsr * ddx / rho;
        Fsy = Fsr * ddy / rho;
    }
    double Fsz = pair_fz(p, &e, single, xn, wn);
    double pref = q_i * q_j / (2 * QO_PI * p->eps_0);
    out[0] = pref * Fsx;
    out[1] = pref * Fsy;
    out[2] = pref * Fsz;
    /* F_short_ij(j, i): same a, b and rho; image signs of l = 1, 4 flip */
    qo_elem ej;
    qo_elem_pair(p, cj[2], ci[2], rho, &ej);
    out[3] = pref * pair_fz(p, &ej, single, xn, wn);
    return 1;
}

/* Force_short.jl:82-107: self (image) z-force on particle i */
double qo_F_short_i(const qo_params *p, double q_i, const double *ci, int single)
{
    double xn[256], wn[256];
    gl_nodes(p, xn, wn);
    qo_elem e;
    qo_elem_self(p, ci[2], &e);
    double Fp1 = 0, Fp2 = 0, Fg = 0;
    for (int l = 1; l <= 4; l++) Fp1 += gl_int(F_SZ_POINT, p, &e, l, point_limit(p, &e, l - 1), xn, wn);
    for (int l = 1; l <= 2; l++) Fp2 += e.b[l] * e.a[l] * e.sa[l] / (e.a[l] * e.a[l] * e.a[l]);
    Fp2 *= 0.5;
    if (!single)
        for (int l = 1; l <= 4; l++) Fg += gl_int(F_SZ_GAUSS, p, &e, l, gauss_limit(p, &e, l - 1), xn, wn);
    /* for g12 > 1 the self force adds the point integral with the opposite sign
       (Force_short_norm_njit.py:330-331 against Force_short_range_njit.py:224), reproduced */
    double Fszi = (norm_active(p) ? Fp1 : -Fp1) + Fp2 + Fg;
    return -q_i * q_i / (2 * QO_PI * p->eps_0) * Fszi;
}

/* ------------------------------------------------------------------ */
/* pair set (CellListMap.neighborlist semantics: min-image d <= cutoff) */
/* ------------------------------------------------------------------ */
/* Canonical (i < j) pairs in lexicographic order.  Returns the number of
 * pairs; writes at most cap pairs. */
long qo_pairs_bruteforce(const qo_params *p, int N, const double *xyz, int *pairs, long cap)
{
    long n = 0;
    double rc2 = p->r_cutoff * p->r_cutoff;
    for (int i = 0; i < N; i++)
        for (int j = i + 1; j < N; j++) {
            double dx, dy;
            min_image(p, xyz + 3 * i, xyz + 3 * j, &dx, &dy);
            if (dx * dx + dy * dy <= rc2) {
                if (n < cap) { pairs[2 * n] = i; pairs[2 * n + 1] = j; }
                n++;
            }
        }
    return n;
}

/* Cell-list variant for large N; same set and the same lexicographic order. */
static int cmp_int(const void *a, const void *b) { return (*(const int *)a > *(const int *)b) - (*(const int *)a < *(const int *)b); }
long qo_pairs_cells(const qo_params *p, int N, const double *xyz, int *pairs, long cap)
{
    int ncx = (int)floor(p->Lx / p->r_cutoff), ncy = (int)floor(p->Ly / p->r_cutoff);
    if (ncx < 3 || ncy < 3) return qo_pairs_bruteforce(p, N, xyz, pairs, cap);
    double lx = p->Lx / ncx, ly = p->Ly / ncy;
    int nc = ncx * ncy;
    int *cnt = calloc(nc + 1, sizeof(int)), *cell = malloc(sizeof(int) * (N > 0 ? N : 1)),
        *lst = malloc(sizeof(int) * (N > 0 ? N : 1));
    for (int i = 0; i < N; i++) {
        double x = xyz[3 * i] - p->Lx * floor(xyz[3 * i] / p->Lx);
        double y = xyz[3 * i + 1] - p->Ly * floor(xyz[3 * i + 1] / p->Ly);
        int cx = (int)(x / lx), cy = (int)(y / ly);
        if (cx >= ncx) cx = ncx - 1;
        if (cy >= ncy) cy = ncy - 1;
        cell[i] = cx * ncy + cy;
        cnt[cell[i] + 1]++;
    }
    for (int c = 0; c < nc; c++) cnt[c + 1] += cnt[c];
    int *fill = malloc(sizeof(int) * (nc + 1));
    memcpy(fill, cnt, sizeof(int) * (nc + 1));
    for (int i = 0; i < N; i++) lst[fill[cell[i]]++] = i;
    free(fill);
    double rc2 = p->r_cutoff * p->r_cutoff;
    long n = 0;
    int *nb = malloc(sizeof(int) * (N > 0 ? N : 1));
    for (int i = 0; i < N; i++) {
        int cx = cell[i] / ncy, cy = cell[i] % ncy, m = 0;
        for (int ox = -1; ox <= 1; ox++)
            for (int oy = -1; oy <= 1; oy++) {
                int c = ((cx + ox + ncx) % ncx) * ncy + (cy + oy + ncy) % ncy;
                for (int t = cnt[c]; t < cnt[c + 1]; t++) {
                    int j = lst[t];
                    if (j <= i) continue;
                    double dx, dy;
                    min_image(p, xyz + 3 * i, xyz + 3 * j, &dx, &dy);
                    if (dx * dx + dy * dy <= rc2) nb[m++] = j;
                }
            }
        qsort(nb, m, sizeof(int), cmp_int);
        for (int t = 0; t < m; t++) {
            if (n < cap) { pairs[2 * n] = i; pairs[2 * n + 1] = nb[t]; }
            n++;
        }
    }
    free(nb); free(cnt); free(cell); free(lst);
    return n;
}

/* ------------------------------------------------------------------ */
/* QEM_short.jl:27-59                                                  */
/* ------------------------------------------------------------------ */
/* F (3N) is overwritten.  Pairs are evaluated in parallel (nthreads) into a
 * per-pair buffer and accumulated sequentially in list order, so the result
 * does not depend on the thread count. */
void qo_short_forces(const qo_params *p, int N, const double *xyz, const double *q,
                     long npairs, const int *pairs, double *F, int nthreads)
{
    double *Fp = malloc(sizeof(double) * 4 * (npairs > 0 ? npairs : 1));
    double *Fs = malloc(sizeof(double) * (N > 0 ? N : 1));
#ifdef _OPENMP
    if (nthreads < 1) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads)
#endif
    for (long t = 0; t < npairs; t++) {
        int i = pairs[2 * t], j = pairs[2 * t + 1];
        qo_F_short_ij(p, q[i], q[j], xyz + 3 * i, xyz + 3 * j, 0, Fp + 4 * t);
    }
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads)
#endif
    for (int i = 0; i < N; i++) Fs[i] = qo_F_short_i(p, q[i], xyz + 3 * i, 0);
    memset(F, 0, sizeof(double) * 3 * N);
    for (long t = 0; t < npairs; t++) {
        int i = pairs[2 * t], j = pairs[2 * t + 1];
        const double *f = Fp + 4 * t;
        F[3 * i] += f[0]; F[3 * i + 1] += f[1]; F[3 * i + 2] += f[2];
        F[3 * j] -= f[0]; F[3 * j + 1] -= f[1];
        if (p->pair_mode == 1) F[3 * j + 2] += f[3];
        else F[3 * j + 2] -= f[2];
    }
    for (int i = 0; i < N; i++) F[3 * i + 2] += Fs[i];
    free(Fp);
    free(Fs);
}

/* ------------------------------------------------------------------ */
/* Substrate_LJ.jl:19-46 (accumulates into F; returns the number of    */
/* particles that violate direction*dz > 0, the reference's @assert)   */
/* ------------------------------------------------------------------ */
int qo_lj_forces(int N, const double *xyz, double cutoff, double sigma, double eps, double sub_pos,
                 double direction, double *F)
{
    int bad = 0;
    double sigma2 = sigma * sigma;
    for (int i = 0; i < N; i++) {
        double dz = xyz[3 * i + 2] - sub_pos;
        if (!(direction * dz > 0)) { bad++; continue; }
        if (dz < cutoff) {
            double invr2 = 1 / (dz * dz);
            double six = pow(sigma2 * invr2, 3);
            F[3 * i + 2] += direction * ((24 * eps * invr2) * (2 * six * six - six));
        }
    }
    return bad;
}

/* ------------------------------------------------------------------ */
/* K_set_generator.jl:5-45.  Writes at most cap entries of (kx, ky, k)  */
/* and Float32 probabilities; returns the number of lattice points.     */
/* ------------------------------------------------------------------ */
long qo_kset_generator(double Lx, double Ly, double alpha, double accuracy, double *K, float *P,
                       double *sum_K_out, long cap)
{
    double k_c = 2 * sqrt(-4 * alpha * log(accuracy));
    long mx_max = (long)ceil(k_c * Lx / (2 * QO_PI)) + 1;
    long my_max = (long)ceil(k_c * Ly / (2 * QO_PI)) + 1;
    double S_x = 0, S_y = 0;
    for (long m = -mx_max; m <= mx_max; m++)
        if (m != 0) { double kx = m * 2 * QO_PI / Lx; S_x += exp(-kx * kx / (4 * alpha)); }
    for (long m = -my_max; m <= my_max; m++)
        if (m != 0) { double ky = m * 2 * QO_PI / Ly; S_y += exp(-ky * ky / (4 * alpha)); }
    double sum_K = S_x + S_y + S_x * S_y;
    long n = 0;
    for (long mx = -mx_max; mx <= mx_max; mx++)
        for (long my = -my_max; my <= my_max; my++) {
            double kx = mx * 2 * QO_PI / Lx, ky = my * 2 * QO_PI / Ly;
            double k = sqrt(kx * kx + ky * ky);
            if (k != 0) {
                if (n < cap) {
                    K[3 * n] = kx; K[3 * n + 1] = ky; K[3 * n + 2] = k;
                    P[n] = (float)(exp(-k * k / (4 * alpha)) / sum_K);
                }
                n++;
            }
        }
    *sum_K_out = sum_K;
    return n;
}

/* ------------------------------------------------------------------ */
/* QEM_long.jl:39-40  sortperm(z): stable ascending (merge sort)        */
/* ------------------------------------------------------------------ */
static void msort(int *a, int *tmp, int n, const double *z)
{
    if (n < 2) return;
    int h = n / 2;
    msort(a, tmp, h, z);
    msort(a + h, tmp, n - h, z);
    int i = 0, j = h, k = 0;
    while (i < h && j < n) tmp[k++] = (z[a[j]] < z[a[i]]) ? a[j++] : a[i++];
    while (i < h) tmp[k++] = a[i++];
    while (j < n) tmp[k++] = a[j++];
    memcpy(a, tmp, sizeof(int) * n);
}
void qo_sortperm_z(int N, const double *xyz, int *zlist)
{
    double *z = malloc(sizeof(double) * (N > 0 ? N : 1));
    int *tmp = malloc(sizeof(int) * (N > 0 ? N : 1));
    for (int i = 0; i < N; i++) { z[i] = xyz[3 * i + 2]; zlist[i] = i; }
    msort(zlist, tmp, N, z);
    free(z);
    free(tmp);
}

/* ------------------------------------------------------------------ */
/* Force_long.jl                                                        */
/* ------------------------------------------------------------------ */
/* Force_long.jl:5-70.  out is 3N (overwritten). */
void qo_Fl_non_sort(const double *kset, int N, const double *xyz, const double *q, double g1, double g2,
                    double Lz, double *out, int nthreads)
{
    double kx = kset[0], ky = kset[1], k = kset[2];
    double f0[4] = {0, 0, 0, 0};
    for (int i = 0; i < N; i++) {
        double x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
        f0[0] += q[i] * cos(kx * x + ky * y) * exp(+k * z);
        f0[1] += q[i] * sin(kx * x + ky * y) * exp(+k * z);
        f0[2] += q[i] * cos(kx * x + ky * y) * exp(-k * z);
        f0[3] += q[i] * sin(kx * x + ky * y) * exp(-k * z);
    }
    double gv = 0.5 / (g1 * g2 * exp(-2 * k * Lz) - 1);
    double Gp[4] = {g2, 1, g1, g1 * g2};
    (void)nthreads;
#ifdef _OPENMP
    if (nthreads < 1) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(static) num_threads(nthreads)
#endif
    for (int i = 0; i < N; i++) {
        double qi = q[i], x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
        double c = cos(kx * x + ky * y), s = sin(kx * x + ky * y);
        double f[4];
        f[0] = f0[0] - qi * c * exp(+k * z);
        f[1] = f0[1] - qi * s * exp(+k * z);
        f[2] = f0[2] - qi * c * exp(-k * z);
        f[3] = f0[3] - qi * s * exp(-k * z);
        double E = exp(-2 * k * Lz), ep = exp(k * z), em = exp(-k * z);
        double sum_xy = qi * gv *
                        (c * (Gp[0] * E * ep * f[1] + Gp[2] * em * f[3] + Gp[3] * E * em * f[1] + Gp[3] * E * ep * f[3]) -
                         s * (Gp[0] * E * ep * f[0] + Gp[2] * em * f[2] + Gp[3] * E * em * f[0] + Gp[3] * E * ep * f[2]));
        double sum_z = qi * gv *
                       (c * (Gp[0] * E * ep * f[0] - Gp[2] * em * f[2] - Gp[3] * E * em * f[0] + Gp[3] * E * ep * f[2]) +
                        s * (Gp[0] * E * ep * f[1] - Gp[2] * em * f[3] - Gp[3] * E * em * f[1] + Gp[3] * E * ep * f[3]));
        out[3 * i] = (kx / k) * sum_xy;
        out[3 * i + 1] = (ky / k) * sum_xy;
        out[3 * i + 2] = sum_z;
    }
}

/* Force_long.jl:72-127.  zlist is 0-based. */
void qo_Fl_sort(const double *kset, int N, const int *zlist, const double *xyz, const double *q, double *out,
                int nthreads)
{
    double kx = kset[0], ky = kset[1], k = kset[2];
    double *A = calloc(4 * (size_t)(N > 0 ? N : 1), sizeof(double));
    double *B = A + N, *C = B + N, *D = C + N;
    for (int i = 1; i < N; i++) {
        int l = zlist[i];
        double x = xyz[3 * l], y = xyz[3 * l + 1], z = xyz[3 * l + 2];
        C[0] += q[l] * exp(-k * z) * cos(kx * x + ky * y);
        D[0] += q[l] * exp(-k * z) * sin(kx * x + ky * y);
    }
    for (int i = 0; i < N - 1; i++) {
        int l = zlist[i], lp1 = zlist[i + 1];
        double x = xyz[3 * l], y = xyz[3 * l + 1], z = xyz[3 * l + 2];
        double x1 = xyz[3 * lp1], y1 = xyz[3 * lp1 + 1], z1 = xyz[3 * lp1 + 2];
        A[i + 1] = A[i] + q[l] * exp(+k * z) * cos(kx * x + ky * y);
        B[i + 1] = B[i] + q[l] * exp(+k * z) * sin(kx * x + ky * y);
        C[i + 1] = C[i] - q[lp1] * exp(-k * z1) * cos(kx * x1 + ky * y1);
        D[i + 1] = D[i] - q[lp1] * exp(-k * z1) * sin(kx * x1 + ky * y1);
    }
    (void)nthreads;
#ifdef _OPENMP
    if (nthreads < 1) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(static) num_threads(nthreads)
#endif
    for (int i = 0; i < N; i++) {
        int l = zlist[i];
        double qi = q[l], x = xyz[3 * l], y = xyz[3 * l + 1], z = xyz[3 * l + 2];
        double c = cos(kx * x + ky * y), s = sin(kx * x + ky * y);
        double sum_xy = s * exp(-k * z) * A[i] - c * exp(-k * z) * B[i] + s * exp(k * z) * C[i] - c * exp(k * z) * D[i];
        out[3 * l] = qi * kx / (2 * k) * sum_xy;
        out[3 * l + 1] = qi * ky / (2 * k) * sum_xy;
        out[3 * l + 2] = (qi / 2) * (c * exp(-k * z) * A[i] + s * exp(-k * z) * B[i] - c * exp(k * z) * C[i] -
                                     s * exp(k * z) * D[i]);
    }
    free(A);
}

/* Force_long.jl:130-161 (returns q_i (Q_1 - Q_2) in out[3i+2], x/y zero) */
void qo_Flz_sort_k0(int N, const int *zlist, const double *q, double *out)
{
    double *Q1 = calloc(2 * (size_t)(N > 0 ? N : 1), sizeof(double)), *Q2 = Q1 + N;
    for (int i = 1; i < N; i++) Q2[0] += q[zlist[i]];
    for (int i = 0; i < N - 1; i++) Q1[i + 1] = Q1[i] + q[zlist[i]];
    for (int i = 1; i < N; i++) Q2[i] = Q2[i - 1] - q[zlist[i]];
    memset(out, 0, sizeof(double) * 3 * N);
    for (int j = 0; j < N; j++) {
        int l = zlist[j];
        out[3 * l + 2] = q[l] * (Q1[j] - Q2[j]);
    }
    free(Q1);
}

/* Equal-z groups of the z order: g0[i], g1[i] = first and one-past-last sorted
 * position of the group of sorted position i (a new group starts where z
 * strictly increases, as the equal_cell construction of
 * Force_long_range_njit_exact.py:130-156). */
static void z_groups(int N, const int *zlist, const double *xyz, int *g0, int *g1)
{
    int s = 0;
    for (int i = 1; i <= N; i++)
        if (i == N || xyz[3 * zlist[i] + 2] > xyz[3 * zlist[i - 1] + 2]) {
            for (int t = s; t < i; t++) {
                g0[t] = s;
                g1[t] = i;
            }
            s = i;
        }
}

/* Fl_sort with equal-z groups (Sigma_Gamma_func_njit.py:168-238): the x / y
 * parts as Fl_sort (F_long_xy_sum_2 takes the plain order), the z part with
 * sums over strictly lower (A, B) and strictly higher (C, D) groups. */
void qo_Fl_sort_ties(const double *kset, int N, const int *zlist, const double *xyz, const double *q, double *out,
                     int nthreads)
{
    qo_Fl_sort(kset, N, zlist, xyz, q, out, nthreads);
    if (N == 0) return;
    double kx = kset[0], ky = kset[1], k = kset[2];
    double *PA = calloc(4 * (size_t)(N + 1), sizeof(double)), *PB = PA + N + 1, *SC = PB + N + 1, *SD = SC + N + 1;
    int *g0 = malloc(sizeof(int) * 2 * (size_t)N), *g1 = g0 + N;
    z_groups(N, zlist, xyz, g0, g1);
    for (int i = 0; i < N; i++) { /* PA[i] = sum over sorted positions < i */
        int l = zlist[i];
        double x = xyz[3 * l], y = xyz[3 * l + 1], z = xyz[3 * l + 2];
        PA[i + 1] = PA[i] + q[l] * exp(+k * z) * cos(kx * x + ky * y);
        PB[i + 1] = PB[i] + q[l] * exp(+k * z) * sin(kx * x + ky * y);
    }
    for (int i = N - 1; i >= 0; i--) { /* SC[i] = sum over sorted positions >= i */
        int l = zlist[i];
        double x = xyz[3 * l], y = xyz[3 * l + 1], z = xyz[3 * l + 2];
        SC[i] = SC[i + 1] + q[l] * exp(-k * z) * cos(kx * x + ky * y);
        SD[i] = SD[i + 1] + q[l] * exp(-k * z) * sin(kx * x + ky * y);
    }
    for (int i = 0; i < N; i++) {
        int l = zlist[i];
        double qi = q[l], x = xyz[3 * l], y = xyz[3 * l + 1], z = xyz[3 * l + 2];
        double c = cos(kx * x + ky * y), s = sin(kx * x + ky * y);
        double A = PA[g0[i]], B = PB[g0[i]], Cs = SC[g1[i]], D = SD[g1[i]];
        out[3 * l + 2] = (qi / 2) * (c * exp(-k * z) * A + s * exp(-k * z) * B - c * exp(k * z) * Cs -
                                     s * exp(k * z) * D);
    }
    free(g0);
    free(PA);
}

/* Flz_sort_k0 with equal-z groups (Sigma_Gamma_func_njit.py:240-281) */
void qo_Flz_sort_k0_ties(int N, const int *zlist, const double *xyz, const double *q, double *out)
{
    memset(out, 0, sizeof(double) * 3 * (size_t)N);
    if (N == 0) return;
    double *P = calloc((size_t)N + 1, sizeof(double)), tot = 0;
    int *g0 = malloc(sizeof(int) * 2 * (size_t)N), *g1 = g0 + N;
    z_groups(N, zlist, xyz, g0, g1);
    for (int i = 0; i < N; i++) P[i + 1] = P[i] + q[zlist[i]];
    tot = P[N];
    for (int i = 0; i < N; i++) {
        int l = zlist[i];
        out[3 * l + 2] = q[l] * (P[g0[i]] - (tot - P[g1[i]]));
    }
    free(g0);
    free(P);
}

/* Force_long.jl:164-184 (z only) */
void qo_Flz_self(const double *kset, int N, const double *xyz, const double *q, double g1, double g2, double Lz,
                 double *out)
{
    double k = kset[2];
    double gv = g1 * g2 * exp(-2 * k * Lz) - 1;
    for (int i = 0; i < N; i++) {
        double z = xyz[3 * i + 2];
        out[3 * i] = 0;
        out[3 * i + 1] = 0;
        out[3 * i + 2] = q[i] * q[i] * (g2 * exp(-2 * k * (Lz - z)) - g1 * exp(-2 * k * z)) / (2 * gv);
    }
}

/* Force_long.jl:186-199.  out (3N) overwritten. */
void qo_F_l_total(const qo_params *p, const double *kset, int N, const double *xyz, const double *q,
                  const int *zlist, double *out, int nthreads)
{
    double *a = malloc(sizeof(double) * 9 * (size_t)(N > 0 ? N : 1)), *b = a + 3 * N, *c = b + 3 * N;
    qo_Fl_non_sort(kset, N, xyz, q, p->gamma_1, p->gamma_2, p->Lz, a, nthreads);
    if (p->z_ties) qo_Fl_sort_ties(kset, N, zlist, xyz, q, b, nthreads);
    else qo_Fl_sort(kset, N, zlist, xyz, q, b, nthreads);
    qo_Flz_self(kset, N, xyz, q, p->gamma_1, p->gamma_2, p->Lz, c);
    double den = p->Lx * p->Ly * p->eps_0;
    for (int t = 0; t < 3 * N; t++) out[t] = (a[t] + b[t] + c[t]) / den;
    free(a);
}

/* Force_long.jl:201-242, random-batch branch, with the sampled k-set given
 * explicitly (P rows of kx, ky, k) and sum_K.  F (3N) overwritten. */
void qo_F_long(const qo_params *p, int N, const double *xyz, const double *q, const int *zlist_in, int P,
               const double *kset, double sum_K, double *F, int nthreads)
{
    int *zlist = malloc(sizeof(int) * (N > 0 ? N : 1));
    if (zlist_in) memcpy(zlist, zlist_in, sizeof(int) * N);
    else qo_sortperm_z(N, xyz, zlist);
    double *t = malloc(sizeof(double) * 3 * (size_t)(N > 0 ? N : 1));
    if (p->z_ties) qo_Flz_sort_k0_ties(N, zlist, xyz, q, t);
    else qo_Flz_sort_k0(N, zlist, q, t);
    double den0 = 2 * p->Lx * p->Ly * p->eps_0;
    for (int i = 0; i < 3 * N; i++) F[i] = 0 + t[i] / den0;
    double w = sum_K / P;
    for (int m = 0; m < P; m++) {
        qo_F_l_total(p, kset + 3 * m, N, xyz, q, zlist, t, nthreads);
        for (int i = 0; i < 3 * N; i++) F[i] += t[i] * w;
    }
    free(t);
    free(zlist);
}

/* ------------------------------------------------------------------ */
/* Energies (python_lib formulas; Julia-mode uses the per-image cutoffs) */
/* ------------------------------------------------------------------ */
/* Energy_short_range_njit.py:34-61 for one unordered pair, returned per
 * unordered pair (q_i q_j / (2 pi eps_0) * U; the python full-list sum
 * counts each ordered pair with 1 / (4 pi)). */
double qo_energy_pair(const qo_params *p, double q_i, double q_j, const double *ci, const double *cj)
{
    double xn[256], wn[256];
    gl_nodes(p, xn, wn);
    double dx, dy;
    min_image(p, ci, cj, &dx, &dy);
    double rho2 = dx * dx + dy * dy;
    if (rho2 > p->r_cutoff * p->r_cutoff) return 0;
    double rho = sqrt(rho2);
    qo_elem e;
    qo_elem_pair(p, ci[2], cj[2], rho, &e);
    double Ug = 0, Up = 0, Ub = 0;
    for (int l = 1; l <= 4; l++) Ug += gl_int(U_GAUSS, p, &e, l, gauss_limit(p, &e, l - 1), xn, wn);
    for (int l = 1; l <= 4; l++) Up += gl_int(U_POINT, p, &e, l, point_limit(p, &e, l - 1), xn, wn);
    for (int l = 0; l < 4; l++) Ub += 0.5 * e.b[l] / sqrt(e.a[l] * e.a[l] + rho * rho);
    return q_i * q_j / (2 * QO_PI * p->eps_0) * (Ug - Up + Ub);
}

/* Energy_short_range_njit.py:64-81 */
double qo_energy_self(const qo_params *p, double q_i, const double *ci)
{
    double xn[256], wn[256];
    gl_nodes(p, xn, wn);
    qo_elem e;
    qo_elem_self(p, ci[2], &e);
    double Ug = 0, Up = 0, Ub = 0;
    for (int l = 1; l <= 4; l++) Ug += gl_int(U_GAUSS, p, &e, l, gauss_limit(p, &e, l - 1), xn, wn);
    for (int l = 1; l <= 4; l++) Up += gl_int(U_POINT, p, &e, l, point_limit(p, &e, l - 1), xn, wn);
    for (int l = 1; l < 4; l++) Ub += 0.5 * e.b[l] / e.a[l];
    return q_i * q_i / (4 * QO_PI * p->eps_0) * (Ug - Up + Ub);
}

/* Energy_short_range_njit.py:84-99 (pair list given, canonical i<j) */
double qo_energy_short(const qo_params *p, int N, const double *xyz, const double *q, long npairs,
                       const int *pairs, int nthreads)
{
    double *Up = malloc(sizeof(double) * (npairs > 0 ? npairs : 1));
    double *Us = malloc(sizeof(double) * (N > 0 ? N : 1));
    (void)nthreads;
#ifdef _OPENMP
    if (nthreads < 1) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads)
#endif
    for (long t = 0; t < npairs; t++) {
        int i = pairs[2 * t], j = pairs[2 * t + 1];
        Up[t] = qo_energy_pair(p, q[i], q[j], xyz + 3 * i, xyz + 3 * j);
    }
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads)
#endif
    for (int i = 0; i < N; i++) Us[i] = qo_energy_self(p, q[i], xyz + 3 * i);
    double E = 0;
    for (long t = 0; t < npairs; t++) E += Up[t];
    for (int i = 0; i < N; i++) E += Us[i];
    free(Up);
    free(Us);
    return E;
}

/* Sigma_Gamma_func_njit.py:8-28 */
double qo_sigma_s(const double *kset, int N, const double *xyz, const double *q, double g1, double g2, double Lz)
{
    double kx = kset[0], ky = kset[1], k = kset[2];
    double f[4] = {0, 0, 0, 0};
    for (int i = 0; i < N; i++) {
        double x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
        f[0] += q[i] * cos(kx * x + ky * y) * exp(+k * z);
        f[1] += q[i] * sin(kx * x + ky * y) * exp(+k * z);
        f[2] += q[i] * cos(kx * x + ky * y) * exp(-k * z);
        f[3] += q[i] * sin(kx * x + ky * y) * exp(-k * z);
    }
    double D = g1 * g2 * exp(-2 * k * Lz) - 1;
    double G0 = g2 / (2 * D), G2 = g1 / (2 * D), G3 = g1 * g2 / (2 * D);
    double v = G0 * (f[0] * f[0] + f[1] * f[1]) * exp(-2 * k * Lz) + G2 * (f[2] * f[2] + f[3] * f[3]) +
               G3 * (f[0] * f[2] + f[1] * f[3]) * exp(-2 * k * Lz);
    return v / k;
}

/* Sigma_Gamma_func_njit.py:31-69 */
double qo_sigma_ns(const double *kset, int N, const double *xyz, const double *q, const int *zlist)
{
    double kx = kset[0], ky = kset[1], k = kset[2];
    double *A = calloc(4 * (size_t)(N > 0 ? N : 1), sizeof(double));
    double *B = A + N, *C = B + N, *D = C + N;
    for (int i = 1; i < N; i++) {
        int l = zlist[i];
        double x = xyz[3 * l], y = xyz[3 * l + 1], z = xyz[3 * l + 2];
        C[0] += q[l] * exp(-k * z) * cos(kx * x + ky * y);
        D[0] += q[l] * exp(-k * z) * sin(kx * x + ky * y);
    }
    for (int i = 0; i < N - 1; i++) {
        int l = zlist[i], lp1 = zlist[i + 1];
        double x = xyz[3 * l], y = xyz[3 * l + 1], z = xyz[3 * l + 2];
        double x1 = xyz[3 * lp1], y1 = xyz[3 * lp1 + 1], z1 = xyz[3 * lp1 + 2];
        A[i + 1] = A[i] + q[l] * exp(+k * z) * cos(kx * x + ky * y);
        B[i + 1] = B[i] + q[l] * exp(+k * z) * sin(kx * x + ky * y);
        C[i + 1] = C[i] - q[lp1] * exp(-k * z1) * cos(kx * x1 + ky * y1);
        D[i + 1] = D[i] - q[lp1] * exp(-k * z1) * sin(kx * x1 + ky * y1);
    }
    double v = 0;
    for (int i = 0; i < N; i++) {
        int l = zlist[i];
        double qi = q[l], x = xyz[3 * l], y = xyz[3 * l + 1], z = xyz[3 * l + 2];
        v += -qi * qi;
        v += -qi * exp(-k * z) * cos(kx * x + ky * y) * A[i];
        v += -qi * exp(-k * z) * sin(kx * x + ky * y) * B[i];
        v += -qi * exp(+k * z) * cos(kx * x + ky * y) * C[i];
        v += -qi * exp(+k * z) * sin(kx * x + ky * y) * D[i];
    }
    free(A);
    v = v / k;
    return v / 2;
}

/* Energy_long_range_njit.py:25-44 */
double qo_energy_k0(const qo_params *p, int N, const double *xyz, const double *q, const int *zlist)
{
    if (N == 0) return 0;
    double *Qa = calloc(2 * (size_t)N, sizeof(double)), *Qb = Qa + N;
    Qa[0] = 0;
    Qb[0] = -q[zlist[0]];
    for (int i = 0; i < N - 1; i++) {
        Qa[i + 1] = Qa[i] + q[zlist[i]];
        Qb[i + 1] = Qb[i] - q[zlist[i + 1]];
    }
    double v = 0;
    for (int i = 0; i < N; i++) v += 2 * q[zlist[i]] * xyz[3 * zlist[i] + 2] * (Qa[i] - Qb[i]);
    free(Qa);
    return -v / (4 * p->eps_0 * p->Lx * p->Ly);
}

/* Energy_long_range_njit.py:10-22 + 25-44 with the sampled k-set given */
double qo_energy_long(const qo_params *p, int N, const double *xyz, const double *q, const int *zlist_in, int P,
                      const double *kset, double sum_K)
{
    int *zlist = malloc(sizeof(int) * (N > 0 ? N : 1));
    if (zlist_in) memcpy(zlist, zlist_in, sizeof(int) * N);
    else qo_sortperm_z(N, xyz, zlist);
    double Es = 0, Ens = 0;
    for (int m = 0; m < P; m++) {
        Es += -(sum_K / P) * qo_sigma_s(kset + 3 * m, N, xyz, q, p->gamma_1, p->gamma_2, p->Lz) /
              (2 * p->eps_0 * p->Lx * p->Ly);
        Ens += -(sum_K / P) * qo_sigma_ns(kset + 3 * m, N, xyz, q, zlist) / (2 * p->eps_0 * p->Lx * p->Ly);
    }
    double E = Es + Ens + qo_energy_k0(p, N, xyz, q, zlist);
    free(zlist);
    return E;
}

/* ------------------------------------------------------------------ */
/* Exact (non-random-batch) k-sum, Force_long.jl:220-233 with its two    */
/* typos fixed: the lattice bound trunc(k_c L / (2 pi)) (written         */
/* k_cutoff * L_x / 2 * pi at 221-222) and k = sqrt(k_x^2 + k_y^2)        */
/* (written sqrt(k_x^2 + k_y) at 227).  The k = 0 lattice point, which    */
/* the loop would pass to F_l_total (k_x / k = 0 / 0), is left out: the   */
/* k = 0 term is Flz_sort_k0.  Every k carries the weight e^{-k^2/4a}     */
/* (232), as in the python exact path (Force_long_range_njit_exact.py:    */
/* 19-34, whose KCAR shells cut at k <= k_f1).                            */
/* ------------------------------------------------------------------ */
/* rows in the Julia loop order (n_x outer, n_y inner); returns the count
 * (rows written up to cap; k3 / w may be NULL to count only) */
long qo_exact_kset(double Lx, double Ly, double alpha, double k_cutoff, double *k3, double *w, long cap)
{
    const long nx = (long)(k_cutoff * Lx / (2 * QO_PI)), ny = (long)(k_cutoff * Ly / (2 * QO_PI));
    long n = 0;
    for (long a = -nx; a <= nx; a++)
        for (long b = -ny; b <= ny; b++) {
            if (a == 0 && b == 0) continue;
            const double kx = 2 * QO_PI * a / Lx, ky = 2 * QO_PI * b / Ly;
            const double k = sqrt(kx * kx + ky * ky);
            if (!(k < k_cutoff)) continue;
            if (n < cap) {
                if (k3) {
                    k3[3 * n] = kx;
                    k3[3 * n + 1] = ky;
                    k3[3 * n + 2] = k;
                }
                if (w) w[n] = exp(-k * k / (4 * alpha));
            }
            n++;
        }
    return n;
}

/* F_long with a per-k weight w[m] in place of sum_K / P (Force_long.jl:232) */
void qo_F_long_w(const qo_params *p, int N, const double *xyz, const double *q, const int *zlist_in, int P,
                 const double *kset, const double *w, double *F, int nthreads)
{
    int *zlist = malloc(sizeof(int) * (N > 0 ? N : 1));
    if (zlist_in) memcpy(zlist, zlist_in, sizeof(int) * N);
    else qo_sortperm_z(N, xyz, zlist);
    double *t = malloc(sizeof(double) * 3 * (size_t)(N > 0 ? N : 1));
    if (p->z_ties) qo_Flz_sort_k0_ties(N, zlist, xyz, q, t);
    else qo_Flz_sort_k0(N, zlist, q, t);
    double den0 = 2 * p->Lx * p->Ly * p->eps_0;
    for (int i = 0; i < 3 * N; i++) F[i] = 0 + t[i] / den0;
    for (int m = 0; m < P; m++) {
        qo_F_l_total(p, kset + 3 * m, N, xyz, q, zlist, t, nthreads);
        for (int i = 0; i < 3 * N; i++) F[i] += t[i] * w[m];
    }
    free(t);
    free(zlist);
}

/* energy_long with a per-k weight w[m] in place of sum_K / P */
double qo_energy_long_w(const qo_params *p, int N, const double *xyz, const double *q, const int *zlist_in, int P,
                        const double *kset, const double *w)
{
    int *zlist = malloc(sizeof(int) * (N > 0 ? N : 1));
    if (zlist_in) memcpy(zlist, zlist_in, sizeof(int) * N);
    else qo_sortperm_z(N, xyz, zlist);
    double Es = 0, Ens = 0;
    for (int m = 0; m < P; m++) {
        Es += -w[m] * qo_sigma_s(kset + 3 * m, N, xyz, q, p->gamma_1, p->gamma_2, p->Lz) /
              (2 * p->eps_0 * p->Lx * p->Ly);
        Ens += -w[m] * qo_sigma_ns(kset + 3 * m, N, xyz, q, zlist) / (2 * p->eps_0 * p->Lx * p->Ly);
    }
    double E = Es + Ens + qo_energy_k0(p, N, xyz, q, zlist);
    free(zlist);
    return E;
}

/* ------------------------------------------------------------------ */
/* Bounded-sample drivers for the timed CPU baseline (bench.py).        */
/* ------------------------------------------------------------------ */
/* F_short_ij for npairs pairs (4 doubles per pair, see qo_F_short_ij). */
void qo_pairs_eval(const qo_params *p, const double *xyz, const double *q, long npairs, const int *pairs,
                   double *out, int nthreads)
{
    (void)nthreads;
#ifdef _OPENMP
    if (nthreads < 1) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads)
#endif
    for (long t = 0; t < npairs; t++) {
        int i = pairs[2 * t], j = pairs[2 * t + 1];
        qo_F_short_ij(p, q[i], q[j], xyz + 3 * i, xyz + 3 * j, 0, out + 4 * t);
    }
}

/* F_short_i for the first n particles. */
void qo_self_eval(const qo_params *p, int n, const double *xyz, const double *q, double *out, int nthreads)
{
    (void)nthreads;
#ifdef _OPENMP
    if (nthreads < 1) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads)
#endif
    for (int i = 0; i < n; i++) out[i] = qo_F_short_i(p, q[i], xyz + 3 * i, 0);
}

int qo_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

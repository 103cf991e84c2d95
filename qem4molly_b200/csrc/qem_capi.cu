// qem_capi.cu -- the C-ABI of libqem.so (include/qem.h): handle, parameter
// validation, device scratch, k-set sampling and the per-call orchestration of
// the binning, short-range and long-range kernels.
#include <algorithm>
#include <functional>
#include <cstddef>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "qem_internal.cuh"

namespace {

struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
};

// set while enqueuing asynchronous (capturable) work: a buffer that would
// have to grow is an error there, as cudaMalloc / cudaFree cannot be captured
thread_local bool g_no_alloc = false;
// counts device (re)allocations of handle buffers: a recorded evaluation graph
// holds buffer addresses and is replayed only while this is unchanged
std::atomic<uint64_t> g_alloc_epoch{0};

cudaError_t grow(DevBuf &b, size_t bytes)
{
    if (bytes <= b.cap && b.p) return cudaSuccess;
    if (g_no_alloc) return cudaErrorMemoryAllocation;
    g_alloc_epoch++;
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.cap = 0;
    size_t nb = std::max<size_t>(bytes + bytes / 4, 256);
    cudaError_t e = cudaMalloc(&b.p, nb);
    if (e == cudaSuccess) b.cap = nb;
    return e;
}

template <typename T>
T *ptr(DevBuf &b) { return (T *)b.p; }

// Gauss-Legendre nodes on [-1, 1] (ascending) by Newton iteration on P_n
void gauss_legendre(int n, double *x, double *w)
{
    for (int i = 0; i < (n + 1) / 2; i++) {
        double z = cos(QEM_PI * (i + 0.75) / (n + 0.5)), dp = 1.0;
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
}

struct Prof {
    bool on = false;
    std::vector<cudaEvent_t> pool;
    int used = 0;
    std::vector<std::string> names;
    std::vector<std::pair<int, int>> spans;
    std::vector<double> ms;
    void begin() { used = 0; names.clear(); spans.clear(); }
    int mark(cudaStream_t s)
    {
        if (!on) return -1;
        if (used == (int)pool.size()) {
            cudaEvent_t e;
            if (cudaEventCreate(&e) != cudaSuccess) return -1;
            pool.push_back(e);
        }
        cudaEventRecord(pool[used], s);
        return used++;
    }
    void span(const char *n, int a, int b)
    {
        if (a >= 0 && b >= 0) { names.push_back(n); spans.push_back({a, b}); }
    }
    void finish()
    {
        ms.assign(spans.size(), 0.0);
        for (size_t i = 0; i < spans.size(); i++) {
            float t = 0;
            cudaEventElapsedTime(&t, pool[spans[i].first], pool[spans[i].second]);
            ms[i] = t;
        }
    }
};

}  // namespace

struct qem_handle {
    qem_params p;
    std::string err;
    // k-set (host master copy)
    std::vector<double> kset;
    std::vector<double> kwt;  // per-k weights of a weighted (exact) k-set; empty: sum_K / P for every k
    std::vector<double> norm_host;  // node sets of the regularised quadrature (gamma_1 gamma_2 > 1)
    double sum_K = 0;
    int P = 0;
    bool has_kset = false, kset_dirty = true;
    int kin_lo = 0, kin_hi = -1;  // rows of the k-set currently in the device copy
    // sharding of one system over ranks (qem_set_shard)
    int shard_rank = 0, shard_world = 1;
    uint64_t cfg_version = 0;  // bumped by k-set and shard changes
    int long_max_ks = QEM_LONG_MAX_KS;  // cap on the k-slices of the long-range force pass
    // random-batch sampler (KSampler): seed of the batches, host copy of its
    // cumulative tables, their device copy and the device batch counter (the
    // number of long-range evaluations since the last qem_sample_kset)
    uint64_t kseed = 0x51ed5eedULL;
    std::vector<double> ktab_host;
    KSampler ksamp{};
    double sampler_sumK = 0;
    double kmax_lattice = 0;  // bound on the |k| the sampler can draw
    DevBuf ktab, kctr;
    bool ktab_on_dev = false;
    bool kctr_reset = true;   // the device counter must be set to 0 before the next draw
    double kmax = 0;
    // geometry / constants
    CellGeom geom;
    int ncell = 0;
    ShortConsts sc;
    // device scratch
    DevBuf xyz, q, F, pos, cell, cell_cnt, cell_start, cell_fill, cell_list, pos_of, pcount, poff, pairs, R, Upair,
        in_cnt, in_off, in_fill, in_list, scan_tmp;
    DevBuf zperm, ztmp, zkey, zkey2, zx, zy, zhd, qd, k0, qscan, kc, kin, kw, tot, off, Utot, kf, Epart,
        status, Eout, Fpart, pos_c;
    int64_t pair_cap = 0;       // capacity of pairs / R / in_list (grown on overflow)
    DevBuf scan_tmp2, Flong;    // long-range scan scratch and forces (side stream)
    DevBuf zP32;                // z-ordered FP32 records of the lane-per-k passes
    DevBuf hmask;               // pair-list hit masks (count pass -> fill pass)
    bool kset_lattice = true;   // every row of the current k-set is 2 pi (m / Lx, n / Ly)
    // adjoint pass
    DevBuf gF, gxyz, gq, RA, gam, gout, zgx, zgy, zgz, w1, w2, ws1, ws2, atot, aoff, lam, ggk, Gpart, gFh, normxw;
    cudaStream_t s2 = nullptr;  // side stream of the long range
    cudaStream_t s3 = nullptr;  // per-k constants (and the batch draw) beside the z order
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_kfork = nullptr, ev_kdone = nullptr;
    unsigned *h_status = nullptr;
    double *h_E = nullptr;
    int64_t *h_np = nullptr;
    // neighbour-list state (QEM_short.jl:32-36)
    int64_t Np = 0;
    int pairs_N = -1;
    bool pairs_valid = false;
    int64_t short_calls = 0;
    Prof prof;
    int64_t counts[4] = {0, 0, 0, 0};
    // replay of a recorded device-memory evaluation (run())
    struct GraphKey {
        int N = -1, mem = -1;
        const void *xyz = nullptr, *q = nullptr, *F = nullptr;
        uint32_t terms = 0;
        int64_t cap = 0;
        int P = 0;
        uint64_t cfg = 0, epoch = 0;
        bool operator==(const GraphKey &o) const
        {
            return N == o.N && mem == o.mem && xyz == o.xyz && q == o.q && F == o.F && terms == o.terms &&
                   cap == o.cap && P == o.P && cfg == o.cfg && epoch == o.epoch;
        }
    };
    GraphKey gkey, gwarm;
    bool gwarm_valid = false;
    int64_t enq_launches = 0;  // kernels enqueued by the last asynchronous (recorded) evaluation
    int64_t glaunches = 0;     // kernels in the recorded evaluation graph
    cudaStream_t gcap = nullptr;
    cudaGraphExec_t gexec = nullptr;
};

static const char *status_str(qem_status s)
{
    switch (s) {
    case QEM_OK: return "ok";
    case QEM_ERR_ARG: return "invalid argument";
    case QEM_ERR_OUT_OF_SLAB: return "particle run out of the box (Substrate_LJ wall)";
    case QEM_ERR_NONFINITE: return "non-finite coordinate or charge";
    case QEM_ERR_NB_OVERFLOW: return "neighbour capacity exceeded";
    case QEM_ERR_TIMEOUT: return "device wait timed out";
    case QEM_ERR_CUDA: return "CUDA error";
    case QEM_ERR_NO_KSET: return "no k-set";
    case QEM_ERR_RANGE: return "exponent range of the FP32 k-space path exceeded";
    }
    return "unknown status";
}

// the FP32 k-space path's device check (k_zgather): e^{+-k (z - Lz/2)} would
// leave FP32 range for a particle far outside the slab
static const char *range_msg = "FP32 k-space path: max(k) * |z - L_z / 2| > 60 for some particle (use QEM_FP64)";

static qem_status fail(qem_handle *h, qem_status s, const std::string &msg)
{
    if (h) h->err = std::string(status_str(s)) + ": " + msg;
    return s;
}

#define CU(call)                                                                                     \
    do {                                                                                             \
        cudaError_t e_ = (call);                                                                     \
        if (e_ != cudaSuccess)                                                                       \
            return fail(h, QEM_ERR_CUDA, std::string(#call) + " -> " + cudaGetErrorString(e_));      \
    } while (0)

static bool finite_pos(double v) { return std::isfinite(v) && v > 0; }

static qem_status validate(const qem_params *p, std::string &why)
{
    if (!p) { why = "params is NULL"; return QEM_ERR_ARG; }
    if (!finite_pos(p->Lx) || !finite_pos(p->Ly) || !finite_pos(p->Lz)) { why = "box lengths must be > 0"; return QEM_ERR_ARG; }
    if (!finite_pos(p->alpha)) { why = "alpha must be > 0"; return QEM_ERR_ARG; }
    if (!finite_pos(p->r_cutoff) || !(p->r_cutoff < 0.5 * std::min(p->Lx, p->Ly))) {
        why = "r_cutoff must be in (0, min(Lx, Ly) / 2)";
        return QEM_ERR_ARG;
    }
    if (!(p->accuracy > 0 && p->accuracy < 1)) { why = "accuracy must be in (0, 1)"; return QEM_ERR_ARG; }
    if (!finite_pos(p->eps_0)) { why = "eps_0 must be > 0"; return QEM_ERR_ARG; }
    if (p->N_t < 1 || p->N_t > QEM_MAX_NT) { why = "N_t must be in 1..64"; return QEM_ERR_ARG; }
    if (p->rbe_p < 0 || p->rbe_p > QEM_MAX_KSET) { why = "rbe_p must be in 0 .. QEM_MAX_KSET"; return QEM_ERR_ARG; }
    if (p->iter_period < 1) { why = "iter_period must be >= 1"; return QEM_ERR_ARG; }
    if (!std::isfinite(p->gamma_up) || !std::isfinite(p->gamma_down) || !(p->gamma_up * p->gamma_down > -1.0) ||
        p->gamma_up * p->gamma_down == 1.0) {
        why = "gamma_up * gamma_down must be in (-1, 1) or > 1";
        return QEM_ERR_ARG;
    }
    if (p->gamma_up * p->gamma_down > 1.0) {  // the regularised quadrature (python_lib)
        const double g12 = p->gamma_up * p->gamma_down, k0 = log(g12) / (2.0 * p->Lz);
        if (p->precision != QEM_FP64 || !(p->mode_flags & QEM_CUTOFF_PYTHON)) {
            why = "gamma_up * gamma_down > 1 needs QEM_FP64 and QEM_CUTOFF_PYTHON (python_lib regularised quadrature)";
            return QEM_ERR_ARG;
        }
        if (!(p->pv_eps > 0 && p->pv_eps < k0)) { why = "pv_eps must be in (0, k_0)"; return QEM_ERR_ARG; }
        const double kf[2] = {std::max(sqrt(-4.0 * p->alpha * log(p->accuracy)), 2.1 * k0),
                              std::max(-log(p->accuracy) / (2.0 * p->Lz), 2.1 * k0)};
        for (double f : kf) {
            const int n1 = (int)(p->N_t * k0 / f);
            if (n1 < 1 || p->N_t - 2 * n1 < 1) {
                why = "gamma_up * gamma_down > 1: N_t k_0 / k_f gives an empty sub-interval (raise N_t)";
                return QEM_ERR_ARG;
            }
        }
    }
    if (p->n_walls < 0 || p->n_walls > 2) { why = "n_walls must be 0..2"; return QEM_ERR_ARG; }
    for (int w = 0; w < p->n_walls; w++) {
        const qem_lj_wall &W = p->walls[w];
        if (!(W.direction == 1.0 || W.direction == -1.0) || !std::isfinite(W.cutoff) || !std::isfinite(W.sigma) ||
            !std::isfinite(W.eps) || !std::isfinite(W.sub_pos)) {
            why = "wall parameters must be finite and direction +-1";
            return QEM_ERR_ARG;
        }
    }
    const uint32_t known = QEM_CUTOFF_PYTHON | QEM_DIR_MINIMAGE | QEM_PAIR_PHYSICAL | QEM_STALE_NEIGHBORS |
                           QEM_RESAMPLE_KSET | QEM_EQUAL_Z_TIES;
    if (p->mode_flags & ~known) { why = "unknown mode flag"; return QEM_ERR_ARG; }
    if (p->precision != QEM_FP64 && p->precision != QEM_FP32_FIX) { why = "precision must be QEM_FP64 or QEM_FP32_FIX"; return QEM_ERR_ARG; }
    if (p->reserved0 != 0) { why = "reserved fields must be zero"; return QEM_ERR_ARG; }
    for (int i = 0; i < 2; i++)
        if (p->reserved[i] != 0) { why = "reserved fields must be zero"; return QEM_ERR_ARG; }
    return QEM_OK;
}

// separable k sampler of the box and alpha of p: w(m) = exp(-(2 pi m / L)^2 /
// (4 alpha)), |m| <= ceil(k_c L / 2 pi) + 1 (K_set_generator.jl:7-9);
// cumulative tables over all m and over m != 0 per axis (KSampler), sum_K
// (K_set_generator.jl:28) and the largest |k| of the lattice
static void make_sampler(const qem_params &p, KSampler &S, std::vector<double> &tab, double &sumK, double &kmax)
{
    const double k_c = 2.0 * sqrt(-4.0 * p.alpha * log(p.accuracy));  // K_set_generator.jl:7
    const int Mx = (int)ceil(k_c * p.Lx / (2.0 * QEM_PI)) + 1, My = (int)ceil(k_c * p.Ly / (2.0 * QEM_PI)) + 1;
    S = KSampler{};
    S.Mx = Mx;
    S.My = My;
    S.Lx = p.Lx;
    S.Ly = p.Ly;
    tab.clear();
    tab.reserve(4 * (size_t)(Mx + My) + 2);
    auto cdf = [&](int M, double L, bool skip0, double &sum) {
        double c = 0;
        for (int m = -M; m <= M; m++) {
            if (skip0 && m == 0) continue;
            const double k = 2.0 * QEM_PI * m / L;
            c += exp(-k * k / (4.0 * p.alpha));
            tab.push_back(c);
        }
        sum = c;
    };
    cdf(Mx, p.Lx, false, S.Tx);
    cdf(Mx, p.Lx, true, S.Sx);
    cdf(My, p.Ly, false, S.Ty);
    cdf(My, p.Ly, true, S.Sy);
    S.tab = tab.data();
    sumK = S.Sx + S.Sy + S.Sx * S.Sy;
    // drawable: Float32(exp(-k^2 / 4 alpha) / sum_K) > 0, i.e. the probability
    // above 2^-150 (K_set_generator.jl:43 keeps the probabilities as Float32)
    S.k2max = 4.0 * p.alpha * (150.0 * log(2.0) - log(sumK));
    const double kxm = 2.0 * QEM_PI * Mx / p.Lx, kym = 2.0 * QEM_PI * My / p.Ly;
    kmax = sqrt(std::min(S.k2max, kxm * kxm + kym * kym));
}

static void build_consts(qem_handle *h)
{
    const qem_params &p = h->p;
    ShortConsts &c = h->sc;
    memset(&c, 0, sizeof(c));
    c.shard_rank = h->shard_rank;
    c.shard_world = h->shard_world;
    c.Lx = p.Lx; c.Ly = p.Ly; c.invLx = 1.0 / p.Lx; c.invLy = 1.0 / p.Ly;
    c.Lz = p.Lz; c.twoLz = 2.0 * p.Lz;
    c.alpha = p.alpha; c.inv4alpha = 1.0 / (4.0 * p.alpha);
    c.rc2 = p.r_cutoff * p.r_cutoff;
    c.g1 = p.gamma_down; c.g2 = p.gamma_up; c.g12 = p.gamma_down * p.gamma_up;
    c.one_minus_g12 = 1.0 - c.g12;
    c.neg_lnacc = -log(p.accuracy);
    c.pref = 1.0 / (2.0 * QEM_PI * p.eps_0);
    c.kf_gauss_py = sqrt(-4.0 * p.alpha * log(p.accuracy));
    c.kf_point_py = -log(p.accuracy) / (2.0 * p.Lz);
    c.Nt = p.N_t;
    c.flags = p.mode_flags;
    c.n_walls = p.n_walls;
    for (int w = 0; w < p.n_walls; w++) {
        c.wall_cut[w] = p.walls[w].cutoff;
        c.wall_sig2[w] = p.walls[w].sigma * p.walls[w].sigma;
        c.wall_eps[w] = p.walls[w].eps;
        c.wall_pos[w] = p.walls[w].sub_pos;
        c.wall_dir[w] = p.walls[w].direction;
    }
    double x[QEM_MAX_NT], w[QEM_MAX_NT];
    gauss_legendre(p.N_t, x, w);
    for (int i = 0; i < p.N_t; i++) {
        c.xd[i] = x[i]; c.wd[i] = w[i];
    }
    if (c.g12 > 1.0) {  // regularised quadrature: node sets of the 4 sub-intervals per family
        c.norm = 1;
        c.k0 = log(c.g12) / (2.0 * p.Lz);
        c.pv_eps = p.pv_eps;
        c.kf_norm[0] = std::max(c.kf_gauss_py, 2.1 * c.k0);
        c.kf_norm[1] = std::max(c.kf_point_py, 2.1 * c.k0);
        h->norm_host.clear();
        for (int f = 0; f < 2; f++) {
            const int n1 = (int)(p.N_t * c.k0 / c.kf_norm[f]);
            const int n[4] = {n1, 10, n1, p.N_t - 2 * n1};
            for (int t = 0; t < 4; t++) {
                double xs[QEM_MAX_NT + 16], ws[QEM_MAX_NT + 16];
                gauss_legendre(n[t], xs, ws);
                c.norm_n[f][t] = n[t];
                c.norm_off[f][t] = (int)h->norm_host.size();
                h->norm_host.insert(h->norm_host.end(), xs, xs + n[t]);
                h->norm_host.insert(h->norm_host.end(), ws, ws + n[t]);
            }
        }
    }
    c.f_nlog2e_2Lz = (float)(-1.4426950408889634 * c.twoLz);
    c.f_nlog2e_c2 = (float)(-1.4426950408889634 * c.inv4alpha);
    c.f_2Lz = (float)c.twoLz;
    c.f_g12 = (float)c.g12;
    c.f_omg12 = (float)c.one_minus_g12;
    c.bins_per_rc2 = QEM_RHO_BINS / c.rc2;
    c.Nt2 = (p.N_t + 1) / 2;
    for (int m = 0; m < c.Nt2; m++) {
        // node pair (2m, 2m + 1); an odd N_t ends with a node at t = 0 of weight 0
        double t[2], wn[2];
        for (int j = 0; j < 2; j++) {
            const int n = 2 * m + j;
            t[j] = n < p.N_t ? 1.0 + x[n] : 0.0;
            wn[j] = n < p.N_t ? w[n] : 0.0;
        }
        c.tf2[m] = make_float2((float)t[0], (float)t[1]);
        c.wf2[m] = make_float2((float)wn[0], (float)wn[1]);
        c.wtf2[m] = make_float2((float)(wn[0] * t[0]), (float)(wn[1] * t[1]));
        c.rtf2[m] = make_float2(t[0] > 0 ? (float)(1.0 / sqrt(t[0])) : 0.0f, t[1] > 0 ? (float)(1.0 / sqrt(t[1])) : 0.0f);
    }
    // in-plane cells of side >= r_cutoff
    CellGeom &g = h->geom;
    int ncx = std::max(1, (int)floor(p.Lx / p.r_cutoff)), ncy = std::max(1, (int)floor(p.Ly / p.r_cutoff));
    while ((int64_t)ncx * ncy > (1 << 24)) {
        ncx = std::max(1, ncx / 2);
        ncy = std::max(1, ncy / 2);
    }
    g.Lx = p.Lx; g.Ly = p.Ly; g.invLx = 1.0 / p.Lx; g.invLy = 1.0 / p.Ly;
    g.ncx = ncx; g.ncy = ncy;
    g.inv_lcx = ncx / p.Lx; g.inv_lcy = ncy / p.Ly;
    h->ncell = ncx * ncy;
    make_sampler(p, h->ksamp, h->ktab_host, h->sampler_sumK, h->kmax_lattice);
}

static bool resampling(const qem_handle *h) { return (h->p.mode_flags & QEM_RESAMPLE_KSET) != 0; }

// rows [0, P) of batch n of the handle's sampler (host copy of the draw the
// per-k constants kernel makes on the device: the same bits)
static void batch_rows(const qem_handle *h, uint64_t n, int P, std::vector<double> &k3)
{
    KSampler S = h->ksamp;
    S.tab = h->ktab_host.data();
    S.seed = h->kseed;
    k3.resize(3 * (size_t)P);
    for (int i = 0; i < P; i++) ksample_row(S, n, i, k3[3 * i], k3[3 * i + 1], k3[3 * i + 2]);
}

// batch 0 of the sampler with the handle's seed becomes the current k-set;
// with QEM_RESAMPLE_KSET the device counter restarts at 0, so the next
// long-range call draws this same batch on the device, and call n batch n
static void sample_kset(qem_handle *h, int P)
{
    batch_rows(h, 0, P, h->kset);
    h->kset_lattice = true;
    h->kwt.clear();
    double kmax = 0;
    for (int i = 0; i < P; i++) kmax = std::max(kmax, h->kset[3 * i + 2]);
    h->P = P;
    h->sum_K = h->sampler_sumK;
    h->kmax = resampling(h) ? h->kmax_lattice : kmax;
    h->has_kset = true;
    h->kset_dirty = true;
    h->kctr_reset = true;
    h->cfg_version++;
}

// device batch counter (number of long-range calls since qem_sample_kset);
// the caller has no work in flight on the handle (calls synchronise)
static bool read_batch_counter(const qem_handle *h, uint64_t *n)
{
    *n = 0;
    if (!h->kctr.p || h->kctr_reset) return true;
    unsigned long long v = 0;
    if (cudaSetDevice(h->p.device) != cudaSuccess ||
        cudaMemcpy(&v, h->kctr.p, sizeof(v), cudaMemcpyDeviceToHost) != cudaSuccess)
        return false;
    *n = v;
    return true;
}

// device buffers of the long range for N particles, Pk k-vectors, nch chunks
// and ks k-slices; Ep: energy partials (long-range part at Ep + nbS)
static qem_status long_buffers(qem_handle *h, int N, int Pk, int nch, int ks, double *Ep, int nbS, int nb0,
                               LongBuffers &b)
{
    CU(grow(h->kin, sizeof(double) * 3 * std::max(Pk, 1)));
    CU(grow(h->kw, sizeof(double) * std::max(Pk, 1)));
    CU(grow(h->zperm, sizeof(int) * N));
    CU(grow(h->ztmp, sizeof(int) * (N + 1)));  // + the z-bucket flag word at ztmp[N]
    CU(grow(h->zkey, sizeof(double) * N));
    CU(grow(h->zkey2, sizeof(double) * N));
    CU(grow(h->zx, sizeof(double) * N));
    CU(grow(h->zy, sizeof(double) * N));
    CU(grow(h->zhd, sizeof(double) * N));
    CU(grow(h->qd, sizeof(double) * N));
    CU(grow(h->k0, sizeof(double) * N));
    CU(grow(h->qscan, sizeof(double) * (N + 1)));
    CU(grow(h->kc, sizeof(KConst) * std::max(Pk, 1)));
    CU(grow(h->tot, sizeof(double) * 4 * (size_t)std::max(Pk, 1) * nch));
    CU(grow(h->off, sizeof(double) * 4 * (size_t)std::max(Pk, 1) * nch));
    CU(grow(h->Fpart, sizeof(double) * 3 * (size_t)ks * N));
    CU(grow(h->Utot, sizeof(double) * 4 * std::max(Pk, 1)));
    CU(grow(h->kf, sizeof(KForce<double>) * std::max(Pk, 1)));
    CU(grow(h->scan_tmp2, qem_scan_tmp_bytes(std::max(N, 1)) + 64));
    CU(grow(h->Flong, sizeof(double) * 3 * N));
    if (h->p.precision == QEM_FP32_FIX) {
        CU(grow(h->zP32, sizeof(uint4) * N));
        b.zP = ptr<uint4>(h->zP32);
    }
    b.zx = ptr<double>(h->zx); b.zy = ptr<double>(h->zy);
    b.zhd = ptr<double>(h->zhd);
    b.qd = ptr<double>(h->qd);
    b.k0 = ptr<double>(h->k0); b.qscan = ptr<double>(h->qscan);
    b.kc = ptr<KConst>(h->kc); b.kin = ptr<double>(h->kin);
    b.kwt = h->kwt.empty() ? nullptr : ptr<double>(h->kw);
    b.tot = ptr<double>(h->tot); b.off = ptr<double>(h->off); b.Utot = ptr<double>(h->Utot);
    b.kf = h->kf.p;
    b.Epart = Ep + nbS;
    b.Eks = Ep + nbS + (size_t)ks * nch + nb0;
    b.Fpart = ptr<double>(h->Fpart);
    b.ks = ks;
    b.stmp = h->scan_tmp2.p; b.stmp_bytes = h->scan_tmp2.cap;
    return QEM_OK;
}

// cells, pair list (owner, other) with its per-particle CSR and the incoming
// lists of every particle (QEM_short.jl:32-36 neighbour build)
static qem_status build_pairs(qem_handle *h, int N, unsigned *st, cudaStream_t s)
{
    CU(grow(h->cell_cnt, sizeof(int) * h->ncell));
    CU(grow(h->cell_start, sizeof(int) * (h->ncell + 1)));
    CU(grow(h->cell_fill, sizeof(int) * h->ncell));
    CU(grow(h->cell_list, sizeof(int) * N));
    CU(grow(h->pos_of, sizeof(int) * N));
    CU(grow(h->pcount, sizeof(int) * N));
    CU(grow(h->poff, sizeof(int64_t) * (N + 1)));
    CU(grow(h->pos_c, sizeof(double4) * N));
    CU(grow(h->hmask, sizeof(unsigned) * QEM_PL_MAXB * (size_t)N));
    // pair capacity: last count + 25 %, first time from the mean density; the
    // count stays on the device (no host round trip inside the call)
    if (h->pair_cap <= 0) {
        const double dens = (double)N / (h->p.Lx * h->p.Ly);
        h->pair_cap = (int64_t)(1.3 * 0.5 * N * QEM_PI * h->p.r_cutoff * h->p.r_cutoff * dens) + 4096;
    }
    const int64_t cap = h->pair_cap;
    CU(grow(h->pairs, sizeof(int2) * cap));
    CU(grow(h->R, sizeof(double4) * cap));
    CU(grow(h->Upair, sizeof(double) * cap));
    CU(grow(h->in_cnt, sizeof(int) * N));
    CU(grow(h->in_fill, sizeof(int) * 5 * (size_t)N));  // per (position, stencil direction) slots
    CU(grow(h->in_off, sizeof(int64_t) * (N + 1)));
    if (cap > INT32_MAX) return fail(h, QEM_ERR_NB_OVERFLOW, "more than 2^31 - 1 pairs");
    CU(grow(h->in_list, sizeof(int) * cap));
    CU(qem_launch_cells(N, h->ncell, ptr<int>(h->cell), ptr<double4>(h->pos), ptr<int>(h->cell_cnt),
                        ptr<int>(h->cell_start), ptr<int>(h->cell_fill), ptr<int>(h->cell_list),
                        ptr<int>(h->pos_of), ptr<double4>(h->pos_c), h->scan_tmp.p, h->scan_tmp.cap, s));
    CU(qem_launch_pair_list(N, h->ncell, ptr<double4>(h->pos_c), ptr<int>(h->cell), ptr<int>(h->cell_start),
                            ptr<int>(h->cell_list), h->geom, h->sc.rc2, ptr<int>(h->pcount), ptr<int64_t>(h->poff),
                            ptr<int2>(h->pairs), cap, ptr<int>(h->in_cnt), ptr<int>(h->in_fill),
                            ptr<int64_t>(h->in_off), ptr<int>(h->in_list), st, h->scan_tmp.p, h->scan_tmp.cap,
                            ptr<unsigned>(h->hmask), s));
    h->pairs_N = N;
    h->pairs_valid = true;
    return QEM_OK;
}

// ---------------------------------------------------------------------------
// one evaluation
// ---------------------------------------------------------------------------
// retry = true asks the caller to evaluate again (the pair list outgrew its
// capacity, which has been enlarged).
//
// async = true enqueues the evaluation only (device memory, no energy): no
// host synchronisation, no allocation, no k-set sampling or upload and a
// pair-list rebuild on every call, so that the work can be captured into a
// CUDA graph; the device status word then accumulates over calls and is
// checked (and cleared) by qem_batch_check.  A synchronous call of the same
// size must have run first.
static qem_status run_once(qem_handle *h, int N, const double *xyz, const double *q, double *F, double *energy,
                           uint32_t terms, int mem, cudaStream_t s, bool &retry, bool async = false)
{
    retry = false;
    if (!h) return QEM_ERR_ARG;
    const int64_t short_calls0 = h->short_calls;
    if (N < 0) return fail(h, QEM_ERR_ARG, "N < 0");
    if (terms & ~QEM_TERM_ALL) return fail(h, QEM_ERR_ARG, "unknown term bit");
    if (mem != QEM_MEM_HOST && mem != QEM_MEM_DEVICE) return fail(h, QEM_ERR_ARG, "mem must be HOST or DEVICE");
    const bool do_short = terms & QEM_TERM_SHORT;
    const bool do_long = terms & QEM_TERM_LONG;
    const bool do_lj = (terms & QEM_TERM_LJ) && h->p.n_walls > 0;
    const bool want_E = energy != nullptr;
    if (N == 0) {
        if (energy) *energy = 0;
        return QEM_OK;
    }
    if (!xyz || !q || !F) return fail(h, QEM_ERR_ARG, "NULL coordinate, charge or force pointer");
    if (async && (mem != QEM_MEM_DEVICE || energy)) return fail(h, QEM_ERR_ARG, "async evaluation: device memory, no energy");
    if (want_E && h->sc.norm && (do_short || do_lj))
        return fail(h, QEM_ERR_ARG, "no short-range energy is defined for gamma_up * gamma_down > 1");
    CU(cudaSetDevice(h->p.device));
    const int prec = h->p.precision;
    const bool prof_on = h->prof.on;
    if (async) h->prof.on = false;
    struct Restore {
        qem_handle *h;
        bool prof;
        bool async;
        ~Restore()
        {
            h->prof.on = prof;
            if (async) g_no_alloc = false;
        }
    } restore{h, prof_on, async};
    if (async) g_no_alloc = true;
    h->prof.begin();
    int launches = 0;
    const int mk0 = h->prof.mark(s);

    CU(grow(h->pos, sizeof(double4) * N));
    CU(grow(h->cell, sizeof(int) * N));
    CU(grow(h->status, 64));
    CU(grow(h->Eout, 64));
    const double *xyz_d = xyz, *q_d = q;
    double *F_d = F;
    if (mem == QEM_MEM_HOST) {
        CU(grow(h->xyz, sizeof(double) * 3 * N));
        CU(grow(h->q, sizeof(double) * N));
        CU(grow(h->F, sizeof(double) * 3 * N));
        CU(cudaMemcpyAsync(h->xyz.p, xyz, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, s));
        CU(cudaMemcpyAsync(h->q.p, q, sizeof(double) * N, cudaMemcpyHostToDevice, s));
        xyz_d = ptr<double>(h->xyz);
        q_d = ptr<double>(h->q);
        F_d = ptr<double>(h->F);
    }
    unsigned *st = ptr<unsigned>(h->status);
    if (!async) CU(cudaMemsetAsync(st, 0, sizeof(unsigned), s));
    const int mk_in = h->prof.mark(s);
    CU(qem_launch_pack(N, xyz_d, q_d, ptr<double4>(h->pos), ptr<int>(h->cell), h->geom, st, s));
    launches++;

    // energy partials: [short blocks | ks x long chunks | k0 blocks | P split terms]
    const int LCH = qem_long_chunk();
    const int nbS = (N + 255) / 256, nch = (N + LCH - 1) / LCH, nb0 = (N + 255) / 256;
    const int P = do_long ? (h->has_kset ? h->P : 0) : 0;
    // k-slices of the force pass, from the size of the whole k-set (or of the
    // batch about to be drawn); small systems with many k-vectors get up to
    // QEM_LONG_MAX_KS slices so that the pass still fills the GPU
    const int ks = qem_long_ksplit(nch, std::max(h->has_kset ? h->P : h->p.rbe_p, 1), h->long_max_ks, prec);
    const size_t nEpart = (size_t)nbS + (size_t)ks * nch + nb0 + std::max(P, h->p.rbe_p) + 8;
    CU(grow(h->Epart, sizeof(double) * nEpart));
    double *Ep = ptr<double>(h->Epart);
    if (want_E) CU(cudaMemsetAsync(Ep, 0, sizeof(double) * nEpart, s));
    CU(grow(h->scan_tmp, qem_scan_tmp_bytes(std::max(std::max(N, h->ncell), 1)) + 64));

    // Long range first, on the side stream when short-range / wall work runs
    // too: the two pipelines are independent until their forces are summed.
    const bool concurrent = do_long && (do_short || do_lj);
    cudaStream_t sl = concurrent ? h->s2 : s;
    int mk_lstart = -1, mk_lprep = -1, mk_lforce = -1;
    h->counts[2] = 0;
    if (do_long) {
        // QEM_RESAMPLE_KSET: a fresh batch on every call (Force_long.jl:235),
        // drawn on the device from (seed, batch counter) by the per-k constants
        // kernel; the counter lives in device memory, so replayed graphs draw
        // new batches as well
        const bool draw = resampling(h);
        if (async) {
            if ((h->p.rbe_p > 0 && !h->has_kset) || h->kset_dirty || (draw && (!h->ktab_on_dev || h->kctr_reset)))
                return fail(h, QEM_ERR_NO_KSET, "async evaluation: the k-set must be on the device (synchronous call first)");
        } else if (!h->has_kset && h->p.rbe_p > 0) {
            sample_kset(h, h->p.rbe_p);
        }
        if (draw) {  // uniform sum_K / P weights of the sampler
            h->kwt.clear();
            h->sum_K = h->sampler_sumK;
        }
        const int Pall = h->has_kset ? h->P : 0;
        const double kmax = draw ? h->kmax_lattice : h->kmax;
        if (prec == QEM_FP32_FIX && Pall > 0 && !draw && !h->kset_lattice)
            return fail(h, QEM_ERR_ARG, "the FP32 k-space path takes lattice k-vectors 2 pi (m / Lx, n / Ly) only "
                                        "(K_set_generator.jl:19-25); use QEM_FP64 for other rows");
        // this rank's rows of the k-set, weighted as part of all Pall rows
        const int k_lo = (int)((int64_t)Pall * h->shard_rank / h->shard_world);
        const int k_hi = (int)((int64_t)Pall * (h->shard_rank + 1) / h->shard_world);
        const int Pk = k_hi - k_lo;
        const double sumK_eff = Pall > 0 ? h->sum_K * Pk / Pall : 0.0;
        if (async && (h->kin_lo != k_lo || h->kin_hi != k_hi))
            return fail(h, QEM_ERR_NO_KSET, "async evaluation: the k-set rows must be on the device (synchronous call first)");
        LongBuffers b;  // allocated before any launch or copy that uses them
        {
            const qem_status ls = long_buffers(h, N, Pk, nch, ks, Ep, nbS, nb0, b);
            if (ls != QEM_OK) return ls;
        }
        b.skip_k0 = h->shard_rank != 0;
        b.zlim = prec == QEM_FP32_FIX && Pk > 0 ? qem_fp32_zlim(kmax) : 0.0;
        if (draw && Pall > 0) {
            if (!async) {  // sampler tables and batch counter on the device (before the fork)
                CU(grow(h->ktab, sizeof(double) * h->ktab_host.size()));
                CU(grow(h->kctr, sizeof(unsigned long long)));
                if (!h->ktab_on_dev) {
                    CU(cudaMemcpyAsync(h->ktab.p, h->ktab_host.data(), sizeof(double) * h->ktab_host.size(),
                                       cudaMemcpyHostToDevice, s));
                    h->ktab_on_dev = true;
                }
                if (h->kctr_reset) {
                    CU(cudaMemsetAsync(h->kctr.p, 0, sizeof(unsigned long long), s));
                    h->kctr_reset = false;
                }
            }
            b.draw_ctr = ptr<unsigned long long>(h->kctr);
            b.sampler = h->ksamp;
            b.sampler.tab = ptr<double>(h->ktab);
            b.sampler.seed = h->kseed;
            b.sampler.row0 = k_lo;
            b.kwt = nullptr;
        }
        if (concurrent) {  // fork after pack (positions) and the energy-partial clear
            CU(cudaEventRecord(h->ev_fork, s));
            CU(cudaStreamWaitEvent(sl, h->ev_fork, 0));
        }
        mk_lstart = h->prof.mark(sl);
        if (draw) {  // the rows [k_lo, k_hi) of this call's batch are drawn into kin on the device
            h->kset_dirty = false;
            h->kin_lo = k_lo;
            h->kin_hi = k_hi;
        } else if ((h->kset_dirty || h->kin_lo != k_lo || h->kin_hi != k_hi) && Pk > 0) {
            CU(cudaMemcpyAsync(h->kin.p, h->kset.data() + 3 * (size_t)k_lo, sizeof(double) * 3 * Pk,
                               cudaMemcpyHostToDevice, sl));
            if (!h->kwt.empty())
                CU(cudaMemcpyAsync(h->kw.p, h->kwt.data() + k_lo, sizeof(double) * Pk, cudaMemcpyHostToDevice, sl));
            h->kset_dirty = false;
            h->kin_lo = k_lo;
            h->kin_hi = k_hi;
        }
        double *FL = concurrent ? ptr<double>(h->Flong) : F_d;
        CU(cudaMemsetAsync(FL, 0, sizeof(double) * 3 * N, sl));
        if (concurrent && Pk > 0 && !qem_long_prep_is_small(N, want_E)) {
            // the per-k constants (with a per-call batch, its draw) on a third
            // stream while the z order runs; the chunk totals wait for them
            CU(cudaEventRecord(h->ev_kfork, sl));
            CU(cudaStreamWaitEvent(h->s3, h->ev_kfork, 0));
            CU(qem_launch_long(prec, want_E, N, Pk, ptr<double4>(h->pos), ptr<int>(h->zperm), b, h->p.Lx, h->p.Ly,
                               h->p.Lz, h->p.gamma_down, h->p.gamma_up, h->p.eps_0, sumK_eff, FL, nch, st, h->s3, 2));
            CU(cudaEventRecord(h->ev_kdone, h->s3));
            b.kconst_done = h->ev_kdone;
        }
        CU(qem_launch_zsort(N, ptr<double4>(h->pos), ptr<int>(h->zperm), ptr<int>(h->ztmp), ptr<double>(h->zkey),
                            ptr<double>(h->zkey2), sl, false, ptr<int>(h->ztmp) + N, h->p.Lz));
        CU(qem_launch_long(prec, want_E, N, Pk, ptr<double4>(h->pos), ptr<int>(h->zperm), b, h->p.Lx, h->p.Ly,
                           h->p.Lz, h->p.gamma_down, h->p.gamma_up, h->p.eps_0, sumK_eff, FL, nch, st, sl, 0));
        mk_lprep = h->prof.mark(sl);
        CU(qem_launch_long(prec, want_E, N, Pk, ptr<double4>(h->pos), ptr<int>(h->zperm), b, h->p.Lx, h->p.Ly,
                           h->p.Lz, h->p.gamma_down, h->p.gamma_up, h->p.eps_0, sumK_eff, FL, nch, st, sl, 1));
        // z sort, zgather + q scan + k = 0 term, per-k constants + totals + scan, force pass + final
        auto long_launches = [&](bool energy_pass) {
            return qem_zsort_launches(N, true) +
                   (!energy_pass && N <= 8192 ? 1 + (Pk > 0 ? 2 : 0) : 2 + qem_scan_f64_launches(N) + (Pk > 0 ? 3 : 0)) +
                   2;
        };
        launches += long_launches(want_E);
        if (h->p.mode_flags & QEM_EQUAL_Z_TIES) {
            // Equal-z ties: a tied pair counts once as below and once as above
            // in the two orders (z, index up) and (z, index down), and every
            // other part of the long range is the same in both, so the mean of
            // the two evaluations is the force with tied particles neither
            // below nor above each other.  The energy does not depend on the
            // order of ties and comes from the first pass.
            CU(qem_launch_zsort(N, ptr<double4>(h->pos), ptr<int>(h->zperm), ptr<int>(h->ztmp),
                                ptr<double>(h->zkey), ptr<double>(h->zkey2), sl, true, ptr<int>(h->ztmp) + N,
                                h->p.Lz));
            b.draw_ctr = nullptr;  // the second pass reuses the rows the first one drew
            b.kconst_done = nullptr;
            for (int stage = 0; stage < 2; stage++)
                CU(qem_launch_long(prec, false, N, Pk, ptr<double4>(h->pos), ptr<int>(h->zperm), b, h->p.Lx,
                                   h->p.Ly, h->p.Lz, h->p.gamma_down, h->p.gamma_up, h->p.eps_0, sumK_eff, FL, nch,
                                   st, sl, stage));
            CU(qem_launch_scale(3 * N, 0.5, FL, FL, sl));
            launches += long_launches(false) + 1;
        }
        mk_lforce = h->prof.mark(sl);
        h->counts[2] = Pk;
    }

    int mk_bin = -1, mk_pair = -1, mk_gather = -1;
    if (do_short) {
        const bool stale = (h->p.mode_flags & QEM_STALE_NEIGHBORS) != 0;
        const bool rebuild =
            async || !stale || !h->pairs_valid || h->pairs_N != N || (h->short_calls % h->p.iter_period) == 0;
        if (rebuild) {
            const qem_status bs = build_pairs(h, N, st, s);
            if (bs != QEM_OK) return bs;
            // cells: count, scan, scatter, sort; pairs: count, scan, (in_base | fill), scan, fill
            // (+ incoming fill and sort on the thread-per-owner path)
            const bool warp_path = h->geom.ncx >= 3 && h->geom.ncy >= 3 && N >= 2 * (int64_t)h->ncell;
            launches += (qem_cells_small(N, h->ncell) ? 1 : 3 + qem_scan_launches(h->ncell)) +
                        (warp_path ? 3 + 2 * qem_scan_launches(N) : (N <= 8192 ? 1 : 4 + 2 * qem_scan_launches(N)));
        }
        h->short_calls++;
        mk_bin = h->prof.mark(s);
        CU(qem_launch_short_pairs(prec, want_E, ptr<int64_t>(h->poff) + N, h->pair_cap, ptr<int2>(h->pairs),
                                  ptr<double4>(h->pos), ptr<double4>(h->R), ptr<double>(h->Upair), h->sc, s));
        launches++;
        mk_pair = h->prof.mark(s);
    }
    if (do_short || do_lj) {
        if (concurrent) {  // join: the long range ran on the side stream into Flong, which the gather adds
            CU(cudaEventRecord(h->ev_join, h->s2));
            CU(cudaStreamWaitEvent(s, h->ev_join, 0));
        }
        CU(qem_launch_short_gather(prec, want_E, do_short, do_lj, N, ptr<double4>(h->pos), ptr<int>(h->pos_of),
                                   ptr<int64_t>(h->poff), ptr<double4>(h->R), ptr<double>(h->Upair),
                                   ptr<int64_t>(h->in_off), ptr<int>(h->in_list), h->pair_cap, h->sc, F_d, Ep,
                                   st, s, concurrent ? ptr<double>(h->Flong) : nullptr));
        launches++;
    } else if (!do_long) {  // (a long-only call has already zeroed F_d in front of its kernels)
        CU(cudaMemsetAsync(F_d, 0, sizeof(double) * 3 * N, s));
    }
    mk_gather = h->prof.mark(s);
    if (want_E) {
        const int nE = nbS + ks * nch + nb0 + (do_long ? (h->has_kset ? h->P : 0) : 0);
        CU(qem_launch_reduce_sum(Ep, nE, ptr<double>(h->Eout), s));
        launches++;
        CU(cudaMemcpyAsync(h->h_E, h->Eout.p, sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    if (async) {
        h->enq_launches = launches;
        return QEM_OK;
    }
    if (mem == QEM_MEM_HOST) CU(cudaMemcpyAsync(F, F_d, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(h->h_status, st, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    if (do_short)
        CU(cudaMemcpyAsync(h->h_np, ptr<int64_t>(h->poff) + N, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    const int mk_end = h->prof.mark(s);
    CU(cudaStreamSynchronize(s));
    CU(cudaGetLastError());
    if (do_short) {
        h->Np = *h->h_np;
        if (*h->h_status & QEM_ST_OVERFLOW) {  // pair capacity too small: grow and evaluate again
            h->pair_cap = h->Np + h->Np / 4 + 4096;
            h->pairs_valid = false;
            h->short_calls = short_calls0;
            retry = true;
            return QEM_OK;
        }
        if (h->Np > h->pair_cap - h->pair_cap / 8) h->pair_cap = h->Np + h->Np / 4 + 4096;  // for the next build
    }
    h->prof.span("upload", mk0, mk_in);
    h->prof.span("bin_pairs", mk_in, mk_bin);
    h->prof.span("short_pair", mk_bin, mk_pair);
    h->prof.span("short_gather", mk_pair >= 0 ? mk_pair : mk_in, mk_gather);
    h->prof.span("long_prep", mk_lstart, mk_lprep);
    h->prof.span("long_force", mk_lprep, mk_lforce);
    h->prof.span("total", mk0, mk_end);
    if (h->prof.on) h->prof.finish();
    h->counts[0] = do_short ? h->Np : 0;
    h->counts[1] = N;
    h->counts[3] = launches;
    const unsigned stv = *h->h_status;
    if (stv & QEM_ST_NONFINITE) return fail(h, QEM_ERR_NONFINITE, "NaN or Inf in coordinates or charges");
    if (stv & QEM_ST_OUT_OF_SLAB) return fail(h, QEM_ERR_OUT_OF_SLAB, "direction * (z - sub_pos) <= 0 for some particle");
    if (stv & QEM_ST_RANGE) return fail(h, QEM_ERR_RANGE, range_msg);
    if (want_E) *energy = *h->h_E;
    h->err.clear();
    return QEM_OK;
}

// Force calls without energy or profiling whose neighbour list is rebuilt and
// whose k-set is kept every call repeat the same launches on the same
// buffers, so after one ordinary call of a configuration the evaluation is
// recorded once as a CUDA graph on the handle's private stream and then
// replayed on the caller's stream: the host issues one launch instead of some
// forty.  Device buffers qualify, and so do page-locked host buffers, whose
// host-to-device and device-to-host copies are then part of the graph
// (pageable host memory cannot be copied inside a graph).  The key covers
// everything the recorded launches depend on (sizes, pointers, memory kind,
// terms, pair capacity, k-set and shard, and every buffer address through the
// allocation count); the status word and the pair count are read back after
// each replay as in an ordinary call, and a pair-list overflow drops the
// graph and re-runs the call the ordinary way.
static void drop_graph(qem_handle *h)
{
    if (h->gexec) cudaGraphExecDestroy(h->gexec);
    h->gexec = nullptr;
}

// first and last byte of [p, p + bytes) in page-locked host memory
static bool host_locked(const void *p, size_t bytes)
{
    const char *c = static_cast<const char *>(p);
    for (const char *a : {c, c + bytes - 1}) {
        cudaPointerAttributes at;
        if (cudaPointerGetAttributes(&at, a) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        if (at.type != cudaMemoryTypeHost) return false;
    }
    return true;
}

static bool graph_eligible(const qem_handle *h, int N, const double *xyz, const double *q, const double *F,
                           const double *energy, uint32_t terms, int mem)
{
    if (energy || h->prof.on || N <= 0 || !xyz || !q || !F || (terms & ~QEM_TERM_ALL) ||
        (h->p.mode_flags & QEM_STALE_NEIGHBORS))
        return false;
    if (mem == QEM_MEM_DEVICE) return true;
    const size_t n3 = sizeof(double) * 3 * (size_t)N;
    return mem == QEM_MEM_HOST && host_locked(xyz, n3) && host_locked(q, sizeof(double) * N) && host_locked(F, n3);
}

static qem_handle::GraphKey graph_key(const qem_handle *h, int N, const double *xyz, const double *q,
                                      const double *F, uint32_t terms, int mem)
{
    qem_handle::GraphKey k;
    k.N = N; k.mem = mem; k.xyz = xyz; k.q = q; k.F = F; k.terms = terms;
    k.cap = h->pair_cap;
    k.P = h->has_kset ? h->P : 0;
    k.cfg = h->cfg_version;
    k.epoch = g_alloc_epoch.load();
    return k;
}

// replays (recording first if needed); fallback = true asks for an ordinary call
// The long-range chain (z sort, scans, per-k totals, force pass) is a row of
// short, latency-bound kernels on the side stream, while the pair kernel on
// the caller's stream fills every SM with long-running blocks.  At equal
// priority the long chain's blocks queue behind pair blocks and it ends last;
// on a high-priority stream each of its blocks takes the next SM slot that a
// pair block frees, so both chains finish together.  A recorded graph keeps
// those priorities (kernel nodes copy the capturing stream's priority) when it
// is instantiated with cudaGraphInstantiateFlagUseNodePriority.
#ifndef QEM_LONG_PRIORITY
#define QEM_LONG_PRIORITY 1
#endif
static cudaError_t create_side_stream(cudaStream_t *s)
{
    int least = 0, greatest = 0;
    if (QEM_LONG_PRIORITY && cudaDeviceGetStreamPriorityRange(&least, &greatest) == cudaSuccess)
        return cudaStreamCreateWithPriority(s, cudaStreamNonBlocking, greatest);
    cudaGetLastError();
    return cudaStreamCreateWithFlags(s, cudaStreamNonBlocking);
}
static unsigned long long graph_instantiate_flags()
{
    return QEM_LONG_PRIORITY ? (unsigned long long)cudaGraphInstantiateFlagUseNodePriority : 0ull;
}

static qem_status run_graph(qem_handle *h, const qem_handle::GraphKey &k, const double *xyz, const double *q,
                            double *F, uint32_t terms, cudaStream_t s, bool &fallback)
{
    fallback = false;
    const int N = k.N;
    CU(cudaSetDevice(h->p.device));
    if (!h->gexec || !(h->gkey == k)) {
        drop_graph(h);
        if (!h->gcap) CU(cudaStreamCreateWithFlags(&h->gcap, cudaStreamNonBlocking));
        // host buffers: staged through the handle's device copies, which the
        // ordinary call of this configuration has already sized
        const bool host = k.mem == QEM_MEM_HOST;
        const size_t n3 = sizeof(double) * 3 * (size_t)N;
        if (host && (h->xyz.cap < n3 || h->q.cap < sizeof(double) * N || h->F.cap < n3)) {
            h->gwarm_valid = false;
            fallback = true;
            return QEM_OK;
        }
        const double *xd = host ? ptr<double>(h->xyz) : xyz, *qd = host ? ptr<double>(h->q) : q;
        double *Fd = host ? ptr<double>(h->F) : F;
        cudaGraph_t g = nullptr;
        CU(cudaStreamBeginCapture(h->gcap, cudaStreamCaptureModeThreadLocal));
        cudaError_t ce = cudaSuccess;
        if (host) {
            ce = cudaMemcpyAsync(h->xyz.p, xyz, n3, cudaMemcpyHostToDevice, h->gcap);
            if (ce == cudaSuccess) ce = cudaMemcpyAsync(h->q.p, q, sizeof(double) * N, cudaMemcpyHostToDevice, h->gcap);
        }
        bool retry = false;
        qem_status st = QEM_ERR_CUDA;
        if (ce == cudaSuccess) st = run_once(h, N, xd, qd, Fd, nullptr, terms, QEM_MEM_DEVICE, h->gcap, retry, true);
        if (st == QEM_OK && host) ce = cudaMemcpyAsync(F, Fd, n3, cudaMemcpyDeviceToHost, h->gcap);
        const cudaError_t ec = cudaStreamEndCapture(h->gcap, &g);
        cudaGraphExec_t ex = nullptr;
        const bool ok = st == QEM_OK && ce == cudaSuccess && ec == cudaSuccess && g &&
                        cudaGraphInstantiateWithFlags(&ex, g, graph_instantiate_flags()) == cudaSuccess;
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        if (!ok || !(graph_key(h, N, xyz, q, F, terms, k.mem) == k)) {
            if (ex) cudaGraphExecDestroy(ex);
            h->gwarm_valid = false;
            fallback = true;
            return QEM_OK;
        }
        h->gexec = ex;
        h->gkey = k;
        h->glaunches = h->enq_launches;
    }
    const bool do_short = terms & QEM_TERM_SHORT;
    unsigned *st = ptr<unsigned>(h->status);
    CU(cudaMemsetAsync(st, 0, sizeof(unsigned), s));
    CU(cudaGraphLaunch(h->gexec, s));
    CU(cudaMemcpyAsync(h->h_status, st, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    if (do_short)
        CU(cudaMemcpyAsync(h->h_np, ptr<int64_t>(h->poff) + N, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    const unsigned stv = *h->h_status;
    if (do_short) {
        h->Np = *h->h_np;
        if (stv & QEM_ST_OVERFLOW) {  // grow and evaluate the ordinary way
            h->pair_cap = h->Np + h->Np / 4 + 4096;
            h->pairs_valid = false;
            drop_graph(h);
            h->gwarm_valid = false;
            fallback = true;
            return QEM_OK;
        }
        if (h->Np > h->pair_cap - h->pair_cap / 8) {  // grow at the next (ordinary) build
            h->pair_cap = h->Np + h->Np / 4 + 4096;
            h->gwarm_valid = false;
        }
    }
    h->counts[0] = do_short ? h->Np : 0;
    h->counts[1] = N;
    h->counts[3] = h->glaunches;  // the recorded kernels, replayed by one graph launch
    if (stv & QEM_ST_NONFINITE) return fail(h, QEM_ERR_NONFINITE, "NaN or Inf in coordinates or charges");
    if (stv & QEM_ST_OUT_OF_SLAB) return fail(h, QEM_ERR_OUT_OF_SLAB, "direction * (z - sub_pos) <= 0 for some particle");
    if (stv & QEM_ST_RANGE) return fail(h, QEM_ERR_RANGE, range_msg);
    h->err.clear();
    return QEM_OK;
}

static qem_status run(qem_handle *h, int N, const double *xyz, const double *q, double *F, double *energy,
                      uint32_t terms, int mem, cudaStream_t s)
{
    if (!h) return QEM_ERR_ARG;
    const bool eligible = graph_eligible(h, N, xyz, q, F, energy, terms, mem);
    if (eligible && h->gwarm_valid && !h->kset_dirty) {
        const qem_handle::GraphKey k = graph_key(h, N, xyz, q, F, terms, mem);
        if (k == h->gwarm) {
            bool fallback = false;
            const qem_status st = run_graph(h, k, xyz, q, F, terms, s, fallback);
            if (!fallback) return st;
        }
    }
    const int64_t cap0 = h->pair_cap;
    bool retry = false;
    qem_status st = run_once(h, N, xyz, q, F, energy, terms, mem, s, retry);
    if (st == QEM_OK && retry) st = run_once(h, N, xyz, q, F, energy, terms, mem, s, retry);
    if (st == QEM_OK && retry) return fail(h, QEM_ERR_NB_OVERFLOW, "pair list grew past its capacity twice");
    // a configuration is recorded once an ordinary call ran it with buffers
    // that are already large enough for the next call
    h->gwarm_valid = st == QEM_OK && eligible && h->pair_cap == cap0;
    if (h->gwarm_valid) h->gwarm = graph_key(h, N, xyz, q, F, terms, mem);
    return st;
}

// ---------------------------------------------------------------------------
// exported C-ABI
// ---------------------------------------------------------------------------
extern "C" {

static_assert(sizeof(qem_params) == 200 && offsetof(qem_params, pv_eps) == 184, "qem_params layout (ABI)");

void qem_default_params(qem_params *p)
{
    if (!p) return;
    memset(p, 0, sizeof(*p));
    p->Lx = p->Ly = p->Lz = 1.0;
    p->alpha = 1.0;
    p->r_cutoff = 0.25;
    p->eps_0 = 1.0;
    p->accuracy = 1e-6;
    p->N_t = 30;
    p->rbe_p = 30;
    p->iter_period = 100;
    p->precision = QEM_FP64;
}

qem_status qem_inter_params(qem_params *p, int64_t n_atoms, double s, int32_t rbe_mode, int32_t rbe_p)
{
    if (!p || n_atoms <= 0 || !(s > 0) || !(p->Lx > 0) || !(p->Ly > 0)) return QEM_ERR_ARG;
    const double area = p->Lx * p->Ly;
    p->alpha = rbe_mode ? (double)n_atoms / area : sqrt((double)n_atoms) / area;  // Quasi_Ewald_Method.jl:6, 14
    p->r_cutoff = s / sqrt(p->alpha);                                             // Quasi_Ewald_Method.jl:7, 15
    p->rbe_p = rbe_mode ? rbe_p : 0;
    return QEM_OK;
}

qem_status qem_create(const qem_params *p, qem_handle **out)
{
    if (!out) return QEM_ERR_ARG;
    *out = nullptr;
    std::string why;
    qem_status st = validate(p, why);
    if (st != QEM_OK) {
        fprintf(stderr, "qem_create: %s\n", why.c_str());
        return st;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || p->device < 0 || p->device >= ndev) return QEM_ERR_CUDA;
    if (cudaSetDevice(p->device) != cudaSuccess) return QEM_ERR_CUDA;
    qem_handle *h = new qem_handle();
    h->p = *p;
    build_consts(h);
    if (cudaMallocHost(&h->h_status, sizeof(unsigned)) != cudaSuccess ||
        cudaMallocHost(&h->h_E, sizeof(double)) != cudaSuccess ||
        cudaMallocHost(&h->h_np, sizeof(int64_t)) != cudaSuccess ||
        create_side_stream(&h->s2) != cudaSuccess || create_side_stream(&h->s3) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_kfork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_kdone, cudaEventDisableTiming) != cudaSuccess) {
        qem_destroy(h);
        return QEM_ERR_CUDA;
    }
    if (h->sc.norm) {
        const size_t bytes = sizeof(double) * h->norm_host.size();
        if (grow(h->normxw, bytes) != cudaSuccess ||
            cudaMemcpy(h->normxw.p, h->norm_host.data(), bytes, cudaMemcpyHostToDevice) != cudaSuccess) {
            qem_destroy(h);
            return QEM_ERR_CUDA;
        }
        h->sc.norm_xw = ptr<double>(h->normxw);
    }
    *out = h;
    return QEM_OK;
}

void qem_destroy(qem_handle *h)
{
    if (!h) return;
    cudaSetDevice(h->p.device);
    DevBuf *bufs[] = {&h->xyz, &h->q, &h->F, &h->pos, &h->cell, &h->cell_cnt, &h->cell_start, &h->cell_fill,
                      &h->cell_list, &h->pos_of, &h->pcount, &h->poff, &h->pairs, &h->R, &h->Upair, &h->in_cnt,
                      &h->in_off, &h->in_fill, &h->in_list, &h->scan_tmp, &h->zperm, &h->ztmp, &h->zkey, &h->zkey2,
                      &h->zx, &h->zy, &h->zhd, &h->qd, &h->k0, &h->qscan, &h->kc, &h->kin, &h->kw,
                      &h->tot, &h->off, &h->Utot, &h->kf, &h->Epart, &h->status, &h->Eout, &h->Fpart,
                      &h->pos_c, &h->scan_tmp2, &h->Flong, &h->gF, &h->gxyz, &h->gq, &h->RA, &h->gam,
                      &h->gout, &h->zgx, &h->zgy, &h->zgz, &h->w1, &h->w2, &h->ws1, &h->ws2, &h->atot, &h->aoff,
                      &h->lam, &h->ggk, &h->Gpart, &h->gFh, &h->normxw, &h->ktab, &h->kctr, &h->zP32,
                      &h->hmask};
    for (DevBuf *b : bufs)
        if (b->p) cudaFree(b->p);
    for (cudaEvent_t e : h->prof.pool) cudaEventDestroy(e);
    if (h->gexec) cudaGraphExecDestroy(h->gexec);
    if (h->gcap) cudaStreamDestroy(h->gcap);
    if (h->s2) {
        cudaStreamSynchronize(h->s2);
        cudaStreamDestroy(h->s2);
    }
    if (h->s3) {
        cudaStreamSynchronize(h->s3);
        cudaStreamDestroy(h->s3);
    }
    if (h->ev_fork) cudaEventDestroy(h->ev_fork);
    if (h->ev_join) cudaEventDestroy(h->ev_join);
    if (h->ev_kfork) cudaEventDestroy(h->ev_kfork);
    if (h->ev_kdone) cudaEventDestroy(h->ev_kdone);
    if (h->h_status) cudaFreeHost(h->h_status);
    if (h->h_E) cudaFreeHost(h->h_E);
    if (h->h_np) cudaFreeHost(h->h_np);
    delete h;
}

const char *qem_last_error(const qem_handle *h) { return h ? h->err.c_str() : "NULL handle"; }
const char *qem_status_string(qem_status s) { return status_str(s); }

// whether every row is a lattice vector 2 pi (m / Lx, n / Ly) (integer m, n
// to 1e-6), as the FP32 k-space phases (fixed-point, lattice_phase) need
static bool lattice_rows(const double *k3, int P, double Lx, double Ly)
{
    for (int i = 0; i < P; i++) {
        const double m = k3[3 * i] * Lx / (2.0 * QEM_PI), n = k3[3 * i + 1] * Ly / (2.0 * QEM_PI);
        if (!(fabs(m) < 1e9 && fabs(n) < 1e9) || fabs(m - rint(m)) > 1e-6 || fabs(n - rint(n)) > 1e-6) return false;
    }
    return true;
}

// rows (kx, ky, |k|) with |k| > 0; returns the largest |k| or -1
static double check_krows(const double *k3, int P)
{
    double kmax = 0;
    for (int i = 0; i < P; i++) {
        const double kx = k3[3 * i], ky = k3[3 * i + 1], k = k3[3 * i + 2];
        if (!std::isfinite(kx) || !std::isfinite(ky) || !(k > 0) || fabs(kx * kx + ky * ky - k * k) > 1e-9 * k * k)
            return -1;
        kmax = std::max(kmax, k);
    }
    return kmax;
}

qem_status qem_set_kset(qem_handle *h, const double *k3, int32_t P, double sum_K)
{
    if (!h) return QEM_ERR_ARG;
    if (P < 0 || (P > 0 && !k3) || !std::isfinite(sum_K)) return fail(h, QEM_ERR_ARG, "bad k-set arguments");
    if (P > QEM_MAX_KSET) return fail(h, QEM_ERR_RANGE, "more k-vectors than QEM_MAX_KSET");
    const double kmax = check_krows(k3, P);
    if (kmax < 0) return fail(h, QEM_ERR_ARG, "k-set rows must be (kx, ky, |k|) with |k| > 0 (Force_long.jl:7)");
    h->kset.assign(k3, k3 + 3 * (size_t)P);
    h->kset_lattice = lattice_rows(k3, P, h->p.Lx, h->p.Ly);
    h->kwt.clear();
    h->P = P;
    h->sum_K = sum_K;
    h->kmax = kmax;
    h->has_kset = true;
    h->kset_dirty = true;
    h->cfg_version++;
    return QEM_OK;
}

qem_status qem_set_kset_weighted(qem_handle *h, const double *k3, const double *w, int32_t P)
{
    if (!h) return QEM_ERR_ARG;
    if (P < 0 || (P > 0 && (!k3 || !w))) return fail(h, QEM_ERR_ARG, "bad k-set arguments");
    if (P > QEM_MAX_KSET) return fail(h, QEM_ERR_RANGE, "more k-vectors than QEM_MAX_KSET");
    const double kmax = check_krows(k3, P);
    if (kmax < 0) return fail(h, QEM_ERR_ARG, "k-set rows must be (kx, ky, |k|) with |k| > 0 (Force_long.jl:7)");
    double sw = 0;
    for (int i = 0; i < P; i++) {
        if (!std::isfinite(w[i])) return fail(h, QEM_ERR_ARG, "k weights must be finite");
        sw += w[i];
    }
    h->kset.assign(k3, k3 + 3 * (size_t)P);
    h->kset_lattice = lattice_rows(k3, P, h->p.Lx, h->p.Ly);
    h->kwt.assign(w, w + P);
    h->P = P;
    h->sum_K = sw;
    h->kmax = kmax;
    h->has_kset = true;
    h->kset_dirty = true;
    h->cfg_version++;
    return QEM_OK;
}

qem_status qem_exact_kset_rows(double Lx, double Ly, double alpha, double k_cutoff, double *k3, double *w,
                               int64_t cap, int64_t *count)
{
    if (!count || !(Lx > 0) || !(Ly > 0) || !(alpha > 0) || !(k_cutoff > 0) || !std::isfinite(k_cutoff) ||
        cap < 0 || (cap > 0 && (!k3 || !w)))
        return QEM_ERR_ARG;
    const double nxf = k_cutoff * Lx / (2.0 * QEM_PI), nyf = k_cutoff * Ly / (2.0 * QEM_PI);
    if (nxf > 1e5 || nyf > 1e5) return QEM_ERR_RANGE;
    const int64_t nx = (int64_t)nxf, ny = (int64_t)nyf;
    int64_t n = 0;
    for (int64_t a = -nx; a <= nx; a++)
        for (int64_t b = -ny; b <= ny; b++) {
            if (a == 0 && b == 0) continue;  // the k = 0 term is separate (Force_long.jl:214)
            const double kx = 2.0 * QEM_PI * (double)a / Lx, ky = 2.0 * QEM_PI * (double)b / Ly;
            const double k = sqrt(kx * kx + ky * ky);
            if (!(k < k_cutoff)) continue;
            if (n < cap) {
                k3[3 * n] = kx;
                k3[3 * n + 1] = ky;
                k3[3 * n + 2] = k;
                w[n] = exp(-k * k / (4.0 * alpha));
            }
            n++;
        }
    *count = n;
    return QEM_OK;
}

qem_status qem_set_kset_exact(qem_handle *h, double k_cutoff, int32_t *P)
{
    if (!h) return QEM_ERR_ARG;
    int64_t n = 0;
    qem_status st = qem_exact_kset_rows(h->p.Lx, h->p.Ly, h->p.alpha, k_cutoff, nullptr, nullptr, 0, &n);
    if (st != QEM_OK) return fail(h, st, "exact k-set: need k_cutoff > 0 and at most 1e5 lattice steps per axis");
    if (n > QEM_MAX_KSET) return fail(h, QEM_ERR_RANGE, "exact k-set larger than QEM_MAX_KSET: lower k_cutoff");
    std::vector<double> k3(3 * (size_t)std::max<int64_t>(n, 1)), w((size_t)std::max<int64_t>(n, 1));
    st = qem_exact_kset_rows(h->p.Lx, h->p.Ly, h->p.alpha, k_cutoff, k3.data(), w.data(), n, &n);
    if (st != QEM_OK) return fail(h, st, "exact k-set generation failed");
    if (P) *P = (int32_t)n;
    return qem_set_kset_weighted(h, k3.data(), w.data(), (int32_t)n);
}

qem_status qem_get_kset_weights(const qem_handle *h, double *w_out, int32_t cap, int32_t *P)
{
    if (!h || !P) return QEM_ERR_ARG;
    *P = h->kwt.empty() ? 0 : h->P;
    if (w_out && cap > 0 && !h->kwt.empty()) memcpy(w_out, h->kwt.data(), sizeof(double) * (size_t)std::min(cap, h->P));
    return QEM_OK;
}

qem_status qem_sample_kset(qem_handle *h, uint64_t seed, int32_t P)
{
    if (!h) return QEM_ERR_ARG;
    if (P < 0) return fail(h, QEM_ERR_ARG, "P < 0");
    if (P > QEM_MAX_KSET) return fail(h, QEM_ERR_RANGE, "more k-vectors than QEM_MAX_KSET");
    h->kseed = seed;
    sample_kset(h, P);
    return QEM_OK;
}

qem_status qem_get_kset(const qem_handle *h, double *k3_out, int32_t cap, int32_t *P, double *sum_K)
{
    if (!h) return QEM_ERR_ARG;
    if (P) *P = h->P;
    if (sum_K) *sum_K = resampling(h) && h->has_kset ? h->sampler_sumK : h->sum_K;
    if (!k3_out || cap <= 0) return QEM_OK;
    uint64_t n = 0;
    if (resampling(h) && h->has_kset) {  // the batch of the latest long-range call
        if (!read_batch_counter(h, &n)) return QEM_ERR_CUDA;
    }
    if (n > 0) {
        std::vector<double> k3;
        batch_rows(h, n - 1, h->P, k3);
        memcpy(k3_out, k3.data(), sizeof(double) * 3 * (size_t)std::min(cap, h->P));
    } else {
        memcpy(k3_out, h->kset.data(), sizeof(double) * 3 * (size_t)std::min(cap, h->P));
    }
    return QEM_OK;
}

qem_status qem_kset_batch(const qem_handle *h, uint64_t *n)
{
    if (!h || !n) return QEM_ERR_ARG;
    *n = 0;
    if (!resampling(h) || !h->has_kset) return QEM_OK;
    return read_batch_counter(h, n) ? QEM_OK : QEM_ERR_CUDA;
}

qem_status qem_draw_kset(const qem_params *p, uint64_t seed, uint64_t n, int64_t row0, int32_t P, double *k3,
                         double *sum_K)
{
    if (!p || P < 0 || row0 < 0 || (P > 0 && !k3) || !finite_pos(p->Lx) || !finite_pos(p->Ly) ||
        !finite_pos(p->alpha) || !(p->accuracy > 0 && p->accuracy < 1))
        return QEM_ERR_ARG;
    const double nmax = 2.0 * sqrt(-4.0 * p->alpha * log(p->accuracy)) * std::max(p->Lx, p->Ly) / (2.0 * QEM_PI);
    if (!(nmax < 1e7)) return QEM_ERR_RANGE;
    KSampler S;
    std::vector<double> tab;
    double sK = 0, kmax = 0;
    make_sampler(*p, S, tab, sK, kmax);
    S.seed = seed;
    for (int i = 0; i < P; i++) ksample_row(S, n, row0 + i, k3[3 * i], k3[3 * i + 1], k3[3 * i + 2]);
    if (sum_K) *sum_K = sK;
    return QEM_OK;
}

qem_status qem_forces(qem_handle *h, int32_t N, const double *xyz, const double *q, double *F, double *energy,
                      uint32_t terms, int32_t mem, void *stream)
{
    return run(h, N, xyz, q, F, energy, terms, mem, (cudaStream_t)stream);
}

qem_status qem_short_forces(qem_handle *h, int32_t N, const double *xyz, const double *q, double *F, int32_t mem,
                            void *stream)
{
    return run(h, N, xyz, q, F, nullptr, QEM_TERM_SHORT, mem, (cudaStream_t)stream);
}

qem_status qem_long_forces(qem_handle *h, int32_t N, const double *xyz, const double *q, double *F, int32_t mem,
                           void *stream)
{
    return run(h, N, xyz, q, F, nullptr, QEM_TERM_LONG, mem, (cudaStream_t)stream);
}

qem_status qem_lj_forces(qem_handle *h, int32_t N, const double *xyz, double *F, int32_t mem, void *stream)
{
    if (!h) return QEM_ERR_ARG;
    if (N < 0) return fail(h, QEM_ERR_ARG, "N < 0");
    if (N == 0) return QEM_OK;
    if (!xyz || !F) return fail(h, QEM_ERR_ARG, "NULL pointer");
    // charges are not used by the walls; feed zeros of the right memory kind
    std::vector<double> qz;
    const double *q = nullptr;
    DevBuf tmp;
    if (mem == QEM_MEM_HOST) {
        qz.assign(N, 0.0);
        q = qz.data();
    } else {
        CU(cudaSetDevice(h->p.device));
        CU(grow(tmp, sizeof(double) * N));
        CU(cudaMemsetAsync(tmp.p, 0, sizeof(double) * N, (cudaStream_t)stream));
        q = ptr<double>(tmp);
    }
    qem_status st = run(h, N, xyz, q, F, nullptr, QEM_TERM_LJ, mem, (cudaStream_t)stream);
    if (tmp.p) cudaFree(tmp.p);
    return st;
}

qem_status qem_potential_energy(qem_handle *h, int32_t N, const double *xyz, const double *q, double *energy,
                                uint32_t terms, int32_t mem, void *stream)
{
    if (!h) return QEM_ERR_ARG;
    if (!energy) return fail(h, QEM_ERR_ARG, "energy is NULL");
    if (N <= 0) return run(h, N, xyz, q, nullptr, energy, terms, mem, (cudaStream_t)stream);
    DevBuf tmp;
    double *F = nullptr;
    std::vector<double> Fh;
    if (mem == QEM_MEM_HOST) {
        Fh.resize(3 * (size_t)N);
        F = Fh.data();
    } else {
        CU(cudaSetDevice(h->p.device));
        CU(grow(tmp, sizeof(double) * 3 * N));
        F = ptr<double>(tmp);
    }
    qem_status st = run(h, N, xyz, q, F, energy, terms, mem, (cudaStream_t)stream);
    if (tmp.p) cudaFree(tmp.p);
    return st;
}

qem_status qem_pair_list(qem_handle *h, int32_t N, const double *xyz, int32_t *pairs, int64_t cap, int64_t *npairs)
{
    if (!h || !npairs || N < 0 || (N > 0 && !xyz)) return QEM_ERR_ARG;
    *npairs = 0;
    if (N == 0) return QEM_OK;
    std::vector<double> q(N, 0.0), F(3 * (size_t)N);
    const uint32_t saved = h->p.mode_flags;
    h->p.mode_flags &= ~QEM_STALE_NEIGHBORS;  // always a fresh list
    qem_status st = run(h, N, xyz, q.data(), F.data(), nullptr, QEM_TERM_SHORT, QEM_MEM_HOST, 0);
    h->p.mode_flags = saved;
    if (st != QEM_OK) return st;
    *npairs = h->Np;
    if (pairs && cap > 0 && h->Np > 0) {
        const int64_t n = std::min(cap, h->Np);
        CU(cudaMemcpy(pairs, h->pairs.p, sizeof(int2) * n, cudaMemcpyDeviceToHost));
        for (int64_t t = 0; t < n; t++)  // stored as (owner, other): report (i, j) with i < j
            if (pairs[2 * t] > pairs[2 * t + 1]) std::swap(pairs[2 * t], pairs[2 * t + 1]);
    }
    return QEM_OK;
}

qem_status qem_cell_index(qem_handle *h, int32_t N, const double *xyz, int32_t *cell, int32_t *cell_start,
                          int32_t cap_cells, int32_t *ncx, int32_t *ncy)
{
    if (!h || N < 0 || (N > 0 && !xyz)) return QEM_ERR_ARG;
    if (ncx) *ncx = h->geom.ncx;
    if (ncy) *ncy = h->geom.ncy;
    if (N == 0) return QEM_OK;
    int64_t np = 0;
    qem_status st = qem_pair_list(h, N, xyz, nullptr, 0, &np);
    if (st != QEM_OK) return st;
    if (cell) CU(cudaMemcpy(cell, h->cell.p, sizeof(int) * N, cudaMemcpyDeviceToHost));
    if (cell_start && cap_cells > 0)
        CU(cudaMemcpy(cell_start, h->cell_start.p, sizeof(int) * std::min(cap_cells, h->ncell + 1),
                      cudaMemcpyDeviceToHost));
    return QEM_OK;
}

qem_status qem_z_order(qem_handle *h, int32_t N, const double *xyz, int32_t *zlist)
{
    if (!h || N < 0 || (N > 0 && (!xyz || !zlist))) return QEM_ERR_ARG;
    if (N == 0) return QEM_OK;
    std::vector<double> q(N, 0.0), F(3 * (size_t)N);
    const int P = h->P;
    const bool had = h->has_kset;
    h->P = 0;  // k = 0 term only: runs the z sort without k-space work
    h->has_kset = true;
    const int32_t saved_rbe = h->p.rbe_p;
    h->p.rbe_p = 0;
    qem_status st = run(h, N, xyz, q.data(), F.data(), nullptr, QEM_TERM_LONG, QEM_MEM_HOST, 0);
    h->P = P;
    h->has_kset = had;
    h->p.rbe_p = saved_rbe;
    if (st != QEM_OK) return st;
    CU(cudaMemcpy(zlist, h->zperm.p, sizeof(int) * N, cudaMemcpyDeviceToHost));
    return QEM_OK;
}

qem_status qem_set_profiling(qem_handle *h, int32_t on)
{
    if (!h) return QEM_ERR_ARG;
    h->prof.on = on != 0;
    return QEM_OK;
}

qem_status qem_get_timings(const qem_handle *h, double *ms, int32_t cap, int32_t *n, char *names, int32_t names_cap)
{
    if (!h) return QEM_ERR_ARG;
    const int cnt = (int)h->prof.ms.size();
    if (n) *n = cnt;
    if (ms)
        for (int i = 0; i < std::min(cap, cnt); i++) ms[i] = h->prof.ms[i];
    if (names && names_cap > 0) {
        std::string s;
        for (int i = 0; i < (int)h->prof.names.size(); i++) {
            if (i) s += ",";
            s += h->prof.names[i];
        }
        snprintf(names, names_cap, "%s", s.c_str());
    }
    return QEM_OK;
}

qem_status qem_get_counts(const qem_handle *h, int64_t *counts, int32_t cap)
{
    if (!h || !counts) return QEM_ERR_ARG;
    for (int i = 0; i < std::min(cap, 4); i++) counts[i] = h->counts[i];
    return QEM_OK;
}

const char *qem_version(void) { return "qem4molly_b200 0.1 (sm_100a)"; }

}  // extern "C"

// ---------------------------------------------------------------------------
// adjoint: L = gE E + sum_i gF_i . F_i
// ---------------------------------------------------------------------------
static qem_status backward_once(qem_handle *h, int N, const double *xyz, const double *q, const double *gF,
                                double gE, double *gxyz, double *gq, double *ggamma, uint32_t terms, int mem,
                                cudaStream_t s, bool &retry)
{
    retry = false;
    bool ties_adj = false;  // long-range gamma gradient of the second tie order in gout[4 .. 6)
    const bool do_short = terms & QEM_TERM_SHORT;
    if (h->sc.norm && do_short)
        return fail(h, QEM_ERR_ARG, "the short-range adjoint is not defined for gamma_up * gamma_down > 1");
    const bool do_long = terms & QEM_TERM_LONG;
    const bool do_lj = (terms & QEM_TERM_LJ) && h->p.n_walls > 0;
    CU(grow(h->pos, sizeof(double4) * N));
    CU(grow(h->cell, sizeof(int) * N));
    CU(grow(h->status, 64));
    const double *xyz_d = xyz, *q_d = q, *gF_d = gF;
    double *gx_d = gxyz, *gq_d = gq;
    if (mem == QEM_MEM_HOST) {
        CU(grow(h->xyz, sizeof(double) * 3 * N));
        CU(grow(h->q, sizeof(double) * N));
        CU(grow(h->gxyz, sizeof(double) * 3 * N));
        CU(cudaMemcpyAsync(h->xyz.p, xyz, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, s));
        CU(cudaMemcpyAsync(h->q.p, q, sizeof(double) * N, cudaMemcpyHostToDevice, s));
        xyz_d = ptr<double>(h->xyz);
        q_d = ptr<double>(h->q);
        gx_d = ptr<double>(h->gxyz);
        if (gF) {
            CU(grow(h->gF, sizeof(double) * 3 * N));
            CU(cudaMemcpyAsync(h->gF.p, gF, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, s));
            gF_d = ptr<double>(h->gF);
        }
        if (gq) {
            CU(grow(h->gq, sizeof(double) * N));
            gq_d = ptr<double>(h->gq);
        }
    }
    unsigned *st = ptr<unsigned>(h->status);
    CU(cudaMemsetAsync(st, 0, sizeof(unsigned), s));
    CU(qem_launch_pack(N, xyz_d, q_d, ptr<double4>(h->pos), ptr<int>(h->cell), h->geom, st, s));
    CU(grow(h->gout, sizeof(double) * 8));
    CU(cudaMemsetAsync(h->gout.p, 0, sizeof(double) * 8, s));
    double *gout = ptr<double>(h->gout);  // [0, 2): short gamma, [2, 4): long gamma
    CU(grow(h->scan_tmp, qem_scan_tmp_bytes(std::max(std::max(N, h->ncell), 1)) + 64));

    std::function<cudaError_t()> long_final;  // the side stream's last step, on s after the short range
    auto long_range = [&]() -> qem_status {
        if (do_long) {
            if (!h->has_kset && h->p.rbe_p > 0) sample_kset(h, h->p.rbe_p);
            uint64_t nb = 0;
            if (resampling(h) && h->has_kset) {  // the batch of the latest forward call
                if (!read_batch_counter(h, &nb)) return fail(h, QEM_ERR_CUDA, "reading the k batch counter");
                if (nb > 0) {
                    batch_rows(h, nb - 1, h->P, h->kset);
                    h->kwt.clear();
                    h->sum_K = h->sampler_sumK;
                    h->kset_dirty = true;
                }
            }
            const int Pk = h->has_kset ? h->P : 0;
            const int LCH = qem_long_chunk();
            const int nch = (N + LCH - 1) / LCH, nbS = (N + 255) / 256, nb0 = (N + 255) / 256;
            const int ks = qem_long_ksplit(nch, std::max(Pk, 1), h->long_max_ks, QEM_FP64);
            CU(grow(h->Epart, sizeof(double) * ((size_t)nbS + (size_t)ks * nch + nb0 + std::max(Pk, 1) + 8)));
            LongBuffers b;
            {
                const qem_status ls = long_buffers(h, N, Pk, nch, ks, ptr<double>(h->Epart), nbS, nb0, b);
                if (ls != QEM_OK) return ls;
            }
            if ((h->kset_dirty || h->kin_lo != 0 || h->kin_hi != Pk) && Pk > 0) {
                CU(cudaMemcpyAsync(h->kin.p, h->kset.data(), sizeof(double) * 3 * Pk, cudaMemcpyHostToDevice, s));
                if (!h->kwt.empty())
                    CU(cudaMemcpyAsync(h->kw.p, h->kwt.data(), sizeof(double) * Pk, cudaMemcpyHostToDevice, s));
                h->kset_dirty = false;
                h->kin_lo = 0;
                h->kin_hi = Pk;
            }
            // the long range runs on the side stream beside the short range
            // (its final pass, which adds into the gradients, after the join);
            // with equal-z ties it stays on s after the short range
            const bool side = !(h->p.mode_flags & QEM_EQUAL_Z_TIES);
            cudaStream_t sl = side ? h->s2 : s;
            if (side) {
                CU(cudaEventRecord(h->ev_fork, s));
                CU(cudaStreamWaitEvent(sl, h->ev_fork, 0));
            }
            CU(qem_launch_zsort(N, ptr<double4>(h->pos), ptr<int>(h->zperm), ptr<int>(h->ztmp), ptr<double>(h->zkey),
                                ptr<double>(h->zkey2), sl, false, ptr<int>(h->ztmp) + N, h->p.Lz));
            CU(qem_launch_long(QEM_FP64, false, N, Pk, ptr<double4>(h->pos), ptr<int>(h->zperm), b, h->p.Lx, h->p.Ly,
                               h->p.Lz, h->p.gamma_down, h->p.gamma_up, h->p.eps_0, h->sum_K, nullptr, nch, st, sl, 0));
            const size_t P1 = std::max(Pk, 1);
            CU(grow(h->zgx, sizeof(double) * N));
            CU(grow(h->zgy, sizeof(double) * N));
            CU(grow(h->zgz, sizeof(double) * N));
            CU(grow(h->w1, sizeof(double) * N));
            CU(grow(h->w2, sizeof(double) * N));
            CU(grow(h->ws1, sizeof(double) * (N + 1)));
            CU(grow(h->ws2, sizeof(double) * (N + 1)));
            CU(grow(h->atot, sizeof(double) * 8 * P1 * nch));
            CU(grow(h->aoff, sizeof(double) * 4 * P1 * nch));
            CU(grow(h->lam, sizeof(double) * 4 * P1));
            CU(grow(h->ggk, sizeof(double) * 2 * P1));
            CU(grow(h->Gpart, sizeof(double) * 4 * (size_t)ks * N));
            LongAdjBuffers a;
            a.zgx = ptr<double>(h->zgx); a.zgy = ptr<double>(h->zgy); a.zgz = ptr<double>(h->zgz);
            a.w1 = ptr<double>(h->w1); a.w2 = ptr<double>(h->w2); a.s1 = ptr<double>(h->ws1); a.s2 = ptr<double>(h->ws2);
            a.atot = ptr<double>(h->atot); a.aoff = ptr<double>(h->aoff); a.lam = ptr<double>(h->lam);
            a.ggk = ptr<double>(h->ggk); a.Gpart = ptr<double>(h->Gpart); a.gam = gout + 2;
            if (side) {
                CU(qem_launch_long_adj(N, Pk, ptr<int>(h->zperm), b, a, h->p.Lx, h->p.Ly, h->p.Lz, h->p.gamma_down,
                                       h->p.gamma_up, h->p.eps_0, gF_d, gE, gx_d, gq_d, nch, ks, sl, 0));
                CU(cudaEventRecord(h->ev_join, sl));
                long_final = [=]() -> cudaError_t {
                    cudaError_t e = cudaStreamWaitEvent(s, h->ev_join, 0);
                    if (e != cudaSuccess) return e;
                    return qem_launch_long_adj(N, Pk, ptr<int>(h->zperm), b, a, h->p.Lx, h->p.Ly, h->p.Lz,
                                               h->p.gamma_down, h->p.gamma_up, h->p.eps_0, gF_d, gE, gx_d, gq_d, nch,
                                               ks, s, 1);
                };
            } else {
                // the forward force is the mean over the two tie orders, so the
                // adjoint is the sum of both orders' adjoints of (gF / 2, gE / 2);
                // the second order's gamma gradient goes to gout[4 .. 6)
                CU(grow(h->gFh, sizeof(double) * 3 * N));
                double *gFh = ptr<double>(h->gFh);
                if (gF_d) CU(qem_launch_scale(3 * N, 0.5, gF_d, gFh, s));
                else CU(cudaMemsetAsync(gFh, 0, sizeof(double) * 3 * N, s));
                CU(qem_launch_long_adj(N, Pk, ptr<int>(h->zperm), b, a, h->p.Lx, h->p.Ly, h->p.Lz, h->p.gamma_down,
                                       h->p.gamma_up, h->p.eps_0, gFh, 0.5 * gE, gx_d, gq_d, nch, ks, s));
                CU(qem_launch_zsort(N, ptr<double4>(h->pos), ptr<int>(h->zperm), ptr<int>(h->ztmp),
                                    ptr<double>(h->zkey), ptr<double>(h->zkey2), s, true, ptr<int>(h->ztmp) + N,
                                    h->p.Lz));
                CU(qem_launch_long(QEM_FP64, false, N, Pk, ptr<double4>(h->pos), ptr<int>(h->zperm), b, h->p.Lx,
                                   h->p.Ly, h->p.Lz, h->p.gamma_down, h->p.gamma_up, h->p.eps_0, h->sum_K, nullptr, nch,
                                   st, s, 0));
                a.gam = gout + 4;
                CU(qem_launch_long_adj(N, Pk, ptr<int>(h->zperm), b, a, h->p.Lx, h->p.Ly, h->p.Lz, h->p.gamma_down,
                                       h->p.gamma_up, h->p.eps_0, gFh, 0.5 * gE, gx_d, gq_d, nch, ks, s));
                ties_adj = true;
            }
        }
        return QEM_OK;
    };
    const bool long_first = do_long && !(h->p.mode_flags & QEM_EQUAL_Z_TIES);
    if (long_first) {
        const qem_status ls_ = long_range();
        if (ls_ != QEM_OK) return ls_;
    }
    if (do_short || do_lj) {
        if (do_short) {
            const bool stale = (h->p.mode_flags & QEM_STALE_NEIGHBORS) != 0;
            if (!stale || !h->pairs_valid || h->pairs_N != N) {
                const qem_status bs = build_pairs(h, N, st, s);
                if (bs != QEM_OK) return bs;
            }
            CU(grow(h->RA, sizeof(double4) * 2 * h->pair_cap));
            CU(qem_launch_short_pair_adj(ptr<int64_t>(h->poff) + N, h->pair_cap, ptr<int2>(h->pairs),
                                         ptr<double4>(h->pos), gF_d, gE, ptr<double4>(h->RA), h->sc, s));
        }
        const int nb = qem_adj_gather_blocks(N);
        CU(grow(h->gam, sizeof(double) * 2 * nb));
        CU(qem_launch_adj_gather(N, do_short, do_lj, ptr<double4>(h->pos), ptr<int>(h->pos_of),
                                 ptr<int64_t>(h->poff), ptr<double4>(h->RA), ptr<int64_t>(h->in_off),
                                 ptr<int>(h->in_list), h->pair_cap, gF_d, gE, h->sc, gx_d, gq_d,
                                 ptr<double>(h->gam), s));
        CU(qem_launch_reduce_sum(ptr<double>(h->gam), nb, gout, s));
        CU(qem_launch_reduce_sum(ptr<double>(h->gam) + nb, nb, gout + 1, s));
    } else {
        CU(cudaMemsetAsync(gx_d, 0, sizeof(double) * 3 * N, s));
        if (gq_d) CU(cudaMemsetAsync(gq_d, 0, sizeof(double) * N, s));
    }

    if (!long_first) {
        const qem_status ls_ = long_range();
        if (ls_ != QEM_OK) return ls_;
    }
    if (long_final) CU(long_final());
    double hg[6] = {0, 0, 0, 0, 0, 0};
    CU(cudaMemcpyAsync(hg, gout, sizeof(double) * 6, cudaMemcpyDeviceToHost, s));
    if (mem == QEM_MEM_HOST) {
        CU(cudaMemcpyAsync(gxyz, gx_d, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, s));
        if (gq) CU(cudaMemcpyAsync(gq, gq_d, sizeof(double) * N, cudaMemcpyDeviceToHost, s));
    }
    CU(cudaMemcpyAsync(h->h_status, st, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    if (do_short)
        CU(cudaMemcpyAsync(h->h_np, ptr<int64_t>(h->poff) + N, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    CU(cudaGetLastError());
    if (do_short) {
        h->Np = *h->h_np;
        if (*h->h_status & QEM_ST_OVERFLOW) {
            h->pair_cap = h->Np + h->Np / 4 + 4096;
            h->pairs_valid = false;
            retry = true;
            return QEM_OK;
        }
    }
    const unsigned stv = *h->h_status;
    if (stv & QEM_ST_NONFINITE) return fail(h, QEM_ERR_NONFINITE, "NaN or Inf in coordinates or charges");
    if (stv & QEM_ST_OUT_OF_SLAB) return fail(h, QEM_ERR_OUT_OF_SLAB, "direction * (z - sub_pos) <= 0 for some particle");
    if (ggamma) {
        ggamma[0] = hg[0] + (ties_adj ? hg[2] + hg[4] : hg[2]);
        ggamma[1] = hg[1] + (ties_adj ? hg[3] + hg[5] : hg[3]);
    }
    h->err.clear();
    return QEM_OK;
}

extern "C" qem_status qem_backward(qem_handle *h, int32_t N, const double *xyz, const double *q, const double *gF,
                                   double gE, double *gxyz, double *gq, double *ggamma, uint32_t terms, int32_t mem,
                                   void *stream)
{
    if (!h) return QEM_ERR_ARG;
    if (N < 0) return fail(h, QEM_ERR_ARG, "N < 0");
    if (terms & ~QEM_TERM_ALL) return fail(h, QEM_ERR_ARG, "unknown term bit");
    if (mem != QEM_MEM_HOST && mem != QEM_MEM_DEVICE) return fail(h, QEM_ERR_ARG, "mem must be HOST or DEVICE");
    if (!std::isfinite(gE)) return fail(h, QEM_ERR_ARG, "gE is not finite");
    if (N == 0) {
        if (ggamma) ggamma[0] = ggamma[1] = 0;
        return QEM_OK;
    }
    if (!xyz || !q || !gxyz) return fail(h, QEM_ERR_ARG, "NULL coordinate, charge or gradient pointer");
    if (cudaSetDevice(h->p.device) != cudaSuccess) return fail(h, QEM_ERR_CUDA, "cudaSetDevice");
    cudaStream_t s = (cudaStream_t)stream;
    bool retry = false;
    qem_status st = backward_once(h, N, xyz, q, gF, gE, gxyz, gq, ggamma, terms, mem, s, retry);
    if (st == QEM_OK && retry) st = backward_once(h, N, xyz, q, gF, gE, gxyz, gq, ggamma, terms, mem, s, retry);
    if (st == QEM_OK && retry) return fail(h, QEM_ERR_NB_OVERFLOW, "pair list outgrew its capacity twice");
    return st;
}

// ---------------------------------------------------------------------------
// internal hooks of the batch API (qem_batch.cu)
// ---------------------------------------------------------------------------
qem_status qem_forces_async(qem_handle *h, int N, const double *xyz, const double *q, double *F, uint32_t terms,
                            cudaStream_t s)
{
    bool retry = false;
    return run_once(h, N, xyz, q, F, nullptr, terms, QEM_MEM_DEVICE, s, retry, true);
}

void qem_handle_set_long_max_ks(qem_handle *h, int max_ks)
{
    if (!h || max_ks < 1) return;
    h->long_max_ks = std::min(max_ks, QEM_LONG_MAX_KS);
    h->cfg_version++;
}

qem_status qem_status_check(qem_handle *h, cudaStream_t s)
{
    if (!h->status.p) return QEM_OK;
    CU(cudaSetDevice(h->p.device));
    CU(cudaMemcpyAsync(h->h_status, h->status.p, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    CU(cudaMemsetAsync(h->status.p, 0, sizeof(unsigned), s));
    CU(cudaStreamSynchronize(s));
    const unsigned stv = *h->h_status;
    if (stv & QEM_ST_OVERFLOW) return fail(h, QEM_ERR_NB_OVERFLOW, "pair list outgrew its capacity in an asynchronous call");
    if (stv & QEM_ST_NONFINITE) return fail(h, QEM_ERR_NONFINITE, "NaN or Inf in coordinates or charges");
    if (stv & QEM_ST_OUT_OF_SLAB) return fail(h, QEM_ERR_OUT_OF_SLAB, "direction * (z - sub_pos) <= 0 for some particle");
    if (stv & QEM_ST_RANGE) return fail(h, QEM_ERR_RANGE, range_msg);
    return QEM_OK;
}

const qem_params *qem_handle_params(const qem_handle *h) { return &h->p; }
const char *qem_handle_error(const qem_handle *h) { return h->err.c_str(); }

uint64_t qem_handle_state(const qem_handle *h)
{
    uint64_t v = mix64(g_alloc_epoch.load() + 0x51ULL);
    v = mix64(v ^ h->cfg_version);
    v = mix64(v ^ (uint64_t)h->pair_cap);
    v = mix64(v ^ ((uint64_t)h->P << 1) ^ (h->has_kset ? 1u : 0u));
    return mix64(v ^ (h->kset_dirty ? 3u : 5u) ^ ((uint64_t)h->pairs_N << 8));
}

// The arguments run_once gives the small-system kernels, collected for one
// system of a fused batch: the same buffers, the same k-slice count (unless
// ks > 0 picks fewer) and the same per-k constants.
qem_status qem_handle_batch_sys(qem_handle *h, int N, int ks, int lch, BatchSys *d, ShortConsts *sc,
                                const char **why)
{
    auto no = [&](const char *m) {
        if (why) *why = m;
        return QEM_ERR_ARG;
    };
    auto not_ready = [&](const char *m) {  // a synchronous call of the system sizes it
        if (why) *why = m;
        return QEM_ERR_NO_KSET;
    };
    if (h->p.precision != QEM_FP32_FIX) return no("precision is not QEM_FP32_FIX");
    if (N <= 0) return no("no particles");
    if (N > 8192 || !qem_cells_small(N, h->ncell)) return no("more than 8192 particles or cells");
    if (h->geom.ncx >= 3 && h->geom.ncy >= 3 && (int64_t)N >= 2 * (int64_t)h->ncell)
        return no("two or more particles per cell (warp-per-cell pair list)");
    if (h->p.mode_flags & QEM_EQUAL_Z_TIES) return no("equal-z tie mode");
    if (h->shard_world != 1) return no("sharded handle");
    if (h->sc.norm) return no("gamma_up * gamma_down > 1");
    if (!h->pairs_valid || h->pairs_N != N || !h->status.p || !h->Epart.p)
        return not_ready("no synchronous call of this size yet");
    const bool draw = resampling(h);
    if ((h->p.rbe_p > 0 && !h->has_kset) || h->kset_dirty || (draw && (!h->ktab_on_dev || h->kctr_reset)))
        return not_ready("the k-set is not on the device (synchronous call first)");
    const int P = h->has_kset ? h->P : 0;
    const double kmax = draw ? h->kmax_lattice : h->kmax;
    if (P > 0 && !draw && !h->kset_lattice) return no("k-set rows off the lattice");
    if (P > 0 && (h->kin_lo != 0 || h->kin_hi != P)) return not_ready("the k rows on the device are not the whole set");
    const int LCH = qem_long_chunk();
    if (lch <= 0) lch = LCH;
    if (lch < 32 || LCH % lch != 0) return no("chunk length must divide qem_long_chunk() and be >= 32");
    const int nch = (N + lch - 1) / lch, nbS = (N + 255) / 256, nb0 = nbS;
    const int ks_own = qem_long_ksplit(nch, std::max(P > 0 ? P : h->p.rbe_p, 1), h->long_max_ks, h->p.precision);
    // energy partials (the scan writes its per-k split terms there) for this chunking
    CU(grow(h->Epart, sizeof(double) * ((size_t)nbS + (size_t)ks_own * nch + nb0 + std::max(P, h->p.rbe_p) + 8)));
    LongBuffers b;
    const qem_status ls = long_buffers(h, N, P, nch, ks_own, ptr<double>(h->Epart), nbS, nb0, b);
    if (ls != QEM_OK) return ls;
    b.ks = ks > 0 ? std::min(ks, ks_own) : ks_own;
    b.zlim = P > 0 ? qem_fp32_zlim(kmax) : 0.0;
    if (draw && P > 0) {
        b.draw_ctr = ptr<unsigned long long>(h->kctr);
        b.sampler = h->ksamp;
        b.sampler.tab = ptr<double>(h->ktab);
        b.sampler.seed = h->kseed;
        b.sampler.row0 = 0;
        b.kwt = nullptr;
    }
    BatchSys &e = *d;
    e = BatchSys{};
    e.N = N;
    e.ncell = h->ncell;
    e.P = P;
    e.nch = nch;
    e.lch = lch;
    e.ks = b.ks;
    e.cap = h->pair_cap;
    e.Flong = ptr<double>(h->Flong);
    e.pos = ptr<double4>(h->pos);
    e.pos_c = ptr<double4>(h->pos_c);
    e.cell = ptr<int>(h->cell);
    e.cstart = ptr<int>(h->cell_start);
    e.clist = ptr<int>(h->cell_list);
    e.pos_of = ptr<int>(h->pos_of);
    e.pcount = ptr<int>(h->pcount);
    e.in_cnt = ptr<int>(h->in_cnt);
    e.in_fill = ptr<int>(h->in_fill);
    e.in_list = ptr<int>(h->in_list);
    e.poff = ptr<int64_t>(h->poff);
    e.in_off = ptr<int64_t>(h->in_off);
    e.pairs = ptr<int2>(h->pairs);
    e.R = ptr<double4>(h->R);
    e.status = ptr<unsigned>(h->status);
    e.geom = h->geom;
    e.rc2 = h->sc.rc2;
    e.zperm = ptr<int>(h->zperm);
    e.ztmp = ptr<int>(h->ztmp);
    e.zkey = ptr<double>(h->zkey);
    e.zkey2 = ptr<double>(h->zkey2);
    e.b = b;
    const double Lx = h->p.Lx, Ly = h->p.Ly, Lz = h->p.Lz, eps0 = h->p.eps_0;
    const double sumK = P > 0 ? h->sum_K * P / P : 0.0;  // run_once's sum_K * Pk / Pall, bit for bit
    e.h = 0.5 * Lz;
    e.fscale = 1.0 / (2.0 * Lx * Ly * eps0);
    e.Lz = Lz;
    e.g1 = h->p.gamma_down;
    e.g2 = h->p.gamma_up;
    e.g12 = e.g1 * e.g2;
    e.wk = P > 0 ? (sumK / P) / (Lx * Ly * eps0) : 0.0;
    e.esc = P > 0 ? -(sumK / P) / (2.0 * eps0 * Lx * Ly) : 0.0;
    e.wden = Lx * Ly * eps0;
    e.eden = 2.0 * eps0 * Lx * Ly;
    e.invLx = 1.0 / Lx;
    e.invLy = 1.0 / Ly;
    e.Lx_2pi = Lx / (2.0 * QEM_PI);
    e.Ly_2pi = Ly / (2.0 * QEM_PI);
    *sc = h->sc;
    return QEM_OK;
}

extern "C" qem_status qem_set_shard(qem_handle *h, int32_t rank, int32_t world)
{
    if (!h) return QEM_ERR_ARG;
    if (world < 1 || world > 4096 || rank < 0 || rank >= world)
        return fail(h, QEM_ERR_ARG, "shard rank must be in 0 .. world - 1, world in 1 .. 4096");
    h->shard_rank = rank;
    h->shard_world = world;
    h->cfg_version++;
    h->sc.shard_rank = rank;
    h->sc.shard_world = world;
    h->err.clear();
    return QEM_OK;
}

// qem_noalloc.cu -- long-range (random-batch k-space) forces that allocate
// no device memory.
//
// Some callers cannot call cudaMalloc: a host framework that hands all device
// memory to its own pool (a foreign allocation would fragment it or exceed
// its budget), or a real-time loop that must not enter the CUDA allocator,
// whose cost and implicit synchronisation are unbounded.  For them
// qem_long_forces_noalloc runs the same kernels as qem_long_forces, with all
// of their scratch (packed particles, z order, z-ordered copies, per-k
// constants, chunk totals and offsets, status word) carved out of one
// file-scope __device__ array of QEM_NOALLOC_SCRATCH_BYTES.  Every GPU that
// loads libqem.so holds that array until the process exits.
//
// Host code never dereferences the array's name: on every call, with the
// call's device current, cudaGetSymbolAddress gives its device address, which
// is passed to the kernels.  The address is not cached: a host framework that
// tears the primary context down and creates it again (or a
// cudaDeviceReset) loads the module anew, and the array may then live
// elsewhere.  The lookup costs little next to the call's own synchronisation.
// The call synchronises its stream and reports non-finite inputs (and, in
// FP32, particles so far outside the slab that e^{+-k (z - L_z/2)} would leave
// FP32 range).  All calls share the
// array, so calls that overlap on the GPU (different streams, host threads)
// race: serialise them.  Nothing in the array needs to start at zero except
// the status word, which is cleared on every call.
#include <cstdio>

#include "qem_internal.cuh"

namespace {

constexpr int NA_MAX_N = QEM_NOALLOC_MAX_N;
constexpr int NA_MAX_P = QEM_NOALLOC_MAX_P;
constexpr int NA_CH = 512;    // particles per long-range chunk (qem_long_chunk())
constexpr int NA_MAX_KS = 2;  // k slices of the force pass
constexpr int NA_MAX_NCH = (NA_MAX_N + NA_CH - 1) / NA_CH;

constexpr size_t al(size_t b) { return (b + 255) & ~(size_t)255; }
constexpr size_t O_POS = 0;
constexpr size_t O_CELL = O_POS + al(sizeof(double4) * NA_MAX_N);
constexpr size_t O_ZPERM = O_CELL + al(sizeof(int) * NA_MAX_N);
constexpr size_t O_ZTMP = O_ZPERM + al(sizeof(int) * NA_MAX_N);
constexpr size_t O_ZKEY = O_ZTMP + al(sizeof(int) * NA_MAX_N);
constexpr size_t O_ZKEY2 = O_ZKEY + al(sizeof(double) * NA_MAX_N);
constexpr size_t O_ZX = O_ZKEY2 + al(sizeof(double) * NA_MAX_N);
constexpr size_t O_ZY = O_ZX + al(sizeof(double) * NA_MAX_N);
constexpr size_t O_ZHD = O_ZY + al(sizeof(double) * NA_MAX_N);
constexpr size_t O_QD = O_ZHD + al(sizeof(double) * NA_MAX_N);
constexpr size_t O_K0 = O_QD + al(sizeof(double) * NA_MAX_N);
constexpr size_t O_QSCAN = O_K0 + al(sizeof(double) * NA_MAX_N);
constexpr size_t O_ZP = O_QSCAN + al(sizeof(double) * (NA_MAX_N + 1));
constexpr size_t O_KIN = O_ZP + al(sizeof(uint4) * NA_MAX_N);
constexpr size_t O_KC = O_KIN + al(sizeof(double) * 3 * NA_MAX_P);
constexpr size_t O_TOT = O_KC + al(sizeof(KConst) * NA_MAX_P);
constexpr size_t O_OFF = O_TOT + al(sizeof(double) * 4 * (size_t)NA_MAX_P * NA_MAX_NCH);
constexpr size_t O_UTOT = O_OFF + al(sizeof(double) * 4 * (size_t)NA_MAX_P * NA_MAX_NCH);
constexpr size_t O_KF = O_UTOT + al(sizeof(double) * 4 * NA_MAX_P);
constexpr size_t O_FPART = O_KF + al(sizeof(KForce<double>) * NA_MAX_P);
constexpr size_t O_EPART = O_FPART + al(sizeof(double) * 3 * (size_t)NA_MAX_KS * NA_MAX_N);
constexpr size_t N_EPART = NA_MAX_KS * NA_MAX_NCH + (NA_MAX_N + 255) / 256 + NA_MAX_P + 8;
constexpr size_t O_STMP = O_EPART + al(sizeof(double) * N_EPART);
constexpr size_t STMP_BYTES = sizeof(double) * ((NA_MAX_N + 1023) / 1024 + 8);
constexpr size_t O_STATUS = O_STMP + al(STMP_BYTES);
constexpr size_t NA_BYTES = O_STATUS + 256;
static_assert(NA_BYTES <= QEM_NOALLOC_SCRATCH_BYTES, "scratch layout exceeds the declared size");

__device__ __align__(256) unsigned char g_noalloc_scratch[QEM_NOALLOC_SCRATCH_BYTES];

// device address of g_noalloc_scratch on the current device, looked up afresh
// on every call (the module, and with it the array, is loaded again after a
// context is destroyed and re-created)
qem_status scratch_address(unsigned char **out)
{
    void *ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || !ptr) {
        fprintf(stderr, "qem_long_forces_noalloc: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
        return QEM_ERR_CUDA;
    }
    *out = (unsigned char *)ptr;
    return QEM_OK;
}

qem_status reject(const char *why)
{
    fprintf(stderr, "qem_long_forces_noalloc: %s\n", why);
    return QEM_ERR_ARG;
}

}  // namespace

extern "C" qem_status qem_long_forces_noalloc(const qem_params *p, int32_t N, const double *xyz, const double *q,
                                              int32_t P, const double *k3, double sum_K, double *F, void *stream)
{
    if (!p) return reject("params is NULL");
    if (N < 0 || N > NA_MAX_N) return reject("N outside 0..QEM_NOALLOC_MAX_N (32768)");
    if (P < 0 || P > NA_MAX_P) return reject("P outside 0..QEM_NOALLOC_MAX_P (512)");
    if (N == 0) return QEM_OK;
    if (!xyz || !q || !F || (P > 0 && !k3)) return reject("NULL pointer");
    if (!(p->Lx > 0 && p->Ly > 0 && p->Lz > 0 && p->eps_0 > 0) || !std::isfinite(sum_K) ||
        !(fabs(p->gamma_up * p->gamma_down) < 1.0) ||
        (p->precision != QEM_FP64 && p->precision != QEM_FP32_FIX) || p->device < 0)
        return reject("invalid parameters");
    double kmax = 0;
    for (int i = 0; i < P; i++) {
        const double kx = k3[3 * i], ky = k3[3 * i + 1], k = k3[3 * i + 2];
        if (!std::isfinite(kx) || !std::isfinite(ky) || !(k > 0) || fabs(kx * kx + ky * ky - k * k) > 1e-9 * k * k)
            return reject("k-set rows must be (kx, ky, |k|) with |k| > 0");
        kmax = std::max(kmax, k);
    }
    if (p->precision == QEM_FP32_FIX) {  // the FP32 phases are fixed-point lattice phases
        for (int i = 0; i < P; i++) {
            const double m = k3[3 * i] * p->Lx / (2.0 * QEM_PI), n = k3[3 * i + 1] * p->Ly / (2.0 * QEM_PI);
            if (!(fabs(m) < 1e9 && fabs(n) < 1e9) || fabs(m - rint(m)) > 1e-6 || fabs(n - rint(n)) > 1e-6)
                return reject("QEM_FP32_FIX takes lattice k-vectors 2 pi (m / Lx, n / Ly) only");
        }
    }
    if (qem_long_chunk() != NA_CH) return reject("scratch layout does not match the long-range chunk size");
    if (cudaSetDevice(p->device) != cudaSuccess) return QEM_ERR_CUDA;
    unsigned char *S = nullptr;
    qem_status st = scratch_address(&S);
    if (st != QEM_OK) return st;
    cudaStream_t s = (cudaStream_t)stream;
    unsigned *status = (unsigned *)(S + O_STATUS);
    double4 *pos = (double4 *)(S + O_POS);
    int *zperm = (int *)(S + O_ZPERM);
    if (cudaMemsetAsync(status, 0, sizeof(unsigned), s) != cudaSuccess) return QEM_ERR_CUDA;
    if (cudaMemsetAsync(F, 0, sizeof(double) * 3 * (size_t)N, s) != cudaSuccess) return QEM_ERR_CUDA;
    if (P > 0 && cudaMemcpyAsync(S + O_KIN, k3, sizeof(double) * 3 * P, cudaMemcpyHostToDevice, s) != cudaSuccess)
        return QEM_ERR_CUDA;
    CellGeom g;
    g.Lx = p->Lx; g.Ly = p->Ly; g.invLx = 1.0 / p->Lx; g.invLy = 1.0 / p->Ly;
    g.ncx = 1; g.ncy = 1; g.inv_lcx = 1.0 / p->Lx; g.inv_lcy = 1.0 / p->Ly;
    cudaError_t e = qem_launch_pack(N, xyz, q, pos, (int *)(S + O_CELL), g, status, s);
    if (e == cudaSuccess)
        e = qem_launch_zsort(N, pos, zperm, (int *)(S + O_ZTMP), (double *)(S + O_ZKEY), (double *)(S + O_ZKEY2), s);
    LongBuffers b;
    b.zx = (double *)(S + O_ZX); b.zy = (double *)(S + O_ZY);
    b.zhd = (double *)(S + O_ZHD);
    b.qd = (double *)(S + O_QD);
    b.k0 = (double *)(S + O_K0); b.qscan = (double *)(S + O_QSCAN);
    b.kc = (KConst *)(S + O_KC); b.kin = (double *)(S + O_KIN);
    b.tot = (double *)(S + O_TOT); b.off = (double *)(S + O_OFF); b.Utot = (double *)(S + O_UTOT);
    b.kf = S + O_KF;
    b.Epart = (double *)(S + O_EPART);
    const int nch = (N + NA_CH - 1) / NA_CH;
    b.ks = qem_long_ksplit(nch, P, NA_MAX_KS, p->precision);
    b.Fpart = (double *)(S + O_FPART);
    b.Eks = b.Epart + (size_t)b.ks * nch + (NA_MAX_N + 255) / 256;
    b.stmp = S + O_STMP; b.stmp_bytes = STMP_BYTES;
    b.zP = (uint4 *)(S + O_ZP);
    b.zlim = p->precision == QEM_FP32_FIX && P > 0 ? qem_fp32_zlim(kmax) : 0.0;
    for (int stage = 0; stage < 2 && e == cudaSuccess; stage++)
        e = qem_launch_long(p->precision, false, N, P, pos, zperm, b, p->Lx, p->Ly, p->Lz, p->gamma_down, p->gamma_up,
                            p->eps_0, sum_K, F, nch, status, s, stage);
    if (e != cudaSuccess) return QEM_ERR_CUDA;
    unsigned host_status = 0;
    if (cudaMemcpyAsync(&host_status, status, sizeof(unsigned), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return QEM_ERR_CUDA;
    if (host_status & QEM_ST_NONFINITE) return QEM_ERR_NONFINITE;
    if (host_status & QEM_ST_RANGE) return QEM_ERR_RANGE;
    return QEM_OK;
}

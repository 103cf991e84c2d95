// qem_batch.cu -- batches of independent systems: batched force evaluation,
// a velocity-Verlet step recorded once as a CUDA graph and replayed, and an
// autotuner for the phase tiling.
//
// Reference: the MD setups of test/QEM_test.jl:40-60 (Molly VelocityVerlet
// over QEM_short + QEM_long + Substrate_LJ) run one system at a time; the
// batch runs many small slabs together.  Each system keeps its own handle
// (parameters, k-set, neighbour list, device buffers).
//
// Two ways to run a batch evaluation:
//  * fused phases (every system small enough for the one-block kernels, in
//    FP32+fix): 16 or 17 launches for the whole batch.  Pack and the
//    sorted 2048-key z tiles run over (system, tile) work lists; then,
//    on a second stream, the z merge passes and the long-range phases
//    (preparation one block per system, chunk totals, their scan, the
//    k-sliced force pass, the final sum), and on the first stream the cells
//    and the pair list (eight phases over cell, particle and pair tiles, the
//    scans one block per system) and the pair forces; the gather joins them.  The blocks run the single-system kernels' per-block code on the
//    system's own buffers, so a system's forces are those of its own
//    qem_forces call.
//  * per-system pipelines forked over a pool of streams (any batch).
// The autotuner times the pool widths and the fused tilings (k-slices per
// system of the force pass, work-list order) and keeps the fastest.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "qem_internal.cuh"

namespace {

// x += v dt + F dt^2 / 2 (unit masses), x and y wrapped into [0, L)
__global__ void k_vv_drift(int n, double *__restrict__ x, const double *__restrict__ v,
                           const double *__restrict__ F, double dt, const int *__restrict__ sys,
                           const double *__restrict__ box)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int s = sys[i];
    for (int c = 0; c < 3; c++) x[3 * i + c] += dt * v[3 * i + c] + 0.5 * dt * dt * F[3 * i + c];
    const double Lx = box[2 * s], Ly = box[2 * s + 1];
    x[3 * i] -= Lx * floor(x[3 * i] / Lx);
    x[3 * i + 1] -= Ly * floor(x[3 * i + 1] / Ly);
}

// v += (F + F') dt / 2, F = F'
__global__ void k_vv_kick(int n3, double *__restrict__ v, double *__restrict__ F, const double *__restrict__ Fn,
                          double dt)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n3) return;
    const double fn = Fn[i];
    v[i] += 0.5 * dt * (F[i] + fn);
    F[i] = fn;
}

// Andersen thermostat (Molly AndersenThermostat(temp, coupling_const), used by
// test/QEM_test.jl:53-56; python_lib Andersen.py:8-22): after each step every
// particle, with probability p = dt / coupling_const, takes a fresh velocity
// with N(0, sigma^2) components, sigma^2 = kT / m (unit masses here).  Random
// numbers come from a counter-based generator: the SplitMix64 finaliser
// (Steele, Lea and Flood, OOPSLA 2014; Vigna's constants) of
// seed + golden-ratio increments of (step, particle, draw), so every draw is
// a pure function of (seed, step, i, draw) (draw64, qem_internal.cuh) and a
// replayed graph draws new numbers through the step counter in device memory.
// uniform in (0, 1]: 53 random bits
__device__ inline double unit53(uint64_t r) { return ((double)(r >> 11) + 1.0) * 0x1.0p-53; }

__global__ void k_andersen(int n, double *__restrict__ v, double p, double sigma, uint64_t seed,
                           const unsigned long long *__restrict__ step)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t st = *step;
    if (unit53(draw64(seed, st, i, 0)) > p) return;  // no collision (P(u <= p) = p)
    // Box-Muller: two uniforms -> two normals; three components from two pairs
    const double u1 = unit53(draw64(seed, st, i, 1)), u2 = unit53(draw64(seed, st, i, 2));
    const double u3 = unit53(draw64(seed, st, i, 3)), u4 = unit53(draw64(seed, st, i, 4));
    const double r1 = sigma * sqrt(-2.0 * log(u1)), r2 = sigma * sqrt(-2.0 * log(u3));
    double s1, c1, s2, c2;
    sincospi(2.0 * u2, &s1, &c1);
    sincospi(2.0 * u4, &s2, &c2);
    v[3 * i] = r1 * c1;
    v[3 * i + 1] = r1 * s1;
    v[3 * i + 2] = r2 * c2;
}

__global__ void k_step_inc(unsigned long long *step) { *step += 1; }

}  // namespace

struct qem_batch {
    int B = 0, Ntot = 0, device = 0;
    std::vector<qem_handle *> h;
    std::vector<int> N, off;
    int W = 1;                          // stream-pool width in use
    std::vector<cudaStream_t> pool;     // up to min(B, 128) streams
    std::vector<cudaEvent_t> ev_done;
    cudaEvent_t ev_start = nullptr;
    cudaStream_t cap = nullptr;         // private stream the graphs are recorded on
    bool warm = false;
    uint32_t warm_terms = 0;
    int *sys = nullptr;                 // particle -> system
    double *box = nullptr;              // (Lx, Ly) per system
    double *Fn = nullptr;               // forces at the new positions (MD)
    cudaGraphExec_t md_exec = nullptr;  // one recorded MD step
    const void *md_key[4] = {nullptr, nullptr, nullptr, nullptr};
    double md_dt = 0;
    uint32_t md_terms = 0;
    int md_W = 0;
    // Andersen thermostat of the MD steps (off while therm_nu == 0)
    double therm_kT = 0, therm_nu = 0;
    uint64_t therm_seed = 0;
    unsigned long long *therm_step = nullptr;  // device step counter of the random draws
    // fused phases
    int mode_req = QEM_BATCH_AUTO;      // requested: auto, fused or pool
    int mode_cur = QEM_BATCH_FUSED;     // in use when the request is auto (the autotuner's choice)
    int fks = 0;                        // k-slices per system of the fused force pass (0: each handle's own)
    int forder = 0;                     // work-list order: 0 batch order, 1 largest system first
    int flch = 0;                       // chunk length of the fused k-space passes (0: qem_long_chunk())
    bool ftab_ok = false;               // device tables built for the current buffers and terms
    std::string fwhy;                   // why the batch cannot run fused (empty: it can)
    bool fneed_warm = false;            // a system needs a synchronous call before the tables can be built
    bool rewarming = false;             // inside the one re-sizing pass of a batch call
    std::vector<uint64_t> fstate;       // per-handle state the tables were built for
    uint32_t fterms = 0;
    int do_lj = 0;
    BatchSys *d_sys = nullptr;
    ShortConsts *d_sc = nullptr;
    BatchWork *d_work = nullptr;
    size_t work_cap = 0;
    // work lists: pairs, particle tiles, totals, scan, force pass, merge passes 0 and 1, cell tiles,
    // z-order tiles
    int nw[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, wo[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    int launches = 0;                   // kernels per fused evaluation
    cudaStream_t s_long = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    std::string err;
};

static qem_status bfail(qem_batch *b, qem_status s, const std::string &m)
{
    b->err = m;
    return s;
}

#define BCU(call)                                                                                \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess) return bfail(b, QEM_ERR_CUDA, std::string(#call) + " -> " + cudaGetErrorString(e_)); \
    } while (0)

static bool fused_current(const qem_batch *b, uint32_t terms)
{
    if (!b->ftab_ok || b->fterms != terms) return false;
    for (int i = 0; i < b->B; i++)
        if (qem_handle_state(b->h[i]) != b->fstate[i]) return false;
    return true;
}

static bool use_fused(const qem_batch *b)
{
    if (b->mode_req == QEM_BATCH_POOL || !b->fwhy.empty()) return false;
    return b->mode_req == QEM_BATCH_FUSED || b->mode_cur == QEM_BATCH_FUSED;
}

// Device tables of the fused phases from the handles' buffers (after their
// synchronous calls); outside any stream capture.  A system that does not
// qualify leaves the reason in fwhy and the batch on the stream pool.
static qem_status build_fused(qem_batch *b, uint32_t terms)
{
    b->ftab_ok = false;
    b->fneed_warm = false;
    b->fwhy.clear();
    if ((terms & (QEM_TERM_SHORT | QEM_TERM_LONG)) != (QEM_TERM_SHORT | QEM_TERM_LONG)) {
        b->fwhy = "terms without both the short and the long range";
        return QEM_OK;
    }
    std::vector<BatchSys> sys(b->B);
    std::vector<ShortConsts> sc(b->B);
    for (int i = 0; i < b->B; i++) {
        const char *why = nullptr;
        const qem_status st = qem_handle_batch_sys(b->h[i], b->N[i], b->fks, b->flch, &sys[i], &sc[i], &why);
        if (st == QEM_ERR_NO_KSET && why) {  // the caller changed the handle: size every system again
            b->fneed_warm = true;
            b->fwhy = "system " + std::to_string(i) + ": " + why;
            return QEM_OK;
        }
        if (st == QEM_ERR_ARG && why) {
            b->fwhy = "system " + std::to_string(i) + ": " + why;
            return QEM_OK;
        }
        if (st != QEM_OK) return bfail(b, st, "system " + std::to_string(i) + ": " + qem_handle_error(b->h[i]));
        sys[i].off = b->off[i];
    }
    std::vector<int> order(b->B);
    for (int i = 0; i < b->B; i++) order[i] = i;
    if (b->forder == 1)
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return b->N[x] > b->N[y]; });
    auto nblk = [](int64_t n, int t) { return (int)((n + t - 1) / t); };
    std::vector<BatchWork> w;
    const int tp = qem_batch_pair_tile(), tpart = qem_batch_particle_tile(), tt = qem_batch_ltot_tile();
    const int ts = qem_batch_lscan_tile(), tf = qem_batch_lforce_tile();
    if (tp != 256 || tpart != 256)
        return bfail(b, QEM_ERR_ARG, "the list phases take pair and particle tiles of 256");
    const int tz = qem_batch_ztile();
    for (int ph = 0; ph < 9; ph++) {
        b->wo[ph] = (int)w.size();
        for (int s : order) {
            const BatchSys &d = sys[s];
            if (ph == 0)
                for (int t = 0; t < nblk(d.cap, tp); t++) w.push_back({s, t, 0, 0});
            if (ph == 1)
                for (int t = 0; t < nblk(d.N, tpart); t++) w.push_back({s, t, 0, 0});
            if (ph == 2 && d.P > 0)
                for (int c = 0; c < d.nch; c++)
                    for (int kb = 0; kb < nblk(d.P, tt); kb++) w.push_back({s, c, kb, 0});
            if (ph == 3 && d.P > 0)
                for (int t = 0; t < nblk(d.P, ts); t++) w.push_back({s, t, 0, 0});
            if (ph == 4)  // also with P = 0: the force pass writes the zero slices the final pass sums
                for (int c = 0; c < d.nch; c++)
                    for (int y = 0; y < nblk(d.ks, tf); y++) w.push_back({s, c, y, 0});
            if ((ph == 5 || ph == 6) && qem_batch_zsort_passes(d.N) > ph - 5)
                for (int t = 0; t < nblk(d.N, 256); t++) w.push_back({s, t, 0, 0});
            if (ph == 7)
                for (int t = 0; t < nblk(d.ncell, 256); t++) w.push_back({s, t, 0, 0});
            if (ph == 8)
                for (int t = 0; t < nblk(d.N, tz); t++) w.push_back({s, t, 0, 0});
        }
        b->nw[ph] = (int)w.size() - b->wo[ph];
    }
    for (int i = 0; i < b->B; i++)
        if (qem_batch_zsort_passes(b->N[i]) > 2) return bfail(b, QEM_ERR_ARG, "more z-merge passes than two");
    b->launches = 16 + (b->nw[5] > 0) + (b->nw[6] > 0);
    if (!b->d_sys) {
        BCU(cudaMalloc(&b->d_sys, sizeof(BatchSys) * b->B));
        BCU(cudaMalloc(&b->d_sc, sizeof(ShortConsts) * b->B));
    }
    if (w.size() > b->work_cap) {
        if (b->d_work) BCU(cudaFree(b->d_work));
        b->d_work = nullptr;
        b->work_cap = w.size() + w.size() / 4;
        BCU(cudaMalloc(&b->d_work, sizeof(BatchWork) * b->work_cap));
    }
    BCU(cudaDeviceSynchronize());  // no recorded evaluation may still read the tables
    BCU(cudaMemcpy(b->d_sys, sys.data(), sizeof(BatchSys) * b->B, cudaMemcpyHostToDevice));
    BCU(cudaMemcpy(b->d_sc, sc.data(), sizeof(ShortConsts) * b->B, cudaMemcpyHostToDevice));
    BCU(cudaMemcpy(b->d_work, w.data(), sizeof(BatchWork) * w.size(), cudaMemcpyHostToDevice));
    b->fstate.resize(b->B);
    for (int i = 0; i < b->B; i++) b->fstate[i] = qem_handle_state(b->h[i]);
    b->fterms = terms;
    b->do_lj = (terms & QEM_TERM_LJ) ? 1 : 0;
    b->ftab_ok = true;
    return QEM_OK;
}

// the fused phases (tables current), forked from and joined to s
static qem_status enqueue_fused(qem_batch *b, const double *xyz, const double *q, double *F, cudaStream_t s)
{
    const BatchWork *w = b->d_work;
    BCU(qem_launch_batch_pack_ztile(b->nw[8], w + b->wo[8], b->d_sys, xyz, q, s));
    BCU(cudaEventRecord(b->ev_fork, s));
    BCU(cudaStreamWaitEvent(b->s_long, b->ev_fork, 0));
    for (int pass = 0; pass < 2; pass++)
        BCU(qem_launch_batch_zmerge(b->nw[5 + pass], w + b->wo[5 + pass], b->d_sys, pass, b->s_long));
    BCU(qem_launch_batch_lprep(b->B, b->d_sys, b->s_long));
    BCU(qem_launch_batch_ltot(b->nw[2], w + b->wo[2], b->d_sys, b->s_long));
    BCU(qem_launch_batch_lscan(b->nw[3], w + b->wo[3], b->d_sys, b->s_long));
    BCU(qem_launch_batch_lforce(b->nw[4], w + b->wo[4], b->d_sys, b->s_long));
    BCU(qem_launch_batch_lfinal(b->nw[1], w + b->wo[1], b->d_sys, b->s_long));
    BCU(cudaEventRecord(b->ev_join, b->s_long));
    BCU(qem_launch_batch_lists(b->B, w + b->wo[7], b->nw[7], w + b->wo[1], b->nw[1], w + b->wo[0], b->nw[0],
                               b->d_sys, s));
    BCU(qem_launch_batch_pairs(b->nw[0], w + b->wo[0], b->d_sys, b->d_sc, s));
    BCU(cudaStreamWaitEvent(s, b->ev_join, 0));
    BCU(qem_launch_batch_gather(b->nw[1], w + b->wo[1], b->d_sys, b->d_sc, b->do_lj, F, s));
    return QEM_OK;
}

// every system's evaluation: the fused phases when their tables are current,
// else the per-system pipelines on the pool, forked from and joined to s
static qem_status enqueue_forces(qem_batch *b, const double *xyz, const double *q, double *F, uint32_t terms,
                                 cudaStream_t s)
{
    if (use_fused(b)) {
        if (!fused_current(b, terms))
            return bfail(b, QEM_ERR_ARG, "fused batch tables out of date (a synchronous batch call first)");
        return enqueue_fused(b, xyz, q, F, s);
    }
    BCU(cudaEventRecord(b->ev_start, s));
    for (int w = 0; w < b->W; w++) BCU(cudaStreamWaitEvent(b->pool[w], b->ev_start, 0));
    for (int i = 0; i < b->B; i++) {
        const size_t o = (size_t)b->off[i];
        const qem_status st =
            qem_forces_async(b->h[i], b->N[i], xyz + 3 * o, q + o, F + 3 * o, terms, b->pool[i % b->W]);
        if (st != QEM_OK)
            return bfail(b, st, "system " + std::to_string(i) + ": " + qem_handle_error(b->h[i]));
    }
    for (int w = 0; w < b->W; w++) {
        BCU(cudaEventRecord(b->ev_done[w], b->pool[w]));
        BCU(cudaStreamWaitEvent(s, b->ev_done[w], 0));
    }
    return QEM_OK;
}

static void drop_md_graph(qem_batch *b)
{
    if (b->md_exec) cudaGraphExecDestroy(b->md_exec);
    b->md_exec = nullptr;
}

extern "C" {

qem_status qem_batch_create(int32_t B, qem_handle *const *handles, const int32_t *N, qem_batch **out)
{
    if (!out || B <= 0 || !handles || !N || !handles[0]) return QEM_ERR_ARG;
    *out = nullptr;
    qem_batch *b = new qem_batch();
    b->B = B;
    b->device = qem_handle_params(handles[0])->device;
    int64_t tot = 0;
    for (int i = 0; i < B; i++) {
        if (!handles[i] || N[i] < 0 || qem_handle_params(handles[i])->device != b->device) {
            delete b;
            return QEM_ERR_ARG;
        }
        b->h.push_back(handles[i]);
        b->N.push_back(N[i]);
        b->off.push_back((int)tot);
        tot += N[i];
    }
    if (tot > (1 << 30)) {
        delete b;
        return QEM_ERR_ARG;
    }
    b->Ntot = (int)tot;
    // the systems run concurrently on the stream pool and fill the GPU
    // together, so each keeps few k-slices (fewer force partials to write
    // and sum per system)
    for (qem_handle *hh : b->h) qem_handle_set_long_max_ks(hh, 8);
    if (cudaSetDevice(b->device) != cudaSuccess) {
        delete b;
        return QEM_ERR_CUDA;
    }
    const int np = std::min(B, 128);
    bool ok = cudaEventCreateWithFlags(&b->ev_start, cudaEventDisableTiming) == cudaSuccess;
    ok = ok && cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking) == cudaSuccess;
    int prio_lo = 0, prio_hi = 0;
    ok = ok && cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi) == cudaSuccess;
    ok = ok && cudaStreamCreateWithPriority(&b->s_long, cudaStreamNonBlocking, prio_hi) == cudaSuccess;
    ok = ok && cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming) == cudaSuccess;
    ok = ok && cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming) == cudaSuccess;
    for (int w = 0; ok && w < np; w++) {
        cudaStream_t s;
        cudaEvent_t e;
        ok = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) == cudaSuccess;
        if (ok) b->pool.push_back(s);
        ok = ok && cudaEventCreateWithFlags(&e, cudaEventDisableTiming) == cudaSuccess;
        if (ok) b->ev_done.push_back(e);
    }
    std::vector<int> sys(std::max(b->Ntot, 1));
    std::vector<double> box(2 * B);
    for (int i = 0; i < B; i++) {
        for (int k = 0; k < N[i]; k++) sys[b->off[i] + k] = i;
        box[2 * i] = qem_handle_params(handles[i])->Lx;
        box[2 * i + 1] = qem_handle_params(handles[i])->Ly;
    }
    ok = ok && cudaMalloc(&b->sys, sizeof(int) * sys.size()) == cudaSuccess;
    ok = ok && cudaMalloc(&b->box, sizeof(double) * box.size()) == cudaSuccess;
    ok = ok && cudaMalloc(&b->Fn, sizeof(double) * 3 * std::max(b->Ntot, 1)) == cudaSuccess;
    ok = ok && cudaMemcpy(b->sys, sys.data(), sizeof(int) * sys.size(), cudaMemcpyHostToDevice) == cudaSuccess;
    ok = ok && cudaMemcpy(b->box, box.data(), sizeof(double) * box.size(), cudaMemcpyHostToDevice) == cudaSuccess;
    if (!ok) {
        qem_batch_destroy(b);
        return QEM_ERR_CUDA;
    }
    b->W = np;
    *out = b;
    return QEM_OK;
}

void qem_batch_destroy(qem_batch *b)
{
    if (!b) return;
    cudaSetDevice(b->device);
    drop_md_graph(b);
    for (cudaStream_t s : b->pool) {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
    }
    for (cudaEvent_t e : b->ev_done) cudaEventDestroy(e);
    if (b->ev_start) cudaEventDestroy(b->ev_start);
    if (b->cap) cudaStreamDestroy(b->cap);
    if (b->sys) cudaFree(b->sys);
    if (b->box) cudaFree(b->box);
    if (b->Fn) cudaFree(b->Fn);
    if (b->therm_step) cudaFree(b->therm_step);
    if (b->s_long) {
        cudaStreamSynchronize(b->s_long);
        cudaStreamDestroy(b->s_long);
    }
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    if (b->ev_join) cudaEventDestroy(b->ev_join);
    if (b->d_sys) cudaFree(b->d_sys);
    if (b->d_sc) cudaFree(b->d_sc);
    if (b->d_work) cudaFree(b->d_work);
    delete b;
}

const char *qem_batch_last_error(const qem_batch *b) { return b ? b->err.c_str() : "NULL batch"; }

// A handle changed since the last sizing pass (its k-set or size): wait for
// any work already enqueued, then size every system again, once.
static qem_status rewarm(qem_batch *b, const double *xyz, const double *q, double *F, uint32_t terms, void *stream)
{
    BCU(cudaDeviceSynchronize());
    b->warm = false;
    b->rewarming = true;
    const qem_status st = qem_batch_forces(b, xyz, q, F, terms, stream);
    b->rewarming = false;
    return st;
}

qem_status qem_batch_forces(qem_batch *b, const double *xyz, const double *q, double *F, uint32_t terms,
                            void *stream)
{
    if (!b || !xyz || !q || !F || (terms & ~QEM_TERM_ALL)) return b ? bfail(b, QEM_ERR_ARG, "bad argument") : QEM_ERR_ARG;
    BCU(cudaSetDevice(b->device));
    cudaStream_t s = (cudaStream_t)stream;
    if (!b->warm || b->warm_terms != terms) {
        // size every system's buffers and upload its k-set (synchronous)
        for (int i = 0; i < b->B; i++) {
            const size_t o = (size_t)b->off[i];
            const qem_status st =
                qem_forces(b->h[i], b->N[i], xyz + 3 * o, q + o, F + 3 * o, nullptr, terms, QEM_MEM_DEVICE, s);
            if (st != QEM_OK) return bfail(b, st, "system " + std::to_string(i) + ": " + qem_handle_error(b->h[i]));
        }
        b->warm = true;
        b->warm_terms = terms;
        drop_md_graph(b);
        if (b->mode_req == QEM_BATCH_POOL) return QEM_OK;
        const qem_status st = build_fused(b, terms);
        if (st == QEM_OK && b->mode_req == QEM_BATCH_FUSED && !b->fwhy.empty())
            return bfail(b, QEM_ERR_ARG, "fused batch: " + b->fwhy);
        return st;
    }
    if (use_fused(b) && !fused_current(b, terms)) {
        drop_md_graph(b);
        const qem_status st = build_fused(b, terms);
        if (st != QEM_OK) return st;
        if (b->fneed_warm && !b->rewarming) return rewarm(b, xyz, q, F, terms, stream);
    }
    if (b->mode_req == QEM_BATCH_FUSED && !b->fwhy.empty()) return bfail(b, QEM_ERR_ARG, "fused batch: " + b->fwhy);
    const qem_status st = enqueue_forces(b, xyz, q, F, terms, s);
    if (st == QEM_ERR_NO_KSET && !b->rewarming) return rewarm(b, xyz, q, F, terms, stream);
    return st;
}

qem_status qem_batch_check(qem_batch *b, void *stream)
{
    if (!b) return QEM_ERR_ARG;
    BCU(cudaSetDevice(b->device));
    cudaStream_t s = (cudaStream_t)stream;
    BCU(cudaStreamSynchronize(s));
    for (int i = 0; i < b->B; i++) {
        const qem_status st = qem_status_check(b->h[i], s);
        if (st == QEM_ERR_NB_OVERFLOW) {  // the next batch call re-sizes every system synchronously
            b->warm = false;
            b->ftab_ok = false;
            drop_md_graph(b);
        }
        if (st != QEM_OK) return bfail(b, st, "system " + std::to_string(i) + ": " + qem_handle_error(b->h[i]));
    }
    b->err.clear();
    return QEM_OK;
}

qem_status qem_batch_md(qem_batch *b, int32_t nsteps, double dt, double *xyz, double *v, const double *q, double *F,
                        uint32_t terms, void *stream)
{
    if (!b || nsteps < 0 || !xyz || !v || !q || !F || !(dt == dt)) return b ? bfail(b, QEM_ERR_ARG, "bad argument") : QEM_ERR_ARG;
    BCU(cudaSetDevice(b->device));
    cudaStream_t s = (cudaStream_t)stream;
    // forces at the initial positions (sizes the buffers on the first call)
    qem_status st = qem_batch_forces(b, xyz, q, F, terms, s);
    if (st != QEM_OK) return st;
    if (b->warm_terms != terms) return bfail(b, QEM_ERR_ARG, "terms changed");
    const void *key[4] = {xyz, v, q, F};
    if (b->md_exec && (!std::equal(key, key + 4, b->md_key) || b->md_dt != dt || b->md_terms != terms || b->md_W != b->W))
        drop_md_graph(b);
    if (!b->md_exec && nsteps > 0) {
        const int n = b->Ntot, T = 256;
        // recorded on the batch's own stream (the caller's may be the legacy
        // default stream, which cannot be captured) and launched on s
        cudaStream_t c = b->cap;
        cudaGraph_t g = nullptr;
        BCU(cudaStreamSynchronize(s));
        BCU(cudaStreamBeginCapture(c, cudaStreamCaptureModeThreadLocal));
        k_vv_drift<<<(n + T - 1) / T, T, 0, c>>>(n, xyz, v, F, dt, b->sys, b->box);
        st = enqueue_forces(b, xyz, q, b->Fn, terms, c);
        k_vv_kick<<<(3 * n + T - 1) / T, T, 0, c>>>(3 * n, v, F, b->Fn, dt);
        if (b->therm_nu > 0) {
            k_andersen<<<(n + T - 1) / T, T, 0, c>>>(n, v, std::min(1.0, b->therm_nu * dt), sqrt(b->therm_kT),
                                                     b->therm_seed, b->therm_step);
            k_step_inc<<<1, 1, 0, c>>>(b->therm_step);
        }
        const cudaError_t ec = cudaStreamEndCapture(c, &g);
        if (st != QEM_OK) {
            if (g) cudaGraphDestroy(g);
            return st;
        }
        if (ec != cudaSuccess) return bfail(b, QEM_ERR_CUDA, std::string("stream capture: ") + cudaGetErrorString(ec));
        const cudaError_t ei = cudaGraphInstantiate(&b->md_exec, g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) {
            b->md_exec = nullptr;
            return bfail(b, QEM_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ei));
        }
        std::copy(key, key + 4, b->md_key);
        b->md_dt = dt;
        b->md_terms = terms;
        b->md_W = b->W;
    }
    for (int k = 0; k < nsteps; k++) BCU(cudaGraphLaunch(b->md_exec, s));
    return qem_batch_check(b, stream);
}

qem_status qem_batch_set_thermostat(qem_batch *b, double kT, double nu, uint64_t seed)
{
    if (!b) return QEM_ERR_ARG;
    if (!(kT >= 0) || !(nu >= 0) || !std::isfinite(kT) || !std::isfinite(nu))
        return bfail(b, QEM_ERR_ARG, "thermostat: kT and nu must be finite and >= 0");
    BCU(cudaSetDevice(b->device));
    BCU(cudaDeviceSynchronize());  // no recorded MD step may still be using the counter
    if (!b->therm_step) BCU(cudaMalloc(&b->therm_step, sizeof(unsigned long long)));
    BCU(cudaMemset(b->therm_step, 0, sizeof(unsigned long long)));
    BCU(cudaDeviceSynchronize());
    b->therm_kT = kT;
    b->therm_nu = kT > 0 ? nu : 0;
    b->therm_seed = seed;
    drop_md_graph(b);
    b->err.clear();
    return QEM_OK;
}

qem_status qem_batch_thermostat_step(const qem_batch *b, uint64_t *step)
{
    if (!b || !step) return QEM_ERR_ARG;
    *step = 0;
    if (!b->therm_step) return QEM_OK;
    unsigned long long v = 0;
    if (cudaSetDevice(b->device) != cudaSuccess ||
        cudaMemcpy(&v, b->therm_step, sizeof(v), cudaMemcpyDeviceToHost) != cudaSuccess)
        return QEM_ERR_CUDA;
    *step = v;
    return QEM_OK;
}

// one batch evaluation recorded as a graph and replayed reps times on s
// (after one warm-up replay): milliseconds per evaluation
static qem_status time_graph(qem_batch *b, const double *xyz, const double *q, double *F, uint32_t terms,
                             cudaStream_t s, cudaEvent_t t0, cudaEvent_t t1, float &ms)
{
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ex = nullptr;
    BCU(cudaStreamSynchronize(s));
    BCU(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal));
    const qem_status st = enqueue_forces(b, xyz, q, F, terms, b->cap);
    const cudaError_t ec = cudaStreamEndCapture(b->cap, &g);
    if (st != QEM_OK || ec != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return st != QEM_OK ? st : bfail(b, QEM_ERR_CUDA, std::string("stream capture: ") + cudaGetErrorString(ec));
    }
    const cudaError_t ei = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) return bfail(b, QEM_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ei));
    const int reps = 5;
    cudaError_t e = cudaGraphLaunch(ex, s);
    e = e == cudaSuccess ? cudaEventRecord(t0, s) : e;
    for (int r = 0; r < reps && e == cudaSuccess; r++) e = cudaGraphLaunch(ex, s);
    e = e == cudaSuccess ? cudaEventRecord(t1, s) : e;
    e = e == cudaSuccess ? cudaEventSynchronize(t1) : e;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, t0, t1);
    cudaGraphExecDestroy(ex);
    if (e != cudaSuccess) return bfail(b, QEM_ERR_CUDA, std::string("autotune timing: ") + cudaGetErrorString(e));
    ms /= reps;
    return QEM_OK;
}

qem_status qem_batch_autotune(qem_batch *b, const double *xyz, const double *q, double *F, uint32_t terms,
                              void *stream, int32_t *width, double *ms_per_eval)
{
    if (!b) return QEM_ERR_ARG;
    BCU(cudaSetDevice(b->device));
    cudaStream_t s = (cudaStream_t)stream;
    qem_status st = qem_batch_forces(b, xyz, q, F, terms, s);
    if (st != QEM_OK) return st;
    // candidates: pool widths 1, 2, 4, ..; fused tilings: k-slices per system
    // of the force pass (the handle's own count, or at most 1, 2, 4) x
    // work-list order (batch order, largest system first)
    struct Cand {
        int fused, w, ks, order, lch;
    };
    std::vector<Cand> cand;
    if (b->mode_req != QEM_BATCH_FUSED) {
        const int wmax = (int)b->pool.size();
        for (int w = 1; w < wmax; w *= 2) cand.push_back({0, w, 0, 0, 0});
        cand.push_back({0, wmax, 0, 0, 0});
    }
    const bool fusable = b->mode_req != QEM_BATCH_POOL && b->fwhy.empty();
    if (fusable)
        for (int lch : {0, 256, 128, 64})
            for (int ks : {0, 2, 4})
                for (int order : {0, 1}) cand.push_back({1, 0, ks, order, lch});
    const int mode0 = b->mode_req, W0 = b->W, ks0 = b->fks, order0 = b->forder, lch0 = b->flch;
    cudaEvent_t t0, t1;
    BCU(cudaEventCreate(&t0));
    BCU(cudaEventCreate(&t1));
    int best = -1;
    float best_ms = 1e30f;
    for (int c = 0; c < (int)cand.size() && st == QEM_OK; c++) {
        const Cand &k = cand[c];
        b->mode_req = k.fused ? QEM_BATCH_FUSED : QEM_BATCH_POOL;
        if (k.fused) {
            b->fks = k.ks;
            b->forder = k.order;
            b->flch = k.lch;
            st = build_fused(b, terms);
        } else {
            b->W = k.w;
        }
        float ms = 0;
        if (st == QEM_OK) st = time_graph(b, xyz, q, F, terms, s, t0, t1, ms);
        if (st == QEM_OK && ms < best_ms) {
            best_ms = ms;
            best = c;
        }
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    b->mode_req = mode0;
    b->W = W0;
    b->fks = ks0;
    b->forder = order0;
    b->flch = lch0;
    if (st == QEM_OK && best >= 0) {
        const Cand &k = cand[best];
        if (k.fused) {
            b->fks = k.ks;
            b->forder = k.order;
            b->flch = k.lch;
            b->mode_cur = QEM_BATCH_FUSED;
        } else {
            b->W = k.w;
            b->mode_cur = QEM_BATCH_POOL;
        }
    }
    if (fusable) {
        const qem_status sb = build_fused(b, terms);
        if (st == QEM_OK) st = sb;
    }
    drop_md_graph(b);
    if (st != QEM_OK) return st;
    if (width) *width = b->mode_cur == QEM_BATCH_FUSED ? 0 : b->W;
    if (ms_per_eval) *ms_per_eval = best_ms;
    return qem_batch_check(b, stream);
}

qem_status qem_batch_set_mode(qem_batch *b, int32_t mode, int32_t ks, int32_t order, int32_t chunk)
{
    if (!b) return QEM_ERR_ARG;
    if (mode != QEM_BATCH_AUTO && mode != QEM_BATCH_FUSED && mode != QEM_BATCH_POOL)
        return bfail(b, QEM_ERR_ARG, "mode must be QEM_BATCH_AUTO, QEM_BATCH_FUSED or QEM_BATCH_POOL");
    if (ks < 0 || ks > QEM_LONG_MAX_KS || (order != 0 && order != 1))
        return bfail(b, QEM_ERR_ARG, "ks must be in 0 .. 64 and order 0 or 1");
    if (chunk != 0 && (chunk < 32 || qem_long_chunk() % chunk != 0))
        return bfail(b, QEM_ERR_ARG, "chunk must be 0 or a divisor of 512 of at least 32");
    BCU(cudaSetDevice(b->device));
    BCU(cudaDeviceSynchronize());
    b->mode_req = mode;
    b->mode_cur = mode == QEM_BATCH_POOL ? QEM_BATCH_POOL : QEM_BATCH_FUSED;
    b->fks = ks;
    b->forder = order;
    b->flch = chunk;
    b->ftab_ok = false;  // rebuilt by the next qem_batch_forces
    drop_md_graph(b);
    b->err.clear();
    return QEM_OK;
}

qem_status qem_batch_get_mode(const qem_batch *b, int32_t *mode, int32_t *ks, int32_t *order, int32_t *chunk,
                              int32_t *launches, const char **why)
{
    if (!b) return QEM_ERR_ARG;
    const bool fused = use_fused(b);
    if (mode) *mode = fused ? QEM_BATCH_FUSED : QEM_BATCH_POOL;
    if (ks) *ks = b->fks;
    if (order) *order = b->forder;
    if (chunk) *chunk = b->flch > 0 ? b->flch : qem_long_chunk();
    if (launches) *launches = fused ? b->launches : -1;
    if (why) *why = b->fwhy.c_str();
    return QEM_OK;
}

}  // extern "C"

// qem_bin.cu -- in-plane cell binning, pair list and z order.
//
// Replaces the neighbour machinery of the reference:
//   CellListMap.neighborlist(xy, r_cutoff; unitcell)   QEM_short.jl:34-35
//   Q2d_neighbor / update_neighbor                     Q2d_neighbor.jl:10-30
//   sortperm(z) / bulket_sorting                       QEM_long.jl:39-40, bulket_sorting.jl:4-10
//
// Everything here is integer/byte work bound by memory latency and bandwidth;
// the outputs are deterministic: cells list their particles in ascending
// index, pairs are emitted in (cell order of i, stencil order, cell order of
// j), the incoming lists are sorted by pair index, and the z order is the
// stable ascending order of (z, index) -- identical to Julia's sortperm.
#include "qem_internal.cuh"

namespace {

constexpr int SCAN_BLOCK = 1024;

// ---------------------------------------------------------------------------
// pack: AoS coordinates + charges -> double4, 2-D cell index, finiteness check
// ---------------------------------------------------------------------------
// returns the z it stored (0 for non-finite input)
__device__ __forceinline__ double pack_one(int i, const double *__restrict__ xyz, const double *__restrict__ q,
                                           double4 *__restrict__ pos, int *__restrict__ cell, const CellGeom &g,
                                           unsigned *status)
{
    double x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2], qq = q[i];
    bool ok = isfinite(x) && isfinite(y) && isfinite(z) && isfinite(qq);
    if (!ok) {
        atomicOr(status, QEM_ST_NONFINITE);
        x = 0; y = 0; z = 0; qq = 0;
    }
    pos[i] = make_double4(x, y, z, qq);
    double xw = x - g.Lx * floor(x * g.invLx);
    double yw = y - g.Ly * floor(y * g.invLy);
    int cx = (int)(xw * g.inv_lcx), cy = (int)(yw * g.inv_lcy);
    cx = min(max(cx, 0), g.ncx - 1);
    cy = min(max(cy, 0), g.ncy - 1);
    cell[i] = cx * g.ncy + cy;
    return z;
}

__global__ void k_pack(int N, const double *__restrict__ xyz, const double *__restrict__ q, double4 *__restrict__ pos,
                       int *__restrict__ cell, CellGeom g, unsigned *status)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) pack_one(i, xyz, q, pos, cell, g, status);
}

// ---------------------------------------------------------------------------
// exclusive scans (block scan + scan of block sums + add); out[n] = total
// ---------------------------------------------------------------------------
template <typename TI, typename TO>
__global__ void k_scan_block(const TI *__restrict__ in, TO *__restrict__ out, int n, TO *__restrict__ bsum)
{
    __shared__ TO warp_tot[SCAN_BLOCK / 32];
    int i = blockIdx.x * SCAN_BLOCK + threadIdx.x;
    TO v = (i < n) ? (TO)in[i] : (TO)0;
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    TO x = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        TO t = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= d) x += t;
    }
    if (lane == 31) warp_tot[w] = x;
    __syncthreads();
    if (w == 0) {
        TO y = warp_tot[lane];
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            TO t = __shfl_up_sync(0xffffffffu, y, d);
            if (lane >= d) y += t;
        }
        warp_tot[lane] = y;  // inclusive over warps
    }
    __syncthreads();
    TO incl = x + (w > 0 ? warp_tot[w - 1] : (TO)0);
    if (i < n) out[i] = incl - v;  // exact for integers; for doubles see k_scan_block_excl
    if (threadIdx.x == SCAN_BLOCK - 1) bsum[blockIdx.x] = incl;
}

// exclusive scan of doubles without the "inclusive minus own" subtraction
__global__ void k_scan_block_excl_f64(const double *__restrict__ in, double *__restrict__ out, int n,
                                      double *__restrict__ bsum)
{
    __shared__ double warp_tot[SCAN_BLOCK / 32];
    int i = blockIdx.x * SCAN_BLOCK + threadIdx.x;
    double v = (i < n) ? in[i] : 0.0;
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    double x = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        double t = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= d) x += t;
    }
    double ex = __shfl_up_sync(0xffffffffu, x, 1);
    if (lane == 0) ex = 0.0;
    if (lane == 31) warp_tot[w] = x;
    __syncthreads();
    if (w == 0) {
        double y = warp_tot[lane];
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            double t = __shfl_up_sync(0xffffffffu, y, d);
            if (lane >= d) y += t;
        }
        double e = __shfl_up_sync(0xffffffffu, y, 1);
        if (lane == 0) e = 0.0;
        warp_tot[lane] = e;  // exclusive over warps
        if (lane == 31) bsum[blockIdx.x] = y;
    }
    __syncthreads();
    if (i < n) out[i] = warp_tot[w] + ex;
}

template <typename T>
__global__ void k_scan_top(T *bsum, int nb)
{
    // one block: exclusive scan of nb block sums in place, chunks of SCAN_BLOCK with a carry
    __shared__ T warp_tot[SCAN_BLOCK / 32];
    __shared__ T carry;
    if (threadIdx.x == 0) carry = (T)0;
    __syncthreads();
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int base = 0; base < nb; base += SCAN_BLOCK) {
        int i = base + threadIdx.x;
        T v = (i < nb) ? bsum[i] : (T)0;
        T x = v;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            T t = __shfl_up_sync(0xffffffffu, x, d);
            if (lane >= d) x += t;
        }
        T ex = __shfl_up_sync(0xffffffffu, x, 1);
        if (lane == 0) ex = (T)0;
        if (lane == 31) warp_tot[w] = x;
        __syncthreads();
        if (w == 0) {
            T y = warp_tot[lane];
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                T t = __shfl_up_sync(0xffffffffu, y, d);
                if (lane >= d) y += t;
            }
            T e = __shfl_up_sync(0xffffffffu, y, 1);
            if (lane == 0) e = (T)0;
            warp_tot[lane] = e;
        }
        __syncthreads();
        T c = carry;
        if (i < nb) bsum[i] = c + warp_tot[w] + ex;
        __syncthreads();
        if (threadIdx.x == SCAN_BLOCK - 1) carry = c + warp_tot[w] + x;
        __syncthreads();
    }
    if (threadIdx.x == 0) bsum[nb] = carry;  // grand total
}

template <typename T>
__global__ void k_scan_add(T *__restrict__ out, int n, const T *__restrict__ bsum)
{
    int i = blockIdx.x * SCAN_BLOCK + threadIdx.x;
    if (i < n) out[i] = bsum[blockIdx.x] + out[i];
    if (i == 0) out[n] = bsum[(n + SCAN_BLOCK - 1) / SCAN_BLOCK];
}

// One-block exclusive scan for small n (one launch instead of three; the
// many-small-systems batch and the binning chain in front of the pair kernel
// are launch-bound): thread t owns elements [t pt, (t + 1) pt),
// pt = ceil(n / SCAN_BLOCK) <= PT, summed in order; the thread totals are
// scanned exclusively without an "inclusive minus own" step; out[n] = total.
// Integer scans (exact in any order) take it up to 16 elements per thread,
// e.g. the 10^4 cells of a 1000 x 1000 slab with r_c = 10; FP64 scans keep
// 8, so their summation order at a given n is unchanged.
constexpr int SCAN_SMALL_PT = 8;
constexpr int SCAN_SMALL_MAX = SCAN_BLOCK * SCAN_SMALL_PT;
constexpr int SCAN_SMALL_PT_INT = 16;
constexpr int SCAN_SMALL_MAX_INT = SCAN_BLOCK * SCAN_SMALL_PT_INT;

template <typename TI, typename TO, int PT>
__global__ void __launch_bounds__(SCAN_BLOCK) k_scan_small(const TI *__restrict__ in, TO *__restrict__ out, int n)
{
    __shared__ TO warp_tot[SCAN_BLOCK / 32];
    qem_block_scan_excl_small<TI, TO, PT>(in, out, n, warp_tot);
}

// ---------------------------------------------------------------------------
// cell counting sort
// ---------------------------------------------------------------------------
__global__ void k_cell_count(int N, const int *__restrict__ cell, int *cnt)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) atomicAdd(&cnt[cell[i]], 1);
}

__global__ void k_cell_scatter(int N, const int *__restrict__ cell, int *fill, int *__restrict__ list)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) list[atomicAdd(&fill[cell[i]], 1)] = i;
}

// ascending order of up to 32 values held one per lane (bitonic network)
template <typename T>
__device__ __forceinline__ T warp_sort32(T v, int lane)
{
#pragma unroll
    for (int size = 2; size <= 32; size <<= 1) {
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            const T other = __shfl_xor_sync(0xffffffffu, v, stride);
            const bool up = ((lane & size) == 0) || size == 32;
            const bool lower = (lane & stride) == 0;
            v = (lower == up) ? (other < v ? other : v) : (other > v ? other : v);
        }
    }
    return v;
}

// one warp per segment [b, e): ascending order (segments longer than 32 fall
// back to an insertion sort by lane 0)
template <typename T>
__device__ __forceinline__ void warp_sort_segment(T *list, int64_t b, int64_t e, int lane, T pad)
{
    const int64_t n = e - b;
    if (n <= 1) return;
    if (n <= 32) {
        T v = lane < n ? list[b + lane] : pad;
        v = warp_sort32(v, lane);
        if (lane < n) list[b + lane] = v;
        return;
    }
    if (lane == 0) {
        for (int64_t s = b + 1; s < e; s++) {
            T v = list[s];
            int64_t t = s - 1;
            while (t >= b && list[t] > v) {
                list[t + 1] = list[t];
                t--;
            }
            list[t + 1] = v;
        }
    }
    __syncwarp();
}

// ascending particle index inside every cell (makes the slot order of the
// atomic scatter irrelevant), the inverse map particle -> sorted slot, and the
// positions in cell order; one warp per cell
__global__ void k_cell_sort(int ncell, const int *__restrict__ start, int *__restrict__ list, int *__restrict__ pos_of,
                            const double4 *__restrict__ pos, double4 *__restrict__ pos_c)
{
    const int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (c >= ncell) return;
    const int b = start[c], e = start[c + 1];
    warp_sort_segment<int>(list, b, e, lane, 0x7fffffff);
    __syncwarp();
    for (int s = b + lane; s < e; s += 32) {
        const int i = list[s];
        pos_of[i] = s;
        pos_c[s] = pos[i];
    }
}

// The whole cell build of a small system (N and ncell at most CELLS_SMALL) in
// one block: counts in shared memory, their scan, the atomic scatter, the
// ascending order inside every cell (one warp per cell, as k_cell_sort) and
// the cell-order positions.  The result is the same as the multi-kernel
// build (the order inside a cell does not depend on the scatter).
constexpr int CELLS_SMALL = 8192;

// SORT = false stops after the scatter (cstart and the unsorted cell lists)
template <bool SORT = true>
__device__ __forceinline__ void cells_small_block(int N, int ncell, const int *__restrict__ cell,
                                                  const double4 *__restrict__ pos, int *__restrict__ cstart,
                                                  int *__restrict__ clist, int *__restrict__ pos_of,
                                                  double4 *__restrict__ pos_c)
{
    __shared__ int cnt[CELLS_SMALL];
    __shared__ int warp_tot[32];
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    for (int c = tid; c < ncell; c += 1024) cnt[c] = 0;
    __syncthreads();
    for (int i = tid; i < N; i += 1024) atomicAdd(&cnt[cell[i]], 1);
    __syncthreads();
    // exclusive scan of cnt into cstart (thread t owns cells [t pt, (t + 1) pt)); cnt becomes the fill pointer
    const int pt = (ncell + 1023) / 1024, b = tid * pt;
    int tot = 0;
    for (int j = 0; j < pt; j++)
        if (b + j < ncell) tot += cnt[b + j];
    int x = tot;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= d) x += t;
    }
    if (lane == 31) warp_tot[w] = x;
    __syncthreads();
    if (w == 0) {
        int y = warp_tot[lane];
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, y, d);
            if (lane >= d) y += t;
        }
        warp_tot[lane] = y;  // inclusive over warps
    }
    __syncthreads();
    int run = x - tot + (w > 0 ? warp_tot[w - 1] : 0);  // exclusive start of this thread's cells
    for (int j = 0; j < pt; j++)
        if (b + j < ncell) {
            const int c = cnt[b + j];
            cstart[b + j] = run;
            cnt[b + j] = run;
            run += c;
        }
    if (tid == 1023) cstart[ncell] = warp_tot[31];
    __syncthreads();
    for (int i = tid; i < N; i += 1024) clist[atomicAdd(&cnt[cell[i]], 1)] = i;
    __syncthreads();
    if (!SORT) return;
    for (int c = w; c < ncell; c += 32) {
        const int cb = cstart[c], ce = cstart[c + 1];
        warp_sort_segment<int>(clist, cb, ce, lane, 0x7fffffff);
    }
    __syncthreads();
    for (int s = tid; s < N; s += 1024) {
        const int i = clist[s];
        pos_of[i] = s;
        pos_c[s] = pos[i];
    }
}

__global__ void __launch_bounds__(1024) k_cells_small(int N, int ncell, const int *__restrict__ cell,
                                                      const double4 *__restrict__ pos, int *__restrict__ cstart,
                                                      int *__restrict__ clist, int *__restrict__ pos_of,
                                                      double4 *__restrict__ pos_c)
{
    cells_small_block(N, ncell, cell, pos, cstart, clist, pos_of, pos_c);
}

// ---------------------------------------------------------------------------
// pair list (j > i, minimum-image rho^2 <= r_c^2)
// ---------------------------------------------------------------------------
// rho^2 with explicitly rounded operations so that the in/out decision is
// bit-identical to an unfused CPU evaluation of the same expression.  The
// image shift n = rint(d / L) is taken as rint(d * (1 / L)): the two differ
// only where d / L lies within rounding of +-1/2, i.e. |d| ~ L / 2 > r_c,
// where both shifts leave the pair out of range.
__device__ __forceinline__ double rho2_exact(double4 a, double4 b, const CellGeom &g)
{
    double dx = __dsub_rn(a.x, b.x), dy = __dsub_rn(a.y, b.y);
    dx = __dsub_rn(dx, __dmul_rn(g.Lx, rint(dx * g.invLx)));
    dy = __dsub_rn(dy, __dmul_rn(g.Ly, rint(dy * g.invLy)));
    return __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
}

__device__ __forceinline__ void stencil_range(int n, int &lo, int &hi)
{
    if (n >= 3) { lo = -1; hi = 1; }
    else if (n == 2) { lo = 0; hi = 1; }
    else { lo = 0; hi = 0; }
}

// pos_c: positions in cell order (pos_c[s] is particle clist[s]).  Pairs are
// stored as (owner, other) -- not ordered by index.  The fill pass writes at
// most cap pairs (QEM_ST_OVERFLOW beyond) and counts each pair's incoming
// entry for its second particle.
template <bool FILL>
__device__ __forceinline__ void pairs_of_owner(int t, const double4 *__restrict__ pos_c, const int *__restrict__ cell,
                                               const int *__restrict__ cstart, const int *__restrict__ clist,
                                               const CellGeom &g, double rc2, int *__restrict__ pcount,
                                               const int64_t *__restrict__ poff, int2 *__restrict__ pairs,
                                               int64_t cap, int *__restrict__ in_cnt, unsigned *status)
{
    int i = clist[t];
    double4 pi = pos_c[t];
    int c = cell[i];
    int cx = c / g.ncy, cy = c - cx * g.ncy;
    // Ownership: with at least 3 cells per direction the pair belongs to the
    // particle whose half stencil (own cell after it, plus the 4 forward
    // cells) contains the other one, so every cell pair is visited once and
    // incoming lists stay balanced; otherwise the full (deduplicated)
    // stencil with "later in cell order" ownership.
    const bool half = g.ncx >= 3 && g.ncy >= 3;
    int xlo, xhi, ylo, yhi;
    stencil_range(g.ncx, xlo, xhi);
    stencil_range(g.ncy, ylo, yhi);
    int cnt = 0;
    int64_t o = FILL ? poff[t] : 0;
    for (int ox = xlo; ox <= xhi; ox++) {
        int nx = cx + ox;
        nx = nx < 0 ? nx + g.ncx : (nx >= g.ncx ? nx - g.ncx : nx);
        for (int oy = ylo; oy <= yhi; oy++) {
            if (half && (ox < 0 || (ox == 0 && oy < 0))) continue;  // backward half of the stencil
            int ny = cy + oy;
            ny = ny < 0 ? ny + g.ncy : (ny >= g.ncy ? ny - g.ncy : ny);
            int cc = nx * g.ncy + ny;
            const bool same = (cc == c);
            int b = cstart[cc], e = cstart[cc + 1];
            for (int s = b; s < e; s++) {
                if ((same || !half) && s <= t) continue;
                int j = clist[s];
                if (rho2_exact(pi, pos_c[s], g) <= rc2) {
                    if (FILL) {
                        if (o + cnt < cap) {
                            pairs[o + cnt] = make_int2(i, j);
                            atomicAdd(&in_cnt[j], 1);
                        } else {
                            atomicOr(status, QEM_ST_OVERFLOW);
                        }
                    }
                    cnt++;
                }
            }
        }
    }
    if (!FILL) pcount[t] = cnt;
}

template <bool FILL>
__global__ void k_pairs(int N, const double4 *__restrict__ pos_c, const int *__restrict__ cell,
                        const int *__restrict__ cstart, const int *__restrict__ clist, CellGeom g, double rc2,
                        int *__restrict__ pcount, const int64_t *__restrict__ poff, int2 *__restrict__ pairs,
                        int64_t cap, int *__restrict__ in_cnt, unsigned *status)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < N) pairs_of_owner<FILL>(t, pos_c, cell, cstart, clist, g, rc2, pcount, poff, pairs, cap, in_cnt, status);
}

// ---------------------------------------------------------------------------
// pair list, at least 3 cells along x and y: one warp per owner cell
// ---------------------------------------------------------------------------
constexpr int PL_MAXB = QEM_PL_MAXB;  // candidate batches of 32 whose hit masks the count pass keeps
// The five cells of the half stencil in visiting order: own cell, then
// (0,+1), (+1,-1), (+1,0), (+1,+1) -- the order of k_pairs.
__device__ __forceinline__ void half_offset(int d, int &ox, int &oy)
{
    ox = d >= 2 ? 1 : 0;
    oy = d == 0 ? 0 : (d == 1 ? 1 : d - 3);
}

__device__ __forceinline__ int wrap_cell(int n, int m) { return n < 0 ? n + m : (n >= m ? n - m : n); }

// The lanes hold 32 consecutive candidates of the concatenated stencil cells
// and the warp walks the cell's owners in order: a ballot per owner gives
// each hit its pair index (the owner's next index plus the hits of lower
// lanes), which reproduces k_pairs' order exactly, and each lane counts the
// hits on its candidate, i.e. the candidate's incoming entries from this
// owner cell in owner order.  The count pass stores, per owner, its number
// of pairs and, per (candidate, stencil direction), its number of incoming
// pairs from that owner cell (`in_slot`, indexed by cell-order position).
// k_in_base turns those into slot bases; the fill pass then writes every
// incoming entry straight to its final slot, so the incoming lists come out
// in ascending pair order without atomics or a sort.  A (candidate,
// direction) entry belongs to exactly one owner cell, hence to one warp, and
// owner blocks of more than 32 owners carry it over in place.  The count pass
// also keeps every owner's hit mask of its first PL_MAXB candidate batches
// (hmask[owner position * PL_MAXB + batch]), so the fill pass tests distances
// only in cells with more than 32 * PL_MAXB candidates.
template <bool FILL>
__global__ void __launch_bounds__(128) k_pairs_cell(int ncell, const double4 *__restrict__ pos_c,
                                                    const int *__restrict__ cstart, const int *__restrict__ clist,
                                                    CellGeom g, double rc2, int *__restrict__ pcount,
                                                    const int64_t *__restrict__ poff, int2 *__restrict__ pairs,
                                                    int64_t cap, int *__restrict__ in_slot,
                                                    const int64_t *__restrict__ in_off, int *__restrict__ in_list,
                                                    unsigned *status, unsigned *__restrict__ hmask)
{
    const int c = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (c >= ncell) return;  // c is the same for the whole warp
    const int cx = c / g.ncy, cy = c - cx * g.ncy;
    int sb[5], sl[5], tot = 0;
#pragma unroll
    for (int d = 0; d < 5; d++) {
        int ox, oy;
        half_offset(d, ox, oy);
        const int cc = wrap_cell(cx + ox, g.ncx) * g.ncy + wrap_cell(cy + oy, g.ncy);
        sb[d] = cstart[cc];
        sl[d] = cstart[cc + 1] - sb[d];
        tot += sl[d];
    }
    const int ob = sb[0], nown = sl[0];
    const unsigned below = (1u << lane) - 1u;
    // the count pass also visits an empty cell once, to zero its candidates' entries
    const int nblkown = nown > 0 ? (nown + 31) >> 5 : (FILL ? 0 : 1);
    for (int blk = 0; blk < nblkown; blk++) {
        const int o0 = ob + 32 * blk;
        const int no = max(0, min(32, ob + nown - o0));
        int my_i = 0, my_cnt = 0;
        int64_t my_next = 0;  // fill: pair index of this lane's owner's next pair
        if (lane < no) {
            my_i = clist[o0 + lane];
            if (FILL) my_next = poff[o0 + lane];
        }
        for (int v0 = 0; v0 < tot; v0 += 32) {
            const int v = v0 + lane;
            const int bt = v0 >> 5;  // candidate batch
            const bool stored = bt < PL_MAXB;
            unsigned my_mask = 0;    // lane k: owner k's hits in this batch
            if (FILL && stored && lane < no) my_mask = hmask[(size_t)(o0 + lane) * PL_MAXB + bt];
            int d = -1, s = 0;
            {
                int acc = 0;
#pragma unroll
                for (int k = 0; k < 5; k++) {
                    if (d < 0 && v < acc + sl[k]) {
                        d = k;
                        s = sb[k] + (v - acc);
                    }
                    acc += sl[k];
                }
            }
            const bool valid = d >= 0;
            double4 pj = make_double4(0.0, 0.0, 0.0, 0.0);
            int j = 0;
            int64_t slot = 0;
            if (valid) {
                pj = pos_c[s];
                j = clist[s];
                if (FILL) slot = in_off[j] + in_slot[(size_t)5 * s + d];
            }
            int r = 0;
            for (int k = 0; k < no; k++) {
                const int t = o0 + k;
                unsigned m;
                bool hit;
                if (FILL && stored) {
                    m = __shfl_sync(0xffffffffu, my_mask, k);
                    hit = (m >> lane) & 1u;
                } else {
                    hit = valid && (d != 0 || s > t) && rho2_exact(pos_c[t], pj, g) <= rc2;
                    m = __ballot_sync(0xffffffffu, hit);
                    if (!FILL && lane == k) my_mask = m;
                }
                if (FILL) {
                    const int64_t base = __shfl_sync(0xffffffffu, my_next, k);
                    const int io = __shfl_sync(0xffffffffu, my_i, k);
                    if (hit) {
                        const int64_t p = base + __popc(m & below);
                        if (p < cap) {
                            pairs[p] = make_int2(io, j);
                            if (slot + r < cap) in_list[slot + r] = (int)p;
                        } else {
                            atomicOr(status, QEM_ST_OVERFLOW);
                        }
                    }
                    if (lane == k) my_next += __popc(m);
                } else if (lane == k) {
                    my_cnt += __popc(m);
                }
                r += hit;
            }
            if (valid) {
                int &w = in_slot[(size_t)5 * s + d];
                w = (FILL || blk > 0) ? w + r : r;
            }
            if (!FILL && stored && lane < no) hmask[(size_t)(o0 + lane) * PL_MAXB + bt] = my_mask;
        }
        if (!FILL && lane < no) pcount[o0 + lane] = my_cnt;
    }
}

// Per cell-order position s of particle j: the owner cells of j's incoming
// pairs are the five cells j - offset(d); pair indices ascend with the owner's
// cell index, so ordering the five cells by index turns the per-direction
// counts into slot bases.  Also j's number of incoming pairs -- zero for
// every particle when the pairs do not fit the capacity (the evaluation is
// then repeated with a larger list), so that in_off[N] <= cap and every
// entry of in_list below in_off[N] names a stored pair.
__global__ void k_in_base(int N, const int *__restrict__ clist, const int *__restrict__ cell, CellGeom g,
                          const int64_t *__restrict__ np, int64_t cap, int *__restrict__ in_slot,
                          int *__restrict__ in_cnt, unsigned *status)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= N) return;
    const int j = clist[s];
    if (*np > cap) {
        in_cnt[j] = 0;
        if (s == 0) atomicOr(status, QEM_ST_OVERFLOW);
        return;
    }
    const int c = cell[j];
    const int cx = c / g.ncy, cy = c - cx * g.ncy;
    int cc[5], n[5], tot = 0;
#pragma unroll
    for (int d = 0; d < 5; d++) {
        int ox, oy;
        half_offset(d, ox, oy);
        cc[d] = wrap_cell(cx - ox, g.ncx) * g.ncy + wrap_cell(cy - oy, g.ncy);
        n[d] = in_slot[(size_t)5 * s + d];
        tot += n[d];
    }
#pragma unroll
    for (int d = 0; d < 5; d++) {
        int b = 0;
#pragma unroll
        for (int e = 0; e < 5; e++) b += cc[e] < cc[d] ? n[e] : 0;
        in_slot[(size_t)5 * s + d] = b;
    }
    in_cnt[j] = tot;
}

// ---------------------------------------------------------------------------
// incoming pairs per particle (CSR over the second index), sorted by pair id
// ---------------------------------------------------------------------------
// the pair count lives on the device (*np = poff[N]); grids are sized for
// the capacity and threads beyond the count return
__global__ void k_in_fill(const int64_t *__restrict__ np, int64_t cap, const int2 *__restrict__ pairs,
                          const int64_t *__restrict__ off, int *fill, int *__restrict__ list)
{
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= *np || p >= cap) return;
    const int j = pairs[p].y;
    list[off[j] + atomicAdd(&fill[j], 1)] = (int)p;
}

// ascending order of M register values (bitonic network; every index is a
// compile-time constant after unrolling, so the array stays in registers)
template <int M>
__device__ __forceinline__ void reg_sort(int (&v)[M])
{
#pragma unroll
    for (int size = 2; size <= M; size <<= 1) {
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
#pragma unroll
            for (int a = 0; a < M; a++) {
                const int b = a ^ stride;
                if (b > a) {
                    const bool up = (a & size) == 0;
                    const int x = v[a], y = v[b];
                    v[a] = up ? min(x, y) : max(x, y);
                    v[b] = up ? max(x, y) : min(x, y);
                }
            }
        }
    }
}

template <int M>
__device__ __forceinline__ void sort_small_segment(int *list, int64_t b, int n)
{
    int v[M];
#pragma unroll
    for (int k = 0; k < M; k++) v[k] = k < n ? list[b + k] : 0x7fffffff;
    reg_sort<M>(v);
#pragma unroll
    for (int k = 0; k < M; k++)
        if (k < n) list[b + k] = v[k];
}

// incoming lists in ascending pair order; one thread per particle, the
// segment sorted in registers (segments of more than 64 entries, which a
// cutoff disc at these densities practically never holds, by insertion in
// place)
__device__ __forceinline__ void sort_incoming(int i, const int64_t *__restrict__ off, int *__restrict__ list)
{
    const int64_t b = off[i], e = off[i + 1];
    const int64_t n = e - b;
    if (n <= 1) return;
    if (n <= 16) {
        sort_small_segment<16>(list, b, (int)n);
    } else if (n <= 32) {
        sort_small_segment<32>(list, b, (int)n);
    } else if (n <= 64) {
        sort_small_segment<64>(list, b, (int)n);
    } else {
        for (int64_t s = b + 1; s < e; s++) {
            const int v = list[s];
            int64_t t = s - 1;
            while (t >= b && list[t] > v) {
                list[t + 1] = list[t];
                t--;
            }
            list[t + 1] = v;
        }
    }
}

__global__ void k_in_sort(int N, const int64_t *__restrict__ off, int *__restrict__ list)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) sort_incoming(i, off, list);
}

// The whole thread-per-owner pair-list build of a small system (N at most
// PAIRS_SMALL) in one block: counts, their scan, the fill with the incoming
// counts, their scan, the incoming scatter and the per-particle sort -- the
// same steps and results as the multi-kernel build.
constexpr int PAIRS_SMALL = 8192;

// exclusive scan of n <= 8192 values by the calling block of 1024 threads; out[n] = total
template <typename TI, typename TO>
__device__ void block_scan_small(const TI *in, TO *out, int n, TO *warp_tot)
{
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int pt = (n + 1023) / 1024, b = tid * pt;
    TO tot = 0;
    for (int j = 0; j < pt; j++)
        if (b + j < n) tot += (TO)in[b + j];
    TO x = tot;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const TO t = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= d) x += t;
    }
    if (lane == 31) warp_tot[w] = x;
    __syncthreads();
    if (w == 0) {
        TO y = warp_tot[lane];
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const TO t = __shfl_up_sync(0xffffffffu, y, d);
            if (lane >= d) y += t;
        }
        warp_tot[lane] = y;  // inclusive over warps
    }
    __syncthreads();
    TO run = x - tot + (w > 0 ? warp_tot[w - 1] : (TO)0);
    for (int j = 0; j < pt; j++)
        if (b + j < n) {
            const TO v = (TO)in[b + j];
            out[b + j] = run;
            run += v;
        }
    if (tid == 1023) out[n] = warp_tot[31];
    __syncthreads();
}

__device__ __forceinline__ void pairs_small_block(int N, const double4 *__restrict__ pos_c,
                                                  const int *__restrict__ cell, const int *__restrict__ cstart,
                                                  const int *__restrict__ clist, const CellGeom &g, double rc2,
                                                  int *__restrict__ pcount, int64_t *__restrict__ poff,
                                                  int2 *__restrict__ pairs, int64_t cap, int *__restrict__ in_cnt,
                                                  int *__restrict__ in_fill, int64_t *__restrict__ in_off,
                                                  int *__restrict__ in_list, unsigned *status)
{
    __shared__ int64_t warp_tot[32];
    const int tid = threadIdx.x;
    for (int t = tid; t < N; t += 1024) {
        pairs_of_owner<false>(t, pos_c, cell, cstart, clist, g, rc2, pcount, nullptr, nullptr, 0, nullptr, nullptr);
        in_cnt[t] = 0;
        in_fill[t] = 0;
    }
    __syncthreads();
    block_scan_small<int, int64_t>(pcount, poff, N, warp_tot);
    for (int t = tid; t < N; t += 1024)
        pairs_of_owner<true>(t, pos_c, cell, cstart, clist, g, rc2, nullptr, poff, pairs, cap, in_cnt, status);
    __syncthreads();
    block_scan_small<int, int64_t>(in_cnt, in_off, N, warp_tot);
    const int64_t np = min(poff[N], cap);
    for (int64_t p = tid; p < np; p += 1024) {
        const int j = pairs[p].y;
        in_list[in_off[j] + atomicAdd(&in_fill[j], 1)] = (int)p;
    }
    __syncthreads();
    for (int i = tid; i < N; i += 1024) sort_incoming(i, in_off, in_list);
}

__global__ void __launch_bounds__(1024) k_pairs_small(int N, const double4 *__restrict__ pos_c,
                                                      const int *__restrict__ cell, const int *__restrict__ cstart,
                                                      const int *__restrict__ clist, CellGeom g, double rc2,
                                                      int *__restrict__ pcount, int64_t *__restrict__ poff,
                                                      int2 *__restrict__ pairs, int64_t cap, int *__restrict__ in_cnt,
                                                      int *__restrict__ in_fill, int64_t *__restrict__ in_off,
                                                      int *__restrict__ in_list, unsigned *status)
{
    pairs_small_block(N, pos_c, cell, cstart, clist, g, rc2, pcount, poff, pairs, cap, in_cnt, in_fill, in_off,
                      in_list, status);
}

// ---------------------------------------------------------------------------
// z order.  Keys are (z, index): a total order, so the result is the stable
// ascending order of z (sortperm, QEM_long.jl:39-40); non-finite z was zeroed
// by k_pack.  REV orders equal z by descending index instead (the second
// order of the equal-z tie mode).  Tiles of ZTILE keys are sorted in shared
// memory by a bitonic network (ZTILE / 2 threads, two keys each), then runs
// are merged ZWAY at a time: every key counts, by binary search, the keys
// that precede it in the other runs of its group.  With distinct keys every
// step places every key exactly.  Above one tile, a single system is ordered
// by z buckets first (k_zb_*, below), and these passes are its fallback.
// ---------------------------------------------------------------------------
constexpr int ZTILE = 2048;
constexpr int ZT_THREADS = ZTILE / 2;
constexpr int ZWAY = 8;

template <bool REV>
__device__ __forceinline__ bool zless(double za, int ia, double zb, int ib)
{
    return (za < zb) || (za == zb && (REV ? ia > ib : ia < ib));
}

// ascending (zless) order of the ZTILE keys (sk, si) of the calling block of
// ZT_THREADS threads: the bitonic network, thread t comparing the pair
// (i, i + stride) with i = 2 t - t mod stride at every stage
template <bool REV>
__device__ __forceinline__ void bitonic_tile(double *sk, int *si)
{
    const int t = threadIdx.x;
#pragma unroll 1
    for (int size = 2; size <= ZTILE; size <<= 1) {
#pragma unroll 1
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            __syncthreads();
            const int i = 2 * t - (t & (stride - 1)), j = i + stride;
            const double zi = sk[i], zj = sk[j];
            const int ii = si[i], ij = si[j];
            const bool up = (i & size) == 0;
            if (up ? zless<REV>(zj, ij, zi, ii) : zless<REV>(zi, ii, zj, ij)) {
                sk[i] = zj;
                sk[j] = zi;
                si[i] = ij;
                si[j] = ii;
            }
        }
    }
    __syncthreads();
}

// tile blockIdx.x of the keys (pos[i].z, i), sorted into key / idx at the
// tile's place (padding, +inf, ranks last and is not written)
template <bool REV>
__global__ void __launch_bounds__(ZT_THREADS) k_ztile(int N, const double4 *__restrict__ pos,
                                                      double *__restrict__ key, int *__restrict__ idx,
                                                      const int *__restrict__ gate)
{
    __shared__ double sk[ZTILE];
    __shared__ int si[ZTILE];
    if (gate && *gate == 0) return;  // the bucket passes placed every key (whole block)
    const int base = blockIdx.x * ZTILE;
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int l = threadIdx.x + h * ZT_THREADS, i = base + l;
        sk[l] = i < N ? pos[i].z : __longlong_as_double(0x7ff0000000000000LL);
        si[l] = i < N ? i : 0x7fffffff;
    }
    bitonic_tile<REV>(sk, si);
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int l = threadIdx.x + h * ZT_THREADS;
        if (base + l < N) {
            key[base + l] = sk[l];
            idx[base + l] = si[l];
        }
    }
}

template <bool REV>
__device__ __forceinline__ void zmerge_one(int p, int N, int width, const double *__restrict__ key,
                                           const int *__restrict__ idx, double *__restrict__ key_out,
                                           int *__restrict__ idx_out)
{
    const int run = p / width;
    const int gstart = (run - run % ZWAY) * width;  // first key of this group of ZWAY runs
    const double kz = key[p];
    const int ki = idx[p];
    int pos = gstart + (p - run * width);  // own rank inside the run
#pragma unroll 1
    for (int r = 0; r < ZWAY; r++) {
        const int rs = gstart + r * width;
        if (rs >= N) break;
        if (rs == run * width) continue;
        int lo = rs, hi = min(rs + width, N);
        while (lo < hi) {  // keys of run r that precede (kz, ki)
            const int mid = (lo + hi) >> 1;
            if (zless<REV>(key[mid], idx[mid], kz, ki)) lo = mid + 1;
            else hi = mid;
        }
        pos += lo - rs;
    }
    key_out[pos] = kz;
    idx_out[pos] = ki;
}

template <bool REV>
__global__ void k_zmerge(int N, int width, const double *__restrict__ key, const int *__restrict__ idx,
                         double *__restrict__ key_out, int *__restrict__ idx_out, const int *__restrict__ gate)
{
    if (gate && *gate == 0) return;  // the bucket passes placed every key
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < N) zmerge_one<REV>(p, N, width, key, idx, key_out, idx_out);
}

// ---------------------------------------------------------------------------
// z order by buckets (one system above one tile).  The slab's z range
// [0, L_z] is cut into nb equal buckets (about ZB_AVG keys each for a
// uniform slab; keys outside the range go to the end buckets, and the bucket
// index never decreases with z).  A count pass (atomics), a one-block scan of
// the counts, a scatter pass (atomics: arbitrary order inside a bucket) and a
// rank pass: a warp per bucket ranks each of its keys against every key of
// the bucket by zless, which restores the exact stable order, since the keys
// (z, index) are distinct.  Four short launches instead of a tile pass and
// merge passes, so the long-range chain behind the z order starts while the
// cell binning still leaves most SMs idle.  A bucket holding more than ZB_CAP
// keys (z far from uniform, many equal z) sets a flag instead, and the tile
// and merge passes, launched behind the rank pass, sort everything when that
// flag is set (and return at once when it is not).
// ---------------------------------------------------------------------------
constexpr int ZB_AVG = 32;     // keys per bucket of a uniform slab
constexpr int ZB_CAP = 256;    // largest bucket the rank pass sorts
constexpr int ZB_WARPS = 8;    // buckets per block of the rank pass
// the workspace (counts nb, starts nb + 1, places N ints) fits the 2 N ints of
// zkey_tmp from the smallest system on the bucket path (N = ZTILE + 1) up,
// since nb <= N / ZB_AVG + 1 grows more slowly than N
static_assert(2 * ((ZTILE + ZB_AVG) / ZB_AVG) + 1 <= ZTILE + 1, "z-bucket workspace exceeds its scratch");
static_assert(ZB_CAP % 32 == 0 && ZB_CAP >= 2 * ZB_AVG, "rank-pass bucket capacity");

struct ZBGeom {
    double z0, scale;  // bucket = floor((z - z0) scale), clamped to [0, nb)
    int nb;
};

__device__ __forceinline__ int zbucket(double z, const ZBGeom &g)
{
    const double f = (z - g.z0) * g.scale;
    return f <= 0.0 ? 0 : (f >= (double)(g.nb - 1) ? g.nb - 1 : (int)f);
}

// count the keys of each bucket; slot[i]: particle i's place inside its bucket
__global__ void k_zb_count(int N, const double4 *__restrict__ pos, ZBGeom g, int *cnt, int *__restrict__ slot,
                           int *__restrict__ flag)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) *flag = 0;  // read by later launches only
    if (i < N) slot[i] = atomicAdd(&cnt[zbucket(pos[i].z, g)], 1);
}

__global__ void k_zb_scatter(int N, const double4 *__restrict__ pos, ZBGeom g, const int *__restrict__ start,
                             const int *__restrict__ slot, double *__restrict__ key, int *__restrict__ idx)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const double z = pos[i].z;
    const int p = start[zbucket(z, g)] + slot[i];
    key[p] = z;
    idx[p] = i;
}

// warp w of the block ranks bucket blockIdx.x ZB_WARPS + w and writes zperm
template <bool REV>
__global__ void __launch_bounds__(32 * ZB_WARPS) k_zb_rank(int nb, const int *__restrict__ start,
                                                           const double *__restrict__ key,
                                                           const int *__restrict__ idx, int *__restrict__ zperm,
                                                           int *__restrict__ flag)
{
    __shared__ double sk[ZB_WARPS][ZB_CAP];
    __shared__ int si[ZB_WARPS][ZB_CAP];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int b = blockIdx.x * ZB_WARPS + w;
    if (b >= nb) return;  // whole warp; no block barrier below
    const int s0 = start[b], n = start[b + 1] - s0;
    if (n > ZB_CAP) {
        if (lane == 0) *flag = 1;
        return;
    }
    for (int e = lane; e < n; e += 32) {
        sk[w][e] = key[s0 + e];
        si[w][e] = idx[s0 + e];
    }
    __syncwarp();
    for (int e = lane; e < n; e += 32) {
        const double ze = sk[w][e];
        const int ie = si[w][e];
        int r = 0;
        for (int j = 0; j < n; j++) r += zless<REV>(sk[w][j], si[w][j], ze, ie) ? 1 : 0;
        zperm[s0 + r] = ie;
    }
}

// number of ZWAY-way merge passes after the tile pass for N keys
__host__ __device__ inline int zsort_pass_count(int N)
{
    int passes = 0;
    for (int64_t w = ZTILE; w < N; w *= ZWAY) passes++;
    return passes;
}

// ---------------------------------------------------------------------------
// fused batches: the small-system binning and z order over all systems
// ---------------------------------------------------------------------------
// (system, particle tile of ZTILE): pack the tile's particles and sort its
// (z, index) keys -- k_pack and k_ztile -- into the buffer the system's
// first merge pass reads (so that its last pass ends in zkey, zperm)
__global__ void __launch_bounds__(ZT_THREADS) k_batch_pack_ztile(const BatchWork *__restrict__ wl,
                                                                 const BatchSys *__restrict__ ds,
                                                                 const double *__restrict__ xyz,
                                                                 const double *__restrict__ q)
{
    __shared__ double sk[ZTILE];
    __shared__ int si[ZTILE];
    const BatchWork t = wl[blockIdx.x];
    const BatchSys &d = ds[t.s];
    const int N = d.N, base = t.x * ZTILE;
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int l = threadIdx.x + h * ZT_THREADS, i = base + l;
        sk[l] = i < N ? pack_one(i, xyz + 3 * d.off, q + d.off, d.pos, d.cell, d.geom, d.status)
                      : __longlong_as_double(0x7ff0000000000000LL);
        si[l] = i < N ? i : 0x7fffffff;
    }
    bitonic_tile<false>(sk, si);
    const bool odd = zsort_pass_count(N) & 1;
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int l = threadIdx.x + h * ZT_THREADS;
        if (base + l < N) {
            (odd ? d.zkey2 : d.zkey)[base + l] = sk[l];
            (odd ? d.ztmp : d.zperm)[base + l] = si[l];
        }
    }
}

// (system, particle tile of 256): merge pass `pass` of the system's z order
__global__ void __launch_bounds__(256) k_batch_zmerge(const BatchWork *__restrict__ wl,
                                                      const BatchSys *__restrict__ ds, int pass)
{
    const BatchWork t = wl[blockIdx.x];
    const BatchSys &d = ds[t.s];
    const int N = d.N, p = t.x * 256 + threadIdx.x;
    const bool odd = ((zsort_pass_count(N) + pass) & 1) != 0;  // pass j reads what pass j - 1 wrote
    int width = ZTILE;
    for (int j = 0; j < pass; j++) width *= ZWAY;
    if (p < N)
        zmerge_one<false>(p, N, width, odd ? d.zkey2 : d.zkey, odd ? d.ztmp : d.zperm, odd ? d.zkey : d.zkey2,
                          odd ? d.zperm : d.ztmp);
}

// The cells and the pair list of the small systems, as separate phases over
// all systems (the steps of k_cells_small and k_pairs_small, so the lists
// are the same): one block per system for the counting scatter into cells
// and for the two scans; thread-per-cell and thread-per-owner tiles for the
// rest, which keeps every thread's chain of dependent loads short.

// one block per system: cell counts, their scan (cstart) and the scatter
__global__ void __launch_bounds__(1024) k_batch_cells(const BatchSys *__restrict__ ds)
{
    QEM_SHARED_COPY(BatchSys, d, ds + blockIdx.x);
    cells_small_block<false>(d.N, d.ncell, d.cell, d.pos, d.cstart, d.clist, d.pos_of, d.pos_c);
}

// (system, tile of 256 cells): ascending index inside each cell (the cells
// of these systems hold a few particles: insertion sort by one thread), the
// inverse map and the positions in cell order
__global__ void __launch_bounds__(256) k_batch_cell_sort(const BatchWork *__restrict__ wl,
                                                         const BatchSys *__restrict__ ds)
{
    const BatchWork t = wl[blockIdx.x];
    const BatchSys &d = ds[t.s];
    const int c = t.x * 256 + threadIdx.x;
    if (c >= d.ncell) return;
    const int b = d.cstart[c], e = d.cstart[c + 1];
    int *list = d.clist;
    for (int s = b + 1; s < e; s++) {
        const int v = list[s];
        int u = s - 1;
        while (u >= b && list[u] > v) {
            list[u + 1] = list[u];
            u--;
        }
        list[u + 1] = v;
    }
    for (int s = b; s < e; s++) {
        const int i = list[s];
        d.pos_of[i] = s;
        d.pos_c[s] = d.pos[i];
    }
}

// (system, tile of 256 cell-order slots): pair count of each owner (and the
// incoming counters cleared)
__global__ void __launch_bounds__(256) k_batch_pair_count(const BatchWork *__restrict__ wl,
                                                          const BatchSys *__restrict__ ds)
{
    const BatchWork t = wl[blockIdx.x];
    const BatchSys &d = ds[t.s];
    const int s = t.x * 256 + threadIdx.x;
    if (s >= d.N) return;
    const CellGeom g = d.geom;
    pairs_of_owner<false>(s, d.pos_c, d.cell, d.cstart, d.clist, g, d.rc2, d.pcount, nullptr, nullptr, 0, nullptr,
                          nullptr);
    d.in_cnt[s] = 0;
    d.in_fill[s] = 0;
}

// one block per system: exclusive scan, pcount -> poff (WHICH = 0) or
// in_cnt -> in_off (WHICH = 1); out[N] = total
template <int WHICH>
__global__ void __launch_bounds__(1024) k_batch_scan(const BatchSys *__restrict__ ds)
{
    __shared__ int64_t warp_tot[32];
    const BatchSys &d = ds[blockIdx.x];
    block_scan_small<int, int64_t>(WHICH == 0 ? d.pcount : d.in_cnt, WHICH == 0 ? d.poff : d.in_off, d.N, warp_tot);
}

// (system, tile of 256 slots): the owners' pairs into their poff ranges
__global__ void __launch_bounds__(256) k_batch_pair_fill(const BatchWork *__restrict__ wl,
                                                         const BatchSys *__restrict__ ds)
{
    const BatchWork t = wl[blockIdx.x];
    const BatchSys &d = ds[t.s];
    const int s = t.x * 256 + threadIdx.x;
    if (s >= d.N) return;
    const CellGeom g = d.geom;
    pairs_of_owner<true>(s, d.pos_c, d.cell, d.cstart, d.clist, g, d.rc2, nullptr, d.poff, d.pairs, d.cap, d.in_cnt,
                         d.status);
}

// (system, tile of 256 pairs): each pair's entry in its second particle's
// incoming list (any slot order; the lists are sorted next)
__global__ void __launch_bounds__(256) k_batch_in_scatter(const BatchWork *__restrict__ wl,
                                                          const BatchSys *__restrict__ ds)
{
    const BatchWork t = wl[blockIdx.x];
    const BatchSys &d = ds[t.s];
    const int64_t p = (int64_t)t.x * 256 + threadIdx.x;
    if (p >= min(d.poff[d.N], d.cap)) return;
    const int j = d.pairs[p].y;
    d.in_list[d.in_off[j] + atomicAdd(&d.in_fill[j], 1)] = (int)p;
}

// (system, tile of 256 particles): incoming lists in ascending pair order
__global__ void __launch_bounds__(256) k_batch_in_sort(const BatchWork *__restrict__ wl,
                                                       const BatchSys *__restrict__ ds)
{
    const BatchWork t = wl[blockIdx.x];
    const BatchSys &d = ds[t.s];
    const int i = t.x * 256 + threadIdx.x;
    if (i < d.N) sort_incoming(i, d.in_off, d.in_list);
}

inline int nblk(int64_t n, int b) { return (int)((n + b - 1) / b); }

template <typename TI, typename TO>
cudaError_t scan_impl(const TI *in, TO *out, int n, void *tmp, size_t tmp_bytes, cudaStream_t s)
{
    if (n <= SCAN_SMALL_MAX_INT) {
        k_scan_small<TI, TO, SCAN_SMALL_PT_INT><<<1, SCAN_BLOCK, 0, s>>>(in, out, n < 0 ? 0 : n);
        return cudaGetLastError();
    }
    int nb = nblk(n, SCAN_BLOCK);
    if (nb < 1) nb = 1;
    if (tmp_bytes < sizeof(TO) * (size_t)(nb + 1)) return cudaErrorInvalidValue;
    TO *bsum = (TO *)tmp;
    k_scan_block<TI, TO><<<nb, SCAN_BLOCK, 0, s>>>(in, out, n, bsum);
    k_scan_top<TO><<<1, SCAN_BLOCK, 0, s>>>(bsum, nb);
    k_scan_add<TO><<<nb, SCAN_BLOCK, 0, s>>>(out, n, bsum);
    return cudaGetLastError();
}

}  // namespace

size_t qem_scan_tmp_bytes(int n) { return sizeof(double) * (size_t)(nblk(n, SCAN_BLOCK) + 2); }

int qem_scan_launches(int n) { return n <= SCAN_SMALL_MAX_INT ? 1 : 3; }
int qem_scan_f64_launches(int n) { return n <= SCAN_SMALL_MAX ? 1 : 3; }

static int zsort_passes(int N) { return zsort_pass_count(N); }

// the bucket passes take over above one tile when the caller gives a flag word and the slab height
static bool zb_path(int N, const int *zflag, double Lz) { return zflag && Lz > 0.0 && N > ZTILE; }
static int zb_buckets(int N) { return (int)std::min<int64_t>(((int64_t)N + ZB_AVG - 1) / ZB_AVG, SCAN_SMALL_MAX_INT); }
int qem_zsort_launches(int N, bool buckets)
{
    return N <= 0 ? 0 : 1 + zsort_passes(N) + (buckets && N > ZTILE ? 4 : 0);
}

cudaError_t qem_scan_i32_to_i64(const int *in, int64_t *out, int n, void *tmp, size_t tmp_bytes, cudaStream_t s)
{
    return scan_impl<int, int64_t>(in, out, n, tmp, tmp_bytes, s);
}

cudaError_t qem_scan_f64_excl(const double *in, double *out, int n, void *tmp, size_t tmp_bytes, cudaStream_t s)
{
    if (n <= SCAN_SMALL_MAX) {
        k_scan_small<double, double, SCAN_SMALL_PT><<<1, SCAN_BLOCK, 0, s>>>(in, out, n < 0 ? 0 : n);
        return cudaGetLastError();
    }
    int nb = nblk(n, SCAN_BLOCK);
    if (nb < 1) nb = 1;
    if (tmp_bytes < sizeof(double) * (size_t)(nb + 1)) return cudaErrorInvalidValue;
    double *bsum = (double *)tmp;
    k_scan_block_excl_f64<<<nb, SCAN_BLOCK, 0, s>>>(in, out, n, bsum);
    k_scan_top<double><<<1, SCAN_BLOCK, 0, s>>>(bsum, nb);
    k_scan_add<double><<<nb, SCAN_BLOCK, 0, s>>>(out, n, bsum);
    return cudaGetLastError();
}

cudaError_t qem_launch_pack(int N, const double *xyz, const double *q, double4 *pos, int *cell, CellGeom g,
                            unsigned *status, cudaStream_t s)
{
    if (N <= 0) return cudaSuccess;
    k_pack<<<nblk(N, 256), 256, 0, s>>>(N, xyz, q, pos, cell, g, status);
    return cudaGetLastError();
}

bool qem_cells_small(int N, int ncell) { return N <= CELLS_SMALL && ncell <= CELLS_SMALL; }

int qem_batch_zsort_passes(int N) { return zsort_pass_count(N); }
int qem_batch_ztile(void) { return ZTILE; }

cudaError_t qem_launch_batch_pack_ztile(int nw, const BatchWork *w, const BatchSys *d, const double *xyz,
                                        const double *q, cudaStream_t s)
{
    if (nw <= 0) return cudaSuccess;
    k_batch_pack_ztile<<<nw, ZT_THREADS, 0, s>>>(w, d, xyz, q);
    return cudaGetLastError();
}

cudaError_t qem_launch_batch_zmerge(int nw, const BatchWork *w, const BatchSys *d, int pass, cudaStream_t s)
{
    if (nw <= 0) return cudaSuccess;
    k_batch_zmerge<<<nw, 256, 0, s>>>(w, d, pass);
    return cudaGetLastError();
}

cudaError_t qem_launch_batch_lists(int B, const BatchWork *cells, int ncells, const BatchWork *parts, int nparts,
                                   const BatchWork *pairs, int npairs, const BatchSys *d, cudaStream_t s)
{
    if (B <= 0) return cudaSuccess;
    k_batch_cells<<<B, 1024, 0, s>>>(d);
    if (ncells > 0) k_batch_cell_sort<<<ncells, 256, 0, s>>>(cells, d);
    if (nparts > 0) k_batch_pair_count<<<nparts, 256, 0, s>>>(parts, d);
    k_batch_scan<0><<<B, 1024, 0, s>>>(d);
    if (nparts > 0) k_batch_pair_fill<<<nparts, 256, 0, s>>>(parts, d);
    k_batch_scan<1><<<B, 1024, 0, s>>>(d);
    if (npairs > 0) k_batch_in_scatter<<<npairs, 256, 0, s>>>(pairs, d);
    if (nparts > 0) k_batch_in_sort<<<nparts, 256, 0, s>>>(parts, d);
    return cudaGetLastError();
}

cudaError_t qem_launch_cells(int N, int ncell, const int *cell, const double4 *pos, int *cell_cnt, int *cell_start,
                             int *cell_fill, int *cell_list, int *pos_of, double4 *pos_c, void *scan_tmp,
                             size_t scan_tmp_bytes, cudaStream_t s)
{
    if (qem_cells_small(N, ncell)) {
        k_cells_small<<<1, 1024, 0, s>>>(N, ncell, cell, pos, cell_start, cell_list, pos_of, pos_c);
        return cudaGetLastError();
    }
    cudaError_t e = cudaMemsetAsync(cell_cnt, 0, sizeof(int) * ncell, s);
    if (e != cudaSuccess) return e;
    k_cell_count<<<nblk(N, 256), 256, 0, s>>>(N, cell, cell_cnt);
    e = scan_impl<int, int>(cell_cnt, cell_start, ncell, scan_tmp, scan_tmp_bytes, s);
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(cell_fill, cell_start, sizeof(int) * ncell, cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return e;
    k_cell_scatter<<<nblk(N, 256), 256, 0, s>>>(N, cell, cell_fill, cell_list);
    k_cell_sort<<<nblk((int64_t)ncell * 32, 256), 256, 0, s>>>(ncell, cell_start, cell_list, pos_of, pos, pos_c);
    return cudaGetLastError();
}

cudaError_t qem_launch_pair_list(int N, int ncell, const double4 *pos_c, const int *cell, const int *cell_start,
                                 const int *cell_list, CellGeom g, double rc2, int *pcount, int64_t *poff,
                                 int2 *pairs, int64_t cap, int *in_cnt, int *in_slot, int64_t *in_off, int *in_list,
                                 unsigned *status, void *scan_tmp, size_t scan_tmp_bytes, unsigned *hmask,
                                 cudaStream_t s)
{
    if (N <= 0) return cudaSuccess;
    cudaError_t e;
    // one warp per owner cell pays off from about two particles per cell;
    // sparser systems take one thread per owner.  Both give the same lists.
    if (g.ncx >= 3 && g.ncy >= 3 && (int64_t)N >= 2 * (int64_t)ncell) {
        const int nb = nblk((int64_t)ncell * 32, 128);
        k_pairs_cell<false><<<nb, 128, 0, s>>>(ncell, pos_c, cell_start, cell_list, g, rc2, pcount, nullptr, nullptr,
                                               0, in_slot, nullptr, nullptr, nullptr, hmask);
        if ((e = scan_impl<int, int64_t>(pcount, poff, N, scan_tmp, scan_tmp_bytes, s)) != cudaSuccess) return e;
        k_in_base<<<nblk(N, 256), 256, 0, s>>>(N, cell_list, cell, g, poff + N, cap, in_slot, in_cnt, status);
        if ((e = scan_impl<int, int64_t>(in_cnt, in_off, N, scan_tmp, scan_tmp_bytes, s)) != cudaSuccess) return e;
        k_pairs_cell<true><<<nb, 128, 0, s>>>(ncell, pos_c, cell_start, cell_list, g, rc2, nullptr, poff, pairs, cap,
                                              in_slot, in_off, in_list, status, hmask);
        return cudaGetLastError();
    }
    // one thread per owner (over the full deduplicated stencil when there are
    // fewer than 3 cells along x or y), incoming entries scattered with
    // atomics and sorted; a small system in one block
    if (N <= PAIRS_SMALL) {
        k_pairs_small<<<1, 1024, 0, s>>>(N, pos_c, cell, cell_start, cell_list, g, rc2, pcount, poff, pairs, cap,
                                         in_cnt, in_slot, in_off, in_list, status);
        return cudaGetLastError();
    }
    k_pairs<false><<<nblk(N, 128), 128, 0, s>>>(N, pos_c, cell, cell_start, cell_list, g, rc2, pcount, nullptr,
                                                 nullptr, 0, nullptr, nullptr);
    if ((e = scan_impl<int, int64_t>(pcount, poff, N, scan_tmp, scan_tmp_bytes, s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(in_cnt, 0, sizeof(int) * N, s)) != cudaSuccess) return e;
    k_pairs<true><<<nblk(N, 128), 128, 0, s>>>(N, pos_c, cell, cell_start, cell_list, g, rc2, nullptr, poff, pairs,
                                                cap, in_cnt, status);
    if ((e = cudaMemsetAsync(in_slot, 0, sizeof(int) * N, s)) != cudaSuccess) return e;
    if ((e = scan_impl<int, int64_t>(in_cnt, in_off, N, scan_tmp, scan_tmp_bytes, s)) != cudaSuccess) return e;
    if (cap > 0) k_in_fill<<<nblk(cap, 256), 256, 0, s>>>(poff + N, cap, pairs, in_off, in_slot, in_list);
    k_in_sort<<<nblk(N, 128), 128, 0, s>>>(N, in_off, in_list);
    return cudaGetLastError();
}

cudaError_t qem_launch_zsort(int N, const double4 *pos, int *zperm, int *ztmp, double *zkey, double *zkey_tmp,
                             cudaStream_t s, bool rev_ties, int *zflag, double Lz)
{
    if (N <= 0) return cudaSuccess;
    const int *gate = nullptr;
    if (zb_path(N, zflag, Lz)) {
        // bucket passes; workspace in zkey_tmp (as ints): counts [0, nb),
        // starts [nb, 2 nb + 1), slots [2 nb + 1, 2 nb + 1 + N) -- within its
        // 2 N ints since nb <= N / 32 + 1 and N > ZTILE
        const int nb = zb_buckets(N);
        int *cnt = reinterpret_cast<int *>(zkey_tmp), *start = cnt + nb, *slot = start + nb + 1;
        const ZBGeom g{0.0, nb / Lz, nb};
        cudaError_t e = cudaMemsetAsync(cnt, 0, sizeof(int) * nb, s);
        if (e != cudaSuccess) return e;
        k_zb_count<<<nblk(N, 256), 256, 0, s>>>(N, pos, g, cnt, slot, zflag);
        k_scan_small<int, int, SCAN_SMALL_PT_INT><<<1, SCAN_BLOCK, 0, s>>>(cnt, start, nb);
        k_zb_scatter<<<nblk(N, 256), 256, 0, s>>>(N, pos, g, start, slot, zkey, ztmp);
        if (rev_ties) k_zb_rank<true><<<nblk(nb, ZB_WARPS), 32 * ZB_WARPS, 0, s>>>(nb, start, zkey, ztmp, zperm, zflag);
        else k_zb_rank<false><<<nblk(nb, ZB_WARPS), 32 * ZB_WARPS, 0, s>>>(nb, start, zkey, ztmp, zperm, zflag);
        gate = zflag;  // the tile and merge passes below run only for a bucket over ZB_CAP
    }
    // ping-pong so that the last pass writes (zkey, zperm)
    const int passes = zsort_passes(N);
    double *ka = (passes & 1) ? zkey_tmp : zkey, *kb = (passes & 1) ? zkey : zkey_tmp;
    int *ia = (passes & 1) ? ztmp : zperm, *ib = (passes & 1) ? zperm : ztmp;
    if (rev_ties) k_ztile<true><<<nblk(N, ZTILE), ZT_THREADS, 0, s>>>(N, pos, ka, ia, gate);
    else k_ztile<false><<<nblk(N, ZTILE), ZT_THREADS, 0, s>>>(N, pos, ka, ia, gate);
    for (int64_t w = ZTILE; w < N; w *= ZWAY) {
        if (rev_ties) k_zmerge<true><<<nblk(N, 256), 256, 0, s>>>(N, (int)w, ka, ia, kb, ib, gate);
        else k_zmerge<false><<<nblk(N, 256), 256, 0, s>>>(N, (int)w, ka, ia, kb, ib, gate);
        double *tk = ka; ka = kb; kb = tk;
        int *ti = ia; ia = ib; ib = ti;
    }
    return cudaGetLastError();
}

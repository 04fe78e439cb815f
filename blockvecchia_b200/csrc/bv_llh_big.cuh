// bv_llh_big.cuh -- FP64 block evaluation for blocks too large for one SM's
// shared memory (M = cs + bs above ~235: cs = 300, skewed blocks, a large
// block 0).
//
// Left-looking blocked Cholesky of the same augmented (M+1) x M system as the
// shared-memory path (rows 0..M-1 covariance, row M the observations), in
// 16-wide panels, with only two panels resident in shared memory:
//
//   * Pcur: panel p (rows k0..M, 16 columns), fully updated; warp 0 factors
//     its diagonal block (Crout) while
//   * Pnext: panel p+1 is generated (Matern) and brought up to date with
//     panels 0..p-1 by warps 1..15: the finished panels live in a per-CTA
//     global slab (L2-resident), and each one's rows n0..M are streamed into
//     shared memory by cp.async.bulk copies on an mbarrier, two stages deep,
//     and applied as rank-16 updates on the FP64 tensor cores (m8n8k4).
//   * then all warps solve panel p's rows against its diagonal block (warp 0
//     starts on its share as soon as it has factored, the others join after
//     their work on panel p+1), panel p is written to the slab, and panel
//     p+1 takes panel p's update from shared memory.
//
// Panel q is stored in the slab as rows k0_q..M of 16 doubles (row-major),
// with column c of row r at position c ^ ((r & 3) << 2) (a swizzle that makes
// the tensor-core fragment loads conflict-free); shared-memory panels and
// stages use the same layout, so the bulk copies move rows unchanged.
//
// The block's contribution is read off the finished panels exactly as in the
// shared-memory path: positive-pivot log-determinant of the last bs columns
// and |u|^2 from row M.  Failure semantics are the same (a non-positive pivot
// stays on the diagonal, its column is zeroed below, the block is flagged).
// Every wait on an mbarrier is bounded; a wait that gives up flags the block
// BV_ST_DEVICE_TIMEOUT and the remaining waits are skipped.
//
// The same function with NS = 0 is the default path for every block whose
// two panels fit (the multi-CTA streamed kernels llh_lean_kernel_t and
// llh_lean_server_kernel, 96-256 threads, several CTAs per SM): no staging;
// the update warps read the earlier panels' fragments straight from the slab
// into registers and accumulate panel p+1's tiles in place on the DMMA
// accumulators (panel_update_direct); optionally the whole matrix is
// generated into the slab first (kBulk).
#pragma once

#include <stdint.h>

#include <algorithm>

#include "bv_llh_fp64.cuh"

namespace bv {

constexpr int kBigRC = 256;              // rows per streamed chunk
constexpr int kBigStages = 2;            // streamed chunks in flight
constexpr int kMaxStages = 4;

__host__ __device__ inline int big_panels(int M) { return (M + kNB - 1) / kNB; }

// Doubles of the per-CTA slab: panel q holds rows 16q..M (M+1-16q rows) x 16.
__host__ __device__ inline size_t big_slab_doubles(int M)
{
    const size_t Mp = (size_t)M + 1, P = (size_t)big_panels(M);
    return 16 * (P * Mp - 8 * P * (P - 1));
}

__host__ __device__ inline size_t big_panel_base(int q, int Mp)
{
    return 16 * ((size_t)q * Mp - 8 * (size_t)q * (q - 1));
}

// Shared-memory layout (bytes): X, Y, Z (observations), T (third
// coordinate, 3-D locations only; nz = 1) (M doubles each), Pcur, Pnext (Mp
// x 16 doubles), ns stages of (rc + 16) x 16 doubles, ns mbarriers.
struct BigLayout {
    unsigned o_X, o_Y, o_Z, o_T, o_cur, o_next, o_stage[kMaxStages], o_bar, total;
};

__host__ __device__ inline unsigned big_align(unsigned v) { return (v + 127u) & ~127u; }

__host__ __device__ inline BigLayout big_layout(int M, int rc = kBigRC, int nz = 0, int ns = kBigStages)
{
    BigLayout l;
    const unsigned Mp = (unsigned)M + 1;
    unsigned o = 0;
    l.o_X = o;      o = big_align(o + 8u * M);
    l.o_Y = o;      o = big_align(o + 8u * M);
    l.o_Z = o;      o = big_align(o + 8u * M);
    l.o_T = o;      if (nz) o = big_align(o + 8u * M);
    l.o_cur = o;    o = big_align(o + 128u * Mp);
    l.o_next = o;   o = big_align(o + 128u * Mp);
    for (int st = 0; st < kMaxStages; ++st) {
        l.o_stage[st] = o;
        if (st < ns) o = big_align(o + 128u * (rc + 16));
    }
    l.o_bar = o;    o = o + 8u * ns;
    l.total = o;
    return l;
}

// Largest M whose streamed-path layout fits in `bytes` of dynamic shared memory.
inline int big_max_m_for_bytes(size_t bytes, int rc = kBigRC, int nz = 0, int ns = kBigStages)
{
    int lo = 1, hi = 8192;
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (big_layout(mid, rc, nz, ns).total <= bytes)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// Dynamic shared memory and per-CTA slab (doubles) for blocks up to M = max_m,
// given the shared-memory path's limit small_m and the streamed path's big_m.
inline size_t big_launch_smem(int max_m, int small_m, int big_m, int nz = 0)
{
    size_t b = block_doubles(std::min(max_m, small_m), nz) * sizeof(double);
    if (max_m > small_m) {
        const size_t t = big_layout(std::min(max_m, big_m), kBigRC, nz).total;
        if (t > b) b = t;
    }
    return b;
}

inline size_t big_slab_stride(int max_m, int small_m, int big_m, int nz = 0)
{
    if (max_m <= small_m) return 0;
    size_t d = big_slab_doubles(std::min(max_m, big_m));
    if (max_m > big_m) d = std::max(d, block_doubles(max_m, nz));
    return (d + 31) & ~(size_t)31;
}

__device__ __forceinline__ int swz(int r, int c) { return c ^ ((r & 3) << 2); }

// CTA size of the multi-CTA streamed kernel for a launch whose largest block
// has M = max_m, from the measured table (the handles and the server use
// it): 128 threads x 4 CTAs per SM for small blocks, 160 x 3, 256 x 2.
inline int lean_table_threads(int max_m) { return max_m <= 170 ? 128 : (max_m <= 250 ? 160 : 256); }

// The static shared scratch the streamed path needs (a subset of
// BlockShared), for kernels that run only this path.
struct alignas(16) LeanShared {
    double Lt[kNB][kNB];  // factored diagonal block, transposed
    double inv[kNB];      // 1 / L_jj (0: failed pivot)
    double red[2][kWarps];
    unsigned status;
    int task;
};

// Named barrier over warps 1..NT/32-1 (the update warps).
template <int NT>
__device__ __forceinline__ void update_warps_sync()
{
    asm volatile("bar.sync 1, %0;" ::"n"(NT - 32) : "memory");
}

// Entry (i, j) of the augmented system: covariance for i < M (plus the
// nugget on the diagonal), the observation of point j on row M.  Same
// argument order and the same nugget addition as the shared-memory path's
// generation, so the entries are identical.
template <bool kXYZ3>
__device__ __forceinline__ double big_entry(const double *X, const double *Y, const double *Z,
                                            const double *T, int M, int i, int j, const MaternParams &mp)
{
    if (i >= M) return Z[j];
    double c;
    if constexpr (kXYZ3)
        c = cov_xyz(X[i], Y[i], T[i], X[j], Y[j], T[j], mp);
    else
        c = matern(X[i], Y[i], X[j], Y[j], mp);
    return (i == j && mp.nugget != 0.0) ? c + mp.nugget : c;
}

// Column c of a 16-column panel starting at row and column q0, rows
// [r_begin, Mp) step `rstep`, into dst (local row r - dst_r0, swizzled): the
// column point is read once and kept in registers; entries above the
// diagonal and columns beyond the matrix (c >= kbq) are zeros.  The same
// entries as big_entry.
template <bool kXYZ3>
__device__ __forceinline__ void gen_column(double *dst, int dst_r0, const double *X, const double *Y,
                                           const double *Z, const double *T, int M, int Mp, int q0, int kbq,
                                           int c, int r_begin, int rstep, const MaternParams &mp)
{
    const int j = q0 + c;
    if (c >= kbq) {
        for (int r = r_begin; r < Mp; r += rstep) dst[(r - dst_r0) * 16 + swz(r, c)] = 0.0;
        return;
    }
    const double xj = X[j], yj = Y[j], tj = kXYZ3 ? T[j] : 0.0, zj = Z[j];
    for (int r = r_begin; r < Mp; r += rstep) {
        double v = 0.0;
        if (r >= M) {
            v = zj;
        } else if (r >= j) {
            if constexpr (kXYZ3)
                v = cov_xyz(X[r], Y[r], T[r], xj, yj, tj, mp);
            else
                v = matern(X[r], Y[r], xj, yj, mp);
            if (r == j && mp.nugget != 0.0) v += mp.nugget;
        }
        dst[(r - dst_r0) * 16 + swz(r, c)] = v;
    }
}

// Rank-16 update of a panel held in shared memory, dst rows [d0, d1) (panel
// local rows relative to dst_r0) and 16 columns:
//     dst(i, n) -= sum_k A(i, k) * B(n, k)
// A rows come from `asrc` (local row = i - a_r0), B rows n = 0..15 from
// `bsrc` (row-major 16 doubles, swizzled by absolute row b_r0 + n).  Tiles of
// 8 rows x 16 columns are dealt to warps [w0, w0 + nw).
__device__ __forceinline__ void panel_update_tiles(double *dst, int dst_r0, const double *asrc, int a_r0,
                                                   const double *bsrc, int b_r0, int r_begin, int r_end,
                                                   int w0, int nw)
{
    const int warp = (threadIdx.x >> 5) - w0, lane = threadIdx.x & 31;
    if (warp < 0 || warp >= nw) return;
    const int r8 = lane >> 2, c4 = lane & 3;
    // B fragments are shared by every tile: B[k][n] = bsrc(n, k).
    double bf[4][2];
#pragma unroll
    for (int kk = 0; kk < 4; ++kk)
#pragma unroll
        for (int nj = 0; nj < 2; ++nj) {
            const int n = 8 * nj + r8, k = 4 * kk + c4;
            bf[kk][nj] = bsrc[n * 16 + swz(b_r0 + n, k)];
        }
    for (int i0 = r_begin + 8 * warp; i0 < r_end; i0 += 8 * nw) {
        double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
        const int ia = i0 + r8;
        const bool in = ia < r_end;
        const double *arow = asrc + (in ? ia - a_r0 : 0) * 16;
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) {
            const int k = 4 * kk + c4;
            const double a = in ? arow[swz(ia, k)] : 0.0;
#pragma unroll
            for (int nj = 0; nj < 2; ++nj) dmma_8x8x4(acc[nj][0], acc[nj][1], a, bf[kk][nj]);
        }
        if (ia < r_end) {
            double *drow = dst + (ia - dst_r0) * 16;
#pragma unroll
            for (int nj = 0; nj < 2; ++nj)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int n = 8 * nj + 2 * c4 + e;
                    drow[swz(ia, n)] -= acc[nj][e];
                }
        }
    }
}

// The left-looking update of panel p+1 without staging: nxt rows [n0, Mp)
// (local row = i - n0) take panels q = 0..p-1 read straight from this CTA's
// slab (L2).  Warps [w0, w0 + nw) own 8-row tiles (tile t on warp t mod nw)
// and keep kDT of them in registers across all q, so the warps never wait
// for one another; the next panel's fragments are loaded while the current
// one is applied.  The tiles are the DMMA accumulators themselves: with B
// negated, D = (-B)^T A + D subtracts each panel's products in place, 2 kDT
// independent accumulation chains per warp.  Per element the operations and
// their order do not depend on the CTA size or the tile count.  A lane's
// DMMA steps 2h and 2h+1 use the adjacent columns k = 8h + 2 c4 + {0, 1},
// one 16-byte load for both (the same columns in A and B, so each step
// still sums four k-products).  kDT = 2 measured fastest (n = 1M, cs = 200:
// 59.1 ms at 2, 63.4 at 3, 69.9 at 4; with 3 or more the live fragments
// crowd the registers).
constexpr int kDT = 2;

// Substitution rows of the factor warp per panel (process_block_big): with
// up to 256 rows below the diagonal block (every panel of M <= ~290) warp 0
// solves them all while the other warps generate and update the next panel.
// Kernel ms for n = 1M, cs = 200 / n = 200k, cs = 120 / n = 20k, cs = 300:
// 32 rows 51.0 / 3.89 / 1.91, 64 rows 50.4 / 3.87 / 1.89, 128 rows 49.7 /
// 3.78 / 1.86, 256 rows 49.2 / 3.77 / 1.84 (rows dealt over the whole CTA
// after a barrier: 51.2 / 3.84 / 1.92).
constexpr int kSubstRows0 = 256;

__device__ __forceinline__ double2 ldcg2(const double *p)
{
    return __ldcg(reinterpret_cast<const double2 *>(p));
}

template <int NTILE>
__device__ __forceinline__ void load_frags(const double *pq, int q0, int Mp, int n0, int i0, int nw,
                                           int r8, int c4, double2 (&bf)[2][2], double2 (&af)[NTILE][2])
{
    // B: the 16 rows n0.. of panel q, read by every tile of the panel,
    // through L1 (n = 1M, cs = 200: 51.2 against 51.8 ms through L2 only);
    // A: each tile's own rows, read once per panel, L2 only.  This CTA wrote
    // both before the last barrier, from this SM.
#pragma unroll
    for (int h = 0; h < 2; ++h) {
#pragma unroll
        for (int nj = 0; nj < 2; ++nj) {
            const int r = n0 + 8 * nj + r8;
            bf[h][nj] = (r < Mp) ? *reinterpret_cast<const double2 *>(pq + (size_t)(r - q0) * 16 +
                                                                      swz(r, 8 * h + 2 * c4))
                                 : make_double2(0.0, 0.0);
        }
#pragma unroll
        for (int m = 0; m < NTILE; ++m) {
            const int ia = i0 + 8 * nw * m + r8;
            af[m][h] = (ia < Mp) ? ldcg2(pq + (size_t)(ia - q0) * 16 + swz(ia, 8 * h + 2 * c4))
                                 : make_double2(0.0, 0.0);
        }
    }
}

template <int NTILE, bool kRaw>
__device__ __forceinline__ void direct_tiles(double *nxt, int n0, const double *slab, int Mp, int p,
                                             int i0, int nw, int r8, int c4)
{
    // Panel p+1 before the update: generated into nxt, or (kRaw) still in
    // the slab where the whole matrix was generated.
    const double *src = kRaw ? slab + big_panel_base(p + 1, Mp) : nxt;
    double d[NTILE][2][2];
#pragma unroll
    for (int m = 0; m < NTILE; ++m) {
        const int ia = i0 + 8 * nw * m + r8;
#pragma unroll
        for (int nj = 0; nj < 2; ++nj)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int o = (ia - n0) * 16 + swz(ia, 8 * nj + 2 * c4 + e);
                d[m][nj][e] = (ia < Mp) ? (kRaw ? __ldcg(src + o) : src[o]) : 0.0;
            }
    }
    double2 bf[2][2], af[NTILE][2], bn[2][2], an[NTILE][2];
    if (p > 0) load_frags<NTILE>(slab + big_panel_base(0, Mp), 0, Mp, n0, i0, nw, r8, c4, bf, af);
    for (int q = 0; q < p; ++q) {
        if (q + 1 < p)
            load_frags<NTILE>(slab + big_panel_base(q + 1, Mp), (q + 1) * kNB, Mp, n0, i0, nw, r8, c4,
                              bn, an);
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) {
            const int h = kk >> 1;
            double b[2];
#pragma unroll
            for (int nj = 0; nj < 2; ++nj) b[nj] = -((kk & 1) ? bf[h][nj].y : bf[h][nj].x);
#pragma unroll
            for (int m = 0; m < NTILE; ++m) {
                const double a = (kk & 1) ? af[m][h].y : af[m][h].x;
#pragma unroll
                for (int nj = 0; nj < 2; ++nj) dmma_8x8x4(d[m][nj][0], d[m][nj][1], a, b[nj]);
            }
        }
        if (q + 1 < p) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
#pragma unroll
                for (int nj = 0; nj < 2; ++nj) bf[h][nj] = bn[h][nj];
#pragma unroll
                for (int m = 0; m < NTILE; ++m) af[m][h] = an[m][h];
            }
        }
    }
#pragma unroll
    for (int m = 0; m < NTILE; ++m) {
        const int ia = i0 + 8 * nw * m + r8;
        if (ia < Mp) {
#pragma unroll
            for (int nj = 0; nj < 2; ++nj)
#pragma unroll
                for (int e = 0; e < 2; ++e) nxt[(ia - n0) * 16 + swz(ia, 8 * nj + 2 * c4 + e)] = d[m][nj][e];
        }
    }
}

// kRaw: panel p+1 is taken from the slab (the whole matrix generated there
// first) and written to nxt updated, also when there is nothing to apply.
template <bool kRaw>
__device__ __forceinline__ void panel_update_direct(double *nxt, int n0, const double *slab, int Mp, int p,
                                                    int w0, int nw)
{
    const int warp = (threadIdx.x >> 5) - w0, lane = threadIdx.x & 31;
    if (warp < 0 || warp >= nw || (!kRaw && p == 0)) return;
    const int r8 = lane >> 2, c4 = lane & 3;
    const int ntiles = (Mp - n0 + 7) >> 3;
    // Groups of kDT tiles per warp, computed whole: the tiles of a group
    // beyond the panel's rows hold zeros and are not stored (one code path
    // keeps the accumulation chains of all kDT tiles interleaved).
    for (int t0 = warp; t0 < ntiles; t0 += nw * kDT)
        direct_tiles<kDT, kRaw>(nxt, n0, slab, Mp, p, n0 + 8 * t0, nw, r8, c4);
}

// One block by the streamed path, run by a CTA of NT threads (warp 0
// factors, the other NT/32 - 1 warps generate and update), with RC rows per
// streamed chunk and NS chunks in flight (NS = 0: no staging, the warps read
// the slab directly, panel_update_direct; with kBulk the whole matrix is
// generated into the slab first).  smem: the dynamic area
// (big_layout(M, RC, nz, NS).total bytes); slab: this CTA's global slab
// (big_slab_doubles(M) doubles).  Every element's operations and their
// order are the same for every NT, RC, NS > 0 and kBulk; the direct update
// (NS = 0) accumulates in place and rounds differently from the staged one.
template <int NT, int RC, typename SH, int NS = kBigStages, bool kXYZ3 = false, bool kBulk = false>
static __device__ __noinline__ void process_block_big(const LlhArgs &a, const MaternParams &mp, int b,
                                                      unsigned char *smem, double *slab, SH &sh)
{
    static_assert(NT % 32 == 0 && NT > 32, "whole warps, at least one besides the factor warp");
    constexpr int kT = NT, kW = NT / 32;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int off = a.acc[b];
    const int bs = a.acc[b + 1] - off;
    const int mc = (b == 0) ? 0 : a.cs;
    const int M = mc + bs, Mp = M + 1;
    const int P = big_panels(M);
    const BigLayout l = big_layout(M, RC, kXYZ3 ? 1 : 0, NS);
    double *X = reinterpret_cast<double *>(smem + l.o_X);
    double *Y = reinterpret_cast<double *>(smem + l.o_Y);
    double *Z = reinterpret_cast<double *>(smem + l.o_Z);
    double *T = kXYZ3 ? reinterpret_cast<double *>(smem + l.o_T) : nullptr;
    double *cur = reinterpret_cast<double *>(smem + l.o_cur);
    double *nxt = reinterpret_cast<double *>(smem + l.o_next);
    double *stage[NS > 0 ? NS : 1];
#pragma unroll
    for (int st = 0; st < NS; ++st) stage[st] = reinterpret_cast<double *>(smem + l.o_stage[st]);
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + l.o_bar);

    const int *kidx = a.knn + (size_t)b * a.cs;
    for (int t = tid; t < M; t += kT) {
        const int src = (t < mc) ? __ldg(kidx + t) : off + (t - mc);
        X[t] = __ldg(a.x + src);
        Y[t] = __ldg(a.y + src);
        Z[t] = __ldg(a.obs + src);
        if constexpr (kXYZ3) T[t] = __ldg(a.z + src);
    }
    if (tid == 0) {
        for (int st = 0; st < NS; ++st) mbar_init(&bar[st], 1);
        fence_mbar_init();
    }
    __syncthreads();
    if constexpr (NS == 0 && kBulk) {
        // Every panel's entries straight into the slab, by all warps (the
        // update warps then take panel p+1 from there): the generation runs
        // at the CTA's full width instead of beside warp 0's pivot chain.
        for (int q = 0; q < P; ++q)
            gen_column<kXYZ3>(slab + big_panel_base(q, Mp), q * kNB, X, Y, Z, T, M, Mp, q * kNB,
                              min(kNB, M - q * kNB), tid & 15, q * kNB + (tid >> 4), kT >> 4, mp);
        __syncthreads();
        for (int e = tid; e < Mp * 8; e += kT)
            reinterpret_cast<double2 *>(cur)[e] = __ldcg(reinterpret_cast<const double2 *>(slab) + e);
    } else {
        // Panel 0 into cur: thread t takes column t mod 16, every (kT/16)-th row.
        gen_column<kXYZ3>(cur, 0, X, Y, Z, T, M, Mp, 0, min(kNB, M), tid & 15, tid >> 4, kT >> 4, mp);
    }
    __syncthreads();

    unsigned st = 0;          // thread 0: pivot flags
    unsigned phase_bits = 0;  // parity of the next wait per stage (update warps)
    bool timed_out = false;

    for (int p = 0; p < P; ++p) {
        const int k0 = p * kNB, kb = min(kNB, M - k0);
        const int n0 = k0 + kb;                       // first row / column of panel p+1
        const int kb1 = max(0, min(kNB, M - n0));     // its width
        if (warp == 0) {
            // Lagged Crout factorization of the diagonal block (lane r < kb
            // owns row k0+r; factor_rows).  With a full panel the upper lanes
            // solve the next 16 rows (k0+16..k0+31, below the diagonal block)
            // on the same chain, so the substitution phase starts 16 rows on.
            const bool low = lane < kNB;
            const int row = k0 + lane;
            const bool valid = low ? lane < kb : (kb == kNB && row < Mp);
            double v[kNB], myinv;
#pragma unroll
            for (int c = 0; c < kNB; ++c)
                v[c] = (valid && c < kb && (!low || c <= lane)) ? cur[lane * 16 + swz(row, c)] : 0.0;
            const unsigned fst = factor_rows(k0, kb, mc, v, myinv);
            if (valid) {
#pragma unroll
                for (int c = 0; c < kNB; ++c)
                    if (c < kb && (!low || c <= lane)) cur[lane * 16 + swz(row, c)] = v[c];
            }
            if (lane < kNB) {
#pragma unroll
                for (int c = 0; c < kNB; ++c) sh.Lt[c][lane] = (c <= lane && lane < kb) ? v[c] : 0.0;
                sh.inv[lane] = (lane < kb) ? myinv : 0.0;
            }
            if (lane == 0) st |= fst;
        } else if (kb1 > 0) {
            const int nrows = Mp - n0;
            if constexpr (NS != 0 || !kBulk) {
                // Panel p+1: generate (update thread u takes column u mod 16,
                // every ((kT - 32)/16)-th row), then apply panels 0..p-1.
                const int u = tid - 32;
                gen_column<kXYZ3>(nxt, n0, X, Y, Z, T, M, Mp, n0, kb1, u & 15, n0 + (u >> 4), (kT - 32) >> 4,
                                  mp);
                update_warps_sync<NT>();
            }
            if constexpr (NS == 0) {
                panel_update_direct<kBulk>(nxt, n0, slab, Mp, p, 1, kW - 1);
            } else {
            const int nchunk = (nrows + RC - 1) / RC;
            const int items = nchunk * p;       // (chunk, q), q fastest
            const bool producer = (tid == 32);
            auto issue = [&](int it) {
                const int ch = it / p, q = it - ch * p;
                const int s = it % NS;
                const int r0 = n0 + ch * RC, r1 = min(Mp, r0 + RC);
                const int nb = min(kNB, Mp - n0);
                const double *pq = slab + big_panel_base(q, Mp);
                const int q0 = q * kNB;
                const unsigned abytes = 128u * (unsigned)(r1 - r0), bbytes = 128u * (unsigned)nb;
                mbar_arrive_expect_tx(&bar[s], abytes + bbytes);
                bulk_g2s(stage[s], pq + (size_t)(r0 - q0) * 16, abytes, &bar[s]);
                bulk_g2s(stage[s] + RC * 16, pq + (size_t)(n0 - q0) * 16, bbytes, &bar[s]);
            };
            // The producer (thread 32) counts the copies it issued per stage
            // and the phases it saw complete, to drain after a timeout.
            int issued[NS], landed[NS];
#pragma unroll
            for (int st = 0; st < NS; ++st) issued[st] = landed[st] = 0;
            if (producer) {
                for (int it = 0; it < min(NS, items); ++it) {
                    issue(it);
                    issued[it % NS]++;
                }
            }
            for (int it = 0; it < items; ++it) {
                const int ch = it / p;
                const int s = it % NS;
                const int r0 = n0 + ch * RC, r1 = min(Mp, r0 + RC);
                const unsigned par = (phase_bits >> s) & 1u;
                if (!timed_out) {
                    if (mbar_wait_bounded(&bar[s], par))
                        landed[s]++;
                    else
                        timed_out = true;
                }
                phase_bits ^= 1u << s;
                panel_update_tiles(nxt, n0, stage[s], r0, stage[s] + RC * 16, n0, r0, r1, 1,
                                   kW - 1);
                update_warps_sync<NT>();
                if (producer && !timed_out && it + NS < items) {
                    fence_proxy_async_shared();
                    issue(it + NS);
                    issued[s]++;
                }
            }
            if (producer && timed_out) {
                // Copies still in flight must land before this shared memory
                // is used again: wait (bounded) for each stage's last phase.
                for (int s = 0; s < NS; ++s)
                    if (issued[s] > landed[s]) mbar_wait_bounded(&bar[s], (unsigned)(issued[s] - 1) & 1u);
            }
            }
        }
        // The substitution needs only the factored diagonal block: warp 0
        // publishes it (named barrier 3 over the CTA: warp 0 arrives, the
        // others wait after their work on panel p+1) and goes on to its rows,
        // which overlap the other warps' generation and update.
        if (warp == 0) {
            __syncwarp();
            asm volatile("bar.arrive 3, %0;" ::"n"(NT) : "memory");
        } else {
            asm volatile("bar.sync 3, %0;" ::"n"(NT) : "memory");
        }
        // Rows below the diagonal block (after the 16 the factor warp solved
        // for a full panel): forward substitution against L_kk, the two
        // operands on step q+1's dependent chain (1 / L_{q+1,q+1} and
        // L_{q+2,q+1}) read one step ahead.  Warp 0, idle for most of the
        // phase before, takes the first kSubstRows0 rows, the other warps the
        // rest.
        const int rs0 = k0 + (kb == kNB ? 2 * kNB : kb);
        const int rw0 = min(Mp, rs0 + kSubstRows0);
        const int rbeg = (warp == 0) ? rs0 + lane : rw0 + tid - 32;
        const int rend = (warp == 0) ? rw0 : Mp;
        const int rstep = (warp == 0) ? 32 : kT - 32;
        for (int r = rbeg; r < rend; r += rstep) {
            double *row = cur + (r - k0) * 16;
            double w[kNB];
#pragma unroll
            for (int c = 0; c < kNB; ++c) w[c] = (c < kb) ? row[swz(r, c)] : 0.0;
            double inv_q = sh.inv[0];
            double l_next = sh.Lt[0][1];
#pragma unroll
            for (int q = 0; q < kNB; ++q) {
                if (q < kb) {
                    asm volatile("" ::: "memory");
                    const double inv_cur = inv_q;
                    const double l_cur = l_next;
                    if (q + 1 < kNB) inv_q = sh.inv[q + 1];
                    if (q + 2 < kNB) l_next = sh.Lt[q + 1][q + 2];
                    double2 col[kNB / 2];
                    const double2 *srcp = reinterpret_cast<const double2 *>(sh.Lt[q]);
#pragma unroll
                    for (int h = (q + 2) >> 1; h < kNB / 2; ++h) col[h] = srcp[h];
                    w[q] *= inv_cur;
                    if (q + 1 < kNB) w[q + 1] = fma(-w[q], l_cur, w[q + 1]);
#pragma unroll
                    for (int c = q + 2; c < kNB; ++c) {
                        const double lc = (c & 1) ? col[c >> 1].y : col[c >> 1].x;
                        w[c] = fma(-w[q], lc, w[c]);
                    }
                }
            }
#pragma unroll
            for (int c = 0; c < kNB; ++c)
                if (c < kb) row[swz(r, c)] = w[c];
        }
        __syncthreads();
        // Panel p to the slab; panel p+1 takes panel p's update.
        {
            double *pg = slab + big_panel_base(p, Mp);
            const double2 *s2 = reinterpret_cast<const double2 *>(cur);
            double2 *g2 = reinterpret_cast<double2 *>(pg);
            for (int e = tid; e < (Mp - k0) * 8; e += kT) g2[e] = s2[e];
        }
        if (kb1 > 0)
            panel_update_tiles(nxt, n0, cur, k0, cur + (n0 - k0) * 16, n0, n0, Mp, 0, kW);
        fence_proxy_async_global();
        __syncthreads();
        double *t = cur;
        cur = nxt;
        nxt = t;
    }

    // log det of the conditional factor (positive pivots) and |u|^2 (row M).
    double ld = 0.0, qf = 0.0;
    for (int j = mc + tid; j < M; j += kT) {
        const int q = j / kNB, c = j - q * kNB;
        const double *pq = slab + big_panel_base(q, Mp);
        const double d = pq[(j - q * kNB) * 16 + swz(j, c)];
        if (d > 0) ld += log(d * d);
        const double u = pq[(M - q * kNB) * 16 + swz(M, c)];
        qf = fma(u, u, qf);
    }
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) {
        ld += __shfl_xor_sync(0xffffffffu, ld, s);
        qf += __shfl_xor_sync(0xffffffffu, qf, s);
    }
    if (lane == 0) {
        sh.red[0][warp] = ld;
        sh.red[1][warp] = qf;
    }
    if (timed_out) atomicOr(&sh.status, kStDeviceTimeout);
    if (tid == 0 && st) atomicOr(&sh.status, st);
    __syncthreads();
    if (tid == 0) {
        double Ls = 0.0, Qs = 0.0;
        for (int w = 0; w < kW; ++w) {
            Ls += sh.red[0][w];
            Qs += sh.red[1][w];
        }
        const double v = -(Qs + Ls + (double)bs * a.log2pi) * 0.5;
        unsigned s2 = sh.status;
        if (!isfinite(v)) s2 |= BV_ST_NONFINITE;
        a.block_llk[b] = v;
        a.block_status[b] = s2 | a.status_or;
        // The barriers are re-initialised for the next block.
        for (int st = 0; st < NS; ++st)
            asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(&bar[st])) : "memory");
    }
}

// One block by the path its size calls for: shared memory, the streamed
// large-block path, or (beyond the streamed path's shared-memory limit) the
// shared-memory algorithm on this CTA's global slab.
// kBig = false compiles the shared-memory and slab paths only, so layouts
// without large blocks run the same code as before the streamed path existed.
template <bool kBig, bool kXYZ3 = false>
__device__ __forceinline__ void run_block(const LlhArgs &a, const MaternParams &mp, int b, double *smem,
                                          BlockShared &sh)
{
    const int tid = threadIdx.x;
    const int bs = a.acc[b + 1] - a.acc[b];
    const int M = ((b == 0) ? 0 : a.cs) + bs;
    if (tid == 0) sh.status = 0u;
    if (bs == 0) {  // empty block: contributes -(0 + 0 + 0) / 2
        if (tid == 0) {
            a.block_llk[b] = -0.0;
            a.block_status[b] = a.status_or;
        }
    } else if (M <= a.smem_max_m) {
        constexpr int nc = kXYZ3 ? 3 : 2;  // coordinate arrays before the matrix
        process_block<kXYZ3>(a, mp, b, smem, smem + M, kXYZ3 ? smem + 2 * M : nullptr, smem + nc * M,
                             sh);
    } else {
        double *slab = a.gslab + (size_t)blockIdx.x * a.gslab_stride;
        if (kBig && M <= a.big_max_m) {
            process_block_big<kThreads, kBigRC, BlockShared, kBigStages, kXYZ3>(
                a, mp, b, reinterpret_cast<unsigned char *>(smem), slab, sh);
        } else {
            constexpr int nc = kXYZ3 ? 3 : 2;
            process_block<kXYZ3>(a, mp, b, slab, slab + M, kXYZ3 ? slab + 2 * M : nullptr,
                                 slab + nc * M, sh);
        }
    }
}

}  // namespace bv

// bv_llh_fp64.cuh -- the fused FP64 per-block kernel of the log-likelihood.
//
// One CTA evaluates one Vecchia block b at a time (persistent CTAs pull block
// ids from a work counter, largest blocks first).  For block b >= 1 with
// conditioning size cs and bs points it forms, in shared memory (or in a
// per-CTA global slab when it does not fit), the lower triangle of the
// augmented (M+1) x M system, M = cs + bs:
//
//        [ Sigma22   .      ]        rows 0..cs-1     (conditioning points)
//        [ Sigma12   Sigma11]        rows cs..M-1     (the block's points)
//        [ z_c^T     z^T    ]        row  M           (observations)
//
// and runs one blocked right-looking Cholesky over its first M columns.  The
// factor's trailing bs x bs block is chol(Sigma11 - Sigma21^T Sigma22^-1
// Sigma21) and row M becomes [w; u] with u = L'^-1 (z - mu), so the block's
// contribution  -(|u|^2 + sum log(L'_jj^2) + bs log(2 pi)) / 2  reads off
// the last bs columns.  This is the sequence of include/llh_Xvecchia_batch.h
// (potrf :295, trsm :320/:332, gemm :352/:370, geadd :407-431, potrf :449,
// trsm :461, core_Xlogdet include/vecchia_helper_method.h:263-280, nrm2
// :475, sum :480-494) as a single factorization.  Block 0 is unconditioned
// (the geadd loop starts at i = 1), so for it M = bs and all rows count.
//
// Packed storage: column j of the (M+1)-row lower triangle starts at
// off(j) = j*Mp - j*(j+1)/2, Mp = M+1; element (i, j), i >= j, is at off(j)+i.
//
// Schedule (512 threads): Matern generation with four independent entries in
// flight per lane; then per 16-wide panel p, warp 0 factors the diagonal
// block while warps 1..15 apply panel p-1 to the columns beyond panel p
// (one panel of look-ahead), all warps solve the panel rows, and all warps
// bring panel p+1's columns up to date.  The rank-16 updates run on the FP64
// tensor cores (mma.sync m8n8k4 f64).
#pragma once

#include <stdint.h>

#include "bv_matern.cuh"

namespace bv {

constexpr int kThreads = 512;
constexpr int kWarps = kThreads / 32;
constexpr int kNB = 16;  // panel width of the blocked Cholesky
constexpr unsigned kWaitIters = 1u << 20;      // bound on every mbarrier wait
constexpr unsigned kStDeviceTimeout = 16u;     // block status: a bounded wait gave up

struct LlhArgs {
    const double *x, *y, *obs;  // [n] block-ordered
    const double *z;            // [n] block-ordered third coordinate, or nullptr (2-D)
    const int *acc;             // [bc+1]
    const int *knn;             // [bc*cs]
    const int *order;           // [bc] processing order (largest first)
    int bc, cs;
    int smem_max_m;             // largest M kept in shared memory
    int slab_max_m;             // largest M of any block (global slab sizing)
    double *block_llk;          // [bc]
    unsigned *block_status;     // [bc]
    unsigned *work_counter;     // persistent scheduler counter (zeroed per eval)
    double *gslab;              // per-CTA global slabs, or nullptr
    size_t gslab_stride;        // doubles per slab
    double log2pi;              // log(2 * 3.141592653589793)
    const MaternParams *mp;     // device copy of this evaluation's parameters
    int task_begin, task_end;   // slice of `order` this launch serves
    const int *task_count;      // if set, the slice also ends at *task_count (device)
    unsigned status_or;         // flags OR-ed into every block status written
    int big_max_m;              // blocks with smem_max_m < M <= big_max_m: streamed path
};

// ---------------------------------------------------------------------------
// mbarrier, bulk-copy and proxy-fence helpers (inline PTX).
// ---------------------------------------------------------------------------

__device__ __forceinline__ unsigned smem_addr(const void *p)
{
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Bounded wait on an mbarrier phase; false when it gave up.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity)
{
    for (unsigned it = 0; it < kWaitIters; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ void fence_proxy_async_shared()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_global()
{
    asm volatile("fence.proxy.async.global;" ::: "memory");
}

__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__host__ __device__ inline size_t packed_elems(int Mp) { return (size_t)Mp * (Mp + 1) / 2; }

// Doubles a block of size M needs: x[M], y[M] (and z[M] for 3-D locations,
// nz = 1), packed (M+1)-row triangle.
__host__ __device__ inline size_t block_doubles(int M, int nz = 0)
{
    return (2 + (size_t)nz) * (size_t)M + packed_elems(M + 1);
}

__device__ __forceinline__ int poff(int j, int Mp) { return j * Mp - ((j * (j + 1)) >> 1); }

// Shared scratch of the kernel besides the block itself.
struct alignas(16) BlockShared {
    double Lt[kNB][kNB];        // factored diagonal block of panel p, transposed:
                                // Lt[c][r] = L_rc (0 above the diagonal), column c contiguous
    double Lnx[kNB][kNB + 2];   // L(rows of panel p+1, columns of panel p)
    double inv[kNB];            // 1 / L_jj of panel p (0: failed pivot)
    double red[2][kWarps];
    uint64_t bar_lready;        // warp 0 -> warps 1..15: panel p's factor is in Lt/Lnx/inv
    uint64_t bar_crit;          // warp 1 -> warp 0: the rows warp 0 needs next are done
    uint64_t bar_free;          // warps 1..15 -> warp 0: Lt/Lnx/inv may be overwritten
    unsigned phase_base;        // panels completed by this CTA (parity of the barriers)
    int bulk_next[2];           // next bulk work item of panels with even / odd index
    uint64_t bar_ls[2];         // chain warps -> bulk warps: panel p's L is stored (by p's parity)
    uint64_t bar_nc[2];         // bulk warps -> chain warps: panel p+1's columns took panel p-1
    unsigned ph_ls[2], ph_nc[2];  // phases those four barriers completed before this block
    int work_next[4];           // next bulk work item, by (2 p + stage) mod 4
    uint64_t bar_g0[2];         // bulk -> critical rows: panel p's first row group is up to date (by parity)
    unsigned ph_g0[2];          // phases bar_g0 completed before this block
    unsigned status;
    int task;
};

// Once per CTA, before the first block.
__device__ __forceinline__ void init_block_sync(BlockShared &sh)
{
    if (threadIdx.x == 0) {
        mbar_init(&sh.bar_lready, 1);
        mbar_init(&sh.bar_crit, 1);
        mbar_init(&sh.bar_free, 1);
        sh.phase_base = 0;
        sh.bulk_next[0] = sh.bulk_next[1] = 0;
        for (int i = 0; i < 2; ++i) {
            mbar_init(&sh.bar_ls[i], 1);
            mbar_init(&sh.bar_nc[i], 1);
            sh.ph_ls[i] = sh.ph_nc[i] = 0;
        }
        for (int i = 0; i < 4; ++i) sh.work_next[i] = 0;
        for (int i = 0; i < 2; ++i) {
            mbar_init(&sh.bar_g0[i], 1);
            sh.ph_g0[i] = 0;
        }
        fence_mbar_init();
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// Matern generation.
// ---------------------------------------------------------------------------

// Lower triangle of rows 0..M-1 with columns paired (q, M-1-q), so each pair
// holds M+1 entries (the middle column of an odd M only M-q).  The pairs'
// entries form one flat index space dealt to the warps in chunks of 32 x
// kGenU, so only the last chunk is partial; a lane computes kGenU entries at a
// time, branch-free (entries past the end are clamped and dropped) and with
// the smoothness dispatch hoisted out of the loop, so the independent exp
// chains interleave.
constexpr int kGenU = 6;

template <int KIND>
__device__ __forceinline__ double matern_kind(double x1, double y1, double x2, double y2,
                                              const MaternParams &mp)
{
    const double r = matern_r(x1, y1, x2, y2, mp);
    if (KIND == kNuGeneral) return (r == 0.0) ? mp.sigma2 : matern_general(r, mp);
    const double e = exp(-r);
    double c;
    if (KIND == kNuHalf)
        c = e;
    else if (KIND == kNuThreeHalves)
        c = (1.0 + r) * e;
    else
        c = fma(r, r * (1.0 / 3.0), 1.0 + r) * e;
    return (r == 0.0) ? mp.sigma2 : mp.sigma2 * c;
}

// KIND kXYZ: locations with a third coordinate T (cov_xyz).
constexpr int kXYZ = 16;

template <int KIND>
__device__ __forceinline__ void generate_t(double *A, const double *X, const double *Y, const double *T,
                                           int M, const MaternParams &mp)
{
    const int Mp = M + 1;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int half = (M + 1) >> 1;
    const int total = half * Mp;
    for (int e0 = (warp * kGenU * 32) + lane; e0 < total; e0 += kWarps * kGenU * 32) {
        int q = e0 / Mp;
        int rr0 = e0 - q * Mp;
        double v[kGenU];
        int dst[kGenU];
#pragma unroll
        for (int u = 0; u < kGenU; ++u) {
            if (u > 0) {
                rr0 += 32;
                while (rr0 >= Mp) {
                    rr0 -= Mp;
                    ++q;
                }
            }
            const int jb = M - 1 - q;
            const int na = M - q;  // rows q..M-1 of column q
            const int nt = (jb == q) ? na : Mp;
            const bool valid = q < half && rr0 < nt;
            const int qq = valid ? q : 0;
            const int rr = valid ? rr0 : 0;
            const int jbb = M - 1 - qq, naa = M - qq;
            const bool first = rr < naa;
            const int i = first ? qq + rr : jbb + (rr - naa);
            const int j = first ? qq : jbb;
            dst[u] = valid ? poff(j, Mp) + i : -1;
            if constexpr (KIND == kXYZ)
                v[u] = cov_xyz(X[i], Y[i], T[i], X[j], Y[j], T[j], mp);
            else
                v[u] = matern_kind<KIND>(X[i], Y[i], X[j], Y[j], mp);
        }
#pragma unroll
        for (int u = 0; u < kGenU; ++u)
            if (dst[u] >= 0) A[dst[u]] = v[u];
    }
}

// kXYZ: locations with a third coordinate (T); the 2-D kernels are
// separate instantiations, so their code and register allocation carry
// nothing of the 3-D path.
template <bool kXYZ3>
__device__ __forceinline__ void generate(double *A, const double *X, const double *Y, const double *T,
                                         int M, const MaternParams &mp)
{
    if constexpr (kXYZ3) {
        generate_t<kXYZ>(A, X, Y, T, M, mp);
        return;
    }
    switch (mp.nu_kind) {
    case kNuHalf:
        generate_t<kNuHalf>(A, X, Y, nullptr, M, mp);
        break;
    case kNuThreeHalves:
        generate_t<kNuThreeHalves>(A, X, Y, nullptr, M, mp);
        break;
    case kNuFiveHalves:
        generate_t<kNuFiveHalves>(A, X, Y, nullptr, M, mp);
        break;
    default:
        generate_t<kNuGeneral>(A, X, Y, nullptr, M, mp);
        break;
    }
}

// ---------------------------------------------------------------------------
// Panel factorization pieces.
// ---------------------------------------------------------------------------

// Warp 0: left-looking (Crout) factorization of the kb x kb diagonal block
// of panel p, with the kb1 rows of panel p+1 solved in the same pass.  Lane r
// < 16 owns row k0+r of the diagonal block, lane 16+r owns row n0+r (panel
// p+1); at pivot q every lane forms a_rq - sum_{k<q} L_rk L_qk (row q comes
// by shuffles from lane q), lane q's value is the pivot, and one rsqrt scales
// the column.  A non-positive or NaN pivot is kept on the diagonal and its
// column is zeroed below (the block is reported; its log-determinant skips
// the pivot, as core_Xlogdet does).  Results: L to A, sh.Lt (diagonal block)
// and sh.Lnx (panel p+1 rows), 1/L_jj to sh.inv (0 for a failed pivot).
__device__ __forceinline__ unsigned factor_diag_regs(const double *A, int Mp, int k0, int kb, int n0,
                                                     int kb1, int mc, double (&v)[kNB], double &myinv)
{
    const int lane = threadIdx.x & 31;
    const bool low = lane < kNB;
    const int r = low ? lane : lane - kNB;  // row within its 16-row group
    const bool valid = low ? (r < kb) : (r < kb1);
    const int row = low ? k0 + r : n0 + r;
#pragma unroll
    for (int c = 0; c < kNB; ++c)
        v[c] = (valid && c < kb && (!low || c <= r)) ? A[poff(k0 + c, Mp) + row] : 0.0;
    unsigned st = 0;
    myinv = 0.0;
    // Lagged Crout: the sum for pivot q over k < q-1 was formed while pivot
    // q-1's reciprocal square root was in flight; only the k = q-1 term (row q
    // of L by one shuffle) stays on the dependent chain.
    // Every lane also forms the pivot itself from lane q's partial sum
    // (broadcast early) and L_{q,q-1}, with the operands lane q uses, so the
    // pivot needs no second shuffle on the chain.
    double pre = v[0];
#pragma unroll
    for (int q = 0; q < kNB; ++q) {
        if (q < kb) {
            const double preq = __shfl_sync(0xffffffffu, pre, q);
            double s = pre, piv = preq;
            if (q > 0) {
                const double l = __shfl_sync(0xffffffffu, v[q - 1], q);
                s = fma(-v[q - 1], l, s);
                piv = fma(-l, l, preq);
            }
            const bool ok = piv > 0.0;
            const double inv = ok ? rsqrt(piv) : 0.0;
            if (q + 1 < kNB) {
                // Four independent partial sums keep this chain short too.
                double s4[4] = {v[q + 1], 0.0, 0.0, 0.0};
#pragma unroll
                for (int k = 0; k < q; ++k) {
                    const double lk = __shfl_sync(0xffffffffu, v[k], q + 1);
                    s4[k & 3] = fma(-v[k], lk, s4[k & 3]);
                }
                pre = (s4[0] + s4[1]) + (s4[2] + s4[3]);
            }
            if (!ok) st |= (k0 + q < mc) ? 1u : 2u;
            if (low && r == q) {
                v[q] = ok ? piv * inv : piv;
                myinv = inv;
            } else if (!low || r > q) {
                v[q] = s * inv;
            }
        }
    }
    return st;
}

// Left-looking (Crout) factorization of the kb x kb diagonal block of panel
// p with 16 rows below it solved in the same pass (one warp, registers):
// lane r < 16 holds row k0+r of the diagonal block (columns <= r), lane 16+r
// a row below.  At pivot q every lane forms a_rq - sum_{k<q} L_rk L_qk with
// row q of L by shuffles from lane q; lane q's value is the pivot and one
// rsqrt scales the column.  The sum over k < q-1 is formed while pivot
// q-1's rsqrt is in flight (four partial sums), and every lane forms the
// pivot itself from lane q's early-broadcast partial sum, so one shuffle
// sits on the dependent chain per pivot.  A non-positive or NaN pivot is
// kept on the diagonal and its column is zeroed below (the block is
// reported; its log-determinant skips the pivot, as core_Xlogdet does).
// Warps that run it on the same diagonal block form identical factors.
__device__ __forceinline__ unsigned factor_rows(int k0, int kb, int mc, double (&v)[kNB], double &myinv)
{
    const int lane = threadIdx.x & 31;
    const bool low = lane < kNB;
    const int r = low ? lane : lane - kNB;
    unsigned st = 0;
    myinv = 0.0;
    double pre = v[0];
#pragma unroll
    for (int q = 0; q < kNB; ++q) {
        if (q < kb) {
            const double preq = __shfl_sync(0xffffffffu, pre, q);
            double s = pre, piv = preq;
            if (q > 0) {
                const double l = __shfl_sync(0xffffffffu, v[q - 1], q);
                s = fma(-v[q - 1], l, s);
                piv = fma(-l, l, preq);
            }
            const bool ok = piv > 0.0;
            const double inv = ok ? rsqrt(piv) : 0.0;
            if (q + 1 < kNB) {
                double s4[4] = {v[q + 1], 0.0, 0.0, 0.0};
#pragma unroll
                for (int k = 0; k < q; ++k) {
                    const double lk = __shfl_sync(0xffffffffu, v[k], q + 1);
                    s4[k & 3] = fma(-v[k], lk, s4[k & 3]);
                }
                pre = (s4[0] + s4[1]) + (s4[2] + s4[3]);
            }
            if (!ok) st |= (k0 + q < mc) ? 1u : 2u;
            if (low && r == q) {
                v[q] = ok ? piv * inv : piv;
                myinv = inv;
            } else if (!low || r > q) {
                v[q] = s * inv;
            }
        }
    }
    return st;
}

// Another 16 rows below the same diagonal block, after factor_rows: the
// lower lanes keep the factor (L rows in v, the scale of their pivot in
// myinv) and only the upper lanes' rows change, by the same operations in
// the same order as in factor_rows (so the results are identical), without
// the pivot chain.
__device__ __forceinline__ void solve_more_rows(int kb, double (&v)[kNB], double myinv)
{
    const int lane = threadIdx.x & 31;
    const bool low = lane < kNB;
    double pre = v[0];
#pragma unroll
    for (int q = 0; q < kNB; ++q) {
        if (q < kb) {
            const double inv = __shfl_sync(0xffffffffu, myinv, q);
            double s = pre;
            if (q > 0) {
                const double l = __shfl_sync(0xffffffffu, v[q - 1], q);
                s = fma(-v[q - 1], l, s);
            }
            if (q + 1 < kNB) {
                double s4[4] = {v[q + 1], 0.0, 0.0, 0.0};
#pragma unroll
                for (int k = 0; k < q; ++k) {
                    const double lk = __shfl_sync(0xffffffffu, v[k], q + 1);
                    s4[k & 3] = fma(-v[k], lk, s4[k & 3]);
                }
                pre = (s4[0] + s4[1]) + (s4[2] + s4[3]);
            }
            if (!low) v[q] = s * inv;
        }
    }
}

// The factored diagonal block to sh.Lt (transposed), its reciprocal pivots
// to sh.inv, and the rows of panel p+1 to sh.Lnx.
__device__ __forceinline__ void publish_diag(BlockShared &sh, const double (&v)[kNB], double myinv, int kb,
                                             int kb1)
{
    const int lane = threadIdx.x & 31;
    const bool low = lane < kNB;
    const int r = low ? lane : lane - kNB;
    // One store per column for both halves of the warp (per-lane address).
#pragma unroll
    for (int c = 0; c < kNB; ++c) {
        const bool keep = low ? (c <= r && r < kb) : (r < kb1 && c < kb);
        double *dst = low ? &sh.Lt[c][r] : &sh.Lnx[r][c];
        *dst = keep ? v[c] : 0.0;
    }
    if (low) sh.inv[r] = (r < kb) ? myinv : 0.0;
}

__device__ __forceinline__ void dmma_8x8x4(double &c0, double &c1, double a, double b)
{
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
        : "+d"(c0), "+d"(c1)
        : "d"(a), "d"(b));
}

// One (8*NI) x (8*NJ) tile at (i0, j0) of A -= P_I P_J^T, P = panel columns
// k0..k0+kb-1, rows limited to < Mp and columns to < ce, lower part only.
// Fragments (m8n8k4, .row.col): lane l holds A[l>>2][l&3], B[l&3][l>>2] and
// C[l>>2][2(l&3)+{0,1}].
template <int NI, int NJ, int KB>
__device__ __forceinline__ void mma_tile(double *A, int Mp, int k0, int kb_rt, int i0, int j0,
                                         int ce, int excl)
{
    const int kb = KB > 0 ? KB : kb_rt;
    const int lane = threadIdx.x & 31;
    const int r8 = lane >> 2, c4 = lane & 3;
    double acc[NI][NJ][2];
#pragma unroll
    for (int mi = 0; mi < NI; ++mi)
#pragma unroll
        for (int nj = 0; nj < NJ; ++nj) acc[mi][nj][0] = acc[mi][nj][1] = 0.0;
#pragma unroll
    for (int kk = 0; kk < (KB > 0 ? KB : kNB); kk += 4) {
        if (KB == 0 && kk >= kb) break;
        const bool kval = kk + c4 < kb;
        const int o = poff(k0 + (kval ? kk + c4 : 0), Mp);
        double a[NI], b[NJ];
#pragma unroll
        for (int mi = 0; mi < NI; ++mi) {
            const int i = i0 + 8 * mi + r8;
            a[mi] = (kval && i < Mp) ? A[o + i] : 0.0;
        }
#pragma unroll
        for (int nj = 0; nj < NJ; ++nj) {
            const int j = j0 + 8 * nj + r8;
            b[nj] = (kval && j < ce) ? A[o + j] : 0.0;
        }
#pragma unroll
        for (int mi = 0; mi < NI; ++mi)
#pragma unroll
            for (int nj = 0; nj < NJ; ++nj) dmma_8x8x4(acc[mi][nj][0], acc[mi][nj][1], a[mi], b[nj]);
    }
#pragma unroll
    for (int nj = 0; nj < NJ; ++nj) {
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const int j = j0 + 8 * nj + 2 * c4 + e;
            if (j < ce) {
                const int o = poff(j, Mp);
#pragma unroll
                for (int mi = 0; mi < NI; ++mi) {
                    const int i = i0 + 8 * mi + r8;
                    if (i < Mp && i >= j && !(i < excl && j < excl)) A[o + i] -= acc[mi][nj][e];
                }
            }
        }
    }
}

// Warp 0: the diagonal block of panel p (rows/cols k0..k0+kb-1, lower part)
// takes the updates of panels p-2 and p-1, which the bulk updates leave to
// it (FP64 tensor cores, three 8x8 sub-tiles).
__device__ __forceinline__ void update_diag_block(double *A, int Mp, int k0, int kb, int p)
{
    const int lane = threadIdx.x & 31;
    const int r8 = lane >> 2, c4 = lane & 3;
    double acc[3][2] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};  // (0,0), (1,0), (1,1)
    const int qb = p >= 2 ? p - 2 : 0;
    for (int q = qb; q < p; ++q) {
#pragma unroll
        for (int kk = 0; kk < kNB; kk += 4) {
            const int o = poff(q * kNB + kk + c4, Mp);
            const int i0 = k0 + r8, i1 = k0 + 8 + r8;
            const double a0 = (r8 < kb) ? A[o + i0] : 0.0;
            const double a1 = (8 + r8 < kb) ? A[o + i1] : 0.0;
            dmma_8x8x4(acc[0][0], acc[0][1], a0, a0);
            dmma_8x8x4(acc[1][0], acc[1][1], a1, a0);
            dmma_8x8x4(acc[2][0], acc[2][1], a1, a1);
        }
    }
#pragma unroll
    for (int t = 0; t < 3; ++t) {
        const int mi = (t == 0) ? 0 : 1, nj = (t == 2) ? 1 : 0;
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const int ii = 8 * mi + r8, jj = 8 * nj + 2 * c4 + e;
            if (ii < kb && jj < kb && ii >= jj) A[poff(k0 + jj, Mp) + k0 + ii] -= acc[t][e];
        }
    }
}

// ---------------------------------------------------------------------------
// Warp-specialised Cholesky of the first M columns of the packed (M+1)-row
// system.
//
// Warp 0 walks the diagonal: for panel p it applies panels p-2 and p-1 to
// the diagonal block, waits until the critical rows below it are done,
// factors the block together with the rows of panel p+1 (registers), waits
// until the bulk warps are done with the previous factor, publishes the new
// one (Lt, Lnx, inv), signals, and stores panel p+1's rows for its next
// diagonal update.  The critical-rows warp then brings the 16 rows below
// panel p+1 up to date in panel p+1's columns (panel p-1's and panel p's
// contributions) and signals warp 0, while the bulk warps solve the
// remaining rows of panel p and apply panel p-1 to the columns beyond panel
// p+1.  Every element of panel c's columns receives panel q's
// contribution exactly once: q = c-1 and c-2 from warp 0 on the diagonal
// block and from the row work of panel c-1 below it, q <= c-3 from the
// column work of iteration q+1.  Hand-offs are mbarriers with bounded waits;
// while one side runs, the data the other side touches is disjoint (the
// diagonal block and next-panel rows for warp 0; everything below or to the
// right of them for the others).
// ---------------------------------------------------------------------------

// Lanes < nl solve rows base+lane of panel p against L_pp (sh.Lt, sh.inv):
// forward substitution, column q of L_pp read per stage as eight 16-byte
// broadcasts behind a compiler fence so the factor values are not all
// hoisted into registers.  The two values on the dependent chain of step
// q + 1 (1 / L_{q+1,q+1} and L_{q+2,q+1}) are read one step ahead.
// The substitution itself on one row held in w (solve_rows).
__device__ __forceinline__ void solve_row_regs(double (&w)[kNB], int kb, const BlockShared &sh)
{
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
            const double2 *src = reinterpret_cast<const double2 *>(sh.Lt[q]);
#pragma unroll
            for (int h = (q + 2) >> 1; h < kNB / 2; ++h) col[h] = src[h];
            w[q] *= inv_cur;
            if (q + 1 < kNB) w[q + 1] = fma(-w[q], l_cur, w[q + 1]);
#pragma unroll
            for (int c = q + 2; c < kNB; ++c) {
                const double l = (c & 1) ? col[c >> 1].y : col[c >> 1].x;
                w[c] = fma(-w[q], l, w[c]);
            }
        }
    }
}

__device__ __forceinline__ void solve_rows(double *A, int Mp, int k0, int kb, int base, int nl,
                                           const BlockShared &sh)
{
    const int lane = threadIdx.x & 31;
    const int r = base + lane;
    if (lane >= nl || r >= Mp) return;
    int cof[kNB];
#pragma unroll
    for (int c = 0; c < kNB; ++c) cof[c] = poff(k0 + (c < kb ? c : 0), Mp);
    double w[kNB];
#pragma unroll
    for (int c = 0; c < kNB; ++c) w[c] = (c < kb) ? A[cof[c] + r] : 0.0;
    solve_row_regs(w, kb, sh);
#pragma unroll
    for (int c = 0; c < kNB; ++c)
        if (c < kb) A[cof[c] + r] = w[c];
}

// One warp: rows i0..i0+15 (below panel p+1) of panel p+1's columns take
// panel p's contribution (solved rows in A, panel p+1's rows from sh.Lnx) and,
// when prev, panel p-1's (both operands in A), on the FP64 tensor cores.
// Fragments (m8n8k4, .row.col): lane l holds A[l>>2][l&3], B[l&3][l>>2] and
// C[l>>2][2(l&3)+{0,1}].
__device__ __forceinline__ void update_next_rows16(double *A, int Mp, int k0, int kb, int n0, int kb1,
                                                   int i0, bool prev, const BlockShared &sh)
{
    const int lane = threadIdx.x & 31;
    const int r8 = lane >> 2, c4 = lane & 3;
    double acc[2][2][2];
#pragma unroll
    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int nj = 0; nj < 2; ++nj) acc[mi][nj][0] = acc[mi][nj][1] = 0.0;
#pragma unroll
    for (int kk = 0; kk < kNB; kk += 4) {
        const int k = kk + c4;
        const bool kval = k < kb;
        const int o = poff(k0 + (kval ? k : 0), Mp);
        double a[2], b[2];
#pragma unroll
        for (int mi = 0; mi < 2; ++mi) {
            const int i = i0 + 8 * mi + r8;
            a[mi] = (kval && i < Mp) ? A[o + i] : 0.0;
        }
#pragma unroll
        for (int nj = 0; nj < 2; ++nj) b[nj] = sh.Lnx[8 * nj + r8][k];  // B[k][n] = Lnx[n][k]
#pragma unroll
        for (int mi = 0; mi < 2; ++mi)
#pragma unroll
            for (int nj = 0; nj < 2; ++nj) dmma_8x8x4(acc[mi][nj][0], acc[mi][nj][1], a[mi], b[nj]);
    }
    if (prev) {
#pragma unroll
        for (int kk = 0; kk < kNB; kk += 4) {
            const int o = poff(k0 - kNB + kk + c4, Mp);
            double a[2], b[2];
#pragma unroll
            for (int mi = 0; mi < 2; ++mi) {
                const int i = i0 + 8 * mi + r8;
                a[mi] = (i < Mp) ? A[o + i] : 0.0;
            }
#pragma unroll
            for (int nj = 0; nj < 2; ++nj) {
                const int j = 8 * nj + r8;
                b[nj] = (j < kb1) ? A[o + n0 + j] : 0.0;
            }
#pragma unroll
            for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                for (int nj = 0; nj < 2; ++nj) dmma_8x8x4(acc[mi][nj][0], acc[mi][nj][1], a[mi], b[nj]);
        }
    }
#pragma unroll
    for (int nj = 0; nj < 2; ++nj)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const int c = 8 * nj + 2 * c4 + e;
            if (c < kb1) {
                const int o = poff(n0 + c, Mp);
#pragma unroll
                for (int mi = 0; mi < 2; ++mi) {
                    const int i = i0 + 8 * mi + r8;
                    if (i < Mp) A[o + i] -= acc[mi][nj][e];
                }
            }
        }
}

// Roles (512 threads): warp 0 walks the diagonal; warp 4 (the same SM
// sub-partition, idle while warp 0 computes and vice versa) handles the
// critical rows; the 12 warps of sub-partitions 1-3 do the bulk work;
// warps 8 and 12 stay out of the way of warps 0 and 4.
constexpr int kCritWarp = 4;
constexpr int kBulkWarps = kWarps - kWarps / 4;  // warps with (warp & 3) != 0

__device__ __forceinline__ void cholesky_ws(double *A, int M, int mc, BlockShared &sh)
{
    const int Mp = M + 1;
    const int P = (M + kNB - 1) / kNB;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const unsigned base = sh.phase_base;
    const unsigned g0b[2] = {sh.ph_g0[0], sh.ph_g0[1]};
    bool timed_out = false;
    if (warp == 0) {
        for (int p = 0; p < P; ++p) {
            const int k0 = p * kNB, kb = min(kNB, M - k0);
            const int n0 = k0 + kb;
            const int kb1 = max(0, min(kNB, M - n0));
            if (p > 0) {
                // Panels p-2 and p-1 on the diagonal block (their rows here are
                // final: panel p-1's were stored below, panel p-2's by the
                // critical rows of two panels ago), then the rows below.
                update_diag_block(A, Mp, k0, kb, p);
                __syncwarp();
                if (!mbar_wait_bounded(&sh.bar_crit, (base + p - 1) & 1u)) timed_out = true;
            }
            double v[kNB];
            double myinv;
            const unsigned st = factor_diag_regs(A, Mp, k0, kb, n0, kb1, mc, v, myinv);
            if (p > 0 && !mbar_wait_bounded(&sh.bar_free, (base + p - 1) & 1u)) timed_out = true;
            publish_diag(sh, v, myinv, kb, kb1);
            if (lane == 0 && st) atomicOr(&sh.status, st);
            // __syncwarp orders the lanes' writes before lane 0's arrive, whose
            // release semantics (CTA scope) publish them to the waiters.
            __syncwarp();
            if (lane == 0) mbar_arrive(&sh.bar_lready);
            // Panel p+1's rows in panel p's columns, for the next diagonal update.
            if (lane >= kNB && lane - kNB < kb1) {
#pragma unroll
                for (int c = 0; c < kNB; ++c)
                    if (c < kb) A[poff(k0 + c, Mp) + n0 + (lane - kNB)] = v[c];
            }
            __syncwarp();
        }
    } else if (warp == kCritWarp) {
        for (int p = 0; p < P; ++p) {
            const int k0 = p * kNB, kb = min(kNB, M - k0);
            const int n0 = k0 + kb;
            const int kb1 = max(0, min(kNB, M - n0));
            const int n1 = n0 + kb1;
            const int n2 = min(Mp, n1 + kNB);
            // The 16 rows below panel p+1: solved in panel p, then brought up
            // to date in panel p+1's columns (panels p and p-1).  Their panel-p
            // values are read while warp 0 still factors: final once the
            // previous panel's first bulk row group (these rows, when the
            // previous panel had bulk groups) has taken its update.
            {
                const int r = n1 + lane;
                const bool act = lane < n2 - n1;
                if (p > 0 && Mp > min(Mp, min(kNB * (p + 1), M) + kNB)) {
                    const int k = (p - 1) & 1;
                    if (!mbar_wait_bounded(&sh.bar_g0[k], (g0b[k] + ((p - 1) >> 1)) & 1u)) timed_out = true;
                }
                int cof[kNB];
                {
                    int o = poff(k0, Mp);
#pragma unroll
                    for (int c = 0; c < kNB; ++c) {
                        cof[c] = o;
                        o += Mp - (k0 + c) - 1;
                    }
                }
                double w[kNB];
#pragma unroll
                for (int c = 0; c < kNB; ++c) w[c] = (act && c < kb) ? A[cof[c] + r] : 0.0;
                if (!mbar_wait_bounded(&sh.bar_lready, (base + p) & 1u)) timed_out = true;
                if (act) {
                    solve_row_regs(w, kb, sh);
#pragma unroll
                    for (int c = 0; c < kNB; ++c)
                        if (c < kb) A[cof[c] + r] = w[c];
                }
            }
            __syncwarp();
            if (kb1 > 0 && n2 > n1) update_next_rows16(A, Mp, k0, kb, n0, kb1, n1, p > 0, sh);
            __syncwarp();
            if (lane == 0) mbar_arrive(&sh.bar_crit);
        }
    } else if ((warp & 3) != 0) {
        const int wb = warp - (warp >> 2) - 1;
        for (int p = 0; p < P; ++p) {
            const int k0 = p * kNB, kb = min(kNB, M - k0);
            const int n0 = k0 + kb;
            const int kb1 = max(0, min(kNB, M - n0));
            const int n1 = n0 + kb1;
            const int n2 = min(Mp, n1 + kNB);
            if (!mbar_wait_bounded(&sh.bar_lready, (base + p) & 1u)) timed_out = true;
            // The factored diagonal block into A.
            {
                const int t = wb * 32 + lane;
                if (t < kNB * kNB) {
                    const int c = t >> 4, r = t & 15;
                    if (c < kb && r < kb && r >= c) A[poff(k0 + c, Mp) + k0 + r] = sh.Lt[c][r];
                }
            }
            // Work items, taken by the warps in turn from a shared counter (the
            // next index is fetched while the current item runs): first the
            // rows >= n2 in 32-row groups (solve, then panel p+1's columns take
            // panels p and p-1; the longest items), then panel p-1 on the
            // columns beyond panel p+1 in 32 x 16 tiles, column tile tc
            // covering row tiles tc/2 .. TR-1.
            const int G = (Mp > n2) ? (Mp - n2 + 31) >> 5 : 0;
            const int TR = (Mp - n1 + 31) >> 5;
            const int TC = (p > 0 && M > n1) ? (M - n1 + 15) >> 4 : 0;
            const int total = G + TC * TR - ((TC - 1) * (TC - 1)) / 4;
            int *ctr = &sh.bulk_next[p & 1];
            int item = __shfl_sync(0xffffffffu, lane == 0 ? atomicAdd(ctr, 1) : 0, 0);
            while (item < total) {
                const int raw = (lane == 0) ? atomicAdd(ctr, 1) : 0;
                if (item < G) {
                    const int rb = n2 + 32 * item;
                    solve_rows(A, Mp, k0, kb, rb, 32, sh);
                    __syncwarp();
                    if (kb1 > 0) {
                        update_next_rows16(A, Mp, k0, kb, n0, kb1, rb, p > 0, sh);
                        if (item == 0) {
                            // The next panel's critical rows are up to date.
                            __syncwarp();
                            if (lane == 0) mbar_arrive(&sh.bar_g0[p & 1]);
                        }
                        if (rb + 16 < Mp) update_next_rows16(A, Mp, k0, kb, n0, kb1, rb + 16, p > 0, sh);
                    }
                } else {
                    int t = item - G, tc = 0;
                    while (t >= TR - (tc >> 1)) t -= TR - (tc++ >> 1);
                    mma_tile<4, 2, kNB>(A, Mp, k0 - kNB, kNB, n1 + (((tc >> 1) + t) << 5), n1 + tc * 16, M, 0);
                }
                item = __shfl_sync(0xffffffffu, raw, 0);
            }
            asm volatile("bar.sync 1, %0;" ::"n"(kBulkWarps * 32) : "memory");
            if (tid == 32) {
                *ctr = 0;  // every bulk warp is done with it; reused two panels on
                mbar_arrive(&sh.bar_free);
            }
        }
    }
    if (timed_out) atomicOr(&sh.status, kStDeviceTimeout);
    __syncthreads();
    if (tid == 0) {
        sh.phase_base = base + (unsigned)P;
        // bar_g0[k] took one arrival per panel p = k, k+2, ... with bulk row
        // groups (those panels are a prefix 0..pg-1).
        int pg = 0;
        while (pg < P && Mp > min(Mp, min(kNB * (pg + 2), M) + kNB)) ++pg;
        sh.ph_g0[0] = g0b[0] + (unsigned)((pg + 1) >> 1);
        sh.ph_g0[1] = g0b[1] + (unsigned)(pg >> 1);
    }
}

// ---------------------------------------------------------------------------
// Panel-parallel Cholesky of the first M columns of the packed (M+1)-row
// system, right-looking with a look-ahead of one panel.
//
// Chain warps (0-11): for panel p each runs the 16-pivot factorization of the
// diagonal block together with 16 rows of its own below it (slice w of the
// rows from c1, the first row below the block; slices w + 12, ... reuse the
// factor by substitution), so the whole panel column is factored and solved
// in one pass of the dependent chain with no separate triangular solve;
// every warp forms the same pivots.  They store their rows, meet at a
// barrier (warp 0 then stores the diagonal block and signals the bulk warps),
// wait until panel p+1's columns have taken panel p-1, apply panel p to their
// own rows in panel p+1's columns (the look-ahead; panel p+1's rows are warp
// 0's first 16) and meet again: panel p+1's columns are then final for the
// next factorization.  Bulk warps (12-15): for panel p they apply panel p-1
// to panel p+1's columns, signal, then apply it to the columns beyond, in
// 32 x 16 tiles taken from a shared counter.  Every element of panel c's
// columns receives panel q's contribution exactly once: q = c-1 from the
// look-ahead of iteration c-1, q <= c-2 from the bulk work of iteration q+1.
// The two signals are mbarriers with bounded waits, one per parity of p, so
// neither side can run two phases ahead of the other.
// ---------------------------------------------------------------------------
constexpr int kChainWarps = 12;
#ifndef BV_PP_MAX_M
#define BV_PP_MAX_M 190
#endif
constexpr int kPpMaxM = BV_PP_MAX_M;
constexpr int kPpBulkWarps = kWarps - kChainWarps;

__device__ __forceinline__ void cholesky_pp(double *A, int M, int mc, BlockShared &sh)
{
    const int Mp = M + 1;
    const int P = (M + kNB - 1) / kNB;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const unsigned bl[2] = {sh.ph_ls[0], sh.ph_ls[1]};
    const unsigned bn[2] = {sh.ph_nc[0], sh.ph_nc[1]};
    bool timed_out = false;
    if (warp < kChainWarps) {
        const bool low = lane < kNB;
        const int r = low ? lane : lane - kNB;
        for (int p = 0; p < P; ++p) {
            const int k0 = p * kNB, kb = min(kNB, M - k0);
            const int c1 = k0 + kb;
            const int kb1 = max(0, min(kNB, M - c1));
            // Slices of 16 rows below the diagonal block: w, w + 12, ... (the
            // first is panel p+1's rows, warp 0's, and warp 0 always runs).
            // The first slice of a warp runs with the factorization, the
            // others reuse the factor it leaves in the lower lanes.
            unsigned st = 0;
            if (warp == 0 || c1 + kNB * warp < Mp) {
                double v[kNB], myinv;
                {
                    const int row = c1 + kNB * warp + r;
                    const bool valid = !low && row < Mp;
#pragma unroll
                    for (int c = 0; c < kNB; ++c) {
                        const bool in = low ? (r < kb && c <= r) : valid;
                        v[c] = (in && c < kb) ? A[poff(k0 + c, Mp) + (low ? k0 + r : row)] : 0.0;
                    }
                    st = factor_rows(k0, kb, mc, v, myinv);
                    if (warp == 0 && low) {
                        // Warp 0's diagonal factor waits in sh.Lt (transposed)
                        // until every chain warp has read the block from A.
#pragma unroll
                        for (int c = 0; c < kNB; ++c) sh.Lt[c][r] = v[c];
                    }
                    if (valid) {
#pragma unroll
                        for (int c = 0; c < kNB; ++c)
                            if (c < kb) A[poff(k0 + c, Mp) + row] = v[c];
                    }
                }
#pragma unroll 1
                for (int sl = warp + kChainWarps; c1 + kNB * sl < Mp; sl += kChainWarps) {
                    const int row = c1 + kNB * sl + r;
                    const bool valid = !low && row < Mp;
                    if (!low) {
#pragma unroll
                        for (int c = 0; c < kNB; ++c) v[c] = (valid && c < kb) ? A[poff(k0 + c, Mp) + row] : 0.0;
                    }
                    solve_more_rows(kb, v, myinv);
                    if (valid) {
#pragma unroll
                        for (int c = 0; c < kNB; ++c)
                            if (c < kb) A[poff(k0 + c, Mp) + row] = v[c];
                    }
                }
            }
            // Every chain warp has read the diagonal block and stored its rows.
            asm volatile("bar.sync 2, %0;" ::"n"(kChainWarps * 32) : "memory");
            if (warp == 0 && lane == 0) {
                if (st) atomicOr(&sh.status, st);
                mbar_arrive(&sh.bar_ls[p & 1]);
            }
            if (warp == kChainWarps - 1) {
                // The diagonal factor into A (off warp 0's path; the last
                // chain warp has the least look-ahead work).
                double l[kNB * kNB / 32];
#pragma unroll
                for (int i = 0; i < kNB * kNB / 32; ++i) {
                    const int t = lane + 32 * i;
                    l[i] = sh.Lt[t >> 4][t & 15];
                }
#pragma unroll
                for (int i = 0; i < kNB * kNB / 32; ++i) {
                    const int t = lane + 32 * i, c = t >> 4, rr = t & 15;
                    if (c < kb && rr < kb && rr >= c) A[poff(k0 + c, Mp) + k0 + rr] = l[i];
                }
            }
            if (!mbar_wait_bounded(&sh.bar_nc[p & 1], (bn[p & 1] + (p >> 1)) & 1u)) timed_out = true;
            if (kb1 > 0) {
                for (int sl = warp; c1 + kNB * sl < Mp; sl += kChainWarps)
                    mma_tile<2, 2, kNB>(A, Mp, k0, kNB, c1 + kNB * sl, c1, c1 + kb1, 0);
            }
            asm volatile("bar.sync 2, %0;" ::"n"(kChainWarps * 32) : "memory");
        }
    } else {
        const int first = kChainWarps * 32;
        for (int p = 0; p < P; ++p) {
            const int k0 = p * kNB, kb = min(kNB, M - k0);
            const int c1 = k0 + kb;
            const int kb1 = max(0, min(kNB, M - c1));
            const int c2 = c1 + kb1;
            if (p > 0 && !mbar_wait_bounded(&sh.bar_ls[(p - 1) & 1], (bl[(p - 1) & 1] + ((p - 1) >> 1)) & 1u))
                timed_out = true;
            // Panel p-1 on panel p+1's columns, 32-row tiles from its diagonal down.
            {
                const int total = (p > 0 && kb1 > 0) ? (Mp - c1 + 31) >> 5 : 0;
                int *ctr = &sh.work_next[(2 * p) & 3];
                int item = __shfl_sync(0xffffffffu, lane == 0 ? atomicAdd(ctr, 1) : 0, 0);
                while (item < total) {
                    const int raw = (lane == 0) ? atomicAdd(ctr, 1) : 0;
                    mma_tile<4, 2, kNB>(A, Mp, k0 - kNB, kNB, c1 + 32 * item, c1, c2, 0);
                    item = __shfl_sync(0xffffffffu, raw, 0);
                }
            }
            asm volatile("bar.sync 1, %0;" ::"n"(kPpBulkWarps * 32) : "memory");
            if (tid == first) {
                sh.work_next[(2 * p) & 3] = 0;
                mbar_arrive(&sh.bar_nc[p & 1]);
            }
            // Panel p-1 on the columns beyond panel p+1: column tile tc covers
            // row tiles tc/2 .. TR-1.
            {
                const int TR = (Mp - c2 + 31) >> 5;
                const int TC = (p > 0 && M > c2) ? (M - c2 + 15) >> 4 : 0;
                const int total = TC * TR - ((TC - 1) * (TC - 1)) / 4;
                int *ctr = &sh.work_next[(2 * p + 1) & 3];
                int item = __shfl_sync(0xffffffffu, lane == 0 ? atomicAdd(ctr, 1) : 0, 0);
                while (item < total) {
                    const int raw = (lane == 0) ? atomicAdd(ctr, 1) : 0;
                    int t = item, tc = 0;
                    while (t >= TR - (tc >> 1)) t -= TR - (tc++ >> 1);
                    mma_tile<4, 2, kNB>(A, Mp, k0 - kNB, kNB, c2 + (((tc >> 1) + t) << 5), c2 + tc * 16, M, 0);
                    item = __shfl_sync(0xffffffffu, raw, 0);
                }
            }
            asm volatile("bar.sync 1, %0;" ::"n"(kPpBulkWarps * 32) : "memory");
            if (tid == first) sh.work_next[(2 * p + 1) & 3] = 0;
        }
    }
    if (timed_out) atomicOr(&sh.status, kStDeviceTimeout);
    __syncthreads();
    if (tid == 0) {
        sh.ph_ls[0] = bl[0] + (unsigned)((P + 1) >> 1);
        sh.ph_ls[1] = bl[1] + (unsigned)(P >> 1);
        sh.ph_nc[0] = bn[0] + (unsigned)((P + 1) >> 1);
        sh.ph_nc[1] = bn[1] + (unsigned)(P >> 1);
    }
}

// One block, with its matrix at A (shared memory or the global slab); T
// holds the third coordinate of 3-D locations (kXYZ3; unused for 2-D).
template <bool kXYZ3>
__device__ __forceinline__ void process_block(const LlhArgs &a, const MaternParams &mp, int b,
                                              double *X, double *Y, double *T, double *A,
                                              BlockShared &sh)
{
    const int tid = threadIdx.x;
    const int off = a.acc[b];
    const int bs = a.acc[b + 1] - off;
    const int mc = (b == 0) ? 0 : a.cs;
    const int M = mc + bs, Mp = M + 1;

    // Gather: conditioning points by index, then the block's own points;
    // observations go to row M.
    const int *kidx = a.knn + (size_t)b * a.cs;
    for (int t = tid; t < M; t += kThreads) {
        const int src = (t < mc) ? __ldg(kidx + t) : off + (t - mc);
        X[t] = __ldg(a.x + src);
        Y[t] = __ldg(a.y + src);
        if constexpr (kXYZ3) T[t] = __ldg(a.z + src);
        A[poff(t, Mp) + M] = __ldg(a.obs + src);
    }
    __syncthreads();
    generate<kXYZ3>(A, X, Y, T, M, mp);
    __syncthreads();
    if (mp.nugget != 0.0) {
        // Nugget: tau^2 on the diagonal of Sigma22 and Sigma11 (a point with
        // itself), not on other pairs at distance 0.
        for (int t = tid; t < M; t += kThreads) A[poff(t, Mp) + t] += mp.nugget;
        __syncthreads();
    }

    // Cholesky of the first M columns; row M rides along as the
    // forward-substitution right-hand side.
    if (M <= kPpMaxM)
        cholesky_pp(A, M, mc, sh);
    else
        cholesky_ws(A, M, mc, sh);

    // log det of the conditional factor (positive pivots only, as
    // core_Xlogdet) and |u|^2 from row M.
    double ld = 0.0, qf = 0.0;
    for (int j = mc + tid; j < M; j += kThreads) {
        const double d = A[poff(j, Mp) + j];
        if (d > 0) ld += log(d * d);
        const double u = A[poff(j, Mp) + M];
        qf = fma(u, u, qf);
    }
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) {
        ld += __shfl_xor_sync(0xffffffffu, ld, s);
        qf += __shfl_xor_sync(0xffffffffu, qf, s);
    }
    if ((tid & 31) == 0) {
        sh.red[0][tid >> 5] = ld;
        sh.red[1][tid >> 5] = qf;
    }
    __syncthreads();
    if (tid == 0) {
        double Ls = 0.0, Qs = 0.0;
        for (int w = 0; w < kWarps; ++w) {
            Ls += sh.red[0][w];
            Qs += sh.red[1][w];
        }
        const double v = -(Qs + Ls + (double)bs * a.log2pi) * 0.5;
        unsigned st = sh.status;
        if (!isfinite(v)) st |= 8u;
        a.block_llk[b] = v;
        a.block_status[b] = st | a.status_or;
    }
}

}  // namespace bv

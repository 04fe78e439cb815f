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

#include "bv_matern.cuh"

namespace bv {

constexpr int kThreads = 512;
constexpr int kWarps = kThreads / 32;
constexpr int kNB = 16;  // panel width of the blocked Cholesky

struct LlhArgs {
    const double *x, *y, *obs;  // [n] block-ordered
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
};

__host__ __device__ inline size_t packed_elems(int Mp) { return (size_t)Mp * (Mp + 1) / 2; }

// Doubles a block of size M needs: x[M], y[M], packed (M+1)-row triangle.
__host__ __device__ inline size_t block_doubles(int M) { return 2 * (size_t)M + packed_elems(M + 1); }

__device__ __forceinline__ int poff(int j, int Mp) { return j * Mp - ((j * (j + 1)) >> 1); }

// Shared scratch of the kernel besides the block itself.
struct alignas(16) BlockShared {
    double L[kNB][kNB + 1];  // factored diagonal block of the current panel
    double Lt[kNB][kNB];     // its transpose: Lt[q][c] = L_(c,q), column q contiguous
    double inv[kNB];         // 1 / L_jj of the current panel (0: failed pivot)
    double red[2][kWarps];
    unsigned status;
    int task;
};

// ---------------------------------------------------------------------------
// Matern generation.
// ---------------------------------------------------------------------------

// Lower triangle of rows 0..M-1 with columns paired (q, M-1-q) so each pair
// holds M+1 entries; warp w takes pairs w, w+16, ...; a lane computes four
// entries of a pair at a time.
__device__ __forceinline__ void generate(double *A, const double *X, const double *Y, int M,
                                         const MaternParams &mp)
{
    const int Mp = M + 1;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int half = (M + 1) >> 1;
    for (int q = warp; q < half; q += kWarps) {
        const int jb = M - 1 - q;          // partner column
        const int na = M - q;              // rows q..M-1 of column q
        const int nt = (jb == q) ? na : M + 1;
        const int oa = poff(q, Mp), ob = poff(jb, Mp);
        const double xq = X[q], yq = Y[q], xb = X[jb], yb = Y[jb];
        for (int r0 = lane; r0 < nt; r0 += 128) {
            double v[4];
            int dst[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int rr = r0 + 32 * u;
                dst[u] = -1;
                v[u] = 0.0;
                if (rr < nt) {
                    int i;
                    double xj, yj;
                    if (rr < na) {
                        i = q + rr;
                        xj = xq;
                        yj = yq;
                        dst[u] = oa + i;
                    } else {
                        i = jb + (rr - na);
                        xj = xb;
                        yj = yb;
                        dst[u] = ob + i;
                    }
                    v[u] = matern(X[i], Y[i], xj, yj, mp);
                }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (dst[u] >= 0) A[dst[u]] = v[u];
        }
    }
}

// ---------------------------------------------------------------------------
// Panel factorization pieces.
// ---------------------------------------------------------------------------

// Factor the kb x kb diagonal block at k0 with warp 0.  Lane r owns row k0+r.
// Per pivot: the owner's value is broadcast, every lane takes one rsqrt, the
// pivot column is scaled and broadcast by shuffles, and the block's remaining
// columns take a rank-1 update.  A non-positive or NaN pivot is kept on the
// diagonal and its column is zeroed below (the block is then reported; its
// log-determinant skips the pivot, as core_Xlogdet does).  The factor also
// goes to sh.L and 1/L_jj to sh.inv (0 for a failed pivot).
__device__ __forceinline__ unsigned factor_diag(double *A, int Mp, int k0, int kb, int mc,
                                                BlockShared &sh)
{
    const int lane = threadIdx.x & 31;
    double v[kNB];
#pragma unroll
    for (int c = 0; c < kNB; ++c)
        v[c] = (lane < kb && c <= lane && c < kb) ? A[poff(k0 + c, Mp) + k0 + lane] : 0.0;
    unsigned st = 0;
#pragma unroll
    for (int q = 0; q < kNB; ++q) {
        if (q < kb) {
            const double piv = __shfl_sync(0xffffffffu, v[q], q);
            const bool ok = piv > 0.0;
            const double inv = ok ? rsqrt(piv) : 0.0;
            if (!ok) st |= (k0 + q < mc) ? 1u : 2u;
            if (lane == q) {
                v[q] = ok ? piv * inv : piv;
                sh.inv[q] = inv;
            } else if (lane > q) {
                v[q] *= inv;
            }
            const double lq = (lane > q) ? v[q] : 0.0;
#pragma unroll
            for (int c = q + 1; c < kNB; ++c) {
                const double lc = __shfl_sync(0xffffffffu, lq, c);
                if (c <= lane) v[c] = fma(-lq, lc, v[c]);
            }
        }
    }
    if (lane < kb) {
#pragma unroll
        for (int c = 0; c < kNB; ++c) {
            if (c <= lane && c < kb) {
                A[poff(k0 + c, Mp) + k0 + lane] = v[c];
                sh.L[lane][c] = v[c];
            }
        }
    }
    if (lane < kNB) {
#pragma unroll
        for (int c = 0; c < kNB; ++c) sh.Lt[c][lane] = (c < lane && lane < kb) ? v[c] : 0.0;
    }
    return st;
}

// Rows i in [k0+kb, Mp): A(i, k0:k0+kb) <- A(i, k0:k0+kb) L_kk^-T
// (forward substitution against the factored diagonal block).  Column q of
// L_kk is read per stage as eight 16-byte broadcasts; a compiler fence keeps
// the stages' loads from being hoisted into registers all at once.
__device__ __forceinline__ void panel_trsm(double *A, int Mp, int k0, int kb,
                                           const BlockShared &sh)
{
    int cof[kNB];
#pragma unroll
    for (int c = 0; c < kNB; ++c) cof[c] = poff(k0 + (c < kb ? c : 0), Mp);
    for (int i = k0 + kb + threadIdx.x; i < Mp; i += kThreads) {
        double w[kNB];
#pragma unroll
        for (int c = 0; c < kNB; ++c) w[c] = (c < kb) ? A[cof[c] + i] : 0.0;
#pragma unroll
        for (int q = 0; q < kNB; ++q) {
            if (q < kb) {
                asm volatile("" ::: "memory");
                double2 col[kNB / 2];
                const double2 *src = reinterpret_cast<const double2 *>(sh.Lt[q]);
#pragma unroll
                for (int h = 0; h < kNB / 2; ++h) col[h] = src[h];
                w[q] *= sh.inv[q];
#pragma unroll
                for (int c = q + 1; c < kNB; ++c) {
                    const double l = (c & 1) ? col[c >> 1].y : col[c >> 1].x;
                    w[c] = fma(-w[q], l, w[c]);
                }
            }
        }
#pragma unroll
        for (int c = 0; c < kNB; ++c)
            if (c < kb) A[cof[c] + i] = w[c];
    }
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
                                         int ce)
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
                    if (i < Mp && i >= j) A[o + i] -= acc[mi][nj][e];
                }
            }
        }
    }
}

// Rows [cb, Mp) x cols [cb, ce) (lower part) with panel k0..k0+kb-1, by warps
// [w0, w0+nw), in tiles of 32 rows x (8*NJ) columns.
// skip_sp0: leave the warps of sub-partition 0 (ids = 0 mod 4) out, so warp
// 0's diagonal factorization does not queue behind their tensor-core work.
template <int NJ>
__device__ __forceinline__ void update_cols(double *A, int Mp, int k0, int kb, int cb, int ce,
                                            bool skip_sp0)
{
    constexpr int TW = 8 * NJ;
    const int nrow = Mp - cb, ncol = ce - cb;
    if (nrow <= 0 || ncol <= 0) return;
    const int wid = threadIdx.x >> 5;
    int warp, nw;
    if (skip_sp0) {
        if ((wid & 3) == 0) return;
        warp = wid - (wid >> 2) - 1;
        nw = kWarps - kWarps / 4;
    } else {
        warp = wid;
        nw = kWarps;
    }
    const int TR = (nrow + 31) >> 5, TC = (ncol + TW - 1) / TW;
    // Enumerate lower tiles (tc, tr >= first row tile reaching column tile tc).
    int t = 0;
    for (int tc = 0; tc < TC; ++tc) {
        const int j0 = cb + tc * TW;
        const int tr0 = (j0 - cb) >> 5;
        for (int tr = tr0; tr < TR; ++tr, ++t) {
            if (t % nw != warp) continue;
            if (kb == kNB)
                mma_tile<4, NJ, kNB>(A, Mp, k0, kb, cb + (tr << 5), j0, ce);
            else
                mma_tile<4, NJ, 0>(A, Mp, k0, kb, cb + (tr << 5), j0, ce);
        }
    }
}

// Blocked right-looking Cholesky of the first M columns of the packed
// (M+1)-row system with one panel of look-ahead.
__device__ __forceinline__ void cholesky_lookahead(double *A, int M, int mc, BlockShared &sh)
{
    const int Mp = M + 1;
    const int P = (M + kNB - 1) / kNB;
    const int tid = threadIdx.x;
    for (int p = 0; p < P; ++p) {
        const int k0 = p * kNB, kb = min(kNB, M - k0);
        const int n0 = k0 + kb;           // first column after panel p
        const int n1 = min(M, n0 + kNB);  // end of panel p+1
        if (tid < 32) {
            const unsigned st = factor_diag(A, Mp, k0, kb, mc, sh);
            if (tid == 0 && st) sh.status |= st;
        } else if (p > 0) {
            // Deferred update with panel p-1 of the columns beyond panel p
            // (warps outside sub-partition 0).
            update_cols<2>(A, Mp, k0 - kNB, kNB, n0, M, true);
        }
        __syncthreads();
        panel_trsm(A, Mp, k0, kb, sh);
        __syncthreads();
        if (n0 < M) {
            // Look-ahead: panel p+1's columns with panel p.
            update_cols<2>(A, Mp, k0, kb, n0, n1, false);
            __syncthreads();
        }
    }
}

// One block, with its matrix at A (shared memory or the global slab).
__device__ __forceinline__ void process_block(const LlhArgs &a, const MaternParams &mp, int b,
                                              double *X, double *Y, double *A, BlockShared &sh)
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
        A[poff(t, Mp) + M] = __ldg(a.obs + src);
    }
    __syncthreads();
    generate(A, X, Y, M, mp);
    __syncthreads();

    // Cholesky of the first M columns; row M rides along as the
    // forward-substitution right-hand side.
    cholesky_lookahead(A, M, mc, sh);

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
        a.block_status[b] = st;
    }
}

// ---------------------------------------------------------------------------
// The kernel.
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(kThreads, 1) llh_fp64_kernel(LlhArgs a)
{
    extern __shared__ __align__(16) double smem[];
    __shared__ BlockShared sh;

    const MaternParams mp = *a.mp;
    const int tid = threadIdx.x;

    for (;;) {
        if (tid == 0) sh.task = (int)atomicAdd(a.work_counter, 1u) + a.task_begin;
        __syncthreads();
        const int task = sh.task;
        if (task >= a.task_end) break;
        const int b = a.order[task];
        const int bs = a.acc[b + 1] - a.acc[b];
        const int M = ((b == 0) ? 0 : a.cs) + bs;
        if (tid == 0) sh.status = 0u;

        if (bs == 0) {  // empty block: contributes -(0 + 0 + 0) / 2
            if (tid == 0) {
                a.block_llk[b] = -0.0;
                a.block_status[b] = 0u;
            }
        } else if (M <= a.smem_max_m) {
            process_block(a, mp, b, smem, smem + M, smem + 2 * M, sh);
        } else {
            double *slab = a.gslab + (size_t)blockIdx.x * a.gslab_stride;
            process_block(a, mp, b, slab, slab + M, slab + 2 * M, sh);
        }
        __syncthreads();
    }
}

}  // namespace bv

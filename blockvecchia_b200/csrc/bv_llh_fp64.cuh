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
#pragma once

#include "bv_matern.cuh"

namespace bv {

constexpr int kThreads = 256;
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

// ---------------------------------------------------------------------------
// Panel factorization pieces.
// ---------------------------------------------------------------------------

// Factor the kb x kb diagonal block at k0 with warp 0.  Lane r owns row k0+r.
// A non-positive or NaN pivot is kept on the diagonal and its column is
// zeroed below (the block is then reported; its log-determinant skips the
// pivot, as core_Xlogdet does).  s_inv receives 1/L_jj (0 for a failed
// pivot).  Returns a status mask in lane 0.
__device__ __forceinline__ unsigned factor_diag(double *A, int Mp, int k0, int kb, int mc,
                                                double *s_inv)
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
            double d, inv;
            if (piv > 0.0) {
                d = sqrt(piv);
                inv = 1.0 / d;
            } else {
                d = piv;
                inv = 0.0;
                st |= (k0 + q < mc) ? 1u : 2u;
            }
            if (lane == q) {
                v[q] = d;
                s_inv[q] = inv;
            } else if (lane > q) {
                v[q] *= inv;
            }
            const double lq = v[q];
#pragma unroll
            for (int c = q + 1; c < kNB; ++c) {
                const double lc = __shfl_sync(0xffffffffu, lq, c);
                if (c <= lane && c < kb) v[c] = fma(-lq, lc, v[c]);
            }
        }
    }
    if (lane < kb) {
#pragma unroll
        for (int c = 0; c < kNB; ++c)
            if (c <= lane && c < kb) A[poff(k0 + c, Mp) + k0 + lane] = v[c];
    }
    return st;
}

// Rows i in [k0+kb, Mp): A(i, k0:k0+kb) <- A(i, k0:k0+kb) L_kk^-T.
__device__ __forceinline__ void panel_trsm(double *A, int Mp, int k0, int kb, const double *s_inv)
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
                w[q] *= s_inv[q];
#pragma unroll
                for (int c = q + 1; c < kNB; ++c)
                    if (c < kb) w[c] = fma(-w[q], A[cof[q] + k0 + c], w[c]);
            }
        }
#pragma unroll
        for (int c = 0; c < kNB; ++c)
            if (c < kb) A[cof[c] + i] = w[c];
    }
}

// Trailing update of rows [c0, Mp) x cols [c0, Mc), lower part, with the
// panel columns k0..k0+kb-1.  Each warp owns 32 x 32 tiles; lane (lr, lc) =
// (lane & 7, lane >> 3) holds rows i0 + lr + 8r (r < 4), cols j0 + lc + 4c
// (c < 8), so every shared load is a broadcast over at most 8 consecutive
// doubles.
__device__ __forceinline__ void trailing_update(double *A, int Mp, int Mc, int k0, int kb)
{
    const int c0 = k0 + kb;
    const int nrow = Mp - c0, ncol = Mc - c0;
    if (nrow <= 0 || ncol <= 0) return;
    const int TR = (nrow + 31) >> 5, TC = (ncol + 31) >> 5;
    // Lower tiles: tr >= tc.  Count = sum_{tc < TC} (TR - tc).
    const int ntiles = TC * TR - (TC * (TC - 1)) / 2;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int lr = lane & 7, lc = lane >> 3;
    for (int t = warp; t < ntiles; t += kWarps) {
        int tc = 0, rem = t;
        while (rem >= TR - tc) {
            rem -= TR - tc;
            ++tc;
        }
        const int tr = tc + rem;
        const int i0 = c0 + (tr << 5), j0 = c0 + (tc << 5);
        double acc[4][8];
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int c = 0; c < 8; ++c) acc[r][c] = 0.0;
        for (int kk = 0; kk < kb; ++kk) {
            const int o = poff(k0 + kk, Mp);
            double a[4], b[8];
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int i = i0 + lr + 8 * r;
                a[r] = (i < Mp) ? A[o + i] : 0.0;
            }
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                const int j = j0 + lc + 4 * c;
                b[c] = (j < Mc) ? A[o + j] : 0.0;
            }
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int c = 0; c < 8; ++c) acc[r][c] = fma(a[r], b[c], acc[r][c]);
        }
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const int j = j0 + lc + 4 * c;
            if (j < Mc) {
                const int o = poff(j, Mp);
#pragma unroll
                for (int r = 0; r < 4; ++r) {
                    const int i = i0 + lr + 8 * r;
                    if (i < Mp && i >= j) A[o + i] -= acc[r][c];
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// The kernel.
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(kThreads, 1) llh_fp64_kernel(LlhArgs a)
{
    extern __shared__ __align__(16) double smem[];
    __shared__ int s_task;
    __shared__ double s_inv[kNB];
    __shared__ unsigned s_status;
    __shared__ double s_red[2][kWarps];

    const MaternParams mp = *a.mp;
    const int tid = threadIdx.x;

    for (;;) {
        if (tid == 0) s_task = (int)atomicAdd(a.work_counter, 1u) + a.task_begin;
        __syncthreads();
        const int task = s_task;
        if (task >= a.task_end) break;
        const int b = a.order[task];
        const int off = a.acc[b];
        const int bs = a.acc[b + 1] - off;
        const int mc = (b == 0) ? 0 : a.cs;
        const int M = mc + bs, Mp = M + 1;

        if (bs == 0) {  // empty block: contributes -(0 + 0 + 0) / 2
            if (tid == 0) {
                a.block_llk[b] = -0.0;
                a.block_status[b] = 0u;
            }
            __syncthreads();
            continue;
        }

        double *X, *Y, *A;
        if (M <= a.smem_max_m) {
            X = smem;
            Y = smem + M;
            A = smem + 2 * M;
        } else {
            double *slab = a.gslab + (size_t)blockIdx.x * a.gslab_stride;
            X = slab;
            Y = slab + M;
            A = slab + 2 * M;
        }
        if (tid == 0) s_status = 0u;

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

        // Matern lower triangle, columns paired (q, M-1-q) so every pair holds
        // M+1 entries.
        {
            const int half = (M + 1) >> 1;
            const int total = half * (M + 1);
            for (int e = tid; e < total; e += kThreads) {
                const int q = e / (M + 1);
                const int rr = e - q * (M + 1);
                int i, j;
                if (rr < M - q) {
                    j = q;
                    i = q + rr;
                } else {
                    j = M - 1 - q;
                    if (j == q) continue;  // odd M: middle column counted once
                    i = j + (rr - (M - q));
                }
                A[poff(j, Mp) + i] = matern(X[i], Y[i], X[j], Y[j], mp);
            }
        }
        __syncthreads();

        // Blocked right-looking Cholesky of the first M columns; row M rides
        // along as the forward-substitution right-hand side.
        for (int k0 = 0; k0 < M; k0 += kNB) {
            const int kb = min(kNB, M - k0);
            if (tid < 32) {
                const unsigned st = factor_diag(A, Mp, k0, kb, mc, s_inv);
                if (tid == 0 && st) s_status |= st;
            }
            __syncthreads();
            panel_trsm(A, Mp, k0, kb, s_inv);
            __syncthreads();
            trailing_update(A, Mp, M, k0, kb);
            __syncthreads();
        }

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
            s_red[0][tid >> 5] = ld;
            s_red[1][tid >> 5] = qf;
        }
        __syncthreads();
        if (tid == 0) {
            double L = 0.0, Q = 0.0;
            for (int w = 0; w < kWarps; ++w) {
                L += s_red[0][w];
                Q += s_red[1][w];
            }
            const double v = -(Q + L + (double)bs * a.log2pi) * 0.5;
            unsigned st = s_status;
            if (!isfinite(v)) st |= 8u;
            a.block_llk[b] = v;
            a.block_status[b] = st;
        }
        __syncthreads();
    }
}

}  // namespace bv

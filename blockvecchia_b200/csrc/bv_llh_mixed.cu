// bv_llh_mixed.cu -- mixed-precision evaluation path (FP32 factor, FP64
// refinement and Schur complement, per-block FP64 fallback); the algorithm
// and its acceptance rule are described in bv_llh_mixed.cuh.
#include <algorithm>
#include <vector>

#include "../../include/bv.h"
#include "bv_common.cuh"
#include "bv_llh_mixed.cuh"

namespace bv {

namespace {

// Column j of the packed FP32 trapezoid (rows j..Mt-1) starts here;
// element (i, j), i >= j, is T[tro(j, Mt) + i - j].
__device__ __forceinline__ int tro(int j, int Mt) { return j * Mt - ((j * (j - 1)) >> 1); }

// Covariance / sigma2 in FP32 (diagonal scaling: the diagonal becomes 1).
// The squared distance is formed in FP64 from the FP64 coordinates, so the
// FP32 entry carries only its own rounding; general nu uses the FP64 routine.
__device__ __forceinline__ float cov_unit_f32(double x1, double y1, double x2, double y2,
                                              const MaternParams &p, float inv_range_f,
                                              float inv_ds_f, double inv_s2)
{
    const double dx = x2 - x1, dy = y2 - y1;
    const double d2 = fma(dx, dx, dy * dy);
    if (d2 == 0.0) return 1.0f;
    if (p.nu_kind == kNuGeneral) return (float)(matern(x1, y1, x2, y2, p) * inv_s2);
    float r = sqrtf((float)d2) * inv_range_f;
    if (!p.scale_is_one) r *= inv_ds_f;
    const float e = expf(-r);
    switch (p.nu_kind) {
    case kNuHalf:
        return e;
    case kNuThreeHalves:
        return (1.0f + r) * e;
    default:
        return fmaf(r, r * (1.0f / 3.0f), 1.0f + r) * e;
    }
}

struct MxShared {
    float Ld[kMxNB][kMxNB + 1];  // diagonal block of the current panel (L), 0 above
    float invd[kMxNB];
    double red[2][kMxWarps];
    int fail;
    int task;
};

// Block-wide sum of two doubles (fixed order: warp butterflies, then warp
// partials in index order).  Every thread gets the result.
__device__ __forceinline__ void block_sum2(double &a, double &b, MxShared &sh)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    if (lane == 0) {
        sh.red[0][warp] = a;
        sh.red[1][warp] = b;
    }
    __syncthreads();
    a = 0.0;
    b = 0.0;
    for (int w = 0; w < kMxWarps; ++w) {
        a += sh.red[0][w];
        b += sh.red[1][w];
    }
    __syncthreads();
}

// FP32 right-looking Cholesky of the first cs columns of the trapezoid T
// (Mt rows: Sigma22 / sigma2 and the bs rows of Sigma21^T / sigma2).  Panel
// p: warp 0 factors the diagonal block (registers and shuffles) and stores
// its inverse in place of it (the solves only need L^-1 there); every thread
// solves one row below against it and copies the solved panel to P (dense,
// kMxPdStride floats per row); then 8x4 register tiles apply the rank-16
// update to the trailing columns.  Returns false on a non-positive pivot.
__device__ bool factor_f32(float *T, float *P, int cs, int Mt, MxShared &sh)
{
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) sh.fail = 0;
    for (int k0 = 0; k0 < cs; k0 += kMxNB) {
        const int kb = min(kMxNB, cs - k0);
        const int n0 = k0 + kb;
        if (warp == 0) {
            float a[kMxNB];
#pragma unroll
            for (int c = 0; c < kMxNB; ++c)
                a[c] = (lane < kb && c <= lane) ? T[tro(k0 + c, Mt) + lane - c] : 0.0f;
            bool bad = false;
#pragma unroll
            for (int q = 0; q < kMxNB; ++q) {
                if (q < kb) {
                    float piv = __shfl_sync(0xffffffffu, a[q], q);
                    if (!(piv > 0.0f)) {
                        bad = true;
                        piv = 1.0f;
                    }
                    const float d = sqrtf(piv);
                    const float id = 1.0f / d;
                    if (lane > q)
                        a[q] *= id;
                    else if (lane == q)
                        a[q] = d;
#pragma unroll
                    for (int c = q + 1; c < kMxNB; ++c) {
                        const float lc = __shfl_sync(0xffffffffu, a[q], c);
                        if (c < kb && lane >= c) a[c] = fmaf(-a[q], lc, a[c]);
                    }
                }
            }
            if (lane < kMxNB) {
#pragma unroll
                for (int c = 0; c < kMxNB; ++c) sh.Ld[lane][c] = (lane < kb && c <= lane) ? a[c] : 0.0f;
                sh.invd[lane] = (lane < kb) ? 1.0f / a[lane] : 0.0f;
            }
            if (lane == 0 && bad) sh.fail = 1;
        }
        __syncthreads();
        if (sh.fail) return false;
        if (warp == 0) {
            // Inverse of the diagonal block (column `lane`) into T's diagonal
            // block, while the other warps solve the rows below.
            if (lane < kb) {
                float lv[kMxNB];
#pragma unroll
                for (int r = 0; r < kMxNB; ++r) {
                    float s = (r == lane) ? 1.0f : 0.0f;
#pragma unroll
                    for (int k = 0; k < r; ++k) s = fmaf(-sh.Ld[r][k], lv[k], s);
                    lv[r] = (r >= lane) ? s * sh.invd[r] : 0.0f;
                }
#pragma unroll
                for (int r = 0; r < kMxNB; ++r)
                    if (r >= lane && r < kb) T[tro(k0 + lane, Mt) + r - lane] = lv[r];
            }
        }
        // Rows below the diagonal block: x L^T = a, one thread of warps 1.. per row.
        for (int i = n0 + tid - 32; tid >= 32 && i < Mt; i += kMxThreads - 32) {
            float r[kMxNB];
#pragma unroll
            for (int c = 0; c < kMxNB; ++c) r[c] = (c < kb) ? T[tro(k0 + c, Mt) + i - k0 - c] : 0.0f;
#pragma unroll
            for (int q = 0; q < kMxNB; ++q) {
                float s = r[q];
#pragma unroll
                for (int c = 0; c < q; ++c) s = fmaf(-r[c], sh.Ld[q][c], s);
                r[q] = s * sh.invd[q];
            }
            float *pr = P + (i - n0) * kMxPdStride;
#pragma unroll
            for (int c = 0; c < kMxNB; ++c) {
                if (c < kb) T[tro(k0 + c, Mt) + i - k0 - c] = r[c];
                pr[c] = r[c];
            }
        }
        __syncthreads();
        if (n0 >= cs) break;
        // Trailing update of columns n0..cs-1 (rows k..Mt-1 of column k):
        // tiles of 8 rows x 4 columns; tile row t of column group g is needed
        // when t >= g/2 (rows 8t..8t+7 reach the diagonal of columns 4g..4g+3).
        const int nrow = Mt - n0, ncol = cs - n0;
        const int ntr = (nrow + 7) >> 3, ncg = (ncol + 3) >> 2;
        auto base = [&](int g) {
            const int m = g >> 1;
            return g * ntr - ((g & 1) ? m * m : m * (m - 1));
        };
        const int total = base(ncg);
        for (int tt = tid; tt < total; tt += kMxThreads) {
            int lo = 0, hi = ncg - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (base(mid) <= tt)
                    lo = mid;
                else
                    hi = mid - 1;
            }
            const int g = lo;
            const int t = (g >> 1) + (tt - base(g));
            float acc[8][4];
#pragma unroll
            for (int ii = 0; ii < 8; ++ii)
#pragma unroll
                for (int kk = 0; kk < 4; ++kk) acc[ii][kk] = 0.0f;
            const float *pa = P + (8 * t) * kMxPdStride;
            const float *pb = P + (4 * g) * kMxPdStride;
#pragma unroll
            for (int q4 = 0; q4 < kMxNB / 4; ++q4) {
                float4 av[8], bv[4];
#pragma unroll
                for (int ii = 0; ii < 8; ++ii)
                    av[ii] = *reinterpret_cast<const float4 *>(pa + ii * kMxPdStride + 4 * q4);
#pragma unroll
                for (int kk = 0; kk < 4; ++kk)
                    bv[kk] = *reinterpret_cast<const float4 *>(pb + kk * kMxPdStride + 4 * q4);
#pragma unroll
                for (int ii = 0; ii < 8; ++ii)
#pragma unroll
                    for (int kk = 0; kk < 4; ++kk) {
                        acc[ii][kk] = fmaf(av[ii].x, bv[kk].x, acc[ii][kk]);
                        acc[ii][kk] = fmaf(av[ii].y, bv[kk].y, acc[ii][kk]);
                        acc[ii][kk] = fmaf(av[ii].z, bv[kk].z, acc[ii][kk]);
                        acc[ii][kk] = fmaf(av[ii].w, bv[kk].w, acc[ii][kk]);
                    }
            }
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) {
                const int k = n0 + 4 * g + kk;
                if (k >= cs) continue;
                float *col = T + tro(k, Mt) - k;
#pragma unroll
                for (int ii = 0; ii < 8; ++ii) {
                    const int i = n0 + 8 * t + ii;
                    if (i >= k && i < Mt) col[i] -= acc[ii][kk];
                }
            }
        }
        __syncthreads();
    }
    return true;
}

// Triangular solves with the FP32 factor, one warp per right-hand side
// (column c of the row-major cs x bs array R), no block barriers: per panel
// the lanes of the diagonal block apply its stored inverse, then the lanes
// sweep the remaining rows with the panel's 16 solved values (shuffles).
// do_fwd: R := L^-1 R; do_bwd: R := L^-T R (both: L^-T L^-1 R).
__device__ void solve_f32(const float *T, float *R, int cs, int bs, int Mt, bool do_fwd, bool do_bwd)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int npan = (cs + kMxNB - 1) / kMxNB;
    for (int c = warp; c < bs; c += kMxWarps) {
        if (do_fwd) {
            for (int p = 0; p < npan; ++p) {
                const int k0 = p * kMxNB, kb = min(kMxNB, cs - k0), n0 = k0 + kb;
                float y = 0.0f;
                if (lane < kb) {
                    for (int r2 = 0; r2 <= lane; ++r2)
                        y = fmaf(T[tro(k0 + r2, Mt) + lane - r2], R[(k0 + r2) * bs + c], y);
                }
                __syncwarp();
                if (lane < kb) R[(k0 + lane) * bs + c] = y;
                float yv[kMxNB];
#pragma unroll
                for (int q = 0; q < kMxNB; ++q) yv[q] = __shfl_sync(0xffffffffu, y, q);
                for (int i = n0 + lane; i < cs; i += 32) {
                    float s = R[i * bs + c];
#pragma unroll
                    for (int q = 0; q < kMxNB; ++q)
                        if (q < kb) s = fmaf(-T[tro(k0 + q, Mt) + i - k0 - q], yv[q], s);
                    R[i * bs + c] = s;
                }
                __syncwarp();
            }
        }
        if (do_bwd) {
            for (int p = npan - 1; p >= 0; --p) {
                const int k0 = p * kMxNB, kb = min(kMxNB, cs - k0);
                float x = 0.0f;
                if (lane < kb) {
                    for (int r2 = lane; r2 < kb; ++r2)
                        x = fmaf(T[tro(k0 + lane, Mt) + r2 - lane], R[(k0 + r2) * bs + c], x);
                }
                __syncwarp();
                if (lane < kb) R[(k0 + lane) * bs + c] = x;
                float xv[kMxNB];
#pragma unroll
                for (int q = 0; q < kMxNB; ++q) xv[q] = __shfl_sync(0xffffffffu, x, q);
                for (int j = lane; j < k0; j += 32) {
                    const float *lj = T + tro(j, Mt) + k0 - j;  // L(k0 + q, j) = lj[q]
                    float s = R[j * bs + c];
#pragma unroll
                    for (int q = 0; q < kMxNB; ++q)
                        if (q < kb) s = fmaf(-lj[q], xv[q], s);
                    R[j * bs + c] = s;
                }
                __syncwarp();
            }
        }
    }
}

// FP64 residual Rd = Sigma21 - Sigma22 X1 (entries regenerated in FP64),
// written to R as FP32 after the 1/sigma2 scaling of the FP32 system.  A warp
// takes a row i: its lanes generate Sigma22(i, :) into the warp's K row, then
// lanes (c, part) form partial dot products, combined in a fixed order.
__device__ void residual(const double *X, const double *Y, const double *S21, const double *X1,
                         double *Kw, float *R, int cs, int bs, const MaternParams &mp,
                         double inv_s2)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double *K = Kw + warp * cs;
    const int parts = (bs <= 16) ? 32 / bs : 1;
    const int c = lane % bs, part = lane / bs;
    const bool active = lane < parts * bs;
    for (int i = warp; i < cs; i += kMxWarps) {
        const double xi = X[i], yi = Y[i];
        for (int j0 = 0; j0 < cs; j0 += 64) {
            const int ja = j0 + lane, jb = j0 + 32 + lane;
            double va = 0.0, vb = 0.0;
            if (ja < cs) va = matern(xi, yi, X[ja], Y[ja], mp) + (ja == i ? mp.nugget : 0.0);
            if (jb < cs) vb = matern(xi, yi, X[jb], Y[jb], mp) + (jb == i ? mp.nugget : 0.0);
            if (ja < cs) K[ja] = va;
            if (jb < cs) K[jb] = vb;
        }
        __syncwarp();
        double s = 0.0;
        if (active)
            for (int j = part; j < cs; j += parts) s = fma(K[j], X1[j * bs + c], s);
        // combine the parts of column c (lanes c, c + bs, ...) in order
        for (int pp = 1; pp < parts; ++pp) {
            const double o = __shfl_sync(0xffffffffu, s, lane + pp * bs < 32 ? lane + pp * bs : lane);
            if (part == 0) s += o;
        }
        if (active && part == 0) R[i * bs + c] = (float)((S21[i * bs + c] - s) * inv_s2);
        __syncwarp();
    }
}

// One conditioned block.  Returns true when the block was accepted (its
// contribution written), false when it goes to the FP64 fallback.
__device__ bool mixed_block(const MixedArgs &a, const MaternParams &mp, int b, const MxLayout &l,
                            unsigned char *sm, MxShared &sh)
{
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int cs = l.cs, bs = l.bs, Mt = l.Mt;
    double *X = reinterpret_cast<double *>(sm + l.o_X);
    double *Y = reinterpret_cast<double *>(sm + l.o_Y);
    double *zc = reinterpret_cast<double *>(sm + l.o_zc);
    double *zb = reinterpret_cast<double *>(sm + l.o_zb);
    double *S21 = reinterpret_cast<double *>(sm + l.o_S21);
    double *X1 = reinterpret_cast<double *>(sm + l.o_X1);
    double *S = reinterpret_cast<double *>(sm + l.o_S);
    float *T = reinterpret_cast<float *>(sm + l.o_T);
    float *R = reinterpret_cast<float *>(sm + l.o_R);
    float *P = reinterpret_cast<float *>(sm + l.o_P);
    const double inv_s2 = 1.0 / mp.sigma2;
    const float inv_range_f = (float)mp.inv_range, inv_ds_f = (float)mp.inv_ds;
    const float nug_unit = (float)(mp.nugget * inv_s2);

    const int off = a.acc[b];
    const int *kidx = a.knn + (size_t)b * cs;
    for (int t = tid; t < Mt; t += kMxThreads) {
        const int src = (t < cs) ? __ldg(kidx + t) : off + (t - cs);
        X[t] = __ldg(a.x + src);
        Y[t] = __ldg(a.y + src);
        const double z = __ldg(a.obs + src);
        if (t < cs)
            zc[t] = z;
        else
            zb[t - cs] = z;
    }
    __syncthreads();
    // FP32 trapezoid, columns paired (q, cs-1-q) for balance.
    const int half = (cs + 1) >> 1;
    for (int q = warp; q < half; q += kMxWarps) {
        const int j1 = q, j2 = cs - 1 - q;
        const int n1 = Mt - j1, n2 = (j2 != j1) ? Mt - j2 : 0;
        for (int r = lane; r < n1 + n2; r += 32) {
            const int j = (r < n1) ? j1 : j2;
            const int i = j + ((r < n1) ? r : r - n1);
            float t = cov_unit_f32(X[i], Y[i], X[j], Y[j], mp, inv_range_f, inv_ds_f, inv_s2);
            if (i == j) t += nug_unit;  // the nugget on Sigma22's diagonal
            T[tro(j, Mt) + i - j] = t;
        }
    }
    // FP64 Sigma21 (row j: conditioning point j, column c: block point c).
    for (int e = tid; e < cs * bs; e += kMxThreads) {
        const int j = e / bs, c = e - j * bs;
        S21[e] = matern(X[cs + c], Y[cs + c], X[j], Y[j], mp);
    }
    __syncthreads();

    if (!factor_f32(T, P, cs, Mt, sh)) return false;

    // X0 = L^-T W, W = the factored Sigma21^T rows.
    for (int e = tid; e < cs * bs; e += kMxThreads) {
        const int j = e / bs, c = e - j * bs;
        R[e] = T[tro(j, Mt) + cs + c - j];
    }
    __syncthreads();
    solve_f32(T, R, cs, bs, Mt, false, true);
    __syncthreads();
    for (int e = tid; e < cs * bs; e += kMxThreads) X1[e] = (double)R[e];
    __syncthreads();

    // Refinement: up to two steps (the residual's covariance rows use P).
    double *Kw = reinterpret_cast<double *>(P);
    bool accepted = false;
    double eta1 = 1.0;
    for (int step = 1; step <= 2; ++step) {
        residual(X, Y, S21, X1, Kw, R, cs, bs, mp, inv_s2);
        __syncthreads();
        solve_f32(T, R, cs, bs, Mt, true, true);
        __syncthreads();
        double nd = 0.0, nx = 0.0;
        for (int e = tid; e < cs * bs; e += kMxThreads) {
            const double d = (double)R[e];
            const double v = X1[e] + d;
            X1[e] = v;
            nd = fma(d, d, nd);
            nx = fma(v, v, nx);
        }
        block_sum2(nd, nx, sh);
        // Every thread holds the same sums, so the decisions are uniform.
        const double eta = (nx > 0.0) ? sqrt(nd / nx) : 1.0;
        if (step == 1) eta1 = eta;
        if (!(eta == eta)) break;  // NaN
        if (eta * eta1 <= a.tol) {
            accepted = true;
            break;
        }
        if (!(eta1 < 0.1)) break;  // refinement does not contract fast enough
    }
    if (!accepted) return false;

    // Schur complement and conditional mean in FP64: rows 0..bs-1 of S hold
    // S = Sigma11 - Sigma21^T X1 (lower), row bs holds (z - mu)^T.
    const int sp = bs + 1;
    for (int e = tid; e < sp * bs; e += kMxThreads) {
        const int r = e / bs, c = e - r * bs;
        if (r < bs && c > r) continue;
        double s;
        if (r < bs) {
            s = matern(X[cs + r], Y[cs + r], X[cs + c], Y[cs + c], mp) + (r == c ? mp.nugget : 0.0);
            for (int j = 0; j < cs; ++j) s = fma(-S21[j * bs + r], X1[j * bs + c], s);
        } else {
            s = zb[c];
            for (int j = 0; j < cs; ++j) s = fma(-X1[j * bs + c], zc[j], s);
        }
        S[r * sp + c] = s;
    }
    __syncthreads();
    // Cholesky of S with row bs riding along (warp 0; lane r owns row r).
    if (warp == 0) {
        bool bad = false;
        double ld = 0.0;
        for (int q = 0; q < bs; ++q) {
            double piv = S[q * sp + q];
            if (!(piv > 0.0)) {
                bad = true;
                piv = 1.0;
            }
            const double d = sqrt(piv);
            const double id = 1.0 / d;
            ld += log(d * d);
            if (lane > q && lane <= bs) S[lane * sp + q] *= id;
            __syncwarp();
            if (lane > q && lane <= bs) {
                const double lq = S[lane * sp + q];
                const int cmax = (lane < bs) ? lane : bs - 1;
                for (int c2 = q + 1; c2 <= cmax; ++c2) S[lane * sp + c2] = fma(-lq, S[c2 * sp + q], S[lane * sp + c2]);
            }
            __syncwarp();
        }
        if (lane == 0) {
            double qf = 0.0;
            for (int c = 0; c < bs; ++c) qf = fma(S[bs * sp + c], S[bs * sp + c], qf);
            const double v = -(qf + ld + (double)bs * a.log2pi) * 0.5;
            sh.fail = bad || !isfinite(v);
            if (!sh.fail) {
                a.block_llk[b] = v;
                a.block_status[b] = 0u;
            }
        }
    }
    __syncthreads();
    return !sh.fail;
}

__global__ void __launch_bounds__(kMxThreads, 1) llh_mixed_kernel(MixedArgs a)
{
    extern __shared__ __align__(16) unsigned char sm[];
    __shared__ MxShared sh;
    if (a.skip && *a.skip) return;
    const MaternParams mp = *a.mp;
    const int tid = threadIdx.x;
    for (;;) {
        if (tid == 0) sh.task = (int)atomicAdd(a.work_counter, 1u);
        __syncthreads();
        const int task = sh.task;
        if (task >= a.task_end) break;
        const int b = a.order[task];
        const int bs = a.acc[b + 1] - a.acc[b];
        const MxLayout l = mx_layout(a.cs, bs);
        const bool fits = b > 0 && a.cs > 0 && bs > 0 && bs <= kMxMaxBs && l.total <= a.smem_bytes;
        bool ok = false;
        if (bs == 0) {
            if (tid == 0) {
                a.block_llk[b] = -0.0;
                a.block_status[b] = 0u;
            }
            ok = true;
        } else if (fits) {
            ok = mixed_block(a, mp, b, l, sm, sh);
        }
        if (!ok && tid == 0) a.fallback_list[atomicAdd(a.fallback_count, 1)] = b;
        __syncthreads();
    }
}

// After the probe: skip the mixed pass when fewer than half of the probe's
// blocks were accepted (or there was nothing to probe), and then hand every
// block to the FP64 pass.
__global__ void mixed_decide_kernel(const int *order, int owned, int nprobe, const int *probe_fail,
                                    int *skip, int *fallback_list, int *fallback_count)
{
    // No conditioned block to probe (a shard of block 0 alone): FP64 throughout.
    const bool sk = nprobe == 0 || 2 * (nprobe - *probe_fail) < nprobe;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (sk && i < owned) fallback_list[i] = order[i];
    if (i == 0) {
        *skip = sk ? 1 : 0;
        *fallback_count = sk ? owned : 0;
    }
}

}  // namespace

int mixed_create(MixedWork &w, int device, int bc, int cs, int max_bs, const int *h_order, int owned,
                 bool fp32)
{
    mixed_free(w);
    w.fp32 = fp32;
    int optin = 0;
    BV_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    cudaFuncAttributes fa;
    BV_CUDA_TRY(cudaFuncGetAttributes(&fa, llh_mixed_kernel));
    const size_t avail = (size_t)optin - fa.sharedSizeBytes - 1024;
    // Shared memory for the largest block size that fits; larger blocks fall back.
    int bs_cap = std::min(max_bs, kMxMaxBs);
    size_t need = 0;
    while (bs_cap > 0) {
        need = mx_layout(cs, bs_cap).total;
        if (need <= avail) break;
        --bs_cap;
    }
    if (bs_cap <= 0 || cs <= 0) need = 16;  // every block falls back
    // The residual's per-warp K rows live in P's region.
    w.smem_bytes = need;
    BV_CUDA_TRY(cudaFuncSetAttribute(llh_mixed_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)avail));
    int occ = 0;
    BV_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, llh_mixed_kernel, kMxThreads, w.smem_bytes));
    if (occ < 1) {
        set_error("mixed: kernel cannot be resident with %zu B of shared memory", w.smem_bytes);
        return BV_E_TOOLARGE;
    }
    int sms = 0;
    BV_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    w.grid = sms * occ;
    (void)bc;
    w.owned = owned;
    std::vector<int> probe;
    // Block 0 (unconditioned) never takes the mixed path: probe its neighbour.
    // Without the FP32 pass nothing is probed and the decision sends every
    // block to the FP64 pass.
    for (int t = 0; fp32 && t < owned; t += kMxProbeStride) {
        const int u = (h_order[t] == 0 && t + 1 < owned) ? t + 1 : t;
        if (h_order[u] != 0) probe.push_back(h_order[u]);
    }
    w.nprobe = (int)probe.size();
    BV_CUDA_TRY(cudaMalloc(&w.counter, 2 * sizeof(unsigned)));
    BV_CUDA_TRY(cudaMalloc(&w.probe_list, std::max<size_t>(1, probe.size()) * sizeof(int)));
    BV_CUDA_TRY(cudaMalloc(&w.probe_fail_list, std::max<size_t>(1, probe.size()) * sizeof(int)));
    BV_CUDA_TRY(cudaMalloc(&w.probe_fail, sizeof(int)));
    BV_CUDA_TRY(cudaMalloc(&w.skip, sizeof(int)));
    BV_CUDA_TRY(cudaMalloc(&w.fallback_list, std::max(1, owned) * sizeof(int)));
    BV_CUDA_TRY(cudaMalloc(&w.fallback_count, sizeof(int)));
    if (!probe.empty())
        BV_CUDA_TRY(cudaMemcpy(w.probe_list, probe.data(), probe.size() * sizeof(int), cudaMemcpyHostToDevice));
    w.active = true;
    return BV_OK;
}

int mixed_enqueue(MixedWork &w, const MixedArgs &a0, cudaStream_t st)
{
    if (!w.active) {
        set_error("mixed: path not initialised");
        return BV_E_INVALID;
    }
    BV_CUDA_TRY(cudaMemsetAsync(w.counter, 0, 2 * sizeof(unsigned), st));
    BV_CUDA_TRY(cudaMemsetAsync(w.probe_fail, 0, sizeof(int), st));
    BV_CUDA_TRY(cudaMemsetAsync(w.fallback_count, 0, sizeof(int), st));
    BV_CUDA_TRY(cudaMemsetAsync(w.skip, 0, sizeof(int), st));
    if (w.owned <= 0) return BV_OK;
    MixedArgs a = a0;
    a.smem_bytes = (unsigned)w.smem_bytes;
    // Probe pass.
    MixedArgs p = a;
    p.order = w.probe_list;
    p.task_end = w.nprobe;
    p.work_counter = w.counter;
    p.fallback_list = w.probe_fail_list;
    p.fallback_count = w.probe_fail;
    p.skip = nullptr;
    if (w.nprobe > 0) {
        llh_mixed_kernel<<<std::min(w.grid, w.nprobe), kMxThreads, w.smem_bytes, st>>>(p);
        BV_CUDA_TRY(cudaGetLastError());
    }
    mixed_decide_kernel<<<(w.owned + 255) / 256, 256, 0, st>>>(a.order, w.owned, w.nprobe, w.probe_fail,
                                                               w.skip, w.fallback_list, w.fallback_count);
    BV_CUDA_TRY(cudaGetLastError());
    if (!w.fp32) return BV_OK;
    // Full pass (returns at once when skipped).
    a.task_end = w.owned;
    a.work_counter = w.counter + 1;
    a.fallback_list = w.fallback_list;
    a.fallback_count = w.fallback_count;
    a.skip = w.skip;
    llh_mixed_kernel<<<std::min(w.grid, w.owned), kMxThreads, w.smem_bytes, st>>>(a);
    BV_CUDA_TRY(cudaGetLastError());
    return BV_OK;
}

void mixed_free(MixedWork &w)
{
    if (w.counter) cudaFree(w.counter);
    if (w.fallback_list) cudaFree(w.fallback_list);
    if (w.probe_list) cudaFree(w.probe_list);
    if (w.probe_fail_list) cudaFree(w.probe_fail_list);
    if (w.probe_fail) cudaFree(w.probe_fail);
    if (w.skip) cudaFree(w.skip);
    if (w.fallback_count) cudaFree(w.fallback_count);
    w = MixedWork();
}

}  // namespace bv

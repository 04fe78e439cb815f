// bv_reduce.cuh -- deterministic reduction of per-block contributions.
#pragma once

#include <cuda_runtime.h>

#include "../../include/bv.h"

namespace bv {

// Result record of one evaluation (device, then pinned host).
struct EvalResult {
    double llk;
    int blocks, cond_fail, schur_fail, fallback, nonfinite;
    unsigned flags_or;
    int failed;  // blocks with a failed pivot in either factor (counted once)
};

constexpr int kReduceThreads = 1024;  // virtual lanes of the reduction tree
constexpr int kReduceScratchBytes =
    2 * kReduceThreads * (int)sizeof(double) + 7 * 32 * (int)sizeof(int);

// Deterministic reduction of the per-block contributions by one CTA: the
// blocks are split into kReduceThreads contiguous chunks (virtual lanes), each
// summed in block order with Neumaier compensation, and the lanes' (sum,
// compensation) pairs are combined in a fixed tree order.  A CTA of any size
// (a multiple of 32, at most 1024 threads) runs the virtual lanes in strides,
// so the arithmetic -- and the result -- is the same for every caller (the
// single-job reduction kernel, the last CTA of a server batch).  `scratch` is
// kReduceScratchBytes of shared memory.  Loads bypass L1 (the contributions
// were written by other CTAs of the same launch).
__device__ __forceinline__ void reduce_blocks(const double *v, const unsigned *st, int n,
                                              EvalResult *out, void *scratch)
{
    double *s_s = reinterpret_cast<double *>(scratch);
    double *s_c = s_s + kReduceThreads;
    int *s_cnt = reinterpret_cast<int *>(s_c + kReduceThreads);  // [6][32]
    unsigned *s_or = reinterpret_cast<unsigned *>(s_cnt + 6 * 32);
    const int T = blockDim.x;
    const int t = threadIdx.x;
    const int chunk = (n + kReduceThreads - 1) / kReduceThreads;
    int cf = 0, sf = 0, fb = 0, nf = 0, nb = 0, fl = 0;
    unsigned fo = 0;
    for (int lane = t; lane < kReduceThreads; lane += T) {
        const int b0 = lane * chunk, b1 = min(n, b0 + chunk);
        double s = 0.0, c = 0.0;
        for (int i = b0; i < b1; ++i) {
            const double x = __ldcg(v + i);
            const double tt = s + x;
            if (fabs(s) >= fabs(x))
                c += (s - tt) + x;
            else
                c += (x - tt) + s;
            s = tt;
            const unsigned f = __ldcg(st + i);
            fo |= f;
            cf += (f & BV_ST_COND_FAIL) ? 1 : 0;
            sf += (f & BV_ST_SCHUR_FAIL) ? 1 : 0;
            fb += (f & BV_ST_FP32_FALLBACK) ? 1 : 0;
            nf += (f & BV_ST_NONFINITE) ? 1 : 0;
            fl += (f & (BV_ST_COND_FAIL | BV_ST_SCHUR_FAIL)) ? 1 : 0;
            ++nb;
        }
        s_s[lane] = s;
        s_c[lane] = c;
    }
    // Integer counts: order-free warp reduction.
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        cf += __shfl_xor_sync(0xffffffffu, cf, o);
        sf += __shfl_xor_sync(0xffffffffu, sf, o);
        fb += __shfl_xor_sync(0xffffffffu, fb, o);
        nf += __shfl_xor_sync(0xffffffffu, nf, o);
        nb += __shfl_xor_sync(0xffffffffu, nb, o);
        fl += __shfl_xor_sync(0xffffffffu, fl, o);
        fo |= __shfl_xor_sync(0xffffffffu, fo, o);
    }
    if ((t & 31) == 0) {
        s_cnt[0 * 32 + (t >> 5)] = cf;
        s_cnt[1 * 32 + (t >> 5)] = sf;
        s_cnt[2 * 32 + (t >> 5)] = fb;
        s_cnt[3 * 32 + (t >> 5)] = nf;
        s_cnt[4 * 32 + (t >> 5)] = nb;
        s_cnt[5 * 32 + (t >> 5)] = fl;
        s_or[t >> 5] = fo;
    }
    __syncthreads();
    for (int w = kReduceThreads / 2; w > 0; w >>= 1) {
        for (int lane = t; lane < w; lane += T) {
            const double a = s_s[lane], b = s_s[lane + w];
            const double tt = a + b;
            double cc = s_c[lane] + s_c[lane + w];
            if (fabs(a) >= fabs(b))
                cc += (a - tt) + b;
            else
                cc += (b - tt) + a;
            s_s[lane] = tt;
            s_c[lane] = cc;
        }
        __syncthreads();
    }
    if (t == 0) {
        EvalResult r;
        r.llk = s_s[0] + s_c[0];
        int c5[6] = {0, 0, 0, 0, 0, 0};
        unsigned o = 0;
        for (int w = 0; w < T / 32; ++w) {
            for (int q = 0; q < 6; ++q) c5[q] += s_cnt[q * 32 + w];
            o |= s_or[w];
        }
        r.cond_fail = c5[0];
        r.schur_fail = c5[1];
        r.fallback = c5[2];
        r.nonfinite = c5[3];
        r.blocks = c5[4];
        r.flags_or = o;
        r.failed = c5[5];
        *out = r;
    }
    __syncthreads();
}

}  // namespace bv

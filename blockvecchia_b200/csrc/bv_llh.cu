// bv_llh.cu -- handle, schedule and C ABI of the block-Vecchia likelihood.
//
// Replaces the device side of the reference's objective
// llh_Xvecchia_batch<double> (include/llh_Xvecchia_batch.h:22-522) and the
// device allocations of its driver (src/test_Xvecchia_batch.cpp:459-600).
// Layout data (locations, observations, conditioning indices) is copied to
// HBM once at bv_create; one evaluation moves 48 bytes of parameters in and
// one result record out, and runs as a CUDA graph:
//   H2D params -> zero work counter -> fused per-block kernel(s)
//   -> deterministic reduction -> D2H result.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <numeric>
#include <vector>

#include "../../include/bv.h"
#include "bv_common.cuh"
#include "bv_knn.cuh"
#include "bv_llh_big.cuh"
#include "bv_llh_fp64.cuh"
#include "bv_llh_mixed.cuh"
#include "bv_reduce.cuh"

namespace bv {

// The fused FP64 kernel: persistent CTAs pull blocks from a work counter
// (largest first) and evaluate each by the path its size calls for.
template <bool kBig, bool kXYZ3>
__global__ void __launch_bounds__(kThreads, 1) llh_fp64_kernel_t(LlhArgs a)
{
    extern __shared__ __align__(128) double smem[];
    __shared__ BlockShared sh;
    const MaternParams mp = *a.mp;
    const int tid = threadIdx.x;
    const int task_end = a.task_count ? min(a.task_end, *a.task_count) : a.task_end;
    init_block_sync(sh);
    for (;;) {
        if (tid == 0) sh.task = (int)atomicAdd(a.work_counter, 1u) + a.task_begin;
        __syncthreads();
        const int task = sh.task;
        if (task >= task_end) break;
        run_block<kBig, kXYZ3>(a, mp, a.order[task], smem, sh);
        __syncthreads();
    }
}

// Without the streamed large-block path compiled in (every layout whose
// blocks fit shared memory, and the allocation-free entry point), and with it.
// 3-D locations (space-time or --3D) run separate instantiations.
static void (*const llh_fp64_kernel)(LlhArgs) = llh_fp64_kernel_t<false, false>;
static void (*const llh_fp64_big_kernel)(LlhArgs) = llh_fp64_kernel_t<true, false>;
static void (*const llh_fp64_kernel3)(LlhArgs) = llh_fp64_kernel_t<false, true>;
static void (*const llh_fp64_big_kernel3)(LlhArgs) = llh_fp64_kernel_t<true, true>;

// The streamed (left-looking, panels through L2) path run by small CTAs,
// several per SM, so that the pivot chains of several blocks overlap on one
// SM: NT threads per CTA, RC rows per streamed chunk, MINB CTAs per SM.
template <int NT, int RC, int MINB, int NS, bool kXYZ3, bool kBulk>
__global__ void __launch_bounds__(NT, MINB) llh_lean_kernel_t(LlhArgs a)
{
    extern __shared__ __align__(128) double smem[];
    __shared__ LeanShared sh;
    const MaternParams mp = *a.mp;
    const int tid = threadIdx.x;
    const int task_end = a.task_count ? min(a.task_end, *a.task_count) : a.task_end;
    double *slab = a.gslab + (size_t)blockIdx.x * a.gslab_stride;
    for (;;) {
        if (tid == 0) {
            sh.task = (int)atomicAdd(a.work_counter, 1u) + a.task_begin;
            sh.status = 0u;
        }
        __syncthreads();
        const int task = sh.task;
        if (task >= task_end) break;
        const int b = a.order[task];
        if (a.acc[b + 1] == a.acc[b]) {  // empty block: contributes -(0 + 0 + 0) / 2
            if (tid == 0) {
                a.block_llk[b] = -0.0;
                a.block_status[b] = a.status_or;
            }
        } else {
            process_block_big<NT, RC, LeanShared, NS, kXYZ3, kBulk>(
                a, mp, b, reinterpret_cast<unsigned char *>(smem), slab, sh);
        }
        __syncthreads();
    }
}

struct LeanVariant {
    void (*kernel)(LlhArgs);   // 2-D locations
    void (*kernel3)(LlhArgs);  // with a third coordinate
    int threads, rc, ns;
    bool bulk;  // the whole matrix generated into the slab before the factorization
};
#define BV_LEAN(NT, RC, MINB, NS, BULK)                                                              \
    {llh_lean_kernel_t<NT, RC, MINB, NS, false, BULK>, llh_lean_kernel_t<NT, RC, MINB, NS, true, BULK>, \
     NT, RC, NS, BULK}
// The left-looking update reads the earlier panels straight from the slab
// (no staging), so the CTAs can be small and several blocks share an SM.
// Kernel ms, n = 200k uniform, bc = 20k, nu = 1.5: the persistent kernel;
// then 96-thread CTAs x5 per SM, 160 x3 and 256 x2 generating panel by panel
// (the first three variants; the whole-matrix generation, the last three,
// wins only where the generation is expensive: general nu):
//   cs =  40 (M <=  74):  2.54 /  0.80 /  1.00 /  1.35
//   cs =  80 (M <= 114):  4.48 /  2.02 /  2.16 /  2.58
//   cs = 120 (M <= 154):  6.88 /  4.13 /  4.01 /  4.40
//   cs = 160 (M <= 194): 10.00 /  8.89 /  6.62 /  7.04
//   cs = 200 (M <= 234): 13.70 / 14.79 / 10.73 / 10.78
//   cs = 240 (M <= 274): 26.23 / 28.65 / 18.41 / 15.43
//   cs = 300 (M <= 334): 40.94 / 47.85 / 30.23 / 25.35
// At the headline shape (n = 1M, cs = 200, nu = 2.5, largest M 240):
// 68.0 / 73.3 / 53.2 / 53.5; at the general-nu stress shape (2M points,
// cs = 300, nu = 0.8) 256 x2 generating the whole matrix first, 526 ms,
// against 537 panel by panel.  128 x4 (four CTAs while two panels of
// M <= ~200 fit) is the fastest up to M ~ 170 (cs = 40 / 80 / 120: 0.78 /
// 1.98 / 3.86).  Larger CTAs spill (288 or 320 threads x2, 192 x3, 160 x4)
// or run one block per SM (512 x1); 128 x3 and 192 x2 lost everywhere.
// All give the same bits (the per-element operations do not
// depend on the CTA size or the generation mode), so bv_opts.tune may pick
// any of them.
static const LeanVariant kLeanVariants[] = {
    BV_LEAN(96, 64, 5, 0, false),
    BV_LEAN(160, 64, 3, 0, false),
    BV_LEAN(256, 64, 2, 0, false),
    BV_LEAN(128, 64, 4, 0, false),
    BV_LEAN(160, 64, 3, 0, true),
    BV_LEAN(256, 64, 2, 0, true),
};
constexpr int kNumLean = (int)(sizeof(kLeanVariants) / sizeof(kLeanVariants[0]));
static int lean_variant(int max_m)
{
    const int t = lean_table_threads(max_m);
    return t == 128 ? 3 : (t == 160 ? 1 : 2);  // the panel-by-panel variants
}

static thread_local char g_err[1024] = "";

void set_error(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}
const char *get_error() { return g_err; }

__global__ void __launch_bounds__(kReduceThreads) reduce_kernel(const double *v,
                                                                const unsigned *st, int n,
                                                                EvalResult *out)
{
    __shared__ __align__(16) unsigned char scratch[kReduceScratchBytes];
    reduce_blocks(v, st, n, out, scratch);
}

}  // namespace bv

using namespace bv;

struct bv_handle {
    std::mutex mu;
    bv_opts opts;
    int device = 0;
    int n = 0, bc = 0, cs = 0;
    int max_m = 0;
    std::vector<int> batchNum, acc, order;
    int owned = 0;  // blocks this handle evaluates (all, or its shard)
    // device
    double *d_x = nullptr, *d_y = nullptr, *d_obs = nullptr;
    double *d_z = nullptr;  // third coordinate of 3-D layouts
    int nz = 0;             // 1 when the layout has a third coordinate
    int *d_acc = nullptr, *d_knn = nullptr, *d_order = nullptr;
    double *d_block_llk = nullptr;
    unsigned *d_block_status = nullptr;
    unsigned *d_counters = nullptr;  // one per launch
    double *d_slab = nullptr;
    size_t slab_stride = 0;
    double *d_slab_lean = nullptr;  // per-CTA slabs of the multi-CTA streamed launch
    int lean_max_m = 0;             // blocks with M <= this run the multi-CTA streamed kernel
    int streamed_blocks = 0;        // of the owned blocks, how many that is
    bool mixed_lean = false;        // mixed path: the FP64 pass runs the streamed kernel (last launch)
    // The streamed launch's order positions and largest M, its CTA size
    // (kLeanVariants index; -1: from the table), and the tuner's record.
    int lean_begin = 0, lean_end = 0, lean_m = 0, lean_choice = -1, lean_threads = 0, lean_vi = -1;
    bool tuned = false;
    double tune_ms[kNumLean] = {};
    MaternParams *d_mp = nullptr;
    EvalResult *d_res = nullptr;
    MixedWork mixed;  // mixed-precision scratch (bv_llh_mixed.cuh)
    // pinned host
    MaternParams *h_mp = nullptr;
    EvalResult *h_res = nullptr;
    // launch plan
    int smem_max_m = 0;
    int big_max_m = 0;  // largest M of the streamed large-block path
    bool use_big = false;
    void (*kernel)(LlhArgs) = nullptr;
    size_t smem_bytes = 0;
    int grid = 0;
    int block_threads = kThreads;
    struct Launch {
        int begin, end, grid;
        void (*kernel)(LlhArgs);
        int threads;
        size_t smem;
        double *slab;
        size_t slab_stride;
    };
    std::vector<Launch> launches;
    cudaStream_t stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, evk0 = nullptr, evk1 = nullptr;
    cudaStream_t own_stream = nullptr;  // the handle's stream; `stream` may be a caller's
    // status
    bv_status status{};
    int iterations = 0;
};

static void handle_free(bv_handle *h)
{
    if (!h) return;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(h->device);
    if (h->gexec) cudaGraphExecDestroy(h->gexec);
    if (h->graph) cudaGraphDestroy(h->graph);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->evk0) cudaEventDestroy(h->evk0);
    if (h->evk1) cudaEventDestroy(h->evk1);
    if (h->own_stream) cudaStreamDestroy(h->own_stream);
    cudaFree(h->d_x);
    cudaFree(h->d_y);
    cudaFree(h->d_obs);
    cudaFree(h->d_z);
    cudaFree(h->d_acc);
    cudaFree(h->d_knn);
    cudaFree(h->d_order);
    cudaFree(h->d_block_llk);
    cudaFree(h->d_block_status);
    cudaFree(h->d_counters);
    cudaFree(h->d_slab);
    cudaFree(h->d_slab_lean);
    cudaFree(h->d_mp);
    cudaFree(h->d_res);
    mixed_free(h->mixed);
    cudaFreeHost(h->h_mp);
    cudaFreeHost(h->h_res);
    cudaSetDevice(prev);
    delete h;
}

extern "C" int bv_abi_sizes(size_t *out, int n)
{
    const size_t v[] = {sizeof(bv_layout), sizeof(bv_opts), sizeof(bv_status), sizeof(bv_server_opts),
                        sizeof(bv_server_stats), sizeof(bv_job_opts)};
    int k = 0;
    for (; out && k < n && k < (int)(sizeof(v) / sizeof(v[0])); ++k) out[k] = v[k];
    return k;
}

extern "C" void bv_default_opts(bv_opts *o)
{
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->precision = BV_PREC_FP64;
    o->kernel = 1;
    o->dist_scale = 1.0;
    o->device = 0;
    o->on_failure = BV_FAIL_NEGINF;
    o->print_iter = 0;
    o->use_graph = 1;
    o->schedule = 0;
    o->mixed_tol = 1e-8;
    o->shard_count = 1;
    o->shard_index = 0;
    o->large_blocks = BV_LARGE_AUTO;
    o->nugget = 0;
    o->earth = 0;
    o->tune = 0;
    o->mixed_fp32 = 0;
}

// Cost rank (largest first, ties by index) shared by the schedule and the
// sharding rule.
static std::vector<int> cost_order(const int *batchNum, int bc, int cs)
{
    std::vector<int> order(bc);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        const int ma = batchNum[a] + (a == 0 ? 0 : cs);
        const int mb = batchNum[b] + (b == 0 ? 0 : cs);
        return ma > mb;
    });
    return order;
}

extern "C" int bv_shard_blocks(const int *batchNum, int bc, int cs, int shard_count,
                               int shard_index, unsigned char *mask)
{
    if (!batchNum || !mask || bc <= 0 || cs < 0 || shard_count < 1 || shard_index < 0 ||
        shard_index >= shard_count) {
        set_error("bv_shard_blocks: invalid argument");
        return BV_E_INVALID;
    }
    const std::vector<int> order = cost_order(batchNum, bc, cs);
    for (int t = 0; t < bc; ++t) mask[order[t]] = (t % shard_count == shard_index) ? 1 : 0;
    return BV_OK;
}

extern "C" const char *bv_last_error(void) { return get_error(); }

int bv::validate_layout(const bv_layout *L)
{
    if (!L || L->n <= 0 || L->bc <= 0 || L->cs < 0 || !L->batchNum || !L->batchNumAccum ||
        !L->x || !L->y || !L->obs) {
        set_error("layout: null or non-positive field");
        return BV_E_INVALID;
    }
    if (L->batchNumAccum[0] != 0 || L->batchNumAccum[L->bc] != L->n) {
        set_error("layout: batchNumAccum must start at 0 and end at n (got %d, %d, n=%d)",
                  L->batchNumAccum[0], L->batchNumAccum[L->bc], L->n);
        return BV_E_INVALID;
    }
    for (int i = 0; i < L->bc; ++i) {
        if (L->batchNum[i] < 0 || L->batchNumAccum[i + 1] - L->batchNumAccum[i] != L->batchNum[i]) {
            set_error("layout: batchNum[%d] inconsistent with batchNumAccum", i);
            return BV_E_INVALID;
        }
    }
    if (L->cs > 0 && L->bc > 1 && L->batchNum[0] < L->cs) {
        set_error("layout: block 0 has %d points < cs=%d (firstbatch merges clusters until "
                  ">= cs)", L->batchNum[0], L->cs);
        return BV_E_INVALID;
    }
    if (L->cs > 0 && L->knn_idx) {
        for (int i = 1; i < L->bc; ++i) {
            const int lim = L->batchNumAccum[i];
            const int *k = L->knn_idx + (size_t)i * L->cs;
            for (int t = 0; t < L->cs; ++t)
                if (k[t] < 0 || k[t] >= lim) {
                    set_error("layout: knn_idx[%d*cs+%d]=%d outside the earlier blocks [0,%d)",
                              i, t, k[t], lim);
                    return BV_E_INVALID;
                }
        }
        for (int t = 0; t < L->cs; ++t)
            if (L->knn_idx[t] < 0 || L->knn_idx[t] >= L->n) {
                set_error("layout: knn_idx[%d]=%d outside [0,n)", t, L->knn_idx[t]);
                return BV_E_INVALID;
            }
    }
    if (L->cs > 0 && !L->knn_idx && (!L->cx || !L->cy)) {
        set_error("layout: knn_idx is NULL and no block centroids were given");
        return BV_E_INVALID;
    }
    return BV_OK;
}

// Static shared memory of the fused kernel plus a margin; the dynamic part
// gets the rest of the per-block opt-in limit.
static size_t fused_static_smem()
{
    cudaFuncAttributes fa, fb;
    if (cudaFuncGetAttributes(&fa, llh_fp64_kernel) != cudaSuccess ||
        cudaFuncGetAttributes(&fb, llh_fp64_big_kernel) != cudaSuccess) {
        cudaGetLastError();
        return 16384;
    }
    // Static plus dynamic shared memory may use the whole opt-in maximum.
    return std::max(fa.sharedSizeBytes, fb.sharedSizeBytes);
}

// Largest M whose block fits in `bytes` of dynamic shared memory.
static int max_m_for_bytes(size_t bytes, size_t per_double, int nz = 0)
{
    int lo = 1, hi = 4096;
    while (lo < hi) {
        int mid = (lo + hi + 1) / 2;
        if (block_doubles(mid, nz) * per_double <= bytes)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

int bv::fp64_limits(int device, size_t *avail, int *small_m, int *big_m, int nz)
{
    int optin = 0;
    BV_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    const size_t av = (size_t)optin - fused_static_smem();
    if (avail) *avail = av;
    if (small_m) *small_m = max_m_for_bytes(av, sizeof(double), nz);
    if (big_m) *big_m = big_max_m_for_bytes(av, kBigRC, nz);
    return BV_OK;
}

bool bv::use_big_path(const int *batchNum, int bc, int cs, int small_m, int big_m, int sm_count)
{
    int n_big = 0;
    for (int b = 0; b < bc; ++b) {
        const int m = batchNum[b] + (b == 0 ? 0 : cs);
        if (m > small_m && m <= big_m) ++n_big;
    }
    return n_big > sm_count;
}

// M of the block at position t of the processing order.
static int order_m(const bv_handle *h, int t)
{
    const int b = h->order[t];
    return h->batchNum[b] + (b == 0 ? 0 : h->cs);
}

// The multi-CTA streamed launch over order positions [begin, end), whose
// largest block has M = max_m.
static int plan_lean_launch(bv_handle *h, const cudaDeviceProp &prop, int begin, int end, int max_m)
{
    const int vi = h->lean_choice >= 0 ? h->lean_choice : lean_variant(max_m);
    const LeanVariant &v = kLeanVariants[vi];
    h->lean_vi = vi;
    h->lean_begin = begin;
    h->lean_end = end;
    h->lean_m = max_m;
    h->lean_threads = v.threads;
    void (*const kern)(LlhArgs) = h->nz ? v.kernel3 : v.kernel;
    cudaFuncAttributes fa;
    BV_CUDA_TRY(cudaFuncGetAttributes(&fa, kern));
    int optin = 0;
    BV_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device));
    const size_t smem = big_layout(max_m, v.rc, h->nz, v.ns).total;
    if (smem > (size_t)optin - fa.sharedSizeBytes) {
        set_error("plan: blocks of M = %d exceed the streamed schedule's shared memory", max_m);
        return BV_E_TOOLARGE;
    }
    BV_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int occ = 0;
    BV_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, v.threads, smem));
    if (occ < 1) {
        set_error("plan: streamed kernel cannot be resident (smem %zu B)", smem);
        return BV_E_TOOLARGE;
    }
    const int grid = std::min(prop.multiProcessorCount * occ, end - begin);
    const size_t stride = (big_slab_doubles(max_m) + 31) & ~(size_t)31;
    const size_t bytes = stride * sizeof(double) * (size_t)grid;
    if (cudaMalloc(&h->d_slab_lean, bytes) != cudaSuccess) {
        cudaGetLastError();
        set_error("plan: cannot allocate %zu B of block slabs", bytes);
        return BV_E_NOMEM;
    }
    h->launches.push_back({begin, end, grid, kern, v.threads, smem, h->d_slab_lean, stride});
    return BV_OK;
}

// Which kernel evaluates which blocks.  Blocks are in the processing order
// (largest first).  Under the default schedule every block whose two panels
// fit the multi-CTA streamed kernel's shared memory (M up to ~780) runs that
// kernel (several blocks per SM, so their pivot chains overlap); larger ones
// run the persistent one-CTA-per-SM kernel on a global slab.  The split
// depends on the layout only, so every shard and every evaluation make the
// same choice.
static int plan_launches(bv_handle *h)
{
    cudaDeviceProp prop;
    BV_CUDA_TRY(cudaGetDeviceProperties(&prop, h->device));
    size_t avail = 0;
    int cap_m = 0;
    {
        const int rc = fp64_limits(h->device, &avail, &cap_m, &h->big_max_m, h->nz);
        if (rc) return rc;
    }
    const int sched = h->opts.schedule;
    // The multi-CTA streamed kernel takes every block whose panels fit its
    // shared memory (by default and under BV_SCHED_STREAMED; for the mixed
    // path's FP64 pass, when every block fits); BV_SCHED_PERSISTENT /
    // BUCKETED keep the persistent kernel.
    int lean_limit = 0;
    {
        int optin = 0;
        BV_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device));
        cudaFuncAttributes fa;
        BV_CUDA_TRY(cudaFuncGetAttributes(&fa, kLeanVariants[2].kernel));
        lean_limit = big_max_m_for_bytes((size_t)optin - fa.sharedSizeBytes, 64, h->nz, 0);
    }
    if ((sched == BV_SCHED_STREAMED || sched == BV_SCHED_AUTO) && h->opts.precision == BV_PREC_FP64)
        h->lean_max_m = lean_limit;
    else
        h->lean_max_m = 0;
    if (sched == BV_SCHED_STREAMED && h->max_m > lean_limit) {
        set_error("plan: blocks of M = %d exceed the streamed schedule's limit %d", h->max_m, lean_limit);
        return BV_E_TOOLARGE;
    }
    int split = 0;  // order positions [split, owned) take the streamed kernel
    while (split < h->owned && order_m(h, split) > h->lean_max_m) ++split;
    h->streamed_blocks = h->owned - split;
    h->launches.clear();
    h->smem_max_m = std::min(cap_m, h->max_m);
    // The cap is per kernel, not per handle: set it to what the device allows
    // so that handles with different block sizes can coexist.
    for (auto k : {llh_fp64_kernel, llh_fp64_big_kernel, llh_fp64_kernel3, llh_fp64_big_kernel3})
        BV_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)avail));
    // Decided on the whole layout (not the shard), so every shard and the
    // server take the same path for a given block.
    h->use_big = (h->opts.large_blocks == BV_LARGE_STREAMED) ||
                 (h->opts.large_blocks == BV_LARGE_AUTO &&
                  use_big_path(h->batchNum.data(), h->bc, h->cs, cap_m, h->big_max_m,
                               prop.multiProcessorCount));
    h->kernel = h->use_big ? (h->nz ? llh_fp64_big_kernel3 : llh_fp64_big_kernel)
                           : (h->nz ? llh_fp64_kernel3 : llh_fp64_kernel);
    if (h->use_big) {
        h->smem_bytes = big_launch_smem(h->max_m, cap_m, h->big_max_m, h->nz);
        h->slab_stride = big_slab_stride(h->max_m, cap_m, h->big_max_m, h->nz);
    } else {
        h->smem_bytes = block_doubles(h->smem_max_m, h->nz) * sizeof(double);
        h->slab_stride = (h->max_m > cap_m) ? (block_doubles(h->max_m, h->nz) + 31) & ~(size_t)31 : 0;
    }
    int occ = 0;
    BV_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, h->kernel, kThreads, h->smem_bytes));
    if (occ < 1) {
        set_error("plan: fused kernel cannot be resident (smem %zu B)", h->smem_bytes);
        return BV_E_TOOLARGE;
    }
    h->grid = prop.multiProcessorCount * occ;
    h->block_threads = kThreads;
    if (h->slab_stride > 0) {
        const size_t bytes = h->slab_stride * sizeof(double) * (size_t)h->grid;
        if (cudaMalloc(&h->d_slab, bytes) != cudaSuccess) {
            cudaGetLastError();
            set_error("plan: cannot allocate %zu B of block slabs", bytes);
            return BV_E_NOMEM;
        }
    }
    if (sched != BV_SCHED_BUCKETED) {
        if (split > 0)
            h->launches.push_back({0, split, h->grid, h->kernel, kThreads, h->smem_bytes, h->d_slab,
                                   h->slab_stride});
    } else {
        // One launch per size bucket of M (width 8), largest first.
        int b = 0;
        while (b < split) {
            const int bucket = order_m(h, b) / 8;
            int e = b;
            while (e < split && order_m(h, e) / 8 == bucket) ++e;
            h->launches.push_back({b, e, std::min(h->grid, e - b), h->kernel, kThreads, h->smem_bytes,
                                   h->d_slab, h->slab_stride});
            b = e;
        }
    }
    if (split < h->owned) {
        const int rc = plan_lean_launch(h, prop, split, h->owned, order_m(h, split));
        if (rc) return rc;
    }
    // Mixed precision: the FP64 pass over the blocks the mixed kernel hands
    // back runs the streamed kernel too when every block fits it (the list
    // is only known on the device, so the launch covers all positions).
    h->mixed_lean = false;
    if (h->opts.precision == BV_PREC_MIXED && (sched == BV_SCHED_STREAMED || sched == BV_SCHED_AUTO) &&
        h->owned > 0 && h->max_m <= lean_limit) {
        const int rc = plan_lean_launch(h, prop, 0, h->owned, h->max_m);
        if (rc) return rc;
        h->mixed_lean = true;
    }
    BV_CUDA_TRY(cudaMalloc(&h->d_counters, sizeof(unsigned) * std::max<size_t>(1, h->launches.size())));
    return BV_OK;
}

// Timing events around the fused kernel: inside a captured graph they must be
// external event-record nodes; on a plain stream, ordinary records.
static cudaError_t record_timing(cudaEvent_t ev, cudaStream_t s)
{
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(s, &cs);
    if (e != cudaSuccess) return e;
    return cs == cudaStreamCaptureStatusActive ? cudaEventRecordWithFlags(ev, s, cudaEventRecordExternal)
                                               : cudaEventRecord(ev, s);
}

static int capture_graph(bv_handle *h);

static int enqueue_eval(bv_handle *h, cudaStream_t s)
{
    BV_CUDA_TRY(cudaMemcpyAsync(h->d_mp, h->h_mp, sizeof(MaternParams), cudaMemcpyHostToDevice, s));
    BV_CUDA_TRY(cudaMemsetAsync(h->d_counters, 0, sizeof(unsigned) * std::max<size_t>(1, h->launches.size()), s));
    BV_CUDA_TRY(record_timing(h->evk0, s));
    auto fp64_args = [&](unsigned *counter, const int *order, int begin, int end) {
        LlhArgs a{};
        a.x = h->d_x;
        a.y = h->d_y;
        a.obs = h->d_obs;
        a.z = h->d_z;
        a.acc = h->d_acc;
        a.knn = h->d_knn;
        a.order = order;
        a.bc = h->bc;
        a.cs = h->cs;
        a.smem_max_m = h->smem_max_m;
        a.slab_max_m = h->max_m;
        a.block_llk = h->d_block_llk;
        a.block_status = h->d_block_status;
        a.work_counter = counter;
        a.gslab = h->d_slab;
        a.gslab_stride = h->slab_stride;
        a.big_max_m = h->use_big ? h->big_max_m : 0;
        a.log2pi = std::log(2 * 3.141592653589793);
        a.mp = h->d_mp;
        a.task_begin = begin;
        a.task_end = end;
        return a;
    };
    if (h->opts.precision == BV_PREC_MIXED) {
        // Mixed pass over the handle's blocks, then the FP64 kernel over the
        // blocks it handed back (the count is read on the device).
        MixedArgs ma{};
        ma.x = h->d_x;
        ma.y = h->d_y;
        ma.obs = h->d_obs;
        ma.acc = h->d_acc;
        ma.knn = h->d_knn;
        ma.order = h->d_order;
        ma.bc = h->bc;
        ma.cs = h->cs;
        ma.task_end = h->owned;
        ma.block_llk = h->d_block_llk;
        ma.block_status = h->d_block_status;
        ma.mp = h->d_mp;
        ma.tol = h->opts.mixed_tol;
        ma.log2pi = std::log(2 * 3.141592653589793);
        int rc = mixed_enqueue(h->mixed, ma, s);
        if (rc) return rc;
        if (h->owned > 0 && h->mixed_lean) {
            const size_t l = h->launches.size() - 1;
            const bv_handle::Launch &ln = h->launches[l];
            LlhArgs a = fp64_args(h->d_counters + l, h->mixed.fallback_list, 0, h->owned);
            a.task_count = h->mixed.fallback_count;
            a.status_or = BV_ST_FP32_FALLBACK;
            a.gslab = ln.slab;
            a.gslab_stride = ln.slab_stride;
            ln.kernel<<<ln.grid, ln.threads, ln.smem, s>>>(a);
            BV_CUDA_TRY(cudaGetLastError());
        } else if (h->owned > 0) {
            LlhArgs a = fp64_args(h->d_counters, h->mixed.fallback_list, 0, h->owned);
            a.task_count = h->mixed.fallback_count;
            a.status_or = BV_ST_FP32_FALLBACK;
            h->kernel<<<h->grid, h->block_threads, h->smem_bytes, s>>>(a);
            BV_CUDA_TRY(cudaGetLastError());
        }
    } else {
        for (size_t l = 0; l < h->launches.size(); ++l) {
            const bv_handle::Launch &ln = h->launches[l];
            LlhArgs a = fp64_args(h->d_counters + l, h->d_order, ln.begin, ln.end);
            a.gslab = ln.slab;
            a.gslab_stride = ln.slab_stride;
            ln.kernel<<<ln.grid, ln.threads, ln.smem, s>>>(a);
            BV_CUDA_TRY(cudaGetLastError());
        }
    }
    BV_CUDA_TRY(record_timing(h->evk1, s));
    reduce_kernel<<<1, kReduceThreads, 0, s>>>(h->d_block_llk, h->d_block_status, h->bc, h->d_res);
    BV_CUDA_TRY(cudaGetLastError());
    BV_CUDA_TRY(cudaMemcpyAsync(h->h_res, h->d_res, sizeof(EvalResult), cudaMemcpyDeviceToHost, s));
    return BV_OK;
}

extern "C" int bv_create(const bv_layout *L, const bv_opts *opts, bv_handle **out)
{
    if (!out) {
        set_error("bv_create: out is NULL");
        return BV_E_INVALID;
    }
    *out = nullptr;
    int rc = validate_layout(L);
    if (rc) return rc;
    bv_handle *h = new (std::nothrow) bv_handle();
    if (!h) return BV_E_NOMEM;
    if (opts)
        h->opts = *opts;
    else
        bv_default_opts(&h->opts);
    if (!(h->opts.dist_scale > 0)) h->opts.dist_scale = 1.0;
    h->device = h->opts.device;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= h->device) {
        cudaGetLastError();
        set_error("bv_create: no CUDA device %d", h->device);
        delete h;
        return BV_E_NODEVICE;
    }
#define BV_TRY_H(expr)            \
    do {                          \
        int _rc = (expr);         \
        if (_rc) {                \
            handle_free(h);       \
            return _rc;           \
        }                         \
    } while (0)
#define BV_CUDA_H(expr)                                                                  \
    do {                                                                                 \
        cudaError_t _e = (expr);                                                         \
        if (_e != cudaSuccess) {                                                         \
            set_error("%s: %s", #expr, cudaGetErrorString(_e));                          \
            handle_free(h);                                                              \
            return (_e == cudaErrorMemoryAllocation) ? BV_E_NOMEM : BV_E_CUDA;           \
        }                                                                                \
    } while (0)
    BV_CUDA_H(cudaSetDevice(h->device));
    cudaDeviceProp prop;
    BV_CUDA_H(cudaGetDeviceProperties(&prop, h->device));
    if (prop.major < 10) {
        set_error("bv_create: device %d is sm_%d%d; this library is built for sm_100a", h->device,
                  prop.major, prop.minor);
        handle_free(h);
        return BV_E_NODEVICE;
    }
    if (h->opts.kernel == 4 && !L->z) {
        set_error("bv_create: the space-time kernel (4) needs the layout's third coordinate (z)");
        handle_free(h);
        return BV_E_INVALID;
    }
    if (L->z && h->opts.precision == BV_PREC_MIXED) {
        set_error("bv_create: the mixed-precision path evaluates 2-D Matern layouts only");
        handle_free(h);
        return BV_E_INVALID;
    }
    if (h->opts.earth && (L->z || h->opts.kernel == 4)) {
        // src/ckernel.cpp:170-172: "Great Circle (GC) distance is only valid for 2d".
        set_error("bv_create: the great-circle distance (earth) is defined for 2-D locations only");
        handle_free(h);
        return BV_E_INVALID;
    }
    if (h->opts.earth && h->opts.precision == BV_PREC_MIXED) {
        set_error("bv_create: the mixed-precision path evaluates Euclidean distances only");
        handle_free(h);
        return BV_E_INVALID;
    }
    // Great-circle layouts run the 3-D kernel instantiations, whose third
    // coordinate then carries cos(latitude) of every point.
    h->nz = (L->z || h->opts.earth) ? 1 : 0;
    h->n = L->n;
    h->bc = L->bc;
    h->cs = L->cs;
    h->batchNum.assign(L->batchNum, L->batchNum + L->bc);
    h->acc.assign(L->batchNumAccum, L->batchNumAccum + L->bc + 1);
    h->max_m = 1;
    for (int b = 0; b < h->bc; ++b)
        h->max_m = std::max(h->max_m, h->batchNum[b] + (b == 0 ? 0 : h->cs));
    // Largest blocks first (longest-processing-time order), ties by index;
    // with sharding, every shard_count-th block of that order.
    if (h->opts.schedule < BV_SCHED_AUTO || h->opts.schedule > BV_SCHED_STREAMED) {
        set_error("bv_create: unknown schedule %d", h->opts.schedule);
        handle_free(h);
        return BV_E_INVALID;
    }
    if (h->opts.shard_count < 1 || h->opts.shard_index < 0 ||
        h->opts.shard_index >= h->opts.shard_count) {
        set_error("bv_create: shard_index %d outside [0, %d)", h->opts.shard_index,
                  h->opts.shard_count);
        handle_free(h);
        return BV_E_INVALID;
    }
    {
        const std::vector<int> all = cost_order(L->batchNum, L->bc, L->cs);
        h->order.clear();
        for (int t = 0; t < h->bc; ++t)
            if (t % h->opts.shard_count == h->opts.shard_index) h->order.push_back(all[t]);
    }
    h->owned = (int)h->order.size();

    BV_CUDA_H(cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking));
    h->stream = h->own_stream;
    BV_CUDA_H(cudaEventCreate(&h->ev0));
    BV_CUDA_H(cudaEventCreate(&h->ev1));
    BV_CUDA_H(cudaEventCreate(&h->evk0));
    BV_CUDA_H(cudaEventCreate(&h->evk1));
    const size_t n = h->n, bc = h->bc, cs = h->cs;
    BV_CUDA_H(cudaMalloc(&h->d_x, n * sizeof(double)));
    BV_CUDA_H(cudaMalloc(&h->d_y, n * sizeof(double)));
    BV_CUDA_H(cudaMalloc(&h->d_obs, n * sizeof(double)));
    BV_CUDA_H(cudaMalloc(&h->d_acc, (bc + 1) * sizeof(int)));
    BV_CUDA_H(cudaMalloc(&h->d_knn, std::max<size_t>(1, bc * cs) * sizeof(int)));
    BV_CUDA_H(cudaMalloc(&h->d_order, bc * sizeof(int)));
    BV_CUDA_H(cudaMalloc(&h->d_block_llk, bc * sizeof(double)));
    BV_CUDA_H(cudaMalloc(&h->d_block_status, bc * sizeof(unsigned)));
    BV_CUDA_H(cudaMalloc(&h->d_mp, sizeof(MaternParams)));
    BV_CUDA_H(cudaMalloc(&h->d_res, sizeof(EvalResult)));
    BV_CUDA_H(cudaMallocHost(&h->h_mp, sizeof(MaternParams)));
    BV_CUDA_H(cudaMallocHost(&h->h_res, sizeof(EvalResult)));
    BV_CUDA_H(cudaMemcpy(h->d_x, L->x, n * sizeof(double), cudaMemcpyHostToDevice));
    BV_CUDA_H(cudaMemcpy(h->d_y, L->y, n * sizeof(double), cudaMemcpyHostToDevice));
    BV_CUDA_H(cudaMemcpy(h->d_obs, L->obs, n * sizeof(double), cudaMemcpyHostToDevice));
    std::vector<double> ccos;  // centroids' cos(latitude), for the great-circle key
    if (L->z) {
        BV_CUDA_H(cudaMalloc(&h->d_z, n * sizeof(double)));
        BV_CUDA_H(cudaMemcpy(h->d_z, L->z, n * sizeof(double), cudaMemcpyHostToDevice));
    } else if (h->opts.earth) {
        std::vector<double> c(n);
        for (size_t p = 0; p < n; ++p) c[p] = earth_cos_lat(L->x[p]);
        BV_CUDA_H(cudaMalloc(&h->d_z, n * sizeof(double)));
        BV_CUDA_H(cudaMemcpy(h->d_z, c.data(), n * sizeof(double), cudaMemcpyHostToDevice));
        if (L->cx) {
            ccos.resize(bc);
            for (size_t b = 0; b < bc; ++b) ccos[b] = earth_cos_lat(L->cx[b]);
        }
    }
    BV_CUDA_H(cudaMemcpy(h->d_acc, L->batchNumAccum, (bc + 1) * sizeof(int), cudaMemcpyHostToDevice));
    if (h->owned > 0)
        BV_CUDA_H(cudaMemcpy(h->d_order, h->order.data(), h->owned * sizeof(int),
                             cudaMemcpyHostToDevice));
    // Blocks outside this handle's shard contribute exact zeros.
    BV_CUDA_H(cudaMemset(h->d_block_llk, 0, bc * sizeof(double)));
    BV_CUDA_H(cudaMemset(h->d_block_status, 0, bc * sizeof(unsigned)));
    if (cs > 0) {
        if (L->knn_idx) {
            BV_CUDA_H(cudaMemcpy(h->d_knn, L->knn_idx, bc * cs * sizeof(int), cudaMemcpyHostToDevice));
        } else {
            // A shard selects only its own blocks' sets (the others are
            // never read by this handle).
            std::vector<unsigned char> mine;
            if (h->opts.shard_count > 1) {
                mine.assign(h->bc, 0);
                for (int t = 0; t < h->owned; ++t) mine[h->order[t]] = 1;
                BV_CUDA_H(cudaMemsetAsync(h->d_knn, 0, bc * cs * sizeof(int), h->stream));
            }
            BV_TRY_H(knn_device(h->d_x, h->d_y, h->d_z, h->n, h->bc, h->cs, h->d_acc, L->cx, L->cy,
                                h->opts.earth ? ccos.data() : L->cz, h->d_knn, h->stream,
                                mine.empty() ? nullptr : mine.data(), h->opts.earth));
            BV_CUDA_H(cudaStreamSynchronize(h->stream));
        }
    }
    BV_TRY_H(plan_launches(h));
    if (h->opts.precision == BV_PREC_MIXED) {
        int max_bs = 0;
        for (int t = 0; t < h->owned; ++t) max_bs = std::max(max_bs, h->batchNum[h->order[t]]);
        BV_TRY_H(mixed_create(h->mixed, h->device, h->bc, h->cs, max_bs, h->order.data(), h->owned,
                              h->opts.mixed_fp32 != 0));
    }
    if (h->opts.use_graph) BV_TRY_H(capture_graph(h));
#undef BV_TRY_H
#undef BV_CUDA_H
    *out = h;
    return BV_OK;
}

extern "C" void bv_destroy(bv_handle *h) { handle_free(h); }

static int fill_params(bv_handle *h, const double *theta)
{
    const double sigma2 = theta[0], range = theta[1], nu = theta[2];
    if (!std::isfinite(sigma2) || !(range > 0) || !(nu > 0) || !std::isfinite(range) ||
        !std::isfinite(nu)) {
        set_error("bv_llh: invalid theta (%g, %g, %g)", sigma2, range, nu);
        return BV_E_INVALID;
    }
    const bool st = h->opts.kernel == 4;
    // The nugget follows the kernel's own parameters: theta[3], or theta[7]
    // after the space-time kernel's seven.
    const double tau2 = h->opts.nugget ? theta[st ? 7 : 3] : 0.0;
    if (!(tau2 >= 0) || !std::isfinite(tau2)) {
        set_error("bv_llh: invalid nugget %g", tau2);
        return BV_E_INVALID;
    }
    MaternParams &p = *h->h_mp;
    p.nugget = tau2;
    p.model = st ? kModelSpaceTime : (h->opts.earth ? kModelEarth : (h->nz ? kModel3D : kModel2D));
    p.st_range_t = p.st_pow = p.st_half = p.st_outer = 0.0;
    if (st) {
        // src/ckernel.cpp:1439-1443 (theta[3..6]).
        if (!(theta[3] > 0) || !std::isfinite(theta[3]) || !std::isfinite(theta[4]) ||
            !std::isfinite(theta[5]) || !std::isfinite(theta[6])) {
            set_error("bv_llh: invalid space-time parameters (%g, %g, %g, %g)", theta[3], theta[4],
                      theta[5], theta[6]);
            return BV_E_INVALID;
        }
        p.st_range_t = theta[3];
        p.st_pow = 2 * theta[4];
        p.st_half = theta[5] / 2.0;
        p.st_outer = theta[5] + theta[6];
    }
    p.sigma2 = sigma2;
    p.range = range;
    p.nu = nu;
    // src/ckernel.cpp:1072-1075, evaluated on the host as the reference does.
    double con = std::pow(2.0, nu - 1.0) * std::tgamma(nu);
    con = 1.0 / con;
    con = sigma2 * con;
    p.con = con;
    p.dist_scale = h->opts.dist_scale;
    p.scale_is_one = (h->opts.dist_scale == 1.0) ? 1 : 0;
    p.inv_range = 1.0 / range;
    p.inv_ds = 1.0 / h->opts.dist_scale;
    p.nu_kind = (nu == 0.5) ? kNuHalf : (nu == 1.5) ? kNuThreeHalves : (nu == 2.5) ? kNuFiveHalves
                                                                                  : kNuGeneral;
    matern_prepare(p);
    return BV_OK;
}

// One evaluation captured into the handle's graph (replacing any earlier).
static int capture_graph(bv_handle *h)
{
    if (h->gexec) cudaGraphExecDestroy(h->gexec);
    if (h->graph) cudaGraphDestroy(h->graph);
    h->gexec = nullptr;
    h->graph = nullptr;
    BV_CUDA_TRY(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    const int erc = enqueue_eval(h, h->stream);
    cudaGraph_t g = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(h->stream, &g);
    if (erc || ce != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        if (!erc) set_error("graph capture: %s", cudaGetErrorString(ce));
        return erc ? erc : BV_E_CUDA;
    }
    h->graph = g;
    BV_CUDA_TRY(cudaGraphInstantiate(&h->gexec, h->graph, 0));
    return BV_OK;
}

// The streamed launch (always the last one planned) again, with CTA size vi.
static int replan_lean(bv_handle *h, int vi)
{
    cudaDeviceProp prop;
    BV_CUDA_TRY(cudaGetDeviceProperties(&prop, h->device));
    h->launches.pop_back();
    cudaFree(h->d_slab_lean);
    h->d_slab_lean = nullptr;
    h->lean_choice = vi;
    return plan_lean_launch(h, prop, h->lean_begin, h->lean_end, h->lean_m);
}

// bv_opts.tune: on the first evaluation, time the streamed kernel at every
// CTA size (twice each, the faster kept) and keep the fastest.  The sizes
// give the same bits, so the evaluation's value does not depend on it.
static int tune_lean(bv_handle *h)
{
    h->tuned = true;
    int best = h->lean_choice >= 0 ? h->lean_choice : lean_variant(h->lean_m);
    double best_ms = 1e300;
    for (int vi = 0; vi < kNumLean; ++vi) {
        int rc = replan_lean(h, vi);
        if (rc) return rc;
        double t = 1e300;
        for (int rep = 0; rep < 2; ++rep) {
            rc = enqueue_eval(h, h->stream);
            if (rc) return rc;
            BV_CUDA_TRY(cudaStreamSynchronize(h->stream));
            float kms = 0.f;
            BV_CUDA_TRY(cudaEventElapsedTime(&kms, h->evk0, h->evk1));
            t = std::min(t, (double)kms);
        }
        h->tune_ms[vi] = t;
        if (t < best_ms) {
            best_ms = t;
            best = vi;
        }
    }
    int rc = replan_lean(h, best);
    if (rc) return rc;
    return h->opts.use_graph ? capture_graph(h) : BV_OK;
}

static int eval_locked(bv_handle *h, const double *theta, double *llk)
{
    int rc = fill_params(h, theta);
    if (rc) return rc;
    BV_CUDA_TRY(cudaSetDevice(h->device));
    if (h->opts.tune && !h->tuned && h->streamed_blocks > 0 && h->opts.precision == BV_PREC_FP64) {
        rc = tune_lean(h);
        if (rc) return rc;
    }
    BV_CUDA_TRY(cudaEventRecord(h->ev0, h->stream));
    if (h->gexec) {
        BV_CUDA_TRY(cudaGraphLaunch(h->gexec, h->stream));
    } else {
        rc = enqueue_eval(h, h->stream);
        if (rc) return rc;
    }
    BV_CUDA_TRY(cudaEventRecord(h->ev1, h->stream));
    BV_CUDA_TRY(cudaStreamSynchronize(h->stream));
    float ms = 0.f, kms = 0.f;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    cudaEventElapsedTime(&kms, h->evk0, h->evk1);
    const EvalResult r = *h->h_res;
    bv_status &s = h->status;
    s.blocks = h->owned;
    s.cond_fail = r.cond_fail;
    s.schur_fail = r.schur_fail;
    s.fp32_fallback = r.fallback;
    s.nonfinite = r.nonfinite;
    s.flags_or = r.flags_or;
    s.failed = r.failed;
    // FP64: the fused launches and the reduction; mixed: the probe (FP32
    // pass enabled and something to probe), the decision, the mixed pass
    // (FP32 pass enabled), the FP64 pass and the reduction.
    const bool mixed = h->opts.precision == BV_PREC_MIXED;
    if (!mixed)
        s.launches = (int)h->launches.size() + 1;
    else if (h->owned <= 0)
        s.launches = 1;
    else
        s.launches = 3 + (h->mixed.fp32 ? 1 + (h->mixed.nprobe > 0 ? 1 : 0) : 0);
    // Without the FP32 pass every block takes the FP64 pass, on the streamed
    // kernel when it covers the layout.
    s.streamed_blocks = !mixed ? h->streamed_blocks : (!h->mixed.fp32 && h->mixed_lean ? h->owned : 0);
    s.streamed_threads = s.streamed_blocks > 0 ? h->lean_threads : 0;
    s.streamed_variant = s.streamed_blocks > 0 ? h->lean_vi : -1;
    for (int i = 0; i < kNumLean; ++i) s.tune_ms[i] = h->tune_ms[i];
    s.llk = r.llk;
    s.device_ms = ms;
    s.kernel_ms = kms;
    double v = r.llk;
    const bool failed = (r.cond_fail + r.schur_fail + r.nonfinite) > 0 || !std::isfinite(v);
    if (failed && h->opts.on_failure == BV_FAIL_NEGINF) v = -HUGE_VAL;
    *llk = v;
    return BV_OK;
}

static void print_iteration(bv_handle *h, const double *theta, double llk)
{
    // include/llh_Xvecchia_batch.h:500-516
    if (h->opts.kernel == 4)
        printf("%dth Model Parameters (Variance, beta, nu, beta_time, nu_time, sep): (%lf, %lf, %lf, "
               "%lf, %lf, %lf) -> Loglik: %lf \n",
               h->iterations, theta[0], theta[1], theta[2], theta[3], theta[4], theta[5], llk);
    else if (h->opts.kernel == 3 || h->opts.nugget)
        printf("%dth Model Parameters (Variance, range, smoothness, nugget): (%1.8lf, %1.8lf, "
               "%1.8lf, %1.8lf) -> Loglik: %.18lf \n",
               h->iterations, theta[0], theta[1], theta[2], theta[3], llk);
    else
        printf("%dth Model Parameters (Variance, range, smoothness): (%1.8lf, %1.8lf, %1.8lf) -> "
               "Loglik: %.18lf \n",
               h->iterations, theta[0], theta[1], theta[2], llk);
}

extern "C" int bv_llh_eval(bv_handle *h, const double *theta, double *llk)
{
    if (!h || !theta || !llk) {
        set_error("bv_llh_eval: null argument");
        return BV_E_INVALID;
    }
    std::lock_guard<std::mutex> lk(h->mu);
    int rc = eval_locked(h, theta, llk);
    if (rc == BV_OK) {
        if (h->opts.print_iter) print_iteration(h, theta, *llk);
        h->iterations += 1;
    }
    return rc;
}

extern "C" double bv_llh(unsigned n, const double *theta, double *grad, void *f_data)
{
    (void)grad;
    bv_handle *h = static_cast<bv_handle *>(f_data);
    const unsigned need = h ? (h->opts.kernel == 4 ? 7u : 3u) + (h->opts.nugget ? 1u : 0u) : 3u;
    if (!h || !theta || n < need) {
        set_error("bv_llh: need a handle and at least %u parameters", need);
        return -HUGE_VAL;
    }
    double v = -HUGE_VAL;
    if (bv_llh_eval(h, theta, &v) != BV_OK) return -HUGE_VAL;
    return v;
}

extern "C" int bv_llh_host(bv_handle *h, const double *x, const double *y, const double *obs,
                           const int *knn_idx, const double *theta, double *llk)
{
    if (!h || !obs || !theta || !llk) {
        set_error("bv_llh_host: null argument");
        return BV_E_INVALID;
    }
    std::lock_guard<std::mutex> lk(h->mu);
    BV_CUDA_TRY(cudaSetDevice(h->device));
    const size_t n = h->n;
    if (x) BV_CUDA_TRY(cudaMemcpyAsync(h->d_x, x, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    if (y) BV_CUDA_TRY(cudaMemcpyAsync(h->d_y, y, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    BV_CUDA_TRY(cudaMemcpyAsync(h->d_obs, obs, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    if (knn_idx && h->cs > 0)
        BV_CUDA_TRY(cudaMemcpyAsync(h->d_knn, knn_idx, (size_t)h->bc * h->cs * sizeof(int),
                                    cudaMemcpyHostToDevice, h->stream));
    int rc = eval_locked(h, theta, llk);
    if (rc == BV_OK) h->iterations += 1;
    return rc;
}

extern "C" int bv_block_llk(bv_handle *h, double *out, int count)
{
    if (!h || !out || count < h->bc) {
        set_error("bv_block_llk: need room for %d values", h ? h->bc : 0);
        return BV_E_INVALID;
    }
    std::lock_guard<std::mutex> lk(h->mu);
    BV_CUDA_TRY(cudaSetDevice(h->device));
    BV_CUDA_TRY(cudaMemcpy(out, h->d_block_llk, sizeof(double) * h->bc, cudaMemcpyDeviceToHost));
    return BV_OK;
}

extern "C" int bv_block_status(bv_handle *h, unsigned *out, int count)
{
    if (!h || !out || count < h->bc) {
        set_error("bv_block_status: need room for %d values", h ? h->bc : 0);
        return BV_E_INVALID;
    }
    std::lock_guard<std::mutex> lk(h->mu);
    BV_CUDA_TRY(cudaSetDevice(h->device));
    BV_CUDA_TRY(cudaMemcpy(out, h->d_block_status, sizeof(unsigned) * h->bc, cudaMemcpyDeviceToHost));
    return BV_OK;
}

extern "C" int bv_get_status(bv_handle *h, bv_status *st)
{
    if (!h || !st) return BV_E_INVALID;
    std::lock_guard<std::mutex> lk(h->mu);
    *st = h->status;
    return BV_OK;
}

extern "C" int bv_iterations(bv_handle *h) { return h ? h->iterations : 0; }

extern "C" int bv_set_stream(bv_handle *h, void *stream)
{
    if (!h) return BV_E_INVALID;
    std::lock_guard<std::mutex> lk(h->mu);
    h->stream = stream ? (cudaStream_t)stream : h->own_stream;
    return BV_OK;
}

extern "C" int bv_get_stream(bv_handle *h, void **stream)
{
    if (!h || !stream) return BV_E_INVALID;
    *stream = (void *)h->stream;
    return BV_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free entry point.  For callers that cannot allocate device
// memory themselves or let a library do it (their allocator owns the GPU,
// or the host application manages every buffer).  Its working memory is one
// fixed array inside this library; see bv_llh_noalloc in include/bv.h.
// ---------------------------------------------------------------------------

namespace bv {

constexpr size_t kNoAllocBlocks = BV_NOALLOC_MAX_BLOCKS;
// Byte offsets of the regions carved out of the array (each 256-aligned).
constexpr size_t kNaLlk = 0;                                         // double[kNoAllocBlocks]
constexpr size_t kNaStatus = kNaLlk + kNoAllocBlocks * 8;            // unsigned[kNoAllocBlocks]
constexpr size_t kNaOrder = kNaStatus + kNoAllocBlocks * 4;          // int[kNoAllocBlocks]
constexpr size_t kNaCounter = kNaOrder + kNoAllocBlocks * 4;         // unsigned work counter
constexpr size_t kNaCheck = kNaCounter + 256;                        // int[4] validation
constexpr size_t kNaParams = kNaCheck + 256;                         // MaternParams
constexpr size_t kNaResult = kNaParams + 256;                        // EvalResult
constexpr size_t kNaBytes = kNaResult + 256;

// The working memory of bv_llh_noalloc: every device that loads the library
// holds it until exit.  Host code must use the address from
// cudaGetSymbolAddress, never the name.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];

static std::mutex g_noalloc_mu;
static unsigned char *g_noalloc_ptr[64] = {nullptr};
static int g_noalloc_smem_max_m[64] = {0};

// Validation of a caller's layout on the device: offsets non-decreasing and
// ending at n, every block fits in shared memory, every conditioning index of
// block b >= 1 lies in [0, batchNumAccum[b]), and block 0 holds at least cs
// points when other blocks condition on it (the rule bv_create applies).
// check[0] = first bad block + 1 (offsets/indices), check[1] = largest M,
// check[2] = 1 when block 0 is smaller than cs.
__global__ void noalloc_check_kernel(const int *acc, const int *knn, int n, int bc, int cs,
                                     int *check, int *order)
{
    const int stride = gridDim.x * blockDim.x;
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < bc; b += stride) {
        order[b] = b;
        const int a0 = acc[b], a1 = acc[b + 1];
        bool ok = a0 >= 0 && a1 >= a0 && a1 <= n && (b + 1 < bc || a1 == n) && (b > 0 || a0 == 0);
        const int M = (a1 - a0) + (b == 0 ? 0 : cs);
        atomicMax(&check[1], M);
        if (b == 0 && cs > 0 && bc > 1 && a1 - a0 < cs) check[2] = 1;
        if (ok && b > 0 && cs > 0) {
            const int *k = knn + (size_t)b * cs;
            for (int t = 0; t < cs; ++t)
                if (k[t] < 0 || k[t] >= a0) {
                    ok = false;
                    break;
                }
        }
        if (!ok) atomicCAS(&check[0], 0, b + 1);
    }
}

// Final value of an allocation-free call: the reduced log-likelihood, or
// -HUGE_VAL when a block failed or the sum is not finite (the handle's
// default failure policy, BV_FAIL_NEGINF).
__global__ void noalloc_result_kernel(const EvalResult *r, double *llk_out)
{
    const double v = r->llk;
    const bool failed = (r->cond_fail + r->schur_fail + r->nonfinite) > 0 || !isfinite(v);
    *llk_out = failed ? -HUGE_VAL : v;
}

}  // namespace bv

extern "C" int bv_llh_noalloc(const double *x, const double *y, const double *obs,
                              const int *batchNumAccum, const int *knn_idx, int n, int bc, int cs,
                              const double *theta, double dist_scale, double *llk_out,
                              unsigned *status_flags, void *stream)
{
    using namespace bv;
    if (!x || !y || !obs || !batchNumAccum || !theta || !llk_out || n <= 0 || bc <= 0 || cs < 0 ||
        (cs > 0 && !knn_idx)) {
        set_error("bv_llh_noalloc: null pointer or non-positive size");
        return BV_E_INVALID;
    }
    if ((size_t)bc > kNoAllocBlocks) {
        set_error("bv_llh_noalloc: %d blocks exceed the fixed maximum of %d", bc,
                  (int)kNoAllocBlocks);
        return BV_E_TOOLARGE;
    }
    cudaStream_t s = (cudaStream_t)stream;
    int dev = 0;
    BV_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) {
        set_error("bv_llh_noalloc: device ordinal %d unsupported", dev);
        return BV_E_NODEVICE;
    }
    unsigned char *base = nullptr;
    int smem_max_m = 0;
    {
        // Once per device, with that device current: the array's device
        // address and the fused kernel's shared-memory size.
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!g_noalloc_ptr[dev]) {
            void *p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) {
                set_error("bv_llh_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
                return BV_E_CUDA;
            }
            int optin = 0;
            BV_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
            g_noalloc_smem_max_m[dev] = max_m_for_bytes((size_t)optin - fused_static_smem(), sizeof(double));
            g_noalloc_ptr[dev] = (unsigned char *)p;
        }
        base = g_noalloc_ptr[dev];
        smem_max_m = g_noalloc_smem_max_m[dev];
    }
    int *check = reinterpret_cast<int *>(base + kNaCheck);
    int *order = reinterpret_cast<int *>(base + kNaOrder);
    unsigned *counter = reinterpret_cast<unsigned *>(base + kNaCounter);
    // Validate the layout on the device; read back 8 bytes.
    BV_CUDA_TRY(cudaMemsetAsync(check, 0, 3 * sizeof(int), s));
    noalloc_check_kernel<<<(bc + 255) / 256, 256, 0, s>>>(batchNumAccum, knn_idx, n, bc, cs, check,
                                                          order);
    BV_CUDA_TRY(cudaGetLastError());
    int hc[3] = {0, 0, 0};
    BV_CUDA_TRY(cudaMemcpyAsync(hc, check, sizeof(hc), cudaMemcpyDeviceToHost, s));
    BV_CUDA_TRY(cudaStreamSynchronize(s));
    if (hc[2]) {
        set_error("bv_llh_noalloc: block 0 has fewer than cs=%d points (firstbatch merges "
                  "clusters until >= cs)", cs);
        return BV_E_INVALID;
    }
    if (hc[0]) {
        set_error("bv_llh_noalloc: block %d has inconsistent offsets or a conditioning index "
                  "outside the earlier blocks", hc[0] - 1);
        return BV_E_INVALID;
    }
    if (hc[1] > smem_max_m) {
        set_error("bv_llh_noalloc: a block needs cs + bs = %d > %d, the largest block one SM's "
                  "shared memory holds", hc[1], smem_max_m);
        return BV_E_TOOLARGE;
    }
    // Parameters (host-computed as in bv_llh_eval) into the array.
    const double sigma2 = theta[0], range = theta[1], nu = theta[2];
    if (!std::isfinite(sigma2) || !(range > 0) || !(nu > 0) || !std::isfinite(range) ||
        !std::isfinite(nu) || !(dist_scale > 0)) {
        set_error("bv_llh_noalloc: invalid theta (%g, %g, %g) or dist_scale %g", sigma2, range,
                  nu, dist_scale);
        return BV_E_INVALID;
    }
    MaternParams mp{};
    mp.model = kModel2D;
    double con = std::pow(2.0, nu - 1.0) * std::tgamma(nu);
    con = 1.0 / con;
    mp.sigma2 = sigma2;
    mp.range = range;
    mp.nu = nu;
    mp.con = sigma2 * con;
    mp.dist_scale = dist_scale;
    mp.scale_is_one = dist_scale == 1.0 ? 1 : 0;
    mp.inv_range = 1.0 / range;
    mp.inv_ds = 1.0 / dist_scale;
    mp.nu_kind = (nu == 0.5) ? kNuHalf : (nu == 1.5) ? kNuThreeHalves : (nu == 2.5) ? kNuFiveHalves
                                                                                  : kNuGeneral;
    matern_prepare(mp);
    MaternParams *d_mp = reinterpret_cast<MaternParams *>(base + kNaParams);
    BV_CUDA_TRY(cudaMemcpyAsync(d_mp, &mp, sizeof(mp), cudaMemcpyHostToDevice, s));
    // The work counter must start at zero; per-block results are fully
    // overwritten by the kernel.
    BV_CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(unsigned), s));
    int sms = 0;
    BV_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    // The kernel's dynamic shared-memory limit is a per-function setting that
    // other callers also set; every caller sets the same device maximum, and
    // it is set for every call.
    const size_t smem = block_doubles(smem_max_m) * sizeof(double);
    int optin_na = 0;
    BV_CUDA_TRY(cudaDeviceGetAttribute(&optin_na, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    BV_CUDA_TRY(cudaFuncSetAttribute(llh_fp64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)((size_t)optin_na - fused_static_smem())));
    LlhArgs a{};
    a.x = x;
    a.y = y;
    a.obs = obs;
    a.acc = batchNumAccum;
    a.knn = knn_idx;
    a.order = order;
    a.bc = bc;
    a.cs = cs;
    a.smem_max_m = smem_max_m;
    a.slab_max_m = smem_max_m;
    a.block_llk = reinterpret_cast<double *>(base + kNaLlk);
    a.block_status = reinterpret_cast<unsigned *>(base + kNaStatus);
    a.work_counter = counter;
    a.gslab = nullptr;  // never used: every block fits in shared memory (checked above)
    a.gslab_stride = 0;
    a.log2pi = std::log(2 * 3.141592653589793);
    a.mp = d_mp;
    a.task_begin = 0;
    a.task_end = bc;
    llh_fp64_kernel<<<sms, kThreads, smem, s>>>(a);
    BV_CUDA_TRY(cudaGetLastError());
    EvalResult *d_res = reinterpret_cast<EvalResult *>(base + kNaResult);
    reduce_kernel<<<1, kReduceThreads, 0, s>>>(a.block_llk, a.block_status, bc, d_res);
    BV_CUDA_TRY(cudaGetLastError());
    noalloc_result_kernel<<<1, 1, 0, s>>>(d_res, llk_out);
    BV_CUDA_TRY(cudaGetLastError());
    unsigned flags = 0;
    BV_CUDA_TRY(cudaMemcpyAsync(&flags, &d_res->flags_or, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    BV_CUDA_TRY(cudaStreamSynchronize(s));
    if (status_flags) *status_flags = flags;
    return BV_OK;
}

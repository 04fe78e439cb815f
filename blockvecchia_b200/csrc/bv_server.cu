// bv_server.cu -- continuous-batching evaluation server for many concurrent
// fitting jobs on one device.
//
// Jobs.  Each job (locations, observations, block offsets, conditioning
// indices) is copied to HBM when its footprint fits the server's budget; jobs
// that do not fit wait in FIFO order and are admitted as others close.
//
// Batches.  A scheduler thread takes every pending request of the admitted
// jobs (up to max_batch) as soon as one of `max_inflight` batch slots is free
// and launches the multi-CTA streamed kernel over the blocks of all of them,
// largest blocks first (blocks beyond its shared memory in a persistent
// launch before it, as under the handles' default schedule).  Each slot has its own stream, so a batch launched while
// another runs starts on the SMs that the running batch's CTAs give up at its
// tail: requests that arrive during a batch overlap with it on the device.
// The CTA that completes the last block of a request reduces that request's
// contributions in the same launch (no trailing kernel that would wait behind
// the next batch's CTAs), and a completion thread per slot hands the results
// back.
//
// Determinism.  Per-block work (process_block_big / run_block) and the
// per-request reduction (reduce_blocks) are the code of the single-job path,
// so a result is bit-identical to bv_llh_eval on the same layout under the
// default schedule, alone or in any mix.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/bv.h"
#include "bv_common.cuh"
#include "bv_llh_big.cuh"
#include "bv_reduce.cuh"

namespace bv {

// One request of a batch: the job's device data and the request's parameters.
struct JobDesc {
    LlhArgs a;       // block_llk/block_status point into the slot's buffers
    MaternParams mp;
    unsigned *done;  // blocks of this request completed so far
    EvalResult *out;
};

// Persistent server kernel.  tasks[t] = (request, block), largest blocks of
// all requests first.  After a block, thread 0 publishes its contribution
// (fence, then the request's completion counter); the CTA that completes a
// request's last block reduces all of the request's blocks.
template <bool kBig>
__global__ void __launch_bounds__(kThreads, 1) llh_fp64_server_kernel(const JobDesc *descs,
                                                                     const int2 *tasks, int ntasks,
                                                                     unsigned *counter)
{
    extern __shared__ __align__(128) double smem[];
    __shared__ BlockShared sh;
    __shared__ int s_last;
    const int tid = threadIdx.x;
    init_block_sync(sh);
    for (;;) {
        if (tid == 0) sh.task = (int)atomicAdd(counter, 1u);
        __syncthreads();
        const int t = sh.task;
        if (t >= ntasks) break;
        const int2 tk = tasks[t];
        const JobDesc &d = descs[tk.x];
        const LlhArgs a = d.a;
        const MaternParams mp = d.mp;
        run_block<kBig>(a, mp, tk.y, smem, sh);
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            const unsigned prev = atomicAdd(d.done, 1u);
            s_last = (prev + 1u == (unsigned)a.bc) ? 1 : 0;
        }
        __syncthreads();
        if (s_last) {
            __threadfence();
            reduce_blocks(a.block_llk, a.block_status, a.bc, d.out, smem);
        }
    }
}

// The multi-CTA streamed kernel's server form: the same task list protocol
// over the blocks whose two panels fit in shared memory (the rest run the
// kernel above), NT threads per CTA, MINB CTAs per SM, one global slab per
// CTA.  Per block the code of the handles' default path (process_block_big,
// panel-by-panel generation), so a request's blocks give the bits a handle
// created with the default schedule gives.
template <int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) llh_lean_server_kernel(const JobDesc *descs, const int2 *tasks,
                                                                   int ntasks, unsigned *counter,
                                                                   double *slab0, size_t slab_stride)
{
    // Only LeanShared as static shared memory, as the handles' kernel, so the
    // two route a block by the same shared-memory limit.  The "last block of
    // its request" flag travels in sh.red, unused between blocks.
    extern __shared__ __align__(128) double smem[];
    __shared__ LeanShared sh;
    const int tid = threadIdx.x;
    double *slab = slab0 + (size_t)blockIdx.x * slab_stride;
    for (;;) {
        if (tid == 0) {
            sh.task = (int)atomicAdd(counter, 1u);
            sh.status = 0u;
        }
        __syncthreads();
        const int t = sh.task;
        if (t >= ntasks) break;
        const int2 tk = tasks[t];
        const JobDesc &d = descs[tk.x];
        const LlhArgs a = d.a;
        const int b = tk.y;
        if (a.acc[b + 1] == a.acc[b]) {  // empty block: contributes -(0 + 0 + 0) / 2
            if (tid == 0) {
                a.block_llk[b] = -0.0;
                a.block_status[b] = a.status_or;
            }
        } else {
            const MaternParams mp = d.mp;
            process_block_big<NT, 64, LeanShared, 0, false, false>(a, mp, b,
                                                                   reinterpret_cast<unsigned char *>(smem),
                                                                   slab, sh);
        }
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            const unsigned prev = atomicAdd(d.done, 1u);
            sh.red[0][0] = (prev + 1u == (unsigned)a.bc) ? 1.0 : 0.0;
        }
        __syncthreads();
        if (sh.red[0][0] != 0.0) {
            __threadfence();
            reduce_blocks(a.block_llk, a.block_status, a.bc, d.out, smem);
        }
    }
}

struct LeanServerVariant {
    void (*kernel)(const JobDesc *, const int2 *, int, unsigned *, double *, size_t);
    int threads;
};
static const LeanServerVariant kLeanServer[] = {
    {llh_lean_server_kernel<128, 4>, 128},
    {llh_lean_server_kernel<160, 3>, 160},
    {llh_lean_server_kernel<256, 2>, 256},
};

}  // namespace bv

using namespace bv;
using Clock = std::chrono::steady_clock;

namespace {

struct Job {
    int id = 0;
    int n = 0, bc = 0, cs = 0, max_m = 1;
    double dist_scale = 1.0;
    bool nugget = false;  // theta[3] = tau^2 on the covariance diagonals
    std::vector<int> acc, knn;
    std::vector<double> x, y, obs;
    std::vector<int> sorted;   // blocks by M descending (ties by index)
    std::vector<int> m_start;  // runs of equal M in `sorted`: start offsets
    std::vector<int> m_value;  // ... and their M
    bool big = false;  // blocks above the shared-memory limit use the streamed path
    size_t footprint = 0;
    bool admitted = false, uploading = false, closing = false;
    int inflight = 0;
    double *d_x = nullptr, *d_y = nullptr, *d_obs = nullptr;
    int *d_acc = nullptr, *d_knn = nullptr;
};

struct Req {
    long long id = 0;
    int job = 0;
    double theta[4] = {0, 0, 0, 0};  // theta[3]: the nugget, 0 unless the job has one
    Clock::time_point submitted;
    bool done = false;
    int rc = BV_OK;
    double llk = 0.0, latency_ms = 0.0;
};

template <class T>
bool grow_async(T *&p, size_t &cap, size_t need, cudaStream_t s)
{
    if (need <= cap) return true;
    if (p) cudaFreeAsync(p, s);
    p = nullptr;
    const size_t c = std::max<size_t>(need, cap + cap / 2);
    if (cudaMallocAsync(reinterpret_cast<void **>(&p), c * sizeof(T), s) != cudaSuccess) {
        cudaGetLastError();
        p = nullptr;
        cap = 0;
        return false;
    }
    cap = c;
    return true;
}

template <class T>
bool grow_pinned(T *&p, size_t &cap, size_t need)
{
    if (need <= cap) return true;
    if (p) cudaFreeHost(p);
    p = nullptr;
    const size_t c = std::max<size_t>(need, cap + cap / 2);
    if (cudaHostAlloc(reinterpret_cast<void **>(&p), c * sizeof(T), cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        p = nullptr;
        cap = 0;
        return false;
    }
    cap = c;
    return true;
}

}  // namespace

struct bv_server {
    struct Slot {
        int index = 0;
        cudaStream_t s = nullptr;
        // device
        double *bllk = nullptr;
        unsigned *bst = nullptr;
        size_t cap_bllk = 0, cap_bst = 0;
        int2 *tasks = nullptr;
        size_t cap_tasks = 0;
        JobDesc *desc = nullptr;
        EvalResult *res = nullptr;
        unsigned *counters = nullptr;  // [0]: work counter, [1 + r]: request r's done count
        double *slab = nullptr;
        size_t slab_stride = 0;
        int slab_max_m = 0;
        double *lean_slab = nullptr;  // the streamed kernel's per-CTA slabs
        size_t lean_bytes = 0;
        // pinned host staging
        int2 *h_tasks = nullptr;
        size_t cap_h_tasks = 0;
        JobDesc *h_desc = nullptr;
        EvalResult *h_res = nullptr;
        // state
        std::vector<long long> batch;
        bool busy = false, launched = false, ok = true;
        std::string err;
        std::condition_variable cv;
        std::thread completer;
    };

    bv_server_opts opts{};
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::thread scheduler;
    bool stop = false;
    int next_job = 1;
    long long next_req = 1;
    std::map<int, std::unique_ptr<Job>> jobs;
    std::deque<int> admit_queue;
    std::deque<long long> pending;
    std::map<long long, Req> reqs;
    size_t bytes_in_use = 0;
    long long evals = 0, batches = 0, batch_requests = 0;
    std::vector<double> latencies;
    std::vector<std::unique_ptr<Slot>> slots;
    // device constants
    int smem_cap_m = 0;
    int big_max_m = 0;
    size_t smem_bytes = 0;
    int grid = 0;
    int lean_limit = 0;  // blocks up to this M run the streamed kernel
    int sms = 0;
    cudaStream_t upload = nullptr;
};

namespace {

size_t job_footprint(const Job &j)
{
    return (size_t)j.n * 3 * sizeof(double) + (size_t)(j.bc + 1) * sizeof(int) +
           (size_t)j.bc * j.cs * sizeof(int);
}

void free_job_device(Job &j, cudaStream_t s)
{
    if (j.d_x) cudaFreeAsync(j.d_x, s);
    if (j.d_y) cudaFreeAsync(j.d_y, s);
    if (j.d_obs) cudaFreeAsync(j.d_obs, s);
    if (j.d_acc) cudaFreeAsync(j.d_acc, s);
    if (j.d_knn) cudaFreeAsync(j.d_knn, s);
    j.d_x = j.d_y = j.d_obs = nullptr;
    j.d_acc = j.d_knn = nullptr;
}

// Copy a job to the device on the upload stream; false on allocation failure.
bool upload_job(bv_server *S, Job &j)
{
    const size_t n = j.n, bc = j.bc, cs = j.cs;
    cudaStream_t s = S->upload;
    bool ok = cudaMallocAsync(reinterpret_cast<void **>(&j.d_x), n * 8, s) == cudaSuccess &&
              cudaMallocAsync(reinterpret_cast<void **>(&j.d_y), n * 8, s) == cudaSuccess &&
              cudaMallocAsync(reinterpret_cast<void **>(&j.d_obs), n * 8, s) == cudaSuccess &&
              cudaMallocAsync(reinterpret_cast<void **>(&j.d_acc), (bc + 1) * 4, s) == cudaSuccess &&
              (bc * cs == 0 ||
               cudaMallocAsync(reinterpret_cast<void **>(&j.d_knn), bc * cs * 4, s) == cudaSuccess);
    if (ok) {
        ok = cudaMemcpyAsync(j.d_x, j.x.data(), n * 8, cudaMemcpyHostToDevice, s) == cudaSuccess &&
             cudaMemcpyAsync(j.d_y, j.y.data(), n * 8, cudaMemcpyHostToDevice, s) == cudaSuccess &&
             cudaMemcpyAsync(j.d_obs, j.obs.data(), n * 8, cudaMemcpyHostToDevice, s) == cudaSuccess &&
             cudaMemcpyAsync(j.d_acc, j.acc.data(), (bc + 1) * 4, cudaMemcpyHostToDevice, s) == cudaSuccess &&
             (bc * cs == 0 ||
              cudaMemcpyAsync(j.d_knn, j.knn.data(), bc * cs * 4, cudaMemcpyHostToDevice, s) == cudaSuccess);
    }
    ok = (cudaStreamSynchronize(s) == cudaSuccess) && ok;
    if (!ok) {
        cudaGetLastError();
        free_job_device(j, s);
        cudaStreamSynchronize(s);
    }
    return ok;
}

void fill_params(MaternParams &p, const double *theta, double dist_scale)
{
    // The same parameter record as the single-job path (src/ckernel.cpp:1072-1075).
    const double sigma2 = theta[0], range = theta[1], nu = theta[2];
    double con = std::pow(2.0, nu - 1.0) * std::tgamma(nu);
    con = 1.0 / con;
    p.sigma2 = sigma2;
    p.range = range;
    p.nu = nu;
    p.con = sigma2 * con;
    p.dist_scale = dist_scale;
    p.scale_is_one = dist_scale == 1.0 ? 1 : 0;
    p.inv_range = 1.0 / range;
    p.inv_ds = 1.0 / dist_scale;
    p.nu_kind = (nu == 0.5) ? kNuHalf : (nu == 1.5) ? kNuThreeHalves : (nu == 2.5) ? kNuFiveHalves
                                                                                  : kNuGeneral;
    p.nugget = theta[3];
    p.model = kModel2D;
    matern_prepare(p);
}

// Requests of admitted jobs are ready to run.
bool has_ready(bv_server *S)
{
    for (long long id : S->pending) {
        auto jt = S->jobs.find(S->reqs[id].job);
        if (jt != S->jobs.end() && jt->second->admitted) return true;
    }
    return false;
}

bv_server::Slot *free_slot(bv_server *S)
{
    for (auto &sl : S->slots)
        if (!sl->busy) return sl.get();
    return nullptr;
}

bool can_admit(bv_server *S)
{
    if (S->admit_queue.empty()) return false;
    const Job &j = *S->jobs[S->admit_queue.front()];
    return S->bytes_in_use + j.footprint <= S->opts.hbm_budget;
}

bool can_release(bv_server *S)
{
    for (auto &kv : S->jobs)
        if (kv.second->closing && kv.second->inflight == 0 && !kv.second->uploading) return true;
    return false;
}

// The streamed server kernel's launch for blocks up to M = max_m: variant
// from the handles' table, shared memory, the full grid (CTAs resident per
// SM x SMs) and the per-CTA slab stride.
struct LeanLaunch {
    const LeanServerVariant *v = nullptr;
    size_t smem = 0, stride = 0;
    int grid = 0;
};

bool lean_launch_for(const bv_server *S, int max_m, LeanLaunch &ll)
{
    const int t = lean_table_threads(max_m);
    ll.v = &kLeanServer[t == 128 ? 0 : (t == 160 ? 1 : 2)];
    ll.smem = std::max<size_t>(big_layout(max_m, 64, 0, 0).total, kReduceScratchBytes);
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, ll.v->kernel, ll.v->threads, ll.smem) != cudaSuccess ||
        occ < 1) {
        cudaGetLastError();
        return false;
    }
    ll.grid = S->sms * occ;
    ll.stride = (big_slab_doubles(max_m) + 31) & ~(size_t)31;
    return true;
}

// Build the batch's descriptors and tasks in the slot and launch it.
// Called by the scheduler without the lock; `jobs[r]` stay alive and
// unchanged while their requests are in flight.
bool launch_batch(bv_server *S, bv_server::Slot &sl, const std::vector<Job *> &jobs,
                  const std::vector<Req> &rq)
{
    const int R = (int)jobs.size();
    size_t total = 0;
    bool any_big = false;
    for (const Job *j : jobs) {
        total += j->bc;
        any_big = any_big || j->big;
    }
    cudaStream_t s = sl.s;
    bool ok = grow_async(sl.bllk, sl.cap_bllk, total, s) && grow_async(sl.bst, sl.cap_bst, total, s) &&
              grow_async(sl.tasks, sl.cap_tasks, total, s) && grow_pinned(sl.h_tasks, sl.cap_h_tasks, total);
    if (!ok) {
        sl.err = "out of memory for the batch buffers";
        return false;
    }
    // Tasks: merge the jobs' runs of equal M, largest M first.  Blocks above
    // the streamed kernel's limit (the first n_pers tasks) run the persistent
    // kernel, the others the streamed kernel, as under the handles' default
    // schedule.
    size_t n_pers = 0;
    int pers_max_m = 0, lean_max_m = 0;
    {
        std::vector<size_t> run(R, 0);
        size_t w = 0;
        for (;;) {
            int best = -1;
            for (int r = 0; r < R; ++r)
                if (run[r] < jobs[r]->m_value.size() &&
                    (best < 0 || jobs[r]->m_value[run[r]] > jobs[best]->m_value[run[best]]))
                    best = r;
            if (best < 0) break;
            const int m = jobs[best]->m_value[run[best]];
            for (int r = best; r < R; ++r) {
                const Job &j = *jobs[r];
                if (run[r] < j.m_value.size() && j.m_value[run[r]] == m) {
                    const int b0 = j.m_start[run[r]];
                    const int b1 = (run[r] + 1 < j.m_start.size()) ? j.m_start[run[r] + 1] : j.bc;
                    for (int p = b0; p < b1; ++p) sl.h_tasks[w++] = make_int2(r, j.sorted[p]);
                    run[r]++;
                }
            }
            if (m > S->lean_limit) {
                n_pers = w;
                pers_max_m = std::max(pers_max_m, m);
            } else {
                lean_max_m = std::max(lean_max_m, m);
            }
        }
        total = w;
    }
    // Slabs: the persistent kernel's (blocks beyond shared memory) and the
    // streamed kernel's per-CTA slabs.
    if (n_pers > 0 && pers_max_m > S->smem_cap_m && pers_max_m > sl.slab_max_m) {
        if (sl.slab) cudaFreeAsync(sl.slab, s);
        // Covers both a streamed-path job and any job whose large blocks take
        // the slab path.
        sl.slab_stride = std::max(big_slab_stride(pers_max_m, S->smem_cap_m, S->big_max_m),
                                  (block_doubles(pers_max_m) + 31) & ~(size_t)31);
        ok = cudaMallocAsync(reinterpret_cast<void **>(&sl.slab), sl.slab_stride * 8 * S->grid, s) ==
             cudaSuccess;
        sl.slab_max_m = ok ? pers_max_m : 0;
        if (!ok) {
            cudaGetLastError();
            sl.slab = nullptr;
        }
    }
    LeanLaunch ll;
    if (ok && total > n_pers) {
        ok = lean_launch_for(S, lean_max_m, ll);
        ll.grid = std::max(1, std::min<int>(ll.grid, (int)(total - n_pers)));
        const size_t bytes = ll.stride * 8 * (size_t)ll.grid;
        if (ok && bytes > sl.lean_bytes) {
            if (sl.lean_slab) cudaFreeAsync(sl.lean_slab, s);
            ok = cudaMallocAsync(reinterpret_cast<void **>(&sl.lean_slab), bytes, s) == cudaSuccess;
            sl.lean_bytes = ok ? bytes : 0;
            if (!ok) {
                cudaGetLastError();
                sl.lean_slab = nullptr;
            }
        }
    }
    if (!ok) {
        sl.err = "out of memory for the batch buffers";
        return false;
    }
    // Descriptors.
    size_t off = 0;
    for (int r = 0; r < R; ++r) {
        const Job &j = *jobs[r];
        JobDesc &d = sl.h_desc[r];
        LlhArgs &a = d.a;
        std::memset(&a, 0, sizeof(a));
        a.x = j.d_x;
        a.y = j.d_y;
        a.obs = j.d_obs;
        a.acc = j.d_acc;
        a.knn = j.d_knn;
        a.order = nullptr;
        a.bc = j.bc;
        a.cs = j.cs;
        a.smem_max_m = S->smem_cap_m;
        a.slab_max_m = sl.slab_max_m;
        a.block_llk = sl.bllk + off;
        a.block_status = sl.bst + off;
        a.work_counter = nullptr;
        a.gslab = sl.slab;
        a.gslab_stride = sl.slab_stride;
        a.big_max_m = j.big ? S->big_max_m : 0;
        a.log2pi = std::log(2 * 3.141592653589793);
        a.mp = nullptr;
        a.task_begin = a.task_end = 0;
        fill_params(d.mp, rq[r].theta, j.dist_scale);
        d.done = sl.counters + 1 + r;
        d.out = sl.res + r;
        off += j.bc;
    }
    ok = cudaMemsetAsync(sl.counters, 0, (2 + R) * sizeof(unsigned), s) == cudaSuccess &&
         cudaMemcpyAsync(sl.desc, sl.h_desc, R * sizeof(JobDesc), cudaMemcpyHostToDevice, s) == cudaSuccess &&
         cudaMemcpyAsync(sl.tasks, sl.h_tasks, total * sizeof(int2), cudaMemcpyHostToDevice, s) == cudaSuccess;
    if (ok && n_pers > 0) {
        const int grid = std::max(1, std::min<int>(S->grid, (int)n_pers));
        // The streamed large-block path is compiled in only when a block needs it.
        auto kern = any_big ? llh_fp64_server_kernel<true> : llh_fp64_server_kernel<false>;
        kern<<<grid, kThreads, S->smem_bytes, s>>>(sl.desc, sl.tasks, (int)n_pers, sl.counters);
        ok = cudaGetLastError() == cudaSuccess;
    }
    if (ok && ll.v) {
        ll.v->kernel<<<ll.grid, ll.v->threads, ll.smem, s>>>(sl.desc, sl.tasks + n_pers, (int)(total - n_pers),
                                                             sl.counters + 1 + R, sl.lean_slab, ll.stride);
        ok = cudaGetLastError() == cudaSuccess;
    }
    ok = ok && cudaMemcpyAsync(sl.h_res, sl.res, R * sizeof(EvalResult), cudaMemcpyDeviceToHost, s) ==
                   cudaSuccess;
    if (!ok) sl.err = cudaGetErrorString(cudaGetLastError());
    return ok;
}

void scheduler_main(bv_server *S)
{
    cudaSetDevice(S->opts.device);
    std::unique_lock<std::mutex> lk(S->mu);
    for (;;) {
        S->cv_work.wait(lk, [&] {
            return S->stop || can_release(S) || can_admit(S) || (free_slot(S) && has_ready(S));
        });
        if (S->stop) break;
        // Release closed jobs whose requests have all completed.
        std::vector<std::unique_ptr<Job>> released;
        for (auto it = S->jobs.begin(); it != S->jobs.end();) {
            Job &j = *it->second;
            if (j.closing && j.inflight == 0 && !j.uploading) {
                if (j.admitted) S->bytes_in_use -= j.footprint;
                S->admit_queue.erase(std::remove(S->admit_queue.begin(), S->admit_queue.end(), j.id),
                                     S->admit_queue.end());
                released.push_back(std::move(it->second));
                it = S->jobs.erase(it);
            } else {
                ++it;
            }
        }
        // Admit waiting jobs, in order, while they fit.
        std::vector<Job *> admit;
        while (can_admit(S)) {
            Job *j = S->jobs[S->admit_queue.front()].get();
            S->admit_queue.pop_front();
            j->uploading = true;
            S->bytes_in_use += j->footprint;
            admit.push_back(j);
        }
        // Take a batch of ready requests (FIFO) if a slot is free.
        bv_server::Slot *sl = free_slot(S);
        std::vector<Job *> bjobs;
        std::vector<Req> breqs;
        if (sl) {
            std::deque<long long> rest;
            for (long long id : S->pending) {
                Req &r = S->reqs[id];
                auto jt = S->jobs.find(r.job);
                Job *j = (jt != S->jobs.end()) ? jt->second.get() : nullptr;
                if (j && j->admitted && (int)breqs.size() < S->opts.max_batch) {
                    sl->batch.push_back(id);
                    bjobs.push_back(j);
                    breqs.push_back(r);
                } else {
                    rest.push_back(id);
                }
            }
            S->pending.swap(rest);
            if (!breqs.empty())
                sl->busy = true;
            else
                sl = nullptr;
        }
        lk.unlock();
        for (auto &j : released)
            if (j->admitted) free_job_device(*j, S->upload);
        std::vector<bool> uploaded;
        for (Job *j : admit) uploaded.push_back(upload_job(S, *j));
        bool launched = false;
        if (sl) {
            sl->ok = launch_batch(S, *sl, bjobs, breqs);
            launched = true;
        }
        lk.lock();
        bool upload_failed = false;
        for (size_t k = 0; k < admit.size(); ++k) {
            Job *j = admit[k];
            j->uploading = false;
            if (uploaded[k]) {
                j->admitted = true;
                std::vector<double>().swap(j->x);
                std::vector<double>().swap(j->y);
                std::vector<double>().swap(j->obs);
                std::vector<int>().swap(j->knn);
            } else {
                // No room on the device after all: back to the head of the queue.
                S->bytes_in_use -= j->footprint;
                S->admit_queue.push_front(j->id);
                upload_failed = true;
            }
        }
        if (launched) {
            sl->launched = true;
            sl->cv.notify_all();
        }
        if (!admit.empty()) S->cv_done.notify_all();
        // After a failed upload, retry admission after a pause, not in a spin.
        if (upload_failed) S->cv_work.wait_for(lk, std::chrono::milliseconds(20));
    }
}

void completer_main(bv_server *S, bv_server::Slot *sl)
{
    cudaSetDevice(S->opts.device);
    std::unique_lock<std::mutex> lk(S->mu);
    for (;;) {
        sl->cv.wait(lk, [&] { return sl->launched || S->stop; });
        if (!sl->launched) break;
        lk.unlock();
        const cudaError_t e = cudaStreamSynchronize(sl->s);
        lk.lock();
        const bool ok = sl->ok && e == cudaSuccess;
        if (e != cudaSuccess) sl->err = cudaGetErrorString(e);
        const auto now = Clock::now();
        for (size_t r = 0; r < sl->batch.size(); ++r) {
            Req &rq = S->reqs[sl->batch[r]];
            rq.done = true;
            rq.latency_ms = std::chrono::duration<double, std::milli>(now - rq.submitted).count();
            if (!ok) {
                rq.rc = BV_E_CUDA;
                rq.llk = -HUGE_VAL;
            } else {
                const EvalResult &res = sl->h_res[r];
                const bool failed = (res.cond_fail + res.schur_fail + res.nonfinite) > 0 ||
                                    !std::isfinite(res.llk);
                rq.llk = (failed && S->opts.on_failure == BV_FAIL_NEGINF) ? -HUGE_VAL : res.llk;
            }
            auto jt = S->jobs.find(rq.job);
            if (jt != S->jobs.end()) jt->second->inflight--;
            S->latencies.push_back(rq.latency_ms);
            S->evals++;
        }
        S->batches++;
        S->batch_requests += sl->batch.size();
        sl->batch.clear();
        sl->launched = false;
        sl->busy = false;
        S->cv_work.notify_all();
        S->cv_done.notify_all();
    }
}

void destroy_slot(bv_server::Slot &sl)
{
    if (sl.s) cudaStreamSynchronize(sl.s);
    cudaFree(sl.bllk);
    cudaFree(sl.bst);
    cudaFree(sl.tasks);
    cudaFree(sl.desc);
    cudaFree(sl.res);
    cudaFree(sl.counters);
    cudaFree(sl.slab);
    cudaFree(sl.lean_slab);
    cudaFreeHost(sl.h_tasks);
    cudaFreeHost(sl.h_desc);
    cudaFreeHost(sl.h_res);
    if (sl.s) cudaStreamDestroy(sl.s);
}

}  // namespace

extern "C" void bv_server_default_opts(bv_server_opts *o)
{
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->device = 0;
    o->hbm_budget = 0;  // 0: 90% of the device memory free at creation
    o->max_batch = 256;
    o->on_failure = BV_FAIL_NEGINF;
    o->max_inflight = 2;
}

extern "C" int bv_server_create(const bv_server_opts *opts, bv_server **out)
{
    if (!out) return BV_E_INVALID;
    *out = nullptr;
    std::unique_ptr<bv_server> S(new bv_server());
    if (opts)
        S->opts = *opts;
    else
        bv_server_default_opts(&S->opts);
    if (S->opts.max_batch <= 0) S->opts.max_batch = 256;
    if (S->opts.max_inflight <= 0) S->opts.max_inflight = 2;
    if (S->opts.max_inflight > 8) S->opts.max_inflight = 8;
    BV_CUDA_TRY(cudaSetDevice(S->opts.device));
    cudaDeviceProp prop;
    BV_CUDA_TRY(cudaGetDeviceProperties(&prop, S->opts.device));
    if (prop.major < 10) {
        set_error("bv_server_create: device is sm_%d%d; built for sm_100a", prop.major, prop.minor);
        return BV_E_NODEVICE;
    }
    if (S->opts.hbm_budget == 0) {
        size_t fr = 0, tot = 0;
        BV_CUDA_TRY(cudaMemGetInfo(&fr, &tot));
        S->opts.hbm_budget = fr / 10 * 9;
    }
    // The same shared-memory limits as the handles, so a block takes the same
    // path (and gives the same bits) here and under bv_llh_eval.
    {
        const int rc = fp64_limits(S->opts.device, nullptr, &S->smem_cap_m, &S->big_max_m);
        if (rc) return rc;
    }
    int optin = 0;
    BV_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, S->opts.device));
    cudaFuncAttributes fa, fb;
    BV_CUDA_TRY(cudaFuncGetAttributes(&fa, llh_fp64_server_kernel<false>));
    BV_CUDA_TRY(cudaFuncGetAttributes(&fb, llh_fp64_server_kernel<true>));
    const size_t stat = std::max(fa.sharedSizeBytes, fb.sharedSizeBytes);
    const size_t need = std::max<size_t>(std::max(block_doubles(S->smem_cap_m) * sizeof(double),
                                                  (size_t)big_layout(S->big_max_m).total),
                                         kReduceScratchBytes);
    if (need + stat > (size_t)optin) {
        set_error("bv_server_create: %zu B of dynamic shared memory does not fit next to %zu B static",
                  need, stat);
        return BV_E_TOOLARGE;
    }
    S->smem_bytes = need;
    BV_CUDA_TRY(cudaFuncSetAttribute(llh_fp64_server_kernel<false>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S->smem_bytes));
    BV_CUDA_TRY(cudaFuncSetAttribute(llh_fp64_server_kernel<true>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S->smem_bytes));
    int occ = 0;
    BV_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, llh_fp64_server_kernel<true>, kThreads,
                                                              S->smem_bytes));
    S->grid = prop.multiProcessorCount * std::max(1, occ);
    S->sms = prop.multiProcessorCount;
    // The streamed kernel: the handles' limit, and its shared memory allowed.
    {
        cudaFuncAttributes fl;
        BV_CUDA_TRY(cudaFuncGetAttributes(&fl, kLeanServer[2].kernel));
        const size_t avail = (size_t)optin - fl.sharedSizeBytes;
        S->lean_limit = big_max_m_for_bytes(avail, 64, 0, 0);
        for (const LeanServerVariant &v : kLeanServer)
            BV_CUDA_TRY(cudaFuncSetAttribute(v.kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)avail));
    }
    BV_CUDA_TRY(cudaStreamCreateWithFlags(&S->upload, cudaStreamNonBlocking));
    for (int k = 0; k < S->opts.max_inflight; ++k) {
        std::unique_ptr<bv_server::Slot> sl(new bv_server::Slot());
        sl->index = k;
        const int R = S->opts.max_batch;
        BV_CUDA_TRY(cudaStreamCreateWithFlags(&sl->s, cudaStreamNonBlocking));
        BV_CUDA_TRY(cudaMalloc(&sl->desc, R * sizeof(JobDesc)));
        BV_CUDA_TRY(cudaMalloc(&sl->res, R * sizeof(EvalResult)));
        BV_CUDA_TRY(cudaMalloc(&sl->counters, (2 + R) * sizeof(unsigned)));
        BV_CUDA_TRY(cudaHostAlloc(&sl->h_desc, R * sizeof(JobDesc), cudaHostAllocDefault));
        BV_CUDA_TRY(cudaHostAlloc(&sl->h_res, R * sizeof(EvalResult), cudaHostAllocDefault));
        // Streamed-kernel slabs for blocks up to M = 350 (cs = 300 with
        // blocks of 50) at every table point, so that batches of such jobs
        // allocate nothing; larger batches grow them.
        size_t pre = 0;
        for (int m : {170, 250, std::min(350, S->lean_limit)}) {
            LeanLaunch ll;
            if (lean_launch_for(S.get(), m, ll)) pre = std::max(pre, ll.stride * 8 * (size_t)ll.grid);
        }
        if (pre > 0) {
            BV_CUDA_TRY(cudaMalloc(&sl->lean_slab, pre));
            sl->lean_bytes = pre;
        }
        S->slots.push_back(std::move(sl));
    }
    bv_server *raw = S.release();
    for (auto &sl : raw->slots) sl->completer = std::thread(completer_main, raw, sl.get());
    raw->scheduler = std::thread(scheduler_main, raw);
    *out = raw;
    return BV_OK;
}

extern "C" void bv_server_destroy(bv_server *S)
{
    if (!S) return;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
    }
    S->cv_work.notify_all();
    if (S->scheduler.joinable()) S->scheduler.join();
    // Completers finish the batches in flight, then exit.
    for (auto &sl : S->slots) {
        {
            std::lock_guard<std::mutex> lk(S->mu);
            sl->cv.notify_all();
        }
        if (sl->completer.joinable()) sl->completer.join();
    }
    cudaSetDevice(S->opts.device);
    for (auto &sl : S->slots) destroy_slot(*sl);
    for (auto &kv : S->jobs)
        if (kv.second->admitted) free_job_device(*kv.second, S->upload);
    if (S->upload) {
        cudaStreamSynchronize(S->upload);
        cudaStreamDestroy(S->upload);
    }
    delete S;
}

extern "C" int bv_server_open_job(bv_server *S, const bv_layout *L, double dist_scale, int *job_id)
{
    bv_job_opts o;
    o.dist_scale = dist_scale;
    o.nugget = 0;
    return bv_server_open_job_ex(S, L, &o, job_id);
}

extern "C" int bv_server_open_job_ex(bv_server *S, const bv_layout *L, const bv_job_opts *jo,
                                     int *job_id)
{
    if (!S || !job_id || !jo) {
        set_error("bv_server_open_job: null argument");
        return BV_E_INVALID;
    }
    const int vr = validate_layout(L);
    if (vr != BV_OK) return vr;
    if (L->z) {
        set_error("bv_server_open_job: the server evaluates 2-D Matern layouts (no third coordinate)");
        return BV_E_INVALID;
    }
    if (L->cs > 0 && !L->knn_idx) {
        set_error("bv_server_open_job: the layout's conditioning indices (knn_idx) are required");
        return BV_E_INVALID;
    }
    std::unique_ptr<Job> j(new Job());
    j->n = L->n;
    j->bc = L->bc;
    j->cs = L->cs;
    j->dist_scale = jo->dist_scale > 0 ? jo->dist_scale : 1.0;
    j->nugget = jo->nugget != 0;
    j->acc.assign(L->batchNumAccum, L->batchNumAccum + L->bc + 1);
    std::vector<int> m(L->bc);
    for (int b = 0; b < L->bc; ++b) {
        m[b] = j->acc[b + 1] - j->acc[b] + (b == 0 ? 0 : L->cs);
        j->max_m = std::max(j->max_m, m[b]);
    }
    j->sorted.resize(L->bc);
    for (int b = 0; b < L->bc; ++b) j->sorted[b] = b;
    std::stable_sort(j->sorted.begin(), j->sorted.end(), [&](int a, int b) { return m[a] > m[b]; });
    for (int p = 0; p < L->bc; ++p)
        if (p == 0 || m[j->sorted[p]] != m[j->sorted[p - 1]]) {
            j->m_start.push_back(p);
            j->m_value.push_back(m[j->sorted[p]]);
        }
    if (L->cs > 0) j->knn.assign(L->knn_idx, L->knn_idx + (size_t)L->bc * L->cs);
    j->x.assign(L->x, L->x + L->n);
    j->y.assign(L->y, L->y + L->n);
    j->obs.assign(L->obs, L->obs + L->n);
    {
        int sms = 0;
        BV_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, S->opts.device));
        j->big = use_big_path(L->batchNum, L->bc, L->cs, S->smem_cap_m, S->big_max_m, sms);
    }
    j->footprint = job_footprint(*j);
    if (j->footprint > S->opts.hbm_budget) {
        set_error("bv_server_open_job: job needs %zu bytes, more than the budget %zu", j->footprint,
                  S->opts.hbm_budget);
        return BV_E_TOOLARGE;
    }
    std::lock_guard<std::mutex> lk(S->mu);
    j->id = S->next_job++;
    *job_id = j->id;
    S->admit_queue.push_back(j->id);
    S->jobs[j->id] = std::move(j);
    S->cv_work.notify_all();
    return BV_OK;
}

extern "C" int bv_server_close_job(bv_server *S, int job_id)
{
    if (!S) return BV_E_INVALID;
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->jobs.find(job_id);
    if (it == S->jobs.end() || it->second->closing) {
        set_error("bv_server_close_job: no open job %d", job_id);
        return BV_E_INVALID;
    }
    it->second->closing = true;
    S->cv_work.notify_all();
    return BV_OK;
}

extern "C" int bv_server_job_admitted(bv_server *S, int job_id, int *admitted)
{
    if (!S || !admitted) return BV_E_INVALID;
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->jobs.find(job_id);
    if (it == S->jobs.end()) {
        set_error("bv_server_job_admitted: no job %d", job_id);
        return BV_E_INVALID;
    }
    *admitted = it->second->admitted ? 1 : 0;
    return BV_OK;
}

extern "C" int bv_server_submit(bv_server *S, int job_id, const double *theta, long long *req_id)
{
    if (!S || !theta || !req_id) return BV_E_INVALID;
    if (!std::isfinite(theta[0]) || !(theta[1] > 0) || !(theta[2] > 0) || !std::isfinite(theta[1]) ||
        !std::isfinite(theta[2])) {
        set_error("bv_server_submit: invalid theta (%g, %g, %g)", theta[0], theta[1], theta[2]);
        return BV_E_INVALID;
    }
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->jobs.find(job_id);
    if (it == S->jobs.end() || it->second->closing) {
        set_error("bv_server_submit: no open job %d", job_id);
        return BV_E_INVALID;
    }
    const bool nug = it->second->nugget;
    if (nug && (!(theta[3] >= 0) || !std::isfinite(theta[3]))) {
        set_error("bv_server_submit: invalid nugget %g", theta[3]);
        return BV_E_INVALID;
    }
    Req r;
    r.id = S->next_req++;
    r.job = job_id;
    std::memcpy(r.theta, theta, (nug ? 4 : 3) * sizeof(double));
    r.submitted = Clock::now();
    it->second->inflight++;
    S->reqs[r.id] = r;
    S->pending.push_back(r.id);
    *req_id = r.id;
    S->cv_work.notify_all();
    return BV_OK;
}

extern "C" int bv_server_wait(bv_server *S, long long req_id, double *llk, double *latency_ms,
                              int timeout_ms)
{
    if (!S || !llk) return BV_E_INVALID;
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->reqs.find(req_id);
    if (it == S->reqs.end()) {
        set_error("bv_server_wait: unknown request %lld", req_id);
        return BV_E_INVALID;
    }
    auto ready = [&] { return S->reqs[req_id].done; };
    if (timeout_ms < 0) {
        S->cv_done.wait(lk, ready);
    } else if (!S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) {
        set_error("bv_server_wait: request %lld not complete after %d ms", req_id, timeout_ms);
        return BV_E_TIMEOUT;
    }
    const Req r = S->reqs[req_id];
    S->reqs.erase(req_id);
    *llk = r.llk;
    if (latency_ms) *latency_ms = r.latency_ms;
    if (r.rc != BV_OK) set_error("bv_server: evaluation %lld failed on the device", req_id);
    return r.rc;
}

extern "C" int bv_server_get_stats(bv_server *S, bv_server_stats *st)
{
    if (!S || !st) return BV_E_INVALID;
    std::lock_guard<std::mutex> lk(S->mu);
    std::memset(st, 0, sizeof(*st));
    st->evals = S->evals;
    st->batches = S->batches;
    st->mean_batch = S->batches ? (double)S->batch_requests / S->batches : 0.0;
    st->bytes_in_use = S->bytes_in_use;
    st->hbm_budget = S->opts.hbm_budget;
    int adm = 0, waiting = 0;
    for (auto &kv : S->jobs) (kv.second->admitted ? adm : waiting)++;
    st->jobs_admitted = adm;
    st->jobs_waiting = waiting;
    std::vector<double> l = S->latencies;
    if (!l.empty()) {
        std::sort(l.begin(), l.end());
        auto q = [&](double p) { return l[std::min(l.size() - 1, (size_t)(p * (l.size() - 1) + 0.5))]; };
        st->p50_ms = q(0.50);
        st->p99_ms = q(0.99);
        st->max_ms = l.back();
    }
    return BV_OK;
}

extern "C" int bv_server_reset_stats(bv_server *S)
{
    if (!S) return BV_E_INVALID;
    std::lock_guard<std::mutex> lk(S->mu);
    S->evals = S->batches = S->batch_requests = 0;
    S->latencies.clear();
    return BV_OK;
}

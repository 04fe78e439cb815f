// bv_knn.cu -- conditioning-set selection on the device, one warp per block.
//
// Follows findNearestPoints (include/nearest_neighbor.h:76-148) as the
// reference's driver calls it for blocks 1..bc-1 with l0 = 0 and
// l1 = batchNumAccum[i] (src/test_Xvecchia_batch.cpp:368-390):
//   key(p) = sqrt(fma(dx, dx, dy*dy)), dx = x[p] - cx, dy = y[p] - cy
//   (calEucDistance :30-35 as the reference's -O3 -march=native build
//   contracts it), then k = cs rounds of a selection sort with swaps and a
//   strict '<' (:115-133), output in selection order.  With a third
//   coordinate (the reference's time_flag, :101-104) the key is
//   sqrt(fma(d, d, dz*dz)), d the 2-D key and dz = cz - z[p], as contracted.
// Both keys are the square root of a "pre-key" computed exactly as the
// reference computes the root's argument; the selection works on pre-keys.
//
// The warp streams the candidates once, keeping those whose squared distance
// is within a few ulps of the running k-th smallest (a threshold that only
// falls) in a shared-memory buffer, and shrinks the buffer by an exact radix
// select whenever it fills.  The final set S = {p : key(p) <= key_k} (all
// ties of the k-th key included) is then put through an exact replay of the
// reference's selection sort: at step t the winner is the unselected member
// of S with the smallest (key, current position), it moves to position t and
// whatever S member occupied position t moves to the winner's old position.
// Members outside S never win and never change the relative positions of S
// members, so the replay reproduces the reference's output, ties included.
// A block whose ties at the k-th key overflow the warp's buffer (hundreds of
// exactly repeated locations at one distance) is listed and redone by
// knn_heavy_kernel: one CTA, keys recomputed on every pass instead of
// buffered, S in a global scratch array, the same replay.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <vector>

#include "../../include/bv.h"
#include "bv_common.cuh"
#include "bv_knn.cuh"

namespace bv {

constexpr int kKnnWarps = 4;
constexpr int kKnnCap = 1024;  // candidate buffer per warp
constexpr int kKnnMaxCs = kKnnCap / 2;

struct KnnWarpSmem {
    unsigned long long key[kKnnCap];  // squared distance bits, later distance bits
    int idx[kKnnCap];
    int pos[kKnnCap];
    unsigned hist[256];
};

struct KnnArgs {
    const double *x, *y;
    const double *z;        // third coordinate, or nullptr (2-D)
    const int *acc;
    const double *cx, *cy;  // device copies
    const double *cz;       // device copy, when z is set
    int bc, cs;
    int *out;
    unsigned *counter;
    int *error;  // first failing block + 1, or 0
    int *heavy;  // blocks whose ties overflow the buffer, for knn_heavy_kernel
    unsigned *heavy_count;
    const int *list;  // blocks to select for (largest prefix first), or nullptr: all
    int nlist;
};

// Key geometries, each a separate instantiation: plane (2-D), 3-D (the
// time_flag key), and the great-circle key of distance_metric = 1 (--earth,
// include/nearest_neighbor.h:93-96: distanceEarth(centroid, point); z and cz
// then carry cos(latitude) of the points and centroids, from the host).
enum KnnGeo : int { kGeoPlane = 0, kGeo3D = 1, kGeoEarth = 2 };

// The argument of the key's final square root for candidate p.
template <int kGeo>
__device__ __forceinline__ double knn_prekey(const KnnArgs &a, int p, double cx, double cy, double cz)
{
    if constexpr (kGeo == kGeoEarth) {
        // distanceEarth up to its square root: lat1 = centroid, lat2 = point.
        const double pi = 3.141592653589793;
        const double lat1r = __ddiv_rn(__dmul_rn(cx, pi), 180.0);
        const double lon1r = __ddiv_rn(__dmul_rn(cy, pi), 180.0);
        const double lat2r = __ddiv_rn(__dmul_rn(__ldg(a.x + p), pi), 180.0);
        const double lon2r = __ddiv_rn(__dmul_rn(__ldg(a.y + p), pi), 180.0);
        const double u = sin(__dmul_rn(__dsub_rn(lat2r, lat1r), 0.5));
        const double v = sin(__dmul_rn(__dsub_rn(lon2r, lon1r), 0.5));
        return __fma_rn(u, u, __dmul_rn(__dmul_rn(__dmul_rn(cz, __ldg(a.z + p)), v), v));
    }
    const double dx = __ldg(a.x + p) - cx;
    const double dy = __ldg(a.y + p) - cy;
    const double s = __fma_rn(dx, dx, __dmul_rn(dy, dy));
    if constexpr (kGeo == kGeoPlane) return s;
    const double d = __dsqrt_rn(s);
    const double dz = cz - __ldg(a.z + p);
    return __fma_rn(d, d, __dmul_rn(dz, dz));
}

// The key (a distance) from its pre-key.
template <int kGeo>
__device__ __forceinline__ double knn_dist(double s)
{
    if constexpr (kGeo == kGeoEarth) return __dmul_rn(12742.0, asin(__dsqrt_rn(s)));
    return __dsqrt_rn(s);
}

__device__ __forceinline__ unsigned lanemask_lt()
{
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Exact k-th smallest (1-based) of the first n keys, MSB-first radix select
// with 8-bit digits.
__device__ unsigned long long warp_kth(KnnWarpSmem &w, int n, int k)
{
    const int lane = threadIdx.x & 31;
    unsigned long long prefix = 0ull, mask = 0ull;
    int kk = k;
    for (int shift = 56; shift >= 0; shift -= 8) {
#pragma unroll
        for (int b = 0; b < 8; ++b) w.hist[lane * 8 + b] = 0u;
        __syncwarp();
        for (int j = lane; j < n; j += 32) {
            const unsigned long long key = w.key[j];
            if ((key & mask) == prefix) atomicAdd(&w.hist[(key >> shift) & 255ull], 1u);
        }
        __syncwarp();
        unsigned loc[8];
        unsigned tot = 0;
#pragma unroll
        for (int b = 0; b < 8; ++b) {
            loc[b] = w.hist[lane * 8 + b];
            tot += loc[b];
        }
        unsigned incl = tot;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        const unsigned excl = incl - tot;
        // The lane whose bin range holds the kk-th element.
        const bool mine = (excl < (unsigned)kk) && ((unsigned)kk <= incl);
        const unsigned who = __ballot_sync(0xffffffffu, mine);
        const int src = who ? __ffs(who) - 1 : 31;  // who != 0 whenever n >= k
        int bin = 0, before = 0;
        if (lane == src) {
            unsigned run = excl;
#pragma unroll
            for (int b = 0; b < 8; ++b) {
                if (run + loc[b] >= (unsigned)kk) {
                    bin = lane * 8 + b;
                    before = (int)run;
                    break;
                }
                run += loc[b];
            }
        }
        bin = __shfl_sync(0xffffffffu, bin, src);
        before = __shfl_sync(0xffffffffu, before, src);
        prefix |= (unsigned long long)bin << shift;
        mask |= 255ull << shift;
        kk -= before;
        __syncwarp();
    }
    return prefix;
}

// Keep entries with key <= lim, in order; returns the new count.
__device__ int warp_compact(KnnWarpSmem &w, int n, unsigned long long lim)
{
    const int lane = threadIdx.x & 31;
    int count = 0;
    for (int base = 0; base < n; base += 32) {
        const int j = base + lane;
        unsigned long long key = 0ull;
        int id = 0;
        bool keep = false;
        if (j < n) {
            key = w.key[j];
            id = w.idx[j];
            keep = key <= lim;
        }
        const unsigned bal = __ballot_sync(0xffffffffu, keep);
        __syncwarp();
        if (keep) {
            const int p = count + __popc(bal & lanemask_lt());
            w.key[p] = key;
            w.idx[p] = id;
        }
        count += __popc(bal);
        __syncwarp();
    }
    return count;
}

// Upper end of the pre-key window whose keys can equal key(s): sqrt halves
// relative spacing, so 2^-49 relative is ample; the great-circle key adds
// asin's few-ulp error and its scaling, covered by 2^-40.
template <int kGeo>
__device__ __forceinline__ unsigned long long window_hi(unsigned long long skey)
{
    const double s = __longlong_as_double((long long)skey);
    const double hi = s * (1.0 + (kGeo == kGeoEarth ? 0x1p-40 : 0x1p-49)) + 0x1p-1070;
    return (unsigned long long)__double_as_longlong(hi);
}

template <int kGeo>
__global__ void __launch_bounds__(kKnnWarps * 32) knn_kernel(KnnArgs a)
{
    extern __shared__ __align__(16) unsigned char knn_smem[];
    KnnWarpSmem &w = reinterpret_cast<KnnWarpSmem *>(knn_smem)[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const int k = a.cs;

    for (;;) {
        unsigned task = 0;
        if (lane == 0) task = atomicAdd(a.counter, 1u);
        task = __shfl_sync(0xffffffffu, task, 0);
        // Largest prefixes first; block 0 is handled by the host (points 0..cs-1).
        int i;
        if (a.list) {
            if ((int)task >= a.nlist) break;
            i = a.list[task];
        } else {
            i = a.bc - 1 - (int)task;
            if (i < 1) break;
        }
        const int P = a.acc[i];
        const double cx = a.cx[i], cy = a.cy[i], cz = (kGeo != kGeoPlane) ? a.cz[i] : 0.0;
        int *out = a.out + (size_t)i * k;
        if (P < k) {
            if (lane == 0) atomicCAS(a.error, 0, i + 1);
            continue;
        }

        // 1. Stream candidates 0..P-1 through the falling threshold.
        unsigned long long lim = ~0ull;
        int count = 0;
        bool overflow = false;
        for (int base = 0; base < P; base += 128) {
            unsigned long long key[4];
            bool keep[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int p = base + 32 * u + lane;
                keep[u] = false;
                key[u] = 0ull;
                if (p < P) {
                    const double s = knn_prekey<kGeo>(a, p, cx, cy, cz);
                    key[u] = (unsigned long long)__double_as_longlong(s);
                    keep[u] = key[u] <= lim;
                }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const unsigned bal = __ballot_sync(0xffffffffu, keep[u]);
                if (keep[u]) {
                    const int p = count + __popc(bal & lanemask_lt());
                    w.key[p] = key[u];
                    w.idx[p] = base + 32 * u + lane;
                }
                count += __popc(bal);
            }
            if (count > kKnnCap - 128) {
                __syncwarp();
                const unsigned long long kth = warp_kth(w, count, k);
                lim = window_hi<kGeo>(kth);
                count = warp_compact(w, count, lim);
                if (count > kKnnCap - 128) {
                    overflow = true;
                    break;
                }
            }
        }
        if (overflow) {
            if (lane == 0) a.heavy[atomicAdd(a.heavy_count, 1u)] = i;
            continue;
        }
        __syncwarp();

        // 2. Exact k-th key; S = members whose distance equals or beats it.
        const unsigned long long kth = warp_kth(w, count, k);
        count = warp_compact(w, count, window_hi<kGeo>(kth));
        double dk = knn_dist<kGeo>(__longlong_as_double((long long)kth));
        if constexpr (kGeo == kGeoEarth) {
            // The great-circle key need not be monotone in its pre-key to the
            // last bit (device asin): the k-th smallest key itself, over the
            // window's members (all keys are non-negative, so their bit
            // patterns order as the values do).
            for (int j = lane; j < count; j += 32)
                w.key[j] = (unsigned long long)__double_as_longlong(
                    knn_dist<kGeo>(__longlong_as_double((long long)w.key[j])));
            __syncwarp();
            dk = __longlong_as_double((long long)warp_kth(w, count, k));
        }
        {
            int m = 0;
            for (int base = 0; base < count; base += 32) {
                const int j = base + lane;
                double d = 0.0;
                int id = 0;
                bool keep = false;
                if (j < count) {
                    const double kj = __longlong_as_double((long long)w.key[j]);
                    d = (kGeo == kGeoEarth) ? kj : knn_dist<kGeo>(kj);  // earth: already keys
                    id = w.idx[j];
                    keep = d <= dk;
                }
                const unsigned bal = __ballot_sync(0xffffffffu, keep);
                __syncwarp();
                if (keep) {
                    const int p = m + __popc(bal & lanemask_lt());
                    w.key[p] = (unsigned long long)__double_as_longlong(d);
                    w.idx[p] = id;
                    w.pos[p] = id;  // initial position = index
                }
                m += __popc(bal);
                __syncwarp();
            }
            count = m;
        }

        // 3. Replay the selection sort on S.
        for (int t = 0; t < k; ++t) {
            unsigned long long bkey = ~0ull;
            int bpos = 0x7fffffff, bslot = -1, occ = -1;
            for (int j = lane; j < count; j += 32) {
                const int pj = w.pos[j];
                if (pj < 0) continue;  // already selected
                const unsigned long long kj = w.key[j];
                if (kj < bkey || (kj == bkey && pj < bpos)) {
                    bkey = kj;
                    bpos = pj;
                    bslot = j;
                }
                if (pj == t) occ = j;
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const unsigned long long ok = __shfl_xor_sync(0xffffffffu, bkey, o);
                const int op = __shfl_xor_sync(0xffffffffu, bpos, o);
                const int os = __shfl_xor_sync(0xffffffffu, bslot, o);
                if (ok < bkey || (ok == bkey && op < bpos)) {
                    bkey = ok;
                    bpos = op;
                    bslot = os;
                }
            }
            const unsigned ob = __ballot_sync(0xffffffffu, occ >= 0);
            const int occ_slot = ob ? __shfl_sync(0xffffffffu, occ, __ffs(ob) - 1) : -1;
            if (bslot < 0) break;  // |S| >= k makes this unreachable
            if (lane == 0) {
                out[t] = w.idx[bslot];
                if (occ_slot >= 0 && occ_slot != bslot) w.pos[occ_slot] = bpos;
                w.pos[bslot] = -1;
            }
            __syncwarp();
        }
    }
}


// Blocks listed by knn_kernel, dealt round-robin to the CTAs.  Each CTA has
// n entries of scratch for S (distance bits, index, current position) of the
// block it works on (S is a subset of the block's candidates, so n suffice).
constexpr int kHeavyThreads = 1024;

struct KnnHeavyScratch {
    unsigned long long *key;
    int *idx;
    int *pos;
};

template <int kGeo>
__device__ __forceinline__ unsigned long long knn_skey(const KnnArgs &a, int p, double cx, double cy,
                                                       double cz)
{
    return (unsigned long long)__double_as_longlong(knn_prekey<kGeo>(a, p, cx, cy, cz));
}

template <int kGeo>
__global__ void __launch_bounds__(kHeavyThreads) knn_heavy_kernel(KnnArgs a, int nheavy, KnnHeavyScratch scr,
                                                                  size_t stride)
{
    KnnHeavyScratch sc{scr.key + blockIdx.x * stride, scr.idx + blockIdx.x * stride,
                       scr.pos + blockIdx.x * stride};
    __shared__ unsigned hist[256];
    __shared__ unsigned long long s_prefix;
    __shared__ int s_kk, s_count, s_occ;
    __shared__ unsigned long long w_key[kHeavyThreads / 32];
    __shared__ int w_pos[kHeavyThreads / 32], w_slot[kHeavyThreads / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int k = a.cs;
    for (int h = blockIdx.x; h < nheavy; h += gridDim.x) {
        const int i = a.heavy[h];
        const int P = a.acc[i];
        const double cx = a.cx[i], cy = a.cy[i], cz = (kGeo != kGeoPlane) ? a.cz[i] : 0.0;
        int *out = a.out + (size_t)i * k;
        // 1. Exact k-th smallest squared distance, MSB-first radix select.
        if (tid == 0) {
            s_prefix = 0ull;
            s_kk = k;
        }
        unsigned long long mask = 0ull;
        for (int shift = 56; shift >= 0; shift -= 8) {
            if (tid < 256) hist[tid] = 0u;
            __syncthreads();
            const unsigned long long prefix = s_prefix;
            for (int p = tid; p < P; p += kHeavyThreads) {
                const unsigned long long key = knn_skey<kGeo>(a, p, cx, cy, cz);
                if ((key & mask) == prefix) atomicAdd(&hist[(key >> shift) & 255ull], 1u);
            }
            __syncthreads();
            if (tid == 0) {
                unsigned run = 0;
                int bin = 255;
                for (int b = 0; b < 256; ++b) {
                    if (run + hist[b] >= (unsigned)s_kk) {
                        bin = b;
                        break;
                    }
                    run += hist[b];
                }
                s_prefix = prefix | ((unsigned long long)bin << shift);
                s_kk -= (int)run;
            }
            mask |= 255ull << shift;
            __syncthreads();
        }
        const unsigned long long kth = s_prefix;
        // 2. S = candidates whose distance equals or beats the k-th.
        const unsigned long long hi = window_hi<kGeo>(kth);
        const double dk = knn_dist<kGeo>(__longlong_as_double((long long)kth));
        if (tid == 0) s_count = 0;
        __syncthreads();
        for (int p = tid; p < P; p += kHeavyThreads) {
            const unsigned long long key = knn_skey<kGeo>(a, p, cx, cy, cz);
            if (key <= hi) {
                const double d = knn_dist<kGeo>(__longlong_as_double((long long)key));
                if (d <= dk) {
                    const int slot = atomicAdd(&s_count, 1);
                    sc.key[slot] = (unsigned long long)__double_as_longlong(d);
                    sc.idx[slot] = p;
                    sc.pos[slot] = p;  // initial position = index
                }
            }
        }
        __syncthreads();
        const int count = s_count;
        // 3. Replay the selection sort on S.
        for (int t = 0; t < k; ++t) {
            unsigned long long bkey = ~0ull;
            int bpos = 0x7fffffff, bslot = -1;
            if (tid == 0) s_occ = -1;
            __syncthreads();
            for (int j = tid; j < count; j += kHeavyThreads) {
                const int pj = sc.pos[j];
                if (pj < 0) continue;  // already selected
                const unsigned long long kj = sc.key[j];
                if (kj < bkey || (kj == bkey && pj < bpos)) {
                    bkey = kj;
                    bpos = pj;
                    bslot = j;
                }
                if (pj == t) s_occ = j;  // positions are distinct: one writer
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const unsigned long long ok = __shfl_xor_sync(0xffffffffu, bkey, o);
                const int op = __shfl_xor_sync(0xffffffffu, bpos, o);
                const int os = __shfl_xor_sync(0xffffffffu, bslot, o);
                if (ok < bkey || (ok == bkey && op < bpos)) {
                    bkey = ok;
                    bpos = op;
                    bslot = os;
                }
            }
            if (lane == 0) {
                w_key[warp] = bkey;
                w_pos[warp] = bpos;
                w_slot[warp] = bslot;
            }
            __syncthreads();
            if (tid == 0) {
                for (int w = 1; w < kHeavyThreads / 32; ++w) {
                    if (w_key[w] < bkey || (w_key[w] == bkey && w_pos[w] < bpos)) {
                        bkey = w_key[w];
                        bpos = w_pos[w];
                        bslot = w_slot[w];
                    }
                }
                if (bslot >= 0) {  // |S| >= k makes bslot >= 0
                    out[t] = sc.idx[bslot];
                    if (s_occ >= 0 && s_occ != bslot) sc.pos[s_occ] = bpos;
                    sc.pos[bslot] = -1;
                }
            }
            __syncthreads();
        }
    }
}

int knn_device(const double *d_x, const double *d_y, const double *d_z, int n, int bc, int cs,
               const int *d_acc, const double *cx, const double *cy, const double *cz, int *d_knn,
               cudaStream_t s, const unsigned char *mask, int earth)
{
    if (d_z && !cz) {
        set_error("bv_knn: 3-D locations need the centroids' third coordinate");
        return BV_E_INVALID;
    }
    if (earth && !d_z) {
        set_error("bv_knn: the great-circle key needs cos(latitude) of points and centroids");
        return BV_E_INVALID;
    }
    const int geo = earth ? kGeoEarth : (d_z ? kGeo3D : kGeoPlane);
    void (*const kern)(KnnArgs) = geo == kGeoEarth ? knn_kernel<kGeoEarth>
                                                   : (geo == kGeo3D ? knn_kernel<kGeo3D> : knn_kernel<kGeoPlane>);
    void (*const heavy)(KnnArgs, int, KnnHeavyScratch, size_t) =
        geo == kGeoEarth ? knn_heavy_kernel<kGeoEarth>
                         : (geo == kGeo3D ? knn_heavy_kernel<kGeo3D> : knn_heavy_kernel<kGeoPlane>);
    if (cs <= 0) return BV_OK;
    if (cs > kKnnMaxCs) {
        set_error("bv_knn: cs=%d exceeds the supported maximum %d", cs, kKnnMaxCs);
        return BV_E_TOOLARGE;
    }
    std::vector<int> first(cs);
    for (int t = 0; t < cs; ++t) first[t] = t;
    double *d_c = nullptr;
    unsigned *d_counter = nullptr;
    int *d_err = nullptr;
    int rc = BV_OK;
    auto fail = [&](cudaError_t e, const char *what) {
        set_error("bv_knn: %s: %s", what, cudaGetErrorString(e));
        rc = BV_E_CUDA;
    };
    cudaError_t e;
    if ((e = cudaMalloc(&d_c, sizeof(double) * 3 * (size_t)bc)) != cudaSuccess) {
        fail(e, "cudaMalloc");
        return rc;
    }
    // Blocks 1..bc-1 to select for, largest prefix first (all, or the mask's).
    std::vector<int> list;
    if (mask) {
        for (int b = bc - 1; b >= 1; --b)
            if (mask[b]) list.push_back(b);
    }
    // counter, error, heavy_count, the heavy list (bc entries), the block list
    if ((e = cudaMalloc(&d_counter, sizeof(unsigned) * 3 + sizeof(int) * (size_t)bc * 2)) != cudaSuccess) {
        cudaFree(d_c);
        fail(e, "cudaMalloc");
        return rc;
    }
    d_err = reinterpret_cast<int *>(d_counter + 1);
    unsigned *d_heavy_count = d_counter + 2;
    int *d_heavy = reinterpret_cast<int *>(d_counter + 3);
    int *d_list = d_heavy + bc;
    KnnHeavyScratch sc{nullptr, nullptr, nullptr};
    do {
        if ((e = cudaMemcpyAsync(d_c, cx, sizeof(double) * bc, cudaMemcpyHostToDevice, s)) ||
            (e = cudaMemcpyAsync(d_c + bc, cy, sizeof(double) * bc, cudaMemcpyHostToDevice, s)) ||
            (d_z && (e = cudaMemcpyAsync(d_c + 2 * (size_t)bc, cz, sizeof(double) * bc,
                                         cudaMemcpyHostToDevice, s))) ||
            (e = cudaMemcpyAsync(d_knn, first.data(), sizeof(int) * cs, cudaMemcpyHostToDevice, s)) ||
            (e = cudaMemsetAsync(d_counter, 0, sizeof(unsigned) * 3, s)) ||
            (!list.empty() && (e = cudaMemcpyAsync(d_list, list.data(), sizeof(int) * list.size(),
                                                   cudaMemcpyHostToDevice, s)))) {
            fail(e, "copy");
            break;
        }
        KnnArgs ka;
        ka.x = d_x;
        ka.y = d_y;
        ka.z = d_z;
        ka.acc = d_acc;
        ka.cx = d_c;
        ka.cy = d_c + bc;
        ka.cz = d_c + 2 * (size_t)bc;
        ka.bc = bc;
        ka.cs = cs;
        ka.out = d_knn;
        ka.counter = d_counter;
        ka.error = d_err;
        ka.heavy = d_heavy;
        ka.heavy_count = d_heavy_count;
        ka.list = mask ? d_list : nullptr;
        ka.nlist = (int)list.size();
        const size_t smem = sizeof(KnnWarpSmem) * kKnnWarps;
        if ((e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem))) {
            fail(e, "attribute");
            break;
        }
        int dev = 0, sms = 0, occ = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kKnnWarps * 32, smem);
        if (occ < 1) occ = 1;
        int grid = sms * occ;
        const int nsel = mask ? (int)list.size() : bc;
        const int need = (nsel + kKnnWarps - 1) / kKnnWarps;
        if (grid > need) grid = need > 0 ? need : 1;
        kern<<<grid, kKnnWarps * 32, smem, s>>>(ka);
        if ((e = cudaGetLastError())) {
            fail(e, "launch");
            break;
        }
        unsigned hbuf[2] = {0u, 0u};  // error, heavy_count
        if ((e = cudaMemcpyAsync(hbuf, d_err, sizeof(unsigned) * 2, cudaMemcpyDeviceToHost, s)) ||
            (e = cudaStreamSynchronize(s))) {
            fail(e, "sync");
            break;
        }
        if (hbuf[0]) {
            set_error("bv_knn: block %d has fewer than cs=%d earlier points", (int)hbuf[0] - 1, cs);
            rc = BV_E_TOOLARGE;
            break;
        }
        const int nheavy = (int)hbuf[1];
        if (nheavy > 0) {
            // Blocks with more ties than the warp buffer holds: S can hold up
            // to every earlier point, so each CTA gets n entries (16 bytes
            // each); at most one CTA per SM and 4 GB of scratch in all.
            const size_t per = (size_t)n * 16;
            int g = (int)std::min<size_t>((size_t)nheavy, std::max<size_t>(1, ((size_t)4 << 30) / per));
            g = std::min(g, sms > 0 ? sms : 1);
            const size_t cnt = (size_t)n * (size_t)g;
            if ((e = cudaMalloc(&sc.key, sizeof(unsigned long long) * cnt)) ||
                (e = cudaMalloc(&sc.idx, sizeof(int) * cnt)) || (e = cudaMalloc(&sc.pos, sizeof(int) * cnt))) {
                fail(e, "cudaMalloc (tie scratch)");
                break;
            }
            heavy<<<g, kHeavyThreads, 0, s>>>(ka, nheavy, sc, (size_t)n);
            if ((e = cudaGetLastError()) || (e = cudaStreamSynchronize(s))) {
                fail(e, "tie pass");
                break;
            }
        }
    } while (0);
    cudaFree(d_c);
    cudaFree(d_counter);
    cudaFree(sc.key);
    cudaFree(sc.idx);
    cudaFree(sc.pos);
    return rc;
}

}  // namespace bv

static int knn_host(const double *x, const double *y, const double *z, int n, int bc, int cs,
                    const int *batchNumAccum, const double *cx, const double *cy, const double *cz,
                    int *knn_idx, int device, const unsigned char *mask = nullptr, int earth = 0)
{
    using namespace bv;
    if (!x || !y || !batchNumAccum || !cx || !cy || !knn_idx || n <= 0 || bc <= 0 || cs < 0 ||
        (z && !cz)) {
        set_error("bv_knn: invalid argument");
        return BV_E_INVALID;
    }
    if (earth && z) {
        // src/ckernel.cpp:170-172: "Great Circle (GC) distance is only valid for 2d".
        set_error("bv_knn: the great-circle distance is defined for 2-D locations only");
        return BV_E_INVALID;
    }
    // The great-circle key reads cos(latitude) of every point and centroid,
    // computed here with the host's libm as the reference computes it.
    std::vector<double> zc, czc;
    if (earth) {
        zc.resize(n);
        czc.resize(bc);
        for (int p = 0; p < n; ++p) zc[p] = earth_cos_lat(x[p]);
        for (int b = 0; b < bc; ++b) czc[b] = earth_cos_lat(cx[b]);
        z = zc.data();
        cz = czc.data();
    }
    if (batchNumAccum[0] != 0 || batchNumAccum[bc] > n) {
        set_error("bv_knn: batchNumAccum must start at 0 and stay within n");
        return BV_E_INVALID;
    }
    for (int i = 1; i < bc; ++i)
        if (batchNumAccum[i] < cs) {
            set_error("bv_knn: block %d has %d earlier points < cs=%d", i, batchNumAccum[i], cs);
            return BV_E_INVALID;
        }
    if (cs == 0) return BV_OK;
    BV_CUDA_TRY(cudaSetDevice(device));
    cudaStream_t s;
    BV_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    double *d_x = nullptr, *d_y = nullptr, *d_z = nullptr;
    int *d_acc = nullptr, *d_knn = nullptr;
    int rc = BV_OK;
    cudaError_t e;
    do {
        if ((e = cudaMalloc(&d_x, sizeof(double) * n)) || (e = cudaMalloc(&d_y, sizeof(double) * n)) ||
            (z && (e = cudaMalloc(&d_z, sizeof(double) * n))) ||
            (e = cudaMalloc(&d_acc, sizeof(int) * (bc + 1))) ||
            (e = cudaMalloc(&d_knn, sizeof(int) * (size_t)bc * cs))) {
            set_error("bv_knn: cudaMalloc: %s", cudaGetErrorString(e));
            rc = (e == cudaErrorMemoryAllocation) ? BV_E_NOMEM : BV_E_CUDA;
            break;
        }
        if ((e = cudaMemcpyAsync(d_x, x, sizeof(double) * n, cudaMemcpyHostToDevice, s)) ||
            (e = cudaMemcpyAsync(d_y, y, sizeof(double) * n, cudaMemcpyHostToDevice, s)) ||
            (z && (e = cudaMemcpyAsync(d_z, z, sizeof(double) * n, cudaMemcpyHostToDevice, s))) ||
            (e = cudaMemcpyAsync(d_acc, batchNumAccum, sizeof(int) * (bc + 1), cudaMemcpyHostToDevice, s))) {
            set_error("bv_knn: copy: %s", cudaGetErrorString(e));
            rc = BV_E_CUDA;
            break;
        }
        rc = knn_device(d_x, d_y, d_z, n, bc, cs, d_acc, cx, cy, cz, d_knn, s, mask, earth);
        if (rc) break;
        // Block 0 and the selected blocks' sets back to the caller (the
        // others' entries stay as the caller had them).
        for (int b = 0; b < bc; ++b) {
            if (mask && b > 0 && !mask[b]) continue;
            int e0 = b, e1 = b + 1;
            if (!mask)
                e1 = bc;
            else
                while (e1 < bc && mask[e1]) ++e1;
            if ((e = cudaMemcpyAsync(knn_idx + (size_t)e0 * cs, d_knn + (size_t)e0 * cs,
                                     sizeof(int) * (size_t)(e1 - e0) * cs, cudaMemcpyDeviceToHost, s))) {
                set_error("bv_knn: copy back: %s", cudaGetErrorString(e));
                rc = BV_E_CUDA;
                break;
            }
            b = e1 - 1;
        }
        if (rc) break;
        if ((e = cudaStreamSynchronize(s))) {
            set_error("bv_knn: copy back: %s", cudaGetErrorString(e));
            rc = BV_E_CUDA;
        }
    } while (0);
    cudaFree(d_x);
    cudaFree(d_y);
    cudaFree(d_z);
    cudaFree(d_acc);
    cudaFree(d_knn);
    cudaStreamDestroy(s);
    return rc;
}

extern "C" int bv_knn(const double *x, const double *y, int n, int bc, int cs,
                      const int *batchNumAccum, const double *cx, const double *cy, int *knn_idx,
                      int device)
{
    return knn_host(x, y, nullptr, n, bc, cs, batchNumAccum, cx, cy, nullptr, knn_idx, device);
}

extern "C" int bv_knn_subset(const double *x, const double *y, const double *z, int n, int bc,
                             int cs, const int *batchNumAccum, const double *cx, const double *cy,
                             const double *cz, const unsigned char *mask, int *knn_idx, int device)
{
    if (!mask) {
        bv::set_error("bv_knn_subset: mask is required");
        return BV_E_INVALID;
    }
    return knn_host(x, y, z, n, bc, cs, batchNumAccum, cx, cy, cz, knn_idx, device, mask);
}

extern "C" int bv_knn3(const double *x, const double *y, const double *z, int n, int bc, int cs,
                       const int *batchNumAccum, const double *cx, const double *cy,
                       const double *cz, int *knn_idx, int device)
{
    if (!z || !cz) {
        bv::set_error("bv_knn3: z and cz are required");
        return BV_E_INVALID;
    }
    return knn_host(x, y, z, n, bc, cs, batchNumAccum, cx, cy, cz, knn_idx, device);
}

extern "C" int bv_knn_ex(const double *x, const double *y, const double *z, int n, int bc, int cs,
                         const int *batchNumAccum, const double *cx, const double *cy,
                         const double *cz, const unsigned char *mask, int metric, int *knn_idx,
                         int device)
{
    if (metric != BV_METRIC_EUCLIDEAN && metric != BV_METRIC_EARTH) {
        bv::set_error("bv_knn_ex: unknown distance metric %d", metric);
        return BV_E_INVALID;
    }
    return knn_host(x, y, z, n, bc, cs, batchNumAccum, cx, cy, cz, knn_idx, device, mask,
                    metric == BV_METRIC_EARTH);
}

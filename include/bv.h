/*
 * bv.h -- C ABI of libbv_b200.so, the B200-native block-Vecchia
 * log-likelihood library.
 *
 * Plain pointers and sizes only.  Host pointers unless a name says "_dev".
 * Every entry point returns 0 on success or a negative BV_E* code; the
 * library never exits the process.  bv_llh keeps the NLopt objective
 * signature of the reference's llh_Xvecchia_batch so it drops into
 * nlopt_set_max_objective unchanged.
 */
#ifndef BV_H
#define BV_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ----------------------------------------------------------------- codes */
#define BV_OK 0
#define BV_E_INVALID (-1)   /* bad argument                                  */
#define BV_E_CUDA (-2)      /* CUDA runtime error (message: bv_last_error)   */
#define BV_E_NOMEM (-3)     /* device allocation failed                      */
#define BV_E_NODEVICE (-4)  /* no usable sm_100 device                       */
#define BV_E_TOOLARGE (-5)  /* a size exceeds a documented maximum           */
#define BV_E_TIMEOUT (-6)   /* a bounded device wait gave up                 */

#define BV_PREC_FP64 0  /* plain FP64 method (reference semantics)           */
#define BV_PREC_MIXED 1 /* FP32 factor + FP64 refinement, FP64 fallback      */

#define BV_LARGE_AUTO 0     /* large-block path choice (bv_opts.large_blocks) */
#define BV_LARGE_STREAMED 1 /* left-looking, panels streamed through L2      */
#define BV_LARGE_SLAB 2     /* shared-memory algorithm on a global slab      */
#define BV_SCHED_AUTO 0
#define BV_SCHED_BUCKETED 1
#define BV_SCHED_PERSISTENT 2
#define BV_SCHED_STREAMED 3
#define BV_FAIL_NEGINF 0   /* a failed block makes bv_llh return -HUGE_VAL  */
#define BV_FAIL_CONTINUE 1 /* keep going like the reference: a non-positive
                              pivot is skipped in the log-determinant        */

/* Per-evaluation block status bits (bv_status.flags_or). */
#define BV_ST_COND_FAIL 1u   /* non-positive / NaN pivot in Sigma22          */
#define BV_ST_SCHUR_FAIL 2u  /* non-positive / NaN pivot in Sigma11'         */
#define BV_ST_FP32_FALLBACK 4u /* mixed path redid the block in FP64         */
#define BV_ST_NONFINITE 8u   /* a block's contribution was not finite        */

/* ---------------------------------------------------------------- layout */
/*
 * The block layout the reference's driver builds before the optimizer runs
 * (src/test_Xvecchia_batch.cpp:240-404): blocks in random centroid order,
 * block 0 = the first clusters merged until >= cs points, points of a block
 * in ascending original index, conditioning sets of cs points per block.
 */
typedef struct {
    int n;                     /* number of locations                        */
    int bc;                    /* number of blocks (batchCount)              */
    int cs;                    /* conditioning size (vecchia_cs)             */
    const int *batchNum;       /* [bc]   points per block                    */
    const int *batchNumAccum;  /* [bc+1] block offsets, [bc] == n            */
    const double *x;           /* [n]    block-ordered locations_new->x      */
    const double *y;           /* [n]    block-ordered locations_new->y      */
    const double *obs;         /* [n]    block-ordered h_obs_new             */
    const int *knn_idx;        /* [bc*cs] conditioning indices into x/y/obs;
                                  NULL: computed on the device by bv_knn
                                  from cx/cy                                 */
    const double *cx;          /* [bc]   block centroids (locsCentroid[i +
                                  firstClusterCount - 1]); used if knn_idx
                                  is NULL                                    */
    const double *cy;
    const double *z;           /* [n]    block-ordered third coordinate (the
                                  reference's time_flag locations_new->z:
                                  time for the space-time kernel, or depth
                                  with --3D), NULL for 2-D                    */
    const double *cz;          /* [bc]   third coordinate of the block
                                  centroids, when z is set and knn_idx NULL  */
} bv_layout;

typedef struct {
    int precision;     /* BV_PREC_FP64 | BV_PREC_MIXED                        */
    int kernel;        /* 1,2,3: Matern (the reference's llh evaluates Matern
                          for all three, include/llh_Xvecchia_batch.h:126-144);
                          with a 3-D layout (z set) its distances include z
                          (core_dcmg with z_flag = 1).  4: space-time Matern
                          (core_dcmg_spacetime_matern, src/ckernel.cpp
                          :1421-1458), theta = {sigma2, range_spatial,
                          smooth_spatial, range_time, smooth_time,
                          separability, aux}; needs a 3-D layout           */
    double dist_scale; /* --dist_scale, default 1.0                           */
    int device;        /* CUDA device ordinal                                 */
    int on_failure;    /* BV_FAIL_NEGINF | BV_FAIL_CONTINUE                   */
    int print_iter;    /* print the reference's per-evaluation line           */
    int use_graph;     /* capture one evaluation in a CUDA graph (default 1)  */
    int schedule;      /* BV_SCHED_AUTO (default): every block whose panels
                          fit (M = cs + bs up to ~780) on the multi-CTA
                          streamed kernel (several blocks per SM), larger
                          ones on the persistent one-CTA-per-SM kernel;
                          BV_SCHED_BUCKETED: the persistent kernel, one
                          launch per size bucket (the comparison baseline);
                          BV_SCHED_PERSISTENT: the persistent kernel for
                          every block (the server's algorithm);
                          BV_SCHED_STREAMED: the streamed kernel for every
                          block (an error if one does not fit).  The two
                          kernels round differently; each choice depends on
                          the layout only, so results are reproducible.    */
    double mixed_tol;  /* mixed path: a block is accepted when the estimated
                          relative error of its refined Sigma22^-1 Sigma21
                          (|dX_last| / |X| times the first step's
                          contraction) is at most this; default 1e-8       */
    int shard_count;   /* > 1: this handle evaluates only its shard of the
                          blocks (bv_shard_blocks); partial log-likelihoods of
                          all shards sum to the full one                      */
    int shard_index;   /* 0 .. shard_count-1                                  */
    int large_blocks;  /* blocks too large for one SM's shared memory:
                          BV_LARGE_AUTO (default: the streamed path when more
                          than one wave of blocks needs it, else the slab),
                          BV_LARGE_STREAMED, BV_LARGE_SLAB                   */
    int nugget;        /* 0 (default): theta = {sigma2, range, nu}; theta[3],
                          if given, is not read -- the reference's likelihood
                          never reads it (include/llh_Xvecchia_batch.h:126-144),
                          even for its 4-parameter kernel 3.  1: theta[3] =
                          tau^2 >= 0 is added to the diagonal of Sigma11 and
                          Sigma22 (a point with itself), and bv_llh needs
                          n >= 4 parameters.                                  */
    int earth;         /* 0 (default): Euclidean distances.  1: the
                          reference's --earth (distance_metric = 1): x is the
                          latitude and y the longitude in degrees, distances
                          are great-circle km by the haversine formula
                          (src/ckernel.cpp:145-154) in the covariance and in
                          the conditioning-set key when the handle selects
                          the sets.  2-D Matern kernels (1-3) and FP64 only,
                          as the reference allows it for 2-D locations only. */
    int tune;          /* 0 (default): the streamed kernel's variant from a
                          measured table by the launch's largest block.  1:
                          the first evaluation times every variant on this
                          layout and the handle keeps the fastest (all give
                          the same bits, so results do not depend on the
                          choice); bv_get_status reports the times.        */
    int mixed_fp32;    /* BV_PREC_MIXED only.  0 (default): every block on the
                          FP64 path (its values exactly): on B200 the FP32
                          factor + FP64 refinement kernel took 4.8-6.3x the
                          FP64 path's time on every layout where FP32 could
                          factor the blocks (nu = 0.5), and smoother kernels
                          fail in FP32.  1: the FP32 pass runs whenever a
                          probe of every 64th block accepts at least half of
                          them; blocks it rejects go to the FP64 path.       */
} bv_opts;

/* Distance metrics of bv_knn_ex (the reference's distance_metric). */
#define BV_METRIC_EUCLIDEAN 0
#define BV_METRIC_EARTH     1

typedef struct {
    int blocks;          /* blocks evaluated                                 */
    int cond_fail;       /* blocks with a failed Sigma22 pivot               */
    int schur_fail;      /* blocks with a failed Sigma11' pivot              */
    int fp32_fallback;   /* mixed path: blocks redone in FP64                */
    int nonfinite;       /* blocks whose contribution was not finite         */
    unsigned flags_or;   /* OR of BV_ST_* over all blocks                    */
    double llk;          /* last log-likelihood (before the failure policy)  */
    double device_ms;    /* device time of the last evaluation               */
    double kernel_ms;    /* of which the fused per-block kernel(s)            */
    int failed;          /* blocks with a failed pivot in either factor
                            (cond_fail and schur_fail may count one block
                            twice; this counts it once)                      */
    int launches;        /* kernel launches per evaluation                   */
    int streamed_blocks; /* FP64 path: blocks on the multi-CTA streamed
                            kernel (the rest on the persistent kernel);
                            0 for the mixed path                             */
    int streamed_threads; /* threads per CTA of that kernel (0: none)       */
    int streamed_variant; /* its variant, an index into tune_ms             */
    double tune_ms[6];   /* with bv_opts.tune: the streamed kernel's time on
                            the first evaluation per variant: 96 x 5 CTAs per
                            SM, 160 x 3, 256 x 2 and 128 x 4 threads per CTA
                            generating panel by panel, then 160 x 3 and
                            256 x 2 generating the whole matrix first (0
                            where not timed)                                 */
} bv_status;

typedef struct bv_handle bv_handle;

/* sizeof of the ABI structs in this build, for bindings that restate them
 * (ctypes, cgo): out[0..5] = bv_layout, bv_opts, bv_status, bv_server_opts,
 * bv_server_stats, bv_job_opts; returns the number written (<= n). */
int bv_abi_sizes(size_t *out, int n);

/* Fill *o with the defaults (FP64, Matern, dist_scale 1, device 0,
 * BV_FAIL_NEGINF, no printing, graphs on, BV_SCHED_AUTO, Euclidean). */
void bv_default_opts(bv_opts *o);

/* Create a handle: validates the layout, copies it to the device once
 * (replaces the device allocations and copies of
 * src/test_Xvecchia_batch.cpp:459-600), computes the conditioning sets on the
 * device when layout->knn_idx is NULL, and plans the block schedule.
 * The caller keeps ownership of its arrays. */
int bv_create(const bv_layout *layout, const bv_opts *opts, bv_handle **out);
void bv_destroy(bv_handle *h);

/* NLopt objective (replaces llh_Xvecchia_batch<double>,
 * include/llh_Xvecchia_batch.h:24): n = number of parameters (3 for Matern,
 * 4 with bv_opts.nugget), theta = {sigma2, range, nu[, tau^2]}, grad ignored
 * (derivative-free optimizer),
 * f_data = bv_handle*.  Returns the block-Vecchia log-likelihood; on a block
 * failure under BV_FAIL_NEGINF, or on an error, returns -HUGE_VAL and records
 * the reason in bv_get_status / bv_last_error. */
double bv_llh(unsigned n, const double *theta, double *grad, void *f_data);

/* Same evaluation with an explicit status code. */
int bv_llh_eval(bv_handle *h, const double *theta, double *llk);

/* Per-block contributions of the last evaluation, copied to host [bc]. */
int bv_block_llk(bv_handle *h, double *out, int count);

/* Per-block BV_ST_* bits of the last evaluation, copied to host [bc] (the
 * reference keeps MAGMA's per-block info arrays but never reads them,
 * include/llh_Xvecchia_batch.h:295-299,449-453). */
int bv_block_status(bv_handle *h, unsigned *out, int count);

int bv_get_status(bv_handle *h, bv_status *st);

/* The CUDA stream (cudaStream_t) the handle launches on, for callers that
 * time evaluations with their own events or order work after them. */
int bv_get_stream(bv_handle *h, void **stream);

/* Launch subsequent evaluations on `stream` (a cudaStream_t of the handle's
 * device; NULL restores the handle's own stream). */
int bv_set_stream(bv_handle *h, void *stream);
int bv_iterations(bv_handle *h);
const char *bv_last_error(void);

/* End-to-end evaluation from host buffers: copies obs[n] (and, when not
 * NULL, x/y[n] and knn_idx[bc*cs]) of a layout with the handle's shapes to
 * the device, evaluates, and returns the log-likelihood.  Used when the
 * observations change between calls (simulation studies, serving). */
int bv_llh_host(bv_handle *h, const double *x, const double *y,
                const double *obs, const int *knn_idx, const double *theta,
                double *llk);

/* Allocation-free evaluation, for callers that cannot allocate device memory
 * (an allocator they do not own, a memory pool that forbids extra
 * cudaMalloc calls, embedding in a host application that manages every
 * buffer itself).  No counterpart in the reference.  The caller passes
 * device pointers to the block-ordered locations and observations (x, y,
 * obs [n]), the block offsets (batchNumAccum [bc+1]) and the conditioning
 * indices (knn_idx [bc*cs]; block 0 unconditioned), the host parameters
 * theta = {sigma2, range, nu}, and a device pointer llk_out that receives the
 * log-likelihood, or -HUGE_VAL when a block meets a non-positive pivot or the
 * sum is not finite (the BV_FAIL_NEGINF policy; *status_flags then says
 * why).  The library's working memory for this call is a fixed 2 MB device
 * array inside the library (every device that loads the library holds it
 * until exit): at most BV_NOALLOC_MAX_BLOCKS blocks, and every block must
 * fit in one SM's shared memory (cs + bs <= about 236), else BV_E_TOOLARGE.
 * Invalid offsets or indices, or a block 0 with fewer than cs points while
 * other blocks condition on it, give BV_E_INVALID.  The first call on a
 * device looks up that array's device address (cached per device ordinal;
 * a cudaDeviceReset invalidates it, so do not call this entry point after
 * one).  Every call
 * shares the array: calls that overlap on the GPU race, so serialise them
 * (one stream, or synchronise).  Runs on `stream` (a cudaStream_t of the
 * current device; NULL = the default stream) and waits for its own work
 * before it returns: it reads back the layout check and the status flags.
 * Allocates nothing: no cudaMalloc, cudaFree or allocating library call.
 * *status_flags (may be NULL) receives the OR of the blocks' BV_ST_* bits. */
#define BV_NOALLOC_MAX_BLOCKS 131072
int bv_llh_noalloc(const double *x, const double *y, const double *obs,
                   const int *batchNumAccum, const int *knn_idx, int n, int bc,
                   int cs, const double *theta, double dist_scale,
                   double *llk_out, unsigned *status_flags, void *stream);

/* ---------------------------------------------------------------- serving */
/* Continuous-batching evaluation server for many concurrent fitting jobs
 * on one device (no counterpart in the reference, whose driver fits one
 * dataset per process).  Jobs are copied to HBM while their footprint
 * (locations, observations, offsets, conditioning indices) fits the budget;
 * the others wait in FIFO order and are admitted as jobs close.  A scheduler
 * thread batches every pending request of the admitted jobs into one launch
 * over all their blocks (the multi-CTA streamed kernel; blocks beyond its
 * shared memory in a persistent launch before it); requests arriving
 * meanwhile join the next batch, which starts on the SMs the running batch
 * releases.  Each result is bit-identical to bv_llh_eval on the same layout
 * under the default schedule, alone or in a mix. */
typedef struct bv_server bv_server;
typedef struct {
    int device;
    size_t hbm_budget;  /* bytes for job data; 0 = 90% of free memory      */
    int max_batch;      /* requests per batch (default 256)                */
    int on_failure;     /* BV_FAIL_NEGINF | BV_FAIL_CONTINUE               */
    int max_inflight;   /* batches on the device at once, 1..8 (default 2) */
} bv_server_opts;
typedef struct {
    long long evals, batches;
    double mean_batch;   /* requests per batch                              */
    double p50_ms, p99_ms, max_ms;  /* request latency, submit to result    */
    size_t bytes_in_use, hbm_budget;
    int jobs_admitted, jobs_waiting;
} bv_server_stats;
void bv_server_default_opts(bv_server_opts *o);
int bv_server_create(const bv_server_opts *opts, bv_server **out);
void bv_server_destroy(bv_server *s);
/* Copies the layout (conditioning indices required); *job_id identifies it. */
int bv_server_open_job(bv_server *s, const bv_layout *layout, double dist_scale,
                       int *job_id);
/* The same with per-job options: nugget = 1 makes the job's requests carry
 * theta = {sigma2, range, nu, tau^2} (bv_opts.nugget semantics). */
typedef struct {
    double dist_scale;
    int nugget;
} bv_job_opts;
int bv_server_open_job_ex(bv_server *s, const bv_layout *layout,
                          const bv_job_opts *opts, int *job_id);
int bv_server_job_admitted(bv_server *s, int job_id, int *admitted);
/* The job's memory is released once its in-flight requests complete. */
int bv_server_close_job(bv_server *s, int job_id);
/* Queue one evaluation at theta = {sigma2, range, nu} (plus tau^2 for a job
 * opened with a nugget); returns at once. */
int bv_server_submit(bv_server *s, int job_id, const double *theta,
                     long long *req_id);
/* Wait for a request (timeout_ms < 0: no limit; BV_E_TIMEOUT otherwise). */
int bv_server_wait(bv_server *s, long long req_id, double *llk,
                   double *latency_ms, int timeout_ms);
int bv_server_get_stats(bv_server *s, bv_server_stats *st);
/* Clears the evaluation count and latency record (e.g. after a warm-up). */
int bv_server_reset_stats(bv_server *s);

/* Block sharding for multi-GPU evaluation (blocks are independent given
 * theta; the reference runs them all on one GPU).  Blocks are ranked by cost
 * (M^3 with M = cs + bs, block 0 unconditioned), largest first, ties by
 * index, and dealt round-robin to shard_count shards.  mask[b] = 1 for the
 * blocks of shard shard_index.  Host only. */
int bv_shard_blocks(const int *batchNum, int bc, int cs, int shard_count,
                    int shard_index, unsigned char *mask);

/* ---------------------------------------------------- conditioning sets */
/* Conditioning sets on the device (replaces findNearestPoints,
 * include/nearest_neighbor.h:76-148, over blocks 1..bc-1 as called at
 * src/test_Xvecchia_batch.cpp:368-390): block i >= 1 takes the cs points of
 * blocks 0..i-1 nearest to (cx[i], cy[i]), in the reference's selection
 * order including its tie order; block 0 takes points 0..cs-1.  Host
 * buffers in and out. */
int bv_knn(const double *x, const double *y, int n, int bc, int cs,
           const int *batchNumAccum, const double *cx, const double *cy,
           int *knn_idx, int device);

/* The same for 3-D locations (findNearestPoints with time_flag, the key
 * sqrt(d^2 + dz^2) of include/nearest_neighbor.h:101-104). */
int bv_knn3(const double *x, const double *y, const double *z, int n, int bc, int cs,
            const int *batchNumAccum, const double *cx, const double *cy,
            const double *cz, int *knn_idx, int device);

/* Conditioning sets with every option: z/cz (3-D locations) may be NULL,
 * mask (may be NULL) selects blocks as bv_knn_subset does, and metric is
 * BV_METRIC_EUCLIDEAN or BV_METRIC_EARTH (findNearestPoints with
 * distance_metric = 1, include/nearest_neighbor.h:93-96: great-circle km
 * from the centroid, x latitude and y longitude in degrees; 2-D only).  The
 * great-circle key uses the device's sin and asin, which may differ from the
 * host libm's in the last bit: two candidates whose distances agree to a few
 * ulps may then be ordered differently from the reference. */
int bv_knn_ex(const double *x, const double *y, const double *z, int n, int bc, int cs,
              const int *batchNumAccum, const double *cx, const double *cy,
              const double *cz, const unsigned char *mask, int metric, int *knn_idx,
              int device);

/* Conditioning sets of a subset of the blocks (one rank's shard, mask from
 * bv_shard_blocks): blocks b >= 1 with mask[b] != 0 get their sets (and
 * block 0 its points 0..cs-1); the other entries of knn_idx are left as
 * they were.  z / cz may be NULL (2-D).  Each rank of a multi-GPU run
 * selects only its own blocks' sets (the reference selects all on one host,
 * src/test_Xvecchia_batch.cpp:368-390). */
int bv_knn_subset(const double *x, const double *y, const double *z, int n, int bc,
                  int cs, const int *batchNumAccum, const double *cx, const double *cy,
                  const double *cz, const unsigned char *mask, int *knn_idx, int device);

/* ------------------------------------------------------- host layout */
/* The driver's setup on the host (src/test_Xvecchia_batch.cpp:240-352):
 * classic Vecchia when n < 2*bc, else k-means (random_initializer + Lloyd
 * kmean_par with `epochs` epochs), random centroid order (srand(42)),
 * reorderIndex, firstbatch, cluster_combine, cluster_to_batch.
 * Outputs are caller-allocated with capacity nclusters (= n < 2*bc ? n : bc)
 * for batchNum / cx / cy, nclusters+1 for batchNumAccum, n for
 * x_new / y_new / obs_new.  *bc_out receives batchCount. */
int bv_layout_build(const double *x, const double *y, const double *obs,
                    int n, int bc, int cs, int seed, int epochs, int threads,
                    int *batchNum, int *batchNumAccum, double *x_new,
                    double *y_new, double *obs_new, double *cx, double *cy,
                    int *bc_out, int *first_cluster_count);

/* The same steps from a given clustering (labels[n], centroids cx/cy[k]). */
int bv_layout_from_clusters(const double *x, const double *y,
                            const double *obs, int n, int k,
                            const int *labels, const double *ccx,
                            const double *ccy, int cs, int *batchNum,
                            int *batchNumAccum, double *x_new, double *y_new,
                            double *obs_new, double *cx, double *cy,
                            int *bc_out, int *first_cluster_count);

/* k-means alone (random_initializer + kmean_par semantics, deterministic,
 * exact nearest-centroid assignment through a uniform grid). */
int bv_kmeans(const double *x, const double *y, int n, int k, int seed,
              int epochs, int threads, int *labels, double *cx, double *cy);

/* GenerateXYLoc (src/ckernel.cpp:43-76): n jittered grid points, glibc
 * rand() seeded with `seed`, Morton-sorted and quantised to 1/65535. */
int bv_generate_xy(int n, int seed, double *x, double *y);

/* GenerateXYLoc_ST (src/ckernel.cpp:78-118): n jittered grid points (grid
 * order) repeated over t_slots time slots, z = (slot + 1) / t_slots; the
 * arrays hold n * t_slots entries. */
int bv_generate_xyt(int n, int t_slots, int seed, double *x, double *y, double *z);

/* bv_layout_build for 3-D locations (the reference's time_flag set-up:
 * k-means on (x, y, z), random_reordering_3d, reorderIndex and
 * cluster_to_batch with z).  z_new[n] and cz[nclusters] receive the
 * block-ordered third coordinate and the block centroids' one. */
int bv_layout_build3(const double *x, const double *y, const double *z,
                     const double *obs, int n, int bc, int cs, int seed, int epochs,
                     int threads, int *batchNum, int *batchNumAccum, double *x_new,
                     double *y_new, double *z_new, double *obs_new, double *cx,
                     double *cy, double *cz, int *bc_out, int *first_cluster_count);

/* Centroid orderings: the reference's --permutation (random, the default;
 * morton, kdtree, hilbert, mmd: src/test_Xvecchia_batch.cpp:286-314 and
 * include/ckernel.h:148-1000, the 3-D variants for 3-D locations).  Morton
 * and Hilbert quantise the centroids to k / 65535 (they need coordinates in
 * [0, 1]); reorderIndex then maps each reordered centroid to its nearest
 * original one, and two centroids mapped to one cluster are an error, as
 * they stop the reference. */
#define BV_ORDER_RANDOM  0
#define BV_ORDER_MORTON  1
#define BV_ORDER_KDTREE  2
#define BV_ORDER_HILBERT 3
#define BV_ORDER_MMD     4

/* bv_layout_build / bv_layout_build3 with a centroid ordering; z, z_new and
 * cz NULL for 2-D locations. */
int bv_layout_build_ex(const double *x, const double *y, const double *z,
                       const double *obs, int n, int bc, int cs, int seed, int epochs,
                       int threads, int ordering, int *batchNum, int *batchNumAccum,
                       double *x_new, double *y_new, double *z_new, double *obs_new,
                       double *cx, double *cy, double *cz, int *bc_out,
                       int *first_cluster_count);

/* bv_layout_from_clusters with an optional third coordinate and a centroid
 * ordering. */
int bv_layout_from_clusters_ex(const double *x, const double *y, const double *z,
                               const double *obs, int n, int k, const int *labels,
                               const double *ccx, const double *ccy, const double *ccz,
                               int cs, int ordering, int *batchNum, int *batchNumAccum,
                               double *x_new, double *y_new, double *z_new,
                               double *obs_new, double *cx, double *cy, double *cz,
                               int *bc_out, int *first_cluster_count);

/* The ordering alone, in place on n centroids (z = NULL: 2-D). */
int bv_order_centroids(int ordering, int n, double *x, double *y, double *z);

#ifdef __cplusplus
}
#endif
#endif /* BV_H */

// bv_layout.cpp -- host-side block layout (k-means ordering stays on the host).
//
// Produces the layout the reference's driver builds before optimisation
// (src/test_Xvecchia_batch.cpp:240-352): locations, k-means clusters, a
// random centroid order, block 0 merged until it holds >= cs points, blocks
// of ascending original point index.  The reference's steps are O(n*bc)
// (cluster_to_batch, include/vecchia_helper_method.h:63-92), O(bc^2)
// (reorderIndex :128-160) and O(n*bc*epochs) (kmean_par, src/kmeans.cpp:59-145);
// here the same results come from bucketing, hashing and a uniform-grid exact
// nearest-centroid search.
#include <omp.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <random>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "../../include/bv.h"

namespace bv {
void set_error(const char *fmt, ...);
}

namespace {

// -------------------------------------------------------------- locations
// 16-bit Morton interleave (x in the even bits, y in the odd bits).
uint32_t spread16(uint32_t v)
{
    uint32_t r = 0;
    for (int b = 0; b < 16; ++b) r |= ((v >> b) & 1u) << (2 * b);
    return r;
}
uint32_t gather16(uint32_t v)
{
    uint32_t r = 0;
    for (int b = 0; b < 16; ++b) r |= ((v >> (2 * b)) & 1u) << b;
    return r;
}

// Squared distance as the reference's Point euclidean_dist evaluates it
// (include/Point.h:73-79, DIM 3), as its -O3 build contracts the
// accumulation: fma(d2, d2, fma(d1, d1, d0*d0)).  2-D points have a zero
// third coordinate, where this is fma(d1, d1, d0*d0) exactly.
inline double kdist(double px, double py, double cx, double cy)
{
    const double d0 = px - cx, d1 = py - cy;
    return std::fma(d1, d1, d0 * d0);
}
inline double kdist3(double px, double py, double pz, double cx, double cy, double cz)
{
    const double d0 = px - cx, d1 = py - cy, d2 = pz - cz;
    return std::fma(d2, d2, std::fma(d1, d1, d0 * d0));
}

// Bit patterns of a point's coordinates, for exact-equality hashing.
struct Key3 {
    uint64_t a, b, c;
    bool operator==(const Key3 &o) const { return a == o.a && b == o.b && c == o.c; }
};
struct Key3Hash {
    size_t operator()(const Key3 &k) const
    {
        uint64_t h = k.a * 0x9E3779B97F4A7C15ull;
        h ^= k.b + 0x632BE59BD9B4E019ull + (h << 6) + (h >> 2);
        h ^= k.c + 0x85EBCA77C2B2AE63ull + (h << 6) + (h >> 2);
        return (size_t)h;
    }
};
// signed_zero_equal: map -0 to +0 (points at zero distance compare equal).
inline Key3 key3(double x, double y, double z, bool signed_zero_equal)
{
    if (signed_zero_equal) {
        if (x == 0.0) x = 0.0;
        if (y == 0.0) y = 0.0;
        if (z == 0.0) z = 0.0;
    }
    Key3 k;
    std::memcpy(&k.a, &x, 8);
    std::memcpy(&k.b, &y, 8);
    std::memcpy(&k.c, &z, 8);
    return k;
}

// Exact nearest centroid (lowest index among equal distances, as the
// reference's strict '<' scan from index 0) through a uniform grid.
struct CentroidGrid {
    int G = 1;
    double x0 = 0, y0 = 0, h = 1;
    std::vector<int> start, items;
    void build(const std::vector<double> &cx, const std::vector<double> &cy)
    {
        const int k = (int)cx.size();
        double xmin = DBL_MAX, xmax = -DBL_MAX, ymin = DBL_MAX, ymax = -DBL_MAX;
        for (int c = 0; c < k; ++c) {
            xmin = std::min(xmin, cx[c]);
            xmax = std::max(xmax, cx[c]);
            ymin = std::min(ymin, cy[c]);
            ymax = std::max(ymax, cy[c]);
        }
        G = std::max(1, (int)std::ceil(std::sqrt(k / 2.0)));
        const double span = std::max(std::max(xmax - xmin, ymax - ymin), 1e-300);
        h = span / G * (1.0 + 1e-12);
        x0 = xmin;
        y0 = ymin;
        std::vector<int> cnt((size_t)G * G + 1, 0);
        std::vector<int> cell(k);
        for (int c = 0; c < k; ++c) {
            cell[c] = cell_of(cx[c], cy[c]);
            cnt[cell[c] + 1]++;
        }
        for (size_t i = 1; i < cnt.size(); ++i) cnt[i] += cnt[i - 1];
        start = cnt;
        items.assign(k, 0);
        std::vector<int> fill(cnt.begin(), cnt.end() - 1);
        for (int c = 0; c < k; ++c) items[fill[cell[c]]++] = c;  // ascending c per cell
    }
    int clampi(int v) const { return v < 0 ? 0 : (v >= G ? G - 1 : v); }
    int cell_of(double x, double y) const
    {
        int ix = clampi((int)std::floor((x - x0) / h));
        int iy = clampi((int)std::floor((y - y0) / h));
        return iy * G + ix;
    }
    // Nearest centroid of (px, py[, pz]); the grid is over (x, y), whose
    // distance bounds the 3-D one from below, so the search stays exact.
    int nearest(double px, double py, const std::vector<double> &cx,
                const std::vector<double> &cy, double pz = 0.0,
                const std::vector<double> *cz = nullptr) const
    {
        const int ix = clampi((int)std::floor((px - x0) / h));
        const int iy = clampi((int)std::floor((py - y0) / h));
        double best = DBL_MAX;
        int bi = -1;
        // Distance from the point to the outside of the clamped cell box of
        // ring r is at least (r - 1) * h minus how far the point sits outside
        // the grid (bounded below by the point-to-grid distance).
        const double outx = std::max(0.0, std::max(x0 - px, px - (x0 + G * h)));
        const double outy = std::max(0.0, std::max(y0 - py, py - (y0 + G * h)));
        const double out = std::max(outx, outy);
        auto visit = [&](int xx, int yy) {
            if (xx < 0 || xx >= G || yy < 0 || yy >= G) return;
            const int cidx = yy * G + xx;
            for (int q = start[cidx]; q < start[cidx + 1]; ++q) {
                const int c = items[q];
                const double d = cz ? kdist3(px, py, pz, cx[c], cy[c], (*cz)[c])
                                    : kdist(px, py, cx[c], cy[c]);
                if (d < best || (d == best && c < bi)) {
                    best = d;
                    bi = c;
                }
            }
        };
        for (int r = 0; r <= G; ++r) {
            if (r == 0) {
                visit(ix, iy);
            } else {
                for (int xx = ix - r; xx <= ix + r; ++xx) {
                    visit(xx, iy - r);
                    visit(xx, iy + r);
                }
                for (int yy = iy - r + 1; yy <= iy + r - 1; ++yy) {
                    visit(ix - r, yy);
                    visit(ix + r, yy);
                }
            }
            // Centroids outside rings 0..r are at least (r * h - out) away
            // (in one coordinate); continue while they could tie or win.
            const double lb = r * h - out;
            if (bi >= 0 && lb > 0 && lb * lb > best * (1.0 + 1e-9) + 1e-300) break;
        }
        return bi;
    }
};

}  // namespace

extern "C" int bv_generate_xy(int n, int seed, double *x, double *y)
{
    if (n <= 0 || !x || !y) {
        bv::set_error("bv_generate_xy: invalid argument");
        return BV_E_INVALID;
    }
    // src/ckernel.cpp:43-76: jittered sqrt(n) x sqrt(n) grid from glibc rand().
    srand(seed);
    const int sqrtn = (int)std::ceil(std::sqrt((double)n));
    int index = 0;
    // uniform_distribution (src/ckernel.cpp:36-41): myRand * range + rangeLow,
    // which the reference's -march=native build contracts to one fma.
    auto unif = [](double lo, double hi) {
        const double u = (double)rand() / (double)(1.0 + RAND_MAX);
        return std::fma(u, hi - lo, lo);
    };
    for (int i = 0; i < sqrtn && index < n; ++i)
        for (int j = 0; j < sqrtn && index < n; ++j) {
            x[index] = ((i + 1) - 0.5 + unif(-0.4, 0.4)) / sqrtn;
            y[index] = ((j + 1) - 0.5 + unif(-0.4, 0.4)) / sqrtn;
            ++index;
        }
    // zsort_locations (include/ckernel.h:103-125): quantise to 16 bits,
    // Morton-sort, decode.
    std::vector<uint32_t> z(n);
    for (int i = 0; i < n; ++i) {
        const uint16_t qx = (uint16_t)(x[i] * (double)UINT16_MAX + .5);
        const uint16_t qy = (uint16_t)(y[i] * (double)UINT16_MAX + .5);
        z[i] = (spread16(qy) << 1) + spread16(qx);
    }
    std::sort(z.begin(), z.end());
    for (int i = 0; i < n; ++i) {
        x[i] = (double)gather16(z[i]) / (double)UINT16_MAX;
        y[i] = (double)gather16(z[i] >> 1) / (double)UINT16_MAX;
    }
    return BV_OK;
}

extern "C" int bv_generate_xyt(int n, int t_slots, int seed, double *x, double *y, double *z)
{
    if (n <= 0 || t_slots <= 0 || !x || !y || !z) {
        bv::set_error("bv_generate_xyt: invalid argument");
        return BV_E_INVALID;
    }
    // src/ckernel.cpp:78-118: the same jittered grid as GenerateXYLoc from
    // glibc rand(), in grid order (no Morton sort or quantisation), repeated
    // for each time slot with z = (slot + 1) / t_slots.
    srand(seed);
    const int sqrtn = (int)std::ceil(std::sqrt((double)n));
    int index = 0;
    // uniform_distribution (src/ckernel.cpp:36-41): myRand * range + rangeLow,
    // which the reference's -march=native build contracts to one fma.
    auto unif = [](double lo, double hi) {
        const double u = (double)rand() / (double)(1.0 + RAND_MAX);
        return std::fma(u, hi - lo, lo);
    };
    for (int i = 0; i < sqrtn && index < n; ++i)
        for (int j = 0; j < sqrtn && index < n; ++j) {
            x[index] = ((i + 1) - 0.5 + unif(-0.4, 0.4)) / sqrtn;
            y[index] = ((j + 1) - 0.5 + unif(-0.4, 0.4)) / sqrtn;
            z[index] = 1.0 / t_slots;
            ++index;
        }
    for (int t = 1; t < t_slots; ++t)
        for (int i = 0; i < n; ++i) {
            x[i + (size_t)t * n] = x[i];
            y[i + (size_t)t * n] = y[i];
            z[i + (size_t)t * n] = (double)(t + 1) / t_slots;
        }
    return BV_OK;
}

// k-means with an optional third coordinate (z = NULL: 2-D).
static int kmeans_impl(const double *x, const double *y, const double *z, int n, int k, int seed,
                       int epochs, int threads, int *labels, double *ccx, double *ccy, double *ccz)
{
    if (!x || !y || !labels || !ccx || !ccy || (z && !ccz) || n <= 0 || k <= 0 || k > n ||
        epochs < 0) {
        bv::set_error("bv_kmeans: invalid argument");
        return BV_E_INVALID;
    }
    // random_initializer (include/initializer.h:35-56): mt19937(seed) draws
    // from [0, n] (a draw of n would read past the array; it is redrawn
    // here), skipping points whose coordinates repeat an earlier centroid.
    std::mt19937 gen(seed);
    std::uniform_int_distribution<> distrib(0, n);
    std::vector<double> cx, cy, cz;
    cx.reserve(k);
    cy.reserve(k);
    // Coordinates as bits (z = 0 for 2-D points, whose third coordinate is zero).
    std::unordered_set<Key3, Key3Hash> seen;
    seen.reserve((size_t)k * 2);
    size_t guard = 0;
    while ((int)cx.size() < k) {
        const int r = distrib(gen);
        if (++guard > (size_t)200 * n + 1000000) {
            bv::set_error("bv_kmeans: fewer than k=%d distinct locations", k);
            return BV_E_INVALID;
        }
        if (r >= n) continue;
        if (!seen.insert(key3(x[r], y[r], z ? z[r] : 0.0, false)).second) continue;
        cx.push_back(x[r]);
        cy.push_back(y[r]);
        if (z) cz.push_back(z[r]);
    }
    // kmean_par (src/kmeans.cpp:59-145): assignment to the nearest centroid
    // (strict '<', lowest index wins ties), sums in point order, an empty
    // cluster takes point mt19937(42)-drawn from [0, n-1] (a fresh generator
    // per empty cluster, so every empty cluster takes the same point), then
    // centroid = sum / count.
    std::vector<int> lab(n, 0);
    std::vector<double> sx(k), sy(k), sz(k);
    std::vector<int> card(k);
    const int nt = threads > 0 ? threads : omp_get_max_threads();
    const std::vector<double> *czp = z ? &cz : nullptr;
    for (int ep = 0; ep < epochs; ++ep) {
        CentroidGrid grid;
        grid.build(cx, cy);
#pragma omp parallel for num_threads(nt) schedule(static, 4096)
        for (int p = 0; p < n; ++p) lab[p] = grid.nearest(x[p], y[p], cx, cy, z ? z[p] : 0.0, czp);
        std::fill(sx.begin(), sx.end(), 0.0);
        std::fill(sy.begin(), sy.end(), 0.0);
        std::fill(sz.begin(), sz.end(), 0.0);
        std::fill(card.begin(), card.end(), 0);
        for (int p = 0; p < n; ++p) {
            const int c = lab[p];
            sx[c] += x[p];
            sy[c] += y[p];
            if (z) sz[c] += z[p];
            card[c]++;
        }
        for (int c = 0; c < k; ++c) {
            if (card[c] == 0) {
                std::mt19937 g42(42);
                std::uniform_int_distribution<> d42(0, n - 1);
                const int r = d42(g42);
                sx[c] += x[r];
                sy[c] += y[r];
                if (z) sz[c] += z[r];
                lab[r] = c;
                card[c] += 1;
            }
            cx[c] = sx[c] / (double)card[c];
            cy[c] = sy[c] / (double)card[c];
            if (z) cz[c] = sz[c] / (double)card[c];
        }
    }
    if (epochs == 0) {
        CentroidGrid grid;
        grid.build(cx, cy);
        for (int p = 0; p < n; ++p) lab[p] = grid.nearest(x[p], y[p], cx, cy, z ? z[p] : 0.0, czp);
    }
    std::memcpy(labels, lab.data(), sizeof(int) * n);
    std::memcpy(ccx, cx.data(), sizeof(double) * k);
    std::memcpy(ccy, cy.data(), sizeof(double) * k);
    if (z) std::memcpy(ccz, cz.data(), sizeof(double) * k);
    return BV_OK;
}

extern "C" int bv_kmeans(const double *x, const double *y, int n, int k, int seed, int epochs,
                         int threads, int *labels, double *ccx, double *ccy)
{
    return kmeans_impl(x, y, nullptr, n, k, seed, epochs, threads, labels, ccx, ccy, nullptr);
}

// The driver's layout steps after clustering, with an optional third
// coordinate (z, ccz, z_new, cz all NULL: 2-D; the reference's time_flag
// variants random_reordering_3d, include/ckernel.h:811-840, and the z terms of
// reorderIndex and cluster_to_batch otherwise).
static int layout_from_clusters_impl(const double *x, const double *y, const double *z,
                                     const double *obs, int n, int k, const int *labels_in,
                                     const double *ccx, const double *ccy, const double *ccz,
                                     int cs, int *batchNum, int *batchNumAccum, double *x_new,
                                     double *y_new, double *z_new, double *obs_new, double *cx,
                                     double *cy, double *cz, int *bc_out, int *first_cluster_count)
{
    if (!x || !y || !obs || !labels_in || !ccx || !ccy || !batchNum || !batchNumAccum || !x_new ||
        !y_new || !obs_new || !cx || !cy || !bc_out || n <= 0 || k <= 0 || cs < 0 ||
        (z && (!ccz || !z_new || !cz))) {
        bv::set_error("bv_layout_from_clusters: invalid argument");
        return BV_E_INVALID;
    }
    std::vector<int> labels(labels_in, labels_in + n);
    // countPointsInClusters (include/vecchia_helper_method.h:207-254)
    std::vector<int> clusterNum(k, 0);
    for (int p = 0; p < n; ++p) {
        if (labels[p] < 0 || labels[p] >= k) {
            bv::set_error("bv_layout_from_clusters: label %d of point %d outside [0,%d)",
                          labels[p], p, k);
            return BV_E_INVALID;
        }
        clusterNum[labels[p]]++;
    }
    // random_reordering (include/ckernel.h:177-202): srand(42), Fisher-Yates
    // from the end with rand() % (i+1).
    std::vector<double> px(ccx, ccx + k), py(ccy, ccy + k), pz(k, 0.0);
    if (z) pz.assign(ccz, ccz + k);
    srand(42);
    for (int i = k - 1; i > 0; --i) {
        const int j = rand() % (i + 1);
        std::swap(px[i], px[j]);
        std::swap(py[i], py[j]);
        std::swap(pz[i], pz[j]);
    }
    // reorderIndex (include/vecchia_helper_method.h:128-160): index of the
    // first original centroid at zero distance = lowest index with the same
    // coordinates.  Where several centroids coincide (clusters of duplicated
    // locations) the reference maps all of them to that lowest index, so one
    // cluster's points are taken twice and the other's are lost; here the
    // k-th shuffled occurrence of a coordinate pair maps to the k-th original
    // with it, which is the same map whenever the centroids are distinct and
    // otherwise puts every point in exactly one block.
    // Coordinates compared by value (-0 and +0 are at zero distance).
    std::unordered_map<Key3, std::vector<int>, Key3Hash> first_at;
    first_at.reserve((size_t)k * 2);
    for (int j = 0; j < k; ++j)  // ascending j
        first_at[key3(ccx[j], ccy[j], z ? ccz[j] : 0.0, true)].push_back(j);
    std::unordered_map<Key3, int, Key3Hash> taken;
    std::vector<int> perm(k);
    for (int i = 0; i < k; ++i) {
        const Key3 key = key3(px[i], py[i], pz[i], true);
        perm[i] = first_at.at(key)[taken[key]++];
    }
    // firstbatch (:95-108)
    int fcs = 0, fcc = 0, acc_sz = 0;
    for (int i = 0; i < k; ++i) {
        acc_sz += clusterNum[perm[i]];
        if (acc_sz >= cs) {
            fcs = acc_sz;
            fcc = i + 1;
            break;
        }
    }
    if (fcc == 0) {
        bv::set_error("bv_layout_from_clusters: n=%d points cannot fill a first block of cs=%d",
                      n, cs);
        return BV_E_INVALID;
    }
    const int bc = k - fcc + 1;
    // cluster_combine (:36-61)
    if (fcc > 1) {
        for (int i = 1; i < fcc; ++i) {
            const int from = perm[i];
            for (int p = 0; p < n; ++p)
                if (labels[p] == from) labels[p] = perm[0];
            perm[i] = perm[0];
            clusterNum[perm[i]] = fcs;
        }
    }
    // batchNum / batchNumAccum (src/test_Xvecchia_batch.cpp:341-349)
    const int *batchIndex = perm.data() + fcc - 1;
    batchNumAccum[0] = 0;
    for (int i = 0; i < bc; ++i) {
        batchNum[i] = clusterNum[batchIndex[i]];
        batchNumAccum[i + 1] = batchNumAccum[i] + batchNum[i];
    }
    if (batchNumAccum[bc] != n) {
        bv::set_error("bv_layout_from_clusters: blocks cover %d of %d points", batchNumAccum[bc],
                      n);
        return BV_E_INVALID;
    }
    // cluster_to_batch (:63-92): block i takes the first batchNum[i] points
    // (ascending index) labelled batchIndex[i].
    std::vector<int> bstart(k + 1, 0), bitems(n);
    for (int p = 0; p < n; ++p) bstart[labels[p] + 1]++;
    for (int c = 0; c < k; ++c) bstart[c + 1] += bstart[c];
    {
        std::vector<int> fill(bstart.begin(), bstart.end() - 1);
        for (int p = 0; p < n; ++p) bitems[fill[labels[p]]++] = p;
    }
    for (int i = 0; i < bc; ++i) {
        const int c = batchIndex[i];
        const int have = bstart[c + 1] - bstart[c];
        if (have < batchNum[i]) {
            bv::set_error("bv_layout_from_clusters: cluster %d has %d points, block %d needs %d", c,
                          have, i, batchNum[i]);
            return BV_E_INVALID;
        }
        for (int j = 0; j < batchNum[i]; ++j) {
            const int p = bitems[bstart[c] + j];
            x_new[batchNumAccum[i] + j] = x[p];
            y_new[batchNumAccum[i] + j] = y[p];
            if (z) z_new[batchNumAccum[i] + j] = z[p];
            obs_new[batchNumAccum[i] + j] = obs[p];
        }
    }
    // Block centroid: locsCentroid[i + firstClusterCount - 1]
    // (include/nearest_neighbor.h:80-81).
    for (int i = 0; i < bc; ++i) {
        cx[i] = px[i + fcc - 1];
        cy[i] = py[i + fcc - 1];
        if (z) cz[i] = pz[i + fcc - 1];
    }
    *bc_out = bc;
    if (first_cluster_count) *first_cluster_count = fcc;
    return BV_OK;
}

extern "C" int bv_layout_from_clusters(const double *x, const double *y, const double *obs, int n,
                                       int k, const int *labels_in, const double *ccx,
                                       const double *ccy, int cs, int *batchNum,
                                       int *batchNumAccum, double *x_new, double *y_new,
                                       double *obs_new, double *cx, double *cy, int *bc_out,
                                       int *first_cluster_count)
{
    return layout_from_clusters_impl(x, y, nullptr, obs, n, k, labels_in, ccx, ccy, nullptr, cs,
                                     batchNum, batchNumAccum, x_new, y_new, nullptr, obs_new, cx,
                                     cy, nullptr, bc_out, first_cluster_count);
}

static int layout_build_impl(const double *x, const double *y, const double *z, const double *obs,
                             int n, int bc, int cs, int seed, int epochs, int threads,
                             int *batchNum, int *batchNumAccum, double *x_new, double *y_new,
                             double *z_new, double *obs_new, double *cx, double *cy, double *cz,
                             int *bc_out, int *first_cluster_count)
{
    if (!x || !y || !obs || n <= 0 || bc <= 0) {
        bv::set_error("bv_layout_build: invalid argument");
        return BV_E_INVALID;
    }
    // src/test_Xvecchia_batch.cpp:104: classic Vecchia when n < 2*bc.
    const int k = (n < 2 * bc) ? n : bc;
    std::vector<int> labels(n);
    std::vector<double> ccx(k), ccy(k), ccz(z ? k : 0);
    if (n < 2 * bc) {
        for (int p = 0; p < n; ++p) {
            labels[p] = p;
            ccx[p] = x[p];
            ccy[p] = y[p];
            if (z) ccz[p] = z[p];
        }
    } else {
        int rc = kmeans_impl(x, y, z, n, k, seed, epochs, threads, labels.data(), ccx.data(),
                             ccy.data(), z ? ccz.data() : nullptr);
        if (rc) return rc;
    }
    return layout_from_clusters_impl(x, y, z, obs, n, k, labels.data(), ccx.data(), ccy.data(),
                                     z ? ccz.data() : nullptr, cs, batchNum, batchNumAccum, x_new,
                                     y_new, z_new, obs_new, cx, cy, cz, bc_out,
                                     first_cluster_count);
}

extern "C" int bv_layout_build(const double *x, const double *y, const double *obs, int n, int bc,
                               int cs, int seed, int epochs, int threads, int *batchNum,
                               int *batchNumAccum, double *x_new, double *y_new, double *obs_new,
                               double *cx, double *cy, int *bc_out, int *first_cluster_count)
{
    return layout_build_impl(x, y, nullptr, obs, n, bc, cs, seed, epochs, threads, batchNum,
                             batchNumAccum, x_new, y_new, nullptr, obs_new, cx, cy, nullptr, bc_out,
                             first_cluster_count);
}

extern "C" int bv_layout_build3(const double *x, const double *y, const double *z,
                                const double *obs, int n, int bc, int cs, int seed, int epochs,
                                int threads, int *batchNum, int *batchNumAccum, double *x_new,
                                double *y_new, double *z_new, double *obs_new, double *cx,
                                double *cy, double *cz, int *bc_out, int *first_cluster_count)
{
    if (!z || !z_new || !cz) {
        bv::set_error("bv_layout_build3: z, z_new and cz are required");
        return BV_E_INVALID;
    }
    return layout_build_impl(x, y, z, obs, n, bc, cs, seed, epochs, threads, batchNum,
                             batchNumAccum, x_new, y_new, z_new, obs_new, cx, cy, cz, bc_out,
                             first_cluster_count);
}

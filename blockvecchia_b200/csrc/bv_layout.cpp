// bv_layout.cpp -- host-side block layout (k-means ordering stays on the host).
//
// Produces the layout the reference's driver builds before optimisation
// (src/test_Xvecchia_batch.cpp:240-352): locations, k-means clusters, a
// centroid order (random by default; Morton, kd-tree, Hilbert or
// maximum-minimum distance), block 0 merged until it holds >= cs points,
// blocks of ascending original point index.  The reference's steps are O(n*bc)
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

// Squared distance as reorderIndex writes it (include/vecchia_helper_method.h:
// 138-144: dx*dx + dy*dy, then += dz*dz), contracted by the same build as
// fma(dx, dx, dy*dy) and fma(dz, dz, that).
inline double rdist(double px, double py, double cx, double cy)
{
    const double dx = px - cx, dy = py - cy;
    return std::fma(dx, dx, dy * dy);
}
inline double rdist3(double px, double py, double pz, double cx, double cy, double cz)
{
    const double dz = pz - cz;
    return std::fma(dz, dz, rdist(px, py, cx, cy));
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
    // kReorder: the squared distance as reorderIndex evaluates it instead of
    // the k-means one.
    template <bool kReorder = false>
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
                double d;
                if constexpr (kReorder)
                    d = cz ? rdist3(px, py, pz, cx[c], cy[c], (*cz)[c]) : rdist(px, py, cx[c], cy[c]);
                else
                    d = cz ? kdist3(px, py, pz, cx[c], cy[c], (*cz)[c]) : kdist(px, py, cx[c], cy[c]);
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

// ------------------------------------------------------- centroid orderings
// The reference's --permutation choices (src/test_Xvecchia_batch.cpp:286-314),
// each rewriting the centroid coordinates in place in its order: random
// (include/ckernel.h:177-202, 3-D :811-840), Morton (:148-174, 3-D :842-868),
// kd-tree (:205-300, 3-D :725-935), Hilbert (:326-432, 3-D :582-705 and
// :870-895) and maximum-minimum distance (:435-523, 3-D :937-1000).  Morton
// and Hilbert leave the coordinates quantised to k / 65535, as there.

// 16-bit quantisation (uint16_t)(v * 65535 + .5), the product and the sum
// contracted into one fma by the reference's build.  Coordinates outside
// [0, 1] have no defined quantisation there; they are rejected here.
inline bool quant16(double v, uint16_t &q)
{
    if (!(v >= 0.0 && v <= 1.0)) return false;
    q = (uint16_t)std::fma(v, 65535.0, 0.5);
    return true;
}

// Bit b of v to bit 4b (Morton 3-D keys: x at 4b, y at 4b+1, z at 4b+2) and
// back; bit b to bit 3b (Hilbert 3-D keys) and back.
uint64_t spread16_by4(uint64_t v)
{
    uint64_t r = 0;
    for (int b = 0; b < 16; ++b) r |= ((v >> b) & 1ull) << (4 * b);
    return r;
}
uint64_t gather16_by4(uint64_t v)
{
    uint64_t r = 0;
    for (int b = 0; b < 16; ++b) r |= ((v >> (4 * b)) & 1ull) << b;
    return r;
}
uint64_t spread16_by3(uint64_t v)
{
    uint64_t r = 0;
    for (int b = 0; b < 16; ++b) r |= ((v >> b) & 1ull) << (3 * b);
    return r;
}
uint64_t gather16_by3(uint64_t v)
{
    uint64_t r = 0;
    for (int b = 0; b < 16; ++b) r |= ((v >> (3 * b)) & 1ull) << b;
    return r;
}

// The reference's Hilbert transforms, as its code computes them (they are
// not the textbook transform: in the first coordinate's step the branch
// without the bit swaps x with itself, i.e. does nothing, and the decoder
// below does not invert the encoder).  Keys interleave the transformed
// coordinates most significant bit first, x ahead of y (ahead of z).
uint32_t hilbert2_key(uint32_t x, uint32_t y)
{
    for (uint32_t q = 1u << 15; q > 1; q >>= 1) {
        const uint32_t p = q - 1;
        if (x & q) x ^= p;
        if (y & q) {
            x ^= p;
        } else {
            const uint32_t t = (x ^ y) & p;
            x ^= t;
            y ^= t;
        }
    }
    y ^= x;
    uint32_t t = 0;
    for (uint32_t q = 1u << 15; q > 1; q >>= 1)
        if (y & q) t ^= q - 1;
    x ^= t;
    y ^= t;
    return (spread16(x & 0xffffu) << 1) | spread16(y & 0xffffu);
}
void hilbert2_point(uint32_t key, uint16_t &ox, uint16_t &oy)
{
    uint32_t x = gather16(key >> 1), y = gather16(key);
    const uint32_t t0 = y >> 1;
    y ^= x;
    x ^= t0;
    for (uint32_t q = 2; q != (1u << 16); q <<= 1) {
        const uint32_t p = q - 1;
        if (y & q) {
            x ^= p;
        } else {
            const uint32_t t = (x ^ y) & p;
            x ^= t;
            y ^= t;
        }
        if (x & q) x ^= p;
    }
    ox = (uint16_t)x;
    oy = (uint16_t)y;
}
uint64_t hilbert3_key(uint64_t x, uint64_t y, uint64_t z)
{
    for (uint64_t q = 1u << 15; q > 1; q >>= 1) {
        const uint64_t p = q - 1;
        if (x & q) x ^= p;
        if (y & q) {
            x ^= p;
        } else {
            const uint64_t t = (x ^ y) & p;
            x ^= t;
            y ^= t;
        }
        if (z & q) {
            x ^= p;
        } else {
            const uint64_t t = (x ^ z) & p;
            x ^= t;
            z ^= t;
        }
    }
    y ^= x;
    z ^= y;
    uint64_t t = 0;
    for (uint64_t q = 1u << 15; q > 1; q >>= 1)
        if (z & q) t ^= q - 1;
    x ^= t;
    y ^= t;
    z ^= t;
    return (spread16_by3(x & 0xffffu) << 2) | (spread16_by3(y & 0xffffu) << 1) |
           spread16_by3(z & 0xffffu);
}
void hilbert3_point(uint64_t key, uint16_t &ox, uint16_t &oy, uint16_t &oz)
{
    uint64_t x = gather16_by3(key >> 2), y = gather16_by3(key >> 1), z = gather16_by3(key);
    const uint64_t t0 = z >> 1;
    z ^= y;
    y ^= x;
    x ^= t0;
    for (uint64_t q = 2; q != (1ull << 16); q <<= 1) {
        const uint64_t p = q - 1;
        if (z & q) {
            x ^= p;
        } else {
            const uint64_t t = (x ^ z) & p;
            x ^= t;
            z ^= t;
        }
        if (y & q) {
            x ^= p;
        } else {
            const uint64_t t = (x ^ y) & p;
            x ^= t;
            y ^= t;
        }
        if (x & q) x ^= p;
    }
    ox = (uint16_t)x;
    oy = (uint16_t)y;
    oz = (uint16_t)z;
}

// kd-tree order: sort by x (depth 0), split at len / 2, recurse on both
// halves with the next axis (y, then z in 3-D), and read the leaves left to
// right -- which is the array after the recursive sorts.  The sorts are
// glibc's qsort on records of the reference's shape (coordinates plus an
// unused weight), so that records with equal keys end in the same order.
struct KdRec2 {
    double x, y, w;
};
struct KdRec3 {
    double x, y, z, w;
};
template <typename R, int kAxis>
int kd_cmp(const void *a, const void *b)
{
    const double u = reinterpret_cast<const double *>(a)[kAxis];
    const double v = reinterpret_cast<const double *>(b)[kAxis];
    return u < v ? -1 : (u == v ? 0 : 1);
}
template <typename R, int kDims>
void kd_order(R *d, int len, int depth)
{
    if (len <= 1) return;
    const int axis = depth % kDims;
    qsort(d, (size_t)len, sizeof(R), axis == 0 ? kd_cmp<R, 0> : (axis == 1 ? kd_cmp<R, 1> : kd_cmp<R, 2>));
    const int mid = len / 2;
    kd_order<R, kDims>(d, mid, depth + 1);
    kd_order<R, kDims>(d + mid, len - mid, depth + 1);
}

// Maximum-minimum distance order: the centroid nearest the mean first (the
// first strictly below the cap), then repeatedly the one whose distance to
// the chosen set is largest (first strict maximum; distances capped at 2,
// 3 in 3-D), the last one remaining at the end.  The reference recomputes
// every minimum over the chosen set at each step (O(n^3)); the running
// minimum kept here takes the same values in O(n^2).  Squared distances as
// its pow(d, 2) sums compile: fma(dx, dx, dy*dy) (and fma(dz, dz, .)).
int mmd_order(int n, double *x, double *y, double *z)
{
    const double cap = z ? 3.0 : 2.0;
    double xm = 0, ym = 0, zm = 0;
    for (int i = 0; i < n; ++i) {
        xm = xm + x[i];
        ym = ym + y[i];
        if (z) zm = zm + z[i];
    }
    xm = xm / n;
    ym = ym / n;
    if (z) zm = zm / n;
    auto d2 = [&](double ax, double ay, double az, double bx, double by, double bz) {
        return z ? rdist3(ax, ay, az, bx, by, bz) : rdist(ax, ay, bx, by);
    };
    std::vector<int> res(n), flag(n, 0);
    double best = cap;
    int first = -1;
    for (int i = 0; i < n; ++i) {
        const double d = d2(x[i], y[i], z ? z[i] : 0.0, xm, ym, zm);
        if (d < best) {
            best = d;
            first = i;
        }
    }
    if (first < 0) return BV_E_INVALID;  // no centroid within the cap of the mean
    res[0] = first;
    flag[first] = 1;
    std::vector<double> mind(n, cap);
    for (int j = 1; j < n - 1; ++j) {
        const int r = res[j - 1];
        double mx = 0.0;
        int arg = n;
        for (int i = 0; i < n; ++i) {
            if (flag[i]) continue;
            const double d = d2(x[i], y[i], z ? z[i] : 0.0, x[r], y[r], z ? z[r] : 0.0);
            if (d < mind[i]) mind[i] = d;
            if (mx < mind[i]) {
                mx = mind[i];
                arg = i;
            }
        }
        if (arg == n) return BV_E_INVALID;  // the rest coincide with chosen centroids
        res[j] = arg;
        flag[arg] = 1;
    }
    if (n > 1)
        for (int i = 0; i < n; ++i)
            if (!flag[i]) res[n - 1] = i;
    std::vector<double> ox(n), oy(n), oz(z ? n : 0);
    for (int i = 0; i < n; ++i) {
        ox[i] = x[res[i]];
        oy[i] = y[res[i]];
        if (z) oz[i] = z[res[i]];
    }
    std::memcpy(x, ox.data(), sizeof(double) * n);
    std::memcpy(y, oy.data(), sizeof(double) * n);
    if (z) std::memcpy(z, oz.data(), sizeof(double) * n);
    return BV_OK;
}

// The ordering named by `ordering` (BV_ORDER_*), in place; z = NULL: 2-D.
int order_centroids(int ordering, int n, double *x, double *y, double *z)
{
    switch (ordering) {
    case BV_ORDER_RANDOM:
        srand(42);
        for (int i = n - 1; i > 0; --i) {
            const int j = rand() % (i + 1);
            std::swap(x[i], x[j]);
            std::swap(y[i], y[j]);
            if (z) std::swap(z[i], z[j]);
        }
        return BV_OK;
    case BV_ORDER_MORTON:
    case BV_ORDER_HILBERT: {
        const bool hil = ordering == BV_ORDER_HILBERT;
        std::vector<uint64_t> key(n);
        for (int i = 0; i < n; ++i) {
            uint16_t qx, qy, qz = 0;
            if (!quant16(x[i], qx) || !quant16(y[i], qy) || (z && !quant16(z[i], qz))) {
                bv::set_error("%s ordering: centroid %d lies outside the unit %s",
                              hil ? "Hilbert" : "Morton", i, z ? "cube" : "square");
                return BV_E_INVALID;
            }
            if (z)
                key[i] = hil ? hilbert3_key(qx, qy, qz)
                             : (spread16_by4(qz) << 2) + (spread16_by4(qy) << 1) + spread16_by4(qx);
            else
                key[i] = hil ? hilbert2_key(qx, qy) : (uint64_t)((spread16(qy) << 1) + spread16(qx));
        }
        // Equal keys decode to equal points: any sort gives the same arrays.
        std::sort(key.begin(), key.end());
        for (int i = 0; i < n; ++i) {
            uint16_t qx, qy, qz = 0;
            if (z && hil) {
                hilbert3_point(key[i], qx, qy, qz);
            } else if (z) {
                qx = (uint16_t)gather16_by4(key[i]);
                qy = (uint16_t)gather16_by4(key[i] >> 1);
                qz = (uint16_t)gather16_by4(key[i] >> 2);
            } else if (hil) {
                hilbert2_point((uint32_t)key[i], qx, qy);
            } else {
                qx = (uint16_t)gather16((uint32_t)key[i]);
                qy = (uint16_t)gather16((uint32_t)key[i] >> 1);
            }
            x[i] = (double)qx / (double)UINT16_MAX;
            y[i] = (double)qy / (double)UINT16_MAX;
            if (z) z[i] = (double)qz / (double)UINT16_MAX;
        }
        return BV_OK;
    }
    case BV_ORDER_KDTREE:
        if (z) {
            std::vector<KdRec3> d(n);
            for (int i = 0; i < n; ++i) d[i] = {x[i], y[i], z[i], 0.0};
            kd_order<KdRec3, 3>(d.data(), n, 0);
            for (int i = 0; i < n; ++i) {
                x[i] = d[i].x;
                y[i] = d[i].y;
                z[i] = d[i].z;
            }
        } else {
            std::vector<KdRec2> d(n);
            for (int i = 0; i < n; ++i) d[i] = {x[i], y[i], 0.0};
            kd_order<KdRec2, 2>(d.data(), n, 0);
            for (int i = 0; i < n; ++i) {
                x[i] = d[i].x;
                y[i] = d[i].y;
            }
        }
        return BV_OK;
    case BV_ORDER_MMD:
        if (mmd_order(n, x, y, z)) {
            bv::set_error("MMD ordering: no centroid within distance %s of the mean, or centroids "
                          "that coincide (the reference's loop has no defined result there)",
                          z ? "sqrt(3)" : "sqrt(2)");
            return BV_E_INVALID;
        }
        return BV_OK;
    default:
        bv::set_error("unknown centroid ordering %d", ordering);
        return BV_E_INVALID;
    }
}

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
                                     int cs, int ordering, int *batchNum, int *batchNumAccum, double *x_new,
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
    // The centroid ordering (random_reordering by default: srand(42),
    // Fisher-Yates from the end with rand() % (i+1)).
    std::vector<double> px(ccx, ccx + k), py(ccy, ccy + k), pz(k, 0.0);
    if (z) pz.assign(ccz, ccz + k);
    {
        const int rc = order_centroids(ordering, k, px.data(), py.data(), z ? pz.data() : nullptr);
        if (rc) return rc;
    }
    std::vector<int> perm(k);
    if (ordering != BV_ORDER_MORTON && ordering != BV_ORDER_HILBERT) {
        // reorderIndex (include/vecchia_helper_method.h:128-160) after an
        // ordering that permutes the centroids: index of the first original
        // centroid at zero distance = lowest index with the same coordinates.
        // Where several centroids coincide (clusters of duplicated locations)
        // the reference maps all of them to that lowest index and stops on the
        // repeated index; here the k-th reordered occurrence of a coordinate
        // pair maps to the k-th original with it, which is the same map
        // whenever the centroids are distinct and otherwise puts every point
        // in exactly one block.  Coordinates compared by value (-0 and +0 are
        // at zero distance).
        std::unordered_map<Key3, std::vector<int>, Key3Hash> first_at;
        first_at.reserve((size_t)k * 2);
        for (int j = 0; j < k; ++j)  // ascending j
            first_at[key3(ccx[j], ccy[j], z ? ccz[j] : 0.0, true)].push_back(j);
        std::unordered_map<Key3, int, Key3Hash> taken;
        for (int i = 0; i < k; ++i) {
            const Key3 key = key3(px[i], py[i], pz[i], true);
            perm[i] = first_at.at(key)[taken[key]++];
        }
    } else {
        // reorderIndex after a quantising ordering: the nearest original
        // centroid (lowest index among equal distances), which must be a
        // different one for every reordered centroid (:154-159).
        const std::vector<double> ox(ccx, ccx + k), oy(ccy, ccy + k);
        std::vector<double> oz;
        if (z) oz.assign(ccz, ccz + k);
        CentroidGrid grid;
        grid.build(ox, oy);
        std::vector<int> seen(k, -1);
        for (int i = 0; i < k; ++i) {
            perm[i] = grid.nearest<true>(px[i], py[i], ox, oy, pz[i], z ? &oz : nullptr);
            if (seen[perm[i]] >= 0) {
                bv::set_error("bv_layout_from_clusters: the %s ordering maps centroids %d and %d to "
                              "cluster %d (the reference stops here too)",
                              ordering == BV_ORDER_MORTON ? "Morton" : "Hilbert", seen[perm[i]], i,
                              perm[i]);
                return BV_E_INVALID;
            }
            seen[perm[i]] = i;
        }
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
                                     BV_ORDER_RANDOM, batchNum, batchNumAccum, x_new, y_new, nullptr, obs_new, cx,
                                     cy, nullptr, bc_out, first_cluster_count);
}

static int layout_build_impl(const double *x, const double *y, const double *z, const double *obs,
                             int n, int bc, int cs, int seed, int epochs, int threads, int ordering,
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
                                     z ? ccz.data() : nullptr, cs, ordering, batchNum, batchNumAccum, x_new,
                                     y_new, z_new, obs_new, cx, cy, cz, bc_out,
                                     first_cluster_count);
}

extern "C" int bv_layout_build(const double *x, const double *y, const double *obs, int n, int bc,
                               int cs, int seed, int epochs, int threads, int *batchNum,
                               int *batchNumAccum, double *x_new, double *y_new, double *obs_new,
                               double *cx, double *cy, int *bc_out, int *first_cluster_count)
{
    return layout_build_impl(x, y, nullptr, obs, n, bc, cs, seed, epochs, threads, BV_ORDER_RANDOM,
                             batchNum,
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
    return layout_build_impl(x, y, z, obs, n, bc, cs, seed, epochs, threads, BV_ORDER_RANDOM,
                             batchNum,
                             batchNumAccum, x_new, y_new, z_new, obs_new, cx, cy, cz, bc_out,
                             first_cluster_count);
}

extern "C" int bv_layout_build_ex(const double *x, const double *y, const double *z,
                                  const double *obs, int n, int bc, int cs, int seed, int epochs,
                                  int threads, int ordering, int *batchNum, int *batchNumAccum,
                                  double *x_new, double *y_new, double *z_new, double *obs_new,
                                  double *cx, double *cy, double *cz, int *bc_out,
                                  int *first_cluster_count)
{
    if (z && (!z_new || !cz)) {
        bv::set_error("bv_layout_build_ex: z needs z_new and cz");
        return BV_E_INVALID;
    }
    return layout_build_impl(x, y, z, obs, n, bc, cs, seed, epochs, threads, ordering, batchNum,
                             batchNumAccum, x_new, y_new, z_new, obs_new, cx, cy, cz, bc_out,
                             first_cluster_count);
}

extern "C" int bv_layout_from_clusters_ex(const double *x, const double *y, const double *z,
                                          const double *obs, int n, int k, const int *labels,
                                          const double *ccx, const double *ccy, const double *ccz,
                                          int cs, int ordering, int *batchNum, int *batchNumAccum,
                                          double *x_new, double *y_new, double *z_new,
                                          double *obs_new, double *cx, double *cy, double *cz,
                                          int *bc_out, int *first_cluster_count)
{
    return layout_from_clusters_impl(x, y, z, obs, n, k, labels, ccx, ccy, ccz, cs, ordering,
                                     batchNum, batchNumAccum, x_new, y_new, z_new, obs_new, cx, cy,
                                     cz, bc_out, first_cluster_count);
}

extern "C" int bv_order_centroids(int ordering, int n, double *x, double *y, double *z)
{
    if (n <= 0 || !x || !y) {
        bv::set_error("bv_order_centroids: invalid argument");
        return BV_E_INVALID;
    }
    return order_centroids(ordering, n, x, y, z);
}

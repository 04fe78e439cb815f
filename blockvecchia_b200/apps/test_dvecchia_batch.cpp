// test_dvecchia_batch -- command-line driver with the reference's flags
// (src/test_Xvecchia_batch.cpp, include/vecchia_helper_data.h:256-739) over
// libbv_b200.so.
//
// Flags kept: --kernel --ikernel --kernel_init --vecchia_cs --vecchia_bc
// --num_loc --knn --perf --seed --xy_path --obs_path --tol --maxiter
// --omp_threads --permutation --dist_scale --lower_bound --upper_bound
// --earth --t_slots --3D.
// --perf evaluates once at --ikernel with zero observations on GenerateXYLoc
// locations and writes the blocks' points and conditioning points to
// ./log/points_<Ordering>.csv and ./log/neighbors_<Ordering>.csv; otherwise the
// locations/observations CSVs are fitted from --kernel_init.  The objective
// is bv_llh (the NLopt signature of llh_Xvecchia_batch); NLopt BOBYQA is used
// when <nlopt.h> exists at build time, else a bounded Nelder-Mead (Nelder &
// Mead, Comput. J. 7 (1965) 308-313) with the same stopping rule (relative
// change of the parameters below --tol, at most --maxiter evaluations).  Additional flags:
// --precision fp64|mixed, --device N, --print-opts (print the parsed options
// as JSON and exit; needs no GPU).
#include <sys/stat.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <limits>
#include <sstream>
#include <string>
#include <vector>

#include "bv.h"

#if defined(__has_include)
#if __has_include(<nlopt.h>)
#include <nlopt.h>
#define BV_HAVE_NLOPT 1
#endif
#endif

namespace {

struct Opts {
    int kernel = 1, num_params = 3, num_loc = 2000;
    double sigma = 1.0, beta = 0.1, nu = 0.5, nugget = 0.0, dist_scale = 1.0;
    double sigma_init = 0.01, beta_init = 0.01, nu_init = 0.01, nugget_init = 0.01;
    // space-time (include/vecchia_helper_data.h:293-302)
    double beta_time = 2.2, nu_time = 0.5, sep = 0.5, aux = 0.0;
    double beta_time_init = 0.01, nu_time_init = 0.01, sep_init = 0.01;
    int time_flag = 0, t_slots = 0, use_nugget = 0, earth = 0;
    int knn = 1, seed = 0, perf = 0, vecchia_cs = 100, vecchia_bc = 200, maxiter = 1000;
    double tol = 1e-5, lower_bound = 0.01, upper_bound = 3.0;
    int omp_threads = 40, device = 0, precision = BV_PREC_FP64, mixed_fp32 = 0, print_opts = 0;
    std::string xy_path, obs_path, permutation = "random";
    int ordering = BV_ORDER_RANDOM;
};

// --permutation names (include/vecchia_helper_data.h:456-476) and the
// perf-mode dump suffixes (src/test_Xvecchia_batch.cpp:409-435).
struct OrderName {
    const char *flag, *dump;
    int ordering;
};
const OrderName kOrders[] = {{"random", "Random", BV_ORDER_RANDOM},
                             {"morton", "Morton", BV_ORDER_MORTON},
                             {"kdtree", "KDtree", BV_ORDER_KDTREE},
                             {"hilbert", "Hilbert", BV_ORDER_HILBERT},
                             {"mmd", "MMD", BV_ORDER_MMD}};

[[noreturn]] void die(const char *msg, const char *arg = "")
{
    fprintf(stderr, "error: %s%s\n", msg, arg);
    exit(1);
}

// "a:b:c[:d[:e:f]]" with "?" keeping the current value
// (include/vecchia_helper_data.h:533-577): the fourth value is the nugget,
// and with six values the fourth to sixth are the space-time range,
// smoothness and separability.
void parse_theta(const char *s, double *a, double *b, double *c, double *d, double *bt, double *nt,
                 double *sp)
{
    std::vector<std::string> parts;
    std::stringstream ss(s);
    std::string tok;
    while (std::getline(ss, tok, ':')) parts.push_back(tok);
    double *dst[4] = {a, b, c, d};
    for (size_t i = 0; i < parts.size() && i < 4; ++i)
        if (parts[i] != "?") *dst[i] = atof(parts[i].c_str());
    if (parts.size() == 6) {
        double *st[3] = {bt, nt, sp};
        for (size_t i = 3; i < 6; ++i)
            if (parts[i] != "?") *st[i - 3] = atof(parts[i].c_str());
    }
}

Opts parse(int argc, char **argv)
{
    Opts o;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        const bool has = i + 1 < argc;
        auto next = [&]() -> const char * { return argv[++i]; };
        if (a == "--help" || a == "-h") {
            printf("Usage: test_dvecchia_batch [--kernel K] [--ikernel s2:range:nu[:nugget]] [--kernel_init ...]\n"
                   "  [--vecchia_cs N] [--vecchia_bc N] [--num_loc N] [--knn x] [--perf x] [--seed N]\n"
                   "  [--xy_path F] [--obs_path F] [--tol k (1e-k)] [--maxiter N] [--omp_threads N]\n"
                   "  [--permutation random|morton|kdtree|hilbert|mmd] [--dist_scale d] [--lower_bound b] [--upper_bound b]\n"
                   "  [--t_slots N] [--3D x] [--use_nugget 0|1]\n"
                   "  [--precision fp64|mixed|mixed_fp32] [--device N] [--print-opts]\n"
                   "  space-time: --kernel univariate_matern_spacetime_stationary\n"
                   "              --ikernel s2:range:nu:range_t:nu_t:sep\n");
            exit(0);
        } else if (a == "--xy_path" && has) {
            o.xy_path = next();
        } else if (a == "--obs_path" && has) {
            o.obs_path = next();
        } else if (a == "--num_loc" && has) {
            o.num_loc = atoi(next());
            if (o.num_loc <= 0) die("--num_loc must be positive");
        } else if (a == "--dist_scale" && has) {
            o.dist_scale = atof(next());
            if (!(o.dist_scale > 0)) die("--dist_scale must be > 0");
        } else if (a == "--vecchia_cs" && has) {
            o.vecchia_cs = atoi(next());
            if (o.vecchia_cs < 0) die("--vecchia_cs must be >= 0");
        } else if (a == "--vecchia_bc" && has) {
            o.vecchia_bc = atoi(next());
            if (o.vecchia_bc <= 0) die("--vecchia_bc must be > 0");
        } else if (a == "--perf" && has) {
            ++i;  // the reference requires (and ignores) an argument
            o.perf = 1;
            o.maxiter = 1;
        } else if (a == "--knn" && has) {
            ++i;
            o.knn = 1;
        } else if (a == "--kernel" && has) {
            const std::string k = next();
            if (k == "univariate_matern_stationary_no_nugget") {
                o.kernel = 1;
                o.num_params = 3;
            } else if (k == "univariate_powexp_stationary_no_nugget") {
                o.kernel = 2;  // evaluated as Matern by the likelihood, as in the reference
                o.num_params = 3;
            } else if (k == "univariate_powexp_nugget_stationary") {
                o.kernel = 3;
                o.num_params = 4;
            } else if (k == "univariate_matern_spacetime_stationary") {
                o.kernel = 4;
                o.num_params = 7;
                o.time_flag = 1;
            } else {
                die("unsupported kernel: ", k.c_str());
            }
        } else if (a == "--ikernel" && has) {
            parse_theta(next(), &o.sigma, &o.beta, &o.nu, &o.nugget, &o.beta_time, &o.nu_time, &o.sep);
        } else if (a == "--kernel_init" && has) {
            parse_theta(next(), &o.sigma_init, &o.beta_init, &o.nu_init, &o.nugget_init,
                        &o.beta_time_init, &o.nu_time_init, &o.sep_init);
        } else if (a == "--seed" && has) {
            o.seed = atoi(next());
        } else if (a == "--omp_threads" && has) {
            o.omp_threads = atoi(next());
        } else if (a == "--maxiter" && has) {
            o.maxiter = atoi(next());
            if (o.maxiter <= 0) die("--maxiter must be > 0");
        } else if (a == "--tol" && has) {
            const int t = atoi(next());
            if (t <= 0) die("--tol must be > 0 (k for 1e-k)");
            o.tol = std::pow(10.0, -t);
        } else if (a == "--lower_bound" && has) {
            o.lower_bound = atof(next());
            if (!(o.lower_bound > 0)) die("--lower_bound must be > 0");
        } else if (a == "--upper_bound" && has) {
            o.upper_bound = atof(next());
            if (!(o.upper_bound < 100)) die("--upper_bound must be < 100");
        } else if (a == "--permutation" && has) {
            o.permutation = next();
            o.ordering = -1;
            for (const auto &k : kOrders)
                if (o.permutation == k.flag) o.ordering = k.ordering;
            // The reference prints "Other ordering is being developed." and stops.
            if (o.ordering < 0) die("unknown --permutation (random, morton, kdtree, hilbert, mmd): ",
                                    o.permutation.c_str());
        } else if (a == "--precision" && has) {
            const std::string p = next();
            // mixed: FP64 throughout unless forced (bv_opts.mixed_fp32);
            // mixed_fp32: the FP32 pass wherever its probe accepts blocks.
            o.precision = (p == "mixed" || p == "mixed_fp32") ? BV_PREC_MIXED : BV_PREC_FP64;
            o.mixed_fp32 = (p == "mixed_fp32") ? 1 : 0;
        } else if (a == "--device" && has) {
            o.device = atoi(next());
        } else if (a == "--print-opts") {
            o.print_opts = 1;
        } else if (a == "--t_slots" && has) {
            o.t_slots = atoi(next());
            if (o.t_slots < 0) die("--t_slots must be >= 0");
        } else if (a == "--3D" && has) {
            ++i;  // include/vecchia_helper_data.h:445-449: 3-D spatial locations
            o.time_flag = 1;
            o.t_slots = 0;
        } else if (a == "--use_nugget" && has) {
            // Not in the reference (its likelihood never reads the nugget):
            // the nugget (fourth --ikernel value) enters the covariance.
            o.use_nugget = atoi(next()) != 0;
        } else if (a == "--earth" && has) {
            // include/vecchia_helper_data.h:451-454: a flag that needs a
            // following argument but does not consume it.
            o.earth = 1;
        } else {
            die("unknown or incomplete option: ", a.c_str());
        }
    }
    // src/test_Xvecchia_batch.cpp:107-111
    if (o.time_flag && o.t_slots != 0 && o.num_loc % o.t_slots != 0)
        die("Your number of locations cannot be divided by t_slot!");
    // src/ckernel.cpp:170-172 (the reference stops at the first covariance).
    if (o.earth && o.time_flag) die("Great Circle (GC) distance is only valid for 2d");
    return o;
}

void print_opts(const Opts &o)
{
    printf("{\"kernel\": %d, \"num_params\": %d, \"num_loc\": %d, \"sigma\": %.17g, \"beta\": %.17g, "
           "\"nu\": %.17g, \"sigma_init\": %.17g, \"beta_init\": %.17g, \"nu_init\": %.17g, "
           "\"vecchia_cs\": %d, \"vecchia_bc\": %d, \"knn\": %d, \"perf\": %d, \"seed\": %d, "
           "\"tol\": %.17g, \"maxiter\": %d, \"lower_bound\": %.17g, \"upper_bound\": %.17g, "
           "\"dist_scale\": %.17g, \"omp_threads\": %d, \"precision\": %d, \"xy_path\": \"%s\", "
           "\"obs_path\": \"%s\", \"time_flag\": %d, \"t_slots\": %d, \"beta_time\": %.17g, "
           "\"nu_time\": %.17g, \"sep\": %.17g, \"nugget\": %.17g, \"use_nugget\": %d, "
           "\"permutation\": \"%s\", \"ordering\": %d, \"earth\": %d, \"mixed_fp32\": %d}\n",
           o.kernel, o.num_params, o.num_loc, o.sigma, o.beta, o.nu, o.sigma_init, o.beta_init,
           o.nu_init, o.vecchia_cs, o.vecchia_bc, o.knn, o.perf, o.seed, o.tol, o.maxiter,
           o.lower_bound, o.upper_bound, o.dist_scale, o.omp_threads, o.precision,
           o.xy_path.c_str(), o.obs_path.c_str(), o.time_flag, o.t_slots, o.beta_time, o.nu_time, o.sep,
           o.nugget, o.use_nugget, o.permutation.c_str(), o.ordering, o.earth, o.mixed_fp32);
}

// include/utils.h:27-87: "x,y" per line ("x,y,z" with time_flag); one
// observation per line.
void load_xy(const std::string &path, int n, std::vector<double> &x, std::vector<double> &y,
             std::vector<double> *z)
{
    std::ifstream f(path);
    if (!f) die("cannot open ", path.c_str());
    x.assign(n, 0.0);
    y.assign(n, 0.0);
    if (z) z->assign(n, 0.0);
    std::string line;
    int i = 0;
    while (i < n && std::getline(f, line)) {
        std::stringstream ss(line);
        std::string t;
        if (!std::getline(ss, t, ',')) continue;
        x[i] = std::stod(t);
        if (!std::getline(ss, t, ',')) die("malformed line in ", path.c_str());
        y[i] = std::stod(t);
        if (z) {
            if (!std::getline(ss, t, ',')) die("missing third coordinate in ", path.c_str());
            (*z)[i] = std::stod(t);
        }
        ++i;
    }
    if (i < n) die("too few locations in ", path.c_str());
}

void load_obs(const std::string &path, int n, std::vector<double> &z)
{
    std::ifstream f(path);
    if (!f) die("cannot open ", path.c_str());
    z.assign(n, 0.0);
    std::string line;
    int i = 0;
    while (i < n && std::getline(f, line)) {
        std::istringstream ss(line);
        double v;
        if (ss >> v) z[i++] = v;
    }
    if (i < n) die("too few observations in ", path.c_str());
}

// Bounded Nelder-Mead maximisation of f on [lb, ub]^d; points are clipped to
// the box.  Stops when every simplex vertex is within tol (relative) of the
// best one in every coordinate, or after maxeval evaluations.
double nelder_mead_max(double (*f)(unsigned, const double *, double *, void *), void *data, int d,
                       std::vector<double> &x, const std::vector<double> &lbv,
                       const std::vector<double> &ubv, double tol, int maxeval, int *evals)
{
    auto clip = [&](std::vector<double> &v) {
        for (int i = 0; i < d; ++i) v[i] = std::min(ubv[i], std::max(lbv[i], v[i]));
    };
    int ne = 0;
    auto F = [&](std::vector<double> &v) {
        clip(v);
        ++ne;
        const double r = f((unsigned)d, v.data(), nullptr, data);
        return std::isfinite(r) ? r : -std::numeric_limits<double>::infinity();
    };
    std::vector<std::vector<double>> s(d + 1, x);
    std::vector<double> fv(d + 1, -std::numeric_limits<double>::infinity());  // unevaluated vertices never win
    clip(s[0]);
    fv[0] = F(s[0]);
    for (int i = 0; i < d && ne < maxeval; ++i) {
        s[i + 1] = s[0];
        double step = 0.1 * (ubv[i] - lbv[i]);  // 0 for a fixed coordinate
        if (s[0][i] + step > ubv[i]) step = -step;
        s[i + 1][i] += step;
        fv[i + 1] = F(s[i + 1]);
    }
    while (ne < maxeval) {
        std::vector<int> idx(d + 1);
        for (int i = 0; i <= d; ++i) idx[i] = i;
        std::sort(idx.begin(), idx.end(), [&](int a, int b) { return fv[a] > fv[b]; });
        std::vector<std::vector<double>> s2(d + 1);
        std::vector<double> f2(d + 1);
        for (int i = 0; i <= d; ++i) {
            s2[i] = s[idx[i]];
            f2[i] = fv[idx[i]];
        }
        s.swap(s2);
        fv.swap(f2);
        double spread = 0.0;
        for (int i = 1; i <= d; ++i)
            for (int j = 0; j < d; ++j)
                spread = std::max(spread, std::fabs(s[i][j] - s[0][j]) / std::max(std::fabs(s[0][j]), 1e-12));
        if (spread <= tol) break;
        std::vector<double> c(d, 0.0);
        for (int i = 0; i < d; ++i)
            for (int j = 0; j < d; ++j) c[j] += s[i][j] / d;
        auto along = [&](double t) {
            std::vector<double> v(d);
            for (int j = 0; j < d; ++j) v[j] = c[j] + t * (s[d][j] - c[j]);
            return v;
        };
        std::vector<double> xr = along(-1.0);
        const double fr = F(xr);
        if (fr > fv[0]) {
            std::vector<double> xe = along(-2.0);
            const double fe = ne < maxeval ? F(xe) : -INFINITY;
            if (fe > fr) {
                s[d] = xe;
                fv[d] = fe;
            } else {
                s[d] = xr;
                fv[d] = fr;
            }
        } else if (fr > fv[d - 1]) {
            s[d] = xr;
            fv[d] = fr;
        } else {
            const bool outside = fr > fv[d];
            std::vector<double> xc = along(outside ? -0.5 : 0.5);
            const double fc = ne < maxeval ? F(xc) : -INFINITY;
            if (fc > (outside ? fr : fv[d])) {
                s[d] = xc;
                fv[d] = fc;
            } else {
                for (int i = 1; i <= d && ne < maxeval; ++i) {
                    for (int j = 0; j < d; ++j) s[i][j] = s[0][j] + 0.5 * (s[i][j] - s[0][j]);
                    fv[i] = F(s[i]);
                }
            }
        }
    }
    int best = 0;
    for (int i = 1; i <= d; ++i)
        if (fv[i] > fv[best]) best = i;
    x = s[best];
    *evals = ne;
    return fv[best];
}

}  // namespace

int main(int argc, char **argv)
{
    Opts o = parse(argc, argv);
    if (o.print_opts) {
        print_opts(o);
        return 0;
    }
    const int n = o.num_loc;
    const bool tf = o.time_flag != 0;
    // src/test_Xvecchia_batch.cpp:206-209: distance_metric = 1 is set for
    // locations read from files only (not for the synthetic --perf locations).
    const int earth = (o.earth && !o.perf) ? 1 : 0;
    std::vector<double> x, y, t3, z;  // t3: third coordinate (time_flag), z: observations
    // Parameter vector: the kernel's (3, or 7 for space-time), then the
    // nugget when --use_nugget (src/test_Xvecchia_batch.cpp:156-235).
    const int np = o.num_params == 7 ? 7 : 3;
    const int d = np + (o.use_nugget ? 1 : 0);
    std::vector<double> theta(d, 0.0);
    auto fill = [&](double s2, double b, double nu, double nug, double bt, double nt, double sp, double ax) {
        theta[0] = s2;
        theta[1] = b;
        theta[2] = nu;
        if (np == 7) {
            theta[3] = bt;
            theta[4] = nt;
            theta[5] = sp;
            theta[6] = ax;
        }
        if (o.use_nugget) theta[np] = nug;
    };
    if (o.perf) {
        x.resize(n);
        y.resize(n);
        if (tf) {
            if (o.t_slots <= 0) die("--perf with time_flag needs --t_slots > 0");
            t3.resize(n);
            if (bv_generate_xyt(n / o.t_slots, o.t_slots, o.seed, x.data(), y.data(), t3.data()))
                die(bv_last_error());
        } else if (bv_generate_xy(n, o.seed, x.data(), y.data())) {
            die(bv_last_error());
        }
        z.assign(n, 0.0);  // src/test_Xvecchia_batch.cpp:151-152
        fill(o.sigma, o.beta, o.nu, o.nugget, o.beta_time, o.nu_time, o.sep, o.aux);
    } else {
        if (o.xy_path.empty() || o.obs_path.empty())
            die("--xy_path and --obs_path are required unless --perf is given");
        load_xy(o.xy_path, n, x, y, tf ? &t3 : nullptr);
        load_obs(o.obs_path, n, z);
        // The auxiliary space-time parameter starts at 0 and is not optimised.
        fill(o.sigma_init, o.beta_init, o.nu_init, o.nugget_init, o.beta_time_init, o.nu_time_init,
             o.sep_init, 0.0);
    }
    fprintf(stderr, n < 2 * o.vecchia_bc ? "You are using the classic Vecchia!\n"
                                         : "You are using the cluster Vecchia!\n");
    const int k = (n < 2 * o.vecchia_bc) ? n : o.vecchia_bc;
    std::vector<int> bn(k), acc(k + 1);
    std::vector<double> xn(n), yn(n), zn(n), cx(k), cy(k), tn(tf ? n : 0), ct(tf ? k : 0);
    int bc = 0, fcc = 0;
    const int lrc = bv_layout_build_ex(x.data(), y.data(), tf ? t3.data() : nullptr, z.data(), n,
                                       o.vecchia_bc, o.vecchia_cs, o.seed, 50, o.omp_threads,
                                       o.ordering, bn.data(), acc.data(), xn.data(), yn.data(),
                                       tf ? tn.data() : nullptr, zn.data(), cx.data(), cy.data(),
                                       tf ? ct.data() : nullptr, &bc, &fcc);
    if (lrc) die(bv_last_error());
    fprintf(stderr, "--------------Clustering Done-----------------\n");
    const int cs = o.vecchia_cs;
    std::vector<int> knn((size_t)bc * cs);
    if (cs > 0) {
        if (o.knn) {
            const int krc = bv_knn_ex(xn.data(), yn.data(), tf ? tn.data() : nullptr, n, bc, cs,
                                      acc.data(), cx.data(), cy.data(), tf ? ct.data() : nullptr,
                                      nullptr, earth ? BV_METRIC_EARTH : BV_METRIC_EUCLIDEAN,
                                      knn.data(), o.device);
            if (krc) die(bv_last_error());
        } else {
            // src/test_Xvecchia_batch.cpp:391-404: the cs points before each block.
            for (int t = 0; t < cs; ++t) knn[t] = t;
            for (int i = 1; i < bc; ++i)
                for (int t = 0; t < cs; ++t) knn[(size_t)i * cs + t] = acc[i] - cs + t;
        }
    }
    if (o.perf) {
        // src/test_Xvecchia_batch.cpp:405-451: every block's points with the
        // block's index, then every block's cs conditioning points with the
        // block's index (block 0's are the first cs points, as the reference
        // fills them at :359-361); file names carry the ordering.
        mkdir("./log", 0755);
        std::string suffix = "Random";
        for (const auto &k : kOrders)
            if (k.ordering == o.ordering) suffix = k.dump;
        std::ofstream pts("./log/points_" + suffix + ".csv");
        pts << "x,y,cluster\n";
        for (int i = 0; i < bc; ++i)
            for (int j = 0; j < bn[i]; ++j) pts << xn[acc[i] + j] << "," << yn[acc[i] + j] << "," << i << "\n";
        std::ofstream nbr("./log/neighbors_" + suffix + ".csv");
        nbr << "x,y,cluster\n";
        for (size_t t = 0; t < (size_t)bc * cs; ++t) {
            const int src = (t < (size_t)cs) ? (int)t : knn[t];
            if (src < 0 || src >= n) continue;  // "previous cs points" before an early block
            nbr << xn[src] << "," << yn[src] << "," << t / cs << "\n";
        }
    }
    fprintf(stderr, "--------------Nearest Neighbor Done-----------------\n");
    bv_layout L = {n, bc, cs, bn.data(), acc.data(), xn.data(), yn.data(), zn.data(), knn.data(),
                   cx.data(), cy.data(), tf ? tn.data() : nullptr, tf ? ct.data() : nullptr};
    bv_opts bo;
    bv_default_opts(&bo);
    bo.kernel = o.kernel;
    bo.nugget = o.use_nugget;
    bo.earth = earth;
    bo.dist_scale = o.dist_scale;
    bo.device = o.device;
    bo.precision = o.precision;
    bo.mixed_fp32 = o.mixed_fp32;
    bo.print_iter = o.perf ? 0 : 1;
    bv_handle *h = nullptr;
    if (bv_create(&L, &bo, &h)) die(bv_last_error());

    const auto t0 = std::chrono::steady_clock::now();
    double maxf = -HUGE_VAL;
    int evals = 0;
    bool ok = true;
    // Bounds (src/test_Xvecchia_batch.cpp:707-720): [lower, upper] for every
    // parameter; the space-time kernel's time smoothness and separability
    // are at most 1 and its auxiliary parameter is held at 0.
    std::vector<double> lb(d, o.lower_bound), ub(d, o.upper_bound);
    if (np == 7) {
        ub[4] = 1.0;
        ub[5] = 1.0;
        lb[6] = 0.0;
        ub[6] = 0.0;
    }
#ifdef BV_HAVE_NLOPT
    nlopt_opt opt = nlopt_create(NLOPT_LN_BOBYQA, d);
    nlopt_set_max_objective(opt, bv_llh, h);
    nlopt_set_lower_bounds(opt, lb.data());
    nlopt_set_upper_bounds(opt, ub.data());
    nlopt_set_xtol_rel(opt, o.tol);
    nlopt_set_maxeval(opt, o.maxiter);
    ok = nlopt_optimize(opt, theta.data(), &maxf) >= 0;
    nlopt_destroy(opt);
    evals = bv_iterations(h);
#else
    maxf = nelder_mead_max(bv_llh, h, d, theta, lb, ub, o.tol, o.maxiter, &evals);
#endif
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    // src/test_Xvecchia_batch.cpp:733-753 and include/utils.h:155-190.
    if (!ok)
        printf("nlopt failed!\n");
    else if (np == 7)
        printf("Found maximum at f(%g, %g, %g, %g, %g, %g) = %0.10g\n", theta[0], theta[1], theta[2],
               theta[3], theta[4], theta[5], maxf);
    else if (d == 4)
        printf("Found maximum at f(%g, %g, %g, %g) = %0.10g\n", theta[0], theta[1], theta[2], theta[3],
               maxf);
    else
        printf("Found maximum at f(%g, %g, %g) = %0.10g\n", theta[0], theta[1], theta[2], maxf);
    printf("Total Number of Iterations = %d \n", bv_iterations(h));
    printf("Total Optimization Time = %lf secs \n", secs);
    mkdir("./log", 0755);
    char path[512];
    snprintf(path, sizeof(path), "./log/locs_%d_cs_%d_bc_%d_seed_%d_kernel_%f:%f:%f_random", n, cs,
             o.vecchia_bc, o.seed, o.sigma, o.beta, o.nu);
    if (np == 3 && d == 3) {
        printf("Model Parameters (Variance, range, smoothness): (%.8f, %.8f, %.8f) -> Loglik: %.18f \n",
               theta[0], theta[1], theta[2], maxf);
        std::ofstream out(path);
        out << "Iterations, variance, range, smoothness, log-likelihood, time " << std::endl;
        out << bv_iterations(h) << ", " << theta[0] << ", " << theta[1] << ", " << theta[2] << ", "
            << std::setprecision(std::numeric_limits<double>::max_digits10) << maxf << ", " << secs
            << std::endl;
    } else if (np == 3) {
        printf("Model Parameters (Variance, range, smoothness, nugget): (%.8f, %.8f, %.8f, %.8f) -> "
               "Loglik: %.18f \n",
               theta[0], theta[1], theta[2], theta[3], maxf);
        std::ofstream out(path);
        out << "Iterations, variance, range, smoothness, nugget, log-likelihood, time " << std::endl;
        out << bv_iterations(h) << ", " << theta[0] << ", " << theta[1] << ", " << theta[2] << ", "
            << theta[3] << ", " << std::setprecision(std::numeric_limits<double>::max_digits10) << maxf
            << ", " << secs << std::endl;
    }
    bv_status st;
    bv_get_status(h, &st);
    if (st.cond_fail + st.schur_fail)
        fprintf(stderr, "note: %d blocks met a non-positive pivot in the last evaluation\n",
                st.cond_fail + st.schur_fail);
    bv_destroy(h);
    fprintf(stderr, "Done! \n");
    (void)evals;
    return 0;
}

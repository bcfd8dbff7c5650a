// host_grid.cpp -- transformed Gauss-Legendre imaginary-frequency grid (host, FP64).
//
// Same algorithm and operation order as the reference (src/gw/frequency_grids.cpp:12-93):
// Gauss-Legendre nodes by Newton iteration on the Legendre recurrence (eps 3e-14, <= 100
// iterations), the map w = (1+y)/(2(1-y)) with weight w_y/(1-y)^2, an ascending sort, and the
// clamp w_0 >= 1e-12.  Compiled with -ffp-contract=off so the nodes round like the reference.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <numeric>
#include <vector>

#include "internal.cuh"

namespace gwb200 {

namespace {

constexpr double kPi = 3.141592653589793238462643383279502884;

void gauss_legendre(double x1, double x2, int64_t n, std::vector<double>& x, std::vector<double>& w) {
    x.assign(static_cast<size_t>(n), 0.0);
    w.assign(static_cast<size_t>(n), 0.0);
    const double eps = 3e-14;
    const int64_t half = (n + 1) / 2;
    const double xm = 0.5 * (x2 + x1);
    const double xl = 0.5 * (x2 - x1);
    for (int64_t i = 0; i < half; ++i) {
        double z = std::cos(kPi * (static_cast<double>(i + 1) - 0.25) / (static_cast<double>(n) + 0.5));
        double dp = 0.0;
        for (int iter = 0; iter < 100; ++iter) {
            double p1 = 1.0, p2 = 0.0;
            for (int64_t j = 1; j <= n; ++j) {
                const double p3 = p2;
                p2 = p1;
                p1 = ((2.0 * static_cast<double>(j) - 1.0) * z * p2 - (static_cast<double>(j) - 1.0) * p3) /
                     static_cast<double>(j);
            }
            dp = static_cast<double>(n) * (z * p1 - p2) / (z * z - 1.0);
            const double z_prev = z;
            z = z_prev - p1 / dp;
            if (std::abs(z - z_prev) <= eps) break;
        }
        x[static_cast<size_t>(i)] = xm - xl * z;
        x[static_cast<size_t>(n - 1 - i)] = xm + xl * z;
        w[static_cast<size_t>(i)] = 2.0 * xl / ((1.0 - z * z) * dp * dp);
        w[static_cast<size_t>(n - 1 - i)] = w[static_cast<size_t>(i)];
    }
}

} // namespace

void transformed_legendre_grid(int64_t n, double* omega, double* weight) {
    if (n <= 0) fail(GWB200_BAD_SHAPE, "nfreq must be positive");
    std::vector<double> y, wy;
    gauss_legendre(-1.0, 1.0, n, y, wy);
    std::vector<double> tv(static_cast<size_t>(n)), tw(static_cast<size_t>(n));
    for (size_t i = 0; i < tv.size(); ++i) {
        tv[i] = 0.5 * (1.0 + y[i]) / (1.0 - y[i]);
        tw[i] = wy[i] / ((1.0 - y[i]) * (1.0 - y[i]));
    }
    std::vector<size_t> order(tv.size());
    std::iota(order.begin(), order.end(), size_t{0});
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return tv[a] < tv[b]; });
    for (size_t i = 0; i < order.size(); ++i) {
        omega[i] = tv[order[i]];
        weight[i] = tw[order[i]];
    }
    if (omega[0] < 1e-12) omega[0] = 1e-12;
}

} // namespace gwb200

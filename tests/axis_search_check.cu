// Host check of the bucket-guided EOS axis search (test infrastructure, built by
// tests/test_axis_search.py with nvcc and run on the CPU; axis_search and bisearch are host and
// device functions): on random axes of every kind the tables meet (evenly and log spaced,
// jittered, with plateaus of equal values, tiny and huge scales), for queries at every node,
// next to it, between nodes, outside the axis, at +-inf and NaN, axis_search returns exactly
// the bisection's index; axes that are not non-decreasing get no table.
#include "salec_device.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <limits>
#include <random>
#include <vector>

using namespace salec;

int main()
{
    std::mt19937_64 rng(7);
    std::uniform_real_distribution<double> U(0.0, 1.0);
    long checks = 0, tables = 0;
    const double inf = std::numeric_limits<double>::infinity(), nan = std::numeric_limits<double>::quiet_NaN();
    for (int trial = 0; trial < 4000; ++trial) {
        const int n = 3 + (int)(rng() % 700);
        std::vector<double> xs(n);
        const int kind = trial % 6;
        for (int k = 0; k < n; ++k) {
            const double u = (double)k / (n - 1);
            switch (kind) {
            case 0: xs[k] = 1.0e3 * u * (1.0 + 0.2 * (U(rng) - 0.5) / n); break;        // jittered, like the table
            case 1: xs[k] = 1.0e-2 * std::pow(1.0e7, u); break;                           // log spaced
            case 2: xs[k] = std::floor(u * 17.0) * 3.0; break;                            // plateaus
            case 3: xs[k] = U(rng) * 5.0e4; break;                                        // random, sorted below
            case 4: xs[k] = 1.0e-300 * (1.0 + u); break;                                  // tiny scale
            default: xs[k] = -1.0e300 + 2.0e300 * u; break;                               // huge scale
            }
        }
        if (kind == 0 || kind == 3) std::sort(xs.begin(), xs.end());
        std::vector<int> bkt;
        double b0 = 0.0, binv = 0.0;
        if (!build_axis_buckets(xs.data(), n, bkt, b0, binv)) continue;   // the device bisects
        ++tables;
        std::vector<double> q = {-inf, inf, nan, xs[0] - 1.0, xs[n - 1] + 1.0};
        for (int k = 0; k < n; ++k) {
            q.push_back(xs[k]);
            q.push_back(std::nextafter(xs[k], -inf));
            q.push_back(std::nextafter(xs[k], inf));
            if (k + 1 < n) q.push_back(0.5 * (xs[k] + xs[k + 1]));
        }
        for (int r = 0; r < 200; ++r) q.push_back(xs[0] + (xs[n - 1] - xs[0]) * U(rng));
        for (double x : q) {
            const int a = bisearch(x, xs.data(), n);
            const int b = axis_search(x, xs.data(), n, bkt.data(), (int)bkt.size(), b0, binv);
            ++checks;
            if (a != b) {
                printf("FAIL kind %d n %d x %.17g bisearch %d axis_search %d\n", kind, n, x, a, b);
                return 1;
            }
        }
    }
    // not monotone: no table
    std::vector<double> bad = {0.0, 2.0, 1.0, 3.0};
    std::vector<int> bkt;
    double b0, binv;
    if (build_axis_buckets(bad.data(), (int)bad.size(), bkt, b0, binv)) {
        printf("FAIL a decreasing axis got a table\n");
        return 1;
    }
    printf("OK tables=%ld queries=%ld\n", tables, checks);
    return 0;
}

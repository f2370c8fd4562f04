// Host check of the adjoint's dual numbers (test infrastructure, built by tests/test_dual.py with
// nvcc and run on the CPU; the dual type and the formulas the reverse sweeps differentiate are
// host and device functions): at random points away from the formulas' kinks, the derivatives a
// Dual<N> carries through the elementary functions, the Tillotson EOS, RockStrengthT and the flux
// geometry (swept volume, cut length, face ratio, normalisation) equal central differences of
// the same formulas in double; at a kink (|x| at 0, min/max ties, ties within rounding) the
// derivative is the average of the one-sided ones.
#include "salec_device.cuh"
#include "salec_dual.cuh"

#include <cmath>
#include <cstdio>
#include <random>

using namespace salec;

static long g_checks = 0, g_fails = 0;

static void expect(const char *what, double got, double want, double tol)
{
    ++g_checks;
    if (!(std::fabs(got - want) <= tol)) {
        if (++g_fails <= 25) std::printf("FAIL %s: dual %.12e, expected %.12e (tol %.3e)\n", what, got, want, tol);
    }
}

// d f / d x_k by central differences of the double evaluation; f takes an array of N Duals and
// returns a Dual (its value is the double evaluation)
template <int N, class F>
static void check_grad(const char *what, F f, const double *x, double rel = 1e-6)
{
    Dual<N> in[N];
    for (int k = 0; k < N; ++k) in[k] = Dual<N>::seed(x[k], k);
    const Dual<N> r = f(in);
    for (int k = 0; k < N; ++k) {
        const double h = 1e-6 * (std::fabs(x[k]) > 1e-3 ? std::fabs(x[k]) : 1e-3);
        Dual<N> p[N], m[N];
        for (int q = 0; q < N; ++q) { p[q] = Dual<N>(x[q]); m[q] = Dual<N>(x[q]); }
        p[k] = Dual<N>(x[k] + h);
        m[k] = Dual<N>(x[k] - h);
        const double fd = (f(p).v - f(m).v) / (2.0 * h);
        // relative tolerance, plus the rounding of the difference quotient itself: the formulas
        // sum terms far larger than their result (the sound speed's c1 + c2), so its error is a
        // multiple of eps |f| / h
        const double tol = rel * std::fmax(std::fabs(fd), std::fabs(r.d[k])) + 1e-10 * std::fabs(r.v) / h;
        expect(what, r.d[k], fd, tol);
    }
}

int main()
{
    std::mt19937_64 rng(11);
    std::uniform_real_distribution<double> U(0.0, 1.0);

    // elementary functions
    for (int t = 0; t < 2000; ++t) {
        double x[2] = {0.5 + 2.5 * U(rng), 0.5 + 2.5 * U(rng)};
        if (std::fabs(x[0] - 2.0 * x[1]) < 1e-2) continue;
        check_grad<2>("elementary", [](const Dual<2> *v) {
            const Dual<2> &a = v[0], &b = v[1];
            return sqrt(a) * exp(0.1 * b) / log(a + 2.0) + tanh(a * b) + pow(a, b) - fabs(a - 2.0 * b) + a / b -
                   fmax(a, b) + fmin(a * 0.5, b);
        }, x);
    }

    // kinks: the average of the one-sided derivatives
    {
        const Dual<2> a = Dual<2>::seed(1.5, 0), b = Dual<2>::seed(1.5, 1);
        const Dual<2> mx = fmax(a, b), mn = fmin(a, b);
        expect("fmax tie d0", mx.d[0], 0.5, 0); expect("fmax tie d1", mx.d[1], 0.5, 0);
        expect("fmin tie d0", mn.d[0], 0.5, 0); expect("fmin tie d1", mn.d[1], 0.5, 0);
        const Dual<2> z = Dual<2>::seed(0.0, 0);
        expect("fabs at 0", fabs(z).d[0], 0.0, 0);
        const Dual<2> c = Dual<2>::seed(1.5 + 1e-15, 1);
        const Dual<2> near = fmax_near(a, c, 1e-12);
        expect("fmax_near value", near.v, 1.5 + 1e-15, 0);
        expect("fmax_near d0", near.d[0], 0.5, 0); expect("fmax_near d1", near.d[1], 0.5, 0);
        const Dual<2> far = fmax_near(a, c, 1e-18);
        expect("fmax_near apart d1", far.d[1], 1.0, 0);
        Dual<2> s = Dual<2>::seed(3e-17, 0);
        snap_zero(s, 1e-12);
        expect("snap_zero value", s.v, 0.0, 0); expect("snap_zero keeps d", s.d[0], 1.0, 0);
    }

    // Tillotson pressure and sound speed in every region, away from the region switches
    const double till[13] = {2700.0, 790.0, 2.67e10, 2.67e10, 4.87e8, 0.5, 1.5, 5.0, 5.0, 4.72e6, 1.82e7, 293.0, 0.0};
    for (int t = 0; t < 4000; ++t) {
        double x[2];
        const int region = t % 4;
        if (region == 0) { x[0] = 1e4 + 4.5e6 * U(rng); x[1] = 2700.0 * (1.01 + 0.6 * U(rng)); }        // compressed
        else if (region == 1) { x[0] = 1e4 + 4.6e6 * U(rng); x[1] = 2700.0 * (0.5 + 0.49 * U(rng)); }  // expanded, cold
        else if (region == 2) { x[0] = 2.0e7 + 5e8 * U(rng); x[1] = 2700.0 * (0.2 + 0.79 * U(rng)); }  // expanded, hot
        else { x[0] = 4.8e6 + 1.33e7 * U(rng); x[1] = 2700.0 * (0.3 + 0.69 * U(rng)); }                // blend
        double pres = 0., cs = 0.;
        till_pressure<double>(till, x[0], x[1], pres, cs);
        if (pres <= 1.0 || cs * cs < 1.0e-2 + 1.0) continue;   // the p <= 0.01 and c^2 < 0.01 switches
        check_grad<2>("tillotson pressure", [&](const Dual<2> *v) {
            Dual<2> p, c;
            till_pressure<Dual<2>>(till, v[0], v[1], p, c);
            return p;
        }, x, 1e-5);
        check_grad<2>("tillotson sound speed", [&](const Dual<2> *v) {
            Dual<2> p, c;
            till_pressure<Dual<2>>(till, v[0], v[1], p, c);
            return c;
        }, x, 1e-5);
    }

    // RockStrengthT with respect to its four parameters, pressure and damage
    DevMat mat;
    std::memset(&mat, 0, sizeof(mat));
    mat.Tmelt0 = 1392.0; mat.Asimon = 1.0 / 6.0e9; mat.Csimon = 1.0 / 3.0; mat.Tfrac = 1.2; mat.Tdelta = 0.0;
    mat.melt_viscosity = 0.0;
    for (int t = 0; t < 2000; ++t) {
        double x[6] = {1e5 + 5e9 * U(rng), 0.05 + 0.9 * U(rng), 1e6 + 5e7 * U(rng), 0.3 + 1.5 * U(rng),
                       1e4 + 1e6 * U(rng), 0.2 + 0.8 * U(rng)};
        const double tem = 300.0 + 800.0 * U(rng);
        // away from the Drucker-Prager cap and the damaged/intact MIN
        const double yint = x[2] + x[0] * x[3] / (1.0 + x[0] * x[3] / (2.5e9 - x[2]));
        const double ydam = x[4] + x[5] * x[0];
        if (std::fabs(ydam - 2.5e9) < 1e-3 * 2.5e9 || std::fabs(ydam - yint) < 1e-3 * yint) continue;
        check_grad<6>("rock strength", [&](const Dual<6> *v) {
            return rock_strength_t<Dual<6>>(v[0], v[1], Dual<6>(0.0), Dual<6>(tem), v[2], v[3], Dual<6>(2.5e9), v[4],
                                            v[5], Dual<6>(2.5e9), mat);
        }, x, 1e-5);
    }

    // flux geometry
    for (int t = 0; t < 2000; ++t) {
        const double xa = 10.0 + 100.0 * U(rng), ya = 100.0 * U(rng), xb = xa + 5.0 * U(rng), yb = ya + 50.0;
        double d[4] = {2.0 * U(rng) - 1.0, 2.0 * U(rng) - 1.0, 2.0 * U(rng) - 1.0, 2.0 * U(rng) - 1.0};
        check_grad<4>("swept volume", [&](const Dual<4> *v) {
            return swept_volume<Dual<4>>(xa, ya, xb, yb, v[0], v[1], v[2], v[3]);
        }, d);
        double c[3] = {U(rng), 10.0 + 40.0 * U(rng), 1.0 + 40.0 * U(rng)};
        const double a = std::fmax(c[1], c[2]), b = std::fmin(c[1], c[2]), crf = 0.5 * b / a;
        if (std::fabs(c[0] - crf) < 1e-3 || std::fabs(c[0] - (1.0 - crf)) < 1e-3 || std::fabs(c[1] - c[2]) < 1e-3 ||
            1e-5 * a > b)
            continue;
        check_grad<3>("cut length", [](const Dual<3> *v) { return cut_length<Dual<3>>(v[0], v[1], v[2]); }, c, 1e-5);
        double f[2] = {0.1 + 10.0 * U(rng), -(0.1 + 10.0 * U(rng))};
        check_grad<2>("face ratio", [](const Dual<2> *v) { return face_ratio<Dual<2>>(v[0], v[1]); }, f);
        double g[2] = {2.0 * U(rng) - 1.0, 2.0 * U(rng) - 1.0};
        if (std::fabs(g[0]) < 1e-2 || std::fabs(g[1]) < 1e-2) continue;
        check_grad<2>("normalised x", [](const Dual<2> *v) {
            Dual<2> gx = v[0], gy = v[1];
            normalise2(gx, gy);
            return gx;
        }, g);
    }

    if (g_fails) {
        std::printf("%ld of %ld checks failed\n", g_fails, g_checks);
        return 1;
    }
    std::printf("OK %ld checks\n", g_checks);
    return 0;
}

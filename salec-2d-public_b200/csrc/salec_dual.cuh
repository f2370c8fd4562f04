// Forward-mode dual numbers for the local Jacobians of the adjoint sweeps.
//
// A Dual<N> carries a value and its derivatives with respect to N chosen inputs. The reverse
// sweeps of salec_adjoint.cu are written by hand at the level of each forward sweep (which
// fields a point reads and writes, which branch it took, how adjoints scatter to neighbours);
// inside them, the long scalar formulas (the Tillotson pressure and sound speed, the yield
// surface of the strength model, the cut-line geometry of the flux) are evaluated once more on
// Dual numbers seeded at their few inputs, which gives their exact local partial derivatives in
// one pass. Comparisons and branches act on the value, so the derivatives are those of the
// branch the forward sweep took. The forward formulas are templates on their scalar type, so
// the Dual evaluation runs the same expressions as the step.
#pragma once
#include <cmath>

namespace salec {

// the double overloads stay visible beside the Dual ones declared below
using ::sqrt;
using ::exp;
using ::log;
using ::tanh;
using ::fabs;
using ::pow;
using ::fmax;
using ::fmin;
using ::floor;

template <int N>
struct Dual {
    double v;
    double d[N];
    __host__ __device__ __forceinline__ Dual() : v(0.0)
    {
#pragma unroll
        for (int k = 0; k < N; ++k) d[k] = 0.0;
    }
    __host__ __device__ __forceinline__ Dual(double x) : v(x)   // a constant
    {
#pragma unroll
        for (int k = 0; k < N; ++k) d[k] = 0.0;
    }
    // the k-th seeded input with value x
    __host__ __device__ static __forceinline__ Dual seed(double x, int k)
    {
        Dual r(x);
        r.d[k] = 1.0;
        return r;
    }
    __host__ __device__ __forceinline__ explicit operator double() const { return v; }
};

template <int N>
__host__ __device__ __forceinline__ Dual<N> lin(const Dual<N> &a, double ca, const Dual<N> &b, double cb, double v)
{
    Dual<N> r(v);
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = ca * a.d[k] + cb * b.d[k];
    return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> scale(const Dual<N> &a, double ca, double v)
{
    Dual<N> r(v);
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = ca * a.d[k];
    return r;
}

template <int N> __host__ __device__ __forceinline__ Dual<N> operator+(const Dual<N> &a, const Dual<N> &b) { return lin(a, 1.0, b, 1.0, a.v + b.v); }
template <int N> __host__ __device__ __forceinline__ Dual<N> operator-(const Dual<N> &a, const Dual<N> &b) { return lin(a, 1.0, b, -1.0, a.v - b.v); }
template <int N> __host__ __device__ __forceinline__ Dual<N> operator*(const Dual<N> &a, const Dual<N> &b) { return lin(a, b.v, b, a.v, a.v * b.v); }
template <int N> __host__ __device__ __forceinline__ Dual<N> operator/(const Dual<N> &a, const Dual<N> &b)
{
    const double q = a.v / b.v;
    return lin(a, 1.0 / b.v, b, -q / b.v, q);
}
template <int N> __host__ __device__ __forceinline__ Dual<N> operator-(const Dual<N> &a) { return scale(a, -1.0, -a.v); }
template <int N> __host__ __device__ __forceinline__ Dual<N> operator+(const Dual<N> &a, double b) { return scale(a, 1.0, a.v + b); }
template <int N> __host__ __device__ __forceinline__ Dual<N> operator+(double a, const Dual<N> &b) { return scale(b, 1.0, a + b.v); }
template <int N> __host__ __device__ __forceinline__ Dual<N> operator-(const Dual<N> &a, double b) { return scale(a, 1.0, a.v - b); }
template <int N> __host__ __device__ __forceinline__ Dual<N> operator-(double a, const Dual<N> &b) { return scale(b, -1.0, a - b.v); }
template <int N> __host__ __device__ __forceinline__ Dual<N> operator*(const Dual<N> &a, double b) { return scale(a, b, a.v * b); }
template <int N> __host__ __device__ __forceinline__ Dual<N> operator*(double a, const Dual<N> &b) { return scale(b, a, a * b.v); }
template <int N> __host__ __device__ __forceinline__ Dual<N> operator/(const Dual<N> &a, double b) { return scale(a, 1.0 / b, a.v / b); }
template <int N> __host__ __device__ __forceinline__ Dual<N> operator/(double a, const Dual<N> &b)
{
    const double q = a / b.v;
    return scale(b, -q / b.v, q);
}
template <int N> __host__ __device__ __forceinline__ Dual<N> &operator+=(Dual<N> &a, const Dual<N> &b) { a = a + b; return a; }
template <int N> __host__ __device__ __forceinline__ Dual<N> &operator-=(Dual<N> &a, const Dual<N> &b) { a = a - b; return a; }
template <int N> __host__ __device__ __forceinline__ Dual<N> &operator*=(Dual<N> &a, const Dual<N> &b) { a = a * b; return a; }
template <int N> __host__ __device__ __forceinline__ Dual<N> &operator/=(Dual<N> &a, const Dual<N> &b) { a = a / b; return a; }

template <int N> __host__ __device__ __forceinline__ bool operator<(const Dual<N> &a, const Dual<N> &b) { return a.v < b.v; }
template <int N> __host__ __device__ __forceinline__ bool operator>(const Dual<N> &a, const Dual<N> &b) { return a.v > b.v; }
template <int N> __host__ __device__ __forceinline__ bool operator<=(const Dual<N> &a, const Dual<N> &b) { return a.v <= b.v; }
template <int N> __host__ __device__ __forceinline__ bool operator>=(const Dual<N> &a, const Dual<N> &b) { return a.v >= b.v; }
template <int N> __host__ __device__ __forceinline__ bool operator<(const Dual<N> &a, double b) { return a.v < b; }
template <int N> __host__ __device__ __forceinline__ bool operator>(const Dual<N> &a, double b) { return a.v > b; }
template <int N> __host__ __device__ __forceinline__ bool operator<=(const Dual<N> &a, double b) { return a.v <= b; }
template <int N> __host__ __device__ __forceinline__ bool operator>=(const Dual<N> &a, double b) { return a.v >= b; }
template <int N> __host__ __device__ __forceinline__ bool operator<(double a, const Dual<N> &b) { return a < b.v; }
template <int N> __host__ __device__ __forceinline__ bool operator>(double a, const Dual<N> &b) { return a > b.v; }

template <int N> __host__ __device__ __forceinline__ Dual<N> sqrt(const Dual<N> &a)
{
    const double s = ::sqrt(a.v);
    return scale(a, s > 0.0 ? 0.5 / s : 0.0, s);
}
template <int N> __host__ __device__ __forceinline__ Dual<N> exp(const Dual<N> &a)
{
    const double e = ::exp(a.v);
    return scale(a, e, e);
}
template <int N> __host__ __device__ __forceinline__ Dual<N> log(const Dual<N> &a) { return scale(a, 1.0 / a.v, ::log(a.v)); }
template <int N> __host__ __device__ __forceinline__ Dual<N> tanh(const Dual<N> &a)
{
    const double t = ::tanh(a.v);
    return scale(a, 1.0 - t * t, t);
}
// At a kink (|x| at 0, ties of min/max) the derivative is the average of the two one-sided
// ones: what a symmetric (central) perturbation of the input sees.
template <int N> __host__ __device__ __forceinline__ Dual<N> fabs(const Dual<N> &a)
{
    return scale(a, a.v < 0.0 ? -1.0 : (a.v > 0.0 ? 1.0 : 0.0), ::fabs(a.v));
}
template <int N> __host__ __device__ __forceinline__ Dual<N> pow(const Dual<N> &a, const Dual<N> &b)
{
    // a^b = exp(b log a), for a > 0; the forward formulas raise positive bases only
    const double p = ::pow(a.v, b.v);
    Dual<N> r(p);
    const double da = a.v != 0.0 ? b.v * p / a.v : 0.0;
    const double db = a.v > 0.0 ? p * ::log(a.v) : 0.0;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = da * a.d[k] + db * b.d[k];
    return r;
}
template <int N> __host__ __device__ __forceinline__ Dual<N> tie(const Dual<N> &a, const Dual<N> &b)
{
    return lin(a, 0.5, b, 0.5, a.v);
}
template <int N> __host__ __device__ __forceinline__ Dual<N> fmax(const Dual<N> &a, const Dual<N> &b)
{
    return a.v > b.v ? a : (b.v > a.v ? b : tie(a, b));
}
template <int N> __host__ __device__ __forceinline__ Dual<N> fmin(const Dual<N> &a, const Dual<N> &b)
{
    return a.v < b.v ? a : (b.v < a.v ? b : tie(a, b));
}
// max of two values that may differ by rounding only: within tol of each other they are a tie
template <int N> __host__ __device__ __forceinline__ Dual<N> fmax_near(const Dual<N> &a, const Dual<N> &b, double tol)
{
    if (::fabs(a.v - b.v) > tol) return a.v > b.v ? a : b;
    return lin(a, 0.5, b, 0.5, a.v > b.v ? a.v : b.v);
}
// a value within tol of zero, a kink of the formulas downstream (|x|, a corner maximum), is put on
// the kink; its derivatives are kept
template <int N> __host__ __device__ __forceinline__ void snap_zero(Dual<N> &a, double tol)
{
    if (::fabs(a.v) <= tol) a.v = 0.0;
}
// the min/max/clamp of the step's templated formulas, with the same tie rule
template <int N> __host__ __device__ __forceinline__ Dual<N> amin(Dual<N> a, Dual<N> b) { return fmin(a, b); }
template <int N> __host__ __device__ __forceinline__ Dual<N> amax(Dual<N> a, Dual<N> b) { return fmax(a, b); }
template <int N> __host__ __device__ __forceinline__ Dual<N> floor(const Dual<N> &a) { return Dual<N>(::floor(a.v)); }
template <int N> __host__ __device__ __forceinline__ double val(const Dual<N> &a) { return a.v; }

} // namespace salec

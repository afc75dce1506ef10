// Hyper-dual numbers a + b e1 + c e2 + d e1 e2 (e1^2 = e2^2 = 0).
//
// Evaluating a function f in this arithmetic with the input x + t1 e1 + t2 e2
// returns f(x) in a, the directional derivatives D_t1 f and D_t2 f in b and
// c, and the mixed second derivative D_t1 D_t2 f in d, each exact to FP64
// rounding (Fike and Alonso, "The development of hyper-dual numbers for exact
// second-derivative calculations", AIAA 2011-886).  A unary function g acts
// as g(a) + g'(a)(b e1 + c e2) + (g'(a) d + g''(a) b c) e1 e2.  The
// functions carry an h prefix (hsqrt, habs, ...) so that they do not hide
// the double overloads inside namespace cr.
#pragma once
#include <cuda_runtime.h>

namespace cr {

struct HD {
  double a, b, c, d;
};

__host__ __device__ __forceinline__ HD hd(double a) { return HD{a, 0.0, 0.0, 0.0}; }
__host__ __device__ __forceinline__ HD hd(double a, double b, double c, double d) { return HD{a, b, c, d}; }

__device__ __forceinline__ HD operator+(HD x, HD y) { return HD{x.a + y.a, x.b + y.b, x.c + y.c, x.d + y.d}; }
__device__ __forceinline__ HD operator-(HD x, HD y) { return HD{x.a - y.a, x.b - y.b, x.c - y.c, x.d - y.d}; }
__device__ __forceinline__ HD operator-(HD x) { return HD{-x.a, -x.b, -x.c, -x.d}; }
__device__ __forceinline__ HD operator*(HD x, HD y) {
  return HD{x.a * y.a, x.a * y.b + x.b * y.a, x.a * y.c + x.c * y.a, x.a * y.d + x.b * y.c + x.c * y.b + x.d * y.a};
}
__device__ __forceinline__ HD operator*(double s, HD x) { return HD{s * x.a, s * x.b, s * x.c, s * x.d}; }
__device__ __forceinline__ HD operator*(HD x, double s) { return HD{s * x.a, s * x.b, s * x.c, s * x.d}; }
__device__ __forceinline__ HD operator+(HD x, double s) { return HD{x.a + s, x.b, x.c, x.d}; }
__device__ __forceinline__ HD operator+(double s, HD x) { return HD{x.a + s, x.b, x.c, x.d}; }
__device__ __forceinline__ HD operator-(HD x, double s) { return HD{x.a - s, x.b, x.c, x.d}; }
__device__ __forceinline__ HD operator-(double s, HD x) { return HD{s - x.a, -x.b, -x.c, -x.d}; }
__device__ __forceinline__ HD& operator+=(HD& x, HD y) { return x = x + y; }
__device__ __forceinline__ HD& operator-=(HD& x, HD y) { return x = x - y; }

// g(x) from g(a), g'(a), g''(a)
__device__ __forceinline__ HD hd_apply(HD x, double g, double g1, double g2) {
  return HD{g, g1 * x.b, g1 * x.c, g1 * x.d + g2 * x.b * x.c};
}
__device__ __forceinline__ HD recip(HD x) {
  const double r = 1.0 / x.a;
  return hd_apply(x, r, -r * r, 2.0 * r * r * r);
}
__device__ __forceinline__ HD operator/(HD x, HD y) { return x * recip(y); }
__device__ __forceinline__ HD operator/(HD x, double s) { return x * (1.0 / s); }
__device__ __forceinline__ HD operator/(double s, HD y) { return s * recip(y); }
__device__ __forceinline__ HD hsqrt(HD x) {
  const double s = ::sqrt(x.a);
  return hd_apply(x, s, 0.5 / s, -0.25 / (s * x.a));
}
__device__ __forceinline__ HD hlog(HD x) { return hd_apply(x, ::log(x.a), 1.0 / x.a, -1.0 / (x.a * x.a)); }
__device__ __forceinline__ HD habs(HD x) { return x.a < 0.0 ? -x : x; }
// atan2 from its partial derivatives in (x, y), r^2 = x^2 + y^2:
//   th_x = -y / r^2, th_y = x / r^2, th_xx = 2xy / r^4, th_yy = -2xy / r^4,
//   th_xy = (y^2 - x^2) / r^4
__device__ __forceinline__ HD hatan2(HD y, HD x) {
  const double r2 = x.a * x.a + y.a * y.a, r4 = r2 * r2;
  const double tx = -y.a / r2, ty = x.a / r2;
  const double txx = 2.0 * x.a * y.a / r4, tyy = -txx, txy = (y.a * y.a - x.a * x.a) / r4;
  return HD{::atan2(y.a, x.a), tx * x.b + ty * y.b, tx * x.c + ty * y.c,
            tx * x.d + ty * y.d + txx * x.b * x.c + tyy * y.b * y.c + txy * (x.b * y.c + x.c * y.b)};
}

struct HD2 {
  HD x, y;
};

}  // namespace cr

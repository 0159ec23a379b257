// FP64 complex arithmetic for device code (double2 storage), with the operations the
// reference's std::complex<double> code uses.  Elementary functions call CUDA's FP64 math.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace hgx {

struct zd {
  double x, y;
  __host__ __device__ zd() : x(0), y(0) {}
  __host__ __device__ zd(double r) : x(r), y(0) {}
  __host__ __device__ zd(double r, double i) : x(r), y(i) {}
  __host__ __device__ explicit zd(double2 v) : x(v.x), y(v.y) {}
  __host__ __device__ double2 d2() const { return make_double2(x, y); }
};

__host__ __device__ __forceinline__ zd operator+(zd a, zd b) { return zd(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ zd operator-(zd a, zd b) { return zd(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ zd operator-(zd a) { return zd(-a.x, -a.y); }
__host__ __device__ __forceinline__ zd operator*(zd a, zd b) {
  return zd(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// complex * real scales both parts (as the reference's operator*(complex, real))
__host__ __device__ __forceinline__ zd operator*(zd a, double s) { return zd(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ zd operator*(double s, zd a) { return zd(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ zd operator/(zd a, double s) { return zd(a.x / s, a.y / s); }
__host__ __device__ __forceinline__ zd operator+(zd a, double s) { return zd(a.x + s, a.y); }
__host__ __device__ __forceinline__ zd operator+(double s, zd a) { return zd(a.x + s, a.y); }
__host__ __device__ __forceinline__ zd operator-(double s, zd a) { return zd(s - a.x, -a.y); }
__host__ __device__ __forceinline__ zd operator-(zd a, double s) { return zd(a.x - s, a.y); }
__host__ __device__ __forceinline__ zd& operator+=(zd& a, zd b) {
  a.x += b.x;
  a.y += b.y;
  return a;
}
// Smith's division (robust against overflow of |b|^2)
__host__ __device__ __forceinline__ zd operator/(zd a, zd b) {
  if (fabs(b.x) >= fabs(b.y)) {
    if (b.x == 0.0 && b.y == 0.0) return zd(a.x / 0.0, a.y / 0.0);
    double r = b.y / b.x, den = b.x + b.y * r;
    return zd((a.x + a.y * r) / den, (a.y - a.x * r) / den);
  }
  double r = b.x / b.y, den = b.x * r + b.y;
  return zd((a.x * r + a.y) / den, (a.y * r - a.x) / den);
}
__host__ __device__ __forceinline__ zd operator/(double s, zd b) { return zd(s) / b; }

__device__ __forceinline__ zd conj(zd a) { return zd(a.x, -a.y); }
__device__ __forceinline__ double norm2(zd a) { return a.x * a.x + a.y * a.y; }
__device__ __forceinline__ double cabs_(zd a) { return hypot(a.x, a.y); }
__device__ __forceinline__ zd cexp_(zd a) {
  double e = exp(a.x), s, c;
  sincos(a.y, &s, &c);
  return zd(e * c, e * s);
}
__device__ __forceinline__ zd expi(double ph) {  // e^{i ph}
  double s, c;
  sincos(ph, &s, &c);
  return zd(c, s);
}
__device__ __forceinline__ zd csin_(zd a) {
  double s, c;
  sincos(a.x, &s, &c);
  return zd(s * cosh(a.y), c * sinh(a.y));
}
__device__ __forceinline__ zd ccos_(zd a) {
  double s, c;
  sincos(a.x, &s, &c);
  return zd(c * cosh(a.y), -s * sinh(a.y));
}
__device__ __forceinline__ zd csqrt_(zd a) {  // principal branch, as C99 csqrt
  if (a.x == 0.0 && a.y == 0.0) return zd(0.0, a.y);
  double m = hypot(a.x, a.y);
  double t = sqrt(0.5 * (m + fabs(a.x)));
  if (a.x >= 0.0) return zd(t, a.y / (2.0 * t));
  return zd(fabs(a.y) / (2.0 * t), copysign(t, a.y));
}
__device__ __forceinline__ zd clog_(zd a) { return zd(log(hypot(a.x, a.y)), atan2(a.y, a.x)); }
// std::pow(complex, real) as libstdc++ evaluates it: a positive real base takes the real
// pow; otherwise polar(exp(y log|x|), y arg x) — the principal branch.
__device__ __forceinline__ zd cpow_std(zd x, double y) {
  if (x.y == 0.0 && x.x > 0.0) return zd(pow(x.x, y), 0.0);
  zd t = clog_(x);
  double rho = exp(y * t.x), th = y * t.y, s, c;
  sincos(th, &s, &c);
  return zd(rho * c, rho * s);
}

// RotMatrix_t::rotate(real x, real y, complex z) (include/numerics/matrix.hpp:123-130)
struct Rot9d {
  double r[9];
};
__device__ __forceinline__ void rotate_q(const Rot9d& R, double x, double y, zd z, zd* m) {
#pragma unroll
  for (int j = 0; j < 3; ++j)
    m[j] = zd(R.r[3 * j] * x + R.r[3 * j + 1] * y + R.r[3 * j + 2] * z.x, R.r[3 * j + 2] * z.y);
}

}  // namespace hgx

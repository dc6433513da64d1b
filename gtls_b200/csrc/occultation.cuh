// Occultation of a star with quadratic limb darkening by an opaque disk, by
// the quadrature of gtls_b200/ldmodel.py (96-node Gauss-Legendre after the
// substitution r = m + h sin(theta)), in forms shared by the adjoint model
// (adjoint.cu, with dual-number derivatives in (z, p)) and the transit
// template generator (templates.cu).  ldmodel stands in for the batman light
// curve of the reference (src/gputls/transit.py:8-42).
#pragma once
#include <cuda_runtime.h>

#include <cmath>

namespace gtls {

constexpr double kPi = 3.14159265358979323846;
constexpr int kGLN = 96;

// Quadrature table: s[j] = sin(theta_j), jw[j] = cos(theta_j) * pi/2 * w_j
// with theta_j = pi/2 x_j for the Gauss-Legendre nodes x_j and weights w_j.
struct GLTable {
  double s[kGLN];
  double jw[kGLN];
};

// Gauss-Legendre nodes and weights on [-1, 1] by Newton's method on the
// three-term recurrence of the Legendre polynomials (Golub-Welsch-free
// classic; converges to a few ulp from the Tricomi starting values).
static GLTable make_gl_table() {
  GLTable g;
  const int n = kGLN;
  for (int i = 0; i < (n + 1) / 2; ++i) {
    double x = std::cos(kPi * (i + 0.75) / (n + 0.5));
    double dp = 1.0;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1.0, p1 = x;
      for (int k = 2; k <= n; ++k) {
        const double p2 = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      dp = n * (x * p1 - p0) / (x * x - 1.0);
      const double dx = p1 / dp;
      x -= dx;
      if (std::fabs(dx) < 1e-17) break;
    }
    const double w = 2.0 / ((1.0 - x * x) * dp * dp);
    // ascending order: node j = n-1-i holds +x, node i holds -x
    const int hi = n - 1 - i, lo = i;
    const double th = 0.5 * kPi * x;
    g.s[hi] = std::sin(th);
    g.jw[hi] = std::cos(th) * (0.5 * kPi) * w;
    g.s[lo] = -g.s[hi];
    g.jw[lo] = g.jw[hi];
  }
  return g;
}

static const GLTable& gl_table() {
  static const GLTable g = make_gl_table();
  return g;
}

// value and derivatives with respect to (z, p)
struct D2 {
  double v, z, p;
};
__device__ __forceinline__ D2 d2(double v) { return {v, 0.0, 0.0}; }
__device__ __forceinline__ D2 operator+(D2 a, D2 b) { return {a.v + b.v, a.z + b.z, a.p + b.p}; }
__device__ __forceinline__ D2 operator-(D2 a, D2 b) { return {a.v - b.v, a.z - b.z, a.p - b.p}; }
__device__ __forceinline__ D2 operator*(D2 a, D2 b) {
  return {a.v * b.v, a.v * b.z + b.v * a.z, a.v * b.p + b.v * a.p};
}
__device__ __forceinline__ D2 operator*(D2 a, double s) { return {a.v * s, a.z * s, a.p * s}; }
__device__ __forceinline__ D2 operator/(D2 a, D2 b) {
  const double q = a.v / b.v;
  return {q, (a.z - q * b.z) / b.v, (a.p - q * b.p) / b.v};
}
// value of double inputs: the same expressions without derivatives
__device__ __forceinline__ double dval(double a) { return a; }
__device__ __forceinline__ double dval(D2 a) { return a.v; }

// mu = sqrt(max(1 - r^2, 0)) and its derivative (0 where clamped)
__device__ __forceinline__ double mu_of(double r) {
  const double x = 1.0 - r * r;
  return x > 0.0 ? sqrt(x) : 0.0;
}
__device__ __forceinline__ D2 mu_of(D2 r) {
  const double x = 1.0 - r.v * r.v;
  if (!(x > 0.0)) return d2(0.0);
  const double m = sqrt(x);
  const double k = -r.v / m;
  return {m, k * r.z, k * r.p};
}
// acos of c clamped to [-1, 1] (derivative 0 where clamped)
__device__ __forceinline__ double acos_clamped(double c) {
  return c >= 1.0 ? 0.0 : (c <= -1.0 ? kPi : acos(c));
}
__device__ __forceinline__ D2 acos_clamped(D2 c) {
  if (c.v >= 1.0) return d2(0.0);
  if (c.v <= -1.0) return d2(kPi);
  const double s = 1.0 - c.v * c.v;
  const double k = s > 0.0 ? -1.0 / sqrt(s) : 0.0;
  return {acos(c.v), k * c.z, k * c.p};
}

// Constants of either scalar type.
template <typename T> __device__ __forceinline__ T cst(double v);
template <> __device__ __forceinline__ double cst<double>(double v) { return v; }
template <> __device__ __forceinline__ D2 cst<D2>(double v) { return d2(v); }

// Moments M0..M2 of the occulted flux: lambda = (M0 - u1 M1 - u2 M2) / (pi K),
// Mk = int (1 - mu)^k x (2 pi r over the covered disk, 2 r acos(c) over the
// partly covered annuli) dr, both by the quadrature of ldmodel.occulted_fraction.
template <typename T>
__device__ __forceinline__ void occultation_moments(T Z, T Pp, const GLTable& g, T (&M)[3]) {
#pragma unroll
  for (int k = 0; k < 3; ++k) M[k] = cst<T>(0.0);
  const double z = dval(Z), p = dval(Pp);
  const T one = cst<T>(1.0);
  // region fully covered by the planet: r in [0, min(p - z, 1)]
  if (p - z > 0.0) {
    const T ih = p - z > 1.0 ? one : Pp - Z;
    const T half = ih * 0.5;
    for (int j = 0; j < kGLN; ++j) {
      const T r = half + half * g.s[j];
      const T wt = half * g.jw[j];
      const T om = one - mu_of(r);
      const T f = r * wt * (2.0 * kPi);
      M[0] = M[0] + f;
      M[1] = M[1] + f * om;
      M[2] = M[2] + f * om * om;
    }
  }
  // partially covered annuli: r in [|z - p|, min(1, z + p)]
  const T lo = z >= p ? Z - Pp : Pp - Z;
  const T hi = z + p > 1.0 ? one : Z + Pp;
  if (dval(hi) > dval(lo)) {
    const T mid = (lo + hi) * 0.5;
    const T half = (hi - lo) * 0.5;
    const T zs = z > 1e-300 ? Z : cst<T>(1e-300);
    const T zp2 = zs * zs - Pp * Pp;
    for (int j = 0; j < kGLN; ++j) {
      const T r = mid + half * g.s[j];
      const T wt = half * g.jw[j];
      const T c = (r * r + zp2) / (r * zs * 2.0);
      const T om = one - mu_of(r);
      const T f = r * acos_clamped(c) * wt * 2.0;
      M[0] = M[0] + f;
      M[1] = M[1] + f * om;
      M[2] = M[2] + f * om * om;
    }
  }
}


// Fraction of the stellar flux blocked by a disk of radius p at separation z
// (ldmodel.occulted_fraction): 0 unless z < 1 + p and p > 0.
__device__ __forceinline__ double occulted_fraction(double z, double p, double u1, double u2, const GLTable& g) {
  if (!(p > 0.0) || !(z < 1.0 + p)) return 0.0;
  double M[3];
  occultation_moments<double>(z, p, g, M);
  return (M[0] - u1 * M[1] - u2 * M[2]) / (kPi * (1.0 - u1 / 3.0 - u2 / 6.0));
}

}  // namespace gtls

// Shared device helpers for the FourierD3 sm_100a kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/fd3.h"

#define FD3_WARP 32
#define FD3_MAX_SPECIES 64
#define FD3_MAX_RANK 32
#define FD3_MAX_ORDER 8

namespace fd3 {

constexpr double kPi = 3.14159265358979323846;
constexpr double kAngToBohr = 1.0 / 0.52917726;   // core.py:120
constexpr double kHartreeToEv = 27.21138505;      // calculator.py:54

// Cell-derived quantities, computed on the device from the (possibly strained) cell.
struct CellInfo {
  double cell[9];   // rows = lattice vectors, Bohr
  double inv[9];    // adjugate / determinant inverse (utils.py:142-167)
  double recip[9];  // rows b_i = 2 pi inv[:, i]
  double volume;    // |det| (utils.py:130-139)
  double stale;     // 1: the device cell differs from the host cell the call's geometry came from
  double pad[4];
};

// Per species-pair constants of the BJ Green's function (pair_pot.py:63-105).
struct GreenPair {
  double R, qq, c6s1, c6s2, c6pre, c8s1, c8s2, c8pre;
};
// The same constants rounded to float once, for the mixed-form filter (no per-use conversion).
struct GreenPairF {
  float R, qq, c6s1, c6s2, c6pre, c8s1, c8s2, c8pre;
};
template <typename T> struct GreenPairOf { using type = GreenPair; };
template <> struct GreenPairOf<float> { using type = GreenPairF; };

// Device-resident per-plan tables (uploaded once by fd3_plan_create).
struct Tables {
  double rcov[FD3_MAX_SPECIES];
  double cnref[FD3_MAX_SPECIES * 7];
  double selfcont[FD3_MAX_SPECIES];          // phi_XX(0) (pair_pot.py:84-89)
  double cncorr[FD3_MAX_SPECIES * 2];
  double eigs[FD3_MAX_RANK];
  double s6, s8, r_cut;
  int n_species, n_rank, has_cncorr, pad;
  // eigvecs (S,7,r) and the (S,S) GreenPair matrix follow in separate device arrays
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Block-wide sum of NV doubles into out[0..NV) (thread 0 writes). blockDim multiple of 32.
template <int NV>
__device__ void block_sum_store(double (&v)[NV], double* out) {
  __shared__ double red[NV][32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double s = warp_sum(v[k]);
    if (lane == 0) red[k][wid] = s;
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double s = lane < nw ? red[k][lane] : 0.0;
      s = warp_sum(s);
      if (lane == 0) out[k] = s;
    }
  }
  __syncthreads();
}

// Exact-order helpers: the neighbour predicate must not be contracted into FMAs.
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }

// Smooth-cutoff CN edge function and its r-derivative (core.py:348-378).
// r: distance (Bohr), rcs: rcov_i + rcov_j, rc: CN cutoff (Bohr).
__device__ __forceinline__ void cn_edge(double r, double rcs, double rc, double& f, double& df) {
  const double rs = fmax(r, 1e-6);
  const double r1 = 0.5 * rcs + 0.5 * rc;
  const bool outer = rs > r1;
  const double coeff = outer ? rs : r1;
  const double t = rc - coeff;
  const double denom = t * t + 1e-6;
  const double dd = coeff - r1;
  const double k = 16.0 + dd * dd / denom;
  const double ratio = (4.0 / 3.0) * rcs;
  const double z = k * (ratio * (1.0 / rs) - 1.0);   // sigmoid argument
  const double e = exp(-z);
  const double s = 1.0 / (1.0 + e);
  if (r > 1e-6) {
    f = s;
    // dk/dr on the outer branch; zero where the clamp or the inner branch is active
    const double dk = outer ? (2.0 * dd / denom + dd * dd * 2.0 * t / (denom * denom)) : 0.0;
    const double dz = dk * (ratio / rs - 1.0) - k * ratio / (rs * rs);
    df = s * (1.0 - s) * dz;
  } else {
    f = 0.0;
    df = 0.0;
  }
}

__device__ __forceinline__ double rsqrt_t(double x) { return rsqrt(x); }
__device__ __forceinline__ float rsqrt_t(float x) { return rsqrtf(x); }
__device__ __forceinline__ double exp_t(double x) { return exp(x); }
__device__ __forceinline__ float exp_t(float x) { return __expf(x); }
__device__ __forceinline__ double rcp_t(double x) { return 1.0 / x; }
__device__ __forceinline__ void sincospi_t(double x, double* s, double* c) { sincospi(x, s, c); }
// sin(pi x) and cos(pi x) in float for the mixed form. Exact reduction by quarter turns,
// x = n/2 + f with n = rint(2x) and |f| <= 1/4 (f is exact: Sterbenz), then the Taylor series of
// sin(pi f) to f^9 and of cos(pi f) to f^10 (truncation below 2e-9 on |f| <= 1/4; coefficients
// (-1)^k pi^(2k+1)/(2k+1)! and (-1)^k pi^(2k)/(2k)! rounded to float), and the rotation by the
// quadrant n mod 4. Valid for |x| < 2^22; measured error below 1 ulp of 1.
__device__ __forceinline__ void sincospi_t(float x, float* s, float* c) {
  const float n = rintf(2.0f * x);
  const float f = fmaf(-0.5f, n, x);
  const float f2 = f * f;
  float ps = 0.08214588463306427f;
  ps = fmaf(ps, f2, -0.5992645025253296f);
  ps = fmaf(ps, f2, 2.550163984298706f);
  ps = fmaf(ps, f2, -5.167712688446045f);
  ps = fmaf(ps, f2, 3.1415927410125732f);
  const float sv = ps * f;
  float pc = -0.025806890800595284f;
  pc = fmaf(pc, f2, 0.23533062636852264f);
  pc = fmaf(pc, f2, -1.3352627754211426f);
  pc = fmaf(pc, f2, 4.058712005615234f);
  pc = fmaf(pc, f2, -4.934802055358887f);
  const float cv = fmaf(pc, f2, 1.0f);
  const int q = ((int)n) & 3;
  const float so = (q & 1) ? cv : sv;
  const float co = (q & 1) ? sv : cv;
  *s = (q & 2) ? -so : so;
  *c = ((q + 1) & 2) ? -co : co;
}
// float: the hardware reciprocal (rcp.approx, at most 1 ulp from the correctly rounded value;
// callers pass normal, positive arguments) -- the mixed form's CN pair function takes two per
// pair, where the correctly rounded reciprocal costs an instruction sequence each
__device__ __forceinline__ float rcp_t(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// The same CN edge function from the squared distance r2 > 1e-12 Bohr^2 (the reference zeroes
// r <= 1e-6): f and a = f'(r) / r with one reciprocal square root and two reciprocals.
// TC = double for the plain form, float (fast exp) for the mixed form.
template <typename TC>
__device__ __forceinline__ void cn_pair(TC r2, TC rcs, TC rc, TC& f, TC& a) {
  const TC inv_r = rsqrt_t(r2);
  const TC r = r2 * inv_r;
  const TC r1 = TC(0.5) * rcs + TC(0.5) * rc;
  const bool outer = r > r1;
  const TC coeff = outer ? r : r1;
  const TC t = rc - coeff;
  const TC inv_den = rcp_t(t * t + TC(1e-6));
  const TC dd = coeff - r1;
  const TC k = TC(16) + dd * dd * inv_den;
  const TC ratio = TC(4.0 / 3.0) * rcs;
  const TC q = ratio * inv_r - TC(1);
  const TC s = rcp_t(TC(1) + exp_t(-(k * q)));
  f = s;
  // dk/dr = 2 dd/den + 2 dd^2 t/den^2 on the outer branch, 0 inside
  const TC dk = outer ? TC(2) * dd * inv_den * (TC(1) + dd * t * inv_den) : TC(0);
  a = s * (TC(1) - s) * (dk * q - k * ratio * inv_r * inv_r) * inv_r;
}

// Order-p cardinal B-spline weights at the p stencil nodes for local coordinate x in
// [-1/2, 1/2]: w[k] = M_p(1/2 - x + k); dw = dw/dx (Cox-de Boor recursion).
template <int P, typename T>
__device__ __forceinline__ void bspline(T x, T* w, T* dw) {
  const T a = T(0.5) - x;
  T m[P];
  m[0] = T(1);
#pragma unroll
  for (int q = 2; q <= P; ++q) {
    if (q == P) {
      // derivative from M_{P-1}: d/da M_P(a+k) = M_{P-1}(a+k) - M_{P-1}(a+k-1)
#pragma unroll
      for (int k = 0; k < P; ++k) {
        const T l = k < P - 1 ? m[k] : T(0);
        const T r = k >= 1 ? m[k - 1] : T(0);
        dw[k] = -(l - r);
      }
    }
    T nm[P];
#pragma unroll
    for (int j = 0; j < q; ++j) {
      const T u = a + T(j);
      const T l = j < q - 1 ? m[j] : T(0);
      const T r = j >= 1 ? m[j - 1] : T(0);
      nm[j] = (u * l + (T(q) - u) * r) / T(q - 1);
    }
#pragma unroll
    for (int j = 0; j < q; ++j) m[j] = nm[j];
  }
  if (P == 1) dw[0] = T(0);
#pragma unroll
  for (int k = 0; k < P; ++k) w[k] = m[k];
}

// p-point Lagrange basis on nodes 0..p-1 with the charge at t = x + (p-1)/2.
template <int P, typename T>
__device__ __forceinline__ void lagrange(T x, T* w, T* dw) {
  const T t = x + T(0.5) * T(P - 1);
#pragma unroll
  for (int k = 0; k < P; ++k) {
    T prod = T(1), der = T(0);
#pragma unroll
    for (int m = 0; m < P; ++m) {
      if (m == k) continue;
      const T f = (t - T(m)) / T(k - m);
      der = der * f + prod / T(k - m);
      prod = prod * f;
    }
    w[k] = prod;
    dw[k] = der;
  }
}

// Green's function G_XY(k) and dG/dk for one species pair (pair_pot.py:142-178).
template <typename T, typename GP>
__device__ __forceinline__ void green_eval(const GP& g, T k, T s6, T s8, T& G, T& dG) {
  const T R = T(g.R);
  const T ksq = k * k;
  if (k * R < T(1e-15)) {
    const T f6 = s6 * (T(g.c6s1) - T(g.c6s2) * ksq);
    const T d6 = s6 * (T(-2) * T(g.c6s2) * k);
    const T f8 = T(3) * s8 * (T(g.c8s1) - T(g.c8s2) * ksq);
    const T d8 = T(3) * s8 * (T(-2) * T(g.c8s2) * k);
    G = f6 + T(g.qq) * f8;
    dG = d6 + T(g.qq) * d8;
    return;
  }
  const T sq3 = T(1.7320508075688772935);
  const T sin8 = T(0.38268343236508977173);   // sin(pi/8)
  const T cos8 = T(0.92387953251128675613);   // cos(pi/8)
  const T u = k * R;
  // exp(-u) = exp(-u/2)^2; the phases pi/3 + u sqrt3/2, pi/4 + u cos(pi/8), 3pi/4 + u sin(pi/8)
  // are evaluated in half-turns with sincospi (exact argument reduction).
  const T e2 = exp_t(-u * T(0.5));
  const T e1 = e2 * e2;
  T sa, ca;
  sincospi_t(T(1.0 / 3.0) + u * T(0.27566444771089604), &sa, &ca);   // sqrt(3) / (2 pi)
  const T n6 = e1 - T(2) * e2 * ca;
  const T dn6 = -e1 + e2 * ca + sq3 * e2 * sa;
  const T e3 = exp_t(-u * sin8);
  const T e4 = exp_t(-u * cos8);
  T s1, c1, s2, c2;
  sincospi_t(T(0.25) + u * T(0.29407998884120140), &s1, &c1);      // cos(pi/8) / pi
  sincospi_t(T(0.75) + u * T(0.12181191980055409), &s2, &c2);      // sin(pi/8) / pi
  const T n8 = e3 * c1 + e4 * c2;
  const T dn8 = -sin8 * e3 * c1 - cos8 * e3 * s1 - cos8 * e4 * c2 - sin8 * e4 * s2;
  const T invk = T(1) / k;
  const T f6 = s6 * ((T(g.c6pre) * invk) * n6);
  const T d6 = s6 * T(g.c6pre) * (R * dn6 * invk - n6 * invk * invk);
  const T f8 = T(3) * s8 * ((T(g.c8pre) * invk) * n8);
  const T d8 = T(3) * s8 * T(g.c8pre) * (R * dn8 * invk - n8 * invk * invk);
  G = f6 + T(g.qq) * f8;
  dG = d6 + T(g.qq) * d8;
}

// ---------------------------------------------------------------- Green's function table
// Mixed form: G_XY(|k|) and dG/d|k| from a per-call table on kGreenKnots intervals of
// [0, kmax], kmax = sum_a (n_a / 2) |b_a| >= every mesh |k|. Knot j of pair p holds, in float,
// {G, h G1, h^2 G2, h^3 G3} (Gm the m-th k-derivative, h = kmax / kGreenKnots) computed in
// float64 from the closed form
//   G = F(kR) / k, G1 = (R F1 - G) / k, G2 = (R^2 F2 - 2 G1) / k, G3 = (R^3 F3 - 3 G2) / k,
//   F = s6 c6pre n6 + 3 s8 qq c8pre n8 (arguments kR, Fm the m-th u-derivative),
// (the Taylor limit at k = 0); between knots G is the quintic Hermite interpolant of (G, G1, G2)
// and dG/dk that of (G1, G2, G3). Over the u = kR range of the dispersion kernel (R up to 10
// Bohr) the relative error is below 1e-9 for both (checked against the closed form in float64),
// under float rounding; the table is 4 KB per species pair, small enough to stay in L1.
constexpr int kGreenKnots = 256;

__host__ __device__ inline double green_kmax(const double (&recip)[9], const int (&n)[3]) {
  double k = 0.0;
  for (int a = 0; a < 3; ++a)
    k += 0.5 * n[a] * sqrt(recip[3 * a] * recip[3 * a] + recip[3 * a + 1] * recip[3 * a + 1] +
                           recip[3 * a + 2] * recip[3 * a + 2]);
  return k;
}

// n6, n8 and their first three u-derivatives (float64). With z = exp(2 pi i / 3),
// n6(u) = e^-u - 2 Re(e^{i pi/3} e^{z u}) and n8(u) = Re(e^{i pi/4} e^{z8 u}) + Re(e^{3 i pi/4} e^{z8' u}),
// z8 = e^{5 i pi/8}, z8' = e^{7 i pi/8}, so each derivative rotates the phases by arg z.
__device__ inline void green_n(double u, double (&n6)[4], double (&n8)[4]) {
  const double sq3 = 1.7320508075688772935, sin8 = 0.38268343236508977173, cos8 = 0.92387953251128675613;
  const double e2 = exp(-0.5 * u), e1 = e2 * e2;
  double sa, ca;
  sincospi(1.0 / 3.0 + u * 0.27566444771089604, &sa, &ca);
  n6[0] = e1 - 2.0 * e2 * ca;
  n6[1] = -e1 + e2 * ca + sq3 * e2 * sa;
  n6[2] = e1 + e2 * ca - sq3 * e2 * sa;
  n6[3] = -e1 - 2.0 * e2 * ca;
  const double e3 = exp(-u * sin8), e4 = exp(-u * cos8);
  double s1, c1, s2, c2;
  sincospi(0.25 + u * 0.29407998884120140, &s1, &c1);
  sincospi(0.75 + u * 0.12181191980055409, &s2, &c2);
  n8[0] = e3 * c1 + e4 * c2;
  n8[1] = -sin8 * e3 * c1 - cos8 * e3 * s1 - cos8 * e4 * c2 - sin8 * e4 * s2;
  n8[2] = 0.70710678118654752440 * (-e3 * c1 + e3 * s1 + e4 * c2 + e4 * s2);
  n8[3] = e3 * (cos8 * c1 + sin8 * s1) - e4 * (sin8 * c2 + cos8 * s2);
}

// Quintic Hermite basis of the fractional position t in a table interval: weights of the value,
// h x first and h^2 x second derivative at the left knot (b0, b1, b2) and at the right knot
// (b5, b4, b3).
struct HermiteF {
  float b0, b1, b2, b3, b4, b5;
};
__device__ __forceinline__ HermiteF hermite_basis(float t) {
  const float t2 = t * t, t3 = t2 * t;
  const float p = t3 * (10.0f + t * (-15.0f + 6.0f * t));   // 10 t^3 - 15 t^4 + 6 t^5
  HermiteF b;
  b.b5 = p;
  b.b0 = 1.0f - p;
  b.b1 = t + t3 * (-6.0f + t * (8.0f - 3.0f * t));
  b.b2 = 0.5f * t2 + t3 * (-1.5f + t * (1.5f - 0.5f * t));
  b.b3 = t3 * (0.5f + t * (-1.0f + 0.5f * t));
  b.b4 = t3 * (-4.0f + t * (7.0f - 3.0f * t));
  return b;
}
// G from the two knots' {G, h G1, h^2 G2, h^3 G3}; h dG/dk from the same two knots
__device__ __forceinline__ float herm_value(const HermiteF& hb, const float4& a, const float4& b) {
  return hb.b0 * a.x + hb.b1 * a.y + hb.b2 * a.z + hb.b5 * b.x + hb.b4 * b.y + hb.b3 * b.z;
}
__device__ __forceinline__ float herm_slope(const HermiteF& hb, const float4& a, const float4& b) {
  return hb.b0 * a.y + hb.b1 * a.z + hb.b2 * a.w + hb.b5 * b.y + hb.b4 * b.z + hb.b3 * b.w;
}

// G and dG/dk of one pair from its table row at interval j (basis hb, 1/h = inv_h).
__device__ __forceinline__ void green_lookup(const float4* __restrict__ row, int j, const HermiteF& hb, float inv_h,
                                             float& G, float& dG) {
  const float4 a = row[j], b = row[j + 1];
  G = herm_value(hb, a, b);
  dG = herm_slope(hb, a, b) * inv_h;
}

// Division of 32-bit unsigned values by a runtime-invariant divisor (round-up multiplier method):
// q = (t + ((n - t) >> 1)) >> (s - 1), t = umulhi(n, m), for every n < 2^32.
struct FastDiv {
  uint32_t d, m, s;
};
inline FastDiv make_fastdiv(uint32_t d) {
  FastDiv f{d, 0u, 0u};
  if (d > 1) {
    uint32_t l = 0;
    while ((1ull << l) < d) ++l;
    f.m = (uint32_t)((((1ull << 32) * ((1ull << l) - d)) / d) + 1);
    f.s = l;
  }
  return f;
}
__device__ __forceinline__ uint32_t fdiv(uint32_t n, const FastDiv& f) {
  if (f.d == 1) return n;
  const uint32_t t = __umulhi(n, f.m);
  return (t + ((n - t) >> 1)) >> (f.s - 1);
}

// floor division / modulo for possibly negative ints
__device__ __forceinline__ int floordiv(int a, int b) { return (a >= 0) ? a / b : -((-a + b - 1) / b); }
__device__ __forceinline__ int posmod(int a, int b) { int m = a % b; return m < 0 ? m + b : m; }

}  // namespace fd3

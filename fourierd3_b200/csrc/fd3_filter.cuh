// Shared device code of the reciprocal-space filters: k-point geometry, the mixed form's
// Green-table lookup position, and the per-k-point filter of up to 8 species
// (src/fourierd3/kspace_filter_d3.py:29-70, src/fourierd3/pair_pot.py:113-228).
#pragma once
#include "fd3_mesh_impl.cuh"

namespace fd3 {

// 1 / h of the table for this cell and mesh, in float, the same in every kernel that reads it
__device__ __forceinline__ float green_inv_h(const MeshDev& g, const CellInfo* __restrict__ ci) {
  double rec[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) rec[c] = ci->recip[c];
  const int n[3] = {g.n[0], g.n[1], g.n[2]};
  return (float)(kGreenKnots / green_kmax(rec, n));
}

__device__ __forceinline__ void table_pos(float k, float inv_h, int& j, HermiteF& hb) {
  const float t = k * inv_h;
  j = (int)t;
  if (j > kGreenKnots - 1) j = kGreenKnots - 1;
  hb = hermite_basis(t - (float)j);
}

// ------------------------------------------------------------------ filter
template <typename T> struct Cplx;
template <> struct Cplx<double> { using type = double2; };
template <> struct Cplx<float> { using type = float2; };

constexpr int kFilterThreads = 256;

// exact float64 SPME window sinc(m/n)^(2p), clamped at 1e-10 (used when no table is given)
__device__ __forceinline__ double sinc_pi(double x) { return x == 0.0 ? 1.0 : sin(kPi * x) / (kPi * x); }

// Geometry of rfft k-point k: k-vector (torch fftfreq order on x, y; rfftfreq on z), |k|, the
// SPME window, the Hermitian weight (1 on the first and last z-plane, pair_pot.py:213-218) and,
// on the self-conjugate planes, the |k| of the stored conjugate partner when it differs.
// Per-k geometry in precision T (double for the plain form, float for the mixed form):
// k-vector, |k|, the SPME window, the Hermitian weight (1 on the first and last z-plane,
// pair_pot.py:213-218) and, on the self-conjugate planes, the |k| of the stored conjugate
// partner when it differs. The reciprocal rows are hoisted into registers by the caller.
// |k| from |k|^2: float64 sqrt, or in float the hardware reciprocal square root times |k|^2
// (a few ulp; the mixed form's tolerance is orders of magnitude wider)
__device__ __forceinline__ double knorm_of(double k2) { return sqrt(k2); }
__device__ __forceinline__ float knorm_of(float k2) { return k2 > 0.f ? k2 * rsqrtf(k2) : 0.f; }

template <typename T>
struct KPoint {
  T kv[3], knorm, inv_sc, wk, kpart;
  bool partner;
};

template <typename T>
__device__ __forceinline__ KPoint<T> kpoint_idx(const MeshDev& g, int ix, int iy, int iz, size_t k, const T (&rc)[9],
                                                const float* __restrict__ deconv, int spme, int P) {
  KPoint<T> q;
  const int mx = ix <= (g.n[0] - 1) / 2 ? ix : ix - g.n[0];
  const int my = iy <= (g.n[1] - 1) / 2 ? iy : iy - g.n[1];
  const int mz = iz;
#pragma unroll
  for (int c = 0; c < 3; ++c) q.kv[c] = T(mx) * rc[c] + T(my) * rc[3 + c] + T(mz) * rc[6 + c];
  q.knorm = knorm_of(q.kv[0] * q.kv[0] + q.kv[1] * q.kv[1] + q.kv[2] * q.kv[2]);
  if (sizeof(T) == 4 && spme && g.win_axes) {
    // mixed form: the window is separable, sinc(mx/nx)^2p sinc(my/ny)^2p sinc(mz/nz)^2p (clamped
    // at 1e-10 like the table); three per-axis values that stay in L1 instead of one table read
    const float* wa = g.win_axes;
    const float w = wa[ix] * wa[g.n[0] + iy] * wa[g.n[0] + g.n[1] + iz];
    q.inv_sc = T(rcp_t(w < 1e-10f ? 1e-10f : w));
  } else if (sizeof(T) == 4 && spme && deconv) {
    q.inv_sc = T(rcp_t(deconv[k]));   // mixed form: the float32 window inverted (hardware reciprocal)
  } else {
    double sc = 1.0;
    if (spme) {
      if (deconv) {
        sc = (double)deconv[k];
      } else {
        const double nzf = (double)(2 * (g.nzh - 1));
        double v = sinc_pi(mx / (double)g.n[0]) * sinc_pi(my / (double)g.n[1]) * sinc_pi(mz / nzf);
        v = pow(v, 2.0 * P);
        sc = v < 1e-10 ? 1e-10 : v;
      }
    }
    q.inv_sc = (T)(1.0 / sc);
  }
  q.wk = (iz == 0 || iz == g.nzh - 1) ? T(1) : T(2);
  // Self-conjugate planes (kz = 0 and the z-Nyquist plane): the entry at (ix, iy) and its conjugate
  // partner (-ix, -iy) are both stored, but at the Nyquist rows their k-vectors differ in a
  // triclinic cell, so G(k) != G(k'). The inverse FFT needs a Hermitian input; using
  // (G(k) + G(k')) / 2 for H keeps the gradient the exact derivative of the energy sum.
  q.partner = false;
  q.kpart = q.knorm;
  const bool plane = (iz == 0) || (iz == g.nzh - 1 && iz > 0);
  if (plane) {
    const int px = ix == 0 ? 0 : g.n[0] - ix, py = iy == 0 ? 0 : g.n[1] - iy;   // (n - i) mod n
    const int qx = px <= (g.n[0] - 1) / 2 ? px : px - g.n[0];
    const int qy = py <= (g.n[1] - 1) / 2 ? py : py - g.n[1];
    if (qx != -mx || qy != -my || mz != 0) {
      T kp[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) kp[c] = T(qx) * rc[c] + T(qy) * rc[3 + c] + T(mz) * rc[6 + c];
      q.kpart = knorm_of(kp[0] * kp[0] + kp[1] * kp[1] + kp[2] * kp[2]);
      q.partner = q.kpart != q.knorm;
    }
  }
  return q;
}

// k-point k of the rfft half mesh (flat index, z fastest)
template <typename T>
__device__ __forceinline__ KPoint<T> kpoint(const MeshDev& g, size_t k, const T (&rc)[9],
                                            const float* __restrict__ deconv, int spme, int P) {
  const uint32_t kq = fdiv((uint32_t)k, g.div_nzh);
  const int iz = (int)((uint32_t)k - kq * (uint32_t)g.nzh);
  const uint32_t kqq = fdiv(kq, g.div_ny);
  const int iy = (int)(kq - kqq * (uint32_t)g.n[1]);
  return kpoint_idx<T>(g, (int)kqq, iy, iz, k, rc, deconv, spme, P);
}

template <typename T>
__device__ __forceinline__ void load_recip(const CellInfo* __restrict__ ci, T (&rc)[9]) {
#pragma unroll
  for (int c = 0; c < 9; ++c) rc[c] = (T)ci->recip[c];
}

// Per-k virial term f k_a k_b / |k| (f = w_k dq), added to the float64 block accumulators.
template <typename T>
__device__ __forceinline__ void virial_acc(const KPoint<T>& q, T dq, double* acc) {
  if (q.knorm > T(0)) {
    // float: one hardware reciprocal instead of a division (the mixed form's virial)
    const T f = sizeof(T) == 4 ? T(q.wk * dq * rcp_t((float)q.knorm)) : q.wk * dq / q.knorm;
    acc[1] += (double)(f * q.kv[0] * q.kv[0]);
    acc[2] += (double)(f * q.kv[1] * q.kv[1]);
    acc[3] += (double)(f * q.kv[2] * q.kv[2]);
    acc[4] += (double)(f * q.kv[0] * q.kv[1]);
    acc[5] += (double)(f * q.kv[0] * q.kv[2]);
    acc[6] += (double)(f * q.kv[1] * q.kv[2]);
  }
}


// G, dG and the Hermitian-averaged Gh of every species pair at one k-point (float64 closed
// form, or the mixed form's table), each divided by the SPME window; unused slots are zero.
template <typename T, int MAXS>
__device__ __forceinline__ void green_block(const KPoint<T>& q, int S,
                                            const typename GreenPairOf<T>::type* __restrict__ gp,
                                            const float4* __restrict__ gtab, float inv_h, T s6, T s8,
                                            T (&G)[MAXS][MAXS], T (&dG)[MAXS][MAXS], T (&Gh)[MAXS][MAXS]) {
  int tj = 0;
  HermiteF hb{};
  if constexpr (sizeof(T) == 4) table_pos(q.knorm, inv_h, tj, hb);
#pragma unroll
  for (int X = 0; X < MAXS; ++X)
#pragma unroll
    for (int Y = X; Y < MAXS; ++Y) {
      T gv = T(0), dv = T(0);
      if (X < S && Y < S) {
        if constexpr (sizeof(T) == 4) {
          const int pi = X * S - X * (X - 1) / 2 + (Y - X);
          green_lookup(gtab + (size_t)pi * (kGreenKnots + 1), tj, hb, inv_h, gv, dv);
        } else {
          green_eval<T>(gp[X * S + Y], q.knorm, s6, s8, gv, dv);
        }
        gv *= q.inv_sc;
        dv *= q.inv_sc;
      }
      G[X][Y] = G[Y][X] = gv;
      dG[X][Y] = dG[Y][X] = dv;
      Gh[X][Y] = Gh[Y][X] = gv;
    }
  if (q.partner) {
    int pj = 0;
    HermiteF pb{};
    if constexpr (sizeof(T) == 4) table_pos(q.kpart, inv_h, pj, pb);
#pragma unroll
    for (int X = 0; X < MAXS; ++X)
#pragma unroll
      for (int Y = X; Y < MAXS; ++Y)
        if (X < S && Y < S) {
          T gv, dv;
          if constexpr (sizeof(T) == 4) {
            const int pi = X * S - X * (X - 1) / 2 + (Y - X);
            green_lookup(gtab + (size_t)pi * (kGreenKnots + 1), pj, pb, inv_h, gv, dv);
          } else {
            green_eval<T>(gp[X * S + Y], q.kpart, s6, s8, gv, dv);
          }
          Gh[X][Y] = Gh[Y][X] = T(0.5) * (G[X][Y] + gv * q.inv_sc);
        }
  }
}

// Filter of one k-point for up to MAXS species: G, dG and Gh of every pair (green_block), the
// pair sums of the energy and virial, and H_X = sum_Y Gh_XY S_Y written over the S*R spectrum
// values v[c * cs] (c = X R + r). Ranks are processed in chunks of MAXR whose S x MAXR values are
// all loaded before any arithmetic. Per-k terms are formed in T and accumulated in float64 into
// acc[0..6].
template <typename T, int MAXS, int MAXR>
__device__ __forceinline__ void filter_point(const KPoint<T>& q, int S, int R,
                                             const typename GreenPairOf<T>::type* __restrict__ gp,
                                             const float4* __restrict__ gtab, float inv_h, T s6, T s8,
                                             const Tables* __restrict__ tab, typename Cplx<T>::type* v, size_t cs,
                                             double* acc) {
  using C2 = typename Cplx<T>::type;
  T G[MAXS][MAXS], dG[MAXS][MAXS], Gh[MAXS][MAXS];
  green_block<T, MAXS>(q, S, gp, gtab, inv_h, s6, s8, G, dG, Gh);
  T qq = T(0), dq = T(0);
  const bool full = S == MAXS && R % MAXR == 0;   // every slot holds a channel: no predication
  const size_t xs = (size_t)R * cs;               // channel stride between species
  for (int r0 = 0; r0 < R; r0 += MAXR) {
    C2 sv[MAXR][MAXS];
    typename Cplx<T>::type* vr = v + (size_t)r0 * cs;
    if (full) {
#pragma unroll
      for (int r = 0; r < MAXR; ++r)
#pragma unroll
        for (int X = 0; X < MAXS; ++X) sv[r][X] = vr[X * xs + r * cs];
    } else {
#pragma unroll
      for (int r = 0; r < MAXR; ++r)
#pragma unroll
        for (int X = 0; X < MAXS; ++X)
          sv[r][X] = (X < S && r0 + r < R) ? v[((size_t)X * R + r0 + r) * cs] : C2{T(0), T(0)};
    }
#pragma unroll
    for (int r = 0; r < MAXR; ++r) {
      T qr = T(0), dqr = T(0);
#pragma unroll
      for (int X = 0; X < MAXS; ++X) {
        T hre = T(0), him = T(0);
#pragma unroll
        for (int Y = 0; Y < MAXS; ++Y) {
          hre += Gh[X][Y] * sv[r][Y].x;
          him += Gh[X][Y] * sv[r][Y].y;
          const T re = sv[r][X].x * sv[r][Y].x + sv[r][X].y * sv[r][Y].y;
          qr += G[X][Y] * re;
          dqr += dG[X][Y] * re;
        }
        if (full)
          vr[X * xs + r * cs] = C2{hre, him};
        else if (X < S && r0 + r < R)
          v[((size_t)X * R + r0 + r) * cs] = C2{hre, him};
      }
      if (r0 + r < R) {
        const T lam = (T)tab->eigs[r0 + r];
        qq += lam * qr;
        dq += lam * dqr;
      }
    }
  }
  acc[0] += (double)(q.wk * qq);
  virial_acc<T>(q, dq, acc);
}

}  // namespace fd3

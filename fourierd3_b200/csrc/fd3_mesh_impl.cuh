// SPME / PME spread and gather kernel templates (reference: src/fourierd3/mesh_interpolator_d3.py:74-189,
// src/fourierd3/kspace_filter_d3.py:29-98, src/fourierd3/pair_pot.py:113-228, core.py:553-581).
//
// spread  : one CTA owns one mesh tile (8x8x8 points) and one species; it pulls the atoms whose
//           stencil can reach the tile from the counting-sorted (tile, species) segments, and every
//           thread sums the contributions for its own points. Each mesh value is written exactly
//           once, in a fixed summation order: no global atomics, no zero-fill pass, deterministic.
// filter  : one thread per rfft k-point; evaluates G_XY(|k|) and dG/d|k| in registers, applies the
//           deconvolution window and the Hermitian weight, accumulates the energy and the virial
//           (float64), and overwrites the spectrum with H_X = sum_Y G_XY S_Y for the inverse FFT.
// gather  : one warp per atom (tile-sorted order); sums phi over the p^3 stencil for the C6-factor
//           adjoint and the spline-gradient force.
#include <math.h>

#pragma once
#include "fd3_internal.h"

namespace fd3 {

struct MeshDev {
  int n[3], nzh, t[3], nt[3], ns[3], S, R;
};
static inline MeshDev to_dev(const MeshGeom& g) {
  MeshDev d;
  for (int a = 0; a < 3; ++a) {
    d.n[a] = g.n[a];
    d.t[a] = g.t[a];
    d.nt[a] = g.nt[a];
    d.ns[a] = g.ns[a];
  }
  d.nzh = g.nzh;
  d.S = g.S;
  d.R = g.R;
  return d;
}

// Fractional mesh coordinate of one atom along all axes and its first stencil node.
// MeshInterpolator.compute_weights (core.py:555): u = n * (x @ inv); reference node round(u)
// (odd p) or floor(u) (even p); local x = u - ref (odd) or u - ref - 1/2 (even).
template <typename T>
__device__ __forceinline__ void mesh_locate(const double* __restrict__ pos, int i, double ps, const CellInfo* ci,
                                            const int* n, int P, int* base, T* xl) {
  const double x0 = pos[3 * i] * ps, x1 = pos[3 * i + 1] * ps, x2 = pos[3 * i + 2] * ps;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double u = n[a] * (x0 * ci->inv[a] + x1 * ci->inv[3 + a] + x2 * ci->inv[6 + a]);
    double ref, x;
    if (P % 2 == 0) {
      ref = floor(u);
      x = u - (ref + 0.5);
    } else {
      ref = rint(u);
      x = u - ref;
    }
    const long long b = (long long)ref + (1 - (P + 1) / 2);
    long long bm = b % n[a];
    if (bm < 0) bm += n[a];
    base[a] = (int)bm;
    xl[a] = (T)x;
  }
}

template <int P, bool LAG, typename T>
__device__ __forceinline__ void stencil_weights(T x, T* w, T* dw) {
  if (LAG)
    lagrange<P, T>(x, w, dw);
  else
    bspline<P, T>(x, w, dw);
}

// ------------------------------------------------------------------ spread
constexpr int kSpreadThreads = 256;
constexpr int kSpreadPts = 2;          // points per thread (512-point tile)

// candidate atoms staged in shared memory per pass (fits the 48 KB static limit)
template <typename T, int P, int MAXR>
struct SpreadChunk {
  static constexpr int bytes_per = 12 + (3 * P + MAXR) * (int)sizeof(T);
  static constexpr int value = bytes_per * 128 <= 40000 ? 128 : (bytes_per * 64 <= 40000 ? 64 : 32);
};

template <typename T, int P, bool LAG, int MAXR>
__global__ void __launch_bounds__(kSpreadThreads) k_spread(MeshDev g, const double* __restrict__ pos, double ps,
                                                            const double* __restrict__ c6,
                                                            const CellInfo* __restrict__ ci,
                                                            const int* __restrict__ key_start,
                                                            const int* __restrict__ order, T* __restrict__ rho) {
  constexpr int kChunk = SpreadChunk<T, P, MAXR>::value;
  __shared__ int s_base[kChunk][3];
  __shared__ T s_w[kChunk][3][P];
  __shared__ T s_c[kChunk][MAXR];
  __shared__ int s_warp_cnt[kSpreadThreads / 32];
  __shared__ int s_nc;

  const int X = blockIdx.y;
  const int tile = blockIdx.x;
  const int tz = tile % g.nt[2];
  const int ty = (tile / g.nt[2]) % g.nt[1];
  const int tx = tile / (g.nt[2] * g.nt[1]);
  const int t0[3] = {tx * g.t[0], ty * g.t[1], tz * g.t[2]};
  const int npts = g.t[0] * g.t[1] * g.t[2];
  const int pf[3] = {P < g.n[0] ? P : g.n[0], P < g.n[1] ? P : g.n[1], P < g.n[2] ? P : g.n[2]};
  const int R = g.R;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;

  int pm[kSpreadPts][3];
  bool pv[kSpreadPts];
#pragma unroll
  for (int q = 0; q < kSpreadPts; ++q) {
    const int id = threadIdx.x + q * kSpreadThreads;
    pv[q] = id < npts;
    const int lz = id % g.t[2], ly = (id / g.t[2]) % g.t[1], lx = id / (g.t[2] * g.t[1]);
    pm[q][0] = t0[0] + lx;
    pm[q][1] = t0[1] + ly;
    pm[q][2] = t0[2] + lz;
  }
  T acc[kSpreadPts][MAXR];
#pragma unroll
  for (int q = 0; q < kSpreadPts; ++q)
#pragma unroll
    for (int r = 0; r < MAXR; ++r) acc[q][r] = T(0);

  for (int sxo = 0; sxo < g.ns[0]; ++sxo)
    for (int syo = 0; syo < g.ns[1]; ++syo)
      for (int szo = 0; szo < g.ns[2]; ++szo) {
        const int sx = posmod(tx - sxo, g.nt[0]);
        const int sy = posmod(ty - syo, g.nt[1]);
        const int sz = posmod(tz - szo, g.nt[2]);
        const int key = ((sx * g.nt[1] + sy) * g.nt[2] + sz) * g.S + X;
        const int a0 = key_start[key], a1 = key_start[key + 1];
        for (int c0 = a0; c0 < a1; c0 += kSpreadThreads) {
          // each thread examines one candidate; keepers are compacted in candidate order
          const int ca = c0 + threadIdx.x;
          bool keep = false;
          int base[3] = {0, 0, 0};
          T xl[3] = {T(0), T(0), T(0)};
          int atom = 0;
          if (ca < a1) {
            atom = order[ca];
            mesh_locate<T>(pos, atom, ps, ci, g.n, P, base, xl);
            keep = true;
#pragma unroll
            for (int a = 0; a < 3; ++a) {
              int d = t0[a] - base[a];
              if (d < 0) d += g.n[a];
              // the stencil covers offsets [0, pf) from base; the tile covers [d, d + t)
              if (!(d < pf[a] || d + g.t[a] > g.n[a])) keep = false;
            }
          }
          const unsigned bal = __ballot_sync(0xffffffffu, keep);
          if (lane == 0) s_warp_cnt[wid] = __popc(bal);
          __syncthreads();
          int off = 0, tot = 0;
          for (int w = 0; w < kSpreadThreads / 32; ++w) {
            if (w < wid) off += s_warp_cnt[w];
            tot += s_warp_cnt[w];
          }
          __syncthreads();   // s_warp_cnt is rewritten by the next candidate pass
          // tot <= kSpreadThreads; stage in two halves if it exceeds the chunk
          for (int h0 = 0; h0 < tot; h0 += kChunk) {
            const int slot = off + __popc(bal & ((1u << lane) - 1u)) - h0;
            if (keep && slot >= 0 && slot < kChunk) {
              T w[3][P], dw[P];
              stencil_weights<P, LAG, T>(xl[0], w[0], dw);
              stencil_weights<P, LAG, T>(xl[1], w[1], dw);
              stencil_weights<P, LAG, T>(xl[2], w[2], dw);
#pragma unroll
              for (int a = 0; a < 3; ++a) {
                s_base[slot][a] = base[a];
                if (pf[a] == P) {
#pragma unroll
                  for (int k = 0; k < P; ++k) s_w[slot][a][k] = w[a][k];
                } else {
                  // fold stencil nodes that wrap onto the same mesh point (n < p)
                  for (int k = 0; k < P; ++k) s_w[slot][a][k] = T(0);
                  for (int k = 0; k < P; ++k) s_w[slot][a][k % pf[a]] += w[a][k];
                }
              }
#pragma unroll
              for (int r = 0; r < MAXR; ++r) s_c[slot][r] = r < R ? (T)c6[(size_t)atom * R + r] : T(0);
            }
            if (threadIdx.x == 0) s_nc = min(kChunk, tot - h0);
            __syncthreads();
            const int nc = s_nc;
#pragma unroll
            for (int q = 0; q < kSpreadPts; ++q) {
              if (!pv[q]) continue;
              for (int c = 0; c < nc; ++c) {
                int kx = pm[q][0] - s_base[c][0];
                if (kx < 0) kx += g.n[0];
                if (kx >= pf[0]) continue;
                int ky = pm[q][1] - s_base[c][1];
                if (ky < 0) ky += g.n[1];
                if (ky >= pf[1]) continue;
                int kz = pm[q][2] - s_base[c][2];
                if (kz < 0) kz += g.n[2];
                if (kz >= pf[2]) continue;
                const T w = s_w[c][0][kx] * s_w[c][1][ky] * s_w[c][2][kz];
#pragma unroll
                for (int r = 0; r < MAXR; ++r) acc[q][r] += w * s_c[c][r];
              }
            }
            __syncthreads();
          }
        }
      }
  const size_t M = (size_t)g.n[0] * g.n[1] * g.n[2];
#pragma unroll
  for (int q = 0; q < kSpreadPts; ++q) {
    if (!pv[q]) continue;
    const size_t m = ((size_t)pm[q][0] * g.n[1] + pm[q][1]) * g.n[2] + pm[q][2];
#pragma unroll
    for (int r = 0; r < MAXR; ++r)
      if (r < R) rho[((size_t)X * R + r) * M + m] = acc[q][r];
  }
}

template <typename T, int P, bool LAG>
static int spread_r(const MeshGeom& mg, dim3 grid, const double* pos, double ps, const double* c6,
                    const CellInfo* ci, const int* ks, const int* order, T* rho, cudaStream_t s) {
  const MeshDev g = to_dev(mg);
  if (mg.R <= 4)
    k_spread<T, P, LAG, 4><<<grid, kSpreadThreads, 0, s>>>(g, pos, ps, c6, ci, ks, order, rho);
  else if (mg.R <= 8)
    k_spread<T, P, LAG, 8><<<grid, kSpreadThreads, 0, s>>>(g, pos, ps, c6, ci, ks, order, rho);
  else if (mg.R <= 16)
    k_spread<T, P, LAG, 16><<<grid, kSpreadThreads, 0, s>>>(g, pos, ps, c6, ci, ks, order, rho);
  else
    k_spread<T, P, LAG, 32><<<grid, kSpreadThreads, 0, s>>>(g, pos, ps, c6, ci, ks, order, rho);
  FD3_LAUNCHED();
  return FD3_OK;
}

template <typename T>
int launch_spread(const MeshGeom& mg, const double* pos, double pos_scale, const int32_t* species,
                  const double* c6, const CellInfo* ci, const int* key_start, const int* order, T* rho,
                  cudaStream_t s) {
  (void)species;
  if (mg.R > 32 || mg.order < 1 || mg.order > FD3_MAX_ORDER) return FD3_EINVAL;
  const dim3 grid(mg.nt[0] * mg.nt[1] * mg.nt[2], mg.S);
#define FD3_SPREAD_CASE(PP)                                                                          \
  case PP:                                                                                           \
    return mg.lagrange ? spread_r<T, PP, true>(mg, grid, pos, pos_scale, c6, ci, key_start, order, rho, s) \
                       : spread_r<T, PP, false>(mg, grid, pos, pos_scale, c6, ci, key_start, order, rho, s);
  switch (mg.order) {
    FD3_SPREAD_CASE(1)
    FD3_SPREAD_CASE(2)
    FD3_SPREAD_CASE(3)
    FD3_SPREAD_CASE(4)
    FD3_SPREAD_CASE(5)
    FD3_SPREAD_CASE(6)
    FD3_SPREAD_CASE(7)
    FD3_SPREAD_CASE(8)
  }
#undef FD3_SPREAD_CASE
  return FD3_EINVAL;
}
// ------------------------------------------------------------------ gather
constexpr int kGatherWarps = 8;

template <typename T, int P, bool LAG, int MAXR>
__global__ void __launch_bounds__(32 * kGatherWarps) k_gather(MeshDev g, int n, const double* __restrict__ pos,
                                                              double ps, const int32_t* __restrict__ species,
                                                              const double* __restrict__ c6,
                                                              const double* __restrict__ dc6,
                                                              const CellInfo* __restrict__ ci,
                                                              const Tables* __restrict__ tab,
                                                              const int* __restrict__ order,
                                                              const T* __restrict__ phi, double* __restrict__ gcn,
                                                              double* __restrict__ gpos,
                                                              double* __restrict__ mcell_part) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int t = blockIdx.x * kGatherWarps + wid;
  const int R = g.R;
  double mc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (t < n) {
    const int i = order[t];
    const int s = species[i];
    int base[3];
    T xl[3];
    mesh_locate<T>(pos, i, ps, ci, g.n, P, base, xl);
    T w[3][P], dw[3][P];
#pragma unroll
    for (int a = 0; a < 3; ++a) stencil_weights<P, LAG, T>(xl[a], w[a], dw[a]);
    double cl[MAXR];
#pragma unroll
    for (int r = 0; r < MAXR; ++r) cl[r] = r < R ? c6[(size_t)i * R + r] * tab->eigs[r] : 0.0;
    const size_t M = (size_t)g.n[0] * g.n[1] * g.n[2];
    double pr[MAXR];
#pragma unroll
    for (int r = 0; r < MAXR; ++r) pr[r] = 0.0;
    double gu0 = 0, gu1 = 0, gu2 = 0;
    constexpr int P3 = P * P * P;
    for (int qn = lane; qn < P3; qn += 32) {
      const int kx = qn / (P * P), ky = (qn / P) % P, kz = qn % P;
      int ix = base[0] + kx; if (ix >= g.n[0]) ix -= g.n[0] * (ix / g.n[0]);
      int iy = base[1] + ky; if (iy >= g.n[1]) iy -= g.n[1] * (iy / g.n[1]);
      int iz = base[2] + kz; if (iz >= g.n[2]) iz -= g.n[2] * (iz / g.n[2]);
      const size_t m = ((size_t)ix * g.n[1] + iy) * g.n[2] + iz;
      const T W = w[0][kx] * w[1][ky] * w[2][kz];
      const T Wx = dw[0][kx] * w[1][ky] * w[2][kz];
      const T Wy = w[0][kx] * dw[1][ky] * w[2][kz];
      const T Wz = w[0][kx] * w[1][ky] * dw[2][kz];
      double cp = 0.0;
#pragma unroll
      for (int r = 0; r < MAXR; ++r) {
        if (r < R) {
          const double ph = (double)phi[((size_t)s * R + r) * M + m];
          pr[r] += (double)W * ph;
          cp += cl[r] * ph;
        }
      }
      gu0 += (double)Wx * cp;
      gu1 += (double)Wy * cp;
      gu2 += (double)Wz * cp;
    }
#pragma unroll
    for (int r = 0; r < MAXR; ++r) pr[r] = warp_sum(pr[r]);
    gu0 = warp_sum(gu0);
    gu1 = warp_sum(gu1);
    gu2 = warp_sum(gu2);
    const double inv_vol = 1.0 / ci->volume;
    // dE/dc_r = -(lambda_r / Omega) P_r + lambda_r c_r phi_ss(0); g = sum_r dE/dc_r dc_r/dCN
    double gsum = 0.0;
#pragma unroll
    for (int r = 0; r < MAXR; ++r) {
      if (r < R) {
        const double lam = tab->eigs[r];
        const double c = c6[(size_t)i * R + r];
        const double dEdc = -lam * inv_vol * pr[r] + lam * c * tab->selfcont[s];
        gsum += dEdc * dc6[(size_t)i * R + r];
      }
    }
    // dE/du_a = -(1/Omega) sum_r lambda_r c_r sum_m phi dW/du_a; dE/dx_b = sum_a dE/du_a n_a inv[b][a]
    const double du[3] = {-inv_vol * gu0, -inv_vol * gu1, -inv_vol * gu2};
    double gx[3];
#pragma unroll
    for (int b = 0; b < 3; ++b)
      gx[b] = du[0] * g.n[0] * ci->inv[3 * b + 0] + du[1] * g.n[1] * ci->inv[3 * b + 1] +
              du[2] * g.n[2] * ci->inv[3 * b + 2];
    if (lane == 0) {
      gcn[i] = gsum;
      gpos[3 * i] = gx[0];
      gpos[3 * i + 1] = gx[1];
      gpos[3 * i + 2] = gx[2];
      // mesh part of dE/dcell with positions fixed: -sum_i s_iA g_ia (s = fractional coordinate)
      if (mcell_part) {
        const double x0 = pos[3 * i] * ps, x1 = pos[3 * i + 1] * ps, x2 = pos[3 * i + 2] * ps;
        double sf[3];
#pragma unroll
        for (int A = 0; A < 3; ++A) sf[A] = x0 * ci->inv[A] + x1 * ci->inv[3 + A] + x2 * ci->inv[6 + A];
#pragma unroll
        for (int A = 0; A < 3; ++A)
#pragma unroll
          for (int a = 0; a < 3; ++a) mc[3 * A + a] = sf[A] * gx[a];
      }
    }
  }
  if (mcell_part) block_sum_store<9>(mc, mcell_part + 9 * blockIdx.x);
}

template <typename T, int P, bool LAG>
static int gather_r(const MeshGeom& mg, int blocks, int n, const double* pos, double ps, const int32_t* species,
                    const double* c6, const double* dc6, const CellInfo* ci, const Tables* tab, const int* order,
                    const T* phi, double* gcn, double* gpos, double* mcell, cudaStream_t s) {
  const MeshDev g = to_dev(mg);
  const int tb = 32 * kGatherWarps;
  if (mg.R <= 4)
    k_gather<T, P, LAG, 4><<<blocks, tb, 0, s>>>(g, n, pos, ps, species, c6, dc6, ci, tab, order, phi, gcn, gpos,
                                                  mcell);
  else if (mg.R <= 8)
    k_gather<T, P, LAG, 8><<<blocks, tb, 0, s>>>(g, n, pos, ps, species, c6, dc6, ci, tab, order, phi, gcn, gpos,
                                                  mcell);
  else if (mg.R <= 16)
    k_gather<T, P, LAG, 16><<<blocks, tb, 0, s>>>(g, n, pos, ps, species, c6, dc6, ci, tab, order, phi, gcn, gpos,
                                                   mcell);
  else
    k_gather<T, P, LAG, 32><<<blocks, tb, 0, s>>>(g, n, pos, ps, species, c6, dc6, ci, tab, order, phi, gcn, gpos,
                                                   mcell);
  FD3_LAUNCHED();
  return FD3_OK;
}

template <typename T>
int launch_gather(const MeshGeom& mg, int n, const double* pos, double pos_scale, const int32_t* species,
                  const double* c6, const double* dc6, const CellInfo* ci, const Tables* tab, const int* order,
                  const T* phi, double* gcn, double* gpos, double* mcell_part, int* n_blocks, cudaStream_t s) {
  const int blocks = (n + kGatherWarps - 1) / kGatherWarps;
  *n_blocks = blocks;
  if (blocks == 0) return FD3_OK;
#define FD3_GATHER_CASE(PP)                                                                                   \
  case PP:                                                                                                    \
    return mg.lagrange ? gather_r<T, PP, true>(mg, blocks, n, pos, pos_scale, species, c6, dc6, ci, tab, order, \
                                               phi, gcn, gpos, mcell_part, s)                                 \
                       : gather_r<T, PP, false>(mg, blocks, n, pos, pos_scale, species, c6, dc6, ci, tab, order, \
                                                phi, gcn, gpos, mcell_part, s);
  switch (mg.order) {
    FD3_GATHER_CASE(1)
    FD3_GATHER_CASE(2)
    FD3_GATHER_CASE(3)
    FD3_GATHER_CASE(4)
    FD3_GATHER_CASE(5)
    FD3_GATHER_CASE(6)
    FD3_GATHER_CASE(7)
    FD3_GATHER_CASE(8)
  }
#undef FD3_GATHER_CASE
  return FD3_EINVAL;
}
}  // namespace fd3

// SPME / PME reciprocal-space kernels (reference: src/fourierd3/mesh_interpolator_d3.py:74-189,
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

#include "fd3_mesh_impl.cuh"

namespace fd3 {

// ------------------------------------------------------------------ cell info
__global__ void k_cellinfo(const double* __restrict__ cell, double scale, CellInfo* __restrict__ ci) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double m[9];
  for (int k = 0; k < 9; ++k) m[k] = cell[k] * scale;
  // utils.py:142-167 (adjugate / determinant) and utils.py:130-139 (cofactor determinant)
  const double c00 = m[4] * m[8] - m[5] * m[7];
  const double c01 = m[2] * m[7] - m[1] * m[8];
  const double c02 = m[1] * m[5] - m[2] * m[4];
  const double c10 = m[5] * m[6] - m[3] * m[8];
  const double c11 = m[0] * m[8] - m[2] * m[6];
  const double c12 = m[2] * m[3] - m[0] * m[5];
  const double c20 = m[3] * m[7] - m[4] * m[6];
  const double c21 = m[1] * m[6] - m[0] * m[7];
  const double c22 = m[0] * m[4] - m[1] * m[3];
  const double det = m[0] * c00 + m[1] * c10 + m[2] * c20;
  const double adj[9] = {c00, c01, c02, c10, c11, c12, c20, c21, c22};
  for (int k = 0; k < 9; ++k) {
    ci->cell[k] = m[k];
    ci->inv[k] = adj[k] / det;
  }
  // reciprocal rows b_i = 2 pi inv[:, i]
  for (int i = 0; i < 3; ++i)
    for (int c = 0; c < 3; ++c) ci->recip[3 * i + c] = 2.0 * kPi * ci->inv[3 * c + i];
  ci->volume = fabs(det);
}

int launch_cellinfo(const double* cell, double scale, CellInfo* ci, cudaStream_t s) {
  k_cellinfo<<<1, 32, 0, s>>>(cell, scale, ci);
  FD3_LAUNCHED();
  return FD3_OK;
}

__global__ void k_mesh_keys(MeshDev g, int n, int P, const double* __restrict__ pos, double ps,
                            const int32_t* __restrict__ species, const CellInfo* __restrict__ ci,
                            int* __restrict__ keys) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int base[3];
  double xl[3];
  mesh_locate<double>(pos, i, ps, ci, g.n, P, base, xl);
  const int tx = base[0] / g.t[0], ty = base[1] / g.t[1], tz = base[2] / g.t[2];
  keys[i] = ((tx * g.nt[1] + ty) * g.nt[2] + tz) * g.S + species[i];
}

int launch_mesh_keys(const MeshGeom& mg, int n, const double* pos, double pos_scale, const int32_t* species,
                     const CellInfo* ci, int* keys, cudaStream_t s) {
  if (n == 0) return FD3_OK;
  const int tb = 256;
  k_mesh_keys<<<(n + tb - 1) / tb, tb, 0, s>>>(to_dev(mg), n, mg.order, pos, pos_scale, species, ci, keys);
  FD3_LAUNCHED();
  return FD3_OK;
}

// ------------------------------------------------------------------ filter
template <typename T> struct Cplx;
template <> struct Cplx<double> { using type = double2; };
template <> struct Cplx<float> { using type = float2; };

constexpr int kFilterThreads = 256;

// exact float64 SPME window sinc(m/n)^(2p), clamped at 1e-10 (used when no table is given)
__device__ __forceinline__ double sinc_pi(double x) { return x == 0.0 ? 1.0 : sin(kPi * x) / (kPi * x); }

template <typename T, int MAXS>
__global__ void __launch_bounds__(kFilterThreads) k_filter(MeshDev g, int P, int spme,
                                                           const CellInfo* __restrict__ ci,
                                                           const GreenPair* __restrict__ gp,
                                                           const Tables* __restrict__ tab,
                                                           const float* __restrict__ deconv,
                                                           typename Cplx<T>::type* __restrict__ spec,
                                                           double* __restrict__ part) {
  using C2 = typename Cplx<T>::type;
  const int S = g.S, R = g.R;
  const size_t Mh = (size_t)g.n[0] * g.n[1] * g.nzh;
  const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  if (k < Mh) {
    const int iz = (int)(k % g.nzh);
    const int iy = (int)((k / g.nzh) % g.n[1]);
    const int ix = (int)(k / ((size_t)g.nzh * g.n[1]));
    // torch.fft.fftfreq order on x and y, rfftfreq on z
    const int mx = ix <= (g.n[0] - 1) / 2 ? ix : ix - g.n[0];
    const int my = iy <= (g.n[1] - 1) / 2 ? iy : iy - g.n[1];
    const int mz = iz;
    double kv[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) kv[c] = mx * ci->recip[c] + my * ci->recip[3 + c] + mz * ci->recip[6 + c];
    const double knorm = sqrt(kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2]);
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
    const double wk = (iz == 0 || iz == g.nzh - 1) ? 1.0 : 2.0;
    const T kt = (T)knorm;
    const T s6 = (T)tab->s6, s8 = (T)tab->s8;
    T G[MAXS][MAXS], dG[MAXS][MAXS], Gh[MAXS][MAXS];
#pragma unroll
    for (int X = 0; X < MAXS; ++X)
#pragma unroll
      for (int Y = X; Y < MAXS; ++Y) {
        if (X < S && Y < S) {
          T gv, dv;
          green_eval<T>(gp[X * S + Y], kt, s6, s8, gv, dv);
          G[X][Y] = (T)((double)gv / sc);
          dG[X][Y] = (T)((double)dv / sc);
        } else {
          G[X][Y] = T(0);
          dG[X][Y] = T(0);
        }
        G[Y][X] = G[X][Y];
        dG[Y][X] = dG[X][Y];
        Gh[X][Y] = G[X][Y];
        Gh[Y][X] = G[X][Y];
      }
    // Self-conjugate planes (kz = 0 and the z-Nyquist plane): the entry at index (ix, iy) and its
    // conjugate partner (-ix, -iy) are both stored, but at the Nyquist rows their k-vectors differ
    // in a triclinic cell, so G(k) != G(k'). The inverse FFT needs a Hermitian input; using
    // (G(k) + G(k')) / 2 for H keeps the gradient the exact derivative of the energy sum.
    const bool plane = (iz == 0) || (2 * iz == 2 * (g.nzh - 1) && iz > 0 && g.nzh > 1);
    if (plane) {
      const int px = (g.n[0] - ix) % g.n[0], py = (g.n[1] - iy) % g.n[1];
      const int qx = px <= (g.n[0] - 1) / 2 ? px : px - g.n[0];
      const int qy = py <= (g.n[1] - 1) / 2 ? py : py - g.n[1];
      if (qx != -mx || qy != -my || mz != 0) {
        double kp[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) kp[c] = qx * ci->recip[c] + qy * ci->recip[3 + c] + mz * ci->recip[6 + c];
        const T kpt = (T)sqrt(kp[0] * kp[0] + kp[1] * kp[1] + kp[2] * kp[2]);
#pragma unroll
        for (int X = 0; X < MAXS; ++X)
#pragma unroll
          for (int Y = X; Y < MAXS; ++Y) {
            if (X < S && Y < S) {
              T gv, dv;
              green_eval<T>(gp[X * S + Y], kpt, s6, s8, gv, dv);
              const T gpv = (T)((double)gv / sc);
              Gh[X][Y] = T(0.5) * (G[X][Y] + gpv);
              Gh[Y][X] = Gh[X][Y];
            }
          }
      }
    }
    double q = 0.0, dq = 0.0;
    for (int r = 0; r < R; ++r) {
      C2 sv[MAXS];
#pragma unroll
      for (int X = 0; X < MAXS; ++X) sv[X] = X < S ? spec[((size_t)X * R + r) * Mh + k] : C2{T(0), T(0)};
      double qr = 0.0, dqr = 0.0;
#pragma unroll
      for (int X = 0; X < MAXS; ++X) {
        T hre = T(0), him = T(0);
#pragma unroll
        for (int Y = 0; Y < MAXS; ++Y) {
          hre += Gh[X][Y] * sv[Y].x;
          him += Gh[X][Y] * sv[Y].y;
          const double re = (double)sv[X].x * (double)sv[Y].x + (double)sv[X].y * (double)sv[Y].y;
          qr += (double)G[X][Y] * re;
          dqr += (double)dG[X][Y] * re;
        }
        if (X < S) spec[((size_t)X * R + r) * Mh + k] = C2{hre, him};
      }
      q += tab->eigs[r] * qr;
      dq += tab->eigs[r] * dqr;
    }
    acc[0] = wk * q;
    if (knorm > 0.0) {
      const double f = wk * dq / knorm;
      acc[1] = f * kv[0] * kv[0];
      acc[2] = f * kv[1] * kv[1];
      acc[3] = f * kv[2] * kv[2];
      acc[4] = f * kv[0] * kv[1];
      acc[5] = f * kv[0] * kv[2];
      acc[6] = f * kv[1] * kv[2];
    }
  }
  block_sum_store<7>(acc, part + 7 * blockIdx.x);
}

template <typename T>
int launch_filter(const MeshGeom& mg, const CellInfo* ci, const GreenPair* gp, const Tables* tab,
                  const float* deconv, int spme, void* spec, double* part, int* n_blocks, cudaStream_t s) {
  using C2 = typename Cplx<T>::type;
  const size_t Mh = (size_t)mg.n[0] * mg.n[1] * mg.nzh;
  const int blocks = (int)((Mh + kFilterThreads - 1) / kFilterThreads);
  *n_blocks = blocks;
  const MeshDev g = to_dev(mg);
  C2* sp = reinterpret_cast<C2*>(spec);
  if (mg.S <= 1)
    k_filter<T, 1><<<blocks, kFilterThreads, 0, s>>>(g, mg.order, spme, ci, gp, tab, deconv, sp, part);
  else if (mg.S <= 2)
    k_filter<T, 2><<<blocks, kFilterThreads, 0, s>>>(g, mg.order, spme, ci, gp, tab, deconv, sp, part);
  else if (mg.S <= 4)
    k_filter<T, 4><<<blocks, kFilterThreads, 0, s>>>(g, mg.order, spme, ci, gp, tab, deconv, sp, part);
  else if (mg.S <= 8)
    k_filter<T, 8><<<blocks, kFilterThreads, 0, s>>>(g, mg.order, spme, ci, gp, tab, deconv, sp, part);
  else
    return FD3_EINVAL;
  FD3_LAUNCHED();
  return FD3_OK;
}
template int launch_filter<double>(const MeshGeom&, const CellInfo*, const GreenPair*, const Tables*, const float*,
                                   int, void*, double*, int*, cudaStream_t);
template int launch_filter<float>(const MeshGeom&, const CellInfo*, const GreenPair*, const Tables*, const float*,
                                  int, void*, double*, int*, cudaStream_t);

// ------------------------------------------------------------------ finalize
// mode 0: energy [Hartree] and dE/dcell [Hartree/Bohr] with positions/shifts fixed (edge path)
// mode 1: energy [eV] and ASE stress [eV/A^3] = (dE/dstrain) / Omega (fused path)
__global__ void k_finalize(Partials p, const CellInfo* __restrict__ ci, int mode, double e_scale,
                           double* __restrict__ energy, double* __restrict__ out9) {
  double v[1 + 7 + 9 + 9];
  for (int k = 0; k < 26; ++k) v[k] = 0.0;
  for (int b = threadIdx.x; b < p.n_self; b += blockDim.x) v[0] += p.self[b];
  for (int b = threadIdx.x; b < p.n_kspc; b += blockDim.x)
    for (int c = 0; c < 7; ++c) v[1 + c] += p.kspc[7 * b + c];
  for (int b = threadIdx.x; b < p.n_cnv; b += blockDim.x)
    for (int c = 0; c < 9; ++c) v[8 + c] += p.cnv[9 * b + c];
  for (int b = threadIdx.x; b < p.n_mcell; b += blockDim.x)
    for (int c = 0; c < 9; ++c) v[17 + c] += p.mcell[9 * b + c];
  __shared__ double tot[26];
  block_sum_store<26>(v, tot);
  if (threadIdx.x != 0) return;
  const double vol = ci->volume;
  const double self = tot[0], Q = tot[1];
  const double E = Q / (-2.0 * vol) + self / 2.0;     // core.py:581
  // strain virial of the k-space energy: (Q delta_ab + V_ab) / (2 Omega)
  double Wk[9];
  const double Vs[9] = {tot[2], tot[5], tot[6], tot[5], tot[3], tot[7], tot[6], tot[7], tot[4]};
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) Wk[3 * a + b] = ((a == b ? Q : 0.0) + Vs[3 * a + b]) / (2.0 * vol);
  if (mode == 0) {
    *energy = E * e_scale;
    if (out9) {
      for (int A = 0; A < 3; ++A)
        for (int a = 0; a < 3; ++a) {
          double s = 0.0;
          for (int b = 0; b < 3; ++b) s += Wk[3 * a + b] * ci->inv[3 * b + A];
          out9[3 * A + a] = (s - tot[17 + 3 * A + a]) * e_scale;
        }
    }
  } else {
    *energy = E * e_scale;
    if (out9) {
      const double a2b3 = kAngToBohr * kAngToBohr * kAngToBohr;
      for (int k = 0; k < 9; ++k) out9[k] = (Wk[k] + tot[8 + k]) * e_scale / vol * a2b3;
    }
  }
}

int launch_finalize(const Partials& p, const CellInfo* ci, int mode, double e_scale, double* energy, double* out9,
                    cudaStream_t s) {
  k_finalize<<<1, 256, 0, s>>>(p, ci, mode, e_scale, energy, out9);
  FD3_LAUNCHED();
  return FD3_OK;
}

}  // namespace fd3

// D4 coordination numbers in reciprocal space (cnfunc = 'd4', src/fourierd3/core.py:388-447):
//   CN_i = phi_{X_i}(r_i) / Omega - f_{X_i X_i}(0),  phi_X = sum_Y G^CN_XY * rho_Y,
// rho_Y the one-hot species density spread with the same stencil as the dispersion mesh, G^CN
// the Fourier transform of the erfc pair function (pair_pot.py:235-406), and the adjoint that
// the reference leaves to autograd:
//   dE/dx_a (CN part)  = sum_m dW_a(m)/dx_a [ (dE/dCN_a / Omega) phi_{X_a}(m) + psi_{X_a}(m) ],
//   psi_Y = sum_X G^CN_YX * sigma_X,  sigma_X = sum_{i in X} (dE/dCN_i / Omega) W_i,
//   dE/dstrain_ab (CN)  = -delta_ab sum_i dE/dCN_i (CN_i + f_ii(0))
//                         - sum_k w_k G^CN'_XY(|k|) k_a k_b / |k| Re(conj(sigma_X(k)) rho_Y(k)),
// (the stencil weights are invariant under the strain protocol, so only the volume and |k| move).
// The kernels: the CN filter (forward: H = G rho; adjoint: H = G sigma plus the k-space strain
// term), the CN value gather, and the gradient gather (forces, volume term, and for the
// edge-list surface the positions-fixed cell term).
#include <math.h>

#include "fd3_filter.cuh"
#include "fd3_internal.h"

namespace fd3 {

// G^CN_XY(k) and dG/dk (pair_pot.py:336-376): 4 pi delta exp(-(k r0)^2 / (4 k0^2)) [(sin u - u cos u) / k^3
// + r0^2 sin u / (2 k0^2 k)], u = k r0; for u < 1e-3 the Taylor form c0 - c2 k^2.
__device__ __forceinline__ void cn4_green(const CnPair& c, double k, double& G, double& dG) {
  const double r0 = c.r0, u = k * r0;
  if (u < 1e-3) {
    G = c.c0 - c.c2 * k * k;
    dG = -2.0 * c.c2 * k;
    return;
  }
  constexpr double k0sq4 = 4.0 * kCn4K0 * kCn4K0;
  const double gauss = exp(-u * u / k0sq4);
  double s, co;
  sincos(u, &s, &co);
  const double ik = 1.0 / k, ik2 = ik * ik, ik3 = ik2 * ik;
  const double t1 = (s - u * co) * ik3;
  const double h = r0 * r0 / (0.5 * k0sq4);     // r0^2 / (2 k0^2)
  const double t2 = h * s * ik;
  const double dt1 = u * s * r0 * ik3 - 3.0 * t1 * ik;
  const double dt2 = h * (co * r0 * ik - s * ik2);
  const double dgauss = -gauss * 2.0 * u * r0 / k0sq4;
  const double pre = 4.0 * kPi * c.delta;
  G = pre * gauss * (t1 + t2);
  dG = pre * (dgauss * (t1 + t2) + gauss * (dt1 + dt2));
}

// Grid-stride over the half spectrum. forward: out_X = sum_Y Gh_XY rhat_Y (out != rhat);
// adjoint: the k-space strain term from (sigma = out on entry, rhat) and out_X <- sum_Y Gh_XY sigma_Y.
// Gh = G on every k-point except the self-conjugate-plane Nyquist entries, where it is the mean
// of G at the entry and at its stored conjugate partner (what the inverse real transform of the
// reference's G rho amounts to there).
template <typename T, int MAXS>
__global__ void __launch_bounds__(256) k_cn4_filter(MeshDev g, int P, int spme, int adjoint,
                                                   const CellInfo* __restrict__ ci, const CnPair* __restrict__ cp,
                                                   const float* __restrict__ deconv,
                                                   const typename Cplx<T>::type* __restrict__ rhat,
                                                   typename Cplx<T>::type* __restrict__ out, double* __restrict__ part) {
  using C2 = typename Cplx<T>::type;
  const int S = g.S;
  const size_t Mh = (size_t)g.n[0] * g.n[1] * g.nzh;
  T rc[9];
  load_recip<T>(ci, rc);
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < Mh; k += (size_t)gridDim.x * blockDim.x) {
    const KPoint<T> q = kpoint<T>(g, k, rc, deconv, spme, P);
    double G[MAXS][MAXS], dG[MAXS][MAXS], Gh[MAXS][MAXS];
#pragma unroll
    for (int X = 0; X < MAXS; ++X)
#pragma unroll
      for (int Y = X; Y < MAXS; ++Y) {
        double gv = 0.0, dv = 0.0;
        if (X < S && Y < S) {
          cn4_green(cp[X * S + Y], (double)q.knorm, gv, dv);
          gv *= (double)q.inv_sc;
          dv *= (double)q.inv_sc;
        }
        G[X][Y] = G[Y][X] = gv;
        dG[X][Y] = dG[Y][X] = dv;
        Gh[X][Y] = Gh[Y][X] = gv;
      }
    if (q.partner) {
#pragma unroll
      for (int X = 0; X < MAXS; ++X)
#pragma unroll
        for (int Y = X; Y < MAXS; ++Y)
          if (X < S && Y < S) {
            double gv, dv;
            cn4_green(cp[X * S + Y], (double)q.kpart, gv, dv);
            Gh[X][Y] = Gh[Y][X] = 0.5 * (G[X][Y] + gv * (double)q.inv_sc);
          }
    }
    C2 src[MAXS], rh[MAXS];
#pragma unroll
    for (int X = 0; X < MAXS; ++X) {
      rh[X] = X < S ? rhat[(size_t)X * Mh + k] : C2{T(0), T(0)};
      src[X] = adjoint ? (X < S ? out[(size_t)X * Mh + k] : C2{T(0), T(0)}) : rh[X];
    }
    if (adjoint) {
      double dq = 0.0;
#pragma unroll
      for (int X = 0; X < MAXS; ++X)
#pragma unroll
        for (int Y = 0; Y < MAXS; ++Y)
          dq += dG[X][Y] * ((double)rh[Y].x * (double)src[X].x + (double)rh[Y].y * (double)src[X].y);
      virial_acc<double>(KPoint<double>{{(double)q.kv[0], (double)q.kv[1], (double)q.kv[2]}, (double)q.knorm, 0.0,
                                        (double)q.wk, 0.0, false},
                         dq, acc);
    }
#pragma unroll
    for (int X = 0; X < MAXS; ++X) {
      if (X < S) {
        double hre = 0.0, him = 0.0;
#pragma unroll
        for (int Y = 0; Y < MAXS; ++Y) {
          hre += Gh[X][Y] * (double)src[Y].x;
          him += Gh[X][Y] * (double)src[Y].y;
        }
        out[(size_t)X * Mh + k] = C2{(T)hre, (T)him};
      }
    }
  }
  if (adjoint) {
    // dE/dstrain_ab = -sum_k w dG k_a k_b / |k| Re(conj sigma rho): acc[1..6] holds the sum
    double v[9] = {-acc[1], -acc[4], -acc[5], -acc[4], -acc[2], -acc[6], -acc[5], -acc[6], -acc[3]};
    block_sum_store<9>(v, part + 9 * blockIdx.x);
  }
}

// Per-atom values spread by the CN pipeline: 1 (the one-hot density) or dE/dCN_i / Omega.
__global__ void __launch_bounds__(256) k_cn4_values(int n, int adjoint, const double* __restrict__ gcn,
                                                   const CellInfo* __restrict__ ci, double* __restrict__ vals) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) vals[i] = adjoint ? gcn[i] / ci->volume : 1.0;
}

// Warp per atom (stencil-record order), lanes over the (y, z) nodes, x nodes unrolled.
// mode 0: cn[i] = sum_m W phi_s / Omega - self_s.
// mode 1: g = sum_m dW/du [ (gcn_i / Omega) phi_s + psi_s ] -> dE/dx; gpos[i] = out_scale (gpos[i] + g);
//         strain partial -gcn_i (cn_i + self_s) on the diagonal; optional -sum s_iA g_ia partials.
template <typename T, int P>
__global__ void __launch_bounds__(256) k_cn4_gather(MeshDev g, int n, int mode, const double* __restrict__ pos,
                                                   double ps, const CellInfo* __restrict__ ci,
                                                   const int* __restrict__ order, const int4* __restrict__ rb,
                                                   const T* __restrict__ rw, const T* __restrict__ rdw,
                                                   const T* __restrict__ phi, const T* __restrict__ psi,
                                                   const double* __restrict__ cnself, const double* __restrict__ gcn,
                                                   double* __restrict__ cn, double* __restrict__ gpos,
                                                   double out_scale, double* __restrict__ vir_part,
                                                   double* __restrict__ mcell_part) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int t = blockIdx.x * 8 + wid;
  double vir[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, mc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (t < n) {
    const int i = order[t];
    const int4 b4 = rb[t];
    const int s = b4.w;
    const size_t M = (size_t)g.n[0] * g.n[1] * g.n[2];
    const T* ph = phi + (size_t)s * M;
    const T* pv = psi ? psi + (size_t)s * M : nullptr;
    const double inv_vol = 1.0 / ci->volume;
    const double a = mode ? gcn[i] * inv_vol : 0.0;
    T w0[P], dw0[P];
    int ixs[P];
#pragma unroll
    for (int k = 0; k < P; ++k) {
      w0[k] = rw[((size_t)t * 3) * P + k];
      dw0[k] = rdw[((size_t)t * 3) * P + k];
      int ix = b4.x + k;
      while (ix >= g.n[0]) ix -= g.n[0];
      ixs[k] = ix;
    }
    double val = 0.0, gu0 = 0.0, gu1 = 0.0, gu2 = 0.0;
    for (int qn = lane; qn < P * P; qn += 32) {
      const int ky = qn / P, kz = qn - ky * P;
      const T wy = rw[((size_t)t * 3 + 1) * P + ky], dwy = rdw[((size_t)t * 3 + 1) * P + ky];
      const T wz = rw[((size_t)t * 3 + 2) * P + kz], dwz = rdw[((size_t)t * 3 + 2) * P + kz];
      int iy = b4.y + ky;
      while (iy >= g.n[1]) iy -= g.n[1];
      int iz = b4.z + kz;
      while (iz >= g.n[2]) iz -= g.n[2];
#pragma unroll
      for (int kx = 0; kx < P; ++kx) {
        const size_t m = ((size_t)ixs[kx] * g.n[1] + iy) * g.n[2] + iz;
        if (mode == 0) {
          val += (double)(w0[kx] * wy * wz) * (double)ph[m];
        } else {
          const double f = a * (double)ph[m] + (double)pv[m];
          gu0 += (double)(dw0[kx] * wy * wz) * f;
          gu1 += (double)(w0[kx] * dwy * wz) * f;
          gu2 += (double)(w0[kx] * wy * dwz) * f;
        }
      }
    }
    if (mode == 0) {
      val = warp_sum(val);
      if (lane == 0) cn[i] = val * inv_vol - cnself[s];
    } else {
      gu0 = warp_sum(gu0);
      gu1 = warp_sum(gu1);
      gu2 = warp_sum(gu2);
      if (lane == 0) {
        double gx[3];
#pragma unroll
        for (int b = 0; b < 3; ++b)
          gx[b] = gu0 * g.n[0] * ci->inv[3 * b + 0] + gu1 * g.n[1] * ci->inv[3 * b + 1] +
                  gu2 * g.n[2] * ci->inv[3 * b + 2];
        const double vt = -gcn[i] * (cn[i] + cnself[s]);
        vir[0] = vir[4] = vir[8] = vt;
        if (mcell_part) {
          const double x0 = pos[3 * i] * ps, x1 = pos[3 * i + 1] * ps, x2 = pos[3 * i + 2] * ps;
#pragma unroll
          for (int A = 0; A < 3; ++A) {
            const double sf = x0 * ci->inv[A] + x1 * ci->inv[3 + A] + x2 * ci->inv[6 + A];
#pragma unroll
            for (int c = 0; c < 3; ++c) mc[3 * A + c] = sf * gx[c];
          }
        }
#pragma unroll
        for (int b = 0; b < 3; ++b) gpos[3 * i + b] = out_scale * (gpos[3 * i + b] + gx[b]);
      }
    }
  }
  if (mode == 1) {
    block_sum_store<9>(vir, vir_part + 9 * blockIdx.x);
    if (mcell_part) block_sum_store<9>(mc, mcell_part + 9 * blockIdx.x);
  }
}

// ------------------------------------------------------------------ launchers
int cn4_gather_blocks(int n) { return (n + 7) / 8; }

int launch_cn4_values(int n, int adjoint, const double* gcn, const CellInfo* ci, double* vals, cudaStream_t s) {
  k_cn4_values<<<(n + 255) / 256, 256, 0, s>>>(n, adjoint, gcn, ci, vals);
  FD3_LAUNCHED();
  return FD3_OK;
}

template <typename T>
int launch_cn4_filter(const MeshGeom& mg, int adjoint, const CellInfo* ci, const CnPair* cp, const float* deconv,
                      int spme, const void* rhat, void* out, double* part, int* n_blocks, cudaStream_t s) {
  using C2 = typename Cplx<T>::type;
  const size_t Mh = (size_t)mg.n[0] * mg.n[1] * mg.nzh;
  size_t blocks = (Mh + 255) / 256;
  const size_t cap = (size_t)filter_max_blocks();
  if (blocks > cap) blocks = cap;
  *n_blocks = (int)blocks;
  const MeshDev g = to_dev(mg);
  const C2* r = static_cast<const C2*>(rhat);
  C2* o = static_cast<C2*>(out);
#define FD3_CN4F(MS) \
  k_cn4_filter<T, MS><<<(int)blocks, 256, 0, s>>>(g, mg.order, spme, adjoint, ci, cp, deconv, r, o, part)
  if (mg.S <= 1)
    FD3_CN4F(1);
  else if (mg.S <= 2)
    FD3_CN4F(2);
  else if (mg.S <= 4)
    FD3_CN4F(4);
  else if (mg.S <= kCn4MaxSpecies)
    FD3_CN4F(8);
  else
    return FD3_EINVAL;
#undef FD3_CN4F
  FD3_LAUNCHED();
  return FD3_OK;
}

template <typename T>
int launch_cn4_gather(const MeshGeom& mg, int n, int mode, const double* pos, double ps, const CellInfo* ci,
                      const int* order, const MeshRecords& rec, const void* phi, const void* psi,
                      const double* cnself, const double* gcn, double* cn, double* gpos, double out_scale,
                      double* vir_part, double* mcell_part, cudaStream_t s) {
  const int blocks = cn4_gather_blocks(n);
  const MeshDev g = to_dev(mg);
  const T* ph = static_cast<const T*>(phi);
  const T* pq = static_cast<const T*>(psi);
#define FD3_CN4G(PP)                                                                                              \
  case PP:                                                                                                        \
    k_cn4_gather<T, PP><<<blocks, 256, 0, s>>>(g, n, mode, pos, ps, ci, order, rec.b, (const T*)rec.w,           \
                                               (const T*)rec.dw, ph, pq, cnself, gcn, cn, gpos, out_scale,        \
                                               vir_part, mcell_part);                                             \
    break;
  switch (mg.order) {
    FD3_CN4G(1)
    FD3_CN4G(2)
    FD3_CN4G(3)
    FD3_CN4G(4)
    FD3_CN4G(5)
    FD3_CN4G(6)
    FD3_CN4G(7)
    FD3_CN4G(8)
    default:
      return FD3_EINVAL;
  }
#undef FD3_CN4G
  FD3_LAUNCHED();
  return FD3_OK;
}

template int launch_cn4_filter<double>(const MeshGeom&, int, const CellInfo*, const CnPair*, const float*, int,
                                       const void*, void*, double*, int*, cudaStream_t);
template int launch_cn4_filter<float>(const MeshGeom&, int, const CellInfo*, const CnPair*, const float*, int,
                                      const void*, void*, double*, int*, cudaStream_t);
template int launch_cn4_gather<double>(const MeshGeom&, int, int, const double*, double, const CellInfo*, const int*,
                                       const MeshRecords&, const void*, const void*, const double*, const double*,
                                       double*, double*, double, double*, double*, cudaStream_t);
template int launch_cn4_gather<float>(const MeshGeom&, int, int, const double*, double, const CellInfo*, const int*,
                                      const MeshRecords&, const void*, const void*, const double*, const double*,
                                      double*, double*, double, double*, double*, cudaStream_t);

}  // namespace fd3

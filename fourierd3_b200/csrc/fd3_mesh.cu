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

#include "fd3_filter.cuh"

namespace fd3 {

// ------------------------------------------------------------------ cell info
struct CellExpect {
  double c[9];
  int on;
};

__global__ void __launch_bounds__(32) k_cellinfo(const double* __restrict__ cell, double scale, CellExpect ex,
                                                CellInfo* __restrict__ ci) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double m[9];
  bool stale = false;
  for (int k = 0; k < 9; ++k) {
    m[k] = cell[k] * scale;
    stale |= ex.on && cell[k] != ex.c[k];
  }
  ci->stale = stale ? 1.0 : 0.0;
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

int launch_cellinfo(const double* cell, double scale, CellInfo* ci, cudaStream_t s, const double* h_expect) {
  CellExpect ex{};
  ex.on = h_expect != nullptr;
  if (h_expect)
    for (int k = 0; k < 9; ++k) ex.c[k] = h_expect[k];
  k_cellinfo<<<1, 32, 0, s>>>(cell, scale, ex, ci);
  FD3_LAUNCHED();
  return FD3_OK;
}

__global__ void __launch_bounds__(256) k_poison_if_stale(const CellInfo* __restrict__ ci, int n,
                                                        double* __restrict__ energy, double* __restrict__ forces,
                                                        double* __restrict__ stress) {
  if (ci->stale == 0.0) return;
  const double nan = __longlong_as_double(0x7ff8000000000000LL);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < 3 * n) forces[i] = nan;
  if (i < 9) stress[i] = nan;
  if (i == 0) *energy = nan;
}

int launch_poison_if_stale(const CellInfo* ci, int n, double* energy, double* forces, double* stress,
                           cudaStream_t s) {
  const int m = 3 * n > 9 ? 3 * n : 9;
  k_poison_if_stale<<<(m + 255) / 256, 256, 0, s>>>(ci, n, energy, forces, stress);
  FD3_LAUNCHED();
  return FD3_OK;
}

__global__ void __launch_bounds__(256) k_mesh_keys(MeshDev g, int n, int P, const double* __restrict__ pos, double ps,
                            const int32_t* __restrict__ species, const CellInfo* __restrict__ ci,
                            int* __restrict__ keys) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int base[3];
  double xl[3];
  mesh_locate<double>(pos, i, ps, ci, g.n[0], g.n[1], g.n[2], P, base, xl);
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

// ------------------------------------------------------------------ Green table (mixed form)
// Thread per (pair X <= Y, knot j); pair index X S - X (X - 1) / 2 + (Y - X).
__global__ void __launch_bounds__(256) k_green_table(MeshDev g, const CellInfo* __restrict__ ci,
                                                     const GreenPair* __restrict__ gp,
                                                     const Tables* __restrict__ tab, float4* __restrict__ out) {
  const int S = g.S, NP = S * (S + 1) / 2;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= NP * (kGreenKnots + 1)) return;
  const int pi = e / (kGreenKnots + 1), j = e - pi * (kGreenKnots + 1);
  int X = 0;
  while ((X + 1) * S - (X + 1) * X / 2 <= pi) ++X;
  const int Y = X + (pi - (X * S - X * (X - 1) / 2));
  const GreenPair& q = gp[X * S + Y];
  double rec[9];
  for (int c = 0; c < 9; ++c) rec[c] = ci->recip[c];
  const int n[3] = {g.n[0], g.n[1], g.n[2]};
  const double h = green_kmax(rec, n) / kGreenKnots;
  const double k = j * h;
  const double s6 = tab->s6, s8 = tab->s8;
  const double A6 = s6 * q.c6pre, A8 = 3.0 * s8 * q.qq * q.c8pre;
  double G, G1, G2, G3;
  if (k * q.R < 1e-15) {
    // k = 0: the value of the reference's Taylor branch (pair_pot.py:146, G = a), and the
    // derivatives of the closed form G = F(kR) / k there, G^(m)(0) = F^(m+1)(0) R^(m+1) / (m+1)
    // with F'(0) = A6 - sqrt2 sin(pi/8) A8, F''(0) = 0, F'''(0) = -2 A6 + sqrt2 sin(pi/8) A8,
    // F''''(0) = 3 A6. (The reference's k^2 coefficient of the C6 term, pair_pot.py:96, scales as
    // R where the expansion of the closed form gives 2 pi^2 / (9 R); it multiplies k^2 = 0 there,
    // so it never enters its results, but the interpolation between knots needs the true G''.)
    const double a = s6 * q.c6s1 + 3.0 * s8 * q.qq * q.c8s1;
    const double r2s8 = 0.54119610014619698440;   // sqrt(2) sin(pi/8)
    const double R3 = q.R * q.R * q.R;
    G = a;
    G1 = 0.0;
    G2 = (-2.0 * A6 + r2s8 * A8) * R3 / 3.0;
    G3 = 3.0 * A6 * R3 * q.R / 4.0;
  } else {
    double n6[4], n8[4];
    green_n(k * q.R, n6, n8);
    double F[4];
    for (int m = 0; m < 4; ++m) F[m] = A6 * n6[m] + A8 * n8[m];
    G = F[0] / k;
    G1 = (q.R * F[1] - G) / k;
    G2 = (q.R * q.R * F[2] - 2.0 * G1) / k;
    G3 = (q.R * q.R * q.R * F[3] - 3.0 * G2) / k;
  }
  out[e] = make_float4((float)G, (float)(h * G1), (float)(h * h * G2), (float)(h * h * h * G3));
}

int launch_green_table(const MeshGeom& mg, const CellInfo* ci, const GreenPair* gp, const Tables* tab,
                       void* table, cudaStream_t s) {
  const int NP = mg.S * (mg.S + 1) / 2;
  const int total = NP * (kGreenKnots + 1);
  k_green_table<<<(total + 255) / 256, 256, 0, s>>>(to_dev(mg), ci, gp, tab, reinterpret_cast<float4*>(table));
  FD3_LAUNCHED();
  return FD3_OK;
}

size_t green_table_bytes(int S) { return (size_t)S * (S + 1) / 2 * (kGreenKnots + 1) * sizeof(float4); }

// Up to 8 species: grid-stride thread per k-point; the spectrum is updated in place (H = Gh S).
// One partial (energy + 6 virial components) per block.
template <typename T, int MAXS, int MAXR>
__global__ void __launch_bounds__(kFilterThreads, sizeof(T) == 8 ? 2 : (MAXS <= 2 ? 3 : 1)) k_filter(MeshDev g, int P, int spme,
                                                           const CellInfo* __restrict__ ci,
                                                           const typename GreenPairOf<T>::type* __restrict__ gp,
                                                           const float4* __restrict__ gtab,
                                                           const Tables* __restrict__ tab,
                                                           const float* __restrict__ deconv,
                                                           typename Cplx<T>::type* __restrict__ spec,
                                                           double* __restrict__ part) {
  const size_t Mh = (size_t)g.n[0] * g.n[1] * g.nzh;
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  const T s6 = (T)tab->s6, s8 = (T)tab->s8;
  T rc[9];
  load_recip<T>(ci, rc);
  float inv_h = 0.f;
  if constexpr (sizeof(T) == 4) inv_h = green_inv_h(g, ci);
  // the grid stride and the start point decomposed once into (rows of ix, rows of iy, iz);
  // each step then advances (ix, iy, iz) by additions with at most one carry per axis
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t st_row = fdiv((uint32_t)stride, g.div_nzh);
  const int st_z = (int)((uint32_t)stride - st_row * (uint32_t)g.nzh);
  const uint32_t st_x = fdiv(st_row, g.div_ny);
  const int st_y = (int)(st_row - st_x * (uint32_t)g.n[1]);
  const uint32_t k_row = fdiv((uint32_t)k, g.div_nzh);
  int iz = (int)((uint32_t)k - k_row * (uint32_t)g.nzh);
  const uint32_t k_x = fdiv(k_row, g.div_ny);
  int iy = (int)(k_row - k_x * (uint32_t)g.n[1]);
  int ix = (int)k_x;
  for (; k < Mh; k += stride) {
    const KPoint<T> q = kpoint_idx<T>(g, ix, iy, iz, k, rc, deconv, spme, P);
    filter_point<T, MAXS, MAXR>(q, g.S, g.R, gp, gtab, inv_h, s6, s8, tab, spec + k, Mh, acc);
    iz += st_z;
    int c = iz >= g.nzh;
    if (c) iz -= g.nzh;
    iy += st_y + c;
    c = iy >= g.n[1];
    if (c) iy -= g.n[1];
    ix += (int)st_x + c;
  }
  block_sum_store<7>(acc, part + 7 * blockIdx.x);
}

// Many species (<= 64), any rank: k-tiled filter. One CTA takes KT consecutive rfft k-points at a
// time and stages their S*R spectrum values in shared memory (one coalesced read of the tile).
// Each thread keeps one k column of the tile (kk = thread % KT) and one of 256/KT slots.
//   phase B: the species pairs X <= Y are grouped in units (X, Y0..Y0+3), ordered by Y0 then X,
//            so that the slots of one warp share their Y rows (broadcast shared-memory reads)
//            and each keeps lambda_r S_Xr in registers for the unit. Per pair and k: G_XY, dG_XY
//            (and the conjugate-partner average on the self-conjugate planes) are evaluated ONCE,
//            the pair's share w_XY G_XY sum_r lambda_r Re(S_Xr S_Yr*) of the energy and virial
//            is accumulated (w = 1 on the diagonal, 2 off it), and the Hermitian-averaged G is
//            kept in shared memory;
//   phase C: thread (X, k) forms H_Xr = sum_Y Gh_XY S_Yr from shared memory and writes it over
//            the spectrum tile it came from (in place: no other CTA reads these k columns).
// Green evaluations per k fall from S^2 to S(S+1)/2 and the spectrum is read from HBM once.
constexpr int kUnitY = 4;
static int filter_units(int S) {
  int n = 0;
  for (int y0 = 0; y0 < S; y0 += kUnitY) n += (y0 + kUnitY < S ? y0 + kUnitY : S);
  return n;
}
// The spectrum tile keeps species X's R rows of KT values at X (R KT + pad) + r KT. In phase B the
// slots of one warp read rows of consecutive species; a 64-bit shared load is served per
// half-warp (16 lanes = 16 / KT slots of KT values each), so the species stride is padded to
// KT modulo 16 complex values: consecutive species then start KT values (one slot's width)
// apart in the banks and a half-warp's loads do not collide.
__host__ __device__ inline int tile_pad(int R, int KT) { return (((KT - R * KT) % 16) + 16) % 16; }
struct FilterTileSmem {
  static size_t bytes(int S, int R, int kt, size_t tsize) {
    const size_t C = (size_t)S * R, np = (size_t)S * (S + 1) / 2;
    size_t b = (C * kt + (size_t)S * tile_pad(R, kt)) * 2 * tsize;   // spectrum tile
    b += 32 * tsize;                                // lambda_r
    b += np * kt * tsize;                           // Gh tile
    b += (size_t)filter_units(S) * sizeof(uint32_t); // units (X, Y0)
    b += (size_t)S * sizeof(int);                   // first pair index of row X
    return (b + 15) & ~(size_t)15;
  }
};

// RF > 0: the rank count is RF at compile time (the rank loops unroll without predicates);
// RF = 0: any rank from the geometry.
template <typename T, int KT, int RF>
__global__ void __launch_bounds__(kFilterThreads) k_filter_tiled(MeshDev g, int P, int spme, int n_units,
                                                                 const CellInfo* __restrict__ ci,
                                                                 const typename GreenPairOf<T>::type* __restrict__ gp,
                                                                 const float4* __restrict__ gtab,
                                                                 const Tables* __restrict__ tab,
                                                                 const float* __restrict__ deconv,
                                                                 typename Cplx<T>::type* __restrict__ spec,
                                                                 double* __restrict__ part) {
  using C2 = typename Cplx<T>::type;
  constexpr int NSLOT = kFilterThreads / KT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int S = g.S, R = RF > 0 ? RF : g.R, C = S * R, NP = S * (S + 1) / 2;
  // sections in decreasing alignment: T-sized arrays first, then the 4-byte tables
  C2* ss = reinterpret_cast<C2*>(smem_raw);                  // [S][R KT + kTilePad]
  const int XS = R * KT + tile_pad(R, KT);                   // species stride of the tile
  T* lam = reinterpret_cast<T*>(ss + (size_t)S * XS);        // [32]
  T* gs = lam + 32;                                          // [NP][KT]
  uint32_t* units = reinterpret_cast<uint32_t*>(gs + (size_t)NP * KT);
  int* row0 = reinterpret_cast<int*>(units + n_units);
  for (int X = threadIdx.x; X < S; X += blockDim.x) row0[X] = X * S - X * (X - 1) / 2;
  if (threadIdx.x == 0) {
    int u = 0;
    for (int y0 = 0; y0 < S; y0 += kUnitY) {
      const int xe = y0 + kUnitY < S ? y0 + kUnitY : S;
      for (int X = 0; X < xe; ++X) units[u++] = ((uint32_t)X << 16) | (uint32_t)y0;
    }
  }
  for (int r = threadIdx.x; r < 32; r += blockDim.x) lam[r] = r < R ? (T)tab->eigs[r] : T(0);
  const size_t Mh = (size_t)g.n[0] * g.n[1] * g.nzh;
  const size_t ntile = (Mh + KT - 1) / KT;
  const int kk = threadIdx.x % KT, slot = threadIdx.x / KT;
  const T s6 = (T)tab->s6, s8 = (T)tab->s8;
  T rc[9];
  load_recip<T>(ci, rc);
  float inv_h = 0.f;
  if constexpr (sizeof(T) == 4) inv_h = green_inv_h(g, ci);
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  for (size_t tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
    const size_t k0 = tile * KT;
    __syncthreads();   // the previous tile's phase C has finished with ss / gs (and the tables are set)
    for (int e = threadIdx.x; e < C * KT; e += kFilterThreads) {
      const int c = e / KT, j = e % KT;
      const size_t k = k0 + j;
      ss[e + (c / R) * (XS - R * KT)] = k < Mh ? spec[(size_t)c * Mh + k] : C2{T(0), T(0)};
    }
    const size_t k = k0 + kk;
    const bool valid = k < Mh;
    const KPoint<T> q = kpoint<T>(g, valid ? k : 0, rc, deconv, spme, P);
    int tj = 0, pj = 0;
    HermiteF hb{}, pb{};
    if constexpr (sizeof(T) == 4) {
      table_pos(q.knorm, inv_h, tj, hb);
      table_pos(q.kpart, inv_h, pj, pb);
    }
    __syncthreads();
    T qq = T(0), dq = T(0);
    for (int u = slot; u < n_units; u += NSLOT) {
      const uint32_t xy = units[u];
      const int X = (int)(xy >> 16), Y0 = (int)(xy & 0xffffu);
      const int ya = X > Y0 ? X : Y0;
      const int yb = Y0 + kUnitY < S ? Y0 + kUnitY : S;
      // mixed form: the unit's Green-table rows are requested before the rank loop
      float4 ta[kUnitY], tb[kUnitY];
      if constexpr (sizeof(T) == 4) {
#pragma unroll
        for (int y = 0; y < kUnitY; ++y) {
          const int Y = Y0 + y;
          if (Y >= ya && Y < yb) {
            const float4* row = gtab + (size_t)(row0[X] + (Y - X)) * (kGreenKnots + 1);
            ta[y] = row[tj];
            tb[y] = row[tj + 1];
          } else {
            ta[y] = tb[y] = make_float4(0.f, 0.f, 0.f, 0.f);
          }
        }
      }
      T pr[kUnitY];
#pragma unroll
      for (int y = 0; y < kUnitY; ++y) pr[y] = T(0);
      for (int r0 = 0; r0 < R; r0 += 8) {
        C2 xl[8];
#pragma unroll
        for (int r = 0; r < 8; ++r) {
          if (r0 + r < R) {
            const C2 a = ss[X * XS + (r0 + r) * KT + kk];
            const T l = lam[r0 + r];
            xl[r] = C2{l * a.x, l * a.y};
          } else {
            xl[r] = C2{T(0), T(0)};
          }
        }
#pragma unroll
        for (int y = 0; y < kUnitY; ++y) {
          const int Y = Y0 + y;
          if (Y >= ya && Y < yb) {
            const C2* sy = ss + Y * XS + r0 * KT + kk;
#pragma unroll
            for (int r = 0; r < 8; ++r)
              if (r0 + r < R) {
                const C2 b = sy[r * KT];
                pr[y] += xl[r].x * b.x + xl[r].y * b.y;
              }
          }
        }
      }
#pragma unroll
      for (int y = 0; y < kUnitY; ++y) {
        const int Y = Y0 + y;
        if (Y >= ya && Y < yb) {
          T gv, dv;
          const int pi = row0[X] + (Y - X);
          if constexpr (sizeof(T) == 4) {
            gv = herm_value(hb, ta[y], tb[y]);
            dv = herm_slope(hb, ta[y], tb[y]) * inv_h;
          } else {
            green_eval<T>(gp[X * S + Y], q.knorm, s6, s8, gv, dv);
          }
          gv *= q.inv_sc;
          dv *= q.inv_sc;
          T gh = gv;
          if (q.partner) {
            T gpv, dpv;
            if constexpr (sizeof(T) == 4)
              green_lookup(gtab + (size_t)pi * (kGreenKnots + 1), pj, pb, inv_h, gpv, dpv);
            else
              green_eval<T>(gp[X * S + Y], q.kpart, s6, s8, gpv, dpv);
            gh = T(0.5) * (gv + gpv * q.inv_sc);
          }
          const T w = X == Y ? T(1) : T(2);
          qq += w * gv * pr[y];
          dq += w * dv * pr[y];
          gs[pi * KT + kk] = gh;
        }
      }
    }
    if (valid) {
      acc[0] += (double)(q.wk * qq);
      virial_acc<T>(q, dq, acc);
    }
    __syncthreads();
    // two species per thread (X and X + NSLOT): every staged S_Yr value serves both
    for (int X = slot; X < S; X += 2 * NSLOT) {
      const int X2 = X + NSLOT;
      const bool two = X2 < S;
      for (int r0 = 0; r0 < R; r0 += 8) {
        C2 h[8], h2[8];
#pragma unroll
        for (int r = 0; r < 8; ++r) h[r] = h2[r] = C2{T(0), T(0)};
        // pair index of (X, Y): row0[Y] + (X - Y) for Y < X, row0[X] + (Y - X) for Y >= X; both
        // advance without a table read: +(S - Y - 1) per Y below the diagonal, +1 above it
        int pa = X, pb2 = two ? X2 : 0;   // row0[0] + X, row0[0] + X2
        const C2* sy = ss + r0 * KT + kk;
        for (int Y = 0; Y < S; ++Y, sy += XS) {
          const T gh = gs[pa * KT + kk];
          const T gh2 = two ? gs[pb2 * KT + kk] : T(0);
          pa += Y < X ? S - Y - 1 : 1;
          pb2 += Y < X2 ? S - Y - 1 : 1;
#pragma unroll
          for (int r = 0; r < 8; ++r)
            if (r0 + r < R) {
              const C2 b = sy[r * KT];
              h[r].x += gh * b.x;
              h[r].y += gh * b.y;
              h2[r].x += gh2 * b.x;
              h2[r].y += gh2 * b.y;
            }
        }
        if (valid) {
#pragma unroll
          for (int r = 0; r < 8; ++r)
            if (r0 + r < R) {
              spec[((size_t)X * R + r0 + r) * Mh + k] = h[r];
              if (two) spec[((size_t)X2 * R + r0 + r) * Mh + k] = h2[r];
            }
        }
      }
    }
  }
  block_sum_store<7>(acc, part + 7 * blockIdx.x);
}

static int device_sms() {
  static int sms = 0;
  if (sms == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
  }
  return sms;
}

static int filter_grid(size_t Mh) {
  const size_t need = (Mh + kFilterThreads - 1) / kFilterThreads;
  const size_t cap = (size_t)device_sms() * 8;
  return (int)(need < cap ? need : cap);
}

int filter_max_blocks() { return 148 * 8 * 4; }

int spread_chunk_in_effect(const MeshGeom& mg, size_t tsize) {
  const int cap = tsize == 8 ? spread_col_cap<double>(mg) : spread_col_cap<float>(mg);
  return cap >= kColMinCap ? spread_zc(mg) : 0;
}

// Largest k-tile width whose shared-memory tile fits (the default when no tuning is set).
int filter_default_kt(int S, int R, size_t tsize) {
  if (S <= 4) return 0;   // register kernel
  for (int kt = 8; kt >= 1; kt >>= 1)
    if (FilterTileSmem::bytes(S, R, kt, tsize) <= 100 * 1024) return kt;
  return 1;
}

bool filter_kt_valid(int kt, int S, int R, size_t tsize) {
  if (kt == 0) return S <= 8;
  if (kt != 1 && kt != 2 && kt != 4 && kt != 8 && kt != 16) return false;
  return FilterTileSmem::bytes(S, R, kt, tsize) <= 220 * 1024;
}

template <typename T, int KT, int RF>
static int launch_tiled_r(const MeshDev& g, const MeshGeom& mg, const CellInfo* ci,
                        const typename GreenPairOf<T>::type* gp, const float4* gtab, const Tables* tab,
                        const float* deconv, int spme, typename Cplx<T>::type* sp, double* part, int* n_blocks,
                        cudaStream_t s) {
  const size_t smem = FilterTileSmem::bytes(mg.S, mg.R, KT, sizeof(T));
  // per instantiation, once (outside any stream capture in practice: the first call is eager):
  // allow the device's whole opt-in shared memory minus the kernel's static part
  static int allowed = -1;
  if (allowed < 0) {
    int dev = 0, optin = 0;
    cudaFuncAttributes fa{};
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess ||
        cudaFuncGetAttributes(&fa, k_filter_tiled<T, KT, RF>) != cudaSuccess ||
        cudaFuncSetAttribute(k_filter_tiled<T, KT, RF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             optin - (int)fa.sharedSizeBytes) != cudaSuccess) {
      set_error("filter", "could not raise the shared-memory limit of the tiled filter");
      return FD3_ECUDA;
    }
    allowed = optin - (int)fa.sharedSizeBytes;
  }
  if (smem > (size_t)allowed) {
    set_error("filter", "shared-memory tile too large for this device; choose a smaller filter k-tile");
    return FD3_EINVAL;
  }
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_filter_tiled<T, KT, RF>, kFilterThreads, smem) !=
          cudaSuccess || per_sm < 1)
    per_sm = 1;
  const size_t Mh = (size_t)mg.n[0] * mg.n[1] * mg.nzh;
  const size_t ntile = (Mh + KT - 1) / KT;
  size_t blocks = (size_t)device_sms() * per_sm;
  if (blocks > ntile) blocks = ntile;
  if (blocks > (size_t)filter_max_blocks()) blocks = filter_max_blocks();
  *n_blocks = (int)blocks;
  k_filter_tiled<T, KT, RF><<<(int)blocks, kFilterThreads, smem, s>>>(g, mg.order, spme, filter_units(mg.S), ci, gp,
                                                                  gtab, tab, deconv, sp, part);
  FD3_LAUNCHED();
  return FD3_OK;
}

template <typename T, int KT>
static int launch_tiled(const MeshDev& g, const MeshGeom& mg, const CellInfo* ci,
                        const typename GreenPairOf<T>::type* gp, const float4* gtab, const Tables* tab,
                        const float* deconv, int spme, typename Cplx<T>::type* sp, double* part, int* n_blocks,
                        cudaStream_t s) {
  if (mg.R == 8)
    return launch_tiled_r<T, KT, 8>(g, mg, ci, gp, gtab, tab, deconv, spme, sp, part, n_blocks, s);
  return launch_tiled_r<T, KT, 0>(g, mg, ci, gp, gtab, tab, deconv, spme, sp, part, n_blocks, s);
}

template <typename T>
int launch_filter(const MeshGeom& mg, const CellInfo* ci, const GreenPair* gp, const GreenPairF* gpf,
                  const float4* gtab, const Tables* tab, const float* deconv, int spme, void* spec, double* part,
                  int* n_blocks, cudaStream_t s) {
  using C2 = typename Cplx<T>::type;
  using GP = typename GreenPairOf<T>::type;
  const GP* gpt = reinterpret_cast<const GP*>(sizeof(T) == 8 ? (const void*)gp : (const void*)gpf);
  const size_t Mh = (size_t)mg.n[0] * mg.n[1] * mg.nzh;
  const MeshDev g = to_dev(mg);
  C2* sp = reinterpret_cast<C2*>(spec);
  if (sizeof(T) == 4 && filter_mma_on(mg))
    return launch_filter_mma(mg, ci, gtab, tab, deconv, spme, spec, part, n_blocks, s);
  const int kt = mg.filter_kt >= 0 ? mg.filter_kt : filter_default_kt(mg.S, mg.R, sizeof(T));
  if (kt == 0 && mg.S <= 8) {
    const int blocks = filter_grid(Mh);
    *n_blocks = blocks;
#define FD3_FILTER(SS, RR) \
  k_filter<T, SS, RR><<<blocks, kFilterThreads, 0, s>>>(g, mg.order, spme, ci, gpt, gtab, tab, deconv, sp, part)
    if (mg.S <= 1)
      FD3_FILTER(1, 4);
    else if (mg.S <= 2 && mg.R <= 4)
      FD3_FILTER(2, 4);
    else if (mg.S <= 2)
      FD3_FILTER(2, 2);
    else if (mg.S <= 4 && mg.R <= 4)
      FD3_FILTER(4, 4);
    else if (mg.S <= 4)
      FD3_FILTER(4, 2);
    else
      FD3_FILTER(8, 1);
#undef FD3_FILTER
    FD3_LAUNCHED();
    return FD3_OK;
  }
  switch (kt) {
    case 16: return launch_tiled<T, 16>(g, mg, ci, gpt, gtab, tab, deconv, spme, sp, part, n_blocks, s);
    case 8: return launch_tiled<T, 8>(g, mg, ci, gpt, gtab, tab, deconv, spme, sp, part, n_blocks, s);
    case 4: return launch_tiled<T, 4>(g, mg, ci, gpt, gtab, tab, deconv, spme, sp, part, n_blocks, s);
    case 2: return launch_tiled<T, 2>(g, mg, ci, gpt, gtab, tab, deconv, spme, sp, part, n_blocks, s);
    default: return launch_tiled<T, 1>(g, mg, ci, gpt, gtab, tab, deconv, spme, sp, part, n_blocks, s);
  }
}
template int launch_filter<double>(const MeshGeom&, const CellInfo*, const GreenPair*, const GreenPairF*,
                                   const float4*, const Tables*, const float*, int, void*, double*, int*,
                                   cudaStream_t);
template int launch_filter<float>(const MeshGeom&, const CellInfo*, const GreenPair*, const GreenPairF*,
                                  const float4*, const Tables*, const float*, int, void*, double*, int*,
                                  cudaStream_t);

// ------------------------------------------------------------------ finalize
// mode 0: energy [Hartree] and dE/dcell [Hartree/Bohr] with positions/shifts fixed (edge path)
// mode 1: energy [eV] and ASE stress [eV/A^3] = (dE/dstrain) / Omega (fused path)
__global__ void __launch_bounds__(1024) k_finalize(Partials p, const CellInfo* __restrict__ ci, int mode, double e_scale,
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
    // the strain derivative (k-space, plus the D4 CN's when present) converted to dE/dcell with
    // positions fixed: (W_ab - sum_i g_ia x_ib) inv_bA
    *energy = E * e_scale;
    if (out9) {
      for (int A = 0; A < 3; ++A)
        for (int a = 0; a < 3; ++a) {
          double s = 0.0;
          for (int b = 0; b < 3; ++b) s += (Wk[3 * a + b] + tot[8 + 3 * a + b]) * ci->inv[3 * b + A];
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
  k_finalize<<<1, 1024, 0, s>>>(p, ci, mode, e_scale, energy, out9);
  FD3_LAUNCHED();
  return FD3_OK;
}

}  // namespace fd3

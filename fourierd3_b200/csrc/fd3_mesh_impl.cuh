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

#include <type_traits>

#pragma once
#include "fd3_internal.h"

namespace fd3 {

struct MeshDev {
  int n[3], nzh, t[3], nt[3], ns[3], S, R;
  int qpitch;   // complex values per ky row of the half spectrum (nzh or nzh + 1)
  FastDiv div_nzh, div_ny, div_qpitch;
  const float* win_axes;
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
  d.div_nzh = make_fastdiv((uint32_t)g.nzh);
  d.qpitch = g.qpitch > 0 ? g.qpitch : g.nzh;
  d.div_qpitch = make_fastdiv((uint32_t)d.qpitch);
  d.div_ny = make_fastdiv((uint32_t)g.n[1]);
  d.win_axes = g.win_axes;
  return d;
}

// Fractional mesh coordinate of one atom along all axes and its first stencil node.
// MeshInterpolator.compute_weights (core.py:555): u = n * (x @ inv); reference node round(u)
// (odd p) or floor(u) (even p); local x = u - ref (odd) or u - ref - 1/2 (even).
template <typename T>
__device__ __forceinline__ void mesh_locate(const double* __restrict__ pos, int i, double ps, const CellInfo* ci,
                                            int n0, int n1, int n2, int P, int* base, T* xl) {
  const double x0 = pos[3 * i] * ps, x1 = pos[3 * i + 1] * ps, x2 = pos[3 * i + 2] * ps;
  const int n[3] = {n0, n1, n2};
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

// ------------------------------------------------------------------ stencil records
// One record per atom in (tile, species)-sorted order: first stencil node + species, the p
// weights and their x-derivatives per axis, and the rank factors in the mesh precision. The
// spread and the gather read these instead of recomputing the float64 mesh location per use.
template <typename T, int P, bool LAG>
__global__ void __launch_bounds__(256) k_mesh_records(MeshDev g, int n, const double* __restrict__ pos, double ps,
                                                      const int32_t* __restrict__ species,
                                                      const double* __restrict__ c6, const CellInfo* __restrict__ ci,
                                                      const int* __restrict__ order, int4* __restrict__ rb,
                                                      T* __restrict__ rw, T* __restrict__ rdw, T* __restrict__ rc) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int atom = order[t];
  int base[3];
  T xl[3];
  mesh_locate<T>(pos, atom, ps, ci, g.n[0], g.n[1], g.n[2], P, base, xl);
  rb[t] = make_int4(base[0], base[1], base[2], species[atom]);
  if (c6)
    for (int r = 0; r < g.R; ++r) rc[(size_t)t * g.R + r] = (T)c6[(size_t)atom * g.R + r];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    T w[P], dw[P];
    stencil_weights<P, LAG, T>(xl[a], w, dw);
#pragma unroll
    for (int k = 0; k < P; ++k) {
      rw[((size_t)t * 3 + a) * P + k] = w[k];
      rdw[((size_t)t * 3 + a) * P + k] = dw[k];
    }
  }
}

// The records' rank factors alone (sorted order), when the nodes and weights were written earlier.
template <typename T>
__global__ void __launch_bounds__(256) k_rank_factors(int n, int R, const double* __restrict__ c6,
                                                      const int* __restrict__ order, T* __restrict__ rc) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int atom = order[t];
  for (int r = 0; r < R; ++r) rc[(size_t)t * R + r] = (T)c6[(size_t)atom * R + r];
}

// ------------------------------------------------------------------ spread
// Tile-owned spread. A CTA owns one (16 x 16 x 8)-point tile of one species; thread (lx, ly)
// owns the z-row of 8 points at (lx, ly). The atoms whose stencil can reach the tile come from
// the counting-sorted (tile, species) segments of the source tiles; they are examined 256 at a
// time, the overlapping ones are compacted (warp ballots, sorted order kept) into shared memory
// as three tile-local 1D weight rows (zero outside the stencil; stencil nodes that wrap onto
// the same point are summed), and every thread accumulates w_x(lx) w_y(ly) w_z(z) c_r for its
// row. Each mesh value is written exactly once: no atomics, no zero fill, fixed summation order.
constexpr int kSpTX = 16, kSpTY = 16, kSpTZ = 8;
constexpr int kSpThreads = kSpTX * kSpTY;
constexpr int kSpRC = 4;                 // ranks accumulated per pass

template <typename T>
struct SpChunk {
  static constexpr int value = sizeof(T) == 8 ? 64 : 128;
};

template <typename T, int P>
__global__ void __launch_bounds__(kSpThreads, sizeof(T) == 8 ? 2 : 4) k_spread(MeshDev g, const int4* __restrict__ rb,
                                                       const T* __restrict__ rw, const T* __restrict__ rc,
                                                       const int* __restrict__ key_start, T* __restrict__ rho) {
  constexpr int CH = SpChunk<T>::value;
  __shared__ T s_wx[CH][kSpTX];
  __shared__ T s_wy[CH][kSpTY];
  __shared__ T s_wz[CH][kSpTZ];
  __shared__ T s_c[CH][kSpRC];
  __shared__ int s_a0[125], s_pref[126];
  __shared__ int s_wcnt[kSpThreads / 32];

  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int X = blockIdx.y;
  const int tile = blockIdx.x;
  const int tz = tile % g.nt[2];
  const int ty = (tile / g.nt[2]) % g.nt[1];
  const int tx = tile / (g.nt[2] * g.nt[1]);
  const int t0[3] = {tx * g.t[0], ty * g.t[1], tz * g.t[2]};
  const int lx = tid / kSpTY, ly = tid % kSpTY;
  const bool row_ok = lx < g.t[0] && ly < g.t[1];
  const int R = g.R;
  const int nsrc = g.ns[0] * g.ns[1] * g.ns[2];

  if (tid < nsrc) {
    const int sxo = tid / (g.ns[1] * g.ns[2]), syo = (tid / g.ns[2]) % g.ns[1], szo = tid % g.ns[2];
    const int sx = posmod(tx - sxo, g.nt[0]), sy = posmod(ty - syo, g.nt[1]), sz = posmod(tz - szo, g.nt[2]);
    const int key = ((sx * g.nt[1] + sy) * g.nt[2] + sz) * g.S + X;
    const int a0 = key_start[key];
    s_a0[tid] = a0;
    s_pref[tid + 1] = key_start[key + 1] - a0;
  }
  __syncthreads();
  if (tid == 0) {
    s_pref[0] = 0;
    for (int k = 0; k < nsrc; ++k) s_pref[k + 1] += s_pref[k];
  }
  __syncthreads();
  const int total = s_pref[nsrc];
  const size_t M = (size_t)g.n[0] * g.n[1] * g.n[2];

  for (int r0 = 0; r0 < R; r0 += kSpRC) {
    T acc[kSpTZ][kSpRC];
#pragma unroll
    for (int z = 0; z < kSpTZ; ++z)
#pragma unroll
      for (int r = 0; r < kSpRC; ++r) acc[z][r] = T(0);

    for (int c0 = 0; c0 < total; c0 += kSpThreads) {
      // examine one candidate per thread
      const int ca = c0 + tid;
      bool keep = false;
      int u = 0, base[3] = {0, 0, 0};
      if (ca < total) {
        int seg = 0;
        while (s_pref[seg + 1] <= ca) ++seg;
        u = s_a0[seg] + (ca - s_pref[seg]);      // record slot (sorted order)
        const int4 b4 = rb[u];
        base[0] = b4.x;
        base[1] = b4.y;
        base[2] = b4.z;
        keep = true;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          int d = t0[a] - base[a];
          if (d < 0) d += g.n[a];
          // stencil offsets [0, min(P, n)) from base; the tile covers offsets [d, d + t)
          const int pf = P < g.n[a] ? P : g.n[a];
          if (!(d < pf || d + g.t[a] > g.n[a])) keep = false;
        }
      }
      const unsigned bal = __ballot_sync(0xffffffffu, keep);
      if (lane == 0) s_wcnt[wid] = __popc(bal);
      __syncthreads();
      int off = 0, tot = 0;
#pragma unroll
      for (int w = 0; w < kSpThreads / 32; ++w) {
        off += w < wid ? s_wcnt[w] : 0;
        tot += s_wcnt[w];
      }
      __syncthreads();   // s_wcnt is rewritten by the next examination pass
      for (int h0 = 0; h0 < tot; h0 += CH) {
        const int slot = off + __popc(bal & ((1u << lane) - 1u)) - h0;
        if (keep && slot >= 0 && slot < CH) {
          T w[3][P];
#pragma unroll
          for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int k = 0; k < P; ++k) w[a][k] = rw[((size_t)u * 3 + a) * P + k];
#pragma unroll
          for (int z = 0; z < kSpTX; ++z) s_wx[slot][z] = T(0);
#pragma unroll
          for (int z = 0; z < kSpTY; ++z) s_wy[slot][z] = T(0);
#pragma unroll
          for (int z = 0; z < kSpTZ; ++z) s_wz[slot][z] = T(0);
#pragma unroll
          for (int k = 0; k < P; ++k) {
            int ix = (base[0] + k - t0[0]) % g.n[0]; if (ix < 0) ix += g.n[0];
            int iy = (base[1] + k - t0[1]) % g.n[1]; if (iy < 0) iy += g.n[1];
            int iz = (base[2] + k - t0[2]) % g.n[2]; if (iz < 0) iz += g.n[2];
            if (ix < g.t[0]) s_wx[slot][ix] += w[0][k];
            if (iy < g.t[1]) s_wy[slot][iy] += w[1][k];
            if (iz < g.t[2]) s_wz[slot][iz] += w[2][k];
          }
#pragma unroll
          for (int r = 0; r < kSpRC; ++r) s_c[slot][r] = r0 + r < R ? rc[(size_t)u * R + r0 + r] : T(0);
        }
        __syncthreads();
        const int nc = min(CH, tot - h0);
        if (row_ok) {
          for (int c = 0; c < nc; ++c) {
            const T wxy = s_wx[c][lx] * s_wy[c][ly];
            if (wxy != T(0)) {
              T cr[kSpRC];
#pragma unroll
              for (int r = 0; r < kSpRC; ++r) cr[r] = wxy * s_c[c][r];
#pragma unroll
              for (int z = 0; z < kSpTZ; ++z) {
                const T wz = s_wz[c][z];
#pragma unroll
                for (int r = 0; r < kSpRC; ++r) acc[z][r] += wz * cr[r];
              }
            }
          }
        }
        __syncthreads();
      }
    }
    if (row_ok) {
      const size_t m0 = ((size_t)(t0[0] + lx) * g.n[1] + (t0[1] + ly)) * g.n[2] + t0[2];
#pragma unroll
      for (int r = 0; r < kSpRC; ++r) {
        if (r0 + r >= R) break;
        T* dst = rho + ((size_t)X * R + r0 + r) * M + m0;
        if (g.t[2] == kSpTZ) {
          // the row starts on an 8-element boundary: two 16-byte stores (float) or four (double)
          if (sizeof(T) == 4) {
            float4* v = reinterpret_cast<float4*>(dst);
            v[0] = make_float4((float)acc[0][r], (float)acc[1][r], (float)acc[2][r], (float)acc[3][r]);
            v[1] = make_float4((float)acc[4][r], (float)acc[5][r], (float)acc[6][r], (float)acc[7][r]);
          } else {
            double2* v = reinterpret_cast<double2*>(dst);
#pragma unroll
            for (int z = 0; z < kSpTZ; z += 2) v[z / 2] = make_double2((double)acc[z][r], (double)acc[z + 1][r]);
          }
        } else {
#pragma unroll
          for (int z = 0; z < kSpTZ; ++z)
            if (z < g.t[2]) dst[z] = acc[z][r];
        }
      }
    }
  }
}

// Column spread. A CTA owns a column of 16 x 16 points in (x, y) and a chunk of ZC z-tiles of one
// species; thread (lx, ly) owns the z-row of 8 points of the current z-tile. The atoms whose x and
// y stencils reach the column are staged ONCE per chunk, in counting-sorted segment order with the
// source z-tile outermost, as tile-local x and y weight rows, rank factors, and two z rows: the
// part of the z stencil inside the atom's own z-tile and the part spilling into the next one
// (a stencil of P <= t_z + 1 nodes spans at most two tiles). The atoms reaching z-tile T are then
// two contiguous ranges of the staged list, those of source tile T (own rows) and of T - 1 (spill
// rows), so the CTA sweeps its z-tiles from shared memory with no selection and no barrier.
// Global loads and the candidate search happen once per ZC tiles. A chunk whose staged set
// exceeds `cap` falls back, inside the same CTA, to staging per tile in pieces of `cap`. Each
// mesh value is written exactly once in a fixed summation order (no atomics); results are
// independent of ZC up to the summation order.
constexpr int kColMaxSeg = 64;

template <typename T>
struct ColSmem {
  T* wx;      // [cap][16]
  T* wy;      // [cap][16]
  T* wzo;     // [cap][8] z row inside the atom's own z-tile
  T* wzn;     // [cap][8] z row spilling into the next z-tile
  T* cc;      // [cap][R]
  int* zi;    // [cap] source z-tile (index into the chunk's source range); bit 30: spills
  int* zst;   // [kColMaxSeg + 1] first staged slot of each source z-tile
};

template <typename T>
__host__ __device__ inline size_t col_smem_bytes(int cap, int R) {
  size_t b = (size_t)cap * (16 + 16 + 2 * kSpTZ + R) * sizeof(T);
  b += (size_t)cap * sizeof(int) + (kColMaxSeg + 1) * sizeof(int);
  return (b + 15) & ~(size_t)15;
}

template <typename T>
__device__ __forceinline__ ColSmem<T> col_carve(unsigned char* base, int cap, int R) {
  ColSmem<T> m;
  T* t = reinterpret_cast<T*>(base);
  m.wx = t;
  m.wy = m.wx + (size_t)cap * 16;
  m.wzo = m.wy + (size_t)cap * 16;
  m.wzn = m.wzo + (size_t)cap * kSpTZ;
  m.cc = m.wzn + (size_t)cap * kSpTZ;
  m.zi = reinterpret_cast<int*>(m.cc + (size_t)cap * R);
  m.zst = m.zi + cap;
  return m;
}

constexpr int kZiSpill = 1 << 30;

// Block-wide ordered compaction of one flag per thread: returns this thread's slot (among the
// set flags, in thread order) and writes the block total to *tot. Two barriers.
__device__ __forceinline__ int block_compact(bool keep, int* s_wcnt, int* tot) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const unsigned bal = __ballot_sync(0xffffffffu, keep);
  if (lane == 0) s_wcnt[wid] = __popc(bal);
  __syncthreads();
  int off = 0, t = 0;
#pragma unroll
  for (int w = 0; w < kSpThreads / 32; ++w) {
    off += w < wid ? s_wcnt[w] : 0;
    t += s_wcnt[w];
  }
  __syncthreads();
  *tot = t;
  return off + __popc(bal & ((1u << lane) - 1u));
}

// Stage candidates [from, total) whose stencil reaches the column in x and y (and z-tile tzt when
// tzt >= 0) into slots [0, cap). Segment e covers source z-tile e / seg_per_z of the chunk.
// Returns the number staged; *next is the first candidate not yet examined or staged (== total
// when all were taken).
template <typename T, int P>
__device__ int col_stage(const MeshDev& g, const int* s_a0, const int* s_pref, int nseg, int seg_per_z, int total,
                         int from, const int (&t0)[3], int tzt, int cap, const int4* __restrict__ rb,
                         const T* __restrict__ rw, const T* __restrict__ rc, const ColSmem<T>& m, int* s_wcnt,
                         int* s_next, int* next) {
  const int R = g.R;
  int staged = 0;
  int c0 = from;
  bool full = false;
  if (threadIdx.x == 0) *s_next = total;
  for (; c0 < total; c0 += kSpThreads) {
    const int ca = c0 + threadIdx.x;
    bool keep = false;
    int u = 0, seg = 0;
    int4 b4 = make_int4(0, 0, 0, 0);
    if (ca < total) {
      int lo = 0, hi = nseg - 1;   // last segment with pref <= ca
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (s_pref[mid] <= ca) lo = mid; else hi = mid - 1;
      }
      seg = lo;
      u = s_a0[lo] + (ca - s_pref[lo]);
      b4 = rb[u];
      keep = true;
      const int base[3] = {b4.x, b4.y, b4.z};
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        if (a == 2 && tzt < 0) break;
        const int ta = a == 2 ? tzt * g.t[2] : t0[a];
        int d = ta - base[a];
        if (d < 0) d += g.n[a];
        const int pf = P < g.n[a] ? P : g.n[a];
        if (!(d < pf || d + g.t[a] > g.n[a])) keep = false;
      }
    }
    int tot;
    const int slot = staged + block_compact(keep, s_wcnt, &tot);
    if (keep && slot < cap) {
      // tile-local x and y rows (stencil nodes that wrap onto the same point are summed)
      T* wxr = m.wx + slot * 16;
      T* wyr = m.wy + slot * 16;
      T* zo = m.wzo + slot * kSpTZ;
      T* zn = m.wzn + slot * kSpTZ;
#pragma unroll
      for (int z = 0; z < 16; ++z) {
        wxr[z] = T(0);
        wyr[z] = T(0);
      }
#pragma unroll
      for (int z = 0; z < kSpTZ; ++z) {
        zo[z] = T(0);
        zn[z] = T(0);
      }
      const T* w = rw + (size_t)u * 3 * P;
      const int oz = b4.z % g.t[2];   // offset of the base inside its own z-tile
      bool spill = false;
#pragma unroll
      for (int k = 0; k < P; ++k) {
        int ix = b4.x + k - t0[0];
        while (ix < 0) ix += g.n[0];
        while (ix >= g.n[0]) ix -= g.n[0];
        int iy = b4.y + k - t0[1];
        while (iy < 0) iy += g.n[1];
        while (iy >= g.n[1]) iy -= g.n[1];
        if (ix < g.t[0]) wxr[ix] += w[k];
        if (iy < g.t[1]) wyr[iy] += w[P + k];
        const int z = oz + k;
        if (z < g.t[2]) {
          zo[z] = w[2 * P + k];
        } else {
          zn[z - g.t[2]] = w[2 * P + k];
          spill = true;
        }
      }
      m.zi[slot] = seg / seg_per_z + (spill ? kZiSpill : 0);
      for (int r = 0; r < R; ++r) m.cc[slot * R + r] = rc[(size_t)u * R + r];
    }
    if (keep && slot >= cap) atomicMin(s_next, ca);
    staged += tot;
    if (staged >= cap) {
      full = true;
      break;
    }
  }
  __syncthreads();
  int nx = *s_next;   // first kept candidate that found no slot, else total
  if (full && c0 + kSpThreads < nx) nx = c0 + kSpThreads;   // the pass filled cap exactly
  *next = nx;
  __syncthreads();
  return staged < cap ? staged : cap;
}

// acc[z][r] += w_x(lx) w_y(ly) w_z(z) c_{r0+r} over staged atoms [a0, a1), with their own-tile
// z rows (spill = false) or spill rows (spill = true). CHECK: the range may hold atoms of other
// source z-tiles (per-tile staging), skip those whose source tile is not zsrc. Atoms are taken
// four at a time so that their x/y weight loads are in flight together; an atom with no spill
// has an all-zero spill row and adds exact zeros.
template <typename T, bool CHECK>
__device__ __forceinline__ void col_atom(const ColSmem<T>& m, const T* zrows, int a, T wxy, int zsrc, int R, int r0,
                                         T (&acc)[kSpTZ][kSpRC]) {
  if (CHECK && (m.zi[a] & ~kZiSpill) != zsrc) return;
  T cr[kSpRC];
  if (sizeof(T) == 4 && kSpRC == 4 && (R & 3) == 0) {
    // a whole 4-rank group in one 16-byte load (rows of R floats start on 16-byte boundaries)
    const float4 c4 = *reinterpret_cast<const float4*>(m.cc + a * R + r0);
    cr[0] = wxy * (T)c4.x;
    cr[1] = wxy * (T)c4.y;
    cr[2] = wxy * (T)c4.z;
    cr[3] = wxy * (T)c4.w;
  } else {
#pragma unroll
    for (int r = 0; r < kSpRC; ++r) cr[r] = r0 + r < R ? wxy * m.cc[a * R + r0 + r] : T(0);
  }
  T zr[kSpTZ];
  if (sizeof(T) == 4) {
    const float4* v = reinterpret_cast<const float4*>(zrows + a * kSpTZ);
    const float4 p0 = v[0], p1 = v[1];
    const float t8[8] = {p0.x, p0.y, p0.z, p0.w, p1.x, p1.y, p1.z, p1.w};
#pragma unroll
    for (int z = 0; z < kSpTZ; ++z) zr[z] = (T)t8[z];
  } else {
#pragma unroll
    for (int z = 0; z < kSpTZ; ++z) zr[z] = zrows[a * kSpTZ + z];
  }
#pragma unroll
  for (int z = 0; z < kSpTZ; ++z)
#pragma unroll
    for (int r = 0; r < kSpRC; ++r) acc[z][r] += zr[z] * cr[r];
}

template <typename T, bool CHECK>
__device__ __forceinline__ void col_accumulate(const ColSmem<T>& m, int a0, int a1, int zsrc, bool spill, int R,
                                               int r0, int lx, int ly, T (&acc)[kSpTZ][kSpRC]) {
  const T* zrows = spill ? m.wzn : m.wzo;
  int a = a0;
  for (; a + 4 <= a1; a += 4) {
    T wxy[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) wxy[u] = m.wx[(a + u) * 16 + lx] * m.wy[(a + u) * 16 + ly];
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (wxy[u] != T(0)) col_atom<T, CHECK>(m, zrows, a + u, wxy[u], zsrc, R, r0, acc);
  }
  for (; a < a1; ++a) {
    const T wxy = m.wx[a * 16 + lx] * m.wy[a * 16 + ly];
    if (wxy != T(0)) col_atom<T, CHECK>(m, zrows, a, wxy, zsrc, R, r0, acc);
  }
}

template <typename T>
__device__ __forceinline__ void col_store(const MeshDev& g, int X, int r0, const int (&t0)[3], int tzt, int lx,
                                          int ly, const T (&acc)[kSpTZ][kSpRC], T* __restrict__ rho) {
  if (lx >= g.t[0] || ly >= g.t[1]) return;
  const size_t M = (size_t)g.n[0] * g.n[1] * g.n[2];
  const size_t m0 = ((size_t)(t0[0] + lx) * g.n[1] + (t0[1] + ly)) * g.n[2] + (size_t)tzt * g.t[2];
#pragma unroll
  for (int r = 0; r < kSpRC; ++r) {
    if (r0 + r >= g.R) break;
    T* dst = rho + ((size_t)X * g.R + r0 + r) * M + m0;
    if (g.t[2] == kSpTZ) {
      if (sizeof(T) == 4) {
        float4* v = reinterpret_cast<float4*>(dst);
        v[0] = make_float4((float)acc[0][r], (float)acc[1][r], (float)acc[2][r], (float)acc[3][r]);
        v[1] = make_float4((float)acc[4][r], (float)acc[5][r], (float)acc[6][r], (float)acc[7][r]);
      } else {
        double2* v = reinterpret_cast<double2*>(dst);
#pragma unroll
        for (int z = 0; z < kSpTZ; z += 2) v[z / 2] = make_double2((double)acc[z][r], (double)acc[z + 1][r]);
      }
    } else {
#pragma unroll
      for (int z = 0; z < kSpTZ; ++z)
        if (z < g.t[2]) dst[z] = acc[z][r];
    }
  }
}

template <typename T, int P>
__global__ void __launch_bounds__(kSpThreads, sizeof(T) == 8 ? 2 : 4) k_spread_col(
    MeshDev g, int zc, int cap, const int4* __restrict__ rb, const T* __restrict__ rw, const T* __restrict__ rc,
    const int* __restrict__ key_start, T* __restrict__ rho) {
  extern __shared__ __align__(16) unsigned char col_raw[];
  __shared__ int s_a0[kColMaxSeg], s_pref[kColMaxSeg + 1];
  __shared__ int s_wcnt[kSpThreads / 32];
  __shared__ int s_next;
  const ColSmem<T> m = col_carve<T>(col_raw, cap, g.R);
  const int tid = threadIdx.x;
  const int X = blockIdx.y;
  const int nzc = (g.nt[2] + zc - 1) / zc;
  const int zch = blockIdx.x % nzc;
  const int cxy = blockIdx.x / nzc;
  const int ty = cxy % g.nt[1], tx = cxy / g.nt[1];
  const int tz0 = zch * zc;
  const int tz1 = tz0 + zc < g.nt[2] ? tz0 + zc : g.nt[2];
  const int t0[3] = {tx * g.t[0], ty * g.t[1], 0};
  const int lx = tid / kSpTY, ly = tid % kSpTY;
  // source z-tiles of the chunk: tz - 1 and tz for tz in [tz0, tz1), each once
  int nzs = (tz1 - tz0) + 1;
  int zs0 = tz0 - 1;
  if (nzs >= g.nt[2]) {
    nzs = g.nt[2];
    zs0 = 0;
  }
  const int spz = g.ns[0] * g.ns[1];   // segments per source z-tile
  const int nseg = spz * nzs;
  for (int e = tid; e < nseg; e += kSpThreads) {
    const int zi = e / spz, xo = (e % spz) / g.ns[1], yo = e % g.ns[1];
    const int sx = posmod(tx - xo, g.nt[0]), sy = posmod(ty - yo, g.nt[1]), sz = posmod(zs0 + zi, g.nt[2]);
    const int key = ((sx * g.nt[1] + sy) * g.nt[2] + sz) * g.S + X;
    const int a0 = key_start[key];
    s_a0[e] = a0;
    s_pref[e + 1] = key_start[key + 1] - a0;
  }
  __syncthreads();
  if (tid < 32) {   // inclusive warp scan of the segment sizes (nseg <= 64)
    int v0 = tid + 1 <= nseg ? s_pref[tid + 1] : 0;
    int v1 = tid + 33 <= nseg ? s_pref[tid + 33] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int a = __shfl_up_sync(0xffffffffu, v0, o);
      const int b = __shfl_up_sync(0xffffffffu, v1, o);
      if (tid >= o) {
        v0 += a;
        v1 += b;
      }
    }
    const int carry = __shfl_sync(0xffffffffu, v0, 31);
    if (tid + 1 <= nseg) s_pref[tid + 1] = v0;
    if (tid + 33 <= nseg) s_pref[tid + 33] = v1 + carry;
    if (tid == 0) s_pref[0] = 0;
  }
  __syncthreads();
  const int total = s_pref[nseg];
  int next = 0;
  const int staged = col_stage<T, P>(g, s_a0, s_pref, nseg, spz, total, 0, t0, -1, cap, rb, rw, rc, m, s_wcnt,
                                     &s_next, &next);
  if (next >= total) {
    // first staged slot of each source z-tile (the staged list is ordered by source z-tile)
    for (int zi = tid; zi <= nzs; zi += kSpThreads) {
      int lo = 0, hi = staged;
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if ((m.zi[mid] & ~kZiSpill) < zi) lo = mid + 1; else hi = mid;
      }
      m.zst[zi] = lo;
    }
    __syncthreads();
    for (int tzt = tz0; tzt < tz1; ++tzt) {
      const int zown = nzs == g.nt[2] ? tzt : tzt - zs0;
      const int zprev = nzs == g.nt[2] ? (tzt + g.nt[2] - 1) % g.nt[2] : zown - 1;
      for (int r0 = 0; r0 < g.R; r0 += kSpRC) {
        T acc[kSpTZ][kSpRC];
#pragma unroll
        for (int z = 0; z < kSpTZ; ++z)
#pragma unroll
          for (int r = 0; r < kSpRC; ++r) acc[z][r] = T(0);
        col_accumulate<T, false>(m, m.zst[zprev], m.zst[zprev + 1], zprev, true, g.R, r0, lx, ly, acc);
        col_accumulate<T, false>(m, m.zst[zown], m.zst[zown + 1], zown, false, g.R, r0, lx, ly, acc);
        col_store<T>(g, X, r0, t0, tzt, lx, ly, acc, rho);
      }
    }
    return;
  }
  // dense column: per z-tile, stage the atoms reaching that tile in pieces of `cap`
  for (int tzt = tz0; tzt < tz1; ++tzt) {
    const int zown = nzs == g.nt[2] ? tzt : tzt - zs0;
    const int zprev = nzs == g.nt[2] ? (tzt + g.nt[2] - 1) % g.nt[2] : zown - 1;
    for (int r0 = 0; r0 < g.R; r0 += kSpRC) {
      T acc[kSpTZ][kSpRC];
#pragma unroll
      for (int z = 0; z < kSpTZ; ++z)
#pragma unroll
        for (int r = 0; r < kSpRC; ++r) acc[z][r] = T(0);
      int from = 0;
      while (from < total) {
        const int st = col_stage<T, P>(g, s_a0, s_pref, nseg, spz, total, from, t0, tzt, cap, rb, rw, rc, m,
                                       s_wcnt, &s_next, &from);
        col_accumulate<T, true>(m, 0, st, zprev, true, g.R, r0, lx, ly, acc);
        col_accumulate<T, true>(m, 0, st, zown, false, g.R, r0, lx, ly, acc);
        __syncthreads();
      }
      col_store<T>(g, X, r0, t0, tzt, lx, ly, acc, rho);
    }
  }
}

// Staged atoms per column chunk: as many as let 4 (float) or 2 (double) CTAs share an SM.
template <typename T>
inline int spread_col_cap(const MeshGeom& mg) {
  constexpr int per_sm = sizeof(T) == 8 ? 2 : 4;
  const size_t fixed = col_smem_bytes<T>(0, mg.R);
  const size_t per_atom = col_smem_bytes<T>(64, mg.R) / 64;
  int cap = (int)((size_t)(220 * 1024 / per_sm - 2048 - fixed) / per_atom);
  if (cap > 1024) cap = 1024;
  if (mg.spread_cap > 0 && mg.spread_cap < cap) cap = mg.spread_cap;
  return cap;
}
constexpr int kColMinCap = 128;

// z-tiles per column chunk in effect for this mesh (0: per-tile kernel).
inline int spread_zc(const MeshGeom& mg) {
  // the column form needs stencils that span at most two z-tiles of a mesh with >= 2 z-tiles
  if (mg.spread_zc == 0 || mg.ns[0] > 2 || mg.ns[1] > 2 || mg.nt[2] < 2 || mg.order > mg.t[2] + 1 ||
      mg.t[2] > kSpTZ)
    return 0;
  int zc = mg.spread_zc > 0 ? mg.spread_zc : 8;
  const int lim = kColMaxSeg / (mg.ns[0] * mg.ns[1]) - 1;
  if (zc > lim) zc = lim;
  if (zc > mg.nt[2]) zc = mg.nt[2];
  return zc < 1 ? 0 : zc;
}

template <typename T, int P, bool LAG>
static int spread_r(const MeshGeom& mg, dim3 grid, int n, const double* pos, double ps, const int32_t* species,
                    const double* c6, const CellInfo* ci, const int* ks, const int* order, const MeshRecords& rec,
                    T* rho, cudaStream_t s, int records) {
  const MeshDev g = to_dev(mg);
  if (n > 0) {
    if (records == 1) {
      k_rank_factors<T><<<(n + 255) / 256, 256, 0, s>>>(n, mg.R, c6, order, (T*)rec.c);
    } else {
      k_mesh_records<T, P, LAG><<<(n + 255) / 256, 256, 0, s>>>(g, n, pos, ps, species,
                                                                records == kSpreadRecordsOnly ? nullptr : c6, ci,
                                                                order, rec.b, (T*)rec.w, (T*)rec.dw, (T*)rec.c);
    }
    FD3_LAUNCHED();
  }
  if (records == kSpreadRecordsOnly) return FD3_OK;
  const int zc = spread_zc(mg);
  if (zc > 0) {
    // staged atoms per chunk: as many as let 3 (float) or 2 (double) CTAs share an SM
    const int cap = spread_col_cap<T>(mg);
    if (cap >= kColMinCap) {
      const size_t smem = col_smem_bytes<T>(cap, mg.R);
      static bool attr = false;
      if (!attr) {
        if (cudaFuncSetAttribute(k_spread_col<T, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) !=
            cudaSuccess) {
          set_error("spread", "could not raise the shared-memory limit of the column spread");
          return FD3_ECUDA;
        }
        attr = true;
      }
      const int nzc = (mg.nt[2] + zc - 1) / zc;
      const dim3 cgrid(mg.nt[0] * mg.nt[1] * nzc, mg.S);
      k_spread_col<T, P><<<cgrid, kSpThreads, smem, s>>>(g, zc, cap, rec.b, (const T*)rec.w, (const T*)rec.c, ks,
                                                        rho);
      FD3_LAUNCHED();
      return FD3_OK;
    }
  }
  k_spread<T, P><<<grid, kSpThreads, 0, s>>>(g, rec.b, (const T*)rec.w, (const T*)rec.c, ks, rho);
  FD3_LAUNCHED();
  return FD3_OK;
}

template <typename T>
int launch_spread(const MeshGeom& mg, int n, const double* pos, double pos_scale, const int32_t* species,
                  const double* c6, const CellInfo* ci, const int* key_start, const int* order,
                  const MeshRecords& rec, T* rho, cudaStream_t s, int records) {
  if (mg.R > FD3_MAX_RANK || mg.order < 1 || mg.order > FD3_MAX_ORDER) return FD3_EINVAL;
  if (mg.t[0] > kSpTX || mg.t[1] > kSpTY || mg.t[2] > kSpTZ || mg.ns[0] * mg.ns[1] * mg.ns[2] > 125)
    return FD3_EINVAL;
  const dim3 grid(mg.nt[0] * mg.nt[1] * mg.nt[2], mg.S);
#define FD3_SPREAD_CASE(PP)                                                                                  \
  case PP:                                                                                                   \
    return mg.lagrange ? spread_r<T, PP, true>(mg, grid, n, pos, pos_scale, species, c6, ci, key_start, order, rec, \
                                               rho, s, records)                                              \
                       : spread_r<T, PP, false>(mg, grid, n, pos, pos_scale, species, c6, ci, key_start, order, rec, \
                                                rho, s, records);
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
}  // namespace fd3
#include "fd3_gather_tile.cuh"   // the tile-staged (TMA) gather, on MeshDev / MeshRecords above
namespace fd3 {

constexpr int kGatherWarps = 8;

template <typename T, int P, bool LAG, int MAXR>
__global__ void __launch_bounds__(32 * kGatherWarps) k_gather(MeshDev g, int n, const double* __restrict__ pos,
                                                              double ps, const int32_t* __restrict__ species,
                                                              const double* __restrict__ c6,
                                                              const double* __restrict__ dc6,
                                                              const CellInfo* __restrict__ ci,
                                                              const Tables* __restrict__ tab,
                                                              const int* __restrict__ order,
                                                              const int4* __restrict__ rb, const T* __restrict__ rw,
                                                              const T* __restrict__ rdw,
                                                              const T* __restrict__ phi, double* __restrict__ gcn,
                                                              double* __restrict__ gpos,
                                                              double* __restrict__ mcell_part) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int t = blockIdx.x * kGatherWarps + wid;
  const int R = g.R;
  double mc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (t < n) {
    const int i = order[t];
    const int4 b4 = rb[t];
    const int s = b4.w;
    const int base[3] = {b4.x, b4.y, b4.z};
    T w0[P], dw0[P];
#pragma unroll
    for (int k = 0; k < P; ++k) {
      w0[k] = rw[((size_t)t * 3) * P + k];
      dw0[k] = rdw[((size_t)t * 3) * P + k];
    }
    double cl[MAXR];
#pragma unroll
    for (int r = 0; r < MAXR; ++r) cl[r] = r < R ? c6[(size_t)i * R + r] * tab->eigs[r] : 0.0;
    const size_t M = (size_t)g.n[0] * g.n[1] * g.n[2];
    double pr[MAXR];
#pragma unroll
    for (int r = 0; r < MAXR; ++r) pr[r] = 0.0;
    double gu0 = 0, gu1 = 0, gu2 = 0;
    // lanes over the (y, z) stencil nodes, x nodes unrolled: every weight index is static
    int ixs[P];
#pragma unroll
    for (int kx = 0; kx < P; ++kx) {
      int ix = base[0] + kx;
      while (ix >= g.n[0]) ix -= g.n[0];
      ixs[kx] = ix;
    }
    for (int q = lane; q < P * P; q += 32) {
      const int ky = q / P, kz = q - ky * P;
      const T wy = rw[((size_t)t * 3 + 1) * P + ky], dwy = rdw[((size_t)t * 3 + 1) * P + ky];
      const T wz = rw[((size_t)t * 3 + 2) * P + kz], dwz = rdw[((size_t)t * 3 + 2) * P + kz];
      int iy = base[1] + ky;
      while (iy >= g.n[1]) iy -= g.n[1];
      int iz = base[2] + kz;
      while (iz >= g.n[2]) iz -= g.n[2];
      const T wyz = wy * wz, dyz = dwy * wz, ydz = wy * dwz;
#pragma unroll
      for (int kx = 0; kx < P; ++kx) {
        const size_t m = ((size_t)ixs[kx] * g.n[1] + iy) * g.n[2] + iz;
        const T W = w0[kx] * wyz;
        const T Wx = dw0[kx] * wyz;
        const T Wy = w0[kx] * dyz;
        const T Wz = w0[kx] * ydz;
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

// Fused-path gather, z-run form: lanes over the (x, y) stencil columns; each lane reads the P
// z-values of its column from every rank channel with aligned 16-byte vector loads (the column
// start is rounded down to the vector boundary; a warp-uniform offset O in [0, 16/sizeof(T))
// selects the run, so every register index stays static) and forms
//   zr_r = sum_z w_z phi_r,  cp_z = sum_r lambda_r c_r phi_r,  s0 = sum_z w_z cp_z,  s2 = sum_z w'_z cp_z,
// in T, then accumulates P_r = sum W phi_r and the three spline-gradient sums in float64.
// A column that wraps the periodic z edge (or a mesh whose nz is not a multiple of the vector
// width) is read element by element with the offset 0.
template <typename T, int P, int MAXR, int O, int NE>
__device__ __forceinline__ void zrun_sums(const T (&v)[MAXR][NE], int R, const T (&wz)[P], const T (&cl)[MAXR],
                                          T (&zr)[MAXR], T (&cp)[P]) {
#pragma unroll
  for (int r = 0; r < MAXR; ++r) {
    if (r < R) {
      T a = T(0);
#pragma unroll
      for (int kz = 0; kz < P; ++kz) {
        const T f = v[r][O + kz];
        a += wz[kz] * f;
        cp[kz] += cl[r] * f;
      }
      zr[r] = a;
    }
  }
}

template <typename T, int P, int MAXR>
__global__ void __launch_bounds__(32 * kGatherWarps, (sizeof(T) == 4 && MAXR <= 4 && P <= 5) ? 4 : 1) k_gather_z(MeshDev g, int n, const double* __restrict__ c6,
                                                                const double* __restrict__ dc6,
                                                                const CellInfo* __restrict__ ci,
                                                                const Tables* __restrict__ tab,
                                                                const int* __restrict__ order,
                                                                const int4* __restrict__ rb,
                                                                const T* __restrict__ rw, const T* __restrict__ rdw,
                                                                const T* __restrict__ phi, double* __restrict__ gcn,
                                                                double* __restrict__ gpos) {
  constexpr int VW = 16 / (int)sizeof(T);          // elements per 16-byte vector
  constexpr int NV = (VW - 1 + P + VW - 1) / VW;   // vectors covering a run at any offset
  constexpr int NE = NV * VW;
  using V = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int t = blockIdx.x * kGatherWarps + wid;
  if (t >= n) return;
  const int R = g.R;
  const int i = order[t];
  const int4 b4 = rb[t];
  const int s = b4.w;
  const T* wr = rw + (size_t)t * 3 * P;
  const T* dwr = rdw + (size_t)t * 3 * P;
  T wz[P], dwz[P];
#pragma unroll
  for (int k = 0; k < P; ++k) {
    wz[k] = wr[2 * P + k];
    dwz[k] = dwr[2 * P + k];
  }
  T cl[MAXR];
#pragma unroll
  for (int r = 0; r < MAXR; ++r) cl[r] = r < R ? (T)(c6[(size_t)i * R + r] * tab->eigs[r]) : T(0);
  const int n2 = g.n[2];
  const int iz0 = b4.z;
  const bool scalar = iz0 + P > n2 || (n2 % VW) != 0;   // warp-uniform
  const int o = scalar ? 0 : iz0 % VW;
  const int za = iz0 - o;
  const int nvec = (o + P + VW - 1) / VW;
  const size_t M = (size_t)g.n[0] * g.n[1] * n2;
  double pr[MAXR];
#pragma unroll
  for (int r = 0; r < MAXR; ++r) pr[r] = 0.0;
  double gu0 = 0.0, gu1 = 0.0, gu2 = 0.0;
  for (int q = lane; q < P * P; q += 32) {
    const int kx = q / P, ky = q - kx * P;
    int ix = b4.x + kx;
    while (ix >= g.n[0]) ix -= g.n[0];   // a stencil wider than the mesh wraps more than once
    int iy = b4.y + ky;
    while (iy >= g.n[1]) iy -= g.n[1];
    const T wx = wr[kx], dwx = dwr[kx], wy = wr[P + ky], dwy = dwr[P + ky];
    const T* col = phi + (size_t)s * R * M + ((size_t)ix * g.n[1] + iy) * n2;
    T v[MAXR][NE];
#pragma unroll
    for (int r = 0; r < MAXR; ++r) {
      if (r < R) {
        const T* src = col + (size_t)r * M;
        if (!scalar) {
          const V* vs = reinterpret_cast<const V*>(src + za);
#pragma unroll
          for (int j = 0; j < NV; ++j)
            if (j < nvec) *reinterpret_cast<V*>(&v[r][j * VW]) = vs[j];
        } else {
#pragma unroll
          for (int kz = 0; kz < P; ++kz) {
            int iz = iz0 + kz;
            while (iz >= n2) iz -= n2;
            v[r][kz] = src[iz];
          }
        }
      }
    }
    T zr[MAXR], cp[P];
#pragma unroll
    for (int kz = 0; kz < P; ++kz) cp[kz] = T(0);
#pragma unroll
    for (int r = 0; r < MAXR; ++r) zr[r] = T(0);
    if constexpr (VW == 4) {
      switch (o) {
        case 0: zrun_sums<T, P, MAXR, 0, NE>(v, R, wz, cl, zr, cp); break;
        case 1: zrun_sums<T, P, MAXR, 1, NE>(v, R, wz, cl, zr, cp); break;
        case 2: zrun_sums<T, P, MAXR, 2, NE>(v, R, wz, cl, zr, cp); break;
        default: zrun_sums<T, P, MAXR, 3, NE>(v, R, wz, cl, zr, cp); break;
      }
    } else {
      if (o == 0)
        zrun_sums<T, P, MAXR, 0, NE>(v, R, wz, cl, zr, cp);
      else
        zrun_sums<T, P, MAXR, 1, NE>(v, R, wz, cl, zr, cp);
    }
    T s0 = T(0), s2 = T(0);
#pragma unroll
    for (int kz = 0; kz < P; ++kz) {
      s0 += wz[kz] * cp[kz];
      s2 += dwz[kz] * cp[kz];
    }
    const T wxy = wx * wy;
#pragma unroll
    for (int r = 0; r < MAXR; ++r) pr[r] += (double)(wxy * zr[r]);
    gu0 += (double)(dwx * wy * s0);
    gu1 += (double)(wx * dwy * s0);
    gu2 += (double)(wxy * s2);
  }
#pragma unroll
  for (int r = 0; r < MAXR; ++r) pr[r] = warp_sum(pr[r]);
  gu0 = warp_sum(gu0);
  gu1 = warp_sum(gu1);
  gu2 = warp_sum(gu2);
  if (lane != 0) return;
  const double inv_vol = 1.0 / ci->volume;
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
  const double du[3] = {-inv_vol * gu0, -inv_vol * gu1, -inv_vol * gu2};
  gcn[i] = gsum;
#pragma unroll
  for (int b = 0; b < 3; ++b)
    gpos[3 * i + b] = du[0] * g.n[0] * ci->inv[3 * b + 0] + du[1] * g.n[1] * ci->inv[3 * b + 1] +
                      du[2] * g.n[2] * ci->inv[3 * b + 2];
}

template <typename T, int P, bool LAG>
static int gather_r(const MeshGeom& mg, int blocks, int n, const double* pos, double ps, const int32_t* species,
                    const double* c6, const double* dc6, const CellInfo* ci, const Tables* tab, const int* order,
                    const int* key_start, const MeshRecords& rec, const T* phi, double* gcn, double* gpos,
                    double* mcell, int* n_mcell, cudaStream_t s) {
  // tile-staged gather (one CTA per (tile, species) key, the key's mesh box staged once by TMA)
  // for the fused path where its box fits two CTAs per SM, when asked for
  if (!mcell && mg.gather_tile == 1 && gather_tile_applies(mg, sizeof(T))) {
    *n_mcell = 0;
    return launch_gather_tile<T, P>(mg, n, c6, dc6, ci, tab, order, key_start, rec, phi, gcn, gpos, s);
  }
  const MeshDev g = to_dev(mg);
  *n_mcell = mcell ? blocks : 0;
  const int tb = 32 * kGatherWarps;
  const int4* rb = rec.b;
  const T* rw = (const T*)rec.w;
  const T* rdw = (const T*)rec.dw;
  // z-run gather where its register arrays (ranks x run) stay small: float up to 4 ranks at any
  // order or 8 ranks up to order 5; double up to 4 ranks up to order 5
  constexpr bool z4 = sizeof(T) == 4 || P <= 5;
  constexpr bool z8 = sizeof(T) == 4 && P <= 5;
  if (!mcell && ((mg.R <= 4 && z4) || (mg.R <= 8 && z8))) {
    if (mg.R <= 4)
      k_gather_z<T, P, 4><<<blocks, tb, 0, s>>>(g, n, c6, dc6, ci, tab, order, rb, rw, rdw, phi, gcn, gpos);
    else if constexpr (z8)
      k_gather_z<T, P, 8><<<blocks, tb, 0, s>>>(g, n, c6, dc6, ci, tab, order, rb, rw, rdw, phi, gcn, gpos);
    FD3_LAUNCHED();
    return FD3_OK;
  }
  if (mg.R <= 4)
    k_gather<T, P, LAG, 4><<<blocks, tb, 0, s>>>(g, n, pos, ps, species, c6, dc6, ci, tab, order, rb, rw, rdw, phi,
                                                  gcn, gpos, mcell);
  else if (mg.R <= 8)
    k_gather<T, P, LAG, 8><<<blocks, tb, 0, s>>>(g, n, pos, ps, species, c6, dc6, ci, tab, order, rb, rw, rdw, phi,
                                                  gcn, gpos, mcell);
  else if (mg.R <= 16)
    k_gather<T, P, LAG, 16><<<blocks, tb, 0, s>>>(g, n, pos, ps, species, c6, dc6, ci, tab, order, rb, rw, rdw, phi,
                                                   gcn, gpos, mcell);
  else
    k_gather<T, P, LAG, 32><<<blocks, tb, 0, s>>>(g, n, pos, ps, species, c6, dc6, ci, tab, order, rb, rw, rdw, phi,
                                                   gcn, gpos, mcell);
  FD3_LAUNCHED();
  return FD3_OK;
}

template <typename T>
int launch_gather(const MeshGeom& mg, int n, const double* pos, double pos_scale, const int32_t* species,
                  const double* c6, const double* dc6, const CellInfo* ci, const Tables* tab, const int* order,
                  const int* key_start, const MeshRecords& rec, const T* phi, double* gcn, double* gpos,
                  double* mcell_part, int* n_blocks, cudaStream_t s) {
  const int blocks = (n + kGatherWarps - 1) / kGatherWarps;
  *n_blocks = 0;
  if (blocks == 0) return FD3_OK;
#define FD3_GATHER_CASE(PP)                                                                                   \
  case PP:                                                                                                    \
    return mg.lagrange ? gather_r<T, PP, true>(mg, blocks, n, pos, pos_scale, species, c6, dc6, ci, tab, order, \
                                               key_start, rec, phi, gcn, gpos, mcell_part, n_blocks, s)       \
                       : gather_r<T, PP, false>(mg, blocks, n, pos, pos_scale, species, c6, dc6, ci, tab, order, \
                                                key_start, rec, phi, gcn, gpos, mcell_part, n_blocks, s);
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

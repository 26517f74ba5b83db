// Cell-list neighbour search, smooth-cutoff coordination numbers, C6 factors and the
// CN adjoint (reference: src/fourierd3/core.py:323-386, 449-478, 525-550 and the matscipy
// neighbour build at src/fourierd3/calculator.py:94-123).
//
// Design: atoms are counting-sorted into a bin grid whose bins are at least r_cut wide (in
// perpendicular height), so a neighbour lies within `reach` bins per axis. Bins are laid out
// with z fastest, so for a fixed (dx, dy) the bins bz-reach..bz+reach are one contiguous run of
// the bin-sorted atom array (split only at the periodic wrap). One warp handles one atom and
// strides its lanes over those runs, so the candidate loads are coalesced.
#include <math.h>
#include <stdio.h>

#include "fd3_internal.h"

namespace fd3 {

// ------------------------------------------------------------------ host geometry
static void inv3_host(const double* m, double* inv, double* det_out) {
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
  const double a[9] = {c00, c01, c02, c10, c11, c12, c20, c21, c22};
  for (int k = 0; k < 9; ++k) inv[k] = a[k] / det;
  if (det_out) *det_out = det;
}

int make_cell_grid(const double* h_cell, double r_cut, CellGrid* g) {
  if (!h_cell || !g) {
    set_error("cell grid", "null cell");
    return FD3_EINVAL;
  }
  if (!(r_cut > 0)) return FD3_EINVAL;
  double det;
  inv3_host(h_cell, g->inv, &det);
  if (!(fabs(det) > 0) || !isfinite(det)) return FD3_EINVAL;
  for (int k = 0; k < 9; ++k) g->cell[k] = h_cell[k];
  for (int a = 0; a < 3; ++a) {
    // perpendicular height of the cell along axis a = 1 / |column a of inv(cell)|
    const double cn = sqrt(g->inv[0 * 3 + a] * g->inv[0 * 3 + a] + g->inv[1 * 3 + a] * g->inv[1 * 3 + a] +
                           g->inv[2 * 3 + a] * g->inv[2 * 3 + a]);
    const double h = 1.0 / cn;
    int nb = (int)floor(h / r_cut);
    if (nb < 1) nb = 1;
    if (nb > 512) nb = 512;
    g->nb[a] = nb;
    g->reach[a] = (int)ceil(r_cut * nb / h + 1e-9);
  }
  g->r_cut = r_cut;
  g->rc2 = r_cut * r_cut;
  return FD3_OK;
}

// ------------------------------------------------------------------ scan / sort
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;

__global__ void __launch_bounds__(1024) k_scan_exclusive(const int* __restrict__ in, int n, int* __restrict__ out) {
  __shared__ int warp_tot[32];
  __shared__ int carry_s;
  if (threadIdx.x == 0) carry_s = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int base = 0; base < n; base += kScanThreads * kScanItems) {
    int v[kScanItems];
    int local = 0;
    const int i0 = base + threadIdx.x * kScanItems;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
      v[k] = (i0 + k < n) ? in[i0 + k] : 0;
      local += v[k];
    }
    int incl = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) warp_tot[wid] = incl;
    __syncthreads();
    if (wid == 0) {
      int w = warp_tot[lane];
      int wi = w;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, wi, o);
        if (lane >= o) wi += t;
      }
      warp_tot[lane] = wi - w;   // exclusive warp offsets
    }
    __syncthreads();
    int run = carry_s + warp_tot[wid] + incl - local;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
      if (i0 + k < n) out[i0 + k] = run;
      run += v[k];
    }
    __syncthreads();
    if (threadIdx.x == kScanThreads - 1) carry_s = run;
    __syncthreads();
  }
  if (threadIdx.x == 0) out[n] = carry_s;
}

int scan_exclusive(const int* in, int n, int* out, cudaStream_t s) {
  k_scan_exclusive<<<1, kScanThreads, 0, s>>>(in, n, out);
  FD3_LAUNCHED();
  return FD3_OK;
}

__global__ void __launch_bounds__(256) k_hist(const int* __restrict__ keys, int n, int* __restrict__ counts) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) atomicAdd(&counts[keys[i]], 1);
}

__global__ void __launch_bounds__(256) k_scatter(const int* __restrict__ keys, int n, const int* __restrict__ starts,
                          int* __restrict__ fill, int* __restrict__ order) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    const int k = keys[i];
    order[starts[k] + atomicAdd(&fill[k], 1)] = i;
  }
}

// Sort each key segment by atom id: makes the order (and every sum taken in that order)
// independent of the atomic slot assignment above. One warp per segment: a segment of at most
// 32 ids is ranked in registers (rank = number of smaller ids, the ids being distinct) and
// written back in one step; a longer one is insertion-sorted by lane 0.
__global__ void __launch_bounds__(256) k_sort_segments(const int* __restrict__ starts, int K, int* __restrict__ order) {
  const int lane = threadIdx.x & 31;
  const int k = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (k >= K) return;
  const int a = starts[k], b = starts[k + 1], m = b - a;
  if (m <= 1) return;
  if (m <= 32) {
    const int v = lane < m ? order[a + lane] : 0x7fffffff;
    int rank = 0;
#pragma unroll 8
    for (int j = 0; j < 32; ++j) {
      const int u = __shfl_sync(0xffffffffu, v, j);
      rank += (j < m && u < v) ? 1 : 0;
    }
    __syncwarp();
    if (lane < m) order[a + rank] = v;
    return;
  }
  if (lane != 0) return;
  for (int u = a + 1; u < b; ++u) {
    const int v = order[u];
    int w = u - 1;
    while (w >= a && order[w] > v) {
      order[w + 1] = order[w];
      --w;
    }
    order[w + 1] = v;
  }
}

int counting_sort(const int* keys, int n, int K, int* counts, int* starts, int* order, cudaStream_t s) {
  const int tb = 256;
  FD3_CUDA(cudaMemsetAsync(counts, 0, sizeof(int) * K, s));
  if (n > 0) {
    k_hist<<<(n + tb - 1) / tb, tb, 0, s>>>(keys, n, counts);
    FD3_LAUNCHED();
  }
  int rc = scan_exclusive(counts, K, starts, s);
  if (rc) return rc;
  FD3_CUDA(cudaMemsetAsync(counts, 0, sizeof(int) * K, s));
  if (n > 0) {
    k_scatter<<<(n + tb - 1) / tb, tb, 0, s>>>(keys, n, starts, counts, order);
    FD3_LAUNCHED();
  }
  k_sort_segments<<<(K + tb / 32 - 1) / (tb / 32), tb, 0, s>>>(starts, K, order);
  FD3_LAUNCHED();
  return FD3_OK;
}

// ------------------------------------------------------------------ cell list
struct GridDev {
  int nb[3], reach[3];
  double cell[9], inv[9];
  double rc2;
};
static GridDev to_dev(const CellGrid& g) {
  GridDev d;
  for (int a = 0; a < 3; ++a) {
    d.nb[a] = g.nb[a];
    d.reach[a] = g.reach[a];
  }
  for (int k = 0; k < 9; ++k) {
    d.cell[k] = g.cell[k];
    d.inv[k] = g.inv[k];
  }
  d.rc2 = g.rc2;
  return d;
}

__global__ void __launch_bounds__(256) k_bin_atoms(GridDev g, int n, const double* __restrict__ x, int* __restrict__ bin_of,
                            int4* __restrict__ off) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double x0 = x[3 * i], x1 = x[3 * i + 1], x2 = x[3 * i + 2];
  int o[3], b[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double f = x0 * g.inv[a] + x1 * g.inv[3 + a] + x2 * g.inv[6 + a];
    const double fl = floor(f);
    o[a] = (int)fl;
    int bb = (int)((f - fl) * g.nb[a]);
    b[a] = bb < 0 ? 0 : (bb >= g.nb[a] ? g.nb[a] - 1 : bb);
  }
  const int bin = (b[0] * g.nb[1] + b[1]) * g.nb[2] + b[2];
  bin_of[i] = bin;
  off[i] = make_int4(o[0], o[1], o[2], bin);
}

__global__ void __launch_bounds__(256) k_gather_sorted(int n, const int* __restrict__ order, const double* __restrict__ x,
                                const int32_t* __restrict__ species, const int4* __restrict__ off,
                                double4* __restrict__ xs, int4* __restrict__ meta) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int i = order[t];
  xs[t] = make_double4(x[3 * i], x[3 * i + 1], x[3 * i + 2], species ? (double)species[i] : 0.0);
  const int4 o = off[i];
  meta[t] = make_int4(o.x, o.y, o.z, i);
}

int build_cell_list(const CellGrid& g, int n, const double* pos_ang, const int32_t* species, CellList& cl,
                    cudaStream_t s) {
  const int K = g.nb[0] * g.nb[1] * g.nb[2];
  const int tb = 256;
  if (n > 0) {
    k_bin_atoms<<<(n + tb - 1) / tb, tb, 0, s>>>(to_dev(g), n, pos_ang, cl.bin_of, cl.off);
    FD3_LAUNCHED();
  }
  int rc = counting_sort(cl.bin_of, n, K, cl.bin_count, cl.bin_start, cl.order, s);
  if (rc) return rc;
  if (n > 0) {
    k_gather_sorted<<<(n + tb - 1) / tb, tb, 0, s>>>(n, cl.order, pos_ang, species, cl.off, cl.xs, cl.meta);
    FD3_LAUNCHED();
  }
  return FD3_OK;
}

// Visit every candidate (j, S) of atom i. All lanes of the warp run the same number of
// iterations; `fn(hit, u, j, S, d)` gets the exact-predicate result (Angstrom, no FMA).
template <class Fn>
__device__ __forceinline__ void visit_neighbors(const GridDev& g, const int* __restrict__ bin_start,
                                                const double4* __restrict__ xs, const int4* __restrict__ meta,
                                                int i, double xi0, double xi1, double xi2, int4 offi, Fn&& fn) {
  const int lane = threadIdx.x & 31;
  const int bin = offi.w;
  const int bz = bin % g.nb[2];
  const int by = (bin / g.nb[2]) % g.nb[1];
  const int bx = bin / (g.nb[2] * g.nb[1]);
  for (int dx = -g.reach[0]; dx <= g.reach[0]; ++dx) {
    const int cx = bx + dx;
    const int sx = floordiv(cx, g.nb[0]);
    const int wx = cx - sx * g.nb[0];
    for (int dy = -g.reach[1]; dy <= g.reach[1]; ++dy) {
      const int cy = by + dy;
      const int sy = floordiv(cy, g.nb[1]);
      const int wy = cy - sy * g.nb[1];
      int zs = bz - g.reach[2];
      const int ze = bz + g.reach[2];
      while (zs <= ze) {
        const int sz = floordiv(zs, g.nb[2]);
        const int wz = zs - sz * g.nb[2];
        int len = g.nb[2] - wz;
        if (len > ze - zs + 1) len = ze - zs + 1;
        const int b0 = (wx * g.nb[1] + wy) * g.nb[2] + wz;
        const int a0 = bin_start[b0], a1 = bin_start[b0 + len];
        for (int u0 = a0; u0 < a1; u0 += 32) {
          const int u = u0 + lane;
          bool hit = false;
          int j = 0;
          int S0 = 0, S1 = 0, S2 = 0;
          double d0 = 0, d1 = 0, d2 = 0;
          if (u < a1) {
            const double4 xj = xs[u];
            const int4 mj = meta[u];
            j = mj.w;
            S0 = sx + offi.x - mj.x;
            S1 = sy + offi.y - mj.y;
            S2 = sz + offi.z - mj.z;
            const double sh0 = dadd(dadd(dmul((double)S0, g.cell[0]), dmul((double)S1, g.cell[3])),
                                    dmul((double)S2, g.cell[6]));
            const double sh1 = dadd(dadd(dmul((double)S0, g.cell[1]), dmul((double)S1, g.cell[4])),
                                    dmul((double)S2, g.cell[7]));
            const double sh2 = dadd(dadd(dmul((double)S0, g.cell[2]), dmul((double)S1, g.cell[5])),
                                    dmul((double)S2, g.cell[8]));
            d0 = dadd(dsub(xj.x, xi0), sh0);
            d1 = dadd(dsub(xj.y, xi1), sh1);
            d2 = dadd(dsub(xj.z, xi2), sh2);
            const double r2 = dadd(dadd(dmul(d0, d0), dmul(d1, d1)), dmul(d2, d2));
            hit = r2 < g.rc2 && !(j == i && S0 == 0 && S1 == 0 && S2 == 0);
          }
          fn(hit, u, j, S0, S1, S2, d0, d1, d2);
        }
        zs += len;
      }
    }
  }
}

constexpr int kWarpsPerBlock = 8;

// Per-atom traversal straight from global memory: the path for bins whose neighbourhood does not
// fit the shared-memory stage (dense clusters, cells much narrower than the cutoff).
__device__ __forceinline__ double cn_atom_global(const GridDev& g, const int* __restrict__ bin_start,
                                                 const double4* __restrict__ xs, const int4* __restrict__ meta,
                                                 const int4* __restrict__ off, const Tables* __restrict__ tab,
                                                 int t) {
  const double4 xi = xs[t];
  const int i = meta[t].w;
  const int4 offi = off[i];
  const double rci = tab->rcov[(int)xi.w];
  double acc = 0.0;
  visit_neighbors(g, bin_start, xs, meta, i, xi.x, xi.y, xi.z, offi,
                  [&](bool hit, int u, int, int, int, int, double d0, double d1, double d2) {
                    if (!hit) return;
                    const double v0 = d0 * kAngToBohr, v1 = d1 * kAngToBohr, v2 = d2 * kAngToBohr;
                    double f, df;
                    cn_edge(sqrt(v0 * v0 + v1 * v1 + v2 * v2), rci + tab->rcov[(int)xs[u].w], tab->r_cut, f, df);
                    acc += f;
                  });
  return warp_sum(acc);
}

__device__ __forceinline__ void cn_adjoint_atom_global(const GridDev& g, const int* __restrict__ bin_start,
                                                       const double4* __restrict__ xs,
                                                       const int4* __restrict__ meta, const int4* __restrict__ off,
                                                       const Tables* __restrict__ tab, const double* __restrict__ gcn,
                                                       int t, double* f, double* v) {
  const double4 xi = xs[t];
  const int i = meta[t].w;
  const int4 offi = off[i];
  const double rci = tab->rcov[(int)xi.w];
  const double gi = gcn[i];
  visit_neighbors(g, bin_start, xs, meta, i, xi.x, xi.y, xi.z, offi,
                  [&](bool hit, int u, int j, int, int, int, double d0, double d1, double d2) {
                    if (!hit) return;
                    const double v0 = d0 * kAngToBohr, v1 = d1 * kAngToBohr, v2 = d2 * kAngToBohr;
                    const double r = sqrt(v0 * v0 + v1 * v1 + v2 * v2);
                    double fe, df;
                    cn_edge(r, rci + tab->rcov[(int)xs[u].w], tab->r_cut, fe, df);
                    if (r > 1e-6) {
                      const double a = df / r;
                      const double w = (gi + gcn[j]) * a;
                      f[0] -= w * v0;
                      f[1] -= w * v1;
                      f[2] -= w * v2;
                      const double b = gi * a;
                      v[0] += b * v0 * v0; v[1] += b * v0 * v1; v[2] += b * v0 * v2;
                      v[4] += b * v1 * v1; v[5] += b * v1 * v2; v[8] += b * v2 * v2;
                    }
                  });
}

// ------------------------------------------------------------------ bin-staged CN
// One CTA per bin: the atoms of the (2 reach + 1)^3 neighbour bins are staged once in shared
// memory as image positions p_j = x_j + (S' - off_j) . cell, and the warps of the CTA run the
// bin's own atoms against that stage (d = p_j - (x_i - off_i . cell)). The same stage and the
// same arithmetic serve the CN and its adjoint, so both see the same pairs.
constexpr int kBinCap = 768;
constexpr int kMaxNbrBins = 343;

// P4 = double4: absolute image positions (the plain form, and the exact pair predicate);
// P4 = float4 (mixed form): positions relative to the bin's own corner, so that float keeps
// ~1e-6 A over the few bins a stage spans.
template <typename P4>
struct BinStage {
  P4 p[kBinCap];   // image position (A), species in .w
  int j[kBinCap];
  int a0[kMaxNbrBins];
  int pref[kMaxNbrBins + 1];
  int img[kMaxNbrBins][3];
};

// Returns the number of staged candidates, or -1 when the neighbourhood does not fit; org is the
// origin subtracted from the staged positions (zero for double4).
// rcov: when given, the staged w component is the candidate's covalent radius rcov[species]
// (the CN kernel's only use of the species) instead of the species index.
template <typename P4>
__device__ int stage_bin(const GridDev& g, int b, const int* __restrict__ bin_start,
                         const double4* __restrict__ xs, const int4* __restrict__ meta, BinStage<P4>& st,
                         double* __restrict__ s_g, const double* __restrict__ gcn, double (&org)[3],
                         const double* __restrict__ rcov = nullptr) {
  const int nx = 2 * g.reach[0] + 1, ny = 2 * g.reach[1] + 1, nz = 2 * g.reach[2] + 1;
  const int nnb = nx * ny * nz;
  if (nnb > kMaxNbrBins) return -1;
  const int bz = b % g.nb[2], by = (b / g.nb[2]) % g.nb[1], bx = b / (g.nb[2] * g.nb[1]);
#pragma unroll
  for (int c = 0; c < 3; ++c)
    org[c] = sizeof(P4) == sizeof(double4)
                 ? 0.0
                 : ((double)bx / g.nb[0]) * g.cell[c] + ((double)by / g.nb[1]) * g.cell[3 + c] +
                       ((double)bz / g.nb[2]) * g.cell[6 + c];
  for (int e = threadIdx.x; e < nnb; e += blockDim.x) {
    const int dz = e % nz - g.reach[2], dy = (e / nz) % ny - g.reach[1], dx = e / (nz * ny) - g.reach[0];
    const int cx = bx + dx, cy = by + dy, cz = bz + dz;
    const int sx = floordiv(cx, g.nb[0]), sy = floordiv(cy, g.nb[1]), sz = floordiv(cz, g.nb[2]);
    const int id = ((cx - sx * g.nb[0]) * g.nb[1] + (cy - sy * g.nb[1])) * g.nb[2] + (cz - sz * g.nb[2]);
    const int a0 = bin_start[id];
    st.a0[e] = a0;
    st.pref[e + 1] = bin_start[id + 1] - a0;
    st.img[e][0] = sx;
    st.img[e][1] = sy;
    st.img[e][2] = sz;
  }
  __syncthreads();
  if (nnb <= 32) {   // one warp scans the bin sizes (27 bins at reach 1)
    if (threadIdx.x < 32) {
      int v = threadIdx.x < nnb ? st.pref[threadIdx.x + 1] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, v, o);
        if ((int)threadIdx.x >= o) v += u;
      }
      if ((int)threadIdx.x < nnb) st.pref[threadIdx.x + 1] = v;
      if (threadIdx.x == 0) st.pref[0] = 0;
    }
  } else if (threadIdx.x == 0) {
    st.pref[0] = 0;
    for (int e = 0; e < nnb; ++e) st.pref[e + 1] += st.pref[e];
  }
  __syncthreads();
  const int total = st.pref[nnb];
  if (total > kBinCap) return -1;
  for (int c = threadIdx.x; c < total; c += blockDim.x) {
    int lo = 0, hi = nnb - 1;          // last entry with pref[e] <= c
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (st.pref[mid] <= c) lo = mid; else hi = mid - 1;
    }
    const int u = st.a0[lo] + (c - st.pref[lo]);
    const double4 xj = xs[u];
    const int4 mj = meta[u];
    const double S0 = st.img[lo][0] - mj.x, S1 = st.img[lo][1] - mj.y, S2 = st.img[lo][2] - mj.z;
    const double px = xj.x + S0 * g.cell[0] + S1 * g.cell[3] + S2 * g.cell[6];
    const double py = xj.y + S0 * g.cell[1] + S1 * g.cell[4] + S2 * g.cell[7];
    const double pz = xj.z + S0 * g.cell[2] + S1 * g.cell[5] + S2 * g.cell[8];
    const double wv = rcov ? rcov[(int)xj.w] : xj.w;
    if constexpr (sizeof(P4) == sizeof(double4))
      st.p[c] = make_double4(px, py, pz, wv);
    else
      st.p[c] = make_float4((float)(px - org[0]), (float)(py - org[1]), (float)(pz - org[2]), (float)wv);
    st.j[c] = mj.w;
    if (s_g) s_g[c] = gcn[mj.w];
  }
  __syncthreads();
  return total;
}

__device__ __forceinline__ void wrapped_pos(const GridDev& g, double4 x, int4 m, double& w0, double& w1,
                                            double& w2) {
  w0 = x.x - (m.x * g.cell[0] + m.y * g.cell[3] + m.z * g.cell[6]);
  w1 = x.y - (m.x * g.cell[1] + m.y * g.cell[4] + m.z * g.cell[7]);
  w2 = x.z - (m.x * g.cell[2] + m.y * g.cell[5] + m.z * g.cell[8]);
}

// The forward CN kernel also records, per atom, every in-cutoff pair: the neighbour id and one
// 4-wide record {f'(r)/r, Bohr vector d} (HitList, TE = double for the plain form, float for the
// mixed form), so the adjoint reads a pair with one vector load instead of searching the cell list
// a second time. An atom with more than `cap` such pairs (or one handled by the global-memory
// path) is marked n = -1 and the adjoint recomputes it.
template <typename TE> struct Vec4;
template <> struct Vec4<float> { using type = float4; };
template <> struct Vec4<double> { using type = double4; };

template <typename TE>
struct HitList {
  int* j;
  typename Vec4<TE>::type* ad;
  int* n;
  int cap;
};

// CN of the atoms of one bin from the shared-memory stage (raw CN, before cncorr), plus the
// pair records. Bins whose neighbourhood does not fit the stage mark their atoms n = -2 and
// leave them to k_cn_global.
// Per atom (one warp) the staged candidates are first tested against the cutoff 32 at a time
// (float64 distances in the plain form, float relative to the bin corner in the mixed form); the
// indices of the pairs inside are compacted in order into a per-warp ring of 64, and whenever 32
// are waiting all lanes evaluate the CN function for them and write their records contiguously. The CN function and the record stores thus run on full warps
// instead of on the ~15 % of lanes that hit in a given candidate batch.
// A bin holds ~15 atoms at r_cut 6 A (SiO2 density): 4 warps per CTA leave fewer idle warps
// waiting for a bin's last atom than 8 do, and more CTAs (bins) fit per SM.
constexpr int kCnRing = 64;
constexpr int kCnWarps = 4;

template <typename TC> struct StagePos { using type = double4; };
template <> struct StagePos<float> { using type = float4; };

template <typename TE, typename TC>
__device__ __forceinline__ void cn_hit(const BinStage<typename StagePos<TC>::type>& st, int c, TC w0, TC w1, TC w2,
                                       TC rci, TC rc, const Tables* __restrict__ tab, HitList<TE>& hl, size_t hb,
                                       int h, TC& acc) {
  const auto pj = st.p[c];
  const TC v0 = (TC)((pj.x - w0) * (TC)kAngToBohr);
  const TC v1 = (TC)((pj.y - w1) * (TC)kAngToBohr);
  const TC v2 = (TC)((pj.z - w2) * (TC)kAngToBohr);
  const TC r2 = v0 * v0 + v1 * v1 + v2 * v2;
  TC f = TC(0), a = TC(0);
  if (r2 > TC(1e-12)) {
    cn_pair<TC>(r2, rci + (TC)pj.w, rc, f, a);   // pj.w: the neighbour's covalent radius
    acc += f;
  }
  if (h < hl.cap) {
    hl.j[hb + h] = st.j[c];
    hl.ad[hb + h] = typename Vec4<TE>::type{(TE)a, (TE)v0, (TE)v1, (TE)v2};
  }
}

template <typename TE, typename TC>
__global__ void __launch_bounds__(32 * kCnWarps) k_cn_bins(GridDev g, const int* __restrict__ bin_start,
                                                const double4* __restrict__ xs, const int4* __restrict__ meta,
                                                const Tables* __restrict__ tab, double* __restrict__ cn,
                                                HitList<TE> hl, int* __restrict__ ovf) {
  using P4 = typename StagePos<TC>::type;
  __shared__ BinStage<P4> st;
  __shared__ int ring[kCnWarps][kCnRing];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int b = blockIdx.x;
  double org[3];
  const int total = stage_bin<P4>(g, b, bin_start, xs, meta, st, nullptr, nullptr, org, tab->rcov);
  const int s0 = bin_start[b], s1 = bin_start[b + 1];
  if (total < 0) {
    for (int t = s0 + threadIdx.x; t < s1; t += blockDim.x) hl.n[t] = -2;
    if (threadIdx.x == 0 && s1 > s0) atomicAdd(ovf, 1);
    return;
  }
  const unsigned lt = (1u << lane) - 1u;
  const TC rc = (TC)tab->r_cut;
  const TC rc2 = (TC)g.rc2;
  int* rg = ring[wid];
  for (int t = s0 + wid; t < s1; t += kCnWarps) {
    const double4 xi = xs[t];
    const int4 mi = meta[t];
    double wd0, wd1, wd2;
    wrapped_pos(g, xi, mi, wd0, wd1, wd2);
    const TC w0 = (TC)(wd0 - org[0]), w1 = (TC)(wd1 - org[1]), w2 = (TC)(wd2 - org[2]);
    const TC rci = (TC)tab->rcov[(int)xi.w];
    TC acc = TC(0);
    int produced = 0, consumed = 0;
    const size_t hb = (size_t)t * hl.cap;
    for (int c0 = 0; c0 < total; c0 += 32) {
      const int c = c0 + lane;
      bool hit = false;
      if (c < total) {
        const P4 pj = st.p[c];
        const TC d0 = pj.x - w0, d1 = pj.y - w1, d2 = pj.z - w2;
        hit = d0 * d0 + d1 * d1 + d2 * d2 < rc2;
      }
      const unsigned m = __ballot_sync(0xffffffffu, hit);
      if (hit) rg[(produced + __popc(m & lt)) & (kCnRing - 1)] = c;
      produced += __popc(m);
      __syncwarp();
      if (produced - consumed >= 32) {
        const int h = consumed + lane;
        cn_hit<TE, TC>(st, rg[h & (kCnRing - 1)], w0, w1, w2, rci, rc, tab, hl, hb, h, acc);
        consumed += 32;
        __syncwarp();
      }
    }
    if (consumed + lane < produced) {
      const int h = consumed + lane;
      cn_hit<TE, TC>(st, rg[h & (kCnRing - 1)], w0, w1, w2, rci, rc, tab, hl, hb, h, acc);
    }
    __syncwarp();
    const double cnv = warp_sum((double)acc);
    if (lane == 0) {
      hl.n[t] = produced <= hl.cap ? produced : -1;
      if (produced > hl.cap) atomicAdd(ovf, 1);
      cn[mi.w] = cnv;
    }
  }
}

constexpr int kFallbackBlocks = 148 * 4;

// Raw CN of atoms whose bin overflowed the stage, straight from the cell list in global memory.
// Returns at once when no bin overflowed (the counter is zero).
__global__ void __launch_bounds__(256) k_cn_global(GridDev g, int n, const int* __restrict__ bin_start,
                                                  const double4* __restrict__ xs, const int4* __restrict__ meta,
                                                  const int4* __restrict__ off, const Tables* __restrict__ tab,
                                                  double* __restrict__ cn, int* __restrict__ hit_n,
                                                  const int* __restrict__ ovf) {
  if (*ovf == 0) return;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int t = blockIdx.x * kWarpsPerBlock + wid; t < n; t += gridDim.x * kWarpsPerBlock) {
    if (hit_n[t] != -2) continue;
    const double v = cn_atom_global(g, bin_start, xs, meta, off, tab, t);
    if (lane == 0) {
      cn[meta[t].w] = v;
      hit_n[t] = -1;
    }
  }
}

int launch_cn_c6_cells(const CellGrid& g, int n, const CellList& cl, const double* pos_ang,
                       const int32_t* species, const Tables* tab, const double* eigvecs, int R, double* cn,
                       double* c6, double* dc6, double* self_part, int* n_self_blocks, const HitStore& hs,
                       cudaStream_t s) {
  (void)pos_ang;
  const int K = g.nb[0] * g.nb[1] * g.nb[2];
  FD3_CUDA(cudaMemsetAsync(hs.ovf, 0, sizeof(int), s));
  if (hs.is_double)
    k_cn_bins<double, double><<<K, 32 * kCnWarps, 0, s>>>(
        to_dev(g), cl.bin_start, cl.xs, cl.meta, tab, cn,
        HitList<double>{hs.j, (double4*)hs.ad, hs.n, hs.cap}, hs.ovf);
  else
    k_cn_bins<float, float><<<K, 32 * kCnWarps, 0, s>>>(
        to_dev(g), cl.bin_start, cl.xs, cl.meta, tab, cn,
        HitList<float>{hs.j, (float4*)hs.ad, hs.n, hs.cap}, hs.ovf);
  FD3_LAUNCHED();
  const int blocks = (n + kWarpsPerBlock - 1) / kWarpsPerBlock;
  if (blocks > 0) {
    const int fb = blocks < kFallbackBlocks ? blocks : kFallbackBlocks;
    k_cn_global<<<fb, 32 * kWarpsPerBlock, 0, s>>>(to_dev(g), n, cl.bin_start, cl.xs, cl.meta, cl.off, tab, cn,
                                                    hs.n, hs.ovf);
    FD3_LAUNCHED();
  }
  return launch_c6_atoms(n, species, tab, eigvecs, R, cn, c6, dc6, self_part, n_self_blocks, s);
}

// CN adjoint: dE/dx_i = -sum_(j,S) (g_i + g_j) f'(r) d / r  (the list is symmetric), and the
// strain virial W_ab = sum_i g_i sum_(j,S) f'(r) d_a d_b / r  (Bohr, Hartree). The force written
// is out_scale * (mesh gradient already in grad + CN gradient). One warp per atom streams the
// atom's recorded pairs; atoms without a record (n < 0) are left to k_cn_adjoint_global.
// The kernel is bound by the latency of its dependent loads (count -> atom -> records -> g_j), so
// a warp fetches the next atom's count and index while it works on this one, issues all of a
// batch of 96 records' loads before the g_j loads that depend on them, and reads the atom's mesh
// gradient at the start. Lane l still sums the records l, l + 32, ... in that order.
template <typename TE>
__global__ void __launch_bounds__(256, 4) k_cn_adjoint_hits(int n, const int4* __restrict__ meta,
                                                        const double* __restrict__ gcn, double* __restrict__ grad,
                                                        double out_scale, double* __restrict__ vir_part,
                                                        HitList<TE> hl) {
  using V4 = typename Vec4<TE>::type;
  constexpr int kU = 3;   // records per lane per batch
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int stride = gridDim.x * kWarpsPerBlock;
  double v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  int t = blockIdx.x * kWarpsPerBlock + wid;
  int nh_next = t < n ? hl.n[t] : -1;
  int i_next = t < n ? meta[t].w : 0;
  // grid-stride over atoms: the block's virial is reduced once, after all its atoms
  for (; t < n; t += stride) {
    const int nh = nh_next, i = i_next;
    if (t + stride < n) {
      nh_next = hl.n[t + stride];
      i_next = meta[t + stride].w;
    }
    if (nh >= 0) {
      const double gi = gcn[i];
      const double gq = lane < 3 ? grad[3 * i + lane] : 0.0;
      double f0 = 0, f1 = 0, f2 = 0;
      const size_t hb = (size_t)t * hl.cap;
      for (int e0 = 0; e0 < nh; e0 += 32 * kU) {
        V4 r4[kU];
        int jj[kU];
        double gj[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
          const int e = e0 + 32 * u + lane;
          if (e < nh) {
            r4[u] = hl.ad[hb + e];
            jj[u] = hl.j[hb + e];
          } else {
            r4[u] = V4{0, 0, 0, 0};
            jj[u] = -1;
          }
        }
#pragma unroll
        for (int u = 0; u < kU; ++u) gj[u] = jj[u] >= 0 ? gcn[jj[u]] : 0.0;
#pragma unroll
        for (int u = 0; u < kU; ++u) {
          if (jj[u] < 0) continue;
          const double a = (double)r4[u].x, v0 = (double)r4[u].y, v1 = (double)r4[u].z, v2 = (double)r4[u].w;
          const double w = (gi + gj[u]) * a;
          f0 -= w * v0;
          f1 -= w * v1;
          f2 -= w * v2;
          const double bb = gi * a;
          v[0] += bb * v0 * v0; v[1] += bb * v0 * v1; v[2] += bb * v0 * v2;
          v[4] += bb * v1 * v1; v[5] += bb * v1 * v2; v[8] += bb * v2 * v2;
        }
      }
      f0 = warp_sum(f0);
      f1 = warp_sum(f1);
      f2 = warp_sum(f2);
      const double q0 = __shfl_sync(0xffffffffu, gq, 0), q1 = __shfl_sync(0xffffffffu, gq, 1),
                   q2 = __shfl_sync(0xffffffffu, gq, 2);
      if (lane == 0) {
        grad[3 * i] = out_scale * (q0 + f0);
        grad[3 * i + 1] = out_scale * (q1 + f1);
        grad[3 * i + 2] = out_scale * (q2 + f2);
      }
    }
  }
  v[3] = v[1];
  v[6] = v[2];
  v[7] = v[5];
  block_sum_store<9>(v, vir_part + 9 * blockIdx.x);
}

__global__ void __launch_bounds__(256) k_cn_adjoint_global(GridDev g, int n, const int* __restrict__ bin_start,
                                                          const double4* __restrict__ xs,
                                                          const int4* __restrict__ meta,
                                                          const int4* __restrict__ off, const Tables* __restrict__ tab,
                                                          const double* __restrict__ gcn, double* __restrict__ grad,
                                                          double out_scale, double* __restrict__ vir_part,
                                                          const int* __restrict__ hit_n, const int* __restrict__ ovf) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  double v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  const bool any = *ovf != 0;
  for (int t = blockIdx.x * kWarpsPerBlock + wid; any && t < n; t += gridDim.x * kWarpsPerBlock) {
    if (hit_n[t] >= 0) continue;
    const int i = meta[t].w;
    double f[3] = {0, 0, 0};
    cn_adjoint_atom_global(g, bin_start, xs, meta, off, tab, gcn, t, f, v);
    f[0] = warp_sum(f[0]);
    f[1] = warp_sum(f[1]);
    f[2] = warp_sum(f[2]);
    if (lane == 0) {
      grad[3 * i] = out_scale * (grad[3 * i] + f[0]);
      grad[3 * i + 1] = out_scale * (grad[3 * i + 1] + f[1]);
      grad[3 * i + 2] = out_scale * (grad[3 * i + 2] + f[2]);
    }
  }
  v[3] = v[1];
  v[6] = v[2];
  v[7] = v[5];
  block_sum_store<9>(v, vir_part + 9 * blockIdx.x);
}

int launch_cn_adjoint_cells(const CellGrid& g, int n, const CellList& cl, const double* pos_ang,
                            const int32_t* species, const Tables* tab, const double* gcn, double* grad,
                            double out_scale, double* vir_part, int* n_blocks, const HitStore& hs,
                            cudaStream_t s) {
  (void)pos_ang;
  (void)species;
  const int need = (n + kWarpsPerBlock - 1) / kWarpsPerBlock;
  const int blocks = need < 148 * 8 ? need : 148 * 8;   // resident grid, grid-stride over atoms
  const int fb = need < kFallbackBlocks ? need : kFallbackBlocks;
  *n_blocks = blocks + fb;
  if (blocks == 0) return FD3_OK;
  if (hs.is_double)
    k_cn_adjoint_hits<double><<<blocks, 32 * kWarpsPerBlock, 0, s>>>(
        n, cl.meta, gcn, grad, out_scale, vir_part,
        HitList<double>{hs.j, (double4*)hs.ad, hs.n, hs.cap});
  else
    k_cn_adjoint_hits<float><<<blocks, 32 * kWarpsPerBlock, 0, s>>>(
        n, cl.meta, gcn, grad, out_scale, vir_part, HitList<float>{hs.j, (float4*)hs.ad, hs.n, hs.cap});
  FD3_LAUNCHED();
  k_cn_adjoint_global<<<fb, 32 * kWarpsPerBlock, 0, s>>>(to_dev(g), n, cl.bin_start, cl.xs, cl.meta, cl.off, tab,
                                                          gcn, grad, out_scale, vir_part + 9 * (size_t)blocks, hs.n,
                                                          hs.ovf);
  FD3_LAUNCHED();
  return FD3_OK;
}

// ------------------------------------------------------------------ edge-list path
// ------------------------------------------------------------------ edge-list path, fixed order
// Edge keys for the stable counting sorts by source and by destination. An edge whose source
// or destination is outside 0..n-1 raises *bad and is keyed to bucket e mod n (so no bucket
// grows with the number of bad edges); every consumer re-checks the range and skips it.
__global__ void __launch_bounds__(256) k_edge_keys(int64_t ne, int n, const int64_t* __restrict__ src,
                                                  const int64_t* __restrict__ dst, int* __restrict__ ks,
                                                  int* __restrict__ kd, int* __restrict__ bad) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  const int64_t i = src[e], j = dst[e];
  const bool ok = i >= 0 && i < n && j >= 0 && j < n;
  const int spill = (int)(e % n);
  ks[e] = ok ? (int)i : spill;
  kd[e] = ok ? (int)j : spill;
  if (!ok) atomicOr(bad, 1);
}

int launch_edge_index(int64_t n_edges, int n, const int64_t* src, const int64_t* dst, const EdgeIndex& ei,
                      cudaStream_t s) {
  FD3_CUDA(cudaMemsetAsync(ei.bad, 0, sizeof(int), s));
  if (n_edges > 0) {
    const int tb = 256;
    k_edge_keys<<<(unsigned)((n_edges + tb - 1) / tb), tb, 0, s>>>(n_edges, n, src, dst, ei.ks, ei.kd, ei.bad);
    FD3_LAUNCHED();
  }
  int rc = counting_sort(ei.ks, (int)n_edges, n, ei.cnt, ei.st_s, ei.ord_s, s);
  if (rc) return rc;
  return counting_sort(ei.kd, (int)n_edges, n, ei.cnt, ei.st_d, ei.ord_d, s);
}

// CN of atom a: the sum of the smooth-cutoff function over its source edges in edge order
// (core.py:323-386, index_add_ on edge_index[0]); one warp per atom, lanes over the edges, a
// fixed butterfly reduction -- the same result on every run. NaN for every atom when an edge
// index was out of range (the range check the reference leaves to torch indexing). Edges with
// |r|^2 >= mask_r2 contribute nothing (mask_r2 = +inf: every edge counts, as in the reference).
__global__ void __launch_bounds__(256) k_cn_edges_seg(int n, int64_t ne, const int* __restrict__ st,
                                                     const int* __restrict__ ord, const double* __restrict__ x,
                                                     const int32_t* __restrict__ species,
                                                     const int64_t* __restrict__ src, const int64_t* __restrict__ dst,
                                                     const double* __restrict__ sh, const Tables* __restrict__ tab,
                                                     double mask_r2, const int* __restrict__ bad,
                                                     double* __restrict__ cn) {
  const int lane = threadIdx.x & 31;
  const int a = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (a >= n) return;
  const double rca = tab->rcov[species[a]];
  double sum = 0.0;
  for (int p = st[a] + lane; p < st[a + 1]; p += 32) {
    const int e = ord[p];
    const int64_t i = src[e], j = dst[e];
    if (i != a || j < 0 || j >= n) continue;
    const double v0 = x[3 * j] - x[3 * i] + sh[3 * (int64_t)e];
    const double v1 = x[3 * j + 1] - x[3 * i + 1] + sh[3 * (int64_t)e + 1];
    const double v2 = x[3 * j + 2] - x[3 * i + 2] + sh[3 * (int64_t)e + 2];
    const double r2 = v0 * v0 + v1 * v1 + v2 * v2;
    if (r2 >= mask_r2) continue;
    double f, df;
    cn_edge(sqrt(r2), rca + tab->rcov[species[j]], tab->r_cut, f, df);
    sum += f;
  }
  sum = warp_sum(sum);
  if (lane == 0) cn[a] = *bad ? __longlong_as_double(0x7ff8000000000000LL) : sum;
}

int launch_cn_edges_seg(int64_t n_edges, int n, const double* pos, const int32_t* species, const int64_t* src,
                        const int64_t* dst, const double* shift, const Tables* tab, double mask_r2,
                        const EdgeIndex& ei, double* cn, cudaStream_t s) {
  const int wpb = 8;
  k_cn_edges_seg<<<(n + wpb - 1) / wpb, 32 * wpb, 0, s>>>(n, n_edges, ei.st_s, ei.ord_s, pos, species, src, dst,
                                                          shift, tab, mask_r2, ei.bad, cn);
  FD3_LAUNCHED();
  return FD3_OK;
}

// dE/dshift of every edge, g_e = dE/dCN_i f'(r) v / r (zero for an edge out of range).
__global__ void __launch_bounds__(256) k_edge_grad(int64_t ne, int n, const double* __restrict__ x,
                                                  const int32_t* __restrict__ species, const int64_t* __restrict__ src,
                                                  const int64_t* __restrict__ dst, const double* __restrict__ sh,
                                                  const Tables* __restrict__ tab, double mask_r2,
                                                  const double* __restrict__ gcn, double* __restrict__ gshift) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  const int64_t i = src[e], j = dst[e];
  double g0 = 0, g1 = 0, g2 = 0;
  if (i >= 0 && i < n && j >= 0 && j < n) {
    const double v0 = x[3 * j] - x[3 * i] + sh[3 * e];
    const double v1 = x[3 * j + 1] - x[3 * i + 1] + sh[3 * e + 1];
    const double v2 = x[3 * j + 2] - x[3 * i + 2] + sh[3 * e + 2];
    const double r2 = v0 * v0 + v1 * v1 + v2 * v2;
    const double r = sqrt(r2);
    double f, df;
    cn_edge(r, tab->rcov[species[i]] + tab->rcov[species[j]], tab->r_cut, f, df);
    if (r > 1e-6 && r2 < mask_r2) {
      const double a = gcn[i] * df / r;
      g0 = a * v0;
      g1 = a * v1;
      g2 = a * v2;
    }
  }
  gshift[3 * e] = g0;
  gshift[3 * e + 1] = g1;
  gshift[3 * e + 2] = g2;
}

// dE/dpos_a += sum over edges into a of g_e - sum over edges out of a of g_e, each in edge order.
__global__ void __launch_bounds__(256) k_edge_grad_atoms(int n, const int* __restrict__ st_s,
                                                        const int* __restrict__ ord_s, const int* __restrict__ st_d,
                                                        const int* __restrict__ ord_d,
                                                        const double* __restrict__ gshift, double* __restrict__ gpos) {
  const int lane = threadIdx.x & 31;
  const int a = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (a >= n) return;
  double g[3] = {0.0, 0.0, 0.0};
  for (int p = st_d[a] + lane; p < st_d[a + 1]; p += 32) {
    const int64_t e = ord_d[p];
#pragma unroll
    for (int c = 0; c < 3; ++c) g[c] += gshift[3 * e + c];
  }
  for (int p = st_s[a] + lane; p < st_s[a + 1]; p += 32) {
    const int64_t e = ord_s[p];
#pragma unroll
    for (int c = 0; c < 3; ++c) g[c] -= gshift[3 * e + c];
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) g[c] = warp_sum(g[c]);
  if (lane == 0) {
#pragma unroll
    for (int c = 0; c < 3; ++c) gpos[3 * (int64_t)a + c] += g[c];
  }
}

int launch_cn_adjoint_edges_seg(int64_t n_edges, int n, const double* pos, const int32_t* species,
                                const int64_t* src, const int64_t* dst, const double* shift, const Tables* tab,
                                double mask_r2, const double* gcn, const EdgeIndex& ei, double* gpos,
                                double* gshift, cudaStream_t s) {
  if (n_edges > 0) {
    const int tb = 256;
    k_edge_grad<<<(unsigned)((n_edges + tb - 1) / tb), tb, 0, s>>>(n_edges, n, pos, species, src, dst, shift, tab,
                                                                   mask_r2, gcn, gshift);
    FD3_LAUNCHED();
  }
  const int wpb = 8;
  k_edge_grad_atoms<<<(n + wpb - 1) / wpb, 32 * wpb, 0, s>>>(n, ei.st_s, ei.ord_s, ei.st_d, ei.ord_d, gshift, gpos);
  FD3_LAUNCHED();
  return FD3_OK;
}


// Softmax interpolation over the 7 reference CNs and the rank-r factors
// c_r = sum_p w_p V[s, p, r] (core.py:449-478, 525-532), their CN derivative (times the
// cncorr slope) and the self term sum_r lambda_r c_r^2 phi_ss(0) (core.py:545-550). One thread
// per atom; cn holds the raw CN on entry and the corrected CN on exit.
__global__ void __launch_bounds__(256) k_c6_atoms(int n, const int32_t* __restrict__ species,
                                                 const Tables* __restrict__ tab, const double* __restrict__ V, int R,
                                                 double* __restrict__ cn, double* __restrict__ c6,
                                                 double* __restrict__ dc6, double* __restrict__ self_part) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double selfv = 0.0;
  if (i < n) {
    const int s = species[i];
    double cnv = cn[i], slope = 1.0;
    if (tab->has_cncorr) {
      slope = tab->cncorr[2 * s + 1];
      cnv = slope * cnv + tab->cncorr[2 * s + 0];
    }
    double lg[7], dl[7];
    double mx = -INFINITY;
#pragma unroll
    for (int p = 0; p < 7; ++p) {
      const double ref = tab->cnref[7 * s + p];
      const double diff = cnv - ref;
      const bool ok = ref != -1.0;
      lg[p] = ok ? -4.0 * (diff * diff) : -INFINITY;
      dl[p] = ok ? -8.0 * diff : 0.0;
      mx = fmax(mx, lg[p]);
    }
    double sum = 0.0;
#pragma unroll
    for (int p = 0; p < 7; ++p) {
      lg[p] = lg[p] == -INFINITY ? 0.0 : exp(lg[p] - mx);
      sum += lg[p];
    }
    const double inv = 1.0 / sum;
    double dlbar = 0.0;
#pragma unroll
    for (int p = 0; p < 7; ++p) {
      lg[p] *= inv;                   // softmax weight w_p
      dlbar += lg[p] * dl[p];
    }
    for (int r = 0; r < R; ++r) {
      double c = 0.0, d = 0.0;
#pragma unroll
      for (int p = 0; p < 7; ++p) {
        const double v = V[(7 * s + p) * R + r];
        c += lg[p] * v;
        d += lg[p] * (dl[p] - dlbar) * v;
      }
      c6[(size_t)i * R + r] = c;
      dc6[(size_t)i * R + r] = slope * d;
      selfv += tab->eigs[r] * c * c * tab->selfcont[s];
    }
    cn[i] = cnv;
  }
  double v1[1] = {selfv};
  block_sum_store<1>(v1, self_part + blockIdx.x);
}

int launch_c6_atoms(int n, const int32_t* species, const Tables* tab, const double* eigvecs, int R,
                    const double* cn, double* c6, double* dc6, double* self_part, int* n_self_blocks,
                    cudaStream_t s) {
  const int blocks = (n + 255) / 256;
  *n_self_blocks = blocks;
  if (blocks == 0) return FD3_OK;
  k_c6_atoms<<<blocks, 256, 0, s>>>(n, species, tab, eigvecs, R, const_cast<double*>(cn), c6, dc6, self_part);
  FD3_LAUNCHED();
  return FD3_OK;
}


// ------------------------------------------------------------------ neighbour export
__global__ void __launch_bounds__(256) k_nbr_count(GridDev g, int n, const int* __restrict__ bin_start,
                                                  const double4* __restrict__ xs, const int4* __restrict__ meta,
                                                  const int4* __restrict__ off, int* __restrict__ counts) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int t = blockIdx.x * kWarpsPerBlock + wid;
  if (t >= n) return;
  const double4 xi = xs[t];
  const int i = meta[t].w;
  int cnt = 0;
  visit_neighbors(g, bin_start, xs, meta, i, xi.x, xi.y, xi.z, off[i],
                  [&](bool hit, int, int, int, int, int, double, double, double) {
                    cnt += __popc(__ballot_sync(0xffffffffu, hit));
                  });
  if (lane == 0) counts[i] = cnt;
}

__global__ void __launch_bounds__(256) k_nbr_fill(GridDev g, int n, const int* __restrict__ bin_start,
                                                 const double4* __restrict__ xs, const int4* __restrict__ meta,
                                                 const int4* __restrict__ off, const int* __restrict__ row_start,
                                                 int64_t* __restrict__ src, int64_t* __restrict__ dst,
                                                 int32_t* __restrict__ shift) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int t = blockIdx.x * kWarpsPerBlock + wid;
  if (t >= n) return;
  const double4 xi = xs[t];
  const int i = meta[t].w;
  int pos = row_start[i];
  visit_neighbors(g, bin_start, xs, meta, i, xi.x, xi.y, xi.z, off[i],
                  [&](bool hit, int, int j, int S0, int S1, int S2, double, double, double) {
                    const unsigned m = __ballot_sync(0xffffffffu, hit);
                    if (hit) {
                      const int k = pos + __popc(m & ((1u << lane) - 1u));
                      src[k] = i;
                      dst[k] = j;
                      shift[3 * k] = S0;
                      shift[3 * k + 1] = S1;
                      shift[3 * k + 2] = S2;
                    }
                    pos += __popc(m);
                  });
}

// ------------------------------------------------------------------ direct pair sum (float64)
// The accuracy oracle's lattice sum on the device: over every image pair (i, j, n) closer than
// the grid's cutoff (r_direct) except i = j at n = 0, with C6_ij = sum_r lambda_r c_ir c_jr
// (the plan's low-rank factors) and the BJ-damped kernel of src/fourierd3/pair_pot.py:64,
//   phi(r) = s6 / (r^6 + R0^6) + 3 s8 qq / (r^8 + R0^8),  E = -1/2 sum C6 phi   (Bohr, Hartree).
// Warp per atom i over the bin-sorted atoms: e_i = sum_j C6 phi, dE/dc_ir = -lambda_r sum_j
// c_jr phi, dE/dx_i = sum_j C6 (phi'/r) d (d = x_j + n - x_i; each pair is seen from both ends),
// and per block e = sum_i e_i and the virial -1/2 sum C6 (phi'/r) d_a d_b (6 components).
__global__ void __launch_bounds__(256) k_direct_pairs(GridDev g, int n, const int* __restrict__ bin_start,
                                                     const double4* __restrict__ xs, const int4* __restrict__ meta,
                                                     const int4* __restrict__ off, const double* __restrict__ c6,
                                                     const Tables* __restrict__ tab, int R, int S,
                                                     const GreenPair* __restrict__ gp, double* __restrict__ dEdc,
                                                     double* __restrict__ grad, double* __restrict__ part) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int t = blockIdx.x * kWarpsPerBlock + wid;
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};   // e, virial xx xy xz yy yz zz
  if (t < n) {
    const double4 xi = xs[t];
    const int i = meta[t].w;
    const int Xi = (int)xi.w;
    const double s6 = tab->s6, s8 = tab->s8;
    double ci[8], gc[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      ci[r] = r < R ? tab->eigs[r] * c6[(size_t)i * R + r] : 0.0;
      gc[r] = 0.0;
    }
    double e = 0.0, g0 = 0.0, g1 = 0.0, g2 = 0.0, v[6] = {0, 0, 0, 0, 0, 0};
    visit_neighbors(g, bin_start, xs, meta, i, xi.x, xi.y, xi.z, off[i],
                    [&](bool hit, int u, int j, int, int, int, double d0, double d1, double d2) {
                      if (!hit) return;
                      const double b0 = d0 * kAngToBohr, b1 = d1 * kAngToBohr, b2 = d2 * kAngToBohr;
                      const double r2 = b0 * b0 + b1 * b1 + b2 * b2;
                      const GreenPair q = gp[Xi * S + (int)xs[u].w];
                      const double R02 = q.R * q.R, R06 = R02 * R02 * R02, R08 = R06 * R02;
                      const double r4 = r2 * r2, r6 = r4 * r2, r8 = r6 * r2;
                      const double den6 = r6 + R06, den8 = r8 + R08;
                      const double phi = s6 / den6 + 3.0 * s8 * q.qq / den8;
                      const double dphi_r = -6.0 * s6 * r4 / (den6 * den6) - 24.0 * s8 * q.qq * r6 / (den8 * den8);
                      double C6 = 0.0;
#pragma unroll
                      for (int r = 0; r < 8; ++r)
                        if (r < R) {
                          const double cj = c6[(size_t)j * R + r];
                          C6 += ci[r] * cj;
                          gc[r] += cj * phi;
                        }
                      e += C6 * phi;
                      const double w = C6 * dphi_r;
                      g0 += w * b0;
                      g1 += w * b1;
                      g2 += w * b2;
                      v[0] += w * b0 * b0;
                      v[1] += w * b0 * b1;
                      v[2] += w * b0 * b2;
                      v[3] += w * b1 * b1;
                      v[4] += w * b1 * b2;
                      v[5] += w * b2 * b2;
                    });
    e = warp_sum(e);
    g0 = warp_sum(g0);
    g1 = warp_sum(g1);
    g2 = warp_sum(g2);
#pragma unroll
    for (int r = 0; r < 8; ++r) gc[r] = warp_sum(gc[r]);
#pragma unroll
    for (int c = 0; c < 6; ++c) v[c] = warp_sum(v[c]);
    if (lane == 0) {
      for (int r = 0; r < R; ++r) dEdc[(size_t)i * R + r] = -tab->eigs[r] * gc[r];
      grad[3 * (size_t)i] = g0;
      grad[3 * (size_t)i + 1] = g1;
      grad[3 * (size_t)i + 2] = g2;
      acc[0] = e;
#pragma unroll
      for (int c = 0; c < 6; ++c) acc[1 + c] = -0.5 * v[c];
    }
  }
  block_sum_store<7>(acc, part + 7 * blockIdx.x);
}

int launch_direct_pairs(const CellGrid& g, int n, const CellList& cl, const double* c6, const Tables* tab, int R,
                        int S, const GreenPair* gp, double* dEdc, double* grad, double* part, int* n_blocks,
                        cudaStream_t s) {
  if (R < 1 || R > 8) {
    set_error("direct sum", "the direct pair sum takes at most 8 ranks");
    return FD3_EINVAL;
  }
  const int blocks = (n + kWarpsPerBlock - 1) / kWarpsPerBlock;
  *n_blocks = blocks;
  if (blocks == 0) return FD3_OK;
  k_direct_pairs<<<blocks, 32 * kWarpsPerBlock, 0, s>>>(to_dev(g), n, cl.bin_start, cl.xs, cl.meta, cl.off, c6, tab,
                                                        R, S, gp, dEdc, grad, part);
  FD3_LAUNCHED();
  return FD3_OK;
}

int launch_nbr_count(const CellGrid& g, int n, const CellList& cl, const double* pos_ang, int* counts,
                     cudaStream_t s) {
  (void)pos_ang;
  const int blocks = (n + kWarpsPerBlock - 1) / kWarpsPerBlock;
  if (blocks == 0) return FD3_OK;
  k_nbr_count<<<blocks, 32 * kWarpsPerBlock, 0, s>>>(to_dev(g), n, cl.bin_start, cl.xs, cl.meta, cl.off, counts);
  FD3_LAUNCHED();
  return FD3_OK;
}

int launch_nbr_fill(const CellGrid& g, int n, const CellList& cl, const double* pos_ang, const int* row_start,
                    int64_t* src, int64_t* dst, int32_t* shift, cudaStream_t s) {
  (void)pos_ang;
  const int blocks = (n + kWarpsPerBlock - 1) / kWarpsPerBlock;
  if (blocks == 0) return FD3_OK;
  k_nbr_fill<<<blocks, 32 * kWarpsPerBlock, 0, s>>>(to_dev(g), n, cl.bin_start, cl.xs, cl.meta, cl.off, row_start,
                                                     src, dst, shift);
  FD3_LAUNCHED();
  return FD3_OK;
}

}  // namespace fd3

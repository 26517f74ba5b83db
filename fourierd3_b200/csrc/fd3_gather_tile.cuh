// Tile-staged mesh gather (reference: src/fourierd3/mesh_interpolator_d3.py:140-189, the
// mesh-to-points interpolation, and the force / C6-factor adjoint that autograd takes of it in
// core.py:553-581).
//
// One CTA per (mesh tile, species) key of the spread's counting sort. The potential of the key's
// species over the tile grown by the stencil reach, a box of (t0+p-1) x (t1+p-1) x (t2+p-1,
// rounded up to 16 bytes) points in every rank channel, comes into shared memory ONCE for all
// of the key's atoms: by one 4-D TMA load (cp.async.bulk.tensor, no multicast, this GPU's own
// mesh) when the box does not cross the upper mesh edge, by plain wrapped loads when it does.
// The CTA's warps then gather their atoms from shared memory: warp per atom, lanes over the
// (y, z) stencil nodes (bank-conflict free for p <= 5 with the 12-point z extent), the x
// nodes unrolled in registers.
//
// Opt-in (FD3_TUNE_GATHER_TILE = 1). On B200 at 2.5 to 8.5 atoms per (tile, species) key (the
// 41,472- and 139,968-atom SiO2 boxes on the 256^3 mesh, p = 5, rank 4) it is 4 to 9 times
// slower than the per-atom gather: each key stages a 76.8 KB box for atoms whose z-runs need
// 3.2 KB each, the box load's latency is exposed with two CTAs per SM, and boxes at the upper
// mesh edge take scalar wrapped loads. It pays only where keys hold many atoms.
//
// Per atom i of species s with stencil weights W = w_x w_y w_z (and dW/du_a):
//   P_r  = sum_m W(m) phi_sr(m)                       (rank-r mesh potential at the atom)
//   g_a  = sum_m dW/du_a(m) sum_r lambda_r c_ir phi_sr(m)
// from which dE/dCN_i and dE/dx_i follow exactly as in the per-atom gather.
//
// Included from fd3_mesh_impl.cuh (it uses MeshDev, to_dev and MeshRecords from there).
#pragma once
#include <cudaTypedefs.h>
#include <string.h>

#include "fd3_async.cuh"

namespace fd3 {

constexpr int kTileGatherWarps = 8;
// dynamic shared memory of one CTA at most (the staged box and its 128-byte alignment pad):
// two CTAs per SM with the 1 KB each reserves
constexpr size_t kTileGatherSmemCap = 113 * 1024;

struct GatherBox {
  int x, y, z;   // staged points per axis (z rounded up to 16 bytes)
};

inline GatherBox gather_box(const MeshGeom& mg, size_t elem) {
  const int vz = (int)(16 / elem);
  GatherBox b;
  b.x = mg.t[0] + mg.order - 1;
  b.y = mg.t[1] + mg.order - 1;
  b.z = (mg.t[2] + mg.order - 1 + vz - 1) / vz * vz;
  return b;
}

// (gather_tile_applies, declared in fd3_internal.h, is defined in fd3_gather_f32.cu)

// One (y, z) stencil column of one atom, x nodes unrolled: xr_r = sum_x w_x phi_r,
// s0 = sum_x w_x cp_x, s1 = sum_x w'_x cp_x with cp_x = sum_r lambda_r c_r phi_r. BOX: from the
// staged box (col = the column's first node, cs / xs its channel and x strides); otherwise from
// global memory at the wrapped nodes (ix0 + kx, iy, iz) of the species' channels gsp.
template <typename T, int P, int MAXR, bool BOX>
__device__ __forceinline__ void tile_column(const T* col, int cs, int xs, const T* gsp, int ix0, int iy, int iz,
                                            const MeshDev& g, int R, const T (&wx)[P], const T (&dwx)[P],
                                            const T (&cl)[MAXR], T (&xr)[MAXR], T& s0, T& s1) {
  size_t yz = 0, M = 0;
  if (!BOX) {
    while (iy >= g.n[1]) iy -= g.n[1];
    while (iz >= g.n[2]) iz -= g.n[2];
    M = (size_t)g.n[0] * g.n[1] * g.n[2];
    yz = (size_t)iy * g.n[2] + iz;
  }
#pragma unroll
  for (int r = 0; r < MAXR; ++r) xr[r] = T(0);
  s0 = T(0);
  s1 = T(0);
#pragma unroll
  for (int kx = 0; kx < P; ++kx) {
    T cp = T(0);
    size_t xo = 0;
    if (!BOX) {
      int ix = ix0 + kx;
      while (ix >= g.n[0]) ix -= g.n[0];
      xo = (size_t)ix * g.n[1] * g.n[2] + yz;
    }
#pragma unroll
    for (int r = 0; r < MAXR; ++r) {
      if (r < R) {
        const T f = BOX ? col[r * cs + kx * xs] : gsp[(size_t)r * M + xo];
        xr[r] += wx[kx] * f;
        cp += cl[r] * f;
      }
    }
    s0 += wx[kx] * cp;
    s1 += dwx[kx] * cp;
  }
}

template <typename T, int P, int MAXR>
__global__ void __launch_bounds__(32 * kTileGatherWarps, 2)
    k_gather_tile(const __grid_constant__ CUtensorMap tmap, MeshDev g, int bx, int by, int bz,
                  const int* __restrict__ key_start, const double* __restrict__ c6, const double* __restrict__ dc6,
                  const CellInfo* __restrict__ ci, const Tables* __restrict__ tab, const int* __restrict__ order,
                  const int4* __restrict__ rb, const T* __restrict__ rw, const T* __restrict__ rdw,
                  const T* __restrict__ phi, double* __restrict__ gcn, double* __restrict__ gpos) {
  extern __shared__ __align__(128) unsigned char gt_smem[];
  __shared__ __align__(8) uint64_t full;
  // the staged box on a 128-byte boundary (the launch adds the padding)
  T* blk = reinterpret_cast<T*>(gt_smem + ((128u - (smem_u32(gt_smem) & 127u)) & 127u));
  const int key = blockIdx.x;
  const int a0 = key_start[key], a1 = key_start[key + 1];
  if (a0 >= a1) return;   // no atoms: nothing staged (uniform over the CTA)
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int R = g.R;
  const int s = key % g.S;
  int tl = key / g.S;
  const int tz = tl % g.nt[2];
  tl /= g.nt[2];
  const int ty = tl % g.nt[1];
  const int tx = tl / g.nt[1];
  const int x0 = tx * g.t[0], y0 = ty * g.t[1], z0 = tz * g.t[2];
  const int cs = bx * by * bz;   // points per channel of the box
  const int xs = by * bz;        // x stride of the box
  const bool tma = x0 + bx <= g.n[0] && y0 + by <= g.n[1] && z0 + bz <= g.n[2];
  bool ok = true;
  if (tma) {
    if (threadIdx.x == 0) {
      mbar_init(&full, 1);
      mbar_fence_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      mbar_arrive_expect_tx(&full, (uint32_t)((size_t)R * cs * sizeof(T)));
      tma_load_4d(blk, &tmap, z0, y0, x0, s * R, &full);
    }
    ok = mbar_wait(&full, 0);
  } else {
    // the box crosses the upper mesh edge: plain loads, each index wrapped (a mesh narrower
    // than the box wraps more than once)
    const size_t M = (size_t)g.n[0] * g.n[1] * g.n[2];
    const T* src = phi + (size_t)s * R * M;
    const int tot = R * cs;
    for (int e = threadIdx.x; e < tot; e += blockDim.x) {
      int q = e;
      const int lz = q % bz;
      q /= bz;
      const int ly = q % by;
      q /= by;
      const int lx = q % bx;
      const int r = q / bx;
      int ix = x0 + lx, iy = y0 + ly, iz = z0 + lz;
      while (ix >= g.n[0]) ix -= g.n[0];
      while (iy >= g.n[1]) iy -= g.n[1];
      while (iz >= g.n[2]) iz -= g.n[2];
      blk[e] = src[(size_t)r * M + ((size_t)ix * g.n[1] + iy) * g.n[2] + iz];
    }
    __syncthreads();
  }
  const double inv_vol = 1.0 / ci->volume;
  for (int t = a0 + wid; t < a1; t += kTileGatherWarps) {
    const int i = order[t];
    if (!ok) {   // the staging load never completed: the results are marked invalid
      if (lane == 0) {
        const double nan = __longlong_as_double(0x7ff8000000000000LL);
        gcn[i] = nan;
        gpos[3 * i] = gpos[3 * i + 1] = gpos[3 * i + 2] = nan;
      }
      continue;
    }
    const int4 b4 = rb[t];
    const T* wr = rw + (size_t)t * 3 * P;
    const T* dwr = rdw + (size_t)t * 3 * P;
    T wx[P], dwx[P];
#pragma unroll
    for (int k = 0; k < P; ++k) {
      wx[k] = wr[k];
      dwx[k] = dwr[k];
    }
    T cl[MAXR];
#pragma unroll
    for (int r = 0; r < MAXR; ++r) cl[r] = r < R ? (T)(c6[(size_t)i * R + r] * tab->eigs[r]) : T(0);
    // the atom's first stencil node inside the box (its tile is the key's tile: the key and the
    // record take the node from the same float64 location; an atom found outside the tile all
    // the same is gathered from global memory)
    const int ox = b4.x - x0, oy = b4.y - y0, oz = b4.z - z0;
    const bool inbox =
        (unsigned)ox < (unsigned)g.t[0] && (unsigned)oy < (unsigned)g.t[1] && (unsigned)oz < (unsigned)g.t[2];
    const T* org = blk + ((size_t)(inbox ? ox : 0) * by + (inbox ? oy : 0)) * bz + (inbox ? oz : 0);
    const T* gsp = phi + (size_t)s * R * ((size_t)g.n[0] * g.n[1] * g.n[2]);
    double pr[MAXR];
#pragma unroll
    for (int r = 0; r < MAXR; ++r) pr[r] = 0.0;
    double gu0 = 0.0, gu1 = 0.0, gu2 = 0.0;
    for (int q = lane; q < P * P; q += 32) {
      const int ky = q / P, kz = q - ky * P;
      const T wy = wr[P + ky], dwy = dwr[P + ky], wz = wr[2 * P + kz], dwz = dwr[2 * P + kz];
      T xr[MAXR], s0, s1;
      if (inbox)
        tile_column<T, P, MAXR, true>(org + ky * bz + kz, cs, xs, nullptr, 0, 0, 0, g, R, wx, dwx, cl, xr, s0, s1);
      else
        tile_column<T, P, MAXR, false>(nullptr, 0, 0, gsp, b4.x, b4.y + ky, b4.z + kz, g, R, wx, dwx, cl, xr, s0, s1);
      const T wyz = wy * wz;
#pragma unroll
      for (int r = 0; r < MAXR; ++r) pr[r] += (double)(wyz * xr[r]);
      gu0 += (double)(wyz * s1);
      gu1 += (double)(dwy * wz * s0);
      gu2 += (double)(wy * dwz * s0);
    }
#pragma unroll
    for (int r = 0; r < MAXR; ++r) pr[r] = warp_sum(pr[r]);
    gu0 = warp_sum(gu0);
    gu1 = warp_sum(gu1);
    gu2 = warp_sum(gu2);
    if (lane == 0) {
      // dE/dc_r = -(lambda_r / Omega) P_r + lambda_r c_r phi_ss(0); dE/dCN = sum_r dE/dc_r dc_r/dCN
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
      // dE/du_a = -(1/Omega) g_a; dE/dx_b = sum_a dE/du_a n_a inv[b][a]
      const double du[3] = {-inv_vol * gu0, -inv_vol * gu1, -inv_vol * gu2};
      gcn[i] = gsum;
#pragma unroll
      for (int b = 0; b < 3; ++b)
        gpos[3 * i + b] = du[0] * g.n[0] * ci->inv[3 * b + 0] + du[1] * g.n[1] * ci->inv[3 * b + 1] +
                          du[2] * g.n[2] * ci->inv[3 * b + 2];
    }
  }
}

// Potential phi (layout (S R, nx, ny, nz)) as a 4-D tensor {nz, ny, nx, S R}; box
// {bz, by, bx, R}: the staged block of one key. Grid: one CTA per key.
template <typename T, int P>
int launch_gather_tile(const MeshGeom& mg, int n, const double* c6, const double* dc6, const CellInfo* ci,
                       const Tables* tab, const int* order, const int* key_start, const MeshRecords& rec,
                       const T* phi, double* gcn, double* gpos, cudaStream_t s) {
  if (!gather_tile_applies(mg, sizeof(T))) {
    set_error("gather", "the tile-staged gather does not apply to this mesh");
    return FD3_EINVAL;
  }
  auto fn = tensor_map_encoder();
  if (!fn) {
    set_error("gather", "cuTensorMapEncodeTiled is not available from the driver");
    return FD3_ECUDA;
  }
  (void)n;
  const GatherBox b = gather_box(mg, sizeof(T));
  const size_t es = sizeof(T);
  const cuuint64_t dims[4] = {(cuuint64_t)mg.n[2], (cuuint64_t)mg.n[1], (cuuint64_t)mg.n[0],
                              (cuuint64_t)mg.S * mg.R};
  const cuuint64_t strides[3] = {(cuuint64_t)mg.n[2] * es, (cuuint64_t)mg.n[1] * mg.n[2] * es,
                                 (cuuint64_t)mg.n[0] * mg.n[1] * mg.n[2] * es};
  const cuuint32_t box[4] = {(cuuint32_t)b.z, (cuuint32_t)b.y, (cuuint32_t)b.x, (cuuint32_t)mg.R};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  CUtensorMap map;
  memset(&map, 0, sizeof(map));
  // a mesh narrower than the box along some axis has no interior tile: every box is staged by
  // plain loads and the (unused) map stays empty
  if (b.x <= mg.n[0] && b.y <= mg.n[1] && b.z <= mg.n[2]) {
    const CUresult r = fn(&map, es == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4,
                          const_cast<T*>(phi), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
      set_error("gather", "cuTensorMapEncodeTiled rejected the potential's tensor map");
      return FD3_ECUDA;
    }
  }
  const size_t smem = (size_t)mg.R * b.x * b.y * b.z * es + 128;   // + alignment padding
  const long long keys = (long long)mg.nt[0] * mg.nt[1] * mg.nt[2] * mg.S;
  if (keys <= 0 || keys > (1LL << 31) - 1) return FD3_EINVAL;
  auto kern = mg.R <= 4 ? k_gather_tile<T, P, 4> : k_gather_tile<T, P, 8>;
  int dev = 0;
  cudaGetDevice(&dev);
  static unsigned attr_set = 0;   // bit 2 dev + (R > 4) per device (set on every call past 16)
  const unsigned bit = dev < 16 ? 1u << (2 * dev + (mg.R > 4 ? 1 : 0)) : 0u;
  if (!bit || !(attr_set & bit)) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTileGatherSmemCap) !=
        cudaSuccess) {
      set_error("gather", "could not raise the shared-memory limit of the tile-staged gather");
      return FD3_ECUDA;
    }
    attr_set |= bit;
  }
  kern<<<(unsigned)keys, 32 * kTileGatherWarps, smem, s>>>(map, to_dev(mg), b.x, b.y, b.z, key_start, c6, dc6, ci,
                                                           tab, order, rec.b, (const T*)rec.w, (const T*)rec.dw, phi,
                                                           gcn, gpos);
  FD3_LAUNCHED();
  return FD3_OK;
}

}  // namespace fd3

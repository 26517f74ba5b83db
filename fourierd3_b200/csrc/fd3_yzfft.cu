// Fused (y, z) plane transforms of the float mesh, one pass each way, on thread-block clusters
// (of 2 or 4 CTAs) that share one 256 x 256 plane through distributed shared memory. They replace
// the 2D cuFFT R2C / C2R around the TMA x-pass (the reference's torch.fft.rfftn / irfftn over the
// mesh, kspace_filter_d3.py:55-68, of which the x axis is transformed by the x-pass): cuFFT makes
// two passes over the mesh each way (z, then y), these kernels make one.
//
// Layouts (as cuFFT's batched 2D transforms over (y, z) leave them): plane p = (channel, x) of
// the real mesh at rho + p 256 256, of the half spectrum at spec + p 256 P (ky rows of the 129
// kz values, P = 129; or P = 130 with a zero pad slot when the TMA x-pass shares the spectrum,
// so that every row starts on a 16-byte boundary).
//
// Columns: kz = 1..127 are complex; kz = 0 and kz = 128 come out of the z transform real, so
// they travel as one packed complex column X[y][0] + i X[y][128] (one y FFT gives both, split by
// Hermitian symmetry). That leaves 128 columns, 128 / CL per CTA of a cluster of CL: rank 0 holds
// the packed column and kz = 1 .. 128/CL - 1, rank r holds kz = r 128/CL .. (r+1) 128/CL - 1.
//
// Forward, per plane (cluster rank q owns rows y in [q 256/CL, (q+1) 256/CL) for the z transform):
//   1. rows arrive in chunks of 64/CL (one bulk copy each, mbarrier-tracked ring of two; one half
//      of the CTA's warps takes the even chunks, the other the odd ones, so one chunk loads while
//      two compute);
//   2. each warp transforms 4 rows: the 256 reals as 128 complex values z[m] = x[2m] + i x[2m+1],
//      a 128-point FFT as 8 x 16 register DFTs (pass 1 from the natural row, pass 2 on a
//      bank-swizzled copy in place), and the real-to-half-complex split
//      X[k] = ((Z[k] + Z*[128-k]) - i W256^k (Z[k] - Z*[128-k])) / 2 from registers (the lane
//      holding Z[128-k] is found by a shuffle);
//   3. X[y][kz] is stored straight into the shared memory of the CTA that owns column kz (its own
//      or another's, st.shared::cluster);
//   4. after a cluster barrier, each CTA runs the 256-point y FFTs of its columns in place
//      (16 x 16 register DFTs, two passes) and writes them to the spectrum from registers.
// Inverse, always on pairs: the mirror image (each CTA's 64 columns of a plane arrive by one 2-D
// TMA load when the rows are padded, by plain loads otherwise; inverse y FFTs; cluster barrier;
// per row the half-complex-to-real packing Z[k] = (X[k] + X*[128-k]) + i W256^-k (X[k] - X*[128-k])
// read across the cluster, an inverse 128-point FFT, the real row written from registers). Both
// are unnormalised, as cuFFT. Both prefetch the next plane into L2 while they work on this one.
//
// The mbarrier waits are bounded; a wait that runs out stops the kernel's loads and marks its
// output NaN so the result cannot pass for a valid one. Every CTA of a cluster always takes the
// same barriers.
#include <cuda.h>

#include "fd3_async.cuh"
#include "fd3_xfilter.cuh"

namespace fd3 {

namespace {

constexpr int kYzN = 256;   // ny = nz
constexpr int kYzH = 129;   // nz / 2 + 1

// Shape of the cluster that shares one plane: CL = 2 (pairs of 512-thread CTAs, one per SM) or
// 4 (quads of 256-thread CTAs, two per SM, so that one CTA's loads overlap the other's
// arithmetic). A CTA owns 256 / CL rows for the z transform and 128 / CL columns (the packed
// kz = 0 / 128 column and kz = 1 .. 127) for the y transform.
template <int CL>
struct YzCfg {
  static constexpr int kThreads = 1024 / CL;
  static constexpr int kWarps = kThreads / 32;
  static constexpr int kRows = kYzN / CL;       // rows per CTA
  static constexpr int kCols = 128 / CL;        // columns per CTA
  static constexpr int kLogCols = CL == 2 ? 6 : 5;
  static constexpr int kLDB = kCols + 4;        // a warp's four rows of 8 columns on distinct banks
  static constexpr int kChunk = 64 / CL;        // rows per staged chunk: 4 per warp of a half-CTA group
  static constexpr int kGroupThreads = kThreads / 2;
  static constexpr int kMinBlocks = CL == 4 ? 2 : 1;
};

template <int CL>
struct YzSmem {
  using C = YzCfg<CL>;
  float2 B[kYzN * C::kLDB];           // the CTA's columns of the plane, rows in y (or ky)
  float2 ring[2][C::kChunk * 128];    // forward: two staged chunks; inverse: 4 row buffers per warp
  float2 tw128[8 * 16];               // W128^(m2 k1) at k1 16 + m2
  float2 tw256[16 * 16];              // W256^(n2 k1) at k1 16 + n2
  float2 wk[kYzH + 1];                // W256^k, k = 0..128
  uint64_t full[2];
  int fail;
};

__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;\n" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t map_rank(uint32_t saddr, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;\n" : "=r"(r) : "r"(saddr), "r"(rank));
  return r;
}
// Distributed-shared-memory store / load. No "memory" clobber: they are ordered against the
// other CTAs' accesses by the cluster barriers (which carry one), and leaving the compiler free
// to schedule ordinary shared-memory accesses around them keeps several of them in flight.
__device__ __forceinline__ void st_cluster(uint32_t addr, float2 v) {
  asm volatile("st.shared::cluster.v2.f32 [%0], {%1, %2};\n" ::"r"(addr), "f"(v.x), "f"(v.y));
}
__device__ __forceinline__ float2 ld_cluster(uint32_t addr) {
  float2 v;
  asm volatile("ld.shared::cluster.v2.f32 {%0, %1}, [%2];\n" : "=f"(v.x), "=f"(v.y) : "r"(addr));
  return v;
}
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release;\nbarrier.cluster.wait.acquire;\n" ::: "memory");
}
// A barrier that orders nothing but execution: for "every CTA has finished reading" points,
// where the reads are complete (their values consumed) before the arrive issues, so no fence
// (and no wait for this thread's outstanding global stores) is needed.
__device__ __forceinline__ void cluster_sync_exec() {
  asm volatile("barrier.cluster.arrive.relaxed;\nbarrier.cluster.wait;\n" ::: "memory");
}
// Bring `bytes` of global memory into L2 ahead of use (no data returned to the SM).
__device__ __forceinline__ void prefetch_l2(const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void group_bar(int g, int nthreads) {   // one half of the CTA
  asm volatile("bar.sync %0, %1;\n" ::"r"(g + 1), "r"(nthreads) : "memory");
}
// 1-D bulk copy global -> shared (this CTA), completion counted on `bar`
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Position of logical element (hi, lo) of a 128-point row in the swizzled layout: lo xor hi xor
// 8 (row parity) keeps both register-DFT passes of a warp's four rows free of bank conflicts.
__device__ __forceinline__ int zsw(int hi, int lo, int par) { return hi * 16 + (lo ^ hi ^ (par << 3)); }

__device__ __forceinline__ float2 cmulc(float2 a, float2 w, bool conj) {
  const float wy = conj ? -w.y : w.y;
  return float2{a.x * w.x - a.y * wy, a.x * wy + a.y * w.x};
}

// 128-point complex FFT (SIGN -1 forward, +1 inverse) of the four rows at rows[r 128 + m]
// (natural order in, m = 16 m1 + m2); on return lane (r = lane / 8, k1 = lane % 8) holds
// Z[k1 + 8 k2], k2 = 0..15, of row r in (re, im), and the rows hold pass-1 values (swizzled).
template <int SIGN>
__device__ __forceinline__ void fft128_rows(float2* rows, const float2* tw128, int lane, float (&re)[16],
                                            float (&im)[16]) {
  const int m2 = lane & 15, rA = lane >> 4;
  float ar[2][8], ai[2][8];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const float2* src = rows + (rA + 2 * h) * 128 + m2;
#pragma unroll
    for (int m1 = 0; m1 < 8; ++m1) {
      const float2 v = src[16 * m1];
      ar[h][m1] = v.x;
      ai[h][m1] = v.y;
    }
  }
  __syncwarp();
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int r = rA + 2 * h;
    dft_reg<float, 8, SIGN>(ar[h], ai[h]);
    float2* dst = rows + r * 128;
#pragma unroll
    for (int k1 = 0; k1 < 8; ++k1)
      dst[zsw(k1, m2, r & 1)] = cmulc(float2{ar[h][k1], ai[h][k1]}, tw128[k1 * 16 + m2], SIGN > 0);
  }
  __syncwarp();
  const int r = lane >> 3, k1 = lane & 7;
  const float2* row = rows + r * 128;
#pragma unroll
  for (int n2 = 0; n2 < 16; ++n2) {
    const float2 v = row[zsw(k1, n2, r & 1)];
    re[n2] = v.x;
    im[n2] = v.y;
  }
  dft_reg<float, 16, SIGN>(re, im);
}

// Pass 1 of the 256-point y FFT (16 x 16) of column col on its 16 natural-order values v[n1]
// (index 16 n1 + n2): DFT over n1, twiddle W256^(SIGN n2 k1), value of (k1, n2) to row 16 k1 + n2.
template <int SIGN, int LDB>
__device__ __forceinline__ void ypass1_store(float (&re)[16], float (&im)[16], int n2, int col, float2* B,
                                             const float2* tw256) {
  dft_reg<float, 16, SIGN>(re, im);
#pragma unroll
  for (int k1 = 0; k1 < 16; ++k1)
    B[(16 * k1 + n2) * LDB + col] = cmulc(float2{re[k1], im[k1]}, tw256[k1 * 16 + n2], SIGN > 0);
}
// Pass 2: rows 16 k1 + n2 of column col -> Y[k1 + 16 k2] in (re[k2], im[k2]).
template <int SIGN, int LDB>
__device__ __forceinline__ void ypass2_load(float (&re)[16], float (&im)[16], int k1, int col, const float2* B) {
#pragma unroll
  for (int n2 = 0; n2 < 16; ++n2) {
    const float2 v = B[(16 * k1 + n2) * LDB + col];
    re[n2] = v.x;
    im[n2] = v.y;
  }
  dft_reg<float, 16, SIGN>(re, im);
}

template <int CL>
__device__ void yz_tables(YzSmem<CL>& sm) {
  for (int m = threadIdx.x; m < 128 + 256 + kYzH; m += blockDim.x) {
    double sn, cs;
    if (m < 128) {
      const int k1 = m >> 4, m2 = m & 15;
      sincospi(-2.0 * ((k1 * m2) % 128) / 128.0, &sn, &cs);
      sm.tw128[m] = float2{(float)cs, (float)sn};
    } else if (m < 384) {
      const int j = m - 128, k1 = j >> 4, n2 = j & 15;
      sincospi(-2.0 * ((k1 * n2) % 256) / 256.0, &sn, &cs);
      sm.tw256[j] = float2{(float)cs, (float)sn};
    } else {
      const int k = m - 384;
      sincospi(-2.0 * k / 256.0, &sn, &cs);
      sm.wk[k] = float2{(float)cs, (float)sn};
    }
  }
}

// row of B that holds the y transform's output index k (k1 + 16 k2 at 16 k1 + k2)
__device__ __forceinline__ int yrow(int k) { return 16 * (k & 15) + (k >> 4); }

// ------------------------------------------------------------------ forward
template <int CL>
__global__ void __launch_bounds__(YzCfg<CL>::kThreads, YzCfg<CL>::kMinBlocks)
    k_yz_forward(const float* __restrict__ rho, float2* __restrict__ spec, int nplanes, int qp) {
  using C = YzCfg<CL>;
  constexpr int LDB = C::kLDB;
  extern __shared__ __align__(128) unsigned char yz_raw[];
  YzSmem<CL>& sm = *reinterpret_cast<YzSmem<CL>*>(yz_raw + ((128u - (smem_u32(yz_raw) & 127u)) & 127u));
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int q = (int)cluster_rank();
  const int cid = blockIdx.x / CL, ncl = gridDim.x / CL;
  const int nmine = cid < nplanes ? (nplanes - cid + ncl - 1) / ncl : 0;
  const int nchunks = 4 * nmine;
  if (tid == 0) {
    mbar_init(&sm.full[0], 1);
    mbar_init(&sm.full[1], 1);
    sm.fail = 0;
    mbar_fence_init();
  }
  yz_tables<CL>(sm);
  __syncthreads();
  cluster_sync_all();   // every CTA of the cluster has started: its shared memory may be written
  auto chunk_src = [&](int j) {
    const int plane = cid + (j >> 2) * ncl;
    return rho + ((size_t)plane * kYzN + C::kRows * q + C::kChunk * (j & 3)) * kYzN;
  };
  constexpr uint32_t kChunkBytes = C::kChunk * kYzN * 4;
  if (tid == 0) {
    for (int j = 0; j < 2 && j < nchunks; ++j) {
      mbar_arrive_expect_tx(&sm.full[j], kChunkBytes);
      bulk_load(sm.ring[j], chunk_src(j), kChunkBytes, &sm.full[j]);
    }
  }
  uint32_t bq[CL];
#pragma unroll
  for (int r = 0; r < CL; ++r) bq[r] = map_rank(smem_u32(sm.B), (uint32_t)r);
  const int g = warp / (C::kWarps / 2), wq = warp % (C::kWarps / 2);   // chunk group, warp within it
  // z-stage lane roles after the 128-point FFT: row r2 of the warp's four, k1; the lane holding
  // Z[128 - k] for this lane's Z[k] (k1 = 0 and 4 pair within the lane)
  const int r2 = lane >> 3, k1 = lane & 7;
  const int partner = (lane & ~7) | ((8 - k1) & 7);
  constexpr uint32_t kShare = (uint32_t)(C::kRows * kYzN * 4);   // this CTA's rows of a plane
  for (int i = 0; i < nmine; ++i) {
    const int plane = cid + i * ncl;
    // the next plane's rows into L2 while this one is transformed (its first chunks follow by
    // bulk copy as soon as this plane's last ones are consumed)
    if (tid == 0 && i + 1 < nmine)
      prefetch_l2(rho + ((size_t)(plane + ncl) * kYzN + C::kRows * q) * kYzN, kShare);
    // ---- z transforms of this CTA's rows, scattered to the column owners
    for (int sub = g; sub < 4; sub += 2) {
      const int j = 4 * i + sub, s = j & 1;
      bool ok = !*(volatile int*)&sm.fail;
      if (ok && !mbar_wait(&sm.full[s], (uint32_t)(j >> 1) & 1u)) {
        sm.fail = 1;
        ok = false;
      }
      if (ok) {
        float re[16], im[16];
        fft128_rows<-1>(sm.ring[s] + wq * 4 * 128, sm.tw128, lane, re, im);
        const uint32_t yoff = (uint32_t)((C::kRows * q + C::kChunk * sub + 4 * wq + r2) * LDB);
#pragma unroll
        for (int k2 = 0; k2 < 16; ++k2) {
          // Z[128 - k], k = k1 + 8 k2: the partner's value 15 - k2, or this lane's (16 - k2) mod 16
          const float pr = __shfl_sync(0xffffffffu, re[15 - k2], partner);
          const float pi = __shfl_sync(0xffffffffu, im[15 - k2], partner);
          const float cx = k1 == 0 ? re[(16 - k2) & 15] : pr;
          const float cy = k1 == 0 ? im[(16 - k2) & 15] : pi;
          const float ax = re[k2], ay = im[k2];
          const int k = k1 + 8 * k2;
          if (k == 0) {   // X[0] and X[128], both real: the packed column 0 of rank 0
            st_cluster(bq[0] + yoff * 8u, float2{ax + ay, ax - ay});
            continue;
          }
          // X[k] = ((a + b) - i W^k (a - b)) / 2 with b = conj(c)
          const float2 w = sm.wk[k];
          const float sx = ax + cx, sy = ay - cy, dx = ax - cx, dy = ay + cy;
          const float2 X{0.5f * (sx + w.x * dy + w.y * dx), 0.5f * (sy - w.x * dx + w.y * dy)};
          // owner rank of kz = k: k >> log2(cols) (the same for every lane at this k2)
          const int rk = (8 * k2) >> C::kLogCols;
          st_cluster(bq[rk] + (yoff + (uint32_t)(k & (C::kCols - 1))) * 8u, X);
        }
      }
      group_bar(g, C::kGroupThreads);   // the group is done with the chunk buffer: load chunk j + 2
      if ((tid % C::kGroupThreads) == 0 && j + 2 < nchunks && !*(volatile int*)&sm.fail) {
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(&sm.full[s], kChunkBytes);
        bulk_load(sm.ring[s], chunk_src(j + 2), kChunkBytes, &sm.full[s]);
      }
    }
    cluster_sync_all();   // every X of the plane is in its owner's columns
    // ---- y transforms of this CTA's columns (two items per thread per pass)
    for (int it = tid; it < C::kCols * 16; it += C::kThreads) {
      const int n2 = it >> C::kLogCols, col = it & (C::kCols - 1);
      float re[16], im[16];
#pragma unroll
      for (int n1 = 0; n1 < 16; ++n1) {
        const float2 v = sm.B[(16 * n1 + n2) * LDB + col];
        re[n1] = v.x;
        im[n1] = v.y;
      }
      ypass1_store<-1, LDB>(re, im, n2, col, sm.B, sm.tw256);
    }
    __syncthreads();
    const bool bad = *(volatile int*)&sm.fail;
    const float nanf_ = __int_as_float(0x7fc00000);
    float2* out = spec + (size_t)plane * kYzN * qp;   // qp = 129, or 130 with a zero pad slot
    for (int it = tid; it < C::kCols * 16; it += C::kThreads) {
      const int kk1 = it >> C::kLogCols, col = it & (C::kCols - 1);
      float re[16], im[16];
      ypass2_load<-1, LDB>(re, im, kk1, col, sm.B);
      if (q == 0 && col == 0) {   // the packed column: split below, once every ky is known
#pragma unroll
        for (int k2 = 0; k2 < 16; ++k2) sm.B[(16 * kk1 + k2) * LDB] = float2{re[k2], im[k2]};
      } else {
        const int kz = q * C::kCols + col;
#pragma unroll
        for (int k2 = 0; k2 < 16; ++k2)
          out[(size_t)(kk1 + 16 * k2) * qp + kz] = bad ? float2{nanf_, 0.f} : float2{re[k2], im[k2]};
      }
    }
    if (q == 0) {
      __syncthreads();
      // C = Y0 + i Y128 with Y0, Y128 the transforms of real columns:
      // Y0[ky] = (C[ky] + C*[-ky]) / 2, Y128[ky] = (C[ky] - C*[-ky]) / (2 i)
      for (int ky = tid; ky < kYzN; ky += C::kThreads) {
        const float2 c = sm.B[yrow(ky) * LDB], cm = sm.B[yrow((kYzN - ky) & (kYzN - 1)) * LDB];
        const float2 y0{0.5f * (c.x + cm.x), 0.5f * (c.y - cm.y)};
        const float2 y128{0.5f * (c.y + cm.y), 0.5f * (cm.x - c.x)};
        out[(size_t)ky * qp] = bad ? float2{nanf_, 0.f} : y0;
        out[(size_t)ky * qp + 128] = bad ? float2{nanf_, 0.f} : y128;
        if (qp > kYzH) out[(size_t)ky * qp + kYzH] = float2{0.f, 0.f};
      }
    }
    cluster_sync_exec();   // every CTA has read its columns: the next plane may scatter
  }
  cluster_sync_all();
}

// ------------------------------------------------------------------ inverse
template <int CL>
__global__ void __launch_bounds__(YzCfg<CL>::kThreads, YzCfg<CL>::kMinBlocks)
    k_yz_inverse(const float2* __restrict__ spec, float* __restrict__ rho, int nplanes) {
  using C = YzCfg<CL>;
  constexpr int LDB = C::kLDB;
  extern __shared__ __align__(128) unsigned char yz_raw[];
  YzSmem<CL>& sm = *reinterpret_cast<YzSmem<CL>*>(yz_raw + ((128u - (smem_u32(yz_raw) & 127u)) & 127u));
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int q = (int)cluster_rank();
  const int cid = blockIdx.x / CL, ncl = gridDim.x / CL;
  const int nmine = cid < nplanes ? (nplanes - cid + ncl - 1) / ncl : 0;
  yz_tables<CL>(sm);
  __syncthreads();
  cluster_sync_all();
  const uint32_t b_local = smem_u32(sm.B);
  float2* wbuf = &sm.ring[0][0] + warp * 4 * 128;   // this warp's four row buffers
  // cluster address of column kz's value in row slot yr (kz = 1..127; kz = 0 / 128: packed column 0)
  auto xaddr = [&](int kz, uint32_t yr) {
    return map_rank(b_local, (uint32_t)(kz >> C::kLogCols)) + (yr + (uint32_t)(kz & (C::kCols - 1))) * 8u;
  };
  // each CTA's share of a plane's spectrum (a multiple of 16 bytes: 256 129 8 / CL)
  constexpr uint32_t kShare = (uint32_t)(kYzN * kYzH * 8 / CL);
  if (tid == 0 && nmine > 0)
    prefetch_l2(reinterpret_cast<const char*>(spec + (size_t)cid * kYzN * kYzH) + q * kShare, kShare);
  for (int i = 0; i < nmine; ++i) {
    const int plane = cid + i * ncl;
    // the next plane's spectrum into L2 while this one is transformed
    if (tid == 0 && i + 1 < nmine)
      prefetch_l2(reinterpret_cast<const char*>(spec + (size_t)(plane + ncl) * kYzN * kYzH) + q * kShare, kShare);
    // ---- inverse y transforms of this CTA's columns, pass 1 straight from the spectrum
    const float2* in = spec + (size_t)plane * kYzN * kYzH;
    for (int it = tid; it < C::kCols * 16; it += C::kThreads) {
      const int n2 = it >> C::kLogCols, col = it & (C::kCols - 1);
      const bool packed = q == 0 && col == 0;
      const int kz = q * C::kCols + col;
      float re[16], im[16];
#pragma unroll
      for (int n1 = 0; n1 < 16; ++n1) {
        const float2* rowp = in + (size_t)(16 * n1 + n2) * kYzH;
        const float2 v = rowp[kz];
        if (packed) {   // H[ky][0] + i H[ky][128]: one transform gives both real columns
          const float2 h = rowp[128];
          re[n1] = v.x - h.y;
          im[n1] = v.y + h.x;
        } else {
          re[n1] = v.x;
          im[n1] = v.y;
        }
      }
      ypass1_store<1, LDB>(re, im, n2, col, sm.B, sm.tw256);
    }
    __syncthreads();
    for (int it = tid; it < C::kCols * 16; it += C::kThreads) {
      const int kk1 = it >> C::kLogCols, col = it & (C::kCols - 1);
      float re[16], im[16];
      ypass2_load<1, LDB>(re, im, kk1, col, sm.B);
#pragma unroll
      for (int k2 = 0; k2 < 16; ++k2) sm.B[(16 * kk1 + k2) * LDB + col] = float2{re[k2], im[k2]};
    }
    cluster_sync_all();   // every CTA's columns transformed: rows may be read across the cluster
    // ---- per row y: half-complex -> complex packing, inverse 128-point FFT, real row out
    for (int round = 0; round < 2; ++round) {
      const int ybase = C::kRows * q + (C::kRows / 2) * round + 4 * warp;
#pragma unroll
      for (int it = lane; it < 4 * 64; it += 32) {
        const int r = it >> 6, k = it & 63;
        const uint32_t yr = (uint32_t)(yrow(ybase + r) * LDB);
        float2* row = wbuf + r * 128;
        // a = X[k] (X[0] is the real part of the packed column 0), c = X[128 - k] (X[128] is the
        // packed column's imaginary part)
        const float2 p0 = ld_cluster(xaddr(k, yr));
        float2 a, c;
        if (k == 0) {
          a = float2{p0.x, 0.f};
          c = float2{p0.y, 0.f};
        } else {
          a = p0;
          c = ld_cluster(xaddr(128 - k, yr));
        }
        // Z[k] = (a + b) + i conj(W^k) (a - b), b = conj(c)
        {
          const float2 w = sm.wk[k];
          const float sx = a.x + c.x, sy = a.y - c.y, dx = a.x - c.x, dy = a.y + c.y;
          row[k] = float2{sx - w.x * dy + w.y * dx, sy + w.x * dx + w.y * dy};
        }
        if (k == 0) {   // Z[64] from X[64] alone
          const float2 x = ld_cluster(xaddr(64, yr));
          const float2 w = sm.wk[64];
          const float dy = 2.f * x.y;
          row[64] = float2{2.f * x.x - w.x * dy, w.y * dy};
        } else {        // Z[128 - k] from a' = c, b' = conj(a)
          const float2 w = sm.wk[128 - k];
          const float sx = c.x + a.x, sy = c.y - a.y, dx = c.x - a.x, dy = c.y + a.y;
          row[128 - k] = float2{sx - w.x * dy + w.y * dx, sy + w.x * dx + w.y * dy};
        }
      }
      __syncwarp();
      float re[16], im[16];
      fft128_rows<1>(wbuf, sm.tw128, lane, re, im);
      // z[k1 + 8 k2] = (x[2m], x[2m+1]) at m = k1 + 8 k2 of row r2
      const int r2 = lane >> 3, k1 = lane & 7;
      float2* dst = reinterpret_cast<float2*>(rho + ((size_t)plane * kYzN + ybase + r2) * kYzN);
#pragma unroll
      for (int k2 = 0; k2 < 16; ++k2) dst[k1 + 8 * k2] = float2{re[k2], im[k2]};
      __syncwarp();   // the row buffers are rewritten in the next iteration
    }
    cluster_sync_exec();   // every CTA has read the cluster's columns: the next plane may load
  }
  cluster_sync_all();
}

// ------------------------------------------------------------------ inverse, TMA-fed (16-byte rows)
// The inverse on CTA pairs for a half spectrum whose ky rows carry a pad slot (130 values, 1,040
// bytes): each CTA's 64 columns of a plane arrive by one 2-D TMA load (rank 0 also loads the
// kz = 128 column), instead of 8-byte loads whose latency the y pass waits on.
struct YzInvT {
  static constexpr int kThreads = 512;
  static constexpr int kCols = 64;
  static constexpr int kLDB = 64;   // the TMA box lands dense
  static constexpr int kRows = 128;
};
struct YzInvTSmem {
  float2 B[kYzN * YzInvT::kLDB];      // the CTA's columns, rows in ky, then the y transform in place
  float4 h128[kYzN];                  // rank 0: (H[ky][128], pad) per ky
  float2 ring[2][32 * 128];           // 16 warps x 4 row buffers of the z stage
  float2 tw128[8 * 16];
  float2 tw256[16 * 16];
  float2 wk[kYzH + 1];
  uint64_t full;
  int fail;
};

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int c0, int c1, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(
          smem_u32(dst)),
      "l"(map), "r"(c0), "r"(c1), "r"(smem_u32(bar))
      : "memory");
}

__global__ void __launch_bounds__(YzInvT::kThreads, 1)
    k_yz_inverse_tma(const __grid_constant__ CUtensorMap tcols, const __grid_constant__ CUtensorMap tnyq,
                     const float2* __restrict__ spec, float* __restrict__ rho, int nplanes) {
  constexpr int CL = 2, LDB = YzInvT::kLDB, QP = kYzH + 1;
  extern __shared__ __align__(128) unsigned char yz_raw[];
  YzInvTSmem& sm = *reinterpret_cast<YzInvTSmem*>(yz_raw + ((128u - (smem_u32(yz_raw) & 127u)) & 127u));
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int q = (int)cluster_rank();
  const int cid = blockIdx.x / CL, ncl = gridDim.x / CL;
  const int nmine = cid < nplanes ? (nplanes - cid + ncl - 1) / ncl : 0;
  if (tid == 0) {
    mbar_init(&sm.full, 1);
    sm.fail = 0;
    mbar_fence_init();
  }
  for (int m = tid; m < 128 + 256 + kYzH; m += blockDim.x) {
    double sn, cs;
    if (m < 128) {
      sincospi(-2.0 * (((m >> 4) * (m & 15)) % 128) / 128.0, &sn, &cs);
      sm.tw128[m] = float2{(float)cs, (float)sn};
    } else if (m < 384) {
      const int j = m - 128;
      sincospi(-2.0 * (((j >> 4) * (j & 15)) % 256) / 256.0, &sn, &cs);
      sm.tw256[j] = float2{(float)cs, (float)sn};
    } else {
      sincospi(-2.0 * (m - 384) / 256.0, &sn, &cs);
      sm.wk[m - 384] = float2{(float)cs, (float)sn};
    }
  }
  __syncthreads();
  cluster_sync_all();
  const uint32_t b_local = smem_u32(sm.B);
  float2* wbuf = &sm.ring[0][0] + warp * 4 * 128;
  constexpr uint32_t kShare = (uint32_t)(kYzN * QP * 8 / CL);   // this CTA's half of a plane's rows
  constexpr uint32_t kColBytes = kYzN * YzInvT::kCols * 8;
  constexpr uint32_t kNyqBytes = kYzN * 16;
  if (tid == 0 && nmine > 0)
    prefetch_l2(reinterpret_cast<const char*>(spec + (size_t)cid * kYzN * QP) + q * kShare, kShare);
  const float nanf_ = __int_as_float(0x7fc00000);
  for (int i = 0; i < nmine; ++i) {
    const int plane = cid + i * ncl;
    if (tid == 0) {
      if (i + 1 < nmine)
        prefetch_l2(reinterpret_cast<const char*>(spec + (size_t)(plane + ncl) * kYzN * QP) + q * kShare, kShare);
      if (!sm.fail) {
        fence_proxy_async_smem();   // the previous plane's reads of B are done (cluster barrier)
        mbar_arrive_expect_tx(&sm.full, q == 0 ? kColBytes + kNyqBytes : kColBytes);
        tma_load_2d(sm.B, &tcols, 128 * q, plane * kYzN, &sm.full);
        if (q == 0) tma_load_2d(sm.h128, &tnyq, 256, plane * kYzN, &sm.full);
      }
    }
    if (!*(volatile int*)&sm.fail && !mbar_wait(&sm.full, (uint32_t)i & 1u)) sm.fail = 1;
    __syncthreads();
    const bool bad = *(volatile int*)&sm.fail;
    // ---- inverse y transforms of this CTA's 64 columns
    for (int it = tid; it < YzInvT::kCols * 16; it += YzInvT::kThreads) {
      const int n2 = it >> 6, col = it & 63;
      const bool packed = q == 0 && col == 0;
      float re[16], im[16];
#pragma unroll
      for (int n1 = 0; n1 < 16; ++n1) {
        const int ky = 16 * n1 + n2;
        float2 v = sm.B[ky * LDB + col];
        if (packed) {   // H[ky][0] + i H[ky][128]: one transform gives both real columns
          const float4 h = sm.h128[ky];
          v = float2{v.x - h.y, v.y + h.x};
        }
        re[n1] = v.x;
        im[n1] = v.y;
      }
      ypass1_store<1, LDB>(re, im, n2, col, sm.B, sm.tw256);
    }
    __syncthreads();
    for (int it = tid; it < YzInvT::kCols * 16; it += YzInvT::kThreads) {
      const int kk1 = it >> 6, col = it & 63;
      float re[16], im[16];
      ypass2_load<1, LDB>(re, im, kk1, col, sm.B);
#pragma unroll
      for (int k2 = 0; k2 < 16; ++k2) sm.B[(16 * kk1 + k2) * LDB + col] = float2{re[k2], im[k2]};
    }
    cluster_sync_all();   // both CTAs' columns transformed: rows may be read across the pair
    // ---- per row y: half-complex -> complex packing, inverse 128-point FFT, real row out.
    // Lane item j (0..7) of a round is row j / 2, k = lane + 32 (j % 2); its two cross-CTA reads
    // are X[k] and X[128 - k] (X[64] for k = 0): all 16 are issued before any is used.
    const uint32_t bq0 = map_rank(b_local, 0u), bq1 = map_rank(b_local, 1u);
    for (int round = 0; round < 2; ++round) {
      const int ybase = YzInvT::kRows * q + 64 * round + 4 * warp;
      float2 va[8], vc[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int k = lane + 32 * (j & 1);   // 0..63: rank 0's columns
        const uint32_t yr = (uint32_t)(yrow(ybase + (j >> 1)) * LDB);
        const int k2 = k == 0 ? 64 : 128 - k;   // 64..128 -> rank 1 (X[128]: the packed column's imaginary part)
        va[j] = ld_cluster(bq0 + (yr + (uint32_t)k) * 8u);
        vc[j] = ld_cluster(bq1 + (yr + (uint32_t)(k2 & 63)) * 8u);
      }
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int k = lane + 32 * (j & 1);
        float2* row = wbuf + (j >> 1) * 128;
        const float2 p0 = va[j];
        float2 a, c;
        if (k == 0) {
          a = float2{p0.x, 0.f};
          c = float2{p0.y, 0.f};
        } else {
          a = p0;
          c = vc[j];
        }
        {
          const float2 w = sm.wk[k];
          const float sx = a.x + c.x, sy = a.y - c.y, dx = a.x - c.x, dy = a.y + c.y;
          row[k] = float2{sx - w.x * dy + w.y * dx, sy + w.x * dx + w.y * dy};
        }
        if (k == 0) {   // Z[64] from X[64] alone
          const float2 x = vc[j];
          const float2 w = sm.wk[64];
          const float dy = 2.f * x.y;
          row[64] = float2{2.f * x.x - w.x * dy, w.y * dy};
        } else {
          const float2 w = sm.wk[128 - k];
          const float sx = c.x + a.x, sy = c.y - a.y, dx = c.x - a.x, dy = c.y + a.y;
          row[128 - k] = float2{sx - w.x * dy + w.y * dx, sy + w.x * dx + w.y * dy};
        }
      }
      __syncwarp();
      float re[16], im[16];
      fft128_rows<1>(wbuf, sm.tw128, lane, re, im);
      const int r2 = lane >> 3, k1 = lane & 7;
      float2* dst = reinterpret_cast<float2*>(rho + ((size_t)plane * kYzN + ybase + r2) * kYzN);
#pragma unroll
      for (int k2 = 0; k2 < 16; ++k2) dst[k1 + 8 * k2] = bad ? float2{nanf_, nanf_} : float2{re[k2], im[k2]};
      __syncwarp();
    }
    cluster_sync_exec();   // both CTAs have read the pair's columns: the next plane may load
  }
  cluster_sync_all();
}

template <int CL>
int launch_yz(const void* kern, int which, int threads, size_t smem, void** args, int nplanes, cudaStream_t s,
              const char* what) {
  static unsigned attr_set[3] = {0, 0, 0};   // per kernel, one bit per device (set every call past 32)
  int dev = 0;
  cudaGetDevice(&dev);
  const unsigned bit = dev < 32 ? 1u << dev : 0u;
  if (!bit || !(attr_set[which] & bit)) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
      set_error(what, "could not raise the shared-memory limit of the (y, z) transform");
      return FD3_ECUDA;
    }
    attr_set[which] |= bit;
  }
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = CL;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  // persistent: as many clusters as can be resident at once (a cluster that waited for free SMs
  // would run its share of planes after everything else)
  cfg.gridDim = dim3(CL);
  int nclusters = 0;
  if (cudaOccupancyMaxActiveClusters(&nclusters, kern, &cfg) != cudaSuccess || nclusters < 1) {
    set_error(what, "no group of SMs can hold the (y, z) transform's clusters");
    return FD3_ECUDA;
  }
  if (nclusters > nplanes) nclusters = nplanes;
  cfg.gridDim = dim3(CL * nclusters);
  if (cudaLaunchKernelExC(&cfg, kern, args) != cudaSuccess) {
    set_error(what, "launch of the (y, z) transform failed");
    return FD3_ECUDA;
  }
  count_launch();
  return FD3_OK;
}

}  // namespace

bool yzfft_applies(const MeshGeom& mg) { return mg.n[1] == kYzN && mg.n[2] == kYzN; }

// variant: 1 = clusters of 2 CTAs (one per SM), 2 = clusters of 4 (two per SM) for the forward
// transform; the inverse always runs on pairs
int launch_yz_forward(const MeshGeom& mg, int nchannels, int variant, const float* rho, void* spec,
                      cudaStream_t s) {
  if (!yzfft_applies(mg) || nchannels < 1 || (variant != 1 && variant != 2)) return FD3_EINVAL;
  const long long np = (long long)nchannels * mg.n[0];
  if (np > (1LL << 30)) return FD3_EINVAL;
  const float* in = rho;
  float2* out = reinterpret_cast<float2*>(spec);
  int n = (int)np;
  int qp = mg.qpitch > 0 ? mg.qpitch : kYzH;
  if (qp != kYzH && qp != kYzH + 1) return FD3_EINVAL;
  void* args[4] = {&in, &out, &n, &qp};
  if (variant == 1)
    return launch_yz<2>(reinterpret_cast<const void*>(k_yz_forward<2>), 0, YzCfg<2>::kThreads,
                        sizeof(YzSmem<2>) + 128, args, n, s, "fft_r2c");
  return launch_yz<4>(reinterpret_cast<const void*>(k_yz_forward<4>), 0, YzCfg<4>::kThreads, sizeof(YzSmem<4>) + 128,
                      args, n, s, "fft_r2c");
}

int launch_yz_inverse(const MeshGeom& mg, int nchannels, int variant, const void* spec, float* rho,
                      cudaStream_t s) {
  if (!yzfft_applies(mg) || nchannels < 1 || (variant != 1 && variant != 2)) return FD3_EINVAL;
  (void)variant;   // the inverse runs on pairs for both variants (quads measured slower)
  const long long np = (long long)nchannels * mg.n[0];
  if (np > (1LL << 30) / kYzN) return FD3_EINVAL;
  const int qp = mg.qpitch > 0 ? mg.qpitch : kYzH;
  const float2* in = reinterpret_cast<const float2*>(spec);
  float* out = rho;
  int n = (int)np;
  if (qp == kYzH) {
    void* args[3] = {&in, &out, &n};
    return launch_yz<2>(reinterpret_cast<const void*>(k_yz_inverse<2>), 1, YzCfg<2>::kThreads,
                        sizeof(YzSmem<2>) + 128, args, n, s, "fft_c2r");
  }
  if (qp != kYzH + 1) return FD3_EINVAL;
  // 16-byte spectrum rows: the columns come by TMA (a 2-D map over (floats of a row, rows))
  auto fn = tensor_map_encoder();
  if (!fn) {
    set_error("fft_c2r", "cuTensorMapEncodeTiled is not available from the driver");
    return FD3_ECUDA;
  }
  const cuuint64_t dims[2] = {(cuuint64_t)(2 * qp), (cuuint64_t)np * kYzN};
  const cuuint64_t strides[1] = {(cuuint64_t)(2 * qp) * 4};
  const cuuint32_t estr[2] = {1, 1};
  const cuuint32_t box_cols[2] = {2 * YzInvT::kCols, kYzN};
  const cuuint32_t box_nyq[2] = {4, kYzN};
  CUtensorMap tcols, tnyq;
  for (int m = 0; m < 2; ++m) {
    const CUresult r = fn(m == 0 ? &tcols : &tnyq, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void*>(spec), dims,
                          strides, m == 0 ? box_cols : box_nyq, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
      set_error("fft_c2r", "cuTensorMapEncodeTiled rejected the spectrum's tensor map");
      return FD3_ECUDA;
    }
  }
  void* args[5] = {&tcols, &tnyq, &in, &out, &n};
  return launch_yz<2>(reinterpret_cast<const void*>(k_yz_inverse_tma), 2, YzInvT::kThreads, sizeof(YzInvTSmem) + 128,
                      args, n, s, "fft_c2r");
}

}  // namespace fd3

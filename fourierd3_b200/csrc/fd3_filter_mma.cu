// Many-species reciprocal-space filter on the 5th-generation tensor cores (tcgen05, sm_100a),
// mixed precision (float spectrum, float32 accumulation of each product).
//
// At every k-point the filter is a small dense product (src/fourierd3/kspace_filter_d3.py:53-68,
// the per-rank S x S bmm of kspace_filter_d3.py:64):
//     H[X, r]  = sum_Y Gh_XY(k) S[Y, r]      (written back over the spectrum)
//     D[X, r]  = sum_Y dG_XY(k) S[Y, r]      (for the virial)
// with a different S x S matrix at every k. One CTA per SM takes tiles of kFmKT consecutive
// k-points; for each k-point it builds the operands in shared memory and one thread issues
// 16 tcgen05.mma.kind::tf32 instructions (M = 128, N = 32, K = 8 each) into TMEM.
//
// tf32 split. Every float operand value a is written as a tf32 pair (ah, al), ah = a rounded to
// tf32, al = (a - ah) rounded to tf32 (a - ah is exact in float). The K dimension interleaves them, k = 2 Y + {0: high, 1: low}:
//     A[m][2Y] = Ah[m][Y],  A[m][2Y+1] = Al[m][Y]          (m: 0-63 Gh rows, 64-127 dG rows)
//     B[n][2Y] = Bh[n][Y],  B[n][2Y+1] = Bh[n][Y]          (n: 0-15, 8 ranks x re/im)
//     B[16+n][2Y] = Bl[n][Y], B[16+n][2Y+1] = 0
// so that one product over K = 2 x 64 gives, in accumulator columns 0-15, Ah Bh + Al Bh and, in
// columns 16-31, Ah Bl: their sum is A B up to the dropped Al Bl term (~2^-22 relative; products
// of tf32 values are exact in the float32 accumulator). Each pair's high and low parts are
// neighbours, so one 8-byte shared store writes both.
//
// Pipeline: operands are double-buffered (stage s = k-point parity), so building the operands of
// k-point j (CUDA cores: Green-table lookups, window, Hermitian average, tf32 split) overlaps the
// MMAs of k-point j-1, whose accumulators the epilogue reads back (tcgen05.ld) after an mbarrier
// signalled by tcgen05.commit. The epilogue writes H over the staged spectrum tile and adds the
// k-point's energy sum_r lambda_r Re(S^* H) and virial sum_r lambda_r Re(S^* D) k k^T / |k| to
// float64 per-thread accumulators. The next tile's spectrum is prefetched with cp.async while
// the current one is filtered. The species pairs a warp evaluates, and their shared-memory
// offsets, are fixed for the whole launch and kept in registers.
//
// On the self-conjugate planes the energy is formed with the Hermitian-averaged Gh instead of G:
// each such k-point and its stored partner k' carry S(k') = conj S(k) and the same weight, so
// S^H Gh S summed over the pair equals S^H G(k) S + S^H G(k') S; the total is unchanged.
//
// Shared-memory operand layout: K-major, no swizzle (the UMMA "interleaved" canonical form):
// 8-row x 16-byte core matrices, element (m, k) at (m / 8) 4096 + (k / 4) 128 + (m % 8) 16 +
// (k % 4) 4 bytes; leading-dimension byte offset 128 (the next 4 k), stride byte offset 4096
// (the next 8 rows); each K-step of 8 advances the start address by 256 bytes.
#include "fd3_async.cuh"
#include "fd3_filter.cuh"

namespace fd3 {

constexpr int kFmWarps = 12;
constexpr int kFmThreads = 32 * kFmWarps;   // all build operands; warps 0-3 read TMEM
constexpr int kFmKT = 4;                    // k-points per spectrum tile
constexpr int kFmMaxS = 64;                 // species (zero padded)
constexpr int kFmK = 2 * kFmMaxS;           // K of the product: species x (high, low)
constexpr int kFmN = 32;                    // 8 ranks x (re, im) x (high B, low B)
constexpr int kFmSBO = (kFmK / 4) * 128;    // bytes between 8-row groups: 4096
constexpr int kFmABytes = 128 * kFmK * 4;   // one A operand: 64 KB
constexpr int kFmBBytes = kFmN * kFmK * 4;  // one B operand: 16 KB
constexpr int kFmDgOff = 8 * kFmSBO;        // dG rows start at row 64
constexpr int kFmTmemCols = 64;             // two 32-column accumulators
constexpr int kFmMaxBlk = 6;                // 8 x 4 pair blocks per warp (72 blocks for 64 species)
constexpr int kFmMaxBBlk = 3;               // 8 x 4 B blocks per warp (32 blocks for 64 species)

// spectrum tile: channel (X, r) row of kFmKT complex values; rank stride CS, species stride XS
// padded so that consecutive species (epilogue lanes) and channels fall on different banks
constexpr int kFmCS = kFmKT + 1;
__host__ __device__ inline int fm_xs(int R) {
  const int base = R * kFmCS;
  return base + ((17 - base % 16) % 16);   // XS = 1 (mod 16) complex values
}
__host__ __device__ inline size_t fm_tile_bytes(int S, int R) { return (size_t)S * fm_xs(R) * sizeof(float2); }

struct FmGeo {         // per k-point of the current tile
  float inv_sc, dscale, wk, knorm, kv0, kv1, kv2;
  int tj, pj, partner, valid;
  HermiteF hb, pb;
};

__host__ __device__ inline int fm_upper_blocks(int S) {
  const int nbx = (S + 7) >> 3, nby = (S + 3) >> 2;
  int n = 0;
  for (int bx = 0; bx < nbx; ++bx) n += nby - 2 * bx > 0 ? nby - 2 * bx : 0;
  return n;
}

__host__ __device__ inline size_t fm_smem_bytes(int S, int R) {
  size_t b = 2 * (size_t)kFmABytes + 2 * (size_t)kFmBBytes;   // A, B: 2 stages
  b += 2 * ((fm_tile_bytes(S, R) + 127) & ~(size_t)127);      // two spectrum tiles
  b += kFmKT * sizeof(FmGeo);
  return b + 1024;                                             // alignment
}

// tf32 value of x rounded to nearest (ties away from zero) by integer arithmetic on the bits: the
// tensor core reads the top 19 bits of each 32-bit operand. Integer ops keep the conversion off
// the (quarter-rate) conversion pipe, which the operand build would otherwise saturate.
__device__ __forceinline__ uint32_t tf32_round(float x) { return (__float_as_uint(x) + 0x1000u) & 0xFFFFE000u; }
__host__ __device__ __forceinline__ uint32_t op_off(int m, int k) {
  return (uint32_t)((m >> 3) * kFmSBO + (k >> 2) * 128 + (m & 7) * 16 + (k & 3) * 4);
}
// UMMA shared-memory descriptor: start >> 4 in [0,14), leading byte offset >> 4 in [16,30),
// stride byte offset >> 4 in [32,46), descriptor version 1 in [46,48), no swizzle.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// Instruction descriptor, kind::tf32: float32 accumulator (bit 4), A and B tf32 (2 at bits 7
// and 10), both K-major, N / 8 at bit 17, M / 16 at bit 24.
constexpr uint32_t kFmIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kFmN >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t ad, uint64_t bd, uint32_t accumulate) {
  const uint32_t mask0 = 0, mask1 = 0, mask2 = 0, mask3 = 0;
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(d_tmem),
      "l"(ad), "l"(bd), "r"(kFmIdesc), "r"(accumulate), "r"(mask0), "r"(mask1), "r"(mask2), "r"(mask3)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
// 32 consecutive accumulator columns of this warp's 32 TMEM lanes
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}
// No compiler memory clobber: table loads of later pairs may be hoisted above these stores; the
// operand buffer is ordered by the proxy fence and the barrier (both clobber memory) before the
// MMA reads it.
__device__ __forceinline__ void st_shared_v2(uint32_t addr, uint32_t a, uint32_t b) {
  asm volatile("st.shared.v2.b32 [%0], {%1, %2};\n" ::"r"(addr), "r"(a), "r"(b));
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
__device__ __forceinline__ void epi_bar() { asm volatile("bar.sync 2, 128;\n" ::: "memory"); }

// Stage one tile's spectrum values (C channels x kFmKT k-points) with 8-byte cp.async copies;
// k-points past the end of the mesh are zero.
__device__ __forceinline__ void fm_prefetch(float2* tile, const float2* __restrict__ spec, size_t Mh, size_t k0,
                                            int S, int R, int XS) {
  const int C = S * R;
  const uint32_t invR = (65536u + (uint32_t)R - 1u) / (uint32_t)R;   // c / R = (c invR) >> 16 for c < 4096
  for (int e = threadIdx.x; e < C * kFmKT; e += kFmThreads) {
    const int c = e / kFmKT, j = e - c * kFmKT;
    const int X = (int)(((uint32_t)c * invR) >> 16), r = c - X * R;
    float2* d = tile + X * XS + r * kFmCS + j;
    const size_t k = k0 + j;
    if (k < Mh)
      cp_async8(d, spec + (size_t)c * Mh + k);
    else
      *d = make_float2(0.f, 0.f);
  }
  cp_async_commit();
}

// The epilogue of k-point j in stage st: wait (bounded) for its MMAs, read the accumulators
// back (warps 0-3, one TMEM lane quarter each), write H over the tile and add the energy and
// virial terms to acc. Every thread waits, so the stage's operands are free again afterwards.
// Returns false if the wait ran out.
__device__ __forceinline__ bool fm_epilogue(int st, int j, float2* tile, uint64_t* bar, uint32_t parity,
                                            uint32_t tmem, int warp, int lane, int S, int R, int XS,
                                            const float* s_lam, const FmGeo* geo, double (&acc)[7]) {
  const bool ok = mbar_wait(bar, parity);
  tc_fence_after();
  if (warp < 4) {
    float d[32];
    tmem_ld32(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(st * kFmN), d);
    const int X = (warp < 2 ? 32 * warp : 32 * (warp - 2)) + lane;
    float2 sv[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) sv[r] = (X < S && r < R) ? tile[X * XS + r * kFmCS + j] : make_float2(0.f, 0.f);
    epi_bar();   // every epilogue lane has read S before rows X are overwritten with H
    float h[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) h[c] = d[c] + d[16 + c];
    float q = 0.f;
#pragma unroll
    for (int r = 0; r < 8; ++r) q += s_lam[r] * (sv[r].x * h[2 * r] + sv[r].y * h[2 * r + 1]);
    const FmGeo& ge = geo[j];
    if (X < S && ge.valid) {
      if (warp < 2) {
        acc[0] += (double)(ge.wk * q);
#pragma unroll
        for (int r = 0; r < 8; ++r)
          if (r < R) tile[X * XS + r * kFmCS + j] = make_float2(h[2 * r], h[2 * r + 1]);
      } else if (ge.knorm > 0.f) {
        const float f = ge.wk * q * __frcp_rn(ge.knorm);
        acc[1] += (double)(f * ge.kv0 * ge.kv0);
        acc[2] += (double)(f * ge.kv1 * ge.kv1);
        acc[3] += (double)(f * ge.kv2 * ge.kv2);
        acc[4] += (double)(f * ge.kv0 * ge.kv1);
        acc[5] += (double)(f * ge.kv0 * ge.kv2);
        acc[6] += (double)(f * ge.kv1 * ge.kv2);
      }
    }
  }
  tc_fence_before();
  return ok;
}

__global__ void __launch_bounds__(kFmThreads, 1) k_filter_mma(MeshDev g, int P, int spme, const CellInfo* __restrict__ ci,
                                                              const float4* __restrict__ gtab,
                                                              const Tables* __restrict__ tab,
                                                              const float* __restrict__ deconv,
                                                              float2* __restrict__ spec, double* __restrict__ part) {
  extern __shared__ __align__(16) unsigned char fm_raw[];
  __shared__ uint64_t s_bar[2];
  __shared__ uint32_t s_tmem;
  __shared__ int s_fail;
  __shared__ float s_lam[8];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int S = g.S, R = g.R, XS = fm_xs(R);
  unsigned char* base = reinterpret_cast<unsigned char*>(((uintptr_t)fm_raw + 1023) & ~(uintptr_t)1023);
  const uint32_t a_sm = smem_u32(base);                        // [stage] x 64 KB
  const uint32_t b_sm = a_sm + 2 * kFmABytes;                  // [stage] x 16 KB
  const size_t tb = (fm_tile_bytes(S, R) + 127) & ~(size_t)127;
  unsigned char* tiles_base = base + 2 * kFmABytes + 2 * kFmBBytes;
  FmGeo* geo = reinterpret_cast<FmGeo*>(tiles_base + 2 * tb);

  // zero both stages' operands once: padding (species >= S, ranks >= R, the zero half of the
  // low-B rows) stays zero
  for (int i = tid; i < (2 * kFmABytes + 2 * kFmBBytes) / 16; i += kFmThreads)
    reinterpret_cast<float4*>(base)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  if (tid < 8) s_lam[tid] = tid < R ? (float)tab->eigs[tid] : 0.f;
  if (tid == 0) {
    mbar_init(&s_bar[0], 1);
    mbar_init(&s_bar[1], 1);
    s_fail = 0;
    mbar_fence_init();
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&s_tmem)),
                 "r"(kFmTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;

  const size_t Mh = (size_t)g.n[0] * g.n[1] * g.nzh;
  const size_t ntile = (Mh + kFmKT - 1) / kFmKT;
  float rc[9];
  load_recip<float>(ci, rc);
  const float inv_h = green_inv_h(g, ci);
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};

  // This lane's species pairs: upper-triangle blocks of 8 rows x 4 columns (block b of the
  // row-major list of blocks with 4 by + 3 >= 8 bx), blocks warp, warp + 12, ...; per block the
  // table row (float4 index, -1: no pair) and the A offsets of (X, 2Y) and of the mirror (Y, 2X).
  int prow[kFmMaxBlk];
  uint32_t poff[kFmMaxBlk], pmir[kFmMaxBlk];
  {
    const int nbx = (S + 7) >> 3, nby = (S + 3) >> 2;
    int b = 0, mine = 0;
    for (int bx = 0; bx < nbx; ++bx)
      for (int by = 2 * bx; by < nby; ++by, ++b) {
        if (b % kFmWarps != warp) continue;
        const int X = 8 * bx + (lane >> 2), Y = 4 * by + (lane & 3);
        const bool ok = X < S && Y < S && Y >= X;
#pragma unroll
        for (int i = 0; i < kFmMaxBlk; ++i)
          if (i == mine) {
            prow[i] = ok ? (X * S - X * (X - 1) / 2 + (Y - X)) * (kGreenKnots + 1) : -1;
            poff[i] = op_off(X, 2 * Y);
            pmir[i] = op_off(ok ? Y : X, 2 * (ok ? X : Y));
          }
        ++mine;
      }
#pragma unroll
    for (int i = 0; i < kFmMaxBlk; ++i)
      if (i >= mine) {
        prow[i] = -1;
        poff[i] = 0;
        pmir[i] = 0;
      }
  }
  // This lane's B entries: blocks of 8 rows n x 4 species Y (blocks warp, warp + 12, ...); per
  // block the tile offset of S[Y, r = n / 2] (-1: padding) and the B offset of (n, 2Y); the lane's
  // component (re or im) is n's parity, the same in every block
  const bool bimag = ((lane >> 2) & 1) != 0;
  int btile[kFmMaxBBlk];
  uint32_t boff[kFmMaxBBlk];
#pragma unroll
  for (int i = 0; i < kFmMaxBBlk; ++i) {
    const int blk = warp + kFmWarps * i;
    const int n = 8 * (blk & 1) + (lane >> 2), Y = 4 * (blk >> 1) + (lane & 3), r = n >> 1;
    const bool ok = blk < 2 * ((S + 3) >> 2) && r < R && Y < S;
    btile[i] = ok ? Y * XS + r * kFmCS : -1;
    boff[i] = ok ? op_off(n, 2 * Y) : 0u;
  }

  // commits waited for / issued per stage (counted by every thread; scalars, not an indexed array)
  uint32_t use0 = 0u, use1 = 0u, iss0 = 0u, iss1 = 0u;
  bool fail = false, stop = false;  // stop: uniform, decided right after a barrier


  int cur = 0;
  size_t tile_id = blockIdx.x;
  // the two spectrum tiles, by offset (no dynamically indexed pointer array)
  auto tile_at = [&](int b) { return reinterpret_cast<float2*>(tiles_base + (b ? tb : 0)); };
  if (tile_id < ntile) fm_prefetch(tile_at(0), spec, Mh, tile_id * kFmKT, S, R, XS);
  for (; tile_id < ntile; tile_id += gridDim.x) {
    const size_t k0 = tile_id * kFmKT;
    float2* tile = tile_at(cur);
    cp_async_wait_all();
    if (tid < kFmKT) {
      FmGeo ge;
      const size_t k = k0 + tid;
      ge.valid = k < Mh;
      const KPoint<float> q = kpoint<float>(g, ge.valid ? k : 0, rc, deconv, spme, P);
      ge.inv_sc = q.inv_sc;
      ge.dscale = q.inv_sc * inv_h;
      ge.wk = q.wk;
      ge.knorm = q.knorm;
      ge.kv0 = q.kv[0];
      ge.kv1 = q.kv[1];
      ge.kv2 = q.kv[2];
      ge.partner = q.partner ? 1 : 0;
      table_pos(q.knorm, inv_h, ge.tj, ge.hb);
      table_pos(q.kpart, inv_h, ge.pj, ge.pb);
      geo[tid] = ge;
    }
    __syncthreads();   // tile staged, geometry set; the other buffer's write-back is done
    if (s_fail) break;
    if (tile_id + gridDim.x < ntile) fm_prefetch(tile_at(cur ^ 1), spec, Mh, (tile_id + gridDim.x) * kFmKT, S, R, XS);
    for (int j = 0; j < kFmKT; ++j) {
      const int st = j & 1;
      const uint32_t a_st = a_sm + st * kFmABytes, b_st = b_sm + st * kFmBBytes;
      // A's table rows for this k-point, all requested before any arithmetic (the B build below
      // runs while they are in flight)
      const FmGeo& ge = geo[j];
      const int tj = ge.tj;
      float4 ta[kFmMaxBlk], tb4[kFmMaxBlk];
#pragma unroll
      for (int i = 0; i < kFmMaxBlk; ++i)
        if (prow[i] >= 0) {
          ta[i] = __ldg(gtab + prow[i] + tj);
          tb4[i] = __ldg(gtab + prow[i] + tj + 1);
        }
      // B: row n = 2 r + (re, im) holds (high, high) at k = 2Y, 2Y+1; row 16 + n holds (low, 0)
#pragma unroll
      for (int i = 0; i < kFmMaxBBlk; ++i)
        if (btile[i] >= 0) {
          const float2 v = tile[btile[i] + j];
          const float x = bimag ? v.y : v.x;
          const uint32_t hbits = tf32_round(x);
          const uint32_t lbits = tf32_round(x - __uint_as_float(hbits));
          st_shared_v2(b_st + boff[i], hbits, hbits);
          st_shared_v2(b_st + boff[i] + 2 * kFmSBO, lbits, 0u);
        }
      // A: Gh at rows X, dG at rows 64 + X; every pair Y >= X evaluated once and written at (X, Y)
      // and (Y, X) (the same place on the diagonal)
      const HermiteF hb = ge.hb;
      const float inv_sc = ge.inv_sc, dscale = ge.dscale;
      const bool partner = ge.partner != 0;
#pragma unroll
      for (int i = 0; i < kFmMaxBlk; ++i) {
        if (prow[i] < 0) continue;
        float gv = herm_value(hb, ta[i], tb4[i]) * inv_sc;
        const float dv = herm_slope(hb, ta[i], tb4[i]) * dscale;
        if (partner) {
          float gpv, dpv;
          green_lookup(gtab + prow[i], ge.pj, ge.pb, inv_h, gpv, dpv);
          gv = 0.5f * (gv + gpv * inv_sc);
        }
        const uint32_t gh = tf32_round(gv), gl = tf32_round(gv - __uint_as_float(gh));
        const uint32_t dh = tf32_round(dv), dl = tf32_round(dv - __uint_as_float(dh));
        const uint32_t ad = a_st + poff[i], am = a_st + pmir[i];
        st_shared_v2(ad, gh, gl);
        st_shared_v2(ad + kFmDgOff, dh, dl);
        st_shared_v2(am, gh, gl);
        st_shared_v2(am + kFmDgOff, dh, dl);
      }
      fence_proxy_async_smem();   // operand stores -> visible to the tensor core
      tc_fence_before();
      __syncthreads();
      if (s_fail) {
        stop = true;
        break;
      }
      if (st) ++iss1; else ++iss0;
      if (tid == 0) {
        tc_fence_after();
        const uint32_t d_tmem = tmem + (uint32_t)(st * kFmN);
#pragma unroll
        for (int ks = 0; ks < kFmK / 8; ++ks)
          mma_tf32(d_tmem, umma_desc(a_st + 256 * ks, 128, kFmSBO), umma_desc(b_st + 256 * ks, 128, kFmSBO),
                   ks > 0 ? 1u : 0u);
        mma_commit(&s_bar[st]);
      }
      if (j > 0) {
        const int sp = st ^ 1;
        const uint32_t par = (sp ? use1 : use0) & 1u;
        if (!fm_epilogue(sp, j - 1, tile, &s_bar[sp], par, tmem, warp, lane, S, R, XS, s_lam, geo, acc)) {
          s_fail = 1;
          fail = true;
        }
        if (sp) ++use1; else ++use0;
      }
    }
    if (stop) break;
    {
      const int sp = (kFmKT - 1) & 1;
      const uint32_t par = (sp ? use1 : use0) & 1u;
      if (!fm_epilogue(sp, kFmKT - 1, tile, &s_bar[sp], par, tmem, warp, lane, S, R, XS, s_lam, geo, acc)) {
        s_fail = 1;
        fail = true;
      }
      if (sp) ++use1; else ++use0;
    }
    __syncthreads();   // H of the whole tile is in shared memory
    if (s_fail) break;
    const int C = S * R;
    const uint32_t invR = (65536u + (uint32_t)R - 1u) / (uint32_t)R;
    for (int e = tid; e < C * kFmKT; e += kFmThreads) {
      const int c = e / kFmKT, jj = e - c * kFmKT;
      const size_t k = k0 + jj;
      if (k < Mh) {
        const int X = (int)(((uint32_t)c * invR) >> 16), r = c - X * R;
        spec[(size_t)c * Mh + k] = tile[X * XS + r * kFmCS + jj];
      }
    }
    cur ^= 1;
  }
  cp_async_wait_all();
  // a wait ran out: wait (bounded again) for every MMA still in flight before TMEM is freed,
  // and make the block's energy partial NaN
  while (use0 < iss0) {
    if (!mbar_wait(&s_bar[0], use0 & 1u)) fail = true;
    ++use0;
  }
  while (use1 < iss1) {
    if (!mbar_wait(&s_bar[1], use1 & 1u)) fail = true;
    ++use1;
  }
  if (fail || s_fail) acc[0] = __longlong_as_double(0x7ff8000000000000LL);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kFmTmemCols) : "memory");
  }
  double fin[7];   // the per-thread sums stay in registers during the loop
#pragma unroll
  for (int c = 0; c < 7; ++c) fin[c] = acc[c];
  block_sum_store<7>(fin, part + 7 * blockIdx.x);
}

// species x ranks whose operands and two spectrum tiles fit the 227 KB of a B200 CTA, and whose
// upper-triangle pair blocks fit kFmMaxBlk per warp
bool filter_mma_applies(const MeshGeom& mg) {
  return mg.S >= 1 && mg.S <= kFmMaxS && mg.R >= 1 && mg.R <= 8 && fm_smem_bytes(mg.S, mg.R) <= 225 * 1024 &&
         fm_upper_blocks(mg.S) <= kFmMaxBlk * kFmWarps;
}

// In effect for a float spectrum when it applies and is asked for (off by default: at 54 species
// building the per-k-point operands costs more than the CUDA-core filter's products; the batch
// autotuner times both).
bool filter_mma_on(const MeshGeom& mg) { return mg.filter_mma == 1 && filter_mma_applies(mg); }

int launch_filter_mma(const MeshGeom& mg, const CellInfo* ci, const float4* gtab, const Tables* tab,
                      const float* deconv, int spme, void* spec, double* part, int* n_blocks, cudaStream_t s) {
  if (!filter_mma_applies(mg)) {
    set_error("filter", "the tensor-core filter takes at most 64 species and 8 ranks");
    return FD3_EINVAL;
  }
  const size_t smem = fm_smem_bytes(mg.S, mg.R);
  static int allowed = -1;
  if (allowed < 0) {
    int dev = 0, optin = 0;
    cudaFuncAttributes fa{};
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess ||
        cudaFuncGetAttributes(&fa, k_filter_mma) != cudaSuccess ||
        cudaFuncSetAttribute(k_filter_mma, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             optin - (int)fa.sharedSizeBytes) != cudaSuccess) {
      set_error("filter", "could not raise the shared-memory limit of the tensor-core filter");
      return FD3_ECUDA;
    }
    allowed = optin - (int)fa.sharedSizeBytes;
  }
  if (smem > (size_t)allowed) {
    set_error("filter", "tensor-core filter tile does not fit in shared memory (too many species x ranks)");
    return FD3_EINVAL;
  }
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const size_t Mh = (size_t)mg.n[0] * mg.n[1] * mg.nzh;
  const size_t ntile = (Mh + kFmKT - 1) / kFmKT;
  size_t blocks = (size_t)sms;
  if (blocks > ntile) blocks = ntile;
  if (blocks > (size_t)filter_max_blocks()) blocks = filter_max_blocks();
  *n_blocks = (int)blocks;
  const MeshDev g = to_dev(mg);
  k_filter_mma<<<(int)blocks, kFmThreads, smem, s>>>(g, mg.order, spme, ci, gtab, tab, deconv,
                                                     reinterpret_cast<float2*>(spec), part);
  FD3_LAUNCHED();
  return FD3_OK;
}

}  // namespace fd3

// Fused x-pass over rank groups, moved by TMA: forward FFT along x, the reciprocal-space
// filter, inverse FFT along x, on the float spectrum of the (y, z) 2D transforms.
//
// Spectrum layout (the reference's channel-major mesh, kspace_filter_d3.py:55): channel
// c = X R + r (species X, rank r), then x, then the flattened (y, kz) index q = y P + kz, with P
// = nz/2+1 values per ky row, or nz/2+2 (a zero pad slot, 16-byte rows) when the fused (y, z)
// transforms write it.
// For fixed (c, x) every q is contiguous, so a pencil of Q consecutive q values across all x is
// nx contiguous runs of Q complex values (Q = 16: one 128-byte line per run), one stride apart.
//
// The filter couples species only within one rank (H[X,r] = sum_Y G_XY S[Y,r], the per-rank
// S x S product of kspace_filter_d3.py:64), so a work unit holds the S species channels of RG
// ranks only: unit = (rank group, q-block), a box of (Q q values) x (nx) x (RG ranks) x (S
// species) that one 4-D TMA copy (cp.async.bulk.tensor, no multicast, this GPU's own memory)
// brings into shared memory and one TMA store writes back in place. Units are ordered q-block
// fastest, so the CTAs running at the same time read neighbouring lines of the same rows.
//
// One CTA per SM: a producer warp keeps a ring of `nstage` unit buffers full (mbarrier
// complete_tx), issues the TMA store of each finished unit, and reuses its buffer for the unit
// `nstage` ahead once the store has read it; 16 compute warps (96 registers each, one item per
// loop trip) run the two register-DFT passes,
// the filter and the two inverse passes on each buffer. Every mbarrier wait is bounded; a wait
// that runs out marks the block's energy partial NaN and ends the block.
#pragma once
#include <cuda.h>

#include "fd3_async.cuh"
#include "fd3_xfilter.cuh"

namespace fd3 {

constexpr int kXpCompute = 512;          // compute threads (16 warps); the producer warp follows
constexpr int kXpThreads = kXpCompute + 32;
constexpr int kXpMaxStages = 4;
constexpr int kXpTwBytes = 8192;         // twiddles (at most 16 x 17 float2) + per-axis SPME window
constexpr int kXpAlignPad = 1024;        // room to align the unit buffers (dynamic shared memory)

__device__ __forceinline__ void compute_bar() {
  asm volatile("bar.sync 1, %0;\n" ::"n"(kXpCompute) : "memory");
}

// ------------------------------------------------------------------ filter of one rank group
// Filter of one k-point over the S species of ranks r0 .. r0+RG-1 (ranks >= R are padding):
// channel (X, r) at v[(X RG + r) cs]. Same arithmetic as filter_point, split by rank.
template <int MAXS, int RG>
__device__ __forceinline__ void filter_group(const KPoint<float>& q, int S, int R, int r0,
                                             const GreenPairF* __restrict__ gp, const float4* __restrict__ gtab,
                                             float inv_h, float s6, float s8, const float (&lam)[RG],
                                             float2* v, int cs, double* acc) {
  float G[MAXS][MAXS], dG[MAXS][MAXS], Gh[MAXS][MAXS];
  green_block<float, MAXS>(q, S, gp, gtab, inv_h, s6, s8, G, dG, Gh);
  float qq = 0.f, dq = 0.f;
  const bool full = S == MAXS;
#pragma unroll
  for (int r = 0; r < RG; ++r) {
    if (r0 + r < R) {
      float2 sv[MAXS];
#pragma unroll
      for (int X = 0; X < MAXS; ++X) sv[X] = (full || X < S) ? v[(X * RG + r) * cs] : float2{0.f, 0.f};
      float qr = 0.f, dqr = 0.f;
#pragma unroll
      for (int X = 0; X < MAXS; ++X) {
        float hre = 0.f, him = 0.f;
#pragma unroll
        for (int Y = 0; Y < MAXS; ++Y) {
          hre += Gh[X][Y] * sv[Y].x;
          him += Gh[X][Y] * sv[Y].y;
          const float re = sv[X].x * sv[Y].x + sv[X].y * sv[Y].y;
          qr += G[X][Y] * re;
          dqr += dG[X][Y] * re;
        }
        if (full || X < S) v[(X * RG + r) * cs] = float2{hre, him};
      }
      qq += lam[r] * qr;
      dq += lam[r] * dqr;
    }
  }
  acc[0] += (double)(q.wk * qq);
  virial_acc<float>(q, dq, acc);
}

// ------------------------------------------------------------------ register-DFT passes
// Two layouts of a unit's values (channel ch < Cg, x slot, q offset qq < Q):
//  * dense, as the TMA box lands: buf[(ch NX + x) Q + qq];
//  * padded working copy: wk[ch CS + (x >> log2 N2) GS + (x mod N2) Q + qq], GS = N2 Q + PADG.
// The forward pass 1 reads the dense unit and writes the working copy, the inverse pass 1 reads the
// working copy and writes the dense unit back for the TMA store; pass 2 and the filter stay in the
// working copy. Pass 2 walks the N2 slots of one k1 group, and with Q < 16 the lanes of a warp span
// several k1 groups: a group stride of N2 Q values (a multiple of 128 bytes) would put them on the
// same banks, so each group carries PADG = Q padding values.
// Forward: natural x order in, slot N2 k1 + k2 holding ix = k1 + N1 k2 out. Inverse: reverse.
template <int N1, int N2, int Q>
struct XpWork {
  static constexpr int PADG = Q < 16 ? Q : 0;
  static constexpr int GS = N2 * Q + PADG;   // values per k1 group
  static constexpr int CS = N1 * GS;         // values per channel
  static constexpr int LN2 = log2_n<N2>();
  __host__ __device__ static constexpr size_t bytes(int Cg) { return (size_t)Cg * CS * sizeof(float2); }
  __device__ static int off(int ch, int x, int qq) { return ch * CS + (x >> LN2) * GS + (x & (N2 - 1)) * Q + qq; }
};

template <int N1, int N2, int Q>
__device__ __forceinline__ void xp_pass_n1(float2* buf, float2* wk, const float2* tw, int Cg, bool inverse) {
  using W = XpWork<N1, N2, Q>;
  constexpr int NX = N1 * N2, LQ = log2_n<Q>(), LN2 = log2_n<N2>();
  const int items = (Cg * N2) << LQ;
#pragma unroll 1
  for (int it = threadIdx.x; it < items; it += kXpCompute) {
    const int qq = it & (Q - 1), n2 = (it >> LQ) & (N2 - 1), ch = it >> (LQ + LN2);
    float2* d = buf + ((size_t)ch * NX + n2) * Q + qq;      // dense: x = N2 n1 + n2 at d[n1 N2 Q]
    float2* w = wk + ch * W::CS + n2 * Q + qq;             // working: slot N2 k1 + n2 at w[k1 GS]
    float re[N1], im[N1];
    if (!inverse) {
#pragma unroll
      for (int n1 = 0; n1 < N1; ++n1) {
        const float2 v = d[n1 * N2 * Q];
        re[n1] = v.x;
        im[n1] = v.y;
      }
      dft_reg<float, N1, -1>(re, im);
#pragma unroll
      for (int k1 = 0; k1 < N1; ++k1) {
        const float2 t = tw[n2 * (N1 + 1) + k1];   // exp(-2 pi i n2 k1 / NX)
        w[k1 * W::GS] = float2{re[k1] * t.x - im[k1] * t.y, re[k1] * t.y + im[k1] * t.x};
      }
    } else {
#pragma unroll
      for (int k1 = 0; k1 < N1; ++k1) {
        const float2 v = w[k1 * W::GS];
        const float2 t = tw[n2 * (N1 + 1) + k1];   // conj: exp(+2 pi i n2 k1 / NX)
        re[k1] = v.x * t.x + v.y * t.y;
        im[k1] = v.y * t.x - v.x * t.y;
      }
      dft_reg<float, N1, 1>(re, im);
#pragma unroll
      for (int n1 = 0; n1 < N1; ++n1) d[n1 * N2 * Q] = float2{re[n1], im[n1]};
    }
  }
}

template <int N1, int N2, int Q>
__device__ __forceinline__ void xp_pass_n2(float2* wk, int Cg, bool inverse) {
  using W = XpWork<N1, N2, Q>;
  constexpr int LQ = log2_n<Q>(), LN1 = log2_n<N1>();
  const int items = (Cg * N1) << LQ;
#pragma unroll 1
  for (int it = threadIdx.x; it < items; it += kXpCompute) {
    const int qq = it & (Q - 1), k1 = (it >> LQ) & (N1 - 1), ch = it >> (LQ + LN1);
    float2* b = wk + ch * W::CS + k1 * W::GS + qq;
    float re[N2], im[N2];
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) {
      const float2 v = b[n2 * Q];
      re[n2] = v.x;
      im[n2] = v.y;
    }
    if (!inverse)
      dft_reg<float, N2, -1>(re, im);
    else
      dft_reg<float, N2, 1>(re, im);
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) b[k2 * Q] = float2{re[k2], im[k2]};
  }
}

// ------------------------------------------------------------------ the kernel
// Units u = group * nqb + qb over the ny (nz/2+1) / Q q-blocks and ceil(R / RG) rank groups;
// CTA b takes units b, b + gridDim.x, ... . Requires nx = N1 N2 (the TMA box spans all x).
template <int N1, int N2, int Q, int RG, int MAXS>
__global__ void __launch_bounds__(kXpThreads, 1)
    k_xpass(const __grid_constant__ CUtensorMap tmap, MeshDev g, int P, int spme, int nstage, int nqb, int nunits,
            const CellInfo* __restrict__ ci, const GreenPairF* __restrict__ gp, const float4* __restrict__ gtab,
            const Tables* __restrict__ tab, const float* __restrict__ deconv, double* __restrict__ part) {
  constexpr int NX = N1 * N2, LQ = log2_n<Q>(), LN2 = log2_n<N2>();
  extern __shared__ __align__(128) unsigned char xp_raw[];
  __shared__ __align__(8) uint64_t full_bar[kXpMaxStages], done_bar[kXpMaxStages];
  __shared__ int xp_fail, prod_fail;
  // TMA destinations 1024-byte aligned whatever the placement of the dynamic shared memory
  unsigned char* xp_base = xp_raw + ((1024u - (smem_u32(xp_raw) & 1023u)) & 1023u);
  float2* tw = reinterpret_cast<float2*>(xp_base);
  float2* bufs = reinterpret_cast<float2*>(xp_base + kXpTwBytes);
  const int S = g.S, R = g.R, Cg = S * RG;
  const int buf_elems = (Cg * NX) << LQ;
  using W = XpWork<N1, N2, Q>;
  float2* wk = bufs + (size_t)nstage * buf_elems;   // padded working copy of the unit in flight
  const uint32_t buf_bytes = (uint32_t)buf_elems * 8u;
  const int tid = threadIdx.x;
  if (tid == 0) {
    for (int s = 0; s < nstage; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&done_bar[s], kXpCompute);
    }
    xp_fail = 0;
    prod_fail = 0;
    mbar_fence_init();
  }
  // the mixed form's per-axis SPME window (nx + ny + nz/2+1 floats), read per k-point, in shared memory
  float* s_win = reinterpret_cast<float*>(xp_base + kXpTwBytes / 2);
  const int nwin = g.n[0] + g.n[1] + g.nzh;
  if (g.win_axes)
    for (int m = tid; m < nwin; m += blockDim.x) s_win[m] = g.win_axes[m];
  for (int m = tid; m < N2 * (N1 + 1); m += blockDim.x) {
    const int a = m / (N1 + 1), b = m % (N1 + 1);
    double sn, cs;
    sincospi(-2.0 * ((a * b) % NX) / NX, &sn, &cs);
    tw[m] = float2{(float)cs, (float)sn};
  }
  __syncthreads();
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  if (tid >= kXpCompute) {
    // ---------------- producer warp: TMA loads and stores of the unit ring
    if (tid == kXpCompute) {
      auto load = [&](int u, int s) {
        const int grp = u / nqb, qb = u - grp * nqb;
        mbar_arrive_expect_tx(&full_bar[s], buf_bytes);
        tma_load_4d(bufs + (size_t)s * buf_elems, &tmap, (qb * Q) * 2, 0, grp * RG, 0, &full_bar[s]);
      };
      for (int s = 0; s < nstage; ++s) {
        const int u = blockIdx.x + s * gridDim.x;
        if (u < nunits) load(u, s);
      }
      for (int k = 0;; ++k) {
        const int u = blockIdx.x + k * gridDim.x;
        if (u >= nunits) break;
        const int s = k % nstage;
        if (!mbar_wait(&done_bar[s], (uint32_t)(k / nstage) & 1u)) {
          prod_fail = 1;   // no further loads: the compute warps' waits run out as well
          break;
        }
        const int grp = u / nqb, qb = u - grp * nqb;
        tma_store_4d(&tmap, (qb * Q) * 2, 0, grp * RG, 0, bufs + (size_t)s * buf_elems);
        bulk_commit();
        const int un = u + nstage * gridDim.x;
        if (un < nunits) {
          bulk_wait_read_all();   // the store has read the buffer: reuse it
          load(un, s);
        }
      }
      bulk_wait_all();
    }
  } else {
    // ---------------- compute warps
    const float s6 = (float)tab->s6, s8 = (float)tab->s8;
    float rc[9];
    load_recip<float>(ci, rc);
    const float inv_h = green_inv_h(g, ci);
    MeshDev gs = g;
    if (g.win_axes) gs.win_axes = s_win;
    const int n1 = g.n[1], nzh = g.nzh, qp = g.qpitch;
    const int nq = n1 * qp;   // flattened (y, kz) slots per x-row, pad slots included
    for (int k = 0;; ++k) {
      const int u = blockIdx.x + k * gridDim.x;
      if (u >= nunits) break;
      const int s = k % nstage;
      // the decision to stop is taken after a barrier, so that every compute thread takes it
      if (!mbar_wait(&full_bar[s], (uint32_t)(k / nstage) & 1u)) xp_fail = 1;
      compute_bar();
      if (*(volatile int*)&xp_fail) break;
      float2* buf = bufs + (size_t)s * buf_elems;
      const int grp = u / nqb, qb = u - grp * nqb;
      xp_pass_n1<N1, N2, Q>(buf, wk, tw, Cg, false);
      compute_bar();
      xp_pass_n2<N1, N2, Q>(wk, Cg, false);
      compute_bar();
      float lam[RG];   // lambda of the unit's ranks (padding ranks: 0, never used)
#pragma unroll
      for (int r = 0; r < RG; ++r) lam[r] = grp * RG + r < R ? (float)tab->eigs[grp * RG + r] : 0.f;
#pragma unroll 1
      for (int pt = tid; pt < (NX << LQ); pt += kXpCompute) {
        const int qq = pt & (Q - 1), slot = pt >> LQ;
        const int qf = qb * Q + qq;
        if (qf >= nq) continue;
        const int y = (int)fdiv((uint32_t)qf, g.div_qpitch);
        const int iz = qf - y * qp;
        if (iz >= nzh) continue;   // the pad slot of a 16-byte spectrum row: zero, left as it is
        const int ix = (slot >> LN2) + N1 * (slot & (N2 - 1));
        const size_t kflat = ((size_t)ix * n1 + y) * nzh + iz;
        const KPoint<float> q = kpoint_idx<float>(gs, ix, y, iz, kflat, rc, deconv, spme, P);
        filter_group<MAXS, RG>(q, S, R, grp * RG, gp, gtab, inv_h, s6, s8, lam, wk + W::off(0, slot, qq), W::CS,
                               acc);
      }
      compute_bar();
      xp_pass_n2<N1, N2, Q>(wk, Cg, true);
      compute_bar();
      xp_pass_n1<N1, N2, Q>(buf, wk, tw, Cg, true);
      fence_proxy_async_smem();
      mbar_arrive(&done_bar[s]);
    }
  }
  __syncthreads();
  if ((xp_fail || prod_fail) && tid == 0) acc[0] = __longlong_as_double(0x7ff8000000000000LL);   // NaN: the result is invalid
  block_sum_store<7>(acc, part + 7 * blockIdx.x);
}

}  // namespace fd3

// Launcher of the TMA fused x-pass (instantiated per x length in fd3_xpass_{64,128,256}.cu).
#pragma once
#include "fd3_xpass.cuh"

namespace fd3 {

// Dynamic shared memory the x-pass may take (the B200 limit is 227 KB per CTA, including the
// kernel's static shared memory).
constexpr size_t kXpSmemCap = 220 * 1024;

// Ring stages that fit for a unit of the given size beside its padded working copy, at most
// kXpMaxStages (0: fewer than 2 fit).
inline int xpass_stages(size_t unit_bytes, size_t work_bytes) {
  const size_t fixed = kXpAlignPad + kXpTwBytes + work_bytes;
  if (fixed >= kXpSmemCap) return 0;
  const size_t n = (kXpSmemCap - fixed) / unit_bytes;
  if (n < 2) return 0;
  return n > (size_t)kXpMaxStages ? kXpMaxStages : (int)n;
}

struct XpassArgs {
  const CUtensorMap* map;
  MeshGeom mg;
  const CellInfo* ci;
  const GreenPairF* gp;
  const float4* gtab;
  const Tables* tab;
  const float* deconv;
  int spme;
  int Q, RG;
  double* part;
  int* n_blocks;
  cudaStream_t s;
};

template <int N1, int N2, int Q, int RG, int MAXS>
int launch_xpass_t(const XpassArgs& a) {
  constexpr int NX = N1 * N2;
  const MeshGeom& mg = a.mg;
  const size_t unit = (size_t)mg.S * RG * NX * Q * sizeof(float2);
  const size_t work = XpWork<N1, N2, Q>::bytes(mg.S * RG);
  const int nstage = xpass_stages(unit, work);
  if (nstage < 2) {
    set_error("filter", "fused x-pass unit does not fit twice in shared memory");
    return FD3_EINVAL;
  }
  const size_t smem = kXpAlignPad + kXpTwBytes + (size_t)nstage * unit + work;
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(k_xpass<N1, N2, Q, RG, MAXS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kXpSmemCap) != cudaSuccess) {
      set_error("filter", "could not raise the shared-memory limit of the fused x-pass");
      return FD3_ECUDA;
    }
    attr = true;
  }
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
  const long long nq = (long long)mg.n[1] * (mg.qpitch > 0 ? mg.qpitch : mg.nzh);
  const int nqb = (int)((nq + Q - 1) / Q);
  const int ngrp = (mg.R + RG - 1) / RG;
  const long long nunits = (long long)nqb * ngrp;
  if (nunits > (1LL << 30)) return FD3_EINVAL;
  long long blocks = sms;   // one CTA per SM, persistent over the units
  if (blocks > nunits) blocks = nunits;
  if (blocks > filter_max_blocks()) blocks = filter_max_blocks();
  *a.n_blocks = (int)blocks;
  k_xpass<N1, N2, Q, RG, MAXS><<<(int)blocks, kXpThreads, smem, a.s>>>(
      *a.map, to_dev(mg), mg.order, a.spme, nstage, nqb, (int)nunits, a.ci, a.gp, a.gtab, a.tab, a.deconv, a.part);
  FD3_LAUNCHED();
  return FD3_OK;
}

template <int N1, int N2, int Q, int RG>
int launch_xpass_s(const XpassArgs& a) {
  if (a.mg.S <= 2) return launch_xpass_t<N1, N2, Q, RG, 2>(a);
  return launch_xpass_t<N1, N2, Q, RG, 4>(a);
}

template <int N1, int N2, int Q>
int launch_xpass_r(const XpassArgs& a) {
  if (a.RG == 1) return launch_xpass_s<N1, N2, Q, 1>(a);
  if (a.RG == 2) return launch_xpass_s<N1, N2, Q, 2>(a);
  if (a.RG == 4) return launch_xpass_s<N1, N2, Q, 4>(a);
  return FD3_EINVAL;
}

template <int N1, int N2>
int launch_xpass_nx(const XpassArgs& a) {
  if (a.Q == 4) return launch_xpass_r<N1, N2, 4>(a);
  if (a.Q == 8) return launch_xpass_r<N1, N2, 8>(a);
  if (a.Q == 16) return launch_xpass_r<N1, N2, 16>(a);
  if (a.Q == 32) return launch_xpass_r<N1, N2, 32>(a);
  return FD3_EINVAL;
}

int launch_xpass_64(const XpassArgs& a);
int launch_xpass_128(const XpassArgs& a);
int launch_xpass_256(const XpassArgs& a);

}  // namespace fd3

// Launcher of the fused x-pass filter (instantiated per precision in fd3_xfilter_f32/f64.cu).
#pragma once
#include "fd3_xfilter.cuh"

namespace fd3 {

template <typename T, int MAXS, int MAXR, int N1, int N2, int LKZ>
static int launch_xk(const MeshGeom& mg, const CellInfo* ci, const typename GreenPairOf<T>::type* gp,
                     const float4* gtab, const Tables* tab, const float* deconv, int spme,
                     typename Cplx<T>::type* sp, double* part, int* n_blocks, cudaStream_t s) {
  constexpr int KZ = 1 << LKZ;
  const size_t smem = xfilter_smem<T, N1, N2>(mg.S * mg.R, KZ);
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(k_xfilter<T, MAXS, MAXR, N1, N2, LKZ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             200 * 1024) != cudaSuccess) {
      set_error("filter", "could not raise the shared-memory limit of the fused x-pass filter");
      return FD3_ECUDA;
    }
    attr = true;
  }
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_xfilter<T, MAXS, MAXR, N1, N2, LKZ>, kFilterThreads,
                                                    smem) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
  // pencils per y: one more when float pairs shift odd-parity rows (kernel: ngz)
  const bool pairs = sizeof(T) == 4 && LKZ >= 1 && (((size_t)mg.n[1] * mg.nzh) & 1) == 0;
  const long long ngroups = (long long)mg.n[1] * ((mg.nzh + (pairs ? 1 : 0) + KZ - 1) / KZ);
  long long blocks = (long long)sms * per_sm;
  if (blocks > ngroups) blocks = ngroups;
  if (blocks > filter_max_blocks()) blocks = filter_max_blocks();
  *n_blocks = (int)blocks;
  k_xfilter<T, MAXS, MAXR, N1, N2, LKZ><<<(int)blocks, kFilterThreads, smem, s>>>(to_dev(mg), mg.order, spme, ci, gp,
                                                                                 gtab, tab, deconv, sp, part);
  FD3_LAUNCHED();
  return FD3_OK;
}

template <typename T, int MAXS, int MAXR, int N1, int N2>
static int launch_x(const MeshGeom& mg, int KZ, const CellInfo* ci, const typename GreenPairOf<T>::type* gp,
                    const float4* gtab, const Tables* tab, const float* deconv, int spme,
                    typename Cplx<T>::type* sp, double* part, int* n_blocks, cudaStream_t s) {
  if (KZ == 4)
    return launch_xk<T, MAXS, MAXR, N1, N2, 2>(mg, ci, gp, gtab, tab, deconv, spme, sp, part, n_blocks, s);
  if (KZ == 2)
    return launch_xk<T, MAXS, MAXR, N1, N2, 1>(mg, ci, gp, gtab, tab, deconv, spme, sp, part, n_blocks, s);
  return launch_xk<T, MAXS, MAXR, N1, N2, 0>(mg, ci, gp, gtab, tab, deconv, spme, sp, part, n_blocks, s);
}

template <typename T, int N1, int N2>
static int launch_x_sr(const MeshGeom& mg, int KZ, const CellInfo* ci, const typename GreenPairOf<T>::type* gp,
                       const float4* gtab, const Tables* tab, const float* deconv, int spme,
                       typename Cplx<T>::type* sp, double* part, int* n_blocks, cudaStream_t s) {
#define FD3_X(SS, RR) \
  return launch_x<T, SS, RR, N1, N2>(mg, KZ, ci, gp, gtab, tab, deconv, spme, sp, part, n_blocks, s)
  if (mg.S <= 1 && mg.R <= 4) FD3_X(1, 4);
  if (mg.S <= 2 && mg.R <= 4) FD3_X(2, 4);
  if (mg.S <= 2) FD3_X(2, 8);
  if (mg.R <= 4) FD3_X(4, 4);
  FD3_X(4, 8);
#undef FD3_X
}

template <typename T>
int launch_xfilter_t(const MeshGeom& mg, const CellInfo* ci, const GreenPair* gp, const GreenPairF* gpf,
                     const float4* gtab, const Tables* tab, const float* deconv, int spme, void* spec, double* part,
                     int* n_blocks, cudaStream_t s) {
  using GP = typename GreenPairOf<T>::type;
  const GP* gpt = reinterpret_cast<const GP*>(sizeof(T) == 8 ? (const void*)gp : (const void*)gpf);
  auto* sp = reinterpret_cast<typename Cplx<T>::type*>(spec);
  const int KZ = xfilter_kz<T>(mg);
  if (KZ < 1) return FD3_EINVAL;
  switch (mg.n[0]) {
    case 64: return launch_x_sr<T, 8, 8>(mg, KZ, ci, gpt, gtab, tab, deconv, spme, sp, part, n_blocks, s);
    case 128: return launch_x_sr<T, 8, 16>(mg, KZ, ci, gpt, gtab, tab, deconv, spme, sp, part, n_blocks, s);
    case 256: return launch_x_sr<T, 16, 16>(mg, KZ, ci, gpt, gtab, tab, deconv, spme, sp, part, n_blocks, s);
    default: return FD3_EINVAL;
  }
}

}  // namespace fd3

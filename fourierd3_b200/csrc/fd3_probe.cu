// Bandwidth probe of the fused x-pass access pattern (measurement only; no compute path calls
// it). Every value of a buffer shaped like the float half spectrum -- C channels, layout
// (C, nx, ny, nz/2+1), complex float -- is read and written back unchanged, pencil by pencil in
// the fused kernel's order: one y and KZ consecutive kz of every (channel, x) row per pencil,
// CTA b taking pencils b, b + grid, ... The time gives the bandwidth this access pattern can
// reach on the device (KZ-value pieces of rows ny * (nz/2+1) values apart): the ceiling of
// k_xfilter's spectrum traffic.
#include "fd3_internal.h"

namespace fd3 {

template <int LKZ>
__global__ void __launch_bounds__(256) k_probe_pencil(float2* __restrict__ spec, int rows, int n1, int nzh) {
  constexpr int KZ = 1 << LKZ, RPI = 256 >> LKZ;   // rows between one thread's consecutive items
  constexpr int BATCH = 16;                        // loads in flight per thread before the stores
  const int ngz = (nzh + KZ - 1) >> LKZ;
  const int j = threadIdx.x & (KZ - 1), r0 = threadIdx.x >> LKZ;
  const size_t xrow = (size_t)n1 * nzh;            // values between consecutive rows (c, x)
  for (int g = blockIdx.x; g < n1 * ngz; g += gridDim.x) {
    const int y = g / ngz;
    const int kz = ((g - y * ngz) << LKZ) + j;
    if (kz >= nzh) continue;
    float2* base = spec + (size_t)y * nzh + kz;
    for (int rb = r0; rb < rows; rb += BATCH * RPI) {
      float2 v[BATCH];
#pragma unroll
      for (int k = 0; k < BATCH; ++k) {
        const int r = rb + k * RPI;
        if (r < rows) v[k] = base[(size_t)r * xrow];
      }
#pragma unroll
      for (int k = 0; k < BATCH; ++k) {
        const int r = rb + k * RPI;
        if (r < rows) base[(size_t)r * xrow] = v[k];
      }
    }
  }
}

int launch_probe_pencil(const MeshGeom& mg, int KZ, void* buf, cudaStream_t s) {
  const int rows = mg.S * mg.R * mg.n[0];
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
  const int grid = 16 * sms;   // many pencils in flight: the pattern's ceiling, not one launch shape's
  float2* p = reinterpret_cast<float2*>(buf);
  if (KZ >= 4)
    k_probe_pencil<2><<<grid, 256, 0, s>>>(p, rows, mg.n[1], mg.nzh);
  else if (KZ == 2)
    k_probe_pencil<1><<<grid, 256, 0, s>>>(p, rows, mg.n[1], mg.nzh);
  else
    k_probe_pencil<0><<<grid, 256, 0, s>>>(p, rows, mg.n[1], mg.nzh);
  FD3_LAUNCHED();
  return FD3_OK;
}

}  // namespace fd3

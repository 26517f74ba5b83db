// Neighbour-list build that allocates nothing: its scratch lives in a fixed device array.
//
// Who needs this: callers that must not, or cannot, allocate device memory themselves -- an MD
// engine or a host-language runtime that hands out device memory only from its own pools and
// forbids raw cudaMalloc in its timestep, a plugin loaded into such a host, or code with a hard,
// pre-checked memory budget. The regular fd3_neighbor_fill needs a caller-allocated workspace
// (fd3_neighbor_workspace_size); fd3_neighbor_fill_static takes the same inputs and outputs but
// keeps the cell-list scratch (bins, bin-sorted copies of the atoms, per-atom counts and row
// offsets) in the file-scope array below, so it calls no cudaMalloc, cudaFree or allocating
// library routine.
//
// Costs and limits:
//  * the array is kStaticScratchBytes (6 MiB) of device memory on every GPU that loads this
//    library, held until the process exits; that is enough for about 65,000 atoms (the exact
//    limit also depends on the number of cell-list bins); larger inputs are rejected with
//    FD3_EINVAL and a message giving the bytes needed;
//  * every call shares the one array and leaves its contents behind; whatever must start at zero
//    (the bin histogram) is cleared inside each call. Calls that overlap on the GPU -- two host
//    threads, or two streams, running it at the same time -- race on the array and must be
//    serialised by the caller;
//  * the first call on a device looks up the array's device address (cudaGetSymbolAddress) with
//    that device current and caches it; make that first call before any stream capture. The
//    cached address belongs to the device's primary context: after cudaDeviceReset (which
//    destroys that context) it is stale, so do not call this entry point again in a process
//    that has reset the device.
#include <stdio.h>

#include <mutex>

#include "fd3_internal.h"

namespace {

constexpr size_t kStaticScratchBytes = (size_t)6 << 20;
constexpr int kMaxDevices = 64;

// Device scratch of the static-scratch neighbour build. Host code must not use the symbol as a
// pointer: its device address comes from cudaGetSymbolAddress (scratch_address below).
static __device__ __align__(256) unsigned char g_nbr_scratch[kStaticScratchBytes];

std::mutex g_scratch_mu;
void* g_scratch_addr[kMaxDevices] = {};

// Device address of g_nbr_scratch on the current device, looked up once per device.
int scratch_address(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    fd3::set_error("fd3_neighbor_fill_static: cudaGetDevice", cudaGetErrorString(e));
    return FD3_ECUDA;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    fd3::set_error("fd3_neighbor_fill_static", "device ordinal out of range");
    return FD3_EINVAL;
  }
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_nbr_scratch);
    if (e != cudaSuccess || !p) {
      fd3::set_error("fd3_neighbor_fill_static: cudaGetSymbolAddress", cudaGetErrorString(e));
      return FD3_ECUDA;
    }
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return FD3_OK;
}

}  // namespace

extern "C" int fd3_neighbor_fill_static(int64_t n_atoms, const double* d_pos_ang, const double* h_cell_ang,
                                        double r_cut_ang, int64_t capacity, int64_t* d_src, int64_t* d_dst,
                                        int32_t* d_shift, int64_t* h_count, void* stream) {
  if (!d_pos_ang || !h_cell_ang || !d_src || !d_dst || !d_shift || !h_count) {
    fd3::set_error("fd3_neighbor_fill_static", "null argument");
    return FD3_EINVAL;
  }
  size_t need = 0;
  int rc = fd3_neighbor_workspace_size(n_atoms, h_cell_ang, r_cut_ang, &need);
  if (rc) return rc;
  if (need > kStaticScratchBytes) {
    char msg[160];
    snprintf(msg, sizeof(msg),
             "needs %zu bytes of scratch for %lld atoms; the static scratch holds %zu bytes (about 65,000 atoms)",
             need, (long long)n_atoms, kStaticScratchBytes);
    fd3::set_error("fd3_neighbor_fill_static", msg);
    return FD3_EINVAL;
  }
  void* scratch = nullptr;
  rc = scratch_address(&scratch);
  if (rc) return rc;
  return fd3_neighbor_fill(n_atoms, d_pos_ang, h_cell_ang, r_cut_ang, scratch, kStaticScratchBytes, capacity, d_src,
                           d_dst, d_shift, h_count, stream);
}

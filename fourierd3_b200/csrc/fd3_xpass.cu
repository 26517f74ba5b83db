// Host side of the TMA fused x-pass: the tensor map over the float half spectrum and the
// dispatch on the x length.
#include <cudaTypedefs.h>

#include <mutex>

#include "fd3_xpass_impl.cuh"

namespace fd3 {

// cuTensorMapEncodeTiled from the driver (null when the driver does not export it).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// Whether the TMA x-pass can run this mesh with Q q values and RG ranks per unit: nx a tabulated
// length, at most 4 species, RG <= R, an even number of values per spectrum row block (the TMA
// strides must be multiples of 16 bytes) and two units in shared memory.
bool xpass_applies(const MeshGeom& mg, int Q, int RG) {
  if (mg.n[0] != 64 && mg.n[0] != 128 && mg.n[0] != 256) return false;
  if (mg.S > 4 || RG > mg.R || (RG != 1 && RG != 2 && RG != 4)) return false;
  if (Q != 4 && Q != 8 && Q != 16 && Q != 32) return false;
  const int qp = mg.qpitch > 0 ? mg.qpitch : mg.nzh;
  if ((((long long)mg.n[1] * qp) & 1) != 0) return false;
  if (mg.n[0] + mg.n[1] + mg.nzh > 1024) return false;   // the per-axis window's shared-memory slot
  // the x transform as N1 x N2 register DFTs (64: 8 x 8, 128: 8 x 16, 256: 16 x 16) and the
  // padded working copy of XpWork
  const int n1 = mg.n[0] == 64 ? 8 : mg.n[0] == 128 ? 8 : 16, n2 = mg.n[0] / n1;
  const size_t work = (size_t)mg.S * RG * n1 * (n2 * Q + (Q < 16 ? Q : 0)) * sizeof(float2);
  return xpass_stages((size_t)mg.S * RG * mg.n[0] * Q * sizeof(float2), work) >= 2;
}

// Spectrum (float2, layout (S, R, nx, ny, P), P = qpitch values per ky row) as a 4-D float
// tensor {2 ny P, nx, R, S}; box {2Q, nx, RG, S}: one unit of the x-pass.
int launch_xpass(const MeshGeom& mg, int Q, int RG, const CellInfo* ci, const GreenPairF* gpf, const float4* gtab,
                 const Tables* tab, const float* deconv, int spme, void* spec, double* part, int* n_blocks,
                 cudaStream_t s) {
  if (!xpass_applies(mg, Q, RG)) {
    set_error("filter", "the TMA x-pass does not apply to this mesh / pencil");
    return FD3_EINVAL;
  }
  auto fn = tensor_map_encoder();
  if (!fn) {
    set_error("filter", "cuTensorMapEncodeTiled is not available from the driver");
    return FD3_ECUDA;
  }
  const cuuint64_t inner = 2ull * mg.n[1] * (mg.qpitch > 0 ? mg.qpitch : mg.nzh);
  const cuuint64_t dims[4] = {inner, (cuuint64_t)mg.n[0], (cuuint64_t)mg.R, (cuuint64_t)mg.S};
  const cuuint64_t strides[3] = {inner * 4, inner * 4 * mg.n[0], inner * 4 * mg.n[0] * mg.R};
  const cuuint32_t box[4] = {(cuuint32_t)(2 * Q), (cuuint32_t)mg.n[0], (cuuint32_t)RG, (cuuint32_t)mg.S};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  CUtensorMap map;
  const CUresult r = fn(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, spec, dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("filter", "cuTensorMapEncodeTiled rejected the spectrum tensor map");
    return FD3_ECUDA;
  }
  XpassArgs a{&map, mg, ci, gpf, gtab, tab, deconv, spme, Q, RG, part, n_blocks, s};
  switch (mg.n[0]) {
    case 64: return launch_xpass_64(a);
    case 128: return launch_xpass_128(a);
    case 256: return launch_xpass_256(a);
    default: return FD3_EINVAL;
  }
}

}  // namespace fd3

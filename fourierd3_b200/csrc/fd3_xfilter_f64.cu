#include "fd3_xfilter_impl.cuh"
namespace fd3 {
template <>
int launch_xfilter<double>(const MeshGeom& mg, const CellInfo* ci, const GreenPair* gp, const GreenPairF* gpf,
                           const float4* gtab, const Tables* tab, const float* deconv, int spme, void* spec,
                           double* part, int* n_blocks, cudaStream_t s) {
  return launch_xfilter_t<double>(mg, ci, gp, gpf, gtab, tab, deconv, spme, spec, part, n_blocks, s);
}
}  // namespace fd3

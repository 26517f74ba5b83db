#include "fd3_xfilter_impl.cuh"
namespace fd3 {
template <>
int launch_xfilter<float>(const MeshGeom& mg, const CellInfo* ci, const GreenPair* gp, const GreenPairF* gpf,
                          const float4* gtab, const Tables* tab, const float* deconv, int spme, void* spec,
                          double* part, int* n_blocks, cudaStream_t s) {
  return launch_xfilter_t<float>(mg, ci, gp, gpf, gtab, tab, deconv, spme, spec, part, n_blocks, s);
}
int xfilter_pencil(const MeshGeom& mg, int is_double) {
  return is_double ? xfilter_kz<double>(mg) : xfilter_kz<float>(mg);
}
}  // namespace fd3

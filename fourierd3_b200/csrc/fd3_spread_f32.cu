// Explicit instantiation of the spread kernels for float32 (mixed precision) meshes (split for parallel compilation).
#include "fd3_mesh_impl.cuh"

namespace fd3 {
template int launch_spread<float>(const MeshGeom&, int, const double*, double, const int32_t*, const double*,
                                  const CellInfo*, const int*, const int*, const MeshRecords&, float*, cudaStream_t,
                                  int);
}  // namespace fd3

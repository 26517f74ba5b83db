// Explicit instantiation of the spread kernels for float64 meshes (split for parallel compilation).
#include "fd3_mesh_impl.cuh"

namespace fd3 {
template int launch_spread<double>(const MeshGeom&, int, const double*, double, const int32_t*, const double*,
                                  const CellInfo*, const int*, const int*, const MeshRecords&, double*, cudaStream_t,
                                  int);
}  // namespace fd3

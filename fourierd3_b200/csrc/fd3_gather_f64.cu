// Explicit instantiation of the gather kernels for float64 meshes (split for parallel compilation).
#include "fd3_mesh_impl.cuh"

namespace fd3 {
template int launch_gather<double>(const MeshGeom&, int, const double*, double, const int32_t*, const double*,
                                  const double*, const CellInfo*, const Tables*, const int*, const int*,
                                  const MeshRecords&, const double*, double*, double*, double*, int*, cudaStream_t);
}  // namespace fd3

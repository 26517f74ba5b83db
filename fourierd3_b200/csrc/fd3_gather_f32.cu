// Explicit instantiation of the gather kernels for float32 (mixed precision) meshes (split for parallel compilation).
#include "fd3_mesh_impl.cuh"

namespace fd3 {

// Whether the tile-staged gather can run this mesh: every channel row a multiple of 16 bytes
// (the TMA strides), at most eight ranks, the box (all ranks of one species) and its alignment
// pad within the shared-memory cap, box edges within the TMA limit of 256.
bool gather_tile_applies(const MeshGeom& mg, size_t elem) {
  if (mg.R < 1 || mg.R > 8 || (elem != 4 && elem != 8)) return false;
  if (((size_t)mg.n[2] * elem) % 16 != 0) return false;
  const GatherBox b = gather_box(mg, elem);
  if (b.x > 256 || b.y > 256 || b.z > 256) return false;
  return (size_t)mg.R * b.x * b.y * b.z * elem + 128 <= kTileGatherSmemCap;
}

template int launch_gather<float>(const MeshGeom&, int, const double*, double, const int32_t*, const double*,
                                  const double*, const CellInfo*, const Tables*, const int*, const int*,
                                  const MeshRecords&, const float*, double*, double*, double*, int*, cudaStream_t);
}  // namespace fd3

// TMA fused x-pass instantiations for nx = 64 (x transform as 8 x 8 register DFTs).
#include "fd3_xpass_impl.cuh"
namespace fd3 {
int launch_xpass_64(const XpassArgs& a) { return launch_xpass_nx<8, 8>(a); }
}  // namespace fd3

// TMA fused x-pass instantiations for nx = 256 (x transform as 16 x 16 register DFTs).
#include "fd3_xpass_impl.cuh"
namespace fd3 {
int launch_xpass_256(const XpassArgs& a) { return launch_xpass_nx<16, 16>(a); }
}  // namespace fd3

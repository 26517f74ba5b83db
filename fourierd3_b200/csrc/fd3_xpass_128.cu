// TMA fused x-pass instantiations for nx = 128 (x transform as 8 x 16 register DFTs).
#include "fd3_xpass_impl.cuh"
namespace fd3 {
int launch_xpass_128(const XpassArgs& a) { return launch_xpass_nx<8, 16>(a); }
}  // namespace fd3

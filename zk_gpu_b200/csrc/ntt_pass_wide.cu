// ntt_pass_wide.cu — launchers of the radix-2^7 .. 2^11 NTT passes, in a
// translation unit of their own (see ntt_tile.cuh and build.py).
#include "ntt_tile.cuh"

namespace zk {

cudaError_t launch_pass_wide(int B, const PassParams& pp, uint64_t ncta, cudaStream_t s) {
  switch (B) {
    case 7: return launch_pass<7>(pp, ncta, s);
    case 8: return launch_pass<8>(pp, ncta, s);
    case 9: return launch_pass<9>(pp, ncta, s);
    case 10: return launch_pass<10>(pp, ncta, s);
    case 11: return launch_pass<11>(pp, ncta, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace zk

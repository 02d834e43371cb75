// Stream kernel instantiations for block lists: tile variants 1-3 (2x8x16,
// 4x8x8, 8x4x8) of the RK4 stage with KO order 8 (R = 4) (stream_launch.h;
// variant 0 is the default tile).
#include "stream_kernel.cuh"
#include "stream_launch.h"

namespace bssn_host {

int launch_batch_r4(int mode, int variant, const bssn::Args& a, cudaStream_t st, int grid) {
  if (mode != bssn::MODE_STAGE) return fail(BSSN_B200_EINVAL, "stream kernel: no batched instantiation for this mode");
  switch (variant) {
    case 1: return launch_stream<4, bssn::MODE_STAGE, bssn::Shape<2, 8, 16>>(a, st, grid);
    case 2: return launch_stream<4, bssn::MODE_STAGE, bssn::Shape<4, 8, 8>>(a, st, grid);
    case 3: return launch_stream<4, bssn::MODE_STAGE, bssn::Shape<8, 4, 8>>(a, st, grid);
    default: return fail(BSSN_B200_EINVAL, "variant out of range");
  }
}

}  // namespace bssn_host

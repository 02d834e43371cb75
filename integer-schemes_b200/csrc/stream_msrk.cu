// Stream kernel instantiations: the fused MSRK stage on the default tile
// (stream_launch.h), Kreiss-Oliger order 6 (R = 3) and 8 (R = 4).
#include "stream_kernel.cuh"
#include "stream_launch.h"

namespace bssn_host {

int launch_msrk_modes(int R, int mode, const bssn::Args& a, cudaStream_t st, int grid) {
  if (mode == bssn::MODE_MSRK) {
    if (R == 3) return launch_stream<3, bssn::MODE_MSRK>(a, st, grid);
    if (R == 4) return launch_stream<4, bssn::MODE_MSRK>(a, st, grid);
  }
  return fail(BSSN_B200_EINVAL, "stream kernel: no MSRK instantiation for this order/mode");
}

int copy_errors_msrk(int* count) { return read_copy_errors(count); }

}  // namespace bssn_host

// Stream kernel instantiations: RHS, constraints and constraint norms on the
// default tile (stream_launch.h).
#include "stream_kernel.cuh"
#include "stream_launch.h"

namespace bssn_host {

int launch_rhs_modes(int R, int mode, const bssn::Args& a, cudaStream_t st, int grid) {
  if (R == 3) {
    switch (mode) {
      case bssn::MODE_RHS: return launch_stream<3, bssn::MODE_RHS>(a, st, grid);
      case bssn::MODE_CON: return launch_stream<3, bssn::MODE_CON>(a, st, grid);
      case bssn::MODE_NORM: return launch_stream<3, bssn::MODE_NORM>(a, st, grid);
      default: break;
    }
  }
  return fail(BSSN_B200_EINVAL, "stream kernel: no RHS-mode instantiation for this order/mode");
}

int copy_errors_rhs(int* count) { return read_copy_errors(count); }

}  // namespace bssn_host

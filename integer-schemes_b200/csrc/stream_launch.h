// Launch entry points of the stream kernel instantiations. Each stream_*.cu
// translation unit instantiates one group, so the groups compile in parallel:
//   stream_rhs.cu     MODE_RHS, MODE_CON, MODE_NORM   (R = 3)   default tile
//   stream_stage.cu   MODE_STAGE                      (R = 3, 4) default tile
//   stream_msrk.cu    MODE_MSRK                       (R = 3, 4) default tile
//   stream_batch3.cu  MODE_RHS, MODE_STAGE            (R = 3)   tile variants 1-3
//   stream_batch4.cu  MODE_STAGE                      (R = 4)   tile variants 1-3
// The default tile (variant 0) serves both single grids and block lists.
#pragma once

#include <cuda_runtime.h>

namespace bssn {
struct Args;
}

namespace bssn_host {

int launch_rhs_modes(int R, int mode, const bssn::Args& a, cudaStream_t st, int grid);
int launch_stage_modes(int R, int mode, const bssn::Args& a, cudaStream_t st, int grid);
int launch_msrk_modes(int R, int mode, const bssn::Args& a, cudaStream_t st, int grid);
int launch_batch_r3(int mode, int variant, const bssn::Args& a, cudaStream_t st, int grid);
int launch_batch_r4(int mode, int variant, const bssn::Args& a, cudaStream_t st, int grid);
int copy_errors_rhs(int* count);
int copy_errors_stage(int* count);
int copy_errors_msrk(int* count);

}  // namespace bssn_host

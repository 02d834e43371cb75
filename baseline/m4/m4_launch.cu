// Launcher for the reference's M4 fused BSSN RHS kernel, baseline use only.
//
// The kernel body is not in this repository: build_m4.py generates it with
// the reference's own generator (3D/src/bssn3d/cuda/gen_fused.py) into
// baseline/_ref/m4/_bssn_fused_kernel.cuh and compiles this file against it
// for sm_100a. This file replaces the reference's XLA FFI handler FusedImpl
// (3D/src/bssn3d/cuda/rhs_fused.cu:22-53) with a plain C entry point that
// launches the kernel the same way: one thread per point of the padded grid,
// blocks of 128 threads (its BSSN_FUSED_BLOCK default), no shared memory
// (NSMEM = 0), dummy_iters = 0.
//
// bench.py times it beside this project's fused kernel on the same state; it
// is never called by the library.
#include <cuda_runtime.h>

#include "_bssn_fused_kernel.cuh"

extern "C" {

// 0 on success, else the cudaError_t of the launch.
int m4_rhs(void* stream, const double* F, const double* S, double* OUT, int Sx, int Sy, int Sz, int block) {
  if (block <= 0) block = 128;
  const long long n = (long long)Sx * Sy * Sz;
  const unsigned grid = (unsigned)((n + block - 1) / block);
  bssn_rhs_fused<<<grid, block, 0, static_cast<cudaStream_t>(stream)>>>(F, S, OUT, Sx, Sy, Sz, 0);
  return (int)cudaGetLastError();
}

// Registers and local-memory (spill) bytes per thread of the compiled kernel.
int m4_attributes(int* regs, int* local_bytes) {
  cudaFuncAttributes a;
  const cudaError_t e = cudaFuncGetAttributes(&a, bssn_rhs_fused);
  if (e != cudaSuccess) return (int)e;
  *regs = a.numRegs;
  *local_bytes = (int)a.localSizeBytes;
  return 0;
}

int m4_nf(void) { return NF; }
int m4_nscal(void) { return NSCAL; }

}  // extern "C"

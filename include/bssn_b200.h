/*
 * bssn_b200 — C ABI of the B200 (sm_100a) BSSN right-hand side and RK4 stage
 * update. Plain pointers and sizes only; every entry point returns 0 on
 * success or a BSSN_B200_E* status, with a message in bssn_b200_last_error().
 *
 * Array conventions (all float64, C order, z contiguous, device memory unless
 * stated otherwise):
 *   state / RHS   (24, Sx, Sy, Sz) in the state order of
 *                 3D/src/bssn3d/state.py:37-46: alpha, chi, K, gt0..5,
 *                 beta0..2, At0..5, Gt0..2, B0..2
 *   S             16 scalars, the pack of 3D/src/bssn3d/fused_rhs_cuda.py:52-55:
 *                 eta, cahd_c, dt, dx, ssl_h, ssl_sigma, t, lambda0..3,
 *                 lambda_f0..1, dx, dy, dz  (device memory, like the
 *                 reference's FFI operand)
 *   derivatives   (138 [+24], Sx, Sy, Sz): 72 first derivatives at 3*f+axis,
 *                 then 66 second derivatives at 72 + 6*m + p for the fields
 *                 m = alpha, chi, gt0..5, beta0..2 and the pairs
 *                 p = 00,01,02,11,12,22 [then 24 Kreiss-Oliger sums]
 *
 * The finite-difference order is 6 (reach 3); Kreiss-Oliger order is 6 or 8.
 * Stencils are evaluated on every point of the padded array with the index
 * clamped at the array ends, like 3D/src/bssn3d/derivative_bundle.py:31-48.
 *
 * Scratch: the fused kernels stage derivatives in a caller-provided device
 * buffer of bssn_b200_scratch_bytes() bytes (no allocation inside). Calls
 * that share one scratch buffer must be ordered on one stream.
 */
#ifndef BSSN_B200_H
#define BSSN_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BSSN_B200_OK 0
#define BSSN_B200_EINVAL 1   /* bad shape, pointer, order or stage */
#define BSSN_B200_ESCRATCH 2 /* scratch buffer missing or too small */
#define BSSN_B200_ECUDA 3    /* a CUDA call or launch failed */

/* Message for the last non-zero status returned on this host thread. */
const char* bssn_b200_last_error(void);

/* Library version, e.g. "bssn_b200 0.1 sm_100a". */
const char* bssn_b200_version(void);

/* Bytes of device scratch the fused kernels need on the current device.
 * Independent of the grid shape (the kernels are persistent); ko_order 6 or 8. */
size_t bssn_b200_scratch_bytes(int ko_order);

/* The BSSN right-hand side: OUT = RHS(F) on every point of the padded grid.
 * Drop-in for the reference's fused FFI handler FusedImpl
 * (3D/src/bssn3d/cuda/rhs_fused.cu:22-53, bound as `Fused` at :55-61):
 * same operands F (24,Sx,Sy,Sz), S (16,), OUT (24,Sx,Sy,Sz), same stream
 * semantics (enqueue only, no host sync), same errors for a bad F shape or
 * scalar count. `stream` is a cudaStream_t (NULL = legacy default stream). */
int bssn_b200_rhs(void* stream, const double* F, const double* S, double* OUT,
                  long long Sx, long long Sy, long long Sz, void* scratch,
                  size_t scratch_bytes);

/* One RK4 stage of BSSNEvolution.step (3D/src/bssn3d/evolve.py:125-137) with
 * the Kreiss-Oliger pass of evolve.py:76-84 and, after stage 3, the
 * enforcement of evolve.py:93-119, fused into the RHS kernel:
 *   rate = RHS(Y at t + c_s*dt) + KO(Y)             c = 0, 1/2, 1/2, 1
 *   stage 0: ACC = rate;          YNEXT = U + (dt/2)*rate
 *   stage 1: ACC = ACC + 2*rate;  YNEXT = U + (dt/2)*rate
 *   stage 2: ACC = ACC + 2*rate;  YNEXT = U + dt*rate
 *   stage 3: YNEXT = enforce(U + (dt/6)*(ACC + rate))
 * S[2] = dt and S[6] = t, the step's start time. ko_sigma <= 0 disables KO.
 * YNEXT must not alias Y (other tiles still read Y's halo); it may alias U
 * at stage 3. Y may alias U at stage 0. */
int bssn_b200_rk4_stage(void* stream, int stage, const double* U, const double* Y,
                        double* ACC, double* YNEXT, const double* S, double ko_sigma,
                        int ko_order, double chi_floor, double alpha_floor,
                        long long Sx, long long Sy, long long Sz, void* scratch,
                        size_t scratch_bytes);

/* The 138 derivatives of F (and, when ko_sigma > 0, the 24 Kreiss-Oliger sums
 * after them) into DOUT (138 or 162, Sx, Sy, Sz): the derivative bundle of
 * 3D/src/bssn3d/derivative_bundle.py:31-48 / 3D/src/bssn3d/deriv_kernel.py. */
int bssn_b200_derivatives(void* stream, const double* F, const double* S,
                          double* DOUT, double ko_sigma, int ko_order, long long Sx,
                          long long Sy, long long Sz);

/* S[6] <- S[6] + S[2] on the device: advances the step start time t by dt
 * between RK4 steps without a host round trip, so a captured step graph can
 * be replayed (the time carry of 3D/src/bssn3d/evolve.py:186-193). */
int bssn_b200_advance_time(void* stream, double* S);

/* The pointwise algebra alone, with the 138 derivatives supplied in D
 * (138, npts): the algebra-only interface of the reference's
 * 3D/src/bssn3d/cuda/microbench_algebra.cu / gen_algebra_cuda.py:55-96.
 * F (24, npts), OUT (24, npts). */
int bssn_b200_rhs_algebra(void* stream, const double* F, const double* D,
                          const double* S, double* OUT, long long npts);

/* Algebraic enforcement in place (3D/src/bssn3d/evolve.py:93-119). */
int bssn_b200_enforce(void* stream, double* U, long long npts, double chi_floor,
                      double alpha_floor);

/* Periodic ghost sync in place (3D/src/bssn3d/evolve.py:65-73). */
int bssn_b200_periodic_sync(void* stream, double* U, long long Sx, long long Sy,
                            long long Sz, int ng);

#ifdef __cplusplus
}
#endif

#endif /* BSSN_B200_H */

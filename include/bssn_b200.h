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
 * Ownership: the caller owns every buffer. No entry point allocates or frees
 * device memory or synchronises the stream; kernels are only enqueued.
 */
#ifndef BSSN_B200_H
#define BSSN_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One block of a batched (AMR) block list. Blocks are stored back to back in
 * one pooled buffer: block b's field f starts at double offset + f*sx*sy*sz
 * and is a C-order (sx, sy, sz) array, the single-grid layout repeated. */
typedef struct bssn_b200_block {
  long long offset; /* first double of the block in the pooled state */
  int sx, sy, sz;   /* padded extents (ghosts included) */
  int tile0;        /* first tile of the block, filled by bssn_b200_batch_plan */
  double h[3];      /* grid spacing dx, dy, dz */
  int core;         /* ghost layers the batched kernels leave alone: tiles cover
                       [core, s - core) on each axis (0 = the whole array; set it
                       to the ghost width when bssn_b200_fill supplies the ghosts) */
  int reserved;     /* 0 */
} bssn_b200_block;

/* One box of a ghost-fill plan (bssn_b200_fill). Every destination point
 * d = (x, y, z) of the half-open box [lo, hi) in block `dst` (local indices
 * of its padded array) receives all 24 fields from block `src`:
 *   BSSN_B200_FILL_COPY      src[d + shift]          same-level copy
 *   BSSN_B200_FILL_RESTRICT  src[2 d + shift]        fine-to-coarse injection
 *   BSSN_B200_FILL_PROLONG   node-centred 2:1 prolongation from the coarser
 *       block src: per axis g = d + shift is the point's index on the refined
 *       src lattice; even g copies src node g/2, odd g takes the 6-point
 *       midpoint Lagrange stencil on src nodes (g-1)/2 - 2 ... (g-1)/2 + 3,
 *       indices clamped to the src array (its edge padding); applied x, then
 *       y, then z like the reference's sequential passes
 *       (3D/src/multipatch/amr/kernels.py:52-71,76-102).
 * Offsets and shapes are those of the block pool (bssn_b200_block). */
#define BSSN_B200_FILL_COPY 0
#define BSSN_B200_FILL_RESTRICT 1
#define BSSN_B200_FILL_PROLONG 2

typedef struct bssn_b200_fill_op {
  long long dst_off, src_off; /* first double of each block in the pool */
  long long point0;           /* first point of the box in the launch, set by bssn_b200_fill_plan */
  int dst_s[3], src_s[3];     /* padded extents of the two blocks */
  int lo[3], hi[3];           /* destination box, half-open, dst-local */
  int shift[3];               /* index map (see above) */
  int kind;                   /* BSSN_B200_FILL_* */
} bssn_b200_fill_op;

/* Tile-shape variants of the batched kernels (the autotuner's search space):
 * 0 = 4x4x16, 1 = 2x8x16, 2 = 4x8x8, 3 = 8x4x8 points (x, y, z). */
#define BSSN_B200_NVARIANTS 4

#define BSSN_B200_OK 0
#define BSSN_B200_EINVAL 1   /* bad shape, pointer, order or stage */
#define BSSN_B200_ECUDA 3    /* a CUDA call or launch failed */

/* Message for the last non-zero status returned on this host thread. */
const char* bssn_b200_last_error(void);

/* Library version, e.g. "bssn_b200 0.3 sm_100a". */
const char* bssn_b200_version(void);

/* Number of bulk-copy waits that gave up since the library was loaded on the
 * current device (synchronises the device). The stream kernel stages halo
 * tiles with bulk-tensor copies completing on an mbarrier; each wait is
 * bounded, and a wait that runs out is counted here (that launch's results
 * are invalid) instead of hanging the GPU. 0 in a healthy run. */
int bssn_b200_async_copy_errors(int* count);

/* The BSSN right-hand side: OUT = RHS(F) on every point of the padded grid.
 * Drop-in for the reference's fused FFI handler FusedImpl
 * (3D/src/bssn3d/cuda/rhs_fused.cu:22-53, bound as `Fused` at :55-61):
 * same operands F (24,Sx,Sy,Sz), S (16,), OUT (24,Sx,Sy,Sz), same stream
 * semantics (enqueue only, no host sync), same errors for a bad F shape or
 * scalar count. `stream` is a cudaStream_t (NULL = legacy default stream). */
int bssn_b200_rhs(void* stream, const double* F, const double* S, double* OUT,
                  long long Sx, long long Sy, long long Sz);

/* Hamiltonian and momentum constraints of F into OUT (4, Sx, Sy, Sz) = H, M0,
 * M1, M2, with the definitions of the reference's ConstraintSolver
 * (3D/src/bssn3d/constraints.py:38-51, Dendro-GR physcon.cpp) on the same
 * 6th-order derivatives; S supplies dx, dy, dz (S[13..15]). */
int bssn_b200_constraints(void* stream, const double* F, const double* S, double* OUT,
                          long long Sx, long long Sy, long long Sz);

/* Device scratch (bytes) bssn_b200_constraint_norms needs on the current
 * device: one pair of partial sums per CTA of its persistent grid. */
size_t bssn_b200_norms_scratch_bytes(void);

/* Interior L2 norms of the constraints, ConstraintSolver.l2
 * (3D/src/bssn3d/constraints.py:53-62): OUT2[0] = sqrt(mean(H^2)),
 * OUT2[1] = sqrt(mean(M0^2 + M1^2 + M2^2)) over [ng, S-ng)^3, written to
 * device memory without materialising H or M. One fused launch accumulates
 * per-CTA partial sums in `scratch` (caller-provided, at least
 * bssn_b200_norms_scratch_bytes()), a second launch adds them in a fixed
 * order, so the result is bit-reproducible run to run. */
int bssn_b200_constraint_norms(void* stream, const double* F, const double* S, long long Sx,
                               long long Sy, long long Sz, int ng, double* scratch,
                               size_t scratch_bytes, double* OUT2);

/* Host-side plan of a block list for tile variant `variant`: fills each
 * block's tile0 (prefix of tile counts) in the HOST table and returns the
 * total tile count, or -1 (with bssn_b200_last_error) on a bad table. Upload
 * the filled table to the device for the batched calls below. */
int bssn_b200_batch_plan(bssn_b200_block* host_blocks, int nblocks, int variant);

/* Batched forms of bssn_b200_rhs / bssn_b200_rk4_stage over a block list:
 * ONE persistent launch covers every block (one CTA per SM walking the global
 * tile list); each block is differentiated on its own padded array with its
 * own spacing h (S[13..15] and S[3] are taken from the block, the other
 * scalars from S). `blocks` is the planned table in DEVICE memory, `ntiles`
 * the value bssn_b200_batch_plan returned for the same variant. The pooled
 * buffers share the table's offsets. No 3D/src/bssn3d counterpart: the
 * reference has no BSSN AMR (3D/src/mcs3d/amr/__init__.py:1); the block pool
 * follows the 2D MCS AMR block pools (2D/src/mcs2d/amr/state.py:77). */
int bssn_b200_batch_rhs(void* stream, const double* F, const double* S, double* OUT,
                        const bssn_b200_block* blocks, int nblocks, int ntiles, int variant);
int bssn_b200_batch_rk4_stage(void* stream, int stage, const double* U, const double* Y,
                              double* ACC, double* YNEXT, const double* S, double ko_sigma,
                              int ko_order, double chi_floor, double alpha_floor,
                              const bssn_b200_block* blocks, int nblocks, int ntiles,
                              int variant);

/* Validates a ghost-fill plan held in HOST memory against a pool of
 * `pool_doubles` doubles (every box inside its destination array, every
 * copied or injected source point inside its source array, no block past the
 * pool's end), orders the boxes copies and injections first, prolongations
 * after (stable; boxes of one list are disjoint, so the order is free), fills
 * each op's point0 with the prefix of box volumes and returns the total point
 * count, or -1 (with bssn_b200_last_error). Upload the filled table for
 * bssn_b200_fill. */
long long bssn_b200_fill_plan(bssn_b200_fill_op* host_ops, int nops, long long pool_doubles);

/* Executes one planned list of fill boxes on `pool` (one launch, one thread
 * per destination point, 24 fields each). `ops` is the table in DEVICE
 * memory, `npoints` the value bssn_b200_fill_plan returned for it, `wmid`
 * (HOST, 6 doubles) the midpoint Lagrange weights for offsets -2..3 at +1/2.
 * The boxes of one list must be disjoint and must not write what another box
 * of the list reads: a same-level list writes ghosts and reads interiors,
 * and a prolongation list reads a coarser level that is complete before it
 * runs. No 3D/src/bssn3d counterpart (the reference has no BSSN AMR); the
 * operators are those of 3D/src/multipatch/amr/kernels.py and sync.py. */
int bssn_b200_fill(void* stream, double* pool, const bssn_b200_fill_op* ops, int nops,
                   long long npoints, const double* wmid);

/* The constraint norms of bssn_b200_constraint_norms for callers that cannot
 * allocate device memory: an XLA FFI handler (XLA owns every device buffer it
 * hands over and gives the handler no allocation of its own outside its
 * scratch protocol), a plugin running inside a host's stream capture (where
 * cudaMalloc would break the capture), or a loop under a no-allocation rule.
 * The partial sums live in a file-scope static __device__ array sized for 256
 * CTAs (4 KB, held on every GPU that loads the library until exit); the
 * persistent grid uses min(tiles, SMs) CTAs, so any grid fits on GPUs with up
 * to 256 SMs and a launch that would need more slots is rejected with
 * BSSN_B200_EINVAL. Inputs and outputs are still the caller's. The first call
 * on a device resolves the array's device address with cudaGetSymbolAddress,
 * so make that first call before any stream capture. The address is kept per
 * device for the life of the process: after cudaDeviceReset the library must
 * be reloaded before this entry point is called again. All calls share the
 * array (each call overwrites the slots it reads, so nothing needs clearing):
 * calls that overlap on the GPU — on two streams, or from two host threads —
 * race. No counterpart in the reference. */
int bssn_b200_constraint_norms_static(void* stream, const double* F, const double* S,
                                      long long Sx, long long Sy, long long Sz, int ng,
                                      double* OUT2);

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
 * at stage 3. Y may alias U at stage 0. ACC aliases nothing. */
int bssn_b200_rk4_stage(void* stream, int stage, const double* U, const double* Y,
                        double* ACC, double* YNEXT, const double* S, double ko_sigma,
                        int ko_order, double chi_floor, double alpha_floor,
                        long long Sx, long long Sy, long long Sz);

/* One stage of the 2-step / 3-stage MSRK step, BSSNEvolution._msrk2_step
 * (3D/src/bssn3d/evolve.py:139-153), with KO and, after stage 2, enforcement
 * fused in as for bssn_b200_rk4_stage. coef (HOST, 9 doubles) =
 * {a20, a21, a30, a31, a32, b0, b1, b2, b3}; node times are t, t + c2*dt,
 * t + c3*dt with c2 = a20 + a21, c3 = a30 + a31 + a32.
 *   rate = RHS(Y at the node time) + KO(Y)
 *   stage 0 (Y = U = y_n, ACC = k0 = f(y_{n-1})):
 *     OUT = Y2 = U + dt*(a20*k0 + a21*rate)
 *     OUT2 = U + dt*(a30*k0 + a31*rate)         (partial Y3)
 *     OUT3 = U + dt*(b0*k0 + b1*rate)           (partial y_{n+1})
 *     ACC = rate                                (k1: the next step's k0)
 *   stage 1 (Y = Y2, U = partial Y3, ACC = partial y_{n+1}):
 *     OUT = Y3 = U + dt*a32*rate;   ACC = ACC + dt*b2*rate
 *   stage 2 (Y = Y3, U = partial y_{n+1}):
 *     OUT = y_{n+1} = enforce(U + dt*b3*rate)
 * S[2] = dt and S[6] = t, the step's start time. Y is read with its stencil
 * halo, so no output may alias it; the other operands are read only at the
 * point they are written, so OUT may alias U at stages 1 and 2 and ACC is
 * updated in place. Stage-0 outputs are distinct from each other and from U. */
int bssn_b200_msrk_stage(void* stream, int stage, const double* U, const double* Y,
                         double* ACC, double* OUT, double* OUT2, double* OUT3,
                         const double* S, const double* coef, double ko_sigma, int ko_order,
                         double chi_floor, double alpha_floor, long long Sx, long long Sy,
                         long long Sz);

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

/* ---- Ozaki INT8 derivative path (tcgen05 tensor cores) -------------------
 * The 138 derivatives (+24 KO sums when ko_sigma > 0) of F into DOUT, like
 * bssn_b200_derivatives, but every stencil is applied as an exact INT8 x INT8
 * -> INT32 tensor-core contraction of k INT8 digit planes (k = 1..8, one
 * power-of-two exponent per line along the differentiation axis), recombined
 * in float64. Mixed second derivatives take the first derivative along the
 * lower axis through the same path twice. Bit-reproducible run to run.
 * The reference has no BSSN Ozaki path; its MCS Ozaki derivative
 * (2D/src/mcs2d/schemes/ozaki.py:257-380) is the design source.
 * Workspace: caller-provided device memory of bssn_b200_ozaki_workspace_bytes
 * bytes, 256-byte aligned; a device int at bssn_b200_ozaki_error_flag() is set
 * to 1 if a tensor-core wait gave up (read it after the stream completes).
 * Errors: bssn_b200_ozaki_last_error(). */
size_t bssn_b200_ozaki_workspace_bytes(long long Sx, long long Sy, long long Sz, int k);
int* bssn_b200_ozaki_error_flag(void* workspace, long long Sx, long long Sy, long long Sz, int k);
const char* bssn_b200_ozaki_last_error(void);
int bssn_b200_ozaki_derivatives(void* stream, const double* F, const double* S, double* DOUT, int k,
                                double ko_sigma, int ko_order, long long Sx, long long Sy,
                                long long Sz, void* workspace, size_t workspace_bytes);

/* Block-list form of the Ozaki path. Derivatives live in a slot pool D:
 * nslot = 162 doubles per point with KO (ko_sigma > 0), else 138; slot s of
 * block b starts at D + (offset_b / 24) * nslot + s * n_b, n_b = sx*sy*sz
 * (the state pool's layout with nslot fields). Each block is differentiated
 * on its own padded array with its own spacing; with core > 0 only the
 * derivatives at [core, s - core)^3 are valid (the passes cover that box,
 * plus the 3-point margins the mixed derivatives read).
 *
 * bssn_b200_batch_ozaki_plan: HOST tables in, HOST tables out. Fills
 * host_tile0 (5 * nblocks ints: first tile of each block for each of the
 * bundle's 5 pass kinds), host_ntiles (5 totals) and host_pts0 (nblocks
 * prefix counts of covered points, for bssn_b200_batch_rk4_stage_derivs) and
 * returns the covered point total, or -1 (bssn_b200_ozaki_last_error).
 * Upload host_tile0 and host_pts0 to the device; pass host_ntiles as is.
 * The workspace of the batched call is 256 bytes (the error flag at its start).
 *
 * bssn_b200_batch_rk4_stage_derivs: one RK4 stage (the update of
 * bssn_b200_batch_rk4_stage) at the covered points from the derivatives in D
 * (KO sums from D when ko_slots != 0), one thread per point. Errors:
 * bssn_b200_last_error. No reference counterpart (the reference has neither
 * BSSN AMR nor a BSSN Ozaki path). */
long long bssn_b200_batch_ozaki_plan(const bssn_b200_block* host_blocks, int nblocks, int* host_tile0,
                                     long long* host_ntiles, long long* host_pts0);
int bssn_b200_batch_ozaki_derivatives(void* stream, const double* F, const double* S, double* D, int k,
                                      double ko_sigma, int ko_order, const bssn_b200_block* blocks,
                                      int nblocks, const int* tile0, const long long* host_ntiles,
                                      void* workspace, size_t workspace_bytes);
int bssn_b200_batch_rk4_stage_derivs(void* stream, int stage, const double* U, const double* Y,
                                     double* ACC, double* YNEXT, const double* D, const double* S,
                                     int ko_slots, double chi_floor, double alpha_floor,
                                     const bssn_b200_block* blocks, int nblocks,
                                     const long long* pts0, long long npoints);

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

// bssn_b200 — fused BSSN right-hand side and RK4 stage kernels for sm_100a,
// behind the C ABI of include/bssn_b200.h.
//
// One persistent kernel per RHS evaluation (stream_kernel). Each 256-thread CTA
// takes 4x4x16-point tiles of the padded grid in turn, one point per thread.
// Per tile it walks the 24 fields in the order of stream.cuh: cp.async stages
// the field's haloed tile in shared memory (double-buffered, the next field
// streams in while this one is differentiated), every thread takes its
// point's axial taps once and forms the first derivative, the diagonal second
// derivative and the Kreiss-Oliger term from them, the mixed second
// derivatives come out of two separable passes through shared memory, and the
// result is consumed at once by the point's BSSN accumulators (bssn::Stream).
// No derivative is written anywhere. The epilogue stores the RHS, performs the
// RK4 stage update (algebraic enforcement fused into stage 3) or stores the
// constraints.
//
// Stencils follow 3D/src/bssn3d/derivative_bundle.py:31-48 and
// common/src/mcs_common/derivatives.py:35-106: the centred sixth-order
// coefficients (integer sums of paired taps, scaled once), index clamped at
// the array ends, mixed second derivatives as a first derivative along the
// lower axis, then along the higher axis of that result.
//
// This header holds the stream kernel template and its host launch template;
// its instantiations are spread over the stream_*.cu translation units
// (declared in stream_launch.h) so that the library compiles in parallel.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <string>
#include <type_traits>

#include "../../include/bssn_b200.h"
#include "host_util.h"
#include "stream.cuh"

namespace bssn {

constexpr int NTHREADS = 256;  // one point per thread, 256-point tiles

// A tile shape X x Y x Z (Z along the contiguous axis, X*Y*Z = 256).
template <int X_, int Y_, int Z_>
struct Shape {
  static constexpr int X = X_, Y = Y_, Z = Z_;
  static_assert(X_ * Y_ * Z_ == NTHREADS, "one point per thread");
  static_assert(Z_ >= 8 && (Z_ & (Z_ - 1)) == 0 && (Y_ & (Y_ - 1)) == 0, "power-of-two tile");
};
using DefaultShape = Shape<4, 4, 16>;

// z pitch of staged rows: >= the row length and 8 mod 16 doubles, so the
// 16 threads of a half-warp (one or two z rows) hit 16 distinct bank pairs.
__host__ __device__ constexpr int zpitch(int len) { return len <= 8 ? 8 : ((len - 8 + 15) / 16) * 16 + 8; }

enum Mode : int { MODE_DERIV = 0, MODE_RHS = 1, MODE_STAGE = 2, MODE_CON = 3, MODE_NORM = 4, MODE_MSRK = 5 };

struct Args {
  const double* F;  // stage input (24, n)
  const double* U;  // u_n (stage mode)
  double* ACC;      // accumulator (stage mode)
  double* OUT;      // RHS | next stage / new state | derivatives | constraints
  const double* S;  // 16 scalars (device)
  long long Sx, Sy, Sz, n;
  int ntx, nty, ntz;
  int stage;
  int use_ko;
  double ko_sigma;
  double chi_floor, alpha_floor;
  int ng;             // norm mode: ghost width of the interior
  double* partials;   // norm mode: [gridDim.x][2] per-CTA sums (scratch)
  const bssn_b200_block* blocks;  // batched mode: block table (device), else NULL
  int nblocks;
  int ntiles;         // batched mode: total tiles over all blocks
  double* OUT2;       // MSRK stage 0: partial Y3
  double* OUT3;       // MSRK stage 0: partial y_{n+1}
  double coef[9];     // MSRK: a20, a21, a30, a31, a32, b0, b1, b2, b3
  double ctime;       // MSRK: this stage's node (stage time t + ctime * dt)
};

// Stencil scale factors, set on the device from the grid spacing (per block
// for block lists). Every stencil is summed with the integer coefficients of
// common/src/mcs_common/derivatives.py:35-49 and scaled once:
//   f1 = 1 / (60 h)           first derivative
//   f2 = 1 / (180 h h)        diagonal second derivative
//   fk = sigma / (64 h)       Kreiss-Oliger, order 6 (sigma / (256 h) for order 8)
//   fm = f1_i * f1_j          mixed second derivative, pairs xy, xz, yz
struct Weights {
  double f1[3], f2[3], fk[3], fm[3];
};

// Stencil sums. The symmetric taps are paired first (v[+k] - v[-k] for the
// first derivative, v[+k] + v[-k] for the even stencils; the KO sum shares
// the second derivative's pairs), then combined with the integer coefficients
// from the outermost pair inwards, each step one fused multiply-add; the
// caller applies the scale factor. The reference forms sum_k (c_k / den *
// factor) * v_k (derivatives.py:78-88); the two orders differ by rounding
// only. The CPU oracle evaluates the same operations in the same order, so
// the derivatives match it bit for bit. v points at the centre tap, st is the
// tap stride.
__device__ __forceinline__ double c1_sum(double m3, double m2, double m1, double p1, double p2, double p3) {
  const double a1 = __dsub_rn(p1, m1), a2 = __dsub_rn(p2, m2), a3 = __dsub_rn(p3, m3);
  return __fma_rn(45.0, a1, __fma_rn(-9.0, a2, a3));
}
__device__ __forceinline__ double c2_sum(double v0, double s1, double s2, double s3) {
  return __fma_rn(-490.0, v0, __fma_rn(270.0, s1, __fma_rn(-27.0, s2, __dadd_rn(s3, s3))));
}
__device__ __forceinline__ double ko6_sum(double v0, double s1, double s2, double s3) {
  return __fma_rn(-20.0, v0, __fma_rn(15.0, s1, __fma_rn(-6.0, s2, s3)));
}
__device__ __forceinline__ double ko8_sum(double v0, double s1, double s2, double s3, double s4) {
  return __fma_rn(-70.0, v0, __fma_rn(56.0, s1, __fma_rn(-28.0, s2, __fma_rn(8.0, s3, -s4))));
}
// first-derivative sum of the 7 taps around p (stride st)
__device__ __forceinline__ double c1_at(const double* p, int st) {
  return c1_sum(p[-3 * st], p[-2 * st], p[-st], p[st], p[2 * st], p[3 * st]);
}

__device__ __forceinline__ long long clampll(long long v, long long hi) {
  return v < 0 ? 0 : (v > hi ? hi : v);
}

__device__ __forceinline__ void cp_async8(double* smem, const double* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// --- bulk-tensor (TMA) loads completing on an mbarrier ----------------------
__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Orders this thread's earlier shared-memory accesses before later async-proxy
// (bulk copy) writes to the same memory.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
// One 4-D tile of the tensor map into shared memory (this CTA only; no multicast).
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, unsigned long long* bar, int c0,
                                            int c1, int c2, int c3) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
      "%5}], [%6];\n" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_addr(bar))
      : "memory");
}
// Bounded wait on an mbarrier phase: gives up after kWaitLimit polls and
// records the failure in g_async_copy_errors instead of spinning forever.
constexpr long long kWaitLimit = 1LL << 24;
// One counter per translation unit that instantiates the stream kernel; the
// C ABI sums them (bssn_host::stream_copy_errors).
static __device__ int g_async_copy_errors = 0;
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity) {
  for (long long it = 0; it < kWaitLimit; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  atomicAdd(&g_async_copy_errors, 1);
  return false;
}

// Compile-time loop: body(std::integral_constant<int, I>) for I = B .. E-1, so
// that every per-field branch and register-array index is resolved statically.
template <int B, int E>
struct Unroll {
  template <class Body>
  __device__ __forceinline__ static void run(Body&& body) {
    body(std::integral_constant<int, B>{});
    Unroll<B + 1, E>::run(body);
  }
};
template <int E>
struct Unroll<E, E> {
  template <class Body>
  __device__ __forceinline__ static void run(Body&&) {}
};

template <int R, class T = DefaultShape>
struct TileGeom {
  static constexpr int TX = T::X, TY = T::Y, TZ = T::Z;
  static constexpr int HX = TX + 2 * R, HY = TY + 2 * R, HZ = TZ + 2 * R;
  static constexpr int HZP = zpitch(HZ);
  // With bulk-copy staging a staged row starts ZS_TMA points further down in z
  // (z0 - R - ZS_TMA), so that the copy starts on a 16-byte boundary when z0 is
  // even; the copy moves BOXZ points per row (a multiple of 2 doubles).
  static constexpr int ZS_TMA = R & 1;
  static constexpr int BOXZ = (HZ + ZS_TMA + 1) / 2 * 2;
  static_assert(BOXZ <= HZP, "a bulk-copied row must fit the staged z pitch");
  static constexpr unsigned TMA_BYTES = (unsigned)(BOXZ * HY * HX * sizeof(double));
  static constexpr int SX = HY * HZP, SY = HZP;
  static constexpr int VOL = HX * HY * HZP;   // doubles per staged buffer
  static constexpr int HZS = HZ;             // staged row length (full 24-wide rows measured 1.5 % slower)
  static constexpr int NELEM = HX * HY * HZS;  // staged elements
  static constexpr int PER_THREAD = (NELEM + NTHREADS - 1) / NTHREADS;
  // separable mixed-derivative passes
  static constexpr int TP = zpitch(TZ + 6);                       // z pitch of T1/T2
  // The T1/T2 passes walk rows of TROW points (the TZ + 6 needed, padded) so
  // that 16 consecutive threads touch 16 consecutive doubles: a whole pitch
  // (rows back to back) or exactly 16; the extra columns are never read.
  static constexpr int TROW = TZ + 6 <= 16 ? 16 : TP;
  static_assert(TROW <= TP, "T rows fit the pitch");
  static constexpr int T1Y = TY + 6;                          // d/dx over the y halo (and the z halo of the central rows)
  static constexpr int T2N = TX * TY * TROW;                 // d/dy over the z halo
  static constexpr int T1VOL = TX * T1Y * TP, T2VOL = TX * TY * TP;
  static constexpr size_t SMEM = (2 * (size_t)VOL + T1VOL + T2VOL) * sizeof(double);
  // + per-point staging of the stage input, u_n and the accumulator (24 each),
  // when it fits next to the tiles in the 227 KB a CTA may use
  static constexpr bool PTS = SMEM + (size_t)3 * NFIELD * NTHREADS * sizeof(double) + 1024 <= 232448;
  static constexpr size_t SMEM_PTS = PTS ? (size_t)3 * NFIELD * NTHREADS * sizeof(double) : 0;
  // Three rotating buffers fit next to the point staging for R = 3, but the
  // shared memory they take comes out of the L1 that holds the register
  // spills: measured 2-6 % slower on B200, so the staging rotates two.
  static constexpr int NBUF = 2;
  static constexpr size_t SMEM_RUN = SMEM + SMEM_PTS;
};

__device__ __forceinline__ Params load_params(const double* __restrict__ S) {
  Params P;
  P.eta = S[0]; P.cahd_c = S[1]; P.dt = S[2]; P.dx = S[3];
  P.ssl_h = S[4]; P.ssl_sigma = S[5]; P.t = S[6];
  P.lam0 = S[7]; P.lam1 = S[8]; P.lam2 = S[9]; P.lam3 = S[10];
  P.lamf0 = S[11]; P.lamf1 = S[12];
  P.hx = S[13]; P.hy = S[14]; P.hz = S[15];
  return P;
}

// The scale factors of one grid or block: thread a < 3 sets axis a and the
// mixed pair a (xy, xz, yz) from the three spacings h.
template <int R>
__device__ __forceinline__ void init_weights_h(Weights& W, const double* h, double ko_sigma, int a) {
  constexpr int PI[3] = {0, 0, 1}, PJ[3] = {1, 2, 2};
  W.f1[a] = 1.0 / (60.0 * h[a]);
  W.f2[a] = 1.0 / ((180.0 * h[a]) * h[a]);
  W.fk[a] = ko_sigma / ((R == 4 ? 256.0 : 64.0) * h[a]);
  W.fm[a] = (1.0 / (60.0 * h[PI[a]])) * (1.0 / (60.0 * h[PJ[a]]));
}

template <int R>
__device__ __forceinline__ void init_weights(Weights& W, const double* __restrict__ S, double ko_sigma, int tid) {
  if (tid < 3) {
    const double h[3] = {S[13], S[14], S[15]};
    init_weights_h<R>(W, h, ko_sigma, tid);
  }
}

// Issue the cp.async copies that stage one field's haloed tile, index clamped
// at the array ends (derivatives.py:83-84 pads with the edge value).
template <int R, class T = DefaultShape, int ZS = 0>
__device__ __forceinline__ void stage_tile(double* buf, const double* __restrict__ Ff, long long x0,
                                           long long y0, long long z0, long long Sx, long long Sy,
                                           long long Sz, int tid) {
  using Geo = TileGeom<R, T>;
  // 32-bit index arithmetic: a grid holds fewer than 2^31 points (check_grid)
  const int bx = (int)x0 - R, by = (int)y0 - R, bz = (int)z0 - R;
  const int mx = (int)Sx - 1, my = (int)Sy - 1, mz = (int)Sz - 1, sy = (int)Sy, sz = (int)Sz;
#pragma unroll
  for (int e = 0; e < Geo::PER_THREAD; ++e) {
    const int idx = tid + e * NTHREADS;
    if (idx < Geo::NELEM) {
      const int hz = idx % Geo::HZS;
      const int hy = (idx / Geo::HZS) % Geo::HY;
      const int hx = idx / (Geo::HZS * Geo::HY);
      const int qx = min(max(bx + hx, 0), mx);
      const int qy = min(max(by + hy, 0), my);
      const int qz = min(max(bz + hz, 0), mz);
      cp_async8(buf + hx * Geo::SX + hy * Geo::SY + hz + ZS, Ff + ((qx * sy + qy) * sz + qz));
    }
  }
}

// Final-stage values of the fields that algebraic enforcement rewrites are
// held back (gt0..5, At0..5, chi, alpha); the rest are stored directly.
__device__ __forceinline__ bool hold_for_enforce(double* en, int k, double un) {
  if (k >= F_GT && k < F_GT + 6) en[k - F_GT] = un;
  else if (k >= F_AT && k < F_AT + 6) en[6 + k - F_AT] = un;
  else if (k == F_CHI) en[12] = un;
  else if (k == F_ALPHA) en[13] = un;
  else return false;
  return true;
}

// Algebraic enforcement of one point (evolve.py:93-119): unit conformal
// determinant, traceless A~ with the unit-det inverse, chi and alpha floors.
__device__ __forceinline__ void enforce_point(double* en, double* O, long long n, double chi_floor,
                                              double alpha_floor) {
  double* g = en;
  double* a = en + 6;
  const double det = g[0] * (g[3] * g[5] - g[4] * g[4]) - g[1] * (g[1] * g[5] - g[4] * g[2]) +
                     g[2] * (g[1] * g[4] - g[3] * g[2]);
  const double scale = pow(det, -1.0 / 3.0);
#pragma unroll
  for (int q = 0; q < 6; ++q) g[q] = g[q] * scale;
  const double iuxx = g[3] * g[5] - g[4] * g[4];
  const double iuxy = g[2] * g[4] - g[1] * g[5];
  const double iuxz = g[1] * g[4] - g[2] * g[3];
  const double iuyy = g[0] * g[5] - g[2] * g[2];
  const double iuyz = g[1] * g[2] - g[0] * g[4];
  const double iuzz = g[0] * g[3] - g[1] * g[1];
  const double trA = iuxx * a[0] + iuyy * a[3] + iuzz * a[5] + 2.0 * (iuxy * a[1] + iuxz * a[2] + iuyz * a[4]);
  const double third = trA / 3.0;
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    O[(long long)(F_GT + q) * n] = g[q];
    O[(long long)(F_AT + q) * n] = a[q] - g[q] * third;
  }
  O[(long long)F_CHI * n] = fmax(en[12], chi_floor);
  O[(long long)F_ALPHA * n] = fmax(en[13], alpha_floor);
}

// ---------------------------------------------------------------------------
// The streaming fused kernel.
// ---------------------------------------------------------------------------
// TMA = true: every tile's halo box is staged by bulk-tensor copies (the
// array is a single grid whose layout allows them); false: per-thread clamped
// cp.async staging (batched block pools, odd z extents). One path per
// instantiation keeps the unrolled field loop small in the instruction cache.
template <int R, int MODE, class T = DefaultShape, bool TMA = false>
__global__ void __launch_bounds__(NTHREADS, 1) stream_kernel(const Args args, const __grid_constant__ CUtensorMap tmF) {
  using Geo = TileGeom<R, T>;
  constexpr int TX = Geo::TX, TY = Geo::TY, TZ = Geo::TZ, HZP = Geo::TP;
  constexpr bool RATES = MODE != MODE_CON && MODE != MODE_NORM;
  constexpr bool CONS = MODE == MODE_CON || MODE == MODE_NORM;
  extern __shared__ __align__(128) double smem[];
  double* const buf0 = smem;
  double* const buf1 = smem + Geo::VOL;
  double* const T1 = smem + 2 * Geo::VOL;
  double* const T2 = T1 + Geo::T1VOL;
  double* const pY = T2 + Geo::T2VOL;      // [24][256] this point's stage-input values
  double* const pU = pY + NFIELD * NTHREADS;  // [24][256] u_n (stage mode)
  double* const pA = pU + NFIELD * NTHREADS;  // [24][256] accumulator (stages 1-3)
  __shared__ Weights W;
  __shared__ __align__(8) unsigned long long tbar[3];  // bulk-copy completion, one per buffer
  // the next field's copies are issued after the field-start barrier, which
  // then also frees the previous field's buffer and T1/T2, so the field step
  // needs no closing barrier
  constexpr int NB = Geo::NBUF;
  static_assert(NB == 2, "the staging pipeline rotates two buffers");
  auto bufp = [&](int b) -> double* { return b == 0 ? buf0 : buf1; };

  const int tid = threadIdx.x;
  const bool batched = args.blocks != nullptr;
  const int lz = tid % TZ, ly = (tid / TZ) % TY, lx = tid / (TZ * TY);
  constexpr int ZS = TMA ? Geo::ZS_TMA : 0;  // z shift of the staged rows
  // padded T rows only where their extra columns stay inside a staged row
  constexpr int TROW = Geo::TROW - 4 + R + ZS <= Geo::HZP - 1 ? Geo::TROW : TZ + 6;
  constexpr int T2N = TX * TY * TROW;
  const int c = (lx + R) * Geo::SX + (ly + R) * Geo::SY + (lz + R + ZS);
  constexpr int st[3] = {Geo::SX, Geo::SY, 1};
  unsigned tphase = 0;    // bit b: parity of the next completion of tbar[b]
  unsigned tpending = 0;  // bit b: a copy into buffer b is in flight
  bool tfailed = false;   // this thread gave up on a wait: skip the rest
  if (TMA) {
    // bulk-tensor destinations must start on 128-byte boundaries: refuse to
    // run (and count the error) rather than issue a misaligned copy
    if (smem_addr(smem) & 127u) {
      if (tid == 0) atomicAdd(&g_async_copy_errors, 1);
      return;
    }
    if (tid == 0) {
      for (int b = 0; b < NB; ++b) mbar_init(&tbar[b], 1);
      asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
  }
  const int ntiles = batched ? args.ntiles : args.ntx * args.nty * args.ntz;
  const bool use_ko = RATES && args.use_ko != 0;
  const Params P0 = load_params(args.S);
  double norm_h = 0.0, norm_m = 0.0;  // norm mode: this thread's interior sums
  const double cs = args.stage == 0 ? 0.0 : (args.stage == 3 ? 1.0 : 0.5);
  if (!batched) {
    init_weights<R>(W, args.S, args.ko_sigma, tid);
    __syncthreads();
  }
  int cur_block = -1;
  bool prefetched = false;  // the tile's first field was staged during the previous tile

  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    // ---- tile geometry: the single grid, or the block that owns this tile ----
    long long Sx = args.Sx, Sy = args.Sy, Sz = args.Sz, n = args.n, base = 0;
    int ntx = args.ntx, nty = args.nty, ntz = args.ntz, lt = tile, core = 0;
    Params P = P0;
    if (batched) {
      int lo = 0, hi = args.nblocks - 1;  // last block with tile0 <= tile
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (args.blocks[mid].tile0 <= tile) lo = mid; else hi = mid - 1;
      }
      const bssn_b200_block bk = args.blocks[lo];
      Sx = bk.sx; Sy = bk.sy; Sz = bk.sz;
      n = Sx * Sy * Sz;
      base = bk.offset;
      core = bk.core;  // tiles cover [core, s - core): the ghosts come from a fill
      ntx = (bk.sx - 2 * core + TX - 1) / TX; nty = (bk.sy - 2 * core + TY - 1) / TY;
      ntz = (bk.sz - 2 * core + TZ - 1) / TZ;
      lt = tile - bk.tile0;
      P.dx = bk.h[0]; P.hx = bk.h[0]; P.hy = bk.h[1]; P.hz = bk.h[2];
      if (lo != cur_block) {
        // every thread must be done with the previous tile's last field step
        __syncthreads();
        if (tid < 3) init_weights_h<R>(W, bk.h, args.ko_sigma, tid);
        cur_block = lo;
      }
    }
    if (MODE == MODE_STAGE) P.t = P0.t + cs * P0.dt;  // stage time t, t+dt/2, t+dt/2, t+dt (evolve.py:125-131)
    if (MODE == MODE_MSRK) P.t = P0.t + args.ctime * P0.dt;  // node times t, t+c2 dt, t+c3 dt (evolve.py:139-153)
    const int tz = lt % ntz, ty = (lt / ntz) % nty, tx = lt / (ntz * nty);
    const long long x0 = core + (long long)tx * TX, y0 = core + (long long)ty * TY, z0 = core + (long long)tz * TZ;
    const long long gx = x0 + lx, gy = y0 + ly, gz = z0 + lz;
    const bool inside = gx < Sx - core && gy < Sy - core && gz < Sz - core;
    // points past the covered range compute on clamped data and store nothing
    const long long gidx = base + (clampll(gx, Sx - 1 - core) * Sy + clampll(gy, Sy - 1 - core)) * Sz +
                           clampll(gz, Sz - 1 - core);
    const double* __restrict__ Fbase = args.F + base;
    // Stage this point's 24 values (and, for the RK update, u_n and the
    // accumulator) in shared memory with cp.async: each thread copies and
    // later reads only its own slots, so no barrier is needed. Two commit
    // groups: the stage input, waited for here, then u_n and the accumulator,
    // read only by the epilogue and waited for at field 1 at the latest.
    if (Geo::PTS) {
#pragma unroll
      for (int k = 0; k < NFIELD; ++k) cp_async8(pY + k * NTHREADS + tid, args.F + gidx + (long long)k * n);
      cp_async_commit();
      if (MODE == MODE_STAGE || MODE == MODE_MSRK) {
#pragma unroll
        for (int k = 0; k < NFIELD; ++k) cp_async8(pU + k * NTHREADS + tid, args.U + gidx + (long long)k * n);
        if (MODE == MODE_STAGE ? args.stage > 0 : args.stage < 2) {
#pragma unroll
          for (int k = 0; k < NFIELD; ++k) cp_async8(pA + k * NTHREADS + tid, args.ACC + gidx + (long long)k * n);
        }
      }
      cp_async_commit();
      cp_async_wait<1>();
    }
    const double* __restrict__ Fp = args.F + gidx;
    auto fld = [&](int k) -> double {
      return Geo::PTS ? pY[k * NTHREADS + tid] : __ldg(Fp + (long long)k * n);
    };

    Stream<RATES, CONS, Geo::PTS> acc;
    if (Geo::PTS) {
      acc.pv = pY + tid;
      acc.ps = NTHREADS;
    }
    acc.init(fld);

    // Bulk-copy staging: thread 0 issues one tensor copy of the halo box per
    // field (the copy fills cells past the array with zeros; on edge tiles
    // the rows are then fixed up to the clamped values).
    const int bz0 = (int)z0 - R - ZS;
    const int bx0 = (int)x0 - R, by0 = (int)y0 - R;
    const bool edge = bx0 < 0 || bx0 + Geo::HX > Sx || by0 < 0 || by0 + Geo::HY > Sy || bz0 < 0 ||
                      bz0 + Geo::BOXZ > Sz;
    auto tma_issue = [&](int field, int b) {
      if (tid == 0) {
        mbar_expect_tx(&tbar[b], Geo::TMA_BYTES);
        tma_load_4d(bufp(b), &tmF, &tbar[b], bz0, by0, bx0, field);
      }
      tpending |= 1u << b;
    };
    // Edge clamp of a bulk-copied box (derivatives.py:83-84 edge padding):
    // thread r < HX*HY owns row r; a row outside the array in x or y copies
    // the clamped in-array row, and cells past the z ends take the clamped
    // z value. Reads touch only cells inside the array, which no thread writes.
    auto clamp_box = [&](double* buf) {
      if (tid < Geo::HX * Geo::HY) {
        const int hy = tid % Geo::HY, hx = tid / Geo::HY;
        const int X = bx0 + hx, Y = by0 + hy;
        const int cx = X < 0 ? 0 : (X >= Sx ? (int)Sx - 1 : X);
        const int cy = Y < 0 ? 0 : (Y >= Sy ? (int)Sy - 1 : Y);
        double* dst = buf + hx * Geo::SX + hy * Geo::SY;
        const double* src = buf + (cx - bx0) * Geo::SX + (cy - by0) * Geo::SY;
        const int zlo = bz0 < 0 ? -bz0 : 0;                                       // first in-array cell
        const int zhi = bz0 + Geo::BOXZ > Sz ? (int)Sz - bz0 : Geo::BOXZ;          // one past the last
        if (cx != X || cy != Y) {
          for (int hz = 0; hz < Geo::BOXZ; ++hz) dst[hz] = src[hz < zlo ? zlo : (hz >= zhi ? zhi - 1 : hz)];
        } else {
          for (int hz = 0; hz < zlo; ++hz) dst[hz] = src[zlo];
          for (int hz = zhi; hz < Geo::BOXZ; ++hz) dst[hz] = src[zhi - 1];
        }
      }
    };
    // the first field's copies; later fields are issued one step ahead, right
    // after the barrier that frees their buffer
    if (TMA) {
      tma_issue(stream_field(0), 0);
    } else if (!prefetched) {
      stage_tile<R, T, ZS>(bufp(0), Fbase + (long long)stream_field(0) * n, x0, y0, z0, Sx, Sy, Sz, tid);
      cp_async_commit();
    }
    const bool first_halo_old = prefetched;  // committed before this tile's point staging
    prefetched = false;
    Unroll<0, NFIELD>::run([&](auto ic) {
      constexpr int idx = decltype(ic)::value;
      constexpr int f = stream_field(idx);
      constexpr int b = idx % NB;
      const double* __restrict__ cur = bufp(b);
      // One barrier per field step: field idx's tile has landed (and, for
      // bulk copies on an edge tile, been clamped) everywhere, and every
      // thread is done with field idx - 1, whose buffer and T1/T2 are then
      // free for the next field's copies.
      if (TMA) {
        if (idx == NFIELD - 1) cp_async_wait<0>();  // the point staging of u_n / accumulator
        if (!tfailed && mbar_wait_bounded(&tbar[b], (tphase >> b) & 1u)) tpending &= ~(1u << b);
        else tfailed = true;  // results of this CTA are garbage; the error count says so
        tphase ^= 1u << b;
        if (edge) {
          clamp_box(bufp(b));
          fence_proxy_async();  // these writes before the next bulk copy into the buffer
        }
        __syncthreads();
        if (idx + 1 < NFIELD) tma_issue(stream_field(idx + 1), (idx + 1) % NB);
      } else {
        // field 0: a halo staged during the previous tile is older than the
        // u_n / accumulator point staging, which may still be in flight
        if (Geo::PTS && idx == 0 && first_halo_old) cp_async_wait<1>();
        else cp_async_wait<0>();
        __syncthreads();
        if (idx + 1 < NFIELD) {
          stage_tile<R, T, ZS>(bufp((idx + 1) % NB), Fbase + (long long)stream_field(idx + 1) * n, x0, y0, z0,
                               Sx, Sy, Sz, tid);
          cp_async_commit();
        } else if (!batched && tile + (int)gridDim.x < ntiles) {
          // single grid: the next tile's first field into the buffer that
          // field idx - 1 just freed, so its copies overlap this tile's last
          // field and epilogue
          const int nt = tile + (int)gridDim.x;
          const int nz_ = nt % ntz, ny_ = (nt / ntz) % nty, nx_ = nt / (ntz * nty);
          stage_tile<R, T, ZS>(bufp((idx + 1) % NB), args.F + (long long)stream_field(0) * n, (long long)nx_ * TX,
                               (long long)ny_ * TY, (long long)nz_ * TZ, Sx, Sy, Sz, tid);
          cp_async_commit();
          prefetched = true;
        }
      }

      // axial taps: first derivative, diagonal second derivative, KO
      double d1[3], d2[6], ko = 0.0;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        double v[2 * R + 1];
#pragma unroll
        for (int k = 0; k <= 2 * R; ++k) v[k] = cur[c + (k - R) * st[a]];
        d1[a] = __dmul_rn(c1_sum(v[R - 3], v[R - 2], v[R - 1], v[R + 1], v[R + 2], v[R + 3]), W.f1[a]);
        const double s1 = __dadd_rn(v[R + 1], v[R - 1]), s2 = __dadd_rn(v[R + 2], v[R - 2]),
                     s3 = __dadd_rn(v[R + 3], v[R - 3]);
        if (has_d2(f)) d2[sym(a, a)] = __dmul_rn(c2_sum(v[R], s1, s2, s3), W.f2[a]);
        if (use_ko) {
          const double sk = R == 4 ? ko8_sum(v[R], s1, s2, s3, __dadd_rn(v[2 * R], v[0])) : ko6_sum(v[R], s1, s2, s3);
          ko = __dadd_rn(ko, __dmul_rn(sk, W.fk[a]));
        }
      }
      if (has_d2(f)) {
        // T1 = unscaled d/dx sums over x in [0,TX) on the L-shaped region the
        // mixed taps read: y in [-3, TY+3) for z in [0, TZ) (for d2/dxdy), and
        // y in [0, TY) for z in [-3, 0) and [TZ, TZ+3) (for d2/dxdz); T1 rows
        // and columns are offset by 3 (row yy holds y = yy - 3).
        for (int e = tid; e < TX * Geo::T1Y * TZ; e += NTHREADS) {
          const int zz = e % TZ + 3;
          const int yy = (e / TZ) % Geo::T1Y;
          const int xx = e / (TZ * Geo::T1Y);
          const int cc = (xx + R) * Geo::SX + (yy - 3 + R) * Geo::SY + (zz - 3 + R + ZS);
          T1[(xx * Geo::T1Y + yy) * HZP + zz] = c1_at(cur + cc, Geo::SX);
        }
        for (int e = tid; e < TX * TY * 6; e += NTHREADS) {
          const int k = e % 6;
          const int zz = k < 3 ? k : TZ + k;
          const int yy = (e / 6) % TY + 3;
          const int xx = e / (6 * TY);
          const int cc = (xx + R) * Geo::SX + (yy - 3 + R) * Geo::SY + (zz - 3 + R + ZS);
          T1[(xx * Geo::T1Y + yy) * HZP + zz] = c1_at(cur + cc, Geo::SX);
        }
        // T2 = unscaled d/dy sums over x in [0,TX), y in [0,TY), z in [-3, TZ+3)
        for (int e = tid; e < T2N; e += NTHREADS) {
          const int zz = e % TROW;
          const int yy = (e / TROW) % TY;
          const int xx = e / (TROW * TY);
          const int cc = (xx + R) * Geo::SX + (yy + R) * Geo::SY + (zz - 3 + R + ZS);
          const double s = c1_at(cur + cc, Geo::SY);
          T2[(xx * TY + yy) * HZP + zz] = s;
        }
        __syncthreads();
        const int t1c = (lx * Geo::T1Y + ly + 3) * HZP + lz + 3;
        const int t2c = (lx * TY + ly) * HZP + lz + 3;
        const double sxy = __dmul_rn(c1_at(T1 + t1c, HZP), W.fm[0]);
        const double sxz = __dmul_rn(c1_at(T1 + t1c, 1), W.fm[1]);
        const double syz = __dmul_rn(c1_at(T2 + t2c, 1), W.fm[2]);
        d2[sym(0, 1)] = sxy;
        d2[sym(0, 2)] = sxz;
        d2[sym(1, 2)] = syz;
      } else {
#pragma unroll
        for (int p = 0; p < 6; ++p) d2[p] = 0.0;
      }
      acc.consume(f, d1, d2, ko, P, fld);
    });

    // ---- epilogue ---------------------------------------------------------
    if (MODE == MODE_RHS) {
      double* O = args.OUT + gidx;
      auto emit = [&](int k, double v) {
        if (inside) O[(long long)k * n] = v;
      };
      acc.finalize(fld, P, emit, NoCon());
    } else if (MODE == MODE_CON) {
      double* O = args.OUT + gidx;
      auto con = [&](double h, double m0, double m1, double m2) {
        if (inside) {
          O[0] = h;
          O[n] = m0;
          O[2 * n] = m1;
          O[3 * n] = m2;
        }
      };
      acc.finalize(fld, P, [](int, double) {}, con);
    } else if (MODE == MODE_NORM) {
      const int g = args.ng;
      const bool interior = inside && gx >= g && gx < Sx - g && gy >= g && gy < Sy - g && gz >= g && gz < Sz - g;
      auto con = [&](double h, double m0, double m1, double m2) {
        if (interior) {
          norm_h += h * h;
          norm_m += m0 * m0 + m1 * m1 + m2 * m2;
        }
      };
      acc.finalize(fld, P, [](int, double) {}, con);
    } else if (MODE == MODE_STAGE) {
      const int stage = args.stage;
      const double dt = P.dt;
      const double hstep = (stage == 2) ? dt : 0.5 * dt;
      const double w6 = dt / 6.0;
      double* A = args.ACC + gidx;
      double* O = args.OUT + gidx;
      double en[14];  // stage 3: gt0..5, At0..5, chi, alpha held for enforcement
#pragma unroll
      for (int q = 0; q < 14; ++q) en[q] = 0.0;
      auto emit = [&](int k, double rate) {
        const double u = Geo::PTS ? pU[k * NTHREADS + tid] : args.U[gidx + (long long)k * n];
        const double acc_k = stage == 0 ? 0.0 : (Geo::PTS ? pA[k * NTHREADS + tid] : A[(long long)k * n]);
        if (stage == 0) {
          if (inside) {
            A[(long long)k * n] = rate;
            O[(long long)k * n] = u + hstep * rate;
          }
        } else if (stage < 3) {
          if (inside) {
            A[(long long)k * n] = acc_k + 2.0 * rate;
            O[(long long)k * n] = u + hstep * rate;
          }
        } else {
          const double un = u + w6 * (acc_k + rate);
          if (!hold_for_enforce(en, k, un) && inside) O[(long long)k * n] = un;
        }
      };
      acc.finalize(fld, P, emit, NoCon());
      if (stage == 3 && inside) enforce_point(en, O, n, args.chi_floor, args.alpha_floor);
    } else {
      // 2-step / 3-stage MSRK (evolve.py:139-153). Stage 0 evaluates k1 = f(y_n)
      // (U = y_n, ACC = k0 = f(y_{n-1}) in, k1 out), stage 1 k2 at Y2 (U = partial
      // Y3, ACC = partial y_{n+1}), stage 2 k3 at Y3 (U = partial y_{n+1}).
      const int stage = args.stage;
      const double dt = P.dt;
      const double* c = args.coef;
      double* A = args.ACC + gidx;
      double* O = args.OUT + gidx;
      double en[14];
#pragma unroll
      for (int q = 0; q < 14; ++q) en[q] = 0.0;
      auto emit = [&](int k, double rate) {
        const long long o = (long long)k * n;
        const double u = Geo::PTS ? pU[k * NTHREADS + tid] : args.U[gidx + o];
        const double a = stage == 2 ? 0.0 : (Geo::PTS ? pA[k * NTHREADS + tid] : A[o]);
        if (stage == 0) {
          if (inside) {
            A[o] = rate;
            O[o] = u + dt * (c[0] * a + c[1] * rate);
            args.OUT2[gidx + o] = u + dt * (c[2] * a + c[3] * rate);
            args.OUT3[gidx + o] = u + dt * (c[5] * a + c[6] * rate);
          }
        } else if (stage == 1) {
          if (inside) {
            O[o] = u + dt * (c[4] * rate);
            A[o] = a + dt * (c[7] * rate);
          }
        } else {
          const double un = u + dt * (c[8] * rate);
          if (!hold_for_enforce(en, k, un) && inside) O[o] = un;
        }
      };
      acc.finalize(fld, P, emit, NoCon());
      if (stage == 2 && inside) enforce_point(en, O, n, args.chi_floor, args.alpha_floor);
    }
  }
  if (TMA && tfailed) {
    // give copies still in flight a bounded time to land before the CTA exits
    for (int b = 0; b < NB; ++b)
      if (tpending & (1u << b)) mbar_wait_bounded(&tbar[b], ((tphase >> b) & 1u) ^ 1u);
  }
  if (MODE == MODE_NORM) {
    // fixed-order block reduction of the per-thread sums (reuses the staging buffer)
    __syncthreads();
    double* red = smem;
    red[2 * tid] = norm_h;
    red[2 * tid + 1] = norm_m;
    __syncthreads();
    for (int w = NTHREADS / 2; w > 0; w >>= 1) {
      if (tid < w) {
        red[2 * tid] += red[2 * (tid + w)];
        red[2 * tid + 1] += red[2 * (tid + w) + 1];
      }
      __syncthreads();
    }
    if (tid == 0) {
      args.partials[2 * blockIdx.x] = red[0];
      args.partials[2 * blockIdx.x + 1] = red[1];
    }
  }
}

}  // namespace bssn

namespace bssn_host {
// Internal linkage for everything below: each translation unit keeps its own
// per-device flags, and two loaded copies of the library never share them.
namespace {

// Opt a kernel into its dynamic shared memory once per device.
template <class K>
int set_smem(K kern, size_t smem, int* flags) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return bssn_host::cuda_fail("cudaGetDevice", e);
  if (dev < 0 || dev >= kMaxDev) return bssn_host::fail(BSSN_B200_EINVAL, "device ordinal out of range");
  if (!flags[dev]) {
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return bssn_host::cuda_fail("cudaFuncSetAttribute", e);
    flags[dev] = 1;
  }
  return 0;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no -lcuda).
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_tiled() {
  static EncodeTiled fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return static_cast<EncodeTiled>(nullptr);
    return reinterpret_cast<EncodeTiled>(p);
  }();
  return fn;
}

// Tensor map of a (24, Sx, Sy, Sz) float64 state for the stream kernel's halo
// boxes (BOXZ x HY x HX x 1 field). False when the layout does not allow bulk
// copies: every stride must be a multiple of 16 bytes (Sz even) and the base
// 16-byte aligned; the kernel then stages every tile with cp.async.
template <int R, class T>
bool make_state_map(CUtensorMap* map, const double* F, long long Sx, long long Sy, long long Sz) {
#ifdef BSSN_B200_NO_TMA
  (void)map; (void)F; (void)Sx; (void)Sy; (void)Sz;
  return false;
#else
  using Geo = bssn::TileGeom<R, T>;
  EncodeTiled enc = encode_tiled();
  if (Geo::BOXZ != Geo::HZP) return false;  // a copied box row must be exactly one staged row
  if (!enc || (Sz & 1) || (reinterpret_cast<uintptr_t>(F) & 15)) return false;
  if (Sx < Geo::HX || Sy < Geo::HY || Sz < Geo::BOXZ) return false;
  const cuuint64_t dims[4] = {(cuuint64_t)Sz, (cuuint64_t)Sy, (cuuint64_t)Sx, (cuuint64_t)bssn::NFIELD};
  const cuuint64_t strides[3] = {(cuuint64_t)Sz * 8, (cuuint64_t)(Sy * Sz) * 8, (cuuint64_t)(Sx * Sy * Sz) * 8};
  const cuuint32_t box[4] = {(cuuint32_t)Geo::BOXZ, (cuuint32_t)Geo::HY, (cuuint32_t)Geo::HX, 1};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<double*>(F), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
#endif
}

// Halo staging of the single-grid stream kernel: per-thread clamped cp.async
// copies (default), or bulk-tensor copies when BSSN_B200_STAGING=tma and the
// layout allows them. Read on every call, like the reference's FFI handler
// reads its environment knobs (3D/src/bssn3d/cuda/rhs_fused.cu:34-41). Both
// give the same bytes; on B200 the per-thread form measured faster for this
// kernel (its warps stay in step through the unrolled field loop).
bool tma_staging_requested() {
  const char* v = std::getenv("BSSN_B200_STAGING");
  return v != nullptr && std::strcmp(v, "tma") == 0;
}

template <int R, int MODE, class T = bssn::DefaultShape>
int launch_stream(const bssn::Args& a, cudaStream_t stream, int grid) {
  using Geo = bssn::TileGeom<R, T>;
  const size_t smem = Geo::SMEM_RUN;
  CUtensorMap map;
  std::memset(&map, 0, sizeof(map));
  if constexpr (std::is_same<T, bssn::DefaultShape>::value) {
    if (!a.blocks && tma_staging_requested() && make_state_map<R, T>(&map, a.F, a.Sx, a.Sy, a.Sz)) {
      const size_t smem_tma = Geo::SMEM_RUN;
      auto kern = bssn::stream_kernel<R, MODE, T, true>;
      static int flags[kMaxDev] = {0};
      int rc = set_smem(kern, smem_tma, flags);
      if (rc) return rc;
      kern<<<grid, bssn::NTHREADS, smem_tma, stream>>>(a, map);
      cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) return bssn_host::cuda_fail("stream kernel launch", e);
      return 0;
    }
  }
  auto kern = bssn::stream_kernel<R, MODE, T, false>;
  static int flags[kMaxDev] = {0};
  int rc = set_smem(kern, smem, flags);
  if (rc) return rc;
  kern<<<grid, bssn::NTHREADS, smem, stream>>>(a, map);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return bssn_host::cuda_fail("stream kernel launch", e);
  return 0;
}

// Reads this translation unit's bulk-copy error counter.
int read_copy_errors(int* count) {
  int v = 0;
  cudaError_t e = cudaMemcpyFromSymbol(&v, bssn::g_async_copy_errors, sizeof(int));
  if (e != cudaSuccess) return cuda_fail("async_copy_errors", e);
  *count = v;
  return 0;
}

}  // namespace
}  // namespace bssn_host

// bssn_b200 — fused BSSN right-hand side and RK4 stage kernels for sm_100a,
// behind the C ABI of include/bssn_b200.h.
//
// The stream kernel itself lives in stream_kernel.cuh, instantiated by the
// stream_*.cu translation units; this file holds the other kernels and the
// C ABI. One persistent kernel per RHS evaluation (stream_kernel). Each 256-thread CTA
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
#include <cuda.h>
#include <cuda_runtime.h>

#include <atomic>
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
#include "stream_kernel.cuh"
#include "stream_launch.h"

namespace bssn {
// ---------------------------------------------------------------------------
// Derivative bundle to global memory (the bssn_b200_derivatives entry).
// ---------------------------------------------------------------------------
template <int R>
__device__ __forceinline__ void field_derivs(const double* __restrict__ t, int c, int f, const Weights& W,
                                             bool ko, double* __restrict__ out, long long n) {
  constexpr int st[3] = {TileGeom<R>::SX, TileGeom<R>::SY, 1};
  double kacc = 0.0;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    double v[2 * R + 1];
#pragma unroll
    for (int k = 0; k <= 2 * R; ++k) v[k] = t[c + (k - R) * st[a]];
    out[(long long)d1slot(f, a) * n] =
        __dmul_rn(c1_sum(v[R - 3], v[R - 2], v[R - 1], v[R + 1], v[R + 2], v[R + 3]), W.f1[a]);
    const double s1 = __dadd_rn(v[R + 1], v[R - 1]), s2 = __dadd_rn(v[R + 2], v[R - 2]),
                 s3 = __dadd_rn(v[R + 3], v[R - 3]);
    if (has_d2(f)) out[(long long)d2slot(f, sym(a, a)) * n] = __dmul_rn(c2_sum(v[R], s1, s2, s3), W.f2[a]);
    if (ko) {
      const double sk = R == 4 ? ko8_sum(v[R], s1, s2, s3, __dadd_rn(v[2 * R], v[0])) : ko6_sum(v[R], s1, s2, s3);
      kacc = __dadd_rn(kacc, __dmul_rn(sk, W.fk[a]));
    }
  }
  if (has_d2(f)) {
    // mixed: the unscaled first-derivative sums along i at the 6 offsets along
    // j, differentiated along j, scaled by f1_i * f1_j
    constexpr int PI[3] = {0, 0, 1}, PJ[3] = {1, 2, 2};
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const int i = PI[q], j = PJ[q];
      double inner[7];
#pragma unroll
      for (int b = 0; b < 7; ++b) inner[b] = b == 3 ? 0.0 : c1_at(t + c + (b - 3) * st[j], st[i]);
      out[(long long)d2slot(f, sym(i, j)) * n] =
          __dmul_rn(c1_sum(inner[0], inner[1], inner[2], inner[4], inner[5], inner[6]), W.fm[q]);
    }
  }
  if (ko) out[(long long)(NDERIV + f) * n] = kacc;
}

template <int R>
__global__ void __launch_bounds__(NTHREADS) deriv_kernel(const Args args) {
  using Geo = TileGeom<R>;
  extern __shared__ __align__(128) double smem[];
  __shared__ Weights W;
  const int tid = threadIdx.x;
  init_weights<R>(W, args.S, args.ko_sigma, tid);
  __syncthreads();
  const long long Sx = args.Sx, Sy = args.Sy, Sz = args.Sz, n = args.n;
  constexpr int TX = Geo::TX, TY = Geo::TY, TZ = Geo::TZ;
  const int lz = tid % TZ, ly = (tid / TZ) % TY, lx = tid / (TZ * TY);
  const int c = (lx + R) * Geo::SX + (ly + R) * Geo::SY + (lz + R);
  const int ntiles = args.ntx * args.nty * args.ntz;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int tz = tile % args.ntz, ty = (tile / args.ntz) % args.nty, tx = tile / (args.ntz * args.nty);
    const long long x0 = (long long)tx * TX, y0 = (long long)ty * TY, z0 = (long long)tz * TZ;
    const long long gx = x0 + lx, gy = y0 + ly, gz = z0 + lz;
    const bool inside = gx < Sx && gy < Sy && gz < Sz;
    double* out = args.OUT + (gx * Sy + gy) * Sz + gz;
    for (int f = 0; f < NFIELD; ++f) {
      stage_tile<R>(smem, args.F + (long long)f * n, x0, y0, z0, Sx, Sy, Sz, tid);
      cp_async_commit();
      cp_async_wait<0>();
      __syncthreads();
      if (inside) field_derivs<R>(smem, c, f, W, args.use_ko != 0, out, n);
      __syncthreads();
    }
  }
}

// Second pass of the constraint norms: the per-CTA partial sums in index
// order (deterministic for a given grid), then RMS over the interior
// (3D/src/bssn3d/constraints.py:53-62).
__global__ void norm_finalize_kernel(const double* __restrict__ partials, int nparts, double count,
                                     double* __restrict__ out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double h = 0.0, m = 0.0;
    for (int i = 0; i < nparts; ++i) {
      h += partials[2 * i];
      m += partials[2 * i + 1];
    }
    out[0] = sqrt(h / count);
    out[1] = sqrt(m / count);
  }
}

// Partial-sum slots for bssn_b200_constraint_norms_static, the entry point for
// callers that cannot allocate device memory. It is a file-scope device array:
// every GPU that loads this library holds it (4 KB) until the process exits,
// and every call of that entry point reuses it.
// CTAs whose partial sums fit (2 doubles each). The norm launch runs at most
// one CTA per SM, so 256 covers every GPU with up to 256 SMs (B200: 148); a
// GPU with more is refused by the entry point's size check.
constexpr int kStaticNormCtas = 256;
static __device__ __align__(256) double g_static_norm_partials[2 * kStaticNormCtas];

// t <- t + dt in the device scalar pack, between captured RK4 steps
// (the fori_loop carry update of 3D/src/bssn3d/evolve.py:186-193).
__global__ void advance_time_kernel(double* S) {
  if (threadIdx.x == 0 && blockIdx.x == 0) S[6] = S[6] + S[2];
}

// Algebra only: derivatives supplied by the caller (the reference's
// algebra-only microbenchmark interface, 3D/src/bssn3d/cuda/gen_algebra_cuda.py:55-96),
// consumed in the stream order of the fused kernel.
__global__ void __launch_bounds__(128) algebra_kernel(const double* __restrict__ F, const double* __restrict__ D,
                                                      const double* __restrict__ S, double* __restrict__ OUT,
                                                      long long n) {
  const Params P = load_params(S);
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    auto fld = [&](int k) -> double { return __ldg(F + (long long)k * n + q); };
    auto drv = [&](int s) -> double { return __ldg(D + (long long)s * n + q); };
    Stream<true, false> acc;
    acc.init(fld);
    Unroll<0, NFIELD>::run([&](auto ic) {
      constexpr int f = stream_field(decltype(ic)::value);
      double d1[3], d2[6];
#pragma unroll
      for (int a = 0; a < 3; ++a) d1[a] = drv(d1slot(f, a));
#pragma unroll
      for (int p = 0; p < 6; ++p) d2[p] = has_d2(f) ? drv(d2slot(f, p)) : 0.0;
      acc.consume(f, d1, d2, 0.0, P, fld);
    });
    auto emit = [&](int k, double v) { OUT[(long long)k * n + q] = v; };
    acc.finalize(fld, P, emit, NoCon());
  }
}

// One RK4 stage from precomputed derivatives over the covered points
// [core, s - core)^3 of every block of a block list: the algebra of
// algebra_kernel on the stage input Y with the block's spacing and the stage
// time, the KO sums taken from slots 138..161 of D when ko_slots is set, and
// the stage epilogue of the stream kernel (evolve.py:125-131, the final stage
// with algebraic enforcement). Derivative slot s of block b is at
// D + (offset_b / 24) * nslot + s * n_b. Points are enumerated block by block
// (pts0 = prefix of covered points), one thread per point.
__global__ void __launch_bounds__(128) stage_derivs_kernel(
    const double* __restrict__ U, const double* __restrict__ Y, double* __restrict__ ACC, double* __restrict__ OUT,
    const double* __restrict__ D, int nslot, const double* __restrict__ S, int stage, int ko_slots,
    double chi_floor, double alpha_floor, const bssn_b200_block* __restrict__ blocks, int nblocks,
    const long long* __restrict__ pts0, long long npoints) {
  const Params P0 = load_params(S);
  const double cs = stage == 0 ? 0.0 : (stage == 3 ? 1.0 : 0.5);
  const double dt = P0.dt;
  const double hstep = (stage == 2) ? dt : 0.5 * dt;
  const double w6 = dt / 6.0;
  const int lane = threadIdx.x & 31;
  const long long stride = (long long)gridDim.x * blockDim.x;
  // warps walk the points together (q0 is the warp's first point), so the
  // block lookup is one 32-way search per warp instead of one per point
  for (long long q0 = blockIdx.x * (long long)blockDim.x + (threadIdx.x & ~31); q0 < npoints; q0 += stride) {
    const long long q = q0 + lane;
    int lo = 0, nb = nblocks;  // last block whose first point is <= q0 (pts0[0] = 0)
    while (nb > 1) {
      const int step = (nb + 31) >> 5;
      const int idx = lo + lane * step;
      const unsigned ok = __ballot_sync(0xffffffffu, idx < lo + nb && pts0[idx] <= q0);
      const int last = 31 - __clz(ok);
      lo += last * step;
      nb = min(step, nb - last * step);
    }
    while (lo + 1 < nblocks && pts0[lo + 1] <= q) ++lo;  // a warp that straddles blocks
    if (q >= npoints) continue;
    const bssn_b200_block bk = blocks[lo];
    const int c = bk.core;
    const int ey = bk.sy - 2 * c, ez = bk.sz - 2 * c;
    const int lq = (int)(q - pts0[lo]);
    const int z = lq % ez + c, y = (lq / ez) % ey + c, x = lq / (ez * ey) + c;
    const long long n = (long long)bk.sx * bk.sy * bk.sz;
    const long long p = ((long long)x * bk.sy + y) * bk.sz + z;
    const long long gidx = bk.offset + p;
    const double* Dq = D + (bk.offset / 24) * nslot + p;
    Params P = P0;
    P.dx = bk.h[0]; P.hx = bk.h[0]; P.hy = bk.h[1]; P.hz = bk.h[2];
    P.t = P0.t + cs * P0.dt;  // stage time t, t+dt/2, t+dt/2, t+dt (evolve.py:125-131)
    auto fld = [&](int k) -> double { return __ldg(Y + gidx + (long long)k * n); };
    auto drv = [&](int s) -> double { return __ldg(Dq + (long long)s * n); };
    Stream<true, false> acc;
    acc.init(fld);
    Unroll<0, NFIELD>::run([&](auto ic) {
      constexpr int f = stream_field(decltype(ic)::value);
      double d1[3], d2[6];
#pragma unroll
      for (int a = 0; a < 3; ++a) d1[a] = drv(d1slot(f, a));
#pragma unroll
      for (int pp = 0; pp < 6; ++pp) d2[pp] = has_d2(f) ? drv(d2slot(f, pp)) : 0.0;
      acc.consume(f, d1, d2, ko_slots ? drv(138 + f) : 0.0, P, fld);
    });
    double* A = ACC + gidx;
    double* O = OUT + gidx;
    double en[14];
#pragma unroll
    for (int k = 0; k < 14; ++k) en[k] = 0.0;
    auto emit = [&](int k, double rate) {
      const long long o = (long long)k * n;
      const double u = U[gidx + o];
      if (stage == 0) {
        A[o] = rate;
        O[o] = u + hstep * rate;
      } else if (stage < 3) {
        A[o] = A[o] + 2.0 * rate;
        O[o] = u + hstep * rate;
      } else {
        const double un = u + w6 * (A[o] + rate);
        if (!hold_for_enforce(en, k, un)) O[o] = un;
      }
    };
    acc.finalize(fld, P, emit, NoCon());
    if (stage == 3) enforce_point(en, O, n, chi_floor, alpha_floor);
  }
}

__global__ void enforce_kernel(double* __restrict__ U, long long n, double chi_floor, double alpha_floor) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    double g[6], a[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) { g[k] = U[(F_GT + k) * n + q]; a[k] = U[(F_AT + k) * n + q]; }
    const double det = g[0] * (g[3] * g[5] - g[4] * g[4]) - g[1] * (g[1] * g[5] - g[4] * g[2]) +
                       g[2] * (g[1] * g[4] - g[3] * g[2]);
    const double scale = pow(det, -1.0 / 3.0);
#pragma unroll
    for (int k = 0; k < 6; ++k) g[k] = g[k] * scale;
    const double iuxx = g[3] * g[5] - g[4] * g[4];
    const double iuxy = g[2] * g[4] - g[1] * g[5];
    const double iuxz = g[1] * g[4] - g[2] * g[3];
    const double iuyy = g[0] * g[5] - g[2] * g[2];
    const double iuyz = g[1] * g[2] - g[0] * g[4];
    const double iuzz = g[0] * g[3] - g[1] * g[1];
    const double trA = iuxx * a[0] + iuyy * a[3] + iuzz * a[5] + 2.0 * (iuxy * a[1] + iuxz * a[2] + iuyz * a[4]);
    const double third = trA / 3.0;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      U[(F_GT + k) * n + q] = g[k];
      U[(F_AT + k) * n + q] = a[k] - g[k] * third;
    }
    U[F_CHI * n + q] = fmax(U[F_CHI * n + q], chi_floor);
    U[F_ALPHA * n + q] = fmax(U[F_ALPHA * n + q], alpha_floor);
  }
}

// One axis of the periodic ghost sync: ghosts [0,ng) <- [S-2ng, S-ng), [S-ng,S) <- [ng, 2ng).
__global__ void periodic_axis_kernel(double* __restrict__ U, long long Sx, long long Sy, long long Sz, int axis, int ng) {
  const long long S[3] = {Sx, Sy, Sz};
  const long long st[3] = {Sy * Sz, Sz, 1};
  const long long n = Sx * Sy * Sz;
  const long long o1 = S[(axis + 1) % 3], o2 = S[(axis + 2) % 3];
  const long long per_field = 2LL * ng * o1 * o2;
  const long long total = per_field * NFIELD;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total; q += (long long)gridDim.x * blockDim.x) {
    const int f = (int)(q / per_field);
    long long r = q % per_field;
    const long long i2 = r % o2; r /= o2;
    const long long i1 = r % o1; r /= o1;
    const int layer = (int)r;  // 0..2ng-1
    const long long cdst = layer < ng ? layer : S[axis] - 2 * ng + layer;
    const long long csrc = layer < ng ? S[axis] - 2 * ng + layer : layer;
    const long long base = i1 * st[(axis + 1) % 3] + i2 * st[(axis + 2) % 3];
    U[f * n + base + cdst * st[axis]] = U[f * n + base + csrc * st[axis]];
  }
}

}  // namespace bssn

// ======================================================================
// host side
// ======================================================================
namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

int cuda_fail(const char* what, cudaError_t e) {
  return fail(BSSN_B200_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

using bssn_host::kMaxDev;
using bssn_host::set_smem;

int device_sms(int* sms) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail("cudaGetDevice", e);
  static int cache[kMaxDev] = {0};
  if (dev >= 0 && dev < kMaxDev && cache[dev] > 0) {
    *sms = cache[dev];
    return 0;
  }
  int v = 0;
  e = cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return cuda_fail("cudaDeviceGetAttribute", e);
  if (dev >= 0 && dev < kMaxDev) cache[dev] = v;
  *sms = v;
  return 0;
}

template <int R>
int launch_deriv(const bssn::Args& a, cudaStream_t stream, int grid) {
  using Geo = bssn::TileGeom<R>;
  const size_t smem = (size_t)Geo::VOL * sizeof(double);
  auto kern = bssn::deriv_kernel<R>;
  static int flags[kMaxDev] = {0};
  int rc = set_smem(kern, smem, flags);
  if (rc) return rc;
  kern<<<grid, bssn::NTHREADS, smem, stream>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail("derivative kernel launch", e);
  return 0;
}

int check_grid(long long Sx, long long Sy, long long Sz) {
  if (Sx < 1 || Sy < 1 || Sz < 1) return fail(BSSN_B200_EINVAL, "grid extents must be >= 1");
  if (Sx > (1LL << 31) / Sy / Sz) return fail(BSSN_B200_EINVAL, "grid has more than 2^31 points");
  return 0;
}

// Fill the shape fields of `a` and the persistent grid size (one CTA per SM).
int prepare(bssn::Args* a, long long Sx, long long Sy, long long Sz, int ctas_per_sm, int* grid) {
  int rc = check_grid(Sx, Sy, Sz);
  if (rc) return rc;
  int sms = 0;
  rc = device_sms(&sms);
  if (rc) return rc;
  a->Sx = Sx; a->Sy = Sy; a->Sz = Sz;
  a->n = Sx * Sy * Sz;
  using D = bssn::DefaultShape;
  a->ntx = (int)((Sx + D::X - 1) / D::X);
  a->nty = (int)((Sy + D::Y - 1) / D::Y);
  a->ntz = (int)((Sz + D::Z - 1) / D::Z);
  const long long ntiles = (long long)a->ntx * a->nty * a->ntz;
  const long long cap = (long long)sms * ctas_per_sm;
  *grid = (int)(ntiles < cap ? ntiles : cap);
  return 0;
}

void variant_shape(int variant, int* tx, int* ty, int* tz) {
  static const int shapes[BSSN_B200_NVARIANTS][3] = {{4, 4, 16}, {2, 8, 16}, {4, 8, 8}, {8, 4, 8}};
  *tx = shapes[variant][0];
  *ty = shapes[variant][1];
  *tz = shapes[variant][2];
}

// One stream-kernel launch on the default tile (variant 0) or a batched tile
// variant; the instantiations live in the stream_*.cu translation units.
int launch_single(int R, int mode, const bssn::Args& a, cudaStream_t st, int grid) {
  switch (mode) {
    case bssn::MODE_STAGE: return bssn_host::launch_stage_modes(R, mode, a, st, grid);
    case bssn::MODE_MSRK: return bssn_host::launch_msrk_modes(R, mode, a, st, grid);
    default: return bssn_host::launch_rhs_modes(R, mode, a, st, grid);
  }
}

int launch_variant(int R, int mode, const bssn::Args& a, cudaStream_t st, int grid, int variant) {
  if (variant == 0) return launch_single(R, mode, a, st, grid);
  if (variant < 0 || variant >= BSSN_B200_NVARIANTS) return fail(BSSN_B200_EINVAL, "variant out of range");
  return R == 4 ? bssn_host::launch_batch_r4(mode, variant, a, st, grid)
                : bssn_host::launch_batch_r3(mode, variant, a, st, grid);
}

int prepare_batch(bssn::Args* a, const bssn_b200_block* blocks, int nblocks, int ntiles, int variant, int* grid) {
  if (!blocks) return fail(BSSN_B200_EINVAL, "batch: NULL block table");
  if (nblocks < 1) return fail(BSSN_B200_EINVAL, "batch: nblocks must be >= 1");
  if (ntiles < 1) return fail(BSSN_B200_EINVAL, "batch: ntiles must be >= 1 (run bssn_b200_batch_plan)");
  if (variant < 0 || variant >= BSSN_B200_NVARIANTS) return fail(BSSN_B200_EINVAL, "batch: variant out of range");
  int sms = 0;
  int rc = device_sms(&sms);
  if (rc) return rc;
  a->blocks = blocks;
  a->nblocks = nblocks;
  a->ntiles = ntiles;
  *grid = ntiles < sms ? ntiles : sms;
  return 0;
}

}  // namespace

namespace bssn_host {
int fail(int code, const std::string& msg) { return ::fail(code, msg); }
int cuda_fail(const char* what, cudaError_t e) { return ::cuda_fail(what, e); }
int device_sms(int* sms) { return ::device_sms(sms); }
}  // namespace bssn_host

extern "C" {

int bssn_b200_batch_plan(bssn_b200_block* host_blocks, int nblocks, int variant) {
  if (!host_blocks || nblocks < 1) {
    fail(BSSN_B200_EINVAL, "batch_plan: empty block table");
    return -1;
  }
  if (variant < 0 || variant >= BSSN_B200_NVARIANTS) {
    fail(BSSN_B200_EINVAL, "batch_plan: variant out of range");
    return -1;
  }
  int tx, ty, tz;
  variant_shape(variant, &tx, &ty, &tz);
  long long t0 = 0;
  for (int b = 0; b < nblocks; ++b) {
    bssn_b200_block& bk = host_blocks[b];
    if (bk.sx < 1 || bk.sy < 1 || bk.sz < 1 || bk.offset < 0 || !(bk.h[0] > 0) || !(bk.h[1] > 0) || !(bk.h[2] > 0)) {
      fail(BSSN_B200_EINVAL, "batch_plan: block " + std::to_string(b) + " has a bad extent, offset or spacing");
      return -1;
    }
    if ((long long)bk.sx * bk.sy * bk.sz >= (1LL << 31)) {
      fail(BSSN_B200_EINVAL, "batch_plan: block " + std::to_string(b) + " has 2^31 points or more");
      return -1;
    }
    if (bk.core < 0 || 2 * bk.core >= bk.sx || 2 * bk.core >= bk.sy || 2 * bk.core >= bk.sz) {
      fail(BSSN_B200_EINVAL, "batch_plan: block " + std::to_string(b) + " has a core margin that leaves no points");
      return -1;
    }
    bk.tile0 = (int)t0;
    const int c2 = 2 * bk.core;
    t0 += (long long)((bk.sx - c2 + tx - 1) / tx) * ((bk.sy - c2 + ty - 1) / ty) * ((bk.sz - c2 + tz - 1) / tz);
    if (t0 > (1LL << 30)) {
      fail(BSSN_B200_EINVAL, "batch_plan: too many tiles");
      return -1;
    }
  }
  return (int)t0;
}

int bssn_b200_batch_rhs(void* stream, const double* F, const double* S, double* OUT,
                        const bssn_b200_block* blocks, int nblocks, int ntiles, int variant) {
  if (!F || !S || !OUT) return fail(BSSN_B200_EINVAL, "batch_rhs: NULL operand");
  if (OUT == F) return fail(BSSN_B200_EINVAL, "batch_rhs: OUT must not alias F");
  bssn::Args a{};
  int grid = 0;
  int rc = prepare_batch(&a, blocks, nblocks, ntiles, variant, &grid);
  if (rc) return rc;
  a.F = F; a.S = S; a.OUT = OUT;
  return launch_variant(3, bssn::MODE_RHS, a, static_cast<cudaStream_t>(stream), grid, variant);
}

int bssn_b200_batch_rk4_stage(void* stream, int stage, const double* U, const double* Y, double* ACC,
                              double* YNEXT, const double* S, double ko_sigma, int ko_order,
                              double chi_floor, double alpha_floor, const bssn_b200_block* blocks,
                              int nblocks, int ntiles, int variant) {
  if (stage < 0 || stage > 3) return fail(BSSN_B200_EINVAL, "batch_rk4_stage: stage must be 0..3");
  if (!U || !Y || !ACC || !YNEXT || !S) return fail(BSSN_B200_EINVAL, "batch_rk4_stage: NULL operand");
  if (YNEXT == Y) return fail(BSSN_B200_EINVAL, "batch_rk4_stage: YNEXT must not alias Y");
  if (stage < 3 && YNEXT == U) return fail(BSSN_B200_EINVAL, "batch_rk4_stage: YNEXT may alias U only at stage 3");
  if (ACC == Y || ACC == U || ACC == YNEXT) return fail(BSSN_B200_EINVAL, "batch_rk4_stage: ACC must not alias another operand");
  const bool use_ko = ko_sigma > 0.0;
  if (use_ko && ko_order != 6 && ko_order != 8) return fail(BSSN_B200_EINVAL, "batch_rk4_stage: ko_order must be 6 or 8");
  bssn::Args a{};
  int grid = 0;
  int rc = prepare_batch(&a, blocks, nblocks, ntiles, variant, &grid);
  if (rc) return rc;
  a.F = Y; a.U = U; a.ACC = ACC; a.OUT = YNEXT; a.S = S;
  a.stage = stage;
  a.use_ko = use_ko ? 1 : 0;
  a.ko_sigma = use_ko ? ko_sigma : 0.0;
  a.chi_floor = chi_floor; a.alpha_floor = alpha_floor;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (use_ko && ko_order == 8) return launch_variant(4, bssn::MODE_STAGE, a, st, grid, variant);
  return launch_variant(3, bssn::MODE_STAGE, a, st, grid, variant);
}

const char* bssn_b200_last_error(void) { return g_err.c_str(); }

const char* bssn_b200_version(void) { return "bssn_b200 0.3 sm_100a"; }

int bssn_b200_async_copy_errors(int* count) {
  if (!count) return fail(BSSN_B200_EINVAL, "async_copy_errors: NULL operand");
  int total = 0;
  int (*const parts[])(int*) = {bssn_host::copy_errors_rhs, bssn_host::copy_errors_stage,
                                bssn_host::copy_errors_msrk};
  for (auto part : parts) {
    int c = 0;
    const int rc = part(&c);
    if (rc) return rc;
    total += c;
  }
  *count = total;
  return 0;
}

int bssn_b200_rhs(void* stream, const double* F, const double* S, double* OUT, long long Sx,
                  long long Sy, long long Sz) {
  if (!F || !S || !OUT) return fail(BSSN_B200_EINVAL, "rhs: NULL operand");
  if (OUT == F) return fail(BSSN_B200_EINVAL, "rhs: OUT must not alias F");
  bssn::Args a{};
  int grid = 0;
  int rc = prepare(&a, Sx, Sy, Sz, 1, &grid);
  if (rc) return rc;
  a.F = F; a.S = S; a.OUT = OUT;
  return launch_single(3, bssn::MODE_RHS, a, static_cast<cudaStream_t>(stream), grid);
}

int bssn_b200_constraints(void* stream, const double* F, const double* S, double* OUT,
                          long long Sx, long long Sy, long long Sz) {
  if (!F || !S || !OUT) return fail(BSSN_B200_EINVAL, "constraints: NULL operand");
  bssn::Args a{};
  int grid = 0;
  int rc = prepare(&a, Sx, Sy, Sz, 1, &grid);
  if (rc) return rc;
  a.F = F; a.S = S; a.OUT = OUT;
  return launch_single(3, bssn::MODE_CON, a, static_cast<cudaStream_t>(stream), grid);
}

size_t bssn_b200_norms_scratch_bytes(void) {
  int sms = 0;
  if (device_sms(&sms)) return 0;
  return (size_t)sms * 2 * sizeof(double);
}

int bssn_b200_constraint_norms(void* stream, const double* F, const double* S, long long Sx,
                               long long Sy, long long Sz, int ng, double* scratch,
                               size_t scratch_bytes, double* OUT2) {
  if (!F || !S || !OUT2) return fail(BSSN_B200_EINVAL, "constraint_norms: NULL operand");
  if (ng < 0 || 2LL * ng >= Sx || 2LL * ng >= Sy || 2LL * ng >= Sz)
    return fail(BSSN_B200_EINVAL, "constraint_norms: the interior [ng, S-ng) is empty");
  bssn::Args a{};
  int grid = 0;
  int rc = prepare(&a, Sx, Sy, Sz, 1, &grid);
  if (rc) return rc;
  if (!scratch) return fail(BSSN_B200_EINVAL, "constraint_norms: scratch is NULL");
  if (scratch_bytes < (size_t)grid * 2 * sizeof(double))
    return fail(BSSN_B200_EINVAL, "constraint_norms: scratch smaller than bssn_b200_norms_scratch_bytes()");
  a.F = F; a.S = S; a.ng = ng; a.partials = scratch;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  rc = launch_single(3, bssn::MODE_NORM, a, st, grid);
  if (rc) return rc;
  const double count = (double)(Sx - 2 * ng) * (double)(Sy - 2 * ng) * (double)(Sz - 2 * ng);
  bssn::norm_finalize_kernel<<<1, 32, 0, st>>>(scratch, grid, count, OUT2);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail("norm_finalize launch", e);
  return 0;
}

int bssn_b200_constraint_norms_static(void* stream, const double* F, const double* S, long long Sx,
                                      long long Sy, long long Sz, int ng, double* OUT2) {
  if (!F || !S || !OUT2) return fail(BSSN_B200_EINVAL, "constraint_norms_static: NULL operand");
  if (ng < 0 || 2LL * ng >= Sx || 2LL * ng >= Sy || 2LL * ng >= Sz)
    return fail(BSSN_B200_EINVAL, "constraint_norms_static: the interior [ng, S-ng) is empty");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail("cudaGetDevice", e);
  if (dev < 0 || dev >= kMaxDev) return fail(BSSN_B200_EINVAL, "constraint_norms_static: device ordinal out of range");
  // In host code g_static_norm_partials names a host-side stand-in, not device
  // memory: resolve its address on this device once, with the device current.
  // Two host threads that race here resolve the same address; the atomic slot
  // makes the publication well defined.
  static std::atomic<double*> addr[kMaxDev];
  double* partials = addr[dev].load(std::memory_order_acquire);
  if (!partials) {
    e = cudaGetSymbolAddress(reinterpret_cast<void**>(&partials), bssn::g_static_norm_partials);
    if (e != cudaSuccess) return cuda_fail("cudaGetSymbolAddress(static norm partials)", e);
    addr[dev].store(partials, std::memory_order_release);
  }
  bssn::Args a{};
  int grid = 0;
  int rc = prepare(&a, Sx, Sy, Sz, 1, &grid);
  if (rc) return rc;
  if (grid > bssn::kStaticNormCtas)
    return fail(BSSN_B200_EINVAL, "constraint_norms_static: this launch needs " + std::to_string(grid) +
                                      " CTA partial sums but the static array holds " +
                                      std::to_string(bssn::kStaticNormCtas) +
                                      "; use bssn_b200_constraint_norms with a caller buffer");
  return bssn_b200_constraint_norms(stream, F, S, Sx, Sy, Sz, ng, partials,
                                    sizeof(double) * 2 * bssn::kStaticNormCtas, OUT2);
}

int bssn_b200_rk4_stage(void* stream, int stage, const double* U, const double* Y, double* ACC,
                        double* YNEXT, const double* S, double ko_sigma, int ko_order,
                        double chi_floor, double alpha_floor, long long Sx, long long Sy, long long Sz) {
  if (stage < 0 || stage > 3) return fail(BSSN_B200_EINVAL, "rk4_stage: stage must be 0..3");
  if (!U || !Y || !ACC || !YNEXT || !S) return fail(BSSN_B200_EINVAL, "rk4_stage: NULL operand");
  if (YNEXT == Y) return fail(BSSN_B200_EINVAL, "rk4_stage: YNEXT must not alias Y");
  if (stage < 3 && YNEXT == U) return fail(BSSN_B200_EINVAL, "rk4_stage: YNEXT may alias U only at stage 3");
  if (ACC == Y || ACC == U || ACC == YNEXT) return fail(BSSN_B200_EINVAL, "rk4_stage: ACC must not alias another operand");
  const bool use_ko = ko_sigma > 0.0;
  if (use_ko && ko_order != 6 && ko_order != 8) return fail(BSSN_B200_EINVAL, "rk4_stage: ko_order must be 6 or 8");
  bssn::Args a{};
  int grid = 0;
  int rc = prepare(&a, Sx, Sy, Sz, 1, &grid);
  if (rc) return rc;
  a.F = Y; a.U = U; a.ACC = ACC; a.OUT = YNEXT; a.S = S;
  a.stage = stage;
  a.use_ko = use_ko ? 1 : 0;
  a.ko_sigma = use_ko ? ko_sigma : 0.0;
  a.chi_floor = chi_floor; a.alpha_floor = alpha_floor;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (use_ko && ko_order == 8) return launch_single(4, bssn::MODE_STAGE, a, st, grid);
  return launch_single(3, bssn::MODE_STAGE, a, st, grid);
}

int bssn_b200_msrk_stage(void* stream, int stage, const double* U, const double* Y, double* ACC,
                         double* OUT, double* OUT2, double* OUT3, const double* S, const double* coef,
                         double ko_sigma, int ko_order, double chi_floor, double alpha_floor,
                         long long Sx, long long Sy, long long Sz) {
  if (stage < 0 || stage > 2) return fail(BSSN_B200_EINVAL, "msrk_stage: stage must be 0..2");
  if (!U || !Y || !OUT || !S || !coef) return fail(BSSN_B200_EINVAL, "msrk_stage: NULL operand");
  if (stage < 2 && !ACC) return fail(BSSN_B200_EINVAL, "msrk_stage: ACC is required at stages 0 and 1");
  if (stage == 0 && (!OUT2 || !OUT3)) return fail(BSSN_B200_EINVAL, "msrk_stage: OUT2 and OUT3 are required at stage 0");
  for (int i = 0; i < 9; ++i)
    if (!std::isfinite(coef[i])) return fail(BSSN_B200_EINVAL, "msrk_stage: coefficients must be finite");
  // Y is read with its stencil halo: no output may overwrite it
  if (OUT == Y || (stage < 2 && ACC == Y) || (stage == 0 && (OUT2 == Y || OUT3 == Y)))
    return fail(BSSN_B200_EINVAL, "msrk_stage: an output aliases the stage input Y");
  if (stage == 0) {
    const void* outs[4] = {ACC, OUT, OUT2, OUT3};
    for (int i = 0; i < 4; ++i) {
      if (outs[i] == U) return fail(BSSN_B200_EINVAL, "msrk_stage: stage-0 outputs must not alias U");
      for (int j = i + 1; j < 4; ++j)
        if (outs[i] == outs[j]) return fail(BSSN_B200_EINVAL, "msrk_stage: stage-0 outputs must be distinct");
    }
  } else if (stage == 1 && (ACC == U || ACC == OUT)) {
    return fail(BSSN_B200_EINVAL, "msrk_stage: ACC must not alias U or OUT at stage 1");
  }
  const bool use_ko = ko_sigma > 0.0;
  if (use_ko && ko_order != 6 && ko_order != 8) return fail(BSSN_B200_EINVAL, "msrk_stage: ko_order must be 6 or 8");
  bssn::Args a{};
  int grid = 0;
  int rc = prepare(&a, Sx, Sy, Sz, 1, &grid);
  if (rc) return rc;
  a.F = Y; a.U = U; a.ACC = ACC; a.OUT = OUT; a.OUT2 = OUT2; a.OUT3 = OUT3; a.S = S;
  for (int i = 0; i < 9; ++i) a.coef[i] = coef[i];
  a.ctime = stage == 0 ? 0.0 : (stage == 1 ? coef[0] + coef[1] : coef[2] + coef[3] + coef[4]);
  a.stage = stage;
  a.use_ko = use_ko ? 1 : 0;
  a.ko_sigma = use_ko ? ko_sigma : 0.0;
  a.chi_floor = chi_floor; a.alpha_floor = alpha_floor;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (use_ko && ko_order == 8) return launch_single(4, bssn::MODE_MSRK, a, st, grid);
  return launch_single(3, bssn::MODE_MSRK, a, st, grid);
}

int bssn_b200_derivatives(void* stream, const double* F, const double* S, double* DOUT,
                          double ko_sigma, int ko_order, long long Sx, long long Sy, long long Sz) {
  if (!F || !S || !DOUT) return fail(BSSN_B200_EINVAL, "derivatives: NULL operand");
  const bool use_ko = ko_sigma > 0.0;
  if (use_ko && ko_order != 6 && ko_order != 8) return fail(BSSN_B200_EINVAL, "derivatives: ko_order must be 6 or 8");
  bssn::Args a{};
  int grid = 0;
  int rc = prepare(&a, Sx, Sy, Sz, 4, &grid);
  if (rc) return rc;
  a.F = F; a.S = S; a.OUT = DOUT;
  a.use_ko = use_ko ? 1 : 0;
  a.ko_sigma = use_ko ? ko_sigma : 0.0;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (use_ko && ko_order == 8) return launch_deriv<4>(a, st, grid);
  return launch_deriv<3>(a, st, grid);
}

int bssn_b200_rhs_algebra(void* stream, const double* F, const double* D, const double* S, double* OUT,
                          long long npts) {
  if (!F || !D || !S || !OUT) return fail(BSSN_B200_EINVAL, "rhs_algebra: NULL operand");
  if (npts < 1 || npts > (1LL << 31) - 1) return fail(BSSN_B200_EINVAL, "rhs_algebra: npts out of range");
  int sms = 0;
  int rc = device_sms(&sms);
  if (rc) return rc;
  long long blocks = (npts + 127) / 128;
  const long long cap = (long long)sms * 16;
  if (blocks > cap) blocks = cap;
  bssn::algebra_kernel<<<(int)blocks, 128, 0, static_cast<cudaStream_t>(stream)>>>(F, D, S, OUT, npts);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail("rhs_algebra launch", e);
  return 0;
}

int bssn_b200_batch_rk4_stage_derivs(void* stream, int stage, const double* U, const double* Y, double* ACC,
                                     double* YNEXT, const double* D, const double* S, int ko_slots,
                                     double chi_floor, double alpha_floor, const bssn_b200_block* blocks,
                                     int nblocks, const long long* pts0, long long npoints) {
  if (stage < 0 || stage > 3) return fail(BSSN_B200_EINVAL, "batch_rk4_stage_derivs: stage must be 0..3");
  if (!U || !Y || !ACC || !YNEXT || !D || !S || !blocks || !pts0)
    return fail(BSSN_B200_EINVAL, "batch_rk4_stage_derivs: NULL operand");
  if (YNEXT == Y) return fail(BSSN_B200_EINVAL, "batch_rk4_stage_derivs: YNEXT must not alias Y");
  if (stage < 3 && YNEXT == U) return fail(BSSN_B200_EINVAL, "batch_rk4_stage_derivs: YNEXT may alias U only at stage 3");
  if (ACC == Y || ACC == U || ACC == YNEXT)
    return fail(BSSN_B200_EINVAL, "batch_rk4_stage_derivs: ACC must not alias another operand");
  if (nblocks < 1 || npoints < 1) return fail(BSSN_B200_EINVAL, "batch_rk4_stage_derivs: empty block list");
  int sms = 0;
  int rc = device_sms(&sms);
  if (rc) return rc;
  long long grid = (npoints + 127) / 128;
  const long long cap = (long long)sms * 16;
  if (grid > cap) grid = cap;
  bssn::stage_derivs_kernel<<<(int)grid, 128, 0, static_cast<cudaStream_t>(stream)>>>(
      U, Y, ACC, YNEXT, D, ko_slots ? 162 : 138, S, stage, ko_slots ? 1 : 0, chi_floor, alpha_floor, blocks, nblocks,
      pts0, npoints);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail("batch_rk4_stage_derivs launch", e);
  return 0;
}

int bssn_b200_advance_time(void* stream, double* S) {
  if (!S) return fail(BSSN_B200_EINVAL, "advance_time: NULL operand");
  bssn::advance_time_kernel<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(S);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail("advance_time launch", e);
  return 0;
}

int bssn_b200_enforce(void* stream, double* U, long long npts, double chi_floor, double alpha_floor) {
  if (!U) return fail(BSSN_B200_EINVAL, "enforce: NULL operand");
  if (npts < 1) return fail(BSSN_B200_EINVAL, "enforce: npts must be >= 1");
  int sms = 0;
  int rc = device_sms(&sms);
  if (rc) return rc;
  long long blocks = (npts + 255) / 256;
  const long long cap = (long long)sms * 8;
  if (blocks > cap) blocks = cap;
  bssn::enforce_kernel<<<(int)blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(U, npts, chi_floor, alpha_floor);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail("enforce launch", e);
  return 0;
}

int bssn_b200_periodic_sync(void* stream, double* U, long long Sx, long long Sy, long long Sz, int ng) {
  if (!U) return fail(BSSN_B200_EINVAL, "periodic_sync: NULL operand");
  int rc = check_grid(Sx, Sy, Sz);
  if (rc) return rc;
  if (ng < 1 || 3LL * ng > Sx || 3LL * ng > Sy || 3LL * ng > Sz)
    return fail(BSSN_B200_EINVAL, "periodic_sync: need 1 <= ng and 3*ng <= every extent");
  int sms = 0;
  rc = device_sms(&sms);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  for (int axis = 0; axis < 3; ++axis) {
    bssn::periodic_axis_kernel<<<sms * 4, 256, 0, st>>>(U, Sx, Sy, Sz, axis, ng);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail("periodic_sync launch", e);
  }
  return 0;
}

}  // extern "C"

// bssn_b200 — fused BSSN right-hand side and RK4 stage kernels for sm_100a,
// behind the C ABI of include/bssn_b200.h.
//
// One persistent kernel per RHS evaluation. Each CTA takes 4x4x16-point tiles
// of the padded grid in turn; per tile it
//   1. stages each of the 24 fields' haloed tile in shared memory
//      (cp.async, double-buffered: field f+1 streams in while field f is
//      differentiated) and writes the 138 derivatives (+24 Kreiss-Oliger
//      sums) of its own point to a per-CTA scratch slab that stays in L2,
//   2. runs the register-scheduled BSSN algebra (algebra.cuh), reading the
//      derivatives of its point back from the slab at their point of use,
//   3. finishes in an epilogue that either stores the RHS or performs the
//      RK4 stage update (with algebraic enforcement fused into stage 3).
// Stencils follow 3D/src/bssn3d/derivative_bundle.py:31-48 and
// common/src/mcs_common/derivatives.py:78-106: pre-scaled taps summed from
// the lowest offset, index clamped at the array ends, mixed second
// derivatives as a first derivative along the lower axis then the higher.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/bssn_b200.h"
#include "algebra.cuh"

namespace bssn {

constexpr int TX = 4, TY = 4, TZ = 16;
constexpr int TILE = TX * TY * TZ;  // 256 points, one per thread
constexpr int NTHREADS = TILE;
constexpr int NSLOT = NDERIV + NFIELD;  // 138 derivatives + 24 KO sums
constexpr int HZP = 24;                 // z pitch of a staged tile (16 + 2*4, 8 mod 16)
constexpr int NSCAL = 16;

enum Mode : int { MODE_DERIV = 0, MODE_RHS = 1, MODE_STAGE = 2 };

struct Args {
  const double* F;      // stage input (24, n)
  const double* U;      // u_n (stage mode)
  double* ACC;          // accumulator (stage mode)
  double* OUT;          // RHS (rhs mode), next stage / new state (stage mode), derivatives (deriv mode)
  const double* S;      // 16 scalars (device)
  double* scratch;      // per-CTA slabs [grid][NSLOT][TILE]
  long long Sx, Sy, Sz, n;
  int ntx, nty, ntz;
  int stage;
  int use_ko;
  double ko_sigma;
  double chi_floor, alpha_floor;
};

// Stencil weights, pre-scaled on the device from S like derivatives.py:78-81.
struct Weights {
  double w1[3][7];
  double w2[3][7];
  double wko[3][9];
};

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

template <int R>
struct TileGeom {
  static constexpr int HX = TX + 2 * R, HY = TY + 2 * R, HZ = TZ + 2 * R;
  static constexpr int SX = HY * HZP, SY = HZP;
  static constexpr int VOL = HX * HY * HZP;  // doubles per staged buffer
  static constexpr int NELEM = HX * HY * HZ; // staged elements
  static constexpr int PER_THREAD = (NELEM + NTHREADS - 1) / NTHREADS;
};

// Issue the cp.async copies that stage field f's haloed tile (clamped indices).
template <int R>
__device__ __forceinline__ void stage_field(double* buf, const double* __restrict__ Ff,
                                           const int (&goff)[TileGeom<R>::PER_THREAD],
                                           const int (&soff)[TileGeom<R>::PER_THREAD]) {
#pragma unroll
  for (int e = 0; e < TileGeom<R>::PER_THREAD; ++e)
    if (soff[e] >= 0) cp_async8(buf + soff[e], Ff + goff[e]);
}

// Derivatives of one field at one point from the staged tile.
template <int R>
__device__ __forceinline__ void field_derivs(const double* __restrict__ t, int c, int f,
                                             const Weights& W, bool ko, double* __restrict__ slab,
                                             long long slot_stride) {
  constexpr int st[3] = {TileGeom<R>::SX, TileGeom<R>::SY, 1};
  // first derivatives (the zero centre tap of the 6th-order stencil is skipped)
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    double acc = 0.0;
#pragma unroll
    for (int k = 0; k < 7; ++k)
      if (k != 3) acc += W.w1[a][k] * t[c + (k - 3) * st[a]];
    slab[(long long)d1(f, a) * slot_stride] = acc;
  }
  const bool has2 = (f <= F_CHI) || (f >= F_GT && f < F_AT);
  if (has2) {
    const int m = g2slot(f);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      double acc = 0.0;
#pragma unroll
      for (int k = 0; k < 7; ++k) acc += W.w2[a][k] * t[c + (k - 3) * st[a]];
      slab[(long long)(72 + 6 * m + sym(a, a)) * slot_stride] = acc;
    }
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = i + 1; j < 3; ++j) {
        double acc = 0.0;
#pragma unroll
        for (int b = 0; b < 7; ++b) {
          if (b == 3) continue;
          double inner = 0.0;
#pragma unroll
          for (int a = 0; a < 7; ++a)
            if (a != 3) inner += W.w1[i][a] * t[c + (a - 3) * st[i] + (b - 3) * st[j]];
          acc += W.w1[j][b] * inner;
        }
        slab[(long long)(72 + 6 * m + sym(i, j)) * slot_stride] = acc;
      }
  }
  if (ko) {
    double acc = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      double s = 0.0;
#pragma unroll
      for (int k = 0; k <= 2 * R; ++k) s += W.wko[a][k] * t[c + (k - R) * st[a]];
      acc += s;
    }
    slab[(long long)(NDERIV + f) * slot_stride] = acc;
  }
}

__device__ __forceinline__ Params load_params(const double* __restrict__ S) {
  Params P;
  P.eta = S[0]; P.cahd_c = S[1]; P.dt = S[2]; P.dx = S[3];
  P.ssl_h = S[4]; P.ssl_sigma = S[5]; P.t = S[6];
  P.lam0 = S[7]; P.lam1 = S[8]; P.lam2 = S[9]; P.lam3 = S[10];
  P.lamf0 = S[11]; P.lamf1 = S[12];
  P.hx = S[13]; P.hy = S[14]; P.hz = S[15];
  return P;
}

template <int R, int MODE>
__global__ void __launch_bounds__(NTHREADS, 1) fused_kernel(const Args args) {
  using Geo = TileGeom<R>;
  extern __shared__ __align__(16) double smem[];
  double* buf0 = smem;
  double* buf1 = smem + Geo::VOL;
  __shared__ Weights W;

  const int tid = threadIdx.x;
  const long long Sx = args.Sx, Sy = args.Sy, Sz = args.Sz, n = args.n;
  if (tid < 3) {
    const int a = tid;
    const double h = args.S[13 + a];
    const double c1[7] = {-1, 9, -45, 0, 45, -9, 1};
    const double c2[7] = {2, -27, 270, -490, 270, -27, 2};
    const double k6[7] = {1, -6, 15, -20, 15, -6, 1};
    const double k8[9] = {-1, 8, -28, 56, -70, 56, -28, 8, -1};
    const double f1 = 1.0 / h, f2 = 1.0 / (h * h), fk = args.ko_sigma / h;
    for (int k = 0; k < 7; ++k) {
      W.w1[a][k] = (c1[k] / 60.0) * f1;
      W.w2[a][k] = (c2[k] / 180.0) * f2;
    }
    for (int k = 0; k < 9; ++k) W.wko[a][k] = 0.0;
    if (R == 4)
      for (int k = 0; k < 9; ++k) W.wko[a][k] = (k8[k] / 256.0) * fk;
    else
      for (int k = 0; k < 7; ++k) W.wko[a][k] = (k6[k] / 64.0) * fk;
  }
  __syncthreads();

  const int lz = tid & (TZ - 1), ly = (tid >> 4) & (TY - 1), lx = tid >> 6;
  const int c = (lx + R) * Geo::SX + (ly + R) * Geo::SY + (lz + R);
  const int ntiles = args.ntx * args.nty * args.ntz;
  double* slab_cta = args.scratch + (long long)blockIdx.x * NSLOT * TILE;
  const bool ko = args.use_ko != 0;

  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int tz = tile % args.ntz;
    const int ty = (tile / args.ntz) % args.nty;
    const int tx = tile / (args.ntz * args.nty);
    const long long x0 = (long long)tx * TX, y0 = (long long)ty * TY, z0 = (long long)tz * TZ;
    const long long gx = x0 + lx, gy = y0 + ly, gz = z0 + lz;
    const bool inside = gx < Sx && gy < Sy && gz < Sz;
    const long long gidx = (gx * Sy + gy) * Sz + gz;

    // per-thread staged-element offsets (the same for every field)
    int goff[Geo::PER_THREAD], soff[Geo::PER_THREAD];
#pragma unroll
    for (int e = 0; e < Geo::PER_THREAD; ++e) {
      const int idx = tid + e * NTHREADS;
      if (idx < Geo::NELEM) {
        const int hz = idx % Geo::HZ;
        const int hy = (idx / Geo::HZ) % Geo::HY;
        const int hx = idx / (Geo::HZ * Geo::HY);
        const long long qx = clampll(x0 - R + hx, Sx - 1);
        const long long qy = clampll(y0 - R + hy, Sy - 1);
        const long long qz = clampll(z0 - R + hz, Sz - 1);
        goff[e] = (int)((qx * Sy + qy) * Sz + qz);
        soff[e] = hx * Geo::SX + hy * Geo::SY + hz;
      } else {
        goff[e] = 0;
        soff[e] = -1;
      }
    }

    double* slab;
    long long slot_stride;
    if (MODE == MODE_DERIV) {
      slab = args.OUT + gidx;
      slot_stride = n;
    } else {
      slab = slab_cta + tid;
      slot_stride = TILE;
    }

    // ---- phase 1: derivatives, field by field -------------------------
    stage_field<R>(buf0, args.F, goff, soff);
    cp_async_commit();
    for (int f = 0; f < NFIELD; ++f) {
      double* cur = (f & 1) ? buf1 : buf0;
      double* nxt = (f & 1) ? buf0 : buf1;
      if (f + 1 < NFIELD) {
        stage_field<R>(nxt, args.F + (long long)(f + 1) * n, goff, soff);
        cp_async_commit();
        cp_async_wait<1>();
      } else {
        cp_async_wait<0>();
      }
      __syncthreads();
      if (inside) field_derivs<R>(cur, c, f, W, ko, slab, slot_stride);
      __syncthreads();
    }
    if (MODE == MODE_DERIV || !inside) continue;

    // ---- phase 2: algebra + epilogue ------------------------------------
    Params P = load_params(args.S);
    const double* __restrict__ Fp = args.F + gidx;
    const double* __restrict__ sl = slab;
    auto fld = [&](int k) -> double { return __ldg(Fp + (long long)k * n); };
    auto drv = [&](int s) -> double { return sl[s * TILE]; };
    if (MODE == MODE_RHS) {
      double* O = args.OUT + gidx;
      auto emit = [&](int k, double v) { O[(long long)k * n] = v; };
      rhs_point(fld, drv, emit, P);
    } else {
      const int stage = args.stage;
      const double dt = P.dt;
      const double cs = stage == 0 ? 0.0 : (stage == 3 ? 1.0 : 0.5);
      P.t = P.t + cs * dt;
      const double hstep = (stage == 2) ? dt : 0.5 * dt;
      const double w6 = dt / 6.0;
      const double* __restrict__ Up = args.U + gidx;
      double* A = args.ACC + gidx;
      double* O = args.OUT + gidx;
      double en[14];  // stage 3: gt0..5, At0..5, chi, alpha held for enforcement
#pragma unroll
      for (int q = 0; q < 14; ++q) en[q] = 0.0;
      auto emit = [&](int k, double v) {
        const double rate = ko ? v + sl[(NDERIV + k) * TILE] : v;
        const double u = Up[(long long)k * n];
        if (stage == 0) {
          A[(long long)k * n] = rate;
          O[(long long)k * n] = u + hstep * rate;
        } else if (stage < 3) {
          A[(long long)k * n] = A[(long long)k * n] + 2.0 * rate;
          O[(long long)k * n] = u + hstep * rate;
        } else {
          const double un = u + w6 * (A[(long long)k * n] + rate);
          if (k >= F_GT && k < F_GT + 6) en[k - F_GT] = un;
          else if (k >= F_AT && k < F_AT + 6) en[6 + k - F_AT] = un;
          else if (k == F_CHI) en[12] = un;
          else if (k == F_ALPHA) en[13] = un;
          else O[(long long)k * n] = un;
        }
      };
      rhs_point(fld, drv, emit, P);
      if (stage == 3) {
        // algebraic enforcement, evolve.py:93-119
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
        O[(long long)F_CHI * n] = fmax(en[12], args.chi_floor);
        O[(long long)F_ALPHA * n] = fmax(en[13], args.alpha_floor);
      }
    }
  }
}

// t <- t + dt in the device scalar pack, between captured RK4 steps
// (the fori_loop carry update of 3D/src/bssn3d/evolve.py:186-193).
__global__ void advance_time_kernel(double* S) {
  if (threadIdx.x == 0 && blockIdx.x == 0) S[6] = S[6] + S[2];
}

// Algebra only: derivatives supplied by the caller (the reference's
// algebra-only microbenchmark interface, 3D/src/bssn3d/cuda/microbench_algebra.cu).
__global__ void __launch_bounds__(128) algebra_kernel(const double* __restrict__ F, const double* __restrict__ D,
                                                      const double* __restrict__ S, double* __restrict__ OUT,
                                                      long long n) {
  const Params P = load_params(S);
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    auto fld = [&](int k) -> double { return __ldg(F + (long long)k * n + q); };
    auto drv = [&](int s) -> double { return __ldg(D + (long long)s * n + q); };
    auto emit = [&](int k, double v) { OUT[(long long)k * n + q] = v; };
    rhs_point(fld, drv, emit, P);
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
  // iterate over the 2*ng ghost layers x the other two axes x 24 fields
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

struct DeviceInfo {
  int device = -1;
  int sms = 0;
  int ctas_per_sm = 1;
};

int device_info(DeviceInfo* out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail("cudaGetDevice", e);
  static thread_local DeviceInfo cache[16];
  if (dev >= 0 && dev < 16 && cache[dev].device == dev) {
    *out = cache[dev];
    return 0;
  }
  DeviceInfo d;
  d.device = dev;
  e = cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return cuda_fail("cudaDeviceGetAttribute", e);
  d.ctas_per_sm = 1;  // __launch_bounds__(256, 1) kernels: one resident CTA per SM
  if (dev >= 0 && dev < 16) cache[dev] = d;
  *out = d;
  return 0;
}

template <int R, int MODE>
int launch_fused(const bssn::Args& a, cudaStream_t stream, int grid) {
  using Geo = bssn::TileGeom<R>;
  const size_t smem = 2 * (size_t)Geo::VOL * sizeof(double);
  auto kern = bssn::fused_kernel<R, MODE>;
  static thread_local int attr_set[16] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 16 && !attr_set[dev]) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_fail("cudaFuncSetAttribute", e);
    attr_set[dev] = 1;
  }
  kern<<<grid, bssn::NTHREADS, smem, stream>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail("fused kernel launch", e);
  return 0;
}

int check_grid(long long Sx, long long Sy, long long Sz) {
  if (Sx < 1 || Sy < 1 || Sz < 1) return fail(BSSN_B200_EINVAL, "grid extents must be >= 1");
  const long long n = Sx * Sy * Sz;
  if (n > (1LL << 31) - 1) return fail(BSSN_B200_EINVAL, "grid has more than 2^31-1 points");
  if ((long long)bssn::NFIELD * n > (1LL << 40)) return fail(BSSN_B200_EINVAL, "grid too large");
  return 0;
}

int prepare(bssn::Args* a, long long Sx, long long Sy, long long Sz, int* grid) {
  int rc = check_grid(Sx, Sy, Sz);
  if (rc) return rc;
  DeviceInfo d;
  rc = device_info(&d);
  if (rc) return rc;
  a->Sx = Sx; a->Sy = Sy; a->Sz = Sz;
  a->n = Sx * Sy * Sz;
  a->ntx = (int)((Sx + bssn::TX - 1) / bssn::TX);
  a->nty = (int)((Sy + bssn::TY - 1) / bssn::TY);
  a->ntz = (int)((Sz + bssn::TZ - 1) / bssn::TZ);
  const long long ntiles = (long long)a->ntx * a->nty * a->ntz;
  const long long cap = (long long)d.sms * d.ctas_per_sm;
  *grid = (int)(ntiles < cap ? ntiles : cap);
  return 0;
}

size_t scratch_for(const DeviceInfo& d) {
  return (size_t)d.sms * d.ctas_per_sm * bssn::NSLOT * bssn::TILE * sizeof(double);
}

int check_scratch(void* scratch, size_t bytes) {
  DeviceInfo d;
  int rc = device_info(&d);
  if (rc) return rc;
  if (!scratch) return fail(BSSN_B200_ESCRATCH, "scratch pointer is NULL");
  if (bytes < scratch_for(d))
    return fail(BSSN_B200_ESCRATCH, "scratch buffer smaller than bssn_b200_scratch_bytes()");
  if ((reinterpret_cast<uintptr_t>(scratch) & 15) != 0) return fail(BSSN_B200_EINVAL, "scratch not 16-byte aligned");
  return 0;
}

}  // namespace

extern "C" {

const char* bssn_b200_last_error(void) { return g_err.c_str(); }

const char* bssn_b200_version(void) { return "bssn_b200 0.1 sm_100a"; }

size_t bssn_b200_scratch_bytes(int ko_order) {
  (void)ko_order;
  DeviceInfo d;
  if (device_info(&d)) return 0;
  return scratch_for(d);
}

int bssn_b200_rhs(void* stream, const double* F, const double* S, double* OUT, long long Sx,
                  long long Sy, long long Sz, void* scratch, size_t scratch_bytes) {
  if (!F || !S || !OUT) return fail(BSSN_B200_EINVAL, "rhs: NULL operand");
  bssn::Args a{};
  int grid = 0;
  int rc = prepare(&a, Sx, Sy, Sz, &grid);
  if (rc) return rc;
  rc = check_scratch(scratch, scratch_bytes);
  if (rc) return rc;
  a.F = F; a.S = S; a.OUT = OUT;
  a.scratch = static_cast<double*>(scratch);
  a.use_ko = 0; a.ko_sigma = 0.0;
  return launch_fused<3, bssn::MODE_RHS>(a, static_cast<cudaStream_t>(stream), grid);
}

int bssn_b200_rk4_stage(void* stream, int stage, const double* U, const double* Y, double* ACC,
                        double* YNEXT, const double* S, double ko_sigma, int ko_order,
                        double chi_floor, double alpha_floor, long long Sx, long long Sy, long long Sz,
                        void* scratch, size_t scratch_bytes) {
  if (stage < 0 || stage > 3) return fail(BSSN_B200_EINVAL, "rk4_stage: stage must be 0..3");
  if (!U || !Y || !ACC || !YNEXT || !S) return fail(BSSN_B200_EINVAL, "rk4_stage: NULL operand");
  if (YNEXT == Y) return fail(BSSN_B200_EINVAL, "rk4_stage: YNEXT must not alias Y");
  if (stage < 3 && YNEXT == U) return fail(BSSN_B200_EINVAL, "rk4_stage: YNEXT may alias U only at stage 3");
  const bool use_ko = ko_sigma > 0.0;
  if (use_ko && ko_order != 6 && ko_order != 8) return fail(BSSN_B200_EINVAL, "rk4_stage: ko_order must be 6 or 8");
  bssn::Args a{};
  int grid = 0;
  int rc = prepare(&a, Sx, Sy, Sz, &grid);
  if (rc) return rc;
  rc = check_scratch(scratch, scratch_bytes);
  if (rc) return rc;
  a.F = Y; a.U = U; a.ACC = ACC; a.OUT = YNEXT; a.S = S;
  a.scratch = static_cast<double*>(scratch);
  a.stage = stage;
  a.use_ko = use_ko ? 1 : 0;
  a.ko_sigma = use_ko ? ko_sigma : 0.0;
  a.chi_floor = chi_floor; a.alpha_floor = alpha_floor;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (use_ko && ko_order == 8) return launch_fused<4, bssn::MODE_STAGE>(a, st, grid);
  return launch_fused<3, bssn::MODE_STAGE>(a, st, grid);
}

int bssn_b200_derivatives(void* stream, const double* F, const double* S, double* DOUT,
                          double ko_sigma, int ko_order, long long Sx, long long Sy, long long Sz) {
  if (!F || !S || !DOUT) return fail(BSSN_B200_EINVAL, "derivatives: NULL operand");
  const bool use_ko = ko_sigma > 0.0;
  if (use_ko && ko_order != 6 && ko_order != 8) return fail(BSSN_B200_EINVAL, "derivatives: ko_order must be 6 or 8");
  bssn::Args a{};
  int grid = 0;
  int rc = prepare(&a, Sx, Sy, Sz, &grid);
  if (rc) return rc;
  a.F = F; a.S = S; a.OUT = DOUT;
  a.scratch = nullptr;
  a.use_ko = use_ko ? 1 : 0;
  a.ko_sigma = use_ko ? ko_sigma : 0.0;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (use_ko && ko_order == 8) return launch_fused<4, bssn::MODE_DERIV>(a, st, grid);
  return launch_fused<3, bssn::MODE_DERIV>(a, st, grid);
}

int bssn_b200_rhs_algebra(void* stream, const double* F, const double* D, const double* S, double* OUT,
                          long long npts) {
  if (!F || !D || !S || !OUT) return fail(BSSN_B200_EINVAL, "rhs_algebra: NULL operand");
  if (npts < 1 || npts > (1LL << 31) - 1) return fail(BSSN_B200_EINVAL, "rhs_algebra: npts out of range");
  DeviceInfo d;
  int rc = device_info(&d);
  if (rc) return rc;
  long long blocks = (npts + 127) / 128;
  const long long cap = (long long)d.sms * 16;
  if (blocks > cap) blocks = cap;
  bssn::algebra_kernel<<<(int)blocks, 128, 0, static_cast<cudaStream_t>(stream)>>>(F, D, S, OUT, npts);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail("rhs_algebra launch", e);
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
  DeviceInfo d;
  int rc = device_info(&d);
  if (rc) return rc;
  long long blocks = (npts + 255) / 256;
  const long long cap = (long long)d.sms * 8;
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
  DeviceInfo d;
  rc = device_info(&d);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  for (int axis = 0; axis < 3; ++axis) {
    bssn::periodic_axis_kernel<<<d.sms * 4, 256, 0, st>>>(U, Sx, Sy, Sz, axis, ng);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail("periodic_sync launch", e);
  }
  return 0;
}

}  // extern "C"

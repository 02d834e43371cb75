// Ozaki-style INT8 derivative path on the sm_100a tensor cores (tcgen05).
//
// Every finite-difference stencil of the BSSN bundle is a banded matrix with
// small integer coefficients (C1 x60, C2 x180, KO6 x64, KO8 x256). A float64
// field is split, line by line along the differentiation axis, into k signed
// INT8 digits under one shared power-of-two exponent per line,
//     f = 2^e * sum_s q_s 2^(-7(s+1)),   |q_s| <= 64,   |f| 2^-e < 1/2,
// the stencil is applied to every digit plane as an exact INT8 x INT8 -> INT32
// tensor-core contraction, and the digit results are recombined in float64.
// The contraction is exact and the recombination order is fixed, so results
// are bit-reproducible run to run; the only approximation is the split
// (|residual| <= 2^(e-7k-1) per value, e the window's exponent).
//
// This follows the banded-integer-stencil design of the reference's MCS
// Ozaki derivative (2D/src/mcs2d/schemes/ozaki.py:286-323: stencil matrix,
// exact integer accumulation, per-block exponent, float64 reconstruction),
// with Ozaki-I digit slicing instead of the reference's RNS residues; the
// reference has no Ozaki path for BSSN.
//
// Layout of one pass (one field, one axis): the lines of the array along the
// axis are the rows (M) of the product, the positions along the line are K,
// and the 16 outputs of a tile times 4 stencils (C1, C2 high digit, C2 low
// digit, KO) are N = 64. A tile is 128 lines x 16 outputs; its K window is 32
// positions (16 outputs + up to 2x4 halo, the rest zero), one tcgen05.mma
// (M=128, N=64, K=32, kind::i8) per digit plane into its own 64 TMEM columns.
// Operands sit in shared memory in the canonical no-swizzle K-major layout
// (8-row x 16-byte core matrices); the banded B matrix is built once per CTA.
// The exponent is shared by the window of one line in one tile (the
// reference shares one per block, ozaki.py:316-323); the digit planes are
// made in shared memory from the float64 window and never touch HBM.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/bssn_b200.h"

namespace ozaki {

constexpr int MAXK = 8;
constexpr int LT = 128;           // lines per tile (MMA M)
constexpr int NO = 16;            // outputs per tile along the axis
constexpr int KW = 32;            // K window in padded positions
constexpr int NCOL = 4 * NO;      // MMA N: C1 | C2 hi | C2 lo | KO
constexpr long long WAIT_LIMIT = 1LL << 26;  // bounded mbarrier polls (~1 s)

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Canonical no-swizzle K-major offset of (row, kbyte) in a rows x 32-byte operand.
__host__ __device__ constexpr int canon(int r, int kb, int rows) {
  return (kb >> 4) * (rows * 16) + (r >> 3) * 128 + (r & 7) * 16 + (kb & 15);
}

// Shared-memory matrix descriptor: start, leading (K-chunk) and stride
// (8-row group) byte offsets, Blackwell version bit, no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | ((uint64_t)1 << 46);
}

// Instruction descriptor: S32 accumulator, signed INT8 A and B, both K-major, N=64, M=128.
constexpr uint32_t IDESC = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(NCOL >> 3) << 17) | ((128u >> 4) << 24);

struct Line {
  int len;           // points along the axis
  long long nlines;  // product of the other two extents
  long long stride;  // element stride along the axis
};

__host__ __device__ inline Line line_geom(int axis, long long Sx, long long Sy, long long Sz) {
  Line L;
  if (axis == 0) { L.len = (int)Sx; L.nlines = Sy * Sz; L.stride = Sy * Sz; }
  else if (axis == 1) { L.len = (int)Sy; L.nlines = Sx * Sz; L.stride = Sz; }
  else { L.len = (int)Sz; L.nlines = Sx * Sy; L.stride = 1; }
  return L;
}

// Offset of the first element of line l (lines ordered with z fastest).
__device__ __forceinline__ long long line_base(int axis, long long l, long long Sy, long long Sz) {
  if (axis == 0) return l;                                   // l = y*Sz + z
  if (axis == 1) return (l / Sz) * Sy * Sz + (l % Sz);       // l = x*Sz + z
  return l * Sz;                                             // l = x*Sy + y
}

// ---- fused split + contraction + recombination -----------------------------
// One CTA (256 threads) per SM walks tiles of 128 lines x 16 outputs of one
// pass. Per tile: the float64 window of each line (16 outputs + 2R halo,
// edge-clamped) lands in shared memory by cp.async, laid out so that the
// copies are coalesced (line-contiguous windows for the z axis, line-
// interleaved for x and y); each line gets one power-of-two exponent for its
// window and two threads per line write its k digit planes straight into the
// canonical operand layout; thread 0 issues the k contractions; the two
// warpgroups read 8 outputs each back from TMEM and recombine them
// smallest digit first; the outputs go out through shared memory so that the
// stores are coalesced as well. The next tile's window is prefetched while a
// tile is contracted.
constexpr int FT = 256;       // threads of the fused kernel
constexpr int FW = 33;        // float64 window pitch (conflict-free rows)
constexpr int OP = 17;        // output staging pitch

struct FusedArgs {
  const double* src;
  int axis;
  long long Sx, Sy, Sz;
  int R, k, ko_reach;
  const double* S;
  double ko_sigma;
  double* d1;
  double* d2;
  double* ko;
  int ko_add;
  int* err;
};

struct FusedSmem {
  int8_t B[NCOL * KW];
  int8_t A[MAXK][LT * KW];
  double F[2][LT * FW];
  double O[3][LT * OP];
  long long base[2][LT];  // first element of each line of the tile in F[buf]
};

__device__ __forceinline__ void cp_async8(double* dst, const double* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}

template <int R, int AXIS>
__global__ void __launch_bounds__(FT, 1) fused_kernel(const FusedArgs a) {
  extern __shared__ __align__(128) unsigned char fsm_raw[];
  FusedSmem& sm = *reinterpret_cast<FusedSmem*>(fsm_raw);
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid >> 5;
  if (smem_u32(fsm_raw) & 127u) {  // operand layouts need an aligned base: refuse rather than misplace
    if (tid == 0) atomicExch(a.err, 1);
    return;
  }
  const Line L = line_geom(AXIS, a.Sx, a.Sy, a.Sz);
  constexpr int KWL = NO + 2 * R;  // window positions the stencils use (22 or 24)
  const double h = a.S[13 + AXIS];
  const double w1 = (1.0 / 60.0) * (1.0 / h);
  const double w2 = (1.0 / 180.0) * (1.0 / (h * h));
  const double wko = (1.0 / (R == 4 ? 256.0 : 64.0)) * (a.ko_sigma / h);
  {
    const int c1[7] = {-1, 9, -45, 0, 45, -9, 1};
    const int c2h[7] = {0, 0, 2, -4, 2, 0, 0};       // 270 = 2*128 + 14, -490 = -4*128 + 22
    const int c2l[7] = {2, -27, 14, 22, 14, -27, 2};
    const int k6[7] = {1, -6, 15, -20, 15, -6, 1};
    const int k8[9] = {-1, 8, -28, 56, -70, 56, -28, 8, -1};
    for (int i = tid; i < NCOL * KW; i += FT) {
      const int n = i / KW, kb = i % KW;
      const int st = n / NO, o = n % NO;
      const int j = kb - R - o;
      int v = 0;
      if (st < 3) {
        if (j >= -3 && j <= 3) v = st == 0 ? c1[j + 3] : (st == 1 ? c2h[j + 3] : c2l[j + 3]);
      } else if (R == 4) {
        if (j >= -4 && j <= 4) v = k8[j + 4];
      } else {
        if (j >= -3 && j <= 3) v = k6[j + 3];
      }
      sm.B[canon(n, kb, NCOL)] = (int8_t)v;
    }
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&mbar)));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_base)),
                 "r"(512));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = tmem_base;

  const long long nlb = (L.nlines + LT - 1) / LT;
  const int nzt = (L.len + NO - 1) / NO;
  const long long ntiles = nlb * nzt;
  constexpr bool zaxis = AXIS == 2;
  // the window of tile t into F[buf] (edge-clamped positions, tail lines repeat
  // the last line); the lines' first elements are tabled once per tile. Ends
  // in a barrier-free state: callers place it right after a barrier.
  auto load_window = [&](long long t, int buf) {
    const long long lb = t / nzt;
    const int z0 = (int)(t % nzt) * NO;
    if (tid < LT) {
      long long l = lb * LT + tid;
      if (l >= L.nlines) l = L.nlines - 1;
      sm.base[buf][tid] = line_base(AXIS, l, a.Sy, a.Sz);
    }
    __syncthreads();
    for (int i = tid; i < LT * KWL; i += FT) {
      const int r = zaxis ? i / KWL : i % LT;
      const int pos = zaxis ? i % KWL : i / LT;
      int q = z0 - R + pos;
      q = q < 0 ? 0 : (q > L.len - 1 ? L.len - 1 : q);  // edge padding (derivatives.py:83-84)
      cp_async8(&sm.F[buf][r * FW + pos], a.src + sm.base[buf][r] + (long long)q * L.stride);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  uint32_t phase = 0;
  bool failed = false;
  long long tile = blockIdx.x;
  if (tile < ntiles) load_window(tile, 0);
  int buf = 0;
  for (; tile < ntiles && !failed; tile += gridDim.x, buf ^= 1) {
    const long long lb = tile / nzt;
    const int z0 = (int)(tile % nzt) * NO;
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    // ---- exponent and digits: threads r and r + 128 take the two 16-position halves of line r ----
    const int r = tid & (LT - 1), half = tid >> 7;
    const double* Fr = &sm.F[buf][r * FW];
    double m0 = 0.0, m1 = 0.0;
#pragma unroll
    for (int pos = 0; pos < KWL; pos += 2) {
      m0 = fmax(m0, fabs(Fr[pos]));
      m1 = fmax(m1, fabs(Fr[pos + 1]));
    }
    const double m = fmax(m0, m1);
    int e = 0;
    if (m > 0.0) {
      int ex;
      frexp(m, &ex);  // m = fr * 2^ex, fr in [0.5, 1)
      e = ex + 1;     // |f| 2^-e < 1/2
    }
    const double sc = ldexp(1.0, e);
    const double isc = ldexp(1.0, -e);  // scaling by a power of two is exact
    {
      uint32_t wd[MAXK][4];
#pragma unroll
      for (int s2 = 0; s2 < MAXK; ++s2) wd[s2][0] = wd[s2][1] = wd[s2][2] = wd[s2][3] = 0u;
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int pos = 16 * half + j;
        double rr = pos < KWL ? Fr[pos] * isc : 0.0;
#pragma unroll
        for (int s2 = 0; s2 < MAXK; ++s2) {
          if (s2 < a.k) {
            const double t = rr * 128.0;
            const double d = rint(t);
            rr = t - d;
            wd[s2][j >> 2] |= (uint32_t)(uint8_t)(int8_t)(int)d << (8 * (j & 3));
          }
        }
      }
#pragma unroll
      for (int s2 = 0; s2 < MAXK; ++s2)
        if (s2 < a.k)
          *reinterpret_cast<uint4*>(&sm.A[s2][canon(r, 16 * half, LT)]) = make_uint4(wd[s2][0], wd[s2][1], wd[s2][2], wd[s2][3]);
    }
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    // ---- prefetch the next tile's window; thread 0 issues the contractions ----
    if (tile + gridDim.x < ntiles) load_window(tile + gridDim.x, buf ^ 1);
    if (tid == 0) {
      const uint64_t db = smem_desc(smem_u32(sm.B), NCOL * 16, 128);
      for (int s2 = 0; s2 < a.k; ++s2) {
        const uint64_t da = smem_desc(smem_u32(&sm.A[s2][0]), LT * 16, 128);
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem + (uint32_t)(NCOL * s2)),
            "l"(da), "l"(db), "r"(IDESC), "r"(0u));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                       smem_u32(&mbar))
                   : "memory");
    }
    uint32_t done = 0;
    for (long long it = 0; it < WAIT_LIMIT && !done; ++it) {
      asm volatile(
          "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
          : "=r"(done)
          : "r"(smem_u32(&mbar)), "r"(phase)
          : "memory");
    }
    if (__syncthreads_or(!done)) {
      if (tid == 0) atomicExch(a.err, 1);
      failed = true;
    }
    phase ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    // ---- recombine: warp w reads TMEM lanes 32 (w % 4).., outputs 8 (w / 4).. ----
    const uint32_t lane = (uint32_t)((warp & 3) * 32) << 16;
    const int oc = 8 * (warp >> 2);
    double r1[8], r2[8], rk[8];
#pragma unroll
    for (int o = 0; o < 8; ++o) { r1[o] = 0.0; r2[o] = 0.0; rk[o] = 0.0; }
    double w = ldexp(1.0, -7 * a.k);  // weight of the smallest digit plane
    for (int s2 = a.k - 1; s2 >= 0; --s2, w *= 128.0) {
      uint32_t v[4][8];
#pragma unroll
      for (int st = 0; st < 4; ++st) {
        const uint32_t addr = tmem + lane + (uint32_t)(NCOL * s2 + NO * st + oc);
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
                     : "=r"(v[st][0]), "=r"(v[st][1]), "=r"(v[st][2]), "=r"(v[st][3]), "=r"(v[st][4]),
                       "=r"(v[st][5]), "=r"(v[st][6]), "=r"(v[st][7])
                     : "r"(addr));
      }
      asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
      for (int o = 0; o < 8; ++o) {
        r1[o] += (double)(int)v[0][o] * w;
        r2[o] += (double)((int)v[1][o] * 128 + (int)v[2][o]) * w;
        rk[o] += (double)(int)v[3][o] * w;
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    // the recombining thread's line is r too (TMEM lane = line): its exponent is sc
#pragma unroll
    for (int o = 0; o < 8; ++o) {
      sm.O[0][r * OP + oc + o] = (r1[o] * sc) * w1;
      sm.O[1][r * OP + oc + o] = (r2[o] * sc) * w2;
      sm.O[2][r * OP + oc + o] = (rk[o] * sc) * wko;
    }
    __syncthreads();
    // ---- coalesced stores of the tile's outputs ----
    for (int i = tid; i < LT * NO; i += FT) {
      const int rr = zaxis ? i / NO : i % LT;
      const int o = zaxis ? i % NO : i / LT;
      const long long l = lb * LT + rr;
      const int z = z0 + o;
      if (l < L.nlines && z < L.len && !failed) {
        const long long pt = sm.base[buf][rr] + (long long)z * L.stride;
        if (a.d1) a.d1[pt] = sm.O[0][rr * OP + o];
        if (a.d2) a.d2[pt] = sm.O[1][rr * OP + o];
        if (a.ko) a.ko[pt] = a.ko_add ? a.ko[pt] + sm.O[2][rr * OP + o] : sm.O[2][rr * OP + o];
      }
    }
    __syncthreads();  // TMEM columns, digits and output staging are reused by the next tile
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(512));
}

}  // namespace ozaki

// ======================================================================
namespace {
thread_local std::string g_oz_err;

template <int R, int AXIS>
cudaError_t launch_fused(const ozaki::FusedArgs& m, int grid, cudaStream_t st, int dev) {
  static bool attr_done[64] = {false};
  constexpr int kSmem = (int)sizeof(ozaki::FusedSmem);
  if (!attr_done[dev]) {
    cudaError_t e = cudaFuncSetAttribute(ozaki::fused_kernel<R, AXIS>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmem);
    if (e != cudaSuccess) return e;
    attr_done[dev] = true;
  }
  ozaki::fused_kernel<R, AXIS><<<grid, ozaki::FT, kSmem, st>>>(m);
  return cudaSuccess;
}
int oz_fail(int code, const std::string& m) {
  g_oz_err = m;
  return code;
}
}  // namespace

extern "C" {

const char* bssn_b200_ozaki_last_error(void) { return g_oz_err.c_str(); }

size_t bssn_b200_ozaki_workspace_bytes(long long Sx, long long Sy, long long Sz, int k) {
  if (Sx < 1 || Sy < 1 || Sz < 1 || k < 1 || k > ozaki::MAXK) return 0;
  return 256;  // the error flag (the digit planes never leave shared memory)
}

int* bssn_b200_ozaki_error_flag(void* workspace, long long Sx, long long Sy, long long Sz, int k) {
  const size_t need = bssn_b200_ozaki_workspace_bytes(Sx, Sy, Sz, k);
  if (!workspace || need == 0) return nullptr;
  return reinterpret_cast<int*>(static_cast<char*>(workspace) + need - 256);
}

int bssn_b200_ozaki_derivatives(void* stream, const double* F, const double* S, double* DOUT, int k,
                                double ko_sigma, int ko_order, long long Sx, long long Sy, long long Sz,
                                void* workspace, size_t workspace_bytes) {
  if (!F || !S || !DOUT || !workspace) return oz_fail(BSSN_B200_EINVAL, "ozaki: NULL operand");
  if (k < 1 || k > ozaki::MAXK) return oz_fail(BSSN_B200_EINVAL, "ozaki: k must be 1..8");
  if (Sx < 8 || Sy < 8 || Sz < 8) return oz_fail(BSSN_B200_EINVAL, "ozaki: every extent must be >= 8");
  if (Sx * Sy * Sz > (1LL << 31)) return oz_fail(BSSN_B200_EINVAL, "ozaki: grid too large");
  const bool use_ko = ko_sigma > 0.0;
  if (use_ko && ko_order != 6 && ko_order != 8) return oz_fail(BSSN_B200_EINVAL, "ozaki: ko_order must be 6 or 8");
  const size_t need = bssn_b200_ozaki_workspace_bytes(Sx, Sy, Sz, k);
  if (workspace_bytes < need) return oz_fail(BSSN_B200_EINVAL, "ozaki: workspace smaller than bssn_b200_ozaki_workspace_bytes()");
  if ((reinterpret_cast<uintptr_t>(workspace) & 255) != 0) return oz_fail(BSSN_B200_EINVAL, "ozaki: workspace not 256-byte aligned");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int dev = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return oz_fail(BSSN_B200_ECUDA, std::string("ozaki: ") + cudaGetErrorString(e));
  // One CTA per SM: the fused kernel owns all 512 TMEM columns.
  if (dev < 0 || dev >= 64) return oz_fail(BSSN_B200_EINVAL, "ozaki: device ordinal out of range");
  int* err = bssn_b200_ozaki_error_flag(workspace, Sx, Sy, Sz, k);
  e = cudaMemsetAsync(err, 0, sizeof(int), st);
  if (e != cudaSuccess) return oz_fail(BSSN_B200_ECUDA, std::string("ozaki: ") + cudaGetErrorString(e));
  const long long n = Sx * Sy * Sz;
  const int R = (use_ko && ko_order == 8) ? 4 : 3;
  auto pass = [&](const double* src, int axis, double* d1, double* d2, double* ko, int ko_add) -> int {
    const ozaki::Line L = ozaki::line_geom(axis, Sx, Sy, Sz);
    ozaki::FusedArgs m{};
    m.src = src; m.axis = axis; m.Sx = Sx; m.Sy = Sy; m.Sz = Sz;
    m.R = R; m.k = k; m.ko_reach = R; m.S = S; m.ko_sigma = use_ko ? ko_sigma : 0.0;
    m.d1 = d1; m.d2 = d2; m.ko = ko; m.ko_add = ko_add; m.err = err;
    const long long tiles = ((L.nlines + ozaki::LT - 1) / ozaki::LT) * ((L.len + ozaki::NO - 1) / ozaki::NO);
    const int grid = (int)(tiles < sms ? tiles : sms);
    cudaError_t le;
    if (R == 4)
      le = axis == 0 ? launch_fused<4, 0>(m, grid, st, dev) : (axis == 1 ? launch_fused<4, 1>(m, grid, st, dev)
                                                                        : launch_fused<4, 2>(m, grid, st, dev));
    else
      le = axis == 0 ? launch_fused<3, 0>(m, grid, st, dev) : (axis == 1 ? launch_fused<3, 1>(m, grid, st, dev)
                                                                        : launch_fused<3, 2>(m, grid, st, dev));
    if (le == cudaSuccess) le = cudaGetLastError();
    if (le != cudaSuccess) return oz_fail(BSSN_B200_ECUDA, std::string("ozaki launch: ") + cudaGetErrorString(le));
    return 0;
  };
  auto has_d2 = [](int f) { return f == 0 || f == 1 || (f >= 3 && f < 12); };
  auto g2slot = [](int f) { return f == 0 ? 0 : (f == 1 ? 1 : (f < 9 ? 2 + f - 3 : 8 + f - 9)); };
  const int diag[3] = {0, 3, 5};
  for (int f = 0; f < 24; ++f) {
    for (int axis = 0; axis < 3; ++axis) {
      double* d1 = DOUT + (long long)(3 * f + axis) * n;
      double* d2 = has_d2(f) ? DOUT + (long long)(72 + 6 * g2slot(f) + diag[axis]) * n : nullptr;
      double* ko = use_ko ? DOUT + (long long)(138 + f) * n : nullptr;
      int rc = pass(F + (long long)f * n, axis, d1, d2, ko, axis > 0);
      if (rc) return rc;
    }
  }
  // mixed second derivatives: the first derivative along the lower axis,
  // differentiated again along the higher one (derivative_bundle.py:31-48)
  for (int f = 0; f < 24; ++f) {
    if (!has_d2(f)) continue;
    const double* tx = DOUT + (long long)(3 * f + 0) * n;
    const double* ty = DOUT + (long long)(3 * f + 1) * n;
    int rc = pass(tx, 1, DOUT + (long long)(72 + 6 * g2slot(f) + 1) * n, nullptr, nullptr, 0);
    if (!rc) rc = pass(tx, 2, DOUT + (long long)(72 + 6 * g2slot(f) + 2) * n, nullptr, nullptr, 0);
    if (!rc) rc = pass(ty, 2, DOUT + (long long)(72 + 6 * g2slot(f) + 4) * n, nullptr, nullptr, 0);
    if (rc) return rc;
  }
  return 0;
}

}  // extern "C"

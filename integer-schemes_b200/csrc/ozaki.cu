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
// (|residual| <= 2^(e-7k-1) per value).
//
// This follows the banded-integer-stencil design of the reference's MCS
// Ozaki derivative (2D/src/mcs2d/schemes/ozaki.py:286-323: stencil matrix,
// exact integer accumulation, per-block exponent, float64 reconstruction),
// with Ozaki-I digit slicing instead of the reference's RNS residues; the
// reference has no Ozaki path for BSSN.
//
// Layout of one pass (one field, one axis): the lines of the array along the
// axis are the rows (M) of the product, the padded positions along the line
// are K, and the 16 outputs of a tile times 4 stencils (C1, C2 high digit,
// C2 low digit, KO) are N = 64. A tile is 128 lines x 16 outputs; its K window
// is 32 padded positions (16 outputs + up to 2x4 halo), one tcgen05.mma
// (M=128, N=64, K=32, kind::i8) per digit plane into its own 64 TMEM columns.
// Operands sit in shared memory in the canonical no-swizzle K-major layout
// (8-row x 16-byte core matrices); the banded B matrix is built once per CTA.
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
constexpr int THREADS = 128;      // one thread per line of the tile
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

// Padded line length: >= len + 2*4 and a multiple of 16, plus one spare
// 16-position chunk so that every tile's 32-position window is in range.
__host__ __device__ constexpr int padded_len(int len) { return ((len + 15) / 16 + 1) * 16; }

// ---- split: one thread per line ------------------------------------------
__global__ void split_kernel(const double* __restrict__ f, int axis, long long Sx, long long Sy, long long Sz,
                             int R, int k, int8_t* __restrict__ Q, double* __restrict__ scale) {
  const Line L = line_geom(axis, Sx, Sy, Sz);
  const int Lp = padded_len(L.len);
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < L.nlines;
       l += (long long)gridDim.x * blockDim.x) {
    const double* p = f + line_base(axis, l, Sy, Sz);
    double m = 0.0;
    for (int i = 0; i < L.len; ++i) m = fmax(m, fabs(p[(long long)i * L.stride]));
    int e = 0;
    if (m > 0.0) {
      int ex;
      frexp(m, &ex);  // m = fr * 2^ex, fr in [0.5, 1)
      e = ex + 1;     // |f| 2^-e < 1/2
    }
    scale[l] = ldexp(1.0, e);
    for (int c = 0; c < Lp / 16; ++c) {
      uint32_t w[MAXK][4];
#pragma unroll
      for (int s = 0; s < MAXK; ++s) w[s][0] = w[s][1] = w[s][2] = w[s][3] = 0u;
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int zp = 16 * c + i;
        double v = 0.0;
        if (zp < L.len + 2 * R) {
          int q = zp - R;
          q = q < 0 ? 0 : (q > L.len - 1 ? L.len - 1 : q);  // edge padding (derivatives.py:83-84)
          v = p[(long long)q * L.stride];
        }
        double r = ldexp(v, -e);
#pragma unroll
        for (int s = 0; s < MAXK; ++s) {
          if (s < k) {
            const double t = r * 128.0;
            const double d = rint(t);
            r = t - d;
            const uint32_t byte = (uint32_t)(uint8_t)(int8_t)(int)d;
            w[s][i >> 2] |= byte << (8 * (i & 3));
          }
        }
      }
#pragma unroll
      for (int s = 0; s < MAXK; ++s) {
        if (s < k) {
          uint4* dst = reinterpret_cast<uint4*>(Q + ((long long)s * L.nlines + l) * Lp + 16 * c);
          *dst = make_uint4(w[s][0], w[s][1], w[s][2], w[s][3]);
        }
      }
    }
  }
}

// ---- contraction + recombination -------------------------------------------
struct MmaArgs {
  const int8_t* Q;
  const double* scale;
  int axis;
  long long Sx, Sy, Sz;
  int R;        // padding reach of the split (3, or 4 with KO8)
  int k;        // digits
  int ko_reach; // 3 (KO6) or 4 (KO8)
  const double* S;  // scalar pack (device); the spacing of `axis` is S[13 + axis]
  double ko_sigma;
  double* d1;   // first derivative out (or NULL)
  double* d2;   // diagonal second derivative out (or NULL)
  double* ko;   // KO term out (or NULL)
  int ko_add;   // add to *ko instead of storing
  int* err;     // set to 1 if a tensor-core wait gives up
};

__global__ void __launch_bounds__(THREADS, 1) mma_kernel(const MmaArgs a) {
  __shared__ __align__(128) int8_t sB[NCOL * KW];
  __shared__ __align__(128) int8_t sA[MAXK][LT * KW];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid >> 5;
  const Line L = line_geom(a.axis, a.Sx, a.Sy, a.Sz);
  const int Lp = padded_len(L.len);
  const double h = a.S[13 + a.axis];
  const double w1 = (1.0 / 60.0) * (1.0 / h);
  const double w2 = (1.0 / 180.0) * (1.0 / (h * h));
  const double wko = (1.0 / (a.ko_reach == 4 ? 256.0 : 64.0)) * (a.ko_sigma / h);

  // banded stencil matrix: row n = stencil*16 + output o, column kb = window position
  {
    const int c1[7] = {-1, 9, -45, 0, 45, -9, 1};
    const int c2h[7] = {0, 0, 2, -4, 2, 0, 0};       // 270 = 2*128 + 14, -490 = -4*128 + 22
    const int c2l[7] = {2, -27, 14, 22, 14, -27, 2};
    const int k6[7] = {1, -6, 15, -20, 15, -6, 1};
    const int k8[9] = {-1, 8, -28, 56, -70, 56, -28, 8, -1};
    for (int i = tid; i < NCOL * KW; i += THREADS) {
      const int n = i / KW, kb = i % KW;
      const int st = n / NO, o = n % NO;
      const int j = kb - a.R - o;  // tap offset
      int v = 0;
      if (st < 3) {
        if (j >= -3 && j <= 3) v = st == 0 ? c1[j + 3] : (st == 1 ? c2h[j + 3] : c2l[j + 3]);
      } else if (a.ko_reach == 4) {
        if (j >= -4 && j <= 4) v = k8[j + 4];
      } else {
        if (j >= -3 && j <= 3) v = k6[j + 3];
      }
      sB[canon(n, kb, NCOL)] = (int8_t)v;
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
  uint32_t phase = 0;
  bool failed = false;
  for (long long tile = blockIdx.x; tile < ntiles && !failed; tile += gridDim.x) {
    const long long lb = tile / nzt;
    const int zt = (int)(tile % nzt);
    const int z0 = zt * NO;
    // ---- stage the digit planes of 128 lines x 32 positions (16-byte cp.async) ----
    for (int i = tid; i < a.k * LT * 2; i += THREADS) {
      const int s = i / (LT * 2);
      const int rem = i % (LT * 2);
      const int r = rem >> 1, kc = rem & 1;
      long long l = lb * LT + r;
      if (l >= L.nlines) l = L.nlines - 1;  // tail rows recompute the last line, results dropped
      const int8_t* src = a.Q + ((long long)s * L.nlines + l) * Lp + z0 + 16 * kc;
      const uint32_t dst = smem_u32(&sA[s][canon(r, 16 * kc, LT)]);
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    // ---- one elected thread issues the k contractions and commits them ----
    if (tid == 0) {
      const uint64_t db = smem_desc(smem_u32(sB), NCOL * 16, 128);
      for (int s = 0; s < a.k; ++s) {
        const uint64_t da = smem_desc(smem_u32(&sA[s][0]), LT * 16, 128);
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem + (uint32_t)(NCOL * s)),
            "l"(da), "l"(db), "r"(IDESC), "r"(0u));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                       smem_u32(&mbar))
                   : "memory");
    }
    // ---- bounded wait for the contractions ----
    uint32_t done = 0;
    for (long long it = 0; it < WAIT_LIMIT && !done; ++it) {
      asm volatile(
          "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
          : "=r"(done)
          : "r"(smem_u32(&mbar)), "r"(phase)
          : "memory");
    }
    if (__syncthreads_or(!done)) {  // one uniform verdict for the whole CTA
      if (tid == 0) atomicExch(a.err, 1);
      failed = true;
    }
    phase ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    // ---- recombine in float64: thread = line (TMEM lane) ----
    const long long l = lb * LT + tid;
    const bool line_ok = l < L.nlines && !failed;
    const double sc = line_ok ? a.scale[l] : 0.0;
    const long long base = line_ok ? line_base(a.axis, l, a.Sy, a.Sz) : 0;
    const uint32_t lane = (uint32_t)(warp * 32) << 16;
    double r1[NO], r2[NO], rk[NO];
#pragma unroll
    for (int o = 0; o < NO; ++o) { r1[o] = 0.0; r2[o] = 0.0; rk[o] = 0.0; }
    for (int s = a.k - 1; s >= 0; --s) {
      uint32_t v[4][NO];
#pragma unroll
      for (int st = 0; st < 4; ++st) {
        const uint32_t addr = tmem + lane + (uint32_t)(NCOL * s + NO * st);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
            : "=r"(v[st][0]), "=r"(v[st][1]), "=r"(v[st][2]), "=r"(v[st][3]), "=r"(v[st][4]), "=r"(v[st][5]),
              "=r"(v[st][6]), "=r"(v[st][7]), "=r"(v[st][8]), "=r"(v[st][9]), "=r"(v[st][10]), "=r"(v[st][11]),
              "=r"(v[st][12]), "=r"(v[st][13]), "=r"(v[st][14]), "=r"(v[st][15])
            : "r"(addr));
      }
      asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
      const double w = ldexp(1.0, -7 * (s + 1));
#pragma unroll
      for (int o = 0; o < NO; ++o) {
        const int i1 = (int)v[0][o];
        const int i2 = (int)v[1][o] * 128 + (int)v[2][o];
        const int ik = (int)v[3][o];
        r1[o] += (double)i1 * w;
        r2[o] += (double)i2 * w;
        rk[o] += (double)ik * w;
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    if (line_ok) {
#pragma unroll
      for (int o = 0; o < NO; ++o) {
        const int z = z0 + o;
        if (z < L.len) {
          const long long pt = base + (long long)z * L.stride;
          if (a.d1) a.d1[pt] = (r1[o] * sc) * w1;
          if (a.d2) a.d2[pt] = (r2[o] * sc) * w2;
          if (a.ko) {
            const double kv = (rk[o] * sc) * wko;
            a.ko[pt] = a.ko_add ? a.ko[pt] + kv : kv;
          }
        }
      }
    }
    __syncthreads();  // TMEM columns and shared operands are reused by the next tile
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(512));
}

}  // namespace ozaki

// ======================================================================
namespace {
thread_local std::string g_oz_err;
int oz_fail(int code, const std::string& m) {
  g_oz_err = m;
  return code;
}
}  // namespace

extern "C" {

const char* bssn_b200_ozaki_last_error(void) { return g_oz_err.c_str(); }

size_t bssn_b200_ozaki_workspace_bytes(long long Sx, long long Sy, long long Sz, int k) {
  if (Sx < 1 || Sy < 1 || Sz < 1 || k < 1 || k > ozaki::MAXK) return 0;
  size_t best = 0;
  for (int axis = 0; axis < 3; ++axis) {
    const ozaki::Line L = ozaki::line_geom(axis, Sx, Sy, Sz);
    const size_t q = (size_t)k * (size_t)L.nlines * (size_t)ozaki::padded_len(L.len);
    const size_t sc = (size_t)L.nlines * sizeof(double);
    const size_t need = ((q + 255) / 256) * 256 + sc;
    if (need > best) best = need;
  }
  return best + 256;  // + the error flag
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
  // One CTA per SM: the contraction kernel owns all 512 TMEM columns.
  static bool attr_done[64] = {false};
  constexpr int kPadSmem = 120 * 1024;
  if (dev >= 0 && dev < 64 && !attr_done[dev]) {
    e = cudaFuncSetAttribute(ozaki::mma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kPadSmem);
    if (e != cudaSuccess) return oz_fail(BSSN_B200_ECUDA, std::string("ozaki: ") + cudaGetErrorString(e));
    attr_done[dev] = true;
  }
  char* ws = static_cast<char*>(workspace);
  int* err = bssn_b200_ozaki_error_flag(workspace, Sx, Sy, Sz, k);
  e = cudaMemsetAsync(err, 0, sizeof(int), st);
  if (e != cudaSuccess) return oz_fail(BSSN_B200_ECUDA, std::string("ozaki: ") + cudaGetErrorString(e));
  const long long n = Sx * Sy * Sz;
  const int R = (use_ko && ko_order == 8) ? 4 : 3;
  auto pass = [&](const double* src, int axis, double* d1, double* d2, double* ko, int ko_add) -> int {
    const ozaki::Line L = ozaki::line_geom(axis, Sx, Sy, Sz);
    const size_t qbytes = (size_t)k * (size_t)L.nlines * (size_t)ozaki::padded_len(L.len);
    int8_t* Q = reinterpret_cast<int8_t*>(ws);
    double* scale = reinterpret_cast<double*>(ws + ((qbytes + 255) / 256) * 256);
    const int sblocks = (int)((L.nlines + 127) / 128);
    ozaki::split_kernel<<<sblocks, 128, 0, st>>>(src, axis, Sx, Sy, Sz, R, k, Q, scale);
    ozaki::MmaArgs m{};
    m.Q = Q; m.scale = scale; m.axis = axis; m.Sx = Sx; m.Sy = Sy; m.Sz = Sz;
    m.R = R; m.k = k; m.ko_reach = R; m.S = S; m.ko_sigma = use_ko ? ko_sigma : 0.0;
    m.d1 = d1; m.d2 = d2; m.ko = ko; m.ko_add = ko_add; m.err = err;
    const long long tiles = ((L.nlines + ozaki::LT - 1) / ozaki::LT) * ((L.len + ozaki::NO - 1) / ozaki::NO);
    const int grid = (int)(tiles < sms ? tiles : sms);
    ozaki::mma_kernel<<<grid, ozaki::THREADS, kPadSmem, st>>>(m);
    cudaError_t le = cudaGetLastError();
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

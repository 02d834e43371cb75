// Ozaki-style INT8 derivative path on the sm_100a tensor cores (tcgen05).
//
// Every finite-difference stencil of the BSSN bundle is a banded matrix with
// small integer coefficients (C1 x60, C2 x180, KO6 x64, KO8 x256). A float64
// field is split, line by line along the differentiation axis, into k INT8
// digits under one shared power-of-two exponent per line: with |f| 2^-e < 1/2,
//     X = rint(f 2^(7k-e)) = q_0 2^(7(k-1)) + sum_{s>0} q_s 2^(7(k-1-s)),
// q_0 = X >> 7(k-1) signed (|q_0| <= 64), q_s the 7-bit groups of X's two's
// complement below it (0 <= q_s < 128), so f ~ 2^e sum_s q_s 2^(-7(s+1));
// the stencil is applied to every digit plane as an exact INT8 x INT8 -> INT32
// tensor-core contraction, and the digit results are recombined in float64.
// The contraction is exact and the recombination order is fixed, so results
// are bit-reproducible run to run; the only approximation is the rounding of
// X (|residual| <= 2^(e-7k-1) per value, e the window's exponent).
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
constexpr int NCOL = 4 * NO;      // widest MMA N: C1 | C2 hi | C2 lo | KO
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
__host__ __device__ constexpr uint32_t idesc(int n) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((128u >> 4) << 24);
}

// The passes of one derivative bundle over a block with ghost margin `core`
// (core = 0 on a single grid): the differentiation axis and how far the
// covered box reaches past the core on each axis. First derivatives along x
// and y of the fields with second derivatives are taken 3 points into the
// ghosts across the line, where the mixed passes read them back.
struct PassKind {
  int axis;
  int ext[3];
};
constexpr int NKIND = 5;
constexpr PassKind KINDS[NKIND] = {{0, {0, 3, 3}}, {0, {0, 0, 0}}, {1, {0, 0, 3}}, {1, {0, 0, 0}}, {2, {0, 0, 0}}};

// Tiles of one pass over one block: 128-line groups x 16-output groups.
inline long long pass_tiles(const bssn_b200_block& b, const PassKind& k) {
  const int s[3] = {b.sx, b.sy, b.sz};
  long long e[3];
  for (int q = 0; q < 3; ++q) e[q] = s[q] - 2LL * (b.core - k.ext[q] > 0 ? b.core - k.ext[q] : 0);
  const int ax = k.axis;
  const long long nlines = e[(ax + 1) % 3] * e[(ax + 2) % 3];
  return ((nlines + LT - 1) / LT) * ((e[ax] + NO - 1) / NO);
}

// ---- fused split + contraction + recombination -----------------------------
// One CTA (256 threads) per SM walks tiles of 128 lines x 16 outputs of one
// pass. Per tile: the float64 window of each line (16 outputs + 2R halo,
// edge-clamped) lands in shared memory by cp.async, laid out so that the
// copies are coalesced (line-contiguous windows for the z axis, line-
// interleaved for x and y); each line gets one power-of-two exponent for its
// window and its threads write its k digit planes straight into the
// canonical operand layout; thread 0 issues the k contractions; the warps
// read the outputs back from TMEM and recombine them smallest digit first;
// the outputs go out through shared memory so that the stores are coalesced
// as well. The next tile's window is prefetched while a tile is contracted.
//
// Two shapes. The small one (the one launched) runs two 256-thread CTAs per
// SM in ~106 KB of shared memory each: at most 256 TMEM columns, the digit
// planes contracted in rounds that fit them (one round for N = 16 or 32,
// two for the passes with second derivatives), output staging inside the
// spent window buffer and digit planes, the KO sums a pass adds to loaded
// into registers during the contractions; one CTA's barriers then overlap
// the other's work. The large one (one 512-thread CTA per SM, all 512
// columns, one round, KO sums prefetched into shared memory) measured
// slower and is kept as the reference shape of the same tile loop.
template <bool SMALL>
struct Cfg {
  static constexpr int FT = SMALL ? 256 : 512;  // threads
  static constexpr int QT = FT / 128;            // threads per line in the digit split
  static constexpr int PPT = 32 / QT;            // window positions per thread
  static constexpr int OPW = 16 / QT;            // outputs per thread in the recombination
  static constexpr int FW = SMALL ? 35 : 33;     // float64 window pitch (conflict-free rows; 35 also holds the staging)
  static constexpr int CTAS = SMALL ? 2 : 1;     // CTAs per SM
};
constexpr int OP = 17;        // output staging pitch

// Sources and destinations are slots of per-block pools: slot s of block b
// starts at pool + (offset_b / 24) * slots + s * n_b, n_b = sx*sy*sz (the
// block layout of bssn_b200_block, whose offsets count 24-field states). A
// single grid is one block at offset 0, passed by value in `one`.
struct FusedArgs {
  const double* src;
  int src_slots, src_slot;
  double* dst;
  int dst_slots;
  int d1_slot, d2_slot, ko_slot;  // -1: not written
  int ko_add;                     // add the KO term to the slot instead of storing it
  int k;
  const double* S;                // scalar pack (device); a single grid's spacing is S[13 + axis]
  double ko_sigma;
  int ext[3];                     // the pass covers [core - ext, s - core + ext) per axis (clamped to the array)
  bssn_b200_block one;            // the single grid (blocks == nullptr)
  const bssn_b200_block* blocks;  // block list (device) or nullptr
  int nblocks;
  const int* tile0;               // block list: first tile of each block along this axis (device)
  long long ntiles;
  int* err;
};

template <bool SMALL>
struct FusedSmem {
  int8_t B[NCOL * KW];
  int8_t A[MAXK][LT * KW];
  double F[2][LT * 33];
  double O[3][LT * OP];
  double K[2][LT * NO];   // KO sums of the earlier axes, prefetched with the window (ko_add passes)
  long long base[2][LT];  // first element of each line of the tile in F[buf]
};
template <>
struct FusedSmem<true> {  // output staging lives in F[buf] once the digits are made
  int8_t B[NCOL * KW];
  int8_t A[MAXK][LT * KW];
  double F[2][LT * 35];
  long long base[2][LT];
};
static_assert(2 * LT * OP <= LT * 35, "two staging groups fit in a window buffer");
static_assert(LT * OP * 8 <= MAXK * LT * KW, "a staging group fits in the digit planes");

// Exact conversions between float64 and integers below 2^51 on the float64
// and integer pipes: adding 1.5 * 2^52 puts rint(v) in the low mantissa bits
// (round to nearest even, like cvt.rni), and the reverse undoes it.
constexpr double MAGIC = 6755399441055744.0;  // 1.5 * 2^52
constexpr long long MAGIC_BITS = 0x4338000000000000LL;
__device__ __forceinline__ long long rint_to_ll(double v) {  // |v| < 2^51
  return __double_as_longlong(__dadd_rn(v, MAGIC)) - MAGIC_BITS;
}
__device__ __forceinline__ double ll_to_double(long long n) {  // |n| < 2^51
  return __dsub_rn(__longlong_as_double(n + MAGIC_BITS), MAGIC);
}

// 32 lanes x N columns of 32-bit TMEM words (N = 4 or 8) into v.
template <int N>
__device__ __forceinline__ void tmem_ld(uint32_t addr, uint32_t (&v)[N]) {
  if constexpr (N == 8)
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                 : "r"(addr));
  else
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3])
                 : "r"(addr));
}

__device__ __forceinline__ void cp_async8(double* dst, const double* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}

// D2: the pass also gives the diagonal second derivative (C2 as a high and a
// low INT8 digit); KOG: it also gives the KO term. The MMA's N holds only the
// stencil groups the pass needs: C1 [| C2 hi | C2 lo] [| KO], 16 columns each.
template <int R, int AXIS, bool D2, bool KOG, bool SMALL>
__global__ void __launch_bounds__(Cfg<SMALL>::FT, Cfg<SMALL>::CTAS) fused_kernel(const FusedArgs a) {
  constexpr int FT = Cfg<SMALL>::FT, PPT = Cfg<SMALL>::PPT, OPW = Cfg<SMALL>::OPW, FW = Cfg<SMALL>::FW;
  constexpr int NG = 1 + (D2 ? 2 : 0) + (KOG ? 1 : 0);
  constexpr int NC = NO * NG;       // MMA N and TMEM columns per digit plane
  constexpr int GKO = D2 ? 3 : 1;   // column group of KO
  extern __shared__ __align__(128) unsigned char fsm_raw[];
  FusedSmem<SMALL>& sm = *reinterpret_cast<FusedSmem<SMALL>*>(fsm_raw);
  // TMEM columns: k planes of NC columns (a power of two of at least 32)
  constexpr uint32_t TCOLS = SMALL ? (NC * MAXK <= 128 ? 128u : 256u) : 512u;
  // digit planes per contraction round: all of them when they fit the
  // columns, else an even count (rounds then hold whole recombination pairs)
  constexpr int PR = NC * MAXK <= (int)TCOLS ? MAXK : (((int)TCOLS / NC) & ~1);
  static_assert(PR >= 2 && PR * NC <= (int)TCOLS, "a contraction round exceeds the allocated TMEM columns");
  constexpr int GKO_OUT = (SMALL && !D2) ? 1 : 2;  // staging group of the KO outputs
  // output staging group g of the tile in buffer b. SMALL: d1 and d2 inside
  // F[b] and KO inside the digit planes, both spent by then.
  auto obuf = [&](int b, int g) -> double* {
    if constexpr (SMALL) return g < 2 ? &sm.F[b][g * LT * OP] : reinterpret_cast<double*>(&sm.A[0][0]);
    else return &sm.O[g][0];
  };
  auto kbuf = [&](int b) -> double* {
    if constexpr (SMALL) return nullptr;
    else return &sm.K[b][0];
  };
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid >> 5;
  if (smem_u32(fsm_raw) & 127u) {  // operand layouts need an aligned base: refuse rather than misplace
    if (tid == 0) atomicExch(a.err, 1);
    return;
  }
  constexpr int KWL = NO + 2 * R;  // window positions the stencils use (22 or 24)
  {
    const int c1[7] = {-1, 9, -45, 0, 45, -9, 1};
    const int c2h[7] = {0, 0, 2, -4, 2, 0, 0};       // 270 = 2*128 + 14, -490 = -4*128 + 22
    const int c2l[7] = {2, -27, 14, 22, 14, -27, 2};
    const int k6[7] = {1, -6, 15, -20, 15, -6, 1};
    const int k8[9] = {-1, 8, -28, 56, -70, 56, -28, 8, -1};
    for (int i = tid; i < NC * KW; i += FT) {
      const int n = i / KW, kb = i % KW;
      const int g = n / NO, o = n % NO;
      const int st = (KOG && g == GKO) ? 3 : g;  // 0 C1, 1 C2 hi, 2 C2 lo, 3 KO
      const int j = kb - R - o;
      int v = 0;
      if (st < 3) {
        if (j >= -3 && j <= 3) v = st == 0 ? c1[j + 3] : (st == 1 ? c2h[j + 3] : c2l[j + 3]);
      } else if (R == 4) {
        if (j >= -4 && j <= 4) v = k8[j + 4];
      } else {
        if (j >= -3 && j <= 3) v = k6[j + 3];
      }
      sm.B[canon(n, kb, NC)] = (int8_t)v;
    }
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&mbar)));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_base)),
                 "r"(TCOLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = tmem_base;

  constexpr bool zaxis = AXIS == 2;
  // Geometry of tile t: its block; the box of the block the pass covers
  // ([m, s - m) per axis, m = max(core - ext, 0)); the box's lines along AXIS
  // (the other two axes, "slow" and "fast" in memory order); the tile's
  // 128-line group lb and first output z0; the pool bases of its slots.
  struct TileInfo {
    long long lb, nlines, stride, st_slow, st_fast;
    long long pbase, n;  // block start in points, points per block
    int z0, len, s_axis, m_axis, e_fast, m_slow, m_fast;
    double h;
  };
  auto tile_info = [&](long long t) -> TileInfo {
    TileInfo ti;
    long long lt = t, offset = 0;
    int s[3] = {a.one.sx, a.one.sy, a.one.sz}, core = 0;
    if (a.blocks) {
      // last block whose first tile is <= t: a 32-way search by the warp
      // (every thread of the CTA asks for the same t; tile0[0] = 0 <= t)
      int lo = 0, n = a.nblocks;
      while (n > 1) {
        const int step = (n + 31) >> 5;
        const int idx = lo + (tid & 31) * step;
        const unsigned ok = __ballot_sync(0xffffffffu, idx < lo + n && a.tile0[idx] <= t);
        const int last = 31 - __clz(ok);
        lo += last * step;
        n = min(step, n - last * step);
      }
      const bssn_b200_block* bk = a.blocks + lo;
      s[0] = bk->sx; s[1] = bk->sy; s[2] = bk->sz;
      core = bk->core;
      offset = bk->offset;
      ti.h = bk->h[AXIS];
      lt = t - a.tile0[lo];
    } else {
      ti.h = a.S[13 + AXIS];
    }
    int m[3], e[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      m[q] = core - a.ext[q] > 0 ? core - a.ext[q] : 0;
      e[q] = s[q] - 2 * m[q];
    }
    constexpr int SLOW = AXIS == 0 ? 1 : 0, FAST = AXIS == 2 ? 1 : 2;
    const long long st[3] = {(long long)s[1] * s[2], (long long)s[2], 1};
    ti.len = e[AXIS];
    ti.s_axis = s[AXIS];
    ti.m_axis = m[AXIS];
    ti.stride = st[AXIS];
    ti.nlines = (long long)e[SLOW] * e[FAST];
    ti.e_fast = e[FAST];
    ti.m_slow = m[SLOW];
    ti.m_fast = m[FAST];
    ti.st_slow = st[SLOW];
    ti.st_fast = st[FAST];
    const int nzt = (ti.len + NO - 1) / NO;
    const int lti = (int)lt;  // tile counts stay below 2^31 (checked on the host)
    ti.lb = lti / nzt;
    ti.z0 = (lti % nzt) * NO;
    ti.n = (long long)s[0] * s[1] * s[2];
    ti.pbase = offset / 24;
    return ti;
  };
  // the window of tile t into F[buf] (positions clamped to the block's array,
  // its edge padding; tail lines repeat the last line); the lines' first
  // elements (block-local, axis coordinate 0) are tabled once per tile.
  // Callers place it right after a barrier.
  // The first four warps look tile t up (the base table needs 128 threads)
  // and thread 0 publishes it in sti[buf]; a barrier must follow before
  // issue_window reads them.
  __shared__ TileInfo sti[2];
  auto lookup = [&](long long t, int buf) {
    if (tid < LT) {
      const TileInfo tw = tile_info(t);
      int l = (int)tw.lb * LT + tid;  // lines of a block stay below 2^31
      if (l >= tw.nlines) l = (int)tw.nlines - 1;
      const int slow = l / tw.e_fast, fast = l % tw.e_fast;
      sm.base[buf][tid] = (long long)(slow + tw.m_slow) * tw.st_slow + (long long)(fast + tw.m_fast) * tw.st_fast;
      if (tid == 0) sti[buf] = tw;
    }
  };
  auto issue_window = [&](int buf) {
    const TileInfo ti = sti[buf];
    const double* src = a.src + ti.pbase * a.src_slots + (long long)a.src_slot * ti.n;
    for (int i = tid; i < LT * KWL; i += FT) {
      const int r = zaxis ? i / KWL : i % LT;
      const int pos = zaxis ? i % KWL : i / LT;
      int q = ti.m_axis + ti.z0 - R + pos;
      q = q < 0 ? 0 : (q > ti.s_axis - 1 ? ti.s_axis - 1 : q);  // edge padding (derivatives.py:83-84)
      cp_async8(&sm.F[buf][r * FW + pos], src + sm.base[buf][r] + (long long)q * ti.stride);
    }
    if (KOG && !SMALL && a.ko_add) {
      // the KO sum this pass adds to, in the store loop's order
      const double* kos = a.dst + ti.pbase * a.dst_slots + (long long)a.ko_slot * ti.n;
      for (int i = tid; i < LT * NO; i += FT) {
        const int rr = zaxis ? i / NO : i % LT;
        const int o = zaxis ? i % NO : i / LT;
        const long long l = ti.lb * LT + rr;
        const int z = ti.z0 + o;
        if (l < ti.nlines && z < ti.len)
          cp_async8(&kbuf(buf)[i], kos + sm.base[buf][rr] + (long long)(ti.m_axis + z) * ti.stride);
      }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  const long long ntiles = a.ntiles;
  const double p7k = ldexp(1.0, 7 * a.k);  // 2^(7k): X is the window value scaled to 7k bits
  uint32_t phase = 0;
  bool failed = false;
  long long tile = blockIdx.x;
  if (tile < ntiles) {
    lookup(tile, 0);
    __syncthreads();
    issue_window(0);
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
  }
  int buf = 0;
  for (; tile < ntiles && !failed; tile += gridDim.x, buf ^= 1) {
    const TileInfo ti = sti[buf];  // published by the load of this tile's window
    const double w1 = (1.0 / 60.0) * (1.0 / ti.h);
    const double w2 = (1.0 / 180.0) * (1.0 / (ti.h * ti.h));
    const double wko = (1.0 / (R == 4 ? 256.0 : 64.0)) * (a.ko_sigma / ti.h);
    // (this tile's window has landed: the barrier that ended the previous
    // tile, or the prologue's, followed every thread's wait for its copies)
    // ---- exponent and digits: the QT threads of line r take PPT positions each ----
    const int r = tid & (LT - 1), q4 = tid >> 7;
    const double* Fr = &sm.F[buf][r * FW + PPT * q4];
    double m = 0.0;
    {
      const double* Fl = &sm.F[buf][r * FW];  // every thread of the line takes the whole window's max
      double m0 = 0.0, m1 = 0.0;
#pragma unroll
      for (int pos = 0; pos < KWL; pos += 2) {
        m0 = fmax(m0, fabs(Fl[pos]));
        m1 = fmax(m1, fabs(Fl[pos + 1]));
      }
      m = fmax(m0, m1);
    }
    // e = frexp(m) + 1 so that |f| 2^-e < 1/2; sc = 2^e, isc = 2^-e (exact).
    // A normal m reads its exponent field; subnormal and huge windows take
    // the library calls.
    int e = 0;
    double sc = 1.0, isc = 1.0;
    if (m > 0.0) {
      const int bexp = (int)((__double_as_longlong(m) >> 52) & 0x7ff);
      if (bexp > 0 && bexp < 2044) {  // e in [-1020, 1022]: both powers are normal
        e = bexp - 1022 + 1;
        sc = __longlong_as_double((long long)(e + 1023) << 52);
        isc = __longlong_as_double((long long)(1023 - e) << 52);
      } else {
        int ex;
        frexp(m, &ex);  // m = fr * 2^ex, fr in [0.5, 1)
        e = ex + 1;
        sc = ldexp(1.0, e);
        isc = ldexp(1.0, -e);
      }
    }
    {
      // X = rint(f 2^(7k - e)), |X| <= 2^(7k-1); two's complement gives
      // X = top 2^(7(k-1)) + sum_j d_j 2^(7j), 0 <= d_j < 128, |top| <= 64
      long long X[PPT];
#pragma unroll
      for (int j = 0; j < PPT; ++j) X[j] = 0;
      if (a.k <= 7) {  // |v| <= 2^48: the float64-pipe rounding
#pragma unroll
        for (int j = 0; j < PPT; ++j)
          if (PPT * q4 + j < KWL) X[j] = rint_to_ll((Fr[j] * isc) * p7k);  // exact power-of-two scaling
      } else {
#pragma unroll
        for (int j = 0; j < PPT; ++j)
          if (PPT * q4 + j < KWL) X[j] = __double2ll_rn((Fr[j] * isc) * p7k);
      }
      int8_t* dst = &sm.A[0][canon(r, PPT * q4, LT)];
      for (int s2 = 0; s2 < a.k; ++s2, dst += LT * KW) {  // plane by plane, most significant first
        const int sh = 7 * (a.k - 1 - s2);
        const uint32_t mask = s2 == 0 ? 255u : 127u;
        uint32_t w[PPT / 4];
#pragma unroll
        for (int c = 0; c < PPT / 4; ++c) w[c] = 0u;
#pragma unroll
        for (int j = 0; j < PPT; ++j) {
          const uint32_t d = (uint32_t)(X[j] >> sh) & mask;
          w[j >> 2] |= d << (8 * (j & 3));
        }
        if constexpr (PPT == 16) *reinterpret_cast<uint4*>(dst) = make_uint4(w[0], w[1], w[2], w[3]);
        else *reinterpret_cast<uint2*>(dst) = make_uint2(w[0], w[1]);
      }
    }
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    // the KO sums this pass adds to (SMALL has no shared-memory room for them):
    // loaded into registers now, in the store loop's order, so that they
    // arrive during the contractions
    constexpr int SPT = LT * NO / FT;  // outputs per thread in the store loop
    double kpre[SPT];
    if constexpr (SMALL && KOG) {
      if (a.ko_add) {
        const double* kos = a.dst + ti.pbase * a.dst_slots + (long long)a.ko_slot * ti.n;
#pragma unroll
        for (int j = 0; j < SPT; ++j) {
          const int i = tid + j * FT;
          const int rr = zaxis ? i / NO : i % LT;
          const int o = zaxis ? i % NO : i / LT;
          const int z = ti.z0 + o;
          kpre[j] = (ti.lb * LT + rr < ti.nlines && z < ti.len)
                        ? kos[sm.base[buf][rr] + (long long)(ti.m_axis + z) * ti.stride] : 0.0;
        }
      }
    }
    // ---- contractions in rounds of PR digit planes, smallest planes first
    // (one round unless the planes exceed the CTA's TMEM columns). Thread 0
    // issues a round; during the first, the first four warps look the next
    // tile up (its base table and sti slot were last read last tile); the
    // barrier after the first wait publishes it and everyone prefetches the
    // next tile's window behind the recombination and stores ----
    const uint32_t lane = (uint32_t)((warp & 3) * 32) << 16;  // warp w reads TMEM lanes 32 (w % 4)..
    const int oc = OPW * (warp >> 2);                           // and outputs OPW (w / 4)..
    double r1[OPW], r2[OPW], rk[OPW];
#pragma unroll
    for (int o = 0; o < OPW; ++o) { r1[o] = 0.0; r2[o] = 0.0; rk[o] = 0.0; }
    // planes in pairs from the smallest: (q_{s-1} 128 + q_s) is an exact
    // int32 (|C2 pair| < 2^25), converted once and added with the weight of
    // plane s; an odd top plane goes alone
    double w = ldexp(1.0, -7 * a.k);  // weight of the smallest digit plane
    int s2 = a.k - 1;                  // planes s2 .. 0 remain
    const bool more = tile + gridDim.x < ntiles;
    for (int round = 0; s2 >= 0 && !failed; ++round) {
      const int lo = s2 - PR + 1 > 0 ? s2 - PR + 1 : 0;  // this round: planes lo .. s2 at columns NC (p - lo)
      if (tid == 0) {
        const uint64_t db = smem_desc(smem_u32(sm.B), NC * 16, 128);
        for (int p = lo; p <= s2; ++p) {
          const uint64_t da = smem_desc(smem_u32(&sm.A[p][0]), LT * 16, 128);
          asm volatile(
              "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
              "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem + (uint32_t)(NC * (p - lo))),
              "l"(da), "l"(db), "r"(idesc(NC)), "r"(0u));
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                         smem_u32(&mbar))
                     : "memory");
      }
      if (round == 0 && more) lookup(tile + gridDim.x, buf ^ 1);
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
      if (failed) break;
      if (round == 0 && more) issue_window(buf ^ 1);
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      for (; s2 - 1 >= lo; s2 -= 2, w *= 16384.0) {
        const uint32_t ca = (uint32_t)(NC * (s2 - 1 - lo)), cb = (uint32_t)(NC * (s2 - lo));
        if constexpr (SMALL && D2) {  // one stencil at a time (registers)
          {
            uint32_t va[OPW], vb[OPW];
            tmem_ld<OPW>(tmem + lane + ca + (uint32_t)oc, va);
            tmem_ld<OPW>(tmem + lane + cb + (uint32_t)oc, vb);
            asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
            for (int o = 0; o < OPW; ++o) r1[o] += ll_to_double((int)va[o] * 128 + (int)vb[o]) * w;
          }
          {
            uint32_t ha[OPW], hb[OPW], la[OPW], lb2[OPW];  // C2 high and low digits of planes s2 - 1, s2
            tmem_ld<OPW>(tmem + lane + ca + (uint32_t)(NO + oc), ha);
            tmem_ld<OPW>(tmem + lane + cb + (uint32_t)(NO + oc), hb);
            tmem_ld<OPW>(tmem + lane + ca + (uint32_t)(2 * NO + oc), la);
            tmem_ld<OPW>(tmem + lane + cb + (uint32_t)(2 * NO + oc), lb2);
            asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
            for (int o = 0; o < OPW; ++o) {
              const int c2a = (int)ha[o] * 128 + (int)la[o];
              const int c2b = (int)hb[o] * 128 + (int)lb2[o];
              r2[o] += ll_to_double(c2a * 128 + c2b) * w;
            }
          }
          if (KOG) {
            uint32_t va[OPW], vb[OPW];
            tmem_ld<OPW>(tmem + lane + ca + (uint32_t)(NO * GKO + oc), va);
            tmem_ld<OPW>(tmem + lane + cb + (uint32_t)(NO * GKO + oc), vb);
            asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
            for (int o = 0; o < OPW; ++o) rk[o] += ll_to_double((int)va[o] * 128 + (int)vb[o]) * w;
          }
        } else {
          uint32_t v[2][NG][OPW];  // [0]: plane s2 - 1 (weight 128 w), [1]: plane s2
#pragma unroll
          for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int g = 0; g < NG; ++g) tmem_ld<OPW>(tmem + lane + (h ? cb : ca) + (uint32_t)(NO * g + oc), v[h][g]);
          asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
          for (int o = 0; o < OPW; ++o) {
            r1[o] += ll_to_double((int)v[0][0][o] * 128 + (int)v[1][0][o]) * w;
            if (D2) {
              const int c2a = (int)v[0][D2 ? 1 : 0][o] * 128 + (int)v[0][D2 ? 2 : 0][o];
              const int c2b = (int)v[1][D2 ? 1 : 0][o] * 128 + (int)v[1][D2 ? 2 : 0][o];
              r2[o] += ll_to_double(c2a * 128 + c2b) * w;
            }
            if (KOG) rk[o] += ll_to_double((int)v[0][KOG ? GKO : 0][o] * 128 + (int)v[1][KOG ? GKO : 0][o]) * w;
          }
        }
      }
      if (s2 == lo) {  // lo == 0: the odd top plane alone
        uint32_t v[NG][OPW];
#pragma unroll
        for (int g = 0; g < NG; ++g) tmem_ld<OPW>(tmem + lane + (uint32_t)(NC * (s2 - lo) + NO * g + oc), v[g]);
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
        for (int o = 0; o < OPW; ++o) {
          r1[o] += (double)(int)v[0][o] * w;
          if (D2) r2[o] += (double)((int)v[D2 ? 1 : 0][o] * 128 + (int)v[D2 ? 2 : 0][o]) * w;
          if (KOG) rk[o] += (double)(int)v[KOG ? GKO : 0][o] * w;
        }
        s2 = -1;
      }
      if (s2 >= 0) {  // every warp has read this round's columns before the next round's contractions
        asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    // the recombining thread's line is r too (TMEM lane = line): its exponent is sc
#pragma unroll
    for (int o = 0; o < OPW; ++o) {
      obuf(buf, 0)[r * OP + oc + o] = (r1[o] * sc) * w1;
      if (D2) obuf(buf, 1)[r * OP + oc + o] = (r2[o] * sc) * w2;
      if (KOG) obuf(buf, GKO_OUT)[r * OP + oc + o] = (rk[o] * sc) * wko;
    }
    __syncthreads();
    // ---- coalesced stores of the tile's outputs ----
#pragma unroll
    for (int j = 0; j < SPT; ++j) {
      const int i = tid + j * FT;
      const int rr = zaxis ? i / NO : i % LT;
      const int o = zaxis ? i % NO : i / LT;
      const long long l = ti.lb * LT + rr;
      const int z = ti.z0 + o;
      if (l < ti.nlines && z < ti.len && !failed) {
        double* out = a.dst + ti.pbase * a.dst_slots + sm.base[buf][rr] + (long long)(ti.m_axis + z) * ti.stride;
        out[(long long)a.d1_slot * ti.n] = obuf(buf, 0)[rr * OP + o];
        if (D2) out[(long long)a.d2_slot * ti.n] = obuf(buf, 1)[rr * OP + o];
        if (KOG) {
          double* kp = out + (long long)a.ko_slot * ti.n;
          const double kv = obuf(buf, GKO_OUT)[rr * OP + o];
          *kp = a.ko_add ? (SMALL ? kpre[j] : kbuf(buf)[i]) + kv : kv;
        }
      }
    }
    // the next tile's window (this thread's copies) has landed; the barrier
    // publishes it and frees TMEM columns, digits and output staging
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TCOLS));
}

}  // namespace ozaki

// ======================================================================
namespace {
thread_local std::string g_oz_err;

template <int R, int AXIS, bool D2, bool KOG>
cudaError_t launch_fused(const ozaki::FusedArgs& m, long long ntiles, int sms, cudaStream_t st, int dev) {
  constexpr bool SMALL = true;
  using C = ozaki::Cfg<SMALL>;
  static bool attr_done[64] = {false};
  constexpr int kSmem = (int)sizeof(ozaki::FusedSmem<SMALL>);
  if (!attr_done[dev]) {
    cudaError_t e = cudaFuncSetAttribute(ozaki::fused_kernel<R, AXIS, D2, KOG, SMALL>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, kSmem);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(ozaki::fused_kernel<R, AXIS, D2, KOG, SMALL>,
                               cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
    attr_done[dev] = true;
  }
  // persistent: C::CTAS CTAs per SM (the TMEM columns of a CTA allow that many)
  const long long cap = (long long)C::CTAS * sms;
  const int grid = (int)(ntiles < cap ? ntiles : cap);
  ozaki::fused_kernel<R, AXIS, D2, KOG, SMALL><<<grid, C::FT, kSmem, st>>>(m);
  return cudaSuccess;
}

// The instantiation for a pass: the KO reach only matters when KO is formed.
template <int AXIS>
cudaError_t launch_axis(const ozaki::FusedArgs& m, int sms, cudaStream_t st, int dev, int R, bool d2, bool ko) {
  const long long t = m.ntiles;
  if (ko) {
    if (R == 4) return d2 ? launch_fused<4, AXIS, true, true>(m, t, sms, st, dev) : launch_fused<4, AXIS, false, true>(m, t, sms, st, dev);
    return d2 ? launch_fused<3, AXIS, true, true>(m, t, sms, st, dev) : launch_fused<3, AXIS, false, true>(m, t, sms, st, dev);
  }
  return d2 ? launch_fused<3, AXIS, true, false>(m, t, sms, st, dev) : launch_fused<3, AXIS, false, false>(m, t, sms, st, dev);
}

int oz_fail(int code, const std::string& m) {
  g_oz_err = m;
  return code;
}

bool has_d2(int f) { return f == 0 || f == 1 || (f >= 3 && f < 12); }
int g2slot(int f) { return f == 0 ? 0 : (f == 1 ? 1 : (f < 9 ? 2 + f - 3 : 8 + f - 9)); }

// One derivative bundle (138 slots, +24 KO sums) of the 24 fields of F into
// the slot pool D: per field and axis one pass giving the first derivative,
// the diagonal second derivative and the KO term (added over the axes), then
// the mixed second derivatives as first derivatives of the x and y first
// derivatives (derivative_bundle.py:31-48). `one` is the single grid when
// blocks == nullptr; else tile0 holds NKIND tables of nblocks first tiles.
int run_bundle(cudaStream_t st, const double* F, const double* S, double* D, int k, double ko_sigma,
               int ko_order, const bssn_b200_block& one, const bssn_b200_block* blocks, int nblocks,
               const int* tile0, const long long* ntiles, int* err) {
  int dev = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return oz_fail(BSSN_B200_ECUDA, std::string("ozaki: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= 64) return oz_fail(BSSN_B200_EINVAL, "ozaki: device ordinal out of range");
  e = cudaMemsetAsync(err, 0, sizeof(int), st);
  if (e != cudaSuccess) return oz_fail(BSSN_B200_ECUDA, std::string("ozaki: ") + cudaGetErrorString(e));
  const bool use_ko = ko_sigma > 0.0;
  const int R = (use_ko && ko_order == 8) ? 4 : 3;
  const int nslot = use_ko ? 162 : 138;
  auto pass = [&](const double* src, int src_slots, int src_slot, int kind, int d1, int d2, int ko,
                  int ko_add) -> int {
    const ozaki::PassKind& pk = ozaki::KINDS[kind];
    ozaki::FusedArgs m{};
    m.src = src; m.src_slots = src_slots; m.src_slot = src_slot;
    m.dst = D; m.dst_slots = nslot; m.d1_slot = d1; m.d2_slot = d2; m.ko_slot = ko; m.ko_add = ko_add;
    m.k = k; m.S = S; m.ko_sigma = use_ko ? ko_sigma : 0.0;
    for (int q = 0; q < 3; ++q) m.ext[q] = pk.ext[q];
    m.one = one; m.blocks = blocks; m.nblocks = nblocks;
    m.tile0 = blocks ? tile0 + (long long)kind * nblocks : nullptr;
    m.ntiles = ntiles[kind];
    m.err = err;
    if (m.ntiles < 1) return 0;
    const int axis = pk.axis;
    const bool has2 = d2 >= 0, hasko = ko >= 0;
    cudaError_t le = axis == 0 ? launch_axis<0>(m, sms, st, dev, R, has2, hasko)
                   : (axis == 1 ? launch_axis<1>(m, sms, st, dev, R, has2, hasko)
                                : launch_axis<2>(m, sms, st, dev, R, has2, hasko));
    if (le == cudaSuccess) le = cudaGetLastError();
    if (le != cudaSuccess) return oz_fail(BSSN_B200_ECUDA, std::string("ozaki launch: ") + cudaGetErrorString(le));
    return 0;
  };
  const int diag[3] = {0, 3, 5};
  for (int f = 0; f < 24; ++f) {
    for (int axis = 0; axis < 3; ++axis) {
      const bool d2f = has_d2(f);
      const int kind = axis == 0 ? (d2f ? 0 : 1) : (axis == 1 ? (d2f ? 2 : 3) : 4);
      const int d2 = d2f ? 72 + 6 * g2slot(f) + diag[axis] : -1;
      int rc = pass(F, 24, f, kind, 3 * f + axis, d2, use_ko ? 138 + f : -1, axis > 0);
      if (rc) return rc;
    }
  }
  for (int f = 0; f < 24; ++f) {
    if (!has_d2(f)) continue;
    const int g = 72 + 6 * g2slot(f);
    int rc = pass(D, nslot, 3 * f + 0, 3, g + 1, -1, -1, 0);   // d/dy of d/dx
    if (!rc) rc = pass(D, nslot, 3 * f + 0, 4, g + 2, -1, -1, 0);  // d/dz of d/dx
    if (!rc) rc = pass(D, nslot, 3 * f + 1, 4, g + 4, -1, -1, 0);  // d/dz of d/dy
    if (rc) return rc;
  }
  return 0;
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

static int check_common(int k, double ko_sigma, int ko_order, void* workspace, size_t workspace_bytes) {
  if (k < 1 || k > ozaki::MAXK) return oz_fail(BSSN_B200_EINVAL, "ozaki: k must be 1..8");
  if (ko_sigma > 0.0 && ko_order != 6 && ko_order != 8) return oz_fail(BSSN_B200_EINVAL, "ozaki: ko_order must be 6 or 8");
  if (workspace_bytes < 256) return oz_fail(BSSN_B200_EINVAL, "ozaki: workspace smaller than bssn_b200_ozaki_workspace_bytes()");
  if ((reinterpret_cast<uintptr_t>(workspace) & 255) != 0) return oz_fail(BSSN_B200_EINVAL, "ozaki: workspace not 256-byte aligned");
  return 0;
}

int bssn_b200_ozaki_derivatives(void* stream, const double* F, const double* S, double* DOUT, int k,
                                double ko_sigma, int ko_order, long long Sx, long long Sy, long long Sz,
                                void* workspace, size_t workspace_bytes) {
  if (!F || !S || !DOUT || !workspace) return oz_fail(BSSN_B200_EINVAL, "ozaki: NULL operand");
  if (Sx < 8 || Sy < 8 || Sz < 8) return oz_fail(BSSN_B200_EINVAL, "ozaki: every extent must be >= 8");
  if (Sx * Sy * Sz > (1LL << 31)) return oz_fail(BSSN_B200_EINVAL, "ozaki: grid too large");
  int rc = check_common(k, ko_sigma, ko_order, workspace, workspace_bytes);
  if (rc) return rc;
  if (workspace_bytes < bssn_b200_ozaki_workspace_bytes(Sx, Sy, Sz, k))
    return oz_fail(BSSN_B200_EINVAL, "ozaki: workspace smaller than bssn_b200_ozaki_workspace_bytes()");
  bssn_b200_block one{};
  one.sx = (int)Sx; one.sy = (int)Sy; one.sz = (int)Sz;
  one.h[0] = one.h[1] = one.h[2] = 1.0;  // the spacing comes from S[13..15]
  long long nt[ozaki::NKIND];
  for (int q = 0; q < ozaki::NKIND; ++q) nt[q] = ozaki::pass_tiles(one, ozaki::KINDS[q]);
  int* err = bssn_b200_ozaki_error_flag(workspace, Sx, Sy, Sz, k);
  return run_bundle(static_cast<cudaStream_t>(stream), F, S, DOUT, k, ko_sigma, ko_order, one, nullptr, 0,
                    nullptr, nt, err);
}

long long bssn_b200_batch_ozaki_plan(const bssn_b200_block* host_blocks, int nblocks, int* host_tile0,
                                     long long* host_ntiles, long long* host_pts0) {
  if (!host_blocks || nblocks < 1 || !host_tile0 || !host_ntiles || !host_pts0) {
    oz_fail(BSSN_B200_EINVAL, "batch_ozaki_plan: NULL or empty table");
    return -1;
  }
  long long t[ozaki::NKIND] = {0, 0, 0, 0, 0}, pts = 0;
  for (int b = 0; b < nblocks; ++b) {
    const bssn_b200_block& bk = host_blocks[b];
    if (bk.sx < 8 || bk.sy < 8 || bk.sz < 8 || bk.offset < 0 || bk.offset % 24 != 0 || !(bk.h[0] > 0) ||
        !(bk.h[1] > 0) || !(bk.h[2] > 0)) {
      oz_fail(BSSN_B200_EINVAL, "batch_ozaki_plan: block " + std::to_string(b) +
                                    " has an extent below 8, a bad offset or a bad spacing");
      return -1;
    }
    if ((long long)bk.sx * bk.sy * bk.sz >= (1LL << 31)) {
      oz_fail(BSSN_B200_EINVAL, "batch_ozaki_plan: block " + std::to_string(b) + " has 2^31 points or more");
      return -1;
    }
    if (bk.core < 0 || 2 * bk.core >= bk.sx || 2 * bk.core >= bk.sy || 2 * bk.core >= bk.sz) {
      oz_fail(BSSN_B200_EINVAL, "batch_ozaki_plan: block " + std::to_string(b) + " has a core margin that leaves no points");
      return -1;
    }
    host_pts0[b] = pts;
    pts += (long long)(bk.sx - 2 * bk.core) * (bk.sy - 2 * bk.core) * (bk.sz - 2 * bk.core);
    for (int q = 0; q < ozaki::NKIND; ++q) {
      host_tile0[(long long)q * nblocks + b] = (int)t[q];
      t[q] += ozaki::pass_tiles(bk, ozaki::KINDS[q]);
      if (t[q] >= (1LL << 31)) {
        oz_fail(BSSN_B200_EINVAL, "batch_ozaki_plan: too many tiles");
        return -1;
      }
    }
  }
  for (int q = 0; q < ozaki::NKIND; ++q) host_ntiles[q] = t[q];
  return pts;
}

int bssn_b200_batch_ozaki_derivatives(void* stream, const double* F, const double* S, double* D, int k,
                                      double ko_sigma, int ko_order, const bssn_b200_block* blocks,
                                      int nblocks, const int* tile0, const long long* host_ntiles,
                                      void* workspace, size_t workspace_bytes) {
  if (!F || !S || !D || !blocks || !tile0 || !host_ntiles || !workspace || nblocks < 1)
    return oz_fail(BSSN_B200_EINVAL, "batch_ozaki_derivatives: NULL operand or empty table");
  int rc = check_common(k, ko_sigma, ko_order, workspace, workspace_bytes);
  if (rc) return rc;
  for (int q = 0; q < ozaki::NKIND; ++q)
    if (host_ntiles[q] < 0 || host_ntiles[q] >= (1LL << 31))
      return oz_fail(BSSN_B200_EINVAL, "batch_ozaki_derivatives: tile count out of range");
  bssn_b200_block one{};
  int* err = static_cast<int*>(workspace);
  return run_bundle(static_cast<cudaStream_t>(stream), F, S, D, k, ko_sigma, ko_order, one, blocks, nblocks,
                    tile0, host_ntiles, err);
}

}  // extern "C"

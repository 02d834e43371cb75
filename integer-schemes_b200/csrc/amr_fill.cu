// Ghost-zone fill for batched AMR block pools: same-level copies, node-centred
// 2:1 prolongation from the next coarser level and fine-to-coarse injection,
// the transfer operators of the reference's node-centred AMR
// (3D/src/multipatch/amr/kernels.py:52-71 prolongation, :114-145 injection;
// 3D/src/multipatch/amr/sync.py:70-122 cross-level and same-level fills),
// applied to the BSSN block pool that the batched stage kernels evolve.
//
// A fill is a host-planned list of boxes (bssn_b200_fill_op), copies and
// injections first, prolongations after (fewer warps mix the two paths). One
// launch executes one list: a thread takes one copied point and moves all 24
// fields, or one (prolongated point, field) pair (points flattened over the
// boxes by a prefix of box volumes, the box found by binary search). The work
// is a gather of a small part of the pool and bound by memory latency: the
// copy path issues its 24 loads before its stores, prolongations run one
// field per thread and a warp's points share their parity class, and the grid
// holds four CTAs per SM.
//
// Prolongation refines the source block x, then y, then z. A point odd on an
// axis sums its 6 taps in offset order starting from 0 (the reference's
// `mids = 0.0; mids = mids + w * slice` loop), a point even on an axis takes
// the coincident node unchanged; every product and sum is rounded
// separately (no fused multiply-add), so the result equals the sequential
// whole-block passes bit for bit.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>

#include "../../include/bssn_b200.h"
#include "host_util.h"

namespace amr {

constexpr int NFIELD = 24;
constexpr int NTHREADS = 256;
constexpr int MIN_CTAS = 4;  // resident CTAs per SM the register budget allows

struct Wmid {
  double w[6];
};

__device__ __forceinline__ int clampi(int v, int hi) { return v < 0 ? 0 : (v > hi ? hi : v); }

// Destination point (d0, d1, d2) of point p in box op, or false past the box.
__device__ __forceinline__ bool decode(const bssn_b200_fill_op& op, long long p, int& d0, int& d1, int& d2) {
  const int bz = op.hi[2] - op.lo[2], by = op.hi[1] - op.lo[1];
  int r = (int)(p - op.point0);  // box volumes stay below 2^31 (checked by the plan)
  d2 = op.lo[2] + r % bz;
  r /= bz;
  d1 = op.lo[1] + r % by;
  d0 = op.lo[0] + r / by;
  return d0 < op.hi[0];  // npoints past the plan's total: nothing to write
}

__device__ __forceinline__ void copy_point(double* __restrict__ pool, const bssn_b200_fill_op& op, long long p) {
  int d0, d1, d2;
  if (!decode(op, p, d0, d1, d2)) return;
  const int ss1 = op.src_s[1], ss2 = op.src_s[2];
  const long long nd = (long long)op.dst_s[0] * op.dst_s[1] * op.dst_s[2];
  const long long ns = (long long)op.src_s[0] * ss1 * ss2;
  double* dst = pool + op.dst_off + ((long long)d0 * op.dst_s[1] + d1) * op.dst_s[2] + d2;
  const int m = op.kind == BSSN_B200_FILL_RESTRICT ? 2 : 1;
  const double* src = pool + op.src_off + ((long long)(m * d0 + op.shift[0]) * ss1 + (m * d1 + op.shift[1])) * ss2 +
                      (m * d2 + op.shift[2]);
  double v[NFIELD];  // all 24 loads in flight before the stores
#pragma unroll
  for (int f = 0; f < NFIELD; ++f) v[f] = src[f * ns];
#pragma unroll
  for (int f = 0; f < NFIELD; ++f) dst[f * nd] = v[f];
}

// Destination point of point p in a prolongation box, with the box's points
// enumerated by parity class first: the class of a point is the parity of its
// refined index g = d + shift on each axis (odd: the 6-tap midpoint stencil,
// even: the coincident node), classes in the order (x, y, z) = 000, 001, ...,
// 111, points of a class in C order on their stride-2 sub-lattice. A warp's
// consecutive points then share their tap counts instead of alternating
// between the 1-tap and 6-tap paths along z.
__device__ __forceinline__ bool decode_by_parity(const bssn_b200_fill_op& op, long long p, int& d0, int& d1,
                                                 int& d2) {
  // per axis: points of even / odd refined index, and the parity of the first
  int ne[3], no[3], first[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int len = op.hi[a] - op.lo[a];
    first[a] = (op.lo[a] + op.shift[a]) & 1;
    ne[a] = first[a] ? len >> 1 : (len + 1) >> 1;
    no[a] = len - ne[a];
  }
  int r = (int)(p - op.point0);  // box volumes stay below 2^31 (checked by the plan)
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const int p0 = c >> 2, p1 = (c >> 1) & 1, p2 = c & 1;  // compile-time after unrolling
    const int n0 = p0 ? no[0] : ne[0], n1 = p1 ? no[1] : ne[1], n2 = p2 ? no[2] : ne[2];
    const int cnt = n0 * n1 * n2;
    if (r < cnt) {
      const int i2 = r % n2;
      const int t = r / n2;
      const int i1 = t % n1;
      const int i0 = t / n1;
      d0 = op.lo[0] + (p0 != first[0]) + 2 * i0;
      d1 = op.lo[1] + (p1 != first[1]) + 2 * i1;
      d2 = op.lo[2] + (p2 != first[2]) + 2 * i2;
      return true;
    }
    r -= cnt;
  }
  return false;  // npoints past the plan's total: nothing to write
}

__device__ __forceinline__ void prolong_point(double* __restrict__ pool, const bssn_b200_fill_op& op, long long p,
                                              const double* __restrict__ w, int f) {
  int d0, d1, d2;
  if (!decode_by_parity(op, p, d0, d1, d2)) return;
  const int ss0 = op.src_s[0], ss1 = op.src_s[1], ss2 = op.src_s[2];
  const long long nd = (long long)op.dst_s[0] * op.dst_s[1] * op.dst_s[2];
  const long long ns = (long long)ss0 * ss1 * ss2;
  double* dst = pool + op.dst_off + ((long long)d0 * op.dst_s[1] + d1) * op.dst_s[2] + d2;
  const double* src = pool + op.src_off;
  // per axis: 1 tap (even, coincident node) or 6 taps (odd, midpoint)
  const int g0 = d0 + op.shift[0], g1 = d1 + op.shift[1], g2 = d2 + op.shift[2];
  const bool o0 = g0 & 1, o1 = g1 & 1, o2 = g2 & 1;
  const int k0 = g0 >> 1, k1 = g1 >> 1, k2 = g2 >> 1;  // arithmetic shift: floor(g / 2)
  const int ny = o1 ? 6 : 1, nz = o2 ? 6 : 1;
  const long long sxs = (long long)ss1 * ss2;
  {
    const double* P = src + f * ns;
    double vz = 0.0;
    for (int c = 0; c < nz; ++c) {
      const int iz = clampi(o2 ? k2 - 2 + c : k2, ss2 - 1);
      double vy = 0.0;
      for (int b = 0; b < ny; ++b) {
        const int iy = clampi(o1 ? k1 - 2 + b : k1, ss1 - 1);
        const double* row = P + (long long)iy * ss2 + iz;
        double vx;
        if (!o0) {
          vx = row[k0 < 0 ? 0 : (k0 > ss0 - 1 ? ss0 - 1 : k0) * sxs];
        } else {
          vx = 0.0;
#pragma unroll
          for (int a = 0; a < 6; ++a) vx = __dadd_rn(vx, __dmul_rn(w[a], row[clampi(k0 - 2 + a, ss0 - 1) * sxs]));
        }
        vy = o1 ? __dadd_rn(vy, __dmul_rn(w[b], vx)) : vx;
      }
      vz = o2 ? __dadd_rn(vz, __dmul_rn(w[c], vy)) : vy;
    }
    dst[f * nd] = vz;
  }
}

// Work items: every copied or injected point (24 fields each), then every
// (prolongated point, field) pair — a prolongation sums up to 216 taps per
// field, so its fields go to separate threads; 32 consecutive items of a warp
// are 32 consecutive points of one field. Every thread takes items by a grid
// stride and finds its box by binary search over the boxes' point prefix.
__global__ void __launch_bounds__(NTHREADS, MIN_CTAS) fill_kernel(double* __restrict__ pool,
                                                                  const bssn_b200_fill_op* __restrict__ ops,
                                                                  int nops, long long npoints, const Wmid W) {
  __shared__ double sw[6];  // midpoint weights (indexed by tap)
  __shared__ long long ncopy_s;  // points before the first prolongation box
  if (threadIdx.x == 0) {
#pragma unroll
    for (int j = 0; j < 6; ++j) sw[j] = W.w[j];
    int lo = 0, hi = nops;  // first prolongation op (the list has them last)
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (ops[mid].kind == BSSN_B200_FILL_PROLONG) hi = mid; else lo = mid + 1;
    }
    ncopy_s = lo < nops ? ops[lo].point0 : npoints;
  }
  __syncthreads();
  const long long ncopy = ncopy_s;
  // whole 32-point chunks of prolongation items (the last one's tail skips)
  const long long items = ncopy + (npoints - ncopy + 31) / 32 * 32 * NFIELD;
  const long long stride = (long long)gridDim.x * NTHREADS;
  for (long long it = (long long)blockIdx.x * NTHREADS + threadIdx.x; it < items; it += stride) {
    long long p;
    int f = 0;
    if (it < ncopy) {
      p = it;
    } else {
      const long long q = it - ncopy;
      const long long r = q % (32 * NFIELD);
      f = (int)(r >> 5);
      p = ncopy + (q / (32 * NFIELD)) * 32 + (r & 31);
      if (p >= npoints) continue;
    }
    int lo = 0, hi = nops - 1;  // last box with point0 <= p
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (ops[mid].point0 <= p) lo = mid; else hi = mid - 1;
    }
    if (ops[lo].kind == BSSN_B200_FILL_PROLONG) prolong_point(pool, ops[lo], p, sw, f);
    else copy_point(pool, ops[lo], p);
  }
}

}  // namespace amr

extern "C" {

long long bssn_b200_fill_plan(bssn_b200_fill_op* host_ops, int nops, long long pool_doubles) {
  using bssn_host::fail;
  if (!host_ops || nops < 1) {
    fail(BSSN_B200_EINVAL, "fill_plan: empty op list");
    return -1;
  }
  long long total = 0;
  for (int i = 0; i < nops; ++i) {
    bssn_b200_fill_op& op = host_ops[i];
    const std::string at = "fill_plan: op " + std::to_string(i) + ": ";
    if (op.kind != BSSN_B200_FILL_COPY && op.kind != BSSN_B200_FILL_RESTRICT && op.kind != BSSN_B200_FILL_PROLONG) {
      fail(BSSN_B200_EINVAL, at + "unknown kind");
      return -1;
    }
    long long nd = 1, ns = 1, vol = 1;
    for (int a = 0; a < 3; ++a) {
      if (op.dst_s[a] < 1 || op.src_s[a] < 1) {
        fail(BSSN_B200_EINVAL, at + "empty block extent");
        return -1;
      }
      if (op.lo[a] < 0 || op.hi[a] > op.dst_s[a] || op.lo[a] >= op.hi[a]) {
        fail(BSSN_B200_EINVAL, at + "box outside its destination block or empty");
        return -1;
      }
      if (op.kind != BSSN_B200_FILL_PROLONG) {
        const long long m = op.kind == BSSN_B200_FILL_RESTRICT ? 2 : 1;
        const long long s_lo = m * op.lo[a] + op.shift[a], s_hi = m * (op.hi[a] - 1) + op.shift[a];
        if (s_lo < 0 || s_hi >= op.src_s[a]) {
          fail(BSSN_B200_EINVAL, at + "source points outside the source block");
          return -1;
        }
      } else if ((long long)op.lo[a] + op.shift[a] < -(1LL << 29) || (long long)op.hi[a] + op.shift[a] > (1LL << 29)) {
        fail(BSSN_B200_EINVAL, at + "prolongation shift out of range");
        return -1;
      }
      nd *= op.dst_s[a];
      ns *= op.src_s[a];
      vol *= op.hi[a] - op.lo[a];
    }
    if (vol >= (1LL << 31)) {
      fail(BSSN_B200_EINVAL, at + "box of 2^31 points or more");
      return -1;
    }
    if (op.dst_off < 0 || op.src_off < 0 || op.dst_off + 24 * nd > pool_doubles || op.src_off + 24 * ns > pool_doubles) {
      fail(BSSN_B200_EINVAL, at + "block outside the pool");
      return -1;
    }
    if (op.dst_off == op.src_off) {
      fail(BSSN_B200_EINVAL, at + "a block cannot fill itself");
      return -1;
    }
  }
  // copies and injections first, prolongations after (the fill launches one
  // kernel per range); boxes of one list never overlap, so order is free
  std::stable_partition(host_ops, host_ops + nops,
                        [](const bssn_b200_fill_op& o) { return o.kind != BSSN_B200_FILL_PROLONG; });
  for (int i = 0; i < nops; ++i) {
    bssn_b200_fill_op& op = host_ops[i];
    op.point0 = total;
    total += (long long)(op.hi[0] - op.lo[0]) * (op.hi[1] - op.lo[1]) * (op.hi[2] - op.lo[2]);
  }
  return total;
}

int bssn_b200_fill(void* stream, double* pool, const bssn_b200_fill_op* ops, int nops, long long npoints,
                   const double* wmid) {
  using bssn_host::fail;
  if (!pool || !ops || !wmid) return fail(BSSN_B200_EINVAL, "fill: NULL operand");
  if (nops < 1 || npoints < 1) return fail(BSSN_B200_EINVAL, "fill: empty plan");
  amr::Wmid W;
  for (int j = 0; j < 6; ++j) W.w[j] = wmid[j];
  int sms = 0;
  int rc = bssn_host::device_sms(&sms);
  if (rc) return rc;
  const long long want = (npoints * amr::NFIELD + amr::NTHREADS - 1) / amr::NTHREADS;
  const long long cap = 4LL * amr::MIN_CTAS * sms;  // four waves of resident CTAs
  amr::fill_kernel<<<(int)(want < cap ? want : cap), amr::NTHREADS, 0, static_cast<cudaStream_t>(stream)>>>(
      pool, ops, nops, npoints, W);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return bssn_host::cuda_fail("fill launch", e);
  return 0;
}

}  // extern "C"

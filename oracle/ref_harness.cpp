// Test infrastructure only: a CPU harness around the reference's own BSSN
// right-hand-side algebra, compiled from the vendored Dendro-GR CSE where it
// lies in the reference tree (3D/src/bssn3d/vendor/bssneqs_SSL_HD_dxsq.cpp).
// Nothing of that file is copied here: the recipe in oracle/Makefile passes
// its directory with -I and this file #includes it inside a point loop, the
// same way the reference's own oracle harness does (3D/src/bssn3d/oracle.py:99-127).
//
// Product code never links or loads this library. Tests use it to pin the
// oracle restatement (oracle/bssn_oracle.c) and the golden fixtures, and
// bench.py's reference arm times it as the reference's CPU implementation.
//
// Layout (shared with the oracle and the C-ABI):
//   F   [24][n]   fields in state order alpha, chi, K, gt0..5, beta0..2,
//                 At0..5, Gt0..2, B0..2            (3D/src/bssn3d/state.py:37-46)
//   D   [138][n]  derivatives: 72 first derivatives at index 3*f + axis for
//                 each field f, then 66 second derivatives at 72 + 6*m + p for
//                 the 11 fields m = alpha, chi, gt0..5, beta0..2 and the
//                 upper-triangular pair p = 00,01,02,11,12,22
//   S   [16]      eta, cahd_c, dt, dx, ssl_h, ssl_sigma, t, lambda0..3,
//                 lambda_f0..1, dx, dy, dz   (3D/src/bssn3d/fused_rhs_cuda.py:52-55)
//   OUT [24][n]   d/dt of each field, state order
#include <cmath>
#include <cstdio>

using std::pow;
using std::sqrt;
using std::exp;

#define FIELD(name, idx) const double* name = F + (long)(idx) * n;
#define G1(name, idx)                                  \
  const double* grad_0_##name = D + (long)(3 * (idx) + 0) * n; \
  const double* grad_1_##name = D + (long)(3 * (idx) + 1) * n; \
  const double* grad_2_##name = D + (long)(3 * (idx) + 2) * n;
#define G2(name, m)                                            \
  const double* grad2_0_0_##name = D + (long)(72 + 6 * (m) + 0) * n; \
  const double* grad2_0_1_##name = D + (long)(72 + 6 * (m) + 1) * n; \
  const double* grad2_0_2_##name = D + (long)(72 + 6 * (m) + 2) * n; \
  const double* grad2_1_1_##name = D + (long)(72 + 6 * (m) + 3) * n; \
  const double* grad2_1_2_##name = D + (long)(72 + 6 * (m) + 4) * n; \
  const double* grad2_2_2_##name = D + (long)(72 + 6 * (m) + 5) * n;
#define OUTP(name, idx) double* name = OUT + (long)(idx) * n;

extern "C" int dendro_ref_rhs_algebra(long n, const double* F, const double* D,
                                      const double* S, double* OUT, int nthreads) {
  FIELD(alpha, 0) FIELD(chi, 1) FIELD(K, 2)
  FIELD(gt0, 3) FIELD(gt1, 4) FIELD(gt2, 5) FIELD(gt3, 6) FIELD(gt4, 7) FIELD(gt5, 8)
  FIELD(beta0, 9) FIELD(beta1, 10) FIELD(beta2, 11)
  FIELD(At0, 12) FIELD(At1, 13) FIELD(At2, 14) FIELD(At3, 15) FIELD(At4, 16) FIELD(At5, 17)
  FIELD(Gt0, 18) FIELD(Gt1, 19) FIELD(Gt2, 20)
  FIELD(B0, 21) FIELD(B1, 22) FIELD(B2, 23)

  G1(alpha, 0) G1(chi, 1) G1(K, 2)
  G1(gt0, 3) G1(gt1, 4) G1(gt2, 5) G1(gt3, 6) G1(gt4, 7) G1(gt5, 8)
  G1(beta0, 9) G1(beta1, 10) G1(beta2, 11)
  G1(At0, 12) G1(At1, 13) G1(At2, 14) G1(At3, 15) G1(At4, 16) G1(At5, 17)
  G1(Gt0, 18) G1(Gt1, 19) G1(Gt2, 20)
  G1(B0, 21) G1(B1, 22) G1(B2, 23)

  G2(alpha, 0) G2(chi, 1)
  G2(gt0, 2) G2(gt1, 3) G2(gt2, 4) G2(gt3, 5) G2(gt4, 6) G2(gt5, 7)
  G2(beta0, 8) G2(beta1, 9) G2(beta2, 10)

  OUTP(a_rhs, 0) OUTP(chi_rhs, 1) OUTP(K_rhs, 2)
  OUTP(gt_rhs00, 3) OUTP(gt_rhs01, 4) OUTP(gt_rhs02, 5)
  OUTP(gt_rhs11, 6) OUTP(gt_rhs12, 7) OUTP(gt_rhs22, 8)
  OUTP(b_rhs0, 9) OUTP(b_rhs1, 10) OUTP(b_rhs2, 11)
  OUTP(At_rhs00, 12) OUTP(At_rhs01, 13) OUTP(At_rhs02, 14)
  OUTP(At_rhs11, 15) OUTP(At_rhs12, 16) OUTP(At_rhs22, 17)
  OUTP(Gt_rhs0, 18) OUTP(Gt_rhs1, 19) OUTP(Gt_rhs2, 20)
  OUTP(B_rhs0, 21) OUTP(B_rhs1, 22) OUTP(B_rhs2, 23)

  const double eta = S[0];
  const double BSSN_CAHD_C = S[1];
  const double dt = S[2];
  const double dx_i = S[3];
  const double h_ssl = S[4];
  const double sig_ssl = S[5];
  const double t = S[6];
  const double lambda[4] = {S[7], S[8], S[9], S[10]};
  const double lambda_f[2] = {S[11], S[12]};

  if (nthreads < 1) nthreads = 1;
#pragma omp parallel for schedule(static) num_threads(nthreads)
  for (long pp = 0; pp < n; ++pp) {
#include "bssneqs_SSL_HD_dxsq.cpp"
  }
  return 0;
}

// Test infrastructure only: a CPU harness around the reference's Hamiltonian
// and momentum constraints, Dendro-GR's physcon CSE
// (3D/src/bssn3d/vendor/physcon.cpp, the "Dendro: {{{ ... }}}" block holding
// ham[pp], lines 360-1287). oracle/Makefile extracts that block where it lies
// into _ref/physcon_block.inc at build time — the same block
// 3D/src/bssn3d/_codegen_constraints.py:36-43 extracts — and this file
// #includes it inside a point loop. Nothing of it is copied here.
//
// Layout as ref_harness.cpp: F [24][n], D [138][n]; out H [n], M [3][n].
#include <cmath>
#include <vector>

using std::pow;
using std::sqrt;

#define FIELD(name, idx) const double* name = F + (long)(idx) * n;
#define G1(name, idx)                                          \
  const double* grad_0_##name = D + (long)(3 * (idx) + 0) * n; \
  const double* grad_1_##name = D + (long)(3 * (idx) + 1) * n; \
  const double* grad_2_##name = D + (long)(3 * (idx) + 2) * n;
#define G2(name, m)                                                  \
  const double* grad2_0_0_##name = D + (long)(72 + 6 * (m) + 0) * n; \
  const double* grad2_0_1_##name = D + (long)(72 + 6 * (m) + 1) * n; \
  const double* grad2_0_2_##name = D + (long)(72 + 6 * (m) + 2) * n; \
  const double* grad2_1_1_##name = D + (long)(72 + 6 * (m) + 3) * n; \
  const double* grad2_1_2_##name = D + (long)(72 + 6 * (m) + 4) * n; \
  const double* grad2_2_2_##name = D + (long)(72 + 6 * (m) + 5) * n;

extern "C" int dendro_ref_constraints(long n, const double* F, const double* D, double* H,
                                      double* M, int nthreads) {
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
  double* ham = H;
  double* mom0 = M;
  double* mom1 = M + n;
  double* mom2 = M + 2 * n;
  // the block also emits psi4 (it alone reads the coordinates x, y, z)
  std::vector<double> p4r(n), p4i(n);
  double* psi4_real = p4r.data();
  double* psi4_img = p4i.data();
  const double x = 0.0, y = 0.0, z = 0.0;
  if (nthreads < 1) nthreads = 1;
#pragma omp parallel for schedule(static) num_threads(nthreads)
  for (long pp = 0; pp < n; ++pp) {
#include "physcon_block.inc"
  }
  return 0;
}

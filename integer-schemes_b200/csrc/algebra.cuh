// Pointwise BSSN right-hand side (CAHD + SSL variant) for one grid point,
// written for the sm_100a register file.
//
// The equations are those the reference evaluates through Dendro-GR's
// generated CSE (3D/src/bssn3d/vendor/bssneqs_SSL_HD_dxsq.cpp, outputs at
// lines 837-883): the moving-puncture BSSN system in chi form with
//   * 1+log-type lapse with SSL lapse locking
//       alpha_t = l0 b^k d_k alpha - 2 alpha K - sqrt(chi) h (alpha - sqrt(chi)) exp(-t^2 / 2 s^2)
//   * Gamma-driver shift  beta^i_t = 3/4 (lf0 + lf1 alpha) B^i + l1 b^k d_k beta^i
//   * CAHD damping on chi  chi_t += C dx^2 chi H / (dt (10 dx^2 + 1))
// Here they are stated in tensor form and scheduled in phases so that the
// live set stays inside the 255-register budget: the 138 derivatives are
// not held, they are fetched through `drv` at their point of use.
//
// Accessors: fld(k) -> field k at this point, drv(s) -> derivative slot s
// (layout of include/bssn_b200.h), emit(k, v) receives d/dt of field k.
#pragma once

namespace bssn {

struct Params {
  double eta, cahd_c, dt, dx, ssl_h, ssl_sigma, t;
  double lam0, lam1, lam2, lam3, lamf0, lamf1;
  double hx, hy, hz;
};

// field rows of the state
enum : int {
  F_ALPHA = 0, F_CHI = 1, F_K = 2, F_GT = 3, F_BETA = 9, F_AT = 12, F_GTI = 18, F_B = 21
};

// upper-triangular symmetric index 00 01 02 11 12 22
__host__ __device__ constexpr int sym(int i, int j) {
  return i <= j ? (i == 0 ? j : (i == 1 ? 2 + j : 5)) : sym(j, i);
}
__host__ __device__ constexpr int sym_i(int p) { return p < 3 ? 0 : (p < 5 ? 1 : 2); }
__host__ __device__ constexpr int sym_j(int p) { return p < 3 ? p : (p < 5 ? p - 2 : 2); }
// weight of a symmetric pair in a full double contraction
__host__ __device__ constexpr double symw(int p) { return (p == 0 || p == 3 || p == 5) ? 1.0 : 2.0; }

// derivative slots
__host__ __device__ constexpr int d1(int field, int axis) { return 3 * field + axis; }
// second-derivative field slot m: alpha, chi, gt0..5, beta0..2
__host__ __device__ constexpr int g2slot(int field) {
  return field == F_ALPHA ? 0 : (field == F_CHI ? 1 : (field < F_BETA ? 2 + field - F_GT : 8 + field - F_BETA));
}
__host__ __device__ constexpr int d2(int field, int i, int j) { return 72 + 6 * g2slot(field) + sym(i, j); }
constexpr int NDERIV = 138;
constexpr int NFIELD = 24;

template <class Fld, class Drv, class Emit>
__device__ __forceinline__ void rhs_point(const Fld& fld, const Drv& drv, const Emit& emit,
                                          const Params& P) {
  const double al = fld(F_ALPHA);
  const double chi = fld(F_CHI);
  const double ichi = 1.0 / chi;

  // ---- inverse conformal metric (adjugate / det) ----------------------
  double gu[6];
  {
    const double g00 = fld(F_GT + 0), g01 = fld(F_GT + 1), g02 = fld(F_GT + 2);
    const double g11 = fld(F_GT + 3), g12 = fld(F_GT + 4), g22 = fld(F_GT + 5);
    const double a00 = g11 * g22 - g12 * g12;
    const double a01 = g02 * g12 - g01 * g22;
    const double a02 = g01 * g12 - g02 * g11;
    const double a11 = g00 * g22 - g02 * g02;
    const double a12 = g01 * g02 - g00 * g12;
    const double a22 = g00 * g11 - g01 * g01;
    const double idet = 1.0 / (g00 * a00 + g01 * a01 + g02 * a02);
    gu[0] = a00 * idet; gu[1] = a01 * idet; gu[2] = a02 * idet;
    gu[3] = a11 * idet; gu[4] = a12 * idet; gu[5] = a22 * idet;
  }
#define GU(i, j) gu[sym(i, j)]
#define G(i, j) fld(F_GT + sym(i, j))
#define A(i, j) fld(F_AT + sym(i, j))
#define D1(f, a) drv(d1(f, a))
#define D2(f, i, j) drv(d2(f, i, j))

  double dchi[3], dal[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) { dchi[a] = D1(F_CHI, a); dal[a] = D1(F_ALPHA, a); }
  double divb = D1(F_BETA + 0, 0) + D1(F_BETA + 1, 1) + D1(F_BETA + 2, 2);

  // ---- A~^ij and A~_ij A~^ij ------------------------------------------
  double AU[6], AA;
  {
    double M[3][3];  // M = A~ . g~^-1
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int j = 0; j < 3; ++j) M[k][j] = A(k, 0) * GU(0, j) + A(k, 1) * GU(1, j) + A(k, 2) * GU(2, j);
#pragma unroll
    for (int p = 0; p < 6; ++p) {
      const int i = sym_i(p), j = sym_j(p);
      AU[p] = GU(i, 0) * M[0][j] + GU(i, 1) * M[1][j] + GU(i, 2) * M[2][j];
    }
    AA = 0.0;
#pragma unroll
    for (int p = 0; p < 6; ++p) AA += symw(p) * A(sym_i(p), sym_j(p)) * AU[p];
  }

  // ---- Christoffel symbols -------------------------------------------
  // C1[k][p] = G~_{k i j}, C2[k][p] = G~^k_{i j}, p = sym(i, j)
  double C1[3][6], C2[3][6];
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int p = 0; p < 6; ++p) {
      const int i = sym_i(p), j = sym_j(p);
      C1[k][p] = 0.5 * (D1(F_GT + sym(k, j), i) + D1(F_GT + sym(k, i), j) - D1(F_GT + p, k));
    }
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int p = 0; p < 6; ++p) C2[k][p] = GU(k, 0) * C1[0][p] + GU(k, 1) * C1[1][p] + GU(k, 2) * C1[2][p];
  double CalGt[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    double s = 0.0;
#pragma unroll
    for (int p = 0; p < 6; ++p) s += symw(p) * gu[p] * C2[i][p];
    CalGt[i] = s;
  }

  // ---- Gamma~^i and B^i right-hand sides -------------------------------
  {
    double dK[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) dK[a] = D1(F_K, a);
    const double b0 = fld(F_BETA + 0), b1 = fld(F_BETA + 1), b2 = fld(F_BETA + 2);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const double advGt = b0 * D1(F_GTI + i, 0) + b1 * D1(F_GTI + i, 1) + b2 * D1(F_GTI + i, 2);
      double v = advGt;
#pragma unroll
      for (int j = 0; j < 3; ++j) v -= CalGt[j] * D1(F_BETA + i, j);
      v += (2.0 / 3.0) * CalGt[i] * divb;
      double lapb = 0.0, gdb = 0.0;
#pragma unroll
      for (int p = 0; p < 6; ++p) lapb += symw(p) * gu[p] * D2(F_BETA + i, sym_i(p), sym_j(p));
#pragma unroll
      for (int j = 0; j < 3; ++j)
        gdb += GU(i, j) * (D2(F_BETA + 0, j, 0) + D2(F_BETA + 1, j, 1) + D2(F_BETA + 2, j, 2));
      v += lapb + (1.0 / 3.0) * gdb;
      double c2au = 0.0;
#pragma unroll
      for (int p = 0; p < 6; ++p) c2au += symw(p) * C2[i][p] * AU[p];
      double t1 = 0.0, t2 = 0.0;
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        t1 += AU[sym(i, j)] * dal[j];
        t2 += 3.0 * ichi * AU[sym(i, j)] * dchi[j] + (4.0 / 3.0) * GU(i, j) * dK[j];
      }
      v += -2.0 * t1 + 2.0 * al * c2au - al * t2;
      emit(F_GTI + i, v);
      const double advB = b0 * D1(F_B + i, 0) + b1 * D1(F_B + i, 1) + b2 * D1(F_B + i, 2);
      emit(F_B + i, v - P.eta * fld(F_B + i) + P.lam2 * advB - P.lam3 * advGt);
    }
  }

  // ---- W[j][k][l] = G~_{jk}^{l} (first kind, last index raised) --------
  double W[3][3][3];
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int l = 0; l < 3; ++l)
        W[j][k][l] = GU(l, 0) * C1[j][sym(k, 0)] + GU(l, 1) * C1[j][sym(k, 1)] + GU(l, 2) * C1[j][sym(k, 2)];
  // Gamma~^k G~_(ij)k with the metric-computed Gamma~^k
  double Yc[6];
#pragma unroll
  for (int p = 0; p < 6; ++p) {
    const int i = sym_i(p), j = sym_j(p);
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k) s += CalGt[k] * (C1[i][sym(j, k)] + C1[j][sym(i, k)]);
    Yc[p] = 0.5 * s;
  }

  // ---- chi pieces ------------------------------------------------------
  double guchi[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) guchi[k] = GU(k, 0) * dchi[0] + GU(k, 1) * dchi[1] + GU(k, 2) * dchi[2];
  const double sqchi = guchi[0] * dchi[0] + guchi[1] * dchi[1] + guchi[2] * dchi[2];
  const double gchial = guchi[0] * dal[0] + guchi[1] * dal[1] + guchi[2] * dal[2];
  double Dchi[6];
  double lapchi = 0.0;
#pragma unroll
  for (int p = 0; p < 6; ++p) {
    Dchi[p] = D2(F_CHI, sym_i(p), sym_j(p)) - (C2[0][p] * dchi[0] + C2[1][p] * dchi[1] + C2[2][p] * dchi[2]);
    lapchi += symw(p) * gu[p] * Dchi[p];
  }

  // ---- Ricci tensor and D_i D_j alpha, pair by pair -----------------------
  double X[6];
  double trR = 0.0, trX = 0.0, lapa = 0.0;
  const double hichi = 0.5 * ichi, qichi2 = 0.25 * ichi * ichi;
#pragma unroll
  for (int p = 0; p < 6; ++p) {
    const int i = sym_i(p), j = sym_j(p);
    const double gij = G(i, j);
    double r = 0.0;
#pragma unroll
    for (int q = 0; q < 6; ++q) r -= 0.5 * symw(q) * gu[q] * D2(F_GT + p, sym_i(q), sym_j(q));
#pragma unroll
    for (int k = 0; k < 3; ++k) r += 0.5 * (G(k, i) * D1(F_GTI + k, j) + G(k, j) * D1(F_GTI + k, i));
    r += Yc[p];
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int l = 0; l < 3; ++l)
        r += C2[k][sym(l, i)] * W[j][k][l] + C2[k][sym(l, j)] * W[i][k][l] + C2[k][sym(i, l)] * W[k][j][l];
    r += hichi * (Dchi[p] + gij * lapchi) - qichi2 * (dchi[i] * dchi[j] + 3.0 * gij * sqchi);
    const double dda = D2(F_ALPHA, i, j) - (C2[0][p] * dal[0] + C2[1][p] * dal[1] + C2[2][p] * dal[2]) +
                       hichi * (dal[i] * dchi[j] + dal[j] * dchi[i] - gij * gchial);
    const double x = al * r - dda;
    X[p] = x;
    const double w = symw(p) * gu[p];
    trR += w * r;
    trX += w * x;
    lapa += w * dda;
  }

  const double K = fld(F_K);
  const double b0 = fld(F_BETA + 0), b1 = fld(F_BETA + 1), b2 = fld(F_BETA + 2);
#define ADV(f) (b0 * D1(f, 0) + b1 * D1(f, 1) + b2 * D1(f, 2))

  // ---- A~_ij right-hand side ---------------------------------------------
  {
    double M[3][3];  // A~ . g~^-1
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int j = 0; j < 3; ++j) M[k][j] = A(k, 0) * GU(0, j) + A(k, 1) * GU(1, j) + A(k, 2) * GU(2, j);
    const double third_trX = (1.0 / 3.0) * trX;
#pragma unroll
    for (int p = 0; p < 6; ++p) {
      const int i = sym_i(p), j = sym_j(p);
      double v = ADV(F_AT + p);
#pragma unroll
      for (int k = 0; k < 3; ++k) v += A(i, k) * D1(F_BETA + k, j) + A(j, k) * D1(F_BETA + k, i);
      v -= (2.0 / 3.0) * A(i, j) * divb;
      v += chi * (X[p] - G(i, j) * third_trX);
      const double aga = M[i][0] * A(0, j) + M[i][1] * A(1, j) + M[i][2] * A(2, j);
      v += al * (K * A(i, j) - 2.0 * aga);
      emit(F_AT + p, v);
    }
  }

  // ---- K, chi ------------------------------------------------------------
  emit(F_K, ADV(F_K) - chi * lapa + al * (K * K * (1.0 / 3.0) + AA));
  {
    const double H = chi * trR + (2.0 / 3.0) * K * K - AA;
    const double dx2 = P.dx * P.dx;
    emit(F_CHI, ADV(F_CHI) + (2.0 / 3.0) * chi * (al * K - divb) +
                    P.cahd_c * dx2 * chi * H / (P.dt * (10.0 * dx2 + 1.0)));
  }

  // ---- lapse, shift, metric ------------------------------------------------
  {
    const double sq = sqrt(chi);
    emit(F_ALPHA, P.lam0 * ADV(F_ALPHA) - 2.0 * al * K -
                      sq * P.ssl_h * (al - sq) * exp(-0.5 * P.t * P.t / (P.ssl_sigma * P.ssl_sigma)));
    const double lf = 0.75 * (P.lamf0 + P.lamf1 * al);
#pragma unroll
    for (int i = 0; i < 3; ++i) emit(F_BETA + i, lf * fld(F_B + i) + P.lam1 * ADV(F_BETA + i));
#pragma unroll
    for (int p = 0; p < 6; ++p) {
      const int i = sym_i(p), j = sym_j(p);
      double v = ADV(F_GT + p);
#pragma unroll
      for (int k = 0; k < 3; ++k) v += G(i, k) * D1(F_BETA + k, j) + G(j, k) * D1(F_BETA + k, i);
      emit(F_GT + p, v - (2.0 / 3.0) * G(i, j) * divb - 2.0 * al * A(i, j));
    }
  }
#undef ADV
#undef GU
#undef G
#undef A
#undef D1
#undef D2
}

}  // namespace bssn

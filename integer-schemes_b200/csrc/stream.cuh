// Streaming form of the pointwise BSSN right-hand side (CAHD + SSL) for the
// sm_100a fused kernel.
//
// The fused kernel differentiates one field at a time out of a shared-memory
// tile. Instead of parking the 138 derivatives anywhere, each field's
// derivatives are handed to `Stream::consume_*` as soon as they exist and are
// folded into running accumulators; only the derivatives that enter
// nonlinearly (d gt, d chi, d alpha) are kept, and only until the
// quantities built from them (Christoffel symbols, Ricci tensor, D_iD_j alpha)
// are complete. Field order is fixed:
//
//   gt0..5 -> finish_metric -> chi -> alpha -> Gt0..2 -> finish_ricci ->
//   beta0..2 -> finish_beta -> K -> At0..5 -> B0..2 -> finalize
//
// The equations are those the reference evaluates through Dendro-GR's
// generated CSE (3D/src/bssn3d/vendor/bssneqs_SSL_HD_dxsq.cpp, outputs at
// lines 837-883), stated in tensor form:
//   alpha_t = l0 b.d alpha - 2 alpha K - sqrt(chi) h (alpha - sqrt(chi)) exp(-t^2/2s^2)
//   beta_t  = 3/4 (lf0 + lf1 alpha) B + l1 b.d beta
//   gt_t    = b.d gt + gt_ik d_j b^k + gt_jk d_i b^k - 2/3 gt div b - 2 alpha At
//   chi_t   = b.d chi + 2/3 chi (alpha K - div b) + C dx^2 chi H / (dt (10 dx^2 + 1))
//   At_t    = b.d At + At_ik d_j b^k + At_jk d_i b^k - 2/3 At div b
//             + chi (alpha R_ij - D_iD_j alpha)^TF + alpha (K At_ij - 2 At_ik gt^kl At_lj)
//   K_t     = b.d K - chi gt^ij D_iD_j alpha + alpha (K^2/3 + At_ij At^ij)
//   Gt_t    = b.d Gt^i - G^j d_j b^i + 2/3 G^i div b + gt^jk d_jk b^i + 1/3 gt^ij d_jk b^k
//             - 2 At^ij d_j alpha + 2 alpha G^i_jk At^jk - alpha (3/chi At^ij d_j chi + 4/3 gt^ij d_j K)
//   B_t     = Gt_t - eta B + l2 b.d B - l3 b.d Gt
// with G^k = gt^ij G^k_ij the metric-computed contracted Christoffel symbol
// (it also enters the Ricci term G^k G_(ij)k), R_ij = R~_ij + R^chi_ij, and
// H = chi gt^ij R_ij + 2/3 K^2 - At_ij At^ij. Constraints (CONS) follow the
// reference's ConstraintSolver (3D/src/bssn3d/constraints.py:38-62).
#pragma once

namespace bssn {

struct Params {
  double eta, cahd_c, dt, dx, ssl_h, ssl_sigma, t;
  double lam0, lam1, lam2, lam3, lamf0, lamf1;
  double hx, hy, hz;
};

// state rows
enum : int {
  F_ALPHA = 0, F_CHI = 1, F_K = 2, F_GT = 3, F_BETA = 9, F_AT = 12, F_GTI = 18, F_B = 21
};
constexpr int NDERIV = 138;
constexpr int NFIELD = 24;

// upper-triangular symmetric index 00 01 02 11 12 22 (written without
// recursion so that it folds to a constant inside unrolled loops and the
// register arrays it indexes stay in registers)
__host__ __device__ constexpr int sym(int i, int j) {
  return i <= j ? (i == 0 ? j : (i == 1 ? 2 + j : 5)) : (j == 0 ? i : (j == 1 ? 2 + i : 5));
}
__host__ __device__ constexpr int sym_i(int p) { return p < 3 ? 0 : (p < 5 ? 1 : 2); }
__host__ __device__ constexpr int sym_j(int p) { return p < 3 ? p : (p < 5 ? p - 2 : 2); }
__host__ __device__ constexpr double symw(int p) { return (p == 0 || p == 3 || p == 5) ? 1.0 : 2.0; }

// derivative slots of the C ABI layout
__host__ __device__ constexpr int d1slot(int field, int axis) { return 3 * field + axis; }
__host__ __device__ constexpr int g2slot(int field) {
  return field == F_ALPHA ? 0 : (field == F_CHI ? 1 : (field < F_BETA ? 2 + field - F_GT : 8 + field - F_BETA));
}
__host__ __device__ constexpr bool has_d2(int field) {
  return field == F_ALPHA || field == F_CHI || (field >= F_GT && field < F_AT);
}
__host__ __device__ constexpr int d2slot(int field, int p) { return 72 + 6 * g2slot(field) + p; }

// the order in which fields are differentiated and consumed
__host__ __device__ constexpr int stream_field(int idx) {
  return idx < 6 ? F_GT + idx
       : idx == 6 ? F_CHI
       : idx == 7 ? F_ALPHA
       : idx < 11 ? F_GTI + (idx - 8)
       : idx < 14 ? F_BETA + (idx - 11)
       : idx == 14 ? F_K
       : idx < 21 ? F_AT + (idx - 15)
       : F_B + (idx - 21);
}

struct NoCon {
  __device__ __forceinline__ void operator()(double, double, double, double) const {}
};

template <bool RATES, bool CONS, bool PV = false>
struct Stream {
  // Point values: held in registers, or (PV) re-read on every use from the
  // point's staged column pv[k * ps] (shared memory), which frees their
  // registers for the accumulators.
  const double* pv = nullptr;
  int ps = 0;
  double al_, chi_, K_, g_[6], b_[3];
  __device__ __forceinline__ double Al() const { return PV ? pv[F_ALPHA * ps] : al_; }
  __device__ __forceinline__ double Chi() const { return PV ? pv[F_CHI * ps] : chi_; }
  __device__ __forceinline__ double Kv() const { return PV ? pv[F_K * ps] : K_; }
  __device__ __forceinline__ double Gv(int p) const { return PV ? pv[(F_GT + p) * ps] : g_[p]; }
  __device__ __forceinline__ double Bv(int i) const { return PV ? pv[(F_BETA + i) * ps] : b_[i]; }
  double ichi;
  double gu[6];
  double AU[6], AA;
  // rates
  double r_gt[6], r_At[6], r_Gt[3], ko_Gt[3], r_beta[3], r_B[3], r_alpha, r_chi, r_K;
  // geometry
  double dg[3][6];       // d_a gt_p (until finish_metric)
  double C2[3][6];       // G~^k_p
  double CalGt[3];
  double R[6], X[6];     // Ricci accumulator; X = alpha R - D_iD_j alpha
  double dchi[3], guchi[3];
  double lapa, trR, trX, divb, dd[3];
  double mom[3];

  template <class Fld>
  __device__ __forceinline__ void init(const Fld& fld) {
    if (!PV) {
      al_ = fld(F_ALPHA);
      chi_ = fld(F_CHI);
      K_ = fld(F_K);
#pragma unroll
      for (int p = 0; p < 6; ++p) g_[p] = fld(F_GT + p);
#pragma unroll
      for (int i = 0; i < 3; ++i) b_[i] = fld(F_BETA + i);
    }
    ichi = 1.0 / Chi();
    {
      const double a00 = Gv(3) * Gv(5) - Gv(4) * Gv(4);
      const double a01 = Gv(2) * Gv(4) - Gv(1) * Gv(5);
      const double a02 = Gv(1) * Gv(4) - Gv(2) * Gv(3);
      const double a11 = Gv(0) * Gv(5) - Gv(2) * Gv(2);
      const double a12 = Gv(1) * Gv(2) - Gv(0) * Gv(4);
      const double a22 = Gv(0) * Gv(3) - Gv(1) * Gv(1);
      const double idet = 1.0 / (Gv(0) * a00 + Gv(1) * a01 + Gv(2) * a02);
      gu[0] = a00 * idet; gu[1] = a01 * idet; gu[2] = a02 * idet;
      gu[3] = a11 * idet; gu[4] = a12 * idet; gu[5] = a22 * idet;
    }
    {
      double A[6];
#pragma unroll
      for (int p = 0; p < 6; ++p) A[p] = fld(F_AT + p);
      double M[3][3];  // A~ . g~^-1
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int j = 0; j < 3; ++j)
          M[k][j] = A[sym(k, 0)] * gu[sym(0, j)] + A[sym(k, 1)] * gu[sym(1, j)] + A[sym(k, 2)] * gu[sym(2, j)];
      AA = 0.0;
#pragma unroll
      for (int p = 0; p < 6; ++p) {
        const int i = sym_i(p), j = sym_j(p);
        AU[p] = gu[sym(i, 0)] * M[0][j] + gu[sym(i, 1)] * M[1][j] + gu[sym(i, 2)] * M[2][j];
        AA += symw(p) * A[p] * AU[p];
      }
    }
#pragma unroll
    for (int p = 0; p < 6; ++p) { R[p] = 0.0; X[p] = 0.0; r_At[p] = 0.0; }
#pragma unroll
    for (int i = 0; i < 3; ++i) { r_Gt[i] = 0.0; r_B[i] = 0.0; dd[i] = 0.0; mom[i] = 0.0; }
    divb = 0.0;
  }

  __device__ __forceinline__ double adv(const double (&d1)[3]) const {
    return Bv(0) * d1[0] + Bv(1) * d1[1] + Bv(2) * d1[2];
  }

  // ---- gt_p: first derivatives kept, second derivatives into R_p ------------
  __device__ __forceinline__ void consume_gt(int p, const double (&d1)[3], const double (&d2)[6], double ko) {
#pragma unroll
    for (int a = 0; a < 3; ++a) dg[a][p] = d1[a];
    r_gt[p] = adv(d1) + ko;
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < 6; ++q) s += symw(q) * gu[q] * d2[q];
    R[p] = -0.5 * s;
  }

  // ---- Christoffel symbols and the quadratic Ricci terms ---------------------
  __device__ __forceinline__ void finish_metric() {
    double C1[3][6];  // G~_{k p}
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int p = 0; p < 6; ++p) {
        const int i = sym_i(p), j = sym_j(p);
        C1[k][p] = 0.5 * (dg[i][sym(k, j)] + dg[j][sym(k, i)] - dg[k][p]);
      }
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int p = 0; p < 6; ++p)
        C2[k][p] = gu[sym(k, 0)] * C1[0][p] + gu[sym(k, 1)] * C1[1][p] + gu[sym(k, 2)] * C1[2][p];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      double s = 0.0;
#pragma unroll
      for (int p = 0; p < 6; ++p) s += symw(p) * gu[p] * C2[i][p];
      CalGt[i] = s;
    }
    // W[j][k][l] = G~_jk^l (first kind, last index raised)
    double W[3][3][3];
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int l = 0; l < 3; ++l)
          W[j][k][l] = gu[sym(l, 0)] * C1[j][sym(k, 0)] + gu[sym(l, 1)] * C1[j][sym(k, 1)] +
                       gu[sym(l, 2)] * C1[j][sym(k, 2)];
#pragma unroll
    for (int p = 0; p < 6; ++p) {
      const int i = sym_i(p), j = sym_j(p);
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < 3; ++k) s += CalGt[k] * (C1[i][sym(j, k)] + C1[j][sym(i, k)]);
      double q = 0.5 * s;
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int l = 0; l < 3; ++l)
          q += C2[k][sym(l, i)] * W[j][k][l] + C2[k][sym(l, j)] * W[i][k][l] + C2[k][sym(i, l)] * W[k][j][l];
      R[p] += q;
    }
    if (RATES) {
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        double c2au = 0.0;
#pragma unroll
        for (int p = 0; p < 6; ++p) c2au += symw(p) * C2[i][p] * AU[p];
        r_Gt[i] += 2.0 * Al() * c2au;
      }
    }
  }

  // ---- chi ----------------------------------------------------------------------
  __device__ __forceinline__ void consume_chi(const double (&d1)[3], const double (&d2)[6], double ko) {
#pragma unroll
    for (int a = 0; a < 3; ++a) dchi[a] = d1[a];
    r_chi = adv(d1) + ko;
#pragma unroll
    for (int k = 0; k < 3; ++k)
      guchi[k] = gu[sym(k, 0)] * dchi[0] + gu[sym(k, 1)] * dchi[1] + gu[sym(k, 2)] * dchi[2];
    const double sqchi = guchi[0] * dchi[0] + guchi[1] * dchi[1] + guchi[2] * dchi[2];
    double Dchi[6], lapchi = 0.0;
#pragma unroll
    for (int p = 0; p < 6; ++p) {
      Dchi[p] = d2[p] - (C2[0][p] * dchi[0] + C2[1][p] * dchi[1] + C2[2][p] * dchi[2]);
      lapchi += symw(p) * gu[p] * Dchi[p];
    }
    const double hichi = 0.5 * ichi, qichi2 = 0.25 * ichi * ichi;
#pragma unroll
    for (int p = 0; p < 6; ++p) {
      const int i = sym_i(p), j = sym_j(p);
      R[p] += hichi * (Dchi[p] + Gv(p) * lapchi) - qichi2 * (dchi[i] * dchi[j] + 3.0 * Gv(p) * sqchi);
    }
    if (RATES) {
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        const double t = AU[sym(i, 0)] * dchi[0] + AU[sym(i, 1)] * dchi[1] + AU[sym(i, 2)] * dchi[2];
        r_Gt[i] -= 3.0 * Al() * ichi * t;
      }
    }
  }

  // ---- alpha: D_i D_j alpha ------------------------------------------------------
  __device__ __forceinline__ void consume_alpha(const double (&dal)[3], const double (&d2)[6], double ko, double lam0) {
    r_alpha = lam0 * adv(dal) + ko;
    const double gchial = guchi[0] * dal[0] + guchi[1] * dal[1] + guchi[2] * dal[2];
    const double hichi = 0.5 * ichi;
    lapa = 0.0;
#pragma unroll
    for (int p = 0; p < 6; ++p) {
      const int i = sym_i(p), j = sym_j(p);
      const double dda = d2[p] - (C2[0][p] * dal[0] + C2[1][p] * dal[1] + C2[2][p] * dal[2]) +
                         hichi * (dal[i] * dchi[j] + dal[j] * dchi[i] - Gv(p) * gchial);
      X[p] = -dda;
      lapa += symw(p) * gu[p] * dda;
    }
    if (RATES) {
#pragma unroll
      for (int i = 0; i < 3; ++i)
        r_Gt[i] -= 2.0 * (AU[sym(i, 0)] * dal[0] + AU[sym(i, 1)] * dal[1] + AU[sym(i, 2)] * dal[2]);
    }
  }

  // ---- Gt^k: derivative terms of R and advection ------------------------------------
  __device__ __forceinline__ void consume_Gt(int k, const double (&d1)[3], double ko, double lam3) {
    const double a = adv(d1);
    r_Gt[k] += a;
    ko_Gt[k] = ko;
    r_B[k] -= lam3 * a;
#pragma unroll
    for (int p = 0; p < 6; ++p) {
      const int i = sym_i(p), j = sym_j(p);
      R[p] += 0.5 * (Gv(sym(k, i)) * d1[j] + Gv(sym(k, j)) * d1[i]);
    }
  }

  __device__ __forceinline__ void finish_ricci() {
    trR = 0.0;
    trX = 0.0;
#pragma unroll
    for (int p = 0; p < 6; ++p) {
      X[p] += Al() * R[p];
      trR += symw(p) * gu[p] * R[p];
      trX += symw(p) * gu[p] * X[p];
    }
  }

  // ---- beta^k -----------------------------------------------------------------
  template <class Fld>
  __device__ __forceinline__ void consume_beta(int k, const double (&d1)[3], const double (&d2)[6], double ko,
                                               double lam1, const Fld& fld) {
    divb += d1[k];
    r_beta[k] = lam1 * adv(d1) + ko;
#pragma unroll
    for (int p = 0; p < 6; ++p) {
      const int i = sym_i(p), j = sym_j(p);
      r_gt[p] += Gv(sym(i, k)) * d1[j] + Gv(sym(j, k)) * d1[i];
      r_At[p] += fld(F_AT + sym(i, k)) * d1[j] + fld(F_AT + sym(j, k)) * d1[i];
    }
    double lapb = 0.0;
#pragma unroll
    for (int q = 0; q < 6; ++q) lapb += symw(q) * gu[q] * d2[q];
    r_Gt[k] += lapb - (CalGt[0] * d1[0] + CalGt[1] * d1[1] + CalGt[2] * d1[2]);
#pragma unroll
    for (int j = 0; j < 3; ++j) dd[j] += d2[sym(j, k)];
  }

  template <class Fld>
  __device__ __forceinline__ void finish_beta(const Fld& fld) {
    const double t23 = 2.0 / 3.0;
#pragma unroll
    for (int p = 0; p < 6; ++p) {
      const double A = fld(F_AT + p);
      r_gt[p] += -t23 * Gv(p) * divb - 2.0 * Al() * A;
      r_At[p] += -t23 * A * divb;
    }
    r_chi += t23 * Chi() * (Al() * Kv() - divb);
#pragma unroll
    for (int i = 0; i < 3; ++i)
      r_Gt[i] += t23 * CalGt[i] * divb +
                 (1.0 / 3.0) * (gu[sym(i, 0)] * dd[0] + gu[sym(i, 1)] * dd[1] + gu[sym(i, 2)] * dd[2]);
  }

  // ---- K -------------------------------------------------------------------------
  __device__ __forceinline__ void consume_K(const double (&d1)[3], double ko) {
    r_K = adv(d1) + ko;
    if (RATES) {
#pragma unroll
      for (int i = 0; i < 3; ++i)
        r_Gt[i] -= (4.0 / 3.0) * Al() * (gu[sym(i, 0)] * d1[0] + gu[sym(i, 1)] * d1[1] + gu[sym(i, 2)] * d1[2]);
    }
    if (CONS) {
#pragma unroll
      for (int i = 0; i < 3; ++i) mom[i] -= (2.0 / 3.0) * d1[i];
    }
  }

  // ---- At_p ----------------------------------------------------------------------
  __device__ __forceinline__ void consume_At(int p, const double (&d1)[3], double ko) {
    r_At[p] += adv(d1) + ko;
    if (CONS) {
      // g~^jk d_j A~_ki, A~_ki = A~_p for {k, i} = pair p
      const int i = sym_i(p), k = sym_j(p);
      mom[i] += gu[sym(0, k)] * d1[0] + gu[sym(1, k)] * d1[1] + gu[sym(2, k)] * d1[2];
      if (i != k) mom[k] += gu[sym(0, i)] * d1[0] + gu[sym(1, i)] * d1[1] + gu[sym(2, i)] * d1[2];
    }
  }

  // ---- B^k -------------------------------------------------------------------------
  __device__ __forceinline__ void consume_B(int k, const double (&d1)[3], double ko, double lam2) {
    r_B[k] += lam2 * adv(d1) + ko;
  }

  // ---- closing terms; emit(field, rate) and con(H, M0, M1, M2) ------------------------
  template <class Fld, class Emit, class Con>
  __device__ __forceinline__ void finalize(const Fld& fld, const Params& P, const Emit& emit, const Con& con) {
    const double H = Chi() * trR + (2.0 / 3.0) * Kv() * Kv() - AA;
    if (CONS) {
      double A[6];
#pragma unroll
      for (int p = 0; p < 6; ++p) A[p] = fld(F_AT + p);
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        double m = 0.0, c = 0.0;
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            const int ji = sym(j, i);
            m += gu[sym(j, k)] * (C2[0][ji] * A[sym(k, 0)] + C2[1][ji] * A[sym(k, 1)] + C2[2][ji] * A[sym(k, 2)]);
            c += gu[sym(j, k)] * A[sym(k, i)] * dchi[j];
          }
        const double gA = fld(F_GTI + 0) * A[sym(i, 0)] + fld(F_GTI + 1) * A[sym(i, 1)] + fld(F_GTI + 2) * A[sym(i, 2)];
        mom[i] += -m - gA - 1.5 * c * ichi;
      }
      con(H, mom[0], mom[1], mom[2]);
    }
    if (!RATES) return;
    // A~_ij
    {
      double A[6];
#pragma unroll
      for (int p = 0; p < 6; ++p) A[p] = fld(F_AT + p);
      double M[3][3];
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int j = 0; j < 3; ++j)
          M[k][j] = A[sym(k, 0)] * gu[sym(0, j)] + A[sym(k, 1)] * gu[sym(1, j)] + A[sym(k, 2)] * gu[sym(2, j)];
      const double third_trX = (1.0 / 3.0) * trX;
#pragma unroll
      for (int p = 0; p < 6; ++p) {
        const int i = sym_i(p), j = sym_j(p);
        const double aga = M[i][0] * A[sym(0, j)] + M[i][1] * A[sym(1, j)] + M[i][2] * A[sym(2, j)];
        emit(F_AT + p, r_At[p] + Chi() * (X[p] - Gv(p) * third_trX) + Al() * (Kv() * A[p] - 2.0 * aga));
      }
    }
    emit(F_K, r_K - Chi() * lapa + Al() * (Kv() * Kv() * (1.0 / 3.0) + AA));
    {
      const double dx2 = P.dx * P.dx;
      emit(F_CHI, r_chi + P.cahd_c * dx2 * Chi() * H / (P.dt * (10.0 * dx2 + 1.0)));
    }
    {
      const double sq = sqrt(Chi());
      emit(F_ALPHA, r_alpha - 2.0 * Al() * Kv() -
                        sq * P.ssl_h * (Al() - sq) * exp(-0.5 * P.t * P.t / (P.ssl_sigma * P.ssl_sigma)));
    }
    const double lf = 0.75 * (P.lamf0 + P.lamf1 * Al());
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const double Bi = fld(F_B + i);
      emit(F_BETA + i, r_beta[i] + lf * Bi);
      emit(F_B + i, r_Gt[i] - P.eta * Bi + r_B[i]);
      emit(F_GTI + i, r_Gt[i] + ko_Gt[i]);
    }
#pragma unroll
    for (int p = 0; p < 6; ++p) emit(F_GT + p, r_gt[p]);
  }

  // Route field f's derivatives to its consumer (f known at compile time after unrolling).
  template <class Fld>
  __device__ __forceinline__ void consume(int f, const double (&d1)[3], const double (&d2)[6], double ko,
                                          const Params& P, const Fld& fld) {
    if (f >= F_GT && f < F_GT + 6) {
      consume_gt(f - F_GT, d1, d2, ko);
      if (f == F_GT + 5) finish_metric();
    } else if (f == F_CHI) {
      consume_chi(d1, d2, ko);
    } else if (f == F_ALPHA) {
      consume_alpha(d1, d2, ko, P.lam0);
    } else if (f >= F_GTI && f < F_GTI + 3) {
      consume_Gt(f - F_GTI, d1, ko, P.lam3);
      if (f == F_GTI + 2) finish_ricci();
    } else if (f >= F_BETA && f < F_BETA + 3) {
      consume_beta(f - F_BETA, d1, d2, ko, P.lam1, fld);
      if (f == F_BETA + 2) finish_beta(fld);
    } else if (f == F_K) {
      consume_K(d1, ko);
    } else if (f >= F_AT && f < F_AT + 6) {
      consume_At(f - F_AT, d1, ko);
    } else {
      consume_B(f - F_B, d1, ko, P.lam2);
    }
  }
};

}  // namespace bssn

/*
 * TEST INFRASTRUCTURE — the CPU oracle for the BSSN right-hand side and its
 * RK4 stage update. Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load this library, and only as the checker. The product
 * (integer-schemes_b200/) never links or calls it.
 *
 * It restates, in plain C and in tensor-index form, what the reference
 * computes on this path:
 *   - centred 6th-order first/second-derivative stencils and the 6th/8th-order
 *     Kreiss-Oliger stencils with edge padding by the stencil's own reach
 *       common/src/mcs_common/derivatives.py:35-49 (coefficients),
 *       derivatives.py:78-88 (_apply: edge pad by the stencil's reach)
 *   - the 138-derivative bundle (mixed second derivative = first derivative
 *     along the lower axis, then along the higher one)
 *       3D/src/bssn3d/derivative_bundle.py:31-48
 *   - the CAHD+SSL BSSN algebra that Dendro-GR's generated CSE evaluates
 *       3D/src/bssn3d/vendor/bssneqs_SSL_HD_dxsq.cpp (24 outputs, lines 837-883),
 *       written here from the BSSN equations, not from that file's statements
 *   - Kreiss-Oliger dissipation, RK4 stages and algebraic enforcement
 *       3D/src/bssn3d/evolve.py:76-84 (_ko), :93-119 (enforce), :125-137 (step)
 *   - periodic ghost sync  evolve.py:65-73
 *
 * Parity of this restatement is pinned against the reference's own compiled
 * algebra (oracle/_ref) and the golden fixtures in tests/golden/.
 *
 * Layouts are those of the C-ABI (include/bssn_b200.h): fields [24][n] in
 * state order, derivatives [138][n], the 16-scalar pack S.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NF 24
#define NDERIV 138
enum {
  ALPHA = 0, CHI = 1, KK = 2, GT = 3, BETA = 9, AT = 12, GTI = 18, BB = 21
};

/* upper-triangular symmetric index: 00 01 02 11 12 22 */
static const int SYM[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
static const int SYM_I[6] = {0, 0, 0, 1, 1, 2};
static const int SYM_J[6] = {0, 1, 2, 1, 2, 2};

/* the 11 fields with second derivatives, in derivative-slot order */
static const int G2FIELDS[11] = {ALPHA, CHI, GT + 0, GT + 1, GT + 2, GT + 3,
                                 GT + 4, GT + 5, BETA + 0, BETA + 1, BETA + 2};

int oracle_g2_slot(int field) {
  for (int m = 0; m < 11; ++m)
    if (G2FIELDS[m] == field) return m;
  return -1;
}

/* ------------------------------------------------------------------ */
/* stencils                                                            */
/* ------------------------------------------------------------------ */

/* Stencil kinds. Every stencil is the integer-coefficient sum of
 * common/src/mcs_common/derivatives.py:35-49 over the taps in[clamp(p + k)],
 * symmetric taps paired first and combined from the outermost pair inwards
 * with fused multiply-adds, then scaled once:
 *   C1  45 (v1 - v-1) - 9 (v2 - v-2) + (v3 - v-3)                   / 60
 *   C2  -490 v0 + 270 (v1 + v-1) - 27 (v2 + v-2) + 2 (v3 + v-3)      / 180
 *   KO6 -20 v0 + 15 (v1 + v-1) - 6 (v2 + v-2) + (v3 + v-3)          / 64
 *   KO8 -70 v0 + 56 (v1 + v-1) - 28 (v2 + v-2) + 8 (v3 + v-3) - (v4 + v-4)  / 256
 * The reference sums (c_k / den * factor) * v_k in tap order
 * (derivatives.py:78-88); the two differ by rounding only. The GPU kernels
 * evaluate exactly these operations in this order, so their derivatives equal
 * this restatement bit for bit. */
enum { ST_C1 = 0, ST_C2 = 1, ST_KO6 = 2, ST_KO8 = 3 };

static inline long clampl(long v, long lo, long hi) {
  return v < lo ? lo : (v > hi ? hi : v);
}

static double stencil_sum(int kind, const double* v /* centre tap, v[-4..4] */) {
  if (kind == ST_C1) {
    const double a1 = v[1] - v[-1], a2 = v[2] - v[-2], a3 = v[3] - v[-3];
    return fma(45.0, a1, fma(-9.0, a2, a3));
  }
  const double s1 = v[1] + v[-1], s2 = v[2] + v[-2], s3 = v[3] + v[-3];
  if (kind == ST_C2) return fma(-490.0, v[0], fma(270.0, s1, fma(-27.0, s2, s3 + s3)));
  if (kind == ST_KO6) return fma(-20.0, v[0], fma(15.0, s1, fma(-6.0, s2, s3)));
  const double s4 = v[4] + v[-4];
  return fma(-70.0, v[0], fma(56.0, s1, fma(-28.0, s2, fma(8.0, s3, -s4))));
}

/* One pass of a centred stencil along `axis` of a (Sx,Sy,Sz) array, edge
 * padded by clamping the tap index (derivatives.py:83-84):
 * out = stencil_sum * scale, or the unscaled sum when scaled == 0. */
static void apply_axis(const double* in, double* out, const long S[3], int axis, int kind,
                       int scaled, double scale) {
  const int reach = kind == ST_KO8 ? 4 : 3;
  const long Sx = S[0], Sy = S[1], Sz = S[2];
  const long stride[3] = {Sy * Sz, Sz, 1};
#pragma omp parallel for collapse(2) schedule(static)
  for (long x = 0; x < Sx; ++x)
    for (long y = 0; y < Sy; ++y)
      for (long z = 0; z < Sz; ++z) {
        const long p[3] = {x, y, z};
        const long base = x * stride[0] + y * stride[1] + z;
        const long pa = p[axis];
        const long off0 = base - pa * stride[axis];
        double v[9];
        for (int k = -reach; k <= reach; ++k)
          v[4 + k] = in[off0 + clampl(pa + k, 0, S[axis] - 1) * stride[axis]];
        const double sum = stencil_sum(kind, v + 4);
        out[base] = scaled ? sum * scale : sum;
      }
}

/* scale factors of the stencils on spacing h (the GPU kernels form them with
 * the same operations) */
static double f1_of(double h) { return 1.0 / (60.0 * h); }
static double f2_of(double h) { return 1.0 / ((180.0 * h) * h); }

/* The 138 derivatives of a (24,Sx,Sy,Sz) state. D is [138][n]. */
void oracle_derivatives(const double* F, long Sx, long Sy, long Sz, double dx,
                        double dy, double dz, double* D) {
  const long S[3] = {Sx, Sy, Sz};
  const long n = Sx * Sy * Sz;
  const double h[3] = {dx, dy, dz};
  double* tmp = (double*)malloc(sizeof(double) * n);
  for (int f = 0; f < NF; ++f)
    for (int a = 0; a < 3; ++a)
      apply_axis(F + f * n, D + (long)(3 * f + a) * n, S, a, ST_C1, 1, f1_of(h[a]));
  for (int m = 0; m < 11; ++m) {
    const double* u = F + (long)G2FIELDS[m] * n;
    for (int p = 0; p < 6; ++p) {
      const int i = SYM_I[p], j = SYM_J[p];
      double* out = D + (long)(72 + 6 * m + p) * n;
      if (i == j) {
        apply_axis(u, out, S, i, ST_C2, 1, f2_of(h[i]));
      } else {
        apply_axis(u, tmp, S, i, ST_C1, 0, 0.0);
        apply_axis(tmp, out, S, j, ST_C1, 1, f1_of(h[i]) * f1_of(h[j]));
      }
    }
  }
  free(tmp);
}

/* Kreiss-Oliger dissipation summed over the three axes, for all 24 fields,
 * added in axis order to a zero accumulator (evolve.py:76-84). ko_order 6 or 8. */
void oracle_ko(const double* F, long Sx, long Sy, long Sz, double dx, double dy,
               double dz, double sigma, int ko_order, double* KO) {
  const long S[3] = {Sx, Sy, Sz};
  const long n = Sx * Sy * Sz;
  const double h[3] = {dx, dy, dz};
  double* tmp = (double*)malloc(sizeof(double) * n);
  const int kind = ko_order == 8 ? ST_KO8 : ST_KO6;
  const double den = ko_order == 8 ? 256.0 : 64.0;
  for (int f = 0; f < NF; ++f) {
    double* acc = KO + (long)f * n;
    for (long q = 0; q < n; ++q) acc[q] = 0.0;
    for (int a = 0; a < 3; ++a) {
      apply_axis(F + (long)f * n, tmp, S, a, kind, 1, sigma / (den * h[a]));
      for (long q = 0; q < n; ++q) acc[q] = acc[q] + tmp[q];
    }
  }
  free(tmp);
}

/* ------------------------------------------------------------------ */
/* the pointwise BSSN algebra                                          */
/* ------------------------------------------------------------------ */

typedef struct {
  double eta, cahd_c, dt, dx, ssl_h, ssl_sigma, t;
  double lam[4], lamf[2];
} params_t;

static params_t unpack(const double* S) {
  params_t p;
  p.eta = S[0]; p.cahd_c = S[1]; p.dt = S[2]; p.dx = S[3];
  p.ssl_h = S[4]; p.ssl_sigma = S[5]; p.t = S[6];
  for (int i = 0; i < 4; ++i) p.lam[i] = S[7 + i];
  p.lamf[0] = S[11]; p.lamf[1] = S[12];
  return p;
}

/* One point. f[24] fields, d[138] derivatives, out[24] rates; H_out (may be
 * NULL) receives the Hamiltonian constraint chi*R~ + 2/3 K^2 - A~_ij A~^ij. */
static void point_rhs(const double* f, const double* d, const params_t* P,
                      double* out, double* H_out) {
#define D1(F, A) d[3 * (F) + (A)]
#define D2(F, I, J) d[72 + 6 * oracle_g2_slot(F) + SYM[I][J]]
  const double al = f[ALPHA], chi = f[CHI], K = f[KK];
  double g[3][3], A[3][3], beta[3], Gt[3], Bv[3];
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) {
      g[i][j] = f[GT + SYM[i][j]];
      A[i][j] = f[AT + SYM[i][j]];
    }
    beta[i] = f[BETA + i];
    Gt[i] = f[GTI + i];
    Bv[i] = f[BB + i];
  }
  /* inverse conformal metric from the adjugate */
  double adj[3][3];
  adj[0][0] = g[1][1] * g[2][2] - g[1][2] * g[1][2];
  adj[0][1] = g[0][2] * g[1][2] - g[0][1] * g[2][2];
  adj[0][2] = g[0][1] * g[1][2] - g[0][2] * g[1][1];
  adj[1][1] = g[0][0] * g[2][2] - g[0][2] * g[0][2];
  adj[1][2] = g[0][1] * g[0][2] - g[0][0] * g[1][2];
  adj[2][2] = g[0][0] * g[1][1] - g[0][1] * g[0][1];
  adj[1][0] = adj[0][1]; adj[2][0] = adj[0][2]; adj[2][1] = adj[1][2];
  const double det = g[0][0] * adj[0][0] + g[0][1] * adj[0][1] + g[0][2] * adj[0][2];
  double gu[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) gu[i][j] = adj[i][j] / det;

  /* Christoffel symbols: C1[k][i][j] = G~_kij, C2[k][i][j] = G~^k_ij */
  double C1[3][3][3], C2[3][3][3], C3[3][3][3];
  for (int k = 0; k < 3; ++k)
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        C1[k][i][j] = 0.5 * (D1(GT + SYM[k][j], i) + D1(GT + SYM[k][i], j) -
                             D1(GT + SYM[i][j], k));
  for (int k = 0; k < 3; ++k)
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        double s = 0.0;
        for (int l = 0; l < 3; ++l) s += gu[k][l] * C1[l][i][j];
        C2[k][i][j] = s;
      }
  double CalGt[3];
  for (int i = 0; i < 3; ++i) {
    double s = 0.0;
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 3; ++k) s += gu[j][k] * C2[i][j][k];
    CalGt[i] = s;
  }
  double dchi[3], dal[3], dK[3], guchi[3];
  for (int a = 0; a < 3; ++a) {
    dchi[a] = D1(CHI, a);
    dal[a] = D1(ALPHA, a);
    dK[a] = D1(KK, a);
  }
  for (int k = 0; k < 3; ++k) {
    double s = 0.0;
    for (int l = 0; l < 3; ++l) s += gu[k][l] * dchi[l];
    guchi[k] = s;
  }
  /* physical Christoffel symbols */
  for (int k = 0; k < 3; ++k)
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        C3[k][i][j] = C2[k][i][j] - (0.5 / chi) * ((k == i ? dchi[j] : 0.0) +
                                                   (k == j ? dchi[i] : 0.0) -
                                                   g[i][j] * guchi[k]);
  double divb = 0.0;
  for (int i = 0; i < 3; ++i) divb += D1(BETA + i, i);

  /* D_i D_j alpha (physical) */
  double DDa[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = D2(ALPHA, i, j);
      for (int k = 0; k < 3; ++k) s -= C3[k][i][j] * dal[k];
      DDa[i][j] = s;
    }

  /* conformal Laplacian pieces of chi */
  double lapchi = 0.0, sqchi = 0.0;
  for (int l = 0; l < 3; ++l)
    for (int m = 0; m < 3; ++m) {
      double s = D2(CHI, l, m);
      for (int k = 0; k < 3; ++k) s -= C2[k][l][m] * dchi[k];
      lapchi += gu[l][m] * s;
      sqchi += gu[l][m] * dchi[l] * dchi[m];
    }

  /* Ricci tensor R_ij = R~_ij + R^chi_ij */
  double R[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double r = 0.0;
      for (int l = 0; l < 3; ++l)
        for (int m = 0; m < 3; ++m) r -= 0.5 * gu[l][m] * D2(GT + SYM[i][j], l, m);
      for (int k = 0; k < 3; ++k)
        r += 0.5 * (g[k][i] * D1(GTI + k, j) + g[k][j] * D1(GTI + k, i));
      for (int k = 0; k < 3; ++k) r += 0.5 * CalGt[k] * (C1[i][j][k] + C1[j][i][k]);
      for (int k = 0; k < 3; ++k)
        for (int l = 0; l < 3; ++l)
          for (int m = 0; m < 3; ++m)
            r += gu[l][m] * (C2[k][l][i] * C1[j][k][m] + C2[k][l][j] * C1[i][k][m] +
                             C2[k][i][m] * C1[k][l][j]);
      double Dchi = D2(CHI, i, j);
      for (int k = 0; k < 3; ++k) Dchi -= C2[k][i][j] * dchi[k];
      r += (0.5 / chi) * (Dchi + g[i][j] * lapchi) -
           (0.25 / (chi * chi)) * (dchi[i] * dchi[j] + 3.0 * g[i][j] * sqchi);
      R[i][j] = r;
    }

  double X[3][3], trX = 0.0, trR = 0.0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      X[i][j] = al * R[i][j] - DDa[i][j];
      trX += gu[i][j] * X[i][j];
      trR += gu[i][j] * R[i][j];
    }
  double AU[3][3], AA = 0.0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0.0;
      for (int k = 0; k < 3; ++k)
        for (int l = 0; l < 3; ++l) s += gu[i][k] * gu[j][l] * A[k][l];
      AU[i][j] = s;
    }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) AA += A[i][j] * AU[i][j];
  const double H = chi * trR + (2.0 / 3.0) * K * K - AA;
  if (H_out) *H_out = H;

#define ADV(F) (beta[0] * D1(F, 0) + beta[1] * D1(F, 1) + beta[2] * D1(F, 2))
  const double sqc = sqrt(chi);
  out[ALPHA] = P->lam[0] * ADV(ALPHA) - 2.0 * al * K -
               sqc * P->ssl_h * (al - sqc) *
                   exp(-0.5 * P->t * P->t / (P->ssl_sigma * P->ssl_sigma));
  for (int i = 0; i < 3; ++i)
    out[BETA + i] = 0.75 * (P->lamf[0] + P->lamf[1] * al) * Bv[i] + P->lam[1] * ADV(BETA + i);
  for (int p = 0; p < 6; ++p) {
    const int i = SYM_I[p], j = SYM_J[p];
    double v = ADV(GT + p);
    for (int k = 0; k < 3; ++k) v += g[i][k] * D1(BETA + k, j) + g[j][k] * D1(BETA + k, i);
    out[GT + p] = v - (2.0 / 3.0) * g[i][j] * divb - 2.0 * al * A[i][j];
  }
  out[CHI] = ADV(CHI) + (2.0 / 3.0) * chi * (al * K - divb) +
             P->cahd_c * P->dx * P->dx * chi * H / (P->dt * (10.0 * P->dx * P->dx + 1.0));
  for (int p = 0; p < 6; ++p) {
    const int i = SYM_I[p], j = SYM_J[p];
    double v = ADV(AT + p);
    for (int k = 0; k < 3; ++k) v += A[i][k] * D1(BETA + k, j) + A[j][k] * D1(BETA + k, i);
    v -= (2.0 / 3.0) * A[i][j] * divb;
    v += chi * (X[i][j] - (1.0 / 3.0) * g[i][j] * trX);
    double AgA = 0.0;
    for (int k = 0; k < 3; ++k)
      for (int l = 0; l < 3; ++l) AgA += A[i][k] * gu[k][l] * A[l][j];
    v += al * (K * A[i][j] - 2.0 * AgA);
    out[AT + p] = v;
  }
  double lapa = 0.0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) lapa += gu[i][j] * DDa[i][j];
  out[KK] = ADV(KK) - chi * lapa + al * (K * K / 3.0 + AA);
  for (int i = 0; i < 3; ++i) {
    double v = ADV(GTI + i);
    for (int j = 0; j < 3; ++j) v -= CalGt[j] * D1(BETA + i, j);
    v += (2.0 / 3.0) * CalGt[i] * divb;
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 3; ++k)
        v += gu[j][k] * D2(BETA + i, j, k) + (1.0 / 3.0) * gu[i][j] * D2(BETA + k, j, k);
    for (int j = 0; j < 3; ++j) v -= 2.0 * AU[i][j] * dal[j];
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 3; ++k) v += 2.0 * al * C2[i][j][k] * AU[j][k];
    for (int j = 0; j < 3; ++j)
      v -= al * ((3.0 / chi) * AU[i][j] * dchi[j] + (4.0 / 3.0) * gu[i][j] * dK[j]);
    out[GTI + i] = v;
    out[BB + i] = v - P->eta * Bv[i] + P->lam[2] * ADV(BB + i) - P->lam[3] * ADV(GTI + i);
  }
#undef ADV
#undef D1
#undef D2
}

/* Pointwise algebra over n points. F [24][n], D [138][n], OUT [24][n]. */
void oracle_rhs_algebra(long n, const double* F, const double* D, const double* S,
                        double* OUT, double* H) {
  const params_t P = unpack(S);
#pragma omp parallel for schedule(static)
  for (long q = 0; q < n; ++q) {
    double f[NF], d[NDERIV], o[NF], h;
    for (int k = 0; k < NF; ++k) f[k] = F[(long)k * n + q];
    for (int k = 0; k < NDERIV; ++k) d[k] = D[(long)k * n + q];
    point_rhs(f, d, &P, o, &h);
    for (int k = 0; k < NF; ++k) OUT[(long)k * n + q] = o[k];
    if (H) H[q] = h;
  }
}

/* Full right-hand side of a (24,Sx,Sy,Sz) state: bundle + algebra. */
void oracle_rhs(const double* F, long Sx, long Sy, long Sz, const double* S,
                double* OUT) {
  const long n = Sx * Sy * Sz;
  double* D = (double*)malloc(sizeof(double) * NDERIV * n);
  oracle_derivatives(F, Sx, Sy, Sz, S[13], S[14], S[15], D);
  oracle_rhs_algebra(n, F, D, S, OUT, NULL);
  free(D);
}

/* Hamiltonian constraint field of a state (same derivatives as the RHS). */
void oracle_hamiltonian(const double* F, long Sx, long Sy, long Sz, double dx,
                        double dy, double dz, double* H) {
  const long n = Sx * Sy * Sz;
  double* D = (double*)malloc(sizeof(double) * NDERIV * n);
  double* OUT = (double*)malloc(sizeof(double) * NF * n);
  double S[16] = {2.0, 0.0, 1.0, dx, 0.0, 1.0, 0.0, 1, 1, 1, 1, 1, 0, dx, dy, dz};
  oracle_derivatives(F, Sx, Sy, Sz, dx, dy, dz, D);
  oracle_rhs_algebra(n, F, D, S, OUT, H);
  free(D);
  free(OUT);
}


/* Hamiltonian and momentum constraints at one point, the definitions of the
 * reference's ConstraintSolver (3D/src/bssn3d/constraints.py:38-62, from
 * Dendro-GR's physcon CSE):
 *   H   = chi R~ + 2/3 K^2 - A~_ij A~^ij      (R~ with the metric-computed G~^k)
 *   M_i = g~^jk (d_j A~_ki - G~^m_ji A~_km) - Gt^j A~_ij
 *         - 3/2 g~^jk A~_ki d_j chi / chi - 2/3 d_i K   (Gt^j the evolved field) */
static void point_constraints(const double* f, const double* d, double* H, double* M) {
  params_t P;
  memset(&P, 0, sizeof(P));
  P.dt = 1.0; P.ssl_sigma = 1.0;
  double out[NF];
  point_rhs(f, d, &P, out, H);
  double g[3][3], A[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      g[i][j] = f[GT + SYM[i][j]];
      A[i][j] = f[AT + SYM[i][j]];
    }
  double adj[3][3];
  adj[0][0] = g[1][1] * g[2][2] - g[1][2] * g[1][2];
  adj[0][1] = g[0][2] * g[1][2] - g[0][1] * g[2][2];
  adj[0][2] = g[0][1] * g[1][2] - g[0][2] * g[1][1];
  adj[1][1] = g[0][0] * g[2][2] - g[0][2] * g[0][2];
  adj[1][2] = g[0][1] * g[0][2] - g[0][0] * g[1][2];
  adj[2][2] = g[0][0] * g[1][1] - g[0][1] * g[0][1];
  adj[1][0] = adj[0][1]; adj[2][0] = adj[0][2]; adj[2][1] = adj[1][2];
  const double det = g[0][0] * adj[0][0] + g[0][1] * adj[0][1] + g[0][2] * adj[0][2];
  double gu[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) gu[i][j] = adj[i][j] / det;
#define D1C(F, A) d[3 * (F) + (A)]
  double C1[3][3][3], C2[3][3][3];
  for (int k = 0; k < 3; ++k)
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        C1[k][i][j] = 0.5 * (D1C(GT + SYM[k][j], i) + D1C(GT + SYM[k][i], j) - D1C(GT + SYM[i][j], k));
  for (int k = 0; k < 3; ++k)
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        double s = 0.0;
        for (int l = 0; l < 3; ++l) s += gu[k][l] * C1[l][i][j];
        C2[k][i][j] = s;
      }
  const double chi = f[CHI];
  for (int i = 0; i < 3; ++i) {
    double m = 0.0;
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 3; ++k) {
        double s = D1C(AT + SYM[k][i], j);
        for (int mm = 0; mm < 3; ++mm) s -= C2[mm][j][i] * A[k][mm];
        m += gu[j][k] * s;
      }
    for (int j = 0; j < 3; ++j) m -= f[GTI + j] * A[i][j];
    double c = 0.0;
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 3; ++k) c += gu[j][k] * A[k][i] * D1C(CHI, j) / chi;
    m -= 1.5 * c;
    m -= (2.0 / 3.0) * D1C(KK, i);
    M[i] = m;
  }
#undef D1C
}

/* Constraint fields of a state: H [n], M [3][n]. */
void oracle_constraints(const double* F, long Sx, long Sy, long Sz, double dx, double dy,
                        double dz, double* H, double* M) {
  const long n = Sx * Sy * Sz;
  double* D = (double*)malloc(sizeof(double) * NDERIV * n);
  oracle_derivatives(F, Sx, Sy, Sz, dx, dy, dz, D);
#pragma omp parallel for schedule(static)
  for (long q = 0; q < n; ++q) {
    double f[NF], d[NDERIV], h, m[3];
    for (int k = 0; k < NF; ++k) f[k] = F[(long)k * n + q];
    for (int k = 0; k < NDERIV; ++k) d[k] = D[(long)k * n + q];
    point_constraints(f, d, &h, m);
    H[q] = h;
    for (int i = 0; i < 3; ++i) M[(long)i * n + q] = m[i];
  }
  free(D);
}

/* Pointwise constraints from supplied derivatives (for pinning against the
 * reference's compiled physcon block). */
void oracle_constraints_algebra(long n, const double* F, const double* D, double* H, double* M) {
#pragma omp parallel for schedule(static)
  for (long q = 0; q < n; ++q) {
    double f[NF], d[NDERIV], h, m[3];
    for (int k = 0; k < NF; ++k) f[k] = F[(long)k * n + q];
    for (int k = 0; k < NDERIV; ++k) d[k] = D[(long)k * n + q];
    point_constraints(f, d, &h, m);
    H[q] = h;
    for (int i = 0; i < 3; ++i) M[(long)i * n + q] = m[i];
  }
}

/* ------------------------------------------------------------------ */
/* time integration                                                    */
/* ------------------------------------------------------------------ */

/* Algebraic enforcement in place (evolve.py:93-119). */
void oracle_enforce(double* F, long n, double chi_floor, double alpha_floor) {
#pragma omp parallel for schedule(static)
  for (long q = 0; q < n; ++q) {
    double g[6], a[6];
    for (int k = 0; k < 6; ++k) {
      g[k] = F[(long)(GT + k) * n + q];
      a[k] = F[(long)(AT + k) * n + q];
    }
    const double det = g[0] * (g[3] * g[5] - g[4] * g[4]) - g[1] * (g[1] * g[5] - g[4] * g[2]) +
                       g[2] * (g[1] * g[4] - g[3] * g[2]);
    const double scale = pow(det, -1.0 / 3.0);
    for (int k = 0; k < 6; ++k) g[k] = g[k] * scale;
    const double iuxx = g[3] * g[5] - g[4] * g[4];
    const double iuxy = g[2] * g[4] - g[1] * g[5];
    const double iuxz = g[1] * g[4] - g[2] * g[3];
    const double iuyy = g[0] * g[5] - g[2] * g[2];
    const double iuyz = g[1] * g[2] - g[0] * g[4];
    const double iuzz = g[0] * g[3] - g[1] * g[1];
    const double trA = iuxx * a[0] + iuyy * a[3] + iuzz * a[5] +
                       2.0 * (iuxy * a[1] + iuxz * a[2] + iuyz * a[4]);
    const double third = trA / 3.0;
    for (int k = 0; k < 6; ++k) {
      F[(long)(GT + k) * n + q] = g[k];
      F[(long)(AT + k) * n + q] = a[k] - g[k] * third;
    }
    double c = F[(long)CHI * n + q], al = F[(long)ALPHA * n + q];
    F[(long)CHI * n + q] = c > chi_floor ? c : (c < chi_floor ? chi_floor : c);
    F[(long)ALPHA * n + q] = al > alpha_floor ? al : (al < alpha_floor ? alpha_floor : al);
  }
}

/* Periodic ghost sync in place (evolve.py:65-73), axis by axis. */
void oracle_periodic_sync(double* F, long Sx, long Sy, long Sz, int ng) {
  const long S[3] = {Sx, Sy, Sz};
  const long stride[3] = {Sy * Sz, Sz, 1};
  const long n = Sx * Sy * Sz;
  for (int axis = 0; axis < 3; ++axis)
    for (int f = 0; f < NF; ++f) {
      double* u = F + (long)f * n;
      for (long x = 0; x < Sx; ++x)
        for (long y = 0; y < Sy; ++y)
          for (long z = 0; z < Sz; ++z) {
            const long p[3] = {x, y, z};
            const long c = p[axis];
            long src = -1;
            if (c < ng) src = c + S[axis] - 2 * ng;
            else if (c >= S[axis] - ng) src = c - S[axis] + 2 * ng;
            if (src < 0) continue;
            const long base = x * stride[0] + y * stride[1] + z - c * stride[axis];
            u[base + c * stride[axis]] = u[base + src * stride[axis]];
          }
    }
}

/* rate = RHS(state) + KO(state), with optional periodic sync of the stage
 * input first (evolve.py:86-91). */
static void stage_rate(const double* U, long Sx, long Sy, long Sz, const double* S,
                       double ko_sigma, int ko_order, int periodic, int ng,
                       double* rate, double* work) {
  const long n = Sx * Sy * Sz;
  const double* src = U;
  if (periodic) {
    memcpy(work, U, sizeof(double) * NF * n);
    oracle_periodic_sync(work, Sx, Sy, Sz, ng);
    src = work;
  }
  oracle_rhs(src, Sx, Sy, Sz, S, rate);
  if (ko_sigma > 0.0) {
    double* ko = (double*)malloc(sizeof(double) * NF * n);
    oracle_ko(src, Sx, Sy, Sz, S[13], S[14], S[15], ko_sigma, ko_order, ko);
    for (long q = 0; q < NF * n; ++q) rate[q] = rate[q] + ko[q];
    free(ko);
  }
}

/* One RK4 step of BSSNEvolution.step (evolve.py:125-137) + enforce.
 * S carries dt (S[2]) and the step's start time t (S[6]); each stage uses its
 * own time and the full dt. U_out may alias nothing. */
void oracle_rk4_step(const double* U, long Sx, long Sy, long Sz, const double* S_in,
                     double ko_sigma, int ko_order, int periodic, int ng,
                     double chi_floor, double alpha_floor, double* U_out) {
  const long n = Sx * Sy * Sz;
  const long N = NF * n;
  double S[16];
  memcpy(S, S_in, sizeof(S));
  const double dt = S[2], t = S[6];
  double* k[4];
  for (int i = 0; i < 4; ++i) k[i] = (double*)malloc(sizeof(double) * N);
  double* Y = (double*)malloc(sizeof(double) * N);
  double* work = (double*)malloc(sizeof(double) * N);
  const double c[4] = {0.0, 0.5, 0.5, 1.0};
  for (int s = 0; s < 4; ++s) {
    const double* in = U;
    if (s > 0) {
      const double h = (s == 3 ? 1.0 : 0.5) * dt;
      for (long q = 0; q < N; ++q) Y[q] = U[q] + h * k[s - 1][q];
      in = Y;
    }
    S[6] = t + c[s] * dt;
    stage_rate(in, Sx, Sy, Sz, S, ko_sigma, ko_order, periodic, ng, k[s], work);
  }
  const double w = dt / 6.0;
  for (long q = 0; q < N; ++q)
    U_out[q] = U[q] + w * (k[0][q] + 2.0 * k[1][q] + 2.0 * k[2][q] + k[3][q]);
  oracle_enforce(U_out, n, chi_floor, alpha_floor);
  for (int i = 0; i < 4; ++i) free(k[i]);
  free(Y);
  free(work);
}

/* rate = RHS + KO at the stage time S[6] (the evaluation BSSNEvolution.rhs
 * makes, evolve.py:86-91). */
void oracle_rate(const double* U, long Sx, long Sy, long Sz, const double* S,
                 double ko_sigma, int ko_order, int periodic, int ng, double* rate) {
  double* work = (double*)malloc(sizeof(double) * NF * Sx * Sy * Sz);
  stage_rate(U, Sx, Sy, Sz, S, ko_sigma, ko_order, periodic, ng, rate, work);
  free(work);
}

/* One 2-step / 3-stage MSRK step of BSSNEvolution._msrk2_step
 * (evolve.py:139-153) + enforce. coef = {a20, a21, a30, a31, a32, b0, b1, b2, b3}.
 * Kprev = f(y_{n-1}) (stage 0 of the method, reused); K_out receives
 * k1 = f(y_n), the next step's Kprev. Nodes c2 = a20 + a21 and
 * c3 = a30 + a31 + a32 give the stage times; dt is the full step throughout. */
void oracle_msrk2_step(const double* U, const double* Kprev, long Sx, long Sy, long Sz,
                       const double* S_in, const double* coef, double ko_sigma, int ko_order,
                       int periodic, int ng, double chi_floor, double alpha_floor,
                       double* U_out, double* K_out) {
  const long n = Sx * Sy * Sz;
  const long N = NF * n;
  double S[16];
  memcpy(S, S_in, sizeof(S));
  const double dt = S[2], t = S[6];
  const double a20 = coef[0], a21 = coef[1], a30 = coef[2], a31 = coef[3], a32 = coef[4];
  const double* b = coef + 5;
  double* k1 = (double*)malloc(sizeof(double) * N);
  double* k2 = (double*)malloc(sizeof(double) * N);
  double* k3 = (double*)malloc(sizeof(double) * N);
  double* Y = (double*)malloc(sizeof(double) * N);
  double* work = (double*)malloc(sizeof(double) * N);
  const double* k0 = Kprev;
  S[6] = t;
  stage_rate(U, Sx, Sy, Sz, S, ko_sigma, ko_order, periodic, ng, k1, work);
  for (long q = 0; q < N; ++q) Y[q] = U[q] + dt * (a20 * k0[q] + a21 * k1[q]);
  S[6] = t + (a20 + a21) * dt;
  stage_rate(Y, Sx, Sy, Sz, S, ko_sigma, ko_order, periodic, ng, k2, work);
  for (long q = 0; q < N; ++q) Y[q] = U[q] + dt * (a30 * k0[q] + a31 * k1[q] + a32 * k2[q]);
  S[6] = t + (a30 + a31 + a32) * dt;
  stage_rate(Y, Sx, Sy, Sz, S, ko_sigma, ko_order, periodic, ng, k3, work);
  for (long q = 0; q < N; ++q)
    U_out[q] = U[q] + dt * (b[0] * k0[q] + b[1] * k1[q] + b[2] * k2[q] + b[3] * k3[q]);
  oracle_enforce(U_out, n, chi_floor, alpha_floor);
  memcpy(K_out, k1, sizeof(double) * N);
  free(k1);
  free(k2);
  free(k3);
  free(Y);
  free(work);
}

// ORACLE -- test infrastructure only.
//
// CPU restatement of HelioCubed's second-order (PLM) per-box MHD update and
// the RK4 stage update that consumes it.  Used only by tests/, by
// __graft_entry__.smoke() and by bench.py's CPU-baseline arm, always as the
// checker or the timed CPU baseline; the product library never links it.
//
// Parity status:
//   * Riemann solvers, the O2 face frame and face flux are pinned against the
//     reference's own headers compiled from source (oracle/ref_pin.cpp ->
//     oracle/_ref/libhcref.so, tests/test_oracle_pin.py).
//   * Cubed-sphere metrics (Proto CubedSphereShell::detA / detA_A / adjA /
//     f_Amatrix), Proto's stencil FluxDivergence, the MBLevelRK4 loop and the
//     MBInterpOp seam weights live in the unvendored Proto library: parity is
//     UNPINNED for those pieces.  They are restated here from the mathematics
//     (exact face/cell averages of the equiangular gnomonic map) and checked
//     against analytic invariants in tests/.
//
// Everything is FP64 (long double only for the metric integrals), compiled
// with -ffp-contract=off so the arithmetic order below is the one executed.

#include <algorithm>
#include <array>
#include <cmath>
#include <limits>
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <vector>

#include "../include/hc_abi.h"

namespace {

constexpr int NC = 8;
// src/MHD_Constants.H:4-7 and src/BoxOp_EulerCubedSphere.H:36
constexpr double c_MP = 1.67262192e-24;
constexpr double RHO00 = 1.67262192e-24 / 100.;
constexpr double c_G = 6.67430e-8;
constexpr double c_M0 = 1.98847e33;
enum { iRHO = 0, iVX = 1, iE = 4, iP = 4, iBX = 5 };

typedef long double LD;
const LD PI_L = 3.14159265358979323846264338327950288L;

// Panel permutation / sign tables, src/BoxOp_Utilities.H:413-416.  Global
// Cartesian component k of a panel-local vector q is SIGN[b][k]*q[PERM[b][k]]
// (this reading makes the six panels the six distinct cube faces).
const int PERM[6][3] = {{1, 2, 0}, {1, 2, 0}, {1, 0, 2}, {0, 1, 2}, {1, 0, 2}, {0, 1, 2}};
const int SIGN[6][3] = {{1, -1, -1}, {1, 1, 1}, {1, -1, 1}, {1, 1, 1}, {-1, 1, 1}, {-1, -1, 1}};

// ---------------------------------------------------------------------------
// Geometry.  Equiangular gnomonic map: alpha = -pi/4 + (pi/2) xi1,
// beta = -pi/4 + (pi/2) xi2 (src/MHD_StateConversion.H:294-297).  The basis
// A has columns (Xhat, dXhat/dxi1, dXhat/dxi2); the face normal of direction
// d is the cofactor row col_{d+1} x col_{d+2}, as in the frame of
// src/MHD_Roe8Wave.H:643-650.
// ---------------------------------------------------------------------------
void localPoint(LD x1, LD x2, LD q[3], LD* pa = nullptr, LD* pc = nullptr) {
  LD a = tanl(-PI_L / 4 + PI_L / 2 * x1), c = tanl(-PI_L / 4 + PI_L / 2 * x2);
  LD rho = sqrtl(1 + a * a + c * c);
  q[0] = 1 / rho; q[1] = a / rho; q[2] = c / rho;
  if (pa) *pa = a;
  if (pc) *pc = c;
}

void unitPoint(int b, LD x1, LD x2, LD X[3]) {
  LD q[3];
  localPoint(x1, x2, q);
  for (int k = 0; k < 3; ++k) X[k] = SIGN[b][k] * q[PERM[b][k]];
}

void basisL(int b, LD x1, LD x2, LD A[3][3]) {
  LD q[3], a, c;
  localPoint(x1, x2, q, &a, &c);
  LD rho = 1 / q[0], r3 = rho * rho * rho;
  LD da = PI_L / 2 * (1 + a * a), dc = PI_L / 2 * (1 + c * c);
  LD q1[3] = {-a / r3 * da, (1 / rho - a * a / r3) * da, (-a * c / r3) * da};
  LD q2[3] = {-c / r3 * dc, (-a * c / r3) * dc, (1 / rho - c * c / r3) * dc};
  for (int k = 0; k < 3; ++k) {
    A[k][0] = SIGN[b][k] * q[PERM[b][k]];
    A[k][1] = SIGN[b][k] * q1[PERM[b][k]];
    A[k][2] = SIGN[b][k] * q2[PERM[b][k]];
  }
}

void crossL(const LD u[3], const LD v[3], LD w[3]) {
  w[0] = u[1] * v[2] - u[2] * v[1];
  w[1] = u[2] * v[0] - u[0] * v[2];
  w[2] = u[0] * v[1] - u[1] * v[0];
}

// Gauss-Legendre nodes/weights on [0,1].
struct GL {
  int n;
  LD x[16], w[16];
  explicit GL(int m) : n(m) {
    for (int i = 0; i < m; ++i) {
      LD z = cosl(PI_L * (i + 0.75L) / (m + 0.5L)), pp = 0;
      for (int it = 0; it < 100; ++it) {
        LD p1 = 1, p2 = 0;
        for (int j = 1; j <= m; ++j) {
          LD p3 = p2; p2 = p1;
          p1 = ((2 * j - 1) * z * p2 - (j - 1) * p3) / j;
        }
        pp = m * (z * p1 - p2) / (z * z - 1);
        LD dz = p1 / pp;
        z -= dz;
        if (fabsl(dz) < 1e-19L) break;
      }
      x[i] = (1 - z) / 2;
      w[i] = 1 / ((1 - z * z) * pp * pp);
    }
  }
};
const GL& gl() { static GL g(12); return g; }

// Cell average over [j h,(j+1)h] x [k h,(k+1)h] of det(A) and det(A)*A.
void cellAverages(int b, int j, int k, LD h, LD& det, LD dA[3][3]) {
  const GL& g = gl();
  det = 0;
  for (int r = 0; r < 3; ++r) for (int s = 0; s < 3; ++s) dA[r][s] = 0;
  for (int p = 0; p < g.n; ++p)
    for (int q = 0; q < g.n; ++q) {
      LD A[3][3];
      basisL(b, (j + g.x[p]) * h, (k + g.x[q]) * h, A);
      LD c1[3] = {A[0][1], A[1][1], A[2][1]}, c2[3] = {A[0][2], A[1][2], A[2][2]}, n[3];
      crossL(c1, c2, n);
      LD d = A[0][0] * n[0] + A[1][0] * n[1] + A[2][0] * n[2];
      LD wt = g.w[p] * g.w[q];
      det += wt * d;
      for (int r = 0; r < 3; ++r) for (int s = 0; s < 3; ++s) dA[r][s] += wt * d * A[r][s];
    }
}

// Face-averaged normal adjA of direction d at the low face of cell (j,k).
// d=0 uses the cell average of col1 x col2; d=1,2 the closed form of the
// integral along a great-circle arc, int Xhat x dXhat = theta * unit(P x Q).
void faceNormal(int b, int d, int j, int k, LD h, LD n[3]) {
  if (d == 0) {
    const GL& g = gl();
    n[0] = n[1] = n[2] = 0;
    for (int p = 0; p < g.n; ++p)
      for (int q = 0; q < g.n; ++q) {
        LD A[3][3], c1[3], c2[3], m[3];
        basisL(b, (j + g.x[p]) * h, (k + g.x[q]) * h, A);
        for (int r = 0; r < 3; ++r) { c1[r] = A[r][1]; c2[r] = A[r][2]; }
        crossL(c1, c2, m);
        for (int r = 0; r < 3; ++r) n[r] += g.w[p] * g.w[q] * m[r];
      }
    return;
  }
  LD P[3], Q[3], c[3];
  if (d == 1) { unitPoint(b, j * h, k * h, P); unitPoint(b, j * h, (k + 1) * h, Q); }
  else        { unitPoint(b, j * h, k * h, P); unitPoint(b, (j + 1) * h, k * h, Q); }
  crossL(P, Q, c);
  LD s = sqrtl(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
  LD theta = atan2l(s, P[0] * Q[0] + P[1] * Q[1] + P[2] * Q[2]);
  LD f = (d == 1 ? -theta : theta) / (s * h);
  for (int r = 0; r < 3; ++r) n[r] = f * c[r];
}

// Face-averaged det(A) on the low face of direction d (d=0: cell average).
LD faceDet(int b, int d, int j, int k, LD h) {
  if (d == 0) { LD det, dA[3][3]; cellAverages(b, j, k, h, det, dA); return det; }
  LD q[3], a0, c0, a1, c1;
  if (d == 1) {
    localPoint(j * h, k * h, q, &a0, &c0);
    localPoint(j * h, (k + 1) * h, q, &a1, &c1);
    return PI_L / 2 / h * (c1 / sqrtl(1 + a0 * a0 + c1 * c1) - c0 / sqrtl(1 + a0 * a0 + c0 * c0));
  }
  localPoint(j * h, k * h, q, &a0, &c0);
  localPoint((j + 1) * h, k * h, q, &a1, &c1);
  return PI_L / 2 / h * (a1 / sqrtl(1 + a1 * a1 + c0 * c0) - a0 / sqrtl(1 + a0 * a0 + c0 * c0));
}

// Pointwise basis at cell centre (centering -1) or at the low face of d.
void pointBasis(int b, int centering, int j, int k, LD h, double A[3][3]) {
  LD oa = 0.5L, ob = 0.5L;
  if (centering == 1) oa = 0;
  if (centering == 2) ob = 0;
  LD L[3][3];
  basisL(b, (j + oa) * h, (k + ob) * h, L);
  for (int r = 0; r < 3; ++r) for (int s = 0; s < 3; ++s) A[r][s] = (double)L[r][s];
}

// 3x3 inverse by cofactors (Proto f_matinv3by3 is unvendored).
void inverse3(const double A[3][3], double inv[3][3]) {
  double c00 = A[1][1] * A[2][2] - A[1][2] * A[2][1];
  double c01 = A[1][2] * A[2][0] - A[1][0] * A[2][2];
  double c02 = A[1][0] * A[2][1] - A[1][1] * A[2][0];
  double det = A[0][0] * c00 + A[0][1] * c01 + A[0][2] * c02;
  double id = 1.0 / det;
  inv[0][0] = c00 * id;
  inv[1][0] = c01 * id;
  inv[2][0] = c02 * id;
  inv[0][1] = (A[0][2] * A[2][1] - A[0][1] * A[2][2]) * id;
  inv[1][1] = (A[0][0] * A[2][2] - A[0][2] * A[2][0]) * id;
  inv[2][1] = (A[0][1] * A[2][0] - A[0][0] * A[2][1]) * id;
  inv[0][2] = (A[0][1] * A[1][2] - A[0][2] * A[1][1]) * id;
  inv[1][2] = (A[0][2] * A[1][0] - A[0][0] * A[1][2]) * id;
  inv[2][2] = (A[0][0] * A[1][1] - A[0][1] * A[1][0]) * id;
}

// Radial cells of the whole shell; a level with radial_cells > 0 is the slab
// [radial_offset, radial_offset + nr) of that shell.
int shellCells(const hc_params& P) { return P.radial_cells > 0 ? P.radial_cells : P.nr; }

// Radial metrics, restated from src/BoxOp_Utilities.H:36-59 (double, libm),
// of the level's radial cell iLocal (the shell's cell iLocal + radial_offset).
struct Radial { double rad, vol, Dr0, area0, areaT, rlow, rhigh; };
Radial radialMetric(const hc_params& P, int iLocal) {
  const double r0 = P.inner_radius, r1 = P.outer_radius, C = P.radial_stretch;
  const int i = iLocal + P.radial_offset;
  const double dxi0 = 1.0 / shellCells(P);
  double R_t = C == 0.0 ? (r1 - r0) : (r1 - r0) / std::expm1(C);
  double etalow = i * dxi0;
  double rlow = r0 + R_t * (C == 0.0 ? etalow : std::expm1(C * etalow));
  double etahigh = (i + 1.0) * dxi0;
  double rhigh = r0 + R_t * (C == 0.0 ? etahigh : std::expm1(C * etahigh));
  double eta_half = (etalow + etahigh) / 2.0;
  double rhalf = r0 + R_t * (C == 0.0 ? eta_half : std::expm1(C * eta_half));
  Radial r;
  r.rad = rhalf;
  r.vol = (rhigh * rhigh * rhigh - rlow * rlow * rlow) / 3.0 / dxi0;
  r.Dr0 = (rhigh - rlow) / dxi0;
  r.area0 = rlow * rlow;
  r.areaT = (rhigh * rhigh - rlow * rlow) / dxi0 / 2.0;
  r.rlow = rlow;
  r.rhigh = rhigh;
  return r;
}

// ---------------------------------------------------------------------------
// Pointwise physics, restated from the reference headers.
// ---------------------------------------------------------------------------

// src/BoxOp_SecondOrder.H:7-37
void plmFace(const double* mm, const double* m, const double* c, const double* p,
             int limiter, double lo[8], double hi[8]) {
  for (int k = 0; k < NC; ++k) {
    double a = m[k] - mm[k], b = c[k] - m[k], d = p[k] - c[k];
    double sl = 0.5 * (a + b), sr = 0.5 * (b + d);
    if (limiter != 0) {
      sl = a * b <= 0 ? 0.0 : (a > 0 ? std::min(a, b) : std::max(a, b));
      sr = b * d <= 0 ? 0.0 : (b > 0 ? std::min(b, d) : std::max(b, d));
      if (limiter == 3) {
        if (a * b > 0) sl = (a > 0 ? 1.0 : -1.0) * std::min(0.5 * std::fabs(a + b), 2.0 * std::min(std::fabs(a), std::fabs(b)));
        if (b * d > 0) sr = (b > 0 ? 1.0 : -1.0) * std::min(0.5 * std::fabs(b + d), 2.0 * std::min(std::fabs(b), std::fabs(d)));
      }
    }
    lo[k] = m[k] + 0.5 * sl;
    hi[k] = c[k] - 0.5 * sr;
  }
  if (!(lo[iRHO] >= RHO00 && lo[iP] >= 0)) for (int k = 0; k < NC; ++k) lo[k] = m[k];
  if (!(hi[iRHO] >= RHO00 && hi[iP] >= 0)) for (int k = 0; k < NC; ++k) hi[k] = c[k];
}

struct Frame { double f[3][3], norm, normal[3]; };

// Exact symmetric values of a face normal: components below 1e-13 of the
// largest are zero and pairs equal in magnitude to 1e-13 take their common
// mean magnitude, so that the least-aligned-axis choice below is the one
// exact arithmetic makes on the cube's symmetry lines.
void symmetricNormal(double n[3]) {
  double mag = std::max(std::fabs(n[0]), std::max(std::fabs(n[1]), std::fabs(n[2])));
  double tol = 1e-13 * mag;
  for (int i = 0; i < 3; ++i) if (std::fabs(n[i]) < tol) n[i] = 0.0;
  for (int a = 0; a < 3; ++a)
    for (int b = a + 1; b < 3; ++b)
      if (n[a] != 0.0 && std::fabs(std::fabs(n[a]) - std::fabs(n[b])) <= tol) {
        double m = 0.5 * (std::fabs(n[a]) + std::fabs(n[b]));
        n[a] = std::copysign(m, n[a]);
        n[b] = std::copysign(m, n[b]);
      }
}

// src/MHD_SecondOrderFlux.H:11-30
Frame secondOrderFrame(const double normal[3]) {
  Frame r{};
  for (int i = 0; i < 3; ++i) r.norm += normal[i] * normal[i];
  r.norm = std::sqrt(r.norm);
  for (int i = 0; i < 3; ++i) r.f[0][i] = normal[i] / r.norm;
  int axis = 0;
  for (int i = 1; i < 3; ++i) if (std::fabs(r.f[0][i]) < std::fabs(r.f[0][axis])) axis = i;
  r.f[1][(axis + 1) % 3] = r.f[0][(axis + 2) % 3];
  r.f[1][(axis + 2) % 3] = -r.f[0][(axis + 1) % 3];
  double t = 0;
  for (int i = 0; i < 3; ++i) t += r.f[1][i] * r.f[1][i];
  for (int i = 0; i < 3; ++i) r.f[1][i] /= std::sqrt(t);
  for (int i = 0; i < 3; ++i) {
    int j = (i + 1) % 3, k = (i + 2) % 3;
    r.f[2][i] = r.f[0][j] * r.f[1][k] - r.f[0][k] * r.f[1][j];
  }
  for (int d = 0; d < 3; ++d) r.normal[d] = normal[d];
  return r;
}

// src/MHD_Roe8Wave.H:16-600, arithmetic averages (iAveraging = 0), eight-wave
// entropy fix, optional intermediate-state fan walk.  Matrix entries keep the
// reference's expressions; rows/columns are held in arrays.
bool roe8(double out[8], const double* wl, const double* wr, double gamma, double entropy, bool check) {
  const double RhoL = wl[0], UL = wl[1], VL = wl[2], WL = wl[3], PGasL = wl[4], BXL = wl[5], BYL = wl[6], BZL = wl[7];
  const double RhoR = wr[0], UR = wr[1], VR = wr[2], WR = wr[3], PGasR = wr[4], BXR = wr[5], BYR = wr[6], BZR = wr[7];
  if (!(RhoL > 0.0 && RhoR > 0.0 && PGasL > 0.0 && PGasR > 0.0)) return false;
  const double d_1_8PI = 0.039788735772973833942220940843128591, half = 0.5, one = 1.0, zero = 0.0, two = 2.0, four = 4.0;
  const double d_SQRT_2 = 0.707106781186547524400844362104849039, d_1_4PI = 0.079577471545947667884441881686257181;
  const double smallB = 1.0e-9, d_PI = 3.14159265358979323846264338327950288, d_2PI = 6.28318530717958647692528676655900576;
  const double del2 = entropy, hgamma = gamma - 1.0;
  double RUL = RhoL * UL, RVL = RhoL * VL, RWL = RhoL * WL;
  double BxBL = d_1_8PI * (BXL * BXL + BYL * BYL + BZL * BZL);
  double RUxUL = half * (RUL * UL + RVL * VL + RWL * WL);
  double PL = PGasL + BxBL, EL = PGasL / hgamma + RUxUL + BxBL, AL2 = gamma * PGasL / RhoL;
  double RUR = RhoR * UR, RVR = RhoR * VR, RWR = RhoR * WR;
  double BxBR = d_1_8PI * (BXR * BXR + BYR * BYR + BZR * BZR);
  double RUxUR = half * (RUR * UR + RVR * VR + RWR * WR);
  double PR = PGasR + BxBR, ER = PGasR / hgamma + RUxUR + BxBR, AR2 = gamma * PGasR / RhoR;
  double ccmi, ccma;
  if (AL2 > AR2) { ccmi = AR2; ccma = AL2; } else { ccmi = AL2; ccma = AR2; }
  double Rho = half * (RhoL + RhoR), U = half * (UL + UR), V = half * (VL + VR), W = half * (WL + WR);
  double BX = half * (BXL + BXR), BY = half * (BYL + BYR), BZ = half * (BZL + BZR), P = half * (PL + PR);
  double BX2 = BX * BX, BY2 = BY * BY, BZ2 = BZ * BZ, BYZ2 = BY2 + BZ2, BxBH = d_1_8PI * (BX2 + BYZ2);
  double kk = half * (U * U + V * V + W * W);
  double PGas = P - BxBH, cc = gamma * PGas / Rho;
  double bb = d_1_4PI * BX2 / Rho, b = std::sqrt(bb);
  if (cc < ccmi) cc = ccmi;
  if (cc > ccma) cc = ccma;
  if (!(cc > 0.0) || !std::isfinite(cc)) return false;
  double c = std::sqrt(cc);
  double hyy, hzz, aaf, aas, af, as;
  if (BYZ2 < smallB * smallB) {
    hyy = d_SQRT_2; hzz = d_SQRT_2;
    if (bb > cc) { aaf = bb; aas = cc; af = b; as = c; }
    else { aaf = cc; aas = bb; af = c; as = b; }
  } else {
    double hyz = std::sqrt(BYZ2);
    hyy = BY / hyz; hzz = BZ / hyz;
    double szb = cc + (BxBH + BxBH) / Rho;
    double h = std::sqrt(std::fmax(0.0, szb * szb - four * cc * bb));
    aas = half * (szb - h);
    if (aas <= zero) { aas = zero; as = zero; }
    else if (aas >= cc) { aas = cc; as = c; }
    else as = std::sqrt(aas);
    aaf = half * (szb + h);
    if (aaf <= cc) { aaf = cc; af = c; } else af = std::sqrt(aaf);
  }
  const double eig[8] = {U, U, U + b, U - b, U + af, U - af, U + as, U - as};
  double eigmax = std::fabs(U) + std::fabs(V) + std::fabs(W) + af;
  double del = del2 * eigmax, dell2 = del * del, Aeig[8];
  for (int q = 0; q < 8; ++q) {
    double z = std::fabs(eig[q]);
    Aeig[q] = z >= del ? z : half * (z * z + dell2) / del;
  }
  double dfs = aaf - aas, alf, als;
  if (dfs < 1.0e-8) { alf = one; als = zero; }
  else if ((cc - aas) <= zero) { alf = zero; als = one; }
  else if ((aaf - cc) <= zero) { alf = one; als = zero; }
  else { alf = std::sqrt((cc - aas) / dfs); als = std::sqrt((aaf - cc) / dfs); }
  double sih = -one;
  if (BX >= zero) sih = one;
  double du[8] = {RhoL - RhoR, RUL - RUR, RVL - RVR, RWL - RWR, EL - ER, BXL - BXR, BYL - BYR, BZL - BZR};
  du[4] = -hgamma * (-kk * du[0] + U * du[1] + V * du[2] + W * du[3] - du[4] + (BX * du[5] + BY * du[6] + BZ * du[7]) * d_1_4PI);
  du[1] = (-U * du[0] + du[1]) / Rho;
  du[2] = (-V * du[0] + du[2]) / Rho;
  du[3] = (-W * du[0] + du[3]) / Rho;
  double sqPiRho = std::sqrt(d_PI * Rho), sq2PiRho = std::sqrt(d_2PI * Rho);
  // sp[row][col] (right eigenvectors as columns), so[row][col] (left rows).
  double sp[8][8] = {
      {one, zero, zero, zero, Rho * alf, Rho * alf, Rho * als, Rho * als},
      {zero, zero, zero, zero, alf * af, -alf * af, als * as, -als * as},
      {zero, zero, -hzz * d_SQRT_2, -hzz * d_SQRT_2, -als * as * hyy * sih, als * as * hyy * sih, alf * af * hyy * sih, -alf * af * hyy * sih},
      {zero, zero, hyy * d_SQRT_2, hyy * d_SQRT_2, -als * as * hzz * sih, als * as * hzz * sih, alf * af * hzz * sih, -alf * af * hzz * sih},
      {zero, zero, zero, zero, alf * Rho * cc, alf * Rho * cc, als * Rho * cc, als * Rho * cc},
      {zero, one, zero, zero, zero, zero, zero, zero},
      {zero, zero, hzz * sq2PiRho * sih, -hzz * sq2PiRho * sih, two * als * sqPiRho * c * hyy, two * als * sqPiRho * c * hyy, -two * alf * sqPiRho * c * hyy, -two * alf * sqPiRho * c * hyy},
      {zero, zero, -hyy * sq2PiRho * sih, hyy * sq2PiRho * sih, two * als * sqPiRho * c * hzz, two * als * sqPiRho * c * hzz, -two * alf * sqPiRho * c * hzz, -two * alf * sqPiRho * c * hzz}};
  double so[8][8] = {
      {one, zero, zero, zero, -one / cc, zero, zero, zero},
      {zero, zero, zero, zero, zero, one, zero, zero},
      {zero, zero, -hzz * d_SQRT_2, hyy * d_SQRT_2, zero, zero, half * hzz * sih / sq2PiRho, -half * hyy * sih / sq2PiRho},
      {zero, zero, -hzz * d_SQRT_2, hyy * d_SQRT_2, zero, zero, -half * hzz * sih / sq2PiRho, half * hyy * sih / sq2PiRho},
      {zero, half * alf * af / cc, -half * als * as * hyy * sih / cc, -half * als * as * hzz * sih / cc, half * alf / (cc * Rho), zero, 0.25 * als * hyy / (c * sqPiRho), 0.25 * als * hzz / (c * sqPiRho)},
      {zero, -half * alf * af / cc, half * als * as * hyy * sih / cc, half * als * as * hzz * sih / cc, half * alf / (cc * Rho), zero, 0.25 * als * hyy / (c * sqPiRho), 0.25 * als * hzz / (c * sqPiRho)},
      {zero, half * als * as / cc, half * alf * af * hyy * sih / cc, half * alf * af * hzz * sih / cc, half * als / (Rho * cc), zero, -0.25 * alf * hyy / (c * sqPiRho), -0.25 * alf * hzz / (c * sqPiRho)},
      {zero, -half * als * as / cc, -half * alf * af * hyy * sih / cc, -half * alf * af * hzz * sih / cc, half * als / (Rho * cc), zero, -0.25 * alf * hyy / (c * sqPiRho), -0.25 * alf * hzz / (c * sqPiRho)}};
  if (check) {
    const int order[8] = {5, 3, 7, 0, 1, 6, 2, 4};
    double state[8] = {RhoL, RUL, RVL, RWL, EL, BXL, BYL, BZL};
    for (int wave = 0; wave < 7; ++wave) {
      const int k = order[wave];
      double amplitude = 0.0;
      for (int q = 0; q < 8; ++q) amplitude -= so[k][q] * du[q];
      double delta[8];
      for (int q = 0; q < 8; ++q) delta[q] = amplitude * sp[q][k];
      delta[4] = kk * delta[0] + Rho * (U * delta[1] + V * delta[2] + W * delta[3]) + delta[4] / hgamma + d_1_4PI * (BX * delta[5] + BY * delta[6] + BZ * delta[7]);
      delta[1] = U * delta[0] + Rho * delta[1];
      delta[2] = V * delta[0] + Rho * delta[2];
      delta[3] = W * delta[0] + Rho * delta[3];
      for (int q = 0; q < 8; ++q) state[q] += delta[q];
      if (eig[order[wave + 1]] > eig[k]) {
        if (!(state[0] > 0.0) || !std::isfinite(state[0])) return false;
        double thermal = state[4] - 0.5 * (state[1] * state[1] + state[2] * state[2] + state[3] * state[3]) / state[0] - d_1_8PI * (state[5] * state[5] + state[6] * state[6] + state[7] * state[7]);
        if (!(thermal >= 0.0) || !std::isfinite(thermal)) return false;
      }
    }
  }
  double lu[8], ra[8];
  for (int q = 0; q < 8; ++q) {
    double s = so[q][0] * du[0];
    for (int r = 1; r < 8; ++r) s = s + so[q][r] * du[r];
    lu[q] = Aeig[q] * s;
  }
  for (int q = 0; q < 8; ++q) {
    double s = sp[q][0] * lu[0];
    for (int r = 1; r < 8; ++r) s = s + sp[q][r] * lu[r];
    ra[q] = s;
  }
  ra[4] = ra[0] * kk + Rho * (U * ra[1] + V * ra[2] + W * ra[3]) + ra[4] / hgamma + d_1_4PI * (BX * ra[5] + BY * ra[6] + BZ * ra[7]);
  ra[1] = U * ra[0] + Rho * ra[1];
  ra[2] = V * ra[0] + Rho * ra[2];
  ra[3] = W * ra[0] + Rho * ra[3];
  for (int q = 0; q < 8; ++q) out[q] = -ra[q];
  for (int q = 0; q < 8; ++q) if (!std::isfinite(out[q])) return false;
  return true;
}

// src/MHD_Roe8Wave.H:604-629
void rusanov(double out[8], const double* wl, const double* wr, double gamma) {
  const double inv4Pi = 0.079577471545947667884441881686257181;
  double cons[2][8], speed = 0.0;
  for (int side = 0; side < 2; ++side) {
    const double* w = side == 0 ? wl : wr;
    double v2 = 0.0, b2 = 0.0;
    cons[side][0] = w[0];
    for (int d = 0; d < 3; ++d) {
      v2 += w[1 + d] * w[1 + d];
      b2 += w[5 + d] * w[5 + d];
      cons[side][1 + d] = w[0] * w[1 + d];
      cons[side][5 + d] = w[5 + d];
    }
    cons[side][4] = w[4] / (gamma - 1.0) + 0.5 * w[0] * v2 + 0.5 * inv4Pi * b2;
    speed = std::fmax(speed, std::fabs(w[1]) + std::sqrt((gamma * w[4] + inv4Pi * b2) / w[0]));
  }
  for (int c = 0; c < 8; ++c) out[c] = speed * (cons[1][c] - cons[0][c]);
}

// src/MHD_SecondOrderFlux.H:34-74
void faceFlux(double out[8], const double* l, const double* r, const Frame& g, double radialArea,
              double gamma, double entropy, bool roe) {
  const double inv4pi = 1.0 / (4.0 * M_PI);
  double local[2][8] = {}, flux[2][8] = {};
  for (int side = 0; side < 2; ++side) {
    const double* s = side == 0 ? l : r;
    local[side][0] = s[0];
    local[side][4] = s[4];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        local[side][1 + i] += g.f[i][j] * s[1 + j];
        local[side][5 + i] += g.f[i][j] * s[5 + j];
      }
    double* q = local[side];
    double v2 = 0, b2 = 0, vb = 0;
    for (int i = 0; i < 3; ++i) { v2 += q[1 + i] * q[1 + i]; b2 += q[5 + i] * q[5 + i]; vb += q[1 + i] * q[5 + i]; }
    const double pressure = q[4] + 0.5 * inv4pi * b2;
    const double energy = q[4] / (gamma - 1) + 0.5 * q[0] * v2 + 0.5 * inv4pi * b2;
    flux[side][0] = q[0] * q[1];
    flux[side][4] = (energy + pressure) * q[1] - inv4pi * q[5] * vb;
    for (int i = 0; i < 3; ++i) {
      flux[side][1 + i] = q[0] * q[1] * q[1 + i] - inv4pi * q[5] * q[5 + i] + (i == 0 ? pressure : 0);
      flux[side][5 + i] = q[1] * q[5 + i] - q[1 + i] * q[5];
    }
  }
  double diss[8], numerical[8];
  if (!roe || !roe8(diss, local[0], local[1], gamma, entropy, true)) rusanov(diss, local[0], local[1], gamma);
  const double area = radialArea * g.norm;
  for (int c = 0; c < 8; ++c) numerical[c] = 0.5 * area * (flux[0][c] + flux[1][c] - diss[c]);
  out[0] = numerical[0];
  out[4] = numerical[4];
  for (int i = 0; i < 3; ++i) {
    out[1 + i] = out[5 + i] = 0;
    for (int j = 0; j < 3; ++j) { out[1 + i] += g.f[j][i] * numerical[1 + j]; out[5 + i] += g.f[j][i] * numerical[5 + j]; }
  }
}

// src/MHD_StateConversion.H:11-32 (constant-background magnetic tests excluded)
void cartesianPrimitiveFromConserved(double out[8], const double in[8], double inverseJ, double gamma) {
  double u[8];
  for (int c = 0; c < 8; ++c) u[c] = in[c] * inverseJ;
  const double rho = u[0] < c_MP / 100 ? c_MP / 100 : u[0];
  double kinetic = 0, magnetic = 0;
  out[0] = rho;
  for (int d = 0; d < 3; ++d) {
    out[1 + d] = u[1 + d] / rho;
    out[5 + d] = u[5 + d];
    kinetic += 0.5 * rho * out[1 + d] * out[1 + d];
    magnetic += u[5 + d] * u[5 + d] / (8 * M_PI);
  }
  const double pressure = 0.0 + (gamma - 1.0) * (u[4] - kinetic - magnetic);
  out[4] = pressure < 0.0 ? 0.0 : pressure;
}

// ---------------------------------------------------------------------------
// Box storage helpers (Proto BoxData SoA, radial fastest).
// ---------------------------------------------------------------------------
struct BoxIdx {
  int lo[3], n[3];
  size_t N;
  BoxIdx(const int l[3], const int h[3]) {
    for (int d = 0; d < 3; ++d) { lo[d] = l[d]; n[d] = h[d] - l[d] + 1; }
    N = (size_t)n[0] * n[1] * n[2];
  }
  size_t operator()(int i, int j, int k) const {
    return (size_t)(i - lo[0]) + (size_t)n[0] * ((size_t)(j - lo[1]) + (size_t)n[1] * (size_t)(k - lo[2]));
  }
};

// Per-context geometry cache of one level (what the reference keeps in
// levelGeometry statics and the per-patch face/CFL/gravity caches).
struct Level {
  hc_params P;
  int nr, na, g;
  double h;
  std::vector<Radial> radial;      // [nr + 2g + 1], index i + g
  std::vector<Frame> frames[3];    // per panel: d=0 [na][na], d=1 [na][na+1], d=2 [na+1][na]
  std::vector<double> det;         // [6][na][na]
  std::vector<double> detAA;       // [6][na][na][9] row-major
  std::vector<double> cellBasis;   // [6][na][na][9]
  std::vector<double> cflDet;      // [6][na][na][3] face det(A), d = 0,1,2
  std::vector<double> cflNormal;   // [6][na][na][3] |adjA| of the low face of d
  std::vector<double> cflFace;     // [6][na][na][2][9] pointwise basis at low faces d=1,2
  // seam plan: per panel, per ghost cell (non-corner): donor panel, 4 donor
  // (j,k) and 4 weights
  struct Donor { int b, j[4], k[4]; double w[4]; };
  std::vector<Donor> seam;         // [6][2 edges axes][2 sides][g][na]
  // seam faces: neighbour panel, axis, side and along-edge index mapping
  struct SeamFace { int b, axis, side; std::vector<int> s; };
  SeamFace edges[6][2][2];

  // cone clouds fed through the inner boundary (hc_level_set_inlet) and the
  // operator's time (the stage time of levelRk4; NaN: no time, no footprint)
  std::vector<hc_cone> inlet;
  mutable double opTime = std::numeric_limits<double>::quiet_NaN();

  explicit Level(const hc_params& p) : P(p), nr(p.nr), na(p.na), g(2) {
    h = 1.0 / na;
    radial.resize(nr + 2 * g + 1);
    for (int i = -g; i <= nr + g; ++i) radial[i + g] = radialMetric(P, i);
    for (int d = 0; d < 3; ++d) frames[d].resize((size_t)6 * (na + 1) * (na + 1));
    det.resize((size_t)6 * na * na);
    detAA.resize((size_t)6 * na * na * 9);
    cellBasis.resize((size_t)6 * na * na * 9);
    cflDet.resize((size_t)6 * na * na * 3);
    cflNormal.resize((size_t)6 * na * na * 3);
    cflFace.resize((size_t)6 * na * na * 18);
    for (int b = 0; b < 6; ++b) {
      for (int k = 0; k <= na; ++k)
        for (int j = 0; j <= na; ++j)
          for (int d = 0; d < 3; ++d) {
            if ((d != 1 && j == na) || (d != 2 && k == na)) continue;
            LD n[3];
            faceNormal(b, d, j, k, (LD)h, n);
            double nd[3] = {(double)n[0], (double)n[1], (double)n[2]};
            symmetricNormal(nd);
            frames[d][frameIdx(b, j, k)] = secondOrderFrame(nd);
          }
      for (int k = 0; k < na; ++k)
        for (int j = 0; j < na; ++j) {
          LD dt, dA[3][3];
          cellAverages(b, j, k, (LD)h, dt, dA);
          size_t c = cellIdx(b, j, k);
          det[c] = (double)dt;
          for (int r = 0; r < 3; ++r) for (int s = 0; s < 3; ++s) detAA[c * 9 + r * 3 + s] = (double)dA[r][s];
          double A[3][3];
          pointBasis(b, -1, j, k, (LD)h, A);
          for (int r = 0; r < 3; ++r) for (int s = 0; s < 3; ++s) cellBasis[c * 9 + r * 3 + s] = A[r][s];
          for (int d = 0; d < 3; ++d) {
            cflDet[c * 3 + d] = d == 0 ? det[c] : (double)faceDet(b, d, j, k, (LD)h);
            const Frame& f = frames[d][frameIdx(b, j, k)];
            double n2 = 0;
            for (int q = 0; q < 3; ++q) n2 += f.normal[q] * f.normal[q];
            cflNormal[c * 3 + d] = std::sqrt(n2);
            if (d) {
              double F[3][3];
              pointBasis(b, d, j, k, (LD)h, F);
              for (int r = 0; r < 3; ++r) for (int s = 0; s < 3; ++s) cflFace[c * 18 + (d - 1) * 9 + r * 3 + s] = F[r][s];
            }
          }
        }
    }
    buildSeams();
  }
  size_t frameIdx(int b, int j, int k) const { return ((size_t)b * (na + 1) + k) * (na + 1) + j; }
  size_t cellIdx(int b, int j, int k) const { return ((size_t)b * na + k) * na + j; }
  const Radial& rad(int i) const { return radial[i + g]; }

  // Which panel holds direction X, and its panel coordinates.
  static void locate(const LD X[3], int& pb, LD& x1, LD& x2) {
    pb = 0;
    LD best = -1;
    for (int b = 0; b < 6; ++b) {
      LD q[3];
      for (int k = 0; k < 3; ++k) q[PERM[b][k]] = SIGN[b][k] * X[k];
      if (q[0] > best) { best = q[0]; pb = b; }
    }
    LD q[3];
    for (int k = 0; k < 3; ++k) q[PERM[pb][k]] = SIGN[pb][k] * X[k];
    x1 = (atanl(q[1] / q[0]) + PI_L / 4) / (PI_L / 2);
    x2 = (atanl(q[2] / q[0]) + PI_L / 4) / (PI_L / 2);
  }

  void buildSeams() {
    const LD hl = h;
    seam.resize((size_t)6 * 2 * 2 * g * na);
    for (int b = 0; b < 6; ++b)
      for (int ax = 1; ax <= 2; ++ax)
        for (int side = 0; side < 2; ++side) {
          // Neighbour panel and its normal axis from the mid-edge ghost.
          auto ghostXi = [&](int m, int s, LD& x1, LD& x2) {
            LD n = side == 0 ? -(m + 0.5L) * hl : 1 + (m + 0.5L) * hl;
            LD t = (s + 0.5L) * hl;
            if (ax == 1) { x1 = n; x2 = t; } else { x1 = t; x2 = n; }
          };
          LD x1, x2, X[3];
          ghostXi(0, na / 2, x1, x2);
          unitPoint(b, x1, x2, X);
          int nb;
          LD y1, y2;
          locate(X, nb, y1, y2);
          int nax = (std::min(y1, 1 - y1) < std::min(y2, 1 - y2)) ? 1 : 2;
          LD yn = nax == 1 ? y1 : y2;
          int nside = yn < 0.5L ? 0 : 1;
          for (int m = 0; m < g; ++m)
            for (int s = 0; s < na; ++s) {
              ghostXi(m, s, x1, x2);
              unitPoint(b, x1, x2, X);
              int pb;
              locate(X, pb, y1, y2);
              // Points exactly on a far corner may locate to a third panel;
              // recompute coordinates in the edge neighbour explicitly.
              LD q[3];
              for (int k = 0; k < 3; ++k) q[PERM[nb][k]] = SIGN[nb][k] * X[k];
              y1 = (atanl(q[1] / q[0]) + PI_L / 4) / (PI_L / 2);
              y2 = (atanl(q[2] / q[0]) + PI_L / 4) / (PI_L / 2);
              LD yt = nax == 1 ? y2 : y1;
              LD u = yt / hl - 0.5L;
              int base = (int)floorl(u) - 1;
              base = std::max(0, std::min(na - 4, base));
              Donor dn;
              dn.b = nb;
              int layer = nside == 0 ? m : na - 1 - m;
              for (int q4 = 0; q4 < 4; ++q4) {
                LD wq = 1;
                for (int r = 0; r < 4; ++r)
                  if (r != q4) wq *= (u - (base + r)) / (LD)(q4 - r);
                dn.w[q4] = (double)wq;
                if (nax == 1) { dn.j[q4] = layer; dn.k[q4] = base + q4; }
                else { dn.j[q4] = base + q4; dn.k[q4] = layer; }
              }
              seam[seamIdx(b, ax, side, m, s)] = dn;
            }
          // Seam faces: along-edge index mapping by face centres.
          SeamFace& sf = edges[b][ax - 1][side];
          sf.b = nb; sf.axis = nax; sf.side = nside; sf.s.resize(na);
          for (int s = 0; s < na; ++s) {
            LD t = (s + 0.5L) * hl, e = side == 0 ? 0 : 1;
            if (ax == 1) unitPoint(b, e, t, X); else unitPoint(b, t, e, X);
            LD q[3];
            for (int k = 0; k < 3; ++k) q[PERM[nb][k]] = SIGN[nb][k] * X[k];
            LD z1 = (atanl(q[1] / q[0]) + PI_L / 4) / (PI_L / 2);
            LD z2 = (atanl(q[2] / q[0]) + PI_L / 4) / (PI_L / 2);
            LD zt = nax == 1 ? z2 : z1;
            sf.s[s] = (int)lroundl(zt / hl - 0.5L);
          }
        }
  }
  size_t seamIdx(int b, int ax, int side, int m, int s) const {
    return ((((size_t)b * 2 + (ax - 1)) * 2 + side) * g + m) * na + s;
  }
};

// Level array indexing: valid arrays [6][8][nr][na][na]; primitive arrays
// [6][8][nr+2g][na+2g][na+2g].
struct LevelArrays {
  int nr, na, g;
  size_t Nv, Ng;
  LevelArrays(const Level& L) : nr(L.nr), na(L.na), g(L.g) {
    Nv = (size_t)nr * na * na;
    Ng = (size_t)(nr + 2 * g) * (na + 2 * g) * (na + 2 * g);
  }
  size_t v(int b, int c, int i, int j, int k) const { return ((size_t)b * NC + c) * Nv + (size_t)i + (size_t)nr * ((size_t)j + (size_t)na * k); }
  size_t w(int b, int c, int i, int j, int k) const {
    size_t n0 = nr + 2 * g, n1 = na + 2 * g;
    return ((size_t)b * NC + c) * Ng + (size_t)(i + g) + n0 * ((size_t)(j + g) + n1 * (size_t)(k + g));
  }
};

// ---------------------------------------------------------------------------
// Per-box second-order operator, restated from the fused HOST face loop of
// src/BoxOp_SecondOrder.H:155-370 with cartesianPrimitives = true, no AMR
// face mask, no CME emergence and no constant-background magnetic test.
// w is on valid.grow(ghost); rhs on valid; flux[d] on valid.extrude(d).
// ---------------------------------------------------------------------------
// A finite cone cloud at time t (expandedSource + sample, src/MHD_CME.H:
// 995-1018, 1139-1143) while its boundary feeding lasts (:968): inside
// flag and, when inside, the radial cloud velocity at `pos`.
bool inletSample(const hc_cone& c, double t, const double pos[3], double v[3]) {
  if (!(t >= c.insertion_time && t < c.end_time)) return false;
  const double shift = c.entry_shift + c.speed * 1e5 * (t - c.entry_time);
  const double q[3] = {pos[0] - shift * c.axis[0], pos[1] - shift * c.axis[1], pos[2] - shift * c.axis[2]};
  if (std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]) > c.radius) return false;
  const double radius = std::sqrt(pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2]) / 69600000000.0;
  if (!(radius > 0)) return false;
  for (int d = 0; d < 3; ++d) v[d] = c.speed * 1e5 * pos[d] / (69600000000.0 * radius);
  return true;
}

void boxOperator(const Level& L, const int lo[3], const int hi[3], int ghost, int block,
                 const double* w, const double* const* panel, double scale, double* rhs,
                 double* const* fluxOut) {
  const hc_params& P = L.P;
  const int limiter = P.limiter;
  const bool roe = P.riemann_solver == 2, powell = P.divergence_cleaning == 1;
  int glo[3], ghi[3];
  for (int d = 0; d < 3; ++d) { glo[d] = lo[d] - ghost; ghi[d] = hi[d] + ghost; }
  BoxIdx W(glo, ghi), V(lo, hi);
  const double dx[3] = {1.0 / shellCells(P), 1.0 / P.na, 1.0 / P.na};
  std::vector<double> minusDiv(V.N, 0.0);
  for (int dir = 0; dir < 3; ++dir) {
    int flo[3] = {lo[0], lo[1], lo[2]}, fhi[3] = {hi[0], hi[1], hi[2]};
    fhi[dir] += 1;
    BoxIdx F(flo, fhi);
    std::vector<double> flux(F.N * NC), bface(F.N);
    const ptrdiff_t step = dir == 0 ? 1 : dir == 1 ? (ptrdiff_t)W.n[0] : (ptrdiff_t)W.n[0] * W.n[1];
    // panel seam state slabs: valid.extrude(dir).face(dir, side)
    const double* pLow = nullptr; const double* pHigh = nullptr;
    if (panel && dir > 0) { pLow = panel[2 * dir]; pHigh = panel[2 * dir + 1]; }
    int slo[3] = {flo[0], flo[1], flo[2]}, shi[3] = {fhi[0], fhi[1], fhi[2]};
    slo[dir] = shi[dir] = flo[dir];
    BoxIdx SL(slo, shi);
    int tlo[3] = {flo[0], flo[1], flo[2]}, thi[3] = {fhi[0], fhi[1], fhi[2]};
    tlo[dir] = thi[dir] = fhi[dir];
    BoxIdx SH(tlo, thi);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = flo[2]; k <= fhi[2]; ++k)
      for (int j = flo[1]; j <= fhi[1]; ++j) {
        const Frame& fr = L.frames[dir][L.frameIdx(block, j, k)];
        for (int i = flo[0]; i <= fhi[0]; ++i) {
          size_t c0 = W(i, j, k);
          double mm[8], m[8], c[8], p[8];
          for (int q = 0; q < NC; ++q) {
            const double* s = w + q * W.N + c0;
            mm[q] = s[-2 * step]; m[q] = s[-step]; c[q] = s[0]; p[q] = s[step];
          }
          double l[8], r[8];
          plmFace(mm, m, c, p, limiter, l, r);
          int fp[3] = {i, j, k};
          if (pLow && fp[dir] == flo[dir]) for (int q = 0; q < NC; ++q) l[q] = pLow[q * SL.N + SL(i, j, k)];
          if (pHigh && fp[dir] == fhi[dir]) for (int q = 0; q < NC; ++q) r[q] = pHigh[q * SH.N + SH(i, j, k)];
          if (dir == 0 && i == 0 && !L.inlet.empty() && !std::isnan(L.opTime)) {
            // inlet footprint, src/BoxOp_SecondOrder.H:175-181, 282-311
            const double pos[3] = {P.inner_radius * fr.f[0][0], P.inner_radius * fr.f[0][1], P.inner_radius * fr.f[0][2]};
            bool footprint = false;
            for (const hc_cone& cone : L.inlet) {
              double v[3];
              if (inletSample(cone, L.opTime, pos, v)) { footprint = true; break; }
            }
            if (footprint) {
              for (int q = 0; q < NC; ++q) {
                const double* s = w + q * W.N + c0;
                const double a = s[step] - s[0], b = s[2 * step] - s[step];
                double slope = 0.5 * (a + b);
                if (limiter != 0) slope = a * b <= 0 ? 0.0 : (a > 0 ? std::min(a, b) : std::max(a, b));
                if (limiter == 3 && a * b > 0)
                  slope = (a > 0 ? 1.0 : -1.0) * std::min(0.5 * std::fabs(a + b), 2.0 * std::min(std::fabs(a), std::fabs(b)));
                r[q] = s[0] - 0.5 * slope;
              }
              if (!(r[iRHO] >= RHO00 && r[iP] > 0))
                for (int q = 0; q < NC; ++q) r[q] = w[q * W.N + c0];
              double jump = 0;
              for (int d = 0; d < 3; ++d) jump += (r[5 + d] - l[5 + d]) * fr.f[0][d];
              for (int d = 0; d < 3; ++d) l[5 + d] += jump * fr.f[0][d];
            }
          }
          const double area = dir == 0 ? L.rad(i).area0 : L.rad(i).areaT;
          double out[8];
          faceFlux(out, l, r, fr, area, P.gamma, P.entropy_fix_coeff, roe);
          size_t f = F(i, j, k);
          for (int q = 0; q < NC; ++q) flux[q * F.N + f] = out[q];
          if (powell) {
            double bf = 0;
            for (int d = 0; d < 3; ++d) bf += 0.5 * (l[iBX + d] + r[iBX + d]) * fr.normal[d] * area;
            bface[f] = bf;
          }
        }
      }
    // FluxDivergence(dir) scaled by -scale/dx[dir]
    const double coef = -scale / dx[dir];
    int sh[3] = {0, 0, 0};
    sh[dir] = 1;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = lo[2]; k <= hi[2]; ++k)
      for (int j = lo[1]; j <= hi[1]; ++j)
        for (int i = lo[0]; i <= hi[0]; ++i) {
          size_t fl = F(i, j, k), fh = F(i + sh[0], j + sh[1], k + sh[2]), v = V(i, j, k);
          for (int q = 0; q < NC; ++q) rhs[q * V.N + v] += coef * (flux[q * F.N + fh] - flux[q * F.N + fl]);
          if (powell) minusDiv[v] += coef * (bface[fh] - bface[fl]);
        }
    if (fluxOut && fluxOut[dir]) std::memcpy(fluxOut[dir], flux.data(), flux.size() * sizeof(double));
  }
  if (powell) {
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = lo[2]; k <= hi[2]; ++k)
      for (int j = lo[1]; j <= hi[1]; ++j)
        for (int i = lo[0]; i <= hi[0]; ++i) {
          size_t v = V(i, j, k), c0 = W(i, j, k);
          double md = minusDiv[v], vb = 0;
          for (int d = 0; d < 3; ++d) {
            const double b = w[(iBX + d) * W.N + c0];
            const double vel = w[(iVX + d) * W.N + c0];
            rhs[(1 + d) * V.N + v] += md * b / (4 * M_PI);
            rhs[(iBX + d) * V.N + v] += md * vel;
            vb += vel * b;
          }
          rhs[iE * V.N + v] += md * vb / (4 * M_PI);
        }
  }
}

// src/BoxOp_Gravity.H:3-61 (HOST branch): cached cell-centre Xhat, cell
// det(A) and the first column of <det(A) A>; radial (rhigh-rlow)/dxi0.
void boxGravity(const Level& L, const int lo[3], const int hi[3], int ghost, int block,
                const double* w, double* rhs) {
  int glo[3], ghi[3];
  for (int d = 0; d < 3; ++d) { glo[d] = lo[d] - ghost; ghi[d] = hi[d] + ghost; }
  BoxIdx W(glo, ghi), V(lo, hi);
  for (int k = lo[2]; k <= hi[2]; ++k)
    for (int j = lo[1]; j <= hi[1]; ++j) {
      size_t c = L.cellIdx(block, j, k);
      double a[7];
      for (int d = 0; d < 3; ++d) { a[d] = L.cellBasis[c * 9 + d * 3 + 0]; a[4 + d] = L.detAA[c * 9 + d * 3 + 0]; }
      a[3] = L.det[c];
      for (int i = lo[0]; i <= hi[0]; ++i) {
        size_t s = W(i, j, k), v = V(i, j, k);
        const double factor = -c_G * c_M0 * L.rad(i).Dr0 * w[s];
        double radialVelocity = 0;
        for (int d = 0; d < 3; ++d) {
          rhs[(1 + d) * V.N + v] += factor * a[4 + d];
          radialVelocity += a[d] * w[(iVX + d) * W.N + s];
        }
        rhs[iE * V.N + v] += factor * a[3] * radialVelocity;
      }
    }
}

// ---------------------------------------------------------------------------
// Level stage preparation (src/BoxOp_SecondOrderPreStage.H:7-77, 103-218 and
// src/BoxOp_PreStage.H:57-141,215-228 for init_condition_type 1).
// ---------------------------------------------------------------------------
void analyticWind(const hc_params& P, double radius, const double X[3], double t, double u[8]) {
  // src/BoxOp_PreStage.H:7-47 (f_radialoutflowIBCs)
  const double gam = P.gamma, r_BC = P.inner_radius;
  double r = std::sqrt(X[0] * X[0] + X[1] * X[1] + X[2] * X[2]);
  double theta = std::atan2(std::sqrt(X[0] * X[0] + X[1] * X[1]), X[2]);
  double phi = std::atan2(X[1], X[0]);
  double p0 = 1.0e-7, rho0 = 700 * c_MP, u0 = 500.0 * 1e5;
  double rho = rho0 * std::pow(r_BC / r, 2.0);
  double p = p0 * std::pow(r_BC / r, 2.0 * gam);
  double carr_rot_time = 25.38 * 24 * 60 * 60;
  double omega = 2.0 * M_PI / carr_rot_time;
  double phit = phi - omega * t;
  const double perturbationScale = P.strength / 100.0;
  const double sinTheta = std::sin(theta);
  const double angularPattern = std::pow(sinTheta, 5) * std::sin(5 * phit) + std::pow(sinTheta, 10) * std::sin(10 * phit);
  double ur = u0 - perturbationScale * u0 / 3 * angularPattern;
  u[0] = rho; u[1] = ur * rho; u[2] = 0.0; u[3] = 0.0; u[5] = 0.0; u[6] = 0.0; u[7] = 0.0;
  double umag = std::sqrt(u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / u[0];
  double Bmag = std::sqrt(u[5] * u[5] + u[6] * u[6] + u[7] * u[7]);
  u[4] = p / (gam - 1.0) + 0.5 * u[0] * umag * umag + Bmag * Bmag / 8.0 / M_PI;
  (void)radius;
}

// Inner-ghost inlet of the clouds crossing r_inner, src/BoxOp_PreStage.H:
// 329-400 (finite clouds: sampled on the boundary sphere, taper weight 1):
// u native conserved, A the cell basis, inv its inverse, pos the ghost
// centre.
void inletGhost(const Level& L, double t, const double pos[3], const double A[3][3], const double inv[3][3],
                double u[8]) {
  const hc_params& P = L.P;
  const double radius = std::sqrt(pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2]);
  const double inner = P.inner_radius;
  for (const hc_cone& c : L.inlet) {
    double v[3];
    const double face[3] = {pos[0] * inner / radius, pos[1] * inner / radius, pos[2] * inner / radius};
    if (!inletSample(c, t, face, v)) continue;
    double old[8] = {u[0], 0, 0, 0, 0, 0, 0, 0};
    double ke = 0, me = 0, radialOld = 0, radialCME = 0;
    for (int d = 0; d < 3; ++d) {
      for (int q = 0; q < 3; ++q) {
        old[1 + d] += A[d][q] * u[1 + q] / old[0];
        old[5 + d] += A[d][q] * u[5 + q];
      }
      ke += .5 * old[0] * old[1 + d] * old[1 + d];
      me += old[5 + d] * old[5 + d] / (8 * M_PI);
      radialOld += old[1 + d] * pos[d] / radius;
      radialCME += v[d] * pos[d] / radius;
    }
    old[4] = std::max(0., (u[4] - ke - me) * (P.gamma - 1));
    for (int d = 0; d < 3; ++d) v[d] = radialCME * pos[d] / radius;
    const double weight = 1;
    for (int d = 0; d < 3; ++d) v[d] = old[1 + d] + weight * (v[d] - old[1 + d]);
    const double density = (1 - weight) * old[0] + weight * c.density;
    double oldKinetic = 0, newKinetic = 0, oldMagnetic = 0, newMagnetic = 0, delta[8];
    delta[0] = density - old[0];
    for (int d = 0; d < 3; ++d) {
      delta[1 + d] = density * v[d] - old[0] * old[1 + d];
      delta[5 + d] = 0.0;
      oldKinetic += .5 * old[0] * old[1 + d] * old[1 + d];
      newKinetic += .5 * density * v[d] * v[d];
      oldMagnetic += old[5 + d] * old[5 + d] / (8 * M_PI);
      newMagnetic += (old[5 + d] + 0.0) * (old[5 + d] + 0.0) / (8 * M_PI);
    }
    const double target = 2 * 1.380649e-16 * c.temperature * c.density / c_MP;
    const double pressure = (1 - weight) * std::max(0., old[4]) + weight * target;
    delta[4] = (pressure - std::max(0., old[4])) / (P.gamma - 1) + newKinetic - oldKinetic + newMagnetic - oldMagnetic;
    u[0] += delta[0];
    u[4] += delta[4];
    for (int d = 0; d < 3; ++d)
      for (int q = 0; q < 3; ++q) {
        u[1 + d] += inv[d][q] * delta[1 + q];
        u[5 + d] += inv[d][q] * delta[5 + q];
      }
  }
}

void levelPrepare(const Level& L, const double* ju, double* w, double t) {
  const hc_params& P = L.P;
  LevelArrays I(L);
  const int nr = L.nr, na = L.na, g = L.g;
  // 1. JU/J -> Cartesian primitives on valid cells.
#pragma omp parallel for collapse(2) schedule(static)
  for (int b = 0; b < 6; ++b)
    for (int k = 0; k < na; ++k)
      for (int j = 0; j < na; ++j) {
        double det = L.det[L.cellIdx(b, j, k)];
        for (int i = 0; i < nr; ++i) {
          double in[8], out[8];
          for (int c = 0; c < NC; ++c) in[c] = ju[I.v(b, c, i, j, k)];
          double invJ = 1.0 / (L.rad(i).vol * det);
          cartesianPrimitiveFromConserved(out, in, invJ, P.gamma);
          for (int c = 0; c < NC; ++c) w[I.w(b, c, i, j, k)] = out[c];
        }
      }
  // 2. Angular seam ghosts: own 4-point along-edge interpolation of the
  //    adjacent panel's Cartesian primitives (Proto MBInterpOp unavailable),
  //    then the floors of src/BoxOp_SecondOrderPreStage.H:70-75.
#pragma omp parallel for collapse(3) schedule(static)
  for (int b = 0; b < 6; ++b)
    for (int ax = 1; ax <= 2; ++ax)
      for (int side = 0; side < 2; ++side)
        for (int m = 0; m < g; ++m)
          for (int s = 0; s < na; ++s) {
            const Level::Donor& dn = L.seam[L.seamIdx(b, ax, side, m, s)];
            int gj, gk;
            int n = side == 0 ? -1 - m : na + m;
            if (ax == 1) { gj = n; gk = s; } else { gj = s; gk = n; }
            for (int i = 0; i < nr; ++i)
              for (int c = 0; c < NC; ++c) {
                double v = 0.;
                for (int q = 0; q < 4; ++q) v += dn.w[q] * w[I.w(dn.b, c, i, dn.j[q], dn.k[q])];
                w[I.w(b, c, i, gj, gk)] = v;
              }
            for (int i = 0; i < nr; ++i) {
              double& rho = w[I.w(b, 0, i, gj, gk)];
              double& p = w[I.w(b, 4, i, gj, gk)];
              rho = std::max(rho, RHO00);
              p = std::max(p, 0.0);
            }
          }
  // 3. Radial ghosts over the valid angular range
  //    (src/BoxOp_SecondOrderPreStage.H:125-216).
#pragma omp parallel for collapse(2) schedule(static)
  for (int b = 0; b < 6; ++b)
    for (int k = 0; k < na; ++k)
      for (int j = 0; j < na; ++j) {
        size_t cidx = L.cellIdx(b, j, k);
        double A[3][3], inv[3][3];
        for (int r = 0; r < 3; ++r) for (int s = 0; s < 3; ++s) A[r][s] = L.cellBasis[cidx * 9 + r * 3 + s];
        inverse3(A, inv);
        auto toPrim = [&](const double u[8], double out[8]) {
          double ww[8];
          ww[0] = u[0]; ww[4] = u[4];
          for (int grp = 0; grp < 2; ++grp) {
            int st = grp == 0 ? 1 : 5;
            for (int d = 0; d < 3; ++d) {
              ww[st + d] = 0;
              for (int q = 0; q < 3; ++q) ww[st + d] += A[d][q] * u[st + q];
            }
          }
          cartesianPrimitiveFromConserved(out, ww, 1.0, P.gamma);
        };
        // inner: analytic wind at ghost-cell centres
        if (P.init_condition_type == 1) {
          LD Xl[3];
          unitPoint(b, (j + 0.5L) * L.h, (k + 0.5L) * L.h, Xl);
          for (int i = -g; i < 0; ++i) {
            double radius = L.rad(i).rad;
            double X[3] = {radius * (double)Xl[0], radius * (double)Xl[1], radius * (double)Xl[2]};
            double u[8], out[8];
            analyticWind(P, radius, X, t, u);
            if (!L.inlet.empty()) inletGhost(L, t, X, A, inv, u);
            toPrim(u, out);
            for (int c = 0; c < NC; ++c) w[I.w(b, c, i, j, k)] = out[c];
          }
        }
        // outer: copy the last owned layer scaled by radius
        // (src/BoxOp_PreStage.H:105-141)
        {
          double wl[8], u[8];
          for (int c = 0; c < NC; ++c) wl[c] = w[I.w(b, c, nr - 1, j, k)];
          u[0] = wl[0];
          double kinetic = 0, magnetic = 0;
          for (int d = 0; d < 3; ++d) {
            kinetic += 0.5 * wl[0] * wl[1 + d] * wl[1 + d];
            magnetic += wl[5 + d] * wl[5 + d] / (8 * M_PI);
            u[1 + d] = u[5 + d] = 0;
            for (int q = 0; q < 3; ++q) {
              u[1 + d] += inv[d][q] * wl[0] * wl[1 + q];
              u[5 + d] += inv[d][q] * wl[5 + q];
            }
          }
          u[4] = (wl[4] - 0.0) / (P.gamma - 1.0) + kinetic + magnetic;
          double rl = L.rad(nr - 1).rad;
          for (int i = nr; i < nr + g; ++i) {
            double rr = L.rad(i).rad, ug[8], out[8];
            double s2 = std::pow(rl / rr, 2.0), s1 = std::pow(rl / rr, 1.0);
            for (int c = 0; c < 6; ++c) ug[c] = u[c] * s2;
            ug[6] = u[6] * s1;
            ug[7] = u[7] * s1;
            toPrim(ug, out);
            for (int c = 0; c < NC; ++c) w[I.w(b, c, i, j, k)] = out[c];
          }
        }
      }
}

// Stage right-hand side of a level: zero, gravity, shared seam states
// (src/BoxOp_SecondOrder.H:68-121), per-panel operator.
void levelRhs(const Level& L, const double* w, double* kOut) {
  const hc_params& P = L.P;
  LevelArrays I(L);
  const int nr = L.nr, na = L.na, g = L.g;
  std::memset(kOut, 0, sizeof(double) * 6 * NC * I.Nv);
  // Each panel's interior-side state at each of its seam faces.
  // own[b][ax-1][side]: slab [8][face slab]
  std::vector<double> own[6][2][2], incoming[6][2][2];
  for (int b = 0; b < 6; ++b)
    for (int ax = 1; ax <= 2; ++ax)
      for (int side = 0; side < 2; ++side) {
        size_t Ns = (size_t)nr * na;
        own[b][ax - 1][side].assign(NC * Ns, 0.0);
        int f = side == 0 ? 0 : na;
        for (int s = 0; s < na; ++s)
          for (int i = 0; i < nr; ++i) {
            double st[4][8], lo[8], hi[8];
            for (int q = 0; q < 4; ++q) {
              int n = f - 2 + q;
              int j = ax == 1 ? n : s, k = ax == 1 ? s : n;
              for (int c = 0; c < NC; ++c) st[q][c] = w[I.w(b, c, i, j, k)];
            }
            plmFace(st[0], st[1], st[2], st[3], P.limiter, lo, hi);
            const double* mine = side == 0 ? hi : lo;
            for (int c = 0; c < NC; ++c) own[b][ax - 1][side][c * Ns + i + (size_t)nr * s] = mine[c];
          }
      }
  // Exchange: the neighbour's interior-side state at the same physical face.
  for (int b = 0; b < 6; ++b)
    for (int ax = 1; ax <= 2; ++ax)
      for (int side = 0; side < 2; ++side) {
        const Level::SeamFace& sf = L.edges[b][ax - 1][side];
        size_t Ns = (size_t)nr * na;
        std::vector<double>& in = incoming[b][ax - 1][side];
        in.assign(NC * Ns, 0.0);
        const std::vector<double>& src = own[sf.b][sf.axis - 1][sf.side];
        for (int s = 0; s < na; ++s)
          for (int i = 0; i < nr; ++i)
            for (int c = 0; c < NC; ++c)
              in[c * Ns + i + (size_t)nr * s] = src[c * Ns + i + (size_t)nr * sf.s[s]];
      }
  for (int b = 0; b < 6; ++b) {
    int lo[3] = {0, 0, 0}, hi[3] = {nr - 1, na - 1, na - 1};
    double* rhs = kOut + (size_t)b * NC * I.Nv;
    const double* wb = w + (size_t)b * NC * I.Ng;
    if (P.sun_gravity == 1) boxGravity(L, lo, hi, g, b, wb, rhs);
    // slab layout of the face slabs valid.extrude(d).face(d,side): for d=1
    // the slab box is (nr, 1, na) -> index i + nr*k; for d=2 (nr, na, 1) ->
    // i + nr*j.  Both equal i + nr*s.
    const double* panel[6] = {nullptr, nullptr,
                              incoming[b][0][0].data(), incoming[b][0][1].data(),
                              incoming[b][1][0].data(), incoming[b][1][1].data()};
    boxOperator(L, lo, hi, g, b, wb, panel, 1.0, rhs, nullptr);
  }
}

// Classical RK4 tableau, src/MHD_AMRRungeKutta.H:10-12, applied as
// stage = U + (dt a) k and U += (dt b_s) k_s in stage order.
void levelRk4(const Level& L, double* ju, double dt, double t) {
  static const double a4[4][4] = {{0, 0, 0, 0}, {0.5, 0, 0, 0}, {0, 0.5, 0, 0}, {0, 0, 1, 0}};
  static const double c4[4] = {0, 0.5, 0.5, 1}, b4[4] = {1.0 / 6, 1.0 / 3, 1.0 / 3, 1.0 / 6};
  LevelArrays I(L);
  const size_t n = 6 * NC * I.Nv;
  std::vector<double> stage(n), w(6 * NC * I.Ng, 0.0), k[4];
  for (int s = 0; s < 4; ++s) {
    std::memcpy(stage.data(), ju, n * sizeof(double));
    for (int prev = 0; prev < s; ++prev)
      if (a4[s][prev] != 0) {
        const double f = dt * a4[s][prev];
#pragma omp parallel for schedule(static)
        for (size_t q = 0; q < n; ++q) stage[q] += f * k[prev][q];
      }
    levelPrepare(L, stage.data(), w.data(), t + c4[s] * dt);
    k[s].resize(n);
    L.opTime = t + c4[s] * dt;
    levelRhs(L, w.data(), k[s].data());
    L.opTime = std::numeric_limits<double>::quiet_NaN();
  }
  for (int s = 0; s < 4; ++s) {
    const double f = dt * b4[s];
#pragma omp parallel for schedule(static)
    for (size_t q = 0; q < n; ++q) ju[q] += f * k[s][q];
  }
}

// src/BoxOp_SecondOrderCFL.H:99-210 (no mapped scale, no cone density).
double levelInvDt(const Level& L, const double* ju, double coneDensity = 0) {
  const hc_params& P = L.P;
  LevelArrays I(L);
  const int nr = L.nr, na = L.na;
  const double gamma = P.gamma, h = L.h;
  double gmax = 0;
  (void)h;
#pragma omp parallel for collapse(2) reduction(max : gmax) schedule(static)
  for (int b = 0; b < 6; ++b)
    for (int k = 0; k < na; ++k)
      for (int j = 0; j < na; ++j) {
        size_t cidx = L.cellIdx(b, j, k);
        double inverseDet = 1.0 / L.det[cidx], dA[3][3], inverseDetA[3][3], cell[3][3], face[2][3][3];
        double fdet[3], normal[3];
        for (int r = 0; r < 3; ++r) for (int s = 0; s < 3; ++s) { dA[r][s] = L.detAA[cidx * 9 + r * 3 + s]; cell[r][s] = L.cellBasis[cidx * 9 + r * 3 + s]; }
        inverse3(dA, inverseDetA);
        for (int d = 0; d < 3; ++d) {
          fdet[d] = L.cflDet[cidx * 3 + d];
          normal[d] = L.cflNormal[cidx * 3 + d];
          if (d) for (int r = 0; r < 3; ++r) for (int s = 0; s < 3; ++s) face[d - 1][r][s] = L.cflFace[cidx * 18 + (d - 1) * 9 + r * 3 + s];
        }
        for (int i = 0; i < nr; ++i) {
          const Radial& r = L.rad(i);
          const double inverseVolume = 1.0 / r.vol, width0 = r.Dr0 * (1.0 / shellCells(L.P));
          const double area[3] = {r.area0, r.areaT, r.areaT};
          double u[8];
          for (int c = 0; c < NC; ++c) u[c] = ju[I.v(b, c, i, j, k)];
          double rho = u[0] * inverseDet;
          rho *= inverseVolume;
          rho = std::max(rho, RHO00);
          double energy = u[4] * inverseDet;
          energy *= inverseVolume;
          double v[3] = {}, bb[3] = {};
          for (int d = 0; d < 3; ++d) {
            for (int q = 0; q < 3; ++q) { v[d] += inverseDetA[d][q] * u[1 + q]; bb[d] += inverseDetA[d][q] * u[5 + q]; }
            v[d] *= inverseVolume; bb[d] *= inverseVolume;
            v[d] /= rho;
          }
          double vc[3] = {}, bc[3] = {}, kinetic = 0, magnetic = 0, b2 = 0;
          for (int d = 0; d < 3; ++d) {
            for (int q = 0; q < 3; ++q) { vc[d] += cell[d][q] * v[q]; bc[d] += cell[d][q] * bb[q]; }
            kinetic += vc[d] * vc[d] / 2;
            magnetic += bc[d] * bc[d] / 8.0 / M_PI;
            b2 += bc[d] * bc[d];
          }
          kinetic *= rho;
          double pressure = (energy - kinetic - magnetic) * (gamma - 1);
          if (pressure < 0) pressure = 0;
          double inverseDt = 0;
          for (int d = 0; d < 3; ++d) {
            const double (*basis)[3] = d == 0 ? cell : face[d - 1];
            double v2 = 0, fullB2 = 0;
            for (int q = 0; q < 3; ++q) {
              double velocity = 0, field = 0;
              for (int s = 0; s < 3; ++s) { velocity += basis[q][s] * v[s]; field += basis[q][s] * bb[s]; }
              v2 += velocity * velocity;
              fullB2 += field * field;
            }
            const double width = d == 0 ? width0 : r.vol * fdet[d] * h / area[d] / normal[d];
            // src/BoxOp_SecondOrderCFL.H:196-200
            const double magneticDensity = coneDensity > 0 ? std::min(rho, coneDensity) : rho;
            const double wave = std::sqrt(gamma * pressure / rho + fullB2 / 4.0 / M_PI / magneticDensity);
            inverseDt += (wave + std::sqrt(v2)) / width;
          }
          gmax = std::max(gmax, inverseDt);
        }
      }
  return gmax;
}

// src/BoxOp_EulerCubedSphereImplem.H:817-876
int levelValid(const Level& L, const double* ju) {
  LevelArrays I(L);
  const size_t n = 6 * NC * I.Nv;
  int ok = 1;
  for (int b = 0; b < 6 && ok; ++b)
    for (int c = 0; c < NC && ok; ++c)
      for (size_t q = 0; q < I.Nv; ++q) {
        double v = ju[((size_t)b * NC + c) * I.Nv + q];
        if (!std::isfinite(v) || (c == 0 && !(v > 0))) { ok = 0; break; }
      }
  (void)n;
  return ok;
}

// Seeded synthetic initial state, kind 1 (the configs' own input):
// rho = rho0 (r_ref/r)^2, v = vr Xhat, p = p0 (r_ref/r)^(2 gamma) (1 + pulse),
// B = b0 (r_ref/r)^2 sign(z) Xhat; pulse = amp exp(-d^2/(2 w^2)), d^2 =
// (i-i*)^2 + (angle(Xhat,Xhat*)/(pi h/2))^2.  JU = dVolr det (rho, rho v, E, B).
void levelInit(const Level& L, const hc_init& in, double* ju) {
  const hc_params& P = L.P;
  LevelArrays I(L);
  const int nr = L.nr, na = L.na;
  LD Xc[3];
  unitPoint(in.pulse_block, (in.pulse_j + 0.5L) * L.h, (in.pulse_k + 0.5L) * L.h, Xc);
  const double cx[3] = {(double)Xc[0], (double)Xc[1], (double)Xc[2]};
  const double dang = M_PI / 2 * L.h;
#pragma omp parallel for collapse(2) schedule(static)
  for (int b = 0; b < 6; ++b)
    for (int k = 0; k < na; ++k)
      for (int j = 0; j < na; ++j) {
        LD Xl[3];
        unitPoint(b, (j + 0.5L) * L.h, (k + 0.5L) * L.h, Xl);
        const double X[3] = {(double)Xl[0], (double)Xl[1], (double)Xl[2]};
        const double det = L.det[L.cellIdx(b, j, k)];
        double cr[3] = {X[1] * cx[2] - X[2] * cx[1], X[2] * cx[0] - X[0] * cx[2], X[0] * cx[1] - X[1] * cx[0]};
        double ang = std::atan2(std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]), X[0] * cx[0] + X[1] * cx[1] + X[2] * cx[2]);
        double da = ang / dang;
        const double sgn = X[2] >= 0 ? 1.0 : -1.0;
        for (int i = 0; i < nr; ++i) {
          const Radial& r = L.rad(i);
          double s = in.r_ref / r.rad, s2 = s * s;
          double rho = in.rho0 * s2;
          double p = in.p0 * std::pow(s, 2.0 * P.gamma);
          double di = (double)(i - in.pulse_i);
          double d2 = di * di + da * da;
          if (in.pulse_amp != 0) p = p * (1.0 + in.pulse_amp * std::exp(-d2 / (2.0 * in.pulse_width * in.pulse_width)));
          double br = in.b0 * s2 * sgn;
          double E = p / (P.gamma - 1.0) + 0.5 * rho * in.vr * in.vr + br * br / (8.0 * M_PI);
          double J = r.vol * det;
          double u[8] = {rho, rho * in.vr * X[0], rho * in.vr * X[1], rho * in.vr * X[2], E, br * X[0], br * X[1], br * X[2]};
          for (int c = 0; c < NC; ++c) ju[I.v(b, c, i, j, k)] = J * u[c];
        }
      }
}

// ---------------------------------------------------------------------------
// Finite cone cloud (CME field model 4).
// Preparation: drag-based trajectory src/MHD_CME.H:1069-1085, boundary
// contact :1087-1110, prepareConeCloud :1111-1136, the analytic cone's axis
// orientation(lat, lon, 0) (0,0,1) of src/MHD_ImportedCME.H:72-79,415-418.
// Per cell: sample() for the finite cloud :995-1018 at the shift of
// expandedSource :1139-1143, increment() / thermalPressure() :1197-1238,
// applied as Insert_CME does for cones (src/BoxOp_EulerCubedSphereImplem.H:
// 1236-1300).
// ---------------------------------------------------------------------------
constexpr double c_SR = 69600000000.0;   // src/MHD_Constants.H:4
constexpr double kBoltzmann = 1.380649e-16;
constexpr double kPiCme = 3.1415926535897932384626433832795;

struct ConeTrajectory {
  double apex, wind, drag, height, reference;
};

bool coneTrajectory(const ConeTrajectory& c, double elapsed, double& height, double& speed) {
  const double dv = c.apex - c.wind;
  double distance = c.apex * elapsed;
  speed = c.apex;
  if (c.drag > 0 && dv != 0) {
    const double argument = c.drag * std::abs(dv) * elapsed;
    if (!(argument > -1)) return false;
    distance = c.wind * elapsed + std::copysign(1., dv) * std::log1p(argument) / c.drag;
    speed = c.wind + dv / (1 + argument);
  }
  height = c.height + 0.0 + distance * 1e5 / c_SR;
  return std::isfinite(height) && std::isfinite(speed) && speed > 0;
}

// Time at which the leading edge reaches the inner boundary; false where the
// reference throws.
bool coneBoundaryStart(const ConeTrajectory& c, double innerRsun, double& start) {
  double lower = -(c.height + 0.0 - innerRsun) * c_SR / (c.apex * 1e5), upper = 0;
  const double dv = c.apex - c.wind;
  if (c.drag == 0 || dv == 0) {
    start = c.reference + lower;
    return true;
  }
  if (c.drag > 0 && dv != 0) {
    if (dv > 0)
      lower = -(1 - 1e-12) / (c.drag * dv);
    else
      lower = (std::abs(dv) / c.wind - 1) / (c.drag * std::abs(dv));
  }
  double height, speed;
  if (!coneTrajectory(c, lower * (1 - 1e-12), height, speed) || height > innerRsun + 1e-8) return false;
  lower *= 1 - 1e-12;
  for (int i = 0; i < 100; ++i) {
    const double mid = .5 * (lower + upper);
    if (!coneTrajectory(c, mid, height, speed) || height < innerRsun)
      lower = mid;
    else
      upper = mid;
  }
  start = c.reference + .5 * (lower + upper);
  return true;
}

int conePrepare(const hc_cone_spec& s, double innerRadius, hc_cone& o) {
  const double innerRsun = innerRadius / c_SR;
  const ConeTrajectory c{s.apex_speed, s.wind_speed, s.drag_gamma, s.reference_height, s.reference_time};
  double entry, height, speed;
  if (!coneBoundaryStart(c, innerRsun, entry)) return -1;
  if (!coneTrajectory(c, entry - c.reference, height, speed)) return -2;
  std::memset(&o, 0, sizeof(o));
  const double inner = innerRsun * c_SR;
  const double lat = s.lat_deg * kPiCme / 180, lon = s.lon_deg * kPiCme / 180;
  const double alpha = s.half_angle_deg * kPiCme / 180;
  o.axis[0] = std::cos(lon) * std::cos(lat);
  o.axis[1] = -(-std::sin(lon) * std::cos(lat));
  o.axis[2] = std::sin(lat);
  o.radius = inner * std::sin(alpha);
  o.entry_time = entry;
  o.speed = speed;
  o.entry_shift = inner - o.radius;
  const double referenceShift = (s.reference_height + 0.0) * c_SR - o.radius;
  o.end_time = entry + 2 * o.radius / (speed * 1e5);
  o.insertion_time = entry + (referenceShift - o.entry_shift) / (speed * 1e5);
  o.density = s.density;
  o.temperature = s.temperature;
  return 0;
}

// The conserved change of one cell at Cartesian position `pos` (cm) with
// Cartesian primitive ambient state `old`; false outside the cloud.
bool coneCellDelta(const hc_cone& c, double shift, const double pos[3], const double old[8], double gamma,
                   double delta[8]) {
  const double q[3] = {pos[0] - shift * c.axis[0], pos[1] - shift * c.axis[1], pos[2] - shift * c.axis[2]};
  if (std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]) > c.radius) return false;
  const double radius = std::sqrt(pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2]) / c_SR;
  if (!(radius > 0)) return false;
  double v[3];
  for (int d = 0; d < 3; ++d) v[d] = c.speed * 1e5 * pos[d] / (c_SR * radius);
  const double weight = 1;  // volume insertion: plasmaWeight 1
  const double density = (1 - weight) * old[0] + weight * c.density;
  double oldKinetic = 0, newKinetic = 0, oldMagnetic = 0, newMagnetic = 0;
  delta[0] = density - old[0];
  for (int d = 0; d < 3; ++d) {
    delta[1 + d] = density * v[d] - old[0] * old[1 + d];
    delta[5 + d] = 0.0;
    oldKinetic += .5 * old[0] * old[1 + d] * old[1 + d];
    newKinetic += .5 * density * v[d] * v[d];
    oldMagnetic += old[5 + d] * old[5 + d] / (8 * kPiCme);
    newMagnetic += (old[5 + d] + 0.0) * (old[5 + d] + 0.0) / (8 * kPiCme);
  }
  const double target = 2 * kBoltzmann * c.temperature * c.density / c_MP;
  const double pressure = (1 - weight) * std::max(0., old[4]) + weight * target;
  const double addedPressure = pressure - std::max(0., old[4]);
  delta[4] = addedPressure / (gamma - 1) + newKinetic - oldKinetic + newMagnetic - oldMagnetic;
  return true;
}

void levelInsertCone(const Level& L, const hc_cone& c, double time, double* ju, double stats[2]) {
  LevelArrays I(L);
  const int nr = L.nr, na = L.na;
  const double shift = c.entry_shift + c.speed * 1e5 * (time - c.entry_time);
  const double dx0 = 1.0 / shellCells(L.P), dx1 = L.h;
  long long affected = 0;
  double added = 0;
  for (int b = 0; b < 6; ++b)
    for (int k = 0; k < na; ++k)
      for (int j = 0; j < na; ++j) {
        LD Xl[3];
        unitPoint(b, (j + 0.5L) * L.h, (k + 0.5L) * L.h, Xl);
        const double X[3] = {(double)Xl[0], (double)Xl[1], (double)Xl[2]};
        const double det = L.det[L.cellIdx(b, j, k)];
        for (int i = 0; i < nr; ++i) {
          const Radial& r = L.rad(i);
          const double pos[3] = {r.rad * X[0], r.rad * X[1], r.rad * X[2]};
          const double J = r.vol * det;
          double u[8], w[8], delta[8];
          for (int q = 0; q < NC; ++q) u[q] = ju[I.v(b, q, i, j, k)];
          cartesianPrimitiveFromConserved(w, u, 1.0 / J, L.P.gamma);
          if (!coneCellDelta(c, shift, pos, w, L.P.gamma, delta)) continue;
          for (int q = 0; q < NC; ++q) ju[I.v(b, q, i, j, k)] += J * delta[q];
          ++affected;
          added += delta[0] * (J * dx0 * dx1 * dx1);
        }
      }
  if (stats) {
    stats[0] = (double)affected;
    stats[1] = added;
  }
}

// CME insertion schedule, src/MHD_CME.H:1243-1334: the CFL fraction of
// cfl() (:1275-1297) and rusanovEndTime() (:1267-1271) over the sources
// inserted by `time`, stabilizationEnd (:1329-1332).
void cmeSchedule(const hc_cme_event* ev, int n, double time, double feeding, double& fraction, double& end) {
  fraction = 1;
  end = -std::numeric_limits<double>::infinity();
  for (int i = 0; i < n; ++i) {
    if (!(time >= ev[i].insertion_time)) continue;
    const double t = ev[i].insertion_time;
    const double stab = ev[i].boundary ? std::max(ev[i].feeding_end + 600, t + 2400) : t + 600;
    const double early = std::clamp((time - t - 600) / 1800., 0., 1.);
    double sourceFraction = .2 + .8 * early;
    if (ev[i].boundary) {
      const double recovery = std::clamp((time - stab) / 1800., 0., 1.);
      sourceFraction = .2 + (feeding - .2) * early + (1 - feeding) * recovery;
    }
    fraction = std::min(fraction, sourceFraction);
    end = std::max(end, stab);
  }
}

#include "hc_oracle_o4.inc"

}  // namespace

// ---------------------------------------------------------------------------
// C entry points (ctypes).  Context = the cached Level.
// ---------------------------------------------------------------------------
extern "C" {

void* orc_level_create(const hc_params* p) { return new Level(*p); }
void orc_level_destroy(void* L) { delete static_cast<Level*>(L); }

int orc_box_rhs(void* L, const hc_box* box, const double* w, const double* const* panel,
                double scale, double* rhs, double* const* flux) {
  boxOperator(*static_cast<Level*>(L), box->lo, box->hi, box->ghost, box->block, w, panel, scale, rhs, flux);
  return 0;
}
int orc_box_rhs_o4(void* L, const hc_box* box, const double* usph, double scale, double* rhs, double* const* flux) {
  o4BoxOperator(*static_cast<Level*>(L), box->lo, box->hi, box->ghost, box->block, usph, scale, rhs, flux);
  return 0;
}
void* orc_o4_level_create(void* L) { return new O4Level(*static_cast<Level*>(L)); }
void orc_o4_level_destroy(void* O) { delete static_cast<O4Level*>(O); }
int orc_o4_prepare(void* O, const double* ju, double* us, double t) { o4Prepare(*static_cast<O4Level*>(O), ju, us, t); return 0; }
int orc_o4_cartesian(void* O, const double* ju, double* cart) {
  const O4Level& o = *static_cast<O4Level*>(O);
  std::fill(cart, cart + (size_t)6 * 8 * o.Nc, 0.0);
  o4Cartesian(o, ju, cart);
  o4Seams(o, cart);
  return 0;
}
int orc_o4_seams(void* O, double* cart) { o4Seams(*static_cast<O4Level*>(O), cart); return 0; }
int orc_o4_box_native(void* O, const double* cart, const int* cart_lo, const int* cart_n, int block, double* us,
                      const int* us_lo, const int* us_n, double t) {
  o4BoxNative(*static_cast<O4Level*>(O), cart, cart_lo, cart_n, block, us, us_lo, us_n, t);
  return 0;
}
long orc_o4_sizes(void* O, long* out) {
  const O4Level& o = *static_cast<O4Level*>(O);
  out[0] = (long)o.Nv; out[1] = (long)o.Ng; out[2] = (long)o.Nc; out[3] = o.g; out[4] = o.ga;
  return 0;
}
int orc_o4_rhs(void* O, const double* us, double* k, double* reg, double weight) { o4Rhs(*static_cast<O4Level*>(O), us, k, reg, weight); return 0; }
int orc_o4_reflux(void* O, const double* reg, double* ju) { o4Reflux(*static_cast<O4Level*>(O), reg, ju); return 0; }
int orc_o4_rk4_step(void* O, double* ju, double dt, double t) { o4Rk4(*static_cast<O4Level*>(O), ju, dt, t); return 0; }
double orc_o4_inv_dt(void* O, const double* ju) { return o4InvDt(*static_cast<O4Level*>(O), ju); }
int orc_box_gravity_o4(void* L, const hc_box* box, const double* usph, double* rhs) {
  o4Gravity(*static_cast<Level*>(L), box->lo, box->hi, box->ghost, box->block, usph, rhs);
  return 0;
}
int orc_box_gravity(void* L, const hc_box* box, const double* w, double* rhs) {
  boxGravity(*static_cast<Level*>(L), box->lo, box->hi, box->ghost, box->block, w, rhs);
  return 0;
}
int orc_level_prepare(void* L, const double* ju, double* w, double t) { levelPrepare(*static_cast<Level*>(L), ju, w, t); return 0; }
int orc_level_rhs(void* L, const double* w, double* k) { levelRhs(*static_cast<Level*>(L), w, k); return 0; }
int orc_level_rk4_step(void* L, double* ju, double dt, double t) { levelRk4(*static_cast<Level*>(L), ju, dt, t); return 0; }
double orc_level_inv_dt(void* L, const double* ju) { return levelInvDt(*static_cast<Level*>(L), ju); }
int orc_level_valid(void* L, const double* ju) { return levelValid(*static_cast<Level*>(L), ju); }
int orc_level_init(void* L, const hc_init* in, double* ju) { levelInit(*static_cast<Level*>(L), *in, ju); return 0; }
// The CFL rate with the cone density floor of the inlet cones active at t
// (minimumConeBoundaryDensity, src/MHD_CME.H:1152-1160).
double orc_level_inv_dt_at(void* Lp, const double* ju, double t) {
  const Level& L = *static_cast<Level*>(Lp);
  double density = 0;
  for (const hc_cone& c : L.inlet)
    if (t >= c.insertion_time && t < c.end_time) density = density > 0 ? std::min(density, c.density) : c.density;
  return levelInvDt(L, ju, density);
}
int orc_level_set_inlet(void* L, const hc_cone* cones, int n) {
  static_cast<Level*>(L)->inlet.assign(cones, cones + n);
  return 0;
}
int orc_cone_prepare(const hc_cone_spec* spec, double inner_radius, hc_cone* out) {
  return conePrepare(*spec, inner_radius, *out);
}
// One cell of the insertion: 1 and delta[8] when `pos` lies in the cloud at `time`.
int orc_cone_cell(const hc_cone* c, double time, const double* pos, const double* ambient, double gamma,
                  double* delta) {
  const double shift = c->entry_shift + c->speed * 1e5 * (time - c->entry_time);
  return coneCellDelta(*c, shift, pos, ambient, gamma, delta) ? 1 : 0;
}
void orc_cme_schedule(const hc_cme_event* ev, int n, double time, double feeding, double* out) {
  cmeSchedule(ev, n, time, feeding, out[0], out[1]);
}
int orc_level_insert_cone(void* L, const hc_cone* c, double time, double* ju, double* stats) {
  levelInsertCone(*static_cast<Level*>(L), *c, time, ju, stats);
  return 0;
}

// Geometry export in the layout of hc_geometry_export.
long orc_geometry(void* Lp, int what, double* out) {
  const Level& L = *static_cast<Level*>(Lp);
  const int nr = L.nr, na = L.na;
  long n = 0;
  if (what == 0) {
    n = (long)(nr + 1) * 4;
    if (out)
      for (int i = 0; i <= nr; ++i) {
        const Radial& r = L.rad(i);
        out[4 * i + 0] = r.area0; out[4 * i + 1] = r.areaT; out[4 * i + 2] = r.Dr0; out[4 * i + 3] = r.vol;
      }
    return n;
  }
  if (what >= 1 && what <= 3) {
    int d = what - 1, ej = d == 1 ? 1 : 0, ek = d == 2 ? 1 : 0;
    n = 6L * (na + ek) * (na + ej) * 3;
    if (out) {
      long q = 0;
      for (int b = 0; b < 6; ++b)
        for (int k = 0; k < na + ek; ++k)
          for (int j = 0; j < na + ej; ++j) {
            const Frame& f = L.frames[d][L.frameIdx(b, j, k)];
            for (int r = 0; r < 3; ++r) out[q++] = f.normal[r];
          }
    }
    return n;
  }
  if (what == 4) {
    n = 6L * na * na;
    if (out) std::memcpy(out, L.det.data(), n * sizeof(double));
    return n;
  }
  if (what == 5) {
    n = 6L * na * na * 9;
    if (out) std::memcpy(out, L.detAA.data(), n * sizeof(double));
    return n;
  }
  return -1;
}

// Pointwise pieces for pinning against the reference headers.
int orc_roe8(const double* wl, const double* wr, double gamma, double ef, int check, double* out) {
  return roe8(out, wl, wr, gamma, ef, check != 0) ? 1 : 0;
}
void orc_rusanov(const double* wl, const double* wr, double gamma, double* out) { rusanov(out, wl, wr, gamma); }
void orc_frame(const double* normal, double* frame9, double* norm) {
  Frame f = secondOrderFrame(normal);
  for (int r = 0; r < 3; ++r) for (int s = 0; s < 3; ++s) frame9[3 * r + s] = f.f[r][s];
  *norm = f.norm;
}
void orc_face_flux(const double* l, const double* r, const double* normal, double radialArea, double gamma,
                   double ef, int roe, double* out) {
  Frame f = secondOrderFrame(normal);
  faceFlux(out, l, r, f, radialArea, gamma, ef, roe != 0);
}
void orc_plm(const double* mm, const double* m, const double* c, const double* p, int limiter, double* lo, double* hi) {
  plmFace(mm, m, c, p, limiter, lo, hi);
}
void orc_cart_prim(const double* in, double inverseJ, double gamma, double* out) {
  cartesianPrimitiveFromConserved(out, in, inverseJ, gamma);
}

// Fourth-order (Berta) pointwise pieces for pinning against the reference's
// own kernels.  States of 8 components, stencils laid out [cell][component].
void orc_berta_wenoz(const double* cells, double* wl, double* wr) {
  for (int c = 0; c < 8; ++c) {
    double in[6];
    for (int s = 0; s < 6; ++s) in[s] = cells[8 * s + c];
    wenozFace(in, wl[c], wr[c]);
  }
}
void orc_berta_weno3(const double* cells, double dx2, double* wl, double* wr) {
  for (int c = 0; c < 8; ++c) {
    double in[4];
    for (int s = 0; s < 4; ++s) in[s] = cells[8 * s + c];
    weno3Face(in, dx2, wl[c], wr[c]);
  }
}
void orc_berta_plm(const double* cells, double* wl, double* wr) {
  for (int c = 0; c < 8; ++c) {
    double in[4];
    for (int s = 0; s < 4; ++s) in[s] = cells[8 * s + c];
    plmFallbackFace(in, wl[c], wr[c]);
  }
}
// n = 4 or 6 values, normalised in place; returns the scale.
double orc_berta_normalize(double* v, int n) {
  if (n == 4) return normalizeStencil(*reinterpret_cast<double(*)[4]>(v));
  if (n == 6) return normalizeStencil(*reinterpret_cast<double(*)[6]>(v));
  return std::nan("");
}
// cells [7][8]: the cell, then the low and high neighbours in directions 0, 1, 2.
double orc_berta_jameson(const double* cells, double eta_d) {
  const double* lo[3] = {cells + 8, cells + 24, cells + 40};
  const double* hi[3] = {cells + 16, cells + 32, cells + 48};
  return jamesonRawFlag(cells, lo, hi, eta_d);
}
void orc_berta_avg_to_point(const double* avg, const double* lap, double theta, double* out) {
  for (int c = 0; c < 8; ++c) out[c] = avgToPoint(avg[c], lap[c], theta);
}
void orc_berta_flux_to_avg(const double* pt, const double* lap, double theta, double* out) {
  for (int c = 0; c < 8; ++c) out[c] = fluxPointToAvg(pt[c], lap[c], theta);
}
// The stencil-flag choice between the WENOZ states (wl4, wr4) and the
// fallback states, then the positivity clamp.
void orc_berta_select(const double* wl4, const double* wr4, const double* wlf, const double* wrf, double theta,
                      double* wl, double* wr) {
  const bool smooth = theta > 0.5;
  for (int c = 0; c < 8; ++c) {
    wl[c] = smooth ? wl4[c] : wlf[c];
    wr[c] = smooth ? wr4[c] : wrf[c];
    clampReconstructed(c, wl[c], wr[c]);
  }
}
// Matrices and fluxes laid out [column][cell], n columns, `size` cells.
void orc_berta_mapped_line(int n, int both, const double* m, const double* m1, const double* m2, const double* f,
                           const double* f1, const double* f2, int size, double* out) {
  for (int cell = 0; cell < size; ++cell) {
    double a[3], a1[3], a2[3], g[3], g1[3], g2[3];
    for (int col = 0; col < n; ++col) {
      const size_t q = (size_t)col * size + cell;
      a[col] = m[q]; a1[col] = m1[q]; a2[col] = m2[q]; g[col] = f[q]; g1[col] = f1[q]; g2[col] = f2[q];
    }
    out[cell] = mappedSum(n, both != 0, a, a1, a2, g, g1, g2);
  }
}
void orc_sph_to_prim_raw(const double* u, double* w) { sphToPrimRaw(u, w); }
void orc_prim_flux(const double* w, double ke, double me, double vb, double gamma, int c, double* f) {
  primFlux(f, w, ke, me, vb, gamma, c);
}
void orc_mapped_roe(const double* wl, const double* wr, const double* A9, double radialArea, int dir, double gamma,
                    double ef, double floor, double* out) {
  double A[3][3];
  for (int r = 0; r < 3; ++r) for (int s = 0; s < 3; ++s) A[r][s] = A9[3 * r + s];
  mappedRoe(out, wl, wr, A, radialArea, dir, gamma, ef, floor);
}
void orc_factored_roe(const double* wl, const double* wr, const double* A9, double radialArea, int dir, double gamma,
                      double ef, double floor, double* out) {
  double A[3][3];
  for (int r = 0; r < 3; ++r) for (int s = 0; s < 3; ++s) A[r][s] = A9[3 * r + s];
  factoredRoe(out, wl, wr, A, radialArea, dir, gamma, ef, floor);
}
int orc_usable_primitive(const double* w) { return usablePrimitive(w) ? 1 : 0; }
double orc_rho_floor() { return RHO00; }
}

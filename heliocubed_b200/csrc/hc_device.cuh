// Device-side pointwise physics of the second-order (PLM) MHD path, FP64.
//
// Each function restates one piece of the reference for sm_100a: scalar
// registers instead of 8x8 arrays, structural zeros of the Roe eigenvectors
// skipped (adding an exact zero term does not change an IEEE sum of finite
// values), matrix entries kept as the reference writes them.
#pragma once

#include <cuda_runtime.h>
#include <math.h>

#include "hc_common.h"

#define HC_DEV __device__ __forceinline__

namespace hc {

// Level kernels loop over flat indices below 2^31 (hc_ctx_create bounds
// the level size), so their loops and index splits run in 32-bit unsigned
// arithmetic.  takeMod returns t mod n and leaves t / n in t.
HC_DEV unsigned takeMod(unsigned& t, unsigned n) {
  const unsigned q = t / n, r = t - q * n;
  t = q;
  return r;
}
#define HC_LEVEL_LOOP(t, n) for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < (n); t += gridDim.x * blockDim.x)

HC_DEV double dmin(double a, double b) { return b < a ? b : a; }  // std::min
HC_DEV double dmax(double a, double b) { return a < b ? b : a; }  // std::max

// src/BoxOp_SecondOrder.H:7-37, one component.  LIM: 0 unlimited,
// 1 minmod (limiter 1 or 2), 3 monotonized central.
template <int LIM>
HC_DEV void plmComponent(double mm, double m, double c, double p, double& lo, double& hi) {
  const double a = m - mm, b = c - m, d = p - c;
  double sl = 0.5 * (a + b), sr = 0.5 * (b + d);
  if (LIM != 0) {
    sl = a * b <= 0 ? 0.0 : (a > 0 ? dmin(a, b) : dmax(a, b));
    sr = b * d <= 0 ? 0.0 : (b > 0 ? dmin(b, d) : dmax(b, d));
    if (LIM == 3) {
      if (a * b > 0) sl = (a > 0 ? 1.0 : -1.0) * dmin(0.5 * fabs(a + b), 2.0 * dmin(fabs(a), fabs(b)));
      if (b * d > 0) sr = (b > 0 ? 1.0 : -1.0) * dmin(0.5 * fabs(b + d), 2.0 * dmin(fabs(b), fabs(d)));
    }
  }
  lo = m + 0.5 * sl;
  hi = c - 0.5 * sr;
}

// Left state of a face from cells (i-2, i-1, i) only (the "lo" half of the
// reference's pair), with its complete-state fallback.
template <int LIM>
HC_DEV void plmLeft(const double* mm, const double* m, const double* c, double lo[8]) {
#pragma unroll
  for (int k = 0; k < NC; ++k) {
    const double a = m[k] - mm[k], b = c[k] - m[k];
    double sl = 0.5 * (a + b);
    if (LIM != 0) {
      sl = a * b <= 0 ? 0.0 : (a > 0 ? dmin(a, b) : dmax(a, b));
      if (LIM == 3 && a * b > 0) sl = (a > 0 ? 1.0 : -1.0) * dmin(0.5 * fabs(a + b), 2.0 * dmin(fabs(a), fabs(b)));
    }
    lo[k] = m[k] + 0.5 * sl;
  }
  if (!(lo[0] >= kRHO00 && lo[4] >= 0)) {
#pragma unroll
    for (int k = 0; k < NC; ++k) lo[k] = m[k];
  }
}

// Right state of a face from cells (i-1, i, i+1) only.
template <int LIM>
HC_DEV void plmRight(const double* m, const double* c, const double* p, double hi[8]) {
#pragma unroll
  for (int k = 0; k < NC; ++k) {
    const double b = c[k] - m[k], d = p[k] - c[k];
    double sr = 0.5 * (b + d);
    if (LIM != 0) {
      sr = b * d <= 0 ? 0.0 : (b > 0 ? dmin(b, d) : dmax(b, d));
      if (LIM == 3 && b * d > 0) sr = (b > 0 ? 1.0 : -1.0) * dmin(0.5 * fabs(b + d), 2.0 * dmin(fabs(b), fabs(d)));
    }
    hi[k] = c[k] - 0.5 * sr;
  }
  if (!(hi[0] >= kRHO00 && hi[4] >= 0)) {
#pragma unroll
    for (int k = 0; k < NC; ++k) hi[k] = c[k];
  }
}

// src/MHD_Roe8Wave.H:604-629.  invGm1 = 1/(gamma-1) replaces the division
// by (gamma-1) (one rounding of difference, inside the parity tolerance).
HC_DEV void rusanovDissipation(double out[8], const double* wl, const double* wr, double gamma, double invGm1) {
  constexpr double inv4Pi = 0.079577471545947667884441881686257181;
  double cl[8], cr[8], speed = 0.0;
#pragma unroll
  for (int side = 0; side < 2; ++side) {
    const double* w = side == 0 ? wl : wr;
    double* cs = side == 0 ? cl : cr;
    double v2 = 0.0, b2 = 0.0;
    cs[0] = w[0];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      v2 += w[1 + d] * w[1 + d];
      b2 += w[5 + d] * w[5 + d];
      cs[1 + d] = w[0] * w[1 + d];
      cs[5 + d] = w[5 + d];
    }
    cs[4] = w[4] * invGm1 + 0.5 * w[0] * v2 + 0.5 * inv4Pi * b2;
    speed = fmax(speed, fabs(w[1]) + sqrt((gamma * w[4] + inv4Pi * b2) / w[0]));
  }
#pragma unroll
  for (int c = 0; c < 8; ++c) out[c] = speed * (cr[c] - cl[c]);
}

// Right-eigenvector entry sp[r][k] of src/MHD_Roe8Wave.H:356-426 (0-based).
struct RoeEig {
  double Rho, alf, als, af, as, hyy, hzz, sih, cc, c, sqPiRho, sq2PiRho;
};

HC_DEV double roeRight(const RoeEig& e, int r, int k) {
  constexpr double s2 = 0.707106781186547524400844362104849039, two = 2.0;
  switch (r * 8 + k) {
    case 0 * 8 + 0: return 1.0;
    case 0 * 8 + 4: return e.Rho * e.alf;
    case 0 * 8 + 5: return e.Rho * e.alf;
    case 0 * 8 + 6: return e.Rho * e.als;
    case 0 * 8 + 7: return e.Rho * e.als;
    case 1 * 8 + 4: return e.alf * e.af;
    case 1 * 8 + 5: return -e.alf * e.af;
    case 1 * 8 + 6: return e.als * e.as;
    case 1 * 8 + 7: return -e.als * e.as;
    case 2 * 8 + 2: return -e.hzz * s2;
    case 2 * 8 + 3: return -e.hzz * s2;
    case 2 * 8 + 4: return -e.als * e.as * e.hyy * e.sih;
    case 2 * 8 + 5: return e.als * e.as * e.hyy * e.sih;
    case 2 * 8 + 6: return e.alf * e.af * e.hyy * e.sih;
    case 2 * 8 + 7: return -e.alf * e.af * e.hyy * e.sih;
    case 3 * 8 + 2: return e.hyy * s2;
    case 3 * 8 + 3: return e.hyy * s2;
    case 3 * 8 + 4: return -e.als * e.as * e.hzz * e.sih;
    case 3 * 8 + 5: return e.als * e.as * e.hzz * e.sih;
    case 3 * 8 + 6: return e.alf * e.af * e.hzz * e.sih;
    case 3 * 8 + 7: return -e.alf * e.af * e.hzz * e.sih;
    case 4 * 8 + 4: return e.alf * e.Rho * e.cc;
    case 4 * 8 + 5: return e.alf * e.Rho * e.cc;
    case 4 * 8 + 6: return e.als * e.Rho * e.cc;
    case 4 * 8 + 7: return e.als * e.Rho * e.cc;
    case 5 * 8 + 1: return 1.0;
    case 6 * 8 + 2: return e.hzz * e.sq2PiRho * e.sih;
    case 6 * 8 + 3: return -e.hzz * e.sq2PiRho * e.sih;
    case 6 * 8 + 4: return two * e.als * e.sqPiRho * e.c * e.hyy;
    case 6 * 8 + 5: return two * e.als * e.sqPiRho * e.c * e.hyy;
    case 6 * 8 + 6: return -two * e.alf * e.sqPiRho * e.c * e.hyy;
    case 6 * 8 + 7: return -two * e.alf * e.sqPiRho * e.c * e.hyy;
    case 7 * 8 + 2: return -e.hyy * e.sq2PiRho * e.sih;
    case 7 * 8 + 3: return e.hyy * e.sq2PiRho * e.sih;
    case 7 * 8 + 4: return two * e.als * e.sqPiRho * e.c * e.hzz;
    case 7 * 8 + 5: return two * e.als * e.sqPiRho * e.c * e.hzz;
    case 7 * 8 + 6: return -two * e.alf * e.sqPiRho * e.c * e.hzz;
    case 7 * 8 + 7: return -two * e.alf * e.sqPiRho * e.c * e.hzz;
    default: return 0.0;
  }
}

HC_DEV bool roeRightNonzero(int r, int k) {
  switch (k) {
    case 0: return r == 0;
    case 1: return r == 5;
    case 2: case 3: return r == 2 || r == 3 || r == 6 || r == 7;
    default: return r != 5;
  }
}

// src/MHD_Roe8Wave.H:16-600: D = |A|(U_R - U_L) with arithmetic averages,
// eight-wave entropy fix and (CHECK) the intermediate-state fan walk.
// Returns false where the reference requests the Rusanov fallback.
// roe8Body is inlined where the caller has registers to spare;
// roe8WaveDissipation is its out-of-line form.
template <bool CHECK>
__device__ __forceinline__ bool roe8Body(double out[8], const double* wl, const double* wr, double gamma, double del2,
                                         double invHg) {
  const double RhoL = wl[0], UL = wl[1], VL = wl[2], WL = wl[3], PGasL = wl[4], BXL = wl[5], BYL = wl[6], BZL = wl[7];
  const double RhoR = wr[0], UR = wr[1], VR = wr[2], WR = wr[3], PGasR = wr[4], BXR = wr[5], BYR = wr[6], BZR = wr[7];
  if (!(RhoL > 0.0 && RhoR > 0.0 && PGasL > 0.0 && PGasR > 0.0)) return false;
  constexpr double d_1_8PI = 0.039788735772973833942220940843128591, half = 0.5, zero = 0.0, four = 4.0;
  constexpr double d_SQRT_2 = 0.707106781186547524400844362104849039, d_1_4PI = 0.079577471545947667884441881686257181;
  constexpr double smallB = 1.0e-9, d_PI = 3.14159265358979323846264338327950288;
  constexpr double d_2PI = 6.28318530717958647692528676655900576;
  const double hgamma = gamma - 1.0;
  const double RUL = RhoL * UL, RVL = RhoL * VL, RWL = RhoL * WL;
  const double BxBL = d_1_8PI * (BXL * BXL + BYL * BYL + BZL * BZL);
  const double RUxUL = half * (RUL * UL + RVL * VL + RWL * WL);
  const double PL = PGasL + BxBL, EL = PGasL * invHg + RUxUL + BxBL, AL2 = gamma * PGasL / RhoL;
  const double RUR = RhoR * UR, RVR = RhoR * VR, RWR = RhoR * WR;
  const double BxBR = d_1_8PI * (BXR * BXR + BYR * BYR + BZR * BZR);
  const double RUxUR = half * (RUR * UR + RVR * VR + RWR * WR);
  const double PR = PGasR + BxBR, ER = PGasR * invHg + RUxUR + BxBR, AR2 = gamma * PGasR / RhoR;
  const double ccmi = AL2 > AR2 ? AR2 : AL2, ccma = AL2 > AR2 ? AL2 : AR2;
  const double Rho = half * (RhoL + RhoR), U = half * (UL + UR), V = half * (VL + VR), W = half * (WL + WR);
  const double BX = half * (BXL + BXR), BY = half * (BYL + BYR), BZ = half * (BZL + BZR), P = half * (PL + PR);
  const double BX2 = BX * BX, BYZ2 = BY * BY + BZ * BZ, BxBH = d_1_8PI * (BX2 + BYZ2);
  const double kk = half * (U * U + V * V + W * W);
  double cc = gamma * (P - BxBH) / Rho;
  const double bb = d_1_4PI * BX2 / Rho, b = sqrt(bb);
  if (cc < ccmi) cc = ccmi;
  if (cc > ccma) cc = ccma;
  if (!(cc > 0.0) || !isfinite(cc)) return false;
  const double c = sqrt(cc);
  double hyy, hzz, aaf, aas, af, as;
  if (BYZ2 < smallB * smallB) {
    hyy = d_SQRT_2;
    hzz = d_SQRT_2;
    if (bb > cc) { aaf = bb; aas = cc; af = b; as = c; }
    else { aaf = cc; aas = bb; af = c; as = b; }
  } else {
    const double hyz = sqrt(BYZ2);
    hyy = BY / hyz;
    hzz = BZ / hyz;
    const double szb = cc + (BxBH + BxBH) / Rho;
    const double h = sqrt(fmax(0.0, szb * szb - four * cc * bb));
    aas = half * (szb - h);
    if (aas <= zero) { aas = zero; as = zero; }
    else if (aas >= cc) { aas = cc; as = c; }
    else as = sqrt(aas);
    aaf = half * (szb + h);
    if (aaf <= cc) { aaf = cc; af = c; }
    else af = sqrt(aaf);
  }
  const double eig[8] = {U, U, U + b, U - b, U + af, U - af, U + as, U - as};
  const double eigmax = fabs(U) + fabs(V) + fabs(W) + af;
  const double del = del2 * eigmax, dell2 = del * del;
  const double dfs = aaf - aas;
  double alf, als;
  if (dfs < 1.0e-8) { alf = 1.0; als = zero; }
  else if ((cc - aas) <= zero) { alf = zero; als = 1.0; }
  else if ((aaf - cc) <= zero) { alf = 1.0; als = zero; }
  else { alf = sqrt((cc - aas) / dfs); als = sqrt((aaf - cc) / dfs); }
  const double sih = BX >= zero ? 1.0 : -1.0;
  double du[8] = {RhoL - RhoR, RUL - RUR, RVL - RVR, RWL - RWR, EL - ER, BXL - BXR, BYL - BYR, BZL - BZR};
  du[4] = -hgamma * (-kk * du[0] + U * du[1] + V * du[2] + W * du[3] - du[4] + (BX * du[5] + BY * du[6] + BZ * du[7]) * d_1_4PI);
  // The left-eigenvector entries divide by a few common factors; their
  // reciprocals are taken once (one rounding from the reference's
  // repeated divisions).
  const double iRho = 1.0 / Rho;
  du[1] = (-U * du[0] + du[1]) * iRho;
  du[2] = (-V * du[0] + du[2]) * iRho;
  du[3] = (-W * du[0] + du[3]) * iRho;
  const double sqPiRho = sqrt(d_PI * Rho), sq2PiRho = sqrt(d_2PI * Rho);
  const double icc = 1.0 / cc, iccRho = 1.0 / (cc * Rho), icSqPi = 1.0 / (c * sqPiRho), iSq2Pi = 1.0 / sq2PiRho;
  RoeEig e{Rho, alf, als, af, as, hyy, hzz, sih, cc, c, sqPiRho, sq2PiRho};
  // Left-eigenvector projections alpha_k = sum_c so[k][c] du[c]
  // (src/MHD_Roe8Wave.H:428-498, zeros skipped).
  double al[8];
  al[0] = du[0] + (-icc) * du[4];
  al[1] = du[5];
  al[2] = -hzz * d_SQRT_2 * du[2] + hyy * d_SQRT_2 * du[3] + half * hzz * sih * iSq2Pi * du[6] + -half * hyy * sih * iSq2Pi * du[7];
  al[3] = -hzz * d_SQRT_2 * du[2] + hyy * d_SQRT_2 * du[3] + -half * hzz * sih * iSq2Pi * du[6] + half * hyy * sih * iSq2Pi * du[7];
  al[4] = half * alf * af * icc * du[1] + -half * als * as * hyy * sih * icc * du[2] + -half * als * as * hzz * sih * icc * du[3] +
          half * alf * iccRho * du[4] + 0.25 * als * hyy * icSqPi * du[6] + 0.25 * als * hzz * icSqPi * du[7];
  al[5] = -half * alf * af * icc * du[1] + half * als * as * hyy * sih * icc * du[2] + half * als * as * hzz * sih * icc * du[3] +
          half * alf * iccRho * du[4] + 0.25 * als * hyy * icSqPi * du[6] + 0.25 * als * hzz * icSqPi * du[7];
  al[6] = half * als * as * icc * du[1] + half * alf * af * hyy * sih * icc * du[2] + half * alf * af * hzz * sih * icc * du[3] +
          half * als * iccRho * du[4] + -0.25 * alf * hyy * icSqPi * du[6] + -0.25 * alf * hzz * icSqPi * du[7];
  al[7] = -half * als * as * icc * du[1] + -half * alf * af * hyy * sih * icc * du[2] + -half * alf * af * hzz * sih * icc * du[3] +
          half * als * iccRho * du[4] + -0.25 * alf * hyy * icSqPi * du[6] + -0.25 * alf * hzz * icSqPi * du[7];
  if (CHECK) {
    // Walk the conservative wave fan in speed order (src/MHD_Roe8Wave.H:500-548).
    constexpr int order[8] = {5, 3, 7, 0, 1, 6, 2, 4};
    double s0 = RhoL, s1 = RUL, s2 = RVL, s3 = RWL, s4 = EL, s5 = BXL, s6 = BYL, s7 = BZL;
#pragma unroll
    for (int wave = 0; wave < 7; ++wave) {
      const int k = order[wave];
      const double amplitude = -al[k];
      double d[8];
#pragma unroll
      for (int r = 0; r < 8; ++r) d[r] = roeRightNonzero(r, k) ? amplitude * roeRight(e, r, k) : 0.0;
      const double d4 = kk * d[0] + Rho * (U * d[1] + V * d[2] + W * d[3]) + d[4] * invHg + d_1_4PI * (BX * d[5] + BY * d[6] + BZ * d[7]);
      const double d1 = U * d[0] + Rho * d[1], d2 = V * d[0] + Rho * d[2], d3 = W * d[0] + Rho * d[3];
      s0 += d[0]; s1 += d1; s2 += d2; s3 += d3; s4 += d4; s5 += d[5]; s6 += d[6]; s7 += d[7];
      if (eig[order[wave + 1]] > eig[k]) {
        if (!(s0 > 0.0) || !isfinite(s0)) return false;
        const double thermal = s4 - 0.5 * (s1 * s1 + s2 * s2 + s3 * s3) / s0 - d_1_8PI * (s5 * s5 + s6 * s6 + s7 * s7);
        if (!(thermal >= 0.0) || !isfinite(thermal)) return false;
      }
    }
  }
  // Entropy-fixed |lambda| (src/MHD_Roe8Wave.H:243-311) times alpha.
  double lu[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const double z = fabs(eig[q]);
    lu[q] = (z >= del ? z : half * (z * z + dell2) / del) * al[q];
  }
  double ra[8];
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    double s = 0.0;
    bool first = true;
#pragma unroll
    for (int k = 0; k < 8; ++k)
      if (roeRightNonzero(r, k)) {
        const double t = roeRight(e, r, k) * lu[k];
        s = first ? t : s + t;
        first = false;
      }
    ra[r] = s;
  }
  const double ra4 = ra[0] * kk + Rho * (U * ra[1] + V * ra[2] + W * ra[3]) + ra[4] * invHg + d_1_4PI * (BX * ra[5] + BY * ra[6] + BZ * ra[7]);
  out[0] = -ra[0];
  out[1] = -(U * ra[0] + Rho * ra[1]);
  out[2] = -(V * ra[0] + Rho * ra[2]);
  out[3] = -(W * ra[0] + Rho * ra[3]);
  out[4] = -ra4;
  out[5] = -ra[5];
  out[6] = -ra[6];
  out[7] = -ra[7];
  bool ok = true;
#pragma unroll
  for (int q = 0; q < 8; ++q) ok = ok && isfinite(out[q]);
  return ok;
}

template <bool CHECK>
__device__ __noinline__ bool roe8WaveDissipation(double out[8], const double* wl, const double* wr, double gamma,
                                                 double del2, double invHg) {
  return roe8Body<CHECK>(out, wl, wr, gamma, del2, invHg);
}

// src/MHD_SecondOrderFlux.H:34-74: local-frame MHD flux of both states,
// Roe (with Rusanov fallback) or Rusanov dissipation, rotated back and
// multiplied by radialArea*|adjA|.
template <bool ROE>
HC_DEV void secondOrderFaceFlux(double out[8], const double* l, const double* r, const FaceGeom& g, double radialArea,
                                double gamma, double invGm1, double entropy) {
  constexpr double inv4pi = 1.0 / (4.0 * kPi);
  double loc[2][8], flux[2][8];
#pragma unroll
  for (int side = 0; side < 2; ++side) {
    const double* s = side == 0 ? l : r;
    double* q = loc[side];
    q[0] = s[0];
    q[4] = s[4];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      q[1 + i] = g.f[3 * i] * s[1] + g.f[3 * i + 1] * s[2] + g.f[3 * i + 2] * s[3];
      q[5 + i] = g.f[3 * i] * s[5] + g.f[3 * i + 1] * s[6] + g.f[3 * i + 2] * s[7];
    }
    double v2 = 0, b2 = 0, vb = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      v2 += q[1 + i] * q[1 + i];
      b2 += q[5 + i] * q[5 + i];
      vb += q[1 + i] * q[5 + i];
    }
    const double pressure = q[4] + 0.5 * inv4pi * b2;
    const double energy = q[4] * invGm1 + 0.5 * q[0] * v2 + 0.5 * inv4pi * b2;
    double* f = flux[side];
    f[0] = q[0] * q[1];
    f[4] = (energy + pressure) * q[1] - inv4pi * q[5] * vb;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      f[1 + i] = q[0] * q[1] * q[1 + i] - inv4pi * q[5] * q[5 + i] + (i == 0 ? pressure : 0);
      f[5 + i] = q[1] * q[5 + i] - q[1 + i] * q[5];
    }
  }
  double diss[8];
  bool done = false;
  if (ROE) done = roe8WaveDissipation<true>(diss, loc[0], loc[1], gamma, entropy, invGm1);
  if (!done) rusanovDissipation(diss, loc[0], loc[1], gamma, invGm1);
  const double area = radialArea * g.norm;
  double num[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) num[c] = 0.5 * area * (flux[0][c] + flux[1][c] - diss[c]);
  out[0] = num[0];
  out[4] = num[4];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    out[1 + i] = g.f[i] * num[1] + g.f[3 + i] * num[2] + g.f[6 + i] * num[3];
    out[5 + i] = g.f[i] * num[5] + g.f[3 + i] * num[6] + g.f[6 + i] * num[7];
  }
}

// src/MHD_StateConversion.H:11-32 (no constant-background magnetic test).
HC_DEV void cartesianPrimitiveFromConserved(double out[8], const double in[8], double inverseJ, double gamma) {
  double u[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) u[c] = in[c] * inverseJ;
  const double rho = u[0] < kMP / 100 ? kMP / 100 : u[0];
  double kinetic = 0, magnetic = 0;
  out[0] = rho;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    out[1 + d] = u[1 + d] / rho;
    out[5 + d] = u[5 + d];
    kinetic += 0.5 * rho * out[1 + d] * out[1 + d];
    magnetic += u[5 + d] * u[5 + d] / (8 * kPi);
  }
  const double pressure = (gamma - 1.0) * (u[4] - kinetic - magnetic);
  out[4] = pressure < 0.0 ? 0.0 : pressure;
}

// Inner analytic wind, native conserved variables at Cartesian point X and
// time t (src/BoxOp_PreStage.H:7-47, f_radialoutflowIBCs).
HC_DEV void windConserved(double gam, double r_BC, double strength, const double X[3], double t, double u[8]) {
  const double r = sqrt(X[0] * X[0] + X[1] * X[1] + X[2] * X[2]);
  const double theta = atan2(sqrt(X[0] * X[0] + X[1] * X[1]), X[2]);
  const double phi = atan2(X[1], X[0]);
  const double p0 = 1.0e-7, rho0 = 700 * kMP, u0 = 500.0 * 1e5;
  const double rho = rho0 * pow(r_BC / r, 2.0);
  const double p = p0 * pow(r_BC / r, 2.0 * gam);
  const double carr_rot_time = 25.38 * 24 * 60 * 60;
  const double omega = 2.0 * kPi / carr_rot_time;
  const double phit = phi - omega * t;
  const double perturbationScale = strength / 100.0;
  const double sinTheta = sin(theta);
  const double angularPattern = pow(sinTheta, 5) * sin(5 * phit) + pow(sinTheta, 10) * sin(10 * phit);
  const double ur = u0 - perturbationScale * u0 / 3 * angularPattern;
  u[0] = rho;
  u[1] = ur * rho;
  u[2] = u[3] = u[5] = u[6] = u[7] = 0.0;
  const double umag = sqrt(u[1] * u[1]) / u[0];
  u[4] = p / (gam - 1.0) + 0.5 * u[0] * umag * umag + 0.0 / 8.0 / kPi;
}

// Native averages of one cell from fourth-order Cartesian averages
// (src/MHD_CachedCartesianConversion.H:65-124): c0 points at the cell's
// component 0 (neighbours j +- 1 at +-sj, k +- 1 at +-sk, components sc
// apart); cf at the cell's 27 conversion coefficients (<A>^-1, D1 <A>,
// D2 <A>), the neighbours' at +-cj, +-ck.
HC_DEV void o4NativeCore(const double* c0, long sj, long sk, long sc, const double* cf,
                         long cj, long ck, double out[8]) {
  out[0] = c0[0];
  out[4] = c0[4 * sc];
  const long nOff[4] = {sj, -sj, sk, -sk};
  const long cOff[4] = {cj, -cj, ck, -ck};
#pragma unroll
  for (int grp = 0; grp < 2; ++grp) {
    const int st = grp == 0 ? 1 : 5;
    const double* cs = c0 + st * sc;
    double q[4][3];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const double* I = cf + cOff[e];
      const double* x = cs + nOff[e];
      const double x0 = x[0];
      const double x1 = x[sc];
      const double x2 = x[2 * sc];
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        double v = 0.0;
        v += I[3 * r] * x0 * 1.0;
        v += I[3 * r + 1] * x1 * 1.0;
        v += I[3 * r + 2] * x2 * 1.0;
        q[e][r] = v;
      }
    }
    double d1[3], d2[3], corrected[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      d1[r] = 0.5 * (q[0][r] - q[1][r]);
      d2[r] = 0.5 * (q[2][r] - q[3][r]);
    }
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      double first = 0.0, second = 0.0;
#pragma unroll
      for (int s = 0; s < 3; ++s) {
        first += cf[9 + 3 * r + s] * d1[s] * (-1.0 / 12.0);
        second += cf[18 + 3 * r + s] * d2[s] * (-1.0 / 12.0);
      }
      double correction = 0.0;
      correction += first;
      correction += second;
      corrected[r] = cs[r * sc] + correction;
    }
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      double v = 0.0;
#pragma unroll
      for (int s = 0; s < 3; ++s) v += cf[3 * r + s] * corrected[s] * 1.0;
      out[st + r] = v;
    }
  }
}

}  // namespace hc

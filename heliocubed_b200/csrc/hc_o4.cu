// Fourth-order Berta pointwise-WENOZ operator on batched ghosted boxes,
// src/BoxOp_BertaCubedSphereImplem.H:1737-2076 with the Roe glue of
// src/BoxOp_RoeCubedSphere.H:29-145 and the Powell terms of
// src/BoxOp_DivBcleaning.H:35-172.  FP64.
//
// Kernels per evaluation: the detector and point values on the ghosted box
// G (cell arrays); per direction d the reconstruction on the face box
// F = G.extrude(d).grow(-3) and the Roe point dissipation (face arrays in
// the face scratch), then one fused face-chain kernel that takes tiles of
// the final faces through the flux average, mapped flux, radial products,
// final flux and divergence with its intermediates in shared memory; the
// Powell terms on a side stream.  Every intermediate covers the box the
// reference computes it on.
#include <cuda.h>
#include <cuda_runtime.h>
#include <math_constants.h>

#include <algorithm>
#include <cstdint>
#include <vector>

#include "hc_device.cuh"
#include "hc_level.h"

namespace hc {
namespace {

struct Box3 {
  int lo[3], hi[3];
  __host__ __device__ Box3 grow(int g) const { Box3 b = *this; for (int d = 0; d < 3; ++d) { b.lo[d] -= g; b.hi[d] += g; } return b; }
  __host__ __device__ Box3 growTrans(int d, int g) const {
    Box3 b = *this;
    for (int t = 0; t < 3; ++t) if (t != d) { b.lo[t] -= g; b.hi[t] += g; }
    return b;
  }
  __host__ __device__ Box3 extrude(int d) const { Box3 b = *this; b.hi[d] += 1; return b; }
  __host__ __device__ int n(int d) const { return hi[d] - lo[d] + 1; }
  __host__ __device__ long size() const { return (long)n(0) * n(1) * n(2); }
};

__host__ __device__ inline Reg regOf(const Box3& b) {
  Reg r;
  for (int d = 0; d < 3; ++d) { r.lo[d] = b.lo[d]; r.n[d] = b.n(d); }
  r.N = b.size();
  return r;
}

// Offset of (i, j, k) in an array laid out on region r.  Every array of a
// box holds fewer than 2^31 points per component (o4BatchCreate rejects
// larger boxes), so the offset is formed in 32-bit arithmetic, which the
// compiler shares between the neighbours of a stencil.
__device__ __forceinline__ long roff(const Reg& r, int i, int j, int k) {
  return (long)((i - r.lo[0]) + r.n[0] * ((j - r.lo[1]) + r.n[1] * (k - r.lo[2])));
}

// Offsets of the face arrays inside a box's face scratch (units of F.N).
enum FaceArr { F_WL = 0, F_WR = 8, F_FS = 16, F_QD = 24, F_THF = 32, F_PS = 33, F_BP = 34, F_BFLUX = 35,
               F_BPROD = 36, F_FA0 = 37, F_PA0 = 45 };  // F_FA0, F_PA0: direction 0's averages (TMA path)

struct Ctx {
  O4Args a;
  int d;
  Box3 V, G, GR, GD, F, F1, F2, V0, V1, V2;
  Reg gr, fr, v1r, v2r, vr;
};

// Regions the operator's kernels loop over (host and device agree through
// this one table): the work lists of a batch are built from it.
enum RegionId { RG_G = 0, RG_GR, RG_F, RG_PB, RG_F1, RG_V0, RG_V, RG_PF, RG_PP, RG_V1, RG_V2, RG_COUNT };
__host__ __device__ inline Box3 regionOf(const Ctx& c, int id) {
  switch (id) {
    case RG_G: return c.G;
    case RG_GR: return c.GR;
    case RG_F: return c.F;
    case RG_PB: return c.V0.growTrans(c.d, 1);
    case RG_F1: return c.F1;
    case RG_V0: return c.V0;
    case RG_V: return c.V;
    case RG_PF: return c.V1.extrude(c.d).growTrans(c.d, 1);
    case RG_PP: return c.V1.extrude(c.d);
    case RG_V1: return c.V1;
    default: return c.V2;
  }
}

// One CTA's work: flat points begin, begin + stride, ... below end (each
// thread adds its index) of one region of box `box`.
struct WorkChunk {
  int box, stride;
  long begin, end;
};
// Points per CTA (128 threads) of a work list: its total points over about
// 148 x 32 CTAs, rounded up to whole passes of the CTA and held within
// [128, 1024], so one launch has as many CTAs whatever the box sizes.
inline long chunkPoints(long total) {
  const long target = (total + 148L * 32 - 1) / (148L * 32);
  const long c = ((target + 127) / 128) * 128;
  return c < 128 ? 128 : c > 1024 ? 1024 : c;
}

// The box the face arrays of every direction are laid out on: the face
// boxes G.extrude(d).grow(-3) together, its radial extent rounded up to an
// even count so that a radial row of doubles spans a multiple of 16 bytes
// (the strides a TMA tensor map accepts).
Box3 faceBox(const Box3& G) {
  Box3 FB = G.grow(-3);
  for (int q = 0; q < 3; ++q) FB.hi[q] += 1;
  if (FB.n(0) & 1) FB.hi[0] += 1;
  return FB;
}

Ctx makeCtx(const O4Args& a, int d) {
  Ctx c;
  c.a = a;
  c.d = d;
  // direction 1 keeps its face arrays apart, so its pass can run beside the
  // passes of directions 0 and 2
  if (d == 1) c.a.face = a.face2;
  for (int q = 0; q < 3; ++q) { c.V.lo[q] = a.vlo[q]; c.V.hi[q] = a.vhi[q]; }
  c.G = c.V.grow(a.ghost);
  c.GR = c.G.grow(-1);
  c.GD = c.G.grow(-2);
  c.F = c.G.extrude(d).grow(-3);
  c.F1 = c.F.growTrans(d, -1);
  c.F2 = c.F1.growTrans(d, -1);
  c.V0 = c.V.extrude(d);
  c.V1 = c.V.grow(1);
  c.V2 = c.V.grow(2);
  c.gr = regOf(c.G);
  // face scratch is laid out on the largest face box over the directions
  c.fr = regOf(faceBox(c.G));
  c.v1r = regOf(c.V1);
  c.v2r = regOf(c.V2);
  c.vr = a.rr.N ? a.rr : regOf(c.V);
  return c;
}

// ---- geometry access -------------------------------------------------------
__device__ __forceinline__ const double* faceRec(const O4Geo& g, int block, int d, int j, int k) {
  const long n = g.na + 2 * g.ext + 1;
  return g.face + ((((long)block * 3 + d) * n + (k + g.ext)) * n + (j + g.ext)) * kO4FaceRec;
}
__device__ __forceinline__ const double* roeRec(const O4Geo& g, int block, int d, int j, int k) {
  const long n = g.na + 2 * g.ext + 1;
  return g.frames + ((((long)block * 3 + d) * n + (k + g.ext)) * n + (j + g.ext)) * kO4RoeRec;
}
__device__ __forceinline__ const double* cellBasis(const O4Geo& g, int block, int j, int k) {
  const long n = g.na + 2 * g.ext + 1;
  return g.cell + (((long)block * n + (k + g.ext)) * n + (j + g.ext)) * 9;
}
__device__ __forceinline__ double4 radialRow(const O4Geo& g, int i) { return g.radial[i + kO4Rad]; }
__device__ __forceinline__ double adjDr(const O4Geo& g, int d, int i) {
  const double4 r = radialRow(g, i);
  return d == 0 ? r.x : r.y;
}
__device__ __forceinline__ double radialPoint(const O4Geo& g, int d, int i) {
  if (d == 0) return adjDr(g, 0, i);
  const double a = adjDr(g, d, i);
  return a - (1.0 / 24.0) * (adjDr(g, d, i + 1) - 2.0 * a + adjDr(g, d, i - 1));
}

// ---- pointwise pieces -----------------------------------------------------
// Divisions by 4 pi and 8 pi are multiplications by the rounded reciprocals
// (a one-ulp difference from the reference's x / 8.0 / M_PI).
constexpr double kInv4Pi = 0.25 / kPi, kInv8Pi = 0.125 / kPi;
// f_sphToPrim + energies + pressure (src/BoxOp_BertaCubedSphereImplem.H:212-340)
__device__ __forceinline__ void sphToPrim(const double u[8], const double* A, double gamma, double w[8]) {
  w[0] = dmax(u[0], kRHO00);
  w[1] = u[1] / w[0];
  w[2] = u[2] / w[0];
  w[3] = u[3] / w[0];
  w[4] = u[4];
  w[5] = u[5]; w[6] = u[6]; w[7] = u[7];
  double ke = 0., me = 0.;
#pragma unroll
  for (int d0 = 0; d0 < 3; ++d0) {
    const double vc = A[3 * d0] * w[1] + A[3 * d0 + 1] * w[2] + A[3 * d0 + 2] * w[3];
    const double bc = A[3 * d0] * w[5] + A[3 * d0 + 1] * w[6] + A[3 * d0 + 2] * w[7];
    ke += vc * vc / 2;
    me += bc * bc * kInv8Pi;
  }
  ke *= w[0];
  w[4] = (w[4] - ke - me) * (gamma - 1.0);
  if (w[4] < 0.0) w[4] = 0.0;
}

// EnergyW (src/BoxOp_Utilities.H:447-520)
__device__ __forceinline__ void energyW(const double w[8], const double* A, double& ke, double& me, double& vb) {
  ke = 0.; me = 0.; vb = 0.;
#pragma unroll
  for (int d0 = 0; d0 < 3; ++d0) {
    const double vc = A[3 * d0] * w[1] + A[3 * d0 + 1] * w[2] + A[3 * d0 + 2] * w[3];
    const double bc = A[3 * d0] * w[5] + A[3 * d0 + 1] * w[6] + A[3 * d0 + 2] * w[7];
    ke += vc * vc;
    me += bc * bc * kInv8Pi;
    vb += vc * bc;
  }
  ke *= w[0] * .5;
}

// f_primflux (src/BoxOp_EulerCubedSphere.H:195-225)
__device__ __forceinline__ void primFlux(double f[8], const double w[8], double ke, double me, double vb, double gamma, int c) {
  const int c1 = (c + 1) % 3, c2 = (c + 2) % 3;
  const double velnorm = w[c + 1], veltan1 = w[c1 + 1], veltan2 = w[c2 + 1];
  const double bnorm = w[c + 5], btan1 = w[c1 + 5], btan2 = w[c2 + 5];
  f[0] = w[0] * velnorm;
  f[c + 1] = f[0] * velnorm - bnorm * bnorm * kInv4Pi;
  f[c1 + 1] = f[0] * veltan1 - bnorm * btan1 * kInv4Pi;
  f[c2 + 1] = f[0] * veltan2 - bnorm * btan2 * kInv4Pi;
  f[4] = (2.0 * me + ke + w[4] * gamma / (gamma - 1.0)) * velnorm - bnorm * vb * kInv4Pi;
  f[5] = velnorm * w[5] - w[1] * bnorm;
  f[6] = velnorm * w[6] - w[2] * bnorm;
  f[7] = velnorm * w[7] - w[3] * bnorm;
}

// bertaNormalizeWenoStencil (:747-773)
template <int N>
__device__ __forceinline__ double normalizeStencil(double (&v)[N]) {
  double scale = 0.0;
#pragma unroll
  for (int i = 0; i < N; ++i) scale = dmax(scale, fabs(v[i]));
  if (scale == 0.0) {
    for (int i = 0; i < N; ++i) if (v[i] != 0.0) return v[i];
    return scale;
  }
  if (scale > 0.0) {
    if (scale >= 2.2250738585072014e-308) {
      const double inverse = 1.0 / scale;
#pragma unroll
      for (int i = 0; i < N; ++i) v[i] *= inverse;
    } else {
      for (int i = 0; i < N; ++i) v[i] /= scale;
    }
  }
  return scale;
}

__device__ __forceinline__ void wenozSide(double m2, double m1, double c0, double p1, double p2, double& num,
                                          double& den) {
  // a_k = d_k (1 + tau / D_k), D_k = beta_k + eps; the state is
  // sum a_k q_k / sum a_k = num / den with a_k replaced by the proportional
  // d_k (D_k + tau) prod_{j != k} D_j (no division here).
  const double eps = 1.0e-40, d0 = 1.0 / 16.0, d1 = 5.0 / 8.0, d2 = 5.0 / 16.0;
  const double q0 = (3.0 * m2 - 10.0 * m1 + 15.0 * c0) * 0.125;
  const double q1 = (-m1 + 6.0 * c0 + 3.0 * p1) * 0.125;
  const double q2 = (3.0 * c0 + 6.0 * p1 - p2) * 0.125;
  const double b0a = m2 - 2.0 * m1 + c0, b0b = m2 - 4.0 * m1 + 3.0 * c0;
  const double b1a = m1 - 2.0 * c0 + p1, b1b = m1 - p1;
  const double b2a = c0 - 2.0 * p1 + p2, b2b = 3.0 * c0 - 4.0 * p1 + p2;
  const double beta0 = (13.0 / 12.0) * b0a * b0a + 0.25 * b0b * b0b;
  const double beta1 = (13.0 / 12.0) * b1a * b1a + 0.25 * b1b * b1b;
  const double beta2 = (13.0 / 12.0) * b2a * b2a + 0.25 * b2b * b2b;
  const double tau5 = fabs(beta0 - beta2);
  const double D0 = beta0 + eps, D1 = beta1 + eps, D2 = beta2 + eps;
  const double w0 = d0 * (D0 + tau5) * (D1 * D2);
  const double w1 = d1 * (D1 + tau5) * (D0 * D2);
  const double w2 = d2 * (D2 + tau5) * (D0 * D1);
  num = w0 * q0 + w1 * q1 + w2 * q2;
  den = w0 + w1 + w2;
}

// f_wenoz_pointwise_faceF (:782-878), one component, cells W[i-3..i+2].
__device__ __forceinline__ void wenozFace(const double in[6], double& L, double& R) {
  double v[6] = {in[0], in[1], in[2], in[3], in[4], in[5]};
  const double scale = normalizeStencil(v);
  if (scale == 0.0) { L = R = 0.0; return; }
  // Both sides' quotients from one division: nl / dl = nl dr / (dl dr).
  // On normalised stencils (|v| <= 1) every weight lies in [6e-122, 5e4], so
  // the product of the denominators neither underflows nor overflows.
  double nl, dl, nr, dr;
  wenozSide(v[0], v[1], v[2], v[3], v[4], nl, dl);
  wenozSide(v[5], v[4], v[3], v[2], v[1], nr, dr);
  const double inv = 1.0 / (dl * dr);
  L = scale * (nl * dr * inv);
  R = scale * (nr * dl * inv);
}

// f_weno3_pointwise_faceF (:881-946), one component, cells W[i-2..i+1].
__device__ __forceinline__ void weno3Face(const double in[4], double dx2, double& L, double& R) {
  // a_k = d_k (1 + tau / (beta_k + eps)) with one division per side, as in wenozSide.
  const double d0 = 3.0 / 4.0, d1 = 1.0 / 4.0, eps = dx2;
  double v[4] = {in[0], in[1], in[2], in[3]};
  const double scale = normalizeStencil(v);
  if (scale == 0.0) { L = R = 0.0; return; }
  {
    const double vm1 = v[0], v0 = v[1], vp1 = v[2];
    const double Dm = v0 - vm1, Dp = vp1 - v0;
    const double tau = (Dp - Dm) * (Dp - Dm), B0 = Dp * Dp + eps, B1 = Dm * Dm + eps;
    const double w0 = d0 * (B0 + tau) * B1, w1 = d1 * (B1 + tau) * B0;
    const double q0 = 0.5 * (vp1 + v0), q1 = 0.5 * (-vm1 + 3.0 * v0);
    L = scale * ((w0 * q0 + w1 * q1) / (w0 + w1));
  }
  {
    const double rm1 = v[3], r0 = v[2], rp1 = v[1];
    const double Dm = r0 - rm1, Dp = rp1 - r0;
    const double tau = (Dp - Dm) * (Dp - Dm), B0 = Dp * Dp + eps, B1 = Dm * Dm + eps;
    const double w0 = d0 * (B0 + tau) * B1, w1 = d1 * (B1 + tau) * B0;
    const double q0 = 0.5 * (rp1 + r0), q1 = 0.5 * (-rm1 + 3.0 * r0);
    R = scale * ((w0 * q0 + w1 * q1) / (w0 + w1));
  }
}

__device__ __forceinline__ double minmod3(double a, double b, double c) {
  if (a > 0.0 && b > 0.0 && c > 0.0) return dmin(a, dmin(b, c));
  if (a < 0.0 && b < 0.0 && c < 0.0) return dmax(a, dmax(b, c));
  return 0.0;
}

// f_plm_pointwise_faceF (:949-991), one component, cells W[i-2..i+1].
__device__ __forceinline__ void plmFallbackFace(const double in[4], double& L, double& R) {
  const double theta = 1.5;
  const double dm = in[1] - in[0], dp = in[2] - in[1], dc = 0.5 * (in[2] - in[0]);
  L = in[1] + 0.5 * minmod3(theta * dm, dc, theta * dp);
  const double rdm = in[2] - in[1], rdp = in[3] - in[2], rdc = 0.5 * (in[3] - in[1]);
  R = in[2] - 0.5 * minmod3(theta * rdm, rdc, theta * rdp);
}

__device__ __forceinline__ bool usablePrimitive(const double w[8]) {
  bool ok = true;
#pragma unroll
  for (int c = 0; c < 8; ++c) ok = ok && isfinite(w[c]);
  return ok && w[0] >= kRHO00 && w[4] >= 0.0;
}

// mappedRoe8WaveDissipation + factoredRoe8WaveDissipation (src/MHD_Roe8Wave.H:634-740)
// with the face's frame from the Roe frame table R (kO4RoeRec): the states
// are rotated into the frame, the 8-wave dissipation (Rusanov where the fan
// check fails) is taken there, rotated back, scaled by the face area and
// mapped through adj A / det A.  The frame is read again after the solver
// (roeLoad2 is not merged with the first read), so it does not occupy
// registers while the solver runs.
__device__ __forceinline__ double2 roeLoad2(const double* p) {
  double2 v;
  asm volatile("ld.global.nc.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
  return v;
}

__device__ __forceinline__ void factoredRoe(double out[8], const double* wl, const double* wr, const double* A,
                                            const double* __restrict__ R, double radialArea, double gamma,
                                            double invGm1, double entropy) {
  double loc[2][8];
  {
    double f[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) f[q] = R[q];
#pragma unroll
    for (int side = 0; side < 2; ++side) {
      const double* w = side == 0 ? wl : wr;
      loc[side][0] = fmax(w[0], kRHO00);
      loc[side][4] = fmax(w[4], 0.0);
      double vC[3], bC[3];
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        vC[i] = A[3 * i] * w[1] + A[3 * i + 1] * w[2] + A[3 * i + 2] * w[3];
        bC[i] = A[3 * i] * w[5] + A[3 * i + 1] * w[6] + A[3 * i + 2] * w[7];
      }
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        loc[side][1 + r] = f[3 * r] * vC[0] + f[3 * r + 1] * vC[1] + f[3 * r + 2] * vC[2];
        loc[side][5 + r] = f[3 * r] * bC[0] + f[3 * r + 1] * bC[1] + f[3 * r + 2] * bC[2];
      }
    }
  }
  double diss[8];
  if (!roe8Body<true>(diss, loc[0], loc[1], gamma, entropy, invGm1))
    rusanovDissipation(diss, loc[0], loc[1], gamma, invGm1);
  double g[22];
#pragma unroll
  for (int q = 0; q < 11; ++q) {
    const double2 v = roeLoad2(R + 2 * q);
    g[2 * q] = v.x;
    g[2 * q + 1] = v.y;
  }
  const double area = radialArea * g[9];
  double mapped[8];
  mapped[0] = area * diss[0];
  mapped[4] = area * diss[4];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    mapped[1 + i] = area * g[i] * diss[1] + area * g[3 + i] * diss[2] + area * g[6 + i] * diss[3];
    mapped[5 + i] = area * g[i] * diss[5] + area * g[3 + i] * diss[6] + area * g[6 + i] * diss[7];
  }
  const double* adj = g + 10;
  const double invDet = g[19], invDet2 = g[20];
  out[0] = mapped[0] * invDet;
  out[4] = mapped[4] * invDet;
#pragma unroll
  for (int dd = 0; dd < 3; ++dd) {
    out[1 + dd] = (adj[3 * dd] * mapped[1] + adj[3 * dd + 1] * mapped[2] + adj[3 * dd + 2] * mapped[3]) * invDet2;
    out[5 + dd] = (adj[3 * dd] * mapped[5] + adj[3 * dd + 1] * mapped[6] + adj[3 * dd + 2] * mapped[7]) * invDet2;
  }
}

// ---- stencils on scratch arrays --------------------------------------------
struct View {
  const double* p;
  Reg r;
  __device__ double operator()(int c, int i, int j, int k) const { return p[c * r.N + roff(r, i, j, k)]; }
};


__device__ __forceinline__ double lapFace(const View& f, int c, int d, int i, int j, int k) {
  const int t1 = d == 0 ? 1 : 0, t2 = d == 2 ? 1 : 2;
  int a[3] = {i, j, k}, b[3] = {i, j, k}, e[3] = {i, j, k}, g[3] = {i, j, k};
  a[t1] -= 1; b[t1] += 1; e[t2] -= 1; g[t2] += 1;
  return (f(c, a[0], a[1], a[2]) + f(c, b[0], b[1], b[2])) + (f(c, e[0], e[1], e[2]) + f(c, g[0], g[1], g[2])) -
         4.0 * f(c, i, j, k);
}

__device__ __forceinline__ double cdiff(const View& f, int c, int t, int i, int j, int k) {
  int a[3] = {i, j, k}, b[3] = {i, j, k};
  a[t] += 1; b[t] -= 1;
  return 0.5 * f(c, a[0], a[1], a[2]) - 0.5 * f(c, b[0], b[1], b[2]);
}

__device__ __forceinline__ double lapCell(const View& f, int c, int i, int j, int k) {
  return (f(c, i - 1, j, k) + f(c, i + 1, j, k)) + (f(c, i, j - 1, k) + f(c, i, j + 1, k)) +
         (f(c, i, j, k - 1) + f(c, i, j, k + 1)) - 6.0 * f(c, i, j, k);
}

__device__ __forceinline__ double faceProd(double f4, double g4, double df0, double dg0, double df1, double dg1) {
  double value = 0.0;
  value += df0 * dg0 * (1.0 / 12.0);
  value += df1 * dg1 * (1.0 / 12.0);
  value += f4 * g4 * 1.0;
  return value;
}


// Thread -> (i, j, k) over the chunk's points of region b (flat index,
// radial fastest) of the chunk's box; the end is clamped to the region.
// Regions hold fewer than 2^31 points (o4BatchCreate rejects larger boxes),
// so the index split runs in 32-bit unsigned arithmetic: two hardware-sized
// divisions per point instead of three 64-bit ones.
template <class F>
__device__ __forceinline__ void forRegion(const Box3& b, const WorkChunk& w, F f) {
  const unsigned n0 = (unsigned)b.n(0), n1 = (unsigned)b.n(1);
  const unsigned n = n0 * n1 * (unsigned)b.n(2);
  const unsigned end = w.end < (long)n ? (unsigned)w.end : n;
  for (unsigned t = (unsigned)w.begin + threadIdx.x; t < end; t += (unsigned)w.stride) {
    const unsigned q = t / n0, kk = q / n1;
    const int i = b.lo[0] + (int)(t - q * n0);
    const int j = b.lo[1] + (int)(q - kk * n1);
    const int k = b.lo[2] + (int)kk;
    f(0, i, j, k);
  }
}

// Roe dissipation unless the device flag switches a Roe context to Rusanov
// (the CME insertion window, exec/main.cpp:406-420).
__device__ __forceinline__ bool roeNow(const O4Geo& G) { return G.roe && !(G.rusanov && *G.rusanov); }

// ---- kernels ------------------------------------------------------------------
// 1. detector primitives of the averages, V(<U>) (:1776).
__global__ void o4PrimAvgKernel(const Ctx* __restrict__ tab, const RegArgs rg, const WorkChunk* __restrict__ wk) {
  const WorkChunk wc = wk[blockIdx.x];
  const Ctx& c = tab[wc.box * 3 + 0];
  const O4Args& a = c.a;
  forRegion(c.G, wc, [&](int b, int i, int j, int k) {
    double u[8], w[8];
    const double* U = a.U + b * a.uStride + roff(a.ur, i, j, k);
#pragma unroll
    for (int q = 0; q < 8; ++q) u[q] = U[q * a.ur.N];
    sphToPrim(u, cellBasis(a.G, a.block0 + b, j, k), a.G.gamma, w);
    double* W = a.WA + (long)b * 8 * c.gr.N + roff(c.gr, i, j, k);
#pragma unroll
    for (int q = 0; q < 8; ++q) W[q * c.gr.N] = w[q];
    // the Powell accumulator -J div B starts at zero on V1
    if (a.G.powell && i >= c.V1.lo[0] && i <= c.V1.hi[0] && j >= c.V1.lo[1] && j <= c.V1.hi[1] && k >= c.V1.lo[2] &&
        k <= c.V1.hi[2])
      a.mj[(long)b * c.v1r.N + roff(c.v1r, i, j, k)] = 0.0;
  });
}

__device__ __forceinline__ double magp(const double* W, long N, long o) {
  const double bx = W[5 * N + o], by = W[6 * N + o], bz = W[7 * N + o];
  return 0.5 * (bx * bx + by * by + bz * bz);
}
__device__ __forceinline__ double eta1(double qm, double q0, double qp) {
  const double num = fabs(qp - 2.0 * q0 + qm);
  const double den = fabs(qp) + 2.0 * fabs(q0) + fabs(qm) + 1.0e-40;
  return num / den;
}

// 2. raw Jameson flag on G.grow(-1) (:347-402).
__global__ void o4ThetaRawKernel(const Ctx* __restrict__ tab, const RegArgs rg, const WorkChunk* __restrict__ wk) {
  const WorkChunk wc = wk[blockIdx.x];
  const Ctx& c = tab[wc.box * 3 + 0];
  const O4Args& a = c.a;
  forRegion(c.GR, wc, [&](int b, int i, int j, int k) {
    const double* W = a.WA + (long)b * 8 * c.gr.N;
    const long N = c.gr.N, o = roff(c.gr, i, j, k);
    double et[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      int m[3] = {i, j, k}, p[3] = {i, j, k};
      m[d] -= 1; p[d] += 1;
      const long om = roff(c.gr, m[0], m[1], m[2]), op = roff(c.gr, p[0], p[1], p[2]);
      const double er = eta1(W[om], W[o], W[op]);
      const double ep = eta1(W[4 * N + om], W[4 * N + o], W[4 * N + op]);
      const double em = eta1(magp(W, N, om), magp(W, N, o), magp(W, N, op));
      et[d] = dmax(er, dmax(ep, em));
    }
    const double eta = sqrt(et[0] * et[0] + et[1] * et[1] + et[2] * et[2]);
    a.thr[(long)b * N + o] = eta < a.G.eta_d ? 1.0 : 0.0;
  });
}

// 3. dilated theta (0 outside G.grow(-2)), theta-aware average-to-point and
// point primitives on G (:404-507, 696-741, 212-275).
__global__ void o4PointKernel(const Ctx* __restrict__ tab, const RegArgs rg, const WorkChunk* __restrict__ wk) {
  const WorkChunk wc = wk[blockIdx.x];
  const Ctx& c = tab[wc.box * 3 + 0];
  const O4Args& a = c.a;
  forRegion(c.G, wc, [&](int b, int i, int j, int k) {
    const long N = c.gr.N, o = roff(c.gr, i, j, k);
    const double* R = a.thr + (long)b * N;
    double t = 0.0;
    const bool inD = i >= c.GD.lo[0] && i <= c.GD.hi[0] && j >= c.GD.lo[1] && j <= c.GD.hi[1] && k >= c.GD.lo[2] &&
                     k <= c.GD.hi[2];
    if (inD) {
      t = R[o];
      t = dmin(t, R[roff(c.gr, i - 1, j, k)]);
      t = dmin(t, R[roff(c.gr, i + 1, j, k)]);
      t = dmin(t, R[roff(c.gr, i, j - 1, k)]);
      t = dmin(t, R[roff(c.gr, i, j + 1, k)]);
      t = dmin(t, R[roff(c.gr, i, j, k - 1)]);
      t = dmin(t, R[roff(c.gr, i, j, k + 1)]);
    }
    const bool inner = i >= c.GR.lo[0] && i <= c.GR.hi[0] && j >= c.GR.lo[1] && j <= c.GR.hi[1] &&
                       k >= c.GR.lo[2] && k <= c.GR.hi[2];
    View U{a.U + b * a.uStride, a.ur};
    double u[8], w[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) u[q] = (inner && t > 0.5) ? U(q, i, j, k) - lapCell(U, q, i, j, k) * (1.0 / 24.0) : U(q, i, j, k);
    sphToPrim(u, cellBasis(a.G, a.block0 + b, j, k), a.G.gamma, w);
    double* W = a.WP + (long)b * 8 * N + o;
#pragma unroll
    for (int q = 0; q < 8; ++q) W[q * N] = w[q];
    // stored last: a store ahead of the state loads would hold them back
    // until the dilation's loads return
    a.th[(long)b * N + o] = t;
  });
}

__device__ __forceinline__ double* faceArr(const Ctx& c, int b, int arr) {
  return c.a.face + ((long)b * kO4FaceArrays + arr) * c.fr.N;
}
__device__ __forceinline__ View faceView(const Ctx& c, int b, int arr) { return View{faceArr(c, b, arr), c.fr}; }
template <int D>
__device__ __forceinline__ const double* faceBasis(const Ctx& c, int b, int j, int k) {
  return D == 0 ? cellBasis(c.a.G, c.a.block0 + b, j, k) : faceRec(c.a.G, c.a.block0 + b, D, j, k) + 13;
}

// 4. reconstruction (WENOZ / WENO3 / PLM with clamps), Roe repair, energies,
// point flux sum, total-pressure sum, centred normal B, Rusanov jump (F).
template <int D, int MB>
__global__ void __launch_bounds__(128, MB) o4FaceReconKernel(const Ctx* __restrict__ tab, const RegArgs rg, const WorkChunk* __restrict__ wk) {
  const WorkChunk wc = wk[blockIdx.x];
  const Ctx& c = tab[wc.box * 3 + D];
  const O4Args& a = c.a;
  constexpr int d = D;
  const double dx2 = a.G.dx[d] * a.G.dx[d];
  forRegion(c.F, wc, [&](int b, int i, int j, int k) {
    const long NG = c.gr.N, NF = c.fr.N;
    const double* th = a.th + (long)b * NG;
    const double* WP = a.WP + (long)b * 8 * NG;
    const double* WA = a.WA + (long)b * 8 * NG;
    long cell[6];
#pragma unroll
    for (int s = -3; s <= 2; ++s) {
      int q[3] = {i, j, k};
      q[d] += s;
      cell[s + 3] = roff(c.gr, q[0], q[1], q[2]);
    }
    const long fo = roff(c.fr, i, j, k);
    double thF = dmin(th[cell[2]], th[cell[3]]);
    double value = th[cell[0]];
    value = dmin(value, th[cell[1]]);
    value = dmin(value, th[cell[2]]);
    value = dmin(value, th[cell[3]]);
    value = dmin(value, th[cell[4]]);
    const double thR = dmin(value, th[cell[5]]);
    const bool smooth = thR > 0.5;
    // one copy of the reconstruction code for the eight components (a rolled
    // loop; the states go through this thread's shared-memory column)
    __shared__ double sLR[16][128];
    // the next component's six cells are loaded while this one is
    // reconstructed (all six cells lie in G for every face of F)
    double nx[6];
#pragma unroll
    for (int s = 0; s < 6; ++s) nx[s] = WP[cell[s]];
#pragma unroll 1
    for (int q = 0; q < 8; ++q) {
      const double cur[6] = {nx[0], nx[1], nx[2], nx[3], nx[4], nx[5]};
      if (q < 7) {
        const double* Wn = WP + (q + 1) * NG;
#pragma unroll
        for (int s = 0; s < 6; ++s) nx[s] = Wn[cell[s]];
      }
      double L, R;
      if (smooth) {
        wenozFace(cur, L, R);
      } else {
        const double st[4] = {cur[1], cur[2], cur[3], cur[4]};
        if (a.G.fallback == 0) weno3Face(st, dx2, L, R);
        else plmFallbackFace(st, L, R);
      }
      if (q == 0) { L = dmax(L, kRHO00); R = dmax(R, kRHO00); }
      if (q == 4) { L = dmax(L, 1.0e-12); R = dmax(R, 1.0e-12); }
      sLR[q][threadIdx.x] = L;
      sLR[8 + q][threadIdx.x] = R;
    }
    double l[8], r[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) { l[q] = sLR[q][threadIdx.x]; r[q] = sLR[8 + q][threadIdx.x]; }
    // Roe repair: only faces whose reconstructed states are unusable read
    // the adjacent cells' average primitives (most faces never do)
    if (roeNow(a.G) && !(usablePrimitive(l) && usablePrimitive(r))) {
      double cl[8], cr[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) { cl[q] = WA[q * NG + cell[2]]; cr[q] = WA[q * NG + cell[3]]; }
      if (usablePrimitive(cl) && usablePrimitive(cr)) {
#pragma unroll
        for (int q = 0; q < 8; ++q) { l[q] = cl[q]; r[q] = cr[q]; }
        thF = 0.0;
      }
    }
    double* base = a.face + (long)b * kO4FaceArrays * NF + fo;
#pragma unroll
    for (int q = 0; q < 8; ++q) { base[(F_WL + q) * NF] = l[q]; base[(F_WR + q) * NF] = r[q]; }
    base[F_THF * NF] = thF;
    const double* A = faceBasis<D>(c, b, j, k);
    double kl, ml, vl, kr, mr, vr, fl[8], fr[8];
    energyW(l, A, kl, ml, vl);
    energyW(r, A, kr, mr, vr);
    primFlux(fl, l, kl, ml, vl, a.G.gamma, d);
    primFlux(fr, r, kr, mr, vr, a.G.gamma, d);
#pragma unroll
    for (int q = 0; q < 8; ++q) base[(F_FS + q) * NF] = fl[q] + fr[q];
    base[F_PS * NF] = (l[4] + ml) + (r[4] + mr);
    base[F_BP * NF] = (l[5 + d] + r[5 + d]) * 0.5;
    if (!roeNow(a.G)) {
      const double rad = radialPoint(a.G, d, i);
      const double g = a.G.gamma;
      base[(F_QD + 0) * NF] = rad * r[0] - rad * l[0];
#pragma unroll
      for (int e = 0; e < 3; ++e) {
        base[(F_QD + 1 + e) * NF] = rad * r[0] * r[1 + e] - rad * l[0] * l[1 + e];
        base[(F_QD + 5 + e) * NF] = rad * r[5 + e] - rad * l[5 + e];
      }
      base[(F_QD + 4) * NF] = rad * (kr + mr + r[4] / (g - 1.0)) - rad * (kl + ml + l[4] / (g - 1.0));
    }
  });
}

// 4b. pointwise factored Roe dissipation on the final faces + one transverse
// ring (src/BoxOp_RoeCubedSphere.H:73-98).
template <int D, int MB>
__global__ void __launch_bounds__(128, MB) o4RoePointKernel(const Ctx* __restrict__ tab, const RegArgs rg, const WorkChunk* __restrict__ wk) {
  const WorkChunk wc = wk[blockIdx.x];
  const Ctx& c = tab[wc.box * 3 + D];
  const O4Args& a = c.a;
  if (!roeNow(a.G)) return;  // the Rusanov window: the reconstruction wrote the Rusanov jump
  constexpr int d = D;
  const Box3 PB = c.V0.growTrans(d, 1);
  forRegion(PB, wc, [&](int b, int i, int j, int k) {
    const long NF = c.fr.N;
    double* base = a.face + (long)b * kO4FaceArrays * NF + roff(c.fr, i, j, k);
    double l[8], r[8], o[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) { l[q] = base[(F_WL + q) * NF]; r[q] = base[(F_WR + q) * NF]; }
    factoredRoe(o, l, r, faceBasis<D>(c, b, j, k), roeRec(a.G, a.block0 + b, D, j, k), radialPoint(a.G, d, i),
                a.G.gamma, a.G.invGm1, a.G.entropy);
#pragma unroll
    for (int q = 0; q < 8; ++q) base[(F_QD + q) * NF] = o[q];
  });
}

// 10. Powell face flux (DivBPowell1, src/BoxOp_DivBcleaning.H:35-74).
template <int D>
__global__ void o4PowellFluxKernel(const Ctx* __restrict__ tab, const RegArgs rg, const WorkChunk* __restrict__ wk) {
  const WorkChunk wc = wk[blockIdx.x];
  const Ctx& c = tab[wc.box * 3 + D];
  const O4Args& a = c.a;
  constexpr int d = D;
  const int t1 = d == 0 ? 1 : 0, t2 = d == 2 ? 1 : 2;
  const int tr[2] = {t1, t2};
  const Box3 BF = c.V1.extrude(d).growTrans(d, 1);
  forRegion(BF, wc, [&](int b, int i, int j, int k) {
    const long NF = c.fr.N, fo = roff(c.fr, i, j, k);
    double* base = a.face + (long)b * kO4FaceArrays * NF;
    const int blk = a.block0 + b;
    const double det = faceRec(a.G, blk, d, j, k)[9];
    double out;
    if (base[F_THF * NF + fo] <= 0.5) {
      out = det * base[F_BP * NF + fo];
    } else {
      View U{a.U + b * a.uStride, a.ur};
      auto bface = [&](int ii, int jj, int kk) {
        int m2[3] = {ii, jj, kk}, m1[3] = {ii, jj, kk}, p1[3] = {ii, jj, kk};
        m2[d] -= 2; m1[d] -= 1; p1[d] += 1;
        return (7.0 / 12.0) * (U(5 + d, m1[0], m1[1], m1[2]) + U(5 + d, ii, jj, kk)) -
               (1.0 / 12.0) * (U(5 + d, m2[0], m2[1], m2[2]) + U(5 + d, p1[0], p1[1], p1[2]));
      };
      double df[2], dg[2];
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int t = tr[q];
        int pa[3] = {i, j, k}, pb[3] = {i, j, k};
        pa[t] += 1; pb[t] -= 1;
        df[q] = 0.5 * faceRec(a.G, blk, d, pa[1], pa[2])[9] - 0.5 * faceRec(a.G, blk, d, pb[1], pb[2])[9];
        dg[q] = 0.5 * bface(pa[0], pa[1], pa[2]) - 0.5 * bface(pb[0], pb[1], pb[2]);
      }
      out = faceProd(det, bface(i, j, k), df[0], dg[0], df[1], dg[1]);
    }
    base[F_BFLUX * NF + fo] = out;
  });
}

// 11. Powell radial-area product and divergence into -J div B (V+1).
template <int D>
__global__ void o4PowellProdKernel(const Ctx* __restrict__ tab, const RegArgs rg, const WorkChunk* __restrict__ wk) {
  const WorkChunk wc = wk[blockIdx.x];
  const Ctx& c = tab[wc.box * 3 + D];
  const O4Args& a = c.a;
  constexpr int d = D;
  const int t1 = d == 0 ? 1 : 0, t2 = d == 2 ? 1 : 2;
  const int tr[2] = {t1, t2};
  const Box3 BP = c.V1.extrude(d);
  forRegion(BP, wc, [&](int b, int i, int j, int k) {
    const long NF = c.fr.N, fo = roff(c.fr, i, j, k);
    double* base = a.face + (long)b * kO4FaceArrays * NF;
    const View BF = faceView(c, b, F_BFLUX);
    double df[2], dg[2];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int t = tr[q];
      df[q] = cdiff(BF, 0, t, i, j, k);
      dg[q] = t == 0 ? 0.5 * adjDr(a.G, d, i + 1) - 0.5 * adjDr(a.G, d, i - 1) : 0.0;
    }
    base[F_BPROD * NF + fo] = faceProd(BF(0, i, j, k), adjDr(a.G, d, i), df[0], dg[0], df[1], dg[1]);
  });
}

template <int D>
__global__ void o4PowellDivKernel(const Ctx* __restrict__ tab, const RegArgs rg, const WorkChunk* __restrict__ wk) {
  const WorkChunk wc = wk[blockIdx.x];
  const Ctx& c = tab[wc.box * 3 + D];
  const O4Args& a = c.a;
  constexpr int d = D;
  const double coef = -1.0 / a.G.dx[d];
  forRegion(c.V1, wc, [&](int b, int i, int j, int k) {
    const View BP = faceView(c, b, F_BPROD);
    int p[3] = {i, j, k};
    p[d] += 1;
    a.mj[(long)b * c.v1r.N + roff(c.v1r, i, j, k)] += coef * (BP(0, p[0], p[1], p[2]) - BP(0, i, j, k));
  });
}

// 12. DivBPowell2 with point primitives (src/BoxOp_DivBcleaning.H:80-172).
__global__ void o4PowellCoefKernel(const Ctx* __restrict__ tab, const RegArgs rg, const WorkChunk* __restrict__ wk) {
  const WorkChunk wc = wk[blockIdx.x];
  const Ctx& c = tab[wc.box * 3 + 0];
  const O4Args& a = c.a;
  forRegion(c.V2, wc, [&](int b, int i, int j, int k) {
    const long NG = c.gr.N, o = roff(c.gr, i, j, k);
    const double* WP = a.WP + (long)b * 8 * NG;
    const double* A = cellBasis(a.G, a.block0 + b, j, k);
    double vel[3], mag[3];
#pragma unroll
    for (int e = 0; e < 3; ++e) {
      vel[e] = A[3 * e] * WP[1 * NG + o] + A[3 * e + 1] * WP[2 * NG + o] + A[3 * e + 2] * WP[3 * NG + o];
      mag[e] = A[3 * e] * WP[5 * NG + o] + A[3 * e + 1] * WP[6 * NG + o] + A[3 * e + 2] * WP[7 * NG + o];
    }
    double* K = a.kp + (long)b * 16 * c.v2r.N + roff(c.v2r, i, j, k);
    const long N = c.v2r.N;
    K[0] = 0;
    double e4 = 0;
#pragma unroll
    for (int e = 0; e < 3; ++e) {
      K[(1 + e) * N] = mag[e] / (4.0 * kPi);
      K[(5 + e) * N] = vel[e];
      e4 += vel[e] * mag[e] / (4.0 * kPi);
    }
    K[4 * N] = e4;
  });
}

__global__ void o4PowellAvgKernel(const Ctx* __restrict__ tab, const RegArgs rg, const WorkChunk* __restrict__ wk) {
  const WorkChunk wc = wk[blockIdx.x];
  const Ctx& c = tab[wc.box * 3 + 0];
  const O4Args& a = c.a;
  forRegion(c.V1, wc, [&](int b, int i, int j, int k) {
    const View KP{a.kp + (long)b * 16 * c.v2r.N, c.v2r};
    double* KA = a.kp + (long)b * 16 * c.v2r.N + 8 * c.v2r.N + roff(c.v2r, i, j, k);
    // all loads before the first store (KA and KP share one array)
    double out[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) out[q] = KP(q, i, j, k) + lapCell(KP, q, i, j, k) * (1.0 / 24.0);
#pragma unroll
    for (int q = 0; q < 8; ++q) KA[q * c.v2r.N] = out[q];
  });
}

__global__ void o4PowellApplyKernel(const Ctx* __restrict__ tab, const RegArgs rg, const WorkChunk* __restrict__ wk) {
  const WorkChunk wc = wk[blockIdx.x];
  const Ctx& c = tab[wc.box * 3 + 0];
  const O4Args& a = c.a;
  forRegion(c.V, wc, [&](int b, int i, int j, int k) {
    const View KA{a.kp + (long)b * 16 * c.v2r.N + 8 * c.v2r.N, c.v2r};
    const View MJ{a.mj + (long)b * c.v1r.N, c.v1r};
    double* R = a.rhs + b * a.rhsStride + roff(c.vr, i, j, k);
    // all loads (including the accumulated rhs) before the first store
    double dmj[3];
#pragma unroll
    for (int t = 0; t < 3; ++t) dmj[t] = cdiff(MJ, 0, t, i, j, k);
    const double mj0 = MJ(0, i, j, k);
    double add[8], rv[8];
#pragma unroll
    for (int q = 1; q < 8; ++q) {
      double value = 0.0;
#pragma unroll
      for (int t = 0; t < 3; ++t) value += dmj[t] * cdiff(KA, q, t, i, j, k) * (1.0 / 12.0);
      value += mj0 * KA(q, i, j, k) * 1.0;
      add[q] = value;
      rv[q] = R[q * c.vr.N];
    }
#pragma unroll
    for (int q = 1; q < 8; ++q) R[q * c.vr.N] = rv[q] + add[q];
  });
}

// Gravity_Euler (src/BoxOp_Gravity.H:84-164) on the valid boxes: with
// dr = D_r (dr/dxi0) the fourth-order cell products <rho dr>, <rho V_r dr>
// (<ab> = <a><b> + (1/12) sum_d D_d a D_d b; dr varies only radially), then
// rhs(m_d) += -GM faceProduct(<det A A>(d, 0), <rho dr>, 0) and
// rhs(E) += -GM faceProduct(<det A>, <rho V_r dr>, 0), faceProduct over the
// two angular directions.
__global__ void o4GravityKernel(const Ctx* __restrict__ tab, const RegArgs rg, const WorkChunk* __restrict__ wk) {
  const WorkChunk wc = wk[blockIdx.x];
  const Ctx& c = tab[wc.box * 3 + 0];
  const O4Args& a = c.a;
  const double minusGM = -kGrav * kMsun;
  forRegion(c.V, wc, [&](int b, int i, int j, int k) {
    const View U{a.U + b * a.uStride, a.ur};
    const int blk = a.block0 + b;
    const double dr0 = radialRow(a.G, i).z;
    const double da = 0.5 * radialRow(a.G, i + 1).z - 0.5 * radialRow(a.G, i - 1).z;
    const int pj[5] = {j, j + 1, j - 1, j, j}, pk[5] = {k, k, k, k + 1, k - 1};
    double rd[5], re[5];
    const double* M[5];
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      const double d0 = 0.5 * U(0, i + 1, pj[q], pk[q]) - 0.5 * U(0, i - 1, pj[q], pk[q]);
      const double d1 = 0.5 * U(1, i + 1, pj[q], pk[q]) - 0.5 * U(1, i - 1, pj[q], pk[q]);
      rd[q] = dr0 * U(0, i, pj[q], pk[q]) + da * d0 * (1.0 / 12.0);
      re[q] = dr0 * U(1, i, pj[q], pk[q]) + da * d1 * (1.0 / 12.0);
      M[q] = faceRec(a.G, blk, 0, pj[q], pk[q]);
    }
    auto faceP = [&](int e, const double* v) {
      double value = M[0][e] * v[0];
      value += (0.5 * M[1][e] - 0.5 * M[2][e]) * (0.5 * v[1] - 0.5 * v[2]) * (1.0 / 12.0);
      value += (0.5 * M[3][e] - 0.5 * M[4][e]) * (0.5 * v[3] - 0.5 * v[4]) * (1.0 / 12.0);
      return value;
    };
    double* R = a.rhs + b * a.rhsStride + roff(c.vr, i, j, k);
#pragma unroll
    for (int d = 0; d < 3; ++d) R[(1 + d) * c.vr.N] += faceP(3 * d, rd) * minusGM;
    R[4 * c.vr.N] += faceP(9, re) * minusGM;
  });
}


// ---- fused face chain ----------------------------------------------------------
// One CTA (128 threads) takes a tile of the final faces of direction d and
// runs the whole chain after the reconstruction and the Roe point
// dissipation on it: the theta-aware point-to-average of the flux sum and of
// the total pressure (5), the mapped flux with its transverse products (6),
// the radial-area products (7), the pressure force, the dissipation average
// and the final flux (8), and the flux divergence into rhs (9).  The
// intermediates (averaged fluxes, mapped fluxes, radial products) live in
// shared memory; only the reconstruction's face arrays (FS, PS, thF, QD and,
// for the Rusanov speed, WL and WR) are read from the face scratch, and the
// only global writes are rhs, the caller's flux and the seam register.
//
// d = 1, 2: the threads cover TI radial x TT angular (t) faces; the CTA
// walks the normal direction over a segment of cells [c0, c1], one face
// slab after another, and keeps each face's flux in registers for the
// divergence of the next cell.  d = 0: the threads cover TI radial cells
// (TI + 1 faces) x TT rows of j and walk k over [c0, c1], the averages of
// rows k - 1, k, k + 1 held in a ring of three shared slabs.
//
// Every product and sum is formed as in the separate steps of the chain
// (same operands, same order), so the results do not depend on the tiling.
struct ChainTile {
  int box;
  int i0, a0;  // first radial index; first angular index across the tile (t for d != 0, j for d = 0)
  int c0, c1;  // walk range of cells (d != 0: along d; d = 0: along k)
};

template <int D>
__device__ __forceinline__ void chainPt(int i, int n, int t, int p[3]) {
  // d != 0: (radial i, normal n, angular t) -> (i, j, k)
  p[0] = i;
  p[1] = D == 1 ? n : t;
  p[2] = D == 1 ? t : n;
}

// Final flux of one face from its mapped-and-radial flux fs (pressure force
// added here), the dissipation inputs and the metrics (the final flux of
// the reference's face pass).  dT3[q]: centred difference of the radial
// pressure product along transverse q (unused where the separable metrics
// skip it).
// The point Roe dissipations a final face averages: component stride and
// the offsets of the face and its four transverse neighbours (lower and
// upper along t1, then along t2), in the face scratch or in a shared tile.
struct QdTaps {
  const double* p;
  long stride;
  long o[5];
};

__device__ __forceinline__ QdTaps scratchTaps(const Ctx& c, int d, int i, int j, int k) {
  const View QD = faceView(c, 0, F_QD);
  const int t1 = d == 0 ? 1 : 0, t2 = d == 2 ? 1 : 2;
  int m1[3] = {i, j, k}, p1[3] = {i, j, k}, m2[3] = {i, j, k}, p2[3] = {i, j, k};
  m1[t1] -= 1; p1[t1] += 1; m2[t2] -= 1; p2[t2] += 1;
  return QdTaps{QD.p, QD.r.N,
                {roff(QD.r, i, j, k), roff(QD.r, m1[0], m1[1], m1[2]), roff(QD.r, p1[0], p1[1], p1[2]),
                 roff(QD.r, m2[0], m2[1], m2[2]), roff(QD.r, p2[0], p2[1], p2[2])}};
}

template <int D>
__device__ __forceinline__ void chainFinal(const Ctx& c, int i, int j, int k, double fs[8], const double t3,
                                           const double dT3[2], const QdTaps& tap, double fx[8]) {
  const O4Args& a = c.a;
  constexpr int d = D;
  const int t1 = d == 0 ? 1 : 0, t2 = d == 2 ? 1 : 2;
  const int tr[2] = {t1, t2};
  const int blk = a.block0;
  const long NF = c.fr.N, fo = roff(c.fr, i, j, k);
  const double* base = a.face;
  const double* M = faceRec(a.G, blk, d, j, k);
#pragma unroll
  for (int row = 0; row < 3; ++row) {
    double value = 0.0;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int t = tr[q];
      if (d != 0 && t == 0) continue;
      int pa[3] = {i, j, k}, pb[3] = {i, j, k};
      pa[t] += 1; pb[t] -= 1;
      const double dn = 0.5 * faceRec(a.G, blk, d, pa[1], pa[2])[10 + row] - 0.5 * faceRec(a.G, blk, d, pb[1], pb[2])[10 + row];
      value += dn * dT3[q] * (1.0 / 12.0);
    }
    value += M[10 + row] * t3 * 1.0;
    fs[1 + row] += value;
  }
  const bool sm = base[F_THF * NF + fo] > 0.5;
  const View QD = faceView(c, 0, F_QD);
  double diss[8];
  if (roeNow(a.G)) {
    double dM[2][10];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int t = tr[q];
      int pa[3] = {i, j, k}, pb[3] = {i, j, k};
      pa[t] += 1; pb[t] -= 1;
      const double* Ma = faceRec(a.G, blk, d, pa[1], pa[2]);
      const double* Mb = faceRec(a.G, blk, d, pb[1], pb[2]);
#pragma unroll
      for (int e = 0; e < 10; ++e) dM[q][e] = 0.5 * Ma[e] - 0.5 * Mb[e];
    }
    double avg[8], dP0[8], dP1[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const double* Q = tap.p + q * tap.stride;
      const double pt = Q[tap.o[0]], a1 = Q[tap.o[1]], b1 = Q[tap.o[2]], a2 = Q[tap.o[3]], b2 = Q[tap.o[4]];
      const double lap = (a1 + b1) + (a2 + b2) - 4.0 * pt;
      avg[q] = sm ? pt + lap * (1.0 / 24.0) : pt;
      dP0[q] = 0.5 * b1 - 0.5 * a1;
      dP1[q] = 0.5 * b2 - 0.5 * a2;
    }
    diss[0] = faceProd(M[9], avg[0], dM[0][9], dP0[0], dM[1][9], dP1[0]);
    diss[4] = faceProd(M[9], avg[4], dM[0][9], dP0[4], dM[1][9], dP1[4]);
#pragma unroll
    for (int bb = 0; bb < 2; ++bb) {
      const int bs = bb == 0 ? 1 : 5;
#pragma unroll
      for (int row = 0; row < 3; ++row) {
        double sum = 0.0;
#pragma unroll
        for (int col = 0; col < 3; ++col)
          sum += faceProd(M[3 * row + col], avg[bs + col], dM[0][3 * row + col], dP0[bs + col], dM[1][3 * row + col],
                          dP1[bs + col]);
        diss[bs + row] = sum;
      }
    }
  } else {
    double qv[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const double pt = QD(q, i, j, k);
      qv[q] = sm ? pt + lapFace(QD, q, d, i, j, k) * (1.0 / 24.0) : pt;
    }
#pragma unroll
    for (int bb = 0; bb < 2; ++bb) {
      const int bs = bb == 0 ? 1 : 5;
#pragma unroll
      for (int row = 0; row < 3; ++row)
        diss[bs + row] = M[3 * row] * qv[bs] * 1.0 + M[3 * row + 1] * qv[bs + 1] * 1.0 + M[3 * row + 2] * qv[bs + 2] * 1.0;
    }
    diss[0] = M[9] * qv[0];
    diss[4] = M[9] * qv[4];
    // face wave-speed bound (:1665-1720)
    double l[8], r[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) { l[q] = base[(F_WL + q) * NF + fo]; r[q] = base[(F_WR + q) * NF + fo]; }
    const double* A = faceBasis<D>(c, 0, j, k);
    double rho = 0.5 * (l[0] + r[0]);
    const double w_d = 0.5 * (l[1 + d] + r[1 + d]);
    const double bs3[3] = {0.5 * (l[5] + r[5]), 0.5 * (l[6] + r[6]), 0.5 * (l[7] + r[7])};
    double p = 0.5 * (l[4] + r[4]);
    if (p < 0.0) p = 0.0;
    rho = dmax(rho, kRHO00);
    double Bn = 0.0, Bm = 0.0;
#pragma unroll
    for (int e0 = 0; e0 < 3; ++e0) {
      const double bC = A[3 * e0] * bs3[0] + A[3 * e0 + 1] * bs3[1] + A[3 * e0 + 2] * bs3[2];
      Bn += A[3 * e0] * bC;
      Bm += bC * bC;
    }
    Bm = sqrt(Bm);
    const double g = a.G.gamma;
    const double ce = sqrt(g * p / rho);
    const double aa = ce * ce + Bm * Bm / (4.0 * kPi * rho);
    const double bb2 = fabs(Bn) * ce / sqrt(kPi * rho);
    const double af = 0.5 * (sqrt(dmax(0.0, aa + bb2)) + sqrt(dmax(0.0, aa - bb2)));
    const double Am = sqrt(A[d] * A[d] + A[3 + d] * A[3 + d] + A[6 + d] * A[6 + d]);
    const double speed = fabs(w_d) + af * Am;
#pragma unroll
    for (int q = 0; q < 8; ++q) diss[q] *= speed;
  }
#pragma unroll
  for (int q = 0; q < 8; ++q) fx[q] = 0.5 * (fs[q] - diss[q]);
}

// The caller's flux and the seam register of one final face.
template <int D>
__device__ __forceinline__ void chainStore(const Ctx& c, const RegArgs& rg, int i, int j, int k, const double fx[8]) {
  const O4Args& a = c.a;
  constexpr int d = D;
  if (a.flux[d]) {
    const Reg r0 = regOf(c.V0);
    double* fo2 = a.flux[d] + roff(r0, i, j, k);
#pragma unroll
    for (int q = 0; q < 8; ++q) fo2[q * r0.N] = fx[q];
  }
  double* const reg = a.seamReg ? a.seamReg : rg.reg;
  if (reg && d > 0) {
    const int f = d == 1 ? j : k;
    if (f == 0 || f == a.G.na) {
      const long nrna = (long)a.G.na * a.G.nr;
      const int side = f == 0 ? 0 : 1, s = d == 1 ? k : j;
      const double w = a.seamReg ? rg.w * (a.seamCfl / *a.seamInvMax) : rg.wDev ? rg.w * (rg.cfl / *rg.wDev) : rg.w;
      double* R = reg + (((long)a.block0 * 2 + (d - 1)) * 2 + side) * 8 * nrna + (long)s * a.G.nr + i;
#pragma unroll
      for (int q = 0; q < 8; ++q) R[q * nrna] += w * fx[q];
    }
  }
}

// Point-to-average of the flux sum and total pressure at one face (5).
__device__ __forceinline__ void chainAverage(const Ctx& c, int d, int i, int j, int k, double fa[8], double& pa) {
  const long NF = c.fr.N, fo = roff(c.fr, i, j, k);
  const double* base = c.a.face;
  const bool sm = base[F_THF * NF + fo] > 0.5;
  const View FS = faceView(c, 0, F_FS);
  const View PS = faceView(c, 0, F_PS);
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const double pt = FS(q, i, j, k);
    fa[q] = sm ? pt + lapFace(FS, q, d, i, j, k) * (1.0 / 24.0) : pt;
  }
  const double pp = PS(0, i, j, k);
  pa = sm ? pp + lapFace(PS, 0, d, i, j, k) * (1.0 / 24.0) : pp;
}

// Directions 1, 2: walk the normal direction.  With TMA, the slab's flux
// sums, flags and total pressures (tile plus a two-face ring) and its point
// Roe dissipations (tile plus a one-face ring) are copied into shared
// memory by the tensor-memory accelerator, the next slab's copies issued as
// soon as the current slab's are consumed, so they overlap the mapped-flux
// and final-flux stages; without it (tensor maps unavailable) the same
// stages read the face scratch through L1.
// TMA tensor maps per box: directions 1 and 2 (8 arrays, 2 arrays each),
// then direction 0 (averages: 9 arrays; dissipations: 8).
constexpr int kChainMaps = 6;

template <int TI>
struct ChainShape {
  static constexpr int TT = 128 / TI, NI = TI + 2, NT = TT + 2;  // averages: tile plus a one-face ring
  static constexpr int NTH = NI * TT;  // threads: one per mapped-flux point (the tile's faces and a radial ring)
  static constexpr int NX = TI + 4, NY = TT + 4, NXY = NX * NY;  // TMA tiles: tile plus a two-face ring
  static constexpr int round16(int n) { return (n + 15) / 16 * 16; }
  static constexpr int oFA = 0, oPA = oFA + round16(8 * NI * NT), oFM = oPA + round16(NI * NT),
                       oT3 = oFM + round16(8 * NI * TT), oIn = oT3 + round16(TI * NT),
                       oQD = oIn + round16(10 * NXY), oBar = oQD + round16(8 * NXY);
  static constexpr int doubles(bool tma) { return tma ? oBar + 2 : oIn; }
};

__device__ __forceinline__ unsigned smemAddr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbarInit(unsigned long long* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smemAddr(bar)) : "memory");
}

__device__ __forceinline__ void mbarExpect(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smemAddr(bar)), "r"(bytes) : "memory");
}

// Bounded wait for phase `parity` of an mbarrier: false when it has not
// completed after kMbarPolls polls (each poll blocks for a short,
// implementation-defined time), so a copy that never lands cannot hang the
// GPU.
constexpr int kMbarPolls = 1 << 22;
__device__ __forceinline__ bool mbarWait(unsigned long long* bar, unsigned parity) {
  const unsigned addr = smemAddr(bar);
  for (int it = 0; it < kMbarPolls; ++it) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// One tiled TMA copy of a 4-D box (radial, j, k, array) of the face scratch
// into shared memory, completing on `bar`.
__device__ __forceinline__ void tmaLoad(double* dst, const CUtensorMap* map, int x, int y, int z, int w,
                                        unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(smemAddr(dst)),
      "l"(map), "r"(x), "r"(y), "r"(z), "r"(w), "r"(smemAddr(bar))
      : "memory");
}

template <int D, int TI, int MB, bool TMA>
__global__ void __launch_bounds__(ChainShape<TI>::NTH, MB) o4FaceChainKernel(const Ctx* __restrict__ tab,
                                                                            const RegArgs rg,
                                                             const ChainTile* __restrict__ tiles,
                                                             const CUtensorMap* __restrict__ maps) {
  static_assert(D == 1 || D == 2, "angular directions");
  using S = ChainShape<TI>;
  constexpr int TT = S::TT, NI = S::NI, NT = S::NT, NX = S::NX, NXY = S::NXY;
  constexpr int tdim = D == 1 ? 2 : 1;
  extern __shared__ __align__(128) double smem[];
  double* sFA = smem + S::oFA;  // [8][NI * NT]
  double* sPA = smem + S::oPA;  // [NI * NT]
  double* sFM = smem + S::oFM;  // [8][NI * TT]
  double* sT3 = smem + S::oT3;  // [TI * NT]
  double* sIn = smem + S::oIn;  // TMA: [FS 8, thF, PS][NY][NX]
  double* sQD = smem + S::oQD;  // TMA: [8][NY][NX]
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(smem + S::oBar);
  const ChainTile tl = tiles[blockIdx.x];
  const Ctx& c = tab[tl.box * 3 + D];
  const O4Args& a = c.a;
  constexpr int NTH = S::NTH;
  const int tid = threadIdx.x, li = tid % TI, lt = tid / TI;
  const int i = tl.i0 + li, t = tl.a0 + lt;
  // threads beyond the tile's TI x TT faces only help with the shared stages
  const bool mine = tid < TI * TT && i <= c.V.hi[0] && t <= c.V.hi[tdim];
  // radial products: area at i and its centred difference
  const double s = adjDr(a.G, D, i), ds = 0.5 * adjDr(a.G, D, i + 1) - 0.5 * adjDr(a.G, D, i - 1);
  const double coef = -a.scale / a.G.dx[D];
  const int ilo = c.V.lo[0] - 1, ihi = c.V.hi[0] + 1, tlo = c.V.lo[tdim] - 1, thi = c.V.hi[tdim] + 1;
  double fxPrev[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) fxPrev[q] = 0.0;
  const int nEnd = tl.c1 + 1;
  const bool lastSegment = tl.c1 == c.V.hi[D];
  // TMA tiles: radial from i0 - 2 (an even offset from the face box's low
  // corner: tiles start at the valid box's low radial index and TI is even),
  // angular from a0 - 2, one face slab; map 0 copies 8 arrays, map 1 two
  const CUtensorMap* map8 = TMA ? maps + (long)tl.box * kChainMaps + (D - 1) * 2 : nullptr;
  const CUtensorMap* map2 = TMA ? map8 + 1 : nullptr;
  const int tx = tl.i0 - 2 - c.fr.lo[0], ta = tl.a0 - 2 - c.fr.lo[tdim], tnLo = c.fr.lo[D];
  auto issue = [&](int n, bool inputs) {
    const int y = D == 1 ? n - tnLo : ta, z = D == 1 ? ta : n - tnLo;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (inputs) {
      mbarExpect(&bar[0], 10u * NXY * sizeof(double));
      tmaLoad(sIn, map8, tx, y, z, F_FS, &bar[0]);
      tmaLoad(sIn + 8 * NXY, map2, tx, y, z, F_THF, &bar[0]);
    } else {
      mbarExpect(&bar[1], 8u * NXY * sizeof(double));
      tmaLoad(sQD, map8, tx, y, z, F_QD, &bar[1]);
    }
  };
  bool failed = false;
  if (TMA) {
    if (tid == 0) {
      mbarInit(&bar[0]);
      mbarInit(&bar[1]);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (tid == 0) {
      issue(tl.c0, true);
      issue(tl.c0, false);
    }
  }
  for (int n = tl.c0; n <= nEnd && !failed; ++n) {
    const unsigned parity = (unsigned)(n - tl.c0) & 1u;
    if (TMA) {
      failed = __syncthreads_or(!mbarWait(&bar[0], parity));
      if (failed) break;
    }
    // (5) averages on radial i0-1 .. i0+TI x angular a0-1 .. a0+TT of face slab n
    for (int q = tid; q < NI * NT; q += NTH) {
      const int ii = tl.i0 - 1 + q % NI, tt = tl.a0 - 1 + q / NI;
      if (ii < ilo || ii > ihi || tt < tlo || tt > thi) continue;
      double fa[8], pa;
      if (TMA) {
        // (ii, tt) in the TMA tile; lapFace's order: radial pair, angular pair
        const int x = q % NI + 1, y = q / NI + 1, o = y * NX + x;
        const bool sm = sIn[8 * NXY + o] > 0.5;
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const double* F = sIn + e * NXY;
          const double pt = F[o];
          fa[e] = sm ? pt + ((F[o - 1] + F[o + 1]) + (F[o - NX] + F[o + NX]) - 4.0 * pt) * (1.0 / 24.0) : pt;
        }
        const double* P = sIn + 9 * NXY;
        const double pp = P[o];
        pa = sm ? pp + ((P[o - 1] + P[o + 1]) + (P[o - NX] + P[o + NX]) - 4.0 * pp) * (1.0 / 24.0) : pp;
      } else {
        int p[3];
        chainPt<D>(ii, n, tt, p);
        chainAverage(c, D, p[0], p[1], p[2], fa, pa);
      }
#pragma unroll
      for (int e = 0; e < 8; ++e) sFA[e * NI * NT + q] = fa[e];
      sPA[q] = pa;
    }
    __syncthreads();
    if (TMA && tid == 0 && n < nEnd) issue(n + 1, true);  // the inputs' tile is free again
    // (6) mapped flux on radial i0-1 .. i0+TI x angular a0 .. a0+TT-1; the
    // radial transverse derivative of the angular metrics vanishes (skipped)
    for (int q = tid; q < NI * TT; q += NTH) {
      const int ii = tl.i0 - 1 + q % NI, tt = tl.a0 + q / NI;
      if (ii < ilo || ii > ihi || tt > c.V.hi[tdim]) continue;
      int p[3];
      chainPt<D>(ii, n, tt, p);
      const double* M = faceRec(a.G, a.block0, D, p[1], p[2]);
      int pa[3] = {p[0], p[1], p[2]}, pb[3] = {p[0], p[1], p[2]};
      pa[tdim] += 1; pb[tdim] -= 1;
      const double* Ma = faceRec(a.G, a.block0, D, pa[1], pa[2]);
      const double* Mb = faceRec(a.G, a.block0, D, pb[1], pb[2]);
      double dM[10];
#pragma unroll
      for (int e = 0; e < 10; ++e) dM[e] = 0.5 * Ma[e] - 0.5 * Mb[e];
      const int qc = q + NI;  // (ii, tt) in the averages' frame (rows from a0 - 1)
      const int qu = qc + NI, qd = qc - NI;
      double fa[8], dF[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        fa[e] = sFA[e * NI * NT + qc];
        dF[e] = 0.5 * sFA[e * NI * NT + qu] - 0.5 * sFA[e * NI * NT + qd];
      }
      double out[8];
#pragma unroll
      for (int qq = 0; qq < 2; ++qq) {
        const int e = qq == 0 ? 0 : 4;
        double term = 0.0;
        term += dM[9] * dF[e] * (1.0 / 12.0);
        term += M[9] * fa[e] * 1.0;
        out[e] = 0.0 + term;
      }
#pragma unroll
      for (int bb = 0; bb < 2; ++bb) {
        const int bs = bb == 0 ? 1 : 5;
#pragma unroll
        for (int row = 0; row < 3; ++row) {
          double sum = 0.0;
#pragma unroll
          for (int col = 0; col < 3; ++col) {
            double term = 0.0;
            term += dM[3 * row + col] * dF[bs + col] * (1.0 / 12.0);
            term += M[3 * row + col] * fa[bs + col] * 1.0;
            sum += term;
          }
          out[bs + row] = sum;
        }
      }
#pragma unroll
      for (int e = 0; e < 8; ++e) sFM[e * NI * TT + q] = out[e];
    }
    // (7) radial product of <p_tot> on radial i0 .. i0+TI-1 x angular a0-1 .. a0+TT
    for (int q = tid; q < TI * NT; q += NTH) {
      const int ii = tl.i0 + q % TI, tt = tl.a0 - 1 + q / TI;
      if (ii > c.V.hi[0] || tt < tlo || tt > thi) continue;
      const double si = adjDr(a.G, D, ii), dsi = 0.5 * adjDr(a.G, D, ii + 1) - 0.5 * adjDr(a.G, D, ii - 1);
      const int qc = (q / TI) * NI + (q % TI) + 1;  // (ii, tt) in the averages' frame
      double value = 0.0;
      value += (0.5 * sPA[qc + 1] - 0.5 * sPA[qc - 1]) * dsi * (1.0 / 12.0);
      value += sPA[qc] * si * 1.0;
      sT3[q] = value;
    }
    if (TMA) {
      failed = __syncthreads_or(!mbarWait(&bar[1], parity));
      if (failed) break;
    } else {
      __syncthreads();
    }
    // (7, 8, 9) this thread's face: radial product of the mapped flux, final
    // flux, divergence of the cell below it
    if (mine) {
      int p[3];
      chainPt<D>(i, n, t, p);
      const int qm = lt * NI + li + 1;  // (i, t) in the mapped-flux frame
      double fs[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        double value = 0.0;
        value += (0.5 * sFM[e * NI * TT + qm + 1] - 0.5 * sFM[e * NI * TT + qm - 1]) * ds * (1.0 / 12.0);
        value += sFM[e * NI * TT + qm] * s * 1.0;
        fs[e] = value;
      }
      const int q3 = (lt + 1) * TI + li;  // (i, t) in the pressure-product frame
      const double dT3[2] = {0.0, 0.5 * sT3[q3 + TI] - 0.5 * sT3[q3 - TI]};
      QdTaps tap;
      if (TMA) {
        const int o = (lt + 2) * NX + (li + 2);  // (i, t) in the TMA tile
        tap = QdTaps{sQD, NXY, {o, o - 1, o + 1, o - NX, o + NX}};
      } else {
        tap = scratchTaps(c, D, p[0], p[1], p[2]);
      }
      double fx[8];
      chainFinal<D>(c, p[0], p[1], p[2], fs, sT3[q3], dT3, tap, fx);
      if (n <= tl.c1 || lastSegment) chainStore<D>(c, rg, p[0], p[1], p[2], fx);
      if (n > tl.c0) {
        int pc[3];
        chainPt<D>(i, n - 1, t, pc);
        double* R = a.rhs + roff(c.vr, pc[0], pc[1], pc[2]);
        double rv[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) rv[e] = R[e * c.vr.N];
#pragma unroll
        for (int e = 0; e < 8; ++e) R[e * c.vr.N] = rv[e] + coef * (fx[e] - fxPrev[e]);
      }
#pragma unroll
      for (int e = 0; e < 8; ++e) fxPrev[e] = fx[e];
    }
    __syncthreads();
    if (TMA && tid == 0 && n < nEnd) issue(n + 1, false);  // the dissipations' tile is free again
  }
  if (TMA && failed) {
    // A copy did not land: report it, wait (bounded) for the copies still in
    // flight, and make this tile's cells visibly invalid.
    if (tid == 0) {
      if (a.G.status) atomicExch(a.G.status, 1);
      mbarWait(&bar[0], 0u);
      mbarWait(&bar[1], 0u);
      mbarWait(&bar[0], 1u);
      mbarWait(&bar[1], 1u);
    }
    __syncthreads();
    if (mine)
      for (int n = tl.c0; n <= tl.c1; ++n) {
        int pc[3];
        chainPt<D>(i, n, t, pc);
#pragma unroll
        for (int e = 0; e < 8; ++e) a.rhs[roff(c.vr, pc[0], pc[1], pc[2]) + e * c.vr.N] = CUDART_NAN;
      }
  }
}

// Direction 0: walk k; shared memory (dynamic): averages of three rows of k
// [3][8][NS], pressure averages [3][NS], final fluxes [8][(TI + 1) TT].
template <int TI>
__host__ __device__ constexpr int chain0Doubles() {
  return 3 * 9 * (TI + 1) * (128 / TI + 2) + 8 * (TI + 1) * (128 / TI);
}

// Threads of the direction-0 chain: one per final face of a row of the tile.
template <int TI>
__host__ __device__ constexpr int chain0Threads() {
  return (TI + 1) * (128 / TI);
}

template <int TI, int MB>
__global__ void __launch_bounds__(chain0Threads<TI>(), MB) o4FaceChain0Kernel(const Ctx* __restrict__ tab,
                                                                              const RegArgs rg,
                                                                              const ChainTile* __restrict__ tiles) {
  constexpr int TT = 128 / TI, NI = TI + 1, NJ = TT + 2, NS = NI * NJ, NTH = chain0Threads<TI>();
  extern __shared__ __align__(128) double smem[];
  double* sFA = smem;              // [3][8][NS]
  double* sPA = sFA + 3 * 8 * NS;  // [3][NS]
  double* sFX = sPA + 3 * NS;      // [8][NI * TT]
  const ChainTile tl = tiles[blockIdx.x];
  const Ctx& c = tab[tl.box * 3 + 0];
  const O4Args& a = c.a;
  const int tid = threadIdx.x;
  const double coef = -a.scale / a.G.dx[0];
  const int ihi = c.V.hi[0] + 1, jlo = c.V.lo[1] - 1, jhi = c.V.hi[1] + 1;
  auto slot = [&](int k) { return (k - tl.c0 + 3) % 3; };
  auto slab = [&](int k) {
    double* fa = sFA + slot(k) * 8 * NS;
    double* pa = sPA + slot(k) * NS;
    for (int q = tid; q < NS; q += NTH) {
      const int ii = tl.i0 + q % NI, jj = tl.a0 - 1 + q / NI;
      if (ii > ihi || jj < jlo || jj > jhi) continue;
      double f[8], pp;
      chainAverage(c, 0, ii, jj, k, f, pp);
#pragma unroll
      for (int e = 0; e < 8; ++e) fa[e * NS + q] = f[e];
      pa[q] = pp;
    }
  };
  slab(tl.c0 - 1);
  slab(tl.c0);
  for (int k = tl.c0; k <= tl.c1; ++k) {
    slab(k + 1);
    __syncthreads();
    const double* F0 = sFA + slot(k) * 8 * NS;
    const double* Fm = sFA + slot(k - 1) * 8 * NS;
    const double* Fp = sFA + slot(k + 1) * 8 * NS;
    const double* P0 = sPA + slot(k) * NS;
    const double* Pm = sPA + slot(k - 1) * NS;
    const double* Pp = sPA + slot(k + 1) * NS;
    // (6, 7, 8) faces i0 .. i0+TI x rows a0 .. a0+TT-1 of row k
    for (int q = tid; q < NI * TT; q += NTH) {
      const int ii = tl.i0 + q % NI, jj = tl.a0 + q / NI;
      if (ii > ihi || jj > c.V.hi[1]) continue;
      const int qc = q + NI;  // (ii, jj) in the slab frame
      const double* M = faceRec(a.G, a.block0, 0, jj, k);
      const double* Mj1 = faceRec(a.G, a.block0, 0, jj + 1, k);
      const double* Mj0 = faceRec(a.G, a.block0, 0, jj - 1, k);
      const double* Mk1 = faceRec(a.G, a.block0, 0, jj, k + 1);
      const double* Mk0 = faceRec(a.G, a.block0, 0, jj, k - 1);
      double dM0[10], dM1[10];
#pragma unroll
      for (int e = 0; e < 10; ++e) {
        dM0[e] = 0.5 * Mj1[e] - 0.5 * Mj0[e];
        dM1[e] = 0.5 * Mk1[e] - 0.5 * Mk0[e];
      }
      double fa[8], dF0[8], dF1[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        fa[e] = F0[e * NS + qc];
        dF0[e] = 0.5 * F0[e * NS + qc + NI] - 0.5 * F0[e * NS + qc - NI];
        dF1[e] = 0.5 * Fp[e * NS + qc] - 0.5 * Fm[e * NS + qc];
      }
      double fm[8];
#pragma unroll
      for (int qq = 0; qq < 2; ++qq) {
        const int e = qq == 0 ? 0 : 4;
        double term = 0.0;
        term += dM0[9] * dF0[e] * (1.0 / 12.0);
        term += dM1[9] * dF1[e] * (1.0 / 12.0);
        term += M[9] * fa[e] * 1.0;
        fm[e] = 0.0 + term;
      }
#pragma unroll
      for (int bb = 0; bb < 2; ++bb) {
        const int bs = bb == 0 ? 1 : 5;
#pragma unroll
        for (int row = 0; row < 3; ++row) {
          double sum = 0.0;
#pragma unroll
          for (int col = 0; col < 3; ++col) {
            double term = 0.0;
            term += dM0[3 * row + col] * dF0[bs + col] * (1.0 / 12.0);
            term += dM1[3 * row + col] * dF1[bs + col] * (1.0 / 12.0);
            term += M[3 * row + col] * fa[bs + col] * 1.0;
            sum += term;
          }
          fm[bs + row] = sum;
        }
      }
      // radial products (direction 0: no radial correction)
      const double si = adjDr(a.G, 0, ii);
      double fs[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        double value = 0.0;
        value += fm[e] * si * 1.0;
        fs[e] = value;
      }
      auto t3 = [&](double pav) {
        double value = 0.0;
        value += pav * si * 1.0;
        return value;
      };
      const double dT3[2] = {0.5 * t3(P0[qc + NI]) - 0.5 * t3(P0[qc - NI]), 0.5 * t3(Pp[qc]) - 0.5 * t3(Pm[qc])};
      double fx[8];
      chainFinal<0>(c, ii, jj, k, fs, t3(P0[qc]), dT3, scratchTaps(c, 0, ii, jj, k), fx);
      chainStore<0>(c, rg, ii, jj, k, fx);
#pragma unroll
      for (int e = 0; e < 8; ++e) sFX[e * NI * TT + q] = fx[e];
    }
    __syncthreads();
    // (9) divergence of the row's cells
    {
      const int li = tid % TI, lj = tid / TI;
      const int i = tl.i0 + li, j = tl.a0 + lj;
      if (tid < TI * TT && i <= c.V.hi[0] && j <= c.V.hi[1]) {
        const int q = lj * NI + li;
        double* R = a.rhs + roff(c.vr, i, j, k);
        double rv[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) rv[e] = R[e * c.vr.N];
#pragma unroll
        for (int e = 0; e < 8; ++e) R[e * c.vr.N] = rv[e] + coef * (sFX[e * NI * TT + q + 1] - sFX[e * NI * TT + q]);
      }
    }
  }
}


// Direction 0 with TMA, in two kernels.  First the theta-aware averages of
// the flux sums and total pressures on the final faces plus a one-face ring
// in j and k (the region of the Roe point dissipation), one thread per face,
// into the face scratch (F_FA0, F_PA0); it runs beside the Roe point
// dissipation.
__global__ void o4FaceAvg0Kernel(const Ctx* __restrict__ tab, const RegArgs rg, const WorkChunk* __restrict__ wk) {
  const WorkChunk wc = wk[blockIdx.x];
  const Ctx& c = tab[wc.box * 3 + 0];
  const Box3 PB = c.V0.growTrans(0, 1);
  forRegion(PB, wc, [&](int b, int i, int j, int k) {
    double fa[8], pa;
    chainAverage(c, 0, i, j, k, fa, pa);
    double* base = c.a.face + roff(c.fr, i, j, k);
    const long NF = c.fr.N;
#pragma unroll
    for (int e = 0; e < 8; ++e) base[(F_FA0 + e) * NF] = fa[e];
    base[F_PA0 * NF] = pa;
  });
}

// Then the chain itself: TI radial cells (TI + 1 faces) x TT rows of j per
// CTA, walking k over [c0, c1]; a ring of three k-slabs of the averages
// (8 + 1 arrays) and one of the point Roe dissipations (8 arrays), each slab
// TI + 2 radial x TT + 2 rows, copied by TMA, the slab k + 2 issued as soon
// as slab k - 1 is consumed.  Everything else as o4FaceChain0Kernel.
template <int TI>
struct Chain0Shape {
  static constexpr int TT = 128 / TI, NI = TI + 1, NTH = NI * TT;
  static constexpr int NX = TI + 2, NY = TT + 2, NXY = NX * NY;  // TMA slab: faces and one row either side
  static constexpr int SA = 9 * NXY, SQ = 8 * NXY;                  // doubles per averages / dissipation slab
  static constexpr int round16(int n) { return (n + 15) / 16 * 16; }
  // slots start on 128-byte boundaries, as a tensor copy's destination must
  static constexpr int PA = round16(SA), PQ = round16(SQ);
  static constexpr int oA = 0, oQ = 3 * PA, oFX = oQ + 3 * PQ, oBar = oFX + round16(8 * NTH);
  static constexpr int doubles() { return oBar + 6; }
};

template <int TI, int MB>
__global__ void __launch_bounds__(Chain0Shape<TI>::NTH, MB)
    o4FaceChain0TmaKernel(const Ctx* __restrict__ tab, const RegArgs rg, const ChainTile* __restrict__ tiles,
                          const CUtensorMap* __restrict__ maps) {
  using S = Chain0Shape<TI>;
  constexpr int TT = S::TT, NI = S::NI, NX = S::NX, NXY = S::NXY, NTH = S::NTH;
  extern __shared__ __align__(128) double smem[];
  double* sA = smem + S::oA;    // [3 slots][9][NY][NX]
  double* sQ = smem + S::oQ;    // [3 slots][8][NY][NX]
  double* sFX = smem + S::oFX;  // [8][NTH]
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(smem + S::oBar);  // [A 3][Q 3]
  const ChainTile tl = tiles[blockIdx.x];
  const Ctx& c = tab[tl.box * 3 + 0];
  const O4Args& a = c.a;
  const int tid = threadIdx.x;
  const double coef = -a.scale / a.G.dx[0];
  const int ihi = c.V.hi[0] + 1;
  const CUtensorMap* mapA = maps + (long)tl.box * kChainMaps + 4;
  const CUtensorMap* mapQ = mapA + 1;
  const int tx = tl.i0 - c.fr.lo[0], ty = tl.a0 - 1 - c.fr.lo[1];
  // slab k lives in slot (k - c0 + 1) % 3 and is that slot's ((k - c0 + 1) / 3)-th copy
  auto slot = [&](int k) { return (k - tl.c0 + 1) % 3; };
  auto use = [&](int k) { return (unsigned)((k - tl.c0 + 1) / 3) & 1u; };
  const int kLast = tl.c1 + 1;
  auto issue = [&](int k) {
    const int sl = slot(k);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbarExpect(&bar[sl], (unsigned)S::SA * sizeof(double));
    tmaLoad(sA + sl * S::PA, mapA, tx, ty, k - c.fr.lo[2], F_FA0, &bar[sl]);
    mbarExpect(&bar[3 + sl], (unsigned)S::SQ * sizeof(double));
    tmaLoad(sQ + sl * S::PQ, mapQ, tx, ty, k - c.fr.lo[2], F_QD, &bar[3 + sl]);
  };
  if (tid == 0) {
    for (int q = 0; q < 6; ++q) mbarInit(&bar[q]);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (tid == 0)
    for (int k = tl.c0 - 1; k <= tl.c0 + 1; ++k) issue(k);
  bool failed = false;
  for (int k = tl.c0; k <= tl.c1 && !failed; ++k) {
    bool ok = true;
    if (k == tl.c0) ok = mbarWait(&bar[slot(k - 1)], use(k - 1)) && mbarWait(&bar[3 + slot(k - 1)], use(k - 1)) &&
                        mbarWait(&bar[slot(k)], use(k)) && mbarWait(&bar[3 + slot(k)], use(k));
    ok = ok && mbarWait(&bar[slot(k + 1)], use(k + 1)) && mbarWait(&bar[3 + slot(k + 1)], use(k + 1));
    failed = __syncthreads_or(!ok);
    if (failed) break;
    const double* F0 = sA + slot(k) * S::PA;
    const double* Fm = sA + slot(k - 1) * S::PA;
    const double* Fp = sA + slot(k + 1) * S::PA;
    // (6, 7, 8) faces i0 .. i0+TI x rows a0 .. a0+TT-1 of row k: one thread each
    {
      const int q = tid, ii = tl.i0 + q % NI, jj = tl.a0 + q / NI;
      if (ii <= ihi && jj <= c.V.hi[1]) {
        const int o = (q / NI + 1) * NX + q % NI;  // (ii, jj) in a slab
        const double* M = faceRec(a.G, a.block0, 0, jj, k);
        const double* Mj1 = faceRec(a.G, a.block0, 0, jj + 1, k);
        const double* Mj0 = faceRec(a.G, a.block0, 0, jj - 1, k);
        const double* Mk1 = faceRec(a.G, a.block0, 0, jj, k + 1);
        const double* Mk0 = faceRec(a.G, a.block0, 0, jj, k - 1);
        double dM0[10], dM1[10];
#pragma unroll
        for (int e = 0; e < 10; ++e) {
          dM0[e] = 0.5 * Mj1[e] - 0.5 * Mj0[e];
          dM1[e] = 0.5 * Mk1[e] - 0.5 * Mk0[e];
        }
        double fa[8], dF0[8], dF1[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          fa[e] = F0[e * NXY + o];
          dF0[e] = 0.5 * F0[e * NXY + o + NX] - 0.5 * F0[e * NXY + o - NX];
          dF1[e] = 0.5 * Fp[e * NXY + o] - 0.5 * Fm[e * NXY + o];
        }
        double fm[8];
#pragma unroll
        for (int qq = 0; qq < 2; ++qq) {
          const int e = qq == 0 ? 0 : 4;
          double term = 0.0;
          term += dM0[9] * dF0[e] * (1.0 / 12.0);
          term += dM1[9] * dF1[e] * (1.0 / 12.0);
          term += M[9] * fa[e] * 1.0;
          fm[e] = 0.0 + term;
        }
#pragma unroll
        for (int bb = 0; bb < 2; ++bb) {
          const int bs = bb == 0 ? 1 : 5;
#pragma unroll
          for (int row = 0; row < 3; ++row) {
            double sum = 0.0;
#pragma unroll
            for (int col = 0; col < 3; ++col) {
              double term = 0.0;
              term += dM0[3 * row + col] * dF0[bs + col] * (1.0 / 12.0);
              term += dM1[3 * row + col] * dF1[bs + col] * (1.0 / 12.0);
              term += M[3 * row + col] * fa[bs + col] * 1.0;
              sum += term;
            }
            fm[bs + row] = sum;
          }
        }
        const double si = adjDr(a.G, 0, ii);
        double fs[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          double value = 0.0;
          value += fm[e] * si * 1.0;
          fs[e] = value;
        }
        auto t3 = [&](double pav) {
          double value = 0.0;
          value += pav * si * 1.0;
          return value;
        };
        const double* P0 = F0 + 8 * NXY;
        const double dT3[2] = {0.5 * t3(P0[o + NX]) - 0.5 * t3(P0[o - NX]),
                               0.5 * t3(Fp[8 * NXY + o]) - 0.5 * t3(Fm[8 * NXY + o])};
        // the five dissipation taps: the face, rows j -+ 1 of slab k, slabs k -+ 1
        const long so = (long)slot(k) * S::PQ + o;
        const QdTaps tap{sQ, NXY, {so, so - NX, so + NX, (long)slot(k - 1) * S::PQ + o, (long)slot(k + 1) * S::PQ + o}};
        double fx[8];
        chainFinal<0>(c, ii, jj, k, fs, t3(P0[o]), dT3, tap, fx);
        chainStore<0>(c, rg, ii, jj, k, fx);
#pragma unroll
        for (int e = 0; e < 8; ++e) sFX[e * NTH + q] = fx[e];
      }
    }
    __syncthreads();
    // slab k - 1 is consumed: its slots take slab k + 2
    if (tid == 0 && k + 2 <= kLast) issue(k + 2);
    // (9) divergence of the row's cells
    {
      const int li = tid % TI, lj = tid / TI;
      const int i = tl.i0 + li, j = tl.a0 + lj;
      if (tid < TI * TT && i <= c.V.hi[0] && j <= c.V.hi[1]) {
        const int q = lj * NI + li;
        double* R = a.rhs + roff(c.vr, i, j, k);
        double rv[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) rv[e] = R[e * c.vr.N];
#pragma unroll
        for (int e = 0; e < 8; ++e) R[e * c.vr.N] = rv[e] + coef * (sFX[e * NTH + q + 1] - sFX[e * NTH + q]);
      }
    }
    __syncthreads();
  }
  if (failed) {
    // A copy did not land: report it, wait (bounded) for the copies still in
    // flight, and make this tile's cells visibly invalid.
    if (tid == 0) {
      if (a.G.status) atomicExch(a.G.status, 1);
      for (int q = 0; q < 6; ++q) {
        mbarWait(&bar[q], 0u);
        mbarWait(&bar[q], 1u);
      }
    }
    __syncthreads();
    const int li = tid % TI, lj = tid / TI;
    const int i = tl.i0 + li, j = tl.a0 + lj;
    if (tid < TI * TT && i <= c.V.hi[0] && j <= c.V.hi[1])
      for (int k = tl.c0; k <= tl.c1; ++k)
#pragma unroll
        for (int e = 0; e < 8; ++e) a.rhs[roff(c.vr, i, j, k) + e * c.vr.N] = CUDART_NAN;
  }
}

}  // namespace

size_t o4CarveScratch(O4Args& a, double* sp) {
  Box3 V;
  for (int q = 0; q < 3; ++q) { V.lo[q] = a.vlo[q]; V.hi[q] = a.vhi[q]; }
  const Box3 G = V.grow(a.ghost);
  const size_t NG = (size_t)G.size(), NF = (size_t)faceBox(G).size(), N1 = (size_t)V.grow(1).size(),
               N2 = (size_t)V.grow(2).size(), nb = (size_t)a.nbox;
  size_t off = 0;
  auto take = [&](double*& dst, size_t n) {
    if (sp) dst = sp + off;
    off += (n + 31) / 32 * 32;  // 256-byte boundaries (TMA wants 16)
  };
  take(a.WA, nb * 8 * NG);
  take(a.WP, nb * 8 * NG);
  take(a.th, nb * NG);
  take(a.thr, nb * NG);
  take(a.face, nb * kO4FaceArrays * NF);
  take(a.face2, nb * kO4FaceArrays * NF);
  take(a.mj, nb * N1);
  take(a.kp, nb * 16 * N2);
  return off;
}

size_t o4ScratchDoubles(int nbox, const int vlo[3], const int vhi[3], int ghost) {
  O4Args a{};
  a.nbox = nbox;
  a.ghost = ghost;
  for (int q = 0; q < 3; ++q) { a.vlo[q] = vlo[q]; a.vhi[q] = vhi[q]; }
  return o4CarveScratch(a, nullptr);
}

// A batch: per box and direction the Ctx of a one-box O4Args, in device
// memory (the kernels' argument) and mirrored on the host (launch sizes).
struct O4Batch {
  int nbox = 0;
  Ctx* dev = nullptr;
  std::vector<Ctx> host;
  bool roe = false, powell = false;
  // work lists: per region kind and direction, chunks of kO4Chunk points of
  // every box's region, all in one device array
  WorkChunk* chunks = nullptr;
  long chunkOff[RG_COUNT][3] = {};
  int chunkCount[RG_COUNT][3] = {};
  int var[kO4TunedKernels] = {0, 0, 0};  // register-cap variant of the tuned kernels
  // tiles of the fused face chain, per direction, in one device array;
  // chainTI: radial width of an angular direction's tile (32, 16 or 8 by
  // the narrowest box); chainTI0 that of direction 0 (16 or 8: its tiles
  // are 8 rows of j deep, which halves the share of recomputed ring rows)
  ChainTile* chainTiles = nullptr;
  long chainOff[3] = {};
  int chainCount[3] = {};
  int chainTI = 32, chainTI0 = 16;
  // TMA tensor maps of the angular chains' face slabs, per box and direction
  // 1, 2: one copying 8 arrays, one copying 2 (device array; null without TMA)
  CUtensorMap* maps = nullptr;
  bool chainTma = false;
  // The Powell face chain of a direction (face flux, radial product,
  // divergence into -J div B) runs on a side stream beside the main face
  // chain: fork after the reconstruction, join before the next direction.
  // The cell-product coefficients and their averages (DivBPowell2's
  // inputs, from the point primitives) go first on the same side stream.
  cudaStream_t side = nullptr;
  cudaEvent_t pointEv = nullptr, forkEv[3] = {}, joinEv[3] = {};
  // The Roe point dissipation (reads the face states, writes only the
  // dissipation) runs on a second side stream beside the face-average,
  // mapped-flux and radial-product kernels, which do not read it; the final
  // flux waits for it.
  cudaStream_t roeSide = nullptr;
  cudaEvent_t roeFork[3] = {}, roeJoin[3] = {};
};

// Minimum resident CTAs per SM (the register cap) of each variant of the
// tuned kernels: reconstruction, Roe point dissipation, fused face chain.
// Variant 0 is the default.  A chain CTA has one thread per face of a tile
// row (132-144 threads); its shared memory (51-66 KB at 32-wide tiles)
// admits at most 4 (direction 0) or 3 (with TMA) CTAs per SM.
constexpr int kO4MinBlocks[kO4TunedKernels][kO4Variants] = {{6, 4, 8}, {4, 3, 5}, {3, 4, 2}};

// Tiles of the fused face chain of direction d over the batch's boxes: TI
// radial x 128/TI across (d = 0: j; d != 0: the other angular index),
// walking d (d != 0) or k (d = 0) in segments of S cells, S the largest of
// 64, 32, 16, 8 that still gives about 16 CTAs per SM.
void chainTiles(const std::vector<Ctx>& host, int nbox, int d, int TI, std::vector<ChainTile>& out) {
  const int TT = 128 / TI;
  const int across = d == 0 ? 1 : (d == 1 ? 2 : 1), walk = d == 0 ? 2 : d;
  long base = 0, longest = 1;
  for (int b = 0; b < nbox; ++b) {
    const Box3& V = host[(size_t)b * 3 + d].V;
    base += (long)((V.n(0) + TI - 1) / TI) * ((V.n(across) + TT - 1) / TT);
    longest = std::max<long>(longest, V.n(walk));
  }
  int S = 64;
  while (S > 8 && base * ((longest + S - 1) / S) < 148L * 16) S /= 2;
  for (int b = 0; b < nbox; ++b) {
    const Box3& V = host[(size_t)b * 3 + d].V;
    for (int c0 = V.lo[walk]; c0 <= V.hi[walk]; c0 += S)
      for (int a0 = V.lo[across]; a0 <= V.hi[across]; a0 += TT)
        for (int i0 = V.lo[0]; i0 <= V.hi[0]; i0 += TI)
          out.push_back(ChainTile{b, i0, a0, c0, std::min(c0 + S - 1, V.hi[walk])});
  }
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library), or null where it is unavailable.
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encodeTiled() {
  static EncodeTiledFn fn = []() -> EncodeTiledFn {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return nullptr;
    return reinterpret_cast<EncodeTiledFn>(p);
  }();
  return fn;
}

// The tensor maps of the angular face chains of every box of a batch:
// 4-D (radial, j, k, array) views of each box's face buffer for direction
// d = 1, 2, boxes of (TI + 4) radial x (TT + 4) angular x 1 normal x 8 or 2
// arrays.  False where a map cannot be made (then the chains read through
// L1 instead).
bool chainMaps(const std::vector<Ctx>& host, int nbox, int TI, int TI0, std::vector<CUtensorMap>& out) {
  const EncodeTiledFn enc = encodeTiled();
  if (!enc) return false;
  const int TT = 128 / TI, TT0 = 128 / TI0;
  out.resize((size_t)nbox * kChainMaps);
  for (int b = 0; b < nbox; ++b) {
    // direction 0: slabs of TI0 + 2 radial faces (an even count from an even
    // offset) x TT0 + 2 rows of j x one k
    {
      const Ctx& c = host[(size_t)b * 3];
      const cuuint64_t n0 = c.fr.n[0], n1 = c.fr.n[1], n2 = c.fr.n[2];
      if ((reinterpret_cast<uintptr_t>(c.a.face) & 15) || (n0 & 1) || ((c.V.lo[0] - c.fr.lo[0]) & 1)) return false;
      const cuuint64_t dims[4] = {n0, n1, n2, (cuuint64_t)kO4FaceArrays};
      const cuuint64_t strides[3] = {n0 * 8, n0 * n1 * 8, n0 * n1 * n2 * 8};
      for (int w = 0; w < 2; ++w) {
        const cuuint32_t box[4] = {(cuuint32_t)(TI0 + 2), (cuuint32_t)(TT0 + 2), 1u, w == 0 ? 9u : 8u};
        const cuuint32_t es[4] = {1, 1, 1, 1};
        if (enc(&out[(size_t)b * kChainMaps + 4 + w], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, c.a.face, dims, strides,
                box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
          return false;
      }
    }
    for (int d = 1; d <= 2; ++d) {
      const Ctx& c = host[(size_t)b * 3 + d];
      const cuuint64_t n0 = c.fr.n[0], n1 = c.fr.n[1], n2 = c.fr.n[2];
      // 16-byte aligned base and rows, and an even radial tile origin
      // (tiles start at the valid box's low radial index, i0 - 2 - fr.lo)
      if ((reinterpret_cast<uintptr_t>(c.a.face) & 15) || (n0 & 1) || ((c.V.lo[0] - 2 - c.fr.lo[0]) & 1)) return false;
      const cuuint64_t dims[4] = {n0, n1, n2, (cuuint64_t)kO4FaceArrays};
      const cuuint64_t strides[3] = {n0 * 8, n0 * n1 * 8, n0 * n1 * n2 * 8};
      for (int w = 0; w < 2; ++w) {
        const cuuint32_t box[4] = {(cuuint32_t)(TI + 4), d == 1 ? 1u : (cuuint32_t)(TT + 4),
                                   d == 1 ? (cuuint32_t)(TT + 4) : 1u, w == 0 ? 8u : 2u};
        const cuuint32_t es[4] = {1, 1, 1, 1};
        if (enc(&out[(size_t)b * kChainMaps + (d - 1) * 2 + w], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, c.a.face, dims,
                strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
          return false;
      }
    }
  }
  return true;
}

// Dynamic shared memory of the angular chain kernels (with and without TMA).
template <int TI, bool TMA>
cudaError_t chainSmemT() {
  const int bytes = ChainShape<TI>::doubles(TMA) * (int)sizeof(double);
  cudaError_t e = cudaSuccess;
#define HC_CHAIN_ATTR(D, MB)                                                                                \
  if (e == cudaSuccess)                                                                                    \
    e = cudaFuncSetAttribute(o4FaceChainKernel<D, TI, MB, TMA>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  HC_CHAIN_ATTR(1, 2) HC_CHAIN_ATTR(1, 3) HC_CHAIN_ATTR(1, 4) HC_CHAIN_ATTR(2, 2) HC_CHAIN_ATTR(2, 3) HC_CHAIN_ATTR(2, 4)
#undef HC_CHAIN_ATTR
  return e;
}

template <int TI>
cudaError_t chain0TmaSmem() {
  const int bytes = Chain0Shape<TI>::doubles() * (int)sizeof(double);
  cudaError_t e = cudaFuncSetAttribute(o4FaceChain0TmaKernel<TI, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(o4FaceChain0TmaKernel<TI, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(o4FaceChain0TmaKernel<TI, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  return e;
}

template <int TI>
cudaError_t chain0Smem() {
  const int bytes = chain0Doubles<TI>() * (int)sizeof(double);
  cudaError_t e = cudaFuncSetAttribute(o4FaceChain0Kernel<TI, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(o4FaceChain0Kernel<TI, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(o4FaceChain0Kernel<TI, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  return e;
}

void o4BatchSetVariants(O4Batch* B, const int v[kO4TunedKernels]) {
  for (int q = 0; q < kO4TunedKernels; ++q) B->var[q] = v[q] >= 0 && v[q] < kO4Variants ? v[q] : 0;
}

int o4VariantMinBlocks(int kernel, int variant) {
  return kernel >= 0 && kernel < kO4TunedKernels && variant >= 0 && variant < kO4Variants ? kO4MinBlocks[kernel][variant]
                                                                                          : 0;
}

O4Batch* o4BatchCreate(const O4Args* boxes, int nbox, cudaError_t* err) {
  *err = cudaSuccess;
  if (nbox <= 0 || nbox > 65535) {
    *err = cudaErrorInvalidValue;
    return nullptr;
  }
  for (int b = 0; b < nbox; ++b)
    if (boxes[b].ur.N >= 0x7fffffffL) {  // roff forms offsets in 32 bits
      *err = cudaErrorInvalidValue;
      return nullptr;
    }
  O4Batch* B = new O4Batch;
  B->nbox = nbox;
  B->host.resize((size_t)nbox * 3);
  for (int b = 0; b < nbox; ++b) {
    O4Args one = boxes[b];
    one.nbox = 1;
    for (int d = 0; d < 3; ++d) B->host[(size_t)b * 3 + d] = makeCtx(one, d);
  }
  B->roe = boxes[0].G.roe;
  B->powell = boxes[0].G.powell;
  std::vector<WorkChunk> work;
  for (int id = 0; id < RG_COUNT; ++id)
    for (int d = 0; d < 3; ++d) {
      B->chunkOff[id][d] = (long)work.size();
      long total = 0, largest = 0;
      bool equal = true;
      for (int b = 0; b < nbox; ++b) {
        const long n = regionOf(B->host[(size_t)b * 3 + d], id).size();
        if (n >= 0x7fffffffL) {  // forRegion splits indices in 32 bits
          *err = cudaErrorInvalidValue;
          o4BatchDestroy(B);
          return nullptr;
        }
        total += n;
        equal = equal && (b == 0 || n == largest);
        largest = n > largest ? n : largest;
      }
      if (equal) {
        // boxes of one size: each box's CTAs stride over it together
        // (about 148 x 32 CTAs in all)
        const long need = (largest + 127) / 128;
        const long perBox = std::max(1L, std::min(need, 148L * 32 / nbox));
        for (int b = 0; b < nbox; ++b)
          for (long x = 0; x < perBox; ++x) work.push_back(WorkChunk{b, (int)(perBox * 128), x * 128, largest});
      } else {
        // uneven boxes: contiguous chunks of equal work
        const long chunk = chunkPoints(total);
        for (int b = 0; b < nbox; ++b) {
          const long n = regionOf(B->host[(size_t)b * 3 + d], id).size();
          for (long t = 0; t < n; t += chunk) work.push_back(WorkChunk{b, 128, t, t + chunk < n ? t + chunk : n});
        }
      }
      const long count = (long)work.size() - B->chunkOff[id][d];
      if (count > 0x7fffffffL) {
        *err = cudaErrorInvalidValue;
        o4BatchDestroy(B);
        return nullptr;
      }
      B->chunkCount[id][d] = (int)count;
    }
  {
    int narrow = 1 << 30;
    for (int b = 0; b < nbox; ++b) narrow = std::min(narrow, B->host[(size_t)b * 3].V.n(0));
    B->chainTI = narrow >= 24 ? 32 : narrow >= 12 ? 16 : 8;
    B->chainTI0 = narrow >= 12 ? 16 : 8;
  }
  std::vector<ChainTile> tiles;
  for (int d = 0; d < 3; ++d) {
    B->chainOff[d] = (long)tiles.size();
    chainTiles(B->host, nbox, d, d == 0 ? B->chainTI0 : B->chainTI, tiles);
    const long count = (long)tiles.size() - B->chainOff[d];
    if (count > 0x7fffffffL) {
      *err = cudaErrorInvalidValue;
      o4BatchDestroy(B);
      return nullptr;
    }
    B->chainCount[d] = (int)count;
  }
  *err = B->chainTI0 == 16 ? chain0Smem<16>() : chain0Smem<8>();
  if (*err == cudaSuccess)
    *err = B->chainTI == 32   ? chainSmemT<32, false>()
           : B->chainTI == 16 ? chainSmemT<16, false>()
                              : chainSmemT<8, false>();
  {
    std::vector<CUtensorMap> maps;
    if (*err == cudaSuccess && chainMaps(B->host, nbox, B->chainTI, B->chainTI0, maps)) {
      cudaError_t e = B->chainTI == 32   ? chainSmemT<32, true>()
                      : B->chainTI == 16 ? chainSmemT<16, true>()
                                         : chainSmemT<8, true>();
      if (e == cudaSuccess) e = B->chainTI0 == 16 ? chain0TmaSmem<16>() : chain0TmaSmem<8>();
      if (e == cudaSuccess) e = cudaMalloc(&B->maps, sizeof(CUtensorMap) * maps.size());
      if (e == cudaSuccess)
        e = cudaMemcpy(B->maps, maps.data(), sizeof(CUtensorMap) * maps.size(), cudaMemcpyHostToDevice);
      B->chainTma = e == cudaSuccess;
      if (e != cudaSuccess) cudaGetLastError();  // no TMA: the chains read through L1
    }
  }
  if (*err == cudaSuccess) *err = cudaMalloc(&B->chainTiles, sizeof(ChainTile) * std::max<size_t>(1, tiles.size()));
  if (*err == cudaSuccess && !tiles.empty())
    *err = cudaMemcpy(B->chainTiles, tiles.data(), sizeof(ChainTile) * tiles.size(), cudaMemcpyHostToDevice);
  if (*err == cudaSuccess) *err = cudaMalloc(&B->dev, sizeof(Ctx) * B->host.size());
  if (*err == cudaSuccess) *err = cudaMemcpy(B->dev, B->host.data(), sizeof(Ctx) * B->host.size(), cudaMemcpyHostToDevice);
  if (*err == cudaSuccess && !work.empty()) {
    *err = cudaMalloc(&B->chunks, sizeof(WorkChunk) * work.size());
    if (*err == cudaSuccess)
      *err = cudaMemcpy(B->chunks, work.data(), sizeof(WorkChunk) * work.size(), cudaMemcpyHostToDevice);
  }
  if (*err == cudaSuccess && B->roe) {
    *err = cudaStreamCreateWithFlags(&B->roeSide, cudaStreamNonBlocking);
    for (int d = 0; d < 3 && *err == cudaSuccess; ++d) {
      *err = cudaEventCreateWithFlags(&B->roeFork[d], cudaEventDisableTiming);
      if (*err == cudaSuccess) *err = cudaEventCreateWithFlags(&B->roeJoin[d], cudaEventDisableTiming);
    }
  }
  if (*err == cudaSuccess && B->powell) {
    *err = cudaStreamCreateWithFlags(&B->side, cudaStreamNonBlocking);
    if (*err == cudaSuccess) *err = cudaEventCreateWithFlags(&B->pointEv, cudaEventDisableTiming);
    for (int d = 0; d < 3 && *err == cudaSuccess; ++d) {
      *err = cudaEventCreateWithFlags(&B->forkEv[d], cudaEventDisableTiming);
      if (*err == cudaSuccess) *err = cudaEventCreateWithFlags(&B->joinEv[d], cudaEventDisableTiming);
    }
  }
  if (*err != cudaSuccess) {
    o4BatchDestroy(B);
    return nullptr;
  }
  return B;
}

void o4BatchDestroy(O4Batch* B) {
  if (!B) return;
  if (B->dev) cudaFree(B->dev);
  if (B->chunks) cudaFree(B->chunks);
  if (B->chainTiles) cudaFree(B->chainTiles);
  if (B->maps) cudaFree(B->maps);
  if (B->pointEv) cudaEventDestroy(B->pointEv);
  for (int d = 0; d < 3; ++d) {
    if (B->roeFork[d]) cudaEventDestroy(B->roeFork[d]);
    if (B->roeJoin[d]) cudaEventDestroy(B->roeJoin[d]);
    if (B->forkEv[d]) cudaEventDestroy(B->forkEv[d]);
    if (B->joinEv[d]) cudaEventDestroy(B->joinEv[d]);
  }
  if (B->side) cudaStreamDestroy(B->side);
  if (B->roeSide) cudaStreamDestroy(B->roeSide);
  delete B;
}

void o4SplitArgs(const O4Args& a, std::vector<O4Args>& out) {
  const Ctx c = makeCtx(a, 0);
  out.assign(a.nbox, a);
  for (int b = 0; b < a.nbox; ++b) {
    O4Args& o = out[b];
    o.nbox = 1;
    o.block0 = a.block0 + b;
    o.U = a.U + (long)b * a.uStride;
    o.rhs = a.rhs + (long)b * a.rhsStride;
    for (int d = 0; d < 3; ++d)
      if (a.flux[d]) o.flux[d] = a.flux[d] + (long)b * 8 * c.V.extrude(d).size();
    o.WA = a.WA + (long)b * 8 * c.gr.N;
    o.WP = a.WP + (long)b * 8 * c.gr.N;
    o.th = a.th + (long)b * c.gr.N;
    o.thr = a.thr + (long)b * c.gr.N;
    o.face = a.face + (long)b * kO4FaceArrays * c.fr.N;
    o.face2 = a.face2 + (long)b * kO4FaceArrays * c.fr.N;
    o.mj = a.mj + (long)b * c.v1r.N;
    o.kp = a.kp + (long)b * 16 * c.v2r.N;
  }
}

namespace {
}  // namespace

cudaError_t launchO4BatchGravity(const O4Batch* B, cudaStream_t s) {
  const RegArgs none{};
  if (B->chunkCount[RG_V][0] == 0) return cudaSuccess;
  o4GravityKernel<<<B->chunkCount[RG_V][0], 128, 0, s>>>(B->dev, none, B->chunks + B->chunkOff[RG_V][0]);
  return cudaGetLastError();
}

// The fused face chain of direction d over the batch's tiles.
template <int TI, int MB>
cudaError_t launchChainT(const O4Batch* B, const RegArgs& rg, int d, cudaStream_t s) {
  const int n = B->chainCount[d];
  const ChainTile* t = B->chainTiles + B->chainOff[d];
  if (n == 0) return cudaSuccess;
  const size_t smemTma = ChainShape<TI>::doubles(true) * sizeof(double);
  const size_t smemL1 = ChainShape<TI>::doubles(false) * sizeof(double);
  if (d == 0 && B->chainTma)
    o4FaceChain0TmaKernel<TI, MB><<<n, Chain0Shape<TI>::NTH, Chain0Shape<TI>::doubles() * sizeof(double), s>>>(
        B->dev, rg, t, B->maps);
  else if (d == 0)
    o4FaceChain0Kernel<TI, MB><<<n, chain0Threads<TI>(), chain0Doubles<TI>() * sizeof(double), s>>>(B->dev, rg, t);
  else if (d == 1 && B->chainTma)
    o4FaceChainKernel<1, TI, MB, true><<<n, ChainShape<TI>::NTH, smemTma, s>>>(B->dev, rg, t, B->maps);
  else if (d == 1)
    o4FaceChainKernel<1, TI, MB, false><<<n, ChainShape<TI>::NTH, smemL1, s>>>(B->dev, rg, t, nullptr);
  else if (B->chainTma)
    o4FaceChainKernel<2, TI, MB, true><<<n, ChainShape<TI>::NTH, smemTma, s>>>(B->dev, rg, t, B->maps);
  else
    o4FaceChainKernel<2, TI, MB, false><<<n, ChainShape<TI>::NTH, smemL1, s>>>(B->dev, rg, t, nullptr);
  return cudaGetLastError();
}

template <int TI>
cudaError_t launchChainV(const O4Batch* B, const RegArgs& rg, int d, cudaStream_t s) {
  switch (kO4MinBlocks[2][B->var[2]]) {
    case 2: return launchChainT<TI, 2>(B, rg, d, s);
    case 4: return launchChainT<TI, 4>(B, rg, d, s);
    default: return launchChainT<TI, 3>(B, rg, d, s);
  }
}

cudaError_t launchChain(const O4Batch* B, const RegArgs& rg, int d, cudaStream_t s) {
  if (d == 0) return B->chainTI0 == 16 ? launchChainV<16>(B, rg, d, s) : launchChainV<8>(B, rg, d, s);
  if (B->chainTI == 32) return launchChainV<32>(B, rg, d, s);
  if (B->chainTI == 16) return launchChainV<16>(B, rg, d, s);
  return launchChainV<8>(B, rg, d, s);
}

cudaError_t launchO4Batch(const O4Batch* B, const RegArgs* reg, cudaStream_t s) {
  const RegArgs none{};
  const RegArgs rg = reg ? *reg : none;
  const Ctx* t = B->dev;
  cudaError_t e;
  cudaStream_t st = s;  // the stream the macros below launch on
#define HC_LAUNCH(kernel, d, region)                                                           \
  if (B->chunkCount[region][d]) {                                                              \
    kernel<<<B->chunkCount[region][d], 128, 0, st>>>(t, rg, B->chunks + B->chunkOff[region][d]); \
    if ((e = cudaGetLastError()) != cudaSuccess) return e;                                     \
  }
#define HC_LAUNCH_D(kernel, region)                                                      \
  if (d == 0) { HC_LAUNCH(kernel<0>, 0, region) }                                       \
  else if (d == 1) { HC_LAUNCH(kernel<1>, 1, region) }                                  \
  else { HC_LAUNCH(kernel<2>, 2, region) }
#define HC_LAUNCH_DM(kernel, q, region)                                                  \
  if (B->var[q] == 1) { HC_LAUNCH_DV(kernel, kO4MinBlocks[q][1], region) }                \
  else if (B->var[q] == 2) { HC_LAUNCH_DV(kernel, kO4MinBlocks[q][2], region) }           \
  else { HC_LAUNCH_DV(kernel, kO4MinBlocks[q][0], region) }
#define HC_LAUNCH_T(d, region, ...)                                                                \
  if (B->chunkCount[region][d]) {                                                                  \
    __VA_ARGS__<<<B->chunkCount[region][d], 128, 0, st>>>(t, rg, B->chunks + B->chunkOff[region][d]); \
    if ((e = cudaGetLastError()) != cudaSuccess) return e;                                         \
  }
#define HC_LAUNCH_DV(kernel, mb, region)                                                 \
  if (d == 0) { HC_LAUNCH_T(0, region, kernel<0, mb>) }                                 \
  else if (d == 1) { HC_LAUNCH_T(1, region, kernel<1, mb>) }                            \
  else { HC_LAUNCH_T(2, region, kernel<2, mb>) }
  HC_LAUNCH(o4PrimAvgKernel, 0, RG_G)
  HC_LAUNCH(o4ThetaRawKernel, 0, RG_GR)
  HC_LAUNCH(o4PointKernel, 0, RG_G)
  if (B->powell) {
    // DivBPowell2's coefficients need only the point primitives: fork them
    // (the side stream runs them before the first direction's Powell chain)
    if ((e = cudaEventRecord(B->pointEv, s)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(B->side, B->pointEv, 0)) != cudaSuccess) return e;
    st = B->side;
    HC_LAUNCH(o4PowellCoefKernel, 0, RG_V2)
    HC_LAUNCH(o4PowellAvgKernel, 0, RG_V1)
    st = s;
  }
  // Direction d's face arrays are face buffer d & 1 (direction 1 has its
  // own), so the passes overlap: the Roe point dissipation of d (second side
  // stream) runs beside the face chain of d - 1 and the reconstruction of
  // d + 1 on the main stream; the Powell face chain of d (first side stream)
  // beside them.  The reconstruction of d + 2 reuses d's buffer and waits
  // for d's Powell chain; d's face chain waits for d's Roe dissipation;
  // the chains add into rhs in direction order on the main stream.
  for (int d = 0; d < 3; ++d) {
    if (d >= 2 && B->powell && (e = cudaStreamWaitEvent(s, B->joinEv[d - 2], 0)) != cudaSuccess) return e;
    HC_LAUNCH_DM(o4FaceReconKernel, 0, RG_F)
    // direction 0's face averages for its TMA chain (beside the Roe point
    // dissipation, which reads neither their inputs' outputs nor them)
    if (d == 0 && B->chainTma) { HC_LAUNCH(o4FaceAvg0Kernel, 0, RG_PB) }
    if (B->powell) {
      // the Powell chain reads the reconstruction's flags and normal B and
      // writes only its own face arrays and -J div B: fork it
      if ((e = cudaEventRecord(B->forkEv[d], s)) != cudaSuccess) return e;
      if ((e = cudaStreamWaitEvent(B->side, B->forkEv[d], 0)) != cudaSuccess) return e;
      st = B->side;
      HC_LAUNCH_D(o4PowellFluxKernel, RG_PF)
      HC_LAUNCH_D(o4PowellProdKernel, RG_PP)
      HC_LAUNCH_D(o4PowellDivKernel, RG_V1)
      st = s;
      if ((e = cudaEventRecord(B->joinEv[d], B->side)) != cudaSuccess) return e;
    }
    if (B->roe) {
      if ((e = cudaEventRecord(B->roeFork[d], s)) != cudaSuccess) return e;
      if ((e = cudaStreamWaitEvent(B->roeSide, B->roeFork[d], 0)) != cudaSuccess) return e;
      st = B->roeSide;
      HC_LAUNCH_DM(o4RoePointKernel, 1, RG_PB)
      st = s;
      if ((e = cudaEventRecord(B->roeJoin[d], B->roeSide)) != cudaSuccess) return e;
    }
    if (d >= 1) {
      if (B->roe && (e = cudaStreamWaitEvent(s, B->roeJoin[d - 1], 0)) != cudaSuccess) return e;
      if ((e = launchChain(B, rg, d - 1, s)) != cudaSuccess) return e;
    }
  }
  if (B->roe && (e = cudaStreamWaitEvent(s, B->roeJoin[2], 0)) != cudaSuccess) return e;
  if ((e = launchChain(B, rg, 2, s)) != cudaSuccess) return e;
  for (int d = 0; d < 3 && B->powell; ++d)
    if ((e = cudaStreamWaitEvent(s, B->joinEv[d], 0)) != cudaSuccess) return e;
  // after the last join: -J div B complete, coefficients averaged
  if (B->powell) { HC_LAUNCH(o4PowellApplyKernel, 0, RG_V) }
#undef HC_LAUNCH_DV
#undef HC_LAUNCH_T
#undef HC_LAUNCH_DM
#undef HC_LAUNCH_D
#undef HC_LAUNCH
  return cudaSuccess;
}

}  // namespace hc

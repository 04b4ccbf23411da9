// sm_100a kernels of the second-order (PLM) per-box MHD update and the RK4
// stage that consumes it.  FP64 throughout.
//
// o2StageKernel -- one CTA per X x Y x Z cell tile (Tile) of one box.  Phase 1
// computes every face of the tile in all three directions (flat loop over
// faces, radial index fastest so stencil loads are coalesced) and keeps the
// face fluxes in shared memory; phase 2 forms the flux divergence, Powell and
// gravity sources per cell and either accumulates the per-box rhs or applies
// the RK4 stage update in registers (k never goes to HBM).
#include <cuda_runtime.h>
#include <stdint.h>

#include "hc_device.cuh"
#include "hc_level.h"

namespace hc {

namespace {

// Cell tiles of o2StageKernel: X x Y x Z cells per CTA (128 threads, one
// cell each) and the minimum resident CTAs per SM that caps the registers
// (Rusanov, Roe).  The autotuner (hc_ctx_autotune) times them per limiter /
// solver pair on the caller's level; every tile computes every face and cell
// with the same arithmetic, so results do not depend on the choice.
template <int X, int Y, int Z, int MB_RUS, int MB_ROE>
struct Tile {
  static constexpr int TX = X, TY = Y, TZ = Z, NT = X * Y * Z;
  static constexpr int NF0 = (X + 1) * Y * Z, NF1 = X * (Y + 1) * Z, NF2 = X * Y * (Z + 1);
  static constexpr int NF = NF0 + NF1 + NF2;
  static constexpr int minBlocks(bool roe) { return roe ? MB_ROE : MB_RUS; }
};
using Tile0 = Tile<16, 4, 2, 3, 2>;
using Tile1 = Tile<32, 2, 2, 3, 2>;
using Tile2 = Tile<8, 8, 2, 3, 2>;
using Tile3 = Tile<16, 2, 4, 3, 2>;
using Tile4 = Tile<16, 4, 2, 4, 3>;
using Tile5 = Tile<32, 4, 1, 3, 2>;
static_assert(Tile0::NT == 128 && Tile1::NT == 128 && Tile2::NT == 128 && Tile3::NT == 128 && Tile4::NT == 128 &&
                  Tile5::NT == 128,
              "stage tiles are 128 threads");

__device__ __forceinline__ long cellOffset(int i, int j, int k, const int lo[3], const int n[3]) {
  return (long)(i - lo[0]) + (long)n[0] * ((long)(j - lo[1]) + (long)n[1] * (long)(k - lo[2]));
}

// Cartesian primitives from native conserved u through the cell basis A
// (src/BoxOp_SecondOrderPreStage.H:199-214).
__device__ __forceinline__ void nativeToPrimitive(const double u[8], const double* A, double gamma, double out[8]) {
  double ww[8];
  ww[0] = u[0];
  ww[4] = u[4];
#pragma unroll
  for (int grp = 0; grp < 2; ++grp) {
    const int st = grp == 0 ? 1 : 5;
#pragma unroll
    for (int d = 0; d < 3; ++d) ww[st + d] = A[3 * d] * u[st] + A[3 * d + 1] * u[st + 1] + A[3 * d + 2] * u[st + 2];
  }
  cartesianPrimitiveFromConserved(out, ww, 1.0, gamma);
}

// Inlet of the cone clouds crossing the inner boundary at time t into the
// native conserved ghost state u at Cartesian position pos
// (src/BoxOp_PreStage.H:329-400, finite clouds: the inlet state is sampled on
// the physical boundary sphere; taper weight 1).  A: cell basis, Ai: its
// inverse.
__device__ void inletGhost(const DevLevel& L, double t, const double pos[3], const double* A, const double* Ai,
                           double u[8]) {
  const double radius = sqrt(pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2]);
  for (int s = 0; s < L.ninlet; ++s) {
    const InletCone c = L.inlet[s];
    if (!(t >= c.insertionTime && t < c.endTime)) continue;
    const double shift = c.entryShift + c.speed * 1e5 * (t - c.entryTime);
    const double face[3] = {pos[0] * L.r0 / radius, pos[1] * L.r0 / radius, pos[2] * L.r0 / radius};
    const double q0 = face[0] - shift * c.axis[0], q1 = face[1] - shift * c.axis[1], q2 = face[2] - shift * c.axis[2];
    if (sqrt(q0 * q0 + q1 * q1 + q2 * q2) > c.radius) continue;
    const double fr = sqrt(face[0] * face[0] + face[1] * face[1] + face[2] * face[2]) / kSolarRadiusCm;
    if (!(fr > 0)) continue;
    double v[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) v[d] = c.speed * 1e5 * face[d] / (kSolarRadiusCm * fr);
    double old[8] = {u[0], 0, 0, 0, 0, 0, 0, 0};
    double ke = 0, me = 0, radialOld = 0, radialCME = 0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        old[1 + d] += A[3 * d + q] * u[1 + q] / old[0];
        old[5 + d] += A[3 * d + q] * u[5 + q];
      }
      ke += .5 * old[0] * old[1 + d] * old[1 + d];
      me += old[5 + d] * old[5 + d] / (8 * kPi);
      radialOld += old[1 + d] * pos[d] / radius;
      radialCME += v[d] * pos[d] / radius;
    }
    old[4] = fmax(0., (u[4] - ke - me) * (L.gamma - 1));
#pragma unroll
    for (int d = 0; d < 3; ++d) v[d] = radialCME * pos[d] / radius;
    // taperBoundarySource with weight 1, then increment() with the
    // prescribed cone plasma (src/MHD_CME.H:982-990, 1215-1238)
    const double weight = 1;
#pragma unroll
    for (int d = 0; d < 3; ++d) v[d] = old[1 + d] + weight * (v[d] - old[1 + d]);
    const double density = (1 - weight) * old[0] + weight * c.density;
    double oldKinetic = 0, newKinetic = 0, oldMagnetic = 0, newMagnetic = 0, delta[8];
    delta[0] = density - old[0];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      delta[1 + d] = density * v[d] - old[0] * old[1 + d];
      delta[5 + d] = 0.0;
      oldKinetic += .5 * old[0] * old[1 + d] * old[1 + d];
      newKinetic += .5 * density * v[d] * v[d];
      oldMagnetic += old[5 + d] * old[5 + d] / (8 * kPi);
      newMagnetic += (old[5 + d] + 0.0) * (old[5 + d] + 0.0) / (8 * kPi);
    }
    const double target = 2 * 1.380649e-16 * c.temperature * c.density / kMP;
    const double pressure = (1 - weight) * fmax(0., old[4]) + weight * target;
    delta[4] = (pressure - fmax(0., old[4])) / (L.gamma - 1) + newKinetic - oldKinetic + newMagnetic - oldMagnetic;
    u[0] += delta[0];
    u[4] += delta[4];
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        u[1 + d] += Ai[3 * d + q] * delta[1 + q];
        u[5 + d] += Ai[3 * d + q] * delta[5 + q];
      }
  }
}

// Analytic inner wind, src/BoxOp_PreStage.H:7-47 (time-dependent form).
__device__ void analyticWind(const DevLevel& L, const double X[3], double t, double u[8]) {
  windConserved(L.gamma, L.r0, L.strength, X, t, u);
}

// ---------------------------------------------------------------------------
// One face of the second-order operator (src/BoxOp_SecondOrder.H:257-324).
// ---------------------------------------------------------------------------
template <int LIM, bool ROE, int MODE>
__device__ __forceinline__ void o2Face(const StageArgs& a, const double* __restrict__ w, int block, int dir, int i,
                                       int j, int k, double out[8], double& bf, bool powell) {
  const DevLevel& L = a.L;
  const long sN = a.wN;
  const long c0 = cellOffset(i, j, k, a.wlo, a.wn);
  const long step = dir == 0 ? 1L : dir == 1 ? (long)a.wn[0] : (long)a.wn[0] * a.wn[1];
  double l[8], r[8];
#pragma unroll
  for (int q = 0; q < NC; ++q) {
    const double* s = w + q * sN + c0;
    plmComponent<LIM>(__ldg(s - 2 * step), __ldg(s - step), __ldg(s), __ldg(s + step), l[q], r[q]);
  }
  // Complete-state fallbacks (src/BoxOp_SecondOrder.H:32-36).
  if (!(l[0] >= kRHO00 && l[4] >= 0)) {
#pragma unroll
    for (int q = 0; q < NC; ++q) l[q] = __ldg(w + q * sN + c0 - step);
  }
  if (!(r[0] >= kRHO00 && r[4] >= 0)) {
#pragma unroll
    for (int q = 0; q < NC; ++q) r[q] = __ldg(w + q * sN + c0);
  }
  if (dir > 0) {
    const int idx = dir == 1 ? j : k;
    if (MODE == MODE_BOX) {
      // Caller-supplied adjacent-panel states (src/BoxOp_SecondOrder.H:252-281).
      const double* pl = a.panel[2 * dir];
      const double* ph = a.panel[2 * dir + 1];
      const bool atLo = pl && idx == a.lo[dir], atHi = ph && idx == a.hi[dir] + 1;
      if (atLo || atHi) {
        const int v0 = a.hi[0] - a.lo[0] + 1, v1 = a.hi[1] - a.lo[1] + 1, v2 = a.hi[2] - a.lo[2] + 1;
        const int s1 = dir == 1 ? 1 : v1;
        const long sidx = (long)(i - a.lo[0]) + (long)v0 * ((dir == 1 ? 0 : j - a.lo[1]) + (long)s1 * (dir == 2 ? 0 : k - a.lo[2]));
        const long sN2 = (long)v0 * s1 * (dir == 2 ? 1 : v2);
        const double* src = atLo ? pl : ph;
        double* dst = atLo ? l : r;
#pragma unroll
        for (int q = 0; q < NC; ++q) dst[q] = src[q * sN2 + sidx];
      }
    } else if (a.seams && (idx == 0 || idx == L.na)) {
      // Shared seam state: the adjacent panel's reconstruction from its own
      // cells at the same physical face (src/BoxOp_SecondOrder.H:68-121).
      const int side = idx == 0 ? 0 : 1;
      const int e = (block * 2 + (dir - 1)) * 2 + side;
      const EdgeLink lk = L.edge[e];
      const int s2 = L.faceMap[e * L.na + (dir == 1 ? k : j)];
      const double* wn = a.w + (long)lk.nb * a.wBoxStride;
      const int first = lk.side == 0 ? -1 : L.na - 2;
      double st[3][8];
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        const int n = first + q;
        const long o = lk.axis == 1 ? cellOffset(i, n, s2, a.wlo, a.wn) : cellOffset(i, s2, n, a.wlo, a.wn);
#pragma unroll
        for (int c = 0; c < NC; ++c) st[q][c] = __ldg(wn + c * sN + o);
      }
      if (lk.side == 0) {
        if (side == 0) plmRight<LIM>(st[0], st[1], st[2], l);
        else plmRight<LIM>(st[0], st[1], st[2], r);
      } else {
        if (side == 0) plmLeft<LIM>(st[0], st[1], st[2], l);
        else plmLeft<LIM>(st[0], st[1], st[2], r);
      }
    }
  }
  const FaceGeom& g = L.face[((size_t)dir * 6 + block) * (L.na + 1) * (L.na + 1) + (size_t)k * (L.na + 1) + j];
  if (MODE == MODE_RK && dir == 0 && i == 0 && L.ninlet) {
    // Inlet footprint on the inner face (src/BoxOp_SecondOrder.H:175-181,
    // 282-311): where an emerging cloud covers the face, the interior state
    // is extrapolated from owned cells only and the ghost side takes the
    // interior's normal field.
    const double dtS = a.invDtMax ? L.cfl_number / *a.invDtMax : a.dtv;
    constexpr double c4[4] = {0, 0.5, 0.5, 1};
    const double t = a.tbase + (a.tdev ? *a.tdev : 0.0) + c4[a.stage] * dtS;
    bool footprint = false;
    for (int s = 0; s < L.ninlet && !footprint; ++s) {
      const InletCone c = L.inlet[s];
      if (!(t >= c.insertionTime && t < c.endTime)) continue;
      const double shift = c.entryShift + c.speed * 1e5 * (t - c.entryTime);
      const double pos[3] = {L.r0 * g.f[0], L.r0 * g.f[1], L.r0 * g.f[2]};
      const double q0 = pos[0] - shift * c.axis[0], q1 = pos[1] - shift * c.axis[1], q2 = pos[2] - shift * c.axis[2];
      if (sqrt(q0 * q0 + q1 * q1 + q2 * q2) > c.radius) continue;
      footprint = sqrt(pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2]) / kSolarRadiusCm > 0;
    }
    if (footprint) {
#pragma unroll
      for (int q = 0; q < NC; ++q) {
        const double cc = __ldg(w + q * sN + c0), pp = __ldg(w + q * sN + c0 + step),
                     qq = __ldg(w + q * sN + c0 + 2 * step);
        const double da = pp - cc, db = qq - pp;
        double slope = 0.5 * (da + db);
        if (LIM != 0) slope = da * db <= 0 ? 0.0 : (da > 0 ? fmin(da, db) : fmax(da, db));
        if (LIM == 3 && da * db > 0) slope = (da > 0 ? 1.0 : -1.0) * fmin(0.5 * fabs(da + db), 2.0 * fmin(fabs(da), fabs(db)));
        r[q] = cc - 0.5 * slope;
      }
      if (!(r[0] >= kRHO00 && r[4] > 0)) {
#pragma unroll
        for (int q = 0; q < NC; ++q) r[q] = __ldg(w + q * sN + c0);
      }
      double jump = 0;
#pragma unroll
      for (int d = 0; d < 3; ++d) jump += (r[5 + d] - l[5 + d]) * g.f[d];
#pragma unroll
      for (int d = 0; d < 3; ++d) l[5 + d] += jump * g.f[d];
    }
  }
  const double4 rd = L.radial[i + L.g];
  const double area = dir == 0 ? rd.x : rd.y;
  secondOrderFaceFlux<ROE>(out, l, r, g, area, L.gamma, L.invGm1, L.entropy);
  if (powell) {
    double f = 0;
#pragma unroll
    for (int d = 0; d < 3; ++d) f += 0.5 * (l[5 + d] + r[5 + d]) * g.n[d] * area;
    bf = f;
  }
}

// CFL rate of one valid cell from its conserved state,
// src/BoxOp_SecondOrderCFL.H:138-202 (no mapped scale, no cone density).
// Smallest density of the cone clouds being fed through r_inner at time t
// (minimumConeBoundaryDensity, src/MHD_CME.H:1152-1160), 0 if none.
__device__ __forceinline__ double coneBoundaryDensity(const DevLevel& L, double t) {
  double density = 0;
  for (int s = 0; s < L.ninlet; ++s)
    if (t >= L.inlet[s].insertionTime && t < L.inlet[s].endTime)
      density = density > 0 ? fmin(density, L.inlet[s].density) : L.inlet[s].density;
  return density;
}

__device__ __forceinline__ double cflRate(const DevLevel& L, int b, int i, int j, int k, const double u[8],
                                          double coneDensity = 0) {
  const CflCell& a = L.cfl[((size_t)b * L.na + k) * L.na + j];
  const double4 rd = L.radial[i + L.g];
  const double volume = rd.w, inverseVolume = 1.0 / rd.w, width0 = rd.z * L.dxi0;
  const double area[3] = {rd.x, rd.y, rd.y};
  double rho = u[0] * a.inverseDet;
  rho *= inverseVolume;
  rho = dmax(rho, kRHO00);
  double energy = u[4] * a.inverseDet;
  energy *= inverseVolume;
  double v[3], bb[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    v[d] = a.inverseDetA[3 * d] * u[1] + a.inverseDetA[3 * d + 1] * u[2] + a.inverseDetA[3 * d + 2] * u[3];
    bb[d] = a.inverseDetA[3 * d] * u[5] + a.inverseDetA[3 * d + 1] * u[6] + a.inverseDetA[3 * d + 2] * u[7];
    v[d] *= inverseVolume;
    bb[d] *= inverseVolume;
    v[d] /= rho;
  }
  double kinetic = 0, magnetic = 0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double vc = a.cell[3 * d] * v[0] + a.cell[3 * d + 1] * v[1] + a.cell[3 * d + 2] * v[2];
    const double bc = a.cell[3 * d] * bb[0] + a.cell[3 * d + 1] * bb[1] + a.cell[3 * d + 2] * bb[2];
    kinetic += vc * vc / 2;
    magnetic += bc * bc / 8.0 / kPi;
  }
  kinetic *= rho;
  double pressure = (energy - kinetic - magnetic) * (L.gamma - 1);
  if (pressure < 0) pressure = 0;
  double inverseDt = 0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double* basis = d == 0 ? a.cell : a.face[d - 1];
    double v2 = 0, fullB2 = 0;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const double velocity = basis[3 * q] * v[0] + basis[3 * q + 1] * v[1] + basis[3 * q + 2] * v[2];
      const double field = basis[3 * q] * bb[0] + basis[3 * q + 1] * bb[1] + basis[3 * q + 2] * bb[2];
      v2 += velocity * velocity;
      fullB2 += field * field;
    }
    const double width = d == 0 ? width0 : volume * a.det[d] * L.h / area[d] / a.normal[d];
    // src/BoxOp_SecondOrderCFL.H:196-200: a cone may impose a lighter total
    // density under the ambient field; bound that Alfven speed
    const double magneticDensity = coneDensity > 0 ? fmin(rho, coneDensity) : rho;
    const double wave = sqrt(L.gamma * pressure / rho + fullB2 / 4.0 / kPi / magneticDensity);
    inverseDt += (wave + sqrt(v2)) / width;
  }
  return inverseDt;
}

// Max over a warp (std::max order: a NaN candidate never replaces the max),
// then one atomic per warp on the bit pattern (non-negative doubles order as
// unsigned integers).
__device__ __forceinline__ void warpMaxAtomic(double v, unsigned long long* out) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double other = __shfl_xor_sync(0xffffffffu, v, o);
    v = v < other ? other : v;
  }
  if ((threadIdx.x & 31) == 0 && v > 0) atomicMax(out, (unsigned long long)__double_as_longlong(v));
}

template <class TL, int DIR, int LIM, bool ROE, int MODE>
__device__ __forceinline__ void o2FaceLoop(const StageArgs& a, const double* __restrict__ w, int block, int oi,
                                           int oj, int ok, int v0, int v1, int v2, double* sF, int base,
                                           bool powell) {
  constexpr int TX = TL::TX, TY = TL::TY, TZ = TL::TZ, NT = TL::NT, NF = TL::NF;
  constexpr int EX = TX + (DIR == 0), EY = TY + (DIR == 1), EZ = TZ + (DIR == 2);
  constexpr int NFD = EX * EY * EZ;
  for (int f = threadIdx.x; f < NFD; f += NT) {
    const int fi = f % EX, fj = (f / EX) % EY, fk = f / (EX * EY);
    const int i = oi + fi, j = oj + fj, k = ok + fk;
    const bool valid = i <= a.hi[0] + (DIR == 0) && j <= a.hi[1] + (DIR == 1) && k <= a.hi[2] + (DIR == 2);
    double out[8];
    double bf = 0;
    if (valid) {
      o2Face<LIM, ROE, MODE>(a, w, block, DIR, i, j, k, out, bf, powell);
      if (MODE == MODE_BOX && a.flux[DIR]) {
        const int f0 = v0 + (DIR == 0), f1 = v1 + (DIR == 1), f2 = v2 + (DIR == 2);
        const long fidx = (long)(i - a.lo[0]) + (long)f0 * ((long)(j - a.lo[1]) + (long)f1 * (k - a.lo[2]));
        const long fN = (long)f0 * f1 * f2;
#pragma unroll
        for (int q = 0; q < NC; ++q) a.flux[DIR][q * fN + fidx] = out[q];
      }
    } else {
#pragma unroll
      for (int q = 0; q < NC; ++q) out[q] = 0;
    }
#pragma unroll
    for (int q = 0; q < NC; ++q) sF[q * NF + base + f] = out[q];
    sF[8 * NF + base + f] = bf;
  }
}

template <class TL, int LIM, bool ROE, int MODE>
__global__ void __launch_bounds__(TL::NT, TL::minBlocks(ROE))
    o2StageKernel(const StageArgs a, const int powell, const int grav) {
  constexpr int TX = TL::TX, TY = TL::TY, TZ = TL::TZ, NF = TL::NF, NF0 = TL::NF0, NF1 = TL::NF1;
  extern __shared__ double sF[];  // [9][NF]: 8 flux components + Powell face B_n
  if (a.solverFlag && ((*a.solverFlag != 0) == (a.exitOnFlag != 0))) return;  // the other solver's launch
  const int v0 = a.hi[0] - a.lo[0] + 1, v1 = a.hi[1] - a.lo[1] + 1, v2 = a.hi[2] - a.lo[2] + 1;
  const int nbx = (v0 + TX - 1) / TX, nby = (v1 + TY - 1) / TY, nbz = (v2 + TZ - 1) / TZ;
  int t = blockIdx.x;
  const int bx = t % nbx; t /= nbx;
  const int by = t % nby; t /= nby;
  const int bz = t % nbz;
  const int box = t / nbz;
  const int block = a.block0 + box;
  const int oi = a.lo[0] + bx * TX, oj = a.lo[1] + by * TY, ok = a.lo[2] + bz * TZ;
  const double* __restrict__ w = a.w + (long)box * a.wBoxStride;

  o2FaceLoop<TL, 0, LIM, ROE, MODE>(a, w, block, oi, oj, ok, v0, v1, v2, sF, 0, powell != 0);
  o2FaceLoop<TL, 1, LIM, ROE, MODE>(a, w, block, oi, oj, ok, v0, v1, v2, sF, NF0, powell != 0);
  o2FaceLoop<TL, 2, LIM, ROE, MODE>(a, w, block, oi, oj, ok, v0, v1, v2, sF, NF0 + NF1, powell != 0);
  __syncthreads();

  const int li = threadIdx.x % TX, lj = (threadIdx.x / TX) % TY, lk = threadIdx.x / (TX * TY);
  const int i = oi + li, j = oj + lj, k = ok + lk;
  // Inactive threads of a partial tile stay for the warp-wide CFL reduction.
  const bool active = i <= a.hi[0] && j <= a.hi[1] && k <= a.hi[2];
  const DevLevel& L = a.L;
  double rate = 0.0;
  if (active) {
    const long cw = cellOffset(i, j, k, a.wlo, a.wn);
    double kv[8];
    long vidx = 0;
    if (MODE == MODE_BOX) {
      vidx = (long)(i - a.lo[0]) + (long)v0 * ((long)(j - a.lo[1]) + (long)v1 * (k - a.lo[2]));
#pragma unroll
      for (int q = 0; q < NC; ++q) kv[q] = a.rhs[q * a.rhsN + vidx];
    } else {
      vidx = (long)box * NC * L.Nv + (long)i + (long)L.nr * ((long)j + (long)L.na * k);
#pragma unroll
      for (int q = 0; q < NC; ++q) kv[q] = 0.0;
      if (grav) {
        // src/BoxOp_Gravity.H:36-58
        const GravCell gc = L.grav[((size_t)block * L.na + k) * L.na + j];
        const double factor = -kGrav * kMsun * L.radial[i + L.g].z * __ldg(w + cw);
        double radialVelocity = 0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          kv[1 + d] += factor * gc.a0[d];
          radialVelocity += gc.x[d] * __ldg(w + (1 + d) * a.wN + cw);
        }
        kv[4] += factor * gc.det * radialVelocity;
      }
    }
    const int fl[3] = {li + (TX + 1) * (lj + TY * lk), NF0 + li + TX * (lj + (TY + 1) * lk),
                       NF0 + NF1 + li + TX * (lj + TY * lk)};
    const int fs[3] = {1, TX, TX * TY};
    const double coef[3] = {-a.scale / L.dxi0, -a.scale / L.h, -a.scale / L.h};
    double md = 0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
#pragma unroll
      for (int q = 0; q < NC; ++q) kv[q] += coef[d] * (sF[q * NF + fl[d] + fs[d]] - sF[q * NF + fl[d]]);
      if (powell) md += coef[d] * (sF[8 * NF + fl[d] + fs[d]] - sF[8 * NF + fl[d]]);
    }
    if (powell) {
      // src/BoxOp_SecondOrder.H:351-369
      double vb = 0;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const double b = __ldg(w + (5 + d) * a.wN + cw), vel = __ldg(w + (1 + d) * a.wN + cw);
        kv[1 + d] += md * b / (4 * kPi);
        kv[5 + d] += md * vel;
        vb += vel * b;
      }
      kv[4] += md * vb / (4 * kPi);
    }
    if (MODE == MODE_BOX) {
#pragma unroll
      for (int q = 0; q < NC; ++q) a.rhs[q * a.rhsN + vidx] = kv[q];
    } else if (MODE == MODE_RHS) {
#pragma unroll
      for (int q = 0; q < NC; ++q) a.rhs[vidx + q * L.Nv] = kv[q];
    } else {
      // Classical RK4 (src/MHD_AMRRungeKutta.H:10-12): stage = U + (dt a) k,
      // U_new = U + sum_s (dt b_s) k_s accumulated in stage order.  The next
      // stage's primitives go straight to wOut (no stage state in HBM).
      const double dt = a.invDtMax ? L.cfl_number / *a.invDtMax : a.dtv;
      constexpr double b4[4] = {1.0 / 6, 1.0 / 3, 1.0 / 3, 1.0 / 6};
      constexpr double a4[3] = {0.5, 0.5, 1.0};
      const long N = L.Nv;
      double u[8];
      if (a.stage < 3) {
        const double fb = dt * b4[a.stage], fa = dt * a4[a.stage];
#pragma unroll
        for (int q = 0; q < NC; ++q) {
          const double u0 = a.ju[vidx + q * N];
          const double ac = a.stage == 0 ? u0 : a.acc[vidx + q * N];
          a.acc[vidx + q * N] = ac + fb * kv[q];
          u[q] = u0 + fa * kv[q];
        }
      } else {
        const double fb = dt * b4[3];
        bool bad = false;
#pragma unroll
        for (int q = 0; q < NC; ++q) {
          u[q] = a.acc[vidx + q * N] + fb * kv[q];
          a.ju[vidx + q * N] = u[q];
          bad = bad || !isfinite(u[q]) || (q == 0 && !(u[q] > 0));
        }
        if (bad && a.invalid) atomicOr(a.invalid, 1);
        if (a.invMaxOut) {
          // the new state's rate, at the end of the step
          const double tEnd = a.tbase + (a.tdev ? *a.tdev : 0.0) + dt;
          rate = cflRate(L, box, i, j, k, u, L.ninlet ? coneBoundaryDensity(L, tEnd) : 0.0);
        }
      }
      // src/BoxOp_SecondOrderPreStage.H:46-54: JU/J -> Cartesian primitives.
      double wv[8];
      const double invJ = 1.0 / (L.radial[i + L.g].w * L.grav[((size_t)block * L.na + k) * L.na + j].det);
      cartesianPrimitiveFromConserved(wv, u, invJ, L.gamma);
      double* wo = a.wOut + (long)box * a.wBoxStride + cw;
#pragma unroll
      for (int q = 0; q < NC; ++q) wo[q * a.wN] = wv[q];
    }
  }
  if (MODE == MODE_RK && a.stage == 3 && a.invMaxOut) warpMaxAtomic(rate, a.invMaxOut);
}

// ---------------------------------------------------------------------------
// Stage preparation (src/BoxOp_SecondOrderPreStage.H:7-218).
// ---------------------------------------------------------------------------
__global__ void primValidKernel(const DevLevel L, const double* __restrict__ ju, double* __restrict__ w) {
  const unsigned n = (unsigned)(6L * L.Nv);
  HC_LEVEL_LOOP(t, n) {
    unsigned q = t;
    const int i = (int)takeMod(q, L.nr);
    const int j = (int)takeMod(q, L.na);
    const int k = (int)takeMod(q, L.na);
    const int b = (int)q;
    const long r = (long)t - (long)b * L.Nv;
    double in[8], out[8];
    const double* src = ju + (long)b * NC * L.Nv + r;
#pragma unroll
    for (int c = 0; c < NC; ++c) in[c] = src[c * L.Nv];
    const double invJ = 1.0 / (L.radial[i + L.g].w * L.grav[((size_t)b * L.na + k) * L.na + j].det);
    cartesianPrimitiveFromConserved(out, in, invJ, L.gamma);
    double* dst = w + (long)b * NC * L.Ng + (long)(i + L.g) + (long)L.n0 * ((long)(j + L.g) + (long)L.n1 * (k + L.g));
#pragma unroll
    for (int c = 0; c < NC; ++c) dst[c * L.Ng] = out[c];
  }
}

__device__ __forceinline__ long gIdx(const DevLevel& L, int b, int i, int j, int k) {
  return (long)b * NC * L.Ng + (long)(i + L.g) + (long)L.n0 * ((long)(j + L.g) + (long)L.n1 * (k + L.g));
}

__global__ void ghostsKernel(const DevLevel L, double* __restrict__ w, const StageTime st) {
  const unsigned nSeam = (unsigned)(6L * 2 * 2 * L.g * L.na * L.nr);
  const unsigned nRad = (unsigned)(6L * L.na * L.na);
  HC_LEVEL_LOOP(t, nSeam + nRad) {
    if (t < nSeam) {
      // Panel-seam ghost: 4-point along-edge interpolation of the adjacent
      // panel's Cartesian primitives, then the floors of :70-75.
      unsigned q = t;
      const int i = (int)takeMod(q, L.nr);
      const int s = (int)takeMod(q, L.na);
      const int m = (int)takeMod(q, L.g);
      const int side = (int)(q & 1u);
      const int ax = (int)((q >> 1) & 1u);
      const int b = (int)(q >> 2);
      const SeamDonor dn = L.seam[((((long)b * 2 + ax) * 2 + side) * L.g + m) * L.na + s];
      const int n = side == 0 ? -1 - m : L.na + m;
      const int gj = ax == 0 ? n : s, gk = ax == 0 ? s : n;
      double v[8];
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        double acc = 0.;
#pragma unroll
        for (int d = 0; d < 4; ++d) acc += dn.w[d] * w[gIdx(L, dn.b, i, dn.j[d], dn.k[d]) + c * L.Ng];
        v[c] = acc;
      }
      v[0] = dmax(v[0], kRHO00);
      v[4] = dmax(v[4], 0.0);
      const long o = gIdx(L, b, i, gj, gk);
#pragma unroll
      for (int c = 0; c < NC; ++c) w[o + c * L.Ng] = v[c];
    } else {
      unsigned r = t - nSeam;
      const int j = (int)takeMod(r, L.na);
      const int k = (int)takeMod(r, L.na);
      const int b = (int)r;
      const size_t cidx = ((size_t)b * L.na + k) * L.na + j;
      const double* A = L.basis + cidx * 9;
      // Inner radial ghosts: analytic wind (src/BoxOp_PreStage.H:215-228).
      if (L.innerBCType == 1) {
        for (int i = -L.g; i < 0; ++i) {
          double u[8], out[8];
          const bool need = !L.innerBC || L.ninlet;
          const double dt = need ? (st.invDtMax ? L.cfl_number / *st.invDtMax : st.dtv) : 0.0;
          const double time = need ? st.tbase + (st.tdev ? *st.tdev : 0.0) + st.cfrac * dt : 0.0;
          const GravCell gc = L.grav[cidx];
          const double radius = L.rc[i + L.g];
          const double X[3] = {radius * gc.x[0], radius * gc.x[1], radius * gc.x[2]};
          if (L.innerBC) {
#pragma unroll
            for (int c = 0; c < NC; ++c) u[c] = L.innerBC[(cidx * L.g + (i + L.g)) * NC + c];
          } else {
            analyticWind(L, X, time, u);
          }
          if (L.ninlet) inletGhost(L, time, X, A, L.basisInv + cidx * 9, u);
          nativeToPrimitive(u, A, L.gamma, out);
          const long o = gIdx(L, b, i, j, k);
#pragma unroll
          for (int c = 0; c < NC; ++c) w[o + c * L.Ng] = out[c];
        }
      }
      // Outer radial ghosts: copy the last owned layer in the native basis,
      // scaled by (r_last/r)^2 (B tangential: ^1) (src/BoxOp_PreStage.H:105-141).
      const double* Ai = L.basisInv + cidx * 9;
      double wl[8], u[8];
      const long ol = gIdx(L, b, L.nr - 1, j, k);
#pragma unroll
      for (int c = 0; c < NC; ++c) wl[c] = w[ol + c * L.Ng];
      u[0] = wl[0];
      double kinetic = 0, magnetic = 0;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        kinetic += 0.5 * wl[0] * wl[1 + d] * wl[1 + d];
        magnetic += wl[5 + d] * wl[5 + d] / (8 * kPi);
        u[1 + d] = Ai[3 * d] * wl[0] * wl[1] + Ai[3 * d + 1] * wl[0] * wl[2] + Ai[3 * d + 2] * wl[0] * wl[3];
        u[5 + d] = Ai[3 * d] * wl[5] + Ai[3 * d + 1] * wl[6] + Ai[3 * d + 2] * wl[7];
      }
      u[4] = (wl[4] - 0.0) / (L.gamma - 1.0) + kinetic + magnetic;
      for (int m = 0; m < L.g; ++m) {
        double ug[8], out[8];
        const double s2 = L.outerScale2[m], s1 = L.outerScale1[m];
#pragma unroll
        for (int c = 0; c < 6; ++c) ug[c] = u[c] * s2;
        ug[6] = u[6] * s1;
        ug[7] = u[7] * s1;
        nativeToPrimitive(ug, A, L.gamma, out);
        const long o = gIdx(L, b, L.nr + m, j, k);
#pragma unroll
        for (int c = 0; c < NC; ++c) w[o + c * L.Ng] = out[c];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// CFL rate (src/BoxOp_SecondOrderCFL.H:117-209): max over cells of
// sum_d (fast bound + |v|)/width_d.  Warp-shuffle then one atomic per warp.
// ---------------------------------------------------------------------------
__global__ void cflKernel(const DevLevel L, const double* __restrict__ ju, unsigned long long* invMaxBits,
                          const double* __restrict__ time) {
  const unsigned n = (unsigned)(6L * L.Nv);
  const double cone = time && L.ninlet ? coneBoundaryDensity(L, *time) : 0.0;
  double best = 0.0;
  HC_LEVEL_LOOP(t, n) {
    unsigned q = t;
    const int i = (int)takeMod(q, L.nr);
    const int j = (int)takeMod(q, L.na);
    const int k = (int)takeMod(q, L.na);
    const int b = (int)q;
    const long r = (long)t - (long)b * L.Nv;
    double u[8];
    const double* src = ju + (long)b * NC * L.Nv + r;
#pragma unroll
    for (int c = 0; c < NC; ++c) u[c] = src[c * L.Nv];
    const double inverseDt = cflRate(L, b, i, j, k, u, cone);
    best = best < inverseDt ? inverseDt : best;  // std::max(localMaximum, x)
  }
  warpMaxAtomic(best, invMaxBits);
}

__global__ void setIntKernel(int* p, int v) { *p = v; }

// src/BoxOp_EulerCubedSphereImplem.H:817-876: finite components, rho > 0.
__global__ void validKernel(const DevLevel L, const double* __restrict__ ju, int* ok) {
  const unsigned n = (unsigned)(6L * NC * L.Nv), nv = (unsigned)L.Nv;
  bool bad = false;
  HC_LEVEL_LOOP(t, n) {
    const double v = ju[t];
    const int c = (int)((t / nv) % NC);
    bad = bad || !isfinite(v) || (c == 0 && !(v > 0));
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicExch(ok, 0);
}

// Seeded synthetic initial state, kind 1 (the formulas are in hc_abi.h, hc_init).
struct InitArgs {
  int kind, pb, pi, pj, pk;
  double rho0, p0, vr, b0, r_ref, amp, width;
  double cx[3];
};

__global__ void initKernel(const DevLevel L, const InitArgs in, double* __restrict__ ju) {
  const long n = 6L * L.Nv;
  const double dang = kPi / 2 * L.h;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
    const int b = (int)(t / L.Nv);
    const long r = t - (long)b * L.Nv;
    const int i = (int)(r % L.nr);
    const int j = (int)((r / L.nr) % L.na);
    const int k = (int)(r / ((long)L.nr * L.na));
    const GravCell gc = L.grav[((size_t)b * L.na + k) * L.na + j];
    const double* X = gc.x;
    const double cr0 = X[1] * in.cx[2] - X[2] * in.cx[1], cr1 = X[2] * in.cx[0] - X[0] * in.cx[2],
                 cr2 = X[0] * in.cx[1] - X[1] * in.cx[0];
    const double ang = atan2(sqrt(cr0 * cr0 + cr1 * cr1 + cr2 * cr2), X[0] * in.cx[0] + X[1] * in.cx[1] + X[2] * in.cx[2]);
    const double da = ang / dang;
    const double sgn = X[2] >= 0 ? 1.0 : -1.0;
    const double4 rd = L.radial[i + L.g];
    const double rc = L.rc[i + L.g];
    const double s = in.r_ref / rc, s2 = s * s;
    const double rho = in.rho0 * s2;
    double p = in.p0 * pow(s, 2.0 * L.gamma);
    const double di = (double)(i - in.pi);
    const double d2 = di * di + da * da;
    if (in.amp != 0) p = p * (1.0 + in.amp * exp(-d2 / (2.0 * in.width * in.width)));
    const double br = in.b0 * s2 * sgn;
    const double E = p / (L.gamma - 1.0) + 0.5 * rho * in.vr * in.vr + br * br / (8.0 * kPi);
    const double J = rd.w * gc.det;
    const double u[8] = {rho, rho * in.vr * X[0], rho * in.vr * X[1], rho * in.vr * X[2], E, br * X[0], br * X[1], br * X[2]};
    double* dst = ju + (long)b * NC * L.Nv + r;
#pragma unroll
    for (int c = 0; c < NC; ++c) dst[c * L.Nv] = J * u[c];
  }
}

__global__ void boxGravityKernel(const DevLevel L, int lo0, int lo1, int lo2, int v0, int v1, int v2, int block,
                                 const double* __restrict__ w, int wl0, int wl1, int wl2, int wn0, int wn1, long wN,
                                 double* __restrict__ rhs) {
  const long n = (long)v0 * v1 * v2;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
    const int i = lo0 + (int)(t % v0);
    const int j = lo1 + (int)((t / v0) % v1);
    const int k = lo2 + (int)(t / ((long)v0 * v1));
    const long s = (long)(i - wl0) + (long)wn0 * ((long)(j - wl1) + (long)wn1 * (k - wl2));
    const GravCell gc = L.grav[((size_t)block * L.na + k) * L.na + j];
    const double factor = -kGrav * kMsun * L.radial[i + L.g].z * w[s];
    double radialVelocity = 0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      rhs[(1 + d) * n + t] += factor * gc.a0[d];
      radialVelocity += gc.x[d] * w[(1 + d) * wN + s];
    }
    rhs[4 * n + t] += factor * gc.det * radialVelocity;
  }
}

// src/MHD_CME.H:1275-1297 (cfl) and :1267-1271, 1329-1332 (rusanovEndTime).
__global__ void cmeScheduleKernel(const CmeSchedule* S, unsigned long long* invMaxBits, const double* time,
                                  int* rusanov) {
  const double t = *time;
  double fraction = 1;
  double end = -INFINITY;
  for (int i = 0; i < S->n; ++i) {
    if (!(t >= S->t[i])) continue;  // not inserted yet
    const double early = fmin(fmax((t - S->t[i] - 600) / 1800., 0.), 1.);
    double sourceFraction = .2 + .8 * early;
    if (S->boundary[i]) {
      const double recovery = fmin(fmax((t - S->stabEnd[i]) / 1800., 0.), 1.);
      sourceFraction = .2 + (S->feeding - .2) * early + (1 - S->feeding) * recovery;
    }
    fraction = fmin(fraction, sourceFraction);
    end = fmax(end, S->stabEnd[i]);
  }
  const bool window = S->roe && t < end - 1e-9 * fmax(1.0, fabs(end));
  double rate = __longlong_as_double((long long)*invMaxBits);
  // boundaryCFLRate (src/MHD_CME.H:1165-1191) for clouds still crossing r_inner
  for (int i = 0; i < S->ninlet; ++i)
    if (t >= S->inletT[i] && t < S->inletEnd[i])
      rate += (S->inletSpeed[i] * 1e5 + sqrt(S->gamma * 2 * 1.380649e-16 * S->inletTemp[i] / kMP)) / S->width;
  rate = rate / fraction;
  if (window) rate = fmax(rate, S->cfl / (end - t));
  *invMaxBits = (unsigned long long)__double_as_longlong(rate);
  if (rusanov) *rusanov = window ? 1 : 0;
}

__global__ void advanceTimeKernel(double* time, const double* invDtMax, double cfl, double* dtOut) {
  const double dt = cfl / *invDtMax;
  if (time) *time += dt;
  if (dtOut) *dtOut = dt;
}

int gridFor(long n, int threads) {
  long g = (n + threads - 1) / threads;
  const long cap = 148L * 16;
  if (g > cap) g = cap;
  return (int)(g < 1 ? 1 : g);
}

template <class TL, int LIM, bool ROE>
cudaError_t launchStageT(const StageArgs& a, int mode, bool powell, bool grav, cudaStream_t s) {
  const int v0 = a.hi[0] - a.lo[0] + 1, v1 = a.hi[1] - a.lo[1] + 1, v2 = a.hi[2] - a.lo[2] + 1;
  const long blocks = (long)a.nbox * ((v0 + TL::TX - 1) / TL::TX) * ((v1 + TL::TY - 1) / TL::TY) *
                      ((v2 + TL::TZ - 1) / TL::TZ);
  const size_t smem = sizeof(double) * 9 * TL::NF;
  if (mode == MODE_RK) o2StageKernel<TL, LIM, ROE, MODE_RK><<<(unsigned)blocks, TL::NT, smem, s>>>(a, powell, grav);
  else o2StageKernel<TL, LIM, ROE, MODE_RHS><<<(unsigned)blocks, TL::NT, smem, s>>>(a, powell, grav);
  return cudaGetLastError();
}

template <int LIM, bool ROE>
cudaError_t launchStageTile(const StageArgs& a, int mode, bool powell, bool grav, int tile, cudaStream_t s) {
  if (mode == MODE_BOX) {
    // per-box calls keep the default tile
    const int v0 = a.hi[0] - a.lo[0] + 1, v1 = a.hi[1] - a.lo[1] + 1, v2 = a.hi[2] - a.lo[2] + 1;
    const long blocks = (long)a.nbox * ((v0 + Tile0::TX - 1) / Tile0::TX) * ((v1 + Tile0::TY - 1) / Tile0::TY) *
                        ((v2 + Tile0::TZ - 1) / Tile0::TZ);
    o2StageKernel<Tile0, LIM, ROE, MODE_BOX>
        <<<(unsigned)blocks, Tile0::NT, sizeof(double) * 9 * Tile0::NF, s>>>(a, powell, grav);
    return cudaGetLastError();
  }
  switch (tile) {
    case 1: return launchStageT<Tile1, LIM, ROE>(a, mode, powell, grav, s);
    case 2: return launchStageT<Tile2, LIM, ROE>(a, mode, powell, grav, s);
    case 3: return launchStageT<Tile3, LIM, ROE>(a, mode, powell, grav, s);
    case 4: return launchStageT<Tile4, LIM, ROE>(a, mode, powell, grav, s);
    case 5: return launchStageT<Tile5, LIM, ROE>(a, mode, powell, grav, s);
    default: return launchStageT<Tile0, LIM, ROE>(a, mode, powell, grav, s);
  }
}

template <class TL>
void tileShape(int* out) {
  out[0] = TL::TX; out[1] = TL::TY; out[2] = TL::TZ; out[3] = TL::minBlocks(false); out[4] = TL::minBlocks(true);
}

}  // namespace

int stageTileShape(int tile, int out[5]) {
  switch (tile) {
    case 0: tileShape<Tile0>(out); return 1;
    case 1: tileShape<Tile1>(out); return 1;
    case 2: tileShape<Tile2>(out); return 1;
    case 3: tileShape<Tile3>(out); return 1;
    case 4: tileShape<Tile4>(out); return 1;
    case 5: tileShape<Tile5>(out); return 1;
    default: return 0;
  }
}

cudaError_t launchStage(const StageArgs& a, int mode, int limiter, bool roe, bool powell, bool grav, cudaStream_t s,
                        int tile) {
  const int lim = limiter == 0 ? 0 : limiter == 3 ? 3 : 1;
  if (lim == 0)
    return roe ? launchStageTile<0, true>(a, mode, powell, grav, tile, s)
               : launchStageTile<0, false>(a, mode, powell, grav, tile, s);
  if (lim == 1)
    return roe ? launchStageTile<1, true>(a, mode, powell, grav, tile, s)
               : launchStageTile<1, false>(a, mode, powell, grav, tile, s);
  return roe ? launchStageTile<3, true>(a, mode, powell, grav, tile, s)
             : launchStageTile<3, false>(a, mode, powell, grav, tile, s);
}

cudaError_t launchPrimValid(const DevLevel& L, const double* ju, double* w, cudaStream_t s) {
  primValidKernel<<<gridFor(6L * L.Nv, 256), 256, 0, s>>>(L, ju, w);
  return cudaGetLastError();
}

cudaError_t launchGhosts(const DevLevel& L, double* w, const StageTime& t, cudaStream_t s) {
  const long n = 6L * 2 * 2 * L.g * L.na * L.nr + 6L * L.na * L.na;
  ghostsKernel<<<gridFor(n, 128), 128, 0, s>>>(L, w, t);
  return cudaGetLastError();
}

cudaError_t launchCfl(const DevLevel& L, const double* ju, unsigned long long* invMaxBits, cudaStream_t s,
                      const double* time) {
  cudaError_t e = cudaMemsetAsync(invMaxBits, 0, sizeof(unsigned long long), s);
  if (e != cudaSuccess) return e;
  cflKernel<<<gridFor(6L * L.Nv, 256), 256, 0, s>>>(L, ju, invMaxBits, time);
  return cudaGetLastError();
}

cudaError_t launchValid(const DevLevel& L, const double* ju, int* ok, cudaStream_t s) {
  setIntKernel<<<1, 1, 0, s>>>(ok, 1);
  validKernel<<<gridFor(6L * NC * L.Nv, 256), 256, 0, s>>>(L, ju, ok);
  return cudaGetLastError();
}

cudaError_t launchInit(const DevLevel& L, const void* init, double* ju, cudaStream_t s) {
  initKernel<<<gridFor(6L * L.Nv, 256), 256, 0, s>>>(L, *static_cast<const InitArgs*>(init), ju);
  return cudaGetLastError();
}

cudaError_t launchBoxGravity(const DevLevel& L, const int lo[3], const int hi[3], int block, const double* w,
                             const int wlo[3], const int wn[3], double* rhs, cudaStream_t s) {
  const int v0 = hi[0] - lo[0] + 1, v1 = hi[1] - lo[1] + 1, v2 = hi[2] - lo[2] + 1;
  const long wN = (long)wn[0] * wn[1] * wn[2];
  boxGravityKernel<<<gridFor((long)v0 * v1 * v2, 256), 256, 0, s>>>(L, lo[0], lo[1], lo[2], v0, v1, v2, block, w, wlo[0],
                                                                     wlo[1], wlo[2], wn[0], wn[1], wN, rhs);
  return cudaGetLastError();
}

cudaError_t launchCmeSchedule(const CmeSchedule* sched, unsigned long long* invMaxBits, const double* time,
                              int* rusanov, cudaStream_t s) {
  cmeScheduleKernel<<<1, 1, 0, s>>>(sched, invMaxBits, time, rusanov);
  return cudaGetLastError();
}

cudaError_t launchAdvanceTime(double* time, const double* invDtMax, double cfl, double* dtOut, cudaStream_t s) {
  advanceTimeKernel<<<1, 1, 0, s>>>(time, invDtMax, cfl, dtOut);
  return cudaGetLastError();
}

cudaError_t launchBitsToDouble(const unsigned long long* bits, double* out, cudaStream_t s) {
  return cudaMemcpyAsync(out, bits, sizeof(double), cudaMemcpyDeviceToDevice, s);
}

}  // namespace hc

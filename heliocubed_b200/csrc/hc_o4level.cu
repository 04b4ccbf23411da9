// Fourth-order level step on one box per panel: stage preparation, RK4
// update and panel-seam flux reconciliation.  FP64.
//
// Stage preparation follows the Cartesian state conversion of
// src/MHD_StateConversion.H:153-316 (state_conversion = 1):
//   1. o4CartesianKernel: JU -> fourth-order Cartesian averages U inside each
//      panel (quotient by <det A> with the (1/12) D(JU/det) D(det) angular
//      correction, then by dVolr with the radial one);
//   2. o4SeamPointKernel, o4SeamKernel: U on kO4Cart angular ghost layers
//      (panel corners included) from the panels that contain the ghost cells
//      (own fourth-order average interpolation; the tables come from the
//      host): point values at the ghost centres and their neighbours, then
//      each ghost average from five of them;
//   3. o4NativeKernel: U -> native averages USph with the fourth-order matrix
//      quotient of src/MHD_CachedCartesianConversion.H:65-210 on the ghosted
//      box, and the radial ghosts of src/BoxOp_PreStage.H:57-228 (inner:
//      analytic wind; outer: last layer scaled by (r_last / r)^2, B_t by r).
// The operator then runs batched over the six panels (hc_o4.cu) and adds
// its seam face fluxes, times b_s dt, into a register; after the fourth
// stage every seam face takes the mean of both sides' time-integrated
// fluxes (src/MHD_AMR.H:1478-1497; src/MHD_LevelRK.H:45-56).
#include <cuda_runtime.h>

#include "hc_device.cuh"
#include "hc_level.h"

namespace hc {
namespace {

constexpr int kThreads = 128;

int blocksFor(long n) {
  long g = (n + kThreads - 1) / kThreads;
  if (g > 148L * 64) g = 148L * 64;
  return (int)(g < 1 ? 1 : g);
}

__device__ __forceinline__ long vIdx(const O4Level& O, int b, int c, int i, int j, int k) {
  return ((long)b * 8 + c) * O.Nv + i + (long)O.nr * (j + (long)O.na * k);
}
__device__ __forceinline__ long cIdx(const O4Level& O, int b, int c, int i, int j, int k) {
  return ((long)b * 8 + c) * O.Nc + i + (long)O.nr * ((j + O.ga) + (long)O.nA * (k + O.ga));
}
__device__ __forceinline__ long gIdx4(const O4Level& O, int b, int c, int i, int j, int k) {
  return ((long)b * 8 + c) * O.Ng + (i + O.g) + (long)(O.nr + 2 * O.g) * ((j + O.g) + (long)O.nG * (k + O.g));
}
__device__ __forceinline__ double detAt(const O4Level& O, int b, int j, int k) {
  return O.detx[((long)b * (O.na + 2) + (k + 1)) * (O.na + 2) + (j + 1)];
}
__device__ __forceinline__ double volAt(const O4Level& O, int i) { return O.radial[i + O.g + 1].x; }

// 1. JU -> Cartesian averages, src/MHD_StateConversion.H:198-262.
// Capped at 102 registers (5 CTAs of 128 threads per SM): the unrolled
// component loop would otherwise take 128 and hold occupancy at 4 CTAs.
__global__ void __launch_bounds__(128, 5) o4CartesianKernel(const O4StageIO io) {
  const O4Level& O = io.O;
  const unsigned n = (unsigned)(6L * O.Nv);
  HC_LEVEL_LOOP(t, n) {
    unsigned r = t;
    const int i = (int)takeMod(r, O.nr);
    const int j = (int)takeMod(r, O.na);
    const int k = (int)takeMod(r, O.na);
    const int b = (int)r;
    const int na = O.na;
    // Quotients use reciprocals of <det A> and dVolr (one rounding from the
    // reference's divisions).
    const double invDet = 1.0 / detAt(O, b, j, k);
    const double dd1 = 0.5 * (detAt(O, b, j + 1, k) - detAt(O, b, j - 1, k));
    const double dd2 = 0.5 * (detAt(O, b, j, k + 1) - detAt(O, b, j, k - 1));
    // CubedSphereShell::deriv3case at (j, k): undivided centred difference
    // inside the panel, second-order one-sided on its first and last cells;
    // the three-cell windows it reads and their weights
    const int ja = j == 0 ? 0 : (j == na - 1 ? na - 3 : j - 1);
    const int ka = k == 0 ? 0 : (k == na - 1 ? na - 3 : k - 1);
    double wj[3], wk[3], wr[3];
    auto weights = [](int x, int n, double w[3]) {
      if (x == 0) { w[0] = -1.5; w[1] = 2.0; w[2] = -0.5; }
      else if (x == n - 1) { w[0] = 0.5; w[1] = -2.0; w[2] = 1.5; }
      else { w[0] = -0.5; w[1] = 0.0; w[2] = 0.5; }
    };
    weights(j, na, wj);
    weights(k, na, wk);
    weights(i, O.nr, wr);
    double invJ[3], invK[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      invJ[q] = 1.0 / detAt(O, b, ja + q, k);
      invK[q] = 1.0 / detAt(O, b, j, ka + q);
    }
    // the radial window of deriv3case at i
    const int ia = i == 0 ? 0 : (i == O.nr - 1 ? O.nr - 3 : i - 1);
    double invV[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) invV[q] = 1.0 / volAt(O, ia + q);
    const double dv = 0.5 * (volAt(O, i + 1) - volAt(O, i - 1));
    const int slot = i - ia;
    // JU addressed from the box's base with fixed strides (component, j, k)
    const long sv = O.Nv, sj = O.nr, sk = (long)O.nr * O.na;
    const double* U0 = io.ju + (long)b * 8 * sv;
    // all loads before the first store (the compiler cannot tell ju and
    // cart apart, so interleaved stores would serialise the components)
    double res[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const double* Uc = U0 + c * sv;
      double dq = 0.0, angI = 0.0;
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        const int ii = ia + q;
        double d1 = 0.0, d2 = 0.0;
#pragma unroll
        for (int m = 0; m < 3; ++m) {
          d1 += wj[m] * (Uc[ii + (ja + m) * sj + k * sk] * invJ[m]);
          d2 += wk[m] * (Uc[ii + j * sj + (ka + m) * sk] * invK[m]);
        }
        const double ang = (Uc[ii + j * sj + k * sk] - (d1 * dd1 + d2 * dd2) * (1.0 / 12.0)) * invDet;
        dq += wr[q] * (ang * invV[q]);
        if (q == slot) angI = ang;
      }
      res[c] = (angI - dq * dv * (1.0 / 12.0)) * invV[slot];
    }
#pragma unroll
    for (int c = 0; c < 8; ++c) io.cart[cIdx(O, b, c, i, j, k)] = res[c];
  }
}

// 2a. Point values of the Cartesian averages at the interpolation points
// (ghost centres and their neighbours): the tensor-product cubic matching
// the 4 x 4 donor cell averages, evaluated at the point.
// One thread per (radial cell, component, point): the 16 donor loads of a
// component are independent of the other components', so splitting them
// over threads puts more of them in flight than a thread's registers hold.
__global__ void o4SeamPointKernel(const O4StageIO io) {
  const O4Level& O = io.O;
  const unsigned n = (unsigned)(6L * 8 * O.npts * O.nr);
  HC_LEVEL_LOOP(t, n) {
    unsigned q = t;
    const int i = (int)takeMod(q, O.nr);
    const int c = (int)takeMod(q, 8);
    const int pt = (int)takeMod(q, O.npts);
    const int b = (int)q;
    const O4Point& P = O.pts[(long)b * O.npts + pt];
    // donors addressed from one base with fixed strides (j, k)
    const long sj = O.nr, sk = (long)O.nr * O.nA;
    const double* base = io.cart + cIdx(O, P.p, c, i, P.j0, P.k0);
    double v = 0.0;
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
      double row = 0.0;
#pragma unroll
      for (int m = 0; m < 4; ++m) row += P.wj[m] * base[kk * sk + m * sj];
      v += P.wk[kk] * row;
    }
    io.pv[(((long)b * 8 + c) * O.npts + pt) * O.nr + i] = v;
  }
}

// 2b. Seam ghost averages: (5/6) U(centre) + (1/24) sum of U at the four
// neighbouring centres, a fourth-order cell average in the ghost panel's
// coordinates.  An inadmissible average (non-finite, density below RHO00 or
// negative thermal energy: a jump, where the linear stencil overshoots)
// takes the average of the donor cell containing the ghost centre, the
// fallback of the reference's AMR ghost interpolation (src/MHD_AMR.H:
// 1382-1391).
__global__ void o4SeamKernel(const O4StageIO io) {
  const O4Level& O = io.O;
  const unsigned n = (unsigned)(6L * O.nring * O.nr);
  HC_LEVEL_LOOP(t, n) {
    unsigned q = t;
    const int i = (int)takeMod(q, O.nr);
    const int pos = (int)takeMod(q, O.nring);
    const int b = (int)q;
    const int2 jk = O.ringJK[pos];
    const int* pt = O.ringPt + (long)pos * 5;
    const double* pv = io.pv + (long)b * 8 * O.npts * O.nr + i;
    const long cs = (long)O.npts * O.nr;
    double u[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const double* v = pv + c * cs;
      const double nb = (v[(long)pt[1] * O.nr] + v[(long)pt[2] * O.nr]) + (v[(long)pt[3] * O.nr] + v[(long)pt[4] * O.nr]);
      u[c] = (5.0 / 6.0) * v[(long)pt[0] * O.nr] + (1.0 / 24.0) * nb;
    }
    bool valid = true;
#pragma unroll
    for (int c = 0; c < 8; ++c) valid &= isfinite(u[c]);
    double thermal = u[4];
    if (u[0] > 0) {
#pragma unroll
      for (int d = 0; d < 3; ++d) thermal -= 0.5 * u[1 + d] * u[1 + d] / u[0] + u[5 + d] * u[5 + d] / (8 * kPi);
    }
    if (!(valid && u[0] >= kRHO00 && thermal >= 0 && isfinite(thermal))) {
      const O4Point P = O.pts[(long)b * O.npts + pt[0]];
      const long src = cIdx(O, P.p, 0, i, P.j0 + (P.cell & 3), P.k0 + (P.cell >> 2));
#pragma unroll
      for (int c = 0; c < 8; ++c) u[c] = io.cart[src + (long)c * O.Nc];
    }
#pragma unroll
    for (int c = 0; c < 8; ++c) io.cart[cIdx(O, b, c, i, jk.x, jk.y)] = u[c];
  }
}

// Native conversion of one cell (src/MHD_CachedCartesianConversion.H:65-124).
// Every operand is addressed from one base pointer per array with fixed
// strides (cell j +- 1, k +- 1, component), so the cell's ~150 loads share
// one index computation.
__device__ void nativeCell(const O4Level& O, const double* __restrict__ cart, int b, int i, int j, int k, double out[8]) {
  const long sj = O.nr, sk = (long)O.nr * O.nA, sc = O.Nc;
  const long cj = 27, ck = 27L * O.nA;
  const double* c0 = cart + cIdx(O, b, 0, i, j, k);
  const double* cf = O.coef + (((long)b * O.nA + (k + O.ga)) * O.nA + (j + O.ga)) * 27;
  out[0] = c0[0];
  out[4] = c0[4 * sc];
  // neighbours (j + 1), (j - 1), (k + 1), (k - 1)
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

// 3. Native averages on the ghosted box and the radial ghosts.
__global__ void o4NativeKernel(const O4StageIO io) {
  const O4Level& O = io.O;
  const int n0 = O.nr + 2 * O.g;
  const unsigned n = (unsigned)(6L * n0 * O.nG * O.nG);
  HC_LEVEL_LOOP(t, n) {
    unsigned q = t;
    const int i = (int)takeMod(q, n0) - O.g;
    const int j = (int)takeMod(q, O.nG) - O.g;
    const int k = (int)takeMod(q, O.nG) - O.g;
    const int b = (int)q;
    double u[8];
    if (i < 0) {
      const long cell = ((long)b * O.nG + (k + O.g)) * O.nG + (j + O.g);
      if (O.inner) {
        const double* w = O.inner + (cell * O.g + (i + O.g)) * 8;
#pragma unroll
        for (int c = 0; c < 8; ++c) u[c] = w[c];
      } else {
        const StageTime& st = io.t;
        const double dt = st.invDtMax ? O.cfl / *st.invDtMax : st.dtv;
        const double time = st.tbase + (st.tdev ? *st.tdev : 0.0) + st.cfrac * dt;
        const double* xh = O.xhat + cell * 3;
        const double radius = O.radial[i + O.g + 1].y;
        const double X[3] = {radius * xh[0], radius * xh[1], radius * xh[2]};
        windConserved(O.gamma, O.r0, O.strength, X, time, u);
      }
    } else if (i < O.nr) {
      nativeCell(O, io.cart, b, i, j, k, u);
    } else {
      nativeCell(O, io.cart, b, O.nr - 1, j, k, u);
      const double rl = O.radial[O.nr - 1 + O.g + 1].y, rr = O.radial[i + O.g + 1].y;
      const double s2 = pow(rl / rr, 2.0), s1 = pow(rl / rr, 1.0);
#pragma unroll
      for (int c = 0; c < 8; ++c) u[c] *= c < 6 ? s2 : s1;
    }
    double* o = io.us + gIdx4(O, b, 0, i, j, k);
#pragma unroll
    for (int c = 0; c < 8; ++c) o[(long)c * O.Ng] = u[c];
  }
}

// RK4 update after stage s (the tableau of src/MHD_AMRRungeKutta.H:10-12).
__global__ void o4UpdateKernel(const O4Level O, int stage, const double* __restrict__ k, double* __restrict__ ju,
                               double* __restrict__ acc, double* __restrict__ next, const double* invDtMax, double cfl,
                               double dtv) {
  const double b4[4] = {1.0 / 6, 1.0 / 3, 1.0 / 3, 1.0 / 6};
  const double a4[4] = {0.5, 0.5, 1.0, 0.0};
  const double dt = invDtMax ? cfl / *invDtMax : dtv;
  const double fb = dt * b4[stage], fa = dt * a4[stage];
  const long n = 6L * 8 * O.Nv;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
    const double kv = k[t];
    if (stage == 0) {
      const double u = ju[t];
      acc[t] = u + fb * kv;
      next[t] = u + fa * kv;
    } else if (stage < 3) {
      acc[t] += fb * kv;
      next[t] = ju[t] + fa * kv;
    } else {
      ju[t] = acc[t] + fb * kv;
    }
  }
}

// Seam reconciliation of one edge axis (cells of different faces of one
// axis never coincide, so each launch is race free).
__global__ void o4RefluxKernel(const O4Level O, const DevLevel L, int ax, const double* __restrict__ reg,
                               double* __restrict__ ju) {
  const long nrna = (long)O.na * O.nr;
  const unsigned n = (unsigned)(6L * 2 * nrna);
  HC_LEVEL_LOOP(t, n) {
    unsigned q = t;
    const int i = (int)takeMod(q, O.nr);
    const int s = (int)takeMod(q, O.na);
    const int side = (int)(q & 1u);
    const int b = (int)(q >> 1);
    const int e = (ax - 1) * 2 + side;
    const EdgeLink nb = L.edge[b * 4 + e];
    const int sn = L.faceMap[((long)b * 4 + e) * O.na + s];
    const double sigma = nb.side != side ? 1.0 : -1.0;
    const double dir = side ? -(double)O.na : (double)O.na;
    const int edge = side ? O.na - 1 : 0;
    const int j = ax == 1 ? edge : s, k = ax == 1 ? s : edge;
    const double* fa = reg + (((long)b * 2 + (ax - 1)) * 2 + side) * 8 * nrna + (long)s * O.nr + i;
    const double* fb = reg + (((long)nb.nb * 2 + (nb.axis - 1)) * 2 + nb.side) * 8 * nrna + (long)sn * O.nr + i;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const double a = fa[c * nrna];
      const double mean = 0.5 * (a + sigma * fb[c * nrna]);
      ju[vIdx(O, b, c, i, j, k)] += dir * (mean - a);
    }
  }
}

}  // namespace

// Every flat index range of the level kernels fits in 31 bits.
bool levelIndexable(const O4Level& O) {
  const long lim = 0x7fffffffL;
  return 6L * (O.nr + 2 * O.g) * O.nG * O.nG < lim && 6L * O.Nv < lim && 48L * O.npts * O.nr < lim &&
         6L * O.nring * O.nr < lim && 12L * O.na * O.nr < lim;
}

cudaError_t launchO4Prepare(const O4StageIO& io, cudaStream_t s) {
  const O4Level& O = io.O;
  if (!levelIndexable(O)) return cudaErrorInvalidValue;
  o4CartesianKernel<<<blocksFor(6L * O.Nv), kThreads, 0, s>>>(io);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  o4SeamPointKernel<<<blocksFor(6L * 8 * O.npts * O.nr), kThreads, 0, s>>>(io);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  o4SeamKernel<<<blocksFor(6L * O.nring * O.nr), kThreads, 0, s>>>(io);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  o4NativeKernel<<<blocksFor(6L * (O.nr + 2 * O.g) * O.nG * O.nG), kThreads, 0, s>>>(io);
  return cudaGetLastError();
}

cudaError_t launchO4Update(const O4Level& O, int stage, const double* k, double* ju, double* acc, double* next,
                           const double* invDtMax, double cfl, double dtv, cudaStream_t s) {
  o4UpdateKernel<<<blocksFor(6L * 8 * O.Nv), kThreads, 0, s>>>(O, stage, k, ju, acc, next, invDtMax, cfl, dtv);
  return cudaGetLastError();
}

cudaError_t launchO4Reflux(const O4Level& O, const DevLevel& L, const double* reg, double* ju, cudaStream_t s) {
  if (!levelIndexable(O)) return cudaErrorInvalidValue;
  for (int ax = 1; ax <= 2; ++ax) {
    o4RefluxKernel<<<blocksFor(6L * 2 * O.na * O.nr), kThreads, 0, s>>>(O, L, ax, reg, ju);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace hc

// AMR Runge-Kutta stage logic on uneven boxes: the tableau combination of
// advanceRungeKuttaSynchronous (src/MHD_AMRRungeKutta.H:5-41) and the
// fine-to-coarse restriction restrictTo / Stencil::AvgDown
// (src/MHD_AMR.H:597-609), each one launch over a device work list: fixed
// chunks of 16384 elements of the boxes (or restrictions), one CTA each, so
// uneven boxes load the GPU evenly.
// The operator itself runs through hc_o4_batch_rhs on the same boxes.
//
// Every increment is rounded as the reference's BoxData::increment rounds
// it, (scale * source) then the add, with explicit round-to-nearest
// operations, so the results do not depend on multiply-add contraction.
#include <cuda_runtime.h>
#include <math_constants.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <functional>
#include <utility>
#include <vector>

#include "../../include/hc_abi.h"
#include "hc_device.cuh"
#include "hc_level.h"

namespace {

constexpr int kThreads = 256;

// Kutta RK3 and classical RK4 tableaus (src/MHD_AMRRungeKutta.H:9-12).
constexpr double kA3[4][4] = {{0, 0, 0, 0}, {0.5, 0, 0, 0}, {-1, 2, 0, 0}, {0, 0, 0, 0}};
constexpr double kA4[4][4] = {{0, 0, 0, 0}, {0.5, 0, 0, 0}, {0, 0.5, 0, 0}, {0, 0, 1, 0}};
constexpr double kB3[4] = {1.0 / 6, 2.0 / 3, 1.0 / 6, 0};
constexpr double kB4[4] = {1.0 / 6, 1.0 / 3, 1.0 / 3, 1.0 / 6};

// Factors of one launch: stage state = state + sum_p f[p] rk[p] over the
// used p (stage < order), or state += f[p] rk[p] for p < order (final).
struct RkFactors {
  double f[4];
  int use[4];
  int final;
};

// One work-list entry: elements [begin, end) of item `item` (a box's 8 x
// ncells doubles, or a restriction's 8 x coarse cells).
struct Chunk {
  int item, pad;
  long long begin, end;
};
constexpr long long kChunk = 16384;  // elements per CTA: 64 per thread

__global__ void __launch_bounds__(kThreads) rkCombineKernel(const hc_rk_box* __restrict__ boxes,
                                                            const Chunk* __restrict__ chunks, const RkFactors F) {
  const Chunk ch = chunks[blockIdx.x];
  const hc_rk_box B = boxes[ch.item];
  for (long long t = ch.begin + threadIdx.x; t < ch.end; t += blockDim.x) {
    double v = B.state[t];
#pragma unroll
    for (int p = 0; p < 4; ++p)
      if (F.use[p]) v = __dadd_rn(v, __dmul_rn(F.f[p], B.rk[p][t]));
    if (F.final)
      B.state[t] = v;
    else
      B.stage[t] = v;
  }
}

__global__ void __launch_bounds__(kThreads) restrictKernel(const hc_restrict_box* __restrict__ items,
                                                            const Chunk* __restrict__ chunks) {
  const Chunk ch = chunks[blockIdx.x];
  const hc_restrict_box R = items[ch.item];
  const int n0 = R.hi[0] - R.lo[0] + 1, n1 = R.hi[1] - R.lo[1] + 1, n2 = R.hi[2] - R.lo[2] + 1;
  const long long cells = (long long)n0 * n1 * n2;
  const long long fineN = (long long)R.fine_n[0] * R.fine_n[1] * R.fine_n[2];
  const long long coarseN = (long long)R.coarse_n[0] * R.coarse_n[1] * R.coarse_n[2];
  const double w = 1.0 / (double)(R.ratio[0] * R.ratio[1] * R.ratio[2]);
  for (long long t = ch.begin + threadIdx.x; t < ch.end; t += blockDim.x) {
    const int c = (int)(t / cells);
    const long long r = t - (long long)c * cells;
    const int I = R.lo[0] + (int)(r % n0);
    const int J = R.lo[1] + (int)((r / n0) % n1);
    const int K = R.lo[2] + (int)(r / ((long long)n0 * n1));
    const double* src = R.fine + (long long)c * fineN;
    double sum = 0.0;
    for (int kk = 0; kk < R.ratio[2]; ++kk)
      for (int jj = 0; jj < R.ratio[1]; ++jj)
        for (int ii = 0; ii < R.ratio[0]; ++ii) {
          const int fi = I * R.ratio[0] + ii - R.fine_lo[0];
          const int fj = J * R.ratio[1] + jj - R.fine_lo[1];
          const int fk = K * R.ratio[2] + kk - R.fine_lo[2];
          sum = __dadd_rn(sum, __dmul_rn(w, src[fi + (long long)R.fine_n[0] * (fj + (long long)R.fine_n[1] * fk)]));
        }
    const long long co = (long long)(I - R.coarse_lo[0]) +
                         (long long)R.coarse_n[0] * ((J - R.coarse_lo[1]) + (long long)R.coarse_n[1] * (K - R.coarse_lo[2]));
    R.coarse[(long long)c * coarseN + co] = sum;
  }
}

// Reflux of coarse faces covered by the fine level: coarse rhs += coef *
// (mean of the fine faces - coarse face flux), coef = -scale when the fine
// cells lie above the face (the corrected coarse cell is the one below),
// +scale otherwise.
__global__ void __launch_bounds__(kThreads) refluxKernel(const hc_reflux_box* __restrict__ items,
                                                         const Chunk* __restrict__ chunks) {
  const Chunk ch = chunks[blockIdx.x];
  const hc_reflux_box R = items[ch.item];
  const int d = R.dir;
  const int t1 = d == 0 ? 1 : 0, t2 = d == 2 ? 1 : 2;
  const int n0 = R.hi[0] - R.lo[0] + 1, n1 = R.hi[1] - R.lo[1] + 1, n2 = R.hi[2] - R.lo[2] + 1;
  const long long faces = (long long)n0 * n1 * n2;
  const long long fineN = (long long)R.fine_n[0] * R.fine_n[1] * R.fine_n[2];
  const long long coarseN = (long long)R.coarse_n[0] * R.coarse_n[1] * R.coarse_n[2];
  const long long rhsN = (long long)R.rhs_n[0] * R.rhs_n[1] * R.rhs_n[2];
  const double w = 1.0 / (double)(R.ratio[t1] * R.ratio[t2]);
  const double coef = R.fine_side ? -R.scale : R.scale;
  for (long long t = ch.begin + threadIdx.x; t < ch.end; t += blockDim.x) {
    const int c = (int)(t / faces);
    const long long r = t - (long long)c * faces;
    int f[3] = {R.lo[0] + (int)(r % n0), R.lo[1] + (int)((r / n0) % n1), R.lo[2] + (int)(r / ((long long)n0 * n1))};
    double mean = 0.0;
    for (int b2 = 0; b2 < R.ratio[t2]; ++b2)
      for (int b1 = 0; b1 < R.ratio[t1]; ++b1) {
        int g[3];
        g[d] = f[d] * R.ratio[d];
        g[t1] = f[t1] * R.ratio[t1] + b1;
        g[t2] = f[t2] * R.ratio[t2] + b2;
        const long long o = (long long)(g[0] - R.fine_lo[0]) +
                            (long long)R.fine_n[0] * ((g[1] - R.fine_lo[1]) + (long long)R.fine_n[1] * (g[2] - R.fine_lo[2]));
        mean = __dadd_rn(mean, __dmul_rn(w, R.fine_flux[(long long)c * fineN + o]));
      }
    const long long co = (long long)(f[0] - R.coarse_lo[0]) +
                         (long long)R.coarse_n[0] * ((f[1] - R.coarse_lo[1]) + (long long)R.coarse_n[1] * (f[2] - R.coarse_lo[2]));
    const double diff = __dsub_rn(mean, R.coarse_flux[(long long)c * coarseN + co]);
    int cell[3] = {f[0], f[1], f[2]};
    if (R.fine_side) cell[d] -= 1;
    const long long ro = (long long)(cell[0] - R.rhs_lo[0]) +
                         (long long)R.rhs_n[0] * ((cell[1] - R.rhs_lo[1]) + (long long)R.rhs_n[1] * (cell[2] - R.rhs_lo[2]));
    double* out = R.rhs + (long long)c * rhsN + ro;
    *out = __dadd_rn(*out, __dmul_rn(coef, diff));
  }
}

// Coarse-fine ghost interpolation (src/MHD_AMRInterpolation.H:39-155,
// applied by src/MHD_AMRFourthOrder.H:27-39).  One thread per fine storage
// cell; the quartic average of the 5 x 5 x 5 coarse cells around the parent
// is summed pass by pass as the reference's separable sweeps do (first
// index, then second, then third; each in increasing index, zero weights
// skipped), every product and sum rounded as written.
constexpr int kCfMaxRatio = 8, kCfMaxComp = 16;
struct CfItem {
  hc_cf_box box;
  double w[3][kCfMaxRatio][5];  // direction, child, coarse offset -2..2
  long long scratch;            // offset of the box's separable-pass results in the plan's scratch
};
// Shared memory of the separable passes: a plane of first-pass sums and a
// ring of five planes of second-pass sums (doubles), at most this many.
constexpr long long kCfPassMaxDoubles = 192 * 1024 / 8;
constexpr int kCfPassMaxFine = 256;  // fine extent per direction of a separable box

__device__ __forceinline__ int floorDiv(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }

// Flat index t (below 2^31: every box of a plan is checked to be) of a box
// of extents n0 x n1 x .. -> its three offsets, in 32-bit arithmetic.
__device__ __forceinline__ void split3(long long t, int n0, int n1, int& x, int& y, int& z) {
  const unsigned u = (unsigned)t, a = u / (unsigned)n0, b = a / (unsigned)n1;
  x = (int)(u - a * (unsigned)n0);
  y = (int)(a - b * (unsigned)n1);
  z = (int)b;
}

__global__ void __launch_bounds__(kThreads) cfInterpKernel(const CfItem* __restrict__ items,
                                                           const Chunk* __restrict__ chunks) {
  const Chunk ch = chunks[blockIdx.x];
  const CfItem& it = items[ch.item];
  const hc_cf_box& B = it.box;
  const long long fineN = (long long)B.fine_n[0] * B.fine_n[1] * B.fine_n[2];
  const long long coarseN = (long long)B.coarse_n[0] * B.coarse_n[1] * B.coarse_n[2];
  for (long long t = ch.begin + threadIdx.x; t < ch.end; t += blockDim.x) {
    int p[3];
    split3(t, B.fine_n[0], B.fine_n[1], p[0], p[1], p[2]);
    for (int d = 0; d < 3; ++d) p[d] += B.fine_lo[d];
    bool inside = true;
    for (int d = 0; d < 3; ++d) inside = inside && p[d] >= B.valid_lo[d] && p[d] <= B.valid_hi[d];
    if (inside) continue;  // valid cells keep their own data
    int q[3];
    const double* w[3];
    for (int d = 0; d < 3; ++d) {
      q[d] = floorDiv(p[d], B.ratio[d]);
      w[d] = it.w[d][p[d] - q[d] * B.ratio[d]];
    }
    double out[kCfMaxComp];
    bool finite = true;
    for (int c = 0; c < B.ncomp; ++c) {
      const double* src = B.coarse + (long long)c * coarseN;
      double value = 0.0;
      for (int k2 = -2; k2 <= 2; ++k2) {
        if (w[2][k2 + 2] == 0.0) continue;
        double v1 = 0.0;
        for (int k1 = -2; k1 <= 2; ++k1) {
          if (w[1][k1 + 2] == 0.0) continue;
          double v0 = 0.0;
          for (int k0 = -2; k0 <= 2; ++k0) {
            if (w[0][k0 + 2] == 0.0) continue;
            const int a = q[0] + k0 - B.coarse_lo[0], b = q[1] + k1 - B.coarse_lo[1], e = q[2] + k2 - B.coarse_lo[2];
            if (a < 0 || a >= B.coarse_n[0] || b < 0 || b >= B.coarse_n[1] || e < 0 || e >= B.coarse_n[2]) {
              v0 = CUDART_NAN;  // the reference's out-of-box marker
              break;
            }
            v0 = __dadd_rn(v0, __dmul_rn(w[0][k0 + 2], src[a + (long long)B.coarse_n[0] * (b + (long long)B.coarse_n[1] * e)]));
          }
          v1 = __dadd_rn(v1, __dmul_rn(w[1][k1 + 2], v0));
        }
        value = __dadd_rn(value, __dmul_rn(w[2][k2 + 2], v1));
      }
      out[c] = value;
      finite = finite && isfinite(value);
    }
    if (!finite) continue;  // left for the caller's fill
    const long long fo = t;
    for (int c = 0; c < B.ncomp; ++c) B.fine[(long long)c * fineN + fo] = out[c];
  }
}

// The same interpolation as separable passes over whole planes (one CTA per
// box and component): for each coarse plane k of the box's footprint, the
// first-pass sums along i for every fine i and coarse j, then the
// second-pass sums along j for every fine (i, j), kept in a ring of five
// planes; each fine plane k takes its third-pass sums from the ring as soon
// as its five parents' planes are there.  Every sum is the per-cell
// kernel's, formed from the same terms in the same order (zero weights
// skipped, a first-pass point outside the coarse box making its sum NaN);
// the results go to scratch, and cfCommitKernel writes the ghost cells
// whose components are all finite.
__global__ void __launch_bounds__(kThreads) cfPassKernel(const CfItem* __restrict__ items,
                                                         const int2* __restrict__ pass, double* __restrict__ scratch) {
  extern __shared__ double sm[];
  // fine index -> parent offset and child of each direction (no division
  // in the passes' loops)
  __shared__ int sq[3][kCfPassMaxFine], sc[3][kCfPassMaxFine];
  __shared__ double sw[3][kCfMaxRatio][5];
  const int2 pc = pass[blockIdx.x];
  const CfItem& it = items[pc.x];
  const hc_cf_box B = it.box;
  const int comp = pc.y, tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
  for (int e = tid; e < 3 * kCfMaxRatio * 5; e += kThreads) (&sw[0][0][0])[e] = (&it.w[0][0][0])[e];
  constexpr int TY = kThreads / 32;
  const int fn0 = B.fine_n[0], fn1 = B.fine_n[1], fn2 = B.fine_n[2];
  int c0[3], c1[3];
  for (int d = 0; d < 3; ++d) {
    c0[d] = floorDiv(B.fine_lo[d], B.ratio[d]) - 2;
    c1[d] = floorDiv(B.fine_lo[d] + B.fine_n[d] - 1, B.ratio[d]) + 2;
  }
  for (int d = 0; d < 3; ++d)
    for (int f = tid; f < B.fine_n[d]; f += kThreads) {
      const int p = B.fine_lo[d] + f, q = floorDiv(p, B.ratio[d]);
      sq[d][f] = q;
      sc[d][f] = p - q * B.ratio[d];
    }
  const int nc1 = c1[1] - c0[1] + 1, plane = fn0 * fn1;
  double* v0 = sm;                // [nc1][fn0]
  double* ring = sm + fn0 * nc1;  // [5][fn1][fn0]
  const long long coarseN = (long long)B.coarse_n[0] * B.coarse_n[1] * B.coarse_n[2];
  const long long fineN = (long long)plane * fn2;
  const double* src = B.coarse + (long long)comp * coarseN;
  double* out = scratch + it.scratch + (long long)comp * fineN;
  __syncthreads();
  for (int ck = c0[2]; ck <= c1[2]; ++ck) {
    const int e2 = ck - B.coarse_lo[2];
    const bool kIn = e2 >= 0 && e2 < B.coarse_n[2];
    for (int r = ty; r < nc1; r += TY) {
      const int b = c0[1] + r - B.coarse_lo[1];
      const bool rowIn = kIn && b >= 0 && b < B.coarse_n[1];
      const double* row = src + (long long)B.coarse_n[0] * (b + (long long)B.coarse_n[1] * e2);
      for (int fi = tx; fi < fn0; fi += 32) {
        const double* w = sw[0][sc[0][fi]];
        const int q0 = sq[0][fi];
        double v = 0.0;
        for (int k0 = -2; k0 <= 2; ++k0) {
          if (w[k0 + 2] == 0.0) continue;
          const int a = q0 + k0 - B.coarse_lo[0];
          if (!rowIn || a < 0 || a >= B.coarse_n[0]) {
            v = CUDART_NAN;
            break;
          }
          v = __dadd_rn(v, __dmul_rn(w[k0 + 2], row[a]));
        }
        v0[r * fn0 + fi] = v;
      }
    }
    __syncthreads();
    double* slot = ring + ((ck - c0[2]) % 5) * plane;
    for (int fj = ty; fj < fn1; fj += TY) {
      const double* w = sw[1][sc[1][fj]];
      const int base = sq[1][fj] - c0[1];
      for (int fi = tx; fi < fn0; fi += 32) {
        double v = 0.0;
        for (int k1 = -2; k1 <= 2; ++k1) {
          if (w[k1 + 2] == 0.0) continue;
          v = __dadd_rn(v, __dmul_rn(w[k1 + 2], v0[(base + k1) * fn0 + fi]));
        }
        slot[fj * fn0 + fi] = v;
      }
    }
    __syncthreads();
    // fine planes whose parent is ck - 2 (their five coarse planes are in)
    const int qk = ck - 2;
    const int plo = max(qk * B.ratio[2], B.fine_lo[2]), phi = min(qk * B.ratio[2] + B.ratio[2] - 1, B.fine_lo[2] + fn2 - 1);
    for (int p2 = plo; p2 <= phi; ++p2) {
      const double* w = sw[2][p2 - qk * B.ratio[2]];
      double* o = out + (long long)plane * (p2 - B.fine_lo[2]);
      for (int e = tid; e < plane; e += kThreads) {
        double v = 0.0;
        for (int k2 = -2; k2 <= 2; ++k2) {
          if (w[k2 + 2] == 0.0) continue;
          v = __dadd_rn(v, __dmul_rn(w[k2 + 2], ring[((qk + k2 - c0[2]) % 5) * plane + e]));
        }
        o[e] = v;
      }
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kThreads) cfCommitKernel(const CfItem* __restrict__ items,
                                                           const Chunk* __restrict__ chunks,
                                                           const double* __restrict__ scratch) {
  const Chunk ch = chunks[blockIdx.x];
  const CfItem& it = items[ch.item];
  const hc_cf_box B = it.box;
  const long long fineN = (long long)B.fine_n[0] * B.fine_n[1] * B.fine_n[2];
  const double* res = scratch + it.scratch;
  for (long long t = ch.begin + threadIdx.x; t < ch.end; t += blockDim.x) {
    int p[3];
    split3(t, B.fine_n[0], B.fine_n[1], p[0], p[1], p[2]);
    for (int d = 0; d < 3; ++d) p[d] += B.fine_lo[d];
    bool inside = true;
    for (int d = 0; d < 3; ++d) inside = inside && p[d] >= B.valid_lo[d] && p[d] <= B.valid_hi[d];
    if (inside) continue;
    bool finite = true;
    for (int c = 0; c < B.ncomp; ++c) finite = finite && isfinite(res[(long long)c * fineN + t]);
    if (!finite) continue;
    for (int c = 0; c < B.ncomp; ++c) B.fine[(long long)c * fineN + t] = res[(long long)c * fineN + t];
  }
}

// The separable passes' shared memory of a box (doubles).
long long cfPassDoubles(const hc_cf_box& B) {
  auto fdiv = [](int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); };
  const long long nc1 = (fdiv(B.fine_lo[1] + B.fine_n[1] - 1, B.ratio[1]) + 2) - (fdiv(B.fine_lo[1], B.ratio[1]) - 2) + 1;
  return (long long)B.fine_n[0] * nc1 + 5LL * B.fine_n[0] * B.fine_n[1];
}

// Fourth-order <JU> of the ghost cells and <U> of the valid cells of a fine
// box (src/MHD_AMRFourthOrder.H:41-80); every operation rounded as written.
__device__ __forceinline__ long long boxOff(const int lo[3], const int n[3], int i, int j, int k) {
  return (long long)(i - lo[0]) + (long long)n[0] * ((j - lo[1]) + (long long)n[1] * (k - lo[2]));
}
__device__ __forceinline__ long long boxSize(const int n[3]) { return (long long)n[0] * n[1] * n[2]; }
__device__ __forceinline__ bool inValid(const hc_cf_fine_box& B, const int p[3]) {
  return p[0] >= B.valid_lo[0] && p[0] <= B.valid_hi[0] && p[1] >= B.valid_lo[1] && p[1] <= B.valid_hi[1] &&
         p[2] >= B.valid_lo[2] && p[2] <= B.valid_hi[2];
}

__global__ void __launch_bounds__(kThreads) cfMappedKernel(const hc_cf_fine_box* __restrict__ items,
                                                           const Chunk* __restrict__ chunks) {
  const Chunk ch = chunks[blockIdx.x];
  const hc_cf_fine_box B = items[ch.item];
  const long long mN = boxSize(B.mapped_n), dN = boxSize(B.donor_n), sN = boxSize(B.state_n);
  for (long long t = ch.begin + threadIdx.x; t < ch.end; t += blockDim.x) {
    int p[3];
    split3(t, B.mapped_n[0], B.mapped_n[1], p[0], p[1], p[2]);
    for (int d = 0; d < 3; ++d) p[d] += B.mapped_lo[d];
    if (inValid(B, p)) {
      const long long so = boxOff(B.state_lo, B.state_n, p[0], p[1], p[2]);
      for (int c = 0; c < 8; ++c) B.mapped[c * mN + t] = B.state[c * sN + so];
      continue;
    }
    const double J = B.jac[boxOff(B.jac_lo, B.jac_n, p[0], p[1], p[2])];
    double dJ[3];
    long long up[3], dn[3];
    for (int d = 0; d < 3; ++d) {
      int a[3] = {p[0], p[1], p[2]}, b[3] = {p[0], p[1], p[2]};
      a[d] += 1;
      b[d] -= 1;
      dJ[d] = __dsub_rn(B.jac[boxOff(B.jac_lo, B.jac_n, a[0], a[1], a[2])], B.jac[boxOff(B.jac_lo, B.jac_n, b[0], b[1], b[2])]);
      up[d] = boxOff(B.donor_lo, B.donor_n, a[0], a[1], a[2]);
      dn[d] = boxOff(B.donor_lo, B.donor_n, b[0], b[1], b[2]);
    }
    const long long o = boxOff(B.donor_lo, B.donor_n, p[0], p[1], p[2]);
    for (int c = 0; c < 8; ++c) {
      const double* U = B.donor + c * dN;
      double value = __dmul_rn(J, U[o]);
      for (int d = 0; d < 3; ++d)
        value = __dadd_rn(value, __ddiv_rn(__dmul_rn(dJ[d], __dsub_rn(U[up[d]], U[dn[d]])), 48.0));
      B.mapped[c * mN + t] = value;
    }
  }
}

__global__ void __launch_bounds__(kThreads) cfQuotientKernel(const hc_cf_fine_box* __restrict__ items,
                                                             const Chunk* __restrict__ chunks) {
  const Chunk ch = chunks[blockIdx.x];
  const hc_cf_fine_box B = items[ch.item];
  const long long mN = boxSize(B.mapped_n), oN = boxSize(B.out_n);
  const int vn[3] = {B.valid_hi[0] - B.valid_lo[0] + 1, B.valid_hi[1] - B.valid_lo[1] + 1, B.valid_hi[2] - B.valid_lo[2] + 1};
  for (long long t = ch.begin + threadIdx.x; t < ch.end; t += blockDim.x) {
    int p[3];
    split3(t, vn[0], vn[1], p[0], p[1], p[2]);
    for (int d = 0; d < 3; ++d) p[d] += B.valid_lo[d];
    auto jacAt = [&](const int x[3]) { return B.jac[boxOff(B.jac_lo, B.jac_n, x[0], x[1], x[2])]; };
    const double Jp = jacAt(p);
    // per direction: the derivative's three cells and weights, and dJ
    int base[3];
    double w[3][3], dj[3];
    for (int d = 0; d < 3; ++d) {
      if (p[d] == B.block_lo[d]) {
        base[d] = p[d];
        w[d][0] = -1.5; w[d][1] = 2.0; w[d][2] = -0.5;
      } else if (p[d] == B.block_hi[d]) {
        base[d] = p[d] - 2;
        w[d][0] = 0.5; w[d][1] = -2.0; w[d][2] = 1.5;
      } else {
        base[d] = p[d] - 1;
        w[d][0] = -0.5; w[d][1] = 0.0; w[d][2] = 0.5;
      }
      int a[3] = {p[0], p[1], p[2]}, b[3] = {p[0], p[1], p[2]};
      a[d] += 1;
      b[d] -= 1;
      dj[d] = __dmul_rn(0.5, __dsub_rn(jacAt(a), jacAt(b)));
    }
    const long long op = boxOff(B.out_lo, B.out_n, p[0], p[1], p[2]);
    for (int c = 0; c < 8; ++c) {
      const double* M = B.mapped + c * mN;
      auto Q = [&](const int x[3]) { return __ddiv_rn(M[boxOff(B.mapped_lo, B.mapped_n, x[0], x[1], x[2])], jacAt(x)); };
      double correction = 0.0;
      for (int d = 0; d < 3; ++d) {
        double derivative = 0.0;
        for (int m = 0; m < 3; ++m) {
          int x[3] = {p[0], p[1], p[2]};
          x[d] = base[d] + m;
          derivative = __dadd_rn(derivative, __dmul_rn(w[d][m], Q(x)));
        }
        correction = __dadd_rn(correction, __dmul_rn(dj[d], derivative));
      }
      B.out[c * oN + op] = __dsub_rn(Q(p), __ddiv_rn(correction, __dmul_rn(12.0, Jp)));
    }
  }
}

// Region copies with a signed-permutation index map (exchanges).
__global__ void __launch_bounds__(kThreads) copyKernel(const hc_copy_box* __restrict__ items,
                                                       const Chunk* __restrict__ chunks) {
  const Chunk ch = chunks[blockIdx.x];
  const hc_copy_box B = items[ch.item];
  const int n0 = B.hi[0] - B.lo[0] + 1, n1 = B.hi[1] - B.lo[1] + 1;
  const long long sN = boxSize(B.src_n), dN = boxSize(B.dst_n);
  for (long long t = ch.begin + threadIdx.x; t < ch.end; t += blockDim.x) {
    int x[3];
    split3(t, n0, n1, x[0], x[1], x[2]);
    for (int d = 0; d < 3; ++d) x[d] += B.lo[d];
    const int y[3] = {B.sign[0] * x[B.perm[0]] + B.shift[0], B.sign[1] * x[B.perm[1]] + B.shift[1],
                      B.sign[2] * x[B.perm[2]] + B.shift[2]};
    const long long so = boxOff(B.src_lo, B.src_n, x[0], x[1], x[2]);
    const long long dO = boxOff(B.dst_lo, B.dst_n, y[0], y[1], y[2]);
    for (int c = 0; c < B.ncomp; ++c) B.dst[c * dN + dO] = B.src[c * sN + so];
  }
}

int cudaFailed(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return HC_OK;
  char msg[256];
  std::snprintf(msg, sizeof msg, "%s: %s", what, cudaGetErrorString(e));
  return hc::setLastError(HC_ERR_CUDA, msg);
}

void addChunks(std::vector<Chunk>& out, int item, long long elems) {
  for (long long b = 0; b < elems; b += kChunk) out.push_back(Chunk{item, 0, b, b + kChunk < elems ? b + kChunk : elems});
}

int argFail(const char* msg) { return hc::setLastError(HC_ERR_ARG, msg); }

}  // namespace

// Faces of a reflux patch inside its boxes (false if any index leaves them).
static bool refluxInside(const hc_reflux_box& R) {
  if (!R.fine_flux || !R.coarse_flux || !R.rhs || R.dir < 0 || R.dir > 2 || (R.fine_side != 0 && R.fine_side != 1))
    return false;
  for (int d = 0; d < 3; ++d) {
    if (R.ratio[d] < 1 || R.ratio[d] > 16 || R.lo[d] > R.hi[d] || R.fine_n[d] < 1 || R.coarse_n[d] < 1 || R.rhs_n[d] < 1)
      return false;
    // coarse faces
    if (R.lo[d] < R.coarse_lo[d] || R.hi[d] >= R.coarse_lo[d] + R.coarse_n[d]) return false;
    // fine faces: ratio * I along dir; ratio * I + 0 .. ratio-1 across
    const long long flo = (long long)R.lo[d] * R.ratio[d];
    const long long fhi = (long long)R.hi[d] * R.ratio[d] + (d == R.dir ? 0 : R.ratio[d] - 1);
    if (flo < R.fine_lo[d] || fhi >= (long long)R.fine_lo[d] + R.fine_n[d]) return false;
    // corrected coarse cells
    const int shift = (d == R.dir && R.fine_side) ? 1 : 0;
    if (R.lo[d] - shift < R.rhs_lo[d] || R.hi[d] - shift >= R.rhs_lo[d] + R.rhs_n[d]) return false;
  }
  return true;
}

struct hc_amr_plan {
  hc_native_box* natives = nullptr;     // fine boxes of the native conversion (device)
  Chunk* nativeChunks = nullptr;
  std::vector<hc_native_box> nativeHost;
  std::vector<int> nativeStart;
  mutable std::vector<std::pair<int, int>> nativeRangesChecked;  // ranges checked against a level
  hc_rk_box* boxes = nullptr;           // device copy
  hc_restrict_box* restricts = nullptr; // device copy
  hc_reflux_box* reflux = nullptr;      // device copy
  Chunk* refluxChunks = nullptr;        // work list of the reflux patches (device), by patch
  std::vector<hc_reflux_box> refluxHost;
  std::vector<int> refluxChunkStart;
  Chunk* boxChunks = nullptr;           // work list of the combine (device)
  Chunk* restrictChunks = nullptr;      // work list of the restrictions (device), by item
  int nbox = 0, nrestrict = 0, nBoxChunks = 0;
  std::vector<int> restrictChunkStart;  // first chunk of each restriction (+ total at the end)
  hc_copy_box* copies = nullptr;        // region copies (device)
  Chunk* copyChunks = nullptr;
  std::vector<hc_copy_box> copyHost;
  std::vector<int> copyStart;
  mutable std::vector<std::pair<int, int>> copyRangesChecked;  // launch ranges already found race free
  hc_cf_fine_box* cfFine = nullptr;     // fine boxes of the <JU> / <U> recovery (device)
  Chunk* cfMappedChunks = nullptr;
  Chunk* cfQuotientChunks = nullptr;
  std::vector<hc_cf_fine_box> cfFineHost;
  std::vector<int> cfMappedStart, cfQuotientStart;
  CfItem* cf = nullptr;                 // coarse-fine interpolation boxes with their weights (device)
  Chunk* cfChunks = nullptr;
  std::vector<hc_cf_box> cfHost;
  std::vector<int> cfChunkStart;
  double* cfScratch = nullptr;          // separable-pass results of every box (device)
  int2* cfPass = nullptr;               // (box, component) of each pass CTA (device)
  std::vector<int> cfPassStart;
  std::vector<char> cfSeparable;        // per box: its planes fit the pass kernel's shared memory
  long long cfPassMax = 0;              // largest shared memory of a separable box (doubles)
  mutable std::vector<std::pair<int, int>> cfRangesChecked, cfFineRangesChecked[2];
};

extern "C" int hc_amr_plan_create(hc_ctx* ctx, const hc_rk_box* boxes, int nbox, const hc_restrict_box* restricts,
                                  int nrestrict, hc_amr_plan** out) {
  if (!ctx || !out || (nbox && !boxes) || (nrestrict && !restricts)) return argFail("hc_amr_plan_create: null argument");
  if (nbox < 0 || nrestrict < 0) return argFail("hc_amr_plan_create: negative count");
  *out = nullptr;
  hc_amr_plan* P = new hc_amr_plan;
  P->nbox = nbox;
  P->nrestrict = nrestrict;
  for (int b = 0; b < nbox; ++b) {
    const hc_rk_box& B = boxes[b];
    if (B.ncells < 0 || (B.ncells > 0 && (!B.state || !B.stage))) {
      delete P;
      return argFail("hc_amr_plan_create: a box needs ncells >= 0, state and stage");
    }
    for (int q = 0; q < 4; ++q)
      if (B.ncells > 0 && !B.rk[q]) {
        delete P;
        return argFail("hc_amr_plan_create: a box needs its four stage right-hand sides");
      }
  }
  for (int r = 0; r < nrestrict; ++r) {
    const hc_restrict_box& R = restricts[r];
    bool ok = R.fine && R.coarse;
    for (int d = 0; d < 3 && ok; ++d) {
      ok = R.ratio[d] >= 1 && R.ratio[d] <= 16 && R.lo[d] <= R.hi[d] && R.fine_n[d] >= 1 && R.coarse_n[d] >= 1 &&
           R.lo[d] >= R.coarse_lo[d] && R.hi[d] < R.coarse_lo[d] + R.coarse_n[d] &&
           (long long)R.lo[d] * R.ratio[d] >= R.fine_lo[d] &&
           ((long long)R.hi[d] + 1) * R.ratio[d] <= (long long)R.fine_lo[d] + R.fine_n[d];
    }
    if (!ok) {
      delete P;
      return argFail("hc_amr_plan_create: a restriction's coarse cells must lie in its coarse box and cover fine "
                     "cells inside its fine box (ratio 1..16)");
    }
  }
  std::vector<Chunk> bc, rc;
  for (int b = 0; b < nbox; ++b) addChunks(bc, b, 8 * boxes[b].ncells);
  for (int r = 0; r < nrestrict; ++r) {
    const hc_restrict_box& R = restricts[r];
    P->restrictChunkStart.push_back((int)rc.size());
    addChunks(rc, r, 8LL * (R.hi[0] - R.lo[0] + 1) * (R.hi[1] - R.lo[1] + 1) * (R.hi[2] - R.lo[2] + 1));
  }
  P->restrictChunkStart.push_back((int)rc.size());
  P->nBoxChunks = (int)bc.size();
  cudaError_t e = cudaSuccess;
  if (!bc.empty()) {
    e = cudaMalloc(&P->boxChunks, sizeof(Chunk) * bc.size());
    if (e == cudaSuccess) e = cudaMemcpy(P->boxChunks, bc.data(), sizeof(Chunk) * bc.size(), cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess && !rc.empty()) {
    e = cudaMalloc(&P->restrictChunks, sizeof(Chunk) * rc.size());
    if (e == cudaSuccess)
      e = cudaMemcpy(P->restrictChunks, rc.data(), sizeof(Chunk) * rc.size(), cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess && nbox) {
    e = cudaMalloc(&P->boxes, sizeof(hc_rk_box) * nbox);
    if (e == cudaSuccess) e = cudaMemcpy(P->boxes, boxes, sizeof(hc_rk_box) * nbox, cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess && nrestrict) {
    e = cudaMalloc(&P->restricts, sizeof(hc_restrict_box) * nrestrict);
    if (e == cudaSuccess)
      e = cudaMemcpy(P->restricts, restricts, sizeof(hc_restrict_box) * nrestrict, cudaMemcpyHostToDevice);
  }
  if (e != cudaSuccess) {
    cudaFree(P->boxes);
    cudaFree(P->restricts);
    cudaFree(P->boxChunks);
    cudaFree(P->restrictChunks);
    delete P;
    return cudaFailed(e, "hc_amr_plan_create");
  }
  *out = P;
  return HC_OK;
}

extern "C" int hc_amr_plan_destroy(hc_amr_plan* P) {
  if (!P) return HC_OK;
  cudaFree(P->natives);
  cudaFree(P->nativeChunks);
  cudaFree(P->boxes);
  cudaFree(P->restricts);
  cudaFree(P->boxChunks);
  cudaFree(P->restrictChunks);
  cudaFree(P->reflux);
  cudaFree(P->refluxChunks);
  cudaFree(P->cf);
  cudaFree(P->cfChunks);
  cudaFree(P->cfScratch);
  cudaFree(P->cfPass);
  cudaFree(P->cfFine);
  cudaFree(P->cfMappedChunks);
  cudaFree(P->cfQuotientChunks);
  cudaFree(P->copies);
  cudaFree(P->copyChunks);
  delete P;
  return HC_OK;
}

extern "C" int hc_amr_plan_set_reflux(hc_amr_plan* P, const hc_reflux_box* patches, int npatch) {
  if (!P || (npatch && !patches) || npatch < 0) return argFail("hc_amr_plan_set_reflux: bad argument");
  for (int r = 0; r < npatch; ++r)
    if (!refluxInside(patches[r]))
      return argFail("hc_amr_plan_set_reflux: a reflux patch must read its faces and write its cells inside its "
                     "arrays' boxes (dir 0..2, side 0/1, ratio 1..16)");
  std::vector<Chunk> rc;
  std::vector<int> start;
  for (int r = 0; r < npatch; ++r) {
    const hc_reflux_box& R = patches[r];
    start.push_back((int)rc.size());
    addChunks(rc, r, 8LL * (R.hi[0] - R.lo[0] + 1) * (R.hi[1] - R.lo[1] + 1) * (R.hi[2] - R.lo[2] + 1));
  }
  start.push_back((int)rc.size());
  hc_reflux_box* dev = nullptr;
  Chunk* devChunks = nullptr;
  cudaError_t e = cudaSuccess;
  if (npatch) {
    e = cudaMalloc(&dev, sizeof(hc_reflux_box) * npatch);
    if (e == cudaSuccess) e = cudaMemcpy(dev, patches, sizeof(hc_reflux_box) * npatch, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&devChunks, sizeof(Chunk) * rc.size());
    if (e == cudaSuccess) e = cudaMemcpy(devChunks, rc.data(), sizeof(Chunk) * rc.size(), cudaMemcpyHostToDevice);
  }
  if (e != cudaSuccess) {
    cudaFree(dev);
    cudaFree(devChunks);
    return cudaFailed(e, "hc_amr_plan_set_reflux");
  }
  cudaFree(P->reflux);
  cudaFree(P->refluxChunks);
  P->reflux = dev;
  P->refluxChunks = devChunks;
  P->refluxHost.assign(patches, patches + npatch);
  P->refluxChunkStart = start;
  return HC_OK;
}

extern "C" int hc_amr_reflux(hc_ctx* ctx, const hc_amr_plan* P, int first, int count, void* stream) {
  if (!ctx || !P) return argFail("hc_amr_reflux: null argument");
  const int n = (int)P->refluxHost.size();
  if (first < 0 || count < 0 || first + count > n) return argFail("hc_amr_reflux: range outside the plan");
  // patches of one launch must correct disjoint coarse cells of each rhs array
  for (int a = first; a < first + count; ++a)
    for (int b = a + 1; b < first + count; ++b) {
      const hc_reflux_box &A = P->refluxHost[a], &B = P->refluxHost[b];
      if (A.rhs != B.rhs) continue;
      bool overlap = true;
      for (int d = 0; d < 3 && overlap; ++d) {
        const int sa = (d == A.dir && A.fine_side) ? 1 : 0, sb = (d == B.dir && B.fine_side) ? 1 : 0;
        overlap = A.lo[d] - sa <= B.hi[d] - sb && B.lo[d] - sb <= A.hi[d] - sa;
      }
      if (overlap) return argFail("hc_amr_reflux: two patches of one launch correct the same coarse cells");
    }
  const int c0 = count ? P->refluxChunkStart[first] : 0, c1 = count ? P->refluxChunkStart[first + count] : 0;
  if (c1 == c0) return HC_OK;
  refluxKernel<<<c1 - c0, kThreads, 0, static_cast<cudaStream_t>(stream)>>>(P->reflux, P->refluxChunks + c0);
  return cudaFailed(cudaGetLastError(), "hc_amr_reflux");
}

extern "C" int hc_amr_rk_stage(hc_ctx* ctx, const hc_amr_plan* P, int order, int stage, double dt, void* stream) {
  if (!ctx || !P) return argFail("hc_amr_rk_stage: null argument");
  if (order != 3 && order != 4) return argFail("hc_amr_rk_stage: order must be 3 or 4");
  if (stage < 0 || stage > order) return argFail("hc_amr_rk_stage: stage must be 0..order");
  if (P->nBoxChunks == 0) return HC_OK;
  const auto& a = order == 3 ? kA3 : kA4;
  const auto& b = order == 3 ? kB3 : kB4;
  RkFactors F{};
  F.final = stage == order ? 1 : 0;
  for (int p = 0; p < 4; ++p) {
    if (F.final) {
      F.use[p] = p < order;
      F.f[p] = dt * b[p];
    } else {
      F.use[p] = p < stage && a[stage][p] != 0.0;
      F.f[p] = dt * a[stage][p];
    }
  }
  rkCombineKernel<<<P->nBoxChunks, kThreads, 0, static_cast<cudaStream_t>(stream)>>>(P->boxes, P->boxChunks, F);
  return cudaFailed(cudaGetLastError(), "hc_amr_rk_stage");
}

extern "C" int hc_amr_restrict(hc_ctx* ctx, const hc_amr_plan* P, int first, int count, void* stream) {
  if (!ctx || !P) return argFail("hc_amr_restrict: null argument");
  if (first < 0 || count < 0 || first + count > P->nrestrict) return argFail("hc_amr_restrict: range outside the plan");
  const int c0 = P->restrictChunkStart[first], c1 = P->restrictChunkStart[first + count];
  if (c1 == c0) return HC_OK;
  restrictKernel<<<c1 - c0, kThreads, 0, static_cast<cudaStream_t>(stream)>>>(P->restricts, P->restrictChunks + c0);
  return cudaFailed(cudaGetLastError(), "hc_amr_restrict");
}

// ---------------------------------------------------------------------------
// Coarse-fine interpolation weights (src/MHD_AMRInterpolation.H:39-56).
// Host arithmetic: the inverse of the five coarse cells' moment matrix in
// exact rationals, rounded to double once, then the child's moments in
// double.
namespace {

struct Rational {
  long long n = 0, d = 1;
};
long long gcdLL(long long a, long long b) {
  a = a < 0 ? -a : a;
  b = b < 0 ? -b : b;
  while (b) {
    const long long t = a % b;
    a = b;
    b = t;
  }
  return a ? a : 1;
}
Rational mk(long long n, long long d) {
  if (d < 0) { n = -n; d = -d; }
  const long long g = gcdLL(n, d);
  return Rational{n / g, d / g};
}
Rational sub(Rational a, Rational b) { return mk(a.n * b.d - b.n * a.d, a.d * b.d); }
Rational mul(Rational a, Rational b) { return mk(a.n * b.n, a.d * b.d); }
Rational divr(Rational a, Rational b) { return mk(a.n * b.d, a.d * b.n); }

// inverse[n][i]: coefficient of the average over coarse cell i (centre
// i - 2) in the n-th coefficient of the quartic matching five averages.
// Row i of the moment matrix holds the averages of x^n over [c - 1/2,
// c + 1/2], c = i - 2: 1, c, c^2 + 1/12, c^3 + c/4, c^4 + c^2/2 + 1/80.
struct InverseMoments {
  double v[5][5];
};
InverseMoments computeInverseMoments() {
  InverseMoments out{};
  Rational a[5][10];
  for (int i = 0; i < 5; ++i) {
    const long long c = i - 2;
    a[i][0] = mk(1, 1);
    a[i][1] = mk(c, 1);
    a[i][2] = mk(12 * c * c + 1, 12);
    a[i][3] = mk(4 * c * c * c + c, 4);
    a[i][4] = mk(80 * c * c * c * c + 40 * c * c + 1, 80);
    for (int j = 0; j < 5; ++j) a[i][5 + j] = mk(i == j ? 1 : 0, 1);
  }
  for (int col = 0; col < 5; ++col) {  // Gauss-Jordan, exact (the matrix is regular)
    int piv = col;
    while (piv < 4 && a[piv][col].n == 0) ++piv;
    if (piv != col)
      for (int j = 0; j < 10; ++j) std::swap(a[piv][j], a[col][j]);
    const Rational pv = a[col][col];
    for (int j = 0; j < 10; ++j) a[col][j] = divr(a[col][j], pv);
    for (int r = 0; r < 5; ++r) {
      if (r == col || a[r][col].n == 0) continue;
      const Rational f = a[r][col];
      for (int j = 0; j < 10; ++j) a[r][j] = sub(a[r][j], mul(f, a[col][j]));
    }
  }
  // a = [I | A^-1] with A[i][n]; A^-1 is indexed [n][i]
  for (int n = 0; n < 5; ++n)
    for (int i = 0; i < 5; ++i) out.v[n][i] = (double)a[n][5 + i].n / (double)a[n][5 + i].d;
  return out;
}
const double (*inverseMoments())[5] {
  static const InverseMoments table = computeInverseMoments();  // initialised once, thread-safe
  return table.v;
}

void cfWeights(int ratio, int child, double w[5]) {
  if (ratio == 1) {
    const double unit[5] = {0, 0, 1, 0, 0};
    for (int i = 0; i < 5; ++i) w[i] = unit[i];
    return;
  }
  const double x = (child + 0.5) / ratio - 0.5, inverse = 1.0 / ratio;
  const double moment[5] = {1, x, x * x + inverse * inverse / 12, x * x * x + x * inverse * inverse / 4,
                            x * x * x * x + x * x * inverse * inverse / 2 + inverse * inverse * inverse * inverse / 80};
  const double(*inv)[5] = inverseMoments();
  for (int i = 0; i < 5; ++i) {
    double v = 0.0;
    for (int n = 0; n < 5; ++n) v += moment[n] * inv[n][i];
    w[i] = v;
  }
}

bool cfBoxOk(const hc_cf_box& B) {
  if (!B.coarse || !B.fine || B.ncomp < 1 || B.ncomp > kCfMaxComp) return false;
  long long fineN = 1, coarseN = 1;
  for (int d = 0; d < 3; ++d) {
    if (B.ratio[d] < 1 || B.ratio[d] > kCfMaxRatio || B.fine_n[d] < 1 || B.coarse_n[d] < 1) return false;
    fineN *= B.fine_n[d];
    coarseN *= B.coarse_n[d];
  }
  return fineN < 0x7fffffffLL && coarseN < 0x7fffffffLL;
}

}  // namespace

extern "C" int hc_amr_cf_weights(int ratio, int child, double* w) {
  if (!w || ratio < 1 || ratio > kCfMaxRatio || child < 0 || child >= ratio)
    return argFail("hc_amr_cf_weights: ratio 1..8 and child 0..ratio-1");
  cfWeights(ratio, child, w);
  return HC_OK;
}

extern "C" int hc_amr_plan_set_cf_interp(hc_amr_plan* P, const hc_cf_box* boxes, int nbox) {
  if (!P || nbox < 0 || (nbox && !boxes)) return argFail("hc_amr_plan_set_cf_interp: bad argument");
  std::vector<CfItem> items(nbox);
  std::vector<Chunk> cc;
  std::vector<int> start;
  for (int b = 0; b < nbox; ++b) {
    if (!cfBoxOk(boxes[b]))
      return argFail("hc_amr_plan_set_cf_interp: a box needs its arrays, ratio 1..8, ncomp 1..16 and boxes of "
                     "fewer than 2^31 cells");
    CfItem& it = items[b];
    it.box = boxes[b];
    for (int d = 0; d < 3; ++d)
      for (int child = 0; child < kCfMaxRatio; ++child) {
        if (child < boxes[b].ratio[d])
          cfWeights(boxes[b].ratio[d], child, it.w[d][child]);
        else
          for (int i = 0; i < 5; ++i) it.w[d][child][i] = 0.0;
      }
    start.push_back((int)cc.size());
    addChunks(cc, b, (long long)boxes[b].fine_n[0] * boxes[b].fine_n[1] * boxes[b].fine_n[2]);
  }
  start.push_back((int)cc.size());
  CfItem* dev = nullptr;
  Chunk* devChunks = nullptr;
  cudaError_t e = cudaSuccess;
  if (nbox) {
    e = cudaMalloc(&dev, sizeof(CfItem) * nbox);
    if (e == cudaSuccess) e = cudaMemcpy(dev, items.data(), sizeof(CfItem) * nbox, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&devChunks, sizeof(Chunk) * cc.size());
    if (e == cudaSuccess) e = cudaMemcpy(devChunks, cc.data(), sizeof(Chunk) * cc.size(), cudaMemcpyHostToDevice);
  }
  if (e != cudaSuccess) {
    cudaFree(dev);
    cudaFree(devChunks);
    return cudaFailed(e, "hc_amr_plan_set_cf_interp");
  }
  // the separable passes: scratch for every box that fits, a CTA per box
  // and component
  std::vector<int2> pass;
  std::vector<int> passStart;
  std::vector<char> separable(nbox, 0);
  long long scratchTotal = 0, passMax = 0;
  for (int b = 0; b < nbox; ++b) {
    passStart.push_back((int)pass.size());
    const long long need = cfPassDoubles(boxes[b]);
    const hc_cf_box& Bb = boxes[b];
    if (need > kCfPassMaxDoubles || Bb.fine_n[0] > kCfPassMaxFine || Bb.fine_n[1] > kCfPassMaxFine ||
        Bb.fine_n[2] > kCfPassMaxFine)
      continue;
    separable[b] = 1;
    passMax = std::max(passMax, need);
    items[b].scratch = scratchTotal;
    scratchTotal += (long long)boxes[b].ncomp * boxes[b].fine_n[0] * boxes[b].fine_n[1] * boxes[b].fine_n[2];
    for (int c = 0; c < boxes[b].ncomp; ++c) pass.push_back(make_int2(b, c));
  }
  passStart.push_back((int)pass.size());
  double* scr = nullptr;
  int2* devPass = nullptr;
  if (e == cudaSuccess && nbox) e = cudaMemcpy(dev, items.data(), sizeof(CfItem) * nbox, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && scratchTotal) e = cudaMalloc(&scr, sizeof(double) * scratchTotal);
  if (e == cudaSuccess && !pass.empty()) e = cudaMalloc(&devPass, sizeof(int2) * pass.size());
  if (e == cudaSuccess && !pass.empty())
    e = cudaMemcpy(devPass, pass.data(), sizeof(int2) * pass.size(), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(dev);
    cudaFree(devChunks);
    cudaFree(scr);
    cudaFree(devPass);
    return cudaFailed(e, "hc_amr_plan_set_cf_interp");
  }
  cudaFree(P->cf);
  cudaFree(P->cfChunks);
  cudaFree(P->cfScratch);
  cudaFree(P->cfPass);
  P->cf = dev;
  P->cfChunks = devChunks;
  P->cfScratch = scr;
  P->cfPass = devPass;
  P->cfPassStart = passStart;
  P->cfSeparable = separable;
  P->cfPassMax = passMax;
  P->cfHost.assign(boxes, boxes + nbox);
  P->cfChunkStart = start;
  P->cfRangesChecked.clear();
  return HC_OK;
}

extern "C" int hc_amr_cf_interpolate(hc_ctx* ctx, const hc_amr_plan* P, int first, int count, void* stream) {
  if (!ctx || !P) return argFail("hc_amr_cf_interpolate: null argument");
  const int n = (int)P->cfHost.size();
  if (first < 0 || count < 0 || first + count > n) return argFail("hc_amr_cf_interpolate: range outside the plan");
  // boxes of one launch must write disjoint fine regions of each array
  // (checked once per launch range: the boxes of a plan do not change)
  const std::pair<int, int> range{first, count};
  if (std::find(P->cfRangesChecked.begin(), P->cfRangesChecked.end(), range) == P->cfRangesChecked.end()) {
    for (int a = first; a < first + count; ++a)
      for (int b = a + 1; b < first + count; ++b) {
        const hc_cf_box &A = P->cfHost[a], &B = P->cfHost[b];
        if (A.fine != B.fine) continue;
        bool overlap = true;
        for (int d = 0; d < 3 && overlap; ++d)
          overlap = A.fine_lo[d] < B.fine_lo[d] + B.fine_n[d] && B.fine_lo[d] < A.fine_lo[d] + A.fine_n[d];
        if (overlap) return argFail("hc_amr_cf_interpolate: two boxes of one launch write the same fine array region");
      }
    P->cfRangesChecked.push_back(range);
  }
  const int c0 = count ? P->cfChunkStart[first] : 0, c1 = count ? P->cfChunkStart[first + count] : 0;
  if (c1 == c0) return HC_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  bool separable = true;
  for (int a = first; a < first + count && separable; ++a) separable = P->cfSeparable[a] != 0;
  if (separable) {
    // separable passes into scratch, then the commit of the finite ghosts
    const size_t smem = sizeof(double) * (size_t)P->cfPassMax;
    cudaError_t e = cudaFuncSetAttribute(cfPassKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cudaFailed(e, "hc_amr_cf_interpolate");
    const int p0 = P->cfPassStart[first], p1 = P->cfPassStart[first + count];
    cfPassKernel<<<p1 - p0, kThreads, smem, s>>>(P->cf, P->cfPass + p0, P->cfScratch);
    if ((e = cudaGetLastError()) != cudaSuccess) return cudaFailed(e, "hc_amr_cf_interpolate");
    cfCommitKernel<<<c1 - c0, kThreads, 0, s>>>(P->cf, P->cfChunks + c0, P->cfScratch);
    return cudaFailed(cudaGetLastError(), "hc_amr_cf_interpolate");
  }
  cfInterpKernel<<<c1 - c0, kThreads, 0, s>>>(P->cf, P->cfChunks + c0);
  return cudaFailed(cudaGetLastError(), "hc_amr_cf_interpolate");
}

namespace {

// region lo .. hi (inclusive) inside the box (lo, n)
bool regionIn(const int lo[3], const int hi[3], const int blo[3], const int bn[3]) {
  for (int d = 0; d < 3; ++d)
    if (lo[d] < blo[d] || hi[d] >= (long long)blo[d] + bn[d]) return false;
  return true;
}

bool cfFineOk(const hc_cf_fine_box& B) {
  if (!B.jac || !B.donor || !B.state || !B.mapped || !B.out) return false;
  int g3lo[3], g3hi[3], g2lo[3], g2hi[3];
  for (int d = 0; d < 3; ++d) {
    if (B.valid_lo[d] > B.valid_hi[d] || B.block_hi[d] - B.block_lo[d] < 2) return false;
    if (B.valid_lo[d] < B.block_lo[d] || B.valid_hi[d] > B.block_hi[d]) return false;
    if (B.jac_n[d] < 1 || B.donor_n[d] < 1 || B.state_n[d] < 1 || B.mapped_n[d] < 1 || B.out_n[d] < 1) return false;
    g3lo[d] = B.valid_lo[d] - 3; g3hi[d] = B.valid_hi[d] + 3;
    g2lo[d] = B.valid_lo[d] - 2; g2hi[d] = B.valid_hi[d] + 2;
  }
  const int* vlo = B.valid_lo;
  const int* vhi = B.valid_hi;
  // the mapped box is valid.grow(2) (its cells read J and the donor one
  // cell further out)
  for (int d = 0; d < 3; ++d)
    if (B.mapped_lo[d] != g2lo[d] || B.mapped_n[d] != g2hi[d] - g2lo[d] + 1) return false;
  long long sizes[5] = {1, 1, 1, 1, 1};
  for (int d = 0; d < 3; ++d) {
    sizes[0] *= B.jac_n[d]; sizes[1] *= B.donor_n[d]; sizes[2] *= B.state_n[d];
    sizes[3] *= B.mapped_n[d]; sizes[4] *= B.out_n[d];
  }
  for (long long v : sizes)
    if (8 * v >= 0x7fffffffLL) return false;
  return regionIn(g3lo, g3hi, B.jac_lo, B.jac_n) && regionIn(g3lo, g3hi, B.donor_lo, B.donor_n) &&
         regionIn(vlo, vhi, B.state_lo, B.state_n) && regionIn(vlo, vhi, B.out_lo, B.out_n);
}

}  // namespace

extern "C" int hc_amr_plan_set_cf_fine(hc_amr_plan* P, const hc_cf_fine_box* boxes, int nbox) {
  if (!P || nbox < 0 || (nbox && !boxes)) return argFail("hc_amr_plan_set_cf_fine: bad argument");
  std::vector<Chunk> mc, qc;
  std::vector<int> ms, qs;
  for (int b = 0; b < nbox; ++b) {
    const hc_cf_fine_box& B = boxes[b];
    if (!cfFineOk(B))
      return argFail("hc_amr_plan_set_cf_fine: a box needs its five arrays, J and the donor on valid.grow(3), the "
                     "mapped box equal to valid.grow(2), state and out on valid, a block containing valid and at "
                     "least 3 cells wide");
    ms.push_back((int)mc.size());
    addChunks(mc, b, (long long)B.mapped_n[0] * B.mapped_n[1] * B.mapped_n[2]);
    qs.push_back((int)qc.size());
    addChunks(qc, b, (long long)(B.valid_hi[0] - B.valid_lo[0] + 1) * (B.valid_hi[1] - B.valid_lo[1] + 1) *
                         (B.valid_hi[2] - B.valid_lo[2] + 1));
  }
  ms.push_back((int)mc.size());
  qs.push_back((int)qc.size());
  hc_cf_fine_box* dev = nullptr;
  Chunk *devM = nullptr, *devQ = nullptr;
  cudaError_t e = cudaSuccess;
  if (nbox) {
    e = cudaMalloc(&dev, sizeof(hc_cf_fine_box) * nbox);
    if (e == cudaSuccess) e = cudaMemcpy(dev, boxes, sizeof(hc_cf_fine_box) * nbox, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&devM, sizeof(Chunk) * mc.size());
    if (e == cudaSuccess) e = cudaMemcpy(devM, mc.data(), sizeof(Chunk) * mc.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&devQ, sizeof(Chunk) * qc.size());
    if (e == cudaSuccess) e = cudaMemcpy(devQ, qc.data(), sizeof(Chunk) * qc.size(), cudaMemcpyHostToDevice);
  }
  if (e != cudaSuccess) {
    cudaFree(dev);
    cudaFree(devM);
    cudaFree(devQ);
    return cudaFailed(e, "hc_amr_plan_set_cf_fine");
  }
  cudaFree(P->cfFine);
  cudaFree(P->cfMappedChunks);
  cudaFree(P->cfQuotientChunks);
  P->cfFine = dev;
  P->cfMappedChunks = devM;
  P->cfQuotientChunks = devQ;
  P->cfFineHost.assign(boxes, boxes + nbox);
  P->cfMappedStart = ms;
  P->cfQuotientStart = qs;
  P->cfFineRangesChecked[0].clear();
  P->cfFineRangesChecked[1].clear();
  return HC_OK;
}

namespace {
int cfFineLaunch(hc_ctx* ctx, const hc_amr_plan* P, int first, int count, void* stream, bool mapped) {
  const char* what = mapped ? "hc_amr_cf_mapped" : "hc_amr_cf_quotient";
  if (!ctx || !P) return argFail(mapped ? "hc_amr_cf_mapped: null argument" : "hc_amr_cf_quotient: null argument");
  const int n = (int)P->cfFineHost.size();
  if (first < 0 || count < 0 || first + count > n)
    return argFail(mapped ? "hc_amr_cf_mapped: range outside the plan" : "hc_amr_cf_quotient: range outside the plan");
  auto& checked = P->cfFineRangesChecked[mapped ? 0 : 1];
  const std::pair<int, int> range{first, count};
  if (std::find(checked.begin(), checked.end(), range) == checked.end()) {
    for (int a = first; a < first + count; ++a)
      for (int b = a + 1; b < first + count; ++b) {
        const hc_cf_fine_box &A = P->cfFineHost[a], &B = P->cfFineHost[b];
        if ((mapped && A.mapped == B.mapped) || (!mapped && A.out == B.out))
          return argFail(mapped ? "hc_amr_cf_mapped: two boxes of one launch write the same array"
                                : "hc_amr_cf_quotient: two boxes of one launch write the same array");
      }
    checked.push_back(range);
  }
  const std::vector<int>& st = mapped ? P->cfMappedStart : P->cfQuotientStart;
  const int c0 = count ? st[first] : 0, c1 = count ? st[first + count] : 0;
  if (c1 == c0) return HC_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (mapped)
    cfMappedKernel<<<c1 - c0, kThreads, 0, s>>>(P->cfFine, P->cfMappedChunks + c0);
  else
    cfQuotientKernel<<<c1 - c0, kThreads, 0, s>>>(P->cfFine, P->cfQuotientChunks + c0);
  return cudaFailed(cudaGetLastError(), what);
}
}  // namespace

extern "C" int hc_amr_cf_mapped(hc_ctx* ctx, const hc_amr_plan* P, int first, int count, void* stream) {
  return cfFineLaunch(ctx, P, first, count, stream, true);
}

extern "C" int hc_amr_cf_quotient(hc_ctx* ctx, const hc_amr_plan* P, int first, int count, void* stream) {
  return cfFineLaunch(ctx, P, first, count, stream, false);
}

// ---------------------------------------------------------------------------
// Native conversion and radial ghosts of fine boxes (the level's stage
// preparation, step 3, on boxes).
namespace {

__device__ __forceinline__ long nbOff(const int lo[3], const int n[3], int i, int j, int k) {
  return (long)(i - lo[0]) + (long)n[0] * ((long)(j - lo[1]) + (long)n[1] * (long)(k - lo[2]));
}

__global__ void __launch_bounds__(kThreads, 2) nativeBoxKernel(const hc::O4Level O, const hc_native_box* __restrict__ boxes,
                                                            const Chunk* __restrict__ chunks, double t) {
  const Chunk ch = chunks[blockIdx.x];
  const hc_native_box B = boxes[ch.item];
  const long NU = (long)B.usph_n[0] * B.usph_n[1] * B.usph_n[2];
  const long NC = (long)B.cart_n[0] * B.cart_n[1] * B.cart_n[2];
  const int b = B.block;
  for (long long e = ch.begin + threadIdx.x; e < ch.end; e += kThreads) {
    int i, j, k;
    split3(e, B.usph_n[0], B.usph_n[1], i, j, k);
    i += B.usph_lo[0];
    j += B.usph_lo[1];
    k += B.usph_lo[2];
    double u[8];
    auto native = [&](int ii, double out[8]) {
      hc::o4NativeCore(B.cart + nbOff(B.cart_lo, B.cart_n, ii, j, k), B.cart_n[0], (long)B.cart_n[0] * B.cart_n[1], NC,
                   O.coef + (((long)b * O.nA + (k + O.ga)) * O.nA + (j + O.ga)) * 27, 27, 27L * O.nA, out);
    };
    if (i < 0) {
      const long cell = ((long)b * O.nG + (k + O.g)) * O.nG + (j + O.g);
      if (O.inner) {
        const double* w = O.inner + (cell * O.g + (i + O.g)) * 8;
#pragma unroll
        for (int c = 0; c < 8; ++c) u[c] = w[c];
      } else {
        const double* xh = O.xhat + cell * 3;
        const double radius = O.radial[i + O.g + 1].y;
        const double X[3] = {radius * xh[0], radius * xh[1], radius * xh[2]};
        hc::windConserved(O.gamma, O.r0, O.strength, X, t, u);
      }
    } else if (i < O.nr) {
      native(i, u);
    } else {
      native(O.nr - 1, u);
      const double rl = O.radial[O.nr - 1 + O.g + 1].y, rr = O.radial[i + O.g + 1].y;
      const double s2 = pow(rl / rr, 2.0), s1 = pow(rl / rr, 1.0);
#pragma unroll
      for (int c = 0; c < 8; ++c) u[c] *= c < 6 ? s2 : s1;
    }
    double* o = B.usph + nbOff(B.usph_lo, B.usph_n, i, j, k);
#pragma unroll
    for (int c = 0; c < 8; ++c) o[c * NU] = u[c];
  }
}

bool nativeShapeOk(const hc_native_box& B) {
  if (!B.cart || !B.usph || B.block < 0 || B.block > 5) return false;
  long long nu = 1, nc = 1;
  for (int d = 0; d < 3; ++d) {
    if (B.usph_n[d] < 1 || B.cart_n[d] < 1) return false;
    nu *= B.usph_n[d];
    nc *= B.cart_n[d];
  }
  return 8 * nu < 0x7fffffffLL && 8 * nc < 0x7fffffffLL;
}

// The box against the level: usph cells inside the tables' range, the cart
// box holding every cell the conversion reads.
bool nativeFits(const hc_native_box& B, const hc::O4Level& O) {
  const int ulo0 = B.usph_lo[0], uhi0 = B.usph_lo[0] + B.usph_n[0] - 1;
  for (int d = 1; d < 3; ++d)
    if (B.usph_lo[d] < -O.g || B.usph_lo[d] + B.usph_n[d] > O.na + O.g) return false;
  if (ulo0 < -O.g || uhi0 >= O.nr + O.g) return false;
  const int i0 = ulo0 < 0 ? 0 : ulo0, i1 = uhi0 >= O.nr ? O.nr - 1 : uhi0;
  if (uhi0 < 0) return true;  // inner ghosts only
  const int need_lo[3] = {uhi0 >= O.nr && ulo0 >= O.nr ? O.nr - 1 : i0, B.usph_lo[1] - 1, B.usph_lo[2] - 1};
  const int need_hi[3] = {i1, B.usph_lo[1] + B.usph_n[1], B.usph_lo[2] + B.usph_n[2]};
  for (int d = 0; d < 3; ++d)
    if (need_lo[d] < B.cart_lo[d] || need_hi[d] > B.cart_lo[d] + B.cart_n[d] - 1) return false;
  return true;
}

}  // namespace

extern "C" int hc_amr_plan_set_native(hc_amr_plan* P, const hc_native_box* boxes, int nbox) {
  if (!P || nbox < 0 || (nbox && !boxes)) return argFail("hc_amr_plan_set_native: bad argument");
  std::vector<Chunk> ch;
  std::vector<int> st;
  for (int b = 0; b < nbox; ++b) {
    if (!nativeShapeOk(boxes[b]))
      return argFail("hc_amr_plan_set_native: a box needs cart and usph arrays, a block 0..5 and non-empty boxes");
    st.push_back((int)ch.size());
    addChunks(ch, b, (long long)boxes[b].usph_n[0] * boxes[b].usph_n[1] * boxes[b].usph_n[2]);
  }
  st.push_back((int)ch.size());
  hc_native_box* dev = nullptr;
  Chunk* devC = nullptr;
  cudaError_t e = cudaSuccess;
  if (nbox) {
    e = cudaMalloc(&dev, sizeof(hc_native_box) * nbox);
    if (e == cudaSuccess) e = cudaMemcpy(dev, boxes, sizeof(hc_native_box) * nbox, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&devC, sizeof(Chunk) * ch.size());
    if (e == cudaSuccess) e = cudaMemcpy(devC, ch.data(), sizeof(Chunk) * ch.size(), cudaMemcpyHostToDevice);
  }
  if (e != cudaSuccess) {
    cudaFree(dev);
    cudaFree(devC);
    return cudaFailed(e, "hc_amr_plan_set_native");
  }
  cudaFree(P->natives);
  cudaFree(P->nativeChunks);
  P->natives = dev;
  P->nativeChunks = devC;
  P->nativeHost.assign(boxes, boxes + nbox);
  P->nativeStart = st;
  P->nativeRangesChecked.clear();
  return HC_OK;
}

extern "C" int hc_amr_native(hc_ctx* ctx, const hc_amr_plan* P, int first, int count, double t, void* stream) {
  if (!ctx || !P) return argFail("hc_amr_native: null argument");
  const hc::O4Level* O = hc::ctxO4Level(ctx);
  if (!O) return hc::setLastError(HC_ERR_UNSUPPORTED, "hc_amr_native: the context is not fourth order");
  const int n = (int)P->nativeHost.size();
  if (first < 0 || count < 0 || first + count > n) return argFail("hc_amr_native: range outside the plan");
  const std::pair<int, int> range{first, count};
  if (std::find(P->nativeRangesChecked.begin(), P->nativeRangesChecked.end(), range) == P->nativeRangesChecked.end()) {
    for (int a = first; a < first + count; ++a) {
      if (!nativeFits(P->nativeHost[a], *O))
        return argFail("hc_amr_native: a usph box leaves the level's tables or its cart box misses cells the "
                       "conversion reads");
      for (int b = a + 1; b < first + count; ++b)
        if (P->nativeHost[a].usph == P->nativeHost[b].usph)
          return argFail("hc_amr_native: two boxes of one launch write the same array");
    }
    P->nativeRangesChecked.push_back(range);
  }
  const int c0 = count ? P->nativeStart[first] : 0, c1 = count ? P->nativeStart[first + count] : 0;
  if (c1 == c0) return HC_OK;
  nativeBoxKernel<<<c1 - c0, kThreads, 0, static_cast<cudaStream_t>(stream)>>>(*O, P->natives,
                                                                                P->nativeChunks + c0, t);
  return cudaFailed(cudaGetLastError(), "hc_amr_native");
}

// ---------------------------------------------------------------------------
// Region copies.
namespace {

struct Box3i {
  int lo[3], hi[3];
};
bool overlaps(const Box3i& a, const Box3i& b) {
  for (int d = 0; d < 3; ++d)
    if (a.hi[d] < b.lo[d] || b.hi[d] < a.lo[d]) return false;
  return true;
}
// image of the copy's region in the destination index space
Box3i copyImage(const hc_copy_box& C) {
  Box3i r;
  for (int d = 0; d < 3; ++d) {
    const int a = C.sign[d] * C.lo[C.perm[d]] + C.shift[d], b = C.sign[d] * C.hi[C.perm[d]] + C.shift[d];
    r.lo[d] = a < b ? a : b;
    r.hi[d] = a < b ? b : a;
  }
  return r;
}
Box3i copyRegion(const hc_copy_box& C) {
  Box3i r;
  for (int d = 0; d < 3; ++d) { r.lo[d] = C.lo[d]; r.hi[d] = C.hi[d]; }
  return r;
}
bool copyOk(const hc_copy_box& C) {
  if (!C.src || !C.dst || C.ncomp < 1 || C.ncomp > 16) return false;
  bool seen[3] = {false, false, false};
  long long sN = 1, dN = 1;
  for (int d = 0; d < 3; ++d) {
    if (C.perm[d] < 0 || C.perm[d] > 2 || seen[C.perm[d]]) return false;
    seen[C.perm[d]] = true;
    if (C.sign[d] != 1 && C.sign[d] != -1) return false;
    if (C.lo[d] > C.hi[d] || C.src_n[d] < 1 || C.dst_n[d] < 1) return false;
    sN *= C.src_n[d];
    dN *= C.dst_n[d];
  }
  if (16 * sN >= 0x7fffffffLL || 16 * dN >= 0x7fffffffLL) return false;
  const Box3i img = copyImage(C);
  return regionIn(C.lo, C.hi, C.src_lo, C.src_n) && regionIn(img.lo, img.hi, C.dst_lo, C.dst_n);
}

}  // namespace

extern "C" int hc_amr_plan_set_copies(hc_amr_plan* P, const hc_copy_box* copies, int ncopy) {
  if (!P || ncopy < 0 || (ncopy && !copies)) return argFail("hc_amr_plan_set_copies: bad argument");
  std::vector<Chunk> cc;
  std::vector<int> start;
  for (int q = 0; q < ncopy; ++q) {
    if (!copyOk(copies[q]))
      return argFail("hc_amr_plan_set_copies: a copy needs both arrays, a signed permutation, ncomp 1..16, its "
                     "region in the source box and the region's image in the destination box");
    start.push_back((int)cc.size());
    const hc_copy_box& C = copies[q];
    addChunks(cc, q, (long long)(C.hi[0] - C.lo[0] + 1) * (C.hi[1] - C.lo[1] + 1) * (C.hi[2] - C.lo[2] + 1));
  }
  start.push_back((int)cc.size());
  hc_copy_box* dev = nullptr;
  Chunk* devChunks = nullptr;
  cudaError_t e = cudaSuccess;
  if (ncopy) {
    e = cudaMalloc(&dev, sizeof(hc_copy_box) * ncopy);
    if (e == cudaSuccess) e = cudaMemcpy(dev, copies, sizeof(hc_copy_box) * ncopy, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&devChunks, sizeof(Chunk) * cc.size());
    if (e == cudaSuccess) e = cudaMemcpy(devChunks, cc.data(), sizeof(Chunk) * cc.size(), cudaMemcpyHostToDevice);
  }
  if (e != cudaSuccess) {
    cudaFree(dev);
    cudaFree(devChunks);
    return cudaFailed(e, "hc_amr_plan_set_copies");
  }
  cudaFree(P->copies);
  cudaFree(P->copyChunks);
  P->copies = dev;
  P->copyChunks = devChunks;
  P->copyHost.assign(copies, copies + ncopy);
  P->copyStart = start;
  P->copyRangesChecked.clear();
  return HC_OK;
}

extern "C" int hc_amr_copy(hc_ctx* ctx, const hc_amr_plan* P, int first, int count, void* stream) {
  if (!ctx || !P) return argFail("hc_amr_copy: null argument");
  const int n = (int)P->copyHost.size();
  if (first < 0 || count < 0 || first + count > n) return argFail("hc_amr_copy: range outside the plan");
  // per array: every written region against every other access of that
  // array in the launch (reads and writes), grouped by array; a range found
  // race free is remembered (the copies of a plan do not change)
  const std::pair<int, int> range{first, count};
  const bool known = std::find(P->copyRangesChecked.begin(), P->copyRangesChecked.end(), range) !=
                     P->copyRangesChecked.end();
  std::vector<std::pair<const void*, std::pair<Box3i, int>>> acc;  // array, (region, copy index * 2 + write)
  for (int q = first; q < first + count && !known; ++q) {
    const hc_copy_box& C = P->copyHost[q];
    acc.push_back({C.src, {copyRegion(C), 2 * q}});
    acc.push_back({C.dst, {copyImage(C), 2 * q + 1}});
  }
  std::sort(acc.begin(), acc.end(), [](const auto& a, const auto& b) {
    return std::less<const void*>()(a.first, b.first);
  });
  for (size_t a = 0; a < acc.size(); ++a)
    for (size_t b = a + 1; b < acc.size() && acc[b].first == acc[a].first; ++b) {
      const bool wa = acc[a].second.second & 1, wb = acc[b].second.second & 1;
      if (!wa && !wb) continue;
      if (overlaps(acc[a].second.first, acc[b].second.first))
        return argFail("hc_amr_copy: a copy of the launch writes a region another access of the launch uses");
    }
  // distinct base pointers must not share memory where one of them is
  // written (sub-views of one allocation would escape the check above)
  if (!known) {
    struct Span { uintptr_t lo, hi; const void* base; bool write; };
    std::vector<Span> spans;
    for (int q = first; q < first + count; ++q) {
      const hc_copy_box& C = P->copyHost[q];
      const uintptr_t ns = (uintptr_t)C.ncomp * C.src_n[0] * C.src_n[1] * C.src_n[2] * sizeof(double);
      const uintptr_t nd = (uintptr_t)C.ncomp * C.dst_n[0] * C.dst_n[1] * C.dst_n[2] * sizeof(double);
      spans.push_back({(uintptr_t)C.src, (uintptr_t)C.src + ns, C.src, false});
      spans.push_back({(uintptr_t)C.dst, (uintptr_t)C.dst + nd, C.dst, true});
    }
    // one span per base pointer: its largest extent, written if any access writes
    std::sort(spans.begin(), spans.end(), [](const Span& a, const Span& b) {
      return a.lo != b.lo ? a.lo < b.lo : a.hi > b.hi;
    });
    std::vector<Span> merged;
    for (const Span& x : spans) {
      if (!merged.empty() && merged.back().base == x.base) {
        merged.back().hi = std::max(merged.back().hi, x.hi);
        merged.back().write = merged.back().write || x.write;
      } else {
        merged.push_back(x);
      }
    }
    for (size_t a = 0; a < merged.size(); ++a)
      for (size_t b = a + 1; b < merged.size() && merged[b].lo < merged[a].hi; ++b)
        if (merged[a].write || merged[b].write)
          return argFail("hc_amr_copy: two arrays of the launch share memory through different base pointers");
  }
  if (!known) P->copyRangesChecked.push_back(range);
  const int c0 = count ? P->copyStart[first] : 0, c1 = count ? P->copyStart[first + count] : 0;
  if (c1 == c0) return HC_OK;
  copyKernel<<<c1 - c0, kThreads, 0, static_cast<cudaStream_t>(stream)>>>(P->copies, P->copyChunks + c0);
  return cudaFailed(cudaGetLastError(), "hc_amr_copy");
}

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

#include <cstdio>
#include <vector>

#include "../../include/hc_abi.h"
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
  cudaFree(P->boxes);
  cudaFree(P->restricts);
  cudaFree(P->boxChunks);
  cudaFree(P->restrictChunks);
  cudaFree(P->reflux);
  cudaFree(P->refluxChunks);
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

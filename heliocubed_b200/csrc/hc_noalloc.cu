// hc_level_rk4_step_noalloc: the level RK4 step for callers that cannot
// allocate device memory when they step.
//
// Who needs it: a host that must not call cudaMalloc once it is running --
// code stepping inside a CUDA stream capture (allocation is not a capturable
// operation), an embedding framework that owns all device memory through its
// own pool and forbids driver allocations after start-up, or a real-time
// serving loop that must not stall on the allocator.  Those callers still
// create the context once (geometry) but do not want the per-context stage
// workspace that hc_level_rk4_step uses.
//
// How: the stage workspace (two ghosted primitive buffers and the RK
// accumulator) lives in one file-scope device array of fixed size.  Every GPU
// that loads this library holds that array until the process exits.  All
// calls on a device share it and it keeps the last call's contents, so calls
// whose kernels overlap on the GPU (two streams, two contexts, two threads)
// race on it: serialise them.  Nothing in it needs to start at zero: every
// cell the kernels read is written earlier in the same call (panel-corner
// ghosts are never read).
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/hc_abi.h"
#include "hc_level.h"

namespace {

// 2 Mi doubles (16 MiB): room for levels of up to 6 x 21 x 21^2 cells
// (2 * 6*8*(nr+4)*(na+4)^2 + 6*8*nr*na^2 doubles).
constexpr size_t kScratchDoubles = size_t(2) * 1024 * 1024;
static __device__ __align__(256) double g_stageScratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_setupMutex;
double* g_scratchAddress[kMaxDevices] = {};

// Device address of the array on the current device, looked up once per
// device.  In host code the array's name is only a host-side stand-in, not a
// device address; only this lookup yields the pointer the kernels may use.
int scratchOnDevice(int device, double** out) {
  if (device < 0 || device >= kMaxDevices) return hc::setLastError(HC_ERR_ARG, "device index out of range");
  std::lock_guard<std::mutex> lock(g_setupMutex);
  if (!g_scratchAddress[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_stageScratch);
    if (e != cudaSuccess) {
      char msg[256];
      std::snprintf(msg, sizeof msg, "hc_level_rk4_step_noalloc: cudaGetSymbolAddress failed: %s",
                    cudaGetErrorString(e));
      return hc::setLastError(HC_ERR_CUDA, msg);
    }
    g_scratchAddress[device] = static_cast<double*>(p);
  }
  *out = g_scratchAddress[device];
  return HC_OK;
}

int launched(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return HC_OK;
  char msg[256];
  std::snprintf(msg, sizeof msg, "hc_level_rk4_step_noalloc: %s: %s", what, cudaGetErrorString(e));
  return hc::setLastError(HC_ERR_CUDA, msg);
}

}  // namespace

extern "C" int hc_level_rk4_step_noalloc(hc_ctx* ctx, double* ju, double dt, double t, void* stream) {
  using namespace hc;
  if (!ctx || !ju) return setLastError(HC_ERR_ARG, "hc_level_rk4_step_noalloc: null argument");
  if (!(dt > 0)) return setLastError(HC_ERR_ARG, "hc_level_rk4_step_noalloc: dt must be positive");
  const DevLevel& L = *ctxLevel(ctx);
  const hc_params& P = *ctxParams(ctx);
  if (P.spatial_order != 2)
    return setLastError(HC_ERR_UNSUPPORTED, "hc_level_rk4_step_noalloc: only second-order contexts are supported");
  const size_t wDoubles = 6 * size_t(NC) * size_t(L.Ng), accDoubles = 6 * size_t(NC) * size_t(L.Nv);
  const size_t need = 2 * wDoubles + accDoubles;
  if (need > kScratchDoubles) {
    char msg[320];
    std::snprintf(msg, sizeof msg,
                  "hc_level_rk4_step_noalloc: a %d x %d^2 x 6 level needs %zu doubles of stage workspace; the "
                  "built-in workspace holds %zu (16 MiB). Use hc_level_rk4_step for larger levels.",
                  P.nr, P.na, need, kScratchDoubles);
    return setLastError(HC_ERR_ARG, msg);
  }
  int current = -1;
  cudaError_t e = cudaGetDevice(&current);
  if (e != cudaSuccess) return launched(e, "cudaGetDevice");
  if (current != ctxDevice(ctx))
    return setLastError(HC_ERR_ARG, "hc_level_rk4_step_noalloc: make the context's device current first");
  double* scratch = nullptr;
  int rc = scratchOnDevice(current, &scratch);
  if (rc != HC_OK) return rc;
  double* W[2] = {scratch, scratch + wDoubles};
  double* acc = scratch + 2 * wDoubles;
  cudaStream_t s = static_cast<cudaStream_t>(stream);

  rc = launched(launchPrimValid(L, ju, W[0], s), "primitives");
  static const double c4[4] = {0, 0.5, 0.5, 1};
  for (int stage = 0; stage < 4 && rc == HC_OK; ++stage) {
    StageTime st{t, nullptr, c4[stage], nullptr, dt};
    rc = launched(launchGhosts(L, W[stage % 2], st, s), "ghosts");
    if (rc != HC_OK) break;
    StageArgs a{};
    a.L = L;
    a.w = W[stage % 2];
    a.wBoxStride = NC * L.Ng;
    a.wN = L.Ng;
    for (int d = 0; d < 3; ++d) a.wlo[d] = -kGhost;
    a.wn[0] = L.n0;
    a.wn[1] = L.n1;
    a.wn[2] = L.n1;
    a.lo[0] = a.lo[1] = a.lo[2] = 0;
    a.hi[0] = P.nr - 1;
    a.hi[1] = a.hi[2] = P.na - 1;
    a.nbox = 6;
    a.block0 = 0;
    a.scale = 1.0;
    a.seams = 1;
    a.stage = stage;
    a.invDtMax = nullptr;
    a.dtv = dt;
    a.ju = ju;
    a.acc = acc;
    a.wOut = W[(stage + 1) % 2];
    a.invMaxOut = nullptr;
    a.invalid = nullptr;
    a.tbase = t;
    rc = launched(launchStage(a, MODE_RK, P.limiter, P.riemann_solver == 2, P.divergence_cleaning == 1,
                              P.sun_gravity == 1, s),
                  "stage");
  }
  return rc;
}

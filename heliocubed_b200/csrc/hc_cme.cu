// Cone CME, finite spherical cloud (CME field model 4): host preparation of
// the cloud from its fitted parameters and the device volume insertion into
// a level state.
//
// Preparation restates src/MHD_CME.H:1069-1136 (drag-based trajectory,
// boundary-contact bisection, prepareConeCloud) with the analytic cone's
// axis orientation(lat, lon, 0) (0,0,1) (src/MHD_ImportedCME.H:72-79,
// 415-418).  Insertion restates the cone branch of Insert_CME
// (src/BoxOp_EulerCubedSphereImplem.H:1236-1300): per valid cell, sample()
// of the finite cloud (src/MHD_CME.H:995-1018) at the shift of
// expandedSource (:1139-1143), the ambient Cartesian primitives of
// cartesianPrimitiveFromConserved, increment() with the prescribed cone
// plasma (:1197-1238) and JU += J delta.  One thread per cell, radial index
// fastest, so every component access is coalesced; the statistics are
// reduced in a fixed order (block tree, then one block over the partials).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>

#include "../../include/hc_abi.h"
#include "hc_device.cuh"
#include "hc_level.h"

namespace {

constexpr double kSolarRadius = 69600000000.0;  // c_SR, src/MHD_Constants.H:4
constexpr double kBoltzmann = 1.380649e-16;
constexpr double kPiCme = 3.1415926535897932384626433832795;
constexpr int kInsertThreads = 256;
constexpr int kInsertMaxBlocks = 148 * 8;

struct Trajectory {
  double apex, wind, drag, height, reference;
};

// Drag-based model position of the leading edge, src/MHD_CME.H:1069-1085.
bool trajectory(const Trajectory& c, double elapsed, double& height, double& speed) {
  const double dv = c.apex - c.wind;
  double distance = c.apex * elapsed;
  speed = c.apex;
  if (c.drag > 0 && dv != 0) {
    const double argument = c.drag * std::abs(dv) * elapsed;
    if (!(argument > -1)) return false;
    distance = c.wind * elapsed + std::copysign(1., dv) * std::log1p(argument) / c.drag;
    speed = c.wind + dv / (1 + argument);
  }
  height = c.height + 0.0 + distance * 1e5 / kSolarRadius;
  return std::isfinite(height) && std::isfinite(speed) && speed > 0;
}

// First contact of the leading edge with the inner boundary,
// src/MHD_CME.H:1087-1110 (bisection of 100 halvings).
bool boundaryStart(const Trajectory& c, double innerRsun, double& start) {
  double lower = -(c.height + 0.0 - innerRsun) * kSolarRadius / (c.apex * 1e5), upper = 0;
  const double dv = c.apex - c.wind;
  if (c.drag == 0 || dv == 0) {
    start = c.reference + lower;
    return true;
  }
  if (dv > 0)
    lower = -(1 - 1e-12) / (c.drag * dv);
  else
    lower = (std::abs(dv) / c.wind - 1) / (c.drag * std::abs(dv));
  double height, speed;
  if (!trajectory(c, lower * (1 - 1e-12), height, speed) || height > innerRsun + 1e-8) return false;
  lower *= 1 - 1e-12;
  for (int i = 0; i < 100; ++i) {
    const double mid = .5 * (lower + upper);
    if (!trajectory(c, mid, height, speed) || height < innerRsun)
      lower = mid;
    else
      upper = mid;
  }
  start = c.reference + .5 * (lower + upper);
  return true;
}

struct ConeNow {
  double axis[3];
  double radius, shift, speed, density, temperature, gamma;
};

__device__ __forceinline__ void blockSum2(double& a, double& b, double* sh) {
  const int t = threadIdx.x;
  sh[t] = a;
  sh[kInsertThreads + t] = b;
  __syncthreads();
  for (int s = kInsertThreads / 2; s > 0; s >>= 1) {
    if (t < s) {
      sh[t] += sh[t + s];
      sh[kInsertThreads + t] += sh[kInsertThreads + t + s];
    }
    __syncthreads();
  }
  a = sh[0];
  b = sh[kInsertThreads];
}

template <bool STATS>
__global__ void __launch_bounds__(kInsertThreads) coneInsertKernel(const hc::DevLevel L, const ConeNow c,
                                                                   double* __restrict__ ju,
                                                                   double* __restrict__ partial) {
  const long n = 6L * L.Nv;
  const double dx0 = 1.0 / L.nr, dx1 = L.h;
  double count = 0, mass = 0;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
    const int b = (int)(t / L.Nv);
    const long r = t - (long)b * L.Nv;
    const int i = (int)(r % L.nr);
    const int j = (int)((r / L.nr) % L.na);
    const int k = (int)(r / ((long)L.nr * L.na));
    const hc::GravCell gc = L.grav[((size_t)b * L.na + k) * L.na + j];
    const double rc = L.rc[i + L.g];
    const double pos[3] = {rc * gc.x[0], rc * gc.x[1], rc * gc.x[2]};
    // sample(): inside the sphere about the current centre
    const double q0 = pos[0] - c.shift * c.axis[0], q1 = pos[1] - c.shift * c.axis[1],
                 q2 = pos[2] - c.shift * c.axis[2];
    if (sqrt(q0 * q0 + q1 * q1 + q2 * q2) > c.radius) continue;
    const double radius = sqrt(pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2]) / kSolarRadius;
    if (!(radius > 0)) continue;
    double v[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) v[d] = c.speed * 1e5 * pos[d] / (kSolarRadius * radius);
    // ambient Cartesian primitives
    const double J = L.radial[i + L.g].w * gc.det;
    double* cell = ju + (long)b * hc::NC * L.Nv + r;
    double u[8], old[8];
#pragma unroll
    for (int q = 0; q < hc::NC; ++q) u[q] = cell[q * L.Nv];
    hc::cartesianPrimitiveFromConserved(old, u, 1.0 / J, c.gamma);
    // increment() with plasmaWeight 1 and no cone field
    const double weight = 1;
    const double density = (1 - weight) * old[0] + weight * c.density;
    double oldKinetic = 0, newKinetic = 0, oldMagnetic = 0, newMagnetic = 0, delta[8];
    delta[0] = density - old[0];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      delta[1 + d] = density * v[d] - old[0] * old[1 + d];
      delta[5 + d] = 0.0;
      oldKinetic += .5 * old[0] * old[1 + d] * old[1 + d];
      newKinetic += .5 * density * v[d] * v[d];
      oldMagnetic += old[5 + d] * old[5 + d] / (8 * kPiCme);
      newMagnetic += (old[5 + d] + 0.0) * (old[5 + d] + 0.0) / (8 * kPiCme);
    }
    const double target = 2 * kBoltzmann * c.temperature * c.density / hc::kMP;
    const double pressure = (1 - weight) * fmax(0., old[4]) + weight * target;
    const double addedPressure = pressure - fmax(0., old[4]);
    delta[4] = addedPressure / (c.gamma - 1) + newKinetic - oldKinetic + newMagnetic - oldMagnetic;
#pragma unroll
    for (int q = 0; q < hc::NC; ++q) cell[q * L.Nv] = u[q] + J * delta[q];
    if (STATS) {
      count += 1;
      mass += delta[0] * (J * dx0 * dx1 * dx1);
    }
  }
  if (STATS) {
    __shared__ double sh[2 * kInsertThreads];
    blockSum2(count, mass, sh);
    if (threadIdx.x == 0) {
      partial[2 * blockIdx.x] = count;
      partial[2 * blockIdx.x + 1] = mass;
    }
  }
}

__global__ void __launch_bounds__(kInsertThreads) coneStatsKernel(const double* __restrict__ partial, int nblk,
                                                                  double* __restrict__ stats) {
  double count = 0, mass = 0;
  for (int t = threadIdx.x; t < nblk; t += kInsertThreads) {
    count += partial[2 * t];
    mass += partial[2 * t + 1];
  }
  __shared__ double sh[2 * kInsertThreads];
  blockSum2(count, mass, sh);
  if (threadIdx.x == 0) {
    stats[0] = count;
    stats[1] = mass;
  }
}

int cudaFailed(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return HC_OK;
  char msg[256];
  std::snprintf(msg, sizeof msg, "hc_level_insert_cone: %s: %s", what, cudaGetErrorString(e));
  return hc::setLastError(HC_ERR_CUDA, msg);
}

}  // namespace

extern "C" int hc_cone_prepare(const hc_cone_spec* spec, double inner_radius, hc_cone* out) {
  using hc::setLastError;
  if (!spec || !out) return setLastError(HC_ERR_ARG, "hc_cone_prepare: null argument");
  const hc_cone_spec& s = *spec;
  if (!(inner_radius > 0)) return setLastError(HC_ERR_ARG, "hc_cone_prepare: inner radius must be positive");
  if (!(s.apex_speed > 0)) return setLastError(HC_ERR_ARG, "hc_cone_prepare: apex speed must be positive");
  if (!(s.drag_gamma >= 0)) return setLastError(HC_ERR_ARG, "hc_cone_prepare: drag coefficient must be >= 0");
  if (s.drag_gamma > 0 && !(s.wind_speed > 0))
    return setLastError(HC_ERR_ARG, "hc_cone_prepare: the drag-based model needs a positive wind speed");
  if (!(s.half_angle_deg > 0 && s.half_angle_deg < 90))
    return setLastError(HC_ERR_ARG, "hc_cone_prepare: half angle must lie in (0, 90) degrees");
  if (!(s.density > 0) || !(s.temperature >= 0))
    return setLastError(HC_ERR_ARG, "hc_cone_prepare: density must be positive and temperature >= 0");
  const double innerRsun = inner_radius / kSolarRadius;
  const Trajectory c{s.apex_speed, s.wind_speed, s.drag_gamma, s.reference_height, s.reference_time};
  double entry, height, speed;
  if (!boundaryStart(c, innerRsun, entry))
    return setLastError(HC_ERR_ARG,
                        "hc_cone_prepare: the drag-based model cannot be extrapolated outward from the inner "
                        "boundary to this cone");
  if (!trajectory(c, entry - c.reference, height, speed))
    return setLastError(HC_ERR_ARG, "hc_cone_prepare: cannot propagate the cone to its first boundary contact");
  hc_cone o;
  std::memset(&o, 0, sizeof o);
  const double inner = innerRsun * kSolarRadius;
  const double lat = s.lat_deg * kPiCme / 180, lon = s.lon_deg * kPiCme / 180;
  const double alpha = s.half_angle_deg * kPiCme / 180;
  o.axis[0] = std::cos(lon) * std::cos(lat);
  o.axis[1] = std::sin(lon) * std::cos(lat);
  o.axis[2] = std::sin(lat);
  o.radius = inner * std::sin(alpha);
  o.entry_time = entry;
  o.speed = speed;
  o.entry_shift = inner - o.radius;
  const double referenceShift = (s.reference_height + 0.0) * kSolarRadius - o.radius;
  o.end_time = entry + 2 * o.radius / (speed * 1e5);
  o.insertion_time = entry + (referenceShift - o.entry_shift) / (speed * 1e5);
  o.density = s.density;
  o.temperature = s.temperature;
  *out = o;
  return HC_OK;
}

extern "C" int hc_level_insert_cone(hc_ctx* ctx, const hc_cone* cone, double time, double* ju, double* stats,
                                    void* stream) {
  using namespace hc;
  if (!ctx || !cone || !ju) return setLastError(HC_ERR_ARG, "hc_level_insert_cone: null argument");
  const hc_cone& k = *cone;
  if (!(k.radius > 0) || !(k.density > 0) || !(k.temperature >= 0) || !(k.speed > 0))
    return setLastError(HC_ERR_ARG, "hc_level_insert_cone: cone not prepared (radius, density, speed)");
  const double an = std::sqrt(k.axis[0] * k.axis[0] + k.axis[1] * k.axis[1] + k.axis[2] * k.axis[2]);
  if (!(std::abs(an - 1) < 1e-12)) return setLastError(HC_ERR_ARG, "hc_level_insert_cone: axis must be a unit vector");
  const DevLevel& L = *ctxLevel(ctx);
  ConeNow c;
  for (int d = 0; d < 3; ++d) c.axis[d] = k.axis[d];
  c.radius = k.radius;
  c.shift = k.entry_shift + k.speed * 1e5 * (time - k.entry_time);
  c.speed = k.speed;
  c.density = k.density;
  c.temperature = k.temperature;
  c.gamma = L.gamma;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const long n = 6L * L.Nv;
  const long want = (n + kInsertThreads - 1) / kInsertThreads;
  const int nblk = (int)(want < kInsertMaxBlocks ? want : kInsertMaxBlocks);
  if (!stats) {
    coneInsertKernel<false><<<nblk, kInsertThreads, 0, s>>>(L, c, ju, nullptr);
    return cudaFailed(cudaGetLastError(), "insert");
  }
  double* partial = nullptr;
  int rc = cudaFailed(cudaMallocAsync(reinterpret_cast<void**>(&partial), sizeof(double) * 2 * nblk, s), "partials");
  if (rc != HC_OK) return rc;
  coneInsertKernel<true><<<nblk, kInsertThreads, 0, s>>>(L, c, ju, partial);
  rc = cudaFailed(cudaGetLastError(), "insert");
  if (rc == HC_OK) {
    coneStatsKernel<<<1, kInsertThreads, 0, s>>>(partial, nblk, stats);
    rc = cudaFailed(cudaGetLastError(), "statistics");
  }
  const int rf = cudaFailed(cudaFreeAsync(partial, s), "free partials");
  return rc != HC_OK ? rc : rf;
}

// ORACLE PIN -- test infrastructure only.
//
// Exposes the reference's own pointwise solvers, compiled from the reference
// sources where they lie (the build recipe passes -I <reference>/src and a
// generated two-line Proto_Accel.H that defines ACCEL_DECORATION as empty).
// These three headers need nothing from the unvendored Proto library:
//   src/MHD_Roe8Wave.H        roe8WaveDissipation, rusanovDissipation,
//                             mappedRoe8WaveDissipation, factoredRoe8WaveDissipation
//   src/MHD_Reconstruction.H  complete-state guards
//   src/MHD_SecondOrderFlux.H secondOrderFrame, secondOrderFaceFlux
// and the cone-CME model, which needs only the standard library:
//   src/MHD_CME.H             prepareConeCloud, expandedSource, sample,
//                             loadDensity, increment (with MHD_ImportedCME.H
//                             analyticCone, MHD_Time.H, MHD_JSON.H)
// The output library oracle/_ref/libhcref.so is git-ignored and is used by
// tests/test_oracle_pin.py to pin the oracle restatement.

#include <cmath>
#include <cstddef>
using std::max;
using std::min;

#include "MHD_Roe8Wave.H"
#include "MHD_Reconstruction.H"
#include "MHD_SecondOrderFlux.H"
#include "MHD_CME.H"

namespace {
struct Arr8 {
  double* p;
  double& operator()(int c) const { return p[c]; }
};
struct CArr8 {
  const double* p;
  const double& operator()(int c) const { return p[c]; }
};
}  // namespace

extern "C" {

int ref_roe8(const double* wl, const double* wr, double gamma, double ef, int check, double* out) {
  return MHD_Riemann_Solvers::roe8WaveDissipation(out, wl, wr, gamma, ef, check != 0) ? 1 : 0;
}

void ref_rusanov(const double* wl, const double* wr, double gamma, double* out) {
  MHD_Riemann_Solvers::rusanovDissipation(out, wl, wr, gamma);
}

void ref_frame(const double* normal, double* frame9, double* norm) {
  HelioCubed::SecondOrderFrame f = HelioCubed::secondOrderFrame(normal);
  for (int r = 0; r < 3; ++r)
    for (int s = 0; s < 3; ++s) frame9[3 * r + s] = f.frame[r][s];
  *norm = f.norm;
}

void ref_face_flux(const double* l, const double* r, const double* normal, double radialArea,
                   double gamma, double ef, int roe, double* out) {
  HelioCubed::SecondOrderFrame f = HelioCubed::secondOrderFrame(normal);
  Arr8 o{out};
  CArr8 L{l}, R{r};
  HelioCubed::secondOrderFaceFlux(o, L, R, f, radialArea, gamma, ef, roe != 0);
}

void ref_mapped_roe(const double* wl, const double* wr, const double* A9, double radialArea, int dir,
                    double gamma, double ef, double floor, double* out) {
  double A[3][3];
  for (int r = 0; r < 3; ++r)
    for (int s = 0; s < 3; ++s) A[r][s] = A9[3 * r + s];
  MHD_Riemann_Solvers::mappedRoe8WaveDissipation(out, wl, wr, A, radialArea, dir, gamma, ef, floor);
}

void ref_factored_roe(const double* wl, const double* wr, const double* A9, double radialArea, int dir,
                      double gamma, double ef, double floor, double* out) {
  double A[3][3];
  for (int r = 0; r < 3; ++r)
    for (int s = 0; s < 3; ++s) A[r][s] = A9[3 * r + s];
  MHD_Riemann_Solvers::factoredRoe8WaveDissipation(out, wl, wr, A, radialArea, dir, gamma, ef, floor);
}

int ref_usable_primitive(const double* w, double floor) {
  CArr8 s{w};
  return MHD_Reconstruction::usablePrimitiveState<8>(s, floor) ? 1 : 0;
}

namespace {
// spec: lat, lon, half angle (deg), apex speed, wind speed (km/s), drag
// (1/km), reference height (Rsun), reference time (s), density, temperature.
CMEParameters coneSource(const double* spec) {
  CMEParameters c;
  c.fieldModel = 4;
  c.lat = spec[0];
  c.lon = spec[1];
  c.halfangle = spec[2];
  c.apex_speed = spec[3];
  c.windSpeed = spec[4];
  c.dragGamma = spec[5];
  c.r1 = spec[6];
  c.r0 = 0;
  c.referenceTime = spec[7];
  c.insertionTime = spec[7];
  c.density = spec[8];
  c.temperature = spec[9];
  c.imported = ImportedCME::Model::analyticCone(spec[6], spec[2], spec[0], spec[1], CalendarEpoch{2024, 0.0L});
  return c;
}
}  // namespace

// prepareConeCloud; out: axis[3], radius, entry shift, entry time, speed,
// end time, insertion time.  Returns -1 where the reference throws.
int ref_cone_prepare(const double* spec, double innerRsun, double* out) {
  CMEParameters c = coneSource(spec);
  try {
    CMEModel::prepareConeCloud(c, innerRsun);
  } catch (const std::exception&) {
    return -1;
  }
  for (int d = 0; d < 3; ++d) out[d] = c.cloudAxis[d];
  out[3] = c.cloudSphereRadius;
  out[4] = c.cloudEntryShift;
  out[5] = c.cloudEntryTime;
  out[6] = c.cloudSpeed;
  out[7] = c.cloudEndTime;
  out[8] = c.insertionTime;
  return 0;
}

// The cone branch of Insert_CME for one cell: expandedSource at `time`,
// sample at `pos`, loadDensity and increment on the Cartesian primitive
// ambient state.  Returns 1 and delta[8] inside the cloud.
int ref_cone_cell(const double* spec, double innerRsun, double time, const double* pos, const double* ambient,
                  double gamma, double* delta) {
  CMEParameters c = coneSource(spec);
  try {
    CMEModel::prepareConeCloud(c, innerRsun);
  } catch (const std::exception&) {
    return -1;
  }
  CMEParameters current;
  if (!CMEModel::expandedSource(c, time, current)) return 0;
  CMEModel::Sample source;
  if (!CMEModel::sample(current, {pos[0], pos[1], pos[2]}, source)) return 0;
  std::array<double, 8> a;
  for (int q = 0; q < 8; ++q) a[q] = ambient[q];
  CMEModel::loadDensity(source, a);
  const auto change = CMEModel::increment(a, source, gamma, current.plasmaBeta);
  for (int q = 0; q < 8; ++q) delta[q] = change[q];
  return 1;
}

// CMEInsertionSchedule of finite cone sources (field model 4) inserted at
// times[i] whose clouds end at cloud_end[i]; the first `inserted` are marked
// inserted.  out: cfl(time, target, feeding), rusanovEndTime().
void ref_cme_schedule(const double* times, const double* cloud_end, int n, int inserted, double time, double target,
                      double feeding, double* out) {
  std::vector<CMEParameters> sources(n);
  for (int i = 0; i < n; ++i) {
    sources[i].fieldModel = 4;
    sources[i].injectionMethod = 0;
    sources[i].insertionTime = times[i];
    sources[i].cloudEndTime = cloud_end[i];
  }
  CMEInsertionSchedule sched(sources);
  for (int i = 0; i < inserted; ++i) sched.markInserted();
  out[0] = sched.cfl(time, target, feeding);
  out[1] = sched.rusanovEndTime();
}
}

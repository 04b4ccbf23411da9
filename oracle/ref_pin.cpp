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
// The output library oracle/_ref/libhcref.so is git-ignored and is used by
// tests/test_oracle_pin.py to pin the oracle restatement.

#include <cmath>
#include <cstddef>
using std::max;
using std::min;

#include "MHD_Roe8Wave.H"
#include "MHD_Reconstruction.H"
#include "MHD_SecondOrderFlux.H"

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
}

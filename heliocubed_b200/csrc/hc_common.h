// Constants and plain structures shared by host code and kernels.
#pragma once

namespace hc {


constexpr int NC = 8;
// src/BoxOp_EulerCubedSphere.H:36 and src/MHD_Constants.H:4-7
constexpr double kMP = 1.67262192e-24;
constexpr double kSolarRadiusCm = 69600000000.0;  // c_SR, src/MHD_Constants.H:4
constexpr double kRHO00 = 1.67262192e-24 / 100.;
constexpr double kGrav = 6.67430e-8;
constexpr double kMsun = 1.98847e33;
constexpr double kPi = 3.14159265358979323846;

// Face geometry of one angular face: unit-normal frame (rows: normal and
// two tangents, src/MHD_SecondOrderFlux.H:11-30), |adjA| and raw adjA.
struct FaceGeom {
  double f[9];
  double norm;
  double n[3];
  double pad[3];
};

}  // namespace hc

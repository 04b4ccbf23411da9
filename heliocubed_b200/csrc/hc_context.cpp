// Host side of the C ABI (include/hc_abi.h): option validation, level
// geometry (the caches the reference keeps in levelGeometry statics and in
// its per-patch face / CFL / gravity caches), workspace, and launch sequences.
//
// Metrics are the exact cell/face averages of the equiangular gnomonic map,
// integrated here with 8-point Gauss-Legendre quadrature in double (the
// reference obtains them from Proto's unvendored CubedSphereShell).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/hc_abi.h"
#include "hc_level.h"

using namespace hc;

namespace {

thread_local std::string g_lastError;

int fail(int code, const std::string& msg) {
  g_lastError = msg;
  return code;
}
int cudaFail(cudaError_t e, const char* where) {
  return fail(HC_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

// src/BoxOp_Utilities.H:413-416, read as: global component k of a panel-local
// vector q is SIGN[b][k] * q[PERM[b][k]].
const int PERM[6][3] = {{1, 2, 0}, {1, 2, 0}, {1, 0, 2}, {0, 1, 2}, {1, 0, 2}, {0, 1, 2}};
const int SIGN[6][3] = {{1, -1, -1}, {1, 1, 1}, {1, -1, 1}, {1, 1, 1}, {-1, 1, 1}, {-1, -1, 1}};
const double PI = 3.14159265358979323846;

struct Vec3 { double x[3]; };

// Basis A = (Xhat, dXhat/dxi1, dXhat/dxi2) at panel coordinates (x1, x2).
void basisAt(int b, double x1, double x2, double A[3][3], double X[3]) {
  const double ta = std::tan(-PI / 4 + PI / 2 * x1), tb = std::tan(-PI / 4 + PI / 2 * x2);
  const double rho2 = 1 + ta * ta + tb * tb, rho = std::sqrt(rho2), r3 = rho * rho2;
  const double q[3] = {1 / rho, ta / rho, tb / rho};
  const double da = PI / 2 * (1 + ta * ta), db = PI / 2 * (1 + tb * tb);
  const double q1[3] = {-ta / r3 * da, (1 / rho - ta * ta / r3) * da, -ta * tb / r3 * da};
  const double q2[3] = {-tb / r3 * db, -ta * tb / r3 * db, (1 / rho - tb * tb / r3) * db};
  for (int k = 0; k < 3; ++k) {
    const int p = PERM[b][k];
    A[k][0] = SIGN[b][k] * q[p];
    A[k][1] = SIGN[b][k] * q1[p];
    A[k][2] = SIGN[b][k] * q2[p];
    if (X) X[k] = A[k][0];
  }
}

void cross(const double u[3], const double v[3], double w[3]) {
  w[0] = u[1] * v[2] - u[2] * v[1];
  w[1] = u[2] * v[0] - u[0] * v[2];
  w[2] = u[0] * v[1] - u[1] * v[0];
}

struct Gauss {
  double x[8], w[8];
  Gauss() {
    const int n = 8;
    for (int i = 0; i < n; ++i) {
      double z = std::cos(PI * (i + 0.75) / (n + 0.5)), pp = 1;
      for (int it = 0; it < 60; ++it) {
        double p1 = 1, p2 = 0;
        for (int j = 1; j <= n; ++j) {
          const double p3 = p2;
          p2 = p1;
          p1 = ((2 * j - 1) * z * p2 - (j - 1) * p3) / j;
        }
        pp = n * (z * p1 - p2) / (z * z - 1);
        const double dz = p1 / pp;
        z -= dz;
        if (std::fabs(dz) < 1e-17) break;
      }
      x[i] = 0.5 * (1 - z);
      w[i] = 1 / ((1 - z * z) * pp * pp);
    }
  }
};

// Cofactor row d of A (normal of a constant-xi_d face), times det when
// d = 0 this is det(A) Xhat.
void cofactorRow(const double A[3][3], int d, double n[3]) {
  const int t1 = (d + 1) % 3, t2 = (d + 2) % 3;
  const double a[3] = {A[0][t1], A[1][t1], A[2][t1]}, c[3] = {A[0][t2], A[1][t2], A[2][t2]};
  cross(a, c, n);
}

double det3(const double A[3][3]) {
  return A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) - A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
         A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
}

void inv3(const double A[3][3], double I[3][3]) {
  const double c00 = A[1][1] * A[2][2] - A[1][2] * A[2][1];
  const double c01 = A[1][2] * A[2][0] - A[1][0] * A[2][2];
  const double c02 = A[1][0] * A[2][1] - A[1][1] * A[2][0];
  const double id = 1.0 / (A[0][0] * c00 + A[0][1] * c01 + A[0][2] * c02);
  I[0][0] = c00 * id;
  I[1][0] = c01 * id;
  I[2][0] = c02 * id;
  I[0][1] = (A[0][2] * A[2][1] - A[0][1] * A[2][2]) * id;
  I[1][1] = (A[0][0] * A[2][2] - A[0][2] * A[2][0]) * id;
  I[2][1] = (A[0][1] * A[2][0] - A[0][0] * A[2][1]) * id;
  I[0][2] = (A[0][1] * A[1][2] - A[0][2] * A[1][1]) * id;
  I[1][2] = (A[0][2] * A[1][0] - A[0][0] * A[1][2]) * id;
  I[2][2] = (A[0][0] * A[1][1] - A[0][1] * A[1][0]) * id;
}

// Components that vanish or coincide in magnitude by the cube's symmetry are
// set to exactly those values: quadrature round-off must not decide the
// least-aligned-axis choice of secondOrderFrame (a strict comparison), on
// which the Roe entropy fix (|V|+|W| in the face frame) depends.
void snapNormal(double n[3]) {
  const double mag = std::max(std::fabs(n[0]), std::max(std::fabs(n[1]), std::fabs(n[2])));
  const double tol = 1e-13 * mag;
  for (int i = 0; i < 3; ++i)
    if (std::fabs(n[i]) < tol) n[i] = 0.0;
  for (int a = 0; a < 3; ++a)
    for (int b = a + 1; b < 3; ++b)
      if (n[a] != 0.0 && std::fabs(std::fabs(n[a]) - std::fabs(n[b])) <= tol) {
        const double m = 0.5 * (std::fabs(n[a]) + std::fabs(n[b]));
        n[a] = std::copysign(m, n[a]);
        n[b] = std::copysign(m, n[b]);
      }
}

// src/MHD_SecondOrderFlux.H:11-30
FaceGeom makeFrame(const double normal[3]) {
  FaceGeom r{};
  double f[3][3] = {};
  double norm = 0;
  for (int i = 0; i < 3; ++i) norm += normal[i] * normal[i];
  norm = std::sqrt(norm);
  for (int i = 0; i < 3; ++i) f[0][i] = normal[i] / norm;
  int axis = 0;
  for (int i = 1; i < 3; ++i)
    if (std::fabs(f[0][i]) < std::fabs(f[0][axis])) axis = i;
  f[1][(axis + 1) % 3] = f[0][(axis + 2) % 3];
  f[1][(axis + 2) % 3] = -f[0][(axis + 1) % 3];
  double t = 0;
  for (int i = 0; i < 3; ++i) t += f[1][i] * f[1][i];
  for (int i = 0; i < 3; ++i) f[1][i] /= std::sqrt(t);
  for (int i = 0; i < 3; ++i) {
    const int j = (i + 1) % 3, k = (i + 2) % 3;
    f[2][i] = f[0][j] * f[1][k] - f[0][k] * f[1][j];
  }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.f[3 * i + j] = f[i][j];
  r.norm = norm;
  for (int d = 0; d < 3; ++d) r.n[d] = normal[d];
  return r;
}

// Radial cells of the whole shell (a slab level holds part of them).
int shellCells(const hc_params& P) { return P.radial_cells > 0 ? P.radial_cells : P.nr; }
bool isSlab(const hc_params& P) { return P.nr < shellCells(P); }

// Radial metrics, src/BoxOp_Utilities.H:36-59, of the level's radial cell
// iLocal (the shell's cell iLocal + radial_offset).
struct RadialRow { double rlow, rhigh, rhalf, vol, Dr0, area0, areaT; };
RadialRow radialRow(const hc_params& P, int iLocal) {
  const int i = iLocal + P.radial_offset;
  const double r0 = P.inner_radius, r1 = P.outer_radius, C = P.radial_stretch, dxi0 = 1.0 / shellCells(P);
  const double R_t = C == 0.0 ? (r1 - r0) : (r1 - r0) / std::expm1(C);
  const double etalow = i * dxi0;
  const double rlow = r0 + R_t * (C == 0.0 ? etalow : std::expm1(C * etalow));
  const double etahigh = (i + 1.0) * dxi0;
  const double rhigh = r0 + R_t * (C == 0.0 ? etahigh : std::expm1(C * etahigh));
  const double eta_half = (etalow + etahigh) / 2.0;
  const double rhalf = r0 + R_t * (C == 0.0 ? eta_half : std::expm1(C * eta_half));
  RadialRow r;
  r.rlow = rlow;
  r.rhigh = rhigh;
  r.rhalf = rhalf;
  r.vol = (rhigh * rhigh * rhigh - rlow * rlow * rlow) / 3.0 / dxi0;
  r.Dr0 = (rhigh - rlow) / dxi0;
  r.area0 = rlow * rlow;
  r.areaT = (rhigh * rhigh - rlow * rlow) / dxi0 / 2.0;
  return r;
}

// Inner analytic wind in the native basis, src/BoxOp_PreStage.H:7-47 at t=0
// (the time-independent case strength = 0 is tabulated on the host).
void windNative(const hc_params& P, const double X[3], double u[8]) {
  const double gam = P.gamma, r_BC = P.inner_radius;
  const double r = std::sqrt(X[0] * X[0] + X[1] * X[1] + X[2] * X[2]);
  const double p0 = 1.0e-7, rho0 = 700 * kMP, u0 = 500.0 * 1e5;
  const double rho = rho0 * std::pow(r_BC / r, 2.0);
  const double p = p0 * std::pow(r_BC / r, 2.0 * gam);
  const double ur = u0 - P.strength / 100.0 * u0 / 3 * 0.0;
  u[0] = rho;
  u[1] = ur * rho;
  u[2] = u[3] = u[5] = u[6] = u[7] = 0.0;
  const double umag = std::sqrt(u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / u[0];
  const double Bmag = 0.0;
  u[4] = p / (gam - 1.0) + 0.5 * u[0] * umag * umag + Bmag * Bmag / 8.0 / PI;
}

// Panel containing direction X and its panel coordinates.
void locate(const double X[3], int& pb) {
  pb = 0;
  double best = -2;
  for (int b = 0; b < 6; ++b) {
    double q0 = 0;
    for (int k = 0; k < 3; ++k)
      if (PERM[b][k] == 0) q0 = SIGN[b][k] * X[k];
    if (q0 > best) { best = q0; pb = b; }
  }
}
void panelCoords(int b, const double X[3], double& x1, double& x2) {
  double q[3];
  for (int k = 0; k < 3; ++k) q[PERM[b][k]] = SIGN[b][k] * X[k];
  x1 = (std::atan2(q[1], q[0]) + PI / 4) / (PI / 2);
  x2 = (std::atan2(q[2], q[0]) + PI / 4) / (PI / 2);
}

template <class T>
T* upload(const std::vector<T>& v, std::vector<void*>& owned, cudaError_t& err) {
  void* p = nullptr;
  if (err != cudaSuccess) return nullptr;
  err = cudaMalloc(&p, std::max<size_t>(1, v.size() * sizeof(T)));
  if (err != cudaSuccess) return nullptr;
  owned.push_back(p);
  if (!v.empty()) err = cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
  return static_cast<T*>(p);
}

}  // namespace

struct hc_ctx {
  hc_params P;
  int device = 0;
  DevLevel L{};
  std::vector<void*> owned;
  // host copies for hc_geometry_export
  std::vector<double> radialExport, detExport, detAAExport, normalExport[3];
  // stage workspace: stage s reads W[s % 2] and writes the next stage's
  // primitives into W[(s + 1) % 2]
  double* W[2] = {nullptr, nullptr};  // ghosted primitives [6][8][na+4][na+4][nr+4]
  double* acc = nullptr;              // RK accumulator [6][8][na][na][nr]
  unsigned long long* invMax = nullptr;  // two CFL slots (bit patterns), ping-pong per step
  int* flag = nullptr;
  // cell tiles of the order-2 stage kernel: fused RK stage, operator alone
  int tileRK = 0, tileRHS = 0;
  // register-cap variants of the fourth-order operator's tuned kernels
  int o4var[kO4TunedKernels] = {0, 0, 0};
  // CME insertion schedule (device) and the Rusanov-window flag it sets
  CmeSchedule* sched = nullptr;
  CmeSchedule schedHost{};
  int* rusanovFlag = nullptr;
  int schedEvents = 0;
  InletCone* inletDev = nullptr;  // cones fed through the inner boundary (device, kInletCones)
  bool tuned = false;
  // fourth-order operator: metric tables and grow-only scratch
  O4Geo o4{};
  double* o4scratch = nullptr;
  size_t o4scratchDoubles = 0;
  // fourth-order level step: tables and level-sized buffers (order 4 only)
  O4Level o4l{};
  double* o4us = nullptr;      // native averages on the ghosted panels [6][8][Ng]
  double* o4cart = nullptr;    // Cartesian averages with seam ghosts [6][8][Nc]
  double* o4next = nullptr;    // next stage state [6][8][Nv]
  double* o4k = nullptr;       // stage right-hand side [6][8][Nv]
  double* o4reg = nullptr;     // seam flux register [6][2][2][8][na][nr]
  double* o4lvlScratch = nullptr;
  double* o4pv = nullptr;      // seam interpolation point values [6][8][npts][nr]
  O4Batch* o4levelBatch = nullptr;  // the six panels on o4us -> o4k
  int winLo = 0, winHi = 0;          // radial window of the level step's operator (winHi 0: all cells)
  // operator batches of recent argument sets (hc_box_rhs_o4, hc_level_rhs on
  // caller arrays), oldest first
  std::vector<std::pair<std::string, O4Batch*>> o4cache;
};

// Several fourth-order levels stepped together: each level prepares its
// own stages, takes its own CFL step, updates and reconciles its own seams;
// the operator runs as one batch over all levels' panels, so every operator
// kernel is one launch for the whole ensemble.
struct hc_ensemble {
  std::vector<hc_ctx*> members;
  O4Batch* batch = nullptr;
  int gravity = 0;
  int device = 0;
  // member q's own kernels (CFL, schedule, preparation, update, seam
  // reconciliation, time) run on lane q % lanes.size(), forked from and
  // joined to the caller's stream around the batched operator
  std::vector<cudaStream_t> lanes;
  cudaEvent_t forkEv = nullptr;
  std::vector<cudaEvent_t> joinEv;
};

namespace {

int buildLevel(hc_ctx* c) {
  const hc_params& P = c->P;
  const int nr = P.nr, na = P.na, g = kGhost;
  const double h = 1.0 / na;
  Gauss G;
  DevLevel& L = c->L;
  L.nr = nr; L.na = na; L.g = g;
  L.n0 = nr + 2 * g; L.n1 = na + 2 * g;
  L.Nv = (long)nr * na * na;
  L.Ng = (long)L.n0 * L.n1 * L.n1;
  L.h = h; L.dxi0 = 1.0 / shellCells(P);
  L.gamma = P.gamma; L.invGm1 = 1.0 / (P.gamma - 1.0); L.entropy = P.entropy_fix_coeff; L.cfl_number = P.cfl; L.strength = P.strength;
  L.r0 = P.inner_radius; L.innerBCType = P.init_condition_type;

  // radial rows i = -g .. nr+g
  std::vector<double4> radial(nr + 2 * g + 1);
  std::vector<double> rc(nr + 2 * g + 1);
  c->radialExport.assign((size_t)(nr + 1) * 4, 0.0);
  for (int i = -g; i <= nr + g; ++i) {
    const RadialRow r = radialRow(P, i);
    radial[i + g] = make_double4(r.area0, r.areaT, r.Dr0, r.vol);
    rc[i + g] = r.rhalf;
    if (i >= 0 && i <= nr) {
      double* e = &c->radialExport[4 * i];
      e[0] = r.area0; e[1] = r.areaT; e[2] = r.Dr0; e[3] = r.vol;
    }
  }
  for (int m = 0; m < g; ++m) {
    const double rl = radialRow(P, nr - 1).rhalf, rr = radialRow(P, nr + m).rhalf;
    L.outerScale2[m] = std::pow(rl / rr, 2.0);
    L.outerScale1[m] = std::pow(rl / rr, 1.0);
  }

  const size_t nf = (size_t)(na + 1) * (na + 1);
  std::vector<FaceGeom> faces(3 * 6 * nf);
  std::vector<GravCell> grav((size_t)6 * na * na);
  std::vector<double> basis((size_t)6 * na * na * 9), basisInv((size_t)6 * na * na * 9);
  std::vector<CflCell> cfl((size_t)6 * na * na);
  for (int d = 0; d < 3; ++d) c->normalExport[d].clear();
  c->detExport.assign((size_t)6 * na * na, 0.0);
  c->detAAExport.assign((size_t)6 * na * na * 9, 0.0);

  for (int b = 0; b < 6; ++b) {
    // Face normals: average over the face of the cofactor row.
    for (int k = 0; k <= na; ++k)
      for (int j = 0; j <= na; ++j)
        for (int d = 0; d < 3; ++d) {
          if ((d != 1 && j == na) || (d != 2 && k == na)) continue;
          double n[3] = {0, 0, 0};
          if (d == 0) {
            for (int p = 0; p < 8; ++p)
              for (int q = 0; q < 8; ++q) {
                double A[3][3], m[3];
                basisAt(b, (j + G.x[p]) * h, (k + G.x[q]) * h, A, nullptr);
                cofactorRow(A, 0, m);
                for (int r = 0; r < 3; ++r) n[r] += G.w[p] * G.w[q] * m[r];
              }
          } else {
            for (int p = 0; p < 8; ++p) {
              double A[3][3], m[3];
              if (d == 1) basisAt(b, j * h, (k + G.x[p]) * h, A, nullptr);
              else basisAt(b, (j + G.x[p]) * h, k * h, A, nullptr);
              cofactorRow(A, d, m);
              for (int r = 0; r < 3; ++r) n[r] += G.w[p] * m[r];
            }
          }
          snapNormal(n);
          faces[((size_t)d * 6 + b) * nf + (size_t)k * (na + 1) + j] = makeFrame(n);
        }
    for (int k = 0; k < na; ++k)
      for (int j = 0; j < na; ++j) {
        const size_t ci = ((size_t)b * na + k) * na + j;
        double det = 0, dA[3][3] = {{0}};
        for (int p = 0; p < 8; ++p)
          for (int q = 0; q < 8; ++q) {
            double A[3][3];
            basisAt(b, (j + G.x[p]) * h, (k + G.x[q]) * h, A, nullptr);
            const double dt = det3(A), wt = G.w[p] * G.w[q];
            det += wt * dt;
            for (int r = 0; r < 3; ++r)
              for (int s = 0; s < 3; ++s) dA[r][s] += wt * dt * A[r][s];
          }
        double Ac[3][3], X[3], Ai[3][3];
        basisAt(b, (j + 0.5) * h, (k + 0.5) * h, Ac, X);
        inv3(Ac, Ai);
        GravCell& gc = grav[ci];
        for (int r = 0; r < 3; ++r) { gc.x[r] = X[r]; gc.a0[r] = dA[r][0]; }
        gc.det = det;
        gc.pad = 0;
        for (int r = 0; r < 3; ++r)
          for (int s = 0; s < 3; ++s) {
            basis[ci * 9 + 3 * r + s] = Ac[r][s];
            basisInv[ci * 9 + 3 * r + s] = Ai[r][s];
            c->detAAExport[ci * 9 + 3 * r + s] = dA[r][s];
          }
        c->detExport[ci] = det;
        // CFL cache (src/BoxOp_SecondOrderCFL.H:46-77)
        CflCell& cc = cfl[ci];
        cc.inverseDet = 1.0 / det;
        double dAi[3][3];
        inv3(dA, dAi);
        for (int r = 0; r < 3; ++r)
          for (int s = 0; s < 3; ++s) {
            cc.inverseDetA[3 * r + s] = dAi[r][s];
            cc.cell[3 * r + s] = Ac[r][s];
          }
        for (int d = 0; d < 3; ++d) {
          const FaceGeom& f = faces[((size_t)d * 6 + b) * nf + (size_t)k * (na + 1) + j];
          double n2 = 0;
          for (int q = 0; q < 3; ++q) n2 += f.n[q] * f.n[q];
          cc.normal[d] = std::sqrt(n2);
          if (d == 0) { cc.det[0] = det; continue; }
          double fd = 0;
          for (int p = 0; p < 8; ++p) {
            double A[3][3];
            if (d == 1) basisAt(b, j * h, (k + G.x[p]) * h, A, nullptr);
            else basisAt(b, (j + G.x[p]) * h, k * h, A, nullptr);
            fd += G.w[p] * det3(A);
          }
          cc.det[d] = fd;
          double F[3][3];
          if (d == 1) basisAt(b, j * h, (k + 0.5) * h, F, nullptr);
          else basisAt(b, (j + 0.5) * h, k * h, F, nullptr);
          for (int r = 0; r < 3; ++r)
            for (int s = 0; s < 3; ++s) cc.face[d - 1][3 * r + s] = F[r][s];
        }
        cc.pad[0] = cc.pad[1] = 0;
      }
  }
  for (int d = 0; d < 3; ++d) {
    const int ej = d == 1 ? 1 : 0, ek = d == 2 ? 1 : 0;
    for (int b = 0; b < 6; ++b)
      for (int k = 0; k < na + ek; ++k)
        for (int j = 0; j < na + ej; ++j) {
          const FaceGeom& f = faces[((size_t)d * 6 + b) * nf + (size_t)k * (na + 1) + j];
          for (int r = 0; r < 3; ++r) c->normalExport[d].push_back(f.n[r]);
        }
  }

  // Seam plan: for each panel edge, the adjacent panel, its normal axis and
  // side; ghost donors (4-point Lagrange along the adjacent edge, stencil
  // kept inside the donor panel) and the seam-face index map.
  std::vector<SeamDonor> seam((size_t)6 * 2 * 2 * g * na);
  std::vector<int> faceMap((size_t)6 * 2 * 2 * na);
  std::vector<EdgeLink> edges(6 * 2 * 2);
  for (int b = 0; b < 6; ++b)
    for (int ax = 1; ax <= 2; ++ax)
      for (int side = 0; side < 2; ++side) {
        const int e = (b * 2 + (ax - 1)) * 2 + side;
        auto ghostX = [&](int m, double t, double X[3]) {
          const double nrm = side == 0 ? -(m + 0.5) * h : 1 + (m + 0.5) * h;
          double A[3][3];
          if (ax == 1) basisAt(b, nrm, t, A, X);
          else basisAt(b, t, nrm, A, X);
        };
        double X[3], y1, y2;
        ghostX(0, 0.5, X);
        int nb;
        locate(X, nb);
        panelCoords(nb, X, y1, y2);
        const int nax = std::min(y1, 1 - y1) < std::min(y2, 1 - y2) ? 1 : 2;
        const int nside = (nax == 1 ? y1 : y2) < 0.5 ? 0 : 1;
        edges[e] = EdgeLink{nb, nax, nside, 0};
        for (int m = 0; m < g; ++m)
          for (int s = 0; s < na; ++s) {
            ghostX(m, (s + 0.5) * h, X);
            panelCoords(nb, X, y1, y2);
            const double u = (nax == 1 ? y2 : y1) / h - 0.5;
            int base = (int)std::floor(u) - 1;
            base = std::max(0, std::min(na - 4, base));
            const int layer = nside == 0 ? m : na - 1 - m;
            SeamDonor dn{};
            dn.b = nb;
            for (int q = 0; q < 4; ++q) {
              double wq = 1;
              for (int r = 0; r < 4; ++r)
                if (r != q) wq *= (u - (base + r)) / (double)(q - r);
              dn.w[q] = wq;
              dn.j[q] = nax == 1 ? layer : base + q;
              dn.k[q] = nax == 1 ? base + q : layer;
            }
            seam[(((size_t)e) * g + m) * na + s] = dn;
          }
        for (int s = 0; s < na; ++s) {
          double A[3][3];
          const double t = (s + 0.5) * h, en = side == 0 ? 0.0 : 1.0;
          if (ax == 1) basisAt(b, en, t, A, X);
          else basisAt(b, t, en, A, X);
          panelCoords(nb, X, y1, y2);
          faceMap[(size_t)e * na + s] = (int)std::lround((nax == 1 ? y2 : y1) / h - 0.5);
        }
      }

  // Inner wind table (time-independent when strength == 0).
  std::vector<double> inner;
  if (P.init_condition_type == 1 && P.strength == 0.0) {
    inner.resize((size_t)6 * na * na * g * NC);
    for (int b = 0; b < 6; ++b)
      for (int k = 0; k < na; ++k)
        for (int j = 0; j < na; ++j) {
          const size_t ci = ((size_t)b * na + k) * na + j;
          for (int i = -g; i < 0; ++i) {
            const double radius = rc[i + g];
            const double X[3] = {radius * grav[ci].x[0], radius * grav[ci].x[1], radius * grav[ci].x[2]};
            windNative(P, X, &inner[(ci * g + (i + g)) * NC]);
          }
        }
  }

  cudaError_t err = cudaSuccess;
  L.radial = upload(radial, c->owned, err);
  L.rc = upload(rc, c->owned, err);
  L.face = upload(faces, c->owned, err);
  L.grav = upload(grav, c->owned, err);
  L.basis = upload(basis, c->owned, err);
  L.basisInv = upload(basisInv, c->owned, err);
  L.cfl = upload(cfl, c->owned, err);
  L.seam = upload(seam, c->owned, err);
  L.faceMap = upload(faceMap, c->owned, err);
  L.edge = upload(edges, c->owned, err);
  L.innerBC = inner.empty() ? nullptr : upload(inner, c->owned, err);
  if (err != cudaSuccess) return cudaFail(err, "geometry upload");
  return HC_OK;
}

// The face frame of the factored Roe dissipation for basis A (row-major
// 3 x 3) and face direction dir, in the record layout of kO4RoeRec.
void roeFrame(const double* A, int dir, double* out) {
  const int t1 = (dir + 1) % 3, t2 = (dir + 2) % 3;
  double f0[3], f1[3], normal2 = 0.0, tangent2 = 0.0;
  for (int i = 0; i < 3; ++i) {
    const int j = (i + 1) % 3, k = (i + 2) % 3;
    f0[i] = A[3 * j + t1] * A[3 * k + t2] - A[3 * k + t1] * A[3 * j + t2];
    f1[i] = A[3 * i + t1];
    normal2 += f0[i] * f0[i];
    tangent2 += f1[i] * f1[i];
  }
  const double normalMag = std::sqrt(normal2), tangentMag = std::sqrt(tangent2);
  const double invN = 1.0 / normalMag, invT = 1.0 / tangentMag;
  for (int i = 0; i < 3; ++i) { f0[i] *= invN; f1[i] *= invT; }
  for (int i = 0; i < 3; ++i) {
    const int j = (i + 1) % 3, k = (i + 2) % 3;
    out[i] = f0[i];
    out[3 + i] = f1[i];
    out[6 + i] = f0[j] * f1[k] - f0[k] * f1[j];
  }
  out[9] = normalMag;
  double adj[3][3];
  for (int dd = 0; dd < 3; ++dd) {
    const int s1 = (dd + 1) % 3, s2 = (dd + 2) % 3;
    for (int i = 0; i < 3; ++i) {
      const int j = (i + 1) % 3, k = (i + 2) % 3;
      adj[dd][i] = A[3 * j + s1] * A[3 * k + s2] - A[3 * k + s1] * A[3 * j + s2];
      out[10 + 3 * dd + i] = adj[dd][i];
    }
  }
  const double det = A[0] * adj[0][0] + A[3] * adj[0][1] + A[6] * adj[0][2];
  out[19] = 1.0 / det;
  out[20] = 1.0 / (det * det);
}

// Fourth-order metric tables over angular indices [-ext, na+ext] (ghost
// cells beyond the panel edges use the gnomonic extension of the map) and the
// radial table over [-kO4Rad, nr+kO4Rad].
int buildO4Geometry(hc_ctx* c) {
  const hc_params& P = c->P;
  const int na = P.na, nr = P.nr, ext = kO4Ang;
  const int n = na + 2 * ext + 1;
  const double h = 1.0 / na;
  Gauss G;
  std::vector<double> face((size_t)6 * 3 * n * n * kO4FaceRec), cell((size_t)6 * n * n * 9);
  for (int b = 0; b < 6; ++b)
    for (int k = -ext; k <= na + ext; ++k)
      for (int j = -ext; j <= na + ext; ++j) {
        double A[3][3];
        basisAt(b, (j + 0.5) * h, (k + 0.5) * h, A, nullptr);
        double* cb = &cell[(((size_t)b * n + (k + ext)) * n + (j + ext)) * 9];
        for (int r = 0; r < 3; ++r)
          for (int q = 0; q < 3; ++q) cb[3 * r + q] = A[r][q];
        for (int d = 0; d < 3; ++d) {
          double* e = &face[((((size_t)b * 3 + d) * n + (k + ext)) * n + (j + ext)) * kO4FaceRec];
          double dA[3][3] = {{0}}, det = 0, nn[3] = {0, 0, 0};
          if (d == 0) {
            for (int p = 0; p < 8; ++p)
              for (int q = 0; q < 8; ++q) {
                double Aq[3][3], m[3];
                basisAt(b, (j + G.x[p]) * h, (k + G.x[q]) * h, Aq, nullptr);
                const double wt = G.w[p] * G.w[q], dt = det3(Aq);
                det += wt * dt;
                cofactorRow(Aq, 0, m);
                for (int r = 0; r < 3; ++r) {
                  nn[r] += wt * m[r];
                  for (int s2 = 0; s2 < 3; ++s2) dA[r][s2] += wt * dt * Aq[r][s2];
                }
              }
          } else {
            for (int p = 0; p < 8; ++p) {
              double Aq[3][3], m[3];
              if (d == 1) basisAt(b, j * h, (k + G.x[p]) * h, Aq, nullptr);
              else basisAt(b, (j + G.x[p]) * h, k * h, Aq, nullptr);
              const double dt = det3(Aq);
              det += G.w[p] * dt;
              cofactorRow(Aq, d, m);
              for (int r = 0; r < 3; ++r) {
                nn[r] += G.w[p] * m[r];
                for (int s2 = 0; s2 < 3; ++s2) dA[r][s2] += G.w[p] * dt * Aq[r][s2];
              }
            }
          }
          snapNormal(nn);
          for (int r = 0; r < 3; ++r)
            for (int q = 0; q < 3; ++q) e[3 * r + q] = dA[r][q];
          e[9] = det;
          for (int r = 0; r < 3; ++r) e[10 + r] = nn[r];
          double F[3][3];
          if (d == 0) basisAt(b, (j + 0.5) * h, (k + 0.5) * h, F, nullptr);
          else if (d == 1) basisAt(b, j * h, (k + 0.5) * h, F, nullptr);
          else basisAt(b, (j + 0.5) * h, k * h, F, nullptr);
          for (int r = 0; r < 3; ++r)
            for (int q = 0; q < 3; ++q) e[13 + 3 * r + q] = F[r][q];
        }
      }
  // Roe frames (the geometry half of the factored Roe dissipation,
  // src/MHD_Roe8Wave.H:634-740, which depends only on the face's angular
  // position): computed once here instead of at every face of every stage.
  std::vector<double> roe((size_t)6 * 3 * n * n * kO4RoeRec, 0.0);
  for (int b = 0; b < 6; ++b)
    for (int d = 0; d < 3; ++d)
      for (int k = 0; k < n; ++k)
        for (int j = 0; j < n; ++j) {
          const size_t at = (((size_t)b * 3 + d) * n + k) * n + j;
          const double* A = d == 0 ? &cell[((size_t)b * n + k) * n * 9 + (size_t)j * 9] : &face[at * kO4FaceRec + 13];
          roeFrame(A, d, &roe[at * kO4RoeRec]);
        }
  std::vector<double4> radial(nr + 2 * kO4Rad + 1);
  for (int i = -kO4Rad; i <= nr + kO4Rad; ++i) {
    const RadialRow r = radialRow(P, i);
    radial[i + kO4Rad] = make_double4(r.area0, r.areaT, r.Dr0, r.vol);
  }
  cudaError_t err = cudaSuccess;
  O4Geo& g = c->o4;
  g.nr = nr; g.na = na; g.ext = ext;
  g.face = upload(face, c->owned, err);
  g.cell = upload(cell, c->owned, err);
  g.frames = upload(roe, c->owned, err);
  g.radial = upload(radial, c->owned, err);
  g.gamma = P.gamma; g.invGm1 = 1.0 / (P.gamma - 1.0); g.entropy = P.entropy_fix_coeff; g.eta_d = P.berta_eta_d;
  g.dx[0] = 1.0 / shellCells(P); g.dx[1] = 1.0 / na; g.dx[2] = 1.0 / na;
  g.roe = P.riemann_solver == 2; g.powell = P.divergence_cleaning == 1; g.fallback = P.berta_fallback_type;
  // the CME insertion window's Rusanov flag (0 until a schedule sets it)
  {
    cudaError_t ferr = cudaMalloc(&c->rusanovFlag, 2 * sizeof(int));
    if (ferr == cudaSuccess) ferr = cudaMemset(c->rusanovFlag, 0, 2 * sizeof(int));
    if (ferr != cudaSuccess) return cudaFail(ferr, "O4 flag");
    c->owned.push_back(c->rusanovFlag);
  }
  g.rusanov = c->rusanovFlag;
  g.status = c->rusanovFlag + 1;
  if (err != cudaSuccess) return cudaFail(err, "O4 geometry upload");
  return HC_OK;
}

// Panel holding direction X; directions within 1e-12 of a panel edge go to
// the lowest panel index, so seam-interpolation stencils do not depend on
// round-off.
int locateTie(const double X[3]) {
  double q0[6], best = -2;
  for (int b = 0; b < 6; ++b) {
    q0[b] = 0;
    for (int k = 0; k < 3; ++k)
      if (PERM[b][k] == 0) q0[b] = SIGN[b][k] * X[k];
    best = std::max(best, q0[b]);
  }
  for (int b = 0; b < 6; ++b)
    if (q0[b] >= best - 1e-12 * std::fabs(best)) return b;
  return 0;
}

// Point value at u (cell m spans [m, m+1]) of the cubic whose averages over
// cells base..base+3 are given: the derivative of the quartic through the
// running sums at faces base..base+4.
void averageInterp(long double u, int base, double w[4], long double scale) {
  long double dL[5];
  for (int n = 0; n < 5; ++n) {
    long double sum = 0;
    for (int r = 0; r < 5; ++r) {
      if (r == n) continue;
      long double t = 1.0L / (n - r);
      for (int q = 0; q < 5; ++q)
        if (q != n && q != r) t *= (u - (base + q)) / (long double)(n - q);
      sum += t;
    }
    dL[n] = sum;
  }
  for (int m = 0; m < 4; ++m) {
    long double acc = 0;
    for (int n = m + 1; n < 5; ++n) acc += dL[n];
    w[m] = (double)(scale * acc);
  }
}

// Tables of the fourth-order level step and its level-sized buffers.
int buildO4Level(hc_ctx* c) {
  const hc_params& P = c->P;
  const int nr = P.nr, na = P.na, g = kO4Ghost, ga = kO4Cart;
  const int nA = na + 2 * ga, nG = na + 2 * g;
  const double h = 1.0 / na;
  Gauss G;
  O4Level& O = c->o4l;
  O.nr = nr; O.na = na; O.g = g; O.ga = ga; O.nA = nA; O.nG = nG;
  O.Nv = (long)nr * na * na;
  O.Ng = (long)(nr + 2 * g) * nG * nG;
  O.Nc = (long)nr * nA * nA;
  O.gamma = P.gamma; O.r0 = P.inner_radius; O.strength = P.strength; O.cfl = P.cfl;
  std::vector<double> coef((size_t)6 * nA * nA * 27, 0.0), Ab((size_t)6 * nA * nA * 9);
  std::vector<double> detx((size_t)6 * (na + 2) * (na + 2)), xhat((size_t)6 * nG * nG * 3);
  std::vector<int2> ringJK;
  for (int k = -ga; k < na + ga; ++k)
    for (int j = -ga; j < na + ga; ++j)
      if (!(j >= 0 && j < na && k >= 0 && k < na)) ringJK.push_back(make_int2(j, k));
  O.nring = (int)ringJK.size();
  // interpolation points: ghost centres and their 4 neighbours
  static const int off[5][2] = {{0, 0}, {1, 0}, {-1, 0}, {0, 1}, {0, -1}};
  const int nP = na + 2 * ga + 2;  // point grid [-ga-1, na+ga+1)
  std::vector<int> ptIndex((size_t)nP * nP, -1), ringPt((size_t)O.nring * 5);
  std::vector<int2> ptJK;
  for (int r = 0; r < O.nring; ++r)
    for (int q = 0; q < 5; ++q) {
      const int j = ringJK[r].x + off[q][0], k = ringJK[r].y + off[q][1];
      int& idx = ptIndex[(size_t)(k + ga + 1) * nP + (j + ga + 1)];
      if (idx < 0) {
        idx = (int)ptJK.size();
        ptJK.push_back(make_int2(j, k));
      }
      ringPt[(size_t)r * 5 + q] = idx;
    }
  O.npts = (int)ptJK.size();
  std::vector<O4Point> pts((size_t)6 * O.npts);
  auto aIdx = [&](int b, int j, int k) { return ((size_t)b * nA + (k + ga)) * nA + (j + ga); };
  for (int b = 0; b < 6; ++b) {
    for (int k = -ga; k < na + ga; ++k)
      for (int j = -ga; j < na + ga; ++j) {
        double A[3][3] = {{0}}, I[3][3];
        for (int p = 0; p < 8; ++p)
          for (int q = 0; q < 8; ++q) {
            double Aq[3][3];
            basisAt(b, (j + G.x[p]) * h, (k + G.x[q]) * h, Aq, nullptr);
            for (int r = 0; r < 3; ++r)
              for (int s2 = 0; s2 < 3; ++s2) A[r][s2] += G.w[p] * G.w[q] * Aq[r][s2];
          }
        inv3(A, I);
        for (int r = 0; r < 3; ++r)
          for (int s2 = 0; s2 < 3; ++s2) {
            Ab[aIdx(b, j, k) * 9 + 3 * r + s2] = A[r][s2];
            coef[aIdx(b, j, k) * 27 + 3 * r + s2] = I[r][s2];
          }
      }
    for (int k = -ga + 1; k < na + ga - 1; ++k)
      for (int j = -ga + 1; j < na + ga - 1; ++j)
        for (int e = 0; e < 9; ++e) {
          coef[aIdx(b, j, k) * 27 + 9 + e] = 0.5 * (Ab[aIdx(b, j + 1, k) * 9 + e] - Ab[aIdx(b, j - 1, k) * 9 + e]);
          coef[aIdx(b, j, k) * 27 + 18 + e] = 0.5 * (Ab[aIdx(b, j, k + 1) * 9 + e] - Ab[aIdx(b, j, k - 1) * 9 + e]);
        }
    for (int k = -1; k <= na; ++k)
      for (int j = -1; j <= na; ++j) {
        double det = 0;
        for (int p = 0; p < 8; ++p)
          for (int q = 0; q < 8; ++q) {
            double Aq[3][3];
            basisAt(b, (j + G.x[p]) * h, (k + G.x[q]) * h, Aq, nullptr);
            det += G.w[p] * G.w[q] * det3(Aq);
          }
        detx[((size_t)b * (na + 2) + (k + 1)) * (na + 2) + (j + 1)] = det;
      }
    for (int k = -g; k < na + g; ++k)
      for (int j = -g; j < na + g; ++j) {
        double A[3][3], X[3];
        basisAt(b, (j + 0.5) * h, (k + 0.5) * h, A, X);
        for (int q = 0; q < 3; ++q) xhat[(((size_t)b * nG + (k + g)) * nG + (j + g)) * 3 + q] = X[q];
      }
    for (int q = 0; q < O.npts; ++q) {
      const int j = ptJK[q].x, k = ptJK[q].y;
      double A[3][3], X[3], y1, y2;
      basisAt(b, (j + 0.5) * h, (k + 0.5) * h, A, X);
      O4Point pt{};
      pt.p = locateTie(X);
      panelCoords(pt.p, X, y1, y2);
      const long double u1 = (long double)y1 / h, u2 = (long double)y2 / h;
      pt.j0 = std::max(0, std::min(na - 4, (int)std::floor((double)u1) - 1));
      pt.k0 = std::max(0, std::min(na - 4, (int)std::floor((double)u2) - 1));
      const int jc = std::max(0, std::min(na - 1, (int)std::floor((double)u1)));
      const int kc = std::max(0, std::min(na - 1, (int)std::floor((double)u2)));
      pt.cell = (jc - pt.j0) | ((kc - pt.k0) << 2);
      averageInterp(u1, pt.j0, pt.wj, 1.0L);
      averageInterp(u2, pt.k0, pt.wk, 1.0L);
      pts[(size_t)b * O.npts + q] = pt;
    }
  }
  std::vector<double2> radial(nr + 2 * g + 2);
  for (int i = -g - 1; i <= nr + g; ++i) {
    const RadialRow rr = radialRow(P, i);
    radial[i + g + 1] = make_double2(rr.vol, rr.rhalf);
  }
  // The inner analytic wind does not depend on time when its perturbation
  // strength is zero: tabulate the inner radial ghosts once.
  std::vector<double> inner;
  if (P.init_condition_type == 1 && P.strength == 0.0) {
    inner.resize((size_t)6 * nG * nG * g * 8);
    for (int b = 0; b < 6; ++b)
      for (int k = -g; k < na + g; ++k)
        for (int j = -g; j < na + g; ++j) {
          const size_t cell = ((size_t)b * nG + (k + g)) * nG + (j + g);
          for (int i = -g; i < 0; ++i) {
            const double radius = radial[i + g + 1].y;
            const double X[3] = {radius * xhat[cell * 3], radius * xhat[cell * 3 + 1], radius * xhat[cell * 3 + 2]};
            windNative(P, X, &inner[(cell * g + (i + g)) * 8]);
          }
        }
  }
  cudaError_t err = cudaSuccess;
  O.coef = upload(coef, c->owned, err);
  O.detx = upload(detx, c->owned, err);
  O.xhat = upload(xhat, c->owned, err);
  O.radial = upload(radial, c->owned, err);
  O.ringJK = upload(ringJK, c->owned, err);
  O.ringPt = upload(ringPt, c->owned, err);
  O.pts = upload(pts, c->owned, err);
  O.inner = inner.empty() ? nullptr : upload(inner, c->owned, err);
  if (err != cudaSuccess) return cudaFail(err, "O4 level tables");
  return HC_OK;
}

// Carve the operator scratch of nbox boxes (valid box [vlo, vhi]) from sp.
void carveO4Scratch(O4Args& a, double* sp) { o4CarveScratch(a, sp); }

int allocWorkspace(hc_ctx* c) {
  const size_t nv = 6 * NC * (size_t)c->L.Nv, ng = 6 * NC * (size_t)c->L.Ng;
  void* p;
  cudaError_t e;
  for (int q = 0; q < 2 && c->P.spatial_order == 2; ++q) {
    if ((e = cudaMalloc(&p, ng * sizeof(double))) != cudaSuccess) return cudaFail(e, "workspace W");
    c->owned.push_back(p); c->W[q] = (double*)p;
    if ((e = cudaMemset(p, 0, ng * sizeof(double))) != cudaSuccess) return cudaFail(e, "workspace W");
  }
  if (c->P.spatial_order == 2) {
    if ((e = cudaMalloc(&p, nv * sizeof(double))) != cudaSuccess) return cudaFail(e, "workspace acc");
    c->owned.push_back(p); c->acc = (double*)p;
  }
  if ((e = cudaMalloc(&p, 64)) != cudaSuccess) return cudaFail(e, "workspace scalars");
  c->owned.push_back(p); c->invMax = (unsigned long long*)p;
  c->flag = (int*)((char*)p + 32);
  return HC_OK;
}

StageArgs levelArgs(hc_ctx* c, const double* w) {
  StageArgs a{};
  a.L = c->L;
  a.w = w;
  a.wBoxStride = NC * c->L.Ng;
  a.wN = c->L.Ng;
  for (int d = 0; d < 3; ++d) a.wlo[d] = -kGhost;
  a.wn[0] = c->L.n0; a.wn[1] = c->L.n1; a.wn[2] = c->L.n1;
  a.lo[0] = a.lo[1] = a.lo[2] = 0;
  a.hi[0] = c->P.nr - 1; a.hi[1] = a.hi[2] = c->P.na - 1;
  a.nbox = 6;
  a.block0 = 0;
  a.scale = 1.0;
  a.seams = 1;
  return a;
}

int checkLaunch(cudaError_t e, const char* what) { return e == cudaSuccess ? HC_OK : cudaFail(e, what); }

// Stage s of one RK4 step on W[0] = primitives of ju (valid cells): fill
// the ghosts of W[s % 2], then the fused operator + update writes the next
// stage's primitives into W[(s + 1) % 2]; stage 3 leaves the new state's
// primitives in W[0] and, with invMaxOut, its CFL rate.
int rkStage(hc_ctx* c, double* ju, int stage, double dtv, const double* invMax, unsigned long long* invMaxOut,
            double tbase, const double* tdev, cudaStream_t s) {
  static const double c4[4] = {0, 0.5, 0.5, 1};
  {
    double* win = c->W[stage % 2];
    StageTime st{tbase, tdev, c4[stage], invMax, dtv};
    int rc = checkLaunch(launchGhosts(c->L, win, st, s), "ghosts");
    if (rc != HC_OK) return rc;
    StageArgs a = levelArgs(c, win);
    a.stage = stage;
    a.invDtMax = invMax;
    a.dtv = dtv;
    a.ju = ju;
    a.acc = c->acc;
    a.wOut = c->W[(stage + 1) % 2];
    a.invMaxOut = stage == 3 ? invMaxOut : nullptr;
    a.invalid = nullptr;
    a.tbase = tbase;
    a.tdev = tdev;
    if (c->P.riemann_solver == 2 && c->sched && c->rusanovFlag) {
      // Roe context under an insertion schedule: the window flag picks the
      // Roe or the Rusanov stage kernel on the device
      a.solverFlag = c->rusanovFlag;
      a.exitOnFlag = 1;
      rc = checkLaunch(launchStage(a, MODE_RK, c->P.limiter, true, c->P.divergence_cleaning == 1,
                                   c->P.sun_gravity == 1, s, c->tileRK),
                       "stage");
      a.exitOnFlag = 0;
      if (rc == HC_OK)
        rc = checkLaunch(launchStage(a, MODE_RK, c->P.limiter, false, c->P.divergence_cleaning == 1,
                                     c->P.sun_gravity == 1, s, c->tileRK),
                         "stage");
    } else {
      rc = checkLaunch(launchStage(a, MODE_RK, c->P.limiter, c->P.riemann_solver == 2, c->P.divergence_cleaning == 1,
                                   c->P.sun_gravity == 1, s, c->tileRK),
                       "stage");
    }
    if (rc != HC_OK) return rc;
  }
  return HC_OK;
}

int rkStep(hc_ctx* c, double* ju, double dtv, const double* invMax, unsigned long long* invMaxOut, double tbase,
           const double* tdev, cudaStream_t s) {
  for (int stage = 0; stage < 4; ++stage) {
    const int rc = rkStage(c, ju, stage, dtv, invMax, invMaxOut, tbase, tdev, s);
    if (rc != HC_OK) return rc;
  }
  return HC_OK;
}

// The batched operator over the six panels of the fourth-order level.
O4Args levelO4Args(hc_ctx* c, const double* us, double* k) {
  O4Args a{};
  a.G = c->o4;
  a.nbox = 6;
  a.block0 = 0;
  a.ghost = kO4Ghost;
  a.vlo[0] = a.vlo[1] = a.vlo[2] = 0;
  a.vhi[0] = c->P.nr - 1;
  a.vhi[1] = a.vhi[2] = c->P.na - 1;
  a.U = us;
  for (int d = 0; d < 3; ++d) {
    a.ur.lo[d] = -kO4Ghost;
    a.ur.n[d] = a.vhi[d] + 1 + 2 * kO4Ghost;
  }
  a.ur.N = c->o4l.Ng;
  a.uStride = 8 * c->o4l.Ng;
  a.scale = 1.0;
  a.rhs = k;
  a.rhsStride = 8 * c->o4l.Nv;
  carveO4Scratch(a, c->o4lvlScratch);
  return a;
}

// The operator batch of an argument set, built on first use (device
// allocations, a copy, the batch's side streams and events: not inside a
// stream capture) and kept for the next calls.
O4Batch* cachedBatch(hc_ctx* c, const O4Args& a, int* rc) {
  std::string key;
  auto put = [&key](const void* p, size_t n) { key.append(static_cast<const char*>(p), n); };
  put(&a.nbox, sizeof a.nbox); put(&a.block0, sizeof a.block0); put(&a.ghost, sizeof a.ghost);
  put(a.vlo, sizeof a.vlo); put(a.vhi, sizeof a.vhi); put(&a.U, sizeof a.U); put(a.ur.lo, sizeof a.ur.lo);
  put(a.ur.n, sizeof a.ur.n); put(&a.uStride, sizeof a.uStride); put(&a.scale, sizeof a.scale);
  put(&a.rhs, sizeof a.rhs); put(&a.rhsStride, sizeof a.rhsStride); put(a.flux, sizeof a.flux);
  put(&a.WA, sizeof a.WA); put(&a.face, sizeof a.face); put(&a.face2, sizeof a.face2); put(&a.kp, sizeof a.kp);
  put(&a.rr, sizeof a.rr);
  for (auto& e : c->o4cache)
    if (e.first == key) return e.second;
  std::vector<O4Args> boxes;
  o4SplitArgs(a, boxes);
  cudaError_t err;
  O4Batch* B = o4BatchCreate(boxes.data(), (int)boxes.size(), &err);
  if (!B) {
    *rc = cudaFail(err, "O4 batch");
    return nullptr;
  }
  if (c->o4cache.size() >= 32) {
    o4BatchDestroy(c->o4cache.front().second);
    c->o4cache.erase(c->o4cache.begin());
  }
  c->o4cache.emplace_back(key, B);
  return B;
}

// The operator batch of the level step: the six panels, or their radial
// window [winLo, winHi) writing into the level-layout k (the cells outside
// keep rhs 0).
int buildO4LevelBatch(hc_ctx* c) {
  O4Args a = levelO4Args(c, c->o4us, c->o4k);
  if (c->winHi > 0) {
    a.vlo[0] = c->winLo;
    a.vhi[0] = c->winHi - 1;
    a.rr.lo[0] = a.rr.lo[1] = a.rr.lo[2] = 0;
    a.rr.n[0] = c->o4l.nr;
    a.rr.n[1] = a.rr.n[2] = c->o4l.na;
    a.rr.N = c->o4l.Nv;
    carveO4Scratch(a, c->o4lvlScratch);
  }
  std::vector<O4Args> boxes;
  o4SplitArgs(a, boxes);
  cudaError_t err;
  c->o4levelBatch = o4BatchCreate(boxes.data(), (int)boxes.size(), &err);
  return c->o4levelBatch ? HC_OK : cudaFail(err, "O4 level batch");
}

// Level-sized buffers of the fourth-order level step and the operator batch
// over them, allocated on the first level call (so a context used only for
// box and batch evaluations holds none): make that first call outside any
// stream capture.
int ensureO4Buffers(hc_ctx* c) {
  if (c->o4levelBatch) return HC_OK;
  if (c->o4us) return buildO4LevelBatch(c);
  const O4Level& O = c->o4l;
  const int nr = O.nr, na = O.na;
  const int vlo[3] = {0, 0, 0}, vhi[3] = {nr - 1, na - 1, na - 1};
  const size_t sizes[8] = {(size_t)6 * 8 * O.Ng, (size_t)6 * 8 * O.Nc, (size_t)6 * 8 * O.Nv, (size_t)6 * 8 * O.Nv,
                           (size_t)6 * 2 * 2 * 8 * na * nr, o4ScratchDoubles(6, vlo, vhi, kO4Ghost),
                           (size_t)6 * 8 * O.Nv, (size_t)6 * 8 * O.npts * nr};
  double** dst[8] = {&c->o4us, &c->o4cart, &c->o4next, &c->o4k, &c->o4reg, &c->o4lvlScratch, &c->acc, &c->o4pv};
  cudaError_t err;
  for (int q = 0; q < 8; ++q) {
    void* p = nullptr;
    if ((err = cudaMalloc(&p, sizes[q] * sizeof(double))) != cudaSuccess) return cudaFail(err, "O4 level buffers");
    c->owned.push_back(p);
    *dst[q] = static_cast<double*>(p);
    if ((err = cudaMemset(p, 0, sizes[q] * sizeof(double))) != cudaSuccess) return cudaFail(err, "O4 level buffers");
  }
  return buildO4LevelBatch(c);
}

// Stage `stage` of one fourth-order RK4 step: prepare USph from the stage
// state, evaluate the operator into k (seam fluxes into the register, which
// stage 0 clears), update the accumulator and the next stage; stage 3 then
// reconciles the seam fluxes.
int o4Stage(hc_ctx* c, double* ju, int stage, double dtv, const double* invMax, double tbase, const double* tdev,
            cudaStream_t s) {
  static const double c4[4] = {0, 0.5, 0.5, 1}, b4[4] = {1.0 / 6, 1.0 / 3, 1.0 / 3, 1.0 / 6};
  const O4Level& O = c->o4l;
  int rc = HC_OK;
  if (stage == 0)
    rc = checkLaunch(cudaMemsetAsync(c->o4reg, 0, sizeof(double) * 6 * 2 * 2 * 8 * O.na * O.nr, s), "register");
  if (rc != HC_OK) return rc;
  O4StageIO io{O, stage == 0 ? ju : c->o4next, c->o4cart, c->o4us, c->o4pv,
               StageTime{tbase, tdev, c4[stage], invMax, dtv}};
  rc = checkLaunch(launchO4Prepare(io, s), "O4 prepare");
  if (rc == HC_OK) rc = checkLaunch(cudaMemsetAsync(c->o4k, 0, sizeof(double) * 6 * 8 * O.Nv, s), "O4 k");
  if (rc != HC_OK) return rc;
  if (c->P.sun_gravity) {
    rc = checkLaunch(launchO4BatchGravity(c->o4levelBatch, s), "O4 gravity");
    if (rc != HC_OK) return rc;
  }
  const RegArgs rg{c->o4reg, invMax ? b4[stage] : dtv * b4[stage], invMax, c->P.cfl};
  o4BatchSetVariants(c->o4levelBatch, c->o4var);
  rc = checkLaunch(launchO4Batch(c->o4levelBatch, &rg, s), "O4 operator");
  if (rc == HC_OK)
    rc = checkLaunch(launchO4Update(O, stage, c->o4k, ju, c->acc, c->o4next, invMax, c->P.cfl, dtv, s), "O4 update");
  if (rc == HC_OK && stage == 3) rc = checkLaunch(launchO4Reflux(O, c->L, c->o4reg, ju, s), "O4 reflux");
  return rc;
}

int o4Step(hc_ctx* c, double* ju, double dtv, const double* invMax, double tbase, const double* tdev, cudaStream_t s) {
  int rc = HC_OK;
  for (int stage = 0; stage < 4 && rc == HC_OK; ++stage) rc = o4Stage(c, ju, stage, dtv, invMax, tbase, tdev, s);
  return rc;
}

}  // namespace

namespace hc {
const DevLevel* ctxLevel(const hc_ctx* c) { return &c->L; }
const hc_params* ctxParams(const hc_ctx* c) { return &c->P; }
int ctxDevice(const hc_ctx* c) { return c->device; }
const O4Level* ctxO4Level(const hc_ctx* c) { return c->P.spatial_order == 4 ? &c->o4l : nullptr; }
int setLastError(int code, const char* msg) { return fail(code, msg); }
}  // namespace hc

extern "C" {

const char* hc_last_error(void) { return g_lastError.c_str(); }

int hc_ctx_create(const hc_params* p, int device, hc_ctx** out) {
  if (!p || !out) return fail(HC_ERR_ARG, "null argument");
  *out = nullptr;
  if (p->spatial_order != 2 && p->spatial_order != 4)
    return fail(HC_ERR_UNSUPPORTED, "spatial_order must be 2 (PLM) or 4 (Berta WENOZ)");
  if (p->spatial_order == 4) {
    if (p->spatial_operator != 2) return fail(HC_ERR_UNSUPPORTED, "at order 4 only spatial_operator 2 (Berta) is built");
    if (p->berta_detector_type != 0) return fail(HC_ERR_UNSUPPORTED, "Berta_detector_type must be 0 (Jameson)");
    if (p->berta_fallback_type != 0 && p->berta_fallback_type != 1) return fail(HC_ERR_ARG, "Berta_fallback_type must be 0 or 1");
    if (!(p->berta_eta_d > 0)) return fail(HC_ERR_ARG, "Berta_eta_d must be positive");
    if (p->na < 2 * kO4Ang) return fail(HC_ERR_ARG, "the fourth-order operator needs na >= 16");
  }
  if (p->limiter < 0 || p->limiter > 3) return fail(HC_ERR_ARG, "limiter must be 0..3");
  if (p->riemann_solver != 1 && p->riemann_solver != 2) return fail(HC_ERR_ARG, "Riemann_solver_type must be 1 or 2");
  if (p->temporal_order != 4) return fail(HC_ERR_UNSUPPORTED, "temporal_order must be 4 (classical RK4)");
  if (p->nr < 4 || p->na < 4) return fail(HC_ERR_ARG, "need nr >= 4 and na >= 4");
  if (p->radial_offset < 0 || p->radial_cells < 0) return fail(HC_ERR_ARG, "radial_offset and radial_cells must be >= 0");
  if (p->radial_cells == 0 ? p->radial_offset != 0 : p->radial_offset + p->nr > p->radial_cells)
    return fail(HC_ERR_ARG, "a radial slab must lie inside its shell: radial_offset + nr <= radial_cells");
  // The level kernels index cells and components in 32 bits: every ghosted
  // component array of the level (ghost layers of either order) must stay
  // below 2^31 entries.
  if (48.0 * (p->nr + 12.0) * (p->na + 12.0) * (p->na + 12.0) >= 2147483647.0)
    return fail(HC_ERR_ARG, "level too large: 48 (nr + 12) (na + 12)^2 must stay below 2^31");
  if (!(p->gamma > 1.0)) return fail(HC_ERR_ARG, "gamma must exceed 1");
  if (!(p->inner_radius > 0.0 && p->outer_radius > p->inner_radius))
    return fail(HC_ERR_ARG, "need 0 < inner_radius < outer_radius");
  if (p->init_condition_type != 1) return fail(HC_ERR_UNSUPPORTED, "radial boundary family must be 1 (analytic wind)");
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return cudaFail(e, "cudaSetDevice");
  hc_ctx* c = new (std::nothrow) hc_ctx;
  if (!c) return fail(HC_ERR_NOMEM, "context allocation");
  c->P = *p;
  c->device = device;
  int rc = buildLevel(c);
  if (rc == HC_OK) rc = allocWorkspace(c);
  if (rc == HC_OK && p->spatial_order == 4) rc = buildO4Geometry(c);
  if (rc == HC_OK && p->spatial_order == 4) rc = buildO4Level(c);
  if (rc != HC_OK) {
    hc_ctx_destroy(c);
    return rc;
  }
  *out = c;
  return HC_OK;
}

int hc_ctx_destroy(hc_ctx* c) {
  if (!c) return HC_OK;
  cudaSetDevice(c->device);
  for (auto& e : c->o4cache) o4BatchDestroy(e.second);
  o4BatchDestroy(c->o4levelBatch);
  for (void* p : c->owned) cudaFree(p);
  if (c->o4scratch) cudaFree(c->o4scratch);
  delete c;
  return HC_OK;
}

size_t hc_level_state_size(const hc_ctx* c) { return c ? 6 * NC * (size_t)c->L.Nv : 0; }
size_t hc_level_primitive_size(const hc_ctx* c) {
  if (!c) return 0;
  return c->P.spatial_order == 4 ? 6 * NC * (size_t)c->o4l.Ng : 6 * NC * (size_t)c->L.Ng;
}

int hc_box_rhs(hc_ctx* c, const hc_box* box, const double* w, const double* const* panel, double scale, double* rhs,
               double* const* flux, void* stream) {
  if (!c || !box || !w || !rhs) return fail(HC_ERR_ARG, "null argument");
  const hc_box& B = *box;
  if (B.block < 0 || B.block > 5) return fail(HC_ERR_ARG, "block must be 0..5");
  if (B.ghost < 2) return fail(HC_ERR_ARG, "the PLM operator needs ghost >= 2");
  const int n[3] = {c->P.nr, c->P.na, c->P.na};
  for (int d = 0; d < 3; ++d)
    if (B.lo[d] < 0 || B.hi[d] >= n[d] || B.hi[d] < B.lo[d]) return fail(HC_ERR_ARG, "box outside the panel");
  StageArgs a{};
  a.L = c->L;
  a.w = w;
  for (int d = 0; d < 3; ++d) {
    a.wlo[d] = B.lo[d] - B.ghost;
    a.wn[d] = B.hi[d] - B.lo[d] + 1 + 2 * B.ghost;
    a.lo[d] = B.lo[d];
    a.hi[d] = B.hi[d];
  }
  a.wN = (long)a.wn[0] * a.wn[1] * a.wn[2];
  a.wBoxStride = 0;
  a.nbox = 1;
  a.block0 = B.block;
  a.scale = scale;
  a.rhs = rhs;
  a.rhsN = (long)(B.hi[0] - B.lo[0] + 1) * (B.hi[1] - B.lo[1] + 1) * (B.hi[2] - B.lo[2] + 1);
  for (int d = 0; d < 3; ++d) a.flux[d] = flux ? flux[d] : nullptr;
  for (int q = 0; q < 6; ++q) a.panel[q] = panel ? panel[q] : nullptr;
  return checkLaunch(launchStage(a, MODE_BOX, c->P.limiter, c->P.riemann_solver == 2, c->P.divergence_cleaning == 1,
                                 false, (cudaStream_t)stream),
                     "hc_box_rhs");
}

int hc_box_rhs_o4(hc_ctx* c, const hc_box* box, const double* usph, double scale, double* rhs, double* const* flux,
                  void* stream) {
  if (!c || !box || !usph || !rhs) return fail(HC_ERR_ARG, "null argument");
  if (c->P.spatial_order != 4) return fail(HC_ERR_UNSUPPORTED, "context was created with spatial_order != 4");
  const hc_box& B = *box;
  if (B.block < 0 || B.block > 5) return fail(HC_ERR_ARG, "block must be 0..5");
  if (B.ghost < kO4Ghost) return fail(HC_ERR_ARG, "the Berta operator needs ghost >= 5");
  const int n[3] = {c->P.nr, c->P.na, c->P.na};
  for (int d = 0; d < 3; ++d)
    if (B.lo[d] < 0 || B.hi[d] >= n[d] || B.hi[d] < B.lo[d]) return fail(HC_ERR_ARG, "box outside the panel");
  O4Args a{};
  a.G = c->o4;
  a.nbox = 1;
  a.block0 = B.block;
  a.ghost = kO4Ghost;
  for (int d = 0; d < 3; ++d) { a.vlo[d] = B.lo[d]; a.vhi[d] = B.hi[d]; }
  a.U = usph;
  for (int d = 0; d < 3; ++d) { a.ur.lo[d] = B.lo[d] - B.ghost; a.ur.n[d] = B.hi[d] - B.lo[d] + 1 + 2 * B.ghost; }
  a.ur.N = (long)a.ur.n[0] * a.ur.n[1] * a.ur.n[2];
  a.uStride = 8 * a.ur.N;
  a.scale = scale;
  a.rhs = rhs;
  a.rhsStride = 8L * (B.hi[0] - B.lo[0] + 1) * (B.hi[1] - B.lo[1] + 1) * (B.hi[2] - B.lo[2] + 1);
  for (int d = 0; d < 3; ++d) a.flux[d] = flux ? flux[d] : nullptr;
  // grow-only scratch (allocated outside any stream capture on first use)
  const size_t need = o4ScratchDoubles(1, a.vlo, a.vhi, kO4Ghost);
  if (need > c->o4scratchDoubles) {
    if (c->o4scratch) cudaFree(c->o4scratch);
    c->o4scratch = nullptr;
    c->o4scratchDoubles = 0;
    void* p = nullptr;
    const cudaError_t e = cudaMalloc(&p, need * sizeof(double));
    if (e != cudaSuccess) return cudaFail(e, "O4 scratch");
    c->o4scratch = static_cast<double*>(p);
    c->o4scratchDoubles = need;
  }
  carveO4Scratch(a, c->o4scratch);
  int rc = HC_OK;
  O4Batch* batch = cachedBatch(c, a, &rc);
  if (!batch) return rc;
  o4BatchSetVariants(batch, c->o4var);
  return checkLaunch(launchO4Batch(batch, nullptr, (cudaStream_t)stream), "hc_box_rhs_o4");
}

}  // extern "C"

struct hc_o4_batch {
  O4Batch* batch = nullptr;
  double* scratch = nullptr;
  int gravity = 0;
  int device = 0;
};

extern "C" {

int hc_o4_batch_create(hc_ctx* c, const hc_box_work* boxes, int nbox, double scale, hc_o4_batch** out) {
  if (!c || !boxes || !out || nbox <= 0) return fail(HC_ERR_ARG, "bad argument");
  *out = nullptr;
  if (c->P.spatial_order != 4) return fail(HC_ERR_UNSUPPORTED, "context was created with spatial_order != 4");
  if (nbox > 65535) return fail(HC_ERR_ARG, "at most 65535 boxes per batch");
  const int n[3] = {c->P.nr, c->P.na, c->P.na};
  std::vector<size_t> off(nbox + 1, 0);
  for (int b = 0; b < nbox; ++b) {
    const hc_box& B = boxes[b].box;
    if (!boxes[b].usph || !boxes[b].rhs) return fail(HC_ERR_ARG, "null usph or rhs in the batch");
    if (B.block < 0 || B.block > 5) return fail(HC_ERR_ARG, "block must be 0..5");
    if (B.ghost < kO4Ghost) return fail(HC_ERR_ARG, "the Berta operator needs ghost >= 5");
    for (int d = 0; d < 3; ++d)
      if (B.lo[d] < 0 || B.hi[d] >= n[d] || B.hi[d] < B.lo[d]) return fail(HC_ERR_ARG, "box outside the panel");
    off[b + 1] = off[b] + o4ScratchDoubles(1, B.lo, B.hi, kO4Ghost);
  }
  hc_o4_batch* h = new (std::nothrow) hc_o4_batch;
  if (!h) return fail(HC_ERR_NOMEM, "batch allocation");
  h->gravity = c->P.sun_gravity;
  h->device = c->device;
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, off[nbox] * sizeof(double));
  if (e != cudaSuccess) {
    delete h;
    return cudaFail(e, "batch scratch");
  }
  h->scratch = static_cast<double*>(p);
  std::vector<O4Args> args(nbox);
  for (int b = 0; b < nbox; ++b) {
    const hc_box& B = boxes[b].box;
    O4Args& a = args[b];
    a = O4Args{};
    a.G = c->o4;
    a.nbox = 1;
    a.block0 = B.block;
    a.ghost = kO4Ghost;
    for (int d = 0; d < 3; ++d) {
      a.vlo[d] = B.lo[d];
      a.vhi[d] = B.hi[d];
      a.ur.lo[d] = B.lo[d] - B.ghost;
      a.ur.n[d] = B.hi[d] - B.lo[d] + 1 + 2 * B.ghost;
      a.flux[d] = boxes[b].flux[d];
    }
    a.ur.N = (long)a.ur.n[0] * a.ur.n[1] * a.ur.n[2];
    a.U = boxes[b].usph;
    a.uStride = 8 * a.ur.N;
    a.scale = scale;
    a.rhs = boxes[b].rhs;
    a.rhsStride = 8L * (B.hi[0] - B.lo[0] + 1) * (B.hi[1] - B.lo[1] + 1) * (B.hi[2] - B.lo[2] + 1);
    carveO4Scratch(a, h->scratch + off[b]);
  }
  h->batch = o4BatchCreate(args.data(), nbox, &e);
  if (!h->batch) {
    cudaFree(h->scratch);
    delete h;
    return cudaFail(e, "batch contexts");
  }
  *out = h;
  return HC_OK;
}

int hc_o4_batch_rhs(hc_ctx* c, hc_o4_batch* h, void* stream) {
  if (!c || !h) return fail(HC_ERR_ARG, "null argument");
  cudaStream_t s = (cudaStream_t)stream;
  if (h->gravity) {
    const int rc = checkLaunch(launchO4BatchGravity(h->batch, s), "batch gravity");
    if (rc != HC_OK) return rc;
  }
  o4BatchSetVariants(h->batch, c->o4var);
  return checkLaunch(launchO4Batch(h->batch, nullptr, s), "batch operator");
}

int hc_o4_batch_destroy(hc_o4_batch* h) {
  if (!h) return HC_OK;
  cudaSetDevice(h->device);
  o4BatchDestroy(h->batch);
  if (h->scratch) cudaFree(h->scratch);
  delete h;
  return HC_OK;
}

int hc_box_gravity_o4(hc_ctx* c, const hc_box* box, const double* usph, double* rhs, void* stream) {
  if (!c || !box || !usph || !rhs) return fail(HC_ERR_ARG, "null argument");
  if (c->P.spatial_order != 4) return fail(HC_ERR_UNSUPPORTED, "context was created with spatial_order != 4");
  const hc_box& B = *box;
  if (B.block < 0 || B.block > 5) return fail(HC_ERR_ARG, "block must be 0..5");
  if (B.ghost < 1) return fail(HC_ERR_ARG, "Gravity_Euler needs ghost >= 1");
  const int n[3] = {c->P.nr, c->P.na, c->P.na};
  for (int d = 0; d < 3; ++d)
    if (B.lo[d] < 0 || B.hi[d] >= n[d] || B.hi[d] < B.lo[d]) return fail(HC_ERR_ARG, "box outside the panel");
  O4Args a{};
  a.G = c->o4;
  a.nbox = 1;
  a.block0 = B.block;
  a.ghost = B.ghost;
  for (int d = 0; d < 3; ++d) { a.vlo[d] = B.lo[d]; a.vhi[d] = B.hi[d]; }
  a.U = usph;
  for (int d = 0; d < 3; ++d) { a.ur.lo[d] = B.lo[d] - B.ghost; a.ur.n[d] = B.hi[d] - B.lo[d] + 1 + 2 * B.ghost; }
  a.ur.N = (long)a.ur.n[0] * a.ur.n[1] * a.ur.n[2];
  a.uStride = 8 * a.ur.N;
  a.rhs = rhs;
  a.rhsStride = 8L * (B.hi[0] - B.lo[0] + 1) * (B.hi[1] - B.lo[1] + 1) * (B.hi[2] - B.lo[2] + 1);
  int rc = HC_OK;
  O4Batch* Bt = cachedBatch(c, a, &rc);
  if (!Bt) return rc;
  return checkLaunch(launchO4BatchGravity(Bt, (cudaStream_t)stream), "hc_box_gravity_o4");
}

int hc_box_gravity(hc_ctx* c, const hc_box* box, const double* w, double* rhs, void* stream) {
  if (!c || !box || !w || !rhs) return fail(HC_ERR_ARG, "null argument");
  const hc_box& B = *box;
  if (B.block < 0 || B.block > 5) return fail(HC_ERR_ARG, "block must be 0..5");
  const int n[3] = {c->P.nr, c->P.na, c->P.na};
  int wlo[3], wn[3];
  for (int d = 0; d < 3; ++d) {
    if (B.lo[d] < 0 || B.hi[d] >= n[d] || B.hi[d] < B.lo[d]) return fail(HC_ERR_ARG, "box outside the panel");
    wlo[d] = B.lo[d] - B.ghost;
    wn[d] = B.hi[d] - B.lo[d] + 1 + 2 * B.ghost;
  }
  return checkLaunch(launchBoxGravity(c->L, B.lo, B.hi, B.block, w, wlo, wn, rhs, (cudaStream_t)stream), "hc_box_gravity");
}

int hc_level_prepare(hc_ctx* c, const double* ju, double* w, double t, void* stream) {
  if (!c || !ju || !w) return fail(HC_ERR_ARG, "null argument");
  cudaStream_t s = (cudaStream_t)stream;
  if (c->P.spatial_order == 4) {
    const int rc4 = ensureO4Buffers(c);
    if (rc4 != HC_OK) return rc4;
    O4StageIO io{c->o4l, ju, c->o4cart, w, c->o4pv, StageTime{t, nullptr, 0.0, nullptr, 0.0}};
    return checkLaunch(launchO4Prepare(io, s), "O4 prepare");
  }
  int rc = checkLaunch(launchPrimValid(c->L, ju, w, s), "prim");
  if (rc != HC_OK) return rc;
  StageTime st{t, nullptr, 0.0, nullptr, 0.0};
  return checkLaunch(launchGhosts(c->L, w, st, s), "ghosts");
}

size_t hc_level_cartesian_size(const hc_ctx* c) {
  return c && c->P.spatial_order == 4 ? (size_t)6 * NC * c->o4l.Nc : 0;
}

int hc_level_prepare_cartesian(hc_ctx* c, const double* ju, double* w, double* cart, double t, void* stream) {
  if (!c || !ju || !w || !cart) return fail(HC_ERR_ARG, "null argument");
  if (c->P.spatial_order != 4) return fail(HC_ERR_UNSUPPORTED, "context was created with spatial_order != 4");
  const int rc4 = ensureO4Buffers(c);
  if (rc4 != HC_OK) return rc4;
  O4StageIO io{c->o4l, ju, cart, w, c->o4pv, StageTime{t, nullptr, 0.0, nullptr, 0.0}};
  return checkLaunch(launchO4Prepare(io, (cudaStream_t)stream), "O4 prepare");
}

int hc_level_rhs_fluxes(hc_ctx* c, const double* w, double* k, double* const* flux, void* stream) {
  if (!c || !w || !k) return fail(HC_ERR_ARG, "null argument");
  if (c->P.spatial_order != 4) return fail(HC_ERR_UNSUPPORTED, "context was created with spatial_order != 4");
  cudaStream_t s = (cudaStream_t)stream;
  int rc = ensureO4Buffers(c);
  if (rc != HC_OK) return rc;
  O4Args args = levelO4Args(c, w, k);
  for (int d = 0; d < 3; ++d) args.flux[d] = flux ? flux[d] : nullptr;
  O4Batch* B = cachedBatch(c, args, &rc);
  if (!B) return rc;
  const O4Level& O = c->o4l;
  rc = checkLaunch(cudaMemsetAsync(k, 0, sizeof(double) * 6 * NC * O.Nv, s), "O4 k");
  if (rc == HC_OK)
    rc = checkLaunch(cudaMemsetAsync(c->o4reg, 0, sizeof(double) * 6 * 2 * 2 * 8 * O.na * O.nr, s), "register");
  if (rc == HC_OK && c->P.sun_gravity) rc = checkLaunch(launchO4BatchGravity(B, s), "O4 gravity");
  if (rc != HC_OK) return rc;
  // this evaluation's seam fluxes (weight 1) into the register, then each
  // seam face's rhs takes the mean of both panels' fluxes
  const RegArgs rg{c->o4reg, 1.0, nullptr, c->P.cfl};
  o4BatchSetVariants(B, c->o4var);
  rc = checkLaunch(launchO4Batch(B, &rg, s), "O4 operator");
  if (rc == HC_OK) rc = checkLaunch(launchO4Reflux(O, c->L, c->o4reg, k, s), "O4 seam reconciliation");
  return rc;
}

int hc_level_rhs(hc_ctx* c, const double* w, double* k, void* stream) {
  if (!c || !w || !k) return fail(HC_ERR_ARG, "null argument");
  if (c->P.spatial_order == 4) {
    cudaStream_t s = (cudaStream_t)stream;
    int rc = ensureO4Buffers(c);
    if (rc != HC_OK) return rc;
    O4Batch* B = (w == c->o4us && k == c->o4k && c->winHi == 0) ? c->o4levelBatch
                                                                 : cachedBatch(c, levelO4Args(c, w, k), &rc);
    if (!B) return rc;
    rc = checkLaunch(cudaMemsetAsync(k, 0, sizeof(double) * 6 * NC * c->o4l.Nv, s), "O4 k");
    if (rc == HC_OK && c->P.sun_gravity) rc = checkLaunch(launchO4BatchGravity(B, s), "O4 gravity");
    if (rc != HC_OK) return rc;
    o4BatchSetVariants(B, c->o4var);
    return checkLaunch(launchO4Batch(B, nullptr, s), "O4 operator");
  }
  StageArgs a = levelArgs(c, w);
  a.rhs = k;
  return checkLaunch(launchStage(a, MODE_RHS, c->P.limiter, c->P.riemann_solver == 2, c->P.divergence_cleaning == 1,
                                 c->P.sun_gravity == 1, (cudaStream_t)stream, c->tileRHS),
                     "hc_level_rhs");
}

}  // extern "C"

namespace {

// Tiles chosen per device, level size and scheme, shared by the contexts of
// the process (a served ensemble creates many contexts of a few shapes).
std::mutex g_tileMutex;
std::map<std::string, std::pair<int, int>> g_tileCache;

std::string tileKey(const hc_ctx* c) {
  const hc_params& P = c->P;
  char key[160];
  std::snprintf(key, sizeof key, "%d:%d:%d:%d:%d:%d:%d", c->device, P.nr, P.na, P.limiter == 0 ? 0 : P.limiter == 3 ? 3 : 1,
                P.riemann_solver == 2 ? 1 : 0, P.divergence_cleaning == 1 ? 1 : 0, P.sun_gravity == 1 ? 1 : 0);
  return key;
}

// Median launch time (ms) of `launch` over `reps` launches after 2 warm-ups.
template <class F>
int timeLaunches(F launch, cudaStream_t s, int reps, double* ms) {
  cudaEvent_t e[2 * 16];
  reps = std::min(reps, 16);
  for (int i = 0; i < 2 * reps; ++i)
    if (cudaEventCreate(&e[i]) != cudaSuccess) {
      for (int j = 0; j < i; ++j) cudaEventDestroy(e[j]);
      return cudaFail(cudaGetLastError(), "autotune events");
    }
  int rc = HC_OK;
  for (int i = 0; i < 2 && rc == HC_OK; ++i) rc = launch();
  for (int i = 0; i < reps && rc == HC_OK; ++i) {
    cudaEventRecord(e[2 * i], s);
    rc = launch();
    cudaEventRecord(e[2 * i + 1], s);
  }
  if (rc == HC_OK) rc = checkLaunch(cudaStreamSynchronize(s), "autotune sync");
  std::vector<float> t;
  for (int i = 0; i < reps && rc == HC_OK; ++i) {
    float v = 0;
    rc = checkLaunch(cudaEventElapsedTime(&v, e[2 * i], e[2 * i + 1]), "autotune timing");
    t.push_back(v);
  }
  for (int i = 0; i < 2 * reps; ++i) cudaEventDestroy(e[i]);
  if (rc != HC_OK) return rc;
  std::sort(t.begin(), t.end());
  *ms = t[t.size() / 2];
  return HC_OK;
}

int autotuneStage(hc_ctx* c, const double* ju, cudaStream_t s, int* tilesOut, double* msOut) {
  const bool roe = c->P.riemann_solver == 2, powell = c->P.divergence_cleaning == 1, grav = c->P.sun_gravity == 1;
  // primitives of ju with ghosts in W[0]; the timed launches write only the
  // workspace (W[1], acc), never ju
  int rc = checkLaunch(launchPrimValid(c->L, ju, c->W[0], s), "autotune prim");
  StageTime st{0.0, nullptr, 0.0, nullptr, 0.0};
  if (rc == HC_OK) rc = checkLaunch(launchGhosts(c->L, c->W[0], st, s), "autotune ghosts");
  double best[2] = {1e300, 1e300};
  int pick[2] = {0, 0};
  for (int mode = 0; mode < 2 && rc == HC_OK; ++mode)
    for (int t = 0; t < kStageTiles && rc == HC_OK; ++t) {
      StageArgs a = levelArgs(c, c->W[0]);
      if (mode == 0) {
        a.stage = 0;  // reads ju, writes acc and the next stage's primitives
        a.invDtMax = nullptr;
        a.dtv = 0.0;
        a.ju = const_cast<double*>(ju);
        a.acc = c->acc;
        a.wOut = c->W[1];
        a.invMaxOut = nullptr;
        a.invalid = nullptr;
      } else {
        a.rhs = c->acc;
      }
      double ms = 0;
      rc = timeLaunches(
          [&]() {
            return checkLaunch(launchStage(a, mode == 0 ? MODE_RK : MODE_RHS, c->P.limiter, roe, powell, grav, s, t),
                               "autotune launch");
          },
          s, 7, &ms);
      if (rc != HC_OK) break;
      if (msOut) msOut[mode * kStageTiles + t] = ms;
      if (ms < best[mode]) { best[mode] = ms; pick[mode] = t; }
    }
  if (rc != HC_OK) return rc;
  c->tileRK = pick[0];
  c->tileRHS = pick[1];
  c->tuned = true;
  {
    std::lock_guard<std::mutex> lock(g_tileMutex);
    g_tileCache[tileKey(c)] = {pick[0], pick[1]};
  }
  if (tilesOut) { tilesOut[0] = pick[0]; tilesOut[1] = pick[1]; }
  return HC_OK;
}

std::map<std::string, std::vector<int>> g_o4Cache;

std::string o4Key(const hc_ctx* c) {
  const hc_params& P = c->P;
  char key[160];
  std::snprintf(key, sizeof key, "o4:%d:%d:%d:%d:%d:%d:%d", c->device, P.nr, P.na, P.riemann_solver == 2 ? 1 : 0,
                P.divergence_cleaning == 1 ? 1 : 0, P.sun_gravity == 1 ? 1 : 0, P.berta_fallback_type);
  return key;
}

// Fourth order: the state's stage preparation into the level workspace, then
// the level operator timed for each register-cap variant of one tuned kernel
// at a time, the others held at the best found so far (coordinate descent
// over reconstruction, Roe point dissipation, final flux).
int autotuneO4(hc_ctx* c, const double* ju, cudaStream_t s, int* tilesOut, double* msOut) {
  int rc = ensureO4Buffers(c);
  if (rc != HC_OK) return rc;
  O4StageIO io{c->o4l, ju, c->o4cart, c->o4us, c->o4pv, StageTime{0.0, nullptr, 0.0, nullptr, 0.0}};
  rc = checkLaunch(launchO4Prepare(io, s), "autotune O4 prepare");
  int best[kO4TunedKernels] = {0, 0, 0};
  for (int q = 0; q < kO4TunedKernels && rc == HC_OK; ++q) {
    if (q == 1 && c->P.riemann_solver != 2) {  // no Roe point kernel with Rusanov
      for (int v = 0; v < kO4Variants && msOut; ++v) msOut[q * kO4Variants + v] = 0.0;
      continue;
    }
    double bestMs = 1e300;
    for (int v = 0; v < kO4Variants && rc == HC_OK; ++v) {
      int var[kO4TunedKernels] = {best[0], best[1], best[2]};
      var[q] = v;
      o4BatchSetVariants(c->o4levelBatch, var);
      double ms = 0;
      rc = timeLaunches([&]() { return checkLaunch(launchO4Batch(c->o4levelBatch, nullptr, s), "autotune O4"); }, s, 5,
                        &ms);
      if (rc != HC_OK) break;
      if (msOut) msOut[q * kO4Variants + v] = ms;
      if (ms < bestMs) { bestMs = ms; best[q] = v; }
    }
  }
  o4BatchSetVariants(c->o4levelBatch, c->o4var);
  if (rc != HC_OK) return rc;
  for (int q = 0; q < kO4TunedKernels; ++q) c->o4var[q] = best[q];
  c->tuned = true;
  {
    std::lock_guard<std::mutex> lock(g_tileMutex);
    g_o4Cache[o4Key(c)] = std::vector<int>(best, best + kO4TunedKernels);
  }
  if (tilesOut)
    for (int q = 0; q < kO4TunedKernels; ++q) tilesOut[q] = best[q];
  return HC_OK;
}

// With hc_params.autotune set: take a cached choice, or time the candidates
// once (outside stream capture only; a capturing stream keeps the current
// choice).
int maybeAutotune(hc_ctx* c, const double* ju, cudaStream_t s) {
  if (!c->P.autotune || c->tuned) return HC_OK;
  {
    std::lock_guard<std::mutex> lock(g_tileMutex);
    if (c->P.spatial_order == 2) {
      auto it = g_tileCache.find(tileKey(c));
      if (it != g_tileCache.end()) {
        c->tileRK = it->second.first;
        c->tileRHS = it->second.second;
        c->tuned = true;
        return HC_OK;
      }
    } else {
      auto it = g_o4Cache.find(o4Key(c));
      if (it != g_o4Cache.end()) {
        for (int q = 0; q < kO4TunedKernels; ++q) c->o4var[q] = it->second[q];
        c->tuned = true;
        return HC_OK;
      }
    }
  }
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return HC_OK;
  return c->P.spatial_order == 2 ? autotuneStage(c, ju, s, nullptr, nullptr) : autotuneO4(c, ju, s, nullptr, nullptr);
}

// One CFL step of every member of an ensemble: the per-level sequence of
// hc_level_advance_cfl (dtCFL, insertion schedule, four stages, seam
// reconciliation, time) with the operator of each stage batched.
int ensembleFork(hc_ensemble* E, cudaStream_t s) {
  cudaError_t e = cudaEventRecord(E->forkEv, s);
  for (size_t l = 0; l < E->lanes.size() && e == cudaSuccess; ++l) e = cudaStreamWaitEvent(E->lanes[l], E->forkEv, 0);
  return checkLaunch(e, "ensemble fork");
}

int ensembleJoin(hc_ensemble* E, cudaStream_t s) {
  cudaError_t e = cudaSuccess;
  for (size_t l = 0; l < E->lanes.size() && e == cudaSuccess; ++l) {
    e = cudaEventRecord(E->joinEv[l], E->lanes[l]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s, E->joinEv[l], 0);
  }
  return checkLaunch(e, "ensemble join");
}

int ensembleStep(hc_ensemble* E, double* const* ju, double* const* time, double* const* dtOut, cudaStream_t s) {
  static const double c4[4] = {0, 0.5, 0.5, 1}, b4[4] = {1.0 / 6, 1.0 / 3, 1.0 / 3, 1.0 / 6};
  const int m = (int)E->members.size();
  auto invMaxOf = [](const hc_ctx* c) { return reinterpret_cast<const double*>(c->invMax); };
  auto lane = [E](int q) { return E->lanes[q % E->lanes.size()]; };
  int rc = ensembleFork(E, s);
  for (int q = 0; q < m && rc == HC_OK; ++q) {
    hc_ctx* c = E->members[q];
    double* tq = time ? time[q] : nullptr;
    rc = checkLaunch(launchCfl(c->L, ju[q], c->invMax, lane(q)), "cfl");
    if (rc == HC_OK && c->sched && tq)
      rc = checkLaunch(launchCmeSchedule(c->sched, c->invMax, tq, c->rusanovFlag, lane(q)), "CME schedule");
    if (rc == HC_OK)
      rc = checkLaunch(
          cudaMemsetAsync(c->o4reg, 0, sizeof(double) * 6 * 2 * 2 * 8 * c->o4l.na * c->o4l.nr, lane(q)), "register");
  }
  for (int stage = 0; stage < 4 && rc == HC_OK; ++stage) {
    for (int q = 0; q < m && rc == HC_OK; ++q) {
      hc_ctx* c = E->members[q];
      const O4StageIO io{c->o4l, stage == 0 ? ju[q] : c->o4next, c->o4cart, c->o4us, c->o4pv,
                         StageTime{0.0, time ? time[q] : nullptr, c4[stage], invMaxOf(c), 0.0}};
      rc = checkLaunch(launchO4Prepare(io, lane(q)), "O4 prepare");
      if (rc == HC_OK)
        rc = checkLaunch(cudaMemsetAsync(c->o4k, 0, sizeof(double) * 6 * 8 * c->o4l.Nv, lane(q)), "O4 k");
    }
    if (rc == HC_OK) rc = ensembleJoin(E, s);
    if (rc == HC_OK && E->gravity) rc = checkLaunch(launchO4BatchGravity(E->batch, s), "O4 gravity");
    if (rc != HC_OK) break;
    const RegArgs rg{nullptr, b4[stage], nullptr, 0.0};  // each box carries its level's register
    o4BatchSetVariants(E->batch, E->members[0]->o4var);
    rc = checkLaunch(launchO4Batch(E->batch, &rg, s), "O4 operator");
    if (rc == HC_OK) rc = ensembleFork(E, s);
    for (int q = 0; q < m && rc == HC_OK; ++q) {
      hc_ctx* c = E->members[q];
      rc = checkLaunch(
          launchO4Update(c->o4l, stage, c->o4k, ju[q], c->acc, c->o4next, invMaxOf(c), c->P.cfl, 0.0, lane(q)),
          "O4 update");
    }
  }
  for (int q = 0; q < m && rc == HC_OK; ++q) {
    hc_ctx* c = E->members[q];
    rc = checkLaunch(launchO4Reflux(c->o4l, c->L, c->o4reg, ju[q], lane(q)), "O4 reflux");
    if (rc == HC_OK)
      rc = checkLaunch(
          launchAdvanceTime(time ? time[q] : nullptr, invMaxOf(c), c->P.cfl, dtOut ? dtOut[q] : nullptr, lane(q)),
          "time");
  }
  // the lanes always end joined to the caller's stream (a capture must end so)
  const int rj = ensembleJoin(E, s);
  return rc != HC_OK ? rc : rj;
}

}  // namespace

extern "C" {

int hc_ensemble_create(hc_ctx* const* members, int m, hc_ensemble** out) {
  if (!members || m <= 0 || !out) return fail(HC_ERR_ARG, "bad argument");
  *out = nullptr;
  if (m > 65535 / 6) return fail(HC_ERR_ARG, "at most 10922 levels per ensemble");
  const hc_ctx* c0 = members[0];
  if (!c0) return fail(HC_ERR_ARG, "null member");
  for (int q = 0; q < m; ++q) {
    const hc_ctx* c = members[q];
    if (!c) return fail(HC_ERR_ARG, "null member");
    if (c->P.spatial_order != 4) return fail(HC_ERR_UNSUPPORTED, "ensembles batch fourth-order levels only");
    if (c->device != c0->device) return fail(HC_ERR_ARG, "ensemble members on different devices");
    if (c->P.riemann_solver != c0->P.riemann_solver || c->P.divergence_cleaning != c0->P.divergence_cleaning ||
        c->P.sun_gravity != c0->P.sun_gravity || c->P.berta_fallback_type != c0->P.berta_fallback_type)
      return fail(HC_ERR_ARG, "ensemble members must share the Riemann solver, Powell, gravity and fallback");
    for (int r = 0; r < q; ++r)
      if (members[r] == c) return fail(HC_ERR_ARG, "a level appears twice in the ensemble");
  }
  std::vector<O4Args> boxes;
  for (int q = 0; q < m; ++q) {
    hc_ctx* c = members[q];
    const int rc = ensureO4Buffers(c);
    if (rc != HC_OK) return rc;
    std::vector<O4Args> own;
    o4SplitArgs(levelO4Args(c, c->o4us, c->o4k), own);
    for (O4Args& a : own) {
      a.seamReg = c->o4reg;
      a.seamInvMax = reinterpret_cast<const double*>(c->invMax);
      a.seamCfl = c->P.cfl;
      boxes.push_back(a);
    }
  }
  hc_ensemble* E = new (std::nothrow) hc_ensemble;
  if (!E) return fail(HC_ERR_NOMEM, "ensemble allocation");
  E->members.assign(members, members + m);
  E->gravity = c0->P.sun_gravity;
  E->device = c0->device;
  cudaError_t e = cudaSuccess;
  E->batch = o4BatchCreate(boxes.data(), (int)boxes.size(), &e);
  const int nl = m < 4 ? m : 4;
  if (E->batch) e = cudaEventCreateWithFlags(&E->forkEv, cudaEventDisableTiming);
  for (int l = 0; l < nl && e == cudaSuccess; ++l) {
    cudaStream_t st = nullptr;
    cudaEvent_t ev = nullptr;
    e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e == cudaSuccess) E->lanes.push_back(st);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e == cudaSuccess) E->joinEv.push_back(ev);
  }
  if (!E->batch || e != cudaSuccess) {
    hc_ensemble_destroy(E);
    return cudaFail(e, "ensemble batch");
  }
  *out = E;
  return HC_OK;
}

int hc_ensemble_advance_cfl(hc_ensemble* E, double* const* ju, int nsteps, double* const* time_dev,
                            double* const* dt_dev, void* stream) {
  if (!E || !ju || nsteps < 0) return fail(HC_ERR_ARG, "bad argument");
  for (size_t q = 0; q < E->members.size(); ++q)
    if (!ju[q]) return fail(HC_ERR_ARG, "null state");
  cudaStream_t s = (cudaStream_t)stream;
  int rc = HC_OK;
  for (int n = 0; n < nsteps && rc == HC_OK; ++n) rc = ensembleStep(E, ju, time_dev, dt_dev, s);
  return rc;
}

int hc_ensemble_destroy(hc_ensemble* E) {
  if (!E) return HC_OK;
  cudaSetDevice(E->device);
  for (cudaStream_t st : E->lanes) cudaStreamSynchronize(st);
  if (E->batch) o4BatchDestroy(E->batch);
  for (cudaStream_t st : E->lanes) cudaStreamDestroy(st);
  for (cudaEvent_t ev : E->joinEv) cudaEventDestroy(ev);
  if (E->forkEv) cudaEventDestroy(E->forkEv);
  delete E;
  return HC_OK;
}

int hc_cone_event(const hc_cone* cone, hc_cme_event* out) {
  if (!cone || !out) return fail(HC_ERR_ARG, "null argument");
  // a finite cloud feeds through the inner boundary while it crosses it
  // (src/MHD_CME.H:1251-1253): boundary source iff it ends after insertion
  std::memset(out, 0, sizeof *out);
  out->insertion_time = cone->insertion_time;
  out->boundary = cone->end_time > cone->insertion_time ? 1 : 0;
  out->feeding_end = std::max(cone->insertion_time, cone->end_time);
  return HC_OK;
}

int hc_level_set_cme_schedule(hc_ctx* c, const hc_cme_event* events, int n, void* stream) {
  if (!c || (n && !events)) return fail(HC_ERR_ARG, "null argument");
  if (n < 0 || n > kCmeEvents) return fail(HC_ERR_ARG, "at most 8 CME events");
  if (n && isSlab(c->P))
    return fail(HC_ERR_UNSUPPORTED, "CME schedules steer the whole shell's dt: not on a radial slab");
  for (int i = 1; i < n; ++i)
    if (events[i].insertion_time < events[i - 1].insertion_time)
      return fail(HC_ERR_ARG, "CME events must be ordered by insertion time");
  CmeSchedule& h = c->schedHost;
  h.n = n;
  h.roe = c->P.riemann_solver == 2 ? 1 : 0;
  h.cfl = c->P.cfl;
  h.feeding = c->P.riemann_solver == 2 ? .5 : 1.;
  for (int i = 0; i < n; ++i) {
    const hc_cme_event& e = events[i];
    h.t[i] = e.insertion_time;
    h.boundary[i] = e.boundary ? 1 : 0;
    // stabilizationEnd, src/MHD_CME.H:1329-1332
    h.stabEnd[i] = e.boundary ? std::max(e.feeding_end + 600, e.insertion_time + 2400) : e.insertion_time + 600;
  }
  cudaStream_t s = (cudaStream_t)stream;
  if (!c->rusanovFlag) {  // order 2 (order 4 allocates it with its geometry)
    cudaError_t err = cudaMalloc(&c->rusanovFlag, sizeof(int));
    if (err == cudaSuccess) err = cudaMemsetAsync(c->rusanovFlag, 0, sizeof(int), s);
    if (err != cudaSuccess) return cudaFail(err, "CME window flag");
    c->owned.push_back(c->rusanovFlag);
  }
  if (!c->sched) {
    cudaError_t err = cudaMalloc(&c->sched, sizeof(CmeSchedule));
    if (err != cudaSuccess) return cudaFail(err, "CME schedule");
    c->owned.push_back(c->sched);
  }
  // pageable source: the copy is staged before the call returns, then
  // ordered on the stream after the work already queued there
  cudaError_t err = cudaMemcpyAsync(c->sched, &h, sizeof h, cudaMemcpyHostToDevice, s);
  if (err == cudaSuccess && n == 0 && c->rusanovFlag) err = cudaMemsetAsync(c->rusanovFlag, 0, sizeof(int), s);
  if (err != cudaSuccess) return cudaFail(err, "CME schedule");
  c->schedEvents = n;
  return HC_OK;
}

int hc_level_set_inlet(hc_ctx* c, const hc_cone* cones, int n, void* stream) {
  if (!c || (n && !cones)) return fail(HC_ERR_ARG, "null argument");
  if (n < 0 || n > kInletCones) return fail(HC_ERR_ARG, "at most 8 inlet cones");
  if (n && isSlab(c->P))
    return fail(HC_ERR_UNSUPPORTED, "the boundary inlet enters the shell's CFL rate: not on a radial slab");
  if (n && c->P.spatial_order != 2) return fail(HC_ERR_UNSUPPORTED, "the boundary inlet is built for order-2 contexts");
  if (n && c->P.init_condition_type != 1) return fail(HC_ERR_UNSUPPORTED, "the inlet needs the analytic-wind inner boundary");
  InletCone h[kInletCones] = {};
  for (int i = 0; i < n; ++i) {
    const hc_cone& k = cones[i];
    if (!(k.radius > 0) || !(k.speed > 0) || !(k.density > 0) || !(k.temperature >= 0))
      return fail(HC_ERR_ARG, "inlet cone not prepared (radius, speed, density, temperature)");
    for (int d = 0; d < 3; ++d) h[i].axis[d] = k.axis[d];
    h[i].radius = k.radius;
    h[i].entryShift = k.entry_shift;
    h[i].entryTime = k.entry_time;
    h[i].speed = k.speed;
    h[i].endTime = k.end_time;
    h[i].insertionTime = k.insertion_time;
    h[i].density = k.density;
    h[i].temperature = k.temperature;
  }
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t err = cudaSuccess;
  if (!c->inletDev) {
    err = cudaMalloc(&c->inletDev, sizeof(InletCone) * kInletCones);
    if (err != cudaSuccess) return cudaFail(err, "inlet");
    c->owned.push_back(c->inletDev);
  }
  if (!c->sched) {
    err = cudaMalloc(&c->sched, sizeof(CmeSchedule));
    if (err != cudaSuccess) return cudaFail(err, "inlet schedule");
    c->owned.push_back(c->sched);
    c->schedHost = CmeSchedule{};
    c->schedHost.cfl = c->P.cfl;
    c->schedHost.feeding = c->P.riemann_solver == 2 ? .5 : 1.;
  }
  err = cudaMemcpyAsync(c->inletDev, h, sizeof h, cudaMemcpyHostToDevice, s);
  // the clouds' crossing rate in the step's CFL rate (exec/main.cpp:365-383)
  CmeSchedule& S = c->schedHost;
  S.ninlet = n;
  for (int i = 0; i < n; ++i) {
    S.inletT[i] = cones[i].insertion_time;
    S.inletEnd[i] = cones[i].end_time;
    S.inletSpeed[i] = cones[i].speed;
    S.inletTemp[i] = cones[i].temperature;
  }
  const double C = c->P.radial_stretch, span = c->P.outer_radius - c->P.inner_radius;
  const int cells = shellCells(c->P);
  S.width = span * (C == 0 ? 1. / cells : std::expm1(C / cells) / std::expm1(C));
  S.gamma = c->P.gamma;
  if (err == cudaSuccess) err = cudaMemcpyAsync(c->sched, &S, sizeof S, cudaMemcpyHostToDevice, s);
  if (err != cudaSuccess) return cudaFail(err, "inlet");
  c->L.inlet = n ? c->inletDev : nullptr;
  c->L.ninlet = n;
  return HC_OK;
}

int hc_stage_tiles(int* shapes, int capacity) {
  for (int t = 0; shapes && t < kStageTiles && t < capacity; ++t) stageTileShape(t, shapes + 5 * t);
  return kStageTiles;
}

int hc_ctx_autotune(hc_ctx* c, const double* ju, int* tiles, double* ms, void* stream) {
  if (!c || !ju) return fail(HC_ERR_ARG, "null argument");
  if (c->P.spatial_order == 4) return autotuneO4(c, ju, (cudaStream_t)stream, tiles, ms);
  return autotuneStage(c, ju, (cudaStream_t)stream, tiles, ms);
}

int hc_o4_variants(int* min_blocks, int capacity) {
  for (int q = 0; min_blocks && q < kO4TunedKernels; ++q)
    for (int v = 0; v < kO4Variants && q * kO4Variants + v < capacity; ++v)
      min_blocks[q * kO4Variants + v] = o4VariantMinBlocks(q, v);
  return kO4Variants;
}

int hc_ctx_set_o4_variants(hc_ctx* c, const int* variants) {
  if (!c || !variants) return fail(HC_ERR_ARG, "null argument");
  for (int q = 0; q < kO4TunedKernels; ++q)
    if (variants[q] < -1 || variants[q] >= kO4Variants) return fail(HC_ERR_ARG, "variant index out of range");
  for (int q = 0; q < kO4TunedKernels; ++q)
    if (variants[q] >= 0) c->o4var[q] = variants[q];
  c->tuned = true;
  return HC_OK;
}

int hc_ctx_set_tiles(hc_ctx* c, int tileRK, int tileRHS) {
  if (!c) return fail(HC_ERR_ARG, "null argument");
  if (tileRK < -1 || tileRK >= kStageTiles || tileRHS < -1 || tileRHS >= kStageTiles)
    return fail(HC_ERR_ARG, "tile index out of range");
  if (tileRK >= 0) c->tileRK = tileRK;
  if (tileRHS >= 0) c->tileRHS = tileRHS;
  c->tuned = true;
  return HC_OK;
}

int hc_level_rk4_step(hc_ctx* c, double* ju, double dt, double t, void* stream) {
  if (!c || !ju) return fail(HC_ERR_ARG, "null argument");
  if (!(dt > 0)) return fail(HC_ERR_ARG, "dt must be positive");
  cudaStream_t s = (cudaStream_t)stream;
  // the insertion schedule belongs to hc_level_advance_cfl: a fixed-dt step
  // runs the context's own solver
  if (c->sched && c->rusanovFlag) {
    const int rcf = checkLaunch(cudaMemsetAsync(c->rusanovFlag, 0, sizeof(int), s), "CME window flag");
    if (rcf != HC_OK) return rcf;
  }
  if (c->P.spatial_order == 4) {
    int rc4 = ensureO4Buffers(c);
    if (rc4 == HC_OK) rc4 = maybeAutotune(c, ju, s);
    return rc4 != HC_OK ? rc4 : o4Step(c, ju, dt, nullptr, t, nullptr, s);
  }
  int rc = maybeAutotune(c, ju, s);
  if (rc == HC_OK) rc = checkLaunch(launchPrimValid(c->L, ju, c->W[0], s), "prim");
  if (rc != HC_OK) return rc;
  return rkStep(c, ju, dt, nullptr, nullptr, t, nullptr, s);
}

int hc_level_rk4_stage(hc_ctx* c, double* ju, int stage, double dt, double t, const double* inv_dt_max,
                       const double* time_dev, void* stream) {
  if (!c || !ju) return fail(HC_ERR_ARG, "null argument");
  if (stage < 0 || stage > 3) return fail(HC_ERR_ARG, "stage must be 0..3");
  if (!inv_dt_max && !(dt > 0)) return fail(HC_ERR_ARG, "dt must be positive");
  cudaStream_t s = (cudaStream_t)stream;
  const double dtv = inv_dt_max ? 0.0 : dt;
  int rc = c->P.spatial_order == 4 ? ensureO4Buffers(c) : HC_OK;
  if (rc == HC_OK && stage == 0) {
    if (c->sched && c->rusanovFlag)
      rc = checkLaunch(cudaMemsetAsync(c->rusanovFlag, 0, sizeof(int), s), "CME window flag");
    if (rc == HC_OK) rc = maybeAutotune(c, ju, s);
    if (rc == HC_OK && c->P.spatial_order == 2) rc = checkLaunch(launchPrimValid(c->L, ju, c->W[0], s), "prim");
  }
  if (rc != HC_OK) return rc;
  if (c->P.spatial_order == 4) return o4Stage(c, ju, stage, dtv, inv_dt_max, t, time_dev, s);
  return rkStage(c, ju, stage, dtv, inv_dt_max, nullptr, t, time_dev, s);
}

int hc_level_set_radial_window(hc_ctx* c, int lo, int hi) {
  if (!c) return fail(HC_ERR_ARG, "null argument");
  if (c->P.spatial_order != 4) return fail(HC_ERR_UNSUPPORTED, "the radial window is built for order-4 contexts");
  if (!(lo == 0 && hi == 0) && !(0 <= lo && lo < hi && hi <= c->P.nr))
    return fail(HC_ERR_ARG, "the radial window needs 0 <= lo < hi <= nr (or 0, 0 for every cell)");
  if (lo == 0 && hi == c->P.nr) hi = 0;
  if (c->winLo == lo && c->winHi == hi) return HC_OK;
  c->winLo = lo;
  c->winHi = hi;
  if (c->o4levelBatch) {
    // the batch's device tables are freed after the device has finished
    // the work already queued on them
    const cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cudaFail(e, "radial window");
    o4BatchDestroy(c->o4levelBatch);
    c->o4levelBatch = nullptr;
  }
  return HC_OK;
}

int hc_level_stage_state(hc_ctx* c, double* ju, int stage, double** data, long* rows, int* row_length, int* first) {
  if (!c || !ju || !data || !rows || !row_length || !first) return fail(HC_ERR_ARG, "null argument");
  if (stage < 0 || stage > 3) return fail(HC_ERR_ARG, "stage must be 0..3");
  const int nr = c->P.nr, na = c->P.na;
  if (stage == 0 || c->P.spatial_order == 4) {
    if (stage > 0) {
      const int rc = ensureO4Buffers(c);
      if (rc != HC_OK) return rc;
    }
    *data = stage == 0 ? ju : c->o4next;
    *rows = 6L * 8 * na * na;
    *row_length = nr;
    *first = 0;
    return HC_OK;
  }
  *data = c->W[stage % 2];
  *rows = 6L * 8 * c->L.n1 * c->L.n1;
  *row_length = c->L.n0;
  *first = c->L.g;
  return HC_OK;
}

int hc_level_advance_cfl(hc_ctx* c, double* ju, int nsteps, double* time_dev, double* dt_dev, void* stream) {
  if (!c || !ju || nsteps < 0) return fail(HC_ERR_ARG, "bad argument");
  if (nsteps == 0) return HC_OK;
  cudaStream_t s = (cudaStream_t)stream;
  if (c->P.spatial_order == 4) {
    // dtCFL of the state at the start of each step, then the step.
    int rc = ensureO4Buffers(c);
    if (rc == HC_OK) rc = maybeAutotune(c, ju, s);
    const double* invMax = reinterpret_cast<const double*>(c->invMax);
    for (int n = 0; n < nsteps && rc == HC_OK; ++n) {
      rc = checkLaunch(launchCfl(c->L, ju, c->invMax, s), "cfl");
      if (rc == HC_OK && c->sched && time_dev)
        rc = checkLaunch(launchCmeSchedule(c->sched, c->invMax, time_dev, c->rusanovFlag, s), "CME schedule");
      if (rc == HC_OK) rc = o4Step(c, ju, 0.0, invMax, 0.0, time_dev, s);
      if (rc == HC_OK) rc = checkLaunch(launchAdvanceTime(time_dev, invMax, c->P.cfl, dt_dev, s), "time");
    }
    return rc;
  }
  // The first step's primitives and CFL rate come from ju; every later
  // step's come from the previous step's last stage.
  int rc = maybeAutotune(c, ju, s);
  if (rc == HC_OK) rc = checkLaunch(launchPrimValid(c->L, ju, c->W[0], s), "prim");
  if (rc == HC_OK) rc = checkLaunch(launchCfl(c->L, ju, c->invMax, s, time_dev), "cfl");
  for (int n = 0; n < nsteps && rc == HC_OK; ++n) {
    const int cur = n % 2;
    unsigned long long* next = c->invMax + (1 - cur);
    const double* invMax = reinterpret_cast<const double*>(c->invMax + cur);
    rc = checkLaunch(cudaMemsetAsync(next, 0, sizeof(unsigned long long), s), "cfl reset");
    if (rc == HC_OK && c->sched && time_dev)
      rc = checkLaunch(launchCmeSchedule(c->sched, c->invMax + cur, time_dev, c->rusanovFlag, s), "CME schedule");
    if (rc == HC_OK) rc = rkStep(c, ju, 0.0, invMax, n + 1 < nsteps ? next : nullptr, 0.0, time_dev, s);
    if (rc == HC_OK) rc = checkLaunch(launchAdvanceTime(time_dev, invMax, c->P.cfl, dt_dev, s), "time");
  }
  return rc;
}

int hc_level_dt_cfl(hc_ctx* c, const double* ju, double* inv_dt_max, void* stream) {
  if (!c || !ju || !inv_dt_max) return fail(HC_ERR_ARG, "null argument");
  cudaStream_t s = (cudaStream_t)stream;
  int rc = checkLaunch(launchCfl(c->L, ju, c->invMax, s), "cfl");
  if (rc != HC_OK) return rc;
  return checkLaunch(launchBitsToDouble(c->invMax, inv_dt_max, s), "cfl copy");
}

int hc_level_valid(hc_ctx* c, const double* ju, int* ok, void* stream) {
  if (!c || !ju || !ok) return fail(HC_ERR_ARG, "null argument");
  return checkLaunch(launchValid(c->L, ju, ok, (cudaStream_t)stream), "valid");
}

int hc_level_init(hc_ctx* c, const hc_init* in, double* ju, void* stream) {
  if (!c || !in || !ju) return fail(HC_ERR_ARG, "null argument");
  if (in->kind != 1) return fail(HC_ERR_UNSUPPORTED, "init kind must be 1");
  if (in->pulse_block < 0 || in->pulse_block > 5) return fail(HC_ERR_ARG, "pulse_block must be 0..5");
  struct InitArgsHost {
    int kind, pb, pi, pj, pk;
    double rho0, p0, vr, b0, r_ref, amp, width;
    double cx[3];
  } a;
  a.kind = in->kind; a.pb = in->pulse_block; a.pi = in->pulse_i; a.pj = in->pulse_j; a.pk = in->pulse_k;
  a.rho0 = in->rho0; a.p0 = in->p0; a.vr = in->vr; a.b0 = in->b0; a.r_ref = in->r_ref;
  a.amp = in->pulse_amp; a.width = in->pulse_width;
  const double h = 1.0 / c->P.na;
  double A[3][3];
  basisAt(in->pulse_block, (in->pulse_j + 0.5) * h, (in->pulse_k + 0.5) * h, A, a.cx);
  return checkLaunch(launchInit(c->L, &a, ju, (cudaStream_t)stream), "init");
}

long hc_geometry_export(const hc_ctx* c, int what, double* out) {
  if (!c) return -1;
  const std::vector<double>* v = nullptr;
  if (what == 0) v = &c->radialExport;
  else if (what >= 1 && what <= 3) v = &c->normalExport[what - 1];
  else if (what == 4) v = &c->detExport;
  else if (what == 5) v = &c->detAAExport;
  else return -1;
  if (out) std::memcpy(out, v->data(), v->size() * sizeof(double));
  return (long)v->size();
}

}  // extern "C"

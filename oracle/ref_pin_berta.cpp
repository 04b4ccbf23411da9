// ORACLE PIN -- test infrastructure only.
//
// Exposes the reference's own fourth-order pointwise kernels, compiled
// unchanged from the text the build recipe (oracle/build.py) reads out of
// src/BoxOp_BertaCubedSphereImplem.H and src/BoxOp_EulerCubedSphere.H into
// oracle/_ref/berta_kernels.inc.  Those files' other functions need Proto's
// BoxData; these kernels touch their arguments only through Proto's Var
// element accessor, stubbed below:
//   f_wenoz_pointwise_faceF, bertaNormalizeWenoStencil   (WENOZ5 face states)
//   f_weno3_pointwise_faceF, f_plm_pointwise_faceF       (fallbacks)
//   f_berta_jameson_theta_rawF                           (detector flag)
//   f_berta_avg_to_point_thetaF, f_flux_point_to_avg_thetaF
//   f_select_reconstructionF                             (choice + clamp)
//   bertaMappedLine                                      (mapped-flux sums)
//   f_sphToPrim_F, f_primflux_F                          (point primitives, flux)
// tests/test_oracle_pin_berta.py requires the oracle's restatement to give
// the same bits.

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <limits>
#include <sys/types.h>

using std::abs;
using std::max;
using std::min;
using std::sqrt;

// Proto's memory-space tag and kernel macros, as far as these kernels use them.
enum MemType { HOST = 0, DEVICE = 1 };
#define ACCEL_DECORATION
#define PROTO_KERNEL_START
#define PROTO_KERNEL_END(local, global)
#define PROTO_LAMBDA

// Element access of one point's components (c) or of a matrix (c, d),
// stored row-major here.
template <typename T, unsigned C = 1, MemType MEM = HOST, unsigned D = 1>
struct Var {
  T* p = nullptr;
  T& operator()(unsigned c) const { return p[c]; }
  T& operator()(unsigned c, unsigned d) const { return p[c * D + d]; }
};

// The 3-D state layout (src/BoxOp_EulerCubedSphere.H:13,37-49).
#define DIM 3
#define NUMCOMPS 8
#define iRHO 0
#define iVX 1
#define iMOMX 1
#define iVY 2
#define iMOMY 2
#define iVZ 3
#define iMOMZ 3
#define iE 4
#define iP 4
#define iBX 5
#define iBY 6
#define iBZ 7

#include "berta_kernels.inc"

namespace {
using V8 = Var<double, 8>;
using V1 = Var<double, 1>;
V8 at(const double* p) { return V8{const_cast<double*>(p)}; }
V1 one(const double* p) { return V1{const_cast<double*>(p)}; }
}  // namespace

extern "C" {

// cells [6][8] = W[i-3 .. i+2] for face i.
void ref_berta_wenoz(const double* cells, double* wl, double* wr) {
  V8 L = at(wl), R = at(wr);
  f_wenoz_pointwise_faceF<double, HOST, 8>(L, R, at(cells), at(cells + 8), at(cells + 16), at(cells + 24),
                                           at(cells + 32), at(cells + 40));
}

// cells [4][8] = W[i-2 .. i+1].
void ref_berta_weno3(const double* cells, double dx2, double* wl, double* wr) {
  V8 L = at(wl), R = at(wr);
  f_weno3_pointwise_faceF<double, HOST, 8>(L, R, at(cells), at(cells + 8), at(cells + 16), at(cells + 24), dx2);
}

void ref_berta_plm(const double* cells, double* wl, double* wr) {
  V8 L = at(wl), R = at(wr);
  f_plm_pointwise_faceF<double, HOST, 8>(L, R, at(cells), at(cells + 8), at(cells + 16), at(cells + 24));
}

double ref_berta_normalize(double* v, int n) {
  if (n == 4) return bertaNormalizeWenoStencil<double, 4>(*reinterpret_cast<double(*)[4]>(v));
  if (n == 6) return bertaNormalizeWenoStencil<double, 6>(*reinterpret_cast<double(*)[6]>(v));
  return std::nan("");
}

// cells [7][8]: the cell, then the low and high neighbours in directions
// 0, 1, 2; eps as BertaComputeThetaJameson passes it.
double ref_berta_jameson(const double* cells, double eta_d) {
  double theta = -1.0;
  V1 t = one(&theta);
  f_berta_jameson_theta_rawF<double, HOST>(t, at(cells + 8), at(cells), at(cells + 16), at(cells + 24),
                                           at(cells + 32), at(cells + 40), at(cells + 48), eta_d, 1.0e-40);
  return theta;
}

void ref_berta_avg_to_point(const double* avg, const double* lap, double theta, double* out) {
  V8 o = at(out);
  f_berta_avg_to_point_thetaF<double, HOST>(o, at(avg), at(lap), one(&theta));
}

void ref_berta_flux_to_avg(const double* pt, const double* lap, double theta, double* out) {
  V8 o = at(out);
  f_flux_point_to_avg_thetaF<double, HOST>(o, at(pt), at(lap), one(&theta));
}

void ref_berta_select(const double* wl4, const double* wr4, const double* wlf, const double* wrf, double theta,
                      double* wl, double* wr) {
  V8 L = at(wl), R = at(wr);
  f_select_reconstructionF<double, HOST>(L, R, at(wl4), at(wr4), at(wlf), at(wrf), one(&theta));
}

// Matrices and fluxes [column][cell], n = 1 or 3 columns, `size` cells.
void ref_berta_mapped_line(int n, int both, const double* m, const double* m1, const double* m2, const double* f,
                           const double* f1, const double* f2, int size, double* out) {
  const double *M[3], *M1[3], *M2[3], *F[3], *F1[3], *F2[3];
  for (int c = 0; c < n; ++c) {
    const size_t q = (size_t)c * size;
    M[c] = m + q; M1[c] = m1 + q; M2[c] = m2 + q; F[c] = f + q; F1[c] = f1 + q; F2[c] = f2 + q;
  }
  if (n == 1 && both) bertaMappedLine<1, true, double>(out, M, M1, M2, F, F1, F2, size);
  if (n == 1 && !both) bertaMappedLine<1, false, double>(out, M, M1, M2, F, F1, F2, size);
  if (n == 3 && both) bertaMappedLine<3, true, double>(out, M, M1, M2, F, F1, F2, size);
  if (n == 3 && !both) bertaMappedLine<3, false, double>(out, M, M1, M2, F, F1, F2, size);
}

void ref_sph_to_prim_raw(const double* u, double* w) {
  V8 o = at(w), in = at(u);
  f_sphToPrim_F<double, HOST>(o, in);
}

void ref_prim_flux(const double* w, double ke, double me, double vb, double gamma, int c, double* f) {
  V8 o = at(f);
  double adj = 1.0;
  f_primflux_F<double, HOST>(o, at(w), one(&ke), one(&me), one(&vb), one(&adj), gamma, 0u, (unsigned)c);
}

double ref_rho_floor() { return RHO00; }
}

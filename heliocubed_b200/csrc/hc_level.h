// Level geometry and kernel argument structures shared by the host context
// (hc_context.cpp) and the kernels (hc_kernels.cu).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include <vector>

#include "hc_common.h"

namespace hc {

constexpr int kGhost = 2;  // ghost width of level primitive arrays (O2)

// Seam ghost donor: 4-point along-edge interpolation in panel `b`.
struct SeamDonor {
  int b;
  int j[4];
  int k[4];
  int pad;
  double w[4];
};

// Neighbour across one panel edge (edge = (axis-1)*2 + side of this panel).
struct EdgeLink {
  int nb, axis, side, pad;
};

// CFL geometry of one angular cell, src/BoxOp_SecondOrderCFL.H:14-20.
struct CflCell {
  double inverseDet;
  double inverseDetA[9];
  double cell[9];
  double face[2][9];
  double det[3];
  double normal[3];
  double pad[2];
};

// Per-cell gravity / conversion data: Xhat at the centre, det, first column
// of <det(A) A>, pad (src/BoxOp_Gravity.H:16-26).
struct GravCell {
  double x[3];
  double det;
  double a0[3];
  double pad;
};

// A cone cloud fed through the inner boundary while it crosses it (the
// finite cloud of hc_cone, src/MHD_CME.H:968,1111-1143).
struct InletCone {
  double axis[3];
  double radius, entryShift, entryTime, speed, endTime, insertionTime, density, temperature;
};
constexpr int kInletCones = 8;

struct DevLevel {
  int nr, na, g;
  int n0, n1;            // ghosted dims nr+2g, na+2g
  long Nv, Ng;           // cells per box: valid, ghosted
  double h, dxi0;
  const double4* radial; // [nr+2g+1], index i+g: {area0 (rlow^2), areaT, Dr0, vol}
  const double* rc;      // [nr+2g+1], index i+g: cell-centre radius rhalf
  const FaceGeom* face;  // [3][6][na+1][na+1]
  const GravCell* grav;  // [6][na][na]
  const double* basis;   // [6][na][na][9] cell-centre A, row-major
  const double* basisInv;// [6][na][na][9]
  const CflCell* cfl;    // [6][na][na]
  const SeamDonor* seam; // [6][2][2][g][na]
  const int* faceMap;    // [6][2][2][na]: neighbour along-edge index of a seam face
  const EdgeLink* edge;  // [6][2][2]
  const double* innerBC; // [6][na][na][g][8] native conserved wind, or null
  double outerScale2[kGhost], outerScale1[kGhost];
  double gamma, invGm1, entropy, cfl_number, strength, r0;
  int innerBCType;
  const InletCone* inlet;  // device array of cones fed through r_inner, or null
  int ninlet;
};

// Operator launch: boxes share the valid region [lo,hi]; box b lies on panel
// block0+b, its primitives start at w + b*wBoxStride on storage box
// (wlo, wn), component stride wN.
struct StageArgs {
  DevLevel L;
  const double* w;
  long wBoxStride, wN;
  int wlo[3], wn[3];
  int lo[3], hi[3];
  int nbox, block0;
  double scale;
  int seams;             // compute shared seam states from neighbour panels
  // per-box outputs (MODE 0): rhs on valid (accumulated), flux on extrude(d)
  double* rhs;
  long rhsBoxStride, rhsN;
  double* flux[3];
  const double* panel[6];
  // level RK stage (MODE 1): k never leaves registers.  The epilogue writes
  // the next stage's primitives (valid cells) into wOut; stage 3 writes the
  // new state into ju, its primitives into wOut and, when invMaxOut is set,
  // the CFL rate of the new state (atomic max of the bit pattern).
  int stage;
  const double* invDtMax;  // device: dt = cfl / *invDtMax (null: use dtv)
  double dtv;
  double* ju;
  double* acc;
  double* wOut;
  unsigned long long* invMaxOut;
  int* invalid;            // OR-ed validity flag of the new state (stage 3)
  // time of the step's start (MODE_RK): tbase + *tdev; the stage adds
  // c_s dt.  Only the inlet footprint of the inner face reads it.
  double tbase;
  const double* tdev;
  // CME insertion window (device flag, may be null): the launch returns at
  // once when (*solverFlag != 0) == exitOnFlag, so a Roe context launches
  // its Roe kernel (exit on 1) and its Rusanov kernel (exit on 0)
  const int* solverFlag;
  int exitOnFlag;
};

enum { MODE_BOX = 0, MODE_RK = 1, MODE_RHS = 2 };

// Host launchers (hc_kernels.cu).  Every launcher returns a cudaError_t.
// tile: cell tile of the stage kernel (0 .. kStageTiles-1, see
// stageTileShape); MODE_BOX launches always use tile 0.
constexpr int kStageTiles = 6;
cudaError_t launchStage(const StageArgs& a, int mode, int limiter, bool roe, bool powell, bool grav,
                        cudaStream_t s, int tile = 0);
// {X, Y, Z, min CTAs/SM with Rusanov, with Roe} of a stage tile; 0 if none.
int stageTileShape(int tile, int out[5]);
cudaError_t launchPrimValid(const DevLevel& L, const double* ju, double* w, cudaStream_t s);
// Time of a stage: t = tbase + (tdev ? *tdev : 0) + cfrac * dt, with
// dt = invDtMax ? cfl / *invDtMax : dtv.
struct StageTime {
  double tbase;
  const double* tdev;
  double cfrac;
  const double* invDtMax;
  double dtv;
};
cudaError_t launchGhosts(const DevLevel& L, double* w, const StageTime& t, cudaStream_t s);
// time (device, may be null): with inlet cones active then, the cone
// density floor of the Alfven speed applies.
cudaError_t launchCfl(const DevLevel& L, const double* ju, unsigned long long* invMaxBits, cudaStream_t s,
                      const double* time = nullptr);
cudaError_t launchValid(const DevLevel& L, const double* ju, int* ok, cudaStream_t s);
cudaError_t launchInit(const DevLevel& L, const void* init, double* ju, cudaStream_t s);
cudaError_t launchBoxGravity(const DevLevel& L, const int lo[3], const int hi[3], int block, const double* w,
                             const int wlo[3], const int wn[3], double* rhs, cudaStream_t s);
cudaError_t launchAdvanceTime(double* time, const double* invDtMax, double cfl, double* dtOut, cudaStream_t s);

// CME insertion schedule (src/MHD_CME.H:1243-1334 CMEInsertionSchedule):
// sources inserted at t (device: once time >= t), their stabilisation ends
// and whether they feed through the boundary.
constexpr int kCmeEvents = 8;
struct CmeSchedule {
  int n, roe;
  double cfl, feeding;  // target CFL; feeding fraction (0.5 with Roe, 1 with Rusanov, exec/main.cpp:374)
  double t[kCmeEvents], stabEnd[kCmeEvents];
  int boundary[kCmeEvents];
  // the inlet clouds' crossing rate (src/MHD_CME.H:1165-1191, finite
  // clouds): + (speed + sound speed of the cloud) / first radial cell width
  int ninlet;
  double inletT[kInletCones], inletEnd[kInletCones], inletSpeed[kInletCones], inletTemp[kInletCones];
  double width, gamma;
};
// At the start of a step: the CFL rate in *invMaxBits (a non-negative double's
// bits) becomes rate / fraction(time), and no smaller than cfl / (window end
// - time) inside the Rusanov window, so dt = cfl / rate lands on the window's
// end; *rusanov = Roe context inside the window.
cudaError_t launchCmeSchedule(const CmeSchedule* sched, unsigned long long* invMaxBits, const double* time,
                              int* rusanov, cudaStream_t s);
cudaError_t launchBitsToDouble(const unsigned long long* bits, double* out, cudaStream_t s);

}  // namespace hc

namespace hc {
// ---------------------------------------------------------------------------
// Fourth-order Berta operator (hc_o4.cu).
// ---------------------------------------------------------------------------
constexpr int kO4Ghost = 5;  // NGHOST: Jameson detector + WENOZ + transverse products
constexpr int kO4Ang = 8;    // angular margin of the O4 metric tables
constexpr int kO4Rad = 10;   // radial margin of the O4 radial table

// Face metrics of direction d at angular (j,k): <det A A> (9), <det A> (1),
// <adjA row d> (3), pointwise basis at the face centre (9; d = 0: cell centre).
constexpr int kO4FaceRec = 22;
// Frame of the factored Roe dissipation at a face of direction d (angular
// (j,k)), from the face-centre basis A (d = 0: cell centre): unit normal f0,
// unit tangent f1, f2 = f0 x f1 (9), |cofactor row d of A| (1), adj A (9),
// 1 / det A, 1 / det A^2 (2); padded to 24 (16-byte aligned pairs).
constexpr int kO4RoeRec = 24;

struct O4Geo {
  int nr, na, ext;        // tables cover angular indices [-ext, na+ext]
  const double* face;     // [6][3][na+2ext+1 (k)][na+2ext+1 (j)][22]
  const double* cell;     // [6][na+2ext+1][na+2ext+1][9] cell-centre basis
  const double* frames;   // [6][3][na+2ext+1 (k)][na+2ext+1 (j)][kO4RoeRec] Roe frames
  const double4* radial;  // [nr+2*kO4Rad+1], index i+kO4Rad: {rlow^2, areaT, Dr0, dVolr}
  double gamma, invGm1, entropy, eta_d, dx[3];
  int roe, powell, fallback;
  const int* rusanov;     // device flag (may be null): nonzero runs a Roe context with Rusanov dissipation
  int* status;            // device word (may be null): set to 1 when a kernel's bounded wait for a
                          // shared-memory tile gave up (that tile's rhs is then NaN)
};

// A box region: low corner, extents, cell count.
struct Reg {
  int lo[3], n[3];
  long N;
};

// One batched O4 operator evaluation: nbox boxes (panels block0 + b) with
// the same valid box [vlo, vhi]; U on valid.grow(ghost) in the caller's
// storage (region ur, box stride uStride); rhs accumulated on the valid box.
struct O4Args {
  O4Geo G;
  int nbox, block0, ghost;
  int vlo[3], vhi[3];
  const double* U;
  Reg ur;
  long uStride;
  double scale;
  double* rhs;
  long rhsStride;
  double* flux[3];
  // scratch (device): cell arrays on the ghosted box, face arrays on the
  // reconstruction face box of the current direction
  double* WA;   // [nbox][8][G]
  double* WP;   // [nbox][8][G]
  double* th;   // [nbox][G]
  double* thr;  // [nbox][G] raw detector flag
  double* face; // [nbox][kO4FaceArrays][F]: face arrays of directions 0 and 2
  double* face2; // [nbox][kO4FaceArrays][F]: face arrays of direction 1 (its pass overlaps its neighbours')
  double* mj;   // [nbox][V+1]
  double* kp;   // [nbox][8][V+2]
  // The seam-flux register of the box's own level when the box runs in one
  // launch with other levels' boxes (an ensemble): null takes the launch's
  // RegArgs; else the face flux times (stage weight) * seamCfl / *seamInvMax
  // is added into seamReg.
  double* seamReg;
  const double* seamInvMax;
  double seamCfl;
  // Storage region of rhs when it is larger than the valid box (a level
  // array of which the box evaluates a radial window); rr.N == 0: the
  // valid box itself.
  Reg rr;
};
constexpr int kO4FaceArrays = 8 * 4 + 5 + 9;  // WL, WR, FS, QD/DP (8 each) + thF, PS, BP, Bflux, Bprod + averages (8 + 1)

size_t o4ScratchDoubles(int nbox, const int vlo[3], const int vhi[3], int ghost);
// Carve the operator scratch of a.nbox boxes with the valid box a.vlo..vhi
// from sp (every array starts on a 256-byte boundary when sp does);
// returns the doubles used (o4ScratchDoubles).
size_t o4CarveScratch(O4Args& a, double* sp);

// Seam flux register of the level step (reg null: off): the final face flux
// of panel-boundary faces of directions 1, 2 of whole-panel boxes is added
// times w (times cfl / *wDev when wDev is set) into reg [6][2][2][8][na][nr].
struct RegArgs {
  double* reg;
  double w;
  const double* wDev;
  double cfl;
};

// A batch of boxes of any sizes for the operator kernels: per box and
// direction a kernel context in device memory; every kernel of the operator
// is one launch over the whole batch (one CTA row per box).  Each entry of
// `boxes` describes one box (nbox 1) with its own input, output and scratch.
struct O4Batch;
// Register-cap variants of the operator's three heaviest kernels
// (reconstruction, Roe point dissipation, final flux), chosen by the
// autotuner; results do not depend on them.
constexpr int kO4TunedKernels = 3, kO4Variants = 3;
void o4BatchSetVariants(O4Batch* b, const int v[kO4TunedKernels]);
int o4VariantMinBlocks(int kernel, int variant);
O4Batch* o4BatchCreate(const O4Args* boxes, int nbox, cudaError_t* err);
void o4BatchDestroy(O4Batch* b);
// The one-box argument sets of a uniform multi-box O4Args (box b on panel
// block0 + b, arrays at b x stride).
void o4SplitArgs(const O4Args& a, std::vector<O4Args>& out);
cudaError_t launchO4Batch(const O4Batch* b, const RegArgs* reg, cudaStream_t s);
// Gravity_Euler on the valid boxes of the batch (reads U, adds into rhs).
cudaError_t launchO4BatchGravity(const O4Batch* b, cudaStream_t s);

// ---------------------------------------------------------------------------
// Fourth-order level step (hc_o4level.cu): one box per panel.
// ---------------------------------------------------------------------------
constexpr int kO4Cart = 6;  // angular ghost layers of the Cartesian averages

// One interpolation point of the seam ghosts: the point value at a cell
// centre of the ghost panel's grid from panel p's 4 x 4 donor cell averages
// starting at (j0, k0), tensor weights wj and wk.  cell: the donor cell that
// contains the point, (j0 + (cell & 3), k0 + (cell >> 2)).
struct O4Point {
  int p, j0, k0, cell;
  double wj[4], wk[4];
};

struct O4Level {
  int nr, na, g, ga;        // g = kO4Ghost, ga = kO4Cart
  int nA, nG;               // na + 2 ga, na + 2 g
  int nring;                // seam ghost positions per panel
  int npts;                 // interpolation points per panel
  long Nv, Ng, Nc;          // per panel: valid, ghosted native, Cartesian
  const double* coef;       // [6][nA][nA][27]: <A>^-1, D1 <A>, D2 <A> (row-major)
  const double* detx;       // [6][na+2][na+2]: <det A>, j, k in [-1, na]
  const double* xhat;       // [6][nG][nG][3]: unit direction of the cell centre
  const double2* radial;    // [nr + 2g + 2], index i + g + 1: {dVolr, cell-centre radius}
  const int2* ringJK;       // [nring]: (j, k) of each seam ghost position
  const int* ringPt;        // [nring][5]: points at the ghost centre and its 4 neighbours
  const O4Point* pts;       // [6][npts]
  const double* inner;      // [6][nG][nG][g][8] inner radial ghosts when time independent, or null
  double gamma, r0, strength, cfl;
};

// Kernel arguments of the stage preparation and the RK update.
struct O4StageIO {
  O4Level O;
  const double* ju;   // stage state [6][8][Nv]
  double* cart;       // [6][8][Nc]
  double* us;         // [6][8][Ng]
  double* pv;         // point values [6][8][npts][nr]
  StageTime t;
};

cudaError_t launchO4Prepare(const O4StageIO& io, cudaStream_t s);
// acc/stage/ju update after stage s (classical RK4, b = 1/6, 1/3, 1/3, 1/6;
// next stage = ju + a_{s+1} dt k with a = 1/2, 1/2, 1).
cudaError_t launchO4Update(const O4Level& O, int stage, const double* k, double* ju, double* acc, double* next,
                           const double* invDtMax, double cfl, double dtv, cudaStream_t s);
// Seam flux reconciliation from the time-integrated register
// [6][2][2][8][na][nr] (edge axis 1..2, side 0..1, component, along-edge, radial).
cudaError_t launchO4Reflux(const O4Level& O, const DevLevel& L, const double* reg, double* ju, cudaStream_t s);
}  // namespace hc

// Context internals for sibling translation units (not part of the C ABI).
struct hc_ctx;
struct hc_params;
namespace hc {
const DevLevel* ctxLevel(const hc_ctx* c);
const hc_params* ctxParams(const hc_ctx* c);
int ctxDevice(const hc_ctx* c);
// The fourth-order level tables of an order-4 context (null otherwise).
const O4Level* ctxO4Level(const hc_ctx* c);
int setLastError(int code, const char* msg);
}  // namespace hc

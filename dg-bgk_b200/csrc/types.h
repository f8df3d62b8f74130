// Data layout shared by the host plan builder and the sm_100a kernels.
//
// HBM layout of the distribution function: f[(e*3 + i)*Vp + v] -- element e
// (in the plan's locality order), DG node i (0..2), discrete velocity v
// fastest, rows padded to a pitch Vp (a multiple of 32 velocities, so every
// row starts on a 128-byte boundary and splits into whole 64-byte sweep
// segments).  The padding velocities hold zeros forever (the buffers are
// cleared at allocation and the kernels write zeros there), so kernels may
// read whole 16-byte vectors past V without bounds checks.  Two such buffers are
// kept (ping-pong): within one pseudo-time step the reference updates every
// element of velocity IV only after all edge fluxes of IV are formed
// (src/advnce.f90:321-367), i.e. a Jacobi update in space, so the sweep reads
// f^n and writes f^{n+1}.
#pragma once
#include <cstdint>

namespace dgbgk {

// Per element and local edge k (from local node k to node (k+1) mod 3).
// The sweep forms every edge flux from an upwind "source" row set: the
// neighbour across an interior side, the element itself on an outflow side
// (the upwind value of an outflow side is always the element's own) and, as a
// placeholder, on inflow sides (no flux) and wall sides (whose flux the wall
// path adds).  The source's two rows (its local nodes at my points k and
// k+1) are given as their byte offsets in the sweep tile at velocity chunk 0
// (tile_row_off below); chunk c of the same row is at offset ^ 16*c.
template <class T> struct alignas(16) ElemEdge {
  T anx, any;      // AL times the outward unit normal; AL = EL/6 (interior) or RSIDO(3)/6 (boundary)
  unsigned offp;   // tile offset of the source's row at point k
  unsigned offq;   // ... at point k+1
};

// Byte offset of 16-byte chunk 0 of row r in a sweep tile (64-byte rows
// with the 64-byte swizzle: chunk c of row r at 16*(c ^ ((r >> 1) & 3)),
// i.e. at tile_row_off(r) ^ 16*c).
#if defined(__CUDACC__)
__host__ __device__
#endif
inline unsigned tile_row_off(int r) { return (unsigned)(r * 64 + 16 * ((r >> 1) & 3)); }

// Everything the sweep needs about one element, in one 16-byte-aligned
// record.  The leading part (shape-function gradients and the GTEQNF /
// COMPMU parameters of the three DG nodes, 21 values) is all a halo element
// needs; the moment kernel rewrites the node parameters every step.
template <class T> struct alignas(16) ElemRec {
  T gx[3], gy[3];  // shape-function gradients GEOME(1:3), GEOME(4:6)
  // GTEQNF's Maxwellian NFO (src/gteqnf.f90:26-40) at node i and velocity c,
  // with A = DISND*BETA2/PI and u = (DISUX, DISUY):
  //  FP32: NFO = A * 2^(ex*|c-u|^2), ex = -BETA2*log2(e): A, ex, ux, uy;
  //  FP64: NFO = exp(a0 + a1*cx + a2*cy + ex*|c|^2), the exponent expanded:
  //        A holds a0 = ln(A) - BETA2*|u|^2, ux a1 = 2*BETA2*ux, uy a2 =
  //        2*BETA2*uy, ex = -BETA2 (a0 = -inf where A = 0).
  // (NFO = 0 where DISPS < 1e-20, src/gteqnf.f90:32.)
  T A[3];
  T ex[3];
  T ux[3];
  T uy[3];
  T mu[3];   // collision frequency MU (src/compmu.f90:90-92)
  T area;    // 0.5 * GEOME(7)   (src/getelc.f90:44)
  T mm[3];   // MMAT (IMMAT = 1) or CMMAT row sums (IMMAT = 0)
  int bside[3];  // boundary side index of each wall edge (kind 3), else -1
  ElemEdge<T> edge[3];
  int flags;  // bits [0,3): DG node i sits on an inflow-side node (INFLOW);
              // bits [3,6): edge k is a wall side; bits [6,9): edge k carries
              // the element-centric flux (interior or outflow side); bit 9:
              // all three edges are interior sides
  int wslot;  // wall element slot (ALPHA < 1: the deferred updates), else -1
  unsigned own01;  // tile offsets (chunk 0) of the element's own rows 0 and 1 (16 bits each)
  unsigned own2;   // ... and row 2
};
constexpr int FLAG_FLUX0 = 1 << 6;      // FLAG_FLUX0 << k: edge k carries the element-centric flux
constexpr int FLAG_INTERIOR = 1 << 9;  // all three edges interior
static_assert(sizeof(ElemRec<float>) == 176 && sizeof(ElemRec<double>) == 336, "record layout");
// values of the leading part a halo element needs (gx .. mu)
constexpr int REC_HEAD_VALUES = 21;

// One type-4 wall side for the wall-flux kernel (FLUCON2).
struct WallSide {
  int elem;     // plan order
  int in1, in2; // local nodes of BSIDO(1), BSIDO(2) in that element
  int bside;    // boundary side index
  double anx, any;     // RSIDO(1:2)
  double sumbottom;    // sqrt(2*PI*R^3*T_w^3)
};

// One type-4 wall side for GETFOR's lift and drag (src/getfor.f90:29-49):
// its two nodes and LEN*PERP, PERP the unit normal of the side vector
// turned 90 degrees anticlockwise.
struct ForceSide {
  int ip1, ip2;  // nodes BSIDO(1), BSIDO(2), 0-based
  double lx, ly; // LEN*PERP(1), LEN*PERP(2)
};

// Device-side control block of one case.
struct Ctrl {
  int done;       // kernels skip the case when set
  int step;       // steps run in this advance call
  int max_steps;
  int nonfinite;  // set when a residual was NaN/Inf
  double tol;     // relative L2 tolerance (<= 0: none)
  double ref;     // reference L2 residual (0: take the first step's)
  double maxmu;   // max MU of the current step (atomicMax on the bits; reset by k_resid)
  double dtc;     // Courant limit DTEc (src/alotim.f90)
  double acc_sq;  // sum of squared changes of the current step (sweep atomics; reset by k_resid)
  double acc_max; // max residual of the current step (atomicMax on the bits; reset by k_resid)
  int cur;        // which f buffer holds the current state (k_resid swaps it)
  int timeout;    // set when a bounded device wait gave up
  int itime0;     // steps the handle ran before this advance call (the reference's ITIME - step - 1)
  int pad0;
};

// Device-side control of one launch set (a case alone or a batch).
struct BatchCtl {
  int sweep_next;  // sweep work units handed out beyond the first wave (reset by k_resid)
  int pad[15];
};

}  // namespace dgbgk

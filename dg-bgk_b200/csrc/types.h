// Data layout shared by the host plan builder and the sm_100a kernels.
//
// HBM layout of the distribution function: f[(e*3 + i)*Vp + v] -- element e
// (in the plan's locality order), DG node i (0..2), discrete velocity v
// fastest, rows padded to a pitch Vp (a multiple of 32 velocities, so every
// row starts on a 128-byte boundary and every TMA box coordinate
// v0 = 32*k is 16-byte aligned).  The padding velocities hold zeros forever
// (the buffers are cleared at allocation and no kernel writes v >= V), so
// kernels may read whole 16-byte vectors past V without bounds checks.  A
// warp reading 32 consecutive velocities of one node issues one fully
// coalesced 128-byte (FP32) or 256-byte (FP64) request.  Two such buffers are
// kept (ping-pong): within one pseudo-time step the reference updates every
// element of velocity IV only after all edge fluxes of IV are formed
// (src/advnce.f90:321-367), i.e. a Jacobi update in space, so the sweep reads
// f^n and writes f^{n+1}.
#pragma once
#include <cstdint>

namespace dgbgk {

constexpr int VTILE = 32;  // velocities per sweep tile (one warp's lanes)

// Per element and local edge k (from local node k to node (k+1) mod 3).
// info bits: [0,2) kind -- 0 interior side, 1 inflow side (no flux),
// 2 outflow side, 3 wall side (any other BSIDO type); bit 2: this element is
// ISIDE(3) (the "left" one); [3,5) neighbour's local node at my point k;
// [5,7) at my point k+1; [8,32) the neighbour's shared-memory slot in the
// sweep tile (interior sides) or the boundary side index in BSIDO order
// (kinds 1..3).
template <class T> struct alignas(16) ElemEdge {
  T nx, ny;   // outward unit normal of this element on this edge
  T alen;     // EL/6 (interior) or RSIDO(3)/6 (boundary)
  int info;
};

// Everything the sweep needs about one element, in one 16-byte-aligned
// record that a bulk copy brings into shared memory.  The leading "UMEAN
// part" (shape-function gradients and the GTEQNF / COMPMU parameters of the
// three DG nodes) is all a halo element needs; the moment kernel rewrites the
// node parameters every step.
template <class T> struct alignas(16) ElemRec {
  T gx[3], gy[3];  // shape-function gradients GEOME(1:3), GEOME(4:6)
  T A[3];    // DISND*BETA2/PI   (0 where DISPS < 1e-20: NFO = 0, src/gteqnf.f90:321)
  T B[3];    // BETA2 = RHO/(2*PS)
  T ux[3];   // DISUX
  T uy[3];   // DISUY
  T mu[3];   // collision frequency MU (src/compmu.f90:284-285)
  T area;    // 0.5 * GEOME(7)   (src/getelc.f90:44)
  T mm[3];   // MMAT (IMMAT = 1) or CMMAT row sums (IMMAT = 0)
  T pad0[3];
  ElemEdge<T> edge[3];
  int inflow;  // bit i: DG node i sits on an inflow-side node (INFLOW)
  int pad1[3];
};
// bytes of the UMEAN part, rounded up to the 16-byte bulk-copy granule
template <class T> constexpr unsigned umean_part_bytes() { return (unsigned)((22 * sizeof(T) + 15) / 16 * 16); }

// One type-4 wall side for the wall-flux kernel (FLUCON2).
struct WallSide {
  int elem;     // plan order
  int in1, in2; // local nodes of BSIDO(1), BSIDO(2) in that element
  int bside;    // boundary side index
  double anx, any;     // RSIDO(1:2)
  double sumbottom;    // sqrt(2*PI*R^3*T_w^3)
};

// Device-side control block of one handle.
struct Ctrl {
  int done;       // kernels return at once when set
  int step;       // steps run in this advance call
  int max_steps;
  int nonfinite;  // set when a residual was NaN/Inf
  double tol;     // relative L2 tolerance (<= 0: none)
  double ref;     // reference L2 residual (0: take the first step's)
  double maxmu;   // max MU of the current step (atomicMax on the bits)
  double dtc;     // Courant limit DTEc (src/alotim.f90)
  int nparts;     // sweep CTAs writing residual partials
  int timeout;    // set when a bounded device wait gave up
};

}  // namespace dgbgk

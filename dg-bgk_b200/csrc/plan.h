// Host-side plan: everything the kernels need that does not change during
// the time loop, derived from the reference's setup arrays.
#pragma once
#include <string>
#include <vector>

#include "../../include/dgbgk.h"
#include "types.h"

namespace dgbgk {

// Element edge before blocking: the device record ElemEdge<T> packs `low`
// with the neighbour's tile slot (interior) or `bside` (boundary) into info.
struct PlanEdge {
  double nx = 0, ny = 0, alen = 0;
  int low = -1;   // info bits [0,7): kind, left flag, neighbour local nodes
  int nbr = -1;   // neighbour element (plan order) or -1
  int bside = -1; // boundary side index or -1
};

// Velocity-independent data of one element (FP64 master copy).
struct PlanGeo {
  double gx[3] = {0, 0, 0}, gy[3] = {0, 0, 0};  // GEOME(1:3), GEOME(4:6)
  double area = 0;                              // 0.5 * GEOME(7)
  double mm[3] = {0, 0, 0};  // MMAT (IMMAT = 1) or CMMAT row sums (IMMAT = 0)
  int inflow = 0;            // bit i: DG node i sits on an inflow-side node
};

struct Plan {
  int E = 0, NP = 0, B = 0, S = 0, V = 0, RORDER = 0, TORDER = 0;
  int immat = 1;
  double alpha = 1, rgas = 1, M = 1, d = 1, rv = 1, sumweight = 1, dtc = 0;
  double cinf[4] = {0, 0, 0, 0};
  // element order: perm[new] = old, inv[old] = new (0-based)
  std::vector<int> perm, inv;
  // sweep blocking
  int EB = 0, nblocks = 0, max_halo = 0;
  std::vector<int> halo_off, halo_list;  // per block, plan order
  std::vector<int> eslot;                // [3E] tile slot of the neighbour
  // per element (plan order), FP64 master copies
  std::vector<PlanGeo> geo;
  std::vector<PlanEdge> edge;               // [3E]
  std::vector<double> cmax, cmin;           // [3E], IMMAT = 0 residual
  // per velocity
  std::vector<double> cx, cy, wjf, nfinf;
  // boundary sides
  std::vector<double> bTw, bUw;  // [B], [2B]
  std::vector<WallSide> walls;   // type-4 sides (FLUCON2)
  std::vector<ForceSide> fsides; // type-4 sides in boundary-side order (GETFOR)
  bool has_wall_incoming = false;  // some side of a kind-3 wall exists
  // nodal gather (MACROS tail / GETMAC): CSR over mesh nodes
  std::vector<int> node_off, node_dg;  // DG node index (plan order) per entry
  std::vector<double> node_ae;         // GEOME(7) of its element
  // Wall accommodation ALPHA < 1 (IMMAT = 1): the specular part of GETBOU.
  // A molecule leaving a wall side at velocity v (TEST < 0) carries
  // (1-ALPHA) times the element's own f at the mirrored velocity, read as
  // the two grid velocities I1, I2 around it and interpolated with ZD1, ZD2
  // (src/getbou.f90:189-255).  The reference reads them from DISNF while its
  // velocity loop updates it in place, so velocities I < v contribute their
  // new values.  Items are (wall element slot, v) pairs with some node
  // deferred; an item whose mirrored velocities include an earlier deferred
  // one is "sequential" (processed per element in velocity order).
  bool spec = false;
  std::vector<int> welem;         // wall elements (plan order) by slot
  std::vector<int> wslot;         // [E] slot of each element, -1 without a wall side
  std::vector<int> rside;         // [B] reflection-table row of each wall side, -1 for others
  std::vector<int> rf_i;          // [rows][V][2] I1, I2 (0-based); -1 where TEST >= 0
  std::vector<double> rf_z;       // [rows][V][2] ZD1, ZD2
  std::vector<int> spec_par;      // items slot*V + v processed in parallel
  std::vector<int> spec_seq_off;  // [slots + 1]
  std::vector<int> spec_seq;      // sequential items, per slot in velocity order
};

// Device edge word of edge i = 3*e + k (ElemEdge::info): the kind, the
// flux source's local nodes and its tile slot -- the neighbour across an
// interior side, the element itself (slot own_slot, nodes k and k+1) on a
// boundary side.
inline int edge_info(const Plan& pl, size_t i, int own_slot) {
  const PlanEdge& e = pl.edge[i];
  const int kind = e.low & 3;
  if (kind == 0) return (e.low & ~4) | (pl.eslot[i] << 8);
  const int k = (int)(i % 3);
  return kind | (k << 3) | (((k + 1) % 3) << 5) | (own_slot << 8);
}

// Builds the plan; returns 0 or a DGBGK_E* code with the message in *err.
int build_plan(const dgbgk_mesh& m, const dgbgk_vspace& vs, const dgbgk_params& p, int EB, Plan& out,
               std::string* err);

// Rebuilds only the blocking (EB, halos, slots) of an existing plan.
void build_blocks(Plan& pl, int EB);

}  // namespace dgbgk

// Host-side plan: everything the kernels need that does not change during
// the time loop, derived from the reference's setup arrays.
#pragma once
#include <string>
#include <vector>

#include "../../include/dgbgk.h"
#include "types.h"

namespace dgbgk {

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
  std::vector<int> eslot;                // [3E] smem slot of the neighbour
  // per element (plan order), FP64 master copies
  std::vector<ElemGeo<double>> geo;
  std::vector<ElemEdge<double>> edge;       // [3E]
  std::vector<double> cmax, cmin;           // [3E], IMMAT = 0 residual
  // per velocity
  std::vector<double> cx, cy, wjf, nfinf;
  // boundary sides
  std::vector<double> bTw, bUw;  // [B], [2B]
  std::vector<WallSide> walls;   // type-4 sides (FLUCON2)
  bool has_wall_incoming = false;  // some side of a kind-3 wall exists
  // nodal gather (MACROS tail / GETMAC): CSR over mesh nodes
  std::vector<int> node_off, node_dg;  // DG node index (plan order) per entry
  std::vector<double> node_ae;         // GEOME(7) of its element
};

// Builds the plan; returns 0 or a DGBGK_E* code with the message in *err.
int build_plan(const dgbgk_mesh& m, const dgbgk_vspace& vs, const dgbgk_params& p, int EB, Plan& out,
               std::string* err);

// Rebuilds only the blocking (EB, halos, slots) of an existing plan.
void build_blocks(Plan& pl, int EB);

}  // namespace dgbgk

// esr_internal.h -- declarations shared by the host runtime files.
#pragma once
#include <string>
#include <vector>

#include "../../include/eulersr.h"
#include "esr_layout.h"

namespace esr {

struct HostMesh {
  int n_cells = 0, n_faces = 0, n_boundary_slots = 0;
  double y_min = 0, y_max = 0;
  std::vector<int> perm;          // new -> old
  std::vector<int> patch_start;   // cells of patch p: [patch_start[p], patch_start[p+1]) in the new order
  std::vector<int> inv;           // old -> new
  std::vector<double> geo;        // n_cells records of G_COUNT values, renumbered
  // The same records formed as the reference forms them on every call, in
  // its operation order, from the points rounded to the run's precision
  // (esr_params.fidelity = ESR_FIDELITY_REFERENCE); float32 adds the
  // per-call least-squares data.
  std::vector<float> geo_ref32;
  std::vector<LsqRef> lsq_ref32;
  std::vector<double> geo_ref64;
  std::vector<float> wall_n_ref32, wall_ds_ref32;
  std::vector<double> wall_n_ref64, wall_ds_ref64;
  std::vector<int> nbr;           // 4 x n_cells (x,y,z neighbours, w packed)
  std::vector<int> wall_cell;     // renumbered owner cell of each force face
  std::vector<double> wall_n;     // (nx, ny) per force face
  std::vector<double> wall_ds;    // face length per force face
  double inlet_subsonic[4] = {1.0, 1.0, 0.0, 1.0};
};

int prepare_mesh(const esr_mesh_desc& d, HostMesh& hm, std::string& err);
// records `msg` as the calling thread's esr_last_error() and returns `code`
int report_error(int code, const std::string& msg);
std::vector<int> rcm_order(int n, const std::vector<int>& nbr);
std::vector<int> patch_order(int n, const std::vector<int>& nbr, const std::vector<int>& seed,
                             std::vector<int>& patch_start);

}  // namespace esr

struct esr_mesh {
  esr::HostMesh hm;
};

// esr_mesh.cpp -- host-side mesh preprocessing for the device solver.
//
// Input: the EulerSR mesh arrays (euler/jax_fvm/src/mesh.py:131-150).
// Output: a renumbered, kernel-ready description in float64:
//   * cells in reverse Cuthill-McKee order (neighbours close in memory),
//   * per cell and edge slot: neighbour, slot kind, the neighbour's slot of the
//     shared face, LSQ coefficients, face offset, unit normal, face length,
//   * per cell: area and the sponge blend^3,
//   * the force faces with their owner cell, normal and length.
// Geometry follows mesh.py:223-260; the LSQ coefficients fold the 2x2 solve
// of helper.py:136-153 into c_k = w_k A^{-1} dx_k so the kernel's gradient is
// sum_k c_k (P_k - P_c).
#include "esr_internal.h"

#include <algorithm>
#include <cmath>
#include <deque>
#include <limits>
#include <numeric>
#include <string>

namespace esr {

static bool is_wall(int m, const std::vector<int>& walls) {
  return std::find(walls.begin(), walls.end(), m) != walls.end();
}

// reverse Cuthill-McKee over the cell adjacency, one BFS per component,
// starting from a minimum-degree cell; neighbours visited by increasing degree
std::vector<int> rcm_order(int n, const std::vector<int>& nbr) {
  std::vector<int> deg(n, 0);
  for (int c = 0; c < n; ++c)
    for (int k = 0; k < 3; ++k) deg[c] += nbr[3 * c + k] >= 0;
  std::vector<int> order;
  order.reserve(n);
  std::vector<char> seen(n, 0);
  std::vector<int> by_deg(n);
  std::iota(by_deg.begin(), by_deg.end(), 0);
  std::stable_sort(by_deg.begin(), by_deg.end(), [&](int a, int b) { return deg[a] < deg[b]; });
  for (int start : by_deg) {
    if (seen[start]) continue;
    std::deque<int> q;
    q.push_back(start);
    seen[start] = 1;
    while (!q.empty()) {
      int c = q.front();
      q.pop_front();
      order.push_back(c);
      int nb[3], m = 0;
      for (int k = 0; k < 3; ++k) {
        int j = nbr[3 * c + k];
        if (j >= 0 && !seen[j]) nb[m++] = j;
      }
      // at most three: insertion sort by (degree, index)
      auto before = [&](int a, int b) { return deg[a] < deg[b] || (deg[a] == deg[b] && a < b); };
      for (int i = 1; i < m; ++i)
        for (int j = i; j > 0 && before(nb[j], nb[j - 1]); --j) std::swap(nb[j], nb[j - 1]);
      for (int i = 0; i < m; ++i) {
        seen[nb[i]] = 1;
        q.push_back(nb[i]);
      }
    }
  }
  std::reverse(order.begin(), order.end());
  return order;
}

// The geometry records as the reference forms them on every call, in its
// operation order and in precision R (float for a float32 run, whose points
// are float32 there): barycentre ((p0 + p1) + p2) / 3 and face midpoint
// (pa + pb) / 2 (jnp.mean), normal (dy, -dx) / sqrt(dx dx + dy dy) and area
// |0.5 ((y1-y0)(x2-x0) - (x1-x0)(y2-y0))| (mesh.py:223-240), face offsets
// midpoint - barycentre (euler_solver.py:49,74,79), least-squares offsets
// (neighbour barycentre - own, or 2 (midpoint - own) on a boundary face),
// weights 1 / |dx|^2 and A = sum_k (w_k dx_k) dx_k^T summed k = 0, 1, 2 in
// turn (helper.py:136-150), sponge blend^3 with width 0.2 (y_max - y_min)
// (helper.py:262-295). The LSQ coefficients of the fast path are derived
// from these offsets in float64. Requires hm.perm / hm.inv / hm.nbr.
template <typename R>
static void reference_geometry(const esr_mesh_desc& d, const std::vector<int>& walls, HostMesh& hm,
                               std::vector<R>& geo, std::vector<LsqRef>* lsq, std::vector<R>& wall_n,
                               std::vector<R>& wall_ds) {
  const int N = d.n_cells, F = d.n_faces, P = d.n_points;
  std::vector<R> px(P), py(P);
  for (int p = 0; p < P; ++p) { px[p] = (R)d.points[2 * p]; py[p] = (R)d.points[2 * p + 1]; }
  std::vector<R> bx(N), by(N), area(N), nrm(6 * N), fmx(F), fmy(F), flen(F);
  for (int c = 0; c < N; ++c) {
    const int* t = d.tris + 3 * c;
    bx[c] = ((px[t[0]] + px[t[1]]) + px[t[2]]) / (R)3;
    by[c] = ((py[t[0]] + py[t[1]]) + py[t[2]]) / (R)3;
    const R cr = (py[t[1]] - py[t[0]]) * (px[t[2]] - px[t[0]]) - (px[t[1]] - px[t[0]]) * (py[t[2]] - py[t[0]]);
    area[c] = std::fabs((R)0.5 * cr);
    for (int k = 0; k < 3; ++k) {
      const R dx = px[t[(k + 1) % 3]] - px[t[k]], dy = py[t[(k + 1) % 3]] - py[t[k]];
      const R ln = std::sqrt(dx * dx + dy * dy);
      nrm[6 * c + 2 * k] = dy / ln;
      nrm[6 * c + 2 * k + 1] = (-dx) / ln;
    }
  }
  for (int f = 0; f < F; ++f) {
    const int a = d.faces[2 * f], b = d.faces[2 * f + 1];
    fmx[f] = (px[a] + px[b]) / (R)2;
    fmy[f] = (py[a] + py[b]) / (R)2;
    const R dx = px[b] - px[a], dy = py[b] - py[a];
    flen[f] = std::sqrt(dx * dx + dy * dy);
  }
  R ymin = py[0], ymax = py[0];
  for (int p = 1; p < P; ++p) { ymin = std::min(ymin, py[p]); ymax = std::max(ymax, py[p]); }
  const R Ly = ymax - ymin;
  const R width = d.sponge_width > 0 ? (R)d.sponge_width : (R)0.2 * Ly;
  geo.assign((size_t)G_COUNT * N, (R)0);
  if (lsq) lsq->assign(N, LsqRef{});
  for (int i = 0; i < N; ++i) {
    const int c = hm.perm[i];
    R* g = geo.data() + (size_t)i * G_COUNT;
    R dxk[3][2], w[3];
    for (int k = 0; k < 3; ++k) {
      const int f = d.face_connectivity[3 * c + k];
      const int j = d.neighbors[3 * c + k];
      const R ox = fmx[f] - bx[c], oy = fmy[f] - by[c];
      g[G_F0X + 2 * k] = ox;
      g[G_F0Y + 2 * k] = oy;
      g[G_N0X + 2 * k] = nrm[6 * c + 2 * k];
      g[G_N0Y + 2 * k] = nrm[6 * c + 2 * k + 1];
      g[G_S0 + k] = flen[f];
      if (d.face_markers[f] > 0) { dxk[k][0] = (R)2 * ox; dxk[k][1] = (R)2 * oy; }
      else { dxk[k][0] = bx[j] - bx[c]; dxk[k][1] = by[j] - by[c]; }
      const R ln = std::sqrt(dxk[k][0] * dxk[k][0] + dxk[k][1] * dxk[k][1]);
      w[k] = (R)1 / (ln * ln);
    }
    // A in the reference's order, then the fast path's c_k = w_k A^-1 dx_k in float64
    R a[4];
    for (int r = 0; r < 2; ++r)
      for (int q = 0; q < 2; ++q) {
        R acc = (w[0] * dxk[0][r]) * dxk[0][q];
        acc = acc + (w[1] * dxk[1][r]) * dxk[1][q];
        acc = acc + (w[2] * dxk[2][r]) * dxk[2][q];
        a[2 * r + q] = acc;
      }
    const double A00 = a[0], A01 = a[1], A10 = a[2], A11 = a[3];
    const double det = A00 * A11 - A01 * A10;
    for (int k = 0; k < 3; ++k) {
      const double wx = (double)w[k] * (double)dxk[k][0], wy = (double)w[k] * (double)dxk[k][1];
      g[G_C0X + 2 * k] = (R)((A11 * wx - A01 * wy) / det);
      g[G_C0Y + 2 * k] = (R)((-A10 * wx + A00 * wy) / det);
    }
    g[G_AREA] = area[c];
    R bl = 0;
    if (d.sponge) {
      const R y = by[c];
      const R dist = std::min(y - ymin, ymax - y);
      bl = std::min((R)1, std::max((R)0, (width - dist) / width));
      bl = std::pow(bl, (R)3);
    }
    g[G_BLEND3] = bl;
    if (lsq) {
      LsqRef& L = (*lsq)[i];
      for (int k = 0; k < 3; ++k) {
        L.w[k] = (float)w[k];
        L.dx[2 * k] = (float)dxk[k][0];
        L.dx[2 * k + 1] = (float)dxk[k][1];
      }
      for (int q = 0; q < 4; ++q) L.a[q] = (float)a[q];
    }
  }
  // force faces: the first slot listing each face, as prepare_mesh picks it
  const int fm = d.force_marker > 0 ? d.force_marker : 2;
  std::vector<int> first(F, -1);
  for (int t = 0; t < 3 * N; ++t)
    if (first[d.face_connectivity[t]] < 0) first[d.face_connectivity[t]] = t;
  wall_n.clear();
  wall_ds.clear();
  for (int f = 0; f < F; ++f) {
    if (d.face_markers[f] != fm || first[f] < 0) continue;
    const int c = first[f] / 3, k = first[f] % 3;
    wall_n.push_back(nrm[6 * c + 2 * k]);
    wall_n.push_back(nrm[6 * c + 2 * k + 1]);
    wall_ds.push_back(flen[f]);
  }
  (void)walls;
}

// Compact patches of at most kPatchCells cells, in the order of `seed`
// (reverse Cuthill-McKee): each patch grows from the first unassigned cell
// by adding, among the unassigned neighbours of the patch, the one with the
// most neighbours already inside it (ties: earliest in `seed`), so that most
// faces of a patch join two of its own cells. Cells are numbered patch by
// patch; patch_start[p] is the first cell of patch p (n_patches + 1 entries).
std::vector<int> patch_order(int n, const std::vector<int>& nbr, const std::vector<int>& seed,
                             std::vector<int>& patch_start) {
  std::vector<int> rank(n), owner(n, -1), order;
  for (int i = 0; i < n; ++i) rank[seed[i]] = i;
  order.reserve(n);
  patch_start.assign(1, 0);
  std::vector<int> members, cand, links(n, 0);
  for (int s0 : seed) {
    if (owner[s0] >= 0) continue;
    const int p = (int)patch_start.size() - 1;
    members.assign(1, s0);
    owner[s0] = p;
    cand.clear();
    auto add_nbrs = [&](int c) {
      for (int k = 0; k < 3; ++k) {
        const int j = nbr[3 * c + k];
        if (j < 0 || owner[j] >= 0) continue;
        if (links[j]++ == 0) cand.push_back(j);
      }
    };
    add_nbrs(s0);
    while ((int)members.size() < kPatchCells && !cand.empty()) {
      int best = -1;
      for (int i = 0; i < (int)cand.size(); ++i) {
        const int j = cand[i];
        if (best < 0 || links[j] > links[cand[best]] || (links[j] == links[cand[best]] && rank[j] < rank[cand[best]]))
          best = i;
      }
      const int c = cand[best];
      cand[best] = cand.back();
      cand.pop_back();
      links[c] = 0;
      owner[c] = p;
      members.push_back(c);
      add_nbrs(c);
    }
    for (int j : cand) links[j] = 0;
    for (int c : members) order.push_back(c);
    patch_start.push_back((int)order.size());
  }
  return order;
}

int prepare_mesh(const esr_mesh_desc& d, HostMesh& hm, std::string& err) {
  const int N = d.n_cells, F = d.n_faces, P = d.n_points;
  if (N <= 0 || F <= 0 || P <= 0 || !d.points || !d.tris || !d.neighbors || !d.faces || !d.face_markers ||
      !d.face_connectivity) {
    err = "mesh: missing arrays or empty mesh";
    return ESR_ERR_ARG;
  }
  std::vector<int> walls;
  if (d.wall_markers && d.n_wall_markers > 0) walls.assign(d.wall_markers, d.wall_markers + d.n_wall_markers);
  else walls.push_back(2);
  for (int i = 0; i < 3 * N; ++i) {
    if (d.tris[i] < 0 || d.tris[i] >= P) { err = "mesh: triangle vertex out of range"; return ESR_ERR_ARG; }
    if (d.neighbors[i] < -1 || d.neighbors[i] >= N) { err = "mesh: neighbour out of range"; return ESR_ERR_ARG; }
    if (d.face_connectivity[i] < 0 || d.face_connectivity[i] >= F) { err = "mesh: face id out of range"; return ESR_ERR_ARG; }
  }
  for (int f = 0; f < 2 * F; ++f)
    if (d.faces[f] < 0 || d.faces[f] >= P) { err = "mesh: face vertex out of range"; return ESR_ERR_ARG; }

  // renumbering: perm[new] = old
  std::vector<int> nb_old(d.neighbors, d.neighbors + 3 * N);
  hm.perm.resize(N);
  if (d.renumber) hm.perm = patch_order(N, nb_old, rcm_order(N, nb_old), hm.patch_start);
  else {
    std::iota(hm.perm.begin(), hm.perm.end(), 0);
    hm.patch_start.clear();   // consecutive cells in patches of kPatchCells
    for (int c = 0; c < N; c += kPatchCells) hm.patch_start.push_back(c);
    hm.patch_start.push_back(N);
  }
  if ((int)hm.perm.size() != N) { err = "mesh: renumbering lost cells"; return ESR_ERR_ARG; }
  hm.inv.assign(N, -1);
  for (int i = 0; i < N; ++i) hm.inv[hm.perm[i]] = i;

  hm.n_cells = N;
  hm.n_faces = F;
  hm.geo.assign((size_t)G_COUNT * N, 0.0);
  hm.nbr.assign((size_t)4 * N, 0);
  auto G = [&](int f, int c) -> double& { return hm.geo[(size_t)c * G_COUNT + f]; };

  // face geometry
  std::vector<double> fmid(2 * F), flen(F);
  for (int f = 0; f < F; ++f) {
    const double* a = d.points + 2 * d.faces[2 * f];
    const double* b = d.points + 2 * d.faces[2 * f + 1];
    fmid[2 * f] = 0.5 * (a[0] + b[0]);
    fmid[2 * f + 1] = 0.5 * (a[1] + b[1]);
    flen[f] = std::hypot(b[0] - a[0], b[1] - a[1]);
  }
  double ymin = std::numeric_limits<double>::infinity(), ymax = -ymin;
  for (int p = 0; p < P; ++p) {
    ymin = std::min(ymin, d.points[2 * p + 1]);
    ymax = std::max(ymax, d.points[2 * p + 1]);
  }
  hm.y_min = ymin;
  hm.y_max = ymax;
  const double width = d.sponge_width > 0 ? d.sponge_width : 0.2 * (ymax - ymin);

  // per old cell: barycentre, area, normals
  std::vector<double> bary(2 * N), area(N), nrm(6 * N);
  for (int c = 0; c < N; ++c) {
    const double* p[3];
    for (int k = 0; k < 3; ++k) p[k] = d.points + 2 * d.tris[3 * c + k];
    bary[2 * c] = (p[0][0] + p[1][0] + p[2][0]) / 3.0;
    bary[2 * c + 1] = (p[0][1] + p[1][1] + p[2][1]) / 3.0;
    const double cr = (p[1][1] - p[0][1]) * (p[2][0] - p[0][0]) - (p[1][0] - p[0][0]) * (p[2][1] - p[0][1]);
    area[c] = std::fabs(0.5 * cr);
    if (!(area[c] > 0)) { err = "mesh: degenerate triangle"; return ESR_ERR_ARG; }
    for (int k = 0; k < 3; ++k) {
      const double dx = p[(k + 1) % 3][0] - p[k][0], dy = p[(k + 1) % 3][1] - p[k][1];
      const double ln = std::hypot(dx, dy);
      nrm[6 * c + 2 * k] = dy / ln;
      nrm[6 * c + 2 * k + 1] = -dx / ln;
    }
  }

  int n_bnd = 0;
  for (int i = 0; i < N; ++i) {
    const int c = hm.perm[i];
    int packed = 0;
    int nbn[3];
    double dxk[3][2];
    for (int k = 0; k < 3; ++k) {
      const int f = d.face_connectivity[3 * c + k];
      const int m = d.face_markers[f];
      const int j = d.neighbors[3 * c + k];
      int kind;
      if (m == 0) {
        if (j < 0) { err = "mesh: interior face marker on a boundary edge"; return ESR_ERR_ARG; }
        kind = K_INTERIOR;
      } else if (m == 3) kind = K_INLET;
      else if (m == 4) kind = K_OUTLET;
      else if (m == 5) kind = K_SUBSONIC;
      else if (is_wall(m, walls)) kind = K_WALL;
      else { err = "mesh: unsupported boundary marker " + std::to_string(m) + " (periodic faces are not supported)"; return ESR_ERR_ARG; }
      int opp = 0;
      if (kind == K_INTERIOR) {
        int found = -1;
        for (int q = 0; q < 3; ++q)
          if (d.face_connectivity[3 * j + q] == f && d.neighbors[3 * j + q] == c) found = q;
        if (found < 0) { err = "mesh: neighbour does not list the shared face"; return ESR_ERR_ARG; }
        opp = found;
        nbn[k] = hm.inv[j];
        dxk[k][0] = bary[2 * j] - bary[2 * c];
        dxk[k][1] = bary[2 * j + 1] - bary[2 * c + 1];
      } else {
        ++n_bnd;
        nbn[k] = -1;
        dxk[k][0] = 2.0 * (fmid[2 * f] - bary[2 * c]);
        dxk[k][1] = 2.0 * (fmid[2 * f + 1] - bary[2 * c + 1]);
      }
      packed |= (kind & 7) << (6 * k);
      packed |= (opp & 3) << (6 * k + 3);
      G(G_F0X + 2 * k, i) = fmid[2 * f] - bary[2 * c];
      G(G_F0Y + 2 * k, i) = fmid[2 * f + 1] - bary[2 * c + 1];
      G(G_N0X + 2 * k, i) = nrm[6 * c + 2 * k];
      G(G_N0Y + 2 * k, i) = nrm[6 * c + 2 * k + 1];
      G(G_S0 + k, i) = flen[f];
    }
    // weighted least squares: A = sum w dx dx^T, c_k = w_k A^{-1} dx_k
    double a11 = 0, a12 = 0, a22 = 0, w[3];
    for (int k = 0; k < 3; ++k) {
      w[k] = 1.0 / (dxk[k][0] * dxk[k][0] + dxk[k][1] * dxk[k][1]);
      a11 += w[k] * dxk[k][0] * dxk[k][0];
      a12 += w[k] * dxk[k][0] * dxk[k][1];
      a22 += w[k] * dxk[k][1] * dxk[k][1];
    }
    const double det = a11 * a22 - a12 * a12;
    if (!(std::fabs(det) > 0)) { err = "mesh: singular least-squares system"; return ESR_ERR_ARG; }
    for (int k = 0; k < 3; ++k) {
      G(G_C0X + 2 * k, i) = w[k] * (a22 * dxk[k][0] - a12 * dxk[k][1]) / det;
      G(G_C0Y + 2 * k, i) = w[k] * (-a12 * dxk[k][0] + a11 * dxk[k][1]) / det;
    }
    G(G_AREA, i) = area[c];
    double bl = 0.0;
    if (d.sponge) {
      const double y = bary[2 * c + 1];
      const double dist = std::min(y - ymin, ymax - y);
      bl = std::min(1.0, std::max(0.0, (width - dist) / width));
      bl = bl * bl * bl;
    }
    G(G_BLEND3, i) = bl;
    hm.nbr[4 * i + 0] = nbn[0];
    hm.nbr[4 * i + 1] = nbn[1];
    hm.nbr[4 * i + 2] = nbn[2];
    hm.nbr[4 * i + 3] = packed;
  }
  hm.n_boundary_slots = n_bnd;

  // force faces: the first (cell, slot) in the caller's row-major order that
  // lists the face (helper.py:373-379)
  const int fm = d.force_marker > 0 ? d.force_marker : 2;
  std::vector<int> first(F, -1);
  for (int t = 0; t < 3 * N; ++t) {
    int f = d.face_connectivity[t];
    if (first[f] < 0) first[f] = t;
  }
  hm.wall_cell.clear();
  hm.wall_n.clear();
  hm.wall_ds.clear();
  for (int f = 0; f < F; ++f) {
    if (d.face_markers[f] != fm || first[f] < 0) continue;
    const int c = first[f] / 3, k = first[f] % 3;
    hm.wall_cell.push_back(hm.inv[c]);
    hm.wall_n.push_back(nrm[6 * c + 2 * k]);
    hm.wall_n.push_back(nrm[6 * c + 2 * k + 1]);
    hm.wall_ds.push_back(flen[f]);
  }
  for (int k = 0; k < 4; ++k) hm.inlet_subsonic[k] = d.inlet_subsonic[k];
  reference_geometry<float>(d, walls, hm, hm.geo_ref32, &hm.lsq_ref32, hm.wall_n_ref32, hm.wall_ds_ref32);
  reference_geometry<double>(d, walls, hm, hm.geo_ref64, nullptr, hm.wall_n_ref64, hm.wall_ds_ref64);
  return ESR_OK;
}

}  // namespace esr

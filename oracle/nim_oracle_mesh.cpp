// The oracle's own cylinder mesh (TEST INFRASTRUCTURE, the checker).
//
// A restatement of the reference's host-side mesh set-up that follows its
// loops and counters literally, so that the CPU baseline and the checks of
// the library's closed-form mesh builder have an input source of their own:
//   create_hollow            create_geometry.f90:321-622 (node, face, mesh
//                            and BC counters in the reference's loop order)
//   fill_global_geometry     create_geometry.f90:626-664 (faces renumbered
//                            BC by BC, cells collect faces and neighbours)
//   deform_nodes             general.f90:428-460 with
//   refine_walls_radial_order general.f90:463-484 and
//   create_hexagon_from_annulus_order_n_flipped_three_regions
//                            general.f90:700-722 (convert_circle_to_hexagon_mine
//                            general.f90:726-788)
// The cells' local frame is the one link_mesh (prepare_mesh.f90:47-132)
// propagates from cell 1 on this O-grid: xi1 = +r, xi2 = +theta, xi3 = +z,
// node k of a cell at corner (xi1, xi2, xi3) of the reference cube
// (create_mesh.f90:326-333).  The two-sided tanh clustering is not in the
// reference: it is the benchmark geometry's extension,
// r -> 0.5 (1 + tanh(b (r - 1/2)) / tanh(b/2)) on the normalised radius.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "nim_mesh.h"

namespace {

const double kMathPi = 3.14159265359;  // parameters.f90:31

// convert_circle_to_hexagon_mine (general.f90:726-788)
void circle_to_hexagon(double x1, double y1, double &x2, double &y2) {
  double theta = std::atan(y1 / x1);
  if (x1 < 0) theta = theta + kMathPi;
  const double R = std::sqrt(x1 * x1 + y1 * y1);
  x2 = x1;
  y2 = y1;
  // intersection of the hexagon side through (pp1, 0) with slope a1 and the
  // ray through (x1, y1)
  auto cut = [&](double pp1, double a1) {
    const double b1 = -1.0, c1 = 0.0 - a1 * pp1;
    const double a2 = y1 / x1, b2 = -1.0, c2 = 0.0;
    x2 = (b1 * c2 - b2 * c1) / (a1 * b2 - a2 * b1);
    y2 = (c1 * a2 - c2 * a1) / (a1 * b2 - a2 * b1);
  };
  const double t1 = kMathPi / 3.0, t2 = 2 * kMathPi / 3.0, t3 = 3 * kMathPi / 3.0, t4 = 4 * kMathPi / 3.0,
               t5 = 5 * kMathPi / 3.0;
  if (theta > 0.0 && theta < t1) {
    cut(R, (std::sin(0.0) - std::sin(t1)) / (std::cos(0.0) - std::cos(t1)));
  } else if (theta > t1 && theta < t2) {
    y2 = R * std::sin(t1);
    x2 = x1 * y2 / y1;
  } else if (theta > t2 && theta < t3) {
    cut(-R, (std::sin(t2) - std::sin(t3)) / (std::cos(t2) - std::cos(t3)));
  } else if (theta > t3 && theta < t4) {
    cut(-R, (std::sin(t3) - std::sin(t4)) / (std::cos(t3) - std::cos(t4)));
  } else if ((theta > t4 && theta < t5) || (theta > -t2 && theta < -t1)) {
    y2 = R * std::sin(t4);
    x2 = x1 * y2 / y1;
  } else if (theta > -t1 && theta < 0.0) {
    cut(R, (std::sin(-t1) - std::sin(0.0)) / (std::cos(-t1) - std::cos(0.0)));
  }
}

}  // namespace

extern "C" int nim_oracle_mesh_build(const nim_mesh_params *p, double *node_xyz, int32_t *meshes_nodes,
                                     int32_t *meshes_faces, int32_t *meshes_neighbors, int32_t *faces_bc,
                                     int32_t *bcs_faces, int32_t *bcs_faces_id, int32_t *bcs_faces_position,
                                     int32_t *bcs_faces_mesh_num) {
  const int n1 = p->n_theta, n2 = p->n_r, n3 = p->n_z;
  if (n1 < 6 || n2 < 3 || n3 < 3) return -1;
  const double R_i = p->R_i, R_o = p->R_o, H = p->L;
  const double cz = H / 2.0;  // create_hollow(R_i,R_o,L,0,0,L/2,...) (main.f90:36)
  // index helpers into the reference's (i,j,k) arrays, 1-based
  auto nid = [&](int i, int j, int k) { return (size_t)(i - 1) + n1 * ((size_t)(j - 1) + (n2 + 1) * (size_t)(k - 1)); };
  auto mid = [&](int i, int j, int k) { return (size_t)(i - 1) + n1 * ((size_t)(j - 1) + n2 * (size_t)(k - 1)); };
  auto fxid = [&](int i, int j, int k) { return (size_t)(i - 1) + n1 * ((size_t)(j - 1) + n2 * (size_t)(k - 1)); };
  auto fyid = [&](int i, int j, int k) { return (size_t)(i - 1) + n1 * ((size_t)(j - 1) + (n2 + 1) * (size_t)(k - 1)); };
  auto fzid = [&](int i, int j, int k) { return (size_t)(i - 1) + n1 * ((size_t)(j - 1) + n2 * (size_t)(k - 1)); };
  const size_t NN = (size_t)n1 * (n2 + 1) * (n3 + 1), NM = (size_t)n1 * n2 * n3;
  const size_t NF = 3 * NM + (size_t)n1 * n3 + (size_t)n1 * n2;

  // ---- nodes (create_geometry.f90:373-393); node number = loop counter
  const double PI = 4.0 * std::atan(1.0);
  const double dr = (R_o - R_i) / n2, dtheta = 2 * PI / n1, dz = H / n3;
  std::vector<int32_t> node_n(NN);
  int32_t counter = 0;
  for (int k = 1; k <= n3 + 1; ++k)
    for (int j = 1; j <= n2 + 1; ++j)
      for (int i = 1; i <= n1; ++i) {
        ++counter;
        const double tmp_r = R_i + (j - 1) * dr, tmp_theta = (i - 1) * dtheta;
        double *x = node_xyz + 3 * (size_t)(counter - 1);
        x[0] = tmp_r * std::cos(tmp_theta) + 0.0;  // + cx, cy (create_geometry.f90:598-603)
        x[1] = tmp_r * std::sin(tmp_theta) + 0.0;
        x[2] = (k - 1) * dz - H / 2.;
        node_n[nid(i, j, k)] = counter;
      }
  // ---- faces x, y, z in the reference's counter order (395-446)
  std::vector<int32_t> fx(NM), fy((size_t)n1 * (n2 + 1) * n3), fz((size_t)n1 * n2 * (n3 + 1));
  counter = 0;
  for (int k = 1; k <= n3; ++k)
    for (int j = 1; j <= n2; ++j)
      for (int i = 1; i <= n1; ++i) fx[fxid(i, j, k)] = ++counter;
  for (int k = 1; k <= n3; ++k)
    for (int j = 1; j <= n2 + 1; ++j)
      for (int i = 1; i <= n1; ++i) fy[fyid(i, j, k)] = ++counter;
  for (int k = 1; k <= n3 + 1; ++k)
    for (int j = 1; j <= n2; ++j)
      for (int i = 1; i <= n1; ++i) fz[fzid(i, j, k)] = ++counter;
  std::vector<int32_t> mesh_n(NM);
  counter = 0;
  for (int k = 1; k <= n3; ++k)
    for (int j = 1; j <= n2; ++j)
      for (int i = 1; i <= n1; ++i) mesh_n[mid(i, j, k)] = ++counter;

  // ---- BC lists with the faces' shared meshes (474-594)
  struct BcFace {
    int32_t face, m1, m2;
  };
  std::vector<BcFace> bc[6];
  for (int j = 1; j <= n2; ++j)
    for (int i = 1; i <= n1; ++i) bc[2].push_back({fz[fzid(i, j, 1)], mesh_n[mid(i, j, 1)], 0});
  for (int j = 1; j <= n2; ++j)
    for (int i = 1; i <= n1; ++i) bc[3].push_back({fz[fzid(i, j, n3 + 1)], mesh_n[mid(i, j, n3)], 0});
  for (int k = 1; k <= n3; ++k)
    for (int i = 1; i <= n1; ++i) bc[4].push_back({fy[fyid(i, 1, k)], mesh_n[mid(i, 1, k)], 0});
  for (int k = 1; k <= n3; ++k)
    for (int i = 1; i <= n1; ++i) bc[5].push_back({fy[fyid(i, n2 + 1, k)], mesh_n[mid(i, n2, k)], 0});
  for (int k = 1; k <= n3; ++k)
    for (int j = 1; j <= n2; ++j)
      for (int i = 1; i <= n1; ++i)
        bc[1].push_back({fx[fxid(i, j, k)], mesh_n[mid(i, j, k)], mesh_n[mid(i == 1 ? n1 : i - 1, j, k)]});
  for (int k = 1; k <= n3; ++k)
    for (int j = 2; j <= n2; ++j)
      for (int i = 1; i <= n1; ++i) bc[1].push_back({fy[fyid(i, j, k)], mesh_n[mid(i, j, k)], mesh_n[mid(i, j - 1, k)]});
  for (int k = 2; k <= n3; ++k)
    for (int j = 1; j <= n2; ++j)
      for (int i = 1; i <= n1; ++i) bc[1].push_back({fz[fzid(i, j, k)], mesh_n[mid(i, j, k)], mesh_n[mid(i, j, k - 1)]});

  // ---- fill_global_geometry (626-664): faces renumbered BC by BC
  std::vector<int32_t> renum(NF + 1, 0);
  int32_t cnt = 1;
  for (int b = 1; b <= 5; ++b)
    for (const BcFace &f : bc[b]) {
      renum[f.face] = cnt;
      faces_bc[cnt - 1] = b;
      ++cnt;
    }
  if ((size_t)(cnt - 1) != NF) return -1;

  // ---- deform_nodes (general.f90:428-460) on every node
  const double Roi = R_o - R_i;
  for (size_t n = 0; n < NN; ++n) {
    double x = node_xyz[3 * n], y = node_xyz[3 * n + 1];
    if (p->cluster != NIM_CLUSTER_NONE) {
      double r = std::sqrt(x * x + y * y) - R_i;
      double theta = std::atan(y / (x));
      if (x < 0) theta = theta + kMathPi;
      r = r / Roi;
      const double b1 = p->cluster_factor;
      if (p->cluster == NIM_CLUSTER_POWER) {
        if (r <= 0.5 && r > 0.) r = std::pow(2 * r, b1) / 2.;
        if (r > 0.5 && r < 1.) r = 1. - std::pow(-2. * (r - 1), b1) / 2.;
      } else {
        r = 0.5 * (1.0 + std::tanh(b1 * (r - 0.5)) / std::tanh(0.5 * b1));
      }
      r = (r * Roi + R_i);
      x = r * std::cos(theta);
      y = r * std::sin(theta);
    }
    if (p->hexagon) {
      const double Ri = p->blend_r1, Ro = p->blend_r2, ne = p->blend_n;
      const double R = std::sqrt(x * x + y * y);
      double p1, p2;
      circle_to_hexagon(x, y, p1, p2);
      if (R <= Ri) {
        x = p1;
        y = p2;
      } else if (R > Ri && R < Ro) {
        const double Rin = std::pow(Ri, ne), Ron = std::pow(Ro, ne), Rn = std::pow(R, ne);
        const double xn = -(x - p1) / (Rin - Ron) * Rn - (p1 * Ron - x * Rin) / (Rin - Ron);
        const double yn = -(y - p2) / (Rin - Ron) * Rn - (p2 * Ron - y * Rin) / (Rin - Ron);
        x = xn;
        y = yn;
      }
    }
    node_xyz[3 * n] = x;
    node_xyz[3 * n + 1] = y;
    node_xyz[3 * n + 2] = node_xyz[3 * n + 2] + cz;
  }

  // ---- cells in the link_mesh frame; faces and neighbours through the
  // renumbering
  for (int k = 1; k <= n3; ++k)
    for (int j = 1; j <= n2; ++j)
      for (int i = 1; i <= n1; ++i) {
        const size_t c = (size_t)mesh_n[mid(i, j, k)] - 1;
        const int ip = (i < n1) ? i + 1 : 1, im = (i > 1) ? i - 1 : n1;
        const int32_t nd[8] = {node_n[nid(i, j, k)],      node_n[nid(i, j + 1, k)],     node_n[nid(ip, j + 1, k)],
                               node_n[nid(ip, j, k)],     node_n[nid(i, j, k + 1)],     node_n[nid(i, j + 1, k + 1)],
                               node_n[nid(ip, j + 1, k + 1)], node_n[nid(ip, j, k + 1)]};
        std::memcpy(meshes_nodes + 8 * c, nd, sizeof(nd));
        const int32_t fc[6] = {renum[fy[fyid(i, j, k)]], renum[fy[fyid(i, j + 1, k)]], renum[fx[fxid(i, j, k)]],
                               renum[fx[fxid(ip, j, k)]], renum[fz[fzid(i, j, k)]], renum[fz[fzid(i, j, k + 1)]]};
        std::memcpy(meshes_faces + 6 * c, fc, sizeof(fc));
        const int32_t nb[6] = {j > 1 ? mesh_n[mid(i, j - 1, k)] : 0, j < n2 ? mesh_n[mid(i, j + 1, k)] : 0,
                               mesh_n[mid(im, j, k)], mesh_n[mid(ip, j, k)],
                               k > 1 ? mesh_n[mid(i, j, k - 1)] : 0, k < n3 ? mesh_n[mid(i, j, k + 1)] : 0};
        std::memcpy(meshes_neighbors + 6 * c, nb, sizeof(nb));
      }

  // ---- boundary lists of fill_global_arrays (geometry.f90:978-1032): the
  // BC 2..5 faces in their new numbers, the cell that owns each (its one
  // shared mesh) and the face's position among that cell's six faces
  size_t l = 0;
  for (int b = 2; b <= 5; ++b)
    for (const BcFace &f : bc[b]) {
      const int32_t face = renum[f.face], cell = f.m1 ? f.m1 : f.m2;
      int32_t where = 0;
      for (int q = 0; q < 6; ++q)
        if (meshes_faces[6 * (size_t)(cell - 1) + q] == face) where = q + 1;
      if (!where) return -1;
      bcs_faces[l] = face;
      bcs_faces_id[l] = b;
      bcs_faces_position[l] = where;
      bcs_faces_mesh_num[l] = cell;
      ++l;
    }
  return (l == 2 * (size_t)n1 * n2 + 2 * (size_t)n1 * n3) ? 0 : -1;
}

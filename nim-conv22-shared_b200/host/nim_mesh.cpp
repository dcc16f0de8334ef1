// Host mesh builder: the structured O-grid of the reference's cylinder case.
//
// Restates, for the single case the reference builds:
//   create_hollow            create_geometry.f90:321-622  (nodes, faces, BC lists)
//   fill_global_geometry     create_geometry.f90:626-664  (face renumbering in BC order)
//   deform_nodes             general.f90:428-460
//   refine_walls_radial_order general.f90:463-484
//   create_hexagon_from_annulus_order_n_flipped_three_regions general.f90:700-722
//   convert_circle_to_hexagon_mine general.f90:726-788
//   link_mesh orientation    prepare_mesh.f90:47-132, create_mesh.f90:413-495
//   fill_global_arrays       geometry.f90:978-1032
//
// link_mesh propagates the local frame of cell 1 by breadth-first search over
// shared faces and edges.  On this O-grid (orientable, no singular vertex) the
// result is the same frame in every cell: xi1 = +r (face 1 inner, face 2
// outer), xi2 = +theta (faces 3/4), xi3 = +z (faces 5 bottom / 6 top), with
// node k of a cell at the corner (xi1,xi2,xi3) of the reference cube drawing
// (create_mesh.f90:326-333).  That frame is written directly here; the face
// sort of mesh_arrange_faces picks it for cell 1 whenever n_theta >= 6.
#include <cmath>
#include <cstdint>
#include <cstring>
#include "nim_mesh.h"

namespace {

// parameters.f90:31 -- the reference's truncated pi, used by the deformation
// routines (create_hollow itself uses 4*atan(1)).
const double MATH_PI = 3.14159265359;

struct Grid {
  int n1, n2, n3;  // theta, r, z cells
  int64_t ninterior() const {
    return 3LL * n1 * n2 * n3 - (int64_t)n1 * n2 - (int64_t)n1 * n3;
  }
  // 1-based numbers, 1-based i,j,k as in create_hollow.
  int32_t node(int i, int j, int k) const { return i + n1 * ((j - 1) + (n2 + 1) * (k - 1)); }
  int32_t cell(int i, int j, int k) const { return i + n1 * ((j - 1) + n2 * (k - 1)); }
  // theta faces faces_x(i,j,k): all interior, numbered first.
  int32_t face_x(int i, int j, int k) const { return i + n1 * ((j - 1) + n2 * (k - 1)); }
  // radial faces faces_y(i,j',k), j' = 1..n2+1
  int32_t face_y(int i, int jp, int k) const {
    const int64_t NI = ninterior();
    if (jp == 1) return (int32_t)(NI + 2LL * n1 * n2 + i + n1 * (k - 1));
    if (jp == n2 + 1) return (int32_t)(NI + 2LL * n1 * n2 + (int64_t)n1 * n3 + i + n1 * (k - 1));
    return (int32_t)((int64_t)n1 * n2 * n3 + i + n1 * ((jp - 2) + (n2 - 1) * (k - 1)));
  }
  // axial faces faces_z(i,j,k'), k' = 1..n3+1
  int32_t face_z(int i, int j, int kp) const {
    const int64_t NI = ninterior();
    if (kp == 1) return (int32_t)(NI + i + n1 * (j - 1));
    if (kp == n3 + 1) return (int32_t)(NI + (int64_t)n1 * n2 + i + n1 * (j - 1));
    return (int32_t)((int64_t)n1 * n2 * n3 + (int64_t)n1 * (n2 - 1) * n3 + i +
                     n1 * ((j - 1) + n2 * (kp - 2)));
  }
};

// convert_circle_to_hexagon_mine, general.f90:726-788.  A point at angle theta
// on a circle of radius R moves along its ray onto the hexagon of
// circumradius R whose corners sit at multiples of 60 degrees.  Points exactly
// on a corner ray fall through every strict comparison and stay put.
void circle_to_hexagon(double x1, double y1, double *x2, double *y2) {
  double theta = std::atan(y1 / x1);
  if (x1 < 0) theta = theta + MATH_PI;
  const double R = std::sqrt(x1 * x1 + y1 * y1);
  *x2 = x1;
  *y2 = y1;
  auto line_cut = [&](double pp1, double a1) {
    const double pp2 = 0.0, b1 = -1.0, c1 = pp2 - a1 * pp1;
    const double a2 = y1 / x1, b2 = -1.0, c2 = 0.0;
    *x2 = (b1 * c2 - b2 * c1) / (a1 * b2 - a2 * b1);
    *y2 = (c1 * a2 - c2 * a1) / (a1 * b2 - a2 * b1);
  };
  if (theta > 0.0 && theta < MATH_PI / 3.0) {
    line_cut(R, (std::sin(0.0) - std::sin(MATH_PI / 3.0)) / (std::cos(0.0) - std::cos(MATH_PI / 3.0)));
  } else if (theta > MATH_PI / 3.0 && theta < 2 * MATH_PI / 3.0) {
    *y2 = R * std::sin(MATH_PI / 3.0);
    *x2 = x1 * (*y2) / y1;
  } else if (theta > 2 * MATH_PI / 3.0 && theta < 3 * MATH_PI / 3.0) {
    line_cut(-R, (std::sin(2 * MATH_PI / 3.0) - std::sin(3 * MATH_PI / 3.0)) /
                     (std::cos(2 * MATH_PI / 3.0) - std::cos(3 * MATH_PI / 3.0)));
  } else if (theta > 3 * MATH_PI / 3.0 && theta < 4 * MATH_PI / 3.0) {
    line_cut(-R, (std::sin(3 * MATH_PI / 3.0) - std::sin(4 * MATH_PI / 3.0)) /
                     (std::cos(3 * MATH_PI / 3.0) - std::cos(4 * MATH_PI / 3.0)));
  } else if ((theta > 4 * MATH_PI / 3.0 && theta < 5 * MATH_PI / 3.0) ||
             (theta > -(2 * MATH_PI / 3.0) && theta < -(MATH_PI / 3.0))) {
    *y2 = R * std::sin(4 * MATH_PI / 3.0);
    *x2 = x1 * (*y2) / y1;
  } else if (theta > -(MATH_PI / 3.0) && theta < 0.0) {
    line_cut(R, (std::sin(-(MATH_PI / 3.0)) - std::sin(0.0)) / (std::cos(-(MATH_PI / 3.0)) - std::cos(0.0)));
  }
}

}  // namespace

extern "C" void nim_mesh_params_reference(nim_mesh_params *p) {
  std::memset(p, 0, sizeof(*p));
  p->n_r = 6;                       // parameters.f90:87
  p->n_theta = 6 * p->n_r;          // parameters.f90:88
  p->n_z = 2 * p->n_r;              // parameters.f90:89
  p->R_i = 1.0 * (MATH_PI / 3.0);   // parameters.f90:90
  p->R_o = 2.0;                     // parameters.f90:91
  p->L = 2.0;                       // parameters.f90:92
  p->cluster = NIM_CLUSTER_POWER;   // general.f90:431
  p->cluster_factor = 1.5;
  p->hexagon = 1;                   // general.f90:434
  p->blend_r1 = 1.25;
  p->blend_r2 = 1.75;
  p->blend_n = -1.0;
}

extern "C" int nim_mesh_sizes(const nim_mesh_params *p, int32_t *nnode, int32_t *nmesh,
                              int32_t *nface, int32_t *nbcface) {
  if (!p || p->n_theta < 6 || p->n_r < 3 || p->n_z < 3) return NIM_ERR_BAD_ARG;
  const int64_t n1 = p->n_theta, n2 = p->n_r, n3 = p->n_z;
  const int64_t nn = n1 * (n2 + 1) * (n3 + 1);             // parameters.f90:119
  const int64_t nf = 3 * n1 * n2 * n3 + n1 * n3 + n1 * n2;  // parameters.f90:117
  if (nf > INT32_MAX || nn > INT32_MAX) return NIM_ERR_BAD_ARG;
  if (nnode) *nnode = (int32_t)nn;
  if (nmesh) *nmesh = (int32_t)(n1 * n2 * n3);
  if (nface) *nface = (int32_t)nf;
  if (nbcface) *nbcface = (int32_t)(2 * n1 * n2 + 2 * n1 * n3);
  return 0;
}

extern "C" int nim_mesh_build(const nim_mesh_params *p, double *node_xyz,
                              int32_t *meshes_nodes, int32_t *meshes_faces,
                              int32_t *meshes_neighbors, int32_t *faces_bc,
                              int32_t *bcs_faces, int32_t *bcs_faces_id,
                              int32_t *bcs_faces_position, int32_t *bcs_faces_mesh_num) {
  int32_t nnode, nmesh, nface, nbc;
  if (nim_mesh_sizes(p, &nnode, &nmesh, &nface, &nbc) != 0) return NIM_ERR_BAD_ARG;
  if (!node_xyz || !meshes_nodes || !meshes_faces || !meshes_neighbors || !faces_bc ||
      !bcs_faces || !bcs_faces_id || !bcs_faces_position || !bcs_faces_mesh_num)
    return NIM_ERR_BAD_ARG;
  if (!(p->R_o > p->R_i) || !(p->R_i > 0) || !(p->L > 0)) return NIM_ERR_BAD_ARG;
  const Grid g{p->n_theta, p->n_r, p->n_z};
  const int n1 = g.n1, n2 = g.n2, n3 = g.n3;

  // ---- nodes: create_hollow(R_i,R_o,L,0,0,L/2,...), create_geometry.f90:343-395
  const double PI = 4.0 * std::atan(1.0);
  const double H = p->L, cz = p->L / 2.0;
  const double dr = (p->R_o - p->R_i) / n2;
  const double dtheta = 2 * PI / n1;
  const double dz = H / n3;
  for (int k = 1; k <= n3 + 1; ++k)
    for (int j = 1; j <= n2 + 1; ++j)
      for (int i = 1; i <= n1; ++i) {
        const double tmp_r = p->R_i + (j - 1) * dr;
        const double tmp_theta = (i - 1) * dtheta;
        const int64_t n = g.node(i, j, k) - 1;
        node_xyz[3 * n + 0] = tmp_r * std::cos(tmp_theta) + 0.0;
        node_xyz[3 * n + 1] = tmp_r * std::sin(tmp_theta) + 0.0;
        node_xyz[3 * n + 2] = ((k - 1) * dz - H / 2.0) + cz;
      }

  // ---- deform_nodes, general.f90:428-460
  const double Roi = p->R_o - p->R_i;
  for (int64_t n = 0; n < nnode; ++n) {
    double x = node_xyz[3 * n + 0], y = node_xyz[3 * n + 1];
    if (p->cluster != NIM_CLUSTER_NONE) {
      // refine_walls_radial_order, general.f90:463-484 (power law), or the
      // tanh extension mapping r in [0,1] to 0.5*(1+tanh(b(r-1/2))/tanh(b/2)).
      double r = std::sqrt(x * x + y * y) - p->R_i;
      double theta = std::atan(y / x);
      if (x < 0) theta = theta + MATH_PI;
      r = r / Roi;
      const double b1 = p->cluster_factor;
      if (p->cluster == NIM_CLUSTER_POWER) {
        if (r <= 0.5 && r > 0.0) r = std::pow(2 * r, b1) / 2.0;
        if (r > 0.5 && r < 1.0) r = 1.0 - std::pow(-(2.0 * (r - 1)), b1) / 2.0;
      } else {
        r = 0.5 * (1.0 + std::tanh(b1 * (r - 0.5)) / std::tanh(0.5 * b1));
      }
      r = (r * Roi + p->R_i);
      x = r * std::cos(theta);
      y = r * std::sin(theta);
    }
    if (p->hexagon) {
      // create_hexagon_from_annulus_order_n_flipped_three_regions(Ri,Ro,n)
      const double Ri = p->blend_r1, Ro = p->blend_r2, ne = p->blend_n;
      const double R = std::sqrt(x * x + y * y);
      double p1, p2;
      circle_to_hexagon(x, y, &p1, &p2);
      if (R <= Ri) {
        x = p1;
        y = p2;
      } else if (R > Ri && R < Ro) {
        const double Rin = std::pow(Ri, ne), Ron = std::pow(Ro, ne), Rn = std::pow(R, ne);
        const double xn = -((x - p1) / (Rin - Ron) * Rn) - (p1 * Ron - x * Rin) / (Rin - Ron);
        const double yn = -((y - p2) / (Rin - Ron) * Rn) - (p2 * Ron - y * Rin) / (Rin - Ron);
        x = xn;
        y = yn;
      }
    }
    node_xyz[3 * n + 0] = x;
    node_xyz[3 * n + 1] = y;
  }

  // ---- cells: arranged nodes, faces and neighbours in the link_mesh frame
  for (int k = 1; k <= n3; ++k)
    for (int j = 1; j <= n2; ++j)
      for (int i = 1; i <= n1; ++i) {
        const int64_t c = g.cell(i, j, k) - 1;
        const int ip = (i % n1) + 1, im = (i == 1) ? n1 : i - 1;
        int32_t *nd = meshes_nodes + 8 * c;
        nd[0] = g.node(i, j, k);
        nd[1] = g.node(i, j + 1, k);
        nd[2] = g.node(ip, j + 1, k);
        nd[3] = g.node(ip, j, k);
        nd[4] = g.node(i, j, k + 1);
        nd[5] = g.node(i, j + 1, k + 1);
        nd[6] = g.node(ip, j + 1, k + 1);
        nd[7] = g.node(ip, j, k + 1);
        int32_t *fc = meshes_faces + 6 * c;
        fc[0] = g.face_y(i, j, k);
        fc[1] = g.face_y(i, j + 1, k);
        fc[2] = g.face_x(i, j, k);
        fc[3] = g.face_x(ip, j, k);
        fc[4] = g.face_z(i, j, k);
        fc[5] = g.face_z(i, j, k + 1);
        int32_t *nb = meshes_neighbors + 6 * c;
        nb[0] = (j > 1) ? g.cell(i, j - 1, k) : 0;
        nb[1] = (j < n2) ? g.cell(i, j + 1, k) : 0;
        nb[2] = g.cell(im, j, k);
        nb[3] = g.cell(ip, j, k);
        nb[4] = (k > 1) ? g.cell(i, j, k - 1) : 0;
        nb[5] = (k < n3) ? g.cell(i, j, k + 1) : 0;
      }

  // ---- face BC ids (faces_BC) and the boundary lists of fill_global_arrays
  const int64_t NI = g.ninterior();
  for (int64_t f = 0; f < nface; ++f) faces_bc[f] = (f < NI) ? 1 : 0;
  int64_t l = 0;
  auto add = [&](int32_t face, int32_t id, int32_t pos, int32_t cell) {
    bcs_faces[l] = face;
    bcs_faces_id[l] = id;
    bcs_faces_position[l] = pos;
    bcs_faces_mesh_num[l] = cell;
    faces_bc[face - 1] = id;
    ++l;
  };
  for (int j = 1; j <= n2; ++j)  // BC 2 bottom, create_geometry.f90:476-487
    for (int i = 1; i <= n1; ++i) add(g.face_z(i, j, 1), 2, 5, g.cell(i, j, 1));
  for (int j = 1; j <= n2; ++j)  // BC 3 top
    for (int i = 1; i <= n1; ++i) add(g.face_z(i, j, n3 + 1), 3, 6, g.cell(i, j, n3));
  for (int k = 1; k <= n3; ++k)  // BC 4 inner (hexagon)
    for (int i = 1; i <= n1; ++i) add(g.face_y(i, 1, k), 4, 1, g.cell(i, 1, k));
  for (int k = 1; k <= n3; ++k)  // BC 5 outer
    for (int i = 1; i <= n1; ++i) add(g.face_y(i, n2 + 1, k), 5, 2, g.cell(i, n2, k));
  return (l == nbc) ? 0 : NIM_ERR_BAD_ARG;
}

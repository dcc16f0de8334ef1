// Shared device-side definitions of the NIM library: structured indexing of
// the O-grid, the 5-point Gauss rule, the curvilinear metric evaluation and
// the gfortran integer-power chains.
//
// Layout in HBM (FP64, structure of arrays, theta fastest):
//   cell c = i + NT*(j + NR*k)          i: theta (xi2), j: r (xi1), k: z (xi3)
//   face arrays of one field hold NF = 3*NT*NR*NZ + NT*NZ + NT*NR doubles:
//     radial faces  [0, offT)        fR(i,j',k) = i + NT*(j' + (NR+1)*k), j'=0..NR
//     theta faces   [offT, offZ)     fT(i',j,k) = offT + i' + NT*(j + NR*k)
//     axial faces   [offZ, NF)       fZ(i,j,k') = offZ + i + NT*(j + NR*k'), k'=0..NZ
//   so the six faces of cell c are
//     f1 = c + NT*k, f2 = f1 + NT, f3 = offT + c, f4 = offT + c - i + ip,
//     f5 = offZ + c, f6 = f5 + NT*NR.
// Local axes follow link_mesh (prepare_mesh.f90:47-132): face 1/2 = -/+ r,
// 3/4 = -/+ theta (periodic), 5/6 = -/+ z; neighbour 0 means a wall.
#pragma once
#include <cstdint>

namespace nim {

struct Dims {
  int NT, NR, NZ;   // cells in theta, r, z
  int Nc;           // NT*NR*NZ
  int offT, offZ;   // start of theta / axial faces in a face array
  int NF;           // faces
  int NBF;          // boundary faces (2*NT*NR + 2*NT*NZ)
  int plane;        // NT*NR
  // cell planes [kown0, kown1) this context owns: the maxima of find_error,
  // check_steady_state and the wall and dilatation sums cover only these.
  // All planes, except in a z-slab, whose outer two planes on a side with a
  // neighbour slab are halo copies of that neighbour's cells.
  int kown0, kown1;
  __host__ __device__ bool owns(int k) const { return k >= kown0 && k < kown1; }
};

struct Cell {
  int i, j, k, c;
  __host__ __device__ static Cell of(const Dims &d, int c) {
    Cell x;
    x.c = c;
    x.i = c % d.NT;
    const int q = c / d.NT;
    x.j = q % d.NR;
    x.k = q / d.NR;
    return x;
  }
  __host__ __device__ static Cell at(const Dims &d, int i, int j, int k) {
    Cell x;
    x.i = i; x.j = j; x.k = k;
    x.c = i + d.NT * (j + d.NR * k);
    return x;
  }
  // neighbour across face pos (1..6); valid() false at a wall
  __host__ __device__ Cell nb(const Dims &d, int pos) const {
    switch (pos) {
      case 1: return at(d, i, j - 1, k);
      case 2: return at(d, i, j + 1, k);
      case 3: return at(d, (i == 0) ? d.NT - 1 : i - 1, j, k);
      case 4: return at(d, (i == d.NT - 1) ? 0 : i + 1, j, k);
      case 5: return at(d, i, j, k - 1);
      default: return at(d, i, j, k + 1);
    }
  }
  __host__ __device__ bool has_nb(const Dims &d, int pos) const {
    switch (pos) {
      case 1: return j > 0;
      case 2: return j < d.NR - 1;
      case 5: return k > 0;
      case 6: return k < d.NZ - 1;
      default: return true;
    }
  }
  // index of face pos (1..6) of this cell in a face array
  __host__ __device__ int face(const Dims &d, int pos) const {
    switch (pos) {
      case 1: return c + d.NT * k;
      case 2: return c + d.NT * k + d.NT;
      case 3: return d.offT + c;
      case 4: return d.offT + c - i + ((i == d.NT - 1) ? 0 : i + 1);
      case 5: return d.offZ + c;
      default: return d.offZ + c + d.plane;
    }
  }
};

__host__ inline Dims make_dims(int NT, int NR, int NZ) {
  Dims d;
  d.NT = NT; d.NR = NR; d.NZ = NZ;
  d.Nc = NT * NR * NZ;
  d.plane = NT * NR;
  d.offT = NT * (NR + 1) * NZ;
  d.offZ = d.offT + d.Nc;
  d.NF = d.offZ + NT * NR * (NZ + 1);
  d.NBF = 2 * NT * NR + 2 * NT * NZ;
  d.kown0 = 0;
  d.kown1 = NZ;
  return d;
}

// Boundary faces in the reference's BC-list order (fill_global_arrays):
// bottom (position 5, BC 2) by (j,i), top (6, BC 3) by (j,i), inner hexagon
// (1, BC 4) by (k,i), outer wall (2, BC 5) by (k,i).
struct BFace {
  Cell cell;
  int pos;  // position of the wall face in its cell
  int id;   // BC id
};
__host__ __device__ inline BFace bface(const Dims &d, int b) {
  BFace r;
  const int nb1 = d.NT * d.NR;
  if (b < nb1) {
    r.cell = Cell::at(d, b % d.NT, b / d.NT, 0); r.pos = 5; r.id = 2;
  } else if (b < 2 * nb1) {
    const int q = b - nb1;
    r.cell = Cell::at(d, q % d.NT, q / d.NT, d.NZ - 1); r.pos = 6; r.id = 3;
  } else if (b < 2 * nb1 + d.NT * d.NZ) {
    const int q = b - 2 * nb1;
    r.cell = Cell::at(d, q % d.NT, 0, q / d.NT); r.pos = 1; r.id = 4;
  } else {
    const int q = b - 2 * nb1 - d.NT * d.NZ;
    r.cell = Cell::at(d, q % d.NT, d.NR - 1, q / d.NT); r.pos = 2; r.id = 5;
  }
  return r;
}

// x^n for the constant exponents of nim.f90's series, multiplied in the order
// gfortran's gfc_conv_powi emits (x^n = x^(n-t[n]) * x^t[n]).
template <class V>
struct PwT {
  V p[13];
  __host__ __device__ explicit PwT(V x) {
    p[0] = 1.0; p[1] = x;
    p[2] = p[1] * p[1]; p[3] = p[1] * p[2]; p[4] = p[2] * p[2];
    p[5] = p[2] * p[3]; p[6] = p[3] * p[3]; p[7] = p[3] * p[4];
    p[8] = p[4] * p[4]; p[9] = p[3] * p[6]; p[10] = p[5] * p[5];
    p[11] = p[5] * p[6]; p[12] = p[6] * p[6];
  }
  __host__ __device__ V operator[](int n) const { return p[n]; }
};
using Pw = PwT<double>;

// 5-point Gauss-Legendre rule (parameters.f90:18-22), filled once from the
// host with the same expressions.
struct GaussRule {
  double x[5], w[5];
};

// Trilinear cell map (create_mesh.f90:254-303): C, D, E coefficient arrays.
struct Map {
  double C[8], D[8], E[8];
};

__device__ __forceinline__ double det3(const double a[3][3]) {
  return a[0][0] * a[1][1] * a[2][2] + a[0][1] * a[1][2] * a[2][0] + a[0][2] * a[1][0] * a[2][1] -
         a[0][2] * a[1][1] * a[2][0] - a[0][1] * a[1][0] * a[2][2] - a[0][0] * a[1][2] * a[2][1];
}

__device__ __forceinline__ void inv3(const double a[3][3], double x[3][3]) {
  const double s = 1.0 / det3(a);
  x[0][0] = s * (a[1][1] * a[2][2] - a[2][1] * a[1][2]);
  x[0][1] = s * (a[0][2] * a[2][1] - a[0][1] * a[2][2]);
  x[0][2] = s * (a[0][1] * a[1][2] - a[0][2] * a[1][1]);
  x[1][0] = s * (a[1][2] * a[2][0] - a[1][0] * a[2][2]);
  x[1][1] = s * (a[0][0] * a[2][2] - a[0][2] * a[2][0]);
  x[1][2] = s * (a[0][2] * a[1][0] - a[0][0] * a[1][2]);
  x[2][0] = s * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
  x[2][1] = s * (a[0][1] * a[2][0] - a[0][0] * a[2][1]);
  x[2][2] = s * (a[0][0] * a[1][1] - a[0][1] * a[1][0]);
}

template <class V>
__device__ __forceinline__ V dot3(const V *a, const V *b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

// Everything evaluate_curvilinear (curvilinear.f90:9-41) produces that the
// hot path consumes.
struct Curvi {
  double x, y, z;
  double jac[3][3];     // jacmat(r,c) = d x_c / d xi_r (rows: covariant g_r)
  double jacinv[3][3];  // columns: contravariant g^a
  double detJ;
};

__device__ __forceinline__ void curvi_point(const Map &M, double x, double y, double z, Curvi &C) {
  const double *Cc = M.C, *Dd = M.D, *Ee = M.E;
  C.x = Cc[0] + Cc[1] * x + Cc[2] * y + Cc[3] * z + Cc[4] * x * y + Cc[5] * x * z + Cc[6] * y * z + Cc[7] * x * y * z;
  C.y = Dd[0] + Dd[1] * x + Dd[2] * y + Dd[3] * z + Dd[4] * x * y + Dd[5] * x * z + Dd[6] * y * z + Dd[7] * x * y * z;
  C.z = Ee[0] + Ee[1] * x + Ee[2] * y + Ee[3] * z + Ee[4] * x * y + Ee[5] * x * z + Ee[6] * y * z + Ee[7] * x * y * z;
  C.jac[0][0] = Cc[1] + Cc[4] * y + Cc[5] * z + Cc[7] * y * z;
  C.jac[0][1] = Dd[1] + Dd[4] * y + Dd[5] * z + Dd[7] * y * z;
  C.jac[0][2] = Ee[1] + Ee[4] * y + Ee[5] * z + Ee[7] * y * z;
  C.jac[1][0] = Cc[2] + Cc[4] * x + Cc[6] * z + Cc[7] * x * z;
  C.jac[1][1] = Dd[2] + Dd[4] * x + Dd[6] * z + Dd[7] * x * z;
  C.jac[1][2] = Ee[2] + Ee[4] * x + Ee[6] * z + Ee[7] * x * z;
  C.jac[2][0] = Cc[3] + Cc[5] * x + Cc[6] * y + Cc[7] * x * y;
  C.jac[2][1] = Dd[3] + Dd[5] * x + Dd[6] * y + Dd[7] * x * y;
  C.jac[2][2] = Ee[3] + Ee[5] * x + Ee[6] * y + Ee[7] * x * y;
  inv3(C.jac, C.jacinv);
  C.detJ = det3(C.jac);
}

// contravariant metric g^ab = g^a . g^b (gij_matrix, curvilinear.f90:87-104)
__device__ __forceinline__ double gup(const Curvi &C, int a, int b) {
  return C.jacinv[0][a] * C.jacinv[0][b] + C.jacinv[1][a] * C.jacinv[1][b] + C.jacinv[2][a] * C.jacinv[2][b];
}
// covariant metric g_ab = g_a . g_b (g_ij_matrix, curvilinear.f90:66-79)
__device__ __forceinline__ double glow(const Curvi &C, int a, int b) {
  return C.jac[a][0] * C.jac[b][0] + C.jac[a][1] * C.jac[b][1] + C.jac[a][2] * C.jac[b][2];
}

// local coordinates of a point of face fn (1..6) with in-face coordinates a,b
__host__ __device__ __forceinline__ void face_point(int fn, double a, double b, double &x, double &y, double &z) {
  const double s = (fn % 2 == 1) ? -1.0 : 1.0;
  if (fn <= 2) { x = s; y = a; z = b; }
  else if (fn <= 4) { x = a; y = s; z = b; }
  else { x = a; y = b; z = s; }
}

// transverse directions of direction d (1..3): e1 < e2
__host__ __device__ __forceinline__ int tr1(int d) { return d == 1 ? 2 : 1; }
__host__ __device__ __forceinline__ int tr2(int d) { return d == 3 ? 2 : 3; }

}  // namespace nim

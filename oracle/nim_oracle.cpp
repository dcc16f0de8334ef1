// CPU oracle of the NIM time advance -- TEST INFRASTRUCTURE ONLY.
//
// A line-by-line C++ restatement of the reference's live FP64 path.  Arrays
// keep the Fortran layout (component, 1-based index) so that every formula can
// be compared with its source line.  Expressions keep Fortran's evaluation
// order (left to right, parentheses respected, no contraction: built with
// -ffp-contract=off), and integer powers use gfortran's fixed multiplication
// chains (gfc_conv_powi), so the arithmetic is the reference's up to libm.
//
// Parity is unpinned: the reference has no tests or golden data and cannot be
// compiled here (no Fortran compiler).  See nim_oracle.h.
#include "nim_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif
#ifdef NIM_ORACLE_TANGENT
#include "nim_dual.h"
#endif

// The scalar of every value the time advance computes: real, or in the
// tangent-linear build (nim_oracle_tl.cpp) a Dual carrying the value and its
// derivative along the seeded direction.  The values are the same bits in
// both builds.
#ifdef NIM_ORACLE_TANGENT
using real = nimtl::Dual;
using nimtl::tan_of;
using nimtl::val;
#define nim_oracle nim_oracle_tl  // a type of its own in the tangent build
#define NIM_ORACLE_FN(name) nim_oracle_tl_##name
#else
using real = double;
inline double val(double a) { return a; }
inline double tan_of(double) { return 0.0; }
#define NIM_ORACLE_FN(name) nim_oracle_##name
#endif

namespace {

// ------------------------------------------------------------------ arrays
// 1-based vectors: a(i) with i = 1..n, and (K, n) column-major blocks.
struct V1 {
  std::vector<real> d;
  void alloc(int64_t n) { d.assign(n + 1, 0.0); }
  real &operator()(int64_t i) { return d[i]; }
  const real &operator()(int64_t i) const { return d[i]; }
};
template <int K>
struct VK {
  std::vector<real> d;
  void alloc(int64_t n) { d.assign((size_t)K * (n + 1), 0.0); }
  real &operator()(int k, int64_t i) { return d[(size_t)K * i + (k - 1)]; }
  const real &operator()(int k, int64_t i) const { return d[(size_t)K * i + (k - 1)]; }
};
template <int K>
struct IK {
  std::vector<int32_t> d;
  void alloc(int64_t n) { d.assign((size_t)K * (n + 1), 0); }
  int32_t &operator()(int k, int64_t i) { return d[(size_t)K * i + (k - 1)]; }
  const int32_t &operator()(int k, int64_t i) const { return d[(size_t)K * i + (k - 1)]; }
};
// (3,3,n) and (3,3,6,n) blocks
struct M33 {
  std::vector<real> d;
  void alloc(int64_t n) { d.assign((size_t)9 * (n + 1), 0.0); }
  real &operator()(int a, int b, int64_t i) { return d[(size_t)9 * i + (a - 1) + 3 * (b - 1)]; }
  const real &operator()(int a, int b, int64_t i) const { return d[(size_t)9 * i + (a - 1) + 3 * (b - 1)]; }
};
struct M336 {
  std::vector<real> d;
  void alloc(int64_t n) { d.assign((size_t)54 * (n + 1), 0.0); }
  real &operator()(int a, int b, int f, int64_t i) {
    return d[(size_t)54 * i + (a - 1) + 3 * (b - 1) + 9 * (f - 1)];
  }
  const real &operator()(int a, int b, int f, int64_t i) const {
    return d[(size_t)54 * i + (a - 1) + 3 * (b - 1) + 9 * (f - 1)];
  }
};
struct M36 {  // (3,6,n)
  std::vector<real> d;
  void alloc(int64_t n) { d.assign((size_t)18 * (n + 1), 0.0); }
  real &operator()(int a, int b, int64_t i) { return d[(size_t)18 * i + (a - 1) + 3 * (b - 1)]; }
  const real &operator()(int a, int b, int64_t i) const { return d[(size_t)18 * i + (a - 1) + 3 * (b - 1)]; }
};

// ------------------------------------------------------------- arithmetic
// x**n for constant integer n the way gfortran expands it (gfc_conv_powi and
// its powi_table: x^n = x^(n-t[n]) * x^t[n]).
struct Pw {
  real p[13];
  explicit Pw(real x) {
    p[0] = 1.0;
    p[1] = x;
    p[2] = p[1] * p[1];
    p[3] = p[1] * p[2];
    p[4] = p[2] * p[2];
    p[5] = p[2] * p[3];
    p[6] = p[3] * p[3];
    p[7] = p[3] * p[4];
    p[8] = p[4] * p[4];
    p[9] = p[3] * p[6];
    p[10] = p[5] * p[5];
    p[11] = p[5] * p[6];
    p[12] = p[6] * p[6];
  }
  real operator[](int n) const { return p[n]; }
};

// det and inv3x3 of general.f90:840-857 on a 0-based 3x3 a[r][c].
inline real det3(const real a[3][3]) {
  return a[0][0] * a[1][1] * a[2][2] + a[0][1] * a[1][2] * a[2][0] + a[0][2] * a[1][0] * a[2][1] -
         a[0][2] * a[1][1] * a[2][0] - a[0][1] * a[1][0] * a[2][2] - a[0][0] * a[1][2] * a[2][1];
}
inline void inv3(const real a[3][3], real x[3][3]) {
  const real s = 1 / det3(a);
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
inline real dot3(const real *a, const real *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// 5-point Gauss-Legendre rule, parameters.f90:18-22
struct Gauss {
  real x[5], w[5];
  Gauss() {
    x[0] = -(1. / 3. * sqrt(5. - 2. * sqrt(10. / 7.)));
    x[1] = 1. / 3. * sqrt(5. - 2. * sqrt(10. / 7.));
    x[2] = 0.;
    x[3] = -(1. / 3. * sqrt(5. + 2. * sqrt(10. / 7.)));
    x[4] = 1. / 3. * sqrt(5. + 2. * sqrt(10. / 7.));
    w[0] = (322. + 13. * sqrt(70.)) / 900.;
    w[1] = (322. + 13. * sqrt(70.)) / 900.;
    w[2] = 128. / 225.;
    w[3] = (322. - 13. * sqrt(70.)) / 900.;
    w[4] = (322. - 13. * sqrt(70.)) / 900.;
  }
};
const Gauss GQ;

// Trilinear map of one cell: mesh%C, %D, %E (create_mesh.f90:254-303).
struct Map {
  real C[8], D[8], E[8];
};

// type curvi3d filled by evaluate_curvilinear (curvilinear.f90:9-41).
struct Curvi {
  real x, y, z;
  real jac[3][3];     // jacmat(r,c) = d x_c / d xi_r
  real jacinv[3][3];  // inv3x3(jacmat)
  real g_ij[3][3];    // covariant metric
  real gij[3][3];     // contravariant metric
  real gam[3][3][3];  // gamma_tensor
  real detJ;
};

void evaluate_curvilinear(const Map &M, real x, real y, real z, Curvi &C) {
  const real *Cc = M.C, *Dd = M.D, *Ee = M.E;
  C.x = Cc[0] + Cc[1] * x + Cc[2] * y + Cc[3] * z + Cc[4] * x * y + Cc[5] * x * z + Cc[6] * y * z + Cc[7] * x * y * z;
  C.y = Dd[0] + Dd[1] * x + Dd[2] * y + Dd[3] * z + Dd[4] * x * y + Dd[5] * x * z + Dd[6] * y * z + Dd[7] * x * y * z;
  C.z = Ee[0] + Ee[1] * x + Ee[2] * y + Ee[3] * z + Ee[4] * x * y + Ee[5] * x * z + Ee[6] * y * z + Ee[7] * x * y * z;
  // jacobian_matrix, curvilinear.f90:44-63
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
  // g_a = jacmat(a,:) (covariant), g^a = jacinv(:,a) (contravariant)
  real gl[3][3], gu[3][3];
  for (int a = 0; a < 3; ++a)
    for (int c = 0; c < 3; ++c) {
      gl[a][c] = C.jac[a][c];
      gu[a][c] = C.jacinv[c][a];
    }
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      C.g_ij[a][b] = dot3(gl[a], gl[b]);
      C.gij[a][b] = dot3(gu[a], gu[b]);
    }
  // find_gamma_tensor, curvilinear.f90:109-160
  const real g1_2[3] = {Cc[4] + Cc[7] * z, Dd[4] + Dd[7] * z, Ee[4] + Ee[7] * z};
  const real g1_3[3] = {Cc[5] + Cc[7] * y, Dd[5] + Dd[7] * y, Ee[5] + Ee[7] * y};
  const real g2_3[3] = {Cc[6] + Cc[7] * x, Dd[6] + Dd[7] * x, Ee[6] + Ee[7] * x};
  for (int a = 0; a < 3; ++a) {
    const real a12 = dot3(gu[a], g1_2), a13 = dot3(gu[a], g1_3), a23 = dot3(gu[a], g2_3);
    C.gam[a][0][0] = 0.;
    C.gam[a][0][1] = a12;
    C.gam[a][0][2] = a13;
    C.gam[a][1][0] = a12;
    C.gam[a][1][1] = 0.;
    C.gam[a][1][2] = a23;
    C.gam[a][2][0] = a13;
    C.gam[a][2][1] = a23;
    C.gam[a][2][2] = 0.;
  }
  C.detJ = det3(C.jac);
}

inline real sq(real x) { return x * x; }

}  // namespace

// ======================================================================
struct nim_oracle {
  int sched = NIM_SCHED_SEQUENTIAL;
  int nthreads = 1;
  nim_params P{};
  int64_t NMESH = 0, NFACE = 0, NNODE = 0, NBF = 0;
  real nu = 0, alpha = 0;  // P.nu, P.alpha: the tangent build seeds their derivatives
  real Re = 0, inv_Re = 0;
  bool initialized = false;
  bool first_iteration = true;
  int32_t STEP = 0;
  real TI = 0;
  double max_rc = 0;
  double nu_tan[2] = {0, 0};  // derivatives of Nu_inner, Nu_outer at the last end_step

  // mesh (Fortran layout, 1-based)
  std::vector<real> node_xyz;  // (3, NNODE) 0-based storage
  IK<8> mnodes;
  IK<6> mfaces, mnb;
  std::vector<int32_t> faces_BC;  // 1-based
  std::vector<int32_t> BCf, BCid, BCpos, BCm;  // 1-based
  IK<5> BCpts;

  // geometry
  std::vector<Map> maps;  // 1-based
  std::vector<int64_t> face_owner;  // highest cell number sharing each face
  V1 volume, G1, G2, G3, faces_area;
  M33 gij, xi_x;
  M336 gf;  // meshes_gij_faces
  VK<3> fnormal, ftan, fbitan, fmid;
  VK<20> BCa;
  VK<8> BCap;
  VK<15> AApx, AApy, AApz;

  // fields
  V1 uxyz, vxyz, wxyz, Txyz, uold, vold, wold, Told, ut, vt, wt, Tt;
  V1 uoc, voc, woc, Toc;  // meshes_*_old_con
  V1 mu, mv, mw, mp, dila, dila_old;
  V1 RBu, RBv, RBw, RDu, RDv, RDw, RBp, RDp, RDT, bz;
  V1 fu, fv, fw, fp, fT, fuo, fvo, fwo, fpo, fTo, fbz;
  V1 dpdx, dpdy, dpdz, dpdxo, dpdyo, dpdzo;
  M36 MA, MTA;
  VK<5> MF1, MF2, MF3, MTF1, MTF2, MTF3;
  VK<8> MF4, MTF4;
  // formulation 1 (nim_formulation = 1): a_t(9), AA_vx/vy/vz(15)
  VK<9> at;
  VK<15> AAvx, AAvy, AAvz;
  // parallel-schedule scratch
  V1 snap, pb_new;
  // Gauss-Seidel visiting orders (1-based cell numbers, BC-list indices):
  // number order for SEQUENTIAL, the level order for LEVELS
  std::vector<int64_t> cord, bord;

  real err[5] = {0, 0, 0, 0, 0};
  real Dilatation = 0, dudt_max = 0, dTdt_max = 0;

  // --------------------------------------------------------- helpers
  int32_t F(int pos, int64_t n) const { return mfaces(pos, n); }
  int32_t NB(int pos, int64_t n) const { return mnb(pos, n); }
};

namespace {

// ====================================================== init-time geometry
// mesh_calculate_mapping_coefficients, create_mesh.f90:254-303
void mapping_coefficients(nim_oracle &o, int64_t m) {
  real x[9], y[9], z[9];
  for (int i = 1; i <= 8; ++i) {
    const int64_t nd = o.mnodes(i, m) - 1;
    x[i] = o.node_xyz[3 * nd + 0];
    y[i] = o.node_xyz[3 * nd + 1];
    z[i] = o.node_xyz[3 * nd + 2];
  }
  auto coef = [](const real *v, real *C) {
    C[0] = (v[7] + v[8] + v[5] + v[6] + v[3] + v[4] + v[1] + v[2]) / 8.;
    C[1] = (v[7] - v[8] - v[5] + v[6] + v[3] - v[4] - v[1] + v[2]) / 8.;
    C[2] = (v[7] + v[8] - v[5] - v[6] + v[3] + v[4] - v[1] - v[2]) / 8.;
    C[3] = (v[7] + v[8] + v[5] + v[6] - v[3] - v[4] - v[1] - v[2]) / 8.;
    C[4] = (v[7] - v[8] + v[5] - v[6] + v[3] - v[4] + v[1] - v[2]) / 8.;
    C[5] = (v[7] - v[8] - v[5] + v[6] - v[3] + v[4] + v[1] - v[2]) / 8.;
    C[6] = (v[7] + v[8] - v[5] - v[6] - v[3] - v[4] + v[1] + v[2]) / 8.;
    C[7] = (v[7] - v[8] + v[5] - v[6] - v[3] + v[4] - v[1] + v[2]) / 8.;
  };
  coef(x, o.maps[m].C);
  coef(y, o.maps[m].D);
  coef(z, o.maps[m].E);
}

// The local coordinates of face fn's centre and of its Gauss points.
inline void face_point(int fn, real a, real b, real &x, real &y, real &z) {
  const real s = (fn % 2 == 1) ? -1.0 : 1.0;
  if (fn <= 2) { x = s; y = a; z = b; }
  else if (fn <= 4) { x = a; y = s; z = b; }
  else { x = a; y = b; z = s; }
}

// evaluate_all_mesh_constants body for cell i (geometry.f90:14-32):
// volume_calculate, find_normal, calculate_defusion_tensor_over_faces,
// convection_diffusion_constants_mesh_i.
void cell_geometry(nim_oracle &o, int64_t m) {
  mapping_coefficients(o, m);
  const Map &M = o.maps[m];
  Curvi C;
  // volume_calculate, create_mesh.f90:306-322
  {
    real Int = 0.;
    for (int i = 0; i < 5; ++i)
      for (int j = 0; j < 5; ++j)
        for (int k = 0; k < 5; ++k) {
          evaluate_curvilinear(M, GQ.x[i], GQ.x[j], GQ.x[k], C);
          Int = Int + GQ.w[i] * GQ.w[j] * GQ.w[k] * (1. * C.detJ);
        }
    o.volume(m) = Int;
  }
  // find_normal, geometry.f90:76-190: unit contravariant normal, unit
  // covariant tangents and the centre point of every face.
  for (int fn = 1; fn <= 6; ++fn) {
    real x, y, z;
    face_point(fn, 0.0, 0.0, x, y, z);
    evaluate_curvilinear(M, x, y, z, C);
    const int d = (fn - 1) / 2;             // normal direction 0..2
    const int t1 = (d == 0) ? 1 : 0;        // first tangent
    const int t2 = (d == 2) ? 1 : 2;        // second tangent
    const int32_t f = o.F(fn, m);
    if (o.face_owner[f] != m) continue;  // a later cell overwrites this face
    const real sn = sqrt(C.gij[d][d]);
    const real s1 = sqrt(C.g_ij[t1][t1]);
    const real s2 = sqrt(C.g_ij[t2][t2]);
    for (int c = 0; c < 3; ++c) {
      o.fnormal(c + 1, f) = C.jacinv[c][d] / sn;
      o.ftan(c + 1, f) = C.jac[t1][c] / s1;
      o.fbitan(c + 1, f) = C.jac[t2][c] / s2;
    }
    o.fmid(1, f) = C.x;
    o.fmid(2, f) = C.y;
    o.fmid(3, f) = C.z;
  }
  // calculate_diffusion_tensor_faces_i, geometry.f90:415-497 (the 25 points
  // of each face that Gauss_integration2d_face keeps)
  for (int fn = 1; fn <= 6; ++fn) {
    const int d = (fn - 1) / 2;
    real dS[5][5], K[3][3][5][5];
    for (int a = 0; a < 5; ++a)
      for (int b = 0; b < 5; ++b) {
        real x, y, z;
        face_point(fn, GQ.x[a], GQ.x[b], x, y, z);
        evaluate_curvilinear(M, x, y, z, C);
        dS[a][b] = C.detJ * sqrt(C.gij[d][d]);
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c) K[r][c][a][b] = C.gij[r][c] / sqrt(C.gij[r][r]) * dS[a][b];
      }
    auto integ = [&](const real A[5][5]) {
      real Int = 0.;
      for (int a = 0; a < 5; ++a)
        for (int b = 0; b < 5; ++b) Int = Int + GQ.w[a] * GQ.w[b] * A[a][b];
      return Int;
    };
    const int32_t f = o.F(fn, m);
    const real area = integ(dS);  // this cell's faces_area(f), read back at geometry.f90:484-492
    if (o.face_owner[f] == m) o.faces_area(f) = area;
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) o.gf(r + 1, c + 1, fn, m) = integ(K[r][c]) / area;
  }
  // convection_diffusion_constants_mesh_i, geometry.f90:500-632
  {
    real sG[3] = {0, 0, 0}, sK[3][3], sJ[3][3];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) sK[r][c] = sJ[r][c] = 0.;
    for (int i = 0; i < 5; ++i)
      for (int j = 0; j < 5; ++j)
        for (int k = 0; k < 5; ++k) {
          evaluate_curvilinear(M, GQ.x[i], GQ.x[j], GQ.x[k], C);
          const real w = GQ.w[i] * GQ.w[j] * GQ.w[k];
          for (int a = 0; a < 3; ++a) {
            const real Ga = (C.gam[a][0][1] * C.gij[0][1] + C.gam[a][1][0] * C.gij[1][0] +
                               C.gam[a][0][2] * C.gij[0][2] + C.gam[a][2][0] * C.gij[2][0] +
                               C.gam[a][1][2] * C.gij[1][2] + C.gam[a][2][1] * C.gij[2][1]);
            sG[a] = sG[a] + w * (Ga * C.detJ);
          }
          for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) {
              sK[r][c] = sK[r][c] + w * (C.gij[r][c] * C.detJ);
              sJ[r][c] = sJ[r][c] + w * (C.jacinv[r][c] * C.detJ);
            }
        }
    const real V = o.volume(m);
    o.G1(m) = sG[0] / V;
    o.G2(m) = sG[1] / V;
    o.G3(m) = sG[2] / V;
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) {
        o.gij(r + 1, c + 1, m) = sK[r][c] / V;
        o.xi_x(c + 1, r + 1, m) = sJ[r][c] / V;  // xi_x(a,b) = <jacinv(b,a)>
      }
  }
}

// evaluate_pressure_bc_array, geometry.f90:879-975: the 5-point stencil and
// its weights for the normal second derivative at every wall face.
void pressure_bc_array(nim_oracle &o) {
  for (int64_t i = 1; i <= o.NBF; ++i) {
    const int32_t f0 = o.BCf[i];
    const real *nv = &o.fnormal(1, f0), *tv = &o.ftan(1, f0), *sv = &o.fbitan(1, f0);
    const int64_t M1 = o.BCm[i];
    const int pos = o.BCpos[i];
    int fn = 0;
    int64_t M2 = 0, M3 = 0, M4 = 0;
    const int t1a = (pos <= 2) ? 4 : 2, t1b = (pos <= 2) ? 3 : 1;
    const int t2a = (pos <= 4) ? 6 : 4, t2b = (pos <= 4) ? 5 : 3;
    fn = (pos % 2 == 1) ? pos + 1 : pos - 1;
    M2 = o.NB(fn, M1);
    M3 = o.NB(t1a, M1);
    if (M3 == 0) M3 = o.NB(t1b, M1);
    M4 = o.NB(t2a, M1);
    if (M4 == 0) M4 = o.NB(t2b, M1);
    o.BCpts(1, i) = f0;
    o.BCpts(2, i) = o.F(fn, M1);
    o.BCpts(3, i) = o.F(fn, M2);
    o.BCpts(4, i) = o.F(fn, M3);
    o.BCpts(5, i) = o.F(fn, M4);
    real n[6], t[6], s[6];
    for (int j = 1; j <= 5; ++j) {
      real dvec[3];
      for (int c = 1; c <= 3; ++c) dvec[c - 1] = o.fmid(c, o.BCpts(j, i)) - o.fmid(c, o.BCpts(1, i));
      n[j] = dot3(dvec, nv);
      t[j] = dot3(dvec, tv);
      s[j] = dot3(dvec, sv);
    }
    const real D =
        (n[3] * s[4] * t[2] - n[3] * s[5] * t[2] - n[2] * s[4] * t[3] + n[2] * s[5] * t[3] - n[3] * s[2] * t[4] +
         n[2] * s[3] * t[4] - n[2] * s[5] * t[4] + n[3] * s[5] * t[4] + n[5] * s[3] * t[2] - n[5] * s[4] * t[2] -
         n[5] * s[2] * t[3] + n[5] * s[4] * t[3] + n[5] * s[2] * t[4] - n[5] * s[3] * t[4] + n[3] * s[2] * t[5] -
         n[2] * s[3] * t[5] + n[2] * s[4] * t[5] - n[3] * s[4] * t[5] +
         n[4] * (s[5] * t[2] + s[2] * t[3] - s[5] * t[3] - s[2] * t[5] + s[3] * (-t[2] + t[5])));
    real a[21];
    a[2] = 2 * (-(n[5] * s[4] * t[3]) + n[4] * s[5] * t[3] + n[5] * s[3] * t[4] - n[3] * s[5] * t[4] -
                n[4] * s[3] * t[5] + n[3] * s[4] * t[5]) / (sq(n[2]) * D);
    a[3] = 2 * (n[5] * s[4] * t[2] - n[4] * s[5] * t[2] - n[5] * s[2] * t[4] + n[2] * s[5] * t[4] +
                n[4] * s[2] * t[5] - n[2] * s[4] * t[5]) / (sq(n[3]) * D);
    a[4] = 2 * (n[5] * s[3] * t[2] - n[3] * s[5] * t[2] - n[5] * s[2] * t[3] + n[2] * s[5] * t[3] +
                n[3] * s[2] * t[5] - n[2] * s[3] * t[5]) / (sq(n[4]) * D);
    a[5] = 2 * (n[4] * s[3] * t[2] - n[3] * s[4] * t[2] - n[4] * s[2] * t[3] + n[2] * s[4] * t[3] +
                n[3] * s[2] * t[4] - n[2] * s[3] * t[4]) / (sq(n[5]) * D);
    a[1] = -a[2] - a[3] - a[4] - a[5];
    for (int k = 1; k <= 5; ++k) o.BCa(k, i) = a[k];
    // BCs_faces_a(6:20) multiply boundary velocity derivatives that are
    // identically zero for this case (BCs_derivatives_*, general.f90:296-420)
    // and are not formed.
  }
}

// calculate_pressure_nim_constants, nim.f90:556-743 (u = 0: series branch of
// B..J_nim, nim.f90:758-875, reduced to its leading terms).
void pressure_constants(nim_oracle &o) {
  const int64_t N = o.NMESH;
  V1 Det;
  Det.alloc(N);
  VK<3> CC, EE, FF, GG, HH, II, JJ;
  CC.alloc(N); EE.alloc(N); FF.alloc(N); GG.alloc(N); HH.alloc(N); II.alloc(N); JJ.alloc(N);
  const real a = 1.;
  for (int64_t i = 1; i <= N; ++i) {
    real K[3];
    for (int d = 1; d <= 3; ++d) K[d - 1] = o.gij(d, d, i) / o.P.rho;
    for (int d = 1; d <= 3; ++d) {
      const real Fk = K[d - 1];
      CC(d, i) = -(a * a / (3. * Fk));  // C_nim case(1), u = 0
      GG(d, i) = 1 / (2. * a);          // G_nim
      HH(d, i) = a / Fk;                // H_nim
      II(d, i) = 1 / (2. * a);          // I_nim
      JJ(d, i) = -(a / Fk);             // J_nim
    }
    Det(i) = 1. / (CC(1, i) * CC(2, i) + CC(2, i) * CC(3, i) + CC(1, i) * CC(3, i));
    for (int d = 1; d <= 3; ++d) {
      EE(d, i) = Det(i) / 2.;  // E_nim case(1), u = 0
      FF(d, i) = Det(i) / 2.;  // F_nim
    }
  }
  for (int64_t i = 1; i <= N; ++i) {
    if (o.NB(2, i) != 0) {
      const int64_t i2 = o.NB(2, i);
      const real g = o.gf(1, 1, 2, i), g2 = o.gf(1, 1, 1, i2);
      real *A = &o.AApx(1, i);
      A[0] = -(GG(1, i) + (CC(2, i) + CC(3, i)) * EE(1, i) * HH(1, i)) * g;
      A[1] = (GG(1, i) - (CC(2, i) + CC(3, i)) * FF(1, i) * HH(1, i)) * g +
             (II(1, i2) + (CC(2, i2) + CC(3, i2)) * EE(1, i2) * JJ(1, i2)) * g2;
      A[2] = -(II(1, i2) - (CC(2, i2) + CC(3, i2)) * FF(1, i2) * JJ(1, i2)) * g2;
      A[3] = CC(3, i) * EE(2, i) * HH(1, i) * g;
      A[4] = CC(3, i) * FF(2, i) * HH(1, i) * g;
      A[5] = -(CC(3, i2) * EE(2, i2) * JJ(1, i2) * g2);
      A[6] = -(CC(3, i2) * FF(2, i2) * JJ(1, i2) * g2);
      A[7] = CC(2, i) * EE(3, i) * HH(1, i) * g;
      A[8] = CC(2, i) * FF(3, i) * HH(1, i) * g;
      A[9] = -(CC(2, i2) * EE(3, i2) * JJ(1, i2) * g2);
      A[10] = -(CC(2, i2) * FF(3, i2) * JJ(1, i2) * g2);
      A[11] = CC(2, i) * CC(3, i) * Det(i) * HH(1, i) * g;
      A[12] = -(CC(2, i) * CC(3, i) * Det(i) * HH(1, i) * g);
      A[13] = -(CC(2, i2) * CC(3, i2) * Det(i2) * JJ(1, i2) * g2);
      A[14] = CC(2, i2) * CC(3, i2) * Det(i2) * JJ(1, i2) * g2;
    }
    if (o.NB(4, i) != 0) {
      const int64_t i2 = o.NB(4, i);
      const real g = o.gf(2, 2, 4, i), g2 = o.gf(2, 2, 3, i2);
      real *A = &o.AApy(1, i);
      A[0] = CC(3, i) * EE(1, i) * HH(2, i) * g;
      A[1] = CC(3, i) * FF(1, i) * HH(2, i) * g;
      A[2] = -(CC(3, i2) * EE(1, i2) * JJ(2, i2) * g2);
      A[3] = -(CC(3, i2) * FF(1, i2) * JJ(2, i2) * g2);
      A[4] = -(GG(2, i) + (CC(1, i) + CC(3, i)) * EE(2, i) * HH(2, i)) * g;
      A[5] = (GG(2, i) - (CC(1, i) + CC(3, i)) * FF(2, i) * HH(2, i)) * g +
             (II(2, i2) + (CC(1, i2) + CC(3, i2)) * EE(2, i2) * JJ(2, i2)) * g2;
      A[6] = -(II(2, i2) - (CC(1, i2) + CC(3, i2)) * FF(2, i2) * JJ(2, i2)) * g2;
      A[7] = CC(1, i) * EE(3, i) * HH(2, i) * g;
      A[8] = CC(1, i) * FF(3, i) * HH(2, i) * g;
      A[9] = -(CC(1, i2) * EE(3, i2) * JJ(2, i2) * g2);
      A[10] = -(CC(1, i2) * FF(3, i2) * JJ(2, i2) * g2);
      A[11] = CC(1, i) * CC(3, i) * Det(i) * HH(2, i) * g;
      A[12] = -(CC(1, i) * CC(3, i) * Det(i) * HH(2, i) * g);
      A[13] = -(CC(1, i2) * CC(3, i2) * Det(i2) * JJ(2, i2) * g2);
      A[14] = CC(1, i2) * CC(3, i2) * Det(i2) * JJ(2, i2) * g2;
    }
    if (o.NB(6, i) != 0) {
      const int64_t i2 = o.NB(6, i);
      const real g = o.gf(3, 3, 6, i), g2 = o.gf(3, 3, 5, i2);
      real *A = &o.AApz(1, i);
      A[0] = CC(2, i) * EE(1, i) * HH(3, i) * g;
      A[1] = CC(2, i) * FF(1, i) * HH(3, i) * g;
      A[2] = -(CC(2, i2) * EE(1, i2) * JJ(3, i2) * g2);
      A[3] = -(CC(2, i2) * FF(1, i2) * JJ(3, i2) * g2);
      A[4] = CC(1, i) * EE(2, i) * HH(3, i) * g;
      A[5] = CC(1, i) * FF(2, i) * HH(3, i) * g;
      A[6] = -(CC(1, i2) * EE(2, i2) * JJ(3, i2) * g2);
      A[7] = -(CC(1, i2) * FF(2, i2) * JJ(3, i2) * g2);
      A[8] = -(GG(3, i) + (CC(1, i) + CC(2, i)) * EE(3, i) * HH(3, i)) * g;
      A[9] = (GG(3, i) - (CC(1, i) + CC(2, i)) * FF(3, i) * HH(3, i)) * g +
             (II(3, i2) + (CC(1, i2) + CC(2, i2)) * EE(3, i2) * JJ(3, i2)) * g2;
      A[10] = -(II(3, i2) - (CC(1, i2) + CC(2, i2)) * FF(3, i2) * JJ(3, i2)) * g2;
      A[11] = CC(1, i) * CC(2, i) * Det(i) * HH(3, i) * g;
      A[12] = -(CC(1, i) * CC(2, i) * Det(i) * HH(3, i) * g);
      A[13] = -(CC(1, i2) * CC(2, i2) * Det(i2) * JJ(3, i2) * g2);
      A[14] = CC(1, i2) * CC(2, i2) * Det(i2) * JJ(3, i2) * g2;
    }
  }
  // boundary faces, nim.f90:683-741
  for (int64_t i = 1; i <= o.NBF; ++i) {
    const int64_t M = o.BCm[i];
    const int pos = o.BCpos[i];
    real *ap = &o.BCap(1, i);
    const int d = (pos + 1) / 2;                    // normal direction 1..3
    const int e1 = (d == 1) ? 2 : 1, e2 = (d == 3) ? 2 : 3;  // transverse
    const bool minus = (pos % 2 == 1);               // wall on the - side
    const real g = o.gf(d, d, pos, M);
    // - side walls use I/J (the "i2" role), + side walls G/H (the "i" role)
    const real P0 = minus ? II(d, M) : GG(d, M);
    const real Q = minus ? JJ(d, M) : HH(d, M);
    const real cs = CC(e1, M) + CC(e2, M);
    const real own_m = -(P0 + cs * EE(d, M) * Q) * g;
    const real own_p = (P0 - cs * FF(d, M) * Q) * g;
    real te1_m = CC(e2, M) * EE(e1, M) * Q * g, te1_p = CC(e2, M) * FF(e1, M) * Q * g;
    real te2_m = CC(e1, M) * EE(e2, M) * Q * g, te2_p = CC(e1, M) * FF(e2, M) * Q * g;
    real a7 = CC(e1, M) * CC(e2, M) * Det(M) * Q * g;
    real a8 = -(CC(e1, M) * CC(e2, M) * Det(M) * Q * g);
    // slots: 2d-1 / 2d own direction, 2e-1 / 2e transverse
    ap[2 * d - 2] = own_m;
    ap[2 * d - 1] = own_p;
    ap[2 * e1 - 2] = te1_m;
    ap[2 * e1 - 1] = te1_p;
    ap[2 * e2 - 2] = te2_m;
    ap[2 * e2 - 1] = te2_p;
    ap[6] = a7;
    ap[7] = a8;
  }
}

// Face average of a constant boundary value c over face fn of cell M:
// apply_dirichlet_bc_i, bc.f90:59-88 (c * dS integrated, over the area).
real dirichlet_face_value(nim_oracle &o, int64_t M, int fn, real c) {
  const int d = (fn - 1) / 2;
  Curvi C;
  real TT[5][5];
  for (int i = 0; i < 5; ++i)
    for (int j = 0; j < 5; ++j) {
      real x, y, z;
      face_point(fn, GQ.x[i], GQ.x[j], x, y, z);
      evaluate_curvilinear(o.maps[M], x, y, z, C);
      const real dS = C.detJ * sqrt(C.gij[d][d]);
      TT[i][j] = c * dS;
    }
  real Int = 0.;
  for (int i = 0; i < 5; ++i)
    for (int j = 0; j < 5; ++j) Int = Int + GQ.w[i] * GQ.w[j] * TT[i][j];
  return Int / o.faces_area(o.F(fn, M));
}

// ============================================================ per step
// NIM coefficients of one direction for contravariant speed u and
// diffusivity k (M_A(d,1:6) / MT_A(d,1:6), nim.f90:181-287 / 354-460).
void nim_direction(real u, real k, real gminus, real gplus, real v_limit, real A[6]) {
  const real a = 1.;
  const real Re = 2 * a * u / k;
  if (fabs(Re) > v_limit) {
    const real e = exp(Re);
    A[0] = (2 * a / (k * (1. / e - 1.)) + 1. / u) * gplus;
    A[1] = (-(2 * a / (k * (1. - e))) - 1. / u) * gminus;
    A[2] = (u / (k * (1. / e - 1.))) * gplus;
    A[3] = (u / (k * (1. - e))) * gminus;
    if (Re > 0) A[4] = (-k + (a * u * (1. / e + 1.) / (-(1. / e) + 1.))) / (u * u);
    if (Re < 0) A[4] = (-k + (a * u * (1. + e) / (-1. + e))) / (u * u);
    if (Re > 0) A[5] = 1. / (-(1. / e) + 1.) - 1. / (Re);
    if (Re < 0) A[5] = e / (-1. + e) - 1. / (Re);
  } else {
    const Pw U(u), K(k);
    A[0] = (-(a / k) - (u) / (3. * K[2]) + (U[3]) / (45. * K[4]) - (2 * U[5]) / (945. * K[6]) +
            -((U[7]) / (4725. * K[8])) - (2 * U[9]) / (93555. * K[10])) * gplus;
    A[1] = (-(a / k) + (u) / (3. * K[2]) - (U[3]) / (45. * K[4]) + (2 * U[5]) / (945. * K[6]) -
            -((U[7]) / (4725. * K[8])) + (2 * U[9]) / (93555. * K[10])) * gminus;
    A[2] = (-(1 / (2. * a)) - u / (2. * k) - (U[2]) / (6. * K[2]) + (U[4]) / (90. * K[4]) -
            -((U[6]) / (945. * K[6])) + (U[8]) / (9450. * K[8]) - (U[10]) / (93555. * K[10])) * gplus;
    A[3] = (-(1 / (2. * a)) + u / (2. * k) - (U[2]) / (6. * K[2]) + (U[4]) / (90. * K[4]) -
            -((U[6]) / (945. * K[6])) + (U[8]) / (9450. * K[8]) - (U[10]) / (93555. * K[10])) * gminus;
    A[4] = 1. / (3. * k) - (U[2]) / (45. * K[3]) + (2 * U[4]) / (945. * K[5]) - -((U[6]) / (4725. * K[7])) +
           (2 * U[8]) / (93555. * K[9]) - -((1382 * U[10]) / (6.38512875e8 * K[11]));
    A[5] = 0.5 + (u) / (6. * k) - (U[3]) / (90. * K[3]) + (U[5]) / (945. * K[5]) - -((U[7]) / (9450. * K[7])) +
           (U[9]) / (93555. * K[9]);
  }
}

// M_F4 / M_F1..3 from M_A (nim.f90:293-328), shared by velocity and T.
void form_F(nim_oracle &o, const M36 &A, VK<8> &F4, VK<5> &F1, VK<5> &F2, VK<5> &F3, int64_t i) {
  const real DT = o.P.DT;
  F4(2, i) = 0.5 * (1. / A(1, 5, i) + 1. / A(2, 5, i) + 1. / A(3, 5, i) - 1. / DT);
  F4(3, i) = -(A(1, 6, i) / A(1, 5, i));
  F4(4, i) = (A(1, 6, i) - 1.) / A(1, 5, i);
  F4(5, i) = -(A(2, 6, i) / A(2, 5, i));
  F4(6, i) = (A(2, 6, i) - 1.) / A(2, 5, i);
  F4(7, i) = -(A(3, 6, i) / A(3, 5, i));
  F4(8, i) = (A(3, 6, i) - 1.) / A(3, 5, i);
  F4(1, i) = F4(2, i) + F4(3, i) + F4(4, i) + F4(5, i) + F4(6, i) + F4(7, i) + F4(8, i);
  VK<5> *FF[3] = {&F1, &F2, &F3};
  for (int d = 1; d <= 3; ++d) {
    if (o.NB(2 * d, i) == 0) continue;
    const int64_t i2 = o.NB(2 * d, i);
    VK<5> &G = *FF[d - 1];
    G(2, i) = A(d, 3, i) - (A(d, 1, i) * A(d, 6, i) / A(d, 5, i));
    G(3, i) = A(d, 4, i2) - A(d, 2, i2) / A(d, 5, i2) + A(d, 2, i2) * A(d, 6, i2) / A(d, 5, i2);
    G(4, i) = A(d, 1, i) / (2. * A(d, 5, i));
    G(5, i) = A(d, 2, i2) / (2. * A(d, 5, i2));
    G(1, i) = G(2, i) + G(3, i) + 2. * G(4, i) + 2. * G(5, i);
  }
}

// calculate_velocity_nim_constants_formulation2, nim.f90:160-330
void velocity_constants(nim_oracle &o) {
  const int64_t N = o.NMESH;
#pragma omp parallel for schedule(static) num_threads(o.nthreads)
  for (int64_t i = 1; i <= N; ++i) {
    o.mu(i) = o.ut(i) * o.xi_x(1, 1, i) + o.vt(i) * o.xi_x(1, 2, i) + o.wt(i) * o.xi_x(1, 3, i);
    o.mv(i) = o.ut(i) * o.xi_x(2, 1, i) + o.vt(i) * o.xi_x(2, 2, i) + o.wt(i) * o.xi_x(2, 3, i);
    o.mw(i) = o.ut(i) * o.xi_x(3, 1, i) + o.vt(i) * o.xi_x(3, 2, i) + o.wt(i) * o.xi_x(3, 3, i);
    const real c[3] = {o.mu(i), o.mv(i), o.mw(i)};
    for (int d = 1; d <= 3; ++d) {
      real A[6];
      nim_direction(c[d - 1], o.gij(d, d, i) * o.nu, o.gf(d, d, 2 * d - 1, i), o.gf(d, d, 2 * d, i),
                    o.P.v_limit, A);
      for (int k = 0; k < 6; ++k) o.MA(d, k + 1, i) = A[k];
    }
  }
#pragma omp parallel for schedule(static) num_threads(o.nthreads)
  for (int64_t i = 1; i <= N; ++i) form_F(o, o.MA, o.MF4, o.MF1, o.MF2, o.MF3, i);
}

// calculate_temperature_nim_constants_formulation2, nim.f90:334-502
void temperature_constants(nim_oracle &o) {
  const int64_t N = o.NMESH;
#pragma omp parallel for schedule(static) num_threads(o.nthreads)
  for (int64_t i = 1; i <= N; ++i) {
    const real ut = 0.5 * (o.uxyz(i) + o.uold(i));
    const real vt = 0.5 * (o.vxyz(i) + o.vold(i));
    const real wt = 0.5 * (o.wxyz(i) + o.wold(i));
    const real c[3] = {ut * o.xi_x(1, 1, i) + vt * o.xi_x(1, 2, i) + wt * o.xi_x(1, 3, i),
                         ut * o.xi_x(2, 1, i) + vt * o.xi_x(2, 2, i) + wt * o.xi_x(2, 3, i),
                         ut * o.xi_x(3, 1, i) + vt * o.xi_x(3, 2, i) + wt * o.xi_x(3, 3, i)};
    for (int d = 1; d <= 3; ++d) {
      real A[6];
      nim_direction(c[d - 1], o.gij(d, d, i) * o.alpha, o.gf(d, d, 2 * d - 1, i), o.gf(d, d, 2 * d, i),
                    o.P.v_limit, A);
      for (int k = 0; k < 6; ++k) o.MTA(d, k + 1, i) = A[k];
    }
  }
#pragma omp parallel for schedule(static) num_threads(o.nthreads)
  for (int64_t i = 1; i <= N; ++i) form_F(o, o.MTA, o.MTF4, o.MTF1, o.MTF2, o.MTF3, i);
  // BCs_faces_aT (nim.f90:509-549) only feeds the uncalled find_Nu.
}

// --------------------------------------------------------- formulation 1
// B_nim, C_nim, G_nim, H_nim, I_nim, J_nim (nim.f90:758-875) of one
// direction, a = 1, for contravariant speed u, diffusivity F and cell Peclet
// number Re = 2u/F.  condition() (nim.f90:748-756): series when |Re| <
// v_limit, exponential form otherwise.  G_nim and H_nim assign P twice in
// their exponential branch; the second assignment is the one that counts.
struct Nim1 {
  real B, C, G, H, I, J;
  bool series;
};
Nim1 nim1_direction(real u, real F, real Re, real v_limit) {
  const real a = 1.;
  Nim1 r;
  r.series = fabs(Re) < v_limit;
  if (r.series) {
    const Pw U(u), K(F);
    r.B = 0;
    r.C = -(a * a / (3. * F)) + (U[2]) / (45. * K[3]) - (2 * U[4]) / (945. * K[5]) + -((U[6]) / (4725. * K[7])) -
          (2 * U[8]) / (93555. * K[9]) + -((1382 * U[10]) / (6.38512875e8 * K[11]));
    r.G = 1 / (2. * a) + u / (2. * F) + (U[2]) / (6. * K[2]) - (U[4]) / (90. * K[4]) + -((U[6]) / (945. * K[6])) -
          (U[8]) / (9450. * K[8]) + (U[10]) / (93555. * K[10]);
    r.H = a / F + (u) / (3. * K[2]) - (U[3]) / (45. * K[4]) + (2 * U[5]) / (945. * K[6]) -
          -((U[7]) / (4725. * K[8])) + (2 * U[9]) / (93555. * K[10]);
    r.I = 1 / (2. * a) - u / (2. * F) + (U[2]) / (6. * K[2]) - (U[4]) / (90. * K[4]) + -((U[6]) / (945. * K[6])) -
          (U[8]) / (9450. * K[8]) + (U[10]) / (93555. * K[10]);
    r.J = -(a / F) + (u) / (3. * K[2]) - (U[3]) / (45. * K[4]) + -((2 * U[5]) / (945. * K[6])) -
          (U[7]) / (4725. * K[8]) + -((2 * U[9]) / (93555. * K[10]));
  } else {
    const real e = exp(Re);
    r.B = 1. / u * (1. / Re - 1. / (e - 1.));
    r.C = (-(1. / u) + 2. * r.B) * a;
    r.G = u / F / (1. - 1. / e);
    r.H = 2. * a / F / (1. - 1. / e) - 1. / u;
    r.I = u / (F * (e - 1.));
    r.J = 2. * a / (F * (e - 1.)) - 1. / u;
  }
  return r;
}
// E_nim, F_nim (nim.f90:787-815) with D = Det
inline real nim1_E(const Nim1 &r, real u, real F, real D) {
  const real a = 1.;
  if (r.series) {
    const Pw U(u), K(F);
    return D / 2. + (a * D * u) / (6. * F) - (D * U[3]) / (90. * K[3]) + (D * U[5]) / (945. * K[5]) -
           -((D * U[7]) / (9450. * K[7])) + (D * U[9]) / (93555. * K[9]);
  }
  return D * (1 - r.B * u);
}
inline real nim1_F(const Nim1 &r, real u, real F, real D) {
  const real a = 1.;
  if (r.series) {
    const Pw U(u), K(F);
    return D / 2. - (a * D * u) / (6. * F) + (D * U[3]) / (90. * K[3]) - (D * U[5]) / (945. * K[5]) +
           -((D * U[7]) / (9450. * K[7])) - (D * U[9]) / (93555. * K[9]);
  }
  return D * (r.B * u);
}

// calculate_velocity_nim_constants (nim.f90:17-157): a_t and AA_vx/vy/vz
void velocity_constants_f1(nim_oracle &o) {
  const int64_t N = o.NMESH;
  VK<3> CC, EE, FF, GG, HH, II, JJ;
  V1 Det;
  CC.alloc(N); EE.alloc(N); FF.alloc(N); GG.alloc(N); HH.alloc(N); II.alloc(N); JJ.alloc(N); Det.alloc(N);
#pragma omp parallel for schedule(static) num_threads(o.nthreads)
  for (int64_t i = 1; i <= N; ++i) {
    o.mu(i) = o.ut(i) * o.xi_x(1, 1, i) + o.vt(i) * o.xi_x(1, 2, i) + o.wt(i) * o.xi_x(1, 3, i);
    o.mv(i) = o.ut(i) * o.xi_x(2, 1, i) + o.vt(i) * o.xi_x(2, 2, i) + o.wt(i) * o.xi_x(2, 3, i);
    o.mw(i) = o.ut(i) * o.xi_x(3, 1, i) + o.vt(i) * o.xi_x(3, 2, i) + o.wt(i) * o.xi_x(3, 3, i);
    const real uc[3] = {o.mu(i), o.mv(i), o.mw(i)};
    real K[3], Re[3];
    Nim1 r[3];
    for (int d = 1; d <= 3; ++d) {
      K[d - 1] = o.gij(d, d, i) * o.nu;
      Re[d - 1] = 2 * uc[d - 1] / K[d - 1];
    }
    for (int d = 1; d <= 3; ++d) {
      r[d - 1] = nim1_direction(uc[d - 1], K[d - 1], Re[d - 1], o.P.v_limit);
      CC(d, i) = r[d - 1].C;
      GG(d, i) = r[d - 1].G;
      HH(d, i) = r[d - 1].H;
      II(d, i) = r[d - 1].I;
      JJ(d, i) = r[d - 1].J;
    }
    Det(i) = 1. / (CC(1, i) * CC(2, i) + CC(2, i) * CC(3, i) + CC(1, i) * CC(3, i));
    for (int d = 1; d <= 3; ++d) {
      EE(d, i) = nim1_E(r[d - 1], uc[d - 1], K[d - 1], Det(i));
      FF(d, i) = nim1_F(r[d - 1], uc[d - 1], K[d - 1], Det(i));
    }
  }
  const real DT = o.P.DT;
#pragma omp parallel for schedule(static) num_threads(o.nthreads)
  for (int64_t i = 1; i <= N; ++i) {
    auto C = [&](int d, int64_t n) { return CC(d, n); };
    auto E = [&](int d, int64_t n) { return EE(d, n); };
    auto Fv = [&](int d, int64_t n) { return FF(d, n); };
    if (o.NB(2, i) != 0) {  // face 2 (nim.f90:87-104)
      const int64_t i2 = o.NB(2, i);
      const real g2 = o.gf(1, 1, 2, i), g1 = o.gf(1, 1, 1, i2);
      VK<15> &A = o.AAvx;
      A(1, i) = -(GG(1, i) + (C(2, i) + C(3, i)) * E(1, i) * HH(1, i)) * g2;
      A(2, i) = (GG(1, i) - (C(2, i) + C(3, i)) * Fv(1, i) * HH(1, i)) * g2 +
                (II(1, i2) + (C(2, i2) + C(3, i2)) * E(1, i2) * JJ(1, i2)) * g1;
      A(3, i) = -(II(1, i2) - (C(2, i2) + C(3, i2)) * Fv(1, i2) * JJ(1, i2)) * g1;
      A(4, i) = C(3, i) * E(2, i) * HH(1, i) * g2;
      A(5, i) = C(3, i) * Fv(2, i) * HH(1, i) * g2;
      A(6, i) = -C(3, i2) * E(2, i2) * JJ(1, i2) * g1;
      A(7, i) = -C(3, i2) * Fv(2, i2) * JJ(1, i2) * g1;
      A(8, i) = C(2, i) * E(3, i) * HH(1, i) * g2;
      A(9, i) = C(2, i) * Fv(3, i) * HH(1, i) * g2;
      A(10, i) = -C(2, i2) * E(3, i2) * JJ(1, i2) * g1;
      A(11, i) = -C(2, i2) * Fv(3, i2) * JJ(1, i2) * g1;
      A(12, i) = C(2, i) * C(3, i) * Det(i) * HH(1, i) * g2 / (2 * DT);
      A(13, i) = -C(2, i) * C(3, i) * Det(i) * HH(1, i) * g2 / (2 * DT);
      A(14, i) = -C(2, i2) * C(3, i2) * Det(i2) * JJ(1, i2) * g1 / (2 * DT);
      A(15, i) = C(2, i2) * C(3, i2) * Det(i2) * JJ(1, i2) * g1 / (2 * DT);
    }
    if (o.NB(4, i) != 0) {  // face 4 (nim.f90:107-124)
      const int64_t i2 = o.NB(4, i);
      const real g4 = o.gf(2, 2, 4, i), g3 = o.gf(2, 2, 3, i2);
      VK<15> &A = o.AAvy;
      A(1, i) = C(3, i) * E(1, i) * HH(2, i) * g4;
      A(2, i) = C(3, i) * Fv(1, i) * HH(2, i) * g4;
      A(3, i) = -C(3, i2) * E(1, i2) * JJ(2, i2) * g3;
      A(4, i) = -C(3, i2) * Fv(1, i2) * JJ(2, i2) * g3;
      A(5, i) = -(GG(2, i) + (C(1, i) + C(3, i)) * E(2, i) * HH(2, i)) * g4;
      A(6, i) = (GG(2, i) - (C(1, i) + C(3, i)) * Fv(2, i) * HH(2, i)) * g4 +
                (II(2, i2) + (C(1, i2) + C(3, i2)) * E(2, i2) * JJ(2, i2)) * g3;
      A(7, i) = -(II(2, i2) - (C(1, i2) + C(3, i2)) * Fv(2, i2) * JJ(2, i2)) * g3;
      A(8, i) = C(1, i) * E(3, i) * HH(2, i) * g4;
      A(9, i) = C(1, i) * Fv(3, i) * HH(2, i) * g4;
      A(10, i) = -C(1, i2) * E(3, i2) * JJ(2, i2) * g3;
      A(11, i) = -C(1, i2) * Fv(3, i2) * JJ(2, i2) * g3;
      A(12, i) = C(1, i) * C(3, i) * Det(i) * HH(2, i) * g4 / (2 * DT);
      A(13, i) = -C(1, i) * C(3, i) * Det(i) * HH(2, i) * g4 / (2 * DT);
      A(14, i) = -C(1, i2) * C(3, i2) * Det(i2) * JJ(2, i2) * g3 / (2 * DT);
      A(15, i) = C(1, i2) * C(3, i2) * Det(i2) * JJ(2, i2) * g3 / (2 * DT);
    }
    if (o.NB(6, i) != 0) {  // face 6 (nim.f90:126-143)
      const int64_t i2 = o.NB(6, i);
      const real g6 = o.gf(3, 3, 6, i), g5 = o.gf(3, 3, 5, i2);
      VK<15> &A = o.AAvz;
      A(1, i) = C(2, i) * E(1, i) * HH(3, i) * g6;
      A(2, i) = C(2, i) * Fv(1, i) * HH(3, i) * g6;
      A(3, i) = -C(2, i2) * E(1, i2) * JJ(3, i2) * g5;
      A(4, i) = -C(2, i2) * Fv(1, i2) * JJ(3, i2) * g5;
      A(5, i) = C(1, i) * E(2, i) * HH(3, i) * g6;
      A(6, i) = C(1, i) * Fv(2, i) * HH(3, i) * g6;
      A(7, i) = -C(1, i2) * E(2, i2) * JJ(3, i2) * g5;
      A(8, i) = -C(1, i2) * Fv(2, i2) * JJ(3, i2) * g5;
      A(9, i) = -(GG(3, i) + (C(1, i) + C(2, i)) * E(3, i) * HH(3, i)) * g6;
      A(10, i) = (GG(3, i) - (C(1, i) + C(2, i)) * Fv(3, i) * HH(3, i)) * g6 +
                 (II(3, i2) + (C(1, i2) + C(2, i2)) * E(3, i2) * JJ(3, i2)) * g5;
      A(11, i) = -(II(3, i2) - (C(1, i2) + C(2, i2)) * Fv(3, i2) * JJ(3, i2)) * g5;
      A(12, i) = C(1, i) * C(2, i) * Det(i) * HH(3, i) * g6 / (2 * DT);
      A(13, i) = -C(1, i) * C(2, i) * Det(i) * HH(3, i) * g6 / (2 * DT);
      A(14, i) = -C(1, i2) * C(2, i2) * Det(i2) * JJ(3, i2) * g5 / (2 * DT);
      A(15, i) = C(1, i2) * C(2, i2) * Det(i2) * JJ(3, i2) * g5 / (2 * DT);
    }
    // a_t, nim.f90:146-154
    o.at(1, i) = 2 * E(1, i) / Det(i) - 2 * (C(2, i) + C(3, i)) * C(1, i) * E(1, i);
    o.at(2, i) = 2 * Fv(1, i) / Det(i) - 2 * (C(2, i) + C(3, i)) * C(1, i) * Fv(1, i);
    o.at(3, i) = 2 * E(2, i) * C(1, i) * C(3, i);
    o.at(4, i) = 2 * Fv(2, i) * C(1, i) * C(3, i);
    o.at(5, i) = 2 * E(3, i) * C(1, i) * C(2, i);
    o.at(6, i) = 2 * Fv(3, i) * C(1, i) * C(2, i);
    o.at(7, i) = 2 * C(1, i) * C(2, i) * C(3, i) * Det(i);
    o.at(8, i) = -o.at(7, i) / (2 * DT) - 1;
    o.at(9, i) = o.at(7, i) / (2 * DT) - 1;
  }
}

// ---------------------------------------------------------------- sources
// Green-Gauss derivative dphi_dx2/dy2/dz2 (nse.f90:2866-2903), component c.
inline real green_gauss(const nim_oracle &o, const real *phi, const int32_t *nf, int64_t i, int c) {
  return 1. / o.volume(i) *
         (phi[2] * o.faces_area(nf[2]) * (o.fnormal(c, nf[2])) - phi[1] * o.faces_area(nf[1]) * (o.fnormal(c, nf[1])) +
          phi[4] * o.faces_area(nf[4]) * (o.fnormal(c, nf[4])) - phi[3] * o.faces_area(nf[3]) * (o.fnormal(c, nf[3])) +
          phi[6] * o.faces_area(nf[6]) * (o.fnormal(c, nf[6])) - phi[5] * o.faces_area(nf[5]) * (o.fnormal(c, nf[5])));
}

// Derivative along local direction e of face field phi on face position fpos
// of cell n, centred or one-sided at walls (the nj/ni/nk stencils of
// calculate_R_D2, nse.f90:1635-1838, and of the pressure sweep).
inline real tangential(const nim_oracle &o, const V1 &phi, int64_t n, int fpos, int e) {
  const int64_t m1 = o.NB(2 * e - 1, n), m2 = o.NB(2 * e, n);
  if (m1 == 0) {
    const int64_t m3 = o.NB(2 * e, m2);
    return (-(3 * phi(o.F(fpos, n))) + 4 * phi(o.F(fpos, m2)) - phi(o.F(fpos, m3))) / 4.;
  } else if (m2 == 0) {
    const int64_t m3 = o.NB(2 * e - 1, m1);
    return (3 * phi(o.F(fpos, n)) - 4 * phi(o.F(fpos, m1)) + phi(o.F(fpos, m3))) / 4.;
  }
  return (phi(o.F(fpos, m2)) - phi(o.F(fpos, m1))) / 4.;
}

// Cross-derivative diffusion source (calculate_R_D2 / R_D_p2 / R_D_T):
// G_i d_i phi - g^ij d_ij phi, before the 1/Re, 1/rho or alpha factor.
inline real diffusion_source(const nim_oracle &o, const V1 &phi, int64_t n) {
  const real pxy = 0.5 * (tangential(o, phi, n, 2, 2) - tangential(o, phi, n, 1, 2));
  const real pzy = 0.5 * (tangential(o, phi, n, 6, 2) - tangential(o, phi, n, 5, 2));
  const real pyx = 0.5 * (tangential(o, phi, n, 4, 1) - tangential(o, phi, n, 3, 1));
  const real pzx = 0.5 * (tangential(o, phi, n, 6, 1) - tangential(o, phi, n, 5, 1));
  const real pxz = 0.5 * (tangential(o, phi, n, 2, 3) - tangential(o, phi, n, 1, 3));
  const real pyz = 0.5 * (tangential(o, phi, n, 4, 3) - tangential(o, phi, n, 3, 3));
  const real px = (phi(o.F(2, n)) - phi(o.F(1, n))) / 2.;
  const real py = (phi(o.F(4, n)) - phi(o.F(3, n))) / 2.;
  const real pz = (phi(o.F(6, n)) - phi(o.F(5, n))) / 2.;
  return (o.G1(n) * px + o.G2(n) * py + o.G3(n) * pz - o.gij(1, 2, n) * pxy - o.gij(2, 1, n) * pyx -
          o.gij(1, 3, n) * pxz - o.gij(3, 1, n) * pzx - o.gij(2, 3, n) * pyz - o.gij(3, 2, n) * pzy);
}

// update_velocity_sources (nse.f90:199-211): calculate_gforces, calculate_R_b,
// calculate_R_c_new, calculate_R_D2 for every cell.
void velocity_sources(nim_oracle &o) {
  const int64_t N = o.NMESH;
  const real gb = o.P.g_beta;
  for (int64_t i = 1; i <= N; ++i) o.bz(i) = -(gb * 0.5 * (o.Txyz(i) + o.Told(i)));
  for (int64_t f = 1; f <= o.NFACE; ++f) o.fbz(f) = -(gb * (o.fT(f)));
  const bool check_rc = (o.sched != NIM_SCHED_PARALLEL);
  double mrc = o.max_rc;
#pragma omp parallel for schedule(static) num_threads(o.nthreads) reduction(max : mrc)
  for (int64_t i = 1; i <= N; ++i) {
    int32_t nf[7];
    for (int k = 1; k <= 6; ++k) nf[k] = o.F(k, i);
    real pf[7];
    for (int k = 1; k <= 6; ++k) pf[k] = o.fp(nf[k]);
    const real dpx = green_gauss(o, pf, nf, i, 1), dpy = green_gauss(o, pf, nf, i, 2),
                 dpz = green_gauss(o, pf, nf, i, 3);
    o.RBu(i) = 0. + 1 / o.P.rho * dpx;  // meshes_bx = 0
    o.RBv(i) = 0. + 1 / o.P.rho * dpy;  // meshes_by = 0
    o.RBw(i) = o.bz(i) + 1 / o.P.rho * dpz;
    if (check_rc) {
      // calculate_R_c_new, nse.f90:1393-1434: (meshes_u - uc) is the same
      // expression on the same values, so R_C is zero; verify it.
      const real uc = o.ut(i) * o.xi_x(1, 1, i) + o.vt(i) * o.xi_x(1, 2, i) + o.wt(i) * o.xi_x(1, 3, i);
      const real vc = o.ut(i) * o.xi_x(2, 1, i) + o.vt(i) * o.xi_x(2, 2, i) + o.wt(i) * o.xi_x(2, 3, i);
      const real wc = o.ut(i) * o.xi_x(3, 1, i) + o.vt(i) * o.xi_x(3, 2, i) + o.wt(i) * o.xi_x(3, 3, i);
      const real r = fabs(o.mu(i) - uc) + fabs(o.mv(i) - vc) + fabs(o.mw(i) - wc);
      mrc = std::max(mrc, val(r));
    }
    o.RDu(i) = o.inv_Re * diffusion_source(o, o.fu, i);
    o.RDv(i) = o.inv_Re * diffusion_source(o, o.fv, i);
    o.RDw(i) = o.inv_Re * diffusion_source(o, o.fw, i);
  }
  o.max_rc = mrc;
}

// Cell-average update of one field (integrate_velocity_field_formulation2_i
// nse.f90:839-872, temperature nse.f90:1017-1026).
inline real cell_update(const nim_oracle &o, const V1 &f, real c, real cold, real B,
                          const VK<8> &F4, int64_t i, real w) {
  return (1 - w) * c +
         (w / F4(1, i)) * (+F4(2, i) * cold + F4(3, i) * f(o.F(1, i)) + F4(4, i) * f(o.F(2, i)) +
                           F4(5, i) * f(o.F(3, i)) + F4(6, i) * f(o.F(4, i)) + F4(7, i) * f(o.F(5, i)) +
                           F4(8, i) * f(o.F(6, i)) + B);
}

// Update of the +d face of cell i (nse.f90:878-1005, 1033-1088).  fr is read,
// the result is returned; the caller stores it.
inline real face_update(const nim_oracle &o, const V1 &fr, const V1 &c, const V1 &cold,
                          const VK<5> &Fd, int d, int64_t i, real w) {
  const int64_t i2 = o.NB(2 * d, i);
  const int e1 = (d == 1) ? 2 : 1, e2 = (d == 3) ? 2 : 3;
  const real B3 = (o.gf(d, e1, 2 * d - 1, i2) - o.gf(d, e1, 2 * d, i)) *
                    (fr(o.F(2 * e1, i)) - fr(o.F(2 * e1 - 1, i)) + fr(o.F(2 * e1, i2)) - fr(o.F(2 * e1 - 1, i2))) / 4.0;
  const real B4 = (o.gf(d, e2, 2 * d - 1, i2) - o.gf(d, e2, 2 * d, i)) *
                    (fr(o.F(2 * e2, i)) - fr(o.F(2 * e2 - 1, i)) + fr(o.F(2 * e2, i2)) - fr(o.F(2 * e2 - 1, i2))) / 4.0;
  return (1 - w) * fr(o.F(2 * d, i)) +
         (w / Fd(1, i)) * (+Fd(2, i) * fr(o.F(2 * d - 1, i)) + Fd(3, i) * fr(o.F(2 * d, i2)) +
                           Fd(4, i) * (c(i) + cold(i)) + Fd(5, i) * (c(i2) + cold(i2)) - B3 - B4);
}

// Formulation 1 cell update of one velocity component (integrate_velocity_
// field_i, nse.f90:341-352); R = R_C + R_D + R_B of the cell.
inline real cell_update_f1(const nim_oracle &o, const V1 &f, real c, real cold, real R, int64_t i,
                             real w) {
  const VK<9> &a = o.at;
  const real Bij = a(7, i) * R;
  return (1 - w) * c + w * (-(a(1, i) * f(o.F(1, i))) - a(2, i) * f(o.F(2, i)) - a(3, i) * f(o.F(3, i)) -
                            a(4, i) * f(o.F(4, i)) - a(5, i) * f(o.F(5, i)) - a(6, i) * f(o.F(6, i)) -
                            a(8, i) * cold - Bij) /
                           (a(9, i));
}

// Formulation 1 update of the +d face of cell n1 (nse.f90:378-826): the
// pressure sweep's ten face terms with AA_v, the two cell time terms, the
// R sums of both cells and the tangential cross terms B3, B4 (the centred
// B3/B4 the source computes first are overwritten before use).
inline real face_update_f1(const nim_oracle &o, const V1 &fr, const V1 &c, const V1 &cold, const V1 &RD,
                             const V1 &RB, int d, int64_t n1, real w) {
  const int64_t n2 = o.NB(2 * d, n1);
  const VK<15> &A = (d == 1) ? o.AAvx : (d == 2) ? o.AAvy : o.AAvz;
  const int e1 = (d == 1) ? 2 : 1, e2 = (d == 3) ? 2 : 3;
  const real DT = o.P.DT;
  const real B1 = (0. + RD(n1) + RB(n1)) * A(13, n1) * 2 * DT;
  const real B2 = (0. + RD(n2) + RB(n2)) * A(15, n1) * 2 * DT;
  const real B3 = (o.gf(d, e1, 2 * d - 1, n2) - o.gf(d, e1, 2 * d, n1)) * tangential(o, fr, n1, 2 * d, e1);
  const real B4 = (o.gf(d, e2, 2 * d - 1, n2) - o.gf(d, e2, 2 * d, n1)) * tangential(o, fr, n1, 2 * d, e2);
  static const int tab[3][10][3] = {
      {{1, 1, 1}, {3, 2, 2}, {4, 3, 1}, {5, 4, 1}, {6, 3, 2}, {7, 4, 2}, {8, 5, 1}, {9, 6, 1}, {10, 5, 2}, {11, 6, 2}},
      {{1, 1, 1}, {2, 2, 1}, {3, 1, 2}, {4, 2, 2}, {5, 3, 1}, {7, 4, 2}, {8, 5, 1}, {9, 6, 1}, {10, 5, 2}, {11, 6, 2}},
      {{1, 1, 1}, {2, 2, 1}, {3, 1, 2}, {4, 2, 2}, {5, 3, 1}, {6, 4, 1}, {7, 3, 2}, {8, 4, 2}, {9, 5, 1}, {11, 6, 2}}};
  static const int diag[3] = {2, 6, 10};
  real s = 0.0;
  for (int t = 0; t < 10; ++t) {
    const int64_t cell = (tab[d - 1][t][2] == 1) ? n1 : n2;
    const real term = A(tab[d - 1][t][0], n1) * fr(o.F(tab[d - 1][t][1], cell));
    s = (t == 0) ? -term : s - term;
  }
  s = s - A(12, n1) * (c(n1) - cold(n1)) - A(14, n1) * (c(n2) - cold(n2));
  return (1 - w) * fr(o.F(2 * d, n1)) + w / (A(diag[d - 1], n1)) * (s + B1 + B2 + B3 + B4);
}

// calculate_R_b_p (nse.f90:2362-2407) + calculate_R_D_p2 (nse.f90:1863-1997)
void pressure_sources(nim_oracle &o) {
  const int64_t N = o.NMESH;
  const real DT = o.P.DT;
#pragma omp parallel for schedule(static) num_threads(o.nthreads)
  for (int64_t n = 1; n <= N; ++n) {
    int32_t nf[7];
    for (int k = 1; k <= 6; ++k) nf[k] = o.F(k, n);
    real uf[7], vf[7], wf[7], bzf[7];
    for (int k = 1; k <= 6; ++k) {
      uf[k] = o.fu(nf[k]);
      vf[k] = o.fv(nf[k]);
      wf[k] = o.fw(nf[k]);
      bzf[k] = o.fbz(nf[k]);
    }
    const real du_dx = green_gauss(o, uf, nf, n, 1), du_dy = green_gauss(o, uf, nf, n, 2),
                 du_dz = green_gauss(o, uf, nf, n, 3);
    const real dv_dx = green_gauss(o, vf, nf, n, 1), dv_dy = green_gauss(o, vf, nf, n, 2),
                 dv_dz = green_gauss(o, vf, nf, n, 3);
    const real dw_dx = green_gauss(o, wf, nf, n, 1), dw_dy = green_gauss(o, wf, nf, n, 2),
                 dw_dz = green_gauss(o, wf, nf, n, 3);
    const real dbz_dz = green_gauss(o, bzf, nf, n, 3);  // faces_bx = faces_by = 0
    const real Dila = du_dx + dv_dy + dw_dz;
    o.dila(n) = Dila;
    o.RBp(n) = -(du_dx * du_dx + dv_dy * dv_dy + dw_dz * dw_dz) -
               2.0 * (du_dy * dv_dx + dv_dz * dw_dy + dw_dx * du_dz) - dbz_dz + Dila / (2 * DT);
    o.RDp(n) = 1 / o.P.rho * diffusion_source(o, o.fp, n);
  }
}

// apply_pressure_bc for boundary face i (bc.f90:148-339); reads pr.
real pressure_bc_face(const nim_oracle &o, const V1 &pr, int64_t i) {
  const int64_t M1 = o.BCm[i];
  const int pos = o.BCpos[i];
  const int32_t fw = o.BCf[i];
  const real *n = &o.fnormal(1, fw);
  const real b[3] = {0., 0., o.fbz(fw)};
  const real b_n = dot3(b, n);
  real vn[6];
  for (int j = 1; j <= 5; ++j) {
    const int32_t pt = o.BCpts(j, i);
    const real v[3] = {o.fu(pt), o.fv(pt), o.fw(pt)};
    vn[j] = dot3(v, n);
  }
  const real d2udn2 = -(o.BCa(1, i) * vn[1]) - o.BCa(2, i) * vn[2] - o.BCa(3, i) * vn[3] - o.BCa(4, i) * vn[4] -
                        o.BCa(5, i) * vn[5];
  const int d = (pos + 1) / 2;
  const int e1 = (d == 1) ? 2 : 1, e2 = (d == 3) ? 2 : 3;
  const int fn = pos;
  real B2 = tangential(o, pr, M1, fn, e1);
  // position 6, centred branch, uses meshes_gij_faces(3,2,...) (bc.f90:318)
  const bool centred_e1 = (o.NB(2 * e1 - 1, M1) != 0 && o.NB(2 * e1, M1) != 0);
  const int e1g = (pos == 6 && centred_e1) ? 2 : e1;
  B2 = B2 * o.gf(d, e1g, fn, M1);
  const real B3 = tangential(o, pr, M1, fn, e2) * o.gf(d, e2, fn, M1);
  const real B1 = o.BCap(8, i) * (o.RDp(M1) + o.RBp(M1));
  real s = 0.0;
  bool first = true;
  for (int k = 1; k <= 6; ++k) {
    if (k == pos) continue;
    const real t = o.BCap(k, i) * pr(o.F(k, M1));
    s = first ? -t : s - t;
    first = false;
  }
  const real w = o.P.w_p2;
  return (1 - w) * pr(o.F(pos, M1)) +
         w / (o.BCap(pos, i)) * (s + B1 - B2 - B3 + (o.nu * o.P.rho * d2udn2 - b_n * o.P.rho));
}

// integrate_pressure_field_i for the +d face of cell n1 (nse.f90:1105-1288).
real pressure_face(const nim_oracle &o, const V1 &pr, int d, int64_t n1) {
  const int64_t n2 = o.NB(2 * d, n1);
  const VK<15> &A = (d == 1) ? o.AApx : (d == 2) ? o.AApy : o.AApz;
  const int e1 = (d == 1) ? 2 : 1, e2 = (d == 3) ? 2 : 3;
  const real B1 = (o.RDp(n1) + o.RBp(n1)) * A(13, n1);
  const real B2 = (o.RDp(n2) + o.RBp(n2)) * A(15, n1);
  const real B3 = (o.gf(d, e1, 2 * d - 1, n2) - o.gf(d, e1, 2 * d, n1)) * tangential(o, pr, n1, 2 * d, e1);
  const real B4 = (o.gf(d, e2, 2 * d - 1, n2) - o.gf(d, e2, 2 * d, n1)) * tangential(o, pr, n1, 2 * d, e2);
  // the ten off-diagonal terms in source order: (coefficient, face, cell)
  static const int tab[3][10][3] = {
      {{1, 1, 1}, {3, 2, 2}, {4, 3, 1}, {5, 4, 1}, {6, 3, 2}, {7, 4, 2}, {8, 5, 1}, {9, 6, 1}, {10, 5, 2}, {11, 6, 2}},
      {{1, 1, 1}, {2, 2, 1}, {3, 1, 2}, {4, 2, 2}, {5, 3, 1}, {7, 4, 2}, {8, 5, 1}, {9, 6, 1}, {10, 5, 2}, {11, 6, 2}},
      {{1, 1, 1}, {2, 2, 1}, {3, 1, 2}, {4, 2, 2}, {5, 3, 1}, {6, 4, 1}, {7, 3, 2}, {8, 4, 2}, {9, 5, 1}, {11, 6, 2}}};
  static const int diag[3] = {2, 6, 10};
  real s = 0.0;
  for (int t = 0; t < 10; ++t) {
    const int64_t cell = (tab[d - 1][t][2] == 1) ? n1 : n2;
    const real term = A(tab[d - 1][t][0], n1) * pr(o.F(tab[d - 1][t][1], cell));
    s = (t == 0) ? -term : s - term;
  }
  const real w = o.P.w_p;
  return (1 - w) * pr(o.F(2 * d, n1)) + w / (A(diag[d - 1], n1)) * (s + B1 + B2 + B3 + B4);
}

// apply_zero_flux (bc.f90:345-390): third-order zero-gradient extrapolation of
// T onto the bottom (position 5) and top (position 6) walls.
void zero_flux(nim_oracle &o) {
  for (int64_t i = 1; i <= o.NBF; ++i) {
    const int pos = o.BCpos[i];
    if (pos != 5 && pos != 6) continue;
    const int64_t M = o.BCm[i];
    const int in = (pos == 5) ? 6 : 5;
    const int32_t f1 = o.BCf[i], f2 = o.F(in, M), f3 = o.F(in, o.NB(in, M)), f4 = o.F(in, o.NB(in, o.NB(in, M)));
    auto dist = [&](int32_t a, int32_t b) {
      return sqrt(sq(o.fmid(1, a) - o.fmid(1, b)) + sq(o.fmid(2, a) - o.fmid(2, b)) + sq(o.fmid(3, a) - o.fmid(3, b)));
    };
    const real h1 = dist(f1, f2), h2 = dist(f2, f3), h3 = dist(f3, f4);
    o.fT(f1) = (+((h1 + h2) * (h1 + h2 + h3)) / (h1 * h2 * (h2 + h3)) * o.fT(f2) -
                (h1 * (h1 + h2 + h3)) / (h2 * h3 * (h1 + h2)) * o.fT(f3) +
                (h1 * (h1 + h2)) / (h3 * (h2 + h3) * (h1 + h2 + h3)) * o.fT(f4)) /
               (1. / h1 + 1. / (h1 + h2) + 1. / (h1 + h2 + h3));
  }
}

// find_error (nse.f90:260-325)
void find_error(nim_oracle &o) {
  real e[5] = {0, 0, 0, 0, 0};
  V1 *cur[5] = {&o.fu, &o.fv, &o.fw, &o.fp, &o.fT};
  V1 *old[5] = {&o.fuo, &o.fvo, &o.fwo, &o.fpo, &o.fTo};
  for (int64_t i = 1; i <= o.NFACE; ++i)
    for (int k = 0; k < 5; ++k) {
      e[k] = std::max(e[k], fabs((*cur[k])(i) - (*old[k])(i)));
      (*old[k])(i) = (*cur[k])(i);
    }
  if (o.P.dpdx_tolerance) {
    real ex = 0, ey = 0, ez = 0;
    for (int64_t i = 1; i <= o.NMESH; ++i) {
      o.dpdx(i) = (o.fp(o.F(2, i)) - o.fp(o.F(1, i))) / 2. * o.xi_x(1, 1, i);
      o.dpdy(i) = (o.fp(o.F(4, i)) - o.fp(o.F(3, i))) / 2. * o.xi_x(2, 2, i);
      o.dpdz(i) = (o.fp(o.F(6, i)) - o.fp(o.F(5, i))) / 2. * o.xi_x(3, 3, i);
      ex = std::max(ex, fabs(o.dpdx(i) - o.dpdxo(i)));
      ey = std::max(ey, fabs(o.dpdy(i) - o.dpdyo(i)));
      ez = std::max(ez, fabs(o.dpdz(i) - o.dpdzo(i)));
      o.dpdxo(i) = o.dpdx(i);
      o.dpdyo(i) = o.dpdy(i);
      o.dpdzo(i) = o.dpdz(i);
    }
    e[3] = std::max(ex, std::max(ey, ez));
  }
  V1 *cc[4] = {&o.uxyz, &o.vxyz, &o.wxyz, &o.Txyz};
  V1 *co[4] = {&o.uoc, &o.voc, &o.woc, &o.Toc};
  const int slot[4] = {0, 1, 2, 4};
  real ce[4] = {0, 0, 0, 0};
  for (int64_t i = 1; i <= o.NMESH; ++i)
    for (int k = 0; k < 4; ++k) {
      ce[k] = std::max(ce[k], fabs((*cc[k])(i) - (*co[k])(i)));
      (*co[k])(i) = (*cc[k])(i);
    }
  for (int k = 0; k < 4; ++k) e[slot[k]] = std::max(e[slot[k]], ce[k]);
  for (int k = 0; k < 5; ++k) o.err[k] = e[k];
}

// One pass of the integrate_nse loop body (nse.f90:131-160).
void iteration(nim_oracle &o) {
  const int64_t N = o.NMESH;
  const int nt = o.nthreads;
  const bool seq = (o.sched != NIM_SCHED_PARALLEL);
  V1 *vf[3] = {&o.fu, &o.fv, &o.fw};
  V1 *vc[3] = {&o.uxyz, &o.vxyz, &o.wxyz};
  V1 *vo[3] = {&o.uold, &o.vold, &o.wold};
  V1 *RD[3] = {&o.RDu, &o.RDv, &o.RDw};
  V1 *RB[3] = {&o.RBu, &o.RBv, &o.RBw};
  const real wv[3] = {o.P.w_u, o.P.w_v, o.P.w_w};
  VK<5> *MF[3] = {&o.MF1, &o.MF2, &o.MF3};
  VK<5> *MTF[3] = {&o.MTF1, &o.MTF2, &o.MTF3};

  // ---- velocity
  velocity_sources(o);
  const bool f1 = (o.P.formulation == 1);
  auto vcell = [&](int k, int64_t i) {
    const real B = (0. + (*RD[k])(i) + (*RB[k])(i));  // R_C = 0
    return f1 ? cell_update_f1(o, *vf[k], (*vc[k])(i), (*vo[k])(i), B, i, wv[k])
              : cell_update(o, *vf[k], (*vc[k])(i), (*vo[k])(i), B, o.MF4, i, wv[k]);
  };
  auto vface = [&](int k, const V1 &fr, int d, int64_t i) {
    return f1 ? face_update_f1(o, fr, *vc[k], *vo[k], *RD[k], *RB[k], d, i, wv[k])
              : face_update(o, fr, *vc[k], *vo[k], *MF[d - 1], d, i, wv[k]);
  };
  if (seq) {
#pragma omp parallel for schedule(static) num_threads(nt)
    for (int64_t q = 0; q < N; ++q) {
      const int64_t i = o.cord[q];
      for (int k = 0; k < 3; ++k) (*vc[k])(i) = vcell(k, i);
      for (int d = 1; d <= 3; ++d) {
        if (o.NB(2 * d, i) == 0) continue;
        for (int k = 0; k < 3; ++k) (*vf[k])(o.F(2 * d, i)) = vface(k, *vf[k], d, i);
      }
    }
  } else {
    // every parallel-schedule loop reads only values from before the loop,
    // so its threads write disjoint entries and the result is thread-count
    // independent
#pragma omp parallel for schedule(static) num_threads(nt)
    for (int64_t i = 1; i <= N; ++i)
      for (int k = 0; k < 3; ++k) (*vc[k])(i) = vcell(k, i);
    for (int k = 0; k < 3; ++k) {
      o.snap.d = vf[k]->d;
#pragma omp parallel for schedule(static) num_threads(nt)
      for (int64_t i = 1; i <= N; ++i)
        for (int d = 1; d <= 3; ++d)
          if (o.NB(2 * d, i) != 0) (*vf[k])(o.F(2 * d, i)) = vface(k, o.snap, d, i);
    }
  }

  // ---- pressure
  pressure_sources(o);
  if (seq) {
    for (int64_t q = 0; q < o.NBF; ++q) {
      const int64_t b = o.bord[q];
      o.fp(o.F(o.BCpos[b], o.BCm[b])) = pressure_bc_face(o, o.fp, b);
    }
#pragma omp parallel for schedule(static) num_threads(nt)
    for (int64_t q = 0; q < N; ++q)
      for (int d = 1, n = (int)o.cord[q]; d <= 3; ++d)
        if (o.faces_BC[o.F(2 * d, n)] == 1) o.fp(o.F(2 * d, n)) = pressure_face(o, o.fp, d, n);
  } else {
#pragma omp parallel for schedule(static) num_threads(nt)
    for (int64_t b = 1; b <= o.NBF; ++b) o.pb_new(b) = pressure_bc_face(o, o.fp, b);
    for (int64_t b = 1; b <= o.NBF; ++b) o.fp(o.F(o.BCpos[b], o.BCm[b])) = o.pb_new(b);
    o.snap.d = o.fp.d;
#pragma omp parallel for schedule(static) num_threads(nt)
    for (int64_t n = 1; n <= N; ++n)
      for (int d = 1; d <= 3; ++d)
        if (o.faces_BC[o.F(2 * d, n)] == 1) o.fp(o.F(2 * d, n)) = pressure_face(o, o.snap, d, n);
  }

  // ---- temperature
  temperature_constants(o);
  zero_flux(o);
#pragma omp parallel for schedule(static) num_threads(nt)
  for (int64_t i = 1; i <= N; ++i) o.RDT(i) = o.alpha * diffusion_source(o, o.fT, i);
  if (seq) {
#pragma omp parallel for schedule(static) num_threads(nt)
    for (int64_t q = 0; q < N; ++q) {
      const int64_t i = o.cord[q];
      o.Txyz(i) = cell_update(o, o.fT, o.Txyz(i), o.Told(i), (o.RDT(i) + 0.), o.MTF4, i, o.P.w_T);
      for (int d = 1; d <= 3; ++d)
        if (o.NB(2 * d, i) != 0) o.fT(o.F(2 * d, i)) = face_update(o, o.fT, o.Txyz, o.Told, *MTF[d - 1], d, i, o.P.w_T);
    }
  } else {
#pragma omp parallel for schedule(static) num_threads(nt)
    for (int64_t i = 1; i <= N; ++i)
      o.Txyz(i) = cell_update(o, o.fT, o.Txyz(i), o.Told(i), (o.RDT(i) + 0.), o.MTF4, i, o.P.w_T);
    o.snap.d = o.fT.d;
#pragma omp parallel for schedule(static) num_threads(nt)
    for (int64_t i = 1; i <= N; ++i)
      for (int d = 1; d <= 3; ++d)
        if (o.NB(2 * d, i) != 0) o.fT(o.F(2 * d, i)) = face_update(o, o.snap, o.Txyz, o.Told, *MTF[d - 1], d, i, o.P.w_T);
  }
  find_error(o);
  o.first_iteration = false;
}

// check_steady_state (nse.f90:1316-1332) and evaluate_D (nse.f90:2504-2537)
void after_integrate(nim_oracle &o) {
  const real tdt = 2 * o.P.DT;
  real mu = 0, mv = 0, mw = 0, mT = 0;
  for (int64_t i = 1; i <= o.NMESH; ++i) {
    mu = std::max(mu, fabs(o.uxyz(i) - o.uold(i)) / tdt);
    mv = std::max(mv, fabs(o.vxyz(i) - o.vold(i)) / tdt);
    mw = std::max(mw, fabs(o.wxyz(i) - o.wold(i)) / tdt);
    mT = std::max(mT, fabs(o.Txyz(i) - o.Told(i)) / tdt);
  }
  o.dudt_max = std::max(mw, std::max(mu, mv));
  o.dTdt_max = mT;
  real sum1 = 0.0;
  for (int64_t n = 1; n <= o.NMESH; ++n) {
    int32_t nf[7];
    for (int k = 1; k <= 6; ++k) nf[k] = o.F(k, n);
    real uf[7], vf[7], wf[7];
    for (int k = 1; k <= 6; ++k) {
      uf[k] = o.fu(nf[k]);
      vf[k] = o.fv(nf[k]);
      wf[k] = o.fw(nf[k]);
    }
    const real Dila = green_gauss(o, uf, nf, n, 1) + green_gauss(o, vf, nf, n, 2) + green_gauss(o, wf, nf, n, 3);
    o.dila(n) = Dila;
    sum1 = sum1 + Dila * Dila;
  }
  o.Dilatation = sqrt(sum1 / o.NMESH);
}

void fill_integrate_stats(const nim_oracle &o, nim_step_stats *s, int iters) {
  if (!s) return;
  s->step = o.STEP;
  s->iters = iters;
  s->err_u = val(o.err[0]);
  s->err_v = val(o.err[1]);
  s->err_w = val(o.err[2]);
  s->err_p = val(o.err[3]);
  s->err_T = val(o.err[4]);
  s->dilatation = val(o.Dilatation);
  s->dudt_max = val(o.dudt_max);
  s->dTdt_max = val(o.dTdt_max);
}

// The visiting orders of the Gauss-Seidel sweeps.  SEQUENTIAL: cell number
// and BC-list order, as the reference's loops run.  LEVELS: cells by the level
// i + 2j + 3k (theta, r, z indices of the structured numbering) and wall faces
// by i + 2j (bottom, top) or i + 2k (inner, outer), the order the CUDA
// library's reference-order sweeps follow; inside a level the numbers run
// downwards and the walls come as top, bottom, outer, inner, so that any
// dependence between faces or cells the level order treats as independent
// changes the result.
void visiting_orders(nim_oracle &o, int NT, int NR, int NZ) {
  const int64_t N = o.NMESH, NB = o.NBF;
  o.cord.resize(N);
  o.bord.resize(NB);
  for (int64_t q = 0; q < N; ++q) o.cord[q] = q + 1;
  for (int64_t q = 0; q < NB; ++q) o.bord[q] = q + 1;
  if (o.sched != NIM_SCHED_LEVELS) return;
  auto by_level = [](std::vector<std::pair<int64_t, int64_t>> &v) {
    std::sort(v.begin(), v.end(), [](const auto &a, const auto &b) {
      return a.first != b.first ? a.first < b.first : a.second > b.second;
    });
  };
  std::vector<std::pair<int64_t, int64_t>> v;
  for (int64_t c = 0; c < N; ++c) {
    const int64_t i = c % NT, j = (c / NT) % NR, k = c / ((int64_t)NT * NR);
    v.push_back({i + 2 * j + 3 * k, c + 1});
  }
  by_level(v);
  for (int64_t q = 0; q < N; ++q) o.cord[q] = v[q].second;
  const int64_t nb1 = (int64_t)NT * NR, nb3 = (int64_t)NT * NZ;
  const int64_t w0[4] = {nb1, 0, 2 * nb1 + nb3, 2 * nb1};  // top, bottom, outer, inner
  const int64_t wn[4] = {nb1, nb1, nb3, nb3};
  int64_t q = 0;
  for (int w = 0; w < 4; ++w) {
    v.clear();
    for (int64_t r = 0; r < wn[w]; ++r) v.push_back({r % NT + 2 * (r / NT), w0[w] + r + 1});
    by_level(v);
    for (const auto &e : v) o.bord[q++] = e.second;
  }
}

}  // namespace

// ================================================================ C API
extern "C" int NIM_ORACLE_FN(create)(const nim_mesh_desc *m, const nim_params *p, int32_t schedule,
                                 int32_t threads, nim_oracle **out) {
  if (!m || !p || !out) return NIM_ERR_BAD_ARG;
  if (m->nmesh <= 0 || m->nface <= 0 || m->nnode <= 0 || m->nbcface <= 0) return NIM_ERR_BAD_ARG;
  if (p->formulation != 1 && p->formulation != 2) return NIM_ERR_BAD_ARG;
  auto *o = new nim_oracle();
  o->sched = schedule;
  o->nthreads = threads > 0 ? threads : 1;
  o->P = *p;
  o->nu = p->nu;
  o->alpha = p->alpha;
  o->Re = 1. / o->nu;       // parameters.f90:172
  o->inv_Re = 1 / o->Re;    // the 1/Re factor of calculate_R_D2
  o->NMESH = m->nmesh;
  o->NFACE = m->nface;
  o->NNODE = m->nnode;
  o->NBF = m->nbcface;
  const int64_t N = o->NMESH, NF = o->NFACE, NB = o->NBF;
  o->node_xyz.assign(m->node_xyz, m->node_xyz + 3 * o->NNODE);
  o->mnodes.alloc(N);
  o->mfaces.alloc(N);
  o->mnb.alloc(N);
  for (int64_t i = 1; i <= N; ++i) {
    for (int k = 1; k <= 8; ++k) o->mnodes(k, i) = m->meshes_nodes[8 * (i - 1) + k - 1];
    for (int k = 1; k <= 6; ++k) {
      o->mfaces(k, i) = m->meshes_faces[6 * (i - 1) + k - 1];
      o->mnb(k, i) = m->meshes_neighbors[6 * (i - 1) + k - 1];
    }
  }
  o->faces_BC.assign(NF + 1, 0);
  for (int64_t f = 1; f <= NF; ++f) o->faces_BC[f] = m->faces_bc[f - 1];
  o->BCf.assign(NB + 1, 0);
  o->BCid.assign(NB + 1, 0);
  o->BCpos.assign(NB + 1, 0);
  o->BCm.assign(NB + 1, 0);
  for (int64_t b = 1; b <= NB; ++b) {
    o->BCf[b] = m->bcs_faces[b - 1];
    o->BCid[b] = m->bcs_faces_id[b - 1];
    o->BCpos[b] = m->bcs_faces_position[b - 1];
    o->BCm[b] = m->bcs_faces_mesh_num[b - 1];
  }
  o->BCpts.alloc(NB);
  o->maps.assign(N + 1, Map{});
  o->volume.alloc(N); o->G1.alloc(N); o->G2.alloc(N); o->G3.alloc(N);
  o->faces_area.alloc(NF);
  o->gij.alloc(N); o->xi_x.alloc(N); o->gf.alloc(N);
  o->fnormal.alloc(NF); o->ftan.alloc(NF); o->fbitan.alloc(NF); o->fmid.alloc(NF);
  o->BCa.alloc(NB); o->BCap.alloc(NB);
  o->AApx.alloc(N); o->AApy.alloc(N); o->AApz.alloc(N);
  for (V1 *v : {&o->uxyz, &o->vxyz, &o->wxyz, &o->Txyz, &o->uold, &o->vold, &o->wold, &o->Told, &o->ut,
                &o->vt, &o->wt, &o->Tt, &o->uoc, &o->voc, &o->woc, &o->Toc, &o->mu, &o->mv, &o->mw, &o->mp,
                &o->dila, &o->dila_old, &o->RBu, &o->RBv, &o->RBw, &o->RDu, &o->RDv, &o->RDw, &o->RBp,
                &o->RDp, &o->RDT, &o->bz, &o->dpdx, &o->dpdy, &o->dpdz, &o->dpdxo, &o->dpdyo, &o->dpdzo})
    v->alloc(N);
  for (V1 *v : {&o->fu, &o->fv, &o->fw, &o->fp, &o->fT, &o->fuo, &o->fvo, &o->fwo, &o->fpo, &o->fTo, &o->fbz})
    v->alloc(NF);
  o->pb_new.alloc(NB);
  visiting_orders(*o, m->n_theta, m->n_r, m->n_z);
  o->MA.alloc(N); o->MTA.alloc(N);
  o->MF1.alloc(N); o->MF2.alloc(N); o->MF3.alloc(N); o->MTF1.alloc(N); o->MTF2.alloc(N); o->MTF3.alloc(N);
  o->MF4.alloc(N); o->MTF4.alloc(N);
  if (p->formulation == 1) {
    o->at.alloc(N); o->AAvx.alloc(N); o->AAvy.alloc(N); o->AAvz.alloc(N);
  }
  *out = o;
  return NIM_OK;
}

// initialize_nse (nse.f90:89-112) + apply_all_dirichlet_bcs (bc.f90:13-57),
// TI = DT, STEP = 1 (nse.f90:31-32).
extern "C" int NIM_ORACLE_FN(init)(nim_oracle *o) {
  if (!o) return NIM_ERR_BAD_ARG;
  o->TI = o->P.DT;
  o->STEP = 1;
#pragma omp parallel for schedule(static) num_threads(o->nthreads)
  for (int64_t i = 1; i <= o->NMESH; ++i) mapping_coefficients(*o, i);
  // Shared faces get their geometry from both cells; in the reference's
  // serial loop the higher cell number writes last and wins, so only that
  // cell (face_owner) writes here and the loop can run in parallel.
  o->face_owner.assign(o->NFACE + 1, 0);
  for (int64_t i = 1; i <= o->NMESH; ++i)
    for (int k = 1; k <= 6; ++k) o->face_owner[o->F(k, i)] = std::max<int64_t>(o->face_owner[o->F(k, i)], i);
#pragma omp parallel for schedule(dynamic, 64) num_threads(o->nthreads)
  for (int64_t i = 1; i <= o->NMESH; ++i) cell_geometry(*o, i);
  pressure_bc_array(*o);
  pressure_constants(*o);
  // initial conditions are zero (general.f90:16-31); Dirichlet faces:
  V1 *ff[5] = {&o->fu, &o->fv, &o->fw, &o->fp, &o->fT};
  for (int64_t b = 1; b <= o->NBF; ++b) {
    const int64_t M = o->BCm[b];
    const int pos = o->BCpos[b];
    const int id = o->BCid[b];
    for (int fld : {0, 1, 2, 4})  // apply_dirichlet_pressure_bcs is not called
      (*ff[fld])(o->BCf[b]) = dirichlet_face_value(*o, M, pos, o->P.bc_value[fld][id - 1]);
  }
  o->initialized = true;
  o->first_iteration = true;
  return NIM_OK;
}

extern "C" int NIM_ORACLE_FN(begin_step)(nim_oracle *o) {
  if (!o || !o->initialized) return NIM_ERR_STATE;
  if (o->P.formulation == 1)
    velocity_constants_f1(*o);
  else
    velocity_constants(*o);
  return NIM_OK;
}

extern "C" int NIM_ORACLE_FN(iterate)(nim_oracle *o, int32_t n, nim_step_stats *s) {
  if (!o || !o->initialized) return NIM_ERR_STATE;
  for (int32_t k = 0; k < n; ++k) iteration(*o);
  fill_integrate_stats(*o, s, n);
  return NIM_OK;
}

extern "C" int NIM_ORACLE_FN(integrate)(nim_oracle *o, nim_step_stats *s) {
  if (!o || !o->initialized) return NIM_ERR_STATE;
  int cnt = 0;
  double e[5] = {1., 1., 1., 1., 1.};
  const double tol[5] = {o->P.tol_u, o->P.tol_v, o->P.tol_w, o->P.tol_p, o->P.tol_T};
  int status = NIM_OK;
  auto busy = [&]() {
    for (int k = 0; k < 5; ++k)
      if (e[k] > tol[k]) return true;
    return false;
  };
  while (busy()) {
    if (o->P.max_iters > 0 && cnt >= o->P.max_iters) {
      status = NIM_ERR_NOT_CONVERGED;
      break;
    }
    ++cnt;
    iteration(*o);
    for (int k = 0; k < 5; ++k) e[k] = val(o->err[k]);
    bool finite = true;
    for (int k = 0; k < 5; ++k) finite = finite && std::isfinite(e[k]);
    if (!finite) {
      status = NIM_ERR_NONFINITE;
      break;
    }
  }
  after_integrate(*o);
  fill_integrate_stats(*o, s, cnt);
  if (s) s->status = status;
  return status;
}

// update_time_step (nse.f90:1292-1313) + find_Nu2 (nse.f90:2699-2798)
extern "C" int NIM_ORACLE_FN(end_step)(nim_oracle *o, nim_step_stats *s) {
  if (!o || !o->initialized) return NIM_ERR_STATE;
  const int step_done = o->STEP;
  o->STEP = o->STEP + 1;
  o->TI = o->TI + 2 * o->P.DT;
  for (int64_t i = 1; i <= o->NMESH; ++i) {
    o->ut(i) = (o->uold(i) + o->uxyz(i)) / 2.;
    o->uold(i) = o->uxyz(i);
    o->vt(i) = (o->vold(i) + o->vxyz(i)) / 2.;
    o->vold(i) = o->vxyz(i);
    o->wt(i) = (o->wold(i) + o->wxyz(i)) / 2.;
    o->wold(i) = o->wxyz(i);
    o->Tt(i) = (o->Told(i) + o->Txyz(i)) / 2.;
    o->Told(i) = o->Txyz(i);
    o->mp(i) = (o->fp(o->F(1, i)) + o->fp(o->F(2, i)) + o->fp(o->F(3, i)) + o->fp(o->F(4, i)) +
                o->fp(o->F(5, i)) + o->fp(o->F(6, i))) / 6.0;
    o->dila_old(i) = o->dila(i);
  }
  real sum1 = 0., sum2 = 0., sumA1 = 0., sumA2 = 0.;
  for (int64_t i = 1; i <= o->NBF; ++i) {
    const int pos = o->BCpos[i];
    if (pos != 1 && pos != 2) continue;
    const int64_t M = o->BCm[i];
    const int in = (pos == 1) ? 2 : 1;
    const int32_t f1 = o->BCf[i], f2 = o->F(in, M), f3 = o->F(in, o->NB(in, M)),
                  f4 = o->F(in, o->NB(in, o->NB(in, M)));
    auto dist = [&](int32_t a, int32_t b) {
      return sqrt(sq(o->fmid(1, a) - o->fmid(1, b)) + sq(o->fmid(2, a) - o->fmid(2, b)) +
                       sq(o->fmid(3, a) - o->fmid(3, b)));
    };
    const real h1 = dist(f1, f2), h2 = dist(f2, f3), h3 = dist(f3, f4);
    const real inner = -((1. / h1 + 1. / (h1 + h2) + 1. / (h1 + h2 + h3)) * o->fT(f1)) +
                         ((h1 + h2) * (h1 + h2 + h3)) / (h1 * h2 * (h2 + h3)) * o->fT(f2) -
                         (h1 * (h1 + h2 + h3)) / (h2 * h3 * (h1 + h2)) * o->fT(f3) +
                         (h1 * (h1 + h2)) / (h3 * (h2 + h3) * (h1 + h2 + h3)) * o->fT(f4);
    const real dTdx = (pos == 1) ? -(inner) : inner;
    const real A = o->faces_area(o->F(pos, M));
    if (pos == 1) {
      sum2 = sum2 + A * dTdx;
      sumA2 = sumA2 + A;
    } else {
      sum1 = sum1 + A * dTdx;
      sumA1 = sumA1 + A;
    }
  }
  const real nu_outer = -(sum1 / sumA1 * o->P.R_o), nu_inner = -(sum2 / sumA2 * o->P.R_i);
  o->nu_tan[0] = tan_of(nu_inner);
  o->nu_tan[1] = tan_of(nu_outer);
  if (s) {
    s->step = step_done;
    s->nu_outer = val(nu_outer);
    s->nu_inner = val(nu_inner);
    s->area_outer = val(sumA1);
    s->area_inner = val(sumA2);
    s->time = val(o->TI);
  }
  return NIM_OK;
}

// The solve_nse time loop (nse.f90:47-75)
extern "C" int NIM_ORACLE_FN(step)(nim_oracle *o, int32_t nsteps, nim_step_stats *per, int32_t *done) {
  if (!o || !o->initialized) return NIM_ERR_STATE;
  int32_t k = 0;
  int status = NIM_OK;
  for (; k < nsteps; ++k) {
    nim_step_stats st{};
    NIM_ORACLE_FN(begin_step)(o);
    status = NIM_ORACLE_FN(integrate)(o, &st);
    if (status != NIM_OK) {
      st.status = status;
      if (per) per[k] = st;
      break;
    }
    if (o->P.check_steady && o->dudt_max < o->P.dudt_epsilon && o->dTdt_max < o->P.dudt_epsilon) {
      st.steady = 1;
      if (per) per[k] = st;
      ++k;
      break;
    }
    NIM_ORACLE_FN(end_step)(o, &st);
    if (per) per[k] = st;
  }
  if (done) *done = k;
  return status;
}

namespace {
int64_t field_len(const nim_oracle &o, int32_t f) {
  switch (f) {
    case NIM_FIELD_FACES_U: case NIM_FIELD_FACES_V: case NIM_FIELD_FACES_W: case NIM_FIELD_FACES_P:
    case NIM_FIELD_FACES_T: case NIM_FIELD_FACES_AREA:
      return o.NFACE;
    case NIM_FIELD_FACES_NORMAL: case NIM_FIELD_FACES_MID: case NIM_FIELD_FACES_TANGENTIAL:
    case NIM_FIELD_FACES_BITANGENTIAL:
      return 3 * o.NFACE;
    case NIM_FIELD_MESHES_GIJ: case NIM_FIELD_MESHES_XI_X: return 9 * o.NMESH;
    case NIM_FIELD_MESHES_G: return 3 * o.NMESH;
    case NIM_FIELD_MESHES_GIJ_FACES: return 54 * o.NMESH;
    case NIM_FIELD_BCS_FACES_A: return 5 * o.NBF;
    case NIM_FIELD_BCS_FACES_AP: return 8 * o.NBF;
    case NIM_FIELD_AA_PX: case NIM_FIELD_AA_PY: case NIM_FIELD_AA_PZ: return 15 * o.NMESH;
    case NIM_FIELD_M_F4: return 8 * o.NMESH;
    case NIM_FIELD_M_F1: case NIM_FIELD_M_F2: case NIM_FIELD_M_F3: return 5 * o.NMESH;
    default:
      if (f >= NIM_FIELD_MESHES_U && f <= NIM_FIELD_MESHES_DILA) return o.NMESH;
      if (f == NIM_FIELD_MESHES_VOLUME) return o.NMESH;
      return -1;
  }
}
V1 *field_ptr(nim_oracle &o, int32_t f) {
  switch (f) {
    case NIM_FIELD_FACES_U: return &o.fu;
    case NIM_FIELD_FACES_V: return &o.fv;
    case NIM_FIELD_FACES_W: return &o.fw;
    case NIM_FIELD_FACES_P: return &o.fp;
    case NIM_FIELD_FACES_T: return &o.fT;
    case NIM_FIELD_MESHES_U: return &o.uxyz;
    case NIM_FIELD_MESHES_V: return &o.vxyz;
    case NIM_FIELD_MESHES_W: return &o.wxyz;
    case NIM_FIELD_MESHES_T: return &o.Txyz;
    case NIM_FIELD_MESHES_U_OLD: return &o.uold;
    case NIM_FIELD_MESHES_V_OLD: return &o.vold;
    case NIM_FIELD_MESHES_W_OLD: return &o.wold;
    case NIM_FIELD_MESHES_T_OLD: return &o.Told;
    case NIM_FIELD_MESHES_UT: return &o.ut;
    case NIM_FIELD_MESHES_VT: return &o.vt;
    case NIM_FIELD_MESHES_WT: return &o.wt;
    case NIM_FIELD_MESHES_TT: return &o.Tt;
    case NIM_FIELD_MESHES_P: return &o.mp;
    case NIM_FIELD_MESHES_DILA: return &o.dila;
    case NIM_FIELD_MESHES_VOLUME: return &o.volume;
    case NIM_FIELD_FACES_AREA: return &o.faces_area;
    default: return nullptr;
  }
}
}  // namespace

extern "C" int NIM_ORACLE_FN(get)(nim_oracle *o, int32_t f, double *out, int64_t n) {
  if (!o || !out) return NIM_ERR_BAD_ARG;
  const int64_t len = field_len(*o, f);
  if (len < 0 || n < len) return NIM_ERR_BAD_ARG;
  if (V1 *v = field_ptr(*o, f)) {
    for (int64_t i = 0; i < len; ++i) out[i] = val(v->d[i + 1]);
    return NIM_OK;
  }
  const real *src = nullptr;
  switch (f) {
    case NIM_FIELD_FACES_NORMAL: src = o->fnormal.d.data() + 3; break;
    case NIM_FIELD_FACES_MID: src = o->fmid.d.data() + 3; break;
    case NIM_FIELD_FACES_TANGENTIAL: src = o->ftan.d.data() + 3; break;
    case NIM_FIELD_FACES_BITANGENTIAL: src = o->fbitan.d.data() + 3; break;
    case NIM_FIELD_MESHES_GIJ: src = o->gij.d.data() + 9; break;
    case NIM_FIELD_MESHES_XI_X: src = o->xi_x.d.data() + 9; break;
    case NIM_FIELD_MESHES_GIJ_FACES: src = o->gf.d.data() + 54; break;
    case NIM_FIELD_BCS_FACES_AP: src = o->BCap.d.data() + 8; break;
    case NIM_FIELD_AA_PX: src = o->AApx.d.data() + 15; break;
    case NIM_FIELD_AA_PY: src = o->AApy.d.data() + 15; break;
    case NIM_FIELD_AA_PZ: src = o->AApz.d.data() + 15; break;
    case NIM_FIELD_M_F4: src = o->MF4.d.data() + 8; break;
    case NIM_FIELD_M_F1: src = o->MF1.d.data() + 5; break;
    case NIM_FIELD_M_F2: src = o->MF2.d.data() + 5; break;
    case NIM_FIELD_M_F3: src = o->MF3.d.data() + 5; break;
    default: break;
  }
  if (src) {
    for (int64_t i = 0; i < len; ++i) out[i] = val(src[i]);
    return NIM_OK;
  }
  if (f == NIM_FIELD_MESHES_G) {
    for (int64_t i = 1; i <= o->NMESH; ++i) {
      out[3 * (i - 1) + 0] = val(o->G1(i));
      out[3 * (i - 1) + 1] = val(o->G2(i));
      out[3 * (i - 1) + 2] = val(o->G3(i));
    }
    return NIM_OK;
  }
  if (f == NIM_FIELD_BCS_FACES_A) {
    for (int64_t b = 1; b <= o->NBF; ++b)
      for (int k = 1; k <= 5; ++k) out[5 * (b - 1) + k - 1] = val(o->BCa(k, b));
    return NIM_OK;
  }
  return NIM_ERR_BAD_ARG;
}

extern "C" int NIM_ORACLE_FN(set)(nim_oracle *o, int32_t f, const double *in, int64_t n) {
  if (!o || !in) return NIM_ERR_BAD_ARG;
  const int64_t len = field_len(*o, f);
  V1 *v = field_ptr(*o, f);
  if (!v || len < 0 || n < len || f >= NIM_FIELD_MESHES_VOLUME) return NIM_ERR_BAD_ARG;
  for (int64_t i = 0; i < len; ++i) v->d[i + 1] = in[i];  // values; derivatives start at zero
  return NIM_OK;
}

extern "C" double NIM_ORACLE_FN(max_rc)(nim_oracle *o) { return o ? o->max_rc : -1.0; }
extern "C" void NIM_ORACLE_FN(destroy)(nim_oracle *o) { delete o; }

extern "C" void NIM_ORACLE_FN(set_threads)(nim_oracle *o, int32_t threads) {
  if (o) o->nthreads = threads > 0 ? threads : 1;
}

// M_A(d,1:6) of nim.f90:181-287 for one direction (exposed for the
// continuity test of the exact and series branches).
extern "C" void NIM_ORACLE_FN(nim_coefficients)(double u, double k, double gminus, double gplus, double v_limit,
                                            double *A) {
  real a[6];
  nim_direction(u, k, gminus, gplus, v_limit, a);
  for (int q = 0; q < 6; ++q) A[q] = val(a[q]);
}

extern "C" void NIM_ORACLE_FN(nim1_coefficients)(double u, double F, double D, double v_limit, double *out) {
  const Nim1 r = nim1_direction(u, F, 2 * u / F, v_limit);
  out[0] = val(r.B);
  out[1] = val(r.C);
  out[2] = val(nim1_E(r, u, F, D));
  out[3] = val(nim1_F(r, u, F, D));
  out[4] = val(r.G);
  out[5] = val(r.H);
  out[6] = val(r.I);
  out[7] = val(r.J);
}

#ifdef NIM_ORACLE_TANGENT
// ---- tangent-linear entry points: the derivatives along one direction of
// (nu, alpha) and the initial/boundary values.
// Seeds d nu and d alpha (Re and 1/Re follow, parameters.f90:172).  For a
// derivative with respect to Ra or Pr: nu = sqrt(Pr / Ra) and alpha = nu / Pr
// (g_beta = th_tc = 1, parameters.f90:169-173), so d/dRa seeds
// (-nu / (2 Ra), -alpha / (2 Ra)) and d/dPr (nu / (2 Pr), -alpha / (2 Pr)).
extern "C" int nim_oracle_tl_seed_params(nim_oracle *o, double dnu, double dalpha) {
  if (!o) return NIM_ERR_BAD_ARG;
  o->nu = nimtl::Dual(o->P.nu, dnu);
  o->alpha = nimtl::Dual(o->P.alpha, dalpha);
  o->Re = 1. / o->nu;
  o->inv_Re = 1 / o->Re;
  return NIM_OK;
}
// derivatives of a state field (the values as nim_oracle_tl_get returns them)
extern "C" int nim_oracle_tl_get_tangent(nim_oracle *o, int32_t f, double *out, int64_t n) {
  if (!o || !out) return NIM_ERR_BAD_ARG;
  const int64_t len = field_len(*o, f);
  V1 *v = field_ptr(*o, f);
  if (!v || len < 0 || n < len) return NIM_ERR_BAD_ARG;
  for (int64_t i = 0; i < len; ++i) out[i] = v->d[i + 1].t;
  return NIM_OK;
}
// seeds the derivatives of a state field (e.g. of the outer-wall faces of
// faces_T: the Dirichlet temperatures, written once at init and never swept)
extern "C" int nim_oracle_tl_set_tangent(nim_oracle *o, int32_t f, const double *in, int64_t n) {
  if (!o || !in) return NIM_ERR_BAD_ARG;
  const int64_t len = field_len(*o, f);
  V1 *v = field_ptr(*o, f);
  if (!v || len < 0 || n < len || f >= NIM_FIELD_MESHES_VOLUME) return NIM_ERR_BAD_ARG;
  for (int64_t i = 0; i < len; ++i) v->d[i + 1].t = in[i];
  return NIM_OK;
}
// d Nu_inner, d Nu_outer of the last end_step (find_Nu2, nse.f90:2794-2795)
extern "C" int nim_oracle_tl_nu_tangent(nim_oracle *o, double *out2) {
  if (!o || !out2) return NIM_ERR_BAD_ARG;
  out2[0] = o->nu_tan[0];
  out2[1] = o->nu_tan[1];
  return NIM_OK;
}
#endif

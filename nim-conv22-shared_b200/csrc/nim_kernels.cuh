// Device kernels of the NIM time advance.
//
// Each kernel restates one or more reference routines; the file:line of the
// routine is given at the kernel.  Arithmetic follows the reference's
// expression order (built with -fmad=false, IEEE division/sqrt, and nim_exp,
// which gives glibc's exp bit for bit) so every value matches the CPU
// oracle's parallel schedule to the last bit.
//
// Iteration schedule (one pass of integrate_nse, nse.f90:131-160), parity
// par = ctrl->iter & 1 selects the current half of every double-buffered face
// array; the other half receives the sweep's results:
//   k_vel_cell   calculate_gforces + calculate_R_b + calculate_R_D2 + the
//                cell-average update of u,v,w                (in place)
//   k_vel_face   +xi face updates of u,v,w                    (cur -> next)
//                (k_vel_face_tile on large meshes: the same sweep with its
//                operands staged in shared memory by TMA boxes)
//   k_p_src      calculate_R_b_p + calculate_R_D_p2           (-> Rp, dila)
//   k_p_bc       apply_pressure_bc                            (cur -> next, walls)
//   k_p_bc_copy  new wall values into cur
//   k_p_face     integrate_pressure_field_i                   (cur -> next)
//   k_zero_flux  apply_zero_flux                              (in place, cur)
//   k_T_cell     calculate_temperature_nim_constants_formulation2 +
//                calculate_R_D_T + cell-average update of T   (in place)
//   k_T_face     +xi face updates of T                        (cur -> next)
//   k_iter_end   find_error's maxima -> convergence flag, iteration count
// Every sweep reads only values from before the sweep, so the result does not
// depend on thread order.
#pragma once
#include <cooperative_groups.h>
#include <cuda.h>  // CUtensorMap (the maps are encoded by the host)
#include <type_traits>

#include "nim_common.cuh"
#include "nim_exp.cuh"
#include "nim_dual.cuh"

namespace nim {

// Arithmetic type of a kernel over storage type R: double for the FP64
// path, float for the float mirror of the FP32 phase (whose kernels compute
// in float, with only the change maxima and reductions in double), DualD
// for the tangent-linear state (value and derivative).
template <class R>
struct ArithOf {
  using type = double;
};
template <>
struct ArithOf<float> {
  using type = float;
};
template <>
struct ArithOf<DualD> {
  using type = DualD;
};
template <class R>
using Ar = typename ArithOf<R>::type;

// ------------------------------------------------------------ device state
// Geometry and field arrays, by storage type R: double for the FP64 path;
// float for the mirror the mixed-precision inner loop sweeps (every array the
// parallel iteration reads or writes; its kernels compute in float, Ar<R>).
template <class R>
struct GeoT {
  R *vol;     // [Nc]
  R *G;       // [3][Nc]   G1, G2, G3
  R *gij;     // [9][Nc]   meshes_gij(a,b) at a-1+3(b-1)
  R *xi;      // [9][Nc]   meshes_xi_x(a,b) at a-1+3(b-1)
  R *gf;      // [54][Nc]  meshes_gij_faces(a,b,f) at a-1+3(b-1)+9(f-1)
  R *gfd;     // [6][Nc]   gf(d,d,2d-1), gf(d,d,2d) at 2(d-1)+{0,1}
  R *dg;      // [6][Nc]   gf(d,e,2d-1,i2)-gf(d,e,2d,i), e=tr1,tr2 at 2(d-1)+{0,1}
  R *area;    // [NF]
  R *normal;  // [3][NF]
  R *mid;     // [3][NF]
  R *tang;    // [3][NF]
  R *bitang;  // [3][NF]
  R *AA;      // [45][Nc]  AA_px/py/pz(k) at 15(d-1)+k-1
  int *bcpts;      // [5][NBF]  BCs_faces_points as structured face indices
  R *bca;     // [5][NBF]  BCs_faces_a(1:5)
  R *bcap;    // [8][NBF]  BCs_faces_ap(1:8)
  R *bcg;     // [2][NBF]  gij_faces factors of B2, B3 in apply_pressure_bc
  R *zf;      // [4][NBF]  zero-flux weights (B, C, D, A) for z walls
  R *nuw;     // [4][NBF]  find_Nu2 weights (A, B, C, D) for r walls
  R *bcval;   // [4][NBF]  Dirichlet face values of u, v, w, T
  R *rvol;    // [Nc]      1/vol, formed once at init in the storage type's own
              //           division (null in the dual copy, whose kernels divide)
};
using Geo = GeoT<double>;

template <class R>
struct FieldsT {
  R *f[5];    // faces u, v, w, p, T: each [2][NF]
  R *c[4];    // cells u, v, w, T (meshes_*xyz)
  R *co[4];   // meshes_*xyz_old
  R *ct[4];   // meshes_*xyzt
  R *mp, *dila, *dila_old, *Rp;
  R *MA;      // [18][Nc] velocity M_A (per step scratch)
  R *MF4;     // [8][Nc]
  R *MF;      // [15][Nc]  M_F1..3(k) at 5(d-1)+k-1
  R *MTF;     // [15][Nc]  MT_F1..3
  R *MTA;     // [18][Nc]  MT_A(q, d) at 3(q-1) + d-1 (float: 1/MT_A(5, d) at q = 5)
  R *dpd;     // [3][Nc]   dpdx_old, dpdy_old, dpdz_old
  // reference-order schedule: sources stored before the ordered sweeps
  R *Bv;      // [3][Nc]   R_C + R_D + R_B of u, v, w
  R *MTF4;    // [8][Nc]   MT_F4
  R *RDT;     // [Nc]      R_D_T
  // formulation 1 (nim_formulation = 1)
  R *N1;      // [22][Nc]  CC, EE, FF, GG, HH, II, JJ (3 each), Det (per step)
  R *AT;      // [9][Nc]   a_t
  R *AAv;     // [45][Nc]  AA_vx, AA_vy, AA_vz (15 each)
  double *part;  // [8][nblk] per-block partial sums (FP64 always)
};
using Fields = FieldsT<double>;

struct Phys {
  double DT, nu, alpha, rho, g_beta;
  double w[4];     // u, v, w, T relaxation
  double w_p, w_p2;
  double tol[5];
  double v_limit, dudt_epsilon, R_i, R_o;
  double inv_Re;   // 1/Re with Re = 1/nu (parameters.f90:172, nse.f90:1852)
  double inv_rho;  // 1/rho
  int max_iters, dpdx_tolerance;
  int formulation; // nim_formulation: 1 or 2
  // derivatives of nu, alpha and 1/Re along the seeded direction: read only
  // by the dual instantiations (nim_gpu_tangent_*), zero otherwise
  double d_nu, d_alpha, d_inv_Re;
};
// a parameter as the arithmetic type V sees it: its value, and in the dual
// instantiations its seeded derivative
template <class V>
struct ParOf {
  __device__ __forceinline__ static V get(double v, double) { return V(v); }
};
template <>
struct ParOf<DualD> {
  __device__ __forceinline__ static DualD get(double v, double t) { return DualD(v, t); }
};
template <class V>
__device__ __forceinline__ V pv(double v, double t) {
  return ParOf<V>::get(v, t);
}
// 1/vol of cell c: the stored reciprocal (the same IEEE division in the
// storage type, formed once at init), or the division itself for the dual
// copy
template <class R>
__device__ __forceinline__ Ar<R> inv_vol(const GeoT<R> &g, int c) {
  if constexpr (std::is_same<R, double>::value || std::is_same<R, float>::value)
    return g.rvol[c];
  else
    return Ar<R>(1.) / g.vol[c];
}

// Control block in device memory; k_iter_end is its only writer during an
// iteration, the host reads it between batches.
struct Ctrl {
  unsigned long long err[2][8];  // max-accumulators per parity: u,v,w,p,T,dpdx
  unsigned long long wall_floor[8];  // max |Dirichlet wall value| bits (find_error
                                     // compares with zero-initialised arrays once);
                                     // with err: the 24 words z-slabs max-reduce
  int iter;         // iterations since init (parity source)
  int step_iters;   // iterations of the current step (cnt)
  int done;         // 1: current step's inner loop has stopped
  int status;       // NIM_OK / NIM_ERR_NOT_CONVERGED / NIM_ERR_NONFINITE
  int first;        // 1 until the first iteration after init has finished
  int pmask;        // 1: face arrays alternate halves each pass (parallel
                    // schedule); 0: one half, updated in place (reference order)
  int pad[2];
  double last_err[5];
  unsigned long long red[4];  // dudt, dTdt maxima (after integrate)
  double dilatation, nu_outer, nu_inner, area_outer, area_inner;
  // FP32 phase of a mixed-precision step: passes run, the smallest maximum
  // change seen per field, passes since a field still above its tolerance
  // last reached a new smallest change
  int lowp_iters, stall;
  double best[5];
};

// FP32 passes without progress after which a mixed-precision step hands over
// to FP64 (the FP32 iterate has reached its rounding floor)
constexpr int kLowpStall = 8;

constexpr int BLK = 256;
constexpr int VC2_MINB = 3;  // resident blocks per SM asked of k_vel_cell2 (56 registers)
// resident blocks per SM the float instantiations of the pass kernels ask
// for: computing in float they need about half the FP64 registers
constexpr int VC2_MINB_F = 3, PSRC_MINB_F = 4, PFACE_MINB_F = 5, TCELL_MINB_F = 5, TFACE_MINB_F = 4;
constexpr int VCN_MINB = 2;  // k_vel_cellN (four float cells a thread)
constexpr int PSN_MINB = 2;  // k_p_srcN (four float or two FP64 cells a thread)
constexpr int TCN_MINB = 2;  // k_T_cellN (four float cells a thread)
constexpr int PFN_MINB = 2;  // k_p_faceN (four float or two FP64 faces a thread)
constexpr int TFN_MINB = 2;  // k_T_faceN (four float faces a thread)
constexpr int VFN_MINB = 2;  // k_vel_faceN (four float faces a thread)
template <class R>
constexpr int minb(int fp64, int fp32) {
  return sizeof(R) == 8 ? fp64 : fp32;
}
// kernels that spread one cell over three threads (component or direction)
constexpr int CB = 128;            // cells per block
constexpr int CB3 = 3 * CB;        // threads per block

// ------------------------------------------------------------ reductions
// Max of non-negative doubles through their bit patterns (IEEE order equals
// integer order for x >= 0; NaN sorts above +Inf and is caught as non-finite).
// NT = threads in the block (flattened).  Call red_init() first (it holds
// the only barrier); block_max() is barrier-free: warps fold their maxima
// into shared memory with atomics and the last warp to finish publishes the
// block's maxima with one global atomic each.
struct BlockRed {
  unsigned long long m[8];
  unsigned int count;
};
template <int N>
__device__ __forceinline__ void red_init(BlockRed &r) {
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    for (int n = 0; n < N; ++n) r.m[n] = 0ull;
    r.count = 0u;
  }
  __syncthreads();
}
template <int N, int NT = BLK>
__device__ __forceinline__ void block_max(BlockRed &r, const double (&v)[N], unsigned long long *dst) {
  const int t = threadIdx.x + blockDim.x * threadIdx.y;
  const int lane = t & 31;
  unsigned long long b[N];
#pragma unroll
  for (int n = 0; n < N; ++n) {
    b[n] = (unsigned long long)__double_as_longlong(v[n]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long u = __shfl_xor_sync(0xffffffffu, b[n], o);
      b[n] = (u > b[n]) ? u : b[n];
    }
  }
  if (lane == 0) {
#pragma unroll
    for (int n = 0; n < N; ++n)
      if (b[n]) atomicMax(&r.m[n], b[n]);
    __threadfence_block();
    const unsigned int done = atomicAdd(&r.count, 1u);
    if (done == NT / 32 - 1) {
      __threadfence_block();
#pragma unroll
      for (int n = 0; n < N; ++n) {
        const unsigned long long m = atomicAdd(&r.m[n], 0ull);
        if (m) atomicMax(dst + n, m);
      }
    }
  }
}

// Deterministic block sums written to part[n][blockIdx.x].
template <int N>
__device__ __forceinline__ void block_sum(const double (&v)[N], double *part, int nblk) {
  __shared__ double sm[N][BLK];
#pragma unroll
  for (int n = 0; n < N; ++n) sm[n][threadIdx.x] = v[n];
  __syncthreads();
  for (int s = BLK / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
#pragma unroll
      for (int n = 0; n < N; ++n) sm[n][threadIdx.x] = sm[n][threadIdx.x] + sm[n][threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
#pragma unroll
    for (int n = 0; n < N; ++n) part[(size_t)n * nblk + blockIdx.x] = sm[n][0];
  }
}

// ================================================================ init
__device__ __forceinline__ int node_index(const Dims &d, int i, int j, int k) {
  return i + d.NT * (j + (d.NR + 1) * k);
}

// mesh_calculate_mapping_coefficients (create_mesh.f90:254-303) from the
// arranged nodes 1..8 of the cell (create_mesh.f90:326-333 drawing).
__device__ void cell_map(const Dims &d, const double *__restrict__ nx, const Cell &x, Map &M) {
  const int ip = (x.i == d.NT - 1) ? 0 : x.i + 1;
  int nd[9];
  nd[1] = node_index(d, x.i, x.j, x.k);
  nd[2] = node_index(d, x.i, x.j + 1, x.k);
  nd[3] = node_index(d, ip, x.j + 1, x.k);
  nd[4] = node_index(d, ip, x.j, x.k);
  nd[5] = node_index(d, x.i, x.j, x.k + 1);
  nd[6] = node_index(d, x.i, x.j + 1, x.k + 1);
  nd[7] = node_index(d, ip, x.j + 1, x.k + 1);
  nd[8] = node_index(d, ip, x.j, x.k + 1);
  for (int comp = 0; comp < 3; ++comp) {
    double v[9];
    for (int n = 1; n <= 8; ++n) v[n] = nx[3 * (size_t)nd[n] + comp];
    double *C = (comp == 0) ? M.C : (comp == 1) ? M.D : M.E;
    C[0] = (v[7] + v[8] + v[5] + v[6] + v[3] + v[4] + v[1] + v[2]) / 8.;
    C[1] = (v[7] - v[8] - v[5] + v[6] + v[3] - v[4] - v[1] + v[2]) / 8.;
    C[2] = (v[7] + v[8] - v[5] - v[6] + v[3] + v[4] - v[1] - v[2]) / 8.;
    C[3] = (v[7] + v[8] + v[5] + v[6] - v[3] - v[4] - v[1] - v[2]) / 8.;
    C[4] = (v[7] - v[8] + v[5] - v[6] + v[3] - v[4] + v[1] - v[2]) / 8.;
    C[5] = (v[7] - v[8] - v[5] + v[6] - v[3] + v[4] + v[1] - v[2]) / 8.;
    C[6] = (v[7] + v[8] - v[5] - v[6] - v[3] - v[4] + v[1] + v[2]) / 8.;
    C[7] = (v[7] - v[8] + v[5] - v[6] - v[3] + v[4] - v[1] + v[2]) / 8.;
  }
}

// Does this cell hold the final (highest cell number) write of its face pos?
// The reference writes shared-face geometry from both cells in cell-number
// order (geometry.f90:100-189, 468-496), so the later cell wins.
__device__ __forceinline__ bool owns_face(const Dims &d, const Cell &x, int pos) {
  switch (pos) {
    case 1: return true;
    case 2: return x.j == d.NR - 1;
    case 3: return x.i > 0;
    case 4: return x.i == d.NT - 1;
    case 5: return true;
    default: return x.k == d.NZ - 1;
  }
}

// evaluate_all_mesh_constants for one cell (geometry.f90:14-32):
// volume_calculate (create_mesh.f90:306-322), find_normal (geometry.f90:
// 76-190), calculate_defusion_tensor_over_faces (geometry.f90:395-497, the 25
// points per face that Gauss_integration2d_face keeps) and
// convection_diffusion_constants_mesh_i (geometry.f90:500-632).  The volume
// and the volume-averaged metrics share their 125 Gauss points.
__global__ void __launch_bounds__(BLK) k_cell_geometry(Dims d, GaussRule gq, const double *__restrict__ nx, Geo g) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.Nc) return;
  const Cell x = Cell::of(d, c);
  Map M;
  cell_map(d, nx, x, M);
  const size_t Nc = d.Nc, NF = d.NF;
  Curvi C;
  {
    double V = 0., sG[3] = {0., 0., 0.}, sK[9], sJ[9];
    for (int n = 0; n < 9; ++n) sK[n] = sJ[n] = 0.;
    for (int i = 0; i < 5; ++i)
      for (int j = 0; j < 5; ++j)
        for (int k = 0; k < 5; ++k) {
          curvi_point(M, gq.x[i], gq.x[j], gq.x[k], C);
          const double w = gq.w[i] * gq.w[j] * gq.w[k];
          V = V + w * (1. * C.detJ);
          // gamma_tensor (curvilinear.f90:109-160) contracted with g^ij
          const double g12[3] = {M.C[4] + M.C[7] * gq.x[k], M.D[4] + M.D[7] * gq.x[k], M.E[4] + M.E[7] * gq.x[k]};
          const double g13[3] = {M.C[5] + M.C[7] * gq.x[j], M.D[5] + M.D[7] * gq.x[j], M.E[5] + M.E[7] * gq.x[j]};
          const double g23[3] = {M.C[6] + M.C[7] * gq.x[i], M.D[6] + M.D[7] * gq.x[i], M.E[6] + M.E[7] * gq.x[i]};
          double gu[3][3];  // gu[a][comp] = g^a
          for (int a = 0; a < 3; ++a)
            for (int cc = 0; cc < 3; ++cc) gu[a][cc] = C.jacinv[cc][a];
          double G[3][3];
          for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) G[a][b] = dot3(gu[a], gu[b]);
          for (int a = 0; a < 3; ++a) {
            const double a12 = dot3(gu[a], g12), a13 = dot3(gu[a], g13), a23 = dot3(gu[a], g23);
            const double Ga = (a12 * G[0][1] + a12 * G[1][0] + a13 * G[0][2] + a13 * G[2][0] + a23 * G[1][2] +
                               a23 * G[2][1]);
            sG[a] = sG[a] + w * (Ga * C.detJ);
          }
          for (int r = 0; r < 3; ++r)
            for (int cc = 0; cc < 3; ++cc) {
              sK[r + 3 * cc] = sK[r + 3 * cc] + w * (G[r][cc] * C.detJ);
              sJ[r + 3 * cc] = sJ[r + 3 * cc] + w * (C.jacinv[r][cc] * C.detJ);
            }
        }
    g.vol[c] = V;
    for (int a = 0; a < 3; ++a) g.G[a * Nc + c] = sG[a] / V;
    for (int r = 0; r < 3; ++r)
      for (int cc = 0; cc < 3; ++cc) {
        g.gij[(r + 3 * cc) * Nc + c] = sK[r + 3 * cc] / V;
        g.xi[(cc + 3 * r) * Nc + c] = sJ[r + 3 * cc] / V;  // xi_x(a,b) = <jacinv(b,a)>
      }
  }
  // find_normal: contravariant unit normal, covariant unit tangents, centre
  for (int fn = 1; fn <= 6; ++fn) {
    if (!owns_face(d, x, fn)) continue;
    double px, py, pz;
    face_point(fn, 0.0, 0.0, px, py, pz);
    curvi_point(M, px, py, pz, C);
    const int dd = (fn - 1) / 2, t1 = (dd == 0) ? 1 : 0, t2 = (dd == 2) ? 1 : 2;
    const int f = x.face(d, fn);
    const double sn = sqrt(gup(C, dd, dd)), s1 = sqrt(glow(C, t1, t1)), s2 = sqrt(glow(C, t2, t2));
    for (int cc = 0; cc < 3; ++cc) {
      g.normal[cc * NF + f] = C.jacinv[cc][dd] / sn;
      g.tang[cc * NF + f] = C.jac[t1][cc] / s1;
      g.bitang[cc * NF + f] = C.jac[t2][cc] / s2;
    }
    g.mid[0 * NF + f] = C.x;
    g.mid[1 * NF + f] = C.y;
    g.mid[2 * NF + f] = C.z;
  }
  // face-averaged metric and face areas
  for (int fn = 1; fn <= 6; ++fn) {
    const int dd = (fn - 1) / 2;
    double A = 0., K[9];
    for (int n = 0; n < 9; ++n) K[n] = 0.;
    for (int a = 0; a < 5; ++a)
      for (int b = 0; b < 5; ++b) {
        double px, py, pz;
        face_point(fn, gq.x[a], gq.x[b], px, py, pz);
        curvi_point(M, px, py, pz, C);
        const double w = gq.w[a] * gq.w[b];
        const double dS = C.detJ * sqrt(gup(C, dd, dd));
        A = A + w * dS;
        for (int r = 0; r < 3; ++r) {
          const double srr = sqrt(gup(C, r, r));
          for (int cc = 0; cc < 3; ++cc) K[r + 3 * cc] = K[r + 3 * cc] + w * (gup(C, r, cc) / srr * dS);
        }
      }
    if (owns_face(d, x, fn)) g.area[x.face(d, fn)] = A;
    for (int n = 0; n < 9; ++n) g.gf[(n + 9 * (fn - 1)) * Nc + c] = K[n] / A;
  }
}

// 1/vol per cell, once at init: the sweeps' Green-Gauss factor (1/V of
// nse.f90:2866-2903) read instead of divided on every pass; the same IEEE
// division, so the same bits
template <class R>
__global__ void __launch_bounds__(BLK) k_reciprocal(const R *__restrict__ v, R *__restrict__ r, int n) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < n) r[c] = R(1) / v[c];
}

// Compact per-cell copies of the metric entries the sweeps read: the
// diagonal face metric (M_A) and the differences of off-diagonal face metric
// across each +xi face (the B3/B4 terms, nse.f90:882-885 and alike).
__global__ void __launch_bounds__(BLK) k_metric_derived(Dims d, Geo g) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.Nc) return;
  const Cell x = Cell::of(d, c);
  const size_t Nc = d.Nc;
  auto gfa = [&](int a, int b, int f, int cell) { return g.gf[(size_t)(a - 1 + 3 * (b - 1) + 9 * (f - 1)) * Nc + cell]; };
  for (int dd = 1; dd <= 3; ++dd) {
    g.gfd[(2 * (dd - 1) + 0) * Nc + c] = gfa(dd, dd, 2 * dd - 1, c);
    g.gfd[(2 * (dd - 1) + 1) * Nc + c] = gfa(dd, dd, 2 * dd, c);
    double v0 = 0., v1 = 0.;
    if (x.has_nb(d, 2 * dd)) {
      const int i2 = x.nb(d, 2 * dd).c;
      v0 = gfa(dd, tr1(dd), 2 * dd - 1, i2) - gfa(dd, tr1(dd), 2 * dd, c);
      v1 = gfa(dd, tr2(dd), 2 * dd - 1, i2) - gfa(dd, tr2(dd), 2 * dd, c);
    }
    g.dg[(2 * (dd - 1) + 0) * Nc + c] = v0;
    g.dg[(2 * (dd - 1) + 1) * Nc + c] = v1;
  }
}

// Zero-velocity NIM constants of calculate_pressure_nim_constants
// (nim.f90:567-612): C_nim..J_nim in their series branch at u = 0.
struct PConst {
  double CC[3], EE[3], FF[3], GG[3], HH[3], II[3], JJ[3], Det;
};
__device__ __forceinline__ PConst pconst(const Geo &g, size_t Nc, int c, double rho) {
  PConst p;
  const double a = 1.;
  for (int dd = 0; dd < 3; ++dd) {
    const double Fk = g.gij[(size_t)(dd + 3 * dd) * Nc + c] / rho;
    p.CC[dd] = -(a * a / (3. * Fk));
    p.GG[dd] = 1 / (2. * a);
    p.HH[dd] = a / Fk;
    p.II[dd] = 1 / (2. * a);
    p.JJ[dd] = -(a / Fk);
  }
  p.Det = 1. / (p.CC[0] * p.CC[1] + p.CC[1] * p.CC[2] + p.CC[0] * p.CC[2]);
  for (int dd = 0; dd < 3; ++dd) {
    p.EE[dd] = p.Det / 2.;
    p.FF[dd] = p.Det / 2.;
  }
  return p;
}

// AA_px/py/pz (nim.f90:616-678)
__global__ void __launch_bounds__(BLK) k_pressure_coeffs(Dims d, Geo g, double rho) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.Nc) return;
  const Cell x = Cell::of(d, c);
  const size_t Nc = d.Nc;
  const PConst P = pconst(g, Nc, c, rho);
  auto gfa = [&](int a, int b, int f, int cell) { return g.gf[(size_t)(a - 1 + 3 * (b - 1) + 9 * (f - 1)) * Nc + cell]; };
  double A[15];
  // +r face
  for (int n = 0; n < 15; ++n) A[n] = 0.;
  if (x.has_nb(d, 2)) {
    const int i2 = x.nb(d, 2).c;
    const PConst Q = pconst(g, Nc, i2, rho);
    const double gg = gfa(1, 1, 2, c), g2 = gfa(1, 1, 1, i2);
    A[0] = -(P.GG[0] + (P.CC[1] + P.CC[2]) * P.EE[0] * P.HH[0]) * gg;
    A[1] = (P.GG[0] - (P.CC[1] + P.CC[2]) * P.FF[0] * P.HH[0]) * gg + (Q.II[0] + (Q.CC[1] + Q.CC[2]) * Q.EE[0] * Q.JJ[0]) * g2;
    A[2] = -(Q.II[0] - (Q.CC[1] + Q.CC[2]) * Q.FF[0] * Q.JJ[0]) * g2;
    A[3] = P.CC[2] * P.EE[1] * P.HH[0] * gg;
    A[4] = P.CC[2] * P.FF[1] * P.HH[0] * gg;
    A[5] = -(Q.CC[2] * Q.EE[1] * Q.JJ[0] * g2);
    A[6] = -(Q.CC[2] * Q.FF[1] * Q.JJ[0] * g2);
    A[7] = P.CC[1] * P.EE[2] * P.HH[0] * gg;
    A[8] = P.CC[1] * P.FF[2] * P.HH[0] * gg;
    A[9] = -(Q.CC[1] * Q.EE[2] * Q.JJ[0] * g2);
    A[10] = -(Q.CC[1] * Q.FF[2] * Q.JJ[0] * g2);
    A[11] = P.CC[1] * P.CC[2] * P.Det * P.HH[0] * gg;
    A[12] = -(P.CC[1] * P.CC[2] * P.Det * P.HH[0] * gg);
    A[13] = -(Q.CC[1] * Q.CC[2] * Q.Det * Q.JJ[0] * g2);
    A[14] = Q.CC[1] * Q.CC[2] * Q.Det * Q.JJ[0] * g2;
  }
  for (int n = 0; n < 15; ++n) g.AA[(size_t)n * Nc + c] = A[n];
  // +theta face
  {
    const int i2 = x.nb(d, 4).c;
    const PConst Q = pconst(g, Nc, i2, rho);
    const double gg = gfa(2, 2, 4, c), g2 = gfa(2, 2, 3, i2);
    A[0] = P.CC[2] * P.EE[0] * P.HH[1] * gg;
    A[1] = P.CC[2] * P.FF[0] * P.HH[1] * gg;
    A[2] = -(Q.CC[2] * Q.EE[0] * Q.JJ[1] * g2);
    A[3] = -(Q.CC[2] * Q.FF[0] * Q.JJ[1] * g2);
    A[4] = -(P.GG[1] + (P.CC[0] + P.CC[2]) * P.EE[1] * P.HH[1]) * gg;
    A[5] = (P.GG[1] - (P.CC[0] + P.CC[2]) * P.FF[1] * P.HH[1]) * gg + (Q.II[1] + (Q.CC[0] + Q.CC[2]) * Q.EE[1] * Q.JJ[1]) * g2;
    A[6] = -(Q.II[1] - (Q.CC[0] + Q.CC[2]) * Q.FF[1] * Q.JJ[1]) * g2;
    A[7] = P.CC[0] * P.EE[2] * P.HH[1] * gg;
    A[8] = P.CC[0] * P.FF[2] * P.HH[1] * gg;
    A[9] = -(Q.CC[0] * Q.EE[2] * Q.JJ[1] * g2);
    A[10] = -(Q.CC[0] * Q.FF[2] * Q.JJ[1] * g2);
    A[11] = P.CC[0] * P.CC[2] * P.Det * P.HH[1] * gg;
    A[12] = -(P.CC[0] * P.CC[2] * P.Det * P.HH[1] * gg);
    A[13] = -(Q.CC[0] * Q.CC[2] * Q.Det * Q.JJ[1] * g2);
    A[14] = Q.CC[0] * Q.CC[2] * Q.Det * Q.JJ[1] * g2;
  }
  for (int n = 0; n < 15; ++n) g.AA[(size_t)(15 + n) * Nc + c] = A[n];
  // +z face
  for (int n = 0; n < 15; ++n) A[n] = 0.;
  if (x.has_nb(d, 6)) {
    const int i2 = x.nb(d, 6).c;
    const PConst Q = pconst(g, Nc, i2, rho);
    const double gg = gfa(3, 3, 6, c), g2 = gfa(3, 3, 5, i2);
    A[0] = P.CC[1] * P.EE[0] * P.HH[2] * gg;
    A[1] = P.CC[1] * P.FF[0] * P.HH[2] * gg;
    A[2] = -(Q.CC[1] * Q.EE[0] * Q.JJ[2] * g2);
    A[3] = -(Q.CC[1] * Q.FF[0] * Q.JJ[2] * g2);
    A[4] = P.CC[0] * P.EE[1] * P.HH[2] * gg;
    A[5] = P.CC[0] * P.FF[1] * P.HH[2] * gg;
    A[6] = -(Q.CC[0] * Q.EE[1] * Q.JJ[2] * g2);
    A[7] = -(Q.CC[0] * Q.FF[1] * Q.JJ[2] * g2);
    A[8] = -(P.GG[2] + (P.CC[0] + P.CC[1]) * P.EE[2] * P.HH[2]) * gg;
    A[9] = (P.GG[2] - (P.CC[0] + P.CC[1]) * P.FF[2] * P.HH[2]) * gg + (Q.II[2] + (Q.CC[0] + Q.CC[1]) * Q.EE[2] * Q.JJ[2]) * g2;
    A[10] = -(Q.II[2] - (Q.CC[0] + Q.CC[1]) * Q.FF[2] * Q.JJ[2]) * g2;
    A[11] = P.CC[0] * P.CC[1] * P.Det * P.HH[2] * gg;
    A[12] = -(P.CC[0] * P.CC[1] * P.Det * P.HH[2] * gg);
    A[13] = -(Q.CC[0] * Q.CC[1] * Q.Det * Q.JJ[2] * g2);
    A[14] = Q.CC[0] * Q.CC[1] * Q.Det * Q.JJ[2] * g2;
  }
  for (int n = 0; n < 15; ++n) g.AA[(size_t)(30 + n) * Nc + c] = A[n];
}

// Boundary-face constants, one thread per wall face b (reference BC order):
// evaluate_pressure_bc_array (geometry.f90:879-975), BCs_faces_ap
// (nim.f90:682-742), apply_dirichlet_bc_i face averages (bc.f90:59-88) and
// the distance weights of apply_zero_flux (bc.f90:355-384) and find_Nu2
// (nse.f90:2721-2764).
__global__ void __launch_bounds__(BLK) k_bc_geometry(Dims d, GaussRule gq, const double *__restrict__ nx, Geo g,
                                                     double rho, const double *__restrict__ bcv /* [5][5] */) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= d.NBF) return;
  const size_t Nc = d.Nc, NF = d.NF, NB = d.NBF;
  const BFace B = bface(d, b);
  const Cell M1 = B.cell;
  const int pos = B.pos;
  const int f0 = M1.face(d, pos);
  // ---- 5-point normal stencil
  const int fn = (pos % 2 == 1) ? pos + 1 : pos - 1;
  const Cell M2 = M1.nb(d, fn);
  const int t1a = (pos <= 2) ? 4 : 2, t1b = (pos <= 2) ? 3 : 1;
  const int t2a = (pos <= 4) ? 6 : 4, t2b = (pos <= 4) ? 5 : 3;
  const Cell M3 = M1.has_nb(d, t1a) ? M1.nb(d, t1a) : M1.nb(d, t1b);
  const Cell M4 = M1.has_nb(d, t2a) ? M1.nb(d, t2a) : M1.nb(d, t2b);
  int pts[6];
  pts[1] = f0;
  pts[2] = M1.face(d, fn);
  pts[3] = M2.face(d, fn);
  pts[4] = M3.face(d, fn);
  pts[5] = M4.face(d, fn);
  for (int j = 1; j <= 5; ++j) g.bcpts[(j - 1) * NB + b] = pts[j];
  double n[6], t[6], s[6];
  const double nv[3] = {g.normal[f0], g.normal[NF + f0], g.normal[2 * NF + f0]};
  const double tv[3] = {g.tang[f0], g.tang[NF + f0], g.tang[2 * NF + f0]};
  const double sv[3] = {g.bitang[f0], g.bitang[NF + f0], g.bitang[2 * NF + f0]};
  for (int j = 1; j <= 5; ++j) {
    double dv[3];
    for (int cc = 0; cc < 3; ++cc) dv[cc] = g.mid[cc * NF + pts[j]] - g.mid[cc * NF + pts[1]];
    n[j] = dot3(dv, nv);
    t[j] = dot3(dv, tv);
    s[j] = dot3(dv, sv);
  }
  const double D =
      (n[3] * s[4] * t[2] - n[3] * s[5] * t[2] - n[2] * s[4] * t[3] + n[2] * s[5] * t[3] - n[3] * s[2] * t[4] +
       n[2] * s[3] * t[4] - n[2] * s[5] * t[4] + n[3] * s[5] * t[4] + n[5] * s[3] * t[2] - n[5] * s[4] * t[2] -
       n[5] * s[2] * t[3] + n[5] * s[4] * t[3] + n[5] * s[2] * t[4] - n[5] * s[3] * t[4] + n[3] * s[2] * t[5] -
       n[2] * s[3] * t[5] + n[2] * s[4] * t[5] - n[3] * s[4] * t[5] +
       n[4] * (s[5] * t[2] + s[2] * t[3] - s[5] * t[3] - s[2] * t[5] + s[3] * (-t[2] + t[5])));
  double a[6];
  a[2] = 2 * (-(n[5] * s[4] * t[3]) + n[4] * s[5] * t[3] + n[5] * s[3] * t[4] - n[3] * s[5] * t[4] -
              n[4] * s[3] * t[5] + n[3] * s[4] * t[5]) / ((n[2] * n[2]) * D);
  a[3] = 2 * (n[5] * s[4] * t[2] - n[4] * s[5] * t[2] - n[5] * s[2] * t[4] + n[2] * s[5] * t[4] +
              n[4] * s[2] * t[5] - n[2] * s[4] * t[5]) / ((n[3] * n[3]) * D);
  a[4] = 2 * (n[5] * s[3] * t[2] - n[3] * s[5] * t[2] - n[5] * s[2] * t[3] + n[2] * s[5] * t[3] +
              n[3] * s[2] * t[5] - n[2] * s[3] * t[5]) / ((n[4] * n[4]) * D);
  a[5] = 2 * (n[4] * s[3] * t[2] - n[3] * s[4] * t[2] - n[4] * s[2] * t[3] + n[2] * s[4] * t[3] +
              n[3] * s[2] * t[4] - n[2] * s[3] * t[4]) / ((n[5] * n[5]) * D);
  a[1] = -a[2] - a[3] - a[4] - a[5];
  for (int k = 1; k <= 5; ++k) g.bca[(k - 1) * NB + b] = a[k];

  // ---- BCs_faces_ap
  auto gfa = [&](int aa, int bb, int f, int cell) { return g.gf[(size_t)(aa - 1 + 3 * (bb - 1) + 9 * (f - 1)) * Nc + cell]; };
  const PConst P = pconst(g, Nc, M1.c, rho);
  {
    const int dd = (pos + 1) / 2, e1 = tr1(dd), e2 = tr2(dd);
    const bool minus = (pos % 2 == 1);
    const double gg = gfa(dd, dd, pos, M1.c);
    const double P0 = minus ? P.II[dd - 1] : P.GG[dd - 1];
    const double Q = minus ? P.JJ[dd - 1] : P.HH[dd - 1];
    const double cs = P.CC[e1 - 1] + P.CC[e2 - 1];
    double ap[8];
    ap[2 * dd - 2] = -(P0 + cs * P.EE[dd - 1] * Q) * gg;
    ap[2 * dd - 1] = (P0 - cs * P.FF[dd - 1] * Q) * gg;
    ap[2 * e1 - 2] = P.CC[e2 - 1] * P.EE[e1 - 1] * Q * gg;
    ap[2 * e1 - 1] = P.CC[e2 - 1] * P.FF[e1 - 1] * Q * gg;
    ap[2 * e2 - 2] = P.CC[e1 - 1] * P.EE[e2 - 1] * Q * gg;
    ap[2 * e2 - 1] = P.CC[e1 - 1] * P.FF[e2 - 1] * Q * gg;
    ap[6] = P.CC[e1 - 1] * P.CC[e2 - 1] * P.Det * Q * gg;
    ap[7] = -(P.CC[e1 - 1] * P.CC[e2 - 1] * P.Det * Q * gg);
    for (int k = 0; k < 8; ++k) g.bcap[k * NB + b] = ap[k];
    // gij_faces factors of B2 / B3; position 6 takes (3,2) in the centred
    // branch of B2 (bc.f90:318)
    const bool centred = M1.has_nb(d, 2 * e1 - 1) && M1.has_nb(d, 2 * e1);
    const int e1g = (pos == 6 && centred) ? 2 : e1;
    g.bcg[0 * NB + b] = gfa(dd, e1g, pos, M1.c);
    g.bcg[1 * NB + b] = gfa(dd, e2, pos, M1.c);
  }
  // ---- Dirichlet face values (u, v, w, T) of this BC id
  {
    Map M;
    cell_map(d, nx, M1, M);
    const int dd = (pos - 1) / 2;
    double dS[25];
    Curvi C;
    for (int i = 0; i < 5; ++i)
      for (int j = 0; j < 5; ++j) {
        double px, py, pz;
        face_point(pos, gq.x[i], gq.x[j], px, py, pz);
        curvi_point(M, px, py, pz, C);
        dS[5 * i + j] = C.detJ * sqrt(gup(C, dd, dd));
      }
    const int fld[4] = {0, 1, 2, 4};
    for (int q = 0; q < 4; ++q) {
      const double cv = bcv[fld[q] * 5 + (B.id - 1)];
      double Int = 0.;
      for (int i = 0; i < 5; ++i)
        for (int j = 0; j < 5; ++j) Int = Int + gq.w[i] * gq.w[j] * (cv * dS[5 * i + j]);
      g.bcval[q * NB + b] = Int / g.area[f0];
    }
  }
  // ---- distance weights along the wall-normal chain of faces
  {
    const int in = (pos % 2 == 1) ? pos + 1 : pos - 1;  // faces on the far side
    const Cell c2 = M1.nb(d, in), c3 = c2.nb(d, in);
    const int f1 = f0, f2 = M1.face(d, in), f3 = c2.face(d, in), f4 = c3.face(d, in);
    auto dist = [&](int p, int q) {
      const double dx = g.mid[p] - g.mid[q], dy = g.mid[NF + p] - g.mid[NF + q], dz = g.mid[2 * NF + p] - g.mid[2 * NF + q];
      return sqrt(dx * dx + dy * dy + dz * dz);
    };
    const double h1 = dist(f1, f2), h2 = dist(f2, f3), h3 = dist(f3, f4);
    const double wA = (1. / h1 + 1. / (h1 + h2) + 1. / (h1 + h2 + h3));
    const double wB = ((h1 + h2) * (h1 + h2 + h3)) / (h1 * h2 * (h2 + h3));
    const double wC = (h1 * (h1 + h2 + h3)) / (h2 * h3 * (h1 + h2));
    const double wD = (h1 * (h1 + h2)) / (h3 * (h2 + h3) * (h1 + h2 + h3));
    double *dst = (pos >= 5) ? g.zf : g.nuw;
    dst[0 * NB + b] = wA;
    dst[1 * NB + b] = wB;
    dst[2 * NB + b] = wC;
    dst[3 * NB + b] = wD;
  }
}

// Dirichlet values into both halves of the u, v, w, T face arrays
// (apply_all_dirichlet_bcs, bc.f90:13-57).
__global__ void k_apply_dirichlet(Dims d, Geo g, Fields F) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= d.NBF) return;
  const BFace B = bface(d, b);
  const int f = B.cell.face(d, B.pos);
  const int fld[4] = {0, 1, 2, 4};
  for (int q = 0; q < 4; ++q) {
    const double v = g.bcval[q * (size_t)d.NBF + b];
    F.f[fld[q]][f] = v;
    F.f[fld[q]][d.NF + f] = v;
  }
}

// ============================================================= per step
// NIM coefficients of one direction for contravariant speed u and
// diffusivity k: M_A(d,1:6) / MT_A(d,1:6) (nim.f90:181-287, 354-460).
template <class V>
__device__ __forceinline__ void nim_direction(V u, V k, V gminus, V gplus, double v_limit, V A[6]) {
  const V a = V(1.);
  const V Re = 2 * a * u / k;
  if (fabs(Re) > v_limit) {
    const V e = nim_exp(Re);
    A[0] = (2 * a / (k * (V(1.) / e - V(1.))) + V(1.) / u) * gplus;
    A[1] = (-(2 * a / (k * (V(1.) - e))) - V(1.) / u) * gminus;
    A[2] = (u / (k * (V(1.) / e - V(1.)))) * gplus;
    A[3] = (u / (k * (V(1.) - e))) * gminus;
    if (Re > 0) {
      A[4] = (-k + (a * u * (V(1.) / e + V(1.)) / (-(V(1.) / e) + V(1.)))) / (u * u);
      A[5] = V(1.) / (-(V(1.) / e) + V(1.)) - V(1.) / (Re);
    } else {
      A[4] = (-k + (a * u * (V(1.) + e) / (-V(1.) + e))) / (u * u);
      A[5] = e / (-V(1.) + e) - V(1.) / (Re);
    }
  } else {
    const PwT<V> U(u), K(k);
    A[0] = (-(a / k) - (u) / (V(3.) * K[2]) + (U[3]) / (V(45.) * K[4]) - (2 * U[5]) / (V(945.) * K[6]) +
            -((U[7]) / (V(4725.) * K[8])) - (2 * U[9]) / (V(93555.) * K[10])) * gplus;
    A[1] = (-(a / k) + (u) / (V(3.) * K[2]) - (U[3]) / (V(45.) * K[4]) + (2 * U[5]) / (V(945.) * K[6]) -
            -((U[7]) / (V(4725.) * K[8])) + (2 * U[9]) / (V(93555.) * K[10])) * gminus;
    A[2] = (-(1 / (V(2.) * a)) - u / (V(2.) * k) - (U[2]) / (V(6.) * K[2]) + (U[4]) / (V(90.) * K[4]) -
            -((U[6]) / (V(945.) * K[6])) + (U[8]) / (V(9450.) * K[8]) - (U[10]) / (V(93555.) * K[10])) * gplus;
    A[3] = (-(1 / (V(2.) * a)) + u / (V(2.) * k) - (U[2]) / (V(6.) * K[2]) + (U[4]) / (V(90.) * K[4]) -
            -((U[6]) / (V(945.) * K[6])) + (U[8]) / (V(9450.) * K[8]) - (U[10]) / (V(93555.) * K[10])) * gminus;
    A[4] = V(1.) / (V(3.) * k) - (U[2]) / (V(45.) * K[3]) + (2 * U[4]) / (V(945.) * K[5]) - -((U[6]) / (V(4725.) * K[7])) +
           (2 * U[8]) / (V(93555.) * K[9]) - -((1382 * U[10]) / (V(6.38512875e8) * K[11]));
    A[5] = V(0.5) + (u) / (V(6.) * k) - (U[3]) / (V(90.) * K[3]) + (U[5]) / (V(945.) * K[5]) - -((U[7]) / (V(9450.) * K[7])) +
           (U[9]) / (V(93555.) * K[9]);
  }
}

// The temperature's NIM coefficients in float for the FP32 phase.  With
// x = 2u/k (the cell Reynolds number) every coefficient follows from
// h(x) = (x/(e^x-1) - 1 + x/2)/x^2 = sum_{n>=1} B_2n x^(2n-2)/(2n)!:
//   A0 = (-1 - 2xh)/k gplus    A1 = (-1 + 2xh)/k gminus
//   A2 = -(1 + x/2 + x^2 h)/2 gplus   A3 = -(1 - x/2 + x^2 h)/2 gminus
//   A4 = 4h/k                  A5 = 1/2 + xh
// (the exact functions the exp form of nim_direction evaluates).  For
// |x| <= 2 h is its Taylor series to x^14 (truncation below 1e-8); above,
// the exp form, which has no cancellation there.  Both keep every
// coefficient within ~1e-6 of the exact value (the FP64 forms lose ~1e-2 in
// float near |x| = v_limit).
__device__ __forceinline__ void nim_direction_f32(float u, float k, float gminus, float gplus, float A[6]) {
  const float ik = 1.f / k;
  const float x = 2.f * u * ik;
  if (fabsf(x) <= 2.f) {
    const float y = x * x;
    float h = -3617.f / 10670622842880000.f;
    h = fmaf(h, y, 1.f / 74724249600.f);
    h = fmaf(h, y, -691.f / 1307674368000.f);
    h = fmaf(h, y, 1.f / 47900160.f);
    h = fmaf(h, y, -1.f / 1209600.f);
    h = fmaf(h, y, 1.f / 30240.f);
    h = fmaf(h, y, -1.f / 720.f);
    h = fmaf(h, y, 1.f / 12.f);
    const float xh = x * h, yh = y * h;
    A[0] = (-1.f - 2.f * xh) * ik * gplus;
    A[1] = (-1.f + 2.f * xh) * ik * gminus;
    A[2] = -0.5f * (1.f + 0.5f * x + yh) * gplus;
    A[3] = -0.5f * (1.f - 0.5f * x + yh) * gminus;
    A[4] = 4.f * h * ik;
    A[5] = 0.5f + xh;
  } else {
    const float e = expf(x), ie = 1.f / e;
    A[0] = (2.f / (k * (ie - 1.f)) + 1.f / u) * gplus;
    A[1] = (-(2.f / (k * (1.f - e))) - 1.f / u) * gminus;
    A[2] = (u / (k * (ie - 1.f))) * gplus;
    A[3] = (u / (k * (1.f - e))) * gminus;
    if (x > 0) {
      A[4] = (-k + u * (ie + 1.f) / (1.f - ie)) / (u * u);
      A[5] = 1.f / (1.f - ie) - 1.f / x;
    } else {
      A[4] = (-k + u * (1.f + e) / (e - 1.f)) / (u * u);
      A[5] = e / (e - 1.f) - 1.f / x;
    }
  }
}

__global__ void k_exp_selftest(const double *x, double *y, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = nim_exp(x[i]);
}

// the six NIM coefficients of one direction (gminus = gplus = 1) for n
// (u, k) pairs: the FP64 form of the FP64 path or the float form of the
// FP32 phase; A[6i + q]
__global__ void k_nim_coef_selftest(const double *u, const double *k, double *A, int64_t n, int lowp,
                                    double v_limit) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (lowp) {
      float a[6];
      nim_direction_f32((float)u[i], (float)k[i], 1.f, 1.f, a);
      for (int q = 0; q < 6; ++q) A[6 * i + q] = a[q];
    } else {
      double a[6];
      nim_direction(u[i], k[i], 1., 1., v_limit, a);
      for (int q = 0; q < 6; ++q) A[6 * i + q] = a[q];
    }
  }
}

// contravariant component dd (1..3) of a Cartesian velocity in cell c
template <class R>
__device__ __forceinline__ Ar<R> contravariant(const R *xi, int Nc, int c, int dd, Ar<R> u, Ar<R> v, Ar<R> w) {
  return u * xi[(dd - 1 + 0) * Nc + c] + v * xi[(dd - 1 + 3) * Nc + c] + w * xi[(dd - 1 + 6) * Nc + c];
}

// calculate_velocity_nim_constants_formulation2, first pass (nim.f90:165-289)
template <class R>
__global__ void __launch_bounds__(BLK) k_vel_coef_A(Dims d, GeoT<R> g, FieldsT<R> F, Phys P) {
  using V = Ar<R>;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.Nc) return;
  const size_t Nc = d.Nc;
  const V ut = F.ct[0][c], vt = F.ct[1][c], wt = F.ct[2][c];
  for (int dd = 1; dd <= 3; ++dd) {
    const V u = contravariant(g.xi, Nc, c, dd, ut, vt, wt);
    V A[6];
    nim_direction<V>(u, g.gij[(size_t)(dd - 1 + 3 * (dd - 1)) * Nc + c] * pv<V>(P.nu, P.d_nu),
                     g.gfd[(2 * (dd - 1)) * Nc + c], g.gfd[(2 * (dd - 1) + 1) * Nc + c], P.v_limit, A);
    for (int k = 0; k < 6; ++k) F.MA[(size_t)(3 * k + dd - 1) * Nc + c] = A[k];
  }
}

// M_F4 and M_F1..3 from M_A (nim.f90:293-328); also used for the
// temperature's MT_F (nim.f90:466-500).
template <class V>
__device__ __forceinline__ void form_F4(const V A[3][6], V DT, V F4[8]) {
  F4[1] = V(0.5) * (V(1.) / A[0][4] + V(1.) / A[1][4] + V(1.) / A[2][4] - V(1.) / DT);
  F4[2] = -(A[0][5] / A[0][4]);
  F4[3] = (A[0][5] - V(1.)) / A[0][4];
  F4[4] = -(A[1][5] / A[1][4]);
  F4[5] = (A[1][5] - V(1.)) / A[1][4];
  F4[6] = -(A[2][5] / A[2][4]);
  F4[7] = (A[2][5] - V(1.)) / A[2][4];
  F4[0] = F4[1] + F4[2] + F4[3] + F4[4] + F4[5] + F4[6] + F4[7];
}
template <class V>
__device__ __forceinline__ void form_Fd(const V Ai[6], const V A2[6], V G[5]) {
  G[1] = Ai[2] - (Ai[0] * Ai[5] / Ai[4]);
  G[2] = A2[3] - A2[1] / A2[4] + A2[1] * A2[5] / A2[4];
  G[3] = Ai[0] / (V(2.) * Ai[4]);
  G[4] = A2[1] / (V(2.) * A2[4]);
  G[0] = G[1] + G[2] + V(2.) * G[3] + V(2.) * G[4];
}

// form_Fd and form_F4 with slot 4 holding 1/A4 (the float MT_A of the FP32
// phase): the same terms with each division by A4 a multiplication
template <class V>
__device__ __forceinline__ void form_Fd_rcp(const V Ai[6], const V A2[6], V G[5]) {
  G[1] = Ai[2] - Ai[0] * Ai[5] * Ai[4];
  G[2] = A2[3] - A2[1] * A2[4] + A2[1] * A2[5] * A2[4];
  G[3] = V(0.5) * Ai[0] * Ai[4];
  G[4] = V(0.5) * A2[1] * A2[4];
  G[0] = G[1] + G[2] + V(2) * G[3] + V(2) * G[4];
}
template <class V>
__device__ __forceinline__ void form_F4_rcp(const V A[3][6], V DT, V F4[8]) {
  F4[1] = V(0.5) * (A[0][4] + A[1][4] + A[2][4] - V(1) / DT);
  F4[2] = -(A[0][5] * A[0][4]);
  F4[3] = (A[0][5] - V(1)) * A[0][4];
  F4[4] = -(A[1][5] * A[1][4]);
  F4[5] = (A[1][5] - V(1)) * A[1][4];
  F4[6] = -(A[2][5] * A[2][4]);
  F4[7] = (A[2][5] - V(1)) * A[2][4];
  F4[0] = F4[1] + F4[2] + F4[3] + F4[4] + F4[5] + F4[6] + F4[7];
}

template <class R>
__global__ void __launch_bounds__(BLK) k_vel_coef_F(Dims d, FieldsT<R> F, Phys P) {
  using V = Ar<R>;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.Nc) return;
  const Cell x = Cell::of(d, c);
  const size_t Nc = d.Nc;
  V A[3][6];
  for (int dd = 0; dd < 3; ++dd)
    for (int k = 0; k < 6; ++k) A[dd][k] = F.MA[(size_t)(3 * k + dd) * Nc + c];
  V F4[8];
  form_F4<V>(A, P.DT, F4);
  for (int k = 0; k < 8; ++k) F.MF4[(size_t)k * Nc + c] = F4[k];
  for (int dd = 1; dd <= 3; ++dd) {
    V G[5] = {0., 0., 0., 0., 0.};
    if (x.has_nb(d, 2 * dd)) {
      const int i2 = x.nb(d, 2 * dd).c;
      V A2[6];
      for (int k = 0; k < 6; ++k) A2[k] = F.MA[(size_t)(3 * k + dd - 1) * Nc + i2];
      form_Fd(A[dd - 1], A2, G);
    }
    for (int k = 0; k < 5; ++k) F.MF[(size_t)(5 * (dd - 1) + k) * Nc + c] = G[k];
  }
}

// ====================================================== formulation 1
// B_nim, C_nim, G_nim, H_nim, I_nim, J_nim (nim.f90:748-875) of one
// direction, a = 1, for contravariant speed u, diffusivity F and cell Peclet
// number Re = 2u/F: series when |Re| < v_limit (condition, nim.f90:748-756),
// exponential form otherwise.  G_nim and H_nim assign P twice in their
// exponential branch; the second assignment is the one that counts.
struct Nim1 {
  double B, C, G, H, I, J;
  bool series;
};
__device__ __forceinline__ Nim1 nim1_direction(double u, double F, double Re, double v_limit) {
  const double a = 1.;
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
    const double e = nim_exp(Re);
    r.B = 1. / u * (1. / Re - 1. / (e - 1.));
    r.C = (-(1. / u) + 2. * r.B) * a;
    r.G = u / F / (1. - 1. / e);
    r.H = 2. * a / F / (1. - 1. / e) - 1. / u;
    r.I = u / (F * (e - 1.));
    r.J = 2. * a / (F * (e - 1.)) - 1. / u;
  }
  return r;
}
// E_nim and F_nim (nim.f90:787-815) with D = Det
__device__ __forceinline__ double nim1_E(const Nim1 &r, double u, double F, double D) {
  const double a = 1.;
  if (r.series) {
    const Pw U(u), K(F);
    return D / 2. + (a * D * u) / (6. * F) - (D * U[3]) / (90. * K[3]) + (D * U[5]) / (945. * K[5]) -
           -((D * U[7]) / (9450. * K[7])) + (D * U[9]) / (93555. * K[9]);
  }
  return D * (1 - r.B * u);
}
__device__ __forceinline__ double nim1_F(const Nim1 &r, double u, double F, double D) {
  const double a = 1.;
  if (r.series) {
    const Pw U(u), K(F);
    return D / 2. - (a * D * u) / (6. * F) + (D * U[3]) / (90. * K[3]) - (D * U[5]) / (945. * K[5]) +
           -((D * U[7]) / (9450. * K[7])) - (D * U[9]) / (93555. * K[9]);
  }
  return D * (r.B * u);
}

// calculate_velocity_nim_constants, first loop (nim.f90:29-83): CC .. JJ
// and Det of every cell, then a_t (nim.f90:146-154), which needs only them.
__global__ void __launch_bounds__(BLK) k_vel1_coef_A(Dims d, Geo g, Fields F, Phys P) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.Nc) return;
  const size_t Nc = d.Nc;
  const double ut = F.ct[0][c], vt = F.ct[1][c], wt = F.ct[2][c];
  double uc[3], K[3], Re[3];
  for (int dd = 1; dd <= 3; ++dd) {
    uc[dd - 1] = contravariant(g.xi, Nc, c, dd, ut, vt, wt);
    K[dd - 1] = g.gij[(size_t)(dd - 1 + 3 * (dd - 1)) * Nc + c] * P.nu;
    Re[dd - 1] = 2 * uc[dd - 1] / K[dd - 1];
  }
  Nim1 r[3];
  double C[3], E[3], Fv[3];
  for (int k = 0; k < 3; ++k) {
    r[k] = nim1_direction(uc[k], K[k], Re[k], P.v_limit);
    C[k] = r[k].C;
  }
  const double Det = 1. / (C[0] * C[1] + C[1] * C[2] + C[0] * C[2]);
  for (int k = 0; k < 3; ++k) {
    E[k] = nim1_E(r[k], uc[k], K[k], Det);
    Fv[k] = nim1_F(r[k], uc[k], K[k], Det);
    F.N1[(size_t)(0 + k) * Nc + c] = C[k];
    F.N1[(size_t)(3 + k) * Nc + c] = E[k];
    F.N1[(size_t)(6 + k) * Nc + c] = Fv[k];
    F.N1[(size_t)(9 + k) * Nc + c] = r[k].G;
    F.N1[(size_t)(12 + k) * Nc + c] = r[k].H;
    F.N1[(size_t)(15 + k) * Nc + c] = r[k].I;
    F.N1[(size_t)(18 + k) * Nc + c] = r[k].J;
  }
  F.N1[(size_t)21 * Nc + c] = Det;
  const double DT = P.DT;
  double at[9];
  at[0] = 2 * E[0] / Det - 2 * (C[1] + C[2]) * C[0] * E[0];
  at[1] = 2 * Fv[0] / Det - 2 * (C[1] + C[2]) * C[0] * Fv[0];
  at[2] = 2 * E[1] * C[0] * C[2];
  at[3] = 2 * Fv[1] * C[0] * C[2];
  at[4] = 2 * E[2] * C[0] * C[1];
  at[5] = 2 * Fv[2] * C[0] * C[1];
  at[6] = 2 * C[0] * C[1] * C[2] * Det;
  at[7] = -at[6] / (2 * DT) - 1;
  at[8] = at[6] / (2 * DT) - 1;
  for (int k = 0; k < 9; ++k) F.AT[(size_t)k * Nc + c] = at[k];
}

// calculate_velocity_nim_constants, second loop (nim.f90:85-143): AA_vx,
// AA_vy, AA_vz of the +r, +theta, +z faces from the cell and its neighbour.
__global__ void __launch_bounds__(BLK) k_vel1_coef_F(Dims d, Geo g, Fields F, Phys P) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.Nc) return;
  const Cell x = Cell::of(d, i);
  const size_t Nc = d.Nc;
  const double DT = P.DT;
  auto C = [&](int k, int n) { return F.N1[(size_t)(k - 1) * Nc + n]; };
  auto E = [&](int k, int n) { return F.N1[(size_t)(2 + k) * Nc + n]; };
  auto Fv = [&](int k, int n) { return F.N1[(size_t)(5 + k) * Nc + n]; };
  auto GG = [&](int k, int n) { return F.N1[(size_t)(8 + k) * Nc + n]; };
  auto HH = [&](int k, int n) { return F.N1[(size_t)(11 + k) * Nc + n]; };
  auto II = [&](int k, int n) { return F.N1[(size_t)(14 + k) * Nc + n]; };
  auto JJ = [&](int k, int n) { return F.N1[(size_t)(17 + k) * Nc + n]; };
  auto Det = [&](int n) { return F.N1[(size_t)21 * Nc + n]; };
  double A[16];
  if (x.has_nb(d, 2)) {  // face 2 (nim.f90:87-104)
    const int i2 = x.nb(d, 2).c;
    const double g2 = g.gfd[1 * Nc + i], g1 = g.gfd[0 * Nc + i2];
    A[1] = -(GG(1, i) + (C(2, i) + C(3, i)) * E(1, i) * HH(1, i)) * g2;
    A[2] = (GG(1, i) - (C(2, i) + C(3, i)) * Fv(1, i) * HH(1, i)) * g2 +
           (II(1, i2) + (C(2, i2) + C(3, i2)) * E(1, i2) * JJ(1, i2)) * g1;
    A[3] = -(II(1, i2) - (C(2, i2) + C(3, i2)) * Fv(1, i2) * JJ(1, i2)) * g1;
    A[4] = C(3, i) * E(2, i) * HH(1, i) * g2;
    A[5] = C(3, i) * Fv(2, i) * HH(1, i) * g2;
    A[6] = -C(3, i2) * E(2, i2) * JJ(1, i2) * g1;
    A[7] = -C(3, i2) * Fv(2, i2) * JJ(1, i2) * g1;
    A[8] = C(2, i) * E(3, i) * HH(1, i) * g2;
    A[9] = C(2, i) * Fv(3, i) * HH(1, i) * g2;
    A[10] = -C(2, i2) * E(3, i2) * JJ(1, i2) * g1;
    A[11] = -C(2, i2) * Fv(3, i2) * JJ(1, i2) * g1;
    A[12] = C(2, i) * C(3, i) * Det(i) * HH(1, i) * g2 / (2 * DT);
    A[13] = -C(2, i) * C(3, i) * Det(i) * HH(1, i) * g2 / (2 * DT);
    A[14] = -C(2, i2) * C(3, i2) * Det(i2) * JJ(1, i2) * g1 / (2 * DT);
    A[15] = C(2, i2) * C(3, i2) * Det(i2) * JJ(1, i2) * g1 / (2 * DT);
    for (int k = 1; k <= 15; ++k) F.AAv[(size_t)(k - 1) * Nc + i] = A[k];
  }
  if (x.has_nb(d, 4)) {  // face 4 (nim.f90:107-124)
    const int i2 = x.nb(d, 4).c;
    const double g4 = g.gfd[3 * Nc + i], g3 = g.gfd[2 * Nc + i2];
    A[1] = C(3, i) * E(1, i) * HH(2, i) * g4;
    A[2] = C(3, i) * Fv(1, i) * HH(2, i) * g4;
    A[3] = -C(3, i2) * E(1, i2) * JJ(2, i2) * g3;
    A[4] = -C(3, i2) * Fv(1, i2) * JJ(2, i2) * g3;
    A[5] = -(GG(2, i) + (C(1, i) + C(3, i)) * E(2, i) * HH(2, i)) * g4;
    A[6] = (GG(2, i) - (C(1, i) + C(3, i)) * Fv(2, i) * HH(2, i)) * g4 +
           (II(2, i2) + (C(1, i2) + C(3, i2)) * E(2, i2) * JJ(2, i2)) * g3;
    A[7] = -(II(2, i2) - (C(1, i2) + C(3, i2)) * Fv(2, i2) * JJ(2, i2)) * g3;
    A[8] = C(1, i) * E(3, i) * HH(2, i) * g4;
    A[9] = C(1, i) * Fv(3, i) * HH(2, i) * g4;
    A[10] = -C(1, i2) * E(3, i2) * JJ(2, i2) * g3;
    A[11] = -C(1, i2) * Fv(3, i2) * JJ(2, i2) * g3;
    A[12] = C(1, i) * C(3, i) * Det(i) * HH(2, i) * g4 / (2 * DT);
    A[13] = -C(1, i) * C(3, i) * Det(i) * HH(2, i) * g4 / (2 * DT);
    A[14] = -C(1, i2) * C(3, i2) * Det(i2) * JJ(2, i2) * g3 / (2 * DT);
    A[15] = C(1, i2) * C(3, i2) * Det(i2) * JJ(2, i2) * g3 / (2 * DT);
    for (int k = 1; k <= 15; ++k) F.AAv[(size_t)(14 + k) * Nc + i] = A[k];
  }
  if (x.has_nb(d, 6)) {  // face 6 (nim.f90:126-143)
    const int i2 = x.nb(d, 6).c;
    const double g6 = g.gfd[5 * Nc + i], g5 = g.gfd[4 * Nc + i2];
    A[1] = C(2, i) * E(1, i) * HH(3, i) * g6;
    A[2] = C(2, i) * Fv(1, i) * HH(3, i) * g6;
    A[3] = -C(2, i2) * E(1, i2) * JJ(3, i2) * g5;
    A[4] = -C(2, i2) * Fv(1, i2) * JJ(3, i2) * g5;
    A[5] = C(1, i) * E(2, i) * HH(3, i) * g6;
    A[6] = C(1, i) * Fv(2, i) * HH(3, i) * g6;
    A[7] = -C(1, i2) * E(2, i2) * JJ(3, i2) * g5;
    A[8] = -C(1, i2) * Fv(2, i2) * JJ(3, i2) * g5;
    A[9] = -(GG(3, i) + (C(1, i) + C(2, i)) * E(3, i) * HH(3, i)) * g6;
    A[10] = (GG(3, i) - (C(1, i) + C(2, i)) * Fv(3, i) * HH(3, i)) * g6 +
            (II(3, i2) + (C(1, i2) + C(2, i2)) * E(3, i2) * JJ(3, i2)) * g5;
    A[11] = -(II(3, i2) - (C(1, i2) + C(2, i2)) * Fv(3, i2) * JJ(3, i2)) * g5;
    A[12] = C(1, i) * C(2, i) * Det(i) * HH(3, i) * g6 / (2 * DT);
    A[13] = -C(1, i) * C(2, i) * Det(i) * HH(3, i) * g6 / (2 * DT);
    A[14] = -C(1, i2) * C(2, i2) * Det(i2) * JJ(3, i2) * g5 / (2 * DT);
    A[15] = C(1, i2) * C(2, i2) * Det(i2) * JJ(3, i2) * g5 / (2 * DT);
    for (int k = 1; k <= 15; ++k) F.AAv[(size_t)(29 + k) * Nc + i] = A[k];
  }
}

// =========================================================== iteration
// Load policies: the parallel kernels read with plain (L1-cached) loads; the
// reference-order sweeps read data that other SMs rewrote one level earlier
// (LdCoh below).
struct LdPlain {
  template <class T>
  __device__ __forceinline__ static Ar<T> ld(const T *p, size_t i) { return p[i]; }
};
// Loads and stores of values the same launch rewrites in place (the
// reference-order sweeps) go through volatile: never the non-coherent
// read-only path, never merged, and kept in program order against each
// other, so a thread sees its own earlier stores and every store made before
// the last grid or block barrier.  Other loads stay free to be scheduled.
struct LdCoh {
  template <class T>
  __device__ __forceinline__ static Ar<T> ld(const T *p, size_t i) {
    return *(const volatile T *)(p + i);
  }
};
__device__ __forceinline__ void st_coh(double *p, size_t i, double v) { *(volatile double *)(p + i) = v; }

// a new value as the storage type R keeps it: the change find_error
// measures is that of the stored field (identity for double)
template <class R>
__device__ __forceinline__ Ar<R> stored(Ar<R> v) { return (Ar<R>)(R)v; }

__device__ __forceinline__ int parity(const Ctrl *ctl) { return ctl->iter & ctl->pmask; }
// half holding the values a sweep earlier in this pass produced
__device__ __forceinline__ int newhalf(const Ctrl *ctl) { return ctl->pmask ? 1 - parity(ctl) : parity(ctl); }

// fn(IC<y + 1>{}) for a warp-uniform y in 0..2: the direction (or component)
// becomes a compile-time constant, so every face/neighbour selection on it
// folds away instead of running as integer code per thread
template <int V>
struct IC {
  static constexpr int value = V;
};
template <class Fn>
__device__ __forceinline__ void by_dir(int y, Fn &&fn) {
  if (y == 0) fn(IC<1>{});
  else if (y == 1) fn(IC<2>{});
  else fn(IC<3>{});
}

// Green-Gauss derivative dphi_dx2/dy2/dz2 (nse.f90:2866-2903), component cc
// in the value type V of phi (the kernel's arithmetic type)
template <class R, class V>
__device__ __forceinline__ V green_gauss(const GeoT<R> &g, size_t NF, V invV, const V phi[7], const int f[7], int cc) {
  const R *A = g.area, *n = g.normal + cc * NF;
  return invV * (phi[2] * A[f[2]] * (n[f[2]]) - phi[1] * A[f[1]] * (n[f[1]]) + phi[4] * A[f[4]] * (n[f[4]]) -
                 phi[3] * A[f[3]] * (n[f[3]]) + phi[6] * A[f[6]] * (n[f[6]]) - phi[5] * A[f[5]] * (n[f[5]]));
}

// Derivative of face field phi along local direction e on face fpos of cell
// x: centred, or second-order one-sided at walls (the ni/nj/nk stencils of
// calculate_R_D2, nse.f90:1635-1838; integrate_pressure_field_i; bc.f90).
template <class Ld = LdPlain, class R>
__device__ __forceinline__ Ar<R> tangential(const Dims &d, const R *__restrict__ phi, const Cell &x, int fpos,
                                            int e) {
  using A = Ar<R>;
  const bool lo = !x.has_nb(d, 2 * e - 1), hi = !x.has_nb(d, 2 * e);
  if (lo) {
    const Cell m2 = x.nb(d, 2 * e), m3 = m2.nb(d, 2 * e);
    return (-(3 * Ld::ld(phi, x.face(d, fpos))) + 4 * Ld::ld(phi, m2.face(d, fpos)) - Ld::ld(phi, m3.face(d, fpos))) / A(4);
  } else if (hi) {
    const Cell m1 = x.nb(d, 2 * e - 1), m3 = m1.nb(d, 2 * e - 1);
    return (3 * Ld::ld(phi, x.face(d, fpos)) - 4 * Ld::ld(phi, m1.face(d, fpos)) + Ld::ld(phi, m3.face(d, fpos))) / A(4);
  }
  return (Ld::ld(phi, x.nb(d, 2 * e).face(d, fpos)) - Ld::ld(phi, x.nb(d, 2 * e - 1).face(d, fpos))) / A(4);
}

// G_i d_i phi - g^ij d_ij phi of calculate_R_D2 / R_D_p2 / R_D_T
// (nse.f90:1852-1859, 1995-1996, 2132-2133), before the coefficient.
template <class R>
__device__ __forceinline__ Ar<R> diffusion_source(const Dims &d, const GeoT<R> &g, const R *__restrict__ phi,
                                                  const Cell &x, const int f[7]) {
  using V = Ar<R>;
  const size_t Nc = d.Nc;
  const int c = x.c;
  const V pxy = V(0.5) * (tangential(d, phi, x, 2, 2) - tangential(d, phi, x, 1, 2));
  const V pzy = V(0.5) * (tangential(d, phi, x, 6, 2) - tangential(d, phi, x, 5, 2));
  const V pyx = V(0.5) * (tangential(d, phi, x, 4, 1) - tangential(d, phi, x, 3, 1));
  const V pzx = V(0.5) * (tangential(d, phi, x, 6, 1) - tangential(d, phi, x, 5, 1));
  const V pxz = V(0.5) * (tangential(d, phi, x, 2, 3) - tangential(d, phi, x, 1, 3));
  const V pyz = V(0.5) * (tangential(d, phi, x, 4, 3) - tangential(d, phi, x, 3, 3));
  const V px = (phi[f[2]] - phi[f[1]]) / V(2.);
  const V py = (phi[f[4]] - phi[f[3]]) / V(2.);
  const V pz = (phi[f[6]] - phi[f[5]]) / V(2.);
  const R *G = g.G, *gij = g.gij;
  return (G[c] * px + G[Nc + c] * py + G[2 * Nc + c] * pz - gij[3 * Nc + c] * pxy - gij[1 * Nc + c] * pyx -
          gij[6 * Nc + c] * pxz - gij[2 * Nc + c] * pzx - gij[7 * Nc + c] * pyz - gij[5 * Nc + c] * pzy);
}

__device__ __forceinline__ void cell_faces(const Dims &d, const Cell &x, int f[7]) {
  f[1] = x.c + d.NT * x.k;
  f[2] = f[1] + d.NT;
  f[3] = d.offT + x.c;
  f[4] = d.offT + x.c - x.i + ((x.i == d.NT - 1) ? 0 : x.i + 1);
  f[5] = d.offZ + x.c;
  f[6] = f[5] + d.plane;
}

// Cell-average update (nse.f90:840-848; T: 1018-1026)
template <class Ld = LdPlain, class R>
__device__ __forceinline__ Ar<R> cell_update(const R *__restrict__ fr, const int f[7], Ar<R> c, Ar<R> cold,
                                             Ar<R> B, const Ar<R> F4[8], Ar<R> w) {
  return (1 - w) * c +
         (w / F4[0]) * (+F4[1] * cold + F4[2] * Ld::ld(fr, f[1]) + F4[3] * Ld::ld(fr, f[2]) +
                        F4[4] * Ld::ld(fr, f[3]) + F4[5] * Ld::ld(fr, f[4]) + F4[6] * Ld::ld(fr, f[5]) +
                        F4[7] * Ld::ld(fr, f[6]) + B);
}

// +xi_d face update (nse.f90:878-1005; T: 1033-1088) from the face values
// fx(pos) of cell x and fx2(pos) of its +xi_d neighbour x2, their cell
// values cx, cx2 and old cell values ox, ox2
template <class V, class FX, class FX2>
__device__ __forceinline__ V face_update_vals(FX &&fx, FX2 &&fx2, V cx, V cx2, V ox, V ox2, const V Fd[5], V dg0,
                                              V dg1, int dd, V w) {
  const int e1 = tr1(dd), e2 = tr2(dd);
  const V B3 = (dg0) * (fx(2 * e1) - fx(2 * e1 - 1) + fx2(2 * e1) - fx2(2 * e1 - 1)) / V(4.0);
  const V B4 = (dg1) * (fx(2 * e2) - fx(2 * e2 - 1) + fx2(2 * e2) - fx2(2 * e2 - 1)) / V(4.0);
  return (1 - w) * fx(2 * dd) +
         (w / Fd[0]) * (+Fd[1] * fx(2 * dd - 1) + Fd[2] * fx2(2 * dd) + Fd[3] * (cx + ox) + Fd[4] * (cx2 + ox2) -
                        B3 - B4);
}
// the same from the face array fr; cx, cx2 the cell values of x and x2
template <class Ld = LdPlain, class R>
__device__ __forceinline__ Ar<R> face_update_cv(const Dims &d, const R *__restrict__ fr, Ar<R> cx, Ar<R> cx2,
                                                const R *__restrict__ co, const Ar<R> Fd[5], Ar<R> dg0, Ar<R> dg1,
                                                int dd, const Cell &x, const Cell &x2, Ar<R> w) {
  return face_update_vals<Ar<R>>([&](int pos) { return Ld::ld(fr, x.face(d, pos)); },
                                 [&](int pos) { return Ld::ld(fr, x2.face(d, pos)); }, cx, cx2, (Ar<R>)co[x.c],
                                 (Ar<R>)co[x2.c], Fd, dg0, dg1, dd, w);
}
template <class Ld = LdPlain, class R>
__device__ __forceinline__ Ar<R> face_update(const Dims &d, const R *__restrict__ fr, const R *__restrict__ cv,
                                             const R *__restrict__ co, const Ar<R> Fd[5], Ar<R> dg0, Ar<R> dg1,
                                             int dd, const Cell &x, const Cell &x2, Ar<R> w) {
  return face_update_cv<Ld>(d, fr, Ld::ld(cv, x.c), Ld::ld(cv, x2.c), co, Fd, dg0, dg1, dd, x, x2, w);
}

// Formulation 1 cell update of one velocity component (integrate_velocity_
// field_i, nse.f90:341-352); Rs = R_C + R_D + R_B of the cell, at = a_t(1:9).
template <class Ld = LdPlain, class R>
__device__ __forceinline__ Ar<R> cell_update_f1(const R *__restrict__ fr, const int f[7], Ar<R> c, Ar<R> cold,
                                                Ar<R> Rs, const Ar<R> at[9], Ar<R> w) {
  const Ar<R> Bij = at[6] * Rs;
  return (1 - w) * c + w * (-(at[0] * Ld::ld(fr, f[1])) - at[1] * Ld::ld(fr, f[2]) - at[2] * Ld::ld(fr, f[3]) -
                            at[3] * Ld::ld(fr, f[4]) - at[4] * Ld::ld(fr, f[5]) - at[5] * Ld::ld(fr, f[6]) -
                            at[7] * cold - Bij) /
                           (at[8]);
}

// ---- bulk copies into shared memory: cp.async.bulk rows whose completion
// is counted in bytes on an mbarrier (phase 0, one arrival: the thread that
// posts the byte count).  Every wait is bounded; a wait that runs out marks
// the step NIM_ERR_TIMEOUT and stopped, then waits (bounded) once more so
// that no copy lands in shared memory after the block has left.
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// dst and src 16-byte aligned, bytes a multiple of 16
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, unsigned long long *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
constexpr int kWaitTries = 1 << 22;  // each try suspends for a hardware-chosen slice
__device__ __noinline__ bool mbar_wait(unsigned long long *bar, unsigned parity, Ctrl *ctl,
                                       int tries = kWaitTries) {
  for (int n = 0; n < tries; ++n)
    if (mbar_try_wait(bar, parity)) return true;
  atomicCAS(&ctl->status, 0, -5);  // NIM_ERR_TIMEOUT
  *(volatile int *)&ctl->done = 1;
  for (int n = 0; n < tries; ++n)
    if (mbar_try_wait(bar, parity)) break;
  return false;
}

// The timeout path of mbar_wait on the device, without a fault: one thread
// posts 16 expected bytes that no copy will bring and waits at most `tries`
// times; the step is then marked NIM_ERR_TIMEOUT and stopped.  No copy is in
// flight, so nothing can land after the block leaves.
__global__ void k_wait_selftest(Ctrl *ctl, int tries) {
  __shared__ alignas(8) unsigned long long bar;
  mbar_init(&bar, 1);
  mbar_expect_tx(&bar, 16);
  mbar_wait(&bar, 0, ctl, tries);
}

// nim_exp over n arguments (self-test of the exp the NIM coefficients use)

// The block coordinates a pass kernel's body works on.  LaunchBlock reads
// the launch's own blockIdx where the body uses a coordinate (the plain
// kernels: the same code as reading blockIdx directly); BatchBlock holds the
// coordinates of one block of one enclosure's grid, decoded by a fused batch
// launch (k_batch_*) from its work list.
struct LaunchBlockX {
  __device__ __forceinline__ operator unsigned() const { return ::blockIdx.x; }
};
struct LaunchBlockY {
  __device__ __forceinline__ operator unsigned() const { return ::blockIdx.y; }
};
struct LaunchBlockZ {
  __device__ __forceinline__ operator unsigned() const { return ::blockIdx.z; }
};
struct LaunchBlock {
  LaunchBlockX x;
  LaunchBlockY y;
  LaunchBlockZ z;
};
struct BatchBlock {
  unsigned x, y, z;
};
// A block of a fused batch launch over cells in cell order: x numbers the
// runs of blockDim.x consecutive cells of plane z (y unused).  Every lane
// has a cell whatever n_theta is, where the 32-wide theta patches of
// patch_cell leave lanes idle on narrow meshes (n_theta = 40: 5 of 8 warps'
// lanes busy); only patch_cell's kernels take it.
struct FlatBlock {
  unsigned x, y, z;
};

__device__ __forceinline__ double errv(double nw, double old, bool first) { return fabs(nw - (first ? 0.0 : old)); }
__device__ __forceinline__ double errv(const DualD &nw, const DualD &old, bool first) {
  return errv(nw.v, old.v, first);
}
// max that keeps a NaN (fmax would drop it and hide a blow-up)
__device__ __forceinline__ double nmax(double a, double b) { return (b > a || b != b) ? b : a; }

// Cell of this thread in a 3D launch over patches of 32 (theta) x R (r)
// cells of one z-plane: grid (ceil(NT/32), ceil(NR/R), NZ), threadIdx.x
// spans the patch (R = blockDim.x / 32).  No division by run-time sizes, and
// the +-r neighbours of a cell mostly sit in the same block.
// bi: the block's coordinates, blockIdx itself (LaunchBlock) or those of a
// block of one enclosure's grid inside a fused batch launch (BatchBlock)
template <class BI>
__device__ __forceinline__ bool patch_cell(const Dims &d, Cell &x, const BI bi) {
  const int i = bi.x * 32 + (threadIdx.x & 31);
  const int j = bi.y * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int k = bi.z;
  x = Cell::at(d, i, j, k);
  return i < d.NT && j < d.NR;
}
__device__ __forceinline__ bool patch_cell(const Dims &d, Cell &x) { return patch_cell(d, x, LaunchBlock{}); }
// The first of the NP theta-adjacent cells of this thread in the NP-cells-
// a-thread sweeps (block (CB, 3)): rows of 32 NP cells (theta) x CB/32 (r)
// per block, or with a FlatBlock runs of CB groups of NP consecutive cells
// of plane z (n_theta % NP == 0).  Row j < NR for a thread with cells.
template <int NP, class BI>
__device__ __forceinline__ void group_cell(const Dims &d, const BI bi, int &i, int &j) {
  i = bi.x * (32 * NP) + NP * (threadIdx.x & 31);
  j = bi.y * (CB / 32) + (threadIdx.x >> 5);
}
template <int NP>
__device__ __forceinline__ void group_cell(const Dims &d, const FlatBlock bi, int &i, int &j) {
  const int t = (int)bi.x * CB + (int)threadIdx.x, per = d.NT / NP;  // group of plane z
  j = t / per;
  i = NP * (t - j * per);
}
__device__ __forceinline__ bool patch_cell(const Dims &d, Cell &x, const FlatBlock bi) {
  const int t = (int)bi.x * (int)blockDim.x + (int)threadIdx.x;  // cell of plane z in cell order
  const int j = t / d.NT, i = t - j * d.NT;
  x = Cell::at(d, i, j, (int)bi.z);
  return j < d.NR;
}

// ---- K1: velocity sources + cell update (update_velocity_sources
// nse.f90:199-211 with calculate_gforces 2484-2502, calculate_R_b 1562-1592,
// calculate_R_D2 1628-1860; cell part of integrate_velocity_field_formulation2_i
// 839-872).  R_C (calculate_R_c_new, 1393-1434) is identically zero.
// Block (CB, 3): threadIdx.y = velocity component.
// SRC_ONLY (reference-order schedule): store R_C + R_D + R_B and leave the
// update to k_seq_vel, as update_velocity_sources precedes the sweep.
// FORM 1 (nim_formulation = 1): the a_t cell update of integrate_velocity_
// field_i (nse.f90:341-378); the R sums are stored too, for the face sweep
// reads them at both cells of a face.
template <bool SRC_ONLY, int FORM, class R, class BI>
__device__ __forceinline__ void vel_cell_body(const Dims &d, const GeoT<R> &g, const FieldsT<R> &F, const Phys &P, Ctrl *ctl, const BI blockIdx) {
  using V = Ar<R>;
  if (ctl->done) return;
  __shared__ BlockRed red;
  red_init<3>(red);
  const int par = parity(ctl);
  const bool first = ctl->first;
  const int q = threadIdx.y;
  Cell x;
  const bool act = patch_cell(d, x, blockIdx);
  const int c = x.c;
  double e[3] = {0., 0., 0.};
  if (act) {
    const size_t Nc = d.Nc, NF = d.NF;
    int f[7];
    cell_faces(d, x, f);
    const R *fp = F.f[3] + par * NF;
    V pf[7];
    for (int k = 1; k <= 6; ++k) pf[k] = fp[f[k]];
    const V invV = inv_vol(g, c);
    const V base = (q == 2) ? -(V(P.g_beta) * V(0.5) * (F.c[3][c] + F.co[3][c])) : V(0.);
    const V RB = base + V(P.inv_rho) * green_gauss(g, NF, invV, pf, f, q);
    const R *fr = F.f[q] + par * NF;
    const V RD = pv<V>(P.inv_Re, P.d_inv_Re) * diffusion_source(d, g, fr, x, f);
    const V B = (V(0.) + RD + RB);
    if (SRC_ONLY || FORM == 1) F.Bv[(size_t)q * Nc + c] = B;
    if (!SRC_ONLY) {
      const V cold = F.c[q][c];
      V nw;
      if (FORM == 1) {
        V at[9];
        for (int k = 0; k < 9; ++k) at[k] = F.AT[(size_t)k * Nc + c];
        nw = stored<R>(cell_update_f1(fr, f, cold, F.co[q][c], B, at, V(P.w[q])));
      } else {
        V F4[8];
        for (int k = 0; k < 8; ++k) F4[k] = F.MF4[(size_t)k * Nc + c];
        nw = stored<R>(cell_update(fr, f, cold, F.co[q][c], B, F4, V(P.w[q])));
      }
      F.c[q][c] = nw;
      e[q] = errv(nw, cold, first);
    }
  }
  // blocks of one z plane: a plane another slab owns adds nothing
  if (!SRC_ONLY && d.owns(blockIdx.z)) block_max<3, CB3>(red, e, ctl->err[par]);
}
template <bool SRC_ONLY, int FORM, class R>
__global__ void __launch_bounds__(CB3, 3) k_vel_cell(Dims d, GeoT<R> g, FieldsT<R> F, Phys P, Ctrl *ctl) {
  vel_cell_body<SRC_ONLY, FORM, R>(d, g, F, P, ctl, LaunchBlock{});
}

// ---- K1, vectorised form (parallel schedule, formulation 2): k_vel_cell
// with each thread on two theta-adjacent cells (i even, i+1) of one
// component, so that nearly every load brings both cells' values at once
// (16 bytes in FP64): the cell arrays, the r and z faces, and the theta faces
// at i and i+1 (the +theta face of cell i is the -theta face of cell i+1).
// Only the faces at i-1 and i+2 that the theta stencils reach, and the
// +theta face of cell i+1, are single loads: ~70 load instructions for two
// cells instead of ~120.  The two cells advance together term by term, in
// each sum's source order, so the arithmetic is k_vel_cell's to the bit.
// Needs n_theta even; block (CB, 3) over patches of 64 x CB/32 cells.
template <class R>
struct Pair2;
template <>
struct Pair2<double> {
  using T = double2;
};
template <>
struct Pair2<float> {
  using T = float2;
};
// p[i], p[i+1] for an even element index i (a 2 x sizeof(R)-aligned pair)
template <class R>
__device__ __forceinline__ void ld2(const R *__restrict__ p, int i, R &a, R &b) {
  const typename Pair2<R>::T v = *reinterpret_cast<const typename Pair2<R>::T *>(p + i);
  a = v.x;
  b = v.y;
}
// tangential() from the values: v0 at the cell, vp1 / vp2 one / two cells
// along +e, vm1 / vm2 along -e (only those the branch reads are used)
template <class V>
__device__ __forceinline__ V tang_vals(bool lo, bool hi, V v0, V vp1, V vp2, V vm1, V vm2) {
  if (lo) return (-(3 * v0) + 4 * vp1 - vp2) / V(4.);
  if (hi) return (3 * v0 - 4 * vm1 + vm2) / V(4.);
  return (vp1 - vm1) / V(4.);
}

// Index arithmetic here is 32-bit (its largest offset is 9 x the cell count;
// nim_gpu_create refuses meshes for which 19 x the cell count would not fit
// an int): 64-bit offsets took registers that the kernel's bound of 56
// turned into spills (184 bytes against 108).
// SLAB: a z-slab context, whose maxima skip the planes a neighbour owns (a
// separate instantiation: at this kernel's register bound the test alone
// costs spills)
template <class R, bool SLAB = false, class BI = LaunchBlock>
__device__ __forceinline__ void vel_cell2_body(const Dims &d, const GeoT<R> &g, const FieldsT<R> &F, const Phys &P, Ctrl *ctl, const BI blockIdx) {
  using V = Ar<R>;
  if (ctl->done) return;
  __shared__ BlockRed red;
  red_init<3>(red);
  const int par = parity(ctl);
  const bool first = ctl->first;
  const int q = threadIdx.y;
  int i = blockIdx.x * 64 + 2 * (threadIdx.x & 31);
  int j = blockIdx.y * (CB / 32) + (threadIdx.x >> 5);
  if constexpr (std::is_same<BI, FlatBlock>::value) group_cell<2>(d, blockIdx, i, j);
  const int k = blockIdx.z;
  double e[3] = {0., 0., 0.};
  if (i < d.NT && j < d.NR) {
    const int Nc = d.Nc, NF = d.NF, NT = d.NT, NR = d.NR, pl = d.plane;
    const int c = i + NT * (j + NR * k);  // cell i; the pair's second cell is c + 1
    const int im1 = (i == 0) ? d.NT - 1 : i - 1, ip2 = (i + 2 >= d.NT) ? i + 2 - d.NT : i + 2;
    // face m of cell i at fi[m]; of cell i+1 at fi[m] + 1, except face 4: f4b
    const int f1 = c + NT * k;
    const int fi[7] = {0, f1, f1 + NT, d.offT + c, d.offT + c + 1, d.offZ + c, d.offZ + c + pl};
    const int f4b = d.offT + c - i + ip2;
    // face m of both cells from array a (pairs; faces 3 and 4 share one pair)
    auto face2 = [&](const R *a, int m, R &v0, R &v1) {
      if (m == 4) {
        v0 = a[fi[3] + 1];
        v1 = a[f4b];
      } else {
        ld2(a, fi[m], v0, v1);
      }
    };
    // RB = base + 1/rho * green_gauss (component q): the sum term by term in
    // source order (faces 2, 1, 4, 3, 6, 5) for both cells
    const R *pp = F.f[3] + par * NF, *nq = g.normal + q * NF;
    V gs0 = V(0.), gs1 = V(0.);
    {
      const int order[6] = {2, 1, 4, 3, 6, 5};
      // face 3 of both cells, loaded with face 4's turn: the pair's second
      // value is also face 4 of the first cell
      R p3[2], a3[2], n3[2];
#pragma unroll
      for (int t = 0; t < 6; ++t) {
        const int m = order[t];
        R p0, p1, a0, a1, n0, n1;
        if (m == 4) {
          ld2(pp, fi[3], p3[0], p3[1]);
          ld2(g.area, fi[3], a3[0], a3[1]);
          ld2(nq, fi[3], n3[0], n3[1]);
          p0 = p3[1], a0 = a3[1], n0 = n3[1];
          p1 = pp[f4b], a1 = g.area[f4b], n1 = nq[f4b];
        } else if (m == 3) {
          p0 = p3[0], a0 = a3[0], n0 = n3[0];
          p1 = p3[1], a1 = a3[1], n1 = n3[1];
        } else {
          face2(pp, m, p0, p1);
          face2(g.area, m, a0, a1);
          face2(nq, m, n0, n1);
        }
        const V t0 = (V)p0 * a0 * (n0), t1 = (V)p1 * a1 * (n1);
        if (t == 0) {
          gs0 = t0;
          gs1 = t1;
        } else if (t & 1) {
          gs0 = gs0 - t0;
          gs1 = gs1 - t1;
        } else {
          gs0 = gs0 + t0;
          gs1 = gs1 + t1;
        }
      }
    }
    V RB0, RB1;
    {
      R v0, v1;
      ld2(g.vol, c, v0, v1);
      V base0 = V(0.), base1 = V(0.);
      if (q == 2) {
        R t0, t1, o0, o1;
        ld2(F.c[3], c, t0, t1);
        ld2(F.co[3], c, o0, o1);
        base0 = -(V(P.g_beta) * V(0.5) * (t0 + o0));
        base1 = -(V(P.g_beta) * V(0.5) * (t1 + o1));
      }
      const V invV0 = V(1.) / v0, invV1 = V(1.) / v1;
      RB0 = base0 + V(P.inv_rho) * (invV0 * gs0);
      RB1 = base1 + V(P.inv_rho) * (invV1 * gs1);
    }
    // own faces of component q (stored values)
    const R *fr = F.f[q] + par * NF;
    R o0[7], o1[7];
    for (int m = 1; m <= 6; ++m)
      if (m != 4) face2(fr, m, o0[m], o1[m]);
    o0[4] = o1[3];  // face 4 of cell i is face 3 of cell i+1
    o1[4] = fr[f4b];
    // rows / planes a and b: the -e,+e neighbours (centred), +1,+2 (lo) or -1,-2 (hi)
    auto along = [&](bool lo, bool hi, V v0, V va, V vb) {
      return lo ? tang_vals(true, false, v0, va, vb, V(0.), V(0.))
                : hi ? tang_vals(false, true, v0, V(0.), V(0.), va, vb) : tang_vals(false, false, v0, vb, V(0.), va, V(0.));
    };
    // R_D: G_i d_i phi - g^ij d_ij phi, term by term in source order; each
    // cross derivative is formed for both cells right before its term
    const bool rlo = (j == 0), rhi = (j == d.NR - 1);
    const int ra = rlo ? j + 1 : j - 1, rb = rlo ? j + 2 : (rhi ? j - 2 : j + 1);
    const bool zlo = (k == 0), zhi = (k == d.NZ - 1);
    const int ka = zlo ? k + 1 : k - 1, kb = zlo ? k + 2 : (zhi ? k - 2 : k + 1);
    V s0, s1;
    {
      const V px0 = (o0[2] - o0[1]) / V(2.), px1 = (o1[2] - o1[1]) / V(2.);
      const V py0 = (o0[4] - o0[3]) / V(2.), py1 = (o1[4] - o1[3]) / V(2.);
      const V pz0 = (o0[6] - o0[5]) / V(2.), pz1 = (o1[6] - o1[5]) / V(2.);
      R a0, a1;
      ld2(g.G, c, a0, a1);
      s0 = a0 * px0;
      s1 = a1 * px1;
      ld2(g.G + Nc, c, a0, a1);
      s0 = s0 + a0 * py0;
      s1 = s1 + a1 * py1;
      ld2(g.G + 2 * Nc, c, a0, a1);
      s0 = s0 + a0 * pz0;
      s1 = s1 + a1 * pz1;
    }
    auto term = [&](int slot, V d0, V d1) {
      R a0, a1;
      ld2(g.gij + slot * Nc, c, a0, a1);
      s0 = s0 - a0 * d0;
      s1 = s1 - a1 * d1;
    };
    {  // pxy: r faces (rows j, j+1) at theta i-1, i+2 (centred in theta)
      const int rrow = NT * (j + (NR + 1) * k);
      const V r_m1 = fr[rrow + im1], r_p2 = fr[rrow + ip2];
      const V r1_m1 = fr[rrow + NT + im1], r1_p2 = fr[rrow + NT + ip2];
      term(3, V(0.5) * (((V)o1[2] - r1_m1) / V(4.) - ((V)o1[1] - r_m1) / V(4.)),
           V(0.5) * ((r1_p2 - (V)o0[2]) / V(4.) - (r_p2 - (V)o0[1]) / V(4.)));
    }
    {  // pyx: theta faces of rows a, b
      const int tra = d.offT + NT * (ra + NR * k), trb = d.offT + NT * (rb + NR * k);
      R a0, a1, b0, b1;
      ld2(fr, tra + i, a0, a1);
      ld2(fr, trb + i, b0, b1);
      const R a2 = fr[tra + ip2], b2 = fr[trb + ip2];
      term(1, V(0.5) * (along(rlo, rhi, o0[4], a1, b1) - along(rlo, rhi, o0[3], a0, b0)),
           V(0.5) * (along(rlo, rhi, o1[4], a2, b2) - along(rlo, rhi, o1[3], a1, b1)));
    }
    {  // pxz: r faces (rows j, j+1) of planes a, b
      const int rka = NT * (j + (NR + 1) * ka), rkb = NT * (j + (NR + 1) * kb);
      R pa0, pa1, pb0, pb1, pA0, pA1, pB0, pB1;
      ld2(fr, rka + i, pa0, pa1);
      ld2(fr, rkb + i, pb0, pb1);
      ld2(fr, rka + NT + i, pA0, pA1);
      ld2(fr, rkb + NT + i, pB0, pB1);
      term(6, V(0.5) * (along(zlo, zhi, o0[2], pA0, pB0) - along(zlo, zhi, o0[1], pa0, pb0)),
           V(0.5) * (along(zlo, zhi, o1[2], pA1, pB1) - along(zlo, zhi, o1[1], pa1, pb1)));
    }
    {  // pzx: z faces (levels k, k+1) of rows a, b
      const int zra = d.offZ + NT * (ra + NR * k), zrb = d.offZ + NT * (rb + NR * k);
      R za0, za1, zb0, zb1, zA0, zA1, zB0, zB1;
      ld2(fr, zra + i, za0, za1);
      ld2(fr, zrb + i, zb0, zb1);
      ld2(fr, zra + pl + i, zA0, zA1);
      ld2(fr, zrb + pl + i, zB0, zB1);
      term(2, V(0.5) * (along(rlo, rhi, o0[6], zA0, zB0) - along(rlo, rhi, o0[5], za0, zb0)),
           V(0.5) * (along(rlo, rhi, o1[6], zA1, zB1) - along(rlo, rhi, o1[5], za1, zb1)));
    }
    {  // pyz: theta faces of planes a, b
      const int tka = d.offT + NT * (j + NR * ka), tkb = d.offT + NT * (j + NR * kb);
      R a0, a1, b0, b1;
      ld2(fr, tka + i, a0, a1);
      ld2(fr, tkb + i, b0, b1);
      const R a2 = fr[tka + ip2], b2 = fr[tkb + ip2];
      term(7, V(0.5) * (along(zlo, zhi, o0[4], a1, b1) - along(zlo, zhi, o0[3], a0, b0)),
           V(0.5) * (along(zlo, zhi, o1[4], a2, b2) - along(zlo, zhi, o1[3], a1, b1)));
    }
    {  // pzy: z faces (levels k, k+1) at theta i-1, i+2
      const int zlev = d.offZ + NT * (j + NR * k);
      const V z_m1 = fr[zlev + im1], z_p2 = fr[zlev + ip2];
      const V z1_m1 = fr[zlev + pl + im1], z1_p2 = fr[zlev + pl + ip2];
      term(5, V(0.5) * (((V)o1[6] - z1_m1) / V(4.) - ((V)o1[5] - z_m1) / V(4.)),
           V(0.5) * ((z1_p2 - (V)o0[6]) / V(4.) - (z_p2 - (V)o0[5]) / V(4.)));
    }
    const V RD0 = pv<V>(P.inv_Re, P.d_inv_Re) * s0, RD1 = pv<V>(P.inv_Re, P.d_inv_Re) * s1;
    const V B0 = (V(0.) + RD0 + RB0), B1 = (V(0.) + RD1 + RB1);
    // cell update (cell_update), term by term
    R cv0, cv1, co0, co1, a0, a1;
    ld2(F.c[q], c, cv0, cv1);
    ld2(F.co[q], c, co0, co1);
    const V w = V(P.w[q]);
    ld2(F.MF4, c, a0, a1);
    const V F40 = a0, F41 = a1;
    ld2(F.MF4 + Nc, c, a0, a1);
    V u0 = +a0 * (V)co0, u1 = +a1 * (V)co1;
#pragma unroll
    for (int m = 2; m <= 7; ++m) {
      ld2(F.MF4 + m * Nc, c, a0, a1);
      u0 = u0 + a0 * (V)o0[m - 1];
      u1 = u1 + a1 * (V)o1[m - 1];
    }
    const V nw0 = stored<R>((1 - w) * (V)cv0 + (w / F40) * (u0 + B0));
    const V nw1 = stored<R>((1 - w) * (V)cv1 + (w / F41) * (u1 + B1));
    typename Pair2<R>::T out;
    out.x = (R)nw0;
    out.y = (R)nw1;
    *reinterpret_cast<typename Pair2<R>::T *>(F.c[q] + c) = out;
    e[q] = nmax(errv(nw0, cv0, first), errv(nw1, cv1, first));
  }
  if (!SLAB || d.owns(k)) block_max<3, CB3>(red, e, ctl->err[par]);
}
template <class R, bool SLAB = false>
__global__ void __launch_bounds__(CB3, minb<R>(VC2_MINB, VC2_MINB_F)) k_vel_cell2(Dims d, GeoT<R> g, FieldsT<R> F, Phys P, Ctrl *ctl) {
  vel_cell2_body<R, SLAB>(d, g, F, P, ctl, LaunchBlock{});
}

// ---- K1, NP cells per thread: k_vel_cell2's sweep over NP theta-adjacent
// cells (i a multiple of NP), every value the NP cells share a row for in
// one NP-wide vector load (float4 for the float mirror: 16 bytes a load,
// as FP64's pairs): the cell arrays, the r and z faces, the theta faces at
// i..i+NP-1 (the +theta face of cell p is the -theta face of cell p+1) and
// the r- and z-stencil rows; single loads only for the theta-stencil ends
// (i-1, i+NP) and the +theta face of the last cell.  Each cell's terms are
// k_vel_cell's in its order.  Needs n_theta % NP == 0 (every vector
// NP-aligned); block (CB, 3) over patches of 32 NP x CB/32 cells.
template <class R, int NP>
struct VecN;
template <>
struct VecN<float, 4> {
  using T = float4;
};
template <>
struct VecN<float, 2> {
  using T = float2;
};
template <>
struct VecN<double, 2> {
  using T = double2;
};
template <class R, int NP>
__device__ __forceinline__ void ldN(const R *__restrict__ p, int i, R (&v)[NP]) {
  const typename VecN<R, NP>::T t = *reinterpret_cast<const typename VecN<R, NP>::T *>(p + i);
  const R *e = reinterpret_cast<const R *>(&t);
#pragma unroll
  for (int q = 0; q < NP; ++q) v[q] = e[q];
}
template <class R, int NP>
__device__ __forceinline__ void stN(R *__restrict__ p, int i, const R (&v)[NP]) {
  typename VecN<R, NP>::T t;
  R *e = reinterpret_cast<R *>(&t);
#pragma unroll
  for (int q = 0; q < NP; ++q) e[q] = v[q];
  *reinterpret_cast<typename VecN<R, NP>::T *>(p + i) = t;
}

template <class R, int NP, bool SLAB = false>
__global__ void __launch_bounds__(CB3, VCN_MINB) k_vel_cellN(Dims d, GeoT<R> g, FieldsT<R> F, Phys P, Ctrl *ctl) {
  using V = Ar<R>;
  if (ctl->done) return;
  __shared__ BlockRed red;
  red_init<3>(red);
  const int par = parity(ctl);
  const bool first = ctl->first;
  const int q = threadIdx.y;
  const int i = blockIdx.x * (32 * NP) + NP * (threadIdx.x & 31);
  const int j = blockIdx.y * (CB / 32) + (threadIdx.x >> 5);
  const int k = blockIdx.z;
  double e[3] = {0., 0., 0.};
  if (i < d.NT && j < d.NR) {
    const int Nc = d.Nc, NF = d.NF, NT = d.NT, NR = d.NR, pl = d.plane;
    const int c = i + NT * (j + NR * k);  // cell i; cell p of the group is c + p
    const int im1 = (i == 0) ? NT - 1 : i - 1, ipn = (i + NP >= NT) ? i + NP - NT : i + NP;
    const int f1 = c + NT * k;
    const int fi[7] = {0, f1, f1 + NT, d.offT + c, d.offT + c + 1, d.offZ + c, d.offZ + c + pl};
    const int f4b = d.offT + c - i + ipn;  // +theta face of the last cell
    // face m of the NP cells from array a
    auto faceN = [&](const R *a, int m, R (&v)[NP]) {
      if (m == 4) {
        R t[NP];
        ldN<R, NP>(a, fi[3], t);
#pragma unroll
        for (int p = 0; p + 1 < NP; ++p) v[p] = t[p + 1];
        v[NP - 1] = a[f4b];
      } else {
        ldN<R, NP>(a, fi[m], v);
      }
    };
    // RB = base + 1/rho * green_gauss (component q), faces 2, 1, 4, 3, 6, 5
    const R *pp = F.f[3] + par * NF, *nq = g.normal + q * NF;
    V gs[NP];
    {
      const int order[6] = {2, 1, 4, 3, 6, 5};
#pragma unroll
      for (int t = 0; t < 6; ++t) {
        const int m = order[t];
        R pv[NP], av[NP], nv[NP];
        faceN(pp, m, pv);
        faceN(g.area, m, av);
        faceN(nq, m, nv);
#pragma unroll
        for (int p = 0; p < NP; ++p) {
          const V tp = (V)pv[p] * av[p] * (nv[p]);
          gs[p] = (t == 0) ? tp : (t & 1) ? gs[p] - tp : gs[p] + tp;
        }
      }
    }
    V RB[NP];
    {
      R vol[NP];
      ldN<R, NP>(g.vol, c, vol);
      V base[NP];
#pragma unroll
      for (int p = 0; p < NP; ++p) base[p] = V(0.);
      if (q == 2) {
        R t[NP], o[NP];
        ldN<R, NP>(F.c[3], c, t);
        ldN<R, NP>(F.co[3], c, o);
#pragma unroll
        for (int p = 0; p < NP; ++p) base[p] = -(V(P.g_beta) * V(0.5) * (t[p] + o[p]));
      }
#pragma unroll
      for (int p = 0; p < NP; ++p) RB[p] = base[p] + V(P.inv_rho) * ((V(1.) / vol[p]) * gs[p]);
    }
    // own faces of component q (stored values)
    const R *fr = F.f[q] + par * NF;
    R o[7][NP];
#pragma unroll
    for (int m = 1; m <= 6; ++m) faceN(fr, m, o[m]);
    auto along = [&](bool lo, bool hi, V v0, V va, V vb) {
      return lo ? tang_vals(true, false, v0, va, vb, V(0.), V(0.))
                : hi ? tang_vals(false, true, v0, V(0.), V(0.), va, vb) : tang_vals(false, false, v0, vb, V(0.), va, V(0.));
    };
    const bool rlo = (j == 0), rhi = (j == NR - 1);
    const int ra = rlo ? j + 1 : j - 1, rb = rlo ? j + 2 : (rhi ? j - 2 : j + 1);
    const bool zlo = (k == 0), zhi = (k == d.NZ - 1);
    const int ka = zlo ? k + 1 : k - 1, kb = zlo ? k + 2 : (zhi ? k - 2 : k + 1);
    V s[NP];
    {
      R a[NP];
      ldN<R, NP>(g.G, c, a);
#pragma unroll
      for (int p = 0; p < NP; ++p) s[p] = a[p] * ((o[2][p] - o[1][p]) / V(2.));
      ldN<R, NP>(g.G + Nc, c, a);
#pragma unroll
      for (int p = 0; p < NP; ++p) s[p] = s[p] + a[p] * ((o[4][p] - o[3][p]) / V(2.));
      ldN<R, NP>(g.G + 2 * Nc, c, a);
#pragma unroll
      for (int p = 0; p < NP; ++p) s[p] = s[p] + a[p] * ((o[6][p] - o[5][p]) / V(2.));
    }
    auto term = [&](int slot, const V (&dv)[NP]) {
      R a[NP];
      ldN<R, NP>(g.gij + slot * Nc, c, a);
#pragma unroll
      for (int p = 0; p < NP; ++p) s[p] = s[p] - a[p] * dv[p];
    };
    {  // pxy: r faces (rows j, j+1) at theta i-1 .. i+NP (centred in theta)
      const int rrow = NT * (j + (NR + 1) * k);
      const V r_m1 = fr[rrow + im1], r_pn = fr[rrow + ipn];
      const V r1_m1 = fr[rrow + NT + im1], r1_pn = fr[rrow + NT + ipn];
      V dv[NP];
#pragma unroll
      for (int p = 0; p < NP; ++p) {
        const V up2 = (p + 1 < NP) ? (V)o[2][p + 1] : r1_pn, um2 = (p > 0) ? (V)o[2][p - 1] : r1_m1;
        const V up1 = (p + 1 < NP) ? (V)o[1][p + 1] : r_pn, um1 = (p > 0) ? (V)o[1][p - 1] : r_m1;
        dv[p] = V(0.5) * ((up2 - um2) / V(4.) - (up1 - um1) / V(4.));
      }
      term(3, dv);
    }
    {  // pyx: theta faces of rows a, b
      const int tra = d.offT + NT * (ra + NR * k), trb = d.offT + NT * (rb + NR * k);
      R av[NP + 1], bv[NP + 1];
      {
        R t[NP];
        ldN<R, NP>(fr, tra + i, t);
#pragma unroll
        for (int p = 0; p < NP; ++p) av[p] = t[p];
        ldN<R, NP>(fr, trb + i, t);
#pragma unroll
        for (int p = 0; p < NP; ++p) bv[p] = t[p];
        av[NP] = fr[tra + ipn];
        bv[NP] = fr[trb + ipn];
      }
      V dv[NP];
#pragma unroll
      for (int p = 0; p < NP; ++p)
        dv[p] = V(0.5) * (along(rlo, rhi, o[4][p], av[p + 1], bv[p + 1]) - along(rlo, rhi, o[3][p], av[p], bv[p]));
      term(1, dv);
    }
    {  // pxz: r faces (rows j, j+1) of planes a, b
      const int rka = NT * (j + (NR + 1) * ka), rkb = NT * (j + (NR + 1) * kb);
      R pa[NP], pb[NP], pA[NP], pB[NP];
      ldN<R, NP>(fr, rka + i, pa);
      ldN<R, NP>(fr, rkb + i, pb);
      ldN<R, NP>(fr, rka + NT + i, pA);
      ldN<R, NP>(fr, rkb + NT + i, pB);
      V dv[NP];
#pragma unroll
      for (int p = 0; p < NP; ++p)
        dv[p] = V(0.5) * (along(zlo, zhi, o[2][p], pA[p], pB[p]) - along(zlo, zhi, o[1][p], pa[p], pb[p]));
      term(6, dv);
    }
    {  // pzx: z faces (levels k, k+1) of rows a, b
      const int zra = d.offZ + NT * (ra + NR * k), zrb = d.offZ + NT * (rb + NR * k);
      R za[NP], zb[NP], zA[NP], zB[NP];
      ldN<R, NP>(fr, zra + i, za);
      ldN<R, NP>(fr, zrb + i, zb);
      ldN<R, NP>(fr, zra + pl + i, zA);
      ldN<R, NP>(fr, zrb + pl + i, zB);
      V dv[NP];
#pragma unroll
      for (int p = 0; p < NP; ++p)
        dv[p] = V(0.5) * (along(rlo, rhi, o[6][p], zA[p], zB[p]) - along(rlo, rhi, o[5][p], za[p], zb[p]));
      term(2, dv);
    }
    {  // pyz: theta faces of planes a, b
      const int tka = d.offT + NT * (j + NR * ka), tkb = d.offT + NT * (j + NR * kb);
      R av[NP + 1], bv[NP + 1];
      {
        R t[NP];
        ldN<R, NP>(fr, tka + i, t);
#pragma unroll
        for (int p = 0; p < NP; ++p) av[p] = t[p];
        ldN<R, NP>(fr, tkb + i, t);
#pragma unroll
        for (int p = 0; p < NP; ++p) bv[p] = t[p];
        av[NP] = fr[tka + ipn];
        bv[NP] = fr[tkb + ipn];
      }
      V dv[NP];
#pragma unroll
      for (int p = 0; p < NP; ++p)
        dv[p] = V(0.5) * (along(zlo, zhi, o[4][p], av[p + 1], bv[p + 1]) - along(zlo, zhi, o[3][p], av[p], bv[p]));
      term(7, dv);
    }
    {  // pzy: z faces (levels k, k+1) at theta i-1 .. i+NP
      const int zlev = d.offZ + NT * (j + NR * k);
      const V z_m1 = fr[zlev + im1], z_pn = fr[zlev + ipn];
      const V z1_m1 = fr[zlev + pl + im1], z1_pn = fr[zlev + pl + ipn];
      V dv[NP];
#pragma unroll
      for (int p = 0; p < NP; ++p) {
        const V up6 = (p + 1 < NP) ? (V)o[6][p + 1] : z1_pn, um6 = (p > 0) ? (V)o[6][p - 1] : z1_m1;
        const V up5 = (p + 1 < NP) ? (V)o[5][p + 1] : z_pn, um5 = (p > 0) ? (V)o[5][p - 1] : z_m1;
        dv[p] = V(0.5) * ((up6 - um6) / V(4.) - (up5 - um5) / V(4.));
      }
      term(5, dv);
    }
    // cell update (cell_update), term by term
    R cv[NP], co[NP], a[NP], F40[NP];
    ldN<R, NP>(F.c[q], c, cv);
    ldN<R, NP>(F.co[q], c, co);
    const V w = V(P.w[q]);
    ldN<R, NP>(F.MF4, c, F40);
    ldN<R, NP>(F.MF4 + Nc, c, a);
    V u[NP];
#pragma unroll
    for (int p = 0; p < NP; ++p) u[p] = +a[p] * (V)co[p];
#pragma unroll
    for (int m = 2; m <= 7; ++m) {
      ldN<R, NP>(F.MF4 + m * Nc, c, a);
#pragma unroll
      for (int p = 0; p < NP; ++p) u[p] = u[p] + a[p] * (V)o[m - 1][p];
    }
    R out[NP];
#pragma unroll
    for (int p = 0; p < NP; ++p) {
      const V B = (V(0.) + pv<V>(P.inv_Re, P.d_inv_Re) * s[p] + RB[p]);
      const V nw = stored<R>((1 - w) * (V)cv[p] + (w / F40[p]) * (u[p] + B));
      out[p] = (R)nw;
      e[q] = nmax(e[q], errv(nw, cv[p], first));
    }
    stN<R, NP>(F.c[q], c, out);
  }
  if (!SLAB || d.owns(k)) block_max<3, CB3>(red, e, ctl->err[par]);
}

// ---- K2: +xi face updates of u, v, w (nse.f90:878-1005).
// Block (CB, 3): threadIdx.y = direction.
template <class R, class BI>
__device__ __forceinline__ void vel_face_body(const Dims &d, const GeoT<R> &g, const FieldsT<R> &F, const Phys &P, Ctrl *ctl, const BI blockIdx) {
  using V = Ar<R>;
  if (ctl->done) return;
  __shared__ BlockRed red;
  red_init<3>(red);
  const int par = parity(ctl);
  const bool first = ctl->first;
  Cell x;
  const bool act = patch_cell(d, x, blockIdx);
  const int c = x.c;
  double e[3] = {0., 0., 0.};
  if (act) {
    const size_t Nc = d.Nc, NF = d.NF;
    by_dir(threadIdx.y, [&](auto D) {
      constexpr int dd = decltype(D)::value;
      if (!x.has_nb(d, 2 * dd)) return;
      const Cell x2 = x.nb(d, 2 * dd);
      V Fd[5];
      for (int k = 0; k < 5; ++k) Fd[k] = F.MF[(size_t)(5 * (dd - 1) + k) * Nc + c];
      const V dg0 = g.dg[(2 * (dd - 1)) * Nc + c], dg1 = g.dg[(2 * (dd - 1) + 1) * Nc + c];
      const int fo = x.face(d, 2 * dd);
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        const R *fr = F.f[q] + par * NF;
        const V nw = stored<R>(face_update(d, fr, F.c[q], F.co[q], Fd, dg0, dg1, dd, x, x2, V(P.w[q])));
        F.f[q][(1 - par) * NF + fo] = nw;
        e[q] = errv(nw, fr[fo], first);
      }
    });
  }
  if (d.owns(blockIdx.z)) block_max<3, CB3>(red, e, ctl->err[par]);
}
template <class R>
__global__ void __launch_bounds__(CB3, 3) k_vel_face(Dims d, GeoT<R> g, FieldsT<R> F, Phys P, Ctrl *ctl) {
  vel_face_body<R>(d, g, F, P, ctl, LaunchBlock{});
}

// ---- K2, z-marching form: the same face updates, one block per patch of
// 32 theta x VT_R r cells marching up a chunk of kc z-planes.  Every value
// the updates read arrives in shared memory by TMA box loads
// (cp.async.bulk.tensor, completion counted in bytes on an mbarrier per
// buffer): per plane p, for each velocity component, the r, theta and z
// (level p) faces of the current half and the cell and old-cell values as
// W x (VT_R + 1 or 2) boxes (the theta halo: columns i0+32, i0+33; at the
// seam those two columns are fetched with plain loads and written in after
// the box lands), in a ring of VT_S planes; and per plane the patch's
// M_F1..3 and metric-difference rows as one 32 x VT_R x 21 box pair in a
// ring of two.  Plane k is computed from ring planes k, k+1, k+2 while the
// block's other resident neighbour on the SM computes; k+3 is issued once
// plane k is done.  The arithmetic is k_vel_face's
// (face_update_vals): the results are identical.
// Needs n_theta % 4 == 0 and n_theta <= 256 (box rows of 16-byte multiples).
constexpr int VT_R = 4;         // r rows of cells per patch
constexpr int VT_T = 32 * VT_R;  // cells per patch = blockDim.x (blockDim.y = 3 directions)
constexpr int VT_S = 3;          // plane ring depth (FP64: 109 KB with the coefficient ring)
constexpr int VT_MINB = 2;       // resident blocks per SM the launch bounds ask for (FP64)
constexpr int VT_MINB_F = 3;     // float: its 57 KB ring allows 3

// tensor maps of one storage type, encoded by the host: per component the
// r / theta / z parts of the face array as {NT, rows, planes, half}, the
// cell and old-cell arrays as {NT, NR, NZ}, M_F1..3 and the metric
// differences as {NT, NR, NZ, rows}
struct VelFaceMaps {
  CUtensorMap rf[3], tf[3], zf[3], cv[3], co[3], mf, dg;
};

// shared-memory layout (elements of R; every box starts on 128 bytes)
template <class R>
struct VtLayout {
  // staged columns: 32 cells + the 2-column halo, rounded to 16-byte box rows
  static constexpr int W = sizeof(R) == 8 ? 34 : 36;
  static constexpr int up(int bytes) { return (bytes + 127) / 128 * 128 / (int)sizeof(R); }
  static constexpr int RF = up((VT_R + 2) * W * (int)sizeof(R));  // r-face box region
  static constexpr int C5 = up((VT_R + 1) * W * (int)sizeof(R));  // theta / z / cell box region
  static constexpr int Q = RF + 4 * C5;                              // one component
  static constexpr int PLANE = 3 * Q;
  static constexpr int MF = 15 * VT_R * 32, DG = 6 * VT_R * 32, COEF = MF + DG;
  static constexpr int BARS = VT_S * PLANE + 2 * COEF;  // element offset of the mbarriers
  // + 128: the kernel rounds the dynamic shared-memory base up to 128 bytes
  static constexpr size_t bytes = (size_t)BARS * sizeof(R) + (VT_S + 2) * sizeof(unsigned long long) + 128;
  static constexpr unsigned plane_tx = 3u * ((VT_R + 2) + 4 * (VT_R + 1)) * W * sizeof(R);
  static constexpr unsigned zlevel_tx = 3u * (VT_R + 1) * W * sizeof(R);
  static constexpr unsigned coef_tx = (unsigned)(COEF * sizeof(R));
};

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z,
                                            unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, int x, int y, int z, int w,
                                            unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
      "%5}], [%6];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(w), "r"(smem_u32(bar))
      : "memory");
}

// plane bundle p (one thread): levels p of the z faces and, for p < NZ, the
// r and theta faces and the cell values of plane p
template <class R>
__device__ void vt_issue_plane(const VelFaceMaps &M, R *slot, unsigned long long *bar, int i0, int j0, int p,
                               int par, int NZ) {
  using L = VtLayout<R>;
  const bool cells = p < NZ;
  mbar_expect_tx(bar, cells ? L::plane_tx : L::zlevel_tx);
  for (int q = 0; q < 3; ++q) {
    R *b = slot + q * L::Q;
    tma_load_4d(b + L::RF + L::C5, &M.zf[q], i0, j0, p, par, bar);
    if (!cells) continue;
    tma_load_4d(b, &M.rf[q], i0, j0, p, par, bar);
    tma_load_4d(b + L::RF, &M.tf[q], i0, j0, p, par, bar);
    tma_load_3d(b + L::RF + 2 * L::C5, &M.cv[q], i0, j0, p, bar);
    tma_load_3d(b + L::RF + 3 * L::C5, &M.co[q], i0, j0, p, bar);
  }
}
template <class R>
__device__ void vt_issue_coef(const VelFaceMaps &M, R *coef, unsigned long long *bar, int i0, int j0, int p) {
  using L = VtLayout<R>;
  mbar_expect_tx(bar, L::coef_tx);
  tma_load_4d(coef, &M.mf, i0, j0, p, 0, bar);
  tma_load_4d(coef + L::MF, &M.dg, i0, j0, p, 0, bar);
}

// the theta-seam columns of plane bundle p: value u (< 3 x 2 x row slots) of the
// patch at the seam, global source and ring position; false if u names a
// row outside the mesh or an array the bundle does not hold
template <class R>
__device__ __forceinline__ bool vt_seam(const Dims &d, const FieldsT<R> &F, int par, int i0, int j0, int ncell, int p,
                                        int u, const R *&src, int &dst) {
  using L = VtLayout<R>;
  constexpr int per_q = 2 * (VT_R + 2 + 4 * (VT_R + 1));  // 2 columns x row slots
  const int q = u / per_q, r = u - q * per_q, col = r & 1, k = r >> 1;
  int kind, row;
  if (k < VT_R + 2) {
    kind = 0;
    row = k;
  } else {
    kind = 1 + (k - (VT_R + 2)) / (VT_R + 1);
    row = (k - (VT_R + 2)) % (VT_R + 1);
  }
  const int j = j0 + row;
  if (kind == 0 ? j > d.NR : j > d.NR - 1) return false;
  if (p >= d.NZ && kind != 2) return false;  // top level: z faces only
  const size_t NT = d.NT, NR = d.NR;
  const R *fq = F.f[q] + (size_t)par * d.NF;
  switch (kind) {
    case 0: src = fq + NT * (j + (NR + 1) * p) + col; break;
    case 1: src = fq + d.offT + NT * (j + NR * p) + col; break;
    case 2: src = fq + d.offZ + NT * (j + NR * p) + col; break;
    case 3: src = F.c[q] + NT * (j + NR * p) + col; break;
    default: src = F.co[q] + NT * (j + NR * p) + col; break;
  }
  const int base = q * L::Q + (kind == 0 ? 0 : L::RF + (kind - 1) * L::C5);
  dst = base + row * L::W + ncell + col;
  return true;
}

// SLAB: a z-slab context, whose maxima skip the planes a neighbour owns
template <class R, bool SLAB = false>
__global__ void __launch_bounds__(3 * VT_T, minb<R>(VT_MINB, VT_MINB_F))
    k_vel_face_tile(Dims d, GeoT<R> g, FieldsT<R> F, Phys P, Ctrl *ctl, int kc, const __grid_constant__ VelFaceMaps M) {
  using V = Ar<R>;
  using L = VtLayout<R>;
  if (ctl->done) return;
  extern __shared__ __align__(128) unsigned char vt_raw[];
  R *ring = reinterpret_cast<R *>(vt_raw + ((128u - (smem_u32(vt_raw) & 127u)) & 127u));
  R *coefs = ring + VT_S * L::PLANE;
  unsigned long long *bar_pl = reinterpret_cast<unsigned long long *>(ring + L::BARS);
  unsigned long long *bar_cf = bar_pl + VT_S;
  __shared__ BlockRed red;
  const int tid = threadIdx.x + VT_T * threadIdx.y;
  const int i0 = blockIdx.x * 32, j0 = blockIdx.y * VT_R;
  const int ncell = min(32, d.NT - i0);
  const bool seam = d.NT - i0 <= 32;  // columns ncell, ncell+1 wrap to theta 0, 1
  const int par = parity(ctl);
  const bool first = ctl->first;
  const int kb = blockIdx.z * kc, ke = min(kb + kc, d.NZ);
  const int nplanes = min(ke + 2, d.NZ + 1) - kb;  // plane bundles kb .. kb+nplanes-1
  const int ncoef = ke - kb;
  if (tid == 0) {
    for (int s = 0; s < VT_S + 2; ++s) mbar_init(&bar_pl[s], 1);
  }
  red_init<3>(red);  // barrier: the mbarriers exist before any copy
  if (tid == 0) {
    for (int l = 0; l < VT_S && l < nplanes; ++l)
      vt_issue_plane(M, ring + l * L::PLANE, &bar_pl[l], i0, j0, kb + l, par, d.NZ);
    for (int l = 0; l < 2 && l < ncoef; ++l) vt_issue_coef(M, coefs + l * L::COEF, &bar_cf[l], i0, j0, kb + l);
  }
  const int ii = threadIdx.x & 31, jj = threadIdx.x >> 5;
  const bool act = ii < ncell && j0 + jj < d.NR;
  const size_t NF = d.NF;
  double e[3] = {0., 0., 0.};
  bool ok = true;
  for (int l = 0; l < ncoef; ++l) {
    const int k = kb + l;
    // bundles that become readable now: 0, 1, 2 at the start, then l + 2
    const int m0 = (l == 0) ? 0 : l + 2, m1 = min(l + 2, nplanes - 1);
    R seamv[3];
    int seamd[3];
    bool have[3] = {false, false, false};
    if (seam && tid < 3 * 2 * (VT_R + 2 + 4 * (VT_R + 1))) {
      for (int m = m0; m <= m1; ++m) {
        const R *src;
        int dst;
        if (vt_seam(d, F, par, i0, j0, ncell, kb + m, tid, src, dst)) {
          have[m - m0] = true;
          seamv[m - m0] = *src;
          seamd[m - m0] = (m % VT_S) * L::PLANE + dst;
        }
      }
    }
    bool mine = true;
    for (int m = m0; m <= m1; ++m) mine = mine && mbar_wait(&bar_pl[m % VT_S], (m / VT_S) & 1, ctl);
    mine = mine && mbar_wait(&bar_cf[l & 1], (l >> 1) & 1, ctl);
    if (mine && seam) {
      for (int n = 0; n < 3; ++n)
        if (have[n]) ring[seamd[n]] = seamv[n];
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // before later boxes into this slot
    }
    if (!__syncthreads_and(mine)) {  // the same decision in every thread
      ok = false;
      break;
    }
    if (act) {
      const Cell x = Cell::at(d, i0 + ii, j0 + jj, k);
      const R *P0 = ring + (l % VT_S) * L::PLANE, *P1 = ring + ((l + 1) % VT_S) * L::PLANE;
      const R *P2 = ring + ((l + 2) % VT_S) * L::PLANE;
      const R *C = coefs + (l & 1) * L::COEF;
      by_dir(threadIdx.y, [&](auto D) {
        constexpr int dd = decltype(D)::value;
        if (!x.has_nb(d, 2 * dd)) return;
        V Fd[5];
        for (int kq = 0; kq < 5; ++kq) Fd[kq] = C[(5 * (dd - 1) + kq) * VT_R * 32 + jj * 32 + ii];
        const V dg0 = C[L::MF + (2 * (dd - 1)) * VT_R * 32 + jj * 32 + ii];
        const V dg1 = C[L::MF + (2 * (dd - 1) + 1) * VT_R * 32 + jj * 32 + ii];
        // x2 = x + e_dd sits at (ii + di, jj + dj) of plane Q0
        constexpr int di = (dd == 2), dj = (dd == 1);
        const R *Q0 = (dd == 3) ? P1 : P0, *Q1 = (dd == 3) ? P2 : P1;
        const int fo = x.face(d, 2 * dd);
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          // face pos of the cell at (a, b) of plane A (B: the plane above)
          auto face = [&](const R *A, const R *B, int a, int b, int pos) -> V {
            const R *qa = A + q * L::Q, *qb = B + q * L::Q;
            switch (pos) {
              case 1: return qa[b * L::W + a];
              case 2: return qa[(b + 1) * L::W + a];
              case 3: return qa[L::RF + b * L::W + a];
              case 4: return qa[L::RF + b * L::W + a + 1];
              case 5: return qa[L::RF + L::C5 + b * L::W + a];
              default: return qb[L::RF + L::C5 + b * L::W + a];
            }
          };
          auto fx = [&](int pos) { return face(P0, P1, ii, jj, pos); };
          auto fx2 = [&](int pos) { return face(Q0, Q1, ii + di, jj + dj, pos); };
          const R *cq0 = P0 + q * L::Q + L::RF + 2 * L::C5, *cq2 = Q0 + q * L::Q + L::RF + 2 * L::C5;
          const V nw = stored<R>(face_update_vals(
              fx, fx2, cq0[jj * L::W + ii], cq2[(jj + dj) * L::W + ii + di], cq0[L::C5 + jj * L::W + ii],
              cq2[L::C5 + (jj + dj) * L::W + ii + di], Fd, dg0, dg1, dd, V(P.w[q])));
          F.f[q][(1 - par) * NF + fo] = nw;
          if (!SLAB || d.owns(k)) e[q] = nmax(e[q], errv(nw, fx(2 * dd), first));
        }
      });
    }
    __syncthreads();  // every thread is done with ring plane l and coefficient buffer l & 1
    if (tid == 0) {
      if (l + VT_S < nplanes)
        vt_issue_plane(M, ring + (l % VT_S) * L::PLANE, &bar_pl[l % VT_S], i0, j0, kb + l + VT_S, par, d.NZ);
      if (l + 2 < ncoef) vt_issue_coef(M, coefs + (l & 1) * L::COEF, &bar_cf[l & 1], i0, j0, kb + l + 2);
    }
  }
  if (!ok) {
    // a wait ran out: let the copies already issued land (bounded) before
    // the block leaves; waiting on both parities covers the pending phase
    for (int s = 0; s < VT_S + 2; ++s) {
      mbar_wait(&bar_pl[s], 0, ctl);
      mbar_wait(&bar_pl[s], 1, ctl);
    }
    return;
  }
  block_max<3, 3 * VT_T>(red, e, ctl->err[par]);
}

// ---- K1, tiled form (parallel schedule, formulation 2): k_vel_cell with the
// face values of u, v, w its stencils read staged in shared memory by TMA
// boxes.  One block per patch of 32 theta x CT_R r cells marches up a chunk
// of z-planes; per plane p, for each component, three boxes of W columns
// from i0-OFF (OFF = 16 bytes of elements, so the box's x coordinate stays
// 16-byte aligned; the theta halo on both sides): r faces, rows j0 .. j0+CT_R;
// theta faces and z faces of level p, rows j0-2 .. j0+CT_R+1 (the two-cell
// one-sided wall stencils in r).  A ring of CT_S bundles holds planes k-2 ..
// k+2 (the one-sided stencils in z) and one in flight.  Pressure faces,
// geometry, M_F4 and the cell values stay direct loads (each read once).
// The theta-seam columns (theta NT-1 left of the first patch, theta 0 right
// of the last) are fetched with plain loads and written in after the box
// lands.  The arithmetic is k_vel_cell's, term for term.
constexpr int CT_R = 4;          // r rows of cells per patch
constexpr int CT_T = 32 * CT_R;  // cells per patch = blockDim.x (blockDim.y = 3 components)
constexpr int CT_S = 6;          // bundle ring depth
constexpr int CT_MINB = 2;       // resident blocks per SM the launch bounds ask for

struct VelCellMaps {
  CUtensorMap rf[3], tf[3], zf[3];
};

template <class R>
struct CtLayout {
  static constexpr int OFF = 16 / (int)sizeof(R);                  // columns left of i0 (2 or 4)
  static constexpr int W = (32 + OFF + 2 + 3) / 4 * 4;             // 36 (double) or 40 (float) columns
  static constexpr int up(int bytes) { return (bytes + 127) / 128 * 128 / (int)sizeof(R); }
  static constexpr int RF = up((CT_R + 1) * W * (int)sizeof(R));  // r-face box region
  static constexpr int TZ = up((CT_R + 4) * W * (int)sizeof(R));  // theta / z box region
  static constexpr int Q = RF + 2 * TZ;                             // one component
  static constexpr int BUNDLE = 3 * Q;
  static constexpr int BARS = CT_S * BUNDLE;
  static constexpr size_t bytes = (size_t)BARS * sizeof(R) + CT_S * sizeof(unsigned long long) + 128;
  static constexpr unsigned full_tx = 3u * ((CT_R + 1) + 2 * (CT_R + 4)) * W * sizeof(R);
  static constexpr unsigned top_tx = 3u * (CT_R + 4) * W * sizeof(R);  // z level NZ only
  static constexpr int SEAM_L = 3 * ((CT_R + 1) + (CT_R + 4));          // r and z rows, column OFF-1
  static constexpr int SEAM_R = 3 * ((CT_R + 1) + 2 * (CT_R + 4));      // r, theta, z rows, column ncell+OFF
};

template <class R>
__device__ void ct_issue(const VelCellMaps &M, R *slot, unsigned long long *bar, int i0, int j0, int p, int par,
                         int NZ) {
  using L = CtLayout<R>;
  const bool cells = p < NZ;
  mbar_expect_tx(bar, cells ? L::full_tx : L::top_tx);
  for (int q = 0; q < 3; ++q) {
    R *b = slot + q * L::Q;
    tma_load_4d(b + L::RF + L::TZ, &M.zf[q], i0 - L::OFF, j0 - 2, p, par, bar);
    if (!cells) continue;
    tma_load_4d(b, &M.rf[q], i0 - L::OFF, j0, p, par, bar);
    tma_load_4d(b + L::RF, &M.tf[q], i0 - L::OFF, j0 - 2, p, par, bar);
  }
}

// seam value u of bundle p: global source and position in the bundle;
// false if u names nothing (no seam on that side, a row outside the mesh,
// or an array the bundle does not hold)
template <class R>
__device__ __forceinline__ bool ct_seam(const Dims &d, const FieldsT<R> &F, int par, int i0, int j0, int ncell,
                                        bool left, bool right, int p, int u, const R *&src, int &dst) {
  using L = CtLayout<R>;
  int q, r, kind, col, ti;  // kind 0 r faces, 1 theta faces, 2 z faces
  if (u < L::SEAM_L) {
    if (!left) return false;
    q = u / (L::SEAM_L / 3);
    r = u - q * (L::SEAM_L / 3);
    kind = (r < CT_R + 1) ? 0 : 2;
    if (kind == 2) r -= CT_R + 1;
    col = L::OFF - 1;
    ti = d.NT - 1;
  } else {
    if (!right) return false;
    u -= L::SEAM_L;
    q = u / (L::SEAM_R / 3);
    r = u - q * (L::SEAM_R / 3);
    if (r < CT_R + 1) {
      kind = 0;
    } else if (r < CT_R + 1 + CT_R + 4) {
      kind = 1;
      r -= CT_R + 1;
    } else {
      kind = 2;
      r -= CT_R + 1 + CT_R + 4;
    }
    col = ncell + L::OFF;
    ti = 0;
  }
  const int j = (kind == 0) ? j0 + r : j0 - 2 + r;
  if (kind == 0 ? (j > d.NR) : (j < 0 || j > d.NR - 1)) return false;
  if (p >= d.NZ && kind != 2) return false;
  const size_t NT = d.NT, NR = d.NR;
  const R *fq = F.f[q] + (size_t)par * d.NF;
  switch (kind) {
    case 0: src = fq + NT * (j + (NR + 1) * p) + ti; break;
    case 1: src = fq + d.offT + NT * (j + NR * p) + ti; break;
    default: src = fq + d.offZ + NT * (j + NR * p) + ti; break;
  }
  dst = q * L::Q + (kind == 0 ? 0 : kind == 1 ? L::RF : L::RF + L::TZ) + r * L::W + col;
  return true;
}

template <class R>
__global__ void __launch_bounds__(3 * CT_T, CT_MINB)
    k_vel_cell_tile(Dims d, GeoT<R> g, FieldsT<R> F, Phys P, Ctrl *ctl, int kc, const __grid_constant__ VelCellMaps M) {
  using V = Ar<R>;
  using L = CtLayout<R>;
  if (ctl->done) return;
  extern __shared__ __align__(128) unsigned char ct_raw[];
  R *ring = reinterpret_cast<R *>(ct_raw + ((128u - (smem_u32(ct_raw) & 127u)) & 127u));
  unsigned long long *bar = reinterpret_cast<unsigned long long *>(ring + L::BARS);
  __shared__ BlockRed red;
  const int tid = threadIdx.x + CT_T * threadIdx.y;
  const int q = threadIdx.y;
  const int i0 = blockIdx.x * 32, j0 = blockIdx.y * CT_R;
  const int ncell = min(32, d.NT - i0);
  const bool left = (i0 == 0), right = (d.NT - i0 <= 32);
  const int par = parity(ctl);
  const bool first = ctl->first;
  const int kb = blockIdx.z * kc, ke = min(kb + kc, d.NZ);
  const int P0 = max(kb - 2, 0), P1 = min(ke + 1, d.NZ);  // bundles P0 .. P1
  const int nb = P1 - P0 + 1;
  if (tid == 0)
    for (int s = 0; s < CT_S; ++s) mbar_init(&bar[s], 1);
  red_init<3>(red);  // barrier: the mbarriers exist before any copy
  int issued = 0;    // bundles issued so far (the same count in every thread)
  for (; issued < nb && issued < CT_S; ++issued)
    if (tid == 0) ct_issue(M, ring + issued * L::BUNDLE, &bar[issued], i0, j0, P0 + issued, par, d.NZ);
  const int ii = threadIdx.x & 31, jj = threadIdx.x >> 5;
  const bool act = ii < ncell && j0 + jj < d.NR;
  const size_t Nc = d.Nc, NF = d.NF;
  double e[3] = {0., 0., 0.};
  bool ok = true;
  int waited = 0;  // bundles 0 .. waited-1 have landed
  for (int k = kb; k < ke; ++k) {
    const int need = min(k + 2, d.NZ) - P0;  // highest bundle plane k reads
    // seam values of the bundles that become readable now (at most 5)
    R seamv[5];
    int seamd[5];
    bool have[5] = {false, false, false, false, false};
    if ((left || right) && tid < L::SEAM_L + L::SEAM_R) {
      for (int b = waited; b <= need; ++b) {
        const R *src;
        int dst;
        if (ct_seam(d, F, par, i0, j0, ncell, left, right, P0 + b, tid, src, dst)) {
          have[b - waited] = true;
          seamv[b - waited] = *src;
          seamd[b - waited] = (b % CT_S) * L::BUNDLE + dst;
        }
      }
    }
    bool mine = true;
    for (int b = waited; b <= need; ++b) mine = mine && mbar_wait(&bar[b % CT_S], (b / CT_S) & 1, ctl);
    if (mine && (left || right)) {
      for (int n = 0; n < 5; ++n)
        if (have[n]) ring[seamd[n]] = seamv[n];
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // before later boxes into these slots
    }
    waited = need + 1;
    if (!__syncthreads_and(mine)) {  // the same decision in every thread
      ok = false;
      break;
    }
    if (act) {
      const Cell x = Cell::at(d, i0 + ii, j0 + jj, k);
      const int c = x.c;
      int f[7];
      cell_faces(d, x, f);
      const R *fp = F.f[3] + par * NF;
      V pf[7];
      for (int m = 1; m <= 6; ++m) pf[m] = fp[f[m]];
      const V invV = V(1.) / g.vol[c];
      const V base = (q == 2) ? -(V(P.g_beta) * V(0.5) * (F.c[3][c] + F.co[3][c])) : V(0.);
      const V RB = base + V(P.inv_rho) * green_gauss(g, NF, invV, pf, f, q);
      // face pos of the cell (di, dj, dk) away, component q, from the ring
      auto fv = [&](int pos, int di, int dj, int dk) -> V {
        const int pb = k + dk + (pos == 6 ? 1 : 0) - P0;
        const R *b = ring + (pb % CT_S) * L::BUNDLE + q * L::Q;
        const int col = ii + di + L::OFF + (pos == 4 ? 1 : 0);
        switch (pos) {
          case 1: return b[(jj + dj) * L::W + col];
          case 2: return b[(jj + dj + 1) * L::W + col];
          case 3:
          case 4: return b[L::RF + (jj + dj + 2) * L::W + col];
          default: return b[L::RF + L::TZ + (jj + dj + 2) * L::W + col];
        }
      };
      // tangential(): centred, or one-sided at the walls, along e
      auto tng = [&](int pos, int e) -> V {
        auto at = [&](int s) { return fv(pos, e == 2 ? s : 0, e == 1 ? s : 0, e == 3 ? s : 0); };
        const bool lo = !x.has_nb(d, 2 * e - 1), hi = !x.has_nb(d, 2 * e);
        if (lo) return (-(3 * at(0)) + 4 * at(1) - at(2)) / V(4.);
        if (hi) return (3 * at(0) - 4 * at(-1) + at(-2)) / V(4.);
        return (at(1) - at(-1)) / V(4.);
      };
      const V pxy = V(0.5) * (tng(2, 2) - tng(1, 2));
      const V pzy = V(0.5) * (tng(6, 2) - tng(5, 2));
      const V pyx = V(0.5) * (tng(4, 1) - tng(3, 1));
      const V pzx = V(0.5) * (tng(6, 1) - tng(5, 1));
      const V pxz = V(0.5) * (tng(2, 3) - tng(1, 3));
      const V pyz = V(0.5) * (tng(4, 3) - tng(3, 3));
      R fr[7];  // the stored values: the differences below are taken in R, as in diffusion_source
      for (int m = 1; m <= 6; ++m) fr[m] = (R)fv(m, 0, 0, 0);
      const V px = (fr[2] - fr[1]) / V(2.);
      const V py = (fr[4] - fr[3]) / V(2.);
      const V pz = (fr[6] - fr[5]) / V(2.);
      const R *G = g.G, *gij = g.gij;
      const V RD =
          pv<V>(P.inv_Re, P.d_inv_Re) * (G[c] * px + G[Nc + c] * py + G[2 * Nc + c] * pz - gij[3 * Nc + c] * pxy -
                      gij[1 * Nc + c] * pyx - gij[6 * Nc + c] * pxz - gij[2 * Nc + c] * pzx - gij[7 * Nc + c] * pyz -
                      gij[5 * Nc + c] * pzy);
      const V B = (V(0.) + RD + RB);
      const V cv = F.c[q][c], cold = F.co[q][c], w = V(P.w[q]);
      V F4[8];
      for (int m = 0; m < 8; ++m) F4[m] = F.MF4[(size_t)m * Nc + c];
      const V nw = stored<R>((1 - w) * cv + (w / F4[0]) * (+F4[1] * cold + F4[2] * fr[1] + F4[3] * fr[2] +
                                                                  F4[4] * fr[3] + F4[5] * fr[4] + F4[6] * fr[5] +
                                                                  F4[7] * fr[6] + B));
      F.c[q][c] = nw;
      e[q] = nmax(e[q], errv(nw, cv, first));
    }
    __syncthreads();  // every thread is done with the bundles plane k+1 no longer reads
    const int low = max(k + 1 - 2, 0) - P0;  // lowest bundle plane k+1 reads
    for (; issued < nb && issued - CT_S < low; ++issued)
      if (tid == 0)
        ct_issue(M, ring + (issued % CT_S) * L::BUNDLE, &bar[issued % CT_S], i0, j0, P0 + issued, par, d.NZ);
  }
  if (!ok) {
    for (int s = 0; s < CT_S; ++s) {  // bounded: let the copies in flight land
      mbar_wait(&bar[s], 0, ctl);
      mbar_wait(&bar[s], 1, ctl);
    }
    return;
  }
  block_max<3, 3 * CT_T>(red, e, ctl->err[par]);
}

// ---- K3: pressure sources (calculate_R_b_p nse.f90:2362-2407,
// calculate_R_D_p2 1863-1997).  Block (CB, 3): thread y forms the gradient of
// velocity component y and two of the six cross derivatives of p (y = 1 also
// d(bz)/dz); thread 0 combines them in the reference's order.
template <class R, class BI>
__device__ __forceinline__ void p_src_body(const Dims &d, const GeoT<R> &g, const FieldsT<R> &F, const Phys &P, Ctrl *ctl, const BI blockIdx) {
  if (ctl->done) return;
  using A = Ar<R>;
  __shared__ A sh[3][3][CB];  // gradients of u, v, w
  __shared__ A sX[3][2][CB];  // cross derivatives of p
  __shared__ A sbz[CB];
  const int par = parity(ctl);
  const int q = threadIdx.y, tx = threadIdx.x;
  Cell x;
  const bool active = patch_cell(d, x, blockIdx);
  const int c = x.c;
  int f[7];
  const size_t Nc = d.Nc, NF = d.NF;
  const R *fp = F.f[3] + par * NF;
  if (active) {
    cell_faces(d, x, f);
    by_dir(threadIdx.y, [&](auto Q) {
      constexpr int q = decltype(Q)::value - 1;
      const A invV = inv_vol(g, c);
      const R *fq = F.f[q] + newhalf(ctl) * NF;
      A vf[7];
      for (int k = 1; k <= 6; ++k) vf[k] = fq[f[k]];
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) sh[q][cc][tx] = green_gauss(g, NF, invV, vf, f, cc);
      if (q == 1) {
        const R *fT = F.f[4] + par * NF;
        A bzf[7];
        for (int k = 1; k <= 6; ++k) bzf[k] = -(A(P.g_beta) * (fT[f[k]]));
        sbz[tx] = green_gauss(g, NF, invV, bzf, f, 2);
      }
      // y=0 pxy,pzy  y=1 pyx,pzx  y=2 pxz,pyz (calculate_R_D_p2 order)
      constexpr int e2 = (q == 0) ? 2 : (q == 1) ? 1 : 3;
      constexpr int fa = (q == 1) ? 4 : 2, fb = (q == 1) ? 3 : 1;
      sX[q][0][tx] = A(0.5) * (tangential(d, fp, x, fa, e2) - tangential(d, fp, x, fb, e2));
      sX[q][1][tx] = (q == 2) ? A(0.5) * (tangential(d, fp, x, 4, 3) - tangential(d, fp, x, 3, 3))
                              : A(0.5) * (tangential(d, fp, x, 6, e2) - tangential(d, fp, x, 5, e2));
    });
  }
  __syncthreads();
  if (active && q == 0) {
    const A du_dx = sh[0][0][tx], du_dy = sh[0][1][tx], du_dz = sh[0][2][tx];
    const A dv_dx = sh[1][0][tx], dv_dy = sh[1][1][tx], dv_dz = sh[1][2][tx];
    const A dw_dx = sh[2][0][tx], dw_dy = sh[2][1][tx], dw_dz = sh[2][2][tx];
    const A dbz_dz = sbz[tx];
    const A Dila = du_dx + dv_dy + dw_dz;
    F.dila[c] = Dila;
    const A RBp = -(du_dx * du_dx + dv_dy * dv_dy + dw_dz * dw_dz) -
                  A(2) * (du_dy * dv_dx + dv_dz * dw_dy + dw_dx * du_dz) - dbz_dz + Dila / (2 * A(P.DT));
    const A pxy = sX[0][0][tx], pzy = sX[0][1][tx], pyx = sX[1][0][tx], pzx = sX[1][1][tx];
    const A pxz = sX[2][0][tx], pyz = sX[2][1][tx];
    const A px = (fp[f[2]] - fp[f[1]]) / A(2);
    const A py = (fp[f[4]] - fp[f[3]]) / A(2);
    const A pz = (fp[f[6]] - fp[f[5]]) / A(2);
    const R *Gv = g.G, *gij = g.gij;
    const A RDp = A(P.inv_rho) * (Gv[c] * px + Gv[Nc + c] * py + Gv[2 * Nc + c] * pz - gij[3 * Nc + c] * pxy -
                                    gij[1 * Nc + c] * pyx - gij[6 * Nc + c] * pxz - gij[2 * Nc + c] * pzx -
                                    gij[7 * Nc + c] * pyz - gij[5 * Nc + c] * pzy);
    F.Rp[c] = RDp + RBp;
  }
}
template <class R>
__global__ void __launch_bounds__(CB3, minb<R>(4, PSRC_MINB_F)) k_p_src(Dims d, GeoT<R> g, FieldsT<R> F, Phys P, Ctrl *ctl) {
  p_src_body<R>(d, g, F, P, ctl, LaunchBlock{});
}

// ---- K3, NP cells per thread (the float mirror with NP = 4, the FP64 path
// with NP = 2; n_theta % NP == 0):
// k_p_src over NP theta-adjacent cells, every value the cells share a row
// for in one NP-wide vector load (as k_vel_cellN).  Thread y forms the
// gradients of velocity component y (y = 1 also d(bz)/dz) and two of the six
// cross derivatives of p for the NP cells; thread 0 combines them in the
// reference's order.  Each cell's arithmetic is k_p_src's.
template <class R, int NP, class BI>
__device__ __forceinline__ void p_srcN_body(const Dims &d, const GeoT<R> &g, const FieldsT<R> &F, const Phys &P, Ctrl *ctl, const BI blockIdx) {
  using V = Ar<R>;
  if (ctl->done) return;
  __shared__ V sh[3][3][CB * NP];  // gradients of u, v, w
  __shared__ V sX[3][2][CB * NP];  // cross derivatives of p
  __shared__ V sbz[CB * NP];
  const int par = parity(ctl);
  const int tx = threadIdx.x;
  int i, j;
  group_cell<NP>(d, blockIdx, i, j);
  const int k = blockIdx.z;
  const bool active = i < d.NT && j < d.NR;
  const int Nc = d.Nc, NF = d.NF, NT = d.NT, NR = d.NR, pl = d.plane;
  const int c = i + NT * (j + NR * k);
  const int im1 = (i == 0) ? NT - 1 : i - 1, ipn = (i + NP >= NT) ? i + NP - NT : i + NP;
  const int f1 = c + NT * k;
  const int fi[7] = {0, f1, f1 + NT, d.offT + c, d.offT + c + 1, d.offZ + c, d.offZ + c + pl};
  const int f4b = d.offT + c - i + ipn;
  auto faceN = [&](const R *a, int m, R (&v)[NP]) {
    if (m == 4) {
      R t[NP];
      ldN<R, NP>(a, fi[3], t);
#pragma unroll
      for (int p = 0; p + 1 < NP; ++p) v[p] = t[p + 1];
      v[NP - 1] = a[f4b];
    } else {
      ldN<R, NP>(a, fi[m], v);
    }
  };
  const R *fp = F.f[3] + par * NF;
  auto along = [&](bool lo, bool hi, V v0, V va, V vb) {
    return lo ? tang_vals(true, false, v0, va, vb, V(0.), V(0.))
              : hi ? tang_vals(false, true, v0, V(0.), V(0.), va, vb) : tang_vals(false, false, v0, vb, V(0.), va, V(0.));
  };
  if (active) by_dir(threadIdx.y, [&](auto Q) {
    constexpr int q = decltype(Q)::value - 1;
    R vol[NP];
    V invV[NP];
    ldN<R, NP>(g.rvol, c, vol);  // 1/vol
#pragma unroll
    for (int p = 0; p < NP; ++p) invV[p] = vol[p];
    // green_gauss (terms of faces 2, 1, 4, 3, 6, 5, then the volume factor)
    auto gauss = [&](const R (&phi)[7][NP], int cc, V (&out)[NP]) {
      const R *nc = g.normal + (size_t)cc * NF;
      const int order[6] = {2, 1, 4, 3, 6, 5};
#pragma unroll
      for (int t = 0; t < 6; ++t) {
        const int m = order[t];
        R a[NP], n[NP];
        faceN(g.area, m, a);
        faceN(nc, m, n);
#pragma unroll
        for (int p = 0; p < NP; ++p) {
          const V tp = (V)phi[m][p] * a[p] * (n[p]);
          out[p] = (t == 0) ? tp : (t & 1) ? out[p] - tp : out[p] + tp;
        }
      }
#pragma unroll
      for (int p = 0; p < NP; ++p) out[p] = invV[p] * out[p];
    };
    {
      const R *fq = F.f[q] + newhalf(ctl) * NF;
      R vf[7][NP];
#pragma unroll
      for (int m = 1; m <= 6; ++m) faceN(fq, m, vf[m]);
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) {
        V gg[NP];
        gauss(vf, cc, gg);
#pragma unroll
        for (int p = 0; p < NP; ++p) sh[q][cc][tx * NP + p] = gg[p];
      }
    }
    if (q == 1) {
      const R *fT = F.f[4] + par * NF;
      R bzf[7][NP];
#pragma unroll
      for (int m = 1; m <= 6; ++m) {
        R t[NP];
        faceN(fT, m, t);
#pragma unroll
        for (int p = 0; p < NP; ++p) bzf[m][p] = -(pv<V>(P.g_beta, 0.) * (t[p]));
      }
      V gz[NP];
      gauss(bzf, 2, gz);
#pragma unroll
      for (int p = 0; p < NP; ++p) sbz[tx * NP + p] = gz[p];
    }
    // p's faces of the NP cells
    R o[7][NP];
#pragma unroll
    for (int m = 1; m <= 6; ++m) faceN(fp, m, o[m]);
    const bool rlo = (j == 0), rhi = (j == NR - 1);
    const int ra = rlo ? j + 1 : j - 1, rb = rlo ? j + 2 : (rhi ? j - 2 : j + 1);
    const bool zlo = (k == 0), zhi = (k == d.NZ - 1);
    const int ka = zlo ? k + 1 : k - 1, kb = zlo ? k + 2 : (zhi ? k - 2 : k + 1);
    if (q == 0) {  // pxy (r faces along theta), pzy (z faces along theta)
      const int rrow = NT * (j + (NR + 1) * k), zlev = d.offZ + NT * (j + NR * k);
      const V r_m1 = fp[rrow + im1], r_pn = fp[rrow + ipn], r1_m1 = fp[rrow + NT + im1], r1_pn = fp[rrow + NT + ipn];
      const V z_m1 = fp[zlev + im1], z_pn = fp[zlev + ipn], z1_m1 = fp[zlev + pl + im1], z1_pn = fp[zlev + pl + ipn];
#pragma unroll
      for (int p = 0; p < NP; ++p) {
        const V up2 = (p + 1 < NP) ? (V)o[2][p + 1] : r1_pn, um2 = (p > 0) ? (V)o[2][p - 1] : r1_m1;
        const V up1 = (p + 1 < NP) ? (V)o[1][p + 1] : r_pn, um1 = (p > 0) ? (V)o[1][p - 1] : r_m1;
        sX[0][0][tx * NP + p] = V(0.5) * ((up2 - um2) / V(4.) - (up1 - um1) / V(4.));
        const V up6 = (p + 1 < NP) ? (V)o[6][p + 1] : z1_pn, um6 = (p > 0) ? (V)o[6][p - 1] : z1_m1;
        const V up5 = (p + 1 < NP) ? (V)o[5][p + 1] : z_pn, um5 = (p > 0) ? (V)o[5][p - 1] : z_m1;
        sX[0][1][tx * NP + p] = V(0.5) * ((up6 - um6) / V(4.) - (up5 - um5) / V(4.));
      }
    } else if (q == 1) {  // pyx (theta faces along r), pzx (z faces along r)
      const int tra = d.offT + NT * (ra + NR * k), trb = d.offT + NT * (rb + NR * k);
      const int zra = d.offZ + NT * (ra + NR * k), zrb = d.offZ + NT * (rb + NR * k);
      R av[NP + 1], bv[NP + 1];
      {
        R t[NP];
        ldN<R, NP>(fp, tra + i, t);
#pragma unroll
        for (int p = 0; p < NP; ++p) av[p] = t[p];
        ldN<R, NP>(fp, trb + i, t);
#pragma unroll
        for (int p = 0; p < NP; ++p) bv[p] = t[p];
        av[NP] = fp[tra + ipn];
        bv[NP] = fp[trb + ipn];
      }
      R za[NP], zb[NP], zA[NP], zB[NP];
      ldN<R, NP>(fp, zra + i, za);
      ldN<R, NP>(fp, zrb + i, zb);
      ldN<R, NP>(fp, zra + pl + i, zA);
      ldN<R, NP>(fp, zrb + pl + i, zB);
#pragma unroll
      for (int p = 0; p < NP; ++p) {
        sX[1][0][tx * NP + p] =
            V(0.5) * (along(rlo, rhi, o[4][p], av[p + 1], bv[p + 1]) - along(rlo, rhi, o[3][p], av[p], bv[p]));
        sX[1][1][tx * NP + p] =
            V(0.5) * (along(rlo, rhi, o[6][p], zA[p], zB[p]) - along(rlo, rhi, o[5][p], za[p], zb[p]));
      }
    } else {  // pxz (r faces along z), pyz (theta faces along z)
      const int rka = NT * (j + (NR + 1) * ka), rkb = NT * (j + (NR + 1) * kb);
      const int tka = d.offT + NT * (j + NR * ka), tkb = d.offT + NT * (j + NR * kb);
      R pa[NP], pb[NP], pA[NP], pB[NP];
      ldN<R, NP>(fp, rka + i, pa);
      ldN<R, NP>(fp, rkb + i, pb);
      ldN<R, NP>(fp, rka + NT + i, pA);
      ldN<R, NP>(fp, rkb + NT + i, pB);
      R av[NP + 1], bv[NP + 1];
      {
        R t[NP];
        ldN<R, NP>(fp, tka + i, t);
#pragma unroll
        for (int p = 0; p < NP; ++p) av[p] = t[p];
        ldN<R, NP>(fp, tkb + i, t);
#pragma unroll
        for (int p = 0; p < NP; ++p) bv[p] = t[p];
        av[NP] = fp[tka + ipn];
        bv[NP] = fp[tkb + ipn];
      }
#pragma unroll
      for (int p = 0; p < NP; ++p) {
        sX[2][0][tx * NP + p] =
            V(0.5) * (along(zlo, zhi, o[2][p], pA[p], pB[p]) - along(zlo, zhi, o[1][p], pa[p], pb[p]));
        sX[2][1][tx * NP + p] =
            V(0.5) * (along(zlo, zhi, o[4][p], av[p + 1], bv[p + 1]) - along(zlo, zhi, o[3][p], av[p], bv[p]));
      }
    }
  });
  __syncthreads();
  if (active && threadIdx.y == 0) {
    R o[7][NP];
#pragma unroll
    for (int m = 1; m <= 6; ++m) faceN(fp, m, o[m]);
    R G0[NP], G1[NP], G2[NP];
    ldN<R, NP>(g.G, c, G0);
    ldN<R, NP>(g.G + Nc, c, G1);
    ldN<R, NP>(g.G + 2 * Nc, c, G2);
    R dila[NP], rp[NP];
    const int slot[6] = {3, 1, 6, 2, 7, 5};
    R gs[6][NP];
#pragma unroll
    for (int s = 0; s < 6; ++s) ldN<R, NP>(g.gij + slot[s] * Nc, c, gs[s]);
#pragma unroll
    for (int p = 0; p < NP; ++p) {
      const int e = tx * NP + p;
      const V du_dx = sh[0][0][e], du_dy = sh[0][1][e], du_dz = sh[0][2][e];
      const V dv_dx = sh[1][0][e], dv_dy = sh[1][1][e], dv_dz = sh[1][2][e];
      const V dw_dx = sh[2][0][e], dw_dy = sh[2][1][e], dw_dz = sh[2][2][e];
      const V dbz_dz = sbz[e];
      const V Dila = du_dx + dv_dy + dw_dz;
      dila[p] = Dila;
      const V RBp = -(du_dx * du_dx + dv_dy * dv_dy + dw_dz * dw_dz) -
                    V(2) * (du_dy * dv_dx + dv_dz * dw_dy + dw_dx * du_dz) - dbz_dz + Dila / (2 * V(P.DT));
      const V pxy = sX[0][0][e], pzy = sX[0][1][e], pyx = sX[1][0][e], pzx = sX[1][1][e];
      const V pxz = sX[2][0][e], pyz = sX[2][1][e];
      const V px = (o[2][p] - o[1][p]) / V(2);
      const V py = (o[4][p] - o[3][p]) / V(2);
      const V pz = (o[6][p] - o[5][p]) / V(2);
      const V RDp = V(P.inv_rho) * (G0[p] * px + G1[p] * py + G2[p] * pz - gs[0][p] * pxy - gs[1][p] * pyx -
                                    gs[2][p] * pxz - gs[3][p] * pzx - gs[4][p] * pyz - gs[5][p] * pzy);
      rp[p] = RDp + RBp;
    }
    stN<R, NP>(F.dila, c, dila);
    stN<R, NP>(F.Rp, c, rp);
  }
}
template <class R, int NP>
__global__ void __launch_bounds__(CB3, PSN_MINB) k_p_srcN(Dims d, GeoT<R> g, FieldsT<R> F, Phys P, Ctrl *ctl) {
  p_srcN_body<R, NP>(d, g, F, P, ctl, LaunchBlock{});
}

// ---- apply_pressure_bc for wall face b (bc.f90:148-339): the new value
// from the pressures pr, the new velocities fu/fv/fwv and the temperatures fT
template <class Ld, class R>
__device__ __forceinline__ Ar<R> p_bc_value(const Dims &d, const GeoT<R> &g, const FieldsT<R> &F, const Phys &P,
                                            const R *pr, const R *fu, const R *fv, const R *fwv, const R *fT,
                                            int b) {
  using V = Ar<R>;
  const int NF = d.NF, NB = d.NBF;
  const BFace B = bface(d, b);
  const Cell M1 = B.cell;
  const int pos = B.pos;
  const int fw0 = M1.face(d, pos);
  const V n[3] = {g.normal[fw0], g.normal[NF + fw0], g.normal[2 * NF + fw0]};
  const V bvec[3] = {V(0), V(0), -(V(P.g_beta) * (fT[fw0]))};
  const V b_n = dot3(bvec, n);
  V vn[6];
  for (int j = 1; j <= 5; ++j) {
    const int pt = g.bcpts[(j - 1) * NB + b];
    const V v[3] = {fu[pt], fv[pt], fwv[pt]};
    vn[j] = dot3(v, n);
  }
  const R *a = g.bca;
  const V d2udn2 = -(a[b] * vn[1]) - a[NB + b] * vn[2] - a[2 * NB + b] * vn[3] - a[3 * NB + b] * vn[4] -
                        a[4 * NB + b] * vn[5];
  const int dd = (pos + 1) / 2;
  const V B2 = tangential<Ld>(d, pr, M1, pos, tr1(dd)) * g.bcg[b];
  const V B3 = tangential<Ld>(d, pr, M1, pos, tr2(dd)) * g.bcg[NB + b];
  const R *ap = g.bcap;
  const V B1 = ap[7 * NB + b] * (F.Rp[M1.c]);
  V s = 0.0;
  bool firstterm = true;
  for (int k = 1; k <= 6; ++k) {
    if (k == pos) continue;
    const V t = ap[(k - 1) * NB + b] * Ld::ld(pr, M1.face(d, k));
    s = firstterm ? -t : s - t;
    firstterm = false;
  }
  const V w = V(P.w_p2);
  return (1 - w) * Ld::ld(pr, fw0) +
         w / (ap[(pos - 1) * NB + b]) * (s + B1 - B2 - B3 + (pv<V>(P.nu, P.d_nu) * V(P.rho) * d2udn2 - b_n * V(P.rho)));
}

// ---- K4: apply_pressure_bc, every wall face from the values before the pass
template <class R, class BI>
__device__ __forceinline__ void p_bc_body(const Dims &d, const GeoT<R> &g, const FieldsT<R> &F, const Phys &P, Ctrl *ctl, const BI blockIdx) {
  if (ctl->done) return;
  __shared__ BlockRed red;
  red_init<1>(red);
  const int par = parity(ctl), nh = newhalf(ctl);
  const bool first = ctl->first;
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  double e[1] = {0.};
  if (b < d.NBF) {
    const int NF = d.NF;
    const R *pr = F.f[3] + par * NF;
    const Ar<R> nw = stored<R>(p_bc_value<LdPlain>(d, g, F, P, pr, F.f[0] + nh * NF, F.f[1] + nh * NF,
                                                   F.f[2] + nh * NF, F.f[4] + par * NF, b));
    const BFace B = bface(d, b);
    const int fw0 = B.cell.face(d, B.pos);
    F.f[3][(1 - par) * NF + fw0] = nw;
    e[0] = d.owns(B.cell.k) ? errv(nw, pr[fw0], first) : 0.;
  }
  block_max<1>(red, e, ctl->err[par] + 3);
}
template <class R>
__global__ void __launch_bounds__(BLK) k_p_bc(Dims d, GeoT<R> g, FieldsT<R> F, Phys P, Ctrl *ctl) {
  p_bc_body<R>(d, g, F, P, ctl, LaunchBlock{});
}

template <class R, class BI>
__device__ __forceinline__ void p_bc_copy_body(const Dims &d, const FieldsT<R> &F, Ctrl *ctl, const BI blockIdx) {
  if (ctl->done) return;
  const int par = parity(ctl);
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= d.NBF) return;
  const BFace B = bface(d, b);
  const int f = B.cell.face(d, B.pos);
  F.f[3][par * d.NF + f] = F.f[3][(1 - par) * d.NF + f];
}
template <class R>
__global__ void k_p_bc_copy(Dims d, FieldsT<R> F, Ctrl *ctl) {
  p_bc_copy_body<R>(d, F, ctl, LaunchBlock{});
}

// (coefficient, face, cell) of the ten off-diagonal terms of the pressure
// face update for the +r, +theta, +z face (dd = 1, 2, 3), in source order
// (nse.f90:1150-1285), packed as coefficient | face << 4 | cell << 7.  A
// constexpr switch: with dd and t known at compile time it folds to
// constants.
__host__ __device__ constexpr int p_term(int dd, int t) {
  switch (10 * dd + t) {
    case 10: return 1 | 1 << 4 | 1 << 7; case 11: return 3 | 2 << 4 | 2 << 7; case 12: return 4 | 3 << 4 | 1 << 7; case 13: return 5 | 4 << 4 | 1 << 7; case 14: return 6 | 3 << 4 | 2 << 7;
    case 15: return 7 | 4 << 4 | 2 << 7; case 16: return 8 | 5 << 4 | 1 << 7; case 17: return 9 | 6 << 4 | 1 << 7; case 18: return 10 | 5 << 4 | 2 << 7; case 19: return 11 | 6 << 4 | 2 << 7;
    case 20: return 1 | 1 << 4 | 1 << 7; case 21: return 2 | 2 << 4 | 1 << 7; case 22: return 3 | 1 << 4 | 2 << 7; case 23: return 4 | 2 << 4 | 2 << 7; case 24: return 5 | 3 << 4 | 1 << 7;
    case 25: return 7 | 4 << 4 | 2 << 7; case 26: return 8 | 5 << 4 | 1 << 7; case 27: return 9 | 6 << 4 | 1 << 7; case 28: return 10 | 5 << 4 | 2 << 7; case 29: return 11 | 6 << 4 | 2 << 7;
    case 30: return 1 | 1 << 4 | 1 << 7; case 31: return 2 | 2 << 4 | 1 << 7; case 32: return 3 | 1 << 4 | 2 << 7; case 33: return 4 | 2 << 4 | 2 << 7; case 34: return 5 | 3 << 4 | 1 << 7;
    case 35: return 6 | 4 << 4 | 1 << 7; case 36: return 7 | 3 << 4 | 2 << 7; case 37: return 8 | 4 << 4 | 2 << 7; case 38: return 9 | 5 << 4 | 1 << 7; case 39: return 11 | 6 << 4 | 2 << 7;
    default: return 0;
  }
}

// ---- integrate_pressure_field_i for the +xi_dd face of cell x
// (nse.f90:1091-1289): the new value from the pressures pr
template <class Ld, class R>
__device__ __forceinline__ Ar<R> p_face_value(const Dims &d, const GeoT<R> &g, const FieldsT<R> &F, const Phys &P,
                                              const R *pr, const Cell &x, int dd) {
  using V = Ar<R>;
  const size_t Nc = d.Nc;
  const int c = x.c;
  const int diag = (dd == 1) ? 2 : (dd == 2) ? 6 : 10;
  const Cell n2 = x.nb(d, 2 * dd);
  const R *A = g.AA + (size_t)15 * (dd - 1) * Nc;
  const V B1 = (F.Rp[c]) * A[12 * Nc + c];
  const V B2 = (F.Rp[n2.c]) * A[14 * Nc + c];
  const V B3 = (g.dg[(2 * (dd - 1)) * Nc + c]) * tangential<Ld>(d, pr, x, 2 * dd, tr1(dd));
  const V B4 = (g.dg[(2 * (dd - 1) + 1) * Nc + c]) * tangential<Ld>(d, pr, x, 2 * dd, tr2(dd));
  V s = 0.0;
#pragma unroll
  for (int t = 0; t < 10; ++t) {
    const int pt = p_term(dd, t), coef = pt & 15, fpos = (pt >> 4) & 7, cell = pt >> 7;
    const Cell &cl = (cell == 1) ? x : n2;
    const V term = A[(size_t)(coef - 1) * Nc + c] * Ld::ld(pr, cl.face(d, fpos));
    s = (t == 0) ? -term : s - term;
  }
  const int fo = x.face(d, 2 * dd);
  const V w = V(P.w_p);
  return (1 - w) * Ld::ld(pr, fo) + w / (A[(size_t)(diag - 1) * Nc + c]) * (s + B1 + B2 + B3 + B4);
}

// ---- integrate_velocity_field_i for the +xi_dd face of cell x, one
// component (nse.f90:378-826): the pressure sweep's ten face terms with
// AA_v, the two cell time terms, the R sums Bq of both cells and the
// tangential cross terms (the centred B3/B4 the source forms first are
// overwritten before use).  fr faces, cv / co cells and old cells.
template <class Ld, class R>
__device__ __forceinline__ Ar<R> v1_face_value(const Dims &d, const GeoT<R> &g, const FieldsT<R> &F, const Phys &P,
                                               const R *fr, const R *cv, const R *co, const R *Bq, const Cell &x,
                                               int dd, Ar<R> w) {
  using V = Ar<R>;
  const size_t Nc = d.Nc;
  const int c = x.c;
  const Cell n2 = x.nb(d, 2 * dd);
  const R *A = F.AAv + (size_t)15 * (dd - 1) * Nc;
  const V B1 = Bq[c] * A[12 * Nc + c] * 2 * V(P.DT);
  const V B2 = Bq[n2.c] * A[14 * Nc + c] * 2 * V(P.DT);
  const V B3 = (g.dg[(2 * (dd - 1)) * Nc + c]) * tangential<Ld>(d, fr, x, 2 * dd, tr1(dd));
  const V B4 = (g.dg[(2 * (dd - 1) + 1) * Nc + c]) * tangential<Ld>(d, fr, x, 2 * dd, tr2(dd));
  V s = V(0.0);
#pragma unroll
  for (int t = 0; t < 10; ++t) {
    const int pt = p_term(dd, t), coef = pt & 15, fpos = (pt >> 4) & 7, cell = pt >> 7;
    const Cell &cl = (cell == 1) ? x : n2;
    const V term = A[(size_t)(coef - 1) * Nc + c] * Ld::ld(fr, cl.face(d, fpos));
    s = (t == 0) ? -term : s - term;
  }
  s = s - A[11 * Nc + c] * (Ld::ld(cv, c) - co[c]) - A[13 * Nc + c] * (Ld::ld(cv, n2.c) - co[n2.c]);
  const int diag = (dd == 1) ? 2 : (dd == 2) ? 6 : 10;
  return (1 - w) * Ld::ld(fr, x.face(d, 2 * dd)) + w / (A[(size_t)(diag - 1) * Nc + c]) * (s + B1 + B2 + B3 + B4);
}

// ---- K2 of formulation 1: +xi face updates of u, v, w (nse.f90:378-826),
// cur -> next.  Block (CB, 3): threadIdx.y = direction.
template <class R>
__global__ void __launch_bounds__(CB3, 2) k_vel1_face(Dims d, GeoT<R> g, FieldsT<R> F, Phys P, Ctrl *ctl) {
  using V = Ar<R>;
  if (ctl->done) return;
  __shared__ BlockRed red;
  red_init<3>(red);
  const int par = parity(ctl);
  const bool first = ctl->first;
  Cell x;
  const bool act = patch_cell(d, x);
  double e[3] = {0., 0., 0.};
  if (act) {
    const size_t Nc = d.Nc, NF = d.NF;
    by_dir(threadIdx.y, [&](auto D) {
      constexpr int dd = decltype(D)::value;
      if (!x.has_nb(d, 2 * dd)) return;
      const int fo = x.face(d, 2 * dd);
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        const R *fr = F.f[q] + par * NF;
        const V nw = stored<R>(
            v1_face_value<LdPlain>(d, g, F, P, fr, F.c[q], F.co[q], F.Bv + (size_t)q * Nc, x, dd, V(P.w[q])));
        F.f[q][(1 - par) * NF + fo] = nw;
        e[q] = errv(nw, fr[fo], first);
      }
    });
  }
  if (d.owns(blockIdx.z)) block_max<3, CB3>(red, e, ctl->err[par]);
}

// ---- K5: integrate_pressure_field_i, cur -> next.
// Block (CB, 3): threadIdx.y = direction.
template <class R, class BI>
__device__ __forceinline__ void p_face_body(const Dims &d, const GeoT<R> &g, const FieldsT<R> &F, const Phys &P, Ctrl *ctl, const BI blockIdx) {
  if (ctl->done) return;
  __shared__ BlockRed red;
  red_init<1>(red);
  const int par = parity(ctl);
  const bool first = ctl->first;
  Cell x;
  const bool act = patch_cell(d, x, blockIdx);
  double e[1] = {0.};
  if (act) {
    by_dir(threadIdx.y, [&](auto D) {
      constexpr int dd = decltype(D)::value;
      if (!x.has_nb(d, 2 * dd)) return;
      const size_t NF = d.NF;
      const R *pr = F.f[3] + par * NF;
      const Ar<R> nw = stored<R>(p_face_value<LdPlain>(d, g, F, P, pr, x, dd));
      const int fo = x.face(d, 2 * dd);
      F.f[3][(1 - par) * NF + fo] = nw;
      e[0] = errv(nw, pr[fo], first);
    });
  }
  if (d.owns(blockIdx.z)) block_max<1, CB3>(red, e, ctl->err[par] + 3);
}
template <class R>
__global__ void __launch_bounds__(CB3, minb<R>(5, PFACE_MINB_F)) k_p_face(Dims d, GeoT<R> g, FieldsT<R> F, Phys P, Ctrl *ctl) {
  p_face_body<R>(d, g, F, P, ctl, LaunchBlock{});
}

// ---- K5, NP cells per thread (the float mirror with NP = 4, the FP64 path
// with NP = 2; n_theta % NP == 0):
// k_p_face over NP theta-adjacent cells.  Thread y updates the +xi face of
// direction y+1 of the NP cells from NP-wide vector loads: the faces of the
// cells and of their +neighbours (for theta the group's own vectors shifted
// by one cell, plus single loads for the last cell's neighbour), AA, R_p and
// the metric differences; the theta faces' new values are stored one by one
// (they start one cell off the vector boundary).  Each face's arithmetic is
// p_face_value's.
template <class R, int NP, class BI>
__device__ __forceinline__ void p_faceN_body(const Dims &d, const GeoT<R> &g, const FieldsT<R> &F, const Phys &P, Ctrl *ctl, const BI blockIdx) {
  using V = Ar<R>;
  if (ctl->done) return;
  __shared__ BlockRed red;
  red_init<1>(red);
  const int par = parity(ctl);
  const bool first = ctl->first;
  const int tx = threadIdx.x;
  int i, j;
  group_cell<NP>(d, blockIdx, i, j);
  const int k = blockIdx.z;
  double e[1] = {0.};
  if (i < d.NT && j < d.NR) by_dir(threadIdx.y, [&](auto D) {
    constexpr int dd = decltype(D)::value;
    const int Nc = d.Nc, NF = d.NF, NT = d.NT, NR = d.NR, pl = d.plane;
    if ((dd == 1 && j == NR - 1) || (dd == 3 && k == d.NZ - 1)) return;  // a wall face: apply_pressure_bc's
    const int c = i + NT * (j + NR * k);
    const int im1 = (i == 0) ? NT - 1 : i - 1, ipn = (i + NP >= NT) ? i + NP - NT : i + NP;
    const R *pr = F.f[3] + par * NF;
    // faces 1..6 of the NP cells starting at (i, jj, kk) (face 4: the +theta
    // face of cell p is the -theta face of cell p+1)
    auto group = [&](int jj, int kk, R (&v)[7][NP]) {
      const int cc = i + NT * (jj + NR * kk), ff = cc + NT * kk;
      ldN<R, NP>(pr, ff, v[1]);
      ldN<R, NP>(pr, ff + NT, v[2]);
      R t[NP];
      ldN<R, NP>(pr, d.offT + cc, t);
#pragma unroll
      for (int p = 0; p < NP; ++p) v[3][p] = t[p];
#pragma unroll
      for (int p = 0; p + 1 < NP; ++p) v[4][p] = t[p + 1];
      v[4][NP - 1] = pr[d.offT + cc - i + ipn];
      ldN<R, NP>(pr, d.offZ + cc, v[5]);
      ldN<R, NP>(pr, d.offZ + cc + pl, v[6]);
    };
    R ox[7][NP], on[7][NP];
    group(j, k, ox);
    if (dd == 1) {
      group(j + 1, k, on);
    } else if (dd == 3) {
      group(j, k + 1, on);
    } else {  // the +theta neighbours: cells i+1 .. i+NP
      const int cw = c - i + ipn;  // the last cell's neighbour
      const int iw = (ipn == NT - 1) ? 0 : ipn + 1;
#pragma unroll
      for (int p = 0; p + 1 < NP; ++p) {
        on[1][p] = ox[1][p + 1];
        on[2][p] = ox[2][p + 1];
        on[4][p] = ox[4][p + 1];
        on[5][p] = ox[5][p + 1];
        on[6][p] = ox[6][p + 1];
      }
#pragma unroll
      for (int p = 0; p < NP; ++p) on[3][p] = ox[4][p];
      on[1][NP - 1] = pr[cw + NT * k];
      on[2][NP - 1] = pr[cw + NT * k + NT];
      on[4][NP - 1] = pr[d.offT + cw - ipn + iw];
      on[5][NP - 1] = pr[d.offZ + cw];
      on[6][NP - 1] = pr[d.offZ + cw + pl];
    }
    const R *A = g.AA + (size_t)15 * (dd - 1) * Nc;
    constexpr int diag = (dd == 1) ? 2 : (dd == 2) ? 6 : 10;
    // the ten off-diagonal terms, in source order
    V s[NP];
#pragma unroll
    for (int t = 0; t < 10; ++t) {
      const int pt = p_term(dd, t), coef = pt & 15, fpos = (pt >> 4) & 7, cell = pt >> 7;
      R a[NP];
      ldN<R, NP>(A + (size_t)(coef - 1) * Nc, c, a);
#pragma unroll
      for (int p = 0; p < NP; ++p) {
        const V term = a[p] * (V)((cell == 1) ? ox[fpos][p] : on[fpos][p]);
        s[p] = (t == 0) ? -term : s[p] - term;
      }
    }
    // R_p of the cells and of their +neighbours
    R rp[NP], rn[NP], a12[NP], a14[NP], ad[NP], dg0[NP], dg1[NP];
    ldN<R, NP>(F.Rp, c, rp);
    if (dd == 2) {
#pragma unroll
      for (int p = 0; p + 1 < NP; ++p) rn[p] = rp[p + 1];
      rn[NP - 1] = F.Rp[c - i + ipn];
    } else {
      ldN<R, NP>(F.Rp, c + (dd == 1 ? NT : pl), rn);
    }
    ldN<R, NP>(A + 12 * (size_t)Nc, c, a12);
    ldN<R, NP>(A + 14 * (size_t)Nc, c, a14);
    ldN<R, NP>(A + (size_t)(diag - 1) * Nc, c, ad);
    ldN<R, NP>(g.dg + (size_t)(2 * (dd - 1)) * Nc, c, dg0);
    ldN<R, NP>(g.dg + (size_t)(2 * (dd - 1) + 1) * Nc, c, dg1);
    // tangential derivatives of face 2dd along tr1(dd) and tr2(dd)
    V t1[NP], t2[NP];
    const bool rlo = (j == 0), rhi = (j == NR - 1);
    const int ra = rlo ? j + 1 : j - 1, rb = rlo ? j + 2 : (rhi ? j - 2 : j + 1);
    const bool zlo = (k == 0), zhi = (k == d.NZ - 1);
    const int ka = zlo ? k + 1 : k - 1, kb = zlo ? k + 2 : (zhi ? k - 2 : k + 1);
    auto along = [&](bool lo, bool hi, V v0, V va, V vb) {
      return lo ? tang_vals(true, false, v0, va, vb, V(0.), V(0.))
                : hi ? tang_vals(false, true, v0, V(0.), V(0.), va, vb) : tang_vals(false, false, v0, vb, V(0.), va, V(0.));
    };
    if (dd == 1) {  // face 2 (r faces of row j+1): along theta (centred), along z
      const int rrow = NT * (j + 1 + (NR + 1) * k);
      const V m1 = pr[rrow + im1], pn = pr[rrow + ipn];
      R za[NP], zb[NP];
      ldN<R, NP>(pr, NT * (j + 1 + (NR + 1) * ka) + i, za);
      ldN<R, NP>(pr, NT * (j + 1 + (NR + 1) * kb) + i, zb);
#pragma unroll
      for (int p = 0; p < NP; ++p) {
        const V up = (p + 1 < NP) ? (V)ox[2][p + 1] : pn, um = (p > 0) ? (V)ox[2][p - 1] : m1;
        t1[p] = (up - um) / V(4.);
        t2[p] = along(zlo, zhi, ox[2][p], za[p], zb[p]);
      }
    } else if (dd == 2) {  // face 4 (theta faces at i+1 ..): along r, along z
      const int tra = d.offT + NT * (ra + NR * k), trb = d.offT + NT * (rb + NR * k);
      const int tka = d.offT + NT * (j + NR * ka), tkb = d.offT + NT * (j + NR * kb);
      R av[NP + 1], bv[NP + 1], ca[NP + 1], cb[NP + 1];
      {
        R t[NP];
        ldN<R, NP>(pr, tra + i, t);
#pragma unroll
        for (int p = 0; p < NP; ++p) av[p] = t[p];
        ldN<R, NP>(pr, trb + i, t);
#pragma unroll
        for (int p = 0; p < NP; ++p) bv[p] = t[p];
        ldN<R, NP>(pr, tka + i, t);
#pragma unroll
        for (int p = 0; p < NP; ++p) ca[p] = t[p];
        ldN<R, NP>(pr, tkb + i, t);
#pragma unroll
        for (int p = 0; p < NP; ++p) cb[p] = t[p];
        av[NP] = pr[tra + ipn];
        bv[NP] = pr[trb + ipn];
        ca[NP] = pr[tka + ipn];
        cb[NP] = pr[tkb + ipn];
      }
#pragma unroll
      for (int p = 0; p < NP; ++p) {
        t1[p] = along(rlo, rhi, ox[4][p], av[p + 1], bv[p + 1]);
        t2[p] = along(zlo, zhi, ox[4][p], ca[p + 1], cb[p + 1]);
      }
    } else {  // face 6 (z faces of level k+1): along r, along theta (centred)
      const int zra = d.offZ + NT * (ra + NR * k) + pl, zrb = d.offZ + NT * (rb + NR * k) + pl;
      const int zlev = d.offZ + NT * (j + NR * k) + pl;
      R za[NP], zb[NP];
      ldN<R, NP>(pr, zra + i, za);
      ldN<R, NP>(pr, zrb + i, zb);
      const V m1 = pr[zlev + im1], pn = pr[zlev + ipn];
#pragma unroll
      for (int p = 0; p < NP; ++p) {
        t1[p] = along(rlo, rhi, ox[6][p], za[p], zb[p]);
        const V up = (p + 1 < NP) ? (V)ox[6][p + 1] : pn, um = (p > 0) ? (V)ox[6][p - 1] : m1;
        t2[p] = (up - um) / V(4.);
      }
    }
    const V w = V(P.w_p);
    R out[NP];
#pragma unroll
    for (int p = 0; p < NP; ++p) {
      const V B1 = (rp[p]) * a12[p];
      const V B2 = (rn[p]) * a14[p];
      const V B3 = (dg0[p]) * t1[p];
      const V B4 = (dg1[p]) * t2[p];
      const V old = ox[2 * dd][p];
      const V nw = stored<R>((1 - w) * old + w / (ad[p]) * (s[p] + B1 + B2 + B3 + B4));
      out[p] = (R)nw;
      e[0] = nmax(e[0], errv(nw, old, first));
    }
    R *dst = F.f[3] + (1 - par) * NF;
    if (dd == 2) {
#pragma unroll
      for (int p = 0; p + 1 < NP; ++p) dst[d.offT + c + p + 1] = out[p];
      dst[d.offT + c - i + ipn] = out[NP - 1];
    } else {
      const int f1 = c + NT * k;
      stN<R, NP>(dst, dd == 1 ? f1 + NT : d.offZ + c + pl, out);
    }
  });
  if (d.owns(blockIdx.z)) block_max<1, CB3>(red, e, ctl->err[par] + 3);
}
template <class R, int NP>
__global__ void __launch_bounds__(CB3, PFN_MINB) k_p_faceN(Dims d, GeoT<R> g, FieldsT<R> F, Phys P, Ctrl *ctl) {
  p_faceN_body<R, NP>(d, g, F, P, ctl, LaunchBlock{});
}

// ---- K5b (is_dpdx_tolerance): cell pressure gradients (nse.f90:292-307)
template <class R, class BI>
__device__ __forceinline__ void p_dpdx_body(const Dims &d, const GeoT<R> &g, const FieldsT<R> &F, Ctrl *ctl, const BI blockIdx) {
  if (ctl->done) return;
  __shared__ BlockRed red;
  red_init<1>(red);
  const int par = parity(ctl);
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  double e[1] = {0.};
  if (c < d.Nc) {
    const Cell x = Cell::of(d, c);
    const size_t Nc = d.Nc, NF = d.NF;
    int f[7];
    cell_faces(d, x, f);
    const R *p = F.f[3] + newhalf(ctl) * NF;
    using V = Ar<R>;
    const V v[3] = {stored<R>((p[f[2]] - p[f[1]]) / V(2.) * g.xi[0 * Nc + c]),
                    stored<R>((p[f[4]] - p[f[3]]) / V(2.) * g.xi[4 * Nc + c]),
                    stored<R>((p[f[6]] - p[f[5]]) / V(2.) * g.xi[8 * Nc + c])};
    for (int q = 0; q < 3; ++q) {
      if (d.owns(x.k)) e[0] = nmax(e[0], fabs(val(v[q]) - val(F.dpd[q * Nc + c])));
      F.dpd[q * Nc + c] = v[q];
    }
  }
  block_max<1>(red, e, ctl->err[par] + 5);
}
template <class R>
__global__ void __launch_bounds__(BLK) k_p_dpdx(Dims d, GeoT<R> g, FieldsT<R> F, Ctrl *ctl) {
  p_dpdx_body<R>(d, g, F, ctl, LaunchBlock{});
}

// ---- K6: apply_zero_flux (bc.f90:345-390) on the z walls, in place
template <class R, class BI>
__device__ __forceinline__ void zero_flux_body(const Dims &d, const GeoT<R> &g, const FieldsT<R> &F, Ctrl *ctl, const BI blockIdx) {
  if (ctl->done) return;
  __shared__ BlockRed red;
  red_init<1>(red);
  const int par = parity(ctl);
  const bool first = ctl->first;
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  double e[1] = {0.};
  if (b < 2 * d.plane) {
    const int NF = d.NF, NB = d.NBF;
    const BFace B = bface(d, b);
    const int in = (B.pos == 5) ? 6 : 5;
    const Cell c2 = B.cell.nb(d, in), c3 = c2.nb(d, in);
    R *T = F.f[4] + par * NF;
    const int f1 = B.cell.face(d, B.pos);
    const Ar<R> nw = stored<R>((+g.zf[NB + b] * T[B.cell.face(d, in)] - g.zf[2 * NB + b] * T[c2.face(d, in)] +
                                g.zf[3 * NB + b] * T[c3.face(d, in)]) / g.zf[b]);
    e[0] = d.owns(B.cell.k) ? errv(nw, T[f1], first) : 0.;
    T[f1] = nw;
  }
  block_max<1>(red, e, ctl->err[par] + 4);
}
template <class R>
__global__ void __launch_bounds__(BLK) k_zero_flux(Dims d, GeoT<R> g, FieldsT<R> F, Ctrl *ctl) {
  zero_flux_body<R>(d, g, F, ctl, LaunchBlock{});
}

// ---- K7a: calculate_temperature_nim_constants_formulation2, first part
// (nim.f90:334-464): MT_A(1:6) of every cell and direction, from the cell
// velocities of this pass.  One thread per (direction, cell) and no
// barriers: in FP64 the divisions of the NIM series make this the one
// instruction-bound piece of the pass, and every warp can issue.
// Grid (3, ceil(Nc/BLK)): blockIdx.x is the direction, so the three
// directions of the same cells run side by side and share their loads.
// The float instantiation (the FP32 phase) computes in float with
// nim_direction_f32, which makes it bound by its bytes.
template <class R, class BI>
__device__ __forceinline__ void T_coef_body(const Dims &d, const GeoT<R> &g, const FieldsT<R> &F, const Phys &P, Ctrl *ctl, const BI blockIdx) {
  if (ctl->done) return;
  const int c = blockIdx.y * BLK + threadIdx.x;
  if (c >= d.Nc) return;
  const int dd = blockIdx.x + 1;
  const int Nc = d.Nc;
  if constexpr (std::is_same<R, float>::value) {
    const float ut = 0.5f * (F.c[0][c] + F.co[0][c]);
    const float vt = 0.5f * (F.c[1][c] + F.co[1][c]);
    const float wt = 0.5f * (F.c[2][c] + F.co[2][c]);
    const float u = ut * g.xi[(dd - 1) * Nc + c] + vt * g.xi[(dd + 2) * Nc + c] + wt * g.xi[(dd + 5) * Nc + c];
    float A[6];
    nim_direction_f32(u, g.gij[(dd - 1 + 3 * (dd - 1)) * Nc + c] * (float)P.alpha, g.gfd[(2 * (dd - 1)) * Nc + c],
                      g.gfd[(2 * (dd - 1) + 1) * Nc + c], A);
    A[4] = 1.f / A[4];  // k_T_cell, the one reader, only divides by A4 (A4 = 4h/k > 0)
    for (int q = 0; q < 6; ++q) F.MTA[(3 * q + dd - 1) * Nc + c] = A[q];
  } else {
    using V = Ar<R>;
    const V ut = V(0.5) * (F.c[0][c] + F.co[0][c]);
    const V vt = V(0.5) * (F.c[1][c] + F.co[1][c]);
    const V wt = V(0.5) * (F.c[2][c] + F.co[2][c]);
    const V u = contravariant(g.xi, Nc, c, dd, ut, vt, wt);
    V A[6];
    nim_direction<V>(u, g.gij[(dd - 1 + 3 * (dd - 1)) * Nc + c] * pv<V>(P.alpha, P.d_alpha),
                     g.gfd[(2 * (dd - 1)) * Nc + c], g.gfd[(2 * (dd - 1) + 1) * Nc + c], P.v_limit, A);
    for (int q = 0; q < 6; ++q) F.MTA[(3 * q + dd - 1) * Nc + c] = A[q];
  }
}
template <class R>
__global__ void __launch_bounds__(BLK, 4) k_T_coef(Dims d, GeoT<R> g, FieldsT<R> F, Phys P, Ctrl *ctl) {
  T_coef_body<R>(d, g, F, P, ctl, LaunchBlock{});
}

// ---- K7b: the rest of calculate_temperature_nim_constants_formulation2
// (MT_F4, MT_F1..3, nim.f90:466-500), calculate_R_D_T (nse.f90:2000-2134)
// and the cell update of T (1017-1026).  Block (CB, 3): thread y forms MT_F
// of direction y+1 from MT_A of the cell and of its +neighbour, and two of
// the six cross derivatives; thread 0 assembles MT_F4, R_D_T and the update
// in the reference's order.
// SRC_ONLY (reference-order schedule): store MT_F4 and R_D_T and leave the
// update to k_seq_T.
template <bool SRC_ONLY, class R, class BI>
__device__ __forceinline__ void T_cell_body(const Dims &d, const GeoT<R> &g, const FieldsT<R> &F, const Phys &P, Ctrl *ctl, const BI blockIdx) {
  using V = Ar<R>;
  if (ctl->done) return;
  __shared__ BlockRed red;
  red_init<1>(red);
  __shared__ V sX[3][2][CB];   // cross derivatives
  __shared__ V sF4[8][CB];     // MT_F4, formed by thread 1
  __shared__ V sG[CB];         // G1 dT/dx + G2 dT/dy + G3 dT/dz, by thread 2
  const int par = parity(ctl);
  const bool first = ctl->first;
  const int tx = threadIdx.x;
  Cell x;
  const bool active = patch_cell(d, x, blockIdx);
  const int c = x.c;
  double e[1] = {0.};
  const size_t Nc = d.Nc, NF = d.NF;
  const R *T = F.f[4] + par * NF;
  int f[7];
  cell_faces(d, x, f);
  if (active) by_dir(threadIdx.y, [&](auto D) {
    constexpr int dd = decltype(D)::value, y = dd - 1;
    const R *MA = F.MTA + (size_t)y * Nc;  // MT_A(q, dd) at MA[3q Nc]
    V G[5] = {V(0.), V(0.), V(0.), V(0.), V(0.)};
    if (x.has_nb(d, 2 * dd)) {
      const int c2 = x.nb(d, 2 * dd).c;
      V A[6], A2[6];
      for (int q = 0; q < 6; ++q) A[q] = MA[3 * q * Nc + c];
      A2[0] = A2[2] = V(0.);  // not used by form_Fd
      A2[1] = MA[3 * Nc + c2];
      A2[3] = MA[9 * Nc + c2];
      A2[4] = MA[12 * Nc + c2];
      A2[5] = MA[15 * Nc + c2];
      if constexpr (std::is_same<R, float>::value)
        form_Fd_rcp(A, A2, G);
      else
        form_Fd(A, A2, G);
    }
    for (int k = 0; k < 5; ++k) F.MTF[(size_t)(5 * (dd - 1) + k) * Nc + c] = G[k];
    // cross derivatives of calculate_R_D_T: y=0 pxy,pzy  y=1 pyx,pzx  y=2 pxz,pyz
    constexpr int e2 = (y == 0) ? 2 : (y == 1) ? 1 : 3;
    constexpr int fa = (y == 1) ? 4 : 2, fb = (y == 1) ? 3 : 1;
    sX[y][0][tx] = V(0.5) * (tangential(d, T, x, (y == 2) ? 2 : fa, e2) - tangential(d, T, x, (y == 2) ? 1 : fb, e2));
    sX[y][1][tx] = (y == 2) ? V(0.5) * (tangential(d, T, x, 4, 3) - tangential(d, T, x, 3, 3))
                            : V(0.5) * (tangential(d, T, x, 6, e2) - tangential(d, T, x, 5, e2));
    if (y == 1) {  // MT_F4 (nim.f90:466-475)
      V Am[3][6];
      for (int k = 0; k < 3; ++k) {
        Am[k][4] = F.MTA[(size_t)(12 + k) * Nc + c];
        Am[k][5] = F.MTA[(size_t)(15 + k) * Nc + c];
      }
      V F4[8];
      if constexpr (std::is_same<R, float>::value)
        form_F4_rcp(Am, V(P.DT), F4);
      else
        form_F4(Am, V(P.DT), F4);
      for (int k = 0; k < 8; ++k) sF4[k][tx] = F4[k];
    } else if (y == 2) {  // the leading G_i d_i T terms of R_D_T, in source order
      const V px = (T[f[2]] - T[f[1]]) / V(2.);
      const V py = (T[f[4]] - T[f[3]]) / V(2.);
      const V pz = (T[f[6]] - T[f[5]]) / V(2.);
      sG[tx] = g.G[c] * px + g.G[Nc + c] * py + g.G[2 * Nc + c] * pz;
    }
  });
  __syncthreads();
  if (active && threadIdx.y == 0) {
    V F4[8];
    for (int k = 0; k < 8; ++k) F4[k] = sF4[k][tx];
    const V pxy = sX[0][0][tx], pzy = sX[0][1][tx], pyx = sX[1][0][tx], pzx = sX[1][1][tx];
    const V pxz = sX[2][0][tx], pyz = sX[2][1][tx];
    const R *gij = g.gij;
    const V RDT = pv<V>(P.alpha, P.d_alpha) * (sG[tx] - gij[3 * Nc + c] * pxy - gij[1 * Nc + c] * pyx - gij[6 * Nc + c] * pxz -
                                  gij[2 * Nc + c] * pzx - gij[7 * Nc + c] * pyz - gij[5 * Nc + c] * pzy);
    if (SRC_ONLY) {
      for (int k = 0; k < 8; ++k) F.MTF4[(size_t)k * Nc + c] = F4[k];
      F.RDT[c] = RDT;
    } else {
      const V cold = F.c[3][c];
      const V nw = stored<R>(cell_update(T, f, cold, F.co[3][c], (RDT + V(0.)), F4, V(P.w[3])));
      F.c[3][c] = nw;
      e[0] = errv(nw, cold, first);
    }
  }
  if (!SRC_ONLY && d.owns(blockIdx.z)) block_max<1, CB3>(red, e, ctl->err[par] + 4);
}
template <bool SRC_ONLY, class R>
__global__ void __launch_bounds__(CB3, minb<R>(5, TCELL_MINB_F)) k_T_cell(Dims d, GeoT<R> g, FieldsT<R> F, Phys P, Ctrl *ctl) {
  T_cell_body<SRC_ONLY, R>(d, g, F, P, ctl, LaunchBlock{});
}

// ---- K7b, NP cells per thread (the float mirror's parallel passes,
// n_theta % NP == 0): k_T_cell over NP theta-adjacent cells with NP-wide
// vector loads and stores (as k_vel_cellN).  Thread y forms MT_F of
// direction y+1 (the +theta neighbour's MT_A is the group's own vector
// shifted by one cell, and one single load for the last cell) and two of the
// six cross derivatives of T; thread 1 forms MT_F4, thread 2 the G_i d_i T
// prefix; thread 0 assembles R_D_T and the cell update.  Each cell's
// arithmetic is k_T_cell's.
template <class R, int NP>
__global__ void __launch_bounds__(CB3, TCN_MINB) k_T_cellN(Dims d, GeoT<R> g, FieldsT<R> F, Phys P, Ctrl *ctl) {
  using V = Ar<R>;
  if (ctl->done) return;
  __shared__ BlockRed red;
  red_init<1>(red);
  __shared__ V sX[3][2][CB * NP];  // cross derivatives
  __shared__ V sF4[8][CB * NP];    // MT_F4, formed by thread 1
  __shared__ V sG[CB * NP];        // G1 dT/dx + G2 dT/dy + G3 dT/dz, by thread 2
  const int par = parity(ctl);
  const bool first = ctl->first;
  const int tx = threadIdx.x;
  const int i = blockIdx.x * (32 * NP) + NP * (tx & 31);
  const int j = blockIdx.y * (CB / 32) + (tx >> 5);
  const int k = blockIdx.z;
  const bool active = i < d.NT && j < d.NR;
  const int Nc = d.Nc, NF = d.NF, NT = d.NT, NR = d.NR, pl = d.plane;
  const int c = i + NT * (j + NR * k);
  const int im1 = (i == 0) ? NT - 1 : i - 1, ipn = (i + NP >= NT) ? i + NP - NT : i + NP;
  const int f1 = c + NT * k;
  const int fi[7] = {0, f1, f1 + NT, d.offT + c, d.offT + c + 1, d.offZ + c, d.offZ + c + pl};
  const int f4b = d.offT + c - i + ipn;
  auto faceN = [&](const R *a, int m, R (&v)[NP]) {
    if (m == 4) {
      R t[NP];
      ldN<R, NP>(a, fi[3], t);
#pragma unroll
      for (int p = 0; p + 1 < NP; ++p) v[p] = t[p + 1];
      v[NP - 1] = a[f4b];
    } else {
      ldN<R, NP>(a, fi[m], v);
    }
  };
  const R *T = F.f[4] + par * NF;
  auto along = [&](bool lo, bool hi, V v0, V va, V vb) {
    return lo ? tang_vals(true, false, v0, va, vb, V(0.), V(0.))
              : hi ? tang_vals(false, true, v0, V(0.), V(0.), va, vb) : tang_vals(false, false, v0, vb, V(0.), va, V(0.));
  };
  double e[1] = {0.};
  if (active) by_dir(threadIdx.y, [&](auto D) {
    constexpr int dd = decltype(D)::value, y = dd - 1;
    const R *MA = F.MTA + (size_t)y * Nc;  // MT_A(q, dd) at MA[3q Nc]
    // MT_F of direction dd (nim.f90:477-500) from MT_A of the cells and of
    // their +dd neighbours
    {
      const bool nb = (dd == 1) ? (j < NR - 1) : (dd == 3) ? (k < d.NZ - 1) : true;
      R A[6][NP];
#pragma unroll
      for (int q = 0; q < 6; ++q) ldN<R, NP>(MA + 3 * q * Nc, c, A[q]);
      V G[5][NP];
#pragma unroll
      for (int p = 0; p < NP; ++p)
        for (int s = 0; s < 5; ++s) G[s][p] = V(0.);
      if (nb) {
        const int slots[4] = {1, 3, 4, 5};
        R B[6][NP];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int q = slots[u];
          if (dd == 2) {
#pragma unroll
            for (int p = 0; p + 1 < NP; ++p) B[q][p] = A[q][p + 1];
            B[q][NP - 1] = MA[3 * q * Nc + c - i + ipn];
          } else {
            ldN<R, NP>(MA + 3 * q * Nc, c + (dd == 1 ? NT : pl), B[q]);
          }
        }
#pragma unroll
        for (int p = 0; p < NP; ++p) {
          V a[6], a2[6], gg[5];
          for (int q = 0; q < 6; ++q) a[q] = A[q][p];
          a2[0] = a2[2] = V(0.);  // not used by form_Fd
          a2[1] = B[1][p];
          a2[3] = B[3][p];
          a2[4] = B[4][p];
          a2[5] = B[5][p];
          if constexpr (std::is_same<R, float>::value)
            form_Fd_rcp(a, a2, gg);
          else
            form_Fd(a, a2, gg);
          for (int s = 0; s < 5; ++s) G[s][p] = gg[s];
        }
      }
#pragma unroll
      for (int s = 0; s < 5; ++s) {
        R out[NP];
#pragma unroll
        for (int p = 0; p < NP; ++p) out[p] = G[s][p];
        stN<R, NP>(F.MTF + (size_t)(5 * (dd - 1) + s) * Nc, c, out);
      }
    }
    // T's faces of the NP cells
    R o[7][NP];
#pragma unroll
    for (int m = 1; m <= 6; ++m) faceN(T, m, o[m]);
    const bool rlo = (j == 0), rhi = (j == NR - 1);
    const int ra = rlo ? j + 1 : j - 1, rb = rlo ? j + 2 : (rhi ? j - 2 : j + 1);
    const bool zlo = (k == 0), zhi = (k == d.NZ - 1);
    const int ka = zlo ? k + 1 : k - 1, kb = zlo ? k + 2 : (zhi ? k - 2 : k + 1);
    // cross derivatives of calculate_R_D_T: y=0 pxy,pzy  y=1 pyx,pzx  y=2 pxz,pyz
    if (y == 0) {
      const int rrow = NT * (j + (NR + 1) * k), zlev = d.offZ + NT * (j + NR * k);
      const V r_m1 = T[rrow + im1], r_pn = T[rrow + ipn], r1_m1 = T[rrow + NT + im1], r1_pn = T[rrow + NT + ipn];
      const V z_m1 = T[zlev + im1], z_pn = T[zlev + ipn], z1_m1 = T[zlev + pl + im1], z1_pn = T[zlev + pl + ipn];
#pragma unroll
      for (int p = 0; p < NP; ++p) {
        const V up2 = (p + 1 < NP) ? (V)o[2][p + 1] : r1_pn, um2 = (p > 0) ? (V)o[2][p - 1] : r1_m1;
        const V up1 = (p + 1 < NP) ? (V)o[1][p + 1] : r_pn, um1 = (p > 0) ? (V)o[1][p - 1] : r_m1;
        sX[0][0][tx * NP + p] = V(0.5) * ((up2 - um2) / V(4.) - (up1 - um1) / V(4.));
        const V up6 = (p + 1 < NP) ? (V)o[6][p + 1] : z1_pn, um6 = (p > 0) ? (V)o[6][p - 1] : z1_m1;
        const V up5 = (p + 1 < NP) ? (V)o[5][p + 1] : z_pn, um5 = (p > 0) ? (V)o[5][p - 1] : z_m1;
        sX[0][1][tx * NP + p] = V(0.5) * ((up6 - um6) / V(4.) - (up5 - um5) / V(4.));
      }
    } else if (y == 1) {
      const int tra = d.offT + NT * (ra + NR * k), trb = d.offT + NT * (rb + NR * k);
      const int zra = d.offZ + NT * (ra + NR * k), zrb = d.offZ + NT * (rb + NR * k);
      R av[NP + 1], bv[NP + 1];
      {
        R t[NP];
        ldN<R, NP>(T, tra + i, t);
#pragma unroll
        for (int p = 0; p < NP; ++p) av[p] = t[p];
        ldN<R, NP>(T, trb + i, t);
#pragma unroll
        for (int p = 0; p < NP; ++p) bv[p] = t[p];
        av[NP] = T[tra + ipn];
        bv[NP] = T[trb + ipn];
      }
      R za[NP], zb[NP], zA[NP], zB[NP];
      ldN<R, NP>(T, zra + i, za);
      ldN<R, NP>(T, zrb + i, zb);
      ldN<R, NP>(T, zra + pl + i, zA);
      ldN<R, NP>(T, zrb + pl + i, zB);
#pragma unroll
      for (int p = 0; p < NP; ++p) {
        sX[1][0][tx * NP + p] =
            V(0.5) * (along(rlo, rhi, o[4][p], av[p + 1], bv[p + 1]) - along(rlo, rhi, o[3][p], av[p], bv[p]));
        sX[1][1][tx * NP + p] =
            V(0.5) * (along(rlo, rhi, o[6][p], zA[p], zB[p]) - along(rlo, rhi, o[5][p], za[p], zb[p]));
      }
      // MT_F4 (nim.f90:466-475)
      R a4[3][NP], a5[3][NP];
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        ldN<R, NP>(F.MTA + (size_t)(12 + q) * Nc, c, a4[q]);
        ldN<R, NP>(F.MTA + (size_t)(15 + q) * Nc, c, a5[q]);
      }
#pragma unroll
      for (int p = 0; p < NP; ++p) {
        V Am[3][6], F4[8];
        for (int q = 0; q < 3; ++q) {
          Am[q][4] = a4[q][p];
          Am[q][5] = a5[q][p];
        }
        if constexpr (std::is_same<R, float>::value)
          form_F4_rcp(Am, V(P.DT), F4);
        else
          form_F4(Am, V(P.DT), F4);
        for (int q = 0; q < 8; ++q) sF4[q][tx * NP + p] = F4[q];
      }
    } else {
      const int rka = NT * (j + (NR + 1) * ka), rkb = NT * (j + (NR + 1) * kb);
      const int tka = d.offT + NT * (j + NR * ka), tkb = d.offT + NT * (j + NR * kb);
      R pa[NP], pb[NP], pA[NP], pB[NP];
      ldN<R, NP>(T, rka + i, pa);
      ldN<R, NP>(T, rkb + i, pb);
      ldN<R, NP>(T, rka + NT + i, pA);
      ldN<R, NP>(T, rkb + NT + i, pB);
      R av[NP + 1], bv[NP + 1];
      {
        R t[NP];
        ldN<R, NP>(T, tka + i, t);
#pragma unroll
        for (int p = 0; p < NP; ++p) av[p] = t[p];
        ldN<R, NP>(T, tkb + i, t);
#pragma unroll
        for (int p = 0; p < NP; ++p) bv[p] = t[p];
        av[NP] = T[tka + ipn];
        bv[NP] = T[tkb + ipn];
      }
      R G0[NP], G1[NP], G2[NP];
      ldN<R, NP>(g.G, c, G0);
      ldN<R, NP>(g.G + Nc, c, G1);
      ldN<R, NP>(g.G + 2 * Nc, c, G2);
#pragma unroll
      for (int p = 0; p < NP; ++p) {
        sX[2][0][tx * NP + p] =
            V(0.5) * (along(zlo, zhi, o[2][p], pA[p], pB[p]) - along(zlo, zhi, o[1][p], pa[p], pb[p]));
        sX[2][1][tx * NP + p] =
            V(0.5) * (along(zlo, zhi, o[4][p], av[p + 1], bv[p + 1]) - along(zlo, zhi, o[3][p], av[p], bv[p]));
        // the leading G_i d_i T terms of R_D_T, in source order
        const V px = (o[2][p] - o[1][p]) / V(2.);
        const V py = (o[4][p] - o[3][p]) / V(2.);
        const V pz = (o[6][p] - o[5][p]) / V(2.);
        sG[tx * NP + p] = G0[p] * px + G1[p] * py + G2[p] * pz;
      }
    }
  });
  __syncthreads();
  if (active && threadIdx.y == 0) {
    R o[7][NP];
#pragma unroll
    for (int m = 1; m <= 6; ++m) faceN(T, m, o[m]);
    const int slot[6] = {3, 1, 6, 2, 7, 5};
    R gs[6][NP];
#pragma unroll
    for (int s = 0; s < 6; ++s) ldN<R, NP>(g.gij + slot[s] * Nc, c, gs[s]);
    R cur[NP], old[NP], out[NP];
    ldN<R, NP>(F.c[3], c, cur);
    ldN<R, NP>(F.co[3], c, old);
    const V w = V(P.w[3]);
#pragma unroll
    for (int p = 0; p < NP; ++p) {
      const int e2 = tx * NP + p;
      V F4[8];
      for (int q = 0; q < 8; ++q) F4[q] = sF4[q][e2];
      const V pxy = sX[0][0][e2], pzy = sX[0][1][e2], pyx = sX[1][0][e2], pzx = sX[1][1][e2];
      const V pxz = sX[2][0][e2], pyz = sX[2][1][e2];
      const V RDT = pv<V>(P.alpha, P.d_alpha) * (sG[e2] - gs[0][p] * pxy - gs[1][p] * pyx - gs[2][p] * pxz -
                                                  gs[3][p] * pzx - gs[4][p] * pyz - gs[5][p] * pzy);
      // cell_update (nse.f90:1018-1026), term by term
      const V c0 = cur[p];
      const V nw = stored<R>((1 - w) * c0 + (w / F4[0]) * (+F4[1] * (V)old[p] + F4[2] * (V)o[1][p] +
                                                            F4[3] * (V)o[2][p] + F4[4] * (V)o[3][p] +
                                                            F4[5] * (V)o[4][p] + F4[6] * (V)o[5][p] +
                                                            F4[7] * (V)o[6][p] + (RDT + V(0.))));
      out[p] = (R)nw;
      e[0] = nmax(e[0], errv(nw, c0, first));
    }
    stN<R, NP>(F.c[3], c, out);
  }
  if (d.owns(blockIdx.z)) block_max<1, CB3>(red, e, ctl->err[par] + 4);
}

// ---- K8: +xi face updates of T (nse.f90:1033-1088), cur -> next; the z-wall
// values set by apply_zero_flux travel to the next half too
template <class R, class BI>
__device__ __forceinline__ void T_face_body(const Dims &d, const GeoT<R> &g, const FieldsT<R> &F, const Phys &P, Ctrl *ctl, const BI blockIdx) {
  using V = Ar<R>;
  if (ctl->done) return;
  __shared__ BlockRed red;
  red_init<1>(red);
  const int par = parity(ctl);
  const bool first = ctl->first;
  Cell x;
  const bool act = patch_cell(d, x, blockIdx);
  const int c = x.c;
  double e[1] = {0.};
  if (act) {
    const int Nc = d.Nc, NF = d.NF;
    const R *T = F.f[4] + par * NF;
    R *Tn = F.f[4] + (1 - par) * NF;
    for (int dd = 1; dd <= 3; ++dd) {
      if (!x.has_nb(d, 2 * dd)) continue;
      const Cell x2 = x.nb(d, 2 * dd);
      V Fd[5];
      for (int k = 0; k < 5; ++k) Fd[k] = F.MTF[(5 * (dd - 1) + k) * Nc + c];
      const int fo = x.face(d, 2 * dd);
      const V nw = stored<R>(face_update(d, T, F.c[3], F.co[3], Fd, g.dg[(2 * (dd - 1)) * Nc + c],
                                              g.dg[(2 * (dd - 1) + 1) * Nc + c], dd, x, x2, V(P.w[3])));
      Tn[fo] = nw;
      e[0] = nmax(e[0], errv(nw, T[fo], first));
    }
    if (x.k == 0) Tn[x.face(d, 5)] = T[x.face(d, 5)];
    if (x.k == d.NZ - 1) Tn[x.face(d, 6)] = T[x.face(d, 6)];
  }
  if (d.owns(blockIdx.z)) block_max<1>(red, e, ctl->err[par] + 4);
}
template <class R>
__global__ void __launch_bounds__(BLK, minb<R>(4, TFACE_MINB_F)) k_T_face(Dims d, GeoT<R> g, FieldsT<R> F, Phys P, Ctrl *ctl) {
  T_face_body<R>(d, g, F, P, ctl, LaunchBlock{});
}

// The +xi_dd face updates of one field (faces fr of the current half, new
// values into fn) for the NP theta-adjacent cells of a group starting at
// (i, j, k), from NP-wide vector loads: the faces of the cells and of their
// +dd neighbours (for theta the group's own vectors shifted by one cell,
// plus single loads for the last cell's neighbour) and the cell and old-cell
// values cv, co; the theta faces' new values are stored one by one (they
// start one cell off the vector boundary).  Each face's arithmetic is
// face_update's.  Returns the largest change.
template <int dd, class R, int NP>
__device__ __forceinline__ double face_updateN(const Dims &d, int i, int j, int k, const R *fr, R *fn, const R *cv,
                                               const R *co, const R (&Fd)[5][NP], const R (&dg0)[NP],
                                               const R (&dg1)[NP], Ar<R> w, bool first) {
  using V = Ar<R>;
  const int NT = d.NT, NR = d.NR, pl = d.plane;
  const int c = i + NT * (j + NR * k);
  const int ipn = (i + NP >= NT) ? i + NP - NT : i + NP;
  auto group = [&](int jj, int kk, R (&v)[7][NP]) {
    const int cc = i + NT * (jj + NR * kk), ff = cc + NT * kk;
    ldN<R, NP>(fr, ff, v[1]);
    ldN<R, NP>(fr, ff + NT, v[2]);
    R t[NP];
    ldN<R, NP>(fr, d.offT + cc, t);
#pragma unroll
    for (int p = 0; p < NP; ++p) v[3][p] = t[p];
#pragma unroll
    for (int p = 0; p + 1 < NP; ++p) v[4][p] = t[p + 1];
    v[4][NP - 1] = fr[d.offT + cc - i + ipn];
    ldN<R, NP>(fr, d.offZ + cc, v[5]);
    ldN<R, NP>(fr, d.offZ + cc + pl, v[6]);
  };
  R ox[7][NP], on[7][NP], cx[NP], cxo[NP], cn[NP], cno[NP];
  group(j, k, ox);
  ldN<R, NP>(cv, c, cx);
  ldN<R, NP>(co, c, cxo);
  if (dd == 1 || dd == 3) {
    if (dd == 1)
      group(j + 1, k, on);
    else
      group(j, k + 1, on);
    ldN<R, NP>(cv, c + (dd == 1 ? NT : pl), cn);
    ldN<R, NP>(co, c + (dd == 1 ? NT : pl), cno);
  } else {  // the +theta neighbours: cells i+1 .. i+NP
    const int cw = c - i + ipn;
    const int iw = (ipn == NT - 1) ? 0 : ipn + 1;
#pragma unroll
    for (int p = 0; p + 1 < NP; ++p) {
      on[1][p] = ox[1][p + 1];
      on[2][p] = ox[2][p + 1];
      on[4][p] = ox[4][p + 1];
      on[5][p] = ox[5][p + 1];
      on[6][p] = ox[6][p + 1];
      cn[p] = cx[p + 1];
      cno[p] = cxo[p + 1];
    }
#pragma unroll
    for (int p = 0; p < NP; ++p) on[3][p] = ox[4][p];
    on[1][NP - 1] = fr[cw + NT * k];
    on[2][NP - 1] = fr[cw + NT * k + NT];
    on[4][NP - 1] = fr[d.offT + cw - ipn + iw];
    on[5][NP - 1] = fr[d.offZ + cw];
    on[6][NP - 1] = fr[d.offZ + cw + pl];
    cn[NP - 1] = cv[cw];
    cno[NP - 1] = co[cw];
  }
  constexpr int e1 = (dd == 1) ? 2 : 1, e2 = (dd == 3) ? 2 : 3;  // tr1(dd), tr2(dd)
  double err = 0.;
  R out[NP];
#pragma unroll
  for (int p = 0; p < NP; ++p) {
    const V B3 = (dg0[p]) * ((V)ox[2 * e1][p] - ox[2 * e1 - 1][p] + on[2 * e1][p] - on[2 * e1 - 1][p]) / V(4.0);
    const V B4 = (dg1[p]) * ((V)ox[2 * e2][p] - ox[2 * e2 - 1][p] + on[2 * e2][p] - on[2 * e2 - 1][p]) / V(4.0);
    const V old = ox[2 * dd][p];
    const V nw = stored<R>((1 - w) * old + (w / Fd[0][p]) * (+Fd[1][p] * (V)ox[2 * dd - 1][p] +
                                                               Fd[2][p] * (V)on[2 * dd][p] +
                                                               Fd[3][p] * ((V)cx[p] + cxo[p]) +
                                                               Fd[4][p] * ((V)cn[p] + cno[p]) - B3 - B4));
    out[p] = (R)nw;
    err = nmax(err, errv(nw, old, first));
  }
  if (dd == 2) {
#pragma unroll
    for (int p = 0; p + 1 < NP; ++p) fn[d.offT + c + p + 1] = out[p];
    fn[d.offT + c - i + ipn] = out[NP - 1];
  } else {
    stN<R, NP>(fn, dd == 1 ? c + NT * k + NT : d.offZ + c + pl, out);
  }
  return err;
}

// ---- K8, NP cells per thread (the float mirror, n_theta % NP == 0):
// k_T_face over NP theta-adjacent cells, block (CB, 3): thread y updates the
// +xi face of direction y+1 of the NP cells from NP-wide vector loads (the
// +theta neighbours as k_p_faceN forms them) and carries the z-wall values
// to the next half (thread 2).  Each face's arithmetic is face_update's.
template <class R, int NP>
__global__ void __launch_bounds__(CB3, TFN_MINB) k_T_faceN(Dims d, GeoT<R> g, FieldsT<R> F, Phys P, Ctrl *ctl) {
  using V = Ar<R>;
  if (ctl->done) return;
  __shared__ BlockRed red;
  red_init<1>(red);
  const int par = parity(ctl);
  const bool first = ctl->first;
  const int tx = threadIdx.x;
  const int i = blockIdx.x * (32 * NP) + NP * (tx & 31);
  const int j = blockIdx.y * (CB / 32) + (tx >> 5);
  const int k = blockIdx.z;
  double e[1] = {0.};
  if (i < d.NT && j < d.NR) by_dir(threadIdx.y, [&](auto D) {
    constexpr int dd = decltype(D)::value;
    const int Nc = d.Nc, NF = d.NF, NT = d.NT, NR = d.NR, pl = d.plane;
    const int c = i + NT * (j + NR * k);
    const int ipn = (i + NP >= NT) ? i + NP - NT : i + NP;
    const R *T = F.f[4] + par * NF;
    R *Tn = F.f[4] + (1 - par) * NF;
    if (dd == 3) {  // the z-wall values set by apply_zero_flux travel to the next half
      R t[NP];
      if (k == 0) {
        ldN<R, NP>(T, d.offZ + c, t);
        stN<R, NP>(Tn, d.offZ + c, t);
      }
      if (k == d.NZ - 1) {
        ldN<R, NP>(T, d.offZ + c + pl, t);
        stN<R, NP>(Tn, d.offZ + c + pl, t);
      }
    }
    if ((dd == 1 && j == NR - 1) || (dd == 3 && k == d.NZ - 1)) return;  // a wall face
    auto group = [&](int jj, int kk, R (&v)[7][NP]) {
      const int cc = i + NT * (jj + NR * kk), ff = cc + NT * kk;
      ldN<R, NP>(T, ff, v[1]);
      ldN<R, NP>(T, ff + NT, v[2]);
      R t[NP];
      ldN<R, NP>(T, d.offT + cc, t);
#pragma unroll
      for (int p = 0; p < NP; ++p) v[3][p] = t[p];
#pragma unroll
      for (int p = 0; p + 1 < NP; ++p) v[4][p] = t[p + 1];
      v[4][NP - 1] = T[d.offT + cc - i + ipn];
      ldN<R, NP>(T, d.offZ + cc, v[5]);
      ldN<R, NP>(T, d.offZ + cc + pl, v[6]);
    };
    R ox[7][NP], on[7][NP], cx[NP], cxo[NP], cn[NP], cno[NP];
    group(j, k, ox);
    ldN<R, NP>(F.c[3], c, cx);
    ldN<R, NP>(F.co[3], c, cxo);
    if (dd == 1 || dd == 3) {
      if (dd == 1)
        group(j + 1, k, on);
      else
        group(j, k + 1, on);
      ldN<R, NP>(F.c[3], c + (dd == 1 ? NT : pl), cn);
      ldN<R, NP>(F.co[3], c + (dd == 1 ? NT : pl), cno);
    } else {  // the +theta neighbours: cells i+1 .. i+NP
      const int cw = c - i + ipn;
      const int iw = (ipn == NT - 1) ? 0 : ipn + 1;
#pragma unroll
      for (int p = 0; p + 1 < NP; ++p) {
        on[1][p] = ox[1][p + 1];
        on[2][p] = ox[2][p + 1];
        on[4][p] = ox[4][p + 1];
        on[5][p] = ox[5][p + 1];
        on[6][p] = ox[6][p + 1];
        cn[p] = cx[p + 1];
        cno[p] = cxo[p + 1];
      }
#pragma unroll
      for (int p = 0; p < NP; ++p) on[3][p] = ox[4][p];
      on[1][NP - 1] = T[cw + NT * k];
      on[2][NP - 1] = T[cw + NT * k + NT];
      on[4][NP - 1] = T[d.offT + cw - ipn + iw];
      on[5][NP - 1] = T[d.offZ + cw];
      on[6][NP - 1] = T[d.offZ + cw + pl];
      cn[NP - 1] = F.c[3][cw];
      cno[NP - 1] = F.co[3][cw];
    }
    R Fd[5][NP], dg0[NP], dg1[NP];
#pragma unroll
    for (int q = 0; q < 5; ++q) ldN<R, NP>(F.MTF + (size_t)(5 * (dd - 1) + q) * Nc, c, Fd[q]);
    ldN<R, NP>(g.dg + (size_t)(2 * (dd - 1)) * Nc, c, dg0);
    ldN<R, NP>(g.dg + (size_t)(2 * (dd - 1) + 1) * Nc, c, dg1);
    constexpr int e1 = (dd == 1) ? 2 : 1, e2 = (dd == 3) ? 2 : 3;  // tr1(dd), tr2(dd)
    const V w = V(P.w[3]);
    R out[NP];
#pragma unroll
    for (int p = 0; p < NP; ++p) {
      const V B3 = (dg0[p]) * ((V)ox[2 * e1][p] - ox[2 * e1 - 1][p] + on[2 * e1][p] - on[2 * e1 - 1][p]) / V(4.0);
      const V B4 = (dg1[p]) * ((V)ox[2 * e2][p] - ox[2 * e2 - 1][p] + on[2 * e2][p] - on[2 * e2 - 1][p]) / V(4.0);
      const V old = ox[2 * dd][p];
      const V nw = stored<R>((1 - w) * old + (w / Fd[0][p]) * (+Fd[1][p] * (V)ox[2 * dd - 1][p] +
                                                                 Fd[2][p] * (V)on[2 * dd][p] +
                                                                 Fd[3][p] * ((V)cx[p] + cxo[p]) +
                                                                 Fd[4][p] * ((V)cn[p] + cno[p]) - B3 - B4));
      out[p] = (R)nw;
      e[0] = nmax(e[0], errv(nw, old, first));
    }
    if (dd == 2) {
#pragma unroll
      for (int p = 0; p + 1 < NP; ++p) Tn[d.offT + c + p + 1] = out[p];
      Tn[d.offT + c - i + ipn] = out[NP - 1];
    } else {
      stN<R, NP>(Tn, dd == 1 ? c + NT * k + NT : d.offZ + c + pl, out);
    }
  });
  if (d.owns(blockIdx.z)) block_max<1, CB3>(red, e, ctl->err[par] + 4);
}

// ---- K2, NP cells per thread (the float mirror, n_theta % NP == 0): the
// +xi face updates of u, v, w (nse.f90:878-1005) over NP theta-adjacent
// cells, block (CB, 3): thread y updates the +xi face of direction y+1 of
// the NP cells for each component (face_updateN), as k_vel_face.
template <class R, int NP>
__global__ void __launch_bounds__(CB3, VFN_MINB) k_vel_faceN(Dims d, GeoT<R> g, FieldsT<R> F, Phys P, Ctrl *ctl) {
  if (ctl->done) return;
  __shared__ BlockRed red;
  red_init<3>(red);
  const int par = parity(ctl);
  const bool first = ctl->first;
  const int tx = threadIdx.x;
  const int i = blockIdx.x * (32 * NP) + NP * (tx & 31);
  const int j = blockIdx.y * (CB / 32) + (tx >> 5);
  const int k = blockIdx.z;
  double e[3] = {0., 0., 0.};
  if (i < d.NT && j < d.NR) by_dir(threadIdx.y, [&](auto D) {
    constexpr int dd = decltype(D)::value;
    if ((dd == 1 && j == d.NR - 1) || (dd == 3 && k == d.NZ - 1)) return;  // a wall face
    const int Nc = d.Nc, NF = d.NF;
    const int c = i + d.NT * (j + d.NR * k);
    R Fd[5][NP], dg0[NP], dg1[NP];
#pragma unroll
    for (int q = 0; q < 5; ++q) ldN<R, NP>(F.MF + (size_t)(5 * (dd - 1) + q) * Nc, c, Fd[q]);
    ldN<R, NP>(g.dg + (size_t)(2 * (dd - 1)) * Nc, c, dg0);
    ldN<R, NP>(g.dg + (size_t)(2 * (dd - 1) + 1) * Nc, c, dg1);
#pragma unroll 1
    for (int q = 0; q < 3; ++q)
      e[q] = face_updateN<dd>(d, i, j, k, F.f[q] + par * NF, F.f[q] + (1 - par) * NF, F.c[q], F.co[q], Fd, dg0, dg1,
                              Ar<R>(P.w[q]), first);
  });
  if (d.owns(blockIdx.z)) block_max<3, CB3>(red, e, ctl->err[par]);
}

// ---- K9: end of one pass (find_error's maxima, the do-while test of
// nse.f90:129 and the max_iters guard).  lowp: a pass of the FP32 phase of a
// mixed-precision step, which ends (done, status untouched) when every field
// meets its tolerance or when kLowpStall passes in a row brought no field
// that is still above its tolerance to a new smallest change; the FP64
// passes that follow apply the reference's test.  max_iters bounds both
// phases together.
template <class BI>
__device__ __forceinline__ void iter_end_body(Ctrl *ctl, const Phys &P, int lowp, const BI blockIdx) {
  if (ctl->done) return;
  const int par = ctl->iter & ctl->pmask;
  double e[5];
  bool finite = true;
  for (int q = 0; q < 5; ++q) {
    unsigned long long b = ctl->err[par][q];
    if (q == 3 && P.dpdx_tolerance) b = ctl->err[par][5];
    if (b >= 0x7FF0000000000000ull) finite = false;
    e[q] = __longlong_as_double((long long)b);
    if (ctl->first) e[q] = nmax(e[q], __longlong_as_double((long long)ctl->wall_floor[q]));
    ctl->last_err[q] = e[q];
  }
  // clear the slot the next pass accumulates into (the other one with
  // double-buffered faces, this one with in-place sweeps)
  const int nxt = (ctl->iter + 1) & ctl->pmask;
  for (int q = 0; q < 8; ++q) ctl->err[nxt][q] = 0ull;
  ctl->iter += 1;
  ctl->step_iters += 1;
  ctl->first = 0;
  bool busy = false;
  for (int q = 0; q < 5; ++q) busy = busy || (e[q] > P.tol[q]);
  if (lowp) {
    ctl->lowp_iters += 1;
    bool progress = false;
    for (int q = 0; q < 5; ++q) {
      if (e[q] > P.tol[q] && e[q] < ctl->best[q]) progress = true;
      if (e[q] < ctl->best[q]) ctl->best[q] = e[q];
    }
    ctl->stall = progress ? 0 : ctl->stall + 1;
    if (!finite) {
      ctl->done = 1;
      ctl->status = -4;  // NIM_ERR_NONFINITE
    } else if (!busy || ctl->stall >= kLowpStall) {
      ctl->done = 1;
    } else if (P.max_iters > 0 && ctl->step_iters >= P.max_iters) {
      ctl->done = 1;
      ctl->status = -3;  // NIM_ERR_NOT_CONVERGED
    }
    return;
  }
  if (!finite) {
    ctl->done = 1;
    ctl->status = -4;  // NIM_ERR_NONFINITE
  } else if (!busy) {
    ctl->done = 1;
  } else if (P.max_iters > 0 && ctl->step_iters >= P.max_iters) {
    ctl->done = 1;
    ctl->status = -3;  // NIM_ERR_NOT_CONVERGED
  }
}
__global__ void k_iter_end(Ctrl *ctl, Phys P, int lowp) {
  iter_end_body(ctl, P, lowp, LaunchBlock{});
}

// start of the FP32 phase of a mixed-precision step (after k_step_reset)
__global__ void k_lowp_begin(Ctrl *ctl) {
  ctl->lowp_iters = 0;
  ctl->stall = 0;
  for (int q = 0; q < 5; ++q) ctl->best[q] = __longlong_as_double(0x7FF0000000000000ll);  // +inf
}

// FP32 phase over, FP64 passes next (not after a non-finite stop)
__global__ void k_lowp_end(Ctrl *ctl) {
  if (ctl->status == 0) ctl->done = 0;
}

// Conversions between the FP64 arrays and their FP32 mirror: entry
// blockIdx.y of the list, grid-stride over its elements
struct CvtList {
  static constexpr int kMax = 32;
  const void *src[kMax];
  void *dst[kMax];
  long long n[kMax];
};
template <class S, class D>
__global__ void __launch_bounds__(BLK) k_convert(CvtList L) {
  const S *__restrict__ src = static_cast<const S *>(L.src[blockIdx.y]);
  D *__restrict__ dst = static_cast<D *>(L.dst[blockIdx.y]);
  const long long n = L.n[blockIdx.y];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dst[i] = (D)src[i];
}

// ============================================ reference-order sweeps
// The reference runs every Gauss-Seidel sweep over cells in number order
// (one OpenMP thread, run.sh:2).  A cell's update reads values of the cells
// (di,dj,dk) in {(+-1,0,0),(0,+-1,0),(0,0,+-1),(0,0,+-2),(0,+-2,0),(+1,-1,0),
// (+1,0,-1),(0,+1,-1),(-1,+1,0),(-1,0,+1),(0,-1,+1)} and no other cell's.
// Ordering cells by the level t = i + 2j + 3k puts every such neighbour with
// a smaller number on a lower level and every larger one on a higher level,
// the theta seam included, so sweeping level by level, in
// place, with a grid-wide barrier between levels reproduces the reference's
// iterates exactly.  order[] lists the cells level by level, lstart[] the
// level boundaries.

// velocity sweep (integrate_velocity_field_formulation2_i, nse.f90:831-1006;
// FORM 1: integrate_velocity_field_i, nse.f90:330-828).  Block (CB, 3):
// threadIdx.y = component; the three components of a cell touch disjoint
// data, so they run side by side.
template <int FORM>
__global__ void __launch_bounds__(CB3) k_seq_vel(Dims d, Geo g, Fields F, Phys P, Ctrl *ctl,
                                                 const int *__restrict__ order, const int *__restrict__ lstart,
                                                 int nlev) {
  namespace cg = cooperative_groups;
  cg::grid_group grid = cg::this_grid();
  if (ctl->done) return;
  __shared__ BlockRed red;
  red_init<3>(red);
  const int par = parity(ctl);
  const bool first = ctl->first;
  const size_t Nc = d.Nc, NF = d.NF;
  const int v = threadIdx.y;
  double e[3] = {0., 0., 0.};
  const int tid = blockIdx.x * CB + threadIdx.x, nth = gridDim.x * CB;
  double *fr = F.f[v] + par * NF;
  double *cv = F.c[v];
  const double *co = F.co[v];
  for (int L = 0; L < nlev; ++L) {
    for (int q = lstart[L] + tid; q < lstart[L + 1]; q += nth) {
      const int c = order[q];
      const Cell x = Cell::of(d, c);
      int f[7];
      cell_faces(d, x, f);
      const double cold = LdCoh::ld(cv, c);
      double nw;
      if (FORM == 1) {
        double at[9];
        for (int k = 0; k < 9; ++k) at[k] = F.AT[(size_t)k * Nc + c];
        nw = cell_update_f1<LdCoh>(fr, f, cold, co[c], F.Bv[(size_t)v * Nc + c], at, P.w[v]);
      } else {
        double F4[8];
        for (int k = 0; k < 8; ++k) F4[k] = F.MF4[(size_t)k * Nc + c];
        nw = cell_update<LdCoh>(fr, f, cold, co[c], F.Bv[(size_t)v * Nc + c], F4, P.w[v]);
      }
      st_coh(cv, c, nw);
      e[v] = nmax(e[v], errv(nw, cold, first));
#pragma unroll
      for (int dd = 1; dd <= 3; ++dd) {
        if (!x.has_nb(d, 2 * dd)) continue;
        const Cell x2 = x.nb(d, 2 * dd);
        const int fo = x.face(d, 2 * dd);
        const double old = LdCoh::ld(fr, fo);
        double nf;
        if (FORM == 1) {
          nf = v1_face_value<LdCoh>(d, g, F, P, fr, cv, co, F.Bv + (size_t)v * Nc, x, dd, P.w[v]);
        } else {
          double Fd[5];
          for (int k = 0; k < 5; ++k) Fd[k] = F.MF[(size_t)(5 * (dd - 1) + k) * Nc + c];
          nf = face_update_cv<LdCoh>(d, fr, nw, LdCoh::ld(cv, x2.c), co, Fd, g.dg[(2 * (dd - 1)) * Nc + c],
                                     g.dg[(2 * (dd - 1) + 1) * Nc + c], dd, x, x2, P.w[v]);
        }
        st_coh(fr, fo, nf);
        e[v] = nmax(e[v], errv(nf, old, first));
      }
    }
    grid.sync();
  }
  block_max<3, CB3>(red, e, ctl->err[par]);
}

// pressure sweep (integrate_pressure_field_i, nse.f90:1091-1289)
__global__ void __launch_bounds__(BLK) k_seq_p(Dims d, Geo g, Fields F, Phys P, Ctrl *ctl,
                                               const int *__restrict__ order, const int *__restrict__ lstart,
                                               int nlev) {
  namespace cg = cooperative_groups;
  cg::grid_group grid = cg::this_grid();
  if (ctl->done) return;
  __shared__ BlockRed red;
  red_init<1>(red);
  const int par = parity(ctl);
  const bool first = ctl->first;
  const size_t NF = d.NF;
  double e[1] = {0.};
  double *pr = F.f[3] + par * NF;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  for (int L = 0; L < nlev; ++L) {
    for (int q = lstart[L] + tid; q < lstart[L + 1]; q += nth) {
      const Cell x = Cell::of(d, order[q]);
#pragma unroll
      for (int dd = 1; dd <= 3; ++dd) {
        if (!x.has_nb(d, 2 * dd)) continue;
        const int fo = x.face(d, 2 * dd);
        const double old = LdCoh::ld(pr, fo);
        const double nw = p_face_value<LdCoh>(d, g, F, P, pr, x, dd);
        st_coh(pr, fo, nw);
        e[0] = nmax(e[0], errv(nw, old, first));
      }
    }
    grid.sync();
  }
  block_max<1>(red, e, ctl->err[par] + 3);
}

// temperature sweep (integrate_temperature_field_formulation2_i, nse.f90:1009-1089)
__global__ void __launch_bounds__(BLK) k_seq_T(Dims d, Geo g, Fields F, Phys P, Ctrl *ctl,
                                               const int *__restrict__ order, const int *__restrict__ lstart,
                                               int nlev) {
  namespace cg = cooperative_groups;
  cg::grid_group grid = cg::this_grid();
  if (ctl->done) return;
  __shared__ BlockRed red;
  red_init<1>(red);
  const int par = parity(ctl);
  const bool first = ctl->first;
  const size_t Nc = d.Nc, NF = d.NF;
  double e[1] = {0.};
  double *T = F.f[4] + par * NF;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  for (int L = 0; L < nlev; ++L) {
    for (int q = lstart[L] + tid; q < lstart[L + 1]; q += nth) {
      const int c = order[q];
      const Cell x = Cell::of(d, c);
      int f[7];
      cell_faces(d, x, f);
      double F4[8];
      for (int k = 0; k < 8; ++k) F4[k] = F.MTF4[(size_t)k * Nc + c];
      const double cold = LdCoh::ld(F.c[3], c);
      const double nw = cell_update<LdCoh>(T, f, cold, F.co[3][c], (F.RDT[c] + 0.), F4, P.w[3]);
      st_coh(F.c[3], c, nw);
      e[0] = nmax(e[0], errv(nw, cold, first));
#pragma unroll
      for (int dd = 1; dd <= 3; ++dd) {
        if (!x.has_nb(d, 2 * dd)) continue;
        const Cell x2 = x.nb(d, 2 * dd);
        double Fd[5];
        for (int k = 0; k < 5; ++k) Fd[k] = F.MTF[(size_t)(5 * (dd - 1) + k) * Nc + c];
        const int fo = x.face(d, 2 * dd);
        const double old = LdCoh::ld(T, fo);
        const double nwf = face_update_cv<LdCoh>(d, T, nw, LdCoh::ld(F.c[3], x2.c), F.co[3], Fd,
                                                g.dg[(2 * (dd - 1)) * Nc + c], g.dg[(2 * (dd - 1) + 1) * Nc + c], dd,
                                                x, x2, P.w[3]);
        st_coh(T, fo, nwf);
        e[0] = nmax(e[0], errv(nwf, old, first));
      }
    }
    grid.sync();
  }
  block_max<1>(red, e, ctl->err[par] + 4);
}

// apply_pressure_bc in the reference's BC-list order (bc.f90:148-340).  Within
// one wall a face reads its in-wall neighbours (+-1, +-2 along the wall), so
// levels t = (in-wall theta index) + 2 (other in-wall index) reproduce the
// order; bottom and top do not read each other, inner and outer read bottom
// and top only, so one block per wall runs {bottom, top} and then
// {inner, outer}.  border[] lists BC-list indices wall by wall and level by
// level; wlev[w] .. wlev[w+1] are wall w's entries of blev[].
__global__ void __launch_bounds__(BLK) k_seq_pbc(Dims d, Geo g, Fields F, Phys P, Ctrl *ctl,
                                                 const int *__restrict__ border, const int *__restrict__ blev,
                                                 const int *__restrict__ wlev, int wall0) {
  if (ctl->done) return;
  __shared__ BlockRed red;
  red_init<1>(red);
  const int par = parity(ctl), nh = newhalf(ctl);
  const bool first = ctl->first;
  const size_t NF = d.NF;
  double e[1] = {0.};
  double *pr = F.f[3] + par * NF;
  const int w = wall0 + blockIdx.x;
  for (int L = wlev[w]; L < wlev[w + 1]; ++L) {
    for (int q = blev[L] + threadIdx.x; q < blev[L + 1]; q += blockDim.x) {
      const int b = border[q];
      const BFace B = bface(d, b);
      const int fw0 = B.cell.face(d, B.pos);
      const double old = LdCoh::ld(pr, fw0);
      const double nw = p_bc_value<LdCoh>(d, g, F, P, pr, F.f[0] + nh * NF, F.f[1] + nh * NF, F.f[2] + nh * NF,
                                            F.f[4] + par * NF, b);
      st_coh(pr, fw0, nw);
      e[0] = nmax(e[0], errv(nw, old, first));
    }
    __syncthreads();
  }
  block_max<1>(red, e, ctl->err[par] + 3);
}

// ====================================================== end of integrate
// check_steady_state (nse.f90:1316-1332) + evaluate_D (nse.f90:2504-2537)
// (the dual instantiation: the maxima and the sum of squares of the values;
// meshes_dila with its derivative)
template <class R>
__global__ void __launch_bounds__(BLK) k_after_integrate(Dims d, GeoT<R> g, FieldsT<R> F, Phys P, Ctrl *ctl,
                                                         int nblk) {
  using V = Ar<R>;
  __shared__ BlockRed red;
  red_init<2>(red);
  const int par = parity(ctl);
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  double m[2] = {0., 0.}, s[1] = {0.};
  if (c < d.Nc) {
    const Cell x = Cell::of(d, c);
    const size_t NF = d.NF;
    const double tdt = 2 * P.DT;
    double mu = 0.;
    for (int q = 0; q < 3; ++q) mu = nmax(mu, fabs(val(F.c[q][c]) - val(F.co[q][c])) / tdt);
    m[0] = mu;
    m[1] = fabs(val(F.c[3][c]) - val(F.co[3][c])) / tdt;
    int f[7];
    cell_faces(d, x, f);
    V uf[7], vf[7], wf[7];
    for (int k = 1; k <= 6; ++k) {
      uf[k] = F.f[0][par * NF + f[k]];
      vf[k] = F.f[1][par * NF + f[k]];
      wf[k] = F.f[2][par * NF + f[k]];
    }
    const V invV = V(1.) / g.vol[c];
    const V Dila = green_gauss(g, NF, invV, uf, f, 0) + green_gauss(g, NF, invV, vf, f, 1) +
                   green_gauss(g, NF, invV, wf, f, 2);
    F.dila[c] = Dila;
    s[0] = val(Dila) * val(Dila);
    if (!d.owns(x.k)) m[0] = m[1] = s[0] = 0.;
  }
  block_max<2>(red, m, ctl->red);
  block_sum<1>(s, F.part, nblk);
}

// one block: fixed-order sum of the per-block partials
__global__ void k_finish_sum(const double *part, int nblk, int nsum, double *out) {
  __shared__ double sm[BLK];
  for (int n = 0; n < nsum; ++n) {
    double acc = 0.;
    for (int b = threadIdx.x; b < nblk; b += BLK) acc = acc + part[(size_t)n * nblk + b];
    sm[threadIdx.x] = acc;
    __syncthreads();
    for (int s = BLK / 2; s > 0; s >>= 1) {
      if (threadIdx.x < s) sm[threadIdx.x] = sm[threadIdx.x] + sm[threadIdx.x + s];
      __syncthreads();
    }
    if (threadIdx.x == 0) out[n] = sm[0];
    __syncthreads();
  }
}

// update_time_step (nse.f90:1292-1313)
template <class R>
__global__ void __launch_bounds__(BLK) k_update_time(Dims d, FieldsT<R> F, Ctrl *ctl) {
  using V = Ar<R>;
  const int par = parity(ctl);
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.Nc) return;
  const Cell x = Cell::of(d, c);
  for (int q = 0; q < 4; ++q) {
    F.ct[q][c] = (F.co[q][c] + F.c[q][c]) / V(2.);
    F.co[q][c] = F.c[q][c];
  }
  int f[7];
  cell_faces(d, x, f);
  const R *p = F.f[3] + par * (size_t)d.NF;
  F.mp[c] = (p[f[1]] + p[f[2]] + p[f[3]] + p[f[4]] + p[f[5]] + p[f[6]]) / V(6.0);
  F.dila_old[c] = F.dila[c];
}

// find_Nu2 (nse.f90:2699-2798): wall-normal one-sided dT/dn on the inner
// (position 1) and outer (position 2) walls, area weighted.
// (the dual instantiation sums the four values, then their derivatives:
// eight partial sums)
template <class R>
__global__ void __launch_bounds__(BLK) k_nusselt(Dims d, GeoT<R> g, FieldsT<R> F, Ctrl *ctl, int nblk) {
  using V = Ar<R>;
  const int par = parity(ctl);
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  V s[4] = {0., 0., 0., 0.};  // sum1, sumA1 (outer), sum2, sumA2 (inner)
  const int nr = 2 * d.NT * d.NZ;
  if (q < nr) {
    const int b = 2 * d.plane + q;
    const size_t NF = d.NF, NB = d.NBF;
    const BFace B = bface(d, b);
    const int in = (B.pos == 1) ? 2 : 1;
    const Cell c2 = B.cell.nb(d, in), c3 = c2.nb(d, in);
    const R *T = F.f[4] + par * NF;
    const R *w = g.nuw;
    const int f1 = B.cell.face(d, B.pos);
    const V inner = -((w[b]) * T[f1]) + w[NB + b] * T[B.cell.face(d, in)] - w[2 * NB + b] * T[c2.face(d, in)] +
                    w[3 * NB + b] * T[c3.face(d, in)];
    const V dTdx = (B.pos == 1) ? -(inner) : inner;
    const V A = g.area[f1];
    if (B.pos == 1) {
      s[2] = A * dTdx;
      s[3] = A;
    } else {
      s[0] = A * dTdx;
      s[1] = A;
    }
    if (!d.owns(B.cell.k)) s[0] = s[1] = s[2] = s[3] = 0.;
  }
  if constexpr (std::is_same<V, DualD>::value) {
    const double sv[8] = {s[0].v, s[1].v, s[2].v, s[3].v, s[0].t, s[1].t, s[2].t, s[3].t};
    block_sum<8>(sv, F.part, nblk);
  } else {
    block_sum<4>(s, F.part, nblk);
  }
}

// max |value| of the Dirichlet walls per field (u, v, w, -, T): find_error
// compares against zero-initialised *_old arrays on the first pass
__global__ void k_wall_floor(Dims d, Geo g, Ctrl *ctl) {
  __shared__ BlockRed red;
  red_init<5>(red);
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  double m[5] = {0., 0., 0., 0., 0.};
  if (b < d.NBF) {
    const BFace B = bface(d, b);
    m[0] = fabs(g.bcval[b]);
    m[1] = fabs(g.bcval[(size_t)d.NBF + b]);
    m[2] = fabs(g.bcval[2 * (size_t)d.NBF + b]);
    if (B.pos <= 2) m[4] = fabs(g.bcval[3 * (size_t)d.NBF + b]);  // r walls keep T; z walls are recomputed
  }
  block_max<5>(red, m, ctl->wall_floor);
}

}  // namespace nim

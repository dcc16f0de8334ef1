// Host side of the NIM CUDA library: the C ABI of include/nim_gpu.h.
//
// Replaces the OpenMP loops the reference runs from solve_nse (nse.f90:23-85):
//   nim_gpu_init       initialize_nse + apply_all_dirichlet_bcs (nse.f90:31-38)
//   nim_gpu_begin_step calculate_velocity_nim_constants_formulation2 (nse.f90:52)
//   nim_gpu_integrate  integrate_nse (nse.f90:57, 117-176)
//   nim_gpu_end_step   update_time_step + find_Nu2 (nse.f90:72-73)
// The inner loop runs as CUDA graphs of whole iterations; the stop test lives
// on the device (k_iter_end) and the host only polls it between batches.
// With NIM_SCHEDULE_REFERENCE the four Gauss-Seidel sweeps run as in-place
// level-by-level sweeps (k_seq_*) that reproduce the reference's cell order.
// With NIM_PRECISION_MIXED each step's inner loop runs first as FP32 passes
// over a float mirror of the arrays the pass touches, then as FP64 passes
// from the widened FP32 iterate until the reference's stop test holds.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "nim_gpu.h"
#include "nim_common.cuh"
#include "nim_kernels.cuh"
#include "nim_batch.cuh"

using namespace nim;

namespace {

const double MATH_PI = 3.14159265359;  // parameters.f90:31

// Scratch of nim_gpu_nusselt_noalloc: per-block partial sums of the four
// wall sums for up to kNoallocBlocks blocks, then the four final sums.
// A file-scope device array: every GPU that loads the library holds it.
constexpr int kNoallocBlocks = NIM_NOALLOC_MAX_WALL_FACES / 256;
__device__ __align__(256) double g_noalloc_scratch[4 * kNoallocBlocks + 8];

// Device address of g_noalloc_scratch per device (host code cannot use the
// symbol itself: on the host it names a stand-in, not device memory).
constexpr int kMaxDevices = 64;
double *g_noalloc_ptr[kMaxDevices] = {nullptr};
std::mutex g_noalloc_mutex;

struct Buf {
  void *p = nullptr;
};

}  // namespace

struct nim_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  Dims d{};
  nim_params params{};
  Phys phys{};
  GaussRule gq{};
  Geo g{};
  Fields F{};
  Ctrl *ctl = nullptr;       // device
  Ctrl *ctl_host = nullptr;  // pinned mirror
  double *node_xyz = nullptr;
  double *bcv = nullptr;     // [5][5] Dirichlet constants
  int *perm = nullptr;       // reference face number - 1 -> structured face index
  double *scratch = nullptr; // gather/scatter staging [54*Nc or 3*NF]
  double *sums = nullptr;    // [8] outputs of k_finish_sum
  int nblk_c = 0, nblk_b = 0, nblk_c3 = 0;
  dim3 g3{1, 1, 1}, g8{1, 1, 1};  // patch grids: 32x4 (x3 threads) and 32x8 cells
  std::vector<void *> allocs;
  cudaGraphExec_t graph = nullptr;
  int graph_iters = 0;
  int graph_G = 4;  // inner iterations per graph launch (nim_gpu_set_graph_iters)
  bool initialized = false;
  bool in_step = false;
  int32_t STEP = 0;
  double TI = 0;
  int last_iters = 0;
  double host_sums[8] = {0};
  long long launches = 0;    // kernels queued since creation
  int kernels_per_iter = 0;
  // reference-order schedule
  bool seq = false;
  int *order = nullptr, *lstart = nullptr;  // cells level by level, level starts
  int nlev = 0;
  int *border = nullptr, *blev = nullptr, *wlev = nullptr;  // wall faces, levels, per-wall level ranges
  int coop_vel = 0, coop_p = 0, coop_T = 0;  // cooperative grid sizes
  // nim_gpu_profile_iterations: while set, every kernel launch of an
  // iteration is followed by an event and its name
  struct Marks {
    std::vector<cudaEvent_t> ev;
    std::vector<const char *> name;
    size_t used = 0;
  } *marks = nullptr;
  std::vector<std::string> prof_names;  // names of the last profile
  // mixed precision: the FP32 mirror of every array a parallel pass reads or
  // writes, the graph of FP32 passes, the phase of the current step (1: FP32
  // passes queued, 2: FP64 passes) and the last step's pass count per phase
  bool mixed = false;
  // k_vel_face_tile (TMA-staged z-marching face sweep): whether it runs, its
  // z-chunk length and its tensor maps, one set per storage type
  bool bulk = false;
  int tile_kc = 0;
  VelFaceMaps vmap64{}, vmap32{};
  // k_vel_cell_tile (TMA-staged cell sweep of u, v, w, formulation 2)
  bool cell_tile = false;
  bool cell_pair = false;  // k_vel_cell2: two theta-adjacent cells per thread
  bool cell_quad = false;  // the float mirror's sweeps four cells a thread (k_vel_cellN, k_p_srcN, ...)
  bool face_quad = false;  // and its face sweep of u, v, w as k_vel_faceN
  bool press_pair = false; // the FP64 pressure sweeps two cells a thread (k_p_srcN, k_p_faceN)
  VelCellMaps cmap64{}, cmap32{};
  GeoT<float> g32{};
  FieldsT<float> F32{};
  cudaGraphExec_t graph32 = nullptr;
  int graph32_iters = 0;
  int phase = 0;
  int last_lowp = 0, last_hi = 0;
  // tangent-linear state (nim_gpu_tangent_*): dual copies of the geometry
  // and of the iterate, their own control block and step counter
  bool dual_alloc = false, dual_ready = false;
  GeoT<DualD> gD{};
  FieldsT<DualD> FD{};
  Ctrl *ctlD = nullptr;
  int32_t dual_STEP = 0;
  double dual_TI = 0;
  // z-slab s of slab_count (nim_gpu_create_slab; slab_count 0: the whole
  // mesh): global plane of local plane 0, and per side (0: the slab below,
  // 1: above) whether it has a neighbour and the element spans of its halo
  // exchange (nim_slab_halo)
  int slab_count = 0, slab_index = 0, slab_lo = 0;
  bool halo_ok[2] = {false, false};
  int64_t halo_recv[2][8] = {}, halo_send[2][8] = {};
  // a time step driven without blocking (the synchronous calls and
  // nim_batch_step share it): graph launches so far, the cap, the event that
  // marks the last control-block (or sums) copy
  struct Run {
    long long launched = 0, cap = 0;
    bool capped = false;
    cudaEvent_t ev = nullptr;
  } run;
  // output sets (nim_gpu_output_begin): device staging, copy stream, events
  cudaStream_t copy_stream = nullptr;
  struct Output {
    void *stage = nullptr;
    cudaEvent_t packed = nullptr, copied = nullptr;
    int gen = 0;
  } out[2];
};

namespace {

#define CK(call)                                                   \
  do {                                                             \
    cudaError_t e_ = (call);                                       \
    if (e_ != cudaSuccess) {                                       \
      std::fprintf(stderr, "nim_gpu: %s failed: %s (%s:%d)\n", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
      return NIM_ERR_CUDA;                                         \
    }                                                              \
  } while (0)

template <typename T>
int dalloc(nim_ctx *x, T **p, size_t n) {
  void *q = nullptr;
  CK(cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T)));
  CK(cudaMemsetAsync(q, 0, std::max<size_t>(n, 1) * sizeof(T), x->stream));
  x->allocs.push_back(q);
  *p = static_cast<T *>(q);
  return NIM_OK;
}

#define TRY(call)            \
  do {                       \
    int s_ = (call);         \
    if (s_ != NIM_OK) return s_; \
  } while (0)

inline int grid(int n) { return (n + BLK - 1) / BLK; }

inline double bits_to_double(unsigned long long b) {
  double v;
  std::memcpy(&v, &b, sizeof(v));
  return v;
}

GaussRule make_gauss() {
  GaussRule g;
  g.x[0] = -(1. / 3. * std::sqrt(5. - 2. * std::sqrt(10. / 7.)));
  g.x[1] = 1. / 3. * std::sqrt(5. - 2. * std::sqrt(10. / 7.));
  g.x[2] = 0.;
  g.x[3] = -(1. / 3. * std::sqrt(5. + 2. * std::sqrt(10. / 7.)));
  g.x[4] = 1. / 3. * std::sqrt(5. + 2. * std::sqrt(10. / 7.));
  g.w[0] = (322. + 13. * std::sqrt(70.)) / 900.;
  g.w[1] = (322. + 13. * std::sqrt(70.)) / 900.;
  g.w[2] = 128. / 225.;
  g.w[3] = (322. - 13. * std::sqrt(70.)) / 900.;
  g.w[4] = (322. - 13. * std::sqrt(70.)) / 900.;
  return g;
}

// Check that the reference arrays describe the structured O-grid that
// create_hollow + link_mesh produce, and build the face permutation.
int verify_mesh(const nim_mesh_desc *m, const Dims &d, std::vector<int> &perm) {
  const int NT = d.NT, NR = d.NR, NZ = d.NZ;
  if ((int64_t)NT * (NR + 1) * (NZ + 1) != m->nnode || d.Nc != m->nmesh || d.NF != m->nface || d.NBF != m->nbcface)
    return NIM_ERR_BAD_ARG;
  // The sweep kernels index with 32-bit integers (fewer registers, so fewer
  // spills); their largest offset is 19 x the cell count (MT_A, 18 rows).
  // 2^31 / 20 = 107 M cells is beyond what one GPU's memory holds in FP64.
  if ((int64_t)d.Nc * 20 >= (int64_t)INT32_MAX) return NIM_ERR_BAD_ARG;
  perm.assign(d.NF, -1);
  std::vector<char> seen(d.NF, 0);
  for (int c = 0; c < d.Nc; ++c) {
    const Cell x = Cell::of(d, c);
    const int ip = (x.i == NT - 1) ? 0 : x.i + 1;
    auto node = [&](int i, int j, int k) { return 1 + i + NT * (j + (NR + 1) * k); };
    const int nd[8] = {node(x.i, x.j, x.k),      node(x.i, x.j + 1, x.k),      node(ip, x.j + 1, x.k),
                       node(ip, x.j, x.k),       node(x.i, x.j, x.k + 1),      node(x.i, x.j + 1, x.k + 1),
                       node(ip, x.j + 1, x.k + 1), node(ip, x.j, x.k + 1)};
    for (int n = 0; n < 8; ++n)
      if (m->meshes_nodes[8 * (size_t)c + n] != nd[n]) return NIM_ERR_BAD_ARG;
    for (int pos = 1; pos <= 6; ++pos) {
      const int nb = x.has_nb(d, pos) ? x.nb(d, pos).c + 1 : 0;
      if (m->meshes_neighbors[6 * (size_t)c + pos - 1] != nb) return NIM_ERR_BAD_ARG;
      const int rf = m->meshes_faces[6 * (size_t)c + pos - 1];
      if (rf < 1 || rf > d.NF) return NIM_ERR_BAD_ARG;
      const int sf = x.face(d, pos);
      if (perm[rf - 1] == -1) {
        if (seen[sf]) return NIM_ERR_BAD_ARG;
        perm[rf - 1] = sf;
        seen[sf] = 1;
      } else if (perm[rf - 1] != sf) {
        return NIM_ERR_BAD_ARG;
      }
      const int bc = m->faces_bc[rf - 1];
      if (x.has_nb(d, pos) != (bc == 1)) return NIM_ERR_BAD_ARG;
    }
  }
  for (int f = 0; f < d.NF; ++f)
    if (perm[f] < 0) return NIM_ERR_BAD_ARG;
  for (int b = 0; b < d.NBF; ++b) {
    const BFace B = bface(d, b);
    if (m->bcs_faces_position[b] != B.pos || m->bcs_faces_id[b] != B.id ||
        m->bcs_faces_mesh_num[b] != B.cell.c + 1)
      return NIM_ERR_BAD_ARG;
    const int rf = m->bcs_faces[b];
    if (rf < 1 || rf > d.NF || perm[rf - 1] != B.cell.face(d, B.pos) || m->faces_bc[rf - 1] != B.id)
      return NIM_ERR_BAD_ARG;
  }
  return NIM_OK;
}

Phys make_phys(const nim_params &p) {
  Phys P;
  P.DT = p.DT; P.nu = p.nu; P.alpha = p.alpha; P.rho = p.rho; P.g_beta = p.g_beta;
  P.w[0] = p.w_u; P.w[1] = p.w_v; P.w[2] = p.w_w; P.w[3] = p.w_T;
  P.w_p = p.w_p; P.w_p2 = p.w_p2;
  P.tol[0] = p.tol_u; P.tol[1] = p.tol_v; P.tol[2] = p.tol_w; P.tol[3] = p.tol_p; P.tol[4] = p.tol_T;
  P.v_limit = p.v_limit; P.dudt_epsilon = p.dudt_epsilon; P.R_i = p.R_i; P.R_o = p.R_o;
  const double Re = 1. / p.nu;
  P.inv_Re = 1 / Re;
  P.inv_rho = 1 / p.rho;
  P.max_iters = p.max_iters;
  P.dpdx_tolerance = p.dpdx_tolerance;
  P.formulation = p.formulation;
  P.d_nu = P.d_alpha = P.d_inv_Re = 0.0;  // seeded by nim_gpu_tangent_seed
  return P;
}

// after a kernel launch: an event named for it, when profiling
int mark(nim_ctx *x, const char *name) {
  nim_ctx::Marks *m = x->marks;
  if (!m) return NIM_OK;
  if (m->used == m->ev.size()) {
    cudaEvent_t e;
    CK(cudaEventCreate(&e));
    m->ev.push_back(e);
    m->name.push_back(nullptr);
  }
  m->name[m->used] = name;
  CK(cudaEventRecord(m->ev[m->used++], x->stream));
  return NIM_OK;
}

// the velocity sources + cell kernel and the face kernel of the context's
// formulation (parallel schedule), over arrays of storage type R
template <class R>
int launch_vel(nim_ctx *x, cudaStream_t s, const GeoT<R> &g, const FieldsT<R> &F) {
  const Dims &d = x->d;
  if (x->phys.formulation == 1) {
    k_vel_cell<false, 1><<<x->g3, dim3(CB, 3), 0, s>>>(d, g, F, x->phys, x->ctl);
    TRY(mark(x, "k_vel_cell"));
    k_vel1_face<<<x->g3, dim3(CB, 3), 0, s>>>(d, g, F, x->phys, x->ctl);
    TRY(mark(x, "k_vel1_face"));
  } else {
    if (x->cell_tile) {
      const dim3 gt((d.NT + 31) / 32, (d.NR + CT_R - 1) / CT_R, (d.NZ + x->tile_kc - 1) / x->tile_kc);
      const VelCellMaps &M = std::is_same<R, double>::value ? x->cmap64 : x->cmap32;
      k_vel_cell_tile<R><<<gt, dim3(CT_T, 3), CtLayout<R>::bytes, s>>>(d, g, F, x->phys, x->ctl, x->tile_kc, M);
      TRY(mark(x, "k_vel_cell_tile"));
    } else if (std::is_same<R, float>::value && x->cell_quad) {
      if constexpr (std::is_same<R, float>::value) {
        const dim3 gq((d.NT + 127) / 128, (d.NR + 3) / 4, d.NZ);
        if (x->slab_count)
          k_vel_cellN<R, 4, true><<<gq, dim3(CB, 3), 0, s>>>(d, g, F, x->phys, x->ctl);
        else
          k_vel_cellN<R, 4><<<gq, dim3(CB, 3), 0, s>>>(d, g, F, x->phys, x->ctl);
        TRY(mark(x, "k_vel_cellN"));
      }
    } else if (x->cell_pair) {
      const dim3 gp((d.NT + 63) / 64, (d.NR + 3) / 4, d.NZ);
      if (x->slab_count)
        k_vel_cell2<R, true><<<gp, dim3(CB, 3), 0, s>>>(d, g, F, x->phys, x->ctl);
      else
        k_vel_cell2<R><<<gp, dim3(CB, 3), 0, s>>>(d, g, F, x->phys, x->ctl);
      TRY(mark(x, "k_vel_cell2"));
    } else {
      k_vel_cell<false, 2><<<x->g3, dim3(CB, 3), 0, s>>>(d, g, F, x->phys, x->ctl);
      TRY(mark(x, "k_vel_cell"));
    }
    if (std::is_same<R, float>::value && x->face_quad) {
      if constexpr (std::is_same<R, float>::value) {  // the float mirror, four cells a thread
        const dim3 gq((d.NT + 127) / 128, (d.NR + 3) / 4, d.NZ);
        k_vel_faceN<R, 4><<<gq, dim3(CB, 3), 0, s>>>(d, g, F, x->phys, x->ctl);
        TRY(mark(x, "k_vel_faceN"));
      }
    } else if (x->bulk) {
      const dim3 gt((d.NT + 31) / 32, (d.NR + VT_R - 1) / VT_R, (d.NZ + x->tile_kc - 1) / x->tile_kc);
      const VelFaceMaps &M = std::is_same<R, double>::value ? x->vmap64 : x->vmap32;
      if (x->slab_count)
        k_vel_face_tile<R, true><<<gt, dim3(VT_T, 3), VtLayout<R>::bytes, s>>>(d, g, F, x->phys, x->ctl, x->tile_kc, M);
      else
        k_vel_face_tile<R><<<gt, dim3(VT_T, 3), VtLayout<R>::bytes, s>>>(d, g, F, x->phys, x->ctl, x->tile_kc, M);
      TRY(mark(x, "k_vel_face_tile"));
    } else {
      k_vel_face<<<x->g3, dim3(CB, 3), 0, s>>>(d, g, F, x->phys, x->ctl);
      TRY(mark(x, "k_vel_face"));
    }
  }
  return NIM_OK;
}
// the tangent-linear state (formulation 2): the gather forms of both sweeps
int launch_vel(nim_ctx *x, cudaStream_t s, const GeoT<DualD> &g, const FieldsT<DualD> &F) {
  k_vel_cell<false, 2><<<x->g3, dim3(CB, 3), 0, s>>>(x->d, g, F, x->phys, x->ctl);
  TRY(mark(x, "k_vel_cell"));
  k_vel_face<<<x->g3, dim3(CB, 3), 0, s>>>(x->d, g, F, x->phys, x->ctl);
  TRY(mark(x, "k_vel_face"));
  return NIM_OK;
}

template <typename K>
int launch_coop(K kern, int blocks, dim3 block, nim_ctx *x) {
  Dims d = x->d;
  Geo g = x->g;
  Fields F = x->F;
  Phys P = x->phys;
  Ctrl *ctl = x->ctl;
  const int *order = x->order, *lstart = x->lstart;
  int nlev = x->nlev;
  void *args[] = {&d, &g, &F, &P, &ctl, &order, &lstart, &nlev};
  CK(cudaLaunchCooperativeKernel((const void *)kern, dim3(blocks), block, args, 0, x->stream));
  return NIM_OK;
}

// one pass of integrate_nse's loop body in the reference's order: the source
// kernels store their terms, the sweeps run level by level in place
int launch_iteration_seq(nim_ctx *x) {
  const Dims &d = x->d;
  cudaStream_t s = x->stream;
  if (x->phys.formulation == 1) {
    k_vel_cell<true, 1><<<x->g3, dim3(CB, 3), 0, s>>>(d, x->g, x->F, x->phys, x->ctl);
    TRY(mark(x, "k_vel_cell(src)"));
    TRY(launch_coop(k_seq_vel<1>, x->coop_vel, dim3(CB, 3), x));
  } else {
    k_vel_cell<true, 2><<<x->g3, dim3(CB, 3), 0, s>>>(d, x->g, x->F, x->phys, x->ctl);
    TRY(mark(x, "k_vel_cell(src)"));
    TRY(launch_coop(k_seq_vel<2>, x->coop_vel, dim3(CB, 3), x));
  }
  TRY(mark(x, "k_seq_vel"));
  k_p_src<<<x->g3, dim3(CB, 3), 0, s>>>(d, x->g, x->F, x->phys, x->ctl);
  TRY(mark(x, "k_p_src"));
  k_seq_pbc<<<2, BLK, 0, s>>>(d, x->g, x->F, x->phys, x->ctl, x->border, x->blev, x->wlev, 0);
  k_seq_pbc<<<2, BLK, 0, s>>>(d, x->g, x->F, x->phys, x->ctl, x->border, x->blev, x->wlev, 2);
  TRY(mark(x, "k_seq_pbc"));
  TRY(launch_coop(k_seq_p, x->coop_p, dim3(BLK), x));
  TRY(mark(x, "k_seq_p"));
  if (x->phys.dpdx_tolerance) {
    k_p_dpdx<<<x->nblk_c, BLK, 0, s>>>(d, x->g, x->F, x->ctl);
    TRY(mark(x, "k_p_dpdx"));
  }
  k_zero_flux<<<grid(2 * d.plane), BLK, 0, s>>>(d, x->g, x->F, x->ctl);
  TRY(mark(x, "k_zero_flux"));
  k_T_coef<<<dim3(3, x->nblk_c), BLK, 0, s>>>(d, x->g, x->F, x->phys, x->ctl);
  TRY(mark(x, "k_T_coef"));
  k_T_cell<true><<<x->g3, dim3(CB, 3), 0, s>>>(d, x->g, x->F, x->phys, x->ctl);
  TRY(mark(x, "k_T_cell(src)"));
  TRY(launch_coop(k_seq_T, x->coop_T, dim3(BLK), x));
  TRY(mark(x, "k_seq_T"));
  k_iter_end<<<1, 1, 0, s>>>(x->ctl, x->phys, 0);
  TRY(mark(x, "k_iter_end"));
  CK(cudaGetLastError());
  x->kernels_per_iter = x->phys.dpdx_tolerance ? 12 : 11;
  x->launches += x->kernels_per_iter;
  return NIM_OK;
}

// the pressure part of a parallel pass (nse.f90:150-156)
template <class R>
int launch_pressure(nim_ctx *x, cudaStream_t s, const GeoT<R> &g, const FieldsT<R> &F) {
  const Dims &d = x->d;
  const dim3 g3 = x->g3;
  // the float mirror sweeps four theta-adjacent cells a thread (n_theta % 4
  // == 0), the FP64 path two (n_theta even: double2 loads; measured at C2,
  // k_p_face 154 -> 113 us, k_p_src 160 -> 159 us; the temperature and
  // velocity sweeps stay one cell a thread, their pair forms were slower)
  const bool quad = std::is_same<R, float>::value && x->cell_quad;
  const bool pair = std::is_same<R, double>::value && x->press_pair;
  const dim3 gq((d.NT + 127) / 128, (d.NR + 3) / 4, d.NZ);
  const dim3 gp((d.NT + 63) / 64, (d.NR + 3) / 4, d.NZ);
  if (quad) {
    if constexpr (std::is_same<R, float>::value) {
      k_p_srcN<R, 4><<<gq, dim3(CB, 3), 0, s>>>(d, g, F, x->phys, x->ctl);
      TRY(mark(x, "k_p_srcN"));
    }
  } else if (pair) {
    if constexpr (std::is_same<R, double>::value) {
      k_p_srcN<R, 2><<<gp, dim3(CB, 3), 0, s>>>(d, g, F, x->phys, x->ctl);
      TRY(mark(x, "k_p_srcN"));
    }
  } else {
    k_p_src<<<g3, dim3(CB, 3), 0, s>>>(d, g, F, x->phys, x->ctl);
    TRY(mark(x, "k_p_src"));
  }
  k_p_bc<<<x->nblk_b, BLK, 0, s>>>(d, g, F, x->phys, x->ctl);
  TRY(mark(x, "k_p_bc"));
  k_p_bc_copy<<<x->nblk_b, BLK, 0, s>>>(d, F, x->ctl);
  TRY(mark(x, "k_p_bc_copy"));
  if (quad) {
    if constexpr (std::is_same<R, float>::value) {
      k_p_faceN<R, 4><<<gq, dim3(CB, 3), 0, s>>>(d, g, F, x->phys, x->ctl);
      TRY(mark(x, "k_p_faceN"));
    }
  } else if (pair) {
    if constexpr (std::is_same<R, double>::value) {
      k_p_faceN<R, 2><<<gp, dim3(CB, 3), 0, s>>>(d, g, F, x->phys, x->ctl);
      TRY(mark(x, "k_p_faceN"));
    }
  } else {
    k_p_face<<<g3, dim3(CB, 3), 0, s>>>(d, g, F, x->phys, x->ctl);
    TRY(mark(x, "k_p_face"));
  }
  if (x->phys.dpdx_tolerance) {
    k_p_dpdx<<<x->nblk_c, BLK, 0, s>>>(d, g, F, x->ctl);
    TRY(mark(x, "k_p_dpdx"));
  }
  return NIM_OK;
}

// the temperature part of a parallel pass (nse.f90:157-162)
template <class R>
int launch_temperature(nim_ctx *x, cudaStream_t s, const GeoT<R> &g, const FieldsT<R> &F) {
  const Dims &d = x->d;
  k_zero_flux<<<grid(2 * d.plane), BLK, 0, s>>>(d, g, F, x->ctl);
  TRY(mark(x, "k_zero_flux"));
  k_T_coef<<<dim3(3, x->nblk_c), BLK, 0, s>>>(d, g, F, x->phys, x->ctl);
  TRY(mark(x, "k_T_coef"));
  if constexpr (std::is_same<R, float>::value) {
    if (x->cell_quad) {  // the float mirror: four theta-adjacent cells a thread
      const dim3 gq((d.NT + 127) / 128, (d.NR + 3) / 4, d.NZ);
      k_T_cellN<R, 4><<<gq, dim3(CB, 3), 0, s>>>(d, g, F, x->phys, x->ctl);
      TRY(mark(x, "k_T_cellN"));
      k_T_faceN<R, 4><<<gq, dim3(CB, 3), 0, s>>>(d, g, F, x->phys, x->ctl);
      TRY(mark(x, "k_T_faceN"));
      return NIM_OK;
    }
  }
  k_T_cell<false><<<x->g3, dim3(CB, 3), 0, s>>>(d, g, F, x->phys, x->ctl);
  TRY(mark(x, "k_T_cell"));
  k_T_face<<<x->g8, BLK, 0, s>>>(d, g, F, x->phys, x->ctl);
  TRY(mark(x, "k_T_face"));
  return NIM_OK;
}

// one pass of the parallel schedule over arrays of storage type R
template <class R>
int launch_parallel(nim_ctx *x, const GeoT<R> &g, const FieldsT<R> &F, int lowp) {
  cudaStream_t s = x->stream;
  TRY(launch_vel(x, s, g, F));
  TRY(launch_pressure(x, s, g, F));
  TRY(launch_temperature(x, s, g, F));
  k_iter_end<<<1, 1, 0, s>>>(x->ctl, x->phys, lowp);
  TRY(mark(x, "k_iter_end"));
  CK(cudaGetLastError());
  x->kernels_per_iter = x->phys.dpdx_tolerance ? 12 : 11;
  x->launches += x->kernels_per_iter;
  return NIM_OK;
}

// one pass of integrate_nse's loop body; lowp: over the FP32 mirror, and
// with stall_rule the pass ends the FP32 phase once the changes stop falling
int launch_iteration(nim_ctx *x, bool lowp = false, bool stall_rule = true) {
  if (x->seq) return launch_iteration_seq(x);
  return lowp ? launch_parallel(x, x->g32, x->F32, stall_rule ? 1 : 0) : launch_parallel(x, x->g, x->F, 0);
}

int build_graph(nim_ctx *x, int iters, bool lowp = false) {
  cudaGraphExec_t &exec = lowp ? x->graph32 : x->graph;
  if (exec) {
    cudaGraphExecDestroy(exec);
    exec = nullptr;
  }
  cudaGraph_t g = nullptr;
  const long long before = x->launches;
  CK(cudaStreamBeginCapture(x->stream, cudaStreamCaptureModeThreadLocal));
  for (int k = 0; k < iters; ++k) {
    const int st = launch_iteration(x, lowp);
    if (st != NIM_OK) {
      cudaStreamEndCapture(x->stream, &g);
      if (g) cudaGraphDestroy(g);
      return st;
    }
  }
  CK(cudaStreamEndCapture(x->stream, &g));
  x->launches = before;
  cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return NIM_ERR_CUDA;
  (lowp ? x->graph32_iters : x->graph_iters) = iters;
  return NIM_OK;
}

// ---- the FP32 mirror of a mixed-precision context
struct Cvt {
  CvtList L{};
  int k = 0;
  long long nmax = 0;
  template <class S, class D>
  void add(const S *src, D *dst, size_t n) {
    L.src[k] = src;
    L.dst[k] = dst;
    L.n[k] = (long long)n;
    nmax = std::max(nmax, (long long)n);
    ++k;
  }
};
template <class S, class D>
int run_cvt(nim_ctx *x, const Cvt &c) {
  if (c.k == 0) return NIM_OK;
  if (c.k > CvtList::kMax) return NIM_ERR_BAD_ARG;
  const long long blocks = std::min<long long>((c.nmax + BLK - 1) / BLK, 148LL * 8);
  k_convert<S, D><<<dim3((unsigned)std::max(1LL, blocks), c.k), BLK, 0, x->stream>>>(c.L);
  CK(cudaGetLastError());
  x->launches += 1;
  return NIM_OK;
}

// geometry (once, after nim_gpu_init's metric kernels)
int mirror_geometry(nim_ctx *x) {
  const Dims &d = x->d;
  const size_t Nc = d.Nc, NF = d.NF, NB = d.NBF;
  const Geo &g = x->g;
  GeoT<float> &h = x->g32;
  Cvt c;
  c.add(g.vol, h.vol, Nc);
  c.add(g.G, h.G, 3 * Nc);
  c.add(g.gij, h.gij, 9 * Nc);
  c.add(g.xi, h.xi, 9 * Nc);
  c.add(g.gfd, h.gfd, 6 * Nc);
  c.add(g.dg, h.dg, 6 * Nc);
  c.add(g.area, h.area, NF);
  c.add(g.normal, h.normal, 3 * NF);
  c.add(g.AA, h.AA, 45 * Nc);
  c.add(g.bca, h.bca, 5 * NB);
  c.add(g.bcap, h.bcap, 8 * NB);
  c.add(g.bcg, h.bcg, 2 * NB);
  c.add(g.zf, h.zf, 4 * NB);
  TRY((run_cvt<double, float>(x, c)));
  // 1/vol in float from the float volumes: the float sweeps' own division
  k_reciprocal<float><<<x->nblk_c, BLK, 0, x->stream>>>(h.vol, h.rvol, d.Nc);
  CK(cudaGetLastError());
  x->launches += 1;
  return NIM_OK;
}

// velocity NIM constants (every step, after nim_gpu_begin_step's kernels)
int mirror_step_coefficients(nim_ctx *x) {
  const size_t Nc = x->d.Nc;
  Cvt c;
  c.add(x->F.MF4, x->F32.MF4, 8 * Nc);
  c.add(x->F.MF, x->F32.MF, 15 * Nc);
  return run_cvt<double, float>(x, c);
}

// the iterate: both halves of the face fields (wall values live in both),
// cell fields, old cell fields, dpdx_old; dir 0 narrows, 1 widens (the old
// cell fields only narrow: the passes do not write them)
int mirror_state(nim_ctx *x, int dir) {
  const size_t Nc = x->d.Nc, NF = x->d.NF;
  const Fields &F = x->F;
  const FieldsT<float> &H = x->F32;
  Cvt c;
  if (dir == 0) {
    for (int q = 0; q < 5; ++q) c.add(F.f[q], H.f[q], 2 * NF);
    for (int q = 0; q < 4; ++q) c.add(F.c[q], H.c[q], Nc);
    for (int q = 0; q < 4; ++q) c.add(F.co[q], H.co[q], Nc);
    c.add(F.dpd, H.dpd, 3 * Nc);
    return run_cvt<double, float>(x, c);
  }
  for (int q = 0; q < 5; ++q) c.add(H.f[q], F.f[q], 2 * NF);
  for (int q = 0; q < 4; ++q) c.add(H.c[q], F.c[q], Nc);
  c.add(H.dpd, F.dpd, 3 * Nc);
  return run_cvt<float, double>(x, c);
}

int read_ctrl(nim_ctx *x) {
  CK(cudaMemcpyAsync(x->ctl_host, x->ctl, sizeof(Ctrl), cudaMemcpyDeviceToHost, x->stream));
  CK(cudaStreamSynchronize(x->stream));
  return NIM_OK;
}

__global__ void k_step_reset(Ctrl *ctl) {
  ctl->done = 0;
  ctl->step_iters = 0;
  ctl->status = 0;
  for (int q = 0; q < 4; ++q) ctl->red[q] = 0ull;
}

// pmask: 1 double-buffers the face fields (parallel schedule), 0 keeps one
// half that the reference-order sweeps update in place
__global__ void k_run_reset(Ctrl *ctl, int pmask) {
  ctl->pmask = pmask;
  for (int p = 0; p < 2; ++p)
    for (int q = 0; q < 8; ++q) ctl->err[p][q] = 0ull;
  for (int q = 0; q < 8; ++q) ctl->wall_floor[q] = 0ull;
  ctl->iter = 0;
  ctl->step_iters = 0;
  ctl->done = 0;
  ctl->status = 0;
  ctl->first = 1;
}

// dst[i*K + k] = src[k*stride + (perm ? perm[i] : i)]
__global__ void k_gather(const double *__restrict__ src, size_t stride, int K, const int *__restrict__ perm, int n,
                         double *__restrict__ dst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int s = perm ? perm[i] : i;
  for (int k = 0; k < K; ++k) dst[(size_t)i * K + k] = src[(size_t)k * stride + s];
}
__global__ void k_scatter(const double *__restrict__ src, const int *__restrict__ perm, int n, double *dst0,
                          double *dst1) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int s = perm ? perm[i] : i;
  dst0[s] = src[i];
  if (dst1) dst1[s] = src[i];
}

// write_data's zone variables as REAL(.,4) (postprocess.f90:92-103)
__global__ void k_pack_plot(Dims d, Fields F, float *__restrict__ dst) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.Nc) return;
  const size_t Nc = d.Nc;
  dst[c] = (float)F.ct[0][c];
  dst[Nc + c] = (float)F.ct[1][c];
  dst[2 * Nc + c] = (float)F.ct[2][c];
  dst[3 * Nc + c] = (float)F.mp[c];
  dst[4 * Nc + c] = (float)F.ct[3][c];
  dst[5 * Nc + c] = (float)F.dila[c];
}

// write_restart's arrays (restart.f90:24-37): five face fields of the
// current half in reference face order, then nine cell fields
__global__ void k_pack_restart(Dims d, Fields F, const int *__restrict__ perm, const Ctrl *ctl,
                               double *__restrict__ dst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const size_t NF = d.NF, Nc = d.Nc;
  const int par = ctl->iter & ctl->pmask;
  if (i < d.NF) {
    const int s = perm[i];
    for (int q = 0; q < 5; ++q) dst[q * NF + i] = F.f[q][par * NF + s];
  }
  if (i < d.Nc) {
    double *o = dst + 5 * NF;
    for (int q = 0; q < 4; ++q) o[q * Nc + i] = F.c[q][i];
    for (int q = 0; q < 4; ++q) o[(4 + q) * Nc + i] = F.co[q][i];
    o[8 * Nc + i] = F.dila_old[i];
  }
}

struct FieldView {
  const double *src = nullptr;
  double *dst1 = nullptr;  // second half (face fields)
  size_t stride = 0;
  int K = 1, n = 0;
  bool face = false, writable = false;
};

int field_view(nim_ctx *x, nim_field f, int par, FieldView &v) {
  const Dims &d = x->d;
  const size_t Nc = d.Nc, NF = d.NF, NB = d.NBF;
  auto cellf = [&](double *p) { v.src = p; v.n = d.Nc; v.stride = Nc; v.writable = true; };
  switch (f) {
    case NIM_FIELD_FACES_U: case NIM_FIELD_FACES_V: case NIM_FIELD_FACES_W: case NIM_FIELD_FACES_P:
    case NIM_FIELD_FACES_T: {
      double *base = x->F.f[(int)f];
      v.src = base + par * NF;
      v.dst1 = base + (1 - par) * NF;
      v.n = d.NF; v.stride = NF; v.face = true; v.writable = true;
      return NIM_OK;
    }
    case NIM_FIELD_MESHES_U: case NIM_FIELD_MESHES_V: case NIM_FIELD_MESHES_W: case NIM_FIELD_MESHES_T:
      cellf(x->F.c[(int)f - 5]); return NIM_OK;
    case NIM_FIELD_MESHES_U_OLD: case NIM_FIELD_MESHES_V_OLD: case NIM_FIELD_MESHES_W_OLD:
    case NIM_FIELD_MESHES_T_OLD:
      cellf(x->F.co[(int)f - 9]); return NIM_OK;
    case NIM_FIELD_MESHES_UT: case NIM_FIELD_MESHES_VT: case NIM_FIELD_MESHES_WT: case NIM_FIELD_MESHES_TT:
      cellf(x->F.ct[(int)f - 13]); return NIM_OK;
    case NIM_FIELD_MESHES_P: cellf(x->F.mp); return NIM_OK;
    case NIM_FIELD_MESHES_DILA: cellf(x->F.dila); return NIM_OK;
    case NIM_FIELD_MESHES_DILA_OLD: cellf(x->F.dila_old); return NIM_OK;
    default: break;
  }
  v.writable = false;
  switch (f) {
    case NIM_FIELD_MESHES_VOLUME: v.src = x->g.vol; v.n = d.Nc; v.stride = Nc; return NIM_OK;
    case NIM_FIELD_FACES_AREA: v.src = x->g.area; v.n = d.NF; v.stride = NF; v.face = true; return NIM_OK;
    case NIM_FIELD_FACES_NORMAL: v.src = x->g.normal; v.n = d.NF; v.stride = NF; v.K = 3; v.face = true; return NIM_OK;
    case NIM_FIELD_FACES_MID: v.src = x->g.mid; v.n = d.NF; v.stride = NF; v.K = 3; v.face = true; return NIM_OK;
    case NIM_FIELD_FACES_TANGENTIAL: v.src = x->g.tang; v.n = d.NF; v.stride = NF; v.K = 3; v.face = true; return NIM_OK;
    case NIM_FIELD_FACES_BITANGENTIAL: v.src = x->g.bitang; v.n = d.NF; v.stride = NF; v.K = 3; v.face = true; return NIM_OK;
    case NIM_FIELD_MESHES_GIJ: v.src = x->g.gij; v.n = d.Nc; v.stride = Nc; v.K = 9; return NIM_OK;
    case NIM_FIELD_MESHES_XI_X: v.src = x->g.xi; v.n = d.Nc; v.stride = Nc; v.K = 9; return NIM_OK;
    case NIM_FIELD_MESHES_G: v.src = x->g.G; v.n = d.Nc; v.stride = Nc; v.K = 3; return NIM_OK;
    case NIM_FIELD_MESHES_GIJ_FACES: v.src = x->g.gf; v.n = d.Nc; v.stride = Nc; v.K = 54; return NIM_OK;
    case NIM_FIELD_BCS_FACES_A: v.src = x->g.bca; v.n = d.NBF; v.stride = NB; v.K = 5; return NIM_OK;
    case NIM_FIELD_BCS_FACES_AP: v.src = x->g.bcap; v.n = d.NBF; v.stride = NB; v.K = 8; return NIM_OK;
    case NIM_FIELD_AA_PX: v.src = x->g.AA; v.n = d.Nc; v.stride = Nc; v.K = 15; return NIM_OK;
    case NIM_FIELD_AA_PY: v.src = x->g.AA + 15 * Nc; v.n = d.Nc; v.stride = Nc; v.K = 15; return NIM_OK;
    case NIM_FIELD_AA_PZ: v.src = x->g.AA + 30 * Nc; v.n = d.Nc; v.stride = Nc; v.K = 15; return NIM_OK;
    case NIM_FIELD_M_F4: v.src = x->F.MF4; v.n = d.Nc; v.stride = Nc; v.K = 8; return NIM_OK;
    case NIM_FIELD_M_F1: v.src = x->F.MF; v.n = d.Nc; v.stride = Nc; v.K = 5; return NIM_OK;
    case NIM_FIELD_M_F2: v.src = x->F.MF + 5 * Nc; v.n = d.Nc; v.stride = Nc; v.K = 5; return NIM_OK;
    case NIM_FIELD_M_F3: v.src = x->F.MF + 10 * Nc; v.n = d.Nc; v.stride = Nc; v.K = 5; return NIM_OK;
    default: return NIM_ERR_BAD_ARG;
  }
}

}  // namespace

// =================================================================== C ABI
extern "C" void nim_params_reference(nim_params *p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  const double Ra = 1.0E5, Pr = 0.7, g_beta = 1., th_tc = 1.;  // parameters.f90:166-170
  p->DT = 0.01;
  p->nu = 1. / std::sqrt(Ra / (g_beta * th_tc * Pr));
  p->alpha = p->nu / Pr;
  p->rho = 1.0;
  p->g_beta = g_beta;
  p->w_u = p->w_v = p->w_w = p->w_p = p->w_p2 = p->w_T = .4;
  p->tol_u = p->tol_v = p->tol_w = p->tol_T = 1E-6;
  p->tol_p = 5E-3;
  p->v_limit = 1E-2;
  p->dudt_epsilon = 1E-5;
  p->R_i = 1.0 * (MATH_PI / 3.0);
  p->R_o = 2.0;
  p->bc_value[4][3] = 1.;  // T = 1 on BC 4 (general.f90:96-97)
  p->max_iters = 100000;
  p->check_steady = 1;
  p->dpdx_tolerance = 0;
  p->formulation = 2;  // parameters.f90:194
}

extern "C" const char *nim_gpu_strerror(int s) {
  switch (s) {
    case NIM_OK: return "ok";
    case NIM_ERR_BAD_ARG: return "bad argument or unsupported mesh";
    case NIM_ERR_CUDA: return "CUDA runtime error";
    case NIM_ERR_NOT_CONVERGED: return "inner iteration reached max_iters";
    case NIM_ERR_NONFINITE: return "non-finite value in the iteration";
    case NIM_ERR_TIMEOUT: return "device wait timed out";
    case NIM_ERR_STATE: return "call out of order";
    default: return "unknown status";
  }
}

// Looks up the device address of g_noalloc_scratch with `device` current.
// nim_gpu_create calls it first (so the lookup, which may load the module,
// happens before any stream capture) and nim_gpu_nusselt_noalloc again on
// every call: after a device reset or a new primary context the module is
// loaded afresh and an address kept from before would dangle.  The lookup
// allocates nothing.
static int noalloc_setup(int device) {
  if (device < 0 || device >= kMaxDevices) return NIM_ERR_BAD_ARG;
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  void *ptr = nullptr;
  CK(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));  // the current device's copy
  g_noalloc_ptr[device] = static_cast<double *>(ptr);
  return NIM_OK;
}

// Level orders of the reference-order sweeps.  Cells: level i + 2j + 3k,
// which every dependence of a sweep crosses in the direction of the cell
// numbers (the argument is in nim_kernels.cuh).  Wall faces, in BC-list
// order bottom, top, inner, outer: level i + 2j on bottom and top, i + 2k on
// inner and outer.  Also the sweep buffers and the cooperative grid sizes.
static int setup_levels(nim_ctx *x) {
  const Dims &d = x->d;
  const size_t Nc = d.Nc;
  TRY(dalloc(x, &x->F.MTF4, 8 * Nc));
  TRY(dalloc(x, &x->F.RDT, Nc));
  // counting sort of the cells by level
  const int nlev = (d.NT - 1) + 2 * (d.NR - 1) + 3 * (d.NZ - 1) + 1;
  std::vector<int> lstart(nlev + 1, 0), order(Nc), fill;
  for (int c = 0; c < d.Nc; ++c) {
    const Cell q = Cell::of(d, c);
    ++lstart[q.i + 2 * q.j + 3 * q.k + 1];
  }
  int maxlev = 0;
  for (int L = 0; L < nlev; ++L) {
    maxlev = std::max(maxlev, lstart[L + 1]);
    lstart[L + 1] += lstart[L];
  }
  fill.assign(lstart.begin(), lstart.end() - 1);
  for (int c = 0; c < d.Nc; ++c) {
    const Cell q = Cell::of(d, c);
    order[fill[q.i + 2 * q.j + 3 * q.k]++] = c;
  }
  // wall faces: per wall, counting sort by the in-wall level
  const int nb1 = d.NT * d.NR, nb3 = d.NT * d.NZ;
  const int w0[4] = {0, nb1, 2 * nb1, 2 * nb1 + nb3}, wn[4] = {nb1, nb1, nb3, nb3};
  const int wl[4] = {d.NT + 2 * (d.NR - 1), d.NT + 2 * (d.NR - 1), d.NT + 2 * (d.NZ - 1), d.NT + 2 * (d.NZ - 1)};
  std::vector<int> border(d.NBF), blev(1, 0), wlev(1, 0);
  int q = 0;
  for (int w = 0; w < 4; ++w) {
    std::vector<int> cnt(wl[w] + 1, 0);
    for (int r = 0; r < wn[w]; ++r) ++cnt[r % d.NT + 2 * (r / d.NT) + 1];
    for (int L = 0; L < wl[w]; ++L) cnt[L + 1] += cnt[L];
    std::vector<int> pos(cnt.begin(), cnt.end() - 1);
    for (int r = 0; r < wn[w]; ++r) border[q + pos[r % d.NT + 2 * (r / d.NT)]++] = w0[w] + r;
    for (int L = 1; L <= wl[w]; ++L) blev.push_back(q + cnt[L]);
    q += wn[w];
    wlev.push_back((int)blev.size() - 1);
  }
  x->nlev = nlev;
  TRY(dalloc(x, &x->order, Nc));
  TRY(dalloc(x, &x->lstart, (size_t)nlev + 1));
  TRY(dalloc(x, &x->border, (size_t)d.NBF));
  TRY(dalloc(x, &x->blev, blev.size()));
  TRY(dalloc(x, &x->wlev, wlev.size()));
  CK(cudaMemcpy(x->order, order.data(), sizeof(int) * Nc, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(x->lstart, lstart.data(), sizeof(int) * (nlev + 1), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(x->border, border.data(), sizeof(int) * d.NBF, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(x->blev, blev.data(), sizeof(int) * blev.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(x->wlev, wlev.data(), sizeof(int) * wlev.size(), cudaMemcpyHostToDevice));
  // cooperative grids: no more blocks than the widest level needs, and no
  // more than can be resident at once (cudaLaunchCooperativeKernel rejects
  // a larger grid rather than running it)
  int sms = 0, coop = 0;
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, x->device));
  CK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, x->device));
  if (!coop) return NIM_ERR_CUDA;
  const int want = std::max(1, (maxlev + BLK - 1) / BLK);
  int per = 0;
  if (x->phys.formulation == 1)
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_seq_vel<1>, CB3, 0));
  else
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_seq_vel<2>, CB3, 0));
  x->coop_vel = std::max(1, std::min((maxlev + CB - 1) / CB, per * sms));
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_seq_p, BLK, 0));
  x->coop_p = std::max(1, std::min(want, per * sms));
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_seq_T, BLK, 0));
  x->coop_T = std::max(1, std::min(want, per * sms));
  if (x->coop_vel < 1 || x->coop_p < 1 || x->coop_T < 1) return NIM_ERR_CUDA;
  return NIM_OK;
}

// ---- tensor maps of k_vel_face_tile (cuTensorMapEncodeTiled through the
// runtime's driver entry point: no link against the driver library)
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(f);
  });
  return fn;
}

// rank-dimensional map of a dense array starting at base: dims[0] fastest,
// strides of dims 1.. in elements, box in elements; out-of-range elements
// of a box read as zero
template <class R>
static bool encode_map(CUtensorMap *map, const R *base, int rank, const uint64_t *dims, const uint64_t *strides,
                       const uint32_t *box) {
  EncodeTiledFn fn = encode_tiled();
  if (!fn) return false;
  cuuint64_t gd[5], gs[4];
  cuuint32_t bx[5], es[5];
  for (int i = 0; i < rank; ++i) {
    gd[i] = dims[i];
    bx[i] = box[i];
    es[i] = 1;
  }
  for (int i = 0; i + 1 < rank; ++i) gs[i] = strides[i] * sizeof(R);
  const CUtensorMapDataType t = sizeof(R) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  return fn(map, t, (cuuint32_t)rank, const_cast<R *>(base), gd, gs, bx, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <class R>
static bool encode_vel_face_maps(const Dims &d, const GeoT<R> &g, const FieldsT<R> &F, VelFaceMaps &M) {
  const uint64_t NT = d.NT, NR = d.NR, NZ = d.NZ, NF = d.NF, Nc = d.Nc;
  bool ok = true;
  for (int q = 0; q < 3; ++q) {
    const uint64_t dr[4] = {NT, NR + 1, NZ, 2}, sr[3] = {NT, NT * (NR + 1), NF};
    const uint32_t br[4] = {(uint32_t)VtLayout<R>::W, VT_R + 2, 1, 1};
    ok = ok && encode_map(&M.rf[q], F.f[q], 4, dr, sr, br);
    const uint64_t dt[4] = {NT, NR, NZ, 2}, dz[4] = {NT, NR, NZ + 1, 2}, st[3] = {NT, NT * NR, NF};
    const uint32_t bt[4] = {(uint32_t)VtLayout<R>::W, VT_R + 1, 1, 1};
    ok = ok && encode_map(&M.tf[q], F.f[q] + d.offT, 4, dt, st, bt);
    ok = ok && encode_map(&M.zf[q], F.f[q] + d.offZ, 4, dz, st, bt);
    const uint64_t dc[3] = {NT, NR, NZ}, sc[2] = {NT, NT * NR};
    const uint32_t bc[3] = {(uint32_t)VtLayout<R>::W, VT_R + 1, 1};
    ok = ok && encode_map(&M.cv[q], F.c[q], 3, dc, sc, bc);
    ok = ok && encode_map(&M.co[q], F.co[q], 3, dc, sc, bc);
  }
  const uint64_t dm[4] = {NT, NR, NZ, 15}, dgd[4] = {NT, NR, NZ, 6}, sm[3] = {NT, NT * NR, Nc};
  const uint32_t bm[4] = {32, VT_R, 1, 15}, bg[4] = {32, VT_R, 1, 6};
  ok = ok && encode_map(&M.mf, F.MF, 4, dm, sm, bm);
  ok = ok && encode_map(&M.dg, g.dg, 4, dgd, sm, bg);
  return ok;
}

template <class R>
static bool encode_vel_cell_maps(const Dims &d, const FieldsT<R> &F, VelCellMaps &M) {
  const uint64_t NT = d.NT, NR = d.NR, NZ = d.NZ, NF = d.NF;
  bool ok = true;
  for (int q = 0; q < 3; ++q) {
    const uint64_t dr[4] = {NT, NR + 1, NZ, 2}, sr[3] = {NT, NT * (NR + 1), NF};
    const uint64_t dt[4] = {NT, NR, NZ, 2}, dz[4] = {NT, NR, NZ + 1, 2}, st[3] = {NT, NT * NR, NF};
    const uint32_t br[4] = {(uint32_t)CtLayout<R>::W, CT_R + 1, 1, 1};
    const uint32_t bt[4] = {(uint32_t)CtLayout<R>::W, CT_R + 4, 1, 1};
    ok = ok && encode_map(&M.rf[q], F.f[q], 4, dr, sr, br);
    ok = ok && encode_map(&M.tf[q], F.f[q] + d.offT, 4, dt, st, bt);
    ok = ok && encode_map(&M.zf[q], F.f[q] + d.offZ, 4, dz, st, bt);
  }
  return ok;
}

// The +xi face sweep of u, v, w runs as k_vel_face_tile when n_theta is a
// multiple of 4 (16-byte box rows), at most 256, and the mesh by itself
// gives at least four waves of blocks (fewer, and the 109 KB blocks cost
// more than they save: at 96x96x64, and for the enclosures of a batch that
// share the GPU); the z-chunk length aims at about six waves of blocks with
// chunks of at least 8 planes.  NIM_FACE_SWEEP=tile or =gather in the
// environment forces the choice (tile still needs the n_theta conditions).
// The source and cell sweep of u, v, w (formulation 2) runs as k_vel_cell2
// (two theta-adjacent cells per thread, paired loads) when n_theta is even,
// and for the float mirror as k_vel_cellN (four cells a thread, float4
// loads) when n_theta % 4 == 0; NIM_CELL_SWEEP=gather forces k_vel_cell,
// =pair k_vel_cell2 (and the float mirror's other sweeps in their
// one-cell forms), =quad the four-cell forms on any n_theta % 4 == 0,
// =tile k_vel_cell_tile (under the tile's n_theta conditions).  The float mirror's face sweep of u, v, w runs four cells a
// thread as well (k_vel_faceN) unless NIM_FACE_SWEEP names a form.
static int choose_face_sweep(nim_ctx *x) {
  const Dims &d = x->d;
  int sms = 0;
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, x->device));
  const int tiles = ((d.NT + 31) / 32) * ((d.NR + VT_R - 1) / VT_R);
  const int want = (6 * sms + tiles - 1) / tiles;
  const int nch = std::max(1, std::min(want, d.NZ / 8));
  x->tile_kc = (d.NZ + nch - 1) / nch;
  const int blocks = tiles * ((d.NZ + x->tile_kc - 1) / x->tile_kc);
  const bool shape = (d.NT % 4 == 0) && d.NT <= 256;
  const char *env = std::getenv("NIM_FACE_SWEEP");
  const std::string force = env ? env : "";
  x->bulk = shape && !x->seq && (force == "tile" || (force != "gather" && blocks >= 4 * sms));
  // the staged cell sweep only on request: its u, v, w faces are a sixth of
  // k_vel_cell's bytes, and the two 110 KB blocks per SM it needs leave the
  // direct loads of the rest with fewer warps than the gather form has
  const char *envc = std::getenv("NIM_CELL_SWEEP");
  const std::string cell = envc ? envc : "";
  x->cell_tile = shape && !x->seq && x->params.formulation == 2 && cell == "tile";
  // the paired-load form whenever n_theta is even, unless another is asked for;
  // the float mirror's sweeps four cells a thread when n_theta % 4 == 0
  x->cell_pair = !x->cell_tile && d.NT % 2 == 0 && !x->seq && x->params.formulation == 2 && cell != "gather";
  // the NP-cells-a-thread sweeps run a row of n_theta / NP threads per
  // theta row of the patch; below 3/4 of the warp's lanes (small meshes,
  // the enclosures of a batch) the idle lanes cost more than the wider
  // loads save.  NIM_CELL_SWEEP=quad / =pair force them.
  auto lane_use = [&](int np) {
    const int lanes = d.NT / np;
    return (double)lanes / (32.0 * ((lanes + 31) / 32));
  };
  x->cell_quad = x->cell_pair && d.NT % 4 == 0 && cell != "pair" && (cell == "quad" || lane_use(4) >= 0.75);
  x->face_quad = x->cell_quad && force != "tile" && force != "gather";
  x->press_pair = x->cell_pair && (cell == "pair" || cell == "quad" || lane_use(2) >= 0.75);
  return NIM_OK;
}

// ---- z-slabs: the cell planes split into nslab contiguous runs of at least
// two planes; each slab's context also holds the two planes either side that
// a neighbour owns (its halo): no stencil of an owned cell or of a face of
// one reaches further (the two-cell chains exist only at the physical walls,
// nse.f90:1638-1639, bc.f90:345-390).
extern "C" int nim_slab_layout(int32_t n_z, int32_t nslab, int32_t s, int32_t *out4) {
  if (!out4 || nslab < 1 || s < 0 || s >= nslab || n_z < 3 || n_z / nslab < 2) return NIM_ERR_BAD_ARG;
  const int32_t base = n_z / nslab, rem = n_z % nslab;
  const int32_t own_lo = s * base + std::min(s, rem);
  const int32_t own_hi = own_lo + base + (s < rem ? 1 : 0);
  out4[0] = std::max(0, own_lo - 2);
  out4[1] = std::min(n_z, own_hi + 2);
  out4[2] = own_lo;
  out4[3] = own_hi;
  return NIM_OK;
}

extern "C" int nim_slab_halo(int32_t n_theta, int32_t n_r, int32_t n_z, int32_t nslab, int32_t s, int32_t side,
                             int64_t *recv8, int64_t *send8) {
  int32_t lay[4];
  if (!recv8 || !send8 || n_theta < 1 || n_r < 1 || (side != 0 && side != 1)) return NIM_ERR_BAD_ARG;
  TRY(nim_slab_layout(n_z, nslab, s, lay));
  if ((side == 0 && s == 0) || (side == 1 && s == nslab - 1)) return NIM_ERR_BAD_ARG;
  const int64_t NT = n_theta, NR = n_r, NZl = lay[1] - lay[0], pl = NT * NR;
  const int64_t offT = NT * (NR + 1) * NZl, offZ = offT + pl * NZl;
  // planes [g0, g0 + 2) of the slab with the z-face rows z0, z0 + 1.  The
  // cut face between two slabs is left out: each computes it from its own
  // first halo plane, so no span written in an exchange is read in it.
  auto spans = [&](int64_t g0, int64_t z0, int64_t *o) {
    const int64_t l0 = g0 - lay[0];
    o[0] = l0 * pl;                o[1] = 2 * pl;
    o[2] = NT * (NR + 1) * l0;     o[3] = 2 * NT * (NR + 1);
    o[4] = offT + l0 * pl;         o[5] = 2 * pl;
    o[6] = offZ + (z0 - lay[0]) * pl;  o[7] = 2 * pl;
  };
  const int64_t olo = lay[2], ohi = lay[3];
  if (side == 0) {
    spans(olo - 2, olo - 2, recv8);  // rows olo-2 (the end face), olo-1
    spans(olo, olo + 1, send8);      // the lower neighbour's rows past its cut
  } else {
    spans(ohi, ohi + 1, recv8);      // rows ohi+1, ohi+2 (the end face)
    spans(ohi - 2, ohi - 2, send8);
  }
  return NIM_OK;
}

// slab: null for the whole mesh, else {nslab, s}: the context holds z-slab s
// of nslab (nim_slab_layout) with its halo planes
static int create_impl(const nim_mesh_desc *m, const nim_params *p, nim_ctx *x, const int32_t *slab = nullptr) {
  CK(cudaGetDevice(&x->device));
  TRY(noalloc_setup(x->device));
  CK(cudaStreamCreateWithFlags(&x->stream, cudaStreamNonBlocking));
  CK(cudaStreamCreateWithFlags(&x->copy_stream, cudaStreamNonBlocking));
  CK(cudaEventCreateWithFlags(&x->run.ev, cudaEventDisableTiming));
  x->d = make_dims(m->n_theta, m->n_r, m->n_z);
  std::vector<int> perm;
  TRY(verify_mesh(m, x->d, perm));
  const double *node_xyz = m->node_xyz;
  int64_t nnode = m->nnode;
  if (slab) {
    // the slab's planes as a cylinder of their own; its faces and cells in
    // the library's structured order (the identity permutation)
    int32_t lay[4];
    TRY(nim_slab_layout(m->n_z, slab[0], slab[1], lay));
    if (p->schedule == NIM_SCHEDULE_REFERENCE || p->formulation == 1 || p->precision == NIM_PRECISION_MIXED)
      return NIM_ERR_BAD_ARG;
    const int NT = m->n_theta, NR = m->n_r;
    x->d = make_dims(NT, NR, lay[1] - lay[0]);
    x->d.kown0 = lay[2] - lay[0];
    x->d.kown1 = lay[3] - lay[0];
    x->slab_count = slab[0];
    x->slab_index = slab[1];
    x->slab_lo = lay[0];
    node_xyz += 3 * (size_t)NT * (NR + 1) * lay[0];
    nnode = (int64_t)NT * (NR + 1) * (x->d.NZ + 1);
    perm.resize(x->d.NF);
    for (int f = 0; f < x->d.NF; ++f) perm[f] = f;
    for (int side = 0; side < 2; ++side)
      x->halo_ok[side] = nim_slab_halo(NT, NR, m->n_z, slab[0], slab[1], side, x->halo_recv[side],
                                       x->halo_send[side]) == NIM_OK;
  }
  const Dims &d = x->d;
  x->params = *p;
  x->seq = (p->schedule == NIM_SCHEDULE_REFERENCE);
  TRY(choose_face_sweep(x));
  if (slab) x->cell_tile = false;  // its maxima are not masked per plane
  x->phys = make_phys(*p);
  x->gq = make_gauss();
  x->nblk_c = grid(d.Nc);
  x->nblk_b = grid(d.NBF);
  x->nblk_c3 = (d.Nc + CB - 1) / CB;
  x->g3 = dim3((d.NT + 31) / 32, (d.NR + 3) / 4, d.NZ);
  x->g8 = dim3((d.NT + 31) / 32, (d.NR + 7) / 8, d.NZ);
  const size_t Nc = d.Nc, NF = d.NF, NB = d.NBF;
  Geo &g = x->g;
  TRY(dalloc(x, &g.vol, Nc));
  TRY(dalloc(x, &g.rvol, Nc));
  TRY(dalloc(x, &g.G, 3 * Nc));
  TRY(dalloc(x, &g.gij, 9 * Nc));
  TRY(dalloc(x, &g.xi, 9 * Nc));
  TRY(dalloc(x, &g.gf, 54 * Nc));
  TRY(dalloc(x, &g.gfd, 6 * Nc));
  TRY(dalloc(x, &g.dg, 6 * Nc));
  TRY(dalloc(x, &g.area, NF));
  TRY(dalloc(x, &g.normal, 3 * NF));
  TRY(dalloc(x, &g.mid, 3 * NF));
  TRY(dalloc(x, &g.tang, 3 * NF));
  TRY(dalloc(x, &g.bitang, 3 * NF));
  TRY(dalloc(x, &g.AA, 45 * Nc));
  TRY(dalloc(x, &g.bcpts, 5 * NB));
  TRY(dalloc(x, &g.bca, 5 * NB));
  TRY(dalloc(x, &g.bcap, 8 * NB));
  TRY(dalloc(x, &g.bcg, 2 * NB));
  TRY(dalloc(x, &g.zf, 4 * NB));
  TRY(dalloc(x, &g.nuw, 4 * NB));
  TRY(dalloc(x, &g.bcval, 4 * NB));
  Fields &F = x->F;
  for (int q = 0; q < 5; ++q) TRY(dalloc(x, &F.f[q], 2 * NF));
  for (int q = 0; q < 4; ++q) {
    TRY(dalloc(x, &F.c[q], Nc));
    TRY(dalloc(x, &F.co[q], Nc));
    TRY(dalloc(x, &F.ct[q], Nc));
  }
  TRY(dalloc(x, &F.mp, Nc));
  TRY(dalloc(x, &F.dila, Nc));
  TRY(dalloc(x, &F.dila_old, Nc));
  TRY(dalloc(x, &F.Rp, Nc));
  TRY(dalloc(x, &F.MA, 18 * Nc));
  TRY(dalloc(x, &F.MF4, 8 * Nc));
  TRY(dalloc(x, &F.MF, 15 * Nc));
  TRY(dalloc(x, &F.MTF, 15 * Nc));
  TRY(dalloc(x, &F.MTA, 18 * Nc));
  if (x->seq || p->formulation == 1) TRY(dalloc(x, &F.Bv, 3 * Nc));
  if (p->formulation == 1) {
    TRY(dalloc(x, &F.N1, 22 * Nc));
    TRY(dalloc(x, &F.AT, 9 * Nc));
    TRY(dalloc(x, &F.AAv, 45 * Nc));
  }
  TRY(dalloc(x, &F.dpd, 3 * Nc));
  x->mixed = (p->precision == NIM_PRECISION_MIXED);
  if (x->mixed) {
    GeoT<float> &h = x->g32;
    TRY(dalloc(x, &h.vol, Nc));
    TRY(dalloc(x, &h.rvol, Nc));
    TRY(dalloc(x, &h.G, 3 * Nc));
    TRY(dalloc(x, &h.gij, 9 * Nc));
    TRY(dalloc(x, &h.xi, 9 * Nc));
    TRY(dalloc(x, &h.gfd, 6 * Nc));
    TRY(dalloc(x, &h.dg, 6 * Nc));
    TRY(dalloc(x, &h.area, NF));
    TRY(dalloc(x, &h.normal, 3 * NF));
    TRY(dalloc(x, &h.AA, 45 * Nc));
    h.bcpts = g.bcpts;  // integer: shared with the FP64 side
    TRY(dalloc(x, &h.bca, 5 * NB));
    TRY(dalloc(x, &h.bcap, 8 * NB));
    TRY(dalloc(x, &h.bcg, 2 * NB));
    TRY(dalloc(x, &h.zf, 4 * NB));
    FieldsT<float> &H = x->F32;
    for (int q = 0; q < 5; ++q) TRY(dalloc(x, &H.f[q], 2 * NF));
    for (int q = 0; q < 4; ++q) {
      TRY(dalloc(x, &H.c[q], Nc));
      TRY(dalloc(x, &H.co[q], Nc));
    }
    TRY(dalloc(x, &H.dila, Nc));
    TRY(dalloc(x, &H.Rp, Nc));
    TRY(dalloc(x, &H.MF4, 8 * Nc));
    TRY(dalloc(x, &H.MF, 15 * Nc));
    TRY(dalloc(x, &H.MTF, 15 * Nc));
    TRY(dalloc(x, &H.MTA, 18 * Nc));
    TRY(dalloc(x, &H.dpd, 3 * Nc));
  }
  TRY(dalloc(x, &F.part, 8 * (size_t)std::max(x->nblk_c, grid(2 * d.NT * d.NZ))));
  TRY(dalloc(x, &x->ctl, 1));
  TRY(dalloc(x, &x->node_xyz, 3 * (size_t)nnode));
  TRY(dalloc(x, &x->bcv, 25));
  TRY(dalloc(x, &x->perm, NF));
  TRY(dalloc(x, &x->scratch, std::max(54 * Nc, 3 * NF)));
  TRY(dalloc(x, &x->sums, 8));
  CK(cudaMallocHost(&x->ctl_host, sizeof(Ctrl)));
  if (x->cell_tile) {
    x->cell_tile = encode_vel_cell_maps(d, x->F, x->cmap64) &&
                   (!x->mixed || encode_vel_cell_maps(d, x->F32, x->cmap32));
    if (x->cell_tile) {
      CK(cudaFuncSetAttribute(k_vel_cell_tile<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)CtLayout<double>::bytes));
      CK(cudaFuncSetAttribute(k_vel_cell_tile<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)CtLayout<float>::bytes));
    }
  }
  if (x->bulk && !x->seq) {
    x->bulk = encode_vel_face_maps(d, x->g, x->F, x->vmap64) &&
              (!x->mixed || encode_vel_face_maps(d, x->g32, x->F32, x->vmap32));
    if (x->bulk) {
      CK(cudaFuncSetAttribute(k_vel_face_tile<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)VtLayout<double>::bytes));
      CK(cudaFuncSetAttribute(k_vel_face_tile<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)VtLayout<float>::bytes));
      CK(cudaFuncSetAttribute(k_vel_face_tile<double, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)VtLayout<double>::bytes));
      CK(cudaFuncSetAttribute(k_vel_face_tile<float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)VtLayout<float>::bytes));
    }
  }
  if (x->seq) TRY(setup_levels(x));
  CK(cudaMemcpyAsync(x->node_xyz, node_xyz, 3 * sizeof(double) * nnode, cudaMemcpyHostToDevice, x->stream));
  double bcv[25];
  for (int f = 0; f < 5; ++f)
    for (int b = 0; b < 5; ++b) bcv[5 * f + b] = p->bc_value[f][b];
  CK(cudaMemcpyAsync(x->bcv, bcv, sizeof(bcv), cudaMemcpyHostToDevice, x->stream));
  CK(cudaMemcpyAsync(x->perm, perm.data(), sizeof(int) * NF, cudaMemcpyHostToDevice, x->stream));
  CK(cudaStreamSynchronize(x->stream));
  return NIM_OK;
}

static int create_checked(const nim_mesh_desc *m, const nim_params *p, nim_ctx **out, const int32_t *slab) {
  if (!m || !p || !out || !m->node_xyz || !m->meshes_nodes || !m->meshes_faces || !m->meshes_neighbors ||
      !m->faces_bc || !m->bcs_faces || !m->bcs_faces_id || !m->bcs_faces_position || !m->bcs_faces_mesh_num)
    return NIM_ERR_BAD_ARG;
  if (m->n_theta < 6 || m->n_r < 3 || m->n_z < 3) return NIM_ERR_BAD_ARG;
  if ((int64_t)m->n_theta * m->n_r * m->n_z > (int64_t)INT32_MAX / 4) return NIM_ERR_BAD_ARG;
  if (!(p->DT > 0) || !(p->nu > 0) || !(p->alpha > 0) || !(p->rho > 0)) return NIM_ERR_BAD_ARG;
  if (p->schedule != NIM_SCHEDULE_PARALLEL && p->schedule != NIM_SCHEDULE_REFERENCE) return NIM_ERR_BAD_ARG;
  if (p->formulation != 1 && p->formulation != 2) return NIM_ERR_BAD_ARG;
  if (p->precision != NIM_PRECISION_FP64 && p->precision != NIM_PRECISION_MIXED) return NIM_ERR_BAD_ARG;
  // the FP32 phase exists for the parallel schedule of formulation 2
  if (p->precision == NIM_PRECISION_MIXED && (p->schedule != NIM_SCHEDULE_PARALLEL || p->formulation != 2))
    return NIM_ERR_BAD_ARG;
  *out = nullptr;
  nim_ctx *x = new (std::nothrow) nim_ctx();
  if (!x) return NIM_ERR_BAD_ARG;
  const int st = create_impl(m, p, x, slab);
  if (st != NIM_OK) {
    nim_gpu_destroy(x);
    return st;
  }
  *out = x;
  return NIM_OK;
}

extern "C" int nim_gpu_create(const nim_mesh_desc *m, const nim_params *p, nim_ctx **out) {
  return create_checked(m, p, out, nullptr);
}

extern "C" int nim_gpu_create_slab(const nim_mesh_desc *m, const nim_params *p, int32_t nslab, int32_t s,
                                   nim_ctx **out) {
  const int32_t slab[2] = {nslab, s};
  return create_checked(m, p, out, slab);
}

extern "C" int nim_gpu_init(nim_ctx *x) {
  if (!x) return NIM_ERR_BAD_ARG;
  CK(cudaSetDevice(x->device));
  const Dims &d = x->d;
  cudaStream_t s = x->stream;
  k_run_reset<<<1, 1, 0, s>>>(x->ctl, x->seq ? 0 : 1);
  k_cell_geometry<<<x->nblk_c, BLK, 0, s>>>(d, x->gq, x->node_xyz, x->g);
  k_metric_derived<<<x->nblk_c, BLK, 0, s>>>(d, x->g);
  k_reciprocal<double><<<x->nblk_c, BLK, 0, s>>>(x->g.vol, x->g.rvol, d.Nc);
  k_pressure_coeffs<<<x->nblk_c, BLK, 0, s>>>(d, x->g, x->params.rho);
  k_bc_geometry<<<x->nblk_b, BLK, 0, s>>>(d, x->gq, x->node_xyz, x->g, x->params.rho, x->bcv);
  // initial conditions: zero (general.f90:16-31), then the Dirichlet faces
  const size_t Nc = d.Nc, NF = d.NF;
  for (int q = 0; q < 5; ++q) CK(cudaMemsetAsync(x->F.f[q], 0, 2 * NF * sizeof(double), s));
  for (int q = 0; q < 4; ++q) {
    CK(cudaMemsetAsync(x->F.c[q], 0, Nc * sizeof(double), s));
    CK(cudaMemsetAsync(x->F.co[q], 0, Nc * sizeof(double), s));
    CK(cudaMemsetAsync(x->F.ct[q], 0, Nc * sizeof(double), s));
  }
  CK(cudaMemsetAsync(x->F.dpd, 0, 3 * Nc * sizeof(double), s));
  CK(cudaMemsetAsync(x->F.dila, 0, Nc * sizeof(double), s));
  CK(cudaMemsetAsync(x->F.dila_old, 0, Nc * sizeof(double), s));
  CK(cudaMemsetAsync(x->F.mp, 0, Nc * sizeof(double), s));
  k_apply_dirichlet<<<x->nblk_b, BLK, 0, s>>>(d, x->g, x->F);
  k_wall_floor<<<x->nblk_b, BLK, 0, s>>>(d, x->g, x->ctl);
  CK(cudaGetLastError());
  if (x->mixed) TRY(mirror_geometry(x));
  CK(cudaStreamSynchronize(s));
  x->TI = x->params.DT;  // nse.f90:31
  x->STEP = 1;           // nse.f90:32
  x->initialized = true;
  x->in_step = false;
  x->last_iters = 0;
  x->last_lowp = x->last_hi = 0;
  return NIM_OK;
}

extern "C" int nim_gpu_begin_step(nim_ctx *x) {
  if (!x) return NIM_ERR_BAD_ARG;
  if (!x->initialized) return NIM_ERR_STATE;
  const Dims &d = x->d;
  k_step_reset<<<1, 1, 0, x->stream>>>(x->ctl);
  if (x->phys.formulation == 1) {  // calculate_velocity_nim_constants (nim.f90:17-157)
    k_vel1_coef_A<<<x->nblk_c, BLK, 0, x->stream>>>(d, x->g, x->F, x->phys);
    k_vel1_coef_F<<<x->nblk_c, BLK, 0, x->stream>>>(d, x->g, x->F, x->phys);
  } else {
    k_vel_coef_A<<<x->nblk_c, BLK, 0, x->stream>>>(d, x->g, x->F, x->phys);
    k_vel_coef_F<<<x->nblk_c, BLK, 0, x->stream>>>(d, x->F, x->phys);
  }
  CK(cudaGetLastError());
  x->launches += 3;
  if (x->mixed) TRY(mirror_step_coefficients(x));
  x->in_step = true;
  return NIM_OK;
}

static int fill_iter_stats(nim_ctx *x, nim_step_stats *s) {
  if (!s) return NIM_OK;
  const Ctrl &c = *x->ctl_host;
  s->step = x->STEP;
  s->iters = c.step_iters;
  s->err_u = c.last_err[0];
  s->err_v = c.last_err[1];
  s->err_w = c.last_err[2];
  s->err_p = c.last_err[3];
  s->err_T = c.last_err[4];
  s->status = c.status;
  s->iters_fp32 = x->mixed ? c.lowp_iters : 0;
  return NIM_OK;
}

// a slab of a split mesh advances only with its neighbours (nim_slab_step,
// nim_slab_part): alone its halo would go stale
static bool lone_slab(const nim_ctx *x) { return x->slab_count > 1; }

extern "C" int nim_gpu_iterate(nim_ctx *x, int32_t n, nim_step_stats *s) {
  if (!x || n < 0 || lone_slab(x)) return NIM_ERR_BAD_ARG;
  if (!x->initialized) return NIM_ERR_STATE;
  // fixed number of passes: keep the stop flag clear and the cap out of reach
  const Phys keep = x->phys;
  x->phys.max_iters = 0;
  for (int q = 0; q < 5; ++q) x->phys.tol[q] = -1.0;
  int st = NIM_OK;
  k_step_reset<<<1, 1, 0, x->stream>>>(x->ctl);
  for (int k = 0; k < n && st == NIM_OK; ++k) st = launch_iteration(x);
  x->phys = keep;
  TRY(st);
  TRY(read_ctrl(x));
  fill_iter_stats(x, s);
  return x->ctl_host->status;
}

// ---- the inner loop and the step end as non-blocking pieces.  Each piece
// queues work on the context's stream and ends with an event (run.ev) the
// caller waits for (cudaEventSynchronize) or polls (cudaEventQuery).
namespace {
int ctrl_async(nim_ctx *x) {
  CK(cudaMemcpyAsync(x->ctl_host, x->ctl, sizeof(Ctrl), cudaMemcpyDeviceToHost, x->stream));
  CK(cudaEventRecord(x->run.ev, x->stream));
  return NIM_OK;
}

int iterations_launch(nim_ctx *x, int batches) {
  const int G = x->graph_G;
  if (x->seq) {
    for (int k = 0; k < batches * G; ++k) TRY(launch_iteration(x));
  } else {
    cudaGraphExec_t graph = (x->phase == 1) ? x->graph32 : x->graph;
    for (int k = 0; k < batches; ++k) CK(cudaGraphLaunch(graph, x->stream));
    x->launches += (long long)batches * G * x->kernels_per_iter;
  }
  x->run.launched += (long long)batches * G;
  return ctrl_async(x);
}

// check_steady_state and evaluate_D after the inner loop (nse.f90:167-168),
// queued with the copy of the control block
int after_loop_start(nim_ctx *x) {
  const Dims &d = x->d;
  k_after_integrate<<<x->nblk_c, BLK, 0, x->stream>>>(d, x->g, x->F, x->phys, x->ctl, x->nblk_c);
  k_finish_sum<<<1, BLK, 0, x->stream>>>(x->F.part, x->nblk_c, 1, x->sums);
  CK(cudaGetLastError());
  x->launches += 2;
  CK(cudaMemcpyAsync(x->host_sums, x->sums, sizeof(double), cudaMemcpyDeviceToHost, x->stream));
  return ctrl_async(x);
}

// integrate_nse, first batch: launch ahead by the previous step's count
int integrate_start(nim_ctx *x) {
  const int G = x->graph_G;
  if (!x->seq && (!x->graph || x->graph_iters != G)) TRY(build_graph(x, G));
  if (x->mixed && (!x->graph32 || x->graph32_iters != G)) TRY(build_graph(x, G, true));
  // with max_iters <= 0 the device never stops on its own; bound the host loop
  x->run.cap = (x->params.max_iters > 0) ? (long long)x->params.max_iters + 2 * G : 100000000LL;
  x->run.launched = 0;
  x->run.capped = false;
  if (x->mixed) {  // FP32 phase from the narrowed FP64 iterate
    TRY(mirror_state(x, 0));
    k_lowp_begin<<<1, 1, 0, x->stream>>>(x->ctl);
    CK(cudaGetLastError());
    x->launches += 1;
    x->phase = 1;
    return iterations_launch(x, std::max(1, (x->last_lowp * 7 / 8) / G));
  }
  x->phase = 0;
  return iterations_launch(x, std::max(1, (x->last_iters * 7 / 8) / G));
}

// after run.ev: 1 = more iterations queued; 0 = the loop has stopped and
// the end-of-loop reductions are queued (wait for run.ev again)
int integrate_advance(nim_ctx *x) {
  if (!x->ctl_host->done) {
    if (x->run.launched < x->run.cap) {
      TRY(iterations_launch(x, 1));
      return 1;
    }
    x->run.capped = true;
  } else if (x->phase == 1 && x->ctl_host->status == NIM_OK) {
    // FP32 phase over: widen its iterate, FP64 passes to the reference's test
    TRY(mirror_state(x, 1));
    k_lowp_end<<<1, 1, 0, x->stream>>>(x->ctl);
    CK(cudaGetLastError());
    x->launches += 1;
    x->phase = 2;
    TRY(iterations_launch(x, std::max(1, (x->last_hi * 7 / 8) / x->graph_G)));
    return 1;
  }
  TRY(after_loop_start(x));
  return 0;
}

int integrate_finish(nim_ctx *x, nim_step_stats *s) {
  const Dims &d = x->d;
  x->last_iters = x->ctl_host->step_iters;
  if (x->mixed) {
    x->last_lowp = x->ctl_host->lowp_iters;
    x->last_hi = x->ctl_host->step_iters - x->ctl_host->lowp_iters;
  }
  x->phase = 0;
  if (x->run.capped && x->ctl_host->status == NIM_OK) x->ctl_host->status = NIM_ERR_NOT_CONVERGED;
  if (s) {
    fill_iter_stats(x, s);
    s->dilatation = std::sqrt(x->host_sums[0] / d.Nc);
    s->dudt_max = bits_to_double(x->ctl_host->red[0]);
    s->dTdt_max = bits_to_double(x->ctl_host->red[1]);
  }
  return x->ctl_host->status;
}

// update_time_step + find_Nu2 (nse.f90:72-73), queued
int end_start(nim_ctx *x) {
  const Dims &d = x->d;
  const int nr = 2 * d.NT * d.NZ, gn = grid(nr);
  k_update_time<<<x->nblk_c, BLK, 0, x->stream>>>(d, x->F, x->ctl);
  k_nusselt<<<gn, BLK, 0, x->stream>>>(d, x->g, x->F, x->ctl, gn);
  k_finish_sum<<<1, BLK, 0, x->stream>>>(x->F.part, gn, 4, x->sums);
  CK(cudaGetLastError());
  x->launches += 3;
  CK(cudaMemcpyAsync(x->host_sums, x->sums, 4 * sizeof(double), cudaMemcpyDeviceToHost, x->stream));
  CK(cudaEventRecord(x->run.ev, x->stream));
  return NIM_OK;
}

void end_finish(nim_ctx *x, nim_step_stats *s) {
  const int32_t step_done = x->STEP;
  x->STEP = x->STEP + 1;                 // nse.f90:1295
  x->TI = x->TI + 2 * x->params.DT;      // nse.f90:1296
  x->in_step = false;
  if (s) {
    const double sum1 = x->host_sums[0], sumA1 = x->host_sums[1], sum2 = x->host_sums[2], sumA2 = x->host_sums[3];
    s->step = step_done;
    s->nu_outer = -(sum1 / sumA1 * x->params.R_o);  // nse.f90:2794, printed Nu_H
    s->nu_inner = -(sum2 / sumA2 * x->params.R_i);  // printed Nu_C (hot hexagon)
    s->area_outer = sumA1;
    s->area_inner = sumA2;
    s->time = x->TI;
  }
}

// the steady-state exit of the time loop (nse.f90:60-69)
bool steady_exit(const nim_ctx *x, const nim_step_stats &rec) {
  return x->params.check_steady && rec.dudt_max < x->params.dudt_epsilon && rec.dTdt_max < x->params.dudt_epsilon;
}
}  // namespace

extern "C" int nim_gpu_set_graph_iters(nim_ctx *x, int32_t n) {
  if (!x || n < 1 || n > 256) return NIM_ERR_BAD_ARG;
  if (x->in_step) return NIM_ERR_STATE;
  x->graph_G = n;  // the graph is rebuilt at the next integrate
  return NIM_OK;
}

extern "C" int nim_gpu_integrate(nim_ctx *x, nim_step_stats *s) {
  if (!x || lone_slab(x)) return NIM_ERR_BAD_ARG;
  if (!x->initialized || !x->in_step) return NIM_ERR_STATE;
  TRY(integrate_start(x));
  for (;;) {
    CK(cudaEventSynchronize(x->run.ev));
    const int r = integrate_advance(x);
    if (r < 0) return r;
    if (r == 0) break;
  }
  CK(cudaEventSynchronize(x->run.ev));
  return integrate_finish(x, s);
}

extern "C" int nim_gpu_end_step(nim_ctx *x, nim_step_stats *s) {
  if (!x) return NIM_ERR_BAD_ARG;
  if (!x->initialized || !x->in_step) return NIM_ERR_STATE;
  TRY(end_start(x));
  CK(cudaEventSynchronize(x->run.ev));
  end_finish(x, s);
  return NIM_OK;
}

extern "C" int nim_gpu_step(nim_ctx *x, int32_t nsteps, nim_step_stats *per, int32_t *done) {
  if (!x || nsteps < 0 || lone_slab(x)) return NIM_ERR_BAD_ARG;
  if (!x->initialized) return NIM_ERR_STATE;
  int32_t k = 0;
  int st = NIM_OK;
  for (; k < nsteps; ++k) {
    nim_step_stats rec;
    std::memset(&rec, 0, sizeof(rec));
    TRY(nim_gpu_begin_step(x));
    st = nim_gpu_integrate(x, &rec);
    rec.status = st;
    if (st != NIM_OK) {
      x->in_step = false;
      if (per) per[k] = rec;
      ++k;
      break;
    }
    // steady-state exit of the time loop (nse.f90:60-69)
    if (steady_exit(x, rec)) {
      rec.steady = 1;
      x->in_step = false;
      if (per) per[k] = rec;
      ++k;
      break;
    }
    const int st2 = nim_gpu_end_step(x, &rec);
    if (per) per[k] = rec;
    if (st2 != NIM_OK) {
      st = st2;
      ++k;
      break;
    }
  }
  if (done) *done = k;
  return st;
}

// nim_gpu_step for several contexts at once: one host thread keeps every
// context's stream fed, polling their events instead of waiting on any, so
// the kernels of all instances share the GPU.  Per instance the calls and
// their order are exactly nim_gpu_step's.
extern "C" int nim_batch_step(int32_t n, nim_ctx *const *ctx, int32_t nsteps, nim_step_stats *per, int32_t *done) {
  if (n <= 0 || !ctx || nsteps < 0) return NIM_ERR_BAD_ARG;
  for (int32_t i = 0; i < n; ++i) {
    if (!ctx[i] || lone_slab(ctx[i])) return NIM_ERR_BAD_ARG;
    if (!ctx[i]->initialized || ctx[i]->in_step) return NIM_ERR_STATE;
    if (ctx[i]->device != ctx[0]->device) return NIM_ERR_BAD_ARG;
    for (int32_t j = 0; j < i; ++j)
      if (ctx[j] == ctx[i]) return NIM_ERR_BAD_ARG;
  }
  if (done)
    for (int32_t i = 0; i < n; ++i) done[i] = 0;
  if (nsteps == 0) return NIM_OK;
  CK(cudaSetDevice(ctx[0]->device));
  enum { ITER, AFTER, END, FINISHED };
  std::vector<int> phase(n, ITER), k(n, 0);
  std::vector<nim_step_stats> rec(n);
  int first_error = NIM_OK;
  auto start_step = [&](int32_t i) -> int {
    std::memset(&rec[i], 0, sizeof(nim_step_stats));
    TRY(nim_gpu_begin_step(ctx[i]));
    phase[i] = ITER;
    return integrate_start(ctx[i]);
  };
  auto finish = [&](int32_t i, int st) -> int {
    if (per) per[(size_t)i * nsteps + k[i]] = rec[i];
    ++k[i];
    if (done) done[i] = k[i];
    if (st != NIM_OK && first_error == NIM_OK) first_error = st;
    if (st != NIM_OK || rec[i].steady || k[i] == nsteps) {
      phase[i] = FINISHED;
      return NIM_OK;
    }
    return start_step(i);
  };
  for (int32_t i = 0; i < n; ++i) TRY(start_step(i));
  int left = n;
  while (left > 0) {
    bool moved = false;
    for (int32_t i = 0; i < n; ++i) {
      nim_ctx *x = ctx[i];
      if (phase[i] == FINISHED) continue;
      const cudaError_t q = cudaEventQuery(x->run.ev);
      if (q == cudaErrorNotReady) continue;
      CK(q);
      moved = true;
      if (phase[i] == ITER) {
        const int r = integrate_advance(x);
        if (r < 0) return r;
        if (r == 0) phase[i] = AFTER;
      } else if (phase[i] == AFTER) {
        const int st = integrate_finish(x, &rec[i]);
        rec[i].status = st;
        if (st != NIM_OK) {
          x->in_step = false;
          TRY(finish(i, st));
        } else if (steady_exit(x, rec[i])) {
          rec[i].steady = 1;
          x->in_step = false;
          TRY(finish(i, NIM_OK));
        } else {
          TRY(end_start(x));
          phase[i] = END;
        }
      } else {  // END
        end_finish(x, &rec[i]);
        TRY(finish(i, NIM_OK));
      }
      if (phase[i] == FINISHED) --left;
    }
    if (!moved) std::this_thread::yield();
  }
  return first_error;
}

// ---- a batch in fused launches (nim_batch_step_fused): every kernel of a
// pass launched once for all the batch's enclosures (nim_batch.cuh)
namespace {
struct FusedBatch {
  int n = 0;
  bool mixed = false;
  int G = 4;  // passes per graph launch
  bool wide = false;  // batched kernels at one resident block per SM fewer
  // NIM_BATCH_FORM=grid: plain launches over groups of kGroup enclosures
  // whose arguments are kernel parameters (kg_*), one per slot and group,
  // the groups rebuilt from the enclosures iterating in each precision
  bool grid_form = false;
  std::vector<BatchGroup<float>> grp32[BS_COUNT];
  std::vector<BatchGroup<double>> grp64[BS_COUNT];
  std::vector<BatchGrid> grids;  // [2][n][BS_COUNT]
  std::vector<BatchInst<double>> h64;
  std::vector<BatchInst<float>> h32;
  cudaStream_t s = nullptr;
  BatchArgs args{};
  void *dev = nullptr;                // tables, phases, work list, states
  int *phase_host = nullptr;          // pinned
  BatchState *state_host = nullptr;   // pinned
  bool use[2][BS_COUNT] = {};         // per phase (float, double): slots some enclosure runs
  int blocks[2][BS_COUNT] = {};       // persistent grid of each slot's kernel
  cudaGraphExec_t graph[3] = {nullptr, nullptr, nullptr};  // passes over phases {FP32}, {FP64}, both
  std::vector<nim_ctx *> ctx;
  std::vector<cudaStream_t> own;      // the contexts' streams, back in place at the end
  size_t state_dev_offset = 0;
  ~FusedBatch() {
    if (s) cudaStreamSynchronize(s);
    for (size_t i = 0; i < own.size(); ++i) ctx[i]->stream = own[i];
    for (auto &g : graph)
      if (g) cudaGraphExecDestroy(g);
    if (dev) cudaFree(dev);
    if (phase_host) cudaFreeHost(phase_host);
    if (state_host) cudaFreeHost(state_host);
    if (s) cudaStreamDestroy(s);
  }
};

template <class K>
int persistent_blocks(K kern, int threads, int sms, int &out) {
  int nb = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, threads, 0));
  out = std::max(1, nb) * sms;
  return NIM_OK;
}

template <class R, int W>
int fused_occupancy(FusedBatch &B, int sms) {
  constexpr int ph = sizeof(R) == 4 ? 0 : 1;
  int *b = B.blocks[ph];
  TRY(persistent_blocks(kb_vel_cell2<R, W>, CB3, sms, b[BS_VEL_CELL2]));
  TRY(persistent_blocks(kb_vel_cell<R, W>, CB3, sms, b[BS_VEL_CELL]));
  TRY(persistent_blocks(kb_vel_face<R, W>, CB3, sms, b[BS_VEL_FACE]));
  if constexpr (ph == 1) {
    TRY(persistent_blocks(kb_p_src2<W>, CB3, sms, b[BS_P_SRC2]));
    TRY(persistent_blocks(kb_p_face2<W>, CB3, sms, b[BS_P_FACE2]));
  }
  TRY(persistent_blocks(kb_p_src<R, W>, CB3, sms, b[BS_P_SRC]));
  TRY(persistent_blocks(kb_p_bc<R, W>, BLK, sms, b[BS_P_BC]));
  TRY(persistent_blocks(kb_p_bc_copy<R, W>, BLK, sms, b[BS_P_BC_COPY]));
  TRY(persistent_blocks(kb_p_face<R, W>, CB3, sms, b[BS_P_FACE]));
  TRY(persistent_blocks(kb_p_dpdx<R, W>, BLK, sms, b[BS_P_DPDX]));
  TRY(persistent_blocks(kb_zero_flux<R, W>, BLK, sms, b[BS_ZERO_FLUX]));
  TRY(persistent_blocks(kb_T_coef<R, W>, BLK, sms, b[BS_T_COEF]));
  TRY(persistent_blocks(kb_T_cell<R, W>, CB3, sms, b[BS_T_CELL]));
  TRY(persistent_blocks(kb_T_face<R, W>, BLK, sms, b[BS_T_FACE]));
  return NIM_OK;
}

// the slots of one storage type, in launch_parallel's order
template <class R, int W>
int fused_slots(FusedBatch &B) {
  constexpr int ph = sizeof(R) == 4 ? 0 : 1;
  const bool *u = B.use[ph];
  const int *b = B.blocks[ph];
  const dim3 t3(CB, 3);
  cudaStream_t s = B.s;
  const BatchArgs &A = B.args;
  if (u[BS_VEL_CELL2]) kb_vel_cell2<R, W><<<b[BS_VEL_CELL2], t3, 0, s>>>(A);
  if (u[BS_VEL_CELL]) kb_vel_cell<R, W><<<b[BS_VEL_CELL], t3, 0, s>>>(A);
  if (u[BS_VEL_FACE]) kb_vel_face<R, W><<<b[BS_VEL_FACE], t3, 0, s>>>(A);
  if constexpr (ph == 1) {
    if (u[BS_P_SRC2]) kb_p_src2<W><<<b[BS_P_SRC2], t3, 0, s>>>(A);
  }
  if (u[BS_P_SRC]) kb_p_src<R, W><<<b[BS_P_SRC], t3, 0, s>>>(A);
  if (u[BS_P_BC]) kb_p_bc<R, W><<<b[BS_P_BC], BLK, 0, s>>>(A);
  if (u[BS_P_BC_COPY]) kb_p_bc_copy<R, W><<<b[BS_P_BC_COPY], BLK, 0, s>>>(A);
  if constexpr (ph == 1) {
    if (u[BS_P_FACE2]) kb_p_face2<W><<<b[BS_P_FACE2], t3, 0, s>>>(A);
  }
  if (u[BS_P_FACE]) kb_p_face<R, W><<<b[BS_P_FACE], t3, 0, s>>>(A);
  if (u[BS_P_DPDX]) kb_p_dpdx<R, W><<<b[BS_P_DPDX], BLK, 0, s>>>(A);
  if (u[BS_ZERO_FLUX]) kb_zero_flux<R, W><<<b[BS_ZERO_FLUX], BLK, 0, s>>>(A);
  if (u[BS_T_COEF]) kb_T_coef<R, W><<<b[BS_T_COEF], BLK, 0, s>>>(A);
  if (u[BS_T_CELL]) kb_T_cell<R, W><<<b[BS_T_CELL], t3, 0, s>>>(A);
  if (u[BS_T_FACE]) kb_T_face<R, W><<<b[BS_T_FACE], BLK, 0, s>>>(A);
  CK(cudaGetLastError());
  return NIM_OK;
}
template <class R>
int fused_slots_of(FusedBatch &B) {
  return B.wide ? fused_slots<R, 1>(B) : fused_slots<R, 0>(B);
}

// one slot's launch over one group of enclosures (NIM_BATCH_FORM=grid)
template <class R>
void group_launch(int slot, const BatchGroup<R> &L, cudaStream_t s) {
  const unsigned nb = L.off[L.n];
  const dim3 t3(CB, 3);
  switch (slot) {
    case BS_VEL_CELL2: kg_vel_cell2<R><<<nb, t3, 0, s>>>(L); break;
    case BS_VEL_CELL: kg_vel_cell<R><<<nb, t3, 0, s>>>(L); break;
    case BS_VEL_FACE: kg_vel_face<R><<<nb, t3, 0, s>>>(L); break;
    case BS_P_SRC: kg_p_src<R><<<nb, t3, 0, s>>>(L); break;
    case BS_P_BC: kg_p_bc<R><<<nb, BLK, 0, s>>>(L); break;
    case BS_P_BC_COPY: kg_p_bc_copy<R><<<nb, BLK, 0, s>>>(L); break;
    case BS_P_FACE: kg_p_face<R><<<nb, t3, 0, s>>>(L); break;
    case BS_P_DPDX: kg_p_dpdx<R><<<nb, BLK, 0, s>>>(L); break;
    case BS_ZERO_FLUX: kg_zero_flux<R><<<nb, BLK, 0, s>>>(L); break;
    case BS_T_COEF: kg_T_coef<R><<<nb, BLK, 0, s>>>(L); break;
    case BS_T_CELL: kg_T_cell<R><<<nb, t3, 0, s>>>(L); break;
    case BS_T_FACE: kg_T_face<R><<<nb, BLK, 0, s>>>(L); break;
    default:
      if constexpr (std::is_same<R, double>::value) {
        if (slot == BS_P_SRC2) kg_p_src2<<<nb, t3, 0, s>>>(L);
        if (slot == BS_P_FACE2) kg_p_face2<<<nb, t3, 0, s>>>(L);
      }
  }
}
template <class R>
int group_slots(FusedBatch &B) {
  constexpr int ph = sizeof(R) == 4 ? 0 : 1;
  for (int q = 0; q < BS_COUNT; ++q) {
    if (!B.use[ph][q]) continue;
    if constexpr (ph == 0) {
      for (const auto &L : B.grp32[q]) group_launch<float>(q, L, B.s);
    } else {
      for (const auto &L : B.grp64[q]) group_launch<double>(q, L, B.s);
    }
  }
  CK(cudaGetLastError());
  return NIM_OK;
}

// the groups of the enclosures whose phase is ph + 1 (host copy of the
// phases), per slot
void fused_groups(FusedBatch &B, const int *phase) {
  for (int q = 0; q < BS_COUNT; ++q) {
    B.grp32[q].clear();
    B.grp64[q].clear();
  }
  for (int ph = 0; ph < 2; ++ph) {
    std::vector<int> mem;
    for (int i = 0; i < B.n; ++i)
      if (phase[i] == ph + 1) mem.push_back(i);
    for (int q = 0; q < BS_COUNT; ++q) {
      if (!B.use[ph][q]) continue;
      for (size_t g0 = 0; g0 < mem.size(); g0 += kGroup) {
        const int m = (int)std::min<size_t>(kGroup, mem.size() - g0);
        auto fill = [&](auto &L, const auto &h) {
          L.n = m;
          L.ph = ph + 1;
          L.phase = B.args.phase;
          unsigned acc = 0;
          for (int a = 0; a < m; ++a) {
            const int i = mem[g0 + a];
            const BatchGrid gr = B.grids[((size_t)ph * B.n + i) * BS_COUNT + q];
            L.idx[a] = i;
            L.off[a] = acc;
            L.grid[a] = gr;
            L.inst[a] = h[i];
            acc += gr.x * gr.y * gr.z;
          }
          L.off[m] = acc;
          return acc;
        };
        if (ph == 0) {
          B.grp32[q].emplace_back();
          if (fill(B.grp32[q].back(), B.h32) == 0) B.grp32[q].pop_back();
        } else {
          B.grp64[q].emplace_back();
          if (fill(B.grp64[q].back(), B.h64) == 0) B.grp64[q].pop_back();
        }
      }
    }
  }
}

int fused_launches(const FusedBatch &B, int phases) {
  int k = B.grid_form ? 1 : 2;  // k_batch_iter_end, and k_batch_plan for the persistent form
  for (int ph = 0; ph < 2; ++ph)
    if (phases & (1 << ph))
      for (int q = 0; q < BS_COUNT; ++q)
        k += !B.use[ph][q] ? 0 : !B.grid_form ? 1 : (int)(ph ? B.grp64[q].size() : B.grp32[q].size());
  return k;
}

// G passes over the enclosures in the given phases (bit 0: FP32, bit 1: FP64)
int fused_graph(FusedBatch &B, int phases) {
  cudaGraphExec_t &exec = B.graph[phases - 1];
  if (exec) return NIM_OK;
  cudaGraph_t g = nullptr;
  CK(cudaStreamBeginCapture(B.s, cudaStreamCaptureModeThreadLocal));
  int st = NIM_OK;
  for (int k = 0; k < B.G && st == NIM_OK; ++k) {
    k_batch_plan<<<1, 1024, 0, B.s>>>(B.args);
    if (phases & 1) st = fused_slots_of<float>(B);
    if (st == NIM_OK && (phases & 2)) st = fused_slots_of<double>(B);
    k_batch_iter_end<<<(B.n + 127) / 128, 128, 0, B.s>>>(B.args);
  }
  const cudaError_t e = cudaStreamEndCapture(B.s, &g);
  if (st != NIM_OK || e != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return st != NIM_OK ? st : NIM_ERR_CUDA;
  }
  const cudaError_t ei = cudaGraphInstantiate(&exec, g, 0);
  cudaGraphDestroy(g);
  return ei == cudaSuccess ? NIM_OK : NIM_ERR_CUDA;
}

int fused_upload_phase(FusedBatch &B) {
  CK(cudaMemcpyAsync((void *)B.args.phase, B.phase_host, sizeof(int) * B.n, cudaMemcpyHostToDevice, B.s));
  return NIM_OK;
}

// the per-enclosure tables, the work list and the persistent grid sizes;
// every context's work moves to the batch stream until B goes out of scope
int fused_setup(FusedBatch &B, int32_t n, nim_ctx *const *ctx) {
  B.n = n;
  B.ctx.assign(ctx, ctx + n);
  B.mixed = ctx[0]->mixed;
  B.G = ctx[0]->graph_G;
  CK(cudaStreamCreateWithFlags(&B.s, cudaStreamNonBlocking));
  for (int32_t i = 0; i < n; ++i) CK(cudaStreamSynchronize(ctx[i]->stream));
  for (int32_t i = 0; i < n; ++i) {
    B.own.push_back(ctx[i]->stream);
    ctx[i]->stream = B.s;
  }
  // device block: i64[n], i32[n], grid[2][n][BS_COUNT], phase[n], state[n], plan
  auto up = [](size_t v) { return (v + 255) & ~(size_t)255; };
  const size_t o64 = 0, o32 = o64 + up(sizeof(BatchInst<double>) * n), og = o32 + up(sizeof(BatchInst<float>) * n),
               oph = og + up(sizeof(BatchGrid) * 2 * n * BS_COUNT), ost = oph + up(sizeof(int) * n),
               opl = ost + up(sizeof(BatchState) * n), bytes = opl + up(sizeof(BatchPlan));
  CK(cudaMalloc(&B.dev, bytes));
  CK(cudaMallocHost(&B.phase_host, sizeof(int) * n));
  CK(cudaMallocHost(&B.state_host, sizeof(BatchState) * n));
  char *base = static_cast<char *>(B.dev);
  std::vector<BatchInst<double>> h64(n);
  std::vector<BatchInst<float>> h32(n);
  std::vector<BatchGrid> grids(2 * (size_t)n * BS_COUNT, BatchGrid{0u, 0u, 0u});
  for (int32_t i = 0; i < n; ++i) {
    const nim_ctx *x = ctx[i];
    const Dims &d = x->d;
    h64[i] = BatchInst<double>{d, x->g, x->F, x->phys, x->ctl};
    if (B.mixed) h32[i] = BatchInst<float>{d, x->g32, x->F32, x->phys, x->ctl};
    // the one-cell sweeps over runs of consecutive cells of a plane (FlatBlock)
    const BatchGrid f3{(unsigned)((d.plane + CB - 1) / CB), 1u, (unsigned)d.NZ};
    const BatchGrid f8{(unsigned)((d.plane + BLK - 1) / BLK), 1u, (unsigned)d.NZ};
    const BatchGrid f3p{(unsigned)((d.plane / 2 + CB - 1) / CB), 1u, (unsigned)d.NZ};  // pairs of cells
    const BatchGrid gb{(unsigned)x->nblk_b, 1u, 1u};
    for (int ph = 0; ph < 2; ++ph) {
      if (ph == 0 && !B.mixed) continue;
      BatchGrid *G = &grids[((size_t)ph * n + i) * BS_COUNT];
      // the enclosure's sweeps in the forms the batch has, all of which give
      // the bits of the enclosure's own pass, over consecutive cells of a
      // plane (every lane busy whatever n_theta): the two-cell forms for
      // even n_theta (FP64 pressure sweeps too), else the one-cell forms
      // (the TMA-staged and four-cell sweeps of large meshes are replaced
      // by their gather forms)
      const bool pair = d.NT % 2 == 0 && (x->cell_pair || x->cell_quad);
      if (pair)
        G[BS_VEL_CELL2] = f3p;
      else
        G[BS_VEL_CELL] = f3;
      G[BS_VEL_FACE] = f3;
      if (ph == 1 && pair) {
        G[BS_P_SRC2] = f3p;
        G[BS_P_FACE2] = f3p;
      } else {
        G[BS_P_SRC] = f3;
        G[BS_P_FACE] = f3;
      }
      G[BS_P_BC] = gb;
      G[BS_P_BC_COPY] = gb;
      if (x->phys.dpdx_tolerance) G[BS_P_DPDX] = BatchGrid{(unsigned)x->nblk_c, 1u, 1u};
      G[BS_ZERO_FLUX] = BatchGrid{(unsigned)grid(2 * d.plane), 1u, 1u};
      G[BS_T_COEF] = BatchGrid{3u, (unsigned)x->nblk_c, 1u};
      G[BS_T_CELL] = f3;
      G[BS_T_FACE] = f8;
      for (int q = 0; q < BS_COUNT; ++q) B.use[ph][q] = B.use[ph][q] || G[q].x > 0;
    }
  }
  CK(cudaMemcpyAsync(base + o64, h64.data(), sizeof(BatchInst<double>) * n, cudaMemcpyHostToDevice, B.s));
  if (B.mixed)
    CK(cudaMemcpyAsync(base + o32, h32.data(), sizeof(BatchInst<float>) * n, cudaMemcpyHostToDevice, B.s));
  CK(cudaMemcpyAsync(base + og, grids.data(), sizeof(BatchGrid) * grids.size(), cudaMemcpyHostToDevice, B.s));
  CK(cudaMemsetAsync(base + oph, 0, sizeof(int) * n, B.s));
  CK(cudaStreamSynchronize(B.s));  // the host vectors go out of scope
  B.args.i64 = reinterpret_cast<const BatchInst<double> *>(base + o64);
  B.args.i32 = B.mixed ? reinterpret_cast<const BatchInst<float> *>(base + o32) : nullptr;
  B.args.grid = reinterpret_cast<const BatchGrid *>(base + og);
  B.args.phase = reinterpret_cast<const int *>(base + oph);
  B.args.plan = reinterpret_cast<BatchPlan *>(base + opl);
  B.args.n = n;
  B.state_dev_offset = ost;
  const char *form = std::getenv("NIM_BATCH_FORM");
  B.grid_form = form && std::string(form) == "grid";
  if (B.grid_form) {  // kept for the groups (fused_groups)
    B.grids = grids;
    B.h64 = h64;
    B.h32 = h32;
  }
  int sms = 0;
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx[0]->device));
  // NIM_BATCH_BOUNDS=wide: the batched kernels one resident block per SM
  // below the plain kernels' bound (more registers, fewer spills)
  const char *bounds = std::getenv("NIM_BATCH_BOUNDS");
  B.wide = bounds && std::string(bounds) == "wide";
  if (B.mixed) TRY((B.wide ? fused_occupancy<float, 1>(B, sms) : fused_occupancy<float, 0>(B, sms)));
  TRY((B.wide ? fused_occupancy<double, 1>(B, sms) : fused_occupancy<double, 0>(B, sms)));
  return NIM_OK;
}
}  // namespace

extern "C" int nim_batch_step_fused(int32_t n, nim_ctx *const *ctx, int32_t nsteps, nim_step_stats *per,
                                    int32_t *done) {
  if (n <= 0 || n > kBatchMax || !ctx || nsteps < 0) return NIM_ERR_BAD_ARG;
  for (int32_t i = 0; i < n; ++i) {
    if (!ctx[i] || lone_slab(ctx[i])) return NIM_ERR_BAD_ARG;
    if (!ctx[i]->initialized || ctx[i]->in_step) return NIM_ERR_STATE;
    if (ctx[i]->device != ctx[0]->device || ctx[i]->seq || ctx[i]->phys.formulation != 2 ||
        ctx[i]->mixed != ctx[0]->mixed)
      return NIM_ERR_BAD_ARG;
    for (int32_t j = 0; j < i; ++j)
      if (ctx[j] == ctx[i]) return NIM_ERR_BAD_ARG;
  }
  if (done)
    for (int32_t i = 0; i < n; ++i) done[i] = 0;
  if (nsteps == 0) return NIM_OK;
  CK(cudaSetDevice(ctx[0]->device));
  FusedBatch B;
  TRY(fused_setup(B, n, ctx));
  BatchState *state_dev = reinterpret_cast<BatchState *>(static_cast<char *>(B.dev) + B.state_dev_offset);
  // Per enclosure: RUN (its inner loop is in the fused passes, phase 1 or
  // 2), AFTER (check_steady_state / evaluate_D queued), END
  // (update_time_step / find_Nu2 queued), FIN.  Every enclosure goes
  // through its own steps at its own pace: one whose loop has stopped ends
  // its step and starts the next while the others keep iterating.
  enum { RUN, AFTER, END, FIN };
  std::vector<int> st(n, RUN), k(n, 0);
  std::vector<nim_step_stats> rec(n);
  int first_error = NIM_OK;
  int *ph = B.phase_host;
  auto start_step = [&](int32_t i) -> int {
    nim_ctx *x = ctx[i];
    std::memset(&rec[i], 0, sizeof(nim_step_stats));
    TRY(nim_gpu_begin_step(x));
    x->run.capped = false;
    x->run.launched = 0;
    x->run.cap = (x->params.max_iters > 0) ? (long long)x->params.max_iters + 2 * B.G : 100000000LL;
    if (B.mixed) {  // FP32 phase from the narrowed FP64 iterate
      TRY(mirror_state(x, 0));
      k_lowp_begin<<<1, 1, 0, B.s>>>(x->ctl);
      CK(cudaGetLastError());
      x->launches += 1;
    }
    ph[i] = B.mixed ? 1 : 2;
    st[i] = RUN;
    return NIM_OK;
  };
  // a step's record is complete: the next step, or the enclosure is done
  auto finish = [&](int32_t i, int status) -> int {
    if (per) per[(size_t)i * nsteps + k[i]] = rec[i];
    ++k[i];
    if (done) done[i] = k[i];
    if (status != NIM_OK && first_error == NIM_OK) first_error = status;
    if (status != NIM_OK || rec[i].steady || k[i] == nsteps) {
      st[i] = FIN;
      return NIM_OK;
    }
    return start_step(i);
  };
  for (int32_t i = 0; i < n; ++i) TRY(start_step(i));
  TRY(fused_upload_phase(B));
  bool regroup = true;  // the grid form's groups follow the phases
  for (;;) {
    int phases = 0, busy = 0;
    for (int32_t i = 0; i < n; ++i) {
      if (st[i] == RUN) phases |= (ph[i] == 1) ? 1 : 2;
      busy += (st[i] != FIN) ? 1 : 0;
    }
    if (!busy) break;
    if (phases) {
      if (B.grid_form) {
        // the groups of this interval's enclosures, then G passes launched
        // directly (the groups change as enclosures change phase)
        if (regroup) fused_groups(B, ph);
        regroup = false;
        for (int k = 0; k < B.G; ++k) {
          if (phases & 1) TRY(group_slots<float>(B));
          if (phases & 2) TRY(group_slots<double>(B));
          k_batch_iter_end<<<(n + 127) / 128, 128, 0, B.s>>>(B.args);
        }
      } else {
        TRY(fused_graph(B, phases));
        CK(cudaGraphLaunch(B.graph[phases - 1], B.s));
      }
      ctx[0]->launches += (long long)B.G * fused_launches(B, phases);
      for (int32_t i = 0; i < n; ++i)
        if (st[i] == RUN) ctx[i]->run.launched += B.G;
      k_batch_state<<<(n + 127) / 128, 128, 0, B.s>>>(B.args, state_dev);
      CK(cudaGetLastError());
      CK(cudaMemcpyAsync(B.state_host, state_dev, sizeof(BatchState) * n, cudaMemcpyDeviceToHost, B.s));
    }
    // every copy queued so far (states, control blocks, sums) has landed
    CK(cudaStreamSynchronize(B.s));
    bool changed = false;
    for (int32_t i = 0; i < n; ++i) {
      nim_ctx *x = ctx[i];
      if (st[i] == RUN) {
        const bool stopped = B.state_host[i].done != 0;
        if (stopped && ph[i] == 1 && B.state_host[i].status == NIM_OK) {
          // FP32 phase over: widen its iterate, FP64 passes to the reference's test
          TRY(mirror_state(x, 1));
          k_lowp_end<<<1, 1, 0, B.s>>>(x->ctl);
          CK(cudaGetLastError());
          x->launches += 1;
          ph[i] = 2;
          changed = true;
        } else if (stopped || x->run.launched >= x->run.cap) {
          x->run.capped = !stopped;
          ph[i] = 0;
          changed = true;
          TRY(after_loop_start(x));
          st[i] = AFTER;
        }
      } else if (st[i] == AFTER) {
        const int s = integrate_finish(x, &rec[i]);
        rec[i].status = s;
        if (s != NIM_OK) {
          x->in_step = false;
          TRY(finish(i, s));
        } else if (steady_exit(x, rec[i])) {
          rec[i].steady = 1;
          x->in_step = false;
          TRY(finish(i, NIM_OK));
        } else {
          TRY(end_start(x));
          st[i] = END;
        }
        changed = changed || st[i] == RUN;
      } else if (st[i] == END) {
        end_finish(x, &rec[i]);
        TRY(finish(i, NIM_OK));
        changed = changed || st[i] == RUN;
      }
    }
    if (changed) TRY(fused_upload_phase(B));
    regroup = regroup || changed;
  }
  return first_error;
}

// ---- a group of z-slabs on one device, advanced together (nim_slab_step)
namespace {
constexpr int kMaxSlabs = 16;
struct CtlList {
  Ctrl *c[kMaxSlabs];
  int n;
};

// find_error's maxima and the Dirichlet wall floor over every slab of the
// group, written back to each slab's control block before its k_iter_end:
// one thread per slot, so reads and writes of a slot never race
__global__ void k_slab_merge(CtlList L) {
  const int q = threadIdx.x;
  if (q >= 16 || L.c[0]->done) return;
  const int par = L.c[0]->iter & L.c[0]->pmask;
  unsigned long long m = 0ull;
  for (int s = 0; s < L.n; ++s) {
    const unsigned long long v = (q < 8) ? L.c[s]->err[par][q] : L.c[s]->wall_floor[q - 8];
    m = (v > m) ? v : m;
  }
  for (int s = 0; s < L.n; ++s) {
    if (q < 8)
      L.c[s]->err[par][q] = m;
    else
      L.c[s]->wall_floor[q - 8] = m;
  }
}

// which arrays a halo exchange carries: after the velocity, pressure and
// temperature parts of a pass, or the whole state
enum { kHaloV = 1, kHaloP = 2, kHaloT = 4, kHaloAll = 8 };

// The device arrays an exchange of `what` carries, in a fixed order: each
// a cell array (Nc doubles) or a face array (both halves, 2*NF doubles).
struct HaloArray {
  double *p;
  bool face;
};
void halo_arrays(const nim_ctx *x, int what, std::vector<HaloArray> &out) {
  const Fields &F = x->F;
  const bool all = (what & kHaloAll) != 0;
  out.clear();
  if (all || (what & kHaloV))
    for (int q = 0; q < 3; ++q) {
      out.push_back({F.c[q], false});
      out.push_back({F.f[q], true});
    }
  if (all || (what & kHaloP)) out.push_back({F.f[3], true});
  if (all || (what & kHaloT)) {
    out.push_back({F.c[3], false});
    out.push_back({F.f[4], true});
  }
  if (all) {
    for (int q = 0; q < 4; ++q) {
      out.push_back({F.co[q], false});
      out.push_back({F.ct[q], false});
    }
    out.push_back({F.mp, false});
    out.push_back({F.dila, false});
    out.push_back({F.dila_old, false});
    for (int q = 0; q < 3; ++q) out.push_back({F.dpd + (size_t)q * x->d.Nc, false});
  }
}

// One launch copies up to kHaloJobs spans (blockIdx.y = span): every copy
// of an exchange in a handful of launches instead of one memcpy per span.
constexpr int kHaloJobs = 120;
struct HaloJobs {
  const double *src[kHaloJobs];
  double *dst[kHaloJobs];
  int n[kHaloJobs];
};
__global__ void __launch_bounds__(BLK) k_halo_copy(HaloJobs J) {
  const int j = blockIdx.y;
  const double *__restrict__ a = J.src[j];
  double *__restrict__ b = J.dst[j];
  for (int i = blockIdx.x * BLK + threadIdx.x; i < J.n[j]; i += gridDim.x * BLK) b[i] = a[i];
}

// src's owned planes next to dst into dst's halo: each cell array over span
// 0, each face array (both halves) over the r, theta and z spans 1..3
int halo_jobs(const nim_ctx *src, const int64_t *snd, const nim_ctx *dst, const int64_t *rcv, int what,
              std::vector<HaloJobs> &jobs, int &used) {
  for (int t = 0; t < 4; ++t)
    if (snd[2 * t + 1] != rcv[2 * t + 1]) return NIM_ERR_BAD_ARG;
  std::vector<HaloArray> A, B;
  halo_arrays(src, what, A);
  halo_arrays(dst, what, B);
  const size_t NFa = src->d.NF, NFb = dst->d.NF;
  auto add = [&](const double *from, double *to, int64_t n) {
    if (used == kHaloJobs || jobs.empty()) {
      jobs.emplace_back();
      used = 0;
    }
    HaloJobs &J = jobs.back();
    J.src[used] = from;
    J.dst[used] = to;
    J.n[used] = (int)n;
    ++used;
  };
  for (size_t a = 0; a < A.size(); ++a) {
    if (!A[a].face) {
      add(A[a].p + snd[0], B[a].p + rcv[0], snd[1]);
      continue;
    }
    for (int h = 0; h < 2; ++h)
      for (int t = 1; t < 4; ++t) add(A[a].p + h * NFa + snd[2 * t], B[a].p + h * NFb + rcv[2 * t], snd[2 * t + 1]);
  }
  return NIM_OK;
}

int halo_exchange(nim_ctx *const *X, int n, cudaStream_t st, int what) {
  std::vector<HaloJobs> jobs;
  int used = 0;
  int64_t longest = 0;
  for (int s = 0; s + 1 < n; ++s) {
    TRY(halo_jobs(X[s], X[s]->halo_send[1], X[s + 1], X[s + 1]->halo_recv[0], what, jobs, used));
    TRY(halo_jobs(X[s + 1], X[s + 1]->halo_send[0], X[s], X[s]->halo_recv[1], what, jobs, used));
    for (int t = 0; t < 4; ++t) longest = std::max(longest, X[s]->halo_send[1][2 * t + 1]);
  }
  const int gx = (int)std::min<int64_t>((longest + BLK - 1) / BLK, 64);
  for (size_t k = 0; k < jobs.size(); ++k) {
    const int nj = (k + 1 == jobs.size()) ? used : kHaloJobs;
    k_halo_copy<<<dim3(std::max(gx, 1), nj), BLK, 0, st>>>(jobs[k]);
    CK(cudaGetLastError());
  }
  return NIM_OK;
}

// G passes of integrate_nse's loop body over the whole group: each part of
// the pass on every slab, then the halos it changed; the merged maxima,
// then every slab's k_iter_end (which therefore all decide alike)
int slab_pass_graph(nim_ctx *const *X, int n, int G, cudaGraphExec_t *exec) {
  cudaStream_t st = X[0]->stream;
  CtlList L{};
  L.n = n;
  for (int s = 0; s < n; ++s) L.c[s] = X[s]->ctl;
  cudaGraph_t g = nullptr;
  CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  int rc = NIM_OK;
  for (int it = 0; it < G && rc == NIM_OK; ++it) {
    for (int s = 0; s < n && rc == NIM_OK; ++s) rc = launch_vel(X[s], st, X[s]->g, X[s]->F);
    if (rc == NIM_OK) rc = halo_exchange(X, n, st, kHaloV);
    for (int s = 0; s < n && rc == NIM_OK; ++s) rc = launch_pressure(X[s], st, X[s]->g, X[s]->F);
    if (rc == NIM_OK) rc = halo_exchange(X, n, st, kHaloP);
    for (int s = 0; s < n && rc == NIM_OK; ++s) rc = launch_temperature(X[s], st, X[s]->g, X[s]->F);
    if (rc == NIM_OK) rc = halo_exchange(X, n, st, kHaloT);
    if (rc == NIM_OK) {
      k_slab_merge<<<1, 32, 0, st>>>(L);
      for (int s = 0; s < n; ++s) k_iter_end<<<1, 1, 0, st>>>(X[s]->ctl, X[s]->phys, 0);
    }
  }
  const cudaError_t ce = cudaStreamEndCapture(st, &g);
  if (rc == NIM_OK && ce != cudaSuccess) rc = NIM_ERR_CUDA;
  if (rc == NIM_OK && cudaGraphInstantiate(exec, g, 0) != cudaSuccess) rc = NIM_ERR_CUDA;
  if (g) cudaGraphDestroy(g);
  return rc;
}

// the step-end reductions of the group: sums[0..n) the dilatation sums,
// red[0..1] the merged dudt / dTdt maxima
int slab_after_integrate(nim_ctx *const *X, int n, cudaStream_t st, double &dsum, double &dudt, double &dTdt) {
  for (int s = 0; s < n; ++s) {
    nim_ctx *x = X[s];
    k_after_integrate<<<x->nblk_c, BLK, 0, st>>>(x->d, x->g, x->F, x->phys, x->ctl, x->nblk_c);
    k_finish_sum<<<1, BLK, 0, st>>>(x->F.part, x->nblk_c, 1, x->sums);
    CK(cudaGetLastError());
    x->launches += 2;
    CK(cudaMemcpyAsync(x->host_sums, x->sums, sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(x->ctl_host, x->ctl, sizeof(Ctrl), cudaMemcpyDeviceToHost, st));
  }
  CK(cudaStreamSynchronize(st));
  dsum = dudt = dTdt = 0.;
  for (int s = 0; s < n; ++s) {
    dsum += X[s]->host_sums[0];
    dudt = std::max(dudt, bits_to_double(X[s]->ctl_host->red[0]));
    dTdt = std::max(dTdt, bits_to_double(X[s]->ctl_host->red[1]));
  }
  return NIM_OK;
}

// update_time_step + find_Nu2 on every slab; sums4 = the group's wall sums
int slab_end(nim_ctx *const *X, int n, cudaStream_t st, double *sums4) {
  for (int s = 0; s < n; ++s) {
    nim_ctx *x = X[s];
    const Dims &d = x->d;
    const int gn = grid(2 * d.NT * d.NZ);
    k_update_time<<<x->nblk_c, BLK, 0, st>>>(d, x->F, x->ctl);
    k_nusselt<<<gn, BLK, 0, st>>>(d, x->g, x->F, x->ctl, gn);
    k_finish_sum<<<1, BLK, 0, st>>>(x->F.part, gn, 4, x->sums);
    CK(cudaGetLastError());
    x->launches += 3;
    CK(cudaMemcpyAsync(x->host_sums, x->sums, 4 * sizeof(double), cudaMemcpyDeviceToHost, st));
  }
  CK(cudaStreamSynchronize(st));
  for (int q = 0; q < 4; ++q) sums4[q] = 0.;
  for (int s = 0; s < n; ++s)
    for (int q = 0; q < 4; ++q) sums4[q] += X[s]->host_sums[q];
  return NIM_OK;
}

int slab_step_impl(nim_ctx *const *X, int n, int32_t nsteps, nim_step_stats *per, int32_t *done,
                   cudaGraphExec_t exec) {
  nim_ctx *x0 = X[0];
  cudaStream_t st = x0->stream;
  const int G = x0->graph_G;
  int64_t owned = 0;
  for (int s = 0; s < n; ++s) owned += (int64_t)(X[s]->d.kown1 - X[s]->d.kown0) * X[s]->d.plane;
  int32_t k = 0;
  int status = NIM_OK;
  for (; k < nsteps; ++k) {
    nim_step_stats rec;
    std::memset(&rec, 0, sizeof(rec));
    for (int s = 0; s < n; ++s) TRY(nim_gpu_begin_step(X[s]));
    for (int s = 0; s < n; ++s) CK(cudaStreamSynchronize(X[s]->stream));
    const long long cap = (x0->params.max_iters > 0) ? (long long)x0->params.max_iters + 2 * G : 100000000LL;
    long long launched = 0;
    bool capped = false;
    for (;;) {
      CK(cudaGraphLaunch(exec, st));
      launched += G;
      for (int s = 0; s < n; ++s) X[s]->launches += (long long)G * (X[s]->phys.dpdx_tolerance ? 12 : 11);
      CK(cudaMemcpyAsync(x0->ctl_host, x0->ctl, sizeof(Ctrl), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      if (x0->ctl_host->done) break;
      if (launched >= cap) {
        capped = true;
        break;
      }
    }
    double dsum, dudt, dTdt;
    TRY(slab_after_integrate(X, n, st, dsum, dudt, dTdt));
    for (int s = 0; s < n; ++s) X[s]->last_iters = X[s]->ctl_host->step_iters;
    if (capped && x0->ctl_host->status == NIM_OK) x0->ctl_host->status = NIM_ERR_NOT_CONVERGED;
    fill_iter_stats(x0, &rec);
    rec.dilatation = std::sqrt(dsum / (double)owned);
    rec.dudt_max = dudt;
    rec.dTdt_max = dTdt;
    status = rec.status;
    if (status != NIM_OK || steady_exit(x0, rec)) {
      if (status == NIM_OK) rec.steady = 1;
      for (int s = 0; s < n; ++s) X[s]->in_step = false;
      if (per) per[k] = rec;
      ++k;
      break;
    }
    double sums[4];
    TRY(slab_end(X, n, st, sums));
    for (int s = 0; s < n; ++s) end_finish(X[s], nullptr);
    rec.step = x0->STEP - 1;
    rec.nu_outer = -(sums[0] / sums[1] * x0->params.R_o);
    rec.nu_inner = -(sums[2] / sums[3] * x0->params.R_i);
    rec.area_outer = sums[1];
    rec.area_inner = sums[3];
    rec.time = x0->TI;
    if (per) per[k] = rec;
  }
  if (done) *done = k;
  return status;
}
}  // namespace

extern "C" int nim_slab_step(int32_t n, nim_ctx *const *X, int32_t nsteps, nim_step_stats *per, int32_t *done) {
  if (n < 1 || n > kMaxSlabs || !X || nsteps < 0) return NIM_ERR_BAD_ARG;
  for (int32_t s = 0; s < n; ++s) {
    if (!X[s] || X[s]->slab_count != n || X[s]->slab_index != s || X[s]->device != X[0]->device ||
        X[s]->graph_G != X[0]->graph_G)
      return NIM_ERR_BAD_ARG;
    if (!X[s]->initialized || X[s]->in_step) return NIM_ERR_STATE;
    // slabs of one mesh: same cross-section, owned planes end to end
    if (X[s]->d.NT != X[0]->d.NT || X[s]->d.NR != X[0]->d.NR) return NIM_ERR_BAD_ARG;
    if (s > 0 && X[s]->slab_lo + X[s]->d.kown0 != X[s - 1]->slab_lo + X[s - 1]->d.kown1) return NIM_ERR_BAD_ARG;
  }
  CK(cudaSetDevice(X[0]->device));
  for (int32_t s = 0; s < n; ++s) CK(cudaStreamSynchronize(X[s]->stream));
  // every halo from its owner: after nim_gpu_init, uploads or a previous call
  TRY(halo_exchange(X, n, X[0]->stream, kHaloAll));
  CK(cudaStreamSynchronize(X[0]->stream));
  cudaGraphExec_t exec = nullptr;
  TRY(slab_pass_graph(X, n, X[0]->graph_G, &exec));
  const int st = slab_step_impl(X, n, nsteps, per, done, exec);
  cudaStreamSynchronize(X[0]->stream);
  cudaGraphExecDestroy(exec);
  if (st != NIM_OK)  // a step left half done: the next call starts a new one
    for (int32_t s = 0; s < n; ++s) X[s]->in_step = false;
  return st;
}

// ---- the pieces of a pass for a host that moves the halos itself (one
// process per GPU: the exchange and the maxima reduction over its own
// transport, on the context's stream, between the parts)
extern "C" int nim_slab_part(nim_ctx *x, int32_t part) {
  if (!x || part < 0 || part > 3) return NIM_ERR_BAD_ARG;
  if (!x->initialized || !x->in_step) return NIM_ERR_STATE;
  if (x->seq || x->mixed) return NIM_ERR_BAD_ARG;
  CK(cudaSetDevice(x->device));
  cudaStream_t s = x->stream;
  switch (part) {
    case 0: TRY(launch_vel(x, s, x->g, x->F)); break;
    case 1: TRY(launch_pressure(x, s, x->g, x->F)); break;
    case 2: TRY(launch_temperature(x, s, x->g, x->F)); break;
    default: k_iter_end<<<1, 1, 0, s>>>(x->ctl, x->phys, 0);
  }
  CK(cudaGetLastError());
  x->launches += (part == 3) ? 1 : 4;
  return NIM_OK;
}

extern "C" int nim_slab_arrays(nim_ctx *x, int32_t set, void **ptr, int32_t *face, int32_t cap) {
  if (!x || !ptr || !face || set < 1 || set > 15 || cap < 0) return NIM_ERR_BAD_ARG;
  std::vector<HaloArray> v;
  halo_arrays(x, set, v);
  if ((int)v.size() > cap) return NIM_ERR_BAD_ARG;
  for (size_t i = 0; i < v.size(); ++i) {
    ptr[i] = v[i].p;
    face[i] = v[i].face ? 1 : 0;
  }
  return (int)v.size();
}

namespace {
// the spans of one side of an exchange of `what`, in payload order: each
// array of halo_arrays, a cell array over span 0, a face array over spans
// 1..3 of its first half then of its second
int side_spans(const nim_ctx *x, int what, int side, bool send, std::vector<std::pair<double *, int64_t>> &out) {
  if ((side != 0 && side != 1) || !x->halo_ok[side]) return NIM_ERR_BAD_ARG;
  const int64_t *sp = send ? x->halo_send[side] : x->halo_recv[side];
  std::vector<HaloArray> A;
  halo_arrays(x, what, A);
  out.clear();
  const size_t NF = x->d.NF;
  for (const HaloArray &a : A) {
    if (!a.face) {
      out.emplace_back(a.p + sp[0], sp[1]);
      continue;
    }
    for (int h = 0; h < 2; ++h)
      for (int t = 1; t < 4; ++t) out.emplace_back(a.p + h * NF + sp[2 * t], sp[2 * t + 1]);
  }
  return NIM_OK;
}

// pack (spans -> buf) or unpack (buf -> spans) on the context's stream
int pack_side(nim_ctx *x, int what, int side, double *buf, bool pack) {
  std::vector<std::pair<double *, int64_t>> sp;
  TRY(side_spans(x, what, side, pack, sp));
  std::vector<HaloJobs> jobs;
  int64_t off = 0, longest = 0;
  int used = 0;
  for (auto &v : sp) {
    if (used == kHaloJobs || jobs.empty()) {
      jobs.emplace_back();
      used = 0;
    }
    HaloJobs &J = jobs.back();
    J.src[used] = pack ? v.first : buf + off;
    J.dst[used] = pack ? buf + off : v.first;
    J.n[used] = (int)v.second;
    ++used;
    off += v.second;
    longest = std::max(longest, v.second);
  }
  CK(cudaSetDevice(x->device));
  const int gx = (int)std::max<int64_t>(1, std::min<int64_t>((longest + BLK - 1) / BLK, 64));
  for (size_t k = 0; k < jobs.size(); ++k) {
    const int nj = (k + 1 == jobs.size()) ? used : kHaloJobs;
    k_halo_copy<<<dim3(gx, nj), BLK, 0, x->stream>>>(jobs[k]);
    CK(cudaGetLastError());
  }
  x->launches += (long long)jobs.size();
  return NIM_OK;
}
}  // namespace

extern "C" int64_t nim_slab_pack_doubles(nim_ctx *x, int32_t set, int32_t side) {
  if (!x || set < 1 || set > 15) return NIM_ERR_BAD_ARG;
  std::vector<std::pair<double *, int64_t>> sp;
  TRY(side_spans(x, set, side, true, sp));
  int64_t n = 0;
  for (auto &v : sp) n += v.second;
  return n;
}

extern "C" int nim_slab_pack(nim_ctx *x, int32_t set, int32_t side, void *buf) {
  if (!x || !buf || set < 1 || set > 15) return NIM_ERR_BAD_ARG;
  return pack_side(x, set, side, static_cast<double *>(buf), true);
}

extern "C" int nim_slab_unpack(nim_ctx *x, int32_t set, int32_t side, const void *buf) {
  if (!x || !buf || set < 1 || set > 15) return NIM_ERR_BAD_ARG;
  return pack_side(x, set, side, const_cast<double *>(static_cast<const double *>(buf)), false);
}

extern "C" int nim_slab_maxima(nim_ctx *x, void **slots24) {
  if (!x || !slots24) return NIM_ERR_BAD_ARG;
  *slots24 = reinterpret_cast<char *>(x->ctl) + offsetof(Ctrl, err);
  return NIM_OK;
}

extern "C" int nim_slab_loop_state(nim_ctx *x, int32_t *state3, double *err5) {
  if (!x || !state3) return NIM_ERR_BAD_ARG;
  CK(cudaSetDevice(x->device));
  TRY(read_ctrl(x));
  const Ctrl &c = *x->ctl_host;
  state3[0] = c.done;
  state3[1] = c.step_iters;
  state3[2] = c.status;
  if (err5)
    for (int q = 0; q < 5; ++q) err5[q] = c.last_err[q];
  return NIM_OK;
}

extern "C" int nim_slab_after_loop(nim_ctx *x, double *out3) {
  if (!x || !out3) return NIM_ERR_BAD_ARG;
  if (!x->initialized || !x->in_step) return NIM_ERR_STATE;
  CK(cudaSetDevice(x->device));
  TRY(slab_after_integrate(&x, 1, x->stream, out3[0], out3[1], out3[2]));
  x->last_iters = x->ctl_host->step_iters;
  return NIM_OK;
}

extern "C" int nim_slab_end_step(nim_ctx *x, double *out4) {
  if (!x || !out4) return NIM_ERR_BAD_ARG;
  if (!x->initialized || !x->in_step) return NIM_ERR_STATE;
  CK(cudaSetDevice(x->device));
  TRY(slab_end(&x, 1, x->stream, out4));
  end_finish(x, nullptr);
  return NIM_OK;
}

extern "C" int nim_gpu_download(nim_ctx *x, nim_field f, double *host, int64_t n) {
  if (!x || !host) return NIM_ERR_BAD_ARG;
  if (!x->initialized) return NIM_ERR_STATE;
  TRY(read_ctrl(x));
  FieldView v;
  TRY(field_view(x, f, x->seq ? 0 : (x->ctl_host->iter & 1), v));
  const int64_t len = (int64_t)v.n * v.K;
  if (n < len) return NIM_ERR_BAD_ARG;
  k_gather<<<grid(v.n), BLK, 0, x->stream>>>(v.src, v.stride, v.K, v.face ? x->perm : nullptr, v.n, x->scratch);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(host, x->scratch, sizeof(double) * len, cudaMemcpyDeviceToHost, x->stream));
  CK(cudaStreamSynchronize(x->stream));
  return NIM_OK;
}

extern "C" int nim_gpu_upload(nim_ctx *x, nim_field f, const double *host, int64_t n) {
  if (!x || !host) return NIM_ERR_BAD_ARG;
  if (!x->initialized) return NIM_ERR_STATE;
  TRY(read_ctrl(x));
  FieldView v;
  TRY(field_view(x, f, x->seq ? 0 : (x->ctl_host->iter & 1), v));
  if (!v.writable || v.K != 1) return NIM_ERR_BAD_ARG;
  if (n < v.n) return NIM_ERR_BAD_ARG;
  CK(cudaMemcpyAsync(x->scratch, host, sizeof(double) * v.n, cudaMemcpyHostToDevice, x->stream));
  k_scatter<<<grid(v.n), BLK, 0, x->stream>>>(x->scratch, v.face ? x->perm : nullptr, v.n, const_cast<double *>(v.src),
                                                 v.dst1);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(x->stream));
  return NIM_OK;
}

extern "C" int64_t nim_gpu_output_bytes(nim_ctx *x, int32_t set) {
  if (!x) return NIM_ERR_BAD_ARG;
  const int64_t Nc = x->d.Nc, NF = x->d.NF;
  switch (set) {
    case NIM_OUTPUT_PLOT: return 6 * Nc * (int64_t)sizeof(float);
    case NIM_OUTPUT_RESTART: return (5 * NF + 9 * Nc) * (int64_t)sizeof(double);
    default: return NIM_ERR_BAD_ARG;
  }
}

extern "C" int nim_gpu_output_begin(nim_ctx *x, int32_t set, void *host, int64_t bytes, int32_t *ticket) {
  if (!x || !host || !ticket) return NIM_ERR_BAD_ARG;
  const int64_t need = nim_gpu_output_bytes(x, set);
  if (need < 0 || bytes < need) return NIM_ERR_BAD_ARG;
  if (!x->initialized) return NIM_ERR_STATE;
  CK(cudaSetDevice(x->device));
  nim_ctx::Output &o = x->out[set];
  if (!o.stage) {
    CK(cudaMalloc(&o.stage, need));
    x->allocs.push_back(o.stage);
    CK(cudaEventCreateWithFlags(&o.packed, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&o.copied, cudaEventDisableTiming));
  } else {
    CK(cudaStreamWaitEvent(x->stream, o.copied, 0));  // the previous copy has left the staging buffer
  }
  const Dims &d = x->d;
  if (set == NIM_OUTPUT_PLOT)
    k_pack_plot<<<grid(d.Nc), BLK, 0, x->stream>>>(d, x->F, static_cast<float *>(o.stage));
  else
    k_pack_restart<<<grid(std::max(d.NF, d.Nc)), BLK, 0, x->stream>>>(d, x->F, x->perm, x->ctl,
                                                                      static_cast<double *>(o.stage));
  CK(cudaGetLastError());
  x->launches += 1;
  CK(cudaEventRecord(o.packed, x->stream));
  CK(cudaStreamWaitEvent(x->copy_stream, o.packed, 0));
  CK(cudaMemcpyAsync(host, o.stage, need, cudaMemcpyDeviceToHost, x->copy_stream));
  CK(cudaEventRecord(o.copied, x->copy_stream));
  o.gen = (o.gen + 1) & 0x3fffffff;
  *ticket = (o.gen << 1) | set;
  return NIM_OK;
}

extern "C" int nim_gpu_output_wait(nim_ctx *x, int32_t ticket) {
  if (!x || ticket < 0) return NIM_ERR_BAD_ARG;
  const int set = ticket & 1, gen = ticket >> 1;
  nim_ctx::Output &o = x->out[set];
  if (!o.copied || gen != o.gen) return NIM_ERR_STATE;  // unknown, or overtaken by a later begin
  CK(cudaEventSynchronize(o.copied));
  return NIM_OK;
}

extern "C" int nim_gpu_synchronize(nim_ctx *x) {
  if (!x) return NIM_ERR_BAD_ARG;
  CK(cudaStreamSynchronize(x->stream));
  return NIM_OK;
}

extern "C" void nim_gpu_destroy(nim_ctx *x) {
  if (!x) return;
  if (x->stream) cudaStreamSynchronize(x->stream);
  if (x->copy_stream) cudaStreamSynchronize(x->copy_stream);  // copies still reading staging
  if (x->graph) cudaGraphExecDestroy(x->graph);
  if (x->graph32) cudaGraphExecDestroy(x->graph32);
  for (void *p : x->allocs) cudaFree(p);
  if (x->ctl_host) cudaFreeHost(x->ctl_host);
  for (auto &o : x->out) {
    if (o.packed) cudaEventDestroy(o.packed);
    if (o.copied) cudaEventDestroy(o.copied);
  }
  if (x->copy_stream) cudaStreamDestroy(x->copy_stream);
  if (x->run.ev) cudaEventDestroy(x->run.ev);
  if (x->stream) cudaStreamDestroy(x->stream);
  delete x;
}

extern "C" void *nim_gpu_stream(nim_ctx *x) { return x ? (void *)x->stream : nullptr; }
extern "C" int64_t nim_gpu_launch_count(nim_ctx *x) { return x ? x->launches : -1; }

extern "C" int nim_gpu_profile_iterations(nim_ctx *x, int32_t n, double *ms, int32_t cap) {
  if (!x || n <= 0 || !ms || cap <= 0) return NIM_ERR_BAD_ARG;
  if (!x->initialized) return NIM_ERR_STATE;
  cudaStream_t s = x->stream;
  const Phys keep = x->phys;
  x->phys.max_iters = 0;
  for (int q = 0; q < 5; ++q) x->phys.tol[q] = -1.0;
  // n + 1 passes queued back to back with an event after every kernel, one
  // wait at the end: no host gap inside the timed passes; the first pass
  // (which starts on an idle stream) is not counted
  nim_ctx::Marks marks;
  std::vector<double> acc;
  std::vector<const char *> names;
  int st = NIM_OK;
  {
    k_step_reset<<<1, 1, 0, s>>>(x->ctl);
    if (x->mixed) st = mirror_state(x, 0);  // FP32 passes over the narrowed iterate
    x->marks = &marks;
    std::vector<size_t> pass_end;
    for (int it = 0; it <= n && st == NIM_OK; ++it) {
      st = launch_iteration(x, x->mixed, false);  // every pass runs: no stop test
      pass_end.push_back(marks.used);
    }
    x->marks = nullptr;
    if (st == NIM_OK && cudaEventSynchronize(marks.ev[marks.used - 1]) != cudaSuccess) st = NIM_ERR_CUDA;
    if (st == NIM_OK) {
      const size_t K = pass_end[0];
      names.assign(marks.name.begin(), marks.name.begin() + K);
      acc.assign(K, 0.0);
      for (int it = 1; it <= n; ++it) {
        const size_t b0 = pass_end[it - 1];
        for (size_t k = 0; k < K; ++k) {
          float t = 0.f;
          cudaEventElapsedTime(&t, marks.ev[b0 + k - 1], marks.ev[b0 + k]);
          acc[k] += t;
        }
      }
    }
  }
  x->phys = keep;
  for (cudaEvent_t e : marks.ev) cudaEventDestroy(e);
  if (st != NIM_OK) return st;
  const int nk = std::min((int)acc.size(), (int)cap);
  x->prof_names.assign(names.begin(), names.begin() + nk);
  for (int k = 0; k < nk; ++k) ms[k] = acc[k] / n;
  return nk;
}

extern "C" int nim_gpu_selftest_wait_timeout(nim_ctx *x, int32_t tries) {
  if (!x || tries < 1 || tries > (1 << 20)) return NIM_ERR_BAD_ARG;
  if (!x->initialized || x->in_step) return NIM_ERR_STATE;
  CK(cudaSetDevice(x->device));
  k_step_reset<<<1, 1, 0, x->stream>>>(x->ctl);
  k_wait_selftest<<<1, 1, 0, x->stream>>>(x->ctl, tries);
  CK(cudaGetLastError());
  TRY(read_ctrl(x));
  const int seen = x->ctl_host->status;
  k_step_reset<<<1, 1, 0, x->stream>>>(x->ctl);  // the context stays usable
  TRY(read_ctrl(x));
  return seen;
}

extern "C" int nim_gpu_selftest_exp(const double *x, double *y, int64_t n) {
  if (n < 0 || (n > 0 && (!x || !y)) || n > (int64_t(1) << 28)) return NIM_ERR_BAD_ARG;
  if (n == 0) return NIM_OK;
  const size_t bytes = (size_t)n * sizeof(double);
  double *dx = nullptr, *dy = nullptr;
  int st = NIM_OK;
  if (cudaMalloc(&dx, bytes) != cudaSuccess || cudaMalloc(&dy, bytes) != cudaSuccess) st = NIM_ERR_CUDA;
  if (st == NIM_OK && cudaMemcpy(dx, x, bytes, cudaMemcpyHostToDevice) != cudaSuccess) st = NIM_ERR_CUDA;
  if (st == NIM_OK) {
    const int64_t blocks = std::min<int64_t>((n + BLK - 1) / BLK, 148 * 16);
    k_exp_selftest<<<(unsigned)blocks, BLK>>>(dx, dy, n);
    if (cudaGetLastError() != cudaSuccess || cudaMemcpy(y, dy, bytes, cudaMemcpyDeviceToHost) != cudaSuccess)
      st = NIM_ERR_CUDA;
  }
  cudaFree(dx);
  cudaFree(dy);
  return st;
}

// ---- tangent-linear steps (forward mode): a dual copy of the iterate and
// geometry advanced by the dual instantiations of the step's kernels
namespace {

int dual_alloc(nim_ctx *x) {
  const Dims &d = x->d;
  const size_t Nc = d.Nc, NF = d.NF, NB = d.NBF;
  GeoT<DualD> &h = x->gD;
  TRY(dalloc(x, &h.vol, Nc));
  TRY(dalloc(x, &h.G, 3 * Nc));
  TRY(dalloc(x, &h.gij, 9 * Nc));
  TRY(dalloc(x, &h.xi, 9 * Nc));
  TRY(dalloc(x, &h.gfd, 6 * Nc));
  TRY(dalloc(x, &h.dg, 6 * Nc));
  TRY(dalloc(x, &h.area, NF));
  TRY(dalloc(x, &h.normal, 3 * NF));
  TRY(dalloc(x, &h.AA, 45 * Nc));
  h.bcpts = x->g.bcpts;  // integer: shared with the FP64 side
  TRY(dalloc(x, &h.bca, 5 * NB));
  TRY(dalloc(x, &h.bcap, 8 * NB));
  TRY(dalloc(x, &h.bcg, 2 * NB));
  TRY(dalloc(x, &h.zf, 4 * NB));
  TRY(dalloc(x, &h.nuw, 4 * NB));
  FieldsT<DualD> &H = x->FD;
  for (int q = 0; q < 5; ++q) TRY(dalloc(x, &H.f[q], 2 * NF));
  for (int q = 0; q < 4; ++q) {
    TRY(dalloc(x, &H.c[q], Nc));
    TRY(dalloc(x, &H.co[q], Nc));
    TRY(dalloc(x, &H.ct[q], Nc));
  }
  TRY(dalloc(x, &H.mp, Nc));
  TRY(dalloc(x, &H.dila, Nc));
  TRY(dalloc(x, &H.dila_old, Nc));
  TRY(dalloc(x, &H.Rp, Nc));
  TRY(dalloc(x, &H.MA, 18 * Nc));
  TRY(dalloc(x, &H.MF4, 8 * Nc));
  TRY(dalloc(x, &H.MF, 15 * Nc));
  TRY(dalloc(x, &H.MTF, 15 * Nc));
  TRY(dalloc(x, &H.MTA, 18 * Nc));
  TRY(dalloc(x, &H.dpd, 3 * Nc));
  H.part = x->F.part;  // per-block partial sums: FP64, shared
  TRY(dalloc(x, &x->ctlD, 1));
  x->dual_alloc = true;
  return NIM_OK;
}

// the FP64 geometry and iterate into the dual arrays, derivatives zero
int dual_copy(nim_ctx *x) {
  const Dims &d = x->d;
  const size_t Nc = d.Nc, NF = d.NF, NB = d.NBF;
  const Geo &g = x->g;
  GeoT<DualD> &h = x->gD;
  Cvt c;
  c.add(g.vol, h.vol, Nc);
  c.add(g.G, h.G, 3 * Nc);
  c.add(g.gij, h.gij, 9 * Nc);
  c.add(g.xi, h.xi, 9 * Nc);
  c.add(g.gfd, h.gfd, 6 * Nc);
  c.add(g.dg, h.dg, 6 * Nc);
  c.add(g.area, h.area, NF);
  c.add(g.normal, h.normal, 3 * NF);
  c.add(g.AA, h.AA, 45 * Nc);
  c.add(g.bca, h.bca, 5 * NB);
  c.add(g.bcap, h.bcap, 8 * NB);
  c.add(g.bcg, h.bcg, 2 * NB);
  c.add(g.zf, h.zf, 4 * NB);
  c.add(g.nuw, h.nuw, 4 * NB);
  TRY((run_cvt<double, DualD>(x, c)));
  const Fields &F = x->F;
  FieldsT<DualD> &H = x->FD;
  Cvt s;
  for (int q = 0; q < 5; ++q) s.add(F.f[q], H.f[q], 2 * NF);
  for (int q = 0; q < 4; ++q) {
    s.add(F.c[q], H.c[q], Nc);
    s.add(F.co[q], H.co[q], Nc);
    s.add(F.ct[q], H.ct[q], Nc);
  }
  s.add(F.mp, H.mp, Nc);
  s.add(F.dila, H.dila, Nc);
  s.add(F.dila_old, H.dila_old, Nc);
  s.add(F.dpd, H.dpd, 3 * Nc);
  TRY((run_cvt<double, DualD>(x, s)));
  CK(cudaMemcpyAsync(x->ctlD, x->ctl, sizeof(Ctrl), cudaMemcpyDeviceToDevice, x->stream));
  return NIM_OK;
}

// the dual state of a field: its array (both halves of a face field) or null
struct DualView {
  DualD *p = nullptr, *p1 = nullptr;
  int n = 0;
  bool face = false;
};
int dual_view(nim_ctx *x, nim_field f, int par, DualView &v) {
  const Dims &d = x->d;
  FieldsT<DualD> &H = x->FD;
  auto cellf = [&](DualD *p) { v.p = p; v.n = d.Nc; };
  switch (f) {
    case NIM_FIELD_FACES_U: case NIM_FIELD_FACES_V: case NIM_FIELD_FACES_W: case NIM_FIELD_FACES_P:
    case NIM_FIELD_FACES_T:
      v.p = H.f[(int)f] + (size_t)par * d.NF;
      v.p1 = H.f[(int)f] + (size_t)(1 - par) * d.NF;
      v.n = d.NF;
      v.face = true;
      return NIM_OK;
    case NIM_FIELD_MESHES_U: case NIM_FIELD_MESHES_V: case NIM_FIELD_MESHES_W: case NIM_FIELD_MESHES_T:
      cellf(H.c[(int)f - 5]); return NIM_OK;
    case NIM_FIELD_MESHES_U_OLD: case NIM_FIELD_MESHES_V_OLD: case NIM_FIELD_MESHES_W_OLD:
    case NIM_FIELD_MESHES_T_OLD:
      cellf(H.co[(int)f - 9]); return NIM_OK;
    case NIM_FIELD_MESHES_UT: case NIM_FIELD_MESHES_VT: case NIM_FIELD_MESHES_WT: case NIM_FIELD_MESHES_TT:
      cellf(H.ct[(int)f - 13]); return NIM_OK;
    case NIM_FIELD_MESHES_P: cellf(H.mp); return NIM_OK;
    case NIM_FIELD_MESHES_DILA: cellf(H.dila); return NIM_OK;
    default: return NIM_ERR_BAD_ARG;
  }
}

__global__ void k_dual_gather(const DualD *__restrict__ src, const int *__restrict__ perm, int n,
                              double *__restrict__ v, double *__restrict__ t) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const DualD a = src[perm ? perm[i] : i];
  v[i] = a.v;
  t[i] = a.t;
}
__global__ void k_dual_seed(const double *__restrict__ t, const int *__restrict__ perm, int n, DualD *dst,
                            DualD *dst1) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int s = perm ? perm[i] : i;
  dst[s].t = t[i];
  if (dst1) dst1[s].t = t[i];
}

// the dual state's control block stands in for the context's while a dual
// step runs (the kernels and read_ctrl use x->ctl)
struct DualCtl {
  nim_ctx *x;
  Ctrl *keep;
  explicit DualCtl(nim_ctx *c) : x(c), keep(c->ctl) { x->ctl = x->ctlD; }
  ~DualCtl() { x->ctl = keep; }
};

constexpr int kDualCap = 4000000;  // passes per step without max_iters

// one dual step: begin_step, the inner loop until the reference's test holds,
// after_integrate, update_time_step, find_Nu2; d Nu_inner, d Nu_outer
int dual_step(nim_ctx *x, nim_step_stats *s, double *dnu2) {
  const Dims &d = x->d;
  cudaStream_t st = x->stream;
  DualCtl use(x);
  k_step_reset<<<1, 1, 0, st>>>(x->ctl);
  k_vel_coef_A<<<x->nblk_c, BLK, 0, st>>>(d, x->gD, x->FD, x->phys);
  k_vel_coef_F<<<x->nblk_c, BLK, 0, st>>>(d, x->FD, x->phys);
  CK(cudaGetLastError());
  x->launches += 3;
  for (;;) {
    for (int k = 0; k < 8; ++k) TRY(launch_parallel(x, x->gD, x->FD, 0));
    TRY(read_ctrl(x));
    if (x->ctl_host->done) break;
    if (x->ctl_host->step_iters >= kDualCap) {
      x->ctl_host->status = NIM_ERR_NOT_CONVERGED;
      break;
    }
  }
  const int status = x->ctl_host->status;
  k_after_integrate<<<x->nblk_c, BLK, 0, st>>>(d, x->gD, x->FD, x->phys, x->ctl, x->nblk_c);
  k_finish_sum<<<1, BLK, 0, st>>>(x->F.part, x->nblk_c, 1, x->sums);
  CK(cudaGetLastError());
  x->launches += 2;
  CK(cudaMemcpyAsync(x->host_sums, x->sums, sizeof(double), cudaMemcpyDeviceToHost, st));
  TRY(read_ctrl(x));
  if (s) {
    fill_iter_stats(x, s);
    s->status = status;
    s->iters_fp32 = 0;
    s->dilatation = std::sqrt(x->host_sums[0] / d.Nc);
    s->dudt_max = bits_to_double(x->ctl_host->red[0]);
    s->dTdt_max = bits_to_double(x->ctl_host->red[1]);
  }
  if (status != NIM_OK) return status;
  const int nr = 2 * d.NT * d.NZ, gn = grid(nr);
  k_update_time<<<x->nblk_c, BLK, 0, st>>>(d, x->FD, x->ctl);
  k_nusselt<<<gn, BLK, 0, st>>>(d, x->gD, x->FD, x->ctl, gn);
  k_finish_sum<<<1, BLK, 0, st>>>(x->F.part, gn, 8, x->sums);
  CK(cudaGetLastError());
  x->launches += 3;
  CK(cudaMemcpyAsync(x->host_sums, x->sums, 8 * sizeof(double), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  const double *h = x->host_sums;
  const DualD sum1(h[0], h[4]), sumA1(h[1], h[5]), sum2(h[2], h[6]), sumA2(h[3], h[7]);
  const DualD nu_outer = -(sum1 / sumA1 * x->params.R_o), nu_inner = -(sum2 / sumA2 * x->params.R_i);
  const int32_t step_done = x->dual_STEP;
  x->dual_STEP = x->dual_STEP + 1;
  x->dual_TI = x->dual_TI + 2 * x->params.DT;
  if (s) {
    s->step = step_done;
    s->nu_outer = nu_outer.v;
    s->nu_inner = nu_inner.v;
    s->area_outer = sumA1.v;
    s->area_inner = sumA2.v;
    s->time = x->dual_TI;
  }
  if (dnu2) {
    dnu2[0] = nu_inner.t;
    dnu2[1] = nu_outer.t;
  }
  return NIM_OK;
}
}  // namespace

extern "C" int nim_gpu_tangent_begin(nim_ctx *x) {
  if (!x) return NIM_ERR_BAD_ARG;
  if (!x->initialized || x->in_step) return NIM_ERR_STATE;
  if (x->seq || x->phys.formulation != 2 || x->slab_count) return NIM_ERR_BAD_ARG;
  CK(cudaSetDevice(x->device));
  if (!x->dual_alloc) TRY(dual_alloc(x));
  TRY(dual_copy(x));
  x->phys.d_nu = x->phys.d_alpha = x->phys.d_inv_Re = 0.0;
  x->dual_STEP = x->STEP;
  x->dual_TI = x->TI;
  x->dual_ready = true;
  CK(cudaStreamSynchronize(x->stream));
  return NIM_OK;
}

extern "C" int nim_gpu_tangent_seed(nim_ctx *x, double dnu, double dalpha) {
  if (!x) return NIM_ERR_BAD_ARG;
  if (!x->dual_ready) return NIM_ERR_STATE;
  // Re = 1/nu and 1/Re as the time advance forms them (parameters.f90:172)
  const DualD nu(x->phys.nu, dnu);
  const DualD Re = DualD(1.) / nu;
  const DualD inv_Re = DualD(1.) / Re;
  x->phys.d_nu = dnu;
  x->phys.d_alpha = dalpha;
  x->phys.d_inv_Re = inv_Re.t;
  return NIM_OK;
}

extern "C" int nim_gpu_tangent_seed_field(nim_ctx *x, nim_field f, const double *t, int64_t n) {
  if (!x || !t) return NIM_ERR_BAD_ARG;
  if (!x->dual_ready) return NIM_ERR_STATE;
  CK(cudaSetDevice(x->device));
  DualCtl use(x);
  TRY(read_ctrl(x));
  DualView v;
  TRY(dual_view(x, f, x->ctl_host->iter & 1, v));
  if (n < v.n) return NIM_ERR_BAD_ARG;
  CK(cudaMemcpyAsync(x->scratch, t, sizeof(double) * v.n, cudaMemcpyHostToDevice, x->stream));
  k_dual_seed<<<grid(v.n), BLK, 0, x->stream>>>(x->scratch, v.face ? x->perm : nullptr, v.n, v.p, v.p1);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(x->stream));
  return NIM_OK;
}

extern "C" int nim_gpu_tangent_get(nim_ctx *x, nim_field f, double *value, double *tangent, int64_t n) {
  if (!x || !value || !tangent) return NIM_ERR_BAD_ARG;
  if (!x->dual_ready) return NIM_ERR_STATE;
  CK(cudaSetDevice(x->device));
  DualCtl use(x);
  TRY(read_ctrl(x));
  DualView v;
  TRY(dual_view(x, f, x->ctl_host->iter & 1, v));
  if (n < v.n) return NIM_ERR_BAD_ARG;
  double *sv = x->scratch, *stt = x->scratch + v.n;
  k_dual_gather<<<grid(v.n), BLK, 0, x->stream>>>(v.p, v.face ? x->perm : nullptr, v.n, sv, stt);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(value, sv, sizeof(double) * v.n, cudaMemcpyDeviceToHost, x->stream));
  CK(cudaMemcpyAsync(tangent, stt, sizeof(double) * v.n, cudaMemcpyDeviceToHost, x->stream));
  CK(cudaStreamSynchronize(x->stream));
  return NIM_OK;
}

extern "C" int nim_gpu_tangent_step(nim_ctx *x, int32_t nsteps, nim_step_stats *per_step, double *dnu) {
  if (!x || nsteps < 0) return NIM_ERR_BAD_ARG;
  if (!x->dual_ready) return NIM_ERR_STATE;
  CK(cudaSetDevice(x->device));
  for (int32_t k = 0; k < nsteps; ++k) {
    nim_step_stats rec;
    std::memset(&rec, 0, sizeof(rec));
    const int st = dual_step(x, &rec, dnu ? dnu + 2 * k : nullptr);
    if (per_step) per_step[k] = rec;
    if (st != NIM_OK) return st;
  }
  return NIM_OK;
}

extern "C" int nim_gpu_selftest_nim_coef(const double *u, const double *k, int64_t n, int32_t precision,
                                         double v_limit, double *A) {
  if (n < 0 || (n > 0 && (!u || !k || !A)) || n > (int64_t(1) << 26)) return NIM_ERR_BAD_ARG;
  if (precision != NIM_PRECISION_FP64 && precision != NIM_PRECISION_MIXED) return NIM_ERR_BAD_ARG;
  if (n == 0) return NIM_OK;
  const size_t bytes = (size_t)n * sizeof(double);
  double *du = nullptr, *dk = nullptr, *dA = nullptr;
  int st = NIM_OK;
  if (cudaMalloc(&du, bytes) != cudaSuccess || cudaMalloc(&dk, bytes) != cudaSuccess ||
      cudaMalloc(&dA, 6 * bytes) != cudaSuccess)
    st = NIM_ERR_CUDA;
  if (st == NIM_OK && (cudaMemcpy(du, u, bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
                       cudaMemcpy(dk, k, bytes, cudaMemcpyHostToDevice) != cudaSuccess))
    st = NIM_ERR_CUDA;
  if (st == NIM_OK) {
    const int64_t blocks = std::min<int64_t>((n + BLK - 1) / BLK, 148 * 16);
    k_nim_coef_selftest<<<(unsigned)blocks, BLK>>>(du, dk, dA, n, precision == NIM_PRECISION_MIXED, v_limit);
    if (cudaGetLastError() != cudaSuccess || cudaMemcpy(A, dA, 6 * bytes, cudaMemcpyDeviceToHost) != cudaSuccess)
      st = NIM_ERR_CUDA;
  }
  cudaFree(du);
  cudaFree(dk);
  cudaFree(dA);
  return st;
}

extern "C" const char *nim_gpu_profile_name(nim_ctx *x, int32_t k) {
  return (x && k >= 0 && k < (int32_t)x->prof_names.size()) ? x->prof_names[k].c_str() : "";
}

extern "C" int nim_gpu_nusselt_noalloc(nim_ctx *x, double *out4) {
  if (!x || !out4) return NIM_ERR_BAD_ARG;
  // between steps only: inside a step the face temperatures are mid-iteration
  if (!x->initialized || x->in_step) return NIM_ERR_STATE;
  const Dims &d = x->d;
  const int nr = 2 * d.NT * d.NZ;
  if (nr > NIM_NOALLOC_MAX_WALL_FACES) return NIM_ERR_BAD_ARG;
  CK(cudaSetDevice(x->device));
  TRY(noalloc_setup(x->device));
  double *scratch = g_noalloc_ptr[x->device];
  if (!scratch) return NIM_ERR_STATE;
  const int gn = grid(nr);
  Fields F = x->F;
  F.part = scratch;  // per-block partials into the static array
  k_nusselt<<<gn, BLK, 0, x->stream>>>(d, x->g, F, x->ctl, gn);
  k_finish_sum<<<1, BLK, 0, x->stream>>>(scratch, gn, 4, scratch + 4 * kNoallocBlocks);
  CK(cudaGetLastError());
  x->launches += 2;
  double sums[4];
  CK(cudaMemcpyAsync(sums, scratch + 4 * kNoallocBlocks, sizeof(sums), cudaMemcpyDeviceToHost, x->stream));
  CK(cudaStreamSynchronize(x->stream));
  out4[0] = -(sums[0] / sums[1] * x->params.R_o);
  out4[1] = -(sums[2] / sums[3] * x->params.R_i);
  out4[2] = sums[1];
  out4[3] = sums[3];
  return NIM_OK;
}

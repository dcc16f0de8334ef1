// Fused batch passes: one launch per pass kernel over every enclosure of a
// batch (nim_batch_step_fused).
//
// The reference advances one enclosure per process (solve_nse,
// nse.f90:23-85).  A batch of small enclosures run one at a time, or side by
// side on streams, leaves the GPU to grids of a few dozen blocks each.  Here
// each kernel of the parallel pass is launched once for the whole batch as a
// persistent grid (a few blocks per SM) that walks a work list of
// (enclosure, block) items: the blocks the enclosure's own launch of that
// kernel would have, for every enclosure that is still iterating in the
// kernel's precision.  The work list is rebuilt at the start of every pass
// (k_batch_plan) from each enclosure's stop flag and phase, so enclosures
// whose inner loop has converged drop out of the next pass and the others
// share the whole GPU.  Each item runs the kernel body of the plain launch
// (the *_body functions of nim_kernels.cuh) with the enclosure's own arrays
// and block coordinates, so every enclosure's arithmetic, and its result, is
// the one of its own launches to the bit.
#pragma once
#include "nim_kernels.cuh"

namespace nim {

constexpr int kBatchMax = 256;  // enclosures in one fused batch

// the kernel forms a fused pass launches (one persistent launch each)
enum BatchSlot {
  BS_VEL_CELL2,  // k_vel_cell2 (n_theta even), pairs of cells in cell order (FlatBlock)
  BS_VEL_CELL,   // k_vel_cell (formulation 2), cells in cell order (FlatBlock)
  BS_VEL_FACE,   // k_vel_face (FlatBlock)
  BS_P_SRC2,     // k_p_srcN<double, 2> (FlatBlock)
  BS_P_SRC,      // k_p_src (FlatBlock)
  BS_P_BC,       // k_p_bc
  BS_P_BC_COPY,  // k_p_bc_copy
  BS_P_FACE2,    // k_p_faceN<double, 2> (FlatBlock)
  BS_P_FACE,     // k_p_face (FlatBlock)
  BS_P_DPDX,     // k_p_dpdx (is_dpdx_tolerance)
  BS_ZERO_FLUX,  // k_zero_flux
  BS_T_COEF,     // k_T_coef
  BS_T_CELL,     // k_T_cell (FlatBlock)
  BS_T_FACE,     // k_T_face (FlatBlock)
  BS_COUNT
};

// one enclosure's arguments in one storage type (FP64 arrays or the float
// mirror of a mixed-precision context)
template <class R>
struct BatchInst {
  Dims d;
  GeoT<R> g;
  FieldsT<R> F;
  Phys P;
  Ctrl *ctl;
};

// the grid one enclosure's own launch of a slot's kernel would have, per
// storage type; x = 0 where the enclosure runs another form of that kernel
struct BatchGrid {
  unsigned x, y, z;
};

// The work list of one pass, per phase (0: FP32 mirror, 1: FP64): the
// enclosures iterating in that phase and, per slot, the running count of
// their blocks (off[ph][s][a] = blocks of enclosures inst[ph][0..a-1]).
struct BatchPlan {
  int n[2];
  int inst[2][kBatchMax];
  int off[2][BS_COUNT][kBatchMax + 1];
};

// phase[i]: 0 = not iterating, 1 = FP32 phase of a mixed step, 2 = FP64 passes
struct BatchArgs {
  const BatchInst<double> *__restrict__ i64;
  const BatchInst<float> *__restrict__ i32;  // null unless mixed
  const BatchGrid *__restrict__ grid;        // [2][n][BS_COUNT] per phase (float, double)
  const int *phase;                          // [n]
  BatchPlan *plan;
  int n;
};

struct BatchState {
  int done, status;
};

template <class R>
__device__ __forceinline__ const BatchInst<R> &batch_inst(const BatchArgs &A, int i);
template <>
__device__ __forceinline__ const BatchInst<double> &batch_inst<double>(const BatchArgs &A, int i) {
  return A.i64[i];
}
template <>
__device__ __forceinline__ const BatchInst<float> &batch_inst<float>(const BatchArgs &A, int i) {
  return A.i32[i];
}

// the work list of the coming pass, by one block of 32 x 32 threads: the
// enclosures still iterating in each phase are compacted by warps 0 and 1
// (ballots over chunks of 32), then warp 2 ph + ... sums the blocks of slot
// s over phase ph's list (warp w = ph * BS_COUNT + s, shuffle scans over
// chunks of 32).
__global__ void __launch_bounds__(1024) k_batch_plan(BatchArgs A) {
  static_assert(2 * BS_COUNT <= 32, "one warp per phase and slot");
  BatchPlan *pl = A.plan;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (w < 2) {
    int m = 0;
    for (int base = 0; base < A.n; base += 32) {
      const int i = base + lane;
      const bool on = i < A.n && A.phase[i] == w + 1 && !A.i64[i].ctl->done;
      const unsigned mask = __ballot_sync(0xffffffffu, on);
      if (on) pl->inst[w][m + __popc(mask & ((1u << lane) - 1u))] = i;
      m += __popc(mask);
    }
    if (lane == 0) pl->n[w] = m;
  }
  __syncthreads();
  if (w < 2 * BS_COUNT) {
    const int ph = w / BS_COUNT, s = w % BS_COUNT, m = pl->n[ph];
    int acc = 0;
    for (int base = 0; base < m; base += 32) {
      const int a = base + lane;
      int v = 0;
      if (a < m) {
        const BatchGrid gr = A.grid[(ph * A.n + pl->inst[ph][a]) * BS_COUNT + s];
        v = (int)(gr.x * gr.y * gr.z);
      }
      int incl = v;  // inclusive scan over the warp
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
      }
      if (a < m) pl->off[ph][s][a] = acc + incl - v;
      acc += __shfl_sync(0xffffffffu, incl, 31);
    }
    if (lane == 0) pl->off[ph][s][m] = acc;
  }
}

// Walk the pass's work list for slot S over the arrays of storage type R
// (phase 0 for float, 1 for double).  The block first copies the list's
// running counts, enclosures and grids for S into shared memory; its items
// (w = blockIdx.x, + gridDim.x, ...) only move forward through the list, so
// each finds its enclosure by a short forward scan.  The enclosure's
// arguments are copied into shared memory when the enclosure changes, and
// the body reads them there.  The barrier after each item keeps one item's
// shared-memory use apart from the next one's.
template <int S, class R, class BI = BatchBlock, class Body>
__device__ __forceinline__ void batch_items(const BatchArgs &A, Body &&body) {
  constexpr int ph = sizeof(R) == 4 ? 0 : 1;
  constexpr int kWords = sizeof(BatchInst<R>) / 8;
  static_assert(sizeof(BatchInst<R>) % 8 == 0, "the enclosure's arguments copy as 8-byte words");
  __shared__ int s_off[kBatchMax + 1];
  __shared__ int s_inst[kBatchMax];
  __shared__ BatchGrid s_grid[kBatchMax];
  __shared__ __align__(16) unsigned long long s_args[kWords];
  const int tid = threadIdx.x + blockDim.x * threadIdx.y, nth = blockDim.x * blockDim.y;
  const BatchPlan *pl = A.plan;
  const int m = pl->n[ph];
  if (blockIdx.x >= pl->off[ph][S][m]) return;  // no item for this block
  for (int a = tid; a <= m; a += nth) s_off[a] = pl->off[ph][S][a];
  for (int a = tid; a < m; a += nth) {
    const int i = pl->inst[ph][a];
    s_inst[a] = i;
    s_grid[a] = A.grid[(ph * A.n + i) * BS_COUNT + S];
  }
  __syncthreads();
  const int total = s_off[m];
  const BatchInst<R> &I = *reinterpret_cast<const BatchInst<R> *>(s_args);
  int lo = 0, cur = -1;
  for (int w = blockIdx.x; w < total; w += gridDim.x) {
    while (s_off[lo + 1] <= w) ++lo;  // the enclosure with blocks at w
    if (lo != cur) {
      const unsigned long long *src = reinterpret_cast<const unsigned long long *>(&batch_inst<R>(A, s_inst[lo]));
      for (int q = tid; q < kWords; q += nth) s_args[q] = src[q];
      cur = lo;
      __syncthreads();
    }
    const BatchGrid gr = s_grid[lo];
    const unsigned l = (unsigned)(w - s_off[lo]), r = l / gr.x;
    BI b;
    b.x = l - r * gr.x;
    b.y = r % gr.y;
    b.z = r / gr.y;
    body(I, b);
    __syncthreads();
  }
}

// The batched launches run the plain kernels' bodies.  W = 0: the plain
// kernels' launch bounds; W = 1: one resident block per SM fewer, which
// leaves registers for the enclosure's arguments (in the plain launches they
// are kernel parameters, read from the constant bank; here they come from
// the enclosure table in global memory and take registers).
constexpr int wider(int blocks, int w) { return blocks - w > 1 ? blocks - w : 1; }
template <class R, int W>
__global__ void __launch_bounds__(CB3, wider(minb<R>(VC2_MINB, VC2_MINB_F), W)) kb_vel_cell2(BatchArgs A) {
  batch_items<BS_VEL_CELL2, R, FlatBlock>(A, [&](const BatchInst<R> &I, FlatBlock b) {
    vel_cell2_body<R, false>(I.d, I.g, I.F, I.P, I.ctl, b);
  });
}
template <class R, int W>
__global__ void __launch_bounds__(CB3, wider(3, W)) kb_vel_cell(BatchArgs A) {
  batch_items<BS_VEL_CELL, R, FlatBlock>(A, [&](const BatchInst<R> &I, FlatBlock b) {
    vel_cell_body<false, 2, R>(I.d, I.g, I.F, I.P, I.ctl, b);
  });
}
template <class R, int W>
__global__ void __launch_bounds__(CB3, wider(3, W)) kb_vel_face(BatchArgs A) {
  batch_items<BS_VEL_FACE, R, FlatBlock>(A, [&](const BatchInst<R> &I, FlatBlock b) {
    vel_face_body<R>(I.d, I.g, I.F, I.P, I.ctl, b);
  });
}
template <int W>
__global__ void __launch_bounds__(CB3, wider(PSN_MINB, W)) kb_p_src2(BatchArgs A) {
  batch_items<BS_P_SRC2, double, FlatBlock>(A, [&](const BatchInst<double> &I, FlatBlock b) {
    p_srcN_body<double, 2>(I.d, I.g, I.F, I.P, I.ctl, b);
  });
}
template <class R, int W>
__global__ void __launch_bounds__(CB3, wider(minb<R>(4, PSRC_MINB_F), W)) kb_p_src(BatchArgs A) {
  batch_items<BS_P_SRC, R, FlatBlock>(A, [&](const BatchInst<R> &I, FlatBlock b) {
    p_src_body<R>(I.d, I.g, I.F, I.P, I.ctl, b);
  });
}
template <class R, int W>
__global__ void __launch_bounds__(BLK) kb_p_bc(BatchArgs A) {
  batch_items<BS_P_BC, R>(A, [&](const BatchInst<R> &I, BatchBlock b) {
    p_bc_body<R>(I.d, I.g, I.F, I.P, I.ctl, b);
  });
}
template <class R, int W>
__global__ void __launch_bounds__(BLK) kb_p_bc_copy(BatchArgs A) {
  batch_items<BS_P_BC_COPY, R>(A, [&](const BatchInst<R> &I, BatchBlock b) {
    p_bc_copy_body<R>(I.d, I.F, I.ctl, b);
  });
}
template <int W>
__global__ void __launch_bounds__(CB3, wider(PFN_MINB, W)) kb_p_face2(BatchArgs A) {
  batch_items<BS_P_FACE2, double, FlatBlock>(A, [&](const BatchInst<double> &I, FlatBlock b) {
    p_faceN_body<double, 2>(I.d, I.g, I.F, I.P, I.ctl, b);
  });
}
template <class R, int W>
__global__ void __launch_bounds__(CB3, wider(minb<R>(5, PFACE_MINB_F), W)) kb_p_face(BatchArgs A) {
  batch_items<BS_P_FACE, R, FlatBlock>(A, [&](const BatchInst<R> &I, FlatBlock b) {
    p_face_body<R>(I.d, I.g, I.F, I.P, I.ctl, b);
  });
}
template <class R, int W>
__global__ void __launch_bounds__(BLK) kb_p_dpdx(BatchArgs A) {
  batch_items<BS_P_DPDX, R>(A, [&](const BatchInst<R> &I, BatchBlock b) {
    p_dpdx_body<R>(I.d, I.g, I.F, I.ctl, b);
  });
}
template <class R, int W>
__global__ void __launch_bounds__(BLK) kb_zero_flux(BatchArgs A) {
  batch_items<BS_ZERO_FLUX, R>(A, [&](const BatchInst<R> &I, BatchBlock b) {
    zero_flux_body<R>(I.d, I.g, I.F, I.ctl, b);
  });
}
template <class R, int W>
__global__ void __launch_bounds__(BLK, wider(4, W)) kb_T_coef(BatchArgs A) {
  batch_items<BS_T_COEF, R>(A, [&](const BatchInst<R> &I, BatchBlock b) {
    T_coef_body<R>(I.d, I.g, I.F, I.P, I.ctl, b);
  });
}
template <class R, int W>
__global__ void __launch_bounds__(CB3, wider(minb<R>(5, TCELL_MINB_F), W)) kb_T_cell(BatchArgs A) {
  batch_items<BS_T_CELL, R, FlatBlock>(A, [&](const BatchInst<R> &I, FlatBlock b) {
    T_cell_body<false, R>(I.d, I.g, I.F, I.P, I.ctl, b);
  });
}
template <class R, int W>
__global__ void __launch_bounds__(BLK, wider(minb<R>(4, TFACE_MINB_F), W)) kb_T_face(BatchArgs A) {
  batch_items<BS_T_FACE, R, FlatBlock>(A, [&](const BatchInst<R> &I, FlatBlock b) {
    T_face_body<R>(I.d, I.g, I.F, I.P, I.ctl, b);
  });
}

// ---- the same pass kernels as plain (non-persistent) launches over up to
// kGroup enclosures whose arguments travel in the launch's own parameters:
// block b -> enclosure by a search over running block counts in the
// parameter block, so the enclosure index, its arrays and its sizes are
// launch constants read from the constant bank, as in the plain kernels,
// instead of values in registers.  The host groups the enclosures that
// iterate in the launch's precision; the blocks of one whose loop stops
// between the host's reads of the stop flags return at once.
constexpr int kGroup = 40;  // enclosures per launch: 40 x 704 bytes of arguments
template <class R>
struct BatchGroup {
  int n;             // enclosures in the group
  int ph;            // the phase this launch serves (1: FP32 mirror, 2: FP64)
  const int *phase;  // [batch] the enclosures' phases
  int idx[kGroup];   // the members' indices in the batch
  unsigned off[kGroup + 1];
  BatchGrid grid[kGroup];
  BatchInst<R> inst[kGroup];
};
static_assert(sizeof(BatchGroup<double>) < 32000, "kernel parameters stay below 32 KB");

template <class R, class BI, class Body>
__device__ __forceinline__ void group_item(const BatchGroup<R> &L, Body &&body) {
  const unsigned w = blockIdx.x;
  int lo = 0, hi = L.n - 1;  // the last a with off[a] <= w
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (L.off[mid] <= w)
      lo = mid;
    else
      hi = mid - 1;
  }
  if (L.phase[L.idx[lo]] != L.ph) return;
  const BatchGrid gr = L.grid[lo];
  const unsigned l = w - L.off[lo], r = l / gr.x;
  BI b;
  b.x = l - r * gr.x;
  b.y = r % gr.y;
  b.z = r / gr.y;
  body(L.inst[lo], b);
}
template <class R>
__global__ void __launch_bounds__(CB3, minb<R>(VC2_MINB, VC2_MINB_F)) kg_vel_cell2(const __grid_constant__ BatchGroup<R> L) {
  group_item<R, FlatBlock>(L, [&](const BatchInst<R> &I, FlatBlock b) { vel_cell2_body<R, false>(I.d, I.g, I.F, I.P, I.ctl, b); });
}
template <class R>
__global__ void __launch_bounds__(CB3, 3) kg_vel_cell(const __grid_constant__ BatchGroup<R> L) {
  group_item<R, FlatBlock>(L, [&](const BatchInst<R> &I, FlatBlock b) { vel_cell_body<false, 2, R>(I.d, I.g, I.F, I.P, I.ctl, b); });
}
template <class R>
__global__ void __launch_bounds__(CB3, 3) kg_vel_face(const __grid_constant__ BatchGroup<R> L) {
  group_item<R, FlatBlock>(L, [&](const BatchInst<R> &I, FlatBlock b) { vel_face_body<R>(I.d, I.g, I.F, I.P, I.ctl, b); });
}
__global__ void __launch_bounds__(CB3, PSN_MINB) kg_p_src2(const __grid_constant__ BatchGroup<double> L) {
  group_item<double, FlatBlock>(L, [&](const BatchInst<double> &I, FlatBlock b) { p_srcN_body<double, 2>(I.d, I.g, I.F, I.P, I.ctl, b); });
}
template <class R>
__global__ void __launch_bounds__(CB3, minb<R>(4, PSRC_MINB_F)) kg_p_src(const __grid_constant__ BatchGroup<R> L) {
  group_item<R, FlatBlock>(L, [&](const BatchInst<R> &I, FlatBlock b) { p_src_body<R>(I.d, I.g, I.F, I.P, I.ctl, b); });
}
template <class R>
__global__ void __launch_bounds__(BLK) kg_p_bc(const __grid_constant__ BatchGroup<R> L) {
  group_item<R, BatchBlock>(L, [&](const BatchInst<R> &I, BatchBlock b) { p_bc_body<R>(I.d, I.g, I.F, I.P, I.ctl, b); });
}
template <class R>
__global__ void __launch_bounds__(BLK) kg_p_bc_copy(const __grid_constant__ BatchGroup<R> L) {
  group_item<R, BatchBlock>(L, [&](const BatchInst<R> &I, BatchBlock b) { p_bc_copy_body<R>(I.d, I.F, I.ctl, b); });
}
__global__ void __launch_bounds__(CB3, PFN_MINB) kg_p_face2(const __grid_constant__ BatchGroup<double> L) {
  group_item<double, FlatBlock>(L, [&](const BatchInst<double> &I, FlatBlock b) { p_faceN_body<double, 2>(I.d, I.g, I.F, I.P, I.ctl, b); });
}
template <class R>
__global__ void __launch_bounds__(CB3, minb<R>(5, PFACE_MINB_F)) kg_p_face(const __grid_constant__ BatchGroup<R> L) {
  group_item<R, FlatBlock>(L, [&](const BatchInst<R> &I, FlatBlock b) { p_face_body<R>(I.d, I.g, I.F, I.P, I.ctl, b); });
}
template <class R>
__global__ void __launch_bounds__(BLK) kg_p_dpdx(const __grid_constant__ BatchGroup<R> L) {
  group_item<R, BatchBlock>(L, [&](const BatchInst<R> &I, BatchBlock b) { p_dpdx_body<R>(I.d, I.g, I.F, I.ctl, b); });
}
template <class R>
__global__ void __launch_bounds__(BLK) kg_zero_flux(const __grid_constant__ BatchGroup<R> L) {
  group_item<R, BatchBlock>(L, [&](const BatchInst<R> &I, BatchBlock b) { zero_flux_body<R>(I.d, I.g, I.F, I.ctl, b); });
}
template <class R>
__global__ void __launch_bounds__(BLK, 4) kg_T_coef(const __grid_constant__ BatchGroup<R> L) {
  group_item<R, BatchBlock>(L, [&](const BatchInst<R> &I, BatchBlock b) { T_coef_body<R>(I.d, I.g, I.F, I.P, I.ctl, b); });
}
template <class R>
__global__ void __launch_bounds__(CB3, minb<R>(5, TCELL_MINB_F)) kg_T_cell(const __grid_constant__ BatchGroup<R> L) {
  group_item<R, FlatBlock>(L, [&](const BatchInst<R> &I, FlatBlock b) { T_cell_body<false, R>(I.d, I.g, I.F, I.P, I.ctl, b); });
}
template <class R>
__global__ void __launch_bounds__(BLK, minb<R>(4, TFACE_MINB_F)) kg_T_face(const __grid_constant__ BatchGroup<R> L) {
  group_item<R, FlatBlock>(L, [&](const BatchInst<R> &I, FlatBlock b) { T_face_body<R>(I.d, I.g, I.F, I.P, I.ctl, b); });
}

// find_error's stop test of every enclosure iterating this pass, in its
// phase's form (k_iter_end; lowp for the FP32 phase)
__global__ void k_batch_iter_end(BatchArgs A) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  const int ph = A.phase[i];
  if (ph == 0) return;
  iter_end_body(A.i64[i].ctl, A.i64[i].P, ph == 1 ? 1 : 0, BatchBlock{0u, 0u, 0u});
}

// every enclosure's stop flag and status, gathered for one copy to the host
__global__ void k_batch_state(BatchArgs A, BatchState *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  const Ctrl *c = A.i64[i].ctl;
  out[i].done = c->done;
  out[i].status = c->status;
}

}  // namespace nim

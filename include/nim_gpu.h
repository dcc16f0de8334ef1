/*
 * nim_gpu.h -- C ABI of the B200 (sm_100a) NIM time-advance library.
 *
 * The reference solver (ijarrah2/NIM-CONV22-SHARED, Fortran 90 + OpenMP)
 * advances incompressible Navier-Stokes + Boussinesq energy with the nodal
 * integral method by calling argument-less subroutines that work on module
 * globals (src/parameters.f90:222-292).  This header replaces those calls
 * with plain-C entry points taking pointers and sizes; a Fortran host binds
 * them with iso_c_binding through a bind(C) interface block.
 *
 * Conventions
 *   - Every entry point returns an int status: NIM_OK (0) or a negative
 *     NIM_ERR_* code; nim_gpu_strerror() turns it into text.
 *   - Arrays crossing the boundary use the reference's own layout:
 *     column-major (component, index) with 1-based cell / face / node
 *     numbers, exactly as meshes_faces(1:6,1:NMESH) etc. in
 *     src/parameters.f90.  The library copies what it needs during the
 *     call and never keeps a host pointer.
 *   - A context is bound to the CUDA device that is current when it is
 *     created and to its own stream; calls on one context must come from one
 *     host thread at a time (the reference runs single-threaded, run.sh:2).
 *   - Device state stays resident between calls; host copies happen only in
 *     nim_gpu_create, nim_gpu_download and nim_gpu_upload.
 */
#ifndef NIM_GPU_H
#define NIM_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
enum {
  NIM_OK = 0,
  NIM_ERR_BAD_ARG = -1,       /* null pointer, bad size, unsupported mesh   */
  NIM_ERR_CUDA = -2,          /* a CUDA runtime call failed                 */
  NIM_ERR_NOT_CONVERGED = -3, /* inner loop hit max_iters (nse.f90:129 has
                                 no cap; this is the added guard)           */
  NIM_ERR_NONFINITE = -4,     /* NaN/Inf seen by the fused error reduction  */
  NIM_ERR_TIMEOUT = -5,       /* a bounded device wait expired              */
  NIM_ERR_STATE = -6          /* call out of order (e.g. step before init)  */
};

/* BC ids of the cylinder case, create_geometry.f90:474-594:
   1 interior, 2 bottom (z=0), 3 top (z=L), 4 inner hexagon, 5 outer wall. */
#define NIM_NBC 5

/* Fields for nim_gpu_download / nim_gpu_upload, in reference names. */
typedef enum nim_field {
  NIM_FIELD_FACES_U = 0,     /* faces_u(NFACE)          */
  NIM_FIELD_FACES_V = 1,     /* faces_v(NFACE)          */
  NIM_FIELD_FACES_W = 2,     /* faces_w(NFACE)          */
  NIM_FIELD_FACES_P = 3,     /* faces_p(NFACE)          */
  NIM_FIELD_FACES_T = 4,     /* faces_T(NFACE)          */
  NIM_FIELD_MESHES_U = 5,    /* meshes_uxyz(NMESH)      */
  NIM_FIELD_MESHES_V = 6,    /* meshes_vxyz(NMESH)      */
  NIM_FIELD_MESHES_W = 7,    /* meshes_wxyz(NMESH)      */
  NIM_FIELD_MESHES_T = 8,    /* meshes_Txyz(NMESH)      */
  NIM_FIELD_MESHES_U_OLD = 9,   /* meshes_uxyz_old       */
  NIM_FIELD_MESHES_V_OLD = 10,  /* meshes_vxyz_old       */
  NIM_FIELD_MESHES_W_OLD = 11,  /* meshes_wxyz_old       */
  NIM_FIELD_MESHES_T_OLD = 12,  /* meshes_Txyz_old       */
  NIM_FIELD_MESHES_UT = 13,  /* meshes_uxyzt (time average, nse.f90:1299) */
  NIM_FIELD_MESHES_VT = 14,  /* meshes_vxyzt            */
  NIM_FIELD_MESHES_WT = 15,  /* meshes_wxyzt            */
  NIM_FIELD_MESHES_TT = 16,  /* meshes_Txyzt            */
  NIM_FIELD_MESHES_P = 17,   /* meshes_p (face mean, nse.f90:1307)        */
  NIM_FIELD_MESHES_DILA = 18,/* meshes_dila (evaluate_D, nse.f90:2530)    */
  NIM_FIELD_MESHES_DILA_OLD = 19, /* meshes_dila_old (write_restart, restart.f90:37) */
  /* init-time geometry (read-only; download only) */
  NIM_FIELD_MESHES_VOLUME = 32,  /* meshes_volume(NMESH)                  */
  NIM_FIELD_FACES_AREA = 33,     /* faces_area(NFACE)                     */
  NIM_FIELD_FACES_NORMAL = 34,   /* faces_normal(3,NFACE)                 */
  NIM_FIELD_FACES_MID = 35,      /* faces_mid_coordinates(3,NFACE)        */
  NIM_FIELD_MESHES_GIJ = 36,     /* meshes_gij(3,3,NMESH)                 */
  NIM_FIELD_MESHES_XI_X = 37,    /* meshes_xi_x(3,3,NMESH)                */
  NIM_FIELD_MESHES_G = 38,       /* (G1,G2,G3) as (3,NMESH)               */
  NIM_FIELD_MESHES_GIJ_FACES = 39,/* meshes_gij_faces(3,3,6,NMESH)        */
  NIM_FIELD_FACES_TANGENTIAL = 40,   /* faces_tangential(3,NFACE)         */
  NIM_FIELD_FACES_BITANGENTIAL = 41, /* faces_bitangential(3,NFACE)       */
  NIM_FIELD_BCS_FACES_A = 42,    /* BCs_faces_a(1:5,tot_faces_bcs) used   */
  NIM_FIELD_BCS_FACES_AP = 43,   /* BCs_faces_ap(8,tot_faces_bcs)         */
  NIM_FIELD_AA_PX = 44,          /* AA_px(15,NMESH) (0 where no +neighbour)*/
  NIM_FIELD_AA_PY = 45,
  NIM_FIELD_AA_PZ = 46,
  /* per-step NIM coefficients (download only) */
  NIM_FIELD_M_F4 = 48,           /* M_F4(8,NMESH)                         */
  NIM_FIELD_M_F1 = 49,           /* M_F1(5,NMESH)                         */
  NIM_FIELD_M_F2 = 50,
  NIM_FIELD_M_F3 = 51
} nim_field;

/*
 * Mesh as the reference host builds it (create_hollow, prepare_mesh,
 * fill_global_arrays: create_geometry.f90:321-664, prepare_mesh.f90:11-183,
 * geometry.f90:978-1032).  All index arrays are 1-based, column-major.
 * The library accepts the structured O-grid these routines produce
 * (n_theta x n_r x n_z cells, periodic in theta); create() verifies the
 * connectivity against that pattern and refuses anything else.
 */
typedef struct nim_mesh_desc {
  int32_t n_theta, n_r, n_z;     /* NMESH_i, NMESH_j, NMESH_k               */
  int32_t nnode, nmesh, nface;   /* NNODE, NMESH, NFACE (parameters.f90:115-119) */
  int32_t nbcface;               /* tot_faces_bcs                           */
  const double  *node_xyz;       /* (3,NNODE): NODES_ARRAY(:)%x,%y,%z       */
  const int32_t *meshes_nodes;   /* (8,NMESH): MESHES_ARRAY(:)%nodes        */
  const int32_t *meshes_faces;   /* (6,NMESH)                               */
  const int32_t *meshes_neighbors; /* (6,NMESH), 0 = wall                   */
  const int32_t *faces_bc;       /* (NFACE): faces_BC                       */
  const int32_t *bcs_faces;      /* (tot_faces_bcs): BCs_faces             */
  const int32_t *bcs_faces_id;   /* BCs_faces_id                            */
  const int32_t *bcs_faces_position; /* BCs_faces_position (1..6)           */
  const int32_t *bcs_faces_mesh_num; /* BCs_faces_mesh_num                  */
} nim_mesh_desc;

/*
 * Run-time counterpart of the compile-time parameters in parameters.f90.
 * nim_params_reference() fills the reference defaults.
 */
typedef struct nim_params {
  double DT;            /* half-width of the NIM time element (parameters.f90:134);
                           one step advances time by 2*DT (nse.f90:1296)       */
  double nu, alpha, rho, g_beta;   /* parameters.f90:163-173                  */
  double w_u, w_v, w_w, w_p, w_p2, w_T; /* relaxation (parameters.f90:152-157) */
  double tol_u, tol_v, tol_w, tol_p, tol_T; /* parameters.f90:146-150          */
  double v_limit;       /* exact/series switch on |cell Peclet| (parameters.f90:128) */
  double dudt_epsilon;  /* steady-state threshold (parameters.f90:151)         */
  double R_i, R_o;      /* radii in the Nusselt scaling of find_Nu2 (nse.f90:2794) */
  /* Dirichlet value of each field on each BC id (general.f90:34-149), used as
     constants integrated over the face like apply_dirichlet_bc_i (bc.f90:59-88).
     Index [field][bc_id-1], field 0..4 = u, v, w, p, T. */
  double bc_value[5][NIM_NBC];
  int32_t max_iters;    /* cap on inner iterations per step (new guard)       */
  int32_t check_steady; /* 1: stop nim_gpu_step when dudt,dTdt < dudt_epsilon
                           (is_check_steady_state, nse.f90:60-69)              */
  int32_t dpdx_tolerance; /* 1: err_p from pressure gradients (is_dpdx_tolerance,
                           nse.f90:292-307)                                     */
  int32_t schedule;     /* NIM_SCHEDULE_PARALLEL (0): every sweep reads the
                           values from before the sweep (fastest);
                           NIM_SCHEDULE_REFERENCE (1): the Gauss-Seidel sweeps
                           run in the reference's cell-number order
                           (run.sh:2, one OpenMP thread), reproducing its
                           iterates                                          */
  int32_t formulation;  /* nim_formulation (parameters.f90:194): 2 (default),
                           or 1 for the velocity NIM constants and sweep of
                           calculate_velocity_nim_constants (nim.f90:17-157)
                           and integrate_velocity_field_i (nse.f90:330-828);
                           pressure and temperature are the same in both.
                           Formulation 1's inner loop converges in the
                           reference's Gauss-Seidel order but can diverge
                           under NIM_SCHEDULE_PARALLEL on coarse meshes:
                           pair it with NIM_SCHEDULE_REFERENCE            */
  int32_t precision;    /* NIM_PRECISION_FP64 (0): every pass in FP64, as the
                           reference; NIM_PRECISION_MIXED (1): each step's
                           inner loop first sweeps a float copy of the
                           fields, NIM constants and geometry (float
                           arithmetic, maxima of the stored changes in
                           double) until the tolerances hold or
                           8 passes in a row bring no new smallest change
                           to a field above its tolerance; the iterate is
                           then widened and FP64 passes run until the
                           reference's test holds.  Per-step work, the
                           reductions and the Nusselt integrals stay FP64.
                           max_iters bounds both phases together.
                           Parallel schedule and formulation 2 only
                           (NIM_ERR_BAD_ARG otherwise); nim_gpu_iterate
                           always runs FP64 passes                        */
} nim_params;

enum { NIM_SCHEDULE_PARALLEL = 0, NIM_SCHEDULE_REFERENCE = 1 };
enum { NIM_PRECISION_FP64 = 0, NIM_PRECISION_MIXED = 1 };

/* Statistics of one time step (the values the reference prints at
   nse.f90:169-171 and nse.f90:2793-2794, returned instead of printed). */
typedef struct nim_step_stats {
  int32_t step;         /* STEP before update_time_step                      */
  int32_t iters;        /* inner iterations (cnt)                            */
  double err_u, err_v, err_w, err_p, err_T;
  double dilatation;    /* evaluate_D RMS continuity residual                */
  double dudt_max, dTdt_max;  /* check_steady_state                          */
  double nu_outer, nu_inner;  /* printed Nu_H (outer, position 2) and Nu_C
                                 (inner hexagon = hot wall, position 1)      */
  double area_outer, area_inner; /* sumA1, sumA2                            */
  double time;          /* TI after update_time_step                         */
  int32_t steady;       /* 1 if the steady-state test fired at this step     */
  int32_t status;       /* NIM_OK or an error of this step                   */
  int32_t iters_fp32;   /* of iters, the FP32 passes (NIM_PRECISION_MIXED)   */
  int32_t pad;
} nim_step_stats;

typedef struct nim_ctx nim_ctx;

/* Fill p with the reference defaults (parameters.f90, nim_formulation=2). */
void nim_params_reference(nim_params *p);

/* Copy the mesh and parameters to the device.  Replaces the module-global
   allocation of parameters.f90:222-292.  *out receives the context.
   The +xi face sweep of u, v, w runs in its TMA-staged form when n_theta is
   a multiple of 4, at most 256, and the mesh gives at least four blocks per
   SM, else in its gather form (the results are identical);
   NIM_FACE_SWEEP=tile or =gather in the environment overrides the choice.
   The u, v, w source and cell sweep (formulation 2) runs on theta-adjacent
   cell pairs with paired loads when n_theta is even, else one cell per
   thread; NIM_CELL_SWEEP=gather forces the one-cell form, =tile a
   TMA-staged form under the face sweep's n_theta conditions (not faster at
   the benchmark sizes, so off by default).  All forms give identical
   results. */
int nim_gpu_create(const nim_mesh_desc *mesh, const nim_params *params,
                   nim_ctx **out);

/* Init-time geometry and constants: evaluate_all_mesh_constants
   (geometry.f90:14-32), evaluate_pressure_bc_array (geometry.f90:879-975),
   calculate_pressure_nim_constants (nim.f90:556-743),
   find_derivatives_pressure_boundary (bc.f90:122-137) and
   apply_all_dirichlet_bcs (bc.f90:13-19); sets TI=DT, STEP=1
   (nse.f90:31-38). */
int nim_gpu_init(nim_ctx *ctx);

/* calculate_velocity_nim_constants_formulation2 (nim.f90:160-330). */
int nim_gpu_begin_step(nim_ctx *ctx);

/* integrate_nse (nse.f90:117-176) with the max_iters guard; fills
   iters, err_u..err_T, dilatation, dudt_max, dTdt_max of *stats
   (stats may be NULL). */
int nim_gpu_integrate(nim_ctx *ctx, nim_step_stats *stats);

/* Exactly n passes of the integrate_nse loop body (nse.f90:131-160) with no
   convergence test: for step-by-step parity checks and fixed-work timing.
   Fills iters and err_u..err_T of *stats (stats may be NULL). */
int nim_gpu_iterate(nim_ctx *ctx, int32_t n, nim_step_stats *stats);

/* update_time_step (nse.f90:1292-1313) + find_Nu2 (nse.f90:2699-2798);
   fills step, nu_outer, nu_inner, area_outer, area_inner and time of
   *stats (stats may be NULL). */
int nim_gpu_end_step(nim_ctx *ctx, nim_step_stats *stats);

/* nsteps iterations of the reference time loop (nse.f90:47-75) fully on
   the device; per_step (may be NULL) receives nsteps records.  Stops early,
   like the reference, when check_steady is set and the steady test fires;
   *done (may be NULL) receives the number of steps advanced. */
int nim_gpu_step(nim_ctx *ctx, int32_t nsteps, nim_step_stats *per_step,
                 int32_t *done);

/* Inner iterations per CUDA-graph launch of nim_gpu_integrate (1..256,
   default 4; no counterpart in the reference).  The device stops the loop
   itself at convergence, so the results never depend on it; larger values
   mean fewer host round trips per step (at most n-1 empty iterations are
   launched after convergence).  Tuning knob for nim_batch_step. */
int nim_gpu_set_graph_iters(nim_ctx *ctx, int32_t n);

/* nim_gpu_step for n independent contexts (enclosures of any size and
   parameters, on one device) advanced together.  No counterpart in the
   reference, which runs one enclosure per process.  One host thread keeps
   every context's stream fed and polls their progress, so the kernels of
   all instances share the GPU; per instance the work and its order are
   exactly nim_gpu_step's, so results are bit-identical to running the
   instances one at a time.  per (may be NULL) receives n*nsteps records,
   row i*nsteps + s for step s of instance i; done (may be NULL) receives
   the steps each instance advanced (an instance stops early on an error or
   the steady test).  Returns the first error any instance met, else
   NIM_OK. */
int nim_batch_step(int32_t n, nim_ctx *const *ctx, int32_t nsteps, nim_step_stats *per, int32_t *done);

/* nim_batch_step with every kernel of a pass launched once for the whole
   batch (no counterpart in the reference).  Each pass kernel runs as a
   persistent grid (a few blocks per SM) over a work list of (enclosure,
   block) items, rebuilt on the device at the start of every pass from each
   enclosure's stop flag, so enclosures whose inner loop has converged drop
   out and the rest share the GPU; the passes are replayed as CUDA graphs
   of nim_gpu_set_graph_iters passes (the first context's setting), and
   between graph launches the host ends the step of each enclosure whose
   loop has stopped and starts its next one, so every enclosure advances
   at its own pace.  The work of each enclosure, and so its result, is
   bit-identical to nim_gpu_step's and nim_batch_step's; per and done as
   for nim_batch_step.  All contexts on
   one device, parallel schedule, formulation 2, the same precision, at
   most 256 (NIM_ERR_BAD_ARG otherwise).  While the call runs, the
   contexts' work goes to a stream of its own; each context's stream is
   synchronised at entry and given back at return.  With the environment
   variable NIM_BATCH_FORM=grid the kernels run instead as plain launches
   over groups of up to 40 enclosures whose arguments are kernel
   parameters, regrouped as enclosures change precision (faster for FP64
   batches); the results are the same bits. */
int nim_batch_step_fused(int32_t n, nim_ctx *const *ctx, int32_t nsteps, nim_step_stats *per, int32_t *done);

/* ---- z-slab decomposition (no counterpart in the reference, which runs
   one enclosure on one node).  The n_z cell planes split into nslab
   contiguous slabs of n_z / nslab or one more planes (at least 2 each).
   A slab's context holds its own planes and, on each side with a
   neighbour slab, that neighbour's two nearest planes (the halo: the
   farthest any stencil of an owned cell or face reaches in z away from
   the physical walls).  find_error's maxima, check_steady_state, evaluate_D
   and find_Nu2 cover only the owned planes.

   nim_slab_layout: out4 = {first plane held, one past the last held, first
   plane owned, one past the last owned}, global plane numbers.
   NIM_ERR_BAD_ARG unless 1 <= nslab, 0 <= s < nslab, n_z / nslab >= 2. */
int nim_slab_layout(int32_t n_z, int32_t nslab, int32_t s, int32_t *out4);

/* The halo exchange of slab s with its neighbour below (side 0) or above
   (side 1), as element spans (offset, count) into the slab context's own
   arrays: {cells, r faces, theta faces, z faces}.  recv8: the halo planes
   the neighbour owns; send8: the owned planes the neighbour holds as its
   halo.  The z span is the two rows of axial faces beyond the cut face
   (which both slabs compute), so no span an exchange writes is read by
   it.  Every cell array carries span 0; every face array carries spans
   1..3 in both of its halves (the face arrays alternate halves each
   pass).  The send spans of slab s, side 1, and the receive spans of slab
   s+1, side 0, have the same counts, and vice versa.  NIM_ERR_BAD_ARG on
   a side without a neighbour. */
int nim_slab_halo(int32_t n_theta, int32_t n_r, int32_t n_z, int32_t nslab, int32_t s, int32_t side,
                  int64_t *recv8, int64_t *send8);

/* nim_gpu_create for slab s of nslab of the mesh described by mesh (the
   whole mesh's arrays, checked as nim_gpu_create checks them).  The
   context is a cylinder of its held planes: nim_gpu_download/upload
   address its cells and faces in the library's structured order (cell
   i + n_theta*(j + n_r*k) with k the held plane from the slab's first;
   faces in the r / theta / z blocks of that numbering).  Parallel
   schedule, formulation 2, FP64 only (NIM_ERR_BAD_ARG otherwise).  With
   nslab > 1 the context advances only with its neighbours (nim_slab_step,
   or the nim_slab_part pieces): nim_gpu_iterate, nim_gpu_integrate,
   nim_gpu_step and nim_batch_step refuse it with NIM_ERR_BAD_ARG. */
int nim_gpu_create_slab(const nim_mesh_desc *mesh, const nim_params *params, int32_t nslab, int32_t s,
                        nim_ctx **ctx);

/* nim_gpu_step for the nslab = n slab contexts ctx[0..n) of one mesh on
   one device (ctx[s] created as slab s of n, each initialised).  Each pass
   runs its velocity, pressure and temperature parts on every slab, each
   part followed by the halo exchange of the fields it changed
   (device-to-device copies), then merges the maxima so every slab takes
   the same convergence decision.  The fields of the owned planes are
   bit-identical to a whole-mesh context's, with the same iteration counts;
   dilatation and the Nusselt numbers are the group's sums (the summation
   order differs).  per (may be NULL) receives nsteps group records. */
int nim_slab_step(int32_t n, nim_ctx *const *ctx, int32_t nsteps, nim_step_stats *per, int32_t *done);

/* ---- the pieces of nim_slab_step for a host that moves the halos itself
   (one process per GPU, each with one slab context).  Per step:
   nim_gpu_begin_step; per pass: part 0, exchange of set 1, part 1,
   exchange of set 2, part 2, exchange of set 4, max-reduction of the 24
   words at nim_slab_maxima over all slabs, part 3; every few passes
   nim_slab_loop_state until done; then nim_slab_after_loop (reduce: sum,
   max, max) and, unless the step stops there, nim_slab_end_step (reduce:
   sums).  Before the first step, and after any upload, exchange set 8.
   Everything is queued on the context's stream (nim_gpu_stream); the
   host's transport must be ordered on it too.

   nim_slab_part: part 0 velocity (update_velocity_sources +
   integrate_velocity_field), 1 pressure, 2 temperature, 3 the pass end
   (find_error's test on the merged maxima). */
int nim_slab_part(nim_ctx *ctx, int32_t part);

/* Device arrays an exchange of set (bits: 1 velocity, 2 pressure, 4
   temperature, 8 the whole state) carries, in a fixed order: ptr[i] and
   face[i] (0: a cell array of the context's cells, exchanged over span 0 of
   nim_slab_halo; 1: a face array of 2 x faces doubles, spans 1..3 in each
   half).  Returns the count (at most 32), or NIM_ERR_BAD_ARG when cap is
   too small. */
int nim_slab_arrays(nim_ctx *ctx, int32_t set, void **ptr, int32_t *face, int32_t cap);

/* One message per neighbour instead of one per span: nim_slab_pack gathers
   the send spans of side `side` of every array of the set into the device
   buffer buf (nim_slab_pack_doubles doubles, in nim_slab_arrays order, a
   face array's first half then its second), nim_slab_unpack scatters a
   neighbour's packed payload into the receive spans.  The send payload of
   slab s, side 1, and the receive payload of slab s+1, side 0, have the
   same length and order, and vice versa.  Both are queued on the
   context's stream. */
int64_t nim_slab_pack_doubles(nim_ctx *ctx, int32_t set, int32_t side);
int nim_slab_pack(nim_ctx *ctx, int32_t set, int32_t side, void *buf);
int nim_slab_unpack(nim_ctx *ctx, int32_t set, int32_t side, const void *buf);

/* Device address of the 24 uint64 words (bit patterns of non-negative
   doubles) every slab must replace by their maximum over all slabs before
   part 3: find_error's accumulators and the Dirichlet wall floor. */
int nim_slab_maxima(nim_ctx *ctx, void **slots24);

/* After the context's stream drains: state3 = {done, passes this step,
   status}; err5 (may be NULL) = the last pass's maxima of u, v, w, p, T. */
int nim_slab_loop_state(nim_ctx *ctx, int32_t *state3, double *err5);

/* check_steady_state + evaluate_D over the owned planes: out3 = {sum of
   squared dilatation, max dudt, max dTdt}. */
int nim_slab_after_loop(nim_ctx *ctx, double *out3);

/* update_time_step + find_Nu2 over the owned planes: out4 = {outer wall
   sum of area x dT/dn, outer area, inner sum, inner area}; advances the
   step counter and time. */
int nim_slab_end_step(nim_ctx *ctx, double *out4);

/* Copy a field to/from host memory in the reference layout (for
   write_data / write_restart / read_restart, postprocess.f90, restart.f90).
   n = number of doubles the host buffer holds. */
int nim_gpu_download(nim_ctx *ctx, nim_field field, double *host, int64_t n);
int nim_gpu_upload(nim_ctx *ctx, nim_field field, const double *host, int64_t n);

/* Output sets packed on the device, copied to the host while the time loop
   goes on.  They replace the host-side array walks of write_data and
   write_restart; the files themselves (Silo, Fortran unformatted) stay with
   the host.
   NIM_OUTPUT_PLOT    write_data's zone variables (postprocess.f90:92-103):
                      REAL(.,4) of meshes_uxyzt, meshes_vxyzt, meshes_wxyzt,
                      meshes_p, meshes_Txyzt, meshes_dila, 6 x NMESH floats.
   NIM_OUTPUT_RESTART write_restart's arrays after TI and STEP
                      (restart.f90:24-37): faces_u, faces_v, faces_w,
                      faces_p, faces_T (5 x NFACE), meshes_uxyz, vxyz, wxyz,
                      Txyz, meshes_uxyz_old .. Txyz_old, meshes_dila_old
                      (9 x NMESH), doubles.
   nim_gpu_output_begin packs the set as it stands after the work already
   queued and starts the copy into host (bytes >= nim_gpu_output_bytes; use
   page-locked memory for the copy to overlap) on a copy stream of its own;
   later calls may advance the state at once.  The packed snapshot is not
   touched by them.  *ticket names the copy for nim_gpu_output_wait, which
   returns once host holds it.  Beginning a set again while its previous
   copy is still running orders the new packing after that copy. */
typedef enum nim_output_set { NIM_OUTPUT_PLOT = 0, NIM_OUTPUT_RESTART = 1 } nim_output_set;
int64_t nim_gpu_output_bytes(nim_ctx *ctx, int32_t set);
int nim_gpu_output_begin(nim_ctx *ctx, int32_t set, void *host, int64_t bytes, int32_t *ticket);
int nim_gpu_output_wait(nim_ctx *ctx, int32_t ticket);

/* Diagnostics and timing hooks (no counterpart in the reference).
   nim_gpu_stream: the cudaStream_t every call of the context queues work on,
   so a caller can record CUDA events on it.
   nim_gpu_launch_count: kernels launched by the context since creation.
   nim_gpu_profile_iterations: n + 1 inner passes of the context's schedule
   and formulation (with NIM_PRECISION_MIXED: FP32 passes over the narrowed
   iterate, leaving the FP64 fields as they were), queued back to back with
   a CUDA event after each kernel; ms[k] receives the mean time of launch
   group k over the last n passes (its name from nim_gpu_profile_name), at
   most cap of them; returns their number. */
void *nim_gpu_stream(nim_ctx *ctx);
int64_t nim_gpu_launch_count(nim_ctx *ctx);
int nim_gpu_profile_iterations(nim_ctx *ctx, int32_t n, double *ms, int32_t cap);
const char *nim_gpu_profile_name(nim_ctx *ctx, int32_t k);

/* ---------------------------------------------------- tangent-linear steps
   Forward-mode derivatives of the time advance (no counterpart in the
   reference): a dual copy of the iterate (value and derivative along one
   seeded direction) advanced by the dual instantiations of the step's
   kernels, the derivative of the hot- and cold-wall Nusselt numbers
   (find_Nu2, nse.f90:2794) with respect to Ra, Pr (through nu = sqrt(Pr/Ra),
   alpha = nu/Pr, parameters.f90:169-173) and the Dirichlet wall
   temperatures.  The FP64 tangent-linear gradient the adjoint is checked
   against; the values are the FP64 parallel path's bit for bit.
   Parallel schedule and formulation 2 only; the FP64 state of the context
   is left as it was (the dual state is a copy). */
/* Copies the context's current FP64 state (after nim_gpu_init or between
   steps) into the dual state with zero derivatives and zero seeds.  The
   first call allocates it (~3.4 kB per cell). */
int nim_gpu_tangent_begin(nim_ctx *ctx);
/* Seeds d nu and d alpha (1/Re follows).  d/dRa: (-nu/(2 Ra), -alpha/(2 Ra));
   d/dPr: (nu/(2 Pr), -alpha/(2 Pr)). */
int nim_gpu_tangent_seed(nim_ctx *ctx, double dnu, double dalpha);
/* Seeds the derivatives of a state field (faces u, v, w, p, T; cells u, v, w,
   T, their old and time-averaged values, meshes_p, meshes_dila), n values
   in the layout of nim_gpu_download; e.g. the outer-wall faces of faces_T
   for the Dirichlet wall temperatures. */
int nim_gpu_tangent_seed_field(nim_ctx *ctx, nim_field field, const double *tangent, int64_t n);
/* nsteps steps of the dual state (nim_gpu_step's work: begin_step, the inner
   loop to the reference's test, update_time_step, find_Nu2); per_step the
   values' statistics, dnu[2k], dnu[2k+1] = d Nu_inner, d Nu_outer of step k.
   Either output may be NULL. */
int nim_gpu_tangent_step(nim_ctx *ctx, int32_t nsteps, nim_step_stats *per_step, double *dnu);
/* Value and derivative of a state field of the dual state (fields as
   nim_gpu_tangent_seed_field). */
int nim_gpu_tangent_get(nim_ctx *ctx, nim_field field, double *value, double *tangent, int64_t n);

/* Self-test of the bounded device waits (no counterpart in the reference):
   runs the wait that the TMA-staged sweeps use on an mbarrier that no copy
   will complete, at most `tries` (1..2^20) times, and returns the status the
   device recorded (NIM_ERR_TIMEOUT when the bound works), then clears it;
   the context stays usable.  Between steps only. */
int nim_gpu_selftest_wait_timeout(nim_ctx *ctx, int32_t tries);

/* Self-test of the device exp (no counterpart in the reference): y[i] =
   the exp that the NIM coefficients use on the device, for n host values x
   (n <= 2^28; the call allocates and frees its device buffers and runs on
   the current device's default stream).  That exp restates glibc's
   algorithm and must equal the host libm's exp bit for bit (the reference's
   exponential NIM coefficients, nim.f90:190-194, call it). */
int nim_gpu_selftest_exp(const double *x, double *y, int64_t n);

/* Self-test of the temperature's NIM coefficients of one direction
   (nim.f90:334-464, with gminus = gplus = 1): A[6i + q] = coefficient q+1
   for the contravariant velocity u[i] and diffusion coefficient k[i] > 0,
   n <= 2^26.  precision NIM_PRECISION_FP64: the FP64 path's form (series
   below |2u/k| = v_limit, exponential above, as the reference);
   NIM_PRECISION_MIXED: the float form of the FP32 phase (no counterpart in
   the reference), which must stay within a few 1e-7 of the FP64 values
   relative.  Allocates and frees its device buffers; default stream. */
int nim_gpu_selftest_nim_coef(const double *u, const double *k, int64_t n, int32_t precision, double v_limit,
                              double *A);

/* Wall-face limit of nim_gpu_nusselt_noalloc: 2*n_theta*n_z inner plus
   outer wall faces, i.e. 4096 blocks of 256 faces. */
#define NIM_NOALLOC_MAX_WALL_FACES 1048576

/* find_Nu2 without any device allocation.  No counterpart in the reference:
   it serves hosts that cannot call cudaMalloc when they want the Nusselt
   numbers, for instance because another allocator already holds all free
   device memory or because the host forbids allocation once its time loop
   has started.  It computes, from the context's current face temperatures,
   out4[0..3] = Nu_outer, Nu_inner, outer wall area, inner wall area (the
   values nim_gpu_end_step reports) into caller-owned host memory.  Its
   scratch is one static device array of 4*4096+8 doubles per device, whose
   address is looked up with the context's device current, first by
   nim_gpu_create and again on every call (a lookup, not an allocation, so
   a device reset cannot leave a stale address behind); the first
   nim_gpu_create on a device should therefore come before any stream
   capture.  Every call reuses the array and leaves the last call's partial
   sums there, so calls that overlap on the GPU (two contexts on one device
   at once) race: the host must serialise them per device.  Between steps
   only (NIM_ERR_STATE after nim_gpu_begin_step until nim_gpu_end_step).
   Meshes with more than NIM_NOALLOC_MAX_WALL_FACES wall faces are refused
   with NIM_ERR_BAD_ARG.
   On a z-slab context the sums cover the slab's owned planes only (the
   areas let a host combine slabs: Nu = sum of Nu_k * area_k / sum of
   area_k per wall).  Synchronises the context's stream. */
int nim_gpu_nusselt_noalloc(nim_ctx *ctx, double *out4);

/* Block until all work queued on the context's stream has finished. */
int nim_gpu_synchronize(nim_ctx *ctx);

void nim_gpu_destroy(nim_ctx *ctx);
const char *nim_gpu_strerror(int status);

#ifdef __cplusplus
}
#endif
#endif /* NIM_GPU_H */

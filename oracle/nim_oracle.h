/*
 * nim_oracle.h -- CPU oracle for the NIM time advance (TEST INFRASTRUCTURE).
 *
 * A plain C++ restatement of the reference's live FP64 path (nse.f90,
 * nim.f90, bc.f90, geometry.f90, curvilinear.f90, general.f90), used only by
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the
 * checker.  Nothing in the product library calls it.
 *
 * Parity is unpinned: the reference ships no test, fixture or golden output
 * and is Fortran, which this image cannot compile (no gfortran), so the
 * oracle is pinned only by its own invariants (tests/test_oracle.py) and by
 * the reference's structure it follows line by line.
 *
 * Two iteration schedules:
 *   NIM_SCHED_SEQUENTIAL -- the reference's own order: one thread, cells in
 *     number order, Gauss-Seidel inside every sweep (run.sh:2 pins
 *     OMP_NUM_THREADS=1).  "faithful" mode.
 *   NIM_SCHED_PARALLEL   -- the order the CUDA library uses: every sweep
 *     reads the values from before the sweep (double-buffered faces).  Same
 *     discrete fixed point, different path; used to check kernels step by
 *     step.
 *   NIM_SCHED_LEVELS     -- SEQUENTIAL's arithmetic with cells visited by
 *     the level i + 2j + 3k and wall faces by their in-wall level, the order
 *     of the library's reference-order sweeps.  Equal to SEQUENTIAL bit for
 *     bit when that order respects every dependence of the sweeps.
 */
#ifndef NIM_ORACLE_H
#define NIM_ORACLE_H
#include <stdint.h>
#include "nim_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

enum { NIM_SCHED_SEQUENTIAL = 0, NIM_SCHED_PARALLEL = 1, NIM_SCHED_LEVELS = 2 };

typedef struct nim_oracle nim_oracle;

int nim_oracle_create(const nim_mesh_desc *mesh, const nim_params *params,
                      int32_t schedule, int32_t threads, nim_oracle **out);
int nim_oracle_init(nim_oracle *o);
int nim_oracle_begin_step(nim_oracle *o);
int nim_oracle_integrate(nim_oracle *o, nim_step_stats *stats);
/* exactly n inner iterations, no convergence test; errors of the last one */
int nim_oracle_iterate(nim_oracle *o, int32_t n, nim_step_stats *stats);
int nim_oracle_end_step(nim_oracle *o, nim_step_stats *stats);
int nim_oracle_step(nim_oracle *o, int32_t nsteps, nim_step_stats *per_step,
                    int32_t *done);
int nim_oracle_get(nim_oracle *o, int32_t field, double *out, int64_t n);
int nim_oracle_set(nim_oracle *o, int32_t field, const double *in, int64_t n);
/* max |R_C| seen by calculate_R_c_new in SEQUENTIAL mode (must be 0) */
double nim_oracle_max_rc(nim_oracle *o);
void nim_oracle_destroy(nim_oracle *o);
void nim_oracle_set_threads(nim_oracle *o, int32_t threads);
/* M_A(d,1:6) of one direction: contravariant speed u, diffusivity k, face
   metrics g_minus/g_plus, branch switch v_limit (nim.f90:181-287) */
void nim_oracle_nim_coefficients(double u, double k, double gminus, double gplus, double v_limit,
                                 double *A);
/* formulation 1: B, C, E, F, G, H, I, J_nim of one direction (nim.f90:758-875)
   for speed u, diffusivity F and Det = D */
void nim_oracle_nim1_coefficients(double u, double F, double D, double v_limit, double *out);

/* Tangent-linear build (libnim_oracle_tl.so, oracle/nim_oracle_tl.cpp): the
   same source with dual-number values.  It exports nim_oracle_tl_<name>
   for every nim_oracle_<name> above (arguments alike, on a nim_oracle_tl
   handle; the values are the FP64 oracle's bit for bit) and the calls
   below, which seed and read the derivatives along one direction of
   (nu, alpha) and the state fields.  The FP64 tangent-linear reference
   gradient of the Nusselt numbers with respect to Ra, Pr (through nu =
   sqrt(Pr/Ra), alpha = nu/Pr) and the Dirichlet wall temperatures. */
typedef struct nim_oracle_tl nim_oracle_tl;
int nim_oracle_tl_seed_params(nim_oracle_tl *o, double dnu, double dalpha);
int nim_oracle_tl_get_tangent(nim_oracle_tl *o, int32_t field, double *out, int64_t n);
int nim_oracle_tl_set_tangent(nim_oracle_tl *o, int32_t field, const double *in, int64_t n);
/* d Nu_inner, d Nu_outer of the last end_step */
int nim_oracle_tl_nu_tangent(nim_oracle_tl *o, double *out2);

/* The oracle's own cylinder mesh (create_hollow + deform_nodes + the
   renumbering of fill_global_geometry, followed loop by loop): fills
   arrays sized as nim_mesh_sizes() gives, like nim_mesh_build(), without
   the library's mesh builder.  0 or -1. */
struct nim_mesh_params;
int nim_oracle_mesh_build(const struct nim_mesh_params *p, double *node_xyz, int32_t *meshes_nodes,
                          int32_t *meshes_faces, int32_t *meshes_neighbors, int32_t *faces_bc,
                          int32_t *bcs_faces, int32_t *bcs_faces_id, int32_t *bcs_faces_position,
                          int32_t *bcs_faces_mesh_num);

#ifdef __cplusplus
}
#endif
#endif

/*
 * nim_mesh.h -- host-side mesh builder for the cylinder-with-hexagon case.
 *
 * This is the host part that stays outside the device library: it produces
 * exactly the arrays the reference's Fortran host hands to the solver
 * (create_hollow, create_geometry.f90:321-622; deform_nodes,
 * general.f90:428-460; the cell orientation of link_mesh,
 * prepare_mesh.f90:47-132; fill_global_arrays, geometry.f90:978-1032).
 * The output fills a nim_mesh_desc (nim_gpu.h) whose arrays the caller
 * owns.  Pure C/C++ (no CUDA).
 */
#ifndef NIM_MESH_H
#define NIM_MESH_H

#include <stdint.h>
#include "nim_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

enum {
  NIM_CLUSTER_NONE = 0,
  NIM_CLUSTER_POWER = 1,  /* refine_walls_radial_order, general.f90:463-484 */
  NIM_CLUSTER_TANH = 2    /* two-sided tanh stretching (extension)          */
};

typedef struct nim_mesh_params {
  int32_t n_theta, n_r, n_z;  /* NMESH_i, NMESH_j, NMESH_k                   */
  double R_i, R_o, L;         /* annulus radii and height (parameters.f90:90-92) */
  int32_t cluster;            /* NIM_CLUSTER_*                                */
  double cluster_factor;      /* b1 = 1.5 (power) or beta (tanh)              */
  int32_t hexagon;            /* 1: map the inner ring to a hexagon           */
  double blend_r1, blend_r2;  /* create_hexagon_..._three_regions(1.25,1.75,.) */
  double blend_n;             /* exponent of the blend (-1 in the reference)  */
} nim_mesh_params;

/* Reference geometry: NMESH_j=6, NMESH_i=36, NMESH_k=12, R_i=MATH_PI/3,
   R_o=2, L=2, power clustering 1.5, hexagon blend (1.25,1.75,-1). */
void nim_mesh_params_reference(nim_mesh_params *p);

/* Sizes of the arrays nim_mesh_build fills. */
int nim_mesh_sizes(const nim_mesh_params *p, int32_t *nnode, int32_t *nmesh,
                   int32_t *nface, int32_t *nbcface);

/* Fill caller-owned arrays (sizes from nim_mesh_sizes):
   node_xyz[3*nnode], meshes_nodes[8*nmesh], meshes_faces[6*nmesh],
   meshes_neighbors[6*nmesh], faces_bc[nface], bcs_faces[nbcface],
   bcs_faces_id[nbcface], bcs_faces_position[nbcface],
   bcs_faces_mesh_num[nbcface].  Returns 0 or NIM_ERR_BAD_ARG. */
int nim_mesh_build(const nim_mesh_params *p, double *node_xyz,
                   int32_t *meshes_nodes, int32_t *meshes_faces,
                   int32_t *meshes_neighbors, int32_t *faces_bc,
                   int32_t *bcs_faces, int32_t *bcs_faces_id,
                   int32_t *bcs_faces_position, int32_t *bcs_faces_mesh_num);

#ifdef __cplusplus
}
#endif
#endif /* NIM_MESH_H */

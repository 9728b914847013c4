/*
 * cfsa_mesh.h — C ABI of the host mesh layer (P1/P2 tetrahedral mesh + fluid boundary tags).
 *
 * Plain C types only. Each entry point replaces a member of the reference's Mesh class
 * (include/Mesh/Mesh.hpp, src/Mesh/Mesh.cpp of sudo-shaka/Cell-Fluid-Structure-Analysis),
 * cited per function. All functions return CFSA_OK (0) or an error code from cfsa_ns.h; the
 * message of the last failure on the calling thread is returned by cfsa_mesh_last_error().
 * Numbering rules are the reference's: faces in sorted-vertex-triple order, P2 edge nodes in
 * first-encounter order over (tet, local edge 0-1,0-2,0-3,1-2,1-3,2-3), P2 global index = nv+id.
 */
#ifndef CFSA_MESH_H
#define CFSA_MESH_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cfsa_mesh cfsa_mesh;

/* Mesh::fromMshFile (include/Mesh/Mesh.hpp:82-86; reader src/Mesh/Mesh.cpp:16-144). */
int cfsa_mesh_from_msh(const char *path, cfsa_mesh **out);

/* Build from raw arrays: xyz[nv][3], tets[nt][4] (0-based). Runs the same post-load pipeline
 * as the MSH reader (src/Mesh/Mesh.cpp:130-143). */
int cfsa_mesh_from_arrays(int64_t nv, const double *xyz, int64_t nt, const int32_t *tets,
                          cfsa_mesh **out);

/* Mesh::structuredRectangularPrism (include/Mesh/Mesh.hpp:87-93; src/Mesh/Mesh.cpp:146-225). */
int cfsa_mesh_structured_prism(double length, double width, double height, int nx, int ny, int nz,
                               cfsa_mesh **out);

/* Procedural cylinder along +x (length, radius, disk rings, axial layers). Replaces
 * Mesh::fromPolyhedron(Polyhedron::cylendar(...)) (src/Mesh/Mesh.cpp:227-323), whose TetGen
 * dependency is not available; see Mesh::generateCylinder for the construction. */
int cfsa_mesh_cylinder(double length, double radius, int rings, int layers, cfsa_mesh **out);
/* Procedural Y-bifurcation with generator-assigned fluid tags (inlet cap at x = 0, both daughter
 * caps outlet, wall elsewhere; P2 tags derived as in Mesh.hpp:198-215). spec[7] = parent radius,
 * parent length, daughter radius, daughter length, daughter angle (degrees, +-, x-y plane),
 * blend radius of the smooth junction, lattice cell edge. Replaces the TetGen meshing of a
 * bifurcation surface for synthetic inputs. */
int cfsa_mesh_y_bifurcation(const double spec[7], cfsa_mesh **out);

/* Mesh::setupBoundaryConditions (src/Mesh/Mesh.cpp:325-417), which ends with
 * setP2BoundariesFromP1Boundaries (include/Mesh/Mesh.hpp:198-215). dir[3] = inlet->outlet. */
int cfsa_mesh_setup_boundary_conditions(cfsa_mesh *m, const double dir[3], double coverage);

/* Overwrite P1 / P2 fluid tags (FluidBCType values) — Mesh::setFluidVertexBC /
 * setFluidP2vertexBC (include/Mesh/Mesh.hpp:180-190). Either pointer may be NULL. */
int cfsa_mesh_set_fluid_bc(cfsa_mesh *m, const int8_t *p1_bc, const int8_t *p2_bc);

/* Write the P1 mesh as Gmsh MSH 4.1. */
int cfsa_mesh_write_msh(const cfsa_mesh *m, const char *path);

/* sizes[0..4] = nv, nt, ne (P2 edge nodes), nfaces, n boundary faces. */
int cfsa_mesh_sizes(const cfsa_mesh *m, int64_t sizes[5]);

/* Array getters (caller-allocated outputs, sizes from cfsa_mesh_sizes). */
int cfsa_mesh_get_vertices(const cfsa_mesh *m, double *xyz /*[nv][3]*/);
int cfsa_mesh_get_tets(const cfsa_mesh *m, int32_t *tets /*[nt][4]*/);
int cfsa_mesh_get_tet_edges(const cfsa_mesh *m, int32_t *edges /*[nt][6]*/);
int cfsa_mesh_get_edge_nodes(const cfsa_mesh *m, double *xyz /*[ne][3]*/);
int cfsa_mesh_get_fluid_bc(const cfsa_mesh *m, int8_t *p1_bc /*[nv]*/, int8_t *p2_bc /*[ne]*/);
/* faces: vertids[nf][3], tets[nf][2] (tet_a, tet_b or -1), geom[nf][7] (normal, area, center). */
int cfsa_mesh_get_faces(const cfsa_mesh *m, int32_t *vertids, int32_t *tets, double *geom);
/* volumes[nt], grads[nt][4][3] (Mesh::getTetGradients, src/Mesh/Mesh.cpp:590-614). */
int cfsa_mesh_get_tet_geometry(const cfsa_mesh *m, double *volumes, double *grads);

void cfsa_mesh_destroy(cfsa_mesh *m);
const char *cfsa_mesh_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* CFSA_MESH_H */

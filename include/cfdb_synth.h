/*
 * cfdb synthetic workloads: box and jittered-tet meshes in the reference's mesh contract
 * (Yipexnn/CFD src/mesh: internal faces sorted by (owner, neighbour) with owner < neighbour,
 * boundary faces by (patch, owner); geometry of mesh.cpp:100-186; FV factors of
 * fv_geometry.cpp:17-69) and the pressure-system inputs derived from them. These produce the
 * inputs of the hot path (face addressing, delta coefficients, face gamma, flux, source); they
 * are not themselves on it.
 */
#ifndef CFDB_SYNTH_H
#define CFDB_SYNTH_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cfdb_mesh cfdb_mesh;

/* Hex box on the given node coordinates (xs: nx+1, ys: ny+1, zs: nz+1 values), cells ordered
 * k outermost, i innermost (box_mesher.cpp:74-92), six wall patches xmin..zmax. */
int cfdb_mesh_box(int nx, int ny, int nz, const double* xs, const double* ys, const double* zs,
                  cfdb_mesh** out);
/* Same lattice, each box cell split into 6 tets sharing its main diagonal; interior node
 * coordinates jittered by U(-jitter*h, +jitter*h) (h: local node spacing) from seed; nodes on
 * a wall keep their wall coordinate. */
int cfdb_mesh_tet(int nx, int ny, int nz, const double* xs, const double* ys, const double* zs,
                  double jitter, uint64_t seed, cfdb_mesh** out);
int cfdb_mesh_destroy(cfdb_mesh* m);
int cfdb_mesh_sizes(const cfdb_mesh* m, int* n_cells, int* n_faces, int* n_internal_faces,
                    int* n_points);
/* Borrowed pointers valid while m lives. owner: n_faces; neighbour: n_internal_faces;
 * vectors are xyz-interleaved. */
int cfdb_mesh_addressing(const cfdb_mesh* m, const int** owner, const int** neighbour);
int cfdb_mesh_geometry(const cfdb_mesh* m, const double** points, const double** face_centres,
                       const double** face_areas, const double** cell_centres,
                       const double** cell_volumes);
/* Face -> node lists (CSR: offsets n_faces+1, nodes). */
int cfdb_mesh_faces(const cfdb_mesh* m, const int** offsets, const int** nodes);
/* Over-relaxed delta coefficients and interpolation weights of the internal faces. */
int cfdb_mesh_fv(const cfdb_mesh* m, const double** delta, const double** weights);

/* Pressure-system inputs on a mesh (flow_solver.cpp:688-783 semantics):
 *   rAU_c = V_c * X_c, X_c ~ LogNormal(0, sigma) (sigma = 0: X_c = 1, rAU_c = 1 when
 *   unit_rau != 0), gamma_f = w rAU_P + (1 - w) rAU_N;
 *   flux_kind 0: flux_f = u_f . S_f with u_f ~ U(-1,1)^3 per face; 1: flux = 0.
 *   source: rhs_kind 0 = zero; 1 = N(0,1) per cell shifted to zero mean.
 * Outputs: gamma, flux (n_internal_faces), source (n_cells). */
int cfdb_synth_pressure_inputs(const cfdb_mesh* m, double sigma, int unit_rau, int flux_kind,
                               int rhs_kind, uint64_t seed, double* gamma, double* flux,
                               double* source);

/* Node coordinates in [0,1]: uniform, one-sided geometric grading (box_mesher.cpp:36-46) or
 * two-sided grading with ratio r between neighbouring cells, smallest at both ends. */
int cfdb_positions_graded(int n, double grading, double* out);
int cfdb_positions_two_sided(int n, double ratio, double* out);

#ifdef __cplusplus
}
#endif
#endif

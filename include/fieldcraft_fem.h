/* fieldcraft_fem.h — the input side of the Cholesky path: structured hex8 models, their
 * fill-reducing node order and the free-DOF stiffness K_ff in compressed rows.
 *
 * These entry points restate, for structured boxes of trilinear hexahedra, what the reference
 * does before it calls its factorisation:
 *   - nodes and elements in label order (crates/solver/src/system.rs:697-702,
 *     crates/solver/tests/common/mod.rs:23-98);
 *   - the node graph (crates/solver/src/sparse.rs:99-126, NodeGraph::new);
 *   - the fill-reducing order (crates/solver/src/ordering.rs:28-281: nested_dissection,
 *     fill_reducing_order, graph_dissection, fill);
 *   - equation numbering of the free DOFs in node order (crates/solver/src/constraints.rs:755-767);
 *   - the hex8 stiffness with 2x2x2 Gauss points (crates/fem/src/element.rs:396-425, 745-774,
 *     shape.rs:95-103, quadrature.rs:28-44, 78-90, material.rs:40-53);
 *   - assembly in element label order (crates/solver/src/analysis.rs:199-234, sparse.rs:209-226)
 *     and the plain-selection reduction to K_ff (constraints.rs:820-905).
 * Index types: row pointers int64, column indices int32, values double. Every function returns
 * 0 on success and a negative FC_FEM_* code on failure; nothing throws across this boundary.
 */
#ifndef FIELDCRAFT_FEM_H
#define FIELDCRAFT_FEM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FC_FEM_OK 0
#define FC_FEM_INVALID (-1)   /* bad sizes, a degenerate element, a non-positive modulus */
#define FC_FEM_NOMEM (-2)

typedef struct fc_problem fc_problem;

/* A box of nx*ny*nz hex8 elements of size lx*ly*lz. young[e] is element e's modulus, elements
 * numbered e = i + nx*(j + ny*k); poisson is shared. clamped[v] != 0 holds every DOF of node v,
 * nodes numbered v = i + (nx+1)*(j + (ny+1)*k). threads <= 0 uses the hardware's count; the
 * result does not depend on it. */
int fc_fem_box(int nx, int ny, int nz, double lx, double ly, double lz, const double *young,
               double poisson, const unsigned char *clamped, int threads, fc_problem **out);
void fc_fem_free(fc_problem *p);
int64_t fc_fem_n(const fc_problem *p);        /* free equations */
int64_t fc_fem_nnz(const fc_problem *p);      /* entries of K_ff, both triangles */
int64_t fc_fem_nodes(const fc_problem *p);
/* K_ff by rows (both triangles, sorted columns): ptr[n+1], idx[nnz], val[nnz]. */
int fc_fem_csr(const fc_problem *p, int64_t *ptr, int32_t *idx, double *val);
/* order[k]: the node eliminated k-th (nodes). eq[3*v + a]: equation of DOF a of node v, or -1. */
int fc_fem_order(const fc_problem *p, int64_t *order);
int fc_fem_equations(const fc_problem *p, int64_t *eq);

/* The orderings on their own, on a node graph given by rows (sorted, each row holding its own
 * node): adj_ptr[n+1], adj_idx. xyz[3*n]. order[n] receives the permutation. */
int fc_nested_dissection(int64_t n, const double *xyz, const int64_t *adj_ptr, const int32_t *adj_idx,
                         int64_t *order);
int fc_graph_dissection(int64_t n, const int64_t *adj_ptr, const int32_t *adj_idx, int64_t *order);
int fc_fill_reducing_order(int64_t n, const double *xyz, const int64_t *adj_ptr, const int32_t *adj_idx,
                           int64_t *order);
/* Entries of the Cholesky factor of the node graph eliminated in `order` (-1 on bad input). */
int64_t fc_fill(int64_t n, const int64_t *adj_ptr, const int32_t *adj_idx, const int64_t *order);

/* The 24x24 stiffness of one hex8 element (corner order of crates/fem/src/shape.rs:51-52),
 * DOFs node by node (x, y, z), row-major into out[576]. */
int fc_hex8_stiffness(const double *xyz24, double young, double poisson, double *out576);

/* K_ff assembled on a GPU (no reference counterpart: the reference assembles on the host,
 * analysis.rs:199-234): every element's matrix, then every entry as the sum over the elements
 * holding both its nodes in element label order; the builder's operations in its order, so the
 * values are fc_fem_box's bits. A context holds the box (nx, ny, nz elements of lx, ly, lz), its
 * pattern (ptr[n+1], idx, as fc_fem_csr gives them), its equations (eq[3 nodes], as
 * fc_fem_equations gives them) and 576 doubles per element of device scratch. Assembly takes the
 * moduli d_young[nx ny nz] in device memory and writes d_val[ptr[n]] in the pattern's order on
 * `stream` (a cudaStream_t), waiting for it; FC_FEM_INVALID for a bad modulus or element. */
typedef struct fc_fem_device fc_fem_device;
int fc_fem_device_create(int nx, int ny, int nz, double lx, double ly, double lz, int64_t n, const int64_t *ptr,
                         const int32_t *idx, const int64_t *eq, int device, fc_fem_device **out);
int fc_fem_assemble_device(fc_fem_device *d, const double *d_young, double poisson, double *d_val, void *stream);
/* After fc_fem_assemble_device, from the free equations' solution d_q[n] (device): the motion of
 * every DOF d_u[3 nodes] (zero where held; Reduction::expand, constraints.rs:929-939) and the
 * reactions d_r[3 nodes] at the held DOFs, K u - f over each whole row in column order (zero at
 * free DOFs; Reduction::reactions, constraints.rs:1001-1015), with the loads d_f[3 nodes] (NULL:
 * none). Either output may be NULL. Waits for `stream`. */
int fc_fem_reactions_device(fc_fem_device *d, const double *d_q, const double *d_f, double *d_r, double *d_u,
                            void *stream);
/* Stress recovery (analysis.rs:478-540, element.rs:587-670, 775-860, material.rs:88-93) from the
 * motion of every DOF d_u[3 nodes]: per element the stresses at its 2 x 2 x 2 Gauss points
 * d_points[elements * 48] (xi fastest; xx yy zz xy xz yz), extrapolated to its corners; per node
 * the mean over the elements holding it d_nodal[nodes * 6] and its von Mises stress
 * d_von_mises[nodes]. Any output may be NULL. Waits for `stream`. */
int fc_fem_stresses_device(fc_fem_device *d, const double *d_young, double poisson, const double *d_u,
                           double *d_points, double *d_nodal, double *d_von_mises, void *stream);
void fc_fem_device_free(fc_fem_device *d);

#ifdef __cplusplus
}
#endif
#endif

/*
 * Plain-C interface shared by the two CPU oracles of the critical-point path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, the smoke check and the CPU-baseline
 * leg of bench.py may load the libraries built from oracle/; the product never
 * links them.
 *
 *   oracle/_ref/libftk2ref.so   the reference's own CPU engine
 *                               (SimplicialEngine<T, CriticalPointPredicate<M,T>>
 *                               ::execute() + get_complex(), engine.hpp:96-99 and
 *                               822-996), compiled unmodified from its headers
 *                               against the ndarray shim in oracle/shim.
 *   oracle/_build/libcporacle.so our own exact, multithreaded C restatement
 *                               of the same algorithm (cp_oracle.c), used where
 *                               the reference is too slow.
 *
 * Both fill the same orc_result, whose content mirrors the reference's
 * FeatureComplex (complex.hpp:14-58): features in Simplex::operator< order,
 * float barycentrics, track_id, type, scalar, and the sorted unique edge list.
 */
#ifndef FTK2B_ORACLE_API_H
#define FTK2B_ORACLE_API_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_MESH_REGULAR = 0, ORC_MESH_EXTRUDED = 1 };
enum { ORC_F32 = 0, ORC_F64 = 1 };
enum { ORC_LAYOUT_MULTI = 0, ORC_LAYOUT_SEPARATE = 1, ORC_LAYOUT_PER_VERTEX = 2 };

typedef struct {
  int kind;                 /* ORC_MESH_* */
  int ndims;                /* regular: dims incl. time (3 = 2D+t, 4 = 3D+t) */
  uint64_t local_dims[4];   /* RegularSimplicialMesh(dims, offset, global)   */
  uint64_t offset[4];
  uint64_t global_dims[4];
  /* extruded: UnstructuredSimplicialMesh(3, cell_dim, coords, cells) wrapped in
   * ExtrudedSimplicialMesh(base, n_layers) */
  uint64_t n_base_verts;
  const double* base_coords;   /* 3 per base vertex */
  uint64_t n_base_cells;
  const uint64_t* base_cells;  /* (base_cell_dim + 1) per cell */
  int base_cell_dim;           /* 2 = triangles, 3 = tets */
  uint64_t n_layers;
} orc_mesh;

typedef struct {
  int dtype;                /* ORC_F32 / ORC_F64 */
  int ncomp;                /* M: 2 or 3 */
  int layout;               /* ORC_LAYOUT_* */
  const void* comp[4];      /* MULTI: comp[0] = [M, dims...]; else one array per component */
  int nd;                   /* array rank, not counting MULTI's leading component dim */
  uint64_t dims[4];         /* Fortran dims (first fastest) */
  const void* scalar;       /* optional scalar field (same dtype) or NULL */
  int scalar_nd;
  uint64_t scalar_dims[4];
  double sos_q;             /* Predicate::sos_q (predicate.hpp:25) */
  int n_threads;            /* restatement only: worker threads (0 = all cores) */
  /* restatement only: FiberPredicate<T> (predicate.hpp:341-362) instead of
   * CriticalPointPredicate<2,T>: values less fiber_thr in the field precision,
   * the centroid where the solve fails */
  int fiber;
  double fiber_thr[2];
} orc_field;

typedef struct {
  int m;                    /* feature simplices have m+1 vertices */
  uint64_t n;               /* number of features */
  uint64_t* simplices;      /* n*(m+1) sorted vertex ids */
  float* bary;              /* n*(m+1) barycentrics as the reference stores them */
  double* lambda;           /* n*(m+1) solver output in the field precision, widened */
  uint64_t* track_id;       /* n */
  uint32_t* type;           /* n (always 0 in the reference) */
  float* scalar;            /* n */
  uint64_t n_edges;
  uint32_t* edges;          /* 2*n_edges, sorted, unique, (lo, hi) */
  uint64_t n_tested;        /* m-simplices evaluated (restatement only) */
  uint32_t* cp_class;       /* n classes (restatement only, regular meshes; else NULL):
                               FTK2B_CLASS_* codes of include/ftk2b.h */
  int cell_dim;             /* restatement of fiber surfaces only: the star-fan */
  uint64_t n_cells;         /* triangles of get_complex, (cell_dim + 1) sorted  */
  uint32_t* cells;          /* feature indices each, rows in lexicographic order */
} orc_result;

/* The high-level caller's critical-point flow (src/high_level/feature_tracker.cpp:
 * 339-357 with the mesh of 480-520): ExtrudedSimplicialMesh over
 * RegularSimplicialMesh(spatial dims) with nt - 1 layers, a multicomponent
 * vector array [m, dims..., nt], and AttributeSpec entries recorded into
 * FeatureElement::attributes (engine.hpp:1143-1199). */
typedef struct {
  int dtype;                   /* ORC_F32 / ORC_F64 */
  int m;                       /* 2 or 3 */
  uint64_t dims[3];            /* spatial dims */
  uint64_t nt;
  const void* vec;             /* [m, dims..., nt], Fortran order */
  int n_attr;                  /* <= 16, slots 0 .. n_attr-1 */
  const void* attr_data[16];
  int attr_nd[16];
  uint64_t attr_dims[16][6];   /* full Fortran shape of the source array */
  int attr_magnitude[16];      /* 1: type "magnitude", else "scalar" */
  int attr_component[16];      /* AttributeSpec::component (-1 = none) */
} orc_tracked;

/* reference engine build */
int ftk2ref_run(const orc_mesh* mesh, const orc_field* field, orc_result* out);
void ftk2ref_free(orc_result* r);
/* attrs receives n * 16 floats (malloc'd; release with ftk2ref_free_attrs) */
int ftk2ref_run_tracked(const orc_tracked* in, orc_result* out, float** attrs);
void ftk2ref_free_attrs(float* attrs);

/* Level sets (ContourPredicate<T>, predicate.hpp:135-183) on a regular mesh:
 * field->comp[0] is the scalar array (layout SEPARATE, ncomp 1).  Features are
 * mesh edges (m = 1); lambda holds the barycentrics the predicate used
 * (solver output, or 0.5 where it falls back), widened.  conn receives the
 * manifold cells of get_complex: triangles (dim 2) on 2D+t meshes, tets
 * (dim 3) on 3D+t meshes, as sorted rows of feature indices. */
typedef struct {
  int dim;
  uint64_t n;
  uint32_t* idx;            /* (dim+1)*n */
} orc_conn;
int ftk2ref_run_contour(const orc_mesh* mesh, const orc_field* field, double threshold, orc_result* out,
                        orc_conn* conn);
void ftk2ref_free_conn(orc_conn* c);
/* Fibers (FiberPredicate<T>, predicate.hpp:341-362) of the two scalar arrays
 * comp[0], comp[1] (layout SEPARATE) on a regular 2D+t mesh; thresholds[2].
 * Flattened as ftk2ref_run, with the star edges of the trajectories. */
int ftk2ref_run_fiber(const orc_mesh* mesh, const orc_field* field, const double* thresholds, orc_result* out);
/* Fiber surfaces: the same on a regular 3D+t mesh (ndims 4); conn receives
 * the star-fan triangles (dim 2) of get_complex. */
int ftk2ref_run_fiber_surface(const orc_mesh* mesh, const orc_field* field, const double* thresholds,
                              orc_result* out, orc_conn* conn);

/* own restatement */
int cporacle_run(const orc_mesh* mesh, const orc_field* field, orc_result* out);
void cporacle_free(orc_result* r);
/* FP64 classification of one spatial Jacobian (m x m, row = component) */
uint32_t cporacle_classify_jacobian(int m, const double* J);

#ifdef __cplusplus
}
#endif

#endif

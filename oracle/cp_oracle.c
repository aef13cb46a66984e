/*
 * Exact CPU restatement of the reference's critical-point tracking path.
 *
 * TEST INFRASTRUCTURE ONLY: this is the oracle the CUDA path is checked
 * against.  Only tests/, the smoke check and bench.py's CPU-baseline leg load
 * it (through oracle/bridge.py); nothing in the product links or calls it.
 *
 * It restates, in plain C with gcc's __int128, what
 * SimplicialEngine<T, CriticalPointPredicate<M,T>>::execute() + get_complex()
 * compute (engine.hpp:96-212, 822-996), multithreaded and without the
 * reference's global mutex.  Parity with the reference engine itself
 * (oracle/_ref) is checked by tests/test_oracle.py at small and medium sizes.
 *
 * Semantics restated (reference file:line):
 *  - quantisation q(v) = (int128)((double)v * Q + (v > 0 ? 0.5 : -0.5))      sos.hpp:15,25,75
 *  - 2D inside test: det2 signs of (v0,v1),(v1,v2),(v2,v0) equal, a zero
 *    determinant broken by vertex-id order                                    sos.hpp:22-35,222-232
 *  - 3D inside test: four det3 signs equal; det3 = sign of the 4x4
 *    [X;origin | 1] determinant, else 13 fixed sub-determinant levels, else +1 sos.hpp:72-200,234-254
 *  - accept iff inside AND the partial-pivot solve succeeds in precision T
 *    (|pivot| >= 1e-12, every lambda in [-1e-9, 1+1e-9])                     zero_crossing.hpp:20-90,
 *                                                                             predicate.hpp:66-99
 *  - regular mesh m-simplices = all m-faces of the Kuhn top cells of the local
 *    box: LUT types per hypercube (mesh.hpp:270-302) plus the upper-boundary
 *    faces that phase 2 discovers (engine.hpp:161-206, 1342-1367)
 *  - star edges per top cell from the smallest encode_simplex_id face         engine.hpp:1375-1387,
 *                                                                             mesh.hpp:736-749
 *  - canonical ids = rank in Simplex order; union-find links the larger root
 *    under the smaller; track_id = root                                       engine.hpp:46-74,838-983
 *  - extruded meshes: spatial, prism and interior m-simplices, pentatope star
 *    edges by node-id order, and the coface unions of
 *    ExtrudedSimplicialMesh::cofaces (mesh.hpp:601-712) for 4D meshes         engine.hpp:896-963
 *  - fiber mode (orc_field.fiber): FiberPredicate<T>, the values less the two
 *    thresholds in precision T, the centroid (T)1.0/3.0 where the solve
 *    fails, scalar 0                                                          predicate.hpp:341-362
 *  - fiber surfaces (fiber mode on a 3D+t mesh): triangle features over the
 *    50 triangle types of the 4-D Kuhn cube, star-fan triangles of
 *    form_general_manifold_patches with k = 2 on every pentatope, tracks as
 *    their components                                                         engine.hpp:1342-1417
 *  - fiber surfaces on extruded tet meshes: phase-1 triangles (spatial, and
 *    the Kuhn pieces over base edges) then the triangles inside the prisms
 *    over base triangles, numbered as sequential patching meets them          mesh.hpp:568-599,
 *                                                                             engine.hpp:101-212
 *
 * Compile without FMA contraction (-ffp-contract=off) so the solve rounds
 * exactly like the reference built for x86-64.
 */
#define _GNU_SOURCE
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "oracle_api.h"

typedef __int128 i128;

/* ------------------------------------------------------------------------ */
/* SoS predicates (sos.hpp)                                                   */

static inline i128 quant(double v, double Q) {
  /* sos.hpp:15: the double is truncated toward zero after adding +-0.5 */
  return (i128)(v * Q + (v > 0 ? 0.5 : -0.5));
}

static inline int sgn128(i128 x) { return x > 0 ? 1 : (x < 0 ? -1 : 0); }

/* sos.hpp:22-35 */
static int sos_det2(const double a[2], const double b[2], uint64_t ia, uint64_t ib, double Q) {
  i128 d = quant(a[0], Q) * quant(b[1], Q) - quant(a[1], Q) * quant(b[0], Q);
  if (d > 0) return 1;
  if (d < 0) return -1;
  if (ia < ib) return 1;
  if (ia > ib) return -1;
  return 0;
}

/* sos.hpp:72-200 with the fourth row being the origin (its quantised value is
 * 0), so every level collapses to a small polynomial in the three rows
 * r0, r1, r2 (the arguments in call order).  Integer arithmetic is exact (and
 * wraps identically on overflow), so any expansion of the same polynomial
 * yields the reference's value. */
static int sos_det3(const double r0d[3], const double r1d[3], const double r2d[3], double Q) {
  i128 a[3], b[3], c[3];
  for (int k = 0; k < 3; ++k) {
    a[k] = quant(r0d[k], Q);
    b[k] = quant(r1d[k], Q);
    c[k] = quant(r2d[k], Q);
  }
  i128 d;
  /* level 0: det [r0; r1; r2] */
  d = a[0] * (b[1] * c[2] - b[2] * c[1]) - a[1] * (b[0] * c[2] - b[2] * c[0]) +
      a[2] * (b[0] * c[1] - b[1] * c[0]);
  if (d) return sgn128(d);
  /* levels 1..13 */
  if ((d = b[0] * c[1] - b[1] * c[0])) return sgn128(d);           /* 1 */
  if ((d = -(b[0] * c[2] - b[2] * c[0]))) return sgn128(d);        /* 2 */
  if ((d = b[1] * c[2] - b[2] * c[1])) return sgn128(d);           /* 3 */
  if ((d = -(a[0] * c[1] - a[1] * c[0]))) return sgn128(d);        /* 4 */
  if ((d = c[0])) return sgn128(d);                                /* 5 */
  if ((d = -c[1])) return sgn128(d);                               /* 6 */
  if ((d = a[0] * c[2] - a[2] * c[0])) return sgn128(d);           /* 7 */
  if ((d = c[2])) return sgn128(d);                                /* 8 */
  if ((d = -(a[1] * c[2] - a[2] * c[1]))) return sgn128(d);        /* 9 */
  if ((d = a[0] * b[1] - a[1] * b[0])) return sgn128(d);           /* 10 */
  if ((d = -b[0])) return sgn128(d);                               /* 11 */
  if ((d = b[1])) return sgn128(d);                                /* 12 */
  if ((d = a[0])) return sgn128(d);                                /* 13 */
  return 1;                                                         /* 14 */
}

static int sos_inside(int M, double v[4][3], const uint64_t idx[4], double Q) {
  if (M == 2) {
    int s0 = sos_det2(v[0], v[1], idx[0], idx[1], Q);
    int s1 = sos_det2(v[1], v[2], idx[1], idx[2], Q);
    int s2 = sos_det2(v[2], v[0], idx[2], idx[0], Q);
    return s0 == s1 && s1 == s2;
  }
  int d0 = sos_det3(v[1], v[3], v[2], Q);
  int d1 = sos_det3(v[0], v[2], v[3], Q);
  int d2 = sos_det3(v[0], v[3], v[1], Q);
  int d3 = sos_det3(v[0], v[1], v[2], Q);
  return d0 == d1 && d1 == d2 && d2 == d3;
}

/* ------------------------------------------------------------------------ */
/* ZeroCrossingSolver<K,T>::solve (zero_crossing.hpp:20-90), in T            */

#define DEFINE_SOLVE(NAME, T, ABS)                                                   \
  static int NAME(int K, T vals[4][3], T lam[4]) {                                   \
    T A[3][3], x[3];                                                                 \
    for (int j = 0; j < K; ++j) {                                                    \
      for (int i = 0; i < K; ++i) A[j][i] = vals[i][j] - vals[K][j];                 \
      x[j] = -vals[K][j];                                                            \
    }                                                                                \
    for (int i = 0; i < K; ++i) {                                                    \
      int p = i;                                                                     \
      for (int j = i + 1; j < K; ++j)                                                \
        if (ABS(A[j][i]) > ABS(A[p][i])) p = j;                                      \
      for (int l = 0; l < K; ++l) { T t = A[i][l]; A[i][l] = A[p][l]; A[p][l] = t; } \
      { T t = x[i]; x[i] = x[p]; x[p] = t; }                                         \
      if (ABS(A[i][i]) < (T)1e-12) return 0;                                         \
      for (int j = i + 1; j < K; ++j) {                                              \
        T f = A[j][i] / A[i][i];                                                     \
        x[j] -= f * x[i];                                                            \
        for (int l = i + 1; l < K; ++l) A[j][l] -= f * A[i][l];                      \
      }                                                                              \
    }                                                                                \
    for (int i = K - 1; i >= 0; --i) {                                               \
      T s = 0;                                                                       \
      for (int j = i + 1; j < K; ++j) s += A[i][j] * x[j];                           \
      x[i] = (x[i] - s) / A[i][i];                                                   \
    }                                                                                \
    T sum = 0;                                                                       \
    for (int i = 0; i < K; ++i) { lam[i] = x[i]; sum += lam[i]; }                    \
    lam[K] = (T)1.0 - sum;                                                           \
    const T eps = (T)1e-9;                                                           \
    for (int i = 0; i <= K; ++i)                                                     \
      if (lam[i] < -eps || lam[i] > (T)1.0 + eps) return 0;                          \
    return 1;                                                                        \
  }

DEFINE_SOLVE(solve_f64, double, fabs)
DEFINE_SOLVE(solve_f32, float, fabsf)

/* ------------------------------------------------------------------------ */
/* Field access (engine.hpp:999-1009 legacy, 1101-1124 multicomponent)        */

typedef struct {
  const orc_field* f;
  int nd_mesh;            /* regular: mesh dims; extruded: 0 */
  uint64_t offset[4];     /* legacy arrays are indexed by global - offset */
} acc_t;

static inline double load_elem(const orc_field* f, const void* base, uint64_t i) {
  return f->dtype == ORC_F64 ? ((const double*)base)[i] : (double)((const float*)base)[i];
}

/* g: global grid coords (regular) ; vid: vertex id */
static double field_value(const acc_t* a, int j, const uint64_t g[4], uint64_t vid) {
  const orc_field* f = a->f;
  if (f->layout == ORC_LAYOUT_PER_VERTEX || (f->layout == ORC_LAYOUT_SEPARATE && f->nd == 1))
    return load_elem(f, f->comp[j], vid);
  if (f->layout == ORC_LAYOUT_MULTI) {
    uint64_t off = 0, mul = 1;
    for (int k = 0; k < a->nd_mesh; ++k) { off += g[k] * mul; mul *= f->dims[k]; }
    return load_elem(f, f->comp[0], (uint64_t)j + (uint64_t)f->ncomp * off);
  }
  uint64_t off = 0, mul = 1;
  for (int k = 0; k < a->nd_mesh; ++k) { off += (g[k] - a->offset[k]) * mul; mul *= f->dims[k]; }
  return load_elem(f, f->comp[j], off);
}

/* scalar interpolation happens only when the predicate sees more than M
 * arrays, i.e. legacy mode (predicate.hpp:81, engine.hpp:1125-1139); it reads
 * the scalar at global coordinates without the offset (predicate.hpp:84-89). */
static double scalar_value(const acc_t* a, const uint64_t g[4], uint64_t vid) {
  const orc_field* f = a->f;
  if (f->scalar_nd == 1) return load_elem(f, f->scalar, vid);
  uint64_t off = 0, mul = 1;
  for (int k = 0; k < a->nd_mesh; ++k) { off += g[k] * mul; mul *= f->scalar_dims[k]; }
  return load_elem(f, f->scalar, off);
}

/* ------------------------------------------------------------------------ */
/* Feature records                                                            */

typedef struct {
  uint64_t v[5];
  double lam[4];
  float scalar;
  int phase;        /* extruded: 0 = found by phase-1 iteration, 1 = interior */
} feat_t;

typedef struct {
  feat_t* a;
  size_t n, cap;
} fvec_t;

static void fvec_push(fvec_t* fv, const feat_t* x) {
  if (fv->n == fv->cap) {
    fv->cap = fv->cap ? fv->cap * 2 : 256;
    fv->a = (feat_t*)realloc(fv->a, fv->cap * sizeof(feat_t));
  }
  fv->a[fv->n++] = *x;
}

static int g_m; /* tuple length - 1 for comparators */

static int cmp_tuple(const uint64_t* a, const uint64_t* b, int m) {
  for (int i = 0; i <= m; ++i)
    if (a[i] != b[i]) return a[i] < b[i] ? -1 : 1;
  return 0;
}

static int cmp_feat(const void* x, const void* y) {
  return cmp_tuple(((const feat_t*)x)->v, ((const feat_t*)y)->v, g_m);
}

/* Evaluate one m-simplex whose sorted vertex ids are vid[] and grid coords g[][].
 * Returns 1 and fills *out if accepted. */
static int evaluate(const acc_t* a, int M, const uint64_t vid[4], uint64_t g[4][4], feat_t* out) {
  const orc_field* f = a->f;
  double vals[4][3];
  for (int i = 0; i <= M; ++i)
    for (int j = 0; j < M; ++j) vals[i][j] = field_value(a, j, g[i], vid[i]);
  if (f->fiber) /* FiberPredicate::extract_it: adj = values - thresholds in T */
    for (int i = 0; i <= M; ++i)
      for (int j = 0; j < M && j < 2; ++j)
        vals[i][j] = f->dtype == ORC_F64 ? vals[i][j] - f->fiber_thr[j]
                                         : (double)((float)vals[i][j] - (float)f->fiber_thr[j]);
  if (!sos_inside(M, vals, vid, f->sos_q)) return 0;
  int ok;
  if (f->dtype == ORC_F64) {
    double lam[4];
    ok = solve_f64(M, vals, lam);
    if (!ok && f->fiber) /* the centroid, (T)1.0 / 3.0 (predicate.hpp:354) */
      for (int i = 0; i <= M; ++i) lam[i] = 1.0 / 3.0;
    else if (!ok)
      return 0;
    for (int i = 0; i <= M; ++i) out->lam[i] = lam[i];
    double s = 0;
    if (f->scalar && f->layout != ORC_LAYOUT_MULTI)
      for (int i = 0; i <= M; ++i) s += lam[i] * scalar_value(a, g[i], vid[i]);
    out->scalar = (float)s;
  } else {
    float fv[4][3], lam[4];
    for (int i = 0; i <= M; ++i)
      for (int j = 0; j < M; ++j) fv[i][j] = (float)vals[i][j];
    ok = solve_f32(M, fv, lam);
    if (!ok && f->fiber)
      for (int i = 0; i <= M; ++i) lam[i] = (float)(1.0 / 3.0);
    else if (!ok)
      return 0;
    for (int i = 0; i <= M; ++i) out->lam[i] = lam[i];
    float s = 0;
    if (f->scalar && f->layout != ORC_LAYOUT_MULTI)
      for (int i = 0; i <= M; ++i) s += lam[i] * (float)scalar_value(a, g[i], vid[i]);
    out->scalar = s;
  }
  for (int i = 0; i <= M; ++i) out->v[i] = vid[i];
  out->phase = 0;
  return 1;
}

/* ------------------------------------------------------------------------ */
/* Regular mesh                                                               */

/* chain types: strictly increasing non-empty bit masks m1 < ... < mM over d
 * bits (m0 = 0), listed in lexicographic order of the mask sequences, which is
 * also the vertex-id order of the simplices they produce at a fixed corner */
typedef struct {
  int d, m, n;
  uint8_t mask[64][5];
} chains_t;

static void build_chains(chains_t* c, int d, int m) {
  c->d = d; c->m = m; c->n = 0;
  int full = (1 << d) - 1;
  uint8_t cur[5] = {0};
  /* depth-first over subset chains, increasing mask values => lexicographic */
  int stack[5] = {0};
  int depth = 1;
  stack[1] = 0;
  while (depth > 0) {
    int prev = cur[depth - 1];
    int next = stack[depth] + 1;
    while (next <= full && !((next & prev) == prev && next != prev)) ++next;
    if (next > full) { --depth; continue; }
    stack[depth] = next;
    cur[depth] = (uint8_t)next;
    if (depth == m) {
      for (int k = 0; k <= m; ++k) c->mask[c->n][k] = cur[k];
      c->n++;
    } else {
      ++depth;
      stack[depth] = 0;
    }
  }
}

typedef struct {
  const orc_mesh* mesh;
  acc_t acc;
  const chains_t* ch;
  int M, d;
  uint64_t n_corners;
  uint64_t start, end;
  fvec_t out;
  uint64_t tested;
} reg_job_t;

static inline uint64_t grid_id(const orc_mesh* me, const uint64_t g[4]) {
  uint64_t id = 0, mul = 1;
  for (int k = 0; k < me->ndims; ++k) { id += g[k] * mul; mul *= me->global_dims[k]; }
  return id;
}

static void* reg_worker(void* arg) {
  reg_job_t* J = (reg_job_t*)arg;
  const orc_mesh* me = J->mesh;
  int d = J->d, M = J->M;
  for (uint64_t ci = J->start; ci < J->end; ++ci) {
    uint64_t c[4] = {0, 0, 0, 0}, t = ci;
    for (int k = 0; k < d; ++k) { c[k] = t % me->local_dims[k]; t /= me->local_dims[k]; }
    for (int ty = 0; ty < J->ch->n; ++ty) {
      const uint8_t* mk = J->ch->mask[ty];
      int last = mk[M], okb = 1;
      for (int k = 0; k < d; ++k)
        if (((last >> k) & 1) && c[k] + 1 >= me->local_dims[k]) okb = 0;
      if (!okb) continue;
      uint64_t g[4][4], vid[4];
      for (int i = 0; i <= M; ++i) {
        for (int k = 0; k < 4; ++k) g[i][k] = 0;
        for (int k = 0; k < d; ++k) g[i][k] = c[k] + me->offset[k] + ((mk[i] >> k) & 1);
        vid[i] = grid_id(me, g[i]);
      }
      J->tested++;
      feat_t fe;
      if (evaluate(&J->acc, M, vid, g, &fe)) fvec_push(&J->out, &fe);
    }
  }
  return NULL;
}

static int nthreads_of(const orc_field* f) {
  if (f->n_threads > 0) return f->n_threads;
  long n = sysconf(_SC_NPROCESSORS_ONLN);
  return n > 0 ? (int)n : 4;
}

/* ------------------------------------------------------------------------ */
/* Union-find with min-root linking (engine.hpp:46-74)                        */

static uint64_t uf_find(uint64_t* p, uint64_t i) {
  uint64_t r = i;
  while (p[r] != r) r = p[r];
  while (p[i] != r) { uint64_t n = p[i]; p[i] = r; i = n; }
  return r;
}

static void uf_unite(uint64_t* p, uint64_t a, uint64_t b) {
  uint64_t ra = uf_find(p, a), rb = uf_find(p, b);
  if (ra == rb) return;
  if (ra < rb) p[rb] = ra; else p[ra] = rb;
}

/* ------------------------------------------------------------------------ */
/* Edge list                                                                  */

typedef struct { uint32_t a, b; } edge_t;
typedef struct { edge_t* e; size_t n, cap; } evec_t;

static void evec_push(evec_t* v, uint32_t a, uint32_t b) {
  if (v->n == v->cap) {
    v->cap = v->cap ? v->cap * 2 : 256;
    v->e = (edge_t*)realloc(v->e, v->cap * sizeof(edge_t));
  }
  v->e[v->n].a = a < b ? a : b;
  v->e[v->n].b = a < b ? b : a;
  v->n++;
}

static int cmp_edge(const void* x, const void* y) {
  const edge_t* a = (const edge_t*)x;
  const edge_t* b = (const edge_t*)y;
  if (a->a != b->a) return a->a < b->a ? -1 : 1;
  if (a->b != b->b) return a->b < b->b ? -1 : 1;
  return 0;
}

static int64_t find_feat(const feat_t* F, size_t n, const uint64_t* key, int m) {
  size_t lo = 0, hi = n;
  while (lo < hi) {
    size_t mid = (lo + hi) / 2;
    int c = cmp_tuple(F[mid].v, key, m);
    if (c == 0) return (int64_t)mid;
    if (c < 0) lo = mid + 1; else hi = mid;
  }
  return -1;
}

static void sort_tuple(uint64_t* v, int m) {
  for (int i = 0; i <= m; ++i)
    for (int j = i + 1; j <= m; ++j)
      if (v[i] > v[j]) { uint64_t t = v[i]; v[i] = v[j]; v[j] = t; }
}

/* For a top cell given by its sorted vertex ids, collect the active m-faces and
 * emit star edges from the first one in the given order. order_key[] gives, for
 * each feature index, the rank used to choose the star centre. */
static void star_cell(const feat_t* F, size_t nf, const uint64_t* cell, int d, int m,
                      const uint64_t* order_key, evec_t* E) {
  int64_t act[6];
  int na = 0;
  for (int r = 0; r <= d; ++r) {
    uint64_t face[5];
    int k = 0;
    for (int i = 0; i <= d; ++i)
      if (i != r) face[k++] = cell[i];
    int64_t idx = find_feat(F, nf, face, m);
    if (idx >= 0) act[na++] = idx;
  }
  if (na < 2) return;
  int c = 0;
  for (int i = 1; i < na; ++i)
    if (order_key[act[i]] < order_key[act[c]]) c = i;
  for (int i = 0; i < na; ++i)
    if (i != c) evec_push(E, (uint32_t)act[c], (uint32_t)act[i]);
}

static int finish(feat_t* F, size_t n, int m, evec_t* E, uint64_t* parent, uint64_t tested,
                  orc_result* out) {
  /* edges: sorted unique (complex.hpp:38-57) */
  if (E->n) qsort(E->e, E->n, sizeof(edge_t), cmp_edge);
  size_t ne = 0;
  for (size_t i = 0; i < E->n; ++i)
    if (ne == 0 || cmp_edge(&E->e[ne - 1], &E->e[i]) != 0) E->e[ne++] = E->e[i];
  for (size_t i = 0; i < ne; ++i) uf_unite(parent, E->e[i].a, E->e[i].b);

  out->m = m;
  out->n = n;
  out->n_tested = tested;
  out->simplices = (uint64_t*)malloc(sizeof(uint64_t) * (n * (m + 1) + 1));
  out->bary = (float*)malloc(sizeof(float) * (n * (m + 1) + 1));
  out->lambda = (double*)malloc(sizeof(double) * (n * (m + 1) + 1));
  out->track_id = (uint64_t*)malloc(sizeof(uint64_t) * (n + 1));
  out->type = (uint32_t*)malloc(sizeof(uint32_t) * (n + 1));
  out->scalar = (float*)malloc(sizeof(float) * (n + 1));
  for (size_t i = 0; i < n; ++i) {
    for (int k = 0; k <= m; ++k) {
      out->simplices[i * (m + 1) + k] = F[i].v[k];
      out->lambda[i * (m + 1) + k] = F[i].lam[k];
      out->bary[i * (m + 1) + k] = (float)F[i].lam[k];
    }
    out->track_id[i] = uf_find(parent, i);
    out->type[i] = 0;
    out->scalar[i] = F[i].scalar;
  }
  out->n_edges = ne;
  out->edges = (uint32_t*)malloc(sizeof(uint32_t) * (2 * ne + 2));
  for (size_t i = 0; i < ne; ++i) {
    out->edges[2 * i] = E->e[i].a;
    out->edges[2 * i + 1] = E->e[i].b;
  }
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Classification (no counterpart in the reference: type = 0 always,          */
/* predicate.hpp:80).  J = spatial Jacobian of the linear interpolant on the  */
/* feature's first coface top cell, in the field precision; invariants in     */
/* FP64 on J scaled by 2^-e (e = exponent of max |J|), every operation        */
/* rounded separately in the order below.  Codes: 1 degenerate, 2 source,     */
/* 3 sink, 4 saddle, 5 spiral source, 6 spiral sink, 7 centre.                */

enum { CL_DEGENERATE = 1, CL_SOURCE = 2, CL_SINK = 3, CL_SADDLE = 4, CL_SPIRAL_SOURCE = 5,
       CL_SPIRAL_SINK = 6, CL_CENTER = 7 };

static int sgnd(double x) { return x > 0 ? 1 : (x < 0 ? -1 : 0); }

static uint32_t decide2(int sdet, int str, int sdisc) {
  if (sdet == 0) return CL_DEGENERATE;
  if (sdet < 0) return CL_SADDLE;
  if (sdisc >= 0) return str > 0 ? CL_SOURCE : (str < 0 ? CL_SINK : CL_DEGENERATE);
  return str > 0 ? CL_SPIRAL_SOURCE : (str < 0 ? CL_SPIRAL_SINK : CL_CENTER);
}

static uint32_t decide3(int sa2, int sa1, int sh, int sa0, int sdelta) {
  if (sa0 == 0) return CL_DEGENERATE;
  /* h = 0: (l + a2)(l^2 + a1) */
  if (sh == 0) return sa1 < 0 ? CL_SADDLE : (sa1 > 0 ? CL_CENTER : CL_DEGENERATE);
  if (sa2 == 0) return CL_SADDLE;
  int c1 = sa2, c2 = sh * sa2, c3 = sa0;
  int npos = (c1 < 0) + (c1 != c2) + (c2 != c3);
  int cpx = sdelta < 0;
  if (npos == 3) return cpx ? CL_SPIRAL_SOURCE : CL_SOURCE;
  if (npos == 0) return cpx ? CL_SPIRAL_SINK : CL_SINK;
  return CL_SADDLE;
}

/* J[j][a] = d v_j / d x_a as doubles holding values of the field precision */
uint32_t cporacle_classify_jacobian(int m, const double* Jin) {
  double mx = 0;
  for (int i = 0; i < m * m; ++i) {
    if (!isfinite(Jin[i])) return CL_DEGENERATE;
    if (fabs(Jin[i]) > mx) mx = fabs(Jin[i]);
  }
  if (mx == 0) return CL_DEGENERATE;
  int e;
  frexp(mx, &e);
  double J[3][3];
  for (int j = 0; j < m; ++j)
    for (int a = 0; a < m; ++a) J[j][a] = ldexp(Jin[j * m + a], -e);
  if (m == 2) {
    double ad = J[0][0] * J[1][1], bc = J[0][1] * J[1][0];
    double det = ad - bc;
    double tr = J[0][0] + J[1][1];
    double disc = tr * tr - 4.0 * det;
    return decide2(sgnd(det), sgnd(tr), sgnd(disc));
  }
  double p0 = J[1][1] * J[2][2], q0 = J[1][2] * J[2][1];
  double p1 = J[0][0] * J[2][2], q1 = J[0][2] * J[2][0];
  double p2 = J[0][0] * J[1][1], q2 = J[0][1] * J[1][0];
  double m0 = p0 - q0, m1 = p1 - q1, m2 = p2 - q2;
  double r1 = J[1][0] * J[2][2], u1 = J[1][2] * J[2][0];
  double r2 = J[1][0] * J[2][1], u2 = J[1][1] * J[2][0];
  double c1 = r1 - u1, c2 = r2 - u2;
  double tr = (J[0][0] + J[1][1]) + J[2][2];
  double a1 = (m0 + m1) + m2;
  double det = (J[0][0] * m0 - J[0][1] * c1) + J[0][2] * c2;
  double a2 = -tr, a0 = -det;
  double h = a2 * a1 - a0;
  double b = a2, c = a1, d = a0;
  double t1 = ((18.0 * b) * c) * d;
  double t2 = (((4.0 * b) * b) * b) * d;
  double t3 = ((b * b) * c) * c;
  double t4 = ((4.0 * c) * c) * c;
  double t5 = (27.0 * d) * d;
  double delta = (((t1 - t2) + t3) - t4) - t5;
  return decide3(sgnd(a2), sgnd(a1), sgnd(h), sgnd(a0), sgnd(delta));
}

/* Class of a regular-mesh feature from its first coface top cell (corner
 * cc, masks cm), or degenerate without one. */
static uint32_t classify_regular_cell(const acc_t* acc, const orc_mesh* me, int d, int nc,
                                      const uint64_t cc[4], const int cm[5]) {
  int m = d - 1;
  if (nc == 0) return CL_DEGENERATE;
  double val[5][3];
  for (int r = 0; r <= d; ++r) {
    uint64_t g[4] = {0, 0, 0, 0};
    for (int k = 0; k < d; ++k) g[k] = cc[k] + ((cm[r] >> k) & 1);
    uint64_t vid = grid_id(me, g);
    for (int j = 0; j < m; ++j) val[r][j] = field_value(acc, j, g, vid);
  }
  double J[9];
  for (int r = 1; r <= d; ++r) {
    int axis = __builtin_ctz(cm[r] ^ cm[r - 1]);
    if (axis >= m) continue;
    for (int j = 0; j < m; ++j) {
      if (acc->f->dtype == ORC_F64) J[j * m + axis] = val[r][j] - val[r - 1][j];
      else J[j * m + axis] = (double)((float)val[r][j] - (float)val[r - 1][j]);
    }
  }
  return cporacle_classify_jacobian(m, J);
}

typedef struct { uint32_t v[3]; } tri_t;

static int cmp_tri(const void* x, const void* y) {
  const uint32_t *a = ((const tri_t*)x)->v, *b = ((const tri_t*)y)->v;
  for (int i = 0; i < 3; ++i)
    if (a[i] != b[i]) return a[i] < b[i] ? -1 : 1;
  return 0;
}

/* Fiber surfaces (triangle features of a 3D+t mesh): form_general_manifold_
 * patches with k = 2 (engine.hpp:1342-1417) on every pentatope of the local
 * mesh.  Its active triangles in feature order (the order of their
 * encode_simplex_id codes), h_S the first; on each tet face holding two or
 * more, h_T the first there and a triangle (h_S, h_T, n) for every later n
 * whenever h_S differs from both.  get_complex keeps the sorted unique
 * triangles and unites their features; a track id is the component's
 * smallest feature index. */
static void fiber_surface_cells(const orc_mesh* me, const feat_t* F, size_t n, uint64_t tested,
                                orc_result* out) {
  chains_t pc;
  build_chains(&pc, 4, 4);
  tri_t* T = NULL;
  size_t nt = 0, cap = 0;
  uint64_t n_corners = 1;
  for (int k = 0; k < 4; ++k) n_corners *= me->local_dims[k];
  for (uint64_t ci = 0; ci < n_corners && n; ++ci) {
    uint64_t c[4], t = ci;
    int inside = 1;
    for (int k = 0; k < 4; ++k) {
      c[k] = t % me->local_dims[k];
      t /= me->local_dims[k];
      if (c[k] + 1 >= me->local_dims[k]) inside = 0;
    }
    if (!inside) continue;
    for (int ty = 0; ty < pc.n; ++ty) {
      uint64_t cell[5];
      for (int r = 0; r <= 4; ++r) {
        uint64_t g[4];
        for (int k = 0; k < 4; ++k) g[k] = c[k] + me->offset[k] + ((pc.mask[ty][r] >> k) & 1);
        cell[r] = grid_id(me, g);
      }
      /* the 10 triangle faces (ids ascending, as the cell's are) */
      int64_t node[10];
      int nn = 0;
      uint64_t nv[10][3];
      for (int a = 0; a < 5; ++a)
        for (int b = a + 1; b < 5; ++b)
          for (int e = b + 1; e < 5; ++e) {
            uint64_t key[3] = {cell[a], cell[b], cell[e]};
            int64_t idx = find_feat(F, n, key, 2);
            if (idx >= 0) {
              node[nn] = idx;
              nv[nn][0] = key[0]; nv[nn][1] = key[1]; nv[nn][2] = key[2];
              nn++;
            }
          }
      if (nn < 2) continue;
      /* feature order */
      for (int i = 1; i < nn; ++i)
        for (int j = i; j > 0 && node[j] < node[j - 1]; --j) {
          int64_t tn = node[j]; node[j] = node[j - 1]; node[j - 1] = tn;
          for (int q = 0; q < 3; ++q) { uint64_t tv = nv[j][q]; nv[j][q] = nv[j - 1][q]; nv[j - 1][q] = tv; }
        }
      const int64_t hS = node[0];
      for (int x = 0; x < 5; ++x) { /* the tet face without cell vertex x */
        int64_t onf[10];
        int no = 0;
        for (int i = 0; i < nn; ++i)
          if (nv[i][0] != cell[x] && nv[i][1] != cell[x] && nv[i][2] != cell[x]) onf[no++] = node[i];
        if (no < 2) continue;
        const int64_t hT = onf[0];
        for (int j = 1; j < no; ++j) {
          if (hS == hT || hS == onf[j]) continue;
          uint32_t v[3] = {(uint32_t)hS, (uint32_t)hT, (uint32_t)onf[j]};
          for (int i = 1; i < 3; ++i)
            for (int q = i; q > 0 && v[q] < v[q - 1]; --q) { uint32_t tv = v[q]; v[q] = v[q - 1]; v[q - 1] = tv; }
          if (nt == cap) {
            cap = cap ? 2 * cap : 1024;
            T = (tri_t*)realloc(T, cap * sizeof(tri_t));
          }
          T[nt].v[0] = v[0]; T[nt].v[1] = v[1]; T[nt].v[2] = v[2];
          nt++;
        }
      }
    }
  }
  if (nt) qsort(T, nt, sizeof(tri_t), cmp_tri);
  size_t nu = 0;
  for (size_t i = 0; i < nt; ++i)
    if (nu == 0 || cmp_tri(&T[nu - 1], &T[i]) != 0) T[nu++] = T[i];
  uint64_t* parent = (uint64_t*)malloc(sizeof(uint64_t) * (n + 1));
  for (size_t i = 0; i < n; ++i) parent[i] = i;
  for (size_t i = 0; i < nu; ++i) {
    uf_unite(parent, T[i].v[0], T[i].v[1]);
    uf_unite(parent, T[i].v[1], T[i].v[2]);
  }
  evec_t none = {0};
  finish((feat_t*)F, n, 2, &none, parent, tested, out);
  out->cp_class = NULL;
  out->cell_dim = 2;
  out->n_cells = nu;
  out->cells = (uint32_t*)malloc(sizeof(uint32_t) * (3 * nu + 3));
  for (size_t i = 0; i < nu; ++i)
    for (int q = 0; q < 3; ++q) out->cells[3 * i + q] = T[i].v[q];
  free(T);
  free(parent);
}

static int run_regular(const orc_mesh* me, const orc_field* f, orc_result* out) {
  int d = me->ndims, M = f->ncomp;
  const int surfaces = f->fiber && d == 4 && M == 2; /* fiber surfaces: triangles of the 3D+t mesh */
  if (!((d == 3 && M == 2) || (d == 4 && M == 3) || surfaces)) return 2;
  chains_t ch;
  build_chains(&ch, d, M);

  uint64_t n_corners = 1;
  for (int k = 0; k < d; ++k) n_corners *= me->local_dims[k];

  int nt = nthreads_of(f);
  reg_job_t* jobs = (reg_job_t*)calloc((size_t)nt, sizeof(reg_job_t));
  pthread_t* th = (pthread_t*)calloc((size_t)nt, sizeof(pthread_t));
  for (int i = 0; i < nt; ++i) {
    reg_job_t* J = &jobs[i];
    J->mesh = me;
    J->acc.f = f;
    J->acc.nd_mesh = d;
    for (int k = 0; k < 4; ++k) J->acc.offset[k] = me->offset[k];
    J->ch = &ch;
    J->M = M;
    J->d = d;
    J->start = n_corners * (uint64_t)i / (uint64_t)nt;
    J->end = n_corners * (uint64_t)(i + 1) / (uint64_t)nt;
    pthread_create(&th[i], NULL, reg_worker, J);
  }
  fvec_t all = {0};
  uint64_t tested = 0;
  for (int i = 0; i < nt; ++i) {
    pthread_join(th[i], NULL);
    for (size_t k = 0; k < jobs[i].out.n; ++k) fvec_push(&all, &jobs[i].out.a[k]);
    free(jobs[i].out.a);
    tested += jobs[i].tested;
  }
  free(jobs);
  free(th);

  g_m = M;
  if (all.n) qsort(all.a, all.n, sizeof(feat_t), cmp_feat);
  size_t n = all.n;
  feat_t* F = all.a;

  if (surfaces) {
    fiber_surface_cells(me, F, n, tested, out);
    free(F);
    return 0;
  }

  /* star edges: every top cell with >= 2 active faces is a coface of each of
   * them, so visiting the cofaces of each feature covers engine.hpp:161-180.
   * For regular meshes the encode_simplex_id order of faces equals the
   * Simplex order, i.e. the feature index. */
  uint64_t* order = (uint64_t*)malloc(sizeof(uint64_t) * (n + 1));
  for (size_t i = 0; i < n; ++i) order[i] = i;
  evec_t E = {0};
  uint32_t* cls = (uint32_t*)malloc(sizeof(uint32_t) * (n + 1));
  acc_t cacc;
  memset(&cacc, 0, sizeof(cacc));
  cacc.f = f;
  cacc.nd_mesh = d;
  for (int k = 0; k < 4; ++k) cacc.offset[k] = me->offset[k];
  int full = (1 << d) - 1;
  uint64_t stride[4] = {1, 1, 1, 1};
  for (int k = 1; k < d; ++k) stride[k] = stride[k - 1] * me->global_dims[k - 1];
  for (size_t i = 0; i < n; ++i) {
    /* recover corner (global) and masks of feature i */
    uint64_t c[4], v0 = F[i].v[0], tmp = v0;
    for (int k = 0; k < d; ++k) { c[k] = tmp % me->global_dims[k]; tmp /= me->global_dims[k]; }
    int mk[5];
    mk[0] = 0;
    for (int j = 1; j <= M; ++j) {
      uint64_t diff = F[i].v[j] - v0;
      int msk = 0;
      for (int k = d - 1; k >= 0; --k)
        if (diff >= stride[k]) { msk |= 1 << k; diff -= stride[k]; }
      mk[j] = msk;
    }
    int missing = full & ~mk[M];
    int cell_m[2][5];
    uint64_t cell_c[2][4];
    int nc = 0;
    if (missing) {
      int a = __builtin_ctz(missing);
      /* prepend: corner c - e_a */
      if (c[a] >= me->offset[a] + 1) {
        for (int k = 0; k < 4; ++k) cell_c[nc][k] = c[k];
        cell_c[nc][a] -= 1;
        cell_m[nc][0] = 0;
        for (int j = 0; j <= M; ++j) cell_m[nc][j + 1] = mk[j] | (1 << a);
        nc++;
      }
      /* append: corner c, final mask full */
      if (c[a] + 1 < me->offset[a] + me->local_dims[a]) {
        for (int k = 0; k < 4; ++k) cell_c[nc][k] = c[k];
        for (int j = 0; j <= M; ++j) cell_m[nc][j] = mk[j];
        cell_m[nc][M + 1] = full;
        nc++;
      }
    } else {
      for (int j = 1; j <= M; ++j) {
        int step = mk[j] & ~mk[j - 1];
        if (__builtin_popcount(step) == 2) {
          int lo = step & -step, hi = step & ~lo;
          int ins[2] = {lo, hi};
          for (int q = 0; q < 2; ++q) {
            for (int k = 0; k < 4; ++k) cell_c[nc][k] = c[k];
            int w = 0;
            for (int jj = 0; jj <= M; ++jj) {
              if (jj == j) cell_m[nc][w++] = mk[j - 1] | ins[q];
              cell_m[nc][w++] = mk[jj];
            }
            nc++;
          }
          break;
        }
      }
    }
    cls[i] = classify_regular_cell(&cacc, me, d, nc, cell_c[0], cell_m[0]);
    for (int q = 0; q < nc; ++q) {
      uint64_t cell[5];
      for (int r = 0; r <= d; ++r) {
        uint64_t g[4] = {0, 0, 0, 0};
        for (int k = 0; k < d; ++k) g[k] = cell_c[q][k] + ((cell_m[q][r] >> k) & 1);
        cell[r] = grid_id(me, g);
      }
      star_cell(F, n, cell, d, M, order, &E);
    }
  }
  uint64_t* parent = (uint64_t*)malloc(sizeof(uint64_t) * (n + 1));
  for (size_t i = 0; i < n; ++i) parent[i] = i;
  finish(F, n, M, &E, parent, tested, out);
  out->cp_class = cls;
  free(parent);
  free(order);
  free(E.e);
  free(F);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Extruded unstructured mesh (mesh.hpp:542-730, unstructured_mesh.hpp)       */

typedef struct {
  uint64_t v[4];
} face_t;

static int cmp_face3(const void* x, const void* y) {
  return cmp_tuple(((const face_t*)x)->v, ((const face_t*)y)->v, 2);
}
static int cmp_face2(const void* x, const void* y) {
  return cmp_tuple(((const face_t*)x)->v, ((const face_t*)y)->v, 1);
}

typedef struct {
  int cd;                 /* base cell dim */
  uint64_t nv, ncell, nface, L;
  uint64_t* cells;        /* sorted vertices, (cd+1) per cell */
  face_t* faces;          /* unique (cd-1)-faces, sorted */
  uint64_t* cof_start;    /* CSR: faces -> cells */
  uint64_t* cof;
} ext_t;

static int64_t find_face(const ext_t* X, const uint64_t* key) {
  size_t lo = 0, hi = X->nface;
  while (lo < hi) {
    size_t mid = (lo + hi) / 2;
    int c = cmp_tuple(X->faces[mid].v, key, X->cd - 1);
    if (c == 0) return (int64_t)mid;
    if (c < 0) lo = mid + 1; else hi = mid;
  }
  return -1;
}

typedef struct {
  const ext_t* X;
  acc_t acc;
  int M;
  int kind;               /* 0 spatial, 1 prism, 2 interior */
  uint64_t start, end;    /* range over items of this kind */
  fvec_t out;
  uint64_t tested;
} ext_job_t;

static void* ext_worker(void* arg) {
  ext_job_t* J = (ext_job_t*)arg;
  const ext_t* X = J->X;
  int M = J->M, cd = X->cd;
  uint64_t ns = X->nv;
  for (uint64_t it = J->start; it < J->end; ++it) {
    uint64_t vid[5];
    int nvx = M + 1;
    if (J->kind == 0) {
      uint64_t cell = it % X->ncell, t = it / X->ncell;
      for (int i = 0; i <= cd; ++i) vid[i] = X->cells[cell * (cd + 1) + i] + t * ns;
      J->tested++;
      uint64_t g[4][4] = {{0}};
      feat_t fe;
      if (evaluate(&J->acc, M, vid, g, &fe)) { fe.phase = 0; fvec_push(&J->out, &fe); }
    } else if (J->kind == 1) {
      uint64_t fidx = it % X->nface, t = it / X->nface;
      const uint64_t* w = X->faces[fidx].v; /* cd vertices */
      for (int j = 0; j < cd; ++j) {
        int k = 0;
        for (int l = 0; l <= j; ++l) vid[k++] = w[l] + t * ns;
        for (int l = j; l < cd; ++l) vid[k++] = w[l] + (t + 1) * ns;
        sort_tuple(vid, M);
        J->tested++;
        uint64_t g[4][4] = {{0}};
        feat_t fe;
        if (evaluate(&J->acc, M, vid, g, &fe)) { fe.phase = 0; fvec_push(&J->out, &fe); }
      }
    } else {
      uint64_t cell = it % X->ncell, t = it / X->ncell;
      const uint64_t* w = &X->cells[cell * (cd + 1)];
      for (int s = 1; s <= cd; ++s) {
        int k = 0;
        for (int l = 0; l < s; ++l) vid[k++] = w[l] + t * ns;
        for (int l = s; l <= cd; ++l) vid[k++] = w[l] + (t + 1) * ns;
        J->tested++;
        uint64_t g[4][4] = {{0}};
        feat_t fe;
        if (evaluate(&J->acc, M, vid, g, &fe)) { fe.phase = 1; fvec_push(&J->out, &fe); }
      }
    }
    (void)nvx;
  }
  return NULL;
}

static void ext_emit_face_faces(const feat_t* F, size_t n, const uint64_t* cell, int d, int m,
                                uint64_t* parent, uint64_t self) {
  for (int r = 0; r <= d; ++r) {
    uint64_t face[5];
    int k = 0;
    for (int i = 0; i <= d; ++i)
      if (i != r) face[k++] = cell[i];
    sort_tuple(face, m);
    int64_t idx = find_feat(F, n, face, m);
    if (idx >= 0) uf_unite(parent, self, (uint64_t)idx);
  }
}

/* Fiber surfaces on an extruded tet mesh: FiberPredicate<T> on
 * ExtrudedSimplicialMesh(UnstructuredSimplicialMesh(tets), L), a 4-D
 * spacetime mesh whose features are triangles (engine.hpp:101-212, 1342-1417;
 * mesh.hpp:568-599).
 *  - phase 1 iterates the spatial triangles of every layer (the base mesh's
 *    unique triangles, sorted) and the two Kuhn pieces of every base edge
 *    between consecutive layers; its accepted triangles get node ids in
 *    Simplex order;
 *  - phase 2 visits the pentatopes in the reference's iteration order (layer,
 *    base tet in stored order, prism piece j) and their 10 triangles in
 *    find_m_subsimplices order (engine.hpp:1645-1652); a triangle no earlier
 *    visit found is tested and, if accepted, takes the next node id.  Those
 *    are the triangles interior to the prisms over base triangles.  This is
 *    the order of the reference run with one worker; with several workers
 *    the reference numbers them in thread-arrival order;
 *  - per pentatope: its active triangles sorted by node id, h_S the first; on
 *    each tet face the face's active triangles in the same order, h_T the
 *    first, and {h_S, h_T, n} for every later n unless h_S is h_T or n;
 *  - get_complex: canonical ids = Simplex order, the triangles sorted and
 *    unique, their features united (the 4-D coface unions see no pentatope
 *    among a triangle's cofaces), track id = the component's smallest index.
 */
typedef struct {
  uint64_t v[3];
  int64_t id; /* node id, or -1: tested and rejected */
  int used;
} tslot_t;

typedef struct {
  tslot_t* s;
  size_t cap, n;
} thash_t;

static uint64_t thash_key(const uint64_t* v) {
  uint64_t h = v[0] * 0x9E3779B97F4A7C15ull;
  h ^= v[1] + 0x7F4A7C159E3779B9ull + (h << 6) + (h >> 2);
  h ^= v[2] + 0x94D049BB133111EBull + (h << 6) + (h >> 2);
  return h;
}

static tslot_t* thash_find(thash_t* H, const uint64_t* v, int insert) {
  if (insert && 2 * (H->n + 1) > H->cap) {
    thash_t G = {0};
    G.cap = H->cap ? 2 * H->cap : 1024;
    G.s = (tslot_t*)calloc(G.cap, sizeof(tslot_t));
    for (size_t i = 0; i < H->cap; ++i)
      if (H->s[i].used) {
        size_t j = thash_key(H->s[i].v) & (G.cap - 1);
        while (G.s[j].used) j = (j + 1) & (G.cap - 1);
        G.s[j] = H->s[i];
        G.n++;
      }
    free(H->s);
    *H = G;
  }
  if (!H->cap) return NULL;
  size_t j = thash_key(v) & (H->cap - 1);
  while (H->s[j].used) {
    if (H->s[j].v[0] == v[0] && H->s[j].v[1] == v[1] && H->s[j].v[2] == v[2]) return &H->s[j];
    j = (j + 1) & (H->cap - 1);
  }
  if (!insert) return NULL;
  H->s[j].used = 1;
  H->s[j].v[0] = v[0]; H->s[j].v[1] = v[1]; H->s[j].v[2] = v[2];
  H->s[j].id = -1;
  H->n++;
  return &H->s[j];
}

static int run_extruded_fiber_surface(const ext_t* X, const acc_t* acc, orc_result* out) {
  const uint64_t ns = X->nv, L = X->L;
  /* unique base edges, sorted (unstructured_mesh.hpp:44-53) */
  face_t* E1 = (face_t*)malloc(sizeof(face_t) * (3 * X->nface + 1));
  size_t n1 = 0;
  for (size_t i = 0; i < X->nface; ++i) {
    const uint64_t* w = X->faces[i].v;
    uint64_t e[3][2] = {{w[0], w[1]}, {w[0], w[2]}, {w[1], w[2]}};
    for (int q = 0; q < 3; ++q) { E1[n1].v[0] = e[q][0]; E1[n1].v[1] = e[q][1]; n1++; }
  }
  qsort(E1, n1, sizeof(face_t), cmp_face2);
  size_t nu1 = 0;
  for (size_t i = 0; i < n1; ++i)
    if (nu1 == 0 || cmp_tuple(E1[nu1 - 1].v, E1[i].v, 1) != 0) E1[nu1++] = E1[i];

  /* phase 1 */
  fvec_t P = {0};
  uint64_t tested = 0;
  uint64_t g[4][4] = {{0}};
  for (uint64_t t = 0; t <= L; ++t)
    for (size_t i = 0; i < X->nface; ++i) {
      uint64_t vid[4] = {X->faces[i].v[0] + t * ns, X->faces[i].v[1] + t * ns, X->faces[i].v[2] + t * ns, 0};
      feat_t fe;
      tested++;
      if (evaluate(acc, 2, vid, g, &fe)) fvec_push(&P, &fe);
    }
  for (uint64_t t = 0; t < L; ++t)
    for (size_t i = 0; i < nu1; ++i) {
      const uint64_t a = E1[i].v[0], b = E1[i].v[1];
      uint64_t pieces[2][4] = {{a + t * ns, a + (t + 1) * ns, b + (t + 1) * ns, 0},
                               {a + t * ns, b + t * ns, b + (t + 1) * ns, 0}};
      for (int j = 0; j < 2; ++j) {
        feat_t fe;
        tested++;
        if (evaluate(acc, 2, pieces[j], g, &fe)) fvec_push(&P, &fe);
      }
    }
  g_m = 2;
  if (P.n) qsort(P.a, P.n, sizeof(feat_t), cmp_feat);

  /* node table: phase-1 nodes first, in Simplex order */
  thash_t H = {0};
  fvec_t all = {0};  /* every node, by node id */
  for (size_t i = 0; i < P.n; ++i) {
    tslot_t* sl = thash_find(&H, P.a[i].v, 1);
    sl->id = (int64_t)all.n;
    fvec_push(&all, &P.a[i]);
  }
  free(P.a);

  /* phase 2: pentatopes in the reference's order */
  typedef struct { uint32_t v[3]; } ntri_t;  /* star-fan triangles in node ids */
  ntri_t* T = NULL;
  size_t nt = 0, tcap = 0;
  for (uint64_t t = 0; t < L; ++t)
    for (uint64_t c = 0; c < X->ncell; ++c) {
      const uint64_t* w = &X->cells[c * 4];
      for (int j = 0; j <= 3; ++j) {
        uint64_t cell[5];
        int k = 0;
        for (int l = 0; l <= j; ++l) cell[k++] = w[l] + t * ns;
        for (int l = j; l <= 3; ++l) cell[k++] = w[l] + (t + 1) * ns;
        int64_t node[10];
        int vs[10];  /* cell positions of the triangle's vertices, as a bit set */
        int nn = 0;
        for (int p0 = 0; p0 < 5; ++p0)
          for (int p1 = p0 + 1; p1 < 5; ++p1)
            for (int p2 = p1 + 1; p2 < 5; ++p2) {
              uint64_t key[3] = {cell[p0], cell[p1], cell[p2]};
              tslot_t* sl = thash_find(&H, key, 0);
              if (!sl) {
                sl = thash_find(&H, key, 1);
                uint64_t vid[4] = {key[0], key[1], key[2], 0};
                feat_t fe;
                tested++;
                if (evaluate(acc, 2, vid, g, &fe)) {
                  sl->id = (int64_t)all.n;
                  fe.phase = 1;
                  fvec_push(&all, &fe);
                }
              }
              if (sl->id >= 0) {
                node[nn] = sl->id;
                vs[nn] = (1 << p0) | (1 << p1) | (1 << p2);
                nn++;
              }
            }
        if (nn < 2) continue;
        for (int i = 1; i < nn; ++i)
          for (int q = i; q > 0 && node[q] < node[q - 1]; --q) {
            int64_t tn = node[q]; node[q] = node[q - 1]; node[q - 1] = tn;
            int tv = vs[q]; vs[q] = vs[q - 1]; vs[q - 1] = tv;
          }
        const int64_t hS = node[0];
        for (int x = 0; x < 5; ++x) { /* the tet face without cell vertex x */
          int seen = 0;
          int64_t hT = -1;
          for (int i = 0; i < nn; ++i) {
            if (vs[i] & (1 << x)) continue;
            if (seen++ == 0) { hT = node[i]; continue; }
            if (hS == hT || hS == node[i]) continue;
            if (nt == tcap) {
              tcap = tcap ? 2 * tcap : 1024;
              T = (ntri_t*)realloc(T, tcap * sizeof(ntri_t));
            }
            T[nt].v[0] = (uint32_t)hS; T[nt].v[1] = (uint32_t)hT; T[nt].v[2] = (uint32_t)node[i];
            nt++;
          }
        }
      }
    }
  free(H.s);

  /* get_complex: canonical order, triangles re-indexed, sorted, unique */
  const size_t n = all.n;
  uint64_t* canon = (uint64_t*)malloc(sizeof(uint64_t) * (n + 1));  /* node id -> canonical index */
  {
    feat_t* F = (feat_t*)malloc(sizeof(feat_t) * (n + 1));
    /* v[3] carries the node id through the sort (the first three entries
     * never tie: every node is a distinct triangle) */
    for (size_t i = 0; i < n; ++i) { F[i] = all.a[i]; F[i].scalar = 0.0f; F[i].v[3] = i; }
    if (n) qsort(F, n, sizeof(feat_t), cmp_feat);
    for (size_t i = 0; i < n; ++i) { canon[F[i].v[3]] = i; F[i].v[3] = 0; }
    free(all.a);
    all.a = F;
  }
  tri_t* C = (tri_t*)malloc(sizeof(tri_t) * (nt + 1));
  for (size_t i = 0; i < nt; ++i) {
    uint32_t v[3] = {(uint32_t)canon[T[i].v[0]], (uint32_t)canon[T[i].v[1]], (uint32_t)canon[T[i].v[2]]};
    for (int a = 1; a < 3; ++a)
      for (int q = a; q > 0 && v[q] < v[q - 1]; --q) { uint32_t tv = v[q]; v[q] = v[q - 1]; v[q - 1] = tv; }
    C[i].v[0] = v[0]; C[i].v[1] = v[1]; C[i].v[2] = v[2];
  }
  free(T);
  free(canon);
  if (nt) qsort(C, nt, sizeof(tri_t), cmp_tri);
  size_t nu = 0;
  for (size_t i = 0; i < nt; ++i)
    if (nu == 0 || cmp_tri(&C[nu - 1], &C[i]) != 0) C[nu++] = C[i];
  uint64_t* parent = (uint64_t*)malloc(sizeof(uint64_t) * (n + 1));
  for (size_t i = 0; i < n; ++i) parent[i] = i;
  for (size_t i = 0; i < nu; ++i) {
    uf_unite(parent, C[i].v[0], C[i].v[1]);
    uf_unite(parent, C[i].v[1], C[i].v[2]);
  }
  evec_t none = {0};
  finish(all.a, n, 2, &none, parent, tested, out);
  out->cp_class = NULL;
  out->cell_dim = 2;
  out->n_cells = nu;
  out->cells = (uint32_t*)malloc(sizeof(uint32_t) * (3 * nu + 3));
  for (size_t i = 0; i < nu; ++i)
    for (int q = 0; q < 3; ++q) out->cells[3 * i + q] = C[i].v[q];
  free(C);
  free(parent);
  free(all.a);
  free(E1);
  return 0;
}

static int run_extruded(const orc_mesh* me, const orc_field* f, orc_result* out) {
  ext_t X;
  memset(&X, 0, sizeof(X));
  X.cd = me->base_cell_dim;
  int M = f->ncomp;
  const int surfaces = f->fiber && X.cd == 3 && M == 2; /* fiber surfaces over tets */
  if (!surfaces && (X.cd != M || (M != 2 && M != 3))) return 2;
  X.ncell = me->n_base_cells;
  X.L = me->n_layers;
  /* n_spatial_verts = max vertex id + 1 over the base's vertices (mesh.hpp:556-561);
   * an UnstructuredSimplicialMesh lists every coordinate as a vertex */
  X.nv = me->n_base_verts;
  X.cells = (uint64_t*)malloc(sizeof(uint64_t) * X.ncell * (X.cd + 1));
  for (uint64_t c = 0; c < X.ncell; ++c) {
    uint64_t* v = &X.cells[c * (X.cd + 1)];
    for (int i = 0; i <= X.cd; ++i) v[i] = me->base_cells[c * (X.cd + 1) + i];
    sort_tuple(v, X.cd);
  }
  /* unique (cd-1)-faces, sorted (unstructured_mesh.hpp:44-53) */
  face_t* all = (face_t*)malloc(sizeof(face_t) * X.ncell * (X.cd + 1));
  size_t na = 0;
  for (uint64_t c = 0; c < X.ncell; ++c) {
    uint64_t* v = &X.cells[c * (X.cd + 1)];
    for (int r = 0; r <= X.cd; ++r) {
      int k = 0;
      for (int i = 0; i <= X.cd; ++i)
        if (i != r) all[na].v[k++] = v[i];
      na++;
    }
  }
  qsort(all, na, sizeof(face_t), X.cd == 3 ? cmp_face3 : cmp_face2);
  size_t nu = 0;
  for (size_t i = 0; i < na; ++i)
    if (nu == 0 || cmp_tuple(all[nu - 1].v, all[i].v, X.cd - 1) != 0) all[nu++] = all[i];
  X.faces = all;
  X.nface = nu;
  /* coface CSR */
  X.cof_start = (uint64_t*)calloc(nu + 1, sizeof(uint64_t));
  for (uint64_t c = 0; c < X.ncell; ++c) {
    uint64_t* v = &X.cells[c * (X.cd + 1)];
    for (int r = 0; r <= X.cd; ++r) {
      uint64_t key[4];
      int k = 0;
      for (int i = 0; i <= X.cd; ++i)
        if (i != r) key[k++] = v[i];
      X.cof_start[find_face(&X, key) + 1]++;
    }
  }
  for (size_t i = 0; i < nu; ++i) X.cof_start[i + 1] += X.cof_start[i];
  X.cof = (uint64_t*)malloc(sizeof(uint64_t) * (X.cof_start[nu] + 1));
  uint64_t* fill = (uint64_t*)calloc(nu + 1, sizeof(uint64_t));
  for (uint64_t c = 0; c < X.ncell; ++c) {
    uint64_t* v = &X.cells[c * (X.cd + 1)];
    for (int r = 0; r <= X.cd; ++r) {
      uint64_t key[4];
      int k = 0;
      for (int i = 0; i <= X.cd; ++i)
        if (i != r) key[k++] = v[i];
      int64_t fi = find_face(&X, key);
      X.cof[X.cof_start[fi] + fill[fi]++] = c;
    }
  }
  free(fill);

  if (surfaces) {
    acc_t acc;
    memset(&acc, 0, sizeof(acc));
    acc.f = f;
    int rc = run_extruded_fiber_surface(&X, &acc, out);
    free(X.cells);
    free(X.faces);
    free(X.cof_start);
    free(X.cof);
    return rc;
  }

  /* evaluate every m-simplex of the extruded mesh */
  int nt = nthreads_of(f);
  uint64_t counts[3] = {X.ncell * (X.L + 1), X.nface * X.L, X.ncell * X.L};
  fvec_t allf = {0};
  uint64_t tested = 0;
  for (int kind = 0; kind < 3; ++kind) {
    ext_job_t* jobs = (ext_job_t*)calloc((size_t)nt, sizeof(ext_job_t));
    pthread_t* th = (pthread_t*)calloc((size_t)nt, sizeof(pthread_t));
    for (int i = 0; i < nt; ++i) {
      ext_job_t* J = &jobs[i];
      J->X = &X;
      J->acc.f = f;
      J->acc.nd_mesh = 0;
      J->M = M;
      J->kind = kind;
      J->start = counts[kind] * (uint64_t)i / (uint64_t)nt;
      J->end = counts[kind] * (uint64_t)(i + 1) / (uint64_t)nt;
      pthread_create(&th[i], NULL, ext_worker, J);
    }
    for (int i = 0; i < nt; ++i) {
      pthread_join(th[i], NULL);
      for (size_t k = 0; k < jobs[i].out.n; ++k) fvec_push(&allf, &jobs[i].out.a[k]);
      free(jobs[i].out.a);
      tested += jobs[i].tested;
    }
    free(jobs);
    free(th);
  }
  g_m = M;
  if (allf.n) qsort(allf.a, allf.n, sizeof(feat_t), cmp_feat);
  feat_t* F = allf.a;
  size_t n = allf.n;

  /* node ids: phase-1 nodes (spatial + prism simplices) in Simplex order, then
   * interior simplices found during patching (engine.hpp:149-158, 1352-1367).
   * The reference numbers the latter in thread-scheduling order; here they are
   * numbered in Simplex order. */
  uint64_t* order = (uint64_t*)malloc(sizeof(uint64_t) * (n + 1));
  {
    uint64_t r = 0;
    for (size_t i = 0; i < n; ++i)
      if (F[i].phase == 0) order[i] = r++;
    for (size_t i = 0; i < n; ++i)
      if (F[i].phase == 1) order[i] = r++;
  }

  /* star edges over every pentatope (prism piece j of a base cell at layer t)
   * that has an active face */
  evec_t E = {0};
  int d = X.cd + 1;
  uint64_t ns = X.nv;
  for (uint64_t c = 0; c < X.ncell; ++c) {
    const uint64_t* w = &X.cells[c * (X.cd + 1)];
    for (uint64_t t = 0; t < X.L; ++t) {
      for (int j = 0; j <= X.cd; ++j) {
        uint64_t cell[5];
        int k = 0;
        for (int l = 0; l <= j; ++l) cell[k++] = w[l] + t * ns;
        for (int l = j; l <= X.cd; ++l) cell[k++] = w[l] + (t + 1) * ns;
        /* faces of a sorted cell drop one vertex, so they are sorted too */
        star_cell(F, n, cell, d, M, order, &E);
      }
    }
  }

  uint64_t* parent = (uint64_t*)malloc(sizeof(uint64_t) * (n + 1));
  for (size_t i = 0; i < n; ++i) parent[i] = i;
  /* star-edge unions happen first in get_complex (engine.hpp:854-863) */
  {
    evec_t Ec = {0};
    for (size_t i = 0; i < E.n; ++i) evec_push(&Ec, E.e[i].a, E.e[i].b);
    for (size_t i = 0; i < Ec.n; ++i) uf_unite(parent, Ec.e[i].a, Ec.e[i].b);
    free(Ec.e);
  }

  /* 4D meshes: union every feature with active faces of its cofaces as
   * ExtrudedSimplicialMesh::cofaces reports them (mesh.hpp:601-712,
   * engine.hpp:896-963).  For an interior tet that routine lifts the wrong
   * base face, which can join features of a neighbouring prism; that is
   * reproduced here. */
  if (d == 4) {
    for (size_t i = 0; i < n; ++i) {
      const uint64_t* v = F[i].v;
      uint64_t sp[4], tl[4];
      for (int q = 0; q <= 3; ++q) { tl[q] = v[q] / ns; sp[q] = v[q] % ns; }
      if (tl[0] == tl[3]) {
        uint64_t t = tl[0];
        if (t < X.L) {
          uint64_t cell[5] = {sp[0] + t * ns, sp[1] + t * ns, sp[2] + t * ns, sp[3] + t * ns,
                              sp[3] + (t + 1) * ns};
          sort_tuple(cell, 4);
          ext_emit_face_faces(F, n, cell, 4, 3, parent, i);
        }
        if (t > 0) {
          uint64_t cell[5] = {sp[0] + (t - 1) * ns, sp[0] + t * ns, sp[1] + t * ns, sp[2] + t * ns,
                              sp[3] + t * ns};
          sort_tuple(cell, 4);
          ext_emit_face_faces(F, n, cell, 4, 3, parent, i);
        }
      } else {
        uint64_t t = tl[0];
        int n_at_t = 0;
        for (int q = 0; q <= 3; ++q) n_at_t += tl[q] == t;
        int j0 = n_at_t - 1;
        uint64_t bs[3];
        int bi = 0;
        for (int q = 0; q <= j0; ++q) bs[bi++] = sp[q];
        for (int q = j0 + 2; q <= 3; ++q) bs[bi++] = sp[q];
        int64_t fi = find_face(&X, bs);
        if (fi < 0) continue;
        for (uint64_t e0 = X.cof_start[fi]; e0 < X.cof_start[fi + 1]; ++e0) {
          const uint64_t* u = &X.cells[X.cof[e0] * 4];
          int e = -1, wi = 0;
          for (int ui = 0; ui <= 3; ++ui) {
            if (wi < 3 && u[ui] == bs[wi]) wi++;
            else e = ui;
          }
          if (e < 0) continue;
          int jp = j0 + (e <= j0 ? 1 : 0);
          uint64_t cell[5];
          int k = 0;
          for (int l = 0; l <= jp; ++l) cell[k++] = u[l] + t * ns;
          for (int l = jp; l <= 3; ++l) cell[k++] = u[l] + (t + 1) * ns;
          sort_tuple(cell, 4);
          ext_emit_face_faces(F, n, cell, 4, 3, parent, i);
        }
      }
    }
  }
  finish(F, n, M, &E, parent, tested, out);
  free(parent);
  free(order);
  free(E.e);
  free(F);
  free(X.cells);
  free(X.faces);
  free(X.cof_start);
  free(X.cof);
  return 0;
}

int cporacle_run(const orc_mesh* mesh, const orc_field* field, orc_result* out) {
  memset(out, 0, sizeof(*out));
  if (mesh->kind == ORC_MESH_REGULAR) return run_regular(mesh, field, out);
  if (mesh->kind == ORC_MESH_EXTRUDED) return run_extruded(mesh, field, out);
  return 2;
}

void cporacle_free(orc_result* r) {
  free(r->simplices);
  free(r->bary);
  free(r->lambda);
  free(r->track_id);
  free(r->type);
  free(r->scalar);
  free(r->edges);
  free(r->cp_class);
  free(r->cells);
  memset(r, 0, sizeof(*r));
}

/* ------------------------------------------------------------------------ */
/* Primitive entry points, checked against the reference's unit-test vectors */

/* sos::sign (sos.hpp:12-20) */
int cporacle_sos_sign(double v, uint64_t index, double Q) {
  i128 q = quant(v, Q);
  if (q > 0) return 1;
  if (q < 0) return -1;
  return (index % 2 == 0) ? 1 : -1;
}

int cporacle_det2(const double* v0, const double* v1, uint64_t i0, uint64_t i1, double Q) {
  return sos_det2(v0, v1, i0, i1, Q);
}

int cporacle_det3(const double* v0, const double* v1, const double* v2, double Q) {
  return sos_det3(v0, v1, v2, Q);
}

/* origin_inside<M> on (M+1) x M values, row-major */
int cporacle_inside(int M, const double* vals, const uint64_t* idx, double Q) {
  double v[4][3];
  for (int i = 0; i <= M; ++i)
    for (int j = 0; j < M; ++j) v[i][j] = vals[i * M + j];
  return sos_inside(M, v, idx, Q);
}

/* ZeroCrossingSolver<K,T>::solve for K = 2, 3 in double (f64 != 0) or float */
int cporacle_solve(int K, int f64, const double* vals, double* lam) {
  if (f64) {
    double v[4][3], l[4];
    for (int i = 0; i <= K; ++i)
      for (int j = 0; j < K; ++j) v[i][j] = vals[i * K + j];
    int ok = solve_f64(K, v, l);
    for (int i = 0; i <= K; ++i) lam[i] = l[i];
    return ok;
  }
  float v[4][3], l[4];
  for (int i = 0; i <= K; ++i)
    for (int j = 0; j < K; ++j) v[i][j] = (float)vals[i * K + j];
  int ok = solve_f32(K, v, l);
  for (int i = 0; i <= K; ++i) lam[i] = l[i];
  return ok;
}

/* number of m-simplex types per d-hypercube (cpu_get_num_simplex_types) */
int cporacle_chain_count(int d, int m) {
  chains_t c;
  if (d < 1 || d > 4 || m < 1 || m > d) return 0;
  build_chains(&c, d, m);
  return c.n;
}

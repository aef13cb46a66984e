/*
 * ftk2b.h - C ABI of the B200-native critical-point tracking path.
 *
 * Drop-in replacement for the reference's
 *   SimplicialEngine<T, CriticalPointPredicate<M,T>>::execute() / execute_cuda()
 *   followed by get_complex()
 * (include/ftk2/core/engine.hpp:96-99, 273-282, 822-996), callable from any
 * language through plain pointers and sizes.  Every function returns a status
 * code; nothing throws or exits across this boundary, and there is no CPU
 * fallback: without a usable CUDA device the calls fail with FTK2B_NO_DEVICE.
 *
 * Results follow the reference's FeatureComplex (complex.hpp:14-58):
 * features in Simplex order (sorted vertex ids), float barycentrics as
 * FeatureElement stores them (feature.hpp:26), track_id = canonical id of the
 * smallest feature of the trajectory, type = 0 (predicate.hpp:80), and the
 * sorted, de-duplicated edge list of the trajectories.
 *
 * Threading: a context is used by one host thread at a time; create one
 * context per thread for concurrency.  All device work of a context runs on
 * its own CUDA stream.
 */
#ifndef FTK2B_H
#define FTK2B_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  FTK2B_OK = 0,
  FTK2B_INVALID_ARG = 1,     /* malformed descriptor (the reference throws or reads out of bounds) */
  FTK2B_OOM = 2,             /* device allocation failed */
  FTK2B_CUDA_ERROR = 3,      /* a CUDA call failed (the reference calls exit(), engine.hpp:29-37) */
  FTK2B_TIMEOUT = 4,         /* a bounded device-side wait gave up */
  FTK2B_OVERFLOW_RETRY = 5,  /* an output buffer overflowed and retries were exhausted */
  FTK2B_NO_DEVICE = 6,       /* no usable CUDA device: there is no CPU fallback */
  FTK2B_UNSUPPORTED = 7,     /* a combination the path does not implement */
  FTK2B_BUSY = 8,            /* the serving queue is full */
  FTK2B_INTERNAL = 9         /* a device self-check failed: a bounds check of the checked build (-DFTK2B_CHECKED) */
} ftk2b_status;

enum { FTK2B_MESH_REGULAR = 0, FTK2B_MESH_EXTRUDED = 1 };
enum { FTK2B_F32 = 0, FTK2B_F64 = 1 };
enum {
  FTK2B_LAYOUT_MULTICOMPONENT = 0, /* one [M, d0, d1, ...] array, component fastest (engine.hpp:1101-1124) */
  FTK2B_LAYOUT_SEPARATE = 1,       /* M arrays [d0, d1, ...] indexed by global - offset (engine.hpp:999-1009) */
  FTK2B_LAYOUT_PER_VERTEX = 2      /* M 1-D arrays indexed by vertex id (engine.hpp:1000) */
};
enum { FTK2B_HOST = 0, FTK2B_DEVICE = 1 };
enum {
  FTK2B_PRECISION_EXACT = 0,   /* solve in the field precision, operation for operation (zero_crossing.hpp:20-90) */
  FTK2B_PRECISION_REFINED = 1  /* same accepted set; reported lambda = FP32 solve + one FP64 refinement step */
};
enum {
  FTK2B_CLASS_NONE = 0,        /* classification not requested */
  FTK2B_CLASS_DEGENERATE = 1,
  FTK2B_CLASS_SOURCE = 2,      /* gradient fields: minimum */
  FTK2B_CLASS_SINK = 3,        /* gradient fields: maximum */
  FTK2B_CLASS_SADDLE = 4,
  FTK2B_CLASS_SPIRAL_SOURCE = 5,
  FTK2B_CLASS_SPIRAL_SINK = 6,
  FTK2B_CLASS_CENTER = 7
};

typedef struct ftk2b_ctx ftk2b_ctx;

/* Spacetime mesh.
 * REGULAR  = RegularSimplicialMesh(local_dims, offset, global_dims)
 *            (mesh.hpp:256-265); ndims counts time (3 = 2D+t, 4 = 3D+t).
 * EXTRUDED = ExtrudedSimplicialMesh(UnstructuredSimplicialMesh(cells), n_layers)
 *            (mesh.hpp:542-562, unstructured_mesh.hpp:16-76): base cells are
 *            triangles (base_cell_dim 2) or tets (3) over n_base_verts vertices. */
typedef struct {
  int kind;
  int ndims;
  uint64_t local_dims[4];
  uint64_t offset[4];
  uint64_t global_dims[4];
  uint64_t n_base_verts;
  const uint64_t* base_cells;  /* host memory, (base_cell_dim + 1) ids per cell */
  uint64_t n_base_cells;
  int base_cell_dim;
  uint64_t n_layers;
} ftk2b_mesh_desc;

/* Vector field (CriticalPointPredicate<M,T>, predicate.hpp:49-64).
 * MULTICOMPONENT: comp[0] = [M, d0, d1, ...] with nd = number of mesh dims.
 * SEPARATE:       comp[0..M-1] = [d0, d1, ...]; nd == 1 means per-vertex.
 * PER_VERTEX:     comp[0..M-1] of length dims[0].
 * scalar: optional scalar field, interpolated at features only for SEPARATE
 * layouts, as the reference does (predicate.hpp:81-92). */
typedef struct {
  int dtype;
  int ncomp;
  int layout;
  int location;       /* FTK2B_HOST or FTK2B_DEVICE (for every pointer below) */
  const void* comp[3];
  int nd;
  uint64_t dims[4];   /* Fortran order, first fastest, excluding the component dim */
  const void* scalar;
  int scalar_nd;
  uint64_t scalar_dims[4];
} ftk2b_field_desc;

typedef struct {
  double sos_q;       /* Predicate::sos_q, default 1e6 (predicate.hpp:25) */
  int precision;      /* FTK2B_PRECISION_* */
  int want_edges;     /* 1 (default): connectivity and track ids */
  int classify;       /* 1: fill cp_class from the Jacobian of the coface top cell */
} ftk2b_cp_params;

/* Result of one extraction; owned by the library until ftk2b_cp_result_free. */
typedef struct {
  int m;                  /* feature simplices have m+1 vertices */
  uint64_t n_features;
  uint64_t* simplices;    /* n*(m+1) sorted vertex ids */
  double* lambda;         /* n*(m+1) barycentrics (exact: field precision widened) */
  float* barycentric;     /* n*(m+1) as FeatureElement::barycentric_coords[0] */
  uint64_t* track_id;     /* n */
  uint32_t* type;         /* n, always 0 like the reference */
  uint32_t* cp_class;     /* n, FTK2B_CLASS_* */
  float* scalar;          /* n */
  uint64_t n_edges;
  uint32_t* edges;        /* 2*n_edges, (lo, hi) indices into the features */
  uint64_t n_tracks;
  uint64_t n_simplices;   /* m-simplices of the mesh: the unit of work */
  double device_ms;       /* device time of the extraction pipeline */
} ftk2b_cp_result;

/* --- context (replaces the engine object; engine.hpp:84-85) --------------- */
ftk2b_status ftk2b_ctx_create(int device, ftk2b_ctx** out);
void ftk2b_ctx_destroy(ftk2b_ctx* ctx);
const char* ftk2b_last_error(const ftk2b_ctx* ctx);
void* ftk2b_ctx_stream(ftk2b_ctx* ctx); /* the context's cudaStream_t */

ftk2b_cp_params ftk2b_cp_params_default(void);

/* Tuning knobs of a context (no reference counterpart: the reference sizes
 * its buffers with fixed guesses, engine.hpp:351-385). */
enum {
  FTK2B_OPT_FEATURE_CAPACITY = 1, /* initial feature capacity; grows on overflow */
  FTK2B_OPT_TIME_CHUNK = 2,       /* time steps per extraction block (0 = all) */
  FTK2B_OPT_DISABLE_TMA = 3,      /* 1: stage slices with plain loads instead of TMA */
  FTK2B_OPT_USE_GRAPHS = 4,       /* 1 (default): replay the device pipeline as a CUDA graph */
  FTK2B_OPT_BLOCKING_SYNC = 5,    /* 1: wait for the device by blocking, not spinning (servers set it) */
  FTK2B_OPT_CULL_MODE = 6,        /* 0: per-vertex cull words only; 1: tile statistics first; 2 (default):
                                     the faster of the two, timed once per workload shape by the context */
  FTK2B_OPT_TEST_STALL_POLLS = 8, /* > 0: failure-path check -- the regular-mesh cull blocks wait, at most
                                     this many polls, on an mbarrier nothing completes, so the call returns
                                     FTK2B_TIMEOUT with every copy landed; 0 (default): off */
  FTK2B_OPT_BATCH_TIME_CHUNK = 7  /* batches: corner time steps per cull item (0, default: chosen by the
                                     context, timed once per batch shape) */
};
ftk2b_status ftk2b_ctx_set_option(ftk2b_ctx* ctx, int option, int64_t value);
/* Reads an option back, or FTK2B_INFO_LAST_TMA: 1 when the last regular-mesh
 * extraction staged its slices with TMA tensor copies, or
 * FTK2B_INFO_LAST_CULL_MODE: the cull mode (0 or 1) it ran, or
 * FTK2B_INFO_LAST_BATCH_TIME_CHUNK: corner time steps per cull item of the
 * last batch (65535: each field's whole time range), or
 * FTK2B_INFO_LAST_CANDIDATES: hypercubes the last regular-mesh cull (one
 * field or a batch) kept for the exact test, or FTK2B_INFO_LAST_TESTED:
 * simplices of those hypercubes the exact test ran on. */
enum { FTK2B_INFO_LAST_TMA = 100, FTK2B_INFO_LAST_CULL_MODE = 101, FTK2B_INFO_LAST_BATCH_TIME_CHUNK = 102,
       FTK2B_INFO_LAST_CANDIDATES = 103, FTK2B_INFO_LAST_TESTED = 104 };
ftk2b_status ftk2b_ctx_get_option(ftk2b_ctx* ctx, int option, int64_t* value);

/* m-simplices a mesh holds for codimension m (2 or 3): the unit of work. */
uint64_t ftk2b_mesh_simplex_count(const ftk2b_mesh_desc* mesh, int m);

/* --- one-shot extraction: execute() + get_complex() ----------------------- */
/* Replaces SimplicialEngine::execute / execute_cuda (engine.hpp:96-99,
 * 273-282) plus get_complex (engine.hpp:822-996). */
ftk2b_status ftk2b_cp_extract(ftk2b_ctx* ctx, const ftk2b_mesh_desc* mesh,
                              const ftk2b_field_desc* field, const ftk2b_cp_params* params,
                              ftk2b_cp_result** out);
void ftk2b_cp_result_free(ftk2b_cp_result* r);

/* Two-step form of ftk2b_cp_extract: run leaves the results in the context's
 * device buffers (valid until the next call on the context); fetch copies
 * them to a host result.  Used to time the device pipeline alone. */
ftk2b_status ftk2b_cp_run(ftk2b_ctx* ctx, const ftk2b_mesh_desc* mesh,
                          const ftk2b_field_desc* field, const ftk2b_cp_params* params,
                          uint64_t* n_features, uint64_t* n_edges);
ftk2b_status ftk2b_cp_fetch(ftk2b_ctx* ctx, ftk2b_cp_result** out);

/* Device timing of the last run on the context's stream (CUDA events):
 * the fused extraction kernel alone and the whole pipeline, in ms, and the
 * number of kernels the context has launched so far. */
ftk2b_status ftk2b_ctx_last_timing(ftk2b_ctx* ctx, double* extract_ms, double* total_ms,
                                   uint64_t* kernels_launched);
/* Host time (ms) of the phases of the last regular-mesh extraction on the
 * context: [0] descriptors, staging copies and buffers, [1] CUDA-graph
 * capture and instantiation, [2] launch to device completion, [3] result
 * copy-back (ftk2b_cp_fetch). */
ftk2b_status ftk2b_ctx_last_phases(ftk2b_ctx* ctx, double* phase_ms);

/* --- attributes ------------------------------------------------------------
 * The values the reference records into FeatureElement::attributes for each
 * accepted simplex (AttributeSpec, predicate.hpp:34-40; engine.hpp:1143-1199),
 * computed on the device for the features of the last ftk2b_cp_run /
 * ftk2b_cp_extract on the context: sum over the feature's vertices of its
 * float barycentric times the array's value there, in the field's precision.
 *   COMPONENT: data is [ncomp, grid dims...]; value = component `component`
 *   MAGNITUDE: data is [ncomp, grid dims...]; value = Euclidean norm
 *   VALUE:     1-D data indexed by vertex id, else read at the vertex's grid
 *              coordinates minus the regular mesh's offset
 * (the reference picks COMPONENT / MAGNITUDE when the array's first dimension
 * is 1..16 and component >= 0 / type "magnitude", VALUE otherwise).  data has
 * the field's dtype; grid coordinates of extruded meshes need the spatial grid
 * (base_grid_dims) of an extruded regular grid, else only 1-D VALUE arrays.
 * out receives 16 floats per feature (slots not given stay 0). */
enum { FTK2B_ATTR_VALUE = 0, FTK2B_ATTR_COMPONENT = 1, FTK2B_ATTR_MAGNITUDE = 2 };
typedef struct {
  int kind;           /* FTK2B_ATTR_* */
  int component;      /* COMPONENT */
  int slot;           /* 0..15 */
  int location;       /* FTK2B_HOST or FTK2B_DEVICE */
  const void* data;
  int nd;
  uint64_t dims[6];   /* Fortran order, first fastest */
} ftk2b_attribute_desc;
ftk2b_status ftk2b_cp_attributes(ftk2b_ctx* ctx, const ftk2b_mesh_desc* mesh, const uint64_t* base_grid_dims,
                                 uint32_t n_attrs, const ftk2b_attribute_desc* attrs, float* out);

/* --- batches ---------------------------------------------------------------
 * No counterpart in the reference (one engine per field).  n independent
 * regular-mesh fields of uneven sizes, 2D and 3D mixed, extracted together:
 * one persistent cull launch walks every field's tiles, one launch runs the
 * exact tests of every candidate, and one canonical-order / star-edge /
 * union-find pipeline covers the whole batch, replayed as a CUDA graph for
 * batches of the same shape.  Field i's result is identical to
 * ftk2b_cp_extract on field i alone.
 * All fields share one dtype and either the multicomponent or the separate /
 * per-vertex layouts; params may be null (defaults) or hold n entries
 * (classify is not supported in batches). */
ftk2b_status ftk2b_cp_run_batch(ftk2b_ctx* ctx, uint32_t n, const ftk2b_mesh_desc* meshes,
                                const ftk2b_field_desc* fields, const ftk2b_cp_params* params,
                                uint64_t* n_features);
/* Copies the last batch's results out: out[0 .. n-1], one result per field,
 * each freed with ftk2b_cp_result_free. */
ftk2b_status ftk2b_cp_fetch_batch(ftk2b_ctx* ctx, ftk2b_cp_result** out);
ftk2b_status ftk2b_cp_extract_batch(ftk2b_ctx* ctx, uint32_t n, const ftk2b_mesh_desc* meshes,
                                    const ftk2b_field_desc* fields, const ftk2b_cp_params* params,
                                    ftk2b_cp_result** out);

/* --- time streams ----------------------------------------------------------
 * Replaces the reference's streaming drivers (SimplicialEngine::execute_stream
 * and execute_cuda_streaming_regular, engine.hpp:214-270, 601-819) with
 * one-shot semantics: after T pushes, ftk2b_stream_result returns exactly what
 * ftk2b_cp_extract returns for the T-timestep spacetime mesh.  Only the two
 * newest timesteps of the field, the features, their star edges and the
 * union-find state stay on the device; each push extracts the simplices whose
 * last layer is the new timestep and links them to the previous layer.
 *
 * mesh: REGULAR with ndims = spatial dims + 1 (the time entries are ignored)
 *       or EXTRUDED (n_layers is ignored).
 * tmpl: dtype, ncomp, layout, location and dims of ONE timestep
 *       (nd = spatial dims; per-vertex arrays for extruded meshes); no scalar.
 * A stream uses its context's stream and scratch buffers: do not interleave
 * calls on one context from several threads. */
typedef struct ftk2b_stream ftk2b_stream;
ftk2b_status ftk2b_stream_open(ftk2b_ctx* ctx, const ftk2b_mesh_desc* mesh, const ftk2b_field_desc* tmpl,
                               const ftk2b_cp_params* params, ftk2b_stream** out);
/* Pushes the next timestep (same dtype / layout / dims as the template);
 * *n_new receives the number of features whose last layer is this timestep. */
ftk2b_status ftk2b_stream_push(ftk2b_stream* s, const ftk2b_field_desc* step, uint64_t* n_new);
/* The complex of every timestep pushed so far (get_complex, engine.hpp:822-996). */
ftk2b_status ftk2b_stream_result(ftk2b_stream* s, ftk2b_cp_result** out);
ftk2b_status ftk2b_stream_info(ftk2b_stream* s, uint64_t* timesteps, uint64_t* n_features, double* last_push_ms);
void ftk2b_stream_close(ftk2b_stream* s);
/* Checkpoint and resume (no reference counterpart: the reference's streaming
 * drivers keep their state in one process).  ftk2b_stream_checkpoint writes
 * everything later pushes and results read -- the configuration, the two
 * newest timesteps, the features, star edges, union-find parents and the
 * newest layer's ids -- to host memory: with buf = NULL it only stores the
 * size needed in *bytes; with a buffer of *bytes bytes it writes the blob
 * (FTK2B_INVALID_ARG, and the size in *bytes, when the buffer is too small).
 * ftk2b_stream_restore opens a stream on ctx (any device) from such a blob;
 * pushing the remaining timesteps to it gives what the original stream would
 * have given.  The blob is checked (magic, version, configuration, sizes)
 * before anything is allocated. */
ftk2b_status ftk2b_stream_checkpoint(ftk2b_stream* s, void* buf, uint64_t* bytes);
ftk2b_status ftk2b_stream_restore(ftk2b_ctx* ctx, const void* buf, uint64_t bytes, ftk2b_stream** out);

/* --- serving ----------------------------------------------------------------
 * No counterpart in the reference (it has no request loop).  A server owns
 * n_slots worker threads, each with its own context (device buffers and CUDA
 * stream), so the device work of concurrent requests overlaps.  Requests are
 * admitted in arrival order as soon as a worker is free and their estimated
 * device memory fits the HBM budget (continuous batching: requests that
 * arrive while others run start as slots and memory free up).  Pushes to one
 * stream run in submission order, on the stream's own context, which keeps
 * the stream's previous timestep and union-find state resident.
 * Every pointer inside a request must stay valid until the request completes. */
typedef struct ftk2b_server ftk2b_server;
enum { FTK2B_REQ_EXTRACT = 0, FTK2B_REQ_STREAM_PUSH = 1 };
typedef struct {
  int kind;                 /* FTK2B_REQ_* */
  ftk2b_mesh_desc mesh;     /* EXTRACT */
  ftk2b_field_desc field;   /* EXTRACT: the field; STREAM_PUSH: one timestep */
  ftk2b_cp_params params;   /* EXTRACT */
  uint64_t stream;          /* STREAM_PUSH: id from ftk2b_server_stream_open */
} ftk2b_request;
typedef struct {
  ftk2b_status status;
  int slot;                 /* worker that ran it */
  double queue_ms;          /* submit -> start */
  double run_ms;            /* start -> done */
  double latency_ms;        /* submit -> done */
  uint64_t n_features;      /* EXTRACT: features; STREAM_PUSH: new features */
  uint64_t n_simplices;     /* EXTRACT: m-simplices of the mesh */
  double phase_ms[4];       /* EXTRACT on a regular mesh: ftk2b_ctx_last_phases */
} ftk2b_request_stats;
typedef struct {
  uint64_t submitted, completed, failed, rejected;
  double p50_ms, p99_ms, max_ms, mean_ms;  /* latency of completed requests */
  double elapsed_s;                        /* first submit -> last completion */
  uint64_t simplices;                      /* m-simplices of completed extractions */
  uint64_t hbm_budget, hbm_reserved_peak;  /* bytes */
  int max_in_flight;
} ftk2b_server_stats;

/* hbm_budget = 0: 90% of the device's free memory at creation.
 * queue_limit = 0: unbounded; otherwise submit returns FTK2B_BUSY when full.
 * The server's contexts allocate in stream order from the device's default
 * memory pool; creation sets that pool to keep freed memory mapped and maps
 * min(hbm_budget / 2, n_slots GiB) up front, so that buffers growing during
 * serving do not map new memory (which would hold up every slot). */
ftk2b_status ftk2b_server_create(int device, int n_slots, uint64_t hbm_budget, int queue_limit,
                                 ftk2b_server** out);
ftk2b_status ftk2b_server_stream_open(ftk2b_server* sv, const ftk2b_mesh_desc* mesh, const ftk2b_field_desc* tmpl,
                                      const ftk2b_cp_params* params, uint64_t* stream_id);
ftk2b_status ftk2b_server_submit(ftk2b_server* sv, const ftk2b_request* req, uint64_t* ticket);
/* Runs an extraction request once on every worker slot and waits: the slots'
 * buffers and cached pipeline graphs then fit requests of that shape, so
 * serving traffic does not pay for first-time set-up.  Not counted in the
 * statistics. */
ftk2b_status ftk2b_server_warm(ftk2b_server* sv, const ftk2b_request* req);
/* Blocks until the request is done (timeout_s < 0: no limit; FTK2B_TIMEOUT
 * otherwise).  *out (may be null) receives an EXTRACT's result, owned by the
 * caller (ftk2b_cp_result_free).  Returns the request's own status. */
ftk2b_status ftk2b_server_wait(ftk2b_server* sv, uint64_t ticket, double timeout_s, ftk2b_cp_result** out,
                               ftk2b_request_stats* stats);
ftk2b_status ftk2b_server_stream_result(ftk2b_server* sv, uint64_t stream_id, ftk2b_cp_result** out);
ftk2b_status ftk2b_server_stream_close(ftk2b_server* sv, uint64_t stream_id);
ftk2b_status ftk2b_server_get_stats(ftk2b_server* sv, ftk2b_server_stats* out);
/* text of the last failure of a server call or request */
const char* ftk2b_server_last_error(ftk2b_server* sv);
void ftk2b_server_destroy(ftk2b_server* sv);

/* --- allocation-free extraction -------------------------------------------
 * No counterpart in the reference.  For callers that may not allocate device
 * memory while they run: an in-situ step inside a simulation whose memory
 * manager owns the whole device, or a serving loop held to a fixed memory
 * budget that cannot absorb cudaMalloc's implicit synchronisation.  It runs
 * the fused regular-mesh extraction on `stream` and writes the accepted
 * simplices, unsorted, to caller-provided device memory: canonical keys
 * (corner vertex id * n_types + chain rank) and 4 doubles of barycentrics per
 * feature; `count` is a device word the call uses as its atomic counter, and
 * *n_features receives the number found.  Field pointers must be device
 * pointers.  Scratch is a static device array of ~9.3 MiB that every GPU
 * loading the library holds until exit.  Limits: capacity <= 262144 features
 * (FTK2B_INVALID_ARG beyond it); more features than `capacity` returns
 * FTK2B_OVERFLOW_RETRY with the count found (retry with a larger output);
 * more than 262144 surviving hypercubes returns FTK2B_UNSUPPORTED (no retry
 * can succeed: split the box into sub-boxes).  The first call on a device
 * looks up the array's device address and uploads the kernels' constant
 * tables; make that first call before any stream capture.  Calls share the
 * array, so calls whose device work overlaps race.  The call waits for
 * `stream` before returning. */
ftk2b_status ftk2b_cp_features_noalloc(const ftk2b_mesh_desc* mesh, const ftk2b_field_desc* field,
                                       double sos_q, void* stream, uint64_t* keys, double* lambda,
                                       uint32_t capacity, uint32_t* count, uint64_t* n_features);

/* --- level sets (ContourPredicate<T>) -------------------------------------
 * Replaces SimplicialEngine<T, ContourPredicate<T>>::execute + get_complex
 * (engine.hpp:95-215, 822-996; predicate.hpp:135-183) on a regular mesh of
 * 3 (2D+t) or 4 (3D+t) dims, or on an extruded mesh over triangles or tets
 * (ExtrudedSimplicialMesh, mesh.hpp:542-599).  field: ncomp 1, layout
 * SEPARATE, comp[0] the scalar array (regular: nd == mesh dims, indexed by
 * local coordinates, or nd 1 indexed by global vertex id; extruded: nd 1,
 * one value per vertex id s + t * n_base_verts).  Features are the mesh edges whose endpoints
 * have different simulation-of-simplicity signs of value - threshold, in
 * simplex order; cells are the manifold cells of get_complex (triangles on
 * 2D+t, tets on 3D+t) as sorted rows of feature indices, sorted and unique;
 * track ids are the components' smallest feature index.  Where the reference
 * numbers nodes in the order its patching meets them (2D+t quads cut along
 * the diagonal from their first node), this follows its sequential order. */
typedef struct {
  uint64_t n_features;
  uint64_t* simplices;    /* 2 per feature: the edge's vertex ids, ascending */
  double* lambda;         /* 2 per feature: the barycentrics in the field precision, widened */
  float* barycentric;     /* 2 per feature, as FeatureElement::barycentric_coords[0] */
  uint64_t* track_id;     /* n */
  float* scalar;          /* n: the threshold as float */
  int cell_dim;           /* 2 (triangles, 2D+t) or 3 (tets, 3D+t) */
  uint64_t n_cells;
  uint32_t* cells;        /* (cell_dim + 1) per cell */
  uint64_t n_tracks;
  uint64_t n_simplices;   /* edges of the mesh: the unit of work */
  double device_ms;       /* device time of the pipeline */
} ftk2b_contour_result;
ftk2b_status ftk2b_contour_extract(ftk2b_ctx* ctx, const ftk2b_mesh_desc* mesh, const ftk2b_field_desc* field,
                                   double threshold, double sos_q, ftk2b_contour_result** out);
void ftk2b_contour_result_free(ftk2b_contour_result* r);

/* --- fibers (FiberPredicate<T>) --------------------------------------------
 * Replaces SimplicialEngine<T, FiberPredicate<T>>::execute + get_complex
 * (predicate.hpp:341-362; form_general_manifold_patches engine.hpp:1341-1418)
 * on a 2D+t mesh (ndims 3: regular, or extruded over triangles with
 * per-vertex fields): features are the triangles where both
 * fields minus their thresholds vanish (simulation of simplicity), kept at the
 * centroid where the barycentric solve fails; edges join each top cell's
 * features to its star centre.  field: ncomp 2 (SEPARATE, MULTICOMPONENT or
 * PER_VERTEX layout as for critical points).  The result is a cp_result with
 * m = 2, type 0 and scalar 0.  3D+t meshes (fiber surfaces): use
 * ftk2b_fiber_surface_extract. */
ftk2b_status ftk2b_fiber_extract(ftk2b_ctx* ctx, const ftk2b_mesh_desc* mesh, const ftk2b_field_desc* field,
                                 const double thresholds[2], double sos_q, ftk2b_cp_result** out);

/* Fiber surfaces: SimplicialEngine<T, FiberPredicate<T>>::execute +
 * get_complex on a regular 3D+t mesh (ndims 4), or on an ExtrudedSimplicialMesh
 * over tets (base_cell_dim 3; mesh.hpp:542-712).  field: ncomp 2, layout
 * SEPARATE (regular: nd 4, indexed by local coordinates, or nd 1 by global
 * vertex id; extruded: nd 1 per vertex id, or PER_VERTEX).  On extruded meshes
 * the triangles inside the prisms over base triangles are ordered as the
 * reference's patching meets them when it runs on one worker (with several
 * workers it numbers them in thread-arrival order).
 * Features are the triangles of the 4-D mesh, in simplex order, with their
 * barycentrics (centroid where the solve fails); cells are the star-fan
 * triangles of form_general_manifold_patches (engine.hpp:1388-1413) as sorted,
 * unique rows of feature indices; track ids are the components' smallest
 * feature index. */
typedef struct {
  uint64_t n_features;
  uint64_t* simplices;    /* 3 per feature: vertex ids, ascending */
  double* lambda;         /* 3 per feature, the field precision widened */
  float* barycentric;     /* 3 per feature, as FeatureElement stores them */
  uint64_t* track_id;     /* n */
  float* scalar;          /* n: 0 */
  uint64_t n_cells;
  uint32_t* cells;        /* 3 per cell */
  uint64_t n_tracks;
  uint64_t n_simplices;   /* triangles of the mesh: the unit of work */
  double device_ms;
} ftk2b_fiber_surface_result;
ftk2b_status ftk2b_fiber_surface_extract(ftk2b_ctx* ctx, const ftk2b_mesh_desc* mesh,
                                         const ftk2b_field_desc* field, const double thresholds[2], double sos_q,
                                         ftk2b_fiber_surface_result** out);
void ftk2b_fiber_surface_result_free(ftk2b_fiber_surface_result* r);

#ifdef __cplusplus
}
#endif

#endif /* FTK2B_H */

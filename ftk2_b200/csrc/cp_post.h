// Device buffers and launchers of the post-extraction stages.
#pragma once

#include "cp_internal.h"

namespace ftk2b {

// Feature capacities up to this run the short post-extraction chain (rank
// sort, star edges, one-block union-find); larger ones the radix-sort chain.
constexpr unsigned kSmallPostCap = 16384;

struct PostBuffers {
  unsigned cap;                     // feature capacity
  int num_sms;
  unsigned edge_cap;
  int key_bits;                     // significant bits of the canonical keys
  int sort_grid;
  // extraction output (unsorted)
  unsigned long long* key;
  double* lam;                      // 4 per feature
  float* bary4;                     // 4 per feature: (float) of the exact-path lambda
  float* scalar;
  unsigned* count;                  // device count of features
  // sort scratch
  unsigned long long* key_alt;
  unsigned* perm0;
  unsigned* perm1;
  unsigned* hist;                   // 256 * sort_grid
  // canonical-order outputs
  double* lam_sorted;
  float* bary4_sorted;
  float* scalar_sorted;
  unsigned long long* simplices;    // (m+1) per feature
  float* bary;                      // (m+1) per feature
  unsigned long long* track;
  unsigned* edge_cnt;               // per feature, scanned in place into offsets
  unsigned* edges;                  // 2 per edge
  unsigned* edge_slots;             // 8 per feature: star edges before compaction
  unsigned* n_edges;
  unsigned* parent;
  unsigned* n_roots;
  unsigned* err;
  unsigned* done;                   // short chain: edge-kernel blocks finished (zeroed per call)
  unsigned* cls;                    // per feature classification (FTK2B_CLASS_*)
};

void upload_post_tables();
cudaError_t launch_post_regular(const RegularMesh& mesh, int nch, const PostBuffers& B,
                                int want_edges, cudaStream_t st, unsigned long long* launches);
cudaError_t launch_classify_regular(int f64, const RegularMesh& mesh, const FieldAccess& fa, int nch,
                                    const PostBuffers& B, cudaStream_t st);
cudaError_t launch_iota(unsigned* v, const unsigned* n_ptr, unsigned cap, cudaStream_t st);
// exclusive scan in place of min(total, *n_ptr) counters (n_ptr may be null);
// the sum lands in *total_out when it is not null
cudaError_t launch_scan(unsigned* a, unsigned total, unsigned* total_out, const unsigned* n_ptr,
                        cudaStream_t st);
// union-find: parent[i] = i, then the edges' endpoints united
cudaError_t launch_uf(unsigned* parent, const unsigned* n_ptr, unsigned cap, const unsigned* edges,
                      const unsigned* ne_ptr, unsigned edge_cap, unsigned* err, cudaStream_t st);
// track[i] = root of i (the component's smallest index), roots counted
cudaError_t launch_uf_label(unsigned* parent, const unsigned* n_ptr, unsigned cap,
                            unsigned long long* track, unsigned* n_roots, cudaStream_t st);
// star edges of the top cells of `mesh` (a window of the full mesh) among the
// sorted keys, as (centre, other) index pairs, sorted; count in *n_edges
cudaError_t launch_window_edges_regular(const RegularMesh& mesh, int nch, const unsigned long long* skeys,
                                        const unsigned* n_ptr, unsigned cap, unsigned* edge_cnt,
                                        unsigned* edge_slots, unsigned* edges, unsigned* n_edges,
                                        unsigned edge_cap, cudaStream_t st);
// vertex ids (and, when bary is not null, float barycentrics) of keys
cudaError_t launch_expand_regular(const RegularMesh& mesh, int nch, const unsigned long long* keys,
                                  const unsigned* n_ptr, unsigned cap, const float* bary4,
                                  unsigned long long* simplices, float* bary, cudaStream_t st);
struct BatchMesh;
// Post-extraction stages of a batch: canonical order over the batch's key
// space (kb[f] = first key of field f, ascending, kb[nf] = end), star edges
// and trajectories (which never cross fields), vertex ids in rows of 4, and
// fbase[f] = first feature of field f (f = 0 .. nf).
cudaError_t launch_post_batch(const BatchMesh* fm, const unsigned long long* kb, int nf, const PostBuffers& B,
                              unsigned* fbase, cudaStream_t st, unsigned long long* launches);
bool radix_sort(unsigned long long* k0, unsigned* v0, unsigned long long* k1, unsigned* v1,
                const unsigned* n_ptr, unsigned cap, int bits, unsigned* hist, int grid,
                cudaStream_t st, unsigned long long* launches);

}  // namespace ftk2b

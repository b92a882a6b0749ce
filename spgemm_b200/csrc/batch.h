// Batched products: many independent C_i = A_i * B_i run as one product of
// block-diagonal operands, so every bin kernel of the pipeline serves all
// products in a single launch; the whole pipeline can be recorded once in a
// CUDA graph and replayed for new values in the same arrays.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "../../include/cm.h"
#include "engine.h"

namespace sg {

// One operand array set to copy into the packed operand: ptr[0..len] (+ the
// nnz offset), idx[0..nnz) (+ idx_add), val[0..nnz).
struct PackSeg {
  const int* ptr;
  const int* idx;
  const float* val;
  long long ptr_out;  // first packed pointer entry
  long long nnz_out;  // first packed entry
  int len;            // pointer entries without the final one
  int nnz;
  int idx_add;        // index offset of this product inside the packed operand
  int last;           // the last product also writes the final pointer entry
};

class Batch {
 public:
  ~Batch();
  // Packs the operands (device arrays; every A_i CSR, or every A_i CSC; B_i
  // CSR), runs the whole multiply once with host synchronisation and keeps
  // its sizes. Replaces the handle's current product.
  int plan(Engine& E, int count, const cm* A, const cm* B, long long* nnz_total);
  // Recomputes every product from the current contents of the planned
  // arrays (same structure, any values): as one CUDA graph launch when
  // use_graph (recorded on first use), else as direct launches. One host
  // synchronisation at the end.
  int execute(Engine& E, int use_graph);
  int offsets(Engine& E, long long* row_off, long long* nnz_off) const;
  int result(Engine& E, int i, cm* C) const;
  int copy_result(Engine& E, int i, int* rowptr, int* col, float* val) const;
  // The whole packed output (per-product row pointers back to back, then all
  // columns and values) in three copies.
  int copy_all(Engine& E, int* rowptr, int* col, float* val) const;

 private:
  int run(Engine& E);  // pack + analysis + symbolic + numeric on E's stream
  void drop_graph();

  int count_ = 0;
  bool planned_ = false;
  long long epoch_ = -1;  // engine epoch of the plan
  cm A_bd_{}, B_bd_{};
  int a_segs_len_max_ = 0, a_segs_nnz_max_ = 0, b_segs_len_max_ = 0, b_segs_nnz_max_ = 0;
  long long max_rows_ = 0, nnz_total_ = 0;
  std::vector<long long> row_off_, nnz_off_;
  std::vector<int> m_, n_;
  DevBuf segs_, a_ptr_, a_idx_, a_val_, b_ptr_, b_idx_, b_val_, row_off_dev_, nnz_off_dev_;
  DevBuf out_rowptr_, out_col_, out_val_;
  cudaGraph_t graph_ = nullptr;
  cudaGraphExec_t exec_ = nullptr;
  long long graph_launches_ = 0;
  cudaStream_t own_stream_ = nullptr;
};

}  // namespace sg

// Batched products on one engine (see batch.h).
//
// Packing: A_bd is block diagonal (product i's rows after those of products
// < i, its k-range after theirs); B_bd stacks the B_i vertically with their
// own column indices. Row r of product i then only meets B_i's rows, so C_bd
// holds every C_i with C_i's own column indices and no unpacking is needed:
// C_i is the row range of product i, with row pointers rebased per product.
#include "batch.h"

#include <algorithm>
#include <string>

#include "../../include/spgemm_b200.h"

namespace sg {
namespace {

constexpr long long I32_MAX = 2147483647ll;

// Copy one product's arrays (blockIdx.y) into the packed operand.
__global__ void __launch_bounds__(256)
k_pack(const PackSeg* __restrict__ segs, int* __restrict__ ptr_out, int* __restrict__ idx_out,
       float* __restrict__ val_out) {
  const PackSeg s = segs[blockIdx.y];
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int add = (int)s.nnz_out;
  for (long long j = t0; j < s.len; j += stride) ptr_out[s.ptr_out + j] = s.ptr[j] + add;
  if (s.last && t0 == 0) ptr_out[s.ptr_out + s.len] = s.ptr[s.len] + add;
  for (long long j = t0; j < s.nnz; j += stride) {
    idx_out[s.nnz_out + j] = s.idx[j] + s.idx_add;
    val_out[s.nnz_out + j] = s.val[j];
  }
}

// nnz_off[p] = first entry of product p in C_bd, p = 0..count.
__global__ void k_batch_nnz_off(const long long* __restrict__ rowptr64,
                                const long long* __restrict__ row_off, int count,
                                long long* __restrict__ nnz_off) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p <= count; p += gridDim.x * blockDim.x)
    nnz_off[p] = rowptr64[row_off[p]];
}

int grid_x(long long work) {
  long long b = (work + 255) / 256;
  return (int)std::max(1ll, std::min(b, 64ll));
}

}  // namespace

Batch::~Batch() {
  drop_graph();
  DevBuf* all[] = {&segs_, &a_ptr_, &a_idx_, &a_val_, &b_ptr_, &b_idx_, &b_val_,
                   &row_off_dev_, &nnz_off_dev_, &out_rowptr_, &out_col_, &out_val_};
  for (DevBuf* b : all) b->release();
  if (own_stream_) cudaStreamDestroy(own_stream_);
}

void Batch::drop_graph() {
  if (exec_) cudaGraphExecDestroy(exec_);
  if (graph_) cudaGraphDestroy(graph_);
  exec_ = nullptr;
  graph_ = nullptr;
  graph_launches_ = 0;
}

int Batch::run(Engine& E) {
  cudaStream_t s = E.stream();
  {
    const dim3 ga(grid_x(std::max(a_segs_len_max_, a_segs_nnz_max_)), count_);
    E.prof_begin("k_pack");
    k_pack<<<ga, 256, 0, s>>>(segs_.as<PackSeg>(), a_ptr_.as<int>(), a_idx_.as<int>(),
                              a_val_.as<float>());
    E.prof_end();
    const dim3 gb(grid_x(std::max(b_segs_len_max_, b_segs_nnz_max_)), count_);
    E.prof_begin("k_pack");
    k_pack<<<gb, 256, 0, s>>>(segs_.as<PackSeg>() + count_, b_ptr_.as<int>(), b_idx_.as<int>(),
                              b_val_.as<float>());
    E.prof_end();
    E.add_launches(2);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return E.cuda_fail(e, "k_pack");
  }
  if (int r = E.analyze(A_bd_, B_bd_)) return r;
  long long nnz = 0;
  if (int r = E.symbolic_pass(&nnz)) return r;
  if (!E.replay()) {
    nnz_total_ = E.nnz_c();
    cudaError_t e = out_rowptr_.ensure(sizeof(int) * (size_t)(A_bd_.num_rows + count_));
    if (e == cudaSuccess) e = out_col_.ensure(sizeof(int) * (size_t)std::max(nnz_total_, 1ll));
    if (e == cudaSuccess) e = out_val_.ensure(sizeof(float) * (size_t)std::max(nnz_total_, 1ll));
    if (e != cudaSuccess) return E.cuda_fail(e, "alloc batch output");
  }
  return E.numeric_batch(count_, row_off_dev_.as<long long>(), max_rows_, out_rowptr_.as<int>(),
                         out_col_.as<int>(), out_val_.as<float>());
}

int Batch::plan(Engine& E, int count, const cm* A, const cm* B, long long* nnz_total) {
  planned_ = false;
  drop_graph();
  if (count < 1 || count > 65535 || !A || !B)
    return E.fail(SPGEMM_ERR_INVALID, "batch: 1 <= count <= 65535 and operand arrays required");
  const bool a_csc = A[0].type == COL_MAJOR;
  long long rows = 0, kk = 0, nnz_a = 0, nnz_b = 0;
  int n_max = 0;
  std::vector<PackSeg> segs(2 * (size_t)count);
  row_off_.assign(count + 1, 0);
  m_.assign(count, 0);
  n_.assign(count, 0);
  a_segs_len_max_ = a_segs_nnz_max_ = b_segs_len_max_ = b_segs_nnz_max_ = 0;
  max_rows_ = 0;
  for (int i = 0; i < count; ++i) {
    const cm& a = A[i];
    const cm& b = B[i];
    const std::string at = "batch product " + std::to_string(i) + ": ";
    if ((a.type == COL_MAJOR) != a_csc) return E.fail(SPGEMM_ERR_INVALID, at + "mixed A formats");
    if (b.type != ROW_MAJOR) return E.fail(SPGEMM_ERR_INVALID, at + "B must be CSR");
    if (a.num_rows < 0 || a.num_cols < 0 || b.num_cols < 0 || a.nnz < 0 || b.nnz < 0)
      return E.fail(SPGEMM_ERR_INVALID, at + "negative dimension or nnz");
    if (a.num_cols != b.num_rows) return E.fail(SPGEMM_ERR_INVALID, at + "A.num_cols != B.num_rows");
    if (!a.ptr || !b.ptr || (a.nnz > 0 && (!a.idx || !a.val)) || (b.nnz > 0 && (!b.idx || !b.val)))
      return E.fail(SPGEMM_ERR_INVALID, at + "null array");
    const int m = a.num_rows, k = a.num_cols;
    m_[i] = m;
    n_[i] = b.num_cols;
    PackSeg& sa = segs[i];
    sa = PackSeg{a.ptr, a.idx, a.val, a_csc ? kk : rows, nnz_a, a_csc ? k : m, a.nnz,
                 (int)(a_csc ? rows : kk), i == count - 1};
    PackSeg& sb = segs[count + i];
    sb = PackSeg{b.ptr, b.idx, b.val, kk, nnz_b, k, b.nnz, 0, i == count - 1};
    a_segs_len_max_ = std::max(a_segs_len_max_, sa.len);
    a_segs_nnz_max_ = std::max(a_segs_nnz_max_, sa.nnz);
    b_segs_len_max_ = std::max(b_segs_len_max_, sb.len);
    b_segs_nnz_max_ = std::max(b_segs_nnz_max_, sb.nnz);
    max_rows_ = std::max<long long>(max_rows_, m);
    rows += m;
    kk += k;
    nnz_a += a.nnz;
    nnz_b += b.nnz;
    n_max = std::max(n_max, b.num_cols);
    row_off_[i + 1] = rows;
    if (rows >= I32_MAX || kk >= I32_MAX || nnz_a > I32_MAX || nnz_b > I32_MAX)
      return E.fail(SPGEMM_ERR_TOO_LARGE, "batch: packed operands exceed the int32 range");
  }
  count_ = count;
  const size_t a_len = (size_t)(a_csc ? kk : rows) + 1;
  cudaError_t e = segs_.ensure(sizeof(PackSeg) * segs.size());
  if (e == cudaSuccess) e = a_ptr_.ensure(sizeof(int) * a_len);
  if (e == cudaSuccess) e = a_idx_.ensure(sizeof(int) * (size_t)std::max(nnz_a, 1ll));
  if (e == cudaSuccess) e = a_val_.ensure(sizeof(float) * (size_t)std::max(nnz_a, 1ll));
  if (e == cudaSuccess) e = b_ptr_.ensure(sizeof(int) * ((size_t)kk + 1));
  if (e == cudaSuccess) e = b_idx_.ensure(sizeof(int) * (size_t)std::max(nnz_b, 1ll));
  if (e == cudaSuccess) e = b_val_.ensure(sizeof(float) * (size_t)std::max(nnz_b, 1ll));
  if (e == cudaSuccess) e = row_off_dev_.ensure(sizeof(long long) * (size_t)(count + 1));
  if (e == cudaSuccess) e = nnz_off_dev_.ensure(sizeof(long long) * (size_t)(count + 1));
  if (e != cudaSuccess) return E.cuda_fail(e, "alloc batch operands");
  cudaStream_t s = E.stream();
  e = cudaMemcpyAsync(segs_.ptr, segs.data(), sizeof(PackSeg) * segs.size(),
                      cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(row_off_dev_.ptr, row_off_.data(), sizeof(long long) * (count + 1),
                        cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return E.cuda_fail(e, "copy batch plan");
  A_bd_ = cm{a_ptr_.as<int>(), a_idx_.as<int>(), a_val_.as<float>(), (int)nnz_a, (int)rows,
             (int)kk, a_csc ? (bool)COL_MAJOR : (bool)ROW_MAJOR};
  B_bd_ = cm{b_ptr_.as<int>(), b_idx_.as<int>(), b_val_.as<float>(), (int)nnz_b, (int)kk, n_max,
             (bool)ROW_MAJOR};

  E.set_replay(false);
  E.set_batch_output(true);
  int r = run(E);
  E.set_batch_output(false);
  if (r) return r;
  k_batch_nnz_off<<<(count + 256) / 256, 256, 0, s>>>(E.rowptr64(), row_off_dev_.as<long long>(),
                                                      count, nnz_off_dev_.as<long long>());
  E.add_launches(1);
  nnz_off_.assign(count + 1, 0);
  e = cudaMemcpyAsync(nnz_off_.data(), nnz_off_dev_.ptr, sizeof(long long) * (count + 1),
                      cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return E.cuda_fail(e, "read batch offsets");
  for (int i = 0; i < count; ++i)
    if (nnz_off_[i + 1] - nnz_off_[i] > I32_MAX)
      return E.fail(SPGEMM_ERR_OVERFLOW, "batch product " + std::to_string(i) +
                                             ": nnz(C) exceeds the int32 range of cm");
  epoch_ = E.epoch();
  planned_ = true;
  if (nnz_total) *nnz_total = nnz_total_;
  return SPGEMM_OK;
}

int Batch::execute(Engine& E, int use_graph) {
  if (!planned_ || E.epoch() != epoch_)
    return E.fail(SPGEMM_ERR_STATE, "batch: no current plan (plan again after other products)");
  cudaStream_t user = E.stream();
  if (!user && use_graph) {  // stream capture needs a stream other than the legacy default
    if (!own_stream_) {
      cudaError_t e = cudaStreamCreateWithFlags(&own_stream_, cudaStreamNonBlocking);
      if (e != cudaSuccess) return E.cuda_fail(e, "create batch stream");
    }
    E.set_stream(own_stream_);
  }
  cudaStream_t s = E.stream();
  E.set_replay(true);
  E.set_batch_output(true);
  int r = 0;
  if (use_graph) {
    if (!exec_) {
      const bool prof = E.profiling();
      E.set_profiling(false);  // no timing events inside the recorded graph
      const long long before = E.launches();
      cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
      if (e != cudaSuccess) {
        r = E.cuda_fail(e, "begin batch capture");
      } else {
        r = run(E);
        cudaGraph_t g = nullptr;
        e = cudaStreamEndCapture(s, &g);
        if (!r && e != cudaSuccess) r = E.cuda_fail(e, "end batch capture");
        if (!r) {
          e = cudaGraphInstantiate(&exec_, g, 0);
          if (e != cudaSuccess) r = E.cuda_fail(e, "instantiate batch graph");
        }
        if (r) {
          if (g) cudaGraphDestroy(g);
          exec_ = nullptr;
        } else {
          graph_ = g;
          graph_launches_ = E.launches() - before;
          E.add_launches(-graph_launches_);  // counted when the graph runs
        }
      }
      E.set_profiling(prof);
    }
    if (!r) {
      cudaError_t e = cudaGraphLaunch(exec_, s);
      if (e != cudaSuccess) r = E.cuda_fail(e, "launch batch graph");
      else E.add_launches(graph_launches_);
    }
  } else {
    r = run(E);
  }
  unsigned st = 0;
  if (!r) r = E.read_status(&st);
  E.set_replay(false);
  E.set_batch_output(false);
  if (!user && use_graph) E.set_stream(user);
  return r;
}

int Batch::offsets(Engine& E, long long* row_off, long long* nnz_off) const {
  if (!planned_) return E.fail(SPGEMM_ERR_STATE, "batch: no plan");
  for (int i = 0; i <= count_; ++i) {
    if (row_off) row_off[i] = row_off_[i];
    if (nnz_off) nnz_off[i] = nnz_off_[i];
  }
  return SPGEMM_OK;
}

int Batch::result(Engine& E, int i, cm* C) const {
  if (!planned_) return E.fail(SPGEMM_ERR_STATE, "batch: no plan");
  if (i < 0 || i >= count_ || !C) return E.fail(SPGEMM_ERR_INVALID, "batch: product index");
  C->ptr = out_rowptr_.as<int>() + row_off_[i] + i;
  C->idx = out_col_.as<int>() + nnz_off_[i];
  C->val = out_val_.as<float>() + nnz_off_[i];
  C->nnz = (int)(nnz_off_[i + 1] - nnz_off_[i]);
  C->num_rows = m_[i];
  C->num_cols = n_[i];
  C->type = ROW_MAJOR;
  return SPGEMM_OK;
}

int Batch::copy_result(Engine& E, int i, int* rowptr, int* col, float* val) const {
  cm C;
  if (int r = result(E, i, &C)) return r;
  if (!rowptr || (C.nnz > 0 && (!col || !val))) return E.fail(SPGEMM_ERR_INVALID, "null host array");
  cudaStream_t s = E.stream();
  cudaError_t e = cudaMemcpyAsync(rowptr, C.ptr, sizeof(int) * ((size_t)C.num_rows + 1),
                                  cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && C.nnz > 0)
    e = cudaMemcpyAsync(col, C.idx, sizeof(int) * (size_t)C.nnz, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && C.nnz > 0)
    e = cudaMemcpyAsync(val, C.val, sizeof(float) * (size_t)C.nnz, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return E.cuda_fail(e, "copy batch result");
  return SPGEMM_OK;
}

int Batch::copy_all(Engine& E, int* rowptr, int* col, float* val) const {
  if (!planned_) return E.fail(SPGEMM_ERR_STATE, "batch: no plan");
  if (!rowptr || (nnz_total_ > 0 && (!col || !val)))
    return E.fail(SPGEMM_ERR_INVALID, "null host array");
  cudaStream_t s = E.stream();
  cudaError_t e = cudaMemcpyAsync(rowptr, out_rowptr_.ptr,
                                  sizeof(int) * (size_t)(row_off_[count_] + count_),
                                  cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && nnz_total_ > 0)
    e = cudaMemcpyAsync(col, out_col_.ptr, sizeof(int) * (size_t)nnz_total_,
                        cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && nnz_total_ > 0)
    e = cudaMemcpyAsync(val, out_val_.ptr, sizeof(float) * (size_t)nnz_total_,
                        cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return E.cuda_fail(e, "copy batch output");
  return SPGEMM_OK;
}

}  // namespace sg

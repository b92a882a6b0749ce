// Host orchestration of the SpGEMM pipeline: workspace, bin scheduling,
// synchronisation points and error capture. One Engine per spgemm handle.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/cm.h"
#include "kernels.cuh"

namespace sg {

// Grow-only device buffer.
struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  cudaError_t ensure(size_t want);
  void release();
  template <class T> T* as() const { return static_cast<T*>(ptr); }
};

// Device-side counters, reset once per product and read back at the two
// synchronisation points.
struct DevCounters {
  int fb_count[16];  // first-pass bins (rows per bin; mid / block lists grow on warp overflow)
  int num_count[16];
  int slice_count;
  int mid_count;
  unsigned status;
  unsigned long long p_total;
  long long grand_total;
  int max_row_len;  // longest row of A (entries)
  int overflow_count;  // warp-bin rows redone by the mid / block kernels
  // whole-row numeric path, per launch (see launch_num_rows): rows per
  // work group, fill cursors of the work order, rows in the work order and
  // the dynamic row queue
  int lpt_hist[3][32];
  int lpt_cursor[3][32];
  int rows_listed[3];
  int row_queue[3];
};

// Whole-row numeric launches per product at most (long_rows = 3).
constexpr int ROWS_LAUNCHES = 3;

class Engine {
 public:
  Engine();
  ~Engine();

  int set_stream(cudaStream_t s);
  int set_precision(int p);
  // Rejects tunings that break the kernels' invariants (returns nonzero).
  int set_tuning(const Tuning& t);
  const Tuning& tuning() const { return tn_; }

  // Phase 1. A: COL_MAJOR (CSC) or ROW_MAJOR (CSR); B: ROW_MAJOR. Device
  // pointers. Synchronises the stream twice (bin counts, then nnz(C)).
  int symbolic(const cm& A, const cm& B, long long* nnz_c);
  // symbolic() in two stages (used by the mm.h shims): analyze() converts A,
  // computes P_i and the bins (first sync); symbolic_pass() computes the
  // exact row counts, row pointers and numeric bins (second sync).
  int analyze(const cm& A, const cm& B);
  int symbolic_pass(long long* nnz_c);
  // Phase 2 into caller-provided device buffers; synchronises once to
  // check the status word.
  int numeric(int* c_rowptr, int* c_col, float* c_val);
  // Phase 2 for a block-diagonal batch: C's row pointers are written per
  // product (product i's m_i + 1 entries, from 0, at c_rowptr + row_off[i] + i;
  // row_off_dev holds count + 1 row offsets on the device), columns and values
  // at their global positions. Allows nnz(C) beyond the int32 range.
  int numeric_batch(int count, const long long* row_off_dev, long long max_rows, int* c_rowptr,
                    int* c_col, float* c_val);
  // Phase 2 in pieces, for callers that overlap the copy of finished rows
  // with the rest: numeric_rows() computes C's columns and values of rows
  // [r0, r1) (stream-ordered, no synchronisation; the ranges of one product
  // must not overlap and must cover [0, m) before numeric_rowptr), and
  // numeric_rowptr() writes the int32 row pointers and synchronises once to
  // check the status word. owned_output() sizes the engine-owned C buffers
  // for the current symbolic result; rowptr64_to_host() copies C's int64
  // row pointers (m + 1) to the host and synchronises.
  int numeric_rows(int* c_col, float* c_val, int r0, int r1);
  int numeric_rowptr(int* c_rowptr);
  int owned_output(cm* C_dev);
  int rowptr64_to_host(long long* host);
  // Both phases into engine-owned output buffers.
  int multiply(const cm& A, const cm& B, cm* C_dev);
  // Numeric pass of the current symbolic result into engine-owned buffers.
  int multiply_numeric_owned(cm* C_dev);

  // Replay mode: the operands have the structure of the last product run
  // with replay off, so the host keeps that run's sizes, bin counts and
  // grids and the pipeline makes no host synchronisation (it can then be
  // recorded by stream capture). The status word is read by read_status().
  void set_replay(bool on) { replay_ = on; }
  bool replay() const { return replay_; }
  // Batch output: nnz(C) may exceed the int32 range of a single cm.
  void set_batch_output(bool on) { batch_out_ = on; }
  int read_status(unsigned* st);
  const long long* rowptr64() const { return c_rowptr64_.as<long long>(); }
  // After analyze(): products per row (int64) and the row list of first-pass
  // bin b (sym_bin_rows(b) entries).
  const long long* row_products() const { return row_p_.as<long long>(); }
  const int* bin_list(int b) const { return sym_rows_.as<int>() + (size_t)b * (size_t)m_; }
  const int* a_rowptr() const { return op_.a_rowptr; }
  void add_launches(long long n) { launches_ += n; }
  // Incremented by every analysis run outside replay mode: device buffers
  // and host sizes of an earlier product may have changed since.
  long long epoch() const { return epoch_; }
  bool profiling() const { return prof_on_; }

  const std::string& last_error() const { return err_; }
  long long launches() const { return launches_; }
  long long intermediate_products() const { return p_total_; }
  long long nnz_c() const { return nnz_c_; }
  int m() const { return m_; }
  int n() const { return n_; }
  int sym_bin_rows(int b) const { return fb_counts_[b]; }
  int overflow_rows() const { return overflow_rows_; }
  int num_bin_rows(int b) const { return num_counts_[b]; }
  int slices() const { return nslices_; }
  cudaStream_t stream() const { return stream_; }
  int precision() const { return precision_; }
  // Device buffers of the last multiply() output.
  int* out_rowptr() const { return out_rowptr_.as<int>(); }
  int* out_col() const { return out_col_.as<int>(); }
  float* out_val() const { return out_val_.as<float>(); }
  // Staging buffers for the host-buffer entry points.
  DevBuf& stage(int i) { return stage_[i]; }

  // Optional per-kernel timing with CUDA events recorded on the engine's
  // stream around every launch; accumulated per kernel name.
  void set_profiling(bool on) { prof_on_ = on; }
  void prof_begin(const char* name);
  void prof_end();
  int prof_collect();  // after a stream sync: fold finished events into totals
  int prof_collect_if_full();
  void prof_reset() {
    prof_collect();
    prof_ms_.clear();
    prof_count_.clear();
  }
  // Totals per kernel name (folds the open event pairs first; the stream
  // must have been synchronised since the last launch).
  const std::map<std::string, double>& prof_ms() {
    prof_collect();
    return prof_ms_;
  }
  const std::map<std::string, long long>& prof_count() {
    prof_collect();
    return prof_count_;
  }

  int fail(int status, const std::string& msg);
  int cuda_fail(cudaError_t e, const char* what);

 private:
  int numeric_values(int* c_col, float* c_val);
  int finish_numeric();
  int launch_first_pass();
  template <int MODE> int launch_fused();
  int launch_numeric_bins(int* c_col, float* c_val, int r0, int r1);
  template <int MODE> int launch_numeric_mode(int* c_col, float* c_val, int r0, int r1);
  size_t big_dir_bytes() const;
  // Whole-row numeric path of the long rows (k_num_rows): the largest nnz_i
  // it takes for this product (0: path off), its shared-memory value
  // capacity, and its launch.
  int rows_cnt_max() const;
  int rows_smem_cap(int threads) const;
  int launch_num_rows(int* c_col, float* c_val, int r0, int r1);
  int scan_counts(const int* in, int n, long long* out);
  int check_status(unsigned st);
  template <class K> cudaError_t smem_attr(K kernel, size_t bytes);

  cudaStream_t stream_ = nullptr;
  int device_ = 0;
  int sms_ = 148;
  int precision_ = 0;
  Tuning tn_;
  std::string err_;
  long long launches_ = 0;
  std::unordered_map<const void*, size_t> smem_set_;

  bool replay_ = false;
  bool batch_out_ = false;
  long long epoch_ = 0;

  // current product
  bool have_sym_ = false;
  int m_ = 0, kdim_ = 0, n_ = 0, n_chunks_ = 0;
  long long p_total_ = 0, nnz_c_ = 0;
  int fb_counts_[16] = {0};
  long long temp_total_ = 0;
  int overflow_rows_ = 0;
  int num_counts_[16] = {0};
  int nslices_ = 0, nmid_ = 0;
  long long big_capacity_ = 0;
  int n_long_sym_ = 0;
  int tn_run_slice_cap_ = 0;
  bool have_analysis_ = false;
  Operands op_{};

  DevBuf a_rowptr_, a_col_, a_val_, cursor_, aoff_;
  DevBuf row_p_, c_cnt_, c_rowptr64_, tiles_;
  DevBuf sym_rows_, num_rows_, long_slot_, chunk_cnt_, slices_buf_, mid_slices_, row_span_;
  DevBuf tcap_, toff_, t_col_, t_val_;  // fused pass: row bounds, temp offsets, temp output
  DevBuf counters_, restrict_scratch_, bitmaps_, lpt_order_;
  DevBuf valid_starts_;  // input validation: first position of every row of B (nnz(B) bits)
  int bitmap_words_ = 0;  // per long row; 0 when the bitmaps are not kept
  int max_row_len_ = 0;
  DevBuf out_rowptr_, out_col_, out_val_;
  DevBuf stage_[6];
  DevCounters* host_counters_ = nullptr;  // pinned

  bool prof_on_ = false;
  struct ProfRec { std::string name; cudaEvent_t a, b; };
  std::vector<ProfRec> prof_open_;
  std::vector<cudaEvent_t> prof_pool_;
  std::map<std::string, double> prof_ms_;
  std::map<std::string, long long> prof_count_;
  const char* prof_pending_ = nullptr;
  cudaEvent_t prof_take();
};

Tuning default_tuning();

// Triplets in any order (device) to compressed form: row_major -> CSR over
// rows, else CSC over columns; minor indices ascending within each major
// index, entries with equal indices in input order. ptr[n_major + 1],
// idx/val[nnz]. Entries with an index outside its dimension are left out and
// set bit 0 of *flags_host (when non-null the call synchronises `stream` to
// read it).
cudaError_t coo_compress(const triplet* t, int nnz, bool row_major, int n_major, int n_minor,
                         int* ptr, int* idx, float* val, DevBuf& scratch, DevBuf& scan_tmp,
                         unsigned* flags_host, cudaStream_t stream);

// Exclusive scan of n int32 counts into n+1 int32 pointers on `stream`.
// `tmp` is scratch (grown as needed); `total_dev` receives the sum (int64).
cudaError_t scan_counts_to_ptr32(const int* cnt, int n, int* ptr, DevBuf& tmp,
                                 long long* total_dev, cudaStream_t stream);

}  // namespace sg

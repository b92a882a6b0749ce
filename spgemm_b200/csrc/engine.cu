// Host orchestration of the SpGEMM pipeline (see pipeline.cuh).
//
// Reference call chain replaced here (src/main.cu:31-37):
//   cudaInitGEMM (src/mm.cu:150-193)      -> row analysis: P_i, P
//   cudaCategorizeGEMM (src/mm.cu:263-286) -> symbolic binning
//   cudaBinGEMM (src/mm.cu:314-327)        -> symbolic pass per bin
//   cudaMergeGEMM (src/mm.cu:407-450)      -> numeric pass per bin
// The reference synchronises after every kernel and copies C back one row at
// a time; this engine synchronises twice per product (bin counts, nnz(C))
// and leaves C in device memory.
#include "engine.h"

#include <algorithm>
#include <cstdio>
#include <cstring>

#include "esc.cuh"
#include "pipeline.cuh"

namespace sg {

cudaError_t DevBuf::ensure(size_t want) {
  if (want <= bytes && ptr) return cudaSuccess;
  if (ptr) { cudaFree(ptr); ptr = nullptr; bytes = 0; }
  if (want == 0) want = 16;
  cudaError_t e = cudaMalloc(&ptr, want);
  if (e != cudaSuccess) { ptr = nullptr; bytes = 0; return e; }
  bytes = want;
  return cudaSuccess;
}

void DevBuf::release() {
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
  bytes = 0;
}

Tuning default_tuning() {
  Tuning t;
  t.warp_p_max = 4096;
  t.warp_table_max = 256;
  t.warp_cap_max = 2048;
  t.long_p = 4096;
  t.long_o_num = 4096;
  t.slice_cap = 0;          // 0: as many as the shared-memory budget allows
  t.slice_cols = 1 << 18;
  t.sym_window = 1 << 20;
  t.keep_bitmaps = 1;
  t.mid_o_min = 256;
  t.mid_cols = 1 << 18;
  t.long_rows = 2;
  t.esc_p_min = 0;
  t.esc_span_min = 0;
  return t;
}

// Big bitmap slices of long rows: threads of one block, blocks resident per
// SM, and the shared memory one block may use.
static constexpr int BIG_THREADS = 1024;
static constexpr int BIG_BLOCKS_PER_SM = 1;
static constexpr size_t BIG_SMEM_BUDGET = 220 * 1024;
static constexpr size_t SEG_SCRATCH_BYTES = sizeof(SegScratch);

Engine::Engine() {
  tn_ = default_tuning();
  cudaGetDevice(&device_);
  int v = 0;
  if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device_) == cudaSuccess && v > 0)
    sms_ = v;
  cudaMallocHost(reinterpret_cast<void**>(&host_counters_), sizeof(DevCounters));
}

cudaEvent_t Engine::prof_take() {
  if (!prof_pool_.empty()) {
    cudaEvent_t e = prof_pool_.back();
    prof_pool_.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

void Engine::prof_begin(const char* name) {
  if (!prof_on_) return;
  cudaEvent_t a = prof_take();
  cudaEventRecord(a, stream_);
  prof_open_.push_back(ProfRec{name, a, nullptr});
}

void Engine::prof_end() {
  if (!prof_on_ || prof_open_.empty() || prof_open_.back().b) return;
  cudaEvent_t b = prof_take();
  cudaEventRecord(b, stream_);
  prof_open_.back().b = b;
}

// Event pairs are folded lazily: when the kernel times are read, or once
// PROF_DEFER records are open, so that a product's own synchronisation is
// not followed by host work on every call while profiling is on.
static constexpr size_t PROF_DEFER = 8192;

int Engine::prof_collect_if_full() { return prof_open_.size() > PROF_DEFER ? prof_collect() : 0; }

int Engine::prof_collect() {
  for (ProfRec& r : prof_open_) {
    if (r.b) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) {
        prof_ms_[r.name] += ms;
        prof_count_[r.name] += 1;
      }
      prof_pool_.push_back(r.b);
    }
    prof_pool_.push_back(r.a);
  }
  prof_open_.clear();
  return 0;
}

Engine::~Engine() {
  DevBuf* all[] = {&a_rowptr_, &a_col_, &a_val_, &cursor_, &aoff_, &row_p_, &c_cnt_,
                   &c_rowptr64_, &tiles_, &sym_rows_, &num_rows_, &long_slot_,
                   &chunk_cnt_, &slices_buf_, &mid_slices_, &row_span_, &counters_, &restrict_scratch_,
                   &tcap_, &toff_, &t_col_, &t_val_,
                   &bitmaps_, &lpt_order_, &valid_starts_, &out_rowptr_,
                   &out_col_, &out_val_};
  for (DevBuf* b : all) b->release();
  for (DevBuf& b : stage_) b.release();
  if (host_counters_) cudaFreeHost(host_counters_);
  for (ProfRec& r : prof_open_) {
    if (r.a) cudaEventDestroy(r.a);
    if (r.b) cudaEventDestroy(r.b);
  }
  for (cudaEvent_t e : prof_pool_) cudaEventDestroy(e);
}

int Engine::fail(int status, const std::string& msg) {
  err_ = msg;
  return status;
}

int Engine::cuda_fail(cudaError_t e, const char* what) {
  err_ = std::string(what) + ": " + cudaGetErrorString(e);
  return e == cudaErrorMemoryAllocation ? 3 /*SPGEMM_ERR_ALLOC*/ : 2 /*SPGEMM_ERR_CUDA*/;
}

int Engine::set_tuning(const Tuning& t) {
  // numeric long rows read the chunk counts and bitmaps that only symbolic
  // long rows write, and the fused tables hold at most 4096 distinct columns
  if (t.long_p < 1 || t.long_p > 4096) return fail(1, "tuning: 1 <= long_p <= 4096");
  if (t.long_o_num < 1 || t.long_o_num > 4096) return fail(1, "tuning: 1 <= long_o_num <= 4096");
  if (t.warp_table_max < 64 || t.warp_table_max > 1024 || (t.warp_table_max & (t.warp_table_max - 1)))
    return fail(1, "tuning: warp_table_max must be a power of two in [64, 1024]");
  if (t.warp_p_max < 0 || t.warp_cap_max < 0) return fail(1, "tuning: warp limits");
  if (t.slice_cols < CHUNK_COLS || t.slice_cols % CHUNK_COLS) return fail(1, "tuning: slice_cols");
  if (t.sym_window < CHUNK_COLS || t.sym_window % CHUNK_COLS || t.sym_window > (1 << 20))
    return fail(1, "tuning: sym_window");
  if (t.slice_cap != 0 && t.slice_cap < CHUNK_COLS)
    return fail(1, "tuning: slice_cap must be 0 (auto) or >= 2048");
  if (t.mid_o_min < 0 || t.mid_cols < 0 || t.mid_cols > (1 << 18))
    return fail(1, "tuning: mid_o_min >= 0 and 0 <= mid_cols <= 2^18");
  if (t.long_rows < 0 || t.long_rows > 3) return fail(1, "tuning: long_rows must be 0..3");
  if (t.esc_p_min < 0 || t.esc_span_min < 0) return fail(1, "tuning: esc_p_min, esc_span_min >= 0");
  tn_ = t;
  return 0;
}

int Engine::set_stream(cudaStream_t s) {
  stream_ = s;
  return 0;
}

int Engine::set_precision(int p) {
  if (p != 0 && p != 1) return fail(1, "precision must be 0 (plain) or 1 (compensated)");
  precision_ = p;
  return 0;
}

template <class K>
cudaError_t Engine::smem_attr(K kernel, size_t bytes) {
  const void* key = reinterpret_cast<const void*>(kernel);
  auto it = smem_set_.find(key);
  if (it != smem_set_.end() && it->second >= bytes) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)bytes);
  if (e == cudaSuccess) smem_set_[key] = bytes;
  return e;
}

#define SG_CK(call, what)                                  \
  do {                                                     \
    cudaError_t e__ = (call);                              \
    if (e__ != cudaSuccess) return cuda_fail(e__, what);   \
  } while (0)

#define SG_LAUNCHED(what)                                  \
  do {                                                     \
    ++launches_;                                           \
    prof_end();                                            \
    cudaError_t e__ = cudaGetLastError();                  \
    if (e__ != cudaSuccess) return cuda_fail(e__, what);   \
  } while (0)

static inline int blocks_for(long long work, int per_block, long long cap) {
  long long b = (work + per_block - 1) / per_block;
  if (b < 1) b = 1;
  if (b > cap) b = cap;
  return (int)b;
}

int Engine::check_status(unsigned st) {
  if (!st) return 0;
  std::string msg = "device check failed:";
  if (st & ST_TABLE_FULL) msg += " hash-table-full";
  if (st & ST_COUNT_MISMATCH) msg += " symbolic/numeric-count-mismatch";
  if (st & ST_ROW_TOO_LONG) msg += " row-with-2^31-or-more-partial-products";
  if (st & ST_SLICE_OVERFLOW) msg += " slice-list-overflow";
  if (st & ST_BAD_INDEX) msg += " index-out-of-range";
  if (st & ST_UNSORTED) msg += " B-row-not-sorted-by-column";
  return fail(st & ST_ROW_TOO_LONG ? 7 : ((st & (ST_BAD_INDEX | ST_UNSORTED)) ? 1 : 6), msg);
}

int Engine::scan_counts(const int* in, int n, long long* out) {
  const int ntiles = (n + SCAN_TILE - 1) / SCAN_TILE;
  SG_CK(tiles_.ensure(sizeof(long long) * (size_t)std::max(ntiles, 1)), "alloc scan tiles");
  long long* tiles = tiles_.as<long long>();
  long long* total = &counters_.as<DevCounters>()->grand_total;
  if (ntiles > 0) {
    prof_begin("k_scan_tiles");
    k_scan_tiles<<<ntiles, SCAN_THREADS, 0, stream_>>>(in, n, tiles);
    SG_LAUNCHED("k_scan_tiles");
  }
  prof_begin("k_scan_tile_sums");
  k_scan_tile_sums<<<1, SCAN_THREADS, 0, stream_>>>(tiles, ntiles, total);
  SG_LAUNCHED("k_scan_tile_sums");
  prof_begin("k_scan_apply");
  k_scan_apply<<<std::max(ntiles, 1), SCAN_THREADS, 0, stream_>>>(in, n, tiles, total, out);
  SG_LAUNCHED("k_scan_apply");
  return 0;
}

int Engine::symbolic(const cm& A, const cm& B, long long* nnz_c) {
  if (int r = analyze(A, B)) return r;
  return symbolic_pass(nnz_c);
}

int Engine::analyze(const cm& A, const cm& B) {
  have_sym_ = false;
  have_analysis_ = false;
  if (!replay_) ++epoch_;
  if (B.type != ROW_MAJOR) return fail(1, "B must be CSR (type ROW_MAJOR)");
  if (A.num_rows < 0 || A.num_cols < 0 || B.num_cols < 0 || A.nnz < 0 || B.nnz < 0)
    return fail(1, "negative dimension or nnz");
  if (A.num_cols != B.num_rows) return fail(1, "A.num_cols != B.num_rows");
  if (!A.ptr || !B.ptr) return fail(1, "null pointer array");
  if ((A.nnz > 0 && (!A.idx || !A.val)) || (B.nnz > 0 && (!B.idx || !B.val)))
    return fail(1, "null index/value array");
  m_ = A.num_rows;
  kdim_ = A.num_cols;
  n_ = B.num_cols;
  const int nnz_a = A.nnz;
  const int m = m_;

  SG_CK(counters_.ensure(sizeof(DevCounters)), "alloc counters");
  DevCounters* dc = counters_.as<DevCounters>();
  SG_CK(cudaMemsetAsync(dc, 0, sizeof(DevCounters), stream_), "memset counters");

  // ---- validate the operands (sync point 1 reports the result) ----
  {
    // flat passes: pointers (marking where B's rows start), then entries
    const long long grid_cap = (long long)sms_ * 16;
    const size_t start_words = ((size_t)std::max(B.nnz, 1) + 31) / 32;
    SG_CK(valid_starts_.ensure(sizeof(unsigned) * start_words), "alloc validation bitmap");
    unsigned* starts = valid_starts_.as<unsigned>();
    SG_CK(cudaMemsetAsync(starts, 0, sizeof(unsigned) * start_words, stream_), "memset bitmap");
    prof_begin("k_validate");
    k_validate_ptr<<<blocks_for((long long)kdim_ + 1, 256, grid_cap), 256, 0, stream_>>>(
        B.ptr, kdim_, B.nnz, starts, &dc->status);
    SG_LAUNCHED("k_validate_ptr(B)");
    if (B.nnz > 0) {
      prof_begin("k_validate");
      k_validate_idx<<<blocks_for(B.nnz, 256, grid_cap), 256, 0, stream_>>>(B.idx, B.nnz, n_, starts,
                                                                           &dc->status);
      SG_LAUNCHED("k_validate_idx(B)");
    }
    const int a_major = A.type == COL_MAJOR ? kdim_ : m;
    const int a_minor = A.type == COL_MAJOR ? m : kdim_;
    prof_begin("k_validate");
    k_validate_ptr<<<blocks_for((long long)a_major + 1, 256, grid_cap), 256, 0, stream_>>>(
        A.ptr, a_major, nnz_a, nullptr, &dc->status);
    SG_LAUNCHED("k_validate_ptr(A)");
    if (nnz_a > 0) {
      prof_begin("k_validate");
      k_validate_idx<<<blocks_for(nnz_a, 256, grid_cap), 256, 0, stream_>>>(A.idx, nnz_a, a_minor,
                                                                           nullptr, &dc->status);
      SG_LAUNCHED("k_validate_idx(A)");
    }
    // The transpose and row analysis guard every index they use; their
    // findings and the validation pass's are read at the first synchronisation below,
    // before any kernel trusts the inputs.
  }

  // ---- A in CSR ----
  const int* a_rowptr;
  const int* a_col;
  const float* a_val;
  SG_CK(c_cnt_.ensure(sizeof(int) * (size_t)std::max(m, 1)), "alloc c_cnt");
  SG_CK(c_rowptr64_.ensure(sizeof(long long) * ((size_t)m + 1)), "alloc c_rowptr64");
  if (A.type == COL_MAJOR) {
    SG_CK(a_rowptr_.ensure(sizeof(int) * ((size_t)m + 1)), "alloc a_rowptr");
    SG_CK(cursor_.ensure(sizeof(int) * ((size_t)m + 1)), "alloc cursor");
    SG_CK(a_col_.ensure(sizeof(int) * (size_t)std::max(nnz_a, 1)), "alloc a_col");
    SG_CK(a_val_.ensure(sizeof(float) * (size_t)std::max(nnz_a, 1)), "alloc a_val");
    int* cnt = c_cnt_.as<int>();
    SG_CK(cudaMemsetAsync(cnt, 0, sizeof(int) * (size_t)std::max(m, 1), stream_), "memset cnt");
    if (nnz_a > 0) {
      prof_begin("k_transpose_hist");
      k_transpose_hist<<<blocks_for(nnz_a, 256, (long long)sms_ * 16), 256, 0, stream_>>>(
          A.idx, nnz_a, m, cnt, &dc->status);
      SG_LAUNCHED("k_transpose_hist");
    }
    if (int r = scan_counts(cnt, m, c_rowptr64_.as<long long>())) return r;
    prof_begin("k_rowptr_i64_to_i32_shift");
    k_rowptr_i64_to_i32_shift<<<blocks_for(m + 1, 256, (long long)sms_ * 16), 256, 0, stream_>>>(
        c_rowptr64_.as<long long>(), m + 1, a_rowptr_.as<int>(), cursor_.as<int>());
    SG_LAUNCHED("k_rowptr_i64_to_i32_shift");
    if (nnz_a > 0) {
      prof_begin("k_transpose_scatter");
      k_transpose_scatter<<<blocks_for(nnz_a, 256, (long long)sms_ * 16), 256, 0, stream_>>>(
          A.ptr, A.idx, A.val, kdim_, nnz_a, m, cursor_.as<int>(), a_col_.as<int>(),
          a_val_.as<float>());
      SG_LAUNCHED("k_transpose_scatter");
    }
    a_rowptr = a_rowptr_.as<int>();
    a_col = a_col_.as<int>();
    a_val = a_val_.as<float>();
  } else {
    a_rowptr = A.ptr;
    a_col = A.idx;
    a_val = A.val;
  }

  // ---- row analysis ----
  SG_CK(aoff_.ensure(sizeof(int) * (size_t)std::max(nnz_a, 1)), "alloc aoff");
  SG_CK(row_p_.ensure(sizeof(long long) * (size_t)std::max(m, 1)), "alloc row_p");
  SG_CK(sym_rows_.ensure(sizeof(int) * (size_t)FB_COUNT * std::max(m, 1)), "alloc bin lists");
  SG_CK(row_span_.ensure(sizeof(int2) * (size_t)std::max(m, 1)), "alloc row spans");
  SG_CK(tcap_.ensure(sizeof(int) * (size_t)std::max(m, 1)), "alloc row bounds");
  SG_CK(toff_.ensure(sizeof(long long) * ((size_t)m + 1)), "alloc temp offsets");
  const int vec_ok = ((reinterpret_cast<uintptr_t>(B.idx) | reinterpret_cast<uintptr_t>(B.val)) & 15) == 0;
  op_ = Operands{a_rowptr, a_col, a_val, aoff_.as<int>(), B.ptr, B.idx, B.val, m_, kdim_, n_,
                 vec_ok, B.nnz};
  if (m > 0) {
    prof_begin("k_row_analysis");
    k_row_analysis<<<(m + RA_ROWS - 1) / RA_ROWS, RA_THREADS, 0, stream_>>>(
        op_, aoff_.as<int>(), row_p_.as<long long>(), c_cnt_.as<int>(), tcap_.as<int>(),
        dc->fb_count, sym_rows_.as<int>(), &dc->p_total, &dc->max_row_len, row_span_.as<int2>(),
        &dc->status, tn_);
    SG_LAUNCHED("k_row_analysis");
  }
  // temporary-buffer slots of the fused rows (grand total = buffer size)
  if (int r = scan_counts(tcap_.as<int>(), m, toff_.as<long long>())) return r;
  if (replay_) {  // same structure as the planned run: keep its sizes
    have_analysis_ = true;
    return 0;
  }
  SG_CK(cudaMemcpyAsync(host_counters_, dc, sizeof(DevCounters), cudaMemcpyDeviceToHost, stream_),
        "read counters");
  SG_CK(cudaStreamSynchronize(stream_), "sync after row analysis");
  if (int r = check_status(host_counters_->status)) return r;
  p_total_ = (long long)host_counters_->p_total;
  for (int b = 0; b < FB_COUNT; ++b) fb_counts_[b] = host_counters_->fb_count[b];
  n_long_sym_ = fb_counts_[FB_LONG];
  max_row_len_ = host_counters_->max_row_len;
  temp_total_ = host_counters_->grand_total;
  n_chunks_ = (n_ + CHUNK_COLS - 1) / CHUNK_COLS;
  have_analysis_ = true;
  return 0;
}

int Engine::symbolic_pass(long long* nnz_c) {
  if (!have_analysis_) return fail(5, "symbolic pass called before row analysis");
  have_sym_ = false;
  const int m = m_;
  DevCounters* dc = counters_.as<DevCounters>();

  // ---- first pass: fused rows to the temporary buffer, long rows counted ----
  SG_CK(t_col_.ensure(sizeof(int) * (size_t)std::max(temp_total_, 1ll)), "alloc temp columns");
  SG_CK(t_val_.ensure(sizeof(float) * (size_t)std::max(temp_total_, 1ll)), "alloc temp values");
  if (n_long_sym_ > 0) {
    SG_CK(long_slot_.ensure(sizeof(int) * (size_t)std::max(m, 1)), "alloc long_slot");
    SG_CK(chunk_cnt_.ensure(sizeof(int) * (size_t)n_long_sym_ * std::max(n_chunks_, 1)),
          "alloc chunk counts");
  }
  if (int r = launch_first_pass()) return r;

  // ---- row pointers + numeric binning of the long rows ----
  if (int r = scan_counts(c_cnt_.as<int>(), m, c_rowptr64_.as<long long>())) return r;
  SG_CK(num_rows_.ensure(sizeof(int) * (size_t)NB_COUNT * std::max(m, 1)), "alloc num_rows");
  big_capacity_ = (long long)n_long_sym_ * std::max(n_chunks_, 1);
  SG_CK(slices_buf_.ensure(sizeof(Slice) * (size_t)std::max(big_capacity_, 1ll)), "alloc slices");
  SG_CK(mid_slices_.ensure(sizeof(Slice) * (size_t)std::max(n_long_sym_, 1)), "alloc mid slices");
  // output capacity of one big slice: what the shared-memory budget leaves
  Tuning tr = tn_;
  {
    // per slot: the value, and (compensated) its column; plain slices store
    // columns straight into C
    const size_t vb = precision_ == 1 ? 8 + sizeof(int) : 4;
    const size_t fixed = (BIG_THREADS / 32) * SEG_SCRATCH_BYTES + big_dir_bytes();
    long long cap = (long long)((BIG_SMEM_BUDGET - fixed) / vb);
    cap = std::min<long long>(cap, 1 << 20);
    if (tn_.slice_cap > 0) cap = std::min<long long>(cap, tn_.slice_cap);
    tr.slice_cap = (int)cap;
    tn_run_slice_cap_ = tr.slice_cap;
  }
  if (m > 0 && n_long_sym_ > 0) {
    prof_begin("k_num_bin");
    k_num_bin<<<(m + NBIN_THREADS - 1) / NBIN_THREADS, NBIN_THREADS, 0, stream_>>>(
        m, n_, c_cnt_.as<int>(), row_p_.as<long long>(), c_rowptr64_.as<long long>(),
        row_span_.as<int2>(), dc->num_count, num_rows_.as<int>(), chunk_cnt_.as<int>(),
        n_chunks_, long_slot_.as<int>(), slices_buf_.as<Slice>(), &dc->slice_count,
        (int)big_capacity_, mid_slices_.as<Slice>(), &dc->mid_count, bitmap_words_ > 0 ? 1 : 0,
        &dc->status, tr, rows_cnt_max(), ROWS_MAX_WORDS);
    SG_LAUNCHED("k_num_bin");
  }
  if (replay_) {
    have_sym_ = true;
    return 0;
  }
  SG_CK(cudaMemcpyAsync(host_counters_, dc, sizeof(DevCounters), cudaMemcpyDeviceToHost, stream_),
        "read counters");
  SG_CK(cudaStreamSynchronize(stream_), "sync after symbolic pass");
  if (int r = check_status(host_counters_->status)) return r;
  nnz_c_ = host_counters_->grand_total;
  for (int b = 0; b < NB_COUNT; ++b) num_counts_[b] = host_counters_->num_count[b];
  nslices_ = host_counters_->slice_count;
  nmid_ = host_counters_->mid_count;
  overflow_rows_ = host_counters_->overflow_count;
  if (nnz_c_ > 2147483647ll && !batch_out_)
    return fail(4, "nnz(C) = " + std::to_string(nnz_c_) + " exceeds the int32 range of cm");
  if (nnz_c) *nnz_c = nnz_c_;
  have_sym_ = true;
  return 0;
}

int Engine::launch_first_pass() {
  const Operands op = op_;
  DevCounters* dc = counters_.as<DevCounters>();
  unsigned* status = &dc->status;
  const int m = m_;
  int* c_cnt = c_cnt_.as<int>();
  const long long* row_p = row_p_.as<long long>();
  int* rows = sym_rows_.as<int>();
  if (!replay_) bitmap_words_ = 0;
  // long rows first: they are the heaviest work items
  if (fb_counts_[FB_LONG] > 0) {
    const int win = std::min(n_, tn_.sym_window);
    const size_t smem = (LONG_THREADS / 32) * SEG_SCRATCH_BYTES + (size_t)((win + 31) / 32) * 4;
    SG_CK(smem_attr(k_sym_long, smem), "smem attr k_sym_long");
    const int cnt = fb_counts_[FB_LONG];
    const int grid = blocks_for(cnt, 1, (long long)sms_ * 2);
    const int stride = 2 * max_row_len_ + 2;
    if (n_ > tn_.sym_window)
      SG_CK(restrict_scratch_.ensure(sizeof(int) * (size_t)grid * stride), "alloc restrict scratch");
    else
      SG_CK(restrict_scratch_.ensure(16), "alloc restrict scratch");
    // Keep the long rows' presence bitmaps for the numeric pass when they fit
    // in a modest share of free device memory; otherwise it rebuilds them.
    if (tn_.keep_bitmaps && !replay_) {
      const size_t words = (size_t)(n_ + 31) / 32;
      const size_t want = words * 4 * (size_t)cnt;
      if (want <= bitmaps_.bytes) {  // the buffer of an earlier product is large enough
        bitmap_words_ = (int)words;
      } else {
        size_t free_b = 0, total_b = 0;
        cudaMemGetInfo(&free_b, &total_b);
        const size_t budget = std::min<size_t>((size_t)16 << 30, (free_b + bitmaps_.bytes) / 4);
        if (want <= budget && bitmaps_.ensure(want) == cudaSuccess) bitmap_words_ = (int)words;
        cudaGetLastError();  // a failed optional allocation is not an error
      }
    }
    prof_begin("k_sym_long");
    k_sym_long<<<grid, LONG_THREADS, smem, stream_>>>(
        op, rows + (size_t)FB_LONG * m, cnt, row_p, c_cnt, long_slot_.as<int>(),
        chunk_cnt_.as<int>(), n_chunks_, restrict_scratch_.as<int>(), stride,
        bitmaps_.as<unsigned>(), bitmap_words_, status, tn_);
    SG_LAUNCHED("k_sym_long");
  }
  return precision_ == 0 ? launch_fused<0>() : launch_fused<1>();
}

template <int MODE>
int Engine::launch_fused() {
  constexpr int WPB = SW_THREADS / 32;
  constexpr int MID_THREADS = 512;
  constexpr size_t VB = sizeof(typename SlotOf<MODE>::T);
  const Operands op = op_;
  DevCounters* dc = counters_.as<DevCounters>();
  unsigned* status = &dc->status;
  const int m = m_;
  int* rows = sym_rows_.as<int>();
  int* c_cnt = c_cnt_.as<int>();
  const long long* row_p = row_p_.as<long long>();
  const long long* toff = toff_.as<long long>();
  int* t_col = t_col_.as<int>();
  float* t_val = t_val_.as<float>();
  int* mid_rows = rows + (size_t)FB_MID * m;
  int* big_rows = rows + (size_t)(FB_BLOCK0 + 2) * m;
  int overflow_bound = 0;  // rows the warp bins may push to the mid / block lists
#define SG_FUSED_WARP(L)                                                                      \
  {                                                                                            \
    const int b = L - 6, cnt = fb_counts_[b];                                                  \
    if (cnt > 0) {                                                                             \
      overflow_bound += cnt;                                                                   \
      const size_t smem = WPB * ((size_t(1) << L) * (VB + 5) + SEG_SCRATCH_BYTES);             \
      SG_CK(smem_attr(k_fused_warp<L, MODE>, smem), "smem attr k_fused_warp");                 \
      prof_begin("k_fused_warp<" #L ">");                                                      \
      k_fused_warp<L, MODE><<<blocks_for(cnt, WPB, (long long)sms_ * 16), SW_THREADS, smem,    \
                              stream_>>>(op, rows + (size_t)b * m, cnt, row_span_.as<int2>(),  \
                                         toff, c_cnt, t_col, t_val, mid_rows,                  \
                                         &dc->fb_count[FB_MID], big_rows,                      \
                                         &dc->fb_count[FB_BLOCK0 + 2], tn_.mid_cols,           \
                                         rows + (size_t)FB_ESC0 * m, &dc->fb_count[FB_ESC0],   \
                                         tn_, row_p, &dc->overflow_count);                     \
      SG_LAUNCHED("k_fused_warp");                                                             \
    }                                                                                          \
  }
  SG_FUSED_WARP(6) SG_FUSED_WARP(7) SG_FUSED_WARP(8) SG_FUSED_WARP(9) SG_FUSED_WARP(10)
#undef SG_FUSED_WARP
  // mid bitmap rows (and warp overflow with a narrow span)
  if (fb_counts_[FB_MID] + overflow_bound > 0) {
    const int width = std::min(n_, tn_.mid_cols) + 32;  // + alignment of lo down to 32
    const int dir_words = (width + 31) / 32;
    const int cap = (int)std::min<long long>(tn_.long_p, n_);
    const size_t smem = (MID_THREADS / 32) * SEG_SCRATCH_BYTES + (size_t)dir_words * sizeof(uint2) +
                        (size_t)cap * (8 + sizeof(int)) + sizeof(unsigned) * ((dir_words + 31) / 32) +
                        sizeof(int) * (size_t)cap;
    SG_CK(smem_attr(k_num_long<MODE, MID_THREADS, true>, smem), "smem attr k_num_long fused");
    const int grid = blocks_for(fb_counts_[FB_MID] + overflow_bound, 1, (long long)sms_ * 4);
    prof_begin("k_fused_mid");
    k_num_long<MODE, MID_THREADS, true><<<grid, MID_THREADS, smem, stream_>>>(
        op, nullptr, 0, row_p, dir_words, cap, restrict_scratch_.as<int>(), 0,
        bitmaps_.as<unsigned>(), 0, long_slot_.as<int>(), t_col, t_val, status, mid_rows,
        &dc->fb_count[FB_MID], row_span_.as<int2>(), toff, c_cnt, 0, m);
    SG_LAUNCHED("k_fused_mid");
  }
#define SG_FUSED_BLOCK(L, NT)                                                                 \
  {                                                                                            \
    const int b = L - 11 + FB_BLOCK0;                                                          \
    const int bound = fb_counts_[b] + (L == 13 ? overflow_bound : 0);                          \
    if (bound > 0) {                                                                           \
      const size_t smem = (size_t(1) << L) * (VB + 5) + (NT / 32) * SEG_SCRATCH_BYTES;         \
      SG_CK(smem_attr(k_fused_block<L, NT, MODE>, smem), "smem attr k_fused_block");           \
      prof_begin("k_fused_block<" #L ">");                                                     \
      k_fused_block<L, NT, MODE><<<blocks_for(bound, 1, (long long)sms_ * 8), NT, smem,         \
                                   stream_>>>(op, rows + (size_t)b * m, &dc->fb_count[b],      \
                                              row_p, toff, row_span_.as<int2>(), c_cnt, t_col, \
                                              t_val, status);                                  \
      SG_LAUNCHED("k_fused_block");                                                            \
    }                                                                                          \
  }
  SG_FUSED_BLOCK(11, 256) SG_FUSED_BLOCK(12, 256) SG_FUSED_BLOCK(13, 512)
#undef SG_FUSED_BLOCK
  // sorted rows (expand, sort, compress), one block per row; the lists may
  // also hold warp rows that overflowed their tables
#define SG_FUSED_ESC(Q, NT, PER_SM)                                                           \
  {                                                                                            \
    const int b = FB_ESC0 + Q, cnt = fb_counts_[b] + overflow_bound;                           \
    if (cnt > 0) {                                                                             \
      const size_t smem = esc_smem_bytes<NT, MODE>();                                          \
      SG_CK(smem_attr(k_fused_esc<NT, MODE>, smem), "smem attr k_fused_esc");                  \
      prof_begin("k_fused_esc<" #NT ">");                                                      \
      k_fused_esc<NT, MODE><<<blocks_for(cnt, 1, (long long)sms_ * (PER_SM)), NT, smem,        \
                              stream_>>>(op, rows + (size_t)b * m, &dc->fb_count[b], row_p,    \
                                         toff, row_span_.as<int2>(), c_cnt, t_col, t_val,      \
                                         status);                                              \
      SG_LAUNCHED("k_fused_esc");                                                              \
    }                                                                                          \
  }
  SG_FUSED_ESC(0, 128, 8) SG_FUSED_ESC(1, 256, 4) SG_FUSED_ESC(2, 512, MODE ? 1 : 2)
#undef SG_FUSED_ESC
  return 0;
}

template int Engine::launch_fused<0>();
template int Engine::launch_fused<1>();

int Engine::numeric_values(int* c_col, float* c_val) { return numeric_rows(c_col, c_val, 0, m_); }

int Engine::numeric_rows(int* c_col, float* c_val, int r0, int r1) {
  if (!have_sym_) return fail(5, "numeric called without a successful symbolic pass");
  if (nnz_c_ > 0 && (!c_col || !c_val)) return fail(1, "null output pointer");
  if (r0 < 0 || r1 > m_ || r0 > r1) return fail(1, "numeric: row range outside [0, m]");
  if (r1 > r0 && temp_total_ > 0) {
    prof_begin("k_copy_fused");
    k_copy_fused<<<blocks_for((long long)(r1 - r0), 256, (long long)sms_ * 16), 256, 0, stream_>>>(
        r0, r1, tcap_.as<int>(), toff_.as<long long>(), c_cnt_.as<int>(),
        c_rowptr64_.as<long long>(), t_col_.as<int>(), t_val_.as<float>(), c_col, c_val);
    SG_LAUNCHED("k_copy_fused");
  }
  return launch_numeric_bins(c_col, c_val, r0, r1);
}

int Engine::numeric_rowptr(int* c_rowptr) {
  if (!have_sym_) return fail(5, "numeric called without a successful symbolic pass");
  if (!c_rowptr) return fail(1, "null output pointer");
  prof_begin("k_rowptr_to_i32");
  k_rowptr_to_i32<<<blocks_for(m_ + 1, 256, (long long)sms_ * 16), 256, 0, stream_>>>(
      c_rowptr64_.as<long long>(), m_ + 1, c_rowptr);
  SG_LAUNCHED("k_rowptr_to_i32");
  return finish_numeric();
}

int Engine::owned_output(cm* C_dev) {
  if (!have_sym_) return fail(5, "output requested without a successful symbolic pass");
  const long long nnz = nnz_c_;
  SG_CK(out_rowptr_.ensure(sizeof(int) * ((size_t)m_ + 1)), "alloc C row pointers");
  SG_CK(out_col_.ensure(sizeof(int) * (size_t)std::max(nnz, 1ll)), "alloc C columns");
  SG_CK(out_val_.ensure(sizeof(float) * (size_t)std::max(nnz, 1ll)), "alloc C values");
  C_dev->ptr = out_rowptr_.as<int>();
  C_dev->idx = out_col_.as<int>();
  C_dev->val = out_val_.as<float>();
  C_dev->nnz = (int)nnz;
  C_dev->num_rows = m_;
  C_dev->num_cols = n_;
  C_dev->type = ROW_MAJOR;
  return 0;
}

int Engine::rowptr64_to_host(long long* host) {
  if (!have_sym_) return fail(5, "row pointers requested without a successful symbolic pass");
  SG_CK(cudaMemcpyAsync(host, c_rowptr64_.as<long long>(), sizeof(long long) * ((size_t)m_ + 1),
                        cudaMemcpyDeviceToHost, stream_),
        "copy row pointers");
  SG_CK(cudaStreamSynchronize(stream_), "sync row pointers");
  return 0;
}

int Engine::finish_numeric() {
  if (replay_) return 0;  // the caller reads the status after the captured work
  DevCounters* dc = counters_.as<DevCounters>();
  SG_CK(cudaMemcpyAsync(&host_counters_->status, &dc->status, sizeof(unsigned),
                        cudaMemcpyDeviceToHost, stream_),
        "read status");
  SG_CK(cudaStreamSynchronize(stream_), "sync after numeric pass");
  prof_collect_if_full();
  return check_status(host_counters_->status);
}

int Engine::numeric(int* c_rowptr, int* c_col, float* c_val) {
  if (!have_sym_) return fail(5, "numeric called without a successful symbolic pass");
  if (!c_rowptr) return fail(1, "null output pointer");
  if (int r = numeric_values(c_col, c_val)) return r;
  prof_begin("k_rowptr_to_i32");
  k_rowptr_to_i32<<<blocks_for(m_ + 1, 256, (long long)sms_ * 16), 256, 0, stream_>>>(
      c_rowptr64_.as<long long>(), m_ + 1, c_rowptr);
  SG_LAUNCHED("k_rowptr_to_i32");
  return finish_numeric();
}

int Engine::numeric_batch(int count, const long long* row_off_dev, long long max_rows,
                          int* c_rowptr, int* c_col, float* c_val) {
  if (!have_sym_) return fail(5, "numeric called without a successful symbolic pass");
  if (!c_rowptr) return fail(1, "null output pointer");
  if (int r = numeric_values(c_col, c_val)) return r;
  if (count > 0) {
    prof_begin("k_batch_rowptr");
    const dim3 grid(blocks_for(max_rows + 1, 256, 64), count);
    k_batch_rowptr<<<grid, 256, 0, stream_>>>(c_rowptr64_.as<long long>(), row_off_dev, c_rowptr);
    SG_LAUNCHED("k_batch_rowptr");
  }
  return finish_numeric();
}

int Engine::read_status(unsigned* st) {
  DevCounters* dc = counters_.as<DevCounters>();
  SG_CK(cudaMemcpyAsync(&host_counters_->status, &dc->status, sizeof(unsigned),
                        cudaMemcpyDeviceToHost, stream_),
        "read status");
  SG_CK(cudaStreamSynchronize(stream_), "sync after batch");
  prof_collect_if_full();
  *st = host_counters_->status;
  return check_status(*st);
}

int Engine::launch_numeric_bins(int* c_col, float* c_val, int r0, int r1) {
  return precision_ == 0 ? launch_numeric_mode<0>(c_col, c_val, r0, r1)
                         : launch_numeric_mode<1>(c_col, c_val, r0, r1);
}

size_t Engine::big_dir_bytes() const {
  return (size_t)((std::min(n_, tn_.slice_cols) + 31) / 32) * sizeof(uint2);
}

template <int MODE>
int Engine::launch_numeric_mode(int* c_col, float* c_val, int r0, int r1) {
  constexpr int MID_THREADS = 512;
  constexpr size_t VB = sizeof(typename SlotOf<MODE>::T);
  const Operands op = op_;
  const int m = m_;
  const int* rows = num_rows_.as<int>();
  const long long* row_p = row_p_.as<long long>();
  const long long* c_rowptr = c_rowptr64_.as<long long>();
  unsigned* status = &counters_.as<DevCounters>()->status;
  const int stride = 2 * max_row_len_ + 2;
  if (MODE == 0 && rows_cnt_max() > 0)
    if (int r = launch_num_rows(c_col, c_val, r0, r1)) return r;
  // big bitmap slices (long rows)
  if (nslices_ > 0) {
    const int dir_words = (int)(big_dir_bytes() / sizeof(uint2));
    const size_t smem = (BIG_THREADS / 32) * SEG_SCRATCH_BYTES + big_dir_bytes() +
                        (size_t)tn_run_slice_cap_ * (MODE ? 8 + sizeof(int) : 4);
    SG_CK(smem_attr(k_num_long<MODE, BIG_THREADS, false>, smem), "smem attr k_num_long");
    const int grid = blocks_for(nslices_, 1, (long long)sms_ * BIG_BLOCKS_PER_SM * 2);
    SG_CK(restrict_scratch_.ensure(sizeof(int) * (size_t)grid * stride), "alloc restrict scratch");
    prof_begin("k_num_long");
    k_num_long<MODE, BIG_THREADS, false><<<grid, BIG_THREADS, smem, stream_>>>(
        op, slices_buf_.as<Slice>(), nslices_, row_p, dir_words, tn_run_slice_cap_,
        restrict_scratch_.as<int>(), stride, bitmaps_.as<unsigned>(), bitmap_words_,
        long_slot_.as<int>(), c_col, c_val, status, nullptr, nullptr, nullptr, nullptr, nullptr,
        r0, r1);
    SG_LAUNCHED("k_num_long");
  }
  // mid bitmap slices of long rows: at most long_o_num outputs, 512 threads
  if (nmid_ > 0) {
    const int width = std::min(n_, tn_.mid_cols) + 32;  // + alignment of lo down to 32
    const int dir_words = (width + 31) / 32;            // <= 8193, so l1 fits 512 threads
    const int cap = tn_.long_o_num;
    const size_t smem = (MID_THREADS / 32) * SEG_SCRATCH_BYTES + (size_t)dir_words * sizeof(uint2) +
                        (size_t)cap * ((MODE ? 8 : 4) + sizeof(int)) +
                        sizeof(unsigned) * ((dir_words + 31) / 32) + sizeof(int) * (size_t)cap;
    SG_CK(smem_attr(k_num_long<MODE, MID_THREADS, true>, smem), "smem attr k_num_long mid");
    const int grid = blocks_for(nmid_, 1, (long long)sms_ * 4);
    prof_begin("k_num_mid");
    k_num_long<MODE, MID_THREADS, true><<<grid, MID_THREADS, smem, stream_>>>(
        op, mid_slices_.as<Slice>(), nmid_, row_p, dir_words, cap,
        restrict_scratch_.as<int>(), 0, bitmaps_.as<unsigned>(), bitmap_words_,
        long_slot_.as<int>(), c_col, c_val, status, nullptr, nullptr, nullptr, nullptr, nullptr,
        r0, r1);
    SG_LAUNCHED("k_num_mid");
  }
#define SG_NUM_BLOCK(L, NT)                                                                  \
  {                                                                                           \
    const int b = L - 10 + 4, cnt = num_counts_[b];                                           \
    if (cnt > 0) {                                                                            \
      const size_t smem = (size_t(1) << L) * (VB + 4) + (NT / 32) * SEG_SCRATCH_BYTES;        \
      SG_CK(smem_attr(k_num_block<L, NT, MODE>, smem), "smem attr k_num_block");              \
      prof_begin("k_num_block<" #L ">");                                                       \
      k_num_block<L, NT, MODE><<<blocks_for(cnt, 1, (long long)sms_ * 8), NT, smem, stream_>>>( \
          op, rows + (size_t)b * m, cnt, r0, r1, row_p, c_rowptr, c_col, c_val, status);      \
      SG_LAUNCHED("k_num_block");                                                             \
    }                                                                                         \
  }
  SG_NUM_BLOCK(10, 256) SG_NUM_BLOCK(11, 256) SG_NUM_BLOCK(12, 512) SG_NUM_BLOCK(13, 512)
#undef SG_NUM_BLOCK
  return 0;
}

template int Engine::launch_numeric_mode<0>(int*, float*, int, int);

// Whole-row numeric path: reductions into C (long_rows = 1, any nnz_i) or
// shared-memory accumulation (long_rows = 2): rows of up to the capacity of
// a 512-thread block (two blocks per SM, so one block's per-row phases --
// directory load, ranks, zeroing, copy-out -- overlap the other's products)
// and, above it, of a 1024-thread block (one per SM). Plain FP32 only, and
// only when the symbolic pass kept the long rows' bitmaps.
static constexpr int ROWS_RED_THREADS = 512;
static constexpr size_t ROWS_SMEM_BUDGET_1 = 225 * 1024;  // one block per SM
static constexpr size_t ROWS_SMEM_BUDGET_2 = 111 * 1024;  // two blocks per SM

int Engine::rows_smem_cap(int threads) const {
  const size_t fixed = (threads / 32) * SEG_SCRATCH_BYTES + ROWS_MAX_WORDS * sizeof(uint2);
  const size_t budget = threads >= 1024 ? ROWS_SMEM_BUDGET_1 : ROWS_SMEM_BUDGET_2;
  return (int)((budget - fixed) / sizeof(float));
}

int Engine::rows_cnt_max() const {
  if (precision_ != 0 || tn_.long_rows == 0 || bitmap_words_ == 0 || n_long_sym_ == 0) return 0;
  return tn_.long_rows == 2 ? rows_smem_cap(1024) : 0x7fffffff;
}

// The whole-row launches of each long_rows mode, as (cnt_min, cnt_max] output
// ranges: 1 = reductions into C for every row; 2 = shared memory in 512- and
// 1024-thread blocks (longer rows take column slices); 3 = the same two, and
// reductions into C above the 1024-thread capacity.
int Engine::launch_num_rows(int* c_col, float* c_val, int r0, int r1) {
  DevCounters* dc = counters_.as<DevCounters>();
  if (r0 != 0 || r1 != m_) {  // one of several row ranges: fresh work orders and queues
    unsigned char* first = reinterpret_cast<unsigned char*>(&dc->lpt_hist);
    unsigned char* last = reinterpret_cast<unsigned char*>(&dc->row_queue) + sizeof(dc->row_queue);
    SG_CK(cudaMemsetAsync(first, 0, (size_t)(last - first), stream_), "reset row orders");
  }
  const int cnt = n_long_sym_;
  const int* rows = sym_rows_.as<int>() + (size_t)FB_LONG * m_;
  SG_CK(lpt_order_.ensure(sizeof(int) * ROWS_LAUNCHES * (size_t)cnt), "alloc row order");
  const int lb = blocks_for(cnt, 256, (long long)sms_ * 4);
  const Operands op = op_;
  unsigned* status = &dc->status;
  enum Kind { RED, SMEM512, SMEM1024 };
  struct Launch { int cmin, cmax; Kind kind; };
  const int small_cap = rows_smem_cap(512), big_cap = rows_smem_cap(1024);
  Launch plan[ROWS_LAUNCHES];
  int nl = 0;
  if (tn_.long_rows == 1) {
    plan[nl++] = {0, 0x7fffffff, RED};
  } else {
    plan[nl++] = {0, small_cap, SMEM512};
    plan[nl++] = {small_cap, big_cap, SMEM1024};
    if (tn_.long_rows == 3) plan[nl++] = {big_cap, 0x7fffffff, RED};
  }
  for (int g = 0; g < nl; ++g) {
    const int cmin = plan[g].cmin, cmax = plan[g].cmax;
    int* order = lpt_order_.as<int>() + (size_t)g * cnt;
    prof_begin("k_lpt_hist");
    k_lpt_hist<<<lb, 256, 0, stream_>>>(rows, cnt, r0, r1, row_p_.as<long long>(), c_cnt_.as<int>(),
                                        row_span_.as<int2>(), cmin, cmax, ROWS_MAX_WORDS,
                                        dc->lpt_hist[g]);
    SG_LAUNCHED("k_lpt_hist");
    prof_begin("k_lpt_scatter");
    k_lpt_scatter<<<lb, 256, 0, stream_>>>(rows, cnt, r0, r1, row_p_.as<long long>(), c_cnt_.as<int>(),
                                           row_span_.as<int2>(), cmin, cmax, ROWS_MAX_WORDS,
                                           dc->lpt_hist[g], dc->lpt_cursor[g], order,
                                           &dc->rows_listed[g]);
    SG_LAUNCHED("k_lpt_scatter");
    if (plan[g].kind == RED) {
      constexpr int NT = ROWS_RED_THREADS;
      const size_t smem = (NT / 32) * SEG_SCRATCH_BYTES + ROWS_MAX_WORDS * sizeof(uint2);
      SG_CK(smem_attr(k_num_rows<NT, true>, smem), "smem attr k_num_rows");
      prof_begin("k_num_rows");
      k_num_rows<NT, true><<<blocks_for(cnt, 1, (long long)sms_ * 2), NT, smem, stream_>>>(
          op, order, &dc->rows_listed[g], &dc->row_queue[g], row_p_.as<long long>(),
          c_rowptr64_.as<long long>(), row_span_.as<int2>(), bitmaps_.as<unsigned>(), bitmap_words_,
          long_slot_.as<int>(), ROWS_MAX_WORDS, 0, c_col, c_val, status);
      SG_LAUNCHED("k_num_rows");
    } else if (plan[g].kind == SMEM512) {
      constexpr int NT = 512;
      const size_t smem = (NT / 32) * SEG_SCRATCH_BYTES + ROWS_MAX_WORDS * sizeof(uint2) +
                          (size_t)small_cap * sizeof(float);
      SG_CK(smem_attr(k_num_rows<NT, false>, smem), "smem attr k_num_rows");
      prof_begin("k_num_rows<512>");
      k_num_rows<NT, false><<<blocks_for(cnt, 1, (long long)sms_ * 2), NT, smem, stream_>>>(
          op, order, &dc->rows_listed[g], &dc->row_queue[g], row_p_.as<long long>(),
          c_rowptr64_.as<long long>(), row_span_.as<int2>(), bitmaps_.as<unsigned>(), bitmap_words_,
          long_slot_.as<int>(), ROWS_MAX_WORDS, small_cap, c_col, c_val, status);
      SG_LAUNCHED("k_num_rows");
    } else {
      constexpr int NT = 1024;
      const size_t smem = (NT / 32) * SEG_SCRATCH_BYTES + ROWS_MAX_WORDS * sizeof(uint2) +
                          (size_t)big_cap * sizeof(float);
      SG_CK(smem_attr(k_num_rows<NT, false>, smem), "smem attr k_num_rows");
      prof_begin("k_num_rows<1024>");
      k_num_rows<NT, false><<<blocks_for(cnt, 1, (long long)sms_), NT, smem, stream_>>>(
          op, order, &dc->rows_listed[g], &dc->row_queue[g], row_p_.as<long long>(),
          c_rowptr64_.as<long long>(), row_span_.as<int2>(), bitmaps_.as<unsigned>(), bitmap_words_,
          long_slot_.as<int>(), ROWS_MAX_WORDS, big_cap, c_col, c_val, status);
      SG_LAUNCHED("k_num_rows");
    }
  }
  return 0;
}

int Engine::multiply(const cm& A, const cm& B, cm* C_dev) {
  long long nnz = 0;
  if (int r = symbolic(A, B, &nnz)) return r;
  return multiply_numeric_owned(C_dev);
}

int Engine::multiply_numeric_owned(cm* C_dev) {
  if (!have_sym_) return fail(5, "numeric called without a successful symbolic pass");
  const long long nnz = nnz_c_;
  SG_CK(out_rowptr_.ensure(sizeof(int) * ((size_t)m_ + 1)), "alloc C row pointers");
  SG_CK(out_col_.ensure(sizeof(int) * (size_t)std::max(nnz, 1ll)), "alloc C columns");
  SG_CK(out_val_.ensure(sizeof(float) * (size_t)std::max(nnz, 1ll)), "alloc C values");
  if (int r = numeric(out_rowptr_.as<int>(), out_col_.as<int>(), out_val_.as<float>())) return r;
  if (C_dev) {
    C_dev->ptr = out_rowptr_.as<int>();
    C_dev->idx = out_col_.as<int>();
    C_dev->val = out_val_.as<float>();
    C_dev->nnz = (int)nnz;
    C_dev->num_rows = m_;
    C_dev->num_cols = n_;
    C_dev->type = ROW_MAJOR;
  }
  return 0;
}

cudaError_t scan_counts_to_ptr32(const int* cnt, int n, int* ptr, DevBuf& tmp,
                                 long long* total_dev, cudaStream_t s) {
  const int ntiles = (n + SCAN_TILE - 1) / SCAN_TILE;
  const size_t tiles_bytes = sizeof(long long) * (size_t)std::max(ntiles, 1);
  const size_t ptr64_bytes = sizeof(long long) * ((size_t)n + 1);
  cudaError_t e = tmp.ensure(tiles_bytes + ptr64_bytes);
  if (e != cudaSuccess) return e;
  long long* tiles = tmp.as<long long>();
  long long* ptr64 = tiles + std::max(ntiles, 1);
  if (ntiles > 0) k_scan_tiles<<<ntiles, SCAN_THREADS, 0, s>>>(cnt, n, tiles);
  k_scan_tile_sums<<<1, SCAN_THREADS, 0, s>>>(tiles, ntiles, total_dev);
  k_scan_apply<<<std::max(ntiles, 1), SCAN_THREADS, 0, s>>>(cnt, n, tiles, total_dev, ptr64);
  k_rowptr_to_i32<<<blocks_for(n + 1, 256, 4096), 256, 0, s>>>(ptr64, n + 1, ptr);
  return cudaGetLastError();
}

}  // namespace sg

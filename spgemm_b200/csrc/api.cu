// C ABI of the engine (include/spgemm_b200.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/spgemm_b200.h"
#include "context.h"

namespace {

int g_verbose = 1;

int copy_in(sg::Engine& E, sg::DevBuf& buf, const void* host, size_t bytes, void** dev) {
  cudaError_t e = buf.ensure(bytes ? bytes : 16);
  if (e != cudaSuccess) return E.cuda_fail(e, "alloc staging buffer");
  if (bytes) {
    e = cudaMemcpyAsync(buf.ptr, host, bytes, cudaMemcpyHostToDevice, E.stream());
    if (e != cudaSuccess) return E.cuda_fail(e, "copy input to device");
  }
  *dev = buf.ptr;
  return SPGEMM_OK;
}

// Stage a host cm into device buffers 3*slot .. 3*slot+2.
int stage_matrix(sg::Engine& E, const cm& H, int slot, cm* D) {
  if (!H.ptr || (H.nnz > 0 && (!H.idx || !H.val)))
    return E.fail(SPGEMM_ERR_INVALID, "null host array");
  if (H.nnz < 0 || H.num_rows < 0 || H.num_cols < 0)
    return E.fail(SPGEMM_ERR_INVALID, "negative dimension or nnz");
  const size_t nptr = (size_t)(H.type == COL_MAJOR ? H.num_cols : H.num_rows) + 1;
  *D = H;
  void* p = nullptr;
  if (int r = copy_in(E, E.stage(3 * slot), H.ptr, sizeof(int) * nptr, &p)) return r;
  D->ptr = static_cast<int*>(p);
  if (int r = copy_in(E, E.stage(3 * slot + 1), H.idx, sizeof(int) * (size_t)H.nnz, &p)) return r;
  D->idx = static_cast<int*>(p);
  if (int r = copy_in(E, E.stage(3 * slot + 2), H.val, sizeof(float) * (size_t)H.nnz, &p)) return r;
  D->val = static_cast<float*>(p);
  return SPGEMM_OK;
}

// Numeric pass of the current symbolic result into the engine-owned C,
// copied to the host arrays piece by piece: the rows are cut into pieces of
// about h->copy_chunk bytes of C (at most MAX_PIECES), each piece is
// computed on the engine's stream and, once its event has fired, copied on
// the handle's copy stream while the later pieces compute. All pieces are
// enqueued before the first copy, so with pageable host memory (where a
// device-to-host cudaMemcpyAsync returns only when done) the computation
// still runs ahead of the copies. The row pointers come last.
int numeric_to_host(spgemm_handle_t h, int* c_rowptr, int* c_colidx, float* c_val) {
  sg::Engine& E = h->eng;
  cm C;
  if (int r = E.owned_output(&C)) return r;
  const int m = C.num_rows;
  const long long nnz = E.nnz_c();
  const long long bytes = 8 * nnz;
  const long long chunk = h->copy_chunk > 0 ? h->copy_chunk : bytes;
  int pieces = (int)std::min<long long>(spgemm_context::MAX_PIECES,
                                        std::max<long long>(1, (bytes + chunk - 1) / std::max(chunk, 1ll)));
  if (m == 0) pieces = 1;
  std::vector<long long> rp;
  std::vector<int> bounds(1, 0);
  if (pieces > 1) {
    rp.resize((size_t)m + 1);
    if (int r = E.rowptr64_to_host(rp.data())) return r;
    for (int j = 1; j < pieces; ++j) {
      const long long target = nnz * j / pieces;
      int r = (int)(std::lower_bound(rp.begin(), rp.end(), target) - rp.begin());
      r = std::min(std::max(r, bounds.back()), m);
      bounds.push_back(r);
    }
  }
  bounds.push_back(m);
  cudaStream_t s = E.stream();
  cudaError_t e = cudaSuccess;
  if (pieces > 1 && !h->copy_stream) {
    e = cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return E.cuda_fail(e, "create copy stream");
  }
  for (int j = 0; j < pieces; ++j) {
    if (int r = E.numeric_rows(C.idx, C.val, bounds[j], bounds[j + 1])) return r;
    if (pieces > 1) {
      if (!h->piece_done[j]) {
        e = cudaEventCreateWithFlags(&h->piece_done[j], cudaEventDisableTiming);
        if (e != cudaSuccess) return E.cuda_fail(e, "create piece event");
      }
      e = cudaEventRecord(h->piece_done[j], s);
      if (e != cudaSuccess) return E.cuda_fail(e, "record piece event");
    }
  }
  // copies: one piece after another on the copy stream (the whole of C on
  // the engine's stream when there is a single piece)
  for (int j = 0; j < pieces && e == cudaSuccess; ++j) {
    const long long e0 = pieces > 1 ? rp[bounds[j]] : 0;
    const long long e1 = pieces > 1 ? rp[bounds[j + 1]] : nnz;
    if (e1 <= e0) continue;
    cudaStream_t cs = s;
    if (pieces > 1) {
      cs = h->copy_stream;
      e = cudaStreamWaitEvent(cs, h->piece_done[j], 0);
    }
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(c_colidx + e0, C.idx + e0, sizeof(int) * (size_t)(e1 - e0),
                          cudaMemcpyDeviceToHost, cs);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(c_val + e0, C.val + e0, sizeof(float) * (size_t)(e1 - e0),
                          cudaMemcpyDeviceToHost, cs);
  }
  int r = e == cudaSuccess ? E.numeric_rowptr(C.ptr) : E.cuda_fail(e, "copy C to host");
  if (r == SPGEMM_OK) {
    e = cudaMemcpyAsync(c_rowptr, C.ptr, sizeof(int) * ((size_t)m + 1), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) r = E.cuda_fail(e, "copy C row pointers to host");
  }
  // the host arrays stay in use until the copy stream is idle
  if (h->copy_stream) {
    e = cudaStreamSynchronize(h->copy_stream);
    if (e != cudaSuccess && r == SPGEMM_OK) r = E.cuda_fail(e, "copy C to host");
  }
  return r;
}

}  // namespace

extern "C" {

int spgemm_internal_verbose(void) { return g_verbose; }

const char* spgemm_version(void) { return "spgemm_b200 0.1.0 (sm_100a)"; }

const char* spgemm_status_string(int s) {
  switch (s) {
    case SPGEMM_OK: return "ok";
    case SPGEMM_ERR_INVALID: return "invalid argument";
    case SPGEMM_ERR_CUDA: return "CUDA error";
    case SPGEMM_ERR_ALLOC: return "allocation failed";
    case SPGEMM_ERR_OVERFLOW: return "nnz(C) exceeds int32";
    case SPGEMM_ERR_STATE: return "call out of order";
    case SPGEMM_ERR_DEVICE: return "device-side check failed";
    case SPGEMM_ERR_TOO_LARGE: return "size exceeds a documented maximum";
    default: return "unknown status";
  }
}

int spgemm_create(spgemm_handle_t* handle) {
  if (!handle) return SPGEMM_ERR_INVALID;
  *handle = nullptr;
  spgemm_context* c = new (std::nothrow) spgemm_context();
  if (!c) return SPGEMM_ERR_ALLOC;
  *handle = c;
  return SPGEMM_OK;
}

int spgemm_destroy(spgemm_handle_t handle) {
  delete handle;
  return SPGEMM_OK;
}

int spgemm_set_stream(spgemm_handle_t h, void* stream) {
  if (!h) return SPGEMM_ERR_INVALID;
  return h->eng.set_stream(static_cast<cudaStream_t>(stream));
}

int spgemm_set_precision(spgemm_handle_t h, int precision) {
  if (!h) return SPGEMM_ERR_INVALID;
  return h->eng.set_precision(precision);
}

int spgemm_get_tuning(spgemm_handle_t h, spgemm_tuning* out) {
  if (!h || !out) return SPGEMM_ERR_INVALID;
  const sg::Tuning& t = h->eng.tuning();
  out->warp_p_max = t.warp_p_max;
  out->warp_table_max = t.warp_table_max;
  out->warp_cap_max = t.warp_cap_max;
  out->long_p = t.long_p;
  out->long_o_num = t.long_o_num;
  out->slice_cap = t.slice_cap;
  out->slice_cols = t.slice_cols;
  out->sym_window = t.sym_window;
  out->keep_bitmaps = t.keep_bitmaps;
  out->mid_o_min = t.mid_o_min;
  out->mid_cols = t.mid_cols;
  out->long_rows = t.long_rows;
  out->esc_p_min = t.esc_p_min;
  out->esc_span_min = t.esc_span_min;
  return SPGEMM_OK;
}

int spgemm_set_tuning(spgemm_handle_t h, const spgemm_tuning* in) {
  if (!h || !in) return SPGEMM_ERR_INVALID;
  sg::Tuning t = h->eng.tuning();
  t.warp_p_max = in->warp_p_max;
  t.warp_table_max = in->warp_table_max;
  t.warp_cap_max = in->warp_cap_max;
  t.long_p = in->long_p;
  t.long_o_num = in->long_o_num;
  t.slice_cap = in->slice_cap;
  t.slice_cols = in->slice_cols;
  t.sym_window = in->sym_window;
  t.keep_bitmaps = in->keep_bitmaps ? 1 : 0;
  t.mid_o_min = in->mid_o_min;
  t.mid_cols = in->mid_cols;
  t.long_rows = in->long_rows;
  t.esc_p_min = in->esc_p_min;
  t.esc_span_min = in->esc_span_min;
  return h->eng.set_tuning(t);
}

const char* spgemm_last_error(spgemm_handle_t h) {
  return h ? h->eng.last_error().c_str() : "null handle";
}

int spgemm_symbolic(spgemm_handle_t h, cm A, cm B, long long* nnz_c) {
  if (!h) return SPGEMM_ERR_INVALID;
  return h->eng.symbolic(A, B, nnz_c);
}

int spgemm_numeric(spgemm_handle_t h, int* c_rowptr, int* c_colidx, float* c_val) {
  if (!h) return SPGEMM_ERR_INVALID;
  return h->eng.numeric(c_rowptr, c_colidx, c_val);
}

int spgemm_multiply(spgemm_handle_t h, cm A, cm B, cm* C) {
  if (!h) return SPGEMM_ERR_INVALID;
  return h->eng.multiply(A, B, C);
}

int spgemm_batch_plan(spgemm_handle_t h, int count, const cm* A, const cm* B,
                      long long* nnz_total) {
  if (!h) return SPGEMM_ERR_INVALID;
  return h->batch.plan(h->eng, count, A, B, nnz_total);
}

int spgemm_batch_execute(spgemm_handle_t h, int use_graph) {
  if (!h) return SPGEMM_ERR_INVALID;
  return h->batch.execute(h->eng, use_graph);
}

int spgemm_batch_offsets(spgemm_handle_t h, long long* row_offsets, long long* nnz_offsets) {
  if (!h) return SPGEMM_ERR_INVALID;
  return h->batch.offsets(h->eng, row_offsets, nnz_offsets);
}

int spgemm_batch_result(spgemm_handle_t h, int i, cm* C) {
  if (!h) return SPGEMM_ERR_INVALID;
  return h->batch.result(h->eng, i, C);
}

int spgemm_batch_copy_result(spgemm_handle_t h, int i, int* c_rowptr, int* c_colidx,
                             float* c_val) {
  if (!h) return SPGEMM_ERR_INVALID;
  return h->batch.copy_result(h->eng, i, c_rowptr, c_colidx, c_val);
}

int spgemm_batch_copy_all(spgemm_handle_t h, int* c_rowptr, int* c_colidx, float* c_val) {
  if (!h) return SPGEMM_ERR_INVALID;
  return h->batch.copy_all(h->eng, c_rowptr, c_colidx, c_val);
}

int spgemm_coo_to_cm(spgemm_handle_t h, const triplet* d_triplets, int nnz, int num_rows,
                     int num_cols, int type, int* d_ptr, int* d_idx, float* d_val) {
  if (!h) return SPGEMM_ERR_INVALID;
  sg::Engine& E = h->eng;
  const bool row_major = type == ROW_MAJOR;
  const int n_major = row_major ? num_rows : num_cols;
  const int n_minor = row_major ? num_cols : num_rows;
  if (nnz < 0 || n_major < 0 || n_minor < 0 || !d_ptr || (nnz > 0 && (!d_triplets || !d_idx || !d_val)))
    return E.fail(SPGEMM_ERR_INVALID, "coo_to_cm: invalid argument");
  unsigned flags = 0;
  cudaError_t e = sg::coo_compress(d_triplets, nnz, row_major, n_major, n_minor, d_ptr, d_idx,
                                   d_val, h->coo_scratch, h->coo_scan, &flags, E.stream());
  if (e != cudaSuccess) return E.cuda_fail(e, "coo_to_cm");
  if (flags & 1u) return E.fail(SPGEMM_ERR_INVALID, "coo_to_cm: index outside the dimensions");
  return SPGEMM_OK;
}

int spgemm_get_stats(spgemm_handle_t h, spgemm_stats* out) {
  if (!h || !out) return SPGEMM_ERR_INVALID;
  memset(out, 0, sizeof(*out));
  const sg::Engine& E = h->eng;
  out->intermediate_products = E.intermediate_products();
  out->nnz_c = E.nnz_c();
  for (int b = 0; b < sg::FB_COUNT; ++b) out->rows_per_symbolic_bin[b] = E.sym_bin_rows(b);
  out->warp_overflow_rows = E.overflow_rows();
  for (int b = 0; b < sg::NB_COUNT; ++b) out->rows_per_numeric_bin[b] = E.num_bin_rows(b);
  out->long_row_slices = E.slices();
  out->kernel_launches = E.launches();
  return SPGEMM_OK;
}

int spgemm_multiply_host_to(spgemm_handle_t h, cm A_host, cm B_host, int* c_rowptr,
                            int* c_colidx, float* c_val, long long capacity,
                            long long* nnz_c) {
  if (!h) return SPGEMM_ERR_INVALID;
  sg::Engine& E = h->eng;
  cm A, B;
  if (int r = stage_matrix(E, A_host, 0, &A)) return r;
  if (int r = stage_matrix(E, B_host, 1, &B)) return r;
  long long nnz = 0;
  if (int r = E.symbolic(A, B, &nnz)) return r;
  if (nnz_c) *nnz_c = nnz;
  if (nnz > capacity || !c_rowptr || (nnz > 0 && (!c_colidx || !c_val)))
    return E.fail(SPGEMM_ERR_TOO_LARGE, "output capacity below nnz(C)");
  return numeric_to_host(h, c_rowptr, c_colidx, c_val);
}

int spgemm_set_copy_chunk(spgemm_handle_t h, long long bytes) {
  if (!h || bytes < 0) return SPGEMM_ERR_INVALID;
  h->copy_chunk = bytes;
  return SPGEMM_OK;
}

int spgemm_multiply_host(spgemm_handle_t h, cm A_host, cm B_host, cm* C_host) {
  if (!h || !C_host) return SPGEMM_ERR_INVALID;
  sg::Engine& E = h->eng;
  cm A, B;
  if (int r = stage_matrix(E, A_host, 0, &A)) return r;
  if (int r = stage_matrix(E, B_host, 1, &B)) return r;
  long long nnz = 0;
  if (int r = E.symbolic(A, B, &nnz)) return r;
  if (nnz > 2147483647ll) return E.fail(SPGEMM_ERR_OVERFLOW, "nnz(C) exceeds the int32 range of cm");
  cm out;
  out.num_rows = A.num_rows;
  out.num_cols = B.num_cols;
  out.nnz = (int)nnz;
  out.type = ROW_MAJOR;
  out.ptr = static_cast<int*>(malloc(sizeof(int) * ((size_t)out.num_rows + 1)));
  out.idx = static_cast<int*>(malloc(sizeof(int) * (size_t)(nnz > 0 ? nnz : 1)));
  out.val = static_cast<float*>(malloc(sizeof(float) * (size_t)(nnz > 0 ? nnz : 1)));
  if (!out.ptr || !out.idx || !out.val) {
    free(out.ptr); free(out.idx); free(out.val);
    return E.fail(SPGEMM_ERR_ALLOC, "host allocation of C failed");
  }
  if (int r = numeric_to_host(h, out.ptr, out.idx, out.val)) {
    free(out.ptr); free(out.idx); free(out.val);
    return r;
  }
  *C_host = out;
  return SPGEMM_OK;
}

void spgemm_set_verbose(int verbose) { g_verbose = verbose ? 1 : 0; }

int spgemm_set_profiling(spgemm_handle_t h, int enable) {
  if (!h) return SPGEMM_ERR_INVALID;
  h->eng.set_profiling(enable != 0);
  return SPGEMM_OK;
}

int spgemm_reset_kernel_times(spgemm_handle_t h) {
  if (!h) return SPGEMM_ERR_INVALID;
  h->eng.prof_reset();
  return SPGEMM_OK;
}

int spgemm_get_kernel_times(spgemm_handle_t h, char* names, int names_len, double* ms,
                            long long* launches, int max_kernels) {
  if (!h || max_kernels < 0) return -SPGEMM_ERR_INVALID;
  const auto& t = h->eng.prof_ms();
  const auto& c = h->eng.prof_count();
  int i = 0;
  size_t pos = 0;
  if (names && names_len > 0) names[0] = 0;
  for (const auto& kv : t) {
    if (i >= max_kernels) break;
    if (ms) ms[i] = kv.second;
    if (launches) {
      auto it = c.find(kv.first);
      launches[i] = it == c.end() ? 0 : it->second;
    }
    if (names && pos + kv.first.size() + 2 <= (size_t)names_len) {
      memcpy(names + pos, kv.first.data(), kv.first.size());
      pos += kv.first.size();
      names[pos++] = '\n';
      names[pos] = 0;
    }
    ++i;
  }
  return i;
}

}  // extern "C"

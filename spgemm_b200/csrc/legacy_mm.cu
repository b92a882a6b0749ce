// mm.h entry family (reference lib/mm.h:17-25, src/mm.cu) on top of the
// engine. Like the reference, the family keeps one product in module state:
// the COL_MAJOR matrix converted last is operand A (CSC), the ROW_MAJOR one
// operand B (CSR), and C lives in device memory after cudaMergeGEMM.
// Printed outputs match the reference: "P P" after cudaInitGEMM
// (src/mm.cu:181) and "nnzC nnzCf" after cudaMergeGEMM (src/mm.cu:449).
#include <cuda_runtime.h>

#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "../../include/mm.h"
#include "../../include/spgemm_b200.h"
#include "engine.h"

extern "C" int spgemm_internal_verbose(void);

namespace {

sg::Engine* g_eng = nullptr;
int g_exit_on_error = 1;
int g_status = SPGEMM_OK;

// Device copies of the two operands (module state of the reference,
// src/mm.cu:19-25).
sg::DevBuf g_a_ptr, g_a_idx, g_a_val;  // A: CSC
sg::DevBuf g_b_ptr, g_b_idx, g_b_val;  // B: CSR
sg::DevBuf g_tmp_triplets, g_tmp_cnt, g_tmp_ptr64, g_tmp_flag, g_tmp_sort;
cm g_A_dev, g_B_dev;
bool g_have_a = false, g_have_b = false, g_have_c = false;

sg::Engine& eng() {
  if (!g_eng) g_eng = new sg::Engine();
  return *g_eng;
}

// Reference error path (src/mm.cu:6-14): print and exit(-1) unless the
// caller switched exiting off.
void legacy_fail(int status, const char* file, int line, const char* msg) {
  g_status = status;
  printf("[%s:%d]CUDA ERROR : %s\n", file, line, msg);
  fflush(stdout);
  if (g_exit_on_error) exit(-1);
}
#define LEGACY_FAIL(st, msg) legacy_fail((st), __FILE__, __LINE__, (msg))

// Split sorted triplets into (minor index, value) and count entries per
// major index. `order_bad` is set if the triplets are not sorted by
// (major, minor), which the reference's protocol requires of the caller
// (src/main.cu:27-30).
__global__ void k_coo_split(const triplet* __restrict__ t, int nnz, bool row_major,
                            int n_major, int n_minor, int* __restrict__ cnt,
                            int* __restrict__ idx, float* __restrict__ val,
                            unsigned* __restrict__ flags) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += gridDim.x * blockDim.x) {
    const triplet x = t[e];
    const int major = row_major ? x.ridx : x.cidx;
    const int minor = row_major ? x.cidx : x.ridx;
    if ((unsigned)major >= (unsigned)n_major || (unsigned)minor >= (unsigned)n_minor) {
      atomicOr(flags, 1u);
      continue;
    }
    if (e > 0) {
      const triplet y = t[e - 1];
      const int pm = row_major ? y.ridx : y.cidx;
      const int pn = row_major ? y.cidx : y.ridx;
      if (pm > major || (pm == major && pn > minor)) atomicOr(flags, 2u);
    }
    idx[e] = minor;
    val[e] = x.val;
    atomicAdd(cnt + major, 1);
  }
}

__global__ void k_count_above(const float* __restrict__ v, long long n, float thr,
                              unsigned long long* __restrict__ out) {
  unsigned long long c = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    c += v[i] > thr;
  for (int d = 16; d > 0; d >>= 1) c += __shfl_xor_sync(0xffffffffu, c, d);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

template <class T>
T* host_alloc(size_t n) {
  return static_cast<T*>(malloc(sizeof(T) * (n ? n : 1)));
}

}  // namespace

extern "C" {

void spgemm_set_exit_on_error(int enable) { g_exit_on_error = enable ? 1 : 0; }
int spgemm_legacy_status(void) { return g_status; }
// shared with the spGEMM.h family (legacy_spgemm.cu)
int spgemm_internal_exit_on_error(void) { return g_exit_on_error; }
void spgemm_internal_set_legacy_status(int s) { g_status = s; }

// Replaces reference src/mm.cu:65-136 (kernel coo2cm at :43-63).
cm cudaCOO2CM(coo mat) {
  g_status = SPGEMM_OK;
  cm ret;
  cmInit(&ret);
  cmSetNNZ(&ret, mat.nnz);
  cmSetNumRows(&ret, mat.num_rows);
  cmSetNumCols(&ret, mat.num_cols);
  cmSetType(&ret, mat.type);
  sg::Engine& E = eng();
  cudaStream_t s = E.stream();
  const bool row_major = mat.type == ROW_MAJOR;
  const int n_major = row_major ? mat.num_rows : mat.num_cols;
  const int n_minor = row_major ? mat.num_cols : mat.num_rows;
  if (mat.nnz < 0 || n_major < 0 || n_minor < 0 || (mat.nnz > 0 && !mat.data)) {
    LEGACY_FAIL(SPGEMM_ERR_INVALID, "cudaCOO2CM: invalid coo");
    return ret;
  }
  sg::DevBuf& dptr = row_major ? g_b_ptr : g_a_ptr;
  sg::DevBuf& didx = row_major ? g_b_idx : g_a_idx;
  sg::DevBuf& dval = row_major ? g_b_val : g_a_val;
  cudaError_t e = cudaSuccess;
  const size_t nnz = (size_t)mat.nnz;
  if (e == cudaSuccess) e = g_tmp_triplets.ensure(sizeof(triplet) * (nnz ? nnz : 1));
  if (e == cudaSuccess) e = g_tmp_cnt.ensure(sizeof(int) * ((size_t)n_major + 1));
  if (e == cudaSuccess) e = g_tmp_flag.ensure(sizeof(unsigned long long) * 2);
  if (e == cudaSuccess) e = dptr.ensure(sizeof(int) * ((size_t)n_major + 1));
  if (e == cudaSuccess) e = didx.ensure(sizeof(int) * (nnz ? nnz : 1));
  if (e == cudaSuccess) e = dval.ensure(sizeof(float) * (nnz ? nnz : 1));
  if (e == cudaSuccess && nnz)
    e = cudaMemcpyAsync(g_tmp_triplets.ptr, mat.data, sizeof(triplet) * nnz,
                        cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(g_tmp_cnt.ptr, 0, sizeof(int) * ((size_t)n_major + 1), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(g_tmp_flag.ptr, 0, sizeof(unsigned long long) * 2, s);
  if (e != cudaSuccess) {
    LEGACY_FAIL(SPGEMM_ERR_CUDA, cudaGetErrorString(e));
    return ret;
  }
  if (nnz) {
    const int blocks = (int)((nnz + 255) / 256 < 4096 ? (nnz + 255) / 256 : 4096);
    k_coo_split<<<blocks, 256, 0, s>>>(g_tmp_triplets.as<triplet>(), mat.nnz, row_major,
                                       n_major, n_minor, g_tmp_cnt.as<int>(), didx.as<int>(),
                                       dval.as<float>(), g_tmp_flag.as<unsigned>());
  }
  // exclusive scan of the per-major counts into int32 pointers
  {
    long long* total = reinterpret_cast<long long*>(g_tmp_flag.as<unsigned long long>() + 1);
    e = cudaGetLastError();
    if (e == cudaSuccess)
      e = sg::scan_counts_to_ptr32(g_tmp_cnt.as<int>(), n_major, dptr.as<int>(), g_tmp_ptr64,
                                   total, s);
    unsigned flags = 0;
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(&flags, g_tmp_flag.ptr, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
    ret.ptr = host_alloc<int>((size_t)n_major + 1);
    ret.idx = host_alloc<int>(nnz);
    ret.val = host_alloc<float>(nnz);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(ret.ptr, dptr.ptr, sizeof(int) * ((size_t)n_major + 1),
                          cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && nnz)
      e = cudaMemcpyAsync(ret.idx, didx.ptr, sizeof(int) * nnz, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && nnz)
      e = cudaMemcpyAsync(ret.val, dval.ptr, sizeof(float) * nnz, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
      LEGACY_FAIL(SPGEMM_ERR_CUDA, cudaGetErrorString(e));
      return ret;
    }
    if (flags & 1u) {
      LEGACY_FAIL(SPGEMM_ERR_INVALID, "cudaCOO2CM: index outside the matrix dimensions");
      return ret;
    }
    if (flags & 2u) {
      // Not in the protocol's order (sortCOO skipped): sort on the device
      // instead of on the host. Entries with equal indices keep their order.
      unsigned f2 = 0;
      e = sg::coo_compress(g_tmp_triplets.as<triplet>(), mat.nnz, row_major, n_major, n_minor,
                           dptr.as<int>(), didx.as<int>(), dval.as<float>(), g_tmp_sort,
                           g_tmp_ptr64, &f2, s);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(ret.ptr, dptr.ptr, sizeof(int) * ((size_t)n_major + 1),
                            cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess && nnz)
        e = cudaMemcpyAsync(ret.idx, didx.ptr, sizeof(int) * nnz, cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess && nnz)
        e = cudaMemcpyAsync(ret.val, dval.ptr, sizeof(float) * nnz, cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) {
        LEGACY_FAIL(SPGEMM_ERR_CUDA, cudaGetErrorString(e));
        return ret;
      }
    }
  }
  cm dev = ret;
  dev.ptr = dptr.as<int>();
  dev.idx = didx.as<int>();
  dev.val = dval.as<float>();
  if (row_major) { g_B_dev = dev; g_have_b = true; }
  else { g_A_dev = dev; g_have_a = true; }
  g_have_c = false;
  return ret;
}

// Replaces reference src/mm.cu:150-193.
cm cudaInitGEMM(cm A, cm B) {
  g_status = SPGEMM_OK;
  cm C;
  cmInit(&C);
  cmSetType(&C, ROW_MAJOR);
  cmSetNumRows(&C, cmGetNumRows(A));
  cmSetNumCols(&C, cmGetNumCols(B));
  if (!g_have_a || !g_have_b) {
    LEGACY_FAIL(SPGEMM_ERR_STATE, "cudaInitGEMM: convert A (COL_MAJOR) and B (ROW_MAJOR) first");
    return C;
  }
  sg::Engine& E = eng();
  g_have_c = false;
  if (int r = E.analyze(g_A_dev, g_B_dev)) {
    LEGACY_FAIL(r, E.last_error().c_str());
    return C;
  }
  const long long p = E.intermediate_products();
  cmSetNNZ(&C, p > INT_MAX ? INT_MAX : (int)p);
  if (spgemm_internal_verbose()) printf("%lld %lld\n", p, p);
  return C;
}

// Replaces reference src/mm.cu:263-286. The engine bins rows while it
// computes P_i (k_row_analysis), so the bins already exist here.
void cudaCategorizeGEMM(cm A, cm B) {
  (void)A;
  (void)B;
  g_status = SPGEMM_OK;
}

// Replaces reference src/mm.cu:314-327: symbolic pass of every bin.
void cudaBinGEMM(cm A, cm B, cm C) {
  (void)A;
  (void)B;
  (void)C;
  g_status = SPGEMM_OK;
  sg::Engine& E = eng();
  long long nnz = 0;
  if (int r = E.symbolic_pass(&nnz)) LEGACY_FAIL(r, E.last_error().c_str());
}

// Replaces reference src/mm.cu:356-364. The reference's unbinned launch
// produces the same buckets as the binned one; here both run the same
// binned symbolic pass.
void cudaSimpleGEMM(cm A, cm B, cm C) { cudaBinGEMM(A, B, C); }

// Replaces reference src/mm.cu:407-450: numeric pass, then the reference's
// two printed counts (merged nnz and entries above 1e-4).
void cudaMergeGEMM(cm C) {
  (void)C;
  g_status = SPGEMM_OK;
  sg::Engine& E = eng();
  cm Cd;
  if (int r = E.multiply_numeric_owned(&Cd)) {
    LEGACY_FAIL(r, E.last_error().c_str());
    return;
  }
  g_have_c = true;
  if (spgemm_internal_verbose()) {
    unsigned long long* cnt = g_tmp_flag.as<unsigned long long>();
    cudaStream_t s = E.stream();
    unsigned long long above = 0;
    cudaError_t e = cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), s);
    if (e == cudaSuccess && Cd.nnz > 0) {
      k_count_above<<<1024, 256, 0, s>>>(Cd.val, Cd.nnz, 0.0001f, cnt);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(&above, cnt, sizeof(above), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
      LEGACY_FAIL(SPGEMM_ERR_CUDA, cudaGetErrorString(e));
      return;
    }
    printf("%d %llu\n", Cd.nnz, above);
  }
}

// Declared in the reference (lib/mm.h:23) without a definition, next to its
// DenseChunk type (lib/mm.h:10-15: a column index and 64 dense values): the
// dense-chunk strategy. Here: the whole product (symbolic and numeric pass)
// with rows accumulated in dense column windows wherever their column span
// allows -- the span-bitmap accumulator (a dense presence bitmap plus values
// in column order) for every fused row with span <= 2^18 instead of warp hash
// tables, and for long rows with few outputs instead of block hash tables.
// Rows wider than that keep the hash paths. The handle's own tuning is
// restored afterwards; the rows are re-binned for the product, so it may
// follow cudaInitGEMM directly or replace cudaBinGEMM + cudaMergeGEMM.
void cudaDCGEMM(cm A, cm B, cm C) {
  (void)A;
  (void)B;
  g_status = SPGEMM_OK;
  if (!g_have_a || !g_have_b) {
    LEGACY_FAIL(SPGEMM_ERR_STATE, "cudaDCGEMM: convert A (COL_MAJOR) and B (ROW_MAJOR) first");
    return;
  }
  sg::Engine& E = eng();
  const sg::Tuning saved = E.tuning();
  sg::Tuning dc = saved;
  dc.warp_p_max = 0;        // no warp hash rows
  dc.mid_cols = 1 << 18;    // dense windows up to 2^18 columns
  dc.mid_o_min = 0;         // long rows with few outputs: dense windows too
  if (int r = E.set_tuning(dc)) {
    LEGACY_FAIL(r, E.last_error().c_str());
    return;
  }
  g_have_c = false;
  if (int r = E.analyze(g_A_dev, g_B_dev)) {
    E.set_tuning(saved);
    LEGACY_FAIL(r, E.last_error().c_str());
    return;
  }
  cudaBinGEMM(A, B, C);
  if (g_status == SPGEMM_OK) cudaMergeGEMM(C);
  E.set_tuning(saved);
}

int spgemm_get_result(cm* out) {
  if (!out) return SPGEMM_ERR_INVALID;
  if (!g_have_c) return SPGEMM_ERR_STATE;
  sg::Engine& E = eng();
  const int m = E.m();
  const long long nnz = E.nnz_c();
  cm h;
  h.type = ROW_MAJOR;
  h.num_rows = m;
  h.num_cols = E.n();
  h.nnz = (int)nnz;
  h.ptr = host_alloc<int>((size_t)m + 1);
  h.idx = host_alloc<int>((size_t)nnz);
  h.val = host_alloc<float>((size_t)nnz);
  if (!h.ptr || !h.idx || !h.val) {
    free(h.ptr); free(h.idx); free(h.val);
    return SPGEMM_ERR_ALLOC;
  }
  cudaStream_t s = E.stream();
  cudaError_t e = cudaMemcpyAsync(h.ptr, E.out_rowptr(), sizeof(int) * ((size_t)m + 1),
                                  cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && nnz)
    e = cudaMemcpyAsync(h.idx, E.out_col(), sizeof(int) * (size_t)nnz, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && nnz)
    e = cudaMemcpyAsync(h.val, E.out_val(), sizeof(float) * (size_t)nnz, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    free(h.ptr); free(h.idx); free(h.val);
    return SPGEMM_ERR_CUDA;
  }
  *out = h;
  return SPGEMM_OK;
}

}  // extern "C"

// spGEMM.h entry family (reference lib/spGEMM.h:81-91, src/spGEMM.cu:704-1262)
// on top of the engine. The family keeps one product in module state, in the
// global variables the header declares (the reference declares them extern
// and defines none; they are defined here): the caller fills CSC_HOST (A) and
// CSR_HOST (B), the passes upload them, compute per-row product counts, find
// the heavy rows, run the engine's symbolic and numeric passes and gather C
// into c_ptr_h / c_idx_h / c_val_h with nnzC.
//
// Pass mapping (reference -> here):
//   cudaPass_ (upload, calcUpp row bounds :772-826)   -> upload, row analysis,
//                                                      exact P_i per row
//   cudaPath_find_thread_count_approx (k bins :704-770) -> row bins (taken in
//                                                      the row analysis)
//   cudaPass_F (dominator rows, findDom :835-904)     -> rows above the long-row
//                                                      threshold (column-sliced)
//   cudaPassB (binned expansion :906-1145)            -> symbolic pass (short rows
//                                                      computed in one fused pass)
//   cudaPassBB (2-D split of heavy products :1147-1180) -> numeric pass: heavy rows
//                                                      in column slices, C on device
//   cudaPassC (merge + gather :1182-1262)             -> C to the host
// The reference's calcUpp uses B's structure for A's rows (valid only for
// A*A); here A and B are independent n x n operands.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/spGEMM.h"
#include "../../include/spgemm_b200.h"
#include "engine.h"

extern "C" int spgemm_internal_verbose(void);
extern "C" int spgemm_internal_exit_on_error(void);
extern "C" void spgemm_internal_set_legacy_status(int s);

// ---- the globals of lib/spGEMM.h ----
extern "C" {
int subMatrixSize = 0;
int depth = 0;
int resCnt = 0;
coo COOC = {};
coo COOR = {};
int* CSC_RIDX_DEV = nullptr;
int* CSC_PTR_DEV = nullptr;
float* CSC_VAL_DEV = nullptr;
int* CSR_CIDX_DEV = nullptr;
int* CSR_PTR_DEV = nullptr;
float* CSR_VAL_DEV = nullptr;
int* RUPP_DEV = nullptr;
int* WLS_DEV = nullptr;
int* RBOX_DEV = nullptr;
PP* P_DEV = nullptr;
int* N_DEV = nullptr;
int* WLS_HOST = nullptr;
int* RUPP_HOST = nullptr;
PP* P_HOST = nullptr;
int* c_jdx_d = nullptr;
int* c_idx_d = nullptr;
float* c_val_d = nullptr;
int* c_ptr_d = nullptr;
int* c_idx_h = nullptr;
float* c_val_h = nullptr;
int* c_ptr_h = nullptr;
coo COO_HOST = {};
csc CSC_HOST = {};
csr CSR_HOST = {};
csr DCSR_HOST = {};
csc DCSC_HOST = {};
float t_pre = 0.f, t_fd = 0.f, t_spgemm_l = 0.f, t_spgemm_d = 0.f, t_merge = 0.f, t_bin = 0.f;
double t_cpu = 0.0;
int nnzC = 0;
int* domR = nullptr;
int* domN = nullptr;
int* domRC = nullptr;
int* domCC = nullptr;
int domRCavg = 0;
int domCCavg = 0;
}

namespace {

sg::Engine* g_eng = nullptr;
int g_n = 0;
bool g_analyzed = false, g_symbolic = false, g_numeric = false;

sg::Engine& eng() {
  if (!g_eng) g_eng = new sg::Engine();
  return *g_eng;
}

// Reference error path (src/spGEMM.cu:13-22 prints, src/mm.cu:6-14 exits):
// print and exit(-1) unless the caller switched exiting off
// (spgemm_set_exit_on_error, shared with the mm.h family).
void legacy_fail(int status, const char* file, int line, const char* msg) {
  spgemm_internal_set_legacy_status(status);
  printf("[%s:%d]CUDA ERROR : %s\n", file, line, msg);
  fflush(stdout);
  if (spgemm_internal_exit_on_error()) exit(-1);
}
#define LEGACY_FAIL(st, msg) legacy_fail((st), __FILE__, __LINE__, (msg))
#define LEGACY_CK(call, what)                                         \
  do {                                                                \
    cudaError_t e__ = (call);                                         \
    if (e__ != cudaSuccess) {                                         \
      LEGACY_FAIL(SPGEMM_ERR_CUDA, cudaGetErrorString(e__));          \
      return;                                                         \
    }                                                                 \
  } while (0)

// Per-row products (int64) to the int32 counts RUPP_DEV holds.
__global__ void k_clamp_counts(const long long* __restrict__ in, int n, int* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = (int)min(in[i], (long long)INT_MAX);
}

template <class T>
void dev_free(T*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

template <class T>
void host_free(T*& p) {
  free(p);
  p = nullptr;
}

struct Timer {
  cudaEvent_t a = nullptr, b = nullptr;
  Timer() {
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, 0);
  }
  float stop() {
    float ms = 0.f;
    cudaEventRecord(b, 0);
    cudaEventSynchronize(b);
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms;
  }
};

cm dev_a() {
  return cm{CSC_PTR_DEV, CSC_RIDX_DEV, CSC_VAL_DEV, CSC_HOST.e, g_n, g_n, (bool)COL_MAJOR};
}
cm dev_b() {
  return cm{CSR_PTR_DEV, CSR_CIDX_DEV, CSR_VAL_DEV, CSR_HOST.e, g_n, g_n, (bool)ROW_MAJOR};
}

}  // namespace

extern "C" {

void cudaPass_(int n, int e) {
  (void)e;  // each operand's own entry count (CSC_HOST.e, CSR_HOST.e) is used
  g_analyzed = g_symbolic = g_numeric = false;
  if (n < 0 || !CSC_HOST.header || !CSR_HOST.header || CSC_HOST.e < 0 || CSR_HOST.e < 0 ||
      (CSC_HOST.e > 0 && (!CSC_HOST.ridx || !CSC_HOST.val)) ||
      (CSR_HOST.e > 0 && (!CSR_HOST.cidx || !CSR_HOST.val))) {
    LEGACY_FAIL(SPGEMM_ERR_INVALID, "cudaPass_: CSC_HOST / CSR_HOST not set up");
    return;
  }
  g_n = n;
  Timer tm;
  dev_free(CSC_RIDX_DEV); dev_free(CSC_PTR_DEV); dev_free(CSC_VAL_DEV);
  dev_free(CSR_CIDX_DEV); dev_free(CSR_PTR_DEV); dev_free(CSR_VAL_DEV);
  dev_free(RUPP_DEV); dev_free(WLS_DEV); dev_free(N_DEV);
  const size_t ea = (size_t)std::max(CSC_HOST.e, 1), eb = (size_t)std::max(CSR_HOST.e, 1);
  LEGACY_CK(cudaMalloc(&CSC_PTR_DEV, sizeof(int) * ((size_t)n + 1)), "alloc");
  LEGACY_CK(cudaMalloc(&CSC_RIDX_DEV, sizeof(int) * ea), "alloc");
  LEGACY_CK(cudaMalloc(&CSC_VAL_DEV, sizeof(float) * ea), "alloc");
  LEGACY_CK(cudaMalloc(&CSR_PTR_DEV, sizeof(int) * ((size_t)n + 1)), "alloc");
  LEGACY_CK(cudaMalloc(&CSR_CIDX_DEV, sizeof(int) * eb), "alloc");
  LEGACY_CK(cudaMalloc(&CSR_VAL_DEV, sizeof(float) * eb), "alloc");
  LEGACY_CK(cudaMalloc(&RUPP_DEV, sizeof(int) * ((size_t)n + 1)), "alloc");
  LEGACY_CK(cudaMalloc(&WLS_DEV, sizeof(int) * ((size_t)n + 1)), "alloc");
  LEGACY_CK(cudaMalloc(&N_DEV, sizeof(int)), "alloc");
  LEGACY_CK(cudaMemcpy(CSC_PTR_DEV, CSC_HOST.header, sizeof(int) * ((size_t)n + 1),
                       cudaMemcpyHostToDevice), "copy A");
  if (CSC_HOST.e > 0) {
    LEGACY_CK(cudaMemcpy(CSC_RIDX_DEV, CSC_HOST.ridx, sizeof(int) * CSC_HOST.e,
                         cudaMemcpyHostToDevice), "copy A");
    LEGACY_CK(cudaMemcpy(CSC_VAL_DEV, CSC_HOST.val, sizeof(float) * CSC_HOST.e,
                         cudaMemcpyHostToDevice), "copy A");
  }
  LEGACY_CK(cudaMemcpy(CSR_PTR_DEV, CSR_HOST.header, sizeof(int) * ((size_t)n + 1),
                       cudaMemcpyHostToDevice), "copy B");
  if (CSR_HOST.e > 0) {
    LEGACY_CK(cudaMemcpy(CSR_CIDX_DEV, CSR_HOST.cidx, sizeof(int) * CSR_HOST.e,
                         cudaMemcpyHostToDevice), "copy B");
    LEGACY_CK(cudaMemcpy(CSR_VAL_DEV, CSR_HOST.val, sizeof(float) * CSR_HOST.e,
                         cudaMemcpyHostToDevice), "copy B");
  }
  LEGACY_CK(cudaMemcpy(N_DEV, &n, sizeof(int), cudaMemcpyHostToDevice), "copy n");

  // per-k workloads nnz(A(:,k)) * nnz(B(k,:))
  if (WLS_HOST) cudaFreeHost(WLS_HOST);
  WLS_HOST = nullptr;
  LEGACY_CK(cudaMallocHost(&WLS_HOST, sizeof(int) * ((size_t)n + 1)), "alloc WLS_HOST");
  for (int k = 0; k < n; ++k) {
    const long long w = (long long)(CSC_HOST.header[k + 1] - CSC_HOST.header[k]) *
                        (CSR_HOST.header[k + 1] - CSR_HOST.header[k]);
    WLS_HOST[k] = (int)std::min<long long>(w, INT_MAX);
  }
  WLS_HOST[n] = 0;
  LEGACY_CK(cudaMemcpy(WLS_DEV, WLS_HOST, sizeof(int) * ((size_t)n + 1), cudaMemcpyHostToDevice),
            "copy WLS");

  // row analysis: exact products per row of C
  sg::Engine& E = eng();
  E.set_stream(nullptr);
  if (int r = E.analyze(dev_a(), dev_b())) {
    LEGACY_FAIL(r, E.last_error().c_str());
    return;
  }
  if (n > 0) {
    k_clamp_counts<<<std::min((n + 255) / 256, 4096), 256>>>(E.row_products(), n, RUPP_DEV);
    LEGACY_CK(cudaGetLastError(), "k_clamp_counts");
  }
  host_free(RUPP_HOST);
  RUPP_HOST = static_cast<int*>(malloc(sizeof(int) * ((size_t)n + 1)));
  if (!RUPP_HOST) {
    LEGACY_FAIL(SPGEMM_ERR_ALLOC, "malloc RUPP_HOST");
    return;
  }
  RUPP_HOST[0] = 0;
  if (n > 0)
    LEGACY_CK(cudaMemcpy(RUPP_HOST + 1, RUPP_DEV, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost),
              "read RUPP");
  t_pre = tm.stop();
  g_analyzed = true;
}

void cudaPath_find_thread_count_approx(int n) {
  (void)n;
  // rows were binned by their work during the row analysis of cudaPass_
  if (!g_analyzed) {
    LEGACY_FAIL(SPGEMM_ERR_STATE, "cudaPath_find_thread_count_approx before cudaPass_");
    return;
  }
  t_bin = 0.f;
}

void cudaPass_F(int n) {
  (void)n;
  if (!g_analyzed) {
    LEGACY_FAIL(SPGEMM_ERR_STATE, "cudaPass_F before cudaPass_");
    return;
  }
  Timer tm;
  sg::Engine& E = eng();
  const int cnt = E.sym_bin_rows(sg::FB_LONG);
  host_free(domR); host_free(domN); host_free(domRC); host_free(domCC);
  domN = static_cast<int*>(malloc(sizeof(int)));
  domR = static_cast<int*>(malloc(sizeof(int) * (size_t)std::max(cnt, 1)));
  domRC = static_cast<int*>(malloc(sizeof(int) * (size_t)std::max(cnt, 1)));
  domCC = static_cast<int*>(malloc(sizeof(int) * (size_t)std::max(cnt, 1)));
  if (!domN || !domR || !domRC || !domCC) {
    LEGACY_FAIL(SPGEMM_ERR_ALLOC, "malloc heavy-row lists");
    return;
  }
  domN[0] = cnt;
  domRCavg = domCCavg = 0;
  if (cnt > 0) {
    LEGACY_CK(cudaMemcpy(domR, E.bin_list(sg::FB_LONG), sizeof(int) * (size_t)cnt,
                         cudaMemcpyDeviceToHost), "read heavy rows");
    std::sort(domR, domR + cnt);
    std::vector<int> aptr((size_t)g_n + 1);
    LEGACY_CK(cudaMemcpy(aptr.data(), E.a_rowptr(), sizeof(int) * ((size_t)g_n + 1),
                         cudaMemcpyDeviceToHost), "read A rows");
    long long sr = 0, sc = 0;
    for (int j = 0; j < cnt; ++j) {
      const int i = domR[j];
      domRC[j] = aptr[i + 1] - aptr[i];
      domCC[j] = RUPP_HOST[i + 1];
      sr += domRC[j];
      sc += domCC[j];
    }
    domRCavg = (int)(sr / cnt);
    domCCavg = (int)(sc / cnt);
  }
  t_fd = tm.stop();
}

void cudaPassB(int n) {
  (void)n;
  if (!g_analyzed) {
    LEGACY_FAIL(SPGEMM_ERR_STATE, "cudaPassB before cudaPass_");
    return;
  }
  Timer tm;
  sg::Engine& E = eng();
  long long nnz = 0;
  if (int r = E.symbolic_pass(&nnz)) {
    LEGACY_FAIL(r, E.last_error().c_str());
    return;
  }
  nnzC = (int)nnz;
  t_spgemm_l = tm.stop();
  g_symbolic = true;
}

void cudaPassBB(int n, int t) {
  (void)t;  // slice shapes come from the engine's tuning
  if (!g_symbolic) {
    LEGACY_FAIL(SPGEMM_ERR_STATE, "cudaPassBB before cudaPassB");
    return;
  }
  Timer tm;
  sg::Engine& E = eng();
  dev_free(c_ptr_d); dev_free(c_idx_d); dev_free(c_val_d); dev_free(c_jdx_d);
  const size_t nz = (size_t)std::max(nnzC, 1);
  LEGACY_CK(cudaMalloc(&c_ptr_d, sizeof(int) * ((size_t)n + 1)), "alloc C");
  LEGACY_CK(cudaMalloc(&c_idx_d, sizeof(int) * nz), "alloc C");
  LEGACY_CK(cudaMalloc(&c_val_d, sizeof(float) * nz), "alloc C");
  if (int r = E.numeric(c_ptr_d, c_idx_d, c_val_d)) {
    LEGACY_FAIL(r, E.last_error().c_str());
    return;
  }
  t_spgemm_d = tm.stop();
  g_numeric = true;
}

void cudaPassC(int n) {
  if (!g_numeric) {
    LEGACY_FAIL(SPGEMM_ERR_STATE, "cudaPassC before cudaPassBB");
    return;
  }
  Timer tm;
  host_free(c_ptr_h); host_free(c_idx_h); host_free(c_val_h);
  const size_t nz = (size_t)std::max(nnzC, 1);
  c_ptr_h = static_cast<int*>(malloc(sizeof(int) * ((size_t)n + 1)));
  c_idx_h = static_cast<int*>(malloc(sizeof(int) * nz));
  c_val_h = static_cast<float*>(malloc(sizeof(float) * nz));
  if (!c_ptr_h || !c_idx_h || !c_val_h) {
    LEGACY_FAIL(SPGEMM_ERR_ALLOC, "malloc C");
    return;
  }
  LEGACY_CK(cudaMemcpy(c_ptr_h, c_ptr_d, sizeof(int) * ((size_t)n + 1), cudaMemcpyDeviceToHost),
            "read C");
  if (nnzC > 0) {
    LEGACY_CK(cudaMemcpy(c_idx_h, c_idx_d, sizeof(int) * (size_t)nnzC, cudaMemcpyDeviceToHost),
              "read C");
    LEGACY_CK(cudaMemcpy(c_val_h, c_val_d, sizeof(float) * (size_t)nnzC, cudaMemcpyDeviceToHost),
              "read C");
  }
  t_merge = tm.stop();
  // the reference prints its dominator-row count here (src/spGEMM.cu:1227)
  if (spgemm_internal_verbose()) printf("%d\n", domN ? domN[0] : 0);
}

void cudaPass0(int n, int e) {
  cudaPass_(n, e);
  if (!g_analyzed) return;
  cudaPath_find_thread_count_approx(n);
  cudaPass_F(n);
}

int cudaPass2(void) {
  if (!g_analyzed) {
    LEGACY_FAIL(SPGEMM_ERR_STATE, "cudaPass2 before cudaPass0");
    return -1;
  }
  cudaPassB(g_n);
  if (!g_symbolic) return -1;
  cudaPassBB(g_n, 0);
  if (!g_numeric) return -1;
  cudaPassC(g_n);
  return nnzC;
}

// The workload tables describe a decomposition of the products into per-k
// outer products (wlt: one record per k, lib/wlt.h:10-23) and, with `cheat`,
// into 2-D tiles of heavy outer products (wlt_cheat: first A entry ridx and
// first B entry cidx of each tile, the pairs calcInterDom works on,
// src/spGEMM.cu:543-589). C = A*B does not depend on how the products are
// decomposed, and the engine derives its own per-row decomposition, so the
// tables steer nothing here; but a table that does not describe these
// operands means the caller's picture of the product is wrong, so it is
// checked and rejected. An empty table (null data or zero records) is not
// checked. Returns an empty string when the tables are consistent.
static std::string check_wlt(const csc& A, const csr& B, const wlt& W) {
  if (!W.data || W.threadblocks <= 0) return "";
  const int n = A.n;
  std::vector<char> seen((size_t)n, 0);
  long long total = 0;
  for (int t = 0; t < W.threadblocks; ++t) {
    const wltData& d = W.data[t];
    if (d.idx < 0 || d.idx >= n) return "wlt record " + std::to_string(t) + ": k out of range";
    if (seen[d.idx]) return "wlt record " + std::to_string(t) + ": k listed twice";
    seen[d.idx] = 1;
    const int ca = A.header[d.idx + 1] - A.header[d.idx];
    const int rb = B.header[d.idx + 1] - B.header[d.idx];
    if (d.num_of_col_elements != ca || d.num_of_row_elements != rb)
      return "wlt record " + std::to_string(t) + ": element counts differ from the operands";
    total += (long long)ca * rb;
  }
  for (int k = 0; k < n; ++k)
    if (!seen[k] && (long long)(A.header[k + 1] - A.header[k]) * (B.header[k + 1] - B.header[k]) > 0)
      return "wlt: the outer product of k = " + std::to_string(k) + " is missing";
  if (total <= INT_MAX && W.workloads != (int)total) return "wlt: workloads differs from the product count";
  return "";
}

// Every tile must lie inside one outer product, and the tiles of an outer
// product must cover it exactly (their areas add up to nnz(A(:,k)) *
// nnz(B(k,:)) and no two tiles overlap).
static std::string check_wlt_cheat(const csc& A, const csr& B, const wlt_cheat& T) {
  if (!T.data || T.threadblocks <= 0) return "";
  struct Tile { int k, r0, r1, c0, c1; };
  std::vector<Tile> tiles;
  tiles.reserve((size_t)T.threadblocks);
  for (int t = 0; t < T.threadblocks; ++t) {
    const wltData_cheat& d = T.data[t];
    if (d.ridx < 0 || d.ridx >= A.e || d.num_of_col_elements <= 0 || d.num_of_row_elements <= 0)
      return "wlt_cheat tile " + std::to_string(t) + ": empty or out of range";
    // column k of A holding entry ridx
    const int k = (int)(std::upper_bound(A.header, A.header + A.n + 1, d.ridx) - A.header) - 1;
    if (k < 0 || k >= A.n || d.ridx + d.num_of_col_elements > A.header[k + 1])
      return "wlt_cheat tile " + std::to_string(t) + ": A entries leave column k";
    if (d.cidx < B.header[k] || d.cidx + d.num_of_row_elements > B.header[k + 1])
      return "wlt_cheat tile " + std::to_string(t) + ": B entries leave row k";
    tiles.push_back(Tile{k, d.ridx, d.ridx + d.num_of_col_elements, d.cidx,
                         d.cidx + d.num_of_row_elements});
  }
  std::sort(tiles.begin(), tiles.end(), [](const Tile& a, const Tile& b) {
    return a.k != b.k ? a.k < b.k : (a.r0 != b.r0 ? a.r0 < b.r0 : a.c0 < b.c0);
  });
  for (size_t s = 0; s < tiles.size();) {
    size_t e = s;
    long long area = 0;
    const int k = tiles[s].k;
    while (e < tiles.size() && tiles[e].k == k) {
      area += (long long)(tiles[e].r1 - tiles[e].r0) * (tiles[e].c1 - tiles[e].c0);
      ++e;
    }
    const long long full = (long long)(A.header[k + 1] - A.header[k]) * (B.header[k + 1] - B.header[k]);
    if (area != full) return "wlt_cheat: the tiles of k = " + std::to_string(k) + " do not cover it";
    for (size_t x = s; x < e; ++x)  // pairwise overlap test inside one outer product
      for (size_t y = x + 1; y < e && tiles[y].r0 < tiles[x].r1; ++y)
        if (tiles[y].c0 < tiles[x].c1 && tiles[x].c0 < tiles[y].c1)
          return "wlt_cheat: overlapping tiles in k = " + std::to_string(k);
    s = e;
  }
  return "";
}

int spGEMM(csc CSC, csr CSR, wlt WLT, wlt_cheat WLT_C, int cheat) {
  if (CSC.n != CSR.n) {
    LEGACY_FAIL(SPGEMM_ERR_INVALID, "spGEMM: A and B must both be n x n");
    return -1;
  }
  if (!CSC.header || !CSR.header || CSC.n < 0) {
    LEGACY_FAIL(SPGEMM_ERR_INVALID, "spGEMM: null pointer array");
    return -1;
  }
  std::string bad = check_wlt(CSC, CSR, WLT);
  if (bad.empty() && cheat) bad = check_wlt_cheat(CSC, CSR, WLT_C);
  if (!bad.empty()) {
    LEGACY_FAIL(SPGEMM_ERR_INVALID, ("spGEMM: " + bad).c_str());
    return -1;
  }
  CSC_HOST = CSC;
  CSR_HOST = CSR;
  cudaPass0(CSC.n, CSC.e);
  if (!g_analyzed) return -1;
  return cudaPass2();
}

}  // extern "C"

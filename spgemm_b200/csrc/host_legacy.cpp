// Host helpers of the legacy spGEMM() family: csc / csr containers and the
// per-k workload tables of wlt.h. The reference declares all of these
// (lib/csc.h:21-24, lib/wlt.h:46-60) and ships no bodies, so the semantics
// below are this library's, chosen to serve the legacy engine entry points:
//
//  * transformCOOToCSC / transformCOOToCSR build the compressed form of a
//    COO matrix (n = number of columns / rows);
//  * makeWLT lists every k with a non-empty outer product A(:,k) * B(k,:),
//    heaviest first, with base_idx = offset of its first partial product in
//    k order (the bucket offsets the reference computes on the GPU,
//    src/spGEMM.cu:51-76);
//  * makeWLT_cheat splits every outer product of at least `min_work`
//    products into tiles of at most `tile_rows` A entries x `tile_cols` B
//    entries -- the 2-D split of calcInterDom (src/spGEMM.cu:543-589);
//  * extractCOOR / extractCOOC keep the entries whose row / column index is
//    listed in a workload table.
#include <algorithm>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/coo.h"
#include "../../include/csc.h"
#include "../../include/csr.h"
#include "../../include/wlt.h"

extern "C" {

int maxWL = 0;

void initCSC(csc* mat) {
  mat->header = nullptr;
  mat->ridx = nullptr;
  mat->val = nullptr;
  mat->n = 0;
  mat->e = 0;
}

void freeCSC(csc* mat) {
  free(mat->header);
  free(mat->ridx);
  free(mat->val);
  initCSC(mat);
}

void dumpCSC(csc m) {
  printf("CSC %d %d\n", m.n, m.e);
  for (int c = 0; c < m.n; ++c)
    for (int j = m.header[c]; j < m.header[c + 1]; ++j)
      printf("%d\t%d\t%f\n", m.ridx[j], c, m.val[j]);
}

void initCSR(csr* mat) {
  mat->header = nullptr;
  mat->cidx = nullptr;
  mat->val = nullptr;
  mat->n = 0;
  mat->e = 0;
}

void freeCSR(csr* mat) {
  free(mat->header);
  free(mat->cidx);
  free(mat->val);
  initCSR(mat);
}

void dumpCSR(csr m) {
  printf("CSR %d %d\n", m.n, m.e);
  for (int r = 0; r < m.n; ++r)
    for (int j = m.header[r]; j < m.header[r + 1]; ++j)
      printf("%d\t%d\t%f\n", r, m.cidx[j], m.val[j]);
}

// Counting sort by the major index, stable in the input order, then each
// major segment sorted by the minor index.
static void compress(const coo& mat, bool by_row, int n_major, int** header, int** minor,
                     float** val) {
  const int nnz = std::max(mat.nnz, 0);
  *header = static_cast<int*>(calloc((size_t)n_major + 1, sizeof(int)));
  *minor = static_cast<int*>(malloc(sizeof(int) * (size_t)std::max(nnz, 1)));
  *val = static_cast<float*>(malloc(sizeof(float) * (size_t)std::max(nnz, 1)));
  int* h = *header;
  for (int e = 0; e < nnz; ++e) {
    const int k = by_row ? mat.data[e].ridx : mat.data[e].cidx;
    if (k >= 0 && k < n_major) h[k + 1]++;
  }
  for (int i = 0; i < n_major; ++i) h[i + 1] += h[i];
  std::vector<int> cur(h, h + n_major);
  for (int e = 0; e < nnz; ++e) {
    const int k = by_row ? mat.data[e].ridx : mat.data[e].cidx;
    if (k < 0 || k >= n_major) continue;
    const int p = cur[k]++;
    (*minor)[p] = by_row ? mat.data[e].cidx : mat.data[e].ridx;
    (*val)[p] = mat.data[e].val;
  }
  std::vector<std::pair<int, float>> seg;
  for (int i = 0; i < n_major; ++i) {
    seg.clear();
    for (int j = h[i]; j < h[i + 1]; ++j) seg.emplace_back((*minor)[j], (*val)[j]);
    std::stable_sort(seg.begin(), seg.end(),
                     [](const std::pair<int, float>& a, const std::pair<int, float>& b) {
                       return a.first < b.first;
                     });
    for (size_t q = 0; q < seg.size(); ++q) {
      (*minor)[h[i] + (int)q] = seg[q].first;
      (*val)[h[i] + (int)q] = seg[q].second;
    }
  }
}

csc transformCOOToCSC(coo mat) {
  csc out;
  initCSC(&out);
  out.n = mat.num_cols;
  compress(mat, false, out.n, &out.header, &out.ridx, &out.val);
  out.e = out.header[out.n];
  return out;
}

csr transformCOOToCSR(coo mat) {
  csr out;
  initCSR(&out);
  out.n = mat.num_rows;
  compress(mat, true, out.n, &out.header, &out.cidx, &out.val);
  out.e = out.header[out.n];
  return out;
}

void buildIdxWLT(int n) {
  (void)n;
  maxWL = 0;
}

void freeWLT(wlt* t) {
  free(t->data);
  t->data = nullptr;
  t->threadblocks = 0;
  t->workloads = 0;
}

void freeWLTC(wlt_cheat* t) {
  free(t->data);
  t->data = nullptr;
  t->threadblocks = 0;
  t->workloads = 0;
}

static long long work_of(int rows, int cols) { return (long long)rows * cols; }

// Heaviest outer product first; ties by k.
int wltDataCompare(const void* a, const void* b) {
  const wltData* x = static_cast<const wltData*>(a);
  const wltData* y = static_cast<const wltData*>(b);
  const long long wx = work_of(x->num_of_row_elements, x->num_of_col_elements);
  const long long wy = work_of(y->num_of_row_elements, y->num_of_col_elements);
  if (wx != wy) return wx > wy ? -1 : 1;
  return (x->idx > y->idx) - (x->idx < y->idx);
}

int wltDataCompare_cheat(const void* a, const void* b) {
  const wltData_cheat* x = static_cast<const wltData_cheat*>(a);
  const wltData_cheat* y = static_cast<const wltData_cheat*>(b);
  const long long wx = work_of(x->num_of_row_elements, x->num_of_col_elements);
  const long long wy = work_of(y->num_of_row_elements, y->num_of_col_elements);
  if (wx != wy) return wx > wy ? -1 : 1;
  if (x->cidx != y->cidx) return (x->cidx > y->cidx) - (x->cidx < y->cidx);
  return (x->base_idx > y->base_idx) - (x->base_idx < y->base_idx);
}

static int clamp_int(long long v) { return v > INT_MAX ? INT_MAX : (int)v; }

wlt makeWLT(csc A, csr B) {
  wlt t;
  t.data = nullptr;
  t.threadblocks = 0;
  t.workloads = 0;
  const int n = std::min(A.n, B.n);
  std::vector<wltData> rows;
  long long base = 0;
  maxWL = 0;
  for (int k = 0; k < n; ++k) {
    const int ca = A.header[k + 1] - A.header[k];
    const int rb = B.header[k + 1] - B.header[k];
    const long long w = work_of(ca, rb);
    if (w == 0) continue;
    rows.push_back(wltData{k, clamp_int(base), rb, ca});
    base += w;
    maxWL = std::max(maxWL, clamp_int(w));
  }
  std::sort(rows.begin(), rows.end(), [](const wltData& a, const wltData& b) {
    return wltDataCompare(&a, &b) < 0;
  });
  t.threadblocks = (int)rows.size();
  t.workloads = clamp_int(base);
  t.data = static_cast<wltData*>(malloc(sizeof(wltData) * std::max<size_t>(rows.size(), 1)));
  if (!rows.empty()) memcpy(t.data, rows.data(), sizeof(wltData) * rows.size());
  return t;
}

wlt_cheat makeWLT_cheat(csc A, csr B, int tile_rows, int tile_cols, int min_work) {
  wlt_cheat t;
  t.data = nullptr;
  t.threadblocks = 0;
  t.workloads = 0;
  if (tile_rows <= 0) tile_rows = 1;
  if (tile_cols <= 0) tile_cols = 1;
  const int n = std::min(A.n, B.n);
  std::vector<wltData_cheat> tiles;
  long long base = 0, total = 0;
  for (int k = 0; k < n; ++k) {
    const int ca = A.header[k + 1] - A.header[k];
    const int rb = B.header[k + 1] - B.header[k];
    const long long w = work_of(ca, rb);
    if (w > 0 && w >= min_work) {
      for (int r0 = 0; r0 < ca; r0 += tile_rows)
        for (int c0 = 0; c0 < rb; c0 += tile_cols) {
          const int h = std::min(tile_rows, ca - r0), wd = std::min(tile_cols, rb - c0);
          // ridx / cidx: first A entry and first B entry of the tile
          tiles.push_back(wltData_cheat{A.header[k] + r0, B.header[k] + c0, clamp_int(base), wd, h});
          base += work_of(h, wd);
        }
      total += w;
    }
  }
  t.threadblocks = (int)tiles.size();
  t.workloads = clamp_int(total);
  t.data = static_cast<wltData_cheat*>(
      malloc(sizeof(wltData_cheat) * std::max<size_t>(tiles.size(), 1)));
  if (!tiles.empty()) memcpy(t.data, tiles.data(), sizeof(wltData_cheat) * tiles.size());
  return t;
}

static coo extract(coo mat, const wltData* w, int cnt, bool by_row) {
  int lim = 0;
  for (int i = 0; i < cnt; ++i) lim = std::max(lim, w[i].idx + 1);
  std::vector<char> keep((size_t)std::max(lim, 1), 0);
  for (int i = 0; i < cnt; ++i)
    if (w[i].idx >= 0) keep[w[i].idx] = 1;
  coo out;
  initCOO(&out);
  out.num_rows = mat.num_rows;
  out.num_cols = mat.num_cols;
  out.type = mat.type;
  out.data = static_cast<triplet*>(malloc(sizeof(triplet) * (size_t)std::max(mat.nnz, 1)));
  int k = 0;
  for (int e = 0; e < mat.nnz; ++e) {
    const int key = by_row ? mat.data[e].ridx : mat.data[e].cidx;
    if (key >= 0 && key < lim && keep[key]) out.data[k++] = mat.data[e];
  }
  out.nnz = k;
  return out;
}

coo extractCOOR(coo mat, wltData* WLTD, int cnt) { return extract(mat, WLTD, cnt, true); }
coo extractCOOC(coo mat, wltData* WLTD, int cnt) { return extract(mat, WLTD, cnt, false); }

}  // extern "C"

// COO helpers and Matrix-Market readers with the reference's observable
// behaviour (reference src/coo.cpp). Arrays are allocated with malloc so that
// freeCOO (free) releases them correctly; the reference allocates with
// new[] (src/coo.cpp:32,93,133,136) and frees with free() (src/coo.cpp:17).
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "../../include/coo.h"

extern "C" int spgemm_internal_verbose(void);

extern "C" {

// ref src/coo.cpp:6-13
void initCOO(coo* mat) {
  mat->data = nullptr;
  mat->nnz = 0;
  mat->num_cols = 0;
  mat->num_rows = 0;
  mat->type = ROW_MAJOR;
}

// ref src/coo.cpp:15-22. Also clears the data pointer (the reference leaves
// it dangling).
void freeCOO(coo* mat) {
  free(mat->data);
  mat->data = nullptr;
  mat->nnz = 0;
  mat->num_cols = 0;
  mat->num_rows = 0;
  mat->type = ROW_MAJOR;
}

// ref src/coo.cpp:24-36. The reference leaves the copy's `type`
// uninitialised; here it is copied.
coo copyCOO(coo mat) {
  coo out;
  out.nnz = mat.nnz;
  out.num_cols = mat.num_cols;
  out.num_rows = mat.num_rows;
  out.type = mat.type;
  out.data = nullptr;
  if (mat.nnz > 0) {
    out.data = static_cast<triplet*>(malloc(sizeof(triplet) * (size_t)mat.nnz));
    if (out.data) memcpy(out.data, mat.data, sizeof(triplet) * (size_t)mat.nnz);
  }
  return out;
}

// ref src/coo.cpp:38-41
void setCOOtype(coo* mat, bool type) { mat->type = type; }

// ref src/coo.cpp:43-79: ROW_MAJOR orders by (row, column, value),
// COL_MAJOR by (column, row, value). Entries with distinct coordinates end
// in the same order as the reference's qsort; exact duplicates are ordered
// by value.
void sortCOO(coo mat) {
  if (mat.nnz <= 1 || !mat.data) return;
  triplet* b = mat.data;
  triplet* e = mat.data + mat.nnz;
  if (mat.type == ROW_MAJOR) {
    std::sort(b, e, [](const triplet& x, const triplet& y) {
      if (x.ridx != y.ridx) return x.ridx < y.ridx;
      if (x.cidx != y.cidx) return x.cidx < y.cidx;
      return x.val < y.val;
    });
  } else {
    std::sort(b, e, [](const triplet& x, const triplet& y) {
      if (x.cidx != y.cidx) return x.cidx < y.cidx;
      if (x.ridx != y.ridx) return x.ridx < y.ridx;
      return x.val < y.val;
    });
  }
}

// ref src/coo.cpp:82-108. Text format: "dim n nnz" then nnz lines of
// "row col [value]"; indices are stored as read (no 1-based shift),
// num_rows = num_cols = n, and the value is 1.1 when dim == 2.
void readCOO(coo* mat, char* path) {
  FILE* fp = fopen(path, "r");
  if (!fp) {
    fprintf(stderr, "readCOO: cannot open %s\n", path);
    return;
  }
  int dim = 0;
  if (fscanf(fp, "%d", &dim) != 1 || fscanf(fp, "%d", &mat->num_cols) != 1 ||
      fscanf(fp, "%d", &mat->nnz) != 1) {
    fclose(fp);
    return;
  }
  mat->num_rows = mat->num_cols;
  mat->data = static_cast<triplet*>(malloc(sizeof(triplet) * (size_t)std::max(mat->nnz, 1)));
  for (int i = 0; i < mat->nnz; ++i) {
    int r = 0, c = 0;
    if (fscanf(fp, "%d", &r) != 1) r = 0;
    if (fscanf(fp, "%d", &c) != 1) c = 0;
    mat->data[i].ridx = r;
    mat->data[i].cidx = c;
    if (dim == 2) {
      mat->data[i].val = 1.1f;
    } else if (fscanf(fp, "%f", &mat->data[i].val) != 1) {
      mat->data[i].val = 0.f;
    }
  }
  fclose(fp);
}

// ref src/coo.cpp:110-173. Observable behaviour kept:
//  * the banner is the first line (read in 100-byte pieces); "symmetric"
//    anywhere in it mirrors off-diagonal entries;
//  * the first token of the size line goes to num_cols, the second to
//    num_rows;
//  * every entry gets the value 1.1 -- the file's values are ignored;
//  * entries are read as "%d %d %s": a pattern file (no value column)
//    therefore misparses exactly as in the reference;
//  * "0 num_cols num_rows" is printed after the size line.
// Guarded against a missing file, over-long tokens, more entries than the
// size line declares (undefined behaviour in the reference) and a token that
// is not an integer (an endless loop in the reference). A partial match
// (1 or 2 fields) still stores an entry, as in the reference.
void readMTX(coo* mat, char* path) {
  FILE* fp = fopen(path, "r");
  if (!fp) {
    fprintf(stderr, "readMTX: cannot open %s\n", path);
    return;
  }
  char line[100];
  int sym = 0;
  if (!fgets(line, 100, fp)) { fclose(fp); return; }
  if (strstr(line, "symmetric")) sym = 1;
  for (;;) {
    if (!fgets(line, 100, fp)) { fclose(fp); return; }
    if (line[0] != '%') break;
  }
  mat->nnz = 0;
  char* t0 = strtok(line, " \n\t");
  char* t1 = t0 ? strtok(nullptr, " \n\t") : nullptr;
  char* t2 = t1 ? strtok(nullptr, " \n\t") : nullptr;
  mat->num_cols = t0 ? atoi(t0) : 0;
  mat->num_rows = t1 ? atoi(t1) : 0;
  const int max_nnz = t2 ? atoi(t2) : 0;
  size_t cap = (size_t)std::max(max_nnz, 0) * (sym ? 2 : 1);
  if (cap == 0) cap = 2;
  mat->data = static_cast<triplet*>(malloc(sizeof(triplet) * cap));
  if (spgemm_internal_verbose()) printf("%d %d %d\n", mat->nnz, mat->num_cols, mat->num_rows);
  int r = 0, c = 0;
  char dummy[200];
  size_t i = 0;
  for (;;) {
    const int got = fscanf(fp, "%d %d %199s ", &r, &c, dummy);
    if (got == EOF) break;
    if (got == 0) break;  // unparsable token: the reference would loop forever here
    const size_t need = i + ((sym && r != c) ? 2 : 1);
    if (need > cap) {
      size_t ncap = cap * 2 + 2;
      triplet* nd = static_cast<triplet*>(realloc(mat->data, sizeof(triplet) * ncap));
      if (!nd) break;
      mat->data = nd;
      cap = ncap;
    }
    mat->data[i].ridx = r - 1;
    mat->data[i].cidx = c - 1;
    mat->data[i].val = 1.1f;
    ++i;
    if (sym && r != c) {
      mat->data[i].ridx = c - 1;
      mat->data[i].cidx = r - 1;
      mat->data[i].val = 1.1f;
      ++i;
    }
  }
  mat->nnz = (int)i;
  fclose(fp);
}

}  // extern "C"

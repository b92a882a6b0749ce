// CompressedMatrix helpers (reference src/cm.cpp).
#include <cstdio>
#include <cstdlib>

#include "../../include/cm.h"

extern "C" {

// ref src/cm.cpp:7-16
void cmInit(cm* mat) {
  mat->ptr = nullptr;
  mat->idx = nullptr;
  mat->val = nullptr;
  mat->nnz = 0;
  mat->num_cols = 0;
  mat->num_rows = 0;
  mat->type = ROW_MAJOR;
}

// ref src/cm.cpp:18-31: frees with free(); arrays handed out by this
// library are malloc'd.
void cmFree(cm* mat) {
  free(mat->ptr);
  free(mat->idx);
  free(mat->val);
  mat->ptr = nullptr;
  mat->idx = nullptr;
  mat->val = nullptr;
  mat->nnz = 0;
  mat->num_cols = 0;
  mat->num_rows = 0;
  mat->type = ROW_MAJOR;
}

int cmGetNumRows(cm mat) { return mat.num_rows; }                     // ref :34-37
int cmGetNumCols(cm mat) { return mat.num_cols; }                     // ref :38-41
int cmGetNNZ(cm mat) { return mat.nnz; }                              // ref :42-45
void cmSetNumRows(cm* mat, int num_rows) { mat->num_rows = num_rows; }  // ref :47-50
void cmSetNumCols(cm* mat, int num_cols) { mat->num_cols = num_cols; }  // ref :51-54
void cmSetNNZ(cm* mat, int nnz) { mat->nnz = nnz; }                   // ref :55-58
void cmSetType(cm* mat, bool type) { mat->type = type; }              // ref :59-62

// ref src/cm.cpp:65-89: header "CSR cols rows nnz" or "CSC cols rows nnz",
// then one "counter<TAB>outer<TAB>inner<TAB>value" line per entry. The
// reference walks num_cols pointers for CSR and num_rows for CSC (swapped,
// which reads past the pointer array of a non-square matrix); here the
// walk covers num_rows+1 pointers for CSR and num_cols+1 for CSC. For
// square matrices the output is identical.
void printCM(cm mat) {
  int outer;
  if (mat.type == ROW_MAJOR) {
    outer = mat.num_rows;
    printf("CSR %d %d %d\n", mat.num_cols, mat.num_rows, mat.nnz);
  } else {
    outer = mat.num_cols;
    printf("CSC %d %d %d\n", mat.num_cols, mat.num_rows, mat.nnz);
  }
  int cnt = 0;
  for (int i = 0; i < outer; ++i) {
    for (int j = mat.ptr[i]; j < mat.ptr[i + 1]; ++j)
      printf("%d\t%d\t%d\t%f\n", cnt++, i, mat.idx[j], mat.val[j]);
  }
}

}  // extern "C"

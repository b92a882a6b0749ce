/* Drop-in driver for the reference's `bin/outer A.mtx B.mtx` (reference
 * src/main.cu:11-45), built against this library's headers instead of the
 * reference's. The call sequence is the reference's; the optional third
 * argument uses this library's spgemm_get_result() to write C as text
 * ("rows cols nnz" then one "row col value" line per entry).
 *
 *   gcc -I include outer.c -L spgemm_b200 -lspgemm_b200 -Wl,-rpath,<dir> -o outer
 */
#include <stdio.h>

#include "cm.h"
#include "coo.h"
#include "mm.h"
#include "spgemm_b200.h"

int main(int argc, char* argv[]) {
  if (argc < 3) {
    fprintf(stderr, "usage: %s A.mtx B.mtx [C.txt]\n", argv[0]);
    return 2;
  }
  coo t_A, t_B;
  initCOO(&t_A);
  initCOO(&t_B);
  setCOOtype(&t_A, COL_MAJOR);
  setCOOtype(&t_B, ROW_MAJOR);
  readMTX(&t_A, argv[1]);
  readMTX(&t_B, argv[2]);
  sortCOO(t_A);
  sortCOO(t_B);
  cm A = cudaCOO2CM(t_A);
  cm B = cudaCOO2CM(t_B);
  cm C = cudaInitGEMM(A, B);
  cudaCategorizeGEMM(A, B);
  cudaBinGEMM(A, B, C);
  cudaMergeGEMM(C);
  if (argc > 3) {
    cm R;
    if (spgemm_get_result(&R) != 0) return 1;
    FILE* f = fopen(argv[3], "w");
    if (!f) return 1;
    fprintf(f, "%d %d %d\n", R.num_rows, R.num_cols, R.nnz);
    for (int i = 0; i < R.num_rows; ++i)
      for (int j = R.ptr[i]; j < R.ptr[i + 1]; ++j) fprintf(f, "%d %d %.9g\n", i, R.idx[j], R.val[j]);
    fclose(f);
    cmFree(&R);
  }
  freeCOO(&t_A);
  freeCOO(&t_B);
  cmFree(&A);
  cmFree(&B);
  return spgemm_legacy_status();
}

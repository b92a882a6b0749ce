/* Driver for the legacy spGEMM() entry family (reference lib/spGEMM.h:81-91),
 * built against this library's headers. Reads two square Matrix-Market files
 * with the reference reader (values forced to 1.1), builds A as CSC and B as
 * CSR, and multiplies them either with the one-call spGEMM() or, with a
 * fourth argument "passes", with the individual passes in protocol order.
 * Prints the heavy-row count (from cudaPassC), then "nnzC <n>", and writes C
 * as text ("rows cols nnz", then one "row col value" line per entry).
 *
 *   gcc -I include legacy_spgemm.c -L spgemm_b200 -lspgemm_b200 -Wl,-rpath,<dir>
 */
#include <stdio.h>
#include <string.h>

#include "coo.h"
#include "csc.h"
#include "csr.h"
#include "spGEMM.h"
#include "wlt.h"

int main(int argc, char* argv[]) {
  if (argc < 4) {
    fprintf(stderr, "usage: %s A.mtx B.mtx C.txt [passes]\n", argv[0]);
    return 2;
  }
  coo ta, tb;
  initCOO(&ta);
  initCOO(&tb);
  readMTX(&ta, argv[1]);
  readMTX(&tb, argv[2]);
  csc A = transformCOOToCSC(ta);
  csr B = transformCOOToCSR(tb);
  int n = A.n;
  if (argc > 4 && strcmp(argv[4], "passes") == 0) {
    CSC_HOST = A;
    CSR_HOST = B;
    cudaPass_(n, A.e);
    cudaPath_find_thread_count_approx(n);
    cudaPass_F(n);
    cudaPassB(n);
    cudaPassBB(n, 0);
    cudaPassC(n);
  } else {
    wlt W = makeWLT(A, B);
    wlt_cheat WC;
    memset(&WC, 0, sizeof(WC));
    if (spGEMM(A, B, W, WC, 0) < 0) return 1;
    freeWLT(&W);
  }
  printf("nnzC %d\n", nnzC);
  FILE* f = fopen(argv[3], "w");
  if (!f) return 1;
  fprintf(f, "%d %d %d\n", n, n, nnzC);
  for (int i = 0; i < n; ++i)
    for (int j = c_ptr_h[i]; j < c_ptr_h[i + 1]; ++j)
      fprintf(f, "%d %d %.9g\n", i, c_idx_h[j], c_val_h[j]);
  fclose(f);
  freeCSC(&A);
  freeCSR(&B);
  freeCOO(&ta);
  freeCOO(&tb);
  return 0;
}

/* Live GPU SpGEMM entry family (reference lib/mm.h:1-33).
 *
 * Call protocol (reference src/main.cu:18-37): the caller sorts two COO
 * matrices (A by column, B by row), converts them with cudaCOO2CM -- the
 * COL_MAJOR one becomes the left operand A (CSC), the ROW_MAJOR one the
 * right operand B (CSR) -- then calls cudaInitGEMM -> cudaCategorizeGEMM ->
 * cudaBinGEMM -> cudaMergeGEMM. These shims keep that protocol and its
 * printed outputs; the product itself is computed by the sm_100a engine
 * (spgemm_b200/csrc). The merged C stays in library-owned device memory;
 * spgemm_get_result() (spgemm_b200.h) copies it to the host as sorted CSR.
 *
 * The reference guards this header with SPGEMM_H_, the same macro as
 * lib/spGEMM.h, so the two could not be included together; here each
 * header has its own guard.
 */
#ifndef MM_H_
#define MM_H_

#ifdef __cplusplus
extern "C" {
#endif
#include "coo.h"
#include "cm.h"

/* A 64-column dense accumulator chunk (reference lib/mm.h:10-15); the
 * struct is kept for binary compatibility (cudaDCGEMM's dense windows are
 * bitmaps over the row's column span, not arrays of these). */
struct DenseChunk
{
    int idx;
    float val[64];
};
typedef struct DenseChunk dc;

/* COO -> CSC (type COL_MAJOR, becomes operand A) or CSR (ROW_MAJOR,
 * becomes operand B) on the GPU; returns a host copy whose arrays are
 * malloc'd. Input sorted by sortCOO (the reference protocol) takes a direct
 * split and scan; any other order is sorted on the device first (the
 * reference requires the host sort). Replaces reference src/mm.cu:65-136. */
cm cudaCOO2CM(coo mat);
/* Row analysis of A*B: returns C's shape with nnz = the number of
 * intermediate products P (clamped to INT_MAX; the exact 64-bit value is
 * printed). Replaces reference src/mm.cu:150-193. */
cm cudaInitGEMM(cm A, cm B);
/* Workload binning of C's rows. Replaces reference src/mm.cu:263-286. */
void cudaCategorizeGEMM(cm A, cm B);
/* Symbolic pass of every row with the unbinned generic kernels.
 * Replaces reference src/mm.cu:356-364. */
void cudaSimpleGEMM(cm A, cm B, cm C);
/* Symbolic pass per bin (exact nnz of every C row, row pointers).
 * Replaces reference src/mm.cu:314-327. */
void cudaBinGEMM(cm A, cm B, cm C);
/* Symbolic + numeric pass with the dense-chunk strategy: every row whose
 * column span is at most 2^18 accumulates in dense column windows (a
 * presence bitmap plus values in column order) instead of hash tables; wider
 * rows keep the hash paths. Re-bins the rows, so it may follow cudaInitGEMM
 * directly. Prints "nnzC nnzCf" like cudaMergeGEMM. Declared but never
 * defined in the reference (lib/mm.h:23). */
void cudaDCGEMM(cm A, cm B, cm C);
/* Numeric pass: merged, column-sorted C; prints "nnzC nnzCf" like the
 * reference. Replaces reference src/mm.cu:407-450. */
void cudaMergeGEMM(cm C);

#ifdef __cplusplus
}
#endif

#endif /* MM_H_ */

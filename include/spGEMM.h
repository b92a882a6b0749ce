/* Legacy spGEMM() entry family (reference lib/spGEMM.h:1-97).
 *
 * Same declarations, same global names and types as the reference header, so
 * a driver written against it links against this library unchanged. The
 * reference ships bodies for the pass functions only (src/spGEMM.cu:704-1262;
 * spGEMM, cudaPass0 and cudaPass2 are declared without bodies, and the
 * globals are declared extern but defined nowhere); this library defines all
 * of them (spgemm_b200/csrc/legacy_spgemm.cu) on top of the sm_100a engine.
 *
 * Protocol (as in the reference): the caller fills CSC_HOST (operand A, CSC)
 * and CSR_HOST (operand B, CSR), both n x n, then runs
 *   cudaPass_(n, e)                      upload, per-row product counts -> RUPP_HOST
 *   cudaPath_find_thread_count_approx(n) workload binning
 *   cudaPass_F(n)                        heavy ("dominator") rows -> domR / domN
 *   cudaPassB(n)                         symbolic pass + short rows
 *   cudaPassBB(n, t)                     heavy rows (column-sliced), C on the device
 *   cudaPassC(n)                         C to the host: c_ptr_h / c_idx_h / c_val_h, nnzC
 * or the one-call forms cudaPass0 + cudaPass2, or spGEMM(). Pass times go to
 * t_pre, t_bin, t_fd, t_spgemm_l, t_spgemm_d, t_merge (milliseconds).
 *
 * The reference's mm.h and spGEMM.h share the guard SPGEMM_H_, so one file
 * cannot include both; this header uses its own guard and the same
 * declarations, so both families can be used from one translation unit.
 */
#ifndef SPGEMM_LEGACY_H_
#define SPGEMM_LEGACY_H_

#ifdef __cplusplus
extern "C" {
#endif
#include "coo.h"
#include "csc.h"
#include "csr.h"
#include "wlt.h"

/* A (row slice, column slice) pair of a 2-D split (lib/spGEMM.h:12-16). */
struct _PP {
    int r;
    int c;
};
typedef struct _PP PP;

extern int subMatrixSize;
extern int depth;
extern int resCnt;

extern coo COOC;
extern coo COOR;

/* Device copies of the operands (host variables holding device addresses). */
extern int* CSC_RIDX_DEV;
extern int* CSC_PTR_DEV;
extern float* CSC_VAL_DEV;

extern int* CSR_CIDX_DEV;
extern int* CSR_PTR_DEV;
extern float* CSR_VAL_DEV;

extern int* RUPP_DEV;   /* per-row products of C (device) */
extern int* WLS_DEV;    /* per-k workload nnz(A(:,k)) * nnz(B(k,:)) (device) */
extern int* RBOX_DEV;
extern PP* P_DEV;
extern int* N_DEV;

extern int* WLS_HOST;   /* WLS_DEV on the host (n entries) */
extern int* RUPP_HOST;  /* RUPP_HOST[0] = 0, RUPP_HOST[i + 1] = products of row i */
extern PP* P_HOST;

/* C after cudaPassBB (device, CSR) and cudaPassC (host, CSR, malloc'd). */
extern int* c_jdx_d;
extern int* c_idx_d;
extern float* c_val_d;
extern int* c_ptr_d;
extern int* c_idx_h;
extern float* c_val_h;
extern int* c_ptr_h;

extern coo COO_HOST;
extern csc CSC_HOST;
extern csr CSR_HOST;
extern csr DCSR_HOST;
extern csc DCSC_HOST;

extern float t_pre, t_fd, t_spgemm_l, t_spgemm_d, t_merge, t_bin;
extern double t_cpu;
extern int nnzC;
extern int* domR;   /* heavy rows of C */
extern int* domN;   /* domN[0] = number of heavy rows */
extern int* domRC;  /* per heavy row: entries of A's row (outer products feeding it) */
extern int* domCC;  /* per heavy row: its products (clamped to INT_MAX) */
extern int domRCavg;
extern int domCCavg;

void cudaPass_(int n, int e);
void cudaPath_find_thread_count_approx(int n);

void cudaPass_F(int n);
void cudaPassB(int n);
void cudaPassBB(int n, int t);
void cudaPassC(int n);

void cudaPass0(int n, int e);
int cudaPass2(void);
int spGEMM(csc CSC, csr CSR, wlt WLT, wlt_cheat WLT_C, int cheat);

#ifdef __cplusplus
}
#endif

#endif /* SPGEMM_LEGACY_H_ */

/* CompressedMatrix: CSR (type ROW_MAJOR) or CSC (type COL_MAJOR).
 *
 * Drop-in for the reference header lib/cm.h:1-38 with the identical
 * struct layout. For CSR `ptr` has num_rows+1 entries and `idx` holds
 * column indices; for CSC `ptr` has num_cols+1 entries and `idx` holds
 * row indices. Arrays handed out by this library are allocated with
 * malloc(), so cmFree() (which calls free()) releases them correctly.
 */
#ifndef CM_H_
#define CM_H_

#ifdef __cplusplus
extern "C" {
#endif

#include "coo.h"

struct CompressedMatrix
{
    int *ptr;
    int *idx;
    float *val;

    int nnz;
    int num_rows;
    int num_cols;
    bool type;
};
typedef struct CompressedMatrix cm;

void cmInit(cm* mat);                        /* ref src/cm.cpp:7-16  */
void cmFree(cm* mat);                        /* ref src/cm.cpp:18-31 */
int cmGetNumRows(cm mat);                    /* ref src/cm.cpp:34-37 */
int cmGetNumCols(cm mat);                    /* ref src/cm.cpp:38-41 */
int cmGetNNZ(cm mat);                        /* ref src/cm.cpp:42-45 */
void cmSetNumRows(cm* mat, int num_rows);    /* ref src/cm.cpp:47-50 */
void cmSetNumCols(cm* mat, int num_cols);    /* ref src/cm.cpp:51-54 */
void cmSetNNZ(cm* mat, int nnz);             /* ref src/cm.cpp:55-58 */
void cmSetType(cm* mat, bool type);          /* ref src/cm.cpp:59-62 */
/* Present in the reference source (src/cm.cpp:65-89) though not in its
 * header; exported here as well. */
void printCM(cm mat);

#ifdef __cplusplus
}
#endif

#endif /* CM_H_ */

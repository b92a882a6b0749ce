/* Coordinate-format sparse matrix and Matrix-Market reader.
 *
 * Drop-in for the reference header lib/coo.h:1-48. Struct layouts, field
 * order, macro values and function signatures are identical so that code
 * compiled against the reference header links against this library
 * unchanged. Implementations live in spgemm_b200/csrc/host_coo.cpp.
 */
#ifndef COO_H_
#define COO_H_

#ifdef __cplusplus
extern "C" {
#endif
#include <stdbool.h>

#define COO_IDX_FORM 2
#define COO_IDX_VALUE_FORM 3
#define SORT_COO_ROW_BASE 0
#define SORT_COO_COL_BASE 1
#define ROW_MAJOR 0
#define COL_MAJOR 1

/* One stored entry: 0-based row, 0-based column, value (lib/coo.h:16-22). */
struct triplet
{
    int ridx;
    int cidx;
    float val;
};
typedef struct triplet triplet;

/* Entry list plus dimensions. `type` selects the sort order used by
 * sortCOO and the compressed form cudaCOO2CM builds: ROW_MAJOR -> CSR,
 * COL_MAJOR -> CSC (lib/coo.h:24-33). */
struct coo
{
    triplet* data;

    int nnz;
    int num_cols;
    int num_rows;
    bool type;
};
typedef struct coo coo;

void initCOO(coo* mat);                  /* ref src/coo.cpp:6-13   */
void freeCOO(coo* mat);                  /* ref src/coo.cpp:15-22  */
void setCOOtype(coo* mat, bool type);    /* ref src/coo.cpp:38-41  */
coo copyCOO(coo mat);                    /* ref src/coo.cpp:24-36  */
void sortCOO(coo mat);                   /* ref src/coo.cpp:73-79  */

void readCOO(coo* mat, char* path);      /* ref src/coo.cpp:82-108 */
void readMTX(coo* mat, char* path);      /* ref src/coo.cpp:110-173 */

#ifdef __cplusplus
}
#endif

#endif /* COO_H_ */

/* Compressed sparse column matrix, as consumed by the legacy spGEMM()
 * entry family. Layout identical to the reference lib/csc.h:10-19:
 * `header` has n+1 column pointers, `ridx`/`val` hold e entries.
 * The reference declares the helper functions (lib/csc.h:21-24) but ships
 * no implementation; this library implements them
 * (spgemm_b200/csrc/host_legacy.cpp).
 */
#ifndef CSC_H_
#define CSC_H_

#ifdef __cplusplus
extern "C" {
#endif

#include "coo.h"

struct csc
{
    int *header;
    int *ridx;
    float *val;

    int n;
    int e;
};
typedef struct csc csc;

void initCSC(csc* mat);
void freeCSC(csc* mat);
void dumpCSC(csc matrix);
csc transformCOOToCSC(coo mat);

#ifdef __cplusplus
}
#endif

#endif /* CSC_H_ */

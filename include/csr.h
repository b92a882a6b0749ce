/* Compressed sparse row matrix for the legacy spGEMM() entry family.
 *
 * The reference includes "csr.h" (src/spGEMM.cu:3, lib/wlt.h:8,
 * lib/spGEMM.h:8) but the file is absent from its tree. The layout here is
 * reconstructed from its uses -- CSR_HOST.header / .cidx / .val / .n / .e
 * at src/spGEMM.cu:782-784 and DCSR_HOST.* at src/spGEMM.cu:1159-1161 --
 * and mirrors `csc` field for field: `header` has n+1 row pointers,
 * `cidx`/`val` hold e entries.
 */
#ifndef CSR_H_
#define CSR_H_

#ifdef __cplusplus
extern "C" {
#endif

#include "coo.h"

struct csr
{
    int *header;
    int *cidx;
    float *val;

    int n;
    int e;
};
typedef struct csr csr;

void initCSR(csr* mat);
void freeCSR(csr* mat);
void dumpCSR(csr matrix);
csr transformCOOToCSR(coo mat);

#ifdef __cplusplus
}
#endif

#endif /* CSR_H_ */

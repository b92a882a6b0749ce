/* spgemm_b200: handle-based C ABI of the sm_100a SpGEMM engine.
 *
 * Computes C = A * B for sparse FP32 matrices. A is given as CSC (type
 * COL_MAJOR, the layout the reference engine consumes, reference
 * src/mm.cu:87-109) or CSR (type ROW_MAJOR); B is CSR. C is produced as CSR
 * with column indices sorted ascending inside every row. The structure of C
 * is the symbolic union of the partial products: an entry exists wherever at
 * least one product A(i,k)*B(k,j) is formed, even when the products cancel
 * to exactly zero (the reference keeps such entries too: it emits a column
 * on first touch, src/mm.cu:386-391, and counts it in nnzC, src/mm.cu:432).
 *
 * Matrices are passed as the reference's `cm` struct (cm.h) holding DEVICE
 * pointers unless a function says otherwise. Every call is asynchronous on
 * the handle's stream except where it must return a count to the host
 * (spgemm_symbolic, spgemm_multiply), which synchronises that stream.
 *
 * Errors: every function returns an spgemm_status; the last failure's text
 * is kept per handle (spgemm_last_error). Nothing calls exit().
 * The reference has no handle API; its error path prints and exits
 * (src/mm.cu:6-14). The legacy shims in mm.h keep that behaviour.
 */
#ifndef SPGEMM_B200_H_
#define SPGEMM_B200_H_

#include <stddef.h>
#include "cm.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef enum spgemm_status {
    SPGEMM_OK = 0,
    SPGEMM_ERR_INVALID = 1,     /* bad argument: shape, type, null pointer */
    SPGEMM_ERR_CUDA = 2,        /* a CUDA runtime call failed */
    SPGEMM_ERR_ALLOC = 3,       /* device or host allocation failed */
    SPGEMM_ERR_OVERFLOW = 4,    /* nnz(C) does not fit the int32 CSR of cm */
    SPGEMM_ERR_STATE = 5,       /* call out of order (e.g. numeric before symbolic) */
    SPGEMM_ERR_DEVICE = 6,      /* a kernel's own range check tripped */
    SPGEMM_ERR_TOO_LARGE = 7    /* a size exceeds a documented maximum */
} spgemm_status;

typedef enum spgemm_precision {
    /* FP32 products, FP32 accumulation. */
    SPGEMM_PRECISION_PLAIN = 0,
    /* FP32 products with their FMA rounding error (TwoProduct) and
     * TwoSum-compensated FP32 accumulation (Ogita, Rump & Oishi, "Accurate
     * Sum and Dot Product", SIAM J. Sci. Comput. 26(6), 2005, Dot2); rows
     * with more than 4096 partial products accumulate in FP64 instead. */
    SPGEMM_PRECISION_COMPENSATED = 1
} spgemm_precision;

typedef struct spgemm_context* spgemm_handle_t;

/* Per-product statistics of the last symbolic/multiply call. */
typedef struct spgemm_stats {
    long long intermediate_products;   /* P = sum_k nnz(A(:,k)) * nnz(B(k,:)) */
    long long nnz_c;                   /* exact nnz(C) */
    int rows_per_symbolic_bin[16];     /* rows per first-pass bin: 0..4 warp hash
                                          (64..1024 slots), 5..7 block hash
                                          (2048..8192), 8 span bitmap, 9 long,
                                          10..12 sorted (rows of <= 1024, 2048,
                                          4096 products) */
    int rows_per_numeric_bin[16];      /* long rows per numeric bin: 4..7 block
                                          hash, 8 column slices, 9 span bitmap */
    int long_row_slices;               /* column slices of the long-row path */
    long long kernel_launches;         /* engine kernels launched by the handle so far */
    int warp_overflow_rows;            /* warp-bin rows redone by a block kernel */
} spgemm_stats;

/* Bin thresholds and slice shapes of the engine (spgemm_get_tuning returns
 * the defaults of a new handle). Row i of C has P_i partial products, nnz_i
 * outputs and a column bound cap_i = min(P_i, columns of C, column span of its
 * products). Rows with P_i <= long_p are computed in one fused pass: one warp
 * per row with a hash table of at most warp_table_max slots (a row with more
 * distinct columns than 4/5 of its table is redone by a block), or one block
 * per row with a bitmap over the column span (span <= mid_cols) or a larger
 * hash table. Rows with P_i > long_p take two passes: a bitmap count, then
 * column-slice blocks (nnz_i > long_o_num), a span bitmap block
 * (nnz_i > mid_o_min) or a block hash table. */
typedef struct spgemm_tuning {
    int warp_p_max;       /* fused warp path only when P_i <= this */
    int warp_table_max;   /* largest per-warp hash table: power of two, 64..1024 */
    int warp_cap_max;     /* rows with cap_i above this skip the warp path */
    int long_p;           /* two-pass long path when P_i > this (1..4096) */
    int long_o_num;       /* long rows: column slices when nnz_i > this (1..4096) */
    int slice_cap;        /* max outputs per column slice; 0 = shared-memory limit */
    int slice_cols;       /* max columns per column slice (multiple of 2048) */
    int sym_window;       /* columns per symbolic bitmap window (multiple of 2048,
                             <= 2^20) */
    int keep_bitmaps;     /* 1: keep the long rows' symbolic bitmaps (device memory
                             permitting) so the numeric pass skips rebuilding them */
    int mid_o_min;        /* long rows: span bitmap when nnz_i > this (else hash) */
    int mid_cols;         /* bitmap paths need a column span <= this (<= 2^18) */
    int long_rows;        /* long rows in plain FP32 whose symbolic bitmaps were kept
                             and whose column span is at most 2^18: 0 = column
                             slices; 1 = one block per whole row, products reduced
                             into C in L2; 2 (default) = one block per whole row,
                             shared-memory accumulation for rows of up to ~38K
                             outputs (longer rows take column slices); 3 = as 2,
                             with the longer rows reduced into C in L2 */
    int esc_p_min;        /* rows outside the warp bins (column bound above
                             warp_cap_max) with esc_p_min < P_i <= long_p and a
                             column span above esc_span_min are merged by
                             sorting their products (one block per row) instead
                             of the span bitmap / block hash; esc_p_min >=
                             long_p turns this off */
    int esc_span_min;
} spgemm_tuning;

/* Library version string. */
const char* spgemm_version(void);
/* Human-readable text of a status code. */
const char* spgemm_status_string(int status);

/* Create a handle bound to the current CUDA device; its stream is the
 * default stream until spgemm_set_stream. */
int spgemm_create(spgemm_handle_t* handle);
/* Free the handle and every device buffer it owns. */
int spgemm_destroy(spgemm_handle_t handle);
/* Use `stream` (a cudaStream_t) for all later work of the handle. */
int spgemm_set_stream(spgemm_handle_t handle, void* stream);
/* Select SPGEMM_PRECISION_PLAIN or SPGEMM_PRECISION_COMPENSATED. */
int spgemm_set_precision(spgemm_handle_t handle, int precision);
/* Read / replace the handle's tuning (validated; SPGEMM_ERR_INVALID if a
 * field breaks a documented range). */
int spgemm_get_tuning(spgemm_handle_t handle, spgemm_tuning* out);
int spgemm_set_tuning(spgemm_handle_t handle, const spgemm_tuning* in);
/* Text of the handle's last error ("" if none). */
const char* spgemm_last_error(spgemm_handle_t handle);

/* Phase 1: row analysis, binning and the symbolic pass of C = A*B.
 * Writes the exact nnz(C) to *nnz_c. A: CSC (COL_MAJOR) or CSR (ROW_MAJOR);
 * B: CSR. A.num_cols must equal B.num_rows. Device pointers; the arrays must
 * stay valid and unchanged until spgemm_numeric returns. */
int spgemm_symbolic(spgemm_handle_t handle, cm A, cm B, long long* nnz_c);
/* Phase 2: numeric pass into caller-allocated device buffers:
 * c_rowptr[A rows + 1], c_colidx[nnz_c], c_val[nnz_c]. */
int spgemm_numeric(spgemm_handle_t handle, int* c_rowptr, int* c_colidx,
                   float* c_val);
/* Both phases into handle-owned device buffers (valid until the next call
 * on the handle or spgemm_destroy); *C receives device pointers and sizes. */
int spgemm_multiply(spgemm_handle_t handle, cm A, cm B, cm* C);
/* Statistics of the last product. */
int spgemm_get_stats(spgemm_handle_t handle, spgemm_stats* out);

/* Host-buffer convenience: copies A (CSC or CSR) and B (CSR) from host
 * memory, multiplies, and returns C as host CSR with malloc'd arrays
 * (release with cmFree). */
int spgemm_multiply_host(spgemm_handle_t handle, cm A_host, cm B_host,
                         cm* C_host);
/* Host-buffer variant writing into caller-provided host arrays (which may
 * be pinned): c_rowptr[A rows + 1], c_colidx/c_val[capacity]. *nnz_c
 * receives nnz(C); SPGEMM_ERR_TOO_LARGE when it exceeds `capacity` (nothing
 * is written then, and the call can be repeated with larger arrays). */
int spgemm_multiply_host_to(spgemm_handle_t handle, cm A_host, cm B_host,
                            int* c_rowptr, int* c_colidx, float* c_val,
                            long long capacity, long long* nnz_c);
/* The two host-buffer entry points above copy C back in pieces of about
 * `bytes` of C each (row ranges; at most 16 pieces): the numeric pass runs
 * piece by piece and each piece's device-to-host copy, on a second stream of
 * the handle, overlaps the computation of the pieces after it. Default
 * 64 MiB; 0 copies C in one piece after the whole product. Pinned host
 * arrays let the copies run asynchronously; with pageable arrays every copy
 * still waits only for its own piece. */
int spgemm_set_copy_chunk(spgemm_handle_t handle, long long bytes);

/* Batched products. The reference multiplies one pair per process
 * (src/main.cu:31-37 drives src/mm.cu once); these entry points run `count`
 * independent products C_i = A_i * B_i together: the operands are packed
 * into one block-diagonal product on the device, so each bin kernel of the
 * pipeline serves every product in one launch.
 *   A[i]: device CSR (every A_i) or device CSC (every A_i); B[i]: device CSR;
 *   A[i].num_cols == B[i].num_rows; ptr[0] == 0 for every operand.
 * spgemm_batch_plan runs the whole batch once (host-synchronised), keeps its
 * sizes and returns the total nnz over all C_i. It replaces the handle's
 * current product. spgemm_batch_execute recomputes every C_i from the
 * current contents of the same operand arrays (same structure, any values)
 * with no host synchronisation inside: with use_graph != 0 the pipeline is
 * recorded into a CUDA graph on its first call and replayed afterwards (on
 * the handle's stream, or a handle-owned stream when that is the default
 * stream). It synchronises once at the end to check the device status.
 * Any other product run on the handle invalidates the plan
 * (SPGEMM_ERR_STATE; plan again).
 * Output (handle-owned device memory, valid until the next plan or
 * spgemm_destroy): spgemm_batch_result gives product i as a device cm with
 * local row pointers (from 0) and B_i's column indices; each C_i holds at
 * most INT32_MAX entries (else SPGEMM_ERR_OVERFLOW at plan time), the total
 * may exceed it. spgemm_batch_offsets writes count + 1 row offsets (product
 * i owns rows [row_off[i], row_off[i+1]) of the packed product; its row
 * pointers start at packed position row_off[i] + i) and count + 1 entry
 * offsets. spgemm_batch_copy_result copies product i to host arrays
 * (rowptr[m_i + 1], colidx/val[nnz_i]); spgemm_batch_copy_all copies the
 * whole packed output (rowptr[row_off[count] + count], colidx/val[total]). */
int spgemm_batch_plan(spgemm_handle_t handle, int count, const cm* A, const cm* B,
                      long long* nnz_total);
int spgemm_batch_execute(spgemm_handle_t handle, int use_graph);
int spgemm_batch_offsets(spgemm_handle_t handle, long long* row_offsets,
                         long long* nnz_offsets);
int spgemm_batch_result(spgemm_handle_t handle, int i, cm* C);
int spgemm_batch_copy_result(spgemm_handle_t handle, int i, int* c_rowptr,
                             int* c_colidx, float* c_val);
int spgemm_batch_copy_all(spgemm_handle_t handle, int* c_rowptr, int* c_colidx,
                          float* c_val);

/* Per-kernel timing: when enabled, CUDA events are recorded on the handle's
 * stream around every engine kernel launch and accumulated per kernel name
 * (folded when the times are read or reset, which must follow a
 * synchronisation of the handle's stream, e.g. the end of a numeric pass). */
int spgemm_set_profiling(spgemm_handle_t handle, int enable);
int spgemm_reset_kernel_times(spgemm_handle_t handle);
/* Writes up to max_kernels entries: names ('\n'-separated into `names`),
 * accumulated milliseconds and launch counts. Returns the entry count (or a
 * negated status). */
int spgemm_get_kernel_times(spgemm_handle_t handle, char* names, int names_len,
                            double* ms, long long* launches, int max_kernels);

/* COO -> compressed on the device, triplets in any order: the conversion of
 * cudaCOO2CM (reference src/mm.cu:65-136) without the host sortCOO the
 * reference's protocol needs first (src/coo.cpp:73-79). d_triplets: nnz
 * device triplets; type ROW_MAJOR -> CSR (d_ptr[num_rows + 1]), COL_MAJOR ->
 * CSC (d_ptr[num_cols + 1]); d_idx / d_val [nnz]. Minor indices come out
 * ascending within each row (column), entries with equal indices in input
 * order. Counting sort on the major index, then per-row sorts in shared
 * memory (warp, block, or block-merged runs for rows above 8192 entries).
 * Uses handle-owned scratch (about 16 bytes per entry) and synchronises the
 * handle's stream once. An index outside its dimension: SPGEMM_ERR_INVALID
 * (the output then omits those entries). cudaCOO2CM takes this path by
 * itself when its input is not sorted. */
int spgemm_coo_to_cm(spgemm_handle_t handle, const triplet* d_triplets, int nnz,
                     int num_rows, int num_cols, int type, int* d_ptr, int* d_idx,
                     float* d_val);

/* Value-preserving Matrix-Market reader. The reference's readMTX
 * (src/coo.cpp:110-173, kept unchanged in coo.h) forces every value to 1.1,
 * reads the first size token as the column count and misparses pattern
 * files; this reader follows the format: "coordinate" files with field real,
 * double, integer or pattern (pattern entries get 1.0) and symmetry general,
 * symmetric (mirrored off-diagonal entries), skew-symmetric (mirrored and
 * negated) or hermitian (as symmetric; real fields only). Indices become
 * 0-based; num_rows / num_cols come from the size line in the format's order
 * (rows first); entries keep file order, mirrored ones right after their
 * source entry; `type` is left as the caller set it (call sortCOO for the
 * order cudaCOO2CM wants). out->data is malloc'd (freeCOO releases it).
 * Returns SPGEMM_OK, SPGEMM_ERR_INVALID for an unreadable, malformed,
 * truncated or out-of-range file (nothing is kept), SPGEMM_ERR_TOO_LARGE
 * beyond INT32_MAX entries. No counterpart in the reference. */
int spgemm_read_mtx(coo* out, const char* path);

/* Allocation-free COO -> compressed conversion. This entry point has no
 * counterpart in the reference; it performs the conversion of cudaCOO2CM
 * (sorted triplets -> CSR for ROW_MAJOR, CSC for COL_MAJOR) on device arrays
 * the caller owns, for callers that cannot allocate device memory at that
 * point: code whose device memory belongs to another allocator (a
 * framework's caching allocator, a fixed arena sized up front), and
 * latency-critical loops in which a cudaMalloc would synchronise the device.
 *   d_triplets: nnz triplets on the device, sorted by (major, minor) index
 *               with every index inside the dimensions;
 *   d_ptr: (major dimension + 1) ints; d_idx, d_val: nnz entries each.
 * Nothing is allocated: the counts are accumulated in d_ptr itself and the
 * scan's scratch is a fixed static device array of about 131 KB, present on
 * every GPU that loads this library until the process exits. It limits the
 * major dimension to SPGEMM_NOALLOC_MAX_MAJOR (larger: SPGEMM_ERR_TOO_LARGE,
 * nothing launched). The first call on a device, with that device current,
 * looks up that array's device address and loads this entry point's kernels;
 * make that first call before any stream capture. The address is kept per
 * device ordinal for the process: only the runtime's primary context is
 * supported, and the library must not be used on a device after
 * cudaDeviceReset. All calls share the array, which keeps the previous
 * call's contents (each call clears what must start at zero): calls that can
 * overlap on the GPU (on different streams without ordering) race and must
 * not be issued.
 * Asynchronous on `stream` unless nnz_check is non-null, in which case the
 * stream is synchronised, *nnz_check receives the number of entries counted,
 * and an out-of-range index or unsorted input returns SPGEMM_ERR_INVALID.
 * With nnz_check == NULL nothing is checked on the host: input that is
 * unsorted or holds an out-of-range index gives undefined output (entries
 * with an out-of-range index are skipped and leave their d_idx / d_val slots
 * unwritten) while the call returns SPGEMM_OK. */
#define SPGEMM_NOALLOC_MAX_MAJOR (1 << 26)
int spgemm_coo_to_cm_noalloc(const triplet* d_triplets, int nnz, int num_rows,
                             int num_cols, int type, int* d_ptr, int* d_idx,
                             float* d_val, void* stream, long long* nnz_check);

/* Companion of the mm.h shims: copy the C that cudaMergeGEMM produced into
 * malloc'd host arrays (sorted CSR, nnz = exact nnz(C)). Returns 0 on
 * success. The reference never returns C (src/mm.cu:420-449). */
int spgemm_get_result(cm* C_host_out);
/* mm.h shims print like the reference (P at cudaInitGEMM, "nnzC nnzCf" at
 * cudaMergeGEMM) when verbose is 1 (default); 0 silences them. */
void spgemm_set_verbose(int verbose);
/* mm.h shims call exit(-1) on a CUDA error like the reference when 1
 * (default); 0 makes them print and return instead. */
void spgemm_set_exit_on_error(int enable);
/* Status of the last mm.h shim call (SPGEMM_OK if it succeeded). */
int spgemm_legacy_status(void);

#ifdef __cplusplus
}
#endif

#endif /* SPGEMM_B200_H_ */

// sm_100a kernels of the SpGEMM pipeline C = A * B.
//
// The reference expands the outer product A(:,k) * B(k,:) of every k into
// per-row buckets of C (src/mm.cu:288-312, "binGEMM") and merges each bucket
// with a dense accumulator (src/mm.cu:366-404, "mergeGEMM"). Materialising the
// buckets costs 8 bytes of HBM write + read per partial product. Here the
// same partials are generated bucket by bucket instead: the row i bucket is
// sum_k A(i,k) * B(k,:), so each C row is expanded and merged in on-chip
// memory by one warp, one block, or (for long rows) several blocks that
// each own a column slice. Partials never touch HBM.
//
// Pipeline (kernel names):
//   k_validate        index ranges and sortedness of the inputs
//   k_transpose_hist / k_transpose_scatter  A CSC -> CSR (row-wise expansion)
//   k_row_analysis    P_i per row, flattened offsets, column spans, bins
//   k_fused_warp/block  rows of at most long_p products in one pass: hash
//                     accumulate, sort, row written to a temporary buffer
//   k_num_long<.,512,sparse> as k_fused_mid  the same for rows whose column
//                     span fits a bitmap (two passes over the row on chip)
//   k_sym_long        exact nnz of long rows via a shared-memory bitmap
//   k_scan_*          row pointers of C
//   k_num_bin         numeric binning + column slicing of long rows
//   k_copy_fused      fused rows from the temporary buffer into C
//   k_num_long        long rows: bitmap-rank merge (a counting sort on the
//                     column) -> sorted CSR slices
//   k_num_block       long rows with few outputs: block hash + sort
#pragma once

#include <type_traits>
#include <utility>

#include "common.cuh"

namespace sg {

// Functors of column-only passes may take the four columns one lane loads
// with a 128-bit load in one call (vec4), to merge updates of the same word.
template <class F, class = void>
struct HasVec4 : std::false_type {};
template <class F>
struct HasVec4<F, std::void_t<decltype(std::declval<F&>().vec4(int4{}))>> : std::true_type {};

// ---------------------------------------------------------------------------
// Operands and tuning
// ---------------------------------------------------------------------------

struct Operands {
  const int* __restrict__ a_rowptr;  // A in CSR (m + 1)
  const int* __restrict__ a_col;     // k index of each A entry
  const float* __restrict__ a_val;
  const int* __restrict__ aoff;      // flattened offset of each A entry in its row
  const int* __restrict__ b_rowptr;  // B in CSR (kdim + 1)
  const int* __restrict__ b_col;
  const float* __restrict__ b_val;
  int m, kdim, n;
  int vec_ok;  // b_col and b_val are 16-byte aligned: 128-bit loads allowed
  int nnz_b;
};

// First-pass bins (k_row_analysis). Rows of at most long_p products are
// computed in one fused pass (sorted output into a temporary buffer):
//   0..4  one warp per row, hash table of 2^6..2^10 slots (optimistic: a row
//         with more distinct columns than 4/5 of the table is redone below)
//   5..7  one block per row, hash table of 2^11..2^13 slots
//   8     one block per row, bitmap over the row's column span ("mid")
// Rows with more products take the two-phase long path:
//   9     symbolic bitmap count (k_sym_long), numeric later
// and, for rows the warp bins do not take, ahead of the mid and block bins
// when the tuning enables it (the default):
//   10..12 one block of 128 / 256 / 512 threads per row of at most 1024 /
//         2048 / 4096 products, sorted instead of hashed (k_fused_esc)
constexpr int FB_WARP_BINS = 5;
constexpr int FB_BLOCK0 = 5;
constexpr int FB_MID = 8;
constexpr int FB_LONG = 9;
constexpr int FB_ESC0 = 10;
constexpr int FB_ESC_BINS = 3;
constexpr int FB_COUNT = 13;
// Numeric bins of long rows: 4..7 block hash (2^10..2^13 slots), 8 column
// slices, 9 bitmap of the whole span (statistics slots 0..3 stay unused).
constexpr int NB_COUNT = 10;
constexpr int NB_LONG = 8;
constexpr int NB_MID = 9;

constexpr int CHUNK_COLS = 2048;               // column granularity of slicing
constexpr int CHUNK_WORDS = CHUNK_COLS / 32;
constexpr long long FP64_ROW_PARTIALS = 4096;  // compensated mode: FP64 above this

struct Tuning {
  int warp_p_max;       // fused warp path only when P_i <= this
  int warp_table_max;   // largest per-warp table (64..1024 slots)
  int warp_cap_max;     // rows whose column bound exceeds this skip the warp path
  int long_p;           // two-phase long path when P_i > this (<= 4096)
  int long_o_num;       // long rows: column-slice numeric when nnz_i > this (<= 4096)
  int slice_cap;        // max outputs of one numeric long slice (0: smem budget)
  int slice_cols;       // max columns of one numeric long slice (multiple of 2048)
  int sym_window;       // columns per symbolic bitmap window (multiple of 2048)
  int keep_bitmaps;     // keep long rows' symbolic bitmaps for the numeric pass
  int mid_o_min;        // long rows: bitmap numeric when nnz_i > this ...
  int mid_cols;         // bitmap paths need a column span of at most this (<= 2^18)
  int long_rows;        // long rows, plain FP32, bitmaps kept: 0 column slices;
                        // 1 whole rows, reductions into C (L2); 2 whole rows,
                        // shared-memory accumulation (rows up to its capacity;
                        // longer rows take slices); 3 as 2, reductions into C
                        // for the longer rows
  int esc_p_min;        // rows outside the warp bins with esc_p_min < P_i <= long_p
  int esc_span_min;     // and a span above esc_span_min are sorted (k_fused_esc)
};

// Whole-row numeric path (k_num_rows): the row's column span must fit the
// block's directory, and (shared-memory form) its outputs the value array.
constexpr int ROWS_MAX_WORDS = (1 << 18) / 32 + 1;  // 2^18 columns, + lo rounded down

__host__ __device__ inline bool whole_row_path(int o, int2 sp, int cnt_max, int max_words) {
  if (o <= 0 || o > cnt_max) return false;
  const int lo = sp.x & ~31;
  return ((sp.y + 1 - lo + 31) >> 5) <= max_words;
}

__host__ __device__ inline int ceil_log2_ll(long long v) {
  int r = 0;
  while ((1ll << r) < v) ++r;
  return r;
}

// Column bound of row i: nnz_i <= min(P_i, n, span_i).
__host__ __device__ inline long long row_cap(long long p, int n, int span) {
  long long c = p < n ? p : n;
  return c < span ? c : span;
}

__host__ __device__ inline int first_bin_of(long long p, long long cap, int span, const Tuning& t) {
  if (p <= 0) return -1;
  if (p > t.long_p) return FB_LONG;
  if (cap <= t.warp_cap_max && p <= t.warp_p_max) {
    int lg = ceil_log2_ll(cap + cap / 4 + 1);  // table >= 1.25 x column bound
    if (lg < 6) lg = 6;
    const int lmax = ceil_log2_ll(t.warp_table_max);
    if (lg > lmax) lg = lmax;
    return lg - 6;
  }
  if (p > t.esc_p_min && span > t.esc_span_min)  // p <= long_p <= 4096
    return p <= 1024 ? FB_ESC0 : (p <= 2048 ? FB_ESC0 + 1 : FB_ESC0 + 2);
  if (span <= t.mid_cols) return FB_MID;
  int lg = ceil_log2_ll(2 * cap);
  if (lg < 11) lg = 11;
  return lg - 11 + FB_BLOCK0;  // cap <= p <= long_p <= 4096, so lg <= 13
}

// Numeric bin of a long row (P_i > long_p) with nnz_i outputs.
__host__ __device__ inline int num_bin_of(int o, long long p, const Tuning& t) {
  (void)p;
  if (o <= 0) return -1;
  if (o > t.long_o_num) return NB_LONG;
  int lg = ceil_log2_ll(2ll * o);
  if (lg < 10) lg = 10;
  return lg - 10 + 4;  // lg <= 13 because o <= long_o_num <= 4096
}

// One column slice of a row for the numeric bitmap kernel.
constexpr int SLICE_WHOLE = 1;      // the slice holds all of the row's outputs
constexpr int SLICE_BITS_KEPT = 2;  // the symbolic pass kept the row's bitmap
constexpr int SLICE_FUSED = 4;      // fused pass: output to the temporary buffer,
                                    // nnz found here and written to c_cnt
struct Slice {
  long long out;  // first output position in C
  int row;
  int lo, hi;     // columns [lo, hi)
  int cnt;        // outputs in the slice
  int flags;
};

// ---------------------------------------------------------------------------
// Expansion primitives
// ---------------------------------------------------------------------------

// Per-warp staging area used to compact non-empty segments to the front.
struct SegScratch {
  int bstart[32];
  int len[32];
  float a[32];
  int count;  // fused warp rows: distinct columns inserted so far
};

// Move the lanes with len > 0 to lanes 0..cnt-1 (order preserved).
__device__ __forceinline__ int compact_segments(int& bstart, int& len, float& a,
                                                SegScratch* sc) {
  const int lane = lane_id();
  const unsigned m = __ballot_sync(FULL, len > 0);
  const int cnt = __popc(m);
  if (m == (cnt == 32 ? FULL : ((1u << cnt) - 1u))) return cnt;  // already a prefix
  const int r = __popc(m & ((1u << lane) - 1u));
  if (len > 0) { sc->bstart[r] = bstart; sc->len[r] = len; sc->a[r] = a; }
  __syncwarp();
  if (lane < cnt) { bstart = sc->bstart[lane]; len = sc->len[lane]; a = sc->a[lane]; }
  else { len = 0; }
  __syncwarp();
  return cnt;
}

// Loop unrolling of the product walks: windows / 128-bit groups whose loads
// are issued before their accumulates, for passes that load values (VAL) or
// only columns (BITS).
constexpr int WIN_UNROLL_VAL = 2, WIN_UNROLL_BITS = 4;
constexpr int VEC_UNROLL_VAL = 2, VEC_UNROLL_BITS = 4;
constexpr int VEC_INTERLEAVE_VAL = 8;  // lane-interleaved value walk: loads in flight per lane

// Generate every partial product of the (<= 32) compacted segments held by
// the warp: lane j < cnt holds B positions [bstart, bstart + len) to be
// scaled by a. The segments are laid end to end and walked 32 products at a
// time, so lanes stay busy whatever the segment lengths. The owner of each
// product is found from the OR of segment-start bits in the current window
// (redux.sync) and a popcount -- O(1) per product, no search.
//
// Each segment is walked from a pseudo-random starting offset (wrapping
// around). B's rows are sorted, so without the rotation every warp would
// begin its segments on the same lowest (for power-law graphs: the most
// popular) columns at the same time, and the shared-memory atomics of all
// warps would collide there.
template <bool NEED_VAL, class F>
__device__ __forceinline__ void run_segments(int cnt, int bstart, int len, float a,
                                             const int* __restrict__ b_col,
                                             const float* __restrict__ b_val, F& f) {
  constexpr int UNROLL = NEED_VAL ? WIN_UNROLL_VAL : WIN_UNROLL_BITS;  // windows in flight
  const int lane = lane_id();
  if (lane >= cnt) len = 0;
  const int incl = warp_incl_scan(len);
  const int total = __shfl_sync(FULL, incl, 31);
  const int s = incl - len;
  const int rot = len > 1 ? (int)(((unsigned)bstart * 2654435761u >> 8) % (unsigned)len) : 0;
  int nbefore = 0;
  for (int base = 0; base < total; base += 32 * UNROLL) {
    int col[UNROLL];
    float bv[UNROLL], oa[UNROLL];
    bool ok[UNROLL];
#pragma unroll
    for (int u = 0; u < UNROLL; ++u) {
      const int wb = base + 32 * u;
      ok[u] = false;
      if (wb < total) {  // warp-uniform
        const unsigned bit =
            (len > 0 && s >= wb && s < wb + 32) ? (1u << (s - wb)) : 0u;
        const unsigned starts = __reduce_or_sync(FULL, bit);
        const int owner = nbefore + __popc(starts & (FULL >> (31 - lane))) - 1;
        nbefore += __popc(starts);
        const int ob = __shfl_sync(FULL, bstart, owner);
        const int os = __shfl_sync(FULL, s, owner);
        const int ol = __shfl_sync(FULL, len, owner);
        const int orot = __shfl_sync(FULL, rot, owner);
        oa[u] = __shfl_sync(FULL, a, owner);
        const int fp = wb + lane;
        if (fp < total) {
          int off = fp - os + orot;
          if (off >= ol) off -= ol;
          const int pos = ob + off;
          col[u] = __ldg(b_col + pos);
          bv[u] = NEED_VAL ? __ldg(b_val + pos) : 0.f;
          ok[u] = true;
        }
      }
    }
#pragma unroll
    for (int u = 0; u < UNROLL; ++u)
      if (ok[u]) f(col[u], oa[u], bv[u]);
  }
}

// Segments at least this long are walked by the whole warp with 128-bit
// loads (4 products per lane per step) instead of the flattened walk.
constexpr int VEC_MIN_SEG = 128;

// One segment B positions [bs, bs + len) scaled by a, whole warp: scalar head
// up to the first 16-byte boundary, int4/float4 body, scalar tail.
template <bool NEED_VAL, class F>
__device__ __forceinline__ void warp_run_segment_vec(int bs, int len, float a,
                                                     const int* __restrict__ b_col,
                                                     const float* __restrict__ b_val, F& f) {
  const int lane = lane_id();
  const int end = bs + len;
  if constexpr (NEED_VAL) {
    // Value passes load lane-interleaved: one warp step covers 32 * VI
    // consecutive positions, lane l taking positions l, l + 32, ... Columns
    // then rise with the lane, so accumulators indexed by column rank are hit
    // on consecutive shared-memory banks (a lane holding four consecutive
    // entries, as the 128-bit form below does, makes every access 4-way
    // bank-conflicted on a dense slot range). Pointers are advanced once per
    // step, so each load is one instruction with an immediate offset.
    constexpr int VI = VEC_INTERLEAVE_VAL;
    const int* __restrict__ pc = b_col + bs + lane;
    const float* __restrict__ pv = b_val + bs + lane;
    for (int q = lane; q < len; q += 32 * VI, pc += 32 * VI, pv += 32 * VI) {
      int c[VI];
      float v[VI];
#pragma unroll
      for (int u = 0; u < VI; ++u) {
        c[u] = q + 32 * u < len ? __ldg(pc + 32 * u) : 0;
        v[u] = q + 32 * u < len ? __ldg(pv + 32 * u) : 0.f;
      }
#pragma unroll
      for (int u = 0; u < VI; ++u)
        if (q + 32 * u < len) f(c[u], a, v[u]);
    }
    return;
  }
  const int head = min((4 - (bs & 3)) & 3, len);
  if (lane < head) {
    const int pos = bs + lane;
    f(__ldg(b_col + pos), a, NEED_VAL ? __ldg(b_val + pos) : 0.f);
  }
  const int body0 = bs + head;
  const int n4 = (end - body0) >> 2;
  const int4* c4 = reinterpret_cast<const int4*>(b_col + body0);
  const float4* v4 = reinterpret_cast<const float4*>(b_val + body0);
  constexpr int VU = NEED_VAL ? VEC_UNROLL_VAL : VEC_UNROLL_BITS;  // groups in flight together
  int g = lane;
  for (; g + 32 * (VU - 1) < n4; g += 32 * VU) {
    int4 c[VU];
    float4 v[VU];
#pragma unroll
    for (int u = 0; u < VU; ++u) {
      c[u] = __ldg(c4 + g + 32 * u);
      v[u] = NEED_VAL ? __ldg(v4 + g + 32 * u) : make_float4(0.f, 0.f, 0.f, 0.f);
    }
#pragma unroll
    for (int u = 0; u < VU; ++u) {
      if constexpr (HasVec4<F>::value) {
        f.vec4(c[u]);
      } else {
        f(c[u].x, a, v[u].x);
        f(c[u].y, a, v[u].y);
        f(c[u].z, a, v[u].z);
        f(c[u].w, a, v[u].w);
      }
    }
  }
  for (; g < n4; g += 32) {
    const int4 c = __ldg(c4 + g);
    const float4 v = NEED_VAL ? __ldg(v4 + g) : make_float4(0.f, 0.f, 0.f, 0.f);
    if constexpr (HasVec4<F>::value) {
      f.vec4(c);
    } else {
      f(c.x, a, v.x);
      f(c.y, a, v.y);
      f(c.z, a, v.z);
      f(c.w, a, v.w);
    }
  }
  const int tail0 = body0 + 4 * n4;
  if (tail0 + lane < end) {
    const int pos = tail0 + lane;
    f(__ldg(b_col + pos), a, NEED_VAL ? __ldg(b_val + pos) : 0.f);
  }
}

// All products of the warp's (<= 32) segments: long ones one at a time with
// the vector walk, the rest compacted and walked flattened.
template <bool NEED_VAL, class F>
__device__ __forceinline__ void warp_run_batch(const Operands& op, int bstart, int len, float a,
                                               F& f, SegScratch* sc) {
  if (op.vec_ok) {
    unsigned big = __ballot_sync(FULL, len >= VEC_MIN_SEG);
    while (big) {
      const int src = __ffs(big) - 1;
      big &= big - 1u;
      const int sbs = __shfl_sync(FULL, bstart, src);
      const int sl = __shfl_sync(FULL, len, src);
      const float sa = __shfl_sync(FULL, a, src);
      warp_run_segment_vec<NEED_VAL>(sbs, sl, sa, op.b_col, op.b_val, f);
    }
    if (len >= VEC_MIN_SEG) len = 0;
  }
  const int cnt = compact_segments(bstart, len, a, sc);
  if (cnt) run_segments<NEED_VAL>(cnt, bstart, len, a, op.b_col, op.b_val, f);
}

// Products per warp work unit when the warps of a block share one row of
// `p` products. Units are equal slices of the row's flattened product
// sequence, so one unit per warp is already balanced; each unit costs one
// binary search to find its first entry.
__device__ __forceinline__ int chunk_for(long long p, int nwarps, int max_chunk) {
  long long u = (p + nwarps - 1) / nwarps;
  u = (u + 31) & ~31ll;
  if (u < 32) u = 32;
  if (u > max_chunk) u = max_chunk;
  return (int)u;
}

// Whole row of A, one warp. With stop_limit >= 0 the walk ends early once
// sc->count exceeds it (checked between 32-entry batches, warp-uniformly).
template <bool NEED_VAL, class F>
__device__ __forceinline__ void warp_expand_row(const Operands& op, int rs, int re,
                                                F& f, SegScratch* sc, int stop_limit = -1) {
  const int lane = lane_id();
  for (int base = rs; base < re; base += 32) {
    if (stop_limit >= 0) {
      __syncwarp();
      if (*((volatile int*)&sc->count) > stop_limit) break;
    }
    const int j = base + lane;
    int bstart = 0, len = 0;
    float a = 0.f;
    if (j < re) {
      const int k = __ldg(op.a_col + j);
      a = __ldg(op.a_val + j);
      bstart = __ldg(op.b_rowptr + k);
      len = __ldg(op.b_rowptr + k + 1) - bstart;
    }
    warp_run_batch<NEED_VAL>(op, bstart, len, a, f, sc);
  }
}

// Products [f0, f1) of the row's flattened product sequence (entries in
// order, each contributing nnz(B(k,:)) products), one warp. Uses the
// per-entry flattened offsets `aoff` written by k_row_analysis.
template <bool NEED_VAL, class F>
__device__ __forceinline__ void warp_expand_range(const Operands& op, int rs, int re,
                                                  int f0, int f1, F& f,
                                                  SegScratch* sc) {
  const int lane = lane_id();
  // Last entry whose offset is <= f0 holds product f0.
  int lo = rs, hi = re;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(op.aoff + mid) <= f0) lo = mid + 1; else hi = mid;
  }
  for (int base = lo - 1; base < re; base += 32) {
    const int j = base + lane;
    int bstart = 0, len = 0;
    float a = 0.f;
    bool past = true;
    if (j < re) {
      const int off = __ldg(op.aoff + j);
      past = off >= f1;
      if (!past) {
        const int k = __ldg(op.a_col + j);
        const int bs = __ldg(op.b_rowptr + k);
        const int bl = __ldg(op.b_rowptr + k + 1) - bs;
        const int l0 = max(off, f0), l1 = min(off + bl, f1);
        if (l1 > l0) {
          a = __ldg(op.a_val + j);
          bstart = bs + (l0 - off);
          len = l1 - l0;
        }
      }
    }
    const bool done = __any_sync(FULL, past);
    warp_run_batch<NEED_VAL>(op, bstart, len, a, f, sc);
    if (done) break;
  }
}

// Block-wide preparation of a column-restricted pass over one row: for each
// entry j of the row (d = re - rs entries), the positions of B(k_j,:) whose
// columns fall in [clo, chi) (binary search; B's rows are sorted) go to
// seg_start[j] / roff (exclusive prefix of their lengths, roff[d] = total).
// The arrays are this block's global scratch. Returns the total (block-uniform).
__device__ __forceinline__ int block_restrict_row(const Operands& op, int rs, int re, int clo,
                                                  int chi, int* seg_start, int* roff,
                                                  long long* scan_shm, int* carry_shm) {
  const int d = re - rs;
  if (threadIdx.x == 0) *carry_shm = 0;
  __syncthreads();
  for (int t0 = 0; t0 < d; t0 += blockDim.x) {
    const int t = t0 + threadIdx.x;
    int s0 = 0, len = 0;
    if (t < d) {
      const int k = __ldg(op.a_col + rs + t);
      const int bs = __ldg(op.b_rowptr + k), be = __ldg(op.b_rowptr + k + 1);
      if (be > bs) {
        const int first = __ldg(op.b_col + bs), last = __ldg(op.b_col + be - 1);
        if (first < chi && last >= clo) {
          s0 = first >= clo ? bs : lower_bound_i32(op.b_col, bs, be, clo);
          const int s1 = last < chi ? be : lower_bound_i32(op.b_col, s0, be, chi);
          len = s1 - s0;
        }
      }
    }
    // block exclusive scan of len (64-bit scan helper from the caller's shm)
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int incl = warp_incl_scan(len);
    if (lane == 31) scan_shm[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      const long long wv = lane < (int)(blockDim.x >> 5) ? scan_shm[lane] : 0;
      const long long wi = warp_incl_scan64(wv);
      scan_shm[lane] = wi - wv;
      if (lane == 31) scan_shm[32] = wi;
    }
    __syncthreads();
    const int carry = *carry_shm;
    if (t < d) {
      seg_start[t] = s0;
      roff[t] = carry + (int)scan_shm[warp] + incl - len;
    }
    __syncthreads();
    if (threadIdx.x == 0) *carry_shm = carry + (int)scan_shm[32];
    __syncthreads();
  }
  const int total = *carry_shm;
  if (threadIdx.x == 0) roff[d] = total;
  __syncthreads();
  return total;
}

// Products [f0, f1) of a row prepared by block_restrict_row, one warp.
// seg_start / roff are written by this block in this kernel, so they are read
// with plain (coherent) loads.
template <bool NEED_VAL, class F>
__device__ __forceinline__ void warp_expand_explicit(const Operands& op, int rs, int d,
                                                     const int* seg_start, const int* roff,
                                                     int f0, int f1, F& f, SegScratch* sc) {
  const int lane = lane_id();
  int lo = 0, hi = d;  // last entry whose offset is <= f0
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (roff[mid] <= f0) lo = mid + 1; else hi = mid;
  }
  for (int base = lo - 1; base < d; base += 32) {
    const int j = base + lane;
    int bstart = 0, len = 0;
    float a = 0.f;
    bool past = true;
    if (j < d) {
      const int off = roff[j];
      past = off >= f1;
      if (!past) {
        const int bl = roff[j + 1] - off;
        const int l0 = max(off, f0), l1 = min(off + bl, f1);
        if (l1 > l0) {
          a = __ldg(op.a_val + rs + j);
          bstart = seg_start[j] + (l0 - off);
          len = l1 - l0;
        }
      }
    }
    const bool done = __any_sync(FULL, past);
    warp_run_batch<NEED_VAL>(op, bstart, len, a, f, sc);
    if (done) break;
  }
}

// Entries [jb, min(jb + 32, re)) of a row, each restricted to the columns
// [clo, chi) of its B row (binary search), one warp.
template <bool NEED_VAL, class F>
__device__ __forceinline__ void warp_expand_restricted(const Operands& op, int jb, int re,
                                                       int clo, int chi, F& f,
                                                       SegScratch* sc) {
  const int lane = lane_id();
  const int j = jb + lane;
  int bstart = 0, len = 0;
  float a = 0.f;
  if (j < re) {
    const int k = __ldg(op.a_col + j);
    const int bs = __ldg(op.b_rowptr + k);
    const int be = __ldg(op.b_rowptr + k + 1);
    if (be > bs) {
      const int first = __ldg(op.b_col + bs), last = __ldg(op.b_col + be - 1);
      if (first < chi && last >= clo) {
        const int s0 = first >= clo ? bs : lower_bound_i32(op.b_col, bs, be, clo);
        const int s1 = last < chi ? be : lower_bound_i32(op.b_col, s0, be, chi);
        bstart = s0;
        len = s1 - s0;
        a = __ldg(op.a_val + j);
      }
    }
  }
  warp_run_batch<NEED_VAL>(op, bstart, len, a, f, sc);
}

// All products of one row (whole: every entry's whole B row; otherwise the
// slice prepared by block_restrict_row) by the nwarps warps of a block, in
// equal per-warp ranges of the row's flattened product sequence.
template <bool VALUES, class F>
__device__ __forceinline__ void block_walk_row(const Operands& op, int rs, int re, bool whole,
                                               const int* seg_start, const int* roff, int p,
                                               F& f, SegScratch* sc, int warp, int nwarps) {
  const int U = chunk_for(p, nwarps, 1 << 20);
  for (int c0 = warp * U; c0 < p; c0 += nwarps * U) {
    const int c1 = min(c0 + U, p);
    if (whole) warp_expand_range<VALUES>(op, rs, re, c0, c1, f, sc);
    else warp_expand_explicit<VALUES>(op, rs, re - rs, seg_start, roff, c0, c1, f, sc);
  }
}

// ---------------------------------------------------------------------------
// Accumulators
// ---------------------------------------------------------------------------

// Linear-probing insert of `col` into a 2^log2t table; returns the slot or -1
// (table full: recorded in the status word).
__device__ __forceinline__ int hash_slot(unsigned* keys, int log2t, unsigned col,
                                         bool& inserted, unsigned* status) {
  const unsigned mask = (1u << log2t) - 1u;
  unsigned h = hash_col(col, log2t);
  inserted = false;
  for (unsigned probe = 0; probe <= mask; ++probe) {
    const unsigned k = ((volatile unsigned*)keys)[h];
    if (k == col) return (int)h;
    if (k == EMPTY_KEY) {
      const unsigned old = atomicCAS(keys + h, EMPTY_KEY, col);
      if (old == EMPTY_KEY) { inserted = true; return (int)h; }
      if (old == col) return (int)h;
    }
    h = (h + 1u) & mask;
  }
  atomicOr(status, ST_TABLE_FULL);
  return -1;
}

struct SymHash {
  unsigned* keys;
  int log2t;
  unsigned* status;
  int nnew;
  __device__ __forceinline__ void operator()(int col, float, float) {
    bool ins;
    hash_slot(keys, log2t, (unsigned)col, ins, status);
    nnew += ins;
  }
};

// Columns outside [lo, lo + width) cannot occur for validated inputs; the
// range test keeps a malformed input from writing outside the bitmap.
// Four columns of one lane, consecutive entries of a sorted B row (their
// offsets x[] from the bitmap's first column): bits that fall in the same
// 32-column word are OR-ed together first and or_word(word, mask) is called
// once per distinct word, so a dense row costs one shared-memory atomic per
// word instead of one per column. Returns false (nothing done) when an
// offset lies outside [0, width): the caller then takes the columns one by
// one with their range checks.
template <class OrWord>
__device__ __forceinline__ bool or_bits4(int4 c4, int lo, unsigned width, OrWord or_word) {
  const unsigned x[4] = {(unsigned)(c4.x - lo), (unsigned)(c4.y - lo), (unsigned)(c4.z - lo),
                         (unsigned)(c4.w - lo)};
  if (!(x[0] < width && x[1] < width && x[2] < width && x[3] < width)) return false;
  unsigned w = x[0] >> 5, m = 1u << (x[0] & 31);
#pragma unroll
  for (int q = 1; q < 4; ++q) {
    if ((x[q] >> 5) == w) {
      m |= 1u << (x[q] & 31);
    } else {
      or_word(w, m);
      w = x[q] >> 5;
      m = 1u << (x[q] & 31);
    }
  }
  or_word(w, m);
  return true;
}

struct SymBits {
  unsigned* bits;
  int lo;
  unsigned width;
  unsigned* status;
  __device__ __forceinline__ void operator()(int col, float, float) {
    const unsigned c = (unsigned)(col - lo);
    if (c < width) atomicOr(bits + (c >> 5), 1u << (c & 31));
    else atomicOr(status, ST_BAD_INDEX);
  }
  __device__ __forceinline__ void vec4(int4 c4) {
    if (!or_bits4(c4, lo, width, [&](unsigned w, unsigned m) { atomicOr(bits + w, m); })) {
      (*this)(c4.x, 0.f, 0.f);
      (*this)(c4.y, 0.f, 0.f);
      (*this)(c4.z, 0.f, 0.f);
      (*this)(c4.w, 0.f, 0.f);
    }
  }
};

struct NumHashPlain {
  unsigned* keys;
  float* vals;
  int log2t;
  unsigned* status;
  __device__ __forceinline__ void operator()(int col, float a, float b) {
    bool ins;
    const int h = hash_slot(keys, log2t, (unsigned)col, ins, status);
    if (h >= 0) atomicAdd(vals + h, __fmul_rn(a, b));
  }
};

// Compensated accumulate of p = a*b into a (sum, comp) pair. The atomic add
// returns the old sum, and since it rounds to nearest like __fadd_rn, the
// exact error of that very addition is known locally (TwoSum); it is added
// to the compensation word together with the product's own rounding error
// (TwoProduct via FMA). This is Dot2 with the summation order set by the
// order of atomic arrival.
__device__ __forceinline__ void twosum_accumulate(float2* slot, float a, float b) {
  const float p = __fmul_rn(a, b);
  const float ep = __fmaf_rn(a, b, -p);
  const float old = atomicAdd(&slot->x, p);
  const float s = __fadd_rn(old, p);
  const float e = two_sum_err(old, p, s);
  atomicAdd(&slot->y, __fadd_rn(e, ep));
}

struct NumHashTwoSum {
  unsigned* keys;
  float2* vals;
  int log2t;
  unsigned* status;
  __device__ __forceinline__ void operator()(int col, float a, float b) {
    bool ins;
    const int h = hash_slot(keys, log2t, (unsigned)col, ins, status);
    if (h >= 0) twosum_accumulate(vals + h, a, b);
  }
};

struct NumHashF64 {
  unsigned* keys;
  double* vals;
  int log2t;
  unsigned* status;
  __device__ __forceinline__ void operator()(int col, float a, float b) {
    bool ins;
    const int h = hash_slot(keys, log2t, (unsigned)col, ins, status);
    if (h >= 0) atomicAdd(vals + h, (double)a * (double)b);  // exact product
  }
};

// Long rows: directory word w holds the presence bits of columns
// lo + 32w .. lo + 32w + 31 (.x) and the number of present columns before
// it (.y), so a column's output slot is .y + popc(.x & lower bits).
struct LongBits {
  uint2* dir;
  int lo;
  unsigned width;
  unsigned* status;
  __device__ __forceinline__ void operator()(int col, float, float) {
    const unsigned c = (unsigned)(col - lo);
    if (c < width) atomicOr(&dir[c >> 5].x, 1u << (c & 31));
    else atomicOr(status, ST_BAD_INDEX);
  }
  __device__ __forceinline__ void vec4(int4 c4) {
    if (!or_bits4(c4, lo, width, [&](unsigned w, unsigned m) { atomicOr(&dir[w].x, m); })) {
      (*this)(c4.x, 0.f, 0.f);
      (*this)(c4.y, 0.f, 0.f);
      (*this)(c4.z, 0.f, 0.f);
      (*this)(c4.w, 0.f, 0.f);
    }
  }
};

// Fused-pass hash insert: like the numeric inserts, but a full table is not an
// error (the caller redoes the row with a larger structure when it counted
// more distinct columns than its limit), and new keys are counted.
__device__ __forceinline__ int hash_slot_soft(unsigned* keys, int log2t, unsigned col,
                                              bool& inserted) {
  const unsigned mask = (1u << log2t) - 1u;
  unsigned h = hash_col(col, log2t);
  inserted = false;
  for (unsigned probe = 0; probe <= mask; ++probe) {
    const unsigned k = ((volatile unsigned*)keys)[h];
    if (k == col) return (int)h;
    if (k == EMPTY_KEY) {
      const unsigned old = atomicCAS(keys + h, EMPTY_KEY, col);
      if (old == EMPTY_KEY) { inserted = true; return (int)h; }
      if (old == col) return (int)h;
    }
    h = (h + 1u) & mask;
  }
  return -1;
}

// `count` (per warp, shared) counts distinct columns; once it exceeds `limit`
// the row will be redone elsewhere, so further products are skipped.
template <int MODE>  // 0: FP32 add; 1: TwoSum-compensated FP32 pair
struct FusedHash {
  unsigned* keys;
  void* vals;
  int log2t;
  int* count;
  int limit;
  __device__ __forceinline__ void operator()(int col, float a, float b) {
    if (*((volatile int*)count) > limit) return;
    bool ins;
    const int h = hash_slot_soft(keys, log2t, (unsigned)col, ins);
    if (ins) atomicAdd(count, 1);
    if (h < 0) return;
    if (MODE == 0) atomicAdd(static_cast<float*>(vals) + h, __fmul_rn(a, b));
    else twosum_accumulate(static_cast<float2*>(vals) + h, a, b);
  }
};

// Bitonic sort of keys/values[0, n) (n a power of two, >= 1) by any number of
// cooperating threads; Sync synchronises them.
template <class V, class Sync>
__device__ __forceinline__ void bitonic_sort_kv_rt(unsigned* keys, V* vals, int n, int tid,
                                                   int nthreads, Sync sync) {
  for (int k = 2; k <= n; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int t = tid; t < (n >> 1); t += nthreads) {
        const int lo = ((t & ~(j - 1)) << 1) | (t & (j - 1));
        const int hi = lo + j;
        const bool up = (lo & k) == 0;
        const unsigned kl = keys[lo], kh = keys[hi];
        if ((kl > kh) == up) {
          keys[lo] = kh;
          keys[hi] = kl;
          const V vl = vals[lo];
          vals[lo] = vals[hi];
          vals[hi] = vl;
        }
      }
      sync();
    }
  }
}

// bitonic_sort_kv_rt for keys alone (n a power of two, keys unique or padded
// with EMPTY_KEY), by the threads of one warp or block.
template <class Sync>
__device__ __forceinline__ void bitonic_sort_keys_rt(unsigned* keys, int n, int tid, int nthreads,
                                                     Sync sync) {
  for (int k = 2; k <= n; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int t = tid; t < (n >> 1); t += nthreads) {
        const int lo = ((t & ~(j - 1)) << 1) | (t & (j - 1));
        const int hi = lo + j;
        const bool up = (lo & k) == 0;
        const unsigned kl = keys[lo], kh = keys[hi];
        if ((kl > kh) == up) {
          keys[lo] = kh;
          keys[hi] = kl;
        }
      }
      sync();
    }
  }
}

struct LongValTwoSum {
  const uint2* dir;
  float2* vals;
  int* cols;
  int lo;
  unsigned width;
  __device__ __forceinline__ void operator()(int col, float a, float b);
};

// LongBits that also records, in a second-level bitmap l1 (one bit per
// directory word), which directory words became non-empty.
struct LongBitsTracked {
  uint2* dir;
  unsigned* l1;
  int lo;
  unsigned width;
  unsigned* status;
  __device__ __forceinline__ void operator()(int col, float, float) {
    const unsigned c = (unsigned)(col - lo);
    if (c < width) {
      const unsigned w = c >> 5;
      const unsigned old = atomicOr(&dir[w].x, 1u << (c & 31));
      if (old == 0u) atomicOr(l1 + (w >> 5), 1u << (w & 31));
    } else {
      atomicOr(status, ST_BAD_INDEX);
    }
  }
  __device__ __forceinline__ void vec4(int4 c4) {
    auto or_word = [&](unsigned w, unsigned m) {
      const unsigned old = atomicOr(&dir[w].x, m);
      if (old == 0u) atomicOr(l1 + (w >> 5), 1u << (w & 31));
    };
    if (!or_bits4(c4, lo, width, or_word)) {
      (*this)(c4.x, 0.f, 0.f);
      (*this)(c4.y, 0.f, 0.f);
      (*this)(c4.z, 0.f, 0.f);
      (*this)(c4.w, 0.f, 0.f);
    }
  }
};

// Output slot of `col` (only columns whose bit pass 1 set reach here, so
// the slot is below the slice's output count).
__device__ __forceinline__ int long_slot(const uint2* dir, int lo, int col) {
  const unsigned c = (unsigned)(col - lo);
  const uint2 d = dir[c >> 5];
  return (int)(d.y + __popc(d.x & ((1u << (c & 31)) - 1u)));
}

// Value-pass functors of the bitmap slices: accumulate into the output slot
// and record the slot's column, so the write-out copies columns like values
// instead of expanding the directory. Slots start at +0.0; the plain form
// stores the column when its add found the slot still at +0.0 (the first
// product of the column does, so every slot gets its column; a later store
// after an exact cancellation writes the same index again).
// Value functor of whole rows accumulated in shared memory: the output slot
// is the column's rank in the row; the product that finds the slot still at
// +0.0 (the first one does, slots start at +0.0) stores the slot's column
// straight into C's column array, so no write-out of columns is needed.
struct RowValCols {
  const uint2* dir;
  float* vals;   // shared memory, one slot per output
  int* out_col;  // C's columns of the row (global)
  int lo;
  unsigned width;
  __device__ __forceinline__ void operator()(int col, float a, float b) {
    if ((unsigned)(col - lo) < width) {
      const int s = long_slot(dir, lo, col);
      const float old = atomicAdd(vals + s, __fmul_rn(a, b));
      if (__float_as_uint(old) == 0u) __stcs(out_col + s, col);
    }
  }
};

struct LongValPlain {
  const uint2* dir;
  float* vals;
  int* cols;
  int lo;
  unsigned width;
  __device__ __forceinline__ void operator()(int col, float a, float b) {
    if ((unsigned)(col - lo) < width) {
      const int s = long_slot(dir, lo, col);
      const float old = atomicAdd(vals + s, __fmul_rn(a, b));
      if (__float_as_uint(old) == 0u) cols[s] = col;
    }
  }
};

__device__ __forceinline__ void LongValTwoSum::operator()(int col, float a, float b) {
  if ((unsigned)(col - lo) < width) {
    const int s = long_slot(dir, lo, col);
    twosum_accumulate(vals + s, a, b);
    cols[s] = col;
  }
}

struct LongValF64 {
  const uint2* dir;
  double* vals;
  int* cols;
  int lo;
  unsigned width;
  __device__ __forceinline__ void operator()(int col, float a, float b) {
    if ((unsigned)(col - lo) < width) {
      const int s = long_slot(dir, lo, col);
      atomicAdd(vals + s, (double)a * (double)b);
      cols[s] = col;
    }
  }
};

// ---------------------------------------------------------------------------
// Bitonic sort of a power-of-two key/value array in shared memory
// ---------------------------------------------------------------------------

struct WarpSync {
  __device__ __forceinline__ void operator()() const { __syncwarp(); }
};
struct BlockSync {
  __device__ __forceinline__ void operator()() const { __syncthreads(); }
};

template <int N, int NT, class V, class Sync>
__device__ __forceinline__ void bitonic_sort_kv(unsigned* keys, V* vals, int tid,
                                                Sync sync) {
#pragma unroll 1
  for (int k = 2; k <= N; k <<= 1) {
#pragma unroll 1
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int t = tid; t < N / 2; t += NT) {
        const int lo = ((t & ~(j - 1)) << 1) | (t & (j - 1));
        const int hi = lo + j;
        const bool up = (lo & k) == 0;
        const unsigned kl = keys[lo], kh = keys[hi];
        if ((kl > kh) == up) {
          keys[lo] = kh;
          keys[hi] = kl;
          const V vl = vals[lo];
          vals[lo] = vals[hi];
          vals[hi] = vl;
        }
      }
      sync();
    }
  }
}

__device__ __forceinline__ float finalize_value(float v) { return v; }
__device__ __forceinline__ float finalize_value(float2 v) { return __fadd_rn(v.x, v.y); }
__device__ __forceinline__ float finalize_value(double v) { return __double2float_rn(v); }

}  // namespace sg

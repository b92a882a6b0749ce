// __global__ kernels of the SpGEMM pipeline (see kernels.cuh for the
// device primitives they are built from).
#pragma once

#include "kernels.cuh"

namespace sg {

// ---------------------------------------------------------------------------
// Input validation
// ---------------------------------------------------------------------------

// Input validation as two flat passes (coalesced, one thread per pointer,
// then one per entry): pointers inside [0, nnz], non-decreasing, ptr[0] == 0
// and ptr[n_major] == nnz, each segment's first position marked in `starts`
// (nnz bits, zeroed by the caller; null when sortedness is not checked) ...
__global__ void k_validate_ptr(const int* __restrict__ ptr, int n_major, int nnz,
                               unsigned* __restrict__ starts, unsigned* status) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= n_major; i += gridDim.x * blockDim.x) {
    const int s = ptr[i];
    bool bad = s < 0 || s > nnz || (i == 0 && s != 0) || (i == n_major && s != nnz);
    if (i < n_major && s > ptr[i + 1]) bad = true;
    if (bad) atomicOr(status, ST_BAD_INDEX);
    else if (starts && i < n_major && s < nnz) atomicOr(starts + (s >> 5), 1u << (s & 31));
  }
}

// ... then every entry inside [0, n_minor) and, with `starts`, above the
// entry before it unless it begins a segment (B's rows must be sorted: the
// long-row kernels binary-search them). Violations set ST_BAD_INDEX (range)
// or ST_UNSORTED; nothing is read outside ptr[0..n_major] and idx[0..nnz).
__global__ void k_validate_idx(const int* __restrict__ idx, int nnz, int n_minor,
                               const unsigned* __restrict__ starts, unsigned* status) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nnz; q += gridDim.x * blockDim.x) {
    const int v = idx[q];
    if ((unsigned)v >= (unsigned)n_minor) atomicOr(status, ST_BAD_INDEX);
    if (starts && q > 0 && !((starts[q >> 5] >> (q & 31)) & 1u) && idx[q - 1] >= v)
      atomicOr(status, ST_UNSORTED);
  }
}

// ---------------------------------------------------------------------------
// A: CSC -> CSR
// ---------------------------------------------------------------------------

// Count entries per row of A. The reference builds A's CSC with the same
// atomic histogram but never zeroes it first (src/mm.cu:43-63, 89); the
// caller of this kernel zeroes `cnt`.
__global__ void k_transpose_hist(const int* __restrict__ rowidx, int nnz, int m,
                                 int* __restrict__ cnt, unsigned* status) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nnz;
       e += gridDim.x * blockDim.x) {
    const int r = rowidx[e];
    if ((unsigned)r < (unsigned)m) atomicAdd(cnt + r, 1);
    else atomicOr(status, ST_BAD_INDEX);
  }
}

// Scatter CSC entries into CSR order. cursor[] starts as the CSR row
// pointers; the entry order inside a row is the atomic arrival order.
__global__ void k_transpose_scatter(const int* __restrict__ colptr,
                                    const int* __restrict__ rowidx,
                                    const float* __restrict__ val, int kdim, int nnz,
                                    int m, int* __restrict__ cursor,
                                    int* __restrict__ out_col,
                                    float* __restrict__ out_val) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nnz;
       e += gridDim.x * blockDim.x) {
    // column of entry e: last k with colptr[k] <= e
    int lo = 0, hi = kdim;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(colptr + mid) <= e) lo = mid; else hi = mid - 1;
    }
    const int r = rowidx[e];
    if ((unsigned)r >= (unsigned)m) continue;
    const int pos = atomicAdd(cursor + r, 1);
    out_col[pos] = lo;
    out_val[pos] = val[e];
  }
}

// ---------------------------------------------------------------------------
// Row analysis + symbolic binning
// ---------------------------------------------------------------------------

constexpr int RA_THREADS = 256;
constexpr int RA_ROWS = 64;  // rows per block
constexpr int RA_UNROLL = 4;  // 32-entry batches of a row in flight together

// Per row i: P_i = sum over A(i,k) of nnz(B(k,:)) (the intermediate product
// count the reference accumulates per row in initGEMM, src/mm.cu:138-148),
// the flattened offset of each A entry, the column span of the row's
// products, the first-pass bin, and tcap[i] = the column bound min(P_i, n,
// span_i) for rows the fused pass computes (0 otherwise), which sizes their
// slot in the temporary output buffer. Rows are appended to their bin's list
// with one global atomic per bin per block. B's pointers are range-checked
// here because the validation pass's result is only read after this kernel.
__global__ void __launch_bounds__(RA_THREADS)
k_row_analysis(Operands op, int* __restrict__ aoff, long long* __restrict__ row_p,
               int* __restrict__ c_cnt, int* __restrict__ tcap, int* __restrict__ fb_count,
               int* __restrict__ fb_rows, unsigned long long* __restrict__ p_total,
               int* __restrict__ max_row_len, int2* __restrict__ row_span, unsigned* status,
               Tuning tn) {
  __shared__ int hist[FB_COUNT], base[FB_COUNT];
  __shared__ int rowbin[RA_ROWS], rowrank[RA_ROWS];
  __shared__ unsigned long long block_p;
  __shared__ int block_max_len;  // longest A row of the block (one global atomic per block)
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row0 = blockIdx.x * RA_ROWS;
  if (threadIdx.x < FB_COUNT) hist[threadIdx.x] = 0;
  if (threadIdx.x == 0) {
    block_p = 0;
    block_max_len = 0;
  }
  __syncthreads();
  for (int lr = warp; lr < RA_ROWS; lr += RA_THREADS / 32) {
    const int i = row0 + lr;
    if (i >= op.m) {
      if (lane == 0) rowbin[lr] = -1;
      continue;
    }
    const int rs = op.a_rowptr[i], re = op.a_rowptr[i + 1];
    long long acc = 0;
    int lo = 0x7fffffff, hi = -1;  // column span of the row's products
    // Entry j's B row length and first/last column (invalid indices are
    // reported and count as empty).
    auto entry = [&](int j, int& bs, int& be) {
      const int k = op.a_col[j];
      bs = be = 0;
      if ((unsigned)k >= (unsigned)op.kdim) {
        atomicOr(status, ST_BAD_INDEX);
        return;
      }
      const int s0 = op.b_rowptr[k], s1 = op.b_rowptr[k + 1];
      if (s0 >= 0 && s1 <= op.nnz_b && s0 <= s1) {
        bs = s0;
        be = s1;
      } else {
        atomicOr(status, ST_BAD_INDEX);
      }
    };
    if (re - rs <= 32) {  // one batch (most rows)
      const int j = rs + lane;
      int bs = 0, be = 0;
      if (j < re) entry(j, bs, be);
      if (be > bs) {
        lo = min(lo, op.b_col[bs]);
        hi = max(hi, op.b_col[be - 1]);
      }
      const long long len = be - bs;
      const long long incl = warp_incl_scan64(len);
      if (j < re) aoff[j] = (int)(incl - len);
      acc = __shfl_sync(FULL, incl, 31);
    } else {
      // RA_UNROLL batches of 32 entries at a time, each level of the
      // dependent loads (A's column, B's row bounds, B's first and last
      // column) issued for all of them before the next, so a long row of A
      // is not walked one round trip after another
      for (int b0 = rs; b0 < re; b0 += 32 * RA_UNROLL) {
        int k[RA_UNROLL], bs[RA_UNROLL], be[RA_UNROLL];
        bool ok[RA_UNROLL];
#pragma unroll
        for (int u = 0; u < RA_UNROLL; ++u) {
          const int j = b0 + 32 * u + lane;
          k[u] = j < re ? op.a_col[j] : 0;
          ok[u] = j < re;
          if (ok[u] && (unsigned)k[u] >= (unsigned)op.kdim) {
            atomicOr(status, ST_BAD_INDEX);
            ok[u] = false;
          }
        }
#pragma unroll
        for (int u = 0; u < RA_UNROLL; ++u) {
          bs[u] = ok[u] ? op.b_rowptr[k[u]] : 0;
          be[u] = ok[u] ? op.b_rowptr[k[u] + 1] : 0;
          if (ok[u] && !(bs[u] >= 0 && be[u] <= op.nnz_b && bs[u] <= be[u])) {
            atomicOr(status, ST_BAD_INDEX);
            ok[u] = false;
          }
        }
#pragma unroll
        for (int u = 0; u < RA_UNROLL; ++u) {
          if (ok[u] && be[u] > bs[u]) {
            lo = min(lo, op.b_col[bs[u]]);
            hi = max(hi, op.b_col[be[u] - 1]);
          }
        }
#pragma unroll
        for (int u = 0; u < RA_UNROLL; ++u) {
          if (b0 + 32 * u < re) {  // warp-uniform
            const int j = b0 + 32 * u + lane;
            const long long len = ok[u] ? (long long)(be[u] - bs[u]) : 0;
            const long long incl = warp_incl_scan64(len);
            if (j < re) aoff[j] = (int)(acc + incl - len);
            acc += __shfl_sync(FULL, incl, 31);
          }
        }
      }
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
      lo = min(lo, __shfl_xor_sync(FULL, lo, d));
      hi = max(hi, __shfl_xor_sync(FULL, hi, d));
    }
    if (lane == 0) {
      if (re - rs > 0) atomicMax(&block_max_len, re - rs);
      const int span = acc > 0 ? hi + 1 - lo : 0;
      row_span[i] = acc > 0 ? make_int2(lo, hi) : make_int2(0, -1);
      row_p[i] = acc;
      if (acc >= (1ll << 31)) atomicOr(status, ST_ROW_TOO_LONG);
      const long long cap = row_cap(acc, op.n, span);
      const int bin = first_bin_of(acc, cap, span, tn);
      if (bin < 0) c_cnt[i] = 0;
      tcap[i] = (bin >= 0 && bin != FB_LONG) ? (int)cap : 0;
      rowbin[lr] = bin;
      if (bin >= 0) rowrank[lr] = atomicAdd(&hist[bin], 1);
      atomicAdd(&block_p, (unsigned long long)acc);
    }
  }
  __syncthreads();
  if (threadIdx.x < FB_COUNT && hist[threadIdx.x])
    base[threadIdx.x] = atomicAdd(fb_count + threadIdx.x, hist[threadIdx.x]);
  if (threadIdx.x == 0) {
    atomicAdd(p_total, block_p);
    if (block_max_len > 0) atomicMax(max_row_len, block_max_len);
  }
  __syncthreads();
  for (int lr = threadIdx.x; lr < RA_ROWS; lr += RA_THREADS) {
    const int b = rowbin[lr];
    if (b >= 0) fb_rows[(size_t)b * op.m + base[b] + rowrank[lr]] = row0 + lr;
  }
}

// ---------------------------------------------------------------------------
// Symbolic pass
// ---------------------------------------------------------------------------

__device__ __forceinline__ long long block_excl_scan64(long long v, long long* shm,
                                                       long long& total);

constexpr int SW_THREADS = 256;  // warp-per-row kernels: 8 warps per block

// Value slot type of each precision mode (0 plain, 1 compensated).
template <int MODE> struct SlotOf { using T = float; };
template <> struct SlotOf<1> { using T = unsigned long long; };  // float2 or double bits

// Fused pass, one warp per row: hash accumulate, compact the table in place,
// sort the occupied entries by column, write the sorted row to the temporary
// buffer at toff[i] and its length to c_cnt[i]. A row that turns out to have
// more distinct columns than 4/5 of the table is pushed to the sorted bins
// (when the tuning sorts rows like it), else to the mid list (span within
// mid_cols) or the largest block list, and redone there.
//
// Sorting: tables of 256 slots and more sort packed keys (column offset in
// the row's span above the slot index; the values stay in their slots) by a
// bucket pass -- NB = T/4 buckets on the column offset's top bits, counts,
// scan, scatter with the keys held in registers -- and an insertion sort of
// each bucket by one lane. Rows whose columns crowd one bucket (more than
// BUCKET_MAX entries: skewed column popularity) take LSD radix passes over
// the column offset instead. Rows of at most SMALL_SORT entries (and small
// tables) sort the packed keys bitonically; rows whose span is too wide to
// pack sort key/value pairs bitonically.
constexpr int BUCKET_MAX = 24;
constexpr int SMALL_SORT = 128;  // rows with at most this many entries sort bitonically

template <int LOG2T, int MODE>
__global__ void __launch_bounds__(SW_THREADS, LOG2T >= 10 ? 2 : 4)
k_fused_warp(Operands op, const int* __restrict__ rows, int nrows,
             const int2* __restrict__ row_span, const long long* __restrict__ toff,
             int* __restrict__ c_cnt, int* __restrict__ t_col, float* __restrict__ t_val,
             int* __restrict__ mid_rows, int* __restrict__ mid_count,
             int* __restrict__ big_rows, int* __restrict__ big_count, int mid_cols,
             int* __restrict__ esc_rows, int* __restrict__ esc_count, Tuning tn,
             const long long* __restrict__ row_p, int* __restrict__ overflow_count) {
  constexpr int T = 1 << LOG2T;
  constexpr int LIMIT = T * 4 / 5;
  constexpr int WPB = SW_THREADS / 32;
  using V = typename SlotOf<MODE>::T;
  extern __shared__ __align__(16) unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  V* vals = reinterpret_cast<V*>(smem) + warp * T;
  unsigned* keys = reinterpret_cast<unsigned*>(smem + WPB * T * sizeof(V)) + warp * T;
  SegScratch* sc = reinterpret_cast<SegScratch*>(smem + WPB * T * (sizeof(V) + 4)) + warp;
  constexpr int NB = T / 4;                   // sort buckets (tables of >= 256 slots)
  constexpr int E = (LIMIT + 31) / 32;        // entries per lane
  int* bucket = reinterpret_cast<int*>(smem + WPB * (T * (sizeof(V) + 4) + sizeof(SegScratch))) +
                warp * NB;
  for (int r = blockIdx.x * WPB + warp; r < nrows; r += gridDim.x * WPB) {
    const int i = rows[r];
    for (int t = lane; t < T; t += 32) { keys[t] = EMPTY_KEY; vals[t] = V(0); }
    if (lane == 0) sc->count = 0;
    __syncwarp();
    FusedHash<MODE> f{keys, vals, LOG2T, &sc->count, LIMIT};
    warp_expand_row<true>(op, op.a_rowptr[i], op.a_rowptr[i + 1], f, sc, LIMIT);
    __syncwarp();
    const int distinct = *((volatile int*)&sc->count);
    __syncwarp();
    if (distinct > LIMIT) {  // redo with a larger structure
      if (lane == 0) {
        const int2 sp = row_span[i];
        const long long p = row_p[i];
        if (p > tn.esc_p_min && sp.y + 1 - sp.x > tn.esc_span_min && p <= 4096) {
          const int q = p <= 1024 ? 0 : (p <= 2048 ? 1 : 2);  // sorted bins, as first_bin_of
          esc_rows[(size_t)q * op.m + atomicAdd(esc_count + q, 1)] = i;
        } else if (sp.y + 1 - (sp.x & ~31) <= mid_cols) {
          mid_rows[atomicAdd(mid_count, 1)] = i;
        } else {
          big_rows[atomicAdd(big_count, 1)] = i;
        }
        atomicAdd(overflow_count, 1);
      }
      continue;
    }
    // compact in place: entries move to lower slots only, after the whole
    // 32-slot group has been read
    int o = 0;
    for (int g = 0; g < T; g += 32) {
      const unsigned k = keys[g + lane];
      const V v = vals[g + lane];
      const bool valid = k != EMPTY_KEY;
      const unsigned bal = __ballot_sync(FULL, valid);
      const int pos = o + __popc(bal & ((1u << lane) - 1u));
      __syncwarp();
      if (valid) { keys[pos] = k; vals[pos] = v; }
      o += __popc(bal);
      __syncwarp();
    }
    int n2 = 1;
    while (n2 < o) n2 <<= 1;
    const long long base = toff[i];
    const int2 sp = row_span[i];
    const unsigned lo = (unsigned)(sp.x & ~31);
    const unsigned span = (unsigned)(sp.y + 1) - lo;
    if (span <= (1u << (32 - LOG2T)) && (LOG2T < 8 || o <= SMALL_SORT)) {
      // packed keys, (column - lo) << LOG2T | slot, sorted bitonically
      for (int t = lane; t < n2; t += 32)
        keys[t] = t < o ? ((keys[t] - lo) << LOG2T) | (unsigned)t : EMPTY_KEY;
      __syncwarp();
      bitonic_sort_keys_rt(keys, n2, lane, 32, WarpSync());
      for (int t = lane; t < o; t += 32) {
        const unsigned p = keys[t];
        const int slot = (int)(p & (T - 1));
        t_col[base + t] = (int)(lo + (p >> LOG2T));
        if (MODE == 0) t_val[base + t] = finalize_value(reinterpret_cast<float*>(vals)[slot]);
        else t_val[base + t] = finalize_value(reinterpret_cast<float2*>(vals)[slot]);
      }
    } else if (LOG2T >= 8 && span <= (1u << (32 - LOG2T))) {
      // packed keys: (column - lo) << LOG2T | slot
      unsigned pk[E];
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int t = lane + 32 * e;
        pk[e] = t < o ? ((keys[t] - lo) << LOG2T) | (unsigned)t : EMPTY_KEY;
      }
      const int bits = 32 - __clz(span > 1 ? span - 1 : 1);
      const int shift = bits > LOG2T - 2 ? bits - (LOG2T - 2) : 0;
      for (int t = lane; t < NB; t += 32) bucket[t] = 0;
      __syncwarp();
#pragma unroll
      for (int e = 0; e < E; ++e)
        if (pk[e] != EMPTY_KEY) atomicAdd(&bucket[(pk[e] >> LOG2T) >> shift], 1);
      __syncwarp();
      constexpr int PER = NB / 32 > 0 ? NB / 32 : 1;
      int cnt[PER];
      int sum = 0, mx = 0;
#pragma unroll
      for (int q = 0; q < PER; ++q) {
        cnt[q] = bucket[lane * PER + q];
        sum += cnt[q];
        mx = max(mx, cnt[q]);
      }
#pragma unroll
      for (int d = 16; d > 0; d >>= 1) mx = max(mx, __shfl_xor_sync(FULL, mx, d));
      if (mx <= BUCKET_MAX) {
        int run = warp_incl_scan(sum) - sum;
#pragma unroll
        for (int q = 0; q < PER; ++q) {
          bucket[lane * PER + q] = run;
          run += cnt[q];
        }
        __syncwarp();
        // every key is in registers: scatter into the key array by bucket
#pragma unroll
        for (int e = 0; e < E; ++e)
          if (pk[e] != EMPTY_KEY) keys[atomicAdd(&bucket[(pk[e] >> LOG2T) >> shift], 1)] = pk[e];
        __syncwarp();
        // bucket b now ends at bucket[b]; each lane sorts its buckets in place
        for (int b = lane; b < NB; b += 32) {
          const int s0 = b ? bucket[b - 1] : 0, s1 = bucket[b];
          for (int x = s0 + 1; x < s1; ++x) {
            const unsigned v = keys[x];
            int y = x - 1;
            while (y >= s0 && keys[y] > v) {
              keys[y + 1] = keys[y];
              --y;
            }
            keys[y + 1] = v;
          }
        }
      } else {
        // crowded buckets (skewed columns): LSD radix sort of the column
        // offset, LOG2T - 2 bits (NB counters) a pass, stable by array order;
        // each pass scatters from registers into the key array, then reloads
        // the keys in the new order
        constexpr int DIG = LOG2T - 2;
        for (int d0 = 0; d0 < bits; d0 += DIG) {
          for (int t = lane; t < NB; t += 32) bucket[t] = 0;
          __syncwarp();
#pragma unroll
          for (int e = 0; e < E; ++e)
            if (pk[e] != EMPTY_KEY) atomicAdd(&bucket[((pk[e] >> LOG2T) >> d0) & (NB - 1)], 1);
          __syncwarp();
          int tot = 0;
#pragma unroll
          for (int q = 0; q < PER; ++q) {
            cnt[q] = bucket[lane * PER + q];
            tot += cnt[q];
          }
          int run = warp_incl_scan(tot) - tot;
#pragma unroll
          for (int q = 0; q < PER; ++q) {
            bucket[lane * PER + q] = run;
            run += cnt[q];
          }
          __syncwarp();
#pragma unroll
          for (int e = 0; e < E; ++e) {
            const bool valid = pk[e] != EMPTY_KEY;
            const unsigned dig = valid ? ((pk[e] >> LOG2T) >> d0) & (NB - 1) : (unsigned)(NB + lane);
            const unsigned peers = __match_any_sync(FULL, dig);
            const int rank = __popc(peers & ((1u << lane) - 1u));
            int pos = 0;
            if (valid) pos = bucket[dig] + rank;
            __syncwarp();
            if (valid) {
              keys[pos] = pk[e];
              if (rank == __popc(peers) - 1) bucket[dig] = pos + 1;
            }
            __syncwarp();
          }
#pragma unroll
          for (int e = 0; e < E; ++e) {
            const int t = lane + 32 * e;
            pk[e] = t < o ? keys[t] : EMPTY_KEY;
          }
          __syncwarp();
        }
      }
      __syncwarp();
      for (int t = lane; t < o; t += 32) {
        const unsigned p = keys[t];
        const int slot = (int)(p & (T - 1));
        t_col[base + t] = (int)(lo + (p >> LOG2T));
        if (MODE == 0) t_val[base + t] = finalize_value(reinterpret_cast<float*>(vals)[slot]);
        else t_val[base + t] = finalize_value(reinterpret_cast<float2*>(vals)[slot]);
      }
    } else {
      for (int t = o + lane; t < n2; t += 32) keys[t] = EMPTY_KEY;
      __syncwarp();
      bitonic_sort_kv_rt(keys, vals, n2, lane, 32, WarpSync());
      for (int t = lane; t < o; t += 32) {
        t_col[base + t] = (int)keys[t];
        if (MODE == 0) t_val[base + t] = finalize_value(reinterpret_cast<float*>(vals)[t]);
        else t_val[base + t] = finalize_value(reinterpret_cast<float2*>(vals)[t]);
      }
    }
    if (lane == 0) c_cnt[i] = o;
    __syncwarp();
  }
}

// Fused pass, one block per row (rows whose column bound needs more than a
// warp's table and whose span is too wide for the bitmap): hash accumulate
// into 2^LOG2T slots (load <= 1/2), block compaction, bitonic sort, write the
// sorted row to the temporary buffer. The row list may grow while earlier
// kernels run (warp overflow), so its length is read from device memory.
template <int LOG2T, int NT, int MODE>
__global__ void __launch_bounds__(NT, NT >= 512 ? 2 : 4)
k_fused_block(Operands op, const int* __restrict__ rows, const int* __restrict__ nrows_p,
              const long long* __restrict__ row_p, const long long* __restrict__ toff,
              const int2* __restrict__ row_span, int* __restrict__ c_cnt,
              int* __restrict__ t_col, float* __restrict__ t_val, unsigned* status) {
  constexpr int T = 1 << LOG2T;
  constexpr int NW = NT / 32;
  constexpr int PER = T / NT;  // slots per thread in the compaction
  using V = typename SlotOf<MODE>::T;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ long long scan_shm[33];
  const int warp = threadIdx.x >> 5;
  V* vals = reinterpret_cast<V*>(smem);
  unsigned* keys = reinterpret_cast<unsigned*>(smem + T * sizeof(V));
  SegScratch* sc = reinterpret_cast<SegScratch*>(smem + T * (sizeof(V) + 4)) + warp;
  constexpr int NB = T / 4;         // sort buckets
  constexpr int PB = NB / NT;       // bucket counters per thread in the scan
  int* bucket = reinterpret_cast<int*>(smem + T * (sizeof(V) + 4) + NW * sizeof(SegScratch));
  __shared__ int bucket_max;
  const int nrows = *nrows_p;
  for (int r = blockIdx.x; r < nrows; r += gridDim.x) {
    const int i = rows[r];
    const long long p = row_p[i];
    for (int t = threadIdx.x; t < T; t += NT) { keys[t] = EMPTY_KEY; vals[t] = V(0); }
    __syncthreads();
    const int rs = op.a_rowptr[i], re = op.a_rowptr[i + 1];
    const int U = chunk_for(p, NW, 1 << 20);
    if (MODE == 0) {
      NumHashPlain f{keys, reinterpret_cast<float*>(vals), LOG2T, status};
      for (int c0 = warp * U; c0 < p; c0 += NW * U)
        warp_expand_range<true>(op, rs, re, c0, (int)min((long long)c0 + U, p), f, sc);
    } else {
      NumHashTwoSum f{keys, reinterpret_cast<float2*>(vals), LOG2T, status};
      for (int c0 = warp * U; c0 < p; c0 += NW * U)
        warp_expand_range<true>(op, rs, re, c0, (int)min((long long)c0 + U, p), f, sc);
    }
    __syncthreads();
    // compaction: read my PER slots, scan the counts, write after a barrier
    unsigned k[PER];
    V v[PER];
    int mine = 0;
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      k[q] = keys[threadIdx.x * PER + q];
      v[q] = vals[threadIdx.x * PER + q];
      mine += k[q] != EMPTY_KEY;
    }
    long long o64;
    long long pos = block_excl_scan64(mine, scan_shm, o64);
    const int o = (int)o64;
    const int pos0 = (int)pos;
#pragma unroll
    for (int q = 0; q < PER; ++q)
      if (k[q] != EMPTY_KEY) { keys[pos] = k[q]; vals[pos] = v[q]; ++pos; }
    __syncthreads();
    int n2 = 1;
    while (n2 < o) n2 <<= 1;
    const long long base = toff[i];
    const int2 sp = row_span[i];
    const unsigned lo = (unsigned)(sp.x & ~31);
    const unsigned span = (unsigned)(sp.y + 1) - lo;
    bool sorted_packed = false;
    if (o > 256 && span <= (1u << (32 - LOG2T))) {
      // packed keys (column - lo) << LOG2T | slot, held in registers; the
      // values stay in their compacted slots. Bucket pass on the column
      // offset's top bits + per-bucket insertion, as in k_fused_warp.
      unsigned pk[PER];
      int j = pos0;
#pragma unroll
      for (int q = 0; q < PER; ++q)
        pk[q] = k[q] != EMPTY_KEY ? ((k[q] - lo) << LOG2T) | (unsigned)(j++) : EMPTY_KEY;
      const int bits = 32 - __clz(span > 1 ? span - 1 : 1);
      const int shift = bits > LOG2T - 2 ? bits - (LOG2T - 2) : 0;
      for (int t = threadIdx.x; t < NB; t += NT) bucket[t] = 0;
      if (threadIdx.x == 0) bucket_max = 0;
      __syncthreads();
#pragma unroll
      for (int q = 0; q < PER; ++q)
        if (pk[q] != EMPTY_KEY) atomicAdd(&bucket[(pk[q] >> LOG2T) >> shift], 1);
      __syncthreads();
      int cnt[PB], sum = 0, mx = 0;
#pragma unroll
      for (int q = 0; q < PB; ++q) {
        cnt[q] = bucket[threadIdx.x * PB + q];
        sum += cnt[q];
        mx = max(mx, cnt[q]);
      }
      if (mx > BUCKET_MAX) atomicMax(&bucket_max, mx);
      long long tot;
      long long run = block_excl_scan64(sum, scan_shm, tot);  // ends with a barrier
      if (bucket_max == 0) {
#pragma unroll
        for (int q = 0; q < PB; ++q) {
          bucket[threadIdx.x * PB + q] = (int)run;
          run += cnt[q];
        }
        __syncthreads();
        // every key is in registers: scatter into the key array by bucket
#pragma unroll
        for (int q = 0; q < PER; ++q)
          if (pk[q] != EMPTY_KEY) keys[atomicAdd(&bucket[(pk[q] >> LOG2T) >> shift], 1)] = pk[q];
        __syncthreads();
        for (int b = threadIdx.x; b < NB; b += NT) {
          const int s0 = b ? bucket[b - 1] : 0, s1 = bucket[b];
          for (int x = s0 + 1; x < s1; ++x) {
            const unsigned kv = keys[x];
            int y = x - 1;
            while (y >= s0 && keys[y] > kv) {
              keys[y + 1] = keys[y];
              --y;
            }
            keys[y + 1] = kv;
          }
        }
        __syncthreads();
        sorted_packed = true;
      }
      // crowded buckets: the key/value bitonic sort below
    }
    if (sorted_packed) {
      for (int t = threadIdx.x; t < o; t += NT) {
        const unsigned p = keys[t];
        const int slot = (int)(p & (T - 1));
        t_col[base + t] = (int)(lo + (p >> LOG2T));
        if (MODE == 0) t_val[base + t] = finalize_value(reinterpret_cast<float*>(vals)[slot]);
        else t_val[base + t] = finalize_value(reinterpret_cast<float2*>(vals)[slot]);
      }
    } else {
      for (int t = o + threadIdx.x; t < n2; t += NT) keys[t] = EMPTY_KEY;
      __syncthreads();
      bitonic_sort_kv_rt(keys, vals, n2, threadIdx.x, NT, BlockSync());
      for (int t = threadIdx.x; t < o; t += NT) {
        t_col[base + t] = (int)keys[t];
        if (MODE == 0) t_val[base + t] = finalize_value(reinterpret_cast<float*>(vals)[t]);
        else t_val[base + t] = finalize_value(reinterpret_cast<float2*>(vals)[t]);
      }
    }
    if (threadIdx.x == 0) c_cnt[i] = o;
    __syncthreads();
  }
}

constexpr int LONG_THREADS = 1024;

// Exact nnz of long rows: presence bitmap of the row's columns in shared
// memory, one window of `tn.sym_window` columns at a time. Also records the
// nnz of every 2048-column chunk, from which k_num_bin cuts column slices.
__global__ void __launch_bounds__(LONG_THREADS, 2)
k_sym_long(Operands op, const int* __restrict__ rows, int nrows,
           const long long* __restrict__ row_p, int* __restrict__ c_cnt,
           int* __restrict__ long_slot, int* __restrict__ chunk_cnt, int n_chunks,
           int* __restrict__ scratch, int scratch_stride, unsigned* __restrict__ bitmaps,
           int bitmap_words, unsigned* status, Tuning tn) {
  constexpr int NW = LONG_THREADS / 32;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int total;
  __shared__ long long scan_shm[33];
  __shared__ int carry_shm;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  SegScratch* sc = reinterpret_cast<SegScratch*>(smem) + warp;
  unsigned* bits = reinterpret_cast<unsigned*>(smem + NW * sizeof(SegScratch));
  int* seg_start = scratch + (size_t)blockIdx.x * scratch_stride;
  const int n = op.n;
  for (int r = blockIdx.x; r < nrows; r += gridDim.x) {
    const int i = rows[r];
    const int p = (int)row_p[i];
    const int rs = op.a_rowptr[i], re = op.a_rowptr[i + 1];
    int* roff = seg_start + (re - rs);
    if (threadIdx.x == 0) { total = 0; long_slot[i] = r; }
    for (int w0 = 0; w0 < n; w0 += tn.sym_window) {
      const int wcols = min(n - w0, tn.sym_window);
      const int nw = (wcols + 31) >> 5;
      for (int t = threadIdx.x; t < nw; t += LONG_THREADS) bits[t] = 0u;
      __syncthreads();
      SymBits f{bits, w0, (unsigned)wcols, status};
      if (w0 == 0 && wcols == n) {
        block_walk_row<false>(op, rs, re, true, nullptr, nullptr, p, f, sc, warp, NW);
      } else {
        const int pw = block_restrict_row(op, rs, re, w0, w0 + wcols, seg_start, roff,
                                          scan_shm, &carry_shm);
        const int U = chunk_for(pw, NW, 1 << 20);
        for (int c0 = warp * U; c0 < pw; c0 += NW * U)
          warp_expand_explicit<false>(op, rs, re - rs, seg_start, roff, c0, min(c0 + U, pw), f, sc);
      }
      __syncthreads();
      // keep the presence bitmap for the numeric pass (when memory allows)
      if (bitmap_words > 0) {
        unsigned* dst = bitmaps + (size_t)r * bitmap_words + (w0 >> 5);
        for (int t = threadIdx.x; t < nw; t += LONG_THREADS) dst[t] = bits[t];
      }
      // chunk counts (w0 is a multiple of CHUNK_COLS)
      const int nchunk_w = (nw + CHUNK_WORDS - 1) / CHUNK_WORDS;
      for (int c = warp; c < nchunk_w; c += NW) {
        int v = 0;
        for (int t = lane; t < CHUNK_WORDS; t += 32) {
          const int w = c * CHUNK_WORDS + t;
          if (w < nw) v += __popc(bits[w]);
        }
        v = warp_sum(v);
        if (lane == 0) {
          chunk_cnt[(size_t)r * n_chunks + w0 / CHUNK_COLS + c] = v;
          if (v) atomicAdd(&total, v);
        }
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) c_cnt[i] = total;
  }
}

// ---------------------------------------------------------------------------
// Scan (row pointers of C)
// ---------------------------------------------------------------------------

constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

__device__ __forceinline__ long long block_excl_scan64(long long v, long long* shm,
                                                       long long& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long long incl = warp_incl_scan64(v);
  if (lane == 31) shm[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    const long long w = (lane < (int)(blockDim.x >> 5)) ? shm[lane] : 0;
    const long long wi = warp_incl_scan64(w);
    shm[lane] = wi - w;
    if (lane == 31) shm[32] = wi;
  }
  __syncthreads();
  const long long r = shm[warp] + incl - v;
  total = shm[32];
  __syncthreads();
  return r;
}

// Phase 1: per-tile sums of an int32 array.
__global__ void __launch_bounds__(SCAN_THREADS)
k_scan_tiles(const int* __restrict__ in, int n, long long* __restrict__ tile_sum) {
  __shared__ long long shm[33];
  const long long base = (long long)blockIdx.x * SCAN_TILE;
  long long v = 0;
#pragma unroll
  for (int q = 0; q < SCAN_ITEMS; ++q) {
    const long long idx = base + threadIdx.x * SCAN_ITEMS + q;
    if (idx < n) v += in[idx];
  }
  long long total;
  block_excl_scan64(v, shm, total);
  if (threadIdx.x == 0) tile_sum[blockIdx.x] = total;
}

// Phase 2: exclusive scan of the tile sums (single block, looping).
__global__ void __launch_bounds__(SCAN_THREADS)
k_scan_tile_sums(long long* __restrict__ tile_sum, int ntiles,
                 long long* __restrict__ grand_total) {
  __shared__ long long shm[33];
  long long carry = 0;
  for (int b = 0; b < ntiles; b += SCAN_THREADS) {
    const int idx = b + threadIdx.x;
    const long long v = idx < ntiles ? tile_sum[idx] : 0;
    long long total;
    const long long ex = block_excl_scan64(v, shm, total);
    if (idx < ntiles) tile_sum[idx] = carry + ex;
    carry += total;
  }
  if (threadIdx.x == 0) *grand_total = carry;
}

// Phase 3: out[i] = exclusive prefix of in (int64), out[n] = total.
__global__ void __launch_bounds__(SCAN_THREADS)
k_scan_apply(const int* __restrict__ in, int n, const long long* __restrict__ tile_off,
             const long long* __restrict__ grand_total, long long* __restrict__ out) {
  __shared__ long long shm[33];
  const long long base = (long long)blockIdx.x * SCAN_TILE;
  int v[SCAN_ITEMS];
  long long sum = 0;
#pragma unroll
  for (int q = 0; q < SCAN_ITEMS; ++q) {
    const long long idx = base + threadIdx.x * SCAN_ITEMS + q;
    v[q] = idx < n ? in[idx] : 0;
    sum += v[q];
  }
  long long total;
  long long run = block_excl_scan64(sum, shm, total) + tile_off[blockIdx.x];
#pragma unroll
  for (int q = 0; q < SCAN_ITEMS; ++q) {
    const long long idx = base + threadIdx.x * SCAN_ITEMS + q;
    if (idx < n) out[idx] = run;
    run += v[q];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = *grand_total;
}

// int64 row pointers -> the int32 row pointers of the cm boundary.
__global__ void k_rowptr_to_i32(const long long* __restrict__ in, int n1,
                                int* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n1; i += gridDim.x * blockDim.x)
    out[i] = (int)in[i];
}

// int32 CSC/CSR pointer array from counts (used by the transpose).
// Row pointers of a block-diagonal batch, per product: product p =
// blockIdx.y owns the global rows [row_off[p], row_off[p + 1]); its m_p + 1
// pointers, relative to its first entry, go to out[row_off[p] + p ...].
__global__ void __launch_bounds__(256)
k_batch_rowptr(const long long* __restrict__ rowptr64, const long long* __restrict__ row_off,
               int* __restrict__ out) {
  const int p = blockIdx.y;
  const long long r0 = row_off[p], r1 = row_off[p + 1];
  const long long base = rowptr64[r0];
  for (long long r = r0 + (long long)blockIdx.x * blockDim.x + threadIdx.x; r <= r1;
       r += (long long)gridDim.x * blockDim.x)
    out[r + p] = (int)(rowptr64[r] - base);
}

__global__ void k_rowptr_i64_to_i32_shift(const long long* __restrict__ in, int n1,
                                          int* __restrict__ out, int* __restrict__ out2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n1; i += gridDim.x * blockDim.x) {
    out[i] = (int)in[i];
    if (out2) out2[i] = (int)in[i];
  }
}

// Rows finished by the fused pass: copy each row's sorted entries from the
// temporary buffer (slot toff[i], c_cnt[i] entries) to its place in C. One
// warp per row; rows with tcap == 0 (empty or long) are skipped.
__global__ void __launch_bounds__(256)
k_copy_fused(int r0, int r1, const int* __restrict__ tcap, const long long* __restrict__ toff,
             const int* __restrict__ c_cnt, const long long* __restrict__ c_rowptr,
             const int* __restrict__ t_col, const float* __restrict__ t_val,
             int* __restrict__ c_col, float* __restrict__ c_val) {
  // Rows [r0, r1). A warp takes 32 rows at a time: each lane loads one row's
  // length and offsets (so the 32 rows' loads are in flight together), then
  // the warp copies the rows one after the other, two entries per lane per
  // step.
  const int lane = threadIdx.x & 31;
  const long long warps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long i0 = r0 + (((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; i0 < r1;
       i0 += warps * 32) {
    const long long i = i0 + lane;
    int n = 0;
    long long src = 0, dst = 0;
    if (i < r1 && tcap[i] != 0) {
      n = c_cnt[i];
      src = toff[i];
      dst = c_rowptr[i];
    }
    for (int r = 0; r < 32; ++r) {
      const int nr = __shfl_sync(FULL, n, r);
      if (nr == 0) continue;  // warp-uniform
      const long long s = __shfl_sync(FULL, src, r), d = __shfl_sync(FULL, dst, r);
      for (int t = lane; t < nr; t += 64) {
        const bool two = t + 32 < nr;
        const int c0 = __ldcs(t_col + s + t);
        const float v0 = __ldcs(t_val + s + t);
        int c1 = 0;
        float v1 = 0.f;
        if (two) {
          c1 = __ldcs(t_col + s + t + 32);
          v1 = __ldcs(t_val + s + t + 32);
        }
        __stcs(c_col + d + t, c0);
        __stcs(c_val + d + t, v0);
        if (two) {
          __stcs(c_col + d + t + 32, c1);
          __stcs(c_val + d + t + 32, v1);
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Numeric binning + long-row slicing
// ---------------------------------------------------------------------------

constexpr int NBIN_THREADS = 256;

__device__ __forceinline__ void push_slice(Slice* list, int* count, int capacity, const Slice& v,
                                           unsigned* status) {
  const int s = atomicAdd(count, 1);
  if (s < capacity) list[s] = v;
  else atomicOr(status, ST_SLICE_OVERFLOW);
}

// Numeric binning of the long rows (P_i > long_p; every other row was
// finished by the fused pass). Rows whose outputs fit one block's shared
// memory and whose column span is narrow enough get one bitmap slice
// covering the span: rows with nnz_i > long_o_num in the big-slice list,
// rows with mid_o_min < nnz_i <= long_o_num in the mid-slice list. Rows that
// do not fit are cut into column slices from the symbolic pass's per-chunk
// counts. The rest go to the block hash bins. `bits_kept`: the symbolic pass
// kept the long rows' bitmaps.
__global__ void __launch_bounds__(NBIN_THREADS)
k_num_bin(int m, int n, const int* __restrict__ c_cnt, const long long* __restrict__ row_p,
          const long long* __restrict__ c_rowptr, const int2* __restrict__ row_span,
          int* __restrict__ num_count, int* __restrict__ num_rows,
          const int* __restrict__ chunk_cnt, int n_chunks, const int* __restrict__ long_slot,
          Slice* __restrict__ big, int* __restrict__ big_count, int big_capacity,
          Slice* __restrict__ mid, int* __restrict__ mid_count, int bits_kept,
          unsigned* status, Tuning tn, int rows_cnt_max, int rows_max_words) {
  __shared__ int hist[NB_COUNT], base[NB_COUNT];
  const int i = blockIdx.x * NBIN_THREADS + threadIdx.x;
  if (threadIdx.x < NB_COUNT) hist[threadIdx.x] = 0;
  __syncthreads();
  int bin = -1, rank = 0;
  bool listed = false;  // bitmap rows go to a slice list, not a row list
  // other rows were done by the fused pass; rows_cnt_max > 0: rows that the
  // whole-row kernel takes are left to it
  if (i < m && row_p[i] > tn.long_p &&
      !(rows_cnt_max > 0 && whole_row_path(c_cnt[i], row_span[i], rows_cnt_max, rows_max_words))) {
    const int o = c_cnt[i];
    const long long p = row_p[i];
    bin = num_bin_of(o, p, tn);
    const int2 sp = row_span[i];
    const int lo = sp.x & ~31;  // word aligned (saved bitmaps are indexed from column 0)
    const int span = sp.y + 1 - lo;
    const long long out0 = c_rowptr[i];
    const int flags = SLICE_WHOLE | (bits_kept ? SLICE_BITS_KEPT : 0);
    if (bin == NB_LONG) {
      atomicAdd(&hist[NB_LONG], 1);
      if (o <= tn.slice_cap && span <= tn.slice_cols) {
        push_slice(big, big_count, big_capacity, Slice{out0, i, lo, sp.y + 1, o, flags}, status);
      } else {
        const int* cc = chunk_cnt + (size_t)long_slot[i] * n_chunks;
        const int sflags = flags & SLICE_BITS_KEPT;
        int lo_c = 0, acc = 0;
        long long out = out0;
        for (int c = 0; c < n_chunks; ++c) {
          const int v = cc[c];
          const bool too_many = acc + v > tn.slice_cap;
          const bool too_wide = (c + 1 - lo_c) * CHUNK_COLS > tn.slice_cols;
          if ((too_many || too_wide) && c > lo_c) {
            if (acc)
              push_slice(big, big_count, big_capacity,
                         Slice{out, i, lo_c * CHUNK_COLS, c * CHUNK_COLS, acc, sflags}, status);
            out += acc;
            lo_c = c;
            acc = 0;
          }
          acc += v;
        }
        if (acc)
          push_slice(big, big_count, big_capacity, Slice{out, i, lo_c * CHUNK_COLS, n, acc, sflags},
                     status);
      }
    } else if (bin >= 0 && o > tn.mid_o_min && span <= tn.mid_cols) {
      atomicAdd(&hist[NB_MID], 1);
      push_slice(mid, mid_count, m, Slice{out0, i, lo, sp.y + 1, o, flags}, status);
    } else if (bin >= 0) {
      rank = atomicAdd(&hist[bin], 1);
      listed = true;
    }
  }
  __syncthreads();
  if (threadIdx.x < NB_COUNT && hist[threadIdx.x])
    base[threadIdx.x] = atomicAdd(num_count + threadIdx.x, hist[threadIdx.x]);
  __syncthreads();
  if (listed) num_rows[(size_t)bin * m + base[bin] + rank] = i;
}

// ---------------------------------------------------------------------------
// Numeric pass: hash rows
// ---------------------------------------------------------------------------

template <int LOG2T, int NT, int MODE>
__global__ void __launch_bounds__(NT)
k_num_block(Operands op, const int* __restrict__ rows, int nrows, int r0, int r1,
            const long long* __restrict__ row_p, const long long* __restrict__ c_rowptr,
            int* __restrict__ c_col, float* __restrict__ c_val, unsigned* status) {
  constexpr int T = 1 << LOG2T;
  constexpr int NW = NT / 32;
  using V = typename SlotOf<MODE>::T;
  extern __shared__ __align__(16) unsigned char smem[];
  const int warp = threadIdx.x >> 5;
  V* vals = reinterpret_cast<V*>(smem);
  unsigned* keys = reinterpret_cast<unsigned*>(smem + T * sizeof(V));
  SegScratch* sc = reinterpret_cast<SegScratch*>(smem + T * (sizeof(V) + 4)) + warp;
  for (int r = blockIdx.x; r < nrows; r += gridDim.x) {
    const int i = rows[r];
    if (i < r0 || i >= r1) continue;  // another row range (block-uniform)
    const long long p = row_p[i];
    for (int t = threadIdx.x; t < T; t += NT) { keys[t] = EMPTY_KEY; vals[t] = V(0); }
    __syncthreads();
    const int rs = op.a_rowptr[i], re = op.a_rowptr[i + 1];
    const bool fp64 = MODE == 1 && p > FP64_ROW_PARTIALS;
    const int U = chunk_for(p, NW, 1 << 20);
    if (MODE == 0) {
      NumHashPlain f{keys, reinterpret_cast<float*>(vals), LOG2T, status};
      for (int c0 = warp * U; c0 < p; c0 += NW * U)
        warp_expand_range<true>(op, rs, re, c0, (int)min((long long)c0 + U, p), f, sc);
    } else if (fp64) {
      NumHashF64 f{keys, reinterpret_cast<double*>(vals), LOG2T, status};
      for (int c0 = warp * U; c0 < p; c0 += NW * U)
        warp_expand_range<true>(op, rs, re, c0, (int)min((long long)c0 + U, p), f, sc);
    } else {
      NumHashTwoSum f{keys, reinterpret_cast<float2*>(vals), LOG2T, status};
      for (int c0 = warp * U; c0 < p; c0 += NW * U)
        warp_expand_range<true>(op, rs, re, c0, (int)min((long long)c0 + U, p), f, sc);
    }
    __syncthreads();
    bitonic_sort_kv<T, NT>(keys, vals, threadIdx.x, BlockSync());
    const long long o = c_rowptr[i];
    const int cnt = (int)(c_rowptr[i + 1] - o);
    if (threadIdx.x == 0 &&
        ((cnt < T && keys[cnt] != EMPTY_KEY) || keys[cnt - 1] == EMPTY_KEY))
      atomicOr(status, ST_COUNT_MISMATCH);
    for (int t = threadIdx.x; t < cnt; t += NT) {
      __stcs(c_col + o + t, (int)keys[t]);
      if (MODE == 0) __stcs(c_val + o + t, finalize_value(reinterpret_cast<float*>(vals)[t]));
      else if (fp64) __stcs(c_val + o + t, finalize_value(reinterpret_cast<double*>(vals)[t]));
      else __stcs(c_val + o + t, finalize_value(reinterpret_cast<float2*>(vals)[t]));
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Numeric pass: bitmap slices (long and mid rows), one block per slice
// ---------------------------------------------------------------------------

// Shared memory: per-warp scratch | directory uint2[dir_words] | values[cap]
// | columns[cap] (| sparse mode: l1 bits[dir_words/32 + 1] | touched word
// list[cap]); plain FP32 slices of long rows have no column array: each
// slot's column is stored into C by the product that touches it first.
// The presence bits come from the symbolic pass when it kept them, else from
// a first expansion pass; a block scan turns popcounts into ranks; the value
// pass adds every product into the slot given by its column's rank (a
// counting sort on the column, so the slice comes out in column order); the
// write-out copies the values (and columns) in order.
//
// SPARSE (used for mid rows, at most `cap` outputs over up to 2^18 columns):
// the directory is cleared once per block and kept clean between slices;
// ranks, write-out and cleanup visit only the directory words that became
// non-empty (tracked in l1), so a slice costs O(products + outputs) instead
// of O(span / 32).
//
// Fused mode (row_list != nullptr, SPARSE only): the work items are whole rows
// of the fused pass; the slice spans the row's columns, the output goes to the
// temporary buffer at toff[i], the row's nnz is found here (written to
// c_cnt[i]) and, in compensated mode, rows of at most 4096 products use
// TwoSum pairs instead of FP64.
// Directory walks shared by the rank scan and the column write-out: list
// item t names directory word word_at(t); each warp takes one contiguous run
// of the list (a multiple of 32 items) and walks it 32 items at a time, lane
// l on item base + l, so shared-memory accesses are conflict-free and the
// ranks, hence the output positions, rise with the lane.
template <int NT>
__device__ __forceinline__ int2 warp_dir_run(int nitems) {
  constexpr int NW = NT / 32;
  const int run = ((nitems + NW * 32 - 1) / (NW * 32)) * 32;
  const int b = min((int)(threadIdx.x >> 5) * run, nitems);
  return make_int2(b, min(b + run, nitems));
}

// Ranks of a bitmap directory: dir[w].y = set bits in the listed words before
// w. Returns the total number of set bits (every thread). The ranks are
// visible to the whole block after the caller's next barrier.
template <int NT, class WordAt>
__device__ __forceinline__ long long dir_ranks(uint2* dir, int nitems, WordAt word_at,
                                               long long* scan_shm) {
  const int lane = lane_id();
  const int2 r = warp_dir_run<NT>(nitems);
  int local = 0;
  for (int t = r.x + lane; t < r.y; t += 32) local += __popc(dir[word_at(t)].x);
  local = warp_sum(local);
  long long total;
  long long base = block_excl_scan64(lane == 0 ? local : 0, scan_shm, total);
  base = __shfl_sync(FULL, base, 0);
  for (int t0 = r.x; t0 < r.y; t0 += 32) {
    const int t = t0 + lane;
    const int w = t < r.y ? word_at(t) : 0;
    const int c = t < r.y ? __popc(dir[w].x) : 0;
    const int incl = warp_incl_scan(c);
    if (t < r.y) dir[w].y = (unsigned)(base + incl - c);
    base += __shfl_sync(FULL, incl, 31);
  }
  return total;
}

// dst[0, n) = f(t) for t in [0, n), by the whole block, each warp store
// covering one aligned 128-byte line of dst (streaming stores: C is not
// read again by this pass).
template <int NT, class T, class F>
__device__ __forceinline__ void block_store_aligned(T* __restrict__ dst, int n, F f) {
  const int head = (int)((reinterpret_cast<size_t>(dst) / sizeof(T)) & (128 / sizeof(T) - 1));
  for (int g = threadIdx.x - head; g < n; g += NT)
    if (g >= 0) __stcs(dst + g, f(g));
}

template <int MODE, int NT, bool SPARSE>
__global__ void __launch_bounds__(NT, NT >= 1024 ? 1 : 2)
k_num_long(Operands op, const Slice* __restrict__ slices, int nslices,
           const long long* __restrict__ row_p, int dir_words, int cap,
           int* __restrict__ scratch, int scratch_stride,
           const unsigned* __restrict__ bitmaps, int bitmap_words,
           const int* __restrict__ long_slot,
           int* __restrict__ c_col, float* __restrict__ c_val, unsigned* status,
           const int* __restrict__ row_list, const int* __restrict__ row_count_p,
           const int2* __restrict__ row_span, const long long* __restrict__ toff,
           int* __restrict__ c_cnt, int r0, int r1) {
  constexpr int NW = NT / 32;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ long long scan_shm[33];
  __shared__ int carry_shm;
  const int warp = threadIdx.x >> 5;
  SegScratch* sc = reinterpret_cast<SegScratch*>(smem) + warp;
  uint2* dir = reinterpret_cast<uint2*>(smem + NW * sizeof(SegScratch));
  unsigned char* vbase = smem + NW * sizeof(SegScratch) + (size_t)dir_words * sizeof(uint2);
  int* cols = reinterpret_cast<int*>(vbase + (size_t)cap * (MODE ? 8 : 4));  // column per slot
  const int l1_words = (dir_words + 31) >> 5;
  unsigned* l1 = reinterpret_cast<unsigned*>(cols + cap);
  int* touched = reinterpret_cast<int*>(l1 + l1_words);
  int* seg_start = scratch + (size_t)blockIdx.x * scratch_stride;
  if (SPARSE) {
    for (int t = threadIdx.x; t < dir_words; t += NT) dir[t] = make_uint2(0u, 0u);
    for (int t = threadIdx.x; t < l1_words; t += NT) l1[t] = 0u;
  }
  if (row_list) nslices = *row_count_p;
  for (int s = blockIdx.x; s < nslices; s += gridDim.x) {
    Slice sl;
    if (row_list) {
      const int ri = row_list[s];
      const int2 sp = row_span[ri];
      sl = Slice{toff[ri], ri, sp.x & ~31, sp.y + 1, -1, SLICE_WHOLE | SLICE_FUSED};
    } else {
      sl = slices[s];
    }
    const int i = sl.row;
    if (i < r0 || i >= r1) continue;  // another row range's slice (block-uniform)
    const bool fused = (sl.flags & SLICE_FUSED) != 0;
    const int rs = op.a_rowptr[i], re = op.a_rowptr[i + 1];
    int* roff = seg_start + (re - rs);
    const bool whole = (sl.flags & SLICE_WHOLE) != 0;
    const int nw = (sl.hi - sl.lo + 31) >> 5;
    const int cnt = sl.cnt;
    if (nw > dir_words || cnt > cap || (SPARSE && !whole)) {  // sizing prevents this
      if (threadIdx.x == 0) atomicOr(status, ST_SLICE_OVERFLOW);
      continue;
    }
    const bool have_bits = bitmap_words > 0 && (sl.flags & SLICE_BITS_KEPT);
    if (have_bits) {  // the symbolic pass kept this row's presence bitmap
      const unsigned* src = bitmaps + (size_t)long_slot[i] * bitmap_words + (sl.lo >> 5);
      if (SPARSE) {
        __syncthreads();  // previous slice's cleanup is complete
        for (int t = threadIdx.x; t < nw; t += NT) {
          const unsigned b = __ldg(src + t);
          if (b) {
            dir[t].x = b;
            atomicOr(l1 + (t >> 5), 1u << (t & 31));
          }
        }
      } else {
        for (int t = threadIdx.x; t < nw; t += NT) dir[t] = make_uint2(__ldg(src + t), 0u);
      }
    } else if (!SPARSE) {
      for (int t = threadIdx.x; t < nw; t += NT) dir[t] = make_uint2(0u, 0u);
    }
    // products of the slice: the whole row, or its restriction to [lo, hi)
    int p;
    if (whole) {
      p = (int)row_p[i];
      __syncthreads();
    } else {
      p = block_restrict_row(op, rs, re, sl.lo, sl.hi, seg_start, roff, scan_shm, &carry_shm);
    }
    // pass 1: presence bits (only when the bitmap was not kept)
    if (!have_bits) {
      if (SPARSE) {
        LongBitsTracked f{dir, l1, sl.lo, (unsigned)(sl.hi - sl.lo), status};
        block_walk_row<false>(op, rs, re, true, seg_start, roff, p, f, sc, warp, NW);
      } else {
        LongBits f{dir, sl.lo, (unsigned)(sl.hi - sl.lo), status};
        block_walk_row<false>(op, rs, re, whole, seg_start, roff, p, f, sc, warp, NW);
      }
      __syncthreads();
    }
    // ranks: exclusive scan of popcounts over the directory words
    long long tot;
    int nt = 0;  // sparse: number of touched words
    if (SPARSE) {
      // touched word list, in column order, from l1
      const int nl1 = (nw + 31) >> 5;
      long long l1tot;
      const unsigned myl1 = threadIdx.x < nl1 ? l1[threadIdx.x] : 0u;  // nl1 <= NT (host)
      long long pos = block_excl_scan64(__popc(myl1), scan_shm, l1tot);
      for (unsigned b = myl1; b; b &= b - 1u) {
        if (pos < cap) touched[pos] = threadIdx.x * 32 + __ffs(b) - 1;  // list holds cap words
        ++pos;
      }
      nt = (int)min(l1tot, (long long)cap);  // more than cap touched words: count mismatch below
      __syncthreads();
      tot = dir_ranks<NT>(dir, nt, [&](int t) { return touched[t]; }, scan_shm);
    } else {
      tot = dir_ranks<NT>(dir, nw, [](int t) { return t; }, scan_shm);
    }
    const int ocount = fused ? (int)tot : cnt;
    if ((!fused && tot != cnt) || tot > cap || (SPARSE && nt == cap && ocount < cap)) {  // block-uniform
      if (threadIdx.x == 0) atomicOr(status, ST_COUNT_MISMATCH);
      __syncthreads();
      if (SPARSE) {  // restore the clean directory before the next slice
        for (int t = threadIdx.x; t < nw; t += NT) dir[t] = make_uint2(0u, 0u);
        for (int t = threadIdx.x; t < l1_words; t += NT) l1[t] = 0u;
        __syncthreads();
      }
      continue;
    }
    if (MODE == 0) {
      float* vals = reinterpret_cast<float*>(vbase);
      for (int t = threadIdx.x; t < ocount; t += NT) vals[t] = 0.f;
    } else {
      double* vals = reinterpret_cast<double*>(vbase);  // zero bits: 0.0 and (0.f, 0.f)
      for (int t = threadIdx.x; t < ocount; t += NT) vals[t] = 0.0;
    }
    __syncthreads();
    const bool pair = MODE == 1 && p <= FP64_ROW_PARTIALS;  // compensated FP32 pairs
    // value pass
    if (MODE == 1 && pair) {
      LongValTwoSum f{dir, reinterpret_cast<float2*>(vbase), cols, sl.lo, (unsigned)(sl.hi - sl.lo)};
      block_walk_row<true>(op, rs, re, whole, seg_start, roff, p, f, sc, warp, NW);
    } else if (MODE == 0 && !SPARSE) {
      // each slot's column goes straight to C at its first touch, so the
      // slice needs shared memory for the values only
      RowValCols f{dir, reinterpret_cast<float*>(vbase), c_col + sl.out, sl.lo,
                   (unsigned)(sl.hi - sl.lo)};
      block_walk_row<true>(op, rs, re, whole, seg_start, roff, p, f, sc, warp, NW);
    } else if (MODE == 0) {
      LongValPlain f{dir, reinterpret_cast<float*>(vbase), cols, sl.lo, (unsigned)(sl.hi - sl.lo)};
      block_walk_row<true>(op, rs, re, whole, seg_start, roff, p, f, sc, warp, NW);
    } else {
      LongValF64 f{dir, reinterpret_cast<double*>(vbase), cols, sl.lo, (unsigned)(sl.hi - sl.lo)};
      block_walk_row<true>(op, rs, re, whole, seg_start, roff, p, f, sc, warp, NW);
    }
    __syncthreads();
    // write-out: values and columns are already in output order
    if (fused && threadIdx.x == 0) c_cnt[i] = ocount;
    if (MODE == 0) {
      const float* vals = reinterpret_cast<const float*>(vbase);
      block_store_aligned<NT>(c_val + sl.out, ocount, [&](int t) { return vals[t]; });
    } else if (pair) {
      const float2* vals = reinterpret_cast<const float2*>(vbase);
      block_store_aligned<NT>(c_val + sl.out, ocount, [&](int t) { return finalize_value(vals[t]); });
    } else {
      const double* vals = reinterpret_cast<const double*>(vbase);
      block_store_aligned<NT>(c_val + sl.out, ocount, [&](int t) { return finalize_value(vals[t]); });
    }
    if (MODE != 0 || SPARSE)
      block_store_aligned<NT>(c_col + sl.out, ocount, [&](int t) { return cols[t]; });
    if (SPARSE) {
      // leave the directory clean for the next slice
      for (int t = threadIdx.x; t < nt; t += NT) dir[touched[t]] = make_uint2(0u, 0u);
      for (int t = threadIdx.x; t < l1_words; t += NT) l1[t] = 0u;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Numeric pass: whole long rows, one block per row (plain FP32)
// ---------------------------------------------------------------------------

// Work order of the long rows: grouped by floor(log2 P_i), heaviest group
// first, so that on the dynamic row queue of k_num_rows the longest rows
// start first and the short ones fill in at the end (longest-processing-time
// first, to a factor of two). Only the rows of [r0, r1) with more than
// cnt_min outputs that whole_row_path(cnt_max) accepts are listed.
constexpr int LPT_GROUPS = 32;

__device__ __forceinline__ int lpt_group(long long p) { return 63 - __clzll(p > 0 ? p : 1); }

__global__ void __launch_bounds__(256)
k_lpt_hist(const int* __restrict__ rows, int nrows, int r0, int r1,
           const long long* __restrict__ row_p, const int* __restrict__ c_cnt,
           const int2* __restrict__ row_span, int cnt_min, int cnt_max, int max_words,
           int* __restrict__ hist) {
  __shared__ int h[LPT_GROUPS];
  if (threadIdx.x < LPT_GROUPS) h[threadIdx.x] = 0;
  __syncthreads();
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nrows; r += gridDim.x * blockDim.x) {
    const int i = rows[r];
    const int o = c_cnt[i];
    if (i >= r0 && i < r1 && o > cnt_min && whole_row_path(o, row_span[i], cnt_max, max_words))
      atomicAdd(&h[min(lpt_group(row_p[i]), LPT_GROUPS - 1)], 1);
  }
  __syncthreads();
  if (threadIdx.x < LPT_GROUPS && h[threadIdx.x]) atomicAdd(hist + threadIdx.x, h[threadIdx.x]);
}

// hist: rows per group (from k_lpt_hist); cursor: zeroed per group counters;
// order: the listed rows, heaviest group first; *nlisted: their count.
__global__ void __launch_bounds__(256)
k_lpt_scatter(const int* __restrict__ rows, int nrows, int r0, int r1,
              const long long* __restrict__ row_p, const int* __restrict__ c_cnt,
              const int2* __restrict__ row_span, int cnt_min, int cnt_max, int max_words,
              const int* __restrict__ hist, int* __restrict__ cursor, int* __restrict__ order,
              int* __restrict__ nlisted) {
  __shared__ int base[LPT_GROUPS];
  if (threadIdx.x == 0) {
    int run = 0;
    for (int g = LPT_GROUPS - 1; g >= 0; --g) {
      base[g] = run;
      run += hist[g];
    }
    if (blockIdx.x == 0) *nlisted = run;
  }
  __syncthreads();
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nrows; r += gridDim.x * blockDim.x) {
    const int i = rows[r];
    const int o = c_cnt[i];
    if (i >= r0 && i < r1 && o > cnt_min && whole_row_path(o, row_span[i], cnt_max, max_words)) {
      const int g = min(lpt_group(row_p[i]), LPT_GROUPS - 1);
      order[base[g] + atomicAdd(cursor + g, 1)] = i;
    }
  }
}

// Value functors of k_num_rows: the product lands in the output slot given by
// its column's rank in the row's directory, either as a reduction into C in
// global memory (performed in L2; nothing is returned to the SM) or as a
// shared-memory atomic add.
__device__ __forceinline__ void red_add_f32(float* p, float v) {
  asm volatile("red.global.add.f32 [%0], %1;" ::"l"(p), "f"(v) : "memory");
}

struct RowValRed {
  const uint2* dir;
  float* out;  // C values of the row
  int lo;
  unsigned width;
  __device__ __forceinline__ void operator()(int col, float a, float b) {
    if ((unsigned)(col - lo) < width) red_add_f32(out + long_slot(dir, lo, col), __fmul_rn(a, b));
  }
};

struct RowValSmem {
  const uint2* dir;
  float* vals;  // shared memory, one slot per output
  int lo;
  unsigned width;
  __device__ __forceinline__ void operator()(int col, float a, float b) {
    if ((unsigned)(col - lo) < width) atomicAdd(vals + long_slot(dir, lo, col), __fmul_rn(a, b));
  }
};

// One block per long row, rows taken from a queue in LPT order. The row's
// presence bitmap, kept by the symbolic pass, is loaded for the whole column
// span into a shared-memory directory (bits + rank of the first column of
// every 32-column word); every product then adds into its final position
// out0 + rank(column), so the row is produced in column order with no
// column slicing and no sort. RED: values accumulate in C itself (zeroed
// first; the row's value range stays in L2 while the block works on it) and
// the columns are written from the directory; otherwise values accumulate in
// shared memory (rows of at most `cap` outputs) and are copied out at the
// end, and each column is stored into C by the product that first touches
// its slot. Shared memory: per-warp scratch | directory uint2[dir_words] |
// (not RED) values float[cap].
template <int NT, bool RED>
__global__ void __launch_bounds__(NT, NT >= 1024 ? 1 : 2)
k_num_rows(Operands op, const int* __restrict__ order, const int* __restrict__ nrows_p,
           int* __restrict__ queue, const long long* __restrict__ row_p,
           const long long* __restrict__ c_rowptr, const int2* __restrict__ row_span,
           const unsigned* __restrict__ bitmaps, int bitmap_words,
           const int* __restrict__ long_slot_of, int dir_words, int cap,
           int* __restrict__ c_col, float* __restrict__ c_val, unsigned* status) {
  constexpr int NW = NT / 32;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ long long scan_shm[33];
  __shared__ int s_item;
  const int warp = threadIdx.x >> 5;
  SegScratch* sc = reinterpret_cast<SegScratch*>(smem) + warp;
  uint2* dir = reinterpret_cast<uint2*>(smem + NW * sizeof(SegScratch));
  float* vals = reinterpret_cast<float*>(dir + dir_words);
  const int nrows = *nrows_p;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(queue, 1);
    __syncthreads();
    const int r = s_item;
    if (r >= nrows) break;
    const int i = order[r];
    const long long out0 = c_rowptr[i];
    const int cnt = (int)(c_rowptr[i + 1] - out0);
    const int2 sp = row_span[i];
    const int lo = sp.x & ~31;  // word aligned: the kept bitmaps are indexed from column 0
    const int nw = (sp.y + 1 - lo + 31) >> 5;
    if (nw > dir_words || (!RED && cnt > cap)) {  // the host's sizing prevents this
      if (threadIdx.x == 0) atomicOr(status, ST_SLICE_OVERFLOW);
      __syncthreads();
      continue;
    }
    const unsigned* src = bitmaps + (size_t)long_slot_of[i] * bitmap_words + (lo >> 5);
    for (int t = threadIdx.x; t < nw; t += NT) dir[t] = make_uint2(__ldg(src + t), 0u);
    __syncthreads();
    const long long tot = dir_ranks<NT>(dir, nw, [](int t) { return t; }, scan_shm);
    if (tot != cnt) {  // block-uniform
      if (threadIdx.x == 0) atomicOr(status, ST_COUNT_MISMATCH);
      __syncthreads();
      continue;
    }
    if (RED) {
      for (int t = threadIdx.x; t < cnt; t += NT) c_val[out0 + t] = 0.f;
    } else {
      for (int t = threadIdx.x; t < cnt; t += NT) vals[t] = 0.f;
    }
    __syncthreads();  // ranks and zeroed values visible to the whole block
    const int rs = op.a_rowptr[i], re = op.a_rowptr[i + 1];
    const int p = (int)row_p[i];
    const unsigned width = (unsigned)(sp.y + 1 - lo);
    if (RED) {
      RowValRed f{dir, c_val + out0, lo, width};
      block_walk_row<true>(op, rs, re, true, nullptr, nullptr, p, f, sc, warp, NW);
    } else {
      RowValCols f{dir, vals, c_col + out0, lo, width};
      block_walk_row<true>(op, rs, re, true, nullptr, nullptr, p, f, sc, warp, NW);
    }
    __syncthreads();
    if (RED) {
      // columns in rank order from the directory, one word per thread at a time
      for (int w = threadIdx.x; w < nw; w += NT) {
        const uint2 d = dir[w];
        unsigned b = d.x;
        int pos = (int)d.y;
        while (b) {
          const int bit = __ffs(b) - 1;
          b &= b - 1u;
          __stcs(c_col + out0 + pos, lo + 32 * w + bit);
          ++pos;
        }
      }
    } else {
      // the columns were stored at first touch; values in output order
      block_store_aligned<NT>(c_val + out0, cnt, [&](int t) { return vals[t]; });
    }
    __syncthreads();
  }
}

}  // namespace sg

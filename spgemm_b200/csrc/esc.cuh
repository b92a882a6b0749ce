// Fused pass by sorting: expand, sort, compress (ESC), one block per row.
//
// The reference materialises every partial product of a row of C in its
// bucket (src/mm.cu:288-312) and merges the bucket with a dense accumulator
// (src/mm.cu:366-404). Rows of at most 4096 products whose column bound is
// too large for a warp's hash table and whose columns spread over a wide
// span (R-MAT rows of 2K-4K products) degrade both of this engine's other
// fused accumulators: a block hash table sized for the bound, and a bitmap
// over the span, which costs span/32 words per row for a few thousand
// products. Measured on a B200, sorting costs several hash inserts per
// product (gather, two or three radix passes, compression), so it serves
// those rows only; rows a warp's table can hold stay hashed. Here the row's partials are written straight to shared memory at
// their position in the row's flattened product sequence, sorted by column
// with a stable LSD radix sort, and runs of equal columns are summed in that
// stable order. No floating-point atomics are used, so the result is
// deterministic: every run is summed in product order (entries of A in
// order, each B row in order), in plain and in compensated mode.
#pragma once

#include "pipeline.cuh"

namespace sg {

constexpr int ESC_KPT = 8;             // products per thread: capacity NT * ESC_KPT
constexpr int ESC_RADIX_BITS = 9;      // digit bits per radix pass (at most)
constexpr int ESC_BUCKETS = 1 << ESC_RADIX_BITS;

// Partial product as stored for the sort: plain FP32 value, or (rounded
// product, its exact rounding error) for the compensated merge.
template <int MODE> struct EscVal { using T = float; };
template <> struct EscVal<1> { using T = float2; };

template <int MODE>
__device__ __forceinline__ typename EscVal<MODE>::T esc_value(float a, float b);
template <>
__device__ __forceinline__ float esc_value<0>(float a, float b) { return __fmul_rn(a, b); }
template <>
__device__ __forceinline__ float2 esc_value<1>(float a, float b) {
  const float p = __fmul_rn(a, b);
  return make_float2(p, __fmaf_rn(a, b, -p));  // TwoProduct: a*b == p + e exactly
}

// Products [f0, f1) of a row's flattened product sequence, one warp. Entry j
// of the row holds positions aoff[j] .. aoff[j] + nnz(B(k_j,:)) - 1, so the
// entries of a 32-entry batch cover one contiguous position range; the
// product at position f is written to keys[f] (its column minus lo) and
// vals[f]. Products are walked 32 at a time with the owner of each position
// found from the OR of segment-start bits (as in run_segments), two windows
// in flight.
template <int MODE>
__device__ __forceinline__ void warp_gather_range(const Operands& op, int rs, int re, int f0,
                                                  int f1, int lo, unsigned* __restrict__ keys,
                                                  typename EscVal<MODE>::T* __restrict__ vals,
                                                  SegScratch* sc) {
  const int lane = lane_id();
  int l = rs, h = re;  // first entry whose offset is > f0
  while (l < h) {
    const int mid = (l + h) >> 1;
    if (__ldg(op.aoff + mid) <= f0) l = mid + 1; else h = mid;
  }
  for (int base = max(l - 1, rs); base < re; base += 32) {
    const int j = base + lane;
    int bstart = 0, len = 0, pos0 = 0;
    float a = 0.f;
    bool past = true;
    if (j < re) {
      const int off = __ldg(op.aoff + j);
      past = off >= f1;
      if (!past) {
        const int k = __ldg(op.a_col + j);
        const int bs = __ldg(op.b_rowptr + k);
        const int bl = __ldg(op.b_rowptr + k + 1) - bs;
        const int s0 = max(off, f0), s1 = min(off + bl, f1);
        if (s1 > s0) {
          a = __ldg(op.a_val + j);
          bstart = bs + (s0 - off);
          len = s1 - s0;
          pos0 = s0;
        }
      }
    }
    const bool done = __any_sync(FULL, past);
    const unsigned ne = __ballot_sync(FULL, len > 0);
    if (ne) {
      const int start = __shfl_sync(FULL, pos0, __ffs(ne) - 1);
      compact_segments(bstart, len, a, sc);
      const int incl = warp_incl_scan(len);
      const int total = __shfl_sync(FULL, incl, 31);
      const int s = incl - len;
      int nbefore = 0;
      for (int wb = 0; wb < total; wb += 64) {
        int col[2], dst[2];
        float bv[2], oa[2];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          const int w = wb + 32 * u;
          dst[u] = -1;
          if (w < total) {  // warp-uniform
            const unsigned bit = (len > 0 && s >= w && s < w + 32) ? (1u << (s - w)) : 0u;
            const unsigned starts = __reduce_or_sync(FULL, bit);
            const int owner = nbefore + __popc(starts & (FULL >> (31 - lane))) - 1;
            nbefore += __popc(starts);
            const int ob = __shfl_sync(FULL, bstart, owner);
            const int os = __shfl_sync(FULL, s, owner);
            oa[u] = __shfl_sync(FULL, a, owner);
            const int fp = w + lane;
            if (fp < total) {
              const int pos = ob + (fp - os);
              col[u] = __ldg(op.b_col + pos);
              bv[u] = __ldg(op.b_val + pos);
              dst[u] = start + fp;
            }
          }
        }
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          if (dst[u] >= 0) {
            keys[dst[u]] = (unsigned)(col[u] - lo);
            vals[dst[u]] = esc_value<MODE>(oa[u], bv[u]);
          }
        }
      }
    }
    if (done) break;
  }
}

// Stable LSD radix sort of (keys, vals)[0, n) by the low `bits` bits of the
// key, one block of NT threads, n <= NT * ESC_KPT. Warp w owns groups
// [w * gpw, (w + 1) * gpw) of 32 consecutive positions (gpw = groups per
// warp); positions n .. NW * gpw * 32 - 1 must hold EMPTY_KEY (every digit
// maximal, so they stay behind the row's keys). Per pass: each warp ranks
// its keys by digit (match.any peers + per-warp counters, in position order),
// one block scan turns the per-(digit, warp) counts into offsets, and every
// key is scattered from registers to offset + rank. The sorted sequence ends
// in buffer 0 or 1 (returned).
template <int NT, class V>
__device__ __forceinline__ int block_radix_sort(unsigned* __restrict__ k0, V* __restrict__ v0,
                                                unsigned* __restrict__ k1, V* __restrict__ v1,
                                                int n, int bits, int* __restrict__ hist,
                                                long long* scan_shm) {
  constexpr int NW = NT / 32;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int groups = (n + 31) >> 5;
  const int gpw = (groups + NW - 1) / NW;  // <= ESC_KPT
  const int npass = (bits + ESC_RADIX_BITS - 1) / ESC_RADIX_BITS;
  const int db = (bits + npass - 1) / npass;
  const unsigned dmask = (1u << db) - 1u;
  const int nb = 1 << db;
  const unsigned lt = (1u << lane) - 1u;
  int* wh = hist + warp * ESC_BUCKETS;
  unsigned* sk = k0;
  V* sv = v0;
  unsigned* dk = k1;
  V* dv = v1;
  for (int pass = 0; pass < npass; ++pass) {
    const int sh = pass * db;
    for (int t = lane; t < nb; t += 32) wh[t] = 0;
    __syncwarp();
    unsigned k[ESC_KPT];
    V v[ESC_KPT];
    int rk[ESC_KPT];
#pragma unroll
    for (int g = 0; g < ESC_KPT; ++g) {
      if (g < gpw) {  // block-uniform
        const int p = (warp * gpw + g) * 32 + lane;
        k[g] = sk[p];
        v[g] = sv[p];
        const unsigned d = (k[g] >> sh) & dmask;
        const unsigned peers = __match_any_sync(FULL, d);
        const int before = wh[d];
        rk[g] = before + __popc(peers & lt);
        __syncwarp();
        if ((peers & lt) == 0) wh[d] = before + __popc(peers);  // lowest peer
        __syncwarp();
      }
    }
    __syncthreads();
    // exclusive scan of the counts in (digit, warp) order
    const int E = nb * NW;
    const int ept = (E + NT - 1) / NT;
    const int e0 = threadIdx.x * ept;
    int sum = 0;
    for (int q = 0; q < ept; ++q) {
      const int e = e0 + q;
      if (e < E) sum += hist[(e % NW) * ESC_BUCKETS + e / NW];
    }
    long long tot;
    int run = (int)block_excl_scan64(sum, scan_shm, tot);  // ends with a barrier
    for (int q = 0; q < ept; ++q) {
      const int e = e0 + q;
      if (e < E) {
        int* hp = hist + (e % NW) * ESC_BUCKETS + e / NW;
        const int c = *hp;
        *hp = run;
        run += c;
      }
    }
    __syncthreads();
#pragma unroll
    for (int g = 0; g < ESC_KPT; ++g) {
      if (g < gpw) {
        const int pos = wh[(k[g] >> sh) & dmask] + rk[g];
        dk[pos] = k[g];
        dv[pos] = v[g];
      }
    }
    __syncthreads();
    unsigned* tk = sk; sk = dk; dk = tk;
    V* tv = sv; sv = dv; dv = tv;
  }
  return npass & 1;
}

__device__ __forceinline__ float esc_run_sum(const float* v, const unsigned* k, int t, int n) {
  const unsigned key = k[t];
  float s = v[t];
  for (int u = t + 1; u < n && k[u] == key; ++u) s = __fadd_rn(s, v[u]);
  return s;
}

// Compensated run sum (Dot2): TwoSum of the rounded products, their rounding
// errors and the TwoSum errors collected in a second word.
__device__ __forceinline__ float esc_run_sum(const float2* v, const unsigned* k, int t, int n) {
  const unsigned key = k[t];
  float s = v[t].x, c = v[t].y;
  for (int u = t + 1; u < n && k[u] == key; ++u) {
    const float p = v[u].x;
    const float ns = __fadd_rn(s, p);
    c = __fadd_rn(c, __fadd_rn(two_sum_err(s, p, ns), v[u].y));
    s = ns;
  }
  return __fadd_rn(s, c);
}

// Compression of the sorted (keys, vals)[0, p) into one output per run of
// equal keys (the run's key and its sum, summed in order by the run's first
// thread), in key order. Warp w takes its groups [w * gpw, (w + 1) * gpw)
// of 32 positions; the outputs before them come from the per-warp run
// counts (one barrier). Returns the number of outputs.
template <int NT, class V>
__device__ __forceinline__ int block_compress(const unsigned* __restrict__ ks,
                                              const V* __restrict__ vs, int p, int gpw, int lo,
                                              int* __restrict__ out_col, float* __restrict__ out_val,
                                              int* warp_runs) {
  constexpr int NW = NT / 32;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  unsigned hm[ESC_KPT];
  int mine = 0;
#pragma unroll
  for (int g = 0; g < ESC_KPT; ++g) {
    hm[g] = 0u;
    if (g < gpw) {  // block-uniform
      const int t = (warp * gpw + g) * 32 + lane;
      hm[g] = __ballot_sync(FULL, t < p && (t == 0 || ks[t - 1] != ks[t]));
      mine += __popc(hm[g]);
    }
  }
  if (lane == 0) warp_runs[warp] = mine;
  __syncthreads();
  int run = 0, total = 0;
#pragma unroll
  for (int w = 0; w < NW; ++w) {
    const int c = warp_runs[w];
    run += w < warp ? c : 0;
    total += c;
  }
#pragma unroll
  for (int g = 0; g < ESC_KPT; ++g) {
    if (g < gpw) {
      const int t = (warp * gpw + g) * 32 + lane;
      if ((hm[g] >> lane) & 1u) {
        const int o = run + __popc(hm[g] & lt);
        out_col[o] = lo + (int)ks[t];
        out_val[o] = esc_run_sum(vs, ks, t, p);
      }
      run += __popc(hm[g]);
    }
  }
  return total;
}

// Rows of P_i <= NT * ESC_KPT products from the bin list, one block per row:
// gather, radix sort of the column offsets (as many bits as the row's span
// needs), compression of equal columns, sorted row written to the temporary
// buffer at toff[i] with its length in c_cnt[i].
//
// Shared memory: vals[2][CAP] | keys[2][CAP] | hist[NW][ESC_BUCKETS] |
// SegScratch[NW].
template <int NT, int MODE>
__global__ void __launch_bounds__(NT, NT <= 128 ? 8 : (NT <= 256 ? 4 : (MODE ? 1 : 2)))
k_fused_esc(Operands op, const int* __restrict__ rows, const int* __restrict__ nrows_p,
            const long long* __restrict__ row_p, const long long* __restrict__ toff,
            const int2* __restrict__ row_span, int* __restrict__ c_cnt,
            int* __restrict__ t_col, float* __restrict__ t_val, unsigned* status) {
  constexpr int NW = NT / 32;
  constexpr int CAP = NT * ESC_KPT;
  using V = typename EscVal<MODE>::T;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ long long scan_shm[33];
  __shared__ int warp_runs[NW];
  const int warp = threadIdx.x >> 5;
  V* v0 = reinterpret_cast<V*>(smem);
  V* v1 = v0 + CAP;
  unsigned* k0 = reinterpret_cast<unsigned*>(v1 + CAP);
  unsigned* k1 = k0 + CAP;
  int* hist = reinterpret_cast<int*>(k1 + CAP);
  SegScratch* sc = reinterpret_cast<SegScratch*>(hist + NW * ESC_BUCKETS) + warp;
  const int nrows = *nrows_p;
  for (int r = blockIdx.x; r < nrows; r += gridDim.x) {
    const int i = rows[r];
    const long long p64 = row_p[i];
    if (p64 > CAP || p64 <= 0) {  // the binning prevents this (block-uniform)
      if (threadIdx.x == 0) {
        if (p64 > CAP) atomicOr(status, ST_SLICE_OVERFLOW);
        c_cnt[i] = 0;
      }
      continue;
    }
    const int p = (int)p64;
    const int2 sp = row_span[i];
    const int lo = sp.x;
    const unsigned width = (unsigned)(sp.y - sp.x);  // largest key
    const int bits = width ? 32 - __clz(width) : 1;
    const int rs = op.a_rowptr[i], re = op.a_rowptr[i + 1];
    const int U = chunk_for(p, NW, CAP);
    for (int f = warp * U; f < p; f += NW * U)
      warp_gather_range<MODE>(op, rs, re, f, min(f + U, p), lo, k0, v0, sc);
    const int gpw = (((p + 31) >> 5) + NW - 1) / NW;
    for (int t = p + threadIdx.x; t < NW * gpw * 32; t += NT) k0[t] = EMPTY_KEY;
    __syncthreads();
    const int which = block_radix_sort<NT>(k0, v0, k1, v1, p, bits, hist, scan_shm);
    const unsigned* ks = which ? k1 : k0;
    const V* vs = which ? v1 : v0;
    const long long base = toff[i];
    const int total = block_compress<NT>(ks, vs, p, gpw, lo, t_col + base, t_val + base,
                                         warp_runs);
    if (threadIdx.x == 0) c_cnt[i] = total;
    __syncthreads();  // the buffers and run counts are reused by the block's next row
  }
}

// Dynamic shared memory of k_fused_esc<NT, MODE>.
template <int NT, int MODE>
constexpr size_t esc_smem_bytes() {
  return (size_t)NT * ESC_KPT * 2 * (sizeof(typename EscVal<MODE>::T) + sizeof(unsigned)) +
         (size_t)(NT / 32) * ESC_BUCKETS * sizeof(int) + (size_t)(NT / 32) * sizeof(SegScratch);
}

}  // namespace sg

// Device conversion of triplets in any order to compressed form (CSR over
// rows or CSC over columns), replacing the host qsort the reference's
// protocol puts before cudaCOO2CM (src/coo.cpp:73-79, src/main.cu:27-30).
//
// Counting sort by the major index (histogram, scan, scatter), then a sort of
// each major index's segment by (minor index, input position): 64-bit keys
// minor << 32 | position, unique, so the result is deterministic and entries
// with equal indices keep their input order. Segments of up to 1024 entries
// are sorted by one warp in shared memory, up to 8192 by one block, longer
// ones by one block as sorted 8192-entry runs merged pairwise in global
// memory (merge-path partitions). Values are gathered from the input by
// position at the end.
#include <cuda_runtime.h>

#include "engine.h"

namespace sg {
namespace {

constexpr int CS_WARP_MAX = 1024;   // entries a warp sorts in shared memory
constexpr int CS_BLOCK_MAX = 8192;  // entries a block sorts in shared memory
constexpr int CS_THREADS = 1024;
constexpr unsigned long long CS_PAD = ~0ull;

struct CsCounters {
  unsigned flags;  // bit 0: an index outside its dimension
  int n_mid;       // segments of (CS_WARP_MAX, CS_BLOCK_MAX] entries
  int n_big;       // segments of more than CS_BLOCK_MAX entries
  long long total;
};

__global__ void k_cs_hist(const triplet* __restrict__ t, int nnz, int row_major, int n_major,
                          int n_minor, int* __restrict__ cnt, CsCounters* cc) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += gridDim.x * blockDim.x) {
    const triplet x = t[e];
    const int major = row_major ? x.ridx : x.cidx;
    const int minor = row_major ? x.cidx : x.ridx;
    if ((unsigned)major >= (unsigned)n_major || (unsigned)minor >= (unsigned)n_minor) {
      atomicOr(&cc->flags, 1u);
      continue;
    }
    atomicAdd(cnt + major, 1);
  }
}

__global__ void k_cs_scatter(const triplet* __restrict__ t, int nnz, int row_major, int n_major,
                             int n_minor, int* __restrict__ cursor,
                             unsigned long long* __restrict__ keys) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += gridDim.x * blockDim.x) {
    const triplet x = t[e];
    const int major = row_major ? x.ridx : x.cidx;
    const int minor = row_major ? x.cidx : x.ridx;
    if ((unsigned)major >= (unsigned)n_major || (unsigned)minor >= (unsigned)n_minor) continue;
    const int pos = atomicAdd(cursor + major, 1);
    keys[pos] = ((unsigned long long)(unsigned)minor << 32) | (unsigned)e;
  }
}

// In-place bitonic sort of n (a power of two) keys by `nthreads` threads.
template <class Sync>
__device__ __forceinline__ void bitonic64(unsigned long long* k, int n, int tid, int nthreads,
                                          Sync sync) {
  for (int size = 2; size <= n; size <<= 1) {
    for (int j = size >> 1; j > 0; j >>= 1) {
      for (int t = tid; t < (n >> 1); t += nthreads) {
        const int lo = ((t & ~(j - 1)) << 1) | (t & (j - 1));
        const int hi = lo + j;
        const bool up = (lo & size) == 0;
        const unsigned long long a = k[lo], b = k[hi];
        if ((a > b) == up) {
          k[lo] = b;
          k[hi] = a;
        }
      }
      sync();
    }
  }
}

struct CsWarpSync {
  __device__ void operator()() const { __syncwarp(); }
};
struct CsBlockSync {
  __device__ void operator()() const { __syncthreads(); }
};

// One warp per segment of 2..CS_WARP_MAX entries; longer segments are listed
// for the block kernels.
constexpr int CS_WARPS = 4;  // warps per block of the warp kernel (32 KB of keys)

__global__ void __launch_bounds__(CS_WARPS * 32)
k_cs_sort_warp(const int* __restrict__ ptr, int n_major, unsigned long long* __restrict__ keys,
               int* __restrict__ mid, int* __restrict__ big, CsCounters* cc) {
  __shared__ unsigned long long buf[CS_WARPS][CS_WARP_MAX];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  unsigned long long* k = buf[warp];
  for (int s = blockIdx.x * CS_WARPS + warp; s < n_major; s += gridDim.x * CS_WARPS) {
    const int b = ptr[s], len = ptr[s + 1] - b;
    if (len <= 1) continue;
    if (len > CS_WARP_MAX) {
      if (lane == 0) {
        if (len > CS_BLOCK_MAX) big[atomicAdd(&cc->n_big, 1)] = s;
        else mid[atomicAdd(&cc->n_mid, 1)] = s;
      }
      continue;
    }
    int n2 = 2;
    while (n2 < len) n2 <<= 1;
    for (int t = lane; t < n2; t += 32) k[t] = t < len ? keys[b + t] : CS_PAD;
    __syncwarp();
    bitonic64(k, n2, lane, 32, CsWarpSync());
    for (int t = lane; t < len; t += 32) keys[b + t] = k[t];
    __syncwarp();
  }
}

// One block per segment of (CS_WARP_MAX, CS_BLOCK_MAX] entries.
__global__ void __launch_bounds__(CS_THREADS)
k_cs_sort_block(const int* __restrict__ ptr, const int* __restrict__ list, const CsCounters* cc,
                unsigned long long* __restrict__ keys) {
  extern __shared__ unsigned long long sk[];
  const int count = cc->n_mid;
  for (int q = blockIdx.x; q < count; q += gridDim.x) {
    const int s = list[q];
    const int b = ptr[s], len = ptr[s + 1] - b;
    int n2 = 2;
    while (n2 < len) n2 <<= 1;
    for (int t = threadIdx.x; t < n2; t += CS_THREADS) sk[t] = t < len ? keys[b + t] : CS_PAD;
    __syncthreads();
    bitonic64(sk, n2, threadIdx.x, CS_THREADS, CsBlockSync());
    for (int t = threadIdx.x; t < len; t += CS_THREADS) keys[b + t] = sk[t];
    __syncthreads();
  }
}

// Merge-path split: the number of entries taken from `a` among the first
// `diag` outputs of merging a[0..na) and b[0..nb).
__device__ __forceinline__ int merge_split(const unsigned long long* a, int na,
                                           const unsigned long long* b, int nb, int diag) {
  int lo = diag > nb ? diag - nb : 0, hi = diag < na ? diag : na;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (a[mid] < b[diag - 1 - mid]) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// One block per segment of more than CS_BLOCK_MAX entries: sorted runs of
// CS_BLOCK_MAX in shared memory, then pairwise merges between the segment
// and its scratch copy; the result ends in `keys`.
__global__ void __launch_bounds__(CS_THREADS)
k_cs_sort_big(const int* __restrict__ ptr, const int* __restrict__ list, const CsCounters* cc,
              unsigned long long* __restrict__ keys, unsigned long long* __restrict__ tmp) {
  extern __shared__ unsigned long long sk[];
  const int count = cc->n_big;
  for (int q = blockIdx.x; q < count; q += gridDim.x) {
    const int s = list[q];
    const int b = ptr[s], len = ptr[s + 1] - b;
    unsigned long long* src = keys + b;
    unsigned long long* dst = tmp + b;
    for (int r0 = 0; r0 < len; r0 += CS_BLOCK_MAX) {
      const int rl = min(CS_BLOCK_MAX, len - r0);
      for (int t = threadIdx.x; t < CS_BLOCK_MAX; t += CS_THREADS)
        sk[t] = t < rl ? src[r0 + t] : CS_PAD;
      __syncthreads();
      bitonic64(sk, CS_BLOCK_MAX, threadIdx.x, CS_THREADS, CsBlockSync());
      for (int t = threadIdx.x; t < rl; t += CS_THREADS) src[r0 + t] = sk[t];
      __syncthreads();
    }
    for (long long w = CS_BLOCK_MAX; w < len; w <<= 1) {
      for (long long p0 = 0; p0 < len; p0 += 2 * w) {
        const int na = (int)min(w, (long long)len - p0);
        const int nb = (int)max(0ll, min(w, (long long)len - p0 - w));
        const unsigned long long* a = src + p0;
        const unsigned long long* bb = src + p0 + na;
        const int tot = na + nb;
        const int per = (tot + CS_THREADS - 1) / CS_THREADS;
        const int d0 = min(threadIdx.x * per, tot), d1 = min(d0 + per, tot);
        int ia = merge_split(a, na, bb, nb, d0);
        int ib = d0 - ia;
        for (int o = d0; o < d1; ++o) {
          const bool take_a = ib >= nb || (ia < na && a[ia] < bb[ib]);
          dst[p0 + o] = take_a ? a[ia++] : bb[ib++];
        }
      }
      __syncthreads();
      unsigned long long* x = src;
      src = dst;
      dst = x;
    }
    if (src != keys + b)
      for (int t = threadIdx.x; t < len; t += CS_THREADS) keys[b + t] = src[t];
    __syncthreads();
  }
}

// Entries placed by the scatter (cc->total: indices out of range are left
// out) to the output: minor index from the key, value from the input entry.
__global__ void k_cs_write(const unsigned long long* __restrict__ keys, const CsCounters* cc,
                           int nnz, const triplet* __restrict__ t, int* __restrict__ idx,
                           float* __restrict__ val) {
  const long long placed = cc->total;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < placed;
       p += (long long)gridDim.x * blockDim.x) {
    const unsigned long long k = keys[p];
    const unsigned e = (unsigned)(k & 0xffffffffu);
    idx[p] = (int)(k >> 32);
    val[p] = e < (unsigned)nnz ? t[e].val : 0.f;
  }
}

int grid_for(long long work, int per_block, int cap) {
  long long g = (work + per_block - 1) / per_block;
  return (int)(g < 1 ? 1 : (g > cap ? cap : g));
}

}  // namespace

cudaError_t coo_compress(const triplet* t, int nnz, bool row_major, int n_major, int n_minor,
                         int* ptr, int* idx, float* val, DevBuf& scratch, DevBuf& scan_tmp,
                         unsigned* flags_host, cudaStream_t s) {
  const size_t cnt_bytes = sizeof(int) * ((size_t)n_major + 1);
  const size_t key_bytes = sizeof(unsigned long long) * (size_t)(nnz > 0 ? nnz : 1);
  const size_t list_bytes = sizeof(int) * ((size_t)n_major + 1);
  size_t off_cc = 0, off_cnt = 256, off_keys = off_cnt + ((cnt_bytes + 255) & ~size_t(255));
  size_t off_tmp = off_keys + ((key_bytes + 255) & ~size_t(255));
  size_t off_mid = off_tmp + ((key_bytes + 255) & ~size_t(255));
  size_t off_big = off_mid + ((list_bytes + 255) & ~size_t(255));
  const size_t total = off_big + ((list_bytes + 255) & ~size_t(255));
  cudaError_t e = scratch.ensure(total);
  if (e != cudaSuccess) return e;
  unsigned char* base = scratch.as<unsigned char>();
  CsCounters* cc = reinterpret_cast<CsCounters*>(base + off_cc);
  int* cnt = reinterpret_cast<int*>(base + off_cnt);
  unsigned long long* keys = reinterpret_cast<unsigned long long*>(base + off_keys);
  unsigned long long* tmp = reinterpret_cast<unsigned long long*>(base + off_tmp);
  int* mid = reinterpret_cast<int*>(base + off_mid);
  int* big = reinterpret_cast<int*>(base + off_big);

  if ((e = cudaMemsetAsync(cc, 0, sizeof(CsCounters), s)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(cnt, 0, cnt_bytes, s)) != cudaSuccess) return e;
  if (nnz > 0) k_cs_hist<<<grid_for(nnz, 256, 4096), 256, 0, s>>>(t, nnz, row_major ? 1 : 0,
                                                                   n_major, n_minor, cnt, cc);
  if ((e = scan_counts_to_ptr32(cnt, n_major, ptr, scan_tmp, &cc->total, s)) != cudaSuccess)
    return e;
  if (nnz > 0) {
    // the counts are free again: reuse them as the scatter cursors
    if ((e = cudaMemcpyAsync(cnt, ptr, sizeof(int) * (size_t)n_major, cudaMemcpyDeviceToDevice, s)) !=
        cudaSuccess)
      return e;
    k_cs_scatter<<<grid_for(nnz, 256, 4096), 256, 0, s>>>(t, nnz, row_major ? 1 : 0, n_major,
                                                          n_minor, cnt, keys);
    k_cs_sort_warp<<<grid_for(n_major, CS_WARPS, 8192), CS_WARPS * 32, 0, s>>>(ptr, n_major, keys,
                                                                              mid, big, cc);
    const size_t smem = sizeof(unsigned long long) * CS_BLOCK_MAX;
    if ((e = cudaFuncSetAttribute(k_cs_sort_block, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem)) != cudaSuccess)
      return e;
    if ((e = cudaFuncSetAttribute(k_cs_sort_big, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem)) != cudaSuccess)
      return e;
    k_cs_sort_block<<<296, CS_THREADS, smem, s>>>(ptr, mid, cc, keys);
    k_cs_sort_big<<<148, CS_THREADS, smem, s>>>(ptr, big, cc, keys, tmp);
    k_cs_write<<<grid_for(nnz, 256, 8192), 256, 0, s>>>(keys, cc, nnz, t, idx, val);
  }
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (flags_host) {
    CsCounters h;
    if ((e = cudaMemcpyAsync(&h, cc, sizeof(h), cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
    *flags_host = h.flags;
  }
  return cudaSuccess;
}

}  // namespace sg

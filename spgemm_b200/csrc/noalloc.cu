// Allocation-free COO -> CSR/CSC conversion (spgemm_coo_to_cm_noalloc).
//
// Some callers cannot call cudaMalloc at the point where they convert a
// matrix: code running under an allocator that owns all device memory (a
// framework's caching allocator, a fixed arena sized up front), or
// latency-sensitive loops where an allocation would synchronise the device.
// They still own the input triplets and the output arrays, so this entry
// point only needs scratch for its prefix scan; that scratch lives in a
// file-scope __device__ array instead of being allocated.
//
// The array is fixed in size (SPGEMM_NOALLOC_MAX_MAJOR rows or columns at
// most) and exists on every GPU that loads this library until the process
// exits. Host code must not pass the array's name to a kernel (in host code
// it is only a stand-in symbol); the device address is looked up once per
// device with cudaGetSymbolAddress, on the first call made on that device,
// which also loads this file's kernels (so that no later call is the first
// use of a kernel under lazy module loading).
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/coo.h"
#include "../../include/spgemm_b200.h"

namespace {

constexpr int NA_THREADS = 1024;
constexpr int NA_ITEMS = 4;
constexpr int NA_TILE = NA_THREADS * NA_ITEMS;
constexpr long long NA_MAX_MAJOR = SPGEMM_NOALLOC_MAX_MAJOR;
constexpr int NA_MAX_TILES = (int)((NA_MAX_MAJOR + 1 + NA_TILE - 1) / NA_TILE);

// Layout: [0, NA_MAX_TILES) tile sums / tile offsets, then the grand total,
// then the status word (bit 0: index out of range, bit 1: unsorted input).
constexpr int NA_TOTAL = NA_MAX_TILES;
constexpr int NA_STATUS = NA_MAX_TILES + 1;
constexpr int NA_WORDS = NA_MAX_TILES + 2;

__device__ __align__(256) long long g_noalloc_scratch[NA_WORDS];

std::mutex g_setup_mutex;
long long* g_scratch_dev[64] = {nullptr};  // device address per device ordinal

__device__ __forceinline__ long long na_warp_incl(long long v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const long long t = __shfl_up_sync(0xffffffffu, v, d);
    if (lane >= d) v += t;
  }
  return v;
}

// Block exclusive scan (blockDim.x == NA_THREADS); *total receives the sum.
__device__ __forceinline__ long long na_block_excl(long long v, long long* shm, long long* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long long incl = na_warp_incl(v);
  if (lane == 31) shm[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    const long long w = shm[lane];
    const long long wi = na_warp_incl(w);
    shm[lane] = wi - w;
    if (lane == 31) shm[32] = wi;
  }
  __syncthreads();
  const long long r = shm[warp] + incl - v;
  *total = shm[32];
  __syncthreads();
  return r;
}

// Split the triplets: minor index and value in input order, entry counts per
// major index accumulated into ptr[major + 1] (ptr zeroed by the caller).
__global__ void na_split(const triplet* __restrict__ t, int nnz, int row_major, int n_major,
                         int n_minor, int* __restrict__ ptr, int* __restrict__ idx,
                         float* __restrict__ val, long long* scratch) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += gridDim.x * blockDim.x) {
    const triplet x = t[e];
    const int major = row_major ? x.ridx : x.cidx;
    const int minor = row_major ? x.cidx : x.ridx;
    if ((unsigned)major >= (unsigned)n_major || (unsigned)minor >= (unsigned)n_minor) {
      atomicOr(reinterpret_cast<unsigned long long*>(scratch + NA_STATUS), 1ull);
      continue;
    }
    if (e > 0) {
      const triplet y = t[e - 1];
      const int pm = row_major ? y.ridx : y.cidx;
      const int pn = row_major ? y.cidx : y.ridx;
      if (pm > major || (pm == major && pn > minor))
        atomicOr(reinterpret_cast<unsigned long long*>(scratch + NA_STATUS), 2ull);
    }
    idx[e] = minor;
    val[e] = x.val;
    atomicAdd(ptr + major + 1, 1);
  }
}

// Tile sums of ptr[0..n) (n = n_major + 1 counts; ptr[0] is 0).
__global__ void __launch_bounds__(NA_THREADS)
na_tile_sums(const int* __restrict__ ptr, int n, long long* scratch) {
  __shared__ long long shm[33];
  const long long base = (long long)blockIdx.x * NA_TILE;
  long long v = 0;
#pragma unroll
  for (int q = 0; q < NA_ITEMS; ++q) {
    const long long i = base + threadIdx.x * NA_ITEMS + q;
    if (i < n) v += ptr[i];
  }
  long long total;
  na_block_excl(v, shm, &total);
  if (threadIdx.x == 0) scratch[blockIdx.x] = total;
}

// Exclusive scan of the tile sums in place (one block), grand total after them.
__global__ void __launch_bounds__(NA_THREADS)
na_tile_offsets(int ntiles, long long* scratch) {
  __shared__ long long shm[33];
  long long carry = 0;
  for (int b = 0; b < ntiles; b += NA_THREADS) {
    const int i = b + threadIdx.x;
    const long long v = i < ntiles ? scratch[i] : 0;
    long long total;
    const long long ex = na_block_excl(v, shm, &total);
    if (i < ntiles) scratch[i] = carry + ex;
    carry += total;
  }
  if (threadIdx.x == 0) scratch[NA_TOTAL] = carry;
}

// Inclusive scan of the counts in place: ptr[i] = ptr[0] + ... + ptr[i], so
// with ptr[0] = 0 and ptr[i + 1] = count of major i, ptr becomes the pointer
// array.
__global__ void __launch_bounds__(NA_THREADS)
na_apply(int* __restrict__ ptr, int n, const long long* __restrict__ scratch) {
  __shared__ long long shm[33];
  const long long base = (long long)blockIdx.x * NA_TILE;
  int v[NA_ITEMS];
  long long sum = 0;
#pragma unroll
  for (int q = 0; q < NA_ITEMS; ++q) {
    const long long i = base + threadIdx.x * NA_ITEMS + q;
    v[q] = i < n ? ptr[i] : 0;
    sum += v[q];
  }
  long long total;
  long long run = na_block_excl(sum, shm, &total) + scratch[blockIdx.x];
#pragma unroll
  for (int q = 0; q < NA_ITEMS; ++q) {
    const long long i = base + threadIdx.x * NA_ITEMS + q;
    run += v[q];
    if (i < n) ptr[i] = (int)run;
  }
}

// Device address of g_noalloc_scratch on the current device (looked up on
// the first call made on that device, which also loads the kernels: a
// cudaFuncGetAttributes query loads a kernel's module without launching it).
cudaError_t scratch_for_current_device(long long** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_dev[dev]) {
    cudaFuncAttributes fa;
    const void* kernels[] = {reinterpret_cast<const void*>(na_split),
                             reinterpret_cast<const void*>(na_tile_sums),
                             reinterpret_cast<const void*>(na_tile_offsets),
                             reinterpret_cast<const void*>(na_apply)};
    for (const void* k : kernels) {
      e = cudaFuncGetAttributes(&fa, k);
      if (e != cudaSuccess) return e;
    }
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_dev[dev] = static_cast<long long*>(p);
  }
  *out = g_scratch_dev[dev];
  return cudaSuccess;
}

}  // namespace

extern "C" int spgemm_coo_to_cm_noalloc(const triplet* d_triplets, int nnz, int num_rows,
                                        int num_cols, int type, int* d_ptr, int* d_idx,
                                        float* d_val, void* stream, long long* nnz_check) {
  const bool row_major = type == ROW_MAJOR;
  const int n_major = row_major ? num_rows : num_cols;
  const int n_minor = row_major ? num_cols : num_rows;
  if (nnz < 0 || n_major < 0 || n_minor < 0 || !d_ptr || (nnz > 0 && (!d_triplets || !d_idx || !d_val)))
    return SPGEMM_ERR_INVALID;
  if ((long long)n_major > NA_MAX_MAJOR) return SPGEMM_ERR_TOO_LARGE;
  long long* scratch = nullptr;
  if (scratch_for_current_device(&scratch) != cudaSuccess) return SPGEMM_ERR_CUDA;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int n = n_major + 1;
  const int ntiles = (n + NA_TILE - 1) / NA_TILE;
  // the status word must start at zero; the tile words are fully rewritten
  if (cudaMemsetAsync(scratch + NA_STATUS, 0, sizeof(long long), s) != cudaSuccess)
    return SPGEMM_ERR_CUDA;
  if (cudaMemsetAsync(d_ptr, 0, sizeof(int) * (size_t)n, s) != cudaSuccess) return SPGEMM_ERR_CUDA;
  if (nnz > 0) {
    const int blocks = (int)(((long long)nnz + 255) / 256 < 4096 ? ((long long)nnz + 255) / 256 : 4096);
    na_split<<<blocks, 256, 0, s>>>(d_triplets, nnz, row_major ? 1 : 0, n_major, n_minor, d_ptr,
                                    d_idx, d_val, scratch);
  }
  na_tile_sums<<<ntiles, NA_THREADS, 0, s>>>(d_ptr, n, scratch);
  na_tile_offsets<<<1, NA_THREADS, 0, s>>>(ntiles, scratch);
  na_apply<<<ntiles, NA_THREADS, 0, s>>>(d_ptr, n, scratch);
  if (cudaGetLastError() != cudaSuccess) return SPGEMM_ERR_CUDA;
  if (nnz_check) {
    // optional check, synchronises the stream: copies back the grand total
    // and the status word
    long long host[2] = {0, 0};
    if (cudaMemcpyAsync(host, scratch + NA_TOTAL, sizeof(host), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
      return SPGEMM_ERR_CUDA;
    *nnz_check = host[0];
    if (host[1] & 1) return SPGEMM_ERR_INVALID;  // an index outside the dimensions
    if (host[1] & 2) return SPGEMM_ERR_INVALID;  // triplets not sorted by (major, minor)
  }
  return SPGEMM_OK;
}

// scan_sort.cu — device prefix sums and the stable LSD radix sort of the LBVH build.
//
// Both are HBM-bound integer passes: the scan reads and writes each word once per level; the
// sort makes one histogram pass and one scatter pass per 4-bit digit over (key, value) pairs,
// each thread owning 16 consecutive pairs (four 16-byte loads) so a tile is one contiguous 16 KB
// read. Stability comes from the blocked arrangement: a tile's pairs are ranked by (digit,
// thread, item), the order they appear in memory.
#include "vt_internal.cuh"

namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;  // 1024 words per block

__device__ __forceinline__ uint32_t warp_inclusive_scan(uint32_t v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t u = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += u;
  }
  return v;
}

// Block-wide exclusive scan of one value per thread (blockDim.x == 256). Returns the exclusive
// prefix; *total receives the block sum.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t *total) {
  __shared__ uint32_t warp_sums[kScanThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t inc = warp_inclusive_scan(v);
  if (lane == 31) warp_sums[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < kScanThreads / 32 ? warp_sums[lane] : 0u;
    uint32_t wi = warp_inclusive_scan(w);
    if (lane < kScanThreads / 32) warp_sums[lane] = wi - w;
  }
  __syncthreads();
  uint32_t out = warp_sums[warp] + inc - v;
  if (total) {
    __shared__ uint32_t tot;
    if (threadIdx.x == kScanThreads - 1) tot = out + v;
    __syncthreads();
    *total = tot;
  }
  return out;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_block(const uint32_t *in, uint32_t *out,
                                                               uint32_t n, uint32_t *block_sums) {
  const uint32_t base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  uint32_t v[kScanItems];
  uint32_t sum = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    v[k] = base + k < n ? in[base + k] : 0u;
    sum += v[k];
  }
  uint32_t total;
  uint32_t prefix = block_exclusive_scan(sum, &total);
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    if (base + k < n) out[base + k] = prefix;
    prefix += v[k];
  }
  if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

__global__ void k_scan_add(uint32_t *out, uint32_t n, const uint32_t *block_prefix) {
  const uint32_t add = block_prefix[blockIdx.x];
  const uint32_t base = blockIdx.x * kScanTile;
  for (uint32_t k = threadIdx.x; k < kScanTile; k += blockDim.x)
    if (base + k < n) out[base + k] += add;
}

__global__ void k_copy_word(const uint32_t *src, uint32_t *dst) { *dst = *src; }

// ---- radix sort ------------------------------------------------------------------------------
constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;  // 4096 pairs per block
constexpr int kDigits = 16;

__device__ __forceinline__ void load_tile(const uint32_t *src, uint32_t base, uint32_t n,
                                          uint32_t (&v)[kSortItems]) {
  if (base + kSortItems <= n) {
    const uint4 *p = reinterpret_cast<const uint4 *>(src + base);
#pragma unroll
    for (int q = 0; q < kSortItems / 4; ++q) {
      uint4 x = p[q];
      v[4 * q] = x.x; v[4 * q + 1] = x.y; v[4 * q + 2] = x.z; v[4 * q + 3] = x.w;
    }
  } else {
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) v[k] = base + k < n ? src[base + k] : 0u;
  }
}

__global__ void __launch_bounds__(kSortThreads) k_radix_hist(const uint32_t *keys, uint32_t n,
                                                               int shift, uint32_t *hist,
                                                               uint32_t nblocks) {
  __shared__ uint32_t cnt[kDigits];
  if (threadIdx.x < kDigits) cnt[threadIdx.x] = 0;
  __syncthreads();
  const uint32_t base = blockIdx.x * kSortTile + threadIdx.x * kSortItems;
  uint32_t k[kSortItems];
  load_tile(keys, base, n, k);
#pragma unroll
  for (int i = 0; i < kSortItems; ++i)
    if (base + i < n) atomicAdd(&cnt[(k[i] >> shift) & (kDigits - 1)], 1u);
  __syncthreads();
  if (threadIdx.x < kDigits) hist[threadIdx.x * nblocks + blockIdx.x] = cnt[threadIdx.x];
}

__global__ void __launch_bounds__(kSortThreads) k_radix_scatter(
    const uint32_t *keys, const uint32_t *vals, uint32_t n, int shift, const uint32_t *offsets,
    uint32_t nblocks, uint32_t *keys_out, uint32_t *vals_out) {
  __shared__ uint32_t cnt[kDigits][kSortThreads];
  __shared__ uint32_t dstart[kDigits], goff[kDigits];
  const int t = threadIdx.x;
#pragma unroll
  for (int d = 0; d < kDigits; ++d) cnt[d][t] = 0;
  const uint32_t base = blockIdx.x * kSortTile + t * kSortItems;
  uint32_t k[kSortItems], v[kSortItems];
  load_tile(keys, base, n, k);
  load_tile(vals, base, n, v);
  // Column t of cnt is private to thread t here.
#pragma unroll
  for (int i = 0; i < kSortItems; ++i)
    if (base + i < n) cnt[(k[i] >> shift) & (kDigits - 1)][t] += 1u;
  __syncthreads();
  // Exclusive scan of cnt in digit-major order: thread t owns the 16 consecutive entries of row
  // t / 16, columns (t % 16) * 16 ...
  const int row = t / 16, col0 = (t % 16) * 16;
  uint32_t local[16];
  uint32_t sum = 0;
#pragma unroll
  for (int j = 0; j < 16; ++j) { local[j] = cnt[row][col0 + j]; sum += local[j]; }
  uint32_t prefix = block_exclusive_scan(sum, nullptr);
  __syncthreads();
#pragma unroll
  for (int j = 0; j < 16; ++j) { cnt[row][col0 + j] = prefix; prefix += local[j]; }
  __syncthreads();
  if (t < kDigits) {
    dstart[t] = cnt[t][0];
    goff[t] = offsets[t * nblocks + blockIdx.x];
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < kSortItems; ++i) {
    if (base + i >= n) break;
    const int d = (k[i] >> shift) & (kDigits - 1);
    const uint32_t pos = goff[d] + (cnt[d][t] - dstart[d]);
    cnt[d][t] += 1u;
    keys_out[pos] = k[i];
    vals_out[pos] = v[i];
  }
}

}  // namespace

size_t vt_scan_temp_words(uint32_t n) {
  size_t words = 4;
  while (n > 1) {
    n = (n + kScanTile - 1) / kScanTile;
    words += n;
  }
  return words;
}

void vt_scan_exclusive(const uint32_t *in, uint32_t *out, uint32_t n, uint32_t *temp,
                       uint32_t *total_dev, cudaStream_t s) {
  if (n == 0) return;
  const uint32_t nb = (n + kScanTile - 1) / kScanTile;
  uint32_t *sums = temp;
  k_scan_block<<<nb, kScanThreads, 0, s>>>(in, out, n, sums);
  if (nb > 1) {
    vt_scan_exclusive(sums, sums, nb, temp + nb, total_dev, s);
    k_scan_add<<<nb, kScanThreads, 0, s>>>(out, n, sums);
  } else if (total_dev) {
    k_copy_word<<<1, 1, 0, s>>>(sums, total_dev);
  }
}

size_t vt_radix_temp_words(uint32_t n) {
  const uint32_t nb = (n + kSortTile - 1) / kSortTile;
  return (size_t)kDigits * nb + vt_scan_temp_words(kDigits * nb) + 4;
}

void vt_radix_sort_pairs(uint32_t *keys, uint32_t *vals, uint32_t *keys_alt, uint32_t *vals_alt,
                         uint32_t n, int bits, uint32_t *temp, cudaStream_t s) {
  if (n <= 1) return;
  const uint32_t nb = (n + kSortTile - 1) / kSortTile;
  uint32_t *hist = temp;
  uint32_t *scan_temp = temp + (size_t)kDigits * nb;
  uint32_t *src_k = keys, *src_v = vals, *dst_k = keys_alt, *dst_v = vals_alt;
  int passes = (bits + 3) / 4;
  for (int p = 0; p < passes; ++p) {
    const int shift = 4 * p;
    k_radix_hist<<<nb, kSortThreads, 0, s>>>(src_k, n, shift, hist, nb);
    vt_scan_exclusive(hist, hist, kDigits * nb, scan_temp, nullptr, s);
    k_radix_scatter<<<nb, kSortThreads, 0, s>>>(src_k, src_v, n, shift, hist, nb, dst_k, dst_v);
    uint32_t *tk = src_k, *tv = src_v;
    src_k = dst_k; src_v = dst_v; dst_k = tk; dst_v = tv;
  }
  if (src_k != keys) {
    cudaMemcpyAsync(keys, src_k, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(vals, src_v, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
  }
}

// nrc_tc.cu — the radiance cache's inference on the fifth-generation tensor cores (tcgen05).
//
// One CTA of 128 threads owns a 128-row tile: thread t encodes query row t (nrc_encode) into the
// tile's fp16 activation matrix X in shared memory; each layer is one 128 x N x 64 product
// D = X W^T issued by a single thread as four tcgen05.mma (kind::f16, M = 128, K = 16 each, fp16
// operands from shared memory, fp32 accumulator in tensor memory), committed to an mbarrier. The
// four warps then read their 32 accumulator lanes back with tcgen05.ld, apply the ReLU and the fp16
// rounding (one cvt.rn.relu.f16x2 per pair) and write the next layer's X in place. Layers 1-5 use
// TMEM columns 0-63 (N = 64), the output layer columns 64-79 (N = 16, the padded output rows).
// Weights are converted to fp16 once per CTA into the same shared-memory layout; CTAs persist over
// tiles, three per SM (58 KB of shared memory and 128 TMEM columns each), so that one CTA's
// hash-grid gathers overlap the others' products.
//
// Operand layout (both K-major, no swizzle): 8 x 8 fp16 core matrices of 128 contiguous bytes (8 rows
// of 16 bytes); core matrix (row group g, k chunk c) at byte (8 g + c) 128 of the operand, so the
// matrix descriptor's leading byte offset (between the two k chunks of one K = 16 step) is 128 and
// its stride byte offset (between row groups) 1024; step kb starts 256 kb bytes in.
//
// Every wait is bounded: a commit that does not arrive within the limit sets bit 4 of the cache's
// status word, the CTA stops issuing, waits (bounded again) for what it issued, frees its tensor
// memory and returns; vt_nrc_get_info then reports the error.
#include <cuda_fp16.h>
#include <stdint.h>

#include <algorithm>

#include "nrc.cuh"
#include "vt_internal.cuh"

namespace {
using namespace vtd;

constexpr int kTcRows = 128;
constexpr uint32_t kTcCols = 128;  // TMEM columns per CTA (a power of two >= 32): 0-63 hidden, 64-79 output
constexpr uint32_t kTcOutCol = 64;
constexpr uint32_t kTcW = kNrcHidden * 64 * 64 * 2;  // 40,960 B
constexpr uint32_t kTcWo = kNrcOutRows * 64 * 2;     // 2,048 B
constexpr uint32_t kTcX = kTcRows * 64 * 2;          // 16,384 B
constexpr uint32_t kTcSmem = kTcW + kTcWo + kTcX + 64;
// At most three CTAs fit an SM's 228 KB of shared memory, so at most 3 x 128 of its 512 TMEM
// columns are ever requested and an allocation never waits on another CTA.
static_assert(4 * (size_t)kTcSmem > 228 * 1024, "more than three CTAs per SM would oversubscribe TMEM");
constexpr uint32_t kNrcWaitTimeout = 4u;  // cache status bit: a tensor-core commit did not arrive
constexpr uint32_t kWaitLimit = 1u << 22;

// Instruction descriptors (kind::f16): D fp32 (bits 4-5 = 1), A and B fp16 (bits 7-12 = 0), both
// K-major (bits 15-16 = 0), N >> 3 in bits 17-22, M >> 4 in bits 24-28.
constexpr uint32_t idesc_f16(uint32_t m, uint32_t n) { return (1u << 4) | ((n >> 3) << 17) | ((m >> 4) << 24); }
constexpr uint32_t kIdescHidden = idesc_f16(128, 64);
constexpr uint32_t kIdescOut = idesc_f16(128, 16);

// Byte offset of element (r, k) of an R x 64 K-major operand in the no-swizzle core-matrix layout.
__device__ __forceinline__ uint32_t tc_off(uint32_t r, uint32_t k) {
  return ((((r >> 3) << 3) + (k >> 3)) << 7) + ((r & 7u) << 4) + ((k & 7u) << 1);
}
// Shared-memory matrix descriptor: start address >> 4 (bits 0-13), leading byte offset 128 >> 4
// (bits 16-29), stride byte offset 1024 >> 4 (bits 32-45), descriptor version 1 (bits 46-47), base
// offset 0, no swizzle (bits 61-63 = 0).
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr) {
  return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)(128u >> 4) << 16) | ((uint64_t)(1024u >> 4) << 32) |
         (1ull << 46);
}
__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void tc_mma(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      :
      : "r"(dtmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}
__device__ __forceinline__ void tc_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Generic-proxy shared-memory writes become visible to the tensor cores' (async proxy) reads.
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Bounded wait for the mbarrier phase with parity `parity` to complete.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  for (uint32_t i = 0; i < kWaitLimit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// 32 consecutive accumulator columns of this thread's lane (row).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]),
        "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
        "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld4(uint32_t taddr, uint32_t (&v)[4]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3])
               : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// 16 fp16 values (8 registers) of row r, columns 16 h .. 16 h + 15, into the operand at X.
__device__ __forceinline__ void store_row16(unsigned char *X, uint32_t r, int h, const uint32_t *p) {
  *reinterpret_cast<uint4 *>(X + tc_off(r, 16 * h)) = make_uint4(p[0], p[1], p[2], p[3]);
  *reinterpret_cast<uint4 *>(X + tc_off(r, 16 * h + 8)) = make_uint4(p[4], p[5], p[6], p[7]);
}

// out[row] = the network's four outputs for rows < n.
__global__ void __launch_bounds__(kTcRows) k_nrc_infer_tc(NrcGrid G, const float *__restrict__ mlp,
                                                          const NrcInput *__restrict__ in, uint32_t n,
                                                          float4 *__restrict__ out) {
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char *W = smem, *Wo = smem + kTcW, *X = smem + kTcW + kTcWo;
  uint64_t *mbar = reinterpret_cast<uint64_t *>(smem + kTcW + kTcWo + kTcX);
  uint32_t *tmemSlot = reinterpret_cast<uint32_t *>(smem + kTcW + kTcWo + kTcX + 16);
  const uint32_t tid = threadIdx.x, warp = tid >> 5;

  // Weights: fp32 masters -> fp16 in the operand layout (hidden layer l at W + l * 8 KB, rows = outputs).
  for (uint32_t i = tid; i < (uint32_t)kNrcHidden * 4096u / 2u; i += blockDim.x) {
    const float2 v = __ldg(reinterpret_cast<const float2 *>(mlp) + i);
    const uint32_t e = 2u * i, l = e >> 12, r = (e >> 6) & 63u, k = e & 63u;
    *reinterpret_cast<__half2 *>(W + (l << 13) + tc_off(r, k)) = __floats2half2_rn(v.x, v.y);
  }
  for (uint32_t i = tid; i < (uint32_t)kNrcOutRows * 64u / 2u; i += blockDim.x) {
    const float2 v = __ldg(reinterpret_cast<const float2 *>(mlp + kNrcHidden * 4096) + i);
    const uint32_t e = 2u * i, r = e >> 6, k = e & 63u;
    *reinterpret_cast<__half2 *>(Wo + tc_off(r, k)) = __floats2half2_rn(v.x, v.y);
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(mbar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmemSlot)),
                 "r"(kTcCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmemSlot;
  const uint32_t lane_base = tmem + ((warp * 32u) << 16);  // this warp's 32 TMEM lanes
  const uint32_t mb = smem_addr(mbar), xs = smem_addr(X), ws = smem_addr(W), wos = smem_addr(Wo);
  uint32_t phase = 0;
  bool ok = true;  // CTA-uniform after each __syncthreads_and

  for (uint32_t base = blockIdx.x * kTcRows; base < n; base += gridDim.x * kTcRows) {
    // The tile's encoded inputs (rows past n encode a zero query; their outputs are not written).
    {
      const uint32_t row = base + tid;
      NrcInput q;
      if (row < n) {
        q = in[row];
      } else {
        q.a = q.b = q.c = q.d = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      }
      __half h[64];
      nrc_encode(G, q, h);
      uint32_t p[32];
#pragma unroll
      for (int j = 0; j < 32; ++j)
        p[j] = (uint32_t)__half_as_ushort(h[2 * j]) | ((uint32_t)__half_as_ushort(h[2 * j + 1]) << 16);
#pragma unroll
      for (int c = 0; c < 4; ++c) store_row16(X, tid, c, p + 8 * c);
    }
#pragma unroll 1
    for (int l = 0; l <= kNrcHidden; ++l) {
      const bool last = l == kNrcHidden;
      fence_async_smem();
      tc_fence_before();
      ok = __syncthreads_and(ok);
      if (!ok) break;
      tc_fence_after();
      if (tid == 0) {
        const uint32_t b0 = last ? wos : ws + ((uint32_t)l << 13);
        const uint32_t d = tmem + (last ? kTcOutCol : 0u);
#pragma unroll
        for (uint32_t kb = 0; kb < 4; ++kb)
          tc_mma(d, tc_desc(xs + 256u * kb), tc_desc(b0 + 256u * kb), last ? kIdescOut : kIdescHidden, kb > 0);
        tc_commit(mb);
      }
      // Warp-uniform, so that the warp's tcgen05.ld runs on all of its lanes or on none.
      if (!__all_sync(0xffffffffu, mbar_wait(mb, phase))) {
        ok = false;
        continue;  // the next barrier makes the stop CTA-wide
      }
      phase ^= 1u;
      tc_fence_after();
      if (!last) {
        // ReLU, fp16, back into X as the next layer's input (the product has read X: its commit arrived).
#pragma unroll
        for (int half = 0; half < 2; ++half) {
          uint32_t v[32];
          tmem_ld32(lane_base + 32u * half, v);
          tmem_wait_ld();
          uint32_t p[16];
#pragma unroll
          for (int j = 0; j < 16; ++j) p[j] = nrc_pack_relu(__uint_as_float(v[2 * j]), __uint_as_float(v[2 * j + 1]));
          store_row16(X, tid, 2 * half, p);
          store_row16(X, tid, 2 * half + 1, p + 8);
        }
      } else {
        uint32_t v[4];
        tmem_ld4(lane_base + kTcOutCol, v);
        tmem_wait_ld();
        const uint32_t row = base + tid;
        if (row < n)
          out[row] = make_float4(__uint_as_float(v[0]), __uint_as_float(v[1]), __uint_as_float(v[2]), __uint_as_float(v[3]));
      }
    }
    tc_fence_before();
    ok = __syncthreads_and(ok);
    if (!ok) break;
  }
  if (!ok) {
    if (tid == 0) nrc_fault(G, kNrcWaitTimeout);
    // Let a product still in flight finish (bounded) before the tensor memory is freed.
    (void)mbar_wait(mb, phase);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcCols) : "memory");
}

}  // namespace

vt_status vt_nrc_infer_tc(vt_ctx *ctx, vt_nrc *nrc, const NrcInput *in, uint32_t n, float4 *out, cudaStream_t s) {
  if (n == 0) return VT_OK;
  static bool attrs = false;
  if (!attrs) {
    VT_CUDA(ctx, cudaFuncSetAttribute(k_nrc_infer_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem));
    attrs = true;
  }
  const uint32_t tiles = (n + kTcRows - 1) / kTcRows;
  const uint32_t grid = std::min<uint32_t>(tiles, (uint32_t)ctx->sm_count * 3u);
  k_nrc_infer_tc<<<grid, kTcRows, kTcSmem, s>>>(nrc->grid, nrc->d_p, in, n, out);
  VT_CUDA(ctx, cudaGetLastError());
  return VT_OK;
}

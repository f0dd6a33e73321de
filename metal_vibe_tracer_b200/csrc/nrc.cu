// nrc.cu — the neural radiance cache's network: parameter initialisation, the fused training kernel
// (forward, relative-L2 loss, backward to the weights and to the hash-grid entries), Adam and the
// host API. Inference runs on the tcgen05 tensor cores (nrc_tc.cu).
//
// The training kernel keeps a 128-row tile per CTA (4 warps x 32 rows) on the warp-level tensor path
// (mma.sync m16n8k16; its backward pass reads every layer's activations and the weights transposed,
// which the register fragments give directly). Activations stay in registers between layers: the
// fp32 accumulator fragment for two adjacent n-tiles is the fp16 A fragment of the next layer's
// k-tile. Each layer's fp16 output also goes to shared memory, where the weight gradient dW = dZ^T H
// reads it (and dZ) through ldmatrix.trans; the data gradient dH = dZ W reads W the same way. Rows
// are padded to 72 halves (144 B), which keeps the fragment loads and stores free of bank conflicts.
#include <cmath>
#include <cstring>
#include <vector>

#include "nrc.cuh"
#include "vt_internal.cuh"

namespace {
using namespace vtd;

constexpr int kLd = kNrcLd;
constexpr size_t kTrainSmem =
    (size_t)(kNrcHidden * 64 * kLd + kNrcOutRows * kLd + kNrcTile * kLd * (kNrcHidden + 2)) * sizeof(__half);
constexpr float kGradClip = 512.0f;  // per-output loss gradient bound before the loss scale (x 64 stays in fp16 range)

__device__ __forceinline__ uint32_t hash_u32(uint32_t x) {
  x ^= x >> 16; x *= 0x7feb352du;
  x ^= x >> 15; x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}
__device__ __forceinline__ float hash_uniform(uint32_t seed, uint64_t i) {
  const uint32_t h = hash_u32(hash_u32((uint32_t)i ^ seed) ^ hash_u32((uint32_t)(i >> 32) + 0x9e3779b9u));
  return (float)(h >> 8) * (1.0f / 16777216.0f);
}

// Xavier-uniform hidden and output weights (output rows 4-15 zero); grid features U(-1e-4, 1e-4).
__global__ void k_nrc_init(float *__restrict__ p, uint64_t n, uint32_t seed) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const float u = hash_uniform(seed, i) * 2.0f - 1.0f;
    float v;
    if (i < (uint64_t)kNrcHidden * 4096u) {
      v = u * 0.21650635f;  // sqrt(6 / (64 + 64))
    } else if (i < (uint64_t)kNrcMlpParams) {
      const uint32_t r = (uint32_t)(i - (uint64_t)kNrcHidden * 4096u) >> 6;
      v = r < (uint32_t)kNrcOut ? u * 0.29704426f : 0.0f;  // sqrt(6 / (64 + 4)); unused rows zero
    } else {
      v = u * 1e-4f;
    }
    p[i] = v;
  }
}

__device__ __forceinline__ void load_weights(const float *__restrict__ mlp, __half *W, __half *Wo) {
  for (int i = threadIdx.x; i < kNrcHidden * 4096 / 4; i += blockDim.x) {
    const float4 v = __ldg(reinterpret_cast<const float4 *>(mlp) + i);
    const int e = 4 * i, l = e >> 12, r = (e >> 6) & 63, c = e & 63;
    __half *d = W + (l * 64 + r) * kLd + c;
    d[0] = __float2half_rn(v.x); d[1] = __float2half_rn(v.y); d[2] = __float2half_rn(v.z); d[3] = __float2half_rn(v.w);
  }
  for (int i = threadIdx.x; i < kNrcOutRows * 64 / 4; i += blockDim.x) {
    const float4 v = __ldg(reinterpret_cast<const float4 *>(mlp + kNrcHidden * 4096) + i);
    const int e = 4 * i, r = e >> 6, c = e & 63;
    __half *d = Wo + r * kLd + c;
    d[0] = __float2half_rn(v.x); d[1] = __float2half_rn(v.y); d[2] = __float2half_rn(v.z); d[3] = __float2half_rn(v.w);
  }
}

// The warp's A fragments (rows row0..row0+31, 2 m-tiles x 4 k-tiles) from a row-major tile.
__device__ __forceinline__ void load_a(uint32_t (&a)[2][4][4], const __half *X, int row0, int lane) {
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int kt = 0; kt < 4; ++kt) nrc_ldsm4(a[mt][kt], X + (row0 + 16 * mt + (lane & 15)) * kLd + 16 * kt + 8 * (lane >> 4));
}

// Accumulator fragments (2 m-tiles x 8 n-tiles) -> fp16 A fragments of the next k-tiles.
__device__ __forceinline__ void acc_to_a(const float (&acc)[2][8][4], uint32_t (&a)[2][4][4], bool relu) {
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
      const float *c0 = acc[mt][2 * kk], *c1 = acc[mt][2 * kk + 1];
      if (relu) {
        a[mt][kk][0] = nrc_pack_relu(c0[0], c0[1]);
        a[mt][kk][1] = nrc_pack_relu(c0[2], c0[3]);
        a[mt][kk][2] = nrc_pack_relu(c1[0], c1[1]);
        a[mt][kk][3] = nrc_pack_relu(c1[2], c1[3]);
      } else {
        a[mt][kk][0] = nrc_pack(c0[0], c0[1]);
        a[mt][kk][1] = nrc_pack(c0[2], c0[3]);
        a[mt][kk][2] = nrc_pack(c1[0], c1[1]);
        a[mt][kk][3] = nrc_pack(c1[2], c1[3]);
      }
    }
}

// A fragments -> the row-major tile (the positions they were loaded from).
__device__ __forceinline__ void store_a(const uint32_t (&a)[2][4][4], __half *T, int row0, int g, int t) {
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
      __half *r = T + (row0 + 16 * mt + g) * kLd + 16 * kk + 2 * t;
      *reinterpret_cast<uint32_t *>(r) = a[mt][kk][0];
      *reinterpret_cast<uint32_t *>(r + 8 * kLd) = a[mt][kk][1];
      *reinterpret_cast<uint32_t *>(r + 8) = a[mt][kk][2];
      *reinterpret_cast<uint32_t *>(r + 8 * kLd + 8) = a[mt][kk][3];
    }
}

// One hidden layer: a <- relu(a W^T), W [64 out][64 in] in shared memory.
__device__ __forceinline__ void hidden_layer(uint32_t (&a)[2][4][4], const __half *W, int g, int t) {
  float acc[2][8][4];
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) acc[mt][nt][0] = acc[mt][nt][1] = acc[mt][nt][2] = acc[mt][nt][3] = 0.0f;
#pragma unroll
  for (int kt = 0; kt < 4; ++kt)
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const __half *w = W + (8 * nt + g) * kLd + 16 * kt + 2 * t;
      const uint32_t b0 = *reinterpret_cast<const uint32_t *>(w), b1 = *reinterpret_cast<const uint32_t *>(w + 8);
      nrc_mma(acc[0][nt], a[0][kt], b0, b1);
      nrc_mma(acc[1][nt], a[1][kt], b0, b1);
    }
  acc_to_a(acc, a, true);
}

// The output layer (rows 0-7 of Wo; 3 used): o[mt] = (row g: cols 2t, 2t+1; row g + 8: same).
__device__ __forceinline__ void output_layer(const uint32_t (&a)[2][4][4], const __half *Wo, int g, int t, float (&o)[2][4]) {
#pragma unroll
  for (int mt = 0; mt < 2; ++mt) o[mt][0] = o[mt][1] = o[mt][2] = o[mt][3] = 0.0f;
#pragma unroll
  for (int kt = 0; kt < 4; ++kt) {
    const __half *w = Wo + g * kLd + 16 * kt + 2 * t;
    const uint32_t b0 = *reinterpret_cast<const uint32_t *>(w), b1 = *reinterpret_cast<const uint32_t *>(w + 8);
    nrc_mma(o[0], a[0][kt], b0, b1);
    nrc_mma(o[1], a[1][kt], b0, b1);
  }
}

// dW[m0 + 0..15][n0 + 0..16 * np2 - 1] += DZ[rows][m0..]^T  Hp[rows][n0..] over the tile's 128 rows.
template <int kNp>
__device__ __forceinline__ void weight_grad(const __half *DZ, const __half *Hp, int m0, int n0, int lane,
                                            float (&acc)[2 * kNp][4]) {
#pragma unroll
  for (int nt = 0; nt < 2 * kNp; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.0f;
#pragma unroll 2
  for (int kt = 0; kt < kNrcTile / 16; ++kt) {
    uint32_t af[4];
    nrc_ldsm4t(af, DZ + (16 * kt + (lane & 7) + 8 * (lane >> 4)) * kLd + m0 + 8 * ((lane >> 3) & 1));
#pragma unroll
    for (int np = 0; np < kNp; ++np) {
      uint32_t bf[4];
      nrc_ldsm4t(bf, Hp + (16 * kt + (lane & 7) + 8 * ((lane >> 3) & 1)) * kLd + n0 + 16 * np + 8 * (lane >> 4));
      nrc_mma(acc[2 * np], af, bf[0], bf[1]);
      nrc_mma(acc[2 * np + 1], af, bf[2], bf[3]);
    }
  }
}

// dH = dZ W over the k-tiles of dZ (kNk of them, out = 16 kNk) into 2 * kNp n-tiles of H.
template <int kNk, int kNp>
__device__ __forceinline__ void data_grad(const uint32_t (&dz)[2][4][4], const __half *W, int lane,
                                          float (&acc)[2][8][4]) {
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) acc[mt][nt][0] = acc[mt][nt][1] = acc[mt][nt][2] = acc[mt][nt][3] = 0.0f;
#pragma unroll
  for (int kt = 0; kt < kNk; ++kt)
#pragma unroll
    for (int np = 0; np < kNp; ++np) {
      uint32_t bf[4];
      nrc_ldsm4t(bf, W + (16 * kt + (lane & 7) + 8 * ((lane >> 3) & 1)) * kLd + 16 * np + 8 * (lane >> 4));
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) {
        nrc_mma(acc[mt][2 * np], dz[mt][kt], bf[0], bf[1]);
        nrc_mma(acc[mt][2 * np + 1], dz[mt][kt], bf[2], bf[3]);
      }
    }
}

// dZ = dH * (H > 0), H the layer's stored fp16 output.
__device__ __forceinline__ void relu_mask(float (&acc)[2][8][4], const __half *H, int row0, int g, int t) {
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const __half *h = H + (row0 + 16 * mt + g) * kLd + 8 * nt + 2 * t;
      const __half2 u = *reinterpret_cast<const __half2 *>(h), v = *reinterpret_cast<const __half2 *>(h + 8 * kLd);
      if (!(__low2float(u) > 0.0f)) acc[mt][nt][0] = 0.0f;
      if (!(__high2float(u) > 0.0f)) acc[mt][nt][1] = 0.0f;
      if (!(__low2float(v) > 0.0f)) acc[mt][nt][2] = 0.0f;
      if (!(__high2float(v) > 0.0f)) acc[mt][nt][3] = 0.0f;
    }
}

// Gradient sums of one batch (rows < min(*count, cap), or cap when count is null) under the relative
// L2 loss sum_c (p_c - y_c)^2 / (lum(p)^2 + 0.01) over the four outputs, lum = lumW . p held constant
// (Mueller et al. 2021; lumW the luminance weights of rgb, or the lanes' mean for a spectral cache):
// the weights' into gmlp, the grid features' into gtable (float2 atomics), both times kNrcLossScale,
// and the loss sum into *loss. One CTA per 128-row tile.
__global__ void __launch_bounds__(kNrcTile, 1) k_nrc_train(NrcGrid G, const float *__restrict__ mlp,
                                                           const NrcInput *__restrict__ in,
                                                           const float4 *__restrict__ target,
                                                           const uint32_t *__restrict__ count, uint32_t cap,
                                                           float *__restrict__ gmlp, float2 *__restrict__ gtable,
                                                           float *__restrict__ loss, float4 lumW) {
  extern __shared__ __align__(16) __half sm[];
  __half *W = sm, *Wo = W + kNrcHidden * 64 * kLd, *X = Wo + kNrcOutRows * kLd, *H = X + kNrcTile * kLd,
         *DZ = H + kNrcHidden * kNrcTile * kLd;
  const uint32_t n = count ? min(*count, cap) : cap;
  const uint32_t base = blockIdx.x * kNrcTile;
  if (base >= n) return;
  load_weights(mlp, W, Wo);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3, row0 = 32 * warp;
  {
    const uint32_t row = base + threadIdx.x;
    NrcInput q;
    if (row < n) {
      q = in[row];
    } else {
      q.a = q.b = q.c = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
    nrc_encode(G, q, X + threadIdx.x * kLd);
  }
  __syncthreads();
  // Forward, keeping every layer's output.
  uint32_t a[2][4][4];
  load_a(a, X, row0, lane);
#pragma unroll 1
  for (int l = 0; l < kNrcHidden; ++l) {
    hidden_layer(a, W + l * 64 * kLd, g, t);
    store_a(a, H + l * kNrcTile * kLd, row0, g, t);
  }
  float o[2][4];
  output_layer(a, Wo, g, t, o);
  // Loss gradient per row (clipped, then times the loss scale), laid out as the A fragment of
  // k-tile 0 (outputs 0-3 of 16).
  uint32_t da[2][4][4];
  float lsum = 0.0f;
#pragma unroll
  for (int mt = 0; mt < 2; ++mt) {
    const int q0 = lane & ~3, q1 = q0 | 1;
    float p[2][4];
    p[0][0] = __shfl_sync(0xffffffffu, o[mt][0], q0);
    p[0][1] = __shfl_sync(0xffffffffu, o[mt][1], q0);
    p[0][2] = __shfl_sync(0xffffffffu, o[mt][0], q1);
    p[0][3] = __shfl_sync(0xffffffffu, o[mt][1], q1);
    p[1][0] = __shfl_sync(0xffffffffu, o[mt][2], q0);
    p[1][1] = __shfl_sync(0xffffffffu, o[mt][3], q0);
    p[1][2] = __shfl_sync(0xffffffffu, o[mt][2], q1);
    p[1][3] = __shfl_sync(0xffffffffu, o[mt][3], q1);
    float d[2][4];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const uint32_t row = base + row0 + 16 * mt + g + 8 * h;
      d[h][0] = d[h][1] = d[h][2] = d[h][3] = 0.0f;
      if (row < n) {
        const float4 y = __ldg(target + row);
        const float lum = lumW.x * p[h][0] + lumW.y * p[h][1] + lumW.z * p[h][2] + lumW.w * p[h][3];
        const float inv = 1.0f / (lum * lum + 0.01f);
        const float e0 = p[h][0] - y.x, e1 = p[h][1] - y.y, e2 = p[h][2] - y.z, e3 = p[h][3] - y.w;
        if (t == 0) lsum += (e0 * e0 + e1 * e1 + e2 * e2 + e3 * e3) * inv;
        d[h][0] = fminf(fmaxf(2.0f * e0 * inv, -kGradClip), kGradClip) * kNrcLossScale;
        d[h][1] = fminf(fmaxf(2.0f * e1 * inv, -kGradClip), kGradClip) * kNrcLossScale;
        d[h][2] = fminf(fmaxf(2.0f * e2 * inv, -kGradClip), kGradClip) * kNrcLossScale;
        d[h][3] = fminf(fmaxf(2.0f * e3 * inv, -kGradClip), kGradClip) * kNrcLossScale;
      }
    }
    da[mt][0][0] = t == 0 ? nrc_pack(d[0][0], d[0][1]) : (t == 1 ? nrc_pack(d[0][2], d[0][3]) : 0u);
    da[mt][0][1] = t == 0 ? nrc_pack(d[1][0], d[1][1]) : (t == 1 ? nrc_pack(d[1][2], d[1][3]) : 0u);
    da[mt][0][2] = da[mt][0][3] = 0u;
#pragma unroll
    for (int kk = 1; kk < 4; ++kk) da[mt][kk][0] = da[mt][kk][1] = da[mt][kk][2] = da[mt][kk][3] = 0u;
  }
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, s);
  if (lane == 0 && lsum != 0.0f) atomicAdd(loss, lsum);
  // The output layer: dWo = dOut^T H4 (warp w: inputs 16w..16w+15), dH4 = dOut Wo.
  store_a(da, DZ, row0, g, t);
  __syncthreads();
  {
    float acc[2][4];
    weight_grad<1>(DZ, H + (kNrcHidden - 1) * kNrcTile * kLd, 0, 16 * warp, lane, acc);
    if (g < kNrcOut) {
      float *dst = gmlp + kNrcHidden * 4096 + g * 64 + 16 * warp + 2 * t;
#pragma unroll
      for (int nt = 0; nt < 2; ++nt) {
        atomicAdd(dst + 8 * nt, acc[nt][0]);
        atomicAdd(dst + 8 * nt + 1, acc[nt][1]);
      }
    }
  }
  float acc[2][8][4];
  data_grad<1, 4>(da, Wo, lane, acc);
  // Hidden layers, last to first.
#pragma unroll 1
  for (int l = kNrcHidden - 1; l >= 0; --l) {
    relu_mask(acc, H + l * kNrcTile * kLd, row0, g, t);
    uint32_t dz[2][4][4];
    acc_to_a(acc, dz, false);
    __syncthreads();  // the previous weight gradient has read DZ
    store_a(dz, DZ, row0, g, t);
    __syncthreads();
    {
      float w[8][4];
      weight_grad<4>(DZ, l > 0 ? H + (l - 1) * kNrcTile * kLd : X, 16 * warp, 0, lane, w);
      float *dst = gmlp + l * 4096 + (16 * warp + g) * 64 + 2 * t;
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) {
        atomicAdd(dst + 8 * nt, w[nt][0]);
        atomicAdd(dst + 8 * nt + 1, w[nt][1]);
        atomicAdd(dst + 8 * 64 + 8 * nt, w[nt][2]);
        atomicAdd(dst + 8 * 64 + 8 * nt + 1, w[nt][3]);
      }
    }
    if (l > 0) data_grad<4, 4>(dz, W + l * 64 * kLd, lane, acc);
    else data_grad<4, 2>(dz, W, lane, acc);  // inputs 0-31: the grid features
  }
  // Grid features: thread (g, t) holds rows g, g + 8 of each m-tile, inputs 8 nt + 2t, + 1 =
  // level 4 nt + t.
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const uint32_t row = base + row0 + 16 * mt + g + 8 * h;
      if (row >= n) continue;
      NrcInput q;
      q.a = __ldg(&in[row].a);
      const float3 pos = nrc_position(G, q);
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
        const uint32_t lev = 4 * nt + t;
        if (lev >= G.levels) continue;
        const float d0 = acc[mt][nt][2 * h], d1 = acc[mt][nt][2 * h + 1];
        if (d0 == 0.0f && d1 == 0.0f) continue;
        uint32_t idx[8];
        float w[8];
        nrc_corners(G, lev, pos, idx, w);
        float2 *dst = gtable + ((size_t)lev << G.logT);
        const uint32_t mask = (1u << G.logT) - 1u;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          if (idx[c] > mask) {
            nrc_fault(G, kNrcBadGradient);
            continue;
          }
          atomicAdd(dst + idx[c], make_float2(w[c] * d0, w[c] * d1));
        }
      }
    }
}

// Adam on params p with moments m, v and gradient sums g (zeroed after use), the batch being
// min(*count, cap) rows; lr already carries the bias corrections. Grid entries (from float4 `dense4`
// on) whose four gradients are all zero are left as they are (lazy Adam, as for embedding tables:
// a step touches a few percent of the hash grid, and the dense update would stream all of it).
__global__ void k_nrc_adam(float4 *__restrict__ p, float4 *__restrict__ m, float4 *__restrict__ v,
                           float4 *__restrict__ gsum, uint64_t n4, uint64_t dense4, const uint32_t *__restrict__ count,
                           uint32_t cap, float lr, float beta1, float beta2, float eps) {
  const uint32_t rows = count ? min(*count, cap) : cap;
  if (rows == 0u) return;
  const float scale = 1.0f / (float(rows) * kNrcLossScale);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n4; i += (uint64_t)gridDim.x * blockDim.x) {
    float4 gg = gsum[i];
    if (i >= dense4 && gg.x == 0.0f && gg.y == 0.0f && gg.z == 0.0f && gg.w == 0.0f) continue;
    float4 mm = m[i], vv = v[i], pp = p[i];
    float *gp = &gg.x, *mp = &mm.x, *vp = &vv.x, *pq = &pp.x;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      float gk = gp[k] * scale;
      if (!isfinite(gk)) gk = 0.0f;
      mp[k] = beta1 * mp[k] + (1.0f - beta1) * gk;
      vp[k] = beta2 * vp[k] + (1.0f - beta2) * gk * gk;
      pq[k] -= lr * mp[k] / (sqrtf(vp[k]) + eps);
    }
    m[i] = mm;
    v[i] = vv;
    p[i] = pp;
    gsum[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  }
}

}  // namespace

// ---- host ------------------------------------------------------------------------------------

namespace {

vt_status nrc_alloc(vt_ctx *ctx, void **p, size_t bytes) {
  VT_CUDA(ctx, cudaMalloc(p, bytes));
  return VT_OK;
}

// The loss normaliser's weights on the four outputs: rgb luminance, or the lanes' mean.
float4 nrc_lum_weights(const vt_nrc *nrc) {
  return nrc->cfg.spectral ? make_float4(0.25f, 0.25f, 0.25f, 0.25f) : make_float4(0.2126f, 0.7152f, 0.0722f, 0.0f);
}

vt_status nrc_check_config(vt_ctx *ctx, const vt_nrc_config &c) {
  if (c.levels < 1 || c.levels > (uint32_t)kNrcMaxLevels) return vt_fail(ctx, VT_ERR_INVALID, "levels must be 1-16");
  if (c.log2_table < 12 || c.log2_table > 24) return vt_fail(ctx, VT_ERR_INVALID, "log2_table must be 12-24");
  if (c.base_resolution < 2 || c.max_resolution < c.base_resolution || c.max_resolution > (1u << 20))
    return vt_fail(ctx, VT_ERR_INVALID, "resolutions must satisfy 2 <= base <= max <= 2^20");
  if (c.train_records == 0 || c.train_records > (1u << 24))
    return vt_fail(ctx, VT_ERR_INVALID, "train_records must be 1 - 2^24");
  if (c.query_vertex == 0 && !(c.spread > 0.0f)) return vt_fail(ctx, VT_ERR_INVALID, "spread must be positive");
  if (c.spectral > 1) return vt_fail(ctx, VT_ERR_INVALID, "spectral must be 0 or 1");
  if (!(c.learning_rate > 0.0f) || !(c.beta1 >= 0.0f && c.beta1 < 1.0f) || !(c.beta2 >= 0.0f && c.beta2 < 1.0f) ||
      !(c.epsilon >= 0.0f))
    return vt_fail(ctx, VT_ERR_INVALID, "bad Adam parameters");
  return VT_OK;
}

}  // namespace

vt_status vt_nrc_reserve_records(vt_ctx *ctx, vt_nrc *nrc, uint32_t n) {
  if (n <= nrc->tcap) return VT_OK;
  cudaFree(nrc->d_tin);
  cudaFree(nrc->d_ttarget);
  nrc->d_tin = nullptr;
  nrc->d_ttarget = nullptr;
  nrc->tcap = 0;
  const uint32_t cap = (n + kNrcTile - 1) / kNrcTile * kNrcTile;
  VT_CUDA(ctx, cudaMalloc(&nrc->d_tin, (size_t)cap * sizeof(NrcInput)));
  VT_CUDA(ctx, cudaMalloc(&nrc->d_ttarget, (size_t)cap * sizeof(float4)));
  nrc->tcap = cap;
  return VT_OK;
}

vt_status vt_nrc_reserve_queries(vt_ctx *ctx, vt_nrc *nrc, size_t n) {
  if (n <= nrc->qcap) return VT_OK;
  cudaFree(nrc->d_q);
  cudaFree(nrc->d_qT);
  cudaFree(nrc->d_qbins);
  cudaFree(nrc->d_qout);
  nrc->d_q = nullptr;
  nrc->d_qT = nullptr;
  nrc->d_qbins = nullptr;
  nrc->d_qout = nullptr;
  nrc->qcap = 0;
  VT_CUDA(ctx, cudaMalloc(&nrc->d_q, n * sizeof(NrcInput)));
  VT_CUDA(ctx, cudaMalloc(&nrc->d_qT, n * sizeof(float4)));
  VT_CUDA(ctx, cudaMalloc(&nrc->d_qbins, n * sizeof(uint2)));
  VT_CUDA(ctx, cudaMalloc(&nrc->d_qout, n * sizeof(float4)));
  nrc->qcap = n;
  return VT_OK;
}

vt_status vt_nrc_step(vt_ctx *ctx, vt_nrc *nrc, uint32_t cap, cudaStream_t s) {
  if (cap == 0) return VT_OK;
  const float *mlp = nrc->d_p;
  float2 *gtable = reinterpret_cast<float2 *>(nrc->d_g + kNrcMlpParams);
  VT_CUDA(ctx, cudaMemsetAsync(nrc->d_loss, 0, sizeof(float), s));
  const uint32_t tiles = (cap + kNrcTile - 1) / kNrcTile;
  k_nrc_train<<<tiles, kNrcTile, kTrainSmem, s>>>(nrc->grid, mlp, nrc->d_tin, nrc->d_ttarget, nrc->d_count, cap,
                                                  nrc->d_g, gtable, nrc->d_loss, nrc_lum_weights(nrc));
  VT_CUDA(ctx, cudaGetLastError());
  ++nrc->steps;
  const double b1 = nrc->cfg.beta1, b2 = nrc->cfg.beta2;
  const double lr = nrc->cfg.learning_rate * std::sqrt(1.0 - std::pow(b2, nrc->steps)) / (1.0 - std::pow(b1, nrc->steps));
  const uint64_t n4 = nrc->nparams / 4;
  const uint32_t blocks = (uint32_t)std::min<uint64_t>((n4 + 255) / 256, (uint64_t)ctx->sm_count * 8u);
  k_nrc_adam<<<blocks, 256, 0, s>>>(reinterpret_cast<float4 *>(nrc->d_p), reinterpret_cast<float4 *>(nrc->d_m),
                                    reinterpret_cast<float4 *>(nrc->d_v), reinterpret_cast<float4 *>(nrc->d_g), n4,
                                    kNrcMlpParams / 4, nrc->d_count, cap, (float)lr, nrc->cfg.beta1, nrc->cfg.beta2,
                                    nrc->cfg.epsilon);
  VT_CUDA(ctx, cudaGetLastError());
  return VT_OK;
}

vt_status vt_nrc_predict(vt_ctx *ctx, vt_nrc *nrc, const NrcInput *in, uint32_t n, float4 *out, cudaStream_t s) {
  return vt_nrc_infer_tc(ctx, nrc, in, n, out, s);
}

extern "C" {

vt_status vt_nrc_config_default(vt_nrc_config *cfg) {
  if (!cfg) return VT_ERR_INVALID;
  std::memset(cfg, 0, sizeof *cfg);
  cfg->levels = 16;
  cfg->log2_table = 19;
  cfg->base_resolution = 16;
  cfg->max_resolution = 2048;
  cfg->train_records = 65536;
  cfg->train_paths = 0;
  cfg->query_vertex = 0;
  cfg->spread = 0.01f;
  cfg->spectral = 0;
  cfg->seed = 1337;
  cfg->learning_rate = 0.01f;
  cfg->beta1 = 0.9f;
  cfg->beta2 = 0.99f;
  cfg->epsilon = 1e-15f;
  return VT_OK;
}

vt_status vt_nrc_create(vt_ctx *ctx, const vt_nrc_config *cfg, const float lo[3], const float hi[3], vt_nrc **out) {
  if (!ctx) return VT_ERR_INVALID;
  if (!out || !lo || !hi) return vt_fail(ctx, VT_ERR_INVALID, "out, lo or hi is null");
  *out = nullptr;
  vt_nrc_config c;
  if (cfg) c = *cfg;
  else vt_nrc_config_default(&c);
  {
    const vt_status st = nrc_check_config(ctx, c);
    if (st != VT_OK) return st;
  }
  for (int k = 0; k < 3; ++k)
    if (!std::isfinite(lo[k]) || !std::isfinite(hi[k]) || !(hi[k] >= lo[k]))
      return vt_fail(ctx, VT_ERR_INVALID, "the cache's box needs finite lo <= hi");
  VT_CUDA(ctx, cudaSetDevice(ctx->device));
  static bool attrs = false;
  if (!attrs) {
    VT_CUDA(ctx, cudaFuncSetAttribute(k_nrc_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrainSmem));
    attrs = true;
  }
  vt_nrc *n = new vt_nrc();
  n->cfg = c;
  NrcGrid &G = n->grid;
  G.levels = c.levels;
  G.logT = c.log2_table;
  // A cube around the box (so that cells stay cubic), 1 % larger.
  float ext = 0.0f;
  for (int k = 0; k < 3; ++k) ext = std::max(ext, hi[k] - lo[k]);
  ext = ext > 0.0f ? ext * 1.02f : 1.0f;
  for (int k = 0; k < 3; ++k) {
    G.lo[k] = 0.5f * (lo[k] + hi[k]) - 0.5f * ext;
    G.inv[k] = 1.0f / ext;
  }
  const double growth = c.levels > 1 ? std::exp((std::log((double)c.max_resolution) - std::log((double)c.base_resolution)) /
                                                (double)(c.levels - 1))
                                     : 1.0;
  G.dense = 0;
  for (uint32_t l = 0; l < (uint32_t)kNrcMaxLevels; ++l) {
    G.res[l] = l < c.levels ? (uint32_t)std::floor((double)c.base_resolution * std::pow(growth, (double)l) + 1e-6) : 1u;
    const uint64_t side = G.res[l] + 1ull;
    if (side * side * side <= (1ull << c.log2_table)) G.dense |= 1u << l;
  }
  n->nparams = (uint64_t)kNrcMlpParams + 2ull * c.levels * (1ull << c.log2_table);
  vt_status st = VT_OK;
  const size_t bytes = n->nparams * sizeof(float);
  if ((st = nrc_alloc(ctx, (void **)&n->d_p, bytes)) != VT_OK || (st = nrc_alloc(ctx, (void **)&n->d_m, bytes)) != VT_OK ||
      (st = nrc_alloc(ctx, (void **)&n->d_v, bytes)) != VT_OK || (st = nrc_alloc(ctx, (void **)&n->d_g, bytes)) != VT_OK ||
      (st = nrc_alloc(ctx, (void **)&n->d_count, 4 * sizeof(uint32_t))) != VT_OK ||
      (st = nrc_alloc(ctx, (void **)&n->d_loss, 4 * sizeof(float))) != VT_OK) {
    vt_nrc_destroy(ctx, n);
    return st;
  }
  G.table = reinterpret_cast<float2 *>(n->d_p + kNrcMlpParams);
  G.status = ctx->d_status + 3;
  {
    cudaError_t e = cudaStreamCreateWithFlags(&n->side, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&n->ev_start, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&n->ev_paths, cudaEventDisableTiming);
    if (e != cudaSuccess) {
      vt_nrc_destroy(ctx, n);
      return vt_cuda_fail(ctx, e, "creating the cache's side stream");
    }
  }
  cudaError_t e = cudaMemsetAsync(n->d_m, 0, bytes, ctx->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(n->d_v, 0, bytes, ctx->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(n->d_g, 0, bytes, ctx->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(n->d_count, 0, 4 * sizeof(uint32_t), ctx->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(n->d_loss, 0, 4 * sizeof(float), ctx->stream);
  if (e == cudaSuccess) {
    k_nrc_init<<<(uint32_t)ctx->sm_count * 8u, 256, 0, ctx->stream>>>(n->d_p, n->nparams, c.seed);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    vt_nrc_destroy(ctx, n);
    return vt_cuda_fail(ctx, e, "initialising the radiance cache");
  }
  *out = n;
  return VT_OK;
}

vt_status vt_nrc_destroy(vt_ctx *ctx, vt_nrc *nrc) {
  if (!nrc) return VT_OK;
  if (ctx) {
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
  }
  cudaDeviceSynchronize();
  for (void *p : {(void *)nrc->d_p, (void *)nrc->d_m, (void *)nrc->d_v, (void *)nrc->d_g, (void *)nrc->d_count,
                  (void *)nrc->d_loss, (void *)nrc->d_tin, (void *)nrc->d_ttarget, (void *)nrc->d_q, (void *)nrc->d_qT,
                  (void *)nrc->d_qbins, (void *)nrc->d_qout, (void *)nrc->d_scratch})
    cudaFree(p);
  if (nrc->ev_start) cudaEventDestroy(nrc->ev_start);
  if (nrc->ev_paths) cudaEventDestroy(nrc->ev_paths);
  if (nrc->side) cudaStreamDestroy(nrc->side);
  delete nrc;
  return VT_OK;
}

vt_status vt_nrc_get_info(vt_ctx *ctx, vt_nrc *nrc, vt_nrc_info *out) {
  if (!ctx) return VT_ERR_INVALID;
  if (!nrc || !out) return vt_fail(ctx, VT_ERR_INVALID, "nrc or out is null");
  VT_CUDA(ctx, cudaSetDevice(ctx->device));
  VT_CUDA(ctx, cudaDeviceSynchronize());
  uint32_t cnt[4];
  float loss[4];
  VT_CUDA(ctx, cudaMemcpy(cnt, nrc->d_count, sizeof cnt, cudaMemcpyDeviceToHost));
  VT_CUDA(ctx, cudaMemcpy(loss, nrc->d_loss, sizeof loss, cudaMemcpyDeviceToHost));
  {
    uint32_t bad = 0;
    VT_CUDA(ctx, cudaMemcpy(&bad, ctx->d_status + 3, sizeof bad, cudaMemcpyDeviceToHost));
    if (bad) {
      VT_CUDA(ctx, cudaMemset(ctx->d_status + 3, 0, sizeof bad));
      return vt_fail(ctx, VT_ERR_DEVICE, "the cache's kernels reported status " + std::to_string(bad) +
                                             " (1, 2: an out-of-range grid index, the access skipped; 4: a tensor-core "
                                             "wait timed out, the inference stopped)");
    }
  }
  std::memset(out, 0, sizeof *out);
  out->mlp_params = kNrcMlpParams;
  out->grid_params = nrc->nparams - kNrcMlpParams;
  out->steps = nrc->steps;
  const uint32_t rec = std::min(cnt[0], cnt[1] ? cnt[1] : cnt[0]);
  out->last_records = rec;
  out->last_loss = rec ? loss[0] / (float)rec : 0.0f;
  return VT_OK;
}

vt_status vt_nrc_get_params(vt_ctx *ctx, const vt_nrc *nrc, float *mlp, float *grid) {
  if (!ctx) return VT_ERR_INVALID;
  if (!nrc || !mlp) return vt_fail(ctx, VT_ERR_INVALID, "nrc or mlp is null");
  VT_CUDA(ctx, cudaSetDevice(ctx->device));
  VT_CUDA(ctx, cudaDeviceSynchronize());
  VT_CUDA(ctx, cudaMemcpy(mlp, nrc->d_p, kNrcMlpParams * sizeof(float), cudaMemcpyDeviceToHost));
  if (grid)
    VT_CUDA(ctx, cudaMemcpy(grid, nrc->d_p + kNrcMlpParams, (nrc->nparams - kNrcMlpParams) * sizeof(float),
                            cudaMemcpyDeviceToHost));
  return VT_OK;
}

vt_status vt_nrc_set_params(vt_ctx *ctx, vt_nrc *nrc, const float *mlp, const float *grid) {
  if (!ctx) return VT_ERR_INVALID;
  if (!nrc || !mlp) return vt_fail(ctx, VT_ERR_INVALID, "nrc or mlp is null");
  VT_CUDA(ctx, cudaSetDevice(ctx->device));
  VT_CUDA(ctx, cudaDeviceSynchronize());
  VT_CUDA(ctx, cudaMemcpy(nrc->d_p, mlp, kNrcMlpParams * sizeof(float), cudaMemcpyHostToDevice));
  if (grid)
    VT_CUDA(ctx, cudaMemcpy(nrc->d_p + kNrcMlpParams, grid, (nrc->nparams - kNrcMlpParams) * sizeof(float),
                            cudaMemcpyHostToDevice));
  const size_t bytes = nrc->nparams * sizeof(float);
  VT_CUDA(ctx, cudaMemset(nrc->d_m, 0, bytes));
  VT_CUDA(ctx, cudaMemset(nrc->d_v, 0, bytes));
  VT_CUDA(ctx, cudaMemset(nrc->d_g, 0, bytes));
  nrc->steps = 0;
  return VT_OK;
}

vt_status vt_nrc_infer(vt_ctx *ctx, vt_nrc *nrc, const vt_nrc_input *in, uint32_t n, float *out) {
  if (!ctx) return VT_ERR_INVALID;
  if (!nrc || ((!in || !out) && n)) return vt_fail(ctx, VT_ERR_INVALID, "nrc, in or out is null");
  if (n == 0) return VT_OK;
  VT_CUDA(ctx, cudaSetDevice(ctx->device));
  {
    const vt_status st = vt_nrc_reserve_queries(ctx, nrc, n);
    if (st != VT_OK) return st;
  }
  VT_CUDA(ctx, cudaMemcpyAsync(nrc->d_q, in, (size_t)n * sizeof(NrcInput), cudaMemcpyHostToDevice, ctx->stream));
  {
    const vt_status st = vt_nrc_predict(ctx, nrc, nrc->d_q, n, nrc->d_qout, ctx->stream);
    if (st != VT_OK) return st;
  }
  VT_CUDA(ctx, cudaMemcpyAsync(out, nrc->d_qout, (size_t)n * sizeof(float4), cudaMemcpyDeviceToHost, ctx->stream));
  VT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return VT_OK;
}

}  // extern "C"

namespace {

// Host records into the training buffers, count = n.
vt_status nrc_upload_records(vt_ctx *ctx, vt_nrc *nrc, const vt_nrc_input *in, const float *target, uint32_t n) {
  {
    const vt_status st = vt_nrc_reserve_records(ctx, nrc, n);
    if (st != VT_OK) return st;
  }
  const uint32_t cnt[4] = {n, n, 0, 0};
  VT_CUDA(ctx, cudaMemcpyAsync(nrc->d_tin, in, (size_t)n * sizeof(NrcInput), cudaMemcpyHostToDevice, ctx->stream));
  VT_CUDA(ctx, cudaMemcpyAsync(nrc->d_ttarget, target, (size_t)n * sizeof(float4), cudaMemcpyHostToDevice, ctx->stream));
  VT_CUDA(ctx, cudaMemcpyAsync(nrc->d_count, cnt, sizeof cnt, cudaMemcpyHostToDevice, ctx->stream));
  VT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return VT_OK;
}

}  // namespace

extern "C" {

vt_status vt_nrc_gradients(vt_ctx *ctx, vt_nrc *nrc, const vt_nrc_input *in, const float *target, uint32_t n,
                           float *mlp_grad, float *grid_grad, double *loss) {
  if (!ctx) return VT_ERR_INVALID;
  if (!nrc || !mlp_grad || ((!in || !target) && n)) return vt_fail(ctx, VT_ERR_INVALID, "null argument");
  if (n > (1u << 24)) return vt_fail(ctx, VT_ERR_LIMIT, "at most 2^24 records");
  VT_CUDA(ctx, cudaSetDevice(ctx->device));
  {
    const vt_status st = nrc_upload_records(ctx, nrc, in, target, n);
    if (st != VT_OK) return st;
  }
  const size_t bytes = nrc->nparams * sizeof(float);
  VT_CUDA(ctx, cudaMemsetAsync(nrc->d_g, 0, bytes, ctx->stream));
  VT_CUDA(ctx, cudaMemsetAsync(nrc->d_loss, 0, sizeof(float), ctx->stream));
  if (n) {
    k_nrc_train<<<(n + kNrcTile - 1) / kNrcTile, kNrcTile, kTrainSmem, ctx->stream>>>(
        nrc->grid, nrc->d_p, nrc->d_tin, nrc->d_ttarget, nrc->d_count, n, nrc->d_g,
        reinterpret_cast<float2 *>(nrc->d_g + kNrcMlpParams), nrc->d_loss, nrc_lum_weights(nrc));
    VT_CUDA(ctx, cudaGetLastError());
  }
  VT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  // The device sums carry the loss scale; the caller gets the loss's own gradient sums.
  VT_CUDA(ctx, cudaMemcpy(mlp_grad, nrc->d_g, kNrcMlpParams * sizeof(float), cudaMemcpyDeviceToHost));
  for (int i = 0; i < kNrcMlpParams; ++i) mlp_grad[i] /= kNrcLossScale;
  if (grid_grad) {
    const size_t ng = nrc->nparams - kNrcMlpParams;
    VT_CUDA(ctx, cudaMemcpy(grid_grad, nrc->d_g + kNrcMlpParams, ng * sizeof(float), cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < ng; ++i) grid_grad[i] /= kNrcLossScale;
  }
  if (loss) {
    float l = 0.0f;
    VT_CUDA(ctx, cudaMemcpy(&l, nrc->d_loss, sizeof l, cudaMemcpyDeviceToHost));
    *loss = l;
  }
  VT_CUDA(ctx, cudaMemset(nrc->d_g, 0, bytes));
  return VT_OK;
}

vt_status vt_nrc_train(vt_ctx *ctx, vt_nrc *nrc, const vt_nrc_input *in, const float *target, uint32_t n, float *loss) {
  if (!ctx) return VT_ERR_INVALID;
  if (!nrc || ((!in || !target) && n)) return vt_fail(ctx, VT_ERR_INVALID, "null argument");
  if (n > (1u << 24)) return vt_fail(ctx, VT_ERR_LIMIT, "at most 2^24 records");
  if (n == 0) return VT_OK;
  VT_CUDA(ctx, cudaSetDevice(ctx->device));
  {
    const vt_status st = nrc_upload_records(ctx, nrc, in, target, n);
    if (st != VT_OK) return st;
  }
  {
    const vt_status st = vt_nrc_step(ctx, nrc, n, ctx->stream);
    if (st != VT_OK) return st;
  }
  VT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (loss) {
    float l = 0.0f;
    VT_CUDA(ctx, cudaMemcpy(&l, nrc->d_loss, sizeof l, cudaMemcpyDeviceToHost));
    *loss = l / (float)n;
  }
  return VT_OK;
}

}  // extern "C"

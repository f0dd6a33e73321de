// qnode.cu — the traversal copy of the 4-wide BVH: 64-byte nodes with 8-bit child boxes.
//
// The reference's MeshWideNode (128 B) stays the exported layout. Traversal reads a quantised copy of
// each node instead (after Ylitie, Karras and Laine, "Efficient Incoherent Ray Traversal on GPUs
// Through Compressed Wide BVHs", HPG 2017, restated for 4 children): the node's box origin p (its
// children's union lower corner), a power-of-two step 2^e per axis, and per child and axis the
// bytes qlo = floor((lo - p) / 2^e) and qhi = ceil((hi - p) / 2^e), so that p + qlo 2^e <= lo and
// p + qhi 2^e >= hi exactly: each decoded box contains the child's box. Child links and leaf counts
// are copied. A node is two 32-byte loads instead of four.
//
// Layout (16 words): p.x p.y p.z | biased exponents (e + 127) in bytes 0-2 | qlo.x qlo.y qlo.z |
// qhi.x qhi.y qhi.z (byte k = child k) | child[4] | leaf counts (4 bits per child) | 0.
#include <cfloat>
#include <cmath>

#include "vt_internal.cuh"

namespace {

// The smallest e in [-126, 112] with 255 * 2^e >= extent (extent in double, exact steps). The
// traversal scales by 2^(e+15), which stays a normal float up to e = 112 (extents below 1e36).
__host__ __device__ inline int quant_exponent(double extent) {
  if (!(extent > 0.0)) return -126;
  int e;
  frexp(extent, &e);
  e -= 8;
  if (e < -126) e = -126;
  if (e > 112) e = 112;
  while (e < 112 && ldexp(255.0, e) < extent) ++e;
  while (e > -126 && ldexp(255.0, e - 1) >= extent) --e;
  return e;
}

__global__ void k_quantize(const vt_wide_node *__restrict__ in, uint32_t n, vt_qnode *__restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const vt_wide_node nd = in[i];
  vt_qnode q;
  for (int w = 0; w < 16; ++w) q.w[w] = 0u;
  float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  bool any = false;
  const float *clo[3] = {nd.lox, nd.loy, nd.loz}, *chi[3] = {nd.hix, nd.hiy, nd.hiz};
  for (int k = 0; k < 4; ++k) {
    if (nd.child[k] == 0) continue;
    any = true;
    for (int a = 0; a < 3; ++a) {
      lo[a] = fminf(lo[a], clo[a][k]);
      hi[a] = fmaxf(hi[a], chi[a][k]);
    }
  }
  if (any) {
    for (int a = 0; a < 3; ++a) {
      const float p = lo[a];
      const int e = quant_exponent((double)hi[a] - (double)p);
      q.w[a] = __float_as_uint(p);
      q.w[3] |= (uint32_t)(e + 127) << (8 * a);
      for (int k = 0; k < 4; ++k) {
        if (nd.child[k] == 0) continue;
        const double l = floor(ldexp((double)clo[a][k] - (double)p, -e));
        const double h = ceil(ldexp((double)chi[a][k] - (double)p, -e));
        const uint32_t ql = (uint32_t)fmin(fmax(l, 0.0), 255.0), qh = (uint32_t)fmin(fmax(h, 0.0), 255.0);
        q.w[4 + a] |= ql << (8 * k);
        q.w[7 + a] |= qh << (8 * k);
      }
    }
  }
  for (int k = 0; k < 4; ++k) {
    q.w[10 + k] = (uint32_t)nd.child[k];
    q.w[14] |= ((uint32_t)nd.count[k] & 15u) << (4 * k);
  }
  out[i] = q;
}

}  // namespace

vt_status vt_quantize_nodes(vt_ctx *ctx, vt_mesh *mesh, cudaStream_t s) {
  cudaFree(mesh->d_qnodes);
  mesh->d_qnodes = nullptr;
  if (mesh->nnodes == 0) return VT_OK;
  VT_CUDA(ctx, cudaMalloc(&mesh->d_qnodes, mesh->nnodes * sizeof(vt_qnode)));
  k_quantize<<<(mesh->nnodes + 255) / 256, 256, 0, s>>>(mesh->d_nodes, mesh->nnodes, mesh->d_qnodes);
  VT_CUDA(ctx, cudaGetLastError());
  return VT_OK;
}

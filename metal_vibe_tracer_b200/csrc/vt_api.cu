// vt_api.cu — the C ABI (include/vt.h): contexts, mesh publish, traversal entry points.
#include <algorithm>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "vt_internal.cuh"

// The error of calls made without a context (context creation, host-only entry points).
thread_local std::string g_no_ctx_error;

vt_status vt_fail(vt_ctx *ctx, vt_status code, const std::string &msg) {
  if (ctx) ctx->error = msg; else g_no_ctx_error = msg;
  return code;
}

vt_status vt_cuda_fail(vt_ctx *ctx, cudaError_t err, const char *what) {
  std::string m = std::string(what) + ": " + cudaGetErrorString(err);
  return vt_fail(ctx, err == cudaErrorMemoryAllocation ? VT_ERR_MEMORY : VT_ERR_CUDA, m);
}

namespace {

void free_mesh(vt_mesh *m) {
  if (!m) return;
  cudaFree(m->d_nodes);
  cudaFree(m->d_tris);
  cudaFree(m->d_order);
  cudaFree(m->d_codes);
  cudaFree(m->d_sorted);
  cudaFree(m->d_bin_child);
  cudaFree(m->d_bin_box);
  cudaFree(m->d_qnodes);
  cudaFree(m->d_nrm);
  delete m;
}

vt_build_options defaults(const vt_build_options *o) {
  vt_build_options r;
  std::memset(&r, 0, sizeof r);
  if (o) r = *o;
  return r;
}

// Device-side copy of the chunk buffers for host pipelining.
vt_status ensure_chunks(vt_ctx *ctx, size_t in_bytes, size_t out_bytes) {
  if (in_bytes > ctx->chunk_in_bytes) {
    for (int k = 0; k < 2; ++k) {
      cudaFree(ctx->d_chunk_in[k]);
      ctx->d_chunk_in[k] = nullptr;
      VT_CUDA(ctx, cudaMalloc(&ctx->d_chunk_in[k], in_bytes));
    }
    ctx->chunk_in_bytes = in_bytes;
  }
  if (out_bytes > ctx->chunk_out_bytes) {
    for (int k = 0; k < 2; ++k) {
      cudaFree(ctx->d_chunk_out[k]);
      ctx->d_chunk_out[k] = nullptr;
      VT_CUDA(ctx, cudaMalloc(&ctx->d_chunk_out[k], out_bytes));
    }
    ctx->chunk_out_bytes = out_bytes;
  }
  return VT_OK;
}

// Ray-ordering scratch of `slot` (0: caller streams, 1-2: the host pipeline's streams).
vt_status order_scratch(vt_ctx *ctx, int slot, uint32_t n, uint32_t **out) {
  size_t words = vt_ray_order_words(n);
  if (words > ctx->order_words[slot]) {
    cudaFree(ctx->d_order[slot]);
    ctx->d_order[slot] = nullptr;
    ctx->order_words[slot] = 0;
    VT_CUDA(ctx, cudaMalloc(&ctx->d_order[slot], words * sizeof(uint32_t)));
    ctx->order_words[slot] = words;
  }
  *out = ctx->d_order[slot];
  return VT_OK;
}

vt_status check_trace_args(vt_ctx *ctx, const vt_mesh *mesh, const void *rays, const void *out, uint32_t n) {
  if (!ctx) return VT_ERR_INVALID;
  if (!mesh) return vt_fail(ctx, VT_ERR_INVALID, "mesh is null");
  if (n > 0 && (!rays || !out)) return vt_fail(ctx, VT_ERR_INVALID, "rays or output is null");
  if (n > 0 && mesh->nfaces > 0 && !mesh->d_nodes) return vt_fail(ctx, VT_ERR_INVALID, "mesh has no nodes");
  // Leaf stack entries hold (node << 2 | slot) in 31 bits.
  if (mesh->nnodes >= (1u << 29)) return vt_fail(ctx, VT_ERR_LIMIT, "traversal supports up to 2^29 - 1 wide nodes");
  return VT_OK;
}

// Chunk of rays per pipeline stage: 2^22 rays = 128 MB in, 64 MB out.
constexpr uint32_t kChunk = 1u << 22;

__global__ void k_fill_miss(int4 *hits, uint32_t n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) hits[i] = make_int4(0, 0, 0, -1);
}

}  // namespace

extern "C" {

uint32_t vt_abi_version(void) { return VT_ABI_VERSION; }

vt_status vt_ctx_create(int32_t device, vt_ctx **out) {
  if (!out) return VT_ERR_INVALID;
  *out = nullptr;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    g_no_ctx_error = std::string("no CUDA device: ") + cudaGetErrorString(e);
    return VT_ERR_CUDA;
  }
  if (device < 0 || device >= count) return VT_ERR_INVALID;
  vt_ctx *c = new vt_ctx();
  c->device = device;
  if ((e = cudaSetDevice(device)) != cudaSuccess ||
      (e = cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess ||
      (e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaStreamCreateWithFlags(&c->pipe[0], cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaStreamCreateWithFlags(&c->pipe[1], cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaEventCreate(&c->ev0)) != cudaSuccess || (e = cudaEventCreate(&c->ev1)) != cudaSuccess ||
      (e = cudaMalloc(&c->d_status, 64)) != cudaSuccess || (e = cudaMalloc(&c->d_counters, kCounterWords * sizeof(uint32_t))) != cudaSuccess) {
    g_no_ctx_error = std::string("context creation: ") + cudaGetErrorString(e);
    vt_ctx_destroy(c);
    return VT_ERR_CUDA;
  }
  cudaMemset(c->d_status, 0, 64);
  *out = c;
  return VT_OK;
}

vt_status vt_ctx_destroy(vt_ctx *ctx) {
  if (!ctx) return VT_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (int k = 0; k < 3; ++k) cudaFree(ctx->d_order[k]);
  for (int k = 0; k < 2; ++k) {
    if (ctx->pipe[k]) cudaStreamSynchronize(ctx->pipe[k]);
    cudaFree(ctx->d_chunk_in[k]);
    cudaFree(ctx->d_chunk_out[k]);
    if (ctx->pipe[k]) cudaStreamDestroy(ctx->pipe[k]);
    cudaFreeHost(ctx->h_stage_in[k]);
    cudaFreeHost(ctx->h_stage_out[k]);
    if (ctx->stage_ev[k]) cudaEventDestroy(ctx->stage_ev[k]);
  }
  cudaFree(ctx->d_status);
  cudaFree(ctx->d_counters);
  cudaFree(ctx->d_fgrid);
  cudaFree(ctx->d_pbr);
  cudaFree(ctx->d_gnodes);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return VT_OK;
}

const char *vt_last_error(const vt_ctx *ctx) { return ctx ? ctx->error.c_str() : g_no_ctx_error.c_str(); }

vt_status vt_sync(vt_ctx *ctx) {
  if (!ctx) return VT_ERR_INVALID;
  VT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return VT_OK;
}

vt_status vt_mesh_build_device(vt_ctx *ctx, const vt_face *faces_dev, uint32_t nfaces,
                               const vt_vertex *verts_dev, uint32_t nverts,
                               const vt_build_options *opts, vt_mesh **out) {
  if (!ctx) return VT_ERR_INVALID;
  if (!out) return vt_fail(ctx, VT_ERR_INVALID, "out is null");
  *out = nullptr;
  if (nfaces > 0 && (!faces_dev || !verts_dev)) return vt_fail(ctx, VT_ERR_INVALID, "faces or vertices is null");
  if (nfaces > (1u << 30)) return vt_fail(ctx, VT_ERR_LIMIT, "more than 2^30 faces");
  VT_CUDA(ctx, cudaSetDevice(ctx->device));
  vt_mesh *m = new vt_mesh();
  vt_build_options o = defaults(opts);
  vt_status st = vt_lbvh_build(ctx, faces_dev, nfaces, verts_dev, nverts, o, m);
  if (st != VT_OK) {
    cudaStreamSynchronize(ctx->stream);
    free_mesh(m);
    return st;
  }
  *out = m;
  return VT_OK;
}

vt_status vt_mesh_build(vt_ctx *ctx, const vt_face *faces, uint32_t nfaces, const vt_vertex *verts,
                        uint32_t nverts, const vt_build_options *opts, vt_mesh **out) {
  if (!ctx) return VT_ERR_INVALID;
  if (nfaces > 0 && (!faces || !verts)) return vt_fail(ctx, VT_ERR_INVALID, "faces or vertices is null");
  VT_CUDA(ctx, cudaSetDevice(ctx->device));
  vt_face *df = nullptr;
  vt_vertex *dv = nullptr;
  if (nfaces > 0) {
    VT_CUDA(ctx, cudaMalloc(&df, (size_t)nfaces * sizeof(vt_face)));
    cudaError_t e = cudaMalloc(&dv, (size_t)(nverts ? nverts : 1) * sizeof(vt_vertex));
    if (e != cudaSuccess) { cudaFree(df); return vt_cuda_fail(ctx, e, "cudaMalloc(vertices)"); }
    e = cudaMemcpyAsync(df, faces, (size_t)nfaces * sizeof(vt_face), cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess && nverts)
      e = cudaMemcpyAsync(dv, verts, (size_t)nverts * sizeof(vt_vertex), cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess) { cudaFree(df); cudaFree(dv); return vt_cuda_fail(ctx, e, "cudaMemcpyAsync(mesh)"); }
  }
  vt_status st = vt_mesh_build_device(ctx, df, nfaces, dv, nverts, opts, out);
  cudaStreamSynchronize(ctx->stream);
  cudaFree(df);
  cudaFree(dv);
  return st;
}

vt_status vt_mesh_destroy(vt_ctx *ctx, vt_mesh *mesh) {
  if (ctx) {
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
  }
  free_mesh(mesh);
  return VT_OK;
}

vt_status vt_mesh_get_info(vt_ctx *ctx, const vt_mesh *mesh, vt_mesh_info *out) {
  if (!ctx) return VT_ERR_INVALID;
  if (!mesh || !out) return vt_fail(ctx, VT_ERR_INVALID, "mesh or out is null");
  out->faces = mesh->nfaces;
  out->wide_nodes = mesh->nnodes;
  out->binary_nodes = mesh->nfaces > 1 ? mesh->nfaces - 1 : 0;
  out->depth = mesh->depth;
  out->sah_cost = mesh->sah;
  out->build_ms = mesh->build_ms;
  for (int k = 0; k < 3; ++k) { out->lo[k] = mesh->lo[k]; out->hi[k] = mesh->hi[k]; }
  return VT_OK;
}

vt_status vt_mesh_get_order(vt_ctx *ctx, const vt_mesh *mesh, int32_t *order, uint32_t n) {
  if (!ctx) return VT_ERR_INVALID;
  if (!mesh || (n && !order)) return vt_fail(ctx, VT_ERR_INVALID, "mesh or order is null");
  if (n != mesh->nfaces) return vt_fail(ctx, VT_ERR_INVALID, "n must equal the face count");
  if (n) VT_CUDA(ctx, cudaMemcpy(order, mesh->d_order, n * sizeof(int32_t), cudaMemcpyDeviceToHost));
  return VT_OK;
}

vt_status vt_mesh_get_nodes(vt_ctx *ctx, const vt_mesh *mesh, vt_wide_node *nodes, uint32_t n) {
  if (!ctx) return VT_ERR_INVALID;
  if (!mesh || (n && !nodes)) return vt_fail(ctx, VT_ERR_INVALID, "mesh or nodes is null");
  if (n != mesh->nnodes) return vt_fail(ctx, VT_ERR_INVALID, "n must equal the wide node count");
  if (n) VT_CUDA(ctx, cudaMemcpy(nodes, mesh->d_nodes, n * sizeof(vt_wide_node), cudaMemcpyDeviceToHost));
  return VT_OK;
}

vt_status vt_mesh_get_morton(vt_ctx *ctx, const vt_mesh *mesh, uint32_t *codes, int32_t *sorted, uint32_t n) {
  if (!ctx) return VT_ERR_INVALID;
  if (!mesh || (n && (!codes || !sorted))) return vt_fail(ctx, VT_ERR_INVALID, "null argument");
  if (n != mesh->nfaces) return vt_fail(ctx, VT_ERR_INVALID, "n must equal the face count");
  if (n) {
    VT_CUDA(ctx, cudaMemcpy(codes, mesh->d_codes, n * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    VT_CUDA(ctx, cudaMemcpy(sorted, mesh->d_sorted, n * sizeof(int32_t), cudaMemcpyDeviceToHost));
  }
  return VT_OK;
}

vt_status vt_mesh_get_binary(vt_ctx *ctx, const vt_mesh *mesh, int32_t *children, float *boxes, uint32_t n) {
  if (!ctx) return VT_ERR_INVALID;
  if (!mesh || (n && (!children || !boxes))) return vt_fail(ctx, VT_ERR_INVALID, "null argument");
  uint32_t expect = mesh->nfaces > 1 ? mesh->nfaces - 1 : 0;
  if (n != expect) return vt_fail(ctx, VT_ERR_INVALID, "n must equal faces - 1");
  if (n) {
    VT_CUDA(ctx, cudaMemcpy(children, mesh->d_bin_child, 2 * (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToHost));
    // Device boxes are (lo xyz, pad, hi xyz, pad); the ABI packs 6 floats.
    float *tmp = new float[8 * (size_t)n];
    cudaError_t e = cudaMemcpy(tmp, mesh->d_bin_box, 8 * (size_t)n * sizeof(float), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) { delete[] tmp; return vt_cuda_fail(ctx, e, "cudaMemcpy(binary boxes)"); }
    for (size_t i = 0; i < n; ++i) {
      boxes[6 * i + 0] = tmp[8 * i + 0]; boxes[6 * i + 1] = tmp[8 * i + 1]; boxes[6 * i + 2] = tmp[8 * i + 2];
      boxes[6 * i + 3] = tmp[8 * i + 4]; boxes[6 * i + 4] = tmp[8 * i + 5]; boxes[6 * i + 5] = tmp[8 * i + 6];
    }
    delete[] tmp;
  }
  return VT_OK;
}

// Shared body of the device-buffer entry points; `slot` picks the ray-ordering scratch.
static vt_status trace_device(vt_ctx *ctx, const vt_mesh *mesh, const vt_ray *rays_dev, uint32_t n, void *out,
                              bool closest, cudaStream_t s, int slot) {
  vt_status st = check_trace_args(ctx, mesh, rays_dev, out, n);
  if (st) return st;
  if (n == 0) return VT_OK;
  if (mesh->nfaces == 0) {
    if (closest) k_fill_miss<<<(n + 255) / 256, 256, 0, s>>>(static_cast<int4 *>(out), n);
    else VT_CUDA(ctx, cudaMemsetAsync(out, 0, n, s));
  } else {
    uint32_t *scratch = nullptr;
    st = order_scratch(ctx, slot, n, &scratch);
    if (st) return st;
    const uint32_t *perm = vt_ray_order(mesh, rays_dev, n, scratch, s);
    if (closest) vt_launch_closest(mesh, rays_dev, n, static_cast<vt_hit *>(out), ctx->sm_count, vt_queue_slot(ctx), perm, ctx->d_status + 1, s);
    else vt_launch_any(mesh, rays_dev, n, static_cast<uint8_t *>(out), ctx->sm_count, vt_queue_slot(ctx), perm, ctx->d_status + 1, s);
  }
  VT_CUDA(ctx, cudaGetLastError());
  return VT_OK;
}

vt_status vt_trace_closest(vt_ctx *ctx, const vt_mesh *mesh, const vt_ray *rays_dev, uint32_t n,
                           vt_hit *hits_dev, void *stream) {
  // NULL stream = the CUDA default stream.
  return trace_device(ctx, mesh, rays_dev, n, hits_dev, true, static_cast<cudaStream_t>(stream), 0);
}

vt_status vt_trace_any(vt_ctx *ctx, const vt_mesh *mesh, const vt_ray *rays_dev, uint32_t n,
                       uint8_t *occluded_dev, void *stream) {
  return trace_device(ctx, mesh, rays_dev, n, occluded_dev, false, static_cast<cudaStream_t>(stream), 0);
}

// Pinned staging buffers for pageable callers (two slots, grown as needed) and their events.
static vt_status ensure_stage(vt_ctx *ctx, size_t in_bytes, size_t out_bytes) {
  for (int k = 0; k < 2; ++k)
    if (!ctx->stage_ev[k]) VT_CUDA(ctx, cudaEventCreateWithFlags(&ctx->stage_ev[k], cudaEventDisableTiming));
  if (in_bytes > ctx->stage_in_bytes) {
    for (int k = 0; k < 2; ++k) {
      cudaFreeHost(ctx->h_stage_in[k]);
      ctx->h_stage_in[k] = nullptr;
      VT_CUDA(ctx, cudaMallocHost(&ctx->h_stage_in[k], in_bytes));
    }
    ctx->stage_in_bytes = in_bytes;
  }
  if (out_bytes > ctx->stage_out_bytes) {
    for (int k = 0; k < 2; ++k) {
      cudaFreeHost(ctx->h_stage_out[k]);
      ctx->h_stage_out[k] = nullptr;
      VT_CUDA(ctx, cudaMallocHost(&ctx->h_stage_out[k], out_bytes));
    }
    ctx->stage_out_bytes = out_bytes;
  }
  return VT_OK;
}

// A host copy split over a few threads: one core's copy bandwidth would otherwise bound a pageable
// caller's throughput.
static void copy_parallel(void *dst, const void *src, size_t bytes) {
  const size_t hw = std::max(1u, std::thread::hardware_concurrency());
  const size_t parts = std::min<size_t>(std::min<size_t>(8, hw), std::max<size_t>(1, bytes >> 22));
  if (parts <= 1) {
    std::memcpy(dst, src, bytes);
    return;
  }
  const size_t step = (bytes + parts - 1) / parts;
  std::vector<std::thread> workers;
  for (size_t p = 1; p < parts; ++p) {
    const size_t off = p * step;
    if (off >= bytes) break;
    workers.emplace_back([=] { std::memcpy(static_cast<char *>(dst) + off, static_cast<const char *>(src) + off, std::min(step, bytes - off)); });
  }
  std::memcpy(dst, src, std::min(step, bytes));
  for (auto &w : workers) w.join();
}

// Whether a host pointer is ordinary (pageable) memory rather than pinned or registered memory.
static bool pageable(const void *p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return true;
  }
  return a.type == cudaMemoryTypeUnregistered;
}

// Host pipeline: chunk c goes on stream c % 2 as copy-in, trace, copy-out; the two streams let
// chunk c + 1's copy-in and chunk c - 1's copy-out overlap chunk c's traversal. Pageable buffers go
// through pinned staging: while the GPU works on chunk c - 1, the host copies chunk c - 2's hits out
// and chunk c's rays in (so the driver's synchronous staging never serialises the pipeline).
static vt_status trace_host(vt_ctx *ctx, const vt_mesh *mesh, const vt_ray *rays, uint32_t n,
                            void *out, size_t out_stride, bool closest) {
  vt_status st = check_trace_args(ctx, mesh, rays, out, n);
  if (st) return st;
  VT_CUDA(ctx, cudaSetDevice(ctx->device));
  if (n == 0) return VT_OK;
  const uint32_t chunk = n < kChunk ? n : kChunk;
  st = ensure_chunks(ctx, (size_t)chunk * sizeof(vt_ray), (size_t)chunk * out_stride);
  if (st) return st;
  // The previous user of these buffers may still be in flight on the other stream.
  VT_CUDA(ctx, cudaStreamSynchronize(ctx->pipe[0]));
  VT_CUDA(ctx, cudaStreamSynchronize(ctx->pipe[1]));
  if (pageable(rays) || pageable(out)) {
    st = ensure_stage(ctx, (size_t)chunk * sizeof(vt_ray), (size_t)chunk * out_stride);
    if (st) return st;
    const uint32_t nchunks = (n + chunk - 1) / chunk;
    auto copy_out = [&](uint32_t c) -> vt_status {
      const int k = c & 1;
      const uint32_t first = c * chunk, m = n - first < chunk ? n - first : chunk;
      VT_CUDA(ctx, cudaEventSynchronize(ctx->stage_ev[k]));
      copy_parallel(static_cast<char *>(out) + (size_t)first * out_stride, ctx->h_stage_out[k], (size_t)m * out_stride);
      return VT_OK;
    };
    for (uint32_t c = 0; c < nchunks; ++c) {
      const int k = c & 1;
      const uint32_t first = c * chunk, m = n - first < chunk ? n - first : chunk;
      if (c >= 2) {  // staging slot k held chunk c - 2: its hits out first
        st = copy_out(c - 2);
        if (st) return st;
      }
      copy_parallel(ctx->h_stage_in[k], rays + first, (size_t)m * sizeof(vt_ray));
      cudaStream_t s = ctx->pipe[k];
      VT_CUDA(ctx, cudaMemcpyAsync(ctx->d_chunk_in[k], ctx->h_stage_in[k], (size_t)m * sizeof(vt_ray), cudaMemcpyHostToDevice, s));
      st = trace_device(ctx, mesh, static_cast<const vt_ray *>(ctx->d_chunk_in[k]), m, ctx->d_chunk_out[k], closest, s, 1 + k);
      if (st) return st;
      VT_CUDA(ctx, cudaMemcpyAsync(ctx->h_stage_out[k], ctx->d_chunk_out[k], (size_t)m * out_stride, cudaMemcpyDeviceToHost, s));
      VT_CUDA(ctx, cudaEventRecord(ctx->stage_ev[k], s));
    }
    for (uint32_t c = nchunks >= 2 ? nchunks - 2 : 0; c < nchunks; ++c) {
      st = copy_out(c);
      if (st) return st;
    }
    return VT_OK;
  }
  for (uint32_t c = 0, first = 0; first < n; ++c, first += chunk) {
    const uint32_t m = n - first < chunk ? n - first : chunk;
    const int k = c & 1;
    cudaStream_t s = ctx->pipe[k];
    VT_CUDA(ctx, cudaMemcpyAsync(ctx->d_chunk_in[k], rays + first, (size_t)m * sizeof(vt_ray),
                                 cudaMemcpyHostToDevice, s));
    const vt_ray *dr = static_cast<const vt_ray *>(ctx->d_chunk_in[k]);
    st = trace_device(ctx, mesh, dr, m, ctx->d_chunk_out[k], closest, s, 1 + k);
    if (st) return st;
    VT_CUDA(ctx, cudaMemcpyAsync(static_cast<char *>(out) + (size_t)first * out_stride, ctx->d_chunk_out[k],
                                 (size_t)m * out_stride, cudaMemcpyDeviceToHost, s));
  }
  VT_CUDA(ctx, cudaStreamSynchronize(ctx->pipe[0]));
  VT_CUDA(ctx, cudaStreamSynchronize(ctx->pipe[1]));
  return VT_OK;
}

vt_status vt_trace_closest_host(vt_ctx *ctx, const vt_mesh *mesh, const vt_ray *rays, uint32_t n,
                                vt_hit *hits) {
  return trace_host(ctx, mesh, rays, n, hits, sizeof(vt_hit), true);
}

vt_status vt_trace_any_host(vt_ctx *ctx, const vt_mesh *mesh, const vt_ray *rays, uint32_t n,
                            uint8_t *occluded) {
  return trace_host(ctx, mesh, rays, n, occluded, 1, false);
}

vt_status vt_trace_count(vt_ctx *ctx, const vt_mesh *mesh, const vt_ray *rays_dev, uint32_t n,
                         int32_t closest, uint64_t *nodes_visited, uint64_t *tris_tested) {
  vt_status st = check_trace_args(ctx, mesh, rays_dev, nodes_visited, n);
  if (st) return st;
  if (!tris_tested) return vt_fail(ctx, VT_ERR_INVALID, "tris_tested is null");
  *nodes_visited = 0;
  *tris_tested = 0;
  if (n == 0 || mesh->nfaces == 0) return VT_OK;
  unsigned long long *acc = vt_count_words(ctx);
  VT_CUDA(ctx, cudaMemsetAsync(acc, 0, 2 * sizeof(unsigned long long), ctx->stream));
  vt_launch_count(mesh, rays_dev, n, closest, acc, ctx->stream);
  VT_CUDA(ctx, cudaGetLastError());
  unsigned long long h[2];
  VT_CUDA(ctx, cudaMemcpyAsync(h, acc, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
  VT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  *nodes_visited = h[0];
  *tris_tested = h[1];
  return VT_OK;
}

}  // extern "C"

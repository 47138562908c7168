// pstm_migrate_noalloc: forward migration + fold that performs no device
// allocation.  Its scratch (grid-local geometry, per-tile trace lists, staged
// trace rows, error flag) lives in one file-scope __device__ array of
// PSTM_NOALLOC_SCRATCH_BYTES, which every GPU that loads the library holds
// until the process exits.
//
// Who needs it: callers that must not allocate device memory while they run --
// for example a process whose caching allocator (PyTorch's, or a host
// application's memory pool) already owns the device's free memory, a real-time
// path that cannot afford the device-wide synchronisation that cudaFree
// implies, or code that issues work where allocation is not permitted.
//
// The host-side symbol of the array is only a stand-in for the device object:
// its device address is obtained once per device with cudaGetSymbolAddress
// (with that device current) and passed to the kernels; the first call on a
// device performs that lookup.  Every call reads the device error flag back
// and synchronises its stream, so the call cannot be captured in a CUDA graph.
// All calls share the one array and it keeps the previous call's contents;
// everything that must start at zero (the error flag) is cleared on each call,
// and calls whose work overlaps on the GPU race on the array.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>

#include "pstm_common.cuh"
#include "pstm_internal.h"

static __device__ __align__(256) unsigned char g_noalloc_scratch[PSTM_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
unsigned char* g_scratch_addr[kMaxDevices] = {nullptr};
pstm_status noalloc_fail(pstm_status st, const std::string& msg) {
  pstm::set_last_error(msg);
  return st;
}

// Device address of the scratch array on the current device (looked up once).
pstm_status scratch_for_current_device(unsigned char** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return noalloc_fail(PSTM_ECUDA, cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return noalloc_fail(PSTM_EINVAL, "device index out of range");
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    unsigned char* ptr = nullptr;
    e = cudaGetSymbolAddress(reinterpret_cast<void**>(&ptr), g_noalloc_scratch);
    if (e != cudaSuccess)
      return noalloc_fail(PSTM_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_scratch_addr[dev] = ptr;
  }
  *out = g_scratch_addr[dev];
  return PSTM_OK;
}

struct DiscGrid {
  int n_il, n_xl, tile_il, tile_xl, tiles_xl;
  float il_dx, il_dy, xl_dx, xl_dy, reach;
};

// Squared cull radius around the tile centre: both legs of a contributing trace
// lie within the aperture of some column, hence within aperture + tile radius
// (plus a rounding margin) of the centre.
__device__ void noalloc_tile_disc(const DiscGrid& g, int tile, float& cx, float& cy, float& r2) {
  const int ti = tile / g.tiles_xl, tx = tile - ti * g.tiles_xl;
  const int i0 = ti * g.tile_il, i1 = min(i0 + g.tile_il, g.n_il) - 1;
  const int x0 = tx * g.tile_xl, x1 = min(x0 + g.tile_xl, g.n_xl) - 1;
  const float ax = i0 * g.il_dx + x0 * g.xl_dx, ay = i0 * g.il_dy + x0 * g.xl_dy;
  const float bx = i1 * g.il_dx + x1 * g.xl_dx, by = i1 * g.il_dy + x1 * g.xl_dy;
  const float px = i1 * g.il_dx + x0 * g.xl_dx, py = i1 * g.il_dy + x0 * g.xl_dy;
  const float qx = i0 * g.il_dx + x1 * g.xl_dx, qy = i0 * g.il_dy + x1 * g.xl_dy;
  cx = 0.25f * (ax + bx + px + qx);
  cy = 0.25f * (ay + by + py + qy);
  float R = fmaxf(fmaxf(hypotf(ax - cx, ay - cy), hypotf(bx - cx, by - cy)),
                  fmaxf(hypotf(px - cx, py - cy), hypotf(qx - cx, qy - cy)));
  const float reach = (g.reach + R) * 1.0001f + 1.0f;
  r2 = reach * reach;
}

__device__ __forceinline__ bool noalloc_in_disc(float4 t, float cx, float cy, float r2) {
  const float a = t.x - cx, b = t.y - cy, c = t.z - cx, d = t.w - cy;
  return (a * a + b * b < r2) && (c * c + d * d < r2);
}

// Grid-local coordinates (origin subtracted in float64).  A non-finite
// coordinate raises PSTM_ERR_COORDS, which the entry point reports as
// PSTM_EINVAL, as the plan path rejects such geometry.
template <typename C>
__global__ void noalloc_geo_kernel(const C* sx, const C* sy, const C* rx, const C* ry, int n,
                                   double ox, double oy, float4* geo, int* err) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const float4 g = make_float4((float)((double)sx[j] - ox), (float)((double)sy[j] - oy),
                               (float)((double)rx[j] - ox), (float)((double)ry[j] - oy));
  if (!(isfinite(g.x) && isfinite(g.y) && isfinite(g.z) && isfinite(g.w)))
    atomicOr(err, PSTM_ERR_COORDS);
  geo[j] = g;
}

__global__ void __launch_bounds__(256) noalloc_count_kernel(DiscGrid g, const float4* geo, int n,
                                                            int64_t* counts) {
  float cx, cy, r2;
  noalloc_tile_disc(g, blockIdx.x, cx, cy, r2);
  int cnt = 0;
  for (int j = threadIdx.x; j < n; j += blockDim.x) cnt += noalloc_in_disc(geo[j], cx, cy, r2);
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
  __shared__ int part[8];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = cnt;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int w = 0; w < 8; ++w) t += part[w];
    counts[blockIdx.x] = t;
  }
}

// Exclusive prefix over n_tiles counts in one CTA; off has n_tiles + 1 entries.
__global__ void __launch_bounds__(1024) noalloc_scan_kernel(const int64_t* counts, int n_tiles,
                                                            int64_t* off) {
  __shared__ int64_t carry;
  __shared__ int64_t warp_sum[32];
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int base = 0; base < n_tiles; base += 1024) {
    const int i = base + threadIdx.x;
    int64_t v = i < n_tiles ? counts[i] : 0;
    int64_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t u = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += u;
    }
    if (lane == 31) warp_sum[w] = x;
    __syncthreads();
    if (w == 0) {
      int64_t y = warp_sum[lane];
      for (int o = 1; o < 32; o <<= 1) {
        const int64_t u = __shfl_up_sync(0xffffffffu, y, o);
        if (lane >= o) y += u;
      }
      warp_sum[lane] = y;
    }
    __syncthreads();
    const int64_t incl = x + (w > 0 ? warp_sum[w - 1] : 0) + carry;
    if (i < n_tiles) off[i] = incl - v;
    __syncthreads();
    if (threadIdx.x == 1023) carry = incl;
    __syncthreads();
  }
  if (threadIdx.x == 0) off[n_tiles] = carry;
}

__global__ void __launch_bounds__(256) noalloc_fill_kernel(DiscGrid g, const float4* geo, int n,
                                                           const int64_t* off, int* list) {
  float cx, cy, r2;
  noalloc_tile_disc(g, blockIdx.x, cx, cy, r2);
  __shared__ int part[8];
  __shared__ int total;
  int64_t base = off[blockIdx.x];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int j0 = 0; j0 < n; j0 += 256) {
    const int j = j0 + threadIdx.x;
    const bool f = j < n && noalloc_in_disc(geo[j], cx, cy, r2);
    const unsigned m = __ballot_sync(0xffffffffu, f);
    if (lane == 0) part[w] = __popc(m);
    __syncthreads();
    int before = 0, tot = 0;
    for (int q = 0; q < 8; ++q) {
      before += q < w ? part[q] : 0;
      tot += part[q];
    }
    if (f) list[base + before + __popc(m & ((1u << lane) - 1u))] = j;
    if (threadIdx.x == 0) total = tot;
    __syncthreads();
    base += total;
    __syncthreads();
  }
}

// (n_s, n) sample-major -> trace-major rows of stride S, same trace order.
__global__ void noalloc_stage_kernel(const float* tr, int n, int n_s, int S, float* rows) {
  __shared__ float t[32][33];
  const int j0 = blockIdx.x * 32, i0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int i = i0 + r, j = j0 + threadIdx.x;
    t[r][threadIdx.x] = (i < n_s && j < n) ? tr[(int64_t)i * n + j] : 0.f;
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int j = j0 + r, i = i0 + threadIdx.x;
    if (j < n && i < S) rows[(int64_t)j * S + i] = i < n_s ? t[threadIdx.x][r] : 0.f;
  }
}

size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

}  // namespace

extern "C" pstm_status pstm_migrate_noalloc(const pstm_grid* grid, const pstm_params* params,
                                            const pstm_geometry* geometry, const float* traces,
                                            const float* velocity, int64_t v_stride_t,
                                            int64_t v_stride_c, float* image, float* fold,
                                            void* stream) {
  using namespace pstm;
  if (!grid || !params || !geometry || !image || !velocity)
    return noalloc_fail(PSTM_EINVAL, "null argument");
  if (grid->n_il < 1 || grid->n_xl < 1 || grid->n_times < 1 || !(grid->dt_ms > 0) ||
      params->n_samples < 2 || !(params->in_dt_ms > 0) || !(params->max_aperture_m > 0) ||
      !(params->max_angle_deg > 0 && params->max_angle_deg <= 90) || params->weight < 0 ||
      params->weight > 3 || params->clamp < 0 || params->clamp > 1 || v_stride_t < 0 ||
      v_stride_c < 0)
    return noalloc_fail(PSTM_EINVAL, "invalid grid or migration parameters");
  if (params->storage != PSTM_F32 || params->antialias)
    return noalloc_fail(PSTM_EINVAL, "the no-allocation entry point stages float32 traces only");
  if (params->taper_width != 0.0 || params->ray_gradient != 0.0)
    return noalloc_fail(PSTM_EINVAL, "the no-allocation entry point applies no aperture taper "
                                     "or curved rays");
  if (geometry->coord_dtype != PSTM_F32 && geometry->coord_dtype != PSTM_F64)
    return noalloc_fail(PSTM_EINVAL, "coordinates must be F32 or F64");
  const int64_t n = geometry->n_traces;
  if (n < 0 || n > (1 << 24)) return noalloc_fail(PSTM_EINVAL, "n_traces out of range");
  if (n > 0 && (!traces || !geometry->source_x || !geometry->source_y || !geometry->receiver_x ||
                !geometry->receiver_y))
    return noalloc_fail(PSTM_EINVAL, "null trace or coordinate pointer");

  Plan p;  // lives on the host stack; every device pointer below is into the scratch array
  p.grid = *grid;
  p.params = *params;
  p.n_traces = n;
  p.n_samples = params->n_samples;
  p.row_stride = (params->n_samples + 7) / 8 * 8;
  p.elt_bytes = 4;
  if (!shape_for_variant(params->variant, grid->n_xl, grid->n_times, &p.shape))
    return noalloc_fail(PSTM_EINVAL, "unknown kernel variant");
  p.tiles_il = (grid->n_il + p.shape.tile_il - 1) / p.shape.tile_il;
  p.tiles_xl = (grid->n_xl + p.shape.tile_xl - 1) / p.shape.tile_xl;
  p.n_tiles = (int64_t)p.tiles_il * p.tiles_xl;
  p.n_windows = (grid->n_times + p.shape.t_window() - 1) / p.shape.t_window();
  if (p.n_tiles > INT32_MAX || p.n_windows > 65535)
    return noalloc_fail(PSTM_EINVAL, "grid too large");
  p.il_dx = (float)grid->il_dx;
  p.il_dy = (float)grid->il_dy;
  p.xl_dx = (float)grid->xl_dx;
  p.xl_dy = (float)grid->xl_dy;
  p.tan_theta = (float)std::tan(params->max_angle_deg * M_PI / 180.0);
  if (forward_smem_bytes(&p) > forward_smem_budget(&p))
    return noalloc_fail(PSTM_EINVAL, "traces too long for the staged kernel");

  // scratch layout (worst case: every trace listed for every tile)
  const size_t o_err = 0;
  const size_t o_geo = align256(o_err + sizeof(int));
  const size_t o_cnt = align256(o_geo + (size_t)n * sizeof(float4));
  const size_t o_off = align256(o_cnt + (size_t)(p.n_tiles + 1) * sizeof(int64_t));
  const size_t o_list = align256(o_off + (size_t)(p.n_tiles + 1) * sizeof(int64_t));
  const size_t o_rows = align256(o_list + (size_t)p.n_tiles * n * sizeof(int));
  const size_t need = o_rows + (size_t)n * p.row_stride * sizeof(float);
  if (need > PSTM_NOALLOC_SCRATCH_BYTES)
    return noalloc_fail(PSTM_EINVAL,
                        "problem needs " + std::to_string(need) + " bytes of scratch; the "
                        "no-allocation entry point holds " +
                            std::to_string((size_t)PSTM_NOALLOC_SCRATCH_BYTES) + " bytes");
  unsigned char* base = nullptr;
  pstm_status st = scratch_for_current_device(&base);
  if (st != PSTM_OK) return st;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  p.err = reinterpret_cast<int*>(base + o_err);
  p.geo = reinterpret_cast<float4*>(base + o_geo);
  int64_t* counts = reinterpret_cast<int64_t*>(base + o_cnt);
  p.tile_off = reinterpret_cast<int64_t*>(base + o_off);
  p.tile_list = reinterpret_cast<int*>(base + o_list);
  p.traces = base + o_rows;
  p.scales = nullptr;
  p.traces_loaded = true;

  auto launched = [&](const char* what) -> pstm_status {
    count_launch();
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PSTM_OK
                            : noalloc_fail(PSTM_ECUDA, std::string(what) + ": " +
                                                           cudaGetErrorString(e));
  };
  cudaError_t e = cudaMemsetAsync(p.err, 0, sizeof(int), s);
  if (e != cudaSuccess) return noalloc_fail(PSTM_ECUDA, cudaGetErrorString(e));
  DiscGrid dg{grid->n_il, grid->n_xl, p.shape.tile_il, p.shape.tile_xl, p.tiles_xl,
              p.il_dx, p.il_dy, p.xl_dx, p.xl_dy, (float)params->max_aperture_m};
  if (n > 0) {
    const unsigned nb = (unsigned)((n + 255) / 256);
    if (geometry->coord_dtype == PSTM_F64)
      noalloc_geo_kernel<double><<<nb, 256, 0, s>>>(
          (const double*)geometry->source_x, (const double*)geometry->source_y,
          (const double*)geometry->receiver_x, (const double*)geometry->receiver_y, (int)n,
          grid->origin_x, grid->origin_y, p.geo, p.err);
    else
      noalloc_geo_kernel<float><<<nb, 256, 0, s>>>(
          (const float*)geometry->source_x, (const float*)geometry->source_y,
          (const float*)geometry->receiver_x, (const float*)geometry->receiver_y, (int)n,
          grid->origin_x, grid->origin_y, p.geo, p.err);
    if ((st = launched("noalloc_geo_kernel")) != PSTM_OK) return st;
  }
  noalloc_count_kernel<<<(unsigned)p.n_tiles, 256, 0, s>>>(dg, p.geo, (int)n, counts);
  if ((st = launched("noalloc_count_kernel")) != PSTM_OK) return st;
  noalloc_scan_kernel<<<1, 1024, 0, s>>>(counts, (int)p.n_tiles, p.tile_off);
  if ((st = launched("noalloc_scan_kernel")) != PSTM_OK) return st;
  if (n > 0) {
    noalloc_fill_kernel<<<(unsigned)p.n_tiles, 256, 0, s>>>(dg, p.geo, (int)n, p.tile_off,
                                                            p.tile_list);
    if ((st = launched("noalloc_fill_kernel")) != PSTM_OK) return st;
    dim3 tb(32, 8), tg((unsigned)((n + 31) / 32), (unsigned)((p.row_stride + 31) / 32));
    noalloc_stage_kernel<<<tg, tb, 0, s>>>(traces, (int)n, p.n_samples, p.row_stride,
                                           reinterpret_cast<float*>(p.traces));
    if ((st = launched("noalloc_stage_kernel")) != PSTM_OK) return st;
  }
  std::string why;
  if ((st = launch_velocity_check(&p, velocity, v_stride_t, v_stride_c, s, &why)) != PSTM_OK)
    return noalloc_fail(st, why);
  // the fold (when asked for) is counted in the forward launch, as pstm_migrate does
  if ((st = launch_forward(&p, velocity, v_stride_t, v_stride_c, image, fold, s, &why)) !=
      PSTM_OK)
    return noalloc_fail(st, why);
  int flags = 0;
  e = cudaMemcpyAsync(&flags, p.err, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return noalloc_fail(PSTM_ECUDA, cudaGetErrorString(e));
  if (flags & PSTM_ERR_TIMEOUT)
    return noalloc_fail(PSTM_ETIMEOUT, "a bounded device-side wait for a trace copy expired");
  if (flags & PSTM_ERR_COORDS) return noalloc_fail(PSTM_EINVAL, "non-finite trace coordinates");
  if (flags & PSTM_ERR_VELOCITY)
    return noalloc_fail(PSTM_EINVAL,
                        "velocity must be positive and finite with V*t0 non-decreasing in t0");
  if (flags) return noalloc_fail(PSTM_EBOUNDS, "device-side check fired");
  return PSTM_OK;
}

// Plan construction (geometry binning, spatial sort, per-tile trace lists),
// trace staging into the sorted device copy, and the C ABI entry points.
#include <cuda_runtime.h>
#include <cub/cub.cuh>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <mutex>
#include <string>
#include <vector>

#include "pstm_common.cuh"
#include "pstm_internal.h"

namespace pstm {
int64_t launch_total();
}

using namespace pstm;

static thread_local std::string g_last_error;

static pstm_status fail(pstm_status st, const std::string& msg) {
  g_last_error = msg;
  return st;
}

void pstm::set_last_error(const std::string& msg) { g_last_error = msg; }

#define CUDA_TRY(expr)                                                               \
  do {                                                                               \
    cudaError_t _e = (expr);                                                         \
    if (_e != cudaSuccess)                                                           \
      return fail(_e == cudaErrorMemoryAllocation ? PSTM_ENOMEM : PSTM_ECUDA,        \
                  std::string(#expr) + ": " + cudaGetErrorString(_e));               \
  } while (0)

#define LAUNCH_CHECK(name)                                                           \
  do {                                                                               \
    count_launch();                                                                  \
    cudaError_t _e = cudaGetLastError();                                             \
    if (_e != cudaSuccess)                                                           \
      return fail(PSTM_ECUDA, std::string(name) + ": " + cudaGetErrorString(_e));    \
  } while (0)

// ------------------------------------------------------------------ kernels ---

// World -> grid-local float32 (origin subtracted in float64), plus midpoints.
template <typename C>
__global__ void geo_local_kernel(const C* sx, const C* sy, const C* rx, const C* ry, int64_t n,
                                 double ox, double oy, float4* geo, float2* mid) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const float a = (float)((double)sx[j] - ox), b = (float)((double)sy[j] - oy);
  const float c = (float)((double)rx[j] - ox), d = (float)((double)ry[j] - oy);
  geo[j] = make_float4(a, b, c, d);
  mid[j] = make_float2(0.5f * (a + c), 0.5f * (b + d));
}

__device__ __forceinline__ int ord_of(float f) {
  const int i = __float_as_int(f);
  return i >= 0 ? i : i ^ 0x7fffffff;
}
__device__ __forceinline__ float float_of_ord(int i) {
  return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff);
}

// bbox[0..3] = ord(min x), ord(min y), ord(max x), ord(max y)
__global__ void bbox_kernel(const float2* mid, int64_t n, int* bbox) {
  float mnx = 3e38f, mny = 3e38f, mxx = -3e38f, mxy = -3e38f;
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n;
       j += (int64_t)gridDim.x * blockDim.x) {
    const float2 m = mid[j];
    mnx = fminf(mnx, m.x);
    mny = fminf(mny, m.y);
    mxx = fmaxf(mxx, m.x);
    mxy = fmaxf(mxy, m.y);
  }
  for (int o = 16; o > 0; o >>= 1) {
    mnx = fminf(mnx, __shfl_xor_sync(0xffffffffu, mnx, o));
    mny = fminf(mny, __shfl_xor_sync(0xffffffffu, mny, o));
    mxx = fmaxf(mxx, __shfl_xor_sync(0xffffffffu, mxx, o));
    mxy = fmaxf(mxy, __shfl_xor_sync(0xffffffffu, mxy, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(bbox + 0, ord_of(mnx));
    atomicMin(bbox + 1, ord_of(mny));
    atomicMax(bbox + 2, ord_of(mxx));
    atomicMax(bbox + 3, ord_of(mxy));
  }
}

__global__ void bbox_init_kernel(int* bbox) {
  bbox[0] = ord_of(3e38f);
  bbox[1] = ord_of(3e38f);
  bbox[2] = ord_of(-3e38f);
  bbox[3] = ord_of(-3e38f);
}

struct CellGrid {
  float x0, y0, cs;
  int ncx, ncy;
};

__global__ void cell_key_kernel(const float2* mid, int64_t n, CellGrid cg, int* key, int* iota) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const float2 m = mid[j];
  int cx = (int)floorf((m.x - cg.x0) / cg.cs);
  int cy = (int)floorf((m.y - cg.y0) / cg.cs);
  cx = min(max(cx, 0), cg.ncx - 1);
  cy = min(max(cy, 0), cg.ncy - 1);
  key[j] = cy * cg.ncx + cx;
  iota[j] = (int)j;
}

// cell_start[c] = first sorted position with key >= c (c = 0..n_cells)
__global__ void cell_start_kernel(const int* keys_sorted, int64_t n, int n_cells,
                                  int64_t* cell_start) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c > n_cells) return;
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (keys_sorted[mid] < c)
      lo = mid + 1;
    else
      hi = mid;
  }
  cell_start[c] = lo;
}

__global__ void gather_geo_kernel(const float4* geo_u, const int* perm, int64_t n, float4* geo,
                                  int* inv_perm) {
  const int64_t jj = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (jj >= n) return;
  const int j = perm[jj];
  geo[jj] = geo_u[j];
  inv_perm[j] = (int)jj;
}

struct TileGeom {
  int n_il, n_xl, tile_il, tile_xl, tiles_xl;
  float il_dx, il_dy, xl_dx, xl_dy;
  float reach;  // aperture (m)
};

// Tile centre and the squared cull radius: a trace can contribute to a column
// of the tile only if both of its legs lie within A of that column, hence within
// A + R of the centre (R = distance from the centre to the farthest corner).
__device__ __forceinline__ void tile_disc(const TileGeom& tg, int tile, float& cx, float& cy,
                                          float& r2, float& rad) {
  const int ti = tile / tg.tiles_xl, tx = tile - ti * tg.tiles_xl;
  const int il0 = ti * tg.tile_il, il1 = min(il0 + tg.tile_il, tg.n_il) - 1;
  const int xl0 = tx * tg.tile_xl, xl1 = min(xl0 + tg.tile_xl, tg.n_xl) - 1;
  float px[4], py[4];
  const int ils[4] = {il0, il1, il0, il1}, xls[4] = {xl0, xl0, xl1, xl1};
  cx = cy = 0.f;
  for (int q = 0; q < 4; ++q) {
    px[q] = ils[q] * tg.il_dx + xls[q] * tg.xl_dx;
    py[q] = ils[q] * tg.il_dy + xls[q] * tg.xl_dy;
    cx += 0.25f * px[q];
    cy += 0.25f * py[q];
  }
  float R = 0.f;
  for (int q = 0; q < 4; ++q) R = fmaxf(R, sqrtf((px[q] - cx) * (px[q] - cx) + (py[q] - cy) * (py[q] - cy)));
  rad = tg.reach + R;
  const float reach = rad * 1.0001f + 1.0f;  // float rounding margin
  r2 = reach * reach;
  rad = reach;
}

__device__ __forceinline__ bool trace_in_disc(float4 g, float cx, float cy, float r2) {
  const float a = g.x - cx, b = g.y - cy, c = g.z - cx, d = g.w - cy;
  return (a * a + b * b < r2) && (c * c + d * d < r2);
}

__device__ __forceinline__ void cell_rows(const CellGrid& cg, float cx, float cy, float rad,
                                          int& cx0, int& cx1, int& cy0, int& cy1) {
  // a midpoint of a passing trace lies within `rad` of the centre
  cx0 = max(0, (int)floorf((cx - rad - cg.x0) / cg.cs));
  cx1 = min(cg.ncx - 1, (int)floorf((cx + rad - cg.x0) / cg.cs));
  cy0 = max(0, (int)floorf((cy - rad - cg.y0) / cg.cs));
  cy1 = min(cg.ncy - 1, (int)floorf((cy + rad - cg.y0) / cg.cs));
}

__global__ void __launch_bounds__(256) tile_count_kernel(TileGeom tg, CellGrid cg,
                                                         const int64_t* cell_start,
                                                         const float4* geo, int64_t* counts) {
  const int tile = blockIdx.x;
  float cx, cy, r2, rad;
  tile_disc(tg, tile, cx, cy, r2, rad);
  int x0, x1, y0, y1;
  cell_rows(cg, cx, cy, rad, x0, x1, y0, y1);
  int64_t cnt = 0;
  if (x0 <= x1) {
    for (int row = y0; row <= y1; ++row) {
      const int64_t a = cell_start[row * cg.ncx + x0], b = cell_start[row * cg.ncx + x1 + 1];
      for (int64_t j = a + threadIdx.x; j < b; j += blockDim.x)
        cnt += trace_in_disc(geo[j], cx, cy, r2) ? 1 : 0;
    }
  }
  using BR = cub::BlockReduce<int64_t, 256>;
  __shared__ typename BR::TempStorage tmp;
  const int64_t total = BR(tmp).Sum(cnt);
  if (threadIdx.x == 0) counts[tile] = total;
}

__global__ void __launch_bounds__(256) tile_fill_kernel(TileGeom tg, CellGrid cg,
                                                        const int64_t* cell_start,
                                                        const float4* geo, const int64_t* off,
                                                        int* list) {
  const int tile = blockIdx.x;
  float cx, cy, r2, rad;
  tile_disc(tg, tile, cx, cy, r2, rad);
  int x0, x1, y0, y1;
  cell_rows(cg, cx, cy, rad, x0, x1, y0, y1);
  using BS = cub::BlockScan<int, 256>;
  __shared__ typename BS::TempStorage tmp;
  __shared__ int chunk_total;
  int64_t base = off[tile];
  if (x0 > x1) return;
  for (int row = y0; row <= y1; ++row) {
    const int64_t a = cell_start[row * cg.ncx + x0], b = cell_start[row * cg.ncx + x1 + 1];
    for (int64_t j0 = a; j0 < b; j0 += blockDim.x) {
      const int64_t j = j0 + threadIdx.x;
      const int flag = (j < b && trace_in_disc(geo[j], cx, cy, r2)) ? 1 : 0;
      int pos, tot;
      BS(tmp).ExclusiveSum(flag, pos, tot);
      if (flag) list[base + pos] = (int)j;
      if (threadIdx.x == 0) chunk_total = tot;
      __syncthreads();
      base += chunk_total;
      __syncthreads();
    }
  }
}

// Sort key of a list entry: the larger squared leg distance from the tile
// centre (non-negative float, so its bits order like the value).  Sorting a
// tile's list by it lines up traces whose first contributing output sample is
// close, so the two traces a warp sweeps together mask out few samples.
__global__ void __launch_bounds__(256) tile_key_kernel(TileGeom tg, const float4* geo,
                                                       const int64_t* off, int tile0,
                                                       const int* list, int64_t base,
                                                       uint32_t* keys, int* seg) {
  const int tile = tile0 + blockIdx.x;
  float cx, cy, r2, rad;
  tile_disc(tg, tile, cx, cy, r2, rad);
  const int64_t a = off[tile], b = off[tile + 1];
  if (threadIdx.x == 0) {
    seg[blockIdx.x] = (int)(a - base);
    seg[blockIdx.x + 1] = (int)(b - base);
  }
  for (int64_t j = a + threadIdx.x; j < b; j += blockDim.x) {
    const float4 g = geo[list[j]];
    const float ds = (g.x - cx) * (g.x - cx) + (g.y - cy) * (g.y - cy);
    const float dr = (g.z - cx) * (g.z - cx) + (g.w - cy) * (g.w - cy);
    keys[j - base] = __float_as_uint(fmaxf(ds, dr));
  }
}

// --------------------------------------------------------- trace staging ---

__global__ void maxabs_kernel(const float* tr, int64_t n_tr, int n_s, int trace_major,
                              const int* inv_perm, float target, float* scales) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n_tr) return;
  float m = 0.f;
  if (trace_major) {
    const float* row = tr + j * n_s;
    for (int i = 0; i < n_s; ++i) m = fmaxf(m, fabsf(row[i]));
  } else {
    for (int i = 0; i < n_s; ++i) m = fmaxf(m, fabsf(tr[(int64_t)i * n_tr + j]));
  }
  scales[inv_perm[j]] = m > 0.f ? m / target : 1.0f;
}

template <typename ST>
__device__ __forceinline__ ST convert_to(float v);
template <>
__device__ __forceinline__ float convert_to<float>(float v) {
  return v;
}
template <>
__device__ __forceinline__ __nv_bfloat16 convert_to<__nv_bfloat16>(float v) {
  return __float2bfloat16_rn(v);
}
template <>
__device__ __forceinline__ __half convert_to<__half>(float v) {
  return __float2half_rn(v);
}

// (n_s, n_tr) sample-major -> sorted trace-major rows, via 32x32 shared tiles.
template <typename ST>
__global__ void stage_transpose_kernel(const float* tr, int64_t n_tr, int n_s, const int* inv_perm,
                                       const float* scales, int S, ST* out) {
  __shared__ float tile[32][33];
  const int64_t j0 = (int64_t)blockIdx.x * 32;
  const int i0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int i = i0 + r;
    const int64_t j = j0 + threadIdx.x;
    tile[r][threadIdx.x] = (i < n_s && j < n_tr) ? tr[(int64_t)i * n_tr + j] : 0.f;
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int64_t j = j0 + r;
    const int i = i0 + threadIdx.x;
    if (j < n_tr && i < n_s) {
      const int jj = inv_perm[j];
      const float inv = scales ? 1.0f / scales[jj] : 1.0f;
      out[(int64_t)jj * S + i] = convert_to<ST>(tile[threadIdx.x][r] * inv);
    }
  }
}

template <typename ST>
__global__ void stage_rows_kernel(const float* tr, int64_t n_tr, int n_s, const int* perm,
                                  const float* scales, int S, ST* out) {
  const int64_t jj = blockIdx.x;
  const int j = perm[jj];
  const float inv = scales ? 1.0f / scales[jj] : 1.0f;
  for (int i = threadIdx.x; i < n_s; i += blockDim.x)
    out[jj * S + i] = convert_to<ST>(tr[(int64_t)j * n_s + i] * inv);
}

// Expanded entry at row position q for the linear piece from x0 to x1:
// (x0 - (q - q0) d, d) with d = x1 - x0 (float32), so that the interpolant at
// position u in [q, q + 1) is one FMA, (u - q0) d + c, with no fractional part
// to form.  The intercept is rounded once from float64; q0 (mid-row) keeps
// |q - q0| small.
__device__ __forceinline__ float2 expanded_entry(float x0, float x1, int q, int q0) {
  const float d = x1 - x0;
  return make_float2((float)((double)x0 - (double)(q - q0) * (double)d), d);
}

// float32 staging into (x[i], x[i+1] - x[i]) entries at row position i + 1
// (x = 0 outside the trace), sample-major input via 33 x 32 shared tiles.  The
// operator keeps this sample-and-step form by default: its interpolant
// x + f (x' - x) rounds like the adjoint's transposed split, which keeps the
// dot-product test of the pair at float32 rounding.  Plans that only migrate
// (q0 > 0) take the intercept form instead (one FMA per tap; against the
// adjoint it adds ~1e-5 on white-noise data).
__device__ __forceinline__ float2 row_entry(float x0, float x1, int q, int q0) {
  return q0 > 0 ? expanded_entry(x0, x1, q, q0) : make_float2(x0, x1 - x0);
}

__global__ void stage_transpose_x2_kernel(const float* tr, int64_t n_tr, int n_s,
                                          const int* inv_perm, int S, int q0, float2* out) {
  __shared__ float tile[33][33];
  const int64_t j0 = (int64_t)blockIdx.x * 32;
  const int i0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 33; r += blockDim.y) {
    const int i = i0 + r;
    const int64_t j = j0 + threadIdx.x;
    tile[r][threadIdx.x] = (i < n_s && j < n_tr) ? tr[(int64_t)i * n_tr + j] : 0.f;
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int64_t j = j0 + r;
    const int i = i0 + threadIdx.x;
    if (j < n_tr && i < n_s) {
      const int jj = inv_perm[j];
      const float x0 = tile[threadIdx.x][r], x1 = tile[threadIdx.x + 1][r];
      out[(int64_t)jj * S + i + 1] = row_entry(x0, x1, i + 1, q0);
      if (i == 0) out[(int64_t)jj * S] = row_entry(0.f, x0, 0, q0);
    }
  }
}

__global__ void stage_rows_x2_kernel(const float* tr, int64_t n_tr, int n_s, const int* perm,
                                     int S, int q0, float2* out) {
  const int64_t jj = blockIdx.x;
  const float* x = tr + (int64_t)perm[jj] * n_s;
  for (int i = (int)threadIdx.x - 1; i < n_s; i += blockDim.x) {
    const float x0 = i >= 0 ? x[i] : 0.f;
    const float x1 = i + 1 < n_s ? x[i + 1] : 0.f;
    out[jj * S + i + 1] = row_entry(x0, x1, i + 1, q0);
  }
}

// sorted trace-major accumulation rows -> caller layout, original order
__global__ void unstage_transpose_kernel(const float* acc, int64_t n_tr, int n_s,
                                         const int* inv_perm, int S, float* out) {
  __shared__ float tile[32][33];
  const int64_t j0 = (int64_t)blockIdx.x * 32;
  const int i0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int64_t j = j0 + r;
    const int i = i0 + threadIdx.x;
    tile[r][threadIdx.x] = (j < n_tr && i < n_s) ? acc[(int64_t)inv_perm[j] * S + i] : 0.f;
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int i = i0 + r;
    const int64_t j = j0 + threadIdx.x;
    if (i < n_s && j < n_tr) out[(int64_t)i * n_tr + j] = tile[threadIdx.x][r];
  }
}

__global__ void unstage_rows_kernel(const float* acc, int64_t n_tr, int n_s, const int* inv_perm,
                                    int S, float* out) {
  const int64_t j = blockIdx.x;
  const int jj = inv_perm[j];
  for (int i = threadIdx.x; i < n_s; i += blockDim.x) out[j * n_s + i] = acc[(int64_t)jj * S + i];
}

// Anti-alias staging, one warp per sorted trace row: the samples (rounded to
// the requested storage precision, bf16 or f16 with a per-trace scale), their
// causal double integral in float64
//   I1[i] = sum_{n<=i} x[n],  I2[i] = sum_{m<i} I1[m]   (i = 0..N),
// extended with I2 = 0 before the trace and I2[N] + (i-N) I1[N-1] after it, and
// a linear trend beta*i removed (beta = I2[N]/N) -- the triangle filter takes
// second differences, to which linear terms contribute nothing -- stored in
// float32 at row positions i + pad.
__device__ __forceinline__ float quantize_sample(float x, int storage, float scale) {
  if (storage == PSTM_BF16) return __bfloat162float(__float2bfloat16_rn(x));
  if (storage == PSTM_F16) return __half2float(__float2half_rn(x / scale)) * scale;
  return x;
}

__global__ void aa_integrate_kernel(const float* rows, int64_t n_tr, int n_s, int S_in, int storage,
                                    int pad, int S_out, int q0, float2* out) {
  const int64_t row = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (row >= n_tr) return;
  const float* x = rows + row * S_in;
  float2* o = out + row * S_out;
  // expanded entry at position i + pad from the float32 values I2'[i], I2'[i+1]
  auto entry = [&](double cur, double nxt, int i) {
    return expanded_entry((float)cur, (float)nxt, i + pad, q0);
  };
  float scale = 1.0f;
  if (storage == PSTM_F16) {
    float m = 0.f;
    for (int i = lane; i < n_s; i += 32) m = fmaxf(m, fabsf(x[i]));
    for (int d = 16; d > 0; d >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, d));
    scale = m > 0.f ? m / 32768.0f : 1.0f;
  }
  // pass 1: totals I2[N] and I1[N-1]
  double c1 = 0.0, c2 = 0.0;
  for (int base = 0; base < n_s; base += 32) {
    const int i = base + lane;
    double v = i < n_s ? (double)quantize_sample(x[i], storage, scale) : 0.0;
    for (int d = 1; d < 32; d <<= 1) {
      const double u = __shfl_up_sync(0xffffffffu, v, d);
      if (lane >= d) v += u;
    }
    const double i1 = v + c1;  // inclusive I1[i]
    double e = i < n_s ? i1 : 0.0;
    for (int d = 16; d > 0; d >>= 1) e += __shfl_xor_sync(0xffffffffu, e, d);
    c1 = __shfl_sync(0xffffffffu, i1, 31);
    c2 += e;
  }
  const double i2_end = c2, i1_last = c1;
  const double beta = i2_end / (double)n_s;
  // pass 2: write I2'[i] = I2[i] - beta i
  c1 = 0.0;
  c2 = 0.0;
  for (int base = 0; base < n_s; base += 32) {
    const int i = base + lane;
    double v = i < n_s ? (double)quantize_sample(x[i], storage, scale) : 0.0;
    for (int d = 1; d < 32; d <<= 1) {
      const double u = __shfl_up_sync(0xffffffffu, v, d);
      if (lane >= d) v += u;
    }
    const double i1 = v + c1;
    // exclusive prefix of I1 within the chunk gives I2[i]
    double ex = __shfl_up_sync(0xffffffffu, i1, 1);
    if (lane == 0) ex = 0.0;
    double acc = ex;
    for (int d = 1; d < 32; d <<= 1) {
      const double u = __shfl_up_sync(0xffffffffu, acc, d);
      if (lane >= d) acc += u;
    }
    // I2[i+1] = I2[i] + I1[i]
    if (i < n_s) o[i + pad] = entry(c2 + acc - beta * (double)i,
                                    c2 + acc + i1 - beta * (double)(i + 1), i);
    double e = i < n_s ? i1 : 0.0;
    for (int d = 16; d > 0; d >>= 1) e += __shfl_xor_sync(0xffffffffu, e, d);
    c1 = __shfl_sync(0xffffffffu, i1, 31);
    c2 += e;
  }
  // before the trace (I2 = 0) and from I2[N] on (linear continuation)
  for (int q = lane; q < pad; q += 32) {
    const int i = q - pad;  // -pad .. -1
    o[q] = entry(-beta * (double)i, -beta * (double)(i + 1), i);
  }
  for (int q = n_s + pad + lane; q < S_out; q += 32) {
    const int i = q - pad;  // N ..
    o[q] = entry(i2_end + (double)(i - n_s) * i1_last - beta * (double)i,
                 i2_end + (double)(i + 1 - n_s) * i1_last - beta * (double)(i + 1), i);
  }
}

__global__ void normalize_kernel(const float* image, const float* fold, float* out, int64_t n,
                                 float min_fold, int mute) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float f = fold[i], v = image[i];
  if (mute) {
    out[i] = f >= min_fold ? v / fmaxf(f, min_fold) : 0.f;
  } else {
    out[i] = f >= min_fold ? v / f : v;
  }
}

// ------------------------------------------------------------------ host ---

static int64_t align_up(int64_t v, int64_t a) { return (v + a - 1) / a * a; }

// One pool per device, created on first use.  Freed blocks stay mapped up to
// kPoolKeepBytes, so a plan built after another one of similar size reuses its
// memory instead of mapping (and later unmapping) fresh gigabytes.
static cudaError_t pool_for(int dev, cudaMemPool_t* out) {
  static std::mutex mu;
  static cudaMemPool_t pools[64] = {};
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(mu);
  if (!pools[dev]) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaError_t e = cudaMemPoolCreate(&pools[dev], &props);
    if (e != cudaSuccess) return e;
    uint64_t keep = kPoolKeepBytes;
    e = cudaMemPoolSetAttribute(pools[dev], cudaMemPoolAttrReleaseThreshold, &keep);
    if (e != cudaSuccess) return e;
  }
  *out = pools[dev];
  return cudaSuccess;
}

cudaError_t pstm::dev_malloc(void** ptr, size_t bytes, cudaStream_t s) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  cudaMemPool_t pool;
  if (e == cudaSuccess) e = pool_for(dev, &pool);
  if (e == cudaSuccess) e = cudaMallocFromPoolAsync(ptr, std::max<size_t>(bytes, 1), pool, s);
  if (e != cudaSuccess) *ptr = nullptr;
  return e;
}

void pstm::dev_free(void* ptr, cudaStream_t s) {
  if (ptr) cudaFreeAsync(ptr, s);
}

template <typename T>
static cudaError_t dalloc(Plan* p, T** ptr, size_t count, cudaStream_t s) {
  const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
  cudaError_t e = dev_malloc(reinterpret_cast<void**>(ptr), bytes, s);
  if (e == cudaSuccess) p->bytes += (int64_t)bytes;
  return e;
}

// Orders every tile's trace list by tile_key_kernel's key (stable, so the
// order is reproducible), in chunks of whole tiles that bound the temporaries.
static cudaError_t sort_tile_lists(Plan* p, const TileGeom& tg, cudaStream_t s) {
  const int64_t n_tiles = p->n_tiles;
  std::vector<int64_t> off(n_tiles + 1);
  cudaError_t e = cudaMemcpyAsync(off.data(), p->tile_off, off.size() * sizeof(int64_t),
                                  cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return e;
  constexpr int64_t kChunk = int64_t(1) << 24;
  int64_t cap = 0, longest = 0;
  for (int64_t t = 0; t < n_tiles; ++t) longest = std::max(longest, off[t + 1] - off[t]);
  p->longest_list = longest;
  cap = std::min(off[n_tiles], std::max(kChunk, longest));
  if (cap <= 1 || cap > INT32_MAX) return cudaSuccess;  // order is only a speed hint
  constexpr int64_t kMaxSegs = 65535;                      // tiles per key launch
  uint32_t *kin = nullptr, *kout = nullptr;
  int *vout = nullptr, *seg = nullptr;
  void* tmp = nullptr;
  size_t tmp_bytes = 0;
  struct Free {
    void** ptrs[5];
    cudaStream_t s;
    ~Free() {
      for (auto pp : ptrs) dev_free(*pp, s);
    }
  } fr{{(void**)&kin, (void**)&kout, (void**)&vout, (void**)&seg, &tmp}, s};
  if ((e = dev_malloc((void**)&kin, cap * sizeof(uint32_t), s)) != cudaSuccess) return e;
  if ((e = dev_malloc((void**)&kout, cap * sizeof(uint32_t), s)) != cudaSuccess) return e;
  if ((e = dev_malloc((void**)&vout, cap * sizeof(int), s)) != cudaSuccess) return e;
  if ((e = dev_malloc((void**)&seg, (kMaxSegs + 1) * sizeof(int), s)) != cudaSuccess) return e;
  for (int64_t ta = 0; ta < n_tiles;) {
    int64_t tb = ta + 1;
    while (tb < n_tiles && tb - ta < kMaxSegs && off[tb + 1] - off[ta] <= cap) ++tb;
    const int64_t base = off[ta], items = off[tb] - base;
    const int nseg = (int)(tb - ta);
    if (items > 1) {
      tile_key_kernel<<<nseg, 256, 0, s>>>(tg, p->geo, p->tile_off, (int)ta, p->tile_list, base,
                                           kin, seg);
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
      size_t need = 0;
      e = cub::DeviceSegmentedSort::StableSortPairs(nullptr, need, kin, kout, p->tile_list + base,
                                                    vout, (int)items, nseg, seg, seg + 1, s);
      if (e != cudaSuccess) return e;
      if (need > tmp_bytes) {
        dev_free(tmp, s);
        tmp = nullptr;
        if ((e = dev_malloc(&tmp, need, s)) != cudaSuccess) return e;
        tmp_bytes = need;
      }
      e = cub::DeviceSegmentedSort::StableSortPairs(tmp, tmp_bytes, kin, kout,
                                                    p->tile_list + base, vout, (int)items, nseg,
                                                    seg, seg + 1, s);
      if (e != cudaSuccess) return e;
      e = cudaMemcpyAsync(p->tile_list + base, vout, items * sizeof(int),
                          cudaMemcpyDeviceToDevice, s);
      if (e != cudaSuccess) return e;
      count_launch();
    }
    ta = tb;
  }
  return cudaStreamSynchronize(s);
}

// The plan may have been used on any stream: wait for the device, then
// return its memory to the pool.
static void free_plan(Plan* p) {
  if (!p) return;
  int cur = -1;
  cudaGetDevice(&cur);
  if (cur != p->device) cudaSetDevice(p->device);
  cudaDeviceSynchronize();
  void* bufs[] = {p->geo,      p->perm,    p->inv_perm, p->tile_off, p->adj_off, p->adj_tiles,
                  p->adj_table, p->tile_list, p->traces,  p->scales,   p->accum,   p->err};
  for (void* b : bufs) dev_free(b, 0);
  cudaStreamSynchronize(0);
  if (cur >= 0 && cur != p->device) cudaSetDevice(cur);
  delete p;
}

static pstm_status validate(const pstm_grid* g, const pstm_params* prm, const pstm_geometry* geo) {
  if (!g || !prm || !geo) return fail(PSTM_EINVAL, "null grid/params/geometry");
  if (g->n_il < 1 || g->n_xl < 1 || g->n_times < 1)
    return fail(PSTM_EINVAL, "output grid dimensions must be positive");
  if (!(g->dt_ms > 0)) return fail(PSTM_EINVAL, "output dt must be positive");
  if (prm->n_samples < 2) return fail(PSTM_EINVAL, "traces need at least 2 samples");
  if (!(prm->in_dt_ms > 0)) return fail(PSTM_EINVAL, "input dt must be positive");
  if (!(prm->max_aperture_m > 0)) return fail(PSTM_EINVAL, "max_aperture_m must be positive");
  if (!(prm->max_angle_deg > 0 && prm->max_angle_deg <= 90))
    return fail(PSTM_EINVAL, "max_angle_deg must be in (0, 90]");
  if (prm->weight < 0 || prm->weight > 3) return fail(PSTM_EINVAL, "unknown weight mode");
  if (prm->clamp < 0 || prm->clamp > 1) return fail(PSTM_EINVAL, "unknown clamp mode");
  if (prm->storage != PSTM_F32 && prm->storage != PSTM_BF16 && prm->storage != PSTM_F16)
    return fail(PSTM_EINVAL, "storage must be F32, BF16 or F16");
  if (prm->antialias && !(prm->aa_max_halfwidth >= 1.0 && prm->aa_max_halfwidth <= 256.0))
    return fail(PSTM_EINVAL, "aa_max_halfwidth must be in [1, 256] samples");
  if (prm->antialias && (!(prm->aa_dx >= 0) || !(prm->aa_dy >= 0)))
    return fail(PSTM_EINVAL, "aa_dx/aa_dy must be non-negative");
  if (prm->forward_only != 0 && prm->forward_only != 1)
    return fail(PSTM_EINVAL, "forward_only must be 0 or 1");
  if (!(prm->taper_width >= 0.0 && prm->taper_width < 1.0))
    return fail(PSTM_EINVAL, "taper_width must be in [0, 1)");
  if (prm->taper_width > 0 && (prm->storage != PSTM_F32 || prm->antialias))
    return fail(PSTM_ENOTSUP, "the aperture taper is built for float32 storage without the "
                              "anti-alias filter");
  if (!std::isfinite(prm->ray_gradient))
    return fail(PSTM_EINVAL, "ray_gradient must be finite");
  if (prm->ray_gradient != 0 &&
      (prm->storage != PSTM_F32 || prm->antialias || prm->taper_width > 0))
    return fail(PSTM_ENOTSUP, "curved rays (ray_gradient) are built for float32 storage "
                              "without the anti-alias filter or the aperture taper");
  if (prm->antialias && prm->weight != PSTM_WEIGHT_OBLIQUITY_SPREADING)
    return fail(PSTM_ENOTSUP, "the anti-alias kernel is built for the obliquity x spreading weight");
  if (geo->n_traces < 0 || geo->n_traces > (int64_t)INT32_MAX)
    return fail(PSTM_EINVAL, "n_traces out of range");
  if (geo->n_traces > 0 && (!geo->source_x || !geo->source_y || !geo->receiver_x || !geo->receiver_y))
    return fail(PSTM_EINVAL, "null coordinate pointer");
  if (geo->coord_dtype != PSTM_F32 && geo->coord_dtype != PSTM_F64)
    return fail(PSTM_EINVAL, "coordinates must be F32 or F64");
  const double n_out = (double)g->n_il * g->n_xl * g->n_times;
  if (n_out > 9.0e18) return fail(PSTM_EINVAL, "output grid too large");
  return PSTM_OK;
}

// The plan's staged-trace rows (and f16 scales), allocated once.
pstm_status pstm::ensure_trace_storage(Plan* p, cudaStream_t s) {
  if (p->traces || p->n_traces == 0) return PSTM_OK;
  const size_t bytes = (size_t)p->n_traces * p->row_stride * p->elt_bytes;
  CUDA_TRY(dev_malloc(&p->traces, bytes, s));
  p->bytes += (int64_t)bytes;
  CUDA_TRY(cudaMemsetAsync(p->traces, 0, bytes, s));
  // f16 needs a per-trace scale for its range; bf16 has float32's exponent
  // range and is stored unscaled
  if (p->params.storage == PSTM_F16 && !p->params.antialias)
    CUDA_TRY(dalloc(p, &p->scales, p->n_traces, s));
  return PSTM_OK;
}

extern "C" {

int32_t pstm_abi_version(void) { return SEISPSTM_ABI_VERSION; }

int32_t pstm_last_error(char* buf, size_t n) {
  if (buf && n > 0) {
    const size_t k = std::min(n - 1, g_last_error.size());
    memcpy(buf, g_last_error.data(), k);
    buf[k] = '\0';
  }
  return (int32_t)g_last_error.size();
}

int64_t pstm_launch_count(void) { return launch_total(); }

pstm_status pstm_plan_create(pstm_plan** out, const pstm_grid* g, const pstm_params* prm,
                             const pstm_geometry* geo, void* stream) {
  if (!out) return fail(PSTM_EINVAL, "null plan pointer");
  *out = nullptr;
  pstm_status st = validate(g, prm, geo);
  if (st != PSTM_OK) return st;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  Plan* p = new (std::nothrow) Plan();
  if (!p) return fail(PSTM_ENOMEM, "host allocation failed");
  struct Guard {
    Plan*& p;
    bool keep = false;
    ~Guard() {
      if (!keep) free_plan(p);
    }
  } guard{p};
  CUDA_TRY(cudaGetDevice(&p->device));
  p->grid = *g;
  p->params = *prm;
  p->n_traces = geo->n_traces;
  p->n_samples = prm->n_samples;
  p->row_stride = (int)align_up(prm->n_samples, 8);
  p->elt_bytes = 2;
  if (prm->storage == PSTM_F32) {
    // (x[i], x[i+1] - x[i]) entries for i = -1 .. N-1 at row positions i + 1
    p->row_stride = (int)align_up(prm->n_samples + 1, 8);
    p->elt_bytes = 8;
    // migration-only plans: intercept form about the middle entry
    if (prm->forward_only) p->row_origin = (prm->n_samples + 1) / 2;
  }
  if (prm->antialias) {
    // rows hold the trend-removed double integral I2[-pad .. N + pad] in float32
    p->aa_pad = (int)std::ceil(prm->aa_max_halfwidth) + 2;
    p->row_stride = (int)align_up(prm->n_samples + 1 + 2 * p->aa_pad, 8);
    p->elt_bytes = 8;  // intercept-form entries of I2
    p->row_origin = (prm->n_samples + 1 + 2 * p->aa_pad) / 2;
  }
  if (!shape_for_variant(prm->variant, g->n_xl, g->n_times, &p->shape))
    return fail(PSTM_EINVAL, "unknown kernel variant");
  if (prm->taper_width > 0 || prm->ray_gradient != 0) {
    // the tapered and curved-ray kernels are built for the 16-column shapes only
    if (prm->variant == 0) {
      shape_for_variant(g->n_xl < 2 ? 9 : 3, g->n_xl, g->n_times, &p->shape);
    } else if (p->shape.id != 3 && p->shape.id != 9) {
      return fail(PSTM_ENOTSUP,
                  "the aperture taper and curved rays run kernel variants 3 and 9 only");
    }
  }
  p->tiles_il = (g->n_il + p->shape.tile_il - 1) / p->shape.tile_il;
  p->tiles_xl = (g->n_xl + p->shape.tile_xl - 1) / p->shape.tile_xl;
  p->n_tiles = (int64_t)p->tiles_il * p->tiles_xl;
  p->n_windows = (g->n_times + p->shape.t_window() - 1) / p->shape.t_window();
  if (p->n_tiles > INT32_MAX || p->n_windows > 65535) return fail(PSTM_EINVAL, "grid too large");
  p->il_dx = (float)g->il_dx;
  p->il_dy = (float)g->il_dy;
  p->xl_dx = (float)g->xl_dx;
  p->xl_dy = (float)g->xl_dy;
  p->tan_theta = (float)std::tan(prm->max_angle_deg * M_PI / 180.0);
  const size_t smem = forward_smem_bytes(p);
  if (smem > forward_smem_budget(p))
    return fail(PSTM_EINVAL, "traces too long for the staged kernel (" +
                                 std::to_string(prm->n_samples) + " samples)");
  CUDA_TRY(dalloc(p, &p->err, 4, s));
  CUDA_TRY(cudaMemsetAsync(p->err, 0, 16, s));
  CUDA_TRY(dalloc(p, &p->tile_off, p->n_tiles + 1, s));
  const int64_t n = p->n_traces;
  if (n == 0) {
    CUDA_TRY(cudaMemsetAsync(p->tile_off, 0, (p->n_tiles + 1) * sizeof(int64_t), s));
    CUDA_TRY(cudaStreamSynchronize(s));
    guard.keep = true;
    *out = reinterpret_cast<pstm_plan*>(p);
    return PSTM_OK;
  }
  // temporaries
  float4* geo_u = nullptr;
  float2* mid = nullptr;
  int *key = nullptr, *key_sorted = nullptr, *iota = nullptr, *bbox = nullptr;
  int64_t *cell_start = nullptr, *counts = nullptr;
  void* cub_tmp = nullptr;
  struct Tmp {
    void** ptrs[9];
    cudaStream_t s;
    ~Tmp() {
      for (auto pp : ptrs)
        if (pp) dev_free(*pp, s);
    }
  } tmp{{(void**)&geo_u, (void**)&mid, (void**)&key, (void**)&key_sorted, (void**)&iota,
         (void**)&bbox, (void**)&cell_start, (void**)&counts, (void**)&cub_tmp}, s};
  CUDA_TRY(dev_malloc((void**)&geo_u, n * sizeof(float4), s));
  CUDA_TRY(dev_malloc((void**)&mid, n * sizeof(float2), s));
  CUDA_TRY(dev_malloc((void**)&key, n * sizeof(int), s));
  CUDA_TRY(dev_malloc((void**)&key_sorted, n * sizeof(int), s));
  CUDA_TRY(dev_malloc((void**)&iota, n * sizeof(int), s));
  CUDA_TRY(dev_malloc((void**)&bbox, 4 * sizeof(int), s));
  CUDA_TRY(dalloc(p, &p->geo, n, s));
  CUDA_TRY(dalloc(p, &p->perm, n, s));
  CUDA_TRY(dalloc(p, &p->inv_perm, n, s));
  const int thr = 256;
  const unsigned nblk = (unsigned)((n + thr - 1) / thr);
  if (geo->coord_dtype == PSTM_F64) {
    geo_local_kernel<double><<<nblk, thr, 0, s>>>(
        (const double*)geo->source_x, (const double*)geo->source_y,
        (const double*)geo->receiver_x, (const double*)geo->receiver_y, n, g->origin_x,
        g->origin_y, geo_u, mid);
  } else {
    geo_local_kernel<float><<<nblk, thr, 0, s>>>(
        (const float*)geo->source_x, (const float*)geo->source_y, (const float*)geo->receiver_x,
        (const float*)geo->receiver_y, n, g->origin_x, g->origin_y, geo_u, mid);
  }
  LAUNCH_CHECK("geo_local_kernel");
  bbox_init_kernel<<<1, 1, 0, s>>>(bbox);
  LAUNCH_CHECK("bbox_init_kernel");
  bbox_kernel<<<std::min<unsigned>(nblk, 1184), thr, 0, s>>>(mid, n, bbox);
  LAUNCH_CHECK("bbox_kernel");
  int hb[4];
  CUDA_TRY(cudaMemcpyAsync(hb, bbox, sizeof(hb), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  auto unord = [](int i) {
    int v = i >= 0 ? i : i ^ 0x7fffffff;
    float f;
    memcpy(&f, &v, 4);
    return f;
  };
  const float mnx = unord(hb[0]), mny = unord(hb[1]), mxx = unord(hb[2]), mxy = unord(hb[3]);
  if (!std::isfinite(mnx) || !std::isfinite(mny) || !std::isfinite(mxx) || !std::isfinite(mxy))
    return fail(PSTM_EINVAL, "non-finite trace coordinates");
  // cell grid over the midpoints
  const double tile_ext = std::hypot(p->shape.tile_il * std::hypot(g->il_dx, g->il_dy),
                                     p->shape.tile_xl * std::hypot(g->xl_dx, g->xl_dy));
  double cs = std::max(10.0, (prm->max_aperture_m + 0.5 * tile_ext) / 4.0);
  const double ex = std::max(1.0, (double)mxx - mnx), ey = std::max(1.0, (double)mxy - mny);
  while ((std::floor(ex / cs) + 1) * (std::floor(ey / cs) + 1) > (double)(1 << 22)) cs *= 2.0;
  CellGrid cg;
  cg.x0 = mnx;
  cg.y0 = mny;
  cg.cs = (float)cs;
  cg.ncx = (int)std::floor(ex / cs) + 1;
  cg.ncy = (int)std::floor(ey / cs) + 1;
  const int n_cells = cg.ncx * cg.ncy;
  cell_key_kernel<<<nblk, thr, 0, s>>>(mid, n, cg, key, iota);
  LAUNCH_CHECK("cell_key_kernel");
  int end_bit = 1;
  while ((1 << end_bit) <= n_cells && end_bit < 31) ++end_bit;
  size_t tmp_bytes = 0;
  CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, key, key_sorted, iota, p->perm,
                                           (int)n, 0, end_bit, s));
  size_t scan_bytes = 0;
  CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, (int64_t*)nullptr,
                                         (int64_t*)nullptr, (int)(p->n_tiles + 1), s));
  tmp_bytes = std::max(tmp_bytes, scan_bytes);
  CUDA_TRY(dev_malloc(&cub_tmp, tmp_bytes, s));
  CUDA_TRY(cub::DeviceRadixSort::SortPairs(cub_tmp, tmp_bytes, key, key_sorted, iota, p->perm,
                                           (int)n, 0, end_bit, s));
  count_launch();
  CUDA_TRY(dev_malloc((void**)&cell_start, (n_cells + 1) * sizeof(int64_t), s));
  cell_start_kernel<<<(n_cells + 1 + thr - 1) / thr, thr, 0, s>>>(key_sorted, n, n_cells,
                                                                   cell_start);
  LAUNCH_CHECK("cell_start_kernel");
  gather_geo_kernel<<<nblk, thr, 0, s>>>(geo_u, p->perm, n, p->geo, p->inv_perm);
  LAUNCH_CHECK("gather_geo_kernel");
  TileGeom tg;
  tg.n_il = g->n_il;
  tg.n_xl = g->n_xl;
  tg.tile_il = p->shape.tile_il;
  tg.tile_xl = p->shape.tile_xl;
  tg.tiles_xl = p->tiles_xl;
  tg.il_dx = p->il_dx;
  tg.il_dy = p->il_dy;
  tg.xl_dx = p->xl_dx;
  tg.xl_dy = p->xl_dy;
  tg.reach = (float)prm->max_aperture_m;
  CUDA_TRY(dev_malloc((void**)&counts, (p->n_tiles + 1) * sizeof(int64_t), s));
  CUDA_TRY(cudaMemsetAsync(counts, 0, (p->n_tiles + 1) * sizeof(int64_t), s));
  tile_count_kernel<<<(unsigned)p->n_tiles, 256, 0, s>>>(tg, cg, cell_start, p->geo, counts);
  LAUNCH_CHECK("tile_count_kernel");
  CUDA_TRY(cub::DeviceScan::ExclusiveSum(cub_tmp, tmp_bytes, counts, p->tile_off,
                                         (int)(p->n_tiles + 1), s));
  count_launch();
  int64_t total = 0;
  CUDA_TRY(cudaMemcpyAsync(&total, p->tile_off + p->n_tiles, sizeof(int64_t),
                           cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  p->list_entries = total;
  if (total == 0) p->longest_list = 0;
  CUDA_TRY(dalloc(p, &p->tile_list, total, s));
  if (total > 0) {
    tile_fill_kernel<<<(unsigned)p->n_tiles, 256, 0, s>>>(tg, cg, cell_start, p->geo, p->tile_off,
                                                          p->tile_list);
    LAUNCH_CHECK("tile_fill_kernel");
    CUDA_TRY(sort_tile_lists(p, tg, s));
  }
  CUDA_TRY(cudaStreamSynchronize(s));
  guard.keep = true;
  *out = reinterpret_cast<pstm_plan*>(p);
  return PSTM_OK;
}

pstm_status pstm_plan_destroy(pstm_plan* plan) {
  free_plan(reinterpret_cast<Plan*>(plan));
  return PSTM_OK;
}

pstm_status pstm_copy_trace_columns(float* dst, const float* src, int64_t n_samples,
                                   int64_t n_traces, int64_t first, int64_t count,
                                   void* stream) {
  if (n_samples < 0 || n_traces < 0 || first < 0 || count < 0 || first + count > n_traces ||
      (n_samples > 0 && count > 0 && (!dst || !src)))
    return fail(PSTM_EINVAL, "pstm_copy_trace_columns: bad arguments");
  if (n_samples == 0 || count == 0) return PSTM_OK;
  CUDA_TRY(cudaMemcpy2DAsync(dst, (size_t)count * sizeof(float), src + first,
                             (size_t)n_traces * sizeof(float), (size_t)count * sizeof(float),
                             (size_t)n_samples, cudaMemcpyHostToDevice,
                             reinterpret_cast<cudaStream_t>(stream)));
  return PSTM_OK;
}

pstm_status pstm_trim_memory(int64_t keep_bytes) {
  if (keep_bytes < 0) return fail(PSTM_EINVAL, "keep_bytes must be >= 0");
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  cudaMemPool_t pool;
  CUDA_TRY(pool_for(dev, &pool));
  CUDA_TRY(cudaDeviceSynchronize());
  CUDA_TRY(cudaMemPoolTrimTo(pool, (size_t)keep_bytes));
  return PSTM_OK;
}

pstm_status pstm_plan_get_stats(const pstm_plan* plan, pstm_plan_stats* st) {
  if (!plan || !st) return fail(PSTM_EINVAL, "null argument");
  const Plan* p = reinterpret_cast<const Plan*>(plan);
  st->n_traces = p->n_traces;
  st->n_tiles = p->n_tiles;
  st->list_entries = p->list_entries;
  st->device_bytes = p->bytes;
  st->tile_il = p->shape.tile_il;
  st->tile_xl = p->shape.tile_xl;
  st->t_window = p->shape.t_window();
  st->variant = p->shape.id;
  return PSTM_OK;
}

pstm_status pstm_load_traces(pstm_plan* plan, const float* traces, int32_t trace_major,
                             void* stream) {
  if (!plan) return fail(PSTM_EINVAL, "null plan");
  Plan* p = reinterpret_cast<Plan*>(plan);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const int64_t n = p->n_traces;
  const int n_s = p->n_samples;
  if (n == 0) {
    p->traces_loaded = true;
    return PSTM_OK;
  }
  if (!traces) return fail(PSTM_EINVAL, "null traces");
  pstm_status st = ensure_trace_storage(p, s);
  if (st != PSTM_OK) return st;
  const int thr = 256;
  if (p->params.antialias) {
    // plain float32 rows into the adjoint accumulator (free until demigration),
    // then one warp per row integrates into the staged rows
    const int S_in = (int)align_up(n_s, 8);
    if (!p->accum) CUDA_TRY(dalloc(p, &p->accum, (size_t)n * p->row_stride, s));
    dim3 tb(32, 8);
    dim3 tg((unsigned)((n + 31) / 32), (unsigned)((n_s + 31) / 32));
    if (trace_major)
      stage_rows_kernel<float><<<(unsigned)n, 256, 0, s>>>(traces, n, n_s, p->perm, nullptr, S_in,
                                                           p->accum);
    else
      stage_transpose_kernel<float><<<tg, tb, 0, s>>>(traces, n, n_s, p->inv_perm, nullptr, S_in,
                                                      p->accum);
    LAUNCH_CHECK("stage kernel");
    aa_integrate_kernel<<<(unsigned)((n + 7) / 8), 256, 0, s>>>(
        p->accum, n, n_s, S_in, p->params.storage, p->aa_pad, p->row_stride, p->row_origin,
        reinterpret_cast<float2*>(p->traces));
    LAUNCH_CHECK("aa_integrate_kernel");
    p->traces_loaded = true;
    return PSTM_OK;
  }
  if (p->params.storage == PSTM_F16) {
    const float target = 32768.0f;
    maxabs_kernel<<<(unsigned)((n + thr - 1) / thr), thr, 0, s>>>(traces, n, n_s, trace_major,
                                                                  p->inv_perm, target, p->scales);
    LAUNCH_CHECK("maxabs_kernel");
  }
  dim3 tb(32, 8);
  dim3 tg((unsigned)((n + 31) / 32), (unsigned)((n_s + 31) / 32));
#define PSTM_STAGE(T)                                                                          \
  if (trace_major)                                                                             \
    stage_rows_kernel<T><<<(unsigned)n, 256, 0, s>>>(traces, n, n_s, p->perm, p->scales,      \
                                                     p->row_stride, (T*)p->traces);            \
  else                                                                                         \
    stage_transpose_kernel<T><<<tg, tb, 0, s>>>(traces, n, n_s, p->inv_perm, p->scales,       \
                                                p->row_stride, (T*)p->traces);
  if (p->params.storage == PSTM_F32) {
    if (trace_major)
      stage_rows_x2_kernel<<<(unsigned)n, 256, 0, s>>>(traces, n, n_s, p->perm, p->row_stride,
                                                       p->row_origin, (float2*)p->traces);
    else
      stage_transpose_x2_kernel<<<tg, tb, 0, s>>>(traces, n, n_s, p->inv_perm, p->row_stride,
                                                  p->row_origin, (float2*)p->traces);
  } else if (p->params.storage == PSTM_BF16) {
    PSTM_STAGE(__nv_bfloat16)
  } else {
    PSTM_STAGE(__half)
  }
#undef PSTM_STAGE
  LAUNCH_CHECK("stage kernel");
  p->traces_loaded = true;
  return PSTM_OK;
}

static pstm_status check_velocity_args(const float* vel, int64_t vst, int64_t vsc) {
  if (!vel) return fail(PSTM_EINVAL, "null velocity");
  if (vst < 0 || vsc < 0) return fail(PSTM_EINVAL, "negative velocity stride");
  return PSTM_OK;
}

pstm_status pstm_migrate_loaded(pstm_plan* plan, const float* vel, int64_t vst, int64_t vsc,
                                float* image, float* fold, void* stream) {
  if (!plan || !image) return fail(PSTM_EINVAL, "null plan or image");
  Plan* p = reinterpret_cast<Plan*>(plan);
  if (!p->traces_loaded) return fail(PSTM_EINVAL, "no traces loaded into the plan");
  pstm_status st = check_velocity_args(vel, vst, vsc);
  if (st != PSTM_OK) return st;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  std::string why;
  st = launch_velocity_check(p, vel, vst, vsc, s, &why);
  if (st != PSTM_OK) return fail(st, why);
  st = launch_forward(p, vel, vst, vsc, image, fold, s, &why);
  if (st != PSTM_OK) return fail(st, why);
  return PSTM_OK;
}

pstm_status pstm_migrate(pstm_plan* plan, const float* traces, int32_t trace_major,
                         const float* vel, int64_t vst, int64_t vsc, float* image, float* fold,
                         void* stream) {
  pstm_status st = pstm_load_traces(plan, traces, trace_major, stream);
  if (st != PSTM_OK) return st;
  return pstm_migrate_loaded(plan, vel, vst, vsc, image, fold, stream);
}

pstm_status pstm_fold(pstm_plan* plan, const float* vel, int64_t vst, int64_t vsc, float* fold,
                      void* stream) {
  if (!plan || !fold) return fail(PSTM_EINVAL, "null plan or fold");
  Plan* p = reinterpret_cast<Plan*>(plan);
  pstm_status st = check_velocity_args(vel, vst, vsc);
  if (st != PSTM_OK) return st;
  std::string why;
  st = launch_fold(p, vel, vst, vsc, fold, reinterpret_cast<cudaStream_t>(stream), &why);
  return st == PSTM_OK ? PSTM_OK : fail(st, why);
}

pstm_status pstm_demigrate(pstm_plan* plan, const float* image, const float* vel, int64_t vst,
                           int64_t vsc, float* traces_out, int32_t trace_major, void* stream) {
  if (!plan || !image || !traces_out) return fail(PSTM_EINVAL, "null argument");
  Plan* p = reinterpret_cast<Plan*>(plan);
  if (p->params.antialias)
    return fail(PSTM_ENOTSUP, "demigration is built for the plain (non-anti-aliased) operator");
  if (p->params.taper_width > 0 || p->params.ray_gradient != 0)
    return fail(PSTM_ENOTSUP, "demigration needs a plan built without taper_width or "
                              "ray_gradient");
  pstm_status st = check_velocity_args(vel, vst, vsc);
  if (st != PSTM_OK) return st;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const int64_t n = p->n_traces;
  const int n_s = p->n_samples;
  if (n == 0) return PSTM_OK;
  // every sample of every row is written by the adjoint kernel: no clearing
  if (!p->accum) CUDA_TRY(dalloc(p, &p->accum, (size_t)n * p->row_stride, s));
  std::string why;
  st = launch_velocity_check(p, vel, vst, vsc, s, &why);
  if (st != PSTM_OK) return fail(st, why);
  st = launch_adjoint(p, image, vel, vst, vsc, s, &why);
  if (st != PSTM_OK) return fail(st, why);
  if (trace_major) {
    unstage_rows_kernel<<<(unsigned)n, 256, 0, s>>>(p->accum, n, n_s, p->inv_perm, p->row_stride,
                                                    traces_out);
  } else {
    dim3 tb(32, 8);
    dim3 tg((unsigned)((n + 31) / 32), (unsigned)((n_s + 31) / 32));
    unstage_transpose_kernel<<<tg, tb, 0, s>>>(p->accum, n, n_s, p->inv_perm, p->row_stride,
                                               traces_out);
  }
  LAUNCH_CHECK("unstage kernel");
  return PSTM_OK;
}

pstm_status pstm_velocity_gradient(pstm_plan* plan, const float* grad_image, const float* vel,
                                   int64_t vst, int64_t vsc, float* grad_v, void* stream) {
  if (!plan || !grad_image || !grad_v) return fail(PSTM_EINVAL, "null argument");
  Plan* p = reinterpret_cast<Plan*>(plan);
  if (!p->traces_loaded) return fail(PSTM_EINVAL, "no traces loaded into the plan");
  if (p->params.weight != PSTM_WEIGHT_OBLIQUITY_SPREADING || p->params.antialias)
    return fail(PSTM_ENOTSUP, "velocity gradient is built for the plain obliquity x spreading "
                              "operator");
  if (p->params.forward_only && p->params.storage == PSTM_F32)
    return fail(PSTM_ENOTSUP, "velocity gradient needs a plan built without forward_only");
  if (p->params.taper_width > 0 || p->params.ray_gradient != 0)
    return fail(PSTM_ENOTSUP, "velocity gradient needs a plan built without taper_width or "
                              "ray_gradient");
  pstm_status st = check_velocity_args(vel, vst, vsc);
  if (st != PSTM_OK) return st;
  std::string why;
  st = launch_vgrad(p, grad_image, vel, vst, vsc, grad_v, reinterpret_cast<cudaStream_t>(stream),
                    &why);
  return st == PSTM_OK ? PSTM_OK : fail(st, why);
}

pstm_status pstm_check(pstm_plan* plan, void* stream) {
  if (!plan) return fail(PSTM_EINVAL, "null plan");
  Plan* p = reinterpret_cast<Plan*>(plan);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  int flags = 0;
  CUDA_TRY(cudaMemcpyAsync(&flags, p->err, sizeof(int), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  if (flags) CUDA_TRY(cudaMemsetAsync(p->err, 0, sizeof(int), s));
  if (flags & PSTM_ERR_TIMEOUT)
    return fail(PSTM_ETIMEOUT, "a bounded device-side wait for a trace copy expired");
  if (flags & PSTM_ERR_BOUNDS) return fail(PSTM_EBOUNDS, "device-side bounds check fired");
  if (flags & PSTM_ERR_VELOCITY)
    return fail(PSTM_EINVAL,
                "velocity must be positive and finite with V*t0 non-decreasing in t0 per column");
  return PSTM_OK;
}

static pstm_status normalize_common(const float* image, const float* fold, float* out, int64_t n,
                                    float min_fold, int mute, void* stream) {
  if (n < 0 || (n > 0 && (!image || !fold || !out))) return fail(PSTM_EINVAL, "bad arguments");
  if (n == 0) return PSTM_OK;
  const int thr = 256;
  normalize_kernel<<<(unsigned)((n + thr - 1) / thr), thr, 0,
                     reinterpret_cast<cudaStream_t>(stream)>>>(image, fold, out, n, min_fold,
                                                               mute);
  LAUNCH_CHECK("normalize_kernel");
  return PSTM_OK;
}

pstm_status pstm_normalize_by_fold(const float* image, const float* fold, float* out, int64_t n,
                                   float min_fold, void* stream) {
  return normalize_common(image, fold, out, n, min_fold, 0, stream);
}

pstm_status pstm_normalize_mute(const float* image, const float* fold, float* out, int64_t n,
                                float min_fold, void* stream) {
  return normalize_common(image, fold, out, n, min_fold, 1, stream);
}

}  // extern "C"

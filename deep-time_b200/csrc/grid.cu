// The flexure step's grid helpers around the solve, on device arrays, so that a step that keeps
// its rasters on the GPU moves them across PCIe only once (crates/deeptime-core/src/surface/
// flexure.rs:1745-1844 and surface/grid.rs:224-270):
//
//   k_restrict        restrict_by: the mean of each f x f block, its cells summed row by row;
//   k_prolong_const   coarse_cell / prolong_const: each coarse value on its f x f cells;
//   k_prolong_linear  prolong_linear / linear_at: bilinear from the coarse cells' centres, x
//                     wrapping, rows clamped;
//   k_binomial_x/_y   binomial: [1/4, 1/2, 1/4] along x (wrapping), then along y (rows clamped);
//   k_blur_rows/_cols box_blur: the running-sum box of radius r along x (wrapping or clamped),
//                     then along y (rows reflected), as many passes as asked.
//
// Every result is bit-for-bit the reference's: the same operations in the same order, and the
// products and sums that the compiler could fuse into one multiply-add written with the
// round-to-nearest intrinsics, which it never fuses. The box blur keeps the reference's running
// sums, so one thread walks each row and each column. All of these are memory-bound and small
// beside the solve; the running sums are latency-bound (one thread per row or column).
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"

namespace dt {

__global__ void k_restrict(int w, int ws, int hs, int f, double norm, const double* __restrict__ v, double* __restrict__ out) {
  const size_t n = (size_t)ws * hs;
  for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
    const size_t i = c % ws, j = c / ws;
    double s = 0.0;
    for (int dj = 0; dj < f; ++dj) {
      const double* row = v + (j * f + dj) * (size_t)w + i * f;
      for (int di = 0; di < f; ++di) s = __dadd_rn(s, row[di]);
    }
    out[c] = __dmul_rn(s, norm);
  }
}

__global__ void k_prolong_const(int ws, int hs, int f, const double* __restrict__ v, double* __restrict__ out) {
  const size_t w = (size_t)ws * f, n = w * hs * f;
  for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
    const size_t i = c % w, j = c / w;
    out[c] = v[(j / f) * ws + i / f];
  }
}

__global__ void k_prolong_linear(int ws, int hs, int f, const double* __restrict__ v, double* __restrict__ out) {
  const size_t w = (size_t)ws * f, n = w * hs * f;
  const double fd = (double)f, top = (double)(hs - 1);
  for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
    const size_t i = c % w, j = c / w;
    const double x = __dsub_rn(__ddiv_rn(__dadd_rn((double)i, 0.5), fd), 0.5);
    const double y = fmin(fmax(__dsub_rn(__ddiv_rn(__dadd_rn((double)j, 0.5), fd), 0.5), 0.0), top);
    const double x0 = floor(x), y0 = floor(y);
    const double tx = __dsub_rn(x, x0), ty = __dsub_rn(y, y0);
    long long iw = (long long)x0 % ws;
    const int i0 = (int)(iw < 0 ? iw + ws : iw), i1 = (i0 + 1) % ws;
    const int j0 = (int)y0, j1 = min(j0 + 1, hs - 1);
    const double ux = __dsub_rn(1.0, tx), uy = __dsub_rn(1.0, ty);
    const double* r0 = v + (size_t)j0 * ws;
    const double* r1 = v + (size_t)j1 * ws;
    const double a = __dadd_rn(__dmul_rn(r0[i0], ux), __dmul_rn(r0[i1], tx));
    const double b = __dadd_rn(__dmul_rn(r1[i0], ux), __dmul_rn(r1[i1], tx));
    out[c] = __dadd_rn(__dmul_rn(a, uy), __dmul_rn(b, ty));
  }
}

// 0.25 a + 0.5 b + 0.25 c, left to right, each product rounded
__device__ __forceinline__ double quarter_half_quarter(double a, double b, double c) {
  return __dadd_rn(__dadd_rn(__dmul_rn(0.25, a), __dmul_rn(0.5, b)), __dmul_rn(0.25, c));
}

__global__ void k_binomial_x(int w, int h, const double* __restrict__ v, double* __restrict__ tmp) {
  const size_t n = (size_t)w * h;
  for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
    const size_t i = c % w, row = c - i;
    tmp[c] = quarter_half_quarter(v[row + (i + w - 1) % w], v[c], v[row + (i + 1) % w]);
  }
}

__global__ void k_binomial_y(int w, int h, const double* __restrict__ tmp, double* __restrict__ v) {
  const size_t n = (size_t)w * h;
  for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
    const size_t i = c % w, j = c / w;
    const size_t no = j > 0 ? j - 1 : 0, so = min(j + 1, (size_t)h - 1);
    v[c] = quarter_half_quarter(tmp[no * w + i], tmp[c], tmp[so * w + i]);
  }
}

// One thread per row: out = the running box of radius r over the row (x wrapping or clamped).
__global__ void k_blur_rows(int w, int h, int r, bool wrap, double norm, const double* __restrict__ v,
                            double* __restrict__ out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= h) return;
  const double* src = v + (size_t)j * w;
  double* dst = out + (size_t)j * w;
  auto at = [&](long long i) -> double {
    if (wrap) {
      long long m = i % w;
      return src[m < 0 ? m + w : m];
    }
    return src[i < 0 ? 0 : (i >= w ? w - 1 : i)];
  };
  double acc = 0.0;
  for (long long i = -r; i <= r; ++i) acc = __dadd_rn(acc, at(i));
  for (long long i = 0; i < w; ++i) {
    dst[i] = __dmul_rn(acc, norm);
    acc = __dadd_rn(acc, __dsub_rn(at(i + r + 1), at(i - r)));
  }
}

// One thread per column: the running box along y, rows reflected at the edges; consecutive
// threads take consecutive columns, so every step reads and writes whole row segments.
__global__ void k_blur_cols(int w, int h, int r, double norm, const double* __restrict__ v, double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= w) return;
  auto at = [&](long long j) -> double {
    long long jj = j < 0 ? -j - 1 : (j >= h ? 2LL * h - j - 1 : j);
    jj = jj < 0 ? 0 : (jj >= h ? h - 1 : jj);
    return v[(size_t)jj * w + i];
  };
  double acc = 0.0;
  for (long long j = -r; j <= r; ++j) acc = __dadd_rn(acc, at(j));
  for (long long j = 0; j < h; ++j) {
    out[(size_t)j * w + i] = __dmul_rn(acc, norm);
    acc = __dadd_rn(acc, __dsub_rn(at(j + r + 1), at(j - r)));
  }
}

static unsigned int grid_for(size_t n) { return std::max(1u, std::min<unsigned int>(ceil_div(n, 256), 148u * 16u)); }

}  // namespace dt

using namespace dt;

extern "C" {

dt_status dt_grid_restrict_dev(int w, int h, int f, const double* fine, double* coarse, void* stream) {
  if (w < 1 || h < 1 || f < 1 || w / f < 1 || h / f < 1 || !fine || !coarse) {
    set_error("dt_grid_restrict_dev: bad arguments (w %d, h %d, f %d)", w, h, f);
    return DT_BAD_ARG;
  }
  const int ws = w / f, hs = h / f;
  const size_t n = (size_t)ws * hs;
  k_restrict<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(w, ws, hs, f, 1.0 / (double)((long long)f * f), fine, coarse);
  DT_CUDA(cudaGetLastError());
  return DT_OK;
}

dt_status dt_grid_prolong_const_dev(int ws, int hs, int f, const double* coarse, double* fine, void* stream) {
  if (ws < 1 || hs < 1 || f < 1 || !coarse || !fine) {
    set_error("dt_grid_prolong_const_dev: bad arguments (ws %d, hs %d, f %d)", ws, hs, f);
    return DT_BAD_ARG;
  }
  const size_t n = (size_t)ws * f * hs * f;
  k_prolong_const<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(ws, hs, f, coarse, fine);
  DT_CUDA(cudaGetLastError());
  return DT_OK;
}

dt_status dt_grid_prolong_linear_dev(int ws, int hs, int f, const double* coarse, double* fine, void* stream) {
  if (ws < 1 || hs < 1 || f < 1 || !coarse || !fine) {
    set_error("dt_grid_prolong_linear_dev: bad arguments (ws %d, hs %d, f %d)", ws, hs, f);
    return DT_BAD_ARG;
  }
  const size_t n = (size_t)ws * f * hs * f;
  if (f == 1) {
    DT_CUDA(cudaMemcpyAsync(fine, coarse, n * sizeof(double), cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
    return DT_OK;
  }
  k_prolong_linear<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(ws, hs, f, coarse, fine);
  DT_CUDA(cudaGetLastError());
  return DT_OK;
}

dt_status dt_grid_binomial_dev(int w, int h, int passes, double* v, double* scratch, void* stream) {
  if (w < 1 || h < 1 || passes < 0 || !v || !scratch) {
    set_error("dt_grid_binomial_dev: bad arguments (w %d, h %d, passes %d)", w, h, passes);
    return DT_BAD_ARG;
  }
  const size_t n = (size_t)w * h;
  for (int p = 0; p < passes; ++p) {
    k_binomial_x<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(w, h, v, scratch);
    k_binomial_y<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(w, h, scratch, v);
  }
  DT_CUDA(cudaGetLastError());
  return DT_OK;
}

dt_status dt_grid_box_blur_dev(int w, int h, int wrap_x, int r, int passes, double* v, double* scratch, void* stream) {
  if (w < 1 || h < 1 || r < 0 || passes < 0 || !v || !scratch) {
    set_error("dt_grid_box_blur_dev: bad arguments (w %d, h %d, r %d, passes %d)", w, h, r, passes);
    return DT_BAD_ARG;
  }
  if (r == 0) return DT_OK;
  const double norm = 1.0 / (double)(2 * r + 1);
  for (int p = 0; p < passes; ++p) {
    k_blur_rows<<<ceil_div(h, 128), 128, 0, (cudaStream_t)stream>>>(w, h, r, wrap_x != 0, norm, v, scratch);
    k_blur_cols<<<ceil_div(w, 128), 128, 0, (cudaStream_t)stream>>>(w, h, r, norm, scratch, v);
  }
  DT_CUDA(cudaGetLastError());
  return DT_OK;
}

}  // extern "C"

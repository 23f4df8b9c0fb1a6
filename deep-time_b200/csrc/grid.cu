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
// sums, so one thread walks each row and each column (k_blur_lines: a block takes 32 lines and
// streams them through a ring of 32 x 32 shared-memory tiles filled by cp.async, so that both
// directions read, and write, whole 256-byte row segments; the differences, the running sums
// and the stores run on separate warps). The element-wise helpers run on 2-D
// grids (a block's threads on consecutive columns, rows strided over the grid's y) with 32-bit
// index arithmetic; all of them are HBM-bound.
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

// The 2-D element-wise grids: blockIdx.x * blockDim.x + threadIdx.x is the column, rows go
// blockIdx.y, blockIdx.y + gridDim.y, ...
// V = 2: a thread takes columns 2c and 2c + 1 and stores them as one 16-byte word (the caller
// checks that rows start on 16 bytes: w even, out aligned)
template <int V>
__global__ void k_prolong_const(int ws, int hs, int f, const double* __restrict__ v, double* __restrict__ out) {
  const int w = ws * f, h = hs * f;
  const int i = V * (blockIdx.x * blockDim.x + threadIdx.x);
  if (i >= w) return;
  if constexpr (V == 2) {
    const int c0 = i / f, c1 = (i + 1) / f;
#pragma unroll 4
    for (int j = blockIdx.y; j < h; j += gridDim.y) {
      const double* row = v + (size_t)(j / f) * ws;
      *reinterpret_cast<double2*>(out + (size_t)j * w + i) = make_double2(row[c0], row[c1]);
    }
  } else {
    const int ci = i / f;
#pragma unroll 4
    for (int j = blockIdx.y; j < h; j += gridDim.y) out[(size_t)j * w + i] = v[(size_t)(j / f) * ws + ci];
  }
}

// The column's share of prolong_linear (the same for every row): the two coarse columns and the
// weights of the bilinear blend
struct XShare {
  int i0, i1;
  double tx, ux;
};
__device__ __forceinline__ XShare x_share(int i, int ws, double fd) {
  const double x = __dsub_rn(__ddiv_rn(__dadd_rn((double)i, 0.5), fd), 0.5);
  const double x0 = floor(x);
  XShare s;
  s.tx = __dsub_rn(x, x0);
  s.ux = __dsub_rn(1.0, s.tx);
  long long iw = (long long)x0 % ws;
  s.i0 = (int)(iw < 0 ? iw + ws : iw);
  s.i1 = (s.i0 + 1) % ws;
  return s;
}
__device__ __forceinline__ double bilinear(const double* r0, const double* r1, const XShare& s, double ty, double uy) {
  const double a = __dadd_rn(__dmul_rn(r0[s.i0], s.ux), __dmul_rn(r0[s.i1], s.tx));
  const double b = __dadd_rn(__dmul_rn(r1[s.i0], s.ux), __dmul_rn(r1[s.i1], s.tx));
  return __dadd_rn(__dmul_rn(a, uy), __dmul_rn(b, ty));
}

// 256 threads a block: the rows' shares (y, its floor and weight) are computed once per row, by
// one thread each, into shared memory, 256 rows at a time. V as in k_prolong_const.
template <int V>
__global__ void __launch_bounds__(256) k_prolong_linear(int ws, int hs, int f, const double* __restrict__ v,
                                                        double* __restrict__ out) {
  __shared__ double s_ty[256];
  __shared__ int s_j0[256];
  const int w = ws * f, h = hs * f;
  const int i = V * (blockIdx.x * blockDim.x + threadIdx.x);
  const double fd = (double)f, top = (double)(hs - 1);
  const XShare sx0 = x_share(min(i, w - 1), ws, fd);
  const XShare sx1 = x_share(min(i + V - 1, w - 1), ws, fd);
  const int step = gridDim.y;
  for (int base = blockIdx.y; base < h; base += 256 * step) {
    const int jr = base + threadIdx.x * step;
    if (jr < h) {
      const double y = fmin(fmax(__dsub_rn(__ddiv_rn(__dadd_rn((double)jr, 0.5), fd), 0.5), 0.0), top);
      const double y0 = floor(y);
      s_ty[threadIdx.x] = __dsub_rn(y, y0);
      s_j0[threadIdx.x] = (int)y0;
    }
    __syncthreads();
    if (i < w) {
      const int rows = min(256, (h - base + step - 1) / step);
#pragma unroll 2
      for (int q = 0; q < rows; ++q) {
        const int j = base + q * step;
        const double ty = s_ty[q], uy = __dsub_rn(1.0, ty);
        const int j0 = s_j0[q], j1 = min(j0 + 1, hs - 1);
        const double* r0 = v + (size_t)j0 * ws;
        const double* r1 = v + (size_t)j1 * ws;
        if constexpr (V == 2) {
          *reinterpret_cast<double2*>(out + (size_t)j * w + i) =
              make_double2(bilinear(r0, r1, sx0, ty, uy), bilinear(r0, r1, sx1, ty, uy));
        } else {
          out[(size_t)j * w + i] = bilinear(r0, r1, sx0, ty, uy);
        }
      }
    }
    __syncthreads();
  }
}

// 0.25 a + 0.5 b + 0.25 c, left to right, each product rounded
__device__ __forceinline__ double quarter_half_quarter(double a, double b, double c) {
  return __dadd_rn(__dadd_rn(__dmul_rn(0.25, a), __dmul_rn(0.5, b)), __dmul_rn(0.25, c));
}

__global__ void k_binomial_x(int w, int h, const double* __restrict__ v, double* __restrict__ tmp) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= w) return;
  const int west = i == 0 ? w - 1 : i - 1, east = i + 1 == w ? 0 : i + 1;
  for (int j = blockIdx.y; j < h; j += gridDim.y) {
    const double* row = v + (size_t)j * w;
    tmp[(size_t)j * w + i] = quarter_half_quarter(row[west], row[i], row[east]);
  }
}

__global__ void k_binomial_y(int w, int h, const double* __restrict__ tmp, double* __restrict__ v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= w) return;
  for (int j = blockIdx.y; j < h; j += gridDim.y) {
    const int no = j > 0 ? j - 1 : 0, so = min(j + 1, h - 1);
    v[(size_t)j * w + i] = quarter_half_quarter(tmp[(size_t)no * w + i], tmp[(size_t)j * w + i], tmp[(size_t)so * w + i]);
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

// The box blur's running sums with the lines streamed through shared memory. A block takes 32
// lines (rows with ROWS, else columns); line line0 + l is lane l's: out(k) = acc (1 / (2r + 1)),
// acc += v(k + r + 1) - v(k - r), with acc started as the sum of v(-r .. r) in order, the
// reference's loop bit for bit. Only the running sum is serial, so six warps split the work, one
// tile of 32 positions a step, skewed by a step and separated by one block barrier a step:
//   warp 1  the loader: keeps up to RING / 32 - B - 1 tiles ahead in flight, 8-byte cp.async
//           copies of one 256-byte row segment per line (ROWS) or per position (columns), into a
//           ring of RING positions per line;
//   warps 2-5  the differences d(k) = v(k + r + 1) - v(k - r) of step s's tile (8 positions
//           each) from the ring, or from global memory past the line's ends (wrap, clamp or
//           reflection); and the stores of step s - 2's sums times 1 / (2r + 1), whole row
//           segments in both directions;
//   warp 0  the running sum over step s - 1's differences.
// The ring is line-major with ROWS (a line's RING positions contiguous, pitch RING + 1) and
// position-major for columns (pitch 33), both free of bank conflicts for the accesses they get,
// and a position's place in it is k & (RING - 1). B = ceil((r + 1) / 32) (1 or 2, so r <= 63):
// the ring holds tiles s - B .. s + B while step s's differences are taken. The row pass has one
// block per 32 rows, fewer than the SMs on the rasters it is meant for, so its ring is deep (512
// positions, one block an SM); the column pass has twice the blocks and keeps two an SM (256).
constexpr int BL_PITCH = 33;
constexpr int BL_TILE = 32 * BL_PITCH;
constexpr int BL_THREADS = 192;
constexpr int BL_RING_ROWS = 512;
constexpr int BL_RING_COLS = 256;

template <bool ROWS>
constexpr size_t blur_lines_smem() {
  return sizeof(double) * ((ROWS ? 32 * (BL_RING_ROWS + 1) : BL_RING_COLS * BL_PITCH) + 4 * BL_TILE);
}

__device__ __forceinline__ void cp_async8(double* dst, const double* src) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

template <bool ROWS, int B>
__global__ void __launch_bounds__(BL_THREADS) k_blur_lines(int w, int h, int r, bool wrap, double norm,
                                                           const double* __restrict__ v, double* __restrict__ out) {
  constexpr int RING = ROWS ? BL_RING_ROWS : BL_RING_COLS;
  constexpr int MASK = RING - 1;
  constexpr int RP = ROWS ? RING + 1 : BL_PITCH;  // ring pitch: per line (ROWS) or per position
  constexpr int AHEAD = RING / 32 - B - 1;        // tiles in flight beyond the one differenced
  constexpr int PENDING = AHEAD - B - 1;          // copy groups left pending once tiles <= s + B + 1 landed
  static_assert(PENDING >= 0, "the ring must hold the window's tiles and one step ahead");
  extern __shared__ double bl_smem[];
  double* const ring = bl_smem;
  double* const dif = bl_smem + (ROWS ? 32 * RP : RING * RP);  // two tiles of differences
  double* const sum = dif + 2 * BL_TILE;                       // two tiles of running sums
  const int lines = ROWS ? h : w, len = ROWS ? w : h;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int line0 = blockIdx.x * 32, line = line0 + lane;
  const bool mine = line < lines, full_block = line0 + 32 <= lines;
  const int tiles = (len + 31) >> 5;
  // this lane's line in the ring: position k at mine_ring[(k & MASK) * step]
  const double* const my_ring = ROWS ? ring + lane * RP : ring + lane;
  constexpr int KSTEP = ROWS ? 1 : RP;

  auto issue = [&](int t) {
    if (t < tiles) {
      const int k0 = 32 * t;
      if (full_block && k0 + 32 <= len) {
        if (ROWS) {
          const double* src = v + (size_t)line0 * len + k0 + lane;
          double* dst = ring + ((k0 + lane) & MASK);
#pragma unroll 8
          for (int rr = 0; rr < 32; ++rr, src += len, dst += RP) cp_async8(dst, src);
        } else {
          const double* src = v + (size_t)k0 * w + line;
          double* dst = ring + (k0 & MASK) * RP + lane;
#pragma unroll 8
          for (int rr = 0; rr < 32; ++rr, src += w, dst += RP) cp_async8(dst, src);
        }
      } else {
        for (int rr = 0; rr < 32; ++rr) {
          if (ROWS) {
            const int ln = line0 + rr, pos = k0 + lane;
            if (ln < lines && pos < len) cp_async8(ring + rr * RP + (pos & MASK), v + (size_t)ln * len + pos);
          } else {
            const int pos = k0 + rr;
            if (mine && pos < len) cp_async8(ring + (pos & MASK) * RP + lane, v + (size_t)pos * w + line);
          }
        }
      }
    }
    cp_async_commit();  // one group per tile, empty past the end, so that the wait counts stay fixed
  };
  // the cell the reference reads for position k of this lane's line
  auto global_at = [&](int k) -> double {
    int m;
    if (ROWS) {
      if (wrap) {
        m = k % len;
        m = m < 0 ? m + len : m;
      } else {
        m = k < 0 ? 0 : (k >= len ? len - 1 : k);
      }
      return v[(size_t)line * len + m];
    }
    m = k < 0 ? -k - 1 : (k >= len ? 2 * len - k - 1 : k);
    m = m < 0 ? 0 : (m >= len ? len - 1 : m);
    return v[(size_t)m * w + line];
  };
  // inside the line: from the ring (the caller keeps k within the resident tiles)
  auto ring_at = [&](int k) -> double { return my_ring[(k & MASK) * KSTEP]; };
  auto at = [&](int k) -> double { return (k < 0 || k >= len) ? global_at(k) : ring_at(k); };

  if (warp == 1) {
    for (int t = 0; t < AHEAD; ++t) issue(t);
    cp_async_wait<PENDING>();  // tiles <= B landed
  }
  __syncthreads();
  double acc = 0.0;
  if (warp == 0 && mine)
    for (int k = -r; k <= r; ++k) acc = __dadd_rn(acc, at(k));
  for (int s = 0; s < tiles + 2; ++s) {
    if (warp == 1) {
      // its ring positions held tile s - B - 1's, which step s - 1 read last
      issue(s + AHEAD);
      cp_async_wait<PENDING>();  // tiles <= s + B + 1 landed, for the next step's differences
    } else if (warp >= 2) {
      const int part = (warp - 2) * 8;
      if (s < tiles && mine) {
        const int k0 = 32 * s;
        double* d = dif + (s & 1) * BL_TILE + lane * BL_PITCH + part;
        const int kh = k0 + part + r + 1, kl = k0 + part - r;
        if (k0 + 32 <= len && k0 - r >= 0 && k0 + 32 + r < len) {
          // every read before the first store: the tiles share one shared-memory array, so the
          // compiler would not move a read above a store
          double hi[8], lo[8];
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            hi[u] = ring_at(kh + u);
            lo[u] = ring_at(kl + u);
          }
#pragma unroll
          for (int u = 0; u < 8; ++u) d[u] = __dsub_rn(hi[u], lo[u]);
        } else {
          const int n = min(8, len - k0 - part);
          for (int u = 0; u < n; ++u) d[u] = __dsub_rn(at(kh + u), at(kl + u));
        }
      }
      if (s >= 2) {
        const int q = s - 2;  // the sums the running-sum warp finished a step ago
        const double* a = sum + (q & 1) * BL_TILE;
        if (ROWS) {
          const int pos = 32 * q + lane;
          if (pos < len) {
            const double* ar = a + part * BL_PITCH + lane;
            double* o = out + (size_t)(line0 + part) * len + pos;
            if (full_block) {
#pragma unroll
              for (int u = 0; u < 8; ++u) o[(size_t)u * len] = __dmul_rn(ar[u * BL_PITCH], norm);
            } else {
              for (int u = 0; u < 8 && line0 + part + u < lines; ++u) o[(size_t)u * len] = __dmul_rn(ar[u * BL_PITCH], norm);
            }
          }
        } else if (mine) {
          const int p0 = 32 * q + part;
          const double* ar = a + lane * BL_PITCH + part;
          double* o = out + (size_t)p0 * w + line;
          if (p0 + 8 <= len) {
#pragma unroll
            for (int u = 0; u < 8; ++u) o[(size_t)u * w] = __dmul_rn(ar[u], norm);
          } else {
            for (int u = 0; p0 + u < len; ++u) o[(size_t)u * w] = __dmul_rn(ar[u], norm);
          }
        }
      }
    } else if (s >= 1 && s <= tiles && mine) {
      // warp 0: the running sum over the previous step's differences
      const int q = s - 1;
      const double* d = dif + (q & 1) * BL_TILE + lane * BL_PITCH;
      double* a = sum + (q & 1) * BL_TILE + lane * BL_PITCH;
      const int kend = min(32, len - 32 * q);
      if (kend == 32) {
        double x[32];  // the reads first, then the serial sum (see the differences above)
#pragma unroll
        for (int kk = 0; kk < 32; ++kk) x[kk] = d[kk];
#pragma unroll
        for (int kk = 0; kk < 32; ++kk) {
          a[kk] = acc;
          acc = __dadd_rn(acc, x[kk]);
        }
      } else {
        for (int kk = 0; kk < kend; ++kk) {
          a[kk] = acc;
          acc = __dadd_rn(acc, d[kk]);
        }
      }
    }
    __syncthreads();
  }
  if (warp == 1) cp_async_wait<0>();
}

static unsigned int grid_for(size_t n) { return std::max(1u, std::min<unsigned int>(ceil_div(n, 256), 148u * 16u)); }

// 2-D grid for w columns and h rows: 256 columns a block, about 16 blocks per SM in all
static dim3 grid2d(int w, int h) {
  const unsigned gx = (unsigned)ceil_div((size_t)w, 256);
  const unsigned gy = (unsigned)std::max<size_t>(1, std::min<size_t>((size_t)h, ceil_div((size_t)148 * 16, gx)));
  return dim3(gx, std::min(gy, 65535u));
}

// Column pairs as 16-byte stores: every row must start on 16 bytes
static bool prolong_pairs(int w, const double* out) { return (w % 2) == 0 && ((uintptr_t)out % 16) == 0; }

// The box blur's line kernel for one direction: false when r is too wide for its ring.
template <bool ROWS>
static bool launch_blur_lines(int w, int h, int r, bool wrap, double norm, const double* v, double* out, cudaStream_t st) {
  const int lines = ROWS ? h : w;
  constexpr size_t smem = blur_lines_smem<ROWS>();
  const unsigned blocks = (unsigned)ceil_div((size_t)lines, 32);
  if (r + 1 <= 32) {
    cudaFuncSetAttribute(k_blur_lines<ROWS, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_blur_lines<ROWS, 1><<<blocks, BL_THREADS, smem, st>>>(w, h, r, wrap, norm, v, out);
    return true;
  }
  if (r + 1 <= 64) {
    cudaFuncSetAttribute(k_blur_lines<ROWS, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_blur_lines<ROWS, 2><<<blocks, BL_THREADS, smem, st>>>(w, h, r, wrap, norm, v, out);
    return true;
  }
  return false;
}

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
  if (prolong_pairs(ws * f, fine)) {
    k_prolong_const<2><<<grid2d((ws * f) / 2, hs * f), 256, 0, (cudaStream_t)stream>>>(ws, hs, f, coarse, fine);
  } else {
    k_prolong_const<1><<<grid2d(ws * f, hs * f), 256, 0, (cudaStream_t)stream>>>(ws, hs, f, coarse, fine);
  }
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
  if (prolong_pairs(ws * f, fine)) {
    k_prolong_linear<2><<<grid2d((ws * f) / 2, hs * f), 256, 0, (cudaStream_t)stream>>>(ws, hs, f, coarse, fine);
  } else {
    k_prolong_linear<1><<<grid2d(ws * f, hs * f), 256, 0, (cudaStream_t)stream>>>(ws, hs, f, coarse, fine);
  }
  DT_CUDA(cudaGetLastError());
  return DT_OK;
}

dt_status dt_grid_binomial_dev(int w, int h, int passes, double* v, double* scratch, void* stream) {
  if (w < 1 || h < 1 || passes < 0 || !v || !scratch) {
    set_error("dt_grid_binomial_dev: bad arguments (w %d, h %d, passes %d)", w, h, passes);
    return DT_BAD_ARG;
  }
  for (int p = 0; p < passes; ++p) {
    k_binomial_x<<<grid2d(w, h), 256, 0, (cudaStream_t)stream>>>(w, h, v, scratch);
    k_binomial_y<<<grid2d(w, h), 256, 0, (cudaStream_t)stream>>>(w, h, scratch, v);
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
  cudaStream_t st = (cudaStream_t)stream;
  for (int p = 0; p < passes; ++p) {
    // radii past the ring's reach (r > 63) take the plain one-thread-per-line kernels
    if (!launch_blur_lines<true>(w, h, r, wrap_x != 0, norm, v, scratch, st))
      k_blur_rows<<<ceil_div(h, 128), 128, 0, st>>>(w, h, r, wrap_x != 0, norm, v, scratch);
    if (!launch_blur_lines<false>(w, h, r, false, norm, scratch, v, st))
      k_blur_cols<<<ceil_div(w, 128), 128, 0, st>>>(w, h, r, norm, scratch, v);
  }
  DT_CUDA(cudaGetLastError());
  return DT_OK;
}

}  // extern "C"

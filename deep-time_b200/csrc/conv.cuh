// 3 x 3 convolutions for the flexure warm-start U-Net: implicit GEMM on the tensor cores, BF16
// operands, FP32 accumulation.
//
// Layout: activations NHWC (channels innermost), BF16; a tensor is addressed by a pixel stride
// (channels per pixel of the buffer) and a channel offset, so a layer can read or write a slice
// of a concatenated buffer. Padding is periodic in x (the raster wraps east-west) and zero in y,
// which makes the gradient with respect to the input the same kernel run on the output gradient
// with the taps mirrored and the weight matrix transposed.
//
// Forward / input-gradient: out[p][co] = sum_{tap, ci} in[p + off(tap)][ci] W[tap][ci][co], a GEMM
// with M = pixels, N = output channels, K = 9 x input channels. A block computes 64 consecutive
// pixels of one image row by BN output channels; K advances one tap and 32 input channels at a
// time. Tiles are staged by cp.async in two stages, fragments are loaded with ldmatrix (x4 for A,
// x4.trans for B, both from XOR-swizzled shared memory) and multiplied with
// mma.sync.m16n8k16.row.col.f32.bf16.bf16.f32; 4 warps as 2 x 2, each 32 x (BN / 2).
//
// Weight gradient: dW[tap][ci][co] = sum_p in[p + off(tap)][ci] g[p][co], a GEMM with M = input
// channels, N = output channels, K = pixels; each block reduces a chunk of pixel tiles and writes
// a partial tile, and a second pass sums the partials in a fixed order (deterministic).
#pragma once
#include <cuda_bf16.h>

#include "common.cuh"

namespace dt {

typedef __nv_bfloat16 bf16;

struct Tensor4 {
  bf16* p;      // base of the buffer
  int stride;   // channels per pixel of the buffer
  int off;      // first channel of this tensor
  int c;        // channels of this tensor
};

__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
  unsigned s = smem_addr(smem);
  int n = valid ? 16 : 0;  // zero-fill when the source is padding
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ void ldmatrix_x4(unsigned& r0, unsigned& r1, unsigned& r2, unsigned& r3, const void* p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(smem_addr(p)));
}
__device__ __forceinline__ void ldmatrix_x4_trans(unsigned& r0, unsigned& r1, unsigned& r2, unsigned& r3, const void* p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(smem_addr(p)));
}

__device__ __forceinline__ void mma_bf16(float* d, const unsigned* a, const unsigned* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Swizzled offsets (in bf16 elements) of 16-byte chunk `chunk` of row `row`:
// A tiles are rows of 32 bf16 (4 chunks, 64 B); B tiles are rows of BN bf16 (BN/8 chunks).
__device__ __forceinline__ int swz_a(int row, int chunk) { return row * 32 + ((chunk ^ ((row >> 1) & 3)) << 3); }
template <int BN>
__device__ __forceinline__ int swz_b(int row, int chunk) {
  if (BN == 32) return row * 32 + ((chunk ^ ((row >> 1) & 3)) << 3);  // 64-byte rows, as swz_a
  return row * BN + ((chunk ^ (row & 7)) << 3);                       // 128-byte rows
}

enum { EPI_BIAS_RELU = 0, EPI_BIAS = 1, EPI_STORE = 2, EPI_ACCUM = 3, EPI_MASK = 4 };

// One 3 x 3 convolution (or its input gradient with mirrored, transposed weights): W is
// [9][Cin][Cout] bf16, tap = ky * 3 + kx reading in[y + ky - 1][x + kx - 1]. Image rows of width
// `w` (a multiple of 64), `h` rows, `nimg` images.
template <int BN, int EPI>
__global__ void __launch_bounds__(128) k_conv3x3(int nimg, int h, int w, Tensor4 in, const bf16* __restrict__ W,
                                                 const float* __restrict__ bias, Tensor4 out, Tensor4 mask) {
  constexpr int BM = 64, BK = 32;
  __shared__ __align__(128) bf16 sA[2][BM * BK];
  __shared__ __align__(128) bf16 sB[2][BK * BN];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1;  // warp tile: rows wm*32.., cols wn*(BN/2)..
  const int tiles_x = w / BM;
  int bid = blockIdx.x;
  const int xt = bid % tiles_x;
  bid /= tiles_x;
  const int y = bid % h;
  const int n = bid / h;
  const int x0 = xt * BM;
  const int co0 = blockIdx.y * BN;
  const int cin = in.c;
  const int kchunks = 9 * (cin / BK);
  constexpr int NT = BN / 16;  // n8 tiles per warp
  float acc[2][NT][4];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < NT; ++b)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[a][b][c] = 0.f;

  auto load = [&](int kc, int stage) {
    int tap = kc / (cin / BK);
    int ci0 = (kc % (cin / BK)) * BK;
    int ky = tap / 3, kx = tap % 3;
    int yy = y + ky - 1;
    bool yok = yy >= 0 && yy < h;
    // A: 64 pixels x 32 channels = 256 chunks of 16 B; 2 a thread
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      int cidx = tid + q * 128;
      int row = cidx >> 2, ch = cidx & 3;
      int xx = x0 + row + kx - 1;
      xx = xx < 0 ? xx + w : (xx >= w ? xx - w : xx);
      const bf16* src = in.p + ((size_t)((size_t)n * h + (yok ? yy : 0)) * w + xx) * in.stride + in.off + ci0 + ch * 8;
      cp_async16(&sA[stage][swz_a(row, ch)], src, yok);
    }
    // B: 32 k-rows x BN channels
    constexpr int BCH = BK * BN / 8;
#pragma unroll
    for (int q = 0; q < (BCH + 127) / 128; ++q) {
      int cidx = tid + q * 128;
      if (cidx < BCH) {
        int row = cidx / (BN / 8), ch = cidx % (BN / 8);
        const bf16* src = W + ((size_t)tap * cin + ci0 + row) * out.c + co0 + ch * 8;
        cp_async16(&sB[stage][swz_b<BN>(row, ch)], src, true);
      }
    }
    cp_async_commit();
  };

  load(0, 0);
  for (int kc = 0; kc < kchunks; ++kc) {
    int stage = kc & 1;
    if (kc + 1 < kchunks) {
      load(kc + 1, stage ^ 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; kk += 16) {
      unsigned af[2][4];
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) {
        int row = wm * 32 + mt * 16 + (lane & 15);
        int chunk = (kk >> 3) + (lane >> 4);
        ldmatrix_x4(af[mt][0], af[mt][1], af[mt][2], af[mt][3], &sA[stage][swz_a(row, chunk)]);
      }
      unsigned bfr[NT][2];
#pragma unroll
      for (int nt = 0; nt < NT; nt += 2) {
        int krow = kk + (lane & 15);
        int chunk = (wn * (BN / 2) + nt * 8) / 8 + (lane >> 4);
        unsigned r0, r1, r2, r3;
        ldmatrix_x4_trans(r0, r1, r2, r3, &sB[stage][swz_b<BN>(krow, chunk)]);
        bfr[nt][0] = r0;
        bfr[nt][1] = r1;
        bfr[nt + 1][0] = r2;
        bfr[nt + 1][1] = r3;
      }
#pragma unroll
      for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) mma_bf16(acc[mt][nt], af[mt], bfr[nt]);
    }
    __syncthreads();
  }
  // epilogue: rows = pixels, cols = output channels
  const int g = lane >> 2, t4 = lane & 3;
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      int row = wm * 32 + mt * 16 + g + half * 8;
      size_t pix = ((size_t)n * h + y) * w + x0 + row;
      bf16* dst = out.p + pix * out.stride + out.off + co0;
#pragma unroll
      for (int nt = 0; nt < NT; ++nt) {
        int col = wn * (BN / 2) + nt * 8 + t4 * 2;
        float v0 = acc[mt][nt][half * 2], v1 = acc[mt][nt][half * 2 + 1];
        if (EPI == EPI_BIAS_RELU || EPI == EPI_BIAS) {
          v0 += bias[co0 + col];
          v1 += bias[co0 + col + 1];
        }
        if (EPI == EPI_BIAS_RELU) {
          v0 = fmaxf(v0, 0.f);
          v1 = fmaxf(v1, 0.f);
        }
        __nv_bfloat162* d2 = reinterpret_cast<__nv_bfloat162*>(dst + col);
        if (EPI == EPI_MASK) {
          // the gradient through the producing ReLU: zero where its output was zero
          __nv_bfloat162 m = *reinterpret_cast<const __nv_bfloat162*>(mask.p + pix * mask.stride + mask.off + co0 + col);
          if (!(__bfloat162float(m.x) > 0.f)) v0 = 0.f;
          if (!(__bfloat162float(m.y) > 0.f)) v1 = 0.f;
        }
        if (EPI == EPI_ACCUM) {
          __nv_bfloat162 prev = *d2;
          v0 += __bfloat162float(prev.x);
          v1 += __bfloat162float(prev.y);
        }
        *d2 = __floats2bfloat162_rn(v0, v1);
      }
    }
}

// Weight gradient partials: block (tap, ci tile of 64, co tile of BN) x chunk of pixel tiles.
// part[chunk][tap][ci][co] (FP32).
template <int BN>
__global__ void __launch_bounds__(128) k_conv3x3_wgrad(int nimg, int h, int w, Tensor4 in, Tensor4 g, int tiles_per_chunk,
                                                       float* __restrict__ part) {
  constexpr int BM = 64;  // input channels per block (GEMM M)
  constexpr int BK = 32;  // pixels per k step
  __shared__ __align__(128) bf16 sA[2][BK * BM];  // [pixel][ci] : 32 rows of 64 channels
  __shared__ __align__(128) bf16 sB[2][BK * BN];  // [pixel][co]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1;
  const int cin = in.c, cout = g.c;
  const int ci_tiles = (cin + BM - 1) / BM;
  int bx = blockIdx.x;
  const int co0 = (bx % (cout / BN)) * BN;
  bx /= cout / BN;
  const int ci0 = (bx % ci_tiles) * BM;
  const int tap = bx / ci_tiles;
  const int ky = tap / 3, kx = tap % 3;
  const int chunk = blockIdx.y;
  const int tiles_x = w / BK;
  const int total_tiles = nimg * h * tiles_x;
  constexpr int NT = BN / 16;
  float acc[2][NT][4];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < NT; ++b)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[a][b][c] = 0.f;
  const int t_begin = chunk * tiles_per_chunk;
  const int t_end = min(total_tiles, t_begin + tiles_per_chunk);

  auto load = [&](int t, int stage) {
    int xt = t % tiles_x;
    int rest = t / tiles_x;
    int y = rest % h, n = rest / h;
    int x0 = xt * BK;
    int yy = y + ky - 1;
    bool yok = yy >= 0 && yy < h;
    // A: 32 pixels x 64 channels (shifted by the tap) = 256 chunks
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      int cidx = tid + q * 128;
      int row = cidx >> 3, ch = cidx & 7;
      int xx = x0 + row + kx - 1;
      xx = xx < 0 ? xx + w : (xx >= w ? xx - w : xx);
      bool ok = yok && (ci0 + ch * 8 < cin);
      const bf16* src = in.p + ((size_t)((size_t)n * h + (yok ? yy : 0)) * w + xx) * in.stride + in.off + (ok ? ci0 + ch * 8 : 0);
      cp_async16(&sA[stage][swz_b<BM>(row, ch)], src, ok);
    }
    // B: 32 pixels x BN output-channel gradients
    constexpr int BCH = BK * BN / 8;
#pragma unroll
    for (int q = 0; q < (BCH + 127) / 128; ++q) {
      int cidx = tid + q * 128;
      if (cidx < BCH) {
        int row = cidx / (BN / 8), ch = cidx % (BN / 8);
        const bf16* src = g.p + ((size_t)((size_t)n * h + y) * w + x0 + row) * g.stride + g.off + co0 + ch * 8;
        cp_async16(&sB[stage][swz_b<BN>(row, ch)], src, true);
      }
    }
    cp_async_commit();
  };

  if (t_begin < t_end) {
    load(t_begin, 0);
    for (int t = t_begin; t < t_end; ++t) {
      int stage = (t - t_begin) & 1;
      if (t + 1 < t_end) {
        load(t + 1, stage ^ 1);
        cp_async_wait<1>();
      } else {
        cp_async_wait<0>();
      }
      __syncthreads();
#pragma unroll
      for (int kk = 0; kk < BK; kk += 16) {
        // A = in^T: rows ci, cols pixels; the tile is [pixel][ci], so load transposed
        unsigned af[2][4];
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
          // matrices: (ci 0-7, px 0-7), (ci 8-15, px 0-7), (ci 0-7, px 8-15), (ci 8-15, px 8-15)
          int prow = kk + (lane & 7) + ((lane >> 4) << 3);
          int chunk = (wm * 32 + mt * 16) / 8 + ((lane >> 3) & 1);
          ldmatrix_x4_trans(af[mt][0], af[mt][1], af[mt][2], af[mt][3], &sA[stage][swz_b<BM>(prow, chunk)]);
        }
        unsigned bfr[NT][2];
#pragma unroll
        for (int nt = 0; nt < NT; nt += 2) {
          int krow = kk + (lane & 15);
          int chunk = (wn * (BN / 2) + nt * 8) / 8 + (lane >> 4);
          unsigned r0, r1, r2, r3;
          ldmatrix_x4_trans(r0, r1, r2, r3, &sB[stage][swz_b<BN>(krow, chunk)]);
          bfr[nt][0] = r0;
          bfr[nt][1] = r1;
          bfr[nt + 1][0] = r2;
          bfr[nt + 1][1] = r3;
        }
#pragma unroll
        for (int mt = 0; mt < 2; ++mt)
#pragma unroll
          for (int nt = 0; nt < NT; ++nt) mma_bf16(acc[mt][nt], af[mt], bfr[nt]);
      }
      __syncthreads();
    }
  }
  const int gq = lane >> 2, t4 = lane & 3;
  float* dst = part + ((size_t)chunk * 9 + tap) * cin * cout;
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      int ci = ci0 + wm * 32 + mt * 16 + gq + half * 8;
      if (ci >= cin) continue;
#pragma unroll
      for (int nt = 0; nt < NT; ++nt) {
        int co = co0 + wn * (BN / 2) + nt * 8 + t4 * 2;
        dst[(size_t)ci * cout + co] = acc[mt][nt][half * 2];
        dst[(size_t)ci * cout + co + 1] = acc[mt][nt][half * 2 + 1];
      }
    }
}

}  // namespace dt

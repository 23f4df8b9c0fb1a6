// The flexure warm-start U-Net on the B200: forward, backward and Adam, all on this project's
// kernels (conv.cuh for the 3 x 3 convolutions on the tensor cores).
//
// The model: 4 levels with 32, 64, 128, 256 channels; two 3 x 3 convolutions with ReLU per level
// on the way down, 2 x 2 average pooling between levels, nearest-neighbour upsampling and a
// concatenation with the level's skip on the way up, two 3 x 3 convolutions with ReLU per level,
// and a 1 x 1 convolution to one output channel. Input: two channels (the load and log10 of the
// rigidity, normalised), zero-padded to 32 so every layer's input is a multiple of 32 channels.
// Weights and activations are BF16, accumulation FP32; the optimiser keeps FP32 master weights.
//
// Buffers are NHWC. The encoder's second convolution of levels 0..2 writes straight into the
// skip slice of that level's decoder input buffer; the upsampled decoder output fills the other
// slice, so the concatenation is free.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "conv.cuh"
#include "conv_tc.cuh"
#include <cstdlib>

namespace dt {

constexpr int UNET_LEVELS = 4;
constexpr int UNET_IN_PAD = 32;

struct ConvLayer {
  int cin, cout;
  size_t w_off, b_off;  // offsets into the FP32 parameter array
  bf16 *W, *WT;         // [9][cin][cout] and the mirrored, transposed [9][cout][cin]
};

// Per-level activation buffers for a batch of one shape.
struct LevelBufs {
  int h, w;
  bf16 *A, *gA;    // first conv output (and its gradient)
  bf16 *U, *gU;    // decoder input: [up | skip] (levels 0..2); level 3: the bottleneck output
  bf16 *P, *gP;    // the pooled skip (input of the next level)
  bf16 *DA, *gDA;  // decoder first conv output
  bf16 *DB, *gDB;  // decoder second conv output
  int cu;          // channels of U
};

// A pixel's UNET_IN_PAD channels are UNET_IN_PAD / 8 words of 16 bytes; consecutive threads write
// consecutive words (the first of a pixel holds its two input channels, the rest zeros).
__global__ void k_pack_input(size_t npix, const float* __restrict__ x, bf16* __restrict__ out) {
  constexpr int WPP = UNET_IN_PAD / 8;
  static_assert(WPP * 8 == UNET_IN_PAD && (WPP & (WPP - 1)) == 0, "whole 16-byte words per pixel");
  uint4* o = reinterpret_cast<uint4*>(out);
  const size_t nw = npix * WPP;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < nw; q += (size_t)gridDim.x * blockDim.x) {
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    if ((q & (WPP - 1)) == 0) {
      const size_t p = q / WPP;
      __nv_bfloat162 b = __floats2bfloat162_rn(x[2 * p], x[2 * p + 1]);
      v.x = *reinterpret_cast<const unsigned int*>(&b);
    }
    o[q] = v;
  }
}

// 2 x 2 average pooling: out[n][y][x][c] = mean of in[n][2y..][2x..][c]
// Eight channels (16 bytes) at a time: every channel count, stride and offset here is a
// multiple of 8, and pixel counts fit 32 bits.
__device__ __forceinline__ void bf8_to_f(uint4 v, float* f) {
  const __nv_bfloat162* b = reinterpret_cast<const __nv_bfloat162*>(&v);
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    float2 t = __bfloat1622float2(b[e]);
    f[2 * e] = t.x;
    f[2 * e + 1] = t.y;
  }
}
__device__ __forceinline__ uint4 f_to_bf8(const float* f) {
  uint4 v;
  __nv_bfloat162* b = reinterpret_cast<__nv_bfloat162*>(&v);
#pragma unroll
  for (int e = 0; e < 4; ++e) b[e] = __floats2bfloat162_rn(f[2 * e], f[2 * e + 1]);
  return v;
}

__global__ void k_pool(int nimg, int h, int w, Tensor4 in, Tensor4 out) {
  const int ho = h / 2, wo = w / 2, c8 = in.c / 8;
  const unsigned total = (unsigned)nimg * ho * wo * c8;
  for (unsigned k = blockIdx.x * blockDim.x + threadIdx.x; k < total; k += gridDim.x * blockDim.x) {
    unsigned c = k % c8, p = k / c8;
    unsigned x = p % wo, r = p / wo, y = r % ho, n = r / ho;
    float s[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int dy = 0; dy < 2; ++dy)
#pragma unroll
      for (int dx = 0; dx < 2; ++dx) {
        size_t q = ((size_t)(n * h + 2 * y + dy) * w + 2 * x + dx) * in.stride + in.off + c * 8;
        float f[8];
        bf8_to_f(*reinterpret_cast<const uint4*>(in.p + q), f);
#pragma unroll
        for (int e = 0; e < 8; ++e) s[e] += f[e];
      }
#pragma unroll
    for (int e = 0; e < 8; ++e) s[e] *= 0.25f;
    *reinterpret_cast<uint4*>(out.p + (size_t)p * out.stride + out.off + c * 8) = f_to_bf8(s);
  }
}

// nearest-neighbour upsampling into a slice: out[n][y][x][c] = in[n][y/2][x/2][c]
__global__ void k_upsample(int nimg, int h, int w, Tensor4 in, Tensor4 out) {
  const int hi = h / 2, wi = w / 2, c8 = in.c / 8;
  const unsigned total = (unsigned)nimg * h * w * c8;
  for (unsigned k = blockIdx.x * blockDim.x + threadIdx.x; k < total; k += gridDim.x * blockDim.x) {
    unsigned c = k % c8, p = k / c8;
    unsigned x = p % w, r = p / w, y = r % h, n = r / h;
    size_t src = ((size_t)(n * hi + y / 2) * wi + x / 2) * in.stride + in.off + c * 8;
    *reinterpret_cast<uint4*>(out.p + (size_t)p * out.stride + out.off + c * 8) = *reinterpret_cast<const uint4*>(in.p + src);
  }
}

// gradient through upsampling and the producing ReLU: g[p][c] = (sum of the 2 x 2 children's
// gradients) where act > 0, else 0
__global__ void k_upsample_bwd_mask(int nimg, int h, int w, Tensor4 gup, Tensor4 act, Tensor4 g) {
  // (h, w): the coarse level's shape; children at 2y.., 2x..
  size_t total = (size_t)nimg * h * w * g.c;
  int hf = 2 * h, wf = 2 * w;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < total; k += (size_t)gridDim.x * blockDim.x) {
    int c = (int)(k % g.c);
    size_t p = k / g.c;
    int x = (int)(p % w), y = (int)((p / w) % h);
    size_t n = p / ((size_t)w * h);
    float s = 0.f;
    for (int dy = 0; dy < 2; ++dy)
      for (int dx = 0; dx < 2; ++dx)
        s += __bfloat162float(gup.p[(((n * hf) + 2 * y + dy) * wf + 2 * x + dx) * gup.stride + gup.off + c]);
    float a = __bfloat162float(act.p[p * act.stride + act.off + c]);
    g.p[p * g.stride + g.off + c] = __float2bfloat16(a > 0.f ? s : 0.f);
  }
}

// gradient of an encoder level's output: its skip gradient plus the pooling's (1/4 of the parent
// cell's), through the ReLU; written over the skip slice
__global__ void k_skip_pool_bwd_mask(int nimg, int h, int w, Tensor4 gskip, Tensor4 gpool, Tensor4 act) {
  size_t total = (size_t)nimg * h * w * act.c;
  int hc = h / 2, wc = w / 2;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < total; k += (size_t)gridDim.x * blockDim.x) {
    int c = (int)(k % act.c);
    size_t p = k / act.c;
    int x = (int)(p % w), y = (int)((p / w) % h);
    size_t n = p / ((size_t)w * h);
    float s = __bfloat162float(gskip.p[p * gskip.stride + gskip.off + c]) +
              0.25f * __bfloat162float(gpool.p[(((n * hc) + y / 2) * wc + x / 2) * gpool.stride + gpool.off + c]);
    float a = __bfloat162float(act.p[p * act.stride + act.off + c]);
    gskip.p[p * gskip.stride + gskip.off + c] = __float2bfloat16(a > 0.f ? s : 0.f);
  }
}

// 1 x 1 head: pred[p] = b + sum_c W[c] act[p][c] (FP32)
__global__ void k_head_fwd(size_t npix, Tensor4 act, const float* __restrict__ Wh, const float* __restrict__ bh,
                           float* __restrict__ pred) {
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < npix; p += (size_t)gridDim.x * blockDim.x) {
    float s = bh[0];
    const bf16* a = act.p + p * act.stride + act.off;
    for (int c = 0; c < act.c; c += 8) {
      float f[8];
      bf8_to_f(*reinterpret_cast<const uint4*>(a + c), f);
#pragma unroll
      for (int e = 0; e < 8; ++e) s += Wh[c + e] * f[e];
    }
    pred[p] = s;
  }
}

// MSE loss against the target and its gradient dpred = 2 (pred - t) / npix; partial losses per
// block (summed on the host in block order)
__global__ void k_mse(size_t npix, const float* __restrict__ pred, const float* __restrict__ t, float* __restrict__ dpred,
                      double* __restrict__ partial) {
  __shared__ double scratch[32];
  double s = 0.0;
  float inv = 2.0f / (float)npix;
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < npix; p += (size_t)gridDim.x * blockDim.x) {
    float d = pred[p] - t[p];
    dpred[p] = d * inv;
    s += (double)d * (double)d;
  }
  double r = block_sum(s, scratch);
  if (threadIdx.x == 0) partial[blockIdx.x] = r;
}

// head backward: g[p][c] = dpred[p] W[c] where act > 0 (the last conv's ReLU); partial weight
// and bias gradients per block: part[block][0..C-1] = sum dpred * act, part[block][C] = sum dpred
__global__ void k_head_bwd(size_t npix, Tensor4 act, const float* __restrict__ Wh, const float* __restrict__ dpred, Tensor4 g,
                           float* __restrict__ part) {
  __shared__ float red[64][33];
  const int C = act.c;  // 32
  float accw[32];
  float accb = 0.f;
  for (int c = 0; c < 32; ++c) accw[c] = 0.f;
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < npix; p += (size_t)gridDim.x * blockDim.x) {
    float dp = dpred[p];
    const bf16* a = act.p + p * act.stride + act.off;
    bf16* gg = g.p + p * g.stride + g.off;
    for (int c = 0; c < C; ++c) {
      float av = __bfloat162float(a[c]);
      gg[c] = __float2bfloat16(av > 0.f ? dp * Wh[c] : 0.f);
      accw[c] += dp * av;
    }
    accb += dp;
  }
  // reduce over the block in a fixed order: warp shuffles then the warps in order
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int c = 0; c <= C; ++c) {
    float v = c < C ? accw[c] : accb;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) red[warp][c] = v;
  }
  __syncthreads();
  if (threadIdx.x <= C) {
    float s = 0.f;
    for (int wi = 0; wi < (int)(blockDim.x >> 5); ++wi) s += red[wi][threadIdx.x];
    part[(size_t)blockIdx.x * (C + 1) + threadIdx.x] = s;
  }
}

// bias gradient partials: part[block][c] = sum over the block's pixels of g[p][c]
__global__ void k_bias_grad(size_t npix, Tensor4 g, float* __restrict__ part) {
  // blockDim = C (<= 256 channels, one thread a channel), pixels strided over blocks
  int c = threadIdx.x;
  float s = 0.f;
  for (size_t p = blockIdx.x; p < npix; p += gridDim.x) s += __bfloat162float(g.p[p * g.stride + g.off + c]);
  part[(size_t)blockIdx.x * g.c + c] = s;
}

// sum of `parts` partial arrays of length n (in order) into out
__global__ void k_sum_parts(size_t n, int parts, const float* __restrict__ part, float* __restrict__ out) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int q = 0; q < parts; ++q) s += part[(size_t)q * n + k];
    out[k] = s;
  }
}

// Adam (Kingma & Ba 2015) on the FP32 master parameters
__global__ void k_adam(size_t n, float* __restrict__ prm, const float* __restrict__ grad, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float eps, float bc1, float bc2) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    float g = grad[k];
    float mk = b1 * m[k] + (1.f - b1) * g;
    float vk = b2 * v[k] + (1.f - b2) * g * g;
    m[k] = mk;
    v[k] = vk;
    prm[k] -= lr * (mk / bc1) / (sqrtf(vk / bc2) + eps);
  }
}

// BF16 weights of a layer: W[t][ci][co] and WT[8 - t][co][ci]
__global__ void k_pack_weights(int cin, int cout, const float* __restrict__ w32, bf16* __restrict__ W, bf16* __restrict__ WT) {
  size_t n = (size_t)9 * cin * cout;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    int co = (int)(k % cout);
    int ci = (int)((k / cout) % cin);
    int t = (int)(k / ((size_t)cout * cin));
    bf16 v = __float2bfloat16(w32[k]);
    W[k] = v;
    WT[((size_t)(8 - t) * cout + co) * cin + ci] = v;
  }
}

}  // namespace dt

struct dt_unet {
  int base = 32;
  std::vector<dt::ConvLayer> conv;  // encoder A0,B0,...,A3,B3 then decoder A2,B2,A1,B1,A0,B0
  size_t n_params = 0, head_w = 0, head_b = 0;
  float *prm = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr;
  long long step = 0;
  // batch buffers (re-made when the shape grows)
  int B = 0, H = 0, W = 0;
  dt::bf16* X0 = nullptr;
  dt::LevelBufs lv[dt::UNET_LEVELS];
  float *pred = nullptr, *dpred = nullptr, *target = nullptr;
  float* part = nullptr;
  size_t part_cap = 0;
  double* loss_part = nullptr;
  std::vector<void*> batch_allocs, allocs;
  cudaStream_t stream = nullptr;
  bool own_stream = true;  // false once bound to a caller's stream (dt_unet_set_stream)
  int sms = 148;
  // forward and input-gradient convolutions on tcgen05 when DT_UNET_TC=1 (default: the mma.sync
  // kernels, faster at this network's channel counts); a device flag the tcgen05 kernels' bounded
  // waits set when one runs out
  bool tc = false;
  int* tc_fault = nullptr;
};

namespace dt {

static dt_status ualloc(std::vector<void*>& list, void** p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, std::max<size_t>(bytes, 16));
  if (e != cudaSuccess) {
    set_error("cudaMalloc of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? DT_OOM : DT_DEVICE_ERROR;
  }
  list.push_back(*p);
  return DT_OK;
}
template <class T>
static dt_status ualloc_t(std::vector<void*>& list, T** p, size_t count) {
  return ualloc(list, reinterpret_cast<void**>(p), count * sizeof(T));
}

static int lvl_ch(const dt_unet* u, int l) { return u->base << l; }

static unsigned int ugrid(const dt_unet* u, size_t n) {
  return std::max(1u, std::min<unsigned int>(ceil_div(n, 256), (unsigned)u->sms * 16));
}

// Batch buffers for B images of H x W (H divisible by 8, W by 512 at the finest level's 64-pixel
// tiles after three halvings).
static dt_status unet_batch(dt_unet* u, int B, int H, int W) {
  if (u->B == B && u->H == H && u->W == W) return DT_OK;
  for (void* p : u->batch_allocs) cudaFree(p);
  u->batch_allocs.clear();
  auto& L = u->batch_allocs;
  size_t npix = (size_t)B * H * W;
  DT_TRY(ualloc_t(L, &u->X0, npix * UNET_IN_PAD));
  for (int l = 0; l < UNET_LEVELS; ++l) {
    LevelBufs& b = u->lv[l];
    b.h = H >> l;
    b.w = W >> l;
    size_t np = (size_t)B * b.h * b.w;
    int c = lvl_ch(u, l);
    b.cu = l + 1 < UNET_LEVELS ? lvl_ch(u, l + 1) + c : c;
    DT_TRY(ualloc_t(L, &b.A, np * c));
    DT_TRY(ualloc_t(L, &b.gA, np * c));
    DT_TRY(ualloc_t(L, &b.U, np * b.cu));
    DT_TRY(ualloc_t(L, &b.gU, np * b.cu));
    if (l + 1 < UNET_LEVELS) {
      size_t npc = np / 4;
      DT_TRY(ualloc_t(L, &b.P, npc * c));
      DT_TRY(ualloc_t(L, &b.gP, npc * c));
      DT_TRY(ualloc_t(L, &b.DA, np * c));
      DT_TRY(ualloc_t(L, &b.gDA, np * c));
      DT_TRY(ualloc_t(L, &b.DB, np * c));
      DT_TRY(ualloc_t(L, &b.gDB, np * c));
    }
  }
  DT_TRY(ualloc_t(L, &u->pred, npix));
  DT_TRY(ualloc_t(L, &u->dpred, npix));
  DT_TRY(ualloc_t(L, &u->target, npix));
  DT_TRY(ualloc_t(L, &u->loss_part, (size_t)u->sms * 16));
  u->B = B;
  u->H = H;
  u->W = W;
  return DT_OK;
}

static Tensor4 T4(bf16* p, int stride, int off, int c) { return Tensor4{p, stride, off, c}; }

// Dynamic shared memory of every tcgen05 convolution instantiation (more than the default 48 KB).
template <int EPI>
static dt_status conv_tc_attributes_epi() {
  DT_CUDA(cudaFuncSetAttribute(k_conv3x3_tc<32, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc_smem_bytes<32>()));
  DT_CUDA(cudaFuncSetAttribute(k_conv3x3_tc<64, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc_smem_bytes<64>()));
  DT_CUDA(cudaFuncSetAttribute(k_conv3x3_tc<128, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc_smem_bytes<128>()));
  DT_CUDA(cudaFuncSetAttribute(k_conv3x3_tc<256, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc_smem_bytes<256>()));
  return DT_OK;
}
static dt_status conv_tc_attributes() {
  DT_TRY(conv_tc_attributes_epi<EPI_BIAS_RELU>());
  DT_TRY(conv_tc_attributes_epi<EPI_BIAS>());
  DT_TRY(conv_tc_attributes_epi<EPI_MASK>());
  DT_TRY(conv_tc_attributes_epi<EPI_STORE>());
  return DT_OK;
}

// The tcgen05 convolution for a problem of `n` output channels over B h w pixels, with B source
// `Bk` (K-major after mirroring the taps); false when the shape does not suit it.
template <int EPI>
static bool conv_tc(dt_unet* u, int B, int h, int w, Tensor4 in, const bf16* Bk, int n, const float* bias, Tensor4 out,
                    Tensor4 mask, cudaStream_t st) {
  size_t pixels = (size_t)B * h * w;
  if (!u->tc || pixels % 128 != 0 || in.c % 32 != 0 || n % 32 != 0 || pixels / 128 > 0x7fffffff) return false;
#ifndef DT_TC_MAX_N
#define DT_TC_MAX_N 128
#endif
  int bn = (n % 256 == 0 && DT_TC_MAX_N >= 256) ? 256 : (n % 128 == 0 && DT_TC_MAX_N >= 128) ? 128 : n % 64 == 0 ? 64 : 32;
  dim3 grid((unsigned)(pixels / 128), n / bn);
  auto go = [&](auto kernel, int smem) {
    kernel<<<grid, 128, smem, st>>>(B, h, w, in, Bk, n, bias, out, mask, u->tc_fault);
  };
  if (bn == 256)
    go(k_conv3x3_tc<256, EPI>, tc_smem_bytes<256>());
  else if (bn == 128)
    go(k_conv3x3_tc<128, EPI>, tc_smem_bytes<128>());
  else if (bn == 64)
    go(k_conv3x3_tc<64, EPI>, tc_smem_bytes<64>());
  else
    go(k_conv3x3_tc<32, EPI>, tc_smem_bytes<32>());
  count_launch();
  return true;
}

static void conv_fwd(dt_unet* u, const ConvLayer& L, int B, int h, int w, Tensor4 in, Tensor4 out, bool relu, cudaStream_t st) {
  {
    // B[tap][co][ci] = W[tap][ci][co] = WT[8 - tap][co][ci]
    const float* bias = u->prm + L.b_off;
    Tensor4 none = T4(nullptr, 0, 0, 0);
    bool done = relu ? conv_tc<EPI_BIAS_RELU>(u, B, h, w, in, L.WT, L.cout, bias, out, none, st)
                     : conv_tc<EPI_BIAS>(u, B, h, w, in, L.WT, L.cout, bias, out, none, st);
    if (done) return;
  }
  bool wide = L.cout % 64 == 0;
  dim3 grid((unsigned)((size_t)B * h * (w / 64)), L.cout / (wide ? 64 : 32));
  const float* bias = u->prm + L.b_off;
  Tensor4 none = T4(nullptr, 0, 0, 0);
  if (wide) {
    if (relu)
      k_conv3x3<64, EPI_BIAS_RELU><<<grid, 128, 0, st>>>(B, h, w, in, L.W, bias, out, none);
    else
      k_conv3x3<64, EPI_BIAS><<<grid, 128, 0, st>>>(B, h, w, in, L.W, bias, out, none);
  } else {
    if (relu)
      k_conv3x3<32, EPI_BIAS_RELU><<<grid, 128, 0, st>>>(B, h, w, in, L.W, bias, out, none);
    else
      k_conv3x3<32, EPI_BIAS><<<grid, 128, 0, st>>>(B, h, w, in, L.W, bias, out, none);
  }
  count_launch();
}

// input gradient gin = conv(g, WT) (times the ReLU mask of `mask` when given)
static void conv_dgrad(dt_unet* u, const ConvLayer& L, int B, int h, int w, Tensor4 g, Tensor4 gin, const Tensor4* mask,
                       cudaStream_t st) {
  int cout = L.cin;  // the transposed problem's output channels (96, 192, 384 at the concatenations)
  bool wide = cout % 64 == 0;
  dim3 grid((unsigned)((size_t)B * h * (w / 64)), cout / (wide ? 64 : 32));
  Tensor4 none = T4(nullptr, 0, 0, 0);
  Tensor4 gout = T4(gin.p, gin.stride, gin.off, cout);
  Tensor4 gg = T4(g.p, g.stride, g.off, L.cout);
  {
    // the transposed problem's B[tap][n = ci][k = co] = W[8 - tap][ci][co]
    bool done = mask ? conv_tc<EPI_MASK>(u, B, h, w, gg, L.W, cout, nullptr, gout, *mask, st)
                     : conv_tc<EPI_STORE>(u, B, h, w, gg, L.W, cout, nullptr, gout, none, st);
    if (done) return;
  }
  if (wide) {
    if (mask)
      k_conv3x3<64, EPI_MASK><<<grid, 128, 0, st>>>(B, h, w, gg, L.WT, nullptr, gout, *mask);
    else
      k_conv3x3<64, EPI_STORE><<<grid, 128, 0, st>>>(B, h, w, gg, L.WT, nullptr, gout, none);
  } else {
    if (mask)
      k_conv3x3<32, EPI_MASK><<<grid, 128, 0, st>>>(B, h, w, gg, L.WT, nullptr, gout, *mask);
    else
      k_conv3x3<32, EPI_STORE><<<grid, 128, 0, st>>>(B, h, w, gg, L.WT, nullptr, gout, none);
  }
  count_launch();
}

// weight and bias gradients of a layer into u->grad
static void conv_wgrad(dt_unet* u, const ConvLayer& L, int B, int h, int w, Tensor4 in, Tensor4 g, cudaStream_t st) {
  int tiles = B * h * (w / 32);
  int chunks = std::min(64, tiles);
  int per = (tiles + chunks - 1) / chunks;
  chunks = (tiles + per - 1) / per;
  int ci_tiles = (L.cin + 63) / 64;
  int bn = L.cout % 64 == 0 ? 64 : 32;
  dim3 grid(9 * ci_tiles * (L.cout / bn), chunks);
  Tensor4 gi = T4(in.p, in.stride, in.off, L.cin);
  if (bn == 64)
    k_conv3x3_wgrad<64><<<grid, 128, 0, st>>>(B, h, w, gi, g, per, u->part);
  else
    k_conv3x3_wgrad<32><<<grid, 128, 0, st>>>(B, h, w, gi, g, per, u->part);
  size_t nw = (size_t)9 * L.cin * L.cout;
  k_sum_parts<<<ugrid(u, nw), 256, 0, st>>>(nw, chunks, u->part, u->grad + L.w_off);
  // bias: per-block partials over pixels, then their sum
  size_t npix = (size_t)B * h * w;
  int bparts = 256;
  k_bias_grad<<<bparts, L.cout, 0, st>>>(npix, g, u->part);
  k_sum_parts<<<1, 256, 0, st>>>((size_t)L.cout, bparts, u->part, u->grad + L.b_off);
  count_launch();
  count_launch();
  count_launch();
  count_launch();
}

static void pack_all(dt_unet* u, cudaStream_t st) {
  for (auto& L : u->conv) {
    size_t n = (size_t)9 * L.cin * L.cout;
    k_pack_weights<<<ugrid(u, n), 256, 0, st>>>(L.cin, L.cout, u->prm + L.w_off, L.W, L.WT);
    count_launch();
  }
}

// Forward over the batch in X0; the prediction in u->pred.
static void unet_forward(dt_unet* u, cudaStream_t st) {
  int B = u->B;
  auto& C = u->conv;
  // encoder
  for (int l = 0; l < UNET_LEVELS; ++l) {
    LevelBufs& b = u->lv[l];
    int c = lvl_ch(u, l);
    Tensor4 in = l == 0 ? T4(u->X0, UNET_IN_PAD, 0, UNET_IN_PAD) : T4(u->lv[l - 1].P, lvl_ch(u, l - 1), 0, lvl_ch(u, l - 1));
    conv_fwd(u, C[2 * l], B, b.h, b.w, in, T4(b.A, c, 0, c), true, st);
    Tensor4 out = l + 1 < UNET_LEVELS ? T4(b.U, b.cu, b.cu - c, c) : T4(b.U, c, 0, c);
    conv_fwd(u, C[2 * l + 1], B, b.h, b.w, T4(b.A, c, 0, c), out, true, st);
    if (l + 1 < UNET_LEVELS) {
      size_t n = (size_t)B * (b.h / 2) * (b.w / 2) * c;
      k_pool<<<ugrid(u, n), 256, 0, st>>>(B, b.h, b.w, out, T4(b.P, c, 0, c));
      count_launch();
    }
  }
  // decoder
  for (int l = UNET_LEVELS - 2; l >= 0; --l) {
    LevelBufs& b = u->lv[l];
    LevelBufs& up = u->lv[l + 1];
    int c = lvl_ch(u, l), cu = lvl_ch(u, l + 1);
    Tensor4 src = l + 1 == UNET_LEVELS - 1 ? T4(up.U, cu, 0, cu) : T4(up.DB, cu, 0, cu);
    size_t n = (size_t)B * b.h * b.w * cu;
    k_upsample<<<ugrid(u, n), 256, 0, st>>>(B, b.h, b.w, src, T4(b.U, b.cu, 0, cu));
    count_launch();
    int di = 2 * UNET_LEVELS + 2 * (UNET_LEVELS - 2 - l);
    conv_fwd(u, C[di], B, b.h, b.w, T4(b.U, b.cu, 0, b.cu), T4(b.DA, c, 0, c), true, st);
    conv_fwd(u, C[di + 1], B, b.h, b.w, T4(b.DA, c, 0, c), T4(b.DB, c, 0, c), true, st);
  }
  size_t npix = (size_t)B * u->H * u->W;
  k_head_fwd<<<ugrid(u, npix), 256, 0, st>>>(npix, T4(u->lv[0].DB, u->base, 0, u->base), u->prm + u->head_w, u->prm + u->head_b,
                                             u->pred);
  count_launch();
}

// Backward from u->dpred; gradients of every parameter in u->grad.
static void unet_backward(dt_unet* u, cudaStream_t st) {
  int B = u->B;
  auto& C = u->conv;
  size_t npix = (size_t)B * u->H * u->W;
  LevelBufs& b0 = u->lv[0];
  int c0 = u->base;
  // head
  int hparts = std::min<int>(256, (int)ceil_div(npix, 256));
  k_head_bwd<<<hparts, 256, 0, st>>>(npix, T4(b0.DB, c0, 0, c0), u->prm + u->head_w, u->dpred, T4(b0.gDB, c0, 0, c0), u->part);
  k_sum_parts<<<1, 64, 0, st>>>((size_t)c0 + 1, hparts, u->part, u->grad + u->head_w);  // head_b follows head_w
  count_launch();
  count_launch();
  // decoder, finest to coarsest
  for (int l = 0; l <= UNET_LEVELS - 2; ++l) {
    LevelBufs& b = u->lv[l];
    int c = lvl_ch(u, l), cu = lvl_ch(u, l + 1);
    int di = 2 * UNET_LEVELS + 2 * (UNET_LEVELS - 2 - l);
    // (gDB holds the gradient of DB's pre-activation already: masked by its producer's ReLU)
    conv_wgrad(u, C[di + 1], B, b.h, b.w, T4(b.DA, c, 0, c), T4(b.gDB, c, 0, c), st);
    Tensor4 mDA = T4(b.DA, c, 0, c);
    conv_dgrad(u, C[di + 1], B, b.h, b.w, T4(b.gDB, c, 0, c), T4(b.gDA, c, 0, c), &mDA, st);
    conv_wgrad(u, C[di], B, b.h, b.w, T4(b.U, b.cu, 0, b.cu), T4(b.gDA, c, 0, c), st);
    conv_dgrad(u, C[di], B, b.h, b.w, T4(b.gDA, c, 0, c), T4(b.gU, b.cu, 0, b.cu), nullptr, st);
    // the upsampled slice's gradient to the coarser level's output (through its ReLU)
    LevelBufs& up = u->lv[l + 1];
    bool bottleneck = l + 1 == UNET_LEVELS - 1;
    Tensor4 act = bottleneck ? T4(up.U, cu, 0, cu) : T4(up.DB, cu, 0, cu);
    Tensor4 gdst = bottleneck ? T4(up.gU, cu, 0, cu) : T4(up.gDB, cu, 0, cu);
    size_t n = (size_t)B * up.h * up.w * cu;
    k_upsample_bwd_mask<<<ugrid(u, n), 256, 0, st>>>(B, up.h, up.w, T4(b.gU, b.cu, 0, cu), act, gdst);
    count_launch();
  }
  // encoder, coarsest to finest
  for (int l = UNET_LEVELS - 1; l >= 0; --l) {
    LevelBufs& b = u->lv[l];
    int c = lvl_ch(u, l);
    Tensor4 gout;  // gradient of the encoder's second conv (pre-activation)
    if (l == UNET_LEVELS - 1) {
      gout = T4(b.gU, c, 0, c);
    } else {
      // skip slice gradient + pooling's, through the ReLU, in place over the skip slice of gU
      Tensor4 gskip = T4(b.gU, b.cu, b.cu - c, c);
      size_t n = (size_t)B * b.h * b.w * c;
      k_skip_pool_bwd_mask<<<ugrid(u, n), 256, 0, st>>>(B, b.h, b.w, gskip, T4(b.gP, c, 0, c), T4(b.U, b.cu, b.cu - c, c));
      count_launch();
      gout = gskip;
    }
    conv_wgrad(u, C[2 * l + 1], B, b.h, b.w, T4(b.A, c, 0, c), gout, st);
    Tensor4 mA = T4(b.A, c, 0, c);
    conv_dgrad(u, C[2 * l + 1], B, b.h, b.w, gout, T4(b.gA, c, 0, c), &mA, st);
    Tensor4 in = l == 0 ? T4(u->X0, UNET_IN_PAD, 0, UNET_IN_PAD) : T4(u->lv[l - 1].P, lvl_ch(u, l - 1), 0, lvl_ch(u, l - 1));
    conv_wgrad(u, C[2 * l], B, b.h, b.w, in, T4(b.gA, c, 0, c), st);
    if (l > 0) {
      int cp = lvl_ch(u, l - 1);
      conv_dgrad(u, C[2 * l], B, b.h, b.w, T4(b.gA, c, 0, c), T4(u->lv[l - 1].gP, cp, 0, cp), nullptr, st);
    }
  }
}

static dt_status unet_make(dt_unet* u, unsigned long long seed) {
  auto add = [&](int cin, int cout) {
    ConvLayer L;
    L.cin = cin;
    L.cout = cout;
    L.w_off = u->n_params;
    u->n_params += (size_t)9 * cin * cout;
    L.b_off = u->n_params;
    u->n_params += cout;
    u->conv.push_back(L);
  };
  for (int l = 0; l < UNET_LEVELS; ++l) {
    int c = lvl_ch(u, l);
    add(l == 0 ? UNET_IN_PAD : lvl_ch(u, l - 1), c);
    add(c, c);
  }
  for (int l = UNET_LEVELS - 2; l >= 0; --l) {
    int c = lvl_ch(u, l);
    add(lvl_ch(u, l + 1) + c, c);
    add(c, c);
  }
  u->head_w = u->n_params;
  u->n_params += u->base;
  u->head_b = u->n_params;
  u->n_params += 1;
  auto& A = u->allocs;
  DT_TRY(ualloc_t(A, &u->prm, u->n_params));
  DT_TRY(ualloc_t(A, &u->grad, u->n_params));
  DT_TRY(ualloc_t(A, &u->m, u->n_params));
  DT_TRY(ualloc_t(A, &u->v, u->n_params));
  for (auto& L : u->conv) {
    DT_TRY(ualloc_t(A, &L.W, (size_t)9 * L.cin * L.cout));
    DT_TRY(ualloc_t(A, &L.WT, (size_t)9 * L.cin * L.cout));
  }
  // He-uniform weights from SplitMix64 (zero for the input's padding channels), zero biases
  std::vector<float> h(u->n_params, 0.f);
  unsigned long long st = seed;
  auto next = [&]() {
    st += 0x9E3779B97F4A7C15ull;
    unsigned long long z = st;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
  };
  for (size_t li = 0; li < u->conv.size(); ++li) {
    auto& L = u->conv[li];
    int fan_cin = li == 0 ? 2 : L.cin;
    float bound = std::sqrt(6.0f / (9.0f * fan_cin));
    for (int t = 0; t < 9; ++t)
      for (int ci = 0; ci < L.cin; ++ci)
        for (int co = 0; co < L.cout; ++co) {
          float v = (float)((2.0 * next() - 1.0) * bound);
          if (li == 0 && ci >= 2) v = 0.f;
          h[L.w_off + ((size_t)t * L.cin + ci) * L.cout + co] = v;
        }
  }
  float hb = std::sqrt(6.0f / u->base) * 0.1f;
  for (int c = 0; c < u->base; ++c) h[u->head_w + c] = (float)((2.0 * next() - 1.0) * hb);
  DT_CUDA(cudaMemcpy(u->prm, h.data(), u->n_params * sizeof(float), cudaMemcpyHostToDevice));
  DT_CUDA(cudaMemset(u->m, 0, u->n_params * sizeof(float)));
  DT_CUDA(cudaMemset(u->v, 0, u->n_params * sizeof(float)));
  // wgrad partials: 64 chunks x the largest layer, or the head/bias partials
  size_t mx = 0;
  for (auto& L : u->conv) mx = std::max(mx, (size_t)9 * L.cin * L.cout);
  u->part_cap = std::max(mx * 64, (size_t)256 * 512);
  DT_TRY(ualloc_t(A, &u->part, u->part_cap));
  pack_all(u, u->stream);
  DT_CUDA(cudaStreamSynchronize(u->stream));
  return DT_OK;
}

static dt_status unet_check_shape(int B, int H, int W) {
  if (B < 1 || H < 8 || W < 512 || H % 8 || W % 512) {
    set_error("unet: batch %d of %d x %d: H must be a multiple of 8 and W of 512 (64-pixel tiles after three halvings)", B, H, W);
    return DT_BAD_ARG;
  }
  return DT_OK;
}

// The forward pass on stream `st`, in stream order (no synchronisation): for callers that run the
// model between kernels of their own (the flexure solve's first guess).
dt_status unet_predict_on(dt_unet* u, cudaStream_t st, const float* x, float* y, int B, int H, int W) {
  if (!u || !x || !y) return DT_BAD_ARG;
  DT_TRY(unet_check_shape(B, H, W));
  DT_TRY(unet_batch(u, B, H, W));
  size_t npix = (size_t)B * H * W;
  k_pack_input<<<ugrid(u, npix * (UNET_IN_PAD / 8)), 256, 0, st>>>(npix, x, u->X0);
  count_launch();
  unet_forward(u, st);
  DT_CUDA(cudaMemcpyAsync(y, u->pred, npix * sizeof(float), cudaMemcpyDeviceToDevice, st));
  return DT_OK;
}

}  // namespace dt

using namespace dt;

extern "C" {

dt_status dt_unet_create(int base_channels, unsigned long long seed, dt_unet** out) {
  if (!out || base_channels != 32) {
    set_error("dt_unet_create: the model has 32 base channels");
    return DT_BAD_ARG;
  }
  auto* u = new dt_unet();
  u->base = base_channels;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, 0) == cudaSuccess) u->sms = prop.multiProcessorCount;
  if (cudaStreamCreateWithFlags(&u->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete u;
    set_error("dt_unet_create: no CUDA device");
    return DT_DEVICE_ERROR;
  }
  dt_status st = unet_make(u, seed);
  if (st != DT_OK) {
    dt_unet_destroy(u);
    return st;
  }
  {
    const char* env = getenv("DT_UNET_TC");
    u->tc = prop.major >= 10 && env && env[0] == '1';
    if (u->tc && (st = dt::conv_tc_attributes()) != DT_OK) {
      dt_unet_destroy(u);
      return st;
    }
    st = dt::ualloc(u->allocs, reinterpret_cast<void**>(&u->tc_fault), sizeof(int));
    if (st == DT_OK && cudaMemset(u->tc_fault, 0, sizeof(int)) != cudaSuccess) st = DT_DEVICE_ERROR;
    if (st != DT_OK) {
      dt_unet_destroy(u);
      return st;
    }
  }
  *out = u;
  return DT_OK;
}

dt_status dt_unet_destroy(dt_unet* u) {
  if (!u) return DT_OK;
  if (u->stream) cudaStreamSynchronize(u->stream);
  for (void* p : u->batch_allocs) cudaFree(p);
  for (void* p : u->allocs) cudaFree(p);
  if (u->stream && u->own_stream) cudaStreamDestroy(u->stream);
  delete u;
  return DT_OK;
}

size_t dt_unet_num_params(const dt_unet* u) { return u ? u->n_params : 0; }

dt_status dt_unet_set_stream(dt_unet* u, void* stream) {
  if (!u) return DT_BAD_ARG;
  if (stream && (cudaStream_t)stream == u->stream) return DT_OK;
  cudaStreamSynchronize(u->stream);
  if (u->own_stream) cudaStreamDestroy(u->stream);
  if (stream) {
    u->stream = (cudaStream_t)stream;
    u->own_stream = false;
  } else {
    if (cudaStreamCreateWithFlags(&u->stream, cudaStreamNonBlocking) != cudaSuccess) return DT_DEVICE_ERROR;
    u->own_stream = true;
  }
  return DT_OK;
}

// x: [B][H][W][2] FP32 (device), y: [B][H][W] FP32 (device)
dt_status dt_unet_predict_dev(dt_unet* u, const float* x, float* y, int B, int H, int W) {
  DT_TRY(dt::unet_predict_on(u, u ? u->stream : nullptr, x, y, B, H, W));
  DT_CUDA(cudaGetLastError());
  DT_CUDA(cudaStreamSynchronize(u->stream));
  int fault = 0;
  DT_CUDA(cudaMemcpy(&fault, u->tc_fault, sizeof(int), cudaMemcpyDeviceToHost));
  if (fault) {
    set_error("dt_unet_predict_dev: a tensor-core convolution's wait ran out");
    return DT_DEVICE_ERROR;
  }
  return DT_OK;
}

// One Adam step on a batch: inputs x [B][H][W][2], targets t [B][H][W] (device, FP32).
dt_status dt_unet_train_step_dev(dt_unet* u, const float* x, const float* t, int B, int H, int W, float lr, double* loss) {
  if (!u || !x || !t) return DT_BAD_ARG;
  DT_TRY(unet_check_shape(B, H, W));
  DT_TRY(unet_batch(u, B, H, W));
  cudaStream_t st = u->stream;
  size_t npix = (size_t)B * H * W;
  k_pack_input<<<ugrid(u, npix * (UNET_IN_PAD / 8)), 256, 0, st>>>(npix, x, u->X0);
  count_launch();
  unet_forward(u, st);
  unsigned int lg = std::min<unsigned int>(ceil_div(npix, 256), (unsigned)u->sms * 16);
  k_mse<<<lg, 256, 0, st>>>(npix, u->pred, t, u->dpred, u->loss_part);
  count_launch();
  unet_backward(u, st);
  u->step += 1;
  const float b1 = 0.9f, b2 = 0.999f;
  float bc1 = 1.f - std::pow(b1, (float)u->step), bc2 = 1.f - std::pow(b2, (float)u->step);
  k_adam<<<ugrid(u, u->n_params), 256, 0, st>>>(u->n_params, u->prm, u->grad, u->m, u->v, lr, b1, b2, 1e-8f, bc1, bc2);
  count_launch();
  pack_all(u, st);
  if (loss) {
    std::vector<double> parts(lg);
    DT_CUDA(cudaMemcpyAsync(parts.data(), u->loss_part, lg * sizeof(double), cudaMemcpyDeviceToHost, st));
    DT_CUDA(cudaStreamSynchronize(st));
    double s = 0.0;
    for (double p : parts) s += p;
    *loss = s / (double)npix;
  }
  DT_CUDA(cudaGetLastError());
  return DT_OK;
}

// The gradient of the last step's loss for every parameter (FP32, host), for tests.
dt_status dt_unet_gradients(dt_unet* u, float* out, size_t n) {
  if (!u || !out || n != u->n_params) return DT_BAD_ARG;
  DT_CUDA(cudaMemcpy(out, u->grad, n * sizeof(float), cudaMemcpyDeviceToHost));
  return DT_OK;
}
// Parameters as FP32 (host) and their replacement (then re-packed to BF16).
dt_status dt_unet_get_params(dt_unet* u, float* out, size_t n) {
  if (!u || !out || n != u->n_params) return DT_BAD_ARG;
  DT_CUDA(cudaMemcpy(out, u->prm, n * sizeof(float), cudaMemcpyDeviceToHost));
  return DT_OK;
}
dt_status dt_unet_set_params(dt_unet* u, const float* in, size_t n) {
  if (!u || !in || n != u->n_params) return DT_BAD_ARG;
  DT_CUDA(cudaMemcpy(u->prm, in, n * sizeof(float), cudaMemcpyHostToDevice));
  pack_all(u, u->stream);
  DT_CUDA(cudaStreamSynchronize(u->stream));
  return DT_OK;
}
// The gradient computation alone (no optimiser step), for tests: loss and gradients of a batch.
dt_status dt_unet_loss_and_grad_dev(dt_unet* u, const float* x, const float* t, int B, int H, int W, double* loss) {
  if (!u || !x || !t) return DT_BAD_ARG;
  DT_TRY(unet_check_shape(B, H, W));
  DT_TRY(unet_batch(u, B, H, W));
  cudaStream_t st = u->stream;
  size_t npix = (size_t)B * H * W;
  k_pack_input<<<ugrid(u, npix * (UNET_IN_PAD / 8)), 256, 0, st>>>(npix, x, u->X0);
  unet_forward(u, st);
  unsigned int lg = std::min<unsigned int>(ceil_div(npix, 256), (unsigned)u->sms * 16);
  k_mse<<<lg, 256, 0, st>>>(npix, u->pred, t, u->dpred, u->loss_part);
  unet_backward(u, st);
  std::vector<double> parts(lg);
  DT_CUDA(cudaMemcpyAsync(parts.data(), u->loss_part, lg * sizeof(double), cudaMemcpyDeviceToHost, st));
  DT_CUDA(cudaStreamSynchronize(st));
  double s = 0.0;
  for (double p : parts) s += p;
  if (loss) *loss = s / (double)npix;
  DT_CUDA(cudaGetLastError());
  return DT_OK;
}

dt_status dt_unet_save(dt_unet* u, const char* path) {
  if (!u || !path) return DT_BAD_ARG;
  std::vector<float> h(u->n_params);
  DT_CUDA(cudaMemcpy(h.data(), u->prm, h.size() * sizeof(float), cudaMemcpyDeviceToHost));
  FILE* f = fopen(path, "wb");
  if (!f) {
    set_error("dt_unet_save: cannot open %s", path);
    return DT_BAD_ARG;
  }
  const char magic[8] = {'D', 'T', 'U', 'N', 'E', 'T', '0', '1'};
  unsigned long long n = u->n_params, steps = (unsigned long long)u->step;
  int base = u->base;
  fwrite(magic, 1, 8, f);
  fwrite(&base, sizeof base, 1, f);
  fwrite(&n, sizeof n, 1, f);
  fwrite(&steps, sizeof steps, 1, f);
  fwrite(h.data(), sizeof(float), h.size(), f);
  fclose(f);
  return DT_OK;
}

dt_status dt_unet_load(dt_unet* u, const char* path) {
  if (!u || !path) return DT_BAD_ARG;
  FILE* f = fopen(path, "rb");
  if (!f) {
    set_error("dt_unet_load: cannot open %s", path);
    return DT_BAD_ARG;
  }
  char magic[8];
  int base = 0;
  unsigned long long n = 0, steps = 0;
  bool ok = fread(magic, 1, 8, f) == 8 && memcmp(magic, "DTUNET01", 8) == 0 && fread(&base, sizeof base, 1, f) == 1 &&
            fread(&n, sizeof n, 1, f) == 1 && fread(&steps, sizeof steps, 1, f) == 1 && base == u->base && n == u->n_params;
  std::vector<float> h(u->n_params);
  ok = ok && fread(h.data(), sizeof(float), h.size(), f) == h.size();
  fclose(f);
  if (!ok) {
    set_error("dt_unet_load: %s is not a weight file of this model", path);
    return DT_BAD_ARG;
  }
  u->step = (long long)steps;
  return dt_unet_set_params(u, h.data(), h.size());
}

}  // extern "C"

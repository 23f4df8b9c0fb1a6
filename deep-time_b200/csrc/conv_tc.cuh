// The 3 x 3 convolution (and its input gradient) on the fifth-generation tensor cores: tcgen05.mma
// with BF16 operands from shared memory and the FP32 accumulator in tensor memory (TMEM).
//
// GEMM: M = 128 consecutive pixels (one image row of >= 128 pixels, or two rows of 64), N = BN
// output channels (32, 64 or 128), K = 9 taps x input channels, 32 channels a step. Operands are
// staged by 16-byte cp.async into the canonical K-major layout without swizzling: 8-row x
// 16-byte core matrices, the four 16-byte chunks of a row's 32 channels 128 bytes apart (leading
// byte offset) and successive 8-row groups 512 bytes apart (stride byte offset). The weights are
// read K-major from the existing copies: forward from WT ([tap][cout][cin], taps mirrored back),
// input gradient from W ([tap][cin][cout], taps mirrored), so B[tap][n][k] = src[(8 - tap) n k].
//
// One thread issues the MMAs (K = 16 each, two per step) and commits them to the step's mbarrier;
// the stage is restaged only after that barrier completes. The accumulator is read back with
// tcgen05.ld (each warp its 32 TMEM lanes = 32 pixels) for the same epilogues as k_conv3x3.
// Every wait is bounded; TMEM is always released before the block leaves.
#pragma once
#include "conv.cuh"

namespace dt {

__device__ __forceinline__ uint32_t tc_smem(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor: start address, leading and stride byte offsets (16-byte units),
// descriptor version 1 (bits 46-47), base offset 0, no swizzling.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor of kind::f16: D FP32, A and B BF16, both K-major, M x N.
template <int M, int N>
__host__ __device__ constexpr uint32_t umma_idesc_bf16() {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n"
      " .reg .pred p;\n"
      " setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n"
      "}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void umma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tc_mbar_init(uint32_t a) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(a) : "memory");
}
__device__ __forceinline__ bool tc_mbar_test(uint32_t a, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n"
      " .reg .pred p;\n"
      " mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(ok)
      : "r"(a), "r"(parity)
      : "memory");
  return ok != 0;
}
// 2^24 tests with short sleeps between them (well under a second): false when the phase did not
// complete.
__device__ __forceinline__ bool tc_mbar_wait(uint32_t a, uint32_t parity) {
  for (int it = 0; it < (1 << 24); ++it) {
    if (tc_mbar_test(a, parity)) return true;
    if (it > 64) __nanosleep(20);
  }
  return false;
}

// Eight consecutive accumulator columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t* r) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Stages of the operand pipeline and their shared memory.
#ifndef DT_TC_STAGES
#define DT_TC_STAGES 4
#endif
constexpr int TC_STAGES = DT_TC_STAGES;
template <int BN>
__host__ __device__ constexpr int tc_smem_bytes() {
  return TC_STAGES * (128 * 32 * 2 + BN * 32 * 2) + 1024;
}

template <int BN, int EPI>
__global__ void __launch_bounds__(128) k_conv3x3_tc(int nimg, int h, int w, Tensor4 in, const bf16* __restrict__ Bk,
                                                    int n_total, const float* __restrict__ bias, Tensor4 out, Tensor4 mask,
                                                    int* fault) {
  constexpr int BM = 128, BK = 32, S = TC_STAGES;
  constexpr int A_BYTES = BM * BK * 2, B_BYTES = BN * BK * 2;
  constexpr uint32_t IDESC = umma_idesc_bf16<BM, BN>();
  static_assert(BN == 32 || BN == 64 || BN == 128 || BN == 256, "TMEM columns: a power of two from 32");
  extern __shared__ __align__(1024) unsigned char tc_dyn[];
  // 1024-aligned stages: A tiles then B tiles
  unsigned char* base = tc_dyn + ((1024 - (tc_smem(tc_dyn) & 1023)) & 1023);
  auto sA = [&](int st) { return base + st * A_BYTES; };
  auto sB = [&](int st) { return base + S * A_BYTES + st * B_BYTES; };
  __shared__ __align__(8) uint64_t mbar[S];
  __shared__ uint32_t s_tmem;
  __shared__ int s_fail;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int k_total = in.c, kpt = k_total / BK, kchunks = 9 * kpt;
  const int p0 = blockIdx.x * BM;
  const int co0 = blockIdx.y * BN;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem(&s_tmem)), "r"(BN)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
#pragma unroll
    for (int q = 0; q < S; ++q) tc_mbar_init(tc_smem(&mbar[q]));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_fail = 0;
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;

  // the four A rows (pixels) this thread stages: their image, row and column
  int pn[4], py[4], px[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    int p = p0 + ((tid + q * 128) >> 2);
    px[q] = p % w;
    int r = p / w;
    py[q] = r % h;
    pn[q] = r / h;
  }
  // stage K step kc into slot st (one cp.async group; an empty group past the last step)
  auto stage = [&](int kc, int st) {
    if (kc < kchunks) {
      const int tap = kc / kpt, ci0 = (kc - tap * kpt) * BK;
      const int ky = tap / 3, kx = tap % 3;
      unsigned char* a = sA(st);
      unsigned char* b = sB(st);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int idx = tid + q * 128, row = idx >> 2, ch = idx & 3;
        const int yy = py[q] + ky - 1;
        const bool ok = yy >= 0 && yy < h;
        int xx = px[q] + kx - 1;
        xx = xx < 0 ? xx + w : (xx >= w ? xx - w : xx);
        const bf16* src = in.p + ((size_t)((size_t)pn[q] * h + (ok ? yy : 0)) * w + xx) * in.stride + in.off + ci0 + ch * 8;
        cp_async16(a + (row >> 3) * 512 + ch * 128 + (row & 7) * 16, src, ok);
      }
#pragma unroll
      for (int q = 0; q < BN * 4 / 128; ++q) {
        const int idx = tid + q * 128, row = idx >> 2, ch = idx & 3;
        const bf16* src = Bk + ((size_t)(8 - tap) * n_total + co0 + row) * k_total + ci0 + ch * 8;
        cp_async16(b + (row >> 3) * 512 + ch * 128 + (row & 7) * 16, src, true);
      }
    }
    cp_async_commit();
  };

  uint32_t phase[S];
#pragma unroll
  for (int q = 0; q < S; ++q) phase[q] = 0u;
#pragma unroll
  for (int q = 0; q < S; ++q) stage(q, q);
  for (int kc = 0; kc < kchunks; ++kc) {
    const int st = kc % S;
    // step kc's group: the prologue committed steps 0 .. S - 1 and every iteration from 1 on
    // commits one more (step kc + S - 1, or an empty group), so at most S - 2 newer groups may
    // still be pending
    cp_async_wait<S - 2>();
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // the staged tiles -> the tensor cores
    __syncthreads();
    if (s_fail) break;  // a wait ran out: every thread leaves here together
    if (tid == 0) {
      tc_fence_after();
      const uint32_t a = tc_smem(sA(st)), b = tc_smem(sB(st));
#pragma unroll
      for (int q = 0; q < BK / 16; ++q)
        umma_bf16(tmem, umma_desc(a + q * 256, 128, 512), umma_desc(b + q * 256, 128, 512), IDESC, (kc | q) != 0);
      umma_commit(tc_smem(&mbar[st]));
    }
    // refill the slot of step kc - 1 (its MMAs were issued an iteration ago) with step kc - 1 + S
    if (kc >= 1) {
      const int sp = (kc - 1) % S;
      if (tc_mbar_wait(tc_smem(&mbar[sp]), phase[sp])) {
        phase[sp] ^= 1u;
        stage(kc - 1 + S, sp);
      } else {
        s_fail = 1;
        cp_async_commit();
      }
    }
  }
  cp_async_wait<0>();
  __syncthreads();
  // all MMAs done: the last step's commit completes after every earlier MMA of the thread
  if (!s_fail) {
    const int st = (kchunks - 1) % S;
    if (!tc_mbar_wait(tc_smem(&mbar[st]), phase[st])) s_fail = 1;
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (!s_fail) {
    const int row = warp * 32 + lane;
    const size_t pix = (size_t)p0 + row;
    bf16* dst = out.p + pix * out.stride + out.off + co0;
#pragma unroll 1
    for (int c0 = 0; c0 < BN; c0 += 8) {
      uint32_t r[8];
      tmem_ld8(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, r);
      tmem_wait_ld();
      float v[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) v[e] = __uint_as_float(r[e]);
      if (EPI == EPI_BIAS_RELU || EPI == EPI_BIAS) {
#pragma unroll
        for (int e = 0; e < 8; ++e) v[e] += bias[co0 + c0 + e];
      }
      if (EPI == EPI_BIAS_RELU) {
#pragma unroll
        for (int e = 0; e < 8; ++e) v[e] = fmaxf(v[e], 0.f);
      }
      if (EPI == EPI_MASK) {
        const __nv_bfloat162* m2 = reinterpret_cast<const __nv_bfloat162*>(mask.p + pix * mask.stride + mask.off + co0 + c0);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          __nv_bfloat162 m = m2[e];
          if (!(__bfloat162float(m.x) > 0.f)) v[2 * e] = 0.f;
          if (!(__bfloat162float(m.y) > 0.f)) v[2 * e + 1] = 0.f;
        }
      }
      __nv_bfloat162* d2 = reinterpret_cast<__nv_bfloat162*>(dst + c0);
      if (EPI == EPI_ACCUM) {
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          __nv_bfloat162 prev = d2[e];
          v[2 * e] += __bfloat162float(prev.x);
          v[2 * e + 1] += __bfloat162float(prev.y);
        }
      }
      uint4 pk;
      __nv_bfloat162 b0 = __floats2bfloat162_rn(v[0], v[1]), b1 = __floats2bfloat162_rn(v[2], v[3]);
      __nv_bfloat162 b2 = __floats2bfloat162_rn(v[4], v[5]), b3 = __floats2bfloat162_rn(v[6], v[7]);
      pk.x = *reinterpret_cast<uint32_t*>(&b0);
      pk.y = *reinterpret_cast<uint32_t*>(&b1);
      pk.z = *reinterpret_cast<uint32_t*>(&b2);
      pk.w = *reinterpret_cast<uint32_t*>(&b3);
      *reinterpret_cast<uint4*>(dst + c0) = pk;
    }
  } else if (tid == 0) {
    atomicExch(fault, 1);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN) : "memory");
  }
}

}  // namespace dt

// The 13-point operator as a persistent kernel fed by the Tensor Memory Accelerator.
//
// Each block loops over tiles (tile t, t + gridDim.x, ...). Two shared-memory stages alternate:
// while a tile is computed, the bulk tensor copies of the block's next tile land in the other
// stage, signalled by that stage's mbarrier (complete_tx). One thread issues the copies. The
// boxes are those of k_apply's tiles: the vector (and J, part) with two halo rows and columns,
// d with one, c and b without; each box starts on the tile's 16-byte-aligned column i0 - OFF.
// The copies zero-fill outside the raster. After they land, the block writes the wrapped halo
// columns of the first and last tile columns from global memory, and repeats the raster's edge
// rows over the rows above and below it (rows clamp). The arithmetic is k_apply's, value for
// value.
//
// Every wait on an mbarrier is bounded. A wait that runs out sets S->fault and S->stop, ends the
// loop's graph condition, waits (bounded again) for the copies still in flight, and returns.
// Included by flexure.cu after k_apply.
#pragma once
#include <cuda.h>

namespace dt {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t a, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint32_t a, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes) : "memory");
}
// Non-blocking test of the phase with parity `parity`.
__device__ __forceinline__ bool mbar_test_wait(uint32_t a, uint32_t parity) {
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
// Bounded wait for the phase with parity `parity` to complete: `polls` tests (2^24 by default)
// with a short sleep between them (well under a second in all), false when it did not complete.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t a, uint32_t parity, int polls = 1 << 24) {
  for (int it = 0; it < polls; ++it) {
    if (mbar_test_wait(a, parity)) return true;
    if (it > 64) __nanosleep(20);
  }
  return false;
}
// A 2-D tile copy from global memory into this CTA's shared memory, completing on the mbarrier.
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(mbar)
      : "memory");
}
// A contiguous copy of `bytes` (a multiple of 16; both addresses 16-byte aligned) from global
// memory into this CTA's shared memory, completing on the mbarrier.
__device__ __forceinline__ void bulk_load_1d(uint32_t dst, const void* src, uint32_t bytes, uint32_t mbar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(reinterpret_cast<unsigned long long>(src)), "r"(bytes), "r"(mbar)
               : "memory");
}
// Orders this thread's generic-proxy shared-memory accesses before later async-proxy (TMA) ones.
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Shared-memory stage of k_apply_tma: the boxes' offsets (bytes, 128-aligned) and the bytes the
// copies of one tile write.
template <class T, int MODE>
struct TmaStage {
  static constexpr bool JAC = MODE == JAC_LEFT || MODE == JAC_FINAL;
  static constexpr bool HAS_C = MODE != BEND;
  static constexpr bool HAS_B = MODE == RESID || MODE == RESID_GATED;
  static constexpr int TBY = tile_rows<T>(), P = Tile<T>::PITCH;
  static constexpr int UR = TBY + 4, MR = TBY + 2;
  static constexpr int BV = UR * P * (int)sizeof(T), BD = MR * P * (int)sizeof(T), BI = TBY * TBX * (int)sizeof(T);
  static constexpr int r128(int b) { return (b + 127) / 128 * 128; }
  static constexpr int OV = 0;
  static constexpr int OJ = OV + r128(BV);
  static constexpr int OP = OJ + (JAC ? r128(BV) : 0);
  static constexpr int OD = OP + (JAC ? r128(BV) : 0);
  static constexpr int OC = OD + r128(BD);
  static constexpr int OB = OC + (HAS_C ? r128(BI) : 0);
  static constexpr int BYTES = OB + (HAS_B ? r128(BI) : 0);
  // part is copied only for JAC_FINAL (JAC_LEFT uses its slot as scratch for u)
  static constexpr int TX = BV + (JAC ? BV : 0) + (MODE == JAC_FINAL ? BV : 0) + BD + (HAS_C ? BI : 0) + (HAS_B ? BI : 0);
  static constexpr int SMEM = 2 * BYTES + 16;  // two stages and their mbarriers
};

template <class T, int MODE>
__global__ void __launch_bounds__(TBX* TTY) k_apply_tma(const __grid_constant__ CUtensorMap mv, const __grid_constant__ CUtensorMap mJ,
                                                        const __grid_constant__ CUtensorMap mpart,
                                                        const __grid_constant__ CUtensorMap md, const __grid_constant__ CUtensorMap mc,
                                                        const __grid_constant__ CUtensorMap mb, int w, int h, T inv_dx2,
                                                        const T* __restrict__ vsrc, const T* __restrict__ J,
                                                        const T* __restrict__ part, const T* __restrict__ d,
                                                        T* __restrict__ y, double* partials, Scalars* S, int tiles_x,
                                                        int ntiles) {
  using ST = TmaStage<T, MODE>;
  constexpr bool JAC = ST::JAC, HAS_B = ST::HAS_B;
  constexpr int TBY = ST::TBY, SEG = TBY / TTY, P = ST::P, OFF = Tile<T>::OFF, UR = ST::UR, MR = ST::MR;
  constexpr int NTH = TBX * TTY;
  if (MODE != PLAIN && MODE != BEND && MODE != RESID) {
    if (S->stop) {
      if (blockIdx.x == 0 && threadIdx.x == 0 && threadIdx.y == 0) set_cond(S, 0);
      return;
    }
  }
  if (MODE == RESID_GATED && S->gate_it != S->it) return;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + 2 * ST::BYTES);
  __shared__ int s_fail;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + ty * TBX;
  if (tid == 0) {
    mbar_init(smem_u32(&mbar[0]), 1);
    mbar_init(smem_u32(&mbar[1]), 1);
    mbar_fence_init();
    s_fail = 0;
  }
  __syncthreads();
  const int G = gridDim.x;
  auto issue = [&](int t, int b) {
    const int i0 = (t % tiles_x) * TBX, j0 = (t / tiles_x) * TBY;
    unsigned char* base = smem + b * ST::BYTES;
    const uint32_t bar = smem_u32(&mbar[b]);
    mbar_expect_tx(bar, ST::TX);
    tma_load_2d(smem_u32(base + ST::OV), &mv, i0 - OFF, j0 - 2, bar);
    if (JAC) tma_load_2d(smem_u32(base + ST::OJ), &mJ, i0 - OFF, j0 - 2, bar);
    if (MODE == JAC_FINAL) tma_load_2d(smem_u32(base + ST::OP), &mpart, i0 - OFF, j0 - 2, bar);
    tma_load_2d(smem_u32(base + ST::OD), &md, i0 - OFF, j0 - 1, bar);
    if (ST::HAS_C) tma_load_2d(smem_u32(base + ST::OC), &mc, i0, j0, bar);
    if (HAS_B) tma_load_2d(smem_u32(base + ST::OB), &mb, i0, j0, bar);
  };
  bool pending[2] = {false, false};
  if (tid == 0) {
    if ((int)blockIdx.x < ntiles) {
      issue(blockIdx.x, 0);
      pending[0] = true;
    }
    if ((int)blockIdx.x + G < ntiles) {
      issue(blockIdx.x + G, 1);
      pending[1] = true;
    }
  }
  uint32_t phase[2] = {0u, 0u};
  Acc<2> acc;
  acc.v[0] = 0.0;
  acc.v[1] = 0.0;
  const int r0 = ty * SEG;
  auto wrapc = [&](int g) { return g < 0 ? g + w : (g >= w ? g - w : g); };
  auto clampr = [&](int g) { return min(max(g, 0), h - 1); };
  int k = 0;
  for (int t = blockIdx.x; t < ntiles; t += G, ++k) {
    const int b = k & 1;
    if (tid == 0) {
      // S->wait_give_up (a test of this path): no test at all, as if the wait had run out
      if (!mbar_wait_bounded(smem_u32(&mbar[b]), phase[b], S->wait_give_up ? 0 : 1 << 24)) s_fail = 1;
      pending[b] = false;
    }
    phase[b] ^= 1u;
    __syncthreads();
    if (s_fail) {
      if (tid == 0) {
        S->fault = 1;
        S->stop = STOP_NONFINITE;
        set_cond(S, 0);
        // the copies still in flight land before the block leaves (bounded again)
        mbar_wait_bounded(smem_u32(&mbar[b]), phase[b] ^ 1u);
        if (pending[b ^ 1]) mbar_wait_bounded(smem_u32(&mbar[b ^ 1]), phase[b ^ 1]);
      }
      return;
    }
    unsigned char* base = smem + b * ST::BYTES;
    T* sv = reinterpret_cast<T*>(base + ST::OV);
    T* sJ = reinterpret_cast<T*>(base + ST::OJ);
    T* sP = reinterpret_cast<T*>(base + ST::OP);
    T* sd = reinterpret_cast<T*>(base + ST::OD);
    const T* sc = reinterpret_cast<const T*>(base + ST::OC);
    const T* sB = reinterpret_cast<const T*>(base + ST::OB);
    const int i0 = (t % tiles_x) * TBX, j0 = (t / tiles_x) * TBY;
    // the first and last tile columns: halo columns from across the seam (x wraps)
    const bool left = i0 == 0, right = i0 + TBX == w;
    if (left || right) {
      for (int e = tid; e < UR * 4; e += NTH) {
        int rr = e >> 2, q = e & 3;
        if ((q < 2 && !left) || (q >= 2 && !right)) continue;
        int lc = q < 2 ? q - 2 : TBX + q - 2;
        size_t gi = (size_t)clampr(j0 - 2 + rr) * w + wrapc(i0 + lc);
        int si = rr * P + OFF + lc;
        sv[si] = vsrc[gi];
        if (JAC) sJ[si] = J[gi];
        if (MODE == JAC_FINAL) sP[si] = part[gi];
      }
      for (int e = tid; e < MR * 2; e += NTH) {
        int rr = e >> 1, q = e & 1;
        if ((q == 0 && !left) || (q == 1 && !right)) continue;
        int lc = q == 0 ? -1 : TBX;
        sd[rr * P + OFF + lc] = d[(size_t)clampr(j0 - 1 + rr) * w + wrapc(i0 + lc)];
      }
      __syncthreads();
    }
    // rows outside the raster repeat its edge rows (the copies zero-filled them)
    const bool top = j0 == 0, bottom = j0 + TBY + 1 >= h;
    if (top || bottom) {
      for (int e = tid; e < UR * P; e += NTH) {
        int rr = e / P, col = e - rr * P;
        int g = j0 - 2 + rr;
        if (g >= 0 && g < h) continue;
        int si = rr * P + col, so = (clampr(g) - j0 + 2) * P + col;
        sv[si] = sv[so];
        if (JAC) sJ[si] = sJ[so];
        if (MODE == JAC_FINAL) sP[si] = sP[so];
      }
      for (int e = tid; e < MR * P; e += NTH) {
        int rr = e / P, col = e - rr * P;
        int g = j0 - 1 + rr;
        if (g >= 0 && g < h) continue;
        sd[rr * P + col] = sd[(clampr(g) - j0 + 1) * P + col];
      }
      __syncthreads();
    }
    if (JAC) {
      // u = J r (+ part); r and J stay readable for the outputs
      for (int e = tid; e < UR * P; e += NTH) {
        T u = sJ[e] * sv[e];
        if (MODE == JAC_FINAL) u += sP[e];
        sP[e] = u;
      }
      __syncthreads();
    }
    const T* su = JAC ? sP : sv;
    // m = d . L u at local rows -1 .. TBY, columns -1 .. TBX (as k_apply)
    {
      const T* ucol = su + OFF + tx;
      T* mcol = sd + OFF + tx;
      T un = ucol[(r0 + 1) * P], uc = ucol[(r0 + 2) * P];
#pragma unroll
      for (int q = 0; q < SEG; ++q) {
        const int lr = r0 + q;
        T us = ucol[(lr + 3) * P];
        T lap = (ucol[(lr + 2) * P - 1] + ucol[(lr + 2) * P + 1] + un + us - (T)4 * uc) * inv_dx2;
        mcol[(lr + 1) * P] = lap * mcol[(lr + 1) * P];
        un = uc;
        uc = us;
      }
    }
    for (int e = tid; e < 2 * (TBX + 2) + 2 * TBY; e += NTH) {
      int lr, lc;
      if (e < 2 * (TBX + 2)) {
        lr = e < TBX + 2 ? -1 : TBY;
        lc = (e < TBX + 2 ? e : e - (TBX + 2)) - 1;
      } else {
        lr = (e - 2 * (TBX + 2)) >> 1;
        lc = (e & 1) ? TBX : -1;
      }
      const T* uc = su + (lr + 2) * P + OFF + lc;
      T lap = (uc[-1] + uc[1] + uc[-P] + uc[P] - (T)4 * uc[0]) * inv_dx2;
      T* m = sd + (lr + 1) * P + OFF + lc;
      *m = lap * *m;
    }
    __syncthreads();
    {
      const int hb = h - 1 - j0;
      const bool mt = j0 == 0, mbt = hb + 1 <= TBY;
      if (mt || mbt) {
        for (int e = tid; e < TBX + 2; e += NTH) {
          if (mt) sd[0 * P + OFF - 1 + e] = sd[1 * P + OFF - 1 + e];
          if (mbt) sd[(hb + 2) * P + OFF - 1 + e] = sd[(hb + 1) * P + OFF - 1 + e];
        }
        __syncthreads();
      }
    }
    {
      const int i = i0 + tx;
      const T* mcol = sd + OFF + tx;
      T mn = mcol[r0 * P], mc = mcol[(r0 + 1) * P];
#pragma unroll
      for (int q = 0; q < SEG; ++q) {
        const int lr = r0 + q;
        T ms = mcol[(lr + 2) * P];
        T lm = (mcol[(lr + 1) * P - 1] + mcol[(lr + 1) * P + 1] + mn + ms - (T)4 * mc) * inv_dx2;
        mn = mc;
        mc = ms;
        const int j = j0 + lr;
        if (j < h) {
          size_t kk = (size_t)j * w + i;
          T u = su[(lr + 2) * P + OFF + tx];
          if (MODE == BEND) {
            y[kk] = lm;
          } else {
            T au = lm + sc[lr * TBX + tx] * u;
            if (MODE == AP_DOT) {
              y[kk] = au;
              acc.v[0] += (double)u * (double)au;
            } else if (MODE == PLAIN) {
              y[kk] = au;
            } else if (HAS_B) {
              T rr = sB[lr * TBX + tx] - au;
              y[kk] = rr;
              acc.v[0] += (double)rr * (double)rr;
            } else if (MODE == JAC_LEFT) {
              y[kk] = sv[(lr + 2) * P + OFF + tx] - au;
            } else {  // JAC_FINAL
              T r = sv[(lr + 2) * P + OFF + tx];
              T z = u + sJ[(lr + 2) * P + OFF + tx] * (r - au);
              y[kk] = z;
              acc.v[0] += (double)r * (double)z;
              acc.v[1] = fmax(acc.v[1], fabs((double)z));
            }
          }
        }
      }
    }
    // every thread is done with this stage: it takes the block's tile after next
    fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0 && t + 2 * G < ntiles) {
      issue(t + 2 * G, b);
      pending[b] = true;
    }
  }
  if (MODE == AP_DOT || MODE == RESID || MODE == RESID_GATED || MODE == JAC_FINAL) {
    const int kind[2] = {0, 1};
    unsigned int nb = gridDim.x;
    int site = MODE == AP_DOT ? SITE_PAP : (MODE == RESID || MODE == RESID_GATED) ? SITE_RESID : SITE_PRECOND;
    bool last = MODE == JAC_FINAL ? reduce_partials<2>(acc, kind, partials, &S->ticket[site], nb)
                                  : reduce_partials<1>(*reinterpret_cast<Acc<1>*>(&acc), kind, partials, &S->ticket[site], nb);
    if (last && tid == 0) {
      if (MODE == AP_DOT) finish_pap(S, acc.v[0]);
      if (MODE == RESID) S->rr = acc.v[0];
      if (MODE == RESID_GATED) S->rr_true = acc.v[0];
      if (MODE == JAC_FINAL) finish_precond(S, acc.v[0], acc.v[1]);
    }
  }
}

}  // namespace dt

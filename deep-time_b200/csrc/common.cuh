// Shared helpers of the deep-time B200 backend: status handling, complex arithmetic on CUDA's
// vector types, and the deterministic block reductions every CG kernel uses.
#pragma once
#include <cuda_runtime.h>

#include <cstdlib>

#include <cstdint>
#include <cstdio>
#include <string>
#include <type_traits>

#include "deeptime_gpu.h"

namespace dt {

// The message behind the last non-OK status of this thread (dt_last_error).
void set_error(const char* fmt, ...);
const char* last_error();

#define DT_CUDA(call)                                                                        \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess) {                                                                 \
      ::dt::set_error("%s:%d: %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_));   \
      return e_ == cudaErrorMemoryAllocation ? DT_OOM : DT_DEVICE_ERROR;                     \
    }                                                                                        \
  } while (0)

// DT_CUDA for functions without a status: records the error, which a later DT_CUDA reports.
#define DT_CUDA_VOID(call)                                                                   \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      ::dt::set_error("%s:%d: %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_));   \
  } while (0)

#define DT_TRY(...)               \
  do {                            \
    dt_status s_ = (__VA_ARGS__); \
    if (s_ != DT_OK) return s_;   \
  } while (0)

template <class T>
struct cx;
template <>
struct cx<double> {
  using type = double2;
};
template <>
struct cx<float> {
  using type = float2;
};
template <class T>
using cplx = typename cx<T>::type;

template <class C>
__host__ __device__ __forceinline__ C mk(decltype(C::x) a, decltype(C::x) b) {
  C r;
  r.x = a;
  r.y = b;
  return r;
}
template <class C>
__device__ __forceinline__ C cadd(C a, C b) { return mk<C>(a.x + b.x, a.y + b.y); }
template <class C>
__device__ __forceinline__ C csub(C a, C b) { return mk<C>(a.x - b.x, a.y - b.y); }
template <class C>
__device__ __forceinline__ C cmul(C a, C b) { return mk<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
template <class C>
__device__ __forceinline__ C cconj(C a) { return mk<C>(a.x, -a.y); }
template <class C>
__device__ __forceinline__ C cscale(C a, decltype(C::x) s) { return mk<C>(a.x * s, a.y * s); }
// i * a
template <class C>
__device__ __forceinline__ C cmuli(C a) { return mk<C>(-a.y, a.x); }

// Single precision: both parts in one paired FP32 instruction (sm_100's add / mul / fma on
// float2), each part rounded as the scalar forms above round it (a - b as fma(b, -1, a), exact
// but for the one rounding of the sum; products contracted into one fma, as the compiler
// contracts the scalar forms).
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return __fmul2_rn(a, make_float2(s, s)); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return __ffma2_rn(make_float2(-a.y, a.y), make_float2(b.y, b.x), __fmul2_rn(make_float2(a.x, a.x), b));
}

// ---- deterministic reductions -------------------------------------------------------------
// A reducing kernel writes one partial per block (fixed grid, fixed in-block order); the last
// block to finish (an atomic ticket) sums the partials in index order. The result therefore does
// not depend on the order blocks ran in.

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}

// Sum over the block (any multiple of 32 threads up to 1024); the result is valid in thread 0.
__device__ __forceinline__ double block_sum(double v, double* scratch32) {
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int nwarps = (blockDim.x * blockDim.y + 31) >> 5;
  int tid = threadIdx.x + threadIdx.y * blockDim.x;
  lane = tid & 31;
  warp = tid >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) scratch32[warp] = v;
  __syncthreads();
  double r = 0.0;
  if (warp == 0) {
    r = lane < nwarps ? scratch32[lane] : 0.0;
    r = warp_sum(r);
  }
  return r;
}
__device__ __forceinline__ double block_max(double v, double* scratch32) {
  int tid = threadIdx.x + threadIdx.y * blockDim.x;
  int lane = tid & 31, warp = tid >> 5;
  int nwarps = (blockDim.x * blockDim.y + 31) >> 5;
  v = warp_max(v);
  __syncthreads();
  if (lane == 0) scratch32[warp] = v;
  __syncthreads();
  double r = -INFINITY;
  if (warp == 0) {
    r = lane < nwarps ? scratch32[lane] : -INFINITY;
    r = warp_max(r);
  }
  return r;
}

// After thread 0 of each block stored its partial(s), returns true in thread 0 of exactly one
// block: the last to arrive, which then sees every partial. `ticket` is reset for reuse.
__device__ __forceinline__ bool last_block(unsigned int* ticket, unsigned int nblocks) {
  __shared__ bool is_last;
  int tid = threadIdx.x + threadIdx.y * blockDim.x;
  if (tid == 0) {
    __threadfence();
    unsigned int t = atomicAdd(ticket, 1u);
    is_last = (t == nblocks - 1);
    if (is_last) *ticket = 0u;
  }
  __syncthreads();
  return is_last;
}

template <int NV>
struct Acc {
  double v[NV];
};

// Writes this block's partial sums (thread 0 holds them) and, in the last block, reduces all of
// them in index order. kind: 0 sum, 1 max (per component).
template <int NV>
__device__ bool reduce_partials(Acc<NV>& a, const int* kind, double* partials, unsigned int* ticket, unsigned int nblocks) {
  __shared__ double scratch[32];
  int tid = threadIdx.x + threadIdx.y * blockDim.x;
  int nthreads = blockDim.x * blockDim.y;
  unsigned int bid = blockIdx.x + blockIdx.y * gridDim.x;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    double r = kind[q] ? block_max(a.v[q], scratch) : block_sum(a.v[q], scratch);
    if (tid == 0) partials[(size_t)q * nblocks + bid] = r;
  }
  if (!last_block(ticket, nblocks)) return false;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    double s = kind[q] ? -INFINITY : 0.0;
    for (unsigned int b = tid; b < nblocks; b += nthreads) {
      double p = __ldcg(partials + (size_t)q * nblocks + b);
      s = kind[q] ? fmax(s, p) : s + p;
    }
    double r = kind[q] ? block_max(s, scratch) : block_sum(s, scratch);
    a.v[q] = r;  // valid in thread 0
  }
  return true;
}

// Kernel launches of the calling thread (eager ones, and those recorded while capturing a graph
// body); defined in flexure.cu.
// The U-Net's forward pass on a given stream, without synchronising (defined in unet.cu).
dt_status unet_predict_on(dt_unet* u, cudaStream_t st, const float* x, float* y, int B, int H, int W);

void count_launch();
long long launches_now();
void add_launches(long long k);
void begin_capture_count();
long long end_capture_count();

inline unsigned int ceil_div(size_t a, size_t b) { return (unsigned int)((a + b - 1) / b); }

// Test support for the allocation failure path: with DT_FAIL_ALLOC_AT=n in the environment, the
// n-th device allocation of a handle (its counter `made`, from 1) fails as if the device were out
// of memory. Without the variable every allocation goes to cudaMalloc.
inline bool alloc_fault(size_t& made) {
  ++made;
  const char* e = getenv("DT_FAIL_ALLOC_AT");
  return e && e[0] && (size_t)strtoull(e, nullptr, 10) == made;
}
inline bool is_pow2(long v) { return v > 0 && (v & (v - 1)) == 0; }
inline int ilog2(long v) {
  int r = 0;
  while ((1L << r) < v) ++r;
  return r;
}

}  // namespace dt

// Shared-memory Stockham FFT (radix 8, 4, 2) for power-of-two lengths, written from the
// Stockham autosort formulation as given by Govindaraju et al., "High performance discrete
// Fourier transforms on graphics processors", SC'08 (their FftIteration): a stage of radix R over
// sub-transforms of span Ns reads x[j + r N/R], twiddles by e^(-+2 pi i r (j mod Ns)/(Ns R)), takes
// a length-R DFT and writes y[(j/Ns) Ns R + (j mod Ns) + r Ns]; the result is in natural order.
//
// Stages run in place through registers: every thread loads its butterflies' inputs, the block
// synchronises, every thread writes its outputs. A block transforms `batch` sequences of length N
// stored back to back in shared memory; each thread holds 8 complex values per stage, so the
// block has batch * N / 8 threads. Twiddles come from a table tw[t] = e^(-2 pi i t / N) built on
// the host (long double angles); the inverse transform (unnormalised) conjugates them.
#pragma once
#include "common.cuh"

namespace dt {

template <class C, bool INV>
__device__ __forceinline__ void dft2(C& a, C& b) {
  C t = a;
  a = cadd(t, b);
  b = csub(t, b);
}

// Multiply by -i (forward) or +i (inverse).
template <class C, bool INV>
__device__ __forceinline__ C rot90(C a) {
  return INV ? mk<C>(-a.y, a.x) : mk<C>(a.y, -a.x);
}

template <class C, bool INV>
__device__ __forceinline__ void dft4(C& a0, C& a1, C& a2, C& a3) {
  C s02 = cadd(a0, a2), d02 = csub(a0, a2);
  C s13 = cadd(a1, a3), d13 = rot90<C, INV>(csub(a1, a3));
  a0 = cadd(s02, s13);
  a2 = csub(s02, s13);
  a1 = cadd(d02, d13);
  a3 = csub(d02, d13);
}

template <class C, bool INV>
__device__ __forceinline__ void dft8(C* v) {
  using T = decltype(C::x);
  const T h = (T)0.70710678118654752440084436210485;
  // even and odd halves
  C e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
  C o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
  dft4<C, INV>(e0, e1, e2, e3);
  dft4<C, INV>(o0, o1, o2, o3);
  // twiddles W8^k, k = 1, 2, 3: forward (1 - i)/sqrt2, -i, (-1 - i)/sqrt2
  C t1 = INV ? mk<C>((o1.x - o1.y) * h, (o1.x + o1.y) * h) : mk<C>((o1.x + o1.y) * h, (o1.y - o1.x) * h);
  C t2 = rot90<C, INV>(o2);
  C t3 = INV ? mk<C>(-(o3.x + o3.y) * h, (o3.x - o3.y) * h) : mk<C>((o3.y - o3.x) * h, -(o3.x + o3.y) * h);
  v[0] = cadd(e0, o0);
  v[4] = csub(e0, o0);
  v[1] = cadd(e1, t1);
  v[5] = csub(e1, t1);
  v[2] = cadd(e2, t2);
  v[6] = csub(e2, t2);
  v[3] = cadd(e3, t3);
  v[7] = csub(e3, t3);
}

// One stage of radix R over `batch` sequences of length N in s; span Ns (product of the earlier
// radices). `tw` has N entries e^(-2 pi i t/N). Threads: batch * N / 8, each owns 8 / R butterflies.
template <class C, int R, bool INV>
__device__ __forceinline__ void stockham_stage(C* s, int N, int logN, int Ns, const C* __restrict__ tw) {
  constexpr int B = 8 / R;  // butterflies per thread
  const int tid = threadIdx.x;
  const int nbf = N / R;    // butterflies per sequence
  C v[B][R];
  int outbase[B];
#pragma unroll
  for (int q = 0; q < B; ++q) {
    int t = tid * B + q;
    int b = t / nbf;          // sequence
    int j = t - b * nbf;      // butterfly within the sequence
    C* base = s + (size_t)b * N;
    int k = j & (Ns - 1);
#pragma unroll
    for (int r = 0; r < R; ++r) v[q][r] = base[j + r * nbf];
    if (Ns > 1) {
      int step = (N / (Ns * R)) * k;
#pragma unroll
      for (int r = 1; r < R; ++r) {
        C w = tw[r * step];
        if (INV) w.y = -w.y;
        v[q][r] = cmul(v[q][r], w);
      }
    }
    outbase[q] = b * N + (j - k) * R + k;
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < B; ++q) {
    if (R == 8) {
      dft8<C, INV>(v[q]);
    } else if (R == 4) {
      dft4<C, INV>(v[q][0], v[q][1], v[q][2], v[q][3]);
    } else {
      dft2<C, INV>(v[q][0], v[q][1]);
    }
#pragma unroll
    for (int r = 0; r < R; ++r) s[outbase[q] + r * Ns] = v[q][r];
  }
  __syncthreads();
}

// Full transform: radix-8 stages, then one radix-4 or radix-2 stage for the remainder.
// The caller synchronises before (data in s) and may read s after it returns.
template <class C, bool INV>
__device__ void smem_fft(C* s, int N, int logN, const C* __restrict__ tw) {
  int Ns = 1;
  int rem = logN;
  while (rem >= 3) {
    stockham_stage<C, 8, INV>(s, N, logN, Ns, tw);
    Ns <<= 3;
    rem -= 3;
  }
  if (rem == 2) {
    stockham_stage<C, 4, INV>(s, N, logN, Ns, tw);
  } else if (rem == 1) {
    stockham_stage<C, 2, INV>(s, N, logN, Ns, tw);
  }
}

}  // namespace dt

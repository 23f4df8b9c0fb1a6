// Shared-memory Stockham FFT (radix 8, 4, 2) for power-of-two lengths, written from the
// Stockham autosort formulation as given by Govindaraju et al., "High performance discrete
// Fourier transforms on graphics processors", SC'08 (their FftIteration): a stage of radix R over
// sub-transforms of span Ns reads x[j + r N/R], twiddles by e^(-+2 pi i r (j mod Ns)/(Ns R)), takes
// a length-R DFT and writes y[(j/Ns) Ns R + (j mod Ns) + r Ns]; the result is in natural order.
//
// Stages run in place through registers: every thread loads its butterflies' inputs, the block
// synchronises, every thread writes its outputs. A block transforms `batch` sequences of length N;
// each thread holds EPT (8 or 16) complex values per stage, so the block has batch * N / EPT
// threads. Twiddles come from a table tw[t] = e^(-2 pi i t / N) built on the host (long double
// angles); the inverse transform (unnormalised) conjugates them.
//
// Shared-memory layout: element i of a sequence lives at pad(i) = i + (i >> PADSHIFT), one spare
// slot after every 16 (8-byte complex) or 8 (16-byte complex) values, i.e. every 128 bytes. The
// stage's strided writes (stride 8 in the first stage) then fall in distinct banks; a sequence
// occupies padded_len(N) slots.
#pragma once
#include "common.cuh"

namespace dt {

template <class C>
struct Pad {
  static constexpr int SHIFT = sizeof(C) == 16 ? 3 : 4;
  static __host__ __device__ __forceinline__ constexpr int at(int i) { return i + (i >> SHIFT); }
  static __host__ __device__ __forceinline__ constexpr int len(int n) { return n + (n >> SHIFT) + 1; }
};

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

// One stage of radix R over the block's sequences of length N = 2^LOGN, each stored at
// s + b * NP (padded); span NS. Everything but the data is known at compile time, so the index
// arithmetic is shifts and masks. Threads: batch * N / EPT, each owns EPT / R butterflies.
template <class C, int R, int EPT, bool INV, int LOGN, int NS>
__device__ __forceinline__ void stockham_stage(C* s, const C* __restrict__ tw) {
  constexpr int N = 1 << LOGN;
  constexpr int NP = Pad<C>::len(N);
  constexpr int B = EPT / R;
  constexpr int NBF = N / R;
  constexpr int LOGNBF = LOGN - (R == 8 ? 3 : R == 4 ? 2 : 1);
  constexpr int STEP = N / (NS * R);
  const int tid = threadIdx.x;
  C v[B][R];
  int obase[B], oidx[B];
#pragma unroll
  for (int q = 0; q < B; ++q) {
    int t = tid + q * blockDim.x;
    int b = t >> LOGNBF;
    int j = t & (NBF - 1);
    C* base = s + b * NP;
    int k = j & (NS - 1);
#pragma unroll
    for (int r = 0; r < R; ++r) v[q][r] = base[Pad<C>::at(j + r * NBF)];
    if (NS > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        C w = tw[r * STEP * k];
        if (INV) w.y = -w.y;
        v[q][r] = cmul(v[q][r], w);
      }
    }
    obase[q] = b * NP;
    oidx[q] = (j - k) * R + k;
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
    for (int r = 0; r < R; ++r) s[obase[q] + Pad<C>::at(oidx[q] + r * NS)] = v[q][r];
  }
  __syncthreads();
}

// Stages from span NS on: radix 8 while three or more factors of two remain, then 4 or 2.
template <class C, int EPT, bool INV, int LOGN, int NS, int REM>
struct Stages {
  static __device__ __forceinline__ void run(C* s, const C* __restrict__ tw) {
    if constexpr (REM >= 3) {
      stockham_stage<C, 8, EPT, INV, LOGN, NS>(s, tw);
      Stages<C, EPT, INV, LOGN, NS * 8, REM - 3>::run(s, tw);
    } else if constexpr (REM == 2) {
      stockham_stage<C, 4, EPT, INV, LOGN, NS>(s, tw);
    } else if constexpr (REM == 1) {
      stockham_stage<C, 2, EPT, INV, LOGN, NS>(s, tw);
    }
  }
};

// Full transform of length 2^LOGN. The caller synchronises before (data in s) and may read s
// after it returns.
template <class C, int EPT, bool INV, int LOGN>
__device__ __forceinline__ void smem_fft(C* s, const C* __restrict__ tw) {
  Stages<C, EPT, INV, LOGN, 1, LOGN>::run(s, tw);
}

}  // namespace dt

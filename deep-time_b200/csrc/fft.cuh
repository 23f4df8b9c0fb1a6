// Shared-memory Stockham FFT (radix 16, 8, 4, 2) for power-of-two lengths, written from the
// Stockham autosort formulation as given by Govindaraju et al., "High performance discrete
// Fourier transforms on graphics processors", SC'08 (their FftIteration): a stage of radix R over
// sub-transforms of span Ns reads x[j + r N/R], twiddles by e^(-+2 pi i r (j mod Ns)/(Ns R)), takes
// a length-R DFT and writes y[(j/Ns) Ns R + (j mod Ns) + r Ns]; the result is in natural order.
//
// Stages run in place through registers: every thread loads its butterflies' inputs, the block
// synchronises, every thread writes its outputs. A block transforms `batch` sequences of length N;
// each thread holds EPT (8 or 16) complex values per stage, so the block has batch * N / EPT
// threads. Twiddles come from a table tw[t] = e^(-2 pi i t / N) built on the host (long double
// angles); the inverse transform (unnormalised) conjugates them. A stage loads w^1, w^2, w^4, w^8
// and forms the other powers by products.
//
// Shared-memory layout: element i of a sequence lives at pad(i) = i + (i >> 4), one spare slot
// after every 16 values. The first stage's writes (stride 16) then fall in distinct banks for
// both 8-byte and 16-byte complex values (17 j slots: banks 2j per half warp for float2, 4j per
// quarter warp for double2); a sequence occupies padded_len(N) slots.
#pragma once
#include "common.cuh"

namespace dt {

template <class C>
struct Pad {
  static constexpr int SHIFT = 4;
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

// 16-point DFT as 4 x 4: DFTs of length 4 over the residues mod 4, twiddles W16^(n2 k1), DFTs of
// length 4 across; X[k1 + 4 k2] lands in v[k1 + 4 k2].
template <class C, bool INV>
__device__ __forceinline__ void dft16(C* v) {
  using T = decltype(C::x);
  const T c1 = (T)0.92387953251128675613, s1 = (T)0.38268343236508977173;  // cos, sin of pi/8
  const T h = (T)0.70710678118654752440;
  C y[4][4];  // y[n2][k1]
#pragma unroll
  for (int n2 = 0; n2 < 4; ++n2) {
    C a0 = v[n2], a1 = v[4 + n2], a2 = v[8 + n2], a3 = v[12 + n2];
    dft4<C, INV>(a0, a1, a2, a3);
    y[n2][0] = a0;
    y[n2][1] = a1;
    y[n2][2] = a2;
    y[n2][3] = a3;
  }
  // W16^m = e^(-+ i pi m / 8): m = 1, 2, 3 (n2 = 1), 2, 4, 6 (n2 = 2), 3, 6, 9 (n2 = 3)
  const T sg = INV ? (T)1 : (T)-1;  // sign of the imaginary part of W16^1
  const C w1 = mk<C>(c1, sg * s1), w2 = mk<C>(h, sg * h), w3 = mk<C>(s1, sg * c1);
  y[1][1] = cmul(y[1][1], w1);
  y[1][2] = cmul(y[1][2], w2);
  y[1][3] = cmul(y[1][3], w3);
  y[2][1] = cmul(y[2][1], w2);
  y[2][2] = rot90<C, INV>(y[2][2]);
  y[2][3] = cmul(y[2][3], mk<C>(-h, sg * h));
  y[3][1] = cmul(y[3][1], w3);
  y[3][2] = cmul(y[3][2], mk<C>(-h, sg * h));
  y[3][3] = cmul(y[3][3], mk<C>(-c1, -sg * s1));
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1) {
    C a0 = y[0][k1], a1 = y[1][k1], a2 = y[2][k1], a3 = y[3][k1];
    dft4<C, INV>(a0, a1, a2, a3);
    v[k1] = a0;
    v[k1 + 4] = a1;
    v[k1 + 8] = a2;
    v[k1 + 12] = a3;
  }
}

// w^r (r = 1 .. R-1) of w = tw[base] (conjugated for the inverse): the table's w, w^2, w^4, w^8
// and products of those (at most three roundings from exact values), four loads instead of R - 1.
template <class C, int R, bool INV>
__device__ __forceinline__ void stage_twiddles(const C* __restrict__ tw, int base, C* w) {
#pragma unroll
  for (int p2 = 1; p2 < R; p2 *= 2) {
    C t = tw[p2 * base];
    if (INV) t.y = -t.y;
    w[p2] = t;
  }
#pragma unroll
  for (int r = 3; r < R; ++r) {
    if ((r & (r - 1)) == 0) continue;
    int hi = 1;
    while (hi * 2 <= r) hi *= 2;
    w[r] = cmul(w[r - hi], w[hi]);
  }
}

// The length-R DFT of v in place.
template <class C, int R, bool INV>
__device__ __forceinline__ void dft_r(C* v) {
  if constexpr (R == 16) {
    dft16<C, INV>(v);
  } else if constexpr (R == 8) {
    dft8<C, INV>(v);
  } else if constexpr (R == 4) {
    dft4<C, INV>(v[0], v[1], v[2], v[3]);
  } else if constexpr (R == 2) {
    dft2<C, INV>(v[0], v[1]);
  }
}

// One stage of radix R over the block's sequences of length N = 2^LOGN, each stored at
// s + b * NP (padded); span NS. Everything but the data is known at compile time, so the index
// arithmetic is shifts and masks. Threads: batch * N / EPT, each owns EPT / R butterflies.
template <class C, int R, int EPT, bool INV, int LOGN, int NS, int PITCH = 0, int NTH = 0>
__device__ __forceinline__ void stockham_stage(C* s, const C* __restrict__ tw) {
  constexpr int N = 1 << LOGN;
  constexpr int NP = PITCH ? PITCH : Pad<C>::len(N);
  constexpr int B = EPT / R;
  constexpr int NBF = N / R;
  constexpr int LOGNBF = LOGN - (R == 16 ? 4 : R == 8 ? 3 : R == 4 ? 2 : 1);
  constexpr int STEP = N / (NS * R);
  const int tid = threadIdx.x;
  C v[B][R];
  int obase[B], oidx[B];
#pragma unroll
  for (int q = 0; q < B; ++q) {
    // NTH: the block's threads when the caller knows them at compile time (index arithmetic
    // folds), else blockDim.x
    int t = tid + q * (NTH ? NTH : (int)blockDim.x);
    int b = t >> LOGNBF;
    int j = t & (NBF - 1);
    C* base = s + b * NP;
    int k = j & (NS - 1);
    if constexpr (NBF % 16 == 0) {
      // j < NBF: pad(j + r NBF) = pad(j) + r (NBF + NBF / 16), constant offsets from one base
      const C* bj = base + Pad<C>::at(j);
#pragma unroll
      for (int r = 0; r < R; ++r) v[q][r] = bj[r * (NBF + NBF / 16)];
    } else {
#pragma unroll
      for (int r = 0; r < R; ++r) v[q][r] = base[Pad<C>::at(j + r * NBF)];
    }
    if (NS > 1) {
      C w[R];
      stage_twiddles<C, R, INV>(tw, STEP * k, w);
#pragma unroll
      for (int r = 1; r < R; ++r) v[q][r] = cmul(v[q][r], w[r]);
    }
    obase[q] = b * NP;
    oidx[q] = (j - k) * R + k;
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < B; ++q) {
    dft_r<C, R, INV>(v[q]);
    if constexpr (NS % 16 == 0) {
      // oidx + r NS with NS a multiple of 16: pad(oidx) + r (NS + NS / 16)
      C* o = s + obase[q] + Pad<C>::at(oidx[q]);
#pragma unroll
      for (int r = 0; r < R; ++r) o[r * (NS + NS / 16)] = v[q][r];
    } else if constexpr (NS == 1) {
      // oidx = j R with R <= 16 and r < R: the 16-slot group does not change, pad(oidx) + r
      C* o = s + obase[q] + Pad<C>::at(oidx[q]);
#pragma unroll
      for (int r = 0; r < R; ++r) o[r] = v[q][r];
    } else {
#pragma unroll
      for (int r = 0; r < R; ++r) s[obase[q] + Pad<C>::at(oidx[q] + r * NS)] = v[q][r];
    }
  }
  __syncthreads();
}

// Stages from span NS on: radix 16 while four or more factors of two remain (and a thread holds
// 16 values), then 8, 4 or 2.
template <class C, int EPT, bool INV, int LOGN, int NS, int REM, int PITCH = 0, int NTH = 0>
struct Stages {
  static __device__ __forceinline__ void run(C* s, const C* __restrict__ tw) {
    if constexpr (REM >= 4 && EPT % 16 == 0) {
      stockham_stage<C, 16, EPT, INV, LOGN, NS, PITCH, NTH>(s, tw);
      Stages<C, EPT, INV, LOGN, NS * 16, REM - 4, PITCH, NTH>::run(s, tw);
    } else if constexpr (REM >= 3) {
      stockham_stage<C, 8, EPT, INV, LOGN, NS, PITCH, NTH>(s, tw);
      Stages<C, EPT, INV, LOGN, NS * 8, REM - 3, PITCH, NTH>::run(s, tw);
    } else if constexpr (REM == 2) {
      stockham_stage<C, 4, EPT, INV, LOGN, NS, PITCH, NTH>(s, tw);
    } else if constexpr (REM == 1) {
      stockham_stage<C, 2, EPT, INV, LOGN, NS, PITCH, NTH>(s, tw);
    }
  }
};

// The adjoint of stockham_stage<C, R, EPT, false, LOGN, NS> (inverse twiddles and DFT, the read
// and write patterns swapped): reads the positions that stage wrote, (j - k) R + k + r NS, takes
// the inverse DFT, multiplies by the conjugated twiddles and writes the positions that stage read,
// j + r N / R. Running a forward transform's stages' adjoints in reverse order gives N times its
// inverse.
template <class C, int R, int EPT, int LOGN, int NS, int PITCH = 0, int NTH = 0>
__device__ __forceinline__ void stockham_stage_adj(C* s, const C* __restrict__ tw) {
  constexpr int N = 1 << LOGN;
  constexpr int NP = PITCH ? PITCH : Pad<C>::len(N);
  constexpr int B = EPT / R;
  constexpr int NBF = N / R;
  constexpr int LOGNBF = LOGN - (R == 16 ? 4 : R == 8 ? 3 : R == 4 ? 2 : 1);
  constexpr int STEP = N / (NS * R);
  static_assert(NS % 16 == 0 && NBF % 16 == 0, "adjoint stage: spans of whole 16-slot groups");
  const int tid = threadIdx.x;
  C v[B][R];
  int wbase[B], kk[B];
#pragma unroll
  for (int q = 0; q < B; ++q) {
    int t = tid + q * (NTH ? NTH : (int)blockDim.x);
    int b = t >> LOGNBF;
    int j = t & (NBF - 1);
    int k = j & (NS - 1);
    const C* src = s + b * NP + Pad<C>::at((j - k) * R + k);
#pragma unroll
    for (int r = 0; r < R; ++r) v[q][r] = src[r * (NS + NS / 16)];
    wbase[q] = b * NP + Pad<C>::at(j);
    kk[q] = k;
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < B; ++q) {
    dft_r<C, R, true>(v[q]);
    C w[R];
    stage_twiddles<C, R, true>(tw, STEP * kk[q], w);
    C* dst = s + wbase[q];
    dst[0] = v[q][0];
#pragma unroll
    for (int r = 1; r < R; ++r) dst[r * (NBF + NBF / 16)] = cmul(v[q][r], w[r]);
  }
  __syncthreads();
}

// The adjoints of Stages<C, EPT, false, LOGN, NS, REM> in reverse order (the last stage's first).
template <class C, int EPT, int LOGN, int NS, int REM, int PITCH = 0, int NTH = 0>
struct StagesAdj {
  static __device__ __forceinline__ void run(C* s, const C* __restrict__ tw) {
    if constexpr (REM >= 4 && EPT % 16 == 0) {
      StagesAdj<C, EPT, LOGN, NS * 16, REM - 4, PITCH, NTH>::run(s, tw);
      stockham_stage_adj<C, 16, EPT, LOGN, NS, PITCH, NTH>(s, tw);
    }
  }
};

// The radix the stages above give a length-2^LOGN transform's last stage.
__host__ __device__ constexpr int last_radix(int logn) {
  return logn % 4 == 0 ? 16 : (1 << (logn % 4));
}

// Full transform of length 2^LOGN. The caller synchronises before (data in s) and may read s
// after it returns.
template <class C, int EPT, bool INV, int LOGN, int NTH = 0>
__device__ __forceinline__ void smem_fft(C* s, const C* __restrict__ tw) {
  Stages<C, EPT, INV, LOGN, 1, LOGN, 0, NTH>::run(s, tw);
}

}  // namespace dt

// The spectral solve's transform along x for any raster width (the reference plans rustfft at
// any length: Spectral::new, flexure.rs:1139-1170; coarsening, flexure.rs:2110-2121, lets widths
// such as 48, 96, 1536 or 3000 reach the solver). Widths whose half is a power of two take the
// shared-memory kernels k_rows_fwd / k_rows_inv; every other width comes here.
//
// As the reference does (forward_with, flexure.rs:1193-1232; inverse_with, :1287-1345), two rows
// of the raster are transformed at once as the real and imaginary parts of one complex row of
// length w:
//   forward   z = a + i b,  Z = DFT_w(z),  A[k] = (Z[k] + conj Z[w-k]) / 2,
//             B[k] = (Z[k] - conj Z[w-k]) / 2i   for k = 0 .. w/2
//   inverse   Z[k] = A[k] + i B[k],  Z[w-k] = conj A[k] + i conj B[k],  a + i b = IDFT_w(Z) / w
// and the half spectrum keeps the packed layout of the power-of-two path: N = ceil(w/2) complex
// values a row, column 0 holding (A[0], A[w/2]) (both real; the second is 0 for odd w), so the
// column pass and the row solve are the same for every width.
//
// DFT_w runs as a sequence of global-memory passes over all row pairs at once:
//   - mixed radix when every prime factor of w is at most ANY_MAX_PRIME: Stockham autosort
//     stages of radix 16, 8, 4, 2, 3, 5, 7 and any other prime, each pass reading one buffer and
//     writing the other (Govindaraju et al., "High performance discrete Fourier transforms on
//     graphics processors", SC 2008);
//   - otherwise Bluestein's chirp z-transform: with c_n = e^(i pi n^2 / w),
//     X_k = conj(c_k) sum_j (x_j conj(c_j)) c_(k-j), a cyclic convolution of length M (the
//     power of two >= 2w - 1) done by two FFTs of length M and the table B = FFT_M(c).
// The inverse transform is the forward one between two conjugations. Twiddles, chirps and B come
// from host tables made in long double; the device calls no trigonometric function.

constexpr int ANY_MAX_STAGES = 24;
constexpr int ANY_MAX_PRIME = 64;  // larger prime factors of w go through Bluestein

struct AnyPlan {
  int w = 0;          // the raster's width (the transform's length)
  int L = 0;          // the passes' length: w, or M for Bluestein
  int pairs = 0;      // row pairs, ceil(h / 2)
  int nst = 0;        // stages of one length-L FFT
  int radix[ANY_MAX_STAGES] = {};
  int span[ANY_MAX_STAGES] = {};  // the product of the radices before each stage
  int bluestein = 0;
};

// Twiddle of exponent e (0 <= e < L) from the table of e^(-2 pi i t / L).
template <class C>
__device__ __forceinline__ C any_tw(const C* __restrict__ tw, int e) {
  return tw[e];
}

// One Stockham stage of radix R (R > 0 known at compile time) on row pair `pr`, butterfly j:
// inputs src[j + r L/R] times w_(Ns R)^(r k), k = j mod Ns; a DFT of length R; outputs to
// dst[(j / Ns) Ns R + k + r Ns].
template <class T, int R>
__global__ void __launch_bounds__(256) k_any_stage(AnyPlan p, int stage, const cplx<T>* __restrict__ src,
                                                   cplx<T>* __restrict__ dst, const cplx<T>* __restrict__ tw,
                                                   const Scalars* S) {
  using C = cplx<T>;
  if (S->stop) return;
  const int L = p.L, Ns = p.span[stage], LR = L / R;
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (size_t)p.pairs * LR) return;
  const int pr = (int)(t / LR), j = (int)(t - (size_t)pr * LR);
  const int k = j % Ns;
  const C* in = src + (size_t)pr * L;
  C* out = dst + (size_t)pr * L;
  const int step = L / (Ns * R);  // twiddle w_(Ns R)^(r k) = tw[r k step]
  C v[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    C x = in[j + r * LR];
    v[r] = (r == 0 || k == 0) ? x : cmul(x, any_tw(tw, r * k * step));
  }
  if constexpr (R == 16) {
    dft16<C, false>(v);
  } else if constexpr (R == 2) {
    dft2<C, false>(v[0], v[1]);
  } else if constexpr (R == 4) {
    dft4<C, false>(v[0], v[1], v[2], v[3]);
  } else if constexpr (R == 8) {
    dft8<C, false>(v);
  } else {
    // a small odd radix by its definition: o_m = sum_r v_r w_R^(r m), w_R^q = tw[q L / R]
    C o[R];
#pragma unroll
    for (int m = 0; m < R; ++m) {
      C acc = v[0];
#pragma unroll
      for (int r = 1; r < R; ++r) acc = cadd(acc, cmul(v[r], any_tw(tw, ((r * m) % R) * LR)));
      o[m] = acc;
    }
#pragma unroll
    for (int m = 0; m < R; ++m) v[m] = o[m];
  }
  const int base = (j / Ns) * Ns * R + k;
#pragma unroll
  for (int r = 0; r < R; ++r) out[base + r * Ns] = v[r];
}

// The same stage for any prime radix R (runtime, at most ANY_MAX_PRIME): one output per thread,
// o_m of butterfly j = sum_r (src[j + r L/R] w_(Ns R)^(r k)) w_R^(r m).
template <class T>
__global__ void __launch_bounds__(256) k_any_stage_prime(AnyPlan p, int stage, const cplx<T>* __restrict__ src,
                                                         cplx<T>* __restrict__ dst, const cplx<T>* __restrict__ tw,
                                                         const Scalars* S) {
  using C = cplx<T>;
  if (S->stop) return;
  const int L = p.L, Ns = p.span[stage], R = p.radix[stage], LR = L / R;
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (size_t)p.pairs * L) return;
  const int pr = (int)(t / L), q = (int)(t - (size_t)pr * L);
  const int j = q / R, m = q - j * R;  // butterfly j, output m
  const int k = j % Ns, step = L / (Ns * R);
  const C* in = src + (size_t)pr * L;
  C acc = in[j];
  for (int r = 1; r < R; ++r) {
    C x = in[j + r * LR];
    if (k) x = cmul(x, any_tw(tw, r * k * step));
    acc = cadd(acc, cmul(x, any_tw(tw, ((r * m) % R) * LR)));
  }
  dst[(size_t)pr * L + (j / Ns) * Ns * R + k + m * Ns] = acc;
}

// Bluestein's middle step, in place: x <- conj(x B) (the conjugation makes the next forward FFT
// an inverse one).
template <class T>
__global__ void __launch_bounds__(256) k_any_chirp_mul(AnyPlan p, cplx<T>* __restrict__ buf, const cplx<T>* __restrict__ bhat,
                                                       const Scalars* S) {
  if (S->stop) return;
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (size_t)p.pairs * p.L) return;
  const int q = (int)(t % p.L);
  buf[t] = cconj(cmul(buf[t], bhat[q]));
}

// Forward load: z = a wt + i b wt for the pair's rows 2 pr and 2 pr + 1 (b = 0 past the last
// row), times conj(c_i) and zero-padded to L for Bluestein.
template <class T, bool WEIGHT>
__global__ void __launch_bounds__(256) k_any_load_rows(AnyPlan p, int h, const T* __restrict__ v, const T* __restrict__ wt,
                                                       cplx<T>* __restrict__ buf, const cplx<T>* __restrict__ chirp,
                                                       const Scalars* S) {
  using C = cplx<T>;
  if (S->stop) return;
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (size_t)p.pairs * p.L) return;
  const int pr = (int)(t / p.L), i = (int)(t - (size_t)pr * p.L);
  const int w = p.w;
  C z = mk<C>((T)0, (T)0);
  if (i < w) {
    const size_t ka = (size_t)(2 * pr) * w + i, kb = ka + w;
    T a = v[ka], b = (2 * pr + 1 < h) ? v[kb] : (T)0;
    if (WEIGHT) {
      a *= wt[ka];
      b = (2 * pr + 1 < h) ? b * wt[kb] : (T)0;
    }
    z = mk<C>(a, b);
    if (p.bluestein) z = cmul(z, cconj(chirp[i]));
  }
  buf[t] = z;
}

// Packed half-spectrum entry k of a row as the complex coefficient A[k], k <= w/2.
template <class C>
__device__ __forceinline__ C any_unpack(const C* __restrict__ row, int k, int w) {
  using T = decltype(C::x);
  if (k == 0) return mk<C>(row[0].x, (T)0);
  if (2 * k == w) return mk<C>(row[0].y, (T)0);
  return row[k];
}

// Inverse load: Z[i] from the pair's half-spectrum rows, conjugated (the inverse as a forward
// DFT between conjugations), times conj(c_i) and zero-padded for Bluestein.
template <class T>
__global__ void __launch_bounds__(256) k_any_load_half(AnyPlan p, int h, int N, const cplx<T>* __restrict__ half,
                                                       cplx<T>* __restrict__ buf, const cplx<T>* __restrict__ chirp,
                                                       const Scalars* S) {
  using C = cplx<T>;
  if (S->stop) return;
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (size_t)p.pairs * p.L) return;
  const int pr = (int)(t / p.L), i = (int)(t - (size_t)pr * p.L);
  const int w = p.w;
  C z = mk<C>((T)0, (T)0);
  if (i < w) {
    const C* ra = half + (size_t)(2 * pr) * N;
    const bool hb = 2 * pr + 1 < h;
    const C* rb = ra + N;
    const int nk = w / 2 + 1;
    C A, B;
    if (i < nk) {
      A = any_unpack(ra, i, w);
      B = hb ? any_unpack(rb, i, w) : mk<C>((T)0, (T)0);
    } else {  // i = w - k with 1 <= k < nk: conj A[k] + i conj B[k]
      A = cconj(any_unpack(ra, w - i, w));
      B = hb ? cconj(any_unpack(rb, w - i, w)) : mk<C>((T)0, (T)0);
    }
    z = cconj(cadd(A, cmuli(B)));
    if (p.bluestein) z = cmul(z, cconj(chirp[i]));
  }
  buf[t] = z;
}

// The DFT's value at k < w from the final pass's buffer: the buffer itself (mixed radix), or
// conj(c_k) conj(R_k) / M after Bluestein's second FFT.
template <class C>
__device__ __forceinline__ C any_fetch(const AnyPlan& p, const C* __restrict__ row, int k, const C* __restrict__ chirp) {
  using T = decltype(C::x);
  C z = row[k];
  if (p.bluestein) z = cscale(cmul(cconj(chirp[k]), cconj(z)), (T)1 / (T)p.L);
  return z;
}

// Forward store: A[k], B[k] of the pair's two rows into the half spectrum (h x N, packed column 0).
template <class T>
__global__ void __launch_bounds__(256) k_any_split(AnyPlan p, int h, int N, const cplx<T>* __restrict__ buf,
                                                   cplx<T>* __restrict__ half, const cplx<T>* __restrict__ chirp,
                                                   const Scalars* S) {
  using C = cplx<T>;
  if (S->stop) return;
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (size_t)p.pairs * N) return;
  const int pr = (int)(t / N), k = (int)(t - (size_t)pr * N);
  const int w = p.w;
  const C* row = buf + (size_t)pr * p.L;
  C* ha = half + (size_t)(2 * pr) * N;
  C* hb = ha + N;
  const bool has_b = 2 * pr + 1 < h;
  const T half_ = (T)0.5;
  auto parts = [&](int kk, C& A, C& B) {
    C z = any_fetch(p, row, kk, chirp), zc = cconj(any_fetch(p, row, kk == 0 ? 0 : w - kk, chirp));
    A = cscale(cadd(z, zc), half_);
    C d = csub(z, zc);
    B = mk<C>(d.y * half_, -d.x * half_);  // (z - conj z') / 2i
  };
  C A, B;
  parts(k, A, B);
  if (k == 0) {
    T an = (T)0, bn = (T)0;
    if ((w & 1) == 0) {
      C A2, B2;
      parts(w / 2, A2, B2);
      an = A2.x;
      bn = B2.x;
    }
    A = mk<C>(A.x, an);
    B = mk<C>(B.x, bn);
  }
  ha[k] = A;
  if (has_b) hb[k] = B;
}

// Inverse store of the pair's rows in the modes of k_rows_inv: out = x (STORE), x wt (STORE_W),
// x with r.x and max|x| reduced (STORE_DOT), or sum over the bank's three levels of x_l wt_l
// (BANK; the levels' final buffers `lvl_stride` complex values apart, the weights n apart).
template <class T, int MODE>
__global__ void __launch_bounds__(256) k_any_emit(AnyPlan p, int h, const cplx<T>* __restrict__ buf, size_t lvl_stride,
                                                  T* __restrict__ out, const T* __restrict__ wt, const T* __restrict__ r,
                                                  const cplx<T>* __restrict__ chirp, double* partials, Scalars* S) {
  using C = cplx<T>;
  if (S->stop) {
    if (MODE == INV_STORE_DOT && blockIdx.x == 0 && threadIdx.x == 0) set_cond(S, 0);
    return;
  }
  constexpr int LEVELS = MODE == INV_BANK ? 3 : 1;
  const int w = p.w;
  const size_t n = (size_t)w * h, total = (size_t)p.pairs * w;
  const T inv_w = (T)1 / (T)w;
  Acc<2> acc;
  acc.v[0] = 0.0;
  acc.v[1] = 0.0;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int pr = (int)(t / w), i = (int)(t - (size_t)pr * w);
    const size_t ka = (size_t)(2 * pr) * w + i, kb = ka + w;
    const bool has_b = 2 * pr + 1 < h;
    T xa = (T)0, xb = (T)0;
#pragma unroll
    for (int lv = 0; lv < LEVELS; ++lv) {
      C z = cconj(any_fetch(p, buf + lv * lvl_stride + (size_t)pr * p.L, i, chirp));
      T a = z.x * inv_w, b = z.y * inv_w;
      if (MODE == INV_STORE_W || MODE == INV_BANK) {
        a *= wt[lv * n + ka];
        b = has_b ? b * wt[lv * n + kb] : (T)0;
      }
      xa += a;
      xb += b;
    }
    out[ka] = xa;
    if (has_b) out[kb] = xb;
    if (MODE == INV_STORE_DOT) {
      acc.v[0] += (double)r[ka] * (double)xa;
      acc.v[1] = fmax(acc.v[1], fabs((double)xa));
      if (has_b) {
        acc.v[0] += (double)r[kb] * (double)xb;
        acc.v[1] = fmax(acc.v[1], fabs((double)xb));
      }
    }
  }
  if (MODE == INV_STORE_DOT) {
    const int kind[2] = {0, 1};
    if (reduce_partials<2>(acc, kind, partials, &S->ticket[SITE_PRECOND], gridDim.x) && threadIdx.x == 0)
      finish_precond(S, acc.v[0], acc.v[1]);
  }
}

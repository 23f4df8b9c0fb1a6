// Lithospheric flexure on the B200: (L D L + C) x = b by preconditioned conjugate gradients.
//
// This is the device implementation behind dt_flex_* (include/deeptime_gpu.h). It solves the
// system of the reference's flexure::Solver (crates/deeptime-core/src/surface/flexure.rs:
// operator :1546-1624, Spectral :1108-1348, Bank :1352-1402, Preconditioner :1405-1468,
// Solver::solve :1680-1740) with its own kernels:
//
//   k_apply      the 13-point variable-D biharmonic y = L(d L v) + c v over a shared-memory tile
//                with a 2-cell halo (x wraps, rows clamp), fused with the CG reduction of its
//                caller (p.Ap, ||b - Ax||^2, or the Jacobi sandwich of the preconditioner);
//   k_rows_fwd   per row: a real FFT of length w as a complex FFT of length w/2 (even samples
//                real, odd imaginary) and the usual split, written in a packed half spectrum:
//                column 0 holds (X[0], X[w/2]), both real;
//   k_cols       per group of columns: the DCT-II along y by Makhoul's reordering and one complex
//                FFT of length h, the division by d lambda^2 + c, the inverse DCT, all in shared
//                memory: one read and one write of the half spectrum;
//   k_rows_inv   the inverse of k_rows_fwd, fused with what its caller needs next (store, weighted
//                accumulation for the bank's blend, or r.z and max|z|);
//   k_update, k_direction  the CG vector updates with their reductions.
//
// Reductions are deterministic: per-block partials in a fixed grid and a fixed order, summed by
// the last block to finish. The PCG loop runs on the device as a CUDA-graph conditional WHILE
// node: the last kernels of an iteration decide whether the body runs again, so a solve makes no
// host round trip per iteration.
//
// Precision: the kernels are templated on T (double or float). DT_PREC_FP64 runs everything in
// double; DT_PREC_MIXED runs the inner PCG in float on a scaled residual and refines in double
// (residual b - A x, the solution and every dot-product accumulator stay double).
#include <cuda_runtime.h>

#include <algorithm>
#include <utility>
#include <cmath>
#include <complex>
#include <cstdarg>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "fft.cuh"
#include <cuda_pipeline.h>

namespace dt {

// ---------------------------------------------------------------------------------------------
// Device-resident solver state. One per precision lane; kernels read and update it.

enum { SITE_PAP = 0, SITE_UPDATE = 1, SITE_PRECOND = 2, SITE_RESID = 3, SITE_STATS = 4, SITE_DOT = 5, SITE_MISC = 6 };
enum { STOP_RUNNING = 0, STOP_CONVERGED = 1, STOP_BREAKDOWN = 2, STOP_CAP = 3, STOP_NONFINITE = 4 };

struct Scalars {
  // problem
  double bb;      // ||b||^2 of the system being solved
  double tol;     // MAX_Z: metres; REL: relative residual
  int max_it;
  int rule;       // DT_STOP_*
  int n;
  // iteration
  double rz, pap, alpha, beta, rr, err, rz_new;
  int it;
  int stop;
  int started;    // the first preconditioning (before the loop) is done
  int body_runs;
  // preconditioner bank (flexure.rs:1352-1402)
  double lo, hi, sum_c, sum_d;
  double node_d[3];
  double c_ref;
  int levels;
  // misc reductions
  double dot_out, max_out;
  unsigned long long cond;  // graph conditional handle, 0 outside a graph
  unsigned int ticket[8];
  // reliable updates (DT_PREC_MIXED_RELIABLE, FP32 lane only): the sloppy residual is replaced by
  // the FP64 one, x by the FP64 accumulation, whenever rr has fallen below delta2 * maxrr or
  // under the tolerance; gate_it == it marks an iteration that does so
  int reliable;
  int gate_it;
  double delta2, maxrr;
  double rr_true, bb_true;  // ||b - A x||^2 and ||b||^2 in FP64, unscaled
  int replacements;         // residual replacements so far
  unsigned long long cond_if;  // the loop body's IF node around the replacement, 0 without one
  int fault;                // a kernel's bounded wait ran out (the solve reports a device error)
  int wait_give_up;         // test support: the TMA stencil's tile waits give up at once
};

__device__ __forceinline__ void set_cond(Scalars* S, unsigned int v) {
  if (S->cond) cudaGraphSetConditional((cudaGraphConditionalHandle)S->cond, v);
}

// ---------------------------------------------------------------------------------------------
// Last-block finishers: the scalar work between kernels.

__device__ void finish_pap(Scalars* S, double pap) {
  S->pap = pap;
  if (!(isfinite(pap) && pap > 0.0)) {
    S->stop = isfinite(pap) ? STOP_BREAKDOWN : STOP_NONFINITE;
    set_cond(S, 0);
    return;
  }
  S->alpha = S->rz / pap;
}

__device__ void finish_update(Scalars* S, double rr) {
  S->rr = rr;
  S->it += 1;
  if (S->reliable) {
    // the sloppy residual only asks for a replacement; the FP64 residual decides convergence
    bool gate = false;
    if (!isfinite(rr)) {
      S->stop = STOP_NONFINITE;
    } else if (rr <= S->tol * S->tol * S->bb || rr < S->delta2 * S->maxrr) {
      S->gate_it = S->it;
      gate = true;
    } else if (S->it >= S->max_it) {
      S->stop = STOP_CAP;
    }
    if (S->cond_if) cudaGraphSetConditional((cudaGraphConditionalHandle)S->cond_if, gate ? 1u : 0u);
    if (S->stop) set_cond(S, 0);
    return;
  }
  if (!isfinite(rr)) {
    S->stop = STOP_NONFINITE;
  } else if (S->rule == DT_STOP_REL_RESIDUAL && rr <= S->tol * S->tol * S->bb) {
    S->stop = STOP_CONVERGED;
  } else if (S->rule == DT_STOP_RMS_RESIDUAL && rr <= S->tol * S->tol * (double)S->n) {
    S->stop = STOP_CONVERGED;
  } else if (S->rule != DT_STOP_MAX_Z && S->it >= S->max_it) {
    S->stop = STOP_CAP;
  }
  if (S->stop) set_cond(S, 0);
}

// After z = M^-1 r: rz = r.z, err = max|z| (flexure.rs:1719-1737).
__device__ void finish_precond(Scalars* S, double rz, double err) {
  S->err = err;
  S->rz_new = rz;
  if (!isfinite(rz) || !isfinite(err)) {
    S->stop = STOP_NONFINITE;
    set_cond(S, 0);
    return;
  }
  if (!S->started) {
    S->started = 1;
    S->rz = rz;
    if (S->rule == DT_STOP_MAX_Z && err < S->tol) S->stop = STOP_CONVERGED;
    return;
  }
  if (S->rule == DT_STOP_MAX_Z) {
    if (err < S->tol) {
      S->stop = STOP_CONVERGED;
    } else if (S->it >= S->max_it) {
      S->stop = STOP_CAP;
    }
  }
  if (S->stop) {
    set_cond(S, 0);
    return;
  }
  S->beta = rz / S->rz;
  S->rz = rz;
}

// Bank::new from ln(alpha) extremes and the sums (flexure.rs:1361-1401); `mean_d` selects the
// single mean level instead.
__device__ void finish_stats(Scalars* S, double lo, double hi, double sum_c, double sum_d, double dx, bool mean_d, size_t cells) {
  const double RHO_MANTLE = 3300.0;
  double n = (double)(cells > 0 ? cells : 1);
  S->lo = lo;
  S->hi = hi;
  S->sum_c = sum_c;
  S->sum_d = sum_d;
  S->c_ref = sum_c / n;
  if (mean_d) {
    S->levels = 1;
    S->node_d[0] = sum_d / n;
    return;
  }
  auto node_d = [&](double ln_a) {
    double a = exp(ln_a) * dx;
    double a2 = a * a;
    return RHO_MANTLE * (a2 * a2) / 4.0;
  };
  double floor_ = log(0.4);
  if (hi - lo < 0.05 || hi <= floor_) {
    S->levels = 1;
    S->node_d[0] = node_d(0.5 * (lo + hi));
    return;
  }
  lo = fmax(lo, floor_);
  S->lo = lo;
  S->levels = 3;
  for (int k = 0; k < 3; ++k) S->node_d[k] = node_d(lo + (hi - lo) * (double)k / 2.0);
}

// ---------------------------------------------------------------------------------------------
// Reduction epilogue shared by the kernels: block partials -> last block -> finisher.

// ---------------------------------------------------------------------------------------------
// The 13-point operator over a tile.

enum {
  AP_DOT = 0,     // y = A v, reduce v.y                        (CG: Ap, p.Ap)
  RESID = 1,      // y = b - A v, reduce y.y                    (refinement residual)
  JAC_LEFT = 2,   // u = J r;         y = r - A u               (preconditioner: left)
  JAC_FINAL = 3,  // u = J r + part;  y = u + J (r - A u), reduce r.y and max|y|
  PLAIN = 4,      // y = A v
  BEND = 5,       // y = L (d L v)
  RESID_GATED = 6 // RESID in an iteration that replaces the residual (S->gate_it == S->it),
                  // ||y||^2 into S->rr_true; otherwise nothing
};

// tiles of 64 x 32 cells (FP32) or 64 x 16 (FP64), 64 x 4 threads: thread (tx, ty) owns column tx
// of the tile and a strip of TBY / 4 rows, which it walks with a sliding window of registers
constexpr int TBX = 64, TTY = 4, TBY_MIN = 16;
template <class T>
__host__ __device__ constexpr int tile_rows() { return sizeof(T) == 8 ? 16 : 32; }

// Shared-memory tile rows: local column lc (relative to the tile's first column) sits at offset
// OFF + lc with OFF = one 16-byte vector, so a row's interior starts on a 16-byte boundary and is
// staged with 16-byte copies; PITCH holds two halo columns either side, rounded to whole vectors.
template <class T>
struct Tile {
  static constexpr int V = 16 / (int)sizeof(T);
  static constexpr int OFF = V;
  static constexpr int PITCH = (OFF + TBX + 2 + V - 1) / V * V;
};

// Stages local rows [LR0, LR0 + ROWS) (relative to the tile's first row, clamped into [0, h)) and
// local columns [-HALO, TBX + HALO) (wrapped) of src into dst, row rr at dst + rr * PITCH. With
// `vec` (a whole tile of 16-byte aligned rows) the interior goes as 16-byte copies and only the
// halo columns one value at a time.
template <class T, int ROWS, int HALO, int LR0>
__device__ __forceinline__ void stage_tile(T* dst, const T* __restrict__ src, int w, int h, int i0, int j0, bool vec,
                                           int tid) {
  constexpr int NTH = TBX * TTY;
  constexpr int V = Tile<T>::V, OFF = Tile<T>::OFF, P = Tile<T>::PITCH;
  if (vec) {
    constexpr int VPR = TBX / V;
    for (int e = tid; e < ROWS * VPR; e += NTH) {
      int rr = e / VPR, q = e - rr * VPR;
      int g = min(max(j0 + LR0 + rr, 0), h - 1);
      __pipeline_memcpy_async(dst + rr * P + OFF + q * V, src + (size_t)g * w + i0 + q * V, 16);
    }
    for (int e = tid; e < ROWS * 2 * HALO; e += NTH) {
      int rr = e / (2 * HALO), hc = e - rr * (2 * HALO);
      int lc = hc < HALO ? hc - HALO : TBX + hc - HALO;
      int gc = i0 + lc;
      gc = gc < 0 ? gc + w : (gc >= w ? gc - w : gc);
      int g = min(max(j0 + LR0 + rr, 0), h - 1);
      __pipeline_memcpy_async(dst + rr * P + OFF + lc, src + (size_t)g * w + gc, sizeof(T));
    }
  } else {
    constexpr int RW = TBX + 2 * HALO;
    for (int e = tid; e < ROWS * RW; e += NTH) {
      int rr = e / RW, lc = e - rr * RW - HALO;
      int gc = (i0 + lc) % w;
      gc = gc < 0 ? gc + w : gc;
      int g = min(max(j0 + LR0 + rr, 0), h - 1);
      __pipeline_memcpy_async(dst + rr * P + OFF + lc, src + (size_t)g * w + gc, sizeof(T));
    }
  }
}

__device__ __forceinline__ bool aligned16(const void* p) { return ((size_t)p & 15) == 0; }

// A row's couplings on the sphere's metric (RowMetric, flexure.rs:954-998): east-west a_j, the
// boundaries above and below b_j, b_(j+1); rows outside the raster take the edge row's.
template <class T, bool MET>
struct RowCoef {
  T a, bn, bs;
};
template <class T, bool MET>
__device__ __forceinline__ RowCoef<T, MET> row_coef(const T* __restrict__ ma, const T* __restrict__ mb, int j, int h) {
  RowCoef<T, MET> r{(T)1, (T)1, (T)1};
  if (MET) {
    const int jc = min(max(j, 0), h - 1);
    r.a = ma[jc];
    r.bn = mb[jc];
    r.bs = mb[jc + 1];
  }
  return r;
}
// The 5-point Laplacian of cell x from its west, east, north and south neighbours: the block
// metric's (flexure.rs:1575-1580), or the sphere's a (W + E - 2x) + bn (N - x) + bs (S - x)
// (flexure.rs:1559-1570), in the reference's order of operations.
template <class T, bool MET>
__device__ __forceinline__ T lap5(T we, T ea, T no, T so, T x, const RowCoef<T, MET>& k, T inv) {
  if (MET) return (k.a * (we + ea - (T)2 * x) + k.bn * (no - x) + k.bs * (so - x)) * inv;
  return (we + ea + no + so - (T)4 * x) * inv;
}

// MET: on the sphere's row metric (ma: h values a_j, mb: h + 1 values b_j); the block metric
// otherwise.
template <class T, int MODE, bool MET = false>
__global__ void __launch_bounds__(TBX* TTY) k_apply(int w, int h, T inv_dx2, const T* __restrict__ v, const T* __restrict__ J,
                                                    const T* __restrict__ part, const T* __restrict__ d,
                                                    const T* __restrict__ c, const T* __restrict__ rb, T* __restrict__ y,
                                                    double* partials, Scalars* S, const T* __restrict__ ma = nullptr,
                                                    const T* __restrict__ mb = nullptr) {
  if (MODE != PLAIN && MODE != BEND && MODE != RESID) {
    if (S->stop) {
      if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0 && threadIdx.y == 0) set_cond(S, 0);
      return;
    }
  }
  if (MODE == RESID_GATED && S->gate_it != S->it) return;
  constexpr bool JAC = MODE == JAC_LEFT || MODE == JAC_FINAL;
  constexpr bool HAS_B = MODE == RESID || MODE == RESID_GATED;
  constexpr int TBY = tile_rows<T>(), SEG = TBY / TTY;
  constexpr int P = Tile<T>::PITCH, OFF = Tile<T>::OFF;
  constexpr int UR = TBY + 4, MR = TBY + 2;  // vector rows -2 .. TBY + 1; d / m rows -1 .. TBY
  __shared__ __align__(16) T sv[UR * P];                    // the vector (JAC: r)
  __shared__ __align__(16) T sJ[JAC ? UR * P : 1];          // JAC: J
  __shared__ __align__(16) T sP[JAC ? UR * P : 1];          // JAC_FINAL: part; then (JAC) u
  __shared__ __align__(16) T sd[MR * P];                    // d; then m = d L u in place
  const int i0 = blockIdx.x * TBX, j0 = blockIdx.y * TBY;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int tid = tx + ty * TBX;
  const T* src = JAC ? rb : v;
  const bool vec = i0 + TBX <= w && (w * (int)sizeof(T)) % 16 == 0 && aligned16(src) && aligned16(d) &&
                   (!JAC || aligned16(J)) && (MODE != JAC_FINAL || aligned16(part));
  // Stage the tiles with asynchronous copies (every load in flight at once): rows clamp, columns
  // wrap.
  stage_tile<T, UR, 2, -2>(sv, src, w, h, i0, j0, vec, tid);
  if (JAC) stage_tile<T, UR, 2, -2>(sJ, J, w, h, i0, j0, vec, tid);
  if (MODE == JAC_FINAL) stage_tile<T, UR, 2, -2>(sP, part, w, h, i0, j0, vec, tid);
  stage_tile<T, MR, 1, -1>(sd, d, w, h, i0, j0, vec, tid);
  __pipeline_commit();
  // c (and b) for the thread's own output cells, in flight with the tiles
  const int i = i0 + tx, r0 = ty * SEG;
  T cr[SEG], br[HAS_B ? SEG : 1];
#pragma unroll
  for (int q = 0; q < SEG; ++q) {
    int j = j0 + r0 + q;
    bool ok = i < w && j < h;
    size_t k = (size_t)j * w + i;
    if (MODE != BEND) cr[q] = ok ? c[k] : (T)0;
    if (HAS_B) br[q] = ok ? rb[k] : (T)0;
  }
  __pipeline_wait_prior(0);
  __syncthreads();
  if (JAC) {
    // the vector the mode forms: u = J r (+ part); r and J stay readable for the outputs
    for (int e = tid; e < UR * P; e += TBX * TTY) {
      T u = sJ[e] * sv[e];
      if (MODE == JAC_FINAL) u += sP[e];
      sP[e] = u;
    }
    __syncthreads();
  }
  const T* su = JAC ? sP : sv;
  // m = d . L u at local rows -1 .. TBY, columns -1 .. TBX. Column tx over the thread's strip
  // (the first strip also takes row -1, the last row TBY) with a sliding window down the column.
  {
    const int a = r0 - (ty == 0 ? 1 : 0);
    const T* ucol = su + OFF + tx;  // row lr at (lr + 2) * P
    T* mcol = sd + OFF + tx;        // row lr at (lr + 1) * P
    T un = ucol[(a + 1) * P], uc = ucol[(a + 2) * P];
#pragma unroll
    for (int q = 0; q < SEG + 1; ++q) {
      int lr = a + q;
      if (q == SEG && !(ty == 0 || ty == TTY - 1)) break;
      T us = ucol[(lr + 3) * P];
      T lap = lap5<T, MET>(ucol[(lr + 2) * P - 1], ucol[(lr + 2) * P + 1], un, us, uc, row_coef<T, MET>(ma, mb, j0 + lr, h),
                           inv_dx2);
      mcol[(lr + 1) * P] = lap * mcol[(lr + 1) * P];
      un = uc;
      uc = us;
    }
  }
  // columns -1 and TBX over all rows
  for (int e = tid; e < 2 * MR; e += TBX * TTY) {
    int lr = (e >> 1) - 1, lc = (e & 1) ? TBX : -1;
    const T* uc = su + (lr + 2) * P + OFF + lc;
    T lap = lap5<T, MET>(uc[-1], uc[1], uc[-P], uc[P], uc[0], row_coef<T, MET>(ma, mb, j0 + lr, h), inv_dx2);
    T* m = sd + (lr + 1) * P + OFF + lc;
    *m = lap * *m;
  }
  __syncthreads();
  // rows of m outside the raster repeat its edge rows (rows clamp): m(-1) = m(0), m(h) = m(h - 1)
  {
    const int hb = h - 1 - j0;  // local index of the raster's last row
    const bool top = j0 == 0, bottom = hb + 1 <= TBY;
    if (top || bottom) {
      for (int e = tid; e < TBX + 2; e += TBX * TTY) {
        if (top) sd[0 * P + OFF - 1 + e] = sd[1 * P + OFF - 1 + e];
        if (bottom) sd[(hb + 2) * P + OFF - 1 + e] = sd[(hb + 1) * P + OFF - 1 + e];
      }
      __syncthreads();
    }
  }
  Acc<2> acc;
  acc.v[0] = 0.0;
  acc.v[1] = 0.0;
  {
    const T* mcol = sd + OFF + tx;  // m row lr at (lr + 1) * P
    T mn = mcol[r0 * P], mc = mcol[(r0 + 1) * P];
#pragma unroll
    for (int q = 0; q < SEG; ++q) {
      const int lr = r0 + q;
      T ms = mcol[(lr + 2) * P];
      T lm = lap5<T, MET>(mcol[(lr + 1) * P - 1], mcol[(lr + 1) * P + 1], mn, ms, mc, row_coef<T, MET>(ma, mb, j0 + lr, h),
                          inv_dx2);
      mn = mc;
      mc = ms;
      int j = j0 + lr;
      if (i < w && j < h) {
        size_t k = (size_t)j * w + i;
        T u = su[(lr + 2) * P + OFF + tx];
        if (MODE == BEND) {
          y[k] = lm;
        } else {
          T au = lm + cr[q] * u;
          if (MODE == AP_DOT) {
            y[k] = au;
            acc.v[0] += (double)u * (double)au;
          } else if (MODE == PLAIN) {
            y[k] = au;
          } else if (HAS_B) {
            T rr = br[q] - au;
            y[k] = rr;
            acc.v[0] += (double)rr * (double)rr;
          } else if (MODE == JAC_LEFT) {
            y[k] = sv[(lr + 2) * P + OFF + tx] - au;
          } else {  // JAC_FINAL
            T r = sv[(lr + 2) * P + OFF + tx];
            T z = u + sJ[(lr + 2) * P + OFF + tx] * (r - au);
            y[k] = z;
            acc.v[0] += (double)r * (double)z;
            acc.v[1] = fmax(acc.v[1], fabs((double)z));
          }
        }
      }
    }
  }
  if (MODE == AP_DOT || MODE == RESID || MODE == RESID_GATED || MODE == JAC_FINAL) {
    const int kind[2] = {0, 1};
    unsigned int nb = gridDim.x * gridDim.y;
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
#include "stencil_tma.cuh"
#include <cudaTypedefs.h>
namespace dt {

// ---------------------------------------------------------------------------------------------
// CG vector kernels (grid-stride).

// 16 bytes of T: the vector kernels move whole 16-byte words (the handle's buffers are aligned)
template <class T>
struct alignas(16) Vec16 {
  T a[16 / sizeof(T)];
};

// x += alpha p; r -= alpha Ap; reduce r.r
template <class T>
__global__ void __launch_bounds__(256) k_update(size_t n, T* __restrict__ x, T* __restrict__ r, const T* __restrict__ p,
                                                const T* __restrict__ ap, double* partials, Scalars* S) {
  if (S->stop) {
    if (blockIdx.x == 0 && threadIdx.x == 0) set_cond(S, 0);
    return;
  }
  constexpr int V = 16 / sizeof(T);
  using W = Vec16<T>;
  T alpha = (T)S->alpha;
  Acc<1> acc;
  acc.v[0] = 0.0;
  const size_t nv = n / V, stride = (size_t)gridDim.x * blockDim.x;
  const size_t t0 = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  W* xv = reinterpret_cast<W*>(x);
  W* rv = reinterpret_cast<W*>(r);
  const W* pv = reinterpret_cast<const W*>(p);
  const W* av = reinterpret_cast<const W*>(ap);
  for (size_t kv = t0; kv < nv; kv += stride) {
    W xx = xv[kv], rr = rv[kv], pp = pv[kv], aa = av[kv];
#pragma unroll
    for (int e = 0; e < V; ++e) {
      xx.a[e] += alpha * pp.a[e];
      rr.a[e] = rr.a[e] - alpha * aa.a[e];
      acc.v[0] += (double)rr.a[e] * (double)rr.a[e];
    }
    xv[kv] = xx;
    rv[kv] = rr;
  }
  for (size_t k = nv * V + t0; k < n; k += stride) {
    x[k] += alpha * p[k];
    T rk = r[k] - alpha * ap[k];
    r[k] = rk;
    acc.v[0] += (double)rk * (double)rk;
  }
  const int kind[1] = {0};
  if (reduce_partials<1>(acc, kind, partials, &S->ticket[SITE_UPDATE], gridDim.x) && threadIdx.x == 0) finish_update(S, acc.v[0]);
}

// p = z + beta p; also the loop's guard: the body runs again only while nothing stopped it and
// fewer than max_it + 2 bodies ran.
template <class T>
__global__ void __launch_bounds__(256) k_direction(size_t n, T* __restrict__ p, const T* __restrict__ z, Scalars* S) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    int runs = ++S->body_runs;
    bool again = S->stop == 0 && runs < S->max_it + 2;
    if (!again && S->stop == 0) S->stop = STOP_CAP;
    set_cond(S, again ? 1u : 0u);
  }
  if (S->stop) return;
  constexpr int V = 16 / sizeof(T);
  using W = Vec16<T>;
  T beta = (T)S->beta;
  const size_t nv = n / V, stride = (size_t)gridDim.x * blockDim.x;
  const size_t t0 = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  W* pv = reinterpret_cast<W*>(p);
  const W* zv = reinterpret_cast<const W*>(z);
  for (size_t kv = t0; kv < nv; kv += stride) {
    W pp = pv[kv], zz = zv[kv];
#pragma unroll
    for (int e = 0; e < V; ++e) pp.a[e] = zz.a[e] + beta * pp.a[e];
    pv[kv] = pp;
  }
  for (size_t k = nv * V + t0; k < n; k += stride) p[k] = z[k] + beta * p[k];
}

template <class A, class B>
__global__ void k_convert(size_t n, const A* __restrict__ a, B* __restrict__ b) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) b[k] = (B)a[k];
}

// r32 = r64 * s (s from the residual's RMS), e32 = 0
__global__ void k_scale_down(size_t n, const double* __restrict__ r, float* __restrict__ r32, float* __restrict__ e32,
                             const Scalars* S64, double* scale_out) {
  double s = S64->rr > 0 ? sqrt((double)n / S64->rr) : 1.0;
  if (blockIdx.x == 0 && threadIdx.x == 0) *scale_out = s;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    r32[k] = (float)(r[k] * s);
    e32[k] = 0.0f;
  }
}

// x64 += e32 / s
__global__ void k_accumulate(size_t n, double* __restrict__ x, const float* __restrict__ e32, const double* scale) {
  double inv = 1.0 / *scale;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) x[k] += (double)e32[k] * inv;
}

// Reliable updates (the sloppy lane holds r32 = s r64 and its correction x32 = s e). In an
// iteration that replaces the residual (gate_it == it):
//   k_reliable_accumulate  x64 += x32 / s; x32 = 0
//   k_apply<double, RESID_GATED>  r64 = b - A x64, ||r64||^2 -> rr_true
//   k_reliable_reset       r32 = s r64; rr, maxrr from rr_true; stop when rr_true meets the
//                          tolerance
__global__ void k_reliable_accumulate(size_t n, double* __restrict__ x, float* __restrict__ e32, const double* scale,
                                      const Scalars* S) {
  if (S->stop || S->gate_it != S->it) return;
  double inv = 1.0 / *scale;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    x[k] += (double)e32[k] * inv;
    e32[k] = 0.0f;
  }
}

__global__ void k_reliable_reset(size_t n, const double* __restrict__ r, float* __restrict__ r32, const double* scale,
                                 Scalars* S) {
  if (S->stop || S->gate_it != S->it) return;
  double sc = *scale;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
    r32[k] = (float)(r[k] * sc);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    double rr = S->rr_true * sc * sc;
    S->rr = rr;
    S->maxrr = rr;
    S->replacements += 1;
    if (!isfinite(S->rr_true)) {
      S->stop = STOP_NONFINITE;
    } else if (S->rr_true <= S->tol * S->tol * S->bb_true) {
      S->stop = STOP_CONVERGED;
    }
    if (S->stop) set_cond(S, 0);
  }
}

// The FP32 lane's problem for reliable updates, from the FP64 lane's (bb, rr of r = b - A x) and
// the scale s of r32 = s r. The tolerance is on the relative residual, or with `rms` on the RMS
// residual (||r||^2 <= tol^2 n).
__global__ void k_reliable_init(Scalars* F, const Scalars* S64, const double* scale, double tol, int max_it, double delta,
                                int rms) {
  double s2 = (*scale) * (*scale);
  double bref = rms ? (double)S64->n : S64->bb;
  F->tol = tol;
  F->max_it = max_it;
  F->rule = DT_STOP_REL_RESIDUAL;
  F->bb = bref * s2;
  F->bb_true = bref;
  F->rr = S64->rr * s2;
  F->maxrr = F->rr;
  F->delta2 = delta * delta;
  F->gate_it = -1;
  F->reliable = 1;
  F->replacements = 0;
  F->cond_if = 0ull;
}

template <class T>
__global__ void k_fill(size_t n, T* __restrict__ a, T v) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) a[k] = v;
}

// reduce a.b (and max |b| when MAXB) into S->dot_out / S->max_out
template <class T>
__global__ void __launch_bounds__(256) k_dot(size_t n, const T* __restrict__ a, const T* __restrict__ b, double* partials, Scalars* S,
                                             int site) {
  Acc<2> acc;
  acc.v[0] = 0.0;
  acc.v[1] = 0.0;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    acc.v[0] += (double)a[k] * (double)b[k];
    acc.v[1] = fmax(acc.v[1], fabs((double)b[k]));
  }
  const int kind[2] = {0, 1};
  if (reduce_partials<2>(acc, kind, partials, &S->ticket[site], gridDim.x) && threadIdx.x == 0) {
    S->dot_out = acc.v[0];
    S->max_out = acc.v[1];
  }
}

// ---------------------------------------------------------------------------------------------
// Preconditioner set-up (flexure.rs:1361-1401 and :1426-1460).

template <class T>
__global__ void __launch_bounds__(256) k_stats(size_t n, const T* __restrict__ d, const T* __restrict__ c, double dx, int mean_d,
                                               double* partials, Scalars* S) {
  const double RHO_MANTLE = 3300.0;
  // ln(alpha) rises with d, so its extremes are those of the least and the greatest d: two
  // evaluations at the end instead of one a cell
  Acc<4> acc;
  acc.v[0] = -INFINITY;  // -(least d) as a max
  acc.v[1] = -INFINITY;  // greatest d
  acc.v[2] = 0.0;        // sum c
  acc.v[3] = 0.0;        // sum d
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    double dv = (double)d[k];
    acc.v[0] = fmax(acc.v[0], -dv);
    acc.v[1] = fmax(acc.v[1], dv);
    acc.v[2] += (double)c[k];
    acc.v[3] += dv;
  }
  const int kind[4] = {1, 1, 0, 0};
  if (reduce_partials<4>(acc, kind, partials, &S->ticket[SITE_STATS], gridDim.x) && threadIdx.x == 0) {
    auto la = [&](double dv) { return log(pow(4.0 * fmax(dv, 1e-30) / RHO_MANTLE, 0.25) / dx); };
    finish_stats(S, la(-acc.v[0]), la(acc.v[1]), acc.v[2], acc.v[3], dx, mean_d != 0, n);
  }
}

// Per cell: the bank's weights (squares sum to one) and the damped Jacobi weight 1/2 / diag.
template <class T>
__global__ void __launch_bounds__(256) k_bank_weights(int w, int h, const T* __restrict__ d, const T* __restrict__ c, double dx,
                                                      T* __restrict__ w0, T* __restrict__ w1, T* __restrict__ w2,
                                                      T* __restrict__ jac, const Scalars* S,
                                                      const double* __restrict__ ma = nullptr,
                                                      const double* __restrict__ mb = nullptr) {
  const double RHO_MANTLE = 3300.0;
  size_t n = (size_t)w * h;
  double lo = S->lo, hi = S->hi;
  double inv4 = 1.0 / (dx * dx * dx * dx);
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    int i = (int)(k % w), j = (int)(k / w);
    double dv = (double)d[k];
    double la = log(pow(4.0 * fmax(dv, 1e-30) / RHO_MANTLE, 0.25) / dx);
    double t = fmin(fmax((la - lo) / (hi - lo), 0.0), 1.0) * 2.0;
    int k0 = min((int)floor(t), 1);
    double f = t - (double)k0;
    double a = sqrt(1.0 - f), b = sqrt(f);
    w0[k] = (T)(k0 == 0 ? a : 0.0);
    w1[k] = (T)(k0 == 0 ? b : a);
    w2[k] = (T)(k0 == 1 ? b : 0.0);
    double east = (double)d[(size_t)j * w + (i + 1) % w], west = (double)d[(size_t)j * w + (i + w - 1) % w];
    double north = (double)d[(size_t)max(j - 1, 0) * w + i], south = (double)d[(size_t)min(j + 1, h - 1) * w + i];
    if (ma) {
      // (L D L)'s diagonal on the sphere's row metric (flexure.rs:1444-1452)
      double a = ma[j], bn = mb[j], bs = mb[j + 1];
      double centre = 2.0 * a + bn + bs;
      double diag = dv * centre * centre + (east + west) * a * a + north * bn * bn + south * bs * bs;
      jac[k] = (T)(0.5 / ((double)c[k] + diag * inv4));
    } else {
      double around = east + west + north + south;
      jac[k] = (T)(0.5 / ((double)c[k] + (16.0 * dv + around) * inv4));
    }
  }
}

// ---------------------------------------------------------------------------------------------
// The spectral solve (flexure.rs:1183-1347), three passes over a packed half spectrum of h rows
// by N = w/2 complex values. Each thread of a transform kernel holds FFT_EPT complex values per
// FFT stage, so a block of `batch` sequences of length L has batch * L / FFT_EPT threads.

// INV_BANK: the bank's three levels in one pass, out = sum_k wt_k x_k, the levels' spectra and
// weights consecutive (half + k h N, wt + k w h)
enum { INV_STORE = 0, INV_STORE_DOT = 2, INV_STORE_W = 3, INV_BANK = 4 };
// Correctly rounded reciprocals (double: one division; float: the intrinsic).
__device__ __forceinline__ double recip(double x) { return 1.0 / x; }
__device__ __forceinline__ float recip(float x) { return __frcp_rn(x); }
// Reciprocals with no slow-path call, for code that keeps many values in registers around them:
// float, the hardware's approximate reciprocal (__fdividef, at most 2 ulp for |x| in
// [2^-126, 2^126]); double, that estimate refined by two Newton-Raphson steps r <- r + r (1 - x r)
// (each squares the relative error: 2^-22 -> 2^-44 -> 2^-88). Used for the spectral divisors
// d lambda^2 + c_ref, which lie in (c_ref, 1e36) for any raster this solver takes.
__device__ __forceinline__ float recip_fast(float x) { return __fdividef(1.0f, x); }
__device__ __forceinline__ double recip_fast(double x) {
  double r = (double)__fdividef(1.0f, (float)x);
  r = fma(r, fma(-x, r, 1.0), r);
  return fma(r, fma(-x, r, 1.0), r);
}
constexpr int FFT_EPT = 16;
constexpr int FFT_BATCH = 8;  // global loads a thread of a transform kernel keeps in flight
constexpr int FFT_MAX_THREADS = 512;

// Rows per block so that a block has at least one warp.
__host__ __device__ constexpr int rows_per_block(int logn) { return (32 * FFT_EPT >> logn) > 1 ? (32 * FFT_EPT >> logn) : 1; }
// Columns per block of the column pass: at least one warp, at most FFT_MAX_THREADS threads,
// 100 KB of padded shared memory, 8 columns.
// Column pitch of the column pass: the padded length rounded up to 4 (mod 16), so that the first
// and last stages' interleaved accesses (CPB columns x consecutive rows) fall in distinct banks.
__host__ __device__ constexpr int col_pitch(int h) {
  int l = h + (h >> 4) + 1;
  return l + ((4 - l % 16) + 16) % 16;
}
__host__ __device__ constexpr int cols_per_block(int logh, int elem) {
  int h = 1 << logh;
  int plen = col_pitch(h);
  int cpb = (32 * FFT_EPT >> logh) > 1 ? (32 * FFT_EPT >> logh) : 1;
  while (cpb < 8 && cpb * 2 * h <= FFT_MAX_THREADS * FFT_EPT && cpb * 2 * plen * elem <= 102400) cpb *= 2;
  return cpb;
}

template <class T, bool WEIGHT, int LOGN>
__global__ void __launch_bounds__(FFT_MAX_THREADS, sizeof(T) == 4 ? 2 : 1) k_rows_fwd(int w, int h, const T* __restrict__ v, const T* __restrict__ wt,
                                                             cplx<T>* __restrict__ half, const cplx<T>* __restrict__ tw,
                                                             const cplx<T>* __restrict__ post, const Scalars* S) {
  using C = cplx<T>;
  using P = Pad<C>;
  if (S->stop) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* s = reinterpret_cast<C*>(smem_raw);
  constexpr int N = 1 << LOGN, NP = P::len(N);
  constexpr int logN = LOGN;
  constexpr int RB = rows_per_block(LOGN);
  // the bank's levels in one launch: level blockIdx.y's weights and spectrum, both consecutive
  if (WEIGHT) wt += (size_t)blockIdx.y * (2 * N) * h;
  half += (size_t)blockIdx.y * h * N;
  const int row0 = blockIdx.x * RB;
  const int tid = threadIdx.x;
  // load rows as complex pairs (v[2n], v[2n+1]): one 2-wide vector load per pair. The block has
  // NT threads (fft_geometry), FFT_EPT pairs each; loads go out in batches before the shared
  // stores so that a thread keeps FFT_BATCH of them in flight.
  constexpr int NT = RB * N / FFT_EPT;
  static_assert(NT * FFT_EPT == RB * N, "rows: whole pairs per thread");
  // the raster's width w is 2 N: row offsets use the compile-time 2 N
  if constexpr (RB == 1 && LOGN >= 4) {
    // one row per block: the first stage (radix 16, span 1) straight from global memory, thread
    // j taking pairs n = j + r N/16 (consecutive threads, consecutive pairs)
    const int j = tid;
    C z[16];
#pragma unroll
    for (int r = 0; r < 16; ++r) {
      z[r] = mk<C>((T)0, (T)0);
      if (row0 < h) {
        size_t k = (size_t)row0 * (2 * N) + 2 * (j + r * (N / 16));
        z[r] = *reinterpret_cast<const C*>(v + k);
        if (WEIGHT) {
          C ww = *reinterpret_cast<const C*>(wt + k);
          z[r].x *= ww.x;
          z[r].y *= ww.y;
        }
      }
    }
    dft_r<C, 16, false>(z);
#pragma unroll
    for (int r = 0; r < 16; ++r) s[17 * j + r] = z[r];  // pad(16 j + r) = 17 j + r
    __syncthreads();
    Stages<C, FFT_EPT, false, LOGN, 16, LOGN - 4, 0, NT>::run(s, tw);
  } else {
#pragma unroll 1
    for (int q0 = 0; q0 < FFT_EPT; q0 += FFT_BATCH) {
      C zb[FFT_BATCH];
#pragma unroll
      for (int u = 0; u < FFT_BATCH; ++u) {
        int idx = tid + (q0 + u) * NT;
        int rb = idx >> logN, nn = idx & (N - 1);
        int j = row0 + rb;
        C z = mk<C>((T)0, (T)0);
        if (j < h) {
          size_t k = (size_t)j * (2 * N) + 2 * nn;
          z = *reinterpret_cast<const C*>(v + k);
          if (WEIGHT) {
            C ww = *reinterpret_cast<const C*>(wt + k);
            z.x *= ww.x;
            z.y *= ww.y;
          }
        }
        zb[u] = z;
      }
#pragma unroll
      for (int u = 0; u < FFT_BATCH; ++u) {
        int idx = tid + (q0 + u) * NT;
        s[(idx >> logN) * NP + P::at(idx & (N - 1))] = zb[u];
      }
    }
    __syncthreads();
    smem_fft<C, FFT_EPT, false, LOGN, NT>(s, tw);
  }
  // split: X[k] = E[k] + W^k O[k], E = (Z[k] + conj Z[N-k]) / 2, O = (Z[k] - conj Z[N-k]) / 2i
  constexpr int half_n = N / 2 + 1;
#pragma unroll 2
  for (int idx = tid; idx < RB * half_n; idx += NT) {
    int rb = idx / half_n, kk = idx - rb * half_n;
    int j = row0 + rb;
    if (j >= h) continue;
    const C* row = s + rb * NP;
    C* out = half + (size_t)j * N;
    if (kk == 0) {
      C z0 = row[0];
      out[0] = mk<C>(z0.x + z0.y, z0.x - z0.y);  // (X[0], X[N]) both real
      continue;
    }
    C zk = row[P::at(kk)], zn = row[P::at(N - kk)];
    C E = mk<C>((zk.x + zn.x) * (T)0.5, (zk.y - zn.y) * (T)0.5);
    C O = mk<C>((zk.y + zn.y) * (T)0.5, (zn.x - zk.x) * (T)0.5);
    C wo = cmul(post[kk], O);
    out[kk] = cadd(E, wo);
    if (kk != N - kk) out[N - kk] = cconj(csub(E, wo));
  }
}

// The column pass: DCT-II along y (Makhoul), divide by d lambda^2 + c_ref, inverse DCT.
// lx[k] = 2 cos(2 pi k / w) - 2 for k = 0..N; ly[m] = 2 cos(pi m / h) - 2.
template <class T, int LOGH>
__global__ void __launch_bounds__(FFT_MAX_THREADS, sizeof(T) == 4 ? 2 : 1) k_cols(int N, cplx<T>* __restrict__ half, const cplx<T>* __restrict__ tw,
                                                         const cplx<T>* __restrict__ omega, const cplx<T>* __restrict__ omega2, const T* __restrict__ lx,
                                                         const T* __restrict__ ly, T inv_dx2, const Scalars* S, int level) {
  using C = cplx<T>;
  using P = Pad<C>;
  if (S->stop) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* s = reinterpret_cast<C*>(smem_raw);
  constexpr int h = 1 << LOGH;
  constexpr int HP = col_pitch(h);
  constexpr int CPB = cols_per_block(LOGH, (int)sizeof(C));
  constexpr int logc = CPB == 1 ? 0 : CPB == 2 ? 1 : CPB == 4 ? 2 : CPB == 8 ? 3 : CPB == 16 ? 4 : CPB == 32 ? 5 : CPB == 64 ? 6 : CPB == 128 ? 7 : 8;
  // the bank's levels in one launch: level + blockIdx.y, its spectrum consecutive
  half += (size_t)blockIdx.y * h * N;
  level += blockIdx.y;
  const int k0 = blockIdx.x * CPB;
  const int tid = threadIdx.x;
  const T dref = (T)S->node_d[level], cref = (T)S->c_ref;
  // NT threads (fft_geometry), FFT_EPT values each
  constexpr int NT = CPB * h / FFT_EPT;
  static_assert(NT * FFT_EPT == CPB * h, "columns: whole values per thread");
  // Makhoul's order: v[p] = x[2p] for p < h/2, x[2(h - 1 - p) + 1] after
  if constexpr (LOGH < 4) {
    // short columns: gather in Makhoul's order (consecutive threads: consecutive columns)
#pragma unroll 1
    for (int q0 = 0; q0 < FFT_EPT; q0 += FFT_BATCH) {
      C xb[FFT_BATCH];
#pragma unroll
      for (int u = 0; u < FFT_BATCH; ++u) {
        int idx = tid + (q0 + u) * NT;
        int j = idx >> logc, k = k0 + (idx & (CPB - 1));
        xb[u] = k < N ? half[(size_t)j * N + k] : mk<C>((T)0, (T)0);
      }
#pragma unroll
      for (int u = 0; u < FFT_BATCH; ++u) {
        int idx = tid + (q0 + u) * NT;
        int j = idx >> logc, cc = idx & (CPB - 1);
        int pos = (j & 1) ? h - 1 - (j >> 1) : (j >> 1);
        s[cc * HP + P::at(pos)] = xb[u];
      }
    }
    __syncthreads();
    Stages<C, FFT_EPT, false, LOGH, 1, LOGH, HP, NT>::run(s, tw);
  } else {
    // The forward transform's first stage (radix 16, span 1) straight from global memory: thread
    // tid takes butterfly j = tid / CPB of column tid % CPB, i.e. v[j + r h/16], r = 0 .. 15; a
    // warp reads 32-byte row segments of CPB columns.
    const int cc = tid & (CPB - 1), j = tid >> logc, k = k0 + cc;
    C v[16];
#pragma unroll
    for (int r = 0; r < 16; ++r) {
      // j < h / 16, so j + r h / 16 < h / 2 exactly when r < 8: Makhoul's branch is known per r
      const int p = j + r * (h / 16), row = r < 8 ? 2 * p : 2 * (h - 1 - p) + 1;
      v[r] = k < N ? half[(size_t)row * N + k] : mk<C>((T)0, (T)0);
    }
    dft_r<C, 16, false>(v);
    C* col = s + cc * HP;
#pragma unroll
    for (int r = 0; r < 16; ++r) col[17 * j + r] = v[r];  // pad(16 j + r) = 17 j + r
    __syncthreads();
    Stages<C, FFT_EPT, false, LOGH, 16, LOGH - 4, HP, NT>::run(s, tw);
  }
  // per column and pair (m, h - m): C[m] = (w_m V[m] + i w_(h-m) V[h-m]) / 2, divide, and back
  constexpr int half_h = h / 2 + 1;
#pragma unroll 1
  for (int idx = tid; idx < CPB * half_h; idx += NT) {
    int cc = idx / half_h, m = idx - cc * half_h;
    int k = k0 + cc;
    if (k >= N) continue;
    C* col = s + cc * HP;
    // divisors: column 0 is packed (real part k = 0, imaginary part k = N)
    // 1 / (d lambda^2 + c): one reciprocal per divisor, then products
    auto rden = [&](int kx, T lyv) {
      T l = (lx[kx] + lyv) * inv_dx2;
      return recip(dref * (l * l) + cref);
    };
    const T lym = ly[m];
    if (m == 0) {
      C v0 = col[0];
      if (k == 0) {
        v0.x *= rden(0, lym);
        v0.y *= rden(N, lym);
      } else {
        T dd = rden(k, lym);
        v0.x *= dd;
        v0.y *= dd;
      }
      col[0] = v0;
      continue;
    }
    int mm = h - m;
    int pm = P::at(m), pn = P::at(mm);
    // w_(h-m) = -i conj(w_m) and ly[h-m] = -ly[m] - 4 (cos(pi - t) = -cos t): one table entry each
    const C wm = omega[m], wn = mk<C>(-wm.y, -wm.x);
    const T lyn = -lym - (T)4;
    C p = cmul(wm, col[pm]);
    C q = cmul(wn, col[pn]);
    C cm = cscale(cadd(p, cmuli(q)), (T)0.5);
    C cn = cscale(cadd(q, cmuli(p)), (T)0.5);
    if (k == 0) {
      cm.x *= rden(0, lym);
      cm.y *= rden(N, lym);
      cn.x *= rden(0, lyn);
      cn.y *= rden(N, lyn);
    } else {
      T a = rden(k, lym), b = rden(k, lyn);
      cm.x *= a;
      cm.y *= a;
      cn.x *= b;
      cn.y *= b;
    }
    // V'[m] = conj(w_m) (C[m] - i C[h-m])
    C vm = cmul(cconj(wm), csub(cm, cmuli(cn)));
    C vn = cmul(cconj(wn), csub(cn, cmuli(cm)));
    col[pm] = vm;
    if (mm != m) col[pn] = vn;
  }
  __syncthreads();
  // the same table through a pointer the compiler cannot prove equal to `tw`: otherwise it keeps
  // the forward stages' twiddles in registers for the inverse stages and spills
  const C* tw_inv;
  asm volatile("mov.b64 %0, %1;" : "=l"(tw_inv) : "l"(tw));
  const T inv_h = (T)1 / (T)h;
  if constexpr (LOGH < 4) {
    Stages<C, FFT_EPT, true, LOGH, 1, LOGH, HP, NT>::run(s, tw_inv);
#pragma unroll 4
    for (int idx = tid; idx < CPB * h; idx += NT) {
      int j = idx >> logc, cc = idx & (CPB - 1);
      int k = k0 + cc;
      if (k >= N) continue;
      int pos = (j & 1) ? h - 1 - (j >> 1) : (j >> 1);
      half[(size_t)j * N + k] = cscale(s[cc * HP + P::at(pos)], inv_h);
    }
  } else {
    // all stages but the last through shared memory; the last (radix RL, span h / RL, twiddles
    // w^(r j)) writes each output straight to its row of the half spectrum, CPB columns per
    // 32-byte segment
    constexpr int RL = last_radix(LOGH);
    constexpr int LOGRL = RL == 16 ? 4 : RL == 8 ? 3 : RL == 4 ? 2 : 1;
    constexpr int NSL = h / RL;
    Stages<C, FFT_EPT, true, LOGH, 1, LOGH - LOGRL, HP, NT>::run(s, tw_inv);
#pragma unroll
    for (int q = 0; q < FFT_EPT / RL; ++q) {
      const int u = tid + q * NT;
      const int cc = u & (CPB - 1), j = u >> logc, k = k0 + cc;
      const C* col = s + cc * HP;
      C v[RL];
#pragma unroll
      for (int r = 0; r < RL; ++r) v[r] = col[P::at(j) + r * (NSL + NSL / 16)];  // j < NSL, a multiple of 16
      if (NSL > 1) {
        C w[RL];
        stage_twiddles<C, RL, true>(tw_inv, j, w);
#pragma unroll
        for (int r = 1; r < RL; ++r) v[r] = cmul(v[r], w[r]);
      }
      dft_r<C, RL, true>(v);
      if (k < N) {
#pragma unroll
        for (int r = 0; r < RL; ++r) {  // j < NSL: the first RL / 2 outputs are even rows
          const int p = j + r * NSL, row = r < RL / 2 ? 2 * p : 2 * (h - 1 - p) + 1;
          half[(size_t)row * N + k] = cscale(v[r], inv_h);
        }
      }
    }
  }
}

// The column pass with the divide in registers, for column lengths h = 2^LOGH whose last radix
// RL = last_radix(LOGH) is below 16 (h = 32 .. 2048 except 256), so that a thread holds
// B = FFT_EPT / RL >= 2 butterflies of the forward transform's last stage. The same values as
// k_cols (forward DCT-II by Makhoul's reordering and one complex FFT, divide by d lambda^2 + c,
// inverse DCT), with fewer shared-memory passes:
//   - forward stages as k_cols (the first straight from global memory);
//   - the last forward stage, span NS = h / RL, into registers: butterfly j's outputs are
//     m = j + r NS, and the partner h - m of each is an output of butterfly NS - j (j = 0 and
//     NS / 2 pair within themselves). A thread takes butterflies t + q T and their partners
//     (T = NS / B threads a column), so every pair (m, h - m) the divide couples is its own;
//   - the divide on the pair: with a = 1 / D_m, b = 1 / D_(h-m) (D = d lambda^2 + c_ref) and
//     w2 = e^(-i pi m / h), V'_m = (a + b)/2 V_m + (a - b)/2 conj(w2) V_(h-m) and
//     V'_(h-m) = (a - b)/2 w2 V_m + (a + b)/2 V_(h-m): the DCT twiddle, the divide and the inverse
//     DCT twiddle of k_cols folded into one 2 x 2 map (column 0, packed with two real
//     wavenumbers, keeps k_cols's separate form);
//   - the inverse transform as the forward stages' adjoints in reverse order, the last stage's
//     adjoint still in registers, the first stage's adjoint writing to global memory.
// Shared memory is written four times a transform pair instead of six, with six block barriers
// instead of nine.
// e^(-i pi e / 8), e = 0 .. 7: the rotations between the DCT twiddles of one last-stage butterfly.
template <class C>
__device__ __forceinline__ C rot_pi(int e) {
  using T = decltype(C::x);
  const T c1 = (T)0.92387953251128675613, s1 = (T)0.38268343236508977173, h = (T)0.70710678118654752440;
  switch (e & 7) {
    case 0: return mk<C>((T)1, (T)0);
    case 1: return mk<C>(c1, -s1);
    case 2: return mk<C>(h, -h);
    case 3: return mk<C>(s1, -c1);
    case 4: return mk<C>((T)0, (T)-1);
    case 5: return mk<C>(-s1, -c1);
    case 6: return mk<C>(-h, -h);
    default: return mk<C>(-c1, -s1);
  }
}

// Columns a block of the fused pass: half of k_cols's, so that three blocks share an SM with
// up to 85 registers a thread (the pass keeps two butterflies and their twiddles in registers).
__host__ __device__ constexpr int cols_per_block_fused(int logh, int elem) {
  return cols_per_block(logh, elem) > 1 ? cols_per_block(logh, elem) / 2 : 1;
}
// Column pitch of the fused pass: the padded length rounded up to 16 / CPB (mod 16). Its first
// stage and the first stage's adjoint have a half warp touch 16 / CPB consecutive butterflies of
// each of CPB columns, slots cc pitch + j + r (mod 16) in 8-byte units, which are then 16
// distinct slots (two columns at a pitch of 4 (mod 16), k_cols's, would overlap in 4 of them).
__host__ __device__ constexpr int col_pitch_fused(int h, int cpb) {
  int l = h + (h >> 4) + 1;
  int want = cpb >= 16 ? 1 : 16 / cpb;
  return l + ((want - l % 16) % 16 + 16) % 16;
}

template <class T, int LOGH>
__global__ void __launch_bounds__(FFT_MAX_THREADS / 2, 3) k_cols_fused(int N, cplx<T>* __restrict__ half, const cplx<T>* __restrict__ tw,
                                                               const cplx<T>* __restrict__ omega, const cplx<T>* __restrict__ omega2,
                                                               const T* __restrict__ lx, const T* __restrict__ ly, T inv_dx2,
                                                               const Scalars* S, int level) {
  using C = cplx<T>;
  using P = Pad<C>;
  if (S->stop) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* s = reinterpret_cast<C*>(smem_raw);
  constexpr int h = 1 << LOGH;
  constexpr int CPB = cols_per_block_fused(LOGH, (int)sizeof(C));
  constexpr int HP = col_pitch_fused(h, CPB);
  constexpr int logc = CPB == 1 ? 0 : CPB == 2 ? 1 : CPB == 4 ? 2 : CPB == 8 ? 3 : CPB == 16 ? 4 : 5;
  constexpr int NT = CPB * h / FFT_EPT;
  constexpr int RL = last_radix(LOGH);
  constexpr int LOGRL = RL == 8 ? 3 : RL == 4 ? 2 : 1;
  constexpr int NS = h / RL;          // the last stage's span, and its butterflies a column
  constexpr int B = FFT_EPT / RL;     // last-stage butterflies a thread
  constexpr int TPC = h / FFT_EPT;    // threads a column
  static_assert(RL < 16 && LOGH >= 5 && B >= 2 && NS % 16 == 0, "the fused column pass: a last radix below 16");
  static_assert(TPC * CPB == NT, "columns: whole threads");
  // the bank's levels in one launch: level + blockIdx.y, its spectrum consecutive
  half += (size_t)blockIdx.y * h * N;
  level += blockIdx.y;
  const int k0 = blockIdx.x * CPB;
  const int tid = threadIdx.x;
  const T dref = (T)S->node_d[level], cref = (T)S->c_ref;
  // ---- forward, first stage (radix 16, span 1) straight from global memory in Makhoul's order:
  // thread tid takes butterfly j = tid / CPB of column tid % CPB, v[j + r h / 16]
  {
    const int cc = tid & (CPB - 1), j = tid >> logc, k = k0 + cc;
    C v[16];
    const int kk = k < N ? k : 0;
#pragma unroll
    for (int r = 0; r < 16; ++r) {
      const int p = j + r * (h / 16), row = r < 8 ? 2 * p : 2 * (h - 1 - p) + 1;
      v[r] = half[row * N + kk];  // h N < 2^31: 32-bit offsets
    }
    if (k >= N) {
#pragma unroll
      for (int r = 0; r < 16; ++r) v[r] = mk<C>((T)0, (T)0);
    }
    dft_r<C, 16, false>(v);
    C* col = s + cc * HP;
#pragma unroll
    for (int r = 0; r < 16; ++r) col[17 * j + r] = v[r];  // pad(16 j + r) = 17 j + r
    __syncthreads();
  }
  // ---- forward, middle stages (radix 16), spans 16 .. NS / 16
  Stages<C, FFT_EPT, false, LOGH, 16, LOGH - 4 - LOGRL, HP, NT>::run(s, tw);
  // ---- forward last stage, divide, its adjoint: in registers
  {
    const int cc = tid / TPC, t = tid & (TPC - 1), k = k0 + cc;
    C* col = s + cc * HP;
    constexpr int T2 = NS / B;  // = TPC: the thread's butterflies t + q T2 and their partners
    int jb[B];
#pragma unroll
    for (int q = 0; q < B / 2; ++q) {
      jb[q] = t + q * T2;
      jb[q + B / 2] = (t == 0 && q == 0) ? NS / 2 : NS - jb[q];
    }
    C v[B][RL];
#pragma unroll
    for (int q = 0; q < B; ++q) {
      const C* src = col + P::at(jb[q]);
#pragma unroll
      for (int r = 0; r < RL; ++r) v[q][r] = src[r * (NS + NS / 16)];
      C w[RL];
      stage_twiddles<C, RL, false>(tw, jb[q], w);  // the last stage's twiddles w_h^(r j)
#pragma unroll
      for (int r = 1; r < RL; ++r) v[q][r] = cmul(v[q][r], w[r]);
      dft_r<C, RL, false>(v[q]);
    }
    if (k < N) {
      const T lxk = lx[k];
      auto rden = [&](T lxv, T lyv) {
        T l = (lxv + lyv) * inv_dx2;
        return recip_fast(dref * (l * l) + cref);
      };
      // the pair (m, h - m) held in (vm, vn); w2 = e^(-i pi m / h), and ly[m] = 2 cos(pi m / h) - 2
      // = 2 Re(w2) - 2 (flexure.rs:1146), ly[h - m] = -ly[m] - 4
      auto pair = [&](C& vm, C& vn, C w2, int m) {
        const T ym = (T)2 * w2.x - (T)2, yn = -ym - (T)4;
        if (k == 0) {  // packed: real part wavenumber 0, imaginary part N (k_cols's form)
          const T lxn = lx[N];
          const C wm = omega[m], wn = mk<C>(-wm.y, -wm.x);
          C p = cmul(wm, vm), q = cmul(wn, vn);
          C cm = cscale(cadd(p, cmuli(q)), (T)0.5), cn = cscale(cadd(q, cmuli(p)), (T)0.5);
          cm.x *= rden(lxk, ym);
          cm.y *= rden(lxn, ym);
          cn.x *= rden(lxk, yn);
          cn.y *= rden(lxn, yn);
          vm = cmul(cconj(wm), csub(cm, cmuli(cn)));
          vn = cmul(cconj(wn), csub(cn, cmuli(cm)));
          return;
        }
        const T a = rden(lxk, ym), b = rden(lxk, yn);
        const T sv = (a + b) * (T)0.5, tv = (a - b) * (T)0.5;
        const C xm = vm, xn = vn;
        vm = cadd(cscale(xm, sv), cscale(cmul(cconj(w2), xn), tv));
        vn = cadd(cscale(cmul(w2, xm), tv), cscale(xn, sv));
      };
      // e^(-i pi m / h) for m = j + r NS: e^(-i pi j / h) e^(-i pi r / RL), one table load a butterfly
      auto w2_at = [&](C w2j, int r) { return r == 0 ? w2j : cmul(w2j, rot_pi<C>(r * (8 / RL))); };
#pragma unroll
      for (int q = 0; q < B / 2; ++q) {
        if (t == 0 && q == 0) {
          // butterfly 0: m = r NS pairs with (RL - r) NS, m = 0 and h / 2 with themselves (for
          // m = h / 2 both divisors are equal, so the pair form with vn = vm is the plain one)
          if (k == 0) {
            v[0][0].x *= rden(lxk, (T)0);
            v[0][0].y *= rden(lx[N], (T)0);
          } else {
            v[0][0] = cscale(v[0][0], rden(lxk, (T)0));
          }
          const C one = mk<C>((T)1, (T)0);
#pragma unroll
          for (int r = 1; r < RL / 2; ++r) pair(v[0][r], v[0][RL - r], w2_at(one, r), r * NS);
          {
            C self = v[0][RL / 2];
            pair(v[0][RL / 2], self, w2_at(one, RL / 2), h / 2);
          }
          // butterfly NS / 2: output r pairs with RL - 1 - r
          const C w2h = omega2[NS / 2];
#pragma unroll
          for (int r = 0; r < RL / 2; ++r) pair(v[B / 2][r], v[B / 2][RL - 1 - r], w2_at(w2h, r), NS / 2 + r * NS);
        } else {
          const C w2j = omega2[jb[q]];
#pragma unroll
          for (int r = 0; r < RL; ++r) pair(v[q][r], v[q + B / 2][RL - 1 - r], w2_at(w2j, r), jb[q] + r * NS);
        }
      }
    }
#pragma unroll
    for (int q = 0; q < B; ++q) {
      dft_r<C, RL, true>(v[q]);
      C w[RL];
      stage_twiddles<C, RL, true>(tw, jb[q], w);
      C* dst = col + P::at(jb[q]);
      dst[0] = v[q][0];
#pragma unroll
      for (int r = 1; r < RL; ++r) dst[r * (NS + NS / 16)] = cmul(v[q][r], w[r]);
    }
    __syncthreads();
  }
  // ---- inverse: the middle stages' adjoints, then the first stage's into global memory
  StagesAdj<C, FFT_EPT, LOGH, 16, LOGH - 4 - LOGRL, HP, NT>::run(s, tw);
  {
    const int cc = tid & (CPB - 1), j = tid >> logc, k = k0 + cc;
    const C* col = s + cc * HP;
    C v[16];
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = col[17 * j + r];
    dft_r<C, 16, true>(v);
    const T inv_h = (T)1 / (T)h;
    if (k < N) {
#pragma unroll
      for (int r = 0; r < 16; ++r) {
        const int p = j + r * (h / 16), row = r < 8 ? 2 * p : 2 * (h - 1 - p) + 1;
        half[row * N + k] = cscale(v[r], inv_h);
      }
    }
  }
}

// The column pass on the sphere's row metric (RowSolve::solve, flexure.rs:1012-1099): no
// transform along y; per wavenumber k the pentadiagonal d L_k^2 + c (L_k: diagonal
// (a_j lx_k - b_j - b_(j+1)) / dx^2, off the diagonal b_(j+1) / dx^2) is factored as L D L^T
// and solved, with the reference's recurrences and order of operations. The factors depend only
// on the level's (d, c) and k, so k_row_factor makes them once per solve (dd, l1, l2: h x (N + 1)
// each, row-major, wavenumber fastest) and k_row_solve does the substitutions at every
// application. One thread per wavenumber q = 0 .. N; column q of the packed half spectrum holds
// wavenumber q (both parts) for 0 < q < N, and column 0 wavenumbers 0 (real part) and N
// (imaginary part), which threads 0 and N solve part by part.
template <class T>
__global__ void __launch_bounds__(128) k_row_factor(int N, int h, const T* __restrict__ lx, const T* __restrict__ ma,
                                                    const T* __restrict__ mb, T inv_dx2, const Scalars* S, int level,
                                                    T* __restrict__ dds, T* __restrict__ l1s, T* __restrict__ l2s) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q > N) return;
  const T d = (T)S->node_d[level], c = (T)S->c_ref;
  const T lxk = lx[q];
  const size_t stride = (size_t)N + 1;
  T dd1 = 0, dd2 = 0, l1p = 0;  // dd[j-1], dd[j-2], l1[j-1]
  T t1 = 0, e1 = 0, e2 = 0;     // t(j-1), e(j-1), e(j-2)
#pragma unroll 4
  for (int j = 0; j < h; ++j) {
    const T tj = (ma[j] * lxk - mb[j] - mb[j + 1]) * inv_dx2;
    const T ej = j + 1 < h ? mb[j + 1] * inv_dx2 : (T)0;
    T p1 = 0, p2 = 0;
    if (j >= 2) p2 = d * e2 * e1 / dd2;  // m2(j-2) / dd[j-2]
    if (j >= 1) {
      T carried = j >= 2 ? p2 * dd2 * l1p : (T)0;
      p1 = (d * e1 * (t1 + tj) - carried) / dd1;  // (m1(j-1) - carried) / dd[j-1]
    }
    const T up = j > 0 ? e1 : (T)0;
    T dj = d * (tj * tj + up * up + ej * ej) + c;  // m0(j)
    if (j >= 1) dj -= p1 * p1 * dd1;
    if (j >= 2) dj -= p2 * p2 * dd2;
    dds[(size_t)j * stride + q] = dj;
    l1s[(size_t)j * stride + q] = p1;
    l2s[(size_t)j * stride + q] = p2;
    dd2 = dd1;
    dd1 = dj;
    l1p = p1;
    e2 = e1;
    e1 = ej;
    t1 = tj;
  }
}

// The substitutions: x[j] -= x[j-1] l1[j] + ... going down, x[j] /= dd[j], x[j] -= x[j+1] l1[j+1]
// + ... going up, in place on the level's spectrum. A thread's recurrence waits on nothing but
// its own arithmetic: it loads RB rows (spectrum and factors) at a time before walking them.
template <class T>
__global__ void __launch_bounds__(128) k_row_solve(int N, int h, cplx<T>* __restrict__ half, const T* __restrict__ dds,
                                                   const T* __restrict__ l1s, const T* __restrict__ l2s, const Scalars* S) {
  using C = cplx<T>;
  constexpr int RB = 8;
  if (S->stop) return;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q > N) return;
  const int col = q == N ? 0 : q;
  const bool re = q != N, im = q != 0;  // the parts this thread owns
  const size_t stride = (size_t)N + 1;
  auto store = [&](int j, C v) {
    // column 0's parts belong to two threads: each stores only its own
    if (re && im) {
      half[(size_t)j * N + col] = v;
    } else if (re) {
      half[(size_t)j * N + col].x = v.x;
    } else {
      half[(size_t)j * N + col].y = v.y;
    }
  };
  C x1 = mk<C>((T)0, (T)0), x2 = x1;  // x'[j-1], x'[j-2] (before the division)
  for (int j0 = 0; j0 < h; j0 += RB) {
    C v[RB];
    T a1[RB], a2[RB], dv[RB];
#pragma unroll
    for (int u = 0; u < RB; ++u) {
      const int j = min(j0 + u, h - 1);
      v[u] = half[(size_t)j * N + col];
      a1[u] = l1s[(size_t)j * stride + q];
      a2[u] = l2s[(size_t)j * stride + q];
      dv[u] = dds[(size_t)j * stride + q];
    }
#pragma unroll
    for (int u = 0; u < RB; ++u) {
      const int j = j0 + u;
      if (j >= h) break;
      C x = v[u];
      if (j >= 1) {
        x.x -= x1.x * a1[u];
        x.y -= x1.y * a1[u];
      }
      if (j >= 2) {
        x.x -= x2.x * a2[u];
        x.y -= x2.y * a2[u];
      }
      x2 = x1;
      x1 = x;
      store(j, mk<C>(x.x / dv[u], x.y / dv[u]));
    }
  }
  // the walk up: x[j] -= x[j+1] l1[j+1]; x[j] -= x[j+2] l2[j+2]
  C y1 = mk<C>((T)0, (T)0), y2 = y1;  // x[j+1], x[j+2]
  T l1n = 0, l2n = 0, l2nn = 0;       // l1[j+1], l2[j+1], l2[j+2]
  for (int j0 = h - 1; j0 >= 0; j0 -= RB) {
    C v[RB];
    T a1[RB], a2[RB];
#pragma unroll
    for (int u = 0; u < RB; ++u) {
      const int j = max(j0 - u, 0);
      v[u] = half[(size_t)j * N + col];
      a1[u] = l1s[(size_t)j * stride + q];
      a2[u] = l2s[(size_t)j * stride + q];
    }
#pragma unroll
    for (int u = 0; u < RB; ++u) {
      const int j = j0 - u;
      if (j < 0) break;
      C x = v[u];
      if (j + 1 < h) {
        x.x -= y1.x * l1n;
        x.y -= y1.y * l1n;
      }
      if (j + 2 < h) {
        x.x -= y2.x * l2nn;
        x.y -= y2.y * l2nn;
      }
      store(j, x);
      y2 = y1;
      y1 = x;
      l2nn = l2n;
      l1n = a1[u];
      l2n = a2[u];
    }
  }
}

// The row solve in chunks: the down and up recurrences of k_row_solve are linear in their two
// carried values, so each column is cut into chunks of ROW_CHUNK rows that run in parallel from a
// zero carry, a short pass per column composes the chunks' 2 x 2 carry transfers (made once per
// solve, from the factors alone), and a second parallel pass reruns each chunk from its true
// carry. The same sums as the sequential solve, differently rounded; (chunk, wavenumber)
// threads, wavenumber fastest, so every row step reads contiguous words.
constexpr int ROW_CHUNK = 64;

// one row of the down recurrence: x = v - s1 l1 - s2 l2, then (s2, s1) <- (s1, x)
template <class C, class T>
__device__ __forceinline__ void row_down(C v, T a1, T a2, C& s1, C& s2) {
  C x = v;
  x.x -= s1.x * a1;
  x.y -= s1.y * a1;
  x.x -= s2.x * a2;
  x.y -= s2.y * a2;
  s2 = s1;
  s1 = x;
}
// the up recurrence's coefficients at row j: l1[j + 1] and l2[j + 2] (0 past the last row)
template <class T>
__device__ __forceinline__ void up_coeffs(const T* __restrict__ l1s, const T* __restrict__ l2s, int j, int h, size_t q,
                                          size_t stride, T& a1, T& a2) {
  a1 = j + 1 < h ? l1s[(size_t)(j + 1) * stride + q] : (T)0;
  a2 = j + 2 < h ? l2s[(size_t)(j + 2) * stride + q] : (T)0;
}

// Per (chunk, wavenumber): the carry transfers of the down recurrence (tf) and of the up one
// (tb), each the state after the chunk from the unit carries (1, 0) and (0, 1): 4 values apiece,
// laid out [4][chunks][N + 1].
template <class T>
__global__ void __launch_bounds__(128) k_row_transfer(int N, int h, int P, const T* __restrict__ l1s,
                                                      const T* __restrict__ l2s, T* __restrict__ tf, T* __restrict__ tb) {
  const size_t stride = (size_t)N + 1, plane = (size_t)P * stride;
  const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t >= plane) return;
  const size_t q = t % stride;
  const int c = (int)(t / stride), a = c * ROW_CHUNK, b = min(h, a + ROW_CHUNK);
  using C = cplx<T>;
  // the two unit carries as one complex pair: .x from (1, 0), .y from (0, 1)
  C s1 = mk<C>((T)1, (T)0), s2 = mk<C>((T)0, (T)1);
  for (int j = a; j < b; ++j)
    row_down(mk<C>((T)0, (T)0), l1s[(size_t)j * stride + q], l2s[(size_t)j * stride + q], s1, s2);
  tf[0 * plane + t] = s1.x;
  tf[1 * plane + t] = s2.x;
  tf[2 * plane + t] = s1.y;
  tf[3 * plane + t] = s2.y;
  C t1 = mk<C>((T)1, (T)0), t2 = mk<C>((T)0, (T)1);
  for (int j = b - 1; j >= a; --j) {
    T a1, a2;
    up_coeffs(l1s, l2s, j, h, q, stride, a1, a2);
    row_down(mk<C>((T)0, (T)0), a1, a2, t1, t2);
  }
  tb[0 * plane + t] = t1.x;
  tb[1 * plane + t] = t2.x;
  tb[2 * plane + t] = t1.y;
  tb[3 * plane + t] = t2.y;
}

// The chunk's down recurrence from a zero carry: its end state (s1, s2) into part[2][chunks][N+1]
template <class T>
__global__ void __launch_bounds__(128) k_row_down_part(int N, int h, int P, const cplx<T>* __restrict__ half,
                                                       const T* __restrict__ l1s, const T* __restrict__ l2s,
                                                       cplx<T>* __restrict__ part, const Scalars* S) {
  using C = cplx<T>;
  if (S->stop) return;
  const size_t stride = (size_t)N + 1, plane = (size_t)P * stride;
  const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t >= plane) return;
  const size_t q = t % stride;
  const int col = q == (size_t)N ? 0 : (int)q;
  const int c = (int)(t / stride), a = c * ROW_CHUNK, b = min(h, a + ROW_CHUNK);
  C s1 = mk<C>((T)0, (T)0), s2 = s1;
#pragma unroll 4
  for (int j = a; j < b; ++j) row_down(half[(size_t)j * N + col], l1s[(size_t)j * stride + q], l2s[(size_t)j * stride + q], s1, s2);
  part[t] = s1;
  part[plane + t] = s2;
}

// Per wavenumber, the chunks in order (down: first to last; up: last to first): each chunk's
// true carry-in (carry[2][chunks][N+1]) from the previous one's carry, transfer and zero-carry
// end state.
template <class T>
__global__ void __launch_bounds__(128) k_row_carry(int N, int P, bool up, const T* __restrict__ tr,
                                                   const cplx<T>* __restrict__ part, cplx<T>* __restrict__ carry,
                                                   const Scalars* S) {
  using C = cplx<T>;
  if (S->stop) return;
  const size_t stride = (size_t)N + 1, plane = (size_t)P * stride;
  const size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (q >= stride) return;
  C s1 = mk<C>((T)0, (T)0), s2 = s1;
  for (int i = 0; i < P; ++i) {
    const int c = up ? P - 1 - i : i;
    const size_t t = (size_t)c * stride + q;
    carry[t] = s1;
    carry[plane + t] = s2;
    const T a1 = tr[0 * plane + t], a2 = tr[1 * plane + t], b1 = tr[2 * plane + t], b2 = tr[3 * plane + t];
    const C p1 = part[t], p2 = part[plane + t];
    const C n1 = mk<C>(p1.x + a1 * s1.x + b1 * s2.x, p1.y + a1 * s1.y + b1 * s2.y);
    const C n2 = mk<C>(p2.x + a2 * s1.x + b2 * s2.x, p2.y + a2 * s1.y + b2 * s2.y);
    s1 = n1;
    s2 = n2;
  }
}

// The chunk's down recurrence from its true carry, y = x' / dd into the spectrum; then the up
// recurrence over the chunk from a zero carry, its end state (z[a], z[a+1]) into part
template <class T>
__global__ void __launch_bounds__(128) k_row_down_final(int N, int h, int P, cplx<T>* __restrict__ half,
                                                        const T* __restrict__ dds, const T* __restrict__ l1s,
                                                        const T* __restrict__ l2s, const cplx<T>* __restrict__ carry,
                                                        cplx<T>* __restrict__ part, const Scalars* S) {
  using C = cplx<T>;
  if (S->stop) return;
  const size_t stride = (size_t)N + 1, plane = (size_t)P * stride;
  const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t >= plane) return;
  const size_t q = t % stride;
  const int col = q == (size_t)N ? 0 : (int)q;
  const bool re = q != (size_t)N, im = q != 0;  // column 0's parts belong to two threads
  const int c = (int)(t / stride), a = c * ROW_CHUNK, b = min(h, a + ROW_CHUNK);
  C s1 = carry[t], s2 = carry[plane + t];
#pragma unroll 4
  for (int j = a; j < b; ++j) {
    row_down(half[(size_t)j * N + col], l1s[(size_t)j * stride + q], l2s[(size_t)j * stride + q], s1, s2);
    const T dv = dds[(size_t)j * stride + q];
    C* o = half + (size_t)j * N + col;
    if (re && im) {
      *o = mk<C>(s1.x / dv, s1.y / dv);
    } else if (re) {
      o->x = s1.x / dv;
    } else {
      o->y = s1.y / dv;
    }
  }
  C t1 = mk<C>((T)0, (T)0), t2 = t1;
  for (int j = b - 1; j >= a; --j) {
    T a1, a2;
    up_coeffs(l1s, l2s, j, h, q, stride, a1, a2);
    row_down(half[(size_t)j * N + col], a1, a2, t1, t2);
  }
  part[t] = t1;
  part[plane + t] = t2;
}

// The chunk's up recurrence from its true carry, z into the spectrum
template <class T>
__global__ void __launch_bounds__(128) k_row_up_final(int N, int h, int P, cplx<T>* __restrict__ half,
                                                      const T* __restrict__ l1s, const T* __restrict__ l2s,
                                                      const cplx<T>* __restrict__ carry, const Scalars* S) {
  using C = cplx<T>;
  if (S->stop) return;
  const size_t stride = (size_t)N + 1, plane = (size_t)P * stride;
  const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t >= plane) return;
  const size_t q = t % stride;
  const int col = q == (size_t)N ? 0 : (int)q;
  const bool re = q != (size_t)N, im = q != 0;
  const int c = (int)(t / stride), a = c * ROW_CHUNK, b = min(h, a + ROW_CHUNK);
  C t1 = carry[t], t2 = carry[plane + t];
#pragma unroll 4
  for (int j = b - 1; j >= a; --j) {
    T a1, a2;
    up_coeffs(l1s, l2s, j, h, q, stride, a1, a2);
    row_down(half[(size_t)j * N + col], a1, a2, t1, t2);
    C* o = half + (size_t)j * N + col;
    if (re && im) {
      *o = t1;
    } else if (re) {
      o->x = t1.x;
    } else {
      o->y = t1.y;
    }
  }
}

// Inverse rows: Z[k] = E[k] + i O[k] with E = (X[k] + conj X[N-k]) / 2,
// O = (X[k] - conj X[N-k]) conj(W^k) / 2; x = IFFT_N(Z) / N de-interleaved.
template <class T, int MODE, int LOGN>
__global__ void __launch_bounds__(FFT_MAX_THREADS, sizeof(T) == 4 ? 2 : 1) k_rows_inv(int w, int h, const cplx<T>* __restrict__ half, T* __restrict__ out,
                                                             const T* __restrict__ wt, const T* __restrict__ r,
                                                             const cplx<T>* __restrict__ tw, const cplx<T>* __restrict__ post,
                                                             double* partials, Scalars* S) {
  using C = cplx<T>;
  using P = Pad<C>;
  if (S->stop) {
    if (MODE == INV_STORE_DOT && blockIdx.x == 0 && threadIdx.x == 0) set_cond(S, 0);
    return;
  }
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* s = reinterpret_cast<C*>(smem_raw);
  constexpr int N = 1 << LOGN, NP = P::len(N);
  constexpr int logN = LOGN;
  constexpr int RB = rows_per_block(LOGN);
  const int row0 = blockIdx.x * RB;
  const int tid = threadIdx.x;
  constexpr int half_n = N / 2 + 1;
  constexpr int NT = RB * N / FFT_EPT;  // the block's threads (fft_geometry)
  constexpr int IB = FFT_BATCH / 2;     // pairs (X[k], X[N-k]) loaded per batch
  constexpr int LEVELS = MODE == INV_BANK ? 3 : 1;
  const T inv_n = (T)1 / (T)N;
  Acc<2> acc;
  acc.v[0] = 0.0;
  acc.v[1] = 0.0;
  const cplx<T>* const half0 = half;
  const T* const wt0 = wt;
#pragma unroll 1
  for (int lv = 0; lv < LEVELS; ++lv) {
  half = half0 + (size_t)lv * h * N;
  wt = wt0 + (size_t)lv * (2 * N) * h;
  if (lv > 0) __syncthreads();  // the previous level's last reads of s are done
#pragma unroll 1
  for (int base = tid; base < RB * half_n; base += IB * NT) {
    C xkb[IB], xnb[IB];
#pragma unroll
    for (int u = 0; u < IB; ++u) {
      int idx = base + u * NT;
      int rb = idx / half_n, kk = idx - rb * half_n;
      int j = row0 + rb;
      xkb[u] = xnb[u] = mk<C>((T)0, (T)0);
      if (idx < RB * half_n && j < h) {
        const C* in = half + (size_t)j * N;
        xkb[u] = in[kk];
        if (kk > 0) xnb[u] = in[N - kk];
      }
    }
#pragma unroll
    for (int u = 0; u < IB; ++u) {
    int idx = base + u * NT;
    if (idx >= RB * half_n) break;
    int rb = idx / half_n, kk = idx - rb * half_n;
    int j = row0 + rb;
    C* row = s + rb * NP;
    if (j >= h) {
      row[P::at(kk)] = mk<C>((T)0, (T)0);
      if (kk > 0 && kk < N) row[P::at(N - kk)] = mk<C>((T)0, (T)0);
      continue;
    }
    if (kk == 0) {
      C p = xkb[u];  // (X[0], X[N])
      row[0] = mk<C>((p.x + p.y) * (T)0.5, (p.x - p.y) * (T)0.5);
      continue;
    }
    C xk = xkb[u], xn = xnb[u];
    C E = mk<C>((xk.x + xn.x) * (T)0.5, (xk.y - xn.y) * (T)0.5);
    C D = mk<C>((xk.x - xn.x) * (T)0.5, (xk.y + xn.y) * (T)0.5);
    C O = cmul(D, cconj(post[kk]));
    row[P::at(kk)] = cadd(E, cmuli(O));
    if (kk != N - kk) {
      // index N - kk: E' = conj E, D' = -conj D, conj(W^(N-k)) = -W^k  =>  O' = conj(D) W^k
      C O2 = cmul(cconj(D), post[kk]);
      row[P::at(N - kk)] = cadd(cconj(E), cmuli(O2));
    }
    }
  }
  __syncthreads();
  // z = x[2 nn] + i x[2 nn + 1] of row j, scaled: the mode's output (the bank's first level
  // stores, the others add to what the same thread stored)
  auto emit = [&](int j, int nn, C z) {
    size_t k = (size_t)j * (2 * N) + 2 * nn;
    C* o = reinterpret_cast<C*>(out + k);
    if (MODE == INV_STORE) {
      *o = z;
    } else if (MODE == INV_STORE_W || (MODE == INV_BANK && lv == 0)) {
      C ww = *reinterpret_cast<const C*>(wt + k);
      *o = mk<C>(z.x * ww.x, z.y * ww.y);
    } else if (MODE == INV_BANK) {
      C ww = *reinterpret_cast<const C*>(wt + k);
      C prev = *o;
      *o = mk<C>(prev.x + z.x * ww.x, prev.y + z.y * ww.y);
    } else {  // INV_STORE_DOT
      *o = z;
      C rr = *reinterpret_cast<const C*>(r + k);
      acc.v[0] += (double)rr.x * (double)z.x + (double)rr.y * (double)z.y;
      acc.v[1] = fmax(acc.v[1], fmax(fabs((double)z.x), fabs((double)z.y)));
    }
  };
  if constexpr (RB == 1 && LOGN >= 4) {
    // one row per block: all stages but the last through shared memory; the last (radix RL,
    // span N / RL, twiddles w^(r j)) hands each output to the mode's epilogue
    constexpr int RL = last_radix(LOGN);
    constexpr int LOGRL = RL == 16 ? 4 : RL == 8 ? 3 : RL == 4 ? 2 : 1;
    constexpr int NSL = N / RL;
    Stages<C, FFT_EPT, true, LOGN, 1, LOGN - LOGRL, 0, NT>::run(s, tw);
#pragma unroll
    for (int q = 0; q < FFT_EPT / RL; ++q) {
      const int j = tid + q * NT;
      C z[RL];
#pragma unroll
      for (int rr = 0; rr < RL; ++rr) z[rr] = s[P::at(j) + rr * (NSL + NSL / 16)];  // j < NSL, a multiple of 16
      if (NSL > 1) {
        C wv[RL];
        stage_twiddles<C, RL, true>(tw, j, wv);
#pragma unroll
        for (int rr = 1; rr < RL; ++rr) z[rr] = cmul(z[rr], wv[rr]);
      }
      dft_r<C, RL, true>(z);
      if (row0 < h) {
#pragma unroll
        for (int rr = 0; rr < RL; ++rr) emit(row0, j + rr * NSL, cscale(z[rr], inv_n));
      }
    }
  } else {
    smem_fft<C, FFT_EPT, true, LOGN, NT>(s, tw);
#pragma unroll 4
    for (int idx = tid; idx < RB * N; idx += NT) {
      int rb = idx >> logN, nn = idx & (N - 1);
      int j = row0 + rb;
      if (j >= h) continue;
      emit(j, nn, cscale(s[rb * NP + P::at(nn)], inv_n));
    }
  }
  }  // levels
  if (MODE == INV_STORE_DOT) {
    const int kind[2] = {0, 1};
    if (reduce_partials<2>(acc, kind, partials, &S->ticket[SITE_PRECOND], gridDim.x) && tid == 0) finish_precond(S, acc.v[0], acc.v[1]);
  }
}

// k_rows_inv's INV_BANK (one row a block) as a persistent kernel fed by bulk copies: block b
// takes rows b, b + gridDim.x, ..., each row's three levels in turn. A level's half row (N complex
// values) and weight row (2 N) land in shared memory by two 1-D bulk copies on two mbarriers; the
// next level's half row is copied as soon as this level's split has read it, its weight row as
// soon as this level's sums have read theirs, so both copies overlap the transform. The three
// levels' weighted outputs are summed in registers and stored once a row. Arithmetic and order of
// operations are k_rows_inv's. Waits are bounded: one that runs out flags a fault, stops the
// solve and waits (bounded again) for the copies in flight before the block leaves.
template <class T>
__host__ __device__ constexpr size_t rows_bank_smem(int logn) {
  return ((size_t)1 << logn) * 2 * sizeof(T) * 2 + (size_t)Pad<cplx<T>>::len(1 << logn) * 2 * sizeof(T);
}
template <class T, int LOGN>
__global__ void __launch_bounds__((1 << LOGN) / FFT_EPT, (1 << LOGN) / FFT_EPT <= 128 && sizeof(T) == 4 ? 4 : 2)
    k_rows_inv_bank(int h, const cplx<T>* __restrict__ half, T* __restrict__ out, const T* __restrict__ wt,
                    const cplx<T>* __restrict__ tw, const cplx<T>* __restrict__ post, Scalars* S) {
  using C = cplx<T>;
  using P = Pad<C>;
  if (S->stop) return;
  constexpr int N = 1 << LOGN;
  constexpr int NT = N / FFT_EPT;
  constexpr int RL = last_radix(LOGN);
  constexpr int LOGRL = RL == 16 ? 4 : RL == 8 ? 3 : RL == 4 ? 2 : 1;
  constexpr int NSL = N / RL;
  constexpr int Q = FFT_EPT / RL;
  constexpr uint32_t XB = N * sizeof(C), WB = 2 * N * sizeof(T);
  static_assert(LOGN >= 4 && NSL % 16 == 0, "one row a block");
  extern __shared__ __align__(128) unsigned char rb_smem[];
  C* xs = reinterpret_cast<C*>(rb_smem);             // the level's half row, as copied
  const C* ws = reinterpret_cast<const C*>(rb_smem + XB);  // its weight row, as pairs
  C* s = reinterpret_cast<C*>(rb_smem + XB + WB);    // the transform
  __shared__ __align__(8) uint64_t bar[2];           // 0: half rows, 1: weight rows
  __shared__ int s_fail;
  const int tid = threadIdx.x;
  const int b0 = blockIdx.x, G = gridDim.x;
  const int items = b0 < h ? 3 * ((h - 1 - b0) / G + 1) : 0;  // (row, level) pairs, level fastest
  auto src_off = [&](int i) { return (size_t)(i % 3) * h + (size_t)(b0 + (i / 3) * G); };  // level-major row index
  auto issue_x = [&](int i) {
    mbar_expect_tx(smem_u32(&bar[0]), XB);
    bulk_load_1d(smem_u32(xs), half + src_off(i) * N, XB, smem_u32(&bar[0]));
  };
  auto issue_w = [&](int i) {
    mbar_expect_tx(smem_u32(&bar[1]), WB);
    bulk_load_1d(smem_u32(rb_smem + XB), wt + src_off(i) * (2 * N), WB, smem_u32(&bar[1]));
  };
  if (tid == 0) {
    mbar_init(smem_u32(&bar[0]), 1);
    mbar_init(smem_u32(&bar[1]), 1);
    mbar_fence_init();
    s_fail = 0;
    if (items > 0) {
      issue_x(0);
      issue_w(0);
    }
  }
  __syncthreads();
  const int polls = S->wait_give_up ? 0 : 1 << 24;
  // a wait that ran out: the copies in flight (x_par / w_par: their phases, -1 for none) land
  // before the block leaves
  auto fail = [&](int x_par, int w_par) {
    if (tid == 0) {
      S->fault = 1;
      S->stop = STOP_NONFINITE;
      set_cond(S, 0);
      if (x_par >= 0) mbar_wait_bounded(smem_u32(&bar[0]), (uint32_t)x_par);
      if (w_par >= 0) mbar_wait_bounded(smem_u32(&bar[1]), (uint32_t)w_par);
    }
  };
  const T inv_n = (T)1 / (T)N;
  C acc[Q][RL];
#pragma unroll 1
  for (int i = 0; i < items; ++i) {
    const int lv = i % 3;
    const uint32_t par = (uint32_t)(i & 1);
    if (tid == 0 && !mbar_wait_bounded(smem_u32(&bar[0]), par, polls)) s_fail = 1;
    __syncthreads();
    if (s_fail) {
      fail((int)par, (int)par);
      return;
    }
    // the split of k_rows_inv: Z[k] = E[k] + i O[k] from the copied half row
#pragma unroll 2
    for (int kk = tid; kk < N / 2 + 1; kk += NT) {
      if (kk == 0) {
        C p = xs[0];  // (X[0], X[N])
        s[0] = mk<C>((p.x + p.y) * (T)0.5, (p.x - p.y) * (T)0.5);
        continue;
      }
      C xk = xs[kk], xn = xs[N - kk];
      C E = mk<C>((xk.x + xn.x) * (T)0.5, (xk.y - xn.y) * (T)0.5);
      C D = mk<C>((xk.x - xn.x) * (T)0.5, (xk.y + xn.y) * (T)0.5);
      C pk = post[kk];
      C O = cmul(D, cconj(pk));
      s[P::at(kk)] = cadd(E, cmuli(O));
      if (kk != N - kk) {
        C O2 = cmul(cconj(D), pk);
        s[P::at(N - kk)] = cadd(cconj(E), cmuli(O2));
      }
    }
    fence_proxy_async_smem();  // this thread's reads of xs before the next copy into it
    __syncthreads();
    if (tid == 0 && i + 1 < items) issue_x(i + 1);
    Stages<C, FFT_EPT, true, LOGN, 1, LOGN - LOGRL, 0, NT>::run(s, tw);
    if (tid == 0 && !mbar_wait_bounded(smem_u32(&bar[1]), par, polls)) s_fail = 1;
    __syncthreads();
    if (s_fail) {
      fail(i + 1 < items ? (int)(par ^ 1u) : -1, (int)par);
      return;
    }
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const int j = tid + q * NT;
      C z[RL];
#pragma unroll
      for (int rr = 0; rr < RL; ++rr) z[rr] = s[P::at(j) + rr * (NSL + NSL / 16)];
      C wv[RL];
      stage_twiddles<C, RL, true>(tw, j, wv);
#pragma unroll
      for (int rr = 1; rr < RL; ++rr) z[rr] = cmul(z[rr], wv[rr]);
      dft_r<C, RL, true>(z);
#pragma unroll
      for (int rr = 0; rr < RL; ++rr) {
        const C zz = cscale(z[rr], inv_n), ww = ws[j + rr * NSL];
        if (lv == 0) {
          acc[q][rr] = mk<C>(zz.x * ww.x, zz.y * ww.y);
        } else {
          acc[q][rr] = mk<C>(acc[q][rr].x + zz.x * ww.x, acc[q][rr].y + zz.y * ww.y);
        }
      }
    }
    if (lv == 2) {
      C* o = reinterpret_cast<C*>(out + (size_t)(b0 + (i / 3) * G) * (2 * N));
#pragma unroll
      for (int q = 0; q < Q; ++q)
#pragma unroll
        for (int rr = 0; rr < RL; ++rr) o[tid + q * NT + rr * NSL] = acc[q][rr];
    }
    fence_proxy_async_smem();  // the reads of ws (and s) before the next copy and split
    __syncthreads();
    if (tid == 0 && i + 1 < items) issue_w(i + 1);
  }
}

#include "rows_any.cuh"

// ---------------------------------------------------------------------------------------------
// Small control kernels.

// Before the loop: give the scalars the graph's conditional handle and run the body only when
// nothing has stopped the solve yet.
__global__ void k_arm(Scalars* S, unsigned long long handle, unsigned long long handle_if) {
  S->cond = handle;
  S->cond_if = handle_if;
  S->body_runs = 0;
  cudaGraphSetConditional((cudaGraphConditionalHandle)handle, S->stop == 0 ? 1u : 0u);
}
__global__ void k_disarm(Scalars* S) {
  S->cond = 0ull;
  S->cond_if = 0ull;
}

// A fresh solve state (keeps the problem fields, the bank and the handle slot cleared).
__global__ void k_reset(Scalars* S) {
  S->fault = 0;
  S->it = 0;
  S->stop = 0;
  S->started = 0;
  S->body_runs = 0;
  S->err = 0.0;
  S->cond = 0ull;
  for (int k = 0; k < 8; ++k) S->ticket[k] = 0u;
}

// bb = dot_out (from a k_dot of b with itself)
__global__ void k_take_bb(Scalars* S) { S->bb = S->dot_out; }
__global__ void k_rr_is_bb(Scalars* S) { S->rr = S->bb; }

// The first guess's fate: keep x0 (r = b - A x0 already formed, S->rr) when it beats x = 0,
// i.e. ||b - A x0|| < ||b||; otherwise x = 0 and r = b.
template <class T>
__global__ void k_warm_decide(size_t n, T* __restrict__ x, T* __restrict__ r, const T* __restrict__ b, const Scalars* S) {
  bool keep = S->rr < S->bb;
  if (keep) return;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    x[k] = (T)0;
    r[k] = b[k];
  }
}
struct WarmInfo {
  int accepted;
  double rel;
};
__global__ void k_warm_record(Scalars* S, WarmInfo* info) {
  info->accepted = S->rr < S->bb ? 1 : 0;
  info->rel = S->bb > 0 ? sqrt(S->rr / S->bb) : 0.0;
  if (!info->accepted) S->rr = S->bb;
}

// The loop's entry checks (flexure.rs:1691-1704 and the relative-residual rule).
__global__ void k_begin(Scalars* S) {
  S->it = 0;
  S->stop = 0;
  S->started = 0;
  S->body_runs = 0;
  S->err = 0.0;
  if (S->fault) {
    S->stop = STOP_NONFINITE;  // a wait ran out before the loop: it does not start
  } else if (!isfinite(S->bb) || !isfinite(S->rr)) {
    S->stop = STOP_NONFINITE;
  } else if (!(S->bb > 0.0)) {
    S->stop = STOP_CONVERGED;  // b = 0: x = 0 is exact
  } else if (S->rule != DT_STOP_MAX_Z) {
    double lim = S->rule == DT_STOP_REL_RESIDUAL ? S->tol * S->tol * S->bb : S->tol * S->tol * (double)S->n;
    if (S->rr <= lim) S->stop = STOP_CONVERGED;
  }
}

// After the first preconditioning under the reference's rule: when max|z| < tol already, the
// preconditioner's answer is the correction (flexure.rs:1699-1702).
template <class T>
__global__ void k_initial_result(size_t n, T* __restrict__ x, const T* __restrict__ z, const Scalars* S) {
  if (!(S->rule == DT_STOP_MAX_Z && S->stop == STOP_CONVERGED && S->started && S->it == 0)) return;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) x[k] += z[k];
}

// The first preconditioner application when it is already known: the kept first guess's M^-1 r0
// (or the zero guess's M^-1 b), computed to choose between them, scaled as r was (z = s z). r.z and
// max|z| go where the application's final pass puts them.
__global__ void k_scale_given_z(size_t n, float* __restrict__ z, const float* __restrict__ r, const double* scale,
                                double* partials, Scalars* S) {
  if (S->stop) return;
  const float sc = (float)*scale;
  Acc<2> acc;
  acc.v[0] = 0.0;
  acc.v[1] = 0.0;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    const float zz = z[k] * sc;
    z[k] = zz;
    acc.v[0] += (double)r[k] * (double)zz;
    acc.v[1] = fmax(acc.v[1], fabs((double)zz));
  }
  const int kind[2] = {0, 1};
  if (reduce_partials<2>(acc, kind, partials, &S->ticket[SITE_PRECOND], gridDim.x) && threadIdx.x == 0)
    finish_precond(S, acc.v[0], acc.v[1]);
}

// The zero guess won: its M^-1 b (kept in `zb`) is the first preconditioned residual
__global__ void k_warm_pick_z(size_t n, float* __restrict__ z, const float* __restrict__ zb, const double* rz) {
  if (rz[1] < rz[0]) return;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) z[k] = zb[k];
}

// ---------------------------------------------------------------------------------------------
// Host side.

static thread_local char g_err[1024] = "";
void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
}
const char* last_error() { return g_err; }

// Kernel launches of the calling thread: eager ones, and those recorded into a graph body while
// capturing (a body's kernels run once per loop pass).
static thread_local long long g_launches = 0, g_captured = 0;
static thread_local bool g_capturing = false;
static inline void counted() {
  if (g_capturing)
    ++g_captured;
  else
    ++g_launches;
}
void count_launch() { counted(); }
long long launches_now() { return g_launches; }
void add_launches(long long k) { g_launches += k; }
void begin_capture_count() {
  g_capturing = true;
  g_captured = 0;
}
long long end_capture_count() {
  g_capturing = false;
  return g_captured;
}

template <class T>
struct Tables {
  cplx<T>* tw_row = nullptr;  // N = w/2 entries e^(-2 pi i t / N)
  cplx<T>* post = nullptr;    // N entries e^(-2 pi i k / w)
  cplx<T>* tw_col = nullptr;  // h entries e^(-2 pi i t / h)
  cplx<T>* omega = nullptr;   // h entries e^(-i pi m / 2h)
  cplx<T>* omega2 = nullptr;  // h entries e^(-i pi m / h)
  T* lx = nullptr;            // N + 1 entries 2 cos(2 pi k / w) - 2
  T* ly = nullptr;            // h entries 2 cos(pi m / h) - 2
};

template <class T>
struct Lane {
  T *d = nullptr, *c = nullptr, *x = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *ap = nullptr;
  T *J = nullptr, *wt[3] = {nullptr, nullptr, nullptr}, *left = nullptr, *part = nullptr;
  cplx<T>* half = nullptr;
  // the bank's levels 1 and 2 transform beside level 0, into their own spectra: the three
  // spectra are consecutive (half + k h N), as are the three weights (wt[k] = wt[0] + k n)
  cplx<T>* half_side[2] = {nullptr, nullptr};
  int bank_blocks = 0;  // k_rows_inv_bank's persistent grid (0: not yet known)
  // the row metric's L D L^T factors per bank level: dd, l1, l2 (h x (N + 1) each); when the
  // rows make more than one chunk, per level the chunks' carry transfers (8 x chunks x (N + 1))
  // and the chunk states and carries (4 complex x chunks x (N + 1))
  T* row_factors = nullptr;
  T* row_transfer = nullptr;
  cplx<T>* row_state = nullptr;
  // widths whose half is not a power of two (rows_any.cuh): per bank level two buffers of
  // pairs x L complex values, the passes' twiddles (L), and for Bluestein the chirp (w) and the
  // chirp's transform (L)
  cplx<T>* any_buf = nullptr;
  cplx<T>* any_tw = nullptr;
  cplx<T>* any_chirp = nullptr;
  cplx<T>* any_bhat = nullptr;
  Tables<T> tab;
  Scalars* S = nullptr;
  cudaGraph_t graph[4] = {};       // [(levels == 3) + 2 * reliable]
  cudaGraphExec_t exec[4] = {};
  long long body_kernels[4] = {};  // kernels in one pass of each loop body
};

static const long double PI_L = 3.14159265358979323846264338327950288L;

}  // namespace dt

struct dt_flex {
  int w = 0, h = 0, N = 0;  // N = ceil(w / 2): complex values a row of the packed half spectrum
  bool any = false;         // the transform along x by rows_any.cuh (w / 2 not a power of two)
  dt::AnyPlan plan;
  double dx = 0;
  size_t n = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  dt::Lane<double> L64;
  dt::Lane<float> L32;
  double* b64 = nullptr;
  double* partials = nullptr;
  double* scale = nullptr;  // mixed: the residual scale of the current refinement
  dt::WarmInfo* warm = nullptr;
  unsigned char* flush = nullptr;  // benchmark support: an L2-sized scratch buffer, allocated on first use
  // learned warm start: the model, its cell size, and the coarse input/output buffers
  dt_unet* unet = nullptr;
  int unet_f = 0;                  // fine cells per model cell along each axis
  float *unet_x = nullptr, *unet_y = nullptr;
  double* unet_sums = nullptr;     // sum of b_coarse^2 and of c
  double* rzpair = nullptr;        // warm start: b.M^-1 b and r0.M^-1 r0
  std::vector<void*> allocs;
  size_t nalloc = 0;  // device allocations made (the DT_FAIL_ALLOC_AT test hook counts them)
  // test support: DT_STENCIL_WAIT_GIVE_UP=1 at create makes the TMA stencil's tile waits give up
  // without testing their barrier, so the solve takes the path of a wait that ran out
  int wait_give_up = 0;
  // the column pass with its divide in registers (k_cols_fused) where the length allows;
  // DT_COLS_FUSED=0 at create keeps k_cols everywhere (the same values, for comparison)
  bool cols_fused = true;
  // the bank's inverse row pass as the persistent, bulk-copy-fed k_rows_inv_bank where the row
  // length allows; DT_ROWS_BANK=0 at create keeps k_rows_inv (the same values, for comparison)
  bool rows_bank = true;
  // the bank's three forward row passes in one launch and its three column passes in another
  // (blockIdx.y the level) where the transforms are the power-of-two kernels; DT_BANK_ONE_LAUNCH=0
  // at create runs each level's two passes as a branch of its own (the same values, for comparison)
  bool bank_one_launch = true;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int sms = 148;
  // the TMA stencil: on when the raster's rows are whole tiles; its tensor maps, one per buffer
  // and box shape, made on first use
  bool tma = false;
  // the sphere's row metric (RowMetric): a (h values) and b (h + 1) in both precisions; for the
  // block metric with a height that is not a power of two, the block metric's own couplings
  // (a = 1, b = 1 inside, 0 at the raster's edges), for the row solve only
  bool metric = false;     // the operator and the Jacobi weights on the row metric
  bool row_solve = false;  // the spectral pass along y by the per-wavenumber row solve
  double *met_a64 = nullptr, *met_b64 = nullptr;
  float *met_a32 = nullptr, *met_b32 = nullptr;
  // the bank levels' side streams and their fork / join events
  cudaStream_t side[2] = {nullptr, nullptr};
  cudaEvent_t ev_fork = nullptr, ev_join[2] = {nullptr, nullptr};
  struct MapEntry {
    const void* p;
    int elem, bw, bh;
    CUtensorMap m;
  };
  std::vector<MapEntry> maps;
};

namespace dt {

template <class T>
static dt_status dalloc(dt_flex* s, T** p, size_t count) {
  void* q = nullptr;
  if (alloc_fault(s->nalloc)) {
    set_error("cudaMalloc of %zu bytes failed: out of memory (DT_FAIL_ALLOC_AT)", count * sizeof(T));
    return DT_OOM;
  }
  cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T));
  if (e != cudaSuccess) {
    set_error("cudaMalloc of %zu bytes failed: %s", count * sizeof(T), cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? DT_OOM : DT_DEVICE_ERROR;
  }
  s->allocs.push_back(q);
  *p = reinterpret_cast<T*>(q);
  return DT_OK;
}

template <class T>
static dt_status make_tables(dt_flex* s, Tables<T>& tb) {
  int N = s->N, h = s->h, w = s->w;
  std::vector<cplx<T>> a(N), b(N), c(h), o(h), o2(h);
  std::vector<T> lx(N + 1), ly(h);
  for (int t = 0; t < N; ++t) {
    long double ang = -2.0L * PI_L * t / N;
    a[t] = mk<cplx<T>>((T)cosl(ang), (T)sinl(ang));
    long double ang2 = -2.0L * PI_L * t / w;
    b[t] = mk<cplx<T>>((T)cosl(ang2), (T)sinl(ang2));
  }
  for (int t = 0; t < h; ++t) {
    long double ang = -2.0L * PI_L * t / h;
    c[t] = mk<cplx<T>>((T)cosl(ang), (T)sinl(ang));
    long double ang2 = -PI_L * t / (2.0L * h);
    o[t] = mk<cplx<T>>((T)cosl(ang2), (T)sinl(ang2));
    long double ang3 = -PI_L * t / h;
    o2[t] = mk<cplx<T>>((T)cosl(ang3), (T)sinl(ang3));
  }
  // the Laplacian's symbols as the reference forms them (flexure.rs:1145-1150), in double
  for (int k = 0; k <= N; ++k) lx[k] = (T)(2.0 * std::cos(6.283185307179586476925286766559 * (double)k / (double)w) - 2.0);
  for (int m = 0; m < h; ++m) ly[m] = (T)(2.0 * std::cos(3.141592653589793238462643383279 * (double)m / (double)h) - 2.0);
  DT_TRY(dalloc(s, &tb.tw_row, N));
  DT_TRY(dalloc(s, &tb.post, N));
  DT_TRY(dalloc(s, &tb.tw_col, h));
  DT_TRY(dalloc(s, &tb.omega, h));
  DT_TRY(dalloc(s, &tb.omega2, h));
  DT_TRY(dalloc(s, &tb.lx, N + 1));
  DT_TRY(dalloc(s, &tb.ly, h));
  DT_CUDA(cudaMemcpy(tb.tw_row, a.data(), N * sizeof(cplx<T>), cudaMemcpyHostToDevice));
  DT_CUDA(cudaMemcpy(tb.post, b.data(), N * sizeof(cplx<T>), cudaMemcpyHostToDevice));
  DT_CUDA(cudaMemcpy(tb.tw_col, c.data(), h * sizeof(cplx<T>), cudaMemcpyHostToDevice));
  DT_CUDA(cudaMemcpy(tb.omega, o.data(), h * sizeof(cplx<T>), cudaMemcpyHostToDevice));
  DT_CUDA(cudaMemcpy(tb.omega2, o2.data(), h * sizeof(cplx<T>), cudaMemcpyHostToDevice));
  DT_CUDA(cudaMemcpy(tb.lx, lx.data(), (N + 1) * sizeof(T), cudaMemcpyHostToDevice));
  DT_CUDA(cudaMemcpy(tb.ly, ly.data(), h * sizeof(T), cudaMemcpyHostToDevice));
  return DT_OK;
}

// The plan of the transform along x for a width whose half is not a power of two: mixed-radix
// stages when every prime factor of w is at most ANY_MAX_PRIME, else Bluestein through the power
// of two M >= 2 w - 1.
static AnyPlan make_any_plan(int w, int h) {
  AnyPlan p;
  p.w = w;
  p.pairs = (h + 1) / 2;
  std::vector<int> f;
  int n = w;
  for (int r : {16, 8, 4, 2})
    while (n % r == 0) {
      f.push_back(r);
      n /= r;
    }
  for (int q = 3; q <= ANY_MAX_PRIME && n > 1; q += 2)
    while (n % q == 0) {
      f.push_back(q);
      n /= q;
    }
  if (n > 1) {  // a prime factor beyond ANY_MAX_PRIME
    p.bluestein = 1;
    int m = 1;
    while (m < 2 * w - 1) m *= 2;
    f.clear();
    for (int r : {16, 8, 4, 2})
      while (m % r == 0) {
        f.push_back(r);
        m /= r;
      }
  }
  p.L = 1;
  for (int x : f) p.L *= x;
  p.nst = (int)f.size();
  int span = 1;
  for (int k = 0; k < p.nst; ++k) {
    p.radix[k] = f[k];
    p.span[k] = span;
    span *= f[k];
  }
  return p;
}

// Host FFT in long double (iterative radix 2, length a power of two): Bluestein's table B.
static void host_fft(std::vector<std::complex<long double>>& a) {
  const size_t n = a.size();
  for (size_t i = 1, j = 0; i < n; ++i) {
    size_t bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) std::swap(a[i], a[j]);
  }
  for (size_t len = 2; len <= n; len <<= 1) {
    for (size_t i = 0; i < n; i += len)
      for (size_t k = 0; k < len / 2; ++k) {
        long double ang = -2.0L * PI_L * (long double)k / (long double)len;
        std::complex<long double> t = a[i + k + len / 2] * std::complex<long double>(cosl(ang), sinl(ang));
        a[i + k + len / 2] = a[i + k] - t;
        a[i + k] += t;
      }
  }
}

template <class T>
static dt_status make_any_tables(dt_flex* s, Lane<T>& L) {
  using C = cplx<T>;
  const AnyPlan& p = s->plan;
  std::vector<C> tw(p.L);
  for (int t = 0; t < p.L; ++t) {
    long double ang = -2.0L * PI_L * t / p.L;
    tw[t] = mk<C>((T)cosl(ang), (T)sinl(ang));
  }
  DT_TRY(dalloc(s, &L.any_tw, p.L));
  DT_CUDA(cudaMemcpy(L.any_tw, tw.data(), p.L * sizeof(C), cudaMemcpyHostToDevice));
  DT_TRY(dalloc(s, &L.any_buf, (size_t)3 * 2 * p.pairs * p.L));
  if (p.bluestein) {
    // c_n = e^(i pi n^2 / w) with n^2 reduced mod 2 w; b_n = c_n, b_(M - n) = c_n; B = FFT_M(b)
    const int w = p.w;
    std::vector<C> chirp(w);
    std::vector<std::complex<long double>> b(p.L, 0.0L);
    for (int q = 0; q < w; ++q) {
      long long m = ((long long)q * q) % (2LL * w);
      long double ang = PI_L * (long double)m / (long double)w;
      std::complex<long double> c(cosl(ang), sinl(ang));
      chirp[q] = mk<C>((T)c.real(), (T)c.imag());
      b[q] = c;
      if (q > 0) b[p.L - q] = c;
    }
    host_fft(b);
    std::vector<C> bh(p.L);
    for (int q = 0; q < p.L; ++q) bh[q] = mk<C>((T)b[q].real(), (T)b[q].imag());
    DT_TRY(dalloc(s, &L.any_chirp, w));
    DT_TRY(dalloc(s, &L.any_bhat, p.L));
    DT_CUDA(cudaMemcpy(L.any_chirp, chirp.data(), w * sizeof(C), cudaMemcpyHostToDevice));
    DT_CUDA(cudaMemcpy(L.any_bhat, bh.data(), p.L * sizeof(C), cudaMemcpyHostToDevice));
  }
  return DT_OK;
}

template <class T>
static dt_status make_lane(dt_flex* s, Lane<T>& L) {
  size_t n = s->n;
  for (T** p : {&L.d, &L.c, &L.x, &L.r, &L.z, &L.p, &L.ap, &L.J, &L.left, &L.part}) DT_TRY(dalloc(s, p, n));
  DT_TRY(dalloc(s, &L.wt[0], 3 * n));
  L.wt[1] = L.wt[0] + n;
  L.wt[2] = L.wt[0] + 2 * n;
  const size_t hn = (size_t)s->h * s->N;
  DT_TRY(dalloc(s, &L.half, 3 * hn));
  L.half_side[0] = L.half + hn;
  L.half_side[1] = L.half + 2 * hn;
  if (s->row_solve) {
    DT_TRY(dalloc(s, &L.row_factors, 9 * (size_t)s->h * (s->N + 1)));
    const size_t P = ceil_div(s->h, ROW_CHUNK);
    if (P > 1) {
      DT_TRY(dalloc(s, &L.row_transfer, 3 * 8 * P * (s->N + 1)));
      DT_TRY(dalloc(s, &L.row_state, 3 * 4 * P * (s->N + 1)));
    }
  }
  DT_TRY(make_tables(s, L.tab));
  if (s->any) DT_TRY(make_any_tables(s, L));
  DT_TRY(dalloc(s, &L.S, 1));
  DT_CUDA(cudaMemset(L.S, 0, sizeof(Scalars)));
  return DT_OK;
}

template <class T>
static void free_graphs(Lane<T>& L) {
  for (int k = 0; k < 4; ++k) {
    if (L.exec[k]) cudaGraphExecDestroy(L.exec[k]);
    if (L.graph[k]) cudaGraphDestroy(L.graph[k]);
    L.exec[k] = nullptr;
    L.graph[k] = nullptr;
  }
}

template <class T>
static const T* metric_a(const dt_flex* s);
template <>
const double* metric_a<double>(const dt_flex* s) { return s->met_a64; }
template <>
const float* metric_a<float>(const dt_flex* s) { return s->met_a32; }
template <class T>
static const T* metric_b(const dt_flex* s);
template <>
const double* metric_b<double>(const dt_flex* s) { return s->met_b64; }
template <>
const float* metric_b<float>(const dt_flex* s) { return s->met_b32; }

static unsigned int ew_grid(const dt_flex* s) { return std::max(1u, std::min<unsigned int>(ceil_div(s->n, 256), (unsigned)s->sms * 8)); }

// ---- the TMA stencil's host side ----
static PFN_cuTensorMapEncodeTiled encode_tiled() {
  static PFN_cuTensorMapEncodeTiled fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return (PFN_cuTensorMapEncodeTiled) nullptr;
    return (PFN_cuTensorMapEncodeTiled)p;
  }();
  return fn;
}

// The 2-D map of a w x h buffer with the given box (columns x rows), zero fill outside; cached.
static bool tensor_map(dt_flex* s, const void* p, int elem, int bw, int bh, CUtensorMap* out) {
  for (auto& e : s->maps)
    if (e.p == p && e.elem == elem && e.bw == bw && e.bh == bh) {
      *out = e.m;
      return true;
    }
  PFN_cuTensorMapEncodeTiled fn = encode_tiled();
  if (!fn || !p || ((size_t)p & 15)) return false;
  dt_flex::MapEntry e{p, elem, bw, bh, {}};
  cuuint64_t dims[2] = {(cuuint64_t)s->w, (cuuint64_t)s->h};
  cuuint64_t strides[1] = {(cuuint64_t)s->w * (cuuint64_t)elem};
  cuuint32_t box[2] = {(cuuint32_t)bw, (cuuint32_t)bh};
  cuuint32_t es[2] = {1, 1};
  CUresult r = fn(&e.m, elem == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void*>(p),
                  dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return false;
  s->maps.push_back(e);
  *out = e.m;
  return true;
}

// Resident blocks per SM of each TMA stencil instantiation ([double][mode]), set at create.
static int g_tma_per_sm[2][7];

template <class T, int MODE>
static void tma_setup() {
  using ST = TmaStage<T, MODE>;
  cudaFuncSetAttribute(k_apply_tma<T, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, ST::SMEM);
  int nb = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_apply_tma<T, MODE>, TBX * TTY, ST::SMEM);
  g_tma_per_sm[sizeof(T) == 8][MODE] = std::max(nb, 1);
}
template <class T>
static void tma_setup_all() {
  tma_setup<T, AP_DOT>();
  tma_setup<T, RESID>();
  tma_setup<T, JAC_LEFT>();
  tma_setup<T, JAC_FINAL>();
  tma_setup<T, PLAIN>();
  tma_setup<T, BEND>();
  tma_setup<T, RESID_GATED>();
}

// The persistent TMA stencil; false (nothing launched) when a buffer cannot be mapped.
template <class T, int MODE>
static bool launch_apply_tma(dt_flex* s, const T* vsrc, const T* J, const T* part, const T* d, const T* c, const T* rb, T* y,
                             Scalars* S, cudaStream_t st) {
  using ST = TmaStage<T, MODE>;
  CUtensorMap mv, mJ, mP, md, mc, mb;
  if (!tensor_map(s, vsrc, sizeof(T), ST::P, ST::UR, &mv)) return false;
  mJ = mP = mc = mb = mv;
  if (ST::JAC && !tensor_map(s, J, sizeof(T), ST::P, ST::UR, &mJ)) return false;
  if (MODE == JAC_FINAL && !tensor_map(s, part, sizeof(T), ST::P, ST::UR, &mP)) return false;
  if (!tensor_map(s, d, sizeof(T), ST::P, ST::MR, &md)) return false;
  if (ST::HAS_C && !tensor_map(s, c, sizeof(T), TBX, ST::TBY, &mc)) return false;
  if (ST::HAS_B && !tensor_map(s, rb, sizeof(T), TBX, ST::TBY, &mb)) return false;
  const int tiles_x = s->w / TBX, ntiles = tiles_x * (int)ceil_div(s->h, ST::TBY);
  const int grid = std::max(1, std::min(ntiles, g_tma_per_sm[sizeof(T) == 8][MODE] * s->sms));
  T inv = (T)(1.0 / (s->dx * s->dx));
  k_apply_tma<T, MODE><<<grid, dim3(TBX, TTY), ST::SMEM, st>>>(mv, mJ, mP, md, mc, mb, s->w, s->h, inv, vsrc, J, part, d, y,
                                                              s->partials, S, tiles_x, ntiles);
  counted();
  return true;
}

// The operator on the sphere's row metric: the per-block kernel (the TMA stencil has the block
// metric only), the handle's couplings in the lane's precision.
template <class T>
static void launch_apply_metric(dt_flex* s, int mode, dim3 grid, dim3 block, T inv, const T* v, const T* J, const T* part,
                                const T* d, const T* c, const T* rb, T* y, Scalars* S, cudaStream_t st) {
  const T* ma = metric_a<T>(s);
  const T* mb = metric_b<T>(s);
#define DT_MET_CASE(M) \
  case M: k_apply<T, M, true><<<grid, block, 0, st>>>(s->w, s->h, inv, v, J, part, d, c, rb, y, s->partials, S, ma, mb); break;
  switch (mode) {
    DT_MET_CASE(AP_DOT)
    DT_MET_CASE(RESID)
    DT_MET_CASE(JAC_LEFT)
    DT_MET_CASE(JAC_FINAL)
    DT_MET_CASE(PLAIN)
    DT_MET_CASE(BEND)
    DT_MET_CASE(RESID_GATED)
  }
#undef DT_MET_CASE
  counted();
}

template <class T>
static void launch_apply(dt_flex* s, int mode, const T* v, const T* J, const T* part, const T* d, const T* c, const T* rb, T* y,
                         Scalars* S, cudaStream_t st) {
  if (s->tma && !s->metric) {
    const T* vsrc = (mode == JAC_LEFT || mode == JAC_FINAL) ? rb : v;
    bool done = false;
    switch (mode) {
      case AP_DOT: done = launch_apply_tma<T, AP_DOT>(s, vsrc, J, part, d, c, rb, y, S, st); break;
      case RESID: done = launch_apply_tma<T, RESID>(s, vsrc, J, part, d, c, rb, y, S, st); break;
      case JAC_LEFT: done = launch_apply_tma<T, JAC_LEFT>(s, vsrc, J, part, d, c, rb, y, S, st); break;
      case JAC_FINAL: done = launch_apply_tma<T, JAC_FINAL>(s, vsrc, J, part, d, c, rb, y, S, st); break;
      case PLAIN: done = launch_apply_tma<T, PLAIN>(s, vsrc, J, part, d, c, rb, y, S, st); break;
      case BEND: done = launch_apply_tma<T, BEND>(s, vsrc, J, part, d, c, rb, y, S, st); break;
      case RESID_GATED: done = launch_apply_tma<T, RESID_GATED>(s, vsrc, J, part, d, c, rb, y, S, st); break;
    }
    if (done) return;
  }
  dim3 grid(ceil_div(s->w, TBX), ceil_div(s->h, tile_rows<T>())), block(TBX, TTY);
  T inv = (T)(1.0 / (s->dx * s->dx));
  if (s->metric) {
    launch_apply_metric<T>(s, mode, grid, block, inv, v, J, part, d, c, rb, y, S, st);
    return;
  }
  switch (mode) {
    case AP_DOT: k_apply<T, AP_DOT><<<grid, block, 0, st>>>(s->w, s->h, inv, v, J, part, d, c, rb, y, s->partials, S); counted(); break;
    case RESID: k_apply<T, RESID><<<grid, block, 0, st>>>(s->w, s->h, inv, v, J, part, d, c, rb, y, s->partials, S); counted(); break;
    case JAC_LEFT: k_apply<T, JAC_LEFT><<<grid, block, 0, st>>>(s->w, s->h, inv, v, J, part, d, c, rb, y, s->partials, S); counted(); break;
    case JAC_FINAL: k_apply<T, JAC_FINAL><<<grid, block, 0, st>>>(s->w, s->h, inv, v, J, part, d, c, rb, y, s->partials, S); counted(); break;
    case PLAIN: k_apply<T, PLAIN><<<grid, block, 0, st>>>(s->w, s->h, inv, v, J, part, d, c, rb, y, s->partials, S); counted(); break;
    case BEND: k_apply<T, BEND><<<grid, block, 0, st>>>(s->w, s->h, inv, v, J, part, d, c, rb, y, s->partials, S); counted(); break;
    case RESID_GATED: k_apply<T, RESID_GATED><<<grid, block, 0, st>>>(s->w, s->h, inv, v, J, part, d, c, rb, y, s->partials, S); counted(); break;
  }
}

// Whether the column pass of length 2^logh runs k_cols_fused: FP32, a last radix below 16, and
// at least two columns a k_cols block (h <= 2048), so that the fused block of half as many
// columns stays within 256 threads.
template <class T>
static constexpr bool cols_fusable(int logh) {
  return sizeof(T) == 4 && logh >= 5 && logh <= 11 && logh % 4 != 0;
}

// Launch geometry of the transform kernels: rows (RB rows a block) and columns (CPB columns a
// block), each thread FFT_EPT complex values, padded shared memory.
struct FftGeo {
  unsigned int rgrid, cgrid;
  int rthreads, cthreads;
  size_t rsmem, csmem;
};
template <class T>
static FftGeo fft_geometry(const dt_flex* s) {
  using C = cplx<T>;
  FftGeo g;
  int logn = ilog2(s->N), logh = ilog2(s->h);
  int N = s->N, RB = rows_per_block(logn);
  g.rgrid = ceil_div(s->h, RB);
  g.rthreads = std::max(1, RB * N / FFT_EPT);
  g.rsmem = (size_t)RB * Pad<C>::len(N) * sizeof(C);
  const bool fused = s->cols_fused && cols_fusable<T>(logh);
  int cpb = fused ? cols_per_block_fused(logh, (int)sizeof(C)) : cols_per_block(logh, (int)sizeof(C));
  g.cgrid = ceil_div(N, cpb);
  g.cthreads = std::max(1, cpb * s->h / FFT_EPT);
  g.csmem = (size_t)cpb * (fused ? col_pitch_fused(s->h, cpb) : col_pitch(s->h)) * sizeof(C);
  return g;
}

// Per-size instantiations of the transform kernels, indexed by log2 of the transform length.
constexpr int FFT_LOGS = 14;  // lengths 1 .. 8192
template <class T, bool W>
using RowsFwdFn = void (*)(int, int, const T*, const T*, cplx<T>*, const cplx<T>*, const cplx<T>*, const Scalars*);
template <class T>
using ColsFn = void (*)(int, cplx<T>*, const cplx<T>*, const cplx<T>*, const cplx<T>*, const T*, const T*, T, const Scalars*,
                        int);
template <class T>
using RowsInvFn = void (*)(int, int, const cplx<T>*, T*, const T*, const T*, const cplx<T>*, const cplx<T>*, double*, Scalars*);

template <class T, bool W, int... L>
static RowsFwdFn<T, W> rows_fwd_fn(int logn, std::integer_sequence<int, L...>) {
  static const RowsFwdFn<T, W> table[] = {&k_rows_fwd<T, W, L>...};
  return table[logn];
}
// The column kernel for length 2^L: the fused form when its last radix is below 16 (and
// `fused`), else k_cols.
template <class T, int L>
static constexpr ColsFn<T> cols_kernel(bool fused) {
  if constexpr (cols_fusable<T>(L))
    return fused ? &k_cols_fused<T, L> : &k_cols<T, L>;
  else
    return &k_cols<T, L>;
}
template <class T, int... L>
static ColsFn<T> cols_fn(int logh, std::integer_sequence<int, L...>, bool fused = true) {
  static const ColsFn<T> table[2][sizeof...(L)] = {{cols_kernel<T, L>(false)...}, {cols_kernel<T, L>(true)...}};
  return table[fused ? 1 : 0][logh];
}
template <class T, int MODE, int... L>
static RowsInvFn<T> rows_inv_fn(int logn, std::integer_sequence<int, L...>) {
  static const RowsInvFn<T> table[] = {&k_rows_inv<T, MODE, L>...};
  return table[logn];
}
using LogSeq = std::make_integer_sequence<int, FFT_LOGS>;
template <class T>
using RowsBankFn = void (*)(int, const cplx<T>*, T*, const T*, const cplx<T>*, const cplx<T>*, Scalars*);
// k_rows_inv_bank for rows of one block (N >= 512) whose three staging buffers take at most
// 112 KB of shared memory (two blocks an SM at least); null for the others
template <class T, int L>
static constexpr RowsBankFn<T> rows_bank_kernel() {
  if constexpr (L >= 9 && rows_bank_smem<T>(L) <= 112 * 1024)
    return &k_rows_inv_bank<T, L>;
  else
    return nullptr;
}
template <class T, int... L>
static RowsBankFn<T> rows_bank_fn(int logn, std::integer_sequence<int, L...>) {
  static const RowsBankFn<T> table[] = {rows_bank_kernel<T, L>()...};
  return table[logn];
}
template <class T>
static RowsInvFn<T> rows_inv_for(int mode, int logn) {
  switch (mode) {
    case INV_STORE: return rows_inv_fn<T, INV_STORE>(logn, LogSeq{});
    case INV_STORE_W: return rows_inv_fn<T, INV_STORE_W>(logn, LogSeq{});
    case INV_BANK: return rows_inv_fn<T, INV_BANK>(logn, LogSeq{});
    default: return rows_inv_fn<T, INV_STORE_DOT>(logn, LogSeq{});
  }
}

// Opt every transform instantiation in to large dynamic shared memory.
template <class T>
static void transform_smem_attributes() {
  int big = 200 * 1024;
  for (int l = 0; l < FFT_LOGS; ++l) {
    cudaFuncSetAttribute(rows_fwd_fn<T, true>(l, LogSeq{}), cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    cudaFuncSetAttribute(rows_fwd_fn<T, false>(l, LogSeq{}), cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    cudaFuncSetAttribute(cols_fn<T>(l, LogSeq{}, false), cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    cudaFuncSetAttribute(cols_fn<T>(l, LogSeq{}, true), cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    for (int m : {INV_STORE, INV_STORE_W, INV_STORE_DOT, INV_BANK})
      cudaFuncSetAttribute(rows_inv_for<T>(m, l), cudaFuncAttributeMaxDynamicSharedMemorySize, big);
    if (RowsBankFn<T> f = rows_bank_fn<T>(l, LogSeq{}))
      cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rows_bank_smem<T>(l));
  }
}

// ---- the transform along x for any width (rows_any.cuh) ----
static unsigned int any_grid(size_t threads) { return ceil_div(threads, 256); }

// One FFT of length L over all row pairs: the stages alternate between a and b; returns the
// buffer holding the result.
template <class T>
static cplx<T>* any_fft(dt_flex* s, Lane<T>& L, cplx<T>* a, cplx<T>* b, Scalars* S, cudaStream_t st) {
  const AnyPlan& p = s->plan;
  for (int k = 0; k < p.nst; ++k) {
    const int R = p.radix[k];
    const size_t bf = (size_t)p.pairs * (p.L / R);
    switch (R) {
      case 2: k_any_stage<T, 2><<<any_grid(bf), 256, 0, st>>>(p, k, a, b, L.any_tw, S); break;
      case 3: k_any_stage<T, 3><<<any_grid(bf), 256, 0, st>>>(p, k, a, b, L.any_tw, S); break;
      case 4: k_any_stage<T, 4><<<any_grid(bf), 256, 0, st>>>(p, k, a, b, L.any_tw, S); break;
      case 5: k_any_stage<T, 5><<<any_grid(bf), 256, 0, st>>>(p, k, a, b, L.any_tw, S); break;
      case 7: k_any_stage<T, 7><<<any_grid(bf), 256, 0, st>>>(p, k, a, b, L.any_tw, S); break;
      case 8: k_any_stage<T, 8><<<any_grid(bf), 256, 0, st>>>(p, k, a, b, L.any_tw, S); break;
      case 16: k_any_stage<T, 16><<<any_grid(bf), 256, 0, st>>>(p, k, a, b, L.any_tw, S); break;
      default:
        k_any_stage_prime<T><<<any_grid((size_t)p.pairs * p.L), 256, 0, st>>>(p, k, a, b, L.any_tw, S);
        break;
    }
    counted();
    std::swap(a, b);
  }
  return a;
}

// DFT_w of each row pair from buffer a (b is scratch); returns the buffer holding the DFT's
// pass output (Bluestein: its second FFT, which any_fetch turns into the DFT).
template <class T>
static cplx<T>* any_dft(dt_flex* s, Lane<T>& L, cplx<T>* a, cplx<T>* b, Scalars* S, cudaStream_t st) {
  cplx<T>* f = any_fft<T>(s, L, a, b, S, st);
  if (s->plan.bluestein) {
    k_any_chirp_mul<T><<<any_grid((size_t)s->plan.pairs * s->plan.L), 256, 0, st>>>(s->plan, f, L.any_bhat, S);
    counted();
    f = any_fft<T>(s, L, f, f == a ? b : a, S, st);
  }
  return f;
}

// The level's scratch pair: 2 x pairs x L complex values a level.
template <class T>
static cplx<T>* any_slot(dt_flex* s, Lane<T>& L, int level) {
  return L.any_buf + (size_t)level * 2 * s->plan.pairs * s->plan.L;
}

template <class T>
static void any_rows_fwd(dt_flex* s, Lane<T>& L, const T* in, const T* wt, cplx<T>* half, int level, Scalars* S,
                         cudaStream_t st) {
  const AnyPlan& p = s->plan;
  cplx<T>* a = any_slot<T>(s, L, level);
  cplx<T>* b = a + (size_t)p.pairs * p.L;
  const unsigned g = any_grid((size_t)p.pairs * p.L);
  if (wt)
    k_any_load_rows<T, true><<<g, 256, 0, st>>>(p, s->h, in, wt, a, L.any_chirp, S);
  else
    k_any_load_rows<T, false><<<g, 256, 0, st>>>(p, s->h, in, wt, a, L.any_chirp, S);
  counted();
  cplx<T>* f = any_dft<T>(s, L, a, b, S, st);
  k_any_split<T><<<any_grid((size_t)p.pairs * s->N), 256, 0, st>>>(p, s->h, s->N, f, half, L.any_chirp, S);
  counted();
}

template <class T>
static void any_rows_inv(dt_flex* s, Lane<T>& L, int mode, const cplx<T>* half, T* out, const T* wt, const T* r,
                         Scalars* S, cudaStream_t st) {
  const AnyPlan& p = s->plan;
  const int levels = mode == INV_BANK ? 3 : 1;
  const size_t pl = (size_t)p.pairs * p.L;
  cplx<T>* f0 = nullptr;
  for (int lv = 0; lv < levels; ++lv) {
    cplx<T>* a = any_slot<T>(s, L, lv);
    k_any_load_half<T><<<any_grid(pl), 256, 0, st>>>(p, s->h, s->N, half + (size_t)lv * s->h * s->N, a, L.any_chirp, S);
    counted();
    cplx<T>* f = any_dft<T>(s, L, a, a + pl, S, st);
    if (lv == 0) f0 = f;  // every level ends in the same buffer of its pair
  }
  const unsigned g = std::min<unsigned>(any_grid((size_t)p.pairs * p.w), (unsigned)s->sms * 4);
  const size_t stride = 2 * pl;
  switch (mode) {
    case INV_STORE: k_any_emit<T, INV_STORE><<<g, 256, 0, st>>>(p, s->h, f0, stride, out, wt, r, L.any_chirp, s->partials, S); break;
    case INV_STORE_W: k_any_emit<T, INV_STORE_W><<<g, 256, 0, st>>>(p, s->h, f0, stride, out, wt, r, L.any_chirp, s->partials, S); break;
    case INV_BANK: k_any_emit<T, INV_BANK><<<g, 256, 0, st>>>(p, s->h, f0, stride, out, wt, r, L.any_chirp, s->partials, S); break;
    default: k_any_emit<T, INV_STORE_DOT><<<g, 256, 0, st>>>(p, s->h, f0, stride, out, wt, r, L.any_chirp, s->partials, S); break;
  }
  counted();
}

template <class T>
static void launch_rows_fwd(dt_flex* s, Lane<T>& L, const T* in, const T* wt, cplx<T>* half, const FftGeo& g, Scalars* S,
                            cudaStream_t st, int level = 0) {
  if (s->any) {
    any_rows_fwd<T>(s, L, in, wt, half, level, S, st);
    return;
  }
  int logn = ilog2(s->N);
  if (wt)
    rows_fwd_fn<T, true>(logn, LogSeq{})<<<g.rgrid, g.rthreads, g.rsmem, st>>>(s->w, s->h, in, wt, half, L.tab.tw_row,
                                                                                  L.tab.post, S);
  else
    rows_fwd_fn<T, false>(logn, LogSeq{})<<<g.rgrid, g.rthreads, g.rsmem, st>>>(s->w, s->h, in, wt, half, L.tab.tw_row,
                                                                                   L.tab.post, S);
  counted();
}
template <class T>
static void launch_cols(dt_flex* s, Lane<T>& L, cplx<T>* half, const FftGeo& g, int level, Scalars* S, cudaStream_t st) {
  if (s->row_solve) {
    // the row solve per wavenumber with the level's factors (made by setup_precond): in chunks
    // of rows when there is more than one, else one walk per wavenumber
    const size_t fac = (size_t)s->h * (s->N + 1);
    const T* dd = L.row_factors + (size_t)level * 3 * fac;
    const T *l1 = dd + fac, *l2 = dd + 2 * fac;
    const int P = (int)ceil_div(s->h, ROW_CHUNK);
    if (P == 1) {
      k_row_solve<T><<<ceil_div(s->N + 1, 128), 128, 0, st>>>(s->N, s->h, half, dd, l1, l2, S);
      counted();
      return;
    }
    const size_t plane = (size_t)P * (s->N + 1);
    const T* tf = L.row_transfer + (size_t)level * 8 * plane;
    const T* tb = tf + 4 * plane;
    cplx<T>* part = L.row_state + (size_t)level * 4 * plane;
    cplx<T>* carry = part + 2 * plane;
    const unsigned gp = ceil_div(plane, 128), gq = ceil_div(s->N + 1, 128);
    k_row_down_part<T><<<gp, 128, 0, st>>>(s->N, s->h, P, half, l1, l2, part, S);
    k_row_carry<T><<<gq, 128, 0, st>>>(s->N, P, false, tf, part, carry, S);
    k_row_down_final<T><<<gp, 128, 0, st>>>(s->N, s->h, P, half, dd, l1, l2, carry, part, S);
    k_row_carry<T><<<gq, 128, 0, st>>>(s->N, P, true, tb, part, carry, S);
    k_row_up_final<T><<<gp, 128, 0, st>>>(s->N, s->h, P, half, l1, l2, carry, S);
    for (int k = 0; k < 5; ++k) counted();
    return;
  }
  cols_fn<T>(ilog2(s->h), LogSeq{}, s->cols_fused)<<<g.cgrid, g.cthreads, g.csmem, st>>>(
      s->N, half, L.tab.tw_col, L.tab.omega, L.tab.omega2, L.tab.lx, L.tab.ly, (T)(1.0 / (s->dx * s->dx)), S, level);
  counted();
}
template <class T>
static void launch_rows_inv(dt_flex* s, Lane<T>& L, int mode, const cplx<T>* half, T* out, const T* wt, const T* r,
                            const FftGeo& g, Scalars* S, cudaStream_t st) {
  if (s->any) {
    any_rows_inv<T>(s, L, mode, half, out, wt, r, S, st);
    return;
  }
  const int logn = ilog2(s->N);
  if (mode == INV_BANK && s->rows_bank) {
    if (RowsBankFn<T> f = rows_bank_fn<T>(logn, LogSeq{})) {
      // persistent: as many blocks as the SMs hold at once, at most one a row
      const int nt = s->N / FFT_EPT;
      const size_t smem = rows_bank_smem<T>(logn);
      if (L.bank_blocks == 0) {
        int per = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, f, nt, smem) != cudaSuccess || per < 1) per = 1;
        L.bank_blocks = per * s->sms;
      }
      f<<<std::min(s->h, L.bank_blocks), nt, smem, st>>>(s->h, half, out, wt, L.tab.tw_row, L.tab.post, S);
      counted();
      return;
    }
  }
  rows_inv_for<T>(mode, logn)<<<g.rgrid, g.rthreads, g.rsmem, st>>>(s->w, s->h, half, out, wt, r, L.tab.tw_row,
                                                                    L.tab.post, s->partials, S);
  counted();
}

// One spectral solve of one bank level: out (op)= S_k (in * wt) (* wt), through the spectrum
// buffer `half` (the lane's own when null).
template <class T>
static void launch_spectral(dt_flex* s, Lane<T>& L, const T* in, const T* wt, T* out, int inv_mode, int level, Scalars* S,
                            cudaStream_t st, cplx<T>* half = nullptr) {
  FftGeo g = fft_geometry<T>(s);
  if (!half) half = L.half;
  launch_rows_fwd<T>(s, L, in, wt, half, g, S, st);
  launch_cols<T>(s, L, half, g, level, S, st);
  launch_rows_inv<T>(s, L, inv_mode, half, out, wt, inv_mode == INV_STORE_DOT ? in : nullptr, g, S, st);
}

// z = M^-1 r with r.z and max|z| reduced into S (finish_precond). levels 1: one spectral solve at
// node_d[0]; levels 3: the reference's bank inside damped Jacobi sweeps (flexure.rs:1630-1651).
template <class T>
static void launch_precondition(dt_flex* s, Lane<T>& L, const T* r, T* z, int levels, cudaStream_t st) {
  if (levels == 1) {
    launch_spectral<T>(s, L, r, nullptr, z, INV_STORE_DOT, 0, L.S, st);
    return;
  }
  launch_apply<T>(s, JAC_LEFT, nullptr, L.J, nullptr, L.d, L.c, r, L.left, L.S, st);  // left = r - A(J r)
  // part = sum_k w_k S_k(w_k left): the three levels' forward transforms and column passes are
  // independent. With the power-of-two kernels each pass takes the three levels in one launch
  // (their spectra and weights are consecutive); otherwise levels 1 and 2 run on side streams
  // (parallel branches when captured into the loop graph). One inverse pass then takes the
  // three spectra to the weighted sum.
  if (s->bank_one_launch && !s->any && !s->row_solve) {
    FftGeo g = fft_geometry<T>(s);
    rows_fwd_fn<T, true>(ilog2(s->N), LogSeq{})<<<dim3(g.rgrid, 3), g.rthreads, g.rsmem, st>>>(
        s->w, s->h, L.left, L.wt[0], L.half, L.tab.tw_row, L.tab.post, L.S);
    counted();
    cols_fn<T>(ilog2(s->h), LogSeq{}, s->cols_fused)<<<dim3(g.cgrid, 3), g.cthreads, g.csmem, st>>>(
        s->N, L.half, L.tab.tw_col, L.tab.omega, L.tab.omega2, L.tab.lx, L.tab.ly, (T)(1.0 / (s->dx * s->dx)), L.S, 0);
    counted();
    launch_rows_inv<T>(s, L, INV_BANK, L.half, L.part, L.wt[0], nullptr, g, L.S, st);
    launch_apply<T>(s, JAC_FINAL, nullptr, L.J, L.part, L.d, L.c, r, z, L.S, st);  // z = u + J(r - A u)
    return;
  }
  cudaEventRecord(s->ev_fork, st);
  cudaStreamWaitEvent(s->side[0], s->ev_fork, 0);
  cudaStreamWaitEvent(s->side[1], s->ev_fork, 0);
  FftGeo g = fft_geometry<T>(s);
  cudaStream_t lst[3] = {st, s->side[0], s->side[1]};
  cplx<T>* lh[3] = {L.half, L.half_side[0], L.half_side[1]};
  for (int k = 0; k < 3; ++k) {
    launch_rows_fwd<T>(s, L, L.left, L.wt[k], lh[k], g, L.S, lst[k], k);
    launch_cols<T>(s, L, lh[k], g, k, L.S, lst[k]);
  }
  cudaEventRecord(s->ev_join[0], s->side[0]);
  cudaEventRecord(s->ev_join[1], s->side[1]);
  cudaStreamWaitEvent(st, s->ev_join[0], 0);
  cudaStreamWaitEvent(st, s->ev_join[1], 0);
  launch_rows_inv<T>(s, L, INV_BANK, L.half, L.part, L.wt[0], nullptr, g, L.S, st);
  launch_apply<T>(s, JAC_FINAL, nullptr, L.J, L.part, L.d, L.c, r, z, L.S, st);  // z = u + J(r - A u)
}

// The residual replacement of a reliable-update iteration (FP32 lane): gated kernels that do
// nothing unless the iteration's update asked for it.
static void launch_reliable(dt_flex* s, cudaStream_t st) {
  Lane<double>& L = s->L64;
  Lane<float>& F = s->L32;
  k_reliable_accumulate<<<ew_grid(s), 256, 0, st>>>(s->n, L.x, F.x, s->scale, F.S); counted();
  launch_apply<double>(s, RESID_GATED, L.x, nullptr, nullptr, L.d, L.c, s->b64, L.r, F.S, st);
  k_reliable_reset<<<ew_grid(s), 256, 0, st>>>(s->n, L.r, F.r, s->scale, F.S); counted();
}

// While `st` captures a loop body: a conditional IF node, its body the residual replacement
// (captured on `aside`), so that iterations that replace nothing launch nothing for it. The
// update's finisher sets the node's condition. The replacement's kernels are left out of the
// body's launch count (a solve counts them from S->replacements).
static dt_status add_reliable_if(dt_flex* s, cudaStream_t st, cudaStream_t aside, unsigned long long* handle_out) {
  cudaStreamCaptureStatus cs;
  unsigned long long id = 0;
  cudaGraph_t graph = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  DT_CUDA(cudaStreamGetCaptureInfo(st, &cs, &id, &graph, &deps, &nd));
  if (cs != cudaStreamCaptureStatusActive || !graph) {
    set_error("flexure loop graph: the stream is not capturing");
    return DT_DEVICE_ERROR;
  }
  cudaGraphConditionalHandle h;
  DT_CUDA(cudaGraphConditionalHandleCreate(&h, graph, 0, cudaGraphCondAssignDefault));
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeIf;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  DT_CUDA(cudaGraphAddNode(&node, graph, deps, nd, &cp));
  DT_CUDA(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
  long long kept = g_captured;
  DT_CUDA(cudaStreamBeginCaptureToGraph(aside, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                        cudaStreamCaptureModeThreadLocal));
  launch_reliable(s, aside);
  cudaGraph_t ifbody;
  DT_CUDA(cudaStreamEndCapture(aside, &ifbody));
  g_captured = kept;
  *handle_out = (unsigned long long)h;
  return DT_OK;
}

// One PCG iteration (flexure.rs:1709-1738): the body of the device loop. With `reliable` (FP32
// lane) the residual replacement sits between the update and the preconditioner, so z, beta and
// p follow the replaced residual and the search direction carries on. Driven from the host its
// kernels run every iteration and do nothing unless gated on; in the graph (`aside` given) they
// sit in an IF node.
template <class T>
static dt_status launch_iteration(dt_flex* s, Lane<T>& L, int levels, cudaStream_t st, bool reliable = false,
                                  cudaStream_t aside = nullptr, unsigned long long* if_handle = nullptr) {
  launch_apply<T>(s, AP_DOT, L.p, nullptr, nullptr, L.d, L.c, nullptr, L.ap, L.S, st);
  k_update<T><<<ew_grid(s), 256, 0, st>>>(s->n, L.x, L.r, L.p, L.ap, s->partials, L.S); counted();
  if constexpr (sizeof(T) == 4) {
    if (reliable) {
      if (aside) {
        DT_TRY(add_reliable_if(s, st, aside, if_handle));
      } else {
        launch_reliable(s, st);
      }
    }
  }
  launch_precondition<T>(s, L, L.r, L.z, levels, st);
  k_direction<T><<<ew_grid(s), 256, 0, st>>>(s->n, L.p, L.z, L.S); counted();
  return DT_OK;
}

// The loop graph: k_arm -> WHILE(iteration) -> k_disarm. Built once per lane and level count.
template <class T>
static dt_status loop_exec(dt_flex* s, Lane<T>& L, int levels, cudaGraphExec_t* out, bool reliable = false) {
  int li = (levels == 3 ? 1 : 0) + (reliable ? 2 : 0);
  if (L.exec[li]) {
    *out = L.exec[li];
    return DT_OK;
  }
  cudaGraph_t g;
  DT_CUDA(cudaGraphCreate(&g, 0));
  cudaGraphConditionalHandle handle;
  DT_CUDA(cudaGraphConditionalHandleCreate(&handle, g, 1, cudaGraphCondAssignDefault));
  unsigned long long hv = (unsigned long long)handle, hv_if = 0ull;
  Scalars* Sp = L.S;
  cudaKernelNodeParams kp = {};
  void* arm_args[] = {&Sp, &hv, &hv_if};
  kp.func = (void*)k_arm;
  kp.gridDim = dim3(1);
  kp.blockDim = dim3(1);
  kp.kernelParams = arm_args;
  cudaGraphNode_t n_arm, n_loop, n_disarm;
  DT_CUDA(cudaGraphAddKernelNode(&n_arm, g, nullptr, 0, &kp));
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = handle;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  DT_CUDA(cudaGraphAddNode(&n_loop, g, &n_arm, 1, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  cudaStream_t aside = nullptr;
  if (reliable) DT_CUDA(cudaStreamCreateWithFlags(&aside, cudaStreamNonBlocking));
  DT_CUDA(cudaStreamBeginCaptureToGraph(s->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  g_capturing = true;
  g_captured = 0;
  dt_status st_body = launch_iteration<T>(s, L, levels, s->stream, reliable, aside, &hv_if);
  g_capturing = false;
  L.body_kernels[li] = g_captured;
  cudaGraph_t captured;
  cudaError_t e_end = cudaStreamEndCapture(s->stream, &captured);
  if (aside) cudaStreamDestroy(aside);
  DT_TRY(st_body);
  DT_CUDA(e_end);
  if (reliable) DT_CUDA(cudaGraphKernelNodeSetParams(n_arm, &kp));  // k_arm learns the IF node's handle
  void* dis_args[] = {&Sp};
  kp.func = (void*)k_disarm;
  kp.kernelParams = dis_args;
  DT_CUDA(cudaGraphAddKernelNode(&n_disarm, g, &n_loop, 1, &kp));
  cudaGraphExec_t exec;
  DT_CUDA(cudaGraphInstantiate(&exec, g, 0));
  L.graph[li] = g;
  L.exec[li] = exec;
  *out = exec;
  return DT_OK;
}

// The preconditioner set-up of a lane for its d, c: the bank (or the mean level), and for three
// levels the per-cell blend and Jacobi weights. Returns the level count (one host sync).
template <class T>
static dt_status setup_precond(dt_flex* s, Lane<T>& L, int precond, int* levels) {
  cudaStream_t st = s->stream;
  k_stats<T><<<ew_grid(s), 256, 0, st>>>(s->n, L.d, L.c, s->dx, precond == DT_PRECOND_MEAN_D, s->partials, L.S); counted();
  int lv = 1;
  DT_CUDA(cudaMemcpyAsync(&lv, &L.S->levels, sizeof(int), cudaMemcpyDeviceToHost, st));
  DT_CUDA(cudaStreamSynchronize(st));
  if (lv == 3) {
    k_bank_weights<T><<<ew_grid(s), 256, 0, st>>>(s->w, s->h, L.d, L.c, s->dx, L.wt[0], L.wt[1], L.wt[2], L.J, L.S,
                                                   s->metric ? s->met_a64 : nullptr, s->metric ? s->met_b64 : nullptr);
    counted();
  }
  if (s->row_solve) {
    // the row solve's factors of each level (its d, the bank's c_ref)
    const size_t fac = (size_t)s->h * (s->N + 1);
    for (int k = 0; k < lv; ++k) {
      T* dd = L.row_factors + (size_t)k * 3 * fac;
      k_row_factor<T><<<ceil_div(s->N + 1, 128), 128, 0, st>>>(s->N, s->h, L.tab.lx, metric_a<T>(s), metric_b<T>(s),
                                                             (T)(1.0 / (s->dx * s->dx)), L.S, k, dd, dd + fac, dd + 2 * fac);
      counted();
      const int P = (int)ceil_div(s->h, ROW_CHUNK);
      if (P > 1) {
        // the chunks' carry transfers, from the factors alone
        const size_t plane = (size_t)P * (s->N + 1);
        T* tf = L.row_transfer + (size_t)k * 8 * plane;
        k_row_transfer<T><<<ceil_div(plane, 128), 128, 0, st>>>(s->N, s->h, P, dd + fac, dd + 2 * fac, tf, tf + 4 * plane);
        counted();
      }
    }
  }
  DT_CUDA(cudaGetLastError());
  *levels = lv;
  return DT_OK;
}

struct HostProblem {
  double tol;
  int max_it;
  int rule;
  int n;
  int wait_give_up;
};
__global__ void k_put_problem(Scalars* S, HostProblem p) {
  S->fault = 0;
  S->wait_give_up = p.wait_give_up;
  S->tol = p.tol;
  S->max_it = p.max_it;
  S->rule = p.rule;
  S->n = p.n;
  S->reliable = 0;
  S->gate_it = -1;
}

// PCG of lane L from its x (guess), r = b - A x and S->rr, S->bb already set: the first
// preconditioning, p = z, then the device loop.
static dt_status read_scalars(dt_flex* s, const Scalars* S, Scalars* out) {
  DT_CUDA(cudaMemcpyAsync(out, S, sizeof(Scalars), cudaMemcpyDeviceToHost, s->stream));
  DT_CUDA(cudaStreamSynchronize(s->stream));
  return DT_OK;
}

// host_loop: 0 the device-side graph loop; 1 a host loop with one sync per iteration; 2 the same
// with each iteration's scalars printed to stderr. Returns with the solve enqueued (graph) or done.
template <class T>
static dt_status run_pcg(dt_flex* s, Lane<T>& L, int levels, int host_loop, bool reliable = false, bool z_given = false) {
  cudaStream_t st = s->stream;
  k_begin<<<1, 1, 0, st>>>(L.S); counted();
  if constexpr (sizeof(T) == 4) {
    if (z_given) {
      // the warm start's choice already preconditioned the first residual (unscaled, in L.z)
      k_scale_given_z<<<ew_grid(s), 256, 0, st>>>(s->n, L.z, L.r, s->scale, s->partials, L.S); counted();
    } else {
      launch_precondition<T>(s, L, L.r, L.z, levels, st);
    }
  } else {
    launch_precondition<T>(s, L, L.r, L.z, levels, st);
  }
  k_initial_result<T><<<ew_grid(s), 256, 0, st>>>(s->n, L.x, L.z, L.S); counted();
  DT_CUDA(cudaMemcpyAsync(L.p, L.z, s->n * sizeof(T), cudaMemcpyDeviceToDevice, st));
  if (!host_loop) {
    cudaGraphExec_t exec;
    DT_TRY(loop_exec<T>(s, L, levels, &exec, reliable));
    DT_CUDA(cudaGraphLaunch(exec, st));
    return DT_OK;
  }
  Scalars h;
  DT_TRY(read_scalars(s, L.S, &h));
  for (int pass = 0; pass < h.max_it + 2 && h.stop == STOP_RUNNING; ++pass) {
    DT_TRY(launch_iteration<T>(s, L, levels, st, reliable));
    DT_CUDA(cudaGetLastError());
    DT_TRY(read_scalars(s, L.S, &h));
    if (host_loop > 1)
      fprintf(stderr, "pcg(%s) it %d stop %d rr %.6e rz %.6e pap %.6e alpha %.6e beta %.6e err %.6e%s\n",
              sizeof(T) == 8 ? "fp64" : "fp32", h.it, h.stop, h.rr, h.rz, h.pap, h.alpha, h.beta, h.err,
              h.reliable && h.gate_it == h.it ? " (residual replaced)" : "");
  }
  return DT_OK;
}

// Kernels the graph loop ran in its last launch (arm and disarm, and a body per pass).
template <class T>
static void count_loop(const Lane<T>& L, int levels, int host_loop, int body_runs, bool reliable = false) {
  if (host_loop) return;
  g_launches += 2 + L.body_kernels[(levels == 3 ? 1 : 0) + (reliable ? 2 : 0)] * (long long)body_runs;
}

// r = b - A x in FP64 with ||r||^2 into S->rr.
static void resid64(dt_flex* s) {
  Lane<double>& L = s->L64;
  launch_apply<double>(s, RESID, L.x, nullptr, nullptr, L.d, L.c, s->b64, L.r, L.S, s->stream);
}

// ||b||^2 into S->bb
template <class T>
static void norm_b(dt_flex* s, const T* b, Scalars* S) {
  k_dot<T><<<ew_grid(s), 256, 0, s->stream>>>(s->n, b, b, s->partials, S, SITE_DOT); counted();
  k_take_bb<<<1, 1, 0, s->stream>>>(S); counted();
}

template <class T>
__global__ void k_add_to64(size_t n, double* __restrict__ x, const T* __restrict__ z) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) x[k] += (double)z[k];
}

__global__ void k_keep_rz(const Scalars* S, double* slot) { *slot = S->rz; }

// Keep x0 when its preconditioned residual is below the zero guess's, r0.M^-1 r0 < b.M^-1 b;
// otherwise x = 0, r = b. The 2-norm of the residual cannot rate a predicted guess: the
// operator multiplies the prediction's grid-scale rounding noise by up to d lambda^2 / c
// (1e5 to 1e8 on these rasters), while M^-1 weighs the residual as the error's energy does.
__global__ void k_warm_decide_pre(size_t n, double* __restrict__ x, double* __restrict__ r, const double* __restrict__ b,
                                  const double* rz) {
  bool keep = rz[1] < rz[0];
  if (keep) return;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    x[k] = 0.0;
    r[k] = b[k];
  }
}
__global__ void k_warm_record_pre(Scalars* S64, const double* rz, WarmInfo* info) {
  info->accepted = rz[1] < rz[0] ? 1 : 0;
  info->rel = rz[0] > 0 ? sqrt(rz[1] / rz[0]) : 0.0;
  if (!info->accepted) S64->rr = S64->bb;
}

// z = M^-1 v with the lane F (its preconditioner set up), v in FP64; v.z into *slot.
template <class T>
static void precond_dot(dt_flex* s, Lane<T>& F, const double* v, int levels, double* slot) {
  cudaStream_t st = s->stream;
  k_reset<<<1, 1, 0, st>>>(F.S);
  counted();
  const T* vin;
  if (sizeof(T) == 4) {
    k_convert<double, T><<<ew_grid(s), 256, 0, st>>>(s->n, v, F.r);
    counted();
    vin = F.r;
  } else {
    // the FP64 lane preconditions a copy in `ap` (free before the loop), leaving r and b
    // untouched (the Jacobi sandwich writes `left`, so that cannot hold the input)
    DT_CUDA_VOID(cudaMemcpyAsync(F.ap, v, s->n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    vin = F.ap;
  }
  launch_precondition<T>(s, F, vin, F.z, levels, st);
  k_keep_rz<<<1, 1, 0, st>>>(F.S, slot);
  counted();
}

// The first guess: x = 0 (r = b), or the given / predicted guess, kept by the preconditioned
// residual rule (k_warm_decide_pre).
template <class T>
static dt_status warm_or_cold(dt_flex* s, bool warm, Lane<T>& F, int levels) {
  Lane<double>& L = s->L64;
  cudaStream_t st = s->stream;
  if (!warm) {
    k_fill<double><<<ew_grid(s), 256, 0, st>>>(s->n, L.x, 0.0); counted();
    resid64(s);  // r = b
    WarmInfo none = {0, 1.0};
    DT_CUDA(cudaMemcpyAsync(s->warm, &none, sizeof none, cudaMemcpyHostToDevice, st));
    return DT_OK;
  }
  precond_dot<T>(s, F, s->b64, levels, s->rzpair);  // b . M^-1 b
  if constexpr (sizeof(T) == 4)  // M^-1 b kept (the FP32 lane's ap is free before its loop)
    DT_CUDA(cudaMemcpyAsync(F.ap, F.z, s->n * sizeof(T), cudaMemcpyDeviceToDevice, st));
  resid64(s);                                       // r0 = b - A x0
  precond_dot<T>(s, F, L.r, levels, s->rzpair + 1);  // r0 . M^-1 r0
  if constexpr (sizeof(T) == 4) {
    // F.z: the first preconditioned residual of whichever guess is kept
    k_warm_pick_z<<<ew_grid(s), 256, 0, st>>>(s->n, F.z, F.ap, s->rzpair);
    counted();
  }
  k_warm_decide_pre<<<ew_grid(s), 256, 0, st>>>(s->n, L.x, L.r, s->b64, s->rzpair);
  k_warm_record_pre<<<1, 1, 0, st>>>(L.S, s->rzpair, s->warm);
  counted();
  counted();
  DT_CUDA(cudaGetLastError());
  return DT_OK;
}

static dt_status fill_report(dt_flex* s, const Scalars& h, int iterations, int refinements, dt_report* rep) {
  WarmInfo wi;
  DT_CUDA(cudaMemcpy(&wi, s->warm, sizeof wi, cudaMemcpyDeviceToHost));
  if (!rep) return DT_OK;
  rep->iterations = iterations;
  rep->error_m = h.err;
  rep->refinements = refinements;
  rep->warm_start_accepted = wi.accepted;
  rep->warm_start_rel_residual = wi.rel;
  rep->kernel_launches = g_launches;
  return DT_OK;
}

// The FP64 solve; inputs in L64.d, L64.c, b64, and the guess in L64.x when warm.
static dt_status solve_fp64(dt_flex* s, const dt_flex_params* p, bool warm, dt_report* rep) {
  Lane<double>& L = s->L64;
  cudaStream_t st = s->stream;
  int levels = 1;
  DT_TRY(setup_precond<double>(s, L, p->precond, &levels));
  k_put_problem<<<1, 1, 0, st>>>(L.S, HostProblem{p->tol, p->max_iterations, p->stop, (int)s->n, s->wait_give_up}); counted();
  norm_b<double>(s, s->b64, L.S);
  DT_TRY(warm_or_cold(s, warm, L, levels));
  DT_TRY(run_pcg<double>(s, L, levels, p->host_loop));
  Scalars h;
  DT_TRY(read_scalars(s, L.S, &h));
  if (h.fault) {
    set_error("flexure solve: a kernel's wait for its tile copies ran out");
    return DT_DEVICE_ERROR;
  }
  count_loop(L, levels, p->host_loop, h.body_runs);
  int iterations = h.it;
  int stop = h.stop;
  double err = h.err;
  // the true residual of the answer
  resid64(s);
  DT_TRY(read_scalars(s, L.S, &h));
  if (h.fault) {
    set_error("flexure solve: a kernel's wait for its tile copies ran out");
    return DT_DEVICE_ERROR;
  }
  h.err = err;
  DT_TRY(fill_report(s, h, iterations, 0, rep));
  if (rep) {
    rep->converged = stop == STOP_CONVERGED;
    rep->rel_residual = h.bb > 0 ? std::sqrt(h.rr / h.bb) : 0.0;
  }
  if (stop == STOP_NONFINITE) {
    set_error("flexure solve: a non-finite value appeared");
    return DT_NONFINITE;
  }
  return stop == STOP_CONVERGED ? DT_OK : DT_NOT_CONVERGED;
}

// FP32 inner PCG inside FP64 iterative refinement. The outer loop stops on the FP64 relative (or
// RMS) residual; each inner solve works on the residual scaled to unit RMS and stops at a
// relative residual of max(inner_tol, 0.3 tol / current) (capped at 0.5): the last refinement
// needs only the reduction that is left.
static dt_status solve_mixed(dt_flex* s, const dt_flex_params* p, bool warm, dt_report* rep) {
  Lane<double>& L = s->L64;
  Lane<float>& F = s->L32;
  cudaStream_t st = s->stream;
  if (p->stop == DT_STOP_MAX_Z) {
    set_error("flexure solve: the mixed-precision path stops on a residual rule (DT_STOP_REL_RESIDUAL or DT_STOP_RMS_RESIDUAL)");
    return DT_UNSUPPORTED;
  }
  k_convert<double, float><<<ew_grid(s), 256, 0, st>>>(s->n, L.d, F.d); counted();
  k_convert<double, float><<<ew_grid(s), 256, 0, st>>>(s->n, L.c, F.c); counted();
  int levels = 1;
  DT_TRY(setup_precond<float>(s, F, p->precond, &levels));
  k_put_problem<<<1, 1, 0, st>>>(L.S, HostProblem{p->tol, p->max_iterations, p->stop, (int)s->n, s->wait_give_up}); counted();
  norm_b<double>(s, s->b64, L.S);
  DT_TRY(warm_or_cold(s, warm, F, levels));
  int iterations = 0, refinements = 0;
  Scalars h, hf;
  hf.err = 0.0;
  hf.stop = STOP_RUNNING;
  bool converged = false, nonfinite = false;
  for (;;) {
    DT_TRY(read_scalars(s, L.S, &h));
    if (h.fault) {
      set_error("flexure solve: a kernel's wait for its tile copies ran out");
      return DT_DEVICE_ERROR;
    }
    if (!std::isfinite(h.rr) || !std::isfinite(h.bb)) {
      nonfinite = true;
      break;
    }
    double rel = h.bb > 0 ? std::sqrt(h.rr / h.bb) : 0.0;
    double lim = p->stop == DT_STOP_REL_RESIDUAL ? p->tol : p->tol * std::sqrt((double)s->n / std::max(h.bb, 1e-300));
    if (h.bb <= 0 || rel <= lim) {
      converged = true;
      break;
    }
    if (refinements >= p->max_refinements || iterations >= p->max_iterations) break;
    double itol = std::min(0.5, std::max(p->inner_tol, 0.3 * lim / rel));
    k_scale_down<<<ew_grid(s), 256, 0, st>>>(s->n, L.r, F.r, F.x, L.S, s->scale); counted();
    k_put_problem<<<1, 1, 0, st>>>(F.S, HostProblem{itol, p->max_iterations - iterations, DT_STOP_REL_RESIDUAL, (int)s->n, s->wait_give_up}); counted();
    norm_b<float>(s, F.r, F.S);
    k_rr_is_bb<<<1, 1, 0, st>>>(F.S); counted();  // x = 0: r = b
    DT_TRY(run_pcg<float>(s, F, levels, p->host_loop));
    k_accumulate<<<ew_grid(s), 256, 0, st>>>(s->n, L.x, F.x, s->scale); counted();
    resid64(s);
    DT_TRY(read_scalars(s, F.S, &hf));
    if (hf.fault) {
      set_error("flexure solve: a kernel's wait for its tile copies ran out");
      return DT_DEVICE_ERROR;
    }
    count_loop(F, levels, p->host_loop, hf.body_runs);
    iterations += hf.it;
    ++refinements;
    if (hf.stop == STOP_NONFINITE) {
      nonfinite = true;
      break;
    }
  }
  DT_TRY(read_scalars(s, L.S, &h));
  h.err = hf.err;
  DT_TRY(fill_report(s, h, iterations, refinements, rep));
  if (rep) {
    rep->converged = converged;
    rep->rel_residual = h.bb > 0 ? std::sqrt(h.rr / h.bb) : 0.0;
  }
  if (nonfinite) {
    set_error("flexure solve: a non-finite value appeared");
    return DT_NONFINITE;
  }
  return converged ? DT_OK : DT_NOT_CONVERGED;
}

// FP32 PCG with reliable updates (the mixed-precision CG of lattice QCD solvers: Clark et al.,
// "Solving lattice QCD systems of equations using mixed precision solvers on GPUs", 2010). One
// FP32 Krylov sequence runs to the end; whenever its residual has fallen by RELIABLE_DELTA since
// the last replacement (or under the tolerance), the correction is added to the FP64 solution,
// the FP64 residual b - A x replaces the FP32 one and the search direction carries on. The FP64
// residual alone decides convergence. Unlike refinement, no restart throws the Krylov space away.
constexpr double RELIABLE_DELTA = 0.1;

static dt_status solve_mixed_reliable(dt_flex* s, const dt_flex_params* p, bool warm, dt_report* rep) {
  Lane<double>& L = s->L64;
  Lane<float>& F = s->L32;
  cudaStream_t st = s->stream;
  if (p->stop == DT_STOP_MAX_Z) {
    set_error("flexure solve: the mixed-precision path stops on a residual rule (DT_STOP_REL_RESIDUAL or DT_STOP_RMS_RESIDUAL)");
    return DT_UNSUPPORTED;
  }
  k_convert<double, float><<<ew_grid(s), 256, 0, st>>>(s->n, L.d, F.d); counted();
  k_convert<double, float><<<ew_grid(s), 256, 0, st>>>(s->n, L.c, F.c); counted();
  int levels = 1;
  DT_TRY(setup_precond<float>(s, F, p->precond, &levels));
  k_put_problem<<<1, 1, 0, st>>>(L.S, HostProblem{p->tol, p->max_iterations, p->stop, (int)s->n, s->wait_give_up}); counted();
  norm_b<double>(s, s->b64, L.S);
  DT_TRY(warm_or_cold(s, warm, F, levels));
  k_scale_down<<<ew_grid(s), 256, 0, st>>>(s->n, L.r, F.r, F.x, L.S, s->scale); counted();
  k_put_problem<<<1, 1, 0, st>>>(F.S, HostProblem{p->tol, p->max_iterations, DT_STOP_REL_RESIDUAL, (int)s->n, s->wait_give_up}); counted();
  k_reliable_init<<<1, 1, 0, st>>>(F.S, L.S, s->scale, p->tol, p->max_iterations, RELIABLE_DELTA,
                                   p->stop == DT_STOP_RMS_RESIDUAL ? 1 : 0);
  counted();
  // warm: the choice's M^-1 r0 (in F.z) is the first preconditioner application
  DT_TRY(run_pcg<float>(s, F, levels, p->host_loop, true, warm));
  // the correction the FP32 lane holds since its last replacement, and the true residual
  k_accumulate<<<ew_grid(s), 256, 0, st>>>(s->n, L.x, F.x, s->scale); counted();
  resid64(s);
  Scalars h, hf;
  DT_TRY(read_scalars(s, F.S, &hf));
  DT_TRY(read_scalars(s, L.S, &h));
  if (hf.fault || h.fault) {  // either lane's stencil (the FP64 residual's too)
    set_error("flexure solve: a kernel's wait for its tile copies ran out");
    return DT_DEVICE_ERROR;
  }
  count_loop(F, levels, p->host_loop, hf.body_runs, true);
  if (!p->host_loop) g_launches += 3LL * hf.replacements;  // the IF node's kernels, when they ran
  bool nonfinite = hf.stop == STOP_NONFINITE || !std::isfinite(h.rr) || !std::isfinite(h.bb);
  double bref = p->stop == DT_STOP_RMS_RESIDUAL ? (double)s->n : h.bb;
  bool converged = !nonfinite && (h.bb <= 0 || h.rr <= p->tol * p->tol * bref);
  h.err = hf.err;
  DT_TRY(fill_report(s, h, hf.it, 0, rep));
  if (rep) {
    rep->converged = converged;
    rep->rel_residual = h.bb > 0 ? std::sqrt(h.rr / h.bb) : 0.0;
  }
  if (nonfinite) {
    set_error("flexure solve: a non-finite value appeared");
    return DT_NONFINITE;
  }
  return converged ? DT_OK : DT_NOT_CONVERGED;
}

}  // namespace dt

using namespace dt;

// =============================================================================================
// C ABI

extern "C" {

const char* dt_last_error(void) { return dt::last_error(); }

int dt_device_info(char* name, int len) {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    if (name && len > 0) name[0] = 0;
    return 0;
  }
  cudaDeviceProp p;
  if (cudaGetDeviceProperties(&p, 0) != cudaSuccess) return 0;
  if (name && len > 0) snprintf(name, len, "%s (sm_%d%d, %d SMs)", p.name, p.major, p.minor, p.multiProcessorCount);
  return 1;
}

void dt_flex_default_params(dt_flex_params* p) {
  if (!p) return;
  p->precond = DT_PRECOND_REFERENCE;
  p->stop = DT_STOP_MAX_Z;
  p->precision = DT_PREC_FP64;
  p->warm_start = DT_WARM_NONE;
  p->tol = 2.0;            // FlexureParams::default tolerance_m (flexure.rs:224)
  p->max_iterations = 60;  // FlexureParams::default max_iterations (flexure.rs:225)
  p->inner_tol = 1e-5;
  p->max_refinements = 8;
  p->host_loop = 0;
}

dt_status dt_flex_destroy(dt_flex* s) {
  if (!s) return DT_OK;
  if (s->stream) cudaStreamSynchronize(s->stream);
  free_graphs(s->L64);
  free_graphs(s->L32);
  for (void* p : s->allocs) cudaFree(p);
  if (s->ev0) cudaEventDestroy(s->ev0);
  if (s->ev1) cudaEventDestroy(s->ev1);
  for (int k = 0; k < 2; ++k) {
    if (s->side[k]) cudaStreamDestroy(s->side[k]);
    if (s->ev_join[k]) cudaEventDestroy(s->ev_join[k]);
  }
  if (s->ev_fork) cudaEventDestroy(s->ev_fork);
  if (s->own_stream && s->stream) cudaStreamDestroy(s->stream);
  delete s;
  return DT_OK;
}

dt_status dt_flex_create(int w, int h, double dx, const double* metric_a, const double* metric_b, dt_flex** out) {
  if (!out) {
    set_error("dt_flex_create: out is NULL");
    return DT_BAD_ARG;
  }
  *out = nullptr;
  if (w < 2 || h < 2 || !(dx > 0.0) || !std::isfinite(dx)) {
    set_error("dt_flex_create: bad raster %d x %d, dx %g", w, h, dx);
    return DT_BAD_ARG;
  }
  // the transform along x takes any width: the shared-memory kernels when w/2 is a power of two
  // up to 8192, the passes of rows_any.cuh otherwise; along y the cosine transform takes a
  // power-of-two h, and any other h is solved per wavenumber (the row solve, with the block
  // metric's couplings when no metric is given)
  if (w > 65536 || h > 8192) {
    set_error("dt_flex_create: the device transforms take w up to 65536 and h up to 8192 (got %d x %d)", w, h);
    return DT_UNSUPPORTED;
  }
  if (!metric_a != !metric_b) {
    set_error("dt_flex_create: the row metric needs both a (h values) and b (h + 1 values)");
    return DT_BAD_ARG;
  }
  if (metric_a) {
    for (int j = 0; j < h; ++j)
      if (!std::isfinite(metric_a[j])) {
        set_error("dt_flex_create: metric a[%d] is not finite", j);
        return DT_BAD_ARG;
      }
    for (int j = 0; j <= h; ++j)
      if (!std::isfinite(metric_b[j])) {
        set_error("dt_flex_create: metric b[%d] is not finite", j);
        return DT_BAD_ARG;
      }
  }
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    set_error("dt_flex_create: no CUDA device");
    return DT_DEVICE_ERROR;
  }
  auto* s = new dt_flex();
  s->w = w;
  s->h = h;
  s->any = (w & 1) || !is_pow2(w / 2) || w / 2 > 8192;
  s->N = (w + 1) / 2;
  if (s->any) s->plan = make_any_plan(w, h);
  s->dx = dx;
  s->n = (size_t)w * h;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, 0) == cudaSuccess) s->sms = prop.multiProcessorCount;
  dt_status st = DT_OK;
  auto fail = [&](dt_status e) {
    dt_flex_destroy(s);
    return e;
  };
  if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) {
    set_error("dt_flex_create: cudaStreamCreate failed");
    return fail(DT_DEVICE_ERROR);
  }
  s->own_stream = true;
  if (const char* e = getenv("DT_STENCIL_WAIT_GIVE_UP")) s->wait_give_up = e[0] == '1';
  if (const char* e = getenv("DT_COLS_FUSED")) s->cols_fused = e[0] != '0';
  if (const char* e = getenv("DT_ROWS_BANK")) s->rows_bank = e[0] != '0';
  if (const char* e = getenv("DT_BANK_ONE_LAUNCH")) s->bank_one_launch = e[0] != '0';

  // RowMetric::block (flexure.rs:1000-1010): the block metric's couplings, for a height the
  // cosine transform does not take
  std::vector<double> block_a, block_b;
  if (!metric_a && !is_pow2(h)) {
    block_a.assign(h, 1.0);
    block_b.assign(h + 1, 1.0);
    block_b[0] = block_b[h] = 0.0;
    metric_a = block_a.data();
    metric_b = block_b.data();
  } else if (metric_a) {
    s->metric = true;
  }
  if (metric_a) {
    // the sphere's row metric (RowMetric, flexure.rs:954-998), or the block one, in both lanes'
    // precisions
    s->row_solve = true;
    std::vector<float> a32(metric_a, metric_a + h), b32(metric_b, metric_b + h + 1);
    if ((st = dalloc(s, &s->met_a64, (size_t)h)) != DT_OK || (st = dalloc(s, &s->met_b64, (size_t)h + 1)) != DT_OK ||
        (st = dalloc(s, &s->met_a32, (size_t)h)) != DT_OK || (st = dalloc(s, &s->met_b32, (size_t)h + 1)) != DT_OK)
      return fail(st);
    if (cudaMemcpy(s->met_a64, metric_a, h * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(s->met_b64, metric_b, (h + 1) * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(s->met_a32, a32.data(), h * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(s->met_b32, b32.data(), (h + 1) * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) {
      set_error("dt_flex_create: metric upload failed");
      return fail(DT_DEVICE_ERROR);
    }
  }
  if ((st = make_lane<double>(s, s->L64)) != DT_OK) return fail(st);
  if ((st = make_lane<float>(s, s->L32)) != DT_OK) return fail(st);
  if ((st = dalloc(s, &s->b64, s->n)) != DT_OK) return fail(st);
  size_t tiles = (size_t)ceil_div(w, TBX) * ceil_div(h, TBY_MIN);
  size_t cap = std::max<size_t>(std::max<size_t>(tiles, (size_t)s->sms * 8), (size_t)h) * 4;
  if ((st = dalloc(s, &s->partials, cap)) != DT_OK) return fail(st);
  if ((st = dalloc(s, &s->scale, 1)) != DT_OK) return fail(st);
  if ((st = dalloc(s, &s->warm, 1)) != DT_OK) return fail(st);
  if ((st = dalloc(s, &s->rzpair, 2)) != DT_OK) return fail(st);
  transform_smem_attributes<double>();
  transform_smem_attributes<float>();
  {
    // the TMA stencil takes rasters whose rows are whole tiles; DT_STENCIL_TMA=0 turns it off
    const char* env = getenv("DT_STENCIL_TMA");
    s->tma = w % TBX == 0 && !s->metric && encode_tiled() != nullptr && !(env && env[0] == '0');
    if (s->tma) {
      tma_setup_all<double>();
      tma_setup_all<float>();
    }
  }
  for (int k = 0; k < 2; ++k)
    if (cudaStreamCreateWithFlags(&s->side[k], cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->ev_join[k], cudaEventDisableTiming) != cudaSuccess) {
      set_error("dt_flex_create: side streams");
      return fail(DT_DEVICE_ERROR);
    }
  if (cudaEventCreateWithFlags(&s->ev_fork, cudaEventDisableTiming) != cudaSuccess) {
    set_error("dt_flex_create: events");
    return fail(DT_DEVICE_ERROR);
  }
  if (cudaEventCreate(&s->ev0) != cudaSuccess || cudaEventCreate(&s->ev1) != cudaSuccess) {
    set_error("dt_flex_create: cudaEventCreate failed");
    return fail(DT_DEVICE_ERROR);
  }
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    set_error("dt_flex_create: %s", cudaGetErrorString(e));
    return fail(DT_DEVICE_ERROR);
  }
  *out = s;
  return DT_OK;
}

dt_status dt_flex_set_stream(dt_flex* s, void* stream) {
  if (!s) return DT_BAD_ARG;
  cudaStreamSynchronize(s->stream);
  if (s->own_stream) cudaStreamDestroy(s->stream);
  if (stream) {
    s->stream = (cudaStream_t)stream;
    s->own_stream = false;
  } else {
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) return DT_DEVICE_ERROR;
    s->own_stream = true;
  }
  return DT_OK;
}

// ---- the learned first guess -------------------------------------------------------------------

// Model inputs at the model's cell size: per coarse cell the block means of b and of
// log10(d g); sums of b_coarse^2 and of c (for the normalisations) into sums[0..1].
__global__ void __launch_bounds__(256) k_unet_restrict(int w, int h, int f, const double* __restrict__ d, const double* __restrict__ c,
                                                       const double* __restrict__ b, float* __restrict__ x, double* partials,
                                                       unsigned int* ticket, double* sums) {
  int wc = w / f, hc = h / f;
  size_t nc = (size_t)wc * hc;
  double inv = 1.0 / ((double)f * f);
  Acc<2> acc;
  acc.v[0] = 0.0;
  acc.v[1] = 0.0;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < nc; k += (size_t)gridDim.x * blockDim.x) {
    int ic = (int)(k % wc), jc = (int)(k / wc);
    double sb = 0.0, sl = 0.0, sc = 0.0;
    for (int dj = 0; dj < f; ++dj)
      for (int di = 0; di < f; ++di) {
        size_t q = (size_t)(jc * f + dj) * w + ic * f + di;
        sb += b[q];
        sl += log10(d[q] * 9.81);
        sc += c[q];
      }
    double bc = sb * inv;
    x[2 * k] = (float)bc;
    x[2 * k + 1] = (float)((sl * inv - 22.5) / 1.5);
    acc.v[0] += bc * bc;
    acc.v[1] += sc;
  }
  const int kind[2] = {0, 0};
  if (reduce_partials<2>(acc, kind, partials, ticket, gridDim.x) && threadIdx.x == 0) {
    sums[0] = acc.v[0];
    sums[1] = acc.v[1];
  }
}

__global__ void k_unet_normalise(size_t nc, float* __restrict__ x, const double* sums) {
  double rms = sqrt(sums[0] / (double)nc);
  float inv = rms > 0 ? (float)(1.0 / rms) : 0.f;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < nc; k += (size_t)gridDim.x * blockDim.x) x[2 * k] *= inv;
}

// The prediction back on the raster, in metres: Catmull-Rom cubic interpolation from the coarse
// cells' centres (x wrapping, rows clamping), times rms(b_coarse) / mean(c). The cubic is C1, so
// the guess has no kinks along the coarse cells' edges; the operator weighs curvature, and a
// bilinear prolongation (prolong_linear, flexure.rs:1816-1844) leaves kinks that cost the guess
// much of its energy-norm accuracy.
__device__ __forceinline__ void catmull_rom(double t, double* c) {
  double t2 = t * t, t3 = t2 * t;
  c[0] = 0.5 * (-t3 + 2.0 * t2 - t);
  c[1] = 0.5 * (3.0 * t3 - 5.0 * t2 + 2.0);
  c[2] = 0.5 * (-3.0 * t3 + 4.0 * t2 + t);
  c[3] = 0.5 * (t3 - t2);
}
__global__ void k_unet_prolong(int w, int h, int f, const float* __restrict__ y, double* __restrict__ x, const double* sums) {
  int ws = w / f, hs = h / f;
  size_t n = (size_t)w * h;
  double scale = sqrt(sums[0] / ((double)ws * hs)) / (sums[1] / (double)n);
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    int i = (int)(k % w), j = (int)(k / w);
    double xf = (i + 0.5) / f - 0.5;
    double yf = fmin(fmax((j + 0.5) / f - 0.5, 0.0), (double)(hs - 1));
    double x0 = floor(xf), y0 = floor(yf);
    double cx[4], cy[4];
    catmull_rom(xf - x0, cx);
    catmull_rom(yf - y0, cy);
    int ix = (int)x0, iy = (int)y0;
    double v = 0.0;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      int jj = min(max(iy - 1 + b, 0), hs - 1);
      double row = 0.0;
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        int ii = ((ix - 1 + a) % ws + ws) % ws;
        row += cx[a] * (double)y[(size_t)jj * ws + ii];
      }
      v += cy[b] * row;
    }
    x[k] = v * scale;
  }
}

// x0 of L64 from the model: restrict, normalise, predict on the model's stream, prolong.
static dt_status unet_first_guess(dt_flex* s) {
  cudaStream_t st = s->stream;
  int f = s->unet_f;
  size_t nc = (size_t)(s->w / f) * (s->h / f);
  unsigned int g = std::max(1u, std::min<unsigned int>(ceil_div(nc, 256), (unsigned)s->sms * 8));
  k_unet_restrict<<<g, 256, 0, st>>>(s->w, s->h, f, s->L64.d, s->L64.c, s->b64, s->unet_x, s->partials,
                                     &s->L64.S->ticket[SITE_MISC], s->unet_sums);
  k_unet_normalise<<<g, 256, 0, st>>>(nc, s->unet_x, s->unet_sums);
  counted();
  counted();
  // the model runs on the solve's stream, in order with the kernels around it
  DT_TRY(unet_predict_on(s->unet, st, s->unet_x, s->unet_y, 1, s->h / f, s->w / f));
  k_unet_prolong<<<ew_grid(s), 256, 0, st>>>(s->w, s->h, f, s->unet_y, s->L64.x, s->unet_sums);
  counted();
  DT_CUDA(cudaGetLastError());
  return DT_OK;
}

dt_status dt_flex_set_unet(dt_flex* s, dt_unet* u, double model_dx) {
  if (!s) return DT_BAD_ARG;
  s->unet = nullptr;
  if (!u) return DT_OK;
  double ratio = model_dx / s->dx;
  int f = (int)std::lround(ratio);
  if (!(model_dx > 0.0) || f < 1 || std::fabs(ratio - f) > 1e-9 * ratio || !is_pow2(f) || s->w % f || s->h % f ||
      (s->w / f) % 512 || (s->h / f) % 8) {
    set_error("dt_flex_set_unet: a %d x %d raster of %g m does not coarsen to the model's %g m cells in a shape it takes "
              "(width a multiple of 512, height of 8, by a power of two)", s->w, s->h, s->dx, model_dx);
    return DT_UNSUPPORTED;
  }
  size_t nc = (size_t)(s->w / f) * (s->h / f);
  if (!s->unet_x) {
    DT_TRY(dalloc(s, &s->unet_x, 2 * nc));
    DT_TRY(dalloc(s, &s->unet_y, nc));
    DT_TRY(dalloc(s, &s->unet_sums, 2));
  }
  s->unet = u;
  s->unet_f = f;
  return DT_OK;
}

static dt_status check_params(const dt_flex_params* p) {
  if (!p) {
    set_error("flexure solve: params is NULL");
    return DT_BAD_ARG;
  }
  if (p->precond != DT_PRECOND_REFERENCE && p->precond != DT_PRECOND_MEAN_D) {
    set_error("flexure solve: unknown preconditioner %d", p->precond);
    return DT_BAD_ARG;
  }
  if (p->stop < DT_STOP_MAX_Z || p->stop > DT_STOP_RMS_RESIDUAL || !(p->tol >= 0.0) || p->max_iterations < 0) {
    set_error("flexure solve: bad stopping rule (rule %d, tol %g, max_iterations %d)", p->stop, p->tol, p->max_iterations);
    return DT_BAD_ARG;
  }
  if (p->precision != DT_PREC_FP64 && p->precision != DT_PREC_MIXED && p->precision != DT_PREC_MIXED_RELIABLE) {
    set_error("flexure solve: unknown precision %d", p->precision);
    return DT_BAD_ARG;
  }
  if (p->warm_start != DT_WARM_NONE && p->warm_start != DT_WARM_GIVEN && p->warm_start != DT_WARM_UNET) {
    set_error("flexure solve: unknown warm start %d", p->warm_start);
    return DT_BAD_ARG;
  }
  return DT_OK;
}

// The solve on inputs already in L64.d, L64.c, b64 (and the guess in L64.x).
static dt_status solve_loaded(dt_flex* s, const dt_flex_params* p, dt_report* rep) {
  bool warm = p->warm_start != DT_WARM_NONE;
  long long launches0 = g_launches;
  cudaEventRecord(s->ev0, s->stream);
  if (p->warm_start == DT_WARM_UNET) {
    if (!s->unet) {
      set_error("flexure solve: DT_WARM_UNET without a model (dt_flex_set_unet)");
      return DT_BAD_ARG;
    }
    DT_TRY(unet_first_guess(s));
  }
  dt_status st = p->precision == DT_PREC_MIXED            ? solve_mixed(s, p, warm, rep)
                 : p->precision == DT_PREC_MIXED_RELIABLE ? solve_mixed_reliable(s, p, warm, rep)
                                                          : solve_fp64(s, p, warm, rep);
  if (rep) rep->kernel_launches = g_launches - launches0;
  cudaEventRecord(s->ev1, s->stream);
  cudaError_t e = cudaEventSynchronize(s->ev1);
  if (e != cudaSuccess) {
    set_error("flexure solve: %s", cudaGetErrorString(e));
    return DT_DEVICE_ERROR;
  }
  float ms = 0.f;
  cudaEventElapsedTime(&ms, s->ev0, s->ev1);
  if (rep) rep->device_ms = ms;
  return st;
}

dt_status dt_flex_solve_dev(dt_flex* s, const double* d, const double* c, const double* b, double* x_inout,
                            const dt_flex_params* p, dt_report* rep) {
  if (!s || !d || !c || !b || !x_inout) {
    set_error("dt_flex_solve_dev: NULL argument");
    return DT_BAD_ARG;
  }
  DT_TRY(check_params(p));
  size_t bytes = s->n * sizeof(double);
  DT_CUDA(cudaMemcpyAsync(s->L64.d, d, bytes, cudaMemcpyDeviceToDevice, s->stream));
  DT_CUDA(cudaMemcpyAsync(s->L64.c, c, bytes, cudaMemcpyDeviceToDevice, s->stream));
  DT_CUDA(cudaMemcpyAsync(s->b64, b, bytes, cudaMemcpyDeviceToDevice, s->stream));
  if (p->warm_start == DT_WARM_GIVEN) DT_CUDA(cudaMemcpyAsync(s->L64.x, x_inout, bytes, cudaMemcpyDeviceToDevice, s->stream));
  dt_status st = solve_loaded(s, p, rep);
  if (st == DT_OK || st == DT_NOT_CONVERGED) {
    DT_CUDA(cudaMemcpyAsync(x_inout, s->L64.x, bytes, cudaMemcpyDeviceToDevice, s->stream));
    DT_CUDA(cudaStreamSynchronize(s->stream));
  }
  return st;
}

dt_status dt_flex_solve(dt_flex* s, const double* d, const double* c, const double* b, double* x_inout, const dt_flex_params* p,
                        dt_report* rep) {
  if (!s || !d || !c || !b || !x_inout) {
    set_error("dt_flex_solve: NULL argument");
    return DT_BAD_ARG;
  }
  DT_TRY(check_params(p));
  size_t bytes = s->n * sizeof(double);
  DT_CUDA(cudaMemcpyAsync(s->L64.d, d, bytes, cudaMemcpyHostToDevice, s->stream));
  DT_CUDA(cudaMemcpyAsync(s->L64.c, c, bytes, cudaMemcpyHostToDevice, s->stream));
  DT_CUDA(cudaMemcpyAsync(s->b64, b, bytes, cudaMemcpyHostToDevice, s->stream));
  if (p->warm_start == DT_WARM_GIVEN) DT_CUDA(cudaMemcpyAsync(s->L64.x, x_inout, bytes, cudaMemcpyHostToDevice, s->stream));
  dt_status st = solve_loaded(s, p, rep);
  if (st == DT_OK || st == DT_NOT_CONVERGED) {
    DT_CUDA(cudaMemcpyAsync(x_inout, s->L64.x, bytes, cudaMemcpyDeviceToHost, s->stream));
    DT_CUDA(cudaStreamSynchronize(s->stream));
  }
  return st;
}

static dt_status apply_host(dt_flex* s, int mode, const double* d, const double* c, const double* v, double* y) {
  if (!s || !d || !v || !y || (mode == PLAIN && !c)) {
    set_error("flexure operator: NULL argument");
    return DT_BAD_ARG;
  }
  size_t bytes = s->n * sizeof(double);
  Lane<double>& L = s->L64;
  DT_CUDA(cudaMemcpyAsync(L.d, d, bytes, cudaMemcpyHostToDevice, s->stream));
  if (c) DT_CUDA(cudaMemcpyAsync(L.c, c, bytes, cudaMemcpyHostToDevice, s->stream));
  DT_CUDA(cudaMemcpyAsync(L.p, v, bytes, cudaMemcpyHostToDevice, s->stream));
  launch_apply<double>(s, mode, L.p, nullptr, nullptr, L.d, L.c, nullptr, L.ap, L.S, s->stream);
  DT_CUDA(cudaGetLastError());
  DT_CUDA(cudaMemcpyAsync(y, L.ap, bytes, cudaMemcpyDeviceToHost, s->stream));
  Scalars hs;
  DT_TRY(read_scalars(s, L.S, &hs));
  if (hs.fault) {
    set_error("flexure operator: a kernel's wait for its tile copies ran out");
    return DT_DEVICE_ERROR;
  }
  return DT_OK;
}

dt_status dt_flex_operator(dt_flex* s, const double* d, const double* c, const double* v, double* y) {
  return apply_host(s, PLAIN, d, c, v, y);
}

dt_status dt_flex_bend(dt_flex* s, const double* d, const double* v, double* y) { return apply_host(s, BEND, d, nullptr, v, y); }

dt_status dt_flex_precondition(dt_flex* s, const double* d, const double* c, const double* r, double* z, int precond, int precision) {
  if (!s || !d || !c || !r || !z) {
    set_error("dt_flex_precondition: NULL argument");
    return DT_BAD_ARG;
  }
  size_t bytes = s->n * sizeof(double);
  cudaStream_t st = s->stream;
  Lane<double>& L = s->L64;
  DT_CUDA(cudaMemcpyAsync(L.d, d, bytes, cudaMemcpyHostToDevice, st));
  DT_CUDA(cudaMemcpyAsync(L.c, c, bytes, cudaMemcpyHostToDevice, st));
  DT_CUDA(cudaMemcpyAsync(L.r, r, bytes, cudaMemcpyHostToDevice, st));
  k_put_problem<<<1, 1, 0, st>>>(L.S, HostProblem{0.0, 0, DT_STOP_REL_RESIDUAL, (int)s->n, s->wait_give_up}); counted();
  if (precision == DT_PREC_MIXED) {
    Lane<float>& F = s->L32;
    k_convert<double, float><<<ew_grid(s), 256, 0, st>>>(s->n, L.d, F.d); counted();
    k_convert<double, float><<<ew_grid(s), 256, 0, st>>>(s->n, L.c, F.c); counted();
    k_convert<double, float><<<ew_grid(s), 256, 0, st>>>(s->n, L.r, F.r); counted();
    k_put_problem<<<1, 1, 0, st>>>(F.S, HostProblem{0.0, 0, DT_STOP_REL_RESIDUAL, (int)s->n, s->wait_give_up}); counted();
    int levels;
    DT_TRY(setup_precond<float>(s, F, precond, &levels));
    k_reset<<<1, 1, 0, st>>>(F.S); counted();
    launch_precondition<float>(s, F, F.r, F.z, levels, st);
    k_convert<float, double><<<ew_grid(s), 256, 0, st>>>(s->n, F.z, L.z); counted();
  } else {
    int levels;
    DT_TRY(setup_precond<double>(s, L, precond, &levels));
    k_reset<<<1, 1, 0, st>>>(L.S); counted();
    launch_precondition<double>(s, L, L.r, L.z, levels, st);
  }
  DT_CUDA(cudaGetLastError());
  DT_CUDA(cudaMemcpyAsync(z, L.z, bytes, cudaMemcpyDeviceToHost, st));
  DT_CUDA(cudaStreamSynchronize(st));
  return DT_OK;
}

}  // extern "C"

// =============================================================================================
// Kernel timing for the benchmark's roofline: each hot kernel of one PCG iteration launched
// `reps` times back to back on the handle's stream between two CUDA events, on the handle's
// current data (after a solve). The CG scalars are reset first with alpha = beta = 0, so the
// vector updates leave x, r and p as they are.

namespace dt {

__global__ void k_profile_state(Scalars* S) {
  S->stop = 0;
  S->started = 1;
  S->cond = 0ull;
  S->alpha = 0.0;
  S->beta = 0.0;
  S->rz = 1.0;
  S->it = 0;
  S->max_it = 1 << 30;
  S->rule = DT_STOP_MAX_Z;
  S->tol = -1.0;
}

static const size_t FLUSH_BYTES = (size_t)256 << 20;

template <class T>
static dt_status profile_lane(dt_flex* s, Lane<T>& L, int reps, double* ms, double* bytes) {
  cudaStream_t st = s->stream;
  if (!s->flush) DT_TRY(dalloc(s, &s->flush, FLUSH_BYTES));
  const double e = sizeof(T), n = (double)s->n;
  // algorithmic bytes per launch: each distinct array read once, each output written once
  const double algo[DT_PROFILE_KERNELS] = {
      4 * e * n,  // apply: p, d, c in; Ap out
      6 * e * n,  // update: x, r, p, Ap in; x, r out
      3 * e * n,  // direction: z, p in; p out
      2 * e * n,  // rows forward: r in; half spectrum out (w/2 complex a row = one T a cell)
      2 * e * n,  // columns: half spectrum in and out
      3 * e * n,  // rows inverse (with r.z): half spectrum, r in; z out
      5 * e * n,  // Jacobi left: r, J, d, c in; left out
      6 * e * n,  // Jacobi final: r, J, part, d, c in; z out
      3 * e * n,  // rows forward weighted: left, w in; half out
      7 * e * n,  // rows inverse of the bank: three spectra, three weights in; part out
      2 * e * n,  // columns of one level (the constant-mean-D preconditioner's pass)
  };
  // the bank's column passes and weighted forward row passes as the solve launches them: the
  // three levels in one launch (each level's bytes again) where it does so
  const bool bank1 = s->bank_one_launch && !s->any && !s->row_solve;
  const double bank_levels = bank1 ? 3.0 : 1.0;
  cudaEvent_t a, b;
  DT_CUDA(cudaEventCreate(&a));
  DT_CUDA(cudaEventCreate(&b));
  for (int k = 0; k < DT_PROFILE_KERNELS; ++k) {
    k_profile_state<<<1, 1, 0, st>>>(L.S);
    auto one = [&]() {
      using C = cplx<T>;
      FftGeo g = fft_geometry<T>(s);
      switch (k) {
        case 0: launch_apply<T>(s, AP_DOT, L.p, nullptr, nullptr, L.d, L.c, nullptr, L.ap, L.S, st); break;
        case 1: k_update<T><<<ew_grid(s), 256, 0, st>>>(s->n, L.x, L.r, L.p, L.ap, s->partials, L.S); break;
        case 2: k_direction<T><<<ew_grid(s), 256, 0, st>>>(s->n, L.p, L.z, L.S); break;
        case 3: launch_rows_fwd<T>(s, L, L.r, nullptr, L.half, g, L.S, st); break;
        case 4:
          if (bank1) {
            cols_fn<T>(ilog2(s->h), LogSeq{}, s->cols_fused)<<<dim3(g.cgrid, 3), g.cthreads, g.csmem, st>>>(
                s->N, L.half, L.tab.tw_col, L.tab.omega, L.tab.omega2, L.tab.lx, L.tab.ly, (T)(1.0 / (s->dx * s->dx)), L.S, 0);
            counted();
          } else {
            launch_cols<T>(s, L, L.half, g, 0, L.S, st);
          }
          break;
        case 5: launch_rows_inv<T>(s, L, INV_STORE_DOT, L.half, L.z, nullptr, L.r, g, L.S, st); break;
        case 6: launch_apply<T>(s, JAC_LEFT, nullptr, L.J, nullptr, L.d, L.c, L.r, L.left, L.S, st); break;
        case 7: launch_apply<T>(s, JAC_FINAL, nullptr, L.J, L.part, L.d, L.c, L.r, L.z, L.S, st); break;
        case 8:
          if (bank1) {
            rows_fwd_fn<T, true>(ilog2(s->N), LogSeq{})<<<dim3(g.rgrid, 3), g.rthreads, g.rsmem, st>>>(
                s->w, s->h, L.left, L.wt[0], L.half, L.tab.tw_row, L.tab.post, L.S);
            counted();
          } else {
            launch_rows_fwd<T>(s, L, L.left, L.wt[0], L.half, g, L.S, st);
          }
          break;
        case 9: launch_rows_inv<T>(s, L, INV_BANK, L.half, L.part, L.wt[0], nullptr, g, L.S, st); break;
        case 10: launch_cols<T>(s, L, L.half, g, 0, L.S, st); break;
      }
    };
    one();  // warm
    // each launch timed alone after a write of a buffer twice the L2 (126 MB), so it reads its
    // inputs from HBM as it does inside a solve on a raster larger than L2
    double total = 0.0;
    for (int r = 0; r < reps; ++r) {
      DT_CUDA(cudaMemsetAsync(s->flush, r & 0xff, FLUSH_BYTES, st));
      k_profile_state<<<1, 1, 0, st>>>(L.S);
      DT_CUDA(cudaEventRecord(a, st));
      one();
      DT_CUDA(cudaEventRecord(b, st));
      DT_CUDA(cudaEventSynchronize(b));
      float t = 0.f;
      DT_CUDA(cudaEventElapsedTime(&t, a, b));
      total += t;
    }
    ms[k] = total / reps;
    bytes[k] = algo[k] * (k == 4 || k == 8 ? bank_levels : 1.0);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  DT_CUDA(cudaGetLastError());
  return DT_OK;
}

}  // namespace dt

extern "C" dt_status dt_flex_profile_kernels(dt_flex* s, int precision, int reps, double* ms, double* bytes) {
  if (!s || !ms || !bytes || reps < 1) {
    set_error("dt_flex_profile_kernels: bad argument");
    return DT_BAD_ARG;
  }
  dt_status st = precision == DT_PREC_MIXED ? profile_lane<float>(s, s->L32, reps, ms, bytes)
                                            : profile_lane<double>(s, s->L64, reps, ms, bytes);
  // leave the scalars of a finished solve stopped
  k_reset<<<1, 1, 0, s->stream>>>(precision == DT_PREC_MIXED ? s->L32.S : s->L64.S);
  cudaStreamSynchronize(s->stream);
  return st;
}

// =============================================================================================
// The flexure operator and its energy v.Av with no allocation.
//
// For callers that cannot allocate device memory when they need the operator: a host code that
// has handed the whole device to its own fixed arena, or one that checks a deflection between
// kernels of its own and must not synchronise the device, as cudaMalloc and cudaFree can. The
// call needs no solver handle (dt_flex_create allocates the solver's arrays). The reduction's
// scratch (the solver-state record for the tile kernel, then one partial sum per tile) lives in
// a file-scope device array of fixed size, found once per device with cudaGetSymbolAddress.

namespace dt {

constexpr size_t NOALLOC_STATE_BYTES = (sizeof(Scalars) + 255) / 256 * 256;
constexpr size_t NOALLOC_MAX_TILES = DT_NOALLOC_MAX_TILES;
constexpr size_t NOALLOC_DOUBLES = NOALLOC_STATE_BYTES / sizeof(double) + NOALLOC_MAX_TILES;
static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_DOUBLES];

constexpr int NOALLOC_MAX_DEVICES = 64;
static std::mutex g_noalloc_lock;
static double* g_noalloc_ptr[NOALLOC_MAX_DEVICES] = {};

// The scratch's device address on the current device: looked up on the first call per device and
// kept for the life of the process (a device reset by the caller leaves it stale).
static dt_status noalloc_scratch(double** out) {
  int dev = -1;
  DT_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) {
    set_error("dt_flex_operator_dot_noalloc: device %d beyond the %d this library tracks", dev, NOALLOC_MAX_DEVICES);
    return DT_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> g(g_noalloc_lock);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    cudaError_t rc = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (rc != cudaSuccess || !p) {
      set_error("dt_flex_operator_dot_noalloc: cudaGetSymbolAddress on device %d: %s", dev, cudaGetErrorString(rc));
      return DT_DEVICE_ERROR;
    }
    g_noalloc_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_noalloc_ptr[dev];
  return DT_OK;
}

}  // namespace dt

extern "C" dt_status dt_flex_operator_dot_noalloc(int w, int h, double dx, const double* d, const double* c, const double* v,
                                                  double* y, double* vav, void* stream) {
  if (!d || !c || !v || !y || !vav) {
    set_error("dt_flex_operator_dot_noalloc: NULL argument");
    return DT_BAD_ARG;
  }
  if (w < 1 || h < 1 || !(dx > 0.0) || !std::isfinite(dx)) {
    set_error("dt_flex_operator_dot_noalloc: bad raster %d x %d, dx %g", w, h, dx);
    return DT_BAD_ARG;
  }
  const size_t tile_rows_y = ceil_div((size_t)h, tile_rows<double>());
  if (tile_rows_y > 65535) {  // the grid's y extent carries the rows of tiles
    set_error("dt_flex_operator_dot_noalloc: %d x %d needs %zu rows of tiles of %d cells; a launch takes at most 65535",
              w, h, tile_rows_y, tile_rows<double>());
    return DT_UNSUPPORTED;
  }
  const size_t tiles = (size_t)ceil_div((size_t)w, TBX) * tile_rows_y;
  if (tiles > NOALLOC_MAX_TILES) {
    set_error("dt_flex_operator_dot_noalloc: %d x %d needs %zu tiles of %d x %d cells; the fixed scratch holds %zu",
              w, h, tiles, TBX, tile_rows<double>(), NOALLOC_MAX_TILES);
    return DT_UNSUPPORTED;
  }
  double* scratch = nullptr;
  DT_TRY(noalloc_scratch(&scratch));
  Scalars* S = reinterpret_cast<Scalars*>(scratch);
  double* partials = scratch + NOALLOC_STATE_BYTES / sizeof(double);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // The state record starts at zero every call: no stop flag (the kernel returns at once when one
  // is set, and a zero v sets one), no graph handle, tickets at zero. Partials need no clearing:
  // every tile writes its own before the last tile reads them.
  DT_CUDA(cudaMemsetAsync(S, 0, sizeof(Scalars), st));
  dim3 grid(ceil_div((size_t)w, TBX), ceil_div((size_t)h, tile_rows<double>())), block(TBX, TTY);
  k_apply<double, AP_DOT><<<grid, block, 0, st>>>(w, h, 1.0 / (dx * dx), v, nullptr, nullptr, d, c, nullptr, y, partials, S);
  counted();
  DT_CUDA(cudaGetLastError());
  DT_CUDA(cudaMemcpyAsync(vav, &S->pap, sizeof(double), cudaMemcpyDeviceToDevice, st));
  return DT_OK;
}

// Implicit hillslope/marine diffusion on the B200: (I + dt L_kd) h' = h by conjugate gradients
// preconditioned with one geometric-multigrid V-cycle.
//
// The device implementation behind dt_diff_* (include/deeptime_gpu.h). It solves the system of
// the reference's diffusion::solve with DiffusionSolver::Multigrid (crates/deeptime-core/src/
// surface/diffusion.rs:77-110 and surface/diffusion/multigrid.rs:530-763) with its own kernels:
//
//   k_d_coeffs     the operator (diffusion.rs:532-603): east/south face couplings
//                  0.5 (kd_i + kd_j) dt / dx^2 (x wraps when the raster does; 0 on the last row)
//                  and the diagonal ((((1 + east) + west) + south) + north);
//   k_d_apply      y = A x in the reference's term order (diag, east, wrap, west, wrap, south,
//                  north; diffusion.rs:606-650), fused with p.Ap, b - Ax or the mass sums;
//   multigrid      the levels of multigrid.rs:96-199 (2 x 2 aggregation, coarse couplings SCALE
//                  times the fine faces crossing, mass the sum) built on the device per solve, and
//                  two cycles: the reference's (damped Jacobi, omega 0.8, nu 2, to <= 64 cells,
//                  16 sweeps there; multigrid.rs:243-357, :500-523) and a symmetric multi-colour
//                  Gauss-Seidel V(2,2) to a 16 x 8 coarsest level (colours forward before the
//                  coarse correction, backward after it);
//   CG             multigrid::cg_on's loop (stop on the RMS residual, at most 400 iterations, or
//                  on the relative residual), then the mass put-back so sum x = sum b
//                  (multigrid.rs:736-761).
// The CG loop runs on the device as a CUDA-graph conditional WHILE node, like the flexure solve.
// Precision: FP64 CG with an FP32 cycle (the reference's split), FP64 throughout, or an FP32
// inner CG (FP32 cycle) inside FP64 iterative refinement.
#include <cuda_runtime.h>

#include <algorithm>
#include <type_traits>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "common.cuh"

namespace dt {

enum { DSITE_PAP = 0, DSITE_UPDATE = 1, DSITE_RZ = 2, DSITE_RESID = 3, DSITE_MASS = 4, DSITE_DOT = 5 };
enum { DSTOP_RUNNING = 0, DSTOP_CONVERGED = 1, DSTOP_BREAKDOWN = 2, DSTOP_CAP = 3, DSTOP_NONFINITE = 4 };

struct DScalars {
  double bb, tol;
  int max_it, rule, n;
  double rz, pap, alpha, beta, rr, rz_new;
  int it, stop, body_runs, started;
  double lost, weight, dot_out;
  unsigned long long cond;
  unsigned int ticket[8];
  // reliable updates (DT_DIFF_MIXED_RELIABLE, the FP32 lane): the FP32 residual is replaced by
  // the FP64 one, and x folded into the FP64 accumulation, whenever rr has fallen below
  // delta2 * maxrr or under the tolerance; gate_it == it marks an iteration that does so
  int reliable, gate_it, replacements;
  double delta2, maxrr, rr_true, bb_true;  // rr_true, bb_true: ||b - A x||^2, the reference ||b||^2, unscaled
  unsigned long long cond_if;              // the loop body's IF node around the replacement, 0 without one
};

__device__ __forceinline__ void dset_cond(DScalars* S, unsigned int v) {
  if (S->cond) cudaGraphSetConditional((cudaGraphConditionalHandle)S->cond, v);
}

__device__ __forceinline__ bool d_converged(const DScalars* S, double rr) {
  if (S->rule == DT_STOP_REL_RESIDUAL) return rr <= S->tol * S->tol * S->bb;
  return rr <= S->tol * S->tol * (double)S->n;  // the reference's RMS rule (multigrid.rs:620)
}

// ---------------------------------------------------------------------------------------------
// The operator (diffusion.rs:532-650).

__global__ void k_d_coeffs(int w, int h, int wrap, const double* __restrict__ kd, double dt_over_dx2, double* __restrict__ east,
                           double* __restrict__ south, double* __restrict__ diag, float* __restrict__ east32,
                           float* __restrict__ south32, float* __restrict__ diag32) {
  size_t n = (size_t)w * h;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    int i = (int)(k % w), j = (int)(k / w);
    const double* krow = kd + (size_t)j * w;
    // east face of cell i and of its west neighbour, each as the reference forms it
    auto face_e = [&](int ii) -> double {
      if (ii + 1 < w) return 0.5 * (krow[ii] + krow[ii + 1]) * dt_over_dx2;
      if (wrap) return 0.5 * (krow[ii] + krow[0]) * dt_over_dx2;
      return 0.0;
    };
    auto face_s = [&](int jj) -> double {
      if (jj + 1 < h) return 0.5 * (kd[(size_t)jj * w + i] + kd[(size_t)(jj + 1) * w + i]) * dt_over_dx2;
      return 0.0;
    };
    double e = face_e(i);
    double west = i > 0 ? face_e(i - 1) : (wrap ? face_e(w - 1) : 0.0);
    double s = face_s(j);
    double north = j > 0 ? face_s(j - 1) : 0.0;
    double g = 1.0 + e + west + s + north;
    east[k] = e;
    south[k] = s;
    diag[k] = g;
    east32[k] = (float)e;
    south32[k] = (float)s;
    diag32[k] = (float)g;
  }
}

// y = A x at cell (i, j): diag, east, (wrap), west, (wrap), south, north (diffusion.rs:614-648).
template <class T>
__device__ __forceinline__ T d_apply_at(int w, int h, bool wrap, const T* __restrict__ east, const T* __restrict__ south,
                                        const T* __restrict__ diag, const T* __restrict__ x, int i, int j) {
  size_t c = (size_t)j * w + i, c0 = (size_t)j * w;
  T o = diag[c] * x[c];
  if (i + 1 < w) o -= east[c] * x[c + 1];
  if (wrap && i == w - 1) o -= east[c] * x[c0];
  if (i > 0) o -= east[c - 1] * x[c - 1];
  if (wrap && i == 0) o -= east[c0 + w - 1] * x[c0 + w - 1];
  if (j + 1 < h) o -= south[c] * x[c + w];
  if (j > 0) o -= south[c - w] * x[c - w];
  return o;
}

enum { DA_PAP = 0, DA_RESID = 1, DA_MASS = 2, DA_PLAIN = 3, DA_RESID_GATED = 4 };

// 16 bytes of T, for whole-word loads and stores of a row chunk
template <class T>
struct alignas(16) DV16 {
  T a[16 / sizeof(T)];
};
__device__ __forceinline__ bool d_aligned16(const void* p) { return p == nullptr || (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

// y = A x on the row chunk of V = 16 / sizeof(T) cells i0 .. i0 + V - 1 of row j (V divides w),
// every cell's terms in d_apply_at's order: 16-byte loads of the chunk's diag, east and x and of
// the rows below and above (south, x), one value each for the neighbours across the chunk's ends
// (the row's other end where x wraps). 32-bit offsets: the raster has fewer than 2^31 cells.
template <class T>
__device__ __forceinline__ void d_apply_chunk(int w, int h, bool wrap, const T* __restrict__ east, const T* __restrict__ south,
                                              const T* __restrict__ diag, const T* __restrict__ x, int i0, int j,
                                              DV16<T>& ax, DV16<T>& xv, DV16<T>& dg) {
  constexpr int V = 16 / sizeof(T);
  using W = DV16<T>;
  const int c0 = j * w, c = c0 + i0;
  dg = *reinterpret_cast<const W*>(diag + c);
  xv = *reinterpret_cast<const W*>(x + c);
  const W ea = *reinterpret_cast<const W*>(east + c);
  T xl = (T)0, el = (T)0, xr = (T)0;
  if (i0 > 0) {
    xl = x[c - 1];
    el = east[c - 1];
  } else if (wrap) {
    xl = x[c0 + w - 1];
    el = east[c0 + w - 1];
  }
  if (i0 + V < w)
    xr = x[c + V];
  else if (wrap)
    xr = x[c0];
  W xs = {}, ss = {}, xn = {}, sn = {};
  if (j + 1 < h) {
    xs = *reinterpret_cast<const W*>(x + c + w);
    ss = *reinterpret_cast<const W*>(south + c);
  }
  if (j > 0) {
    xn = *reinterpret_cast<const W*>(x + c - w);
    sn = *reinterpret_cast<const W*>(south + c - w);
  }
#pragma unroll
  for (int e = 0; e < V; ++e) {
    const int i = i0 + e;
    const T xe = e + 1 < V ? xv.a[e + 1] : xr;  // east neighbour; x[c0] across the seam
    const T xw = e > 0 ? xv.a[e - 1] : xl, ew = e > 0 ? ea.a[e - 1] : el;  // west neighbour and its east face
    T o = dg.a[e] * xv.a[e];
    if (i + 1 < w) o -= ea.a[e] * xe;
    if (wrap && i == w - 1) o -= ea.a[e] * xe;
    if (i > 0) o -= ew * xw;
    if (wrap && i == 0) o -= ew * xw;
    if (j + 1 < h) o -= ss.a[e] * xs.a[e];
    if (j > 0) o -= sn.a[e] * xn.a[e];
    ax.a[e] = o;
  }
}

// DA_PAP: y = A x, reduce x.y; DA_RESID: y = b - A x, ym = (TM) y, reduce y.y;
// DA_MASS: reduce sum (b - A x) and sum (diag - 1); DA_PLAIN: y = A x; DA_RESID_GATED: in an
// iteration that replaces the residual (S->gate_it == S->it), y = b - A x and y.y -> S->rr_true.
template <class T, class TM, int MODE>
__global__ void __launch_bounds__(256) k_d_apply(int w, int h, int wrap, const T* __restrict__ east, const T* __restrict__ south,
                                                 const T* __restrict__ diag, const T* __restrict__ x, const T* __restrict__ b,
                                                 T* __restrict__ y, TM* __restrict__ ym, double* partials, DScalars* S) {
  if (MODE == DA_PAP && S->stop) {
    if (blockIdx.x == 0 && threadIdx.x == 0) dset_cond(S, 0);
    return;
  }
  if (MODE == DA_RESID_GATED && (S->stop || S->gate_it != S->it)) return;
  size_t n = (size_t)w * h;
  Acc<2> acc;
  acc.v[0] = 0.0;
  acc.v[1] = 0.0;
  constexpr int V = 16 / sizeof(T);
  if (w % V == 0 && n < ((size_t)1 << 31) && d_aligned16(east) && d_aligned16(south) && d_aligned16(diag) && d_aligned16(x) &&
      d_aligned16(b) && d_aligned16(y)) {
    // whole rows of 16-byte chunks, fewer than 2^31 cells: each thread a chunk at a time
    const unsigned int chunks = (unsigned int)(w / V), nch = chunks * (unsigned int)h;
    for (unsigned int q = blockIdx.x * blockDim.x + threadIdx.x; q < nch; q += gridDim.x * blockDim.x) {
      const int j = (int)(q / chunks), i0 = (int)(q - (unsigned int)j * chunks) * V;
      const int c = j * w + i0;
      DV16<T> ax, xv, dg;
      d_apply_chunk<T>(w, h, wrap != 0, east, south, diag, x, i0, j, ax, xv, dg);
      DV16<T> bv = {};
      if (MODE == DA_RESID || MODE == DA_RESID_GATED || MODE == DA_MASS) bv = *reinterpret_cast<const DV16<T>*>(b + c);
      DV16<T> out;
#pragma unroll
      for (int e = 0; e < V; ++e) {
        const T a = ax.a[e];
        if (MODE == DA_PAP) {
          out.a[e] = a;
          acc.v[0] += (double)xv.a[e] * (double)a;
        } else if (MODE == DA_RESID) {
          const T r = bv.a[e] - a;
          out.a[e] = r;
          ym[c + e] = (TM)r;
          acc.v[0] += (double)r * (double)r;
        } else if (MODE == DA_RESID_GATED) {
          const T r = bv.a[e] - a;
          out.a[e] = r;
          acc.v[0] += (double)r * (double)r;
        } else if (MODE == DA_MASS) {
          acc.v[0] += (double)bv.a[e] - (double)a;
          acc.v[1] += (double)dg.a[e] - 1.0;
        } else {
          out.a[e] = a;
        }
      }
      if (MODE != DA_MASS) *reinterpret_cast<DV16<T>*>(y + c) = out;
    }
  } else {
    // other widths and unaligned arrays: one cell at a time
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
      int i = (int)(k % w), j = (int)(k / w);
      T ax = d_apply_at<T>(w, h, wrap != 0, east, south, diag, x, i, j);
      if (MODE == DA_PAP) {
        y[k] = ax;
        acc.v[0] += (double)x[k] * (double)ax;
      } else if (MODE == DA_RESID) {
        T r = b[k] - ax;
        y[k] = r;
        ym[k] = (TM)r;
        acc.v[0] += (double)r * (double)r;
      } else if (MODE == DA_RESID_GATED) {
        T r = b[k] - ax;
        y[k] = r;
        acc.v[0] += (double)r * (double)r;
      } else if (MODE == DA_MASS) {
        acc.v[0] += (double)b[k] - (double)ax;
        acc.v[1] += (double)diag[k] - 1.0;
      } else {
        y[k] = ax;
      }
    }
  }
  if (MODE == DA_PLAIN) return;
  const int kind[2] = {0, 0};
  int site = MODE == DA_PAP ? DSITE_PAP : (MODE == DA_RESID || MODE == DA_RESID_GATED) ? DSITE_RESID : DSITE_MASS;
  if (reduce_partials<2>(acc, kind, partials, &S->ticket[site], gridDim.x) && threadIdx.x == 0) {
    if (MODE == DA_PAP) {
      S->pap = acc.v[0];
      if (!(acc.v[0] > 0.0) || !isfinite(acc.v[0])) {
        S->stop = isfinite(acc.v[0]) ? DSTOP_BREAKDOWN : DSTOP_NONFINITE;
        dset_cond(S, 0);
      } else {
        S->alpha = S->rz / acc.v[0];
      }
    } else if (MODE == DA_RESID) {
      S->rr = acc.v[0];
    } else if (MODE == DA_RESID_GATED) {
      S->rr_true = acc.v[0];
    } else {
      S->lost = acc.v[0];
      S->weight = acc.v[1];
    }
  }
}

// x += alpha p; r -= alpha Ap; rm = (TM) r; reduce r.r and test the stopping rule.
template <class T, class TM>
__global__ void __launch_bounds__(256) k_d_update(size_t n, T* __restrict__ x, T* __restrict__ r, TM* __restrict__ rm,
                                                  const T* __restrict__ p, const T* __restrict__ ap, double* partials, DScalars* S) {
  if (S->stop) {
    if (blockIdx.x == 0 && threadIdx.x == 0) dset_cond(S, 0);
    return;
  }
  T alpha = (T)S->alpha;
  Acc<1> acc;
  acc.v[0] = 0.0;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    x[k] += alpha * p[k];
    T rv = r[k] - alpha * ap[k];
    r[k] = rv;
    rm[k] = (TM)rv;
    acc.v[0] += (double)rv * (double)rv;
  }
  const int kind[1] = {0};
  if (reduce_partials<1>(acc, kind, partials, &S->ticket[DSITE_UPDATE], gridDim.x) && threadIdx.x == 0) {
    double rr = acc.v[0];
    S->rr = rr;
    S->it += 1;
    if (S->reliable) {
      // the FP32 residual only asks for a replacement; the FP64 residual decides convergence
      bool gate = false;
      if (!isfinite(rr)) {
        S->stop = DSTOP_NONFINITE;
      } else if (rr <= S->tol * S->tol * S->bb || rr < S->delta2 * S->maxrr) {
        S->gate_it = S->it;
        gate = true;
      } else if (S->it >= S->max_it) {
        S->stop = DSTOP_CAP;
      }
      if (S->cond_if) cudaGraphSetConditional((cudaGraphConditionalHandle)S->cond_if, gate ? 1u : 0u);
      if (S->stop) dset_cond(S, 0);
      return;
    }
    if (!isfinite(rr))
      S->stop = DSTOP_NONFINITE;
    else if (d_converged(S, rr))
      S->stop = DSTOP_CONVERGED;
    else if (S->it >= S->max_it)
      S->stop = DSTOP_CAP;
    if (S->stop) dset_cond(S, 0);
  }
}

// rz = r . z after the cycle; beta = rz / rz_old (multigrid.rs:721-727).
template <class T, class TM>
__global__ void __launch_bounds__(256) k_d_rz(size_t n, const T* __restrict__ r, const TM* __restrict__ z, double* partials,
                                              DScalars* S) {
  if (S->stop) return;
  Acc<1> acc;
  acc.v[0] = 0.0;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
    acc.v[0] += (double)r[k] * (double)z[k];
  const int kind[1] = {0};
  if (reduce_partials<1>(acc, kind, partials, &S->ticket[DSITE_RZ], gridDim.x) && threadIdx.x == 0) {
    double rz = acc.v[0];
    if (!S->started) {
      S->started = 1;
      S->rz = rz;
      if (!isfinite(rz)) S->stop = DSTOP_NONFINITE;
      return;
    }
    if (!(isfinite(rz) && S->rz > 0.0)) {
      S->stop = isfinite(rz) ? DSTOP_BREAKDOWN : DSTOP_NONFINITE;
      dset_cond(S, 0);
      return;
    }
    S->beta = rz / S->rz;
    S->rz = rz;
  }
}

// p = z + beta p (p = z on the first direction), and the loop guard.
template <class T, class TM>
__global__ void __launch_bounds__(256) k_d_direction(size_t n, T* __restrict__ p, const TM* __restrict__ z, DScalars* S, int first) {
  if (!first && blockIdx.x == 0 && threadIdx.x == 0) {
    int runs = ++S->body_runs;
    bool again = S->stop == 0 && runs < S->max_it + 2;
    if (!again && S->stop == 0) S->stop = DSTOP_CAP;
    dset_cond(S, again ? 1u : 0u);
  }
  if (S->stop) return;
  T beta = first ? (T)0 : (T)S->beta;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
    p[k] = first ? (T)z[k] : (T)z[k] + beta * p[k];
}

// ---------------------------------------------------------------------------------------------
// The multigrid levels (multigrid.rs:96-199).

template <class TM>
struct DLevel {
  int w, h, wrap;
  TM *east, *south, *diag, *wd, *mass, *r, *z, *t;
};

template <class TM>
__global__ void k_mg_finest(size_t n, const double* __restrict__ e, const double* __restrict__ s, const double* __restrict__ g,
                            TM omega, TM* __restrict__ east, TM* __restrict__ south, TM* __restrict__ diag, TM* __restrict__ wd,
                            TM* __restrict__ mass) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    east[k] = (TM)e[k];
    south[k] = (TM)s[k];
    TM gg = (TM)g[k];
    diag[k] = gg;
    wd[k] = omega / gg;
    mass[k] = (TM)1;
  }
}

// Coarse mass and faces: mass = sum of the 2 x 2 block's; east = SCALE * the fine east faces
// leaving its last column (wrapping), south = SCALE * the fine south faces of its last row.
template <class TM>
__global__ void k_mg_coarsen(DLevel<TM> f, DLevel<TM> c, TM scale) {
  size_t nc = (size_t)c.w * c.h;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < nc; k += (size_t)gridDim.x * blockDim.x) {
    int ic = (int)(k % c.w), jc = (int)(k / c.w);
    int r0 = 2 * jc, r1 = min(2 * jc + 2, f.h), c0 = 2 * ic, c1 = min(2 * ic + 2, f.w);
    int last_row = r1 - 1, last_col = c1 - 1;
    TM m = 0;
    for (int j = r0; j < r1; ++j)
      for (int i = c0; i < c1; ++i) m += f.mass[(size_t)j * f.w + i];
    c.mass[k] = m;
    TM e = 0;
    if (ic + 1 < c.w || c.wrap) {
      for (int j = r0; j < r1; ++j) e += f.east[(size_t)j * f.w + last_col];
      e = scale * e;
    }
    c.east[k] = e;
    TM s = 0;
    if (jc + 1 < c.h) {
      for (int i = c0; i < c1; ++i) s += f.south[(size_t)last_row * f.w + i];
      s = scale * s;
    }
    c.south[k] = s;
  }
}

template <class TM>
__global__ void k_mg_diag(DLevel<TM> c, TM omega) {
  size_t nc = (size_t)c.w * c.h;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < nc; k += (size_t)gridDim.x * blockDim.x) {
    int i = (int)(k % c.w), j = (int)(k / c.w);
    size_t c0 = (size_t)j * c.w;
    TM west = i > 0 ? c.east[k - 1] : (c.wrap ? c.east[c0 + c.w - 1] : (TM)0);
    TM north = j > 0 ? c.south[k - c.w] : (TM)0;
    TM g = c.mass[k] + c.east[k] + west + c.south[k] + north;
    c.diag[k] = g;
    c.wd[k] = omega / g;
  }
}

// Products rounded on their own (never fused into an add): the cycle's kernels form the same
// values whichever kernel runs them, as the reference forms them (no fused multiply-adds).
__device__ __forceinline__ float mulr(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mulr(double a, double b) { return __dmul_rn(a, b); }

// A z at a cell of a level, in the level's term order (multigrid.rs:202-240), reading z (+ the
// coarse correction of each cell's parent when zc is given).
template <class TM>
__device__ __forceinline__ TM mg_apply_at(const DLevel<TM>& L, const TM* __restrict__ z, const TM* __restrict__ zc, int wc, int i,
                                          int j) {
  auto zat = [&](int ii, int jj) -> TM {
    TM v = z[(size_t)jj * L.w + ii];
    if (zc) v += zc[(size_t)(jj / 2) * wc + ii / 2];
    return v;
  };
  size_t c = (size_t)j * L.w + i, c0 = (size_t)j * L.w;
  TM o = mulr(L.diag[c], zat(i, j));
  if (i + 1 < L.w) o -= mulr(L.east[c], zat(i + 1, j));
  if (i > 0) o -= mulr(L.east[c - 1], zat(i - 1, j));
  if (L.wrap) {
    if (i == L.w - 1) o -= mulr(L.east[c], zat(0, j));
    if (i == 0) o -= mulr(L.east[c0 + L.w - 1], zat(L.w - 1, j));
  }
  if (j + 1 < L.h) o -= mulr(L.south[c], zat(i, j + 1));
  if (j > 0) o -= mulr(L.south[c - L.w], zat(i, j - 1));
  return o;
}

// z = wd r (the first sweep from z = 0)
template <class TM>
__global__ void k_mg_first(DLevel<TM> L, TM* __restrict__ z) {
  size_t n = (size_t)L.w * L.h;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) z[k] = L.wd[k] * L.r[k];
}

// zout = z' + wd (r - A z'), z' = zin (+ the coarse correction)
template <class TM>
__global__ void k_mg_sweep(DLevel<TM> L, const TM* __restrict__ zin, TM* __restrict__ zout, const TM* __restrict__ zc, int wc) {
  size_t n = (size_t)L.w * L.h;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    int i = (int)(k % L.w), j = (int)(k / L.w);
    TM zk = zin[k];
    if (zc) zk += zc[(size_t)(j / 2) * wc + i / 2];
    TM az = mg_apply_at<TM>(L, zin, zc, wc, i, j);
    zout[k] = zk + L.wd[k] * (L.r[k] - az);
  }
}

// rc = sum over each 2 x 2 block of (r - A z) (multigrid.rs:332-356)
template <class TM, class K>
__device__ __forceinline__ void restrict_cell(const DLevel<TM>& L, const TM* __restrict__ z, const DLevel<TM>& C, K k) {
  int ic = (int)(k % C.w), jc = (int)(k / C.w);
  TM acc = 0;
  for (int j = 2 * jc; j < min(2 * jc + 2, L.h); ++j)
    for (int i = 2 * ic; i < min(2 * ic + 2, L.w); ++i) acc += L.r[(size_t)j * L.w + i] - mg_apply_at<TM>(L, z, nullptr, 0, i, j);
  C.r[k] = acc;
}
template <class TM>
__global__ void k_mg_restrict(DLevel<TM> L, const TM* __restrict__ z, DLevel<TM> C) {
  size_t nc = (size_t)C.w * C.h;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < nc; k += (size_t)gridDim.x * blockDim.x)
    restrict_cell<TM>(L, z, C, k);
}

// The colour of a cell for the Gauss-Seidel sweeps: (i + j) % 2, and on a wrapping level of odd
// width the last column takes two colours of its own (2 + j % 2), since a ring of odd length has
// no two-colouring. No two cells of one colour are neighbours.
__device__ __forceinline__ int gs_colour(int w, int wrap, int i, int j) {
  if (wrap && (w & 1) && i == w - 1) return 2 + (j & 1);
  return (i + j) & 1;
}
inline int gs_colours(int w, int wrap) { return (wrap && (w & 1)) ? 4 : 2; }

// One Gauss-Seidel update of cell k = (i, j) of colour `colour`: z_c += (r - A z)_c / diag_c.
// FIRST: z is taken as 0 where this sweep has not written (the cycle's first sweep).
template <class TM, bool FIRST>
__device__ __forceinline__ void gs_cell_at(const DLevel<TM>& L, TM* __restrict__ z, int colour, size_t k, int i, int j) {
  // in the first forward sweep, cells of later colours still hold 0 (not yet written)
  auto zat = [&](int ii, int jj) -> TM {
    if (FIRST && gs_colour(L.w, L.wrap, ii, jj) >= colour) return (TM)0;
    return z[(size_t)jj * L.w + ii];
  };
  size_t c = k, c0 = (size_t)j * L.w;
  TM zk = FIRST ? (TM)0 : z[c];
  TM o = mulr(L.diag[c], zk);
  if (i + 1 < L.w) o -= mulr(L.east[c], zat(i + 1, j));
  if (i > 0) o -= mulr(L.east[c - 1], zat(i - 1, j));
  if (L.wrap) {
    if (i == L.w - 1) o -= mulr(L.east[c], zat(0, j));
    if (i == 0) o -= mulr(L.east[c0 + L.w - 1], zat(L.w - 1, j));
  }
  if (j + 1 < L.h) o -= mulr(L.south[c], zat(i, j + 1));
  if (j > 0) o -= mulr(L.south[c - L.w], zat(i, j - 1));
  z[c] = zk + mulr(L.r[c] - o, L.wd[c]);  // wd = 1 / diag on the Gauss-Seidel hierarchy
}
template <class TM, bool FIRST>
__device__ __forceinline__ void gs_cell(const DLevel<TM>& L, TM* __restrict__ z, int colour, size_t k) {
  gs_cell_at<TM, FIRST>(L, z, colour, k, (int)(k % L.w), (int)(k / L.w));
}

// One Gauss-Seidel pass over the cells of colour `colour`.
template <class TM, bool FIRST>
__global__ void k_mg_gs(DLevel<TM> L, TM* __restrict__ z, int colour) {
  size_t n = (size_t)L.w * L.h;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    int i = (int)(k % L.w), j = (int)(k / L.w);
    if (gs_colour(L.w, L.wrap, i, j) != colour) continue;
    gs_cell<TM, FIRST>(L, z, colour, k);
  }
}

// z += P zc (piecewise constant)
template <class TM>
__global__ void k_mg_prolong(DLevel<TM> L, TM* __restrict__ z, const TM* __restrict__ zc, int wc) {
  size_t n = (size_t)L.w * L.h;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    int i = (int)(k % L.w), j = (int)(k / L.w);
    z[k] += zc[(size_t)(j / 2) * wc + i / 2];
  }
}

// The coarsest level in one block (at most 128 cells): KIND 0 the reference's first sweep and
// 15 damped Jacobi sweeps (multigrid.rs:504-512); KIND 1 eight forward and eight backward
// multi-colour Gauss-Seidel sweeps. Result in z. Every thread of the block takes part.
template <class TM, int KIND>
__device__ __forceinline__ void coarsest_solve(const DLevel<TM>& L, TM* __restrict__ z, int sweeps) {
  __shared__ TM sz[2][256];
  int n = L.w * L.h;
  int k = threadIdx.x;
  if (KIND == 0) {
    if (k < n) sz[0][k] = L.wd[k] * L.r[k];
    __syncthreads();
    int cur = 0;
    for (int s = 1; s < sweeps; ++s) {
      if (k < n) {
        int i = k % L.w, j = k / L.w;
        TM az = mg_apply_at<TM>(L, sz[cur], nullptr, 0, i, j);
        sz[cur ^ 1][k] = sz[cur][k] + L.wd[k] * (L.r[k] - az);
      }
      __syncthreads();
      cur ^= 1;
    }
    if (k < n) z[k] = sz[cur][k];
  } else {
    if (k < n) sz[0][k] = (TM)0;
    __syncthreads();
    int ncol = (L.wrap && (L.w & 1)) ? 4 : 2;
    for (int pass = 0; pass < 2 * sweeps; ++pass) {
      bool forward = pass < sweeps;
      for (int q = 0; q < ncol; ++q) {
        int colour = forward ? q : ncol - 1 - q;
        if (k < n) {
          int i = k % L.w, j = k / L.w;
          if (gs_colour(L.w, L.wrap, i, j) == colour) {
            TM az = mg_apply_at<TM>(L, sz[0], nullptr, 0, i, j);
            sz[0][k] = sz[0][k] + mulr(L.r[k] - az, L.wd[k]);
          }
        }
        __syncthreads();
      }
    }
    if (k < n) z[k] = sz[0][k];
  }
}
template <class TM, int KIND>
__global__ void k_mg_coarsest(DLevel<TM> L, TM* __restrict__ z, int sweeps) {
  coarsest_solve<TM, KIND>(L, z, sweeps);
}

// The Gauss-Seidel V-cycle's part from a level of at most MG_BLOCK_CELLS cells down, in one
// block of 1024 threads (the coarsest level on the first 128): the same passes in the same order as the separate launches (pre-sweeps,
// restriction, the coarser levels, prolongation, post-sweeps), a block barrier where a launch
// ended, so the same values. The levels' arrays are staged in shared memory first (off[q]: the
// level's first cell there, six arrays of `total` cells); the top level's z goes back at the end.
constexpr int MG_BLOCK_LEVELS = 8;
template <class TM>
struct MgChain {
  DLevel<TM> lv[MG_BLOCK_LEVELS];
  int off[MG_BLOCK_LEVELS];
  int count, total;
};
template <class TM>
__global__ void __launch_bounds__(1024) k_mg_coarse_rb(MgChain<TM> g, int nu, int coarse_sweeps) {
  const int tid = threadIdx.x, nt = blockDim.x;
  extern __shared__ __align__(16) unsigned char mg_chain_smem[];
  TM* const sbase = reinterpret_cast<TM*>(mg_chain_smem);
  // level q as staged in shared memory (built in registers where it is used)
  auto sl = [&](int q) {
    DLevel<TM> L = g.lv[q];
    L.z = sbase + 0 * g.total + g.off[q];
    L.r = sbase + 1 * g.total + g.off[q];
    L.diag = sbase + 2 * g.total + g.off[q];
    L.wd = sbase + 3 * g.total + g.off[q];
    L.east = sbase + 4 * g.total + g.off[q];
    L.south = sbase + 5 * g.total + g.off[q];
    return L;
  };
  for (int q = 0; q < g.count; ++q) {
    const DLevel<TM> L = sl(q);
    const DLevel<TM>& G = g.lv[q];
    const int n = G.w * G.h;
    for (int k = tid; k < n; k += nt) {
      L.z[k] = (TM)0;
      L.r[k] = q == 0 ? G.r[k] : (TM)0;
      L.diag[k] = G.diag[k];
      L.wd[k] = G.wd[k];
      L.east[k] = G.east[k];
      L.south[k] = G.south[k];
    }
  }
  __syncthreads();
  for (int q = 0; q + 1 < g.count; ++q) {
    const DLevel<TM> L = sl(q);
    const int n = L.w * L.h;
    const int ncol = (L.wrap && (L.w & 1)) ? 4 : 2;
    for (int sweep = 0; sweep < nu; ++sweep)
      for (int c = 0; c < ncol; ++c) {
        for (int k = tid; k < n; k += nt) {
          const int j = k / L.w, i = k - j * L.w;
          if (gs_colour(L.w, L.wrap, i, j) != c) continue;
          if (sweep == 0)
            gs_cell_at<TM, true>(L, L.z, c, k, i, j);
          else
            gs_cell_at<TM, false>(L, L.z, c, k, i, j);
        }
        __syncthreads();
      }
    const DLevel<TM> C = sl(q + 1);
    for (int k = tid; k < C.w * C.h; k += nt) restrict_cell<TM>(L, L.z, C, k);
    __syncthreads();
  }
  {
    // the coarsest level (at most 128 cells, one a thread) on the block's first 128 threads:
    // coarsest_solve's Gauss-Seidel passes in place on the staged z, with a barrier of those
    // threads between passes
    const DLevel<TM> L = sl(g.count - 1);
    if (tid < 128) {
      const int n = L.w * L.h;
      const int ncol = (L.wrap && (L.w & 1)) ? 4 : 2;
      const int j = tid / L.w, i = tid - j * L.w;
      for (int pass = 0; pass < 2 * coarse_sweeps; ++pass) {
        const bool forward = pass < coarse_sweeps;
        for (int q = 0; q < ncol; ++q) {
          const int colour = forward ? q : ncol - 1 - q;
          if (tid < n && gs_colour(L.w, L.wrap, i, j) == colour) {
            TM az = mg_apply_at<TM>(L, L.z, nullptr, 0, i, j);
            L.z[tid] = L.z[tid] + mulr(L.r[tid] - az, L.wd[tid]);
          }
          asm volatile("bar.sync 1, 128;" ::: "memory");
        }
      }
    }
    __syncthreads();
  }
  for (int q = g.count - 2; q >= 0; --q) {
    const DLevel<TM> L = sl(q), C = sl(q + 1);
    const int n = L.w * L.h;
    const int ncol = (L.wrap && (L.w & 1)) ? 4 : 2;
    for (int k = tid; k < n; k += nt) {
      const int j = k / L.w, i = k - j * L.w;
      L.z[k] += C.z[(j / 2) * C.w + i / 2];
    }
    __syncthreads();
    for (int sweep = 0; sweep < nu; ++sweep)
      for (int c = ncol - 1; c >= 0; --c) {
        for (int k = tid; k < n; k += nt) {
          const int j = k / L.w, i = k - j * L.w;
          if (gs_colour(L.w, L.wrap, i, j) != c) continue;
          gs_cell_at<TM, false>(L, L.z, c, k, i, j);
        }
        __syncthreads();
      }
  }
  {
    const DLevel<TM> L = sl(0);
    for (int k = tid; k < L.w * L.h; k += nt) g.lv[0].z[k] = L.z[k];
  }
}

// Two red-black Gauss-Seidel sweeps (four colour passes) of a level in one launch, over tiles of
// TX x TY cells staged in shared memory with a halo: pass p updates its colour on the tile and
// the rings around it that the later passes read, so the tile's cells end with the values four
// separate passes give (temporal blocking; each update is gs_cell's, term for term).
//   PRE   the pre-smoothing: z from 0, colours 0, 1, 0, 1; then the residual r - A z of each
//         of the tile's cells (mg_apply_at's order) and its 2 x 2 sums, in k_mg_restrict's
//         order, into the coarser level's r, so the restriction needs no launch of its own
//         (halo 5: z is final one ring out);
//   !PRE  the post-smoothing: z += P zc (the coarse correction, piecewise constant), then
//         colours 1, 0, 1, 0 (halo 4). It reads z around its tile, which neighbouring tiles
//         finish at the same time, so it writes its result to another buffer (zout = L.t; PRE,
//         which reads no z, writes L.z).
// For levels of two colours (no wrap, or an even width) at least TX + 10 cells wide, so that no
// cell sits twice in a tile, and of fewer than 2^31 cells (32-bit offsets). Shared memory holds
// the region in red-black order, so that a colour pass reads and writes consecutive words with
// no idle lanes. A tile whose region lies inside the raster (most tiles) stages and updates
// without the bounds and seam tests, whose outcome is known there: every neighbour exists and
// none lies across the seam.
// Tiles: 32 x 16 cells and 256 threads; FP32 levels of many tiles take 64 x 32 cells and 512
// threads, which cuts the halo's staged cells per tile cell from 2.1 to 1.5 and its updates
// from 3.1 to 2.5.
constexpr int MG_TX = 32, MG_TY = 16, MG_BTX = 64, MG_BTY = 32;
// One value from global into shared memory by an asynchronous copy (completes at the block's
// cp.async.wait_all).
__device__ __forceinline__ void rb2_cp_async(float* dst, const float* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void rb2_cp_async(double* dst, const double* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src) : "memory");
}
template <class TM, bool PRE, int TX, int TY, int NT>
__global__ void __launch_bounds__(NT) k_mg_rb2(DLevel<TM> L, DLevel<TM> C, const TM* __restrict__ zc, TM* __restrict__ zout) {
  constexpr int HALO = PRE ? 5 : 4;
  constexpr int SX = TX + 2 * HALO, SY = TY + 2 * HALO;
  constexpr int HX = SX / 2, NC = HX * SY;  // a colour's cells of a row, of the region
  static_assert(SX % 2 == 0 && 2 * NC >= TX * TY, "rb2: even rows");
  // red-black layout: cell (lx, ly) of colour k = (i0 + lx + j0 + ly) & 1 at a[k][ly * HX + lx / 2]
  extern __shared__ __align__(16) unsigned char mg_smem[];
  TM* const base = reinterpret_cast<TM*>(mg_smem);
  // array a (0 z, 1 r, 2 diag, 3 wd, 4 east, 5 south) of colour k
  auto A = [&](int a, int k) { return base + (2 * a + k) * NC; };
  const int i0 = blockIdx.x * TX - HALO, j0 = blockIdx.y * TY - HALO;
  const int off = (i0 + j0) & 1;
  const int tid = threadIdx.x;
  const int w = L.w, h = L.h;
  const bool inner = i0 >= 0 && j0 >= 0 && i0 + SX <= w && j0 + SY <= h;
  auto gcol = [&](int lx) {
    int gi = i0 + lx;
    if (L.wrap) gi = gi < 0 ? gi + w : (gi >= w ? gi - w : gi);
    return gi;
  };
  // staging by asynchronous copies into the colour arrays, so that all of a thread's copies are
  // in flight at once (a load into registers and a store per value would wait out each load
  // in turn); the post-smoothing then adds the coarse correction to its own staged z values
  auto stage = [&](int lx, int ly, int gi, int gj) {
    const int k = (lx + ly + off) & 1, q = ly * HX + (lx >> 1);
    const int c = gj * w + gi;
    if (PRE)
      A(0, k)[q] = (TM)0;
    else
      rb2_cp_async(A(0, k) + q, L.z + c);
    rb2_cp_async(A(1, k) + q, L.r + c);
    rb2_cp_async(A(2, k) + q, L.diag + c);
    rb2_cp_async(A(3, k) + q, L.wd + c);
    rb2_cp_async(A(4, k) + q, L.east + c);
    rb2_cp_async(A(5, k) + q, L.south + c);
  };
  if (inner) {
    for (int e = tid; e < SX * SY; e += NT) {
      const int ly = e / SX, lx = e - ly * SX;
      stage(lx, ly, i0 + lx, j0 + ly);
    }
  } else {
    for (int e = tid; e < SX * SY; e += NT) {
      const int ly = e / SX, lx = e - ly * SX;
      const int gi = gcol(lx), gj = j0 + ly;
      if (gj < 0 || gj >= h || gi < 0 || gi >= w) continue;
      stage(lx, ly, gi, gj);
    }
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  if (!PRE) {
    // z = z + zc (P zc piecewise constant), each thread on the cells it staged
#pragma unroll 4
    for (int e = tid; e < SX * SY; e += NT) {
      const int ly = e / SX, lx = e - ly * SX;
      const int gi = inner ? i0 + lx : gcol(lx), gj = j0 + ly;
      if (!inner && (gj < 0 || gj >= h || gi < 0 || gi >= w)) continue;
      A(0, (lx + ly + off) & 1)[ly * HX + (lx >> 1)] += zc[(gj >> 1) * C.w + (gi >> 1)];
    }
  }
  __syncthreads();
  // pass p updates its colour at least p + 1 cells from the region's border: a row's cells of
  // one colour are consecutive, so consecutive threads take consecutive cells
#pragma unroll
  for (int pass = 0; pass < 4; ++pass) {
    const int k = PRE ? (pass & 1) : 1 - (pass & 1), o_ = 1 - k;
    const int lo = pass + 1, RW = SX - 2 * lo, RH = SY - 2 * lo, HW = RW / 2;
    TM* const zs = A(0, k);
    const TM* const zo = A(0, o_);
    const TM *const rk = A(1, k), *const dk = A(2, k), *const wk = A(3, k);
    const TM *const ek = A(4, k), *const eo = A(4, o_), *const sk = A(5, k), *const so = A(5, o_);
    for (int idx = tid; idx < RH * HW; idx += NT) {
      const int ly = lo + idx / HW;
      const int p = (k + ly + off) & 1;  // the parity of lx of colour k on this row
      const int lx = lo + ((p - lo) & 1) + 2 * (idx - (ly - lo) * HW);
      const int q = ly * HX + (lx >> 1);
      const int qw = ly * HX + ((lx - 1) >> 1), qe = ly * HX + ((lx + 1) >> 1);  // the other colour's
      const TM zk = zs[q];
      TM o = mulr(dk[q], zk);
      if (inner) {
        o -= mulr(ek[q], zo[qe]);
        o -= mulr(eo[qw], zo[qw]);
        o -= mulr(sk[q], zo[q + HX]);
        o -= mulr(so[q - HX], zo[q - HX]);
      } else {
        const int gi = gcol(lx), gj = j0 + ly;
        if (gj < 0 || gj >= h || gi < 0 || gi >= w) continue;
        if (gi + 1 < w) o -= mulr(ek[q], zo[qe]);
        if (gi > 0) o -= mulr(eo[qw], zo[qw]);
        if (L.wrap) {
          if (gi == w - 1) o -= mulr(ek[q], zo[qe]);
          if (gi == 0) o -= mulr(eo[qw], zo[qw]);
        }
        if (gj + 1 < h) o -= mulr(sk[q], zo[q + HX]);
        if (gj > 0) o -= mulr(so[q - HX], zo[q - HX]);
      }
      zs[q] = zk + mulr(rk[q] - o, wk[q]);
    }
    __syncthreads();
  }
  auto at = [&](int a, int lx, int ly) -> TM { return A(a, (lx + ly + off) & 1)[ly * HX + (lx >> 1)]; };
  if (PRE) {
    // the residual of each of the tile's cells, in mg_apply_at's order, into the slots of 1/diag
    // (no longer read); then each coarse cell's 2 x 2 sum in k_mg_restrict's order
    TM* const res = A(3, 0);
    for (int e = tid; e < TX * TY; e += NT) {
      const int lx = HALO + e % TX, ly = HALO + e / TX;
      const int i = i0 + lx, j = j0 + ly;
      if (i >= w || j >= h) continue;
      TM o = mulr(at(2, lx, ly), at(0, lx, ly));
      if (i + 1 < w) o -= mulr(at(4, lx, ly), at(0, lx + 1, ly));
      if (i > 0) o -= mulr(at(4, lx - 1, ly), at(0, lx - 1, ly));
      if (L.wrap) {
        if (i == w - 1) o -= mulr(at(4, lx, ly), at(0, lx + 1, ly));
        if (i == 0) o -= mulr(at(4, lx - 1, ly), at(0, lx - 1, ly));
      }
      if (j + 1 < h) o -= mulr(at(5, lx, ly), at(0, lx, ly + 1));
      if (j > 0) o -= mulr(at(5, lx, ly - 1), at(0, lx, ly - 1));
      res[e] = at(1, lx, ly) - o;
    }
    __syncthreads();
    constexpr int CX = TX / 2, CY = TY / 2;
    for (int t = tid; t < CX * CY; t += NT) {
      const int ic = blockIdx.x * CX + t % CX, jc = blockIdx.y * CY + t / CX;
      if (ic >= C.w || jc >= C.h) continue;
      TM acc = 0;
      for (int j = 2 * jc; j < min(2 * jc + 2, h); ++j)
        for (int i = 2 * ic; i < min(2 * ic + 2, w); ++i) acc += res[(j - j0 - HALO) * TX + (i - i0 - HALO)];
      C.r[jc * C.w + ic] = acc;
    }
  }
  for (int e = tid; e < TX * TY; e += NT) {
    const int ly = HALO + e / TX, lx = HALO + e % TX;
    const int gi = i0 + lx, gj = j0 + ly;
    if (gi < w && gj < h) zout[gj * w + gi] = at(0, lx, ly);
  }
}
template <class TM, bool PRE, int TX = MG_TX, int TY = MG_TY>
constexpr size_t mg_rb2_smem() {
  return (size_t)6 * (TX + 2 * (PRE ? 5 : 4)) * (TY + 2 * (PRE ? 5 : 4)) * sizeof(TM);
}

// ---------------------------------------------------------------------------------------------
// LOD first guess (diffusion.rs:370-489): an implicit sweep along x per row (cyclic tridiagonal,
// Sherman-Morrison, :1050-1071) and then along y per column (Thomas, :1029-1046). One thread
// per row or column; scratch arrays of the raster's size.

__device__ void thomas_strided(int n, const double* lo, const double* di, const double* up, double* b, double* c, size_t stride,
                               size_t base) {
  // lo/di/up/b/c accessed at base + i * stride
  if (n == 0) return;
  double beta = di[base];
  b[base] /= beta;
  for (int i = 1; i < n; ++i) {
    size_t at = base + (size_t)i * stride, prev = at - stride;
    c[at] = up[prev] / beta;
    beta = di[at] - lo[at] * c[at];
    b[at] = (b[at] - lo[at] * b[prev]) / beta;
  }
  for (int i = n - 2; i >= 0; --i) {
    size_t at = base + (size_t)i * stride;
    double next = b[at + stride];
    b[at] -= c[at + stride] * next;
  }
}

__global__ void k_lod_rows(int w, int h, int wrap, double* __restrict__ hf, const double* __restrict__ kd, double dtdx2,
                           double* lo, double* di, double* up, double* xs, double* zs, double* cs) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= h) return;
  size_t c0 = (size_t)j * w;
  const double* krow = kd + c0;
  auto face = [&](int i) -> double {
    if (i + 1 < w) return 0.5 * (krow[i] + krow[i + 1]) * dtdx2;
    if (wrap && w > 1) return 0.5 * (krow[w - 1] + krow[0]) * dtdx2;
    return 0.0;
  };
  for (int i = 0; i < w; ++i) {
    double west = i == 0 ? face(w - 1) : face(i - 1);
    double east = face(i);
    lo[c0 + i] = -west;
    up[c0 + i] = -east;
    di[c0 + i] = 1.0 + west + east;
  }
  if (wrap && w > 2) {
    // cyclic: corners alpha = up[w-1] (row w-1, column 0), beta = lo[0] (row 0, column w-1)
    double alpha = up[c0 + w - 1], beta = lo[c0];
    double gamma = -di[c0];
    di[c0] = di[c0] - gamma;
    di[c0 + w - 1] = di[c0 + w - 1] - alpha * beta / gamma;
    lo[c0] = 0.0;
    up[c0 + w - 1] = 0.0;
    for (int i = 0; i < w; ++i) {
      xs[c0 + i] = hf[c0 + i];
      zs[c0 + i] = 0.0;
    }
    zs[c0] = gamma;
    zs[c0 + w - 1] = alpha;
    thomas_strided(w, lo, di, up, xs, cs, 1, c0);
    thomas_strided(w, lo, di, up, zs, cs, 1, c0);
    double fact = (xs[c0] + beta * xs[c0 + w - 1] / gamma) / (1.0 + zs[c0] + beta * zs[c0 + w - 1] / gamma);
    for (int i = 0; i < w; ++i) hf[c0 + i] = xs[c0 + i] - fact * zs[c0 + i];
  } else {
    if (w == 2 && wrap) {
      double f = face(0) + face(1);
      lo[c0 + 1] = -f;
      up[c0] = -f;
      di[c0] = 1.0 + f;
      di[c0 + 1] = 1.0 + f;
    }
    lo[c0] = 0.0;
    up[c0 + w - 1] = 0.0;
    if (w == 1) di[c0] = 1.0;
    thomas_strided(w, lo, di, up, hf, cs, 1, c0);
  }
}

// 32 x 32 tiles through shared memory: out (cols x rows) = the transpose of in (rows x cols)
__global__ void k_transpose(int rows, int cols, const double* __restrict__ in, double* __restrict__ out) {
  __shared__ double tile[32][33];
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int r = r0 + k, c = c0 + threadIdx.x;
    if (r < rows && c < cols) tile[k][threadIdx.x] = in[(size_t)r * cols + c];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int c = c0 + k, r = r0 + threadIdx.x;
    if (r < rows && c < cols) out[(size_t)c * rows + r] = tile[threadIdx.x][k];
  }
}

// The LOD passes as partitioned tridiagonal solves: L independent lines of n unknowns, stored
// line-fastest (element (l, i) at i L + l: the rows on transposed copies, the columns as they lie),
// each split into chunks of LOD_CHUNK unknowns solved in parallel (L x chunks threads instead of
// L): a thread eliminates its chunk (Thomas, diffusion.rs:1029-1046) for the right-hand sides
// and for the two unit couplings to the unknowns just outside the chunk, y = p + q y_(s-1) +
// r y_e; one thread a line then solves the chunks' end values from those relations (a two-term
// recurrence, forward and back), and every cell forms its y. The coefficients are the LOD's
// (diffusion.rs:370-489), formed on the fly from kd: faces 0.5 (k_i + k_(i+1)) dt / dx^2 and
// diagonal (1 + west) + east. ROWS: the periodic rows through Sherman-Morrison (diffusion.rs:
// 1048-1071): the system with the corners folded into the first and last diagonal, solved for b
// and for u = (gamma, 0, .., 0, alpha), then x - fact z. Columns: rows closed, one right-hand side.
constexpr int LOD_CHUNK = 64;
template <bool ROWS>
struct LodLine {
  const double* kd;
  int L, n, l;
  double dtdx2;
  __device__ double K(int i) const { return kd[(size_t)i * L + l]; }
  // the face between positions i and i + 1 (across the seam for the rows' last one)
  __device__ double face(int i) const {
    if (i + 1 < n) return 0.5 * (K(i) + K(i + 1)) * dtdx2;
    return ROWS ? 0.5 * (K(n - 1) + K(0)) * dtdx2 : 0.0;
  }
};

template <bool ROWS>
__global__ void __launch_bounds__(128) k_lod_chunks(int L, int n, int P, double dtdx2, const double* __restrict__ kd,
                                                    double* __restrict__ p0, double* __restrict__ p1, double* __restrict__ q,
                                                    double* __restrict__ r, double* __restrict__ c, double* __restrict__ edge) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= L * P) return;
  const int l = t % L, k = t / L;
  const int s = k * LOD_CHUNK, e = min(s + LOD_CHUNK, n);
  const LodLine<ROWS> ln{kd, L, n, l, dtdx2};
  auto at = [&](int i) { return (size_t)i * L + l; };
  // rows: the folded corners (k_lod_rows' alpha = up[n-1], beta = lo[0], gamma = -di[0])
  double fw = 0.0, alpha = 0.0, beta = 0.0, gamma = -1.0;
  if (ROWS) {
    fw = ln.face(n - 1);
    const double di0 = 1.0 + fw + ln.face(0);
    alpha = -fw;
    beta = -fw;
    gamma = -di0;
  }
  double west = s == 0 ? (ROWS ? fw : 0.0) : ln.face(s - 1);
  double bt = 1.0, cprev = 0.0, pv0 = 0.0, pv1 = 0.0, qv = 0.0, rv = 0.0;
  // the walk's inputs one position ahead (K(i + 1) and the right-hand side), so that their loads
  // overlap the recurrence; each K read once (face(i) = 0.5 (K(i) + K(i + 1)) dt / dx^2)
  double kn = ln.K(s), bn = p0[at(s)];
  for (int i = s; i < e; ++i) {
    const double ki = kn, b0 = bn;
    double east;
    if (i + 1 < n) {
      kn = ln.K(i + 1);
      east = 0.5 * (ki + kn) * dtdx2;
    } else {
      east = ROWS ? 0.5 * (ki + ln.K(0)) * dtdx2 : 0.0;
    }
    if (i + 1 < e) bn = p0[at(i + 1)];
    double di = 1.0 + west + east;
    if (ROWS && i == 0) di = di - gamma;
    if (ROWS && i == n - 1) di = di - alpha * beta / gamma;
    const double lo = i == 0 ? 0.0 : -west;
    const double up = (ROWS && i == n - 1) ? 0.0 : -east;
    const double b1 = ROWS ? (i == 0 ? gamma : (i == n - 1 ? alpha : 0.0)) : 0.0;
    const double rr = i == e - 1 ? -up : 0.0;
    // one reciprocal a position for the five quotients
    bt = i == s ? di : di - lo * cprev;
    const double ib = 1.0 / bt;
    if (i == s) {
      pv0 = b0 * ib;
      pv1 = b1 * ib;
      qv = -lo * ib;
      rv = rr * ib;
    } else {
      pv0 = (b0 - lo * pv0) * ib;
      pv1 = (b1 - lo * pv1) * ib;
      qv = (0.0 - lo * qv) * ib;
      rv = (rr - lo * rv) * ib;
    }
    cprev = up * ib;
    c[at(i)] = cprev;
    p0[at(i)] = pv0;
    if (ROWS) p1[at(i)] = pv1;
    q[at(i)] = qv;
    r[at(i)] = rv;
    west = east;
  }
  // back substitution inside the chunk: y_i -= c_i y_(i+1)
  const double e0 = pv0, e1 = pv1, eq = qv, er = rv;  // the last position's values are final
#pragma unroll 4
  for (int i = e - 2; i >= s; --i) {
    const double ci = c[at(i)];
    pv0 = p0[at(i)] - ci * pv0;
    p0[at(i)] = pv0;
    if (ROWS) {
      pv1 = p1[at(i)] - ci * pv1;
      p1[at(i)] = pv1;
    }
    qv = q[at(i)] - ci * qv;
    q[at(i)] = qv;
    rv = r[at(i)] - ci * rv;
    r[at(i)] = rv;
  }
  double* ed = edge + (size_t)t * 8;  // (k L + l) * 8: first position, then last
  ed[0] = pv0;
  ed[1] = pv1;
  ed[2] = qv;
  ed[3] = rv;
  ed[4] = e0;
  ed[5] = e1;
  ed[6] = eq;
  ed[7] = er;
}

// One thread a line: the chunks' first (A_k) and last (B_k) values from A_k = pA + qA B_(k-1) +
// rA A_(k+1), B_k = pB + qB B_(k-1) + rB A_(k+1): forward, B_(k-1) = g + h A_k; back from A_P = 0.
// Written over the edge record's p entries (A_k into [0], [1], B_k into [4], [5]); ROWS: fact of
// the line into fact[l].
template <bool ROWS>
__global__ void __launch_bounds__(128) k_lod_reduce(int L, int n, int P, double dtdx2, const double* __restrict__ kd,
                                                    double* __restrict__ edge, double* __restrict__ al,
                                                    double* __restrict__ fact) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= L) return;
  constexpr int NR = ROWS ? 2 : 1;
  double A0[NR], Bl[NR];
  for (int rhs = 0; rhs < NR; ++rhs) {
    double g = 0.0, hh = 0.0;
    for (int k = 0; k < P; ++k) {
      const double* ed = edge + ((size_t)k * L + l) * 8;
      const double pA = ed[rhs], qA = ed[2], rA = ed[3], pB = ed[4 + rhs], qB = ed[6], rB = ed[7];
      const double d = 1.0 - qA * hh;
      const double a = (pA + qA * g) / d, be = rA / d;
      // scratch for the way back: alpha, beta, g, h of chunk k
      double* sk = al + ((size_t)k * L + l) * 4;
      sk[0] = a;
      sk[1] = be;
      g = pB + qB * g + qB * hh * a;
      hh = qB * hh * be + rB;
      sk[2] = g;
      sk[3] = hh;
    }
    double An = 0.0;
    for (int k = P - 1; k >= 0; --k) {
      const double* sk = al + ((size_t)k * L + l) * 4;
      const double A = sk[0] + sk[1] * An, B = sk[2] + sk[3] * An;
      double* ed = edge + ((size_t)k * L + l) * 8;
      ed[rhs] = A;
      ed[4 + rhs] = B;
      if (k == P - 1) Bl[rhs] = B;
      An = A;
    }
    A0[rhs] = An;
  }
  if (ROWS) {
    const LodLine<true> ln{kd, L, n, l, dtdx2};
    const double fw = ln.face(n - 1);
    const double beta = -fw, gamma = -(1.0 + fw + ln.face(0));
    fact[l] = (A0[0] + beta * Bl[0] / gamma) / (1.0 + A0[1] + beta * Bl[1] / gamma);
  }
}

// Every cell: y = p + q B_(k-1) + r A_(k+1) per right-hand side; ROWS: out = y_b - fact y_u.
// The result over p0.
template <bool ROWS>
__global__ void __launch_bounds__(256) k_lod_finish(int L, int n, int P, double* __restrict__ p0, const double* __restrict__ p1,
                                                    const double* __restrict__ q, const double* __restrict__ r,
                                                    const double* __restrict__ edge, const double* __restrict__ fact) {
  const size_t total = (size_t)L * n;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int l = (int)(t % L), i = (int)(t / L), k = i / LOD_CHUNK;
    const double* em = k > 0 ? edge + ((size_t)(k - 1) * L + l) * 8 : nullptr;
    const double* ep = k + 1 < P ? edge + ((size_t)(k + 1) * L + l) * 8 : nullptr;
    const double qv = q[t], rv = r[t];
    const double y0 = p0[t] + qv * (em ? em[4] : 0.0) + rv * (ep ? ep[0] : 0.0);
    if (ROWS) {
      const double y1 = p1[t] + qv * (em ? em[5] : 0.0) + rv * (ep ? ep[1] : 0.0);
      p0[t] = y0 - fact[l] * y1;
    } else {
      p0[t] = y0;
    }
  }
}

// ---------------------------------------------------------------------------------------------
// Small control kernels.

__global__ void k_d_arm(DScalars* S, unsigned long long handle, unsigned long long handle_if) {
  S->cond = handle;
  S->cond_if = handle_if;
  S->body_runs = 0;
  cudaGraphSetConditional((cudaGraphConditionalHandle)handle, S->stop == 0 ? 1u : 0u);
}
// dt_diff_profile_kernels: a solve's state record ready for one more operator launch
__global__ void k_d_profile_state(DScalars* S) {
  S->stop = 0;
  S->cond = 0ull;
}
__global__ void k_d_disarm(DScalars* S) {
  S->cond = 0ull;
  S->cond_if = 0ull;
}

struct DProblem {
  double tol;
  int max_it, rule, n;
  int reliable;  // the FP32 lane of DT_DIFF_MIXED_RELIABLE (its other fields from k_d_rel_init)
};
__global__ void k_d_begin(DScalars* S, DProblem p, int bb_from_dot) {
  S->tol = p.tol;
  S->max_it = p.max_it;
  S->rule = p.rule;
  S->n = p.n;
  if (bb_from_dot) S->bb = S->dot_out;
  S->it = 0;
  S->stop = 0;
  S->started = 0;
  S->body_runs = 0;
  S->cond = 0ull;
  S->reliable = p.reliable;
  S->gate_it = -1;
  if (!isfinite(S->rr) || !isfinite(S->bb))
    S->stop = DSTOP_NONFINITE;
  else if (!(S->rr > 0.0) || d_converged(S, S->rr))
    S->stop = DSTOP_CONVERGED;
}

template <class T>
__global__ void __launch_bounds__(256) k_d_dot(size_t n, const T* __restrict__ a, const T* __restrict__ b, double* partials,
                                               DScalars* S) {
  Acc<1> acc;
  acc.v[0] = 0.0;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
    acc.v[0] += (double)a[k] * (double)b[k];
  const int kind[1] = {0};
  if (reduce_partials<1>(acc, kind, partials, &S->ticket[DSITE_DOT], gridDim.x) && threadIdx.x == 0) S->dot_out = acc.v[0];
}

// x += (lost / weight)(diag - 1) when weight > 0 and lost != 0 (multigrid.rs:755-761)
__global__ void k_d_massfix(size_t n, double* __restrict__ x, const double* __restrict__ diag, const DScalars* S) {
  double lost = S->lost, weight = S->weight;
  if (!(weight > 0.0 && lost != 0.0)) return;
  double k = lost / weight;
  for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) x[c] += k * (diag[c] - 1.0);
}

__global__ void k_d_scale_down(size_t n, const double* __restrict__ r, float* __restrict__ r32, float* __restrict__ x32,
                               const DScalars* S64, double* scale) {
  double s = S64->rr > 0 ? sqrt((double)n / S64->rr) : 1.0;
  if (blockIdx.x == 0 && threadIdx.x == 0) *scale = s;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    r32[k] = (float)(r[k] * s);
    x32[k] = 0.0f;
  }
}
__global__ void k_d_accumulate(size_t n, double* __restrict__ x, const float* __restrict__ x32, const double* scale) {
  double inv = 1.0 / *scale;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) x[k] += (double)x32[k] * inv;
}
__global__ void k_d_rr_is_bb(DScalars* S) { S->rr = S->bb; }

// Reliable updates (the FP32 lane holds r32 = s r64 and its correction x32 = s e, s fixed from the
// first residual's RMS). In an iteration that replaces the residual (gate_it == it):
//   k_d_rel_accumulate                x64 += x32 / s; x32 = 0
//   k_d_apply<.., DA_RESID_GATED>     r64 = b - A x64, ||r64||^2 -> rr_true
//   k_d_rel_reset                     r32 = s r64 (and the cycle's copy); rr, maxrr from rr_true;
//                                     stop when rr_true meets the tolerance
__global__ void k_d_rel_accumulate(size_t n, double* __restrict__ x, float* __restrict__ x32, const double* scale,
                                   const DScalars* S) {
  if (S->stop || S->gate_it != S->it) return;
  double inv = 1.0 / *scale;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    x[k] += (double)x32[k] * inv;
    x32[k] = 0.0f;
  }
}
__global__ void k_d_rel_reset(size_t n, const double* __restrict__ r, float* __restrict__ r32, float* __restrict__ rm,
                              const double* scale, DScalars* S) {
  if (S->stop || S->gate_it != S->it) return;
  double sc = *scale;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    float v = (float)(r[k] * sc);
    r32[k] = v;
    rm[k] = v;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    double rr = S->rr_true * sc * sc;
    S->rr = rr;
    S->maxrr = rr;
    S->replacements += 1;
    if (!isfinite(S->rr_true)) {
      S->stop = DSTOP_NONFINITE;
    } else if (S->rr_true <= S->tol * S->tol * S->bb_true) {
      S->stop = DSTOP_CONVERGED;
    }
    if (S->stop) dset_cond(S, 0);
  }
}
// The FP32 lane's problem for reliable updates, from the FP64 lane's (bb, rr of r = b - A x) and
// the scale s of r32 = s r: the tolerance on the relative residual, or with `rms` on the RMS
// residual (||r||^2 <= tol^2 n).
__global__ void k_d_rel_init(DScalars* F, const DScalars* S64, const double* scale, double delta, int rms) {
  double s2 = (*scale) * (*scale);
  double bref = rms ? (double)S64->n : S64->bb;
  F->bb = bref * s2;
  F->bb_true = bref;
  F->rr = S64->rr * s2;
  F->maxrr = F->rr;
  F->delta2 = delta * delta;
  F->replacements = 0;
  F->cond_if = 0ull;
}
__global__ void k_convert_dr(size_t n, const double* __restrict__ a, float* __restrict__ b) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) b[k] = (float)a[k];
}

}  // namespace dt

// =============================================================================================
// Host side.

namespace dt {

static const float OMEGA = 0.8f;    // multigrid.rs:45
static const int NU = 2;            // multigrid.rs:48
static const float SCALE = 0.5f;    // multigrid.rs:52
static const int COARSEST = 64;     // multigrid.rs:54
static const int COARSE_SWEEPS = 16;  // multigrid.rs:56
static const int COARSEST_GS = 128;   // the Gauss-Seidel cycle's coarsest level: 16 x 8 cells
static const int COARSE_SWEEPS_GS = 8;
static const int MG_BLOCK_CELLS = 2048;  // Gauss-Seidel levels this small run their part of the cycle in one block

template <class TM>
struct Hier {
  std::vector<DLevel<TM>> lv;
  bool built = false;
};

// CG lanes: 0 FP64 CG + FP32 cycle, 1 FP64 CG + FP64 cycle, 2 FP32 CG + FP32 cycle (mixed inner)
struct DGraph {
  cudaGraph_t g = nullptr;
  cudaGraphExec_t exec = nullptr;
  long long body_kernels = 0;
};

}  // namespace dt

struct dt_diff {
  int w = 0, h = 0, wrap = 0;
  double dx = 0;
  size_t n = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int sms = 148;
  std::vector<void*> allocs;
  size_t nalloc = 0;  // device allocations made (the DT_FAIL_ALLOC_AT test hook counts them)
  double *kd = nullptr, *b = nullptr, *x = nullptr, *r = nullptr, *p = nullptr, *ap = nullptr;
  double *east = nullptr, *south = nullptr, *diag = nullptr;
  float *east32 = nullptr, *south32 = nullptr, *diag32 = nullptr;
  float *x32 = nullptr, *r32 = nullptr, *p32 = nullptr, *ap32 = nullptr;
  double* lod[7] = {};  // the LOD first guess's scratch (lod[6]: its chunks' end values)
  double* partials = nullptr;
  double* scale = nullptr;
  dt::DScalars *S64 = nullptr, *S32 = nullptr;
  dt::Hier<float> hf[2];
  dt::Hier<double> hd[2];
  dt::DGraph graph[4][2];  // [lane: 0 split, 1 FP64, 2 FP32 inner, 3 FP32 reliable][cycle]
  // the Gauss-Seidel cycle's fused kernels (k_mg_rb2, k_mg_coarse_rb); DT_MG_FUSED=0 at create
  // keeps one launch per colour pass (the same values)
  bool mg_fused = true;
  // k_mg_rb2's 64 x 32 tiles on FP32 levels of many tiles; DT_MG_BIG_TILES=0 at create keeps
  // 32 x 16 tiles everywhere (the same values)
  bool mg_big_tiles = true;
};

namespace dt {

// Opt k_mg_rb2's instantiations in to their dynamic shared memory.
template <class TM>
static void rb2_attributes() {
  cudaFuncSetAttribute(k_mg_rb2<TM, true, MG_TX, MG_TY, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)mg_rb2_smem<TM, true>());
  cudaFuncSetAttribute(k_mg_rb2<TM, false, MG_TX, MG_TY, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)mg_rb2_smem<TM, false>());
  cudaFuncSetAttribute(k_mg_rb2<TM, true, MG_BTX, MG_BTY, 512>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)mg_rb2_smem<TM, true, MG_BTX, MG_BTY>());
  cudaFuncSetAttribute(k_mg_rb2<TM, false, MG_BTX, MG_BTY, 512>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)mg_rb2_smem<TM, false, MG_BTX, MG_BTY>());
}

template <class T>
static dt_status ddalloc(dt_diff* s, T** p, size_t count) {
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

static unsigned int dgrid(const dt_diff* s, size_t n) {
  return std::max(1u, std::min<unsigned int>(ceil_div(n, 256), (unsigned)s->sms * 8));
}

// The level shapes of the hierarchy (multigrid.rs:117-123): halve (rounding up) until the level
// has at most `coarsest` cells or stops shrinking; x wraps on a level while it is wider than 1.
template <class TM>
static dt_status build_levels(dt_diff* s, Hier<TM>& H, int coarsest) {
  if (H.built) return DT_OK;
  int w = s->w, h = s->h, wrap = s->wrap && s->w > 1;
  for (;;) {
    DLevel<TM> L;
    L.w = w;
    L.h = h;
    L.wrap = wrap;
    size_t n = (size_t)w * h;
    for (TM** q : {&L.east, &L.south, &L.diag, &L.wd, &L.mass, &L.r, &L.z, &L.t}) DT_TRY(ddalloc(s, q, n));
    H.lv.push_back(L);
    int wc = (w + 1) / 2, hc = (h + 1) / 2;
    if ((long)w * h <= coarsest || (wc == w && hc == h)) break;
    wrap = wrap && wc > 1;
    w = wc;
    h = hc;
  }
  H.built = true;
  return DT_OK;
}

// Level coefficients for the current operator: the finest from the FP64 couplings, the rest by
// aggregation.
// wd: omega / diag for the damped-Jacobi cycle, 1 / diag for the Gauss-Seidel one.
template <class TM>
static void fill_levels(dt_diff* s, Hier<TM>& H, int kind, cudaStream_t st) {
  DLevel<TM>& f = H.lv[0];
  const TM omega = kind == DT_CYCLE_JACOBI ? (TM)OMEGA : (TM)1;
  k_mg_finest<TM><<<dgrid(s, s->n), 256, 0, st>>>(s->n, s->east, s->south, s->diag, omega, f.east, f.south, f.diag, f.wd, f.mass);
  count_launch();
  for (size_t l = 1; l < H.lv.size(); ++l) {
    size_t nc = (size_t)H.lv[l].w * H.lv[l].h;
    k_mg_coarsen<TM><<<dgrid(s, nc), 256, 0, st>>>(H.lv[l - 1], H.lv[l], (TM)SCALE);
    k_mg_diag<TM><<<dgrid(s, nc), 256, 0, st>>>(H.lv[l], omega);
    count_launch();
    count_launch();
  }
}

// Whether k_mg_rb2 takes a level: at least MG_TX + 10 cells wide (no cell twice in a tile's
// region) and fewer than 2^31 cells (its 32-bit offsets).
template <class TM>
static bool rb2_fits(const DLevel<TM>& L) {
  return L.w >= MG_TX + 10 && (size_t)L.w * L.h < ((size_t)1 << 31);
}
// The two tiled sweeps of a level (PRE: from z = 0 with the restriction into C.r; else with the
// coarse correction zc): 64 x 32 tiles for FP32 levels of at least four tiles an SM, else 32 x 16.
template <class TM, bool PRE>
static void launch_rb2(dt_diff* s, const DLevel<TM>& L, const DLevel<TM>& C, const TM* zc, TM* zout, cudaStream_t st) {
  const bool big = std::is_same<TM, float>::value && s->mg_big_tiles && L.w >= MG_BTX + 10 &&
                   (size_t)ceil_div(L.w, MG_BTX) * ceil_div(L.h, MG_BTY) >= (size_t)4 * s->sms;
  if (big) {
    const dim3 tg(ceil_div(L.w, MG_BTX), ceil_div(L.h, MG_BTY));
    k_mg_rb2<TM, PRE, MG_BTX, MG_BTY, 512><<<tg, 512, mg_rb2_smem<TM, PRE, MG_BTX, MG_BTY>(), st>>>(L, C, zc, zout);
  } else {
    const dim3 tg(ceil_div(L.w, MG_TX), ceil_div(L.h, MG_TY));
    k_mg_rb2<TM, PRE, MG_TX, MG_TY, 256><<<tg, 256, mg_rb2_smem<TM, PRE>(), st>>>(L, C, zc, zout);
  }
  count_launch();
}

// One V-cycle from z = 0 on level l with r set; returns the buffer holding the level's z.
template <class TM>
static TM* vcycle(dt_diff* s, Hier<TM>& H, size_t l, int kind, cudaStream_t st) {
  DLevel<TM>& L = H.lv[l];
  size_t n = (size_t)L.w * L.h;
  unsigned int g = dgrid(s, n);
  bool coarsest = l + 1 == H.lv.size();
  if (coarsest) {
    if (kind == DT_CYCLE_JACOBI)
      k_mg_coarsest<TM, 0><<<1, 256, 0, st>>>(L, L.z, COARSE_SWEEPS);
    else
      k_mg_coarsest<TM, 1><<<1, 256, 0, st>>>(L, L.z, COARSE_SWEEPS_GS);
    count_launch();
    return L.z;
  }
  DLevel<TM>& C = H.lv[l + 1];
  if (kind == DT_CYCLE_JACOBI) {
    // multigrid.rs:514-522
    TM *cur = L.z, *nxt = L.t;
    k_mg_first<TM><<<g, 256, 0, st>>>(L, cur);
    count_launch();
    for (int k = 1; k < NU; ++k) {
      k_mg_sweep<TM><<<g, 256, 0, st>>>(L, cur, nxt, nullptr, 0);
      count_launch();
      std::swap(cur, nxt);
    }
    k_mg_restrict<TM><<<dgrid(s, (size_t)C.w * C.h), 256, 0, st>>>(L, cur, C);
    count_launch();
    TM* zc = vcycle<TM>(s, H, l + 1, kind, st);
    k_mg_sweep<TM><<<g, 256, 0, st>>>(L, cur, nxt, zc, C.w);
    count_launch();
    std::swap(cur, nxt);
    for (int k = 1; k < NU; ++k) {
      k_mg_sweep<TM><<<g, 256, 0, st>>>(L, cur, nxt, nullptr, 0);
      count_launch();
      std::swap(cur, nxt);
    }
    return cur;
  }
  // multi-colour Gauss-Seidel V(NU, NU): colours forward, coarse correction, colours backward
  int ncol = gs_colours(L.w, L.wrap);
  if (s->mg_fused) {
    // this level and every coarser one in one block, when it is small enough
    if (n <= (size_t)MG_BLOCK_CELLS && H.lv.size() - l <= (size_t)MG_BLOCK_LEVELS) {
      MgChain<TM> m{};
      m.count = (int)(H.lv.size() - l);
      m.total = 0;
      for (int q = 0; q < m.count; ++q) {
        m.lv[q] = H.lv[l + q];
        m.off[q] = m.total;
        m.total += H.lv[l + q].w * H.lv[l + q].h;
      }
      const size_t smem = (size_t)6 * m.total * sizeof(TM);
      const DLevel<TM>& last = H.lv.back();
      if (smem <= 200 * 1024 && last.w * last.h <= 128) {  // the coarsest takes one thread a cell of 128
        k_mg_coarse_rb<TM><<<1, 1024, smem, st>>>(m, NU, COARSE_SWEEPS_GS);
        count_launch();
        return L.z;
      }
    }
    // both sweeps of the smoothing in one launch over tiles, the restriction fused into the
    // pre-smoothing (two-colour levels wide enough)
    if (ncol == 2 && NU == 2 && rb2_fits(L)) {
      launch_rb2<TM, true>(s, L, C, nullptr, L.z, st);
      TM* zc = vcycle<TM>(s, H, l + 1, kind, st);
      launch_rb2<TM, false>(s, L, C, zc, L.t, st);
      return L.t;  // the level's z, in its spare buffer
    }
  }
  for (int sweep = 0; sweep < NU; ++sweep)
    for (int c = 0; c < ncol; ++c) {
      if (sweep == 0)
        k_mg_gs<TM, true><<<g, 256, 0, st>>>(L, L.z, c);
      else
        k_mg_gs<TM, false><<<g, 256, 0, st>>>(L, L.z, c);
      count_launch();
    }
  k_mg_restrict<TM><<<dgrid(s, (size_t)C.w * C.h), 256, 0, st>>>(L, L.z, C);
  count_launch();
  TM* zc = vcycle<TM>(s, H, l + 1, kind, st);
  k_mg_prolong<TM><<<g, 256, 0, st>>>(L, L.z, zc, C.w);
  count_launch();
  for (int sweep = 0; sweep < NU; ++sweep)
    for (int c = ncol - 1; c >= 0; --c) {
      k_mg_gs<TM, false><<<g, 256, 0, st>>>(L, L.z, c);
      count_launch();
    }
  return L.z;
}

// The CG of one lane: vectors x, r, p, ap in TC; the cycle in TM on the levels of H; rm = H's
// finest r. Coefficients of the operator in TC.
template <class TC, class TM>
struct CgLane {
  TC *x, *r, *p, *ap, *east, *south, *diag;
  Hier<TM>* H;
  DScalars* S;
  TM* z;  // where the cycle leaves its result (set when the launch sequence is built)
};

// The residual replacement of a reliable-update iteration (the FP32 lane): gated kernels that do
// nothing unless the iteration's update asked for it. `count`: count their launches (not inside
// the loop body's IF node, whose runs are counted from the replacements).
static void launch_reliable_d(dt_diff* s, Hier<float>& H, cudaStream_t st, bool count) {
  unsigned int g = dgrid(s, s->n);
  k_d_rel_accumulate<<<g, 256, 0, st>>>(s->n, s->x, s->x32, s->scale, s->S32);
  k_d_apply<double, float, DA_RESID_GATED><<<g, 256, 0, st>>>(s->w, s->h, s->wrap && s->w > 1, s->east, s->south, s->diag, s->x,
                                                              s->b, s->r, nullptr, s->partials, s->S32);
  k_d_rel_reset<<<g, 256, 0, st>>>(s->n, s->r, s->r32, H.lv[0].r, s->scale, s->S32);
  if (count)
    for (int k = 0; k < 3; ++k) count_launch();
}

// While `st` captures a loop body: a conditional IF node, its body the residual replacement
// (captured on `aside`), so that iterations that replace nothing launch nothing for it.
static dt_status add_reliable_if_d(dt_diff* s, Hier<float>& H, cudaStream_t st, cudaStream_t aside,
                                   unsigned long long* handle_out) {
  cudaStreamCaptureStatus cs;
  unsigned long long id = 0;
  cudaGraph_t graph = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  DT_CUDA(cudaStreamGetCaptureInfo(st, &cs, &id, &graph, &deps, &nd));
  if (cs != cudaStreamCaptureStatusActive || !graph) {
    set_error("diffusion loop graph: the stream is not capturing");
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
  DT_CUDA(cudaStreamBeginCaptureToGraph(aside, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                        cudaStreamCaptureModeThreadLocal));
  launch_reliable_d(s, H, aside, false);
  cudaGraph_t ifbody;
  DT_CUDA(cudaStreamEndCapture(aside, &ifbody));
  *handle_out = (unsigned long long)h;
  return DT_OK;
}

// One CG iteration (multigrid.rs:698-733). With `reliable` (the FP32 lane of
// DT_DIFF_MIXED_RELIABLE) the residual replacement follows the update: under an IF node when
// `aside` is given (capturing a loop body; its handle goes to *if_handle), else launched gated.
template <class TC, class TM>
static dt_status cg_iteration(dt_diff* s, CgLane<TC, TM>& C, int kind, cudaStream_t st, bool reliable = false,
                              cudaStream_t aside = nullptr, unsigned long long* if_handle = nullptr) {
  unsigned int g = dgrid(s, s->n);
  k_d_apply<TC, TM, DA_PAP><<<g, 256, 0, st>>>(s->w, s->h, s->wrap && s->w > 1, C.east, C.south, C.diag, C.p, nullptr, C.ap,
                                                nullptr, s->partials, C.S);
  count_launch();
  k_d_update<TC, TM><<<g, 256, 0, st>>>(s->n, C.x, C.r, C.H->lv[0].r, C.p, C.ap, s->partials, C.S);
  count_launch();
  if constexpr (std::is_same<TM, float>::value) {
    if (reliable) {
      if (aside)
        DT_TRY(add_reliable_if_d(s, *C.H, st, aside, if_handle));
      else
        launch_reliable_d(s, *C.H, st, true);
    }
  }
  TM* z = vcycle<TM>(s, *C.H, 0, kind, st);
  C.z = z;
  k_d_rz<TC, TM><<<g, 256, 0, st>>>(s->n, C.r, z, s->partials, C.S);
  count_launch();
  k_d_direction<TC, TM><<<g, 256, 0, st>>>(s->n, C.p, z, C.S, 0);
  count_launch();
  return DT_OK;
}

template <class TC, class TM>
static dt_status cg_graph(dt_diff* s, CgLane<TC, TM>& C, int lane, int kind, DGraph** out, bool reliable = false) {
  DGraph& G = s->graph[lane][kind];
  if (G.exec) {
    *out = &G;
    return DT_OK;
  }
  cudaGraph_t g;
  DT_CUDA(cudaGraphCreate(&g, 0));
  cudaGraphConditionalHandle handle;
  DT_CUDA(cudaGraphConditionalHandleCreate(&handle, g, 1, cudaGraphCondAssignDefault));
  unsigned long long hv = (unsigned long long)handle, hv_if = 0ull;
  DScalars* Sp = C.S;
  cudaKernelNodeParams kp = {};
  void* arm_args[] = {&Sp, &hv, &hv_if};
  kp.func = (void*)k_d_arm;
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
  begin_capture_count();
  dt_status st_body = cg_iteration<TC, TM>(s, C, kind, s->stream, reliable, aside, &hv_if);
  G.body_kernels = end_capture_count();
  cudaGraph_t captured;
  cudaError_t e_end = cudaStreamEndCapture(s->stream, &captured);
  if (aside) cudaStreamDestroy(aside);
  DT_TRY(st_body);
  DT_CUDA(e_end);
  if (reliable) DT_CUDA(cudaGraphKernelNodeSetParams(n_arm, &kp));  // k_d_arm learns the IF node's handle
  void* dis_args[] = {&Sp};
  kp.func = (void*)k_d_disarm;
  kp.kernelParams = dis_args;
  DT_CUDA(cudaGraphAddKernelNode(&n_disarm, g, &n_loop, 1, &kp));
  DT_CUDA(cudaGraphInstantiate(&G.exec, g, 0));
  G.g = g;
  *out = &G;
  return DT_OK;
}

static dt_status dread(dt_diff* s, const DScalars* S, DScalars* out) {
  DT_CUDA(cudaMemcpyAsync(out, S, sizeof(DScalars), cudaMemcpyDeviceToHost, s->stream));
  DT_CUDA(cudaStreamSynchronize(s->stream));
  return DT_OK;
}

// CG of lane C from x with r = b - A x, rm and S->rr, S->bb already set.
template <class TC, class TM>
static dt_status run_cg(dt_diff* s, CgLane<TC, TM>& C, int lane, int kind, const DProblem& prob, int host_loop, DScalars* out,
                        bool reliable = false) {
  cudaStream_t st = s->stream;
  unsigned int g = dgrid(s, s->n);
  k_d_begin<<<1, 1, 0, st>>>(C.S, prob, 0);
  count_launch();
  // the first direction: z = M^-1 r, rz, p = z
  TM* z = vcycle<TM>(s, *C.H, 0, kind, st);
  k_d_rz<TC, TM><<<g, 256, 0, st>>>(s->n, C.r, z, s->partials, C.S);
  k_d_direction<TC, TM><<<g, 256, 0, st>>>(s->n, C.p, z, C.S, 1);
  count_launch();
  count_launch();
  if (!host_loop) {
    DGraph* G;
    DT_TRY(cg_graph<TC, TM>(s, C, lane, kind, &G, reliable));
    DT_CUDA(cudaGraphLaunch(G->exec, st));
    DT_TRY(dread(s, C.S, out));
    add_launches(2 + G->body_kernels * (long long)out->body_runs);
    return DT_OK;
  }
  DT_TRY(dread(s, C.S, out));
  for (int pass = 0; pass < prob.max_it + 2 && out->stop == DSTOP_RUNNING; ++pass) {
    DT_TRY(cg_iteration<TC, TM>(s, C, kind, st, reliable));
    DT_CUDA(cudaGetLastError());
    DT_TRY(dread(s, C.S, out));
    if (host_loop > 1)
      fprintf(stderr, "diffusion cg it %d stop %d rr %.6e rz %.6e alpha %.6e beta %.6e\n", out->it, out->stop, out->rr, out->rz,
              out->alpha, out->beta);
  }
  return DT_OK;
}

static dt_status diff_first_guess(dt_diff* s, const dt_diff_params* p, double dt) {
  cudaStream_t st = s->stream;
  DT_CUDA(cudaMemcpyAsync(s->x, s->b, s->n * sizeof(double), cudaMemcpyDeviceToDevice, st));
  if (p->first_guess) {
    double dtdx2 = dt / (s->dx * s->dx);
    if (s->wrap && s->w > 2) {
      // rows through transposed copies, so each thread's walk reads contiguous words
      const dim3 tb(32, 8), tg_in(ceil_div(s->w, 32), ceil_div(s->h, 32)), tg_out(ceil_div(s->h, 32), ceil_div(s->w, 32));
      k_transpose<<<tg_in, tb, 0, st>>>(s->h, s->w, s->kd, s->lod[0]);
      k_transpose<<<tg_in, tb, 0, st>>>(s->h, s->w, s->x, s->lod[1]);
      // the rows (lines of w unknowns, h of them) in chunks: lod[1] b -> x, lod[2] z, lod[3] q, lod[4] r,
      // lod[5] c, lod[6] the chunks' end values and the recurrence's scratch (8 + 4 values a chunk)
      // and the rows' Sherman-Morrison factors
      const int P = (int)ceil_div(s->w, LOD_CHUNK);
      double* edge = s->lod[6];
      double* al = edge + (size_t)8 * P * s->h;
      double* fact = al + (size_t)4 * P * s->h;
      k_lod_chunks<true><<<ceil_div((size_t)s->h * P, 128), 128, 0, st>>>(s->h, s->w, P, dtdx2, s->lod[0], s->lod[1], s->lod[2],
                                                                        s->lod[3], s->lod[4], s->lod[5], edge);
      k_lod_reduce<true><<<ceil_div(s->h, 128), 128, 0, st>>>(s->h, s->w, P, dtdx2, s->lod[0], edge, al, fact);
      k_lod_finish<true><<<dgrid(s, s->n), 256, 0, st>>>(s->h, s->w, P, s->lod[1], s->lod[2], s->lod[3], s->lod[4], edge, fact);
      k_transpose<<<tg_out, tb, 0, st>>>(s->w, s->h, s->lod[1], s->x);
      for (int k = 0; k < 6; ++k) count_launch();
    } else {
      k_lod_rows<<<ceil_div(s->h, 64), 64, 0, st>>>(s->w, s->h, s->wrap, s->x, s->kd, dtdx2, s->lod[0], s->lod[1], s->lod[2],
                                                    s->lod[3], s->lod[4], s->lod[5]);
      count_launch();
    }
    {
      // the columns (lines of h unknowns, w of them, as they lie) in chunks: x in place, lod[2] q,
      // lod[3] r, lod[4] c, lod[6] the chunks' end values
      const int P = (int)ceil_div(s->h, LOD_CHUNK);
      double* edge = s->lod[6];
      double* al = edge + (size_t)8 * P * s->w;
      k_lod_chunks<false><<<ceil_div((size_t)s->w * P, 128), 128, 0, st>>>(s->w, s->h, P, dtdx2, s->kd, s->x, nullptr,
                                                                         s->lod[2], s->lod[3], s->lod[4], edge);
      k_lod_reduce<false><<<ceil_div(s->w, 128), 128, 0, st>>>(s->w, s->h, P, dtdx2, s->kd, edge, al, nullptr);
      k_lod_finish<false><<<dgrid(s, s->n), 256, 0, st>>>(s->w, s->h, P, s->x, nullptr, s->lod[2], s->lod[3], edge, nullptr);
      for (int k = 0; k < 3; ++k) count_launch();
    }
  }
  return DT_OK;
}

template <class TM>
static Hier<TM>& hier_for(dt_diff* s, int kind);
template <>
Hier<float>& hier_for<float>(dt_diff* s, int kind) {
  return s->hf[kind];
}
template <>
Hier<double>& hier_for<double>(dt_diff* s, int kind) {
  return s->hd[kind];
}

// FP64 CG with a TM cycle (lane 0: TM = float, the reference's split; lane 1: TM = double).
template <class TM>
static dt_status solve_fp64_cg(dt_diff* s, const dt_diff_params* p, int lane, dt_report* rep, DScalars* fin) {
  cudaStream_t st = s->stream;
  Hier<TM>& H = hier_for<TM>(s, p->cycle);
  DT_TRY(build_levels<TM>(s, H, p->cycle == DT_CYCLE_JACOBI ? COARSEST : COARSEST_GS));
  fill_levels<TM>(s, H, p->cycle, st);
  unsigned int g = dgrid(s, s->n);
  int wrap = s->wrap && s->w > 1;
  // bb, then r = b - A x, rm, rr
  k_d_dot<double><<<g, 256, 0, st>>>(s->n, s->b, s->b, s->partials, s->S64);
  k_d_begin<<<1, 1, 0, st>>>(s->S64, DProblem{p->tol, p->max_iterations, p->stop, (int)s->n}, 1);
  k_d_apply<double, TM, DA_RESID><<<g, 256, 0, st>>>(s->w, s->h, wrap, s->east, s->south, s->diag, s->x, s->b, s->r, H.lv[0].r,
                                                     s->partials, s->S64);
  count_launch();
  count_launch();
  count_launch();
  CgLane<double, TM> C{s->x, s->r, s->p, s->ap, s->east, s->south, s->diag, &H, s->S64, nullptr};
  DT_TRY(run_cg<double, TM>(s, C, lane, p->cycle, DProblem{p->tol, p->max_iterations, p->stop, (int)s->n}, p->host_loop, fin));
  if (rep) rep->iterations = fin->it;
  return DT_OK;
}

// FP32 inner CG (FP32 cycle) inside FP64 refinement on the residual scaled to unit RMS.
static dt_status solve_mixed_cg(dt_diff* s, const dt_diff_params* p, dt_report* rep, DScalars* fin) {
  cudaStream_t st = s->stream;
  Hier<float>& H = s->hf[p->cycle];
  DT_TRY(build_levels<float>(s, H, p->cycle == DT_CYCLE_JACOBI ? COARSEST : COARSEST_GS));
  fill_levels<float>(s, H, p->cycle, st);
  unsigned int g = dgrid(s, s->n);
  int wrap = s->wrap && s->w > 1;
  k_d_dot<double><<<g, 256, 0, st>>>(s->n, s->b, s->b, s->partials, s->S64);
  k_d_begin<<<1, 1, 0, st>>>(s->S64, DProblem{p->tol, p->max_iterations, p->stop, (int)s->n}, 1);
  count_launch();
  count_launch();
  int iterations = 0, refinements = 0;
  DScalars h64, h32;
  h32.stop = DSTOP_RUNNING;
  bool nonfinite = false;
  for (;;) {
    k_d_apply<double, float, DA_RESID><<<g, 256, 0, st>>>(s->w, s->h, wrap, s->east, s->south, s->diag, s->x, s->b, s->r, s->r32,
                                                          s->partials, s->S64);
    count_launch();
    DT_TRY(dread(s, s->S64, &h64));
    if (!std::isfinite(h64.rr) || !std::isfinite(h64.bb)) {
      nonfinite = true;
      break;
    }
    double lim2 = p->stop == DT_STOP_REL_RESIDUAL ? p->tol * p->tol * h64.bb : p->tol * p->tol * (double)s->n;
    if (h64.rr <= lim2) break;
    if (refinements >= p->max_refinements || iterations >= p->max_iterations) break;
    double rel = std::sqrt(h64.rr / std::max(lim2, 1e-300));  // > 1: how far above the target
    double itol = std::min(0.5, std::max(p->inner_tol, 0.3 / rel));
    k_d_scale_down<<<g, 256, 0, st>>>(s->n, s->r, s->r32, s->x32, s->S64, s->scale);
    // the inner system's b is the scaled residual: bb = its r.r, x = 0
    k_d_dot<float><<<g, 256, 0, st>>>(s->n, s->r32, s->r32, s->partials, s->S32);
    k_d_begin<<<1, 1, 0, st>>>(s->S32, DProblem{itol, p->max_iterations - iterations, DT_STOP_REL_RESIDUAL, (int)s->n}, 1);
    k_d_rr_is_bb<<<1, 1, 0, st>>>(s->S32);
    // the cycle's finest rhs is the inner CG's r in FP32
    cudaMemcpyAsync(H.lv[0].r, s->r32, s->n * sizeof(float), cudaMemcpyDeviceToDevice, st);
    count_launch();
    count_launch();
    count_launch();
    count_launch();
    CgLane<float, float> C{s->x32, s->r32, s->p32, s->ap32, s->east32, s->south32, s->diag32, &H, s->S32, nullptr};
    DT_TRY(run_cg<float, float>(s, C, 2, p->cycle, DProblem{itol, p->max_iterations - iterations, DT_STOP_REL_RESIDUAL, (int)s->n},
                                p->host_loop, &h32));
    k_d_accumulate<<<g, 256, 0, st>>>(s->n, s->x, s->x32, s->scale);
    count_launch();
    iterations += h32.it;
    ++refinements;
    if (h32.stop == DSTOP_NONFINITE) {
      nonfinite = true;
      break;
    }
  }
  *fin = h64;
  fin->it = iterations;
  fin->stop = nonfinite ? DSTOP_NONFINITE
                        : (h64.rr <= (p->stop == DT_STOP_REL_RESIDUAL ? p->tol * p->tol * h64.bb : p->tol * p->tol * (double)s->n)
                               ? DSTOP_CONVERGED
                               : DSTOP_CAP);
  if (rep) {
    rep->iterations = iterations;
    rep->refinements = refinements;
  }
  return DT_OK;
}

// One FP32 CG (FP32 cycle) with reliable updates: the residual scaled to unit RMS once, then
// replaced by the FP64 b - A x (x folded into the FP64 accumulation) each time the FP32 residual
// has fallen a hundredfold or meets the tolerance; the FP64 residual alone decides convergence, and the
// search direction carries on, so the Krylov space is never restarted.
static dt_status solve_mixed_reliable(dt_diff* s, const dt_diff_params* p, dt_report* rep, DScalars* fin) {
  cudaStream_t st = s->stream;
  Hier<float>& H = s->hf[p->cycle];
  DT_TRY(build_levels<float>(s, H, p->cycle == DT_CYCLE_JACOBI ? COARSEST : COARSEST_GS));
  fill_levels<float>(s, H, p->cycle, st);
  unsigned int g = dgrid(s, s->n);
  int wrap = s->wrap && s->w > 1;
  k_d_dot<double><<<g, 256, 0, st>>>(s->n, s->b, s->b, s->partials, s->S64);
  k_d_begin<<<1, 1, 0, st>>>(s->S64, DProblem{p->tol, p->max_iterations, p->stop, (int)s->n}, 1);
  k_d_apply<double, float, DA_RESID><<<g, 256, 0, st>>>(s->w, s->h, wrap, s->east, s->south, s->diag, s->x, s->b, s->r, s->r32,
                                                        s->partials, s->S64);
  k_d_scale_down<<<g, 256, 0, st>>>(s->n, s->r, s->r32, s->x32, s->S64, s->scale);
  // replace when the FP32 residual has fallen a hundredfold: the V-cycle cuts it more than
  // tenfold an iteration, so a tenfold trigger would replace it every iteration
  k_d_rel_init<<<1, 1, 0, st>>>(s->S32, s->S64, s->scale, 0.01, p->stop == DT_STOP_RMS_RESIDUAL);
  DT_CUDA(cudaMemcpyAsync(H.lv[0].r, s->r32, s->n * sizeof(float), cudaMemcpyDeviceToDevice, st));  // the cycle's rhs
  for (int k = 0; k < 6; ++k) count_launch();
  CgLane<float, float> C{s->x32, s->r32, s->p32, s->ap32, s->east32, s->south32, s->diag32, &H, s->S32, nullptr};
  DScalars h32;
  DT_TRY(run_cg<float, float>(s, C, 3, p->cycle, DProblem{p->tol, p->max_iterations, DT_STOP_REL_RESIDUAL, (int)s->n, 1},
                              p->host_loop, &h32, true));
  if (!p->host_loop) add_launches(3LL * h32.replacements);
  // the correction since the last replacement (zero when the solve ended on one)
  k_d_accumulate<<<g, 256, 0, st>>>(s->n, s->x, s->x32, s->scale);
  count_launch();
  *fin = h32;
  if (rep) {
    rep->iterations = h32.it;
    rep->refinements = h32.replacements;
  }
  return DT_OK;
}

}  // namespace dt

using namespace dt;

extern "C" {

void dt_diff_default_params(dt_diff_params* p) {
  if (!p) return;
  p->cycle = DT_CYCLE_JACOBI;
  p->precision = DT_DIFF_FP64_CG_FP32_CYCLE;
  p->stop = DT_STOP_RMS_RESIDUAL;
  p->tol = 1e-5;             // surface.numerics.diffusion_tol_m (params.rs:197-200)
  p->max_iterations = 400;   // CG_MAX_ITER (diffusion.rs:497)
  p->first_guess = 1;        // the LOD splitting (diffusion.rs:101-110)
  p->inner_tol = 1e-5;
  p->max_refinements = 8;
  p->host_loop = 0;
}

dt_status dt_diff_destroy(dt_diff* s) {
  if (!s) return DT_OK;
  if (s->stream) cudaStreamSynchronize(s->stream);
  for (auto& a : s->graph)
    for (auto& G : a) {
      if (G.exec) cudaGraphExecDestroy(G.exec);
      if (G.g) cudaGraphDestroy(G.g);
    }
  for (void* q : s->allocs) cudaFree(q);
  if (s->ev0) cudaEventDestroy(s->ev0);
  if (s->ev1) cudaEventDestroy(s->ev1);
  if (s->own_stream && s->stream) cudaStreamDestroy(s->stream);
  delete s;
  return DT_OK;
}

dt_status dt_diff_create(int w, int h, double dx, int wrap_x, dt_diff** out) {
  if (!out) {
    set_error("dt_diff_create: out is NULL");
    return DT_BAD_ARG;
  }
  *out = nullptr;
  if (w < 1 || h < 1 || !(dx > 0.0) || !std::isfinite(dx)) {
    set_error("dt_diff_create: bad raster %d x %d, dx %g", w, h, dx);
    return DT_BAD_ARG;
  }
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    set_error("dt_diff_create: no CUDA device");
    return DT_DEVICE_ERROR;
  }
  auto* s = new dt_diff();
  s->w = w;
  s->h = h;
  s->dx = dx;
  s->wrap = wrap_x ? 1 : 0;
  if (const char* e = getenv("DT_MG_FUSED")) s->mg_fused = e[0] != '0';
  // the one-block coarse cycle stages at most about 4/3 MG_BLOCK_CELLS cells (plus the levels'
  // rounding up) in six arrays
  cudaFuncSetAttribute(k_mg_coarse_rb<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(k_mg_coarse_rb<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  if (const char* e = getenv("DT_MG_BIG_TILES")) s->mg_big_tiles = e[0] != '0';
  rb2_attributes<float>();
  rb2_attributes<double>();
  s->n = (size_t)w * h;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, 0) == cudaSuccess) s->sms = prop.multiProcessorCount;
  auto fail = [&](dt_status e) {
    dt_diff_destroy(s);
    return e;
  };
  if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(DT_DEVICE_ERROR);
  s->own_stream = true;
  dt_status st;
  for (double** q : {&s->kd, &s->b, &s->x, &s->r, &s->p, &s->ap, &s->east, &s->south, &s->diag})
    if ((st = ddalloc(s, q, s->n)) != DT_OK) return fail(st);
  for (float** q : {&s->east32, &s->south32, &s->diag32, &s->x32, &s->r32, &s->p32, &s->ap32})
    if ((st = ddalloc(s, q, s->n)) != DT_OK) return fail(st);
  for (int k = 0; k < 6; ++k)
    if ((st = ddalloc(s, &s->lod[k], s->n)) != DT_OK) return fail(st);
  {
    // the LOD chunks' end values, their recurrence's scratch (12 values a chunk of a line) and
    // the rows' Sherman-Morrison factors
    const size_t chunks = (size_t)ceil_div(s->w, LOD_CHUNK) * s->h + (size_t)ceil_div(s->h, LOD_CHUNK) * s->w;
    if ((st = ddalloc(s, &s->lod[6], 12 * chunks + s->h + s->w)) != DT_OK) return fail(st);
  }
  if ((st = ddalloc(s, &s->partials, (size_t)s->sms * 8 * 2)) != DT_OK) return fail(st);
  if ((st = ddalloc(s, &s->scale, 1)) != DT_OK) return fail(st);
  if ((st = ddalloc(s, &s->S64, 1)) != DT_OK) return fail(st);
  if ((st = ddalloc(s, &s->S32, 1)) != DT_OK) return fail(st);
  cudaMemset(s->S64, 0, sizeof(DScalars));
  cudaMemset(s->S32, 0, sizeof(DScalars));
  if (cudaEventCreate(&s->ev0) != cudaSuccess || cudaEventCreate(&s->ev1) != cudaSuccess) return fail(DT_DEVICE_ERROR);
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    set_error("dt_diff_create: %s", cudaGetErrorString(e));
    return fail(DT_DEVICE_ERROR);
  }
  *out = s;
  return DT_OK;
}

dt_status dt_diff_set_stream(dt_diff* s, void* stream) {
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

static dt_status diff_check(const dt_diff_params* p, double dt) {
  if (!p) {
    set_error("diffusion solve: params is NULL");
    return DT_BAD_ARG;
  }
  if ((p->cycle != DT_CYCLE_JACOBI && p->cycle != DT_CYCLE_RBGS) || p->precision < 0 || p->precision > 3 ||
      (p->stop != DT_STOP_RMS_RESIDUAL && p->stop != DT_STOP_REL_RESIDUAL) || !(p->tol >= 0.0) || p->max_iterations < 0) {
    set_error("diffusion solve: bad parameters (cycle %d, precision %d, rule %d, tol %g)", p->cycle, p->precision, p->stop, p->tol);
    return DT_BAD_ARG;
  }
  if (!(dt > 0.0) || !std::isfinite(dt)) {
    set_error("diffusion solve: dt must be positive and finite (got %g)", dt);
    return DT_BAD_ARG;
  }
  return DT_OK;
}

// The solve on kd and b already on the device (the handle's buffers).
static dt_status diff_solve_loaded(dt_diff* s, double dt, const dt_diff_params* p, dt_report* rep) {
  cudaStream_t st = s->stream;
  long long l0 = launches_now();
  cudaEventRecord(s->ev0, st);
  double dtdx2 = dt / (s->dx * s->dx);
  k_d_coeffs<<<dgrid(s, s->n), 256, 0, st>>>(s->w, s->h, s->wrap && s->w > 1, s->kd, dtdx2, s->east, s->south, s->diag, s->east32,
                                             s->south32, s->diag32);
  count_launch();
  DT_TRY(diff_first_guess(s, p, dt));
  DScalars fin;
  memset(&fin, 0, sizeof fin);
  if (rep) memset(rep, 0, sizeof *rep);
  if (p->precision == DT_DIFF_MIXED) {
    DT_TRY(solve_mixed_cg(s, p, rep, &fin));
  } else if (p->precision == DT_DIFF_MIXED_RELIABLE) {
    DT_TRY(solve_mixed_reliable(s, p, rep, &fin));
  } else if (p->precision == DT_DIFF_FP64) {
    DT_TRY(solve_fp64_cg<double>(s, p, 1, rep, &fin));
  } else {
    DT_TRY(solve_fp64_cg<float>(s, p, 0, rep, &fin));
  }
  // mass put-back: sum x = sum b (multigrid.rs:736-761)
  unsigned int g = dgrid(s, s->n);
  int wrap = s->wrap && s->w > 1;
  k_d_apply<double, float, DA_MASS><<<g, 256, 0, st>>>(s->w, s->h, wrap, s->east, s->south, s->diag, s->x, s->b, nullptr, nullptr,
                                                       s->partials, s->S64);
  k_d_massfix<<<g, 256, 0, st>>>(s->n, s->x, s->diag, s->S64);
  // the answer's relative residual
  k_d_apply<double, float, DA_RESID><<<g, 256, 0, st>>>(s->w, s->h, wrap, s->east, s->south, s->diag, s->x, s->b, s->ap, s->r32,
                                                        s->partials, s->S64);
  count_launch();
  count_launch();
  count_launch();
  cudaEventRecord(s->ev1, st);
  DScalars h;
  DT_TRY(dread(s, s->S64, &h));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, s->ev0, s->ev1);
  if (rep) {
    rep->converged = fin.stop == DSTOP_CONVERGED;
    rep->rel_residual = h.bb > 0 ? std::sqrt(h.rr / h.bb) : 0.0;
    rep->error_m = std::sqrt(h.rr / (double)s->n);  // the RMS residual, m
    rep->device_ms = ms;
    rep->kernel_launches = launches_now() - l0;
  }
  if (fin.stop == DSTOP_NONFINITE || !std::isfinite(h.rr)) {
    set_error("diffusion solve: a non-finite value appeared");
    return DT_NONFINITE;
  }
  return fin.stop == DSTOP_CONVERGED ? DT_OK : DT_NOT_CONVERGED;
}

dt_status dt_diff_solve(dt_diff* s, double* h_inout, const double* kd, double dt, const dt_diff_params* p, dt_report* rep) {
  if (!s || !h_inout || !kd) {
    set_error("dt_diff_solve: NULL argument");
    return DT_BAD_ARG;
  }
  DT_TRY(diff_check(p, dt));
  size_t bytes = s->n * sizeof(double);
  DT_CUDA(cudaMemcpyAsync(s->kd, kd, bytes, cudaMemcpyHostToDevice, s->stream));
  DT_CUDA(cudaMemcpyAsync(s->b, h_inout, bytes, cudaMemcpyHostToDevice, s->stream));
  dt_status st = diff_solve_loaded(s, dt, p, rep);
  if (st == DT_OK || st == DT_NOT_CONVERGED) {
    DT_CUDA(cudaMemcpyAsync(h_inout, s->x, bytes, cudaMemcpyDeviceToHost, s->stream));
    DT_CUDA(cudaStreamSynchronize(s->stream));
  }
  return st;
}

dt_status dt_diff_solve_dev(dt_diff* s, double* h_inout, const double* kd, double dt, const dt_diff_params* p, dt_report* rep) {
  if (!s || !h_inout || !kd) {
    set_error("dt_diff_solve_dev: NULL argument");
    return DT_BAD_ARG;
  }
  DT_TRY(diff_check(p, dt));
  size_t bytes = s->n * sizeof(double);
  DT_CUDA(cudaMemcpyAsync(s->kd, kd, bytes, cudaMemcpyDeviceToDevice, s->stream));
  DT_CUDA(cudaMemcpyAsync(s->b, h_inout, bytes, cudaMemcpyDeviceToDevice, s->stream));
  dt_status st = diff_solve_loaded(s, dt, p, rep);
  if (st == DT_OK || st == DT_NOT_CONVERGED) {
    DT_CUDA(cudaMemcpyAsync(h_inout, s->x, bytes, cudaMemcpyDeviceToDevice, s->stream));
    DT_CUDA(cudaStreamSynchronize(s->stream));
  }
  return st;
}

dt_status dt_diff_operator(dt_diff* s, const double* kd, double dt, const double* x, double* y) {
  if (!s || !kd || !x || !y) {
    set_error("dt_diff_operator: NULL argument");
    return DT_BAD_ARG;
  }
  size_t bytes = s->n * sizeof(double);
  cudaStream_t st = s->stream;
  DT_CUDA(cudaMemcpyAsync(s->kd, kd, bytes, cudaMemcpyHostToDevice, st));
  DT_CUDA(cudaMemcpyAsync(s->p, x, bytes, cudaMemcpyHostToDevice, st));
  int wrap = s->wrap && s->w > 1;
  k_d_coeffs<<<dgrid(s, s->n), 256, 0, st>>>(s->w, s->h, wrap, s->kd, dt / (s->dx * s->dx), s->east, s->south, s->diag, s->east32,
                                             s->south32, s->diag32);
  k_d_apply<double, float, DA_PLAIN><<<dgrid(s, s->n), 256, 0, st>>>(s->w, s->h, wrap, s->east, s->south, s->diag, s->p, nullptr,
                                                                    s->ap, nullptr, s->partials, s->S64);
  DT_CUDA(cudaGetLastError());
  DT_CUDA(cudaMemcpyAsync(y, s->ap, bytes, cudaMemcpyDeviceToHost, st));
  DT_CUDA(cudaStreamSynchronize(st));
  return DT_OK;
}

// x = the LOD splitting's first guess from h (host arrays; diffusion.rs:370-489)
dt_status dt_diff_lod(dt_diff* s, const double* h, const double* kd, double dt, double* x) {
  if (!s || !h || !kd || !x || !(dt > 0.0)) {
    set_error("dt_diff_lod: bad argument");
    return DT_BAD_ARG;
  }
  size_t bytes = s->n * sizeof(double);
  cudaStream_t st = s->stream;
  DT_CUDA(cudaMemcpyAsync(s->kd, kd, bytes, cudaMemcpyHostToDevice, st));
  DT_CUDA(cudaMemcpyAsync(s->b, h, bytes, cudaMemcpyHostToDevice, st));
  dt_diff_params p;
  dt_diff_default_params(&p);
  p.first_guess = 1;
  DT_TRY(diff_first_guess(s, &p, dt));
  DT_CUDA(cudaGetLastError());
  DT_CUDA(cudaMemcpyAsync(x, s->x, bytes, cudaMemcpyDeviceToHost, st));
  DT_CUDA(cudaStreamSynchronize(st));
  return DT_OK;
}

dt_status dt_diff_vcycle(dt_diff* s, const double* kd, double dt, int cycle, const double* r, float* z, int* levels) {
  if (!s || !kd || !r || !z || (cycle != DT_CYCLE_JACOBI && cycle != DT_CYCLE_RBGS)) {
    set_error("dt_diff_vcycle: bad argument");
    return DT_BAD_ARG;
  }
  size_t bytes = s->n * sizeof(double);
  cudaStream_t st = s->stream;
  DT_CUDA(cudaMemcpyAsync(s->kd, kd, bytes, cudaMemcpyHostToDevice, st));
  DT_CUDA(cudaMemcpyAsync(s->r, r, bytes, cudaMemcpyHostToDevice, st));
  int wrap = s->wrap && s->w > 1;
  k_d_coeffs<<<dgrid(s, s->n), 256, 0, st>>>(s->w, s->h, wrap, s->kd, dt / (s->dx * s->dx), s->east, s->south, s->diag, s->east32,
                                             s->south32, s->diag32);
  Hier<float>& H = s->hf[cycle];
  DT_TRY(build_levels<float>(s, H, cycle == DT_CYCLE_JACOBI ? COARSEST : COARSEST_GS));
  fill_levels<float>(s, H, cycle, st);
  k_convert_dr<<<dgrid(s, s->n), 256, 0, st>>>(s->n, s->r, H.lv[0].r);
  float* zz = vcycle<float>(s, H, 0, cycle, st);
  DT_CUDA(cudaGetLastError());
  DT_CUDA(cudaMemcpyAsync(z, zz, s->n * sizeof(float), cudaMemcpyDeviceToHost, st));
  DT_CUDA(cudaStreamSynchronize(st));
  if (levels) *levels = (int)H.lv.size();
  return DT_OK;
}

// Benchmark support: the CG operator (with p.Ap) and the Gauss-Seidel cycle's two tiled sweep
// pairs on the finest level, each launch timed alone (CUDA events on the handle's stream) after
// a write of a buffer twice the L2, so that it reads its inputs from HBM; ms[k] the mean of
// `reps` launches, bytes[k] the launch's algorithmic bytes (each array read once, each output
// written once). Inputs: x and the levels' r from kd, the coarse correction zero.
dt_status dt_diff_profile_kernels(dt_diff* s, const double* kd, double dt, int reps, double* ms, double* bytes) {
  if (!s || !kd || !ms || !bytes || reps < 1 || !(dt > 0.0)) {
    set_error("dt_diff_profile_kernels: bad argument");
    return DT_BAD_ARG;
  }
  cudaStream_t st = s->stream;
  const size_t n = s->n;
  const int wrap = s->wrap && s->w > 1;
  DT_CUDA(cudaMemcpyAsync(s->kd, kd, n * sizeof(double), cudaMemcpyHostToDevice, st));
  k_d_coeffs<<<dgrid(s, n), 256, 0, st>>>(s->w, s->h, wrap, s->kd, dt / (s->dx * s->dx), s->east, s->south, s->diag, s->east32,
                                          s->south32, s->diag32);
  Hier<float>& HF = s->hf[DT_CYCLE_RBGS];
  Hier<double>& HD = s->hd[DT_CYCLE_RBGS];
  DT_TRY(build_levels<float>(s, HF, COARSEST_GS));
  DT_TRY(build_levels<double>(s, HD, COARSEST_GS));
  if (HF.lv.size() < 2 || gs_colours(HF.lv[0].w, HF.lv[0].wrap) != 2 || !rb2_fits(HF.lv[0])) {
    set_error("dt_diff_profile_kernels: the finest level of a %d x %d raster does not take the tiled sweeps", s->w, s->h);
    return DT_UNSUPPORTED;
  }
  fill_levels<float>(s, HF, DT_CYCLE_RBGS, st);
  fill_levels<double>(s, HD, DT_CYCLE_RBGS, st);
  DT_CUDA(cudaMemcpyAsync(s->p, s->kd, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
  k_convert_dr<<<dgrid(s, n), 256, 0, st>>>(n, s->kd, s->p32);
  k_convert_dr<<<dgrid(s, n), 256, 0, st>>>(n, s->kd, HF.lv[0].r);
  DT_CUDA(cudaMemcpyAsync(HD.lv[0].r, s->kd, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
  DLevel<float> &F0 = HF.lv[0], &F1 = HF.lv[1];
  DLevel<double> &D0 = HD.lv[0], &D1 = HD.lv[1];
  const size_t nc = (size_t)F1.w * F1.h;
  DT_CUDA(cudaMemsetAsync(F1.z, 0, nc * sizeof(float), st));
  DT_CUDA(cudaMemsetAsync(D1.z, 0, nc * sizeof(double), st));
  const unsigned g = dgrid(s, n);
  auto one = [&](int k) {
    switch (k) {
      case 0:
        k_d_apply<double, float, DA_PAP><<<g, 256, 0, st>>>(s->w, s->h, wrap, s->east, s->south, s->diag, s->p, nullptr, s->ap,
                                                            nullptr, s->partials, s->S64);
        break;
      case 1:
        k_d_apply<float, float, DA_PAP><<<g, 256, 0, st>>>(s->w, s->h, wrap, s->east32, s->south32, s->diag32, s->p32, nullptr,
                                                           s->ap32, nullptr, s->partials, s->S32);
        break;
      case 2: launch_rb2<float, true>(s, F0, F1, nullptr, F0.z, st); break;
      case 3: launch_rb2<float, false>(s, F0, F1, F1.z, F0.t, st); break;
      case 4: launch_rb2<double, true>(s, D0, D1, nullptr, D0.z, st); break;
      default: launch_rb2<double, false>(s, D0, D1, D1.z, D0.t, st); break;
    }
  };
  // algorithmic bytes: the operator x, east, south, diag in and y out; the pre-smoothing r, diag,
  // 1/diag, east, south in, z and the coarse r out; the post-smoothing z, the coarse z, r, diag,
  // 1/diag, east, south in and z out
  const double nf = (double)n, ncd = (double)nc;
  const double algo[DT_DIFF_PROFILE_KERNELS] = {40 * nf, 20 * nf, 4 * (6 * nf + ncd), 4 * (7 * nf + ncd),
                                                8 * (6 * nf + ncd), 8 * (7 * nf + ncd)};
  const size_t flush_bytes = (size_t)256 << 20;
  void* flush = nullptr;
  DT_CUDA(cudaMalloc(&flush, flush_bytes));
  cudaEvent_t a = nullptr, b = nullptr;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  dt_status rc = DT_OK;
  for (int k = 0; k < DT_DIFF_PROFILE_KERNELS && rc == DT_OK; ++k) {
    k_d_profile_state<<<1, 1, 0, st>>>(s->S64);
    k_d_profile_state<<<1, 1, 0, st>>>(s->S32);
    one(k);  // warm
    double total = 0.0;
    for (int r = 0; r < reps; ++r) {
      cudaMemsetAsync(flush, r & 0xff, flush_bytes, st);
      cudaEventRecord(a, st);
      one(k);
      cudaEventRecord(b, st);
      cudaEventSynchronize(b);
      float t = 0.f;
      cudaEventElapsedTime(&t, a, b);
      total += t;
    }
    if (cudaGetLastError() != cudaSuccess) {
      set_error("dt_diff_profile_kernels: a launch failed");
      rc = DT_DEVICE_ERROR;
    }
    ms[k] = total / reps;
    bytes[k] = algo[k];
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaStreamSynchronize(st);
  cudaFree(flush);
  return rc;
}

}  // extern "C"

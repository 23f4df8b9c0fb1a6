// Implicit diffusion on the cube grid, preconditioned by one multigrid V-cycle, on the B200: the
// device implementation behind dt_cube_* (include/deeptime_gpu.h) of the reference's
// surface/cube/diffusion.rs::solve with DiffusionSolver::Multigrid and its V-cycle
// (surface/cube/multigrid.rs):
//
//   k_cube_couplings  the operator (diffusion.rs:88-113, :147-240): per cell and neighbour slot
//                     K = dt/mean_area D w, D the side pair's mean diffusivity or, for a diagonal,
//                     the least of its quad's four side means; mu = area / mean_area; diag =
//                     mu + sum K;
//   k_cube_lod_*      the locally one-dimensional first guess (diffusion.rs:315-381): a Thomas
//                     solve per face row, then per face column, couplings across a face's edge
//                     at the old values;
//   the hierarchy     2 x 2 blocks of each face down to <= 64 cells (multigrid.rs:92-186), its
//                     sparsity built on the host once per grid (create), its values per solve on
//                     the device (k_mg_val0, k_mg_valc, k_mg_mass);
//   the V-cycle       damped Jacobi (omega 0.8, two sweeps before and after, the first from
//                     zero), residuals summed over blocks, the coarse correction handed to each
//                     block's cells, 16 sweeps on the coarsest level, all in FP32 with the
//                     reference's products and sums (no fused multiply-adds), so it is the
//                     oracle's cycle bit for bit;
//   CG                FP64, the reference's two passes an iteration (the direction fused with
//                     A p and p.Ap; x, r and r.r), stop at an RMS residual of tol over every cell
//                     or after 400 iterations, then the residual's sum put back in proportion to
//                     each cell's coupling (diffusion.rs:387-500, :283-301).
//
// The grid's geometry (neighbour slots, the coupling Laplacian's weights, the cell areas) comes
// from the caller's CubeGrid at create. The CG loop runs on the device as a CUDA graph (a WHILE
// node, the iteration's tail under an IF node), with one read back at its end.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <vector>

#include "common.cuh"

namespace dt {

constexpr uint32_t CUBE_NO_CELL = 0xFFFFFFFFu;
constexpr float CUBE_OMEGA = 0.8f;     // diffusion/multigrid.rs:45
constexpr int CUBE_NU = 2;             // multigrid.rs:48
constexpr float CUBE_SCALE = 0.5f;     // multigrid.rs:52
constexpr size_t CUBE_COARSEST = 64;   // multigrid.rs:54
constexpr int CUBE_COARSE_SWEEPS = 16; // multigrid.rs:56
constexpr int CUBE_CG_MAX_ITER = 400;  // surface/diffusion.rs:497
constexpr int CUBE_RED_BLOCKS = 592;   // partial sums per reduction (4 per SM)
constexpr size_t CUBE_FUSE_CELLS = 1536;  // levels this small run their part of the cycle in one block
constexpr int CUBE_MAX_FUSED = 24;        // levels one fused launch carries

// ---- the operator ----
__global__ void k_cube_couplings(size_t cells, const uint32_t* __restrict__ slots, const double* __restrict__ lap,
                                 const double* __restrict__ kd, const double* __restrict__ mu, double scale,
                                 double* __restrict__ k, double* __restrict__ s, double* __restrict__ diag) {
  for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < cells; c += (size_t)gridDim.x * blockDim.x) {
    const uint32_t* sl = slots + c * 8;
    auto m2 = [&](size_t x, size_t y) { return __dmul_rn(0.5, __dadd_rn(kd[x], kd[y])); };
    double sum = 0.0;
    for (int slot = 0; slot < 8; ++slot) {
      const uint32_t m = sl[slot];
      double kv = 0.0;
      if (m != CUBE_NO_CELL) {
        double d;
        if ((slot & 1) == 0) {
          d = m2(c, m);
        } else {
          const size_t a = sl[slot - 1], b = sl[(slot + 1) & 7];
          d = fmin(fmin(fmin(m2(c, a), m2(a, m)), m2(m, b)), m2(b, c));
        }
        kv = __dmul_rn(__dmul_rn(scale, d), lap[c * 8 + slot]);
      }
      k[c * 8 + slot] = kv;
      sum = __dadd_rn(sum, kv);
    }
    s[c] = sum;
    diag[c] = __dadd_rn(mu[c], sum);
  }
}

// The operator's row i: diag p_i - sum_slots K p_j
template <class P>
__device__ __forceinline__ double cube_row(size_t i, const uint32_t* __restrict__ slots, const double* __restrict__ k,
                                           const double* __restrict__ diag, P p) {
  double acc = __dmul_rn(diag[i], p(i));
  for (int t = 0; t < 8; ++t) {
    const uint32_t j = slots[i * 8 + t];
    if (j != CUBE_NO_CELL) acc = __dsub_rn(acc, __dmul_rn(k[i * 8 + t], p(j)));
  }
  return acc;
}

__global__ void k_cube_apply(size_t cells, const uint32_t* __restrict__ slots, const double* __restrict__ k,
                             const double* __restrict__ diag, const double* __restrict__ x, double* __restrict__ y) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < cells; i += (size_t)gridDim.x * blockDim.x)
    y[i] = cube_row(i, slots, k, diag, [&](size_t j) { return x[j]; });
}

// ---- deterministic sums: per-block partials in a fixed grid, then one block adds them in order ----
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double sh[32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  v = 0.0;
  if (warp == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    v = lane < nw ? sh[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  }
  __syncthreads();
  return v;  // thread 0 holds the block's sum
}

__global__ void k_cube_finish(int nparts, const double* __restrict__ partials, double* __restrict__ out) {
  double v = 0.0;
  for (int q = threadIdx.x; q < nparts; q += blockDim.x) v += partials[q];
  v = block_sum(v);
  if (threadIdx.x == 0) *out = v;
}

// r = rhs - A x; partial r.r
__global__ void k_cube_resid(size_t cells, const uint32_t* __restrict__ slots, const double* __restrict__ k,
                             const double* __restrict__ diag, const double* __restrict__ rhs, const double* __restrict__ x,
                             double* __restrict__ r, double* __restrict__ partials) {
  double acc = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < cells; i += (size_t)gridDim.x * blockDim.x) {
    const double rv = __dsub_rn(rhs[i], cube_row(i, slots, k, diag, [&](size_t j) { return x[j]; }));
    r[i] = rv;
    acc += rv * rv;
  }
  acc = block_sum(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = acc;
}

// partial a.b
__global__ void k_cube_dot(size_t cells, const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ partials) {
  double acc = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < cells; i += (size_t)gridDim.x * blockDim.x)
    acc += a[i] * b[i];
  acc = block_sum(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = acc;
}

// the direction pn = z + beta po (z alone on the first), A pn, partial pn.A pn (diffusion.rs:407-443)
// loop: the device loop's scalars (null when the host drives the loop): its stop flag ends the
// kernel's work, its iteration count tells the first direction
__global__ void k_cube_direction(size_t cells, const uint32_t* __restrict__ slots, const double* __restrict__ k,
                                 const double* __restrict__ diag, const double* __restrict__ z, const double* __restrict__ po,
                                 const double* __restrict__ beta_p, int first, double* __restrict__ pn,
                                 double* __restrict__ ap, double* __restrict__ partials, const double* __restrict__ loop) {
  if (loop) {
    if (loop[13] != 0.0) return;
    first = loop[12] == 0.0;
  }
  const double beta = first ? 0.0 : *beta_p;
  auto dir = [&](size_t j) { return first ? z[j] : __dadd_rn(z[j], __dmul_rn(beta, po[j])); };
  double acc = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < cells; i += (size_t)gridDim.x * blockDim.x) {
    const double pi = dir(i);
    const double a = cube_row(i, slots, k, diag, dir);
    pn[i] = pi;
    ap[i] = a;
    acc += pi * a;
  }
  acc = block_sum(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = acc;
}

// x += alpha p; r -= alpha A p; partial r.r (diffusion.rs:448-475)
__global__ void k_cube_update(size_t cells, const double* __restrict__ alpha_p, const double* __restrict__ broke,
                              const double* __restrict__ p, const double* __restrict__ ap, double* __restrict__ x,
                              double* __restrict__ r, double* __restrict__ partials, const double* __restrict__ loop) {
  if (*broke != 0.0) return;  // the loop stops before the update
  if (loop && loop[13] != 0.0) return;
  const double alpha = *alpha_p;
  double acc = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < cells; i += (size_t)gridDim.x * blockDim.x) {
    x[i] = __dadd_rn(x[i], __dmul_rn(alpha, p[i]));
    const double rv = __dsub_rn(r[i], __dmul_rn(alpha, ap[i]));
    r[i] = rv;
    acc += rv * rv;
  }
  acc = block_sum(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = acc;
}

// x += kk s / mu, the residual's sum put back (diffusion.rs:290-301)
__global__ void k_cube_putback(size_t cells, const double* __restrict__ kk_p, const double* __restrict__ s,
                               const double* __restrict__ mu, double* __restrict__ x) {
  const double kk = *kk_p;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < cells; i += (size_t)gridDim.x * blockDim.x)
    x[i] = __dadd_rn(x[i], __ddiv_rn(__dmul_rn(kk, s[i]), mu[i]));
}

// rhs = mu h; x = b = h
__global__ void k_cube_start(size_t cells, const double* __restrict__ h, const double* __restrict__ mu,
                             double* __restrict__ rhs, double* __restrict__ x, double* __restrict__ b) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < cells; i += (size_t)gridDim.x * blockDim.x) {
    rhs[i] = __dmul_rn(mu[i], h[i]);
    x[i] = h[i];
    b[i] = h[i];
  }
}

// ---- the LOD first guess (diffusion.rs:315-381, thomas :1029-1046) ----
// Face rows, then face columns, each a tridiagonal (1 + (k_a + k_b)/mu, -k_a/mu, -k_b/mu) solved
// by Thomas, the couplings across a face's edge taken at the old values (b for the rows, the
// rows' answer for the columns).
// Every walk reads contiguous words: k_cube_lod_prep lays out, per cell, the row systems'
// coefficients and right-hand side in face-transposed order (cell (f, i, j) at f n^2 + i n + j,
// so that consecutive face rows are consecutive words) and the column systems' coefficients in
// the cells' own order.
__global__ void k_cube_lod_prep(int n, const uint32_t* __restrict__ slots, const double* __restrict__ k,
                                const double* __restrict__ mu, const double* __restrict__ b, double* __restrict__ rloT,
                                double* __restrict__ rupT, double* __restrict__ rdiT, double* __restrict__ rbT,
                                double* __restrict__ clo, double* __restrict__ cup, double* __restrict__ cdi) {
  const size_t nn = (size_t)n * n, cells = 6 * nn;
  for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < cells; c += (size_t)gridDim.x * blockDim.x) {
    const size_t f = c / nn, rest = c % nn, j = rest / n, i = rest % n, t = f * nn + i * n + j;
    const double ke = k[c * 8 + 0], kw = k[c * 8 + 4], kn = k[c * 8 + 2], ks = k[c * 8 + 6], m = mu[c];
    rloT[t] = __ddiv_rn(-kw, m);
    rupT[t] = __ddiv_rn(-ke, m);
    rdiT[t] = __dadd_rn(1.0, __ddiv_rn(__dadd_rn(ke, kw), m));
    double v = b[c];
    if (i == 0) v = __dadd_rn(v, __ddiv_rn(__dmul_rn(kw, b[slots[c * 8 + 4]]), m));
    if (i == (size_t)n - 1) v = __dadd_rn(v, __ddiv_rn(__dmul_rn(ke, b[slots[c * 8 + 0]]), m));
    rbT[t] = v;
    clo[c] = __ddiv_rn(-kn, m);
    cup[c] = __ddiv_rn(-ks, m);
    cdi[c] = __dadd_rn(1.0, __ddiv_rn(__dadd_rn(kn, ks), m));
  }
}

// Thomas along a line of n values at base + r * stride (r = 0 .. n - 1): x from the line's
// lo, up, di and right-hand side; c: the coefficients (diffusion.rs:1029-1046)
__device__ __forceinline__ void thomas_line(int n, size_t base, size_t stride, const double* __restrict__ lo,
                                            const double* __restrict__ up, const double* __restrict__ di,
                                            const double* __restrict__ rhs, double* __restrict__ x,
                                            double* __restrict__ c) {
  double beta = di[base];
  double prev = __ddiv_rn(rhs[base], beta);
  x[base] = prev;
  for (int r = 1; r < n; ++r) {
    const size_t at = base + (size_t)r * stride;
    const double ci = __ddiv_rn(up[at - stride], beta);
    c[at] = ci;
    beta = __dsub_rn(di[at], __dmul_rn(lo[at], ci));
    prev = __ddiv_rn(__dsub_rn(rhs[at], __dmul_rn(lo[at], prev)), beta);
    x[at] = prev;
  }
  double next = prev;
  for (int r = n - 2; r >= 0; --r) {
    const size_t at = base + (size_t)r * stride;
    next = __dsub_rn(x[at], __dmul_rn(c[at + stride], next));
    x[at] = next;
  }
}

// Face columns in the cells' order: thread (f, i) walks j at f n^2 + j n + i; the right-hand
// side y plus the couplings across the face's north and south edges at y's values (into rhs)
__global__ void k_cube_lod_cols_rhs(int n, const uint32_t* __restrict__ slots, const double* __restrict__ k,
                                    const double* __restrict__ mu, const double* __restrict__ y, double* __restrict__ rhs) {
  const size_t nn = (size_t)n * n, cells = 6 * nn;
  for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < cells; c += (size_t)gridDim.x * blockDim.x) {
    const size_t j = (c % nn) / n;
    double v = y[c];
    if (j == 0) v = __dadd_rn(v, __ddiv_rn(__dmul_rn(k[c * 8 + 2], y[slots[c * 8 + 2]]), mu[c]));
    if (j == (size_t)n - 1) v = __dadd_rn(v, __ddiv_rn(__dmul_rn(k[c * 8 + 6], y[slots[c * 8 + 6]]), mu[c]));
    rhs[c] = v;
  }
}
// One serial walk a line (the rows' transposed systems and the columns' alike: line l = f n + m
// at f n^2 + m + r n): the comparison path of the chunked solves below.
__global__ void k_cube_lod_cols_f(int n, const double* __restrict__ lo, const double* __restrict__ up,
                                  const double* __restrict__ di, const double* __restrict__ rhs, double* __restrict__ x,
                                  double* __restrict__ c) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= 6 * n) return;
  const size_t nn = (size_t)n * n, f = col / n, i = col % n;
  thomas_line(n, f * nn + i, (size_t)n, lo, up, di, rhs, x, c);
}

// The same line solves in chunks, for parallelism: the 6 n lines of n positions at
// f n^2 + m + r n (line l = f n + m, r = 0 .. n - 1) in chunks of CUBE_LOD_CHUNK positions, one
// thread a chunk. With the couplings to the neighbouring chunks moved to the right-hand side,
// x_i = p_i + q_i x_(s-1) + r_i x_e on chunk [s, e): p, q and r solve the chunk's own tridiagonal
// system for the right-hand sides b, -lo_s e_s and -up_(e-1) e_(e-1) (a line's first lo and last
// up couple nothing). k_cube_lod_reduce then solves each line's chunk end values, one thread a
// line, and k_cube_lod_join forms x over p. Every product, quotient and difference is rounded on
// its own, as in thomas_line.
constexpr int CUBE_LOD_CHUNK = 32;
__global__ void __launch_bounds__(128) k_cube_lod_chunks(int n, int P, const double* __restrict__ lo, const double* __restrict__ up,
                                                         const double* __restrict__ di, const double* __restrict__ rhs,
                                                         double* __restrict__ p, double* __restrict__ q, double* __restrict__ r,
                                                         double* __restrict__ c, double* __restrict__ edge) {
  const int L = 6 * n;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= L * P) return;
  const int l = t % L, k = t / L;  // consecutive threads: consecutive lines, consecutive words
  const size_t base = (size_t)(l / n) * n * n + (size_t)(l % n);
  const int s = k * CUBE_LOD_CHUNK, e = min(s + CUBE_LOD_CHUNK, n);
  double bt = 1.0, cprev = 0.0, pv = 0.0, qv = 0.0, rv = 0.0;
  for (int i = s; i < e; ++i) {
    const size_t a = base + (size_t)i * n;
    const double lov = i == 0 ? 0.0 : lo[a];
    const double upv = i == n - 1 ? 0.0 : up[a];
    const double dv = di[a], bv = rhs[a];
    const double rr = i == e - 1 ? -upv : 0.0;
    if (i == s) {
      bt = dv;
      pv = __ddiv_rn(bv, bt);
      qv = __ddiv_rn(-lov, bt);
      rv = __ddiv_rn(rr, bt);
    } else {
      bt = __dsub_rn(dv, __dmul_rn(lov, cprev));
      pv = __ddiv_rn(__dsub_rn(bv, __dmul_rn(lov, pv)), bt);
      qv = __ddiv_rn(-__dmul_rn(lov, qv), bt);
      rv = __ddiv_rn(__dsub_rn(rr, __dmul_rn(lov, rv)), bt);
    }
    cprev = __ddiv_rn(upv, bt);
    c[a] = cprev;
    p[a] = pv;
    q[a] = qv;
    r[a] = rv;
  }
  // back substitution inside the chunk: y_i -= c_i y_(i+1) (the last position's values are final)
  const double e0 = pv, eq = qv, er = rv;
  for (int i = e - 2; i >= s; --i) {
    const size_t a = base + (size_t)i * n;
    const double ci = c[a];
    pv = __dsub_rn(p[a], __dmul_rn(ci, pv));
    qv = __dsub_rn(q[a], __dmul_rn(ci, qv));
    rv = __dsub_rn(r[a], __dmul_rn(ci, rv));
    p[a] = pv;
    q[a] = qv;
    r[a] = rv;
  }
  double* ed = edge + (size_t)t * 6;  // the chunk's first position's p, q, r, then its last's
  ed[0] = pv;
  ed[1] = qv;
  ed[2] = rv;
  ed[3] = e0;
  ed[4] = eq;
  ed[5] = er;
}

// One thread a line: the chunks' first (A_k) and last (B_k) values from A_k = pA + qA B_(k-1) +
// rA A_(k+1) and B_k = pB + qB B_(k-1) + rB A_(k+1) (B_(-1) = A_P = 0): forward with
// B_(k-1) = g + hh A_k, back from A_P; A_k and B_k written over the chunk's p entries.
__global__ void __launch_bounds__(128) k_cube_lod_reduce(int n, int P, double* __restrict__ edge, double* __restrict__ al) {
  const int L = 6 * n;
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= L) return;
  double g = 0.0, hh = 0.0;
  for (int k = 0; k < P; ++k) {
    const double* ed = edge + ((size_t)k * L + l) * 6;
    const double pA = ed[0], qA = ed[1], rA = ed[2], pB = ed[3], qB = ed[4], rB = ed[5];
    const double d = __dsub_rn(1.0, __dmul_rn(qA, hh));
    const double a = __ddiv_rn(__dadd_rn(pA, __dmul_rn(qA, g)), d), be = __ddiv_rn(rA, d);
    double* sk = al + ((size_t)k * L + l) * 4;
    sk[0] = a;
    sk[1] = be;
    g = __dadd_rn(__dadd_rn(pB, __dmul_rn(qB, g)), __dmul_rn(__dmul_rn(qB, hh), a));
    hh = __dadd_rn(__dmul_rn(__dmul_rn(qB, hh), be), rB);
    sk[2] = g;
    sk[3] = hh;
  }
  double An = 0.0;
  for (int k = P - 1; k >= 0; --k) {
    const double* sk = al + ((size_t)k * L + l) * 4;
    const double A = __dadd_rn(sk[0], __dmul_rn(sk[1], An)), B = __dadd_rn(sk[2], __dmul_rn(sk[3], An));
    double* ed = edge + ((size_t)k * L + l) * 6;
    ed[0] = A;
    ed[3] = B;
    An = A;
  }
}

// Every position: x = p + q B_(k-1) + r A_(k+1), over p.
__global__ void __launch_bounds__(256) k_cube_lod_join(int n, int P, double* __restrict__ p, const double* __restrict__ q,
                                                       const double* __restrict__ r, const double* __restrict__ edge) {
  const int L = 6 * n;
  const size_t nn = (size_t)n * n, cells = 6 * nn;
  for (size_t a = blockIdx.x * (size_t)blockDim.x + threadIdx.x; a < cells; a += (size_t)gridDim.x * blockDim.x) {
    const size_t f = a / nn, rest = a % nn;
    const int i = (int)(rest / n), l = (int)(f * n + rest % n), k = i / CUBE_LOD_CHUNK;
    const double Bm = k > 0 ? edge[((size_t)(k - 1) * L + l) * 6 + 3] : 0.0;
    const double Ap = k + 1 < P ? edge[((size_t)(k + 1) * L + l) * 6 + 0] : 0.0;
    p[a] = __dadd_rn(__dadd_rn(p[a], __dmul_rn(q[a], Bm)), __dmul_rn(r[a], Ap));
  }
}

// x (face row-major) from the column pass's face-column-major result
__global__ void k_cube_untranspose(int n, const double* __restrict__ t, double* __restrict__ x) {
  const size_t nn = (size_t)n * n, cells = 6 * nn;
  for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < cells; c += (size_t)gridDim.x * blockDim.x) {
    const size_t f = c / nn, rest = c % nn, j = rest / n, i = rest % n;
    x[c] = t[f * nn + i * n + j];
  }
}

// ---- the V-cycle's levels (multigrid.rs:199-363), FP32 without fused multiply-adds ----
__global__ void k_mg_val0(size_t cells, const uint32_t* __restrict__ slots, const double* __restrict__ k,
                          const double* __restrict__ mu, const double* __restrict__ diag64, const uint32_t* __restrict__ ptr,
                          float* __restrict__ val, float* __restrict__ mass, float* __restrict__ diag) {
  for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < cells; c += (size_t)gridDim.x * blockDim.x) {
    uint32_t at = ptr[c];
    for (int s = 0; s < 8; ++s)
      if (slots[c * 8 + s] != CUBE_NO_CELL) val[at++] = (float)k[c * 8 + s];
    mass[c] = (float)mu[c];
    diag[c] = (float)diag64[c];
  }
}

__global__ void k_mg_valc(size_t nnz, const uint32_t* __restrict__ src_ptr, const uint32_t* __restrict__ src,
                          const float* __restrict__ fval, float* __restrict__ cval) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < nnz; e += (size_t)gridDim.x * blockDim.x) {
    float s = 0.f;
    for (uint32_t q = src_ptr[e]; q < src_ptr[e + 1]; ++q) s = __fadd_rn(s, fval[src[q]]);
    cval[e] = __fmul_rn(CUBE_SCALE, s);
  }
}

__global__ void k_mg_mass(size_t cells, const uint32_t* __restrict__ kid_ptr, const uint32_t* __restrict__ kids,
                          const float* __restrict__ fmass, const uint32_t* __restrict__ ptr, const float* __restrict__ val,
                          float* __restrict__ mass, float* __restrict__ diag) {
  for (size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x; r < cells; r += (size_t)gridDim.x * blockDim.x) {
    float s = 0.f;
    for (uint32_t q = kid_ptr[r]; q < kid_ptr[r + 1]; ++q) s = __fadd_rn(s, fmass[kids[q]]);
    float kk = 0.f;
    for (uint32_t e = ptr[r]; e < ptr[r + 1]; ++e) kk = __fadd_rn(kk, val[e]);
    mass[r] = s;
    diag[r] = __fadd_rn(s, kk);
  }
}

__device__ __forceinline__ float mg_az(size_t i, const uint32_t* __restrict__ ptr, const uint32_t* __restrict__ col,
                                       const float* __restrict__ val, const float* __restrict__ diag,
                                       const float* __restrict__ z) {
  float az = __fmul_rn(diag[i], z[i]);
  for (uint32_t e = ptr[i]; e < ptr[i + 1]; ++e) az = __fsub_rn(az, __fmul_rn(val[e], z[col[e]]));
  return az;
}

__global__ void k_mg_sweep_first(size_t cells, const float* __restrict__ r, const float* __restrict__ diag, float* __restrict__ z) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < cells; i += (size_t)gridDim.x * blockDim.x)
    z[i] = __fdiv_rn(__fmul_rn(CUBE_OMEGA, r[i]), diag[i]);
}

__global__ void k_mg_sweep(size_t cells, const uint32_t* __restrict__ ptr, const uint32_t* __restrict__ col,
                           const float* __restrict__ val, const float* __restrict__ diag, const float* __restrict__ r,
                           const float* __restrict__ z, float* __restrict__ t) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < cells; i += (size_t)gridDim.x * blockDim.x) {
    const float az = mg_az(i, ptr, col, val, diag, z);
    t[i] = __fadd_rn(z[i], __fdiv_rn(__fmul_rn(CUBE_OMEGA, __fsub_rn(r[i], az)), diag[i]));
  }
}

__global__ void k_mg_resid(size_t cells, const uint32_t* __restrict__ ptr, const uint32_t* __restrict__ col,
                           const float* __restrict__ val, const float* __restrict__ diag, const float* __restrict__ r,
                           const float* __restrict__ z, float* __restrict__ t) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < cells; i += (size_t)gridDim.x * blockDim.x)
    t[i] = __fsub_rn(r[i], mg_az(i, ptr, col, val, diag, z));
}

__global__ void k_mg_restrict(size_t cells, const uint32_t* __restrict__ kid_ptr, const uint32_t* __restrict__ kids,
                              const float* __restrict__ t, float* __restrict__ rc) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < cells; q += (size_t)gridDim.x * blockDim.x) {
    float s = 0.f;
    for (uint32_t e = kid_ptr[q]; e < kid_ptr[q + 1]; ++e) s = __fadd_rn(s, t[kids[e]]);
    rc[q] = s;
  }
}

__global__ void k_mg_prolong(size_t cells, const uint32_t* __restrict__ parent, const float* __restrict__ zc, float* __restrict__ z) {
  for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < cells; c += (size_t)gridDim.x * blockDim.x)
    z[c] = __fadd_rn(z[c], zc[parent[c]]);
}

__global__ void k_to_f32(size_t n, const double* __restrict__ a, float* __restrict__ b) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) b[i] = (float)a[i];
}
__global__ void k_to_f64(size_t n, const float* __restrict__ a, double* __restrict__ b) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) b[i] = (double)a[i];
}

// The coarse levels' part of the V-cycle in one block of 1024 threads: the launches of those
// levels (sweeps, residual, restriction, the coarsest level's sweeps, prolongation) in the same
// order and with the same arithmetic per cell, a block barrier where a launch ended. The vectors
// written here are read through plain pointers (not the read-only path), so that every phase sees
// the last one's writes.
struct MgLevelDev {
  unsigned cells;
  const uint32_t *ptr, *col, *kid_ptr, *kids, *parent;
  const float *val, *diag;
  float *r, *z, *t;
};
struct MgCoarse {
  int count;  // levels carried; the last is the coarsest
  MgLevelDev lv[CUBE_MAX_FUSED];
};

__device__ __forceinline__ float mg_az_plain(unsigned i, const MgLevelDev& L, const float* z) {
  float az = __fmul_rn(L.diag[i], z[i]);
  for (uint32_t e = L.ptr[i]; e < L.ptr[i + 1]; ++e) az = __fsub_rn(az, __fmul_rn(L.val[e], z[L.col[e]]));
  return az;
}

__global__ void __launch_bounds__(1024) k_mg_coarse_cycle(MgCoarse m) {
  const unsigned tid = threadIdx.x, nt = blockDim.x;
  float* z[CUBE_MAX_FUSED];
  float* t[CUBE_MAX_FUSED];
  for (int l = 0; l < m.count; ++l) {
    z[l] = m.lv[l].z;
    t[l] = m.lv[l].t;
  }
  auto sweep = [&](int l, bool first) {
    const MgLevelDev& L = m.lv[l];
    if (first) {
      for (unsigned i = tid; i < L.cells; i += nt) z[l][i] = __fdiv_rn(__fmul_rn(CUBE_OMEGA, L.r[i]), L.diag[i]);
    } else {
      for (unsigned i = tid; i < L.cells; i += nt) {
        const float az = mg_az_plain(i, L, z[l]);
        t[l][i] = __fadd_rn(z[l][i], __fdiv_rn(__fmul_rn(CUBE_OMEGA, __fsub_rn(L.r[i], az)), L.diag[i]));
      }
      float* q = z[l];
      z[l] = t[l];
      t[l] = q;
    }
    __syncthreads();
  };
  const int last = m.count - 1;
  for (int l = 0; l < last; ++l) {
    for (int k = 0; k < CUBE_NU; ++k) sweep(l, k == 0);
    const MgLevelDev& L = m.lv[l];
    for (unsigned i = tid; i < L.cells; i += nt) t[l][i] = __fsub_rn(L.r[i], mg_az_plain(i, L, z[l]));
    __syncthreads();
    const MgLevelDev& C = m.lv[l + 1];
    for (unsigned q = tid; q < C.cells; q += nt) {
      float sum = 0.f;
      for (uint32_t e = C.kid_ptr[q]; e < C.kid_ptr[q + 1]; ++e) sum = __fadd_rn(sum, t[l][C.kids[e]]);
      C.r[q] = sum;
    }
    __syncthreads();
  }
  for (int k = 0; k < CUBE_COARSE_SWEEPS; ++k) sweep(last, k == 0);
  for (int l = last - 1; l >= 0; --l) {
    const MgLevelDev& L = m.lv[l];
    const MgLevelDev& C = m.lv[l + 1];
    for (unsigned c = tid; c < L.cells; c += nt) z[l][c] = __fadd_rn(z[l][c], z[l + 1][C.parent[c]]);
    __syncthreads();
    for (int k = 0; k < CUBE_NU; ++k) sweep(l, false);
  }
}

// alpha = rz / pap; beta = rz_new / rz, rz = rz_new (the CG scalars, on the device)
// alpha = rz / pap, or the breakdown flag (pap not positive, or NaN: diffusion.rs:444-446)
__global__ void k_cube_alpha(const double* __restrict__ rz, const double* __restrict__ pap, double* __restrict__ alpha,
                             double* __restrict__ broke, const double* __restrict__ loop) {
  if (loop && loop[13] != 0.0) return;
  const double p = *pap;
  if (isnan(p) || p <= 0.0) {
    *broke = 1.0;
  } else {
    *broke = 0.0;
    *alpha = *rz / p;
  }
}
__global__ void k_cube_beta(const double* __restrict__ rz_new, double* __restrict__ rz, double* __restrict__ beta) {
  *beta = *rz_new / *rz;
  *rz = *rz_new;
}

// The device loop's control: sc[12] iterations, sc[13] the stop flag, sc[14] tol^2 n, sc[15] the
// iteration cap. After an iteration's update (or its breakdown): the host loop's tests, the
// WHILE node's condition and the IF node's around the iteration's tail (preconditioner, r.z,
// beta), so that nothing runs after the stop.
__global__ void k_cube_arm(const double* __restrict__ sc, unsigned long long while_h) {
  cudaGraphSetConditional((cudaGraphConditionalHandle)while_h, sc[13] == 0.0 ? 1u : 0u);
}
__global__ void k_cube_check(double* __restrict__ sc, unsigned long long while_h, unsigned long long if_h) {
  bool stop = sc[13] != 0.0;
  if (!stop) {
    if (sc[10] != 0.0) {  // p.Ap not positive or NaN: no update (diffusion.rs:444-446)
      stop = true;
    } else {
      sc[0] = sc[11];
      sc[12] += 1.0;
      stop = sc[11] <= sc[14] || sc[12] >= sc[15];
    }
  }
  if (stop) sc[13] = 1.0;
  cudaGraphSetConditional((cudaGraphConditionalHandle)while_h, stop ? 0u : 1u);
  cudaGraphSetConditional((cudaGraphConditionalHandle)if_h, stop ? 0u : 1u);
}
__global__ void k_cube_copy(size_t cells, const double* __restrict__ a, double* __restrict__ b) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < cells; i += (size_t)gridDim.x * blockDim.x) b[i] = a[i];
}

// partials of (rhs - ap) and of s, for the put-back
__global__ void k_cube_lost(size_t cells, const double* __restrict__ rhs, const double* __restrict__ ap,
                            const double* __restrict__ s, double* __restrict__ partials) {
  double a = 0.0, w = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < cells; i += (size_t)gridDim.x * blockDim.x) {
    a += rhs[i] - ap[i];
    w += s[i];
  }
  a = block_sum(a);
  w = block_sum(w);
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = a;
    partials[CUBE_RED_BLOCKS + blockIdx.x] = w;
  }
}

}  // namespace dt

using namespace dt;

namespace {

// One level of the hierarchy: its sparsity (device), its values and vectors.
struct CubeLevel {
  size_t cells = 0, nnz = 0, side = 0;
  uint32_t *ptr = nullptr, *col = nullptr;                      // CSR neighbours
  uint32_t *src_ptr = nullptr, *src = nullptr;                  // level >= 1: the finer entries summed
  uint32_t *kid_ptr = nullptr, *kids = nullptr, *parent = nullptr;  // level >= 1: blocks
  float *val = nullptr, *mass = nullptr, *diag = nullptr, *r = nullptr, *z = nullptr, *t = nullptr;
};

// The hierarchy's sparsity on the host (multigrid.rs:65-186), built once per grid.
struct HostPattern {
  size_t side = 0, cells = 0;
  std::vector<uint32_t> ptr, col, src_ptr, src, kid_ptr, kids, parent;
};

HostPattern finest_pattern(size_t n, const uint32_t* slots) {
  HostPattern p;
  p.side = n;
  p.cells = 6 * n * n;
  p.ptr.push_back(0);
  for (size_t c = 0; c < p.cells; ++c) {
    for (int k = 0; k < 8; ++k)
      if (slots[c * 8 + k] != CUBE_NO_CELL) p.col.push_back(slots[c * 8 + k]);
    p.ptr.push_back((uint32_t)p.col.size());
  }
  return p;
}

HostPattern coarser_pattern(const HostPattern& f) {
  const size_t nf = f.side, m = (nf + 1) / 2, cells = 6 * m * m;
  HostPattern p;
  p.side = m;
  p.cells = cells;
  p.parent.resize(f.cells);
  for (size_t c = 0; c < f.cells; ++c) {
    const size_t face = c / (nf * nf), rest = c % (nf * nf), i = rest % nf, j = rest / nf;
    p.parent[c] = (uint32_t)(face * m * m + (j / 2) * m + i / 2);
  }
  p.kid_ptr.assign(cells + 1, 0);
  for (uint32_t q : p.parent) p.kid_ptr[q + 1] += 1;
  for (size_t k = 0; k < cells; ++k) p.kid_ptr[k + 1] += p.kid_ptr[k];
  std::vector<uint32_t> fill(p.kid_ptr.begin(), p.kid_ptr.end() - 1);
  p.kids.resize(f.cells);
  for (size_t c = 0; c < f.cells; ++c) p.kids[fill[p.parent[c]]++] = (uint32_t)c;
  // each coarse cell's neighbours ascending, and per neighbour the fine entries in their order
  p.ptr.push_back(0);
  p.src_ptr.push_back(0);
  std::vector<std::pair<uint32_t, uint32_t>> pairs;
  for (size_t r = 0; r < cells; ++r) {
    pairs.clear();
    for (uint32_t q = p.kid_ptr[r]; q < p.kid_ptr[r + 1]; ++q) {
      const uint32_t c = p.kids[q];
      for (uint32_t e = f.ptr[c]; e < f.ptr[c + 1]; ++e) {
        const uint32_t to = p.parent[f.col[e]];
        if (to != r) pairs.push_back({to, e});
      }
    }
    std::stable_sort(pairs.begin(), pairs.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    for (size_t k = 0; k < pairs.size(); ++k) {
      if (k == 0 || pairs[k].first != pairs[k - 1].first) {
        if (k > 0) p.src_ptr.push_back((uint32_t)p.src.size());
        p.col.push_back(pairs[k].first);
      }
      p.src.push_back(pairs[k].second);
    }
    if (!pairs.empty()) p.src_ptr.push_back((uint32_t)p.src.size());
    p.ptr.push_back((uint32_t)p.col.size());
  }
  return p;
}

unsigned int cube_grid(size_t n) { return std::max(1u, std::min<unsigned int>(ceil_div(n, 256), 148u * 8u)); }

}  // namespace

struct dt_cube {
  int n = 0;
  size_t cells = 0;
  double mean_area = 0.0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::vector<void*> allocs;
  size_t nalloc = 0;  // device allocations made (the DT_FAIL_ALLOC_AT test hook counts them)
  uint32_t* slots = nullptr;
  double *lap = nullptr, *mu = nullptr;
  double *kd = nullptr, *h = nullptr;  // staging for the host entry points
  double *k = nullptr, *s = nullptr, *diag = nullptr;
  double *rhs = nullptr, *x = nullptr, *b = nullptr, *tmp = nullptr, *cb = nullptr;
  double* lodw[7] = {};  // the LOD's row systems (transposed) and column systems
  // the chunked line solves' scratch: q, r (a value a cell), the chunks' end records (6 a chunk)
  // and the reduction's (4 a chunk); DT_CUBE_LOD_CHUNKED=0 at create keeps one serial walk a line
  double *lq = nullptr, *lr = nullptr, *ledge = nullptr, *lal = nullptr;
  bool lod_chunked = true;
  double *r = nullptr, *z = nullptr, *po = nullptr, *pn = nullptr, *ap = nullptr;
  double* partials = nullptr;
  double* sc = nullptr;  // scalars: 0 rr, 1 pap, 2 rz, 3 rz_new, 4 alpha, 5 beta, 6 lost, 7 weight, 8 kk, 9 rhs.rhs,
                        // 10 breakdown flag, 11 the update's r.r
  std::vector<CubeLevel> levels;
  // The V-cycle's launches as CUDA graphs. Every level swaps its sweep buffers an odd number of
  // times a cycle, so the buffers alternate between two layouts: one graph for each, captured on
  // first use.
  cudaGraphExec_t vcycle_exec[2] = {nullptr, nullptr};
  int vcycle_layout = 0;
  // the CG loop as a graph (a WHILE node over one iteration, the tail under an IF node), made on
  // the first solve; DT_CUBE_HOST_LOOP=1 at create drives the loop from the host instead (the
  // same kernels, three scalars read back an iteration)
  cudaGraphExec_t cg_exec = nullptr;
  cudaStream_t aside = nullptr;
  bool host_loop = false;
  // levels of at most this many cells run their part of the cycle in one block; the environment
  // variable DT_CUBE_FUSE_CELLS, read at dt_cube_create, overrides it (0: every level launches
  // its own kernels, the form the fused block reproduces bit for bit)
  size_t fuse_cells = 0;
};

namespace {

template <class T>
dt_status cube_alloc(dt_cube* s, T** p, size_t count) {
  void* q = nullptr;
  if (alloc_fault(s->nalloc)) {
    set_error("cudaMalloc of %zu bytes failed: out of memory (DT_FAIL_ALLOC_AT)", count * sizeof(T));
    return DT_OOM;
  }
  cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T));
  if (e != cudaSuccess) {
    set_error("dt_cube: cudaMalloc of %zu bytes failed: %s", count * sizeof(T), cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? DT_OOM : DT_DEVICE_ERROR;
  }
  s->allocs.push_back(q);
  *p = reinterpret_cast<T*>(q);
  return DT_OK;
}

template <class T>
dt_status cube_upload(dt_cube* s, T** p, const std::vector<T>& v) {
  DT_TRY(cube_alloc(s, p, v.size()));
  if (!v.empty()) DT_CUDA(cudaMemcpy(*p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  return DT_OK;
}

// the sum of n values of partials, in a fixed order, into *out
void cube_finish(dt_cube* s, const double* partials, double* out) {
  k_cube_finish<<<1, 1024, 0, s->stream>>>(CUBE_RED_BLOCKS, partials, out);
}

// K, s, diag for kd and dt (Workspace::build with every cell, diffusion.rs:147-240)
void cube_build(dt_cube* s, const double* kd, double dt) {
  k_cube_couplings<<<cube_grid(s->cells), 256, 0, s->stream>>>(s->cells, s->slots, s->lap, kd, s->mu, dt / s->mean_area,
                                                               s->k, s->s, s->diag);
}

// the hierarchy's values for the built operator (multigrid.rs:199-269)
void cube_prepare(dt_cube* s) {
  CubeLevel& l0 = s->levels[0];
  k_mg_val0<<<cube_grid(s->cells), 256, 0, s->stream>>>(s->cells, s->slots, s->k, s->mu, s->diag, l0.ptr, l0.val, l0.mass,
                                                        l0.diag);
  for (size_t l = 1; l < s->levels.size(); ++l) {
    CubeLevel &f = s->levels[l - 1], &c = s->levels[l];
    k_mg_valc<<<cube_grid(c.nnz), 256, 0, s->stream>>>(c.nnz, c.src_ptr, c.src, f.val, c.val);
    k_mg_mass<<<cube_grid(c.cells), 256, 0, s->stream>>>(c.cells, c.kid_ptr, c.kids, f.mass, c.ptr, c.val, c.mass, c.diag);
  }
}

void cube_sweep(dt_cube* s, CubeLevel& lv, bool first) {
  if (first) {
    k_mg_sweep_first<<<cube_grid(lv.cells), 256, 0, s->stream>>>(lv.cells, lv.r, lv.diag, lv.z);
    return;
  }
  k_mg_sweep<<<cube_grid(lv.cells), 256, 0, s->stream>>>(lv.cells, lv.ptr, lv.col, lv.val, lv.diag, lv.r, lv.z, lv.t);
  std::swap(lv.z, lv.t);
}

// The cycle from level l0 down in one block (k_mg_coarse_cycle). The host's view of each level's
// z and t then takes the swaps the replaced launches make: NU - 1 + NU on a level with a coarser
// one below, COARSE_SWEEPS - 1 on the coarsest.
void cube_coarse_cycle(dt_cube* s, size_t l0) {
  MgCoarse m{};
  m.count = (int)(s->levels.size() - l0);
  for (int i = 0; i < m.count; ++i) {
    const CubeLevel& lv = s->levels[l0 + i];
    m.lv[i] = MgLevelDev{(unsigned)lv.cells, lv.ptr, lv.col, lv.kid_ptr, lv.kids, lv.parent, lv.val, lv.diag, lv.r, lv.z, lv.t};
  }
  k_mg_coarse_cycle<<<1, 1024, 0, s->stream>>>(m);
  for (size_t l = l0; l < s->levels.size(); ++l) {
    const int swaps = l + 1 == s->levels.size() ? CUBE_COARSE_SWEEPS - 1 : 2 * CUBE_NU - 1;
    if (swaps & 1) std::swap(s->levels[l].z, s->levels[l].t);
  }
}

// multigrid.rs:312-363
void cube_vcycle(dt_cube* s, size_t l) {
  CubeLevel& lv = s->levels[l];
  if (lv.cells <= s->fuse_cells && s->levels.size() - l <= (size_t)CUBE_MAX_FUSED) {
    cube_coarse_cycle(s, l);
    return;
  }
  if (l + 1 == s->levels.size()) {
    for (int k = 0; k < CUBE_COARSE_SWEEPS; ++k) cube_sweep(s, lv, k == 0);
    return;
  }
  for (int k = 0; k < CUBE_NU; ++k) cube_sweep(s, lv, k == 0);
  k_mg_resid<<<cube_grid(lv.cells), 256, 0, s->stream>>>(lv.cells, lv.ptr, lv.col, lv.val, lv.diag, lv.r, lv.z, lv.t);
  CubeLevel& cl = s->levels[l + 1];
  k_mg_restrict<<<cube_grid(cl.cells), 256, 0, s->stream>>>(cl.cells, cl.kid_ptr, cl.kids, lv.t, cl.r);
  cube_vcycle(s, l + 1);
  k_mg_prolong<<<cube_grid(lv.cells), 256, 0, s->stream>>>(lv.cells, cl.parent, cl.z, lv.z);
  for (int k = 0; k < CUBE_NU; ++k) cube_sweep(s, lv, false);
}

// z = V-cycle(r) (multigrid.rs:271-282)
void cube_precondition_launches(dt_cube* s, const double* r, double* z) {
  CubeLevel& l0 = s->levels[0];
  k_to_f32<<<cube_grid(s->cells), 256, 0, s->stream>>>(s->cells, r, l0.r);
  cube_vcycle(s, 0);
  k_to_f64<<<cube_grid(s->cells), 256, 0, s->stream>>>(s->cells, l0.z, z);
}

// z = V-cycle(r) for the handle's r and z, through the graph of the current buffer layout
// (captured the first time; capturing runs the host side of the cycle, which leaves the layout
// flipped as the graph's run does)
dt_status cube_precondition(dt_cube* s) {
  const int lay = s->vcycle_layout;
  if (!s->vcycle_exec[lay]) {
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      // a stream that cannot be captured (the legacy default stream): the launches themselves
      cudaGetLastError();
      cube_precondition_launches(s, s->r, s->z);
      s->vcycle_layout ^= 1;
      return DT_OK;
    }
    cube_precondition_launches(s, s->r, s->z);
    DT_CUDA(cudaStreamEndCapture(s->stream, &g));
    cudaError_t e = cudaGraphInstantiate(&s->vcycle_exec[lay], g, 0);
    cudaGraphDestroy(g);
    DT_CUDA(e);
  } else {
    for (CubeLevel& lv : s->levels) std::swap(lv.z, lv.t);  // the layout the run leaves
  }
  DT_CUDA(cudaGraphLaunch(s->vcycle_exec[lay], s->stream));
  s->vcycle_layout ^= 1;
  return DT_OK;
}

// the LOD first guess: x from b (diffusion.rs:315-381)
void cube_lod(dt_cube* s, const double* b, double* x) {
  const int rows = 6 * s->n;
  double** w = s->lodw;
  // the systems laid out for contiguous walks; the rows' answer comes back transposed in tmp
  k_cube_lod_prep<<<cube_grid(s->cells), 256, 0, s->stream>>>(s->n, s->slots, s->k, s->mu, b, w[0], w[1], w[2], w[3], w[4],
                                                              w[5], w[6]);
  const int P = (s->n + CUBE_LOD_CHUNK - 1) / CUBE_LOD_CHUNK;
  // one pass of line solves: x over the lines' systems (lo, up, di, rhs)
  auto lines = [&](const double* lo, const double* up, const double* di, const double* rhs, double* out) {
    if (!s->lod_chunked) {
      k_cube_lod_cols_f<<<ceil_div(rows, 128), 128, 0, s->stream>>>(s->n, lo, up, di, rhs, out, s->cb);
      return;
    }
    k_cube_lod_chunks<<<ceil_div((size_t)rows * P, 128), 128, 0, s->stream>>>(s->n, P, lo, up, di, rhs, out, s->lq, s->lr, s->cb,
                                                                             s->ledge);
    k_cube_lod_reduce<<<ceil_div(rows, 128), 128, 0, s->stream>>>(s->n, P, s->ledge, s->lal);
    k_cube_lod_join<<<cube_grid(s->cells), 256, 0, s->stream>>>(s->n, P, out, s->lq, s->lr, s->ledge);
  };
  lines(w[0], w[1], w[2], w[3], s->tmp);
  k_cube_untranspose<<<cube_grid(s->cells), 256, 0, s->stream>>>(s->n, s->tmp, x);
  k_cube_lod_cols_rhs<<<cube_grid(s->cells), 256, 0, s->stream>>>(s->n, s->slots, s->k, s->mu, x, w[3]);
  lines(w[4], w[5], w[6], w[3], x);
}

// One device scalar to the host (a sync); a device error reads as NaN, which ends the loop and
// is reported as DT_NONFINITE or by the final error check.
double read_scalar(dt_cube* s, int i) {
  double v = 0.0;
  if (cudaMemcpyAsync(&v, s->sc + i, sizeof(double), cudaMemcpyDeviceToHost, s->stream) != cudaSuccess ||
      cudaStreamSynchronize(s->stream) != cudaSuccess)
    return std::nan("");
  return v;
}

// The CG loop as a graph, made once per handle: arm -> WHILE { direction + A p + p.Ap, alpha, x and
// r with r.r, the stop test; IF not stopped { p_old = p, the V-cycle, r.z, beta } }. The same
// kernels and values as the host-driven loop; the buffers are fixed, so the new direction is
// copied to p_old where the host loop swaps the two.
dt_status cube_cg_graph(dt_cube* s) {
  if (s->cg_exec) return DT_OK;
  if (!s->aside) DT_CUDA(cudaStreamCreateWithFlags(&s->aside, cudaStreamNonBlocking));
  const size_t l = s->cells;
  const unsigned int G = CUBE_RED_BLOCKS;
  cudaGraph_t g = nullptr;
  DT_CUDA(cudaGraphCreate(&g, 0));
  cudaGraphConditionalHandle hw;
  DT_CUDA(cudaGraphConditionalHandleCreate(&hw, g, 0, cudaGraphCondAssignDefault));
  unsigned long long hwv = (unsigned long long)hw;
  double* sc = s->sc;
  void* arm_args[] = {&sc, &hwv};
  cudaKernelNodeParams kp = {};
  kp.func = (void*)k_cube_arm;
  kp.gridDim = dim3(1);
  kp.blockDim = dim3(1);
  kp.kernelParams = arm_args;
  cudaGraphNode_t n_arm, n_loop;
  DT_CUDA(cudaGraphAddKernelNode(&n_arm, g, nullptr, 0, &kp));
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = hw;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  DT_CUDA(cudaGraphAddNode(&n_loop, g, &n_arm, 1, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  cudaGraphConditionalHandle hif;
  DT_CUDA(cudaGraphConditionalHandleCreate(&hif, body, 0, cudaGraphCondAssignDefault));
  const unsigned long long hifv = (unsigned long long)hif;
  if (cudaStreamBeginCaptureToGraph(s->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGraphDestroy(g);
    set_error("dt_cube: the CG loop's graph: the stream cannot be captured");
    return DT_DEVICE_ERROR;
  }
  k_cube_direction<<<G, 256, 0, s->stream>>>(l, s->slots, s->k, s->diag, s->z, s->po, s->sc + 5, 0, s->pn, s->ap, s->partials,
                                             s->sc);
  cube_finish(s, s->partials, s->sc + 1);
  k_cube_alpha<<<1, 1, 0, s->stream>>>(s->sc + 2, s->sc + 1, s->sc + 4, s->sc + 10, s->sc);
  k_cube_update<<<G, 256, 0, s->stream>>>(l, s->sc + 4, s->sc + 10, s->pn, s->ap, s->x, s->r, s->partials, s->sc);
  cube_finish(s, s->partials, s->sc + 11);
  k_cube_check<<<1, 1, 0, s->stream>>>(s->sc, hwv, hifv);
  // the IF node after the head, its body captured on the side stream (the launch helpers use
  // s->stream, so it stands in for the side stream meanwhile; the capture's host-side swaps of
  // the levels' sweep buffers are undone after it)
  cudaError_t err = cudaSuccess;
  {
    cudaStreamCaptureStatus csx;
    unsigned long long id = 0;
    cudaGraph_t cg = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    err = cudaStreamGetCaptureInfo(s->stream, &csx, &id, &cg, &deps, &nd);
    cudaGraphNodeParams ip = {};
    ip.type = cudaGraphNodeTypeConditional;
    ip.conditional.handle = hif;
    ip.conditional.type = cudaGraphCondTypeIf;
    ip.conditional.size = 1;
    cudaGraphNode_t n_if;
    if (err == cudaSuccess) err = cudaGraphAddNode(&n_if, cg, deps, nd, &ip);
    if (err == cudaSuccess) err = cudaStreamUpdateCaptureDependencies(s->stream, &n_if, 1, cudaStreamSetCaptureDependencies);
    if (err == cudaSuccess)
      err = cudaStreamBeginCaptureToGraph(s->aside, ip.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal);
    if (err == cudaSuccess) {
      std::vector<std::pair<float*, float*>> keep;
      for (const CubeLevel& lv : s->levels) keep.emplace_back(lv.z, lv.t);
      cudaStream_t main = s->stream;
      s->stream = s->aside;
      k_cube_copy<<<cube_grid(l), 256, 0, s->stream>>>(l, s->pn, s->po);
      cube_precondition_launches(s, s->r, s->z);
      k_cube_dot<<<G, 256, 0, s->stream>>>(l, s->r, s->z, s->partials);
      cube_finish(s, s->partials, s->sc + 3);
      k_cube_beta<<<1, 1, 0, s->stream>>>(s->sc + 3, s->sc + 2, s->sc + 5);
      s->stream = main;
      for (size_t q = 0; q < s->levels.size(); ++q) {
        s->levels[q].z = keep[q].first;
        s->levels[q].t = keep[q].second;
      }
      cudaGraph_t ifbody = nullptr;
      err = cudaStreamEndCapture(s->aside, &ifbody);
    }
  }
  cudaGraph_t captured = nullptr;
  const cudaError_t end = cudaStreamEndCapture(s->stream, &captured);
  if (err == cudaSuccess) err = end;
  if (err == cudaSuccess) err = cudaGraphInstantiate(&s->cg_exec, g, 0);
  cudaGraphDestroy(g);
  if (err != cudaSuccess) {
    s->cg_exec = nullptr;
    set_error("dt_cube: the CG loop's graph: %s", cudaGetErrorString(err));
    return DT_DEVICE_ERROR;
  }
  return DT_OK;
}

// The solve's two timing events, destroyed on every way out.
struct EventPair {
  cudaEvent_t a = nullptr, b = nullptr;
  ~EventPair() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
};

// diffusion.rs:270-313 and :387-500 on device arrays h (in/out) and kd
dt_status cube_solve(dt_cube* s, double* h, const double* kd, double dt, double tol_m, dt_report* rep) {
  dt_report out{};
  if (std::isnan(dt) || dt <= 0.0) {
    if (rep) *rep = out;
    return DT_OK;
  }
  EventPair ev;
  DT_CUDA(cudaEventCreate(&ev.a));
  DT_CUDA(cudaEventCreate(&ev.b));
  DT_CUDA(cudaEventRecord(ev.a, s->stream));
  const size_t l = s->cells;
  const unsigned int G = CUBE_RED_BLOCKS;
  cube_build(s, kd, dt);
  k_cube_start<<<cube_grid(l), 256, 0, s->stream>>>(l, h, s->mu, s->rhs, s->x, s->b);
  cube_lod(s, s->b, s->x);
  cube_prepare(s);
  const double tol2 = tol_m * tol_m * (double)l;
  k_cube_dot<<<G, 256, 0, s->stream>>>(l, s->rhs, s->rhs, s->partials);
  cube_finish(s, s->partials, s->sc + 9);
  k_cube_resid<<<G, 256, 0, s->stream>>>(l, s->slots, s->k, s->diag, s->rhs, s->x, s->r, s->partials);
  cube_finish(s, s->partials, s->sc + 0);
  double rr = read_scalar(s, 0);
  int iterations = 0;
  if (!(rr <= tol2)) {
    DT_TRY(cube_precondition(s));
    k_cube_dot<<<G, 256, 0, s->stream>>>(l, s->r, s->z, s->partials);
    cube_finish(s, s->partials, s->sc + 2);
    // the loop on the device, one read back at its end; on a stream that cannot be captured (the
    // legacy default stream), driven from the host
    bool host = s->host_loop;
    if (!host && cube_cg_graph(s) != DT_OK) {
      cudaGetLastError();
      host = true;
    }
    if (!host) {
      const double init[4] = {0.0, 0.0, tol2, (double)CUBE_CG_MAX_ITER};
      DT_CUDA(cudaMemcpyAsync(s->sc + 12, init, sizeof init, cudaMemcpyHostToDevice, s->stream));
      DT_CUDA(cudaGraphLaunch(s->cg_exec, s->stream));
      double back[13];
      if (cudaMemcpyAsync(back, s->sc, sizeof back, cudaMemcpyDeviceToHost, s->stream) != cudaSuccess ||
          cudaStreamSynchronize(s->stream) != cudaSuccess) {
        back[0] = std::nan("");
        back[12] = 0.0;
      }
      rr = back[0];
      iterations = (int)back[12];
    }
    for (int it = 0; host && it < CUBE_CG_MAX_ITER; ++it) {
      k_cube_direction<<<G, 256, 0, s->stream>>>(l, s->slots, s->k, s->diag, s->z, s->po, s->sc + 5, it == 0, s->pn, s->ap,
                                                 s->partials, nullptr);
      cube_finish(s, s->partials, s->sc + 1);
      std::swap(s->po, s->pn);
      k_cube_alpha<<<1, 1, 0, s->stream>>>(s->sc + 2, s->sc + 1, s->sc + 4, s->sc + 10, nullptr);
      k_cube_update<<<G, 256, 0, s->stream>>>(l, s->sc + 4, s->sc + 10, s->po, s->ap, s->x, s->r, s->partials, nullptr);
      cube_finish(s, s->partials, s->sc + 11);
      // one read back an iteration: the new r.r and the breakdown flag
      double back[2] = {std::nan(""), 1.0};
      if (cudaMemcpyAsync(back, s->sc + 10, 2 * sizeof(double), cudaMemcpyDeviceToHost, s->stream) != cudaSuccess ||
          cudaStreamSynchronize(s->stream) != cudaSuccess)
        back[0] = 1.0, back[1] = std::nan("");
      if (back[0] != 0.0) {  // pap <= 0 or NaN (or a failed read): no update
        if (std::isnan(back[1])) rr = back[1];
        break;
      }
      rr = back[1];
      DT_CUDA(cudaMemcpyAsync(s->sc + 0, s->sc + 11, sizeof(double), cudaMemcpyDeviceToDevice, s->stream));
      ++iterations;
      if (rr <= tol2) break;
      DT_TRY(cube_precondition(s));
      k_cube_dot<<<G, 256, 0, s->stream>>>(l, s->r, s->z, s->partials);
      cube_finish(s, s->partials, s->sc + 3);
      k_cube_beta<<<1, 1, 0, s->stream>>>(s->sc + 3, s->sc + 2, s->sc + 5);
    }
  }
  // the residual's sum back to the cells, in proportion to their coupling
  k_cube_apply<<<cube_grid(l), 256, 0, s->stream>>>(l, s->slots, s->k, s->diag, s->x, s->ap);
  k_cube_lost<<<G, 256, 0, s->stream>>>(l, s->rhs, s->ap, s->s, s->partials);
  cube_finish(s, s->partials, s->sc + 6);
  cube_finish(s, s->partials + CUBE_RED_BLOCKS, s->sc + 7);
  const double lost = read_scalar(s, 6), weight = read_scalar(s, 7);
  if (weight > 0.0 && lost != 0.0) {
    const double kk = lost / weight;
    DT_CUDA(cudaMemcpyAsync(s->sc + 8, &kk, sizeof(double), cudaMemcpyHostToDevice, s->stream));
    k_cube_putback<<<cube_grid(l), 256, 0, s->stream>>>(l, s->sc + 8, s->s, s->mu, s->x);
  }
  DT_CUDA(cudaMemcpyAsync(h, s->x, l * sizeof(double), cudaMemcpyDeviceToDevice, s->stream));
  DT_CUDA(cudaEventRecord(ev.b, s->stream));
  DT_CUDA(cudaEventSynchronize(ev.b));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ev.a, ev.b);
  DT_CUDA(cudaGetLastError());
  out.iterations = iterations;
  out.converged = rr <= tol2;
  out.error_m = std::sqrt(rr / (double)l);  // the RMS residual the stop reads, m
  const double bb = read_scalar(s, 9);
  out.rel_residual = bb > 0.0 ? std::sqrt(rr / bb) : 0.0;  // ||mu h - A x|| / ||mu h|| before the put-back
  out.device_ms = ms;
  if (rep) *rep = out;
  if (!std::isfinite(rr)) {
    set_error("dt_cube_diff_solve: the residual is not finite");
    return DT_NONFINITE;
  }
  return out.converged ? DT_OK : DT_NOT_CONVERGED;
}

}  // namespace

extern "C" {

dt_status dt_cube_destroy(dt_cube* s) {
  if (!s) return DT_OK;
  if (s->stream) cudaStreamSynchronize(s->stream);
  for (cudaGraphExec_t& e : s->vcycle_exec)
    if (e) cudaGraphExecDestroy(e);
  if (s->cg_exec) cudaGraphExecDestroy(s->cg_exec);
  if (s->aside) cudaStreamDestroy(s->aside);
  for (void* p : s->allocs) cudaFree(p);
  if (s->own_stream && s->stream) cudaStreamDestroy(s->stream);
  delete s;
  return DT_OK;
}

dt_status dt_cube_create(int n, const uint32_t* slots, const double* lap, const double* areas, dt_cube** out) {
  if (!out) {
    set_error("dt_cube_create: out is NULL");
    return DT_BAD_ARG;
  }
  *out = nullptr;
  if (n < 2 || n > 8192 || !slots || !lap || !areas) {
    set_error("dt_cube_create: bad arguments (n %d)", n);
    return DT_BAD_ARG;
  }
  const size_t cells = 6 * (size_t)n * n;
  for (size_t c = 0; c < cells; ++c) {
    if (!(areas[c] > 0.0) || !std::isfinite(areas[c])) {
      set_error("dt_cube_create: area[%zu] is not a positive number", c);
      return DT_BAD_ARG;
    }
    for (int k = 0; k < 8; ++k) {
      const uint32_t m = slots[c * 8 + k];
      if ((m != CUBE_NO_CELL && m >= cells) || !std::isfinite(lap[c * 8 + k])) {
        set_error("dt_cube_create: slot %d of cell %zu is out of range or its weight not finite", k, c);
        return DT_BAD_ARG;
      }
      // only diagonals go missing (a diagonal's coupling reads its two side cells)
      if ((k & 1) == 0 && m == CUBE_NO_CELL) {
        set_error("dt_cube_create: side slot %d of cell %zu is empty", k, c);
        return DT_BAD_ARG;
      }
    }
  }
  auto* s = new dt_cube();
  s->n = n;
  s->fuse_cells = CUBE_FUSE_CELLS;
  if (const char* e = std::getenv("DT_CUBE_FUSE_CELLS")) s->fuse_cells = std::strtoull(e, nullptr, 10);
  if (const char* e = std::getenv("DT_CUBE_HOST_LOOP")) s->host_loop = e[0] == '1';
  s->cells = cells;
  auto fail = [&](dt_status e) {
    dt_cube_destroy(s);
    return e;
  };
  // the mean cell area in the reference's order: per face row, rows in order, faces in order
  // (sphere/cube.rs:437-449)
  double total = 0.0;
  for (int f = 0; f < 6; ++f) {
    double fs = 0.0;
    for (int j = 0; j < n; ++j) {
      double r = 0.0;
      for (int i = 0; i < n; ++i) r += areas[((size_t)f * n + j) * n + i];
      fs += r;
    }
    total += fs;
  }
  s->mean_area = total / (double)cells;
  std::vector<double> mu(cells);
  for (size_t c = 0; c < cells; ++c) mu[c] = areas[c] / s->mean_area;
  if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) {
    set_error("dt_cube_create: cudaStreamCreate failed");
    return fail(DT_DEVICE_ERROR);
  }
  s->own_stream = true;
  dt_status st;
  if ((st = cube_upload(s, &s->slots, std::vector<uint32_t>(slots, slots + cells * 8))) != DT_OK) return fail(st);
  if ((st = cube_upload(s, &s->lap, std::vector<double>(lap, lap + cells * 8))) != DT_OK) return fail(st);
  if ((st = cube_upload(s, &s->mu, mu)) != DT_OK) return fail(st);
  if ((st = cube_alloc(s, &s->k, cells * 8)) != DT_OK) return fail(st);
  for (double** p : {&s->kd, &s->h, &s->s, &s->diag, &s->rhs, &s->x, &s->b, &s->tmp, &s->cb, &s->r, &s->z, &s->po, &s->pn, &s->ap})
    if ((st = cube_alloc(s, p, cells)) != DT_OK) return fail(st);
  for (double*& p : s->lodw)
    if ((st = cube_alloc(s, &p, cells)) != DT_OK) return fail(st);
  {
    const size_t chunks = (size_t)6 * n * ((n + CUBE_LOD_CHUNK - 1) / CUBE_LOD_CHUNK);
    for (double** p : {&s->lq, &s->lr})
      if ((st = cube_alloc(s, p, cells)) != DT_OK) return fail(st);
    if ((st = cube_alloc(s, &s->ledge, chunks * 6)) != DT_OK) return fail(st);
    if ((st = cube_alloc(s, &s->lal, chunks * 4)) != DT_OK) return fail(st);
  }
  if (const char* e = std::getenv("DT_CUBE_LOD_CHUNKED")) s->lod_chunked = e[0] != '0';
  if ((st = cube_alloc(s, &s->partials, 2 * CUBE_RED_BLOCKS)) != DT_OK) return fail(st);
  if ((st = cube_alloc(s, &s->sc, 16)) != DT_OK) return fail(st);
  // the hierarchy (multigrid.rs:170-186): coarsen while a level has more than 64 cells and a side
  // above 1
  std::vector<HostPattern> pats;
  pats.push_back(finest_pattern(n, slots));
  while (!(pats.back().cells <= CUBE_COARSEST || pats.back().side <= 1)) pats.push_back(coarser_pattern(pats.back()));
  s->levels.resize(pats.size());
  for (size_t l = 0; l < pats.size(); ++l) {
    const HostPattern& p = pats[l];
    CubeLevel& lv = s->levels[l];
    lv.cells = p.cells;
    lv.nnz = p.col.size();
    lv.side = p.side;
    if ((st = cube_upload(s, &lv.ptr, p.ptr)) != DT_OK || (st = cube_upload(s, &lv.col, p.col)) != DT_OK) return fail(st);
    if (l > 0 && ((st = cube_upload(s, &lv.src_ptr, p.src_ptr)) != DT_OK || (st = cube_upload(s, &lv.src, p.src)) != DT_OK ||
                  (st = cube_upload(s, &lv.kid_ptr, p.kid_ptr)) != DT_OK || (st = cube_upload(s, &lv.kids, p.kids)) != DT_OK ||
                  (st = cube_upload(s, &lv.parent, p.parent)) != DT_OK))
      return fail(st);
    if ((st = cube_alloc(s, &lv.val, lv.nnz)) != DT_OK) return fail(st);
    for (float** q : {&lv.mass, &lv.diag, &lv.r, &lv.z, &lv.t})
      if ((st = cube_alloc(s, q, lv.cells)) != DT_OK) return fail(st);
  }
  if (cudaDeviceSynchronize() != cudaSuccess) {
    set_error("dt_cube_create: %s", cudaGetErrorString(cudaGetLastError()));
    return fail(DT_DEVICE_ERROR);
  }
  *out = s;
  return DT_OK;
}

dt_status dt_cube_set_stream(dt_cube* s, void* stream) {
  if (!s) {
    set_error("dt_cube_set_stream: NULL handle");
    return DT_BAD_ARG;
  }
  cudaStreamSynchronize(s->stream);
  if (s->own_stream) cudaStreamDestroy(s->stream);
  s->stream = (cudaStream_t)stream;
  s->own_stream = false;
  return DT_OK;
}

int dt_cube_levels(const dt_cube* s) { return s ? (int)s->levels.size() : -1; }

dt_status dt_cube_diff_solve_dev(dt_cube* s, double* h, const double* kd, double dt, double tol_m, dt_report* rep) {
  if (!s || !h || !kd || !(tol_m > 0.0)) {
    set_error("dt_cube_diff_solve_dev: bad arguments");
    return DT_BAD_ARG;
  }
  return cube_solve(s, h, kd, dt, tol_m, rep);
}

dt_status dt_cube_diff_solve(dt_cube* s, double* h, const double* kd, double dt, double tol_m, dt_report* rep) {
  if (!s || !h || !kd || !(tol_m > 0.0)) {
    set_error("dt_cube_diff_solve: bad arguments");
    return DT_BAD_ARG;
  }
  const size_t bytes = s->cells * sizeof(double);
  DT_CUDA(cudaMemcpyAsync(s->h, h, bytes, cudaMemcpyHostToDevice, s->stream));
  DT_CUDA(cudaMemcpyAsync(s->kd, kd, bytes, cudaMemcpyHostToDevice, s->stream));
  dt_status st = cube_solve(s, s->h, s->kd, dt, tol_m, rep);
  if (st != DT_OK && st != DT_NOT_CONVERGED) return st;
  DT_CUDA(cudaMemcpyAsync(h, s->h, bytes, cudaMemcpyDeviceToHost, s->stream));
  DT_CUDA(cudaStreamSynchronize(s->stream));
  return st;
}

// y = A x for kd and dt (host arrays): the built operator (diffusion.rs:64-86)
dt_status dt_cube_operator(dt_cube* s, const double* kd, double dt, const double* x, double* y) {
  if (!s || !kd || !x || !y) {
    set_error("dt_cube_operator: bad arguments");
    return DT_BAD_ARG;
  }
  const size_t bytes = s->cells * sizeof(double);
  DT_CUDA(cudaMemcpyAsync(s->kd, kd, bytes, cudaMemcpyHostToDevice, s->stream));
  DT_CUDA(cudaMemcpyAsync(s->h, x, bytes, cudaMemcpyHostToDevice, s->stream));
  cube_build(s, s->kd, dt);
  k_cube_apply<<<cube_grid(s->cells), 256, 0, s->stream>>>(s->cells, s->slots, s->k, s->diag, s->h, s->ap);
  DT_CUDA(cudaMemcpyAsync(y, s->ap, bytes, cudaMemcpyDeviceToHost, s->stream));
  DT_CUDA(cudaStreamSynchronize(s->stream));
  DT_CUDA(cudaGetLastError());
  return DT_OK;
}

// z = V-cycle(r) on the hierarchy of the operator for kd and dt (host arrays)
dt_status dt_cube_vcycle(dt_cube* s, const double* kd, double dt, const double* r, double* z) {
  if (!s || !kd || !r || !z) {
    set_error("dt_cube_vcycle: bad arguments");
    return DT_BAD_ARG;
  }
  const size_t bytes = s->cells * sizeof(double);
  DT_CUDA(cudaMemcpyAsync(s->kd, kd, bytes, cudaMemcpyHostToDevice, s->stream));
  DT_CUDA(cudaMemcpyAsync(s->r, r, bytes, cudaMemcpyHostToDevice, s->stream));
  cube_build(s, s->kd, dt);
  cube_prepare(s);
  DT_TRY(cube_precondition(s));
  DT_CUDA(cudaMemcpyAsync(z, s->z, bytes, cudaMemcpyDeviceToHost, s->stream));
  DT_CUDA(cudaStreamSynchronize(s->stream));
  DT_CUDA(cudaGetLastError());
  return DT_OK;
}

// the LOD first guess x from h for kd and dt (host arrays; diffusion.rs:315-381)
dt_status dt_cube_lod(dt_cube* s, const double* kd, double dt, const double* h, double* x) {
  if (!s || !kd || !h || !x) {
    set_error("dt_cube_lod: bad arguments");
    return DT_BAD_ARG;
  }
  const size_t bytes = s->cells * sizeof(double);
  DT_CUDA(cudaMemcpyAsync(s->kd, kd, bytes, cudaMemcpyHostToDevice, s->stream));
  DT_CUDA(cudaMemcpyAsync(s->b, h, bytes, cudaMemcpyHostToDevice, s->stream));
  cube_build(s, s->kd, dt);
  cube_lod(s, s->b, s->x);
  DT_CUDA(cudaMemcpyAsync(x, s->x, bytes, cudaMemcpyDeviceToHost, s->stream));
  DT_CUDA(cudaStreamSynchronize(s->stream));
  DT_CUDA(cudaGetLastError());
  return DT_OK;
}

}  // extern "C"

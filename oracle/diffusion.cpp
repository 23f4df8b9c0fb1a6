// Test infrastructure only: the CPU oracle for deep-time's implicit hillslope/marine diffusion
// solve. Only the tests, the smoke check and the benchmark's CPU-baseline leg load this.
//
// A restatement, in C++17 with OpenMP, of crates/deeptime-core/src/ (paths relative to it):
//   diffusion::lod, thomas, cyclic           surface/diffusion.rs:370-489, :1029-1071
//   diffusion::Operator::{new, apply_row}     surface/diffusion.rs:513-664
//   diffusion::cg (Jacobi PCG, every row)     surface/diffusion.rs:749-1026
//   multigrid constants                       surface/diffusion/multigrid.rs:42-56
//   multigrid::Level::{finest, coarsen, apply_row, first_sweep, sweep, restrict_into}
//                                             surface/diffusion/multigrid.rs:96-357
//   multigrid::vcycle, cg_on                  surface/diffusion/multigrid.rs:500-763
//   submarine_kd                              surface/marine.rs:44-59
//   multigrid tests' apply_reference / reference (unpreconditioned CG to 1e-13)
//                                             surface/diffusion/multigrid/tests.rs:17-74
// The reference's row skipping (`Live`) is for the crust-spreading caller and is not restated:
// every row is visited, which is the reference's own `Live::all` path that the multigrid solve
// always takes (surface/diffusion/multigrid.rs:586).
//
// Additions that the reference does not have, each labelled where it is defined: the cycle in
// f64 as well as f32, the red-black Gauss-Seidel V(2,2) cycle to a 16 x 8 coarsest level, and the
// relative-residual stopping rule of the benchmark's configurations.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "oracle.h"

namespace oracle {

struct Dims {
  size_t w, h;
  double dx;
  bool wrap_x;
  size_t cells() const { return w * h; }
};

// surface/diffusion.rs:1029-1046
void thomas(const double* lo, const double* di, const double* up, double* b, size_t n) {
  if (n == 0) return;
  std::vector<double> c(n, 0.0);
  double beta = di[0];
  b[0] /= beta;
  for (size_t i = 1; i < n; ++i) {
    c[i] = up[i - 1] / beta;
    beta = di[i] - lo[i] * c[i];
    b[i] = (b[i] - lo[i] * b[i - 1]) / beta;
  }
  for (size_t i = n - 1; i-- > 0;) {
    double next = b[i + 1];
    b[i] -= c[i + 1] * next;
  }
}

// surface/diffusion.rs:1050-1071
void cyclic(const double* lo, const double* di, const double* up, double alpha, double beta, double* b, size_t n) {
  double gamma = -di[0];
  std::vector<double> bb(di, di + n), l(lo, lo + n), u(up, up + n), x(b, b + n), z(n, 0.0);
  bb[0] = di[0] - gamma;
  bb[n - 1] = di[n - 1] - alpha * beta / gamma;
  l[0] = 0.0;
  u[n - 1] = 0.0;
  thomas(l.data(), bb.data(), u.data(), x.data(), n);
  z[0] = gamma;
  z[n - 1] = alpha;
  thomas(l.data(), bb.data(), u.data(), z.data(), n);
  double fact = (x[0] + beta * x[n - 1] / gamma) / (1.0 + z[0] + beta * z[n - 1] / gamma);
  for (size_t i = 0; i < n; ++i) b[i] = x[i] - fact * z[i];
}

// surface/diffusion.rs:370-489 (every row visited)
void lod(const Dims& d, double* h, const double* kd, double dt) {
  size_t w = d.w, hh = d.h;
  double s2 = d.dx * d.dx;
#pragma omp parallel
  {
    std::vector<double> lo(w), di(w), up(w);
#pragma omp for schedule(static)
    for (long jl = 0; jl < (long)hh; ++jl) {
      size_t j = (size_t)jl;
      double* row = h + j * w;
      const double* krow = kd + j * w;
      auto face = [&](size_t i) -> double {
        if (i + 1 < w) return 0.5 * (krow[i] + krow[i + 1]) * dt / s2;
        if (d.wrap_x && w > 1) return 0.5 * (krow[w - 1] + krow[0]) * dt / s2;
        return 0.0;
      };
      for (size_t i = 0; i < w; ++i) {
        double west = i == 0 ? face(w - 1) : face(i - 1);
        double east = face(i);
        lo[i] = -west;
        up[i] = -east;
        di[i] = 1.0 + west + east;
      }
      if (d.wrap_x && w > 2) {
        double corner_lo = lo[0];
        double corner_up = up[w - 1];
        cyclic(lo.data(), di.data(), up.data(), corner_up, corner_lo, row, w);
      } else {
        if (w == 2 && d.wrap_x) {
          double f = face(0) + face(1);
          lo[1] = -f;
          up[0] = -f;
          di[0] = 1.0 + f;
          di[1] = 1.0 + f;
        }
        lo[0] = 0.0;
        up[w - 1] = 0.0;
        if (w == 1) di[0] = 1.0;
        thomas(lo.data(), di.data(), up.data(), row, w);
      }
    }
  }
#pragma omp parallel
  {
    std::vector<double> col(hh), lo(hh), di(hh), up(hh);
#pragma omp for schedule(static)
    for (long il = 0; il < (long)w; ++il) {
      size_t i = (size_t)il;
      auto face = [&](size_t j) -> double {
        if (j + 1 < hh) return 0.5 * (kd[j * w + i] + kd[(j + 1) * w + i]) * dt / s2;
        return 0.0;
      };
      for (size_t j = 0; j < hh; ++j) col[j] = h[j * w + i];
      for (size_t j = 0; j < hh; ++j) {
        double north = j == 0 ? 0.0 : face(j - 1);
        double south = face(j);
        lo[j] = -north;
        up[j] = -south;
        di[j] = 1.0 + north + south;
      }
      thomas(lo.data(), di.data(), up.data(), col.data(), hh);
      for (size_t j = 0; j < hh; ++j) h[j * w + i] = col[j];
    }
  }
}

// surface/diffusion.rs:513-664: east/south couplings and the diagonal of I + dt L.
struct Operator {
  size_t w, h;
  bool wrap;
  std::vector<double> east, south, diag;

  Operator(const Dims& d, const double* kd, double dt) : w(d.w), h(d.h), wrap(d.wrap_x && d.w > 1) {
    size_t n = w * h;
    double s2 = d.dx * d.dx;
    east.assign(n, 0.0);
    south.assign(n, 0.0);
    diag.assign(n, 0.0);
#pragma omp parallel for schedule(static)
    for (long jl = 0; jl < (long)h; ++jl) {
      size_t j = (size_t)jl;
      const double* krow = kd + j * w;
      for (size_t i = 0; i < w; ++i) {
        if (i + 1 < w)
          east[j * w + i] = 0.5 * (krow[i] + krow[i + 1]) * dt / s2;
        else if (wrap)
          east[j * w + i] = 0.5 * (krow[i] + krow[0]) * dt / s2;
        else
          east[j * w + i] = 0.0;
      }
      if (j + 1 < h) {
        const double* below = kd + (j + 1) * w;
        for (size_t i = 0; i < w; ++i) south[j * w + i] = 0.5 * (krow[i] + below[i]) * dt / s2;
      }
    }
#pragma omp parallel for schedule(static)
    for (long jl = 0; jl < (long)h; ++jl) {
      size_t j = (size_t)jl, c0 = j * w;
      for (size_t i = 0; i < w; ++i) {
        double west = i > 0 ? east[c0 + i - 1] : (wrap ? east[c0 + w - 1] : 0.0);
        double north = j > 0 ? south[c0 - w + i] : 0.0;
        diag[c0 + i] = 1.0 + east[c0 + i] + west + south[c0 + i] + north;
      }
    }
  }

  // Row j of y = A x: diagonal, east, (wrap), west, (wrap), south, north, in that order.
  void apply_row(size_t j, const double* north, const double* cur, const double* southr, double* out) const {
    size_t c0 = j * w;
    const double* dg = diag.data() + c0;
    const double* e = east.data() + c0;
    for (size_t i = 0; i < w; ++i) out[i] = dg[i] * cur[i];
    for (size_t i = 0; i + 1 < w; ++i) out[i] -= e[i] * cur[i + 1];
    if (wrap) out[w - 1] -= e[w - 1] * cur[0];
    for (size_t i = 1; i < w; ++i) out[i] -= e[i - 1] * cur[i - 1];
    if (wrap) out[0] -= e[w - 1] * cur[w - 1];
    if (southr) {
      const double* s = south.data() + c0;
      for (size_t i = 0; i < w; ++i) out[i] -= s[i] * southr[i];
    }
    if (north) {
      const double* a = south.data() + c0 - w;
      for (size_t i = 0; i < w; ++i) out[i] -= a[i] * north[i];
    }
  }
  void apply(const double* x, double* y) const {
#pragma omp parallel for schedule(static)
    for (long jl = 0; jl < (long)h; ++jl) {
      size_t j = (size_t)jl;
      apply_row(j, j > 0 ? x + (j - 1) * w : nullptr, x + j * w, j + 1 < h ? x + (j + 1) * w : nullptr, y + j * w);
    }
  }
};

static double row_ordered_sum(size_t w, size_t h, const std::vector<double>& rows) {
  (void)w;
  double s = 0.0;
  for (size_t j = 0; j < h; ++j) s += rows[j];
  return s;
}

// surface/diffusion.rs:927-1026: Jacobi-preconditioned CG to an RMS residual of 1e-6 m (at most
// 400 iterations), then the mass put-back. Returns the iterations.
int jacobi_cg(const Dims& d, double* x, const double* b, const double* kd, double dt, double tol_m, int max_it) {
  size_t n = d.cells(), w = d.w, h = d.h;
  Operator op(d, kd, dt);
  std::vector<double> r(n), p(n), ap(n), rows(h), z(n);
  op.apply(x, r.data());
  for (size_t k = 0; k < n; ++k) r[k] = b[k] - r[k];
  auto sums = [&](double* rr, double* rz) {
#pragma omp parallel for schedule(static)
    for (long j = 0; j < (long)h; ++j) {
      double a = 0.0;
      for (size_t i = 0; i < w; ++i) {
        double v = r[j * w + i];
        a += v * v;
      }
      rows[j] = a;
    }
    *rr = row_ordered_sum(w, h, rows);
#pragma omp parallel for schedule(static)
    for (long j = 0; j < (long)h; ++j) {
      double a = 0.0;
      for (size_t i = 0; i < w; ++i) {
        double v = r[j * w + i];
        a += v * (v / op.diag[j * w + i]);
      }
      rows[j] = a;
    }
    *rz = row_ordered_sum(w, h, rows);
  };
  double rr, rz;
  sums(&rr, &rz);
  double tol2 = tol_m * tol_m * (double)n;
  int its = 0;
  if (rr > tol2) {
    bool first = true;
    double beta = 0.0;
    while (its < max_it) {
      ++its;
      for (size_t k = 0; k < n; ++k) p[k] = first ? r[k] / op.diag[k] : r[k] / op.diag[k] + beta * p[k];
      first = false;
      op.apply(p.data(), ap.data());
#pragma omp parallel for schedule(static)
      for (long j = 0; j < (long)h; ++j) {
        double a = 0.0;
        for (size_t i = 0; i < w; ++i) a += p[j * w + i] * ap[j * w + i];
        rows[j] = a;
      }
      double pap = row_ordered_sum(w, h, rows);
      if (pap <= 0.0) break;
      double alpha = rz / pap;
      for (size_t k = 0; k < n; ++k) {
        x[k] += alpha * p[k];
        r[k] -= alpha * ap[k];
      }
      double rz_new;
      sums(&rr, &rz_new);
      if (rr <= tol2) break;
      beta = rz_new / rz;
      rz = rz_new;
    }
  }
  // mass put-back, surface/diffusion.rs:991-1024
  op.apply(x, ap.data());
  double lost = 0.0, weight = 0.0;
  for (size_t k = 0; k < n; ++k) lost += b[k] - ap[k];
  for (size_t k = 0; k < n; ++k) weight += op.diag[k] - 1.0;
  if (weight > 0.0 && lost != 0.0) {
    double kk = lost / weight;
    for (size_t k = 0; k < n; ++k) x[k] += kk * (op.diag[k] - 1.0);
  }
  return its;
}

// ---------------------------------------------------------------------------------------------
// The multigrid cycle, surface/diffusion/multigrid.rs:42-523, templated on the level precision.

static const float OMEGA = 0.8f;        // multigrid.rs:45
static const int NU = 2;                // multigrid.rs:48
static const float SCALE = 0.5f;        // multigrid.rs:52
static const size_t COARSEST = 64;      // multigrid.rs:54
static const int COARSE_SWEEPS = 16;    // multigrid.rs:56
// Not in the reference: the benchmark's cycle's coarsest level (16 x 8 cells) and its sweeps.
static const size_t COARSEST_RB = 128;
static const int COARSE_SWEEPS_RB = 8;

template <typename T>
struct Level {
  size_t w, h;
  bool wrap;
  std::vector<T> east, south, diag, wd, mass, r, z, t;

  static Level finest(const Operator& op, T omega) {
    Level l;
    l.w = op.w;
    l.h = op.h;
    l.wrap = op.wrap;
    size_t n = l.w * l.h;
    l.east.resize(n);
    l.south.resize(n);
    l.diag.resize(n);
    l.wd.resize(n);
    for (size_t k = 0; k < n; ++k) {
      l.east[k] = (T)op.east[k];
      l.south[k] = (T)op.south[k];
      l.diag[k] = (T)op.diag[k];
      l.wd[k] = omega / l.diag[k];
    }
    l.r.assign(n, 0);
    l.z.assign(n, 0);
    l.t.assign(n, 0);
    return l;
  }

  // multigrid.rs:117-199
  bool coarsen(T omega, T scale, size_t coarsest, Level& out) const {
    size_t wc = (w + 1) / 2, hc = (h + 1) / 2;
    if (w * h <= coarsest || (wc == w && hc == h)) return false;
    size_t nc = wc * hc;
    bool cwrap = wrap && wc > 1;
    out.w = wc;
    out.h = hc;
    out.wrap = cwrap;
    out.east.assign(nc, 0);
    out.south.assign(nc, 0);
    out.mass.assign(nc, 0);
    for (size_t jc = 0; jc < hc; ++jc) {
      size_t r0 = 2 * jc, r1 = std::min(2 * jc + 2, h), last_row = r1 - 1;
      for (size_t ic = 0; ic < wc; ++ic) {
        size_t c0 = 2 * ic, c1 = std::min(2 * ic + 2, w), last_col = c1 - 1;
        T m = 0;
        for (size_t j = r0; j < r1; ++j)
          for (size_t i = c0; i < c1; ++i) m += mass.empty() ? (T)1 : mass[j * w + i];
        out.mass[jc * wc + ic] = m;
        if (ic + 1 < wc || cwrap) {
          T e = 0;
          for (size_t j = r0; j < r1; ++j) e += east[j * w + last_col];
          out.east[jc * wc + ic] = scale * e;
        }
        if (jc + 1 < hc) {
          T s = 0;
          for (size_t i = c0; i < c1; ++i) s += south[last_row * w + i];
          out.south[jc * wc + ic] = scale * s;
        }
      }
    }
    out.diag.assign(nc, 0);
    out.wd.assign(nc, 0);
    for (size_t j = 0; j < hc; ++j) {
      size_t c0 = j * wc;
      for (size_t i = 0; i < wc; ++i) {
        T west = i > 0 ? out.east[c0 + i - 1] : (cwrap ? out.east[c0 + wc - 1] : (T)0);
        T north = j > 0 ? out.south[c0 - wc + i] : (T)0;
        out.diag[c0 + i] = out.mass[c0 + i] + out.east[c0 + i] + west + out.south[c0 + i] + north;
        out.wd[c0 + i] = omega / out.diag[c0 + i];
      }
    }
    out.r.assign(nc, 0);
    out.z.assign(nc, 0);
    out.t.assign(nc, 0);
    return true;
  }

  // multigrid.rs:202-240
  void apply_row(size_t j, const T* north, const T* cur, const T* southr, T* out) const {
    size_t c0 = j * w;
    const T* dg = diag.data() + c0;
    const T* e = east.data() + c0;
    for (size_t i = 0; i < w; ++i) out[i] = dg[i] * cur[i];
    for (size_t i = 0; i + 1 < w; ++i) out[i] -= e[i] * cur[i + 1];
    for (size_t i = 1; i < w; ++i) out[i] -= e[i - 1] * cur[i - 1];
    if (wrap) {
      out[w - 1] -= e[w - 1] * cur[0];
      out[0] -= e[w - 1] * cur[w - 1];
    }
    if (southr) {
      const T* s = south.data() + c0;
      for (size_t i = 0; i < w; ++i) out[i] -= s[i] * southr[i];
    }
    if (north) {
      const T* a = south.data() + c0 - w;
      for (size_t i = 0; i < w; ++i) out[i] -= a[i] * north[i];
    }
  }

  void first_sweep() {
    for (size_t k = 0; k < w * h; ++k) z[k] = wd[k] * r[k];
  }

  // multigrid.rs:260-329: z <- z' + wd (r - A z'), z' = z + P coarse; with dot, returns sum dot*z.
  double sweep(const T* coarse, size_t wc, const double* dot) {
    std::vector<double> rows(h, 0.0);
#pragma omp parallel
    {
      std::vector<T> r0(w), r1(w), r2(w), ax(w);
      auto corrected = [&](size_t j, T* out) {
        const T* zr = z.data() + j * w;
        if (coarse) {
          const T* crow = coarse + (j / 2) * wc;
          for (size_t i = 0; i < w; ++i) out[i] = zr[i] + crow[i / 2];
        } else {
          std::copy(zr, zr + w, out);
        }
      };
#pragma omp for schedule(static)
      for (long jl = 0; jl < (long)h; ++jl) {
        size_t j = (size_t)jl;
        if (j > 0) corrected(j - 1, r0.data());
        corrected(j, r1.data());
        if (j + 1 < h) corrected(j + 1, r2.data());
        apply_row(j, j > 0 ? r0.data() : nullptr, r1.data(), j + 1 < h ? r2.data() : nullptr, ax.data());
        size_t c0 = j * w;
        T* tr = t.data() + c0;
        for (size_t i = 0; i < w; ++i) tr[i] = r1[i] + wd[c0 + i] * (r[c0 + i] - ax[i]);
        if (dot) {
          double acc = 0.0;
          for (size_t i = 0; i < w; ++i) acc += dot[c0 + i] * (double)tr[i];
          rows[j] = acc;
        }
      }
    }
    std::swap(z, t);
    double s = 0.0;
    for (double v : rows) s += v;
    return s;
  }

  // multigrid.rs:332-356
  void restrict_into(Level& coarse) const {
    size_t wc = coarse.w;
    std::fill(coarse.r.begin(), coarse.r.end(), (T)0);
    std::vector<T> res(w);
    for (size_t jc = 0; jc < coarse.h; ++jc) {
      T* rc = coarse.r.data() + jc * wc;
      for (size_t j = 2 * jc; j < std::min(2 * jc + 2, h); ++j) {
        apply_row(j, j > 0 ? z.data() + (j - 1) * w : nullptr, z.data() + j * w, j + 1 < h ? z.data() + (j + 1) * w : nullptr,
                  res.data());
        const T* rr = r.data() + j * w;
        for (size_t i = 0; i < w; ++i) rc[i / 2] += rr[i] - res[i];
      }
    }
  }

  // Not in the reference (the benchmark's smoother): the colour of cell (i, j) for the multi-colour
  // Gauss-Seidel sweeps. Red/black is (i + j) % 2; on a wrapping level of odd width the ring of a
  // row is an odd cycle, so its last column takes two colours of its own (2 + j % 2). No two
  // cells of one colour are neighbours, so a colour's cells may be updated in any order (or all
  // at once) with the same result.
  int colour(size_t i, size_t j) const {
    if (wrap && (w & 1) && i == w - 1) return 2 + (int)(j & 1);
    return (int)((i + j) & 1);
  }
  int colours() const { return (wrap && (w & 1)) ? 4 : 2; }

  // One Gauss-Seidel pass over the cells of colour `c`: z_c <- z_c + (r - A z)_c / diag_c.
  void rb_half(int c) {
    for (size_t j = 0; j < h; ++j) {
      size_t c0 = j * w;
      for (size_t i = 0; i < w; ++i) {
        if (colour(i, j) != c) continue;
        size_t k = c0 + i;
        T o = diag[k] * z[k];
        if (i + 1 < w) o -= east[k] * z[k + 1];
        if (i > 0) o -= east[k - 1] * z[k - 1];
        if (wrap) {
          if (i == w - 1) o -= east[k] * z[c0];
          if (i == 0) o -= east[c0 + w - 1] * z[c0 + w - 1];
        }
        if (j + 1 < h) o -= south[k] * z[k + w];
        if (j > 0) o -= south[k - w] * z[k - w];
        z[k] = z[k] + (r[k] - o) / diag[k];
      }
    }
  }
  // A forward sweep visits the colours in ascending order, a backward one in descending order.
  void gs_forward() {
    for (int c = 0; c < colours(); ++c) rb_half(c);
  }
  void gs_backward() {
    for (int c = colours(); c-- > 0;) rb_half(c);
  }
};

template <typename T>
struct Hierarchy {
  std::vector<Level<T>> levels;
  int kind;  // DTO_CYCLE_JACOBI (the reference's) or DTO_CYCLE_RBGS (the benchmark's)
  T omega, scale;
  int nu;

  Hierarchy(const Operator& op, int kind_, T omega_, int nu_, T scale_) : kind(kind_), omega(omega_), scale(scale_), nu(nu_) {
    levels.push_back(Level<T>::finest(op, omega));
    size_t coarsest = kind == DTO_CYCLE_RBGS ? COARSEST_RB : COARSEST;
    for (;;) {
      Level<T> next;
      if (!levels.back().coarsen(omega, scale, coarsest, next)) break;
      levels.push_back(std::move(next));
    }
  }

  // multigrid.rs:500-523
  double vcycle_jacobi(size_t li, const double* dot) {
    Level<T>& l = levels[li];
    if (li + 1 == levels.size()) {
      l.first_sweep();
      double acc = 0.0;
      int total = std::max(COARSE_SWEEPS, 2);
      for (int k = 1; k < total; ++k) {
        bool last = k + 1 == total;
        acc = l.sweep(nullptr, 0, last ? dot : nullptr);
      }
      return acc;
    }
    l.first_sweep();
    for (int k = 1; k < nu; ++k) l.sweep(nullptr, 0, nullptr);
    l.restrict_into(levels[li + 1]);
    vcycle_jacobi(li + 1, nullptr);
    size_t wc = levels[li + 1].w;
    double acc = l.sweep(levels[li + 1].z.data(), wc, nu == 1 ? dot : nullptr);
    for (int k = 1; k < nu; ++k) acc = l.sweep(nullptr, 0, k + 1 == nu ? dot : nullptr);
    return acc;
  }

  // Not in the reference: the benchmark's symmetric red-black Gauss-Seidel V(nu, nu) cycle from z = 0.
  // Pre-smoothing sweeps the colours forward, post-smoothing backward (the adjoint order), so the
  // cycle is a symmetric positive definite operator; the coarsest level takes COARSE_SWEEPS_RB
  // forward sweeps and as many backward ones.
  void vcycle_rb(size_t li) {
    Level<T>& l = levels[li];
    std::fill(l.z.begin(), l.z.end(), (T)0);
    if (li + 1 == levels.size()) {
      for (int k = 0; k < COARSE_SWEEPS_RB; ++k) l.gs_forward();
      for (int k = 0; k < COARSE_SWEEPS_RB; ++k) l.gs_backward();
      return;
    }
    for (int k = 0; k < nu; ++k) l.gs_forward();
    l.restrict_into(levels[li + 1]);
    vcycle_rb(li + 1);
    const Level<T>& c = levels[li + 1];
    for (size_t j = 0; j < l.h; ++j)
      for (size_t i = 0; i < l.w; ++i) l.z[j * l.w + i] += c.z[(j / 2) * c.w + i / 2];
    for (int k = 0; k < nu; ++k) l.gs_backward();
  }

  // z = M^-1 r on the finest level (whose r the caller set); returns sum r64 * z.
  double precondition(const double* r64) {
    if (kind == DTO_CYCLE_JACOBI) return vcycle_jacobi(0, r64);
    vcycle_rb(0);
    const Level<T>& l = levels[0];
    std::vector<double> rows(l.h, 0.0);
    for (size_t j = 0; j < l.h; ++j) {
      double a = 0.0;
      for (size_t i = 0; i < l.w; ++i) a += r64[j * l.w + i] * (double)l.z[j * l.w + i];
      rows[j] = a;
    }
    double s = 0.0;
    for (double v : rows) s += v;
    return s;
  }
};

// multigrid.rs:562-763, with the cycle's kind and precision and the stopping rule as options.
template <typename T>
int mg_cg(const Dims& d, double* x, const double* b, const double* kd, double dt, double tol, int stop, int kind, int max_it,
          double* rel_res_out) {
  size_t n = d.cells(), w = d.w, h = d.h;
  if (n == 0) return 0;
  Operator op(d, kd, dt);
  Hierarchy<T> mg(op, kind, (T)OMEGA, NU, (T)SCALE);
  std::vector<double> r(n), pold(n, 0.0), pnew(n), ap(n), rows(h);
  T* r32 = mg.levels[0].r.data();
  op.apply(x, r.data());
  for (size_t k = 0; k < n; ++k) {
    r[k] = b[k] - r[k];
    r32[k] = (T)r[k];
  }
  auto rowsum2 = [&](const double* a, const double* bb) {
#pragma omp parallel for schedule(static)
    for (long j = 0; j < (long)h; ++j) {
      double s = 0.0;
      for (size_t i = 0; i < w; ++i) s += a[j * w + i] * bb[j * w + i];
      rows[j] = s;
    }
    double s = 0.0;
    for (double v : rows) s += v;
    return s;
  };
  double rr0 = rowsum2(r.data(), r.data());
  double bb = rowsum2(b, b);
  double tol2 = stop == DTO_STOP_REL_RESIDUAL ? tol * tol * bb : tol * tol * (double)n;
  int its = 0;
  double rr = rr0;
  if (rr0 > tol2) {
    double rz = mg.precondition(r.data());
    bool have_beta = false, have_pending = false;
    double beta = 0.0, pending = 0.0;
    while (its < max_it) {
      ++its;
      const T* z = mg.levels[0].z.data();
      for (size_t k = 0; k < n; ++k) {
        if (have_pending) x[k] += pending * pold[k];
        pnew[k] = have_beta ? (double)z[k] + beta * pold[k] : (double)z[k];
      }
      have_pending = false;
      op.apply(pnew.data(), ap.data());
      double pap = rowsum2(pnew.data(), ap.data());
      std::swap(pold, pnew);
      if (pap <= 0.0 || !std::isfinite(pap)) break;
      double alpha = rz / pap;
      pending = alpha;
      have_pending = true;
      for (size_t k = 0; k < n; ++k) {
        r[k] -= alpha * ap[k];
        r32[k] = (T)r[k];
      }
      rr = rowsum2(r.data(), r.data());
      if (rr <= tol2) break;
      double rz_new = mg.precondition(r.data());
      if (!(std::isfinite(rz_new) && rz > 0.0)) break;
      beta = rz_new / rz;
      have_beta = true;
      rz = rz_new;
    }
    if (have_pending)
      for (size_t k = 0; k < n; ++k) x[k] += pending * pold[k];
  }
  // mass put-back, multigrid.rs:736-761
  op.apply(x, ap.data());
  double lost = 0.0, weight = 0.0;
  for (size_t j = 0; j < h; ++j) {
    double l = 0.0, g = 0.0;
    for (size_t i = 0; i < w; ++i) {
      size_t k = j * w + i;
      l += b[k] - ap[k];
      g += op.diag[k] - 1.0;
    }
    lost += l;
    weight += g;
  }
  if (weight > 0.0 && lost != 0.0) {
    double kk = lost / weight;
    for (size_t k = 0; k < n; ++k) x[k] += kk * (op.diag[k] - 1.0);
  }
  if (rel_res_out) {
    op.apply(x, ap.data());
    for (size_t k = 0; k < n; ++k) ap[k] = b[k] - ap[k];
    double rrf = rowsum2(ap.data(), ap.data());
    *rel_res_out = bb > 0 ? std::sqrt(rrf / bb) : 0.0;
  }
  return its;
}

// multigrid/tests.rs:17-74: (I + dt L) x from the definition, and unpreconditioned CG to a
// relative residual of 1e-13.
void apply_reference(const Dims& d, const double* kd, double dt, const double* x, double* y) {
  size_t w = d.w, h = d.h;
  double s2 = d.dx * d.dx;
  bool wrap = d.wrap_x && w > 1;
#pragma omp parallel for schedule(static)
  for (long jl = 0; jl < (long)h; ++jl) {
    size_t j = (size_t)jl;
    for (size_t i = 0; i < w; ++i) {
      size_t c = j * w + i;
      long nb[4];
      nb[0] = i + 1 < w ? (long)(c + 1) : (wrap ? (long)(j * w) : -1);
      nb[1] = i > 0 ? (long)(c - 1) : (wrap ? (long)(j * w + w - 1) : -1);
      nb[2] = j + 1 < h ? (long)(c + w) : -1;
      nb[3] = j > 0 ? (long)(c - w) : -1;
      double v = x[c];
      for (long m : nb)
        if (m >= 0) v += 0.5 * (kd[c] + kd[m]) * dt / s2 * (x[c] - x[m]);
      y[c] = v;
    }
  }
}

void reference_cg(const Dims& d, const double* b, const double* kd, double dt, double* x, double rel) {
  size_t n = d.cells();
  std::copy(b, b + n, x);
  std::vector<double> ax(n), r(n), p(n);
  apply_reference(d, kd, dt, x, ax.data());
  for (size_t k = 0; k < n; ++k) r[k] = b[k] - ax[k];
  p = r;
  double rr = 0.0, bb = 0.0;
  for (size_t k = 0; k < n; ++k) {
    rr += r[k] * r[k];
    bb += b[k] * b[k];
  }
  bb = std::max(bb, 1.0);
  for (size_t it = 0; it < 20 * n + 100; ++it) {
    if (rr <= rel * rel * bb) break;
    apply_reference(d, kd, dt, p.data(), ax.data());
    double pap = 0.0;
    for (size_t k = 0; k < n; ++k) pap += p[k] * ax[k];
    double alpha = rr / pap;
    for (size_t k = 0; k < n; ++k) {
      x[k] += alpha * p[k];
      r[k] -= alpha * ax[k];
    }
    double rr_new = 0.0;
    for (size_t k = 0; k < n; ++k) rr_new += r[k] * r[k];
    double beta = rr_new / rr;
    rr = rr_new;
    for (size_t k = 0; k < n; ++k) p[k] = r[k] + beta * p[k];
  }
}

// surface/marine.rs:44-59
double submarine_kd(double z, double d0, double wave_base, double tidal_range, double land) {
  double f1 = tidal_range > 0.0 ? (std::tanh(z / tidal_range) + 1.0) / 2.0 : (z >= 0.0 ? 1.0 : 0.0);
  double f2 = (z > wave_base && wave_base > 0.0) ? std::exp(-(z - wave_base) / wave_base) : 1.0;
  return d0 * f1 * f2 + land * (1.0 - f1);
}

}  // namespace oracle

using namespace oracle;

extern "C" {

int dto_diff_operator(int w, int h, double dx, int wrap, const double* kd, double dt, const double* x, double* y) {
  Dims d{(size_t)w, (size_t)h, dx, wrap != 0};
  Operator op(d, kd, dt);
  op.apply(x, y);
  return 0;
}

int dto_diff_operator_coeffs(int w, int h, double dx, int wrap, const double* kd, double dt, double* east, double* south, double* diag) {
  Dims d{(size_t)w, (size_t)h, dx, wrap != 0};
  Operator op(d, kd, dt);
  std::copy(op.east.begin(), op.east.end(), east);
  std::copy(op.south.begin(), op.south.end(), south);
  std::copy(op.diag.begin(), op.diag.end(), diag);
  return 0;
}

int dto_diff_apply_reference(int w, int h, double dx, int wrap, const double* kd, double dt, const double* x, double* y) {
  Dims d{(size_t)w, (size_t)h, dx, wrap != 0};
  apply_reference(d, kd, dt, x, y);
  return 0;
}

int dto_diff_lod(int w, int h, double dx, int wrap, double* hfield, const double* kd, double dt) {
  Dims d{(size_t)w, (size_t)h, dx, wrap != 0};
  lod(d, hfield, kd, dt);
  return 0;
}

void dto_thomas(const double* lo, const double* di, const double* up, double* b, int n) { thomas(lo, di, up, b, (size_t)n); }
void dto_cyclic(const double* lo, const double* di, const double* up, double alpha, double beta, double* b, int n) {
  cyclic(lo, di, up, alpha, beta, b, (size_t)n);
}

int dto_diff_solve_jacobi(int w, int h, double dx, int wrap, double* hfield, const double* kd, double dt, int use_lod) {
  Dims d{(size_t)w, (size_t)h, dx, wrap != 0};
  std::vector<double> b(hfield, hfield + d.cells());
  if (use_lod) lod(d, hfield, kd, dt);
  return jacobi_cg(d, hfield, b.data(), kd, dt, 1.0e-6, 400);
}

int dto_diff_solve_mg(int w, int h, double dx, int wrap, double* hfield, const double* kd, double dt, double tol, int stop, int cycle,
                      int precision, int use_lod, int max_it, double* rel_res) {
  Dims d{(size_t)w, (size_t)h, dx, wrap != 0};
  std::vector<double> b(hfield, hfield + d.cells());
  if (use_lod) lod(d, hfield, kd, dt);
  if (precision == 64) return mg_cg<double>(d, hfield, b.data(), kd, dt, tol, stop, cycle, max_it, rel_res);
  return mg_cg<float>(d, hfield, b.data(), kd, dt, tol, stop, cycle, max_it, rel_res);
}

// One cycle z = M^-1 r (f32 levels), returning sum r*z; `levels_out` receives the level count.
double dto_diff_vcycle(int w, int h, double dx, int wrap, const double* kd, double dt, int cycle, const double* r, float* z,
                       int* levels_out) {
  Dims d{(size_t)w, (size_t)h, dx, wrap != 0};
  Operator op(d, kd, dt);
  Hierarchy<float> mg(op, cycle, OMEGA, NU, SCALE);
  for (size_t k = 0; k < d.cells(); ++k) mg.levels[0].r[k] = (float)r[k];
  double rz = mg.precondition(r);
  std::copy(mg.levels[0].z.begin(), mg.levels[0].z.end(), z);
  if (levels_out) *levels_out = (int)mg.levels.size();
  return rz;
}

int dto_diff_reference_cg(int w, int h, double dx, int wrap, const double* b, const double* kd, double dt, double rel, double* x) {
  Dims d{(size_t)w, (size_t)h, dx, wrap != 0};
  reference_cg(d, b, kd, dt, x, rel);
  return 0;
}

double dto_submarine_kd(double z, double d0, double wave_base, double tidal_range, double land) {
  return submarine_kd(z, d0, wave_base, tidal_range, land);
}

}  // extern "C"

// Test infrastructure only: the CPU oracle for deep-time's lithospheric flexure solve. Only the
// tests, the smoke check and the benchmark's CPU-baseline leg load this; the product never does.
//
// A restatement, in C++17 with OpenMP, of the reference's block-metric and sphere-metric solver in
// crates/deeptime-core/src/surface/flexure.rs (paths below are relative to that crate's src/):
//   rigidity_per_g / flexural_parameter_m  surface/flexure.rs:377-385
//   RowMetric::from_sin_faces              surface/flexure.rs:964-1010
//   RowSolve::solve                        surface/flexure.rs:1016-1099
//   Spectral::{new, forward_with, inverse_with}  surface/flexure.rs:1108-1348
//   Bank::new                              surface/flexure.rs:1352-1402
//   Preconditioner::new                    surface/flexure.rs:1405-1468
//   Solver::{laplacian_then, bend, operator_from, precondition, spectral_solve, solve}
//                                          surface/flexure.rs:1471-1741
//   box_blur                               surface/grid.rs:224-270
// The operation order of each cell's arithmetic follows the reference (no fused multiply-add:
// built with -ffp-contract=off). Two additions that the reference does not have are labelled:
// the single-level constant-mean-D preconditioner and the relative-residual stopping rule of the
// benchmark configurations.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#include <omp.h>

#include "fft.hpp"
#include "oracle.h"

namespace oracle {

static const double RHO_MANTLE = 3300.0;  // surface/flexure.rs:102
static const double YOUNG_PA = 70.0e9;    // surface/flexure.rs:106
static const double POISSON = 0.25;       // surface/flexure.rs:107

double rigidity_per_g(double te_km, double g) {
  double te = te_km * 1000.0;
  return YOUNG_PA * te * te * te / (12.0 * (1.0 - POISSON * POISSON)) / g;
}
double flexural_parameter_m(double d_per_g) { return std::pow(4.0 * d_per_g / RHO_MANTLE, 0.25); }

// Row-ordered sum: per row in ascending column order, then the row sums in ascending row order
// (surface/flexure.rs:1495-1503): the same value at any thread count.
static double dot(size_t w, size_t n, const double* a, const double* b) {
  size_t h = n / w;
  std::vector<double> rows(h);
#pragma omp parallel for schedule(static)
  for (long j = 0; j < (long)h; ++j) {
    double s = 0.0;
    for (size_t i = 0; i < w; ++i) s += a[j * w + i] * b[j * w + i];
    rows[j] = s;
  }
  double s = 0.0;
  for (double v : rows) s += v;
  return s;
}
static double max_abs(size_t n, const double* v) {
  double m = 0.0;
#pragma omp parallel for reduction(max : m) schedule(static)
  for (long k = 0; k < (long)n; ++k) m = std::max(m, std::fabs(v[k]));
  return m;
}

struct RowSolve {  // surface/flexure.rs:1016-1099
  std::vector<double> a, b, lx;
  double inv;
  void solve(size_t k, double d, double c, cd* x, size_t h, double* dd, double* l1, double* l2) const {
    double lxk = lx[k];
    auto t = [&](size_t j) { return (a[j] * lxk - b[j] - b[j + 1]) * inv; };
    auto e = [&](size_t j) { return j + 1 < h ? b[j + 1] * inv : 0.0; };
    auto m0 = [&](size_t j) {
      double up = j > 0 ? e(j - 1) : 0.0;
      return d * (t(j) * t(j) + up * up + e(j) * e(j)) + c;
    };
    auto m1 = [&](size_t j) { return d * e(j) * (t(j) + t(j + 1)); };
    auto m2 = [&](size_t j) { return d * e(j) * e(j + 1); };
    for (size_t j = 0; j < h; ++j) {
      double p1 = 0.0, p2 = 0.0;
      if (j >= 2) p2 = m2(j - 2) / dd[j - 2];
      if (j >= 1) {
        double carried = j >= 2 ? p2 * dd[j - 2] * l1[j - 1] : 0.0;
        p1 = (m1(j - 1) - carried) / dd[j - 1];
      }
      double dj = m0(j);
      if (j >= 1) dj -= p1 * p1 * dd[j - 1];
      if (j >= 2) dj -= p2 * p2 * dd[j - 2];
      dd[j] = dj;
      l1[j] = p1;
      l2[j] = p2;
    }
    for (size_t j = 0; j < h; ++j) {
      cd v = x[j];
      if (j >= 1) v -= x[j - 1] * l1[j];
      if (j >= 2) v -= x[j - 2] * l2[j];
      x[j] = v;
    }
    for (size_t j = 0; j < h; ++j) x[j] /= dd[j];
    for (size_t jj = h; jj-- > 0;) {
      cd v = x[jj];
      if (jj + 1 < h) v -= x[jj + 1] * l1[jj + 1];
      if (jj + 2 < h) v -= x[jj + 2] * l2[jj + 2];
      x[jj] = v;
    }
  }
};

struct Spectral {  // surface/flexure.rs:1108-1348
  size_t w, h, nk;
  Fft fx, ix, fy, iy;
  std::vector<cd> twiddle;  // e^(-i pi m / 2h)
  std::vector<double> lam2;  // column-major k*h + m
  bool has_rows = false;
  RowSolve rows;

  Spectral(size_t w_, size_t h_, double dx) : w(w_), h(h_), nk(w_ / 2 + 1), fx(w_, false), ix(w_, true), fy(h_, false), iy(h_, true) {
    twiddle.resize(h);
    for (size_t m = 0; m < h; ++m) twiddle[m] = unit_root(-(long double)m, 2.0L * h, 1);
    std::vector<double> lx(nk), ly(h);
    const double TAU = 6.283185307179586476925286766559;
    const double PI = 3.141592653589793238462643383279;
    for (size_t k = 0; k < nk; ++k) lx[k] = 2.0 * std::cos(TAU * (double)k / (double)w) - 2.0;
    for (size_t m = 0; m < h; ++m) ly[m] = 2.0 * std::cos(PI * (double)m / (double)h) - 2.0;
    double inv = 1.0 / (dx * dx);
    lam2.assign(nk * h, 0.0);
    for (size_t k = 0; k < nk; ++k)
      for (size_t m = 0; m < h; ++m) {
        double l = (lx[k] + ly[m]) * inv;
        lam2[k * h + m] = l * l;
      }
  }
  void set_rows(const double* a, const double* b, double dx) {
    has_rows = true;
    rows.a.assign(a, a + h);
    rows.b.assign(b, b + h + 1);
    rows.lx.resize(nk);
    const double TAU = 6.283185307179586476925286766559;
    for (size_t k = 0; k < nk; ++k) rows.lx[k] = 2.0 * std::cos(TAU * (double)k / (double)w) - 2.0;
    rows.inv = 1.0 / (dx * dx);
  }

  // spec (nk x h, column-major) <- transform of v (x weight), each coefficient divided by
  // d*lam2 + c when divide is given. half is h x nk scratch.
  void forward_with(const double* v, const double* weight, const double* divide, cd* half, cd* spec) const {
    size_t pairs = (h + 1) / 2;
#pragma omp parallel
    {
      std::vector<cd> buf(w);
#pragma omp for schedule(static)
      for (long pair = 0; pair < (long)pairs; ++pair) {
        size_t ja = 2 * pair, jb = 2 * pair + 1;
        const double* a = v + ja * w;
        const double* b = jb < h ? v + jb * w : nullptr;
        for (size_t i = 0; i < w; ++i) {
          if (weight) {
            buf[i] = cd(a[i] * weight[ja * w + i], b ? b[i] * weight[jb * w + i] : 0.0);
          } else {
            buf[i] = cd(a[i], b ? b[i] : 0.0);
          }
        }
        fx.run(buf.data());
        cd* oa = half + ja * nk;
        cd* ob = jb < h ? half + jb * nk : nullptr;
        for (size_t k = 0; k < nk; ++k) {
          cd z = buf[k], zc = std::conj(buf[(w - k) % w]);
          oa[k] = (z + zc) * 0.5;
          if (ob) {
            cd dd = z - zc;
            ob[k] = cd(dd.imag(), -dd.real()) * 0.5;
          }
        }
      }
    }
    if (has_rows) {
#pragma omp parallel
      {
        std::vector<double> dd(h), l1(h), l2(h);
#pragma omp for schedule(static)
        for (long k = 0; k < (long)nk; ++k) {
          cd* col = spec + k * h;
          for (size_t j = 0; j < h; ++j) col[j] = half[j * nk + k];
          if (divide) rows.solve(k, divide[0], divide[1], col, h, dd.data(), l1.data(), l2.data());
        }
      }
      return;
    }
#pragma omp parallel
    {
      std::vector<cd> buf(h);
#pragma omp for schedule(static)
      for (long k = 0; k < (long)nk; ++k) {
        cd* col = spec + k * h;
        for (size_t j = 0; j < h; ++j) {
          cd x = half[j * nk + k];
          if (j % 2 == 0)
            buf[j / 2] = x;
          else
            buf[h - 1 - j / 2] = x;
        }
        fy.run(buf.data());
        col[0] = buf[0];
        for (size_t m = 1; m < h; ++m) {
          cd p = twiddle[m] * buf[m];
          cd q = twiddle[h - m] * buf[h - m];
          col[m] = (p + cd(-q.imag(), q.real())) * 0.5;
        }
        if (divide) {
          for (size_t m = 0; m < h; ++m) col[m] /= divide[0] * lam2[k * h + m] + divide[1];
        }
      }
    }
  }

  // out <- inverse transform of spec (overwritten); with weight, out += inverse x weight.
  void inverse_with(cd* spec, const double* weight, double* out) const {
    double norm_y = 1.0 / (double)h;
    if (!has_rows) {
#pragma omp parallel
      {
        std::vector<cd> buf(h);
#pragma omp for schedule(static)
        for (long k = 0; k < (long)nk; ++k) {
          cd* col = spec + k * h;
          buf[0] = col[0];
          for (size_t m = 1; m < h; ++m) {
            cd c = col[h - m];
            buf[m] = std::conj(twiddle[m]) * (col[m] + cd(c.imag(), -c.real()));
          }
          iy.run(buf.data());
          for (size_t j = 0; j < h; ++j) col[j] = (j % 2 == 0 ? buf[j / 2] : buf[h - 1 - j / 2]) * norm_y;
        }
      }
    }
    double norm_x = 1.0 / (double)w;
    size_t pairs = (h + 1) / 2;
#pragma omp parallel
    {
      std::vector<cd> buf(w);
      const cd i1(0.0, 1.0);
#pragma omp for schedule(static)
      for (long pair = 0; pair < (long)pairs; ++pair) {
        size_t ja = 2 * pair, jb = 2 * pair + 1;
        for (size_t k = 0; k < nk; ++k) {
          cd a = spec[k * h + ja];
          cd b = jb < h ? spec[k * h + jb] : cd(0.0, 0.0);
          buf[k] = a + i1 * b;
          if (k > 0 && k < w - k) buf[w - k] = std::conj(a) + i1 * std::conj(b);
        }
        ix.run(buf.data());
        double* ra = out + ja * w;
        double* rb = jb < h ? out + jb * w : nullptr;
        if (weight) {
          for (size_t i = 0; i < w; ++i) {
            double p = buf[i].real() * norm_x;
            ra[i] += p * weight[ja * w + i];
            if (rb) {
              double q = buf[i].imag() * norm_x;
              rb[i] += q * weight[jb * w + i];
            }
          }
        } else {
          for (size_t i = 0; i < w; ++i) {
            ra[i] = buf[i].real() * norm_x;
            if (rb) rb[i] = buf[i].imag() * norm_x;
          }
        }
      }
    }
  }
};

struct Bank {  // surface/flexure.rs:1352-1402
  std::vector<double> d;
  std::vector<std::vector<double>> weights;
  double c_ref = 0.0;

  static Bank reference(size_t n, const double* dv, const double* c, double dx) {
    Bank bk;
    std::vector<double> ln_alpha(n);
#pragma omp parallel for schedule(static)
    for (long k = 0; k < (long)n; ++k) ln_alpha[k] = std::log(flexural_parameter_m(std::max(dv[k], 1e-30)) / dx);
    double lo = INFINITY, hi = -INFINITY;
    for (double a : ln_alpha) {
      lo = std::min(lo, a);
      hi = std::max(hi, a);
    }
    double s = 0.0;
    for (size_t k = 0; k < n; ++k) s += c[k];
    bk.c_ref = s / (double)std::max<size_t>(n, 1);
    auto node_d = [&](double ln_a) { return RHO_MANTLE * std::pow(std::exp(ln_a) * dx, 4) / 4.0; };
    double floor = std::log(0.4);
    if (hi - lo < 0.05 || hi <= floor) {
      bk.d.push_back(node_d(0.5 * (lo + hi)));
      return bk;
    }
    lo = std::max(lo, floor);
    const int K = 3;
    std::vector<double> nodes(K);
    for (int k = 0; k < K; ++k) nodes[k] = lo + (hi - lo) * (double)k / (double)(K - 1);
    bk.weights.assign(K, std::vector<double>(n, 0.0));
    for (size_t c2 = 0; c2 < n; ++c2) {
      double t = std::clamp((ln_alpha[c2] - lo) / (hi - lo), 0.0, 1.0) * (double)(K - 1);
      int k0 = std::min((int)std::floor(t), K - 2);
      double f = t - (double)k0;
      bk.weights[k0][c2] = std::sqrt(1.0 - f);
      bk.weights[k0 + 1][c2] = std::sqrt(f);
    }
    for (int k = 0; k < K; ++k) bk.d.push_back(node_d(nodes[k]));
    return bk;
  }

  // Not in the reference: the benchmark's constant-mean-D preconditioner, one spectral level at the
  // arithmetic means of d and c (the prototype's method D, docs/design/flexure.md:190).
  static Bank mean(size_t n, const double* dv, const double* c) {
    Bank bk;
    double sd = 0.0, sc = 0.0;
    for (size_t k = 0; k < n; ++k) {
      sd += dv[k];
      sc += c[k];
    }
    bk.d.push_back(sd / (double)std::max<size_t>(n, 1));
    bk.c_ref = sc / (double)std::max<size_t>(n, 1);
    return bk;
  }
};

struct Metric {
  std::vector<double> a, b;
};

class Solver {  // surface/flexure.rs:1471-1741
 public:
  size_t w, h, n;
  double dx;
  bool has_metric = false;
  Metric metric;
  Spectral spectral;
  std::vector<cd> half, spec;
  std::vector<double> tmp;

  Solver(size_t w_, size_t h_, double dx_, const double* ma, const double* mb)
      : w(w_), h(h_), n(w_ * h_), dx(dx_), spectral(w_, h_, dx_), half(h_ * (w_ / 2 + 1)), spec((w_ / 2 + 1) * h_), tmp(w_ * h_) {
    if (ma && mb) {
      has_metric = true;
      metric.a.assign(ma, ma + h);
      metric.b.assign(mb, mb + h + 1);
      spectral.set_rows(ma, mb, dx);
    }
  }

  enum ThenKind { NOTHING, SCALE, ADD };
  // surface/flexure.rs:1551-1595
  void laplacian_then(const double* v, ThenKind kind, const double* s, const double* c, const double* u, const double* from,
                      double* out) const {
    double inv = 1.0 / (dx * dx);
#pragma omp parallel for schedule(static)
    for (long jl = 0; jl < (long)h; ++jl) {
      size_t j = (size_t)jl;
      const double* mid = v + j * w;
      const double* north = v + (j == 0 ? 0 : j - 1) * w;
      const double* south = v + std::min(j + 1, h - 1) * w;
      double* row = out + j * w;
      if (has_metric) {
        double a = metric.a[j], bn = metric.b[j], bs = metric.b[j + 1];
        for (size_t i = 0; i < w; ++i) {
          double west = mid[i == 0 ? w - 1 : i - 1];
          double east = mid[i + 1 == w ? 0 : i + 1];
          double x = mid[i];
          row[i] = (a * (west + east - 2.0 * x) + bn * (north[i] - x) + bs * (south[i] - x)) * inv;
        }
      } else {
        for (size_t i = 0; i < w; ++i) {
          double west = mid[i == 0 ? w - 1 : i - 1];
          double east = mid[i + 1 == w ? 0 : i + 1];
          row[i] = (west + east + north[i] + south[i] - 4.0 * mid[i]) * inv;
        }
      }
      size_t c0 = j * w;
      if (kind == SCALE) {
        for (size_t i = 0; i < w; ++i) row[i] *= s[c0 + i];
      } else if (kind == ADD) {
        for (size_t i = 0; i < w; ++i) {
          size_t k = c0 + i;
          row[i] += c[k] * u[k];
          if (from) row[i] = from[k] - row[i];
        }
      }
    }
  }

  void bend(const double* d, const double* v, double* out) {
    laplacian_then(v, SCALE, d, nullptr, nullptr, nullptr, tmp.data());
    laplacian_then(tmp.data(), NOTHING, nullptr, nullptr, nullptr, nullptr, out);
  }
  void operator_from(const double* d, const double* c, const double* v, const double* from, double* out) {
    laplacian_then(v, SCALE, d, nullptr, nullptr, nullptr, tmp.data());
    laplacian_then(tmp.data(), ADD, nullptr, c, v, from, out);
  }

  // surface/flexure.rs:1654-1675
  void spectral_solve(const Bank& bank, const double* r, double* z) {
    if (bank.weights.empty()) {
      double divide[2] = {bank.d[0], bank.c_ref};
      spectral.forward_with(r, nullptr, divide, half.data(), spec.data());
      spectral.inverse_with(spec.data(), nullptr, z);
    } else {
      std::fill(z, z + n, 0.0);
      for (size_t k = 0; k < bank.weights.size(); ++k) {
        double divide[2] = {bank.d[k], bank.c_ref};
        spectral.forward_with(r, bank.weights[k].data(), divide, half.data(), spec.data());
        spectral.inverse_with(spec.data(), bank.weights[k].data(), z);
      }
    }
  }

  struct Pre {
    Bank bank;
    const double* d;
    const double* c;
    std::vector<double> jacobi, left, part;
  };

  // surface/flexure.rs:1417-1468 (reference) or the single mean level (the benchmark's plain method, no sweeps).
  Pre make_pre(const double* d, const double* c, int precond) const {
    Pre pre;
    pre.d = d;
    pre.c = c;
    if (precond == DTO_PRECOND_MEAN_D) {
      pre.bank = Bank::mean(n, d, c);
      return pre;
    }
    pre.bank = Bank::reference(n, d, c, dx);
    double inv = 1.0 / (dx * dx * dx * dx);
    if (!pre.bank.weights.empty()) {
      pre.jacobi.resize(n);
#pragma omp parallel for schedule(static)
      for (long kl = 0; kl < (long)n; ++kl) {
        size_t k = (size_t)kl, i = k % w, j = k / w;
        double east = d[j * w + (i + 1) % w], west = d[j * w + (i + w - 1) % w];
        double north = d[(j == 0 ? 0 : j - 1) * w + i], south = d[std::min(j + 1, h - 1) * w + i];
        if (!has_metric) {
          double around = east + west + north + south;
          pre.jacobi[k] = 0.5 / (c[k] + (16.0 * d[k] + around) * inv);
        } else {
          double a = metric.a[j], bn = metric.b[j], bs = metric.b[j + 1];
          double centre = 2.0 * a + bn + bs;
          double diag = d[k] * centre * centre + (east + west) * a * a + north * bn * bn + south * bs * bs;
          pre.jacobi[k] = 0.5 / (c[k] + diag * inv);
        }
      }
    }
    pre.left.assign(n, 0.0);
    pre.part.assign(n, 0.0);
    return pre;
  }

  // surface/flexure.rs:1630-1651
  void precondition(Pre& pre, const double* r, double* z) {
    if (pre.bank.weights.empty()) {
      spectral_solve(pre.bank, r, z);
      return;
    }
    double* left = pre.left.data();
    double* part = pre.part.data();
    const double* jac = pre.jacobi.data();
#pragma omp parallel for schedule(static)
    for (long k = 0; k < (long)n; ++k) z[k] = r[k] * jac[k];
    operator_from(pre.d, pre.c, z, r, left);
    spectral_solve(pre.bank, left, part);
#pragma omp parallel for schedule(static)
    for (long k = 0; k < (long)n; ++k) z[k] += part[k];
    operator_from(pre.d, pre.c, z, nullptr, left);
#pragma omp parallel for schedule(static)
    for (long k = 0; k < (long)n; ++k) z[k] += (r[k] - left[k]) * jac[k];
  }

  // surface/flexure.rs:1680-1740, with the benchmark's stopping rule as an option.
  void solve(const double* d, const double* c, const double* b, double* x, double tol, int max_it, int precond, int stop,
             dto_report* rep) {
    Pre pre = make_pre(d, c, precond);
    std::vector<double> r(b, b + n), z(n, 0.0), p, ap(n);
    std::fill(x, x + n, 0.0);
    double bb = dot(w, n, b, b);
    double bnorm = std::sqrt(bb);
    precondition(pre, r.data(), z.data());
    rep->iterations = 0;
    rep->error_m = max_abs(n, z.data());
    rep->converged = 1;
    rep->rel_residual = bnorm > 0 ? 1.0 : 0.0;
    if (stop == DTO_STOP_MAX_Z) {
      if (rep->error_m < tol) {
        std::copy(z.begin(), z.end(), x);
        // the returned correction's own residual
        std::vector<double> ax(n);
        operator_from(d, c, x, b, ax.data());
        rep->rel_residual = bnorm > 0 ? std::sqrt(dot(w, n, ax.data(), ax.data())) / bnorm : 0.0;
        return;
      }
    } else {
      if (bnorm == 0.0) {
        rep->rel_residual = 0.0;
        return;
      }
    }
    p = z;
    double rz = dot(w, n, r.data(), z.data());
    rep->converged = 0;
    for (int it = 1; it <= max_it; ++it) {
      operator_from(d, c, p.data(), nullptr, ap.data());
      double pap = dot(w, n, p.data(), ap.data());
      if (!(std::isfinite(pap) && pap > 0.0)) break;
      double alpha = rz / pap;
#pragma omp parallel for schedule(static)
      for (long k = 0; k < (long)n; ++k) {
        x[k] += alpha * p[k];
        r[k] -= alpha * ap[k];
      }
      rep->iterations = it;
      if (stop == DTO_STOP_REL_RESIDUAL) {
        double rr = dot(w, n, r.data(), r.data());
        rep->rel_residual = std::sqrt(rr) / bnorm;
        if (rep->rel_residual <= tol) {
          rep->converged = 1;
          break;
        }
      }
      precondition(pre, r.data(), z.data());
      double error = max_abs(n, z.data());
      double rz_new = dot(w, n, r.data(), z.data());
      rep->error_m = error;
      if (stop == DTO_STOP_MAX_Z && error < tol) {
        rep->converged = 1;
        break;
      }
      double beta = rz_new / rz;
      rz = rz_new;
#pragma omp parallel for schedule(static)
      for (long k = 0; k < (long)n; ++k) p[k] = z[k] + beta * p[k];
    }
    if (stop == DTO_STOP_MAX_Z) {
      double rr = dot(w, n, r.data(), r.data());
      rep->rel_residual = bnorm > 0 ? std::sqrt(rr) / bnorm : 0.0;
    }
  }
};

// surface/grid.rs:224-270: box blur, x wrapping when wrap, rows reflecting.
void box_blur(size_t w, size_t h, bool wrap, double* v, size_t r, size_t passes) {
  if (r == 0) return;
  double norm = 1.0 / (double)(2 * r + 1);
  long R = (long)r;
  for (size_t pass = 0; pass < passes; ++pass) {
#pragma omp parallel
    {
      std::vector<double> src(std::max(w, h));
#pragma omp for schedule(static)
      for (long j = 0; j < (long)h; ++j) {
        double* row = v + j * w;
        std::copy(row, row + w, src.begin());
        auto at = [&](long i) -> double {
          if (wrap) return src[(size_t)(((i % (long)w) + (long)w) % (long)w)];
          return src[(size_t)std::clamp(i, 0L, (long)w - 1)];
        };
        double acc = 0.0;
        for (long i = -R; i <= R; ++i) acc += at(i);
        for (size_t i = 0; i < w; ++i) {
          row[i] = acc * norm;
          acc += at((long)i + R + 1) - at((long)i - R);
        }
      }
    }
    std::vector<double> cols(w * h);
#pragma omp parallel
    {
      std::vector<double> src(h);
#pragma omp for schedule(static)
      for (long i = 0; i < (long)w; ++i) {
        for (size_t j = 0; j < h; ++j) src[j] = v[j * w + i];
        auto at = [&](long j) -> double {
          long jj = j < 0 ? -j - 1 : (j >= (long)h ? 2 * (long)h - j - 1 : j);
          return src[(size_t)std::clamp(jj, 0L, (long)h - 1)];
        };
        double acc = 0.0;
        for (long j = -R; j <= R; ++j) acc += at(j);
        for (size_t j = 0; j < h; ++j) {
          cols[i * h + j] = acc * norm;
          acc += at((long)j + R + 1) - at((long)j - R);
        }
      }
    }
#pragma omp parallel for schedule(static)
    for (long j = 0; j < (long)h; ++j)
      for (size_t i = 0; i < w; ++i) v[j * w + i] = cols[i * h + j];
  }
}

// surface/flexure.rs:1773-1795 (restrict_by): the mean of each f x f block, its cells summed
// row by row, then times 1 / (f f); a copy where f = 1.
void restrict_by(size_t w, size_t h, size_t f, const double* v, double* out) {
  if (f == 1) {
    std::copy(v, v + w * h, out);
    return;
  }
  size_t ws = w / f, hs = h / f;
  double norm = 1.0 / (double)(f * f);
#pragma omp parallel for schedule(static)
  for (long c = 0; c < (long)(ws * hs); ++c) {
    size_t i = (size_t)c % ws, j = (size_t)c / ws;
    double s = 0.0;
    for (size_t dj = 0; dj < f; ++dj)
      for (size_t di = 0; di < f; ++di) s += v[(j * f + dj) * w + i * f + di];
    out[c] = s * norm;
  }
}

// surface/flexure.rs:1797-1813 (coarse_cell, prolong_const): each coarse value on its f x f cells.
void prolong_const(size_t ws, size_t hs, size_t f, const double* v, double* out) {
  size_t w = ws * f, n = w * hs * f;
#pragma omp parallel for schedule(static)
  for (long c = 0; c < (long)n; ++c) {
    size_t i = (size_t)c % w, j = (size_t)c / w;
    out[c] = v[(j / f) * ws + i / f];
  }
}

// surface/flexure.rs:1815-1844 (prolong_linear, linear_at): bilinear from the coarse cells'
// centres, x wrapping, rows clamped.
void prolong_linear(size_t ws, size_t hs, size_t f, const double* v, double* out) {
  size_t w = ws * f, n = w * hs * f;
  if (f == 1) {
    std::copy(v, v + n, out);
    return;
  }
#pragma omp parallel for schedule(static)
  for (long c = 0; c < (long)n; ++c) {
    size_t i = (size_t)c % w, j = (size_t)c / w;
    double x = ((double)i + 0.5) / (double)f - 0.5;
    double y = std::clamp(((double)j + 0.5) / (double)f - 0.5, 0.0, (double)(hs - 1));
    double x0 = std::floor(x), y0 = std::floor(y);
    double tx = x - x0, ty = y - y0;
    long iw = (long)x0 % (long)ws;
    size_t i0 = (size_t)(iw < 0 ? iw + (long)ws : iw), i1 = (i0 + 1) % ws;
    size_t j0 = (size_t)y0, j1 = std::min(j0 + 1, hs - 1);
    out[c] = (v[j0 * ws + i0] * (1.0 - tx) + v[j0 * ws + i1] * tx) * (1.0 - ty) +
             (v[j1 * ws + i0] * (1.0 - tx) + v[j1 * ws + i1] * tx) * ty;
  }
}

// surface/flexure.rs:1745-1762 (binomial): passes of the [1/4, 1/2, 1/4] filter along x
// (wrapping) then along y (rows clamped).
void binomial(size_t w, size_t h, size_t passes, double* v) {
  std::vector<double> tmp(w * h);
  for (size_t pass = 0; pass < passes; ++pass) {
#pragma omp parallel for schedule(static)
    for (long j = 0; j < (long)h; ++j)
      for (size_t i = 0; i < w; ++i) {
        const double* row = v + j * w;
        tmp[j * w + i] = 0.25 * row[(i + w - 1) % w] + 0.5 * row[i] + 0.25 * row[(i + 1) % w];
      }
#pragma omp parallel for schedule(static)
    for (long j = 0; j < (long)h; ++j) {
      size_t n = j > 0 ? (size_t)j - 1 : 0, s = std::min((size_t)j + 1, h - 1);
      for (size_t i = 0; i < w; ++i) v[j * w + i] = 0.25 * tmp[n * w + i] + 0.5 * tmp[j * w + i] + 0.25 * tmp[s * w + i];
    }
  }
}

}  // namespace oracle

using namespace oracle;

extern "C" {

// The OpenMP team size of the oracle's parallel loops (the timing legs run it at all host
// threads and at 8, the reference's own benchmark setting); 0 or less restores all threads.
void dto_set_threads(int n) { omp_set_num_threads(n > 0 ? n : omp_get_num_procs()); }
int dto_threads(void) { return omp_get_max_threads(); }

double dto_rigidity_per_g(double te_km, double g) { return rigidity_per_g(te_km, g); }
double dto_flexural_parameter_m(double d_per_g) { return flexural_parameter_m(d_per_g); }

int dto_flex_spectral_roundtrip(int w, int h, double dx, const double* v, double* out) {
  Solver s(w, h, dx, nullptr, nullptr);
  s.spectral.forward_with(v, nullptr, nullptr, s.half.data(), s.spec.data());
  s.spectral.inverse_with(s.spec.data(), nullptr, out);
  return 0;
}

int dto_flex_operator(int w, int h, double dx, const double* ma, const double* mb, const double* d, const double* c, const double* v,
                      double* y) {
  Solver s(w, h, dx, ma, mb);
  s.operator_from(d, c, v, nullptr, y);
  return 0;
}

int dto_flex_bend(int w, int h, double dx, const double* d, const double* v, double* y) {
  Solver s(w, h, dx, nullptr, nullptr);
  s.bend(d, v, y);
  return 0;
}

int dto_flex_precondition(int w, int h, double dx, const double* ma, const double* mb, const double* d, const double* c, const double* r,
                          double* z, int precond) {
  Solver s(w, h, dx, ma, mb);
  Solver::Pre pre = s.make_pre(d, c, precond);
  s.precondition(pre, r, z);
  return 0;
}

int dto_flex_bank(int w, int h, double dx, const double* d, const double* c, double* node_d, double* c_ref, double* weights) {
  size_t n = (size_t)w * h;
  Bank bk = Bank::reference(n, d, c, dx);
  for (size_t k = 0; k < bk.d.size(); ++k) node_d[k] = bk.d[k];
  *c_ref = bk.c_ref;
  if (weights)
    for (size_t k = 0; k < bk.weights.size(); ++k) std::copy(bk.weights[k].begin(), bk.weights[k].end(), weights + k * n);
  return (int)bk.d.size();
}

int dto_flex_solve(int w, int h, double dx, const double* ma, const double* mb, const double* d, const double* c, const double* b,
                   double* x, double tol, int max_it, int precond, int stop, dto_report* rep) {
  Solver s(w, h, dx, ma, mb);
  s.solve(d, c, b, x, tol, max_it, precond, stop, rep);
  return 0;
}

void dto_row_metric_from_sin_faces(const double* sin_faces, int nfaces, int f, double* a, double* b) {
  // surface/flexure.rs:977-1000
  f = std::max(f, 1);
  int h = (nfaces - 1) / f;
  auto s = [&](int k) { return std::clamp(sin_faces[k * f], -1.0, 1.0); };
  double full = 0.0;
  for (int j = 0; j < h; ++j) full = std::max(full, std::fabs(s(j + 1) - s(j)));
  double least = std::max(0.5 * full, 1e-12);
  for (int j = 0; j < h; ++j) {
    double m = 0.5 * (s(j) + s(j + 1));
    a[j] = 1.0 / std::max(1.0 - m * m, least);
  }
  for (int k = 0; k <= h; ++k) b[k] = (k == 0 || k == h) ? 0.0 : 1.0 - s(k) * s(k);
}

void dto_box_blur(int w, int h, int wrap, double* v, int r, int passes) { box_blur(w, h, wrap != 0, v, r, passes); }
void dto_restrict_by(int w, int h, int f, const double* v, double* out) { restrict_by(w, h, f, v, out); }
void dto_prolong_const(int ws, int hs, int f, const double* v, double* out) { prolong_const(ws, hs, f, v, out); }
void dto_prolong_linear(int ws, int hs, int f, const double* v, double* out) { prolong_linear(ws, hs, f, v, out); }
void dto_binomial(int w, int h, int passes, double* v) { binomial(w, h, passes, v); }

}  // extern "C"

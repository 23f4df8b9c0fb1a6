// Test infrastructure only (the oracle; never linked into the product): a restatement, in C++17
// with OpenMP, of the reference's implicit diffusion on the cube grid with its multigrid
// preconditioner (DiffusionSolver::Multigrid):
//
//   ADJACENCY, cell_on, Iso::cell / Across::cell   deeptime-format/src/cube.rs:158-199, :264-412
//   CubeTopology::new (slots in OFFSETS order)      deeptime-core/src/sphere/cube.rs:69-128,
//                                                   surface/grid.rs:21-30
//   face_sum (the mean cell area's order)           sphere/cube.rs:437-449
//   couplings, Workspace::build (every cell)        surface/cube/diffusion.rs:88-240
//   solve, run, lod, cg                             surface/cube/diffusion.rs:244-500
//   Hierarchy (finest, coarsen), prepare,           surface/cube/multigrid.rs:65-363
//   precondition, sweep, vcycle
//   ordered_sum, CHUNK                              surface/cube.rs:48-58
//
// The grid's geometry (cell areas and the coupling Laplacian's weights, CubeGrid::areas / lap)
// is an input: it comes from the caller's CubeGrid. Compiled with -ffp-contract=off, so every
// sum and product is the reference's, in the reference's order.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "oracle.h"

namespace oracle {
void thomas(const double* lo, const double* di, const double* up, double* b, size_t n);
}

namespace oracle_cube {

constexpr uint32_t NO_CELL = 0xFFFFFFFFu;
constexpr size_t CHUNK = 4096;           // surface/cube.rs:48
constexpr float OMEGA = 0.8f;            // diffusion/multigrid.rs:45
constexpr int NU = 2;                    // multigrid.rs:48
constexpr float SCALE = 0.5f;            // multigrid.rs:52
constexpr size_t COARSEST = 64;          // multigrid.rs:54
constexpr int COARSE_SWEEPS = 16;        // multigrid.rs:56
constexpr int CG_MAX_ITER = 400;         // surface/diffusion.rs:497

// Faces F0, F1, F2, F3, N, S (0..5); sides east, south, west, north (0..3).
struct Across {
  int face, side, turns, sx, sy;
};
// deeptime-format/src/cube.rs:321-369, [face][side]
static const Across ADJ[6][4] = {
    {{1, 2, 0, -1, 0}, {5, 3, 0, 0, -1}, {3, 0, 0, 1, 0}, {4, 1, 0, 0, 1}},
    {{2, 2, 0, -1, 0}, {5, 0, 1, 2, 0}, {0, 0, 0, 1, 0}, {4, 0, 3, 1, 1}},
    {{3, 2, 0, -1, 0}, {5, 1, 2, 1, 2}, {1, 0, 0, 1, 0}, {4, 3, 2, 1, 0}},
    {{0, 2, 0, -1, 0}, {5, 2, 3, -1, 1}, {2, 0, 0, 1, 0}, {4, 2, 1, 0, 0}},
    {{1, 3, 1, 1, -1}, {0, 3, 0, 0, -1}, {3, 3, 3, 0, 0}, {2, 3, 2, 1, 0}},
    {{1, 1, 3, 0, 2}, {2, 1, 2, 1, 2}, {3, 1, 1, 1, 1}, {0, 1, 0, 0, 1}},
};
// surface/grid.rs:21-30: E, NE, N, NW, W, SW, S, SE (j grows southward)
static const int OFF[8][2] = {{1, 0}, {1, -1}, {0, -1}, {-1, -1}, {-1, 0}, {-1, 1}, {0, 1}, {1, 1}};

// cube.rs:374-399: cell (i, j) of `face`, or the neighbour face's cell across one side.
static bool cell_on(int face, long n, long i, long j, int* f2, long* i2, long* j2) {
  bool out_i = i < 0 || i >= n, out_j = j < 0 || j >= n;
  if (!out_i && !out_j) {
    *f2 = face;
    *i2 = i;
    *j2 = j;
    return true;
  }
  if (out_i && out_j) return false;
  if (i < -n || i >= 2 * n || j < -n || j >= 2 * n) return false;
  int side = i >= n ? 0 : i < 0 ? 2 : j >= n ? 1 : 3;
  const Across& a = ADJ[face][side];
  long rx, rz;  // Iso::cell: clockwise cell turns, then the translation n * shift
  switch (a.turns) {
    case 1: rx = -j - 1, rz = i; break;
    case 2: rx = -i - 1, rz = -j - 1; break;
    case 3: rx = j, rz = -i - 1; break;
    default: rx = i, rz = j;
  }
  *f2 = a.face;
  *i2 = rx + n * a.sx;
  *j2 = rz + n * a.sy;
  return true;
}

// sphere/cube.rs:76-93
void topology(size_t n, uint32_t* slots) {
  size_t nn = n * n;
#pragma omp parallel for schedule(static)
  for (long c = 0; c < (long)(6 * nn); ++c) {
    int face = (int)(c / nn);
    long i = (long)(c % nn % n), j = (long)(c % nn / n);
    for (int k = 0; k < 8; ++k) {
      int f;
      long a, b;
      slots[c * 8 + k] = cell_on(face, (long)n, i + OFF[k][0], j + OFF[k][1], &f, &a, &b)
                             ? (uint32_t)(f * nn + b * n + a)
                             : NO_CELL;
    }
  }
}

// sphere/cube.rs:437-449: per face row, rows in order, faces in order
static double face_sum(size_t n, const double* v) {
  double total = 0.0;
  for (size_t f = 0; f < 6; ++f) {
    double fs = 0.0;
    for (size_t j = 0; j < n; ++j) {
      double r = 0.0;
      for (size_t i = 0; i < n; ++i) r += v[(f * n + j) * n + i];
      fs += r;
    }
    total += fs;
  }
  return total;
}

// surface/cube.rs:52-58: chunks of CHUNK summed in order, then the chunk sums in order
template <class F>
static double ordered_sum(size_t len, F f) {
  size_t nc = (len + CHUNK - 1) / CHUNK;
  std::vector<double> parts(nc);
#pragma omp parallel for schedule(static)
  for (long q = 0; q < (long)nc; ++q) {
    double s = 0.0;
    for (size_t i = q * CHUNK; i < std::min(len, (q + 1) * CHUNK); ++i) s += f(i);
    parts[q] = s;
  }
  double t = 0.0;
  for (double p : parts) t += p;
  return t;
}

// The operator (mu + sum K) - K on every cell (surface/cube/diffusion.rs:47-240).
struct Op {
  size_t n = 0, cells = 0;
  const uint32_t* slots = nullptr;
  std::vector<double> k, mu, s, diag;  // k: 8 per cell
  double row(size_t i, const double* p) const {
    double acc = diag[i] * p[i];
    for (int t = 0; t < 8; ++t) {
      uint32_t j = slots[i * 8 + t];
      if (j != NO_CELL) acc -= k[i * 8 + t] * p[j];
    }
    return acc;
  }
  void apply(const double* p, double* out) const {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)cells; ++i) out[i] = row(i, p);
  }
};

// diffusion.rs:88-113 (couplings) and :147-240 (build, every cell taking part)
static void build(Op& op, size_t n, const uint32_t* slots, const double* lap, const double* areas, const double* kd, double dt) {
  op.n = n;
  op.cells = 6 * n * n;
  op.slots = slots;
  const size_t cells = op.cells;
  const double mean = face_sum(n, areas) / (double)cells;
  const double scale = dt / mean;
  op.k.assign(cells * 8, 0.0);
  op.mu.resize(cells);
  op.s.resize(cells);
  op.diag.resize(cells);
  auto m2 = [&](size_t x, size_t y) { return 0.5 * (kd[x] + kd[y]); };
#pragma omp parallel for schedule(static)
  for (long c = 0; c < (long)cells; ++c) {
    const uint32_t* s = slots + c * 8;
    for (int slot = 0; slot < 8; ++slot) {
      uint32_t m = s[slot];
      if (m == NO_CELL) continue;
      double d;
      if (slot % 2 == 0) {
        d = m2(c, m);
      } else {
        size_t a = s[slot - 1], b = s[(slot + 1) % 8];
        d = std::fmin(std::fmin(std::fmin(m2(c, a), m2(a, m)), m2(m, b)), m2(b, c));
      }
      op.k[c * 8 + slot] = scale * d * lap[c * 8 + slot];
    }
    op.mu[c] = areas[c] / mean;
    double sum = 0.0;
    for (int t = 0; t < 8; ++t) sum += op.k[c * 8 + t];
    op.s[c] = sum;
    op.diag[c] = op.mu[c] + sum;
  }
}

// diffusion.rs:315-381 (lod): rows of each face (slots E = 0, W = 4), then columns (N = 2,
// S = 6), each tridiagonal (mu + K) y = mu b divided through by mu; across a face's edge the
// coupling takes the old value.
static void lod(const Op& op, const double* b, double* x, double* tmp) {
  const size_t n = op.n, nn = n * n;
  const uint32_t* t = op.slots;
#pragma omp parallel
  {
    std::vector<double> lo(n), di(n), up(n);
#pragma omp for schedule(static)
    for (long row = 0; row < (long)(6 * n); ++row) {
      size_t c0 = row * n;
      double* xr = x + c0;
      std::fill(lo.begin(), lo.end(), 0.0);
      std::fill(up.begin(), up.end(), 0.0);
      for (size_t i = 0; i < n; ++i) {
        size_t c = c0 + i;
        double ke = op.k[c * 8 + 0], kw = op.k[c * 8 + 4], mu = op.mu[c];
        di[i] = 1.0 + (ke + kw) / mu;
        double v = b[c];
        if (i > 0)
          lo[i] = -kw / mu;
        else
          v += kw * b[t[c * 8 + 4]] / mu;
        if (i + 1 < n)
          up[i] = -ke / mu;
        else
          v += ke * b[t[c * 8 + 0]] / mu;
        xr[i] = v;
      }
      oracle::thomas(lo.data(), di.data(), up.data(), xr, n);
    }
#pragma omp for schedule(static)
    for (long col = 0; col < (long)(6 * n); ++col) {
      size_t f = col / n, i = col % n;
      double* tc = tmp + col * n;
      std::fill(lo.begin(), lo.end(), 0.0);
      std::fill(up.begin(), up.end(), 0.0);
      for (size_t j = 0; j < n; ++j) {
        size_t c = f * nn + j * n + i;
        double kn = op.k[c * 8 + 2], ks = op.k[c * 8 + 6], mu = op.mu[c];
        di[j] = 1.0 + (kn + ks) / mu;
        double v = x[c];
        if (j > 0)
          lo[j] = -kn / mu;
        else
          v += kn * x[t[c * 8 + 2]] / mu;
        if (j + 1 < n)
          up[j] = -ks / mu;
        else
          v += ks * x[t[c * 8 + 6]] / mu;
        tc[j] = v;
      }
      oracle::thomas(lo.data(), di.data(), up.data(), tc, n);
    }
#pragma omp for schedule(static)
    for (long row = 0; row < (long)(6 * n); ++row) {
      size_t f = row / n, j = row % n;
      for (size_t i = 0; i < n; ++i) x[row * n + i] = tmp[f * nn + i * n + j];
    }
  }
}

// ---- the multigrid hierarchy (surface/cube/multigrid.rs) ----
struct Pattern {
  size_t side = 0, cells = 0;
  std::vector<uint32_t> ptr, col, src_ptr, src, kid_ptr, kids, parent;
};
struct Level {
  std::vector<float> val, mass, diag, r, z, t;
};

// multigrid.rs:65-90: the grid's neighbour table in slot order
static Pattern finest(size_t n, const uint32_t* slots) {
  Pattern p;
  p.side = n;
  p.cells = 6 * n * n;
  p.ptr.push_back(0);
  for (size_t c = 0; c < p.cells; ++c) {
    for (int k = 0; k < 8; ++k)
      if (slots[c * 8 + k] != NO_CELL) p.col.push_back(slots[c * 8 + k]);
    p.ptr.push_back((uint32_t)p.col.size());
  }
  return p;
}

// multigrid.rs:92-166: 2 x 2 blocks of each face (the last row or column alone when odd)
static Pattern coarsen(const Pattern& f) {
  size_t nf = f.side, m = (nf + 1) / 2, cells = 6 * m * m;
  Pattern p;
  p.side = m;
  p.cells = cells;
  p.parent.resize(f.cells);
  for (size_t c = 0; c < f.cells; ++c) {
    size_t face = c / (nf * nf), rest = c % (nf * nf), i = rest % nf, j = rest / nf;
    p.parent[c] = (uint32_t)(face * m * m + (j / 2) * m + i / 2);
  }
  p.kid_ptr.assign(cells + 1, 0);
  for (uint32_t q : p.parent) p.kid_ptr[q + 1] += 1;
  for (size_t k = 0; k < cells; ++k) p.kid_ptr[k + 1] += p.kid_ptr[k];
  std::vector<uint32_t> fill(p.kid_ptr.begin(), p.kid_ptr.end());
  p.kids.resize(f.cells);
  for (size_t c = 0; c < f.cells; ++c) p.kids[fill[p.parent[c]]++] = (uint32_t)c;
  p.ptr.push_back(0);
  p.src_ptr.push_back(0);
  for (size_t r = 0; r < cells; ++r) {
    std::vector<std::pair<uint32_t, uint32_t>> pairs;
    for (uint32_t k = p.kid_ptr[r]; k < p.kid_ptr[r + 1]; ++k) {
      uint32_t c = p.kids[k];
      for (uint32_t e = f.ptr[c]; e < f.ptr[c + 1]; ++e) {
        uint32_t q = p.parent[f.col[e]];
        if (q != r) pairs.push_back({q, e});
      }
    }
    std::stable_sort(pairs.begin(), pairs.end(), [](auto& a, auto& b) { return a.first < b.first; });
    uint32_t at = p.src_ptr.back();
    for (size_t k = 0; k < pairs.size(); ++k) {
      if (k == 0 || pairs[k].first != pairs[k - 1].first) {
        p.col.push_back(pairs[k].first);
        if (k > 0) p.src_ptr.push_back(at);
      }
      ++at;
      p.src.push_back(pairs[k].second);
    }
    if (!pairs.empty()) p.src_ptr.push_back(at);
    p.ptr.push_back((uint32_t)p.col.size());
  }
  return p;
}

struct Hierarchy {
  std::vector<Pattern> pats;
  std::vector<Level> levels;
};

// multigrid.rs:170-186 and :199-269 (prepare)
static void prepare(Hierarchy& H, const Op& op) {
  H.pats.clear();
  H.pats.push_back(finest(op.n, op.slots));
  while (!(H.pats.back().cells <= COARSEST || H.pats.back().side <= 1)) H.pats.push_back(coarsen(H.pats.back()));
  H.levels.assign(H.pats.size(), Level());
  {
    const Pattern& p = H.pats[0];
    Level& lv = H.levels[0];
    lv.val.resize(p.col.size());
    size_t at = 0;
    for (size_t c = 0; c < p.cells; ++c)
      for (int s = 0; s < 8; ++s)
        if (op.slots[c * 8 + s] != NO_CELL) lv.val[at++] = (float)op.k[c * 8 + s];
    lv.mass.resize(p.cells);
    lv.diag.resize(p.cells);
    for (size_t c = 0; c < p.cells; ++c) {
      lv.mass[c] = (float)op.mu[c];
      lv.diag[c] = (float)op.diag[c];
    }
    lv.r.assign(p.cells, 0.f);
    lv.z.assign(p.cells, 0.f);
    lv.t.assign(p.cells, 0.f);
  }
  for (size_t l = 1; l < H.pats.size(); ++l) {
    const Pattern& p = H.pats[l];
    const Level& fl = H.levels[l - 1];
    Level& cl = H.levels[l];
    cl.val.resize(p.col.size());
    for (size_t e = 0; e < p.col.size(); ++e) {
      float s = 0.f;
      for (uint32_t q = p.src_ptr[e]; q < p.src_ptr[e + 1]; ++q) s += fl.val[p.src[q]];
      cl.val[e] = SCALE * s;
    }
    cl.mass.resize(p.cells);
    cl.diag.resize(p.cells);
    for (size_t r = 0; r < p.cells; ++r) {
      float s = 0.f;
      for (uint32_t q = p.kid_ptr[r]; q < p.kid_ptr[r + 1]; ++q) s += fl.mass[p.kids[q]];
      float k = 0.f;
      for (uint32_t e = p.ptr[r]; e < p.ptr[r + 1]; ++e) k += cl.val[e];
      cl.mass[r] = s;
      cl.diag[r] = s + k;
    }
    cl.r.assign(p.cells, 0.f);
    cl.z.assign(p.cells, 0.f);
    cl.t.assign(p.cells, 0.f);
  }
}

// multigrid.rs:284-310: one damped Jacobi sweep (from z = 0 when `first`)
static void sweep(const Pattern& p, Level& lv, bool first) {
  if (first) {
    for (size_t i = 0; i < p.cells; ++i) lv.z[i] = OMEGA * lv.r[i] / lv.diag[i];
    return;
  }
#pragma omp parallel for schedule(static)
  for (long i = 0; i < (long)p.cells; ++i) {
    float az = lv.diag[i] * lv.z[i];
    for (uint32_t e = p.ptr[i]; e < p.ptr[i + 1]; ++e) az -= lv.val[e] * lv.z[p.col[e]];
    lv.t[i] = lv.z[i] + OMEGA * (lv.r[i] - az) / lv.diag[i];
  }
  std::swap(lv.z, lv.t);
}

// multigrid.rs:312-363
static void vcycle(Hierarchy& H, size_t l) {
  const Pattern& p = H.pats[l];
  Level& lv = H.levels[l];
  if (l + 1 == H.pats.size()) {
    for (int k = 0; k < COARSE_SWEEPS; ++k) sweep(p, lv, k == 0);
    return;
  }
  for (int k = 0; k < NU; ++k) sweep(p, lv, k == 0);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < (long)p.cells; ++i) {
    float az = lv.diag[i] * lv.z[i];
    for (uint32_t e = p.ptr[i]; e < p.ptr[i + 1]; ++e) az -= lv.val[e] * lv.z[p.col[e]];
    lv.t[i] = lv.r[i] - az;
  }
  const Pattern& cp = H.pats[l + 1];
  Level& cl = H.levels[l + 1];
  for (size_t rc = 0; rc < cp.cells; ++rc) {
    float s = 0.f;
    for (uint32_t q = cp.kid_ptr[rc]; q < cp.kid_ptr[rc + 1]; ++q) s += lv.t[cp.kids[q]];
    cl.r[rc] = s;
  }
  vcycle(H, l + 1);
  for (size_t c = 0; c < p.cells; ++c) lv.z[c] += cl.z[cp.parent[c]];
  for (int k = 0; k < NU; ++k) sweep(p, lv, false);
}

// multigrid.rs:271-282
static void precondition(Hierarchy& H, const double* r, double* z) {
  Level& lv = H.levels[0];
  for (size_t i = 0; i < lv.r.size(); ++i) lv.r[i] = (float)r[i];
  vcycle(H, 0);
  for (size_t i = 0; i < lv.z.size(); ++i) z[i] = (double)lv.z[i];
}

// diffusion.rs:387-500: CG from x, preconditioned by the V-cycle; RMS stop over every cell
static int cg(const Op& op, Hierarchy& H, const double* rhs, double* x, double tol_m) {
  const size_t l = op.cells;
  const double tol2 = tol_m * tol_m * (double)l;
  std::vector<double> r(l), po(l, 0.0), pn(l), ap(l), z(l);
  op.apply(x, r.data());
  for (size_t i = 0; i < l; ++i) r[i] = rhs[i] - r[i];
  double rr0 = ordered_sum(l, [&](size_t i) { return r[i] * r[i]; });
  if (rr0 <= tol2) return 0;
  precondition(H, r.data(), z.data());
  double rz = ordered_sum(l, [&](size_t i) { return r[i] * z[i]; });
  bool has_beta = false;
  double beta = 0.0;
  int iterations = 0;
  for (int it = 0; it < CG_MAX_ITER; ++it) {
    auto dir = [&](size_t j) { return has_beta ? z[j] + beta * po[j] : z[j]; };
    double pap = ordered_sum(l, [&](size_t i) {
      double pi = dir(i);
      double acc = op.diag[i] * pi;
      for (int t = 0; t < 8; ++t) {
        uint32_t j = op.slots[i * 8 + t];
        if (j != NO_CELL) acc -= op.k[i * 8 + t] * dir(j);
      }
      pn[i] = pi;
      ap[i] = acc;
      return pi * acc;
    });
    std::swap(po, pn);
    if (std::isnan(pap) || pap <= 0.0) break;
    double alpha = rz / pap;
    double rr = ordered_sum(l, [&](size_t i) {
      x[i] += alpha * po[i];
      double rv = r[i] - alpha * ap[i];
      r[i] = rv;
      return rv * rv;
    });
    ++iterations;
    if (rr <= tol2) break;
    precondition(H, r.data(), z.data());
    double rz_new = ordered_sum(l, [&](size_t i) { return r[i] * z[i]; });
    beta = rz_new / rz;
    has_beta = true;
    rz = rz_new;
  }
  return iterations;
}

}  // namespace oracle_cube

using namespace oracle_cube;

extern "C" {

void dto_cube_topology(int n, uint32_t* slots) { topology((size_t)n, slots); }

// y = A x, the built operator (diffusion.rs:64-86)
void dto_cube_operator(int n, const uint32_t* slots, const double* lap, const double* areas, const double* kd, double dt,
                       const double* x, double* y) {
  Op op;
  build(op, n, slots, lap, areas, kd, dt);
  op.apply(x, y);
}

// z = V-cycle(r) on the built operator's hierarchy (multigrid.rs:199-282)
void dto_cube_vcycle(int n, const uint32_t* slots, const double* lap, const double* areas, const double* kd, double dt,
                     const double* r, double* z) {
  Op op;
  build(op, n, slots, lap, areas, kd, dt);
  Hierarchy H;
  prepare(H, op);
  precondition(H, r, z);
}

// The LOD first guess alone (diffusion.rs:315-381), x from b = h
void dto_cube_lod(int n, const uint32_t* slots, const double* lap, const double* areas, const double* kd, double dt,
                  const double* h, double* x) {
  Op op;
  build(op, n, slots, lap, areas, kd, dt);
  std::vector<double> tmp(op.cells);
  std::copy(h, h + op.cells, x);
  lod(op, h, x, tmp.data());
}

// diffusion::solve with DiffusionSolver::Multigrid on the cube (diffusion.rs:244-313): h in/out;
// returns the iterations (0 for dt <= 0 or NaN).
int dto_cube_diff_solve(int n, const uint32_t* slots, const double* lap, const double* areas, const double* kd, double dt,
                        double tol_m, double* h) {
  if (std::isnan(dt) || dt <= 0.0) return 0;
  Op op;
  build(op, n, slots, lap, areas, kd, dt);
  const size_t l = op.cells;
  std::vector<double> rhs(l), x(l), b(l), tmp(l), ap(l);
  for (size_t i = 0; i < l; ++i) {
    rhs[i] = op.mu[i] * h[i];
    x[i] = h[i];
  }
  b = x;
  lod(op, b.data(), x.data(), tmp.data());
  Hierarchy H;
  prepare(H, op);
  int iterations = cg(op, H, rhs.data(), x.data(), tol_m);
  // the residual's sum back to the cells in proportion to their coupling (diffusion.rs:290-301)
  op.apply(x.data(), ap.data());
  double lost = ordered_sum(l, [&](size_t i) { return rhs[i] - ap[i]; });
  double weight = ordered_sum(l, [&](size_t i) { return op.s[i]; });
  if (weight > 0.0 && lost != 0.0) {
    double kk = lost / weight;
    for (size_t i = 0; i < l; ++i) x[i] += kk * op.s[i] / op.mu[i];
  }
  std::copy(x.begin(), x.end(), h);
  return iterations;
}

}  // extern "C"

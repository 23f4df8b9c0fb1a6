// Test infrastructure only: the CPU oracle's complex FFT. Nothing in the product links this.
//
// The reference plans its transforms with rustfft 6.4.1 (crates/deeptime-core/Cargo.toml:31,
// Cargo.lock:1207-1209; plans at crates/deeptime-core/src/surface/flexure.rs:1140-1166). rustfft
// is not vendored in the reference, so this is a restatement of the published algorithms it
// computes: the unnormalised DFT X[k] = sum_n x[n] e^(-+2 pi i nk/N) (forward -, inverse +).
// Power-of-two sizes use an iterative radix-2 Cooley-Tukey transform; every other size uses
// Bluestein's chirp-z algorithm (Bluestein 1970) on a power-of-two convolution. Twiddles are
// computed from k*k mod 2N so the chirp angle never loses precision.
#pragma once
#include <cmath>
#include <complex>
#include <memory>
#include <vector>

namespace oracle {

using cd = std::complex<double>;

inline bool is_pow2(size_t n) { return n && !(n & (n - 1)); }

// exp(sign * i * pi * num / den), evaluated in long double.
inline cd unit_root(long double num, long double den, int sign) {
  long double a = 3.14159265358979323846264338327950288L * num / den;
  return cd((double)cosl(a), (double)(sign * sinl(a)));
}

class Fft {
 public:
  Fft() : n_(0), sign_(-1) {}
  Fft(size_t n, bool inverse) : n_(n), sign_(inverse ? 1 : -1) {
    if (n_ <= 1) return;
    if (is_pow2(n_)) {
      tw_.resize(n_ / 2);
      for (size_t k = 0; k < n_ / 2; ++k) tw_[k] = unit_root(2.0L * k, (long double)n_, sign_);
    } else {
      m_ = 1;
      while (m_ < 2 * n_ - 1) m_ <<= 1;
      inner_f_ = std::make_shared<Fft>(m_, false);
      inner_i_ = std::make_shared<Fft>(m_, true);
      chirp_.resize(n_);
      for (size_t k = 0; k < n_; ++k) {
        unsigned long long kk = (unsigned long long)k * k % (2ULL * n_);
        chirp_[k] = unit_root((long double)kk, (long double)n_, sign_);  // e^(s i pi k^2/n)
      }
      bhat_.assign(m_, cd(0, 0));
      bhat_[0] = std::conj(chirp_[0]);
      for (size_t k = 1; k < n_; ++k) bhat_[k] = bhat_[m_ - k] = std::conj(chirp_[k]);
      inner_f_->run(bhat_.data());
    }
  }
  size_t size() const { return n_; }

  void run(cd* x) const {
    if (n_ <= 1) return;
    if (is_pow2(n_)) {
      radix2(x);
      return;
    }
    std::vector<cd> a(m_, cd(0, 0));
    for (size_t k = 0; k < n_; ++k) a[k] = x[k] * chirp_[k];
    inner_f_->run(a.data());
    for (size_t k = 0; k < m_; ++k) a[k] *= bhat_[k];
    inner_i_->run(a.data());
    double inv = 1.0 / (double)m_;
    for (size_t k = 0; k < n_; ++k) x[k] = a[k] * inv * chirp_[k];
  }

 private:
  void radix2(cd* x) const {
    const size_t n = n_;
    for (size_t i = 1, j = 0; i < n; ++i) {
      size_t bit = n >> 1;
      for (; j & bit; bit >>= 1) j ^= bit;
      j ^= bit;
      if (i < j) std::swap(x[i], x[j]);
    }
    for (size_t len = 2; len <= n; len <<= 1) {
      size_t step = n / len;
      for (size_t i = 0; i < n; i += len) {
        for (size_t k = 0; k < len / 2; ++k) {
          cd u = x[i + k];
          cd v = x[i + k + len / 2] * tw_[k * step];
          x[i + k] = u + v;
          x[i + k + len / 2] = u - v;
        }
      }
    }
  }
  size_t n_;
  int sign_;
  size_t m_ = 0;
  std::vector<cd> tw_;
  std::vector<cd> chirp_, bhat_;
  std::shared_ptr<Fft> inner_f_, inner_i_;
};

}  // namespace oracle

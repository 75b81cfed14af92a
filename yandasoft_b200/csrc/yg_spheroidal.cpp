// Host-side spheroidal function, grid-correction vectors and a small FFT.
#include "yg_spheroidal.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <stdexcept>

namespace yg {

namespace {

// Eigen-decomposition of a small symmetric matrix by cyclic Jacobi rotations.
// a is n x n row-major (destroyed); returns eigenvalues, eigenvectors in
// columns of v.
void jacobi_eigen(std::vector<double>& a, int n, std::vector<double>& evals, std::vector<double>& v) {
  v.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) v[(size_t)i * n + i] = 1.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) off += a[(size_t)p * n + q] * a[(size_t)p * n + q];
    if (off < 1e-30) break;
    for (int p = 0; p < n; ++p) {
      for (int q = p + 1; q < n; ++q) {
        const double apq = a[(size_t)p * n + q];
        if (std::fabs(apq) < 1e-300) continue;
        const double app = a[(size_t)p * n + p], aqq = a[(size_t)q * n + q];
        const double theta = (aqq - app) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; ++k) {
          const double akp = a[(size_t)k * n + p], akq = a[(size_t)k * n + q];
          a[(size_t)k * n + p] = c * akp - s * akq;
          a[(size_t)k * n + q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {
          const double apk = a[(size_t)p * n + k], aqk = a[(size_t)q * n + k];
          a[(size_t)p * n + k] = c * apk - s * aqk;
          a[(size_t)q * n + k] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          const double vkp = v[(size_t)k * n + p], vkq = v[(size_t)k * n + q];
          v[(size_t)k * n + p] = c * vkp - s * vkq;
          v[(size_t)k * n + q] = s * vkp + c * vkq;
        }
      }
    }
  }
  evals.resize(n);
  for (int i = 0; i < n; ++i) evals[i] = a[(size_t)i * n + i];
}

}  // namespace

Spheroidal::Spheroidal(double c, double alpha, int nterms) : alpha_(alpha), m_((int)alpha), nterms_(nterms) {
  const int n = nterms;
  const double c2 = c * c;
  const int m = m_;
  std::vector<double> b((size_t)n * n, 0.0);
  for (int row = 0; row < n; ++row) {
    const double l = 2.0 * row + m;
    b[(size_t)row * n + row] =
        l * (l + 1) + c2 * ((2 * l + 3) * (l + m) * (l - m) + (2 * l - 1) * (l + m + 1) * (l - m + 1)) /
                          ((2 * l + 1) * (2 * l - 1) * (2 * l + 3));
    if (row >= 1)
      b[(size_t)row * n + row - 1] =
          c2 / (2 * l - 1) * std::sqrt((l + m) * (l + m - 1) * (l - m) * (l - m - 1) / ((2 * l + 1) * (2 * l - 3)));
    if (row + 1 < n)
      b[(size_t)row * n + row + 1] = c2 / (2 * l + 3) *
                                     std::sqrt((l + m + 1) * (l + m + 2) * (l - m + 1) * (l - m + 2) /
                                               ((2 * l + 1) * (2 * l + 5)));
  }
  // symmetrise numerically (the analytic matrix is symmetric)
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j) {
      const double s = 0.5 * (b[(size_t)i * n + j] + b[(size_t)j * n + i]);
      b[(size_t)i * n + j] = b[(size_t)j * n + i] = s;
    }
  std::vector<double> ev, vec;
  jacobi_eigen(b, n, ev, vec);
  int best = 0;
  for (int i = 1; i < n; ++i)
    if (ev[i] < ev[best]) best = i;
  coeffs_.resize(n);
  for (int i = 0; i < n; ++i) coeffs_[i] = vec[(size_t)i * n + best];
  sum0_ = series(0.0);
}

// sum_k coeffs_k * Pbar_{m+2k}^m(eta) with orthonormal associated Legendre
// functions evaluated by the upward three-term recurrence in l.
double Spheroidal::series(double x) const {
  const int m = m_;
  const int lmax = m + 2 * (nterms_ - 1);
  const double s = std::sqrt(std::max(0.0, 1.0 - x * x));
  double pmm = std::sqrt(0.5);
  for (int k = 1; k <= m; ++k) pmm = -pmm * std::sqrt((2.0 * k + 1.0) / (2.0 * k)) * s;
  double sum = coeffs_[0] * pmm;
  if (lmax == m) return sum;
  double pm1 = x * std::sqrt(2.0 * m + 3.0) * pmm;
  double prev = pmm, cur = pm1;
  for (int l = m + 2; l <= lmax; ++l) {
    const double a = std::sqrt((4.0 * l * l - 1.0) / ((double)l * l - (double)m * m));
    const double bb = std::sqrt(((l - 1.0) * (l - 1.0) - (double)m * m) / (4.0 * (l - 1.0) * (l - 1.0) - 1.0));
    const double next = a * (x * cur - bb * prev);
    prev = cur;
    cur = next;
    if (((l - m) & 1) == 0) sum += coeffs_[(l - m) / 2] * next;
  }
  return sum;
}

double Spheroidal::operator()(double nu) const {
  if (!(std::fabs(nu) < 1.0)) return 0.0;
  return series(nu) / sum0_ * std::pow(1.0 - nu * nu, -alpha_ / 2.0);
}

void fft1d_centred(std::vector<double>& re, std::vector<double>& im, bool forward) {
  const int n = (int)re.size();
  // ifftshift
  std::vector<std::complex<double>> a(n), out(n);
  for (int i = 0; i < n; ++i) a[i] = std::complex<double>(re[(i + n / 2) % n], im[(i + n / 2) % n]);
  const double sign = forward ? -1.0 : 1.0;
  if ((n & (n - 1)) == 0) {
    // iterative radix-2
    for (int i = 1, j = 0; i < n; ++i) {
      int bit = n >> 1;
      for (; j & bit; bit >>= 1) j ^= bit;
      j ^= bit;
      if (i < j) std::swap(a[i], a[j]);
    }
    for (int len = 2; len <= n; len <<= 1) {
      const double ang = sign * 2.0 * M_PI / len;
      for (int i = 0; i < n; i += len) {
        for (int k = 0; k < len / 2; ++k) {
          const std::complex<double> w(std::cos(ang * k), std::sin(ang * k));
          const std::complex<double> u = a[i + k], v = a[i + k + len / 2] * w;
          a[i + k] = u + v;
          a[i + k + len / 2] = u - v;
        }
      }
    }
    out = a;
  } else {
    for (int k = 0; k < n; ++k) {
      std::complex<double> s(0.0, 0.0);
      for (int j = 0; j < n; ++j) {
        const double ang = sign * 2.0 * M_PI * (double)((long long)j * k % n) / n;
        s += a[j] * std::complex<double>(std::cos(ang), std::sin(ang));
      }
      out[k] = s;
    }
  }
  const double scale = forward ? 1.0 : 1.0 / n;
  // fftshift
  for (int i = 0; i < n; ++i) {
    const std::complex<double> v = out[(i + n - n / 2) % n] * scale;
    re[i] = v.real();
    im[i] = v.imag();
  }
}

std::vector<double> sph_correction(int n, const Spheroidal& grdsf, bool interp) {
  const int half = n / 2;
  std::vector<double> re(n), im(n, 0.0);
  for (int i = 0; i < n; ++i) {
    const double nu = std::fabs((double)(i - half)) / (double)half;
    re[i] = (float)grdsf(nu);
  }
  if (interp && n > 3) {
    re[0] = (float)((float)3.0f * ((float)re[1] - (float)re[2]) + (float)re[3]);
    if (n % 2 == 1) re[n - 1] = re[0];
  }
  const int support = 3;
  const double max_before = re[half];
  fft1d_centred(re, im, true);
  for (int i = 0; i < half - support; ++i) re[i] = im[i] = 0.0;
  for (int i = half + support + 1; i < n; ++i) re[i] = im[i] = 0.0;
  fft1d_centred(re, im, false);
  // normalisation = maxBefore / buf(n/2) (complex), applied to the whole vector
  const std::complex<double> norm = std::complex<double>(max_before, 0.0) / std::complex<double>(re[half], im[half]);
  std::vector<double> ccf(n);
  for (int i = 0; i < n; ++i) {
    const double v = (std::complex<double>(re[i], im[i]) * norm).real();
    ccf[i] = std::fabs(v) > 1e-10 ? 1.0 / v : 0.0;
  }
  return ccf;
}

}  // namespace yg

// Prolate spheroidal wave function psi_{alpha,0}(c, nu), normalised to 1 at
// nu = 0 and zero for |nu| >= 1: the grdsf() of yandasoft's gridders
// (askap/gridding/SphFuncVisGridder.h:101, constructed as
// SpheroidalFunction(pi*support, alpha) at SphFuncVisGridder.cc:47).  The
// class itself is in the un-vendored base-scimath library; the method is the
// Legendre-series eigenvector expansion that the reference documents in
// apps/gridderExperiments.cc:180-260.
#pragma once
#include <vector>

namespace yg {

class Spheroidal {
 public:
  Spheroidal(double c, double alpha, int nterms = 16);
  double operator()(double nu) const;

 private:
  double series(double eta) const;
  double alpha_;
  int m_;
  int nterms_;
  std::vector<double> coeffs_;
  double sum0_;
};

// 1-D filtered correction factors of SphFuncVisGridder::correctConvolution
// (askap/gridding/SphFuncVisGridder.cc:171-248) for an axis of n pixels.
std::vector<double> sph_correction(int n, const Spheroidal& grdsf, bool interp = true);

// In-place centred complex FFT of length n (origin at n/2), double precision:
// forward = exp(-2 pi i), backward = exp(+2 pi i) / n.
void fft1d_centred(std::vector<double>& re, std::vector<double>& im, bool forward);

}  // namespace yg

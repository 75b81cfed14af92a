// Shared device-side definitions of the B200 gridder.
//
// FP64 index arithmetic here is written with explicit round-to-nearest
// intrinsics (__dmul_rn, __ddiv_rn, __dadd_rn) so that no multiply-add is
// contracted: every uv-cell, oversample offset and w-plane choice is the
// IEEE result of the same operation sequence as the reference's C++
// (askap/gridding/TableVisGridder.cc:616-650, WDependentGridderBase.cc:118-150).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace yg {

constexpr double kC = 299792458.0;
constexpr double kPi = 3.14159265358979323846;

// Error codes shared by device kernels, the host classes and the C-ABI.
enum : int {
  YG_OK = 0,
  YG_ERR_ARG = 1,
  YG_ERR_CUDA = 2,
  YG_ERR_FRAC = 3,       // fractional offset outside [0, oversample)
  YG_ERR_WRANGE = 4,     // w outside (-wmax, wmax) and wmaxclip off
  YG_ERR_WEIGHT = 5,     // non-positive visibility weight
  YG_ERR_CINDEX = 6,     // convolution-function index out of range
  YG_ERR_SUPPORT = 7,    // support search failed / CF overflow
  YG_ERR_STATE = 8,      // call out of sequence
  YG_ERR_UNSUPPORTED = 9,
  YG_ERR_FREQ = 10,
  YG_ERR_TIMEOUT = 11,
  YG_ERR_NOMEM = 12
};

// askap::nint (base-askap): round half away from zero by adding +-0.5 in FP64
// and truncating.
__host__ __device__ inline int nint_d(double x) {
#ifdef __CUDA_ARCH__
  return x > 0 ? (int)__dadd_rn(x, 0.5) : (int)__dsub_rn(x, 0.5);
#else
  return x > 0 ? (int)(x + 0.5) : (int)(x - 0.5);
#endif
}

// w-sampling kinds of WDependentGridderBase
enum { WS_LINEAR = 0, WS_POWER = 1, WS_GAUSS = 2 };

struct WSampling {
  int nwplanes;
  int kind;
  int wmaxclip;
  int pad_;
  double wscale;      // wmax / ((n-1)/2) (1 when n == 1)
  double exponent;    // power law
  double two_sigma2;  // gaussian
  double amplitude;   // gaussian
};

// IWSampling::index for the non-linear samplings (PowerWSampling.cc:69-80,
// GaussianWSampling.cc:82-103).  Returns false where the reference throws.
__device__ inline bool ws_index(const WSampling& s, double wt, double* out) {
  if (s.kind == WS_POWER) {
    if (wt > 0) { *out = pow(wt, 1.0 / s.exponent); return true; }
    if (wt < 0) { *out = -pow(-wt, 1.0 / s.exponent); return true; }
    *out = 0.0;
    return true;
  }
  if (wt == -1.0 || wt == 1.0) { *out = wt; return true; }
  const double expterm = 1.0 - fabs(wt) / s.amplitude;
  if (!(expterm > 0.0)) return false;
  const double p2 = -log(expterm) * s.two_sigma2;
  if (!(p2 >= 0.0)) return false;
  *out = wt < 0 ? -sqrt(p2) : (wt > 0 ? sqrt(p2) : 0.0);
  return true;
}

// WDependentGridderBase::getWPlane.  Returns the plane, -1 when clipped; sets
// *err when the reference would throw.
__device__ inline int get_wplane(const WSampling& s, double w, int* err) {
  int result;
  if (s.kind != WS_LINEAR && s.nwplanes > 1) {
    const int half = (s.nwplanes - 1) / 2;
    const double wmaxv = __dmul_rn(s.wscale, (double)half);
    double scaled;
    if (!ws_index(s, __ddiv_rn(w, wmaxv), &scaled)) { *err = YG_ERR_WRANGE; return -1; }
    result = half + nint_d(__dmul_rn(scaled, (double)half));
  } else {
    result = s.nwplanes > 1 ? (s.nwplanes - 1) / 2 + nint_d(__ddiv_rn(w, s.wscale)) : 0;
  }
  if (result < s.nwplanes && result > -1) return result;
  if (!s.wmaxclip) *err = YG_ERR_WRANGE;
  return -1;
}

// uv scaling of one axis: scaled = f*coord/(C*cell); i = nint(scaled);
// frac = nint(os*(i - scaled)); fold frac into [0, os); i += n/2.
__device__ inline bool axis_index(double f, double coord, double cell, int os, int n, int* pi, int* pf) {
  const double scaled = __ddiv_rn(__dmul_rn(f, coord), __dmul_rn(kC, cell));
  int i = nint_d(scaled);
  int frac = nint_d(__dmul_rn((double)os, __dsub_rn((double)i, scaled)));
  if (frac < 0) { i += 1; frac += os; }
  else if (frac >= os) { i -= 1; frac -= os; }
  *pi = i + n / 2;
  *pf = frac;
  return frac >= 0 && frac < os;
}

// Record of the first device-side error, read back by the host.
struct DevError {
  int code;
  int pad_;
  long long where;  // sample / item index
};

__device__ inline void raise_error(DevError* e, int code, long long where) {
  if (atomicCAS(&e->code, 0, code) == 0) e->where = where;
}

// Where-field of a bounded wait that gave up (YG_ERR_TIMEOUT): the kernel
// (1 k_grid, 2 k_grid_pl, 3 k_degrid_t, 4 k_degrid_r), the waiting role (1 the
// producer warp for a free stage, 2 a tap warp for a filled one, 3 the
// producer for the plane buffer), the segment index and the block.
__device__ inline long long timeout_where(int kernel, int role, int seg, int block) {
  return ((long long)kernel << 60) | ((long long)role << 56) | ((long long)(seg & 0xffffff) << 32) |
         (long long)(unsigned)block;
}

}  // namespace yg

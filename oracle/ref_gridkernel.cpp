// Test infrastructure (oracle/_ref): C entry points around the reference's
// own GridKernel::grid / GridKernel::degrid (askap/gridding/GridKernel.cc,
// compiled unchanged from the reference tree with ASKAP_GRID_WITH_POINTERS,
// as its CMakeLists.txt:189,342 enables), with the signatures of the oracle's
// tap loops, so that the oracle's generic loop can run on the reference's
// compiled arithmetic (orc_set_tap_kernels) and be compared bit for bit.
#include <askap/gridding/GridKernel.h>

using askap::synthesis::GridKernel;

extern "C" {

// grid plane: column-major complex (nx rows); cf: (2S+1)^2 column-major complex
void ref_grid_kernel(float* grid, int nx, const float* cf, float rv, float iv, int iu, int ivv, int support) {
  const int w = 2 * support + 1;
  casacore::Matrix<casacore::Complex> g(reinterpret_cast<casacore::Complex*>(grid), nx, 1 << 30);
  casacore::Matrix<casacore::Complex> c(reinterpret_cast<casacore::Complex*>(const_cast<float*>(cf)), w, w);
  GridKernel::grid(g, c, casacore::Complex(rv, iv), iu, ivv, support);
}

void ref_degrid_kernel(float* out, const float* grid, int nx, const float* cf, int iu, int ivv, int support) {
  const int w = 2 * support + 1;
  const casacore::Matrix<casacore::Complex> g(reinterpret_cast<casacore::Complex*>(const_cast<float*>(grid)), nx,
                                              1 << 30);
  const casacore::Matrix<casacore::Complex> c(reinterpret_cast<casacore::Complex*>(const_cast<float*>(cf)), w, w);
  casacore::Complex v;
  GridKernel::degrid(v, c, g, iu, ivv, support);
  out[0] = v.real();
  out[1] = v.imag();
}

int ref_grid_kernel_info(char* buf, int n) {
  const std::string s = GridKernel::info();
  int k = 0;
  for (; k + 1 < n && k < (int)s.size(); ++k) buf[k] = s[k];
  if (n > 0) buf[k] = 0;
  return (int)s.size();
}
}

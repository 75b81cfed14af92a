// Image-side FFT steps (finaliseGrid / initialiseDegrid) on the GPU.
#pragma once
#include <cufft.h>

#include <vector>

#include "yg_internal.h"

namespace yg {

struct StackScreen {
  int nx, ny;
  float cellx, celly;   // FP32 image cell (radians), as WStackVisGridder::multiply
  float w;              // FP32 2 pi w
};

StackScreen make_stack_screen(int nx, int ny, double uvcell_u, double uvcell_v, double wterm);

struct ImageFFT {
  cufftHandle plan = 0;
  bool plan_ok = false;
  int nx = 0, ny = 0, nplanes = 0;
  DevBuf work;
  int ensure(int nx, int ny, int nplanes, cudaStream_t st);
  ~ImageFFT();
};

int image_finalise(ImageFFT& f, const float2* grids, int ngrids, int nx, int ny, int nplanes,
                   const std::vector<StackScreen>* screens, const double* corr_x, const double* corr_y, float* out,
                   cudaStream_t st);
int image_to_grids(ImageFFT& f, const float* image, int nx, int ny, int nplanes,
                   const std::vector<StackScreen>* screens, int ngrids, const double* corr_x, const double* corr_y,
                   float* corrected_tmp, float2* grids, cudaStream_t st);

// AWProject finaliseWeights: planes[r] = CF index of sum-of-weights row r with
// data, offs[r] its CF offset, wts[r * nplanes + pol + npol * chan] its
// weights; out is (onx, ony, nplanes) on the device.  taper (cnx + cny
// values, x then y), when given, is the CFs' spheroidal taper, divided out of
// every transformed CF before its |.|^2 is summed
int aw_weights_image(const CFView& cf, const std::vector<int>& planes, const std::vector<int2>& offs,
                     const std::vector<double>& wts, int nplanes, int cnx, int cny, int nx, int ny, int onx, int ony,
                     float* out, cudaStream_t st, const std::vector<double>* taper = nullptr);

}  // namespace yg

// Image-side steps of the gridders on the GPU: finaliseGrid and
// initialiseDegrid (askap/gridding/TableVisGridder.cc:1109-1236,1286-1319)
// and the w-stack variants (askap/gridding/WStackVisGridder.cc:134-171,
// 216-337).  Transforms are batched cuFFT C2C over all (pol, chan) planes with
// the centred-transform checkerboard folded into the element-wise kernels;
// the grid correction (SphFuncVisGridder::correctConvolution) is applied as
// separable FP64 factors in the same pass.
#include <cufft.h>

#include <cmath>
#include <vector>

#include "yg_image.h"

namespace yg {

#define IM_TRY(x)                                 \
  do {                                            \
    cudaError_t e_ = (x);                         \
    if (e_ != cudaSuccess) return YG_ERR_CUDA;    \
  } while (0)

__device__ __forceinline__ float sgn_in(int x, int y) { return ((x + y) & 1) ? -1.f : 1.f; }
__device__ __forceinline__ float sgn_out(int x, int y, int nx, int ny) {
  return ((x + y + nx / 2 + ny / 2) & 1) ? -1.f : 1.f;
}

// FP32 w-stack screen exp(-i w (1 - sqrt(1 - r^2))) of WStackVisGridder::multiply
__device__ __forceinline__ bool wstack_screen(const StackScreen& s, int x, int y, float* cr, float* ci) {
  const float yy = __fmul_rn((float)(y - s.ny / 2), s.celly);
  const float xx = __fmul_rn((float)(x - s.nx / 2), s.cellx);
  const float r2 = __fadd_rn(__fmul_rn(xx, xx), __fmul_rn(yy, yy));
  if (!(r2 < 1.0f)) return false;
  const float phase = (float)((double)s.w * (1.0 - sqrt(1.0 - (double)r2)));
  *cr = cosf(phase);
  *ci = -sinf(phase);
  return true;
}

__global__ void k_sign_copy(const float2* __restrict__ in, float2* __restrict__ out, int nx, int ny, long long total) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % nx), y = (int)((i / nx) % ny);
    const float s = sgn_in(x, y);
    const float2 v = in[i];
    out[i] = make_float2(v.x * s, v.y * s);
  }
}

// acc (+)= real(out_sign * v [* screen])
__global__ void k_accum_real(const float2* __restrict__ f, float* __restrict__ acc, int nx, int ny, long long total,
                             int first, int use_screen, StackScreen scr) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % nx), y = (int)((i / nx) % ny);
    const float s = sgn_out(x, y, nx, ny);
    float2 v = f[i];
    v.x *= s;
    v.y *= s;
    float r = v.x;
    if (use_screen) {
      float cr, ci;
      if ((v.x != 0.f || v.y != 0.f) && wstack_screen(scr, x, y, &cr, &ci)) r = __fsub_rn(__fmul_rn(v.x, cr), __fmul_rn(v.y, ci));
    }
    acc[i] = first ? r : __fadd_rn(acc[i], r);
  }
}

// img *= ccfx[x] * ccfy[y] (FP64 factors, FP32 result)
__global__ void k_correct(float* __restrict__ img, const double* __restrict__ cx, const double* __restrict__ cy,
                          int nx, int ny, long long total) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % nx), y = (int)((i / nx) % ny);
    img[i] = (float)((double)img[i] * (cx[x] * cy[y]));
  }
}

// image (already corrected) -> in_sign * [conj](complex(img) [* screen])
__global__ void k_image_to_c(const float* __restrict__ img, float2* __restrict__ out, int nx, int ny, long long total,
                             int use_screen, StackScreen scr) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % nx), y = (int)((i / nx) % ny);
    float2 v = make_float2(img[i], 0.f);
    if (use_screen) {
      float cr, ci;
      if (v.x != 0.f && wstack_screen(scr, x, y, &cr, &ci)) v = make_float2(__fmul_rn(v.x, cr), __fmul_rn(v.x, ci));
      v.y = -v.y;
    }
    const float s = sgn_in(x, y);
    out[i] = make_float2(v.x * s, v.y * s);
  }
}

__global__ void k_sign_out(float2* __restrict__ g, int nx, int ny, long long total) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % nx), y = (int)((i / nx) % ny);
    const float s = sgn_out(x, y, nx, ny);
    const float2 v = g[i];
    g[i] = make_float2(v.x * s, v.y * s);
  }
}

static int blocks_for(long long total) {
  long long b = (total + 255) / 256;
  return (int)(b > 148 * 64 ? 148 * 64 : (b < 1 ? 1 : b));
}

StackScreen make_stack_screen(int nx, int ny, double uvcell_u, double uvcell_v, double wterm) {
  StackScreen s;
  s.nx = nx;
  s.ny = ny;
  s.cellx = (float)(1.0 / ((double)(float)nx * uvcell_u));
  s.celly = (float)(1.0 / ((double)(float)ny * uvcell_v));
  s.w = (float)(2.0 * M_PI * wterm);
  return s;
}

int ImageFFT::ensure(int nx_, int ny_, int nplanes_, cudaStream_t st) {
  if (plan_ok && nx == nx_ && ny == ny_ && nplanes == nplanes_) {
    cufftSetStream(plan, st);
    return YG_OK;
  }
  if (plan_ok) cufftDestroy(plan);
  plan_ok = false;
  nx = nx_;
  ny = ny_;
  nplanes = nplanes_;
  int dims[2] = {ny, nx};
  if (cufftPlanMany(&plan, 2, dims, nullptr, 1, nx * ny, nullptr, 1, nx * ny, CUFFT_C2C, nplanes) != CUFFT_SUCCESS)
    return YG_ERR_CUDA;
  plan_ok = true;
  cufftSetStream(plan, st);
  IM_TRY(work.ensure((size_t)nx * ny * nplanes * sizeof(float2)));
  return YG_OK;
}

ImageFFT::~ImageFFT() {
  if (plan_ok) cufftDestroy(plan);
}

// image[nx, ny, nplanes] = sum_g real(backward FFT(grid_g) [* screen_g]) * corr
int image_finalise(ImageFFT& f, const float2* grids, int ngrids, int nx, int ny, int nplanes,
                   const std::vector<StackScreen>* screens, const double* corr_x, const double* corr_y, float* out,
                   cudaStream_t st) {
  int rc = f.ensure(nx, ny, nplanes, st);
  if (rc) return rc;
  const long long total = (long long)nx * ny * nplanes;
  for (int g = 0; g < ngrids; ++g) {
    k_sign_copy<<<blocks_for(total), 256, 0, st>>>(grids + (size_t)g * total, f.work.as<float2>(), nx, ny, total);
    if (cufftExecC2C(f.plan, (cufftComplex*)f.work.p, (cufftComplex*)f.work.p, CUFFT_INVERSE) != CUFFT_SUCCESS)
      return YG_ERR_CUDA;
    StackScreen s{};
    const bool use = screens != nullptr;
    if (use) s = (*screens)[g];
    k_accum_real<<<blocks_for(total), 256, 0, st>>>(f.work.as<float2>(), out, nx, ny, total, g == 0, use, s);
  }
  if (corr_x && corr_y) k_correct<<<blocks_for(total), 256, 0, st>>>(out, corr_x, corr_y, nx, ny, total);
  IM_TRY(cudaGetLastError());
  return YG_OK;
}

// grids_g = forward FFT(in_sign * [conj](corr * image [* screen_g]))
int image_to_grids(ImageFFT& f, const float* image, int nx, int ny, int nplanes,
                   const std::vector<StackScreen>* screens, int ngrids, const double* corr_x, const double* corr_y,
                   float* corrected_tmp, float2* grids, cudaStream_t st) {
  int rc = f.ensure(nx, ny, nplanes, st);
  if (rc) return rc;
  const long long total = (long long)nx * ny * nplanes;
  IM_TRY(cudaMemcpyAsync(corrected_tmp, image, total * sizeof(float), cudaMemcpyDeviceToDevice, st));
  if (corr_x && corr_y) k_correct<<<blocks_for(total), 256, 0, st>>>(corrected_tmp, corr_x, corr_y, nx, ny, total);
  for (int g = 0; g < ngrids; ++g) {
    float2* dst = grids + (size_t)g * total;
    StackScreen s{};
    const bool use = screens != nullptr;
    if (use) s = (*screens)[g];
    k_image_to_c<<<blocks_for(total), 256, 0, st>>>(corrected_tmp, dst, nx, ny, total, use, s);
    if (cufftExecC2C(f.plan, (cufftComplex*)dst, (cufftComplex*)dst, CUFFT_FORWARD) != CUFFT_SUCCESS) return YG_ERR_CUDA;
    k_sign_out<<<blocks_for(total), 256, 0, st>>>(dst, nx, ny, total);
  }
  IM_TRY(cudaGetLastError());
  return YG_OK;
}

}  // namespace yg

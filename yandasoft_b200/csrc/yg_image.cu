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

namespace yg {

// ---------------------------------------------------------------------------
// AWProject finaliseWeights (AWProjectVisGridder.cc:616-766, no spheroidal
// taper): for every sum-of-weights row with data, the CF of its first
// oversampling plane centred in a cnx x cny grid and backward-transformed
// (unnormalised); wt |val|^2 summed per (pol, chan) in row order in FP32 with
// the product in FP64; then a Fourier-domain interpolation to the padded image
// and its centre kept.
// ---------------------------------------------------------------------------
__global__ void k_aw_embed(CFView cf, const int* __restrict__ planes, const int2* __restrict__ offs, int nb, int cnx,
                           int cny, float2* __restrict__ buf) {
  const long long per = (long long)cnx * cny;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < per * nb; i += (long long)gridDim.x * blockDim.x) {
    const int b = (int)(i / per);
    const int x = (int)(i % cnx), y = (int)((i / cnx) % cny);
    float2 v = make_float2(0.f, 0.f);
    const int plane = planes[b];
    if (plane >= 0) {
      const int w = cf.size[plane], s = (w - 1) / 2;
      const int ix = x - cnx / 2 - offs[b].x, iy = y - cny / 2 - offs[b].y;
      if (ix >= -s && ix <= s && iy >= -s && iy <= s) v = cf.data[cf.off[plane] + (ix + s) + (long long)w * (iy + s)];
    }
    const float sg = sgn_in(x, y);
    buf[i] = make_float2(v.x * sg, v.y * sg);
  }
}

__global__ void k_aw_accum(const float2* __restrict__ buf, const double* __restrict__ wts, int nb, int cnx, int cny,
                           int nplanes, const double* __restrict__ tx, const double* __restrict__ ty,
                           float* __restrict__ acc) {
  const long long per = (long long)cnx * cny;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < per * nplanes; i += (long long)gridDim.x * blockDim.x) {
    const int pc = (int)(i / per);
    const long long px = i % per;
    const int x = (int)(px % cnx), y = (int)(px / cnx);
    const float sg = sgn_out(x, y, cnx, cny);
    // a spheroidal taper of the CFs is divided out where it is positive
    // (AWProjectVisGridder.cc:735-745); elsewhere the value is dropped
    const float taper = tx ? (float)__dmul_rn(tx[x], ty[y]) : 1.f;
    float a = acc[i];
    for (int b = 0; b < nb; ++b) {
      const double wt = wts[(size_t)b * nplanes + pc];
      if (!(wt > 0.0)) continue;
      const float2 v = buf[(size_t)b * per + px];
      float vr = v.x * sg, vi = v.y * sg;
      if (tx) {
        vr = taper > 0.f ? __fdiv_rn(vr, taper) : 0.f;
        vi = taper > 0.f ? __fdiv_rn(vi, taper) : 0.f;
      }
      const float r = __fsub_rn(__fmul_rn(vr, vr), __fmul_rn(vi, -vi));
      a = (float)((double)a + wt * (double)r);
    }
    acc[i] = a;
  }
}

__global__ void k_real_to_c_scaled(const float* __restrict__ a, float2* __restrict__ out, int nx, int ny, long long total,
                                   float scale) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % nx), y = (int)((i / nx) % ny);
    out[i] = make_float2(__fmul_rn(a[i], scale) * sgn_in(x, y), 0.f);
  }
}

// spectrum (centred, cnx x cny, forward-transformed with the checkerboard)
// into the centre of an nx x ny zero grid, ready for the backward transform
__global__ void k_embed_spectrum(const float2* __restrict__ in, int cnx, int cny, float2* __restrict__ out, int nx,
                                 int ny, long long total) {
  const int x0 = (nx - cnx) / 2, y0 = (ny - cny) / 2;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % nx), y = (int)((i / nx) % ny);
    const long long p = i / ((long long)nx * ny);
    const int cx = x - x0, cy = y - y0;
    float2 v = make_float2(0.f, 0.f);
    if (cx >= 0 && cy >= 0 && cx < cnx && cy < cny) {
      v = in[(size_t)p * cnx * cny + cx + (size_t)cnx * cy];
      const float so = sgn_out(cx, cy, cnx, cny);
      v.x *= so;
      v.y *= so;
    }
    const float si = sgn_in(x, y);
    out[i] = make_float2(v.x * si, v.y * si);
  }
}

// out[onx, ony, planes] = centre of real(sgn_out * in) / (nx ny)
__global__ void k_extract_real(const float2* __restrict__ in, int nx, int ny, float inv_n, float* __restrict__ out,
                               int onx, int ony, long long total) {
  const int x0 = (nx - onx) / 2, y0 = (ny - ony) / 2;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int ox = (int)(i % onx), oy = (int)((i / onx) % ony);
    const long long p = i / ((long long)onx * ony);
    const int x = ox + x0, y = oy + y0;
    const float2 v = in[(size_t)p * nx * ny + x + (size_t)nx * y];
    out[i] = __fmul_rn(v.x * sgn_out(x, y, nx, ny), inv_n);
  }
}

__global__ void k_extract_plain(const float* __restrict__ in, int nx, int ny, float* __restrict__ out, int onx, int ony,
                                long long total) {
  const int x0 = (nx - onx) / 2, y0 = (ny - ony) / 2;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int ox = (int)(i % onx), oy = (int)((i / onx) % ony);
    const long long p = i / ((long long)onx * ony);
    out[i] = in[(size_t)p * nx * ny + (ox + x0) + (size_t)nx * (oy + y0)];
  }
}

int aw_weights_image(const CFView& cf, const std::vector<int>& planes, const std::vector<int2>& offs,
                     const std::vector<double>& wts, int nplanes, int cnx, int cny, int nx, int ny, int onx, int ony,
                     float* out, cudaStream_t st, const std::vector<double>* taper) {
  const int nrows = (int)planes.size();
  const long long per = (long long)cnx * cny;
  DevBuf acc;
  IM_TRY(acc.ensure((size_t)per * nplanes * sizeof(float)));
  IM_TRY(cudaMemsetAsync(acc.p, 0, (size_t)per * nplanes * sizeof(float), st));
  DevBuf dtaper;
  if (taper) {
    IM_TRY(dtaper.ensure(taper->size() * sizeof(double)));
    IM_TRY(cudaMemcpy(dtaper.p, taper->data(), taper->size() * sizeof(double), cudaMemcpyHostToDevice));
  }
  const double* tx = taper ? dtaper.as<double>() : nullptr;
  const double* ty = taper ? dtaper.as<double>() + cnx : nullptr;
  if (nrows > 0) {
    const int B = std::min(nrows, 32);
    DevBuf buf, dplanes, doffs, dwts;
    IM_TRY(buf.ensure((size_t)per * B * sizeof(float2)));
    IM_TRY(dplanes.ensure(B * sizeof(int)));
    IM_TRY(doffs.ensure(B * sizeof(int2)));
    IM_TRY(dwts.ensure((size_t)B * nplanes * sizeof(double)));
    cufftHandle plan;
    int dims[2] = {cny, cnx};
    if (cufftPlanMany(&plan, 2, dims, nullptr, 1, cnx * cny, nullptr, 1, cnx * cny, CUFFT_C2C, B) != CUFFT_SUCCESS)
      return YG_ERR_CUDA;
    cufftSetStream(plan, st);
    int rc = YG_OK;
    for (int b0 = 0; b0 < nrows && rc == YG_OK; b0 += B) {
      const int nb = std::min(B, nrows - b0);
      std::vector<int> pl(B, -1);
      std::vector<int2> of(B, make_int2(0, 0));
      std::vector<double> w((size_t)B * nplanes, 0.0);
      for (int b = 0; b < nb; ++b) {
        pl[b] = planes[b0 + b];
        of[b] = offs[b0 + b];
        for (int q = 0; q < nplanes; ++q) w[(size_t)b * nplanes + q] = wts[(size_t)(b0 + b) * nplanes + q];
      }
      if (cudaMemcpyAsync(dplanes.p, pl.data(), B * sizeof(int), cudaMemcpyHostToDevice, st) != cudaSuccess ||
          cudaMemcpyAsync(doffs.p, of.data(), B * sizeof(int2), cudaMemcpyHostToDevice, st) != cudaSuccess ||
          cudaMemcpyAsync(dwts.p, w.data(), w.size() * sizeof(double), cudaMemcpyHostToDevice, st) != cudaSuccess) {
        rc = YG_ERR_CUDA;
        break;
      }
      k_aw_embed<<<blocks_for(per * B), 256, 0, st>>>(cf, dplanes.as<int>(), doffs.as<int2>(), B, cnx, cny,
                                                      buf.as<float2>());
      if (cufftExecC2C(plan, (cufftComplex*)buf.p, (cufftComplex*)buf.p, CUFFT_INVERSE) != CUFFT_SUCCESS) {
        rc = YG_ERR_CUDA;
        break;
      }
      k_aw_accum<<<blocks_for(per * nplanes), 256, 0, st>>>(buf.as<float2>(), dwts.as<double>(), B, cnx, cny, nplanes,
                                                           tx, ty, acc.as<float>());
      if (cudaStreamSynchronize(st) != cudaSuccess) rc = YG_ERR_CUDA;   // host staging vectors are reused
    }
    cufftDestroy(plan);
    if (rc) return rc;
  }
  const long long total_out = (long long)onx * ony * nplanes;
  if (cnx == nx && cny == ny) {
    k_extract_plain<<<blocks_for(total_out), 256, 0, st>>>(acc.as<float>(), nx, ny, out, onx, ony, total_out);
  } else {
    DevBuf c1, c2;
    IM_TRY(c1.ensure((size_t)per * nplanes * sizeof(float2)));
    IM_TRY(c2.ensure((size_t)nx * ny * nplanes * sizeof(float2)));
    k_real_to_c_scaled<<<blocks_for(per * nplanes), 256, 0, st>>>(
        acc.as<float>(), c1.as<float2>(), cnx, cny, per * nplanes, (float)((double)nx * ny / ((double)cnx * cny)));
    cufftHandle p1, p2;
    int d1[2] = {cny, cnx}, d2[2] = {ny, nx};
    if (cufftPlanMany(&p1, 2, d1, nullptr, 1, cnx * cny, nullptr, 1, cnx * cny, CUFFT_C2C, nplanes) != CUFFT_SUCCESS)
      return YG_ERR_CUDA;
    if (cufftPlanMany(&p2, 2, d2, nullptr, 1, nx * ny, nullptr, 1, nx * ny, CUFFT_C2C, nplanes) != CUFFT_SUCCESS) {
      cufftDestroy(p1);
      return YG_ERR_CUDA;
    }
    cufftSetStream(p1, st);
    cufftSetStream(p2, st);
    int rc = YG_OK;
    if (cufftExecC2C(p1, (cufftComplex*)c1.p, (cufftComplex*)c1.p, CUFFT_FORWARD) != CUFFT_SUCCESS) rc = YG_ERR_CUDA;
    const long long tot2 = (long long)nx * ny * nplanes;
    if (!rc) k_embed_spectrum<<<blocks_for(tot2), 256, 0, st>>>(c1.as<float2>(), cnx, cny, c2.as<float2>(), nx, ny, tot2);
    if (!rc && cufftExecC2C(p2, (cufftComplex*)c2.p, (cufftComplex*)c2.p, CUFFT_INVERSE) != CUFFT_SUCCESS) rc = YG_ERR_CUDA;
    if (!rc)
      k_extract_real<<<blocks_for(total_out), 256, 0, st>>>(c2.as<float2>(), nx, ny,
                                                           (float)(1.0 / ((double)nx * ny)), out, onx, ony, total_out);
    cudaStreamSynchronize(st);
    cufftDestroy(p1);
    cufftDestroy(p2);
    if (rc) return rc;
  }
  IM_TRY(cudaGetLastError());
  IM_TRY(cudaStreamSynchronize(st));
  return YG_OK;
}

}  // namespace yg

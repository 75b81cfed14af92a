// Convolution-function (CF) generation on the GPU.
//
// WProject (askap/gridding/WProjectVisGridder.cc:435-726): per w-plane the
// spheroidal taper times the w phase screen exp(-i 2 pi w (1 - sqrt(1-r^2))),
// phase in FP64 and stored in FP32 as the reference stores it, is filled into
// a maxsupport^2 buffer; all planes are transformed by one batched cuFFT;
// the support is found on the device with the reference's SupportSearcher
// rules (SupportSearcher.tcc:88-262); the oversampled (2S+1)^2 cuts are
// written straight into the packed HBM CF cache and each is normalised by
// the sequential FP32 sum of its real parts (WProjectVisGridder.cc:612-631).
//
// AWProject (AWProjectVisGridder.cc:259-611, DiskIllumination.cc:85-181): per
// (feed, channel) the disk aperture with the beam-offset phase slope is built
// on the device, inverse transformed, and every w-plane of |A|^2 x w-screen is
// transformed in one batch, scaled by 1/(nx ny) and cut with the os^2 rescale.
//
// SphFunc (SphFuncVisGridder.cc:90-167) is tabulated on the host.
//
// Centred FFTs (origin at N/2) use the checkerboard identity
//   Y = (-1)^(kx+ky) (-1)^(Nx/2+Ny/2) FFT[(-1)^(nx+ny) x]   (Nx, Ny even).
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "yg_cf.h"
#include "yg_spheroidal.h"

namespace yg {

#define CF_TRY(x)                                 \
  do {                                            \
    cudaError_t e_ = (x);                         \
    if (e_ != cudaSuccess) return YG_ERR_CUDA;    \
  } while (0)

#define FFT_TRY(x)                                \
  do {                                            \
    cufftResult r_ = (x);                         \
    if (r_ != CUFFT_SUCCESS) return YG_ERR_CUDA;  \
  } while (0)

// input-side and output-side signs of a centred transform
__device__ __forceinline__ float cb_in(int x, int y) { return ((x + y) & 1) ? -1.f : 1.f; }
__device__ __forceinline__ float cb_out(int x, int y, int nx, int ny) {
  return ((x + y + nx / 2 + ny / 2) & 1) ? -1.f : 1.f;
}

// ---------------------------------------------------------------------------
// cache bookkeeping
// ---------------------------------------------------------------------------
CFView CFCacheDev::view() const {
  CFView v;
  v.data = data.as<float2>();
  v.off = off.as<long long>();
  v.size = size.as<int>();
  v.offsets = noffsets ? offsets.as<int2>() : nullptr;
  v.ncf = ncf;
  v.noffsets = noffsets;
  v.maxsize = maxsize;
  v.varsup = 0;
  for (int sz : h_size)
    if (sz != 0 && sz != maxsize) v.varsup = 1;
  v.pad = pad.p ? pad.as<float2>() : nullptr;
  v.wpad = wpad;
  return v;
}

// padded copy: plane c at c*wpad^2, taps beyond the plane's own size are 0
__global__ void k_cf_pad(const float2* __restrict__ data, const long long* __restrict__ off,
                         const int* __restrict__ size, int ncf, int wpad, float2* __restrict__ out) {
  const long long per = (long long)wpad * wpad;
  const long long total = per * ncf;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i / per);
    const int t = (int)(i % per);
    const int jx = t % wpad, jy = t / wpad;
    const int w = size[c];
    out[i] = (jx < w && jy < w) ? data[off[c] + jx + (long long)w * jy] : make_float2(0.f, 0.f);
  }
}

int CFCacheDev::refresh_pad(cudaStream_t st) {
  wpad = ((maxsize + 15) / 16) * 16;
  if (ncf == 0 || wpad == 0) return YG_OK;
  const long long total = (long long)wpad * wpad * ncf;
  CF_TRY(pad.ensure(total * sizeof(float2)));
  k_cf_pad<<<(int)std::min<long long>((total + 255) / 256, 148 * 64), 256, 0, st>>>(
      data.as<float2>(), off.as<long long>(), size.as<int>(), ncf, wpad, pad.as<float2>());
  CF_TRY(cudaGetLastError());
  return YG_OK;
}

int CFCacheDev::layout(const std::vector<int>& sizes, const std::vector<int2>& offs) {
  ncf = (int)sizes.size();
  h_size = sizes;
  h_off.assign(ncf, 0);
  long long tot = 0;
  maxsize = 0;
  for (int i = 0; i < ncf; ++i) {
    // every plane starts on a 16-byte boundary (an even complex index) so
    // that it can be bulk-copied into shared memory
    tot = (tot + 1) & ~1ll;
    h_off[i] = tot;
    tot += (long long)sizes[i] * sizes[i];
    maxsize = std::max(maxsize, sizes[i]);
  }
  total = tot;
  h_offsets = offs;
  noffsets = (int)offs.size();
  // slack so that a copy rounded up to 16 bytes never leaves the allocation
  CF_TRY(data.ensure((std::max<long long>(tot, 1) + 2) * sizeof(float2)));
  CF_TRY(cudaMemset(data.p, 0, (std::max<long long>(tot, 1) + 2) * sizeof(float2)));
  CF_TRY(off.ensure(std::max(ncf, 1) * sizeof(long long)));
  CF_TRY(size.ensure(std::max(ncf, 1) * sizeof(int)));
  CF_TRY(offsets.ensure(std::max(noffsets, 1) * sizeof(int2)));
  CF_TRY(cudaMemcpy(off.p, h_off.data(), ncf * sizeof(long long), cudaMemcpyHostToDevice));
  CF_TRY(cudaMemcpy(size.p, h_size.data(), ncf * sizeof(int), cudaMemcpyHostToDevice));
  if (noffsets) CF_TRY(cudaMemcpy(offsets.p, h_offsets.data(), noffsets * sizeof(int2), cudaMemcpyHostToDevice));
  return YG_OK;
}

int CFCacheDev::download(std::vector<float2>& out) const {
  out.resize(total);
  if (total) CF_TRY(cudaMemcpy(out.data(), data.p, total * sizeof(float2), cudaMemcpyDeviceToHost));
  return YG_OK;
}

// ---------------------------------------------------------------------------
// SphFunc (host)
// ---------------------------------------------------------------------------
int cf_build_sphfunc(CFCacheDev& cache, int support, int os, double alpha) {
  Spheroidal grdsf(M_PI * support, alpha);
  const int cs = 2 * support + 1;
  std::vector<int> sizes(os * os, cs);
  int e = cache.layout(sizes, {});
  if (e) return e;
  std::vector<float2> h(cache.total + 2, make_float2(0.f, 0.f));
  std::vector<float> bx(cs), by(cs);
  for (int fv = 0; fv < os; ++fv) {
    for (int fu = 0; fu < os; ++fu) {
      const int plane = fu + os * fv;
      for (int i = 0; i < cs; ++i) {
        const double nux = std::fabs((double)(os * (i - support) + fu)) / (double)(support * os);
        const double nuy = std::fabs((double)(os * (i - support) + fv)) / (double)(support * os);
        bx[i] = (float)(grdsf(nux) * std::pow(1.0 - nux * nux, alpha));
        by[i] = (float)(grdsf(nuy) * std::pow(1.0 - nuy * nuy, alpha));
      }
      float2* c = h.data() + cache.h_off[plane];
      // norm = float sum of |cf| over column-major order
      float norm = 0.f;
      for (int iy = 0; iy < cs; ++iy)
        for (int ix = 0; ix < cs; ++ix) {
          const float v = bx[ix] * by[iy];
          c[ix + cs * iy] = make_float2(v, 0.f);
          norm += std::fabs(v);
        }
      // limited-range complex division by (norm, 0): (a*c)/(c*c)
      const float n2 = norm * norm;
      for (int i = 0; i < cs * cs; ++i) {
        const float a = c[i].x * norm;
        c[i].x = a / n2;
        c[i].y = 0.f;
      }
    }
  }
  cache.support = support;
  CF_TRY(cudaMemcpy(cache.data.p, h.data(), h.size() * sizeof(float2), cudaMemcpyHostToDevice));
  int rc = cache.refresh_pad(0);
  if (rc) return rc;
  CF_TRY(cudaDeviceSynchronize());
  return YG_OK;
}

// ---------------------------------------------------------------------------
// device support search
// ---------------------------------------------------------------------------
struct PeakInfo {
  int px, py;
  double peak;
  int blc0, blc1, trc0, trc1;
};

// per column (fixed y): first maximum of |c|^2 in FP64 over x
__global__ void k_colmax(const float2* __restrict__ buf, int nx, int ny, double* colmax, int* colarg) {
  const int y = blockIdx.x;
  double best = -1.0;
  int barg = 0;
  for (int x = threadIdx.x; x < nx; x += blockDim.x) {
    const float2 v = buf[x + (size_t)nx * y];
    const double a = (double)v.x * (double)v.x + (double)v.y * (double)v.y;
    if (a > best) { best = a; barg = x; }
  }
  __shared__ double sb[256];
  __shared__ int sa[256];
  sb[threadIdx.x] = best;
  sa[threadIdx.x] = barg;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      const double b2 = sb[threadIdx.x + o];
      const int a2 = sa[threadIdx.x + o];
      if (b2 > sb[threadIdx.x] || (b2 == sb[threadIdx.x] && a2 < sa[threadIdx.x])) {
        sb[threadIdx.x] = b2;
        sa[threadIdx.x] = a2;
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    colmax[y] = sb[0];
    colarg[y] = sa[0];
  }
}

// across columns: strictly greater than peak^2 wins (peak = sqrt of the best)
// then scans along the peak row/column for the first |c|^2 (FP32) above the
// threshold from each edge.
__global__ void k_peak_support(const float2* __restrict__ buf, int nx, int ny, const double* colmax,
                               const int* colarg, double cutoff, double value, PeakInfo* out) {
  __shared__ PeakInfo pi;
  if (threadIdx.x == 0) {
    double peak = -1.0;
    int px = 0, py = 0;
    for (int y = 0; y < ny; ++y) {
      const double t = colmax[y];
      if (peak < 0 || peak * peak < t) {
        px = colarg[y];
        py = y;
        peak = sqrt(t);
      }
    }
    if (value > 0) peak = value;
    pi.px = px;
    pi.py = py;
    pi.peak = peak;
    pi.blc0 = pi.blc1 = pi.trc0 = pi.trc1 = -1;
  }
  __syncthreads();
  const double c = cutoff * pi.peak;
  const double thr = fabs(c) * fabs(c);
  auto amp = [&](int x, int y) {
    const float2 v = buf[x + (size_t)nx * y];
    return (double)__fadd_rn(__fmul_rn(v.x, v.x), __fmul_rn(v.y, v.y));
  };
  if (threadIdx.x == 0) {
    for (int x = 0; x <= pi.px; ++x) if (amp(x, pi.py) > thr) { pi.blc0 = x; break; }
  } else if (threadIdx.x == 1) {
    for (int y = 0; y <= pi.py; ++y) if (amp(pi.px, y) > thr) { pi.blc1 = y; break; }
  } else if (threadIdx.x == 2) {
    for (int x = nx - 1; x >= pi.px; --x) if (amp(x, pi.py) > thr) { pi.trc0 = x; break; }
  } else if (threadIdx.x == 3) {
    for (int y = ny - 1; y >= pi.py; --y) if (amp(pi.px, y) > thr) { pi.trc1 = y; break; }
  }
  __syncthreads();
  if (threadIdx.x == 0) *out = pi;
}

// WProjectVisGridder::extractSupport -> (size, offU, offV); YG_ERR_SUPPORT on failure
static int extract_support(const PeakInfo& pk, int nx, int ny, int os, bool offsetsupport, int* size, int* offu,
                           int* offv) {
  if (!(pk.peak > 0.0)) return YG_ERR_SUPPORT;
  if (!(pk.px > 0 && pk.py > 0 && pk.px + 1 < nx && pk.py + 1 < ny)) return YG_ERR_SUPPORT;
  if (pk.blc0 < 0 || pk.blc1 < 0 || pk.trc0 < 0 || pk.trc1 < 0) return YG_ERR_SUPPORT;
  int s;
  *offu = *offv = 0;
  if (offsetsupport) {
    s = std::max(pk.trc0 - pk.blc0, pk.trc1 - pk.blc1);
    *offu = (pk.px - nx / 2) / os;
    *offv = (pk.py - ny / 2) / os;
  } else {
    const int cx = nx / 2, cy = ny / 2;
    const int xm = std::max(std::abs(pk.trc0 - cx), std::abs(cx - pk.blc0));
    const int ym = std::max(std::abs(pk.trc1 - cy), std::abs(cy - pk.blc1));
    s = std::max(xm, ym) * 2;
    if (!(s > 0)) return YG_ERR_SUPPORT;
  }
  s /= 2 * os;
  if (s < 3) s = 3;
  *size = s;
  return YG_OK;
}

static int search_plane(const float2* buf, int nx, int ny, double cutoff, double value, DevBuf& tmp,
                        PeakInfo* host, cudaStream_t st) {
  CF_TRY(tmp.ensure((size_t)ny * (sizeof(double) + sizeof(int)) + sizeof(PeakInfo) + 64));
  double* colmax = tmp.as<double>();
  int* colarg = reinterpret_cast<int*>(colmax + ny);
  PeakInfo* pk = reinterpret_cast<PeakInfo*>(tmp.as<char>() + (((size_t)ny * 12 + 15) / 16) * 16);
  k_colmax<<<ny, 256, 0, st>>>(buf, nx, ny, colmax, colarg);
  k_peak_support<<<1, 32, 0, st>>>(buf, nx, ny, colmax, colarg, cutoff, value, pk);
  CF_TRY(cudaGetLastError());
  CF_TRY(cudaMemcpyAsync(host, pk, sizeof(PeakInfo), cudaMemcpyDeviceToHost, st));
  CF_TRY(cudaStreamSynchronize(st));
  return YG_OK;
}

static int check_overflow(int support, int offu, int offv, int os, int nx, int ny) {
  const int kxmin = (-support + offu) * os + nx / 2;
  const int kxmax = (support + offu) * os + os - 1 + nx / 2;
  const int kymin = (-support + offv) * os + ny / 2;
  const int kymax = (support + offv) * os + os - 1 + ny / 2;
  if (kxmin < 0 || kxmax >= nx || kymin < 0 || kymax >= ny) return YG_ERR_SUPPORT;
  return YG_OK;
}

// ---------------------------------------------------------------------------
// WProject
// ---------------------------------------------------------------------------
struct WScreenArgs {
  int nx, ny, qnx, qny;
  double ccellx, ccelly;
  const float* ccfx;
  const float* ccfy;
  const double* wphase;   // per plane in the batch: 2 pi w
  float2* buf;            // batch x nx x ny
};

__global__ void k_wscreen(WScreenArgs a, long long total) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % a.nx);
    const int y = (int)((i / a.nx) % a.ny);
    const int b = (int)(i / ((long long)a.nx * a.ny));
    const int ix = x - a.nx / 2 + a.qnx / 2;
    const int iy = y - a.ny / 2 + a.qny / 2;
    float2 v = make_float2(0.f, 0.f);
    if (ix >= 0 && ix < a.qnx && iy >= 0 && iy < a.qny) {
      double y2 = __dmul_rn((double)(iy - a.qny / 2), a.ccelly);
      y2 = __dmul_rn(y2, y2);
      double x2 = __dmul_rn((double)(ix - a.qnx / 2), a.ccellx);
      x2 = __dmul_rn(x2, x2);
      const double r2 = __dadd_rn(x2, y2);
      if (r2 < 1.0) {
        const double phase = __dmul_rn(a.wphase[b], __dsub_rn(1.0, sqrt(__dsub_rn(1.0, r2))));
        const float wt = __fmul_rn(a.ccfx[ix], a.ccfy[iy]);
        double s, c;
        sincos(phase, &s, &c);
        v.x = (float)__dmul_rn((double)wt, c);
        v.y = (float)(-__dmul_rn((double)wt, s));
      }
    }
    const float sg = cb_in(x, y);
    a.buf[i] = make_float2(v.x * sg, v.y * sg);
  }
}

struct CutArgs {
  const float2* buf;      // batch x nx x ny (checkerboarded FFT output)
  int nx, ny, os;
  int plane0;             // global index (before oversampling) of batch plane 0
  const int* support;     // per batch plane
  const int2* offs;       // per batch plane
  const long long* off;   // cache offsets per cf index
  float2* data;           // cache data
  float rescale;          // multiply after scale (1 = none)
  float prescale;         // multiply first (1 = none)
};

__global__ void k_cut(CutArgs a, int nbatch, int maxsize) {
  // grid: x over taps of the largest CF, y over (fracu, fracv), z over batch planes
  const int b = blockIdx.z;
  const int fu = blockIdx.y % a.os, fv = blockIdx.y / a.os;
  const int s = a.support[b];
  const int cs = 2 * s + 1;
  const int2 o = a.offs[b];
  const long long plane = fu + a.os * (fv + (long long)a.os * (a.plane0 + b));
  float2* dst = a.data + a.off[plane];
  const float2* src = a.buf + (size_t)b * a.nx * a.ny;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < cs * cs; t += gridDim.x * blockDim.x) {
    const int ix = t % cs - s, iy = t / cs - s;
    const int kx = (ix + o.x) * a.os + fu + a.nx / 2;
    const int ky = (iy + o.y) * a.os + fv + a.ny / 2;
    float2 v = src[kx + (size_t)a.nx * ky];
    const float sg = cb_out(kx, ky, a.nx, a.ny);
    v.x *= sg;
    v.y *= sg;
    if (a.prescale != 1.f) { v.x = __fmul_rn(v.x, a.prescale); v.y = __fmul_rn(v.y, a.prescale); }
    if (a.rescale != 1.f) { v.x = __fmul_rn(a.rescale, v.x); v.y = __fmul_rn(a.rescale, v.y); }
    dst[t] = v;
  }
  (void)nbatch;
  (void)maxsize;
}

// one thread per CF: sequential FP32 sum of real parts, scale by (float)(1/sum)
__global__ void k_normalise(float2* data, const long long* off, const int* size, int ncf) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncf) return;
  const int n = size[c] * size[c];
  if (n == 0) return;
  float2* d = data + off[c];
  float s = 0.f;
  for (int i = 0; i < n; ++i) s = __fadd_rn(s, d[i].x);
  if (s > 0.f) {
    const float inv = (float)(1.0 / (double)s);
    for (int i = 0; i < n; ++i) d[i] = make_float2(__fmul_rn(d[i].x, inv), __fmul_rn(d[i].y, inv));
  }
}

static void wproject_taper(int q, float* out, const Spheroidal& g) {
  for (int i = 0; i < q; ++i) {
    const float nu = std::fabs((float)(i - q / 2)) / (float)(q / 2);
    out[i] = (float)(g((double)nu) / (double)(float)q);
  }
  if (q > 3) {
    out[0] = 3.f * (out[1] - out[2]) + out[3];
    if (q % 2 == 1) out[q - 1] = out[0];
  }
}

int cf_build_wproject(CFCacheDev& cache, const WProjCFParams& p, DevBuf& work, cudaStream_t st) {
  const int nx = p.maxsupport, ny = p.maxsupport;
  const int os = p.os;
  if (nx % 2 || nx <= 0 || os <= 0) return YG_ERR_ARG;
  const int qnx = nx / os, qny = ny / os;
  if (qnx < 4) return YG_ERR_ARG;
  const int nw = (int)p.wterms.size();
  const double cellx = 1.0 / ((double)p.shape_x * p.uvcell_u);
  const double celly = 1.0 / ((double)p.shape_y * p.uvcell_v);
  Spheroidal grdsf(M_PI * 3, p.alpha);
  std::vector<float> ccfx(qnx), ccfy(qny);
  wproject_taper(qnx, ccfx.data(), grdsf);
  wproject_taper(qny, ccfy.data(), grdsf);
  // batch of planes transformed together
  const size_t plane_bytes = (size_t)nx * ny * sizeof(float2);
  int batch = (int)std::max<size_t>(1, std::min<size_t>(nw, ((size_t)4 << 30) / plane_bytes));
  DevBuf dtaper, dphase, dsup, doffs, tmp;
  CF_TRY(dtaper.ensure((qnx + qny) * sizeof(float)));
  CF_TRY(cudaMemcpy(dtaper.p, ccfx.data(), qnx * sizeof(float), cudaMemcpyHostToDevice));
  CF_TRY(cudaMemcpy(dtaper.as<float>() + qnx, ccfy.data(), qny * sizeof(float), cudaMemcpyHostToDevice));
  CF_TRY(dphase.ensure(batch * sizeof(double)));
  CF_TRY(dsup.ensure(batch * sizeof(int)));
  CF_TRY(doffs.ensure(batch * sizeof(int2)));
  CF_TRY(work.ensure(plane_bytes * batch));
  cufftHandle plan;
  int dims[2] = {ny, nx};
  FFT_TRY(cufftPlanMany(&plan, 2, dims, nullptr, 1, nx * ny, nullptr, 1, nx * ny, CUFFT_C2C, batch));
  cufftSetStream(plan, st);
  int its_support = 0;
  std::vector<int> sup(nw, 0);
  std::vector<int2> offs(nw, make_int2(0, 0));
  // pass 1: supports (plane 0, or every plane with variable support)
  // pass 2: cut.  Both passes need the transformed planes; batches are
  // recomputed in pass 2 only when they do not all fit at once.
  const bool single_batch = batch >= nw;
  int rc = YG_OK;
  for (int pass = 0; pass < 2 && rc == YG_OK; ++pass) {
    if (pass == 1) {
      std::vector<int> sizes((size_t)nw * os * os);
      for (int iw = 0; iw < nw; ++iw)
        for (int k = 0; k < os * os; ++k) sizes[(size_t)iw * os * os + k] = 2 * sup[iw] + 1;
      rc = cache.layout(sizes, p.offsetsupport ? offs : std::vector<int2>());
      if (rc) break;
    }
    for (int b0 = 0; b0 < nw && rc == YG_OK; b0 += batch) {
      if (pass == 0 && !p.variablesupport && b0 > 0) break;  // common support: plane 0 only
      const int nb = std::min(batch, nw - b0);
      if (!(pass == 1 && single_batch)) {
        std::vector<double> wph(nb);
        for (int b = 0; b < nb; ++b) wph[b] = 2.0 * M_PI * p.wterms[b0 + b];
        CF_TRY(cudaMemcpyAsync(dphase.p, wph.data(), nb * sizeof(double), cudaMemcpyHostToDevice, st));
        WScreenArgs a{nx, ny, qnx, qny, (double)p.shape_x * cellx / (double)qnx,
                      (double)p.shape_y * celly / (double)qny, dtaper.as<float>(), dtaper.as<float>() + qnx,
                      dphase.as<double>(), work.as<float2>()};
        const long long total = (long long)nb * nx * ny;
        k_wscreen<<<(int)std::min<long long>((total + 255) / 256, 148 * 64), 256, 0, st>>>(a, total);
        CF_TRY(cudaGetLastError());
        FFT_TRY(cufftExecC2C(plan, (cufftComplex*)work.p, (cufftComplex*)work.p, CUFFT_FORWARD));
      }
      if (pass == 0) {
        for (int b = 0; b < nb; ++b) {
          const int iw = b0 + b;
          if (p.variablesupport || its_support == 0) {
            PeakInfo pk;
            rc = search_plane(work.as<float2>() + (size_t)b * nx * ny, nx, ny, p.cutoff, p.cutoff_abs ? 1.0 : -1.0, tmp, &pk, st);
            if (rc) break;
            int s, ou, ov;
            rc = extract_support(pk, nx, ny, os, p.offsetsupport, &s, &ou, &ov);
            if (rc) break;
            if (!((s + 1) * os < nx / 2)) { rc = YG_ERR_SUPPORT; break; }
            if (p.limitsupport > 0 && s > p.limitsupport) s = p.limitsupport;
            if (its_support == 0) its_support = s;
            sup[iw] = p.variablesupport ? s : its_support;
            if (p.offsetsupport) offs[iw] = make_int2(ou, ov);
          } else {
            sup[iw] = its_support;
          }
          rc = check_overflow(sup[iw], offs[iw].x, offs[iw].y, os, nx, ny);
          if (rc) break;
        }
        if (!p.variablesupport && b0 == 0 && rc == YG_OK) {
          for (int iw = 0; iw < nw; ++iw) sup[iw] = its_support;
        }
      } else {
        CF_TRY(cudaMemcpyAsync(dsup.p, sup.data() + b0, nb * sizeof(int), cudaMemcpyHostToDevice, st));
        CF_TRY(cudaMemcpyAsync(doffs.p, offs.data() + b0, nb * sizeof(int2), cudaMemcpyHostToDevice, st));
        CutArgs c{work.as<float2>(), nx, ny, os, b0, dsup.as<int>(), doffs.as<int2>(), cache.off.as<long long>(),
                  cache.data.as<float2>(), 1.f, 1.f};
        const int maxcs = 2 * (*std::max_element(sup.begin() + b0, sup.begin() + b0 + nb)) + 1;
        dim3 g((maxcs * maxcs + 255) / 256, os * os, nb);
        k_cut<<<g, 256, 0, st>>>(c, nb, maxcs);
        CF_TRY(cudaGetLastError());
        CF_TRY(cudaStreamSynchronize(st));
      }
    }
  }
  cufftDestroy(plan);
  if (rc) return rc;
  k_normalise<<<(cache.ncf + 127) / 128, 128, 0, st>>>(cache.data.as<float2>(), cache.off.as<long long>(),
                                                      cache.size.as<int>(), cache.ncf);
  CF_TRY(cudaGetLastError());
  cache.support = its_support;
  rc = cache.refresh_pad(st);
  if (rc) return rc;
  CF_TRY(cudaStreamSynchronize(st));
  return YG_OK;
}

// ---------------------------------------------------------------------------
// AWProject with DiskIllumination
// ---------------------------------------------------------------------------
struct DiskArgs {
  int nu, nv;
  double l_scaled, m_scaled, rmin2, rmax2;
  float scale;
  float2* buf;
};

__global__ void k_disk(DiskArgs a) {
  const long long total = (long long)a.nu * a.nv;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int iu = (int)(i % a.nu), iv = (int)(i / a.nu);
    const double ou = (double)iu - (double)a.nu / 2.0;
    const double ov = (double)iv - (double)a.nv / 2.0;
    const double r2 = __dadd_rn(__dmul_rn(ou, ou), __dmul_rn(ov, ov));
    float2 v = make_float2(0.f, 0.f);
    if (r2 >= a.rmin2 && r2 <= a.rmax2) {
      const double ph = __dadd_rn(__dmul_rn(a.l_scaled, ou), __dmul_rn(a.m_scaled, ov));
      double s, c;
      sincos(ph, &s, &c);
      v = make_float2(__fmul_rn((float)c, a.scale), __fmul_rn((float)(-s), a.scale));
    }
    // checkerboard for the centred inverse transform
    const float sg = cb_in(iu, iv);
    a.buf[i] = make_float2(v.x * sg, v.y * sg);
  }
}

struct AWScreenArgs {
  int nx, ny, qnx, qny;
  double ccellx, ccelly;
  const float2* pattern;   // inverse-transformed pattern (checkerboarded)
  float inv_n;             // 1/(nx*ny) normalisation of the backward transform
  const double* wphase;
  float2* buf;
  const double* tx;        // spheroidal taper per qnx / qny column (null: no taper)
  const double* ty;
};

__global__ void k_awscreen(AWScreenArgs a, long long total) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % a.nx);
    const int y = (int)((i / a.nx) % a.ny);
    const int b = (int)(i / ((long long)a.nx * a.ny));
    const double y2 = __dmul_rn(__dmul_rn((double)y - (double)a.ny / 2, a.ccelly), __dmul_rn((double)y - (double)a.ny / 2, a.ccelly));
    const double x2 = __dmul_rn(__dmul_rn((double)x - (double)a.nx / 2, a.ccellx), __dmul_rn((double)x - (double)a.nx / 2, a.ccellx));
    const double r2 = __dadd_rn(x2, y2);
    float2 v = make_float2(0.f, 0.f);
    // the spheroidal taper is defined in the central qnx x qny region only
    const int qix = x + a.qnx / 2 - a.nx / 2, qiy = y + a.qny / 2 - a.ny / 2;
    const bool inq = !a.tx || (qix >= 0 && qix < a.qnx && qiy >= 0 && qiy < a.qny);
    if (r2 < 1.0 && inq) {
      const float taper = a.tx ? (float)__dmul_rn(a.tx[qix], a.ty[qiy]) : 1.f;
      const float so = cb_out(x, y, a.nx, a.ny);
      float2 pt = a.pattern[x + (size_t)a.nx * y];
      pt.x = __fmul_rn(pt.x * so, a.inv_n);
      pt.y = __fmul_rn(pt.y * so, a.inv_n);
      // pattern * conj(pattern), then * taper
      const float wr = __fmul_rn(__fsub_rn(__fmul_rn(pt.x, pt.x), __fmul_rn(pt.y, -pt.y)), taper);
      const float wi = __fmul_rn(__fadd_rn(__fmul_rn(pt.x, -pt.y), __fmul_rn(pt.y, pt.x)), taper);
      const double phase = __dmul_rn(a.wphase[b], __dsub_rn(1.0, sqrt(__dsub_rn(1.0, r2))));
      double s, c;
      sincos(phase, &s, &c);
      const float cr = (float)c, ci = (float)(-s);
      v.x = __fsub_rn(__fmul_rn(wr, cr), __fmul_rn(wi, ci));
      v.y = __fadd_rn(__fmul_rn(wr, ci), __fmul_rn(wi, cr));
    }
    const float sg = cb_in(x, y);
    a.buf[i] = make_float2(v.x * sg, v.y * sg);
  }
}

static double disk_count(int nu, int nv, double rmin2, double rmax2) {
  double sum = 0.0;
  for (int iu = 0; iu < nu; ++iu) {
    const double ou = (double)iu - (double)nu / 2.;
    for (int iv = 0; iv < nv; ++iv) {
      const double ov = (double)iv - (double)nv / 2.;
      const double r2 = ou * ou + ov * ov;
      if (r2 >= rmin2 && r2 <= rmax2) sum += 1.0;
    }
  }
  return sum;
}

int cf_build_aw(CFCacheDev& cache, const AWCFParams& p, const std::vector<AWFeedJob>& jobs, DevBuf& work,
                cudaStream_t st) {
  const int nx = p.maxsupport, ny = p.maxsupport, os = p.os;
  if (nx % 2 || os <= 0) return YG_ERR_ARG;
  const int qnx = nx / os, qny = ny / os;
  const int nw = (int)p.wterms.size();
  const double ccellx = 1.0 / ((double)qnx * p.uvcell_u);
  const double ccelly = 1.0 / ((double)qny * p.uvcell_v);
  const size_t plane_bytes = (size_t)nx * ny * sizeof(float2);
  CF_TRY(work.ensure(plane_bytes * (nw + 1)));
  float2* pat = work.as<float2>() + (size_t)nw * nx * ny;
  DevBuf dphase, dsup, doffs, tmp, dtaper;
  if (p.spheroidaltaper) {
    // AWProjectVisGridder.cc:338-354: grdsf(|q - qn/2| / (qn/2)) per column,
    // the edge value interpolated from its neighbours
    Spheroidal grdsf(M_PI * 3, p.alpha);
    std::vector<double> t(qnx + qny);
    for (int k = 0; k < 2; ++k) {
      const int q = k ? qny : qnx;
      double* f = t.data() + (k ? qnx : 0);
      for (int i = 0; i < q; ++i) f[i] = grdsf(std::fabs((double)i - (double)(q / 2)) / (double)(q / 2));
      if (q > 3) {
        f[0] = 3.0 * (f[1] - f[2]) + f[3];
        if (q % 2 == 1) f[q - 1] = f[0];
      }
    }
    CF_TRY(dtaper.ensure(t.size() * sizeof(double)));
    CF_TRY(cudaMemcpy(dtaper.p, t.data(), t.size() * sizeof(double), cudaMemcpyHostToDevice));
  }
  CF_TRY(dphase.ensure(nw * sizeof(double)));
  CF_TRY(dsup.ensure(nw * sizeof(int)));
  CF_TRY(doffs.ensure(nw * sizeof(int2)));
  std::vector<double> wph(nw);
  for (int i = 0; i < nw; ++i) wph[i] = 2.0 * M_PI * p.wterms[i];
  CF_TRY(cudaMemcpy(dphase.p, wph.data(), nw * sizeof(double), cudaMemcpyHostToDevice));
  cufftHandle plan1, planw;
  int dims[2] = {ny, nx};
  FFT_TRY(cufftPlanMany(&plan1, 2, dims, nullptr, 1, nx * ny, nullptr, 1, nx * ny, CUFFT_C2C, 1));
  FFT_TRY(cufftPlanMany(&planw, 2, dims, nullptr, 1, nx * ny, nullptr, 1, nx * ny, CUFFT_C2C, nw));
  cufftSetStream(plan1, st);
  cufftSetStream(planw, st);
  int rc = YG_OK;
  const int ncfplanes = nw * p.maxfeeds * p.maxfields * p.nchan_cf;
  for (const AWFeedJob& j : jobs) {
    for (int chan = 0; chan < p.nchan_cf && rc == YG_OK; ++chan) {
      const double freq = p.freqs[chan];
      const double cell_u = p.uvcell_u / os, cell_v = p.uvcell_v / os;
      if (!(std::fabs(std::fabs(cell_u / cell_v) - 1.) < 1e-7)) { rc = YG_ERR_UNSUPPORTED; break; }
      const double cell = std::fabs(cell_u * (kC / freq));
      const double radius = p.diameter / (2.0 * cell);
      const double rmax2 = radius * radius;
      double rmin2 = (p.blockage / (2.0 * cell)) * (p.blockage / (2.0 * cell));
      if (!(rmax2 > rmin2)) { rc = YG_ERR_ARG; break; }
      if (!((double)nx * nx > rmax2 && (double)ny * ny > rmax2)) { rc = YG_ERR_ARG; break; }
      if (rmin2 + 1 >= rmax2) rmin2 -= 1;
      const double cnt = disk_count(nx, ny, rmin2, rmax2);
      if (!(cnt > 0)) { rc = YG_ERR_ARG; break; }
      const float scale = (float)nx * (float)ny / (float)cnt;
      DiskArgs d{nx, ny, 2. * M_PI * cell_u * j.l, 2. * M_PI * cell_v * j.m, rmin2, rmax2, scale, pat};
      k_disk<<<(nx * ny + 255) / 256, 256, 0, st>>>(d);
      FFT_TRY(cufftExecC2C(plan1, (cufftComplex*)pat, (cufftComplex*)pat, CUFFT_INVERSE));
      // pattern now checkerboard-signed centred inverse transform x N
      AWScreenArgs a{nx, ny, qnx, qny, ccellx, ccelly, pat, 1.f / ((float)nx * (float)ny), dphase.as<double>(),
                     work.as<float2>(), p.spheroidaltaper ? dtaper.as<double>() : nullptr,
                     p.spheroidaltaper ? dtaper.as<double>() + qnx : nullptr};
      const long long total = (long long)nw * nx * ny;
      k_awscreen<<<(int)std::min<long long>((total + 255) / 256, 148 * 64), 256, 0, st>>>(a, total);
      FFT_TRY(cufftExecC2C(planw, (cufftComplex*)work.p, (cufftComplex*)work.p, CUFFT_FORWARD));
      CF_TRY(cudaGetLastError());
      const float inv = (float)(1.0 / ((double)nx * (double)ny));
      std::vector<int> sup(nw, cache.support);
      std::vector<int2> offs(nw, make_int2(0, 0));
      for (int iw = 0; iw < nw; ++iw) {
        if (p.variablesupport || cache.support == 0) {
          PeakInfo pk;
          // the support search runs on the scaled plane; scaling by the exact
          // power of two 1/(nx ny) commutes with the search
          // the plane is searched before the 1/(nx ny) scaling; an absolute
          // cutoff is scaled to match
          rc = search_plane(work.as<float2>() + (size_t)iw * nx * ny, nx, ny, p.cutoff,
                            p.cutoff_abs ? (double)nx * (double)ny : -1.0, tmp, &pk, st);
          if (rc) break;
          int s, ou, ov;
          rc = extract_support(pk, nx, ny, os, p.offsetsupport, &s, &ou, &ov);
          if (rc) break;
          if (!((s + 1) * os < nx / 2)) { rc = YG_ERR_SUPPORT; break; }
          if (p.limitsupport > 0 && s > p.limitsupport) s = p.limitsupport;
          if (cache.support == 0) {
            cache.support = s;
            if (!p.variablesupport) {
              std::vector<int> sizes((size_t)ncfplanes * os * os, 2 * s + 1);
              rc = cache.layout(sizes, p.offsetsupport ? std::vector<int2>(ncfplanes, make_int2(0, 0))
                                                        : std::vector<int2>());
              if (rc) break;
            }
          }
          if (p.variablesupport) sup[iw] = s;
          if (p.offsetsupport) offs[iw] = make_int2(ou, ov);
        }
        // fixed support: every plane takes the support found on the first one
        if (!p.variablesupport) sup[iw] = cache.support;
        rc = check_overflow(sup[iw], offs[iw].x, offs[iw].y, os, nx, ny);
        if (rc) break;
      }
      if (rc) break;
      if (p.variablesupport) { rc = YG_ERR_UNSUPPORTED; break; }
      const int z0 = nw * (chan + p.nchan_cf * (j.feed + p.maxfeeds * j.field));
      if (p.offsetsupport) {
        for (int iw = 0; iw < nw; ++iw) cache.h_offsets[z0 + iw] = offs[iw];
        CF_TRY(cudaMemcpyAsync(cache.offsets.as<int2>() + z0, offs.data(), nw * sizeof(int2), cudaMemcpyHostToDevice, st));
      }
      CF_TRY(cudaMemcpyAsync(dsup.p, sup.data(), nw * sizeof(int), cudaMemcpyHostToDevice, st));
      CF_TRY(cudaMemcpyAsync(doffs.p, offs.data(), nw * sizeof(int2), cudaMemcpyHostToDevice, st));
      CutArgs c{work.as<float2>(), nx, ny, os, z0, dsup.as<int>(), doffs.as<int2>(), cache.off.as<long long>(),
                cache.data.as<float2>(), (float)(os * os), inv};
      const int cs = 2 * cache.support + 1;
      dim3 g((cs * cs + 255) / 256, os * os, nw);
      k_cut<<<g, 256, 0, st>>>(c, nw, cs);
      CF_TRY(cudaGetLastError());
      CF_TRY(cudaStreamSynchronize(st));
    }
    if (rc) break;
  }
  cufftDestroy(plan1);
  cufftDestroy(planw);
  if (rc == YG_OK) {
    rc = cache.refresh_pad(st);
    if (rc == YG_OK && cudaStreamSynchronize(st) != cudaSuccess) rc = YG_ERR_CUDA;
  }
  return rc;
}

}  // namespace yg

// Degridding that allocates no device memory.
//
// Some callers of this library cannot call cudaMalloc: an application that
// hands each GPU a fixed memory budget when it starts and forbids any later
// allocation, so that a long-running imaging service never fails half way
// through a major cycle for lack of memory, or a host framework whose own
// pool allocator owns the device's memory and gives no other code a share of
// it.  yg_degrid_noalloc serves them: it degrids a device-resident chunk with
// the convolution functions and the model grid that the gridder already
// holds, and keeps every per-call temporary in the statically allocated array
// below.
//
// The array is a file-scope __device__ array, so every GPU that loads this
// library holds its kNATotal bytes until the process exits.  In host code its
// name is only a host-side stand-in, never a device address; the address is
// obtained once per device with cudaGetSymbolAddress (with that device
// current) the first time a call runs on it.  Every call shares the one array
// and the array keeps the previous call's contents, so everything a call needs
// zeroed is written before use; calls that overlap on the GPU (two streams, or
// two host threads) race on it and must be serialised by the caller.  A call
// reads the chunk's frequencies back to the host and waits for the gridder's
// stream before it returns, as yg_degrid does.
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "yg_gridder.h"

namespace yg {

namespace {

void na_require(bool ok, int code, const std::string& msg) {
  if (!ok) throw YgError{code, msg};
}

void na_cuda(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw YgError{YG_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e)};
}

constexpr long long kNAMaxSamples = 1ll << 20;   // rows x channels per call
constexpr int kNAMaxPol = 4;
constexpr int kNAMaxChan = 1 << 16;
constexpr int kNAMaxDevices = 64;

constexpr size_t align256(size_t x) { return (x + 255) / 256 * 256; }
constexpr size_t kNAMetaOff = 0;
constexpr size_t kNAValsOff = align256(kNAMetaOff + kNAMaxSamples * sizeof(int4));
constexpr size_t kNAMarkOff = align256(kNAValsOff + kNAMaxSamples * kNAMaxPol * sizeof(float2));
constexpr size_t kNARowOff = align256(kNAMarkOff + kNAMaxSamples * sizeof(int));
constexpr size_t kNAChanOff = align256(kNARowOff + kNAMaxSamples);
constexpr size_t kNAMfsOff = align256(kNAChanOff + kNAMaxChan * sizeof(int));
constexpr int kNAScanBlock = 1024;                // elements per block of the max-scan
constexpr int kNAScanBlocks = (int)(kNAMaxSamples / kNAScanBlock);
constexpr size_t kNAAggrOff = align256(kNAMfsOff + kNAMaxChan * sizeof(float));
constexpr size_t kNATotal = align256(kNAAggrOff + kNAScanBlocks * sizeof(int));

__device__ __align__(256) unsigned char g_noalloc_scratch[kNATotal];

std::mutex g_na_mutex;
void* g_na_addr[kNAMaxDevices] = {};

// device address of the static array on the current device (set-up on first use)
unsigned char* scratch_address(int dev) {
  if (dev < 0 || dev >= kNAMaxDevices) throw YgError{YG_ERR_ARG, "device ordinal out of range"};
  std::lock_guard<std::mutex> lock(g_na_mutex);
  if (!g_na_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      throw YgError{YG_ERR_CUDA, std::string("cudaGetSymbolAddress of the no-alloc scratch failed: ") +
                                     cudaGetErrorString(e)};
    g_na_addr[dev] = p;
  }
  return static_cast<unsigned char*>(g_na_addr[dev]);
}

// Classification of every (row, chan) sample, as in the plan binning: status
// 0 unused, 1 w out of range (clipped), 2 off the grid, 3 degridded; the
// on-grid cell (CF offset applied), CF index and grid plane.
__global__ void k_na_index(BinArgs a, int4* __restrict__ meta, DevError* err) {
  const long long n = a.nrow * (long long)a.nchan;
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n; s += (long long)gridDim.x * blockDim.x) {
    const long long row = s % a.nrow;
    const int chan = (int)(s / a.nrow);
    int4 m = make_int4(0, 0, 0, 0);
    if (!a.row_ok || a.row_ok[row]) {
      const double f = a.freq[chan];
      int iu, iv, fu, fv;
      if (!axis_index(f, a.uvw[3 * row + 0], a.cellu, a.os, a.nx, &iu, &fu) ||
          !axis_index(f, a.uvw[3 * row + 1], a.cellv, a.os, a.ny, &iv, &fv)) {
        raise_error(err, YG_ERR_FRAC, s);
      } else {
        int e = 0, plane = 0, gind = 0;
        if (a.cf_mode != CF_MODE_SINGLE || a.grid_mode != GRID_MODE_SINGLE) {
          const double wf = __dmul_rn(__ddiv_rn(a.uvw[3 * row + 2], kC), f);
          if (a.cf_mode == CF_MODE_WSTACK_WPROJ) {
            gind = get_wplane(a.ws_stack, wf, &e);
            if (gind >= 0) {
              const int half = (a.ws_stack.nwplanes - 1) / 2;
              plane = get_wplane(a.ws, __dsub_rn(wf, __dmul_rn((double)(gind - half), a.ws_stack.wscale)), &e);
            } else {
              plane = -1;
            }
          } else {
            plane = get_wplane(a.ws, wf, &e);
            gind = (a.grid_mode == GRID_MODE_WPLANE) ? plane : 0;
          }
          if (e) raise_error(err, e, s);
        }
        int cplane = 0;
        if (a.cf_mode == CF_MODE_WPLANE || a.cf_mode == CF_MODE_WSTACK_WPROJ) {
          cplane = plane;
        } else if (a.cf_mode == CF_MODE_AW) {
          const int fd = a.feed ? a.feed[row] : 0;
          cplane = plane;
          if (plane >= 0) {
            const int c = a.aw_nchan > 1 ? chan : 0;
            cplane = plane + a.ws.nwplanes * (c + a.aw_nchan * (fd + a.aw_maxfeeds * a.aw_field));
          }
        }
        bool good = true;
        if (a.flag)
          for (int p = 0; p < a.npol; ++p)
            if (a.flag[s + n * p]) { good = false; break; }
        if (good && a.chan_map[chan] >= 0) {
          if (gind < 0 || cplane < 0) {
            m.w = 1;
          } else {
            const int cfi = fu + a.os * (fv + a.os * cplane);
            if (cfi < 0 || cfi >= a.cf.ncf || a.cf.size[cfi] <= 0) {
              raise_error(err, YG_ERR_CINDEX, s);
            } else {
              const int sup = (a.cf.size[cfi] - 1) / 2;
              int ou = 0, ov = 0;
              if (a.cf.offsets && cplane < a.cf.noffsets) {
                ou = a.cf.offsets[cplane].x;
                ov = a.cf.offsets[cplane].y;
              }
              const int iuo = iu + ou, ivo = iv + ov;
              if ((iuo - sup) > 0 && (ivo - sup) > 0 && (iuo + sup) < a.nx && (ivo + sup) < a.ny) {
                m = make_int4(iuo, ivo, cfi, 3 | (gind << 4));
              } else {
                m.w = 2;
              }
            }
          }
        }
      }
    }
    meta[s] = m;
  }
}

// One warp per degridded sample: sum CF * conj(grid) over the taps read from
// the grid in HBM, then * MFS weight * phasor (GridKernel.cc:99-137,
// TableVisGridder.cc:765-773).
template <int NPOL>
__global__ void k_na_degrid(const int4* __restrict__ meta, VisArgs v, CFView cf, const float2* __restrict__ grid,
                            int nx, int ny, int nchan_img, const int* __restrict__ chan_map,
                            float2* __restrict__ vals) {
  const long long n = v.nrow * (long long)v.nchan;
  const long long plane_cells = (long long)nx * ny;
  const int lane = threadIdx.x & 31;
  const long long warp0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long s = warp0; s < n; s += nwarps) {
    const int4 m = meta[s];
    if ((m.w & 15) != 3) continue;
    const int gind = m.w >> 4;
    const long long row = s % v.nrow;
    const int chan = (int)(s / v.nrow);
    const int ichan = chan_map[chan];
    const int c = m.z;
    const int w = cf.size[c];
    const int sup = (w - 1) / 2;
    const float2* base = grid + (size_t)gind * plane_cells * NPOL * nchan_img + plane_cells * ((size_t)NPOL * ichan) +
                         (m.x - sup) + (size_t)nx * (m.y - sup);
    const float2* cfp = cf.data + cf.off[c];
    float re[NPOL], im[NPOL];
#pragma unroll
    for (int p = 0; p < NPOL; ++p) re[p] = im[p] = 0.f;
    for (int t = lane; t < w * w; t += 32) {
      const int jx = t % w, jy = t / w;
      const float2 cv = cfp[t];
#pragma unroll
      for (int p = 0; p < NPOL; ++p) {
        const float2 g = base[plane_cells * p + jx + (size_t)nx * jy];
        re[p] = fmaf(cv.x, g.x, fmaf(cv.y, g.y, re[p]));
        im[p] = fmaf(cv.y, g.x, fmaf(-cv.x, g.y, im[p]));
      }
    }
#pragma unroll
    for (int p = 0; p < NPOL; ++p)
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        re[p] += __shfl_xor_sync(0xffffffffu, re[p], o);
        im[p] += __shfl_xor_sync(0xffffffffu, im[p], o);
      }
    if (lane == 0) {
      float pr = 1.f, pi = 0.f;
      if (v.delay) {
        const double ph = __ddiv_rn(__dmul_rn(__dmul_rn(__dmul_rn(2.0, kPi), v.freq[chan]), v.delay[row]), kC);
        pr = (float)cos(ph);
        pi = (float)sin(ph);
      }
#pragma unroll
      for (int p = 0; p < NPOL; ++p) {
        float cr = re[p], ci = im[p];
        if (v.mfs) {
          cr = __fmul_rn(cr, v.mfs[chan]);
          ci = __fmul_rn(ci, v.mfs[chan]);
        }
        vals[(size_t)s * NPOL + p] =
            make_float2(__fsub_rn(__fmul_rn(cr, pr), __fmul_rn(ci, pi)), __fadd_rn(__fmul_rn(cr, pi), __fmul_rn(ci, pr)));
      }
    }
  }
}

// marks[o] = o when the sample at loop position o = row * nchan + chan was
// degridded, else -1; an inclusive max-scan over the marks then gives, for
// every o, the last degridded position at or before o.
__global__ void k_na_marks(const int4* __restrict__ meta, long long nrow, int nchan, int* __restrict__ marks) {
  const long long n = nrow * (long long)nchan;
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < n; o += (long long)gridDim.x * blockDim.x) {
    const long long s = o / nchan + nrow * (o % nchan);
    marks[o] = ((meta[s].w & 15) == 3) ? (int)o : -1;
  }
}

// inclusive max over the threads of a 1024-thread block (warp shuffles, then
// the 32 warp totals by the first warp)
__device__ __forceinline__ int block_incl_max(int v, int* wsum) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v = max(v, t);
  }
  if (lane == 31) wsum[warp] = v;
  __syncthreads();
  if (warp == 0) {
    int x = wsum[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x = max(x, t);
    }
    wsum[lane] = x;
  }
  __syncthreads();
  return warp > 0 ? max(v, wsum[warp - 1]) : v;
}

// Max-scan in three passes over blocks of kNAScanBlock marks: each block's
// inclusive scan in place with its total in aggr[b]; one block scans the
// totals; each element then takes the max with the totals of the blocks before
// its own.
__global__ void __launch_bounds__(kNAScanBlock) k_na_scan_blocks(int* __restrict__ x, long long n,
                                                                  int* __restrict__ aggr) {
  __shared__ int wsum[32];
  const long long i = (long long)blockIdx.x * kNAScanBlock + threadIdx.x;
  const int v = block_incl_max(i < n ? x[i] : -1, wsum);
  if (i < n) x[i] = v;
  if (threadIdx.x == kNAScanBlock - 1) aggr[blockIdx.x] = v;
}

__global__ void __launch_bounds__(kNAScanBlock) k_na_scan_aggr(int* __restrict__ aggr, int nblocks) {
  __shared__ int wsum[32];
  const int v = block_incl_max(threadIdx.x < nblocks ? aggr[threadIdx.x] : -1, wsum);
  if (threadIdx.x < nblocks) aggr[threadIdx.x] = v;
}

__global__ void k_na_scan_add(int* __restrict__ x, long long n, const int* __restrict__ aggr) {
  for (long long i = (long long)(blockIdx.x + 1) * kNAScanBlock + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int b = (int)(i / kNAScanBlock);
    x[i] = max(x[i], aggr[b - 1]);
  }
}

// vis += value; valid off-grid samples take the last degridded value in loop
// order, or the value carried from the previous call (TableVisGridder.cc:857-865)
__global__ void k_na_writeback(const int4* __restrict__ meta, const int* __restrict__ prev,
                               const float2* __restrict__ vals, const float2* __restrict__ carry, long long nrow,
                               int nchan, int npol, float2* __restrict__ vis) {
  const long long n = nrow * (long long)nchan;
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < n; o += (long long)gridDim.x * blockDim.x) {
    const long long s = o / nchan + nrow * (o % nchan);
    if ((meta[s].w & 15) < 2) continue;
    const int q = prev[o];
    const long long sq = q >= 0 ? (q / nchan) + nrow * (q % nchan) : 0;
    for (int p = 0; p < npol; ++p) {
      const float2 val = q >= 0 ? vals[(size_t)sq * npol + p] : carry[p];
      float2 o2 = vis[s + n * p];
      o2.x += val.x;
      o2.y += val.y;
      vis[s + n * p] = o2;
    }
  }
}

__global__ void k_na_carry(const int* __restrict__ prev, long long nrow, int nchan, int npol,
                           const float2* __restrict__ vals, float2* __restrict__ carry) {
  const long long n = nrow * (long long)nchan;
  if (n == 0) return;
  const int q = prev[n - 1];
  if (q < 0) return;
  const long long sq = (q / nchan) + nrow * (q % nchan);
  for (int p = threadIdx.x; p < npol; p += blockDim.x) carry[p] = vals[(size_t)sq * npol + p];
}

int na_blocks(long long n) {
  long long b = (n + 255) / 256;
  return (int)(b < 1 ? 1 : (b > 148 * 16 ? 148 * 16 : b));
}

}  // namespace

size_t noalloc_scratch_bytes() { return kNATotal; }
long long noalloc_max_samples() { return kNAMaxSamples; }

void Gridder::degrid_noalloc(Chunk& c) {
  na_require(!psf_, YG_ERR_STATE, "the gridder is not supposed to be used for degridding in the PSF mode");
  // AWProject builds its CFs per chunk (field, beams, channels), which needs
  // device memory; the learned CF forms run through the plan kernels
  na_require(kind_ != Kind::AWProject, YG_ERR_UNSUPPORTED,
             "yg_degrid_noalloc does not take AWProject gridders (their CFs are built per chunk); use yg_degrid");
  na_require(cf_form_ == 0, YG_ERR_UNSUPPORTED,
             "yg_degrid_noalloc uses the tabulated CFs only; set the CF form back to 0 or use yg_degrid");
  na_require(c.on_device, YG_ERR_ARG, "yg_degrid_noalloc needs a device-resident chunk (on_device = 1)");
  na_require(nx_ > 0 && grids_.p && device_ready_, YG_ERR_STATE,
             "initialiseDegrid must be called before yg_degrid_noalloc");
  if (model_empty_) return;
  na_require(cf_built_, YG_ERR_STATE,
             "convolution functions are not built: call yg_build_cf (or one yg_degrid) before yg_degrid_noalloc");
  const long long n = c.nrow * (long long)c.nchan;
  na_require(n <= kNAMaxSamples, YG_ERR_ARG,
             "yg_degrid_noalloc takes at most " + std::to_string(kNAMaxSamples) + " rows x channels per call, got " +
                 std::to_string(n));
  na_require(c.nchan <= kNAMaxChan, YG_ERR_ARG, "yg_degrid_noalloc takes at most 65536 channels");
  na_require(c.npol == npol_, YG_ERR_UNSUPPORTED, "visibility and image polarisation frames must match");
  na_require(c.npol == 1 || c.npol == 2 || c.npol == 4, YG_ERR_UNSUPPORTED, "1, 2 or 4 polarisations");
  if (n == 0) return;
  int dev = -1;
  na_cuda(cudaGetDevice(&dev), "cudaGetDevice");
  na_require(dev == device_, YG_ERR_STATE, "the gridder's device must be current");
  unsigned char* base = scratch_address(dev);
  int4* meta = reinterpret_cast<int4*>(base + kNAMetaOff);
  float2* vals = reinterpret_cast<float2*>(base + kNAValsOff);
  int* marks = reinterpret_cast<int*>(base + kNAMarkOff);
  uint8_t* rowok = base + kNARowOff;
  int* chanmap = reinterpret_cast<int*>(base + kNAChanOff);
  float* mfsw = reinterpret_cast<float*>(base + kNAMfsOff);

  std::vector<double> freqs(c.nchan);
  na_cuda(cudaMemcpyAsync(freqs.data(), c.freq, c.nchan * sizeof(double), cudaMemcpyDeviceToHost, stream_),
             "frequencies");
  na_cuda(cudaStreamSynchronize(stream_), "frequencies");
  na_require(freqs[0] / kC > 0.1 && freqs[0] / kC < 30000, YG_ERR_FREQ,
             "Check frequencies in the input file as the order of magnitude is likely to be wrong");
  const std::vector<int> cmap = chan_map(freqs.data(), c.nchan);
  na_cuda(cudaMemcpyAsync(chanmap, cmap.data(), c.nchan * sizeof(int), cudaMemcpyHostToDevice, stream_), "chan map");
  const float* mfs = nullptr;
  std::vector<float> w;
  if (mfs_) {
    w.resize(c.nchan);
    for (int i = 0; i < c.nchan; ++i) {
      const double ratio = (freqs[i] - mfs_reffreq_) / mfs_reffreq_;
      w[i] = mfs_order_ == 0 ? 1.0f
                             : (mfs_order_ == 1 ? (float)ratio
                                                : (mfs_order_ == 2 ? (float)(ratio * ratio) : (float)std::pow(ratio, mfs_order_)));
    }
    na_cuda(cudaMemcpyAsync(mfsw, w.data(), c.nchan * sizeof(float), cudaMemcpyHostToDevice, stream_), "mfs");
    mfs = mfsw;
  }
  std::vector<uint8_t> rows = psf_rows(c);
  const uint8_t* row_ok = nullptr;
  if (!rows.empty()) {
    na_cuda(cudaMemcpyAsync(rowok, rows.data(), rows.size(), cudaMemcpyHostToDevice, stream_), "row mask");
    row_ok = rowok;
  }
  BinArgs a;
  fill_bin_args(a, c, chanmap, row_ok);
  k_na_index<<<na_blocks(n), 256, 0, stream_>>>(a, meta, err_.as<DevError>());
  VisArgs v;
  v.vis = c.vis;
  v.noise = c.noise;
  v.delay = c.delay;
  v.mfs = mfs;
  v.freq = c.freq;
  v.nrow = c.nrow;
  v.nchan = c.nchan;
  v.npol = c.npol;
  v.psf = 0;
  v.psf_ok = nullptr;
  const CFView cf = cf_.view();
  const int blocks = (int)std::min<long long>((n * 32 + 255) / 256, 148 * 32);
  switch (c.npol) {
    case 1: k_na_degrid<1><<<blocks, 256, 0, stream_>>>(meta, v, cf, grids_.as<float2>(), nx_, ny_, nchan_, chanmap, vals); break;
    case 2: k_na_degrid<2><<<blocks, 256, 0, stream_>>>(meta, v, cf, grids_.as<float2>(), nx_, ny_, nchan_, chanmap, vals); break;
    default: k_na_degrid<4><<<blocks, 256, 0, stream_>>>(meta, v, cf, grids_.as<float2>(), nx_, ny_, nchan_, chanmap, vals); break;
  }
  k_na_marks<<<na_blocks(n), 256, 0, stream_>>>(meta, c.nrow, c.nchan, marks);
  const int nsb = (int)((n + kNAScanBlock - 1) / kNAScanBlock);
  int* aggr = reinterpret_cast<int*>(base + kNAAggrOff);
  k_na_scan_blocks<<<nsb, kNAScanBlock, 0, stream_>>>(marks, n, aggr);
  k_na_scan_aggr<<<1, kNAScanBlock, 0, stream_>>>(aggr, nsb);
  if (nsb > 1) k_na_scan_add<<<nsb - 1, kNAScanBlock, 0, stream_>>>(marks, n, aggr);
  k_na_writeback<<<na_blocks(n), 256, 0, stream_>>>(meta, marks, vals, carry_.as<float2>(), c.nrow, c.nchan, c.npol, c.vis);
  k_na_carry<<<1, 32, 0, stream_>>>(marks, c.nrow, c.nchan, c.npol, vals, carry_.as<float2>());
  na_cuda(cudaGetLastError(), "yg_degrid_noalloc launch");
  check_error();
}

}  // namespace yg

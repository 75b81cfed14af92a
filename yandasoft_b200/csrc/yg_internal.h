// Internal (non-ABI) structures of the B200 gridder shared by the host
// classes and the CUDA kernels.
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "yg_common.cuh"

namespace yg {

// ---------------------------------------------------------------------------
// device memory helpers
// ---------------------------------------------------------------------------
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  // grows (never shrinks) the buffer; contents are not preserved
  cudaError_t ensure(size_t n) {
    if (n <= bytes && p) return cudaSuccess;
    release();
    if (n == 0) n = 16;
    cudaError_t e = cudaMalloc(&p, n);
    if (e != cudaSuccess) { p = nullptr; return e; }
    bytes = n;
    return cudaSuccess;
  }
  // as ensure, but a buffer that has to grow gets an eighth more than asked:
  // sizes that vary a little from call to call (valid samples, work items of
  // the row pieces of one chunk) then stop reallocating, and so stop the
  // device-wide synchronisation of cudaFree between pieces
  cudaError_t ensure_headroom(size_t n) {
    if (n <= bytes && p) return cudaSuccess;
    return ensure(n + n / 8);
  }
  template <typename T> T* as() const { return static_cast<T*>(p); }
};

// Small page-locked host buffer mapped into the device's address space: a
// kernel writes it and the host reads it after synchronising the stream, so a
// read-back of a few values never waits in a copy engine's queue behind a
// large transfer of another stream.
struct HostMapped {
  void* p = nullptr;
  size_t bytes = 0;
  HostMapped() = default;
  HostMapped(const HostMapped&) = delete;
  HostMapped& operator=(const HostMapped&) = delete;
  ~HostMapped() {
    if (p) cudaFreeHost(p);
  }
  cudaError_t ensure(size_t n) {
    if (n <= bytes && p) return cudaSuccess;
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
    cudaError_t e = cudaHostAlloc(&p, n, cudaHostAllocMapped | cudaHostAllocPortable);
    if (e != cudaSuccess) { p = nullptr; return e; }
    bytes = n;
    return cudaSuccess;
  }
  template <typename T> T* as() const { return static_cast<T*>(p); }
};

// Convolution-function cache in HBM: every CF matrix (odd size, u fastest)
// packed back to back.
struct CFView {
  const float2* data = nullptr;
  const long long* off = nullptr;  // per cf index, in complex elements
  const int* size = nullptr;       // per cf index: 2S+1 (0 = unused)
  const int2* offsets = nullptr;   // per plane before oversampling (offU, offV)
  int ncf = 0;
  int noffsets = 0;
  int maxsize = 0;                 // max 2S+1 over the cache
  int varsup = 0;                  // 1 when CF sizes differ (variable support)
  const float2* pad = nullptr;      // every CF zero-padded to wpad x wpad (row stride wpad)
  int wpad = 0;                    // round_up(maxsize, 16)
};

// How a (row, chan, feed) sample maps to a CF plane and a grid.
enum { CF_MODE_SINGLE = 0, CF_MODE_WPLANE = 1, CF_MODE_AW = 2, CF_MODE_WSTACK_WPROJ = 3 };
enum { GRID_MODE_SINGLE = 0, GRID_MODE_WPLANE = 1, GRID_MODE_STACK = 2 };

struct BinArgs {
  long long nrow;
  int nchan;
  int npol;
  const double* uvw;       // nrow x 3 (row-major)
  const double* freq;      // nchan
  const int* chan_map;     // nchan: image channel or -1
  const uint8_t* flag;     // (nrow, nchan, npol) column-major, may be null
  const int* feed;         // nrow, may be null
  const uint8_t* row_ok;   // nrow, may be null
  double cellu, cellv;
  int os;
  int nx, ny;
  WSampling ws;            // w -> CF plane (W gridders)
  WSampling ws_stack;      // w -> grid plane (stacked gridders)
  int cf_mode;
  int grid_mode;
  int aw_nchan;            // channels of the AW cache (1 if not frequency dependent)
  int aw_maxfeeds;
  int aw_field;
  int nchan_img;
  int tile;                // tile side T
  int ntx, nty;            // tiles per axis
  int mbits;               // bits of the within-tile Morton code
  int wy;                  // row modulus of the residues in the records (0: the padded CF width)
  int pos_major;           // also build second-order records (rec_pos): 1 position-major, 2 plane-major
  int key_planes;          // a plan for gridding only: sort once, by the plane-major key (pos_major 2)
  int need_inv;            // build the inverse permutation (the cube-order gather of the CF-major kernels)
  unsigned long long invalid_key;  // one past the largest valid key
  CFView cf;
};

// Sorted, binned sample list of one chunk, reusable for every grid and degrid
// pass over the same uvw/frequency/flag data (the major cycle).
struct Plan {
  long long nsamples = 0;       // nrow * nchan
  long long nvalid = 0;         // on-grid samples
  int nitems = 0;               // work items
  int tile = 0, ntx = 0, nty = 0, ngc = 0;
  int smax = 0;                 // max support in the plan
  int pad = 0;                  // P = T + 2 smax
  int vmax = 0;                 // samples per work item
  long long ntiles_total = 0;
  long long nrow = 0;
  int nchan = 0, npol = 0;
  DevBuf key, key_alt, val, val_alt, pos, cfi, status;
  DevBuf tstart, tend, nit, itembase, items, nvalid_d, sort_tmp;
  HostMapped info_h;            // read-back of the item count and on-grid samples
  DevBuf order_prev;            // degrid stale-value scan: marks, then loop-order predecessors
  bool prev_ready = false;      // order_prev holds this plan's predecessors
  DevBuf last;                  // grid carry: loop-order index of the last used sample
  DevBuf chanmap;               // accessor channel -> image channel of the binned chunk
  DevBuf rec;                   // per sorted sample: cell, residues|w, CF index, sample id (int4)
  DevBuf rec_pos;               // the same records ordered by tile, then position in the tile, then CF
  DevBuf pos_val2;              // alternate values of the rec_pos sort
  DevBuf inv, inv_pos;          // per sample id: its index in rec (rec_pos), -1 off the grid
  bool pos_ready = false;       // rec_pos is built
  bool grid_only = false;       // sorted once, plane-major: rec_pos only (no CF-major records)
  bool inv_ready = false, inv_pos_ready = false;   // inv / inv_pos are built
  int pos_mode = 0;             // its order: 1 position then CF index; 2 CF plane, position, offset
  int os2 = 1;                  // oversampling offsets per CF plane
  DevBuf ext;                   // continuous learned CF: per sorted sample (ru, rv, w, 0)
  bool ext_ready = false;
  int mbits = 0, ncf = 0;       // sort-key layout
  int wy = 0;                   // row modulus of the records' residues
  double taps = 0;              // sum of (2S+1)^2 over valid samples (per pol)
};

// Grid-side inputs of one grid/degrid call.
struct VisArgs {
  const float2* vis;        // (nrow, nchan, npol) column-major
  const float2* noise;      // same, may be null (unit noise)
  const double* delay;      // nrow, may be null
  const float* mfs;         // nchan, may be null
  const double* freq;       // nchan
  long long nrow;
  int nchan;
  int npol;
  int psf;                  // grid the weight instead of the visibility
  const uint8_t* psf_ok;    // nrow representative feed/field mask (PSF), may be null
  int pcf = 0;              // preconditioner function: grid the weight (no MFS factor) with the
                            // conjugate CF on one half of the uv plane (TableVisGridder.cc:825-851)
};

// Sums of weights (rows, npol, image channels), column-major, in double; rows
// are CF planes (or CF indices when the weight is tracked per oversampling
// plane).  sumw == nullptr: not accumulated.
struct SumwArgs {
  double* sumw;
  const int* chan_map;
  int os, track_per_os, nrows, nchan_img;
};

}  // namespace yg

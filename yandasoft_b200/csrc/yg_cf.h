// Convolution-function cache and its GPU builders.
#pragma once
#include <atomic>
#include <vector>

#include "yg_internal.h"

namespace yg {

struct CFCacheDev {
  DevBuf data, off, size, offsets;
  int ncf = 0;
  int noffsets = 0;
  int maxsize = 0;
  int support = 0;          // itsSupport
  long long total = 0;      // complex elements
  std::vector<int> h_size;
  std::vector<long long> h_off;
  std::vector<int2> h_offsets;
  DevBuf pad;               // zero-padded wpad x wpad copy of every CF (gridding layout)
  int wpad = 0;
  CFView view() const;
  int layout(const std::vector<int>& sizes, const std::vector<int2>& offs);
  // rebuilds the padded copy from data; call after every change of the cache
  int refresh_pad(cudaStream_t st);
  int download(std::vector<float2>& out) const;
};

struct WProjCFParams {
  int shape_x = 0, shape_y = 0;   // padded grid shape
  double uvcell_u = 0, uvcell_v = 0;
  int os = 8;
  int maxsupport = 256;
  std::vector<double> wterms;     // per w-plane (wavelengths)
  double cutoff = 1e-3;
  bool cutoff_abs = false;
  int limitsupport = 0;
  bool variablesupport = false;
  bool offsetsupport = false;
  double alpha = 1.0;
};

struct AWCFParams : WProjCFParams {
  double diameter = 12.0;
  double blockage = 2.0;
  int maxfeeds = 1;
  int maxfields = 1;
  int nchan_cf = 1;               // channels of the cache (1 unless frequency dependent)
  std::vector<double> freqs;      // per cache channel
  bool spheroidaltaper = false;   // anti-aliasing spheroidal taper on the image-plane screen
};

struct AWFeedJob {
  int feed;
  int field;
  double l, m;                    // beam offset direction cosines (0 for the PSF)
};

int cf_build_sphfunc(CFCacheDev& cache, int support, int os, double alpha);
int cf_build_wproject(CFCacheDev& cache, const WProjCFParams& p, DevBuf& work, cudaStream_t st);
int cf_build_aw(CFCacheDev& cache, const AWCFParams& p, const std::vector<AWFeedJob>& jobs, DevBuf& work,
                cudaStream_t st);

// gridding entry points (yg_gridding.cu)
int plan_build(Plan& pl, const BinArgs& a, int vmax, DevError* err, cudaStream_t st);
// Grids the samples of a plan and, when sw.sumw is set, adds their weights into
// the sums of weights (one fused pass over the sorted samples).
int plan_grid(const Plan& pl, const VisArgs& v, const CFView& cf, float2* grid, int nx, int ny, int nchan_img,
              const SumwArgs& sw, DevBuf& scratch, DevBuf& svis, DevError* err, cudaStream_t st,
              cudaEvent_t ev0 = nullptr, cudaEvent_t ev1 = nullptr, int mode = 0,
              const struct LearnedCF* lcf = nullptr);
int plan_degrid(Plan& pl, const VisArgs& v, float2* vis_out, const CFView& cf, const float2* grid, int nx, int ny,
                int nchan_img, const int* chan_map, DevBuf& tmp_vals, float2* carry, DevError* err,
                cudaStream_t st, cudaEvent_t ev0 = nullptr, cudaEvent_t ev1 = nullptr,
                const struct LearnedCF* lcf = nullptr, int variant = 0, bool alone = true);
int plan_grid_carry(Plan& pl, const VisArgs& v, float2* carry, cudaStream_t st);
// per sorted sample inputs of the continuous learned CF (once per plan)
int plan_learned_inputs(Plan& pl, const double* uvw, const double* freq, double cellu, double cellv, int os,
                        int nchan_img, const double* wstack, double wnorm, cudaStream_t st);
int grid_cf_buffer_bytes(int wpad);
int grid_tile_for(int smax, int npol, bool varsup);
int grid_tile_stride(int tile, int wpad, int smax, bool varsup);
extern std::atomic<long long> g_kernel_launches;

}  // namespace yg

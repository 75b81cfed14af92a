// Autotuner: picks the uv tile side, the samples per work item and the k_grid
// thread layout for a CF width class (padded width Wp, polarisations) by
// timing a degrid + grid pass over a caller's device-resident chunk for each
// candidate, and remembers the winner for every later gridder of the process
// with the same class.  No counterpart in the reference (its gridding loop has
// no such parameters).
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "yg_gridder.h"

namespace yg {

namespace {

std::mutex g_tune_mutex;
std::map<std::pair<int, int>, TuneChoice> g_tune_table;

void throw_if(bool cond, int code, const char* msg) {
  if (cond) throw YgError{code, msg};
}

void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw YgError{YG_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e)};
}

}  // namespace

bool tune_lookup(int wpad, int npol, TuneChoice* out) {
  std::lock_guard<std::mutex> lk(g_tune_mutex);
  auto it = g_tune_table.find({wpad, npol});
  if (it == g_tune_table.end()) return false;
  *out = it->second;
  return true;
}

void tune_store(int wpad, int npol, const TuneChoice& c) {
  std::lock_guard<std::mutex> lk(g_tune_mutex);
  g_tune_table[{wpad, npol}] = c;
}

void tune_clear() {
  std::lock_guard<std::mutex> lk(g_tune_mutex);
  g_tune_table.clear();
}

// Times candidates on chunk dc (device resident).  The model grids of this
// gridder are used for the degrid half, so call it after initialiseDegrid or
// initialiseGrid; its grids and sums of weights are left as they were found
// only up to the passes it adds (re-initialise before real use).
TuneReport Gridder::autotune(const Chunk& dc, int max_trials) {
  throw_if(!dc.on_device, YG_ERR_ARG, "the autotuner needs a device-resident chunk");
  throw_if(!grids_.p || nx_ == 0, YG_ERR_STATE, "initialiseGrid or initialiseDegrid must come first");
  prepare_plan_cf(dc);
  const int smax = (cf_.maxsize - 1) / 2;
  const int wpad = ((2 * smax + 1) + 15) / 16 * 16;
  const int def_tile = grid_tile_for(smax, npol_, cf_.view().varsup != 0);
  std::vector<int> tiles;
  for (int t : {def_tile, def_tile / 2, def_tile * 3 / 4, def_tile * 3 / 2, def_tile * 2}) {
    t = t / 8 * 8;
    if (t >= 8 && t <= 256 && t <= def_tile * 2 && std::find(tiles.begin(), tiles.end(), t) == tiles.end())
      tiles.push_back(t);
  }
  const long long n = dc.nrow * (long long)dc.nchan;
  const int def_vmax = (int)std::min<long long>(1 << 20, std::max<long long>(512, n / (148 * 8)));
  std::vector<int> vmaxes = {def_vmax};
  for (int v : {def_vmax / 4, def_vmax * 4})
    if (v >= 128 && v <= (1 << 20)) vmaxes.push_back(v);
  // thread layouts: the default; for 16-wide CFs the plane-major records with
  // staged CF planes (tile in global memory, 193, or in shared memory, 65;
  // two polarisation groups, 194), half the threads, tap sums in registers
  // over the CF-major records (17); for wider CFs the default, 17 and half
  // the threads.  Position-major records with taps through L2 (32) measured
  // slower on the benchmark workloads and are not tried.
  const std::vector<int> variants =
      wpad == 16 ? std::vector<int>{1, 193, 65, 194, 2, 17} : std::vector<int>{1, 17, 2};
  const int save_tile = tile_override_, save_vmax = vmax_, save_mode = grid_mode_;
  Chunk scratch_chunk = dc;
  DevBuf model;
  const size_t bytes = (size_t)dc.nrow * dc.nchan * dc.npol * sizeof(float2);
  ck(model.ensure(bytes), "alloc");
  scratch_chunk.vis = model.as<float2>();
  const float* mfs = mfs_weights(dc);
  TuneReport rep;
  rep.wpad = wpad;
  rep.npol = npol_;
  cudaEvent_t e0, e1;
  ck(cudaEventCreate(&e0), "event");
  ck(cudaEventCreate(&e1), "event");
  int trials = 0;
  auto trial = [&](int t, int vm, int v) {
    tile_override_ = t;
    vmax_ = vm;
    grid_mode_ = v;
    float ms = -1.f;
    try {
      Plan pl;
      bin(dc, pl);
      ck(cudaMemsetAsync(model.p, 0, bytes, stream_), "clear");
      degrid_enqueue(scratch_chunk, pl, mfs, stream_);
      grid_enqueue(dc, pl, mfs, stream_);
      check_error();
      ck(cudaEventRecord(e0, stream_), "event");
      degrid_enqueue(scratch_chunk, pl, mfs, stream_);
      grid_enqueue(dc, pl, mfs, stream_);
      ck(cudaEventRecord(e1, stream_), "event");
      ck(cudaEventSynchronize(e1), "trial");
      check_error();
      cudaEventElapsedTime(&ms, e0, e1);
    } catch (const YgError& e) {
      if (e.code != YG_ERR_UNSUPPORTED) {
        tile_override_ = save_tile;
        vmax_ = save_vmax;
        grid_mode_ = save_mode;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        throw;
      }
    }
    ++trials;
    rep.trials.push_back(TuneTrial{t, vm, v, ms});
    if (ms > 0.f && (rep.best_ms < 0.f || ms < rep.best_ms)) {
      rep.best_ms = ms;
      rep.best = TuneChoice{t, vm, v};
    }
    if (t == def_tile && vm == def_vmax && v == 1) rep.default_ms = ms;
  };
  // the layouts at the default tile (the default first), then the other tiles
  // with the best layout, then the work-item size around the best of those
  for (int v : variants)
    if (trials < max_trials) trial(tiles[0], def_vmax, v);
  const int lead_variant = rep.best.variant;
  for (size_t k = 1; k < tiles.size(); ++k)
    if (trials < max_trials) trial(tiles[k], def_vmax, lead_variant);
  const TuneChoice lead = rep.best;
  for (int vm : vmaxes)
    if (vm != def_vmax && trials < max_trials && lead.tile > 0) trial(lead.tile, vm, lead.variant);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  tile_override_ = save_tile;
  vmax_ = save_vmax;
  grid_mode_ = save_mode;
  throw_if(rep.best_ms < 0.f, YG_ERR_UNSUPPORTED, "no candidate ran");
  tune_store(wpad, npol_, rep.best);
  apply_tuning(rep.best);
  return rep;
}

}  // namespace yg

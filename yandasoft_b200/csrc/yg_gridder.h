// C++ host side of the B200 gridder: the IVisGridder surface
// (askap/gridding/IVisGridder.h:64-140) and the VisGridderFactory parset
// handling (askap/gridding/VisGridderFactory.cc:112-285) for the SphFunc,
// WProject, WStack and AWProject gridders, on top of the CUDA kernels.
#pragma once
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "yg_cf.h"
#include "yg_image.h"
#include "yg_internal.h"
#include "yg_learned.h"
#include "yg_mlp.cuh"
#include "yg_spheroidal.h"

namespace yg {

class Parset {
 public:
  static Parset parse(const std::string& text);
  bool has(const std::string& k) const { return kv_.count(k) > 0; }
  std::string get(const std::string& k, const std::string& dflt) const;
  std::string get(const std::string& k) const;  // throws when missing
  double get_double(const std::string& k, double dflt) const;
  int get_int(const std::string& k, int dflt) const;
  bool get_bool(const std::string& k, bool dflt) const;
  Parset subset(const std::string& prefix) const;
  std::map<std::string, std::string> kv_;
};

struct YgError {
  int code;
  std::string msg;
};

// image axes: what initialiseCellSize / FrequencyMapper / getImageCentre read
struct Axes {
  double cell[2] = {0, 0};        // direction axis increments (radians)
  double centre[2] = {0, 0};      // image centre (ra, dec) radians
  double tangent[2] = {0, 0};     // tangent point (ra, dec) radians
  int has_freq = 0;
  double freq_start = 0, freq_end = 0;
};

// one accessor chunk
struct Chunk {
  long long nrow = 0;
  int nchan = 0, npol = 0;
  const double* uvw = nullptr;
  const double* delay = nullptr;
  const double* freq = nullptr;
  float2* vis = nullptr;
  const float2* noise = nullptr;
  const uint8_t* flag = nullptr;
  const int* feed1 = nullptr;
  const double* pointing = nullptr;
  int on_device = 0;
  const double* host_freq = nullptr;   // the caller's host copy of freq, when there is one
};

enum class Kind { SphFunc, WProject, WStack, AWProject, WStackWProject };

struct Stats {
  double samples_gridded = 0, taps_gridded = 0;
  double samples_degridded = 0, taps_degridded = 0;
  double time_grid_ms = 0, time_degrid_ms = 0, time_cf_ms = 0;
  double cf_generations = 0;
  double kgrid_ms = 0, kdegrid_ms = 0;   // k_grid / k_degrid only (CUDA events)
  double kgrid_calls = 0, kdegrid_calls = 0;
};

// autotuner (yg_autotune.cu)
struct TuneChoice {
  int tile = 0, vmax = 0, variant = 0;
};
struct TuneTrial {
  int tile, vmax, variant;
  float ms;        // degrid + grid pass; < 0: the candidate does not fit
};
struct TuneReport {
  int wpad = 0, npol = 0;
  TuneChoice best;
  float best_ms = -1.f, default_ms = -1.f;
  std::vector<TuneTrial> trials;
};
bool tune_lookup(int wpad, int npol, TuneChoice* out);
void tune_store(int wpad, int npol, const TuneChoice& c);
void tune_clear();

class Gridder {
 public:
  // VisGridderFactory::make
  static std::unique_ptr<Gridder> make(const Parset& parset);
  std::unique_ptr<Gridder> clone() const;
  ~Gridder();

  void initialise_grid(const Axes& axes, int nx, int ny, int npol, int nchan, bool dopsf, bool dopcf);
  void grid(const Chunk& c);
  void finalise_grid(float* out, bool out_on_device);
  void finalise_weights(float* out, bool out_on_device);
  void initialise_degrid(const Axes& axes, int nx, int ny, int npol, int nchan, const float* image, bool on_device);
  void degrid(Chunk& c);
  void finalise_degrid();
  void customise_for_context(const std::string& context);
  void init_vis_weights_mfs(double reffreq);
  bool is_model_empty() const { return model_empty_; }
  bool is_psf() const { return psf_; }
  bool is_pcf() const { return pcf_; }

  // inspection helpers
  Kind kind() const { return kind_; }
  int support() const { return cf_.support; }
  int oversample() const { return os_; }
  int ncf() const { return cf_.ncf; }
  void cf_sizes(std::vector<int>& sizes, std::vector<long long>& offs) const { sizes = cf_.h_size; offs = cf_.h_off; }
  void cf_offsets(std::vector<int2>& o) const { o = cf_.h_offsets; }
  void cf_data(std::vector<float2>& out) const;
  void sum_weights(std::vector<double>& out, int* nrows) const;
  void grid_data(std::vector<float2>& out) const;
  long long grid_elems() const;
  int ngrids() const;
  const Stats& stats() const { return stats_; }
  void shape(int* nx, int* ny, int* npol, int* nchan) const;
  double uvcell(int i) const { return uvcell_[i]; }
  // explicit CF build without data (WProject/SphFunc/WStack)
  void build_cf();
  float2* device_grid() { return grids_.as<float2>(); }
  cudaStream_t stream() const { return stream_; }
  // plan-level API for repeated passes over the same data
  // what a plan serves: both passes; gridding only (with the plane-major
  // kernel: one sort, by its key); degridding only (no gridding record order)
  enum PlanUse { PLAN_BOTH = 0, PLAN_GRID = 1, PLAN_DEGRID = 2 };
  void bin(const Chunk& c, Plan& pl, cudaStream_t st = nullptr, int use = PLAN_BOTH);
  void grid_plan(const Chunk& c, const Plan& pl);
  void degrid_plan(Chunk& c, Plan& pl);
  // launch-only cores of grid_plan / degrid_plan: no host synchronisation,
  // no allocation once sized, any stream (what a CUDA graph records)
  void grid_enqueue(const Chunk& dc, const Plan& pl, const float* mfs, cudaStream_t st, cudaEvent_t k0 = nullptr,
                    cudaEvent_t k1 = nullptr);
  // alone = false asks the degrid kernels for their all-warps ring protocol
  // instead of owned segments
  void degrid_enqueue(Chunk& dc, Plan& pl, const float* mfs, cudaStream_t st, cudaEvent_t k0 = nullptr,
                      cudaEvent_t k1 = nullptr, bool alone = true);
  const float* mfs_weights(const Chunk& dc);
  TuneReport autotune(const Chunk& dc, int max_trials);
  void apply_tuning(const TuneChoice& c) {
    tile_override_ = c.tile;
    vmax_ = c.vmax;
    grid_mode_ = c.variant;
  }
  void check_device_error() { check_error(); }
  void set_tile(int t) { tile_override_ = t; }
  void set_grid_mode(int m) { grid_mode_ = m; }
  int tile_for(int smax, int npol) const;
  int grid_variant() const;
  int items_vmax() const { return vmax_; }
  void set_vmax(int v) { vmax_ = v; }
  void sync();
  void ensure_device();
  // builds whatever CFs a chunk needs (AWProject builds from the data)
  void prepare_plan_cf(const Chunk& c) {
    ensure_device();
    init_cf(c);
  }
  // degrid of a device-resident chunk with no device allocation (yg_noalloc.cu)
  void degrid_noalloc(Chunk& c);

  // learned convolution function (no counterpart in the reference)
  void learned_train(const LearnParams& lp, int nw_train, LearnReport* rep);
  void learned_train_aw(const LearnParams& lp, LearnReport* rep);
  void set_cf_form(int form);  // 0 tabulated, 1 learned at the tabulated planes, 2 learned continuous
  int cf_form() const { return cf_form_; }
  void learned_params(std::vector<float>& out) const;
  void set_learned_params(const float* p, float scale);
  double learned_scale() const { return net_.scale; }
  size_t cf_table_bytes() const;
  // per-sample on-grid position (with CF offset), CF index and status of a plan
  void plan_samples(const Plan& pl, int* iu, int* iv, int* cfi, unsigned char* status) const;

 private:
  Gridder() = default;
  void configure(Kind k, const Parset& sub, const Parset& full);
  void init_axes(const Axes& axes, int nx, int ny, int npol, int nchan);
  void init_sumw();
  void init_cf(const Chunk& dc);
  void check_error(cudaStream_t st = nullptr);
  void upload_chunk(const Chunk& c, Chunk& dc, bool need_vis, bool vis_writable);
  std::vector<int> chan_map(const double* freq_host, int nchan) const;
  void fill_bin_args(BinArgs& a, const Chunk& dc, const int* dchan_map, const uint8_t* row_ok) const;
  double wterm_cf(int plane) const;
  void prepare_corrections();
  std::vector<uint8_t> psf_rows(const Chunk& hc);

  Kind kind_ = Kind::SphFunc;
  // parameters
  int os_ = 128;
  int sph_support_ = 3;
  double alpha_ = 1.0;
  WSampling ws_{};           // CF-side w sampling (W gridders)
  WSampling ws_stack_{};     // stack sampling (WStackWProject)
  double wmax_ = 0;
  double cutoff_ = 1e-3;
  bool cutoff_abs_ = false;
  int maxsupport_ = 256;
  int limitsupport_ = 0;
  bool variablesupport_ = false;
  bool offsetsupport_ = false;
  bool track_per_os_ = false;
  bool alldatapsf_ = false;
  double max_pointing_sep_ = -1.0;
  float padding_ = 1.0f;
  bool clear_grids_ = false;
  // AW
  double diameter_ = 12.0, blockage_ = 2.0;
  int maxfeeds_ = 1, maxfields_ = 1;
  bool aw_taper_ = false;               // AWProject spheroidaltaper
  double aw_weights_cutoff_ = 0.0;      // AWProject spheroidalweightscutoff
  bool freqdep_ = true;
  double pointing_tol_ = 1e-4, pa_tol_ = 0.1, freq_tol_ = 1e-6;
  std::vector<std::vector<int>> aw_done_;          // [field][feed]
  std::vector<std::vector<std::pair<double, double>>> aw_pointings_;
  std::vector<double> aw_cached_freqs_;
  int aw_last_field_ = -1, aw_current_field_ = 0;
  int aw_nchan_ = 0;
  // MFS weights
  bool mfs_ = false;
  double mfs_reffreq_ = 1.405e9;
  int mfs_order_ = 0;

  // state
  Axes axes_;
  int nx_ = 0, ny_ = 0, npol_ = 0, nchan_ = 0;
  double uvcell_[2] = {0, 0};
  bool psf_ = false, pcf_ = false;
  bool model_empty_ = false;
  bool first_psf_row_ = true;
  int rep_feed_ = 0;
  double rep_pointing_[2] = {0, 0};
  int tile_override_ = 0;
  int vmax_ = 0;   // samples per work item, 0 = automatic
  int grid_mode_ = 0;  // k_grid accumulation variant, 0 = automatic
  bool exact_rows_ = true;  // 16-wide CFs: residue rows modulo the real CF width

  CFCacheDev cf_;
  bool cf_built_ = false;
  LearnedNet net_;
  int cf_form_ = 0;
  DevBuf wterm_d_, wstack_d_, learn_X_, learn_T_, fb_d_;
  // AWProject learned CF: network inputs per CF plane (w term; frequency and
  // beam in [-1, 1]), kept on the host for clones
  std::vector<double> learn_wterm_h_;
  std::vector<float2> learn_fb_h_;
  std::vector<double> aw_cf_freqs_;     // frequencies of the AWProject CF cache channels
  void upload_learn_tables();
  double learn_wnorm_ = 1.0;
  LearnedCF learned_view() const;
  LearnedCF learned_view_for(const Chunk& dc, Plan& pl);
  DevBuf grids_, sumw_, carry_, err_, chanmap_d_, rowok_d_, corr_d_;
  HostMapped err_h_;                   // mapped host mirror of err_ for the read-back
  std::vector<float> mfs_w_;           // host MFS weights of the last upload
  std::vector<double> mfs_freqs_;      // frequencies they were made for
  int mfs_key_order_ = -1;
  double mfs_key_ref_ = 0.0;
  DevBuf up_uvw_, up_delay_, up_freq_, up_vis_, up_noise_, up_flag_, up_feed_;
  DevBuf scratch_, svis_, tmpvals_, cfwork_, img_tmp_, mfs_d_;
  int nsumw_rows_ = 1;
  Plan plan_;
  // host chunks in row pieces (upload / download overlapping the passes)
  struct Staging {
    DevBuf uvw, delay, freq, vis, noise, flag, feed;
  };
  static constexpr double kPipeMinBytes = 256.0 * (1 << 20);   // smaller chunks go in one piece
  static constexpr double kPipePieceBytes = 1024.0 * (1 << 20);
  Staging staging_[2];
  Plan piece_plan_[2];
  cudaStream_t copy_stream_ = nullptr;   // uploads
  cudaStream_t down_stream_ = nullptr;   // downloads of degridded pieces (the other PCIe direction)
  cudaEvent_t piece_up_[2] = {nullptr, nullptr};
  cudaEvent_t piece_down_[2] = {nullptr, nullptr};
  cudaEvent_t piece_done_ = nullptr;
  cudaStream_t bin_stream_ = nullptr;    // binning of the next host piece, beside the current pass
  cudaEvent_t piece_pass_[2] = {nullptr, nullptr};   // pass over a staging buffer done
  cudaEvent_t piece_binned_ = nullptr;
  bool pipelined(const Chunk& c) const;
  Chunk stage_rows(const Chunk& c, long long r0, long long nr, int b, bool need_vis);
  void run_pieces(Chunk& c, bool degridding);
  ImageFFT fft_;
  cudaStream_t stream_ = nullptr;
  Stats stats_;
  int device_ = 0;
  bool device_ready_ = false;
};

// size of the static device array used by Gridder::degrid_noalloc and the
// largest rows x channels it accepts per call
size_t noalloc_scratch_bytes();
long long noalloc_max_samples();

}  // namespace yg

// Host-side gridder classes: parset handling, state and call sequence of
// yandasoft's IVisGridder implementations, dispatching to the CUDA kernels.
//
// Reference behaviour followed here:
//   VisGridderFactory::make                 VisGridderFactory.cc:112-285
//   SphFuncVisGridder::createGridder        SphFuncVisGridder.cc:67-77
//   WStackVisGridder::createGridder         WStackVisGridder.cc:354-362
//   WProjectVisGridder::createGridder /
//     configureGridder                      WProjectVisGridder.cc:303-363
//   WDependentGridderBase (w sampling)      WDependentGridderBase.cc:53-67,192-245
//   AProjectGridderBase::createAProjectGridder / makeIllumination /
//     indexField / validateCFCache          AProjectGridderBase.tcc:54-118,
//                                           AProjectGridderBase.cc:166-301
//   TableVisGridder::initialiseGrid / initialiseCellSize / finaliseGrid /
//     finaliseWeights / initialiseDegrid / customiseForContext
//                                           TableVisGridder.cc:997-1079,1109-1319,1381-1405
//   FrequencyMapper::setupImage / setupMapping  FrequencyMapper.cc:55-107
#include "yg_gridder.h"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <sstream>
#include <stdexcept>

namespace yg {

static void throw_if(bool cond, int code, const std::string& msg) {
  if (cond) throw YgError{code, msg};
}

static void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw YgError{YG_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e)};
}

static void rc_check(int rc, const char* what) {
  if (rc != YG_OK) {
    std::string m = what;
    if (rc == YG_ERR_CUDA) {
      cudaError_t e = cudaGetLastError();
      m += std::string(": CUDA error ") + cudaGetErrorString(e);
    }
    if (rc == YG_ERR_SUPPORT)
      m += ": unable to determine the support of the convolution function, or it overflows the buffer - "
           "increase maxsupport or cutoff or decrease oversample";
    if (rc == YG_ERR_UNSUPPORTED) m += ": configuration not supported by this gridder";
    throw YgError{rc, m};
  }
}

// ---------------------------------------------------------------------------
// Parset
// ---------------------------------------------------------------------------
static std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace((unsigned char)s[a])) ++a;
  while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
  return s.substr(a, b - a);
}

Parset Parset::parse(const std::string& text) {
  Parset p;
  std::istringstream in(text);
  std::string line;
  while (std::getline(in, line)) {
    const size_t hash = line.find('#');
    if (hash != std::string::npos) line = line.substr(0, hash);
    const size_t eq = line.find('=');
    if (eq == std::string::npos) continue;
    std::string k = trim(line.substr(0, eq)), v = trim(line.substr(eq + 1));
    if (k.rfind("Cimager.", 0) == 0) k = k.substr(8);
    if (!k.empty()) p.kv_[k] = v;
  }
  return p;
}

std::string Parset::get(const std::string& k, const std::string& dflt) const {
  auto it = kv_.find(k);
  return it == kv_.end() ? dflt : it->second;
}

std::string Parset::get(const std::string& k) const {
  auto it = kv_.find(k);
  throw_if(it == kv_.end(), YG_ERR_ARG, "Parameter " + k + " is not defined");
  return it->second;
}

double Parset::get_double(const std::string& k, double dflt) const {
  auto it = kv_.find(k);
  if (it == kv_.end()) return dflt;
  char* end = nullptr;
  const double v = std::strtod(it->second.c_str(), &end);
  throw_if(end == it->second.c_str(), YG_ERR_ARG, "Parameter " + k + " is not a number: " + it->second);
  return v;
}

int Parset::get_int(const std::string& k, int dflt) const {
  auto it = kv_.find(k);
  if (it == kv_.end()) return dflt;
  char* end = nullptr;
  const long v = std::strtol(it->second.c_str(), &end, 10);
  throw_if(end == it->second.c_str(), YG_ERR_ARG, "Parameter " + k + " is not an integer: " + it->second);
  return (int)v;
}

bool Parset::get_bool(const std::string& k, bool dflt) const {
  auto it = kv_.find(k);
  if (it == kv_.end()) return dflt;
  std::string v = it->second;
  std::transform(v.begin(), v.end(), v.begin(), ::tolower);
  if (v == "true" || v == "t" || v == "1" || v == "yes" || v == "y") return true;
  if (v == "false" || v == "f" || v == "0" || v == "no" || v == "n") return false;
  throw YgError{YG_ERR_ARG, "Parameter " + k + " is not a boolean: " + it->second};
}

Parset Parset::subset(const std::string& prefix) const {
  Parset p;
  for (const auto& kv : kv_)
    if (kv.first.rfind(prefix, 0) == 0) p.kv_[kv.first.substr(prefix.size())] = kv.second;
  return p;
}

// quantity string -> value in the requested unit (rad or m)
static double convert_quantity(const std::string& s, const std::string& unit) {
  char* end = nullptr;
  const double v = std::strtod(s.c_str(), &end);
  throw_if(end == s.c_str(), YG_ERR_ARG, "Unable to parse quantity " + s);
  std::string u = trim(std::string(end));
  if (u.empty()) return v;
  if (unit == "rad") {
    if (u == "rad") return v;
    if (u == "deg") return v * M_PI / 180.0;
    if (u == "arcmin") return v * M_PI / (180.0 * 60.0);
    if (u == "arcsec") return v * M_PI / (180.0 * 3600.0);
  } else if (unit == "m") {
    if (u == "m") return v;
    if (u == "km") return v * 1000.0;
    if (u == "cm") return v * 0.01;
  }
  throw YgError{YG_ERR_ARG, "Unable to convert quantity " + s + " to " + unit};
}

// ---------------------------------------------------------------------------
// w sampling
// ---------------------------------------------------------------------------
static void gauss_params(double wplanes50, double* ts2_out, double* amp_out) {
  throw_if(!(wplanes50 > 0), YG_ERR_ARG, "Fraction of w-planes containing 50% of -wmax,wmax range should be positive");
  throw_if(!(wplanes50 * std::sqrt(2.0) < 1.), YG_ERR_ARG,
           "Normalised fraction of w-planes containing 50% of the w range should not exceed 1/sqrt(2)");
  auto target = [](double ts2) { return std::sqrt(-ts2 * std::log(0.5 + 0.5 * std::exp(-1. / ts2))); };
  double lo = wplanes50 * wplanes50 / std::log(2.) / 2.;
  double hi = 0.2 / (1 / std::sqrt(2) - wplanes50);
  if (hi < lo) {
    lo = hi;
    hi = 5.;
  }
  double ts2 = 1.;
  for (int it = 0; it < 100; ++it) {
    ts2 = (lo + hi) / 2.;
    if (target(ts2) < wplanes50) lo = ts2; else hi = ts2;
    if (hi - lo < 1e-5) break;
  }
  *ts2_out = ts2;
  *amp_out = 1. / (1. - std::exp(-1. / ts2));
}

static WSampling make_wsampling(double wmax, int nwplanes, const Parset& ps) {
  throw_if(!(wmax > 0.0), YG_ERR_ARG, "Baseline length must be greater than zero");
  throw_if(nwplanes <= 0, YG_ERR_ARG, "Number of w planes must be greater than zero");
  throw_if(nwplanes % 2 != 1, YG_ERR_ARG, "Number of w planes must be odd, you have nwplanes=" + std::to_string(nwplanes));
  WSampling s{};
  s.nwplanes = nwplanes;
  s.wscale = nwplanes > 1 ? wmax / double((nwplanes - 1) / 2) : 1.0;
  s.kind = WS_LINEAR;
  s.two_sigma2 = 1.0;
  const std::string smp = ps.get("wsampling", "linear");
  if (smp == "powerlaw") {
    s.kind = WS_POWER;
    s.exponent = ps.get_double("wsampling.exponent", 0.0);
    throw_if(!ps.has("wsampling.exponent"), YG_ERR_ARG, "Parameter wsampling.exponent is not defined");
    throw_if(s.exponent == 0., YG_ERR_ARG, "Zero exponent in power law doesn't make sense");
  } else if (smp == "gaussian") {
    s.kind = WS_GAUSS;
    throw_if(!ps.has("wsampling.nwplanes50"), YG_ERR_ARG, "Parameter wsampling.nwplanes50 is not defined");
    const double n50 = ps.get_double("wsampling.nwplanes50", 0.0);
    throw_if(!(n50 > 0. && n50 < double(nwplanes) / std::sqrt(2.)), YG_ERR_ARG,
             "Number of w-planes covering 50% of w-range has to be positive and below nwplanes/sqrt(2)");
    gauss_params(n50 / nwplanes, &s.two_sigma2, &s.amplitude);
  } else if (smp != "linear") {
    throw YgError{YG_ERR_ARG, "W-sampling " + smp + " is not implemented"};
  }
  s.wmaxclip = ps.get_bool("wmaxclip", false) ? 1 : 0;
  return s;
}

static double wterm_of(const WSampling& s, int plane) {
  const int half = (s.nwplanes - 1) / 2;
  if (s.kind != WS_LINEAR && s.nwplanes > 1) {
    const double x = double(plane - half) / double(half);
    double m;
    if (s.kind == WS_POWER) {
      m = x > 0 ? std::pow(x, s.exponent) : (x < 0 ? -std::pow(-x, s.exponent) : 0.);
    } else {
      const double a = s.amplitude * (1 - std::exp(-x * x / s.two_sigma2));
      m = x < 0 ? -a : (x > 0 ? a : 0.);
    }
    return m * (s.wscale * half);
  }
  return double(plane - half) * s.wscale;
}

double Gridder::wterm_cf(int plane) const { return wterm_of(ws_, plane); }

// ---------------------------------------------------------------------------
// factory
// ---------------------------------------------------------------------------
std::unique_ptr<Gridder> Gridder::make(const Parset& parset) {
  const std::string name = parset.get("gridder");
  const Parset sub = parset.subset("gridder." + name + ".");
  Kind k;
  if (name == "SphFunc") k = Kind::SphFunc;
  else if (name == "WProject") k = Kind::WProject;
  else if (name == "WStack") k = Kind::WStack;
  else if (name == "AWProject") k = Kind::AWProject;
  else if (name == "WStackWProject") k = Kind::WStackWProject;
  else throw YgError{YG_ERR_ARG, "Unknown gridder " + name};
  std::unique_ptr<Gridder> g(new Gridder());
  g->configure(k, sub, parset);
  return g;
}

void Gridder::ensure_device() {
  if (device_ready_) return;
  cuda_check(cudaGetDevice(&device_), "cudaGetDevice");
  cuda_check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
  cuda_check(err_.ensure(sizeof(DevError)), "alloc");
  cuda_check(cudaMemset(err_.p, 0, sizeof(DevError)), "memset");
  cuda_check(carry_.ensure(8 * sizeof(float2)), "alloc");
  cuda_check(cudaMemset(carry_.p, 0, 8 * sizeof(float2)), "memset");
  device_ready_ = true;
}

void Gridder::configure(Kind k, const Parset& p, const Parset& full) {
  kind_ = k;
  alpha_ = p.get_double("alpha", 1.0);
  throw_if(!(alpha_ >= 0. && alpha_ <= 2.), YG_ERR_ARG, "alpha must be in [0, 2]");
  switch (k) {
    case Kind::SphFunc:
      os_ = p.get_int("oversample", 128);
      sph_support_ = p.get_int("support", 3);
      throw_if(sph_support_ < 3 || os_ < 1, YG_ERR_ARG, "SphFunc needs support >= 3 and oversample >= 1");
      break;
    case Kind::WStack:
      os_ = 128;
      sph_support_ = 3;
      wmax_ = p.get_double("wmax", 35000.0);
      ws_ = make_wsampling(wmax_, p.get_int("nwplanes", 65), p);
      break;
    case Kind::WProject:
    case Kind::WStackWProject:
    case Kind::AWProject: {
      const bool aw = k == Kind::AWProject;
      wmax_ = p.get_double("wmax", aw ? 10000.0 : 35000.0);
      const int nw = p.get_int("nwplanes", k == Kind::WStackWProject ? 33 : 65);
      cutoff_ = p.get_double("cutoff", 1e-3);
      os_ = p.get_int("oversample", 8);
      maxsupport_ = p.get_int("maxsupport", aw ? 128 : 256);
      limitsupport_ = p.get_int("limitsupport", 0);
      throw_if(os_ <= 0, YG_ERR_ARG, "Oversampling must be greater than 0");
      throw_if(maxsupport_ <= 0, YG_ERR_ARG, "Maximum support must be greater than 0");
      variablesupport_ = p.get_bool("variablesupport", false);
      offsetsupport_ = p.get_bool("offsetsupport", false);
      throw_if(offsetsupport_ && !variablesupport_, YG_ERR_ARG,
               "offsetsupport option of the gridder should only be used together with variablesupport option");
      cutoff_abs_ = p.get_bool("cutoff.absolute", false);
      if (!cutoff_abs_) {
        throw_if(!(cutoff_ > 0.0), YG_ERR_ARG, "Cutoff must be positive");
        throw_if(!(cutoff_ < 1.0), YG_ERR_ARG, "Cutoff must be less than 1.0");
      }
      if (k == Kind::WStackWProject) {
        const int nst = p.get_int("nwstacks", 17);
        ws_stack_ = make_wsampling(wmax_, nst, Parset());
        ws_stack_.wmaxclip = p.get_bool("wmaxclip", false) ? 1 : 0;
        // residual w within one stack spans half a stack spacing either side
        const double half_spacing = 0.5 * ws_stack_.wscale;
        ws_ = make_wsampling(half_spacing > 0 ? half_spacing : wmax_, nw, Parset());
        ws_.wmaxclip = 0;
      } else {
        ws_ = make_wsampling(wmax_, nw, p);
      }
      if (aw) {
        pointing_tol_ = convert_quantity(p.get("pointingtolerance", "0.0001rad"), "rad");
        pa_tol_ = convert_quantity(p.get("patolerance", "0.1rad"), "rad");
        std::string ft = p.get("freqtolerance", "undefined");
        std::string ftl = ft;
        std::transform(ftl.begin(), ftl.end(), ftl.begin(), ::tolower);
        if (ftl == "infinite") {
          freq_tol_ = -1.0;
        } else {
          freq_tol_ = p.get_double("freqtolerance", 1e-6);
          throw_if(!(freq_tol_ >= 0.), YG_ERR_ARG, "Frequency tolerance must be non-negative or infinite");
        }
        maxfeeds_ = p.get_int("maxfeeds", 1);
        maxfields_ = p.get_int("maxfields", 1);
        throw_if(maxfeeds_ <= 0, YG_ERR_ARG, "Maximum number of feeds must be one or more");
        throw_if(maxfields_ <= 0, YG_ERR_ARG, "Maximum number of fields must be one or more");
        freqdep_ = p.get_bool("frequencydependent", true);
        aw_taper_ = p.get_bool("spheroidaltaper", false);
        aw_weights_cutoff_ = p.get_double("spheroidalweightscutoff", 0.0);
        const std::string illum = p.get("illumination", "disk");
        throw_if(illum != "disk", YG_ERR_UNSUPPORTED, "Illumination " + illum + " is not supported (disk only)");
        diameter_ = convert_quantity(p.get("diameter"), "m");
        blockage_ = convert_quantity(p.get("blockage"), "m");
        throw_if(!(diameter_ > 0 && blockage_ >= 0 && diameter_ > blockage_), YG_ERR_ARG,
                 "Disk illumination needs diameter > blockage >= 0");
        aw_done_.assign(maxfields_, std::vector<int>(maxfeeds_, 0));
        aw_pointings_.assign(maxfields_, std::vector<std::pair<double, double>>(maxfeeds_, {0.0, 0.0}));
      }
      break;
    }
  }
  // generic keys of VisGridderFactory::make
  if (full.has("gridder.padding")) padding_ = (float)full.get_double("gridder.padding", 1.0);
  throw_if(!(padding_ > 0), YG_ERR_ARG, "padding must be positive");
  if (full.has("gridder.MaxPointingSeparation"))
    max_pointing_sep_ = convert_quantity(full.get("gridder.MaxPointingSeparation", "-1rad"), "rad");
  alldatapsf_ = full.get_bool("gridder.alldatapsf", false);
  track_per_os_ = full.get_bool("gridder.oversampleweight", false);
  throw_if(full.get_bool("gridder.parotation", false), YG_ERR_UNSUPPORTED,
           "gridder.parotation needs a polarisation converter, which this gridder does not provide");
  clear_grids_ = full.get_bool("gridder.cleargrids", false);
  if (full.get("visweights", "") == "MFS") init_vis_weights_mfs(full.get_double("visweights.MFS.reffreq", 1.405e9));
  throw_if(full.get_bool("gridder.snapshotimaging", false), YG_ERR_UNSUPPORTED,
           "gridder.snapshotimaging adapter is not provided by this gridder");
  throw_if(full.get_bool("gridder.bwsmearing", false), YG_ERR_UNSUPPORTED,
           "gridder.bwsmearing adapter is not provided by this gridder");
}

std::unique_ptr<Gridder> Gridder::clone() const {
  std::unique_ptr<Gridder> g(new Gridder());
  g->kind_ = kind_;
  g->os_ = os_;
  g->sph_support_ = sph_support_;
  g->alpha_ = alpha_;
  g->ws_ = ws_;
  g->ws_stack_ = ws_stack_;
  g->wmax_ = wmax_;
  g->cutoff_ = cutoff_;
  g->cutoff_abs_ = cutoff_abs_;
  g->maxsupport_ = maxsupport_;
  g->limitsupport_ = limitsupport_;
  g->variablesupport_ = variablesupport_;
  g->offsetsupport_ = offsetsupport_;
  g->track_per_os_ = track_per_os_;
  g->alldatapsf_ = alldatapsf_;
  g->max_pointing_sep_ = max_pointing_sep_;
  g->padding_ = padding_;
  g->clear_grids_ = clear_grids_;
  g->diameter_ = diameter_;
  g->blockage_ = blockage_;
  g->maxfeeds_ = maxfeeds_;
  g->maxfields_ = maxfields_;
  g->freqdep_ = freqdep_;
  g->aw_taper_ = aw_taper_;
  g->aw_weights_cutoff_ = aw_weights_cutoff_;
  g->pointing_tol_ = pointing_tol_;
  g->pa_tol_ = pa_tol_;
  g->freq_tol_ = freq_tol_;
  g->aw_done_.assign(maxfields_, std::vector<int>(maxfeeds_, 0));
  g->aw_pointings_.assign(maxfields_, std::vector<std::pair<double, double>>(maxfeeds_, {0.0, 0.0}));
  g->mfs_ = mfs_;
  g->mfs_reffreq_ = mfs_reffreq_;
  g->mfs_order_ = mfs_order_;
  g->tile_override_ = tile_override_;
  g->vmax_ = vmax_;
  if (net_.ready) {
    std::vector<float> p;
    learned_params(p);
    g->set_learned_params(p.data(), net_.scale);
    g->learn_wnorm_ = learn_wnorm_;
    g->learn_wterm_h_ = learn_wterm_h_;
    g->learn_fb_h_ = learn_fb_h_;
    if (!learn_fb_h_.empty()) g->upload_learn_tables();
    g->cf_form_ = cf_form_;
  }
  if (device_ready_) {
    // the copy constructor copies itsImagePolFrameVis (TableVisGridder.cc:156):
    // off-grid samples that a clone degrids before its first on-grid one take
    // the value this gridder last carried
    cuda_check(cudaStreamSynchronize(stream_), "cudaStreamSynchronize");
    g->ensure_device();
    cuda_check(cudaMemcpy(g->carry_.p, carry_.p, 8 * sizeof(float2), cudaMemcpyDeviceToDevice), "carry copy");
  }
  return g;
}

Gridder::~Gridder() {
  for (cudaStream_t* cs : {&copy_stream_, &down_stream_, &bin_stream_}) {
    if (*cs) {
      cudaStreamSynchronize(*cs);
      cudaStreamDestroy(*cs);
    }
  }
  for (auto& e : piece_up_)
    if (e) cudaEventDestroy(e);
  for (auto& e : piece_down_)
    if (e) cudaEventDestroy(e);
  if (piece_done_) cudaEventDestroy(piece_done_);
  for (auto& e : piece_pass_)
    if (e) cudaEventDestroy(e);
  if (piece_binned_) cudaEventDestroy(piece_binned_);
  if (stream_) {
    cudaStreamSynchronize(stream_);
    cudaStreamDestroy(stream_);
  }
}

void Gridder::sync() {
  ensure_device();
  cuda_check(cudaStreamSynchronize(stream_), "cudaStreamSynchronize");
}

// the device error record copied into mapped host memory
__global__ void k_error_out(const DevError* __restrict__ d, DevError* h) {
  h->code = d->code;
  h->where = d->where;
}

void Gridder::check_error(cudaStream_t st) {
  if (!st) st = stream_;
  cuda_check(err_h_.ensure(sizeof(DevError)), "alloc error mirror");
  k_error_out<<<1, 1, 0, st>>>(err_.as<DevError>(), err_h_.as<DevError>());
  cuda_check(cudaGetLastError(), "error readback");
  cuda_check(cudaStreamSynchronize(st), "kernel execution");
  DevError h{};
  h.code = err_h_.as<volatile DevError>()->code;
  h.where = err_h_.as<volatile DevError>()->where;
  if (h.code != YG_OK) {
    cudaMemsetAsync(err_.p, 0, sizeof(DevError), stream_);
    cudaStreamSynchronize(stream_);
    std::string m;
    switch (h.code) {
      case YG_ERR_FRAC: m = "Fractional offset in u or v outside [0, oversample)"; break;
      case YG_ERR_WRANGE: m = "W scaling error: recommend allowing larger range of w"; break;
      case YG_ERR_WEIGHT: m = "Weight is supposed to be a positive number"; break;
      case YG_ERR_CINDEX: m = "Index into convolution functions exceeds number of planes"; break;
      case YG_ERR_TIMEOUT: {
        // timeout_where(): kernel, waiting role, segment, block
        static const char* kern[] = {"?", "k_grid", "k_grid_pl", "k_degrid_t", "k_degrid_r"};
        static const char* role[] = {"?", "producer waiting for a free stage", "tap warp waiting for a filled stage",
                                     "producer waiting for the plane buffer"};
        const unsigned long long w = (unsigned long long)h.where;
        const int k = (int)(w >> 60) & 7, r = (int)(w >> 56) & 15;
        throw YgError{h.code, std::string("a bounded wait gave up in ") + kern[k < 5 ? k : 0] + " (" +
                                  role[r < 4 ? r : 0] + ", segment " + std::to_string((w >> 32) & 0xffffff) +
                                  ", block " + std::to_string(w & 0xffffffffull) + ")"};
      }
      default: m = "device error"; break;
    }
    throw YgError{h.code, m + " (sample " + std::to_string(h.where) + ")"};
  }
}

// ---------------------------------------------------------------------------
// axes, shapes, weights
// ---------------------------------------------------------------------------
void Gridder::init_axes(const Axes& axes, int nx, int ny, int npol, int nchan) {
  throw_if(nx <= 0 || ny <= 0 || npol <= 0 || nchan <= 0, YG_ERR_ARG, "bad image shape");
  axes_ = axes;
  nx_ = (int)(nx * padding_);
  ny_ = (int)(ny * padding_);
  throw_if(nx_ % 2 || ny_ % 2, YG_ERR_ARG, "padded grid sizes must be even");
  throw_if(nx_ > 65535 || ny_ > 65535, YG_ERR_ARG, "grid sizes above 65535 are not supported");
  npol_ = npol;
  nchan_ = nchan;
  throw_if(!(axes.cell[0] != 0 && axes.cell[1] != 0), YG_ERR_ARG, "Direction axis increments are missing");
  uvcell_[0] = 1. / (axes.cell[0] * double(nx_));
  uvcell_[1] = 1. / (axes.cell[1] * double(ny_));
}

int Gridder::ngrids() const {
  if (kind_ == Kind::WStack) return ws_.nwplanes;
  if (kind_ == Kind::WStackWProject) return ws_stack_.nwplanes;
  return 1;
}

long long Gridder::grid_elems() const { return (long long)nx_ * ny_ * npol_ * nchan_; }

void Gridder::shape(int* nx, int* ny, int* npol, int* nchan) const {
  *nx = nx_;
  *ny = ny_;
  *npol = npol_;
  *nchan = nchan_;
}

void Gridder::init_sumw() {
  int numcf = 1;
  if (kind_ == Kind::WProject || kind_ == Kind::WStackWProject) numcf = ws_.nwplanes;
  if (kind_ == Kind::AWProject) {
    numcf = (cf_built_ && aw_nchan_ > 0) ? ws_.nwplanes * maxfeeds_ * maxfields_ * aw_nchan_ : ws_.nwplanes;
  }
  nsumw_rows_ = track_per_os_ ? numcf * os_ * os_ : numcf;
  cuda_check(sumw_.ensure((size_t)nsumw_rows_ * npol_ * nchan_ * sizeof(double)), "alloc sumw");
  cuda_check(cudaMemsetAsync(sumw_.p, 0, (size_t)nsumw_rows_ * npol_ * nchan_ * sizeof(double), stream_), "memset");
}

void Gridder::initialise_grid(const Axes& axes, int nx, int ny, int npol, int nchan, bool dopsf, bool dopcf) {
  ensure_device();
  throw_if(dopsf && dopcf, YG_ERR_UNSUPPORTED,
           "a gridder is configured for the PSF or for the preconditioner function, not both at once");
  throw_if(dopcf && cf_form_ != 0, YG_ERR_UNSUPPORTED, "the preconditioner function uses the tabulated CFs");
  init_axes(axes, nx, ny, npol, nchan);
  psf_ = dopsf;
  pcf_ = dopcf;
  model_empty_ = false;
  const size_t bytes = (size_t)ngrids() * grid_elems() * sizeof(float2);
  cuda_check(grids_.ensure(bytes), "alloc grids");
  cuda_check(cudaMemsetAsync(grids_.p, 0, bytes, stream_), "memset grids");
  first_psf_row_ = true;
  init_sumw();
  sync();
}

void Gridder::customise_for_context(const std::string& context) {
  // ImageParamsHelper: ".taylor.N" selects Taylor term N, otherwise order 1
  int order = 1;
  const size_t t = context.find(".taylor.");
  if (t != std::string::npos) order = std::atoi(context.c_str() + t + 8);
  if (mfs_) mfs_order_ = order;
}

void Gridder::init_vis_weights_mfs(double reffreq) {
  throw_if(!(reffreq != 0.), YG_ERR_ARG, "MFS reference frequency must be non-zero");
  mfs_ = true;
  mfs_reffreq_ = reffreq;
  mfs_order_ = 0;
}

// FrequencyMapper: accessor channel -> image channel
std::vector<int> Gridder::chan_map(const double* freq, int nchan) const {
  std::vector<int> m(nchan, 0);
  if (!axes_.has_freq || nchan_ == 1) return m;
  const double inc = (axes_.freq_end - axes_.freq_start) / double(nchan_ - 1);
  throw_if(!(std::fabs(inc) > 0), YG_ERR_ARG, "Frequency axis in the image has the same start and end frequency");
  for (int c = 0; c < nchan; ++c) {
    double d = (freq[c] - axes_.freq_start) / inc;
    d += (d < 0.) ? -0.5 : 0.5;
    const int ic = int(d);
    m[c] = (ic < 0 || ic >= nchan_) ? -1 : ic;
  }
  return m;
}

// ---------------------------------------------------------------------------
// uploads
// ---------------------------------------------------------------------------
void Gridder::upload_chunk(const Chunk& c, Chunk& dc, bool need_vis, bool vis_writable) {
  dc = c;
  if (c.on_device) return;
  const long long n = c.nrow * (long long)c.nchan;
  auto up = [&](DevBuf& b, const void* src, size_t bytes) -> void* {
    if (!src) return nullptr;
    cuda_check(b.ensure(bytes), "alloc upload");
    cuda_check(cudaMemcpyAsync(b.p, src, bytes, cudaMemcpyHostToDevice, stream_), "upload");
    return b.p;
  };
  dc.uvw = (const double*)up(up_uvw_, c.uvw, (size_t)c.nrow * 3 * sizeof(double));
  dc.delay = (const double*)up(up_delay_, c.delay, (size_t)c.nrow * sizeof(double));
  dc.freq = (const double*)up(up_freq_, c.freq, (size_t)c.nchan * sizeof(double));
  if (need_vis || vis_writable) dc.vis = (float2*)up(up_vis_, c.vis, (size_t)n * c.npol * sizeof(float2));
  dc.noise = (const float2*)up(up_noise_, c.noise, (size_t)n * c.npol * sizeof(float2));
  dc.flag = (const uint8_t*)up(up_flag_, c.flag, (size_t)n * c.npol);
  dc.feed1 = (const int*)up(up_feed_, c.feed1, (size_t)c.nrow * sizeof(int));
  dc.pointing = c.pointing;  // host-side use only
  dc.host_freq = c.freq;
  dc.on_device = 1;
}

// The chunk's frequencies on the host: from the caller's host array when the
// chunk was staged from one, else read back from the device.
static std::vector<double> host_freqs(const Chunk& c) {
  std::vector<double> f(c.nchan);
  if (c.host_freq) std::memcpy(f.data(), c.host_freq, c.nchan * sizeof(double));
  else if (c.on_device) cuda_check(cudaMemcpy(f.data(), c.freq, c.nchan * sizeof(double), cudaMemcpyDeviceToHost), "freq");
  else std::memcpy(f.data(), c.freq, c.nchan * sizeof(double));
  return f;
}

static double separation(double ra1, double dec1, double ra2, double dec2) {
  const double c = std::sin(dec1) * std::sin(dec2) + std::cos(dec1) * std::cos(dec2) * std::cos(ra1 - ra2);
  return std::acos(std::max(-1.0, std::min(1.0, c)));
}

// ---------------------------------------------------------------------------
// convolution functions
// ---------------------------------------------------------------------------
void Gridder::build_cf() {
  ensure_device();
  if (cf_built_) return;
  throw_if(nx_ == 0, YG_ERR_STATE, "initialiseGrid or initialiseDegrid must be called first");
  if (kind_ == Kind::SphFunc || kind_ == Kind::WStack) {
    rc_check(cf_build_sphfunc(cf_, sph_support_, os_, alpha_), "SphFunc CF");
  } else if (kind_ == Kind::WProject || kind_ == Kind::WStackWProject) {
    WProjCFParams p;
    p.shape_x = nx_;
    p.shape_y = ny_;
    p.uvcell_u = uvcell_[0];
    p.uvcell_v = uvcell_[1];
    p.os = os_;
    p.maxsupport = maxsupport_;
    p.wterms.resize(ws_.nwplanes);
    for (int i = 0; i < ws_.nwplanes; ++i) p.wterms[i] = wterm_cf(i);
    p.cutoff = cutoff_;
    p.cutoff_abs = cutoff_abs_;
    p.limitsupport = limitsupport_;
    p.variablesupport = variablesupport_;
    p.offsetsupport = offsetsupport_;
    p.alpha = alpha_;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, stream_);
    rc_check(cf_build_wproject(cf_, p, cfwork_, stream_), "WProject CF generation");
    cudaEventRecord(e1, stream_);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    stats_.time_cf_ms += ms;
    stats_.cf_generations += ws_.nwplanes;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cfwork_.release();
  } else {
    throw YgError{YG_ERR_STATE, "AWProject convolution functions are built from the data"};
  }
  cf_built_ = true;
}

void Gridder::init_cf(const Chunk& dc) {
  if (kind_ != Kind::AWProject) {
    build_cf();
    return;
  }
  // AProjectGridderBase::indexField (first row of the chunk)
  throw_if(!dc.pointing && maxfields_ > 1, YG_ERR_ARG, "AWProject needs pointing directions");
  std::vector<int> feed(dc.nrow, 0);
  if (dc.feed1) {
    if (dc.on_device && up_feed_.p == (void*)dc.feed1) {
      cuda_check(cudaMemcpy(feed.data(), dc.feed1, dc.nrow * sizeof(int), cudaMemcpyDeviceToHost), "feed");
    } else if (dc.on_device) {
      cuda_check(cudaMemcpy(feed.data(), dc.feed1, dc.nrow * sizeof(int), cudaMemcpyDeviceToHost), "feed");
    } else {
      std::memcpy(feed.data(), dc.feed1, dc.nrow * sizeof(int));
    }
  }
  const std::vector<double> freqs = host_freqs(dc);
  auto pnt = [&](long long r) -> std::pair<double, double> {
    if (!dc.pointing) return {axes_.centre[0], axes_.centre[1]};
    return {dc.pointing[2 * r], dc.pointing[2 * r + 1]};
  };
  const int first_feed = feed.empty() ? 0 : feed[0];
  throw_if(first_feed < 0 || first_feed >= maxfeeds_, YG_ERR_ARG, "Too many feeds: increase maxfeeds");
  const auto fp = pnt(0);
  bool new_field = true;
  for (int f = aw_last_field_; f > -1; --f) {
    const auto& q = aw_pointings_[f][first_feed];
    if (separation(fp.first, fp.second, q.first, q.second) < pointing_tol_) {
      aw_current_field_ = f;
      new_field = false;
      break;
    }
  }
  if (new_field) {
    ++aw_last_field_;
    aw_current_field_ = aw_last_field_;
    throw_if(aw_current_field_ >= maxfields_, YG_ERR_ARG, "Too many fields: increase maxfields");
    aw_pointings_[aw_current_field_][first_feed] = fp;
  }
  // validateCFCache: the disk illumination is symmetric, so only frequencies
  bool invalid_freq = false;
  if (freq_tol_ >= 0.) {
    if (freqs.size() != aw_cached_freqs_.size()) {
      invalid_freq = true;
    } else {
      for (size_t c = 0; c < freqs.size(); ++c)
        if (std::fabs(aw_cached_freqs_[c] - freqs[c]) / freqs[c] > freq_tol_) { invalid_freq = true; break; }
    }
    if (invalid_freq) {
      for (auto& v : aw_done_) std::fill(v.begin(), v.end(), 0);
      aw_cached_freqs_ = freqs;
    }
  }
  const int nchan_cf = freqdep_ ? dc.nchan : 1;
  if (!cf_built_) aw_nchan_ = nchan_cf;
  std::vector<AWFeedJob> jobs;
  for (long long r = 0; r < dc.nrow; ++r) {
    const int f = feed[r];
    throw_if(f < 0 || f >= maxfeeds_, YG_ERR_ARG, "Exceeded specified maximum number of feeds");
    if (!aw_done_[aw_current_field_][f]) {
      aw_done_[aw_current_field_][f] = 1;
      AWFeedJob j{f, aw_current_field_, 0.0, 0.0};
      if (!psf_) {
        const auto b = pnt(r);
        const double ra0 = axes_.centre[0], dec0 = axes_.centre[1];
        j.l = std::sin(b.first - ra0) * std::cos(b.second);
        j.m = std::sin(b.second) * std::cos(dec0) - std::cos(b.second) * std::sin(dec0) * std::cos(b.first - ra0);
      }
      jobs.push_back(j);
    }
  }
  if (!jobs.empty()) {
    AWCFParams p;
    p.shape_x = nx_;
    p.shape_y = ny_;
    p.uvcell_u = uvcell_[0];
    p.uvcell_v = uvcell_[1];
    p.os = os_;
    p.maxsupport = maxsupport_;
    p.wterms.resize(ws_.nwplanes);
    for (int i = 0; i < ws_.nwplanes; ++i) p.wterms[i] = wterm_cf(i);
    p.cutoff = cutoff_;
    p.cutoff_abs = cutoff_abs_;
    p.limitsupport = limitsupport_;
    p.variablesupport = variablesupport_;
    p.offsetsupport = offsetsupport_;
    p.alpha = alpha_;
    p.diameter = diameter_;
    p.blockage = blockage_;
    p.maxfeeds = maxfeeds_;
    p.maxfields = maxfields_;
    p.nchan_cf = aw_nchan_;
    p.freqs.resize(aw_nchan_);
    for (int c = 0; c < aw_nchan_; ++c) p.freqs[c] = freqs[c];
    aw_cf_freqs_ = p.freqs;
    p.spheroidaltaper = aw_taper_;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, stream_);
    rc_check(cf_build_aw(cf_, p, jobs, cfwork_, stream_), "AWProject CF generation");
    cudaEventRecord(e1, stream_);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    stats_.time_cf_ms += ms;
    stats_.cf_generations += (double)jobs.size() * aw_nchan_ * ws_.nwplanes;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (!cf_built_) {
      cf_built_ = true;
      if (!model_empty_ && grids_.p && sumw_.bytes) {
        // AWProject sizes the sum of weights by its CF cache on the first build
        init_sumw();
      }
    }
  }
  throw_if(cf_.support <= 0, YG_ERR_SUPPORT, "Support not calculated correctly");
}

// ---------------------------------------------------------------------------
// binning
// ---------------------------------------------------------------------------
// the k_grid thread layout: the caller's, else the autotuner's for this CF
// width class, else the default
int Gridder::grid_variant() const {
  if (grid_mode_ > 0) return grid_mode_;
  TuneChoice c;
  const int smax = (cf_.maxsize - 1) / 2;
  if (tune_lookup(((2 * smax + 1) + 15) / 16 * 16, npol_, &c)) return c.variant;
  return 0;
}

int Gridder::tile_for(int smax, int npol) const {
  if (tile_override_ > 0) return tile_override_;
  TuneChoice c;
  if (tune_lookup(((2 * smax + 1) + 15) / 16 * 16, npol, &c) && c.tile > 0) return c.tile;
  return grid_tile_for(smax, npol, cf_.view().varsup != 0);
}

void Gridder::fill_bin_args(BinArgs& a, const Chunk& dc, const int* dchan_map, const uint8_t* row_ok) const {
  a = BinArgs{};
  a.nrow = dc.nrow;
  a.nchan = dc.nchan;
  a.npol = dc.npol;
  a.uvw = dc.uvw;
  a.freq = dc.freq;
  a.chan_map = dchan_map;
  a.flag = dc.flag;
  a.feed = dc.feed1;
  a.row_ok = row_ok;
  a.cellu = uvcell_[0];
  a.cellv = uvcell_[1];
  a.os = os_;
  a.nx = nx_;
  a.ny = ny_;
  a.ws = ws_;
  a.ws_stack = ws_stack_;
  switch (kind_) {
    case Kind::SphFunc: a.cf_mode = CF_MODE_SINGLE; a.grid_mode = GRID_MODE_SINGLE; break;
    case Kind::WStack: a.cf_mode = CF_MODE_SINGLE; a.grid_mode = GRID_MODE_WPLANE; break;
    case Kind::WProject: a.cf_mode = CF_MODE_WPLANE; a.grid_mode = GRID_MODE_SINGLE; break;
    case Kind::AWProject: a.cf_mode = CF_MODE_AW; a.grid_mode = GRID_MODE_SINGLE; break;
    case Kind::WStackWProject: a.cf_mode = CF_MODE_WSTACK_WPROJ; a.grid_mode = GRID_MODE_STACK; break;
  }
  a.aw_nchan = aw_nchan_ > 0 ? aw_nchan_ : 1;
  a.aw_maxfeeds = maxfeeds_;
  a.aw_field = aw_current_field_;
  a.nchan_img = nchan_;
  a.cf = cf_.view();
  const int smax = (a.cf.maxsize - 1) / 2;
  a.tile = tile_for(smax, dc.npol);
  // 16-wide CFs grid with residue rows modulo their real width (exact rows)
  // unless a layout of several slots per thread was asked for
  const int wpad16 = ((2 * smax + 1) + 15) / 16 * 16;
  // (the plane-major kernel keeps exact rows with every layout)
  a.wy = (wpad16 == 16 && ((grid_variant() & 15) <= 1 || (grid_variant() & 64)) && exact_rows_) ? 2 * smax + 1 : 0;
  a.pos_major = (grid_variant() & 64) ? 2 : ((grid_variant() & 32) ? 1 : 0);
  a.key_planes = 0;
  a.need_inv = 1;
  a.ntx = (nx_ + a.tile - 1) / a.tile;
  a.nty = (ny_ + a.tile - 1) / a.tile;
  int mb = 0;
  while ((1 << mb) < a.tile) ++mb;
  a.mbits = 2 * mb;
  int ngp = 1;
  if (a.grid_mode == GRID_MODE_WPLANE) ngp = ws_.nwplanes;
  if (a.grid_mode == GRID_MODE_STACK) ngp = ws_stack_.nwplanes;
  const unsigned long long ntiles = (unsigned long long)ngp * nchan_ * a.ntx * a.nty;
  a.invalid_key = (ntiles * (unsigned long long)a.cf.ncf) << a.mbits;
}

std::vector<uint8_t> Gridder::psf_rows(const Chunk& c) {
  std::vector<uint8_t> ok;
  const bool need_psf = psf_ && !alldatapsf_;
  const bool need_sep = max_pointing_sep_ > 0.;
  if (!need_psf && !need_sep) return ok;
  ok.assign(c.nrow, 1);
  std::vector<int> feed(c.nrow, 0);
  if (c.feed1) {
    if (c.on_device) cuda_check(cudaMemcpy(feed.data(), c.feed1, c.nrow * sizeof(int), cudaMemcpyDeviceToHost), "feed");
    else std::memcpy(feed.data(), c.feed1, c.nrow * sizeof(int));
  }
  for (long long r = 0; r < c.nrow; ++r) {
    const double ra = c.pointing ? c.pointing[2 * r] : axes_.centre[0];
    const double dec = c.pointing ? c.pointing[2 * r + 1] : axes_.centre[1];
    if (need_sep && separation(axes_.centre[0], axes_.centre[1], ra, dec) > max_pointing_sep_) {
      ok[r] = 0;
      continue;
    }
    if (need_psf) {
      if (first_psf_row_) {
        rep_feed_ = feed[r];
        rep_pointing_[0] = ra;
        rep_pointing_[1] = dec;
        first_psf_row_ = false;
      }
      if (!(feed[r] == rep_feed_ && separation(rep_pointing_[0], rep_pointing_[1], ra, dec) < 1e-6)) ok[r] = 0;
    }
  }
  return ok;
}

void Gridder::bin(const Chunk& dc, Plan& pl, cudaStream_t st, int use) {
  if (!st) st = stream_;
  throw_if(dc.npol != npol_, YG_ERR_UNSUPPORTED,
           "visibility and image polarisation frames must match (no polarisation conversion)");
  const std::vector<double> freqs = host_freqs(dc);
  if (dc.nchan > 0) {
    const double r = freqs[0] / kC;
    throw_if(!(r > 0.1 && r < 30000), YG_ERR_FREQ,
             "Check frequencies in the input file as the order of magnitude is likely to be wrong");
  }
  const std::vector<int> cmap = chan_map(freqs.data(), dc.nchan);
  cuda_check(pl.chanmap.ensure(std::max(1, dc.nchan) * sizeof(int)), "alloc");
  cuda_check(cudaMemcpyAsync(pl.chanmap.p, cmap.data(), dc.nchan * sizeof(int), cudaMemcpyHostToDevice, st), "up");
  std::vector<uint8_t> rows = psf_rows(dc);
  const uint8_t* row_ok = nullptr;
  if (!rows.empty()) {
    cuda_check(rowok_d_.ensure(rows.size()), "alloc");
    cuda_check(cudaMemcpyAsync(rowok_d_.p, rows.data(), rows.size(), cudaMemcpyHostToDevice, st), "up");
    row_ok = rowok_d_.as<uint8_t>();
  }
  BinArgs a;
  fill_bin_args(a, dc, pl.chanmap.as<int>(), row_ok);
  if (use == PLAN_DEGRID) a.pos_major = 0;
  // a gridding-only plan for the plane-major kernel sorts once, by its key
  const int wpad_b = ((cf_.maxsize + 15) / 16) * 16;
  a.key_planes = (use == PLAN_GRID && a.pos_major == 2 && wpad_b == 16 && a.wy > 0 && a.wy <= 16 &&
                  !cf_.view().varsup && dc.npol <= 4 && cf_form_ == 0)
                     ? 1
                     : 0;
  a.need_inv = (use != PLAN_DEGRID && !a.key_planes) ? 1 : 0;
  // samples per work item: enough items for ~8 per SM, never below 512
  int vmax = vmax_;
  TuneChoice tc;
  const int smax_b = (cf_.maxsize - 1) / 2;
  const bool tuned = tune_lookup(((2 * smax_b + 1) + 15) / 16 * 16, npol_, &tc);
  if (vmax <= 0 && tuned && tile_override_ <= 0) vmax = tc.vmax;
  if (vmax <= 0) {
    const long long n = dc.nrow * (long long)dc.nchan;
    vmax = (int)std::min<long long>(1 << 20, std::max<long long>(512, n / (148 * 8)));
  }
  rc_check(plan_build(pl, a, vmax, err_.as<DevError>(), st), "binning");
  check_error(st);
}

static VisArgs vis_args(const Chunk& dc, const float* mfs, bool psf, bool pcf = false) {
  VisArgs v;
  v.vis = dc.vis;
  v.noise = dc.noise;
  v.delay = dc.delay;
  v.mfs = mfs;
  v.freq = dc.freq;
  v.nrow = dc.nrow;
  v.nchan = dc.nchan;
  v.npol = dc.npol;
  v.psf = psf ? 1 : 0;
  v.psf_ok = nullptr;
  v.pcf = pcf ? 1 : 0;
  return v;
}

// ---------------------------------------------------------------------------
// grid / degrid
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// host chunks in row pieces: the next piece's upload (a copy stream) overlaps
// the binning and gridding of the current one; degridded pieces go back to
// the host while the next is degridded.  Row order is kept, so the result is
// that of one call (sums of weights, the carried value of off-grid samples).
// ---------------------------------------------------------------------------
bool Gridder::pipelined(const Chunk& c) const {
  const double bytes = (double)c.nrow * c.nchan * c.npol * sizeof(float2);
  return !c.on_device && kind_ != Kind::AWProject && !psf_ && bytes >= kPipeMinBytes && c.nrow >= 16;
}

Chunk Gridder::stage_rows(const Chunk& c, long long r0, long long nr, int b, bool need_vis) {
  Staging& s = staging_[b];
  cudaStream_t cs = copy_stream_;
  const size_t nrows = (size_t)nr;
  const size_t planes = (size_t)c.nchan * c.npol;
  auto up = [&](DevBuf& d, const void* src, size_t bytes) -> void* {
    if (!src) return nullptr;
    cuda_check(d.ensure(bytes), "alloc upload");
    cuda_check(cudaMemcpyAsync(d.p, src, bytes, cudaMemcpyHostToDevice, cs), "upload");
    return d.p;
  };
  auto up2 = [&](DevBuf& d, const void* src, size_t elem) -> void* {
    if (!src) return nullptr;
    cuda_check(d.ensure(nrows * planes * elem), "alloc upload");
    cuda_check(cudaMemcpy2DAsync(d.p, nrows * elem, (const char*)src + r0 * elem, (size_t)c.nrow * elem,
                                 nrows * elem, planes, cudaMemcpyHostToDevice, cs),
               "upload rows");
    return d.p;
  };
  // the buffers' last piece may still be going back to the host
  if (piece_down_[b]) cuda_check(cudaStreamWaitEvent(cs, piece_down_[b], 0), "wait download");
  Chunk dc = c;
  dc.nrow = nr;
  dc.uvw = (const double*)up(s.uvw, c.uvw + 3 * r0, nrows * 3 * sizeof(double));
  dc.delay = c.delay ? (const double*)up(s.delay, c.delay + r0, nrows * sizeof(double)) : nullptr;
  dc.freq = (const double*)up(s.freq, c.freq, (size_t)c.nchan * sizeof(double));
  dc.vis = need_vis ? (float2*)up2(s.vis, c.vis, sizeof(float2)) : nullptr;
  dc.noise = (const float2*)up2(s.noise, c.noise, sizeof(float2));
  dc.flag = (const uint8_t*)up2(s.flag, c.flag, 1);
  dc.feed1 = c.feed1 ? (const int*)up(s.feed, c.feed1 + r0, nrows * sizeof(int)) : nullptr;
  dc.pointing = c.pointing ? c.pointing + 2 * r0 : nullptr;
  dc.host_freq = c.freq;
  dc.on_device = 1;
  if (!piece_up_[b]) cuda_check(cudaEventCreateWithFlags(&piece_up_[b], cudaEventDisableTiming), "event");
  cuda_check(cudaEventRecord(piece_up_[b], cs), "event");
  return dc;
}

void Gridder::run_pieces(Chunk& c, bool degridding) {
  auto stream = [&](cudaStream_t& cs) {
    if (!cs) cuda_check(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking), "stream");
  };
  auto event = [&](cudaEvent_t& e) {
    if (!e) cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
  };
  stream(copy_stream_);
  stream(bin_stream_);
  if (degridding) stream(down_stream_);
  for (auto& e : piece_down_) event(e);
  for (auto& e : piece_pass_) event(e);
  event(piece_binned_);
  const double bytes = (double)c.nrow * c.nchan * c.npol * sizeof(float2);
  const int K = (int)std::max(2.0, std::min(16.0, std::ceil(bytes / kPipePieceBytes)));
  const long long rows = (c.nrow + K - 1) / K;
  const int npieces = (int)((c.nrow + rows - 1) / rows);
  // Each piece: upload (copy stream) -> binning (bin stream; the host waits
  // for its item count) -> pass (the gridder's stream) -> download (degrid,
  // its own stream).  Piece k + 1 is uploaded and binned while the pass over
  // piece k runs; a staging buffer and its plan are reused once the pass two
  // pieces back (and its download) is done.  Passes stay in row order on one
  // stream, so sums of weights and the carried value of off-grid samples are
  // those of one call; device errors are read once at the end.
  std::vector<Chunk> staged(2);
  auto stage_and_bin = [&](int k) {
    const int b = k & 1;
    const long long r0 = k * rows;
    cuda_check(cudaStreamWaitEvent(copy_stream_, piece_pass_[b], 0), "wait pass");
    staged[b] = stage_rows(c, r0, std::min(rows, c.nrow - r0), b, true);
    cuda_check(cudaStreamWaitEvent(bin_stream_, piece_up_[b], 0), "wait upload");
    cuda_check(cudaStreamWaitEvent(bin_stream_, piece_pass_[b], 0), "wait pass");
    init_cf(staged[b]);
    bin(staged[b], piece_plan_[b], bin_stream_, degridding ? PLAN_DEGRID : PLAN_GRID);
    cuda_check(cudaEventRecord(piece_binned_, bin_stream_), "event");
  };
  // no pass has used the buffers yet: their pass events complete at once
  for (auto& e : piece_pass_) cuda_check(cudaEventRecord(e, stream_), "event");
  stage_and_bin(0);
  for (int k = 0; k < npieces; ++k) {
    const int b = k & 1;
    const long long r0 = k * rows, nr = std::min(rows, c.nrow - r0);
    Chunk& dc = staged[b];
    Plan& pl = piece_plan_[b];
    cuda_check(cudaStreamWaitEvent(stream_, piece_binned_, 0), "wait binning");
    const float* mfs = mfs_weights(dc);
    const double w = 2.0 * cf_.support + 1.0;
    if (degridding) {
      degrid_enqueue(dc, pl, mfs, stream_);
      stats_.samples_degridded += (double)pl.nvalid * dc.npol;
      stats_.taps_degridded += (double)pl.nvalid * dc.npol * w * w;
    } else {
      grid_enqueue(dc, pl, mfs, stream_);
      stats_.samples_gridded += (double)pl.nvalid * dc.npol;
      stats_.taps_gridded += (double)pl.nvalid * dc.npol * w * w;
    }
    cuda_check(cudaEventRecord(piece_pass_[b], stream_), "event");
    if (degridding) {
      // the download runs on a stream of its own, beside the next upload
      cuda_check(cudaStreamWaitEvent(down_stream_, piece_pass_[b], 0), "wait degrid");
      cuda_check(cudaMemcpy2DAsync((char*)c.vis + r0 * sizeof(float2), (size_t)c.nrow * sizeof(float2), dc.vis,
                                   (size_t)nr * sizeof(float2), (size_t)nr * sizeof(float2),
                                   (size_t)c.nchan * c.npol, cudaMemcpyDeviceToHost, down_stream_),
                 "download rows");
      cuda_check(cudaEventRecord(piece_down_[b], down_stream_), "event");
    }
    if (k + 1 < npieces) stage_and_bin(k + 1);
  }
  check_error();
  cuda_check(cudaStreamSynchronize(copy_stream_), "pieces");
  if (degridding) cuda_check(cudaStreamSynchronize(down_stream_), "pieces");
}

void Gridder::grid(const Chunk& c) {
  throw_if(nx_ == 0 || !grids_.p, YG_ERR_STATE, "initialiseGrid must be called before grid");
  throw_if(!sumw_.p, YG_ERR_STATE, "SumWeights not yet initialised");
  if (pipelined(c)) {
    ensure_device();
    Chunk cc = c;
    run_pieces(cc, false);
    return;
  }
  Chunk dc;
  upload_chunk(c, dc, !psf_, false);
  if (!c.on_device) dc.pointing = c.pointing;
  init_cf(dc);
  Plan& pl = plan_;
  bin(dc, pl, nullptr, PLAN_GRID);
  grid_plan(dc, pl);
}

// MFS weights of the chunk's channels on the device (null without MFS); made
// again only when the frequencies or the MFS order change.
const float* Gridder::mfs_weights(const Chunk& dc) {
  if (!mfs_) return nullptr;
  const std::vector<double> f = host_freqs(dc);
  if (f == mfs_freqs_ && mfs_key_order_ == mfs_order_ && mfs_key_ref_ == mfs_reffreq_ && mfs_d_.p)
    return mfs_d_.as<float>();
  mfs_w_.resize(dc.nchan);
  for (int i = 0; i < dc.nchan; ++i) {
    const double ratio = (f[i] - mfs_reffreq_) / mfs_reffreq_;
    mfs_w_[i] = mfs_order_ == 0 ? 1.0f : (mfs_order_ == 1 ? (float)ratio : (mfs_order_ == 2 ? (float)(ratio * ratio) : (float)std::pow(ratio, mfs_order_)));
  }
  cuda_check(mfs_d_.ensure(dc.nchan * sizeof(float)), "alloc");
  // the host vector stays alive in the gridder until the copy has run
  cuda_check(cudaMemcpyAsync(mfs_d_.p, mfs_w_.data(), dc.nchan * sizeof(float), cudaMemcpyHostToDevice, stream_), "up");
  cuda_check(cudaStreamSynchronize(stream_), "up");
  mfs_freqs_ = f;
  mfs_key_order_ = mfs_order_;
  mfs_key_ref_ = mfs_reffreq_;
  return mfs_d_.as<float>();
}

// The kernels of one grid pass over a plan, enqueued on st with no host
// synchronisation and no allocation once the buffers have their size (the
// part of grid_plan that a CUDA graph records).
void Gridder::grid_enqueue(const Chunk& dc, const Plan& pl, const float* mfs, cudaStream_t st, cudaEvent_t k0,
                           cudaEvent_t k1) {
  VisArgs v = vis_args(dc, mfs, psf_, pcf_);
  // the preconditioner function adds nothing to the sums of weights
  const SumwArgs sw{pcf_ ? nullptr : sumw_.as<double>(), pl.chanmap.as<int>(), os_, track_per_os_ ? 1 : 0,
                    nsumw_rows_, nchan_};
  const LearnedCF lcf = learned_view_for(dc, const_cast<Plan&>(pl));
  rc_check(plan_grid(pl, v, cf_.view(), grids_.as<float2>(), nx_, ny_, nchan_, sw, scratch_, svis_,
                     err_.as<DevError>(), st, k0, k1, grid_variant(), cf_form_ != 0 ? &lcf : nullptr),
           "gridding");
  rc_check(plan_grid_carry(const_cast<Plan&>(pl), v, carry_.as<float2>(), st), "carry");
}

void Gridder::grid_plan(const Chunk& dc, const Plan& pl) {
  throw_if(!grids_.p || nx_ == 0, YG_ERR_STATE, "initialiseGrid must be called before grid");
  if (kind_ != Kind::AWProject) build_cf();
  throw_if(!cf_built_, YG_ERR_STATE, "convolution functions are not built");
  const float* mfs = mfs_weights(dc);
  cudaEvent_t e0, e1, k0, k1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventCreate(&k0);
  cudaEventCreate(&k1);
  cudaEventRecord(e0, stream_);
  grid_enqueue(dc, pl, mfs, stream_, k0, k1);
  cudaEventRecord(e1, stream_);
  check_error();
  float ms = 0, kms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  if (pl.nitems > 0 && cudaEventElapsedTime(&kms, k0, k1) == cudaSuccess) {
    stats_.kgrid_ms += kms;
    stats_.kgrid_calls += 1;
  }
  cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaEventDestroy(k0);
  cudaEventDestroy(k1);
  stats_.time_grid_ms += ms;
  stats_.samples_gridded += (double)pl.nvalid * dc.npol;
  const double w = 2.0 * cf_.support + 1.0;
  stats_.taps_gridded += (double)pl.nvalid * dc.npol * w * w;
}

void Gridder::degrid(Chunk& c) {
  throw_if(psf_, YG_ERR_STATE, "the gridder is not supposed to be used for degridding in the PSF mode");
  throw_if(pcf_, YG_ERR_STATE, "the gridder is not supposed to be used for degridding in the PCF mode");
  if (model_empty_) return;
  throw_if(nx_ == 0 || !grids_.p, YG_ERR_STATE, "initialiseDegrid must be called before degrid");
  if (pipelined(c)) {
    ensure_device();
    run_pieces(c, true);
    return;
  }
  Chunk dc;
  upload_chunk(c, dc, true, true);
  if (!c.on_device) dc.pointing = c.pointing;
  init_cf(dc);
  Plan& pl = plan_;
  bin(dc, pl, nullptr, PLAN_DEGRID);
  degrid_plan(dc, pl);
  if (!c.on_device) {
    const size_t bytes = (size_t)c.nrow * c.nchan * c.npol * sizeof(float2);
    cuda_check(cudaMemcpyAsync(c.vis, dc.vis, bytes, cudaMemcpyDeviceToHost, stream_), "download vis");
    sync();
  }
}

// The kernels of one degrid pass over a plan on st (see grid_enqueue).
void Gridder::degrid_enqueue(Chunk& dc, Plan& pl, const float* mfs, cudaStream_t st, cudaEvent_t k0,
                             cudaEvent_t k1, bool alone) {
  VisArgs v = vis_args(dc, mfs, false);
  const LearnedCF lcf = learned_view_for(dc, pl);
  rc_check(plan_degrid(pl, v, dc.vis, cf_.view(), grids_.as<float2>(), nx_, ny_, nchan_, pl.chanmap.as<int>(), tmpvals_,
                       carry_.as<float2>(), err_.as<DevError>(), st, k0, k1, cf_form_ != 0 ? &lcf : nullptr,
                       grid_variant(), alone),
           "degridding");
}

void Gridder::degrid_plan(Chunk& dc, Plan& pl) {
  throw_if(!grids_.p || nx_ == 0, YG_ERR_STATE, "initialiseDegrid must be called before degrid");
  if (kind_ != Kind::AWProject) build_cf();
  throw_if(!cf_built_, YG_ERR_STATE, "convolution functions are not built");
  const float* mfs = mfs_weights(dc);
  cudaEvent_t e0, e1, k0, k1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventCreate(&k0);
  cudaEventCreate(&k1);
  cudaEventRecord(e0, stream_);
  degrid_enqueue(dc, pl, mfs, stream_, k0, k1);
  cudaEventRecord(e1, stream_);
  check_error();
  float ms = 0, kms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  if (pl.nitems > 0 && cudaEventElapsedTime(&kms, k0, k1) == cudaSuccess) {
    stats_.kdegrid_ms += kms;
    stats_.kdegrid_calls += 1;
  }
  cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaEventDestroy(k0);
  cudaEventDestroy(k1);
  stats_.time_degrid_ms += ms;
  stats_.samples_degridded += (double)pl.nvalid * dc.npol;
  const double w = 2.0 * cf_.support + 1.0;
  stats_.taps_degridded += (double)pl.nvalid * dc.npol * w * w;
}

// ---------------------------------------------------------------------------
// finalise / initialise degrid
// ---------------------------------------------------------------------------
void Gridder::prepare_corrections() {
  // SphFuncVisGridder::correctConvolution factors for the padded shape; the
  // AWProject gridder applies them only with a spheroidal taper
  // (AWProjectVisGridder::correctConvolution).
  if (kind_ == Kind::AWProject && !aw_taper_) {
    corr_d_.release();
    return;
  }
  const int support = (kind_ == Kind::SphFunc) ? sph_support_ : 3;
  Spheroidal g(M_PI * support, alpha_);
  std::vector<double> cx = sph_correction(nx_, g), cy = sph_correction(ny_, g);
  cuda_check(corr_d_.ensure((nx_ + ny_) * sizeof(double)), "alloc");
  cuda_check(cudaMemcpy(corr_d_.p, cx.data(), nx_ * sizeof(double), cudaMemcpyHostToDevice), "up");
  cuda_check(cudaMemcpy(corr_d_.as<double>() + nx_, cy.data(), ny_ * sizeof(double), cudaMemcpyHostToDevice), "up");
}

static void extract_centre(const float* src, int snx, int sny, int nplanes, float* dst, int dnx, int dny, bool dst_dev,
                           cudaStream_t st) {
  const int x0 = (snx - dnx) / 2, y0 = (sny - dny) / 2;
  for (int p = 0; p < nplanes; ++p) {
    const float* s = src + (size_t)p * snx * sny + x0 + (size_t)snx * y0;
    float* d = dst + (size_t)p * dnx * dny;
    cuda_check(cudaMemcpy2DAsync(d, dnx * sizeof(float), s, snx * sizeof(float), dnx * sizeof(float), dny,
                                 dst_dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st),
               "extract");
  }
}

void Gridder::finalise_grid(float* out, bool out_on_device) {
  throw_if(!grids_.p || nx_ == 0, YG_ERR_STATE, "finaliseGrid called before gridding");
  prepare_corrections();
  const int nplanes = npol_ * nchan_;
  const long long total = (long long)nx_ * ny_ * nplanes;
  cuda_check(img_tmp_.ensure(total * sizeof(float)), "alloc");
  std::vector<StackScreen> screens;
  const std::vector<StackScreen>* sp = nullptr;
  if (kind_ == Kind::WStack || kind_ == Kind::WStackWProject) {
    const WSampling& s = (kind_ == Kind::WStack) ? ws_ : ws_stack_;
    for (int i = 0; i < s.nwplanes; ++i) screens.push_back(make_stack_screen(nx_, ny_, uvcell_[0], uvcell_[1], wterm_of(s, i)));
    sp = &screens;
  }
  const double* cx = corr_d_.p ? corr_d_.as<double>() : nullptr;
  const double* cy = corr_d_.p ? corr_d_.as<double>() + nx_ : nullptr;
  rc_check(image_finalise(fft_, grids_.as<float2>(), ngrids(), nx_, ny_, nplanes, sp, cx, cy, img_tmp_.as<float>(),
                          stream_),
           "finaliseGrid");
  const int onx = (int)std::lround(nx_ / padding_), ony = (int)std::lround(ny_ / padding_);
  extract_centre(img_tmp_.as<float>(), nx_, ny_, nplanes, out, onx, ony, out_on_device, stream_);
  sync();
  if (clear_grids_) grids_.release();
}

void Gridder::finalise_weights(float* out, bool out_on_device) {
  throw_if(!sumw_.p, YG_ERR_STATE, "Sum of weights not yet initialised");
  std::vector<double> sw;
  int rows = 0;
  sum_weights(sw, &rows);
  const int onx = (int)std::lround(nx_ / padding_), ony = (int)std::lround(ny_ / padding_);
  if (kind_ == Kind::AWProject) {
    throw_if(!cf_built_, YG_ERR_STATE, "AWProject finaliseWeights needs the convolution functions of the gridding");
    const int np = npol_ * nchan_;
    std::vector<int> planes;
    std::vector<int2> offs;
    std::vector<double> wts;
    for (int z = 0; z < rows; ++z) {
      bool data = false;
      for (int q = 0; q < np; ++q) data = data || sw[z + (size_t)rows * q] > 0.0;
      if (!data) continue;
      planes.push_back(track_per_os_ ? z : os_ * os_ * z);
      offs.push_back(z < (int)cf_.h_offsets.size() ? cf_.h_offsets[z] : make_int2(0, 0));
      for (int q = 0; q < np; ++q) wts.push_back(sw[z + (size_t)rows * q]);
    }
    const int cnx = std::min(maxsupport_, nx_), cny = std::min(maxsupport_, ny_);
    DevBuf dout;
    float* dst = out;
    if (!out_on_device) {
      cuda_check(dout.ensure((size_t)onx * ony * np * sizeof(float)), "alloc");
      dst = dout.as<float>();
    }
    // the CFs' spheroidal taper over the weights grid, values at or below
    // spheroidalweightscutoff set to zero (AWProjectVisGridder.cc:641-664)
    std::vector<double> taper;
    if (aw_taper_) {
      Spheroidal grdsf(M_PI * 3, alpha_);
      taper.resize(cnx + cny);
      for (int k = 0; k < 2; ++k) {
        const int n = k ? cny : cnx, c = n / 2;
        double* f = taper.data() + (k ? cnx : 0);
        for (int i = 0; i < n; ++i) {
          const double val = grdsf(std::fabs((double)i - (double)c) / (double)c);
          f[i] = val > aw_weights_cutoff_ ? val : 0.0;
        }
        if (n > 3) {
          f[0] = 3.0 * (f[1] - f[2]) + f[3];
          if (n % 2 == 1) f[n - 1] = f[0];
        }
      }
    }
    rc_check(aw_weights_image(cf_.view(), planes, offs, wts, np, cnx, cny, nx_, ny_, onx, ony, dst, stream_,
                              aw_taper_ ? &taper : nullptr),
             "AWProject weights");
    if (!out_on_device)
      cuda_check(cudaMemcpy(out, dst, (size_t)onx * ony * np * sizeof(float), cudaMemcpyDeviceToHost), "weights");
    return;
  }
  std::vector<float> h((size_t)onx * ony * npol_ * nchan_);
  for (int c = 0; c < nchan_; ++c)
    for (int p = 0; p < npol_; ++p) {
      double s = 0.0;
      for (int z = 0; z < rows; ++z) s += sw[z + (size_t)rows * (p + (size_t)npol_ * c)];
      std::fill(h.begin() + (size_t)(p + npol_ * c) * onx * ony, h.begin() + (size_t)(p + npol_ * c + 1) * onx * ony,
                (float)s);
    }
  if (out_on_device) cuda_check(cudaMemcpy(out, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice), "weights");
  else std::memcpy(out, h.data(), h.size() * sizeof(float));
}

void Gridder::initialise_degrid(const Axes& axes, int nx, int ny, int npol, int nchan, const float* image,
                                bool on_device) {
  ensure_device();
  init_axes(axes, nx, ny, npol, nchan);
  psf_ = false;
  pcf_ = false;
  const int nplanes = npol * nchan;
  const long long in_total = (long long)nx * ny * nplanes;
  const long long total = (long long)nx_ * ny_ * nplanes;
  // model emptiness check on the host copy (or a device download)
  std::vector<float> h;
  const float* hp = image;
  if (on_device) {
    h.resize(in_total);
    cuda_check(cudaMemcpy(h.data(), image, in_total * sizeof(float), cudaMemcpyDeviceToHost), "download model");
    hp = h.data();
  }
  bool empty = true;
  for (long long i = 0; i < in_total; ++i)
    if (std::fabs(hp[i]) > 0.f) { empty = false; break; }
  model_empty_ = empty;
  const size_t gbytes = (size_t)ngrids() * total * sizeof(float2);
  cuda_check(grids_.ensure(gbytes), "alloc grids");
  if (empty) {
    cuda_check(cudaMemsetAsync(grids_.p, 0, gbytes, stream_), "memset");
    sync();
    return;
  }
  // padded model on the device
  cuda_check(img_tmp_.ensure(total * sizeof(float) * 2), "alloc");
  float* padded = img_tmp_.as<float>();
  float* corrected = padded + total;
  cuda_check(cudaMemsetAsync(padded, 0, total * sizeof(float), stream_), "memset");
  const int x0 = (nx_ - nx) / 2, y0 = (ny_ - ny) / 2;
  for (int p = 0; p < nplanes; ++p) {
    cuda_check(cudaMemcpy2DAsync(padded + (size_t)p * nx_ * ny_ + x0 + (size_t)nx_ * y0, nx_ * sizeof(float),
                                 image + (size_t)p * nx * ny, nx * sizeof(float), nx * sizeof(float), ny,
                                 on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, stream_),
               "upload model");
  }
  prepare_corrections();
  std::vector<StackScreen> screens;
  const std::vector<StackScreen>* sp = nullptr;
  if (kind_ == Kind::WStack || kind_ == Kind::WStackWProject) {
    const WSampling& s = (kind_ == Kind::WStack) ? ws_ : ws_stack_;
    for (int i = 0; i < s.nwplanes; ++i) screens.push_back(make_stack_screen(nx_, ny_, uvcell_[0], uvcell_[1], wterm_of(s, i)));
    sp = &screens;
  }
  const double* cx = corr_d_.p ? corr_d_.as<double>() : nullptr;
  const double* cy = corr_d_.p ? corr_d_.as<double>() + nx_ : nullptr;
  rc_check(image_to_grids(fft_, padded, nx_, ny_, nplanes, sp, ngrids(), cx, cy, corrected, grids_.as<float2>(),
                          stream_),
           "initialiseDegrid");
  sync();
}

void Gridder::finalise_degrid() {
  if (clear_grids_) grids_.release();
}

void Gridder::cf_data(std::vector<float2>& out) const { rc_check(cf_.download(out), "cf download"); }

void Gridder::sum_weights(std::vector<double>& out, int* nrows) const {
  *nrows = nsumw_rows_;
  out.resize((size_t)nsumw_rows_ * npol_ * nchan_);
  if (stream_) cudaStreamSynchronize(stream_);
  if (sumw_.p) cuda_check(cudaMemcpy(out.data(), sumw_.p, out.size() * sizeof(double), cudaMemcpyDeviceToHost), "sumw");
}

void Gridder::grid_data(std::vector<float2>& out) const {
  out.resize((size_t)ngrids() * grid_elems());
  if (stream_) cudaStreamSynchronize(stream_);
  if (grids_.p) cuda_check(cudaMemcpy(out.data(), grids_.p, out.size() * sizeof(float2), cudaMemcpyDeviceToHost), "grid");
}

}  // namespace yg

namespace yg {
void Gridder::plan_samples(const Plan& pl, int* iu, int* iv, int* cfi, unsigned char* status) const {
  const long long n = pl.nsamples;
  if (n == 0) return;
  std::vector<unsigned int> pos(n);
  cuda_check(cudaMemcpy(pos.data(), pl.pos.p, n * 4, cudaMemcpyDeviceToHost), "pos");
  for (long long i = 0; i < n; ++i) {
    iu[i] = (int)(pos[i] & 0xffffu);
    iv[i] = (int)(pos[i] >> 16);
  }
  cuda_check(cudaMemcpy(cfi, pl.cfi.p, n * 4, cudaMemcpyDeviceToHost), "cfi");
  cuda_check(cudaMemcpy(status, pl.status.p, n, cudaMemcpyDeviceToHost), "status");
}
}  // namespace yg

namespace yg {

// ---------------------------------------------------------------------------
// learned convolution function
// ---------------------------------------------------------------------------
LearnedCF Gridder::learned_view() const {
  LearnedCF L{};
  if (!net_.ready || !wterm_d_.p) return L;
  L.w16 = net_.w16.as<__half>();
  L.wterm = wterm_d_.as<double>();
  L.wnorm = learn_wnorm_;
  L.fb = fb_d_.p ? fb_d_.as<float2>() : nullptr;
  L.scale = net_.scale;
  L.os = os_;
  return L;
}

// The view for one grid or degrid call: the continuous form (2) also needs the
// plan's per-sample inputs, made once per plan.
LearnedCF Gridder::learned_view_for(const Chunk& dc, Plan& pl) {
  LearnedCF L = learned_view();
  if (cf_form_ != 2 || !L.w16) return L;
  const double* wstack = nullptr;
  if (kind_ == Kind::WStackWProject) {
    if (!wstack_d_.p) {
      std::vector<double> w(ws_stack_.nwplanes);
      for (int g = 0; g < ws_stack_.nwplanes; ++g) w[g] = wterm_of(ws_stack_, g);
      cuda_check(wstack_d_.ensure(w.size() * sizeof(double)), "alloc");
      cuda_check(cudaMemcpyAsync(wstack_d_.p, w.data(), w.size() * sizeof(double), cudaMemcpyHostToDevice, stream_),
                 "up");
    }
    wstack = wstack_d_.as<double>();
  }
  rc_check(plan_learned_inputs(pl, dc.uvw, dc.freq, uvcell_[0], uvcell_[1], os_, nchan_, wstack, learn_wnorm_,
                               stream_),
           "continuous CF inputs");
  L.ext = pl.ext.as<float4>();
  return L;
}

size_t Gridder::cf_table_bytes() const {
  return (size_t)cf_.total * sizeof(float2) + cf_.pad.bytes;
}

// Trains the network on this gridder's tabulated CFs, or (nw_train > its
// plane count) on a denser table of nw_train planes spread linearly over the
// same w range, built on the GPU for the purpose and released afterwards.
void Gridder::upload_learn_tables() {
  ensure_device();
  cuda_check(wterm_d_.ensure(learn_wterm_h_.size() * sizeof(double)), "alloc");
  cuda_check(fb_d_.ensure(learn_fb_h_.size() * sizeof(float2)), "alloc");
  cuda_check(cudaMemcpy(wterm_d_.p, learn_wterm_h_.data(), learn_wterm_h_.size() * sizeof(double),
                        cudaMemcpyHostToDevice), "up");
  cuda_check(cudaMemcpy(fb_d_.p, learn_fb_h_.data(), learn_fb_h_.size() * sizeof(float2), cudaMemcpyHostToDevice),
             "up");
}

// AWProject: the network learns every CF plane of the cache, plane z = w-plane
// + nw (channel + nchan beam) with inputs (w term / wmax, frequency, beam), the
// last two mapped linearly onto [-1, 1] over the cache's channels and beams.
// It trains on the gridder's own cache (every beam of the one field must have
// its CFs), not on a denser table.
void Gridder::learned_train_aw(const LearnParams& lp, LearnReport* rep) {
  throw_if(!cf_built_, YG_ERR_STATE, "AWProject learns its CFs after they are built (grid or degrid first)");
  throw_if(maxfields_ != 1, YG_ERR_UNSUPPORTED, "the learned AWProject CF covers one field");
  for (int f = 0; f < maxfeeds_; ++f)
    throw_if(!aw_done_[0][f], YG_ERR_STATE, "the learned AWProject CF needs the CFs of every beam (maxfeeds)");
  if (!net_.ready) rc_check(net_.init(mlp_initial_params(lp.seed), stream_), "network set-up");
  const int nw = ws_.nwplanes, nc = aw_nchan_, nf = maxfeeds_;
  double wn = 0.0;
  for (int i = 0; i < nw; ++i) wn = std::max(wn, std::fabs(wterm_cf(i)));
  learn_wnorm_ = wn > 0.0 ? wn : 1.0;
  double f0 = 0.0, f1 = 0.0;
  throw_if((int)aw_cf_freqs_.size() < nc, YG_ERR_STATE, "AWProject CF frequencies unknown");
  if (nc > 1) {
    f0 = *std::min_element(aw_cf_freqs_.begin(), aw_cf_freqs_.begin() + nc);
    f1 = *std::max_element(aw_cf_freqs_.begin(), aw_cf_freqs_.begin() + nc);
  }
  learn_wterm_h_.assign((size_t)nw * nc * nf, 0.0);
  learn_fb_h_.assign((size_t)nw * nc * nf, make_float2(0.f, 0.f));
  for (int b = 0; b < nf; ++b)
    for (int c = 0; c < nc; ++c)
      for (int i = 0; i < nw; ++i) {
        const size_t z = (size_t)i + (size_t)nw * (c + (size_t)nc * b);
        learn_wterm_h_[z] = wterm_cf(i);
        const float fx = f1 > f0 ? (float)(2.0 * (aw_cf_freqs_[c] - f0) / (f1 - f0) - 1.0) : 0.f;
        const float bx = nf > 1 ? (float)(2.0 * b / (double)(nf - 1) - 1.0) : 0.f;
        learn_fb_h_[z] = make_float2(fx, bx);
      }
  upload_learn_tables();
  rc_check(net_.train(cf_.view(), wterm_d_.as<double>(), learn_wnorm_, os_, lp, learn_X_, learn_T_, stream_, rep,
                      fb_d_.as<float2>()),
           "training");
  learn_X_.release();
  learn_T_.release();
}

void Gridder::learned_train(const LearnParams& lp, int nw_train, LearnReport* rep) {
  throw_if(variablesupport_ || offsetsupport_, YG_ERR_UNSUPPORTED,
           "the learned CF needs one common support without offsets");
  if (kind_ == Kind::AWProject) {
    learned_train_aw(lp, rep);
    return;
  }
  throw_if(kind_ != Kind::WProject && kind_ != Kind::WStackWProject, YG_ERR_UNSUPPORTED,
           "the learned CF covers the W-projection gridders (WProject, WStackWProject) and AWProject");
  build_cf();
  if (!net_.ready) rc_check(net_.init(mlp_initial_params(lp.seed), stream_), "network set-up");
  const int nw = ws_.nwplanes;
  std::vector<double> wt(nw);
  for (int i = 0; i < nw; ++i) wt[i] = wterm_cf(i);
  double wn = 0.0;
  for (double w : wt) wn = std::max(wn, std::fabs(w));
  learn_wnorm_ = wn > 0.0 ? wn : 1.0;
  cuda_check(wterm_d_.ensure(nw * sizeof(double)), "alloc");
  cuda_check(cudaMemcpyAsync(wterm_d_.p, wt.data(), nw * sizeof(double), cudaMemcpyHostToDevice, stream_), "up");
  if (nw_train > nw && nw_train > 1) {
    CFCacheDev dense;
    WProjCFParams p;
    p.shape_x = nx_;
    p.shape_y = ny_;
    p.uvcell_u = uvcell_[0];
    p.uvcell_v = uvcell_[1];
    p.os = os_;
    p.maxsupport = maxsupport_;
    p.wterms.resize(nw_train);
    const double w0 = wt.front(), w1 = wt.back();
    for (int i = 0; i < nw_train; ++i) p.wterms[i] = w0 + (w1 - w0) * (double)i / (double)(nw_train - 1);
    p.cutoff = cutoff_;
    p.cutoff_abs = cutoff_abs_;
    p.limitsupport = limitsupport_;
    p.variablesupport = false;
    p.offsetsupport = false;
    p.alpha = alpha_;
    rc_check(cf_build_wproject(dense, p, cfwork_, stream_), "dense CF table");
    cfwork_.release();
    throw_if(dense.support != cf_.support, YG_ERR_STATE, "dense CF table has another support");
    DevBuf wd;
    cuda_check(wd.ensure(nw_train * sizeof(double)), "alloc");
    cuda_check(cudaMemcpyAsync(wd.p, p.wterms.data(), nw_train * sizeof(double), cudaMemcpyHostToDevice, stream_),
               "up");
    rc_check(net_.train(dense.view(), wd.as<double>(), learn_wnorm_, os_, lp, learn_X_, learn_T_, stream_, rep),
             "training");
    sync();
  } else {
    rc_check(net_.train(cf_.view(), wterm_d_.as<double>(), learn_wnorm_, os_, lp, learn_X_, learn_T_, stream_, rep),
             "training");
  }
  learn_X_.release();
  learn_T_.release();
}

void Gridder::set_cf_form(int form) {
  throw_if(form < 0 || form > 2, YG_ERR_ARG,
           "CF form must be 0 (tabulated), 1 (learned, tabulated planes) or 2 (learned, continuous)");
  throw_if(form != 0 && (!net_.ready || !wterm_d_.p), YG_ERR_STATE, "the learned CF has not been trained");
  throw_if(form == 2 && kind_ == Kind::AWProject, YG_ERR_UNSUPPORTED,
           "the continuous learned CF covers the W-projection gridders; AWProject takes form 1");
  cf_form_ = form;
}

void Gridder::learned_params(std::vector<float>& out) const {
  throw_if(!net_.ready, YG_ERR_STATE, "the learned CF has not been trained");
  out.resize(kMlpParams);
  cuda_check(cudaMemcpyAsync(out.data(), net_.p.p, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost, stream_),
             "download");
  cuda_check(cudaStreamSynchronize(stream_), "sync");
}

void Gridder::set_learned_params(const float* p, float scale) {
  ensure_device();
  std::vector<float> v(p, p + kMlpParams);
  rc_check(net_.init(v, stream_), "network set-up");
  net_.scale = scale;
  if (!wterm_d_.p && (kind_ == Kind::WProject || kind_ == Kind::WStackWProject)) {
    const int nw = ws_.nwplanes;
    std::vector<double> wt(nw);
    double wn = 0.0;
    for (int i = 0; i < nw; ++i) {
      wt[i] = wterm_cf(i);
      wn = std::max(wn, std::fabs(wt[i]));
    }
    learn_wnorm_ = wn > 0.0 ? wn : 1.0;
    cuda_check(wterm_d_.ensure(nw * sizeof(double)), "alloc");
    cuda_check(cudaMemcpyAsync(wterm_d_.p, wt.data(), nw * sizeof(double), cudaMemcpyHostToDevice, stream_), "up");
  }
  sync();
}

}  // namespace yg

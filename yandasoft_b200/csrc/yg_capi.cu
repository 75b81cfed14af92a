// extern "C" boundary of the B200 gridder: translates between the plain C
// structures of include/yg.h and the C++ Gridder, and turns exceptions into
// status codes plus a thread-local message (the reference's ASKAPCHECK /
// AskapError convention, askap/gridding/*.cc).
#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>
#include <new>
#include <string>

#include "../../include/yg.h"
#include "yg_cycle.h"
#include "yg_gridder.h"
#include "yg_sort.h"

struct yg_gridder {
  std::unique_ptr<yg::Gridder> g;
};

struct yg_plan {
  yg::Plan pl;
};

struct yg_cycle {
  yg::CycleBatch b;
};

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

template <typename F>
int guarded(F&& f) {
  try {
    f();
    g_last_error.clear();
    return YG_OK;
  } catch (const yg::YgError& e) {
    return fail(e.code, e.msg);
  } catch (const std::bad_alloc&) {
    return fail(YG_ERR_NOMEM, "out of host memory");
  } catch (const std::exception& e) {
    return fail(YG_ERR_ARG, e.what());
  } catch (...) {
    return fail(YG_ERR_ARG, "unknown error");
  }
}

yg::Axes to_axes(const yg_axes* a) {
  yg::Axes x;
  if (!a) throw yg::YgError{YG_ERR_ARG, "axes must not be NULL"};
  x.cell[0] = a->cell[0];
  x.cell[1] = a->cell[1];
  x.centre[0] = a->centre[0];
  x.centre[1] = a->centre[1];
  x.tangent[0] = a->tangent[0];
  x.tangent[1] = a->tangent[1];
  x.has_freq = a->has_freq;
  x.freq_start = a->freq_start;
  x.freq_end = a->freq_end;
  return x;
}

yg::Chunk to_chunk(const yg_chunk* c) {
  if (!c) throw yg::YgError{YG_ERR_ARG, "chunk must not be NULL"};
  if (c->nrow < 0 || c->nchan < 0 || c->npol <= 0) throw yg::YgError{YG_ERR_ARG, "bad chunk shape"};
  if (c->nrow > 0 && c->nchan > 0 && (!c->uvw || !c->freq || !c->vis))
    throw yg::YgError{YG_ERR_ARG, "chunk needs uvw, freq and vis"};
  yg::Chunk x;
  x.nrow = c->nrow;
  x.nchan = c->nchan;
  x.npol = c->npol;
  x.uvw = c->uvw;
  x.delay = c->delay;
  x.freq = c->freq;
  x.vis = reinterpret_cast<float2*>(c->vis);
  x.noise = reinterpret_cast<const float2*>(c->noise);
  x.flag = c->flag;
  x.feed1 = c->feed1;
  x.pointing = c->pointing;
  x.on_device = c->on_device;
  return x;
}

yg::Gridder& G(yg_gridder* g) {
  if (!g || !g->g) throw yg::YgError{YG_ERR_ARG, "NULL gridder handle"};
  return *g->g;
}

const yg::Gridder& G(const yg_gridder* g) {
  if (!g || !g->g) throw yg::YgError{YG_ERR_ARG, "NULL gridder handle"};
  return *g->g;
}

}  // namespace

extern "C" {

const char* yg_last_error(void) { return g_last_error.c_str(); }

int yg_create(const char* parset, yg_gridder** out) {
  return guarded([&] {
    if (!parset || !out) throw yg::YgError{YG_ERR_ARG, "NULL argument"};
    *out = nullptr;
    auto h = std::make_unique<yg_gridder>();
    h->g = yg::Gridder::make(yg::Parset::parse(parset));
    *out = h.release();
  });
}

int yg_clone(const yg_gridder* g, yg_gridder** out) {
  return guarded([&] {
    if (!out) throw yg::YgError{YG_ERR_ARG, "NULL argument"};
    auto h = std::make_unique<yg_gridder>();
    h->g = G(g).clone();
    *out = h.release();
  });
}

void yg_destroy(yg_gridder* g) { delete g; }

int yg_initialise_grid(yg_gridder* g, const yg_axes* axes, int32_t nx, int32_t ny, int32_t npol, int32_t nchan,
                       int32_t dopsf, int32_t dopcf) {
  return guarded([&] { G(g).initialise_grid(to_axes(axes), nx, ny, npol, nchan, dopsf != 0, dopcf != 0); });
}

int yg_grid(yg_gridder* g, const yg_chunk* chunk) {
  return guarded([&] { G(g).grid(to_chunk(chunk)); });
}

int yg_finalise_grid(yg_gridder* g, float* image, int32_t on_device) {
  return guarded([&] {
    if (!image) throw yg::YgError{YG_ERR_ARG, "NULL image"};
    G(g).finalise_grid(image, on_device != 0);
  });
}

int yg_finalise_weights(yg_gridder* g, float* weights, int32_t on_device) {
  return guarded([&] {
    if (!weights) throw yg::YgError{YG_ERR_ARG, "NULL weights"};
    G(g).finalise_weights(weights, on_device != 0);
  });
}

int yg_initialise_degrid(yg_gridder* g, const yg_axes* axes, int32_t nx, int32_t ny, int32_t npol, int32_t nchan,
                         const float* image, int32_t on_device) {
  return guarded([&] {
    if (!image) throw yg::YgError{YG_ERR_ARG, "NULL image"};
    G(g).initialise_degrid(to_axes(axes), nx, ny, npol, nchan, image, on_device != 0);
  });
}

int yg_degrid(yg_gridder* g, yg_chunk* chunk) {
  return guarded([&] {
    yg::Chunk c = to_chunk(chunk);
    G(g).degrid(c);
  });
}

int yg_finalise_degrid(yg_gridder* g) {
  return guarded([&] { G(g).finalise_degrid(); });
}

int yg_customise_for_context(yg_gridder* g, const char* context) {
  return guarded([&] { G(g).customise_for_context(context ? context : ""); });
}

int yg_init_vis_weights_mfs(yg_gridder* g, double reffreq) {
  return guarded([&] { G(g).init_vis_weights_mfs(reffreq); });
}

int yg_is_model_empty(const yg_gridder* g, int32_t* empty) {
  return guarded([&] {
    if (!empty) throw yg::YgError{YG_ERR_ARG, "NULL argument"};
    *empty = G(g).is_model_empty() ? 1 : 0;
  });
}

int yg_get_support(const yg_gridder* g, int32_t* support, int32_t* oversample, int32_t* ncf) {
  return guarded([&] {
    const yg::Gridder& x = G(g);
    if (support) *support = x.support();
    if (oversample) *oversample = x.oversample();
    if (ncf) *ncf = x.ncf();
  });
}

int yg_get_cf(const yg_gridder* g, int32_t* sizes, int64_t* offsets, float* data, int64_t data_capacity) {
  return guarded([&] {
    const yg::Gridder& x = G(g);
    std::vector<int> s;
    std::vector<long long> o;
    x.cf_sizes(s, o);
    if (sizes) std::memcpy(sizes, s.data(), s.size() * sizeof(int));
    if (offsets)
      for (size_t i = 0; i < o.size(); ++i) offsets[i] = o[i];
    if (data) {
      std::vector<float2> d;
      x.cf_data(d);
      if ((int64_t)d.size() > data_capacity) throw yg::YgError{YG_ERR_ARG, "CF buffer too small"};
      std::memcpy(data, d.data(), d.size() * sizeof(float2));
    }
  });
}

int yg_get_cf_offsets(const yg_gridder* g, int32_t* offsets, int32_t capacity, int32_t* n) {
  return guarded([&] {
    std::vector<int2> o;
    G(g).cf_offsets(o);
    if (n) *n = (int32_t)o.size();
    if (offsets) {
      if ((int32_t)o.size() > capacity) throw yg::YgError{YG_ERR_ARG, "offset buffer too small"};
      for (size_t i = 0; i < o.size(); ++i) {
        offsets[2 * i] = o[i].x;
        offsets[2 * i + 1] = o[i].y;
      }
    }
  });
}

int yg_get_sum_weights(const yg_gridder* g, double* out, int64_t capacity, int32_t* nrows) {
  return guarded([&] {
    std::vector<double> w;
    int rows = 0;
    G(g).sum_weights(w, &rows);
    if (nrows) *nrows = rows;
    if (out) {
      if ((int64_t)w.size() > capacity) throw yg::YgError{YG_ERR_ARG, "buffer too small"};
      std::memcpy(out, w.data(), w.size() * sizeof(double));
    }
  });
}

int yg_get_grid(const yg_gridder* g, float* out, int64_t capacity_complex, int32_t* ngrids) {
  return guarded([&] {
    const yg::Gridder& x = G(g);
    if (ngrids) *ngrids = x.ngrids();
    if (out) {
      std::vector<float2> d;
      x.grid_data(d);
      if ((int64_t)d.size() > capacity_complex) throw yg::YgError{YG_ERR_ARG, "grid buffer too small"};
      std::memcpy(out, d.data(), d.size() * sizeof(float2));
    }
  });
}

int yg_get_shape(const yg_gridder* g, int32_t* nx, int32_t* ny, int32_t* npol, int32_t* nchan) {
  return guarded([&] {
    int a, b, c, d;
    G(g).shape(&a, &b, &c, &d);
    if (nx) *nx = a;
    if (ny) *ny = b;
    if (npol) *npol = c;
    if (nchan) *nchan = d;
  });
}

int yg_get_kernel_times(const yg_gridder* g, double* out4) {
  return guarded([&] {
    if (!out4) throw yg::YgError{YG_ERR_ARG, "NULL argument"};
    const yg::Stats& s = G(g).stats();
    out4[0] = s.kgrid_ms;
    out4[1] = s.kgrid_calls;
    out4[2] = s.kdegrid_ms;
    out4[3] = s.kdegrid_calls;
  });
}

int64_t yg_kernel_launch_count(void) { return yg::g_kernel_launches.load(); }

int yg_get_stats(const yg_gridder* g, double* out8) {
  return guarded([&] {
    if (!out8) throw yg::YgError{YG_ERR_ARG, "NULL argument"};
    const yg::Stats& s = G(g).stats();
    out8[0] = s.samples_gridded;
    out8[1] = s.taps_gridded;
    out8[2] = s.samples_degridded;
    out8[3] = s.taps_degridded;
    out8[4] = s.time_grid_ms;
    out8[5] = s.time_degrid_ms;
    out8[6] = s.time_cf_ms;
    out8[7] = s.cf_generations;
  });
}

int yg_build_cf(yg_gridder* g) {
  return guarded([&] { G(g).build_cf(); });
}

int yg_plan_create(yg_gridder* g, const yg_chunk* chunk, yg_plan** out) {
  return guarded([&] {
    if (!out) throw yg::YgError{YG_ERR_ARG, "NULL argument"};
    yg::Gridder& x = G(g);
    yg::Chunk c = to_chunk(chunk);
    if (!c.on_device) throw yg::YgError{YG_ERR_ARG, "plans need device-resident chunks"};
    auto p = std::make_unique<yg_plan>();
    x.prepare_plan_cf(c);
    x.bin(c, p->pl);
    *out = p.release();
  });
}

int yg_plan_grid(yg_gridder* g, const yg_plan* plan, const yg_chunk* chunk) {
  return guarded([&] {
    if (!plan) throw yg::YgError{YG_ERR_ARG, "NULL plan"};
    yg::Chunk c = to_chunk(chunk);
    if (!c.on_device) throw yg::YgError{YG_ERR_ARG, "plans need device-resident chunks"};
    G(g).prepare_plan_cf(c);
    G(g).grid_plan(c, plan->pl);
  });
}

int yg_plan_degrid(yg_gridder* g, yg_plan* plan, yg_chunk* chunk) {
  return guarded([&] {
    if (!plan) throw yg::YgError{YG_ERR_ARG, "NULL plan"};
    yg::Chunk c = to_chunk(chunk);
    if (!c.on_device) throw yg::YgError{YG_ERR_ARG, "plans need device-resident chunks"};
    yg::Gridder& x = G(g);
    if (x.is_model_empty()) return;
    // a plan made by another gridder of the same parset: this one's CFs
    // (AWProject builds them from the chunk's beams and frequencies)
    x.prepare_plan_cf(c);
    x.degrid_plan(c, plan->pl);
  });
}

int yg_plan_info(const yg_plan* plan, int64_t* nvalid, int32_t* nitems, int32_t* tile) {
  return guarded([&] {
    if (!plan) throw yg::YgError{YG_ERR_ARG, "NULL plan"};
    if (nvalid) *nvalid = plan->pl.nvalid;
    if (nitems) *nitems = plan->pl.nitems;
    if (tile) *tile = plan->pl.tile;
  });
}

int yg_plan_samples(const yg_gridder* g, const yg_plan* plan, int32_t* iu, int32_t* iv, int32_t* cfi,
                    uint8_t* status) {
  return guarded([&] {
    if (!plan || !iu || !iv || !cfi || !status) throw yg::YgError{YG_ERR_ARG, "NULL argument"};
    G(g).plan_samples(plan->pl, iu, iv, cfi, status);
  });
}

void yg_plan_destroy(yg_plan* plan) { delete plan; }

int yg_set_tile(yg_gridder* g, int32_t tile) {
  return guarded([&] {
    if (tile < 0 || (tile > 0 && tile < 8)) throw yg::YgError{YG_ERR_ARG, "tile must be 0 or >= 8"};
    G(g).set_tile(tile);
  });
}

int yg_set_grid_variant(yg_gridder* g, int32_t variant) {
  return guarded([&] {
    if (variant < 0 || (variant & ~(240 | 256 | 512)) > 3)
      throw yg::YgError{YG_ERR_ARG, "variant must be 0 to 3, plus 16 (register accumulation), 32 "
                                    "(position-major records) or 64 (plane-major records, staged CF planes; "
                                    "plus 128: their tile in global memory), plus 256 (degridding by "
                                    "k_degrid_t) or 512 (one degridded sample per half-warp pass)"};
    G(g).set_grid_mode(variant);
  });
}

int yg_set_item_size(yg_gridder* g, int32_t vmax) {
  return guarded([&] {
    if (vmax < 1) throw yg::YgError{YG_ERR_ARG, "item size must be positive"};
    G(g).set_vmax(vmax);
  });
}

int yg_get_stream(yg_gridder* g, void** stream) {
  return guarded([&] {
    if (!stream) throw yg::YgError{YG_ERR_ARG, "NULL argument"};
    yg::Gridder& x = G(g);
    x.ensure_device();
    *stream = (void*)x.stream();
  });
}

int yg_synchronize(yg_gridder* g) {
  return guarded([&] { G(g).sync(); });
}

int yg_degrid_noalloc(yg_gridder* g, yg_chunk* chunk) {
  return guarded([&] {
    yg::Chunk c = to_chunk(chunk);
    G(g).degrid_noalloc(c);
  });
}

int32_t yg_mlp_nparams(void) { return yg::kMlpParams; }

int yg_learned_train(yg_gridder* g, const yg_learn_params* p, yg_learn_report* rep) {
  return guarded([&] {
    if (!p) throw yg::YgError{YG_ERR_ARG, "learn parameters must not be NULL"};
    yg::LearnParams lp;
    lp.ntrain = p->ntrain;
    lp.batch = p->batch;
    lp.steps = p->steps;
    lp.lr = p->lr;
    lp.seed = p->seed;
    if (lp.ntrain <= 0 || lp.batch <= 0 || lp.steps < 0 || !(lp.lr > 0.0))
      throw yg::YgError{YG_ERR_ARG, "ntrain, batch and lr must be positive, steps non-negative"};
    yg::LearnReport r;
    G(g).learned_train(lp, p->nwplanes_train, &r);
    if (rep) {
      rep->final_loss = r.final_loss;
      rep->train_ms = r.train_ms;
      rep->steps = r.steps;
      rep->scale = r.scale;
      rep->cf_table_bytes = (double)G(g).cf_table_bytes();
      rep->network_bytes = (double)yg::kMlpParams * 2.0;
    }
  });
}

int yg_set_cf_form(yg_gridder* g, int32_t form) {
  return guarded([&] { G(g).set_cf_form(form); });
}

int yg_learned_get_params(yg_gridder* g, float* params, float* scale) {
  return guarded([&] {
    if (!params) throw yg::YgError{YG_ERR_ARG, "params must not be NULL"};
    std::vector<float> p;
    G(g).learned_params(p);
    std::memcpy(params, p.data(), p.size() * sizeof(float));
    if (scale) *scale = (float)G(g).learned_scale();
  });
}

int yg_learned_set_params(yg_gridder* g, const float* params, float scale) {
  return guarded([&] {
    if (!params || !(scale > 0.f)) throw yg::YgError{YG_ERR_ARG, "params must be given and scale positive"};
    G(g).set_learned_params(params, scale);
  });
}

int yg_mlp_loss_grad(const float* params, const float* x, const float* t, int64_t n, float scale, float* grad,
                     double* loss) {
  return guarded([&] {
    if (!params || !grad || n < 0 || (n > 0 && (!x || !t)))
      throw yg::YgError{YG_ERR_ARG, "params, x, t and grad must be given"};
    yg::DevBuf p, X, T, G_, L;
    auto ck = [](cudaError_t e) {
      if (e != cudaSuccess) throw yg::YgError{YG_ERR_CUDA, cudaGetErrorString(e)};
    };
    ck(p.ensure(yg::kMlpParamsPadded * sizeof(float)));
    ck(X.ensure(std::max<int64_t>(1, n) * yg::kMlpIn * sizeof(float)));
    ck(T.ensure(std::max<int64_t>(1, n) * 2 * sizeof(float)));
    ck(G_.ensure(yg::kMlpParamsPadded * sizeof(float)));
    ck(L.ensure(sizeof(double)));
    ck(cudaMemcpy(p.p, params, yg::kMlpParams * sizeof(float), cudaMemcpyHostToDevice));
    if (n > 0) {
      ck(cudaMemcpy(X.p, x, n * yg::kMlpIn * sizeof(float), cudaMemcpyHostToDevice));
      ck(cudaMemcpy(T.p, t, n * 2 * sizeof(float), cudaMemcpyHostToDevice));
    }
    const int rc = yg::mlp_grad(p.as<float>(), X.as<float>(), T.as<float>(), n, scale, G_.as<float>(),
                                L.as<double>(), 0);
    if (rc) throw yg::YgError{rc, "network gradient"};
    ck(cudaMemcpy(grad, G_.p, yg::kMlpParams * sizeof(float), cudaMemcpyDeviceToHost));
    double l = 0.0;
    ck(cudaMemcpy(&l, L.p, sizeof(double), cudaMemcpyDeviceToHost));
    if (loss) *loss = l;
  });
}

int yg_mlp_eval(const float* params, const float* x, int64_t n, float* y) {
  return guarded([&] {
    if (!params || n < 0 || (n > 0 && (!x || !y))) throw yg::YgError{YG_ERR_ARG, "params, x and y must be given"};
    yg::DevBuf p, w16, X, Y;
    auto ck = [](cudaError_t e) {
      if (e != cudaSuccess) throw yg::YgError{YG_ERR_CUDA, cudaGetErrorString(e)};
    };
    yg::LearnedNet net;
    std::vector<float> v(params, params + yg::kMlpParams);
    if (net.init(v, 0)) throw yg::YgError{YG_ERR_CUDA, "network set-up"};
    ck(X.ensure(std::max<int64_t>(1, n) * yg::kMlpIn * sizeof(float)));
    ck(Y.ensure(std::max<int64_t>(1, n) * 2 * sizeof(float)));
    if (n > 0) ck(cudaMemcpy(X.p, x, n * yg::kMlpIn * sizeof(float), cudaMemcpyHostToDevice));
    const int rc = yg::mlp_eval_batch(net.w16.as<__half>(), X.as<float>(), n, Y.as<float>(), 0);
    if (rc) throw yg::YgError{rc, "network evaluation"};
    if (n > 0) ck(cudaMemcpy(y, Y.p, n * 2 * sizeof(float), cudaMemcpyDeviceToHost));
  });
}

int yg_sort_pairs(uint64_t* keys, uint32_t* vals, int64_t n, int32_t end_bit) {
  return guarded([&] {
    if (n < 0 || end_bit < 0 || end_bit > 64 || (n > 0 && (!keys || !vals)))
      throw yg::YgError{YG_ERR_ARG, "keys and vals must be given, 0 <= end_bit <= 64"};
    if (n >= (1ll << 31)) throw yg::YgError{YG_ERR_ARG, "n must be below 2^31"};
    if (n == 0) return;
    yg::DevBuf k0, k1, v0, v1, tmp;
    auto ck = [](cudaError_t e) {
      if (e != cudaSuccess) throw yg::YgError{YG_ERR_CUDA, cudaGetErrorString(e)};
    };
    ck(k0.ensure(n * 8));
    ck(k1.ensure(n * 8));
    ck(v0.ensure(n * 4));
    ck(v1.ensure(n * 4));
    ck(tmp.ensure(yg::sort_pairs_tmp_bytes(n)));
    ck(cudaMemcpy(k0.p, keys, n * 8, cudaMemcpyHostToDevice));
    ck(cudaMemcpy(v0.p, vals, n * 4, cudaMemcpyHostToDevice));
    int alt = 0;
    ck(yg::sort_pairs(k0.as<unsigned long long>(), k1.as<unsigned long long>(), v0.as<unsigned int>(),
                      v1.as<unsigned int>(), n, end_bit, tmp.p, tmp.bytes, 0, &alt));
    ck(cudaMemcpy(keys, alt ? k1.p : k0.p, n * 8, cudaMemcpyDeviceToHost));
    ck(cudaMemcpy(vals, alt ? v1.p : v0.p, n * 4, cudaMemcpyDeviceToHost));
  });
}

int yg_scan_i32(const int32_t* in, int32_t* out, int64_t n, int32_t op, int32_t exclusive) {
  return guarded([&] {
    if (n < 0 || op < 0 || op > 2 || (n > 0 && (!in || !out)))
      throw yg::YgError{YG_ERR_ARG, "in and out must be given, op 0 (sum), 1 (min) or 2 (max)"};
    if (n >= (1ll << 31)) throw yg::YgError{YG_ERR_ARG, "n must be below 2^31"};
    if (n == 0) return;
    yg::DevBuf a, tmp;
    auto ck = [](cudaError_t e) {
      if (e != cudaSuccess) throw yg::YgError{YG_ERR_CUDA, cudaGetErrorString(e)};
    };
    ck(a.ensure(n * 4));
    ck(tmp.ensure(yg::scan_tmp_bytes(n)));
    ck(cudaMemcpy(a.p, in, n * 4, cudaMemcpyHostToDevice));
    ck(yg::scan_i32(a.as<int>(), a.as<int>(), n, op, exclusive != 0, tmp.p, tmp.bytes, 0));
    ck(cudaMemcpy(out, a.p, n * 4, cudaMemcpyDeviceToHost));
  });
}

int yg_cycle_create(int32_t n, yg_gridder* const* degridders, yg_gridder* const* gridders, const yg_chunk* chunks,
                    yg_cycle** out) {
  return guarded([&] {
    if (n <= 0 || !degridders || !gridders || !chunks || !out) throw yg::YgError{YG_ERR_ARG, "NULL argument"};
    std::vector<yg::Gridder*> dg(n), gg(n);
    std::vector<yg::Chunk> ch(n);
    for (int i = 0; i < n; ++i) {
      dg[i] = &G(degridders[i]);
      gg[i] = &G(gridders[i]);
      ch[i] = to_chunk(&chunks[i]);
    }
    auto c = std::make_unique<yg_cycle>();
    c->b.build(dg, gg, ch);
    *out = c.release();
  });
}

int yg_cycle_create_roles(int32_t n, const yg_cycle_roles* roles, const yg_chunk* chunks, yg_cycle** out) {
  return guarded([&] {
    if (n <= 0 || !roles || !chunks || !out) throw yg::YgError{YG_ERR_ARG, "NULL argument"};
    std::vector<yg::Gridder*> dg(n), gg(n), psf(n, nullptr), pcf(n, nullptr);
    std::vector<yg::Chunk> ch(n);
    bool any_psf = false, any_pcf = false;
    for (int i = 0; i < n; ++i) {
      if (!roles[i].model || !roles[i].residual) throw yg::YgError{YG_ERR_ARG, "every instance needs a model and a residual gridder"};
      dg[i] = &G(roles[i].model);
      gg[i] = &G(roles[i].residual);
      if (roles[i].psf) { psf[i] = &G(roles[i].psf); any_psf = true; }
      if (roles[i].pcf) { pcf[i] = &G(roles[i].pcf); any_pcf = true; }
      ch[i] = to_chunk(&chunks[i]);
    }
    auto c = std::make_unique<yg_cycle>();
    c->b.build(dg, gg, ch, any_psf ? psf : std::vector<yg::Gridder*>{}, any_pcf ? pcf : std::vector<yg::Gridder*>{});
    *out = c.release();
  });
}

int yg_cycle_run(yg_cycle* c, int32_t cycles, float* gpu_ms) {
  return guarded([&] {
    if (!c || cycles < 0) throw yg::YgError{YG_ERR_ARG, "NULL cycle or negative count"};
    const float ms = c->b.run(cycles);
    if (gpu_ms) *gpu_ms = ms;
  });
}

int yg_cycle_info(const yg_cycle* c, int64_t* nodes) {
  return guarded([&] {
    if (!c || !nodes) throw yg::YgError{YG_ERR_ARG, "NULL argument"};
    *nodes = c->b.nodes;
  });
}

void yg_cycle_destroy(yg_cycle* c) { delete c; }

int yg_autotune(yg_gridder* g, const yg_chunk* chunk, int32_t max_trials, yg_tune_report* rep) {
  return guarded([&] {
    if (!chunk || max_trials < 1) throw yg::YgError{YG_ERR_ARG, "chunk and a positive trial count are required"};
    yg::Chunk c = to_chunk(chunk);
    const yg::TuneReport r = G(g).autotune(c, max_trials);
    if (rep) {
      rep->tile = r.best.tile;
      rep->items = r.best.vmax;
      rep->variant = r.best.variant;
      rep->trials = (int32_t)r.trials.size();
      rep->best_ms = r.best_ms;
      rep->default_ms = r.default_ms;
      rep->cf_width = r.wpad;
      rep->npol = r.npol;
    }
  });
}

void yg_autotune_reset(void) { yg::tune_clear(); }

}  // extern "C"

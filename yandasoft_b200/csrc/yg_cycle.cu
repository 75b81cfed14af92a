// Major cycle as a CUDA graph: for each of n imaging instances (a degridder
// holding the model, a gridder for the residual, optionally a PSF gridder and
// a preconditioner-function gridder, one device-resident chunk of observed
// visibilities), degrid the model into model visibilities, subtract them from
// the observed ones and grid the residual, then the PSF and the
// preconditioner function from the same buffer
// (ImageFFTEquation::calcImagingEquations, ImageFFTEquation.cc:437-479).
// The instances are recorded once, each on a branch of its own (eight side
// streams, fork/join events), into one graph that every later cycle replays
// with a single launch; the GPU runs independent instances side by side.
#include <cuda_runtime.h>

#include <algorithm>
#include <memory>
#include <string>
#include <vector>

#include "yg_cycle.h"

namespace yg {

namespace {

__global__ void k_subtract(const float2* __restrict__ obs, const float2* __restrict__ model, float2* __restrict__ res,
                           long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float2 o = obs[i], m = model[i];
    res[i] = make_float2(o.x - m.x, o.y - m.y);
  }
}

void throw_if(bool cond, int code, const char* msg) {
  if (cond) throw YgError{code, msg};
}

void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw YgError{YG_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e)};
}

}  // namespace

CycleBatch::~CycleBatch() {
  if (exec) cudaGraphExecDestroy(exec);
  if (graph) cudaGraphDestroy(graph);
  for (auto e : events) cudaEventDestroy(e);
  for (auto s : side) cudaStreamDestroy(s);
  if (main) cudaStreamDestroy(main);
}

void CycleBatch::enqueue(Instance& in, cudaStream_t st) {
  const size_t bytes = (size_t)in.obs.nrow * in.obs.nchan * in.obs.npol * sizeof(float2);
  ck(cudaMemsetAsync(in.model_vis.p, 0, bytes, st), "clear model visibilities");
  if (!in.dg->is_model_empty()) in.dg->degrid_enqueue(in.model, in.plan, in.mfs_dg, st);
  const long long n = (long long)in.obs.nrow * in.obs.nchan * in.obs.npol;
  const int blocks = (int)std::min<long long>((n + 255) / 256, 148 * 16);
  k_subtract<<<std::max(1, blocks), 256, 0, st>>>(in.obs.vis, in.model_vis.as<float2>(), in.resid_vis.as<float2>(), n);
  ck(cudaGetLastError(), "subtract");
  in.gg->grid_enqueue(in.resid, in.plan, in.mfs_gg, st);
  // the PSF and the preconditioner grid the weights of the same buffer
  if (in.psf) in.psf->grid_enqueue(in.resid, in.psf_plan, in.mfs_psf, st);
  if (in.pcf) in.pcf->grid_enqueue(in.resid, in.pcf_plan, in.mfs_pcf, st);
}

void CycleBatch::build(const std::vector<Gridder*>& dgs, const std::vector<Gridder*>& ggs,
                       const std::vector<Chunk>& chunks, const std::vector<Gridder*>& psfs,
                       const std::vector<Gridder*>& pcfs) {
  const size_t n = dgs.size();
  throw_if(n == 0 || ggs.size() != n || chunks.size() != n, YG_ERR_ARG, "instances need a degridder, a gridder and a chunk each");
  throw_if(!psfs.empty() && psfs.size() != n, YG_ERR_ARG, "one PSF gridder entry per instance");
  throw_if(!pcfs.empty() && pcfs.size() != n, YG_ERR_ARG, "one preconditioner gridder entry per instance");
  ck(cudaStreamCreateWithFlags(&main, cudaStreamNonBlocking), "stream");
  const int nside = (int)std::min<size_t>(8, n);
  side.resize(nside);
  for (auto& s : side) ck(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
  for (size_t i = 0; i < n; ++i) inst.emplace_back(new Instance());
  for (size_t i = 0; i < n; ++i) {
    Instance& in = *inst[i];
    throw_if(!chunks[i].on_device, YG_ERR_ARG, "major cycles need device-resident chunks");
    in.dg = dgs[i];
    in.gg = ggs[i];
    in.obs = chunks[i];
    const size_t bytes = (size_t)in.obs.nrow * in.obs.nchan * in.obs.npol * sizeof(float2);
    ck(in.model_vis.ensure(bytes), "model visibilities");
    ck(in.resid_vis.ensure(bytes), "residual visibilities");
    in.model = in.obs;
    in.model.vis = in.model_vis.as<float2>();
    in.resid = in.obs;
    in.resid.vis = in.resid_vis.as<float2>();
    in.gg->prepare_plan_cf(in.obs);
    in.gg->bin(in.obs, in.plan);
    in.dg->prepare_plan_cf(in.obs);
    in.mfs_dg = in.dg->mfs_weights(in.obs);
    in.mfs_gg = in.gg->mfs_weights(in.obs);
    in.psf = psfs.empty() ? nullptr : psfs[i];
    in.pcf = pcfs.empty() ? nullptr : pcfs[i];
    if (in.psf) {
      throw_if(!in.psf->is_psf(), YG_ERR_STATE, "the PSF gridder must be initialised with dopsf");
      in.psf->prepare_plan_cf(in.obs);
      in.psf->bin(in.obs, in.psf_plan);
      in.mfs_psf = in.psf->mfs_weights(in.obs);
    }
    if (in.pcf) {
      throw_if(!in.pcf->is_pcf(), YG_ERR_STATE, "the preconditioner gridder must be initialised with dopcf");
      in.pcf->prepare_plan_cf(in.obs);
      in.pcf->bin(in.obs, in.pcf_plan);
      in.mfs_pcf = in.pcf->mfs_weights(in.obs);
    }
  }
  // one uncaptured cycle sizes every buffer and makes the once-per-plan tables
  for (auto& in : inst) {
    enqueue(*in, main);
    ck(cudaStreamSynchronize(main), "warm-up cycle");
    in->dg->check_device_error();
    in->gg->check_device_error();
    if (in->psf) in->psf->check_device_error();
    if (in->pcf) in->pcf->check_device_error();
  }
  events.resize(1 + n);
  for (auto& e : events) ck(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
  ck(cudaStreamBeginCapture(main, cudaStreamCaptureModeThreadLocal), "begin capture");
  try {
    ck(cudaEventRecord(events[0], main), "fork");
    for (size_t i = 0; i < n; ++i) {
      cudaStream_t s = side[i % nside];
      ck(cudaStreamWaitEvent(s, events[0], 0), "fork wait");
      enqueue(*inst[i], s);
      ck(cudaEventRecord(events[1 + i], s), "join");
    }
    for (size_t i = 0; i < n; ++i) ck(cudaStreamWaitEvent(main, events[1 + i], 0), "join wait");
  } catch (...) {
    cudaGraph_t g = nullptr;
    cudaStreamEndCapture(main, &g);
    if (g) cudaGraphDestroy(g);
    throw;
  }
  ck(cudaStreamEndCapture(main, &graph), "end capture");
  ck(cudaGraphInstantiate(&exec, graph, 0), "instantiate");
  size_t nn = 0;
  cudaGraphGetNodes(graph, nullptr, &nn);
  nodes = (long long)nn;
}

float CycleBatch::run(int cycles) {
  cudaEvent_t e0, e1;
  ck(cudaEventCreate(&e0), "event");
  ck(cudaEventCreate(&e1), "event");
  ck(cudaEventRecord(e0, main), "event");
  for (int c = 0; c < cycles; ++c) ck(cudaGraphLaunch(exec, main), "graph launch");
  ck(cudaEventRecord(e1, main), "event");
  ck(cudaEventSynchronize(e1), "cycle");
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  for (auto& in : inst) {
    in->dg->check_device_error();
    in->gg->check_device_error();
    if (in->psf) in->psf->check_device_error();
    if (in->pcf) in->pcf->check_device_error();
  }
  return ms;
}

}  // namespace yg

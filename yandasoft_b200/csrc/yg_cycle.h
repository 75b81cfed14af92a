// Major-cycle batches recorded as one CUDA graph (yg_cycle.cu).
#pragma once
#include <cuda_runtime.h>

#include <memory>
#include <vector>

#include "yg_gridder.h"

namespace yg {

struct CycleBatch {
  struct Instance {
    Gridder* dg = nullptr;     // holds the model grids
    Gridder* gg = nullptr;     // receives the residual
    Gridder* psf = nullptr;    // PSF gridder (initialised with dopsf), optional
    Gridder* pcf = nullptr;    // preconditioner-function gridder (dopcf), optional
    Chunk obs, model, resid;   // device chunks sharing uvw, frequencies, flags and noise
    DevBuf model_vis, resid_vis;
    Plan plan, psf_plan, pcf_plan;
    const float* mfs_dg = nullptr;
    const float* mfs_gg = nullptr;
    const float* mfs_psf = nullptr;
    const float* mfs_pcf = nullptr;
  };
  std::vector<std::unique_ptr<Instance>> inst;
  std::vector<cudaStream_t> side;
  std::vector<cudaEvent_t> events;
  cudaStream_t main = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  long long nodes = 0;

  CycleBatch() = default;
  CycleBatch(const CycleBatch&) = delete;
  ~CycleBatch();
  // psfs / pcfs: empty, or one (possibly null) gridder per instance
  void build(const std::vector<Gridder*>& dgs, const std::vector<Gridder*>& ggs, const std::vector<Chunk>& chunks,
             const std::vector<Gridder*>& psfs = {}, const std::vector<Gridder*>& pcfs = {});
  // replays the graph `cycles` times; returns the GPU milliseconds
  float run(int cycles);

 private:
  void enqueue(Instance& in, cudaStream_t st);
};

}  // namespace yg

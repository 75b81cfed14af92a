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
    Chunk obs, model, resid;   // device chunks sharing uvw, frequencies, flags and noise
    DevBuf model_vis, resid_vis;
    Plan plan;
    const float* mfs_dg = nullptr;
    const float* mfs_gg = nullptr;
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
  void build(const std::vector<Gridder*>& dgs, const std::vector<Gridder*>& ggs, const std::vector<Chunk>& chunks);
  // replays the graph `cycles` times; returns the GPU milliseconds
  float run(int cycles);

 private:
  void enqueue(Instance& in, cudaStream_t st);
};

}  // namespace yg

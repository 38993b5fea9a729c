// mm_persist.cuh -- the persistent RK4 step kernel's host program (internal;
// see mm_persist.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "mm_launch.cuh"

namespace mm {

// MMCUDA_PERSIST=1 turns the persistent path on (off by default)
bool persist_enabled();

class PersistProgram {
 public:
  PersistProgram() = default;
  ~PersistProgram();
  PersistProgram(const PersistProgram&) = delete;
  PersistProgram& operator=(const PersistProgram&) = delete;
  // Phases from the recorded steps of one or more meshes (all records must
  // have a persistent form).  0, or -1 (not representable) / -2 (CUDA).
  int build(const std::vector<std::vector<LaunchRec>>& recs, bool fp32, char* err, size_t nerr);
  // nsteps steps on st, then waits for them: 0, 1 (a barrier wait ran out:
  // MM_ERR_TIMEOUT) or 2 (CUDA error).
  int run(int64_t nsteps, cudaStream_t st);
  bool ready() const { return nphases > 0; }
  void release();

 private:
  void* dev = nullptr;
  unsigned* bar = nullptr;
  int* status = nullptr;
  int* host_status = nullptr;
  int nphases = 0;
  int blocks = 0;
  size_t smem = 0;
  bool f32 = true;
};

}  // namespace mm

// mm_persist.cu -- persistent RK4 step kernel: one cooperative launch runs
// many RK4 steps of a small mesh or of a batch of meshes (internal).
//
// A step is recorded once (mm_launch.cuh: every launch of the handles'
// rk4_enqueue becomes a record) and merged into phases: the records of the
// same kernel that come next for several meshes form one phase.  The kernel
// keeps one block per SM slot resident and, for every step and phase, walks
// the phase's blocks (blockIdx.x, blockIdx.x + gridDim.x, ...): each looks
// its mesh up, stages that mesh's arguments in shared memory and runs the
// descriptor's body.  Phases are separated by a grid barrier.  The barrier
// spins a bounded number of times; a block whose wait runs out sets the
// status word (MM_ERR_TIMEOUT on the host) and every block then leaves at its
// next barrier, so a broken schedule ends the kernel instead of hanging it.
// Co-residency of all blocks is guaranteed by the cooperative launch.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "mm_cell.cuh"
#include "mm_passes.cuh"
#include "mm_persist.cuh"

namespace mm {

namespace {

constexpr int kPersistNT = 256;
constexpr int kPersistArgs = 1024;  // bytes of the largest descriptor argument struct (checked on the host)

struct PPhase {
  int kind;    // PersistKind
  int nparts;  // meshes
  int blocks;  // sum of the meshes' grids
  int args_size;
  const unsigned char* args;  // nparts argument structs
  const int* begins;          // first block of each mesh
  const uint3* grids;         // each mesh's grid
};

template <class K>
__device__ __forceinline__ void run_desc(const unsigned char* a, uint3 bid) {
  K::body(*reinterpret_cast<const typename K::Args*>(a), bid);
}

template <typename R>
__device__ __forceinline__ void run_kind(int kind, const unsigned char* a, uint3 bid) {
  switch (kind) {
    case 0: run_desc<FwdX<R, XM_MAGN, kHotNT>>(a, bid); break;
    case 1: run_desc<InvX<R, kHotNT>>(a, bid); break;
    case 2: run_desc<YLines<R, YL_FWD, kHotNT, true, false>>(a, bid); break;
    case 3: run_desc<YLines<R, YL_INV, kHotNT, true, false>>(a, bid); break;
    case 4: run_desc<YLines<R, YL_CONV2D, kHotNT, true, false>>(a, bid); break;
    case 5: run_desc<YLines<R, YL_CONV2D, kHotNT, true, true>>(a, bid); break;
    case 6: run_desc<ZConv<R, kHotNT, true>>(a, bid); break;
    case 7: run_desc<ZSmall<R, 3>>(a, bid); break;
    case 8: run_desc<ZSmall<R, 5>>(a, bid); break;
    case 9: run_desc<ZSmall<R, 7>>(a, bid); break;
    case 10: run_desc<ZSmall<R, 9>>(a, bid); break;
    default: run_desc<StagePlain<R>>(a, bid); break;
  }
}

// Grid barrier: arrival counter bar[0], generation bar[1].  Returns false
// when this block's wait ran out or another block's did (status set).
__device__ __forceinline__ bool grid_barrier(unsigned* bar, int* status, unsigned long long spins, int* s_ok) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* vgen = bar + 1;
    const unsigned gen = *vgen;
    __threadfence();
    if (atomicAdd(bar, 1u) + 1 == gridDim.x) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      unsigned long long n = 0;
      while (*vgen == gen) {
        if (++n > spins) {
          atomicExch(status, 1);
          break;
        }
        if (*reinterpret_cast<volatile int*>(status)) break;  // another block gave up
        __nanosleep(64);
      }
    }
    __threadfence();
    *s_ok = *reinterpret_cast<volatile int*>(status) == 0;
  }
  __syncthreads();
  return *s_ok != 0;
}

template <typename R>
__global__ void __launch_bounds__(kPersistNT, 1) k_persist(const PPhase* __restrict__ ph, int nph, int nsteps,
                                                          unsigned* bar, int* status, unsigned long long spins) {
  __shared__ __align__(16) unsigned char sa[kPersistArgs];
  __shared__ int s_ok;
  for (int step = 0; step < nsteps; ++step) {
    for (int p = 0; p < nph; ++p) {
      const PPhase P = ph[p];
      for (int vb = blockIdx.x; vb < P.blocks; vb += gridDim.x) {
        int lo = 0, hi = P.nparts - 1;
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (P.begins[mid] <= vb) lo = mid;
          else hi = mid - 1;
        }
        const unsigned* src = reinterpret_cast<const unsigned*>(P.args + static_cast<size_t>(lo) * P.args_size);
        for (int w = threadIdx.x; w < P.args_size / 4; w += kPersistNT) reinterpret_cast<unsigned*>(sa)[w] = src[w];
        __syncthreads();
        const uint3 g = P.grids[lo];
        const unsigned local = static_cast<unsigned>(vb - P.begins[lo]);
        uint3 bid;
        bid.x = local % g.x;
        bid.y = (local / g.x) % g.y;
        bid.z = local / (g.x * g.y);
        run_kind<R>(P.kind, sa, bid);
        __syncthreads();  // the staged arguments and shared buffers are reused
      }
      if (!grid_barrier(bar, status, spins, &s_ok)) return;
    }
  }
}

unsigned long long barrier_spins() {
  static const unsigned long long v = [] {
    const char* e = getenv("MMCUDA_BARRIER_SPINS");
    const long long s = e ? atoll(e) : 0;
    return s > 0 ? static_cast<unsigned long long>(s) : (1ull << 24);
  }();
  return v;
}

}  // namespace

// Opt-in (MMCUDA_PERSIST=1): measured slower than the graphs of separate
// launches on the small meshes it serves (200x50 film 0.153 vs 0.127 ms a
// step; 32 NEB images of 128x128, 1.01 vs 0.38 ms): at 255 registers one
// block per SM is resident, and each phase of a small mesh is a serial
// latency chain either way.
bool persist_enabled() {
  static const bool on = [] {
    const char* e = getenv("MMCUDA_PERSIST");
    return e && e[0] == '1';
  }();
  return on;
}

PersistProgram::~PersistProgram() { release(); }

void PersistProgram::release() {
  if (dev) cudaFree(dev);
  if (host_status) cudaFreeHost(host_status);
  dev = nullptr;
  host_status = nullptr;
  nphases = 0;
}

int PersistProgram::build(const std::vector<std::vector<LaunchRec>>& recs, bool fp32, char* err, size_t nerr) {
  release();
  // greedy in-order merge: the kernel that is next for the most meshes
  struct Ph {
    int kind;
    std::vector<const LaunchRec*> parts;
  };
  std::vector<Ph> phs;
  std::vector<size_t> next(recs.size(), 0);
  for (;;) {
    std::vector<std::pair<const void*, int>> cnt;
    for (size_t j = 0; j < recs.size(); ++j) {
      if (next[j] >= recs[j].size()) continue;
      const void* k = recs[j][next[j]].kind;
      auto it = std::find_if(cnt.begin(), cnt.end(), [&](const auto& q) { return q.first == k; });
      if (it == cnt.end()) cnt.push_back({k, 1});
      else ++it->second;
    }
    if (cnt.empty()) break;
    const void* kind =
        std::max_element(cnt.begin(), cnt.end(), [](const auto& a, const auto& b) { return a.second < b.second; })
            ->first;
    Ph ph;
    for (size_t j = 0; j < recs.size(); ++j)
      if (next[j] < recs[j].size() && recs[j][next[j]].kind == kind) ph.parts.push_back(&recs[j][next[j]++]);
    ph.kind = ph.parts[0]->pkind;
    if (ph.kind < 0 || ph.parts[0]->args_size > static_cast<size_t>(kPersistArgs)) {
      snprintf(err, nerr, "persistent step: a recorded kernel has no persistent form");
      return -1;
    }
    phs.push_back(std::move(ph));
  }
  // device image: [PPhase x n][per phase: args | begins | grids] + barrier + status
  size_t off = (sizeof(PPhase) * phs.size() + 255) / 256 * 256;
  std::vector<size_t> oa(phs.size()), ob(phs.size()), og(phs.size());
  smem = 0;
  for (size_t p = 0; p < phs.size(); ++p) {
    const size_t n = phs[p].parts.size();
    oa[p] = off;
    off += (phs[p].parts[0]->args_size * n + 255) / 256 * 256;
    ob[p] = off;
    off += (sizeof(int) * n + 255) / 256 * 256;
    og[p] = off;
    off += (sizeof(uint3) * n + 255) / 256 * 256;
    for (const LaunchRec* r : phs[p].parts) smem = std::max(smem, r->smem);
  }
  const size_t obar = off;
  off += 256;
  std::vector<unsigned char> img(off, 0);
  if (cudaMalloc(&dev, off) != cudaSuccess) {
    snprintf(err, nerr, "persistent step: cudaMalloc(%zu) failed", off);
    return -2;
  }
  unsigned char* d = static_cast<unsigned char*>(dev);
  for (size_t p = 0; p < phs.size(); ++p) {
    PPhase P{};
    P.kind = phs[p].kind;
    P.nparts = static_cast<int>(phs[p].parts.size());
    P.args_size = static_cast<int>(phs[p].parts[0]->args_size);
    P.args = d + oa[p];
    P.begins = reinterpret_cast<const int*>(d + ob[p]);
    P.grids = reinterpret_cast<const uint3*>(d + og[p]);
    int beg = 0;
    for (size_t q = 0; q < phs[p].parts.size(); ++q) {
      const LaunchRec* r = phs[p].parts[q];
      std::memcpy(img.data() + oa[p] + q * P.args_size, r->args.data(), P.args_size);
      std::memcpy(img.data() + ob[p] + q * sizeof(int), &beg, sizeof(int));
      const uint3 g{r->grid.x, r->grid.y, r->grid.z};
      std::memcpy(img.data() + og[p] + q * sizeof(uint3), &g, sizeof(uint3));
      beg += r->blocks;
    }
    P.blocks = beg;
    std::memcpy(img.data() + p * sizeof(PPhase), &P, sizeof(PPhase));
  }
  if (cudaMemcpy(dev, img.data(), off, cudaMemcpyHostToDevice) != cudaSuccess) {
    snprintf(err, nerr, "persistent step: upload failed");
    return -2;
  }
  bar = reinterpret_cast<unsigned*>(d + obar);
  status = reinterpret_cast<int*>(d + obar + 16);
  nphases = static_cast<int>(phs.size());
  f32 = fp32;
  const void* fn = f32 ? reinterpret_cast<const void*>(&k_persist<float>) : reinterpret_cast<const void*>(&k_persist<double>);
  if (smem > 48 * 1024) smem_optin(fn);
  int dev_id = 0, nsm = 0, per_sm = 0;
  cudaGetDevice(&dev_id);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev_id);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kPersistNT, smem);
  blocks = nsm * std::max(0, per_sm);
  if (blocks < 1) {
    snprintf(err, nerr, "persistent step: no resident block fits (%zu bytes of shared memory)", smem);
    return -1;
  }
  if (cudaMallocHost(&host_status, sizeof(int)) != cudaSuccess) {
    snprintf(err, nerr, "persistent step: host status allocation failed");
    return -2;
  }
  return 0;
}

int PersistProgram::run(int64_t nsteps, cudaStream_t st) {
  const void* fn = f32 ? reinterpret_cast<const void*>(&k_persist<float>) : reinterpret_cast<const void*>(&k_persist<double>);
  const PPhase* ph = static_cast<const PPhase*>(dev);
  unsigned long long spins = barrier_spins();
  int rc = 0;
  if (cudaMemsetAsync(bar, 0, 16 + sizeof(int), st) != cudaSuccess) return 2;
  for (int64_t done = 0; done < nsteps;) {
    // bounded kernels: at most 256 steps a launch
    int n = static_cast<int>(std::min<int64_t>(256, nsteps - done));
    void* args[] = {const_cast<PPhase**>(&ph), &nphases, &n, &bar, &status, &spins};
    if (cudaLaunchCooperativeKernel(fn, dim3(blocks), dim3(kPersistNT), args, smem, st) != cudaSuccess) return 2;
    done += n;
  }
  if (cudaMemcpyAsync(host_status, status, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess) return 2;
  if (cudaStreamSynchronize(st) != cudaSuccess) return 2;
  if (*host_status) rc = 1;
  return rc;
}

}  // namespace mm

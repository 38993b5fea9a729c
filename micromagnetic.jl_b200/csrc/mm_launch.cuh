// mm_launch.cuh -- kernels as descriptors, launched for one mesh or for many
// meshes at once (internal).
//
// A descriptor K holds the kernel's arguments (K::Args, with the grid it was
// sized for), its block size K::kNT, its occupancy hint K::kMinB and a device
// body K::body(args, block index).  k_one<K> runs the body on one mesh's grid;
// k_many<K> runs it over the concatenated grids of several meshes -- block b
// finds its mesh i (begins[i] <= b < begins[i+1]) and its block index within
// that mesh's grid -- so one launch covers a pass of every mesh of a batch.
//
// launch_k<K>() launches k_one<K>, or, while a LaunchRecorder is active on the
// calling thread, appends a record (the arguments as bytes and the grid) that
// the batch builder later merges with the same pass of other meshes.
#pragma once
#include <cuda_runtime.h>

#include <cstring>
#include <vector>

#include "mm_common.cuh"

namespace mm {

template <class K>
__global__ void __launch_bounds__(K::kNT, K::kMinB) k_one(const typename K::Args a) {
  pdl_enter();
  K::body(a, blockIdx);
}

template <class K>
__global__ void __launch_bounds__(K::kNT, K::kMinB) k_many(const typename K::Args* __restrict__ A,
                                                           const int* __restrict__ begins, int n) {
  pdl_enter();
  int lo = 0, hi = n - 1;
  const int b = static_cast<int>(blockIdx.x);
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (begins[mid] <= b) lo = mid;
    else hi = mid - 1;
  }
  // the mesh's arguments are copied to shared memory once: the body reads
  // them often (plans, strides), as k_one reads its parameter bank
  using Args = typename K::Args;
  static_assert(sizeof(Args) % 4 == 0, "argument structs are word multiples");
  __shared__ __align__(16) unsigned char sa[sizeof(Args)];
  {
    const unsigned* src = reinterpret_cast<const unsigned*>(A + lo);
    unsigned* dst = reinterpret_cast<unsigned*>(sa);
    for (int w = threadIdx.x; w < static_cast<int>(sizeof(Args) / 4); w += K::kNT) dst[w] = src[w];
  }
  __syncthreads();
  const Args& a = *reinterpret_cast<const Args*>(sa);
  const unsigned local = static_cast<unsigned>(b - begins[lo]);
  uint3 bid;
  bid.x = local % a.grid.x;
  bid.y = (local / a.grid.x) % a.grid.y;
  bid.z = local / (a.grid.x * a.grid.y);
  K::body(a, bid);
}

// Index of a descriptor in the persistent step kernel's dispatch
// (mm_persist.cu), -1 for descriptors it does not run.
template <class K> struct PersistKind { static constexpr int value = -1; };

// One recorded launch: which kernel (its multi-mesh launcher), its arguments
// and its launch shape.
struct LaunchRec {
  const void* kind;  // identity of the descriptor (k_many<K>)
  int pkind;         // PersistKind<K>::value
  dim3 grid;
  // launches k_many<K> over n meshes whose Args (device) and block offsets
  // (device) are given; total blocks, dynamic shared memory
  cudaError_t (*many)(const void* args_dev, const int* begins_dev, int n, int blocks, size_t smem, cudaStream_t st);
  size_t args_size;
  std::vector<unsigned char> args;
  int blocks;   // grid.x * grid.y * grid.z
  size_t smem;  // dynamic shared memory
};

struct LaunchRecorder {
  std::vector<LaunchRec> recs;
};
LaunchRecorder*& launch_recorder();  // the calling thread's active recorder (null: launch)
// Raises the dynamic shared-memory limit of a kernel to the opt-in maximum,
// once per (kernel, current device).
void smem_optin(const void* kernel);

template <class K>
cudaError_t launch_many(const void* args_dev, const int* begins_dev, int n, int blocks, size_t smem, cudaStream_t st) {
  if (smem > 48 * 1024) smem_optin(reinterpret_cast<const void*>(&k_many<K>));
  // an ordinary launch: with the programmatic attribute the merged NEB batch
  // (32 images of 128 x 128, 16 launches a step) took 0.42 ms a step against
  // 0.36 in paired runs (that batch also varies between the two run to run)
  k_many<K><<<blocks, K::kNT, smem, st>>>(static_cast<const typename K::Args*>(args_dev), begins_dev, n);
  return cudaGetLastError();
}

template <class K>
void launch_k(dim3 grid, size_t smem, cudaStream_t st, typename K::Args a) {
  a.grid = grid;
  if (LaunchRecorder* r = launch_recorder()) {
    LaunchRec rec;
    rec.kind = reinterpret_cast<const void*>(&k_many<K>);
    rec.pkind = PersistKind<K>::value;
    rec.grid = grid;
    rec.many = &launch_many<K>;
    rec.args_size = sizeof(a);
    rec.args.resize(sizeof(a));
    std::memcpy(rec.args.data(), &a, sizeof(a));
    rec.blocks = static_cast<int>(grid.x * grid.y * grid.z);
    rec.smem = smem;
    r->recs.push_back(std::move(rec));
    return;
  }
  if (smem > 48 * 1024) smem_optin(reinterpret_cast<const void*>(&k_one<K>));
  launch_pdl(k_one<K>, grid, dim3(K::kNT), smem, st, a);
}

}  // namespace mm

// mm_noalloc.cu -- mm_energy_noalloc: the energy reduction of the local
// interaction terms without any device allocation.
//
// Who needs it: callers that cannot call cudaMalloc at the point where they
// want energies -- a host that owns the device memory through its own pool
// allocator (a Julia/CUDA.jl or PyTorch caching allocator that must stay the
// only allocator), code on a latency-critical path where cudaMalloc's implicit
// device synchronisation is not acceptable, or an embedding that has no
// handle.  They pass device pointers to the magnetisation and Ms and to a
// 6-double output; the per-block partial sums live in a statically allocated
// device array of this library.
//
// The array holds kNoAllocMaxBlocks x 6 doubles (3 MiB) on every GPU that
// loads the library, until the process exits; meshes are limited to
// kNoAllocMaxCells = 2^24 cells (one 256-thread block per 256 cells).
// Every call writes each partial it later reads, so nothing has to start at
// zero; calls that overlap on the GPU (concurrent streams, devices sharing
// the symbol through peer access) race on the array.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/mmcuda.h"

namespace mm {
int set_last_error(int code, const char* msg);  // mm_api.cu
}

namespace {

constexpr int kNoAllocThreads = 256;
constexpr int64_t kNoAllocMaxCells = int64_t(1) << 24;
constexpr int kNoAllocMaxBlocks = static_cast<int>(kNoAllocMaxCells / kNoAllocThreads);
constexpr double kMu0 = 4.0 * 3.14159265358979323846 * 1e-7;

// shared scratch: per-block partial sums of the six term energies
static __device__ __align__(256) double g_noalloc_partials[kNoAllocMaxBlocks * MM_NTERMS];

struct LocalTerms {
  int nx, ny, nz, pbc;
  double dx, dy, dz;
  double A, D, Ku, ux, uy, uz, Hx, Hy, Hz;
};

// One thread per cell: FP64 energies of exchange, bulk DMI, uniaxial
// anisotropy and Zeeman with uniform parameters (the formulas of
// src/micro/kernels.jl:14-20, 54-75, 269-344), the neighbour test
// "exists and has Ms > 0" evaluated inline; block sums to partials.
__global__ void k_energy_noalloc(LocalTerms t, const double* __restrict__ m, const double* __restrict__ Ms,
                                 double* __restrict__ partials) {
  const int64_t N = static_cast<int64_t>(t.nx) * t.ny * t.nz;
  const int64_t I = blockIdx.x * static_cast<int64_t>(kNoAllocThreads) + threadIdx.x;
  double e[MM_NTERMS] = {0, 0, 0, 0, 0, 0};
  if (I < N) {
    const double V = t.dx * t.dy * t.dz;
    const double ms = Ms[I] * kMu0;
    const double mx = m[I], my = m[N + I], mz = m[2 * N + I];
    if (ms != 0.0) {
      const int nxy = t.nx * t.ny;
      const int i = static_cast<int>(I % t.nx), j = static_cast<int>((I / t.nx) % t.ny),
                k = static_cast<int>(I / nxy);
      const bool px = t.pbc & 1, py = t.pbc & 2, pz = t.pbc & 4;
      int64_t nb[6];
      nb[0] = i > 0 ? I - 1 : (px ? I + t.nx - 1 : -1);
      nb[1] = i < t.nx - 1 ? I + 1 : (px ? I - (t.nx - 1) : -1);
      nb[2] = j > 0 ? I - t.nx : (py ? I + static_cast<int64_t>(t.ny - 1) * t.nx : -1);
      nb[3] = j < t.ny - 1 ? I + t.nx : (py ? I - static_cast<int64_t>(t.ny - 1) * t.nx : -1);
      nb[4] = k > 0 ? I - nxy : (pz ? I + static_cast<int64_t>(t.nz - 1) * nxy : -1);
      nb[5] = k < t.nz - 1 ? I + nxy : (pz ? I - static_cast<int64_t>(t.nz - 1) * nxy : -1);
      const double ex[6] = {2 * t.A / (t.dx * t.dx), 2 * t.A / (t.dx * t.dx), 2 * t.A / (t.dy * t.dy),
                            2 * t.A / (t.dy * t.dy), 2 * t.A / (t.dz * t.dz), 2 * t.A / (t.dz * t.dz)};
      const double Dd[6] = {t.D / t.dx, t.D / t.dx, t.D / t.dy, t.D / t.dy, t.D / t.dz, t.D / t.dz};
      double fx = 0, fy = 0, fz = 0, gx = 0, gy = 0, gz = 0;
      for (int d = 0; d < 6; ++d) {
        const int64_t q = nb[d];
        if (q < 0 || !(Ms[q] > 0.0)) continue;
        const double ax = m[q], ay = m[N + q], az = m[2 * N + q];
        fx += ex[d] * (ax - mx);
        fy += ex[d] * (ay - my);
        fz += ex[d] * (az - mz);
        // a_d x m_d with a = +x,-x,+y,-y,+z,-z for d = -x,+x,-y,+y,-z,+z
        const double s = (d & 1) ? -1.0 : 1.0;
        if (d < 2) { gy += Dd[d] * (-s * az); gz += Dd[d] * (s * ay); }
        else if (d < 4) { gx += Dd[d] * (s * az); gz += Dd[d] * (-s * ax); }
        else { gx += Dd[d] * (-s * ay); gy += Dd[d] * (s * ax); }
      }
      e[MM_TERM_EXCH] = -0.5 * (fx * mx + fy * my + fz * mz) * V;
      e[MM_TERM_DMI_BULK] = -0.5 * (gx * mx + gy * my + gz * mz) * V;
      const double sa = mx * t.ux + my * t.uy + mz * t.uz;
      e[MM_TERM_ANIS] = t.Ku * (1.0 - sa * sa) * V;
    }
    e[MM_TERM_ZEEMAN] = -V * ms * (mx * t.Hx + my * t.Hy + mz * t.Hz);
  }
  __shared__ double sh[kNoAllocThreads];
  for (int c = 0; c < MM_NTERMS; ++c) {
    sh[threadIdx.x] = e[c];
    __syncthreads();
    for (int o = kNoAllocThreads / 2; o > 0; o >>= 1) {
      if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
      __syncthreads();
    }
    if (threadIdx.x == 0) partials[blockIdx.x * MM_NTERMS + c] = sh[0];
    __syncthreads();
  }
}

__global__ void k_energy_noalloc_final(const double* __restrict__ partials, int nblocks, double* __restrict__ out) {
  __shared__ double sh[kNoAllocThreads];
  for (int c = 0; c < MM_NTERMS; ++c) {
    double acc = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += kNoAllocThreads) acc += partials[b * MM_NTERMS + c];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int o = kNoAllocThreads / 2; o > 0; o >>= 1) {
      if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
      __syncthreads();
    }
    if (threadIdx.x == 0) out[c] = sh[0];
    __syncthreads();
  }
}

// Device address of the static scratch in the current context.  It is looked
// up on every call (cudaGetSymbolAddress is a host-side lookup and allocates
// nothing): a cached address would go stale when the host resets or re-creates
// the primary context (cudaDeviceReset, CUDA.jl's device_reset!), which reloads
// the module and its array at another address.  The host-side name of the
// array is not a device address and is never passed to a kernel.
int scratch_for_current_device(double** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
  if (e != cudaSuccess) return mm::set_last_error(MM_ERR_CUDA, cudaGetErrorString(e));
  *out = static_cast<double*>(p);
  return MM_OK;
}

}  // namespace

extern "C" int mm_energy_noalloc(const mm_mesh_desc* mesh, const double* m_soa_dev, const double* Ms_dev, double A,
                                 double D, double Ku, double ax, double ay, double az, double Hx, double Hy, double Hz,
                                 double* energies_dev, void* stream) {
  if (!mesh || !m_soa_dev || !Ms_dev || !energies_dev)
    return mm::set_last_error(MM_ERR_ARG, "mm_energy_noalloc: null argument");
  if (mesh->nx < 1 || mesh->ny < 1 || mesh->nz < 1 || !(mesh->dx > 0) || !(mesh->dy > 0) || !(mesh->dz > 0))
    return mm::set_last_error(MM_ERR_ARG, "mm_energy_noalloc: bad mesh");
  const int64_t N = static_cast<int64_t>(mesh->nx) * mesh->ny * mesh->nz;
  if (N > kNoAllocMaxCells) {
    char msg[160];
    snprintf(msg, sizeof(msg), "mm_energy_noalloc: %lld cells exceed the static scratch limit of %lld cells",
             static_cast<long long>(N), static_cast<long long>(kNoAllocMaxCells));
    return mm::set_last_error(MM_ERR_ARG, msg);
  }
  const double lt = std::sqrt(ax * ax + ay * ay + az * az);
  if (Ku != 0.0 && !(lt > 0)) return mm::set_last_error(MM_ERR_ARG, "mm_energy_noalloc: zero anisotropy axis");
  double* partials = nullptr;
  if (int rc = scratch_for_current_device(&partials)) return rc;
  LocalTerms t{mesh->nx, mesh->ny, mesh->nz, mesh->pbc, mesh->dx, mesh->dy, mesh->dz, A, D, Ku,
               lt > 0 ? ax / lt : 0.0, lt > 0 ? ay / lt : 0.0, lt > 0 ? az / lt : 0.0, Hx, Hy, Hz};
  const int nblocks = static_cast<int>((N + kNoAllocThreads - 1) / kNoAllocThreads);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_energy_noalloc<<<nblocks, kNoAllocThreads, 0, st>>>(t, m_soa_dev, Ms_dev, partials);
  k_energy_noalloc_final<<<1, kNoAllocThreads, 0, st>>>(partials, nblocks, energies_dev);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return mm::set_last_error(MM_ERR_CUDA, cudaGetErrorString(e));
  return MM_OK;
}

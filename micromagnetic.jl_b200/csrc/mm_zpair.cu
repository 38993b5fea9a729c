// mm_zpair.cu -- register-resident z convolution for Pz = 32 (nz <= 16), FP32.
//
// The z step of the demag convolution (src/micro/demag.jl:114-123: forward
// FFT along z, the 6-component tensor product, inverse FFT along z) for one
// (kx, ky) line of the three components.  With the line zero-padded from
// nz <= 16 to 32 points, the forward transform splits by output parity,
//     X[2k + s] = sum_{n<16} (x[n] w32^(n s)) w16^(n k),   s = 0, 1,
// and the kept half of the inverse (z < 16) recombines the two halves,
//     y[n] = u0[n] + w32^(-n) u1[n],   us = DFT16^-1(X[2k + s]),
// so the pair of threads (s = 0, 1) of a line each run 16-point transforms on
// 16 values a component held in registers, apply the tensor at their 16 kz,
// and exchange half of their results once (shfl.xor 16).  Each thread issues
// its 48 row loads up front; the block's tensor entries arrive in shared
// memory meanwhile -- by one tiled bulk copy through a tensor map
// (cp.async.bulk.tensor, completion counted on an mbarrier; column-major
// spectra) or by cp.async (row-major) -- with one barrier before the product.
//
// Lanes: t = lane & 15 is the line within the warp, s = lane >> 4 the half.
// A block of 8 warps takes 128 consecutive lines along the fastest spectrum
// index: ky of one kx column (column-major spectra, DemagGeom::yT) or kx of
// one ky row (row-major).
#include <cuda.h>
#include <cudaTypedefs.h>

#include <cstdlib>
#include <cstring>

#include "mm_demag.cuh"
#include "mm_fft.cuh"
#include "mm_launch.cuh"

namespace mm {

namespace {

constexpr int kZpNT = 256;
constexpr int kZpLines = kZpNT / 2;  // lines per block
// Shared tensor row (one component, one kz quadrant row, the block's 128
// lines) padded by 16 floats: the two halves of a thread pair read rows kzq
// and kzq +/- 1, which then fall 16 banks apart.
constexpr int kZpRow = kZpLines + 16;
constexpr int kZpTzq = 17;  // kz quadrant rows of Pz = 32

// tensor entries a block stages: 6 components x 17 kz quadrant rows x the
// block's 128 lines (their ky mirror index, or kx, is one contiguous run)
constexpr int kZpTensor = 6 * kZpTzq * kZpRow;

// ky width of the tiled copy of a column-major block: its 128 lines map to a
// contiguous run of at most 128 tensor rows (ascending, or descending past
// Py / 2), which starts up to 3 entries after the 16-byte-aligned copy start
static_assert(kZpRow >= kZpLines + 3, "tensor box holds the block's rows");
constexpr unsigned kZpBoxBytes = 6u * kZpTzq * kZpRow * sizeof(float);
constexpr unsigned kZpDrainSpins = 1u << 24;
__device__ int g_zpair_timeout;

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
// bounded wait of every thread of the block on the slice's mbarrier, with
// one outcome for all; on a timeout the copy in flight is drained first
__device__ __forceinline__ bool slice_wait(unsigned long long* bar, unsigned spins) {
  const unsigned a = smem_addr(bar);
  bool ok = false;
  for (unsigned i = 0; i < spins && !ok; ++i) {
    unsigned r;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(r)
        : "r"(a)
        : "memory");
    ok = r != 0;
  }
  if (__syncthreads_or(!ok)) {
    if (threadIdx.x == 0) atomicExch(&g_zpair_timeout, 1);
    for (unsigned i = 0; i < kZpDrainSpins; ++i) {
      unsigned r;
      asm volatile(
          "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n selp.u32 %0, 1, 0, p;\n}\n"
          : "=r"(r)
          : "r"(a)
          : "memory");
      if (r) break;
    }
    return false;
  }
  return true;
}

__device__ __forceinline__ void cp_async4(float* smem, const float* gmem) {
  const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(a), "l"(gmem));
}

// FULL: nz = 16 and every line of every block is live (column-major, Py a
// multiple of 128), so no load or store is predicated
template <bool YT, bool FULL>
__global__ void __launch_bounds__(kZpNT, 2) k_zpair(float2* __restrict__ Y, const float* __restrict__ Nhat, DemagGeom g,
                                                    const __grid_constant__ CUtensorMap tmap, unsigned spins) {
  using C = float2;
  extern __shared__ __align__(128) float tn[];  // kZpTensor entries, then the mbarrier (YT)
  pdl_enter();
  if (g.gate && !*g.gate) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int t = lane & 15, s = lane >> 4;
  const int Hx = g.Hx, Py = g.Py, nz = g.nz, Tyq = g.Tyq;
  const int line0 = blockIdx.x * kZpLines;
  const int line = line0 + warp * 16 + t;
  int kx, ky;
  if (YT) {
    kx = blockIdx.y;
    ky = line;
  } else {
    ky = blockIdx.y;
    kx = line;
  }
  const bool live = FULL || (YT ? ky < Py : kx < Hx);
  // The block's tensor entries: entry (c6, kzq) of block line l at
  // tn[(c6 * 17 + kzq) * kZpRow + col(l)], from the tensor row of line l's
  // mirror index (ky or Py - ky, column-major) or its kx, in flight while the
  // rows load and the forward transforms run.
  int col;           // this thread's line's column in the shared rows
  unsigned long long* bar = nullptr;
  if constexpr (YT) {
    // one tiled bulk copy of the box {kZpRow ky, 1 kx, 17 kz, 6 c} starting
    // at the 16-byte-aligned ky0 at or below the block's smallest row index
    const int nl = min(kZpLines, Py - line0);
    const int last = line0 + nl - 1;
    const int kmin = last <= Py / 2 ? line0 : min(line0, Py - last);
    const int ky0 = kmin & ~3;
    col = (ky > Py / 2 ? Py - ky : ky) - ky0;
    bar = reinterpret_cast<unsigned long long*>(tn + kZpTensor);
    if (threadIdx.x == 0) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_addr(bar)) : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(kZpBoxBytes)
                   : "memory");
      asm volatile(
          "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
          "[%6];\n" ::"r"(smem_addr(tn)),
          "l"(reinterpret_cast<unsigned long long>(&tmap)), "r"(ky0), "r"(kx), "r"(0), "r"(0), "r"(smem_addr(bar))
          : "memory");
    }
    __syncthreads();  // the mbarrier is initialised before anyone waits on it
  } else {
    // cp.async: thread (l, h) copies line l's entries of components 3h .. 3h + 2
    col = line - line0;
    const int l = threadIdx.x & (kZpLines - 1), h = threadIdx.x >> 7;
    if (l < Hx - line0) {
      const int64_t Ts = static_cast<int64_t>(kZpTzq) * Tyq * Hx;  // component stride
      const int64_t kzs = static_cast<int64_t>(Tyq) * Hx;            // kz quadrant row stride
      const int64_t off = static_cast<int64_t>(ky > Py / 2 ? Py - ky : ky) * Hx + line0 + l;
      const float* src = Nhat + 3 * h * Ts + off;
      float* dst = tn + 3 * h * kZpTzq * kZpRow + l;
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const float* sp = src + j * Ts;
#pragma unroll
        for (int kzq = 0; kzq < kZpTzq; ++kzq) {
          cp_async4(dst + (j * kZpTzq + kzq) * kZpRow, sp);
          sp += kzs;
        }
      }
    }
    asm volatile("cp.async.commit_group;\n" ::);
  }
  // element (c, z) of this line
  const int64_t cs = static_cast<int64_t>(nz) * Py * Hx;  // component stride
  const int64_t zs = YT ? Py : static_cast<int64_t>(Py) * Hx;
  const int64_t base = YT ? static_cast<int64_t>(kx) * nz * Py + ky : static_cast<int64_t>(ky) * Hx + kx;
  // YT: component c starts at c*Hx*nz*Py = c*cs as well
  C v[3][16];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int n = 0; n < 16; ++n) {
      if constexpr (FULL)
        v[c][n] = Y[c * cs + n * zs + base];
      else
        v[c][n] = (live && n < nz) ? Y[c * cs + n * zs + base] : make_float2(0.f, 0.f);
    }
  // forward: x[n] w32^(n s), DFT16 -> X[2k + s]
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    if (s) {
#pragma unroll
      for (int n = 1; n < 16; ++n) {
        const float wr = static_cast<float>(w32_cs(n, 0)), wi = -static_cast<float>(w32_cs(n, 1));
        v[c][n] = cmul(v[c][n], make_float2(wr, wi));
      }
    }
    dft16<false>(v[c]);
  }
  if constexpr (YT) {
    if (!slice_wait(bar, spins)) return;
  } else {
    asm volatile("cp.async.wait_group 0;\n" ::);
    __syncthreads();
  }
  // tensor product at kz = 2k + s (one quadrant stored; xy odd in ky, xz in
  // kz, yz in both): kz <= 15 for k < 8 (kzq = kz), kz >= 18 for k > 8
  // (kzq = 32 - kz, xz and yz negated), and k = 8 gives kz = 16 (s = 0) or
  // the mirrored 17 -> 15 (s = 1).  The odd half also takes (-1)^k, which
  // rotates its inverse transform by 8: register r then holds u1[(r + 8) % 16]
  // and both halves keep registers 0..7 and send 8..15 (no selects).
  if (live) {
    const float sy = ky > Py / 2 ? -1.f : 1.f;
    const float so = s ? -1.f : 1.f, syo = sy * so;
    const float* lo = tn + s * kZpRow + col;          // row s (+ 2k)
    const float* hi = tn + (16 - s) * kZpRow + col;   // row 16 - s (+ 16 - 2k)
    constexpr int cr = kZpTzq * kZpRow;             // component stride
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const float* tb = k < 8 ? lo + 2 * k * kZpRow : hi + (16 - 2 * k) * kZpRow;
      float xx = tb[0], yy = tb[cr], zz = tb[2 * cr], xy, xz, yz;
      if (k & 1) {  // odd k: never 8, so the kz sign is fixed
        const float szk = k < 8 ? 1.f : -1.f;
        xx *= so;
        yy *= so;
        zz *= so;
        xy = syo * tb[3 * cr];
        xz = (szk * so) * tb[4 * cr];
        yz = (syo * szk) * tb[5 * cr];
      } else {
        const float sz = k < 8 ? 1.f : (k > 8 ? -1.f : (s ? -1.f : 1.f));
        xy = sy * tb[3 * cr];
        xz = sz * tb[4 * cr];
        yz = sy * sz * tb[5 * cr];
      }
      const C p0 = v[0][k], p1 = v[1][k], p2 = v[2][k];
      v[0][k] = make_float2(xx * p0.x + xy * p1.x + xz * p2.x, xx * p0.y + xy * p1.y + xz * p2.y);
      v[1][k] = make_float2(xy * p0.x + yy * p1.x + yz * p2.x, xy * p0.y + yy * p1.y + yz * p2.y);
      v[2][k] = make_float2(xz * p0.x + yz * p1.x + zz * p2.x, xz * p0.y + yz * p1.y + zz * p2.y);
    }
  }
  // inverse: u_s = DFT16^-1(X[2k + s]); the odd half (rotated by 8) is
  // twiddled by w32^(-n), n = (r + 8) % 16 in register r
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    dft16<true>(v[c]);
    if (s) {
#pragma unroll
      for (int r = 0; r < 16; ++r) {
        const int n = (r + 8) & 15;
        if (n == 0) continue;
        const float wr = static_cast<float>(w32_cs(n, 0)), wi = static_cast<float>(w32_cs(n, 1));
        v[c][r] = cmul(v[c][r], make_float2(wr, wi));
      }
    }
  }
  // y[z] = u0[z] + w32^(-z) u1[z]: the s = 0 thread keeps z < 8 (registers
  // 0..7 of u0), the s = 1 thread z >= 8 (registers 0..7 of the rotated u1);
  // each sends registers 8..15 to its partner (lane ^ 16)
#pragma unroll
  for (int c = 0; c < 3; ++c) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const C mine = v[c][i], send = v[c][8 + i];
      const float rx = __shfl_xor_sync(0xffffffffu, send.x, 16);
      const float ry = __shfl_xor_sync(0xffffffffu, send.y, 16);
      const int z = i + 8 * s;
      if (FULL || (live && z < nz)) Y[c * cs + z * zs + base] = make_float2(mine.x + rx, mine.y + ry);
    }
  }
}

}  // namespace

bool zpair_applies(const DemagGeom& g) { return g.Pz == 32 && g.Tzq == kZpTzq && g.nz <= 16 && g.nz >= 1; }

unsigned copy_wait_spins() {
  static const unsigned v = [] {
    const char* e = getenv("MMCUDA_COPY_SPINS");
    return e ? static_cast<unsigned>(strtoul(e, nullptr, 10)) : (1u << 22);
  }();
  return v;
}

bool zpair_take_timeout() {
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, g_zpair_timeout, sizeof(int)) != cudaSuccess || !v) return false;
  const int zero = 0;
  cudaMemcpyToSymbol(g_zpair_timeout, &zero, sizeof(int));
  return true;
}

// Nhat[((c*17 + kz)*Hx + kx)*Tys + ky] as a 4-D FP32 tensor (ky fastest,
// extent Tyq: the zero padding up to Tys is never read), box {kZpRow, 1, 17, 6}
bool zpair_tensor_map(const DemagGeom& g, const float* Nhat, void* map128) {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return static_cast<PFN_cuTensorMapEncodeTiled_v12000>(nullptr);
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }();
  if (!encode || (g.Tys & 3) || (reinterpret_cast<uintptr_t>(Nhat) & 15)) return false;
  const cuuint64_t dims[4] = {static_cast<cuuint64_t>(g.Tyq), static_cast<cuuint64_t>(g.Hx),
                              static_cast<cuuint64_t>(kZpTzq), 6};
  const cuuint64_t row = static_cast<cuuint64_t>(g.Tys) * sizeof(float);
  const cuuint64_t strides[3] = {row, row * g.Hx, row * g.Hx * kZpTzq};
  const cuuint32_t box[4] = {static_cast<cuuint32_t>(kZpRow), 1, static_cast<cuuint32_t>(kZpTzq), 6};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  CUtensorMap m;
  std::memset(&m, 0, sizeof(m));
  const CUresult r = encode(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<float*>(Nhat), dims, strides, box, estr,
                            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return false;
  static_assert(sizeof(CUtensorMap) == 128, "tensor map size");
  std::memcpy(map128, &m, sizeof(m));
  return true;
}

void launch_zpair_f32(const DemagGeom& g, float2* Y, const float* Nhat, const void* map128, cudaStream_t st) {
  CUtensorMap m;
  std::memcpy(&m, map128, sizeof(m));
  if (g.yT) {
    const size_t sm = sizeof(float) * kZpTensor + 16;  // + the mbarrier
    dim3 grid((g.Py + kZpLines - 1) / kZpLines, g.Hx, 1);
    if (g.nz == 16 && g.Py % kZpLines == 0) {
      smem_optin(reinterpret_cast<const void*>(&k_zpair<true, true>));
      launch_pdl(k_zpair<true, true>, grid, dim3(kZpNT), sm, st, Y, Nhat, g, m, copy_wait_spins());
    } else {
      smem_optin(reinterpret_cast<const void*>(&k_zpair<true, false>));
      launch_pdl(k_zpair<true, false>, grid, dim3(kZpNT), sm, st, Y, Nhat, g, m, copy_wait_spins());
    }
  } else {
    const size_t sm = sizeof(float) * kZpTensor;
    smem_optin(reinterpret_cast<const void*>(&k_zpair<false, false>));
    dim3 grid((g.Hx + kZpLines - 1) / kZpLines, g.Py, 1);
    launch_pdl(k_zpair<false, false>, grid, dim3(kZpNT), sm, st, Y, Nhat, g, m, copy_wait_spins());
  }
}

}  // namespace mm

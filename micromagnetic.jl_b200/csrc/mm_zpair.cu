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
// its 48 row loads up front; the block's tensor entries are prefetched into
// shared memory (cp.async) meanwhile, with one barrier before the product.
//
// Lanes: t = lane & 15 is the line within the warp, s = lane >> 4 the half.
// A block of 8 warps takes 128 consecutive lines along the fastest spectrum
// index: ky of one kx column (column-major spectra, DemagGeom::yT) or kx of
// one ky row (row-major).
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

__device__ __forceinline__ void cp_async4(float* smem, const float* gmem) {
  const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(a), "l"(gmem));
}

template <bool YT>
__global__ void __launch_bounds__(kZpNT, 2) k_zpair(float2* __restrict__ Y, const float* __restrict__ Nhat, DemagGeom g) {
  using C = float2;
  extern __shared__ __align__(16) float tn[];  // kZpTensor entries
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
  const bool live = YT ? ky < Py : kx < Hx;
  // Prefetch the block's tensor entries into shared memory (cp.async), in
  // flight while the rows load and the forward transforms run: entry
  // (c6, kzq) of block line l at tn[(c6 * 17 + kzq) * kZpRow + l], from the
  // tensor row of line l's mirror index (ky or Py - ky, column-major) or kx.
  // Thread (l, h) copies line l's entries of components 3h .. 3h + 2.
  {
    const int l = threadIdx.x & (kZpLines - 1), h = threadIdx.x >> 7;
    if (l < (YT ? Py : Hx) - line0) {
      const int64_t Ts = static_cast<int64_t>(kZpTzq) * Tyq * Hx;  // component stride
      const int64_t kzs = static_cast<int64_t>(Tyq) * Hx;            // kz quadrant row stride
      int64_t off;
      if (YT) {
        const int kyl = line0 + l;
        off = static_cast<int64_t>(kx) * Tyq + (kyl > Py / 2 ? Py - kyl : kyl);
      } else {
        off = static_cast<int64_t>(ky > Py / 2 ? Py - ky : ky) * Hx + line0 + l;
      }
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
    for (int n = 0; n < 16; ++n) v[c][n] = (live && n < nz) ? Y[c * cs + n * zs + base] : make_float2(0.f, 0.f);
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
  asm volatile("cp.async.wait_group 0;\n" ::);
  __syncthreads();
  // tensor product at kz = 2k + s (one quadrant stored; xy odd in ky, xz in
  // kz, yz in both): kz <= 15 for k < 8 (kzq = kz), kz >= 18 for k > 8
  // (kzq = 32 - kz, xz and yz negated), and k = 8 gives kz = 16 (s = 0) or
  // the mirrored 17 -> 15 (s = 1)
  if (live) {
    const float sy = ky > Py / 2 ? -1.f : 1.f;
    const int l = line - line0;
    const float* lo = tn + s * kZpRow + l;          // row s (+ 2k)
    const float* hi = tn + (16 - s) * kZpRow + l;   // row 16 - s (+ 16 - 2k)
    constexpr int cr = kZpTzq * kZpRow;             // component stride
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const float* tb = k < 8 ? lo + 2 * k * kZpRow : hi + (16 - 2 * k) * kZpRow;
      const float sz = k < 8 ? 1.f : (k > 8 ? -1.f : (s ? -1.f : 1.f));
      const float xx = tb[0], yy = tb[cr], zz = tb[2 * cr];
      const float xy = sy * tb[3 * cr], xz = sz * tb[4 * cr], yz = sy * sz * tb[5 * cr];
      const C p0 = v[0][k], p1 = v[1][k], p2 = v[2][k];
      v[0][k] = make_float2(xx * p0.x + xy * p1.x + xz * p2.x, xx * p0.y + xy * p1.y + xz * p2.y);
      v[1][k] = make_float2(xy * p0.x + yy * p1.x + yz * p2.x, xy * p0.y + yy * p1.y + yz * p2.y);
      v[2][k] = make_float2(xz * p0.x + yz * p1.x + zz * p2.x, xz * p0.y + yz * p1.y + zz * p2.y);
    }
  }
  // inverse: u_s = DFT16^-1(X[2k + s]); the odd half is twiddled by w32^(-n)
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    dft16<true>(v[c]);
    if (s) {
#pragma unroll
      for (int n = 1; n < 16; ++n) {
        const float wr = static_cast<float>(w32_cs(n, 0)), wi = static_cast<float>(w32_cs(n, 1));
        v[c][n] = cmul(v[c][n], make_float2(wr, wi));
      }
    }
  }
  // y[n] = u0[n] + w32^(-n) u1[n]: the s = 0 thread keeps n < 8, the s = 1
  // thread n >= 8; each sends the other half to its partner (lane ^ 16)
#pragma unroll
  for (int c = 0; c < 3; ++c) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const C mine = s ? v[c][8 + i] : v[c][i];
      const C send = s ? v[c][i] : v[c][8 + i];
      const float rx = __shfl_xor_sync(0xffffffffu, send.x, 16);
      const float ry = __shfl_xor_sync(0xffffffffu, send.y, 16);
      const int z = i + 8 * s;
      if (live && z < nz) Y[c * cs + z * zs + base] = make_float2(mine.x + rx, mine.y + ry);
    }
  }
}

}  // namespace

bool zpair_applies(const DemagGeom& g) { return g.Pz == 32 && g.Tzq == kZpTzq && g.nz <= 16 && g.nz >= 1; }

void launch_zpair_f32(const DemagGeom& g, float2* Y, const float* Nhat, cudaStream_t st) {
  const size_t sm = sizeof(float) * kZpTensor;
  if (g.yT) {
    smem_optin(reinterpret_cast<const void*>(&k_zpair<true>));
    dim3 grid((g.Py + kZpLines - 1) / kZpLines, g.Hx, 1);
    k_zpair<true><<<grid, kZpNT, sm, st>>>(Y, Nhat, g);
  } else {
    smem_optin(reinterpret_cast<const void*>(&k_zpair<false>));
    dim3 grid((g.Hx + kZpLines - 1) / kZpLines, g.Py, 1);
    k_zpair<false><<<grid, kZpNT, sm, st>>>(Y, Nhat, g);
  }
}

}  // namespace mm

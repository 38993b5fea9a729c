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

// tensor entries a block uses: 6 components x 17 kz quadrant rows x the
// block's 128 lines (their ky mirror index, or kx, is one contiguous run)
constexpr int kZpTensor = 6 * 17 * kZpLines;

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
  const int Hx = g.Hx, Py = g.Py, nz = g.nz, Tyq = g.Tyq, Tzq = g.Tzq;
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
  const int64_t Ts = static_cast<int64_t>(Tzq) * Tyq * Hx;
  // Prefetch the block's tensor entries into shared memory (cp.async), in
  // flight while the rows load and the forward transforms run: entry
  // (c6 * 17 + kzq, line l) at tn[(c6 * 17 + kzq) * 128 + l], the tensor row
  // of line l's mirror index (ky or Py - ky, column-major) or its kx.
  {
    const int nlines = min(kZpLines, (YT ? Py : Hx) - line0);
    for (int e = threadIdx.x; e < 6 * 17 * kZpLines; e += kZpNT) {
      const int r = e / kZpLines, l = e - r * kZpLines;  // r = c6 * 17 + kzq
      if (l >= nlines) continue;
      const int c6 = r / 17, kzq = r - c6 * 17;
      if (kzq >= Tzq) continue;
      int64_t src;
      if (YT) {
        const int kyl = line0 + l;
        const int kyq = kyl > Py / 2 ? Py - kyl : kyl;
        src = c6 * Ts + (static_cast<int64_t>(kzq) * Hx + kx) * Tyq + kyq;
      } else {
        const int kyq = ky > Py / 2 ? Py - ky : ky;
        src = c6 * Ts + (static_cast<int64_t>(kzq) * Tyq + kyq) * Hx + line0 + l;
      }
      cp_async4(tn + e, Nhat + src);
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
        const float wr = static_cast<float>(c_w32[n][0]), wi = -static_cast<float>(c_w32[n][1]);
        v[c][n] = cmul(v[c][n], make_float2(wr, wi));
      }
    }
    dft16<false>(v[c]);
  }
  asm volatile("cp.async.wait_group 0;\n" ::);
  __syncthreads();
  // tensor product at kz = 2k + s (one quadrant stored; xy odd in ky, xz in
  // kz, yz in both)
  if (live) {
    const bool fy = ky > Py / 2;
    const float sy = fy ? -1.f : 1.f;
    const int l = line - line0;
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const int kz = 2 * k + s;
      const bool fz = kz > 16;
      const int kzq = fz ? 32 - kz : kz;
      const float sz = fz ? -1.f : 1.f;
      const float* tb = tn + kzq * kZpLines + l;
      constexpr int cs = 17 * kZpLines;
      const float xx = tb[0], yy = tb[cs], zz = tb[2 * cs];
      const float xy = sy * tb[3 * cs], xz = sz * tb[4 * cs], yz = sy * sz * tb[5 * cs];
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
        const float wr = static_cast<float>(c_w32[n][0]), wi = static_cast<float>(c_w32[n][1]);
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

bool zpair_applies(const DemagGeom& g) { return g.Pz == 32 && g.nz <= 16 && g.nz >= 1; }

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

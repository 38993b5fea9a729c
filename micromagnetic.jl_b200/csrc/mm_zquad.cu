// mm_zquad.cu -- register-resident z convolution for Pz = 32 (nz <= 16), FP64,
// column-major spectra (DemagGeom::yT).
//
// The z step of the demag convolution (src/micro/demag.jl:114-123: forward
// FFT along z, the 6-component tensor product, inverse FFT along z) for one
// (kx, ky) line of the three components, split over four threads by output
// residue S = kz mod 4.  With the line zero-padded from nz <= 16 to 32 points,
//     X[4k + S] = DFT8(a_S)[k],  a_S[m] = w32^(m S) (x[m] + (-i)^S x[m + 8]),
// so thread S folds its line to 8 values a component and runs one 8-point
// transform; it applies the tensor at its 8 kz; its inverse 8-point transform
// gives u_S, and the kept outputs z < 16 are
//     y[m] = sum_S w32^(-m S) u_S[m],  y[m + 8] = sum_S i^S w32^(-m S) u_S[m],
// which the four threads of a line combine through shared memory, each
// producing z = m and m + 8 for its two m.  S is uniform in a warp (warp w of
// a block takes S = w and the block's 32 lines, one a lane), so every
// twiddle and tensor row index is a compile-time constant of that warp's
// code path; the four warps read the same rows (one HBM read, the others hit
// L1), and each load or store instruction moves 32 consecutive ky (512
// bytes).  A block takes 32 ky lines of one kx column; consecutive blocks
// take a ky tile and its mirror, which read the same tensor rows.
#include <cstdlib>

#include "mm_demag.cuh"
#include "mm_fft.cuh"
#include "mm_launch.cuh"

namespace mm {

namespace {

constexpr int kZqNT = 128;   // four warps: S = 0..3
constexpr int kZqLines = 32;  // ky lines per block
constexpr int kZqTzq = 17;    // kz quadrant rows of Pz = 32
// the exchange tile: [c][m][S][line] complex values
constexpr size_t kZqSmem = 3 * 8 * 4 * kZqLines * sizeof(double2);

// w32^j (forward: exp(-2 pi i j / 32); INV: its conjugate), j fixed at compile time
template <bool INV>
__device__ __forceinline__ double2 w32c(int j) {
  j &= 31;
  const double c = j < 16 ? w32_cs(j, 0) : -w32_cs(j - 16, 0);
  const double s = j < 16 ? w32_cs(j, 1) : -w32_cs(j - 16, 1);
  return make_double2(c, INV ? s : -s);
}

// (-i)^S a (forward) or i^S a
template <int S, bool INV>
__device__ __forceinline__ double2 rot4(double2 a) {
  constexpr int e = INV ? (4 - S) & 3 : S;  // power of -i
  if constexpr (e == 0) return a;
  else if constexpr (e == 1) return make_double2(a.y, -a.x);
  else if constexpr (e == 2) return make_double2(-a.x, -a.y);
  else return make_double2(-a.y, a.x);
}

// Thread S of a line: forward fold and transform, tensor product, inverse
// transform; its twiddled u_S goes to the exchange tile.
template <int S, bool FULL>
__device__ __forceinline__ void zquad_line(const double2* __restrict__ Y, const double* __restrict__ Nhat,
                                           const DemagGeom& g, int kx, int ky, bool live, double2* __restrict__ xs,
                                           int l) {
  const int Hx = g.Hx, Py = g.Py, nz = g.nz;
  const int64_t cs = static_cast<int64_t>(nz) * Py * Hx;  // component stride
  const int64_t base = static_cast<int64_t>(kx) * nz * Py + ky;
  double2 v[3][8];
  // forward: fold to 8 values, twiddle by w32^(m S), DFT8 -> X[4k + S]
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    double2 x[16];
#pragma unroll
    for (int n = 0; n < 16; ++n) {
      if constexpr (FULL)
        x[n] = Y[c * cs + n * Py + base];
      else
        x[n] = (live && n < nz) ? Y[c * cs + n * Py + base] : make_double2(0.0, 0.0);
    }
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const double2 a = cadd(x[m], rot4<S, false>(x[m + 8]));
      v[c][m] = (m * S) % 32 == 0 ? a : cmul(a, w32c<false>(m * S));
    }
    dft8<false>(v[c]);
  }
  // tensor product at kz = 4k + S (one quadrant stored: xy odd in ky, xz in
  // kz, yz in both; kz = 16 is its own mirror)
  if (live) {
    const int Tys = g.Tys;
    const int64_t Ts = static_cast<int64_t>(kZqTzq) * Hx * Tys;  // tensor component stride
    const bool fy = ky > Py / 2;
    const double sy = fy ? -1.0 : 1.0;
    const double* tb = Nhat + static_cast<int64_t>(kx) * Tys + (fy ? Py - ky : ky);
    const int64_t kzs = static_cast<int64_t>(Hx) * Tys;  // kz quadrant row stride
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int kz = 4 * k + S;
      const int kzq = kz > 16 ? 32 - kz : kz;
      const double sz = kz > 16 ? -1.0 : 1.0;
      const double* t = tb + kzq * kzs;
      const double xx = __ldg(t), yy = __ldg(t + Ts), zz = __ldg(t + 2 * Ts);
      const double xy = sy * __ldg(t + 3 * Ts), xz = sz * __ldg(t + 4 * Ts), yz = sy * sz * __ldg(t + 5 * Ts);
      const double2 p0 = v[0][k], p1 = v[1][k], p2 = v[2][k];
      v[0][k] = make_double2(xx * p0.x + xy * p1.x + xz * p2.x, xx * p0.y + xy * p1.y + xz * p2.y);
      v[1][k] = make_double2(xy * p0.x + yy * p1.x + yz * p2.x, xy * p0.y + yy * p1.y + yz * p2.y);
      v[2][k] = make_double2(xz * p0.x + yz * p1.x + zz * p2.x, xz * p0.y + yz * p1.y + zz * p2.y);
    }
  }
  // inverse: u_S = DFT8^-1(X[4k + S]), twiddled by w32^(-m S), to the tile
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    dft8<true>(v[c]);
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const double2 u = (m * S) % 32 == 0 ? v[c][m] : cmul(v[c][m], w32c<true>(m * S));
      xs[((c * 8 + m) * 4 + S) * kZqLines + l] = u;
    }
  }
}

// After the block's barrier: y[m] = sum_s z_s[m] and y[m + 8] = sum_s i^s
// z_s[m] for this thread's m = 2S, 2S + 1
template <bool FULL>
__device__ __forceinline__ void zquad_out(double2* __restrict__ Y, const DemagGeom& g, int S, int kx, int ky,
                                          const double2* __restrict__ xs, int l) {
  const int Hx = g.Hx, Py = g.Py, nz = g.nz;
  const int64_t cs = static_cast<int64_t>(nz) * Py * Hx;
  const int64_t base = static_cast<int64_t>(kx) * nz * Py + ky;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int m = 2 * S + h;
      const double2* zq = xs + ((c * 8 + m) * 4) * kZqLines + l;
      const double2 z0 = zq[0], z1 = zq[kZqLines], z2 = zq[2 * kZqLines], z3 = zq[3 * kZqLines];
      const double2 lo = make_double2((z0.x + z1.x) + (z2.x + z3.x), (z0.y + z1.y) + (z2.y + z3.y));
      // i^s z_s: z0 + i z1 - z2 - i z3
      const double2 hi = make_double2((z0.x - z1.y) - (z2.x - z3.y), (z0.y + z1.x) - (z2.y + z3.x));
      if (FULL || m < nz) Y[c * cs + m * Py + base] = lo;
      if (FULL || m + 8 < nz) Y[c * cs + (m + 8) * Py + base] = hi;
    }
  }
}

// FULL: nz = 16 and Py a multiple of the block's lines: no predicated access
template <bool FULL>
__global__ void __launch_bounds__(kZqNT, 2) k_zquad(double2* __restrict__ Y, const double* __restrict__ Nhat,
                                                    DemagGeom g) {
  extern __shared__ __align__(16) unsigned char zq_raw[];
  double2* xs = reinterpret_cast<double2*>(zq_raw);
  pdl_enter();
  if (g.gate && !*g.gate) return;
  const int l = threadIdx.x & 31, S = threadIdx.x >> 5;
  const int nq = gridDim.x, bq = blockIdx.x;
  const int tile = (bq & 1) ? nq - 1 - (bq >> 1) : (bq >> 1);  // a ky tile next to its mirror
  const int kx = blockIdx.y, ky = tile * kZqLines + l;
  const bool live = FULL || ky < g.Py;
  switch (S) {  // uniform in a warp
    case 0: zquad_line<0, FULL>(Y, Nhat, g, kx, ky, live, xs, l); break;
    case 1: zquad_line<1, FULL>(Y, Nhat, g, kx, ky, live, xs, l); break;
    case 2: zquad_line<2, FULL>(Y, Nhat, g, kx, ky, live, xs, l); break;
    default: zquad_line<3, FULL>(Y, Nhat, g, kx, ky, live, xs, l); break;
  }
  __syncthreads();  // the four threads of every line have written their u_S
  if (live) zquad_out<FULL>(Y, g, S, kx, ky, xs, l);
}

}  // namespace

bool zquad_applies(const DemagGeom& g) {
  static const bool on = [] {
    const char* e = getenv("MMCUDA_ZQUAD");
    return !(e && e[0] == '0');
  }();
  return on && g.yT && g.Pz == 32 && g.Tzq == kZqTzq && g.nz >= 1 && g.nz <= 16;
}

void launch_zquad_f64(const DemagGeom& g, double2* Y, const double* Nhat, cudaStream_t st) {
  const dim3 grid((g.Py + kZqLines - 1) / kZqLines, g.Hx, 1);
  if (g.nz == 16 && g.Py % kZqLines == 0)
    launch_pdl(k_zquad<true>, grid, dim3(kZqNT), kZqSmem, st, Y, Nhat, g);
  else
    launch_pdl(k_zquad<false>, grid, dim3(kZqNT), kZqSmem, st, Y, Nhat, g);
}

}  // namespace mm

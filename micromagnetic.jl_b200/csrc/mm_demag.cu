// mm_demag.cu -- demag tensor assembly (FP64) and FFT convolution passes.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "mm_demag.cuh"
#include "mm_fft.cuh"

namespace mm {

// Threads per block and register elements per thread of the FFT passes; one
// block transforms at most E*T complex values (64 KB of shared memory).
template <typename R> struct FftCfg;
template <> struct FftCfg<float> { static constexpr int T = 512, E = 16; };
template <> struct FftCfg<double> { static constexpr int T = 512, E = 8; };
template <typename R> constexpr int fft_cap() { return FftCfg<R>::T * FftCfg<R>::E; }

// Symmetry of the six tensor components under x -> -x, y -> -y, z -> -z
// (fill_tensors calls, src/micro/demag.jl:56-83): xx yy zz even; xy odd in x,y;
// xz odd in x,z; yz odd in y,z.
__host__ __device__ inline int odd_axis(int c, int ax) {
  const int tbl[6] = {0, 0, 0, 3, 5, 6};  // bit0 x, bit1 y, bit2 z
  return (tbl[c] >> ax) & 1;
}

// ============================================================== kernels ====
enum XMode { XM_MAGN = 0, XM_TENSOR = 1 };

// Forward x pass: real rows (zero padded / mirrored to Px) -> half spectrum.
// line = c*rows + row;  X[line*Hx + k].
template <typename R, int MODE>
__global__ void __launch_bounds__(512, 1) k_fwd_x(const R* __restrict__ m, const R* __restrict__ Ms,
                                               const double* __restrict__ Tr, int tsign,
                                               cplx_t<R>* __restrict__ X, DemagGeom g,
                                               int lines_total, int nl,
                                               const cplx_t<R>* __restrict__ twx) {
  using C = cplx_t<R>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* buf = reinterpret_cast<C*>(smem_raw);
  if (g.gate && !*g.gate) return;
  const int Lc = g.Lc, LS = Lc | 1, nx = g.nx, Px = g.Px;
  const int rows = g.ny * g.nz;
  const int64_t N = static_cast<int64_t>(rows) * nx;
  const int line0 = blockIdx.x * nl;
  const int nlh = min(nl, lines_total - line0);
  for (int e = threadIdx.x; e < nlh * Lc; e += blockDim.x) {
    const int l = e / Lc, t = e - l * Lc;
    const int line = line0 + l;
    const int c = line / rows, row = line - c * rows;
    R v[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int u = 2 * t + h;
      R x = R(0);
      if (MODE == XM_MAGN) {
        if (u < nx) {
          const int64_t I = static_cast<int64_t>(row) * nx + u;
          x = m[c * N + I] * Ms[I];
        }
      } else {
        const int64_t I = static_cast<int64_t>(row) * nx;
        if (u < nx) x = static_cast<R>(Tr[I + u]);
        else if (u >= Px - nx + 1) x = static_cast<R>(tsign * Tr[I + (Px - u)]);
      }
      v[h] = x;
    }
    buf[l * LS + t] = cmk<C>(v[0], v[1]);
  }
  __syncthreads();
  fft_lines<false, FftCfg<R>::E>(buf, LS, nlh, g.plx, twx, 2);
  const int Hx = g.Hx;
  const R half = R(0.5);
  for (int e = threadIdx.x; e < nlh * Hx; e += blockDim.x) {
    const int l = e / Hx, k = e - l * Hx;
    const C zk = buf[l * LS + (k == Lc ? 0 : k)];
    const C zc = cconj(buf[l * LS + (k == 0 ? 0 : Lc - k)]);
    const C ev = cscale(cadd(zk, zc), half);
    const C od = crot<false>(cscale(csub(zk, zc), half));  // (zk - zc)/(2i)
    const C w = __ldg(twx + k);
    X[static_cast<int64_t>(line0 + l) * Hx + k] = cadd(ev, cmul(w, od));
  }
}

// Px == 1 (nx == 1): the x "transform" is the identity.
template <typename R, int MODE>
__global__ void k_fwd_x1(const R* __restrict__ m, const R* __restrict__ Ms,
                         const double* __restrict__ Tr, cplx_t<R>* __restrict__ X, int rows,
                         int lines_total, const int* __restrict__ gate) {
  using C = cplx_t<R>;
  if (gate && !*gate) return;
  const int line = blockIdx.x * blockDim.x + threadIdx.x;
  if (line >= lines_total) return;
  const int c = line / rows, row = line - c * rows;
  R x;
  if (MODE == XM_MAGN) x = m[static_cast<int64_t>(c) * rows + row] * Ms[row];
  else x = static_cast<R>(Tr[row]);
  X[line] = cmk<C>(x, R(0));
}

// Inverse x pass: half spectrum -> real rows (unnormalised c2r), keeps nx.
template <typename R>
__global__ void __launch_bounds__(512, 1) k_inv_x(const cplx_t<R>* __restrict__ X, R* __restrict__ H,
                                               DemagGeom g, int lines_total, int nl,
                                               const cplx_t<R>* __restrict__ twx) {
  using C = cplx_t<R>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* buf = reinterpret_cast<C*>(smem_raw);
  if (g.gate && !*g.gate) return;
  const int Lc = g.Lc, LS = Lc | 1, nx = g.nx, Hx = g.Hx;
  const int rows = g.ny * g.nz;
  const int64_t N = static_cast<int64_t>(rows) * nx;
  const int line0 = blockIdx.x * nl;
  const int nlh = min(nl, lines_total - line0);
  for (int e = threadIdx.x; e < nlh * Lc; e += blockDim.x) {
    const int l = e / Lc, k = e - l * Lc;
    const C* xr = X + static_cast<int64_t>(line0 + l) * Hx;
    const C a = xr[k];
    const C b = cconj(xr[Lc - k]);
    const C w = cconj(__ldg(twx + k));
    // Z'[k] = (A + B) + i (A - B) conj(W^k)
    buf[l * LS + k] = cadd(cadd(a, b), crot<true>(cmul(csub(a, b), w)));
  }
  __syncthreads();
  fft_lines<true, FftCfg<R>::E>(buf, LS, nlh, g.plx, twx, 2);
  for (int e = threadIdx.x; e < nlh * Lc; e += blockDim.x) {
    const int l = e / Lc, t = e - l * Lc;
    const int line = line0 + l;
    const int c = line / rows, row = line - c * rows;
    const C z = buf[l * LS + t];
    const int u = 2 * t;
    R* out = H + c * N + static_cast<int64_t>(row) * nx;
    if (u < nx) out[u] = z.x;
    if (u + 1 < nx) out[u + 1] = z.y;
  }
}

template <typename R>
__global__ void k_inv_x1(const cplx_t<R>* __restrict__ X, R* __restrict__ H, int lines_total,
                         const int* __restrict__ gate) {
  if (gate && !*gate) return;
  const int line = blockIdx.x * blockDim.x + threadIdx.x;
  if (line >= lines_total) return;
  H[line] = X[line].x;
}

// Product with the tensor spectrum, in shared memory: lines (c*W + w) of
// length L hold the 3 components; along y (kz = kz_fixed) or along z
// (ky = ky_fixed).
template <typename R, bool ALONG_Y>
__device__ __forceinline__ void tensor_product(cplx_t<R>* buf, int LS, int W, int L, int kx0,
                                               int ky_fixed, const R* __restrict__ Nhat,
                                               const int Hx, const int Py, const int Pz) {
  using C = cplx_t<R>;
  const int Tyq = Py / 2 + 1, Tzq = Pz / 2 + 1;
  const int64_t Ts = static_cast<int64_t>(Tzq) * Tyq * Hx;
  for (int e = threadIdx.x; e < W * L; e += blockDim.x) {
    const int w = e / L, t = e - w * L;
    const int kx = kx0 + w;
    if (kx >= Hx) continue;
    const int ky = ALONG_Y ? t : ky_fixed;
    const int kz = ALONG_Y ? 0 : t;
    const bool fy = ky > Py / 2, fz = kz > Pz / 2;
    const int kyq = fy ? Py - ky : ky, kzq = fz ? Pz - kz : kz;
    const R sy = fy ? R(-1) : R(1), sz = fz ? R(-1) : R(1);
    const int64_t b = (static_cast<int64_t>(kzq) * Tyq + kyq) * Hx + kx;
    const R xx = __ldg(Nhat + b), yy = __ldg(Nhat + Ts + b), zz = __ldg(Nhat + 2 * Ts + b);
    const R xy = sy * __ldg(Nhat + 3 * Ts + b), xz = sz * __ldg(Nhat + 4 * Ts + b),
            yz = sy * sz * __ldg(Nhat + 5 * Ts + b);
    C* p0 = buf + (0 * W + w) * LS + t;
    C* p1 = buf + (1 * W + w) * LS + t;
    C* p2 = buf + (2 * W + w) * LS + t;
    const C a = *p0, bb = *p1, c = *p2;
    *p0 = cmk<C>(xx * a.x + xy * bb.x + xz * c.x, xx * a.y + xy * bb.y + xz * c.y);
    *p1 = cmk<C>(xy * a.x + yy * bb.x + yz * c.x, xy * a.y + yy * bb.y + yz * c.y);
    *p2 = cmk<C>(xz * a.x + yz * bb.x + zz * c.x, xz * a.y + yz * bb.y + zz * c.y);
  }
  __syncthreads();
}

enum YMode { YM_FWD = 0, YM_INV = 1, YM_CONV2D = 2, YM_TENSOR = 3, YM_TENSOR_Q = 4 };

// y pass over column tiles [kx0, kx0+W) of one z plane for ncompc components.
// grid: (tiles, nz, 3/ncompc)
template <typename R, int MODE>
__global__ void __launch_bounds__(512, 1) k_ypass(const cplx_t<R>* in, cplx_t<R>* out,
                                               const R* __restrict__ Nhat, double* __restrict__ Tq,
                                               DemagGeom g, int W, int ncompc,
                                               const cplx_t<R>* __restrict__ twy, int tsign,
                                               double tscale) {
  using C = cplx_t<R>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* buf = reinterpret_cast<C*>(smem_raw);
  if (g.gate && !*g.gate) return;
  const int Py = g.Py, LS = Py | 1, Hx = g.Hx, ny = g.ny, nz = g.nz;
  const int kx0 = blockIdx.x * W;
  const int z = blockIdx.y;
  const int c0 = blockIdx.z * ncompc;
  const int rows_in = (MODE == YM_INV) ? Py : ny;
  // load
  for (int e = threadIdx.x; e < ncompc * Py * W; e += blockDim.x) {
    const int w = e % W;
    const int r = e / W;
    const int j = r % Py;
    const int cl = r / Py;
    const int kx = kx0 + w;
    C v = cmk<C>(R(0), R(0));
    if (kx < Hx) {
      const int64_t base = static_cast<int64_t>((c0 + cl) * nz + z) * rows_in;
      if (j < rows_in) {
        v = in[(base + j) * Hx + kx];
      } else if (MODE == YM_TENSOR || MODE == YM_TENSOR_Q) {
        if (j >= Py - ny + 1) {
          v = in[(base + (Py - j)) * Hx + kx];
          if (tsign < 0) v = cmk<C>(-v.x, -v.y);
        }
      }
    }
    buf[(cl * W + w) * LS + j] = v;
  }
  __syncthreads();
  fft_lines<MODE == YM_INV, FftCfg<R>::E>(buf, LS, ncompc * W, g.ply, twy, 1);
  if (MODE == YM_CONV2D) {
    tensor_product<R, true>(buf, LS, W, Py, kx0, 0, Nhat, Hx, Py, g.Pz);
    fft_lines<true, FftCfg<R>::E>(buf, LS, ncompc * W, g.ply, twy, 1);
  }
  // store
  if (MODE == YM_TENSOR_Q) {
    for (int e = threadIdx.x; e < g.Tyq * W; e += blockDim.x) {
      const int w = e % W, j = e / W;
      const int kx = kx0 + w;
      if (kx < Hx) Tq[static_cast<int64_t>(j) * Hx + kx] = static_cast<double>(buf[w * LS + j].x) * tscale;
    }
    return;
  }
  const int rows_out = (MODE == YM_FWD || MODE == YM_TENSOR) ? Py : ny;
  for (int e = threadIdx.x; e < ncompc * rows_out * W; e += blockDim.x) {
    const int w = e % W;
    const int r = e / W;
    const int j = r % rows_out;
    const int cl = r / rows_out;
    const int kx = kx0 + w;
    if (kx < Hx) {
      const int64_t base = static_cast<int64_t>((c0 + cl) * nz + z) * rows_out;
      out[(base + j) * Hx + kx] = buf[(cl * W + w) * LS + j];
    }
  }
}

enum ZMode { ZM_CONV = 0, ZM_TENSOR_Q = 1 };

// z pass over column tiles of one ky row.  grid: (tiles, Py or Tyq)
template <typename R, int MODE>
__global__ void __launch_bounds__(512, 1) k_zpass(cplx_t<R>* __restrict__ Y, const R* __restrict__ Nhat,
                                               double* __restrict__ Tq, DemagGeom g, int W,
                                               int ncompc, const cplx_t<R>* __restrict__ twz,
                                               int tsign, double tscale) {
  using C = cplx_t<R>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* buf = reinterpret_cast<C*>(smem_raw);
  if (g.gate && !*g.gate) return;
  const int Pz = g.Pz, LS = Pz | 1, Hx = g.Hx, Py = g.Py, nz = g.nz;
  const int kx0 = blockIdx.x * W;
  const int ky = blockIdx.y;
  for (int e = threadIdx.x; e < ncompc * Pz * W; e += blockDim.x) {
    const int w = e % W;
    const int r = e / W;
    const int kz = r % Pz;
    const int cl = r / Pz;
    const int kx = kx0 + w;
    C v = cmk<C>(R(0), R(0));
    if (kx < Hx) {
      if (kz < nz) {
        v = Y[(static_cast<int64_t>(cl * nz + kz) * Py + ky) * Hx + kx];
      } else if (MODE == ZM_TENSOR_Q && kz >= Pz - nz + 1) {
        v = Y[(static_cast<int64_t>(cl * nz + (Pz - kz)) * Py + ky) * Hx + kx];
        if (tsign < 0) v = cmk<C>(-v.x, -v.y);
      }
    }
    buf[(cl * W + w) * LS + kz] = v;
  }
  __syncthreads();
  fft_lines<false, FftCfg<R>::E>(buf, LS, ncompc * W, g.plz, twz, 1);
  if (MODE == ZM_TENSOR_Q) {
    for (int e = threadIdx.x; e < g.Tzq * W; e += blockDim.x) {
      const int w = e % W, kz = e / W;
      const int kx = kx0 + w;
      if (kx < Hx)
        Tq[(static_cast<int64_t>(kz) * g.Tyq + ky) * Hx + kx] = static_cast<double>(buf[w * LS + kz].x) * tscale;
    }
    return;
  }
  tensor_product<R, false>(buf, LS, W, Pz, kx0, ky, Nhat, Hx, Py, Pz);
  fft_lines<true, FftCfg<R>::E>(buf, LS, ncompc * W, g.plz, twz, 1);
  for (int e = threadIdx.x; e < ncompc * nz * W; e += blockDim.x) {
    const int w = e % W;
    const int r = e / W;
    const int kz = r % nz;
    const int cl = r / nz;
    const int kx = kx0 + w;
    if (kx < Hx) Y[(static_cast<int64_t>(cl * nz + kz) * Py + ky) * Hx + kx] = buf[(cl * W + w) * LS + kz];
  }
}

template <typename RO>
__global__ void k_cast(const double* __restrict__ a, RO* __restrict__ b, int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    b[i] = static_cast<RO>(a[i]);
}

// ------------------------------------------------------ Newell (FP64) -----
// newell_f / newell_g: src/micro/demag.jl:133-192; dipole far field
// src/atomistic/demag.jl:106-120; switch at R > 60 cells, demag.jl:196-201.
__device__ double dev_newell_f(double x, double y, double z) {
  const double x2 = x * x, y2 = y * y, z2 = z * z;
  const double R = sqrt(x2 + y2 + z2);
  if (R == 0.0) return 0.0;
  double f = 1.0 / 6 * (2 * x2 - y2 - z2) * R;
  if (x2 > 0) f -= x * y * z * atan(y * z / (x * R));
  if (x2 + z2 > 0) f += 0.5 * y * (z2 - x2) * asinh(y / sqrt(x2 + z2));
  if (x2 + y2 > 0) f += 0.5 * z * (y2 - x2) * asinh(z / sqrt(x2 + y2));
  return f;
}

__device__ double dev_newell_g(double x, double y, double z) {
  const double x2 = x * x, y2 = y * y, z2 = z * z;
  const double R = sqrt(x2 + y2 + z2);
  if (R == 0.0) return 0.0;
  double g = -1.0 / 3 * x * y * R;
  if (z2 > 0) g -= 1.0 / 6 * z2 * z * atan(x * y / (z * R));
  if (y2 > 0) g -= 0.5 * y2 * z * atan(x * z / (y * R));
  if (x2 > 0) g -= 0.5 * x2 * z * atan(y * z / (x * R));
  if (x2 + y2 > 0) g += x * y * z * asinh(z / sqrt(x2 + y2));
  if (y2 + z2 > 0) g += 1.0 / 6 * y * (3 * z2 - y2) * asinh(x / sqrt(y2 + z2));
  if (x2 + z2 > 0) g += 1.0 / 6 * x * (3 * z2 - x2) * asinh(y / sqrt(x2 + z2));
  return g;
}

template <bool G>
__device__ double dev_newell_tensor(double x, double y, double z, double dx, double dy, double dz) {
  const double R = sqrt(x * x + y * y + z * z) / fmax(dx, fmax(dy, dz));
  if (R > 60) {
    const double r2 = x * x + y * y + z * z;
    const double d = G ? -3 * x * y : -(2 * x * x - y * y - z * z);
    return (r2 == 0 ? 0.0 : d / (r2 * r2 * sqrt(r2))) * dx * dy * dz / (4 * kPi);
  }
  // 27-point second difference, 1-D weights w(0) = 2, w(+-1) = -1
  double s = 0.0;
  for (int a = -1; a <= 1; ++a)
    for (int b = -1; b <= 1; ++b)
      for (int c = -1; c <= 1; ++c) {
        const double w = (a == 0 ? 2.0 : -1.0) * (b == 0 ? 2.0 : -1.0) * (c == 0 ? 2.0 : -1.0);
        s += w * (G ? dev_newell_g(x + a * dx, y + b * dy, z + c * dz)
                    : dev_newell_f(x + a * dx, y + b * dy, z + c * dz));
      }
  return s / (4.0 * kPi * dx * dy * dz);
}

__device__ double dev_tensor_comp(int c, double x, double y, double z, double dx, double dy, double dz) {
  switch (c) {
    case 0: return dev_newell_tensor<false>(x, y, z, dx, dy, dz);
    case 1: return dev_newell_tensor<false>(y, x, z, dy, dx, dz);
    case 2: return dev_newell_tensor<false>(z, y, x, dz, dy, dx);
    case 3: return dev_newell_tensor<true>(x, y, z, dx, dy, dz);
    case 4: return dev_newell_tensor<true>(x, z, y, dx, dz, dy);
    default: return dev_newell_tensor<true>(y, z, x, dy, dz, dx);
  }
}

// tensors_kernel_*!  src/micro/demag.jl:298-386 (sum over macro-PBC images)
__global__ void k_newell(double* __restrict__ out, int nx, int ny, int nz, double dx, double dy,
                         double dz, int Nx, int Ny, int Nz) {
  const int64_t N = static_cast<int64_t>(nx) * ny * nz;
  const int64_t gid = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (gid >= 6 * N) return;
  const int c = static_cast<int>(gid / N);
  const int64_t I = gid - c * N;
  const int i = static_cast<int>(I % nx), j = static_cast<int>((I / nx) % ny),
            k = static_cast<int>(I / (static_cast<int64_t>(nx) * ny));
  double sum = 0.0;
  for (int p = -Nx; p <= Nx; ++p)
    for (int q = -Ny; q <= Ny; ++q)
      for (int r = -Nz; r <= Nz; ++r) {
        const double x = (i + static_cast<double>(p) * nx) * dx;
        const double y = (j + static_cast<double>(q) * ny) * dy;
        const double z = (k + static_cast<double>(r) * nz) * dz;
        sum += dev_tensor_comp(c, x, y, z, dx, dy, dz);
      }
  out[gid] = sum;
}

int newell_tensor_device(int nx, int ny, int nz, double dx, double dy, double dz, int Nx, int Ny,
                         int Nz, double* out_dev, cudaStream_t st) {
  const double mx = std::max(dx, std::max(dy, dz));
  const int64_t N = static_cast<int64_t>(nx) * ny * nz;
  const int64_t tot = 6 * N;
  const int T = 128;
  const int64_t blocks = (tot + T - 1) / T;
  k_newell<<<static_cast<unsigned>(blocks), T, 0, st>>>(out_dev, nx, ny, nz, dx / mx, dy / mx, dz / mx,
                                                        Nx, Ny, Nz);
  return static_cast<int>(cudaGetLastError());
}

// ============================================================ host side ====
template <typename C>
static C* upload_twiddles(int L, size_t& bytes, cudaStream_t st) {
  std::vector<C> h(L);
  for (int t = 0; t < L; ++t) {
    const long double a = -2.0L * 3.141592653589793238462643383279502884L * t / L;
    h[t].x = static_cast<decltype(C::x)>(static_cast<double>(cosl(a)));
    h[t].y = static_cast<decltype(C::x)>(static_cast<double>(sinl(a)));
  }
  C* d = nullptr;
  if (cudaMalloc(&d, sizeof(C) * L) != cudaSuccess) return nullptr;
  bytes += sizeof(C) * L;
  cudaMemcpyAsync(d, h.data(), sizeof(C) * L, cudaMemcpyHostToDevice, st);
  cudaStreamSynchronize(st);
  return d;
}

template <typename R>
static void set_smem_attrs() {
  static uint64_t done_mask = 0;  // one bit per device
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && ((done_mask >> dev) & 1ull)) return;
  if (dev < 64) done_mask |= 1ull << dev;
  const int mx = 200 * 1024;
  cudaFuncSetAttribute(k_fwd_x<R, XM_MAGN>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  cudaFuncSetAttribute(k_fwd_x<R, XM_TENSOR>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  cudaFuncSetAttribute(k_inv_x<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  cudaFuncSetAttribute(k_ypass<R, YM_FWD>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  cudaFuncSetAttribute(k_ypass<R, YM_INV>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  cudaFuncSetAttribute(k_ypass<R, YM_CONV2D>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  cudaFuncSetAttribute(k_ypass<R, YM_TENSOR>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  cudaFuncSetAttribute(k_ypass<R, YM_TENSOR_Q>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  cudaFuncSetAttribute(k_zpass<R, ZM_CONV>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  cudaFuncSetAttribute(k_zpass<R, ZM_TENSOR_Q>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
}

template <typename R>
DemagPlan<R>::~DemagPlan() {
  cudaFree(X);
  cudaFree(Y);
  cudaFree(Nhat);
  cudaFree(twx);
  cudaFree(twy);
  cudaFree(twz);
}

template <typename R>
int DemagPlan<R>::init(int nx, int ny, int nz, cudaStream_t st, char* err, size_t nerr) {
  g.nx = nx; g.ny = ny; g.nz = nz;
  g.gate = nullptr;
  g.Px = padded_fft_len(nx, true);
  g.Py = padded_fft_len(ny, false);
  g.Pz = padded_fft_len(nz, false);
  g.Lc = g.Px > 1 ? g.Px / 2 : 0;
  g.Hx = g.Px > 1 ? g.Lc + 1 : 1;
  g.Tyq = g.Py / 2 + 1;
  g.Tzq = g.Pz / 2 + 1;
  // every pass (including the FP64 tensor passes) must fit one block
  const int cap64 = fft_cap<double>();
  if (g.Lc > cap64 || g.Py > cap64 || 3 * g.Pz > cap64) {
    snprintf(err, nerr, "demag: mesh %dx%dx%d exceeds the FFT pass limits (nx<=%d, ny<=%d, nz<=%d)", nx, ny,
             nz, cap64, cap64 / 2, cap64 / 6);
    return -1;
  }
  if (!make_fft_plan(g.Lc > 0 ? g.Lc : 1, g.plx) || !make_fft_plan(g.Py, g.ply) ||
      !make_fft_plan(g.Pz, g.plz)) {
    snprintf(err, nerr, "demag: no radix plan");
    return -1;
  }
  fused2d = (g.Pz == 1) && (3 * g.Py <= fft_cap<R>());
  set_smem_attrs<R>();
  set_smem_attrs<double>();
  const int64_t nX = 3LL * nz * ny * g.Hx;
  if (cudaMalloc(&X, sizeof(C) * nX) != cudaSuccess) return 2;
  bytes_ += sizeof(C) * nX;
  if (!fused2d) {
    const int64_t nY = 3LL * nz * g.Py * g.Hx;
    if (cudaMalloc(&Y, sizeof(C) * nY) != cudaSuccess) return 2;
    bytes_ += sizeof(C) * nY;
  }
  const int64_t nT = 6LL * g.Tzq * g.Tyq * g.Hx;
  if (cudaMalloc(&Nhat, sizeof(R) * nT) != cudaSuccess) return 2;
  bytes_ += sizeof(R) * nT;
  cudaMemsetAsync(Nhat, 0, sizeof(R) * nT, st);
  if (g.Px > 1 && !(twx = upload_twiddles<C>(g.Px, bytes_, st))) return 2;
  if (!(twy = upload_twiddles<C>(g.Py, bytes_, st))) return 2;
  if (!(twz = upload_twiddles<C>(g.Pz, bytes_, st))) return 2;
  return static_cast<int>(cudaGetLastError());
}

// ---- launch helpers shared by apply() and the tensor assembly ------------
template <typename R, int MODE>
static void launch_fwd_x(const DemagGeom& g, const R* m, const R* Ms, const double* Tr, int tsign,
                         cplx_t<R>* X, int ncomp, const cplx_t<R>* twx, cudaStream_t st) {
  using C = cplx_t<R>;
  const int rows = g.ny * g.nz;
  const int lines = ncomp * rows;
  if (g.Px == 1) {
    k_fwd_x1<R, MODE><<<(lines + 255) / 256, 256, 0, st>>>(m, Ms, Tr, X, rows, lines, g.gate);
    return;
  }
  const int nl = std::max(1, fft_cap<R>() / g.Lc);
  const int blocks = (lines + nl - 1) / nl;
  const size_t sm = sizeof(C) * nl * (g.Lc | 1);
  k_fwd_x<R, MODE><<<blocks, FftCfg<R>::T, sm, st>>>(m, Ms, Tr, tsign, X, g, lines, nl, twx);
}

template <typename R, int MODE>
static void launch_ypass(const DemagGeom& g, const cplx_t<R>* in, cplx_t<R>* out, const R* Nhat,
                         double* Tq, int ncompc, int ncomp, const cplx_t<R>* twy, int tsign,
                         double tscale, cudaStream_t st) {
  using C = cplx_t<R>;
  const int W = std::max(1, std::min(g.Hx, fft_cap<R>() / (ncompc * g.Py)));
  dim3 grid((g.Hx + W - 1) / W, g.nz, ncomp / ncompc);
  const size_t sm = sizeof(C) * ncompc * W * (g.Py | 1);
  k_ypass<R, MODE><<<grid, FftCfg<R>::T, sm, st>>>(in, out, Nhat, Tq, g, W, ncompc, twy, tsign, tscale);
}

template <typename R, int MODE>
static void launch_zpass(const DemagGeom& g, cplx_t<R>* Y, const R* Nhat, double* Tq, int ncompc,
                         int kyrows, const cplx_t<R>* twz, int tsign, double tscale, cudaStream_t st) {
  using C = cplx_t<R>;
  const int W = std::max(1, std::min(g.Hx, fft_cap<R>() / (ncompc * g.Pz)));
  dim3 grid((g.Hx + W - 1) / W, kyrows, 1);
  const size_t sm = sizeof(C) * ncompc * W * (g.Pz | 1);
  k_zpass<R, MODE><<<grid, FftCfg<R>::T, sm, st>>>(Y, Nhat, Tq, g, W, ncompc, twz, tsign, tscale);
}

template <typename R>
static bool run_pass(const DemagPlan<R>& p, DemagGeom g, int which, const R* m, const R* mu0Ms, R* Hd,
                     cudaStream_t st) {
  using C = cplx_t<R>;
  switch (which) {
    case 0:
      launch_fwd_x<R, XM_MAGN>(g, m, mu0Ms, nullptr, 1, p.X, 3, p.twx, st);
      return true;
    case 1:
      if (p.fused2d) return false;
      launch_ypass<R, YM_FWD>(g, p.X, p.Y, p.Nhat, nullptr, 1, 3, p.twy, 1, 0.0, st);
      return true;
    case 2:
      if (p.fused2d) launch_ypass<R, YM_CONV2D>(g, p.X, p.X, p.Nhat, nullptr, 3, 3, p.twy, 1, 0.0, st);
      else launch_zpass<R, ZM_CONV>(g, p.Y, p.Nhat, nullptr, 3, g.Py, p.twz, 1, 0.0, st);
      return true;
    case 3:
      if (p.fused2d) return false;
      launch_ypass<R, YM_INV>(g, p.Y, p.X, p.Nhat, nullptr, 1, 3, p.twy, 1, 0.0, st);
      return true;
    case 4: {
      const int lines = 3 * g.ny * g.nz;
      if (g.Px == 1) {
        k_inv_x1<R><<<(lines + 255) / 256, 256, 0, st>>>(p.X, Hd, lines, g.gate);
      } else {
        const int nl = std::max(1, fft_cap<R>() / g.Lc);
        const size_t sm = sizeof(C) * nl * (g.Lc | 1);
        k_inv_x<R><<<(lines + nl - 1) / nl, FftCfg<R>::T, sm, st>>>(p.X, Hd, g, lines, nl, p.twx);
      }
      return true;
    }
    default:
      return false;
  }
}

template <typename R>
void DemagPlan<R>::apply(const R* m, const R* mu0Ms, R* Hd, cudaStream_t st, const int* gate) {
  DemagGeom gg = this->g;
  gg.gate = gate;
  for (int which = 0; which < 5; ++which) run_pass(*this, gg, which, m, mu0Ms, Hd, st);
}

template <typename R>
bool DemagPlan<R>::launch_pass(int which, const R* m, const R* mu0Ms, R* Hd, cudaStream_t st) {
  return run_pass(*this, this->g, which, m, mu0Ms, Hd, st);
}

template <typename R>
double DemagPlan<R>::pass_bytes(int which) const {
  const double w = sizeof(R), cw = 2.0 * sizeof(R);
  const double rows = static_cast<double>(g.ny) * g.nz, N = rows * g.nx;
  const double nX = 3.0 * rows * g.Hx, nY = 3.0 * g.nz * g.Py * g.Hx;
  const double Ts = static_cast<double>(g.Tzq) * g.Tyq * g.Hx;
  switch (which) {
    case 0: return 4.0 * N * w + nX * cw;
    case 1: return fused2d ? 0.0 : (nX + nY) * cw;
    case 2: return (fused2d ? 2.0 * nX : 2.0 * nY) * cw + 6.0 * Ts * w;
    case 3: return fused2d ? 0.0 : (nX + nY) * cw;
    case 4: return nX * cw + 3.0 * N * w;
    default: return 0.0;
  }
}

template <typename R>
int DemagPlan<R>::launches_per_apply() const {
  return fused2d ? 3 : 5;
}

// Tensor spectrum: for each component, forward r2c-x / y / z transforms of
// the mirrored, padded real-space tensor in FP64, real part of the
// (kx, ky<=Py/2, kz<=Pz/2) quadrant, scaled by -1/(mu0 Px Py Pz).
template <typename R>
int DemagPlan<R>::set_tensor(const double* T6N, cudaStream_t st) {
  using C64 = double2;
  size_t b64 = 0;
  C64 *tx = nullptr, *ty = nullptr, *tz = nullptr, *X64 = nullptr, *Y64 = nullptr;
  double* Tq = nullptr;
  const int64_t N = static_cast<int64_t>(g.nx) * g.ny * g.nz;
  const int64_t nX = static_cast<int64_t>(g.nz) * g.ny * g.Hx;
  const int64_t nY = static_cast<int64_t>(g.nz) * g.Py * g.Hx;
  const int64_t Ts = static_cast<int64_t>(g.Tzq) * g.Tyq * g.Hx;
  int rc = 0;
  if (g.Px > 1 && !(tx = upload_twiddles<C64>(g.Px, b64, st))) rc = 2;
  if (!rc && !(ty = upload_twiddles<C64>(g.Py, b64, st))) rc = 2;
  if (!rc && !(tz = upload_twiddles<C64>(g.Pz, b64, st))) rc = 2;
  if (!rc && cudaMalloc(&X64, sizeof(C64) * nX) != cudaSuccess) rc = 2;
  if (!rc && g.Pz > 1 && cudaMalloc(&Y64, sizeof(C64) * nY) != cudaSuccess) rc = 2;
  if (!rc && cudaMalloc(&Tq, sizeof(double) * 6 * Ts) != cudaSuccess) rc = 2;
  if (!rc) {
    const double scale = -1.0 / (kMu0 * static_cast<double>(g.Px) * g.Py * g.Pz);
    for (int c = 0; c < 6; ++c) {
      const int sx = odd_axis(c, 0) ? -1 : 1, sy = odd_axis(c, 1) ? -1 : 1, sz = odd_axis(c, 2) ? -1 : 1;
      launch_fwd_x<double, XM_TENSOR>(g, nullptr, nullptr, T6N + c * N, sx, X64, 1, tx, st);
      if (g.Pz == 1) {
        launch_ypass<double, YM_TENSOR_Q>(g, X64, nullptr, nullptr, Tq + c * Ts, 1, 1, ty, sy, scale, st);
      } else {
        launch_ypass<double, YM_TENSOR>(g, X64, Y64, nullptr, nullptr, 1, 1, ty, sy, 0.0, st);
        launch_zpass<double, ZM_TENSOR_Q>(g, Y64, nullptr, Tq + c * Ts, 1, g.Tyq, tz, sz, scale, st);
      }
    }
    k_cast<R><<<1024, 256, 0, st>>>(Tq, Nhat, 6 * Ts);
    rc = static_cast<int>(cudaGetLastError());
    cudaStreamSynchronize(st);
  }
  cudaFree(tx); cudaFree(ty); cudaFree(tz); cudaFree(X64); cudaFree(Y64); cudaFree(Tq);
  return rc;
}

template class DemagPlan<float>;
template class DemagPlan<double>;

}  // namespace mm

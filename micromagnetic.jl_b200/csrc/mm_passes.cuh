// mm_passes.cuh -- the shared-memory FFT passes of the demag convolution as
// launch descriptors (FwdX, InvX, YLines, ZConv, ZSmall; mm_launch.cuh), the
// strided tensor passes and their configuration.  Shared by mm_demag.cu and
// the persistent step kernel (mm_persist.cu).  Internal.
#pragma once
#include <type_traits>

#include "mm_demag.cuh"
#include "mm_fft.cuh"
#include "mm_launch.cuh"
#include "mm_lines.cuh"

namespace mm {

// Pass configuration: NT threads per block and the number of complex values
// a block transforms.  The hot passes run 256-thread blocks (three per SM
// overlap their loads with the transforms of the others); the one-time FP64
// tensor passes run 512.
template <typename R, int NT> struct PassCfg {
  // complex values per block (each of the two ping-pong buffers): 32 KB
  // (64 KB of shared memory per block for the hot passes)
  static constexpr int cap = (sizeof(R) == 4 || NT == 512) ? 4096 : 2048;
  static constexpr int minb = NT == 256 ? 3 : 1;
};
constexpr int kHotNT = 256;
// threads of the fused-middle z kernel: one per middle task of the widest
// tile (W * RA: FP32 16 x 16, FP64 8 x 16 for Pz = 128).  384 in FP32, so
// that the first stage of a 16-column tile takes one round, measured 17 %
// slower (register cap); FP64 at 128 threads is 5 % faster than at 256, whose
// middle left half the threads idle.
template <typename R> constexpr int zconv2_nt() { return sizeof(R) == 4 ? 256 : 128; }
// blocks per SM the fused z kernels are compiled for: 80 (FP32) and 128
// (FP64) registers a thread
template <typename R, int NT> constexpr int zconv2_minb() { return (sizeof(R) == 4 ? 3 : 2) * 256 / NT; }
constexpr size_t kMaxSmem = 227 * 1024;  // dynamic shared memory per block (opt-in maximum)
constexpr int kTensorNT = 512;
template <typename R> constexpr int hot_cap() { return PassCfg<R, kHotNT>::cap; }
constexpr int tensor_cap() { return PassCfg<double, kTensorNT>::cap; }

// Symmetry of the six tensor components under x -> -x, y -> -y, z -> -z
// (fill_tensors calls, src/micro/demag.jl:56-83): xx yy zz even; xy odd in x,y;
// xz odd in x,z; yz odd in y,z.
__host__ __device__ inline int odd_axis(int c, int ax) {
  const int tbl[6] = {0, 0, 0, 3, 5, 6};  // bit0 x, bit1 y, bit2 z
  return (tbl[c] >> ax) & 1;
}

// ============================================================== kernels ====
template <typename R> struct Vec2;
template <> struct Vec2<float> { using T = float2; };
template <> struct Vec2<double> { using T = double2; };

enum XMode { XM_MAGN = 0, XM_TENSOR = 1 };

// Forward x pass: real rows (zero padded / mirrored to Px) -> half spectrum.
// line = c*rows + row;  X[line*Hx + k].
template <typename R, int MODE, int NT>
struct FwdX {
  static constexpr int kNT = NT, kMinB = (PassCfg<R, NT>::minb);
  struct Args {
    const R* __restrict__ m;
    const R* __restrict__ Ms;
    const double* __restrict__ Tr;
    int tsign;
    cplx_t<R>* __restrict__ X;
    DemagGeom g;
    int lines_total;
    int nl;
    const cplx_t<R>* __restrict__ twx;
    int half;
    FastDiv fnl;
    dim3 grid;
  };
  static __device__ __forceinline__ void body(const Args& args, uint3 blockIdx) {
    const auto& [m, Ms, Tr, tsign, X, g, lines_total, nl, twx, half, fnl, grid] = args;

  using C = cplx_t<R>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* buf = reinterpret_cast<C*>(smem_raw);
  C* buf2 = buf + half;
  if (g.gate && !*g.gate) return;
  const int Lc = g.Lc, LS = Lc | 1, nx = g.nx, Px = g.Px;
  const int rows = g.ny * g.nz;
  const int64_t N = static_cast<int64_t>(rows) * nx;
  const int line0 = blockIdx.x * nl;
  const int nlh = min(nl, lines_total - line0);
#pragma unroll 4  // several iterations' global loads in flight
  for (int e = threadIdx.x; e < nlh * Lc; e += NT) {
    const int l = fdiv(e, g.fLc), t = e - l * Lc;
    const int line = line0 + l;
    const int c = fdiv(line, g.frows), row = line - c * rows;
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
  buf = line_fft_to_smem<false, NT>(SmemLines<C>{buf, LS}, buf2, buf, LS, nl, fnl, g.plx, twx, 2);
  const int Hx = g.Hx;
  const R one_half = R(0.5);
  auto spectrum = [&](int l, int k) {
    const C zk = buf[l * LS + (k == Lc ? 0 : k)];
    const C zc = cconj(buf[l * LS + (k == 0 ? 0 : Lc - k)]);
    const C ev = cscale(cadd(zk, zc), one_half);
    const C od = crot<false>(cscale(csub(zk, zc), one_half));  // (zk - zc)/(2i)
    const C w = __ldg(twx + k);
    return cadd(ev, cmul(w, od));
  };
  if (MODE == XM_MAGN && g.xT) {
    // column-major X: consecutive threads write consecutive rows of one kx
    for (int e = threadIdx.x; e < nl * Hx; e += NT) {
      const int k = fdiv(e, fnl), l = e - k * nl;
      if (l >= nlh) continue;
      const int line = line0 + l;
      const int c = fdiv(line, g.frows), row = line - c * rows;
      X[(static_cast<int64_t>(c) * Hx + k) * rows + row] = spectrum(l, k);
    }
  } else {
    for (int e = threadIdx.x; e < nlh * Hx; e += NT) {
      const int l = fdiv(e, g.fHx), k = e - l * Hx;
      X[static_cast<int64_t>(line0 + l) * Hx + k] = spectrum(l, k);
    }
  }
  }
};


// Px == 1 (nx == 1): the x "transform" is the identity.
template <typename R, int MODE>
__global__ void k_fwd_x1(const R* __restrict__ m, const R* __restrict__ Ms, const double* __restrict__ Tr,
                         cplx_t<R>* __restrict__ X, int rows, int lines_total, const int* __restrict__ gate) {
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
template <typename R, int NT>
struct InvX {
  static constexpr int kNT = NT, kMinB = (PassCfg<R, NT>::minb);
  struct Args {
    const cplx_t<R>* __restrict__ X;
    R* __restrict__ H;
    DemagGeom g;
    int lines_total;
    int nl;
    const cplx_t<R>* __restrict__ twx;
    int half;
    FastDiv fnl;
    dim3 grid;
  };
  static __device__ __forceinline__ void body(const Args& args, uint3 blockIdx) {
    const auto& [X, H, g, lines_total, nl, twx, half, fnl, grid] = args;

  using C = cplx_t<R>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* buf = reinterpret_cast<C*>(smem_raw);
  C* buf2 = buf + half;
  if (g.gate && !*g.gate) return;
  const int Lc = g.Lc, LS = Lc | 1, nx = g.nx, Hx = g.Hx;
  const int rows = g.ny * g.nz;
  const int64_t N = static_cast<int64_t>(rows) * nx;
  const int line0 = blockIdx.x * nl;
  const int nlh = min(nl, lines_total - line0);
  // Z'[k] = (A + B) + i (A - B) conj(W^k), A = X[k], B = conj(X[Lc - k])
  auto pre = [&](int l, int k, C a, C b) {
    const C w = cconj(__ldg(twx + k));
    buf[l * LS + k] = cadd(cadd(a, b), crot<true>(cmul(csub(a, b), w)));
  };
  if (g.xT && !g.yT) {
    // column-major X (films): consecutive threads read consecutive rows of one kx
#pragma unroll 4  // several iterations' global loads in flight
    for (int e = threadIdx.x; e < nl * Lc; e += NT) {
      const int k = fdiv(e, fnl), l = e - k * nl;
      if (l >= nlh) continue;
      const int line = line0 + l;
      const int c = fdiv(line, g.frows), row = line - c * rows;
      const C* xc = X + static_cast<int64_t>(c) * Hx * rows + row;
      pre(l, k, xc[static_cast<int64_t>(k) * rows], cconj(xc[static_cast<int64_t>(Lc - k) * rows]));
    }
  } else {
#pragma unroll 4  // several iterations' global loads in flight
    for (int e = threadIdx.x; e < nlh * Lc; e += NT) {
      const int l = fdiv(e, g.fLc), k = e - l * Lc;
      const C* xr = X + static_cast<int64_t>(line0 + l) * Hx;
      pre(l, k, xr[k], cconj(xr[Lc - k]));
    }
  }
  __syncthreads();
  buf = line_fft_to_smem<true, NT>(SmemLines<C>{buf, LS}, buf2, buf, LS, nl, fnl, g.plx, twx, 2);
  if (!(nx & 1) && N * 3 < (int64_t(1) << 31)) {
    using V2 = typename Vec2<R>::T;
    const int Ni = static_cast<int>(N);
    for (int e = threadIdx.x; e < nlh * Lc; e += NT) {
      const int l = fdiv(e, g.fLc), t = e - l * Lc;
      const int line = line0 + l;
      const int c = fdiv(line, g.frows), row = line - c * rows;
      if (2 * t >= nx) continue;
      const C z = buf[l * LS + t];
      V2 o;
      o.x = z.x;
      o.y = z.y;
      *reinterpret_cast<V2*>(H + c * Ni + row * nx + 2 * t) = o;
    }
  } else {
    for (int e = threadIdx.x; e < nlh * Lc; e += NT) {
      const int l = fdiv(e, g.fLc), t = e - l * Lc;
      const int line = line0 + l;
      const int c = fdiv(line, g.frows), row = line - c * rows;
      const C z = buf[l * LS + t];
      const int u = 2 * t;
      R* out = H + c * N + static_cast<int64_t>(row) * nx;
      if (u < nx) out[u] = z.x;
      if (u + 1 < nx) out[u + 1] = z.y;
    }
  }
  }
};


template <typename R>
__global__ void k_inv_x1(const cplx_t<R>* __restrict__ X, R* __restrict__ H, int lines_total,
                         const int* __restrict__ gate) {
  if (gate && !*gate) return;
  const int line = blockIdx.x * blockDim.x + threadIdx.x;
  if (line >= lines_total) return;
  H[line] = X[line].x;
}

// Product with the tensor spectrum, in shared memory: lines (c*W + w) of
// length L hold the 3 components at (kx0 + w, ky, kz); along y (kz = 0) or
// along z (ky fixed).  The stored quadrant is unfolded with the component
// parities (odd in y: xy, yz; odd in z: xz, yz).
template <typename R, bool ALONG_Y, int NT, bool COLS = false>
__device__ __forceinline__ void tensor_product(cplx_t<R>* buf, int LS, int lgW, int L, const FastDiv fL,
                                               int kx0, int ky_fixed, const R* __restrict__ Nhat, int Hx, int Py,
                                               int Pz) {
  using C = cplx_t<R>;
  const int W = 1 << lgW;
  const int Tyq = Py / 2 + 1, Tzq = Pz / 2 + 1;
  const int64_t Ts = static_cast<int64_t>(Tzq) * Tyq * Hx;
  for (int e = threadIdx.x; e < W * L; e += NT) {
    // coalesced tensor reads: w fastest (row-major tensor), t fastest (COLS,
    // the column-major film tensor Nhat[(c*Hx + kx)*Tyq + ky])
    int w, t;
    if (COLS) {
      w = fdiv(e, fL);
      t = e - w * L;
    } else {
      w = e & (W - 1);
      t = e >> lgW;
    }
    const int kx = kx0 + w;
    if (kx >= Hx) continue;
    const int ky = ALONG_Y ? t : ky_fixed;
    const int kz = ALONG_Y ? 0 : t;
    const bool fy = ky > Py / 2, fz = kz > Pz / 2;
    const int kyq = fy ? Py - ky : ky, kzq = fz ? Pz - kz : kz;
    const R sy = fy ? R(-1) : R(1), sz = fz ? R(-1) : R(1);
    const int64_t b = COLS ? static_cast<int64_t>(kx) * Tyq + kyq : (static_cast<int64_t>(kzq) * Tyq + kyq) * Hx + kx;
    const R xx = __ldg(Nhat + b), yy = __ldg(Nhat + Ts + b), zz = __ldg(Nhat + 2 * Ts + b);
    const R xy = sy * __ldg(Nhat + 3 * Ts + b), xz = sz * __ldg(Nhat + 4 * Ts + b),
            yz = sy * sz * __ldg(Nhat + 5 * Ts + b);
    const int tp = COLS ? t + (t >> 4) : t;  // COLS blocks use padded lines (SmemLines PAD)
    C* p0 = buf + (0 * W + w) * LS + tp;
    C* p1 = buf + (1 * W + w) * LS + tp;
    C* p2 = buf + (2 * W + w) * LS + tp;
    const C a = *p0, bb = *p1, c = *p2;
    *p0 = cmk<C>(xx * a.x + xy * bb.x + xz * c.x, xx * a.y + xy * bb.y + xz * c.y);
    *p1 = cmk<C>(xy * a.x + yy * bb.x + yz * c.x, xy * a.y + yy * bb.y + yz * c.y);
    *p2 = cmk<C>(xz * a.x + yz * bb.x + zz * c.x, xz * a.y + yz * bb.y + zz * c.y);
  }
  __syncthreads();
}

enum YMode { YM_FWD = 0, YM_INV = 1, YM_CONV2D = 2, YM_TENSOR = 3, YM_TENSOR_Q = 4 };

// y pass over column tiles [kx0, kx0 + 2^lgW) of one z plane for ncompc
// components.  grid: (tiles, nz, 3/ncompc).  Shared layout: line (cl*W + w),
// position j (LS = Py | 1 keeps the transposed stores free of bank conflicts).
template <typename R, int MODE, int NT>
__global__ void __launch_bounds__(NT, (PassCfg<R, NT>::minb)) k_ypass(
    const cplx_t<R>* in, cplx_t<R>* out, const R* __restrict__ Nhat, double* __restrict__ Tq, DemagGeom g,
    int lgW, int ncompc, const cplx_t<R>* __restrict__ twy, int tsign, double tscale, int half) {
  using C = cplx_t<R>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* buf = reinterpret_cast<C*>(smem_raw);
  C* buf2 = buf + half;
  if (g.gate && !*g.gate) return;
  const int Py = g.Py, LS = Py | 1, Hx = g.Hx, ny = g.ny, nz = g.nz;
  const int W = 1 << lgW;
  const int kx0 = blockIdx.x * W;
  const int z = blockIdx.y;
  const int c0 = blockIdx.z * ncompc;
  const int rows_in = (MODE == YM_INV) ? Py : ny;
  // zero the padded rows, then load the rows that hold data
  if (MODE != YM_INV) {
    const int pad = (MODE == YM_TENSOR || MODE == YM_TENSOR_Q) ? 0 : Py - ny;
    for (int e = threadIdx.x; e < ncompc * W * pad; e += NT) {
      const int l = fdiv(e, g.fpady), j = ny + (e - l * pad);
      buf[l * LS + j] = cmk<C>(R(0), R(0));
    }
  }
  const int nload = (MODE == YM_TENSOR || MODE == YM_TENSOR_Q) ? Py : rows_in;
  const FastDiv fr = (MODE == YM_INV || MODE == YM_TENSOR || MODE == YM_TENSOR_Q) ? g.fPy : g.fny;
  for (int e = threadIdx.x; e < ncompc * nload * W; e += NT) {
    const int w = e & (W - 1);
    const int r = e >> lgW;
    const int cl = fdiv(r, fr);
    const int j = r - cl * nload;
    const int kx = kx0 + w;
    C v = cmk<C>(R(0), R(0));
    if (kx < Hx) {
      const int64_t base = static_cast<int64_t>((c0 + cl) * nz + z) * rows_in;
      if (j < rows_in) {
        v = in[(base + j) * Hx + kx];
      } else if (j >= Py - ny + 1) {  // tensor modes: mirrored rows
        v = in[(base + (Py - j)) * Hx + kx];
        if (tsign < 0) v = cmk<C>(-v.x, -v.y);
      }
    }
    buf[(cl * W + w) * LS + j] = v;
  }
  __syncthreads();
  {
    C* res = fft_lines<MODE == YM_INV, NT>(buf, buf2, LS, ncompc * W, g.ply, twy, 1);
    if (res != buf) {
      buf2 = buf;
      buf = res;
    }
  }
  if (MODE == YM_CONV2D) {
    tensor_product<R, true, NT>(buf, LS, lgW, Py, g.fPy, kx0, 0, Nhat, Hx, Py, g.Pz);
    buf = fft_lines<true, NT>(buf, buf2, LS, ncompc * W, g.ply, twy, 1);
  }
  // store
  if (MODE == YM_TENSOR_Q) {
    for (int e = threadIdx.x; e < g.Tyq * W; e += NT) {
      const int w = e & (W - 1), j = e >> lgW;
      const int kx = kx0 + w;
      if (kx < Hx) Tq[static_cast<int64_t>(j) * Hx + kx] = static_cast<double>(buf[w * LS + j].x) * tscale;
    }
    return;
  }
  const int rows_out = (MODE == YM_FWD || MODE == YM_TENSOR) ? Py : ny;
  const FastDiv fo = (MODE == YM_FWD || MODE == YM_TENSOR) ? g.fPy : g.fny;
  for (int e = threadIdx.x; e < ncompc * rows_out * W; e += NT) {
    const int w = e & (W - 1);
    const int r = e >> lgW;
    const int cl = fdiv(r, fo);
    const int j = r - cl * rows_out;
    const int kx = kx0 + w;
    if (kx < Hx) {
      const int64_t base = static_cast<int64_t>((c0 + cl) * nz + z) * rows_out;
      out[(base + j) * Hx + kx] = buf[(cl * W + w) * LS + j];
    }
  }
}

enum ZMode { ZM_CONV = 0, ZM_TENSOR_Q = 1 };

// z pass over column tiles of one ky row (and, in ZM_CONV, of its mirror row
// Py - ky in the same block, so each tensor entry is fetched once).
// grid: (tiles, Py/2 + 1 or Tyq)
template <typename R, int MODE, int NT>
__global__ void __launch_bounds__(NT, (PassCfg<R, NT>::minb)) k_zpass(
    cplx_t<R>* __restrict__ Y, const R* __restrict__ Nhat, double* __restrict__ Tq, DemagGeom g, int lgW,
    int ncompc, const cplx_t<R>* __restrict__ twz, int tsign, double tscale, int half) {
  using C = cplx_t<R>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* buf = reinterpret_cast<C*>(smem_raw);
  C* buf2 = buf + half;
  if (g.gate && !*g.gate) return;
  const int Pz = g.Pz, LS = Pz | 1, Hx = g.Hx, Py = g.Py, nz = g.nz;
  const int W = 1 << lgW;
  const int kx0 = blockIdx.x * W;
  const int kyA = blockIdx.y;
  // rows handled: ky and (for the product) its mirror, when distinct
  const int kyB = (MODE == ZM_CONV && kyA > 0 && 2 * kyA != Py) ? Py - kyA : -1;
  const int nrow = kyB >= 0 ? 2 : 1;
  const int ncl = ncompc * nrow;  // line groups of W lines
  const int pad = (MODE == ZM_TENSOR_Q) ? 0 : Pz - nz;
  for (int e = threadIdx.x; e < ncl * W * pad; e += NT) {
    const int l = fdiv(e, g.fpadz), kz = nz + (e - l * pad);
    buf[l * LS + kz] = cmk<C>(R(0), R(0));
  }
  const int nload = (MODE == ZM_TENSOR_Q) ? Pz : nz;
  const FastDiv fr = (MODE == ZM_TENSOR_Q) ? g.fPz : g.fnz;
  for (int e = threadIdx.x; e < ncl * nload * W; e += NT) {
    const int w = e & (W - 1);
    const int r = e >> lgW;
    const int q = fdiv(r, fr);  // line group = row * ncompc + cl
    const int kz = r - q * nload;
    const int row = q / ncompc, cl = q - row * ncompc;
    const int ky = row == 0 ? kyA : kyB;
    const int kx = kx0 + w;
    C v = cmk<C>(R(0), R(0));
    if (kx < Hx) {
      if (kz < nz) {
        v = Y[(static_cast<int64_t>(cl * nz + kz) * Py + ky) * Hx + kx];
      } else if (kz >= Pz - nz + 1) {  // tensor mode: mirrored rows
        v = Y[(static_cast<int64_t>(cl * nz + (Pz - kz)) * Py + ky) * Hx + kx];
        if (tsign < 0) v = cmk<C>(-v.x, -v.y);
      }
    }
    buf[(q * W + w) * LS + kz] = v;
  }
  __syncthreads();
  {
    C* res = fft_lines<false, NT>(buf, buf2, LS, ncl * W, g.plz, twz, 1);
    if (res != buf) {
      buf2 = buf;
      buf = res;
    }
  }
  if (MODE == ZM_TENSOR_Q) {
    for (int e = threadIdx.x; e < g.Tzq * W; e += NT) {
      const int w = e & (W - 1), kz = e >> lgW;
      const int kx = kx0 + w;
      if (kx < Hx)
        Tq[(static_cast<int64_t>(kz) * g.Tyq + kyA) * Hx + kx] = static_cast<double>(buf[w * LS + kz].x) * tscale;
    }
    return;
  }
  tensor_product<R, false, NT>(buf, LS, lgW, Pz, g.fPz, kx0, kyA, Nhat, Hx, Py, Pz);
  if (kyB >= 0)
    tensor_product<R, false, NT>(buf + 3 * W * LS, LS, lgW, Pz, g.fPz, kx0, kyB, Nhat, Hx, Py, Pz);
  buf = fft_lines<true, NT>(buf, buf2, LS, ncl * W, g.plz, twz, 1);
  for (int e = threadIdx.x; e < ncl * nz * W; e += NT) {
    const int w = e & (W - 1);
    const int r = e >> lgW;
    const int q = fdiv(r, g.fnz);
    const int kz = r - q * nz;
    const int row = q / ncompc, cl = q - row * ncompc;
    const int ky = row == 0 ? kyA : kyB;
    const int kx = kx0 + w;
    if (kx < Hx) Y[(static_cast<int64_t>(cl * nz + kz) * Py + ky) * Hx + kx] = buf[(q * W + w) * LS + kz];
  }
}

// ---- hot-path strided passes (fused global I/O, line-fastest mapping) -----
enum YLMode { YL_FWD = 0, YL_INV = 1, YL_CONV2D = 2 };

// y lines of one z plane over a W-wide kx tile.  grid: (tiles, nz, 3/ncompc)
//   YL_FWD:    X rows y < ny            -> Y rows 0..Py-1
//   YL_INV:    Y rows 0..Py-1           -> X rows y < ny
//   YL_CONV2D: X rows y < ny, forward y, tensor product (kz = 0), inverse y -> X
// XT (YL_CONV2D of films): X column-major, see DemagGeom::xT.
// Row-major: blocks blockIdx.x >= nfull take one leftover column each
// (kx = nfull W + blockIdx.x - nfull; Hx = 16 m + 1 for nx = 2^k) instead of
// a W-wide tile of mostly absent columns; fnl1 divides by ncompc.
template <typename R, int MODE, int NT, bool I32, bool XT = false>
struct YLines {
  static constexpr int kNT = NT, kMinB = (sizeof(R) == 4 ? 3 : 2);
  struct Args {
    const cplx_t<R>* in;
    cplx_t<R>* out;
    const R* __restrict__ Nhat;
    DemagGeom g;
    int lgW0;
    int ncompc;
    FastDiv fnl0;
    const cplx_t<R>* __restrict__ twy;
    int half;
    int nfull;
    FastDiv fnl1;
    dim3 grid;
  };
  static __device__ __forceinline__ void body(const Args& args, uint3 blockIdx) {
    const auto& [in, out, Nhat, g, lgW0, ncompc, fnl0, twy, half, nfull, fnl1, grid] = args;
    int lgW = lgW0;  // a leftover column takes one-column tiles
    FastDiv fnl = fnl0;

  using C = cplx_t<R>;
  using IX = std::conditional_t<I32, int, int64_t>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* a = reinterpret_cast<C*>(smem_raw);
  C* b = a + half;
  if (g.gate && !*g.gate) return;
  const int Py = g.Py, LS = XT ? padded_line_stride(Py) : Py | 1, Hx = g.Hx, ny = g.ny, nz = g.nz;
  const int W = 1 << lgW;
  const bool left = !XT && static_cast<int>(blockIdx.x) >= nfull;
  if (left) {
    lgW = 0;
    fnl = fnl1;
  }
  const int kx0 = left ? nfull * W + (static_cast<int>(blockIdx.x) - nfull) : blockIdx.x * W;
  const int z = blockIdx.y, c0 = blockIdx.z * ncompc;
  const int nlines = ncompc << lgW;
  const int rin = MODE == YL_INV ? Py : ny, rout = MODE == YL_FWD ? Py : ny;
  RowsIn<C, IX> src{in + static_cast<int64_t>(c0 * nz + z) * rin * Hx, static_cast<IX>(static_cast<int64_t>(nz) * rin * Hx),
                    static_cast<IX>(Hx), lgW, kx0, Hx, rin};
  RowsOut<C, IX> dst{out + static_cast<int64_t>(c0 * nz + z) * rout * Hx,
                     static_cast<IX>(static_cast<int64_t>(nz) * rout * Hx), static_cast<IX>(Hx), lgW, kx0, Hx, rout};
  if (MODE == YL_CONV2D && XT) {
    // films (nz = 1): the three components of W columns, each contiguous
    const ColsIn<C, IX> cin{in, ny, lgW, kx0, Hx, ny};
    const ColsOut<C, IX> cout{out, ny, lgW, kx0, Hx, ny};
    C* res = line_fft_to_smem<false, NT, true>(cin, a, b, LS, nlines, fnl, g.ply, twy, 1);
    tensor_product<R, true, NT, true>(res, LS, lgW, Py, g.fPy, kx0, 0, Nhat, Hx, Py, g.Pz);
    line_fft_from_smem<true, NT, true>(res, res == a ? b : a, cout, LS, nlines, fnl, g.ply, twy, 1);
  } else if (MODE == YL_CONV2D) {
    C* res = line_fft_to_smem<false, NT>(src, a, b, LS, nlines, fnl, g.ply, twy, 1);
    tensor_product<R, true, NT>(res, LS, lgW, Py, g.fPy, kx0, 0, Nhat, Hx, Py, g.Pz);
    line_fft_from_smem<true, NT>(res, res == a ? b : a, dst, LS, nlines, fnl, g.ply, twy, 1);
  } else if (XT) {
    // 3-D column-major spectra (DemagGeom::yT): the forward pass reads W
    // contiguous columns of X[((c*Hx + kx)*nz + z)*ny + y] and writes Y
    // columns Y[((c*Hx + kx)*nz + z)*Py + ky]; the inverse pass reads Y
    // columns and writes X back row-major (the inverse x pass reads rows)
    const int64_t yoff = (static_cast<int64_t>(c0) * Hx * nz + z) * Py;
    if (MODE == YL_FWD) {
      const ColsIn<C, IX> cin{in + (static_cast<int64_t>(c0) * Hx * nz + z) * ny, nz * ny, lgW, kx0, Hx, ny};
      const ColsOut<C, IX> cout{out + yoff, nz * Py, lgW, kx0, Hx, Py};
      line_fft<false, NT, true>(cin, cout, a, b, LS, nlines, fnl, g.ply, twy, 1);
    } else {
      const ColsIn<C, IX> cin{in + yoff, nz * Py, lgW, kx0, Hx, Py};
      line_fft<true, NT, true>(cin, dst, a, b, LS, nlines, fnl, g.ply, twy, 1);
    }
  } else {
    line_fft<MODE == YL_INV, NT>(src, dst, a, b, LS, nlines, fnl, g.ply, twy, 1);
  }
  }
};


// z lines (forward z, tensor product, inverse z, in place on Y) of one ky row
// over a W-wide kx tile.  grid: (tiles, Py); consecutive blockIdx.y take ky
// and Py - ky so the two reads of each tensor entry are close in time (L2).
// Short z lines (Pz = 3, 5, 7, 9: nz = 2 .. 5) on row-major spectra: one
// thread per (kx, ky) line holds the three components in registers and runs
// the forward transform of its nz inputs as a direct DFT (Pz x nz products),
// the tensor product at every kz and the inverse DFT for the nz kept outputs
// only -- no shared memory, no barrier.  The twiddles w_Pz^t (t < Pz) come with
// the arguments.  (demag.jl:114-123 on the z axis.)
template <typename R, int PZ>
struct ZSmall {
  static constexpr int kNT = 256, kMinB = sizeof(R) == 4 ? 2 : 1;
  static constexpr int NZ = (PZ + 1) / 2;  // nz <= (Pz + 1) / 2 (Pz >= 2 nz - 1)
  struct Args {
    cplx_t<R>* Y;
    const R* __restrict__ Nhat;
    int Hx, Py, nz, Tyq, Tzq;
    R twr[PZ], twi[PZ];  // w^t = exp(-2 pi i t / PZ)
    dim3 grid;
  };
  static __device__ __forceinline__ void body(const Args& a, uint3 blockIdx) {
    using C = cplx_t<R>;
    const int64_t line = static_cast<int64_t>(blockIdx.x) * kNT + threadIdx.x;
    const int Hx = a.Hx, Py = a.Py, nz = a.nz;
    if (line >= static_cast<int64_t>(Hx) * Py) return;
    const int ky = static_cast<int>(line / Hx), kx = static_cast<int>(line - static_cast<int64_t>(ky) * Hx);
    const int64_t zs = static_cast<int64_t>(Py) * Hx, cs = zs * nz;
    C* y0 = a.Y + static_cast<int64_t>(ky) * Hx + kx;
    C x[3][NZ], v[3][PZ];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int n = 0; n < NZ; ++n) x[c][n] = n < nz ? y0[c * cs + n * zs] : cmk<C>(R(0), R(0));
    // forward: v[k] = sum_{n < nz} x[n] w^(nk)
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int k = 0; k < PZ; ++k) {
        C acc = x[c][0];
#pragma unroll
        for (int n = 1; n < NZ; ++n) {
          if (n >= nz) break;
          const int t = (n * k) % PZ;
          acc = cadd(acc, cmul(x[c][n], cmk<C>(a.twr[t], a.twi[t])));
        }
        v[c][k] = acc;
      }
    // tensor product (xy odd in ky, xz in kz, yz in both)
    const bool fy = ky > Py / 2;
    const int kyq = fy ? Py - ky : ky;
    const R sy = fy ? R(-1) : R(1);
    const int64_t Ts = static_cast<int64_t>(a.Tzq) * a.Tyq * Hx;
#pragma unroll
    for (int k = 0; k < PZ; ++k) {
      const bool fz = k > PZ / 2;
      const int kzq = fz ? PZ - k : k;
      const R sz = fz ? R(-1) : R(1);
      const int64_t b = (static_cast<int64_t>(kzq) * a.Tyq + kyq) * Hx + kx;
      const R xx = __ldg(a.Nhat + b), yy = __ldg(a.Nhat + Ts + b), zz = __ldg(a.Nhat + 2 * Ts + b);
      const R xy = sy * __ldg(a.Nhat + 3 * Ts + b), xz = sz * __ldg(a.Nhat + 4 * Ts + b),
              yz = sy * sz * __ldg(a.Nhat + 5 * Ts + b);
      const C p0 = v[0][k], p1 = v[1][k], p2 = v[2][k];
      v[0][k] = cmk<C>(xx * p0.x + xy * p1.x + xz * p2.x, xx * p0.y + xy * p1.y + xz * p2.y);
      v[1][k] = cmk<C>(xy * p0.x + yy * p1.x + yz * p2.x, xy * p0.y + yy * p1.y + yz * p2.y);
      v[2][k] = cmk<C>(xz * p0.x + yz * p1.x + zz * p2.x, xz * p0.y + yz * p1.y + zz * p2.y);
    }
    // inverse, kept outputs n < nz: y[n] = sum_k v[k] w^(-nk)
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int n = 0; n < NZ; ++n) {
        if (n >= nz) break;
        C acc = v[c][0];
#pragma unroll
        for (int k = 1; k < PZ; ++k) {
          const int t = (n * k) % PZ;
          acc = cadd(acc, cmul(v[c][k], cmk<C>(a.twr[t], -a.twi[t])));
        }
        y0[c * cs + n * zs] = acc;
      }
  }
};

template <typename R, int NT, bool I32>
struct ZConv {
  static constexpr int kNT = NT, kMinB = 2;
  struct Args {
    cplx_t<R>* Y;
    const R* __restrict__ Nhat;
    DemagGeom g;
    int lgW;
    FastDiv fnl;
    const cplx_t<R>* __restrict__ twz;
    int half;
    dim3 grid;
  };
  static __device__ __forceinline__ void body(const Args& args, uint3 blockIdx) {
    const auto& [Y, Nhat, g, lgW, fnl, twz, half, grid] = args;

  using C = cplx_t<R>;
  using IX = std::conditional_t<I32, int, int64_t>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* a = reinterpret_cast<C*>(smem_raw);
  C* b = a + half;
  if (g.gate && !*g.gate) return;
  const int Pz = g.Pz, LS = Pz | 1, Hx = g.Hx, Py = g.Py, nz = g.nz;
  const int W = 1 << lgW;
  const int kx0 = blockIdx.x * W;
  const int bq = blockIdx.y;
  const int q = (bq + 1) >> 1;
  const int ky = bq == 0 ? 0 : ((bq & 1) ? q : Py - q);
  const int nlines = 3 * W;
  const IX cs = static_cast<IX>(static_cast<int64_t>(nz) * Py * Hx), rs = static_cast<IX>(static_cast<int64_t>(Py) * Hx);
  RowsIn<C, IX> src{Y + static_cast<int64_t>(ky) * Hx, cs, rs, lgW, kx0, Hx, nz};
  RowsOut<C, IX> dst{Y + static_cast<int64_t>(ky) * Hx, cs, rs, lgW, kx0, Hx, nz};
  C* res = line_fft_to_smem<false, NT>(src, a, b, LS, nlines, fnl, g.plz, twz, 1);
  tensor_product<R, false, NT>(res, LS, lgW, Pz, g.fPz, kx0, ky, Nhat, Hx, Py, Pz);
  line_fft_from_smem<true, NT>(res, res == a ? b : a, dst, LS, nlines, fnl, g.plz, twz, 1);
  }
};


// descriptors the persistent step kernel runs (mm_persist.cu)
template <typename R> struct PersistKind<FwdX<R, XM_MAGN, kHotNT>> { static constexpr int value = 0; };
template <typename R> struct PersistKind<InvX<R, kHotNT>> { static constexpr int value = 1; };
template <typename R> struct PersistKind<YLines<R, YL_FWD, kHotNT, true, false>> { static constexpr int value = 2; };
template <typename R> struct PersistKind<YLines<R, YL_INV, kHotNT, true, false>> { static constexpr int value = 3; };
template <typename R> struct PersistKind<YLines<R, YL_CONV2D, kHotNT, true, false>> { static constexpr int value = 4; };
template <typename R> struct PersistKind<YLines<R, YL_CONV2D, kHotNT, true, true>> { static constexpr int value = 5; };
template <typename R> struct PersistKind<ZConv<R, kHotNT, true>> { static constexpr int value = 6; };
template <typename R> struct PersistKind<ZSmall<R, 3>> { static constexpr int value = 7; };
template <typename R> struct PersistKind<ZSmall<R, 5>> { static constexpr int value = 8; };
template <typename R> struct PersistKind<ZSmall<R, 7>> { static constexpr int value = 9; };
template <typename R> struct PersistKind<ZSmall<R, 9>> { static constexpr int value = 10; };

}  // namespace mm

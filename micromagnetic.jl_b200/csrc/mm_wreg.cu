// mm_wreg.cu -- register-resident x and y passes of the demag convolution for
// power-of-two meshes, FP32 form (internal).
//
// Applies when nx = Lc and ny are 32 Q with Q in {4, 8, 16, 32} (padded
// Px = 2 nx, Py = 2 ny), on 3-D meshes.  Every line is transformed by a group
// of Q lanes holding 32 values each (mm_wfft.cuh); shared memory only carries
// the warp transposes and the block's staging of coalesced HBM segments, and
// each block synchronises three or four times.  Layout (DemagGeom::wreg):
//   X  [3][Hx][nz][ny] column-major in both directions (the x passes stage
//      tiles of RB consecutive rows through shared memory so that a column
//      segment of RB rows is one coalesced HBM access);
//   Y  [3][Hx][nz][Py] column-major, as for DemagGeom::yT.
// The zero padding is pruned: the x transform of real rows packs pairs
// (x[2n], x[2n+1]) into the Lc-point complex transform, half of whose inputs
// are zero; the forward y transform of ny inputs into Py = 2 ny outputs is
// two ny-point transforms by output parity s,
//     Y[2k + s] = DFT_ny(x[n] w_Py^(n s))[k],
// and the inverse keeps y < ny as u0[y] + w_Py^(-y) u1[y], us the ny-point
// inverse transform of Y[2k + s].  (src/micro/demag.jl:102-131.)
#include <algorithm>
#include <cstdlib>

#include "mm_demag.cuh"
#include "mm_wfft.cuh"

namespace mm {

namespace {

constexpr int kWyNT = 256;  // y passes: 8 warps, 4 lines x 2 halves (Q = 32)

// rows of one x-pass block: W warps x (32 / Q) groups
template <int Q, int W> constexpr int x_rows() { return W * (32 / Q); }
// Staging stride (complex values between consecutive k of the block's RB
// rows): lanes of a half warp touch 16 distinct 8-byte banks, i.e. the stride
// is odd for Q >= 16 (one group of 16 lanes) and 2 or 4 mod 16 for Q = 8 or 4
// (lane groups side by side; RB is then a multiple of 16).
template <int Q, int W> constexpr int x_stride() { return x_rows<Q, W>() + (Q >= 16 ? 1 : (Q == 8 ? 2 : 4)); }
// shared memory of an x-pass block (complex values): the transpose tiles or
// the staged rows
template <int Q, int W> constexpr int x_smem() {
  return W * wtile_size<Q>() > (32 * Q + 1) * x_stride<Q, W>() ? W * wtile_size<Q>()
                                                                : (32 * Q + 1) * x_stride<Q, W>();
}

// Warps of an x-pass block: the FP32 forward pass runs 4 (128 registers,
// four blocks an SM), the inverse pass 8 (128 registers, two blocks an SM), which moves
// column segments of RB = 8 rows (64 bytes for Q = 32).  Measured on c5
// (1024 x 1024 x 16, Q = 32): forward 0.248 ms with 4 warps, 0.273 with 8
// (0.287 with 4 capped at 96 registers); inverse 0.287 ms with 4 warps, 0.273
// with 8.  FP64 blocks run 4 warps in both directions (RB = 4 rows of 16-byte
// values: 64-byte segments, 82 KB of shared memory, two blocks an SM).
template <typename R> constexpr int x_fwd_warps() { return 4; }
template <typename R> constexpr int x_inv_warps() { return sizeof(R) == 4 ? 8 : 4; }
template <typename R, int W> constexpr int x_fwd_minb() { return sizeof(R) == 4 ? 4 : 2; }
// two blocks an SM: the FP32 inverse pass capped at 80 registers (three
// blocks) spilled, and took 0.258 ms on c5 against 0.200 with 128 registers
template <typename R, int W> constexpr int x_inv_minb() { return 2; }

// ---------------------------------------------------------------- x forward
// Rows of m * mu0Ms (zero padded to Px = 2 Lc) -> X column-major.  A block
// transforms its RB rows for the three components in turn, so that each row
// of Ms is read from HBM once (the later reads hit the caches; c5: 0.243 ->
// 0.235 ms against blocks of one component).
template <int Q, int W, typename R>
__global__ void __launch_bounds__(32 * W, (x_fwd_minb<R, W>())) k_xfwd_w(const R* __restrict__ m, const R* __restrict__ Ms,
                                                  cplx_t<R>* __restrict__ X, DemagGeom g, const cplx_t<R>* __restrict__ twx) {
  using C = cplx_t<R>;
  constexpr int RB = x_rows<Q, W>(), L = 32 * Q, S = x_stride<Q, W>();
  extern __shared__ __align__(16) unsigned char xsm_raw[];  // x_smem<Q, W>() values
  C* sm = reinterpret_cast<C*>(xsm_raw);
  pdl_enter();
  if (g.gate && !*g.gate) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gq = lane / Q, q = lane % Q;
  const int rows = g.ny * g.nz, Hx = g.Hx, nx = g.nx;
  const int64_t N = static_cast<int64_t>(rows) * nx;
  const int row0 = blockIdx.x * RB;  // rows % RB == 0
  const int rl = warp * (32 / Q) + gq;
  const int64_t rb = static_cast<int64_t>(row0 + rl) * nx;
  const C* s2 = reinterpret_cast<const C*>(Ms + rb);
  constexpr int KS = 32 * W / RB;
  const int r = threadIdx.x & (RB - 1), k0 = threadIdx.x / RB;
  const int64_t step = static_cast<int64_t>(KS) * rows;
#pragma unroll 1
  for (int c = 0; c < 3; ++c) {
    const C* m2 = reinterpret_cast<const C*>(m + c * N + rb);
    C v[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      if (j < 16) {  // z[n] = (x[2n], x[2n+1]), nonzero for n < Lc / 2
        const C a = m2[q + Q * j], b = s2[q + Q * j];
        v[j] = cmk<C>(a.x * b.x, a.y * b.y);
      } else {
        v[j] = cmk<C>(R(0), R(0));
      }
    }
    if (c > 0) __syncthreads();  // the previous component's staged rows are written out
    wfft<Q, false, 2>(v, sm + warp * wtile_size<Q>(), twx);
    __syncthreads();  // every warp is done with its transpose tile
#pragma unroll
    for (int r = 0; r < 32; ++r) sm[(q + Q * (r / Q) + 32 * (r % Q)) * S + rl] = v[r];
    __syncthreads();
    // X[k] = E + w_Px^k O, E = (Z[k] + conj Z[Lc-k]) / 2, O = (Z[k] - conj Z[Lc-k]) / 2i
    // (Z is L-periodic: k = L reads Z[0]).  Thread (k0, r) writes row r of
    // k = k0, k0 + KS, ... through a pointer stepped by KS columns.
    C* xp = X + (static_cast<int64_t>(c) * Hx + k0) * rows + row0 + r;
#pragma unroll 4
    for (int k = k0; k < Hx; k += KS, xp += step) {
      const C zk = sm[(k & (L - 1)) * S + r];
      C zc = sm[((L - k) & (L - 1)) * S + r];
      zc.y = -zc.y;
      const C ev = cmk<C>(R(0.5) * (zk.x + zc.x), R(0.5) * (zk.y + zc.y));
      const C od = cmk<C>(R(0.5) * (zk.y - zc.y), R(-0.5) * (zk.x - zc.x));
      *xp = cadd(ev, cmul(__ldg(twx + k), od));
    }
  }
}

// ---------------------------------------------------------------- x inverse
// X column-major -> real rows (c2r, unnormalised), keeps x < nx.
template <int Q, int W, typename R>
__global__ void __launch_bounds__(32 * W, (x_inv_minb<R, W>())) k_xinv_w(const cplx_t<R>* __restrict__ X, R* __restrict__ H,
                                                  DemagGeom g, const cplx_t<R>* __restrict__ twx) {
  using C = cplx_t<R>;
  constexpr int RB = x_rows<Q, W>(), L = 32 * Q, S = x_stride<Q, W>();
  extern __shared__ __align__(16) unsigned char xsm_raw[];  // x_smem<Q, W>() values
  C* sm = reinterpret_cast<C*>(xsm_raw);
  pdl_enter();
  if (g.gate && !*g.gate) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gq = lane / Q, q = lane % Q;
  const int rows = g.ny * g.nz, Hx = g.Hx, nx = g.nx;
  const int64_t N = static_cast<int64_t>(rows) * nx;
  const int line0 = blockIdx.x * RB;
  const int c = line0 / rows, row0 = line0 - c * rows;
  const int rl = warp * (32 / Q) + gq;
  {
    // thread (k0, r) stages row r of k = k0, k0 + KS, ... with cp.async, so
    // that all of its copies are in flight at once without holding registers;
    // each miss fetches 256 bytes into L2 (the column segments of the next
    // blocks, which run alongside this one)
    constexpr int KS = 32 * W / RB;
    const int r = threadIdx.x & (RB - 1), k0 = threadIdx.x / RB;
    const int64_t step = static_cast<int64_t>(KS) * rows;
    const C* xp = X + (static_cast<int64_t>(c) * Hx + k0) * rows + row0 + r;
    unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(sm + k0 * S + r));
    for (int k = k0; k < Hx; k += KS, xp += step, sa += KS * S * sizeof(C)) {
      if constexpr (sizeof(C) == 8)
        asm volatile("cp.async.ca.shared.global.L2::256B [%0], [%1], 8;\n" ::"r"(sa), "l"(xp) : "memory");
      else
        asm volatile("cp.async.ca.shared.global.L2::256B [%0], [%1], 16;\n" ::"r"(sa), "l"(xp) : "memory");
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  }
  __syncthreads();
  // Z'[k] = (A + B) + i (A - B) conj(w_Px^k), A = X[k], B = conj X[Lc - k]
  C v[32];
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    const int k = q + Q * j;
    const C a = sm[k * S + rl];
    C b = sm[(L - k) * S + rl];
    b.y = -b.y;
    C w = __ldg(twx + k);
    w.y = -w.y;
    const C d = cmul(csub(a, b), w);
    v[j] = cmk<C>(a.x + b.x - d.y, a.y + b.y + d.x);
  }
  __syncthreads();  // the staging tile becomes the transpose tiles
  wfft<Q, true, 2>(v, sm + warp * wtile_size<Q>(), twx);
  // z[n] = (x[2n], x[2n+1]) for n < Lc / 2: registers with k2 = r % Q < Q / 2
  C* h2 = reinterpret_cast<C*>(H + c * N + static_cast<int64_t>(row0 + rl) * nx);
#pragma unroll
  for (int r = 0; r < 32; ++r) {
    if (r % Q < Q / 2) h2[q + Q * (r / Q) + 32 * (r % Q)] = v[r];
  }
}

// ---------------------------------------------------------------- y forward
// X column (ny values) -> Y column (Py = 2 ny values); line = (c Hx + kx) nz + z.
// Unit u = group in the block: line (u >> 1), half s = u & 1.
template <int Q>
__global__ void __launch_bounds__(kWyNT, 3) k_yfwd_w(const float2* __restrict__ X, float2* __restrict__ Y, DemagGeom g,
                                                 const float2* __restrict__ twy, int nlines) {
  constexpr int NL = 4 * (32 / Q), Py = 64 * Q;  // lines a block, padded length
  extern __shared__ __align__(16) float2 smy[];
  pdl_enter();
  if (g.gate && !*g.gate) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gq = lane / Q, q = lane % Q;
  const int u = warp * (32 / Q) + gq, s = u & 1, ll = u >> 1;
  const int line0 = blockIdx.x * NL;
  const int line = line0 + ll;
  const bool live = line < nlines;
  const float2* xc = X + static_cast<int64_t>(line) * (Py / 2);
  float2 v[32];
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    float2 a = live ? xc[q + Q * j] : make_float2(0.f, 0.f);
    if (s) a = cmul(a, __ldg(twy + q + Q * j));
    v[j] = a;
  }
  wfft<Q, false, 2>(v, smy + warp * wtile_size<Q>(), twy);
  __syncthreads();  // transposes done: the tiles become the block's output columns
  // Y[2k + s] of line ll staged as half column (ll, s), k contiguous
  float2* half = smy + (2 * ll + s) * (Py / 2);
#pragma unroll
  for (int r = 0; r < 32; ++r) half[q + Q * (r / Q) + 32 * (r % Q)] = v[r];
  __syncthreads();
  const int nl = min(NL, nlines - line0);
  float4* dst = reinterpret_cast<float4*>(Y + static_cast<int64_t>(line0) * Py);
  for (int e = threadIdx.x; e < nl * Py / 2; e += kWyNT) {
    const int l = e / (Py / 2), k = e - l * (Py / 2);
    const float2 a = smy[(2 * l) * (Py / 2) + k], b = smy[(2 * l + 1) * (Py / 2) + k];
    dst[e] = make_float4(a.x, a.y, b.x, b.y);
  }
}

// ---------------------------------------------------------------- y inverse
// Y column (Py values) -> X column (y < ny).
template <int Q>
__global__ void __launch_bounds__(kWyNT, 3) k_yinv_w(const float2* __restrict__ Y, float2* __restrict__ X, DemagGeom g,
                                                 const float2* __restrict__ twy, int nlines) {
  constexpr int NL = 4 * (32 / Q), Py = 64 * Q, ny = 32 * Q;
  extern __shared__ __align__(16) float2 smy[];
  pdl_enter();
  if (g.gate && !*g.gate) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gq = lane / Q, q = lane % Q;
  const int u = warp * (32 / Q) + gq, s = u & 1, ll = u >> 1;
  const int line0 = blockIdx.x * NL;
  const int nl = min(NL, nlines - line0);
  {
    // Y[2k + s] of line l staged as half column (l, s), k contiguous
    const float4* src = reinterpret_cast<const float4*>(Y + static_cast<int64_t>(line0) * Py);
    for (int e = threadIdx.x; e < nl * Py / 2; e += kWyNT) {
      const int l = e / (Py / 2), k = e - l * (Py / 2);
      const float4 p = src[e];
      smy[(2 * l) * (Py / 2) + k] = make_float2(p.x, p.y);
      smy[(2 * l + 1) * (Py / 2) + k] = make_float2(p.z, p.w);
    }
  }
  __syncthreads();
  float2 v[32];
  const float2* col = smy + (2 * ll + s) * (Py / 2);
#pragma unroll
  for (int j = 0; j < 32; ++j) v[j] = ll < nl ? col[q + Q * j] : make_float2(0.f, 0.f);
  __syncthreads();  // the staged columns become the transpose tiles
  wfft<Q, true, 2>(v, smy + warp * wtile_size<Q>(), twy);
  if (s) {
#pragma unroll
    for (int r = 0; r < 32; ++r) {
      float2 w = __ldg(twy + q + Q * (r / Q) + 32 * (r % Q));
      w.y = -w.y;
      v[r] = cmul(v[r], w);
    }
  }
  __syncthreads();
  float2* half = smy + (ll * 2 + s) * ny;
#pragma unroll
  for (int r = 0; r < 32; ++r) half[q + Q * (r / Q) + 32 * (r % Q)] = v[r];
  __syncthreads();
  float2* xo = X + static_cast<int64_t>(line0) * ny;
  for (int e = threadIdx.x; e < nl * ny; e += kWyNT) {
    const int l = e / ny, y = e - l * ny;
    const float2 a = smy[(2 * l) * ny + y], b = smy[(2 * l + 1) * ny + y];
    xo[e] = make_float2(a.x + b.x, a.y + b.y);
  }
}

// ------------------------------------------------- y passes, warp-direct
// The same transforms with no block-wide barrier: every group reads its
// inputs from and writes its outputs to HBM directly, so the warps of a
// block run their load, transform and store phases independently and the
// loads of some warps overlap the arithmetic of others.  Half s of a line
// touches every other complex value of the padded column (Y[2k + s]); the two
// halves of a line (the two groups of a warp for Q = 16, a warp pair for
// Q = 32) cover whole 32-byte sectors between them.
constexpr int kWdNT = 256;

// The warp-direct y passes unless MMCUDA_YDIRECT=0 keeps the block-staged ones
bool ydirect_enabled() {
  static const bool on = [] {
    const char* e = getenv("MMCUDA_YDIRECT");
    return !(e && e[0] == '0');
  }();
  return on;
}

template <int Q>
__global__ void __launch_bounds__(kWdNT, 3) k_yfwd_d(const float2* __restrict__ X, float2* __restrict__ Y, DemagGeom g,
                                                 const float2* __restrict__ twy, int nlines) {
  constexpr int Py = 64 * Q;
  extern __shared__ __align__(16) float2 tiles[];  // (kWdNT / 32) warp tiles
  pdl_enter();
  if (g.gate && !*g.gate) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gq = lane / Q, q = lane % Q;
  const int u = (blockIdx.x * (kWdNT / 32) + warp) * (32 / Q) + gq, s = u & 1;
  const int line = u >> 1;
  if (line >= nlines) return;  // both halves of a line (whole warps) leave together
  const float2* xc = X + static_cast<int64_t>(line) * (Py / 2);
  float2 v[32];
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    float2 a = xc[q + Q * j];
    if (s) a = cmul(a, __ldg(twy + q + Q * j));
    v[j] = a;
  }
  wfft<Q, false, 2>(v, tiles + warp * wtile_size<Q>(), twy);
  float2* yc = Y + static_cast<int64_t>(line) * Py + s;
#pragma unroll
  for (int r = 0; r < 32; ++r) yc[2 * (q + Q * (r / Q) + 32 * (r % Q))] = v[r];
}

template <int Q>
__global__ void __launch_bounds__(kWdNT, 3) k_yinv_d(const float2* __restrict__ Y, float2* __restrict__ X, DemagGeom g,
                                                 const float2* __restrict__ twy, int nlines) {
  constexpr int Py = 64 * Q, ny = 32 * Q;
  extern __shared__ __align__(16) float2 tiles[];  // (kWdNT / 32) warp tiles
  pdl_enter();
  if (g.gate && !*g.gate) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gq = lane / Q, q = lane % Q;
  const int u = (blockIdx.x * (kWdNT / 32) + warp) * (32 / Q) + gq, s = u & 1;
  const int line = u >> 1;
  // a Q = 32 warp pair meets at a named barrier: both warps of a pair hold
  // the same line, so they stay or leave together
  if (line >= nlines) return;
  const float2* yc = Y + static_cast<int64_t>(line) * Py + s;
  float2 v[32];
#pragma unroll
  for (int j = 0; j < 32; ++j) v[j] = yc[2 * (q + Q * j)];
  float2* tile = tiles + warp * wtile_size<Q>();
  wfft<Q, true, 2>(v, tile, twy);
  if (s) {
#pragma unroll
    for (int r = 0; r < 32; ++r) {
      float2 w = __ldg(twy + q + Q * (r / Q) + 32 * (r % Q));
      w.y = -w.y;
      v[r] = cmul(v[r], w);
    }
  }
  // x[y] = u0[y] + w^(-y) u1[y], y = q + Q (r / Q) + 32 (r % Q): half s keeps
  // the registers r with r % 2 == s and receives those from its partner
  float2* xo = X + static_cast<int64_t>(line) * ny;
  if constexpr (Q == 32) {
    // partner = the other warp of the pair: send through this warp's tile
#pragma unroll
    for (int i = 0; i < 16; ++i) tile[i * 32 + lane] = s ? v[2 * i] : v[2 * i + 1];
    asm volatile("bar.sync %0, 64;\n" ::"r"(1 + (warp >> 1)) : "memory");
    const float2* pt = tiles + (warp ^ 1) * wtile_size<Q>();
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      const float2 a = s ? v[2 * i + 1] : v[2 * i], b = pt[i * 32 + lane];
      xo[q + 32 * (2 * i + s)] = make_float2(a.x + b.x, a.y + b.y);
    }
  } else {
    // partner = the other group of this warp (lane ^ Q)
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      const float2 mine = s ? v[2 * i + 1] : v[2 * i], send = s ? v[2 * i] : v[2 * i + 1];
      const float bx = __shfl_xor_sync(0xffffffffu, send.x, Q);
      const float by = __shfl_xor_sync(0xffffffffu, send.y, Q);
      const int r = 2 * i + s;
      xo[q + Q * (r / Q) + 32 * (r % Q)] = make_float2(mine.x + bx, mine.y + by);
    }
  }
}

// ------------------------------------------ y passes, Q = 32, bulk-copy fed
// One block of two warps (the two output parities of a line) walks lines
// blockIdx.x, blockIdx.x + gridDim.x, ...  Its input line arrives in shared
// memory by one bulk copy (cp.async.bulk, completion counted on an
// mbarrier); as soon as both warps hold the line in registers the copy of
// the block's next line is issued into the same buffer, so the load of line
// i + 1 overlaps the transform and the stores of line i.  Waits on the
// mbarrier are bounded (copy_wait_spins() tries): a wait that runs out sets
// g_wreg_timeout, waits once more (a fixed, larger bound) for the copy in
// flight, and the block leaves; mm_synchronize reports it as MM_ERR_TIMEOUT.
constexpr int kWpNT = 64;
constexpr unsigned kDrainSpins = 1u << 24;  // the second wait, after a timeout
__device__ int g_wreg_timeout;

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_addr(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
// one arrival that also expects `bytes` of copies, then the copy itself
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");  // earlier reads of dst before the copy's writes
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, unsigned spins) {
  const unsigned a = smem_addr(bar);
  for (unsigned i = 0; i < spins; ++i) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}
// the bounded wait of every thread of the block, with one outcome for all
__device__ __forceinline__ bool block_wait(unsigned long long* bar, unsigned parity, unsigned spins) {
  const bool ok = mbar_wait(bar, parity, spins);
  if (__syncthreads_or(!ok)) {
    if ((threadIdx.x & 31) == 0) asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory");  // bulk stores in flight complete
    if (threadIdx.x == 0) atomicExch(&g_wreg_timeout, 1);
    mbar_wait(bar, parity, kDrainSpins);  // the copy in flight lands before the block leaves
    return false;
  }
  return true;
}
// one bulk copy of `bytes` from shared to global memory, in its own group;
// the writes of every thread to src must precede it (fence + barrier)
__device__ __forceinline__ void bulk_store(void* dst, const void* src, unsigned bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;\n" ::"l"(dst), "r"(smem_addr(src)),
               "r"(bytes)
               : "memory");
  asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
}

// forward: X column (1024 values) -> Y column (2048), Y[2k + s] from warp s.
// The staged output line leaves by one bulk copy issued by thread 0: the
// warps go on to the next line at once, and the staging tiles are reused only
// after that copy has read them (c5: 0.358 -> 0.272 ms against 16-byte stores
// of every thread).  FP32 and FP64 (C = float2 or double2).
template <typename R>
__global__ void __launch_bounds__(kWpNT, sizeof(R) == 4 ? 8 : 4) k_yfwd_p(const cplx_t<R>* __restrict__ X,
                                                                        cplx_t<R>* __restrict__ Y, DemagGeom g,
                                                                        const cplx_t<R>* __restrict__ twy, int nlines,
                                                                        unsigned spins) {
  using C = cplx_t<R>;
  constexpr int NY = 1024, Py = 2048;
  extern __shared__ __align__(128) unsigned char yfp_raw[];
  C* sp = reinterpret_cast<C*>(yfp_raw);
  C* buf = sp;                                                          // NY
  C* tile = sp + NY + (threadIdx.x >> 5) * wtile_size<32>();           // this warp's
  auto* bar = reinterpret_cast<unsigned long long*>(sp + NY + 2 * wtile_size<32>());
  pdl_enter();
  if (g.gate && !*g.gate) return;
  int line = blockIdx.x;
  if (line >= nlines) return;
  const int lane = threadIdx.x & 31, s = threadIdx.x >> 5;
  if (threadIdx.x == 0) {
    mbar_init(bar);
    bulk_load(buf, X + static_cast<int64_t>(line) * NY, NY * sizeof(C), bar);
  }
  __syncthreads();
  for (unsigned it = 0; line < nlines; ++it, line += gridDim.x) {
    if (!block_wait(bar, it & 1, spins)) return;
    C v[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      C a = buf[lane + 32 * j];
      if (s) a = cmul(a, __ldg(twy + lane + 32 * j));
      v[j] = a;
    }
    // the previous line's bulk store has read the staging tiles
    if (threadIdx.x == 0) asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory");
    __syncthreads();  // both warps hold the line: the buffer takes the next one
    if (threadIdx.x == 0 && line + static_cast<int>(gridDim.x) < nlines)
      bulk_load(buf, X + static_cast<int64_t>(line + gridDim.x) * NY, NY * sizeof(C), bar);
    wfft<32, false, 2>(v, tile, twy);
    // the two parities interleave in the tiles' space (2048 values), which
    // leave as one copy (Y[2k], Y[2k + 1], ...)
    __syncthreads();
    C* stg = sp + NY;
#pragma unroll
    for (int r = 0; r < 32; ++r) stg[2 * (lane + 32 * r) + s] = v[r];
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");  // the staged line, to the copy engine
    __syncthreads();
    if (threadIdx.x == 0) bulk_store(Y + static_cast<int64_t>(line) * Py, stg, Py * sizeof(C));
  }
  // the shared memory of the last store stays valid until the copy is done
  if (threadIdx.x == 0) asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory");
}

// inverse: Y column (2048 values) -> X column (y < 1024); warp s transforms
// Y[2k + s] and the pair adds u0[y] + w^(-y) u1[y] through the warp tiles,
// warp s producing y in [512 s, 512 s + 512).  BULK (the FP32 form): each
// warp stages its half in the upper part of its own tile (the lower part
// carries what it sends) and its lane 0 writes it by one bulk copy; else every
// thread stores.  Measured on c5: FP32 0.305 -> 0.292 ms with the bulk copy,
// FP64 0.775 -> 0.836 ms (slower), so FP64 keeps the thread stores.
template <typename R, bool BULK>
__global__ void __launch_bounds__(kWpNT, sizeof(R) == 4 ? 6 : 3) k_yinv_p(const cplx_t<R>* __restrict__ Y,
                                                                        cplx_t<R>* __restrict__ X, DemagGeom g,
                                                                        const cplx_t<R>* __restrict__ twy, int nlines,
                                                                        unsigned spins) {
  using C = cplx_t<R>;
  constexpr int NY = 1024, Py = 2048;
  extern __shared__ __align__(128) unsigned char yip_raw[];
  C* sp = reinterpret_cast<C*>(yip_raw);
  C* buf = sp;                                          // Py
  C* tiles = sp + Py;                                   // two warp tiles
  auto* bar = reinterpret_cast<unsigned long long*>(sp + Py + 2 * wtile_size<32>());
  pdl_enter();
  if (g.gate && !*g.gate) return;
  int line = blockIdx.x;
  if (line >= nlines) return;
  const int lane = threadIdx.x & 31, s = threadIdx.x >> 5;
  C* tile = tiles + s * wtile_size<32>();
  const C* pt = tiles + (s ^ 1) * wtile_size<32>();
  if (threadIdx.x == 0) {
    mbar_init(bar);
    bulk_load(buf, Y + static_cast<int64_t>(line) * Py, Py * sizeof(C), bar);
  }
  __syncthreads();
  for (unsigned it = 0; line < nlines; ++it, line += gridDim.x) {
    if (!block_wait(bar, it & 1, spins)) return;
    C v[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] = buf[2 * (lane + 32 * j) + s];
    // this warp's previous bulk store has read its staging half
    if (BULK && lane == 0) asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory");
    __syncthreads();  // both warps hold the line (and are done with last line's tiles)
    if (threadIdx.x == 0 && line + static_cast<int>(gridDim.x) < nlines)
      bulk_load(buf, Y + static_cast<int64_t>(line + gridDim.x) * Py, Py * sizeof(C), bar);
    wfft<32, true, 2>(v, tile, twy);
    if (s) {
#pragma unroll
      for (int r = 0; r < 32; ++r) {
        C w = __ldg(twy + lane + 32 * r);
        w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
    }
    // y = lane + 32 r: warp s keeps r in [16 s, 16 s + 16) and sends the others
#pragma unroll
    for (int i = 0; i < 16; ++i) tile[i * 32 + lane] = s ? v[i] : v[16 + i];
    __syncthreads();
    C* xo = X + static_cast<int64_t>(line) * NY + 512 * s;
    C* stg = tile + 512;  // words 512..1023 of this warp's tile
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      const C a = s ? v[16 + i] : v[i], b = pt[i * 32 + lane];
      if (BULK) stg[lane + 32 * i] = cmk<C>(a.x + b.x, a.y + b.y);
      else xo[lane + 32 * i] = cmk<C>(a.x + b.x, a.y + b.y);
    }
    if (BULK) {
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");  // the staged half, to the copy engine
      __syncwarp();
      if (lane == 0) bulk_store(xo, stg, 512 * sizeof(C));
    }
  }
  // the shared memory of the last store stays valid until the copy is done
  if (BULK && lane == 0) asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory");
}

static_assert(2 * wtile_size<32>() >= 2048, "the forward pass stages a padded line in its warp tiles");
template <typename R> constexpr size_t yfp_smem() { return (1024 + 2 * wtile_size<32>()) * sizeof(cplx_t<R>) + 8; }
template <typename R> constexpr size_t yip_smem() { return (2048 + 2 * wtile_size<32>()) * sizeof(cplx_t<R>) + 8; }

// The bulk-copy y passes for Q = 32 unless MMCUDA_YPIPE=0 (warp-direct ones)
bool ypipe_enabled() {
  static const bool on = [] {
    const char* e = getenv("MMCUDA_YPIPE");
    return !(e && e[0] == '0');
  }();
  return on;
}
// resident blocks of a persistent pass on the current device
int resident_blocks(const void* kernel, int nt, size_t smem) {
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, nt, smem);
  return std::max(1, sms) * std::max(1, per);
}

template <int Q, typename R>
void launch_q(int which, const DemagGeom& g, const R* m, const R* Ms, cplx_t<R>* X, cplx_t<R>* Y, R* H,
              const cplx_t<R>* twx, const cplx_t<R>* twy, cudaStream_t st) {
  using C = cplx_t<R>;
  constexpr int XF = x_fwd_warps<R>(), XI = x_inv_warps<R>();
  const int rows = g.ny * g.nz;
  const int ylines = 3 * g.Hx * g.nz;
  switch (which) {
    case 0:
      launch_pdl(k_xfwd_w<Q, XF, R>, dim3(rows / x_rows<Q, XF>()), dim3(32 * XF), x_smem<Q, XF>() * sizeof(C), st, m,
                 Ms, X, g, twx);
      break;
    case 1:
      if (Q == 32 && (sizeof(R) == 8 || ypipe_enabled())) {
        static const int nb = resident_blocks(reinterpret_cast<const void*>(&k_yfwd_p<R>), kWpNT, yfp_smem<R>());
        launch_pdl(k_yfwd_p<R>, dim3(std::min(ylines, nb)), dim3(kWpNT), yfp_smem<R>(), st, X, Y, g, twy, ylines,
                   copy_wait_spins());
      } else if constexpr (sizeof(R) == 4) {
        constexpr int NL = 4 * (32 / Q), DL = (kWdNT / 32) * (32 / Q) / 2;
        const size_t ysm = static_cast<size_t>(8) * wtile_size<Q>() * sizeof(float2);
        if (ydirect_enabled())
          launch_pdl(k_yfwd_d<Q>, dim3((ylines + DL - 1) / DL), dim3(kWdNT), ysm, st, X, Y, g, twy, ylines);
        else
          launch_pdl(k_yfwd_w<Q>, dim3((ylines + NL - 1) / NL), dim3(kWyNT), ysm, st, X, Y, g, twy, ylines);
      }
      break;
    case 3:
      if (Q == 32 && (sizeof(R) == 8 || ypipe_enabled())) {
        constexpr bool kBulk = sizeof(R) == 4;
        static const int nb = resident_blocks(reinterpret_cast<const void*>(&k_yinv_p<R, kBulk>), kWpNT, yip_smem<R>());
        launch_pdl(k_yinv_p<R, kBulk>, dim3(std::min(ylines, nb)), dim3(kWpNT), yip_smem<R>(), st, Y, X, g, twy, ylines,
                   copy_wait_spins());
      } else if constexpr (sizeof(R) == 4) {
        constexpr int NL = 4 * (32 / Q), DL = (kWdNT / 32) * (32 / Q) / 2;
        const size_t ysm = static_cast<size_t>(8) * wtile_size<Q>() * sizeof(float2);
        if (ydirect_enabled())
          launch_pdl(k_yinv_d<Q>, dim3((ylines + DL - 1) / DL), dim3(kWdNT), ysm, st, Y, X, g, twy, ylines);
        else
          launch_pdl(k_yinv_w<Q>, dim3((ylines + NL - 1) / NL), dim3(kWyNT), ysm, st, Y, X, g, twy, ylines);
      }
      break;
    case 4:
      launch_pdl(k_xinv_w<Q, XI, R>, dim3(3 * rows / x_rows<Q, XI>()), dim3(32 * XI), x_smem<Q, XI>() * sizeof(C), st,
                 X, H, g, twx);
      break;
    default:
      break;
  }
}

template <int Q>
void set_attrs_q() {
  const int b = 8 * wtile_size<Q>() * static_cast<int>(sizeof(float2));
  cudaFuncSetAttribute(k_yfwd_w<Q>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
  cudaFuncSetAttribute(k_yinv_w<Q>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
  cudaFuncSetAttribute(k_yfwd_d<Q>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
  cudaFuncSetAttribute(k_yinv_d<Q>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
  constexpr int XF = x_fwd_warps<float>(), XI = x_inv_warps<float>();
  cudaFuncSetAttribute(k_xfwd_w<Q, XF, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       static_cast<int>(x_smem<Q, XF>() * sizeof(float2)));
  cudaFuncSetAttribute(k_xinv_w<Q, XI, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       static_cast<int>(x_smem<Q, XI>() * sizeof(float2)));
}

// FP64: x passes for Q = 16, 32, y passes for Q = 32
template <int Q>
void set_attrs_q64() {
  constexpr int XF = x_fwd_warps<double>(), XI = x_inv_warps<double>();
  cudaFuncSetAttribute(k_xfwd_w<Q, XF, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       static_cast<int>(x_smem<Q, XF>() * sizeof(double2)));
  cudaFuncSetAttribute(k_xinv_w<Q, XI, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       static_cast<int>(x_smem<Q, XI>() * sizeof(double2)));
}

int wq(int n) {
  switch (n) {
    case 128: return 4;
    case 256: return 8;
    case 512: return 16;
    case 1024: return 32;
    default: return 0;
  }
}

}  // namespace

// ny >= 512: with shorter y lines the shared-memory y passes (wide row tiles)
// and the row-major z kernel measured faster (c2, 256 x 256 x 64: 2.77 vs
// 2.71 ms a step; c5, 1024 x 1024 x 16: 10.3 vs 12.7 ms).  The FP64 form
// takes nx = 512 or 1024 and ny = 1024 (the bulk-copy y passes).
bool wreg_applies(int nx, int ny, int nz, int Px, int Py, bool f64) {
  if (!(nz > 1 && wq(nx) && wq(ny) && ny >= 512 && Px == 2 * nx && Py == 2 * ny)) return false;
  return !f64 || (wq(nx) >= 16 && ny == 1024);
}

void wreg_set_attrs() {
  set_attrs_q<4>();
  set_attrs_q<8>();
  set_attrs_q<16>();
  set_attrs_q<32>();
  set_attrs_q64<16>();
  set_attrs_q64<32>();
  cudaFuncSetAttribute(k_yfwd_p<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       static_cast<int>(yfp_smem<double>()));
  cudaFuncSetAttribute(k_yinv_p<double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       static_cast<int>(yip_smem<double>()));
}

bool wreg_take_timeout() {
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, g_wreg_timeout, sizeof(int)) != cudaSuccess || !v) return false;
  const int zero = 0;
  cudaMemcpyToSymbol(g_wreg_timeout, &zero, sizeof(int));
  return true;
}

void launch_wreg(int which, const DemagGeom& g, const float* m, const float* Ms, float2* X, float2* Y, float* H,
                 const float2* twx, const float2* twy, cudaStream_t st) {
  // the x passes run on rows (Q of nx), the y passes on columns (Q of ny)
  const int q = (which == 0 || which == 4) ? wq(g.nx) : wq(g.ny);
  switch (q) {
    case 4: launch_q<4>(which, g, m, Ms, X, Y, H, twx, twy, st); break;
    case 8: launch_q<8>(which, g, m, Ms, X, Y, H, twx, twy, st); break;
    case 16: launch_q<16>(which, g, m, Ms, X, Y, H, twx, twy, st); break;
    default: launch_q<32>(which, g, m, Ms, X, Y, H, twx, twy, st); break;
  }
}

void launch_wreg(int which, const DemagGeom& g, const double* m, const double* Ms, double2* X, double2* Y, double* H,
                 const double2* twx, const double2* twy, cudaStream_t st) {
  const int q = (which == 0 || which == 4) ? wq(g.nx) : wq(g.ny);
  if (q == 16) launch_q<16>(which, g, m, Ms, X, Y, H, twx, twy, st);
  else launch_q<32>(which, g, m, Ms, X, Y, H, twx, twy, st);
}

}  // namespace mm

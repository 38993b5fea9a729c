// mm_common.cuh -- shared types and helpers of libmmcuda (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>

namespace mm {

constexpr double kPi = 3.14159265358979323846;
constexpr double kMu0 = 4.0 * kPi * 1e-7;  // vacuum permeability (MicroMagnetic.jl src/const.jl:1)

// ---------------------------------------------------------------- complex ---
template <typename R> struct Cplx;
template <> struct Cplx<float> { using T = float2; };
template <> struct Cplx<double> { using T = double2; };
template <typename R> using cplx_t = typename Cplx<R>::T;

template <typename C> __host__ __device__ __forceinline__ C cmk(decltype(C::x) a, decltype(C::x) b) {
  C c; c.x = a; c.y = b; return c;
}
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return cmk<C>(a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return cmk<C>(a.x - b.x, a.y - b.y); }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  return cmk<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename C> __device__ __forceinline__ C cconj(C a) { return cmk<C>(a.x, -a.y); }

// ------------------------------------------- programmatic dependent launch --
// The kernels of an RK step follow one another on one stream, each reading
// what the previous one wrote.  Launched with the programmatic-serialisation
// attribute (launch_pdl), a kernel may be launched as the previous kernel's
// blocks exit, before that grid's completion has been processed; pdl_enter(),
// the first statement of every such kernel, waits until the previous grid has
// completed and its writes are visible.  A grid is therefore complete only
// after its predecessor is.  (No block triggers its dependents early: blocks
// of the next kernel made resident during a pass's last wave, waiting there,
// made every multi-wave workload slower.)  Kernels without pdl_enter() are
// launched the ordinary way; in one launched without the attribute the wait
// returns at once.
__device__ __forceinline__ void pdl_enter() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
// MMCUDA_PDL=0 launches every kernel the ordinary way (default: on).
bool pdl_enabled();
template <typename... KA, typename... A>
cudaError_t launch_pdl(void (*kern)(KA...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, A&&... args) {
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cfg.attrs = at;
  cfg.numAttrs = pdl_enabled() ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kern, static_cast<KA>(args)...);
}
template <typename C, typename R> __device__ __forceinline__ C cscale(C a, R s) { return cmk<C>(a.x * s, a.y * s); }
// multiply by (sgn * i): sgn = -1 for the forward transform, +1 for the inverse
template <bool INV, typename C> __device__ __forceinline__ C crot(C a) {
  return INV ? cmk<C>(-a.y, a.x) : cmk<C>(a.y, -a.x);
}

// ------------------------------------------------------------ FFT plans -----
constexpr int kMaxStages = 16;
// Radix sequence of a 1-D transform, 3 bits per stage (stage s in bits
// 3s..3s+2: 0=32 1=2 2=3 3=4 4=5 5=7 6=8 7=16), so that device code decodes
// it without an indexed array.
struct FftPlan1 {
  int L;                    // complex transform length (1 = identity)
  int nst;                  // number of radix stages
  int pow2;                 // L is a power of two
  unsigned long long code;  // radices
};
__host__ __device__ __forceinline__ int plan_radix(const FftPlan1& p, int s) {
  const int c = static_cast<int>((p.code >> (3 * s)) & 7ull);
  return c == 0 ? 32 : c == 1 ? 2 : c == 2 ? 3 : c == 3 ? 4 : c == 4 ? 5 : c == 5 ? 7 : c == 6 ? 8 : 16;
}

inline int radix_code(int r) {
  switch (r) {
    case 2: return 1;
    case 3: return 2;
    case 4: return 3;
    case 5: return 4;
    case 7: return 5;
    case 8: return 6;
    case 16: return 7;
    default: return 0;  // 32
  }
}

// Stage radices for a 7-smooth length.  The power-of-two factor is split into
// the fewest stages of radix <= max_pow2_radix with balanced exponents (2^11
// with 16 -> 16,16,8); the odd factor takes 7, 5, 3 (2000 with 16 -> 16,5,5,5).
inline bool make_fft_plan(int L, FftPlan1& p, int max_pow2_radix = 8) {
  p.L = L;
  p.nst = 0;
  p.code = 0;
  p.pow2 = (L & (L - 1)) == 0;
  auto push = [&](int r) {
    if (p.nst >= kMaxStages) return false;
    p.code |= static_cast<unsigned long long>(radix_code(r)) << (3 * p.nst);
    ++p.nst;
    return true;
  };
  if (L < 1) return false;
  int m = L, lg = 0;
  while (m % 2 == 0) {
    m /= 2;
    ++lg;
  }
  if (lg > 0) {
    int lmax = 0;
    while ((1 << lmax) < max_pow2_radix) ++lmax;
    const int ns = (lg + lmax - 1) / lmax;
    for (int s = 0; s < ns; ++s) {
      const int e = lg / ns + (s < lg % ns ? 1 : 0);
      if (!push(1 << e)) return false;
    }
  }
  while (m > 1) {
    int r = 0;
    if (m % 7 == 0) r = 7;
    else if (m % 5 == 0) r = 5;
    else if (m % 3 == 0) r = 3;
    else return false;
    if (!push(r)) return false;
    m /= r;
  }
  return true;
}

// Division by a run-time invariant d for 0 <= x < 2^31 with one multiply-high
// (Granlund & Montgomery, "Division by invariant integers using
// multiplication", PLDI 1994): q = (umulhi(x, m) + x) >> l.
struct FastDiv {
  unsigned d, m, l;
};
inline FastDiv make_fastdiv(unsigned d) {
  FastDiv f;
  f.d = d;
  f.l = 0;
  while ((1ull << f.l) < d) ++f.l;
  f.m = static_cast<unsigned>(((1ull << (32 + f.l)) / d) - (1ull << 32) + 1);
  return f;
}
__device__ __forceinline__ int fdiv(int x, const FastDiv f) {
  const unsigned t = __umulhi(static_cast<unsigned>(x), f.m);
  return static_cast<int>((t + static_cast<unsigned>(x)) >> f.l);
}

inline bool is_7smooth(int n) {
  if (n < 1) return false;
  for (int p : {2, 3, 5, 7})
    while (n % p == 0) n /= p;
  return n == 1;
}

// Padded FFT length for the zero-padded linear convolution of n cells: any
// P >= 2n-1 gives the same physical-cell result (the reference uses 2n, or
// 2n-1 for n <= 3, src/micro/demag.jl:41-44); the smallest 7-smooth length is
// used, even where the real-to-complex x transform needs it.
inline int padded_fft_len(int n, bool even) {
  if (n <= 1) return 1;
  int P = 2 * n - 1;
  while (!is_7smooth(P) || (even && (P % 2))) ++P;
  return P;
}

}  // namespace mm

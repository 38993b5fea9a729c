// mm_fft.cuh -- batched 1-D complex FFT of lines held in shared memory.
//
// Self-sorting (Stockham) decimation-in-time formulation: a stage of radix R
// over a span p (product of the radices already applied) maps butterfly i of
// a line of length L (L/R butterflies) as
//     v[r] = x[i + r*L/R] * exp(s*2*pi*i * r*(i mod p) / (p*R)),   r = 0..R-1
//     v    = DFT_R(v)
//     y[(i - i mod p)*R + (i mod p) + r*p] = v[r]
// and leaves the result in natural order after the last stage.  Stages
// ping-pong between two shared buffers, so a thread holds one butterfly at a
// time.  Power-of-two lengths take shift/mask index arithmetic.
//
// Twiddles come from a table tw[t] = exp(-2*pi*i*t / (L*tw_mul)) held in
// global memory (read through the read-only cache); tw_mul = 2 lets the
// half-length complex transform of a real x-line share the real-length table.
#pragma once
#include "mm_common.cuh"

namespace mm {

// cos/sin of 2*pi*k/n for the odd-prime and radix-16 butterflies (mathematical constants)
constexpr double kS3 = 0.86602540378443864676;  // sin(2pi/3)
constexpr double kC51 = 0.30901699437494742410, kS51 = 0.95105651629515357212;
constexpr double kC52 = -0.80901699437494742410, kS52 = 0.58778525229247312917;
constexpr double kC71 = 0.62348980185873353053, kS71 = 0.78183148246802980871;
constexpr double kC72 = -0.22252093395631440429, kS72 = 0.97492791218182360702;
constexpr double kC73 = -0.90096886790241912624, kS73 = 0.43388373911755812048;
constexpr double kR2 = 0.70710678118654752440;   // cos(pi/4)
constexpr double kC16 = 0.92387953251128675613;  // cos(pi/8)
constexpr double kS16 = 0.38268343236508977173;  // sin(pi/8)

template <bool INV, typename C> __device__ __forceinline__ void dft2(C* v) {
  C a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

template <bool INV, typename C> __device__ __forceinline__ void dft4(C* v) {
  C a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
  C c = cadd(v[1], v[3]), d = crot<INV>(csub(v[1], v[3]));
  v[0] = cadd(a, c);
  v[2] = csub(a, c);
  v[1] = cadd(b, d);
  v[3] = csub(b, d);
}

template <bool INV, typename C> __device__ __forceinline__ void dft8(C* v) {
  using R = decltype(C::x);
  C e[4] = {v[0], v[2], v[4], v[6]};
  C o[4] = {v[1], v[3], v[5], v[7]};
  dft4<INV>(e);
  dft4<INV>(o);
  const R h = static_cast<R>(kR2);
  // w8^1 = h(1 + s i), w8^2 = s i, w8^3 = h(-1 + s i), s = -1 forward
  C o1 = cmul(o[1], INV ? cmk<C>(h, h) : cmk<C>(h, -h));
  C o2 = crot<INV>(o[2]);
  C o3 = cmul(o[3], INV ? cmk<C>(-h, h) : cmk<C>(-h, -h));
  v[0] = cadd(e[0], o[0]);
  v[4] = csub(e[0], o[0]);
  v[1] = cadd(e[1], o1);
  v[5] = csub(e[1], o1);
  v[2] = cadd(e[2], o2);
  v[6] = csub(e[2], o2);
  v[3] = cadd(e[3], o3);
  v[7] = csub(e[3], o3);
}

// 16 = 4 x 4: DFT4 over the four residues mod 4, twiddles w16^(r*k1), DFT4 over r
template <bool INV, typename C> __device__ __forceinline__ void dft16(C* v) {
  using R = decltype(C::x);
  C a[4][4];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    a[r][0] = v[r];
    a[r][1] = v[r + 4];
    a[r][2] = v[r + 8];
    a[r][3] = v[r + 12];
    dft4<INV>(a[r]);
  }
  const R s = INV ? R(1) : R(-1);
  const R c1 = static_cast<R>(kC16), s1 = static_cast<R>(kS16), h = static_cast<R>(kR2);
  // w16^1, w16^2, w16^3, w16^4 = s i, w16^6 = h(-1 + s i), w16^9 = -w16^1
  const C w1 = cmk<C>(c1, s * s1), w2 = cmk<C>(h, s * h), w3 = cmk<C>(s1, s * c1);
  a[1][1] = cmul(a[1][1], w1);
  a[1][2] = cmul(a[1][2], w2);
  a[1][3] = cmul(a[1][3], w3);
  a[2][1] = cmul(a[2][1], w2);
  a[2][2] = crot<INV>(a[2][2]);
  a[2][3] = cmul(a[2][3], cmk<C>(-h, s * h));
  a[3][1] = cmul(a[3][1], w3);
  a[3][2] = cmul(a[3][2], cmk<C>(-h, s * h));
  a[3][3] = cmul(a[3][3], cmk<C>(-c1, -s * s1));
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1) {
    C t[4] = {a[0][k1], a[1][k1], a[2][k1], a[3][k1]};
    dft4<INV>(t);
    v[k1] = t[0];
    v[k1 + 4] = t[1];
    v[k1 + 8] = t[2];
    v[k1 + 12] = t[3];
  }
}

// cos, sin of 2*pi*k/32, k = 0..15 (mathematical constants).  A constexpr
// function rather than a __constant__ table: the butterflies read it at
// indices fixed by loop unrolling, which then fold into immediate operands
// of the right precision instead of constant-bank loads of doubles.
__host__ __device__ constexpr double w32_cs(int k, int sin_part) {
  constexpr double t[16][2] = {
      {1.00000000000000000000, 0.00000000000000000000},
      {0.98078528040323044913, 0.19509032201612826785},
      {0.92387953251128675613, 0.38268343236508977173},
      {0.83146961230254523708, 0.55557023301960222474},
      {0.70710678118654752440, 0.70710678118654752440},
      {0.55557023301960222474, 0.83146961230254523708},
      {0.38268343236508977173, 0.92387953251128675613},
      {0.19509032201612826785, 0.98078528040323044913},
      {0.00000000000000000000, 1.00000000000000000000},
      {-0.19509032201612826785, 0.98078528040323044913},
      {-0.38268343236508977173, 0.92387953251128675613},
      {-0.55557023301960222474, 0.83146961230254523708},
      {-0.70710678118654752440, 0.70710678118654752440},
      {-0.83146961230254523708, 0.55557023301960222474},
      {-0.92387953251128675613, 0.38268343236508977173},
      {-0.98078528040323044913, 0.19509032201612826785},
  };
  return t[k][sin_part];
}

// 32 = 2 x 16: DFT16 of the even and odd samples, twiddles w32^k
template <bool INV, typename C> __device__ __forceinline__ void dft32(C* v) {
  using R = decltype(C::x);
  C e[16], o[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    e[i] = v[2 * i];
    o[i] = v[2 * i + 1];
  }
  dft16<INV>(e);
  dft16<INV>(o);
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    const R c = static_cast<R>(w32_cs(k, 0)), sn = static_cast<R>(w32_cs(k, 1));
    const C t = cmul(o[k], cmk<C>(c, INV ? sn : -sn));
    v[k] = cadd(e[k], t);
    v[k + 16] = csub(e[k], t);
  }
}

template <bool INV, typename C> __device__ __forceinline__ void dft3(C* v) {
  using R = decltype(C::x);
  C t = cadd(v[1], v[2]);
  C u = csub(v[0], cscale(t, static_cast<R>(0.5)));
  C w = crot<INV>(cscale(csub(v[1], v[2]), static_cast<R>(kS3)));
  v[0] = cadd(v[0], t);
  v[1] = cadd(u, w);
  v[2] = csub(u, w);
}

template <bool INV, typename C> __device__ __forceinline__ void dft5(C* v) {
  using R = decltype(C::x);
  C t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
  C t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
  C x0 = v[0];
  C a1 = cadd(x0, cadd(cscale(t1, static_cast<R>(kC51)), cscale(t2, static_cast<R>(kC52))));
  C a2 = cadd(x0, cadd(cscale(t1, static_cast<R>(kC52)), cscale(t2, static_cast<R>(kC51))));
  C b1 = crot<INV>(cadd(cscale(t3, static_cast<R>(kS51)), cscale(t4, static_cast<R>(kS52))));
  C b2 = crot<INV>(csub(cscale(t3, static_cast<R>(kS52)), cscale(t4, static_cast<R>(kS51))));
  v[0] = cadd(x0, cadd(t1, t2));
  v[1] = cadd(a1, b1);
  v[4] = csub(a1, b1);
  v[2] = cadd(a2, b2);
  v[3] = csub(a2, b2);
}

template <bool INV, typename C> __device__ __forceinline__ void dft7(C* v) {
  using R = decltype(C::x);
  C p1 = cadd(v[1], v[6]), p2 = cadd(v[2], v[5]), p3 = cadd(v[3], v[4]);
  C q1 = csub(v[1], v[6]), q2 = csub(v[2], v[5]), q3 = csub(v[3], v[4]);
  C x0 = v[0];
  const R c1 = static_cast<R>(kC71), c2 = static_cast<R>(kC72), c3 = static_cast<R>(kC73);
  const R s1 = static_cast<R>(kS71), s2 = static_cast<R>(kS72), s3 = static_cast<R>(kS73);
  // a_j = x0 + sum_k cos(2 pi jk/7) p_k ; b_j = sum_k sin(2 pi jk/7) q_k
  C a1 = cadd(x0, cadd(cscale(p1, c1), cadd(cscale(p2, c2), cscale(p3, c3))));
  C a2 = cadd(x0, cadd(cscale(p1, c2), cadd(cscale(p2, c3), cscale(p3, c1))));
  C a3 = cadd(x0, cadd(cscale(p1, c3), cadd(cscale(p2, c1), cscale(p3, c2))));
  C b1 = crot<INV>(cadd(cscale(q1, s1), cadd(cscale(q2, s2), cscale(q3, s3))));
  C b2 = crot<INV>(csub(cscale(q1, s2), cadd(cscale(q2, s3), cscale(q3, s1))));
  C b3 = crot<INV>(cadd(cscale(q1, s3), csub(cscale(q3, s2), cscale(q2, s1))));
  v[0] = cadd(x0, cadd(p1, cadd(p2, p3)));
  v[1] = cadd(a1, b1);
  v[6] = csub(a1, b1);
  v[2] = cadd(a2, b2);
  v[5] = csub(a2, b2);
  v[3] = cadd(a3, b3);
  v[4] = csub(a3, b3);
}

template <int R, bool INV, typename C> __device__ __forceinline__ void dftR(C* v) {
  if constexpr (R == 2) dft2<INV>(v);
  else if constexpr (R == 3) dft3<INV>(v);
  else if constexpr (R == 4) dft4<INV>(v);
  else if constexpr (R == 5) dft5<INV>(v);
  else if constexpr (R == 7) dft7<INV>(v);
  else if constexpr (R == 8) dft8<INV>(v);
  else if constexpr (R == 16) dft16<INV>(v);
  else dft32<INV>(v);
}

template <int R, bool INV, bool POW2, int NT, typename C>
__device__ __forceinline__ void fft_stage(const C* __restrict__ src, C* __restrict__ dst, int L, int LS, int nlines,
                                          int p, const C* __restrict__ tw, int tw_mul) {
  const int T = L / R;
  const int total = nlines * T;
  const int twstep = (L / (p * R)) * tw_mul;
  const int lgT = POW2 ? __ffs(T) - 1 : 0;
  for (int idx = threadIdx.x; idx < total; idx += NT) {
    int line, i, k;
    if (POW2) {
      line = idx >> lgT;
      i = idx & (T - 1);
      k = i & (p - 1);
    } else {
      line = idx / T;
      i = idx - line * T;
      k = i % p;
    }
    C v[R];
    const C* s = src + line * LS + i;
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = s[r * T];
    if (p > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        C w = __ldg(tw + r * k * twstep);
        if (INV) w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
    }
    dftR<R, INV>(v);
    C* d = dst + line * LS + (i - k) * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) d[r * p] = v[r];
  }
  __syncthreads();
}

template <bool INV, bool POW2, int NT, typename C>
__device__ __forceinline__ C* fft_lines_impl(C* a, C* b, int LS, int nlines, const FftPlan1 pl,
                                             const C* __restrict__ tw, int tw_mul) {
  int p = 1;
  const int L = pl.L;
  for (int s = 0; s < pl.nst; ++s) {
    const int R = plan_radix(pl, s);
    switch (R) {
      case 32:
        if constexpr (sizeof(decltype(C::x)) == 4) fft_stage<32, INV, POW2, NT>(a, b, L, LS, nlines, p, tw, tw_mul);
        break;
      case 16:
        if constexpr (sizeof(decltype(C::x)) == 4) fft_stage<16, INV, POW2, NT>(a, b, L, LS, nlines, p, tw, tw_mul);
        break;
      case 8: fft_stage<8, INV, POW2, NT>(a, b, L, LS, nlines, p, tw, tw_mul); break;
      case 7: fft_stage<7, INV, false, NT>(a, b, L, LS, nlines, p, tw, tw_mul); break;
      case 5: fft_stage<5, INV, false, NT>(a, b, L, LS, nlines, p, tw, tw_mul); break;
      case 4: fft_stage<4, INV, POW2, NT>(a, b, L, LS, nlines, p, tw, tw_mul); break;
      case 3: fft_stage<3, INV, false, NT>(a, b, L, LS, nlines, p, tw, tw_mul); break;
      default: fft_stage<2, INV, POW2, NT>(a, b, L, LS, nlines, p, tw, tw_mul); break;
    }
    C* t = a;
    a = b;
    b = t;
    p *= R;
  }
  return a;
}

// Transforms nlines lines of length pl.L stored at a[line*LS + t], using b as
// the second buffer of the ping-pong; returns the buffer holding the result
// (a or b).  Must be called by every thread of the block.
template <bool INV, int NT, typename C>
__device__ C* fft_lines(C* a, C* b, int LS, int nlines, const FftPlan1 pl, const C* __restrict__ tw, int tw_mul) {
  if (pl.pow2) return fft_lines_impl<INV, true, NT>(a, b, LS, nlines, pl, tw, tw_mul);
  return fft_lines_impl<INV, false, NT>(a, b, LS, nlines, pl, tw, tw_mul);
}

}  // namespace mm

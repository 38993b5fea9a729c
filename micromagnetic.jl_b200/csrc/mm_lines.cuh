// mm_lines.cuh -- strided line transforms with the first stage reading HBM and
// the last stage writing HBM directly (internal).
//
// A block transforms `nlines` lines that run across memory rows (y or z
// lines of the spectra X / Y); line index = component * W + w, with w the
// column (kx) inside a W-wide tile.  Butterfly work is mapped with the line
// index fastest, so
//   * a warp's global accesses for one butterfly element touch W consecutive
//     kx of one row (W-wide coalesced segments), and
//   * a warp's shared accesses touch consecutive lines at the same position,
//     lines LS apart with LS odd: conflict-free.
// The first stage reads its operands straight from the source rows (rows past
// the physical extent are zero and are not read), the last stage writes its
// results straight to the destination rows (rows past the kept extent are not
// written); the stages between ping-pong through shared memory.
#pragma once
#include "mm_fft.cuh"

namespace mm {

// Lines in shared memory, element (line, pos) at line * LS + pos.  PAD
// inserts one slot after every 16 elements (pos + pos / 16; LS >= padded
// length): with few lines per block (the three components of one film
// column), a warp spans consecutive butterflies of one line, whose Stockham
// stores at stride R would otherwise fall into the same banks.
template <typename C, bool PAD = false>
struct SmemLines {
  C* b;
  int LS;
  __device__ __forceinline__ int at(int line, int pos) const { return line * LS + (PAD ? pos + (pos >> 4) : pos); }
  __device__ __forceinline__ C load(int line, int pos) const { return b[at(line, pos)]; }
  __device__ __forceinline__ void store(int line, int pos, C v) const { b[at(line, pos)] = v; }
};
// line stride of PAD lines of length L
__host__ __device__ __forceinline__ int padded_line_stride(int L) { return (L + (L >> 4)) | 1; }

// rows of a spectrum array: element (line, pos) at
// base[comp * comp_stride + pos * row_stride + kx0 + w], comp = line >> lgW.
// IX is the offset type: int where every offset of the array fits in 31 bits
// (the launchers check), which keeps the per-element address arithmetic in
// 32-bit integer instructions.
template <typename C, typename IX = int64_t>
struct RowsIn {
  const C* base;
  IX comp_stride, row_stride;
  int lgW, kx0, Hx, nrows;  // pos >= nrows reads as zero
  __device__ __forceinline__ C load(int line, int pos) const {
    const int w = line & ((1 << lgW) - 1), comp = line >> lgW;
    const int kx = kx0 + w;
    if (pos >= nrows || kx >= Hx) return cmk<C>(0, 0);
    return base[static_cast<IX>(comp) * comp_stride + static_cast<IX>(pos) * row_stride + kx];
  }
};

template <typename C, typename IX = int64_t>
struct RowsOut {
  C* base;
  IX comp_stride, row_stride;
  int lgW, kx0, Hx, nrows;  // pos >= nrows is not written
  __device__ __forceinline__ void store(int line, int pos, C v) const {
    const int w = line & ((1 << lgW) - 1), comp = line >> lgW;
    const int kx = kx0 + w;
    if (pos >= nrows || kx >= Hx) return;
    base[static_cast<IX>(comp) * comp_stride + static_cast<IX>(pos) * row_stride + kx] = v;
  }
};

// rows of a spectrum array with a run-time step between the W entries of a
// row: element (line, pos) at base[comp * comp_stride + pos * row_stride +
// (t0 + w) * wstride], t0 + w < tn (the fused z kernel's tiles along kx, or
// along ky of one kx column)
template <typename C, typename IX = int64_t>
struct RowsInW {
  const C* base;
  IX comp_stride, row_stride, wstride;
  int lgW, t0, tn, nrows;  // pos >= nrows reads as zero
  __device__ __forceinline__ C load(int line, int pos) const {
    const int w = line & ((1 << lgW) - 1), comp = line >> lgW;
    const int t = t0 + w;
    if (pos >= nrows || t >= tn) return cmk<C>(0, 0);
    return base[static_cast<IX>(comp) * comp_stride + static_cast<IX>(pos) * row_stride + static_cast<IX>(t) * wstride];
  }
};

template <typename C, typename IX = int64_t>
struct RowsOutW {
  C* base;
  IX comp_stride, row_stride, wstride;
  int lgW, t0, tn, nrows;  // pos >= nrows is not written
  __device__ __forceinline__ void store(int line, int pos, C v) const {
    const int w = line & ((1 << lgW) - 1), comp = line >> lgW;
    const int t = t0 + w;
    if (pos >= nrows || t >= tn) return;
    base[static_cast<IX>(comp) * comp_stride + static_cast<IX>(pos) * row_stride + static_cast<IX>(t) * wstride] = v;
  }
};

// columns of a column-major spectrum (films): element (line, pos) at
// base[(comp * Hx + kx) * ld + pos], kx = kx0 + w, comp = line >> lgW.
template <typename C, typename IX = int64_t>
struct ColsIn {
  const C* base;
  int ld, lgW, kx0, Hx, nrows;  // pos >= nrows reads as zero
  __device__ __forceinline__ C load(int line, int pos) const {
    const int w = line & ((1 << lgW) - 1), comp = line >> lgW;
    const int kx = kx0 + w;
    if (pos >= nrows || kx >= Hx) return cmk<C>(0, 0);
    return base[(static_cast<IX>(comp) * Hx + kx) * ld + pos];
  }
};

template <typename C, typename IX = int64_t>
struct ColsOut {
  C* base;
  int ld, lgW, kx0, Hx, nrows;  // pos >= nrows is not written
  __device__ __forceinline__ void store(int line, int pos, C v) const {
    const int w = line & ((1 << lgW) - 1), comp = line >> lgW;
    const int kx = kx0 + w;
    if (pos >= nrows || kx >= Hx) return;
    base[(static_cast<IX>(comp) * Hx + kx) * ld + pos] = v;
  }
};

template <int R, bool INV, bool POW2, int NT, class SRC, class DST, typename C>
__device__ __forceinline__ void lstage(const SRC& src, const DST& dst, int L, int nlines, const FastDiv fnl, int p,
                                       const C* __restrict__ tw, int tw_mul) {
  const int T = L / R;
  const int total = nlines * T;
  const int twstep = (L / (p * R)) * tw_mul;
  for (int idx = threadIdx.x; idx < total; idx += NT) {
    const int i = fdiv(idx, fnl);
    const int line = idx - i * nlines;
    const int k = POW2 ? (i & (p - 1)) : (i % p);
    C v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src.load(line, i + r * T);
    if (p > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        C w = __ldg(tw + r * k * twstep);
        if (INV) w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
    }
    dftR<R, INV>(v);
    const int o = (i - k) * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) dst.store(line, o + r * p, v[r]);
  }
  __syncthreads();
}

template <bool INV, bool POW2, int NT, class SRC, class DST, typename C>
__device__ __forceinline__ void lstage_any(int R, const SRC& src, const DST& dst, int L, int nlines, const FastDiv fnl,
                                           int p, const C* __restrict__ tw, int tw_mul) {
  switch (R) {
    case 32:
      if constexpr (sizeof(decltype(C::x)) == 4) lstage<32, INV, POW2, NT>(src, dst, L, nlines, fnl, p, tw, tw_mul);
      break;
    case 16:
      if constexpr (sizeof(decltype(C::x)) == 4) lstage<16, INV, POW2, NT>(src, dst, L, nlines, fnl, p, tw, tw_mul);
      break;
    case 8: lstage<8, INV, POW2, NT>(src, dst, L, nlines, fnl, p, tw, tw_mul); break;
    case 7: lstage<7, INV, false, NT>(src, dst, L, nlines, fnl, p, tw, tw_mul); break;
    case 5: lstage<5, INV, false, NT>(src, dst, L, nlines, fnl, p, tw, tw_mul); break;
    case 4: lstage<4, INV, POW2, NT>(src, dst, L, nlines, fnl, p, tw, tw_mul); break;
    case 3: lstage<3, INV, false, NT>(src, dst, L, nlines, fnl, p, tw, tw_mul); break;
    default: lstage<2, INV, POW2, NT>(src, dst, L, nlines, fnl, p, tw, tw_mul); break;
  }
}

// All stages of pl: src -> (shared ping-pong a, b) -> dst.  Identity copy for L == 1.
template <bool INV, bool POW2, int NT, bool PAD, class SRC, class DST, typename C>
__device__ __forceinline__ void line_fft_impl(const SRC& src, const DST& dst, C* a, C* b, int LS, int nlines,
                                              const FastDiv fnl, const FftPlan1 pl, const C* __restrict__ tw,
                                              int tw_mul) {
  const int L = pl.L;
  if (pl.nst == 0) {
    for (int line = threadIdx.x; line < nlines; line += NT) dst.store(line, 0, src.load(line, 0));
    __syncthreads();
    return;
  }
  if (pl.nst == 1) {
    lstage_any<INV, POW2, NT>(plan_radix(pl, 0), src, dst, L, nlines, fnl, 1, tw, tw_mul);
    return;
  }
  SmemLines<C, PAD> A{a, LS}, B{b, LS};
  int p = 1;
  int R = plan_radix(pl, 0);
  lstage_any<INV, POW2, NT>(R, src, A, L, nlines, fnl, p, tw, tw_mul);
  p *= R;
  for (int s = 1; s + 1 < pl.nst; ++s) {
    R = plan_radix(pl, s);
    lstage_any<INV, POW2, NT>(R, A, B, L, nlines, fnl, p, tw, tw_mul);
    p *= R;
    const SmemLines<C, PAD> t = A;
    A = B;
    B = t;
  }
  R = plan_radix(pl, pl.nst - 1);
  lstage_any<INV, POW2, NT>(R, A, dst, L, nlines, fnl, p, tw, tw_mul);
}

template <bool INV, int NT, bool PAD = false, class SRC, class DST, typename C>
__device__ void line_fft(const SRC& src, const DST& dst, C* a, C* b, int LS, int nlines, const FastDiv fnl,
                         const FftPlan1 pl, const C* __restrict__ tw, int tw_mul) {
  if (pl.pow2) line_fft_impl<INV, true, NT, PAD>(src, dst, a, b, LS, nlines, fnl, pl, tw, tw_mul);
  else line_fft_impl<INV, false, NT, PAD>(src, dst, a, b, LS, nlines, fnl, pl, tw, tw_mul);
}

// All stages of pl from src into shared memory (a and b ping-pong); returns
// the buffer that holds the result.
template <bool INV, bool POW2, int NT, bool PAD, class SRC, typename C>
__device__ __forceinline__ C* line_fft_to_smem_impl(const SRC& src, C* a, C* b, int LS, int nlines,
                                                    const FastDiv fnl, const FftPlan1 pl, const C* __restrict__ tw,
                                                    int tw_mul) {
  const int L = pl.L;
  SmemLines<C, PAD> A{a, LS}, B{b, LS};
  if (pl.nst == 0) {
    for (int line = threadIdx.x; line < nlines; line += NT) A.store(line, 0, src.load(line, 0));
    __syncthreads();
    return a;
  }
  int p = 1;
  int R = plan_radix(pl, 0);
  lstage_any<INV, POW2, NT>(R, src, A, L, nlines, fnl, p, tw, tw_mul);
  p *= R;
  for (int s = 1; s < pl.nst; ++s) {
    R = plan_radix(pl, s);
    lstage_any<INV, POW2, NT>(R, A, B, L, nlines, fnl, p, tw, tw_mul);
    p *= R;
    const SmemLines<C, PAD> t = A;
    A = B;
    B = t;
  }
  return A.b;
}

// All stages of pl from shared buffer x (y is free) into dst.
template <bool INV, bool POW2, int NT, bool PAD, class DST, typename C>
__device__ __forceinline__ void line_fft_from_smem_impl(C* x, C* y, const DST& dst, int LS, int nlines,
                                                        const FastDiv fnl, const FftPlan1 pl,
                                                        const C* __restrict__ tw, int tw_mul) {
  const int L = pl.L;
  SmemLines<C, PAD> A{x, LS}, B{y, LS};
  if (pl.nst == 0) {
    for (int line = threadIdx.x; line < nlines; line += NT) dst.store(line, 0, A.load(line, 0));
    __syncthreads();
    return;
  }
  int p = 1;
  for (int s = 0; s + 1 < pl.nst; ++s) {
    const int R = plan_radix(pl, s);
    lstage_any<INV, POW2, NT>(R, A, B, L, nlines, fnl, p, tw, tw_mul);
    p *= R;
    const SmemLines<C, PAD> t = A;
    A = B;
    B = t;
  }
  lstage_any<INV, POW2, NT>(plan_radix(pl, pl.nst - 1), A, dst, L, nlines, fnl, p, tw, tw_mul);
}

template <bool INV, int NT, bool PAD = false, class SRC, typename C>
__device__ C* line_fft_to_smem(const SRC& src, C* a, C* b, int LS, int nlines, const FastDiv fnl, const FftPlan1 pl,
                               const C* __restrict__ tw, int tw_mul) {
  if (pl.pow2) return line_fft_to_smem_impl<INV, true, NT, PAD>(src, a, b, LS, nlines, fnl, pl, tw, tw_mul);
  return line_fft_to_smem_impl<INV, false, NT, PAD>(src, a, b, LS, nlines, fnl, pl, tw, tw_mul);
}

template <bool INV, int NT, bool PAD = false, class DST, typename C>
__device__ void line_fft_from_smem(C* x, C* y, const DST& dst, int LS, int nlines, const FastDiv fnl,
                                   const FftPlan1 pl, const C* __restrict__ tw, int tw_mul) {
  if (pl.pow2) line_fft_from_smem_impl<INV, true, NT, PAD>(x, y, dst, LS, nlines, fnl, pl, tw, tw_mul);
  else line_fft_from_smem_impl<INV, false, NT, PAD>(x, y, dst, LS, nlines, fnl, pl, tw, tw_mul);
}

// Number of shared buffers line_fft needs for a plan (0 for one stage).
inline int line_fft_buffers(const FftPlan1& pl) { return pl.nst <= 1 ? 0 : (pl.nst == 2 ? 1 : 2); }

}  // namespace mm

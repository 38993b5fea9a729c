// mm_wfft.cuh -- register-resident FFT of lines of L = 32 Q points (Q = 4, 8,
// 16 or 32) by groups of Q lanes of one warp (32 / Q lines a warp), FP32 or
// FP64 (C = float2 or double2; internal).
//
// Four-step decomposition L = 32 x Q.  Lane q of a group holds the 32 values
// x[q + Q j], j < 32, in registers:
//   1. a 32-point DFT over j in registers          A[q][k1], k1 < 32
//   2. twiddles w_L^(q k1)                          (table, L entries)
//   3. a transpose through a shared tile private to the warp (__syncwarp only)
//   4. Q-point DFTs over q, 32 / Q of them a lane
// and leaves X[k1 + 32 k2] in lane q' of the group, register v[i Q + k2], for
// k1 = q' + Q i (i < 32 / Q), k2 < Q.  Unnormalised; INV conjugates the
// twiddles and the butterflies.  The twiddle table holds exp(-2 pi i t / (L
// TWS)), read at stride TWS (the tables of the padded length serve the
// half-length transforms).  The tile needs wtile_size<Q>() complex values a
// warp.
#pragma once
#include "mm_fft.cuh"

namespace mm {

// complex values of one warp's transpose tile: 32 / Q groups of 32 rows of Q + 1
template <int Q> constexpr int wtile_size() { return (32 / Q) * 32 * (Q + 1); }

// Element (group g, row k1, column q) of a warp's tile: each group's 32 rows
// of Q columns, rows padded to Q + 1 so that the column reads of step 4 do
// not hit one bank.
template <int Q>
__device__ __forceinline__ int wtile_at(int g, int k1, int q) {
  return g * (32 * (Q + 1)) + k1 * (Q + 1) + q;
}

template <int Q, bool INV, int TWS = 1, typename C>
__device__ __forceinline__ void wfft(C (&v)[32], C* __restrict__ tile, const C* __restrict__ tw) {
  const int lane = threadIdx.x & 31;
  const int g = lane / Q, q = lane % Q;
  dft32<INV>(v);
#pragma unroll
  for (int k1 = 1; k1 < 32; ++k1) {
    C w = __ldg(tw + TWS * q * k1);  // q k1 < 32 Q = L
    if (INV) w.y = -w.y;
    v[k1] = cmul(v[k1], w);
  }
  __syncwarp();
#pragma unroll
  for (int k1 = 0; k1 < 32; ++k1) tile[wtile_at<Q>(g, k1, q)] = v[k1];
  __syncwarp();
#pragma unroll
  for (int i = 0; i < 32 / Q; ++i) {
    C u[Q];
#pragma unroll
    for (int r = 0; r < Q; ++r) u[r] = tile[wtile_at<Q>(g, q + Q * i, r)];
    dftR<Q, INV>(u);
#pragma unroll
    for (int k2 = 0; k2 < Q; ++k2) v[i * Q + k2] = u[k2];
  }
  __syncwarp();
}

}  // namespace mm

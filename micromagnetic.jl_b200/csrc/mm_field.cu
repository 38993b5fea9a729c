// mm_field.cu -- fused effective field + LLG + integrator stage kernels.
#include <cmath>

#include "mm_cell.cuh"
#include "mm_field.cuh"
#include "mm_launch.cuh"

namespace mm {

int stage_blocks(int64_t N) { return static_cast<int>((N + kStageThreads - 1) / kStageThreads); }

// Stage kernels run one thread per cell on a 3-D grid: blocks of BX x BY
// cells of one z plane (BX*BY = 256, BY up to 8 so that the y neighbours of
// a block are mostly its own rows).
StageGrid stage_grid(int nx, int ny, int nz) {
  StageGrid g;
  int by = 1;
  while (by < 8 && by < ny) by *= 2;
  const int bx = kStageThreads / by;
  g.block = dim3(bx, by, 1);
  g.grid = dim3((nx + bx - 1) / bx, (ny + by - 1) / by, nz);
  g.nblocks = static_cast<int>(g.grid.x * g.grid.y * g.grid.z);
  return g;
}

// --------------------------------------------------------------- masks ---
template <typename R>
__global__ void k_nbmask(int nx, int ny, int nz, int pbc, const R* __restrict__ Ms, uint8_t* __restrict__ nbm) {
  const int64_t N = static_cast<int64_t>(nx) * ny * nz;
  const int64_t I = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (I >= N) return;
  const int64_t nxy = static_cast<int64_t>(nx) * ny;
  const int i = static_cast<int>(I % nx), j = static_cast<int>((I / nx) % ny), k = static_cast<int>(I / nxy);
  const bool px = pbc & 1, py = pbc & 2, pz = pbc & 4;
  int64_t nb[6];
  nb[0] = i > 0 ? I - 1 : (px ? I + nx - 1 : -1);
  nb[1] = i < nx - 1 ? I + 1 : (px ? I - (nx - 1) : -1);
  nb[2] = j > 0 ? I - nx : (py ? I + static_cast<int64_t>(ny - 1) * nx : -1);
  nb[3] = j < ny - 1 ? I + nx : (py ? I - static_cast<int64_t>(ny - 1) * nx : -1);
  nb[4] = k > 0 ? I - nxy : (pz ? I + (nz - 1) * nxy : -1);
  nb[5] = k < nz - 1 ? I + nxy : (pz ? I - (nz - 1) * nxy : -1);
  uint8_t b = 0;
#pragma unroll
  for (int d = 0; d < 6; ++d)
    if (nb[d] >= 0 && Ms[nb[d]] > R(0)) b |= static_cast<uint8_t>(1u << d);
  nbm[I] = b;
}

template <typename R>
void launch_nbmask(int nx, int ny, int nz, int pbc, const R* Ms, uint8_t* nbm, cudaStream_t st) {
  const int64_t N = static_cast<int64_t>(nx) * ny * nz;
  k_nbmask<R><<<stage_blocks(N), kStageThreads, 0, st>>>(nx, ny, nz, pbc, Ms, nbm);
}

// Butcher tables of the adaptive methods (src/integrator/adaptive_rk_steps.jl:
// bs23 11-47, dopri54 49-107, cashkarp54 110-168, fehlberg54 171-229), laid
// out as RkTableau: rows a[s-1] give the input of stage s+1; row sol-1 is the
// solution; w are the error weights.
#define MM_RK_TABLES                                                                                          \
  {                                                                                                           \
    {7, 6, 7, 0, 5, 4,                                                                                        \
     {{1.0 / 5},                                                                                              \
      {3.0 / 40, 9.0 / 40},                                                                                   \
      {44.0 / 45, -56.0 / 15, 32.0 / 9},                                                                      \
      {19372.0 / 6561, -25360.0 / 2187, 64448.0 / 6561, -212.0 / 729},                                        \
      {9017.0 / 3168, -355.0 / 33, 46732.0 / 5247, 49.0 / 176, -5103.0 / 18656},                              \
      {35.0 / 384, 0, 500.0 / 1113, 125.0 / 192, -2187.0 / 6784, 11.0 / 84}},                                 \
     {71.0 / 57600, 0, -71.0 / 16695, 71.0 / 1920, -17253.0 / 339200, 22.0 / 525, -1.0 / 40}},               \
    {4, 3, 4, 1, 3, 2,                                                                                        \
     {{0.5}, {0, 0.75}, {2.0 / 9, 1.0 / 3, 4.0 / 9}},                                                         \
     {-5.0 / 72, 1.0 / 12, 1.0 / 9, -1.0 / 8}},                                                               \
    {6, 6, 6, 0, 5, 4,                                                                                        \
     {{1.0 / 5},                                                                                              \
      {3.0 / 40, 9.0 / 40},                                                                                   \
      {3.0 / 10, -9.0 / 10, 6.0 / 5},                                                                         \
      {-11.0 / 54, 5.0 / 2, -70.0 / 27, 35.0 / 27},                                                           \
      {1631.0 / 55296, 175.0 / 512, 575.0 / 13824, 44275.0 / 110592, 253.0 / 4096},                           \
      {37.0 / 378, 0, 250.0 / 621, 125.0 / 594, 0, 512.0 / 1771}},                                            \
     {-277.0 / 64512, 0, 6925.0 / 370944, -6925.0 / 202752, -277.0 / 14336, 277.0 / 7084}},                  \
    {6, 6, 6, 0, 5, 4,                                                                                        \
     {{1.0 / 4},                                                                                              \
      {3.0 / 32, 9.0 / 32},                                                                                   \
      {1932.0 / 2197, -7200.0 / 2197, 7296.0 / 2197},                                                         \
      {439.0 / 216, -8.0, 3680.0 / 513, -845.0 / 4104},                                                       \
      {-8.0 / 27, 2.0, -3544.0 / 2565, 1859.0 / 4104, -11.0 / 40},                                            \
      {16.0 / 135, 0, 6656.0 / 12825, 28561.0 / 56430, -9.0 / 50, 2.0 / 55}},                                 \
     {-1.0 / 360, 0, 128.0 / 4275, 2197.0 / 75240, -1.0 / 50, -2.0 / 55}},                                    \
  }

__constant__ RkTableau c_rk[RK_NMETHODS] = MM_RK_TABLES;
static const RkTableau h_rk[RK_NMETHODS] = MM_RK_TABLES;
const RkTableau& rk_tableau(int method) { return h_rk[method]; }

template <typename R, int MODE, bool EXTRA>
__global__ void __launch_bounds__(kStageThreads, sizeof(R) == 4 ? 3 : 2) k_stage(FieldArgs<R> a, const R* __restrict__ y, StageArgs<R> s) {
  constexpr bool kF32 = sizeof(R) == 4;
  pdl_enter();
  if (MODE == SM_DOPRI && !s.ctrl->active) return;
  const int64_t N = a.N;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  const bool live = i < a.nx && j < a.ny;
  const int I = (k * a.ny + j) * a.nx + i;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int blin = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
  double e[kNTerms];
  R m[3], h[3];
  double red = 0.0;  // SM_DOPRI stage 7: error max
  // RK4 operands of this cell, loaded together with the field inputs
  R mN[3], mL[3], av[3];
  if (MODE == SM_RK4 && live) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      mN[c] = s.m[c * N + I];
      mL[c] = kF32 ? s.m_lo[c * N + I] : R(0);
      av[c] = s.stage > 1 ? s.acc[c * N + I] : R(0);
    }
  }
  // FSAL: stage 1 takes k1 from the last stage of the accepted attempt
  const bool reuse = MODE == SM_DOPRI && s.stage == 1 && !s.ctrl->eval1;
  if (live) {
    if (!reuse) cell_heff<R, MODE == SM_ENERGY || MODE == SM_FIELD, EXTRA>(a, y, I, i, j, k, m, h, e);
    if (MODE == SM_FIELD) {
      s.out[I] = h[0];
      s.out[N + I] = h[1];
      s.out[2 * N + I] = h[2];
      if (s.ecell) {
        double et = 0.0;
#pragma unroll
        for (int t = 0; t < kNTerms; ++t) et += e[t];
        s.ecell[I] = static_cast<R>(et);
      }
    } else if (MODE == SM_RHS) {
      R f[3];
      llg_rhs(a, I, m, h, f);
      s.out[I] = f[0];
      s.out[N + I] = f[1];
      s.out[2 * N + I] = f[2];
    } else if (MODE == SM_RK4) {
      rk4_update(a, s, I, m, h, mN, mL, av);
    } else if (MODE == SM_DOPRI) {
      // rk_step_bs23! / rk_step_dopri54! / rk_step_cashkarp54! /
      // rk_step_fehlberg54!  src/integrator/adaptive_rk_steps.jl:11-229
      const RkTableau& tb = c_rk[s.method];
      const int st = s.stage;
      R f[3];
      if (reuse) {
#pragma unroll
        for (int c = 0; c < 3; ++c) f[c] = s.k[tb.nstage - 1][c * N + I];
      } else {
        llg_rhs(a, I, m, h, f);
      }
      const double hstep = s.ctrl->step;
      if (st < tb.err || (tb.fsal && st == tb.nstage)) {
#pragma unroll
        for (int c = 0; c < 3; ++c) s.k[st - 1][c * N + I] = f[c];
      }
      R yabs[3];  // y_next of the error norm
      if (st <= tb.sol) {
        const double* arow = tb.a[st - 1];
        R v[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          if constexpr (kF32) {
            float sum = 0.f;
            for (int j = 0; j < st; ++j) {
              if (arow[j] == 0.0) continue;
              const float kj = j == st - 1 ? f[c] : s.k[j][c * N + I];
              sum += static_cast<float>(arow[j] * hstep) * kj;
            }
            v[c] = sum;
          } else {
            double acc = s.m[c * N + I];
            for (int j = 0; j < st; ++j) {
              if (arow[j] == 0.0) continue;
              const double kj = j == st - 1 ? f[c] : s.k[j][c * N + I];
              acc = acc + (arow[j] * hstep) * kj;
            }
            v[c] = static_cast<R>(acc);
          }
        }
        if (st < tb.sol) {
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            if constexpr (kF32) v[c] = s.m[c * N + I] + (s.m_lo[c * N + I] + v[c]);
            s.ynext[c * N + I] = v[c];
          }
        } else {
          // the solution is normalised before it is used (adaptive_rk_steps.jl:35,96,156,217)
          if constexpr (kF32) {
            float hi[3], lo[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              hi[c] = s.m[c * N + I];
              lo[c] = s.m_lo[c * N + I];
              df_add(hi[c], lo[c], v[c]);
            }
            df_normalise(hi, lo);
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              s.ynext[c * N + I] = hi[c];
              s.ynext_lo[c * N + I] = lo[c];
              yabs[c] = hi[c];
            }
          } else {
            plain_normalise(v);
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              s.ynext[c * N + I] = v[c];
              yabs[c] = v[c];
            }
          }
        }
      } else {
#pragma unroll
        for (int c = 0; c < 3; ++c) yabs[c] = m[c];
      }
      if (st == tb.err) {
        // error estimate: max |sum_j w_j k_j| / (1 + |y_next|)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          double et = 0.0;
          for (int j = 0; j < st; ++j) {
            if (tb.w[j] == 0.0) continue;
            const double kj = j == st - 1 ? double(f[c]) : double(s.k[j][c * N + I]);
            et += tb.w[j] * kj;
          }
          const double v = fabs(et / (1.0 + fabs(double(yabs[c]))));
          red = (v > red || isnan(v)) ? v : red;
        }
      }
    }
  }
  if (MODE == SM_ENERGY || (MODE == SM_DOPRI && s.stage == c_rk[s.method].err)) {
    // deterministic block reduction in FP64
    __shared__ double sh[kStageThreads / 32][kNTerms];
    const int lane = tid & 31, warp = tid >> 5;
    constexpr int W = MODE == SM_ENERGY ? kNTerms : 1;
    double v[W];
#pragma unroll
    for (int t = 0; t < W; ++t) v[t] = live ? (MODE == SM_ENERGY ? e[t] : red) : 0.0;
#pragma unroll
    for (int t = 0; t < W; ++t) {
      for (int o = 16; o > 0; o >>= 1) {
        const double u = __shfl_down_sync(0xffffffffu, v[t], o);
        if (MODE == SM_ENERGY) v[t] += u;
        else v[t] = (u > v[t] || isnan(u)) ? u : v[t];
      }
      if (lane == 0) sh[warp][t] = v[t];
    }
    __syncthreads();
    if (tid < W) {
      double acc = 0.0;
      for (int w = 0; w < kStageThreads / 32; ++w) {
        const double u = sh[w][tid];
        if (MODE == SM_ENERGY) acc += u;
        else acc = (u > acc || isnan(u)) ? u : acc;
      }
      s.partials[blin * W + tid] = acc;
    }
  }
}

// RK4 / Heun stage on halo tiles (handles without the further terms): a
// block of BX x BY threads walks kStageTileZ consecutive z planes of its
// BX x BY column, keeping the planes k-1, k, k+1 of the stage input as
// (BX+2) x (BY+2) tiles in shared memory (a rolling window of three; each
// plane is loaded once per block, with coalesced row segments), so the six
// neighbours of every cell come from shared memory.  Same arithmetic as
// k_stage.
constexpr int kStageTileZ = 8;

template <typename R>
struct StageTile {
  static constexpr int kNT = kStageThreads, kMinB = sizeof(R) == 4 ? 3 : 2;
  struct Args {
    FieldArgs<R> a;
    const R* y;
    StageArgs<R> s;
    int bx, by;  // the block's cells along x and y (bx * by = kNT)
    dim3 grid;
  };
  static __device__ __forceinline__ void body(const Args& args, uint3 blockIdx);
};

template <typename R>
__device__ __forceinline__ void StageTile<R>::body(const Args& args, uint3 blockIdx) {
  const FieldArgs<R>& a = args.a;
  const StageArgs<R>& s = args.s;
  const R* __restrict__ y = args.y;
  constexpr bool kF32 = sizeof(R) == 4;
  extern __shared__ __align__(16) unsigned char smraw[];
  R* T = reinterpret_cast<R*>(smraw);
  const int bx = args.bx, by = args.by, TX = bx + 2, TY = by + 2, TP = TX * TY;
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const int64_t N = a.N;
  const bool px = a.pbc & 1, py = a.pbc & 2, pz = a.pbc & 4;
  const int i0 = blockIdx.x * bx, j0 = blockIdx.y * by, k0 = blockIdx.z * kStageTileZ;
  const int k1 = min(nz, k0 + kStageTileZ);
  const int tid = threadIdx.x, tx = tid % bx, ty = tid / bx, nth = bx * by;
  const int i = i0 + tx, j = j0 + ty;
  const bool live = i < nx && j < ny;
  auto slot = [](int p) { return (p + 3) % 3; };
  // plane p (-1 <= p <= nz) of the stage input into its slot; cells outside
  // the mesh (and not wrapped by periodic boundaries) are zero
  auto load_plane = [&](int p) {
    R* dst = T + slot(p) * 3 * TP;
    int pk = p;
    if (pk < 0 || pk >= nz) pk = pz ? (pk < 0 ? pk + nz : pk - nz) : -1;
    for (int e = tid; e < TP; e += nth) {
      const int hy = e / TX, hx = e - hy * TX;
      int gi = i0 + hx - 1, gj = j0 + hy - 1;
      if (gi == -1 && px) gi = nx - 1;
      else if (gi == nx && px) gi = 0;
      if (gj == -1 && py) gj = ny - 1;
      else if (gj == ny && py) gj = 0;
      const bool ok = pk >= 0 && gi >= 0 && gi < nx && gj >= 0 && gj < ny;
      const int64_t g = ok ? (static_cast<int64_t>(pk) * ny + gj) * nx + gi : 0;
#pragma unroll
      for (int c = 0; c < 3; ++c) dst[c * TP + e] = ok ? y[c * N + g] : R(0);
    }
  };
  load_plane(k0 - 1);
  load_plane(k0);
  for (int k = k0; k < k1; ++k) {
    load_plane(k + 1);
    const int I = (k * ny + j) * nx + i;
    R mN[3], mL[3], av[3];
    if (live) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        mN[c] = s.m[c * N + I];
        mL[c] = kF32 ? s.m_lo[c * N + I] : R(0);
        av[c] = s.stage > 1 ? s.acc[c * N + I] : R(0);
      }
    }
    __syncthreads();
    if (live) {
      const int sk = slot(k) * 3 * TP;
      TileNb<R> tn{T + sk, TP, (ty + 1) * TX + tx + 1, TX, slot(k - 1) * 3 * TP - sk, slot(k + 1) * 3 * TP - sk};
      R m[3], h[3];
      cell_heff<R, false, false, true>(a, y, I, i, j, k, m, h, nullptr, tn);
      rk4_update(a, s, I, m, h, mN, mL, av);
    }
    __syncthreads();  // before plane k + 2 replaces plane k - 1
  }
}

// Halo-tiled RK4 / Heun stages only with MMCUDA_STAGETILE=1: measured slower
// than the one-plane-per-block kernel (c5 0.59 vs 0.38 ms, c2 0.16 vs 0.10 ms
// a stage) -- each block waits for every plane's tile before computing it.
static bool stage_tile_enabled() {
  static const bool on = [] {
    const char* e = getenv("MMCUDA_STAGETILE");
    return e && e[0] == '1';
  }();
  return on;
}

// The compiled term sets of the RK4 / Heun stage unless MMCUDA_STAGE_FIX=0
static bool stage_fix_enabled() {
  static const bool on = [] {
    const char* e = getenv("MMCUDA_STAGE_FIX");
    return !(e && e[0] == '0');
  }();
  return on;
}

template <typename R, unsigned FIX>
typename StagePlain<R, FIX>::Args fix_args(const typename StagePlain<R>::Args& a) {
  return {a.a, a.y, a.s, a.bx, a.by, a.grid};
}

template <typename R>
bool stage_descriptor_used(const FieldArgs<R>& fa) {
  return !((fa.mask & kExtraBits) || ((fa.mask & TB_DMI_BULK) && fa.x.bD[0]));
}

template <typename R>
void launch_stage(int mode, const FieldArgs<R>& fa, const R* y, const StageArgs<R>& sa, cudaStream_t st) {
  const StageGrid g = stage_grid(fa.nx, fa.ny, fa.nz);
  // handles without the extra terms run the kernel compiled without them
  if ((fa.mask & kExtraBits) || ((fa.mask & TB_DMI_BULK) && fa.x.bD[0])) {
    switch (mode) {
      case SM_FIELD: launch_pdl(k_stage<R, SM_FIELD, true>, g.grid, g.block, 0, st, fa, y, sa); break;
      case SM_RHS: launch_pdl(k_stage<R, SM_RHS, true>, g.grid, g.block, 0, st, fa, y, sa); break;
      case SM_RK4: launch_pdl(k_stage<R, SM_RK4, true>, g.grid, g.block, 0, st, fa, y, sa); break;
      case SM_ENERGY: launch_pdl(k_stage<R, SM_ENERGY, true>, g.grid, g.block, 0, st, fa, y, sa); break;
      default: launch_pdl(k_stage<R, SM_DOPRI, true>, g.grid, g.block, 0, st, fa, y, sa); break;
    }
    return;
  }
  const size_t tsm = 3 * 3 * static_cast<size_t>(g.block.x + 2) * (g.block.y + 2) * sizeof(R);
  if (mode == SM_RK4 && stage_tile_enabled() && tsm <= 48 * 1024) {
    const dim3 grid(g.grid.x, g.grid.y, (fa.nz + kStageTileZ - 1) / kStageTileZ);
    launch_k<StageTile<R>>(grid, tsm, st,
                           {fa, y, sa, static_cast<int>(g.block.x), static_cast<int>(g.block.y), dim3()});
    return;
  }
  if (mode == SM_RK4) {
    const typename StagePlain<R>::Args args{fa, y, sa, static_cast<int>(g.block.x), static_cast<int>(g.block.y), dim3()};
    // a compiled term set when the handle's terms are exactly one of them
    // with uniform parameters (MMCUDA_STAGE_FIX=0 keeps the general kernel)
    const bool uni = !fa.A && !fa.D && !fa.Ku && !fa.Hz && stage_fix_enabled();
    const unsigned fx = uni ? fa.mask : 0u;
    switch (fx) {
      case kFixExDemag: launch_k<StagePlain<R, kFixExDemag>>(g.grid, 0, st, fix_args<R, kFixExDemag>(args)); break;
      case kFixExDemagZee: launch_k<StagePlain<R, kFixExDemagZee>>(g.grid, 0, st, fix_args<R, kFixExDemagZee>(args)); break;
      case kFixExBulkAnisDemag:
        launch_k<StagePlain<R, kFixExBulkAnisDemag>>(g.grid, 0, st, fix_args<R, kFixExBulkAnisDemag>(args));
        break;
      case kFixExIntDemag: launch_k<StagePlain<R, kFixExIntDemag>>(g.grid, 0, st, fix_args<R, kFixExIntDemag>(args)); break;
      default: launch_k<StagePlain<R>>(g.grid, 0, st, args); break;
    }
    return;
  }
  switch (mode) {
    case SM_FIELD: launch_pdl(k_stage<R, SM_FIELD, false>, g.grid, g.block, 0, st, fa, y, sa); break;
    case SM_RHS: launch_pdl(k_stage<R, SM_RHS, false>, g.grid, g.block, 0, st, fa, y, sa); break;
    case SM_ENERGY: launch_pdl(k_stage<R, SM_ENERGY, false>, g.grid, g.block, 0, st, fa, y, sa); break;
    default: launch_pdl(k_stage<R, SM_DOPRI, false>, g.grid, g.block, 0, st, fa, y, sa); break;
  }
}

// --------------------------------------------------------- conversions ---
// host element type T: double, or float (the reference's Float32 mode)
template <typename R, typename T>
__global__ void k_aos_to_soa(const T* __restrict__ aos, R* __restrict__ hi, R* __restrict__ lo, int64_t N,
                             int* __restrict__ nanflag) {
  const int64_t I = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (I >= N) return;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double v = static_cast<double>(aos[3 * I + c]);
    if (nanflag && isnan(v)) *nanflag = 1;
    const R h = static_cast<R>(v);
    hi[c * N + I] = h;
    if (lo) lo[c * N + I] = static_cast<R>(v - static_cast<double>(h));
  }
}

template <typename R, typename T>
__global__ void k_soa_to_aos(const R* __restrict__ hi, const R* __restrict__ lo, T* __restrict__ aos, int64_t N) {
  const int64_t I = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (I >= N) return;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    double v = static_cast<double>(hi[c * N + I]);
    if (lo) v += static_cast<double>(lo[c * N + I]);
    aos[3 * I + c] = static_cast<T>(v);
  }
}

template <typename R>
__global__ void k_scalar_to_R(const double* __restrict__ a, R* __restrict__ b, int64_t n, double scale) {
  const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (i < n) b[i] = static_cast<R>(a[i] * scale);
}

template <typename R, typename T>
void launch_aos_to_soa(const T* aos, R* hi, R* lo, int64_t N, int* nanflag, cudaStream_t st) {
  k_aos_to_soa<R, T><<<stage_blocks(N), kStageThreads, 0, st>>>(aos, hi, lo, N, nanflag);
}
template <typename R, typename T>
void launch_soa_to_aos(const R* hi, const R* lo, T* aos, int64_t N, cudaStream_t st) {
  k_soa_to_aos<R, T><<<stage_blocks(N), kStageThreads, 0, st>>>(hi, lo, aos, N);
}
template <typename R>
void launch_scalar_to_R(const double* a, R* b, int64_t n, double scale, cudaStream_t st) {
  k_scalar_to_R<R><<<stage_blocks(n), kStageThreads, 0, st>>>(a, b, n, scale);
}

// ---------------------------------------------------------- reductions ---
// out[t] = sum_b partials[b*width + t], fixed order (one block).
__global__ void k_reduce_sum(const double* __restrict__ partials, int nblocks, int width, double* __restrict__ out) {
  __shared__ double sh[256];
  for (int t = 0; t < width; ++t) {
    double acc = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) acc += partials[static_cast<int64_t>(b) * width + t];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
      if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
      __syncthreads();
    }
    if (threadIdx.x == 0) out[t] = sh[0];
    __syncthreads();
  }
}

void launch_reduce_sum(const double* partials, int nblocks, int width, double* out, cudaStream_t st) {
  k_reduce_sum<<<1, 256, 0, st>>>(partials, nblocks, width, out);
}

template <typename R>
__global__ void k_sum_m(const R* __restrict__ m, const R* __restrict__ lo, int64_t N, double* __restrict__ partials) {
  __shared__ double sh[3][kStageThreads];
  const int64_t I = blockIdx.x * static_cast<int64_t>(kStageThreads) + threadIdx.x;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    double v = 0.0;
    if (I < N) {
      v = m[c * N + I];
      if (lo) v += lo[c * N + I];
    }
    sh[c][threadIdx.x] = v;
  }
  __syncthreads();
  for (int o = kStageThreads / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int c = 0; c < 3; ++c) sh[c][threadIdx.x] += sh[c][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x < 3) partials[blockIdx.x * 3 + threadIdx.x] = sh[threadIdx.x][0];
}

template <typename R>
void launch_average_m(const R* m, const R* m_lo, int64_t N, double* partials, double* out, cudaStream_t st) {
  const int nb = stage_blocks(N);
  k_sum_m<R><<<nb, kStageThreads, 0, st>>>(m, m_lo, N, partials);
  k_reduce_sum<<<1, 256, 0, st>>>(partials, nb, 3, out);
}

// ------------------------------------------------------------- thermal ---
template <typename R>
__global__ void k_thermal(uint32_t k0, uint32_t k1, const long long* __restrict__ step,
                          const double* __restrict__ dt_dev, double dt, double c, const R* __restrict__ T,
                          double T_uni, double T0, const R* __restrict__ mu0Ms, R* __restrict__ H, int64_t N,
                          const int* __restrict__ gate) {
  if (gate && !*gate) return;
  const int64_t I = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (I >= N) return;
  const uint64_t n = static_cast<uint64_t>(*step);
  const double ms = double(mu0Ms[I]);
  double v[3] = {0.0, 0.0, 0.0};
  if (ms > 0) {
    uint32_t ctr[4] = {static_cast<uint32_t>(I), static_cast<uint32_t>(static_cast<uint64_t>(I) >> 32),
                       static_cast<uint32_t>(n), static_cast<uint32_t>(n >> 32)};
    philox4x32_10(ctr, k0, k1);
    const double s32 = 2.3283064365386963e-10;  // 2^-32
    const double r0 = sqrt(-2.0 * log((double(ctr[0]) + 1.0) * s32));
    const double r1 = sqrt(-2.0 * log((double(ctr[2]) + 1.0) * s32));
    const double t0 = 6.283185307179586 * (double(ctr[1]) * s32);
    const double t1 = 6.283185307179586 * (double(ctr[3]) * s32);
    const double h = dt_dev ? *dt_dev : dt;
    const double Tl = (T ? double(T[I]) : T_uni) + T0;
    const double scale = sqrt(c / h * Tl / ms);
    v[0] = r0 * cos(t0) * scale;
    v[1] = r0 * sin(t0) * scale;
    v[2] = r1 * cos(t1) * scale;
  }
  H[I] = static_cast<R>(v[0]);
  H[N + I] = static_cast<R>(v[1]);
  H[2 * N + I] = static_cast<R>(v[2]);
}

template <typename R>
void launch_thermal(uint64_t seed, const long long* step, const double* dt_dev, double dt, double c, const R* T,
                    double T_uni, double T0, const R* mu0Ms, R* Hth, int64_t N, const int* gate, cudaStream_t st) {
  k_thermal<R><<<stage_blocks(N), kStageThreads, 0, st>>>(static_cast<uint32_t>(seed),
                                                          static_cast<uint32_t>(seed >> 32), step, dt_dev, dt, c, T,
                                                          T_uni, T0, mu0Ms, Hth, N, gate);
}

__global__ void k_count_step(long long* step) { *step += 1; }
void launch_count_step(long long* step, cudaStream_t st) { k_count_step<<<1, 1, 0, st>>>(step); }

// ------------------------------------------------------------- adjoint ---
// Reverse mode through one RK4 step.  The forward step is
//   Y1 = y, Yi = y + c_i h k_{i-1} (c = 1/2, 1/2, 1), k_i = f(Y_i),
//   z = y + h/6 (k1 + 2k2 + 2k3 + k4), y' = z / |z|,
// with f the LLG right-hand side of the effective field.  Every field term
// of the path is H_i = (1/mu0Ms_i) sum_j K_ij m_j + Zeeman with a symmetric
// K (it is minus the gradient of a quadratic energy: exchange, both DMIs,
// anisotropy, and demag = N * (Ms m) with a symmetric Newell tensor), so the
// transpose of dH/dm applied to q is mu0Ms * H_lin(q / mu0Ms): the same
// kernels (stencil and demag passes) evaluated on w = q / mu0Ms.

template <typename R>
__global__ void k_adj_stage_input(const R* __restrict__ y, const R* __restrict__ y_lo, const R* __restrict__ k,
                                  R coef, R* __restrict__ out, int64_t n3) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n3;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    if (y_lo) out[i] = y[i] + (y_lo[i] + coef * k[i]);
    else out[i] = y[i] + coef * k[i];
  }
}

template <typename R>
void launch_adj_stage_input(const R* y, const R* y_lo, const R* k, double coef, R* out, int64_t n3, cudaStream_t st) {
  k_adj_stage_input<R><<<1184, 256, 0, st>>>(y, y_lo, k, static_cast<R>(coef), out, n3);
}

template <typename R>
__global__ void k_adj_normalise(const R* __restrict__ y, const R* __restrict__ y_lo, const R* __restrict__ k1,
                                const R* __restrict__ k2, const R* __restrict__ k3, const R* __restrict__ k4,
                                double h6, double* __restrict__ lam, double* __restrict__ mu, double* __restrict__ g,
                                int64_t N) {
  const int64_t I = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (I >= N) return;
  double z[3], l[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const int64_t p = c * N + I;
    const double acc = ((double(k1[p]) + 2.0 * double(k2[p])) + 2.0 * double(k3[p])) + double(k4[p]);
    z[c] = double(y[p]) + (y_lo ? double(y_lo[p]) : 0.0) + h6 * acc;
    l[c] = lam[p];
  }
  const double n2 = z[0] * z[0] + z[1] * z[1] + z[2] * z[2];
  double u[3] = {0, 0, 0}, inv = 0.0;
  if (n2 > 0) {
    inv = 1.0 / sqrt(n2);
    u[0] = z[0] * inv; u[1] = z[1] * inv; u[2] = z[2] * inv;
  }
  const double lu = l[0] * u[0] + l[1] * u[1] + l[2] * u[2];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double v = n2 > 0 ? (l[c] - lu * u[c]) * inv : 0.0;
    lam[c * N + I] = v;
    mu[c * N + I] = v;
    g[c * N + I] = h6 * v;
  }
}

template <typename R>
void launch_adj_normalise(const R* y, const R* y_lo, const R* const k[4], double h, double* lam, double* mu,
                          double* g, int64_t N, cudaStream_t st) {
  k_adj_normalise<R><<<stage_blocks(N), kStageThreads, 0, st>>>(y, y_lo, k[0], k[1], k[2], k[3], h / 6.0, lam, mu,
                                                                  g, N);
}

// VJP of f = C (m x p - alpha p), p = |m|^2 H - (m.H) m, C = c + c_lo, for
// the upstream u:  v = C u, r = v x m - alpha v (no v x m without
// precession), q = dL/dH = |m|^2 r - (r.m) m,
// dL/dm = p x v + 2 (r.H) m - (r.m) H - (m.H) r.
template <typename R>
__global__ void __launch_bounds__(kStageThreads) k_adj_rhs(FieldArgs<R> a, int zeeman, const R* __restrict__ Y,
                                                           const R* __restrict__ HdY, const double* __restrict__ g,
                                                           R* __restrict__ q, R* __restrict__ w,
                                                           double* __restrict__ aexp, AdjGrads gr) {
  const int64_t N = a.N;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= a.nx || j >= a.ny) return;
  const int I = (k * a.ny + j) * a.nx + i;
  R mr[3], hl[3];
  cell_heff<R, false, true>(a, Y, I, i, j, k, mr, hl, nullptr);  // local terms only
  const double ms = double(a.Ms[I]);
  const bool pinned = a.pins && a.pins[I];
  if (ms == 0.0 || pinned) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      q[c * N + I] = R(0);
      w[c * N + I] = R(0);
      aexp[c * N + I] = 0.0;
    }
    return;
  }
  double m[3], h[3], hloc[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    m[c] = double(mr[c]);
    hloc[c] = double(hl[c]);
    h[c] = hloc[c];
  }
  if (HdY) {
    h[0] += double(HdY[I]); h[1] += double(HdY[N + I]); h[2] += double(HdY[2 * N + I]);
  }
  if (zeeman) {
    h[0] += double(a.hz_x); h[1] += double(a.hz_y); h[2] += double(a.hz_z);
    if (a.Hz) {
      h[0] += double(a.Hz[I]); h[1] += double(a.Hz[N + I]); h[2] += double(a.Hz[2 * N + I]);
    }
  }
  const double C = double(a.llg_c) + double(a.llg_c_lo);
  const double alpha = double(a.alpha);
  const double v[3] = {C * g[I], C * g[N + I], C * g[2 * N + I]};
  const double mm = m[0] * m[0] + m[1] * m[1] + m[2] * m[2];
  const double mh = m[0] * h[0] + m[1] * h[1] + m[2] * h[2];
  const double p[3] = {mm * h[0] - mh * m[0], mm * h[1] - mh * m[1], mm * h[2] - mh * m[2]};
  double r[3] = {-alpha * v[0], -alpha * v[1], -alpha * v[2]};
  double ae[3] = {0, 0, 0};
  if (a.precession) {
    r[0] += v[1] * m[2] - v[2] * m[1];
    r[1] += v[2] * m[0] - v[0] * m[2];
    r[2] += v[0] * m[1] - v[1] * m[0];
    ae[0] = p[1] * v[2] - p[2] * v[1];
    ae[1] = p[2] * v[0] - p[0] * v[2];
    ae[2] = p[0] * v[1] - p[1] * v[0];
  }
  const double rh = r[0] * h[0] + r[1] * h[1] + r[2] * h[2];
  const double rm = r[0] * m[0] + r[1] * m[1] + r[2] * m[2];
  double qq[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    ae[c] += 2.0 * rh * m[c] - rm * h[c] - mh * r[c];
    qq[c] = mm * r[c] - rm * m[c];
    q[c * N + I] = static_cast<R>(qq[c]);
    w[c * N + I] = static_cast<R>(qq[c] / ms);
    aexp[c * N + I] = ae[c];
  }
  // H_loc = G / mu0Ms: dH_loc/dMs = -H_loc / Ms (Ms in A/m = mu0Ms / mu0)
  const double qh = qq[0] * hloc[0] + qq[1] * hloc[1] + qq[2] * hloc[2];
  gr.Ms[I] += -kMu0 * qh / ms;
  if (gr.Ku && (a.mask & TB_ANIS)) {
    const double ux = double(a.ux), uy = double(a.uy), uz = double(a.uz);
    const double sa = m[0] * ux + m[1] * uy + m[2] * uz;
    gr.Ku[I] += 2.0 * sa * (qq[0] * ux + qq[1] * uy + qq[2] * uz) / ms;
  }
}

template <typename R>
void launch_adj_rhs(const FieldArgs<R>& fa_loc, bool zeeman, const R* Y, const R* HdY, const double* g, R* q, R* w,
                    double* aexp, AdjGrads gr, cudaStream_t st) {
  const StageGrid sg = stage_grid(fa_loc.nx, fa_loc.ny, fa_loc.nz);
  k_adj_rhs<R><<<sg.grid, sg.block, 0, st>>>(fa_loc, zeeman ? 1 : 0, Y, HdY, g, q, w, aexp, gr);
}

// r_d x m for the interfacial DMI directions d = -x, +x, -y, +y
// (r = +y, -y, -x, +x; the forward stencil of cell_heff)
__device__ __forceinline__ void idmi_cross(int d, const double m[3], double out[3]) {
  if (d == 0) { out[0] = m[2]; out[1] = 0.0; out[2] = -m[0]; }
  else if (d == 1) { out[0] = -m[2]; out[1] = 0.0; out[2] = m[0]; }
  else if (d == 2) { out[0] = 0.0; out[1] = m[2]; out[2] = -m[1]; }
  else { out[0] = 0.0; out[1] = -m[2]; out[2] = m[1]; }
}

template <typename R>
__global__ void __launch_bounds__(kStageThreads)
    k_adj_field(FieldArgs<R> a, const R* __restrict__ w, const R* __restrict__ q, const R* __restrict__ Y,
                const double* __restrict__ aexp, double* __restrict__ lam, const double* __restrict__ mu, double cm,
                double ca, double* __restrict__ gnext, AdjGrads gr) {
  const int64_t N = a.N;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= a.nx || j >= a.ny) return;
  const int I = (k * a.ny + j) * a.nx + i;
  R wr[3], hw[3];
  cell_heff<R, false, true>(a, w, I, i, j, k, wr, hw, nullptr);  // linear local terms on w + demag(w)
  const double ms = double(a.Ms[I]);
  double av[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    av[c] = aexp[c * N + I] + ms * double(hw[c]);
    lam[c * N + I] += av[c];
    if (gnext) gnext[c * N + I] = cm * mu[c * N + I] + ca * av[c];
  }
  if (ms == 0.0) return;
  const double y[3] = {double(Y[I]), double(Y[N + I]), double(Y[2 * N + I])};
  if (a.mask & TB_DEMAG) {
    // H_d = demag(Ms m): dL/dMs_j = m_j . demag(q)_j = mu0 m_j . demag(w)_j
    const double hd[3] = {double(a.Hd[I]), double(a.Hd[N + I]), double(a.Hd[2 * N + I])};
    gr.Ms[I] += kMu0 * (y[0] * hd[0] + y[1] * hd[1] + y[2] * hd[2]);
  }
  if (gr.D && (a.mask & TB_DMI_INTERFACIAL)) {
    // pair (I, n) enters H at both cells with the coefficient
    // hm(D_I, D_n) / d, hm(a, b) = 2ab / (a + b)
    const int nx = a.nx, ny = a.ny;
    const bool px = a.pbc & 1, py = a.pbc & 2;
    const int nb[4] = {i > 0 ? I - 1 : (px ? I + nx - 1 : I), i < nx - 1 ? I + 1 : (px ? I - (nx - 1) : I),
                       j > 0 ? I - nx : (py ? I + (ny - 1) * nx : I),
                       j < ny - 1 ? I + nx : (py ? I - (ny - 1) * nx : I)};
    const unsigned nbm = a.nbm[I];
    const double dd[4] = {double(a.id_x), double(a.id_x), double(a.id_y), double(a.id_y)};
    const double DI = a.D ? double(a.D[I]) : double(a.D_uni);
    const double qI[3] = {double(q[I]), double(q[N + I]), double(q[2 * N + I])};
    double acc = 0.0;
#pragma unroll
    for (int d = 0; d < 4; ++d) {
      if (!((nbm >> d) & 1u)) continue;
      const int n = nb[d];
      double dc;  // d(coefficient)/dD_I
      if (a.D) {
        const double Dn = double(a.D[n]);
        if (DI + Dn == 0.0) continue;
        dc = 2.0 * Dn * Dn / ((DI + Dn) * (DI + Dn)) * dd[d];
      } else {
        dc = 0.5 * dd[d];
      }
      const double yn[3] = {double(Y[n]), double(Y[N + n]), double(Y[2 * N + n])};
      const double qn[3] = {double(q[n]), double(q[N + n]), double(q[2 * N + n])};
      double x1[3], x2[3];
      idmi_cross(d, yn, x1);      // field at I from n
      idmi_cross(d ^ 1, y, x2);   // field at n from I (opposite direction)
      const double t1 = (qI[0] * x1[0] + qI[1] * x1[1] + qI[2] * x1[2]) / ms;
      const double t2 = (qn[0] * x2[0] + qn[1] * x2[1] + qn[2] * x2[2]) / double(a.Ms[n]);
      acc += dc * (t1 + t2);
    }
    gr.D[I] += acc;
  }
}

template <typename R>
void launch_adj_field(const FieldArgs<R>& fa_lin, const R* w, const R* q, const R* Y, const double* aexp,
                      double* lam, const double* mu, double cm, double ca, double* gnext, AdjGrads gr,
                      cudaStream_t st) {
  const StageGrid sg = stage_grid(fa_lin.nx, fa_lin.ny, fa_lin.nz);
  k_adj_field<R><<<sg.grid, sg.block, 0, st>>>(fa_lin, w, q, Y, aexp, lam, mu, cm, ca, gnext, gr);
}

#define MM_INST(R)                                                                                       \
  template void launch_stage<R>(int, const FieldArgs<R>&, const R*, const StageArgs<R>&, cudaStream_t); \
  template bool stage_descriptor_used<R>(const FieldArgs<R>&);                                            \
  template void launch_nbmask<R>(int, int, int, int, const R*, uint8_t*, cudaStream_t);                 \
  template void launch_aos_to_soa<R, double>(const double*, R*, R*, int64_t, int*, cudaStream_t);           \
  template void launch_aos_to_soa<R, float>(const float*, R*, R*, int64_t, int*, cudaStream_t);             \
  template void launch_soa_to_aos<R, double>(const R*, const R*, double*, int64_t, cudaStream_t);           \
  template void launch_soa_to_aos<R, float>(const R*, const R*, float*, int64_t, cudaStream_t);             \
  template void launch_scalar_to_R<R>(const double*, R*, int64_t, double, cudaStream_t);                \
  template void launch_average_m<R>(const R*, const R*, int64_t, double*, double*, cudaStream_t);      \
  template void launch_thermal<R>(uint64_t, const long long*, const double*, double, double, const R*, double,   \
                                  double, const R*, R*, int64_t, const int*, cudaStream_t);                     \
  template void launch_adj_stage_input<R>(const R*, const R*, const R*, double, R*, int64_t, cudaStream_t); \
  template void launch_adj_normalise<R>(const R*, const R*, const R* const[4], double, double*, double*,   \
                                        double*, int64_t, cudaStream_t);                                   \
  template void launch_adj_rhs<R>(const FieldArgs<R>&, bool, const R*, const R*, const double*, R*, R*,    \
                                  double*, AdjGrads, cudaStream_t);                                        \
  template void launch_adj_field<R>(const FieldArgs<R>&, const R*, const R*, const R*, const double*,      \
                                    double*, const double*, double, double, double*, AdjGrads, cudaStream_t);
MM_INST(float)
MM_INST(double)

}  // namespace mm

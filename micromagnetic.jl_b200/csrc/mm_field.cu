// mm_field.cu -- fused effective field + LLG + integrator stage kernels.
#include <cmath>

#include "mm_field.cuh"
#include "mm_launch.cuh"

namespace mm {

constexpr int kStageThreads = 256;

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

// ------------------------------------------------- compensated FP32 math ---
// Error-free transforms (Knuth two-sum, FMA two-product) used to keep the FP32
// form's integrator state m = hi + lo at well beyond FP32 precision.
__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e) {
  s = a + b;
  const float bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}

// hi + lo + d  ->  (hi', lo')
__device__ __forceinline__ void df_add(float& hi, float& lo, float d) {
  float s, e;
  two_sum(hi, lo + d, s, e);
  hi = s;
  lo = e;
}

// Normalise (hi + lo) per cell to unit length in double-float arithmetic
// (normalise, src/helper.jl:255-271: unchanged when |m|^2 == 0).
__device__ __forceinline__ void df_normalise(float* hi, float* lo) {
  float n2h = 0.f, n2l = 0.f;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float p = hi[c] * hi[c];
    const float pe = fmaf(hi[c], hi[c], -p);
    float s, e;
    two_sum(n2h, p, s, e);
    n2h = s;
    n2l += e + pe + 2.f * hi[c] * lo[c];
  }
  if (!(n2h + n2l > 0.f)) return;
  const float d = (n2h - 1.f) + n2l;  // |m|^2 - 1
  if (fabsf(d) < 1e-2f) {
    // 1/sqrt(1+d) - 1 = -d/2 + 3d^2/8 - 5d^3/16 + 35d^4/128
    const float eps = d * (-0.5f + d * (0.375f + d * (-0.3125f + d * 0.2734375f)));
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float s, e;
      two_sum(hi[c], fmaf(hi[c], eps, lo[c] * (1.f + eps)), s, e);
      hi[c] = s;
      lo[c] = e;
    }
  } else {
    const float r = 1.f / sqrtf(n2h + n2l);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float v = hi[c] * r;
      lo[c] = fmaf(hi[c], r, -v) + lo[c] * r;
      float s, e;
      two_sum(v, lo[c], s, e);
      hi[c] = s;
      lo[c] = e;
    }
  }
}

template <typename R>
__device__ __forceinline__ void plain_normalise(R* a) {
  const R m2 = a[0] * a[0] + a[1] * a[1] + a[2] * a[2];
  if (m2 > 0) {
    const R len = R(1) / sqrt(m2);
    a[0] *= len;
    a[1] *= len;
    a[2] *= len;
  }
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

// --------------------------------------------------------- cell H_eff ---
// Field (A/m) of the masked terms at cell I from stage state y; optional
// per-term energies (J) of the cell.  Restates the KernelAbstractions
// kernels of src/micro/kernels.jl (zeeman 14-20, anisotropy 54-75, exchange
// 226-304, bulk DMI 306-344, interfacial DMI 426-466) and the demag energy of
// src/micro/demag.jl:435-456; terms with Ms == 0 contribute nothing.
// The cell and its six neighbours from a shared-memory halo tile instead of
// global memory: component c of the cell at p[c*cs + c0], the x neighbours
// at c0 -+ 1, the y neighbours at c0 -+ sx, the z neighbours at c0 + dm and
// c0 + dp (the tile's planes k-1 and k+1).  Tile cells of absent neighbours
// are never read: their mask bit drops the term.
template <typename R> struct TileNb {
  const R* p;
  int cs, c0, sx, dm, dp;
};

template <typename R, bool ENERGY, bool EXTRA = false, bool TILE = false>
__device__ __forceinline__ void cell_heff(const FieldArgs<R>& a, const R* __restrict__ y, int I, int i, int j,
                                          int k, R m[3], R h[3], double* e, const TileNb<R>& tn = TileNb<R>{}) {
  const int64_t N = a.N;
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const int nxy = nx * ny;
  const unsigned mask = a.mask;
  const bool local = (mask & (TB_EXCH | TB_DMI_BULK | TB_DMI_INTERFACIAL | TB_ANIS)) != 0 ||
                     (EXTRA && (mask & TB_STT_ZL));
  // Every load is issued before any use: neighbour indices are clamped to the
  // cell itself where a neighbour does not exist (the mask bit then drops the
  // term), so no load waits on another.
  const bool px = a.pbc & 1, py = a.pbc & 2, pz = a.pbc & 4;
  int nb[6];
  nb[0] = i > 0 ? I - 1 : (px ? I + nx - 1 : I);
  nb[1] = i < nx - 1 ? I + 1 : (px ? I - (nx - 1) : I);
  nb[2] = j > 0 ? I - nx : (py ? I + (ny - 1) * nx : I);
  nb[3] = j < ny - 1 ? I + nx : (py ? I - (ny - 1) * nx : I);
  nb[4] = k > 0 ? I - nxy : (pz ? I + (nz - 1) * nxy : I);
  nb[5] = k < nz - 1 ? I + nxy : (pz ? I - (nz - 1) * nxy : I);
  if constexpr (TILE) {
#pragma unroll
    for (int c = 0; c < 3; ++c) m[c] = tn.p[c * tn.cs + tn.c0];
  } else {
    m[0] = y[I];
    m[1] = y[N + I];
    m[2] = y[2 * N + I];
  }
  const R Ms = a.Ms[I];
  unsigned nbm = 0;
  R mn[6][3];
  if (local) {
    nbm = a.nbm[I];
    if constexpr (TILE) {
      const int off[6] = {-1, 1, -tn.sx, tn.sx, tn.dm, tn.dp};
#pragma unroll
      for (int d = 0; d < 6; ++d)
#pragma unroll
        for (int c = 0; c < 3; ++c) mn[d][c] = tn.p[c * tn.cs + tn.c0 + off[d]];
    } else {
#pragma unroll
      for (int d = 0; d < 6; ++d) {
        mn[d][0] = __ldg(y + nb[d]);
        mn[d][1] = __ldg(y + N + nb[d]);
        mn[d][2] = __ldg(y + 2 * N + nb[d]);
      }
    }
  }
  R An[6] = {R(0), R(0), R(0), R(0), R(0), R(0)}, AI = R(0);
  if ((mask & TB_EXCH) && a.A) {
    AI = a.A[I];
#pragma unroll
    for (int d = 0; d < 6; ++d) An[d] = __ldg(a.A + nb[d]);
  }
  R Dn[4] = {R(0), R(0), R(0), R(0)}, DI = a.D_uni;
  if ((mask & TB_DMI_INTERFACIAL) && a.D) {
    DI = a.D[I];
#pragma unroll
    for (int d = 0; d < 4; ++d) Dn[d] = __ldg(a.D + nb[d]);
  }
  const R Ku = ((mask & TB_ANIS) && a.Ku) ? a.Ku[I] : a.Ku_uni;
  R hd[3] = {R(0), R(0), R(0)};
  if (mask & TB_DEMAG) {
    hd[0] = a.Hd[I];
    hd[1] = a.Hd[N + I];
    hd[2] = a.Hd[2 * N + I];
  }
  R zx = a.hz_x, zy = a.hz_y, zz = a.hz_z;  // uniform part plus the per-cell part
  if ((mask & TB_ZEEMAN) && a.Hz) {
    zx += a.Hz[I];
    zy += a.Hz[N + I];
    zz += a.Hz[2 * N + I];
  }

  h[0] = h[1] = h[2] = R(0);
  if (ENERGY) {
#pragma unroll
    for (int t = 0; t < kNTerms; ++t) e[t] = 0.0;
  }
  if (Ms != R(0) && local) {
    const R Ms_inv = R(1) / Ms;
    // exchange
    if (mask & TB_EXCH) {
      R fx = 0, fy = 0, fz = 0;
      const R coef[6] = {a.ex_x, a.ex_x, a.ex_y, a.ex_y, a.ex_z, a.ex_z};
      const bool on = a.A ? (AI != R(0)) : true;
      if (on) {
#pragma unroll
        for (int d = 0; d < 6; ++d) {
          if ((nbm >> d) & 1u) {
            R c = coef[d];
            if (a.A) {
              if (An[d] == R(0)) continue;
              const R Aeff = 2 * AI * An[d] / (AI + An[d]);
              c = Aeff * coef[d];
            }
            fx += c * (mn[d][0] - m[0]);
            fy += c * (mn[d][1] - m[1]);
            fz += c * (mn[d][2] - m[2]);
          }
        }
        if (ENERGY) e[1] = -0.5 * (double(fx) * m[0] + double(fy) * m[1] + double(fz) * m[2]) * double(a.V);
        h[0] += fx * Ms_inv;
        h[1] += fy * Ms_inv;
        h[2] += fz * Ms_inv;
      }
    }
    // spatial bulk DMI (spatial_vector_bulkdmi_kernel!, kernels.jl:347-422):
    // per axis the harmonic mean of the two cells' D, pairs with a zero D dropped
    if (EXTRA && (mask & TB_DMI_BULK) && a.x.bD[0]) {
      R fx = 0, fy = 0, fz = 0;
#pragma unroll
      for (int d = 0; d < 6; ++d) {
        if (!((nbm >> d) & 1u)) continue;
        const int ax = d >> 1;
        const R Di = a.x.bD[ax][I], Dn = a.x.bD[ax][nb[d]];
        if (Di == R(0) || Dn == R(0)) continue;
        const R Deff = 2 * Di * Dn / (Di + Dn);
        const R s = (d & 1) ? -a.x.inv_d[ax] : a.x.inv_d[ax];
        if (ax == 0) { fy += Deff * (-s * mn[d][2]); fz += Deff * (s * mn[d][1]); }
        else if (ax == 1) { fx += Deff * (s * mn[d][2]); fz += Deff * (-s * mn[d][0]); }
        else { fx += Deff * (-s * mn[d][1]); fy += Deff * (s * mn[d][0]); }
      }
      if (ENERGY) e[2] = -0.5 * (double(fx) * m[0] + double(fy) * m[1] + double(fz) * m[2]) * double(a.V);
      h[0] += fx * Ms_inv;
      h[1] += fy * Ms_inv;
      h[2] += fz * Ms_inv;
    } else
    // bulk DMI: sum_d (D/d) a_d x m_d, a = +x,-x,+y,-y,+z,-z for d = -x,+x,-y,+y,-z,+z
    if (mask & TB_DMI_BULK) {
      R fx = 0, fy = 0, fz = 0;
      if (nbm & 1u) { fy += a.bd_x * (-mn[0][2]); fz += a.bd_x * mn[0][1]; }
      if (nbm & 2u) { fy += a.bd_x * mn[1][2]; fz += a.bd_x * (-mn[1][1]); }
      if (nbm & 4u) { fx += a.bd_y * mn[2][2]; fz += a.bd_y * (-mn[2][0]); }
      if (nbm & 8u) { fx += a.bd_y * (-mn[3][2]); fz += a.bd_y * mn[3][0]; }
      if (nbm & 16u) { fx += a.bd_z * (-mn[4][1]); fy += a.bd_z * mn[4][0]; }
      if (nbm & 32u) { fx += a.bd_z * mn[5][1]; fy += a.bd_z * (-mn[5][0]); }
      if (ENERGY) e[2] = -0.5 * (double(fx) * m[0] + double(fy) * m[1] + double(fz) * m[2]) * double(a.V);
      h[0] += fx * Ms_inv;
      h[1] += fy * Ms_inv;
      h[2] += fz * Ms_inv;
    }
    // interfacial DMI: r = +y,-y,-x,+x for d = -x,+x,-y,+y; harmonic mean of D
    if ((mask & TB_DMI_INTERFACIAL) && DI != R(0)) {
      R fx = 0, fy = 0, fz = 0;
      const R dd[4] = {a.id_x, a.id_x, a.id_y, a.id_y};
#pragma unroll
      for (int d = 0; d < 4; ++d) {
        if (!((nbm >> d) & 1u)) continue;
        R c;
        if (a.D) {
          if (Dn[d] == R(0)) continue;
          c = (2 * DI * Dn[d] / (DI + Dn[d])) * dd[d];
        } else {
          c = DI * dd[d];
        }
        // r x m_nb
        if (d == 0) { fx += c * mn[0][2]; fz += c * (-mn[0][0]); }
        else if (d == 1) { fx += c * (-mn[1][2]); fz += c * mn[1][0]; }
        else if (d == 2) { fy += c * mn[2][2]; fz += c * (-mn[2][1]); }
        else { fy += c * (-mn[3][2]); fz += c * mn[3][1]; }
      }
      if (ENERGY) e[3] = -0.5 * (double(fx) * m[0] + double(fy) * m[1] + double(fz) * m[2]) * double(a.V);
      h[0] += fx * Ms_inv;
      h[1] += fy * Ms_inv;
      h[2] += fz * Ms_inv;
    }
    // uniaxial anisotropy
    if (mask & TB_ANIS) {
      const R inv2 = R(2) / Ms;
      const R sa = m[0] * a.ux + m[1] * a.uy + m[2] * a.uz;
      h[0] += Ku * sa * a.ux * inv2;
      h[1] += Ku * sa * a.uy * inv2;
      h[2] += Ku * sa * a.uz * inv2;
      if (ENERGY) e[4] = double(Ku) * (1.0 - double(sa) * sa) * double(a.V);
    }
  }
  if (mask & TB_DEMAG) {
    h[0] += hd[0];
    h[1] += hd[1];
    h[2] += hd[2];
    if (ENERGY)
      e[5] = -0.5 * double(Ms) * double(a.V) * (double(m[0]) * hd[0] + double(m[1]) * hd[1] + double(m[2]) * hd[2]);
  }
  if (mask & TB_ZEEMAN) {
    h[0] += zx;
    h[1] += zy;
    h[2] += zz;
    if (ENERGY) e[0] = -double(a.V) * double(Ms) * (double(m[0]) * zx + double(m[1]) * zy + double(m[2]) * zz);
  }
  if constexpr (EXTRA) {
    const ExtraTerms<R>& x = a.x;
    // df_torque_kernel! (kernels.jl:619-632): h = (aj/gamma) m x p + (bj/gamma) p
    if (mask & TB_SOT) {
      const R aa = (x.sot_aj ? x.sot_aj[I] : x.sot_aj_uni) * x.sot_inv_g;
      h[0] += aa * (m[1] * x.sot_p[2] - m[2] * x.sot_p[1]) + x.sot_b * x.sot_p[0];
      h[1] += aa * (m[2] * x.sot_p[0] - m[0] * x.sot_p[2]) + x.sot_b * x.sot_p[1];
      h[2] += aa * (m[0] * x.sot_p[1] - m[1] * x.sot_p[0]) + x.sot_b * x.sot_p[2];
    }
    // zhangli_torque_kernel! (kernels.jl:680-739): f = ut sum_axis bJ_axis (m_+ - m_-)
    // / (2d or d), neighbours by existence in the mesh; h = m x f + xi f
    if (mask & TB_STT_ZL) {
      const bool px = a.pbc & 1, py = a.pbc & 2, pz = a.pbc & 4;
      const bool ex[6] = {i > 0 || px, i < nx - 1 || px, j > 0 || py, j < ny - 1 || py, k > 0 || pz, k < nz - 1 || pz};
      R f[3] = {R(0), R(0), R(0)};
#pragma unroll
      for (int ax = 0; ax < 3; ++ax) {
        const R dd = ax == 0 ? x.inv_d[0] : (ax == 1 ? x.inv_d[1] : x.inv_d[2]);
        const R fac = (ex[2 * ax] && ex[2 * ax + 1]) ? R(0.5) * dd : dd;
        const R u = x.zl_bJ[ax * N + I] * fac;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const R mp = ex[2 * ax + 1] ? mn[2 * ax + 1][c] : m[c];
          const R mm = ex[2 * ax] ? mn[2 * ax][c] : m[c];
          f[c] += u * (mp - mm);
        }
      }
      const R xi = x.zl_xi ? x.zl_xi[I] : x.zl_xi_uni;
#pragma unroll
      for (int c = 0; c < 3; ++c) f[c] *= x.zl_ut;
      h[0] += (m[1] * f[2] - m[2] * f[1]) + xi * f[0];
      h[1] += (m[2] * f[0] - m[0] * f[2]) + xi * f[1];
      h[2] += (m[0] * f[1] - m[1] * f[0]) + xi * f[2];
    }
    // slonczewski_torque_kernel!: eps = P L^2 / (L^2 + 1 + (L^2 - 1) m.p),
    // h = J ft beta (eps m x p + xi p)
    if (mask & TB_STT_SL) {
      const R mp = m[0] * x.sl_p[0] + m[1] * x.sl_p[1] + m[2] * x.sl_p[2];
      const R eps = x.sl_P * x.sl_L2 / (x.sl_L2 + R(1) + (x.sl_L2 - R(1)) * mp);
      const R aa = (x.sl_J ? x.sl_J[I] : x.sl_J_uni) * x.sl_ftb;
      h[0] += aa * (eps * (m[1] * x.sl_p[2] - m[2] * x.sl_p[1]) + x.sl_xi * x.sl_p[0]);
      h[1] += aa * (eps * (m[2] * x.sl_p[0] - m[0] * x.sl_p[2]) + x.sl_xi * x.sl_p[1]);
      h[2] += aa * (eps * (m[0] * x.sl_p[1] - m[1] * x.sl_p[0]) + x.sl_xi * x.sl_p[2]);
    }
    if (mask & TB_THERMAL) {
      h[0] += x.Hth[I];
      h[1] += x.Hth[N + I];
      h[2] += x.Hth[2 * N + I];
    }
  }
}

// llg_rhs_kernel!  src/llg/llg.jl:6-40
template <typename R>
__device__ __forceinline__ void llg_rhs(const FieldArgs<R>& a, int64_t I, const R m[3], const R h[3], R f[3]) {
  if (a.pins && a.pins[I]) {
    f[0] = f[1] = f[2] = R(0);
    return;
  }
  const R alpha = a.alpha;
  const R c = a.llg_c, cl = a.llg_c_lo;
  const R mm = m[0] * m[0] + m[1] * m[1] + m[2] * m[2];
  const R mh = m[0] * h[0] + m[1] * h[1] + m[2] * h[2];
  const R h1 = mm * h[0] - mh * m[0];
  const R h2 = mm * h[1] - mh * m[1];
  const R h3 = mm * h[2] - mh * m[2];
  R f1 = 0, f2 = 0, f3 = 0;
  if (a.precession) {
    f1 = -m[2] * h2 + m[1] * h3;
    f2 = m[2] * h1 - m[0] * h3;
    f3 = -m[1] * h1 + m[0] * h2;
  }
  const R g1 = f1 - h1 * alpha, g2 = f2 - h2 * alpha, g3 = f3 - h3 * alpha;
  f[0] = c * g1 + cl * g1;
  f[1] = c * g2 + cl * g2;
  f[2] = c * g3 + cl * g3;
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

// The RK4 / Heun stage update of one cell from its field h at the stage input
// m: advance_step(::RungeKutta) src/integrator/rk.jl:23-52 and
// advance_step(::ModifiedEuler) src/integrator/heun.jl:28-49.  mN, mL: the
// step's start state (hi, lo); av: the accumulator.
template <typename R>
__device__ __forceinline__ void rk4_update(const FieldArgs<R>& a, const StageArgs<R>& s, int I, const R m[3],
                                           const R h[3], const R mN[3], const R mL[3], const R av[3]) {
  constexpr bool kF32 = sizeof(R) == 4;
  const int64_t N = a.N;
  if (s.scheme == 1) {
    // advance_step(::ModifiedEuler)  src/integrator/heun.jl:28-49:
    // k1 = f(m); y = m + h k1; k2 = f(y); m = normalise(m + (h/2) k1 + (h/2) k2)
    R f[3];
    llg_rhs(a, I, m, h, f);
    if (s.stage == 1) {
      const R hh = static_cast<R>(s.h);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        s.acc[c * N + I] = f[c];
        s.ynext[c * N + I] = kF32 ? mN[c] + (mL[c] + hh * f[c]) : mN[c] + hh * f[c];
      }
    } else {
      const R h2 = static_cast<R>(0.5 * s.h);
      R mv[3];
      if constexpr (kF32) {
        float lo[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          mv[c] = mN[c];
          lo[c] = mL[c];
          df_add(mv[c], lo[c], h2 * av[c] + h2 * f[c]);
        }
        df_normalise(mv, lo);
#pragma unroll
        for (int c = 0; c < 3; ++c) s.m_lo[c * N + I] = lo[c];
      } else {
#pragma unroll
        for (int c = 0; c < 3; ++c) mv[c] = mN[c] + h2 * av[c] + h2 * f[c];
        plain_normalise(mv);
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) s.m[c * N + I] = mv[c];
    }
  } else {
    // advance_step(::RungeKutta)  src/integrator/rk.jl:23-52
    R f[3];
    llg_rhs(a, I, m, h, f);
    const int st = s.stage;
    if (st < 4) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const R kc = f[c];
        s.acc[c * N + I] = st == 1 ? kc : av[c] + 2 * kc;
      }
      const R cf = static_cast<R>(st == 3 ? s.h : 0.5 * s.h);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        R v;
        if (kF32) v = mN[c] + (mL[c] + cf * f[c]);
        else v = mN[c] + cf * f[c];
        s.ynext[c * N + I] = v;
      }
    } else {
      const R c6 = static_cast<R>(1.0 / 6 * s.h);
      R mv[3];
      if constexpr (kF32) {
        float lo[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          mv[c] = mN[c];
          lo[c] = mL[c];
          df_add(mv[c], lo[c], c6 * (av[c] + f[c]));
        }
        df_normalise(mv, lo);
#pragma unroll
        for (int c = 0; c < 3; ++c) s.m_lo[c * N + I] = lo[c];
      } else {
#pragma unroll
        for (int c = 0; c < 3; ++c) mv[c] = mN[c] + c6 * (av[c] + f[c]);
        plain_normalise(mv);
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) s.m[c * N + I] = mv[c];
    }
  }
}

template <typename R, int MODE, bool EXTRA>
__global__ void __launch_bounds__(kStageThreads, sizeof(R) == 4 ? 3 : 2) k_stage(FieldArgs<R> a, const R* __restrict__ y, StageArgs<R> s) {
  constexpr bool kF32 = sizeof(R) == 4;
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

// RK4 / Heun stage, one cell a thread and one z plane a block (k_stage's
// SM_RK4 mode without the further terms) as a descriptor, so that batches can
// merge it; blocks are 1-D, the cell tile bx x by comes with the arguments.
template <typename R>
struct StagePlain {
  static constexpr int kNT = kStageThreads, kMinB = sizeof(R) == 4 ? 3 : 2;
  struct Args {
    FieldArgs<R> a;
    const R* y;
    StageArgs<R> s;
    int bx, by;
    dim3 grid;
  };
  static __device__ __forceinline__ void body(const Args& args, uint3 blockIdx) {
    const FieldArgs<R>& a = args.a;
    const StageArgs<R>& s = args.s;
    constexpr bool kF32 = sizeof(R) == 4;
    const int64_t N = a.N;
    const int tid = threadIdx.x, bx = args.bx;
    const int i = blockIdx.x * bx + tid % bx;
    const int j = blockIdx.y * args.by + tid / bx;
    const int k = blockIdx.z;
    if (i >= a.nx || j >= a.ny) return;
    const int I = (k * a.ny + j) * a.nx + i;
    R mN[3], mL[3], av[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      mN[c] = s.m[c * N + I];
      mL[c] = kF32 ? s.m_lo[c * N + I] : R(0);
      av[c] = s.stage > 1 ? s.acc[c * N + I] : R(0);
    }
    R m[3], h[3];
    cell_heff<R, false, false>(a, args.y, I, i, j, k, m, h, nullptr);
    rk4_update(a, s, I, m, h, mN, mL, av);
  }
};

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
      case SM_FIELD: k_stage<R, SM_FIELD, true><<<g.grid, g.block, 0, st>>>(fa, y, sa); break;
      case SM_RHS: k_stage<R, SM_RHS, true><<<g.grid, g.block, 0, st>>>(fa, y, sa); break;
      case SM_RK4: k_stage<R, SM_RK4, true><<<g.grid, g.block, 0, st>>>(fa, y, sa); break;
      case SM_ENERGY: k_stage<R, SM_ENERGY, true><<<g.grid, g.block, 0, st>>>(fa, y, sa); break;
      default: k_stage<R, SM_DOPRI, true><<<g.grid, g.block, 0, st>>>(fa, y, sa); break;
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
    launch_k<StagePlain<R>>(g.grid, 0, st, {fa, y, sa, static_cast<int>(g.block.x), static_cast<int>(g.block.y), dim3()});
    return;
  }
  switch (mode) {
    case SM_FIELD: k_stage<R, SM_FIELD, false><<<g.grid, g.block, 0, st>>>(fa, y, sa); break;
    case SM_RHS: k_stage<R, SM_RHS, false><<<g.grid, g.block, 0, st>>>(fa, y, sa); break;
    case SM_ENERGY: k_stage<R, SM_ENERGY, false><<<g.grid, g.block, 0, st>>>(fa, y, sa); break;
    default: k_stage<R, SM_DOPRI, false><<<g.grid, g.block, 0, st>>>(fa, y, sa); break;
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

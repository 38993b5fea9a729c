// mm_cell.cuh -- the per-cell device functions of the fused stage kernels:
// compensated FP32 arithmetic, the effective field of one cell (cell_heff),
// the LLG right-hand side, the RK4 / Heun update, and the RK4 stage as a
// launch descriptor (StagePlain).  Shared by mm_field.cu and the persistent
// step kernel (mm_persist.cu).  Internal.
#pragma once
#include <cmath>

#include "mm_field.cuh"
#include "mm_launch.cuh"

namespace mm {

constexpr int kStageThreads = 256;

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

// FIX != 0: the term set is the compile-time mask FIX and every parameter is
// uniform (no A, D, Ku or Zeeman array), so the branches on terms that are
// absent and on per-cell parameters compile away; FIX == 0 reads the mask.
template <typename R, bool ENERGY, bool EXTRA = false, bool TILE = false, unsigned FIX = 0>
__device__ __forceinline__ void cell_heff(const FieldArgs<R>& a, const R* __restrict__ y, int I, int i, int j,
                                          int k, R m[3], R h[3], double* e, const TileNb<R>& tn = TileNb<R>{}) {
  const int64_t N = a.N;
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const int nxy = nx * ny;
  const unsigned mask = FIX ? FIX : a.mask;
  const R* const pA = FIX ? nullptr : a.A;
  const R* const pD = FIX ? nullptr : a.D;
  const R* const pKu = FIX ? nullptr : a.Ku;
  const R* const pHz = FIX ? nullptr : a.Hz;
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
  if ((mask & TB_EXCH) && pA) {
    AI = pA[I];
#pragma unroll
    for (int d = 0; d < 6; ++d) An[d] = __ldg(pA + nb[d]);
  }
  R Dn[4] = {R(0), R(0), R(0), R(0)}, DI = a.D_uni;
  if ((mask & TB_DMI_INTERFACIAL) && pD) {
    DI = pD[I];
#pragma unroll
    for (int d = 0; d < 4; ++d) Dn[d] = __ldg(pD + nb[d]);
  }
  const R Ku = ((mask & TB_ANIS) && pKu) ? pKu[I] : a.Ku_uni;
  R hd[3] = {R(0), R(0), R(0)};
  if (mask & TB_DEMAG) {
    hd[0] = a.Hd[I];
    hd[1] = a.Hd[N + I];
    hd[2] = a.Hd[2 * N + I];
  }
  R zx = a.hz_x, zy = a.hz_y, zz = a.hz_z;  // uniform part plus the per-cell part
  if ((mask & TB_ZEEMAN) && pHz) {
    zx += pHz[I];
    zy += pHz[N + I];
    zz += pHz[2 * N + I];
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
      const bool on = pA ? (AI != R(0)) : true;
      if (on) {
#pragma unroll
        for (int d = 0; d < 6; ++d) {
          if ((nbm >> d) & 1u) {
            R c = coef[d];
            if (pA) {
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
        if (pD) {
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

// RK4 / Heun stage, one cell a thread and one z plane a block (k_stage's
// SM_RK4 mode without the further terms) as a descriptor, so that batches can
// merge it; blocks are 1-D, the cell tile bx x by comes with the arguments.
template <typename R, unsigned FIX = 0>
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
    const int tid = threadIdx.x, bx = args.bx;  // bx: a power of two
    const int i = blockIdx.x * bx + (tid & (bx - 1));
    const int j = blockIdx.y * args.by + (tid >> (__ffs(bx) - 1));
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
    cell_heff<R, false, false, false, FIX>(a, args.y, I, i, j, k, m, h, nullptr);
    rk4_update(a, s, I, m, h, mN, mL, av);
  }
};

// Term sets with a compiled stage kernel of their own (all parameters
// uniform): exchange + demag (c5), + Zeeman (fig9, c1), exchange + bulk DMI +
// anisotropy + demag (c2), exchange + interfacial DMI + demag (c3 films)
constexpr unsigned kFixExDemag = TB_EXCH | TB_DEMAG;
constexpr unsigned kFixExDemagZee = TB_EXCH | TB_DEMAG | TB_ZEEMAN;
constexpr unsigned kFixExBulkAnisDemag = TB_EXCH | TB_DMI_BULK | TB_ANIS | TB_DEMAG;
constexpr unsigned kFixExIntDemag = TB_EXCH | TB_DMI_INTERFACIAL | TB_DEMAG;

template <typename R> struct PersistKind<StagePlain<R>> { static constexpr int value = 11; };

}  // namespace mm

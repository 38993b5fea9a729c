// mm_field.cuh -- fused effective-field / LLG / integrator-stage kernels
// (internal interface of libmmcuda).
//
// One thread per cell, SoA state y[c*N + cell] (x fastest).  The local terms
// (exchange, bulk and interfacial DMI, uniaxial anisotropy, Zeeman) are
// evaluated from the cell and its six neighbours, the demag field is read
// from the buffer written by the FFT passes, and the LLG right-hand side and
// the integrator-stage update are applied in the same kernel.
#pragma once
#include "mm_common.cuh"

namespace mm {

enum TermBit : unsigned {
  TB_ZEEMAN = 1u << 0,
  TB_EXCH = 1u << 1,
  TB_DMI_BULK = 1u << 2,
  TB_DMI_INTERFACIAL = 1u << 3,
  TB_ANIS = 1u << 4,
  TB_DEMAG = 1u << 5,
  TB_SOT = 1u << 6,        // add_sot: field-like / damping-like torque field
  TB_STT_ZL = 1u << 7,     // add_stt(model=:zhang_li)
  TB_STT_SL = 1u << 8,     // add_stt(model=:slonczewski)
  TB_THERMAL = 1u << 9,    // add_thermal_noise
};
constexpr int kNTerms = 6;  // terms with an energy (Zeeman .. demag)
constexpr int kNTermIds = 10;
constexpr unsigned kExtraBits = TB_SOT | TB_STT_ZL | TB_STT_SL | TB_THERMAL;

// Terms outside the base set, evaluated in the same per-cell kernel when a
// handle has them (src/micro/kernels.jl: spatial_vector_bulkdmi 347-422,
// df_torque 619-632, zhangli_torque 680-739, slonczewski_torque;
// stochastic_field 469-494).  Torque terms enter as equivalent fields, as the
// reference adds them to the effective field.
template <typename R> struct ExtraTerms {
  const R* bD[3];          // spatial bulk DMI: per-cell Dx, Dy, Dz (null: uniform bd_*)
  R inv_d[3];              // 1/dx, 1/dy, 1/dz
  const R* sot_aj;         // SOT: h = (aj/gamma)(m x p) + (bj/gamma) p
  R sot_aj_uni, sot_b, sot_inv_g;
  R sot_p[3];
  const R* zl_bJ;          // Zhang-Li: b*J per cell, SoA 3N
  const R* zl_xi;
  R zl_xi_uni, zl_ut;      // ut = ft / gamma
  const R* sl_J;           // Slonczewski: J per cell
  R sl_J_uni, sl_ftb, sl_L2, sl_P, sl_xi;
  R sl_p[3];
  const R* Hth;            // thermal field of the current step, SoA 3N
};

template <typename R> struct FieldArgs {
  int nx, ny, nz, pbc;
  int64_t N;
  R V;                    // cell volume
  const R* Ms;            // mu0*Ms (T), N
  const uint8_t* nbm;     // bit d: neighbour d exists and has Ms > 0
  unsigned mask;          // TermBit set
  // exchange: uniform coefficients 2A/d^2, or 2/d^2 with the A array
  R ex_x, ex_y, ex_z;
  const R* A;             // null: uniform
  // bulk DMI: D/d per axis
  R bd_x, bd_y, bd_z;
  // interfacial DMI: D (uniform) or D array, and 1/dx, 1/dy
  R D_uni;
  const R* D;
  R id_x, id_y;
  // uniaxial anisotropy
  R Ku_uni;
  const R* Ku;
  R ux, uy, uz;
  // Zeeman (A/m), uniform or SoA array
  R hz_x, hz_y, hz_z;
  const R* Hz;
  // demag field (SoA, written by the FFT passes)
  const R* Hd;
  // LLG: c = -gamma/(1 + alpha^2) evaluated in FP64 on the host and passed
  // as c + c_lo (c_lo = 0 in the FP64 form) so that the FP32 form carries no
  // systematic precession-frequency error from rounding the constant
  R alpha, llg_c, llg_c_lo;
  int precession;
  const uint8_t* pins;
  ExtraTerms<R> x;
};

enum StageMode { SM_FIELD = 0, SM_RHS = 1, SM_RK4 = 2, SM_ENERGY = 3, SM_DOPRI = 4 };

// Adaptive Runge-Kutta methods of src/integrator/adaptive_rk.jl:248-266
enum RkMethod { RK_DOPRI54 = 0, RK_BS23 = 1, RK_CASHKARP54 = 2, RK_FEHLBERG54 = 3, RK_NMETHODS = 4 };

// One embedded pair in the layout the stage kernel walks (the Butcher tables
// of src/integrator/adaptive_rk_steps.jl).  Stage s (1-based) evaluates
// k_s = f(y_s); for s <= sol it then forms sum_j a[s-1][j] h k_{j+1}, which
// is the input of stage s+1, or for s == sol the solution y_next (normalised).
// The error sum_j w[j] k_{j+1} is taken at stage err (sol, or sol+1 when it
// needs f(y_next)).
struct RkTableau {
  int nstage, sol, err, fsal, order_main, order_emb;
  double a[7][7];
  double w[7];
};
const RkTableau& rk_tableau(int method);  // host copy

// Adaptive RK device-side controller state (src/integrator/adaptive_rk.jl:93-186)
struct DopriCtrl {
  double t, step, step_next, t_final, tol;
  double err;               // last scaled error norm
  long long nsteps, nfevals, attempts, rejected;
  int inner;                // attempts of the current advance_step (nstep)
  int active;               // 1 while integrating
  int status;               // 0 ok, 1 NaN, 2 too many attempts
  int accepted_last;        // last attempt accepted
  int need_init;            // compute_initial_step pending
  int single;               // stop after one accepted step (advance_step)
  double init_rmax;         // max |f| for the initial step
  int succeed;              // integrator.succeed: last attempt that reached the acceptance test
  int eval1;                // stage 1 evaluates f (0: FSAL reuse of the last stage, or inactive)
  int fsal, order, nstage;  // of the method in use
};

template <typename R> struct StageArgs {
  R* out;                   // SM_FIELD: H (SoA); SM_RHS: dm/dt (SoA)
  R* ecell;                 // SM_FIELD: per-cell energy of the masked terms (may be null)
  double* partials;         // SM_ENERGY: [blocks][kNTerms]; SM_DOPRI stage 7: [blocks] max
  // integrator state m_n = m + m_lo (m_lo null in the FP64 form)
  R* m;
  R* m_lo;
  R* acc;                   // RK4 accumulator
  R* ynext;                 // next stage input
  R* ynext_lo;              // DOPRI stage 7: low part of y_next
  R* k[7];                  // adaptive RK stage derivatives
  double h;                 // RK4 / Heun step
  int stage;                // 1-based
  int scheme;               // fixed-step scheme: 0 RK4, 1 Heun (modified Euler)
  int method;               // SM_DOPRI: RkMethod
  const DopriCtrl* ctrl;    // SM_DOPRI: step size and active flag
};

template <typename R>
void launch_stage(int mode, const FieldArgs<R>& fa, const R* y, const StageArgs<R>& sa, cudaStream_t st);

int stage_blocks(int64_t N);

// launch_stage(SM_RK4, fa, ...) runs a descriptor kernel (mm_launch.cuh) for
// these field arguments (no further terms)
template <typename R>
bool stage_descriptor_used(const FieldArgs<R>& fa);

struct StageGrid {
  dim3 grid, block;
  int nblocks;
};
StageGrid stage_grid(int nx, int ny, int nz);

template <typename R>
void launch_nbmask(int nx, int ny, int nz, int pbc, const R* Ms, uint8_t* nbm, cudaStream_t st);

// AoS T (double or float) <-> SoA R (+ compensated low part)
template <typename R, typename T = double>
void launch_aos_to_soa(const T* aos, R* hi, R* lo, int64_t N, int* nanflag, cudaStream_t st);
template <typename R, typename T = double>
void launch_soa_to_aos(const R* hi, const R* lo, T* aos, int64_t N, cudaStream_t st);
template <typename R>
void launch_scalar_to_R(const double* a, R* b, int64_t n, double scale, cudaStream_t st);

// deterministic final reductions
void launch_reduce_sum(const double* partials, int nblocks, int width, double* out, cudaStream_t st);

template <typename R>
void launch_average_m(const R* m, const R* m_lo, int64_t N, double* partials, double* out, cudaStream_t st);

// ------------------------------------------------------------- thermal ---
// Counter-based normal deviates: Philox-4x32-10 (Salmon, Moraes, Dror, Shaw,
// SC'11) on the counter (cell, step) with the seed as key, Box-Muller on the
// four 32-bit outputs.  Identical on host and device, so the thermal field of
// step n is a function of (seed, n, cell) only.
__host__ __device__ inline void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = static_cast<uint64_t>(0xD2511F53u) * c[0];
    const uint64_t p1 = static_cast<uint64_t>(0xCD9E8D57u) * c[2];
    const uint32_t hi0 = static_cast<uint32_t>(p0 >> 32), lo0 = static_cast<uint32_t>(p0);
    const uint32_t hi1 = static_cast<uint32_t>(p1 >> 32), lo1 = static_cast<uint32_t>(p1);
    const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0;
    c[1] = lo1;
    c[2] = n2;
    c[3] = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

// add_thermal_noise: H = eta sqrt(factor (T + T0) / mu0Ms), factor =
// 2 alpha k_B scaling / (V gamma dt)  (stochastic_field_kernel!,
// src/micro/kernels.jl:469-494; src/micro/field.jl:244-280).  The step index
// is read from step (device); dt from dt_dev when non-null, else dt.
template <typename R>
void launch_thermal(uint64_t seed, const long long* step, const double* dt_dev, double dt, double alpha_kB_s_over_Vg,
                    const R* T, double T_uni, double T0, const R* mu0Ms, R* Hth, int64_t N, const int* gate,
                    cudaStream_t st);
void launch_count_step(long long* step, cudaStream_t st);

// ------------------------------------------------------------- adjoint ---
// Discrete adjoint of one RK4 step (src/integrator/rk.jl:23-52 with the
// field of src/micro/kernels.jl and the LLG right-hand side of
// src/llg/llg.jl:6-40).  lam, mu, g and a are FP64 SoA arrays of 3N.
struct AdjGrads {
  double* Ms;   // dL/dMs (per A/m), N, accumulated
  double* Ku;   // dL/dKu, N, accumulated (null: not wanted)
  double* D;    // dL/dD of interfacial DMI, N, accumulated (null: not wanted)
};

// Y_next = y (+ y_lo) + coef * k, the RK4 stage input exactly as the forward
// stage kernel forms it
template <typename R>
void launch_adj_stage_input(const R* y, const R* y_lo, const R* k, double coef, R* out, int64_t n3, cudaStream_t st);

// Normalisation at the end of the step: z = y + h/6 (((k1 + 2k2) + 2k3) + k4),
// m_{n+1} = z/|z|.  In: lam = dL/dm_{n+1}.  Out: mu = dL/dz (also in lam),
// g = (h/6) mu, the upstream gradient of k4.
template <typename R>
void launch_adj_normalise(const R* y, const R* y_lo, const R* const k[4], double h, double* lam, double* mu,
                          double* g, int64_t N, cudaStream_t st);

// Stage VJP, part 1: with the field H(Y) (local terms of fa_loc, plus Hd and
// Zeeman), dL/dH = q and the explicit dL/dY of the LLG right-hand side for
// the upstream gradient g of k = f(Y).  Writes q, w = q / (mu0 Ms), aexp and
// accumulates the Ms and Ku gradients of the local terms.
template <typename R>
void launch_adj_rhs(const FieldArgs<R>& fa_loc, bool zeeman, const R* Y, const R* HdY, const double* g, R* q, R* w,
                    double* aexp, AdjGrads gr, cudaStream_t st);

// Stage VJP, part 2: a = aexp + mu0 Ms * H_lin(w) (H_lin: the linear local
// terms on w plus the demag field Hdw = demag(w)), lam += a, Ms gradient of
// demag, interfacial-D gradient of the pairs; if gnext: gnext = cm*mu + ca*a.
template <typename R>
void launch_adj_field(const FieldArgs<R>& fa_lin, const R* w, const R* q, const R* Y, const double* aexp,
                      double* lam, const double* mu, double cm, double ca, double* gnext, AdjGrads gr,
                      cudaStream_t st);

}  // namespace mm

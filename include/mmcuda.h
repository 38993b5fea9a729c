/*
 * mmcuda.h -- C ABI of libmmcuda.so, a B200 (sm_100a) implementation of the
 * MicroMagnetic.jl finite-difference hot path: effective field (exchange,
 * bulk / interfacial DMI, uniaxial anisotropy, Zeeman, FFT demag), LLG
 * right-hand side, RK4 and Dormand-Prince integration, steepest-descent relax.
 *
 * Conventions
 *  - Plain pointers and sizes only.  Host arrays are float64, cell id
 *    (k*ny + j)*nx + i with x fastest; vector fields are AoS
 *    [x1, y1, z1, x2, ...] exactly like MicroMagnetic.jl's `sim.spin` /
 *    `sim.field` (src/micro/mesh.jl:24-29).
 *  - A handle owns its device memory and a CUDA stream; the state stays on
 *    the device between calls.  Calls on one handle must come from one host
 *    thread at a time.  Compute calls are asynchronous unless they return
 *    data to the host; mm_synchronize() waits for the handle's stream.
 *  - Every function returns MM_OK (0) or a negative mm_status; no exception
 *    crosses the ABI.  mm_last_error() gives the message of the calling
 *    thread's last failure.
 *  - form MM_FP64: state, fields and FFTs in FP64.  MM_FP32: state and
 *    fields in FP32 with the integrator state kept compensated
 *    (hi + lo), FP64 for the Newell tensor assembly, the Dormand-Prince
 *    error norm and the energy reductions.
 */
#ifndef MMCUDA_H
#define MMCUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MMCUDA_ABI_VERSION 1

typedef struct mm_handle mm_handle;

enum mm_status {
  MM_OK = 0,
  MM_ERR_ARG = -1,         /* bad argument / size */
  MM_ERR_CUDA = -2,        /* CUDA runtime failure */
  MM_ERR_NAN = -3,         /* NaN in inputs or in the integration */
  MM_ERR_NOCONVERGE = -4,  /* > 50 rejected attempts in one adaptive step */
  MM_ERR_TIMEOUT = -5,     /* bounded device wait ran out */
  MM_ERR_STATE = -6,       /* call out of order (e.g. no Ms set) */
  MM_ERR_UNSUPPORTED = -7  /* valid in the reference, not on this path */
};

enum mm_form { MM_FP64 = 0, MM_FP32 = 1 };

/* interaction terms; bit i of a term mask selects term i */
enum mm_term {
  MM_TERM_ZEEMAN = 0,
  MM_TERM_EXCH = 1,
  MM_TERM_DMI_BULK = 2,
  MM_TERM_DMI_INTERFACIAL = 3,
  MM_TERM_ANIS = 4,
  MM_TERM_DEMAG = 5,
  MM_NTERMS = 6, /* terms with an energy; mm_energy reports these */
  /* field-only terms (mm_term_field; no energy) */
  MM_TERM_SOT = 6,
  MM_TERM_STT_ZHANG_LI = 7,
  MM_TERM_STT_SLONCZEWSKI = 8,
  MM_TERM_THERMAL = 9
};

enum mm_driver { MM_DRIVER_SD = 0, MM_DRIVER_LLG = 1 };

/* FDMesh(; dx, dy, dz, nx, ny, nz, pbc)  src/micro/mesh.jl:69-98 */
typedef struct {
  int32_t nx, ny, nz;
  double dx, dy, dz;
  int32_t pbc; /* bit0 x, bit1 y, bit2 z periodic */
} mm_mesh_desc;

/* Adaptive integrator statistics, cf. get_statistics
 * src/integrator/adaptive_rk.jl:188-192 */
typedef struct {
  double t, step, step_next;
  int64_t nsteps, nfevals, attempts, rejected;
  int32_t status; /* 0 ok, 1 NaN, 2 too many attempts */
} mm_stats;

int mm_abi_version(void);
/* Message of the calling thread's last failing call (always NUL-terminated). */
int mm_last_error(char* buf, size_t n);

/* Sim(mesh)  src/sim.jl:48-107 (state + driver storage on `device`) */
int mm_create(const mm_mesh_desc* mesh, int form, int device, mm_handle** out);
int mm_destroy(mm_handle* h);
/* CUDA stream (cudaStream_t) the handle launches on. */
int mm_get_stream(mm_handle* h, void** stream);
/* Waits for the handle's stream.  MM_ERR_TIMEOUT: a bounded device wait of a
 * demag pass (the bulk-copy fed y passes and z convolution of the FP32
 * register path) ran out on this device since the last call; the fields
 * computed meanwhile are incomplete. */
int mm_synchronize(mm_handle* h);
/* Bytes of device memory held by the handle. */
int mm_device_bytes(mm_handle* h, size_t* bytes);

/* set_Ms(sim, Ms)  src/sim.jl:129-143 -- A/m; Ms == NULL uses Ms_uniform */
int mm_set_Ms(mm_handle* h, const double* Ms, double Ms_uniform);
/* init_m0 copy-in  src/sim.jl:278-309 (the caller normalises / zeroes) */
int mm_set_m(mm_handle* h, const double* m_aos);
/* sim.spin copy-out */
int mm_get_m(mm_handle* h, double* m_aos);
/* The same with a Float32 host array: sim.spin in the reference's Float32
   mode (set_precision(Float32), src/MicroMagnetic.jl:22-38; sim.spin =
   create_zeros(3n) of Float[], src/sim.jl:70).  Half the host<->device bytes
   of the double calls; the state keeps its form's precision. */
int mm_set_m_f32(mm_handle* h, const float* m_aos);
int mm_get_m_f32(mm_handle* h, float* m_aos);
/* set_pinning  src/sim.jl (sim.pins): NULL clears */
int mm_set_pins(mm_handle* h, const uint8_t* pins);
/* LLG driver parameters  src/driver.jl:15-21 (alpha, gamma, precession) */
int mm_set_llg(mm_handle* h, double alpha, double gamma, int precession);

/* add_zeeman / update_zeeman  src/micro/add_field.jl:11-48: H in A/m,
 * AoS 3N or NULL for the uniform (Hx, Hy, Hz).  add accumulates, update replaces. */
int mm_add_zeeman(mm_handle* h, const double* H_aos, double Hx, double Hy, double Hz);
int mm_update_zeeman(mm_handle* h, const double* H_aos, double Hx, double Hy, double Hz);
/* add_exch  src/micro/add_field.jl:233-263: A (J/m) per cell, or NULL for the
 * uniform / per-axis (Ax, Ay, Az) of UniformExchange */
int mm_add_exch(mm_handle* h, const double* A, double Ax, double Ay, double Az);
/* add_dmi(type="bulk")  src/micro/add_field.jl:299-326 (uniform Dx, Dy, Dz, J/m^2) */
int mm_add_dmi_bulk(mm_handle* h, double Dx, double Dy, double Dz);
/* add_dmi(type="interfacial")  src/micro/add_field.jl:327-335 */
int mm_add_dmi_interfacial(mm_handle* h, const double* D, double D_uniform);
/* add_anis  src/micro/add_field.jl:430-465: Ku (J/m^3) per cell or uniform; axis normalised */
int mm_add_anis(mm_handle* h, const double* Ku, double Ku_uniform, double ax, double ay, double az);
/* add_demag(sim; Nx, Ny, Nz)  src/micro/add_field.jl:403-419 -> init_demag
 * src/micro/demag.jl:30-100 (FP64 Newell tensor assembled on the device) */
int mm_add_demag(mm_handle* h, int Nx, int Ny, int Nz);
/* Same, with a caller-supplied real-space tensor (6 x N, order xx yy zz xy
 * xz yz, dimensionless) in place of the Newell assembly. */
int mm_add_demag_tensor(mm_handle* h, const double* tensor_6N);

/* effective_field(sim, spin, t)  src/micro/field.jl:496-505 -> H_aos (3N, A/m) */
int mm_effective_field(mm_handle* h, double* H_aos);
/* Field (3N) and per-cell energy (N) of one term (term.field / term.energy
 * after effective_field(term, sim, spin, t), src/micro/field.jl:1-242);
 * either output may be NULL. */
int mm_term_field(mm_handle* h, int term, double* field_aos, double* energy_cells);
/* compute_system_energy  src/micro/field.jl:520-536: per-term sums (J) in
 * FP64, indexed by mm_term; either output may be NULL. */
int mm_energy(mm_handle* h, double* per_term, double* total);
/* llg_call_back(sim, dm_dt, spin, t)  src/llg/llg.jl:45-59 -> dm/dt AoS */
int mm_llg_rhs(mm_handle* h, double* dmdt_aos);
/* average_m(sim) */
int mm_average_m(mm_handle* h, double* m3);

/* advance_step(sim, ::RungeKutta) x nsteps  src/integrator/rk.jl:23-52 */
int mm_rk4_run(mm_handle* h, double dt, int64_t nsteps);
/* RungeKutta / ModifiedEuler t and nsteps (t = nsteps * dt) */
int mm_rk4_state(mm_handle* h, double* t, int64_t* nsteps);
/* advance_step(sim, ::ModifiedEuler) x nsteps (Heun)  src/integrator/heun.jl:28-49 */
int mm_heun_run(mm_handle* h, double dt, int64_t nsteps);

/* Dormand-Prince (DOPRI54) tolerance, default 1e-6  src/driver.jl:126,134 */
int mm_dopri_set_tol(mm_handle* h, double tol);
/* run_until(sim, t_end)  src/sim.jl:547-574 with integrate_to_time
 * src/integrator/adaptive_rk.jl:168-186 (step control on the device) */
int mm_run_until(mm_handle* h, double t_end, mm_stats* stats);
/* advance_step(sim, ::AdaptiveRK)  src/integrator/adaptive_rk.jl:93-148 */
int mm_advance_step(mm_handle* h, mm_stats* stats);
/* Reset the adaptive integrator (t = 0, step sizes and counters cleared). */
int mm_dopri_reset(mm_handle* h);

/* Adaptive Runge-Kutta methods: Sim(mesh; integrator="DormandPrince" |
 * "BS23" | "CashKarp54" | "Fehlberg54")  src/driver.jl:102-140,
 * src/integrator/adaptive_rk.jl:248-266 */
typedef enum {
  MM_RK_DORMAND_PRINCE = 0,
  MM_RK_BS23 = 1,
  MM_RK_CASH_KARP54 = 2,
  MM_RK_FEHLBERG54 = 3
} mm_rk_method;
/* Select the method used by mm_run_until / mm_advance_step / mm_relax(LLG);
 * resets the adaptive state as a new Sim would (default MM_RK_DORMAND_PRINCE). */
int mm_set_adaptive_method(mm_handle* h, int method);

/* Tile widths (kx columns per block) the autotuner chose for the demag
 * passes 0..4 (0: not tuned / static rule) and their timed milliseconds per
 * launch; measurement hook, no reference counterpart.  Set MMCUDA_AUTOTUNE=0
 * to keep the static rule. */
int mm_demag_tiles(mm_handle* h, int* tiles5, float* ms5);

/* ---- Further terms --------------------------------------------------------
 * Evaluated in the same fused per-cell kernel (a variant compiled with them,
 * so handles without them keep the base kernel).  Array arguments are per
 * cell (N) or NULL for the uniform value; one term of each kind per handle. */
/* add_dmi(sim, (Dx, Dy, Dz), type="bulk") with spatial D: per-axis arrays,
 * harmonic mean per pair, pairs with a zero D dropped
 * (SpatialVectorBulkDMI, src/micro/add_field.jl:299-326, kernels.jl:347-422);
 * takes the place of mm_add_dmi_bulk */
int mm_add_dmi_bulk_spatial(mm_handle* h, const double* Dx, const double* Dy, const double* Dz);
/* add_sot(sim, aj, bj, p): field H = (aj/gamma) m x p + (bj/gamma) p
 * (DFTorqueField, src/micro/add_field.jl:951-966, kernels.jl:619-632) */
int mm_add_sot(mm_handle* h, const double* aj, double aj_uniform, double bj, double px, double py, double pz);
/* add_stt(sim; model=:zhang_li): bJ = b * J per cell (AoS 3N, with the
 * 1/(1+xi^2) factor already applied when b came from (P, Ms)), xi per cell,
 * ft = the current-scale value (the reference's ft(t), taken constant);
 * H = m x f + xi f, f = (ft/gamma) (bJ . nabla) m (src/micro/add_field.jl:1150-1190,
 * kernels.jl:680-739) */
int mm_add_stt_zhang_li(mm_handle* h, const double* bJ, const double* xi, double xi_uniform, double ft);
/* add_stt(sim; model=:slonczewski): J per cell, ft_beta = ft * beta with
 * beta = hbar / (mu0 Ms e tf), Lambda, P, xi, polarisation p
 * (src/micro/add_field.jl:1192-1226, slonczewski_torque_kernel!) */
int mm_add_stt_slonczewski(mm_handle* h, const double* J, double J_uniform, double ft_beta, double Lambda, double P,
                           double xi, double px, double py, double pz);
/* add_thermal_noise(sim, Temp; T0, scaling, k_B): H = eta sqrt(2 alpha k_B
 * scaling (T + T0) / (V gamma dt mu0Ms)) with eta ~ N(0,1) redrawn once per
 * step (src/micro/add_field.jl:734-760, field.jl:244-280, kernels.jl:469-494).
 * eta of step n in cell i is a counter-based draw (Philox-4x32-10 on
 * (i, n) keyed by seed, Box-Muller), so runs are reproducible; dt is used for
 * evaluations outside a step (fixed steps use their own dt, the adaptive
 * stepper its current step). */
int mm_add_thermal_noise(mm_handle* h, const double* T, double T_uniform, double T0, double scaling, double k_B,
                         uint64_t seed, double dt);

/* ---- Adjoint of fixed-step RK4 ------------------------------------------
 * The reference has no differentiation of this path; these give reverse-mode
 * gradients of a loss L(m_T) through nsteps RK4 steps of
 * advance_step(sim, ::RungeKutta) (src/integrator/rk.jl:23-52) with the
 * handle's terms (discrete adjoint: exact for the scheme up to rounding).
 * mm_adjoint_record runs the steps from the current m (advancing it to m_T,
 * like mm_rk4_run) and keeps (m) every ckpt_every steps on the device.
 * mm_adjoint_backward takes dL/dm_T (AoS, 3N) and returns, for any non-NULL
 * output: dL/dm0 (AoS, 3N), dL/dMs per cell (N, Ms in A/m), dL/dKu per cell
 * (N, uniaxial anisotropy) and dL/dD per cell (N, interfacial DMI; for a
 * uniform D the scalar gradient is the sum).  Segments of ckpt_every steps
 * are recomputed forward (3N*ckpt_every state words kept); m is left at m_T.
 * Changing parameters between the two calls is refused (MM_ERR_STATE). */
int mm_adjoint_record(mm_handle* h, double dt, int64_t nsteps, int64_t ckpt_every);
int mm_adjoint_backward(mm_handle* h, const double* dL_dmT, double* g_m0, double* g_Ms, double* g_Ku, double* g_D);

/* ---- OOMMF OVF 2.0 files (src/ovf2.jl) ----------------------------------
 * Data blocks in the AoS cell order of mm_set_m / mm_get_m.  A path without
 * the ".ovf" suffix gets it appended, as save_ovf / read_ovf do.  The mm_ovf_*
 * functions are host-only (no device needed). */
typedef enum { MM_OVF_TEXT = 0, MM_OVF_BINARY4 = 4, MM_OVF_BINARY8 = 8 } mm_ovf_type;
/* save_ovf(ovf::OVF2, fname; type)  src/ovf2.jl:70-153 (mag2ovf :293-343) */
int mm_ovf_write(const char* path, const mm_mesh_desc* mesh, const double* m_aos, int type, const char* title);
/* header fields of read_ovf(fname)  src/ovf2.jl:246-291 (pbc = 0); the
 * Title into title[title_cap] (truncated, NUL-terminated) when title != NULL */
int mm_ovf_read_header(const char* path, mm_mesh_desc* mesh, int* type, char* title, size_t title_cap);
/* data of read_ovf(fname) as float64; ncells must equal xnodes*ynodes*znodes */
int mm_ovf_read(const char* path, double* m_aos, int64_t ncells);
/* save_ovf(sim, fname; type)  src/ovf2.jl:44-62: the handle's m */
int mm_save_ovf(mm_handle* h, const char* path, int type, const char* title);
/* read_ovf(sim, fname)  src/ovf2.jl:197-208: m of the handle from a file
 * whose cell count matches (MM_ERR_ARG "The ovf does not match the sim.mesh") */
int mm_load_ovf(mm_handle* h, const char* path);

/* relax(sim; max_steps, stopping_dmdt)  src/sim.jl:392-490 with the SD
 * driver (src/sd.jl:9-98) or the LLG driver with Dormand-Prince */
int mm_relax(mm_handle* h, int driver, int64_t max_steps, double stopping_dmdt, int64_t* steps_done,
             double* max_dmdt);

/* ---- measurement hooks (the reference times host sections with TimerOutputs,
 * src/MicroMagnetic.jl:7-13; these time device kernels with CUDA events) ---- */
enum mm_kernel {
  MM_K_DEMAG_FWD_X = 0,  /* r2c x pass (m*mu0*Ms -> X) */
  MM_K_DEMAG_FWD_Y = 1,  /* forward y pass (3-D meshes) */
  MM_K_DEMAG_CONV = 2,   /* z (3-D) or y (films) pass with the tensor product */
  MM_K_DEMAG_INV_Y = 3,  /* inverse y pass (3-D meshes) */
  MM_K_DEMAG_INV_X = 4,  /* c2r x pass (-> H_demag) */
  MM_K_RK4_STAGE = 5,    /* fused H_eff + LLG + RK4 stage-2 update */
  MM_K_RK4_STEP = 6,     /* one whole RK4 step (graph) */
  MM_NKERNELS = 7
};
/* Launches `kernel` `reps` times on the handle's stream after one warm-up and
 * reports the mean CUDA-event duration per launch (ms) and the algorithmic
 * HBM bytes one launch must move (compulsory reads + writes).  Kernels that
 * a handle does not use report 0. */
int mm_kernel_time(mm_handle* h, int kernel, int reps, double* ms_per_launch, double* alg_bytes);
/* Number of kernel launches in one RK4 step. */
int mm_rk4_launches_per_step(mm_handle* h, int* launches);

/* ---- batches: several meshes (ensembles, NEB images) stepped together ----
 * The reference evaluates NEB images one after another (src/neb/neb.jl:220-232).
 * A batch captures one RK4 step of every handle (same device, same dt) in one
 * CUDA graph and replays it once per step: the demag passes and stage
 * kernels of meshes that take the shared-memory FFT paths are launched once
 * per pass for all of them (mm_batch_launches), other meshes run as parallel
 * branches of the graph; work
 * queued on the handles before mm_batch_rk4_run precedes the batch and work
 * queued after it follows.  The handles stay owned by the caller and must
 * outlive the batch. */
typedef struct mm_batch mm_batch;
int mm_batch_create(mm_handle* const* handles, int n, mm_batch** out);
int mm_batch_rk4_run(mm_batch* b, double dt, int64_t nsteps);
int mm_batch_get_stream(mm_batch* b, void** stream);
/* Measurement hook (no reference counterpart): kernel launches of one batched
 * RK4 step and the number of handles whose passes were merged into shared
 * launches (each pass kernel launched once for all of them, its blocks
 * looking their mesh up); valid after the first mm_batch_rk4_run.  The other
 * handles run as parallel graph branches.  MMCUDA_BATCH_MERGE=0 disables the
 * merging. */
int mm_batch_launches(mm_batch* b, int* launches_per_step, int* merged_handles);
int mm_batch_destroy(mm_batch* b);

/* ---- energies without device allocation ----------------------------------
 * No counterpart in the reference.  For callers that cannot call cudaMalloc
 * (a host whose pool allocator must own all device memory, a latency-critical
 * path where cudaMalloc's implicit synchronisation is not acceptable, code
 * with no handle): total energies (J, FP64, indexed by mm_term; demag and
 * interfacial DMI entries are 0) of uniform exchange A, bulk DMI D (all
 * axes), uniaxial anisotropy Ku along (ax, ay, az) and a uniform Zeeman field
 * (Hx, Hy, Hz) for m_soa_dev (device, SoA [mx..., my..., mz...], float64) and
 * Ms_dev (device, A/m, float64), written to energies_dev (device, 6 doubles),
 * enqueued on `stream` (cudaStream_t, 0 = legacy default stream).
 * Allocates nothing: the per-block partial sums live in a static device array
 * of the library (3 MiB on every GPU that loads it), so meshes are limited to
 * 2^24 cells (MM_ERR_ARG beyond).  Every call looks the array's device
 * address up in the current context (cudaGetSymbolAddress, a host-side lookup
 * that allocates nothing), so a reset or re-created primary context is
 * followed; the first call on a device (which loads the library's device code
 * and the array) should come before any stream capture.  Calls share the
 * array: calls that overlap on the GPU race. */
int mm_energy_noalloc(const mm_mesh_desc* mesh, const double* m_soa_dev, const double* Ms_dev, double A, double D,
                      double Ku, double ax, double ay, double az, double Hx, double Hy, double Hz,
                      double* energies_dev, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* MMCUDA_H */

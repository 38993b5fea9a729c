// mm_api.cu -- handle/engine and the extern "C" ABI of libmmcuda.so.
//
// A handle (mm_handle) owns an Engine<R> (R = double for MM_FP64, float for
// MM_FP32): the device state, the term parameters, the demag plan and the
// integrator state.  Integration loops are captured once into CUDA graphs
// (one RK4 step; one Dormand-Prince attempt with a device-side step-size
// controller) and replayed; the host only synchronises between batches.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/mmcuda.h"
#include "mm_demag.cuh"
#include "mm_launch.cuh"
#include "mm_persist.cuh"
#include "mm_field.cuh"
#include "mm_integ.cuh"

namespace mm {

static thread_local std::string g_err;

static int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

// Sets the calling thread's last error message (used by translation units
// outside this file) and returns code.
int set_last_error(int code, const char* msg) {
  g_err = msg;
  return code;
}

#define MM_CUDA(call)                                                                          \
  do {                                                                                         \
    cudaError_t e_ = (call);                                                                   \
    if (e_ != cudaSuccess) return fail(MM_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

template <typename R>
__global__ void k_zeeman_accumulate(const double* __restrict__ aos, R* __restrict__ Hz, int64_t N, int replace) {
  const int64_t I = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (I >= N) return;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const R v = static_cast<R>(aos[3 * I + c]);
    Hz[c * N + I] = replace ? v : Hz[c * N + I] + v;
  }
}

template <typename R>
__global__ void k_to_double(const R* __restrict__ a, double* __restrict__ b, int64_t n) {
  const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (i < n) b[i] = static_cast<double>(a[i]);
}

class EngineBase {
 public:
  virtual ~EngineBase() = default;
  virtual int set_Ms(const double* Ms, double uni) = 0;
  virtual int set_m(const double* m) = 0;
  virtual int get_m(double* m) = 0;
  virtual int set_m_f32(const float* m) = 0;
  virtual int get_m_f32(float* m) = 0;
  virtual int set_pins(const uint8_t* p) = 0;
  virtual int set_llg(double alpha, double gamma, int prec) = 0;
  virtual int zeeman(const double* H, double hx, double hy, double hz, bool replace) = 0;
  virtual int add_exch(const double* A, double ax, double ay, double az) = 0;
  virtual int add_dmi_bulk(double dx, double dy, double dz) = 0;
  virtual int add_dmi_interfacial(const double* D, double uni) = 0;
  virtual int add_anis(const double* Ku, double uni, double ax, double ay, double az) = 0;
  virtual int add_dmi_bulk_spatial(const double* Dx, const double* Dy, const double* Dz) = 0;
  virtual int demag_tiles(int* tiles, float* ms) = 0;
  virtual int add_sot(const double* aj, double aj_uni, double bj, double px, double py, double pz) = 0;
  virtual int add_stt_zhang_li(const double* bJ, const double* xi, double xi_uni, double ft) = 0;
  virtual int add_stt_slonczewski(const double* J, double J_uni, double ft_beta, double Lambda, double P, double xi,
                                  double px, double py, double pz) = 0;
  virtual int add_thermal_noise(const double* T, double T_uni, double T0, double scaling, double kB, uint64_t seed,
                                double dt) = 0;
  virtual int add_demag(int Nx, int Ny, int Nz, const double* T6N_host) = 0;
  virtual int effective_field(double* H) = 0;
  virtual int term_field(int term, double* f, double* e) = 0;
  virtual int energy(double* per, double* total) = 0;
  virtual int llg_rhs(double* out) = 0;
  virtual int average_m(double* m3) = 0;
  virtual int rk4_run(double dt, int64_t n) = 0;
  virtual int rk4_state(double* t, int64_t* n) = 0;
  virtual int heun_run(double dt, int64_t n) = 0;
  virtual int dopri_tol(double tol) = 0;
  virtual int run_until(double t_end, mm_stats* st) = 0;
  virtual int advance_step(mm_stats* st) = 0;
  virtual int dopri_reset() = 0;
  virtual int set_method(int method) = 0;
  virtual int adjoint_record(double dt, int64_t nsteps, int64_t ckpt) = 0;
  virtual int adjoint_backward(const double* dLdm, double* gm0, double* gMs, double* gKu, double* gD) = 0;
  virtual int relax(int driver, int64_t max_steps, double stop, int64_t* steps, double* max_dmdt) = 0;
  virtual int kernel_time(int kernel, int reps, double* ms, double* bytes) = 0;
  virtual int rk4_launches() const = 0;
  // batch support: buffers ready, one RK4 step enqueued on the handle's stream,
  // step counters advanced after a batch ran n steps
  virtual int rk4_prepare() = 0;
  virtual void rk4_enqueue(double dt) = 0;
  // every launch of rk4_enqueue is a descriptor kernel (mm_launch.cuh)
  virtual bool rk4_batchable() const = 0;
  virtual bool is_fp32() const = 0;
  virtual void rk4_count(int64_t n, double dt) = 0;
  virtual uint64_t params_version() const = 0;
  virtual cudaStream_t stream() const = 0;
  virtual size_t device_bytes() const = 0;
  int device = 0;
};

template <typename R>
class Engine : public EngineBase {
 public:
  static constexpr bool kF32 = sizeof(R) == 4;

  ~Engine() override {
    cudaSetDevice(device);
    if (rk_graph) cudaGraphExecDestroy(rk_graph);
    if (dp_graph) cudaGraphExecDestroy(dp_graph);
    if (he_graph) cudaGraphExecDestroy(he_graph);
    demag.reset();
    for (void* p : allocs_) cudaFree(p);
    if (st_) cudaStreamDestroy(st_);
  }

  int init(const mm_mesh_desc& d, int dev) {
    device = dev;
    nx = d.nx; ny = d.ny; nz = d.nz; pbc = d.pbc;
    dx = d.dx; dy = d.dy; dz = d.dz;
    N = static_cast<int64_t>(nx) * ny * nz;
    MM_CUDA(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
    const int nb = std::max(stage_blocks(N), stage_grid(nx, ny, nz).nblocks);
    int rc = 0;
    if ((rc = alloc(m, 3 * N)) || (kF32 && (rc = alloc(m_lo, 3 * N))) || (rc = alloc(Ms, N)) ||
        (rc = alloc(nbm, N)) || (rc = alloc(yA, 3 * N)) || (rc = alloc(work, 3 * N)) ||
        (rc = alloc(stage64, 3 * N)) || (rc = alloc(partials, static_cast<int64_t>(nb) * kNTerms + 1024)) ||
        (rc = alloc(scal, 64)))
      return rc;
    return MM_OK;
  }

  cudaStream_t stream() const override { return st_; }
  size_t device_bytes() const override { return bytes_ + (demag ? demag->device_bytes() : 0); }

  // ------------------------------------------------------------ setup --
  int set_Ms(const double* Msh, double uni) override {
    if (Msh) {
      for (int64_t i = 0; i < N; ++i)
        if (std::isnan(Msh[i])) return fail(MM_ERR_NAN, "NaN is given by the input Ms!");
      MM_CUDA(cudaMemcpyAsync(stage64, Msh, sizeof(double) * N, cudaMemcpyHostToDevice, st_));
    } else {
      if (std::isnan(uni)) return fail(MM_ERR_NAN, "NaN is given by the input Ms!");
      std::vector<double> tmp(N, uni);
      MM_CUDA(cudaMemcpyAsync(stage64, tmp.data(), sizeof(double) * N, cudaMemcpyHostToDevice, st_));
      MM_CUDA(cudaStreamSynchronize(st_));
    }
    // stored as mu0*Ms in Tesla (src/sim.jl:138): Ms .*= mu_0 in FP64 then cast
    launch_scalar_to_R<R>(stage64, Ms, N, kMu0, st_);
    launch_nbmask<R>(nx, ny, nz, pbc, Ms, nbm, st_);
    MM_CUDA(cudaStreamSynchronize(st_));
    ms_set = true;
    ++version;
    return MM_OK;
  }

  int set_m(const double* mh) override { return set_m_t(mh); }
  int set_m_f32(const float* mh) override { return set_m_t(mh); }
  int get_m(double* mh) override { return get_m_t(mh); }
  int get_m_f32(float* mh) override { return get_m_t(mh); }

  // host AoS of T (double, or float in the reference's Float32 mode) through
  // the FP64 staging buffer (3N doubles hold 3N floats)
  template <typename T>
  int set_m_t(const T* mh) {
    // NaN check of init_m0 (src/sim.jl:295-297), done by the conversion kernel
    int* flag = reinterpret_cast<int*>(scal + 63);
    T* stage = reinterpret_cast<T*>(stage64);
    MM_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), st_));
    MM_CUDA(cudaMemcpyAsync(stage, mh, sizeof(T) * 3 * N, cudaMemcpyHostToDevice, st_));
    launch_aos_to_soa<R, T>(stage, m, m_lo, N, flag, st_);
    int hflag = 0;
    MM_CUDA(cudaMemcpyAsync(&hflag, flag, sizeof(int), cudaMemcpyDeviceToHost, st_));
    MM_CUDA(cudaStreamSynchronize(st_));
    if (hflag) return fail(MM_ERR_NAN, "NaN is given by the input m0!");
    if (ctrl && hctrl.fsal) {
      // a new state: the stored last-stage derivative of an FSAL method no
      // longer belongs to y_current, so the next attempt evaluates k1
      if (int rc = pull_ctrl()) return rc;
      hctrl.succeed = 0;
      return push_ctrl();
    }
    return MM_OK;
  }

  template <typename T>
  int get_m_t(T* mh) {
    T* stage = reinterpret_cast<T*>(stage64);
    launch_soa_to_aos<R, T>(m, m_lo, stage, N, st_);
    MM_CUDA(cudaMemcpyAsync(mh, stage, sizeof(T) * 3 * N, cudaMemcpyDeviceToHost, st_));
    MM_CUDA(cudaStreamSynchronize(st_));
    return MM_OK;
  }

  int set_pins(const uint8_t* p) override {
    if (!p) {
      pins_on = false;
      ++version;
      return MM_OK;
    }
    int rc;
    if (!pins && (rc = alloc(pins, N))) return rc;
    MM_CUDA(cudaMemcpyAsync(pins, p, N, cudaMemcpyHostToDevice, st_));
    MM_CUDA(cudaStreamSynchronize(st_));
    pins_on = true;
    ++version;
    return MM_OK;
  }

  int set_llg(double a, double g, int prec) override {
    alpha = a;
    gamma = g;
    precession = prec;
    ++version;
    return MM_OK;
  }

  int upload_R(const double* h, R*& dst, int64_t n) {
    int rc;
    if (!dst && (rc = alloc(dst, n))) return rc;
    MM_CUDA(cudaMemcpyAsync(stage64, h, sizeof(double) * n, cudaMemcpyHostToDevice, st_));
    launch_scalar_to_R<R>(stage64, dst, n, 1.0, st_);
    MM_CUDA(cudaStreamSynchronize(st_));
    return MM_OK;
  }

  // an array whose entries are all equal is kept as a scalar
  static bool uniform(const double* a, int64_t n, double& v) {
    v = a[0];
    for (int64_t i = 1; i < n; ++i)
      if (a[i] != v) return false;
    return true;
  }

  int zeeman(const double* H, double hx, double hy, double hz, bool replace) override {
    if (replace) {
      hz_uni[0] = hz_uni[1] = hz_uni[2] = 0.0;
      hz_arr = false;
    }
    if (H) {
      int rc;
      if (!Hz && (rc = alloc(Hz, 3 * N))) return rc;
      MM_CUDA(cudaMemcpyAsync(stage64, H, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, st_));
      k_zeeman_accumulate<R><<<stage_blocks(N), 256, 0, st_>>>(stage64, Hz, N, hz_arr ? 0 : 1);
      MM_CUDA(cudaStreamSynchronize(st_));
      hz_arr = true;
    } else {
      hz_uni[0] += hx;
      hz_uni[1] += hy;
      hz_uni[2] += hz;
    }
    mask |= TB_ZEEMAN;
    ++version;
    return MM_OK;
  }

  int add_exch(const double* Ah, double ax, double ay, double az) override {
    if (mask & TB_EXCH) return fail(MM_ERR_UNSUPPORTED, "one exchange term per handle");
    double v;
    if (Ah && !uniform(Ah, N, v)) {
      int rc;
      if ((rc = upload_R(Ah, A, N))) return rc;
      ex_spatial = true;
    } else {
      if (Ah) ax = ay = az = v;
      ex_A[0] = ax; ex_A[1] = ay; ex_A[2] = az;
      ex_spatial = false;
    }
    mask |= TB_EXCH;
    ++version;
    return MM_OK;
  }

  int add_dmi_bulk(double Dx, double Dy, double Dz) override {
    if (mask & TB_DMI_BULK) return fail(MM_ERR_UNSUPPORTED, "one bulk DMI term per handle");
    bd[0] = Dx; bd[1] = Dy; bd[2] = Dz;
    mask |= TB_DMI_BULK;
    ++version;
    return MM_OK;
  }

  // add_dmi(sim, (Dx, Dy, Dz) arrays / functions, type="bulk")  src/micro/add_field.jl:299-326
  int add_dmi_bulk_spatial(const double* Dxh, const double* Dyh, const double* Dzh) override {
    if (mask & TB_DMI_BULK) return fail(MM_ERR_UNSUPPORTED, "one bulk DMI term per handle");
    if (!Dxh || !Dyh || !Dzh) return fail(MM_ERR_ARG, "spatial bulk DMI needs Dx, Dy and Dz arrays");
    int rc;
    if ((rc = upload_R(Dxh, bDx, N)) || (rc = upload_R(Dyh, bDy, N)) || (rc = upload_R(Dzh, bDz, N))) return rc;
    bulk_spatial = true;
    mask |= TB_DMI_BULK;
    ++version;
    return MM_OK;
  }

  int demag_tiles(int* tiles, float* ms) override {
    if (!demag) return fail(MM_ERR_STATE, "no demag term");
    for (int i = 0; i < 5; ++i) {
      if (tiles) tiles[i] = demag->tile[i];
      if (ms) ms[i] = demag->tile_ms[i];
    }
    return MM_OK;
  }

  // add_sot(sim, aj, bj, p)  src/micro/add_field.jl:951-966 (DFTorqueField)
  int add_sot(const double* ajh, double aj_uni, double bj, double px, double py, double pz) override {
    if (mask & TB_SOT) return fail(MM_ERR_UNSUPPORTED, "one SOT term per handle");
    double v;
    if (ajh && !uniform(ajh, N, v)) {
      int rc;
      if ((rc = upload_R(ajh, sot_aj, N))) return rc;
      sot_spatial = true;
    } else {
      sot_aj_uni = ajh ? v : aj_uni;
    }
    sot_bj = bj;
    sot_p[0] = px; sot_p[1] = py; sot_p[2] = pz;
    mask |= TB_SOT;
    ++version;
    return MM_OK;
  }

  // add_stt(sim; model=:zhang_li, ...)  src/micro/add_field.jl:1150-1190: b*J (AoS 3N), xi
  int add_stt_zhang_li(const double* bJh, const double* xih, double xi_uni, double ft) override {
    if (mask & TB_STT_ZL) return fail(MM_ERR_UNSUPPORTED, "one Zhang-Li torque per handle");
    if (!bJh) return fail(MM_ERR_ARG, "Zhang-Li torque needs the b*J array");
    int rc;
    if (!zl_bJ && (rc = alloc(zl_bJ, 3 * N))) return rc;
    MM_CUDA(cudaMemcpyAsync(stage64, bJh, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, st_));
    launch_aos_to_soa<R>(stage64, zl_bJ, nullptr, N, nullptr, st_);
    double v;
    if (xih && !uniform(xih, N, v)) {
      if ((rc = upload_R(xih, zl_xi, N))) return rc;
      zl_spatial = true;
    } else {
      zl_xi_uni = xih ? v : xi_uni;
    }
    zl_ft = ft;
    MM_CUDA(cudaStreamSynchronize(st_));
    mask |= TB_STT_ZL;
    ++version;
    return MM_OK;
  }

  // add_stt(sim; model=:slonczewski, ...)  src/micro/add_field.jl:1192-1226
  int add_stt_slonczewski(const double* Jh, double J_uni, double ft_beta, double Lambda, double P, double xi,
                          double px, double py, double pz) override {
    if (mask & TB_STT_SL) return fail(MM_ERR_UNSUPPORTED, "one Slonczewski torque per handle");
    double v;
    if (Jh && !uniform(Jh, N, v)) {
      int rc;
      if ((rc = upload_R(Jh, sl_J, N))) return rc;
      sl_spatial = true;
    } else {
      sl_J_uni = Jh ? v : J_uni;
    }
    sl_ftb = ft_beta;
    sl_L2 = Lambda * Lambda;
    sl_P = P;
    sl_xi = xi;
    sl_p[0] = px; sl_p[1] = py; sl_p[2] = pz;
    mask |= TB_STT_SL;
    ++version;
    return MM_OK;
  }

  // add_thermal_noise(sim, Temp; T0, scaling, k_B)  src/micro/add_field.jl:734-760
  int add_thermal_noise(const double* Th, double T_uni, double T0, double scaling, double kB, uint64_t seed,
                        double dt) override {
    if (mask & TB_THERMAL) return fail(MM_ERR_UNSUPPORTED, "one thermal term per handle");
    if (!(dt > 0)) return fail(MM_ERR_ARG, "thermal noise needs dt > 0 for evaluations outside a step");
    int rc;
    double v;
    if (Th && !uniform(Th, N, v)) {
      if ((rc = upload_R(Th, th_T, N))) return rc;
    } else {
      th_T_uni = Th ? v : T_uni;
    }
    if ((rc = alloc(Hth, 3 * N)) || (rc = alloc(th_step, 1))) return rc;
    th_T0 = T0;
    th_scaling = scaling;
    th_kB = kB;
    th_seed = seed;
    th_dt = dt;
    mask |= TB_THERMAL;
    ++version;
    MM_CUDA(cudaStreamSynchronize(st_));
    return MM_OK;
  }

  // the thermal field of the step whose index is *step (fixed-step counter or
  // the adaptive stepper's accepted-step count)
  void enqueue_thermal(const long long* step, const double* dt_dev, double dt, const int* gate) {
    if (!(mask & TB_THERMAL)) return;
    const double c = 2.0 * alpha * th_kB * th_scaling / (dx * dy * dz * gamma);
    launch_thermal<R>(th_seed, step, dt_dev, dt, c, th_T, th_T_uni, th_T0, Ms, Hth, N, gate, st_);
  }

  int add_dmi_interfacial(const double* Dh, double uni) override {
    if (mask & TB_DMI_INTERFACIAL) return fail(MM_ERR_UNSUPPORTED, "one interfacial DMI term per handle");
    double v;
    if (Dh && !uniform(Dh, N, v)) {
      int rc;
      if ((rc = upload_R(Dh, D, N))) return rc;
      id_spatial = true;
    } else {
      id_D = Dh ? v : uni;
      id_spatial = false;
    }
    mask |= TB_DMI_INTERFACIAL;
    ++version;
    return MM_OK;
  }

  int add_anis(const double* Kh, double uni, double ax, double ay, double az) override {
    if (mask & TB_ANIS) return fail(MM_ERR_UNSUPPORTED, "one uniaxial anisotropy term per handle");
    const double lt = std::sqrt(ax * ax + ay * ay + az * az);
    if (!(lt > 0)) return fail(MM_ERR_ARG, "anisotropy axis has zero length");
    // axis normalised at add time (src/micro/add_field.jl:441-444)
    an_u[0] = ax / lt; an_u[1] = ay / lt; an_u[2] = az / lt;
    double v;
    if (Kh && !uniform(Kh, N, v)) {
      int rc;
      if ((rc = upload_R(Kh, Ku, N))) return rc;
      an_spatial = true;
    } else {
      an_K = Kh ? v : uni;
      an_spatial = false;
    }
    mask |= TB_ANIS;
    ++version;
    return MM_OK;
  }

  int add_demag(int Nx, int Ny, int Nz, const double* T6N_host) override {
    if (mask & TB_DEMAG) return fail(MM_ERR_UNSUPPORTED, "one demag term per handle");
    if (Nx < 0 || Ny < 0 || Nz < 0) return fail(MM_ERR_ARG, "macro-PBC image counts must be >= 0");
    auto plan = std::make_unique<DemagPlan<R>>();
    char msg[256] = {0};
    int rc = plan->init(nx, ny, nz, st_, msg, sizeof(msg));
    if (rc == -1) return fail(MM_ERR_ARG, "%s", msg);
    if (rc) return fail(MM_ERR_CUDA, "demag plan allocation failed (%d)", rc);
    double* T = nullptr;
    MM_CUDA(cudaMalloc(&T, sizeof(double) * 6 * N));
    if (T6N_host) {
      cudaMemcpyAsync(T, T6N_host, sizeof(double) * 6 * N, cudaMemcpyHostToDevice, st_);
    } else if ((rc = newell_tensor_device(nx, ny, nz, dx, dy, dz, Nx, Ny, Nz, T, st_))) {
      cudaFree(T);
      return fail(MM_ERR_CUDA, "Newell tensor assembly failed: %s", cudaGetErrorString(static_cast<cudaError_t>(rc)));
    }
    rc = plan->set_tensor(T, st_);
    cudaStreamSynchronize(st_);
    cudaFree(T);
    if (rc) return fail(MM_ERR_CUDA, "demag tensor assembly failed: %s", cudaGetErrorString(static_cast<cudaError_t>(rc)));
    if (!Hd && (rc = alloc(Hd, 3 * N))) return rc;
    // tile widths of the strided passes, timed on this plan's own buffers
    if ((rc = plan->autotune(m, Ms, Hd, st_))) return fail(MM_ERR_CUDA, "demag tile autotuning failed (%d)", rc);
    demag = std::move(plan);
    mask |= TB_DEMAG;
    ++version;
    MM_CUDA(cudaGetLastError());
    return MM_OK;
  }

  FieldArgs<R> fargs(unsigned msk) const {
    FieldArgs<R> a{};
    a.nx = nx; a.ny = ny; a.nz = nz; a.pbc = pbc; a.N = N;
    a.V = static_cast<R>(dx * dy * dz);
    a.Ms = Ms; a.nbm = nbm;
    a.mask = msk & mask;
    if (ex_spatial) {
      a.ex_x = static_cast<R>(2.0 / (dx * dx)); a.ex_y = static_cast<R>(2.0 / (dy * dy)); a.ex_z = static_cast<R>(2.0 / (dz * dz));
      a.A = A;
    } else {
      a.ex_x = static_cast<R>(2 * ex_A[0] / (dx * dx));
      a.ex_y = static_cast<R>(2 * ex_A[1] / (dy * dy));
      a.ex_z = static_cast<R>(2 * ex_A[2] / (dz * dz));
      a.A = nullptr;
    }
    a.bd_x = static_cast<R>(bd[0] / dx); a.bd_y = static_cast<R>(bd[1] / dy); a.bd_z = static_cast<R>(bd[2] / dz);
    a.D_uni = static_cast<R>(id_D);
    a.D = id_spatial ? D : nullptr;
    a.id_x = static_cast<R>(1.0 / dx); a.id_y = static_cast<R>(1.0 / dy);
    a.Ku_uni = static_cast<R>(an_K);
    a.Ku = an_spatial ? Ku : nullptr;
    a.ux = static_cast<R>(an_u[0]); a.uy = static_cast<R>(an_u[1]); a.uz = static_cast<R>(an_u[2]);
    a.hz_x = static_cast<R>(hz_uni[0]); a.hz_y = static_cast<R>(hz_uni[1]); a.hz_z = static_cast<R>(hz_uni[2]);
    a.Hz = hz_arr ? Hz : nullptr;
    a.Hd = Hd;
    a.alpha = static_cast<R>(alpha);
    const double c = -gamma / (1 + alpha * alpha);  // llg.jl:24
    a.llg_c = static_cast<R>(c);
    a.llg_c_lo = static_cast<R>(c - static_cast<double>(a.llg_c));
    a.precession = precession;
    a.pins = pins_on ? pins : nullptr;
    ExtraTerms<R>& x = a.x;
    x.bD[0] = bulk_spatial ? bDx : nullptr;
    x.bD[1] = bulk_spatial ? bDy : nullptr;
    x.bD[2] = bulk_spatial ? bDz : nullptr;
    x.inv_d[0] = static_cast<R>(1.0 / dx); x.inv_d[1] = static_cast<R>(1.0 / dy); x.inv_d[2] = static_cast<R>(1.0 / dz);
    x.sot_aj = sot_spatial ? sot_aj : nullptr;
    x.sot_aj_uni = static_cast<R>(sot_aj_uni);
    x.sot_b = static_cast<R>(sot_bj / gamma);
    x.sot_inv_g = static_cast<R>(1.0 / gamma);
    for (int c3 = 0; c3 < 3; ++c3) {
      x.sot_p[c3] = static_cast<R>(sot_p[c3]);
      x.sl_p[c3] = static_cast<R>(sl_p[c3]);
    }
    x.zl_bJ = zl_bJ;
    x.zl_xi = zl_spatial ? zl_xi : nullptr;
    x.zl_xi_uni = static_cast<R>(zl_xi_uni);
    x.zl_ut = static_cast<R>(zl_ft / gamma);
    x.sl_J = sl_spatial ? sl_J : nullptr;
    x.sl_J_uni = static_cast<R>(sl_J_uni);
    x.sl_ftb = static_cast<R>(sl_ftb);
    x.sl_L2 = static_cast<R>(sl_L2);
    x.sl_P = static_cast<R>(sl_P);
    x.sl_xi = static_cast<R>(sl_xi);
    x.Hth = Hth;
    return a;
  }

  // ------------------------------------------------------ evaluation --
  void enqueue_field(const R* y, R* out, unsigned msk, R* ecell) {
    if (msk & mask & TB_THERMAL) enqueue_thermal(th_step, nullptr, th_dt, nullptr);
    if ((msk & mask & TB_DEMAG) && demag) demag->apply(y, Ms, Hd, st_);
    StageArgs<R> s{};
    s.out = out;
    s.ecell = ecell;
    launch_stage<R>(SM_FIELD, fargs(msk), y, s, st_);
  }

  void enqueue_rhs(const R* y, R* out, bool thermal_draw = true) {
    if (thermal_draw) enqueue_thermal(th_step, nullptr, th_dt, nullptr);
    if ((mask & TB_DEMAG) && demag) demag->apply(y, Ms, Hd, st_);
    StageArgs<R> s{};
    s.out = out;
    launch_stage<R>(SM_RHS, fargs(~0u), y, s, st_);
  }

  int need_ms() const { return ms_set ? MM_OK : fail(MM_ERR_STATE, "set_Ms must be called first"); }

  int download_aos(const R* soa, double* out) {
    launch_soa_to_aos<R>(soa, nullptr, stage64, N, st_);
    MM_CUDA(cudaMemcpyAsync(out, stage64, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, st_));
    MM_CUDA(cudaStreamSynchronize(st_));
    return MM_OK;
  }

  int effective_field(double* H) override {
    if (int rc = need_ms()) return rc;
    enqueue_field(m, work, ~0u, nullptr);
    MM_CUDA(cudaGetLastError());
    if (!H) return MM_OK;
    return download_aos(work, H);
  }

  int term_field(int term, double* f, double* e) override {
    if (int rc = need_ms()) return rc;
    if (term < 0 || term >= kNTermIds) return fail(MM_ERR_ARG, "bad term index %d", term);
    if (!(mask & (1u << term))) return fail(MM_ERR_ARG, "term %d was not added", term);
    int rc;
    if (!ecell && (rc = alloc(ecell, N))) return rc;
    enqueue_field(m, work, 1u << term, ecell);
    MM_CUDA(cudaGetLastError());
    if (e) {
      k_to_double<R><<<stage_blocks(N), 256, 0, st_>>>(ecell, stage64, N);
      MM_CUDA(cudaMemcpyAsync(e, stage64, sizeof(double) * N, cudaMemcpyDeviceToHost, st_));
      MM_CUDA(cudaStreamSynchronize(st_));
    }
    if (f) return download_aos(work, f);
    return MM_OK;
  }

  int energy(double* per, double* total) override {
    if (int rc = need_ms()) return rc;
    enqueue_thermal(th_step, nullptr, th_dt, nullptr);
    if ((mask & TB_DEMAG) && demag) demag->apply(m, Ms, Hd, st_);
    StageArgs<R> s{};
    s.partials = partials;
    launch_stage<R>(SM_ENERGY, fargs(~0u), m, s, st_);
    launch_reduce_sum(partials, stage_grid(nx, ny, nz).nblocks, kNTerms, scal, st_);
    double e[kNTerms];
    MM_CUDA(cudaMemcpyAsync(e, scal, sizeof(e), cudaMemcpyDeviceToHost, st_));
    MM_CUDA(cudaStreamSynchronize(st_));
    double t = 0.0;
    for (int i = 0; i < kNTerms; ++i) {
      if (!(mask & (1u << i))) e[i] = 0.0;
      t += e[i];
      if (per) per[i] = e[i];
    }
    if (total) *total = t;
    return MM_OK;
  }

  int llg_rhs(double* out) override {
    if (int rc = need_ms()) return rc;
    enqueue_rhs(m, work);
    MM_CUDA(cudaGetLastError());
    return download_aos(work, out);
  }

  int average_m(double* m3) override {
    launch_average_m<R>(m, m_lo, N, partials, scal, st_);
    double s[3];
    MM_CUDA(cudaMemcpyAsync(s, scal, sizeof(s), cudaMemcpyDeviceToHost, st_));
    MM_CUDA(cudaStreamSynchronize(st_));
    for (int c = 0; c < 3; ++c) m3[c] = s[c] / static_cast<double>(N);
    return MM_OK;
  }

  // -------------------------------------------------------------- RK4 --
  void enqueue_rk4_step(double h) {
    const FieldArgs<R> fa = fargs(~0u);
    enqueue_thermal(th_step, nullptr, h, nullptr);
    for (int s = 1; s <= 4; ++s) {
      // stage inputs ping-pong so that no kernel overwrites a field it reads
      const R* yin = s == 1 ? m : (s == 3 ? yB : yA);
      R* ynext = (s == 2) ? yB : yA;
      if ((mask & TB_DEMAG) && demag) demag->apply(yin, Ms, Hd, st_);
      StageArgs<R> sa{};
      sa.m = m;
      sa.m_lo = m_lo;
      sa.acc = acc;
      sa.ynext = ynext;
      sa.h = h;
      sa.stage = s;
      launch_stage<R>(SM_RK4, fa, yin, sa, st_);
    }
    if (mask & TB_THERMAL) launch_count_step(th_step, st_);
  }

  // advance_step(sim, ::ModifiedEuler) x nsteps  src/integrator/heun.jl:28-49
  void enqueue_heun_step(double h) {
    const FieldArgs<R> fa = fargs(~0u);
    enqueue_thermal(th_step, nullptr, h, nullptr);
    for (int st = 1; st <= 2; ++st) {
      const R* yin = st == 1 ? m : yA;
      if ((mask & TB_DEMAG) && demag) demag->apply(yin, Ms, Hd, st_);
      StageArgs<R> sa{};
      sa.m = m;
      sa.m_lo = m_lo;
      sa.acc = acc;
      sa.ynext = yA;
      sa.h = h;
      sa.stage = st;
      sa.scheme = 1;
      launch_stage<R>(SM_RK4, fa, yin, sa, st_);
    }
    if (mask & TB_THERMAL) launch_count_step(th_step, st_);
  }

  int heun_run(double dt, int64_t n) override {
    if (int rc = need_ms()) return rc;
    if (n < 0 || !(dt > 0)) return fail(MM_ERR_ARG, "heun: need dt > 0 and nsteps >= 0");
    th_dt = dt;
    int rc;
    if (!acc && (rc = alloc(acc, 3 * N))) return rc;
    if (!he_graph || he_dt != dt || he_version != version) {
      if (he_graph) cudaGraphExecDestroy(he_graph);
      he_graph = nullptr;
      cudaGraph_t g;
      MM_CUDA(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
      enqueue_heun_step(dt);
      MM_CUDA(cudaStreamEndCapture(st_, &g));
      MM_CUDA(cudaGraphInstantiate(&he_graph, g, 0));
      cudaGraphDestroy(g);
      he_dt = dt;
      he_version = version;
    }
    for (int64_t i = 0; i < n; ++i) MM_CUDA(cudaGraphLaunch(he_graph, st_));
    rk_n += n;
    rk_t = static_cast<double>(rk_n) * dt;  // integrator.t = nsteps * h (heun.jl:45)
    MM_CUDA(cudaGetLastError());
    return MM_OK;
  }
  cudaGraphExec_t he_graph = nullptr;
  double he_dt = 0.0;
  uint64_t he_version = 0;

  // Small meshes run their RK4 steps in the persistent step kernel
  // (mm_persist.cu): one cooperative launch for up to 256 steps instead of
  // one graph of about 4 x 6 kernels a step.
  static constexpr int64_t kPersistCells = int64_t(1) << 17;
  PersistProgram persist_;
  double ps_dt = 0.0;
  uint64_t ps_version = ~0ull;

  int rk4_run_persistent(double dt, int64_t n) {
    if (!persist_.ready() || ps_dt != dt || ps_version != version) {
      std::vector<std::vector<LaunchRec>> recs(1);
      LaunchRecorder rec;
      launch_recorder() = &rec;
      enqueue_rk4_step(dt);
      launch_recorder() = nullptr;
      recs[0] = std::move(rec.recs);
      char msg[256] = {0};
      const int rc = persist_.build(recs, kF32, msg, sizeof(msg));
      if (rc == -1) return -1;  // a kernel without a persistent form: the caller takes the graph
      if (rc) return fail(MM_ERR_CUDA, "%s", msg);
      ps_dt = dt;
      ps_version = version;
    }
    const int rc = persist_.run(n, st_);
    if (rc == 1) return fail(MM_ERR_TIMEOUT, "persistent RK4 step: a grid-barrier wait ran out");
    if (rc) return fail(MM_ERR_CUDA, "persistent RK4 step: %s", cudaGetErrorString(cudaGetLastError()));
    rk_n += n;
    rk_t = static_cast<double>(rk_n) * dt;
    return MM_OK;
  }

  int rk4_run(double dt, int64_t n) override {
    if (int rc = need_ms()) return rc;
    if (n < 0 || !(dt > 0)) return fail(MM_ERR_ARG, "rk4: need dt > 0 and nsteps >= 0");
    th_dt = dt;
    int rc;
    if (!acc && (rc = alloc(acc, 3 * N))) return rc;
    if (!yB && (rc = alloc(yB, 3 * N))) return rc;
    if (n > 0 && persist_enabled() && N <= kPersistCells && rk4_batchable()) {
      const int prc = rk4_run_persistent(dt, n);
      if (prc != -1) return prc;
    }
    if (!rk_graph || rk_dt != dt || rk_version != version) {
      if (rk_graph) cudaGraphExecDestroy(rk_graph);
      rk_graph = nullptr;
      cudaGraph_t g;
      MM_CUDA(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
      enqueue_rk4_step(dt);
      MM_CUDA(cudaStreamEndCapture(st_, &g));
      MM_CUDA(cudaGraphInstantiate(&rk_graph, g, 0));
      cudaGraphDestroy(g);
      rk_dt = dt;
      rk_version = version;
    }
    for (int64_t i = 0; i < n; ++i) MM_CUDA(cudaGraphLaunch(rk_graph, st_));
    rk_n += n;
    rk_t = static_cast<double>(rk_n) * dt;  // integrator.t = nsteps * h (rk.jl:50)
    MM_CUDA(cudaGetLastError());
    return MM_OK;
  }

  int rk4_state(double* t, int64_t* n) override {
    if (t) *t = rk_t;
    if (n) *n = rk_n;
    return MM_OK;
  }

  int rk4_prepare() override {
    if (int rc = need_ms()) return rc;
    int rc;
    if (!acc && (rc = alloc(acc, 3 * N))) return rc;
    if (!yB && (rc = alloc(yB, 3 * N))) return rc;
    return MM_OK;
  }
  void rk4_enqueue(double dt) override { enqueue_rk4_step(dt); }
  bool is_fp32() const override { return kF32; }
  bool rk4_batchable() const override {
    if (mask & TB_THERMAL) return false;
    if (!stage_descriptor_used<R>(fargs(~0u))) return false;
    return !((mask & TB_DEMAG) && demag) || demag->batchable();
  }
  void rk4_count(int64_t n, double dt) override {
    rk_n += n;
    rk_t = static_cast<double>(rk_n) * dt;
  }
  uint64_t params_version() const override { return version; }

  int rk4_launches() const override {
    const int passes = ((mask & TB_DEMAG) && demag) ? demag->launches_per_apply() : 0;
    return 4 * (passes + 1);
  }

  // Compulsory bytes of one fused RK4 stage-2 kernel: y, Ms, [H_demag], m_n, acc
  // read; acc and the next stage input written (the canonical schedule), plus
  // one word per spatially varying parameter array and the Zeeman array.
  double stage_bytes() const {
    double words = 16.0 + (((mask & TB_DEMAG) && demag) ? 3.0 : 0.0);
    if ((mask & TB_EXCH) && ex_spatial) words += 1.0;
    if ((mask & TB_DMI_INTERFACIAL) && id_spatial) words += 1.0;
    if ((mask & TB_ANIS) && an_spatial) words += 1.0;
    if ((mask & TB_ZEEMAN) && hz_arr) words += 3.0;
    return words * sizeof(R) * static_cast<double>(N);
  }

  int kernel_time(int kernel, int reps, double* ms, double* bytes) override {
    if (int rc = need_ms()) return rc;
    if (kernel < 0 || kernel >= MM_NKERNELS || reps < 1) return fail(MM_ERR_ARG, "bad kernel id or reps");
    int rc;
    if (!acc && (rc = alloc(acc, 3 * N))) return rc;
    if (!yB && (rc = alloc(yB, 3 * N))) return rc;
    const bool dm = (mask & TB_DEMAG) && demag;
    double b = 0.0;
    if (kernel <= MM_K_DEMAG_INV_X) {
      b = dm ? demag->pass_bytes(kernel) : 0.0;
    } else if (kernel == MM_K_RK4_STAGE) {
      b = stage_bytes();
    } else {
      b = 4.0 * stage_bytes() - 4.0 * 3.0 * sizeof(R) * N;  // stage 1 reads no m_n/acc, stage 4 writes no y
      if (dm)
        for (int p = 0; p < 5; ++p) b += 4.0 * demag->pass_bytes(p);
    }
    if (bytes) *bytes = b;
    if (ms) *ms = 0.0;
    if (b == 0.0) return MM_OK;
    // the whole-step timing runs on the live state: save and restore it
    R* save = nullptr;
    R* save_lo = nullptr;
    const int64_t n0 = rk_n;
    const double t0 = rk_t;
    if (kernel == MM_K_RK4_STEP) {
      if ((rc = scratch(save, save_lo))) return rc;
      MM_CUDA(cudaMemcpyAsync(save, m, sizeof(R) * 3 * N, cudaMemcpyDeviceToDevice, st_));
      if (m_lo) MM_CUDA(cudaMemcpyAsync(save_lo, m_lo, sizeof(R) * 3 * N, cudaMemcpyDeviceToDevice, st_));
      if ((rc = rk4_run(rk_dt > 0 ? rk_dt : 1e-15, 0))) return rc;  // make sure the step graph exists
    }
    auto launch = [&]() {
      if (kernel <= MM_K_DEMAG_INV_X) {
        demag->launch_pass(kernel, yA, Ms, Hd, st_);
      } else if (kernel == MM_K_RK4_STAGE) {
        StageArgs<R> sa{};
        sa.m = m; sa.m_lo = m_lo; sa.acc = acc; sa.ynext = yB; sa.h = 1e-15; sa.stage = 2;
        launch_stage<R>(SM_RK4, fargs(~0u), yA, sa, st_);
      } else {
        cudaGraphLaunch(rk_graph, st_);
      }
    };
    launch();  // warm-up
    cudaEvent_t e0, e1;
    MM_CUDA(cudaEventCreate(&e0));
    MM_CUDA(cudaEventCreate(&e1));
    MM_CUDA(cudaEventRecord(e0, st_));
    for (int r = 0; r < reps; ++r) launch();
    MM_CUDA(cudaEventRecord(e1, st_));
    MM_CUDA(cudaEventSynchronize(e1));
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (kernel == MM_K_RK4_STEP) {
      MM_CUDA(cudaMemcpyAsync(m, save, sizeof(R) * 3 * N, cudaMemcpyDeviceToDevice, st_));
      if (m_lo) MM_CUDA(cudaMemcpyAsync(m_lo, save_lo, sizeof(R) * 3 * N, cudaMemcpyDeviceToDevice, st_));
      MM_CUDA(cudaStreamSynchronize(st_));
      rk_n = n0;
      rk_t = t0;
    }
    MM_CUDA(cudaGetLastError());
    if (ms) *ms = static_cast<double>(t) / reps;
    return MM_OK;
  }

  int scratch(R*& a, R*& b) {
    int rc;
    if (!save_ && (rc = alloc(save_, 3 * N))) return rc;
    if (kF32 && !save_lo_ && (rc = alloc(save_lo_, 3 * N))) return rc;
    a = save_;
    b = save_lo_;
    return MM_OK;
  }
  R* save_ = nullptr;
  R* save_lo_ = nullptr;

  // ---------------------------------------------------- Dormand-Prince --
  int dopri_alloc() {
    int rc;
    if (ctrl) return MM_OK;
    for (int i = 0; i < 7; ++i)
      if ((rc = alloc(ks[i], 3 * N))) return rc;
    if ((rc = alloc(yB, 3 * N)) || (rc = alloc(yn, 3 * N)) || (kF32 && (rc = alloc(yn_lo, 3 * N))) ||
        (rc = alloc(ctrl, 1)))
      return rc;
    fresh_ctrl();
    MM_CUDA(cudaMemcpyAsync(ctrl, &hctrl, sizeof(DopriCtrl), cudaMemcpyHostToDevice, st_));
    MM_CUDA(cudaStreamSynchronize(st_));
    return MM_OK;
  }

  // AdaptiveRK(n_total, method, rhs_fun, tol) state  src/integrator/adaptive_rk.jl:57-87
  void fresh_ctrl() {
    const RkTableau& tb = rk_tableau(method);
    hctrl = DopriCtrl{};
    hctrl.tol = tol;
    hctrl.inner = 1;
    hctrl.fsal = tb.fsal;
    hctrl.order = tb.order_emb;
    hctrl.nstage = tb.nstage;
  }

  // Sim(mesh; integrator=...) with an adaptive method  src/driver.jl:102-140
  int set_method(int mth) override {
    if (mth < 0 || mth >= RK_NMETHODS) return fail(MM_ERR_ARG, "unknown adaptive method %d", mth);
    method = mth;
    if (dp_graph) cudaGraphExecDestroy(dp_graph);
    dp_graph = nullptr;
    if (!ctrl) return MM_OK;
    fresh_ctrl();
    return push_ctrl();
  }
  int method = RK_DOPRI54;

  // stage s of one attempt reads the output of stage s-1 (m for s = 1) and
  // writes the next input to yA / yB alternately, the solution to yn
  void enqueue_dopri_attempt() {
    const FieldArgs<R> fa = fargs(~0u);
    const RkTableau& tb = rk_tableau(method);
    auto target_of = [&](int s) { return s == tb.sol ? yn : (s % 2 == 1 ? yA : yB); };
    // the thermal field of the accepted-step count, as the reference redraws
    // it when integrator.nsteps advances (src/micro/field.jl:250-253)
    enqueue_thermal(&ctrl->nsteps, &ctrl->step, 0.0, &ctrl->active);
    for (int s = 1; s <= tb.nstage; ++s) {
      const R* yin = s == 1 ? m : target_of(s - 1);
      R* target = s <= tb.sol ? target_of(s) : nullptr;
      if ((mask & TB_DEMAG) && demag) demag->apply(yin, Ms, Hd, st_, s == 1 ? &ctrl->eval1 : &ctrl->active);
      StageArgs<R> sa{};
      sa.method = method;
      sa.m = m;
      sa.m_lo = m_lo;
      sa.ynext = target;
      sa.ynext_lo = yn_lo;
      for (int i = 0; i < 7; ++i) sa.k[i] = ks[i];
      sa.stage = s;
      sa.ctrl = ctrl;
      sa.partials = partials;
      launch_stage<R>(SM_DOPRI, fa, yin, sa, st_);
    }
    launch_dopri_control(ctrl, partials, stage_grid(nx, ny, nz).nblocks, st_);
    launch_dopri_accept<R>(ctrl, m, m_lo, yn, yn_lo, 3 * N, st_);
  }

  int pull_ctrl() {
    MM_CUDA(cudaMemcpyAsync(&hctrl, ctrl, sizeof(DopriCtrl), cudaMemcpyDeviceToHost, st_));
    MM_CUDA(cudaStreamSynchronize(st_));
    return MM_OK;
  }
  int push_ctrl() {
    MM_CUDA(cudaMemcpyAsync(ctrl, &hctrl, sizeof(DopriCtrl), cudaMemcpyHostToDevice, st_));
    return MM_OK;
  }

  // compute_initial_step(sim, integrator, 1e-12)  adaptive_rk.jl:151-165
  int initial_step(double& out) {
    // the right-hand side sees integrator.step = 1e-15 (adaptive_rk.jl:154)
    enqueue_thermal(&ctrl->nsteps, nullptr, 1e-15, nullptr);
    enqueue_rhs(m, work, false);
    launch_absmax<R>(work, 3 * N, partials, scal, st_);
    double mx = 0.0;
    MM_CUDA(cudaMemcpyAsync(&mx, scal, sizeof(double), cudaMemcpyDeviceToHost, st_));
    MM_CUDA(cudaStreamSynchronize(st_));
    const double order_main = rk_tableau(method).order_main;
    const double r_step = mx / (0.824 * std::pow(hctrl.tol, 1.0 / order_main));
    double abs_step = 1e-12, tmp = 1e-12;
    if (abs_step * r_step > 0.001) tmp = 0.001 / r_step;
    hctrl.nfevals += 1;
    out = std::min(abs_step, tmp);
    return MM_OK;
  }

  int run_attempts() {
    if (!dp_graph || dp_version != version) {
      if (dp_graph) cudaGraphExecDestroy(dp_graph);
      dp_graph = nullptr;
      cudaGraph_t g;
      MM_CUDA(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
      enqueue_dopri_attempt();
      MM_CUDA(cudaStreamEndCapture(st_, &g));
      MM_CUDA(cudaGraphInstantiate(&dp_graph, g, 0));
      cudaGraphDestroy(g);
      dp_version = version;
    }
    int batch = 1;
    const long long a0 = hctrl.attempts;
    for (int guard = 0; guard < 1 << 24; ++guard) {
      for (int b = 0; b < batch; ++b) MM_CUDA(cudaGraphLaunch(dp_graph, st_));
      if (int rc = pull_ctrl()) return rc;
      if (!hctrl.active) break;
      batch = std::min(batch * 2, 64);
      (void)a0;
    }
    MM_CUDA(cudaGetLastError());
    return MM_OK;
  }

  static void fill_stats(const DopriCtrl& c, mm_stats* s) {
    if (!s) return;
    s->t = c.t;
    s->step = c.step;
    s->step_next = c.step_next;
    s->nsteps = c.nsteps;
    s->nfevals = c.nfevals;
    s->attempts = c.attempts;
    s->rejected = c.rejected;
    s->status = c.status;
  }

  int dopri_tol(double t) override {
    if (!(t > 0)) return fail(MM_ERR_ARG, "tolerance must be > 0");
    tol = t;
    if (ctrl) {
      if (int rc = pull_ctrl()) return rc;
      hctrl.tol = t;
      return push_ctrl();
    }
    return MM_OK;
  }

  int dopri_reset() override {
    if (!ctrl) return MM_OK;
    fresh_ctrl();
    return push_ctrl();
  }

  int finish_status() {
    if (hctrl.status == 1) return fail(MM_ERR_NAN, "NaN error detected in the adaptive step (t = %g)", hctrl.t);
    if (hctrl.status == 2) return fail(MM_ERR_NOCONVERGE, "Too many inner steps, system may not converge (t = %g)", hctrl.t);
    return MM_OK;
  }

  int run_until(double t_end, mm_stats* st) override {
    if (int rc = need_ms()) return rc;
    if (int rc = dopri_alloc()) return rc;
    if (int rc = pull_ctrl()) return rc;
    hctrl.status = 0;
    if (t_end < hctrl.t - hctrl.step || t_end == hctrl.t || !(hctrl.t < t_end)) {
      fill_stats(hctrl, st);
      return MM_OK;
    }
    // integrate_to_time: clip to the end time, then advance_step's init
    if (hctrl.step_next + hctrl.t > t_end) hctrl.step_next = t_end - hctrl.t;
    if (hctrl.step_next <= 0) {
      double s0;
      if (int rc = initial_step(s0)) return rc;
      hctrl.step_next = s0;
    }
    hctrl.step = hctrl.step_next;
    hctrl.t_final = t_end;
    hctrl.inner = 1;
    hctrl.single = 0;
    hctrl.active = 1;
    hctrl.eval1 = (hctrl.fsal && hctrl.succeed) ? 0 : 1;
    if (int rc = push_ctrl()) return rc;
    if (int rc = run_attempts()) return rc;
    fill_stats(hctrl, st);
    return finish_status();
  }

  int advance_step(mm_stats* st) override {
    if (int rc = need_ms()) return rc;
    if (int rc = dopri_alloc()) return rc;
    if (int rc = pull_ctrl()) return rc;
    hctrl.status = 0;
    if (hctrl.step_next <= 0) {
      double s0;
      if (int rc = initial_step(s0)) return rc;
      hctrl.step_next = s0;
    }
    hctrl.step = hctrl.step_next;
    hctrl.t_final = INFINITY;
    hctrl.inner = 1;
    hctrl.single = 1;
    hctrl.active = 1;
    hctrl.eval1 = (hctrl.fsal && hctrl.succeed) ? 0 : 1;
    if (int rc = push_ctrl()) return rc;
    if (int rc = run_attempts()) return rc;
    fill_stats(hctrl, st);
    return finish_status();
  }

  // ------------------------------------------------------------ relax --
  int relax(int driver, int64_t max_steps, double stop, int64_t* steps, double* max_dmdt_out) override {
    if (int rc = need_ms()) return rc;
    int rc;
    if (!pre && (rc = alloc(pre, 3 * N))) return rc;
    const double time_factor = 2.21e5 / 2;
    const double dmdt_factor = (2 * kPi / 360) * 1e9;
    double max_dmdt = 0.0;
    int64_t i = 1;
    if (driver == MM_DRIVER_SD) {
      if (!gk && (rc = alloc(gk, 3 * N))) return rc;
      if (!sd && (rc = alloc(sd, 1))) return rc;
      if (kF32) MM_CUDA(cudaMemsetAsync(m_lo, 0, sizeof(R) * 3 * N, st_));
      SdState hs{0.0, 1.0, 1e-10, sd_steps};
      MM_CUDA(cudaMemcpyAsync(sd, &hs, sizeof(hs), cudaMemcpyHostToDevice, st_));
      const int nb = stage_blocks(N);
      for (; i <= max_steps; ++i) {
        enqueue_field(m, work, ~0u, nullptr);
        launch_sd_gk<R>(m, pre, work, gk, N, sd_steps == 0 ? 1 : 0, partials, st_);
        launch_sd_tau(sd, partials, nb, st_);
        launch_sd_update<R>(m, pre, work, gk, pins_on ? pins : nullptr, sd, N, st_);
        launch_sd_count(sd, st_);
        ++sd_steps;
        if (sd_steps % 10 == 0) launch_normalise<R>(m, N, st_);
        launch_max_dm<R>(m, nullptr, pre, nullptr, N, partials + 3 * nb, scal, st_);
        double out[2];
        MM_CUDA(cudaMemcpyAsync(&out[0], scal, sizeof(double), cudaMemcpyDeviceToHost, st_));
        MM_CUDA(cudaMemcpyAsync(&out[1], &sd->tau, sizeof(double), cudaMemcpyDeviceToHost, st_));
        MM_CUDA(cudaStreamSynchronize(st_));
        const double step_size = out[1] / time_factor;
        max_dmdt = out[0] / step_size;
        if (max_dmdt < stop * dmdt_factor) break;
      }
    } else {
      if ((rc = dopri_alloc())) return rc;
      for (; i <= max_steps; ++i) {
        MM_CUDA(cudaMemcpyAsync(pre, m, sizeof(R) * 3 * N, cudaMemcpyDeviceToDevice, st_));
        if (kF32) {
          if (!pre_lo && (rc = alloc(pre_lo, 3 * N))) return rc;
          MM_CUDA(cudaMemcpyAsync(pre_lo, m_lo, sizeof(R) * 3 * N, cudaMemcpyDeviceToDevice, st_));
        }
        mm_stats s;
        rc = advance_step(&s);
        if (rc && rc != MM_ERR_NOCONVERGE && rc != MM_ERR_NAN) return rc;
        launch_max_dm<R>(m, m_lo, pre, pre_lo, N, partials, scal, st_);
        double dm = 0.0;
        MM_CUDA(cudaMemcpyAsync(&dm, scal, sizeof(double), cudaMemcpyDeviceToHost, st_));
        MM_CUDA(cudaStreamSynchronize(st_));
        max_dmdt = dm / hctrl.step;
        if (max_dmdt < stop * dmdt_factor) break;
      }
    }
    if (steps) *steps = i > max_steps ? max_steps : i;
    if (max_dmdt_out) *max_dmdt_out = max_dmdt / dmdt_factor;
    MM_CUDA(cudaGetLastError());
    return MM_OK;
  }

  // ---------------------------------------------------------- adjoint --
  // Reverse mode through nsteps fixed RK4 steps with checkpointing: the
  // recorded run keeps (m, m_lo) every `ck` steps; the backward sweep
  // recomputes one segment forward at a time (states of the segment kept),
  // then walks it backwards, recomputing each step's stage inputs, demag
  // fields and slopes before the stage VJPs.
  int adjoint_record(double dt, int64_t n, int64_t ck) override {
    if (int rc = need_ms()) return rc;
    if (n < 1 || !(dt > 0) || ck < 1) return fail(MM_ERR_ARG, "adjoint: need dt > 0, nsteps >= 1, ckpt_every >= 1");
    if (mask & kExtraBits)
      return fail(MM_ERR_UNSUPPORTED, "adjoint: torque and thermal terms are not differentiated");
    const int64_t nck = (n + ck - 1) / ck;
    MM_CUDA(cudaStreamSynchronize(st_));
    adj_release();
    int rc;
    if ((rc = alloc(adj_ck, nck * 3 * N)) || (kF32 && (rc = alloc(adj_ck_lo, nck * 3 * N)))) return rc;
    adj_n = n;
    adj_every = ck;
    adj_nck = nck;
    adj_dt = dt;
    for (int64_t s = 0; s < n; ++s) {
      if (s % ck == 0) {
        const int64_t slot = s / ck;
        MM_CUDA(cudaMemcpyAsync(adj_ck + slot * 3 * N, m, sizeof(R) * 3 * N, cudaMemcpyDeviceToDevice, st_));
        if (kF32)
          MM_CUDA(cudaMemcpyAsync(adj_ck_lo + slot * 3 * N, m_lo, sizeof(R) * 3 * N, cudaMemcpyDeviceToDevice, st_));
      }
      if ((rc = rk4_run(dt, 1))) return rc;
    }
    adj_version = version;
    MM_CUDA(cudaStreamSynchronize(st_));
    return MM_OK;
  }

  void adj_release() {
    release(adj_ck, adj_nck * 3 * N);
    release(adj_ck_lo, adj_nck * 3 * N);
    adj_n = adj_nck = 0;
  }

  int adj_buffers() {
    int rc;
    const int64_t n3 = 3 * N;
    if (adj_seg_cap < adj_every) {
      release(adj_seg, adj_seg_cap * n3);
      release(adj_seg_lo, adj_seg_cap * n3);
      adj_seg_cap = 0;
      if ((rc = alloc(adj_seg, adj_every * n3)) || (kF32 && (rc = alloc(adj_seg_lo, adj_every * n3)))) return rc;
      adj_seg_cap = adj_every;
    }
    if (adj_lam) return MM_OK;
    for (int i = 0; i < 4; ++i)
      if ((rc = alloc(adj_Y[i], n3)) || (rc = alloc(adj_k[i], n3)) || (rc = alloc(adj_Hd[i], n3))) return rc;
    if ((rc = alloc(adj_q, n3)) || (rc = alloc(adj_w, n3)) || (rc = alloc(adj_Hdw, n3)) || (rc = alloc(adj_a, n3)) ||
        (rc = alloc(adj_mu, n3)) || (rc = alloc(adj_g, n3)) || (rc = alloc(adj_gMs, N)) || (rc = alloc(adj_gKu, N)) ||
        (rc = alloc(adj_gD, N)) || (rc = alloc(adj_end, n3)) || (kF32 && (rc = alloc(adj_end_lo, n3))) ||
        (rc = alloc(adj_lam, n3)))
      return rc;
    return MM_OK;
  }

  // the slopes k1..k4 of the RK4 step from y (+ y_lo), with their stage
  // inputs and demag fields kept for the VJPs
  void adj_recompute_stages(const R* y, const R* ylo, double h) {
    static const double cin[4] = {0.0, 0.5, 0.5, 1.0};
    for (int i = 0; i < 4; ++i) {
      const R* Yi = y;
      if (i > 0) {
        launch_adj_stage_input<R>(y, ylo, adj_k[i - 1], cin[i] * h, adj_Y[i], 3 * N, st_);
        Yi = adj_Y[i];
      }
      adj_Yp[i] = Yi;
      FieldArgs<R> fa = fargs(~0u);
      if ((mask & TB_DEMAG) && demag) {
        demag->apply(Yi, Ms, adj_Hd[i], st_);
        fa.Hd = adj_Hd[i];
      }
      StageArgs<R> sa{};
      sa.out = adj_k[i];
      launch_stage<R>(SM_RHS, fa, Yi, sa, st_);
    }
  }

  // one step backwards: adj_lam holds dL/dy_{n+1} on entry, dL/dy_n on exit
  void adj_step_back(const R* y, const R* ylo, double h) {
    adj_recompute_stages(y, ylo, h);
    const R* const ks[4] = {adj_k[0], adj_k[1], adj_k[2], adj_k[3]};
    launch_adj_normalise<R>(y, ylo, ks, h, adj_lam, adj_mu, adj_g, N, st_);
    const unsigned loc = TB_EXCH | TB_DMI_BULK | TB_DMI_INTERFACIAL | TB_ANIS;
    const bool dem = (mask & TB_DEMAG) && demag;
    const bool zee = (mask & TB_ZEEMAN) != 0;
    AdjGrads gr{adj_gMs, (mask & TB_ANIS) ? adj_gKu : nullptr, (mask & TB_DMI_INTERFACIAL) ? adj_gD : nullptr};
    static const double wt[4] = {1.0, 2.0, 2.0, 1.0};
    static const double cin[4] = {0.0, 0.5, 0.5, 1.0};
    for (int i = 3; i >= 0; --i) {
      launch_adj_rhs<R>(fargs(loc), zee, adj_Yp[i], dem ? adj_Hd[i] : nullptr, adj_g, adj_q, adj_w, adj_a, gr, st_);
      FieldArgs<R> fl = fargs(loc | TB_DEMAG);
      if (dem) {
        demag->apply(adj_w, Ms, adj_Hdw, st_);
        fl.Hd = adj_Hdw;
      }
      const double cm = i > 0 ? wt[i - 1] * h / 6.0 : 0.0;
      const double ca = i > 0 ? cin[i] * h : 0.0;
      launch_adj_field<R>(fl, adj_w, adj_q, adj_Yp[i], adj_a, adj_lam, adj_mu, cm, ca, i > 0 ? adj_g : nullptr, gr,
                          st_);
    }
  }

  int adjoint_backward(const double* dLdm, double* gm0, double* gMs, double* gKu, double* gD) override {
    if (!adj_n) return fail(MM_ERR_STATE, "mm_adjoint_record must run first");
    if (adj_version != version) return fail(MM_ERR_STATE, "parameters changed since mm_adjoint_record");
    if (!dLdm) return fail(MM_ERR_ARG, "null dL/dm");
    int rc;
    if ((rc = adj_buffers())) return rc;
    const int64_t n3 = 3 * N;
    // dL/dm_T (AoS) -> SoA FP64
    int* flag = reinterpret_cast<int*>(scal + 63);
    MM_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), st_));
    MM_CUDA(cudaMemcpyAsync(stage64, dLdm, sizeof(double) * n3, cudaMemcpyHostToDevice, st_));
    launch_aos_to_soa<double>(stage64, adj_lam, nullptr, N, flag, st_);
    MM_CUDA(cudaMemsetAsync(adj_gMs, 0, sizeof(double) * N, st_));
    MM_CUDA(cudaMemsetAsync(adj_gKu, 0, sizeof(double) * N, st_));
    MM_CUDA(cudaMemsetAsync(adj_gD, 0, sizeof(double) * N, st_));
    // keep the final state; the segment recomputation steps m
    MM_CUDA(cudaMemcpyAsync(adj_end, m, sizeof(R) * n3, cudaMemcpyDeviceToDevice, st_));
    if (kF32) MM_CUDA(cudaMemcpyAsync(adj_end_lo, m_lo, sizeof(R) * n3, cudaMemcpyDeviceToDevice, st_));
    const int64_t rk_n0 = rk_n;
    const double rk_t0 = rk_t;
    for (int64_t sg = adj_nck - 1; sg >= 0; --sg) {
      const int64_t s0 = sg * adj_every, s1 = std::min(adj_n, s0 + adj_every);
      MM_CUDA(cudaMemcpyAsync(m, adj_ck + sg * n3, sizeof(R) * n3, cudaMemcpyDeviceToDevice, st_));
      if (kF32) MM_CUDA(cudaMemcpyAsync(m_lo, adj_ck_lo + sg * n3, sizeof(R) * n3, cudaMemcpyDeviceToDevice, st_));
      for (int64_t s = s0; s < s1; ++s) {
        MM_CUDA(cudaMemcpyAsync(adj_seg + (s - s0) * n3, m, sizeof(R) * n3, cudaMemcpyDeviceToDevice, st_));
        if (kF32)
          MM_CUDA(cudaMemcpyAsync(adj_seg_lo + (s - s0) * n3, m_lo, sizeof(R) * n3, cudaMemcpyDeviceToDevice, st_));
        if (s + 1 < s1 && (rc = rk4_run(adj_dt, 1))) return rc;
      }
      for (int64_t s = s1 - 1; s >= s0; --s)
        adj_step_back(adj_seg + (s - s0) * n3, kF32 ? adj_seg_lo + (s - s0) * n3 : nullptr, adj_dt);
      MM_CUDA(cudaGetLastError());
    }
    rk_n = rk_n0;
    rk_t = rk_t0;
    MM_CUDA(cudaMemcpyAsync(m, adj_end, sizeof(R) * n3, cudaMemcpyDeviceToDevice, st_));
    if (kF32) MM_CUDA(cudaMemcpyAsync(m_lo, adj_end_lo, sizeof(R) * n3, cudaMemcpyDeviceToDevice, st_));
    int hflag = 0;
    MM_CUDA(cudaMemcpyAsync(&hflag, flag, sizeof(int), cudaMemcpyDeviceToHost, st_));
    if (gm0) {
      launch_soa_to_aos<double>(adj_lam, nullptr, stage64, N, st_);
      MM_CUDA(cudaMemcpyAsync(gm0, stage64, sizeof(double) * n3, cudaMemcpyDeviceToHost, st_));
    }
    if (gMs) MM_CUDA(cudaMemcpyAsync(gMs, adj_gMs, sizeof(double) * N, cudaMemcpyDeviceToHost, st_));
    if (gKu) MM_CUDA(cudaMemcpyAsync(gKu, adj_gKu, sizeof(double) * N, cudaMemcpyDeviceToHost, st_));
    if (gD) MM_CUDA(cudaMemcpyAsync(gD, adj_gD, sizeof(double) * N, cudaMemcpyDeviceToHost, st_));
    MM_CUDA(cudaStreamSynchronize(st_));
    if (hflag) return fail(MM_ERR_NAN, "NaN in dL/dm");
    return MM_OK;
  }

  R *adj_ck = nullptr, *adj_ck_lo = nullptr, *adj_seg = nullptr, *adj_seg_lo = nullptr;
  R *adj_Y[4] = {}, *adj_k[4] = {}, *adj_Hd[4] = {};
  const R* adj_Yp[4] = {};
  R *adj_q = nullptr, *adj_w = nullptr, *adj_Hdw = nullptr, *adj_end = nullptr, *adj_end_lo = nullptr;
  double *adj_lam = nullptr, *adj_mu = nullptr, *adj_g = nullptr, *adj_a = nullptr;
  double *adj_gMs = nullptr, *adj_gKu = nullptr, *adj_gD = nullptr;
  int64_t adj_n = 0, adj_every = 0, adj_nck = 0, adj_seg_cap = 0;
  double adj_dt = 0.0;
  uint64_t adj_version = 0;

  // extra terms
  R *bDx = nullptr, *bDy = nullptr, *bDz = nullptr;
  bool bulk_spatial = false;
  R* sot_aj = nullptr;
  bool sot_spatial = false;
  double sot_aj_uni = 0.0, sot_bj = 0.0, sot_p[3] = {0, 0, 0};
  R *zl_bJ = nullptr, *zl_xi = nullptr;
  bool zl_spatial = false;
  double zl_xi_uni = 0.0, zl_ft = 1.0;
  R* sl_J = nullptr;
  bool sl_spatial = false;
  double sl_J_uni = 0.0, sl_ftb = 0.0, sl_L2 = 4.0, sl_P = 0.0, sl_xi = 0.0, sl_p[3] = {0, 0, 0};
  R *th_T = nullptr, *Hth = nullptr;
  long long* th_step = nullptr;
  double th_T_uni = 0.0, th_T0 = 0.0, th_scaling = 1.0, th_kB = 1.3806505e-23, th_dt = 1e-14;
  uint64_t th_seed = 0;

  // ------------------------------------------------------------ state --
  int nx = 1, ny = 1, nz = 1, pbc = 0;
  int64_t N = 1;
  double dx = 1e-9, dy = 1e-9, dz = 1e-9;
  R *m = nullptr, *m_lo = nullptr, *Ms = nullptr, *yA = nullptr, *yB = nullptr, *acc = nullptr, *work = nullptr;
  R *Hd = nullptr, *ecell = nullptr, *A = nullptr, *D = nullptr, *Ku = nullptr, *Hz = nullptr;
  R *ks[7] = {}, *yn = nullptr, *yn_lo = nullptr, *pre = nullptr, *pre_lo = nullptr, *gk = nullptr;
  uint8_t *nbm = nullptr, *pins = nullptr;
  double *stage64 = nullptr, *partials = nullptr, *scal = nullptr;
  DopriCtrl* ctrl = nullptr;
  DopriCtrl hctrl{};
  SdState* sd = nullptr;
  long long sd_steps = 0;
  std::unique_ptr<DemagPlan<R>> demag;
  unsigned mask = 0;
  bool ms_set = false, pins_on = false, ex_spatial = false, id_spatial = false, an_spatial = false, hz_arr = false;
  double ex_A[3] = {0, 0, 0}, bd[3] = {0, 0, 0}, id_D = 0, an_K = 0, an_u[3] = {0, 0, 1}, hz_uni[3] = {0, 0, 0};
  double alpha = 0.1, gamma = 2.21e5, tol = 1e-6;  // src/driver.jl:126,148
  int precession = 1;
  uint64_t version = 1;
  double rk_t = 0.0, rk_dt = 0.0;
  int64_t rk_n = 0;
  cudaGraphExec_t rk_graph = nullptr, dp_graph = nullptr;
  uint64_t rk_version = 0, dp_version = 0;

 private:
  template <typename T>
  int alloc(T*& p, int64_t n) {
    void* q = nullptr;
    const size_t b = sizeof(T) * static_cast<size_t>(n);
    cudaError_t e = cudaMalloc(&q, b);
    if (e != cudaSuccess) return fail(MM_ERR_CUDA, "cudaMalloc(%zu): %s", b, cudaGetErrorString(e));
    e = cudaMemsetAsync(q, 0, b, st_);
    if (e != cudaSuccess) return fail(MM_ERR_CUDA, "cudaMemset: %s", cudaGetErrorString(e));
    allocs_.push_back(q);
    bytes_ += b;
    p = static_cast<T*>(q);
    return MM_OK;
  }
  // free a buffer of alloc() (after the stream has drained)
  template <typename T>
  void release(T*& p, int64_t n) {
    if (!p) return;
    for (size_t i = 0; i < allocs_.size(); ++i)
      if (allocs_[i] == static_cast<void*>(p)) {
        allocs_.erase(allocs_.begin() + static_cast<std::ptrdiff_t>(i));
        break;
      }
    cudaFree(p);
    bytes_ -= sizeof(T) * static_cast<size_t>(n);
    p = nullptr;
  }
  cudaStream_t st_ = nullptr;
  std::vector<void*> allocs_;
  size_t bytes_ = 0;
};

}  // namespace mm

struct mm_handle {
  std::unique_ptr<mm::EngineBase> eng;
  mm_mesh_desc mesh{};
};

// A set of handles on one device stepped together: one RK4 step of every
// instance is captured as parallel branches (fork/join over the handles' own
// streams) of a single CUDA graph, launched once per step on the batch stream.
// Handles whose RK4 step launches descriptor kernels only are merged pass by
// pass: their steps are recorded (mm_launch.cuh) and the records of the same
// kernel across meshes become one launch over all of them (blocks look their
// mesh up), scheduled so that each mesh keeps its own order.  Other handles
// run as parallel branches of the same graph.
struct mm_batch {
  std::vector<mm_handle*> hs;
  int device = 0;
  cudaStream_t st = nullptr;
  cudaEvent_t fork = nullptr, done = nullptr;
  std::vector<cudaEvent_t> joins;
  cudaGraphExec_t graph = nullptr;
  double dt = 0.0;
  std::vector<uint64_t> versions;
  void* merged_args = nullptr;  // device: per merged launch, the meshes' Args and block offsets
  int launches = 0;             // kernel launches of one step
  int merged = 0;               // handles in the merged launches
  // small batches whose launches all have a persistent form run in the
  // persistent step kernel instead of the graph (one launch per 256 steps)
  mm::PersistProgram persist;
  bool use_persist = false;
  ~mm_batch() {
    cudaSetDevice(device);
    if (graph) cudaGraphExecDestroy(graph);
    if (merged_args) cudaFree(merged_args);
    for (cudaEvent_t e : joins) cudaEventDestroy(e);
    if (fork) cudaEventDestroy(fork);
    if (done) cudaEventDestroy(done);
    if (st) cudaStreamDestroy(st);
  }
};

using mm::fail;

// batches of at most this many cells run in the persistent step kernel
static constexpr int64_t kPersistBatchCells = int64_t(1) << 20;

// merged pass launches in batches unless MMCUDA_BATCH_MERGE=0
static bool batch_merge_enabled() {
  static const bool on = [] {
    const char* e = getenv("MMCUDA_BATCH_MERGE");
    return !(e && e[0] == '0');
  }();
  return on;
}

#define MM_HANDLE(h)                                                          \
  do {                                                                        \
    if (!(h) || !(h)->eng) return fail(MM_ERR_ARG, "null handle");            \
    if (cudaSetDevice((h)->eng->device) != cudaSuccess)                       \
      return fail(MM_ERR_CUDA, "cudaSetDevice(%d) failed", (h)->eng->device); \
  } while (0)

#define MM_GUARD(expr)                                          \
  try {                                                         \
    return (expr);                                              \
  } catch (const std::exception& ex) {                          \
    return fail(MM_ERR_CUDA, "exception: %s", ex.what());       \
  } catch (...) {                                               \
    return fail(MM_ERR_CUDA, "unknown exception");              \
  }

extern "C" {

int mm_abi_version(void) { return MMCUDA_ABI_VERSION; }

int mm_last_error(char* buf, size_t n) {
  if (!buf || n == 0) return MM_ERR_ARG;
  snprintf(buf, n, "%s", mm::g_err.c_str());
  return MM_OK;
}

int mm_create(const mm_mesh_desc* d, int form, int device, mm_handle** out) {
  if (!d || !out) return fail(MM_ERR_ARG, "null argument");
  *out = nullptr;
  if (d->nx < 1 || d->ny < 1 || d->nz < 1) return fail(MM_ERR_ARG, "mesh sizes must be >= 1");
  if (!(d->dx > 0) || !(d->dy > 0) || !(d->dz > 0)) return fail(MM_ERR_ARG, "cell sizes must be > 0");
  if (static_cast<int64_t>(d->nx) * d->ny * d->nz >= (1LL << 31))
    return fail(MM_ERR_ARG, "mesh has 2^31 or more cells");
  if (form != MM_FP64 && form != MM_FP32) return fail(MM_ERR_ARG, "form must be MM_FP64 or MM_FP32");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(MM_ERR_CUDA, "no CUDA device");
  if (device < 0 || device >= ndev) return fail(MM_ERR_ARG, "bad device %d", device);
  if (cudaSetDevice(device) != cudaSuccess) return fail(MM_ERR_CUDA, "cudaSetDevice failed");
  try {
    auto h = std::make_unique<mm_handle>();
    int rc;
    if (form == MM_FP64) {
      auto e = std::make_unique<mm::Engine<double>>();
      rc = e->init(*d, device);
      h->eng = std::move(e);
    } else {
      auto e = std::make_unique<mm::Engine<float>>();
      rc = e->init(*d, device);
      h->eng = std::move(e);
    }
    if (rc) return rc;
    h->mesh = *d;
    *out = h.release();
    return MM_OK;
  } catch (...) {
    return fail(MM_ERR_CUDA, "allocation failed");
  }
}

int mm_destroy(mm_handle* h) {
  if (!h) return MM_OK;
  delete h;
  return MM_OK;
}

int mm_get_stream(mm_handle* h, void** s) {
  MM_HANDLE(h);
  if (!s) return fail(MM_ERR_ARG, "null argument");
  *s = static_cast<void*>(h->eng->stream());
  return MM_OK;
}

int mm_synchronize(mm_handle* h) {
  MM_HANDLE(h);
  cudaError_t e = cudaStreamSynchronize(h->eng->stream());
  if (e != cudaSuccess) return fail(MM_ERR_CUDA, "%s", cudaGetErrorString(e));
  const bool y_timeout = mm::wreg_take_timeout(), z_timeout = mm::zpair_take_timeout();
  if (y_timeout || z_timeout)
    return fail(MM_ERR_TIMEOUT, "demag %s pass: a bounded bulk-copy wait ran out (fields of that pass are incomplete)",
                y_timeout ? "y" : "z");
  return MM_OK;
}

int mm_device_bytes(mm_handle* h, size_t* b) {
  MM_HANDLE(h);
  if (!b) return fail(MM_ERR_ARG, "null argument");
  *b = h->eng->device_bytes();
  return MM_OK;
}

int mm_set_Ms(mm_handle* h, const double* Ms, double uni) { MM_HANDLE(h); MM_GUARD(h->eng->set_Ms(Ms, uni)); }
int mm_set_m(mm_handle* h, const double* m) {
  MM_HANDLE(h);
  if (!m) return fail(MM_ERR_ARG, "null m");
  MM_GUARD(h->eng->set_m(m));
}
int mm_get_m(mm_handle* h, double* m) {
  MM_HANDLE(h);
  if (!m) return fail(MM_ERR_ARG, "null m");
  MM_GUARD(h->eng->get_m(m));
}
int mm_set_m_f32(mm_handle* h, const float* m) {
  MM_HANDLE(h);
  if (!m) return fail(MM_ERR_ARG, "null m");
  MM_GUARD(h->eng->set_m_f32(m));
}
int mm_get_m_f32(mm_handle* h, float* m) {
  MM_HANDLE(h);
  if (!m) return fail(MM_ERR_ARG, "null m");
  MM_GUARD(h->eng->get_m_f32(m));
}
int mm_set_pins(mm_handle* h, const uint8_t* p) { MM_HANDLE(h); MM_GUARD(h->eng->set_pins(p)); }
int mm_set_llg(mm_handle* h, double a, double g, int p) { MM_HANDLE(h); MM_GUARD(h->eng->set_llg(a, g, p)); }
int mm_add_zeeman(mm_handle* h, const double* H, double x, double y, double z) {
  MM_HANDLE(h);
  MM_GUARD(h->eng->zeeman(H, x, y, z, false));
}
int mm_update_zeeman(mm_handle* h, const double* H, double x, double y, double z) {
  MM_HANDLE(h);
  MM_GUARD(h->eng->zeeman(H, x, y, z, true));
}
int mm_add_exch(mm_handle* h, const double* A, double ax, double ay, double az) {
  MM_HANDLE(h);
  MM_GUARD(h->eng->add_exch(A, ax, ay, az));
}
int mm_add_dmi_bulk(mm_handle* h, double x, double y, double z) { MM_HANDLE(h); MM_GUARD(h->eng->add_dmi_bulk(x, y, z)); }
int mm_add_dmi_interfacial(mm_handle* h, const double* D, double u) {
  MM_HANDLE(h);
  MM_GUARD(h->eng->add_dmi_interfacial(D, u));
}
int mm_add_anis(mm_handle* h, const double* K, double u, double ax, double ay, double az) {
  MM_HANDLE(h);
  MM_GUARD(h->eng->add_anis(K, u, ax, ay, az));
}
int mm_add_demag(mm_handle* h, int Nx, int Ny, int Nz) { MM_HANDLE(h); MM_GUARD(h->eng->add_demag(Nx, Ny, Nz, nullptr)); }
int mm_add_demag_tensor(mm_handle* h, const double* T) {
  MM_HANDLE(h);
  if (!T) return fail(MM_ERR_ARG, "null tensor");
  MM_GUARD(h->eng->add_demag(0, 0, 0, T));
}
int mm_effective_field(mm_handle* h, double* H) { MM_HANDLE(h); MM_GUARD(h->eng->effective_field(H)); }
int mm_term_field(mm_handle* h, int term, double* f, double* e) { MM_HANDLE(h); MM_GUARD(h->eng->term_field(term, f, e)); }
int mm_energy(mm_handle* h, double* per, double* tot) { MM_HANDLE(h); MM_GUARD(h->eng->energy(per, tot)); }
int mm_llg_rhs(mm_handle* h, double* out) {
  MM_HANDLE(h);
  if (!out) return fail(MM_ERR_ARG, "null output");
  MM_GUARD(h->eng->llg_rhs(out));
}
int mm_average_m(mm_handle* h, double* m3) {
  MM_HANDLE(h);
  if (!m3) return fail(MM_ERR_ARG, "null output");
  MM_GUARD(h->eng->average_m(m3));
}
int mm_rk4_run(mm_handle* h, double dt, int64_t n) { MM_HANDLE(h); MM_GUARD(h->eng->rk4_run(dt, n)); }
int mm_rk4_state(mm_handle* h, double* t, int64_t* n) { MM_HANDLE(h); MM_GUARD(h->eng->rk4_state(t, n)); }
int mm_heun_run(mm_handle* h, double dt, int64_t n) { MM_HANDLE(h); MM_GUARD(h->eng->heun_run(dt, n)); }
int mm_dopri_set_tol(mm_handle* h, double tol) { MM_HANDLE(h); MM_GUARD(h->eng->dopri_tol(tol)); }
int mm_run_until(mm_handle* h, double t, mm_stats* s) { MM_HANDLE(h); MM_GUARD(h->eng->run_until(t, s)); }
int mm_advance_step(mm_handle* h, mm_stats* s) { MM_HANDLE(h); MM_GUARD(h->eng->advance_step(s)); }
int mm_dopri_reset(mm_handle* h) { MM_HANDLE(h); MM_GUARD(h->eng->dopri_reset()); }
int mm_set_adaptive_method(mm_handle* h, int method) { MM_HANDLE(h); MM_GUARD(h->eng->set_method(method)); }

int mm_demag_tiles(mm_handle* h, int* tiles, float* ms) {
  MM_HANDLE(h);
  MM_GUARD(h->eng->demag_tiles(tiles, ms));
}

int mm_add_dmi_bulk_spatial(mm_handle* h, const double* Dx, const double* Dy, const double* Dz) {
  MM_HANDLE(h);
  MM_GUARD(h->eng->add_dmi_bulk_spatial(Dx, Dy, Dz));
}
int mm_add_sot(mm_handle* h, const double* aj, double aj_uniform, double bj, double px, double py, double pz) {
  MM_HANDLE(h);
  MM_GUARD(h->eng->add_sot(aj, aj_uniform, bj, px, py, pz));
}
int mm_add_stt_zhang_li(mm_handle* h, const double* bJ, const double* xi, double xi_uniform, double ft) {
  MM_HANDLE(h);
  MM_GUARD(h->eng->add_stt_zhang_li(bJ, xi, xi_uniform, ft));
}
int mm_add_stt_slonczewski(mm_handle* h, const double* J, double J_uniform, double ft_beta, double Lambda, double P,
                           double xi, double px, double py, double pz) {
  MM_HANDLE(h);
  MM_GUARD(h->eng->add_stt_slonczewski(J, J_uniform, ft_beta, Lambda, P, xi, px, py, pz));
}
int mm_add_thermal_noise(mm_handle* h, const double* T, double T_uniform, double T0, double scaling, double k_B,
                         uint64_t seed, double dt) {
  MM_HANDLE(h);
  MM_GUARD(h->eng->add_thermal_noise(T, T_uniform, T0, scaling, k_B, seed, dt));
}

int mm_adjoint_record(mm_handle* h, double dt, int64_t nsteps, int64_t ckpt_every) {
  MM_HANDLE(h);
  MM_GUARD(h->eng->adjoint_record(dt, nsteps, ckpt_every));
}
int mm_adjoint_backward(mm_handle* h, const double* dL_dmT, double* g_m0, double* g_Ms, double* g_Ku, double* g_D) {
  MM_HANDLE(h);
  MM_GUARD(h->eng->adjoint_backward(dL_dmT, g_m0, g_Ms, g_Ku, g_D));
}

int mm_save_ovf(mm_handle* h, const char* path, int type, const char* title) {
  MM_HANDLE(h);
  const mm_mesh_desc& d = h->mesh;
  std::vector<double> m(static_cast<size_t>(3) * d.nx * d.ny * d.nz);
  if (int rc = h->eng->get_m(m.data())) return rc;
  return mm_ovf_write(path, &d, m.data(), type, title);
}

int mm_load_ovf(mm_handle* h, const char* path) {
  MM_HANDLE(h);
  const mm_mesh_desc& d = h->mesh;
  std::vector<double> m(static_cast<size_t>(3) * d.nx * d.ny * d.nz);
  if (int rc = mm_ovf_read(path, m.data(), static_cast<int64_t>(d.nx) * d.ny * d.nz)) return rc;
  MM_GUARD(h->eng->set_m(m.data()));
}
int mm_relax(mm_handle* h, int driver, int64_t max_steps, double stop, int64_t* steps, double* mx) {
  MM_HANDLE(h);
  if (driver != MM_DRIVER_SD && driver != MM_DRIVER_LLG) return fail(MM_ERR_ARG, "driver must be SD or LLG");
  MM_GUARD(h->eng->relax(driver, max_steps, stop, steps, mx));
}

int mm_kernel_time(mm_handle* h, int kernel, int reps, double* ms, double* bytes) {
  MM_HANDLE(h);
  MM_GUARD(h->eng->kernel_time(kernel, reps, ms, bytes));
}
int mm_rk4_launches_per_step(mm_handle* h, int* n) {
  MM_HANDLE(h);
  if (!n) return fail(MM_ERR_ARG, "null output");
  *n = h->eng->rk4_launches();
  return MM_OK;
}

int mm_batch_create(mm_handle* const* handles, int n, mm_batch** out) {
  if (!handles || !out || n < 1) return fail(MM_ERR_ARG, "mm_batch_create: need n >= 1 handles");
  *out = nullptr;
  const int dev = handles[0] && handles[0]->eng ? handles[0]->eng->device : -1;
  for (int i = 0; i < n; ++i) {
    if (!handles[i] || !handles[i]->eng) return fail(MM_ERR_ARG, "mm_batch_create: null handle %d", i);
    if (handles[i]->eng->device != dev) return fail(MM_ERR_ARG, "mm_batch_create: handles on different devices");
    for (int j = 0; j < i; ++j)
      if (handles[j] == handles[i]) return fail(MM_ERR_ARG, "mm_batch_create: handle %d repeated", i);
  }
  if (cudaSetDevice(dev) != cudaSuccess) return fail(MM_ERR_CUDA, "cudaSetDevice failed");
  auto b = std::make_unique<mm_batch>();
  b->device = dev;
  b->hs.assign(handles, handles + n);
  if (cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming) != cudaSuccess)
    return fail(MM_ERR_CUDA, "mm_batch_create: stream/event creation failed");
  b->joins.resize(n);
  for (int i = 0; i < n; ++i)
    if (cudaEventCreateWithFlags(&b->joins[i], cudaEventDisableTiming) != cudaSuccess)
      return fail(MM_ERR_CUDA, "mm_batch_create: event creation failed");
  *out = b.release();
  return MM_OK;
}

int mm_batch_launches(mm_batch* b, int* launches_per_step, int* merged_handles) {
  if (!b) return fail(MM_ERR_ARG, "null batch");
  if (launches_per_step) *launches_per_step = b->launches;
  if (merged_handles) *merged_handles = b->merged;
  return MM_OK;
}

int mm_batch_destroy(mm_batch* b) {
  delete b;
  return MM_OK;
}

int mm_batch_get_stream(mm_batch* b, void** s) {
  if (!b || !s) return fail(MM_ERR_ARG, "null argument");
  *s = static_cast<void*>(b->st);
  return MM_OK;
}

int mm_batch_rk4_run(mm_batch* b, double dt, int64_t nsteps) {
  if (!b) return fail(MM_ERR_ARG, "null batch");
  if (nsteps < 0 || !(dt > 0)) return fail(MM_ERR_ARG, "rk4: need dt > 0 and nsteps >= 0");
  if (cudaSetDevice(b->device) != cudaSuccess) return fail(MM_ERR_CUDA, "cudaSetDevice failed");
  try {
    const int n = static_cast<int>(b->hs.size());
    bool stale = (!b->graph && !b->use_persist) || b->dt != dt || static_cast<int>(b->versions.size()) != n;
    for (int i = 0; i < n && !stale; ++i) stale = b->versions[i] != b->hs[i]->eng->params_version();
    for (int i = 0; i < n; ++i)
      if (int rc = b->hs[i]->eng->rk4_prepare()) return rc;
    // earlier work of every handle precedes the batch
    for (int i = 0; i < n; ++i) {
      MM_CUDA(cudaEventRecord(b->joins[i], b->hs[i]->eng->stream()));
      MM_CUDA(cudaStreamWaitEvent(b->st, b->joins[i], 0));
    }
    if (stale) {
      if (b->graph) cudaGraphExecDestroy(b->graph);
      b->graph = nullptr;
      if (b->merged_args) cudaFree(b->merged_args);
      b->merged_args = nullptr;
      b->persist.release();
      b->use_persist = false;
      int64_t cells = 0;
      bool all = mm::persist_enabled() && batch_merge_enabled();
      for (int i = 0; i < n && all; ++i) {
        all = b->hs[i]->eng->rk4_batchable() && b->hs[i]->eng->is_fp32() == b->hs[0]->eng->is_fp32();
        cells += static_cast<int64_t>(b->hs[i]->mesh.nx) * b->hs[i]->mesh.ny * b->hs[i]->mesh.nz;
      }
      if (all && cells <= kPersistBatchCells) {
        std::vector<std::vector<mm::LaunchRec>> recs(n);
        for (int i = 0; i < n; ++i) {
          mm::LaunchRecorder rec;
          mm::launch_recorder() = &rec;
          b->hs[i]->eng->rk4_enqueue(dt);
          mm::launch_recorder() = nullptr;
          recs[i] = std::move(rec.recs);
        }
        char msg[256] = {0};
        b->use_persist = b->persist.build(recs, b->hs[0]->eng->is_fp32(), msg, sizeof(msg)) == 0;
      }
    }
    if (b->use_persist) {
      b->dt = dt;
      b->versions.resize(n);
      for (int i = 0; i < n; ++i) b->versions[i] = b->hs[i]->eng->params_version();
      b->launches = 1;
      b->merged = n;
      const int rc = b->persist.run(nsteps, b->st);
      if (rc == 1) return fail(MM_ERR_TIMEOUT, "persistent batch step: a grid-barrier wait ran out");
      if (rc) return fail(MM_ERR_CUDA, "persistent batch step failed");
      MM_CUDA(cudaEventRecord(b->done, b->st));
      for (int i = 0; i < n; ++i) {
        MM_CUDA(cudaStreamWaitEvent(b->hs[i]->eng->stream(), b->done, 0));
        b->hs[i]->eng->rk4_count(nsteps, dt);
      }
      return MM_OK;
    }
    if (stale) {
      // record the steps of the handles whose launches can be merged
      std::vector<int> rec_h, branch_h;
      for (int i = 0; i < n; ++i)
        (batch_merge_enabled() && b->hs[i]->eng->rk4_batchable() ? rec_h : branch_h).push_back(i);
      if (rec_h.size() < 2) {
        branch_h.insert(branch_h.end(), rec_h.begin(), rec_h.end());
        rec_h.clear();
      }
      std::vector<std::vector<mm::LaunchRec>> recs(rec_h.size());
      for (size_t j = 0; j < rec_h.size(); ++j) {
        mm::LaunchRecorder rec;
        mm::launch_recorder() = &rec;
        b->hs[rec_h[j]]->eng->rk4_enqueue(dt);
        mm::launch_recorder() = nullptr;
        recs[j] = std::move(rec.recs);
      }
      // the merged kernels keep the mesh's arguments in static shared
      // memory: meshes whose passes need nearly all of a block's shared
      // memory stay on their own branch
      for (size_t j = 0; j < recs.size();) {
        bool fits = true;
        for (const mm::LaunchRec& r : recs[j]) fits = fits && r.smem + 4096 <= 227 * 1024;
        if (fits) {
          ++j;
          continue;
        }
        branch_h.push_back(rec_h[j]);
        rec_h.erase(rec_h.begin() + j);
        recs.erase(recs.begin() + j);
      }
      // Meshes with the same sequence of kernels (e.g. films on the fused y
      // convolution, 3-D meshes on the z convolution) form a family; each
      // family runs on its own graph branch, its k-th launch merged over
      // all its meshes, so the families overlap as independent meshes did.
      struct Merged {
        const mm::LaunchRec* first;
        std::vector<const mm::LaunchRec*> parts;
        int blocks = 0;
        size_t smem = 0, off_args = 0, off_begins = 0;
        int family = 0;
      };
      std::vector<Merged> plan;
      std::vector<std::vector<size_t>> families;  // members (indices into recs)
      for (size_t j = 0; j < recs.size(); ++j) {
        auto same = [&](size_t o) {
          if (recs[o].size() != recs[j].size()) return false;
          for (size_t q = 0; q < recs[j].size(); ++q)
            if (recs[o][q].kind != recs[j][q].kind) return false;
          return true;
        };
        auto f = std::find_if(families.begin(), families.end(), [&](const auto& fam) { return same(fam[0]); });
        if (f == families.end()) families.push_back({j});
        else f->push_back(j);
      }
      for (size_t fi = 0; fi < families.size(); ++fi) {
        const auto& fam = families[fi];
        for (size_t q = 0; q < recs[fam[0]].size(); ++q) {
          Merged mg;
          mg.first = &recs[fam[0]][q];
          mg.family = static_cast<int>(fi);
          for (size_t j : fam) {
            const mm::LaunchRec* r = &recs[j][q];
            mg.parts.push_back(r);
            mg.blocks += r->blocks;
            mg.smem = std::max(mg.smem, r->smem);
          }
          plan.push_back(std::move(mg));
        }
      }
      // one device buffer: per merged launch its Args array and block offsets
      size_t bytes = 0;
      for (Merged& mg : plan) {
        mg.off_args = bytes;
        bytes += (mg.first->args_size * mg.parts.size() + 255) / 256 * 256;
        mg.off_begins = bytes;
        bytes += (sizeof(int) * mg.parts.size() + 255) / 256 * 256;
      }
      if (bytes) {
        std::vector<unsigned char> host(bytes, 0);
        for (Merged& mg : plan) {
          int beg = 0;
          for (size_t q = 0; q < mg.parts.size(); ++q) {
            std::memcpy(host.data() + mg.off_args + q * mg.first->args_size, mg.parts[q]->args.data(),
                        mg.first->args_size);
            std::memcpy(host.data() + mg.off_begins + q * sizeof(int), &beg, sizeof(int));
            beg += mg.parts[q]->blocks;
          }
        }
        MM_CUDA(cudaMalloc(&b->merged_args, bytes));
        MM_CUDA(cudaMemcpy(b->merged_args, host.data(), bytes, cudaMemcpyHostToDevice));
      }
      cudaGraph_t g;
      MM_CUDA(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
      MM_CUDA(cudaEventRecord(b->fork, b->st));
      int launches = 0;
      for (int i : branch_h) {
        cudaStream_t hs = b->hs[i]->eng->stream();
        MM_CUDA(cudaStreamWaitEvent(hs, b->fork, 0));
        b->hs[i]->eng->rk4_enqueue(dt);
        MM_CUDA(cudaEventRecord(b->joins[i], hs));
        launches += b->hs[i]->eng->rk4_launches();
      }
      // each family on the stream of its first handle (forked from the batch
      // stream, joined back below)
      unsigned char* base = static_cast<unsigned char*>(b->merged_args);
      for (size_t fi = 0; fi < families.size(); ++fi) {
        const int hi = rec_h[families[fi][0]];
        cudaStream_t fs = b->hs[hi]->eng->stream();
        MM_CUDA(cudaStreamWaitEvent(fs, b->fork, 0));
        for (const Merged& mg : plan) {
          if (mg.family != static_cast<int>(fi)) continue;
          MM_CUDA(mg.first->many(base + mg.off_args, reinterpret_cast<const int*>(base + mg.off_begins),
                                 static_cast<int>(mg.parts.size()), mg.blocks, mg.smem, fs));
          ++launches;
        }
        MM_CUDA(cudaEventRecord(b->joins[hi], fs));
      }
      for (int i : branch_h) MM_CUDA(cudaStreamWaitEvent(b->st, b->joins[i], 0));
      for (const auto& fam : families) MM_CUDA(cudaStreamWaitEvent(b->st, b->joins[rec_h[fam[0]]], 0));
      MM_CUDA(cudaStreamEndCapture(b->st, &g));
      b->launches = launches;
      b->merged = static_cast<int>(rec_h.size());
      MM_CUDA(cudaGraphInstantiate(&b->graph, g, 0));
      cudaGraphDestroy(g);
      b->dt = dt;
      b->versions.resize(n);
      for (int i = 0; i < n; ++i) b->versions[i] = b->hs[i]->eng->params_version();
    }
    for (int64_t k = 0; k < nsteps; ++k) MM_CUDA(cudaGraphLaunch(b->graph, b->st));
    // later work of every handle follows the batch
    MM_CUDA(cudaEventRecord(b->done, b->st));
    for (int i = 0; i < n; ++i) {
      MM_CUDA(cudaStreamWaitEvent(b->hs[i]->eng->stream(), b->done, 0));
      b->hs[i]->eng->rk4_count(nsteps, dt);
    }
    MM_CUDA(cudaGetLastError());
    return MM_OK;
  } catch (...) {
    return fail(MM_ERR_CUDA, "mm_batch_rk4_run: exception");
  }
}

}  // extern "C"

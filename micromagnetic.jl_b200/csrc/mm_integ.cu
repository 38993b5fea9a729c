// mm_integ.cu -- device-side integrator control: Dormand-Prince step-size
// controller, steepest-descent (Barzilai-Borwein) relax kernels, and the
// relax stop-criterion reduction.
#include <cmath>

#include "mm_field.cuh"
#include "mm_integ.cuh"

namespace mm {

// advance_step(sim, ::AdaptiveRK) decision logic after one attempt
// (src/integrator/adaptive_rk.jl:105-146) followed by the integrate_to_time
// loop condition and end-time clipping (adaptive_rk.jl:168-186).  One block;
// partials hold per-block maxima of |err|/(1+|y|) from the stage-7 kernel.
__global__ void k_dopri_control(DopriCtrl* __restrict__ c, const double* __restrict__ partials, int nblocks) {
  __shared__ double sh[256];
  if (!c->active) {
    if (threadIdx.x == 0) c->accepted_last = 0;
    return;
  }
  double v = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
    const double u = partials[b];
    v = (u > v || isnan(u)) ? u : v;
  }
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      const double u = sh[threadIdx.x + o];
      if (u > sh[threadIdx.x] || isnan(u)) sh[threadIdx.x] = u;
    }
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  const double safety = 0.824, facmax = 5.0, facmin = 0.2;
  const int order = c->order;  // order_embedded of the method
  c->attempts += 1;
  c->nfevals += c->eval1 + (c->nstage - 1);
  const double err = sh[0] * c->step / c->tol;
  c->err = err;
  if (isnan(err)) {
    c->step_next = 1e-14;
    c->status = 1;
    c->active = 0;
    c->eval1 = 0;
    c->accepted_last = 0;
    return;
  }
  c->inner += 1;
  if (c->inner > 50) {
    c->status = 2;
    c->active = 0;
    c->eval1 = 0;
    c->accepted_last = 0;
    return;
  }
  c->succeed = err <= 1.0;
  // the next attempt reuses the last stage as k1 after an accepted FSAL step
  c->eval1 = (c->succeed && c->fsal) ? 0 : 1;
  if (err <= 1.0) {
    c->accepted_last = 1;
    c->nsteps += 1;
    c->t += c->step;
    const double factor = safety * pow(1.0 / err, 1.0 / (order + 1));
    c->step_next = c->step * fmin(facmax, fmax(facmin, factor));
    c->inner = 1;
    if (c->single || !(c->t < c->t_final)) {
      c->active = 0;
      c->eval1 = 0;
    } else {
      if (c->step_next + c->t > c->t_final) c->step_next = c->t_final - c->t;
      c->step = c->step_next;
    }
  } else {
    c->accepted_last = 0;
    c->rejected += 1;
    const double factor = safety * pow(1.0 / err, 1.0 / order);
    c->step = c->step * fmin(facmax, fmax(facmin, factor));
  }
}

// y_current .= y_next on acceptance (adaptive_rk.jl:126)
template <typename R>
__global__ void k_dopri_accept(const DopriCtrl* __restrict__ c, R* __restrict__ m, R* __restrict__ m_lo,
                               const R* __restrict__ yn, const R* __restrict__ yn_lo, int64_t n3) {
  if (!c->accepted_last) return;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n3;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    m[i] = yn[i];
    if (m_lo) m_lo[i] = yn_lo[i];
  }
}

void launch_dopri_control(DopriCtrl* c, const double* partials, int nblocks, cudaStream_t st) {
  k_dopri_control<<<1, 256, 0, st>>>(c, partials, nblocks);
}

template <typename R>
void launch_dopri_accept(const DopriCtrl* c, R* m, R* m_lo, const R* yn, const R* yn_lo, int64_t n3, cudaStream_t st) {
  k_dopri_accept<R><<<1184, 256, 0, st>>>(c, m, m_lo, yn, yn_lo, n3);
}

// ------------------------------------------------------------- SD relax ---
// src/sd.jl: compute_gk_kernel_1! (9-17), compute_gk_kernel_2! (19-37),
// compute_tau (56-82), run_step_kernel! (39-54).  Sums are FP64.
template <typename R>
__global__ void k_sd_gk(const R* __restrict__ m, const R* __restrict__ pre, const R* __restrict__ h,
                        R* __restrict__ gk, int64_t N, int first, double* __restrict__ partials) {
  __shared__ double sh[3][256];
  const int64_t I = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  double ss = 0, sf = 0, ff = 0;
  if (I < N) {
    const R mx = m[I], my = m[N + I], mz = m[2 * N + I];
    const R hx = h[I], hy = h[N + I], hz = h[2 * N + I];
    const R fx = -mz * hy + my * hz, fy = mz * hx - mx * hz, fz = -my * hx + mx * hy;
    const R gx = -mz * fy + my * fz, gy = mz * fx - mx * fz, gz = -my * fx + mx * fy;
    if (!first) {
      const R sx = mx - pre[I], sy = my - pre[N + I], sz = mz - pre[2 * N + I];
      const R dx = gx - gk[I], dy = gy - gk[N + I], dz = gz - gk[2 * N + I];
      ss = double(sx) * sx + double(sy) * sy + double(sz) * sz;
      sf = double(sx) * dx + double(sy) * dy + double(sz) * dz;
      ff = double(dx) * dx + double(dy) * dy + double(dz) * dz;
    }
    gk[I] = gx;
    gk[N + I] = gy;
    gk[2 * N + I] = gz;
  }
  if (first) return;
  sh[0][threadIdx.x] = ss;
  sh[1][threadIdx.x] = sf;
  sh[2][threadIdx.x] = ff;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int c = 0; c < 3; ++c) sh[c][threadIdx.x] += sh[c][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x < 3) partials[blockIdx.x * 3 + threadIdx.x] = sh[threadIdx.x][0];
}

// tau from the Barzilai-Borwein sums (compute_tau, src/sd.jl:56-82)
__global__ void k_sd_tau(SdState* __restrict__ s, const double* __restrict__ partials, int nblocks) {
  __shared__ double sh[3][256];
  if (s->steps == 0) {
    if (threadIdx.x == 0) s->tau = s->min_tau;
    return;
  }
  double a[3] = {0, 0, 0};
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
    for (int c = 0; c < 3; ++c) a[c] += partials[b * 3 + c];
  for (int c = 0; c < 3; ++c) sh[c][threadIdx.x] = a[c];
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int c = 0; c < 3; ++c) sh[c][threadIdx.x] += sh[c][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double s1 = sh[0][0], s2 = sh[1][0], s3 = sh[2][0];
    const double tau1 = s2 != 0.0 ? s1 / s2 : s->min_tau;
    const double tau2 = s3 != 0.0 ? s2 / s3 : s->min_tau;
    double tau = (s->steps % 2 == 0) ? fabs(tau2) : fabs(tau1);
    if (tau > s->max_tau) tau = s->max_tau;
    s->tau = tau;
  }
}

template <typename R>
__global__ void k_sd_update(R* __restrict__ m, R* __restrict__ pre, const R* __restrict__ h,
                            const R* __restrict__ gk, const uint8_t* __restrict__ pins, const SdState* __restrict__ s,
                            int64_t N) {
  const int64_t I = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (I >= N) return;
  const R mx = m[I], my = m[N + I], mz = m[2 * N + I];
  pre[I] = mx;
  pre[N + I] = my;
  pre[2 * N + I] = mz;
  if (pins && pins[I]) return;
  const R tau = static_cast<R>(s->tau);
  const R hx = h[I], hy = h[N + I], hz = h[2 * N + I];
  const R fx = -mz * hy + my * hz, fy = mz * hx - mx * hz, fz = -my * hx + mx * hy;
  const R factor = R(0.25) * (fx * fx + fy * fy + fz * fz) * tau * tau;
  const R nx = (1 - factor) * mx - tau * gk[I];
  const R ny = (1 - factor) * my - tau * gk[N + I];
  const R nz = (1 - factor) * mz - tau * gk[2 * N + I];
  m[I] = nx / (1 + factor);
  m[N + I] = ny / (1 + factor);
  m[2 * N + I] = nz / (1 + factor);
}

__global__ void k_sd_count(SdState* __restrict__ s) { s->steps += 1; }

template <typename R>
__global__ void k_normalise(R* __restrict__ m, int64_t N) {
  const int64_t I = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (I >= N) return;
  const R x = m[I], y = m[N + I], z = m[2 * N + I];
  const R m2 = x * x + y * y + z * z;
  if (m2 > 0) {
    const R len = R(1) / sqrt(m2);
    m[I] = x * len;
    m[N + I] = y * len;
    m[2 * N + I] = z * len;
  }
}

// max over cells of |a - b| (compute_dm! + maximum, src/helper.jl:273-286)
template <typename R>
__global__ void k_max_dm(const R* __restrict__ a, const R* __restrict__ alo, const R* __restrict__ b,
                         const R* __restrict__ blo, int64_t N, double* __restrict__ partials) {
  __shared__ double sh[256];
  const int64_t I = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  double v = 0.0;
  if (I < N) {
    double s = 0.0;
    for (int c = 0; c < 3; ++c) {
      double d = double(a[c * N + I]) - double(b[c * N + I]);
      if (alo) d += double(alo[c * N + I]);
      if (blo) d -= double(blo[c * N + I]);
      s += d * d;
    }
    v = sqrt(s);
  }
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) partials[blockIdx.x] = sh[0];
}

__global__ void k_reduce_max(const double* __restrict__ partials, int nblocks, double* __restrict__ out) {
  __shared__ double sh[256];
  double v = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) v = fmax(v, partials[b]);
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sh[0];
}

// max_i |v_i| over a 3N vector (compute_initial_step, adaptive_rk.jl:156)
template <typename R>
__global__ void k_absmax(const R* __restrict__ v, int64_t n, double* __restrict__ partials) {
  __shared__ double sh[256];
  double mx = 0.0;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double u = fabs(double(v[i]));
    mx = (u > mx || isnan(u)) ? u : mx;
  }
  sh[threadIdx.x] = mx;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      const double u = sh[threadIdx.x + o];
      if (u > sh[threadIdx.x] || isnan(u)) sh[threadIdx.x] = u;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) partials[blockIdx.x] = sh[0];
}

template <typename R>
void launch_sd_gk(const R* m, const R* pre, const R* h, R* gk, int64_t N, int first, double* partials, cudaStream_t st) {
  k_sd_gk<R><<<stage_blocks(N), 256, 0, st>>>(m, pre, h, gk, N, first, partials);
}
void launch_sd_tau(SdState* s, const double* partials, int nblocks, cudaStream_t st) {
  k_sd_tau<<<1, 256, 0, st>>>(s, partials, nblocks);
}
template <typename R>
void launch_sd_update(R* m, R* pre, const R* h, const R* gk, const uint8_t* pins, const SdState* s, int64_t N, cudaStream_t st) {
  k_sd_update<R><<<stage_blocks(N), 256, 0, st>>>(m, pre, h, gk, pins, s, N);
}
void launch_sd_count(SdState* s, cudaStream_t st) { k_sd_count<<<1, 1, 0, st>>>(s); }
template <typename R>
void launch_normalise(R* m, int64_t N, cudaStream_t st) {
  k_normalise<R><<<stage_blocks(N), 256, 0, st>>>(m, N);
}
template <typename R>
void launch_max_dm(const R* a, const R* alo, const R* b, const R* blo, int64_t N, double* partials, double* out, cudaStream_t st) {
  const int nb = stage_blocks(N);
  k_max_dm<R><<<nb, 256, 0, st>>>(a, alo, b, blo, N, partials);
  k_reduce_max<<<1, 256, 0, st>>>(partials, nb, out);
}
template <typename R>
void launch_absmax(const R* v, int64_t n, double* partials, double* out, cudaStream_t st) {
  k_absmax<R><<<592, 256, 0, st>>>(v, n, partials);
  k_reduce_max<<<1, 256, 0, st>>>(partials, 592, out);
}

#define MM_INST2(R)                                                                                          \
  template void launch_dopri_accept<R>(const DopriCtrl*, R*, R*, const R*, const R*, int64_t, cudaStream_t); \
  template void launch_sd_gk<R>(const R*, const R*, const R*, R*, int64_t, int, double*, cudaStream_t);      \
  template void launch_sd_update<R>(R*, R*, const R*, const R*, const uint8_t*, const SdState*, int64_t,     \
                                    cudaStream_t);                                                           \
  template void launch_normalise<R>(R*, int64_t, cudaStream_t);                                              \
  template void launch_max_dm<R>(const R*, const R*, const R*, const R*, int64_t, double*, double*,          \
                                 cudaStream_t);                                                              \
  template void launch_absmax<R>(const R*, int64_t, double*, double*, cudaStream_t);
MM_INST2(float)
MM_INST2(double)

}  // namespace mm

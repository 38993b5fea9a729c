// mm_integ.cuh -- integrator control kernels (internal interface).
#pragma once
#include "mm_field.cuh"

namespace mm {

// SD driver state (src/driver.jl:3-12, defaults src/driver.jl:95-102)
struct SdState {
  double tau, max_tau, min_tau;
  long long steps;
};

void launch_dopri_control(DopriCtrl* c, const double* partials, int nblocks, cudaStream_t st);
template <typename R>
void launch_dopri_accept(const DopriCtrl* c, R* m, R* m_lo, const R* yn, const R* yn_lo, int64_t n3, cudaStream_t st);

template <typename R>
void launch_sd_gk(const R* m, const R* pre, const R* h, R* gk, int64_t N, int first, double* partials, cudaStream_t st);
void launch_sd_tau(SdState* s, const double* partials, int nblocks, cudaStream_t st);
template <typename R>
void launch_sd_update(R* m, R* pre, const R* h, const R* gk, const uint8_t* pins, const SdState* s, int64_t N,
                      cudaStream_t st);
void launch_sd_count(SdState* s, cudaStream_t st);
template <typename R>
void launch_normalise(R* m, int64_t N, cudaStream_t st);
template <typename R>
void launch_max_dm(const R* a, const R* alo, const R* b, const R* blo, int64_t N, double* partials, double* out,
                   cudaStream_t st);
template <typename R>
void launch_absmax(const R* v, int64_t n, double* partials, double* out, cudaStream_t st);

}  // namespace mm

// mm_oracle.cpp -- CPU FP64 restatement of the MicroMagnetic.jl finite-difference
// hot path (effective field, LLG right-hand side, RK4 / Dormand-Prince, SD relax).
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker: it is loaded by tests/,
// by __graft_entry__.smoke() and by bench.py's CPU-baseline leg.  The product
// library (libmmcuda.so) never links, loads or calls it.
//
// Every routine cites the reference file:line whose behaviour it restates
// (paths relative to the MicroMagnetic.jl project root).  Array conventions
// follow the reference: m, H are AoS [mx1,my1,mz1,mx2,...], cell id
// (k*ny + j)*nx + i with x fastest (src/micro/mesh.jl:24-29, 0-based here).
#include <quadmath.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

using cd = std::complex<double>;
constexpr double kPi = 3.14159265358979323846;
constexpr double kMu0 = 4.0 * kPi * 1e-7;  // src/const.jl:1

// ---------------------------------------------------------------------------
// Mesh and neighbour table: src/micro/mesh.jl:24-43 (index, indexpbc) and
// mesh.jl:69-98 (FDMesh constructor).  ngb[6*id + d] = neighbour id or -1, with
// d = 0:-x 1:+x 2:-y 3:+y 4:-z 5:+z.
// ---------------------------------------------------------------------------
struct Mesh {
  int nx = 1, ny = 1, nz = 1;
  double dx = 1e-9, dy = 1e-9, dz = 1e-9;
  bool px = false, py = false, pz = false;
  int64_t n = 1;
  double volume = 1e-27;
  std::vector<int64_t> ngb;

  int64_t index_pbc(int i, int j, int k) const {
    if (px) { if (i < 0) i += nx; if (i >= nx) i -= nx; }
    if (py) { if (j < 0) j += ny; if (j >= ny) j -= ny; }
    if (pz) { if (k < 0) k += nz; if (k >= nz) k -= nz; }
    if (i < 0 || j < 0 || k < 0 || i >= nx || j >= ny || k >= nz) return -1;
    return (static_cast<int64_t>(k) * ny + j) * nx + i;
  }
  void build() {
    n = static_cast<int64_t>(nx) * ny * nz;
    volume = dx * dy * dz;
    ngb.assign(6 * n, -1);
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          int64_t id = (static_cast<int64_t>(k) * ny + j) * nx + i;
          ngb[6 * id + 0] = index_pbc(i - 1, j, k);
          ngb[6 * id + 1] = index_pbc(i + 1, j, k);
          ngb[6 * id + 2] = index_pbc(i, j - 1, k);
          ngb[6 * id + 3] = index_pbc(i, j + 1, k);
          ngb[6 * id + 4] = index_pbc(i, j, k - 1);
          ngb[6 * id + 5] = index_pbc(i, j, k + 1);
        }
  }
};

// a x b with the component formulas of src/util.jl:6-16.
inline void cross3(double a1, double a2, double a3, double b1, double b2, double b3,
                   double& c1, double& c2, double& c3) {
  c1 = -a3 * b2 + a2 * b3;
  c2 = a3 * b1 - a1 * b3;
  c3 = -a2 * b1 + a1 * b2;
}

// ---------------------------------------------------------------------------
// Plain mixed-radix FFT (any length; O(n * p) per level for a prime factor p).
// Stands in for FFTW's plan_rfft/plan_irfft used at src/micro/demag.jl:49,91.
// Forward: X[k] = sum_n x[n] exp(-2 pi i k n / N); inverse unnormalised.
// ---------------------------------------------------------------------------
struct Fft1 {
  int n;
  std::vector<cd> w;  // exp(-2 pi i j / n)
  explicit Fft1(int n_) : n(n_), w(n_) {
    for (int j = 0; j < n; ++j) {
      double a = -2.0 * kPi * static_cast<double>(j) / static_cast<double>(n);
      w[j] = cd(std::cos(a), std::sin(a));
    }
  }
  static int smallest_factor(int m) {
    for (int p : {4, 2, 3, 5, 7}) if (m % p == 0) return p;
    for (int p = 11; p * p <= m; p += 2) if (m % p == 0) return p;
    return m;
  }
  // out[0..m) = DFT_m of in[0], in[s], ..., using twiddle table of size n (m | n)
  void rec(const cd* in, int s, cd* out, int m, cd* tmp) const {
    if (m == 1) { out[0] = in[0]; return; }
    int p = smallest_factor(m);
    int q = m / p;
    for (int r = 0; r < p; ++r) rec(in + static_cast<int64_t>(r) * s, s * p, out + r * q, q, tmp);
    int step = n / m;  // W_m^t = w[t * step]
    for (int k = 0; k < q; ++k) {
      for (int c = 0; c < p; ++c) {
        cd acc = 0.0;
        int kk = k + c * q;
        for (int r = 0; r < p; ++r) {
          int64_t e = (static_cast<int64_t>(r) * kk) % m;
          acc += out[r * q + k] * w[e * step];
        }
        tmp[c] = acc;
      }
      for (int c = 0; c < p; ++c) out[k + c * q] = tmp[c];
    }
  }
  void forward(const cd* in, cd* out) const {
    std::vector<cd> tmp(n);
    rec(in, 1, out, n, tmp.data());
  }
};

std::mutex g_fft_mu;
std::map<int, std::shared_ptr<Fft1>> g_fft_cache;
std::shared_ptr<Fft1> get_fft(int n) {
  std::lock_guard<std::mutex> g(g_fft_mu);
  auto it = g_fft_cache.find(n);
  if (it != g_fft_cache.end()) return it->second;
  auto p = std::make_shared<Fft1>(n);
  g_fft_cache[n] = p;
  return p;
}

// In-place 3-D complex FFT of a (Pz, Py, Px) array, x fastest.  inverse uses
// conj(FFT(conj x)) and is NOT normalised.
void fft3(std::vector<cd>& a, int Px, int Py, int Pz, bool inverse) {
  const int dims[3] = {Px, Py, Pz};
  const int64_t strides[3] = {1, Px, static_cast<int64_t>(Px) * Py};
  for (int ax = 0; ax < 3; ++ax) {
    int L = dims[ax];
    if (L == 1) continue;
    auto plan = get_fft(L);
    int64_t total = static_cast<int64_t>(Px) * Py * Pz;
    int64_t nlines = total / L;
    int64_t st = strides[ax];
#pragma omp parallel
    {
      std::vector<cd> buf(L), out(L);
#pragma omp for schedule(static)
      for (int64_t line = 0; line < nlines; ++line) {
        // decompose line index into base offset
        int64_t base;
        if (ax == 0) base = line * Px;
        else if (ax == 1) { int64_t z = line / Px, x = line % Px; base = z * Px * Py + x; }
        else base = line;
        for (int t = 0; t < L; ++t) {
          cd v = a[base + t * st];
          buf[t] = inverse ? std::conj(v) : v;
        }
        plan->forward(buf.data(), out.data());
        for (int t = 0; t < L; ++t) a[base + t * st] = inverse ? std::conj(out[t]) : out[t];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Newell demag tensor: src/micro/demag.jl:133-296 (newell_f, newell_g,
// demag_tensor_xx/xy and their permutations) and the far-field dipole
// switch using src/atomistic/demag.jl:106-138 (dipolar_tensor_xx/xy).
// Newell, Williams & Dunlop, J. Geophys. Res. 98 (1993) 9551.
// ---------------------------------------------------------------------------
double newell_f(double x, double y, double z) {
  double x2 = x * x, y2 = y * y, z2 = z * z;
  double R = std::sqrt(x2 + y2 + z2);
  if (R == 0.0) return 0.0;
  double f = 1.0 / 6 * (2 * x2 - y2 - z2) * R;
  if (x2 > 0) f -= x * y * z * std::atan(y * z / (x * R));
  if (x2 + z2 > 0) f += 0.5 * y * (z2 - x2) * std::asinh(y / std::sqrt(x2 + z2));
  if (x2 + y2 > 0) f += 0.5 * z * (y2 - x2) * std::asinh(z / std::sqrt(x2 + y2));
  return f;
}

double newell_g(double x, double y, double z) {
  double x2 = x * x, y2 = y * y, z2 = z * z;
  double R = std::sqrt(x2 + y2 + z2);
  if (R == 0.0) return 0.0;
  double g = -1.0 / 3 * x * y * R;
  if (z2 > 0) g -= 1.0 / 6 * z2 * z * std::atan(x * y / (z * R));
  if (y2 > 0) g -= 0.5 * y2 * z * std::atan(x * z / (y * R));
  if (x2 > 0) g -= 0.5 * x2 * z * std::atan(y * z / (x * R));
  if (x2 + y2 > 0) g += x * y * z * std::asinh(z / std::sqrt(x2 + y2));
  if (y2 + z2 > 0) g += 1.0 / 6 * y * (3 * z2 - y2) * std::asinh(x / std::sqrt(y2 + z2));
  if (x2 + z2 > 0) g += 1.0 / 6 * x * (3 * z2 - x2) * std::asinh(y / std::sqrt(x2 + z2));
  return g;
}

double dipole_xx(double x, double y, double z) {
  double R = x * x + y * y + z * z;
  if (R == 0) return 0.0;
  return -(2 * x * x - y * y - z * z) / (R * R * std::sqrt(R));
}
double dipole_xy(double x, double y, double z) {
  double R = x * x + y * y + z * z;
  if (R == 0) return 0.0;
  return -3 * x * y / (R * R * std::sqrt(R));
}

// 27-point second difference in the reference's own order and FP64
// arithmetic: demag_tensor_xx / demag_tensor_xy (demag.jl:194-296):
// 8 f(0), then -4 f at the six face offsets, +2 f at the twelve edge offsets,
// -f at the eight corners, accumulated left to right.
template <typename F>
double newell_sum(F fn, double x, double y, double z, double dx, double dy, double dz) {
  double t = 8.0 * fn(x, y, z);
  t -= 4.0 * fn(x + dx, y, z);
  t -= 4.0 * fn(x - dx, y, z);
  t -= 4.0 * fn(x, y - dy, z);
  t -= 4.0 * fn(x, y + dy, z);
  t -= 4.0 * fn(x, y, z - dz);
  t -= 4.0 * fn(x, y, z + dz);
  t += 2.0 * fn(x + dx, y + dy, z);
  t += 2.0 * fn(x + dx, y - dy, z);
  t += 2.0 * fn(x - dx, y - dy, z);
  t += 2.0 * fn(x - dx, y + dy, z);
  t += 2.0 * fn(x + dx, y, z + dz);
  t += 2.0 * fn(x + dx, y, z - dz);
  t += 2.0 * fn(x - dx, y, z + dz);
  t += 2.0 * fn(x - dx, y, z - dz);
  t += 2.0 * fn(x, y - dy, z - dz);
  t += 2.0 * fn(x, y - dy, z + dz);
  t += 2.0 * fn(x, y + dy, z + dz);
  t += 2.0 * fn(x, y + dy, z - dz);
  t -= fn(x + dx, y + dy, z + dz);
  t -= fn(x + dx, y + dy, z - dz);
  t -= fn(x + dx, y - dy, z + dz);
  t -= fn(x + dx, y - dy, z - dz);
  t -= fn(x - dx, y + dy, z + dz);
  t -= fn(x - dx, y + dy, z - dz);
  t -= fn(x - dx, y - dy, z + dz);
  t -= fn(x - dx, y - dy, z - dz);
  return t;
}

// R in cells as demag_tensor_xx computes it (demag.jl:196)
double cells_R(double x, double y, double z, double dx, double dy, double dz) {
  return std::sqrt(x * x + y * y + z * z) / std::max(dx, std::max(dy, dz));
}

double tensor_xx(double x, double y, double z, double dx, double dy, double dz) {
  if (cells_R(x, y, z, dx, dy, dz) > 60) return dipole_xx(x, y, z) * dx * dy * dz / (4 * kPi);
  return newell_sum(newell_f, x, y, z, dx, dy, dz) / (4.0 * kPi * dx * dy * dz);
}
double tensor_xy(double x, double y, double z, double dx, double dy, double dz) {
  if (cells_R(x, y, z, dx, dy, dz) > 60) return dipole_xy(x, y, z) * dx * dy * dz / (4 * kPi);
  return newell_sum(newell_g, x, y, z, dx, dy, dz) / (4.0 * kPi * dx * dy * dz);
}
// component c: 0 xx, 1 yy, 2 zz, 3 xy, 4 xz, 5 yz (demag.jl:188-296)
double tensor_comp(int c, double x, double y, double z, double dx, double dy, double dz) {
  switch (c) {
    case 0: return tensor_xx(x, y, z, dx, dy, dz);
    case 1: return tensor_xx(y, x, z, dy, dx, dz);
    case 2: return tensor_xx(z, y, x, dz, dy, dx);
    case 3: return tensor_xy(x, y, z, dx, dy, dz);
    case 4: return tensor_xy(x, z, y, dx, dz, dy);
    default: return tensor_xy(y, z, x, dy, dz, dx);
  }
}

// ---------------------------------------------------------------------------
// Accurate tensor (the default): the same Newell formulas evaluated in IEEE
// binary128 (__float128, libquadmath's sqrtq / atanq / asinhq) at the exact
// coordinates X * dx (X an integer offset: the product of an int32 and a
// double is exact in binary128).  The 27-point differences cancel up to
// R^6 (5e10 at R = 60 cells) of the function values; with a 113-bit
// significand the near-field entries keep ~1e-23 relative accuracy, so each
// rounds correctly to FP64.  The far-field dipole terms (no cancellation)
// keep the reference's FP64 formula; image sums are accumulated in binary128
// and rounded once.  The switch R > 60 is the reference's FP64 test.
// ---------------------------------------------------------------------------
using q128 = __float128;
bool g_reference_tensor = false;  // orc_set_reference_tensor

q128 qf(q128 x, q128 y, q128 z) {
  const q128 x2 = x * x, y2 = y * y, z2 = z * z;
  const q128 R = sqrtq(x2 + y2 + z2);
  if (R == 0) return 0;
  q128 f = (2 * x2 - y2 - z2) * R / 6;
  if (x2 > 0) f -= x * y * z * atanq(y * z / (x * R));
  if (x2 + z2 > 0) f += y * (z2 - x2) * asinhq(y / sqrtq(x2 + z2)) / 2;
  if (x2 + y2 > 0) f += z * (y2 - x2) * asinhq(z / sqrtq(x2 + y2)) / 2;
  return f;
}

q128 qg(q128 x, q128 y, q128 z) {
  const q128 x2 = x * x, y2 = y * y, z2 = z * z;
  const q128 R = sqrtq(x2 + y2 + z2);
  if (R == 0) return 0;
  q128 g = -x * y * R / 3;
  if (z2 > 0) g -= z2 * z * atanq(x * y / (z * R)) / 6;
  if (y2 > 0) g -= y2 * z * atanq(x * z / (y * R)) / 2;
  if (x2 > 0) g -= x2 * z * atanq(y * z / (x * R)) / 2;
  if (x2 + y2 > 0) g += x * y * z * asinhq(z / sqrtq(x2 + y2));
  if (y2 + z2 > 0) g += y * (3 * z2 - y2) * asinhq(x / sqrtq(y2 + z2)) / 6;
  if (x2 + z2 > 0) g += x * (3 * z2 - x2) * asinhq(y / sqrtq(x2 + z2)) / 6;
  return g;
}

// f or g of component c at integer offsets, arguments permuted as
// demag_tensor_yy / zz / xz / yz (demag.jl:236-296) do
q128 q_newell(int c, int64_t X, int64_t Y, int64_t Z, double dx, double dy, double dz) {
  const q128 x = static_cast<q128>(X) * dx, y = static_cast<q128>(Y) * dy, z = static_cast<q128>(Z) * dz;
  switch (c) {
    case 0: return qf(x, y, z);
    case 1: return qf(y, x, z);
    case 2: return qf(z, y, x);
    case 3: return qg(x, y, z);
    case 4: return qg(x, z, y);
    default: return qg(y, z, x);
  }
}

// Real-space tensor out[c*N + I] (6 x N, xx yy zz xy xz yz) for normalised
// cell sizes, with macro-PBC images (tensors_kernel_*!, demag.jl:298-386).
// accurate = false: the reference's FP64 arithmetic (tensor_comp).
void newell_table(int nx, int ny, int nz, double dx, double dy, double dz, int Nx, int Ny, int Nz, bool accurate,
                  double* out) {
  const int64_t N = static_cast<int64_t>(nx) * ny * nz;
  // near-field function table over offsets 0..e (f even in each argument,
  // g odd in its first two): R <= 60 cells plus the stencil's +-1
  auto extent = [](double d, int n, int Nimg) {
    return static_cast<int>(std::min(std::floor(60.0 / d) + 2.0, static_cast<double>(n - 1) + Nimg * 1.0 * n + 1.0));
  };
  const int ex = extent(dx, nx, Nx), ey = extent(dy, ny, Ny), ez = extent(dz, nz, Nz);
  const int64_t gx = ex + 1, gy = ey + 1, gz = ez + 1;
  const bool odd[6][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}};
  std::vector<q128> F;
  if (accurate) {
    F.resize(static_cast<size_t>(6 * gx * gy * gz));
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t t = 0; t < 6 * gx * gy * gz; ++t) {
      const int64_t X = t % gx, Y = (t / gx) % gy, Z = (t / (gx * gy)) % gz;
      const int c = static_cast<int>(t / (gx * gy * gz));
      F[static_cast<size_t>(t)] = q_newell(c, X, Y, Z, dx, dy, dz);
    }
  }
  auto at = [&](int c, int64_t X, int64_t Y, int64_t Z) -> q128 {
    const int64_t ax = X < 0 ? -X : X, ay = Y < 0 ? -Y : Y, az = Z < 0 ? -Z : Z;
    if (ax > ex || ay > ey || az > ez) return q_newell(c, X, Y, Z, dx, dy, dz);
    const q128 v = F[static_cast<size_t>(((c * gz + az) * gy + ay) * gx + ax)];
    const bool flip = (odd[c][0] && X < 0) != ((odd[c][1] && Y < 0) != (odd[c][2] && Z < 0));
    return flip ? -v : v;
  };
  const q128 qpi = 4 * atanq(static_cast<q128>(1));
  const q128 inv_near = 1 / (4 * qpi * static_cast<q128>(dx) * dy * dz);
  for (int c = 0; c < 6; ++c) {
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t I = 0; I < N; ++I) {
      const int i = static_cast<int>(I % nx), j = static_cast<int>((I / nx) % ny),
                k = static_cast<int>(I / (static_cast<int64_t>(nx) * ny));
      double sum = 0.0;
      q128 qsum = 0;
      for (int p = -Nx; p <= Nx; ++p)
        for (int q = -Ny; q <= Ny; ++q)
          for (int r = -Nz; r <= Nz; ++r) {
            const int64_t X = i + static_cast<int64_t>(p) * nx, Y = j + static_cast<int64_t>(q) * ny,
                          Z = k + static_cast<int64_t>(r) * nz;
            const double x = static_cast<double>(X) * dx, y = static_cast<double>(Y) * dy,
                         z = static_cast<double>(Z) * dz;
            if (!accurate) {
              sum += tensor_comp(c, x, y, z, dx, dy, dz);
              continue;
            }
            if (cells_R(x, y, z, dx, dy, dz) > 60) {
              qsum += tensor_comp(c, x, y, z, dx, dy, dz);
              continue;
            }
            q128 s = 0;
            for (int a = -1; a <= 1; ++a)
              for (int b = -1; b <= 1; ++b)
                for (int e = -1; e <= 1; ++e) {
                  const int w = (a == 0 ? 2 : -1) * (b == 0 ? 2 : -1) * (e == 0 ? 2 : -1);
                  s += w * at(c, X + a, Y + b, Z + e);
                }
            qsum += s * inv_near;
          }
      out[c * N + I] = accurate ? static_cast<double>(qsum) : sum;
    }
  }
}

// ---------------------------------------------------------------------------
// Terms (src/head.jl:150-310).  Each keeps its own field (3N) and energy (N)
// buffers, exactly like the reference's interaction structs.
// ---------------------------------------------------------------------------
enum TermKind {
  T_ZEEMAN = 0, T_EXCH = 1, T_DMI_BULK = 2, T_DMI_INTERFACIAL = 3, T_ANIS = 4, T_DEMAG = 5,
  T_DMI_BULK_SPATIAL = 6, T_SOT = 7, T_STT_ZL = 8, T_STT_SL = 9, T_THERMAL = 10
};

struct Term {
  TermKind kind;
  // exchange (uniform: Ax,Ay,Az; spatial: A array)
  double Ax = 0, Ay = 0, Az = 0;
  std::vector<double> A;
  // bulk DMI
  double Dx = 0, Dy = 0, Dz = 0;
  // interfacial DMI
  std::vector<double> D;
  // anisotropy
  std::vector<double> Ku;
  double ux = 0, uy = 0, uz = 1;
  // zeeman field (A/m)
  std::vector<double> H;
  // demag
  int Px = 1, Py = 1, Pz = 1;
  std::vector<double> Nhat[6];  // real spectra, full (Pz,Py,Px) grid
  // spatial bulk DMI (per-axis arrays)
  std::vector<double> bD[3];
  // SOT (DFTorqueField): aj per cell, bj, p
  std::vector<double> aj;
  double bj = 0, p[3] = {0, 0, 0};
  // Zhang-Li: b*J (AoS 3N), xi per cell, ft;  Slonczewski: J per cell, ft*beta, Lambda, P, xi, p
  std::vector<double> bJ, xi, J;
  double ft = 1.0, ftb = 0.0, Lambda = 2.0, P = 0.0, xi_s = 0.0;
  // thermal: T per cell, T0, scaling, k_B, seed, dt outside a step
  std::vector<double> T;
  double T0 = 0.0, scaling = 1.0, kB = 1.3806505e-23, dt = 1e-14;
  uint64_t seed = 0;
  std::vector<double> field, energy;
};

struct Sim {
  Mesh mesh;
  std::vector<double> mu0Ms;  // Tesla (src/sim.jl:138)
  std::vector<double> m;      // spin
  std::vector<double> prespin;
  std::vector<uint8_t> pins;
  std::vector<std::unique_ptr<Term>> terms;
  std::vector<double> field;  // total H_eff
  double alpha = 0.1, gamma = 2.21e5;  // src/driver.jl:148
  bool precession = true;
  // RK4 (src/integrator/rk.jl:3-52)
  double rk_t = 0.0;
  int64_t rk_nsteps = 0;
  // Dormand-Prince (src/integrator/adaptive_rk.jl:37-86)
  double tol = 1e-6, t = 0.0, step = 0.0, step_next = 0.0;
  double facmax = 5.0, facmin = 0.2, safety = 0.824;
  int64_t nsteps = 0, nfevals = 0;
  bool succeed = false;
  int method = 0;  // 0 DOPRI54, 1 BS23, 2 CashKarp54, 3 Fehlberg54
  // thermal noise: fixed-step counter; the (step, dt) the current evaluation draws for
  int64_t th_step = 0;
  int64_t th_cur_step = 0;
  double th_cur_dt = 0.0;
  double th_dt = 1e-14;  // dt of evaluations outside a step: the add-time value, then the last fixed step
  std::vector<double> y_current, y_next, y_temp;
  std::vector<double> ks[7];
  // SD driver (src/sd.jl; src/driver.jl:95-102)
  std::vector<double> gk, ss, sf, ff;
  double tau = 0.0, max_tau = 1.0, min_tau = 1e-10;
  int64_t sd_steps = 0;
  int threads = 0;
};

// ----- per-term field kernels (src/micro/kernels.jl) -----------------------

// uniform_exchange_kernel!  kernels.jl:269-304
void exch_uniform(const Sim& s, const Term& tm, const double* m, double* h, double* e) {
  const Mesh& g = s.mesh;
  const double ax = 2 * tm.Ax / (g.dx * g.dx), ay = 2 * tm.Ay / (g.dy * g.dy),
               az = 2 * tm.Az / (g.dz * g.dz);
  const double nabla[6] = {ax, ax, ay, ay, az, az};
#pragma omp parallel for schedule(static)
  for (int64_t I = 0; I < g.n; ++I) {
    double Ms = s.mu0Ms[I];
    int64_t i = 3 * I;
    if (Ms == 0.0) { e[I] = 0; h[i] = h[i + 1] = h[i + 2] = 0; continue; }
    double fx = 0, fy = 0, fz = 0;
    for (int d = 0; d < 6; ++d) {
      int64_t id = g.ngb[6 * I + d];
      if (id >= 0 && s.mu0Ms[id] > 0) {
        int64_t k = 3 * id;
        fx += nabla[d] * (m[k] - m[i]);
        fy += nabla[d] * (m[k + 1] - m[i + 1]);
        fz += nabla[d] * (m[k + 2] - m[i + 2]);
      }
    }
    double Ms_inv = 1.0 / Ms;
    e[I] = -0.5 * (fx * m[i] + fy * m[i + 1] + fz * m[i + 2]) * g.volume;
    h[i] = fx * Ms_inv; h[i + 1] = fy * Ms_inv; h[i + 2] = fz * Ms_inv;
  }
}

// exchange_kernel! (spatial A, harmonic mean)  kernels.jl:226-266
void exch_spatial(const Sim& s, const Term& tm, const double* m, double* h, double* e) {
  const Mesh& g = s.mesh;
  const double ax = 2.0 / (g.dx * g.dx), ay = 2.0 / (g.dy * g.dy), az = 2.0 / (g.dz * g.dz);
  const double nabla[6] = {ax, ax, ay, ay, az, az};
  const double* A = tm.A.data();
#pragma omp parallel for schedule(static)
  for (int64_t I = 0; I < g.n; ++I) {
    double Ms = s.mu0Ms[I];
    double AI = A[I];
    int64_t i = 3 * I;
    if (Ms == 0.0 || AI == 0.0) { e[I] = 0; h[i] = h[i + 1] = h[i + 2] = 0; continue; }
    double fx = 0, fy = 0, fz = 0;
    for (int d = 0; d < 6; ++d) {
      int64_t id = g.ngb[6 * I + d];
      if (id >= 0 && s.mu0Ms[id] > 0) {
        double An = A[id];
        if (An != 0.0) {
          int64_t k = 3 * id;
          double Aeff = 2 * AI * An / (AI + An);
          double c = Aeff * nabla[d];
          fx += c * (m[k] - m[i]);
          fy += c * (m[k + 1] - m[i + 1]);
          fz += c * (m[k + 2] - m[i + 2]);
        }
      }
    }
    double Ms_inv = 1.0 / Ms;
    e[I] = -0.5 * (fx * m[i] + fy * m[i + 1] + fz * m[i + 2]) * g.volume;
    h[i] = fx * Ms_inv; h[i + 1] = fy * Ms_inv; h[i + 2] = fz * Ms_inv;
  }
}

// bulkdmi_kernel!  kernels.jl:306-344
void dmi_bulk(const Sim& s, const Term& tm, const double* m, double* h, double* e) {
  const Mesh& g = s.mesh;
  const double Ds[6] = {tm.Dx / g.dx, tm.Dx / g.dx, tm.Dy / g.dy, tm.Dy / g.dy, tm.Dz / g.dz, tm.Dz / g.dz};
  const double ax[6] = {1, -1, 0, 0, 0, 0}, ay[6] = {0, 0, 1, -1, 0, 0}, az[6] = {0, 0, 0, 0, 1, -1};
#pragma omp parallel for schedule(static)
  for (int64_t I = 0; I < g.n; ++I) {
    double Ms = s.mu0Ms[I];
    int64_t i = 3 * I;
    if (Ms == 0.0) { e[I] = 0; h[i] = h[i + 1] = h[i + 2] = 0; continue; }
    double fx = 0, fy = 0, fz = 0;
    for (int d = 0; d < 6; ++d) {
      int64_t id = g.ngb[6 * I + d];
      if (id >= 0 && s.mu0Ms[id] > 0) {
        int64_t k = 3 * id;
        double cx, cy, cz;
        cross3(ax[d], ay[d], az[d], m[k], m[k + 1], m[k + 2], cx, cy, cz);
        fx += Ds[d] * cx; fy += Ds[d] * cy; fz += Ds[d] * cz;
      }
    }
    double Ms_inv = 1.0 / Ms;
    e[I] = -0.5 * (fx * m[i] + fy * m[i + 1] + fz * m[i + 2]) * g.volume;
    h[i] = fx * Ms_inv; h[i + 1] = fy * Ms_inv; h[i + 2] = fz * Ms_inv;
  }
}

// interfacial_dmi_kernel!  kernels.jl:426-466
void dmi_interfacial(const Sim& s, const Term& tm, const double* m, double* h, double* e) {
  const Mesh& g = s.mesh;
  const double Dd[4] = {1 / g.dx, 1 / g.dx, 1 / g.dy, 1 / g.dy};
  const double ax[4] = {0, 0, -1, 1}, ay[4] = {1, -1, 0, 0}, az[4] = {0, 0, 0, 0};
  const double* D = tm.D.data();
#pragma omp parallel for schedule(static)
  for (int64_t I = 0; I < g.n; ++I) {
    double Ms = s.mu0Ms[I];
    double DI = D[I];
    int64_t i = 3 * I;
    if (Ms == 0.0 || DI == 0.0) { e[I] = 0; h[i] = h[i + 1] = h[i + 2] = 0; continue; }
    double fx = 0, fy = 0, fz = 0;
    for (int d = 0; d < 4; ++d) {
      int64_t id = g.ngb[6 * I + d];
      if (id >= 0 && s.mu0Ms[id] > 0) {
        double Dn = D[id];
        if (Dn != 0.0) {
          int64_t k = 3 * id;
          double Deff = 2 * DI * Dn / (DI + Dn);
          double c = Deff * Dd[d];
          double cx, cy, cz;
          cross3(ax[d], ay[d], az[d], m[k], m[k + 1], m[k + 2], cx, cy, cz);
          fx += c * cx; fy += c * cy; fz += c * cz;
        }
      }
    }
    double Ms_inv = 1.0 / Ms;
    e[I] = -0.5 * (fx * m[i] + fy * m[i + 1] + fz * m[i + 2]) * g.volume;
    h[i] = fx * Ms_inv; h[i + 1] = fy * Ms_inv; h[i + 2] = fz * Ms_inv;
  }
}

// anisotropy_kernel!  kernels.jl:54-75
void anis_uniaxial(const Sim& s, const Term& tm, const double* m, double* h, double* e) {
  const Mesh& g = s.mesh;
  const double* Ku = tm.Ku.data();
#pragma omp parallel for schedule(static)
  for (int64_t I = 0; I < g.n; ++I) {
    double Ms = s.mu0Ms[I];
    int64_t i = 3 * I;
    if (Ms == 0.0) { e[I] = 0; h[i] = h[i + 1] = h[i + 2] = 0; continue; }
    double Ms_inv = 2.0 / Ms;
    double sa = m[i] * tm.ux + m[i + 1] * tm.uy + m[i + 2] * tm.uz;
    h[i] = Ku[I] * sa * tm.ux * Ms_inv;
    h[i + 1] = Ku[I] * sa * tm.uy * Ms_inv;
    h[i + 2] = Ku[I] * sa * tm.uz * Ms_inv;
    e[I] = Ku[I] * (1.0 - sa * sa) * g.volume;
  }
}

// zeeman_kernel!  kernels.jl:14-20 (energy only; the field is constant)
void zeeman(const Sim& s, const Term& tm, const double* m, double* h, double* e) {
  const Mesh& g = s.mesh;
  std::copy(tm.H.begin(), tm.H.end(), h);
#pragma omp parallel for schedule(static)
  for (int64_t I = 0; I < g.n; ++I) {
    int64_t j = 3 * I;
    double mh = m[j] * h[j] + m[j + 1] * h[j + 1] + m[j + 2] * h[j + 2];
    e[I] = -g.volume * s.mu0Ms[I] * mh;
  }
}

// ----- demag: src/micro/demag.jl:30-131, 394-489 ----------------------------
int padded_len(int n) { return n > 3 ? 2 * n : 2 * n - 1; }  // demag.jl:41-44

void demag_init(const Sim& s, Term& tm, int Nx, int Ny, int Nz, const double* tensor_override) {
  const Mesh& g = s.mesh;
  const double mx = std::max(g.dx, std::max(g.dy, g.dz));
  const double dx = g.dx / mx, dy = g.dy / mx, dz = g.dz / mx;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  tm.Px = padded_len(nx); tm.Py = padded_len(ny); tm.Pz = padded_len(nz);
  const int Px = tm.Px, Py = tm.Py, Pz = tm.Pz;
  const int64_t P = static_cast<int64_t>(Px) * Py * Pz;
  const int64_t N = g.n;
  std::vector<double> t(N);
  std::vector<cd> pad(P);
  // tensors_kernel_*!  demag.jl:298-386 (macro-PBC image sums)
  std::vector<double> table;
  if (!tensor_override) {
    table.resize(static_cast<size_t>(6 * N));
    newell_table(nx, ny, nz, dx, dy, dz, Nx, Ny, Nz, !g_reference_tensor, table.data());
  }
  // tensor components and the odd axes of each (fill_tensors calls, demag.jl:56-83)
  const bool odd[6][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}};
  for (int c = 0; c < 6; ++c) {
    if (tensor_override) {
      std::copy(tensor_override + c * N, tensor_override + (c + 1) * N, t.begin());
    } else {
      std::copy(table.begin() + c * N, table.begin() + (c + 1) * N, t.begin());
    }
    // fill_tensors_kernel!  demag.jl:394-412
    std::fill(pad.begin(), pad.end(), cd(0.0, 0.0));
    for (int k = 0; k < Pz; ++k)
      for (int j = 0; j < Py; ++j)
        for (int i = 0; i < Px; ++i) {
          if ((Px % 2 == 0 && i == nx) || (Py % 2 == 0 && j == ny) || (Pz % 2 == 0 && k == nz)) continue;
          int x = i < nx ? i : Px - i, y = j < ny ? j : Py - j, z = k < nz ? k : Pz - k;
          int sx = (odd[c][0] && i >= nx) ? -1 : 1;
          int sy = (odd[c][1] && j >= ny) ? -1 : 1;
          int sz = (odd[c][2] && k >= nz) ? -1 : 1;
          pad[(static_cast<int64_t>(k) * Py + j) * Px + i] =
              static_cast<double>(sx * sy * sz) * t[(static_cast<int64_t>(z) * ny + y) * nx + x];
        }
    fft3(pad, Px, Py, Pz, false);
    tm.Nhat[c].resize(P);
    for (int64_t p = 0; p < P; ++p) tm.Nhat[c][p] = pad[p].real();  // real(plan * mx_pad)
  }
}

// effective_field(::Demag)  demag.jl:102-131 with distribute_m (419-433),
// add_tensor_M (463-489) and collect_h (435-456).
void demag_field(const Sim& s, const Term& tm, const double* m, double* h, double* e) {
  const Mesh& g = s.mesh;
  const int nx = g.nx, ny = g.ny, nz = g.nz, Px = tm.Px, Py = tm.Py, Pz = tm.Pz;
  const int64_t P = static_cast<int64_t>(Px) * Py * Pz;
  std::vector<cd> M[3];
  for (int c = 0; c < 3; ++c) M[c].assign(P, cd(0.0, 0.0));
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        int64_t I = (static_cast<int64_t>(k) * ny + j) * nx + i;
        int64_t p = (static_cast<int64_t>(k) * Py + j) * Px + i;
        for (int c = 0; c < 3; ++c) M[c][p] = m[3 * I + c] * s.mu0Ms[I];
      }
  for (int c = 0; c < 3; ++c) fft3(M[c], Px, Py, Pz, false);
  const auto &xx = tm.Nhat[0], &yy = tm.Nhat[1], &zz = tm.Nhat[2], &xy = tm.Nhat[3],
             &xz = tm.Nhat[4], &yz = tm.Nhat[5];
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < P; ++p) {
    cd a = M[0][p], b = M[1][p], c = M[2][p];
    M[0][p] = xx[p] * a + xy[p] * b + xz[p] * c;
    M[1][p] = xy[p] * a + yy[p] * b + yz[p] * c;
    M[2][p] = xz[p] * a + yz[p] * b + zz[p] * c;
  }
  for (int c = 0; c < 3; ++c) fft3(M[c], Px, Py, Pz, true);
  const double scale = 1.0 / static_cast<double>(P);
  const double factor = -1.0 / kMu0;
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        int64_t I = (static_cast<int64_t>(k) * ny + j) * nx + i;
        int64_t p = (static_cast<int64_t>(k) * Py + j) * Px + i;
        for (int c = 0; c < 3; ++c) h[3 * I + c] = factor * (M[c][p].real() * scale);
        double mh = m[3 * I] * h[3 * I] + m[3 * I + 1] * h[3 * I + 1] + m[3 * I + 2] * h[3 * I + 2];
        e[I] = -0.5 * s.mu0Ms[I] * g.volume * mh;
      }
}

// spatial_vector_bulkdmi_kernel!  src/micro/kernels.jl:347-422
void dmi_bulk_spatial(const Sim& s, const Term& tm, const double* m, double* h, double* e) {
  const Mesh& g = s.mesh;
  const double axes[6] = {1 / g.dx, -1 / g.dx, 1 / g.dy, -1 / g.dy, 1 / g.dz, -1 / g.dz};
#pragma omp parallel for schedule(static)
  for (int64_t I = 0; I < g.n; ++I) {
    const int64_t i = 3 * I;
    const double Ms = s.mu0Ms[I];
    if (Ms == 0.0) { e[I] = 0; h[i] = h[i + 1] = h[i + 2] = 0; continue; }
    double fx = 0, fy = 0, fz = 0;
    for (int d = 0; d < 6; ++d) {
      const int64_t id = g.ngb[6 * I + d];
      if (id < 0 || !(s.mu0Ms[id] > 0)) continue;
      const int ax = d / 2;
      const double Di = tm.bD[ax][I], Dn = tm.bD[ax][id];
      if (Di == 0 || Dn == 0) continue;
      const double Deff = 2 * Di * Dn / (Di + Dn), a = axes[d];
      const int64_t k = 3 * id;
      if (ax == 0) { fy += Deff * (-a * m[k + 2]); fz += Deff * (a * m[k + 1]); }
      else if (ax == 1) { fx += Deff * (a * m[k + 2]); fz += Deff * (-a * m[k]); }
      else { fx += Deff * (-a * m[k + 1]); fy += Deff * (a * m[k]); }
    }
    const double Ms_inv = 1.0 / Ms;
    e[I] = -0.5 * (fx * m[i] + fy * m[i + 1] + fz * m[i + 2]) * g.volume;
    h[i] = fx * Ms_inv; h[i + 1] = fy * Ms_inv; h[i + 2] = fz * Ms_inv;
  }
}

// df_torque_kernel!  src/micro/kernels.jl:619-632
void sot_field(const Sim& s, const Term& tm, const double* m, double* h, double* e) {
  const Mesh& g = s.mesh;
  for (int64_t I = 0; I < g.n; ++I) {
    const int64_t j = 3 * I;
    const double a = tm.aj[I] / s.gamma, b = tm.bj / s.gamma;
    double cx, cy, cz;
    cross3(m[j], m[j + 1], m[j + 2], tm.p[0], tm.p[1], tm.p[2], cx, cy, cz);
    h[j] = a * cx + b * tm.p[0]; h[j + 1] = a * cy + b * tm.p[1]; h[j + 2] = a * cz + b * tm.p[2];
    e[I] = 0;
  }
}

// zhangli_torque_kernel!  src/micro/kernels.jl:680-739 (ut = ft / gamma)
void zhangli_field(const Sim& s, const Term& tm, const double* m, double* h, double* e) {
  const Mesh& g = s.mesh;
  const double ds[3] = {g.dx, g.dy, g.dz};
  const double ut = tm.ft / s.gamma;
  for (int64_t I = 0; I < g.n; ++I) {
    const int64_t j = 3 * I;
    double f[3] = {0, 0, 0};
    for (int ax = 0; ax < 3; ++ax) {
      int64_t i1 = g.ngb[6 * I + 2 * ax], i2 = g.ngb[6 * I + 2 * ax + 1];
      const double factor = (i1 >= 0 && i2 >= 0) ? 1 / (2 * ds[ax]) : 1 / ds[ax];
      if (i1 < 0) i1 = I;
      if (i2 < 0) i2 = I;
      const double u = tm.bJ[j + ax] * factor;
      for (int c = 0; c < 3; ++c) f[c] += u * (m[3 * i2 + c] - m[3 * i1 + c]);
    }
    for (int c = 0; c < 3; ++c) f[c] *= ut;
    double cx, cy, cz;
    cross3(m[j], m[j + 1], m[j + 2], f[0], f[1], f[2], cx, cy, cz);
    h[j] = cx + tm.xi[I] * f[0]; h[j + 1] = cy + tm.xi[I] * f[1]; h[j + 2] = cz + tm.xi[I] * f[2];
    e[I] = 0;
  }
}

// slonczewski_torque_kernel!  src/micro/kernels.jl (ft multiplied by beta)
void slonczewski_field(const Sim& s, const Term& tm, const double* m, double* h, double* e) {
  const Mesh& g = s.mesh;
  const double L2 = tm.Lambda * tm.Lambda;
  for (int64_t I = 0; I < g.n; ++I) {
    const int64_t j = 3 * I;
    const double mp = m[j] * tm.p[0] + m[j + 1] * tm.p[1] + m[j + 2] * tm.p[2];
    const double eps = tm.P * L2 / (L2 + 1 + (L2 - 1) * mp);
    const double a = tm.J[I] * tm.ftb;
    double cx, cy, cz;
    cross3(m[j], m[j + 1], m[j + 2], tm.p[0], tm.p[1], tm.p[2], cx, cy, cz);
    h[j] = a * (eps * cx + tm.xi_s * tm.p[0]);
    h[j + 1] = a * (eps * cy + tm.xi_s * tm.p[1]);
    h[j + 2] = a * (eps * cz + tm.xi_s * tm.p[2]);
    e[I] = 0;
  }
}

// Philox-4x32-10 (Salmon et al., SC'11), ten rounds with the Weyl key bumps
void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = static_cast<uint64_t>(0xD2511F53u) * c[0];
    const uint64_t p1 = static_cast<uint64_t>(0xCD9E8D57u) * c[2];
    const uint32_t n0 = static_cast<uint32_t>(p1 >> 32) ^ c[1] ^ k0;
    const uint32_t n2 = static_cast<uint32_t>(p0 >> 32) ^ c[3] ^ k1;
    c[1] = static_cast<uint32_t>(p1);
    c[3] = static_cast<uint32_t>(p0);
    c[0] = n0;
    c[2] = n2;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

// stochastic_field_kernel!  src/micro/kernels.jl:469-494 with eta of step
// th_cur_step drawn per cell from Philox((cell, step), seed) + Box-Muller;
// factor = 2 alpha k_B scaling / (V gamma dt)  (src/micro/field.jl:244-280)
void thermal_field(const Sim& s, const Term& tm, const double* m, double* h, double* e) {
  const Mesh& g = s.mesh;
  const double factor = 2 * s.alpha * tm.kB * tm.scaling / (g.volume * s.gamma * s.th_cur_dt);
  const uint64_t n = static_cast<uint64_t>(s.th_cur_step);
  const double s32 = 2.3283064365386963e-10;
  for (int64_t I = 0; I < g.n; ++I) {
    const int64_t j = 3 * I;
    const double Ms = s.mu0Ms[I];
    if (Ms > 0) {
      uint32_t c[4] = {static_cast<uint32_t>(I), static_cast<uint32_t>(static_cast<uint64_t>(I) >> 32),
                       static_cast<uint32_t>(n), static_cast<uint32_t>(n >> 32)};
      philox4x32_10(c, static_cast<uint32_t>(tm.seed), static_cast<uint32_t>(tm.seed >> 32));
      const double r0 = std::sqrt(-2.0 * std::log((double(c[0]) + 1.0) * s32));
      const double r1 = std::sqrt(-2.0 * std::log((double(c[2]) + 1.0) * s32));
      const double t0 = 6.283185307179586 * (double(c[1]) * s32), t1 = 6.283185307179586 * (double(c[3]) * s32);
      const double scale = std::sqrt(factor * (tm.T[I] + tm.T0) / Ms);
      h[j] = r0 * std::cos(t0) * scale;
      h[j + 1] = r0 * std::sin(t0) * scale;
      h[j + 2] = r1 * std::cos(t1) * scale;
      e[I] = -Ms * g.volume * (m[j] * h[j] + m[j + 1] * h[j + 1] + m[j + 2] * h[j + 2]);
    } else {
      h[j] = h[j + 1] = h[j + 2] = 0;
      e[I] = 0;
    }
  }
}

void term_eval(const Sim& s, Term& tm, const double* m) {
  double* h = tm.field.data();
  double* e = tm.energy.data();
  switch (tm.kind) {
    case T_ZEEMAN: zeeman(s, tm, m, h, e); break;
    case T_EXCH: if (tm.A.empty()) exch_uniform(s, tm, m, h, e); else exch_spatial(s, tm, m, h, e); break;
    case T_DMI_BULK: dmi_bulk(s, tm, m, h, e); break;
    case T_DMI_INTERFACIAL: dmi_interfacial(s, tm, m, h, e); break;
    case T_ANIS: anis_uniaxial(s, tm, m, h, e); break;
    case T_DEMAG: demag_field(s, tm, m, h, e); break;
    case T_DMI_BULK_SPATIAL: dmi_bulk_spatial(s, tm, m, h, e); break;
    case T_SOT: sot_field(s, tm, m, h, e); break;
    case T_STT_ZL: zhangli_field(s, tm, m, h, e); break;
    case T_STT_SL: slonczewski_field(s, tm, m, h, e); break;
    case T_THERMAL: thermal_field(s, tm, m, h, e); break;
  }
}

// Aggregator effective_field(sim, spin, t)  src/micro/field.jl:496-505:
// zero, then for each term in insertion order compute (Zeeman is not
// recomputed; its stored field is added) and add.
void effective_field(Sim& s, const double* m) {
  std::fill(s.field.begin(), s.field.end(), 0.0);
  for (auto& tp : s.terms) {
    Term& tm = *tp;
    if (tm.kind != T_ZEEMAN) term_eval(s, tm, m);
    const int64_t n3 = 3 * s.mesh.n;
    const double* f = tm.kind == T_ZEEMAN ? tm.H.data() : tm.field.data();
    for (int64_t i = 0; i < n3; ++i) s.field[i] = s.field[i] + f[i];  // util.jl:75-83
  }
}

// llg_rhs_kernel!  src/llg/llg.jl:6-40 ; llg_call_back llg.jl:45-59
void llg_rhs(Sim& s, double* dm, const double* m) {
  effective_field(s, m);
  const double* h = s.field.data();
  const double a = -s.gamma / (1 + s.alpha * s.alpha);
  const double alpha = s.alpha;
  const bool prec = s.precession;
#pragma omp parallel for schedule(static)
  for (int64_t I = 0; I < s.mesh.n; ++I) {
    int64_t j = 3 * I;
    if (!s.pins.empty() && s.pins[I]) { dm[j] = dm[j + 1] = dm[j + 2] = 0; continue; }
    double mx = m[j], my = m[j + 1], mz = m[j + 2];
    double mm = mx * mx + my * my + mz * mz;
    double mh = mx * h[j] + my * h[j + 1] + mz * h[j + 2];
    double h1 = mm * h[j] - mh * mx, h2 = mm * h[j + 1] - mh * my, h3 = mm * h[j + 2] - mh * mz;
    double f1 = 0, f2 = 0, f3 = 0;
    if (prec) cross3(mx, my, mz, h1, h2, h3, f1, f2, f3);
    dm[j] = a * (f1 - h1 * alpha);
    dm[j + 1] = a * (f2 - h2 * alpha);
    dm[j + 2] = a * (f3 - h3 * alpha);
  }
}

// normalise  src/helper.jl:255-271
void normalise(double* a, int64_t n) {
#pragma omp parallel for schedule(static)
  for (int64_t I = 0; I < n; ++I) {
    int64_t j = 3 * I;
    double m2 = a[j] * a[j] + a[j + 1] * a[j + 1] + a[j + 2] * a[j + 2];
    if (m2 > 0) {
      double len = 1 / std::sqrt(m2);
      a[j] *= len; a[j + 1] *= len; a[j + 2] *= len;
    }
  }
}

// advance_step(sim, ::RungeKutta)  src/integrator/rk.jl:23-52
// evaluations outside a step draw the thermal field of the fixed-step
// counter with the last fixed step (or the add-time dt)
void standalone_context(Sim& s) {
  s.th_cur_step = s.th_step;
  s.th_cur_dt = s.th_dt;
}

void rk4_step(Sim& s, double h) {
  s.th_cur_step = s.th_step;
  s.th_cur_dt = h;
  const int64_t n3 = 3 * s.mesh.n;
  std::vector<double>& k1 = s.ks[0];
  std::vector<double>& k2 = s.ks[1];
  std::vector<double>& k3 = s.ks[2];
  std::vector<double>& k4 = s.ks[3];
  std::vector<double>& y = s.prespin;
  double* m = s.m.data();
  llg_rhs(s, k1.data(), m);
  for (int64_t i = 0; i < n3; ++i) y[i] = m[i] + (0.5 * h) * k1[i];
  llg_rhs(s, k2.data(), y.data());
  for (int64_t i = 0; i < n3; ++i) y[i] = m[i] + (0.5 * h) * k2[i];
  llg_rhs(s, k3.data(), y.data());
  for (int64_t i = 0; i < n3; ++i) y[i] = m[i] + h * k3[i];
  llg_rhs(s, k4.data(), y.data());
  for (int64_t i = 0; i < n3; ++i) y[i] = m[i];
  const double c = 1.0 / 6 * h;
  for (int64_t i = 0; i < n3; ++i) m[i] += c * (((k1[i] + 2 * k2[i]) + 2 * k3[i]) + k4[i]);
  normalise(m, s.mesh.n);
  s.rk_nsteps += 1;
  s.rk_t = s.rk_nsteps * h;
  s.th_step += 1;
}

// advance_step(sim, ::ModifiedEuler)  src/integrator/heun.jl:28-49
// (vector_add2 / vector_add3 of src/util.jl)
void heun_step(Sim& s, double h) {
  s.th_cur_step = s.th_step;
  s.th_cur_dt = h;
  const int64_t n3 = 3 * s.mesh.n;
  std::vector<double>& k1 = s.ks[0];
  std::vector<double>& k2 = s.ks[1];
  std::vector<double>& y = s.prespin;
  double* m = s.m.data();
  llg_rhs(s, k1.data(), m);
  for (int64_t i = 0; i < n3; ++i) y[i] = m[i] + h * k1[i];
  llg_rhs(s, k2.data(), y.data());
  for (int64_t i = 0; i < n3; ++i) m[i] = m[i] + (0.5 * h) * k1[i] + (0.5 * h) * k2[i];
  normalise(m, s.mesh.n);
  s.rk_nsteps += 1;
  s.rk_t = s.rk_nsteps * h;
  s.th_step += 1;
}

// rk_step_dopri54!  src/integrator/adaptive_rk_steps.jl:49-... (vector_add2..6b
// of src/util.jl:86-183; error norm with atol = rtol = tol)
double dopri54_attempt(Sim& s, double step, double t) {
  (void)t;
  const double a1 = 1.0 / 5;
  const double a2[2] = {3.0 / 40, 9.0 / 40};
  const double a3[3] = {44.0 / 45, -56.0 / 15, 32.0 / 9};
  const double a4[4] = {19372.0 / 6561, -25360.0 / 2187, 64448.0 / 6561, -212.0 / 729};
  const double a5[5] = {9017.0 / 3168, -355.0 / 33, 46732.0 / 5247, 49.0 / 176, -5103.0 / 18656};
  const double a6[6] = {35.0 / 384, 0, 500.0 / 1113, 125.0 / 192, -2187.0 / 6784, 11.0 / 84};
  const double w[7] = {71.0 / 57600, 0, -71.0 / 16695, 71.0 / 1920, -17253.0 / 339200, 22.0 / 525, -1.0 / 40};
  const int64_t n3 = 3 * s.mesh.n;
  double* y0 = s.y_current.data();
  double* yn = s.y_next.data();
  double *k1 = s.ks[0].data(), *k2 = s.ks[1].data(), *k3 = s.ks[2].data(), *k4 = s.ks[3].data(),
         *k5 = s.ks[4].data(), *k6 = s.ks[5].data(), *k7 = s.ks[6].data();
  llg_rhs(s, k1, y0); s.nfevals += 1;
  {
    double c = a1 * step;
    for (int64_t i = 0; i < n3; ++i) yn[i] = y0[i] + c * k1[i];
  }
  llg_rhs(s, k2, yn);
  {
    double c2 = a2[0] * step, c3 = a2[1] * step;
    for (int64_t i = 0; i < n3; ++i) yn[i] = y0[i] + c2 * k1[i] + c3 * k2[i];
  }
  llg_rhs(s, k3, yn);
  {
    double c2 = a3[0] * step, c3 = a3[1] * step, c4 = a3[2] * step;
    for (int64_t i = 0; i < n3; ++i) yn[i] = y0[i] + c2 * k1[i] + c3 * k2[i] + c4 * k3[i];
  }
  llg_rhs(s, k4, yn);
  {
    double c2 = a4[0] * step, c3 = a4[1] * step, c4 = a4[2] * step, c5 = a4[3] * step;
    for (int64_t i = 0; i < n3; ++i) yn[i] = y0[i] + c2 * k1[i] + c3 * k2[i] + c4 * k3[i] + c5 * k4[i];
  }
  llg_rhs(s, k5, yn);
  {
    double c2 = a5[0] * step, c3 = a5[1] * step, c4 = a5[2] * step, c5 = a5[3] * step, c6 = a5[4] * step;
    for (int64_t i = 0; i < n3; ++i)
      yn[i] = y0[i] + c2 * k1[i] + c3 * k2[i] + c4 * k3[i] + c5 * k4[i] + c6 * k5[i];
  }
  llg_rhs(s, k6, yn);
  {
    double c2 = a6[0] * step, c3 = a6[2] * step, c4 = a6[3] * step, c5 = a6[4] * step, c6 = a6[5] * step;
    for (int64_t i = 0; i < n3; ++i)
      yn[i] = y0[i] + c2 * k1[i] + c3 * k3[i] + c4 * k4[i] + c5 * k5[i] + c6 * k6[i];
  }
  normalise(yn, s.mesh.n);
  llg_rhs(s, k7, yn);
  s.nfevals += 6;
  double* yt = s.y_temp.data();
  double mx = 0.0;
  bool nan = false;
  for (int64_t i = 0; i < n3; ++i) {
    yt[i] = w[0] * k1[i] + w[2] * k3[i] + w[3] * k4[i] + w[4] * k5[i] + w[5] * k6[i] + w[6] * k7[i];
    double v = std::fabs(yt[i] / (1 + std::fabs(yn[i])));
    if (std::isnan(v)) nan = true;
    if (v > mx) mx = v;
  }
  if (nan) return std::nan("");
  return mx * step / s.tol;
}

// rk_step_bs23!  src/integrator/adaptive_rk_steps.jl:11-47 (FSAL: k1 = k4
// after an accepted attempt)
double bs23_attempt(Sim& s, double step, double t) {
  const int64_t n3 = 3 * s.mesh.n;
  double* y0 = s.y_current.data();
  double* yn = s.y_next.data();
  double* yt = s.y_temp.data();
  double *k1 = s.ks[0].data(), *k2 = s.ks[1].data(), *k3 = s.ks[2].data(), *k4 = s.ks[3].data();
  if (s.succeed && t >= s.t) {
    for (int64_t i = 0; i < n3; ++i) k1[i] = k4[i];
  } else {
    llg_rhs(s, k1, y0);
    s.nfevals += 1;
  }
  for (int64_t i = 0; i < n3; ++i) yt[i] = y0[i] + step * 0.5 * k1[i];
  llg_rhs(s, k2, yt);
  for (int64_t i = 0; i < n3; ++i) yt[i] = y0[i] + step * 0.75 * k2[i];
  llg_rhs(s, k3, yt);
  for (int64_t i = 0; i < n3; ++i) yn[i] = y0[i] + step * (2.0 / 9 * k1[i] + 1.0 / 3 * k2[i] + 4.0 / 9 * k3[i]);
  normalise(yn, s.mesh.n);
  llg_rhs(s, k4, yn);
  s.nfevals += 3;
  double mx = 0.0;
  bool nan = false;
  for (int64_t i = 0; i < n3; ++i) {
    yt[i] = -(5.0 / 72) * k1[i] + (1.0 / 12) * k2[i] + (1.0 / 9) * k3[i] + (-1.0 / 8) * k4[i];
    double v = std::fabs(yt[i] / (1 + std::fabs(yn[i])));
    if (std::isnan(v)) nan = true;
    if (v > mx) mx = v;
  }
  if (nan) return std::nan("");
  return mx * step / s.tol;
}

// The six-stage 5(4) pairs: table IV (Cash-Karp) and table III (Fehlberg)
// of src/integrator/adaptive_rk_steps.jl:110-229.  b2..b6 build the stage
// inputs, c the solution, w the error (c2 = w2 = 0).
struct SixStage {
  double b[5][5];
  double c[6];
  double w[6];
};
const SixStage kCashKarp54 = {{{1.0 / 5},
                               {3.0 / 40, 9.0 / 40},
                               {3.0 / 10, -9.0 / 10, 6.0 / 5},
                               {-11.0 / 54, 5.0 / 2, -70.0 / 27, 35.0 / 27},
                               {1631.0 / 55296, 175.0 / 512, 575.0 / 13824, 44275.0 / 110592, 253.0 / 4096}},
                              {37.0 / 378, 0, 250.0 / 621, 125.0 / 594, 0, 512.0 / 1771},
                              {-277.0 / 64512, 0, 6925.0 / 370944, -6925.0 / 202752, -277.0 / 14336, 277.0 / 7084}};
const SixStage kFehlberg54 = {{{1.0 / 4},
                               {3.0 / 32, 9.0 / 32},
                               {1932.0 / 2197, -7200.0 / 2197, 7296.0 / 2197},
                               {439.0 / 216, -8.0, 3680.0 / 513, -845.0 / 4104},
                               {-8.0 / 27, 2.0, -3544.0 / 2565, 1859.0 / 4104, -11.0 / 40}},
                              {16.0 / 135, 0, 6656.0 / 12825, 28561.0 / 56430, -9.0 / 50, 2.0 / 55},
                              {-1.0 / 360, 0, 128.0 / 4275, 2197.0 / 75240, -1.0 / 50, -2.0 / 55}};

// rk_step_cashkarp54! / rk_step_fehlberg54!  src/integrator/adaptive_rk_steps.jl:110-229
double six_stage_attempt(Sim& s, double step, const SixStage& tb) {
  const int64_t n3 = 3 * s.mesh.n;
  double* y0 = s.y_current.data();
  double* yn = s.y_next.data();
  double* k[6];
  for (int j = 0; j < 6; ++j) k[j] = s.ks[j].data();
  llg_rhs(s, k[0], y0);
  for (int st = 1; st < 6; ++st) {
    double cf[5];
    for (int j = 0; j < st; ++j) cf[j] = tb.b[st - 1][j] * step;
    for (int64_t i = 0; i < n3; ++i) {
      double v = y0[i];
      for (int j = 0; j < st; ++j) v += cf[j] * k[j][i];
      yn[i] = v;
    }
    llg_rhs(s, k[st], yn);
  }
  double cs[6];
  for (int j = 0; j < 6; ++j) cs[j] = tb.c[j] * step;
  for (int64_t i = 0; i < n3; ++i)
    yn[i] = y0[i] + cs[0] * k[0][i] + cs[2] * k[2][i] + cs[3] * k[3][i] + cs[4] * k[4][i] + cs[5] * k[5][i];
  normalise(yn, s.mesh.n);
  s.nfevals += 6;
  double* yt = s.y_temp.data();
  double mx = 0.0;
  bool nan = false;
  for (int64_t i = 0; i < n3; ++i) {
    yt[i] = tb.w[0] * k[0][i] + tb.w[2] * k[2][i] + tb.w[3] * k[3][i] + tb.w[4] * k[4][i] + tb.w[5] * k[5][i];
    double v = std::fabs(yt[i] / (1 + std::fabs(yn[i])));
    if (std::isnan(v)) nan = true;
    if (v > mx) mx = v;
  }
  if (nan) return std::nan("");
  return mx * step / s.tol;
}

// method-specific step function  src/integrator/adaptive_rk.jl:67-89
double rk_attempt(Sim& s, double step, double t) {
  // the thermal field is redrawn when integrator.nsteps advances (src/micro/field.jl:250-253)
  s.th_cur_step = s.nsteps;
  s.th_cur_dt = step;
  switch (s.method) {
    case 1: return bs23_attempt(s, step, t);
    case 2: return six_stage_attempt(s, step, kCashKarp54);
    case 3: return six_stage_attempt(s, step, kFehlberg54);
    default: return dopri54_attempt(s, step, t);
  }
}
// (order_main, order_embedded) of DOPRI54, BS23, CashKarp54, Fehlberg54
// (src/integrator/adaptive_rk.jl:248-266)
int order_main(const Sim& s) { return s.method == 1 ? 3 : 5; }
int order_embedded(const Sim& s) { return s.method == 1 ? 2 : 4; }

// compute_initial_step  src/integrator/adaptive_rk.jl:151-165
double compute_initial_step(Sim& s, double dt) {
  double abs_step = dt, abs_step_tmp = dt;
  s.step = 1e-15;
  s.th_cur_step = s.nsteps;  // the rhs sees integrator.step = 1e-15
  s.th_cur_dt = s.step;
  llg_rhs(s, s.y_temp.data(), s.y_current.data());
  double mx = 0.0;
  for (double v : s.y_temp) mx = std::max(mx, std::fabs(v));
  double r_step = mx / (s.safety * std::pow(s.tol, 1.0 / order_main(s)));
  s.nfevals += 1;
  if (abs_step * r_step > 0.001) abs_step_tmp = 0.001 / r_step;
  return std::min(abs_step, abs_step_tmp);
}

// advance_step(sim, ::AdaptiveRK)  src/integrator/adaptive_rk.jl:93-148
// returns 1 on success, 0 on failure (NaN or too many attempts)
int dopri_advance(Sim& s, int64_t* attempts) {
  const int max_nsteps = 50;
  const int order = order_embedded(s);
  double t = s.t;
  if (s.step_next <= 0) s.step_next = compute_initial_step(s, 1e-12);
  s.step = s.step_next;
  int nstep = 1;
  while (true) {
    double err = rk_attempt(s, s.step, t);
    if (attempts) *attempts += 1;
    if (std::isnan(err)) { s.step_next = 1e-14; return 0; }
    nstep += 1;
    if (nstep > max_nsteps) return 0;
    s.succeed = err <= 1.0;
    if (s.succeed) {
      s.y_current = s.y_next;
      s.nsteps += 1;
      s.t += s.step;
      double factor = s.safety * std::pow(1.0 / err, 1.0 / (order + 1));
      s.step_next = s.step * std::min(s.facmax, std::max(s.facmin, factor));
      break;
    } else {
      double factor = s.safety * std::pow(1.0 / err, 1.0 / order);
      s.step = s.step * std::min(s.facmax, std::max(s.facmin, factor));
    }
  }
  return 1;
}

// integrate_to_time  src/integrator/adaptive_rk.jl:168-186
int dopri_integrate_to(Sim& s, double t_final, int64_t* attempts) {
  while (s.t < t_final) {
    if (s.step_next + s.t > t_final) s.step_next = t_final - s.t;
    if (!dopri_advance(s, attempts)) return 0;
  }
  return s.succeed ? 1 : 0;
}

// SD driver (src/sd.jl:9-98)
void sd_step(Sim& s) {
  const int64_t n = s.mesh.n;
  effective_field(s, s.m.data());
  const double* h = s.field.data();
  double* m = s.m.data();
  double* pre = s.prespin.data();
  double* gk = s.gk.data();
  if (s.sd_steps == 0) {
    for (int64_t I = 0; I < n; ++I) {  // compute_gk_kernel_1!
      int64_t j = 3 * I;
      double fx, fy, fz, gx, gy, gz;
      cross3(m[j], m[j + 1], m[j + 2], h[j], h[j + 1], h[j + 2], fx, fy, fz);
      cross3(m[j], m[j + 1], m[j + 2], fx, fy, fz, gx, gy, gz);
      gk[j] = gx; gk[j + 1] = gy; gk[j + 2] = gz;
    }
    s.tau = s.min_tau;
  } else {
    double sum1 = 0, sum2 = 0, sum3 = 0;
    for (int64_t I = 0; I < n; ++I) {  // compute_gk_kernel_2!
      int64_t j = 3 * I;
      double sx = m[j] - pre[j], sy = m[j + 1] - pre[j + 1], sz = m[j + 2] - pre[j + 2];
      double fx, fy, fz, gx, gy, gz;
      cross3(m[j], m[j + 1], m[j + 2], h[j], h[j + 1], h[j + 2], fx, fy, fz);
      cross3(m[j], m[j + 1], m[j + 2], fx, fy, fz, gx, gy, gz);
      fx = gx - gk[j]; fy = gy - gk[j + 1]; fz = gz - gk[j + 2];
      gk[j] = gx; gk[j + 1] = gy; gk[j + 2] = gz;
      s.ss[I] = sx * sx + sy * sy + sz * sz;
      s.sf[I] = sx * fx + sy * fy + sz * fz;
      s.ff[I] = fx * fx + fy * fy + fz * fz;
    }
    for (int64_t I = 0; I < n; ++I) { sum1 += s.ss[I]; sum2 += s.sf[I]; sum3 += s.ff[I]; }
    double tau1 = sum2 != 0 ? sum1 / sum2 : s.min_tau;
    double tau2 = sum3 != 0 ? sum2 / sum3 : s.min_tau;
    s.tau = s.sd_steps % 2 == 0 ? std::fabs(tau2) : std::fabs(tau1);
    if (s.tau > s.max_tau) s.tau = s.max_tau;
  }
  std::copy(s.m.begin(), s.m.end(), s.prespin.begin());
  const double tau = s.tau;
  for (int64_t I = 0; I < n; ++I) {  // run_step_kernel!
    if (!s.pins.empty() && s.pins[I]) continue;
    int64_t j = 3 * I;
    double fx, fy, fz;
    cross3(m[j], m[j + 1], m[j + 2], h[j], h[j + 1], h[j + 2], fx, fy, fz);
    double factor = 0.25 * (fx * fx + fy * fy + fz * fz) * tau * tau;
    double mx = (1 - factor) * m[j] - tau * gk[j];
    double my = (1 - factor) * m[j + 1] - tau * gk[j + 1];
    double mz = (1 - factor) * m[j + 2] - tau * gk[j + 2];
    m[j] = mx / (1 + factor); m[j + 1] = my / (1 + factor); m[j + 2] = mz / (1 + factor);
  }
  s.sd_steps += 1;
  if (s.sd_steps % 10 == 0) normalise(m, n);
}

// max over cells of |m1 - m2| (compute_dm! src/helper.jl:273-286 + maximum)
double max_dm(const double* a, const double* b, int64_t n) {
  double mx = 0.0;
  for (int64_t I = 0; I < n; ++I) {
    int64_t j = 3 * I;
    double x = a[j] - b[j], y = a[j + 1] - b[j + 1], z = a[j + 2] - b[j + 2];
    mx = std::max(mx, std::sqrt(x * x + y * y + z * z));
  }
  return mx;
}

std::string g_err;

}  // namespace

// ===========================================================================
// C ABI of the oracle (ctypes from oracle/oracle.py)
// ===========================================================================
extern "C" {

const char* orc_last_error() { return g_err.c_str(); }

void orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

int orc_max_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void* orc_create(int nx, int ny, int nz, double dx, double dy, double dz, int pbc) {
  if (nx < 1 || ny < 1 || nz < 1) { g_err = "bad mesh size"; return nullptr; }
  auto* s = new Sim();
  s->mesh.nx = nx; s->mesh.ny = ny; s->mesh.nz = nz;
  s->mesh.dx = dx; s->mesh.dy = dy; s->mesh.dz = dz;
  s->mesh.px = pbc & 1; s->mesh.py = pbc & 2; s->mesh.pz = pbc & 4;
  s->mesh.build();
  const int64_t n = s->mesh.n;
  s->mu0Ms.assign(n, 0.0);
  s->m.assign(3 * n, 0.0);
  s->prespin.assign(3 * n, 0.0);
  s->field.assign(3 * n, 0.0);
  s->y_current.assign(3 * n, 0.0);
  s->y_next.assign(3 * n, 0.0);
  s->y_temp.assign(3 * n, 0.0);
  for (auto& k : s->ks) k.assign(3 * n, 0.0);
  s->gk.assign(3 * n, 0.0);
  s->ss.assign(n, 0.0); s->sf.assign(n, 0.0); s->ff.assign(n, 0.0);
  return s;
}

void orc_destroy(void* h) { delete static_cast<Sim*>(h); }

// set_Ms  src/sim.jl:129-143 (input in A/m, stored as mu0*Ms in Tesla)
void orc_set_Ms(void* h, const double* Ms) {
  Sim* s = static_cast<Sim*>(h);
  for (int64_t i = 0; i < s->mesh.n; ++i) s->mu0Ms[i] = Ms[i] * kMu0;
}

void orc_set_m(void* h, const double* m) {
  Sim* s = static_cast<Sim*>(h);
  std::copy(m, m + 3 * s->mesh.n, s->m.begin());
  std::copy(m, m + 3 * s->mesh.n, s->prespin.begin());
  std::copy(m, m + 3 * s->mesh.n, s->y_current.begin());  // set_initial_condition!
}

void orc_get_m(void* h, double* m) {
  Sim* s = static_cast<Sim*>(h);
  std::copy(s->m.begin(), s->m.end(), m);
}

void orc_set_pins(void* h, const uint8_t* pins) {
  Sim* s = static_cast<Sim*>(h);
  s->pins.assign(pins, pins + s->mesh.n);
}

void orc_set_llg(void* h, double alpha, double gamma, int precession) {
  Sim* s = static_cast<Sim*>(h);
  s->alpha = alpha; s->gamma = gamma; s->precession = precession != 0;
}

static Term* new_term(Sim* s, TermKind k) {
  auto t = std::make_unique<Term>();
  t->kind = k;
  t->field.assign(3 * s->mesh.n, 0.0);
  t->energy.assign(s->mesh.n, 0.0);
  Term* raw = t.get();
  s->terms.push_back(std::move(t));
  return raw;
}

int orc_add_zeeman(void* h, const double* H) {
  Sim* s = static_cast<Sim*>(h);
  Term* t = new_term(s, T_ZEEMAN);
  t->H.assign(H, H + 3 * s->mesh.n);
  return static_cast<int>(s->terms.size()) - 1;
}

int orc_add_exch(void* h, const double* A, double Ax, double Ay, double Az) {
  Sim* s = static_cast<Sim*>(h);
  Term* t = new_term(s, T_EXCH);
  if (A) t->A.assign(A, A + s->mesh.n);
  t->Ax = Ax; t->Ay = Ay; t->Az = Az;
  return static_cast<int>(s->terms.size()) - 1;
}

int orc_add_dmi_bulk(void* h, double Dx, double Dy, double Dz) {
  Sim* s = static_cast<Sim*>(h);
  Term* t = new_term(s, T_DMI_BULK);
  t->Dx = Dx; t->Dy = Dy; t->Dz = Dz;
  return static_cast<int>(s->terms.size()) - 1;
}

int orc_add_dmi_interfacial(void* h, const double* D) {
  Sim* s = static_cast<Sim*>(h);
  Term* t = new_term(s, T_DMI_INTERFACIAL);
  t->D.assign(D, D + s->mesh.n);
  return static_cast<int>(s->terms.size()) - 1;
}

int orc_add_dmi_bulk_spatial(void* h, const double* Dx, const double* Dy, const double* Dz) {
  Sim* s = static_cast<Sim*>(h);
  Term* t = new_term(s, T_DMI_BULK_SPATIAL);
  const int64_t n = s->mesh.n;
  t->bD[0].assign(Dx, Dx + n); t->bD[1].assign(Dy, Dy + n); t->bD[2].assign(Dz, Dz + n);
  return static_cast<int>(s->terms.size()) - 1;
}

int orc_add_sot(void* h, const double* aj, double bj, double px, double py, double pz) {
  Sim* s = static_cast<Sim*>(h);
  Term* t = new_term(s, T_SOT);
  t->aj.assign(aj, aj + s->mesh.n);
  t->bj = bj; t->p[0] = px; t->p[1] = py; t->p[2] = pz;
  return static_cast<int>(s->terms.size()) - 1;
}

int orc_add_stt_zhang_li(void* h, const double* bJ, const double* xi, double ft) {
  Sim* s = static_cast<Sim*>(h);
  Term* t = new_term(s, T_STT_ZL);
  t->bJ.assign(bJ, bJ + 3 * s->mesh.n);
  t->xi.assign(xi, xi + s->mesh.n);
  t->ft = ft;
  return static_cast<int>(s->terms.size()) - 1;
}

int orc_add_stt_slonczewski(void* h, const double* J, double ftb, double Lambda, double P, double xi, double px,
                            double py, double pz) {
  Sim* s = static_cast<Sim*>(h);
  Term* t = new_term(s, T_STT_SL);
  t->J.assign(J, J + s->mesh.n);
  t->ftb = ftb; t->Lambda = Lambda; t->P = P; t->xi_s = xi;
  t->p[0] = px; t->p[1] = py; t->p[2] = pz;
  return static_cast<int>(s->terms.size()) - 1;
}

int orc_add_thermal_noise(void* h, const double* T, double T0, double scaling, double kB, uint64_t seed, double dt) {
  Sim* s = static_cast<Sim*>(h);
  Term* t = new_term(s, T_THERMAL);
  t->T.assign(T, T + s->mesh.n);
  t->T0 = T0; t->scaling = scaling; t->kB = kB; t->seed = seed; t->dt = dt;
  s->th_dt = dt;
  return static_cast<int>(s->terms.size()) - 1;
}

// Philox-4x32-10 of one counter block (test access)
void orc_philox(const uint32_t* ctr, const uint32_t* key, uint32_t* out) {
  uint32_t c[4] = {ctr[0], ctr[1], ctr[2], ctr[3]};
  philox4x32_10(c, key[0], key[1]);
  for (int i = 0; i < 4; ++i) out[i] = c[i];
}

// add_anis  src/micro/add_field.jl:430-465 (axis normalised at add time)
int orc_add_anis(void* h, const double* Ku, double ux, double uy, double uz) {
  Sim* s = static_cast<Sim*>(h);
  Term* t = new_term(s, T_ANIS);
  t->Ku.assign(Ku, Ku + s->mesh.n);
  double lt = std::sqrt(ux * ux + uy * uy + uz * uz);
  t->ux = ux / lt; t->uy = uy / lt; t->uz = uz / lt;
  return static_cast<int>(s->terms.size()) - 1;
}

// add_demag  src/micro/add_field.jl:403-419 -> init_demag demag.jl:30-100.
// tensor (may be null): caller-supplied real-space tensor, 6 x N in the order
// xx, yy, zz, xy, xz, yz, replacing the Newell assembly.
int orc_add_demag(void* h, int Nx, int Ny, int Nz, const double* tensor) {
  Sim* s = static_cast<Sim*>(h);
  Term* t = new_term(s, T_DEMAG);
  demag_init(*s, *t, Nx, Ny, Nz, tensor);
  return static_cast<int>(s->terms.size()) - 1;
}

// Newell real-space tensor (6 x N, order xx yy zz xy xz yz) in normalised
// cell units, with macro-PBC images: tensors_kernel_*! demag.jl:298-386.
// accurate != 0: binary128 near field (the default of add_demag); 0: the
// reference's FP64 arithmetic.
void orc_demag_tensor(int nx, int ny, int nz, double dx, double dy, double dz, int Nx, int Ny, int Nz, int accurate,
                      double* out) {
  const double mx = std::max(dx, std::max(dy, dz));
  newell_table(nx, ny, nz, dx / mx, dy / mx, dz / mx, Nx, Ny, Nz, accurate != 0, out);
}

// Tensor arithmetic of the following add_demag calls: 1 = the reference's
// FP64 arithmetic, 0 = binary128 near field (default).
void orc_set_reference_tensor(int on) { g_reference_tensor = on != 0; }

// f or g of component c (xx yy zz xy xz yz, permuted as in demag.jl) at
// x = X dx, y = Y dy, z = Z dz, in binary128, returned as hi + lo doubles
void orc_newell_fn(int c, int64_t X, int64_t Y, int64_t Z, double dx, double dy, double dz, double* hi_lo) {
  const q128 v = q_newell(c, X, Y, Z, dx, dy, dz);
  hi_lo[0] = static_cast<double>(v);
  hi_lo[1] = static_cast<double>(v - static_cast<q128>(hi_lo[0]));
}

// Evaluate one term on m (or on the stored m if m == null); field 3N, energy N.
int orc_term_field(void* h, int idx, const double* m, double* field, double* energy) {
  standalone_context(*static_cast<Sim*>(h));
  Sim* s = static_cast<Sim*>(h);
  if (idx < 0 || idx >= static_cast<int>(s->terms.size())) { g_err = "bad term"; return -1; }
  Term& t = *s->terms[idx];
  term_eval(*s, t, m ? m : s->m.data());
  if (field) std::copy(t.field.begin(), t.field.end(), field);
  if (energy) std::copy(t.energy.begin(), t.energy.end(), energy);
  return 0;
}

// Aggregated H_eff (field.jl:496-505) on m (or stored m).
void orc_effective_field(void* h, const double* m, double* field) {
  standalone_context(*static_cast<Sim*>(h));
  Sim* s = static_cast<Sim*>(h);
  effective_field(*s, m ? m : s->m.data());
  if (field) std::copy(s->field.begin(), s->field.end(), field);
}

// dm/dt = llg_call_back(sim, dm_dt, m, t)
void orc_llg_rhs(void* h, const double* m, double* dmdt) {
  standalone_context(*static_cast<Sim*>(h));
  Sim* s = static_cast<Sim*>(h);
  llg_rhs(*s, dmdt, m ? m : s->m.data());
}

// compute_system_energy  field.jl:520-536: total and per-term energies
double orc_energy(void* h, double* per_term) {
  standalone_context(*static_cast<Sim*>(h));
  Sim* s = static_cast<Sim*>(h);
  double total = 0.0;
  for (size_t i = 0; i < s->terms.size(); ++i) {
    Term& t = *s->terms[i];
    term_eval(*s, t, s->m.data());
    double e = 0.0;
    for (double v : t.energy) e += v;
    if (per_term) per_term[i] = e;
    total += e;
  }
  return total;
}

void orc_rk4(void* h, double dt, int64_t nsteps) {
  Sim* s = static_cast<Sim*>(h);
  s->th_dt = dt;
  for (int64_t i = 0; i < nsteps; ++i) rk4_step(*s, dt);
}

double orc_rk4_time(void* h) { return static_cast<Sim*>(h)->rk_t; }

void orc_heun(void* h, double dt, int64_t nsteps) {
  Sim* s = static_cast<Sim*>(h);
  s->th_dt = dt;
  for (int64_t i = 0; i < nsteps; ++i) heun_step(*s, dt);
}

// a new AdaptiveRK of the given method (Sim(mesh; integrator=...), src/driver.jl:102-140)
void orc_set_method(void* h, int method) {
  Sim* s = static_cast<Sim*>(h);
  s->method = method;
  s->t = 0.0;
  s->step = 0.0;
  s->step_next = 0.0;
  s->nsteps = 0;
  s->nfevals = 0;
  s->succeed = false;
}

void orc_dopri_set(void* h, double tol) {
  Sim* s = static_cast<Sim*>(h);
  s->tol = tol;
}

// run_until(sim, t_end) for an AdaptiveRK integrator  src/sim.jl:547-574.
// stats: [t, step, step_next, nsteps, nfevals, attempts]
int orc_run_until(void* h, double t_end, double* stats) {
  Sim* s = static_cast<Sim*>(h);
  int64_t attempts = 0;
  int ok = 1;
  if (!(t_end < s->t - s->step) && t_end != s->t) {
    std::copy(s->m.begin(), s->m.end(), s->prespin.begin());
    ok = dopri_integrate_to(*s, t_end, &attempts);
    std::copy(s->y_current.begin(), s->y_current.end(), s->m.begin());
  }
  if (stats) {
    stats[0] = s->t; stats[1] = s->step; stats[2] = s->step_next;
    stats[3] = static_cast<double>(s->nsteps); stats[4] = static_cast<double>(s->nfevals);
    stats[5] = static_cast<double>(attempts);
  }
  return ok;
}

// integrator.y_current of the adaptive stepper (advance_step does not copy it
// into sim.spin; run_until does)
void orc_get_y_current(void* h, double* y) {
  Sim* s = static_cast<Sim*>(h);
  std::copy(s->y_current.begin(), s->y_current.end(), y);
}

// One advance_step(sim, ::AdaptiveRK) (used by relax with the LLG driver).
int orc_dopri_advance(void* h, double* stats) {
  Sim* s = static_cast<Sim*>(h);
  int64_t attempts = 0;
  int ok = dopri_advance(*s, &attempts);
  if (stats) {
    stats[0] = s->t; stats[1] = s->step; stats[2] = s->step_next;
    stats[3] = static_cast<double>(s->nsteps); stats[4] = static_cast<double>(s->nfevals);
    stats[5] = static_cast<double>(attempts);
  }
  return ok;
}

// relax(sim)  src/sim.jl:392-490 for the SD driver (driver=0) or the LLG driver
// with Dormand-Prince (driver=1).  Returns the number of steps run; *max_dmdt
// receives the last max_dmdt / dmdt_factor.
int64_t orc_relax(void* h, int driver, int64_t max_steps, double stopping_dmdt, double* max_dmdt_out) {
  standalone_context(*static_cast<Sim*>(h));
  Sim* s = static_cast<Sim*>(h);
  const double time_factor = 2.21e5 / 2;
  const double dmdt_factor = (2 * kPi / 360) * 1e9;
  const int64_t n = s->mesh.n;
  double max_dmdt = 0.0;
  int64_t i = 1;
  for (; i <= max_steps; ++i) {
    double step_size;
    if (driver == 0) {
      sd_step(*s);
      step_size = s->tau / time_factor;
    } else {
      dopri_advance(*s, nullptr);
      std::copy(s->m.begin(), s->m.end(), s->prespin.begin());
      std::copy(s->y_current.begin(), s->y_current.end(), s->m.begin());
      step_size = s->step;
    }
    max_dmdt = max_dm(s->prespin.data(), s->m.data(), n) / step_size;
    if (max_dmdt < stopping_dmdt * dmdt_factor) break;
  }
  if (max_dmdt_out) *max_dmdt_out = max_dmdt / dmdt_factor;
  return i > max_steps ? max_steps : i;
}

}  // extern "C"

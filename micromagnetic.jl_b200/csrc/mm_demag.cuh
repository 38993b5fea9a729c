// mm_demag.cuh -- zero-padded FFT demagnetising-field convolution (internal).
//
// Follows MicroMagnetic.jl src/micro/demag.jl:30-131: H = -(1/mu0) * N (*) M,
// M = mu0*Ms*m, with the Newell tensor N assembled in FP64
// (demag.jl:133-417, far field atomistic/demag.jl:106-138).
//
// Layout in HBM (x fastest everywhere):
//   X    [3][nz][ny][Hx] complex   x half-spectrum of the physical rows only
//   Y    [3][nz][Py][Hx] complex   after the forward y pass (3-D meshes)
//   Nhat [6][Pz/2+1][Py/2+1][Hx]   real tensor spectrum, one quadrant
//        (xx yy zz xy xz yz), pre-scaled by -1/(mu0 Px Py Pz); the other
//        quadrants follow from the even/odd symmetry of each component.
// Passes per evaluation: fwd-x (r2c, pruned to ny*nz rows), fwd-y,
// z-conv (fwd-z * Nhat * inv-z), inv-y, inv-x (c2r).  For nz == 1 the
// y passes and the product fuse into one y-conv pass.
#pragma once
#include "mm_common.cuh"

namespace mm {

struct DemagGeom {
  int nx, ny, nz;
  int Px, Py, Pz;  // padded lengths
  int Lc, Hx;      // Lc = Px/2 (0 when Px == 1), Hx = Lc + 1 (1 when Px == 1)
  int Tyq, Tzq;    // Py/2 + 1, Pz/2 + 1
  // ky row stride of the column-major 3-D tensor, Nhat[((c*Tzq + kz)*Hx +
  // kx)*Tys + ky]: Tyq, or Tyq rounded up to a multiple of 4 (16-byte rows,
  // zero padded) where the register z convolution loads its tensor slice
  // with tiled bulk copies
  int Tys;
  FftPlan1 plx, ply, plz;
  FastDiv fLc, fHx, fPy, fPz, fny, fnz, frows, fpady, fpadz;
  // films on the fused y-convolution path keep the x spectrum column-major,
  // X[(c*Hx + kx)*ny + y], and the tensor quadrant as Nhat[(c*Hx + kx)*Tyq + ky],
  // so that a y line is contiguous in HBM (row-major: X[(c*ny + y)*Hx + kx])
  int xT;
  // 3-D meshes whose y lines are too long for wide row tiles keep the spectra
  // column-major too: Y[((c*Hx + kx)*nz + z)*Py + ky] and
  // Nhat[((c*Tzq + kz)*Hx + kx)*Tyq + ky] (the z convolution then tiles along
  // ky); X is column-major, X[((c*Hx + kx)*nz + z)*ny + y], from the forward
  // x pass to the forward y pass (xT is set), and row-major again from the
  // inverse y pass to the inverse x pass
  int yT;
  // power-of-two meshes (nx, ny = 32 Q, Px = 2 nx, Py = 2 ny, 3-D; FP64:
  // nx = 512 or 1024, ny = 1024): the x and y passes run register-resident
  // (mm_wreg.cu) with X column-major in both directions (yT and xT are set)
  int wreg;
  const int* gate;  // device flag: kernels return at once when *gate == 0 (null: always run)
};

template <typename R>
class DemagPlan {
 public:
  using C = cplx_t<R>;
  DemagPlan() = default;
  ~DemagPlan();
  DemagPlan(const DemagPlan&) = delete;
  DemagPlan& operator=(const DemagPlan&) = delete;

  // Geometry, buffers and twiddle tables.  Returns 0 or a cudaError/-1 (size).
  int init(int nx, int ny, int nz, cudaStream_t st, char* err, size_t nerr);
  // Tensor spectrum from a real-space FP64 tensor on the device (6 x N,
  // order xx yy zz xy xz yz).
  int set_tensor(const double* T6N_dev, cudaStream_t st);
  // H_demag (SoA 3N) of the magnetisation m (SoA 3N) with mu0*Ms (N).
  void apply(const R* m, const R* mu0Ms, R* Hd, cudaStream_t st, const int* gate = nullptr);
  // Number of kernel launches of one apply().
  int launches_per_apply() const;
  // Every launch of apply() is a descriptor kernel (mm_launch.cuh), so that a
  // batch can merge the passes of several meshes into one launch each.
  bool batchable() const;
  // One pass alone (0 fwd-x, 1 fwd-y, 2 conv, 3 inv-y, 4 inv-x), for timing;
  // false when this geometry does not use it.
  bool launch_pass(int which, const R* m, const R* mu0Ms, R* Hd, cudaStream_t st);
  // Compulsory HBM bytes of one launch of that pass.
  double pass_bytes(int which) const;
  size_t device_bytes() const { return bytes_; }

  // Tile widths (kx columns per block) of the strided passes 1..3, chosen by
  // autotune(); 0 keeps the static rule (largest W whose tile fits the
  // shared-memory budget).  Any W gives bit-identical results: each line is
  // transformed by the same arithmetic whatever block it lands in.
  int autotune(const R* m, const R* mu0Ms, R* Hd, cudaStream_t st);
  int tile[5] = {0, 0, 0, 0, 0};
  float tile_ms[5] = {0, 0, 0, 0, 0};

  DemagGeom g{};
  bool fused2d = false;
  // x / y lines longer than one block holds run as global-memory radix
  // stages (plans gplx / gply, radix <= 8) through ping-pong buffers:
  // S (same shape as Y) for y, Zx / Zx2 ([3 ny nz][Lc]) for x
  bool long_x = false, long_y = false;
  FftPlan1 gplx{}, gply{};
  C* S = nullptr;
  C* Zx = nullptr;
  C* Zx2 = nullptr;
  C* X = nullptr;
  C* Y = nullptr;
  R* Nhat = nullptr;
  alignas(64) unsigned char zmap[128] = {};  // tensor map of the z convolution's slice loads (FP32, yT)
  C* twx = nullptr;
  C* twy = nullptr;
  C* twz = nullptr;

 private:
  size_t bytes_ = 0;
};

// Register-resident z convolution for Pz = 32 (nz <= 16), FP32 form
// (mm_zpair.cu): in place on Y, either spectrum layout.
bool zpair_applies(const DemagGeom& g);
// Column-major spectra (g.yT): the block's tensor slice arrives by one tiled
// bulk copy through a tensor map over Nhat (built by zpair_tensor_map, 128
// bytes); the row-major layout copies it with cp.async.
bool zpair_tensor_map(const DemagGeom& g, const float* Nhat, void* map128);
void launch_zpair_f32(const DemagGeom& g, float2* Y, const float* Nhat, const void* map128, cudaStream_t st);
// Tries of a bounded bulk-copy wait (MMCUDA_COPY_SPINS overrides; 0 makes
// every first wait run out, which the tests use to check the timeout path).
unsigned copy_wait_spins();
bool zpair_take_timeout();

// Register-resident z convolution for Pz = 32 (nz <= 16), FP64 form,
// column-major spectra (mm_zquad.cu): in place on Y.  MMCUDA_ZQUAD=0 keeps
// the shared-memory kernel.
bool zquad_applies(const DemagGeom& g);
void launch_zquad_f64(const DemagGeom& g, double2* Y, const double* Nhat, cudaStream_t st);

// Register-resident x and y passes (mm_wreg.cu): which = 0 fwd-x (m, Ms ->
// X), 1 fwd-y (X -> Y), 3 inv-y (Y -> X), 4 inv-x (X -> H); both forms (the
// FP64 form for fewer shapes, f64).
bool wreg_applies(int nx, int ny, int nz, int Px, int Py, bool f64);
void wreg_set_attrs();
// True (and cleared) when a bounded wait of a bulk-copy y pass ran out on the
// current device since the last call (synchronises the device).
bool wreg_take_timeout();
void launch_wreg(int which, const DemagGeom& g, const float* m, const float* Ms, float2* X, float2* Y, float* H,
                 const float2* twx, const float2* twy, cudaStream_t st);
void launch_wreg(int which, const DemagGeom& g, const double* m, const double* Ms, double2* X, double2* Y, double* H,
                 const double2* twx, const double2* twy, cudaStream_t st);

// FP64 Newell tensor (real space) with macro-PBC images, on the device:
// out[c*N + I], c = xx yy zz xy xz yz.  dx,dy,dz are the raw cell sizes.
int newell_tensor_device(int nx, int ny, int nz, double dx, double dy, double dz, int Nx, int Ny,
                         int Nz, double* out_dev, cudaStream_t st);

}  // namespace mm

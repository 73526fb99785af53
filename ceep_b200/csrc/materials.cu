// Per-cell update coefficients of the 2D solver from its FP64 material maps,
// in one pass on the device: the material update of every sample
// (BatchedFDTD2D.update_materials) uploads only the FP64 maps.
//
// The arithmetic is the host formulas' (fdtd_2d_batched.py:151-167 for
// ca/cb, dispersive.py:240-339 for the ADE coefficients), one IEEE-rounded
// FP64 operation at a time in the same order, with the explicit _rn
// intrinsics so that no multiply-add is contracted: the FP32 results equal the
// host formulas' bit for bit.
#include "../../include/ceep_b200.h"
#include "capi_internal.h"

namespace {

struct PoleMaps {
  const double* a[2][3];  // Debye (delta_eps, tau), then Lorentz (delta_eps, omega_0, delta)
};

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dv(double a, double b) { return __ddiv_rn(a, b); }

// One cell (x, y) of the (nx, ny) maps per thread; outputs in the kernels'
// (y, x) order: coef (ny, nx, 4) = (ca, cb, dt/(eps_r eps0), 0), ade
// (poles, ny, nx, 4) = Debye (k1, k2, (1 + k1)/2, 0), Lorentz (k1, k2, k3, 0).
__global__ void __launch_bounds__(256) material_coef_kernel(const double* __restrict__ eps_r,
                                                            const double* __restrict__ sigma, PoleMaps pm,
                                                            int n_debye, int n_lorentz, int nx, int ny, double dt,
                                                            double eps0, float4* __restrict__ coef,
                                                            float4* __restrict__ ade) {
  const long long cells = (long long)nx * ny;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= cells) return;
  const int x = (int)(t % nx), y = (int)(t / nx);  // output order: consecutive threads write consecutive cells
  const long long in = (long long)x * ny + y;
  const double two_eps0 = mul(2.0, eps0);
  double eps_add = 0.0;
  int q = 0;
  for (int k = 0; k < n_debye; ++k, ++q) {
    const double de = pm.a[q][0][in], tau = pm.a[q][1][in];
    const double den = add(mul(2.0, tau), dt);
    const double k1 = dv(sub(mul(2.0, tau), dt), den);
    const double k2 = dv(mul(mul(two_eps0, de), dt), den);
    const bool v = tau > 0.0;
    ade[(size_t)q * cells + t] = v ? make_float4(__double2float_rn(k1), __double2float_rn(k2),
                                                 __double2float_rn(dv(add(1.0, k1), 2.0)), 0.f)
                                   : make_float4(0.f, 0.f, 0.f, 0.f);
    if (v) eps_add = add(eps_add, dv(k2, 2.0));
  }
  for (int k = 0; k < n_lorentz; ++k, ++q) {
    const double de = pm.a[q][0][in], w0 = pm.a[q][1][in], d = pm.a[q][2][in];
    const double w02 = mul(w0, w0), dt2 = mul(dt, dt);
    const double den = add(add(4.0, mul(mul(2.0, d), dt)), mul(w02, dt2));
    const double k2 = dv(mul(mul(mul(two_eps0, de), w02), dt2), den);
    const double k1 = dv(sub(8.0, mul(mul(2.0, w02), dt2)), den);
    const double k3 = dv(-add(sub(4.0, mul(mul(2.0, d), dt)), mul(w02, dt2)), den);
    const bool v = w0 > 0.0;
    ade[(size_t)q * cells + t] = v ? make_float4(__double2float_rn(k1), __double2float_rn(k2),
                                                 __double2float_rn(k3), 0.f)
                                   : make_float4(0.f, 0.f, 0.f, 0.f);
    if (v) eps_add = add(eps_add, dv(k2, 2.0));
  }
  const double er = eps_r[in];
  double eps = mul(er, eps0);
  if (q > 0) eps = add(eps, eps_add);
  const double s = dv(mul(sigma[in], dt), mul(2.0, eps));
  const double ca = dv(sub(1.0, s), add(1.0, s));
  const double cb = dv(dv(dt, eps), add(1.0, s));
  const double dteps = dv(dt, mul(er, eps0));
  coef[t] = make_float4(__double2float_rn(ca), __double2float_rn(cb), __double2float_rn(dteps), 0.f);
}

}  // namespace

extern "C" int ceep2d_material_coefficients(const double* eps_r, const double* sigma, const double* const* poles,
                                            int32_t n_debye, int32_t n_lorentz, int32_t nx, int32_t ny, double dt,
                                            double eps0, float* coef, float* ade, void* stream) {
  if (!eps_r || !sigma || !coef || nx < 1 || ny < 1 || n_debye < 0 || n_lorentz < 0 || n_debye + n_lorentz > 2)
    return ceep::fail(CEEP_ERR_INVALID, "ceep2d_material_coefficients: bad argument (nx=%d ny=%d poles=%d+%d)", nx,
                      ny, n_debye, n_lorentz);
  PoleMaps pm = {};
  const int np = n_debye + n_lorentz;
  if (np > 0 && (!poles || !ade)) return ceep::fail(CEEP_ERR_INVALID, "ceep2d_material_coefficients: null pole maps");
  for (int q = 0, i = 0; q < np; ++q) {
    const int w = q < n_debye ? 2 : 3;
    for (int c = 0; c < w; ++c, ++i) {
      if (!poles[i]) return ceep::fail(CEEP_ERR_INVALID, "ceep2d_material_coefficients: null pole map %d", i);
      pm.a[q][c] = poles[i];
    }
  }
  const long long cells = (long long)nx * ny;
  const unsigned blocks = (unsigned)((cells + 255) / 256);
  material_coef_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      eps_r, sigma, pm, n_debye, n_lorentz, nx, ny, dt, eps0, reinterpret_cast<float4*>(coef),
      reinterpret_cast<float4*>(ade));
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? CEEP_OK : ceep::cuda_fail(e, "material_coef_kernel launch");
}

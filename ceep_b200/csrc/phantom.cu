// Device rasteriser of the concentric-circle brain phantom of
// src/ceep/phantoms/head_models.py:519-631 (BrainPhantom2D with the fixed
// tissue table, use_gabriel_database=False) and of the hemorrhage mask of
// scripts/generate_corrected_dataset.py:110-118, for a batch of phantoms.
//
// Every distance is evaluated in FP64 with explicitly rounded operations
// (no contraction into FMAs), in the order of the NumPy expressions:
//   r     = sqrt(((x - cx) dx)^2 + ((y - cy) dx)^2)
//   r_hem = sqrt(((x - cx) dx - hx)^2 + ((y - cy) dx - hy)^2)
// so the layer and hemorrhage boundaries fall on the same cells as NumPy's.
#include "../../include/ceep_b200.h"
#include "capi_internal.h"
#include "common.cuh"

namespace ceep {

struct BrainPhantomParams {
  int batch, nx, ny;
  double dx;
  double r_skin, r_skull, r_csf, r_gray, r_white;  // outer radius of each layer
  double tissue[6][2];                             // (eps_r, sigma): skin, skull, csf, gray, white, blood
};

__global__ void brain_phantom_kernel(const BrainPhantomParams p, const double* __restrict__ hem,
                                     double* __restrict__ eps, double* __restrict__ sigma,
                                     double* __restrict__ mask) {
  const long long cells = (long long)p.nx * p.ny;
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= cells * p.batch) return;
  const int b = (int)(id / cells);
  const long long c = id % cells;
  const int x = (int)(c / p.ny), y = (int)(c % p.ny);  // (nx, ny) maps, y fastest
  const int cx = p.nx / 2, cy = p.ny / 2;
  const double ux = __dmul_rn((double)(x - cx), p.dx), uy = __dmul_rn((double)(y - cy), p.dx);
  const double r = __dsqrt_rn(__dadd_rn(__dmul_rn(ux, ux), __dmul_rn(uy, uy)));
  int t = -1;  // layer (head_models.py:598-616, outside-in)
  if (r <= p.r_skin && r > p.r_skull) t = 0;
  else if (r <= p.r_skull && r > p.r_csf) t = 1;
  else if (r <= p.r_csf && r > p.r_gray) t = 2;
  else if (r <= p.r_gray && r > p.r_white) t = 3;
  else if (r <= p.r_white) t = 4;
  double m = 0.0;
  const double hr = hem[3 * b + 2];
  if (hr >= 0.0) {  // hemorrhage disk (head_models.py:618-629)
    const double vx = __dsub_rn(ux, hem[3 * b]), vy = __dsub_rn(uy, hem[3 * b + 1]);
    const double rh = __dsqrt_rn(__dadd_rn(__dmul_rn(vx, vx), __dmul_rn(vy, vy)));
    if (rh <= hr) {
      t = 5;
      m = 1.0;
    }
  }
  const size_t o = (size_t)b * cells + c;
  eps[o] = t >= 0 ? p.tissue[t][0] : 1.0;
  sigma[o] = t >= 0 ? p.tissue[t][1] : 0.0;
  if (mask) mask[o] = m;
}

}  // namespace ceep

// radii and tissue are host arrays (copied into the kernel's parameters);
// hem and the outputs are device arrays.
extern "C" int ceep_brain_phantom_2d(int32_t batch, int32_t nx, int32_t ny, double dx, const double* radii,
                                     const double* tissue, const double* hem, double* eps_out, double* sigma_out,
                                     double* mask_out, void* stream) {
  if (!radii || !tissue || !hem || !eps_out || !sigma_out)
    return ceep::fail(CEEP_ERR_INVALID, "ceep_brain_phantom_2d: null pointer");
  if (batch < 1 || nx < 1 || ny < 1 || !(dx > 0.0))
    return ceep::fail(CEEP_ERR_INVALID, "ceep_brain_phantom_2d: batch=%d grid %dx%d dx=%g", batch, nx, ny, dx);
  ceep::BrainPhantomParams p;
  p.batch = batch;
  p.nx = nx;
  p.ny = ny;
  p.dx = dx;
  p.r_skin = radii[0];
  p.r_skull = radii[1];
  p.r_csf = radii[2];
  p.r_gray = radii[3];
  p.r_white = radii[4];
  for (int t = 0; t < 6; ++t) {
    p.tissue[t][0] = tissue[2 * t];
    p.tissue[t][1] = tissue[2 * t + 1];
  }
  const long long n = (long long)batch * nx * ny;
  const unsigned blocks = (unsigned)((n + 255) / 256);
  ceep::brain_phantom_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(p, hem, eps_out, sigma_out,
                                                                                     mask_out);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? CEEP_OK : ceep::cuda_fail(e, "brain_phantom_kernel launch");
}

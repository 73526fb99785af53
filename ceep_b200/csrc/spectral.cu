// On-device DFT into the S-matrix and delay-and-sum imaging (sm_100a).
#include <cuda_runtime.h>

#include "../../include/ceep_b200.h"
#include "capi_internal.h"
#include "common.cuh"

namespace ceep {

// --------------------------------------------------------------------------
// DFT: S[f, rx, tx] = sum_n series[tx, rx, n] * tw[f, n]   (dft.py:55-90)
// A (freq x pair) tile per block, the time axis staged through shared memory
// in chunks of 32 samples; each thread owns a 2x2 block of outputs.  FP32
// accumulation over <= a few thousand samples stays ~1e-6 relative.
// --------------------------------------------------------------------------
constexpr int kDftT = 32;   // tile edge (freqs and pairs)
constexpr int kDftC = 32;   // samples per chunk

__global__ void __launch_bounds__(256) dft_kernel(const float* __restrict__ series, const float2* __restrict__ tw,
                                                  float2* __restrict__ out, int ntx, int nprobe, int nsteps,
                                                  int nfreq) {
  __shared__ float2 s_tw[kDftT][kDftC + 1];
  __shared__ float s_x[kDftT][kDftC + 1];
  const int npair = ntx * nprobe;
  const int f0 = blockIdx.x * kDftT, k0 = blockIdx.y * kDftT;
  const int tf = threadIdx.x / 16, tk = threadIdx.x % 16;
  float2 acc[2][2] = {};
  for (int c0 = 0; c0 < nsteps; c0 += kDftC) {
    for (int i = threadIdx.x; i < kDftT * kDftC; i += blockDim.x) {
      const int r = i / kDftC, c = i % kDftC, n = c0 + c;
      const int f = f0 + r, k = k0 + r;
      s_tw[r][c] = (f < nfreq && n < nsteps) ? tw[(size_t)f * nsteps + n] : make_float2(0.f, 0.f);
      s_x[r][c] = (k < npair && n < nsteps) ? series[(size_t)k * nsteps + n] : 0.f;
    }
    __syncthreads();
#pragma unroll 8
    for (int c = 0; c < kDftC; ++c) {
      const float2 w0 = s_tw[tf][c], w1 = s_tw[tf + 16][c];
      const float x0 = s_x[tk][c], x1 = s_x[tk + 16][c];
      acc[0][0].x = fmaf(w0.x, x0, acc[0][0].x); acc[0][0].y = fmaf(w0.y, x0, acc[0][0].y);
      acc[0][1].x = fmaf(w0.x, x1, acc[0][1].x); acc[0][1].y = fmaf(w0.y, x1, acc[0][1].y);
      acc[1][0].x = fmaf(w1.x, x0, acc[1][0].x); acc[1][0].y = fmaf(w1.y, x0, acc[1][0].y);
      acc[1][1].x = fmaf(w1.x, x1, acc[1][1].x); acc[1][1].y = fmaf(w1.y, x1, acc[1][1].y);
    }
    __syncthreads();
  }
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      const int f = f0 + tf + 16 * a, k = k0 + tk + 16 * b;
      if (f < nfreq && k < npair) {
        const int tx = k / nprobe, rx = k % nprobe;
        out[((size_t)f * nprobe + rx) * ntx + tx] = acc[a][b];
      }
    }
}

// --------------------------------------------------------------------------
// Frequency-domain DAS (beamforming.py:210-257).
// The two-way phasor factorises: exp(-j k (d_tx + d_rx)) = a_tx * a_rx with
// a_m = exp(-j k d_m), so per (pixel, f) the image term is
//   sum_tx a_tx * sum_rx S[f, rx, tx] a_rx
// i.e. N sincos + N^2 complex MACs instead of N^2 sincos.  Pixels map to
// threads; frequencies are split into chunks across blockIdx.y so a small
// image still fills all SMs; each chunk writes its partial complex sum to
// the caller's workspace and a finishing kernel adds the chunks, takes |.|
// and applies (I - min) / max.
// --------------------------------------------------------------------------
constexpr int kDasThreads = 128;
constexpr int kDasMaxAnt = 32;
// Largest image (pixels) the image kernels take: pixel indices are int, and
// the last block's thread indices must stay below INT_MAX too.
constexpr int64_t kMaxPixels = int64_t(1) << 30;

// Pixel count of an nx x ny image formed in 64 bits; -1 when either side is
// below 1 or the count exceeds kMaxPixels.
static int64_t pixel_count(int32_t nx, int32_t ny) {
  if (nx < 1 || ny < 1) return -1;
  const int64_t n = (int64_t)nx * (int64_t)ny;
  return n > kMaxPixels ? -1 : n;
}

static int das_chunks(int64_t npix, int nfreq) {
  const int64_t pixblocks = (npix + kDasThreads - 1) / kDasThreads;
  int chunks = (int)((2 * 148 + pixblocks - 1) / pixblocks);
  if (chunks > nfreq) chunks = nfreq;
  if (chunks < 1) chunks = 1;
  return chunks;
}

template <int MAXN>
__global__ void __launch_bounds__(kDasThreads) das_partial_kernel(const float2* __restrict__ s,
                                                                 const float* __restrict__ kfreq,
                                                                 const float* __restrict__ ant, int nfreq, int nant,
                                                                 int nxp, int nyp, float px0, float py0, float pix,
                                                                 int chunks, float2* __restrict__ partial) {
  extern __shared__ float2 s_s[];  // (fchunk, nant, nant)
  const int npix = nxp * nyp;
  const int fpc = (nfreq + chunks - 1) / chunks;
  const int fa = blockIdx.y * fpc, fb = min(nfreq, fa + fpc);
  const int nn = nant * nant;
  for (int i = threadIdx.x; i < (fb - fa) * nn; i += blockDim.x) s_s[i] = s[(size_t)fa * nn + i];
  __syncthreads();
  const int pid = blockIdx.x * blockDim.x + threadIdx.x;
  if (pid >= npix) return;
  const int i = pid / nyp, j = pid % nyp;
  const float px = px0 + i * pix, py = py0 + j * pix;
  float d[MAXN];
#pragma unroll
  for (int m = 0; m < MAXN; ++m) {
    if (m < nant) {
      const float dx = px - ant[2 * m], dy = py - ant[2 * m + 1];
      d[m] = sqrtf(dx * dx + dy * dy);
    }
  }
  float accx = 0.f, accy = 0.f;
  for (int f = fa; f < fb; ++f) {
    const float k = kfreq[f];
    float ar[MAXN], ai[MAXN];
#pragma unroll
    for (int m = 0; m < MAXN; ++m) {
      if (m < nant) {
        float sn, cs;
        sincosf(k * d[m], &sn, &cs);
        ar[m] = cs;
        ai[m] = -sn;
      }
    }
    const float2* S = s_s + (size_t)(f - fa) * nn;
#pragma unroll
    for (int tx = 0; tx < MAXN; ++tx) {
      if (tx < nant) {
        float tr = 0.f, ti = 0.f;
#pragma unroll
        for (int rx = 0; rx < MAXN; ++rx) {
          if (rx < nant) {
            const float2 v = S[rx * nant + tx];
            tr = fmaf(v.x, ar[rx], fmaf(-v.y, ai[rx], tr));
            ti = fmaf(v.x, ai[rx], fmaf(v.y, ar[rx], ti));
          }
        }
        accx = fmaf(tr, ar[tx], fmaf(-ti, ai[tx], accx));
        accy = fmaf(tr, ai[tx], fmaf(ti, ar[tx], accy));
      }
    }
  }
  partial[(size_t)blockIdx.y * npix + pid] = make_float2(accx, accy);
}

// Single block: add the chunks, |.|, min/max with warp shuffles, normalise.
__global__ void __launch_bounds__(1024) das_finish_kernel(const float2* __restrict__ partial, int chunks, int npix,
                                                          int normalize, float* __restrict__ image) {
  __shared__ float s_min[32], s_max[32];
  float lo = 3.4e38f, hi = 0.f;
  for (int p = threadIdx.x; p < npix; p += blockDim.x) {
    float x = 0.f, y = 0.f;
    for (int c = 0; c < chunks; ++c) {
      const float2 v = partial[(size_t)c * npix + p];
      x += v.x;
      y += v.y;
    }
    const float m = hypotf(x, y);
    image[p] = m;
    lo = fminf(lo, m);
    hi = fmaxf(hi, m);
  }
  if (!normalize) return;
  for (int o = 16; o > 0; o >>= 1) {
    lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  const int w = threadIdx.x / 32, ln = threadIdx.x % 32;
  if (ln == 0) { s_min[w] = lo; s_max[w] = hi; }
  __syncthreads();
  if (w == 0) {
    const int nw = (blockDim.x + 31) / 32;
    lo = ln < nw ? s_min[ln] : 3.4e38f;
    hi = ln < nw ? s_max[ln] : 0.f;
    for (int o = 16; o > 0; o >>= 1) {
      lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
      hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if (ln == 0) { s_min[0] = lo; s_max[0] = hi; }
  }
  __syncthreads();
  lo = s_min[0];
  const float range = s_max[0] - lo;
  for (int p = threadIdx.x; p < npix; p += blockDim.x) {
    const float v = image[p] - lo;
    image[p] = range > 0.f ? v / range : v;
  }
}

// --------------------------------------------------------------------------
// Frequency-domain DMAS (beamforming.py:259-313).  One block per pixel, one
// thread per transmit/receive pair k = tx * N + rx (the reference's loop
// order): the thread accumulates the delayed pair signal
//   s_k = sum_f S[f, rx, tx] a_tx(f) a_rx(f),  a_n(f) = exp(-j k_f d_n),
// with the antenna phasors of a chunk of frequencies built once per pixel in
// shared memory (the DAS kernel's factorisation).  The block then forms the
// ordered pair sum  sum_{k1<k2} s_k1 conj(s_k2) = sum_k s_k conj(R_k),
// R_k = sum_{k'>k} s_k', from an inclusive suffix scan over k, and writes the
// complex result; das_finish_kernel takes |.| and normalises.
// --------------------------------------------------------------------------
constexpr int kDmasMaxAnt = 32;  // N^2 <= 1024 pairs, one thread each
constexpr int kDmasFreqChunk = 32;

__global__ void __launch_bounds__(1024) dmas_kernel(const float2* __restrict__ S, const float* __restrict__ kf,
                                                    const float* __restrict__ ant, int F, int N, int nyp, float px0,
                                                    float py0, float pix, float2* __restrict__ out) {
  extern __shared__ float2 dm_smem[];
  float2* a = dm_smem;                          // (N, kDmasFreqChunk) phasors
  float2* scan = dm_smem + N * kDmasFreqChunk;  // (blockDim.x) pair signals, then suffix sums
  __shared__ float d[kDmasMaxAnt];
  __shared__ float2 wsum[32];
  const int pid = blockIdx.x, i = pid / nyp, j = pid % nyp;
  const float px = px0 + i * pix, py = py0 + j * pix;
  const int K = N * N, t = threadIdx.x;
  if (t < N) d[t] = hypotf(px - ant[2 * t], py - ant[2 * t + 1]);
  __syncthreads();
  const int tx = t / N, rx = t % N;
  float sx = 0.f, sy = 0.f;
  for (int f0 = 0; f0 < F; f0 += kDmasFreqChunk) {
    const int fc = min(kDmasFreqChunk, F - f0);
    for (int e = t; e < N * fc; e += blockDim.x) {
      const int nn = e / fc, ff = e % fc;
      float sn, cs;
      sincosf(-kf[f0 + ff] * d[nn], &sn, &cs);
      a[nn * kDmasFreqChunk + ff] = make_float2(cs, sn);
    }
    __syncthreads();
    if (t < K) {
      for (int ff = 0; ff < fc; ++ff) {
        const float2 v = __ldg(S + ((size_t)(f0 + ff) * N + rx) * N + tx);
        const float2 at = a[tx * kDmasFreqChunk + ff], ar = a[rx * kDmasFreqChunk + ff];
        const float ph_x = at.x * ar.x - at.y * ar.y, ph_y = at.x * ar.y + at.y * ar.x;
        sx += v.x * ph_x - v.y * ph_y;
        sy += v.x * ph_y + v.y * ph_x;
      }
    }
    __syncthreads();
  }
  // inclusive suffix scan: scan[k] = sum_{k' >= k} s_k'
  scan[t] = t < K ? make_float2(sx, sy) : make_float2(0.f, 0.f);
  __syncthreads();
  for (int off = 1; off < K; off <<= 1) {
    const float2 v = t + off < K ? scan[t + off] : make_float2(0.f, 0.f);
    __syncthreads();
    scan[t].x += v.x;
    scan[t].y += v.y;
    __syncthreads();
  }
  // s_k conj(R_k), R_k = scan[k + 1]
  float ax = 0.f, ay = 0.f;
  if (t + 1 < K) {
    const float2 r = scan[t + 1];
    ax = sx * r.x + sy * r.y;
    ay = sy * r.x - sx * r.y;
  }
  for (int o = 16; o > 0; o >>= 1) {
    ax += __shfl_xor_sync(0xffffffffu, ax, o);
    ay += __shfl_xor_sync(0xffffffffu, ay, o);
  }
  if ((t & 31) == 0) wsum[t / 32] = make_float2(ax, ay);
  __syncthreads();
  if (t < 32) {
    const int nw = blockDim.x / 32;
    float2 v = t < nw ? wsum[t] : make_float2(0.f, 0.f);
    for (int o = 16; o > 0; o >>= 1) {
      v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
      v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    if (t == 0) out[pid] = v;
  }
}

// --------------------------------------------------------------------------
// Time-domain DAS (scripts/verify_dataset_with_das.py:37-103), one thread per
// pixel.  The delay index is truncated like int() in FP64, so every rounding
// matters: |v| is sqrt(fma(v1, v1, v0*v0)), the rounding sequence of
// np.linalg.norm on a 2-vector (its BLAS dot product), then the two sums and
// divisions in the reference's order.
// --------------------------------------------------------------------------
__global__ void das_time_kernel(const float2* __restrict__ s, const double* __restrict__ ant, int nant, int ntime,
                                int grid, double dx, double dt, float* __restrict__ image) {
  const int pid = blockIdx.x * blockDim.x + threadIdx.x;
  if (pid >= grid * grid) return;
  const int i = pid / grid, j = pid % grid;
  const double px = __dmul_rn((double)i, dx), py = __dmul_rn((double)j, dx);
  const double C = 3e8;
  double acc = 0.0;
  for (int tx = 0; tx < nant; ++tx) {
    const double ax = __dsub_rn(ant[2 * tx], px), ay = __dsub_rn(ant[2 * tx + 1], py);
    const double dtx = __dsqrt_rn(__fma_rn(ay, ay, __dmul_rn(ax, ax)));
    for (int rx = 0; rx < nant; ++rx) {
      if (rx == tx) continue;
      const double bx = __dsub_rn(ant[2 * rx], px), by = __dsub_rn(ant[2 * rx + 1], py);
      const double drx = __dsqrt_rn(__fma_rn(by, by, __dmul_rn(bx, bx)));
      const double t = __ddiv_rn(__ddiv_rn(__dadd_rn(dtx, drx), C), dt);
      const long long idx = (long long)t;  // truncation toward zero, as int()
      if (idx >= 0 && idx < ntime) {
        const float2 v = s[((size_t)tx * nant + rx) * ntime + idx];
        acc += hypot((double)v.x, (double)v.y);
      }
    }
  }
  image[pid] = (float)acc;
}

}  // namespace ceep

using ceep::fail;

extern "C" int ceep_dft(const float* series, const float* twiddle, float* s_out, int32_t ntx, int32_t nprobe,
                        int32_t nsteps, int32_t nfreq, void* stream) {
  if (!series || !twiddle || !s_out) return fail(CEEP_ERR_INVALID, "ceep_dft: null pointer");
  if (ntx < 1 || nprobe < 1 || nsteps < 1 || nfreq < 1)
    return fail(CEEP_ERR_INVALID, "ceep_dft: sizes ntx=%d nprobe=%d nsteps=%d nfreq=%d", ntx, nprobe, nsteps,
                nfreq);
  dim3 grid((nfreq + ceep::kDftT - 1) / ceep::kDftT, (ntx * nprobe + ceep::kDftT - 1) / ceep::kDftT);
  ceep::dft_kernel<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      series, reinterpret_cast<const float2*>(twiddle), reinterpret_cast<float2*>(s_out), ntx, nprobe, nsteps,
      nfreq);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? CEEP_OK : ceep::cuda_fail(e, "dft_kernel launch");
}

extern "C" int64_t ceep_das_workspace_bytes(int32_t nx_pix, int32_t ny_pix, int32_t nfreq) {
  const int64_t npix = ceep::pixel_count(nx_pix, ny_pix);
  if (npix < 0 || nfreq < 1) return 0;
  return (int64_t)ceep::das_chunks(npix, nfreq) * npix * (int64_t)sizeof(float2);
}

extern "C" int ceep_das(const float* s, const float* kfreq, const float* ant_xy, int32_t nfreq, int32_t nant,
                        int32_t nx_pix, int32_t ny_pix, float px0, float py0, float pix, int normalize, void* work,
                        float* image, void* stream) {
  if (!s || !kfreq || !ant_xy || !work || !image) return fail(CEEP_ERR_INVALID, "ceep_das: null pointer");
  if (nfreq < 1 || nant < 1 || nx_pix < 1 || ny_pix < 1)
    return fail(CEEP_ERR_INVALID, "ceep_das: sizes nfreq=%d nant=%d image %dx%d", nfreq, nant, nx_pix, ny_pix);
  if (nant > ceep::kDasMaxAnt)
    return fail(CEEP_ERR_UNSUPPORTED, "ceep_das: %d antennas (at most %d)", nant, ceep::kDasMaxAnt);
  if (ceep::pixel_count(nx_pix, ny_pix) < 0)
    return fail(CEEP_ERR_UNSUPPORTED, "ceep_das: image %dx%d exceeds %lld pixels", nx_pix, ny_pix,
                (long long)ceep::kMaxPixels);
  const int npix = nx_pix * ny_pix;
  const int chunks = ceep::das_chunks(npix, nfreq);
  const int fpc = (nfreq + chunks - 1) / chunks;
  const size_t smem = (size_t)fpc * nant * nant * sizeof(float2);
  if (smem > 200 * 1024) return fail(CEEP_ERR_UNSUPPORTED, "ceep_das: S chunk of %zu bytes too large", smem);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  dim3 grid((npix + ceep::kDasThreads - 1) / ceep::kDasThreads, chunks);
  float2* partial = static_cast<float2*>(work);
  const float2* S = reinterpret_cast<const float2*>(s);
  cudaError_t e;
#define CEEP_DAS_LAUNCH(M)                                                                                 \
  e = cudaFuncSetAttribute(ceep::das_partial_kernel<M>, cudaFuncAttributeMaxDynamicSharedMemorySize,      \
                           (int)smem);                                                                     \
  if (e == cudaSuccess) {                                                                                  \
    ceep::das_partial_kernel<M><<<grid, ceep::kDasThreads, smem, st>>>(S, kfreq, ant_xy, nfreq, nant,      \
                                                                      nx_pix, ny_pix, px0, py0, pix,       \
                                                                      chunks, partial);                    \
    e = cudaGetLastError();                                                                                \
  }
  if (nant <= 8) {
    CEEP_DAS_LAUNCH(8)
  } else if (nant <= 16) {
    CEEP_DAS_LAUNCH(16)
  } else {
    CEEP_DAS_LAUNCH(32)
  }
#undef CEEP_DAS_LAUNCH
  if (e != cudaSuccess) return ceep::cuda_fail(e, "das_partial_kernel launch");
  ceep::das_finish_kernel<<<1, 1024, 0, st>>>(partial, chunks, npix, normalize, image);
  e = cudaGetLastError();
  return e == cudaSuccess ? CEEP_OK : ceep::cuda_fail(e, "das_finish_kernel launch");
}

extern "C" int64_t ceep_dmas_workspace_bytes(int32_t nx_pix, int32_t ny_pix) {
  const int64_t npix = ceep::pixel_count(nx_pix, ny_pix);
  return npix > 0 ? npix * (int64_t)sizeof(float2) : 0;
}

extern "C" int ceep_dmas(const float* s, const float* kfreq, const float* ant_xy, int32_t nfreq, int32_t nant,
                         int32_t nx_pix, int32_t ny_pix, float px0, float py0, float pix, int normalize, void* work,
                         float* image, void* stream) {
  if (!s || !kfreq || !ant_xy || !work || !image) return fail(CEEP_ERR_INVALID, "ceep_dmas: null pointer");
  if (nfreq < 1 || nant < 1 || nx_pix < 1 || ny_pix < 1)
    return fail(CEEP_ERR_INVALID, "ceep_dmas: sizes nfreq=%d nant=%d image %dx%d", nfreq, nant, nx_pix, ny_pix);
  if (nant > ceep::kDmasMaxAnt)
    return fail(CEEP_ERR_UNSUPPORTED, "ceep_dmas: %d antennas (at most %d)", nant, ceep::kDmasMaxAnt);
  if (ceep::pixel_count(nx_pix, ny_pix) < 0)
    return fail(CEEP_ERR_UNSUPPORTED, "ceep_dmas: image %dx%d exceeds %lld pixels", nx_pix, ny_pix,
                (long long)ceep::kMaxPixels);
  const int npix = nx_pix * ny_pix;
  const int K = nant * nant;
  const int threads = ((K + 31) / 32) * 32;
  const size_t smem = ((size_t)nant * ceep::kDmasFreqChunk + threads) * sizeof(float2);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  float2* acc = static_cast<float2*>(work);
  ceep::dmas_kernel<<<npix, threads, smem, st>>>(reinterpret_cast<const float2*>(s), kfreq, ant_xy, nfreq, nant,
                                                 ny_pix, px0, py0, pix, acc);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return ceep::cuda_fail(e, "dmas_kernel launch");
  ceep::das_finish_kernel<<<1, 1024, 0, st>>>(acc, 1, npix, normalize, image);
  e = cudaGetLastError();
  return e == cudaSuccess ? CEEP_OK : ceep::cuda_fail(e, "das_finish_kernel launch");
}

extern "C" int ceep_das_time(const float* s, const double* ant_xy, int32_t nant, int32_t ntime, int32_t grid,
                             double dx, double frequency, float* image, void* stream) {
  if (!s || !ant_xy || !image) return fail(CEEP_ERR_INVALID, "ceep_das_time: null pointer");
  if (nant < 1 || ntime < 1 || grid < 1 || !(frequency > 0))
    return fail(CEEP_ERR_INVALID, "ceep_das_time: sizes nant=%d ntime=%d grid=%d", nant, ntime, grid);
  if (ceep::pixel_count(grid, grid) < 0)
    return fail(CEEP_ERR_UNSUPPORTED, "ceep_das_time: image %dx%d exceeds %lld pixels", grid, grid,
                (long long)ceep::kMaxPixels);
  const double dt = 1.0 / (4.0 * frequency);
  const int npix = grid * grid;
  ceep::das_time_kernel<<<(npix + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(
      reinterpret_cast<const float2*>(s), ant_xy, nant, ntime, grid, dx, dt, image);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? CEEP_OK : ceep::cuda_fail(e, "das_time_kernel launch");
}

// --------------------------------------------------------------------------
// Delay-and-sum without a caller workspace.
//
// Some callers cannot hand this library any device memory: for example an
// imaging pipeline that reserves all of its GPU memory in its own pool at
// start-up and must not allocate while a scan is running, or a host
// application whose allocator this library cannot reach.  For them the
// partial sums of ceep_das live in one fixed array that the library itself
// declares at file scope, so the call needs no cudaMalloc at all.
//
// Facts a caller must know:
//  * The array holds kDasNoAllocScratch complex partial sums (2 MiB).  Every
//    GPU that loads this library keeps that much memory reserved until the
//    process exits.  Images whose (frequency chunks x pixels) exceed it are
//    rejected with CEEP_ERR_UNSUPPORTED before anything is launched.
//  * In host code the array's name is only a host-side stand-in; its device
//    address is looked up with cudaGetSymbolAddress on the first call made
//    on each device (with that device current) and cached.  That first call
//    therefore does set-up work and should be made before any stream capture.
//    With lazy module loading (the CUDA 12.2+ default) the array is made
//    resident by that first call too, so a host that reserves all of its GPU
//    memory up front makes one call first (or sets CUDA_MODULE_LOADING=EAGER).
//  * A call that fails with a CUDA error drops the cached address, so the
//    next call looks it up again (after a device reset the module, and with
//    it the array, can move).
//  * Every call on a device shares the one array.  Two calls whose kernels
//    overlap on the GPU (different streams, no ordering between them) race
//    on it and give wrong images; order them on one stream or serialise them.
//  * Nothing in the array needs to start at zero: the partial-sum kernel
//    writes every entry that the finishing kernel later reads, so the
//    contents a previous call left behind are never used.
// --------------------------------------------------------------------------
namespace ceep {
constexpr int64_t kDasNoAllocScratch = 262144;  // float2 entries = 2 MiB
static __device__ __align__(256) float2 g_das_noalloc_scratch[kDasNoAllocScratch];
}  // namespace ceep

#include <mutex>

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_das_scratch_mu;
void* g_das_scratch_ptr[kMaxDevices] = {};
}  // namespace

extern "C" int64_t ceep_das_noalloc_capacity(void) { return ceep::kDasNoAllocScratch; }

extern "C" int ceep_das_noalloc(const float* s, const float* kfreq, const float* ant_xy, int32_t nfreq,
                                int32_t nant, int32_t nx_pix, int32_t ny_pix, float px0, float py0, float pix,
                                int normalize, float* image, void* stream) {
  if (!s || !kfreq || !ant_xy || !image) return fail(CEEP_ERR_INVALID, "ceep_das_noalloc: null pointer");
  if (nfreq < 1 || nant < 1 || nx_pix < 1 || ny_pix < 1)
    return fail(CEEP_ERR_INVALID, "ceep_das_noalloc: sizes nfreq=%d nant=%d image %dx%d", nfreq, nant, nx_pix,
                ny_pix);
  if (ceep::pixel_count(nx_pix, ny_pix) < 0)
    return fail(CEEP_ERR_UNSUPPORTED, "ceep_das_noalloc: image %dx%d exceeds %lld pixels", nx_pix, ny_pix,
                (long long)ceep::kMaxPixels);
  const int64_t need = ceep_das_workspace_bytes(nx_pix, ny_pix, nfreq) / (int64_t)sizeof(float2);
  if (need > ceep::kDasNoAllocScratch)
    return fail(CEEP_ERR_UNSUPPORTED,
                "ceep_das_noalloc: %dx%d pixels x %d frequencies need %lld partial sums, the fixed scratch holds "
                "%lld; use ceep_das with a workspace",
                nx_pix, ny_pix, nfreq, (long long)need, (long long)ceep::kDasNoAllocScratch);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return ceep::cuda_fail(e, "ceep_das_noalloc: cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) return fail(CEEP_ERR_UNSUPPORTED, "ceep_das_noalloc: device %d", dev);
  void* scratch;
  {
    std::lock_guard<std::mutex> lock(g_das_scratch_mu);
    if (!g_das_scratch_ptr[dev]) {
      void* ptr = nullptr;
      e = cudaGetSymbolAddress(&ptr, ceep::g_das_noalloc_scratch);
      if (e != cudaSuccess || !ptr) return ceep::cuda_fail(e, "ceep_das_noalloc: cudaGetSymbolAddress");
      g_das_scratch_ptr[dev] = ptr;
    }
    scratch = g_das_scratch_ptr[dev];
  }
  const int rc = ceep_das(s, kfreq, ant_xy, nfreq, nant, nx_pix, ny_pix, px0, py0, pix, normalize, scratch, image,
                          stream);
  if (rc == CEEP_ERR_CUDA) {
    std::lock_guard<std::mutex> lock(g_das_scratch_mu);
    g_das_scratch_ptr[dev] = nullptr;
  }
  return rc;
}

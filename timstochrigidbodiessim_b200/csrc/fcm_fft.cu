// fcm_fft.cu -- standalone fft_solver (fft_solver.hpp:10-31, fft_solver.cpp:17-42):
// in-place 3-D real transforms of the reference's padded [x][y][pad] arrays with
// FFTW 2.x rfftwnd_mpi semantics on one rank:
//   forward : unnormalised R2C, sign e^{-iqx}, result in FFTW_TRANSPOSED_ORDER
//             [y][x][kz] (re,im);
//   inverse : complex inverse along x and y, then half-complex-to-real along z
//             ignoring Im of kz = 0 and kz = nz/2.  cuFFT's C2R is only defined
//             for Hermitian input, so the kz = 0 and kz = nz/2 planes are first
//             replaced by their Hermitian parts (H(k) + conj H(-k))/2, which is
//             exactly what the real part of FFTW's 2-D inverse keeps.
#include <cstring>
#include <vector>

#include "fcm_internal.cuh"

struct fcm_fft {
  int nx, ny, nz, nzh;
  long long G, Gc;
  double* real = nullptr;                // G
  cufftDoubleComplex* spec = nullptr;    // Gc, [x][y][kz]
  cufftDoubleComplex* tspec = nullptr;   // Gc, [y][x][kz]
  cufftHandle r2c = 0, c2r = 0;
};

namespace fcm {
namespace {

__global__ void k_transpose_xy(const cufftDoubleComplex* __restrict__ in, cufftDoubleComplex* __restrict__ out,
                               int n0, int n1, int nzh) {
  // in [n0][n1][nzh] -> out [n1][n0][nzh]
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long total = (long long)n0 * n1 * nzh;
  if (t >= total) return;
  const int k = (int)(t % nzh);
  const long long ab = t / nzh;
  const int b = (int)(ab % n1), a = (int)(ab / n1);
  out[((long long)b * n0 + a) * nzh + k] = in[t];
}

// Hermitian part of the kz = 0 and kz = nz/2 planes, one thread per {k,-k} pair.
__global__ void k_hermitian_planes(cufftDoubleComplex* __restrict__ s, int nx, int ny, int nz, int nzh) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int nplanes = (nz % 2 == 0 && nz / 2 != 0) ? 2 : 1;
  const long long per = (long long)nx * ny;
  if (t >= per * nplanes) return;
  const int kz = (t < per) ? 0 : nz / 2;
  const long long xy = t % per;
  const int y = (int)(xy % ny), x = (int)(xy / ny);
  const int xp = (nx - x) % nx, yp = (ny - y) % ny;
  const long long i = ((long long)x * ny + y) * nzh + kz, ip = ((long long)xp * ny + yp) * nzh + kz;
  if (ip < i) return;
  const cufftDoubleComplex a = s[i];
  if (ip == i) {
    s[i].y = 0.0;
    return;
  }
  const cufftDoubleComplex b = s[ip];
  cufftDoubleComplex h;
  h.x = 0.5 * (a.x + b.x);
  h.y = 0.5 * (a.y - b.y);
  s[i] = h;
  h.y = -h.y;
  s[ip] = h;
}

}  // namespace
}  // namespace fcm

using namespace fcm;

extern "C" {

int fcm_fft_create(int32_t nx, int32_t ny, int32_t nz, fcm_fft** out) {
  if (!out || nx < 1 || ny < 1 || nz < 2) {
    set_error("fcm_fft_create: bad sizes");
    return FCM_ERR_INVALID;
  }
  fcm_fft* f = new fcm_fft();
  f->nx = nx;
  f->ny = ny;
  f->nz = nz;
  f->nzh = nz / 2 + 1;
  f->G = (long long)nx * ny * nz;
  f->Gc = (long long)nx * ny * f->nzh;
  if (cudaMalloc(&f->real, sizeof(double) * f->G) != cudaSuccess ||
      cudaMalloc(&f->spec, sizeof(cufftDoubleComplex) * f->Gc) != cudaSuccess ||
      cudaMalloc(&f->tspec, sizeof(cufftDoubleComplex) * f->Gc) != cudaSuccess) {
    cudaGetLastError();
    fcm_fft_destroy(f);
    set_error("fcm_fft_create: cudaMalloc failed");
    return FCM_ERR_NOMEM;
  }
  if (cufftPlan3d(&f->r2c, nx, ny, nz, CUFFT_D2Z) != CUFFT_SUCCESS ||
      cufftPlan3d(&f->c2r, nx, ny, nz, CUFFT_Z2D) != CUFFT_SUCCESS) {
    fcm_fft_destroy(f);
    set_error("fcm_fft_create: cufftPlan3d failed");
    return FCM_ERR_CUFFT;
  }
  *out = f;
  return FCM_OK;
}

int fcm_fft_destroy(fcm_fft* f) {
  if (!f) return FCM_OK;
  cudaFree(f->real);
  cudaFree(f->spec);
  cudaFree(f->tspec);
  if (f->r2c) cufftDestroy(f->r2c);
  if (f->c2r) cufftDestroy(f->c2r);
  delete f;
  return FCM_OK;
}

int fcm_fft_local_sizes(const fcm_fft* f, int32_t* local_nx, int32_t* local_x_start, int32_t* local_ny_after_transpose,
                        int32_t* local_y_start_after_transpose, int64_t* total_local_size, int32_t* pad) {
  if (!f) return FCM_ERR_INVALID;
  if (local_nx) *local_nx = f->nx;
  if (local_x_start) *local_x_start = 0;
  if (local_ny_after_transpose) *local_ny_after_transpose = f->ny;
  if (local_y_start_after_transpose) *local_y_start_after_transpose = 0;
  if (total_local_size) *total_local_size = (int64_t)f->nx * f->ny * 2 * f->nzh;
  if (pad) *pad = 2 * f->nzh;
  return FCM_OK;
}

int fcm_fft_transform(fcm_fft* f, double* in) {
  if (!f || !in) return FCM_ERR_INVALID;
  const size_t pad = 2 * (size_t)f->nzh;
  FCM_CUDA(cudaMemcpy2D(f->real, sizeof(double) * f->nz, in, sizeof(double) * pad, sizeof(double) * f->nz,
                        (size_t)f->nx * f->ny, cudaMemcpyDefault));
  FCM_CUFFT(cufftExecD2Z(f->r2c, f->real, f->spec));
  k_transpose_xy<<<(unsigned)((f->Gc + 255) / 256), 256>>>(f->spec, f->tspec, f->nx, f->ny, f->nzh);
  FCM_LAUNCH_CHECK();
  FCM_CUDA(cudaMemcpy(in, f->tspec, sizeof(cufftDoubleComplex) * f->Gc, cudaMemcpyDefault));
  return FCM_OK;
}

int fcm_fft_inverse_transform(fcm_fft* f, double* in) {
  if (!f || !in) return FCM_ERR_INVALID;
  const size_t pad = 2 * (size_t)f->nzh;
  FCM_CUDA(cudaMemcpy(f->tspec, in, sizeof(cufftDoubleComplex) * f->Gc, cudaMemcpyDefault));
  k_transpose_xy<<<(unsigned)((f->Gc + 255) / 256), 256>>>(f->tspec, f->spec, f->ny, f->nx, f->nzh);
  FCM_LAUNCH_CHECK();
  const long long np = (long long)f->nx * f->ny * 2;
  k_hermitian_planes<<<(unsigned)((np + 255) / 256), 256>>>(f->spec, f->nx, f->ny, f->nz, f->nzh);
  FCM_LAUNCH_CHECK();
  FCM_CUFFT(cufftExecZ2D(f->c2r, f->spec, f->real));
  // real result with zeroed padding slots, staged through the host
  std::vector<double> h((size_t)f->G);
  FCM_CUDA(cudaMemcpy(h.data(), f->real, sizeof(double) * f->G, cudaMemcpyDeviceToHost));
  std::vector<double> o((size_t)f->nx * f->ny * pad, 0.0);
  for (size_t l = 0; l < (size_t)f->nx * f->ny; ++l)
    std::memcpy(&o[l * pad], &h[l * f->nz], sizeof(double) * f->nz);
  FCM_CUDA(cudaMemcpy(in, o.data(), sizeof(double) * o.size(), cudaMemcpyDefault));
  return FCM_OK;
}

}  // extern "C"

// shim.cpp -- TEST INFRASTRUCTURE ONLY.  Implementations behind the stand-in
// headers of the reference build (oracle/ref_shim): the SPRNG uniform stream,
// the Armadillo random draws and the FFTW 2.x MPI real 3-D transforms, all for
// one rank.  Project-written; see the headers for the conventions followed.
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../philox.h"
#include "armadillo"
#include "rfftw_mpi.h"
#include "sprng.h"

namespace {
orcrng::UniformStream g_sprng(1234, 0);
orcrng::UniformStream g_arma(0x61726d61, 0);
}  // namespace

extern "C" double sprng(void) { return g_sprng.next(); }
extern "C" void ref_sprng_reset(uint64_t seed, uint64_t stream) { g_sprng = orcrng::UniformStream(seed, stream); }

namespace arma {
double ref_arma_uniform() { return g_arma.next(); }
double ref_arma_normal() { return g_arma.gaussian_random(); }
void ref_arma_seed(unsigned long long seed) { g_arma = orcrng::UniformStream(seed, 0); }
}  // namespace arma

// ------------------------------------------------------------------ FFT
namespace {
typedef std::complex<double> cd;
const double PI = 3.14159265358979323846264338327950288;

// Unnormalised DFT of n points read from in[0], in[s], ... into out[0..n):
// decimation in time by the smallest factor 2 or 3, a direct sum for other n.
void dft(const cd* in, long s, cd* out, int n, int sign) {
  if (n == 1) {
    out[0] = in[0];
    return;
  }
  const int p = n % 2 == 0 ? 2 : n % 3 == 0 ? 3 : n;
  if (p == n && n > 3) {
    for (int k = 0; k < n; ++k) {
      cd acc = 0.0;
      for (int j = 0; j < n; ++j) {
        const double a = sign * 2.0 * PI * (double)((long long)j * k % n) / n;
        acc += in[j * s] * cd(std::cos(a), std::sin(a));
      }
      out[k] = acc;
    }
    return;
  }
  const int m = n / p;
  std::vector<cd> sub(n);
  for (int r = 0; r < p; ++r) dft(in + r * s, s * p, sub.data() + r * m, m, sign);
  for (int k = 0; k < m; ++k)
    for (int q = 0; q < p; ++q) {
      cd acc = 0.0;
      for (int r = 0; r < p; ++r) {
        const double a = sign * 2.0 * PI * (double)((long long)r * (k + m * q) % n) / n;
        acc += sub[r * m + k] * cd(std::cos(a), std::sin(a));
      }
      out[k + m * q] = acc;
    }
}

// Transform the complex line of n points at base[0], base[stride], ... in place.
void line(cd* base, long stride, int n, int sign, std::vector<cd>& in, std::vector<cd>& out) {
  in.resize(n);
  out.resize(n);
  for (int i = 0; i < n; ++i) in[i] = base[i * stride];
  dft(in.data(), 1, out.data(), n, sign);
  for (int i = 0; i < n; ++i) base[i * stride] = out[i];
}
}  // namespace

struct ref_rfftw_plan {
  int nx, ny, nz, dir;
};

rfftwnd_mpi_plan rfftw3d_mpi_create_plan(MPI_Comm, int nx, int ny, int nz, fftw_direction dir, int) {
  return new ref_rfftw_plan{nx, ny, nz, (int)dir};
}

void rfftwnd_mpi_local_sizes(rfftwnd_mpi_plan p, int* local_nx, int* local_x_start, int* local_ny_after_transpose,
                             int* local_y_start_after_transpose, int* total_local_size) {
  *local_nx = p->nx;
  *local_x_start = 0;
  *local_ny_after_transpose = p->ny;
  *local_y_start_after_transpose = 0;
  *total_local_size = p->nx * p->ny * 2 * (p->nz / 2 + 1);
}

void rfftwnd_mpi_destroy_plan(rfftwnd_mpi_plan p) { delete p; }

// In place on the real array [nx][ny][pad], pad = 2(nz/2+1).  Forward: real
// transform along z (nz/2+1 complex terms), complex along y and x (e^{-i}),
// result stored transposed [ny][nx][nz/2+1].  Inverse: from the transposed
// layout, complex along x and y (e^{+i}), then along z from the half-complex
// terms kz = 0..nz/2 (the imaginary parts at kz = 0 and nz/2 have no place in
// that form and are not read) to nz real values.  Unnormalised both ways.
void rfftwnd_mpi(rfftwnd_mpi_plan p, int n_fields, fftw_real* a, fftw_real*, fftwnd_mpi_output_order) {
  const int nx = p->nx, ny = p->ny, nz = p->nz, nh = nz / 2 + 1;
  const long pad = 2L * nh;
  std::vector<cd> in, out;
  for (int f = 0; f < n_fields; ++f) {
    fftw_real* d = a + (size_t)f * nx * ny * pad;
    cd* c = reinterpret_cast<cd*>(d);  // complex element (row, kz) at c[row * nh + kz]
    std::vector<fftw_real> tmp((size_t)nx * ny * pad);
    if (p->dir == FFTW_REAL_TO_COMPLEX) {
      std::vector<cd> rz(nz), oz(nz);
      for (long row = 0; row < (long)nx * ny; ++row) {
        for (int z = 0; z < nz; ++z) rz[z] = d[row * pad + z];
        dft(rz.data(), 1, oz.data(), nz, -1);
        for (int k = 0; k < nh; ++k) c[row * nh + k] = oz[k];
      }
      for (int x = 0; x < nx; ++x)
        for (int k = 0; k < nh; ++k) line(c + (long)x * ny * nh + k, nh, ny, -1, in, out);
      for (int y = 0; y < ny; ++y)
        for (int k = 0; k < nh; ++k) line(c + (long)y * nh + k, (long)ny * nh, nx, -1, in, out);
      std::memcpy(tmp.data(), d, sizeof(fftw_real) * tmp.size());
      const cd* t = reinterpret_cast<const cd*>(tmp.data());
      for (int x = 0; x < nx; ++x)
        for (int y = 0; y < ny; ++y)
          for (int k = 0; k < nh; ++k) c[((long)y * nx + x) * nh + k] = t[((long)x * ny + y) * nh + k];
    } else {
      std::memcpy(tmp.data(), d, sizeof(fftw_real) * tmp.size());
      const cd* t = reinterpret_cast<const cd*>(tmp.data());
      for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x)
          for (int k = 0; k < nh; ++k) c[((long)x * ny + y) * nh + k] = t[((long)y * nx + x) * nh + k];
      for (int y = 0; y < ny; ++y)
        for (int k = 0; k < nh; ++k) line(c + (long)y * nh + k, (long)ny * nh, nx, +1, in, out);
      for (int x = 0; x < nx; ++x)
        for (int k = 0; k < nh; ++k) line(c + (long)x * ny * nh + k, nh, ny, +1, in, out);
      std::vector<cd> full(nz), oz(nz);
      for (long row = 0; row < (long)nx * ny; ++row) {
        for (int k = 0; k < nh; ++k) full[k] = c[row * nh + k];
        full[0] = cd(full[0].real(), 0.0);
        if (nz % 2 == 0) full[nz / 2] = cd(full[nz / 2].real(), 0.0);
        for (int k = 1; 2 * k < nz; ++k) full[nz - k] = std::conj(full[k]);
        dft(full.data(), 1, oz.data(), nz, +1);
        for (int z = 0; z < nz; ++z) d[row * pad + z] = oz[z].real();
      }
    }
  }
}

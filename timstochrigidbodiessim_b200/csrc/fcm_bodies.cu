// fcm_bodies.cu -- rigid-body kernels: blob positions, K, K^T, the
// block-diagonal preconditioner, rigid projection and body updates.
//
// Body state per body: x[3], q[4] (scalar, vector).  Rotation matrices are
// recomputed from q on every use, as the reference does
// (collection_of_rigid_bodies.cpp:707-757, gmres_solver.cpp:97-134).
#include "fcm_internal.cuh"

namespace fcm {

namespace {

// quaternion.cpp:61-103 with round-to-nearest intrinsics, so the product order
// (and therefore every bit) matches a non-contracting CPU build.
__device__ __forceinline__ void quat_matrix(const double* q, double R[3][3]) {
  const double s = q[0], v0 = q[1], v1 = q[2], v2 = q[3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) R[i][j] = (i == j) ? 1.0 : 0.0;
  double t = __dmul_rn(__dmul_rn(2.0, v0), v0);
  R[1][1] = __dsub_rn(R[1][1], t); R[2][2] = __dsub_rn(R[2][2], t);
  t = __dmul_rn(__dmul_rn(2.0, v1), v1);
  R[0][0] = __dsub_rn(R[0][0], t); R[2][2] = __dsub_rn(R[2][2], t);
  t = __dmul_rn(__dmul_rn(2.0, v2), v2);
  R[0][0] = __dsub_rn(R[0][0], t); R[1][1] = __dsub_rn(R[1][1], t);
  t = __dmul_rn(__dmul_rn(2.0, v0), v1);
  R[1][0] = __dadd_rn(R[1][0], t); R[0][1] = __dadd_rn(R[0][1], t);
  t = __dmul_rn(__dmul_rn(2.0, v0), v2);
  R[2][0] = __dadd_rn(R[2][0], t); R[0][2] = __dadd_rn(R[0][2], t);
  t = __dmul_rn(__dmul_rn(2.0, v1), v2);
  R[1][2] = __dadd_rn(R[1][2], t); R[2][1] = __dadd_rn(R[2][1], t);
  t = __dmul_rn(__dmul_rn(2.0, s), v2);
  R[1][0] = __dadd_rn(R[1][0], t); R[0][1] = __dsub_rn(R[0][1], t);
  t = __dmul_rn(__dmul_rn(2.0, s), v1);
  R[2][0] = __dsub_rn(R[2][0], t); R[0][2] = __dadd_rn(R[0][2], t);
  t = __dmul_rn(__dmul_rn(2.0, s), v0);
  R[2][1] = __dadd_rn(R[2][1], t); R[1][2] = __dsub_rn(R[1][2], t);
}

__device__ __forceinline__ void rot(const double R[3][3], const double* v, double* o) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
    o[i] = __dadd_rn(__dadd_rn(__dmul_rn(R[i][0], v[0]), __dmul_rn(R[i][1], v[1])), __dmul_rn(R[i][2], v[2]));
}
__device__ __forceinline__ void rotT(const double R[3][3], const double* v, double* o) {
#pragma unroll
  for (int i = 0; i < 3; ++i) o[i] = R[0][i] * v[0] + R[1][i] * v[1] + R[2][i] * v[2];
}
__device__ __forceinline__ void cross3(const double* a, const double* b, double* c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

// collection_of_rigid_bodies.cpp:155-193: Y = x + R r_m, wrapped p - L floor(p/L).
// Body n's shape starts at ref + n*rs (rs = 0: one shape shared by all bodies).
__global__ void k_fill_blob_pos(const double* __restrict__ x, const double* __restrict__ q,
                                const double* __restrict__ ref, int rs, int Nb, int nb, double Lx, double Ly,
                                double Lz, double* __restrict__ Y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= Nb) return;
  const int n = i / nb, m = i - n * nb;
  double R[3][3];
  quat_matrix(q + 4 * n, R);
  double r[3];
  rot(R, ref + (size_t)n * rs + 3 * m, r);
  const double L[3] = {Lx, Ly, Lz};
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double p = __dadd_rn(x[3 * n + d], r[d]);
    Y[3 * i + d] = __dsub_rn(p, __dmul_rn(L[d], floor(__ddiv_rn(p, L[d]))));
  }
}

// collection_of_rigid_bodies.cpp:707-731: out_m (+)= U + Omega x (R r_m).
__device__ __forceinline__ void multiply_K_one(const double* __restrict__ q, const double* __restrict__ ref, int rs,
                                               const double* __restrict__ in, double* __restrict__ out, int i,
                                               int nb, int subtract) {
  const int n = i / nb, m = i - n * nb;
  double R[3][3];
  quat_matrix(q + 4 * n, R);
  double r[3], c[3];
  rot(R, ref + (size_t)n * rs + 3 * m, r);
  cross3(in + 6 * n + 3, r, c);
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double v = in[6 * n + d] + c[d];
    out[3 * i + d] = subtract ? out[3 * i + d] - v : v;
  }
}

__global__ void k_multiply_K(const double* __restrict__ q, const double* __restrict__ ref, int rs,
                             const double* __restrict__ in, double* __restrict__ out, int Nb, int nb, int subtract) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= Nb) return;
  multiply_K_one(q, ref, rs, in, out, i, nb, subtract);
}

// collection_of_rigid_bodies.cpp:733-757: F = sum lambda_m, T = sum (R r_m) x lambda_m;
// out = scale * K^T in + add_scale * add.
__device__ __forceinline__ void multiply_KT_one(const double* __restrict__ q, const double* __restrict__ ref, int rs,
                                                const double* __restrict__ in, double* __restrict__ out, int n,
                                                int nb, double scale, const double* __restrict__ add,
                                                double add_scale) {
  double R[3][3];
  quat_matrix(q + 4 * n, R);
  ref += (size_t)n * rs;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int m = 0; m < nb; ++m) {
    const double* l = in + 3 * (n * nb + m);
    double r[3], c[3];
    rot(R, ref + 3 * m, r);
    cross3(r, l, c);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      acc[d] += l[d];
      acc[3 + d] += c[d];
    }
  }
#pragma unroll
  for (int d = 0; d < 6; ++d) out[6 * n + d] = scale * acc[d] + (add ? add_scale * add[6 * n + d] : 0.0);
}

__global__ void k_multiply_KT(const double* __restrict__ q, const double* __restrict__ ref, int rs,
                              const double* __restrict__ in, double* __restrict__ out, int M, int nb, double scale,
                              const double* __restrict__ add, double add_scale) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= M) return;
  multiply_KT_one(q, ref, rs, in, out, n, nb, scale, add, add_scale);
}

// gmres_solver.cpp:85-146, one warp per body, applied in the body frame:
// with B = blockdiag(R) and C = diag(R^T, R^T), the reference's rotated
// matrices are B ref_Minv B^T, K_rot = B K_ref C and C^T ref_N C, so
//   U' = ref_N (-C in_U - K_ref^T ref_Minv B^T in_l),   out_U = C^T U'
//   out_l = B ref_Minv (K_ref U' + B^T in_l).
// Shared memory per warp: 2*(3nb) + 12 doubles.  With per-body shapes body n's
// shape, ref_Minv and ref_N start at ref + n*rs, Minv + n*ms and Nm + n*ns.
// Columns of the per-body matrix-vector products unrolled together (their loads in
// flight at once; the products are latency-bound with one warp per body).
#ifndef FCM_PINV_UNROLL
#define FCM_PINV_UNROLL 6
#endif
constexpr int kPinvUnroll = FCM_PINV_UNROLL;

__device__ __forceinline__ void pinv_block(const double* __restrict__ q, const double* __restrict__ ref, int rs,
                                           const double* __restrict__ Minv, long long ms,
                                           const double* __restrict__ Nm, int ns,
                                           const double* __restrict__ in, double* __restrict__ out, int M, int nb,
                                           int Nb, double* sm) {
  const int warps = blockDim.x >> 5;
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n = blockIdx.x * warps + wid;
  const int n3 = 3 * nb;
  double* xl = sm + (size_t)wid * (2 * n3 + 12);  // body-frame lambda, then K U' + lambda'
  double* t = xl + n3;                           // Minv * lambda'
  double* u = t + n3;                            // 12: in_U' (6), U' (6)
  if (n >= M) return;
  ref += (size_t)n * rs;
  Minv += (size_t)n * ms;
  Nm += (size_t)n * ns;
  double R[3][3];
  quat_matrix(q + 4 * n, R);
  const double* inl = in + (size_t)n3 * n;
  const double* inU = in + (size_t)3 * Nb + 6 * n;
  for (int m = lane; m < nb; m += 32) rotT(R, inl + 3 * m, xl + 3 * m);
  if (lane == 0) {
    rotT(R, inU, u);
    rotT(R, inU + 3, u + 3);
  }
  __syncwarp();
  for (int row = lane; row < n3; row += 32) {
    double s = 0.0;
#pragma unroll kPinvUnroll
    for (int j = 0; j < n3; ++j) s += Minv[(size_t)j * n3 + row] * xl[j];
    t[row] = s;
  }
  __syncwarp();
  if (lane == 0) {
    double kt[6] = {0, 0, 0, 0, 0, 0};
    for (int m = 0; m < nb; ++m) {
      double c[3];
      cross3(ref + 3 * m, t + 3 * m, c);
      for (int d = 0; d < 3; ++d) {
        kt[d] += t[3 * m + d];
        kt[3 + d] += c[d];
      }
    }
    double v[6];
    for (int d = 0; d < 6; ++d) v[d] = -u[d] - kt[d];
    for (int i = 0; i < 6; ++i) {
      double s = 0.0;
      for (int j = 0; j < 6; ++j) s += Nm[j * 6 + i] * v[j];
      u[6 + i] = s;
    }
    double* oU = out + (size_t)3 * Nb + 6 * n;
    rot(R, u + 6, oU);
    rot(R, u + 9, oU + 3);
  }
  __syncwarp();
  for (int m = lane; m < nb; m += 32) {
    double c[3];
    cross3(u + 9, ref + 3 * m, c);
    for (int d = 0; d < 3; ++d) xl[3 * m + d] += u[6 + d] + c[d];
  }
  __syncwarp();
  for (int row = lane; row < n3; row += 32) {
    double s = 0.0;
#pragma unroll kPinvUnroll
    for (int j = 0; j < n3; ++j) s += Minv[(size_t)j * n3 + row] * xl[j];
    t[row] = s;
  }
  __syncwarp();
  double* ol = out + (size_t)n3 * n;
  for (int m = lane; m < nb; m += 32) rot(R, t + 3 * m, ol + 3 * m);
}

__global__ void k_pinv(const double* __restrict__ q, const double* __restrict__ ref, int rs,
                       const double* __restrict__ Minv, long long ms, const double* __restrict__ Nm, int ns,
                       const double* __restrict__ in, double* __restrict__ out, int M, int nb, int Nb) {
  extern __shared__ double sm[];
  pinv_block(q, ref, rs, Minv, ms, Nm, ns, in, out, M, nb, Nb, sm);
}

// Rigid projection of blob velocities with ref_KTKinv
// (collection_of_rigid_bodies.cpp:580-600, :909-939); per-body shapes carry their
// own ref_KTKinv (strides rs, ks).
__global__ void k_rigid_projection(const double* __restrict__ q, const double* __restrict__ ref, int rs,
                                   const double* __restrict__ KTKinv, int ks, const double* __restrict__ V,
                                   double* __restrict__ U, int M, int nb) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= M) return;
  ref += (size_t)n * rs;
  KTKinv += (size_t)n * ks;
  double R[3][3];
  quat_matrix(q + 4 * n, R);
  double b[6] = {0, 0, 0, 0, 0, 0};
  for (int i = 0; i < nb; ++i) {
    const double* vel = V + 3 * (n * nb + i);
    double r[3], c[3];
    rot(R, ref + 3 * i, r);
    cross3(r, vel, c);
    for (int d = 0; d < 3; ++d) {
      b[d] += vel[d];
      b[3 + d] += c[d];
    }
  }
  double bt[6];
  rotT(R, b, bt);
  rotT(R, b + 3, bt + 3);
  double u[6];
  for (int i = 0; i < 6; ++i) {
    double s = 0.0;
    for (int j = 0; j < 6; ++j) s += KTKinv[j * 6 + i] * bt[j];
    u[i] = s;
  }
  rot(R, u, U + 6 * n);
  rot(R, u + 3, U + 6 * n + 3);
}

// particle.cpp:49-58 with quaternion.cpp:128-145 (lie_exp) and quaternion.hpp:55-62.
__device__ void body_update_one(double* x, double* q, const double u[6], double Lx, double Ly, double Lz) {
  x[0] += u[0];
  x[1] += u[1];
  x[2] += u[2];
  const double theta = sqrt(u[3] * u[3] + u[4] * u[4] + u[5] * u[5]);
  double e[4] = {1.0, 0.0, 0.0, 0.0};
  if (!(theta < 1e-10)) {
    double sn, cs;
    sincos(0.5 * theta, &sn, &cs);
    e[0] = cs;
    e[1] = sn * u[3] / theta;
    e[2] = sn * u[4] / theta;
    e[3] = sn * u[5] / theta;
  }
  const double p0 = q[0], p1 = q[1], p2 = q[2], p3 = q[3];
  const double o0 = e[0] * p0 - (e[1] * p1 + e[2] * p2 + e[3] * p3);
  const double cx = e[2] * p3 - e[3] * p2, cy = e[3] * p1 - e[1] * p3, cz = e[1] * p2 - e[2] * p1;
  q[0] = o0;
  q[1] = e[0] * p1 + p0 * e[1] + cx;
  q[2] = e[0] * p2 + p0 * e[2] + cy;
  q[3] = e[0] * p3 + p0 * e[3] + cz;
  const double L[3] = {Lx, Ly, Lz};
  for (int d = 0; d < 3; ++d) x[d] -= L[d] * floor(x[d] / L[d]);
}

__global__ void k_body_update(double* __restrict__ x, double* __restrict__ q, const double* __restrict__ U, int M,
                              double scale, const double* __restrict__ d_nu, double Lx, double Ly, double Lz) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= M) return;
  if (d_nu) scale = __dmul_rn(*d_nu, scale);  // nu * dt with nu from device memory
  double u[6];
  for (int d = 0; d < 6; ++d) u[d] = scale * U[6 * n + d];
  body_update_one(x + 3 * n, q + 4 * n, u, Lx, Ly, Lz);
}

__global__ void k_body_update_uniform(double* __restrict__ x, double* __restrict__ q, int M, double e0, double e1,
                                      double e2, double e3, double e4, double e5, double Lx, double Ly, double Lz) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= M) return;
  const double u[6] = {e0, e1, e2, e3, e4, e5};
  body_update_one(x + 3 * n, q + 4 * n, u, Lx, Ly, Lz);
}

// main.cpp:126-150 and collection_of_rigid_bodies.cpp:759-776: save the body,
// draw the proposal scale (2u - 1) per component (rotations divided by the body
// radius) and apply bodies[n].update(nu DT move) with nu = 1.
__global__ void k_mcmc_propose(double* __restrict__ x, double* __restrict__ q, double* __restrict__ xs,
                               double* __restrict__ qs, int M, const McmcDev* __restrict__ st, double Lx, double Ly,
                               double Lz) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= M) return;
  for (int d = 0; d < 3; ++d) xs[3 * n + d] = x[3 * n + d];
  for (int d = 0; d < 4; ++d) qs[4 * n + d] = q[4 * n + d];
  const uint64_t seed = st->seed, attempt = (uint64_t)st->attempt;
  const double scale = st->scale, dt = st->dt;
  double u[6];
  for (int d = 0; d < 6; ++d) {
    double mv = scale * (2.0 * mcmc_uniform(seed, attempt, (unsigned int)(6 * n + d)) - 1.0);
    if (d >= 3) mv /= st->body_radius;
    u[d] = dt * mv;
  }
  body_update_one(x + 3 * n, q + 4 * n, u, Lx, Ly, Lz);
}

__global__ void k_mcmc_restore(double* __restrict__ x, double* __restrict__ q, const double* __restrict__ xs,
                               const double* __restrict__ qs, int M, const McmcDev* __restrict__ st) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= M || !st->restore) return;
  for (int d = 0; d < 3; ++d) x[3 * n + d] = xs[3 * n + d];
  for (int d = 0; d < 4; ++d) q[4 * n + d] = qs[4 * n + d];
}

// contribution of every body to div(U) for perturbation `comp`
// (collection_of_rigid_bodies.cpp:941-948).
__global__ void k_divU_terms(const double* __restrict__ U, const double* __restrict__ U0, int M, int comp,
                             double delta, double* __restrict__ out) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= M) return;
  out[n] = (U[6 * n + comp] - U0[6 * n + comp]) / delta;
}

}  // namespace

int launch_fill_blob_pos(const Ctx& c, const double* x, const double* q, double* Y, cudaStream_t s) {
  if (c.Nb == 0) return FCM_OK;
  k_fill_blob_pos<<<(c.Nb + 127) / 128, 128, 0, s>>>(x, q, c.d_ref, c.ref_stride, c.Nb, c.nb, c.g.Lx, c.g.Ly, c.g.Lz, Y);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

int launch_multiply_K(const Ctx& c, const double* qm, const double* in6, double* out3, double subtract,
                      cudaStream_t s) {
  if (c.Nb == 0) return FCM_OK;
  k_multiply_K<<<(c.Nb + 127) / 128, 128, 0, s>>>(qm, c.d_ref, c.ref_stride, in6, out3, c.Nb, c.nb, subtract != 0.0 ? 1 : 0);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

int launch_multiply_KT(const Ctx& c, const double* qm, const double* in3, double* out6, double scale,
                       const double* add6, double add_scale, cudaStream_t s) {
  if (c.M == 0) return FCM_OK;
  k_multiply_KT<<<(c.M + 127) / 128, 128, 0, s>>>(qm, c.d_ref, c.ref_stride, in3, out6, c.M, c.nb, scale, add6, add_scale);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

int launch_pinv(const Ctx& c, const double* qm, const double* in, double* out, cudaStream_t s) {
  if (c.M == 0) return FCM_OK;
  const int warps = 4;
  const size_t shm = sizeof(double) * warps * (size_t)(6 * c.nb + 12);
  k_pinv<<<(c.M + warps - 1) / warps, 32 * warps, shm, s>>>(qm, c.d_ref, c.ref_stride, c.d_Minv, c.minv_stride, c.d_N,
                                                                 c.n_stride, in, out, c.M, c.nb, c.Nb);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

int launch_rigid_projection(const Ctx& c, const double* q, const double* V, double* U6, cudaStream_t s) {
  if (c.M == 0) return FCM_OK;
  k_rigid_projection<<<(c.M + 127) / 128, 128, 0, s>>>(q, c.d_ref, c.ref_stride, c.d_KTKinv, c.n_stride, V, U6,
                                                       c.M, c.nb);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

int launch_body_update(const Ctx& c, double* x, double* q, const double* U6, double scale, cudaStream_t s,
                       const double* d_nu) {
  if (c.M == 0) return FCM_OK;
  k_body_update<<<(c.M + 127) / 128, 128, 0, s>>>(x, q, U6, c.M, scale, d_nu, c.g.Lx, c.g.Ly, c.g.Lz);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

int launch_mcmc_propose(const Ctx& c, const McmcDev* st, cudaStream_t s) {
  if (c.M == 0) return FCM_OK;
  k_mcmc_propose<<<(c.M + 127) / 128, 128, 0, s>>>(c.d_x, c.d_q, c.d_xs, c.d_qs, c.M, st, c.g.Lx, c.g.Ly, c.g.Lz);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

int launch_mcmc_restore(const Ctx& c, const McmcDev* st, cudaStream_t s) {
  if (c.M == 0) return FCM_OK;
  k_mcmc_restore<<<(c.M + 127) / 128, 128, 0, s>>>(c.d_x, c.d_q, c.d_xs, c.d_qs, c.M, st);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

int launch_body_update_uniform(const Ctx& c, double* x, double* q, const double* e6, cudaStream_t s) {
  if (c.M == 0) return FCM_OK;
  k_body_update_uniform<<<(c.M + 127) / 128, 128, 0, s>>>(x, q, c.M, e6[0], e6[1], e6[2], e6[3], e6[4], e6[5],
                                                          c.g.Lx, c.g.Ly, c.g.Lz);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

int launch_divU_accumulate(const Ctx& c, const double* U6, const double* U0, int component, double delta,
                           double* acc, cudaStream_t s) {
  if (c.M == 0) return FCM_OK;
  k_divU_terms<<<(c.M + 127) / 128, 128, 0, s>>>(U6, U0, c.M, component, delta, acc);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

}  // namespace fcm

// ============================================================ batched
namespace fcm {
namespace {

__global__ void k_b_pinv(const BMember* __restrict__ mem, int in, int out, int mask) {
  extern __shared__ double sm[];
  const BMember& m = mem[blockIdx.y];
  if (bskip(m, mask)) return;
  pinv_block(m.qm, m.ref, m.ref_stride, m.Minv, m.minv_stride, m.N, m.n_stride, bvec(m, in), bvec(m, out), m.M,
             m.nb, m.Nb, sm);
}

// out[lambda] -= K in[U] (blocks [0, blob_blocks)) and out[U] = -K^T in[lambda]
// (the rest): the rigid-body part of the saddle-point product.
__global__ void k_b_K_KT(const BMember* __restrict__ mem, int in, int out, int blob_blocks, int mask) {
  const BMember& m = mem[blockIdx.y];
  if (bskip(m, mask)) return;
  const double* x = bvec(m, in);
  double* y = bvec(m, out);
  if ((int)blockIdx.x < blob_blocks) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m.Nb) multiply_K_one(m.qm, m.ref, m.ref_stride, x + 3 * (size_t)m.Nb, y, i, m.nb, 1);
  } else {
    const int n = (blockIdx.x - blob_blocks) * blockDim.x + threadIdx.x;
    if (n < m.M) multiply_KT_one(m.qm, m.ref, m.ref_stride, x, y + 3 * (size_t)m.Nb, n, m.nb, -1.0, nullptr, 0.0);
  }
}

}  // namespace

int b_pinv(const BatchGeom& b, int in, int out, int mask, cudaStream_t s) {
  const int warps = 4;
  const size_t shm = sizeof(double) * warps * (size_t)(6 * b.max_nb + 12);
  k_b_pinv<<<dim3(b.max_pinv_blocks, b.n), 32 * warps, shm, s>>>(b.mem, in, out, mask);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

int b_multiply_K_KT(const BatchGeom& b, int in, int out, int mask, cudaStream_t s) {
  k_b_K_KT<<<dim3(b.max_blob_blocks + b.max_body_blocks, b.n), 128, 0, s>>>(b.mem, in, out, b.max_blob_blocks, mask);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

}  // namespace fcm

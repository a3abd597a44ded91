// Polarised sky: frame rotation of the source coherency.
//
// Reference: calc_coherency_rotation and its helpers (coordinates.py:288-580)
// and CoordinateRotation._rotate_frame_coherency (core/coords.py:152-175).  Per
// above-horizon source, in FP64:
//   frame = unit vector of (ra, dec); altaz = unit vector of (az, alt) in the
//   alt/az cartesian frame (x north, y east, z up), az / alt from the topocentric
//   (E, N, U) vector as enu_to_az_za(orientation="astropy") gives them;
//   R_exact = R_perturb . R_avg, where R_avg is the frame's rigid ICRS -> alt/az
//   rotation and R_perturb (Rodrigues) carries R_avg . frame onto altaz
//   (identity when the two coincide exactly: the reference divides 0 by 0 there);
//   bh = R_exact^T theta_hat(za, az); cos X = bh . theta_hat(pi/2 - dec, ra),
//   sin X = bh . phi_hat(pi/2 - dec, ra);  R = [[cos X, sin X], [-sin X, cos X]].
// The rotated coherency is C' = R^T C R.
#include "common.cuh"

namespace mvb {

struct Mat3 {
  double m[9];
};

__device__ __forceinline__ void coherency_rotation_one(double ra, double dec, double e, double n, const Mat3 &ravg,
                                                       double &cos_x, double &sin_x) {
  const double kPi = 3.141592653589793;
  // enu_to_az_za, astropy orientation, periodic azimuth (coordinates.py:31-88)
  const double lsqr = n * n + e * e;
  const double zeta = lsqr < 1.0 ? sqrt(1.0 - lsqr) : 0.0;
  double az = atan2(e, n);
  az = az - 2.0 * kPi * floor(az / (2.0 * kPi));
  const double za = 0.5 * kPi - asin(zeta);
  const double alt = 0.5 * kPi - za;
  // unit vectors
  const double cd = cos(dec), sd = sin(dec), cr = cos(ra), sr = sin(ra);
  const double frame[3] = {cd * cr, cd * sr, sd};
  const double ca = cos(alt), sa = sin(alt), caz = cos(az), saz = sin(az);
  const double altaz[3] = {ca * caz, ca * saz, sa};
  double r1[3];
  for (int i = 0; i < 3; ++i) r1[i] = ravg.m[3 * i] * frame[0] + ravg.m[3 * i + 1] * frame[1] + ravg.m[3 * i + 2] * frame[2];
  // vecs2rot (coordinates.py:387-411)
  const double ax[3] = {r1[1] * altaz[2] - r1[2] * altaz[1], r1[2] * altaz[0] - r1[0] * altaz[2],
                        r1[0] * altaz[1] - r1[1] * altaz[0]};
  const double sin_psi = sqrt(ax[0] * ax[0] + ax[1] * ax[1] + ax[2] * ax[2]);
  const double cos_psi = r1[0] * altaz[0] + r1[1] * altaz[1] + r1[2] * altaz[2];
  const double psi = atan2(sin_psi, cos_psi);
  double u[3] = {0.0, 0.0, 0.0};
  if (sin_psi > 0.0)
    for (int i = 0; i < 3; ++i) u[i] = ax[i] / sin_psi;
  // axis_angle_rotation_matrix (coordinates.py:414-452): I + sin K + (1 - cos) K^2
  const double K[9] = {0.0, -u[2], u[1], u[2], 0.0, -u[0], -u[1], u[0], 0.0};
  const double sp = sin(psi), omc = 1.0 - cos(psi);
  double P[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double k2 = 0.0;
      for (int l = 0; l < 3; ++l) k2 += K[3 * i + l] * K[3 * l + j];
      P[3 * i + j] = (i == j ? 1.0 : 0.0) + sp * K[3 * i + j] + omc * k2;
    }
  double E[9];  // R_exact = R_perturb . R_avg
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      E[3 * i + j] = P[3 * i] * ravg.m[j] + P[3 * i + 1] * ravg.m[3 + j] + P[3 * i + 2] * ravg.m[6 + j];
  // spherical_basis_vector_rotation_matrix (coordinates.py:455-490)
  const double theta = 0.5 * kPi - dec, ct = cos(theta), st = sin(theta);
  const double th[3] = {cr * ct, sr * ct, -st};
  const double ph[3] = {-sr, cr, 0.0};
  const double beta = 0.5 * kPi - alt, cb = cos(beta), sb = sin(beta);
  const double tb[3] = {caz * cb, saz * cb, -sb};
  double bh[3];
  for (int a = 0; a < 3; ++a) bh[a] = E[a] * tb[0] + E[3 + a] * tb[1] + E[6 + a] * tb[2];
  cos_x = bh[0] * th[0] + bh[1] * th[1] + bh[2] * th[2];
  sin_x = bh[0] * ph[0] + bh[1] * ph[1] + bh[2] * ph[2];
}

// One thread per compacted source slot s < n: rot[s] = (cos X, sin X).
__global__ void coherency_rotation_kernel(const double *__restrict__ radec, int64_t N, const int32_t *__restrict__ kept,
                                          const double *__restrict__ crd, int64_t ld, const int32_t *__restrict__ n_dev,
                                          int64_t cap, Mat3 ravg, double2 *__restrict__ rot) {
  const int64_t n = n_dev ? min((int64_t)*n_dev, cap) : cap;
  for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < n; s += (int64_t)gridDim.x * blockDim.x) {
    const int64_t src = kept ? kept[s] : s;
    if (src < 0 || src >= N) continue;
    double c, sn;
    coherency_rotation_one(radec[src], radec[N + src], crd[s], crd[ld + s], ravg, c, sn);
    rot[s] = make_double2(c, sn);
  }
}

// C' = R^T C R for every compacted source and frequency; C is the caller's
// (N, Nf, 2, 2) complex128 coherency, out is (cap, Nf, 2, 2) complex128 with
// slots >= n zeroed (core/coords.py:128-147).
__global__ void rotate_coherency_kernel(const double2 *__restrict__ rot, const int32_t *__restrict__ kept,
                                        const int32_t *__restrict__ n_dev, const double2 *__restrict__ coh, int64_t N,
                                        int nf, double2 *__restrict__ out, int64_t cap) {
  const int64_t n = n_dev ? min((int64_t)*n_dev, cap) : cap;
  const int64_t total = cap * nf;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s = e / nf;
    double2 *o = out + 4 * e;
    if (s >= n) {
      for (int k = 0; k < 4; ++k) o[k] = make_double2(0.0, 0.0);
      continue;
    }
    const int64_t src = kept ? kept[s] : s;
    const double2 *c = coh + 4 * (src * nf + (e % nf));
    const double cx = rot[s].x, sx = rot[s].y;
    // R = [[cx, sx], [-sx, cx]];  C'_{ad} = sum_{bc} R_{ba} C_{bc} R_{cd}
    const double R[2][2] = {{cx, sx}, {-sx, cx}};
    for (int a = 0; a < 2; ++a)
      for (int d = 0; d < 2; ++d) {
        double re = 0.0, im = 0.0;
        for (int b = 0; b < 2; ++b)
          for (int cc = 0; cc < 2; ++cc) {
            const double w = R[b][a] * R[cc][d];
            re += w * c[2 * b + cc].x;
            im += w * c[2 * b + cc].y;
          }
        o[2 * a + d] = make_double2(re, im);
      }
  }
}

}  // namespace mvb

using namespace mvb;

extern "C" int mvb_coherency_rotation(const double *radec, int64_t N, const int32_t *kept, const double *crd,
                                      int64_t ld, const int32_t *n_dev, int64_t cap, const double *r_avg,
                                      double *rot, void *stream) {
  if (N < 0 || cap < 0 || !r_avg || ld < cap || (cap > 0 && (!radec || !crd || !rot)))
    return fail(MVB_ERR_ARG, "mvb_coherency_rotation: bad arguments");
  if (cap == 0) return MVB_OK;
  Mat3 m;
  for (int k = 0; k < 9; ++k) m.m[k] = r_avg[k];
  const int threads = 128;
  const int64_t blocks = std::min<int64_t>(ceil_div(cap, threads), (int64_t)num_sms() * 8);
  coherency_rotation_kernel<<<(unsigned)blocks, threads, 0, as_stream(stream)>>>(
      radec, N, kept, crd, ld, n_dev, cap, m, reinterpret_cast<double2 *>(rot));
  return check_launch("coherency_rotation_kernel");
}

extern "C" int mvb_rotate_coherency(const double *rot, const int32_t *kept, const int32_t *n_dev, const void *coh,
                                    int64_t N, int nf, void *out, int64_t cap, void *stream) {
  if (N < 0 || cap < 0 || nf <= 0 || (cap > 0 && (!rot || !coh || !out)))
    return fail(MVB_ERR_ARG, "mvb_rotate_coherency: bad arguments");
  if (cap == 0) return MVB_OK;
  const int threads = 256;
  const int64_t blocks = std::min<int64_t>(ceil_div(cap * nf, threads), (int64_t)num_sms() * 8);
  rotate_coherency_kernel<<<(unsigned)blocks, threads, 0, as_stream(stream)>>>(
      reinterpret_cast<const double2 *>(rot), kept, n_dev, static_cast<const double2 *>(coh), N, nf,
      static_cast<double2 *>(out), cap);
  return check_launch("rotate_coherency_kernel");
}

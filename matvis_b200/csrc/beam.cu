// A5: beam interpolation at the above-horizon sources.
//
// Reference: gpu/beams.py:127-200 (gpu_beam_interpolation: order-1
// map_coordinates per (beam, feed, axis) at row = za / dza, col = (az - azmin) /
// daz, sqrt after interpolating a power beam), gpu/beams.py:103-124 and
// coordinates.py:31-88 (enu_to_az_za with orientation="uvbeam").
//
// Edge rule (scipy / cupyx map_coordinates, mode='constant', order=1): a point
// whose row or column coordinate lies outside [0, n-1] gives 0; inside, the
// 2x2 neighbours are blended with FP64 weights (a neighbour index of n carries
// weight 0).
//
// Layout: grids (nbeam, nax, nfeed, nza, naz), complex64 or float32 power;
// output (nbeam, nfeed, nax, nout) complex.  One CTA stages ONE real plane
// (a component of one (beam, ax, feed) grid, <= 200 KB) in shared memory and
// interpolates it for a slice of the sources.  With a workspace, a first kernel
// computes each source's FP64 (az, za) and its grid coordinates for every beam
// once; without one, every plane's CTA recomputes them.  Planes larger than the
// shared memory budget are read through L2 instead.
#include <math_constants.h>

#include "common.cuh"

namespace mvb {

constexpr int kBeamThreads = 256;
constexpr size_t kBeamSmemMax = 200 * 1024;

struct BeamParams {
  double daz, dza, azmin;
};

// numpy.mod(a, b) for b > 0: result in [0, b).
__device__ __forceinline__ double py_mod(double a, double b) {
  double m = fmod(a, b);
  if (m != 0.0 && m < 0.0) m += b;
  return m;
}

// enu_to_az_za(orientation="uvbeam", periodic_azimuth=True), FP64.
__device__ __forceinline__ void az_za_uvbeam(double e, double n, double &az, double &za) {
  const double lsqr = n * n + e * e;
  const double zeta = lsqr < 1.0 ? sqrt(1.0 - lsqr) : 0.0;
  const double a = atan2(e, n);
  za = 0.5 * CUDART_PI - asin(zeta);
  az = py_mod(0.5 * CUDART_PI - a, 2.0 * CUDART_PI);
}

// Bilinear (order-1, mode='constant') sample of a real plane `p` (nza x naz,
// row-major, element stride `es` floats).
template <typename Load>
__device__ __forceinline__ double bilinear(Load p, int nza, int naz, double row, double col) {
  if (!(row >= 0.0 && row <= (double)(nza - 1) && col >= 0.0 && col <= (double)(naz - 1))) return 0.0;
  const int r0 = min((int)floor(row), nza - 1);
  const int c0 = min((int)floor(col), naz - 1);
  const double fr = row - r0, fc = col - c0;
  const int r1 = min(r0 + 1, nza - 1), c1 = min(c0 + 1, naz - 1);
  const double v00 = p(r0, c0), v01 = p(r0, c1), v10 = p(r1, c0), v11 = p(r1, c1);
  return (1.0 - fr) * ((1.0 - fc) * v00 + fc * v01) + fr * ((1.0 - fc) * v10 + fc * v11);
}

// Grid coordinates of every source for every beam, once per call:
// rc[(2 b) nout + i] = za / dza_b, rc[(2 b + 1) nout + i] = (az - azmin_b) / daz_b
// (the plane kernel's own FP64 expressions), and row -1 (outside every grid:
// a zero) for the slots i >= n.  One thread per source.
__global__ void beam_rowcol_kernel(const BeamParams *__restrict__ params, int nbeam, const double *__restrict__ crd,
                                   int64_t ld, const int32_t *__restrict__ n_dev, int64_t nsrc, int64_t nout,
                                   double *__restrict__ rc) {
  const int64_t n = n_dev ? min((int64_t)*n_dev, nsrc) : nsrc;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nout; i += (int64_t)gridDim.x * blockDim.x) {
    double az = 0.0, za = 0.0;
    if (i < n) az_za_uvbeam(crd[i], crd[ld + i], az, za);
    for (int b = 0; b < nbeam; ++b) {
      const BeamParams bp = params[b];
      rc[(2 * b) * nout + i] = i < n ? za / bp.dza : -1.0;
      rc[(2 * b + 1) * nout + i] = i < n ? (az - bp.azmin) / bp.daz : -1.0;
    }
  }
}

// grid_kind 0: complex64 (ncomp = 2), 1: float32 power (ncomp = 1).
// plane q = ((b * nax + ax) * nfeed + fd) * ncomp + comp.
// kCoord 0: crd holds ENU (e, n) rows, az/za computed here per plane;
// 1: crd holds (az, za) rows; 2: crd holds beam_rowcol_kernel's grid
// coordinates (leading dimension nout), so no per-plane trigonometry.
template <bool kStaged, int kCoord = 0>
__global__ void __launch_bounds__(kBeamThreads)
    beam_plane_kernel(const float *__restrict__ grids, int grid_kind, int nbeam, int nax, int nfeed, int nza, int naz,
                      const BeamParams *__restrict__ params, const double *__restrict__ crd, int64_t ld,
                      const int32_t *__restrict__ n_dev, int64_t nsrc, void *__restrict__ out, int out_c128,
                      int64_t nout, int32_t *__restrict__ status) {
  extern __shared__ float plane_smem[];
  const int ncomp = grid_kind == 0 ? 2 : 1;
  const int q = blockIdx.x;
  const int comp = q % ncomp;
  const int gidx = q / ncomp;  // (b, ax, fd) flattened
  const int fd = gidx % nfeed;
  const int ax = (gidx / nfeed) % nax;
  const int b = gidx / (nfeed * nax);
  const int64_t plane_elems = (int64_t)nza * naz;
  const float *src = grids + (int64_t)gidx * plane_elems * ncomp + comp;

  if (kStaged) {
    for (int64_t i = threadIdx.x; i < plane_elems; i += kBeamThreads) plane_smem[i] = src[i * ncomp];
    __syncthreads();
  }
  const int64_t n = n_dev ? min((int64_t)*n_dev, nsrc) : nsrc;
  const BeamParams bp = params[b];
  const int64_t out_row = (((int64_t)b * nfeed + fd) * nax + ax) * nout;  // (b, fd, ax, :)

  for (int64_t i = blockIdx.y * (int64_t)kBeamThreads + threadIdx.x; i < nout; i += (int64_t)gridDim.y * kBeamThreads) {
    double v = 0.0;
    if (i < n) {
      double row, col;
      if constexpr (kCoord == 2) {
        row = crd[(2 * b) * nout + i];
        col = crd[(2 * b + 1) * nout + i];
      } else {
        double az, za;
        if constexpr (kCoord == 1) {
          az = crd[i];
          za = crd[ld + i];
        } else {
          az_za_uvbeam(crd[i], crd[ld + i], az, za);
        }
        row = za / bp.dza;
        col = (az - bp.azmin) / bp.daz;
      }
      if (kStaged)
        v = bilinear([&](int r, int c) { return (double)plane_smem[(int64_t)r * naz + c]; }, nza, naz, row, col);
      else
        v = bilinear([&](int r, int c) { return (double)__ldg(src + ((int64_t)r * naz + c) * ncomp); }, nza, naz,
                     row, col);
      if (grid_kind == 1) v = sqrt(v);
      if (status && !isfinite(v)) atomicOr(status, MVB_DEV_NONFINITE);
    }
    if (out_c128) {
      double *o = static_cast<double *>(out) + 2 * (out_row + i);
      o[comp] = v;
      if (ncomp == 1) o[1] = 0.0;
    } else {
      float *o = static_cast<float *>(out) + 2 * (out_row + i);
      o[comp] = (float)v;
      if (ncomp == 1) o[1] = 0.0f;
    }
  }
}

__global__ void beam_gaussian_kernel(const double *__restrict__ sigmas, int nbeam, const double *__restrict__ crd,
                                     int64_t ld, const int32_t *__restrict__ n_dev, int64_t nsrc, void *__restrict__ out,
                                     int out_c128, int64_t nout) {
  const int64_t n = n_dev ? min((int64_t)*n_dev, nsrc) : nsrc;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nout; i += (int64_t)gridDim.x * blockDim.x) {
    double za = 0.0;
    if (i < n) {
      double az;
      az_za_uvbeam(crd[i], crd[ld + i], az, za);
    }
    for (int b = 0; b < nbeam; ++b) {
      const double s = sigmas[b];
      // sqrt of the power exp(-za^2 / s^2)
      const double v = i < n ? exp(-(za * za) / (2.0 * s * s)) : 0.0;
      if (out_c128) {
        double *o = static_cast<double *>(out) + 2 * ((int64_t)b * nout + i);
        o[0] = v;
        o[1] = 0.0;
      } else {
        float *o = static_cast<float *>(out) + 2 * ((int64_t)b * nout + i);
        o[0] = (float)v;
        o[1] = 0.0f;
      }
    }
  }
}

}  // namespace mvb

using namespace mvb;

static int beam_interp_impl(bool azza, const void *grids, int grid_kind, int nbeam, int nax, int nfeed, int nza,
                            int naz, const double *params, const double *crd, int64_t ld, const int32_t *n_dev,
                            int64_t nsrc, void *out, int out_c128, int64_t nout, int32_t *status, void *ws,
                            size_t ws_bytes, void *stream) {
  const char *who = azza ? "mvb_beam_interp_azza" : "mvb_beam_interp";
  if (!grids || !params || !out || (nsrc > 0 && !crd) || nbeam <= 0 || nax <= 0 || nfeed <= 0 || nza < 1 || naz < 1 ||
      (grid_kind != 0 && grid_kind != 1) || nout < nsrc || nsrc < 0)
    return fail(MVB_ERR_ARG, "%s: bad arguments", who);
  if (ws && (ws_bytes < (size_t)2 * nbeam * nout * sizeof(double) || reinterpret_cast<uintptr_t>(ws) % 8))
    return fail(MVB_ERR_ARG, "%s: workspace too small", who);
  if (nout == 0) return MVB_OK;
  const int ncomp = grid_kind == 0 ? 2 : 1;
  const int nplanes = nbeam * nax * nfeed * ncomp;
  const size_t plane_bytes = (size_t)nza * naz * sizeof(float);
  const int nsm = num_sms();
  const int64_t ychunks = std::max<int64_t>(1, std::min<int64_t>(ceil_div(nout, kBeamThreads),
                                                                  ceil_div((int64_t)nsm * 2, nplanes)));
  dim3 grid(nplanes, (unsigned)ychunks);
  cudaStream_t s = as_stream(stream);
  const BeamParams *bp = reinterpret_cast<const BeamParams *>(params);
  const float *g = static_cast<const float *>(grids);
  // with a workspace, the grid coordinates of each source are computed once for
  // all planes (the ENU form only)
  const bool pre = ws && !azza;
  const double *coords = crd;
  if (pre) {
    const int64_t blocks = std::min<int64_t>(ceil_div(nout, kBeamThreads), (int64_t)nsm * 8);
    beam_rowcol_kernel<<<(unsigned)blocks, kBeamThreads, 0, s>>>(bp, nbeam, crd, ld, n_dev, nsrc, nout,
                                                                 static_cast<double *>(ws));
    int rc = check_launch("beam_rowcol_kernel");
    if (rc) return rc;
    coords = static_cast<const double *>(ws);
  }
#define MVB_BEAM(ST, CO, SM)                                                                                        \
  beam_plane_kernel<ST, CO><<<grid, kBeamThreads, SM, s>>>(g, grid_kind, nbeam, nax, nfeed, nza, naz, bp, coords, ld, \
                                                           n_dev, nsrc, out, out_c128, nout, status)
  const int co = pre ? 2 : (azza ? 1 : 0);
  if (plane_bytes <= kBeamSmemMax) {
    const void *fn = co == 2 ? reinterpret_cast<const void *>(beam_plane_kernel<true, 2>)
                             : (co == 1 ? reinterpret_cast<const void *>(beam_plane_kernel<true, 1>)
                                        : reinterpret_cast<const void *>(beam_plane_kernel<true, 0>));
    int rc = set_smem_once(fn, (int)kBeamSmemMax, 10 + co);
    if (rc) return rc;
    if (co == 2)
      MVB_BEAM(true, 2, plane_bytes);
    else if (co == 1)
      MVB_BEAM(true, 1, plane_bytes);
    else
      MVB_BEAM(true, 0, plane_bytes);
  } else {
    if (co == 2)
      MVB_BEAM(false, 2, 0);
    else if (co == 1)
      MVB_BEAM(false, 1, 0);
    else
      MVB_BEAM(false, 0, 0);
  }
#undef MVB_BEAM
  return check_launch("beam_plane_kernel");
}

extern "C" size_t mvb_beam_interp_ws_bytes(int nbeam, int64_t nout) {
  if (nbeam <= 0 || nout <= 0) return 8;
  return (size_t)2 * nbeam * nout * sizeof(double);
}

extern "C" int mvb_beam_interp(const void *grids, int grid_kind, int nbeam, int nax, int nfeed, int nza, int naz,
                               const double *params, const double *crd, int64_t ld, const int32_t *n_dev, int64_t nsrc,
                               void *out, int out_c128, int64_t nout, int32_t *status, void *ws, size_t ws_bytes,
                               void *stream) {
  return beam_interp_impl(false, grids, grid_kind, nbeam, nax, nfeed, nza, naz, params, crd, ld, n_dev, nsrc, out,
                          out_c128, nout, status, ws, ws_bytes, stream);
}

extern "C" int mvb_beam_interp_azza(const void *grids, int grid_kind, int nbeam, int nax, int nfeed, int nza, int naz,
                                    const double *params, const double *azza, int64_t ld, int64_t nsrc, void *out,
                                    int out_c128, void *stream) {
  return beam_interp_impl(true, grids, grid_kind, nbeam, nax, nfeed, nza, naz, params, azza, ld, nullptr, nsrc, out,
                          out_c128, nsrc, nullptr, nullptr, 0, stream);
}

extern "C" int mvb_beam_gaussian(const double *sigmas, int nbeam, const double *crd, int64_t ld, const int32_t *n_dev,
                                 int64_t nsrc, void *out, int out_c128, int64_t nout, void *stream) {
  if (!sigmas || !out || nbeam <= 0 || nsrc < 0 || nout < nsrc || (nsrc > 0 && !crd))
    return fail(MVB_ERR_ARG, "mvb_beam_gaussian: bad arguments");
  if (nout == 0) return MVB_OK;
  const int threads = 256;
  const int64_t blocks = std::min<int64_t>(ceil_div(nout, threads), (int64_t)num_sms() * 8);
  beam_gaussian_kernel<<<(unsigned)blocks, threads, 0, as_stream(stream)>>>(sigmas, nbeam, crd, ld, n_dev, nsrc, out,
                                                                            out_c128, nout);
  return check_launch("beam_gaussian_kernel");
}

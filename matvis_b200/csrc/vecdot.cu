// A8: per-pair source sums for an explicit antenna-pair list.
//
// Reference: gpu/matprod.py:66-98 (GPUVectorDot: one cuBLAS complex_matmul per
// pair per time and chunk), cpu/matprod.py:35-53 (CPUVectorDot:
// out[i] = z[aj] . z[ai]^H, i.e. out[i, p, q] = sum_k Z[aj*F+p, k] conj(Z[ai*F+q, k])).
//
// One warp per (k-slice, pair), pairs fastest so concurrently running warps
// read the same Z columns from L2.  Lanes stride over k with FP32 FMA partial
// sums (coalesced 256-byte row reads), the warp reduces in FP64 and the slices
// are summed in FP64 in a fixed order by the second kernel.
#include "common.cuh"

namespace mvb {

__device__ __forceinline__ int64_t vd_valid_k(const int32_t *n_dev, int64_t n_host, int kmul, int64_t Kcap) {
  int64_t n = n_dev ? (int64_t)*n_dev : n_host;
  n = n < 0 ? 0 : n;
  return min(n * kmul, Kcap);
}

template <int F>
__global__ void __launch_bounds__(256)
    vecdot_kernel(const float2 *__restrict__ z, int64_t Kcap, const int32_t *__restrict__ n_dev, int64_t n_host,
                  int kmul, const int32_t *__restrict__ pairs, int64_t npairs, int k_chunk,
                  double *__restrict__ part) {
  const int lane = threadIdx.x & 31;
  const int64_t kvalid = vd_valid_k(n_dev, n_host, kmul, Kcap);
  const int64_t nsplit = (kvalid + k_chunk - 1) / k_chunk;
  const int64_t total = nsplit * npairs;
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t u = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); u < total; u += nwarps) {
    const int64_t s = u / npairs, pr = u % npairs;
    const int ai = pairs[2 * pr], aj = pairs[2 * pr + 1];
    const int64_t k0 = s * k_chunk, k1 = min(k0 + k_chunk, kvalid);
    float are[F][F], aim[F][F];
#pragma unroll
    for (int p = 0; p < F; ++p)
#pragma unroll
      for (int q = 0; q < F; ++q) are[p][q] = aim[p][q] = 0.f;
    const float2 *zi = z + (int64_t)ai * F * Kcap;
    const float2 *zj = z + (int64_t)aj * F * Kcap;
    for (int64_t k = k0 + lane; k < k1; k += 32) {
      float2 vj[F], vi[F];
#pragma unroll
      for (int p = 0; p < F; ++p) vj[p] = zj[p * Kcap + k];
#pragma unroll
      for (int q = 0; q < F; ++q) vi[q] = zi[q * Kcap + k];
#pragma unroll
      for (int p = 0; p < F; ++p)
#pragma unroll
        for (int q = 0; q < F; ++q) {
          are[p][q] = fmaf(vj[p].x, vi[q].x, fmaf(vj[p].y, vi[q].y, are[p][q]));
          aim[p][q] = fmaf(vj[p].y, vi[q].x, fmaf(-vj[p].x, vi[q].y, aim[p][q]));
        }
    }
#pragma unroll
    for (int p = 0; p < F; ++p)
#pragma unroll
      for (int q = 0; q < F; ++q) {
        double r = are[p][q], i = aim[p][q];
        for (int o = 16; o > 0; o >>= 1) {
          r += __shfl_xor_sync(0xffffffffu, r, o);
          i += __shfl_xor_sync(0xffffffffu, i, o);
        }
        if (lane == 0) {
          part[(u * F * F + p * F + q) * 2] = r;
          part[(u * F * F + p * F + q) * 2 + 1] = (ai == aj && p == q) ? 0.0 : i;  // one-feed autos are real
        }
      }
  }
}

template <typename OT>
__global__ void vecdot_reduce_kernel(const double *__restrict__ part, int64_t Kcap, const int32_t *__restrict__ n_dev,
                                     int64_t n_host, int kmul, int F, int64_t npairs, int k_chunk,
                                     void *__restrict__ out, int accumulate) {
  const int64_t kvalid = vd_valid_k(n_dev, n_host, kmul, Kcap);
  const int64_t nsplit = (kvalid + k_chunk - 1) / k_chunk;
  const int64_t per = npairs * F * F;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < per; e += (int64_t)gridDim.x * blockDim.x) {
    double r = 0, i = 0;
    for (int64_t s = 0; s < nsplit; ++s) {
      r += part[(s * per + e) * 2];
      i += part[(s * per + e) * 2 + 1];
    }
    OT *o = static_cast<OT *>(out) + e;
    if (accumulate) {
      o->x += r;
      o->y += i;
    } else {
      o->x = r;
      o->y = i;
    }
  }
}

}  // namespace mvb

using namespace mvb;

extern "C" size_t mvb_vecdot_ws_bytes(int64_t npairs, int nfeed, int64_t Kcap, int k_chunk) {
  if (npairs <= 0 || k_chunk <= 0 || Kcap <= 0) return 8;
  return (size_t)ceil_div(Kcap, k_chunk) * npairs * nfeed * nfeed * 2 * sizeof(double);
}

extern "C" int mvb_vecdot(const void *z, int64_t Kcap, const int32_t *n_dev, int64_t n_host, int kmul, int nfeed,
                          const int32_t *pairs, int64_t npairs, int k_chunk, void *ws, size_t ws_bytes, void *out,
                          int out_c128, int accumulate, void *stream) {
  if (!z || !ws || !out || Kcap <= 0 || (nfeed != 1 && nfeed != 2) || npairs < 0 || (npairs > 0 && !pairs) ||
      k_chunk <= 0 || kmul <= 0 || n_host < 0 || (!n_dev && n_host * kmul > Kcap))
    return fail(MVB_ERR_ARG, "mvb_vecdot: bad arguments");
  if (ws_bytes < mvb_vecdot_ws_bytes(npairs, nfeed, Kcap, k_chunk))
    return fail(MVB_ERR_ARG, "mvb_vecdot: workspace too small");
  if (npairs == 0) return MVB_OK;
  cudaStream_t s = as_stream(stream);
  double *part = static_cast<double *>(ws);
  const int64_t max_units = ceil_div(Kcap, k_chunk) * npairs;
  const int64_t blocks = std::min<int64_t>(ceil_div(max_units, 8), (int64_t)num_sms() * 16);
  const float2 *zz = static_cast<const float2 *>(z);
  if (nfeed == 1)
    vecdot_kernel<1><<<(unsigned)blocks, 256, 0, s>>>(zz, Kcap, n_dev, n_host, kmul, pairs, npairs, k_chunk, part);
  else
    vecdot_kernel<2><<<(unsigned)blocks, 256, 0, s>>>(zz, Kcap, n_dev, n_host, kmul, pairs, npairs, k_chunk, part);
  int rc = check_launch("vecdot_kernel");
  if (rc) return rc;
  const int64_t per = npairs * nfeed * nfeed;
  const int64_t rblocks = std::min<int64_t>(ceil_div(per, 256), (int64_t)num_sms() * 8);
  if (out_c128)
    vecdot_reduce_kernel<double2><<<(unsigned)rblocks, 256, 0, s>>>(part, Kcap, n_dev, n_host, kmul, nfeed, npairs,
                                                                    k_chunk, out, accumulate);
  else
    vecdot_reduce_kernel<float2><<<(unsigned)rblocks, 256, 0, s>>>(part, Kcap, n_dev, n_host, kmul, nfeed, npairs,
                                                                   k_chunk, out, accumulate);
  return check_launch("vecdot_reduce_kernel");
}

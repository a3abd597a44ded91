// A6: phase term and Z matrix.
//
// Reference: core/tau.py:30-31, 48-71 (exptau = exp(+i 2 pi nu / c * D . X), the
// sign the code uses), core/getz.py:52-105 (Z[a, f, x, s] = exptau[a, s] *
// sqrt_flux[s] * beam[beam_idx[a], f, x, s], rows a * nfeed + f, columns
// x * nsrc + s).
//
// Phase: t = (nu / c) (D . X) in cycles, evaluated in FP64 and reduced to
// r = t - rint(t) in [-1/2, 1/2] before an FP32 sincospi(2 r); at 1 km and
// 200 MHz |t| reaches 670 cycles, where an FP32 phase would carry 2.4e-4 rad of
// error.  Z columns are ordered k = s * nax + x (the source sum is the same).
//
// Split formats (the operand of the tensor-core Hermitian product):
//   bf16, P terms: t0 = bf16_rn(v), t1 = bf16_rn(v - t0), t2 = bf16_rn(v - t0 - t1)
//   tf32, 2 terms: t0 = tf32_rna(v), t1 = tf32_rna(v - t0)
//   fp16, 2 terms of s*v: t0 = fp16_rn(s v), t1 = fp16_rn(s v - t0), s = zscale
// each residual being exact in FP32.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "common.cuh"

namespace mvb {

constexpr double kInvC = 1.0 / 299792458.0;

__device__ __forceinline__ float tf32_rna(float v) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(v));
  return __uint_as_float(r);
}

// Writes NV consecutive real values of one component (c = 0 real, 1 imaginary)
// as the P split terms into planes [2p + c] of a panel row, with vector stores:
// NV = 8 bf16 (16 bytes) or NV = 4 bf16 (8 bytes), NV float32 (16-byte stores).
template <int MODE, int NV>
__device__ __forceinline__ void put_split(void *z, int64_t plane_stride, int64_t off, int comp, const float *v,
                                          float zscale) {
  if constexpr (MODE == MVB_GEMM_F16_3) {
#pragma unroll
    for (int p = 0; p < 2; ++p) {
      uint32_t w[NV / 2];
#pragma unroll
      for (int i = 0; i < NV; i += 2) {
        const float r0 = v[i] * zscale, r1 = v[i + 1] * zscale;
        const __half h0 = __float2half_rn(r0), h1 = __float2half_rn(r1);
        const __half q0 = p == 0 ? h0 : __float2half_rn(r0 - __half2float(h0));
        const __half q1 = p == 0 ? h1 : __float2half_rn(r1 - __half2float(h1));
        w[i / 2] = (uint32_t)__half_as_ushort(q0) | ((uint32_t)__half_as_ushort(q1) << 16);
      }
      __half *pp = static_cast<__half *>(z) + off + (int64_t)(2 * p + comp) * plane_stride;
      if constexpr (NV == 8)
        *reinterpret_cast<uint4 *>(pp) = make_uint4(w[0], w[1], w[2], w[3]);
      else
        *reinterpret_cast<uint2 *>(pp) = make_uint2(w[0], w[1]);
    }
  } else if constexpr (MODE == MVB_GEMM_TF32_3) {
    float hi[NV], lo[NV];
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      hi[i] = tf32_rna(v[i]);
      lo[i] = tf32_rna(v[i] - hi[i]);
    }
    float *p0 = static_cast<float *>(z) + off + (int64_t)(0 + comp) * plane_stride;
    float *p1 = static_cast<float *>(z) + off + (int64_t)(2 + comp) * plane_stride;
#pragma unroll
    for (int i = 0; i < NV; i += 4) {
      *reinterpret_cast<float4 *>(p0 + i) = make_float4(hi[i], hi[i + 1], hi[i + 2], hi[i + 3]);
      *reinterpret_cast<float4 *>(p1 + i) = make_float4(lo[i], lo[i + 1], lo[i + 2], lo[i + 3]);
    }
  } else {
    constexpr int P = MODE == MVB_GEMM_BF16_6 ? 3 : 2;
    float r[NV];
#pragma unroll
    for (int i = 0; i < NV; ++i) r[i] = v[i];
#pragma unroll
    for (int p = 0; p < P; ++p) {
      uint32_t w[NV / 2];
#pragma unroll
      for (int i = 0; i < NV; i += 2) {
        const __nv_bfloat16 t0 = __float2bfloat16_rn(r[i]);
        const __nv_bfloat16 t1 = __float2bfloat16_rn(r[i + 1]);
        r[i] -= __bfloat162float(t0);
        r[i + 1] -= __bfloat162float(t1);
        w[i / 2] = (uint32_t)__bfloat16_as_ushort(t0) | ((uint32_t)__bfloat16_as_ushort(t1) << 16);
      }
      __nv_bfloat16 *pp = static_cast<__nv_bfloat16 *>(z) + off + (int64_t)(2 * p + comp) * plane_stride;
      if constexpr (NV == 8)
        *reinterpret_cast<uint4 *>(pp) = make_uint4(w[0], w[1], w[2], w[3]);
      else
        *reinterpret_cast<uint2 *>(pp) = make_uint2(w[0], w[1]);
    }
  }
}

// Single-value writer kept for the pack kernel (2 consecutive values).
template <int MODE>
struct PanelWriter {
  static constexpr int P = MODE == MVB_GEMM_BF16_6 ? 3 : 2;
  static __device__ __forceinline__ void put(void *z, int64_t plane_stride, int64_t off, int comp, const float *v,
                                             int X, float zscale) {
    if constexpr (MODE == MVB_GEMM_F16_3) {
      __half *zp = static_cast<__half *>(z) + off;
      for (int x = 0; x < X; ++x) {
        const float r = v[x] * zscale;
        const __half hi = __float2half_rn(r);
        zp[(2 * 0 + comp) * plane_stride + x] = hi;
        zp[(2 * 1 + comp) * plane_stride + x] = __float2half_rn(r - __half2float(hi));
      }
    } else if constexpr (MODE == MVB_GEMM_TF32_3) {
      float *zp = static_cast<float *>(z) + off;
      float hi[2], lo[2];
      for (int x = 0; x < X; ++x) {
        hi[x] = tf32_rna(v[x]);
        lo[x] = tf32_rna(v[x] - hi[x]);
      }
      float *p0 = zp + (2 * 0 + comp) * plane_stride;
      float *p1 = zp + (2 * 1 + comp) * plane_stride;
      if (X == 2) {
        *reinterpret_cast<float2 *>(p0) = make_float2(hi[0], hi[1]);
        *reinterpret_cast<float2 *>(p1) = make_float2(lo[0], lo[1]);
      } else {
        *p0 = hi[0];
        *p1 = lo[0];
      }
    } else {
      __nv_bfloat16 *zp = static_cast<__nv_bfloat16 *>(z) + off;
      __nv_bfloat16 t[3][2];
      for (int x = 0; x < X; ++x) {
        float r = v[x];
#pragma unroll
        for (int p = 0; p < P; ++p) {
          t[p][x] = __float2bfloat16_rn(r);
          r = r - __bfloat162float(t[p][x]);
        }
      }
#pragma unroll
      for (int p = 0; p < P; ++p) {
        __nv_bfloat16 *pp = zp + (2 * p + comp) * plane_stride;
        if (X == 2) {
          __nv_bfloat162 two;
          two.x = t[p][0];
          two.y = t[p][1];
          *reinterpret_cast<__nv_bfloat162 *>(pp) = two;
        } else {
          *pp = t[p][0];
        }
      }
    }
  }
};

constexpr int kTauZThreads = 64;
constexpr int kTauZSrc = 4;      // consecutive sources per thread
constexpr int kTauZAnts = 32;    // antennas per CTA (the CTA's beam block is read once per 32 antennas)
constexpr int kTauZMaxBFX = 16;  // beams staged in shared memory up to nbeam * F * X = 16, else read from L2
constexpr int kTauZBlockSrc = kTauZThreads * kTauZSrc;

// grid.x: blocks of kTauZBlockSrc sources, grid.y: antenna blocks.  Dynamic
// shared memory: the CTA's beam values, [q][j][thread] (thread fastest, so the
// per-antenna reads are conflict-free), q = (beam * F + f) * X + x.
// EXT = 0: phase from antpos . crd (fused tau); EXT = 1 / 2: phase factor read
// from a caller exptau (A, e_ld) in complex64 / complex128, multiplied by sflux.
template <int MODE, int X, int EXT = 0, bool STAGED = true>
__global__ void __launch_bounds__(kTauZThreads)
    tau_z_kernel(const double *__restrict__ antpos, int A, double f_over_c, const double *__restrict__ crd, int64_t ld,
                 const int32_t *__restrict__ n_dev, int64_t nsrc, const float *__restrict__ sflux,
                 const int32_t *__restrict__ sidx, const float2 *__restrict__ beam, int64_t beam_ld, int nbeam,
                 const int32_t *__restrict__ beam_idx, int F, float zscale, void *__restrict__ z, int64_t Mpad,
                 int64_t Kcap, const void *__restrict__ ext = nullptr, int64_t e_ld = 0) {
  extern __shared__ float2 bsm[];
  const int64_t n = n_dev ? min((int64_t)*n_dev, nsrc) : nsrc;
  const int64_t s_end = round_up(n * X, kKAlign) / X;  // zero-fill up to here
  const int64_t s0 = ((int64_t)blockIdx.x * kTauZThreads + threadIdx.x) * kTauZSrc;
  if ((int64_t)blockIdx.x * kTauZBlockSrc >= s_end) return;  // uniform per CTA
  const bool write = s0 < s_end;  // s_end is a multiple of kTauZSrc (64 / X)

  double cx[kTauZSrc], cy[kTauZSrc], cz[kTauZSrc];
  float sf[kTauZSrc];
#pragma unroll
  for (int j = 0; j < kTauZSrc; ++j) {
    const int64_t s = s0 + j;
    const bool live = s < n;
    cx[j] = cy[j] = cz[j] = 0.0;
    sf[j] = 0.f;
    if (live) {
      if (EXT == 0) {
        cx[j] = crd[s];
        cy[j] = crd[ld + s];
        cz[j] = crd[2 * ld + s];
      }
      sf[j] = sflux[sidx ? sidx[s] : s];
    }
  }
  const int nbfx = nbeam * F * X;
  if constexpr (STAGED) {
    for (int q = 0; q < nbfx; ++q)
#pragma unroll
      for (int j = 0; j < kTauZSrc; ++j)
        bsm[(q * kTauZSrc + j) * kTauZThreads + threadIdx.x] =
            (s0 + j < n) ? beam[(int64_t)q * beam_ld + s0 + j] : make_float2(0.f, 0.f);
  }
  // (each thread reads only its own entries of bsm: no barrier needed)

  const int a0 = blockIdx.y * kTauZAnts;
  const int a1 = min(a0 + kTauZAnts, A);
  const int64_t plane = Mpad * Kcap;
  for (int a = a0; a < a1; ++a) {
    float er[kTauZSrc], ei[kTauZSrc];
    double dx = 0, dy = 0, dz = 0;
    if (EXT == 0) {
      dx = antpos[3 * a];
      dy = antpos[3 * a + 1];
      dz = antpos[3 * a + 2];
    }
#pragma unroll
    for (int j = 0; j < kTauZSrc; ++j) {
      er[j] = ei[j] = 0.f;
      if (s0 + j >= n) continue;
      if (EXT == 1) {
        const float2 e = static_cast<const float2 *>(ext)[(int64_t)a * e_ld + s0 + j];
        er[j] = e.x * sf[j];
        ei[j] = e.y * sf[j];
      } else if (EXT == 2) {
        const double2 e = static_cast<const double2 *>(ext)[(int64_t)a * e_ld + s0 + j];
        er[j] = (float)(e.x * (double)sf[j]);
        ei[j] = (float)(e.y * (double)sf[j]);
      } else {
        const double t = (dx * cx[j] + dy * cy[j] + dz * cz[j]) * f_over_c;
        const double r = t - rint(t);
        float sn, cs;
        sincospif((float)(2.0 * r), &sn, &cs);
        er[j] = cs * sf[j];
        ei[j] = sn * sf[j];
      }
    }
    const int b = beam_idx ? beam_idx[a] : 0;
    for (int f = 0; f < F; ++f) {
      float vr[kTauZSrc * X], vi[kTauZSrc * X];
#pragma unroll
      for (int j = 0; j < kTauZSrc; ++j)
#pragma unroll
        for (int x = 0; x < X; ++x) {
          const int q = (b * F + f) * X + x;
          float2 bv;
          if constexpr (STAGED)
            bv = bsm[(q * kTauZSrc + j) * kTauZThreads + threadIdx.x];
          else
            bv = (s0 + j < n) ? beam[(int64_t)q * beam_ld + s0 + j] : make_float2(0.f, 0.f);
          vr[j * X + x] = er[j] * bv.x - ei[j] * bv.y;
          vi[j * X + x] = er[j] * bv.y + ei[j] * bv.x;
        }
      if (!write) continue;
      const int64_t m = (int64_t)a * F + f;
      if constexpr (MODE == MVB_Z_C64) {
        float2 *zp = static_cast<float2 *>(z) + m * Kcap + s0 * X;
#pragma unroll
        for (int i = 0; i < kTauZSrc * X; i += 2)
          *reinterpret_cast<float4 *>(zp + i) = make_float4(vr[i], vi[i], vr[i + 1], vi[i + 1]);
      } else {
        // kTauZSrc * X consecutive k from a multiple of kTauZSrc * X: inside one k-block
        const int64_t off = panel_off(m, s0 * X, Mpad, kKBlockBytes / (MODE == MVB_GEMM_TF32_3 ? 4 : 2));
        put_split<MODE, kTauZSrc * X>(z, plane, off, 0, vr, zscale);
        put_split<MODE, kTauZSrc * X>(z, plane, off, 1, vi, zscale);
      }
    }
  }
}

__global__ void exptau_kernel(const double *__restrict__ antpos, int A, double f_over_c, const double *__restrict__ crd,
                              int64_t ld, int64_t nsrc, void *__restrict__ out, int out_c128) {
  const int64_t total = (int64_t)A * nsrc;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t a = i / nsrc, s = i % nsrc;
    const double t = (antpos[3 * a] * crd[s] + antpos[3 * a + 1] * crd[ld + s] + antpos[3 * a + 2] * crd[2 * ld + s]) *
                     f_over_c;
    const double r = t - rint(t);
    if (out_c128) {
      double sn, cs;
      sincospi(2.0 * r, &sn, &cs);
      static_cast<double2 *>(out)[i] = make_double2(cs, sn);
    } else {
      float sn, cs;
      sincospif((float)(2.0 * r), &sn, &cs);
      static_cast<float2 *>(out)[i] = make_float2(cs, sn);
    }
  }
}

// Packs a caller complex matrix (M, K) into a panel; one thread per (m, k-pair).
template <int MODE, typename CT>
__global__ void z_pack_kernel(const CT *__restrict__ zs, int64_t M, int64_t K, int64_t ldz, float zscale,
                              void *__restrict__ z, int64_t Mpad, int64_t Kcap) {
  const int64_t kend = round_up(K, kKAlign);
  const int64_t half = kend / 2;
  const int64_t total = M * half;
  const int64_t plane = Mpad * Kcap;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t m = i / half, k = (i % half) * 2;
    float vr[2], vi[2];
    for (int x = 0; x < 2; ++x) {
      if (k + x < K) {
        const CT v = zs[m * ldz + k + x];
        vr[x] = (float)v.x;
        vi[x] = (float)v.y;
      } else {
        vr[x] = vi[x] = 0.f;
      }
    }
    if constexpr (MODE == MVB_Z_C64) {
      *reinterpret_cast<float4 *>(static_cast<float2 *>(z) + m * Kcap + k) = make_float4(vr[0], vi[0], vr[1], vi[1]);
    } else {
      // (k, k + 1), k even: inside one k-block
      const int64_t off = panel_off(m, k, Mpad, kKBlockBytes / (MODE == MVB_GEMM_TF32_3 ? 4 : 2));
      PanelWriter<MODE>::put(z, plane, off, 0, vr, 2, zscale);
      PanelWriter<MODE>::put(z, plane, off, 1, vi, 2, zscale);
    }
  }
}

template <typename CT>
__global__ void absmax_kernel(const CT *__restrict__ z, int64_t n, float *__restrict__ out) {
  float m = 0.f;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const CT v = z[i];
    m = fmaxf(m, (float)sqrt((double)v.x * v.x + (double)v.y * v.y));
  }
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  // non-negative floats order like their bit patterns
  if ((threadIdx.x & 31) == 0) atomicMax(reinterpret_cast<int *>(out), __float_as_int(m));
}

}  // namespace mvb

using namespace mvb;

extern "C" int mvb_absmax(const void *z, int z_c128, int64_t n, float *out, void *stream) {
  if (!out || n < 0 || (n > 0 && !z)) return fail(MVB_ERR_ARG, "mvb_absmax: bad arguments");
  if (n == 0) return MVB_OK;
  const int threads = 256;
  const int64_t blocks = std::min<int64_t>(ceil_div(n, threads), (int64_t)num_sms() * 8);
  if (z_c128)
    absmax_kernel<double2><<<(unsigned)blocks, threads, 0, as_stream(stream)>>>(static_cast<const double2 *>(z), n, out);
  else
    absmax_kernel<float2><<<(unsigned)blocks, threads, 0, as_stream(stream)>>>(static_cast<const float2 *>(z), n, out);
  return check_launch("absmax_kernel");
}

extern "C" size_t mvb_zpanel_bytes(int mode, int64_t Mpad, int64_t Kcap) {
  if (mode == MVB_Z_C64) return (size_t)Mpad * Kcap * 8;
  return (size_t)2 * mode_terms(mode) * Mpad * Kcap * mode_elem_bytes(mode);
}

static int check_panel(int mode, int64_t M, int64_t Mpad, int64_t Kcap, const char *who) {
  if (mode < MVB_GEMM_BF16_3 || mode > MVB_GEMM_F16_3) return fail(MVB_ERR_ARG, "%s: unknown mode %d", who, mode);
  if (Kcap % kKAlign) return fail(MVB_ERR_ARG, "%s: Kcap must be a multiple of %d", who, kKAlign);
  if (Mpad < M) return fail(MVB_ERR_ARG, "%s: Mpad < M", who);
  if (mode != MVB_Z_C64 && Mpad % kTile) return fail(MVB_ERR_ARG, "%s: Mpad must be a multiple of %d", who, kTile);
  return MVB_OK;
}

extern "C" int mvb_exptau(const double *antpos, int A, double freq, const double *crd, int64_t ld, int64_t nsrc,
                          void *exptau, int out_c128, void *stream) {
  if (A < 0 || nsrc < 0 || ((int64_t)A * nsrc > 0 && (!antpos || !crd || !exptau)))
    return fail(MVB_ERR_ARG, "mvb_exptau: bad arguments");
  const int64_t total = (int64_t)A * nsrc;
  if (total == 0) return MVB_OK;
  const int threads = 256;
  const int64_t blocks = std::min<int64_t>(ceil_div(total, threads), (int64_t)num_sms() * 16);
  exptau_kernel<<<(unsigned)blocks, threads, 0, as_stream(stream)>>>(antpos, A, freq * kInvC, crd, ld, nsrc, exptau,
                                                                     out_c128);
  return check_launch("exptau_kernel");
}

extern "C" int mvb_tau_z(const double *antpos, int A, double freq, const double *crd, int64_t ld, const int32_t *n_dev,
                         int64_t nsrc, const float *sflux, const int32_t *sidx, const void *beam, int64_t beam_ld,
                         int nbeam, const int32_t *beam_idx, int F, int X, int mode, float zscale, void *z,
                         int64_t Mpad, int64_t Kcap, void *stream) {
  if (A <= 0 || nsrc < 0 || !antpos || !z || !beam || !sflux || (nsrc > 0 && !crd) || (F != 1 && F != 2) ||
      (X != 1 && X != 2) || nbeam <= 0 || beam_ld < nsrc)
    return fail(MVB_ERR_ARG, "mvb_tau_z: bad arguments");
  const bool staged = nbeam * F * X <= kTauZMaxBFX;
  int rc = check_panel(mode, (int64_t)A * F, Mpad, Kcap, "mvb_tau_z");
  if (rc) return rc;
  if (round_up(nsrc * X, kKAlign) > Kcap) return fail(MVB_ERR_ARG, "mvb_tau_z: Kcap too small for nsrc * nax");
  const int64_t s_max = round_up(nsrc * X, kKAlign) / X;
  if (s_max == 0) return MVB_OK;
  dim3 grid((unsigned)ceil_div(s_max, kTauZBlockSrc), (unsigned)ceil_div(A, kTauZAnts));
  const double foc = freq * kInvC;
  const size_t smem = staged ? (size_t)nbeam * F * X * kTauZSrc * kTauZThreads * sizeof(float2) : 0;
  const float2 *bm = static_cast<const float2 *>(beam);
  cudaStream_t s = as_stream(stream);
#define MVB_TAUZ(M, XX)                                                                                        \
  do {                                                                                                         \
  if (staged)                                                                                                  \
    tau_z_kernel<M, XX, 0, true><<<grid, kTauZThreads, smem, s>>>(antpos, A, foc, crd, ld, n_dev, nsrc, sflux, sidx, \
                                                                bm, beam_ld, nbeam, beam_idx, F, zscale, z, Mpad, Kcap); \
  else                                                                                                         \
    tau_z_kernel<M, XX, 0, false><<<grid, kTauZThreads, 0, s>>>(antpos, A, foc, crd, ld, n_dev, nsrc, sflux, sidx, \
                                                              bm, beam_ld, nbeam, beam_idx, F, zscale, z, Mpad, Kcap); \
  } while (0)
#define MVB_TAUZ2(M) \
  if (X == 2)        \
    MVB_TAUZ(M, 2);  \
  else               \
    MVB_TAUZ(M, 1)
  switch (mode) {
    case MVB_GEMM_BF16_3: MVB_TAUZ2(MVB_GEMM_BF16_3); break;
    case MVB_GEMM_BF16_6: MVB_TAUZ2(MVB_GEMM_BF16_6); break;
    case MVB_GEMM_TF32_3: MVB_TAUZ2(MVB_GEMM_TF32_3); break;
    case MVB_GEMM_F16_3: MVB_TAUZ2(MVB_GEMM_F16_3); break;
    default: MVB_TAUZ2(MVB_Z_C64); break;
  }
#undef MVB_TAUZ2
#undef MVB_TAUZ
  return check_launch("tau_z_kernel");
}

extern "C" int mvb_z_pack(const void *zsrc, int z_c128, int64_t M, int64_t K, int64_t ldz, int mode, float zscale,
                          void *z, int64_t Mpad, int64_t Kcap, void *stream) {
  if (M < 0 || K < 0 || ldz < K || !z || (M * K > 0 && !zsrc)) return fail(MVB_ERR_ARG, "mvb_z_pack: bad arguments");
  int rc = check_panel(mode, M, Mpad, Kcap, "mvb_z_pack");
  if (rc) return rc;
  if (round_up(K, kKAlign) > Kcap) return fail(MVB_ERR_ARG, "mvb_z_pack: Kcap too small");
  const int64_t total = M * (round_up(K, kKAlign) / 2);
  if (total == 0) return MVB_OK;
  const int threads = 256;
  const int64_t blocks = std::min<int64_t>(ceil_div(total, threads), (int64_t)num_sms() * 16);
  cudaStream_t s = as_stream(stream);
#define MVB_PACK(M_, CT)                                                                                             \
  z_pack_kernel<M_, CT><<<(unsigned)blocks, threads, 0, s>>>(static_cast<const CT *>(zsrc), M, K, ldz, zscale, z, Mpad, \
                                                             Kcap)
#define MVB_PACK2(M_) \
  if (z_c128)         \
    MVB_PACK(M_, double2); \
  else                \
    MVB_PACK(M_, float2)
  switch (mode) {
    case MVB_GEMM_BF16_3: MVB_PACK2(MVB_GEMM_BF16_3); break;
    case MVB_GEMM_BF16_6: MVB_PACK2(MVB_GEMM_BF16_6); break;
    case MVB_GEMM_TF32_3: MVB_PACK2(MVB_GEMM_TF32_3); break;
    case MVB_GEMM_F16_3: MVB_PACK2(MVB_GEMM_F16_3); break;
    default: MVB_PACK2(MVB_Z_C64); break;
  }
#undef MVB_PACK2
#undef MVB_PACK
  return check_launch("z_pack_kernel");
}

extern "C" int mvb_z_from_exptau(const void *exptau, int e_c128, int64_t e_ld, int A, int64_t nsrc, const float *sflux,
                                 const void *beam, int64_t beam_ld, int nbeam, const int32_t *beam_idx, int F, int X,
                                 int mode, float zscale, void *z, int64_t Mpad, int64_t Kcap, void *stream) {
  if (A <= 0 || nsrc < 0 || !exptau || !z || !beam || !sflux || (F != 1 && F != 2) || (X != 1 && X != 2) ||
      nbeam <= 0 || beam_ld < nsrc || e_ld < nsrc)
    return fail(MVB_ERR_ARG, "mvb_z_from_exptau: bad arguments");
  const bool staged = nbeam * F * X <= kTauZMaxBFX;
  int rc = check_panel(mode, (int64_t)A * F, Mpad, Kcap, "mvb_z_from_exptau");
  if (rc) return rc;
  if (round_up(nsrc * X, kKAlign) > Kcap) return fail(MVB_ERR_ARG, "mvb_z_from_exptau: Kcap too small");
  const int64_t s_max = round_up(nsrc * X, kKAlign) / X;
  if (s_max == 0) return MVB_OK;
  dim3 grid((unsigned)ceil_div(s_max, kTauZBlockSrc), (unsigned)ceil_div(A, kTauZAnts));
  const size_t smem = staged ? (size_t)nbeam * F * X * kTauZSrc * kTauZThreads * sizeof(float2) : 0;
  const float2 *bm = static_cast<const float2 *>(beam);
  cudaStream_t s = as_stream(stream);
#define MVB_ZX(M, XX, E)                                                                                       \
  do {                                                                                                         \
  if (staged)                                                                                                  \
    tau_z_kernel<M, XX, E, true><<<grid, kTauZThreads, smem, s>>>(nullptr, A, 0.0, nullptr, 0, nullptr, nsrc, sflux, \
                                                                nullptr, bm, beam_ld, nbeam, beam_idx, F, zscale, z, \
                                                                Mpad, Kcap, exptau, e_ld);                    \
  else                                                                                                         \
    tau_z_kernel<M, XX, E, false><<<grid, kTauZThreads, 0, s>>>(nullptr, A, 0.0, nullptr, 0, nullptr, nsrc, sflux,  \
                                                              nullptr, bm, beam_ld, nbeam, beam_idx, F, zscale, z,  \
                                                              Mpad, Kcap, exptau, e_ld);                    \
  } while (0)
#define MVB_ZX3(M, E) \
  if (X == 2)         \
    MVB_ZX(M, 2, E);  \
  else                \
    MVB_ZX(M, 1, E)
#define MVB_ZX2(M)    \
  if (e_c128)         \
    MVB_ZX3(M, 2);    \
  else                \
    MVB_ZX3(M, 1)
  switch (mode) {
    case MVB_GEMM_BF16_3: MVB_ZX2(MVB_GEMM_BF16_3); break;
    case MVB_GEMM_BF16_6: MVB_ZX2(MVB_GEMM_BF16_6); break;
    case MVB_GEMM_TF32_3: MVB_ZX2(MVB_GEMM_TF32_3); break;
    case MVB_GEMM_F16_3: MVB_ZX2(MVB_GEMM_F16_3); break;
    default: MVB_ZX2(MVB_Z_C64); break;
  }
#undef MVB_ZX2
#undef MVB_ZX3
#undef MVB_ZX
  return check_launch("tau_z_kernel(exptau)");
}

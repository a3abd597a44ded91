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

// Nearest integer (ties to even) of |t| < 2^51 with two FP64 adds: adding and
// subtracting 1.5 * 2^52 leaves no fraction bits, so the first add rounds t to
// an integer in the current (round-to-nearest-even) mode -- the same value as
// rint(t), on the FP64 add pipe instead of the conversion unit.  |t| here is a
// path difference in wavelengths (< 2^40 for any physical array).
__device__ __forceinline__ double round_half_even(double t) {
  const double magic = 6755399441055744.0;  // 1.5 * 2^52
  return __dsub_rn(__dadd_rn(t, magic), magic);
}

__device__ __forceinline__ float tf32_rna(float v) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(v));
  return __uint_as_float(r);
}

// Vector stores of W consecutive 32-bit words (W = 1, 2, 4, 8: 4 to 32 bytes,
// aligned to min(size, 16) bytes by the callers).
template <int W>
__device__ __forceinline__ void store_words(void *p, const uint32_t *w) {
  static_assert(W == 1 || W == 2 || W == 4 || W == 8, "1, 2, 4 or 8 words");
  if constexpr (W == 8) {
    *reinterpret_cast<uint4 *>(p) = make_uint4(w[0], w[1], w[2], w[3]);
    *(reinterpret_cast<uint4 *>(p) + 1) = make_uint4(w[4], w[5], w[6], w[7]);
  } else if constexpr (W == 4)
    *reinterpret_cast<uint4 *>(p) = make_uint4(w[0], w[1], w[2], w[3]);
  else if constexpr (W == 2)
    *reinterpret_cast<uint2 *>(p) = make_uint2(w[0], w[1]);
  else
    *reinterpret_cast<uint32_t *>(p) = w[0];
}

// One 32-byte store of 8 words (p 32-byte aligned): a whole L2 sector in one
// instruction.
__device__ __forceinline__ void store_sector(void *p, const uint32_t *w) {
  asm volatile("st.global.v8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(p), "r"(w[0]), "r"(w[1]), "r"(w[2]),
               "r"(w[3]), "r"(w[4]), "r"(w[5]), "r"(w[6]), "r"(w[7])
               : "memory");
}

// Writes NV consecutive real values of one component (c = 0 real, 1 imaginary)
// as the P split terms into planes [2p + c] of a panel row, with vector stores:
// NV = 4 or 8 values: 8- or 16-byte stores of bf16 / fp16 (inside one 16-byte
// chunk of the swizzled row, at off), 16 bytes of float32 at off, or 2 x 16
// bytes of float32 at off (values 0..3) and off2 (values 4..7: the next chunk,
// which the swizzle may place anywhere in the row).
template <int MODE, int NV>
__device__ __forceinline__ void put_split(void *z, int64_t plane_stride, int64_t off, int64_t off2, int comp,
                                          const float *v, float zscale) {
  if constexpr (MODE == MVB_GEMM_F16_3) {
    // one paired conversion per two values for each term (cvt.rn.f16x2.f32)
    uint32_t whi[NV / 2], wlo[NV / 2];
#pragma unroll
    for (int i = 0; i < NV; i += 2) {
      const float r0 = v[i] * zscale, r1 = v[i + 1] * zscale;
      const __half2 hi = __floats2half2_rn(r0, r1);
      const float2 back = __half22float2(hi);
      const __half2 lo = __floats2half2_rn(r0 - back.x, r1 - back.y);
      whi[i / 2] = *reinterpret_cast<const uint32_t *>(&hi);
      wlo[i / 2] = *reinterpret_cast<const uint32_t *>(&lo);
    }
    __half *p0 = static_cast<__half *>(z) + off + (int64_t)(0 + comp) * plane_stride;
    __half *p1 = static_cast<__half *>(z) + off + (int64_t)(2 + comp) * plane_stride;
    store_words<NV / 2>(p0, whi);
    store_words<NV / 2>(p1, wlo);
  } else if constexpr (MODE == MVB_GEMM_TF32_3) {
    float hi[NV], lo[NV];
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      hi[i] = tf32_rna(v[i]);
      lo[i] = tf32_rna(v[i] - hi[i]);
    }
    float *p0 = static_cast<float *>(z) + off + (int64_t)(0 + comp) * plane_stride;
    float *p1 = static_cast<float *>(z) + off + (int64_t)(2 + comp) * plane_stride;
    uint32_t whi[NV], wlo[NV];
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      whi[i] = __float_as_uint(hi[i]);
      wlo[i] = __float_as_uint(lo[i]);
    }
    if constexpr (NV == 8) {
      // values 0..3 and 4..7 fill the two 16-byte chunks of one 32-byte sector
      // (the 64-byte swizzle keeps chunk pairs {0, 1} and {2, 3} together, in
      // either order): one sector store per plane
      const bool swapped = off2 < off;
      const int64_t base = swapped ? off2 : off;
      uint32_t shi[8], slo[8];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        shi[i] = swapped ? whi[4 + i] : whi[i];
        shi[4 + i] = swapped ? whi[i] : whi[4 + i];
        slo[i] = swapped ? wlo[4 + i] : wlo[i];
        slo[4 + i] = swapped ? wlo[i] : wlo[4 + i];
      }
      store_sector(static_cast<float *>(z) + base + (int64_t)(0 + comp) * plane_stride, shi);
      store_sector(static_cast<float *>(z) + base + (int64_t)(2 + comp) * plane_stride, slo);
    } else {
      store_words<NV>(p0, whi);
      store_words<NV>(p1, wlo);
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
        // one paired conversion per two values (cvt.rn.bf16x2.f32); bf16 -> f32 is exact
        const __nv_bfloat162 t = __floats2bfloat162_rn(r[i], r[i + 1]);
        const float2 back = __bfloat1622float2(t);
        r[i] -= back.x;
        r[i + 1] -= back.y;
        w[i / 2] = *reinterpret_cast<const uint32_t *>(&t);
      }
      __nv_bfloat16 *pp = static_cast<__nv_bfloat16 *>(z) + off + (int64_t)(2 * p + comp) * plane_stride;
      store_words<NV / 2>(pp, w);
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

// CTA = 128 threads over 32 sources x 64 antennas: thread bits 0..2 pick a group
// of 4 consecutive sources (16-byte stores per plane at X = 2), bits 3..6 one of
// 16 antenna lanes, each lane taking every 16th antenna of the block.  A CTA
// thus writes only 4 k-blocks (X = 2) of 128 rows, so the Z lines it has open at
// any time fit, summed over the resident CTAs, well inside L2 (a wider k-range
// per CTA left partially written lines to be evicted); a warp's store writes 16
// whole 32-byte sectors.  The CTA's beam values (nbeam * F * X x 32 sources)
// are staged once in shared memory for its 16 antenna lanes.
constexpr int kTauZThreads = 128;
constexpr int kTauZSrc = 4;                 // consecutive sources per thread
constexpr int kTauZGroups = 8;              // source groups per CTA
constexpr int kTauZAntLanes = kTauZThreads / kTauZGroups;
constexpr int kTauZAnts = 64;               // antennas per CTA
constexpr int kTauZBlockSrc = kTauZGroups * kTauZSrc;
constexpr int kTauZRow = kTauZBlockSrc + 1;  // staged beam values per q, padded
constexpr int kTauZMaxBFX = 16;              // beam planes staged in shared memory, else read through L1

// grid.x: blocks of kTauZBlockSrc sources, grid.y: blocks of kTauZAnts antennas,
// grid.z: the frequencies of a grouped launch (freqs != nullptr): frequency
// freqs[z], fluxes sflux + z sflux_ld (coh + z coh_ld), panel z + z zstride bytes.
// EXT = 0: phase from antpos . crd (fused tau); EXT = 1 / 2: phase factor read
// from a caller exptau (A, e_ld) in complex64 / complex128, multiplied by sflux.
// POL (EXT = 0, X = 2): polarised sky.  Instead of sqrt(0.5 I) the source
// carries its coherency C (coh[sidx[s]] = C00, C11, Re C01, Im C01 at this
// frequency) and frame rotation R (rot[s] = cos X, sin X); with C' = R^T C R =
// L L^H (lower-triangular L), Z[a, f, (s, y)] = exptau(a, s) sum_x
// beam[f, x, s] L[x, y, s], so that Z Z^H gives exptau_j conj(exptau_i)
// E_j C' E_i^H per source.
template <int MODE, int X, int EXT = 0, bool STAGED = true, bool POL = false>
__global__ void __launch_bounds__(kTauZThreads)
    tau_z_kernel(const double *__restrict__ antpos, int A, double f_over_c, const double *__restrict__ crd, int64_t ld,
                 const int32_t *__restrict__ n_dev, int64_t nsrc, const float *__restrict__ sflux,
                 const int32_t *__restrict__ sidx, const float2 *__restrict__ beam, int64_t beam_ld, int nbeam,
                 const int32_t *__restrict__ beam_idx, int F, float zscale, void *__restrict__ z, int64_t Mpad,
                 int64_t Kcap, const void *__restrict__ ext = nullptr, int64_t e_ld = 0,
                 const float4 *__restrict__ coh = nullptr, const double2 *__restrict__ rot = nullptr,
                 const double *__restrict__ freqs = nullptr, int64_t sflux_ld = 0, int64_t coh_ld = 0,
                 int64_t zstride = 0) {
  static_assert(!POL || (X == 2 && EXT == 0), "the polarised sky needs two beam axes and the fused phase");
  if (freqs) {  // grouped: this block's frequency
    const int gz = blockIdx.z;
    f_over_c = freqs[gz] * kInvC;
    if (sflux) sflux += gz * sflux_ld;
    if (coh) coh += gz * coh_ld;
    z = static_cast<uint8_t *>(z) + gz * zstride;
  }
  const int64_t n = n_dev ? min((int64_t)*n_dev, nsrc) : nsrc;
  const int64_t s_end = round_up(n * X, kKAlign) / X;  // zero-fill up to here
  const int64_t s0 = (int64_t)blockIdx.x * kTauZBlockSrc + (threadIdx.x % kTauZGroups) * kTauZSrc;
  const int alane = threadIdx.x / kTauZGroups;
  if ((int64_t)blockIdx.x * kTauZBlockSrc >= s_end) return;  // uniform per CTA
  const bool write = s0 < s_end;  // s_end is a multiple of kTauZSrc (64 / X)

  double cx[kTauZSrc], cy[kTauZSrc], cz[kTauZSrc];
  float sf[kTauZSrc];
  float l00[POL ? kTauZSrc : 1], l10r[POL ? kTauZSrc : 1], l10i[POL ? kTauZSrc : 1], l11[POL ? kTauZSrc : 1];
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
      if constexpr (POL) {
        // C' = R^T C R, then its Cholesky factor (clamped at the PSD boundary)
        const float4 c = coh[sidx ? sidx[s] : s];
        const double2 r = rot[s];
        const double cr = r.x, sr = r.y;
        const double a = c.x, d = c.y, br = c.z, bi = c.w;
        const double c00 = cr * cr * a + sr * sr * d - 2.0 * cr * sr * br;
        const double c11 = sr * sr * a + cr * cr * d + 2.0 * cr * sr * br;
        // C'_10 = conj(C'_01), C'_01 = cr sr (a - d) + cr^2 b - sr^2 conj(b)
        const double c10r = cr * sr * (a - d) + (cr * cr - sr * sr) * br;
        const double c10i = -(cr * cr + sr * sr) * bi;
        const double L00 = sqrt(fmax(c00, 0.0));
        const double L10r = L00 > 0.0 ? c10r / L00 : 0.0, L10i = L00 > 0.0 ? c10i / L00 : 0.0;
        l00[j] = (float)L00;
        l10r[j] = (float)L10r;
        l10i[j] = (float)L10i;
        l11[j] = (float)sqrt(fmax(c11 - L10r * L10r - L10i * L10i, 0.0));
        sf[j] = 1.f;
      } else {
        sf[j] = sflux[sidx ? sidx[s] : s];
      }
    } else if constexpr (POL) {
      l00[j] = l10r[j] = l10i[j] = l11[j] = 0.f;
    }
  }
  // STAGED: the CTA's beam values, shared by its 16 antenna lanes, in shared
  // memory as [q][j][group] with a row of 33 values per q (q = (beam * F + f) *
  // X + x): the 8 source groups of a warp read 8 consecutive values, and lanes
  // with different beams land on different banks.  Otherwise (more than 16 beam
  // planes) the values are read through L1 per antenna.
  extern __shared__ float2 bsm[];
  if constexpr (STAGED) {
    const int nq = nbeam * F * X;
    for (int e = threadIdx.x; e < nq * kTauZBlockSrc; e += kTauZThreads) {
      const int q = e / kTauZBlockSrc, sl = e % kTauZBlockSrc;  // sl = group * kTauZSrc + j
      const int64_t ss = (int64_t)blockIdx.x * kTauZBlockSrc + sl;
      bsm[q * kTauZRow + (sl % kTauZSrc) * kTauZGroups + sl / kTauZSrc] =
          ss < n ? __ldg(beam + (int64_t)q * beam_ld + ss) : make_float2(0.f, 0.f);
    }
    __syncthreads();
  }
  const int sg = threadIdx.x % kTauZGroups;
  const int a0 = blockIdx.y * kTauZAnts;
  const int a1 = min(a0 + kTauZAnts, A);
  {
    for (int a = a0 + alane; a < a1; a += kTauZAntLanes) {
      const int b = beam_idx ? beam_idx[a] : 0;
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
          const double r = t - round_half_even(t);
          float sn, cs;
          sincospif((float)(2.0 * r), &sn, &cs);
          er[j] = cs * sf[j];
          ei[j] = sn * sf[j];
        }
      }
#pragma unroll
      for (int f = 0; f < 2; ++f) {
        if (f >= F) break;
        float vr[kTauZSrc * X], vi[kTauZSrc * X];
#pragma unroll
        for (int j = 0; j < kTauZSrc; ++j)
#pragma unroll
          for (int x = 0; x < X; ++x) {
            const int q = (b * F + f) * X + x;
            float2 bv;
            if constexpr (STAGED)
              bv = bsm[q * kTauZRow + j * kTauZGroups + sg];
            else
              bv = (s0 + j < n) ? __ldg(beam + (int64_t)q * beam_ld + s0 + j) : make_float2(0.f, 0.f);
            vr[j * X + x] = er[j] * bv.x - ei[j] * bv.y;
            vi[j * X + x] = er[j] * bv.y + ei[j] * bv.x;
          }
        if constexpr (POL) {
          // (g0, g1) = exptau * beam[f, 0:2]  ->  (g0 L00 + g1 L10, g1 L11)
#pragma unroll
          for (int j = 0; j < kTauZSrc; ++j) {
            const float g0r = vr[2 * j], g0i = vi[2 * j], g1r = vr[2 * j + 1], g1i = vi[2 * j + 1];
            vr[2 * j] = g0r * l00[j] + g1r * l10r[j] - g1i * l10i[j];
            vi[2 * j] = g0i * l00[j] + g1r * l10i[j] + g1i * l10r[j];
            vr[2 * j + 1] = g1r * l11[j];
            vi[2 * j + 1] = g1i * l11[j];
          }
        }
        if (!write) continue;
        const int64_t m = (int64_t)a * F + f;
        if constexpr (MODE == MVB_Z_C64) {
          // the row's kTauZSrc * X values start 32-byte aligned (Kcap a multiple
          // of 64, s0 X of 4): whole 32-byte sectors, four values each
          float2 *zp = static_cast<float2 *>(z) + m * Kcap + s0 * X;
#pragma unroll
          for (int i = 0; i < kTauZSrc * X; i += 4) {
            const uint32_t w[8] = {__float_as_uint(vr[i]),     __float_as_uint(vi[i]),     __float_as_uint(vr[i + 1]),
                                   __float_as_uint(vi[i + 1]), __float_as_uint(vr[i + 2]), __float_as_uint(vi[i + 2]),
                                   __float_as_uint(vr[i + 3]), __float_as_uint(vi[i + 3])};
            store_sector(zp + i, w);
          }
        } else {
          // kTauZSrc * X consecutive k from a multiple of kTauZSrc * X: inside one k-block
          constexpr int KB = kKBlockBytes / (MODE == MVB_GEMM_TF32_3 ? 4 : 2);
          constexpr int NPL = MODE == MVB_GEMM_BF16_6 ? 6 : 4;
          const int64_t off = panel_off(m, s0 * X, Mpad, KB, NPL);
          const int64_t off2 = panel_off(m, s0 * X + kTauZSrc * X / 2, Mpad, KB, NPL);
          put_split<MODE, kTauZSrc * X>(z, panel_plane_stride(KB), off, off2, 0, vr, zscale);
          put_split<MODE, kTauZSrc * X>(z, panel_plane_stride(KB), off, off2, 1, vi, zscale);
        }
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
      // (k, k + 1), k even: inside one 16-byte chunk of one k-block row
      constexpr int KB = kKBlockBytes / (MODE == MVB_GEMM_TF32_3 ? 4 : 2);
      constexpr int NPL = MODE == MVB_GEMM_BF16_6 ? 6 : 4;
      const int64_t off = panel_off(m, k, Mpad, KB, NPL);
      PanelWriter<MODE>::put(z, panel_plane_stride(KB), off, 0, vr, 2, zscale);
      PanelWriter<MODE>::put(z, panel_plane_stride(KB), off, 1, vi, 2, zscale);
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

// Fused phase + Z writer for nfreq frequencies: freqs_dev == nullptr means one
// frequency, freq; otherwise freqs_dev[0 .. nfreq) on the device, with the
// fluxes sflux_ld floats and the panels z_stride bytes apart.
static int tau_z_impl(const char *who, const double *antpos, int A, double freq, const double *freqs_dev, int nfreq,
                      const double *crd, int64_t ld, const int32_t *n_dev, int64_t nsrc, const float *sflux,
                      int64_t sflux_ld, const int32_t *sidx, const void *beam, int64_t beam_ld, int nbeam,
                      const int32_t *beam_idx, int F, int X, int mode, float zscale, void *z, int64_t z_stride,
                      int64_t Mpad, int64_t Kcap, void *stream) {
  if (A <= 0 || nsrc < 0 || !antpos || !z || !beam || !sflux || (nsrc > 0 && !crd) || (F != 1 && F != 2) ||
      (X != 1 && X != 2) || nbeam <= 0 || beam_ld < nsrc || nfreq <= 0 || nfreq > 65535)
    return fail(MVB_ERR_ARG, "%s: bad arguments", who);
  int rc = check_panel(mode, (int64_t)A * F, Mpad, Kcap, who);
  if (rc) return rc;
  if (round_up(nsrc * X, kKAlign) > Kcap) return fail(MVB_ERR_ARG, "%s: Kcap too small for nsrc * nax", who);
  if (nfreq > 1 && (sflux_ld < nsrc || z_stride < (int64_t)mvb_zpanel_bytes(mode, Mpad, Kcap) || z_stride % 16))
    return fail(MVB_ERR_ARG, "%s: flux rows or panels overlap", who);
  const int64_t s_max = round_up(nsrc * X, kKAlign) / X;
  if (s_max == 0) return MVB_OK;
  dim3 grid((unsigned)ceil_div(s_max, kTauZBlockSrc), (unsigned)ceil_div(A, kTauZAnts), (unsigned)nfreq);
  const bool staged = nbeam * F * X <= kTauZMaxBFX;
  const size_t smem = staged ? (size_t)nbeam * F * X * kTauZRow * sizeof(float2) : 0;
  const double foc = freq * kInvC;
  const float2 *bm = static_cast<const float2 *>(beam);
  cudaStream_t s = as_stream(stream);
#define MVB_TAUZ(M, XX)                                                                                       \
  do {                                                                                                        \
    if (staged)                                                                                               \
      tau_z_kernel<M, XX, 0, true, false><<<grid, kTauZThreads, smem, s>>>(                                   \
          antpos, A, foc, crd, ld, n_dev, nsrc, sflux, sidx, bm, beam_ld, nbeam, beam_idx, F, zscale, z, Mpad, \
          Kcap, nullptr, 0, nullptr, nullptr, freqs_dev, sflux_ld, 0, z_stride);                              \
    else                                                                                                      \
      tau_z_kernel<M, XX, 0, false, false><<<grid, kTauZThreads, 0, s>>>(                                     \
          antpos, A, foc, crd, ld, n_dev, nsrc, sflux, sidx, bm, beam_ld, nbeam, beam_idx, F, zscale, z, Mpad, \
          Kcap, nullptr, 0, nullptr, nullptr, freqs_dev, sflux_ld, 0, z_stride);                              \
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

extern "C" int mvb_tau_z(const double *antpos, int A, double freq, const double *crd, int64_t ld, const int32_t *n_dev,
                         int64_t nsrc, const float *sflux, const int32_t *sidx, const void *beam, int64_t beam_ld,
                         int nbeam, const int32_t *beam_idx, int F, int X, int mode, float zscale, void *z,
                         int64_t Mpad, int64_t Kcap, void *stream) {
  return tau_z_impl("mvb_tau_z", antpos, A, freq, nullptr, 1, crd, ld, n_dev, nsrc, sflux, 0, sidx, beam, beam_ld,
                    nbeam, beam_idx, F, X, mode, zscale, z, 0, Mpad, Kcap, stream);
}

extern "C" int mvb_tau_z_grouped(const double *antpos, int A, const double *freqs, int nfreq, const double *crd,
                                 int64_t ld, const int32_t *n_dev, int64_t nsrc, const float *sflux, int64_t sflux_ld,
                                 const int32_t *sidx, const void *beam, int64_t beam_ld, int nbeam,
                                 const int32_t *beam_idx, int F, int X, int mode, float zscale, void *z,
                                 size_t z_stride, int64_t Mpad, int64_t Kcap, void *stream) {
  if (!freqs || z_stride > (size_t)INT64_MAX) return fail(MVB_ERR_ARG, "mvb_tau_z_grouped: bad arguments");
  return tau_z_impl("mvb_tau_z_grouped", antpos, A, 0.0, freqs, nfreq, crd, ld, n_dev, nsrc, sflux, sflux_ld, sidx,
                    beam, beam_ld, nbeam, beam_idx, F, X, mode, zscale, z, (int64_t)z_stride, Mpad, Kcap, stream);
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

static int tau_z_pol_impl(const char *who, const double *antpos, int A, double freq, const double *freqs_dev,
                          int nfreq, const double *crd, int64_t ld, const int32_t *n_dev, int64_t nsrc,
                          const float *coh, int64_t coh_ld, const int32_t *sidx, const double *rot, const void *beam,
                          int64_t beam_ld, int nbeam, const int32_t *beam_idx, int mode, float zscale, void *z,
                          int64_t z_stride, int64_t Mpad, int64_t Kcap, void *stream) {
  const int F = 2, X = 2;
  if (A <= 0 || nsrc < 0 || !antpos || !z || !beam || !coh || !rot || (nsrc > 0 && !crd) || nbeam <= 0 ||
      beam_ld < nsrc || nfreq <= 0 || nfreq > 65535)
    return fail(MVB_ERR_ARG, "%s: bad arguments", who);
  int rc = check_panel(mode, (int64_t)A * F, Mpad, Kcap, who);
  if (rc) return rc;
  if (round_up(nsrc * X, kKAlign) > Kcap) return fail(MVB_ERR_ARG, "%s: Kcap too small for nsrc * nax", who);
  if (reinterpret_cast<uintptr_t>(coh) % 16 || reinterpret_cast<uintptr_t>(rot) % 16)
    return fail(MVB_ERR_ARG, "%s: coh and rot must be 16-byte aligned", who);
  if (nfreq > 1 && (coh_ld < nsrc || z_stride < (int64_t)mvb_zpanel_bytes(mode, Mpad, Kcap) || z_stride % 16))
    return fail(MVB_ERR_ARG, "%s: coherency rows or panels overlap", who);
  const int64_t s_max = round_up(nsrc * X, kKAlign) / X;
  if (s_max == 0) return MVB_OK;
  dim3 grid((unsigned)ceil_div(s_max, kTauZBlockSrc), (unsigned)ceil_div(A, kTauZAnts), (unsigned)nfreq);
  const bool staged = nbeam * F * X <= kTauZMaxBFX;
  const size_t smem = staged ? (size_t)nbeam * F * X * kTauZRow * sizeof(float2) : 0;
  const double foc = freq * kInvC;
  const float2 *bm = static_cast<const float2 *>(beam);
  const float4 *c4 = reinterpret_cast<const float4 *>(coh);
  const double2 *r2 = reinterpret_cast<const double2 *>(rot);
  cudaStream_t s = as_stream(stream);
#define MVB_TZP(M)                                                                                                \
  do {                                                                                                             \
    if (staged)                                                                                                    \
      tau_z_kernel<M, 2, 0, true, true><<<grid, kTauZThreads, smem, s>>>(antpos, A, foc, crd, ld, n_dev, nsrc,      \
          nullptr, sidx, bm, beam_ld, nbeam, beam_idx, F, zscale, z, Mpad, Kcap, nullptr, 0, c4, r2, freqs_dev, 0,  \
          coh_ld, z_stride);                                                                                       \
    else                                                                                                           \
      tau_z_kernel<M, 2, 0, false, true><<<grid, kTauZThreads, 0, s>>>(antpos, A, foc, crd, ld, n_dev, nsrc,        \
          nullptr, sidx, bm, beam_ld, nbeam, beam_idx, F, zscale, z, Mpad, Kcap, nullptr, 0, c4, r2, freqs_dev, 0,  \
          coh_ld, z_stride);                                                                                       \
  } while (0)
  switch (mode) {
    case MVB_GEMM_BF16_3: MVB_TZP(MVB_GEMM_BF16_3); break;
    case MVB_GEMM_BF16_6: MVB_TZP(MVB_GEMM_BF16_6); break;
    case MVB_GEMM_TF32_3: MVB_TZP(MVB_GEMM_TF32_3); break;
    case MVB_GEMM_F16_3: MVB_TZP(MVB_GEMM_F16_3); break;
    default: MVB_TZP(MVB_Z_C64); break;
  }
#undef MVB_TZP
  return check_launch("tau_z_kernel(pol)");
}

extern "C" int mvb_tau_z_pol(const double *antpos, int A, double freq, const double *crd, int64_t ld,
                             const int32_t *n_dev, int64_t nsrc, const float *coh, const int32_t *sidx,
                             const double *rot, const void *beam, int64_t beam_ld, int nbeam,
                             const int32_t *beam_idx, int mode, float zscale, void *z, int64_t Mpad, int64_t Kcap,
                             void *stream) {
  return tau_z_pol_impl("mvb_tau_z_pol", antpos, A, freq, nullptr, 1, crd, ld, n_dev, nsrc, coh, 0, sidx, rot, beam,
                        beam_ld, nbeam, beam_idx, mode, zscale, z, 0, Mpad, Kcap, stream);
}

extern "C" int mvb_tau_z_pol_grouped(const double *antpos, int A, const double *freqs, int nfreq, const double *crd,
                                     int64_t ld, const int32_t *n_dev, int64_t nsrc, const float *coh, int64_t coh_ld,
                                     const int32_t *sidx, const double *rot, const void *beam, int64_t beam_ld,
                                     int nbeam, const int32_t *beam_idx, int mode, float zscale, void *z,
                                     size_t z_stride, int64_t Mpad, int64_t Kcap, void *stream) {
  if (!freqs || z_stride > (size_t)INT64_MAX) return fail(MVB_ERR_ARG, "mvb_tau_z_pol_grouped: bad arguments");
  return tau_z_pol_impl("mvb_tau_z_pol_grouped", antpos, A, 0.0, freqs, nfreq, crd, ld, n_dev, nsrc, coh, coh_ld,
                        sidx, rot, beam, beam_ld, nbeam, beam_idx, mode, zscale, z, (int64_t)z_stride, Mpad, Kcap,
                        stream);
}

extern "C" int mvb_z_from_exptau(const void *exptau, int e_c128, int64_t e_ld, int A, int64_t nsrc, const float *sflux,
                                 const void *beam, int64_t beam_ld, int nbeam, const int32_t *beam_idx, int F, int X,
                                 int mode, float zscale, void *z, int64_t Mpad, int64_t Kcap, void *stream) {
  if (A <= 0 || nsrc < 0 || !exptau || !z || !beam || !sflux || (F != 1 && F != 2) || (X != 1 && X != 2) ||
      nbeam <= 0 || beam_ld < nsrc || e_ld < nsrc)
    return fail(MVB_ERR_ARG, "mvb_z_from_exptau: bad arguments");
  int rc = check_panel(mode, (int64_t)A * F, Mpad, Kcap, "mvb_z_from_exptau");
  if (rc) return rc;
  if (round_up(nsrc * X, kKAlign) > Kcap) return fail(MVB_ERR_ARG, "mvb_z_from_exptau: Kcap too small");
  const int64_t s_max = round_up(nsrc * X, kKAlign) / X;
  if (s_max == 0) return MVB_OK;
  dim3 grid((unsigned)ceil_div(s_max, kTauZBlockSrc), (unsigned)ceil_div(A, kTauZAnts));
  const bool staged = nbeam * F * X <= kTauZMaxBFX;
  const size_t smem = staged ? (size_t)nbeam * F * X * kTauZRow * sizeof(float2) : 0;
  const float2 *bm = static_cast<const float2 *>(beam);
  cudaStream_t s = as_stream(stream);
#define MVB_ZX(M, XX, E)                                                                                      \
  do {                                                                                                             \
    if (staged)                                                                                                    \
      tau_z_kernel<M, XX, E, true, false><<<grid, kTauZThreads, smem, s>>>(nullptr, A, 0.0, nullptr, 0, nullptr,    \
          nsrc, sflux, nullptr, bm, beam_ld, nbeam, beam_idx, F, zscale, z, Mpad, Kcap, exptau, e_ld);              \
    else                                                                                                           \
      tau_z_kernel<M, XX, E, false, false><<<grid, kTauZThreads, 0, s>>>(nullptr, A, 0.0, nullptr, 0, nullptr,      \
          nsrc, sflux, nullptr, bm, beam_ld, nbeam, beam_idx, F, zscale, z, Mpad, Kcap, exptau, e_ld);              \
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

// sqrt(0.5 I) per source and frequency (cpu/cpu.py:188), transposed from the
// caller's (N, Nf) float64 Stokes I to the (Nf, N) float32 rows the Z writers
// read; 32 x 32 tiles through shared memory so both sides are coalesced.
namespace mvb {
__global__ void flux_sqrt_half_kernel(const double *__restrict__ flux, int64_t N, int nf, float *__restrict__ out) {
  __shared__ float tile[32][33];
  const int64_t s0 = (int64_t)blockIdx.x * 32;
  const int f0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int64_t s = s0 + r;
    const int f = f0 + threadIdx.x;
    if (s < N && f < nf) tile[r][threadIdx.x] = (float)sqrt(0.5 * flux[s * nf + f]);
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int f = f0 + r;
    const int64_t s = s0 + threadIdx.x;
    if (s < N && f < nf) out[(int64_t)f * N + s] = tile[threadIdx.x][r];
  }
}
}  // namespace mvb

extern "C" int mvb_flux_sqrt_half(const double *flux, int64_t N, int nf, float *sflux, void *stream) {
  if (N < 0 || nf <= 0 || (N > 0 && (!flux || !sflux))) return fail(MVB_ERR_ARG, "mvb_flux_sqrt_half: bad arguments");
  if (N == 0) return MVB_OK;
  if (ceil_div(N, 32) > 0x7fffffff || ceil_div(nf, 32) > 65535)
    return fail(MVB_ERR_ARG, "mvb_flux_sqrt_half: too many sources or frequencies");
  dim3 grid((unsigned)ceil_div(N, 32), (unsigned)ceil_div(nf, 32));
  flux_sqrt_half_kernel<<<grid, dim3(32, 8), 0, as_stream(stream)>>>(flux, N, nf, sflux);
  return check_launch("flux_sqrt_half_kernel");
}

// A8: per-pair source sums for an explicit antenna-pair list.
//
// Reference: gpu/matprod.py:66-98 (GPUVectorDot: one cuBLAS complex_matmul per
// pair per time and chunk), cpu/matprod.py:35-53 (CPUVectorDot:
// out[i] = z[aj] . z[ai]^H, i.e. out[i, p, q] = sum_k Z[aj*F+p, k] conj(Z[ai*F+q, k])).
//
// Two forms:
// * mvb_vecdot: one warp per (k-slice, pair), pairs fastest so concurrently
//   running warps read the same Z columns from L2.  Lanes stride over k with
//   FP32 FMA partial sums (coalesced 256-byte row reads), the warp reduces in
//   FP64 and the slices are summed in FP64 in a fixed order by a second kernel.
//   Any array size; each pair reads both antennas' rows through L2.
// * mvb_vecdot_staged: the panel is read from HBM once.  A persistent CTA per
//   SM stages kb columns of EVERY row in shared memory (one 1-D bulk copy per
//   row, rows padded by 16 bytes) and its 512 threads run up to 3 pair slots
//   each over the stage from there, two columns per 16-byte load.  The slots
//   come from mvb_vecdot_plan, which orders them so that the 8 lanes sharing a
//   shared-memory wavefront read antennas of 8 distinct residues mod 8, which
//   with the padded pitch makes every load conflict-free.  FP32 sums over one
//   stage, FP64 over the k-slice, FP64 slice sums in a fixed order.
#include <cudaTypedefs.h>

#include <algorithm>
#include <type_traits>
#include <vector>

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

// 15 compute warps (one bundle per thread) and one copy-issuing warp: 4 warps
// per scheduler, so each thread may hold 128 registers
constexpr int kVdThreads = 480;
constexpr int kVdCtaThreads = kVdThreads + 32;
constexpr int kVdSteps = 3;               // pairs of a bundle, all sharing its antenna i
constexpr int kVdSmemBytes = 220 * 1024;  // the stages of kb columns x all rows
constexpr int kVdMaxStages = 4;
constexpr int kVdClasses = 8;             // lanes served by one 128-byte shared-memory wavefront
constexpr int kVdBundleInts = 8;          // {i, j[3], pair[3], flip bits}
constexpr int kVdSplitExtra = 31;         // extra k-slices the planner may add to fill the SMs
constexpr int kVdSliceMax = 1024;         // longest k-slice: FP32 sums over at most 1,024 columns
constexpr uint64_t kVdDrainNs = 200000000ull;  // 0.2 s: limit of the in-flight wait on abort

// Splits K_valid into nsplit k-slices of kc columns (a multiple of 16, at most
// kmax) so that nsplit * ngroups units fill whole waves of nsm CTAs as evenly
// as possible: nsplit from ceil(K / kmax) to 31 more, a candidate replacing the
// best only when 1e-3 more efficient (ties keep fewer slices).  Evaluated
// identically by the product and its reduction.
__host__ __device__ inline void vd_plan(int64_t kvalid, int ngroups, int kmax, int nsm, int64_t &nsplit,
                                        int64_t &kc) {
  nsplit = 0;
  kc = kmax;
  if (kvalid <= 0) return;
  const int64_t nmin = (kvalid + kmax - 1) / kmax;
  double best = -1.0;
  for (int64_t n = nmin; n <= nmin + kVdSplitExtra; ++n) {
    const int64_t c = ((kvalid + n - 1) / n + 15) / 16 * 16;
    const int64_t ne = (kvalid + c - 1) / c;
    const int64_t units = ne * ngroups;
    const int64_t waves = (units + nsm - 1) / nsm;
    const double eff = (double)units / (double)(waves * nsm);
    if (eff > best + 1e-3) {
      best = eff;
      nsplit = ne;
      kc = c;
    }
    if (c <= 16) break;
  }
}

// 2-D tiled bulk-tensor load (no multicast) of a box at (x, y) into shared memory.
__device__ __forceinline__ void tma_load_2d(void *smem_dst, const CUtensorMap *map, int x, int y, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
          "r"(smem_u32(smem_dst)),
      "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// Units are (k-slice, bundle group); groups fastest so the CTAs of one slice
// read its columns from L2 together, and rotating with the slice so that a
// CTA's units cycle through the groups.  Compute thread t of a unit runs bundle
// s0 + t: the lane class t mod 8 matches the plan's order.  A bundle holds up to
// 3 pairs sharing the conjugated antenna i, whose rows are loaded once per
// column pair for all three.
//
// The copy warp stages the unit's columns kb at a time, NS stages in flight:
// nbox bulk-tensor loads of box_rows rows x kb columns (8 kb bytes, swizzled in
// 16-byte units by the 8 kb-byte swizzle mode) complete on the stage's full
// barrier; each compute warp releases a stage on its empty barrier.  In the
// swizzled layout the 16-byte unit u of a 128-byte row r sits in bank group
// u ^ (r mod 8) (64- and 32-byte rows share a 128-byte line two or four to a
// line, with the XOR taken from the line index), so 8 rows of distinct residues
// mod 8 never share a bank group.  A thread
// loads 16 bytes = two columns of one row.  For F = 2 the rows of antenna a are
// 2a and 2a + 1; the thread reads row 2a + ba first (ba = bit 2 of a), then
// row 2a + 1 - ba: 8 antennas of distinct residues mod 8 give rows of distinct
// residues mod 8 both times, so every load is conflict-free.  The feed order of
// each bundle step's four sums is thus permuted by (bj, bi); the reduction
// undoes it.  Every wait is bounded: one that runs out sets MVB_DEV_TIMEOUT,
// the CTA stops, and the copy warp waits (bounded) for its copies in flight.
template <int F>
__global__ void __launch_bounds__(kVdCtaThreads, 1)
    vecdot_staged_kernel(const __grid_constant__ CUtensorMap tmap, int64_t Kcap, const int32_t *__restrict__ n_dev,
                         int64_t n_host, int kmul, int nant, const int4 *__restrict__ bundles, int nbundles,
                         int group_size, int ngroups, int kb, int nstage, int box_rows, int nbox, int kmax,
                         double *__restrict__ part, int32_t *__restrict__ status, uint64_t wait_ns) {
  extern __shared__ uint8_t vd_raw[];
  __shared__ __align__(8) uint64_t full_bar[kVdMaxStages], empty_bar[kVdMaxStages];
  __shared__ volatile int abort_flag;
  constexpr int E = 2 * F * F;  // real values per pair
  constexpr int S = kVdSteps;
  uint8_t *stage0 = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(vd_raw) + 1023) & ~uintptr_t(1023));
  const int rowbytes = kb * 8;
  const int stage_bytes = nbox * box_rows * rowbytes;  // a multiple of 1024
  const int swz = kb / 2 - 1;                          // the swizzle's row-bit mask (7, 3 or 1)
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int64_t kvalid = vd_valid_k(n_dev, n_host, kmul, Kcap);
  int64_t nsplit, kc;
  vd_plan(kvalid, ngroups, kmax, gridDim.x, nsplit, kc);
  const int64_t nunits = nsplit * ngroups;
  if (t == 0) {
    for (int b = 0; b < nstage; ++b) {
      mbar_init(&full_bar[b], 1);
      mbar_init(&empty_bar[b], kVdThreads / 32);
    }
    abort_flag = 0;
    fence_mbar_init();
  }
  __syncthreads();

  if (warp == kVdThreads / 32) {
    // ---------------- copy warp ----------------
    if (lane != 0) return;
    int64_t g = 0;  // stages issued
    uint32_t empty_ph = 0;
    for (int64_t u = blockIdx.x; u < nunits && !abort_flag; u += gridDim.x) {
      const int64_t slice = u / ngroups;
      const int64_t k0 = slice * kc, k1 = min(k0 + kc, kvalid);
      const int nst = (int)((k1 - k0 + kb - 1) / kb);
      for (int st = 0; st < nst && !abort_flag; ++st, ++g) {
        const int b = (int)(g % nstage);
        if (!mbar_wait(&empty_bar[b], ((empty_ph >> b) & 1u) ^ 1u, wait_ns)) {
          if (status) atomicOr(status, MVB_DEV_TIMEOUT);
          abort_flag = 1;
          break;
        }
        empty_ph ^= 1u << b;
        mbar_arrive_expect_tx(&full_bar[b], (uint32_t)stage_bytes);
        const int x = (int)(2 * (k0 + (int64_t)st * kb));  // float column of the box
        for (int q = 0; q < nbox; ++q)
          tma_load_2d(stage0 + (size_t)b * stage_bytes + (size_t)q * box_rows * rowbytes, &tmap, x, q * box_rows,
                      &full_bar[b]);
      }
    }
    if (abort_flag) {
      // copies in flight land in this CTA's shared memory: wait (bounded) for the
      // last stage issued into each buffer
      for (int64_t x = g - nstage; x < g; ++x)
        if (x >= 0) mbar_wait(&full_bar[x % nstage], (uint32_t)((x / nstage) & 1), kVdDrainNs);
    }
    return;
  }

  // ---------------- compute warps ----------------
  // Row r of a stage starts at r rowbytes in a 1024-aligned buffer, so the
  // swizzled offset of its 16-byte unit holding columns (c, c + 1) is
  // (r rowbytes + m_r) ^ (8 c), m_r < rowbytes the row's swizzle mask: each row
  // read is kept as that one offset.
  int64_t g = 0;  // stages consumed
  for (int64_t u = blockIdx.x; u < nunits; u += gridDim.x) {
    const int64_t slice = u / ngroups;
    const int s0 = (int)((u % ngroups + slice) % ngroups) * group_size;
    const bool live = t < min(group_size, nbundles - s0);  // uniform per warp
    const int64_t k0 = slice * kc, k1 = min(k0 + kc, kvalid);
    // rows read: i's first row (F i + bi) then its other row; likewise each j
    uint32_t ri[F], rj[S][F];
#pragma unroll
    for (int x = 0; x < F; ++x) {
      ri[x] = 0;
#pragma unroll
      for (int q = 0; q < S; ++q) rj[q][x] = 0;
    }
    if (live) {
      const int4 lo = bundles[2 * (s0 + t)];
      const int js[S] = {lo.y, lo.z, lo.w};
      // a plan from mvb_vecdot_plan keeps every antenna in range; clamp anyway
      auto rows = [&](int a, uint32_t (&r)[F]) {
        a = min(max(a, 0), nant - 1);
        const int ba = F == 2 ? (a >> 2) & 1 : 0;
#pragma unroll
        for (int x = 0; x < F; ++x) {
          const uint32_t off = (uint32_t)((F * a + (x ^ ba)) * rowbytes);
          r[x] = off + ((((off >> 7) & swz)) << 4);  // row offset with its swizzle mask
        }
      };
      rows(lo.x, ri);
#pragma unroll
      for (int q = 0; q < S; ++q) rows(js[q], rj[q]);
    }
    // FP32 sums over 16 columns (acc1) and over the k-slice (acc2, at most
    // kVdSliceMax columns), FP64 across slices in the reduction
    float acc2[S][E], acc1[S][E];
#pragma unroll
    for (int q = 0; q < S; ++q)
#pragma unroll
      for (int e = 0; e < E; ++e) acc2[q][e] = acc1[q][e] = 0.f;

    const int nst = (int)((k1 - k0 + kb - 1) / kb);
    const int per16 = 16 / kb;  // stages per 16-column block
    bool stop = false;
    for (int st = 0; st < nst; ++st, ++g) {
      const int b = (int)(g % nstage);
      if (abort_flag || !mbar_wait(&full_bar[b], (uint32_t)((g / nstage) & 1), wait_ns)) {
        if (lane == 0 && status && !abort_flag) atomicOr(status, MVB_DEV_TIMEOUT);
        abort_flag = 1;
        stop = true;
        break;
      }
      const uint8_t *buf = stage0 + (size_t)b * stage_bytes;
      // columns of this stage inside [k0, k1): all but the kvalid tail
      const int ncols = (int)min((int64_t)kb, k1 - (k0 + (int64_t)st * kb));
      // acc[y][x] += Zj[y] conj(Zi[x]): y, x the feeds in load order;
      // H = 4 (columns c, c + 1) or 2 (the odd last column)
      auto step = [&](uint32_t c8, auto hw) {
        constexpr int H = decltype(hw)::value;
        float vi[F][H];
#pragma unroll
        for (int x = 0; x < F; ++x) {
          const uint8_t *ad = buf + (ri[x] ^ c8);
          if constexpr (H == 4) {
            const float4 v = *reinterpret_cast<const float4 *>(ad);
            vi[x][0] = v.x, vi[x][1] = v.y, vi[x][2] = v.z, vi[x][3] = v.w;
          } else {
            const float2 v = *reinterpret_cast<const float2 *>(ad);
            vi[x][0] = v.x, vi[x][1] = v.y;
          }
        }
#pragma unroll
        for (int q = 0; q < S; ++q) {
          float vj[F][H];
#pragma unroll
          for (int y = 0; y < F; ++y) {
            const uint8_t *ad = buf + (rj[q][y] ^ c8);
            if constexpr (H == 4) {
              const float4 v = *reinterpret_cast<const float4 *>(ad);
              vj[y][0] = v.x, vj[y][1] = v.y, vj[y][2] = v.z, vj[y][3] = v.w;
            } else {
              const float2 v = *reinterpret_cast<const float2 *>(ad);
              vj[y][0] = v.x, vj[y][1] = v.y;
            }
          }
#pragma unroll
          for (int y = 0; y < F; ++y)
#pragma unroll
            for (int x = 0; x < F; ++x) {
              float &re = acc1[q][2 * (y * F + x)], &im = acc1[q][2 * (y * F + x) + 1];
#pragma unroll
              for (int h = 0; h < H; h += 2) {
                re = fmaf(vj[y][h], vi[x][h], fmaf(vj[y][h + 1], vi[x][h + 1], re));
                im = fmaf(vj[y][h + 1], vi[x][h], fmaf(-vj[y][h], vi[x][h + 1], im));
              }
            }
        }
      };
      if (live) {
#pragma unroll 1
        for (int c = 0; c + 1 < ncols; c += 2) step((uint32_t)(c * 8), std::integral_constant<int, 4>{});
        if (ncols & 1) step((uint32_t)((ncols - 1) * 8), std::integral_constant<int, 2>{});
        if ((st + 1) % per16 == 0 || st + 1 == nst) {
#pragma unroll
          for (int q = 0; q < S; ++q)
#pragma unroll
            for (int e = 0; e < E; ++e) {
              acc2[q][e] += acc1[q][e];
              acc1[q][e] = 0.f;
            }
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty_bar[b]);  // this warp is done with the stage
    }
    if (stop) break;
    if (live) {
#pragma unroll
      for (int q = 0; q < S; ++q) {
        double2 *o = reinterpret_cast<double2 *>(part + (((size_t)slice * nbundles + s0 + t) * S + q) * E);
#pragma unroll
        for (int e = 0; e < E; e += 2) o[e / 2] = make_double2(acc2[q][e], acc2[q][e + 1]);
      }
    }
  }
}

// out[pair] (+)= sum over k-slices of its bundle step's partials: one warp per
// output element, lane l summing slices l, l + 32, ... in FP64, then a fixed
// shuffle tree (the same order every run).  The step's sums are held as
// acc[y][x] with y = p ^ bj, x = q ^ bi (feed order of the staged loads, F = 2);
// a flipped step (i = aj, j = ai) holds conj of the transposed feed block.
template <typename OT, int F>
__global__ void vecdot_bundles_reduce_kernel(const double *__restrict__ part, const int4 *__restrict__ bundles,
                                             int nbundles, int nant, int64_t Kcap, const int32_t *__restrict__ n_dev,
                                             int64_t n_host, int kmul, int ngroups, int kmax, int nsm,
                                             int64_t npairs, void *__restrict__ out, int accumulate) {
  constexpr int E = 2 * F * F;
  constexpr int S = kVdSteps;
  const int lane = threadIdx.x & 31;
  const int64_t kvalid = vd_valid_k(n_dev, n_host, kmul, Kcap);
  int64_t nslices, kc;
  vd_plan(kvalid, ngroups, kmax, nsm, nslices, kc);
  const int64_t total = (int64_t)nbundles * S * F * F;
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t x = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; x < total; x += nwarps) {
    const int pq = (int)(x % (F * F));
    const int64_t bs = x / (F * F);  // bundle * S + step
    const int b = (int)(bs / S), q0 = (int)(bs % S);
    const int4 lo = bundles[2 * b], hi = bundles[2 * b + 1];
    const int js[S] = {lo.y, lo.z, lo.w}, ps[S] = {hi.x, hi.y, hi.z};
    const int pair = ps[q0];
    if (pair < 0 || pair >= npairs) continue;  // a filler step (uniform over the warp)
    const int i = min(max(lo.x, 0), nant - 1), j = min(max(js[q0], 0), nant - 1);
    int p = pq / F, q = pq % F;  // acc[p][q] = sum Z[j, p] conj(Z[i, q])
    const int held = F == 2 ? (p ^ ((j >> 2) & 1)) * F + (q ^ ((i >> 2) & 1)) : 0;
    double re = 0.0, im = 0.0;
    for (int64_t c = lane; c < nslices; c += 32) {
      const double2 v = *reinterpret_cast<const double2 *>(part + ((size_t)c * nbundles * S + bs) * E + 2 * held);
      re += v.x;
      im += v.y;
    }
    for (int o = 16; o > 0; o >>= 1) {
      re += __shfl_xor_sync(0xffffffffu, re, o);
      im += __shfl_xor_sync(0xffffffffu, im, o);
    }
    if (lane != 0) continue;
    if ((hi.w >> q0) & 1) {  // out[q][p] = conj(acc[p][q])
      const int tmp = p;
      p = q;
      q = tmp;
      im = -im;
    }
    if (i == j && p == q) im = 0.0;  // one-feed autos are real
    OT *o = static_cast<OT *>(out) + (int64_t)pair * F * F + p * F + q;
    if (accumulate) {
      o->x += re;
      o->y += im;
    } else {
      o->x = re;
      o->y = im;
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

// ---------------------------------------------------------------------------
// staged form: plan (host) and launch
// ---------------------------------------------------------------------------

extern "C" size_t mvb_vecdot_plan_bytes(int64_t npairs, int nfeed) {
  if (npairs < 0 || (nfeed != 1 && nfeed != 2)) return 0;
  // each step of a phase places at least one pair (the lane holding the antenna
  // with the most pairs left always has a partner class), so a phase of 8
  // bundles places 3 while 3 are left: at most npairs / 3 + 1 phases, plus
  // fillers to whole warps
  return (size_t)(kVdClasses * (npairs / kVdSteps + 2) + 32) * kVdBundleInts * sizeof(int32_t);
}

namespace {
// Largest matching of 8 lanes to 8 partner classes (lane l may take class c
// when bit c of adj[l] is set), by augmenting paths.
struct ClassMatching {
  uint8_t adj[kVdClasses];
  int owner[kVdClasses], lane_cls[kVdClasses];
  bool augment(int l, uint8_t &seen) {
    for (int c = 0; c < kVdClasses; ++c) {
      if (!((adj[l] >> c) & 1) || ((seen >> c) & 1)) continue;
      seen |= (uint8_t)(1u << c);
      if (owner[c] < 0 || augment(owner[c], seen)) {
        owner[c] = l;
        lane_cls[l] = c;
        return true;
      }
    }
    return false;
  }
  void run() {
    for (int c = 0; c < kVdClasses; ++c) owner[c] = lane_cls[c] = -1;
    for (int l = 0; l < kVdClasses; ++l) {
      uint8_t seen = 0;
      augment(l, seen);
    }
  }
};
}  // namespace

// Bundles for mvb_vecdot_staged, 8 int32 each: {i, j0, j1, j2, pair0, pair1,
// pair2, flip bits}.  Phases of 8 bundles are built greedily: lane c holds the
// antenna of residue class c (mod 8) with the most pairs left, which becomes
// the conjugated side i of up to 3 of its pairs; at each of the 3 steps the
// lanes are matched to distinct residue classes of the partner antenna j (a
// maximum bipartite matching; within the class the partner with the fewest
// pairs left is taken).  A pair (ai, aj) taken by lane aj is flipped (i = aj,
// j = ai).  Lanes and steps left empty get fillers (pair -1) on unused
// classes, so that the 8 lanes of a phase always read 8 distinct residues.
// Deterministic for a given list.
extern "C" int mvb_vecdot_plan(const int32_t *pairs, int64_t npairs, int nant, int nfeed, void *plan,
                               size_t plan_bytes, int64_t *nbundles) {
  if ((npairs > 0 && !pairs) || npairs < 0 || nant <= 0 || (nfeed != 1 && nfeed != 2) || !plan || !nbundles)
    return fail(MVB_ERR_ARG, "mvb_vecdot_plan: bad arguments");
  if (plan_bytes < mvb_vecdot_plan_bytes(npairs, nfeed)) return fail(MVB_ERR_ARG, "mvb_vecdot_plan: plan too small");
  if (npairs > (int64_t)1 << 24) return fail(MVB_ERR_ARG, "mvb_vecdot_plan: more than 2^24 pairs");
  for (int64_t k = 0; k < npairs; ++k)
    if (pairs[2 * k] < 0 || pairs[2 * k] >= nant || pairs[2 * k + 1] < 0 || pairs[2 * k + 1] >= nant)
      return fail(MVB_ERR_ARG, "mvb_vecdot_plan: pair %lld names an antenna outside [0, %d)", (long long)k, nant);
  *nbundles = 0;
  if (npairs == 0) return MVB_OK;
  constexpr int C = kVdClasses, S = kVdSteps;
  // inc[a * C + c]: pairs of antenna a whose partner has residue c (taken ones removed lazily)
  std::vector<std::vector<int32_t>> inc((size_t)nant * C);
  std::vector<int64_t> left_of(nant, 0);
  for (int64_t k = 0; k < npairs; ++k) {
    const int a = pairs[2 * k], b = pairs[2 * k + 1];
    inc[(size_t)a * C + b % C].push_back((int32_t)k);
    ++left_of[a];
    if (b != a) {
      inc[(size_t)b * C + a % C].push_back((int32_t)k);
      ++left_of[b];
    }
  }
  std::vector<uint8_t> taken(npairs, 0);
  auto partner = [&](int32_t k, int a) { return pairs[2 * k] == a ? pairs[2 * k + 1] : pairs[2 * k]; };
  auto live = [&](size_t list) {  // drop taken pairs; true if any is left
    std::vector<int32_t> &v = inc[list];
    size_t w = 0;
    for (size_t r = 0; r < v.size(); ++r)
      if (!taken[v[r]]) v[w++] = v[r];
    v.resize(w);
    return w > 0;
  };
  const int64_t cap = (int64_t)(plan_bytes / (kVdBundleInts * sizeof(int32_t)));
  int32_t *out = static_cast<int32_t *>(plan);
  int64_t left = npairs, nb = 0;
  while (left > 0 || nb % 32) {
    if (nb + C > cap) return fail(MVB_ERR_ARG, "mvb_vecdot_plan: plan too small");
    int ant[C];
    for (int c = 0; c < C; ++c) {
      ant[c] = -1;
      for (int a = c; a < nant; a += C)
        if (left_of[a] > 0 && (ant[c] < 0 || left_of[a] > left_of[ant[c]])) ant[c] = a;
    }
    int js[C][S], ps[C][S];
    uint32_t flips[C] = {};
    for (int s = 0; s < S; ++s) {
      ClassMatching mt;
      for (int l = 0; l < C; ++l) {
        mt.adj[l] = 0;
        if (ant[l] >= 0)
          for (int c = 0; c < C; ++c)
            if (live((size_t)ant[l] * C + c)) mt.adj[l] |= (uint8_t)(1u << c);
      }
      mt.run();
      uint8_t used = 0;
      for (int l = 0; l < C; ++l) {
        js[l][s] = -1;
        ps[l][s] = -1;
        const int c = mt.lane_cls[l];
        if (c < 0 || !live((size_t)ant[l] * C + c)) continue;  // unmatched, or the pair went to another lane
        int32_t best = -1;
        for (int32_t k : inc[(size_t)ant[l] * C + c])
          if (best < 0 || left_of[partner(k, ant[l])] < left_of[partner(best, ant[l])]) best = k;
        const int a = ant[l], x = partner(best, a);
        taken[best] = 1;
        --left;
        --left_of[a];
        if (x != a) --left_of[x];
        js[l][s] = x;
        ps[l][s] = best;
        if (pairs[2 * best] != a) flips[l] |= 1u << s;  // a is aj: i = aj, j = ai
        used |= (uint8_t)(1u << c);
      }
      int next = 0;  // fillers take the unused classes in order
      for (int l = 0; l < C; ++l) {
        if (ps[l][s] >= 0) continue;
        while (next < C && ((used >> next) & 1)) ++next;
        const int c = next < C ? next++ : 0;
        js[l][s] = c < nant ? c : 0;
      }
    }
    for (int l = 0; l < C; ++l) {
      int32_t *bd = out + (nb + l) * kVdBundleInts;
      bd[0] = ant[l] >= 0 ? ant[l] : (l < nant ? l : 0);
      for (int s = 0; s < S; ++s) {
        bd[1 + s] = js[l][s];
        bd[4 + s] = ps[l][s];
      }
      bd[7] = (int32_t)flips[l];
    }
    nb += C;
  }
  *nbundles = nb;
  return MVB_OK;
}

// Shared-memory stages of the staged kernel for P rows: kb columns of 8 kb
// bytes per row, the widest of which two fit (up to four stages; measured on
// 700 rows: 16 columns in two stages 5.6 ms, 8 columns in four 10.0 ms), as
// nbox boxes of box_rows rows, each box a whole number of 1024-byte blocks so
// that every box starts on a swizzle-pattern boundary.
struct VdStages {
  int kb = 0, nstage = 0, box_rows = 0, nbox = 0, stage_bytes = 0;
};
static VdStages vd_stages(int64_t P) {
  VdStages v;
  if (P <= 0) return v;
  for (int kb = 16; kb >= 4; kb /= 2) {
    const int nbox = (int)ceil_div(P, 256);
    const int box_rows = (int)round_up(ceil_div(P, nbox), 1024 / (kb * 8));
    const int64_t bytes = (int64_t)nbox * box_rows * kb * 8;
    const int64_t n = (kVdSmemBytes - 1024) / bytes;
    if (n >= 2) {
      v.kb = kb;
      v.nstage = (int)std::min<int64_t>(n, kVdMaxStages);
      v.box_rows = box_rows;
      v.nbox = nbox;
      v.stage_bytes = (int)bytes;
      return v;
    }
  }
  return v;
}

extern "C" int mvb_vecdot_stage_columns(int nant, int nfeed) {
  if (nant <= 0 || (nfeed != 1 && nfeed != 2)) return 0;
  return vd_stages((int64_t)nant * nfeed).kb;
}

extern "C" size_t mvb_vecdot_staged_ws_bytes(int64_t nbundles, int nfeed, int64_t Kcap, int k_chunk) {
  if (nbundles <= 0 || k_chunk <= 0 || Kcap <= 0 || (nfeed != 1 && nfeed != 2)) return 8;
  // the planner may use up to kVdSplitExtra slices beyond ceil(K / min(k_chunk, kVdSliceMax))
  return (size_t)(ceil_div(Kcap, std::min(k_chunk, kVdSliceMax)) + kVdSplitExtra) * nbundles * kVdSteps * 2 * nfeed *
         nfeed * sizeof(double);
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link to libcuda).
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

extern "C" int mvb_vecdot_staged(const void *z, int64_t Kcap, const int32_t *n_dev, int64_t n_host, int kmul,
                                 int nfeed, int nant, const void *plan, int64_t nbundles, int64_t npairs, int k_chunk,
                                 void *ws, size_t ws_bytes, void *out, int out_c128, int accumulate, int32_t *status,
                                 void *stream) {
  if (!z || !ws || !out || Kcap <= 0 || Kcap % 16 || Kcap > ((int64_t)1 << 30) || (nfeed != 1 && nfeed != 2) ||
      nant <= 0 || nbundles < 0 || npairs < 0 || (nbundles > 0 && !plan) || nbundles % 32 ||
      nbundles > ((int64_t)1 << 28) || k_chunk <= 0 || k_chunk % 16 || kmul <= 0 || n_host < 0 ||
      (!n_dev && n_host * kmul > Kcap) || reinterpret_cast<uintptr_t>(z) % 16 ||
      reinterpret_cast<uintptr_t>(plan) % 16)
    return fail(MVB_ERR_ARG, "mvb_vecdot_staged: bad arguments");
  const VdStages sg = vd_stages((int64_t)nant * nfeed);
  if (sg.kb == 0) return fail(MVB_ERR_UNSUPPORTED, "mvb_vecdot_staged: %d x %d rows do not fit the stages", nant, nfeed);
  if (ws_bytes < mvb_vecdot_staged_ws_bytes(nbundles, nfeed, Kcap, k_chunk))
    return fail(MVB_ERR_ARG, "mvb_vecdot_staged: workspace too small");
  if (npairs == 0 || nbundles == 0) return MVB_OK;
  PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
  if (!encode) return fail(MVB_ERR_CUDA, "mvb_vecdot_staged: cuTensorMapEncodeTiled unavailable");
  // the panel as (rows, 2 Kcap floats); boxes of box_rows rows x 2 kb floats
  CUtensorMap tmap;
  const cuuint64_t gdim[2] = {(cuuint64_t)(2 * Kcap), (cuuint64_t)nant * nfeed};
  const cuuint64_t gstride[1] = {(cuuint64_t)Kcap * 8};
  const cuuint32_t box[2] = {(cuuint32_t)(2 * sg.kb), (cuuint32_t)sg.box_rows};
  const cuuint32_t estride[2] = {1, 1};
  const CUtensorMapSwizzle swizzle = sg.kb == 16 ? CU_TENSOR_MAP_SWIZZLE_128B
                                                 : (sg.kb == 8 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B);
  CUresult cr = encode(&tmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void *>(z), gdim, gstride, box, estride,
                       CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                       CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (cr != CUDA_SUCCESS) return fail(MVB_ERR_CUDA, "mvb_vecdot_staged: tensor map encode failed (%d)", (int)cr);
  cudaStream_t s = as_stream(stream);
  const int ngroups = (int)ceil_div(nbundles, kVdThreads);
  const int group_size = (int)round_up(ceil_div(nbundles, ngroups), 32);
  const size_t smem = (size_t)sg.nstage * sg.stage_bytes + 1024;
  const int nsm = num_sms();
  const int kmax = std::min(k_chunk, kVdSliceMax);
  const int4 *bd = static_cast<const int4 *>(plan);
  double *part = static_cast<double *>(ws);
  int rc;
  if (nfeed == 2) {
    rc = set_smem_once(reinterpret_cast<const void *>(vecdot_staged_kernel<2>), kVdSmemBytes, 48);
    if (rc) return rc;
    vecdot_staged_kernel<2><<<nsm, kVdCtaThreads, smem, s>>>(tmap, Kcap, n_dev, n_host, kmul, nant, bd,
                                                            (int)nbundles, group_size, ngroups, sg.kb, sg.nstage,
                                                            sg.box_rows, sg.nbox, kmax, part, status, wait_limit_ns());
  } else {
    rc = set_smem_once(reinterpret_cast<const void *>(vecdot_staged_kernel<1>), kVdSmemBytes, 49);
    if (rc) return rc;
    vecdot_staged_kernel<1><<<nsm, kVdCtaThreads, smem, s>>>(tmap, Kcap, n_dev, n_host, kmul, nant, bd,
                                                            (int)nbundles, group_size, ngroups, sg.kb, sg.nstage,
                                                            sg.box_rows, sg.nbox, kmax, part, status, wait_limit_ns());
  }
  rc = check_launch("vecdot_staged_kernel");
  if (rc) return rc;
  const int64_t total = nbundles * kVdSteps * nfeed * nfeed;  // one warp each
  const int rblocks = (int)std::min<int64_t>(ceil_div(total, 8), (int64_t)nsm * 16);
#define MVB_VD_REDUCE(OT, F)                                                                                           \
  vecdot_bundles_reduce_kernel<OT, F><<<rblocks, 256, 0, s>>>(part, bd, (int)nbundles, nant, Kcap, n_dev, n_host, kmul, \
                                                              ngroups, kmax, nsm, npairs, out, accumulate)
  if (out_c128) {
    if (nfeed == 2)
      MVB_VD_REDUCE(double2, 2);
    else
      MVB_VD_REDUCE(double2, 1);
  } else {
    if (nfeed == 2)
      MVB_VD_REDUCE(float2, 2);
    else
      MVB_VD_REDUCE(float2, 1);
  }
#undef MVB_VD_REDUCE
  return check_launch("vecdot_bundles_reduce_kernel");
}

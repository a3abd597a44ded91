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

constexpr int kVdThreads = 512;           // threads of a staged CTA: one bundle each
constexpr int kVdSteps = 3;               // pairs of a bundle, all sharing its antenna i
constexpr int kVdSmemBytes = 224 * 1024;  // two stages of kb columns x all rows
constexpr int kVdClasses = 8;             // lanes served by one 128-byte shared-memory wavefront
constexpr int kVdBundleInts = 8;          // {i, j[3], pair[3], flip bits}

// a stage row: kb columns of one panel row (8 kb bytes) and 16 bytes of padding,
// so that row r's 16-byte unit u sits in bank group (r + u) mod 8
__host__ __device__ constexpr int vd_pitch(int kb) { return kb * 8 + 16; }

// Units are (k-slice, bundle group), groups fastest so the CTAs of one slice
// read its columns from L2 together.  Thread t of a unit runs bundle s0 + t: the
// lane class t mod 8 matches the plan's order, and a group's bundle count is a
// multiple of 32.  A bundle holds up to 3 pairs that share the conjugated
// antenna i, whose rows are loaded once per column pair for all three.
// The CTA stages the unit's columns kb at a time, two stages in flight: 16-byte
// cp.async copies (two columns of one row each; a warp copies whole 128-byte
// row segments) into rows of pitch 8 kb + 16.  A thread loads 16 bytes = two
// columns of one row at a time.  For F = 2 the rows of antenna a are 2a and
// 2a + 1; the thread reads row 2a + ba first (ba = bit 2 of a), then row
// 2a + 1 - ba: within an 8-lane wavefront the 8 antennas have distinct
// residues mod 8, and so do the rows 2a + ba (and 2a + 1 - ba), so every load
// is conflict-free.  The feed order of each slot's four sums is thus permuted
// by (bj, bi); the reduction undoes it.
__device__ __forceinline__ void cp_async16(void *smem_dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(smem_dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

template <int F>
__global__ void __launch_bounds__(kVdThreads, 1)
    vecdot_staged_kernel(const float2 *__restrict__ z, int64_t Kcap, const int32_t *__restrict__ n_dev,
                         int64_t n_host, int kmul, int nant, const int4 *__restrict__ bundles, int nbundles,
                         int group_size, int ngroups, int kb, int k_chunk, double *__restrict__ part) {
  extern __shared__ __align__(16) uint8_t vd_stage[];
  constexpr int E = 2 * F * F;  // real values per pair
  constexpr int S = kVdSteps;
  const int P = nant * F;       // panel rows staged
  const int pitch = vd_pitch(kb);
  const int stage_bytes = P * pitch;
  const int lg = kb == 16 ? 3 : (kb == 8 ? 2 : 1);  // log2 of the 16-byte copies per row
  const int t = threadIdx.x;
  const int64_t kvalid = vd_valid_k(n_dev, n_host, kmul, Kcap);
  const int64_t nunits = (kvalid + k_chunk - 1) / k_chunk * ngroups;
  for (int64_t u = blockIdx.x; u < nunits; u += gridDim.x) {
    const int64_t slice = u / ngroups;
    // groups rotate with the slice: a CTA's units cycle through the groups, so
    // a smaller last group costs no CTA more than the others
    const int s0 = (int)((u % ngroups + slice) % ngroups) * group_size;
    const bool live = t < min(group_size, nbundles - s0);  // uniform per warp
    const int64_t k0 = slice * k_chunk, k1 = min(k0 + (int64_t)k_chunk, kvalid);
    // row byte offsets of the first row read and steps to the other feed's row
    int oi = 0, di = 0, oj[S], dj[S];
#pragma unroll
    for (int q = 0; q < S; ++q) oj[q] = dj[q] = 0;
    if (live) {
      const int4 lo = bundles[2 * (s0 + t)], hi = bundles[2 * (s0 + t) + 1];
      const int js[S] = {lo.y, lo.z, lo.w};
      // a plan from mvb_vecdot_plan keeps every antenna in range; clamp anyway
      const int i = min(max(lo.x, 0), nant - 1);
      const int bi = F == 2 ? (i >> 2) & 1 : 0;
      oi = (F * i + bi) * pitch;
      di = (1 - 2 * bi) * pitch;
#pragma unroll
      for (int q = 0; q < S; ++q) {
        const int j = min(max(js[q], 0), nant - 1);
        const int bj = F == 2 ? (j >> 2) & 1 : 0;
        oj[q] = (F * j + bj) * pitch;
        dj[q] = (1 - 2 * bj) * pitch;
      }
      (void)hi;
    }
    double acc2[S][E];
#pragma unroll
    for (int q = 0; q < S; ++q)
#pragma unroll
      for (int e = 0; e < E; ++e) acc2[q][e] = 0.0;

    const int nst = (int)((k1 - k0 + kb - 1) / kb);
    auto issue = [&](int st) {
      uint8_t *buf = vd_stage + (size_t)(st & 1) * stage_bytes;
      const float2 *src = z + k0 + (int64_t)st * kb;
      for (int e = t; e < (P << lg); e += kVdThreads) {
        const int m = e >> lg, q = e & ((1 << lg) - 1);
        cp_async16(buf + (size_t)m * pitch + q * 16, src + (int64_t)m * Kcap + 2 * q);
      }
      cp_async_commit();
    };
    issue(0);
    for (int st = 0; st < nst; ++st) {
      if (st + 1 < nst)
        issue(st + 1);  // its buffer was released at the last barrier
      else
        cp_async_commit();  // an empty group: the wait below always leaves one
      cp_async_wait1();
      __syncthreads();
      const uint8_t *buf = vd_stage + (size_t)(st & 1) * stage_bytes;
      // columns of this stage inside [k0, k1): all but the kvalid tail
      const int ncols = (int)min((int64_t)kb, k1 - (k0 + (int64_t)st * kb));
      float acc1[S][E];
#pragma unroll
      for (int q = 0; q < S; ++q)
#pragma unroll
        for (int e = 0; e < E; ++e) acc1[q][e] = 0.f;
      // acc[y][x] += Zj[y] conj(Zi[x]): y, x the feeds in load order (x = 0 the
      // antenna's first row); H = 4 (two columns) or 2 (the odd last column)
      auto step = [&](int c, auto hw) {
        constexpr int H = decltype(hw)::value;
        float vi[F][H];
#pragma unroll
        for (int x = 0; x < F; ++x) {
          const uint8_t *pi = buf + oi + x * di + c * 8;
          if constexpr (H == 4) {
            const float4 a = *reinterpret_cast<const float4 *>(pi);
            vi[x][0] = a.x, vi[x][1] = a.y, vi[x][2] = a.z, vi[x][3] = a.w;
          } else {
            const float2 a = *reinterpret_cast<const float2 *>(pi);
            vi[x][0] = a.x, vi[x][1] = a.y;
          }
        }
#pragma unroll
        for (int q = 0; q < S; ++q) {
          float vj[F][H];
#pragma unroll
          for (int y = 0; y < F; ++y) {
            const uint8_t *pj = buf + oj[q] + y * dj[q] + c * 8;
            if constexpr (H == 4) {
              const float4 w = *reinterpret_cast<const float4 *>(pj);
              vj[y][0] = w.x, vj[y][1] = w.y, vj[y][2] = w.z, vj[y][3] = w.w;
            } else {
              const float2 w = *reinterpret_cast<const float2 *>(pj);
              vj[y][0] = w.x, vj[y][1] = w.y;
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
        for (int c = 0; c + 1 < ncols; c += 2) step(c, std::integral_constant<int, 4>{});
        if (ncols & 1) step(ncols - 1, std::integral_constant<int, 2>{});
#pragma unroll
        for (int q = 0; q < S; ++q)
#pragma unroll
          for (int e = 0; e < E; ++e) acc2[q][e] += (double)acc1[q][e];
      }
      __syncthreads();  // the buffer is refilled two stages on
    }
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

// out[pair] (+)= sum over k-slices of its bundle step's partials, in slice
// order.  The step's sums are held as acc[y][x] with y = p ^ bj, x = q ^ bi
// (feed order of the staged loads, F = 2); a flipped step (i = aj, j = ai)
// holds conj of the transposed feed block.
template <typename OT, int F>
__global__ void vecdot_bundles_reduce_kernel(const double *__restrict__ part, const int4 *__restrict__ bundles,
                                             int nbundles, int nant, int64_t Kcap, const int32_t *__restrict__ n_dev,
                                             int64_t n_host, int kmul, int k_chunk, int64_t npairs,
                                             void *__restrict__ out, int accumulate) {
  constexpr int E = 2 * F * F;
  constexpr int S = kVdSteps;
  const int64_t kvalid = vd_valid_k(n_dev, n_host, kmul, Kcap);
  const int64_t nslices = (kvalid + k_chunk - 1) / k_chunk;
  const int64_t total = (int64_t)nbundles * S * F * F;
  for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < total; x += (int64_t)gridDim.x * blockDim.x) {
    const int pq = (int)(x % (F * F));
    const int64_t bs = x / (F * F);  // bundle * S + step
    const int b = (int)(bs / S), q0 = (int)(bs % S);
    const int4 lo = bundles[2 * b], hi = bundles[2 * b + 1];
    const int js[S] = {lo.y, lo.z, lo.w}, ps[S] = {hi.x, hi.y, hi.z};
    const int pair = ps[q0];
    if (pair < 0 || pair >= npairs) continue;  // a filler step
    const int i = min(max(lo.x, 0), nant - 1), j = min(max(js[q0], 0), nant - 1);
    int p = pq / F, q = pq % F;  // acc[p][q] = sum Z[j, p] conj(Z[i, q])
    const int held = F == 2 ? (p ^ ((j >> 2) & 1)) * F + (q ^ ((i >> 2) & 1)) : 0;
    double re = 0.0, im = 0.0;
    for (int64_t c = 0; c < nslices; ++c) {
      const double *v = part + ((size_t)c * nbundles * S + bs) * E + 2 * held;
      re += v[0];
      im += v[1];
    }
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
  // every phase of 8 bundles places at least one pair; fillers complete warps
  return (size_t)(kVdClasses * npairs + 32) * kVdBundleInts * sizeof(int32_t);
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

extern "C" int mvb_vecdot_stage_columns(int nant, int nfeed) {
  if (nant <= 0 || (nfeed != 1 && nfeed != 2)) return 0;
  for (int kb = 16; kb >= 4; kb /= 2)
    if (2 * (int64_t)nant * nfeed * vd_pitch(kb) <= kVdSmemBytes) return kb;
  return 0;
}

extern "C" size_t mvb_vecdot_staged_ws_bytes(int64_t nbundles, int nfeed, int64_t Kcap, int k_chunk) {
  if (nbundles <= 0 || k_chunk <= 0 || Kcap <= 0 || (nfeed != 1 && nfeed != 2)) return 8;
  return (size_t)ceil_div(Kcap, k_chunk) * nbundles * kVdSteps * 2 * nfeed * nfeed * sizeof(double);
}

extern "C" int mvb_vecdot_staged(const void *z, int64_t Kcap, const int32_t *n_dev, int64_t n_host, int kmul,
                                 int nfeed, int nant, const void *plan, int64_t nbundles, int64_t npairs, int k_chunk,
                                 void *ws, size_t ws_bytes, void *out, int out_c128, int accumulate, void *stream) {
  if (!z || !ws || !out || Kcap <= 0 || Kcap % 16 || (nfeed != 1 && nfeed != 2) || nant <= 0 || nbundles < 0 ||
      npairs < 0 || (nbundles > 0 && !plan) || nbundles % 32 || nbundles > ((int64_t)1 << 28) || k_chunk <= 0 ||
      k_chunk % 16 || kmul <= 0 || n_host < 0 || (!n_dev && n_host * kmul > Kcap) ||
      reinterpret_cast<uintptr_t>(z) % 16 || reinterpret_cast<uintptr_t>(plan) % 16)
    return fail(MVB_ERR_ARG, "mvb_vecdot_staged: bad arguments");
  const int kb = mvb_vecdot_stage_columns(nant, nfeed);
  if (kb == 0) return fail(MVB_ERR_UNSUPPORTED, "mvb_vecdot_staged: %d x %d rows do not fit the stages", nant, nfeed);
  if (ws_bytes < mvb_vecdot_staged_ws_bytes(nbundles, nfeed, Kcap, k_chunk))
    return fail(MVB_ERR_ARG, "mvb_vecdot_staged: workspace too small");
  if (npairs == 0 || nbundles == 0) return MVB_OK;
  cudaStream_t s = as_stream(stream);
  const int ngroups = (int)ceil_div(nbundles, kVdThreads);
  const int group_size = (int)round_up(ceil_div(nbundles, ngroups), 32);
  const size_t smem = (size_t)2 * nant * nfeed * vd_pitch(kb);
  const int64_t max_units = ceil_div(Kcap, k_chunk) * ngroups;
  const int grid = (int)std::min<int64_t>(max_units, num_sms());
  const int4 *bd = static_cast<const int4 *>(plan);
  double *part = static_cast<double *>(ws);
  const float2 *zz = static_cast<const float2 *>(z);
  int rc;
  if (nfeed == 2) {
    rc = set_smem_once(reinterpret_cast<const void *>(vecdot_staged_kernel<2>), kVdSmemBytes, 48);
    if (rc) return rc;
    vecdot_staged_kernel<2><<<grid, kVdThreads, smem, s>>>(zz, Kcap, n_dev, n_host, kmul, nant, bd, (int)nbundles,
                                                          group_size, ngroups, kb, k_chunk, part);
  } else {
    rc = set_smem_once(reinterpret_cast<const void *>(vecdot_staged_kernel<1>), kVdSmemBytes, 49);
    if (rc) return rc;
    vecdot_staged_kernel<1><<<grid, kVdThreads, smem, s>>>(zz, Kcap, n_dev, n_host, kmul, nant, bd, (int)nbundles,
                                                          group_size, ngroups, kb, k_chunk, part);
  }
  rc = check_launch("vecdot_staged_kernel");
  if (rc) return rc;
  const int64_t total = nbundles * kVdSteps * nfeed * nfeed;
  const int rblocks = (int)std::min<int64_t>(ceil_div(total, 256), (int64_t)num_sms() * 8);
#define MVB_VD_REDUCE(OT, F)                                                                                          \
  vecdot_bundles_reduce_kernel<OT, F><<<rblocks, 256, 0, s>>>(part, bd, (int)nbundles, nant, Kcap, n_dev, n_host, kmul, \
                                                              k_chunk, npairs, out, accumulate)
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

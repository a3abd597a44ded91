// A3 / A4: FP64 rotation of source unit vectors to topocentric ENU and the
// strict z > 0 horizon selection with ascending kept indices.
//
// Reference: coordinates.py:91-125 (eci_to_enu_matrix), :174-200
// (point_source_crd_eq), core/coords.py:99-150 (select_chunk).
//
// The rotation evaluates (R[r,0]*x + R[r,1]*y) + R[r,2]*z with every multiply and
// add rounded on its own (__dmul_rn / __dadd_rn forbid FMA contraction), the
// same operation sequence as the FP64 oracle, so the kept set is bit-identical.
//
// Compaction is two wait-free launches over blocks of 1024 sources: a count pass
// (ballot + popc) and a scatter pass in which each block sums the counts of the
// blocks before it, then ranks its own sources with warp ballots.  No block
// waits on another, so there is no inter-block spin.
#include <mutex>

#include "common.cuh"

namespace mvb {

struct Rot3 {
  double r[9];
};

__global__ void rotate_kernel(const double *__restrict__ eci, int64_t n, Rot3 R, double *__restrict__ topo) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double x = eci[i], y = eci[n + i], z = eci[2 * n + i];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      const double a = __dmul_rn(R.r[3 * r + 0], x);
      const double b = __dmul_rn(R.r[3 * r + 1], y);
      const double c = __dmul_rn(R.r[3 * r + 2], z);
      topo[r * n + i] = __dadd_rn(__dadd_rn(a, b), c);
    }
  }
}

constexpr int kCompactThreads = 256;
constexpr int kCompactPerThread = 4;
constexpr int kCompactBlock = kCompactThreads * kCompactPerThread;  // sources per block

__global__ void __launch_bounds__(kCompactThreads) horizon_count_kernel(const double *__restrict__ zrow, int64_t count,
                                                                         int32_t *__restrict__ block_counts) {
  __shared__ int warp_tot[kCompactThreads / 32];
  const int64_t base = (int64_t)blockIdx.x * kCompactBlock;
  int mine = 0;
#pragma unroll
  for (int j = 0; j < kCompactPerThread; ++j) {
    const int64_t i = base + j * kCompactThreads + threadIdx.x;
    mine += (i < count && zrow[i] > 0.0) ? 1 : 0;
  }
  for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, o);
  if ((threadIdx.x & 31) == 0) warp_tot[threadIdx.x >> 5] = mine;
  __syncthreads();
  if (threadIdx.x == 0) {
    int s = 0;
    for (int w = 0; w < kCompactThreads / 32; ++w) s += warp_tot[w];
    block_counts[blockIdx.x] = s;
  }
}

__global__ void __launch_bounds__(kCompactThreads)
    horizon_scatter_kernel(const double *__restrict__ topo, int64_t ld, int64_t c0, int64_t count,
                           const int32_t *__restrict__ block_counts, int nblocks, const double *__restrict__ flux,
                           double *__restrict__ crd_out, int32_t *__restrict__ idx_out, double *__restrict__ flux_out,
                           int32_t *__restrict__ n_out, int64_t cap, int32_t *__restrict__ status) {
  __shared__ long long red_before[kCompactThreads / 32];
  __shared__ long long red_total[kCompactThreads / 32];
  __shared__ int warp_cnt[kCompactThreads / 32];
  __shared__ int warp_off[kCompactThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

  // counts of earlier blocks, and the grand total
  long long before = 0, total = 0;
  for (int b = threadIdx.x; b < nblocks; b += kCompactThreads) {
    const long long c = block_counts[b];
    total += c;
    if (b < (int)blockIdx.x) before += c;
  }
  for (int o = 16; o > 0; o >>= 1) {
    before += __shfl_xor_sync(0xffffffffu, before, o);
    total += __shfl_xor_sync(0xffffffffu, total, o);
  }
  if (lane == 0) {
    red_before[warp] = before;
    red_total[warp] = total;
  }
  __syncthreads();
  before = 0;
  total = 0;
  for (int w = 0; w < kCompactThreads / 32; ++w) {
    before += red_before[w];
    total += red_total[w];
  }

  const double *xr = topo + c0;
  const double *yr = topo + ld + c0;
  const double *zr = topo + 2 * ld + c0;
  const int64_t base = (int64_t)blockIdx.x * kCompactBlock;
  long long run = before;
  if ((int)blockIdx.x < nblocks) {
    for (int j = 0; j < kCompactPerThread; ++j) {
      const int64_t i = base + j * kCompactThreads + threadIdx.x;
      const bool keep = i < count && zr[i] > 0.0;
      const unsigned m = __ballot_sync(0xffffffffu, keep);
      if (lane == 0) warp_cnt[warp] = __popc(m);
      __syncthreads();
      if (threadIdx.x == 0) {
        int s = 0;
        for (int w = 0; w < kCompactThreads / 32; ++w) {
          warp_off[w] = s;
          s += warp_cnt[w];
        }
      }
      __syncthreads();
      if (keep) {
        const long long pos = run + warp_off[warp] + __popc(m & ((1u << lane) - 1u));
        if (pos < cap) {
          crd_out[pos] = xr[i];
          crd_out[cap + pos] = yr[i];
          crd_out[2 * cap + pos] = zr[i];
          idx_out[pos] = (int32_t)(c0 + i);
          if (flux != nullptr) flux_out[pos] = flux[c0 + i];
        }
      }
      run += warp_off[kCompactThreads / 32 - 1] + warp_cnt[kCompactThreads / 32 - 1];
      __syncthreads();
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *n_out = (int32_t)total;
    if (total > cap && status != nullptr) atomicOr(status, MVB_DEV_OVERFLOW);
  }
  // zero the flux tail [total, cap)
  if (flux != nullptr) {
    for (long long i = total + (long long)blockIdx.x * kCompactThreads + threadIdx.x; i < cap;
         i += (long long)gridDim.x * kCompactThreads)
      flux_out[i] = 0.0;
  }
}

// ERFA-style apparent place of each source (cpu/coords.py:118-181): light
// deflection by the Sun (_ld), aberration (_ab), bias-precession-nutation
// (_bpn), in FP64.  The aberration follows the reference expression, whose w2
// term uses the direction already scaled by bm1.
constexpr double kErfaSrs = 1.97412574336e-8;  // Schwarzschild radius of the Sun (au)

struct Astrom {
  double eh[3], em, dlim, v[3], bm1, bpn[9];
};

__global__ void bcrs_kernel(const double *__restrict__ eci, int64_t n, Astrom a, double *__restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double p0 = eci[i], p1 = eci[n + i], p2 = eci[2 * n + i];
    const double e0 = a.eh[0], e1 = a.eh[1], e2 = a.eh[2];
    // light deflection: p += w p x (e x p), w = SRS / em / max(p.(p + e), dlim)
    double qdqpe = p0 * (p0 + e0) + p1 * (p1 + e1) + p2 * (p2 + e2);
    qdqpe = qdqpe < a.dlim ? a.dlim : qdqpe;
    const double w = kErfaSrs / a.em / qdqpe;
    const double q0 = e1 * p2 - e2 * p1, q1 = e2 * p0 - e0 * p2, q2 = e0 * p1 - e1 * p0;  // e x p
    const double r0 = p1 * q2 - p2 * q1, r1 = p2 * q0 - p0 * q2, r2 = p0 * q1 - p1 * q0;  // p x (e x p)
    p0 += w * r0;
    p1 += w * r1;
    p2 += w * r2;
    // aberration
    const double pdv = a.v[0] * p0 + a.v[1] * p1 + a.v[2] * p2;
    const double w1 = 1.0 + pdv / (1.0 + a.bm1);
    const double w2 = kErfaSrs / a.em;
    p0 *= a.bm1;
    p1 *= a.bm1;
    p2 *= a.bm1;
    p0 += a.v[0] * w1 + w2 * (a.v[0] - pdv * p0);
    p1 += a.v[1] * w1 + w2 * (a.v[1] - pdv * p1);
    p2 += a.v[2] * w1 + w2 * (a.v[2] - pdv * p2);
    const double rinv = 1.0 / sqrt(p0 * p0 + p1 * p1 + p2 * p2);
    p0 *= rinv;
    p1 *= rinv;
    p2 *= rinv;
    // bias-precession-nutation
    out[i] = a.bpn[0] * p0 + a.bpn[1] * p1 + a.bpn[2] * p2;
    out[n + i] = a.bpn[3] * p0 + a.bpn[4] * p1 + a.bpn[5] * p2;
    out[2 * n + i] = a.bpn[6] * p0 + a.bpn[7] * p1 + a.bpn[8] * p2;
  }
}

}  // namespace mvb

using namespace mvb;

extern "C" int mvb_rotate(const double *eci, int64_t N, const double *R, double *topo, void *stream) {
  if (N < 0 || (N > 0 && (!eci || !topo)) || !R) return fail(MVB_ERR_ARG, "mvb_rotate: bad arguments");
  if (N == 0) return MVB_OK;
  Rot3 r;
  for (int i = 0; i < 9; ++i) r.r[i] = R[i];
  const int threads = 256;
  const int64_t blocks = std::min<int64_t>(ceil_div(N, threads), (int64_t)num_sms() * 16);
  rotate_kernel<<<(unsigned)blocks, threads, 0, as_stream(stream)>>>(eci, N, r, topo);
  return check_launch("rotate_kernel");
}

extern "C" int mvb_bcrs(const double *eci, int64_t N, const double *astrom, double *bcrs, void *stream) {
  if (N < 0 || !astrom || (N > 0 && (!eci || !bcrs))) return fail(MVB_ERR_ARG, "mvb_bcrs: bad arguments");
  if (N == 0) return MVB_OK;
  Astrom a;
  for (int k = 0; k < 3; ++k) a.eh[k] = astrom[k];
  a.em = astrom[3];
  a.dlim = astrom[4];
  for (int k = 0; k < 3; ++k) a.v[k] = astrom[5 + k];
  a.bm1 = astrom[8];
  for (int k = 0; k < 9; ++k) a.bpn[k] = astrom[9 + k];
  if (!(a.em > 0.0) || !(a.bm1 > 0.0)) return fail(MVB_ERR_ARG, "mvb_bcrs: em and bm1 must be positive");
  const int threads = 256;
  const int64_t blocks = std::min<int64_t>(ceil_div(N, threads), (int64_t)num_sms() * 16);
  bcrs_kernel<<<(unsigned)blocks, threads, 0, as_stream(stream)>>>(eci, N, a, bcrs);
  return check_launch("bcrs_kernel");
}

extern "C" size_t mvb_horizon_ws_bytes(int64_t count) {
  return (size_t)std::max<int64_t>(1, ceil_div(std::max<int64_t>(count, 0), kCompactBlock)) * sizeof(int32_t);
}

extern "C" int mvb_horizon_compact(const double *topo, int64_t ld, int64_t c0, int64_t c1, const double *flux,
                                   double *crd_out, int32_t *idx_out, double *flux_out, int32_t *n_out, int64_t cap,
                                   int32_t *status, void *ws, size_t ws_bytes, void *stream) {
  const int64_t count = c1 - c0;
  if (count < 0 || c0 < 0 || c1 > ld || cap < 0 || !n_out || !ws || (count > 0 && !topo) ||
      (cap > 0 && (!crd_out || !idx_out)) || (flux && cap > 0 && !flux_out))
    return fail(MVB_ERR_ARG, "mvb_horizon_compact: bad arguments");
  if (count > INT32_MAX) return fail(MVB_ERR_ARG, "mvb_horizon_compact: chunk too large");
  if (ws_bytes < mvb_horizon_ws_bytes(count)) return fail(MVB_ERR_ARG, "mvb_horizon_compact: workspace too small");
  const int nblocks = (int)ceil_div(count, kCompactBlock);
  int32_t *counts = static_cast<int32_t *>(ws);
  cudaStream_t s = as_stream(stream);
  if (nblocks > 0) {
    horizon_count_kernel<<<nblocks, kCompactThreads, 0, s>>>(topo + 2 * ld + c0, count, counts);
    int rc = check_launch("horizon_count_kernel");
    if (rc) return rc;
  }
  const int grid = std::max(nblocks, 1);
  horizon_scatter_kernel<<<grid, kCompactThreads, 0, s>>>(topo, ld, c0, count, counts, nblocks, flux, crd_out, idx_out,
                                                         flux_out, n_out, cap, status);
  return check_launch("horizon_scatter_kernel");
}

// ---------------------------------------------------------------------------
// Allocation-free variant of mvb_horizon_compact.
//
// Some callers cannot allocate device memory at the moment they select sources:
// a pipeline that plans all of its device memory once at start-up and forbids
// allocation afterwards (cudaMalloc / cudaFree can synchronise the device and
// stall every other stream), or a host that is handed only a stream and its
// input / output buffers by another library.  For them the per-block counts
// live in this fixed device array instead of a caller workspace.  Every GPU that
// loads the library holds it (16 KB) until the process exits.
// ---------------------------------------------------------------------------
namespace mvb {

constexpr int kStaticCompactBlocks = 4096;  // chunks of up to 4096 x 1024 sources
static __device__ __align__(256) int32_t g_compact_counts[kStaticCompactBlocks];

// Device address of g_compact_counts for the current device, looked up once
// per device (with that device current) and cached for the life of the
// process.  A reset of the device's primary context (cudaDeviceReset) reloads
// the module and invalidates the cached address: a process that resets a
// device must not call mvb_horizon_compact_static on it afterwards.
static int static_counts_ptr(int32_t **out) {
  static int32_t *cache[64] = {};
  static std::mutex mu;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(MVB_ERR_CUDA, "mvb_horizon_compact_static: cudaGetDevice: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= 64) return fail(MVB_ERR_UNSUPPORTED, "mvb_horizon_compact_static: device ordinal %d", dev);
  std::lock_guard<std::mutex> lock(mu);
  if (cache[dev] == nullptr) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_compact_counts);
    if (e != cudaSuccess || p == nullptr)
      return fail(MVB_ERR_CUDA, "mvb_horizon_compact_static: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
    cache[dev] = static_cast<int32_t *>(p);
  }
  *out = cache[dev];
  return MVB_OK;
}

}  // namespace mvb

extern "C" int mvb_horizon_compact_static(const double *topo, int64_t ld, int64_t c0, int64_t c1, const double *flux,
                                          double *crd_out, int32_t *idx_out, double *flux_out, int32_t *n_out,
                                          int64_t cap, int32_t *status, void *stream) {
  const int64_t count = c1 - c0;
  if (count < 0 || c0 < 0 || c1 > ld || cap < 0 || !n_out || (count > 0 && !topo) ||
      (cap > 0 && (!crd_out || !idx_out)) || (flux && cap > 0 && !flux_out))
    return fail(MVB_ERR_ARG, "mvb_horizon_compact_static: bad arguments");
  const int64_t nblocks = ceil_div(count, kCompactBlock);
  if (nblocks > kStaticCompactBlocks)
    return fail(MVB_ERR_ARG,
                "mvb_horizon_compact_static: chunk of %lld sources exceeds the static limit of %lld sources "
                "(use mvb_horizon_compact with a workspace)",
                (long long)count, (long long)kStaticCompactBlocks * kCompactBlock);
  int32_t *counts = nullptr;
  int rc = static_counts_ptr(&counts);
  if (rc) return rc;
  // Every count the scatter pass reads is written by the count pass first, so
  // nothing in the shared array has to start at zero.
  cudaStream_t s = as_stream(stream);
  if (nblocks > 0) {
    horizon_count_kernel<<<(unsigned)nblocks, kCompactThreads, 0, s>>>(topo + 2 * ld + c0, count, counts);
    rc = check_launch("horizon_count_kernel");
    if (rc) return rc;
  }
  const int grid = (int)std::max<int64_t>(nblocks, 1);
  horizon_scatter_kernel<<<grid, kCompactThreads, 0, s>>>(topo, ld, c0, count, counts, (int)nblocks, flux, crd_out,
                                                         idx_out, flux_out, n_out, cap, status);
  return check_launch("horizon_scatter_kernel");
}

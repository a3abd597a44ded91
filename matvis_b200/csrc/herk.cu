// A7: V = conj(Z) Z^T on the 5th-generation tensor cores (tcgen05 + TMEM),
// upper-triangle tiles only, in split precision.
//
// Reference: gpu/matprod.py:31-36 / gpu/_cublas.py:7-65 (one full c/zgemm with
// OP_C, OP_N per time and chunk), cpu/matprod.py:11-32 (z.conj().dot(z.T)),
// core/matprod.py:103-115 (sum over source chunks).
//
// Formulation.  For rows m, n of Z (row = ant * nfeed + feed):
//   Re V[m, n] = sum_k Zr[m,k] Zr[n,k] + Zi[m,k] Zi[n,k]
//   Im V[m, n] = sum_k Zr[m,k] Zi[n,k] - Zi[m,k] Zr[n,k]
// A 128 x 128 complex tile (I, J), I <= J, lives in one 128 x 256 FP32 TMEM
// block D (columns 0..127 real, 128..255 imaginary) filled by three UMMAs per
// k-step and split-term product (pa, pb), issued in this order:
//   D[:,   0:128] += Zi_I^pa . Zi_J^pb^T                  (N = 128)
//   D[:, 128:256] += Zi_I^pa . (-Zr_J^pb)^T               (N = 128, negate-B bit)
//   D[:,   0:256] += Zr_I^pa . [Zr_J^pb ; Zi_J^pb]^T     (N = 256)
// (with the N = 256 product first the whole-slice error measured 3.6e-7
// against 3.0e-7 at the same speed).  A diagonal tile (I = J) drops the
// Zr_I . Zi_I^T half of the last UMMA (N = 128, real half only): its
// imaginary half then holds W = -sum Zi^pa Zr^pb^T, and since the split-term
// products are symmetric under pa <-> pb, Im V = W - W^T, which the reduction
// forms from the partial tile's two triangles.  Three of the four real
// 128 x 128 products on 6 of the 21 tiles of a 700-row panel: 7 % fewer
// tensor-core cycles per slice.
//
// Accuracy.  The tensor core rounds its FP32 accumulator toward zero at every
// UMMA, so a long in-TMEM sum drifts by about one ulp per instruction (3e-5
// relative after 2,048 columns).  Each group of KD k-steps (32-byte column
// blocks; KD = 2 by default, one stage) is therefore accumulated into a FRESH
// TMEM block, products in ascending order of magnitude -- BF16_6 {11, 02, 20, 01,
// 10, 00}, BF16_3 / TF32_3 / F16_3 {01, 10, 00}, each product over all the
// block's k-steps before the next -- so only the final hi x hi UMMAs round at
// full magnitude, and the block is drained by the epilogue warps into FP32
// registers with round-to-nearest adds.  (Issuing the cross terms of both
// k-steps of a stage before its hi x hi products, instead of k-step by k-step,
// measured 3.6e-7 against 5.0e-7 on a whole config-2 slice and a 4 % shorter
// product.)  One
// k-slice (k_chunk columns) of register sums is one partial tile; slices are
// summed in float-float (TwoSum, ~2^-44) and rounded to FP64 by herk_reduce_*.
//
// Schedule.  Work unit u = (panel g, k-slice s, tile t), t fastest so the CTAs
// that run together read the same Z columns (L2 reuse).  A launch covers ngroup
// panels of one shape (the frequencies of a time step, zstride bytes apart)
// that share the column count; with ngroup = 1 it is one product.
// Persistent CTAs (one per SM, 192 KB of shared memory) take units in index
// order from a counter in the workspace (zeroed on the stream before each
// launch), so a CTA that drew cheaper diagonal tiles takes more units: with
// static round-robin the CTAs' loads differed by up to a tile's work (one
// panel of 700 rows: 0.92-0.96 of the mean).  Each unit's sums do not depend
// on which CTA computes it.  Warp roles (576 threads):
//   warp 0 lane 0 : producer; fetches the CTA's next unit index and hands it
//                   to the other roles through a 4-entry shared-memory ring
//                   (full / empty mbarriers); one 1-D bulk copy per operand
//                   per stage: the panel stores each (k-block, row block) as
//                   the stage's shared-memory image (all 2P split/component
//                   planes of 128 rows x 64 bytes, 64-byte swizzled; two
//                   k-steps), so an operand is one contiguous 2P x 8 KB run.  A bulk copy of it
//                   completes in about half the time of the same bytes as tiled
//                   TMA boxes of 64-byte rows, and the three stages in flight no
//                   longer leave the MMA waiting;
//   warp 1        : TMEM owner (512 columns = two k-step blocks); lane 0 issues
//                   the UMMAs and tcgen05.commit's the stage / block barriers;
//   warps 2..17   : epilogue; warp w drains TMEM lane quadrant (w % 4), column
//                   quarter (w - 2) / 4 (64 of the 256 columns), 64 FP32
//                   register sums per thread, and at the end of a unit stores
//                   them coalesced to the workspace [u][256 columns][128 rows].
// K_valid is cut into equal k-slices (multiples of 64 columns, at most k_chunk)
// whose number is chosen on the device, from the device-side source count, to
// fill whole waves of SMs (plan_splits).
// Every mbarrier wait is bounded by wall time (wait_ns, 4 s unless
// mvb_set_wait_limit_ns changed it); on expiry the CTA records MVB_DEV_TIMEOUT
// in the status word, stops issuing work, drains the copies and MMAs it issued
// (each drain wait bounded by kDrainLimitNs), frees TMEM and returns.
#include <algorithm>
#include <atomic>

#include "common.cuh"

namespace mvb {

constexpr int kEpiWarps = 16;
constexpr int kPlanExtra = 31;  // extra k-slices the split planner may add to fill the SMs (one per lane)
constexpr int kHerkThreads = 64 + 32 * kEpiWarps;
constexpr uint64_t kWaitLimitNs = 4000000000ull;   // 4 s: the default limit of a pipeline wait
constexpr uint64_t kDrainLimitNs = 200000000ull;   // 0.2 s
constexpr int kPlaneBytes = 128 * 64;              // one 128-row x 64-byte plane tile (two k-steps)
constexpr int kSmemBudget = 192 * 1024;
constexpr int kUnitRing = 4;       // unit indices the producer may fetch ahead of the MMA and epilogue
constexpr size_t kCounterBytes = 256;  // the launch's unit counter, in the last 16 bytes of the workspace

template <int MODE>
struct HerkCfg {
  static constexpr int P = MODE == MVB_GEMM_BF16_6 ? 3 : 2;
  static constexpr int ES = MODE == MVB_GEMM_TF32_3 ? 4 : 2;
  static constexpr int KSTEP = 32 / ES;  // elements per 32-byte k-step (= UMMA K)
  static constexpr int KB = 64 / ES;     // elements per 64-byte k-block: one stage, two k-steps
  static_assert(KB * ES == kKBlockBytes, "one stage is one k-block of the panel");
  static constexpr int OPER_BYTES = 2 * P * kPlaneBytes;
  static constexpr int STAGE_BYTES = 2 * OPER_BYTES;
  static constexpr int STAGES = kSmemBudget / STAGE_BYTES;
  static_assert(STAGES >= 2, "a drained block of four k-steps holds two stages");
  static constexpr int NPROD = P == 3 ? 6 : 3;
  // UMMA operand format: 0 = F16, 1 = BF16, 2 = TF32
  static constexpr uint32_t FMT = MODE == MVB_GEMM_TF32_3 ? 2u : (MODE == MVB_GEMM_F16_3 ? 0u : 1u);
  static constexpr uint32_t ID256 = umma_idesc(FMT, 256, 0);
  static constexpr uint32_t ID128 = umma_idesc(FMT, 128, 0);
  static constexpr uint32_t ID128N = umma_idesc(FMT, 128, 1);
};

// Split-term products (pa, pb), ascending magnitude 2^-8(pa + pb).
// Tables packed one nibble per product: 6 products pa = 1,0,2,0,1,0 and
// pb = 1,2,0,1,0,0; 3 products pa = 0,1,0 and pb = 1,0,0.
__device__ __forceinline__ void product_terms(int nprod, int q, uint32_t &pa, uint32_t &pb) {
  const uint32_t ta = nprod == 6 ? 0x010201u : 0x010u;
  const uint32_t tb = nprod == 6 ? 0x001021u : 0x001u;
  pa = (ta >> (4 * q)) & 0xFu;
  pb = (tb >> (4 * q)) & 0xFu;
}

// Splits K_valid into nsplit equal slices of kc columns (a multiple of 64, at
// most kmax), choosing nsplit in [ceil(K/kmax), +kPlanExtra] so that
// n_tiles * nsplit work units fill whole waves of nsm SMs as evenly as possible
// (a candidate replaces the best so far only when 1e-3 more efficient, so ties
// keep fewer slices; the scan stops at the first candidate of 64 columns).
// Each lane of a warp evaluates one candidate and the scan runs over the
// shuffled efficiencies, so every warp reaches the same plan in one candidate's
// arithmetic; every lane of the warp must call it.  Used identically by the
// product and its reductions.
__device__ __forceinline__ void plan_splits(int64_t kvalid, int n_tiles, int kmax, int nsm, int &nsplit, int64_t &kc) {
  if (kvalid <= 0) {  // kvalid is uniform over the grid
    nsplit = 0;
    kc = kmax;
    return;
  }
  const int64_t nmin = (kvalid + kmax - 1) / kmax;
  const int64_t n = nmin + (threadIdx.x & 31);
  int64_t c = (kvalid + n - 1) / n;
  c = ((c + 63) / 64) * 64;
  const int64_t ne = (kvalid + c - 1) / c;
  const int64_t units = (int64_t)n_tiles * ne;
  const int64_t waves = (units + nsm - 1) / nsm;
  const double eff = (double)units / (double)(waves * nsm);
  const unsigned stop = __ballot_sync(0xffffffffu, c <= 64);
  double best = -1.0;
  int win = 0;
  for (int l = 0; l <= kPlanExtra; ++l) {
    const double e = __shfl_sync(0xffffffffu, eff, l);
    if (e > best + 1e-3) {
      best = e;
      win = l;
    }
    if ((stop >> l) & 1u) break;
  }
  nsplit = (int)__shfl_sync(0xffffffffu, ne, win);
  kc = __shfl_sync(0xffffffffu, c, win);
}

// Valid K columns: (source count) x (columns per source), clamped to the panel.
__device__ __forceinline__ int64_t valid_k(const int32_t *n_dev, int64_t n_host, int kmul, int64_t Kcap) {
  int64_t n = n_dev ? (int64_t)*n_dev : n_host;
  n = n < 0 ? 0 : n;
  return min(n * kmul, Kcap);
}

__device__ __forceinline__ void decode_tile(int t, int T, int &I, int &J) {
  int i = 0;
  while (t >= T - i) {
    t -= T - i;
    ++i;
  }
  I = i;
  J = i + t;
}

template <int MODE>
__device__ __forceinline__ void umma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  if constexpr (MODE == MVB_GEMM_TF32_3)
    umma_tf32(d, a, b, idesc, acc);
  else
    umma_bf16(d, a, b, idesc, acc);
}

// A launch's work units come either from one panel shape repeated ngroup
// times (the frequencies of a job's time step), or from a table of panels of
// different shapes (the panel groups of several jobs, mvb_herk_batch).  A table
// entry is one panel: its k-slice plan fills waves for plan_tiles tiles and its
// partial tiles sit at index in its group's workspace, so that each group's
// sums equal those of its own grouped launch.
constexpr int kMaxBatchPanels = 32;
struct HerkPanel {
  const uint8_t *panel;
  const int32_t *n_dev;
  float *partials;  // the group's workspace
  int32_t *status;
  int64_t n_host, Kcap;
  int T, kmul, k_chunk, plan_tiles, index;
};
struct HerkTable {
  HerkPanel p[kMaxBatchPanels];
  int n;
};

// KD: k-steps accumulated in one TMEM block before it is drained (1, 2 or 4).
// TABLE: the units come from the table (a batch) instead of one repeated shape.
template <int MODE, int KD, bool TABLE>
__global__ void __launch_bounds__(kHerkThreads, 1)
    herk_kernel(const uint8_t *__restrict__ zpanels, int64_t zstride, int ngroup, int T, int n_tiles,
                const int32_t *__restrict__ n_dev, int64_t n_host, int kmul, int64_t Kcap, int k_chunk, int nsm,
                float *__restrict__ partials, int32_t *__restrict__ status, int *__restrict__ unit_next,
                uint64_t wait_ns, const __grid_constant__ HerkTable table) {
  using C = HerkCfg<MODE>;
  extern __shared__ uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t full_bar[C::STAGES];
  __shared__ __align__(8) uint64_t empty_bar[C::STAGES];
  __shared__ __align__(8) uint64_t dfull_bar[2];
  __shared__ __align__(8) uint64_t dempty_bar[2];
  __shared__ __align__(8) uint64_t drain_bar;
  __shared__ __align__(8) uint64_t ufull_bar[kUnitRing];   // a unit index is in unit_q
  __shared__ __align__(8) uint64_t uempty_bar[kUnitRing];  // every role has read it
  __shared__ int unit_q[kUnitRing];
  __shared__ uint32_t tmem_base_sh;
  __shared__ volatile int abort_flag;

  __shared__ int s_first[kMaxBatchPanels + 1];  // a table's first unit per panel
  __shared__ int s_nsplit[kMaxBatchPanels];
  __shared__ int64_t s_kc[kMaxBatchPanels], s_kvalid[kMaxBatchPanels];

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr bool tabled = TABLE;
  int64_t kvalid = 0, kc = 0;
  int per_panel = 0, n_units;
  if constexpr (tabled) {
    if (warp == 0) {  // every lane plans (plan_splits is warp-wide); lane 0 records
      int acc = 0;
      for (int q = 0; q < table.n; ++q) {
        const HerkPanel &e = table.p[q];
        const int64_t kv = valid_k(e.n_dev, e.n_host, e.kmul, e.Kcap);
        int ns;
        int64_t kcq;
        plan_splits(kv, e.plan_tiles, e.k_chunk, nsm, ns, kcq);
        if (lane == 0) {
          s_first[q] = acc;
          s_nsplit[q] = ns;
          s_kc[q] = kcq;
          s_kvalid[q] = kv;
        }
        acc += ns * (e.T * (e.T + 1) / 2);
      }
      if (lane == 0) s_first[table.n] = acc;
    }
    __syncthreads();
    n_units = s_first[table.n];
  } else {
    kvalid = valid_k(n_dev, n_host, kmul, Kcap);
    int nsplit;
    plan_splits(kvalid, n_tiles * ngroup, k_chunk, nsm, nsplit, kc);
    per_panel = n_tiles * nsplit;
    n_units = per_panel * ngroup;
  }
  if ((int)blockIdx.x >= n_units) return;  // uniform over the CTA

  // Where unit u is: its panel and block count, tile, columns and partial tile.
  auto place = [&](int u, const uint8_t *&zpanel, float *&partial, int &Tu, int &I, int &J, int64_t &k0,
                   int64_t &klen) {
    if constexpr (tabled) {
      int q = 0;
      while (q + 1 < table.n && s_first[q + 1] <= u) ++q;
      const HerkPanel &e = table.p[q];
      const int nt = e.T * (e.T + 1) / 2;
      const int r = u - s_first[q];
      Tu = e.T;
      decode_tile(r % nt, e.T, I, J);
      zpanel = e.panel;
      partial = e.partials + ((size_t)e.index * s_nsplit[q] * nt + r) * (256 * 128);
      k0 = (int64_t)(r / nt) * s_kc[q];
      klen = min(s_kc[q], s_kvalid[q] - k0);
    } else {
      const int r = u % per_panel;
      Tu = T;
      decode_tile(r % n_tiles, T, I, J);
      zpanel = zpanels + (int64_t)(u / per_panel) * zstride;
      partial = partials + (size_t)u * (256 * 128);
      k0 = (int64_t)(r / n_tiles) * kc;
      klen = min(kc, kvalid - k0);
    }
  };
  // a bounded wait ran out: every status word of the launch learns it
  auto flag_timeout = [&]() {
    if (status) atomicOr(status, MVB_DEV_TIMEOUT);
    if constexpr (tabled)
      for (int q = 0; q < table.n; ++q)
        if (table.p[q].status) atomicOr(table.p[q].status, MVB_DEV_TIMEOUT);
  };

  uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));

  if (threadIdx.x == 0) {
    for (int s = 0; s < C::STAGES; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&dfull_bar[b], 1);
      mbar_init(&dempty_bar[b], kEpiWarps);
    }
    mbar_init(&drain_bar, 1);
    for (int i = 0; i < kUnitRing; ++i) {
      mbar_init(&ufull_bar[i], 1);
      mbar_init(&uempty_bar[i], 1 + kEpiWarps);
    }
    abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 1) {
    tmem_alloc(&tmem_base_sh, 512);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = tmem_base_sh;

  uint64_t issued = 0;  // producer: stages issued
  if (warp == 0 && lane == 0) {
    // ---------------- bulk-copy producer ----------------
    uint32_t st = 0, ph = 0;
    for (uint32_t uk = 0; !abort_flag; ++uk) {
      // the CTA's next unit from the launch's counter, handed to the other roles
      const int us = uk % kUnitRing;
      if (!mbar_wait(&uempty_bar[us], ((uk / kUnitRing) & 1u) ^ 1u, wait_ns)) {
        flag_timeout();
        abort_flag = 1;
        break;
      }
      const int u = min(atomicAdd(unit_next, 1), n_units);
      unit_q[us] = u;
      mbar_arrive(&ufull_bar[us]);
      if (u >= n_units) break;
      const uint8_t *zpanel;
      float *partial;
      int Tu, I, J;
      int64_t k0, klen;
      place(u, zpanel, partial, Tu, I, J, k0, klen);
      const int nkb = (int)((klen + C::KB - 1) / C::KB);
      const bool diag = I == J;
      const uint32_t bytes = diag ? C::OPER_BYTES : 2 * C::OPER_BYTES;
      for (int kbi = 0; kbi < nkb; ++kbi) {
        if (!mbar_wait(&empty_bar[st], ph ^ 1, wait_ns)) {
          flag_timeout();
          abort_flag = 1;
          break;
        }
        mbar_arrive_expect_tx(&full_bar[st], bytes);
        uint8_t *a = smem + (size_t)st * C::STAGE_BYTES;
        // k-block index: k0 is a multiple of 64 elements, a k-block 64 bytes;
        // operand (kb, R) starts at ((kb T + R) 2P) planes of 8 KB
        const int64_t kb = (k0 + (int64_t)kbi * C::KB) / C::KB;
        bulk_load(a, zpanel + (kb * Tu + I) * (int64_t)C::OPER_BYTES, C::OPER_BYTES, &full_bar[st]);
        if (!diag)
          bulk_load(a + C::OPER_BYTES, zpanel + (kb * Tu + J) * (int64_t)C::OPER_BYTES, C::OPER_BYTES, &full_bar[st]);
        ++issued;
        if (++st == C::STAGES) {
          st = 0;
          ph ^= 1;
        }
      }
    }
  } else if (warp == 1 && lane == 0) {
    // ---------------- UMMA issuer: one fresh TMEM block per KD k-steps ----------------
    uint32_t st = 0, ph = 0, buf = 0, dph = 0;
    for (uint32_t uk = 0; !abort_flag; ++uk) {
      const int us = uk % kUnitRing;
      if (!mbar_wait(&ufull_bar[us], (uk / kUnitRing) & 1u, wait_ns)) {
        flag_timeout();
        abort_flag = 1;
        break;
      }
      const int u = unit_q[us];
      mbar_arrive(&uempty_bar[us]);
      if (u >= n_units) break;
      const uint8_t *zpanel;
      float *partial;
      int Tu, I, J;
      int64_t k0, klen;
      place(u, zpanel, partial, Tu, I, J, k0, klen);
      const int nks = (int)((klen + C::KSTEP - 1) / C::KSTEP);
      const bool diag = I == J;
      bool ok = true;
      if constexpr (KD == 2 || KD == 4) {
        // a TMEM block is KD / 2 whole stages (two k-steps each): products
        // ordered by magnitude across the block's k-steps -- every cross term,
        // then the hi x hi products -- so that the block's large partial sum
        // exists only for its last instructions (the accumulator is truncated
        // toward zero at each)
        constexpr int SPB = KD / 2;
        for (int ks = 0; ks < nks; ks += KD) {
          const int nk = min(KD, nks - ks);
          const int nst = (nk + 1) / 2;
          uint32_t slot[SPB];
          if (!mbar_wait(&dempty_bar[buf], ((dph >> buf) & 1u) ^ 1u, wait_ns)) ok = false;
#pragma unroll
          for (int j = 0; j < SPB; ++j) {
            if (j >= nst || !ok) break;
            if (!mbar_wait(&full_bar[st], ph, wait_ns)) {
              ok = false;
              break;
            }
            slot[j] = st;
            if (++st == C::STAGES) {
              st = 0;
              ph ^= 1;
            }
          }
          if (!ok) break;
          tc_fence_after();
          const uint32_t d = tbase + buf * 256;
#pragma unroll
          for (int q = 0; q < C::NPROD; ++q) {
            uint32_t pa, pb;
            product_terms(C::NPROD, q, pa, pb);
#pragma unroll
            for (int kk = 0; kk < KD; ++kk) {
              if (kk >= nk) break;
              const uint32_t a_base =
                  smem_u32(smem + (size_t)slot[kk >> 1] * C::STAGE_BYTES) + (uint32_t)(kk & 1) * 32;
              const uint32_t b_base = diag ? a_base : a_base + C::OPER_BYTES;
              const uint64_t a_re = umma_desc_sw64(a_base + (2 * pa) * kPlaneBytes);
              const uint64_t a_im = umma_desc_sw64(a_base + (2 * pa + 1) * kPlaneBytes);
              const uint64_t b_re = umma_desc_sw64(b_base + (2 * pb) * kPlaneBytes);
              const uint64_t b_im = umma_desc_sw64(b_base + (2 * pb + 1) * kPlaneBytes);
              // the two N = 128 products first: the block's real and imaginary
              // halves each start from Zi terms, then take the Zr terms
              const uint32_t acc = (q > 0 || kk > 0) ? 1u : 0u;
              umma<MODE>(d, a_im, b_im, C::ID128, acc);
              umma<MODE>(d + 128, a_im, b_re, C::ID128N, acc);
              umma<MODE>(d, a_re, b_re, diag ? C::ID128 : C::ID256, 1u);
            }
          }
#pragma unroll
          for (int j = 0; j < SPB; ++j)
            if (j < nst) tc_commit(&empty_bar[slot[j]]);  // the block's stages are consumed
          tc_commit(&dfull_bar[buf]);                      // the block is complete
          dph ^= 1u << buf;
          buf ^= 1u;
        }
      } else {
      // k-steps in order; a TMEM block holds KD of them, a stage (one 64-byte
      // k-block) two: the block and stage boundaries are independent
      for (int ks = 0; ks < nks; ++ks) {
        if (ks % KD == 0) {  // a fresh TMEM block
          if (!mbar_wait(&dempty_bar[buf], ((dph >> buf) & 1u) ^ 1u, wait_ns)) {
            ok = false;
            break;
          }
          tc_fence_after();
        }
        if ((ks & 1) == 0) {  // a new stage
          if (!mbar_wait(&full_bar[st], ph, wait_ns)) {
            ok = false;
            break;
          }
          tc_fence_after();
        }
        const uint32_t d = tbase + buf * 256;
        const uint32_t koff = (uint32_t)(ks & 1) * 32;  // the k-step's 32 bytes within the 64-byte rows
        const uint32_t a_base = smem_u32(smem + (size_t)st * C::STAGE_BYTES) + koff;
        const uint32_t b_base = diag ? a_base : a_base + C::OPER_BYTES;
#pragma unroll
        for (int q = 0; q < C::NPROD; ++q) {
          uint32_t pa, pb;
          product_terms(C::NPROD, q, pa, pb);
          const uint64_t a_re = umma_desc_sw64(a_base + (2 * pa) * kPlaneBytes);
          const uint64_t a_im = umma_desc_sw64(a_base + (2 * pa + 1) * kPlaneBytes);
          const uint64_t b_re = umma_desc_sw64(b_base + (2 * pb) * kPlaneBytes);
          const uint64_t b_im = umma_desc_sw64(b_base + (2 * pb + 1) * kPlaneBytes);
          const uint32_t acc = (ks % KD != 0 || q > 0) ? 1u : 0u;
          umma<MODE>(d, a_im, b_im, C::ID128, acc);
          umma<MODE>(d + 128, a_im, b_re, C::ID128N, acc);
          umma<MODE>(d, a_re, b_re, diag ? C::ID128 : C::ID256, 1u);
        }
        if ((ks & 1) == 1 || ks == nks - 1) {  // the stage is consumed
          tc_commit(&empty_bar[st]);
          if (++st == C::STAGES) {
            st = 0;
            ph ^= 1;
          }
        }
        if (ks % KD == KD - 1 || ks == nks - 1) {  // the block is complete
          tc_commit(&dfull_bar[buf]);
          dph ^= 1u << buf;
          buf ^= 1u;
        }
      }
      }
      if (!ok) {
        flag_timeout();
        abort_flag = 1;
        break;
      }
    }
  } else if (warp >= 2) {
    // ---------------- epilogue: drain every k-step block into FP32 registers ----------------
    const int quad = warp & 3;
    const int quarter = (warp - 2) >> 2;  // columns [64 quarter, 64 quarter + 64)
    const int row = quad * 32 + lane;
    uint32_t buf = 0, dph = 0;
    float acc[64];
#pragma unroll
    for (int j = 0; j < 64; ++j) acc[j] = 0.f;
    for (uint32_t uk = 0; !abort_flag; ++uk) {
      const int us = uk % kUnitRing;
      // every lane waits; the vote keeps the warp converged
      if (!__all_sync(0xffffffffu, mbar_wait(&ufull_bar[us], (uk / kUnitRing) & 1u, wait_ns))) {
        if (lane == 0) flag_timeout();
        abort_flag = 1;
        break;
      }
      const int u = unit_q[us];
      __syncwarp();
      if (lane == 0) mbar_arrive(&uempty_bar[us]);
      if (u >= n_units) break;
      const uint8_t *zpanel;
      float *partial;
      int Tu, I, J;
      int64_t k0, klen;
      place(u, zpanel, partial, Tu, I, J, k0, klen);
      const int nks = (int)((klen + C::KSTEP - 1) / C::KSTEP);
      bool ok = true;
      for (int g0 = 0; g0 < nks; g0 += KD) {
        // every lane waits; the vote keeps the warp converged for tcgen05.ld
        ok = __all_sync(0xffffffffu, mbar_wait(&dfull_bar[buf], (dph >> buf) & 1u, wait_ns));
        if (!ok) break;
        tc_fence_after();
        const uint32_t taddr = tbase + ((uint32_t)(quad * 32) << 16) + buf * 256 + quarter * 64;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          uint32_t v[16];
          tmem_ld16(taddr + c * 16, v);
          tmem_ld_wait();
#pragma unroll
          for (int j = 0; j < 16; ++j) acc[c * 16 + j] += __uint_as_float(v[j]);
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&dempty_bar[buf]);
        dph ^= 1u << buf;
        buf ^= 1u;
      }
      if (!ok) {
        if (lane == 0) flag_timeout();
        abort_flag = 1;
        break;
      }
      float *dst = partial + (size_t)quarter * 64 * 128;
#pragma unroll
      for (int j = 0; j < 64; ++j) {
        dst[j * 128 + row] = acc[j];
        acc[j] = 0.f;
      }
    }
  }

  __syncthreads();
  if (abort_flag) {
    if (warp == 0 && lane == 0) {
      // wait for the copies still in flight (the last STAGES issued)
      const uint64_t first = issued > (uint64_t)C::STAGES ? issued - C::STAGES : 0;
      for (uint64_t i = first; i < issued; ++i)
        mbar_wait(&full_bar[i % C::STAGES], (uint32_t)((i / C::STAGES) & 1), kDrainLimitNs);
    }
    if (warp == 1 && lane == 0) {
      tc_commit(&drain_bar);
      mbar_wait(&drain_bar, 0, kDrainLimitNs);
    }
    __syncthreads();
  }
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(tbase, 512);
  }
}

// ---------------------------------------------------------------------------
// FP64 reduction of the partial tiles into the reference output layout
// out[pair, p, q] = V[ant_i * F + q, ant_j * F + p].
// ---------------------------------------------------------------------------
constexpr int kRedGroups = 16;  // 8-column groups per 128-column tile

__device__ __forceinline__ int tile_index(int I, int J, int T) { return I * T - (I * (I - 1)) / 2 + (J - I); }

template <typename OT>
__device__ __forceinline__ void store_out(void *out, int64_t idx, double re, double im, int accumulate) {
  OT *o = static_cast<OT *>(out) + idx;
  if (accumulate) {
    o->x += re;
    o->y += im;
  } else {
    o->x = re;
    o->y = im;
  }
}

// Float-float accumulator: Knuth's TwoSum keeps the exact rounding error of each
// FP32 addition in a second FP32 word (about 2^-44 relative), on the FP32 pipe;
// the per-element float -> double conversions it replaces ran on the
// conversion unit and bounded the reduction's rate.
struct FF {
  float hi = 0.f, lo = 0.f;
  __device__ __forceinline__ void add(float v) {
    const float s = __fadd_rn(hi, v);
    const float bb = __fsub_rn(s, hi);
    const float err = __fadd_rn(__fsub_rn(hi, __fsub_rn(s, bb)), __fsub_rn(v, bb));
    hi = s;
    lo = __fadd_rn(lo, err);
  }
  __device__ __forceinline__ double value() const { return (double)hi + (double)lo; }
};

// Sums of the k-slices' partial values of this thread's four rows r0 .. r0 + 3
// of column c, real and imaginary halves.
__device__ __forceinline__ void sum_slices(const float *__restrict__ tile, int nsplit, size_t tstride, int c, int r0,
                                           FF (&are)[4], FF (&aim)[4]) {
  const size_t sstride = tstride / 4;  // in float4
  const float4 *pre = reinterpret_cast<const float4 *>(tile + c * 128 + r0);
  const float4 *pim = reinterpret_cast<const float4 *>(tile + (128 + c) * 128 + r0);
  int s = 0;
  // eight slices per step: 16 independent 16-byte loads in flight, sums in slice order
  for (; s + 8 <= nsplit; s += 8) {
    float4 vr[8], vi[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      vr[u] = __ldg(pre + (s + u) * sstride);
      vi[u] = __ldg(pim + (s + u) * sstride);
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      are[0].add(vr[u].x), are[1].add(vr[u].y), are[2].add(vr[u].z), are[3].add(vr[u].w);
      aim[0].add(vi[u].x), aim[1].add(vi[u].y), aim[2].add(vi[u].z), aim[3].add(vi[u].w);
    }
  }
  for (; s < nsplit; ++s) {
    const float4 vr = __ldg(pre + s * sstride), vi = __ldg(pim + s * sstride);
    are[0].add(vr.x), are[1].add(vr.y), are[2].add(vr.z), are[3].add(vr.w);
    aim[0].add(vi.x), aim[1].add(vi.y), aim[2].add(vi.z), aim[3].add(vi.w);
  }
}

// sum_slices for a diagonal tile, plus the imaginary half's transposed elements
// (row c, columns r0 .. r0 + 3) for Im V = W - W^T.  The CTA (columns c0 ..
// c0 + 7, warp w = c - c0) stages them through shared memory two slices at a
// time (eight held 176 registers a thread and four spilled at the 80 registers
// that keep three CTAs of the kernel on an SM): thread i loads 16 bytes of column i / 2 (rows c0 + 4 (i % 2) .. + 3, two
// threads per 32-byte sector) and scatters them so that every thread then
// reads its four values as one 16-byte word.  Every thread of the CTA must
// call it: it holds __syncthreads, and nsplit is uniform over the CTA.
__device__ __forceinline__ void sum_slices_diag(const float *__restrict__ tile, int nsplit, size_t tstride, int c0,
                                                int w, int lane, FF (&are)[4], FF (&aim)[4], FF (&aimt)[4]) {
  constexpr int kS = 2;              // slices per step
  __shared__ float4 tsm[kS][8][32];  // [slice of the step][column warp][lane]: rows 4 lane .. 4 lane + 3
  const int c = c0 + w, r0 = 4 * lane;
  const size_t sstride = tstride / 4;  // in float4
  const float4 *pre = reinterpret_cast<const float4 *>(tile + c * 128 + r0);
  const float4 *pim = reinterpret_cast<const float4 *>(tile + (128 + c) * 128 + r0);
  const int rr = threadIdx.x >> 1, hh = threadIdx.x & 1;  // this thread's load: column rr, rows c0 + 4 hh ..
  const float4 *pt = reinterpret_cast<const float4 *>(tile + (128 + rr) * 128 + c0 + 4 * hh);
  // element (row c0 + 4 hh + j, column rr) belongs to warp 4 hh + j, lane rr / 4, component rr % 4
  float *tdst = reinterpret_cast<float *>(&tsm[0][4 * hh][rr >> 2]) + (rr & 3);
  for (int s = 0; s < nsplit; s += kS) {
    const int nu = min(kS, nsplit - s);
    float4 vr[kS], vi[kS], vt[kS];
#pragma unroll
    for (int u = 0; u < kS; ++u)
      if (u < nu) {
        vr[u] = __ldg(pre + (s + u) * sstride);
        vi[u] = __ldg(pim + (s + u) * sstride);
        vt[u] = __ldg(pt + (s + u) * sstride);
      }
    __syncthreads();  // the previous step's reads of tsm are done
#pragma unroll
    for (int u = 0; u < kS; ++u)
      if (u < nu) {
        float *d = tdst + u * (8 * 32 * 4);
        d[0 * 32 * 4] = vt[u].x;
        d[1 * 32 * 4] = vt[u].y;
        d[2 * 32 * 4] = vt[u].z;
        d[3 * 32 * 4] = vt[u].w;
      }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < kS; ++u)
      if (u < nu) {
        const float4 t4 = tsm[u][w][lane];
        are[0].add(vr[u].x), are[1].add(vr[u].y), are[2].add(vr[u].z), are[3].add(vr[u].w);
        aim[0].add(vi[u].x), aim[1].add(vi[u].y), aim[2].add(vi[u].z), aim[3].add(vi[u].w);
        aimt[0].add(t4.x), aimt[1].add(t4.y), aimt[2].add(t4.z), aimt[3].add(t4.w);
      }
  }
}

// One CTA (8 warps) per 8 columns of an upper tile: warp w sums column c0 + w,
// lane l rows 4l .. 4l + 3 (a 16-byte load per component per k-slice; a warp
// reads the column's two contiguous 512-byte runs).  A diagonal tile's
// imaginary half is W - W^T of its partial sums (the product leaves W there).
// F is a template parameter (no runtime integer division in the index
// arithmetic).  blockIdx.y is the panel of a grouped product; its output is
// out_stride bytes further.
template <typename OT, int F>
__global__ void __launch_bounds__(256, 3)
    herk_reduce_all_kernel(const float *__restrict__ part, int ngroup, int T, int n_tiles,
                           const int32_t *__restrict__ n_dev, int64_t n_host, int kmul, int64_t Kcap, int k_chunk,
                           int nsm, int A, void *__restrict__ out_base, int64_t out_stride, double vscale,
                           int accumulate) {
  const int t = blockIdx.x / kRedGroups, g = blockIdx.x % kRedGroups;
  int I, J;
  decode_tile(t, T, I, J);
  const int64_t kvalid = valid_k(n_dev, n_host, kmul, Kcap);
  int nsplit;
  int64_t kc;
  plan_splits(kvalid, n_tiles * ngroup, k_chunk, nsm, nsplit, kc);
  void *out = static_cast<uint8_t *>(out_base) + (int64_t)blockIdx.y * out_stride;
  part += (size_t)blockIdx.y * nsplit * n_tiles * (256 * 128);
  const int M = A * F;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int c = g * 8 + w;
  const int n = J * 128 + c;
  const int r0 = 4 * lane;
  const bool live = n < M && I * 128 + r0 < M;  // this thread has outputs to write
  FF are[4], aim[4], aimt[4];
  const float *tile = part + (size_t)t * (256 * 128);
  const size_t tstride = (size_t)n_tiles * (256 * 128);
  if (I == J) {
    // every thread takes part (the staging synchronises the CTA); its reads stay inside the tile
    sum_slices_diag(tile, nsplit, tstride, g * 8, w, lane, are, aim, aimt);
    if (!live) return;
  } else {
    if (!live) return;
    sum_slices(tile, nsplit, tstride, c, r0, are, aim);
  }
  const int64_t AF2 = (int64_t)A * F * F;
  const int jj = n / F, pp = n % F;  // F is 1 or 2: shifts and masks
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int m = I * 128 + r0 + k;
    if (m >= M) break;
    // an autocorrelation of one feed (m == n) is real, as conj(z) z is in the reference
    const double wi = I == J ? aim[k].value() - aimt[k].value() : aim[k].value();
    const double re = are[k].value() * vscale, im = m == n ? 0.0 : wi * vscale;
    const int i = m / F, q = m % F;
    // direct: rows m -> (i, q), columns n -> (j, p); out[(i*A + j)*F*F + p*F + q]
    store_out<OT>(out, i * AF2 + (int64_t)jj * F * F + pp * F + q, re, im, accumulate);
    // mirror: V[n, m] = conj(V[m, n]) for the off-diagonal tiles (a diagonal tile
    // holds both triangles and is written directly)
    if (I != J) store_out<OT>(out, jj * AF2 + (int64_t)i * F * F + q * F + pp, re, -im, accumulate);
  }
}

// Explicit pair list: one thread per (pair, p, q).
// A pair naming an antenna outside [0, A) reads nothing and gets NaN.
// blockIdx.y is the panel of a grouped product.
template <typename OT>
__global__ void herk_reduce_pairs_kernel(const float *__restrict__ part, int ngroup, int T, int n_tiles,
                                         const int32_t *__restrict__ n_dev, int64_t n_host, int kmul, int64_t Kcap,
                                         int k_chunk, int nsm, int A, int F, const int32_t *__restrict__ pairs,
                                         int64_t npairs, void *__restrict__ out_base, int64_t out_stride,
                                         double vscale, int accumulate) {
  const int64_t total = npairs * F * F;
  const int64_t kvalid = valid_k(n_dev, n_host, kmul, Kcap);
  int nsplit;
  int64_t kc;
  plan_splits(kvalid, n_tiles * ngroup, k_chunk, nsm, nsplit, kc);
  void *out = static_cast<uint8_t *>(out_base) + (int64_t)blockIdx.y * out_stride;
  part += (size_t)blockIdx.y * nsplit * n_tiles * (256 * 128);
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t pr = e / (F * F);
    const int p = (int)((e / F) % F), q = (int)(e % F);
    const int ai = pairs[2 * pr], aj = pairs[2 * pr + 1];
    if (ai < 0 || ai >= A || aj < 0 || aj >= A) {
      store_out<OT>(out, e, __longlong_as_double(0x7ff8000000000000ll), 0.0, 0);
      continue;
    }
    int m = ai * F + q, n = aj * F + p;
    bool conj = false;
    if (m / 128 > n / 128) {
      const int tmp = m;
      m = n;
      n = tmp;
      conj = true;
    }
    const int t = tile_index(m / 128, n / 128, T);
    const int r = m % 128, c = n % 128;
    const bool diag = m / 128 == n / 128;  // imaginary half W - W^T (see herk_reduce_all_kernel)
    FF re, im, imt;
    for (int s = 0; s < nsplit; ++s) {
      const float *p0 = part + ((size_t)s * n_tiles + t) * (256 * 128);
      re.add(__ldg(p0 + c * 128 + r));
      im.add(__ldg(p0 + (128 + c) * 128 + r));
      if (diag) imt.add(__ldg(p0 + (128 + r) * 128 + c));
    }
    const double wi = diag ? im.value() - imt.value() : im.value();
    const double vi = m == n ? 0.0 : (conj ? -wi : wi) * vscale;  // one-feed autos are real
    store_out<OT>(out, e, re.value() * vscale, vi, accumulate);
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
// Raises a kernel's dynamic shared-memory limit once per (device, slot); the
// attribute is not touched again, in particular not during graph capture.
int set_smem_once(const void *fn, int bytes, int slot) {
  static bool done[64][64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64 || slot < 0 || slot >= 64)
    return fail(MVB_ERR_CUDA, "set_smem_once: bad device");
  if (done[dev][slot]) return MVB_OK;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e != cudaSuccess) return fail(MVB_ERR_CUDA, "smem attribute: %s", cudaGetErrorString(e));
  done[dev][slot] = true;
  return MVB_OK;
}

// Wall-time limit of the product's pipeline waits, process-wide (see
// mvb_set_wait_limit_ns); read at each launch.
static std::atomic<uint64_t> g_wait_limit_ns{kWaitLimitNs};
uint64_t wait_limit_ns() { return g_wait_limit_ns.load(std::memory_order_relaxed); }

// table.n > 0: the units come from the table (z, ngroup, shape and status arguments unused).
template <int MODE, int KD>
static int launch_herk(const void *z, int64_t zstride, int ngroup, int64_t Mpad, int64_t Kcap, const int32_t *n_dev,
                       int64_t n_host, int kmul, int k_chunk, float *partials, int32_t *status, int *unit_next,
                       cudaStream_t s, const HerkTable &table) {
  using C = HerkCfg<MODE>;
  const int T = (int)(Mpad / 128);
  const int n_tiles = T * (T + 1) / 2;
  const int nsm = num_sms();
  int64_t max_units = (int64_t)ngroup * n_tiles * (ceil_div(Kcap, k_chunk) + kPlanExtra);
  if (table.n > 0) {
    max_units = 0;
    for (int q = 0; q < table.n; ++q) {
      const HerkPanel &e = table.p[q];
      max_units += (int64_t)(e.T * (e.T + 1) / 2) * (ceil_div(e.Kcap, e.k_chunk) + kPlanExtra);
    }
  }
  const int grid = (int)std::min<int64_t>(max_units, nsm);
  const size_t smem = (size_t)C::STAGES * C::STAGE_BYTES + 1024;
  // slots 16 + 3 * MODE + {0, 1, 2} for KD = {1, 2, 4}, 15 more for the table forms
  const int slot = 16 + 3 * MODE + (KD == 4 ? 2 : KD - 1) + (table.n > 0 ? 15 : 0);
  const void *fn = table.n > 0 ? reinterpret_cast<const void *>(herk_kernel<MODE, KD, true>)
                               : reinterpret_cast<const void *>(herk_kernel<MODE, KD, false>);
  int rc = set_smem_once(fn, (int)smem, slot);
  if (rc) return rc;
  if (grid <= 0) return MVB_OK;
  const uint64_t wait_ns = wait_limit_ns();
  // the CTAs take units from this counter, zeroed on the launch's stream
  cudaError_t e = cudaMemsetAsync(unit_next, 0, sizeof(int), s);
  if (e != cudaSuccess) return fail(MVB_ERR_CUDA, "herk unit counter: %s", cudaGetErrorString(e));
  if (table.n > 0)
    herk_kernel<MODE, KD, true><<<grid, kHerkThreads, smem, s>>>(static_cast<const uint8_t *>(z), zstride, ngroup, T,
                                                                 n_tiles, n_dev, n_host, kmul, Kcap, k_chunk, nsm,
                                                                 partials, status, unit_next, wait_ns, table);
  else
    herk_kernel<MODE, KD, false><<<grid, kHerkThreads, smem, s>>>(static_cast<const uint8_t *>(z), zstride, ngroup, T,
                                                                  n_tiles, n_dev, n_host, kmul, Kcap, k_chunk, nsm,
                                                                  partials, status, unit_next, wait_ns, table);
  return check_launch("herk_kernel");
}

// Argument checks shared by the product and its reductions (the slice plan
// the reductions recompute is the product's only if these hold).
static int check_herk_shape(const char *who, int ngroup, int64_t Mpad, int64_t Kcap, const int32_t *n_dev,
                            int64_t n_host, int kmul, int k_chunk) {
  if (ngroup <= 0 || Mpad <= 0 || Mpad % 128 || Kcap <= 0 || Kcap % kKAlign || k_chunk <= 0 || k_chunk % kKAlign ||
      n_host < 0 || kmul <= 0)
    return fail(MVB_ERR_ARG, "%s: bad arguments", who);
  if (!n_dev && n_host * kmul > Kcap) return fail(MVB_ERR_ARG, "%s: n * kmul exceeds Kcap", who);
  if (Kcap > INT32_MAX || Mpad > 65536) return fail(MVB_ERR_ARG, "%s: panel too large", who);
  const int64_t T = Mpad / 128;
  if ((int64_t)ngroup * (T * (T + 1) / 2) * (ceil_div(Kcap, k_chunk) + kPlanExtra) > INT32_MAX)
    return fail(MVB_ERR_ARG, "%s: too many work units", who);
  return MVB_OK;
}

// The checks of one product (a group of ngroup panels of one shape).
static int check_herk_group(const char *who, const void *z, int64_t zstride, int ngroup, int mode, int64_t Mpad,
                            int64_t Kcap, const int32_t *n_dev, int64_t n_host, int kmul, int k_chunk, const void *ws,
                            size_t ws_bytes, const int32_t *status) {
  if (!z || !ws || !status) return fail(MVB_ERR_ARG, "%s: bad arguments", who);
  int rc = check_herk_shape(who, ngroup, Mpad, Kcap, n_dev, n_host, kmul, k_chunk);
  if (rc) return rc;
  if (reinterpret_cast<uintptr_t>(z) % 16 || zstride % 16) return fail(MVB_ERR_ARG, "%s: panel not 16-byte aligned", who);
  if (ngroup > 1 && (size_t)zstride < mvb_zpanel_bytes(mode, Mpad, Kcap))
    return fail(MVB_ERR_ARG, "%s: panels overlap (stride below mvb_zpanel_bytes)", who);
  if (ws_bytes / (size_t)ngroup < mvb_herk_ws_bytes(Mpad, Kcap, k_chunk))
    return fail(MVB_ERR_ARG, "%s: workspace too small", who);
  if (reinterpret_cast<uintptr_t>(ws) % 16) return fail(MVB_ERR_ARG, "%s: ws must be 16-byte aligned", who);
  return MVB_OK;
}

static int herk_impl(const char *who, const void *z, int64_t zstride, int ngroup, int mode, int64_t Mpad, int64_t Kcap,
                     const int32_t *n_dev, int64_t n_host, int kmul, int k_chunk, int drain_ksteps, void *ws,
                     size_t ws_bytes, int32_t *status, void *stream, const HerkTable &table = HerkTable{}) {
  if (table.n == 0) {
    int rc = check_herk_group(who, z, zstride, ngroup, mode, Mpad, Kcap, n_dev, n_host, kmul, k_chunk, ws, ws_bytes,
                              status);
    if (rc) return rc;
  }
  if (drain_ksteps < 0 || drain_ksteps > 4 || drain_ksteps == 3)
    return fail(MVB_ERR_ARG, "%s: drain_ksteps must be 0, 1, 2 or 4", who);
  // default: a block per stage (two k-steps), the fastest interval in every mode
  const int kd = drain_ksteps ? drain_ksteps : 2;
  cudaStream_t s = as_stream(stream);
  float *part = static_cast<float *>(ws);
  // past every partial tile: each group's share of ws_bytes holds kCounterBytes spare
  int *next = reinterpret_cast<int *>(static_cast<uint8_t *>(ws) + ((ws_bytes - 16) & ~size_t(15)));
#define MVB_HERK(M)                                                                                          \
  return kd == 1   ? launch_herk<M, 1>(z, zstride, ngroup, Mpad, Kcap, n_dev, n_host, kmul, k_chunk, part, status, \
                                       next, s, table)                                                       \
         : kd == 2 ? launch_herk<M, 2>(z, zstride, ngroup, Mpad, Kcap, n_dev, n_host, kmul, k_chunk, part, status, \
                                       next, s, table)                                                       \
                   : launch_herk<M, 4>(z, zstride, ngroup, Mpad, Kcap, n_dev, n_host, kmul, k_chunk, part, status, \
                                       next, s, table)
  switch (mode) {
    case MVB_GEMM_BF16_3: MVB_HERK(MVB_GEMM_BF16_3);
    case MVB_GEMM_BF16_6: MVB_HERK(MVB_GEMM_BF16_6);
    case MVB_GEMM_TF32_3: MVB_HERK(MVB_GEMM_TF32_3);
    case MVB_GEMM_F16_3: MVB_HERK(MVB_GEMM_F16_3);
    default: return fail(MVB_ERR_ARG, "%s: unknown mode %d", who, mode);
  }
#undef MVB_HERK
}

static int reduce_impl(const char *who, const void *ws, size_t ws_bytes, int ngroup, int64_t Mpad, int64_t Kcap,
                       const int32_t *n_dev, int64_t n_host, int kmul, int k_chunk, int nant, int nfeed,
                       const int32_t *pairs, int64_t npairs, void *out, int64_t out_stride, int out_c128,
                       double vscale, int accumulate, void *stream) {
  // the checks of mvb_herk: the slice plan recomputed here is then the product's
  if (!ws || !out || nant <= 0 || (nfeed != 1 && nfeed != 2) || (int64_t)nant * nfeed > Mpad || (pairs && npairs < 0))
    return fail(MVB_ERR_ARG, "%s: bad arguments", who);
  int rc = check_herk_shape(who, ngroup, Mpad, Kcap, n_dev, n_host, kmul, k_chunk);
  if (rc) return rc;
  if (ws_bytes / (size_t)ngroup < mvb_herk_ws_bytes(Mpad, Kcap, k_chunk))
    return fail(MVB_ERR_ARG, "%s: workspace smaller than the product's (mvb_herk_ws_bytes)", who);
  if (reinterpret_cast<uintptr_t>(ws) % 16) return fail(MVB_ERR_ARG, "%s: ws must be 16-byte aligned", who);
  const int64_t per_out = (pairs ? npairs : (int64_t)nant * nant) * nfeed * nfeed * (out_c128 ? 16 : 8);
  if (ngroup > 1 && out_stride < per_out) return fail(MVB_ERR_ARG, "%s: outputs overlap (out_stride too small)", who);
  if (ngroup > 65535) return fail(MVB_ERR_ARG, "%s: at most 65535 panels per launch", who);
  const int T = (int)(Mpad / 128);
  const int n_tiles = T * (T + 1) / 2;
  const int nsm = num_sms();
  const float *part = static_cast<const float *>(ws);
  cudaStream_t s = as_stream(stream);
  if (!pairs) {
    const dim3 grid((unsigned)(n_tiles * kRedGroups), (unsigned)ngroup);
#define MVB_RED(OT, FF_)                                                                                    \
  herk_reduce_all_kernel<OT, FF_><<<grid, 256, 0, s>>>(part, ngroup, T, n_tiles, n_dev, n_host, kmul, Kcap, \
                                                       k_chunk, nsm, nant, out, out_stride, vscale, accumulate)
    if (out_c128) {
      if (nfeed == 2) MVB_RED(double2, 2); else MVB_RED(double2, 1);
    } else {
      if (nfeed == 2) MVB_RED(float2, 2); else MVB_RED(float2, 1);
    }
#undef MVB_RED
  } else {
    if (npairs == 0) return MVB_OK;
    const int64_t total = npairs * nfeed * nfeed;
    const dim3 grid((unsigned)std::min<int64_t>(ceil_div(total, 256), (int64_t)nsm * 8), (unsigned)ngroup);
    if (out_c128)
      herk_reduce_pairs_kernel<double2><<<grid, 256, 0, s>>>(part, ngroup, T, n_tiles, n_dev, n_host, kmul, Kcap,
                                                             k_chunk, nsm, nant, nfeed, pairs, npairs, out, out_stride,
                                                             vscale, accumulate);
    else
      herk_reduce_pairs_kernel<float2><<<grid, 256, 0, s>>>(part, ngroup, T, n_tiles, n_dev, n_host, kmul, Kcap,
                                                            k_chunk, nsm, nant, nfeed, pairs, npairs, out, out_stride,
                                                            vscale, accumulate);
  }
  return check_launch(who);
}

}  // namespace mvb

using namespace mvb;

extern "C" uint64_t mvb_set_wait_limit_ns(uint64_t limit_ns) {
  return g_wait_limit_ns.exchange(limit_ns ? limit_ns : kWaitLimitNs);
}

extern "C" size_t mvb_herk_ws_bytes(int64_t Mpad, int64_t Kcap, int k_chunk) {
  if (Mpad <= 0 || Kcap <= 0 || k_chunk <= 0) return 0;
  const int64_t T = Mpad / 128;
  return (size_t)(T * (T + 1) / 2) * (size_t)(ceil_div(Kcap, k_chunk) + kPlanExtra) * 256 * 128 * sizeof(float) +
         kCounterBytes;
}

extern "C" int mvb_herk(const void *z, int mode, int64_t Mpad, int64_t Kcap, const int32_t *n_dev, int64_t n_host,
                        int kmul, int k_chunk, int drain_ksteps, void *ws, size_t ws_bytes, int32_t *status,
                        void *stream) {
  return herk_impl("mvb_herk", z, 0, 1, mode, Mpad, Kcap, n_dev, n_host, kmul, k_chunk, drain_ksteps, ws, ws_bytes,
                   status, stream);
}

extern "C" int mvb_herk_grouped(const void *z, size_t z_stride, int ngroup, int mode, int64_t Mpad, int64_t Kcap,
                                const int32_t *n_dev, int64_t n_host, int kmul, int k_chunk, int drain_ksteps,
                                void *ws, size_t ws_bytes, int32_t *status, void *stream) {
  if (z_stride > (size_t)INT64_MAX) return fail(MVB_ERR_ARG, "mvb_herk_grouped: bad arguments");
  return herk_impl("mvb_herk_grouped", z, (int64_t)z_stride, ngroup, mode, Mpad, Kcap, n_dev, n_host, kmul, k_chunk,
                   drain_ksteps, ws, ws_bytes, status, stream);
}

extern "C" int mvb_herk_batch(const mvb_herk_group *groups, int ngroups, int mode, int drain_ksteps, void *stream) {
  if (!groups || ngroups <= 0) return fail(MVB_ERR_ARG, "mvb_herk_batch: bad arguments");
  HerkTable table{};
  for (int g = 0; g < ngroups; ++g) {
    const mvb_herk_group &e = groups[g];
    if (e.z_stride > (size_t)INT64_MAX) return fail(MVB_ERR_ARG, "mvb_herk_batch: bad arguments");
    int rc = check_herk_group("mvb_herk_batch", e.z, (int64_t)e.z_stride, e.ngroup, mode, e.Mpad, e.Kcap, e.n_dev,
                              e.n_host, e.kmul, e.k_chunk, e.ws, e.ws_bytes, e.status);
    if (rc) return rc;
    if (table.n + e.ngroup > kMaxBatchPanels)
      return fail(MVB_ERR_ARG, "mvb_herk_batch: more than %d panels in one launch", kMaxBatchPanels);
    const int T = (int)(e.Mpad / 128);
    for (int j = 0; j < e.ngroup; ++j) {
      HerkPanel &p = table.p[table.n++];
      p.panel = static_cast<const uint8_t *>(e.z) + (int64_t)j * (int64_t)e.z_stride;
      p.n_dev = e.n_dev;
      p.partials = static_cast<float *>(e.ws);
      p.status = e.status;
      p.n_host = e.n_host;
      p.Kcap = e.Kcap;
      p.T = T;
      p.kmul = e.kmul;
      p.k_chunk = e.k_chunk;
      p.plan_tiles = e.ngroup * (T * (T + 1) / 2);
      p.index = j;
    }
  }
  const mvb_herk_group &e0 = groups[0];
  return herk_impl("mvb_herk_batch", e0.z, 0, 1, mode, e0.Mpad, e0.Kcap, e0.n_dev, e0.n_host, e0.kmul, e0.k_chunk,
                   drain_ksteps, e0.ws, e0.ws_bytes, nullptr, stream, table);
}

extern "C" int mvb_herk_reduce(const void *ws, size_t ws_bytes, int64_t Mpad, int64_t Kcap, const int32_t *n_dev,
                               int64_t n_host, int kmul, int k_chunk, int nant, int nfeed, const int32_t *pairs,
                               int64_t npairs, void *out, int out_c128, double vscale, int accumulate, void *stream) {
  return reduce_impl("mvb_herk_reduce", ws, ws_bytes, 1, Mpad, Kcap, n_dev, n_host, kmul, k_chunk, nant, nfeed, pairs,
                     npairs, out, 0, out_c128, vscale, accumulate, stream);
}

extern "C" int mvb_herk_reduce_grouped(const void *ws, size_t ws_bytes, int ngroup, int64_t Mpad, int64_t Kcap,
                                       const int32_t *n_dev, int64_t n_host, int kmul, int k_chunk, int nant,
                                       int nfeed, const int32_t *pairs, int64_t npairs, void *out, size_t out_stride,
                                       int out_c128, double vscale, int accumulate, void *stream) {
  if (out_stride > (size_t)INT64_MAX) return fail(MVB_ERR_ARG, "mvb_herk_reduce_grouped: bad arguments");
  return reduce_impl("mvb_herk_reduce_grouped", ws, ws_bytes, ngroup, Mpad, Kcap, n_dev, n_host, kmul, k_chunk, nant,
                     nfeed, pairs, npairs, out, (int64_t)out_stride, out_c128, vscale, accumulate, stream);
}

// ---------------------------------------------------------------------------
// Sum of per-chunk visibilities (MatProd.sum_chunks, core/matprod.py:103-115):
// out[i] = sum_c vis[c][i] in chunk order, accumulated in FP64.
// ---------------------------------------------------------------------------
namespace mvb {
template <typename T>
__global__ void chunk_sum_kernel(const T *__restrict__ vis, int64_t nchunks, int64_t n, T *__restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double re = 0.0, im = 0.0;
    for (int64_t c = 0; c < nchunks; ++c) {
      const T v = vis[c * n + i];
      re += (double)v.x;
      im += (double)v.y;
    }
    out[i].x = re;
    out[i].y = im;
  }
}
}  // namespace mvb

extern "C" int mvb_chunk_sum(const void *vis, int64_t nchunks, int64_t n, int c128, void *out, void *stream) {
  if (nchunks < 1 || n < 0 || (n > 0 && (!vis || !out))) return fail(MVB_ERR_ARG, "mvb_chunk_sum: bad arguments");
  if (n == 0) return MVB_OK;
  const int64_t blocks = std::min<int64_t>(ceil_div(n, 256), (int64_t)num_sms() * 8);
  if (c128)
    chunk_sum_kernel<double2><<<(unsigned)blocks, 256, 0, as_stream(stream)>>>(static_cast<const double2 *>(vis),
                                                                               nchunks, n, static_cast<double2 *>(out));
  else
    chunk_sum_kernel<float2><<<(unsigned)blocks, 256, 0, as_stream(stream)>>>(static_cast<const float2 *>(vis),
                                                                              nchunks, n, static_cast<float2 *>(out));
  return check_launch("chunk_sum_kernel");
}

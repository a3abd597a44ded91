// Shared helpers for the sm_100a kernels: status handling, PTX wrappers for
// mbarriers, bulk copies (cp.async.bulk) and tcgen05 (TMEM, UMMA).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdarg>
#include <cstdio>
#include <string>

#include "../../include/matvis_b200.h"

namespace mvb {

// ---------------------------------------------------------------------------
// host-side status
// ---------------------------------------------------------------------------
std::string &last_error();

inline int fail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  last_error() = buf;
  return code;
}

inline int check_launch(const char *what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(MVB_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  return MVB_OK;
}

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

__host__ __device__ inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }
__host__ __device__ inline int64_t round_up(int64_t a, int64_t b) { return ceil_div(a, b) * b; }

int num_sms();
// Sets a kernel's max dynamic shared memory once per (device, slot < 64);
// slots 10..12 are the beam kernels, 16..45 the Hermitian-product variants,
// 48 and 49 the staged pair kernels.
int set_smem_once(const void *fn, int bytes, int slot);
// Wall-time limit of a pipeline wait in the product and the staged pair kernel
// (process-wide, set by mvb_set_wait_limit_ns; 4 s by default).
uint64_t wait_limit_ns();

// Columns of a Z panel are zero-filled up to a multiple of this.
constexpr int kKAlign = 64;
// Rows of a Z panel are padded to a multiple of the Hermitian tile.
constexpr int kTile = 128;

// Split terms per component for a Hermitian-product mode.
__host__ __device__ inline int mode_terms(int mode) { return mode == MVB_GEMM_BF16_6 ? 3 : 2; }
__host__ __device__ inline int mode_elem_bytes(int mode) { return mode == MVB_GEMM_TF32_3 ? 4 : 2; }

// Split-plane panel layout: the Hermitian product's shared-memory image, stored.
// For k-block kb (KB = 64 bytes of elements: 32 bf16 / fp16, 16 tf32) and row
// block I (128 rows), the npl = 2P planes follow each other as 128 rows x 64
// bytes, [Kcap / KB][Mpad / 128][npl][128][KB], and inside each 64-byte row the
// four 16-byte chunks are permuted by the 64-byte swizzle (chunk c of row r is
// stored at chunk c ^ ((r >> 1) & 3), the pattern the UMMA shared-memory
// descriptors read).  One operand of one product stage (two k-steps, all planes)
// is then one contiguous run of npl x 8 KB, fetched with a single bulk copy.
// panel_off gives plane 0's element; plane p is 128 * KB elements further.
constexpr int kKBlockBytes = 64;
__host__ __device__ inline int64_t panel_off(int64_t m, int64_t k, int64_t Mpad, int kb, int npl) {
  const int64_t blk = ((k / kb) * (Mpad / 128) + m / 128) * npl;
  const int r = (int)(m % 128), c = (int)(k % kb);
  const int epc = kb / 4;  // elements per 16-byte chunk
  return blk * (128 * kb) + (int64_t)r * kb + ((c / epc) ^ ((r >> 1) & 3)) * epc + c % epc;
}
__host__ __device__ constexpr int64_t panel_plane_stride(int kb) { return 128 * (int64_t)kb; }

// ---------------------------------------------------------------------------
// device helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t global_timer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// ---- mbarrier -------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Waits for the phase with the given parity to complete; gives up after
// limit_ns nanoseconds of wall time and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint64_t limit_ns) {
  const uint32_t a = smem_u32(bar);
  if (mbar_try_wait(a, parity)) return true;
  const uint64_t t0 = global_timer_ns();
  while (true) {
    if (mbar_try_wait(a, parity)) return true;
    if (global_timer_ns() - t0 > limit_ns) return false;
  }
}

// ---- bulk copies ----------------------------------------------------------
// 1-D bulk copy global -> this CTA's shared memory, no multicast (both
// addresses 16-byte aligned, bytes a multiple of 16).
__device__ __forceinline__ void bulk_load(void *smem_dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(smem_dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// ---- tcgen05 --------------------------------------------------------------
__device__ __forceinline__ void tmem_alloc(uint32_t *smem_dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(smem_dst)),
               "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Arrives on an mbarrier once all prior tcgen05 async operations of this
// thread have completed.
__device__ __forceinline__ void tc_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// D[tmem] (+)= A[smem] * B[smem]^T, both K-major; kind::f16 (bf16 inputs).
__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// Same with tf32 inputs (fp32 containers).
__device__ __forceinline__ void umma_tf32(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// 32 lanes x 32 consecutive 32-bit columns from TMEM into registers.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
}
// 32 lanes x 16 consecutive 32-bit columns from TMEM into registers.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
}
__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Shared-memory matrix descriptor (tcgen05 / UMMA), K-major, 64-byte swizzle:
// rows of 64 bytes, 8-row core-matrix groups of 512 B (SBO); the second
// 32-byte k-step of a row is the start address + 32 B.
__device__ __forceinline__ uint64_t umma_desc_sw64(uint32_t smem_addr) {
  uint64_t d = 0;
  d |= static_cast<uint64_t>((smem_addr & 0x3FFFF) >> 4);  // start address  [0, 14)
  d |= static_cast<uint64_t>(1) << 16;                      // LBO (unused)   [16, 30)
  d |= static_cast<uint64_t>(512 >> 4) << 32;               // SBO            [32, 46)
  d |= static_cast<uint64_t>(1) << 46;                      // version = 1    [46, 48)
  d |= static_cast<uint64_t>(4) << 61;                      // SWIZZLE_64B    [61, 64)
  return d;
}

// Instruction descriptor for kind::f16 / kind::tf32, FP32 accumulate,
// both operands K-major, M = 128.
//   fmt: 1 = BF16, 2 = TF32 (A and B), negb: negate B.
__host__ __device__ constexpr uint32_t umma_idesc(uint32_t fmt, uint32_t n, uint32_t negb) {
  return (1u << 4)              // c_format = F32
         | (fmt << 7)           // a_format
         | (fmt << 10)          // b_format
         | (negb << 14)         // b_negate
         | ((n >> 3) << 17)     // N >> 3
         | ((128u >> 4) << 24); // M >> 4
}

}  // namespace mvb

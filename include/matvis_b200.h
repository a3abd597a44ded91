/*
 * matvis_b200.h -- C ABI of the B200 (sm_100a) visibility-path library
 * (libmatvis_b200.so).
 *
 * Every entry point takes caller-owned DEVICE pointers (the 3x3 rotation of
 * mvb_rotate is the one host array), plain sizes and a CUDA
 * stream (cudaStream_t passed as void*), enqueues its kernels on that stream
 * and returns an int status (MVB_OK = 0).  No entry point allocates device
 * memory: scratch space is a caller-provided workspace whose size a *_ws_bytes
 * query returns.  Device-side failures (buffer overflow, a bounded wait that
 * ran out) are written to a caller-provided int32 status word on the device,
 * never raised with a trap; the host reads it after the stream synchronises.
 *
 * Paths in the comments below are relative to the matvis project root; each
 * entry point names the reference interface it replaces.
 *
 * Array conventions
 *   - "SoA (3, ld)" coordinates: x at [0, ld), y at [ld, 2 ld), z at [2 ld, 3 ld).
 *   - complex64 = interleaved float2, complex128 = interleaved double2.
 *   - Z panel (the operand of the Hermitian product): real planes
 *       plane[q][m][k],  q in [0, 2P),  m in [0, Mpad),  k in [0, Kcap)
 *     with plane q = 2 p + c holding split term p (p = 0 most significant)
 *     of component c (0 = real, 1 = imaginary).  Row m = ant * nfeed + feed,
 *     column k = src * nax + ax.  Rows >= M and columns >= K_valid are zero.
 *     Element type: bfloat16 for MVB_GEMM_BF16_*, float32 for MVB_GEMM_TF32_3,
 *     float16 for MVB_GEMM_F16_3, whose panel holds s*Z for a power-of-two
 *     scale s (zscale) chosen by the caller so that max |s Z| < 2^15; the
 *     product's reduction multiplies by vscale = 1 / s^2.
 */
#ifndef MATVIS_B200_H
#define MATVIS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ----------------------------------------------------- */
#define MVB_OK 0
#define MVB_ERR_ARG 1         /* bad argument (shape, alignment, enum)      */
#define MVB_ERR_CUDA 2        /* a CUDA runtime call failed                 */
#define MVB_ERR_OVERFLOW 3    /* above-horizon count exceeds the capacity   */
#define MVB_ERR_NONFINITE 4   /* non-finite value in an interpolated beam   */
#define MVB_ERR_TIMEOUT 5     /* a bounded device-side wait ran out         */
#define MVB_ERR_UNSUPPORTED 6 /* device or configuration not supported      */

/* device status word bits (OR-ed by kernels into *status) */
#define MVB_DEV_OVERFLOW 0x1
#define MVB_DEV_TIMEOUT 0x2
#define MVB_DEV_NONFINITE 0x4

/* ---- Hermitian-product precision modes ---------------------------------- */
#define MVB_GEMM_BF16_3 0 /* 2-term bf16 split, 3 products (hh+hl+lh)        */
#define MVB_GEMM_BF16_6 1 /* 3-term bf16 split, 6 products (order <= 2)      */
#define MVB_GEMM_TF32_3 2 /* 2-term tf32 split, 3 products (3xTF32)          */
#define MVB_Z_C64 3       /* plain complex64 Z (M, Kcap), for the pair loop */
#define MVB_GEMM_F16_3 4  /* 2-term fp16 split of s*Z (s a power of two), 3 products */

/* ---- library ----------------------------------------------------------- */
int mvb_version(void);
/* Message for the last non-OK status returned on the calling host thread. */
const char *mvb_last_error(void);
/* Number of SMs and compute capability of the current device. */
int mvb_device_info(int *sm_count, int *cc_major, int *cc_minor);

/* ---- A3: rotation ------------------------------------------------------- */
/* topo(3, N) = R(3x3, row-major, host) @ eci(3, N), FP64, each row evaluated as
 * (R[r,0]*x + R[r,1]*y) + R[r,2]*z with separately rounded operations.
 * Replaces CoordinateRotation.rotate (core/coords.py:177-179; the LST form of
 * coordinates.eci_to_enu_matrix @ point_source_crd_eq, coordinates.py:91-125,
 * 174-200).  eci and topo are SoA with leading dimension N. */
int mvb_rotate(const double *eci, int64_t N, const double *R, double *topo, void *stream);

/* ERFA-style apparent place of every source (SoA (3, N) in and out, FP64):
 * light deflection by the Sun, aberration and bias-precession-nutation, the
 * cached "BCRS" directions of CoordinateRotationERFA._set_bcrs
 * (cpu/coords.py:118-215; the per-source _ld kernel of gpu/coords.py:7-53).
 * astrom: 18 host doubles {eh[3], em, dlim, v[3], bm1, bpn[9] (row-major)},
 * the pyerfa apco quantities.  The CIRS -> ENU step (_atioq) is a 3x3 applied
 * with mvb_rotate. */
int mvb_bcrs(const double *eci, int64_t N, const double *astrom, double *bcrs, void *stream);

/* ---- A4: horizon selection ---------------------------------------------- */
/* Bytes of workspace mvb_horizon_compact needs for a chunk of `count` sources. */
size_t mvb_horizon_ws_bytes(int64_t count);
/* Strict z > 0 selection over sources [c0, c1) of topo (SoA, leading dim ld):
 * kept sources in ascending index order -> crd_out (SoA, leading dim cap),
 * idx_out (global source index), n_out (device int32).  If flux != NULL,
 * flux_out[i] = flux[idx_out[i]] for i < n and 0 for n <= i < cap.  If n > cap
 * the first cap entries are written, *n_out = n and MVB_DEV_OVERFLOW is set.
 * Replaces CoordinateRotation.select_chunk (core/coords.py:99-150). */
int mvb_horizon_compact(const double *topo, int64_t ld, int64_t c0, int64_t c1, const double *flux, double *crd_out,
                        int32_t *idx_out, double *flux_out, int32_t *n_out, int64_t cap, int32_t *status, void *ws,
                        size_t ws_bytes, void *stream);

/* Allocation-free form of mvb_horizon_compact; this entry point has no
 * counterpart in the reference.  It is for callers that cannot allocate device
 * memory when they select sources (memory planned once at start-up with
 * allocation forbidden afterwards, since cudaMalloc / cudaFree can synchronise
 * the device; or a host handed only a stream and its buffers by another
 * library).  The per-block scratch is a 16 KB static device array inside the
 * library, held by every GPU that loads it until exit; chunks are limited to
 * 4,194,304 sources (c1 - c0), larger ones are rejected with MVB_ERR_ARG.  The
 * first call on a device looks up the array's device address (with that device
 * current) and caches it, so that first call should come before any stream
 * capture; a reset of the device's primary context (cudaDeviceReset)
 * invalidates the cached address, so the entry point must not be called on a
 * device after its context was reset.  All calls share the one array: calls
 * that overlap on the GPU race,
 * so serialise them (one stream, or events).  Inputs, outputs and semantics are
 * those of mvb_horizon_compact; it calls no allocator. */
int mvb_horizon_compact_static(const double *topo, int64_t ld, int64_t c0, int64_t c1, const double *flux,
                               double *crd_out, int32_t *idx_out, double *flux_out, int32_t *n_out, int64_t cap,
                               int32_t *status, void *stream);

/* ---- A5: beam interpolation ---------------------------------------------- */
/* Bilinear interpolation (order-1 map_coordinates, 0 outside [0, n-1] on either
 * axis) of grids (nbeam, nax, nfeed, nza, naz) at the sources of crd (SoA,
 * leading dim ld): az/za from enu_to_az_za(orientation="uvbeam").  grid_kind:
 * 0 complex64 E-field, 1 float32 power (sqrt applied after interpolation).
 * params: nbeam x 3 doubles (daz, dza, azmin).  Output (nbeam, nfeed, nax, nout)
 * complex64 (out_c128 = 0) or complex128 (1); sources i >= n (n = *n_dev if
 * n_dev != NULL, else nsrc) are written as 0.  Grids of up to 200 KB per real
 * plane are staged in shared memory.  If status != NULL, a non-finite result
 * sets MVB_DEV_NONFINITE.  Replaces BeamInterpolator.__call__ /
 * GPUBeamInterpolator._interp (core/beams.py:184-208, gpu/beams.py:103-200). */
int mvb_beam_interp(const void *grids, int grid_kind, int nbeam, int nax, int nfeed, int nza, int naz,
                    const double *params, const double *crd, int64_t ld, const int32_t *n_dev, int64_t nsrc,
                    void *out, int out_c128, int64_t nout, int32_t *status, void *ws, size_t ws_bytes,
                    void *stream);
/* Workspace of mvb_beam_interp (2 nbeam nout doubles).  With it (ws != NULL)
 * each source's az/za and grid coordinates are computed once for all planes
 * (a first kernel), with the same FP64 expressions; with ws = NULL every
 * plane's threads recompute them. */
size_t mvb_beam_interp_ws_bytes(int nbeam, int64_t nout);
/* Same interpolation at given (azimuth, zenith angle) rows azza (SoA, leading
 * dim ld): the reference's gpu_beam_interpolation(beam, daz, dza, azmin, az, za)
 * (gpu/beams.py:127-200).  Output (nbeam, nfeed, nax, nsrc). */
int mvb_beam_interp_azza(const void *grids, int grid_kind, int nbeam, int nax, int nfeed, int nza, int naz,
                         const double *params, const double *azza, int64_t ld, int64_t nsrc, void *out, int out_c128,
                         void *stream);
/* Achromatic Gaussian power beam, amplitude exp(-za^2 / (2 sigma^2)), one beam
 * per sigma (nbeam entries), nfeed = nax = 1.  Replaces the analytic-beam path
 * of GPUBeamInterpolator.interp (gpu/beams.py:100-101), on the device. */
int mvb_beam_gaussian(const double *sigmas, int nbeam, const double *crd, int64_t ld, const int32_t *n_dev,
                      int64_t nsrc, void *out, int out_c128, int64_t nout, void *stream);

/* ---- A6: tau and Z --------------------------------------------------------- */
/* exptau(A, nsrc) = exp(+2 pi i (freq/c) antpos . crd) with the phase in cycles
 * reduced mod 1 in FP64 before an FP32 (out_c128 = 0) or FP64 sincospi.
 * Replaces TauCalculator.__call__ (core/tau.py:48-71). */
int mvb_exptau(const double *antpos, int A, double freq, const double *crd, int64_t ld, int64_t nsrc,
               void *exptau, int out_c128, void *stream);
/* Z panel layout (modes MVB_GEMM_*): 2P planes (plane 2p + c holds split term
 * p of component c, c = 0 real, 1 imaginary), stored as the Hermitian product's
 * shared-memory image [Kcap / KB][Mpad / 128][2P][128][KB] with KB = 64 bytes
 * of elements (32 for bf16 / fp16, 16 for tf32), the four 16-byte chunks of
 * each 64-byte row in 64-byte swizzled order: element (m, k) of plane pl is at
 *   ((k / KB) * (Mpad / 128) + m / 128) * 2P * 128 * KB + pl * 128 * KB
 *   + (m % 128) * KB + ((c / E) ^ ((m % 128 / 2) % 4)) * E + c % E,
 * c = k % KB, E = KB / 4 elements per chunk.
 * Mpad is a multiple of 128, Kcap of 64.  Bytes: 2P x Mpad x Kcap x element size. */
size_t mvb_zpanel_bytes(int mode, int64_t Mpad, int64_t Kcap);
/* sflux[f * N + s] = (float) sqrt(0.5 * flux[s * nf + f]) (cpu/cpu.py:188): the
 * per-frequency sqrt(0.5 I) rows the Z writers read, from the caller's
 * (N, nf) float64 Stokes I. */
int mvb_flux_sqrt_half(const double *flux, int64_t N, int nf, float *sflux, void *stream);
/* Fused tau + Z: Z[a*F+f, s*X+x] = exptau(a, s) * sflux[j] * beam[bidx[a], f, x, s]
 * with j = sidx[s] (sidx != NULL: sflux is the full per-source sqrt(0.5 I) at
 * this frequency, float32) or j = s (sidx == NULL: sflux already compacted),
 * written straight into a Z panel (mode MVB_GEMM_*) or a plain complex64 Z
 * (mode MVB_Z_C64, row pitch Kcap).  n = *n_dev (or nsrc); sources in
 * [n, roundup(n*X, 64)/X) are written as zeros.  beam: complex64 (nbeam, F, X,
 * beam_ld) (device); beam_idx: int32 per antenna (NULL = beam 0 for all).
 * Replaces TauCalculator.__call__ + ZMatrixCalc.__call__ (core/tau.py:48-71,
 * core/getz.py:52-105) with no exptau round trip through HBM. */
int mvb_tau_z(const double *antpos, int A, double freq, const double *crd, int64_t ld, const int32_t *n_dev,
              int64_t nsrc, const float *sflux, const int32_t *sidx, const void *beam, int64_t beam_ld, int nbeam,
              const int32_t *beam_idx, int F, int X, int mode, float zscale, void *z, int64_t Mpad, int64_t Kcap,
              void *stream);
/* mvb_tau_z for nfreq frequencies of one time step in one launch (the grouped
 * chain of a batched job): frequency g = freqs[g] (a DEVICE array of nfreq
 * doubles, Hz), its fluxes sflux + g * sflux_ld (floats) and its panel
 * z + g * z_stride bytes (z_stride >= mvb_zpanel_bytes, a multiple of 16).
 * Each panel equals what mvb_tau_z writes for that frequency.  Replaces the
 * per-frequency TauCalculator / ZMatrixCalc calls of wrapper.py:180-199. */
int mvb_tau_z_grouped(const double *antpos, int A, const double *freqs, int nfreq, const double *crd, int64_t ld,
                      const int32_t *n_dev, int64_t nsrc, const float *sflux, int64_t sflux_ld, const int32_t *sidx,
                      const void *beam, int64_t beam_ld, int nbeam, const int32_t *beam_idx, int F, int X, int mode,
                      float zscale, void *z, size_t z_stride, int64_t Mpad, int64_t Kcap, void *stream);
/* Z panel (or plain complex64 Z) from a caller exptau (A, e_ld), complex64
 * (e_c128 = 0) or complex128: Z[a*F+f, s*X+x] = exptau[a, s] * sflux[s] *
 * beam[bidx[a], f, x, s] for s < nsrc, zeros up to roundup(nsrc*X, 64)/X.
 * Replaces ZMatrixCalc.__call__ (core/getz.py:52-105); the caller's exptau is
 * not modified (the reference scales it in place). */
int mvb_z_from_exptau(const void *exptau, int e_c128, int64_t e_ld, int A, int64_t nsrc, const float *sflux,
                      const void *beam, int64_t beam_ld, int nbeam, const int32_t *beam_idx, int F, int X, int mode,
                      float zscale, void *z, int64_t Mpad, int64_t Kcap, void *stream);
/* Z panel (or plain complex64 Z) from a caller complex matrix z (M, K) with row
 * pitch ldz elements, complex64 (z_c128 = 0) or complex128.  Columns in
 * [K, roundup(K, 64)) are zero-filled.  Serves MatProd.__call__(z, chunk)
 * on an externally built Z (core/matprod.py:83-101). */
int mvb_z_pack(const void *zsrc, int z_c128, int64_t M, int64_t K, int64_t ldz, int mode, float zscale, void *z,
               int64_t Mpad, int64_t Kcap, void *stream);
/* max |z| over n complex values (complex64 or complex128) -> *out (device
 * float32, caller-zeroed); used to choose the MVB_GEMM_F16_3 scale. */
int mvb_absmax(const void *z, int z_c128, int64_t n, float *out, void *stream);

/* ---- A7: Hermitian product on the tensor cores ------------------------------ */
/* In the entry points below the valid K extent of the panel is
 *   K_valid = min(n * kmul, Kcap),  n = *n_dev if n_dev != NULL else n_host,
 * i.e. a source count times the columns per source (nax); the device count
 * comes straight from mvb_horizon_compact, with no host round trip. */
/* Workspace bytes: one FP32 partial tile (256 x 128 floats) per (k-slice, tile)
 * and 256 bytes for the launch's work-unit counter (its last 16 bytes; the
 * product zeroes it on its stream before each launch, so two products must not
 * run at once on one workspace); the workspace must be 16-byte aligned. */
size_t mvb_herk_ws_bytes(int64_t Mpad, int64_t Kcap, int k_chunk);
/* Upper-triangle 128 x 128 complex tiles of V = conj(Z) Z^T over K_valid
 * columns, on the tcgen05 tensor cores with TMEM accumulators, fed by one bulk
 * copy (cp.async.bulk) per operand and stage from the panel's stored
 * shared-memory image; mode MVB_GEMM_* selects the split precision.
 * K_valid is cut into equal k-slices of at most k_chunk columns (a multiple of
 * 64).  Their count, between ceil(K_valid / k_chunk) and 31 more, is chosen on
 * the device from K_valid so that tiles x slices fills whole waves of SMs; one
 * partial tile is written per (k-slice, tile).  The persistent CTAs take these
 * work units in order from the counter in the workspace; a diagonal tile's
 * imaginary half holds W, with Im V = W - W^T formed by the reductions, so the
 * partial tiles are meant for mvb_herk_reduce* only.
 * drain_ksteps (1, 2 or 4; 0 = default 2) is the number of 32-byte k-steps
 * summed in one TMEM block before the block is added to FP32 registers: the
 * tensor core rounds its accumulator toward zero at every instruction, so short
 * blocks bound that drift; a block's products are issued in ascending
 * magnitude (the hi x hi products last).
 * Replaces GPUMatMul.compute -> zdotz -> cublas.c/zgemm (gpu/matprod.py:31-36,
 * gpu/_cublas.py:7-65) and CPUMatMul.compute's z.conj().dot(z.T)
 * (cpu/matprod.py:11-32); computes only the upper-triangle tiles. */
int mvb_herk(const void *z, int mode, int64_t Mpad, int64_t Kcap, const int32_t *n_dev, int64_t n_host, int kmul,
             int k_chunk, int drain_ksteps, void *ws, size_t ws_bytes, int32_t *status, void *stream);
/* mvb_herk over ngroup panels of one shape in one launch: panel g at
 * z + g * z_stride bytes (z_stride >= mvb_zpanel_bytes(mode, Mpad, Kcap), a
 * multiple of 16), all with the same column count (n_dev / n_host, kmul).  The
 * work units of all panels share the persistent CTAs, and the k-slice plan
 * fills whole waves for ngroup x tiles units; ws holds ngroup x
 * mvb_herk_ws_bytes(Mpad, Kcap, k_chunk) bytes.  Each panel's sums equal
 * those of its own product under that plan.  Replaces the per-frequency
 * GPUMatMul calls (gpu/gpu.py:197-254, wrapper.py:180-199). */
int mvb_herk_grouped(const void *z, size_t z_stride, int ngroup, int mode, int64_t Mpad, int64_t Kcap,
                     const int32_t *n_dev, int64_t n_host, int kmul, int k_chunk, int drain_ksteps, void *ws,
                     size_t ws_bytes, int32_t *status, void *stream);
/* One group of mvb_herk_batch: ngroup panels of one shape, z_stride bytes apart,
 * with the arguments mvb_herk_grouped takes for them. */
typedef struct {
  const void *z;
  size_t z_stride;
  int ngroup;
  int64_t Mpad, Kcap;
  const int32_t *n_dev;
  int64_t n_host;
  int kmul, k_chunk;
  void *ws;
  size_t ws_bytes;
  int32_t *status;
} mvb_herk_group;
/* The products of several panel groups of different shapes -- the current
 * frequency groups of several jobs of a server -- in one launch on the
 * persistent CTAs (at most 32 panels in all).  Every group is planned and
 * summed exactly as its own mvb_herk_grouped call, so the partial tiles in its
 * ws, and the visibilities mvb_herk_reduce_grouped then writes from them, are
 * bit-identical to that call's.  A bounded wait that runs out sets
 * MVB_DEV_TIMEOUT in every group's status word.  Replaces the per-job GPUMatMul
 * calls of jobs run side by side (gpu/matprod.py:31-36); the reference runs one
 * job at a time. */
int mvb_herk_batch(const mvb_herk_group *groups, int ngroups, int mode, int drain_ksteps, void *stream);
/* Sums the FP32 partial tiles over k-slices in float-float (TwoSum, about
 * 2^-44 relative), rounds to FP64 and writes the visibilities in the
 * reference layout out[pair, p, q] = V[ant_i*F + q, ant_j*F + p]
 * (cpu/matprod.py:21-30): all nant^2 pairs (pairs = NULL, i slow) or the
 * npairs listed in pairs (int32 [npairs][2], each entry in [0, nant); an entry
 * outside that range reads nothing and its outputs are NaN).  out: complex64
 * (out_c128 = 0) or complex128, each sum multiplied by vscale (1 / s^2 for
 * MVB_GEMM_F16_3, else 1); accumulate != 0 adds to out (the sum over source
 * chunks).  ws / ws_bytes, Mpad, Kcap, n_dev / n_host, kmul and k_chunk must be
 * those of the mvb_herk call that filled ws: the slice plan is recomputed from
 * them, and the same argument checks apply (ws_bytes at least
 * mvb_herk_ws_bytes(Mpad, Kcap, k_chunk)).
 * Replaces MatProd.sum_chunks and the host transpose/gather of
 * GPUMatMul.sum_chunks (core/matprod.py:103-115, gpu/matprod.py:38-63). */
int mvb_herk_reduce(const void *ws, size_t ws_bytes, int64_t Mpad, int64_t Kcap, const int32_t *n_dev,
                    int64_t n_host, int kmul, int k_chunk, int nant, int nfeed, const int32_t *pairs, int64_t npairs,
                    void *out, int out_c128, double vscale, int accumulate, void *stream);
/* mvb_herk_reduce for the ngroup panels of one mvb_herk_grouped call (same
 * ws, ngroup and shape arguments): panel g's visibilities go to
 * out + g * out_stride bytes. */
int mvb_herk_reduce_grouped(const void *ws, size_t ws_bytes, int ngroup, int64_t Mpad, int64_t Kcap,
                            const int32_t *n_dev, int64_t n_host, int kmul, int k_chunk, int nant, int nfeed,
                            const int32_t *pairs, int64_t npairs, void *out, size_t out_stride, int out_c128,
                            double vscale, int accumulate, void *stream);
/* Wall-time limit, in nanoseconds, of each pipeline wait inside mvb_herk
 * (and its grouped and batched forms) and mvb_vecdot_staged (process-wide; 0
 * restores the default of 4 s).  Returns the previous limit.  A wait that runs
 * out sets MVB_DEV_TIMEOUT in the status word; the kernel then stops issuing
 * work, waits (at most 0.2 s) for the copies and tensor-core operations it
 * issued, releases its tensor memory and returns, so the context stays usable.  For failure-detection tests and diagnostics: a limit shorter
 * than a normal wait makes products fail.  No counterpart in the reference,
 * whose device waits are unbounded (gpu/gpu.py:249). */
uint64_t mvb_set_wait_limit_ns(uint64_t limit_ns);
/* out[i] = sum_c vis[c * n + i] over nchunks per-chunk results (complex64 when
 * c128 = 0, else complex128), accumulated in FP64 in chunk order.
 * Replaces MatProd.sum_chunks (core/matprod.py:103-115). */
int mvb_chunk_sum(const void *vis, int64_t nchunks, int64_t n, int c128, void *out, void *stream);

/* ---- A8: per-pair source sums ----------------------------------------------- */
size_t mvb_vecdot_ws_bytes(int64_t npairs, int nfeed, int64_t Kcap, int k_chunk);
/* out[i, p, q] = sum_k Z[aj*F+p, k] conj(Z[ai*F+q, k]) for (ai, aj) = pairs[i]
 * (each entry in [0, nant), the rows of Z being nant * nfeed)
 * over K_valid columns (as for mvb_herk), Z a plain complex64 panel (row pitch
 * Kcap), one warp per (k-slice, pair), FP64 slice sums in a fixed order.
 * Replaces GPUVectorDot.compute (one cuBLAS call per pair, gpu/matprod.py:66-98)
 * and CPUVectorDot.compute (cpu/matprod.py:35-53). */
int mvb_vecdot(const void *z, int64_t Kcap, const int32_t *n_dev, int64_t n_host, int kmul, int nfeed,
               const int32_t *pairs, int64_t npairs, int k_chunk, void *ws, size_t ws_bytes, void *out, int out_c128,
               int accumulate, void *stream);
/* Staged form of mvb_vecdot: the same output, with the panel read from HBM
 * once.  Three steps: (1) mvb_vecdot_plan, host only, orders a HOST pair list
 * into bundles of 8 int32 {i, j0, j1, j2, pair0, pair1, pair2, flip bits}: up
 * to three pairs sharing antenna i (pair -1: a filler step; flip bit s: pair s
 * is (ai, aj) = (j_s, i)).  plan_bytes from mvb_vecdot_plan_bytes; *nbundles
 * receives the bundle count, a multiple of 32; MVB_ERR_ARG for an antenna
 * outside [0, nant).  Done once per pair list, at the plugin's setup
 * (MatProd.setup -> GPUVectorDot.allocate_vis, core/matprod.py:65,
 * gpu/matprod.py:69-79).  (2) The caller copies the nbundles x 32 plan bytes to
 * the device (16-byte aligned).  (3) mvb_vecdot_staged runs it: nant antennas
 * (the panel's first nant * nfeed rows), npairs outputs, workspace of
 * mvb_vecdot_staged_ws_bytes, k_chunk (the longest k-slice; the kernel picks
 * the slices that fill whole waves of SMs) and Kcap multiples of 16, z 16-byte
 * aligned.  The panel is staged by bulk-tensor copies; every wait is bounded
 * (mvb_set_wait_limit_ns), and one that runs out sets MVB_DEV_TIMEOUT in
 * *status (if not NULL) and ends the kernel.  mvb_vecdot_stage_columns gives the columns of one
 * shared-memory stage (4, 8 or 16), 0 when nant * nfeed rows do not fit (then
 * mvb_vecdot_staged returns MVB_ERR_UNSUPPORTED and mvb_vecdot applies). */
size_t mvb_vecdot_plan_bytes(int64_t npairs, int nfeed);
int mvb_vecdot_plan(const int32_t *pairs, int64_t npairs, int nant, int nfeed, void *plan, size_t plan_bytes,
                    int64_t *nbundles);
int mvb_vecdot_stage_columns(int nant, int nfeed);
size_t mvb_vecdot_staged_ws_bytes(int64_t nbundles, int nfeed, int64_t Kcap, int k_chunk);
int mvb_vecdot_staged(const void *z, int64_t Kcap, const int32_t *n_dev, int64_t n_host, int kmul, int nfeed,
                      int nant, const void *plan, int64_t nbundles, int64_t npairs, int k_chunk, void *ws,
                      size_t ws_bytes, void *out, int out_c128, int accumulate, int32_t *status, void *stream);

/* ---- Polarised sky ------------------------------------------------------- */
/* Frame rotation of the source coherency, per above-horizon source slot s < n
 * (n = *n_dev, or cap): rot[2 s] = cos X, rot[2 s + 1] = sin X of the 2 x 2
 * rotation [[cos X, sin X], [-sin X, cos X]] that carries the coherency from
 * the (ra, dec) basis to the (alt, az) basis.  radec: (2, N) float64 (ra row,
 * dec row, radians); kept: original source index per slot (mvb_horizon_compact's
 * idx_out); crd: (3, ld) topocentric (E, N, U) of the slots; r_avg: host 3 x 3
 * row-major rigid ICRS -> alt/az-cartesian rotation of this time (x north,
 * y east, z up).  Replaces calc_coherency_rotation (coordinates.py:288-330) with
 * the astropy-derived average rotation supplied by the caller; where the
 * rotated and the alt/az unit vectors coincide exactly the perturbation is the
 * identity (the reference's vecs2rot divides 0 by 0 there). */
int mvb_coherency_rotation(const double *radec, int64_t N, const int32_t *kept, const double *crd, int64_t ld,
                           const int32_t *n_dev, int64_t cap, const double *r_avg, double *rot, void *stream);
/* C' = R^T C R for the slots (CoordinateRotation._rotate_frame_coherency,
 * core/coords.py:152-175, and the flux gather of select_chunk, :128-147):
 * coh (N, nf, 2, 2) complex128 -> out (cap, nf, 2, 2) complex128, slots >= n
 * zeroed. */
int mvb_rotate_coherency(const double *rot, const int32_t *kept, const int32_t *n_dev, const void *coh, int64_t N,
                         int nf, void *out, int64_t cap, void *stream);
/* mvb_tau_z for a polarised sky (F = X = 2): the source carries its coherency
 * coh[sidx[s]] = (C00, C11, Re C01, Im C01) float32 (16-byte aligned, one
 * frequency) and rotation rot[s] (from mvb_coherency_rotation); with
 * C' = R^T C R = L L^H, Z[a*2+f, s*2+y] = exptau(a, s) sum_x beam[bidx[a], f, x, s]
 * L[x, y], so that the Hermitian product gives V_ij = exptau_j conj(exptau_i)
 * E_j C' E_i^H, the beam's axis x being the coherency's index.  An unpolarised
 * source (C = I/2 x identity) gives the Z of mvb_tau_z.  No counterpart runs
 * in the reference: its ZMatrixCalc takes a scalar flux only (core/getz.py:80). */
int mvb_tau_z_pol(const double *antpos, int A, double freq, const double *crd, int64_t ld, const int32_t *n_dev,
                  int64_t nsrc, const float *coh, const int32_t *sidx, const double *rot, const void *beam,
                  int64_t beam_ld, int nbeam, const int32_t *beam_idx, int mode, float zscale, void *z, int64_t Mpad,
                  int64_t Kcap, void *stream);
/* mvb_tau_z_pol for nfreq frequencies in one launch, as mvb_tau_z_grouped:
 * freqs a DEVICE array, frequency g's coherency rows at coh + g * coh_ld
 * records of 4 floats, its panel at z + g * z_stride bytes. */
int mvb_tau_z_pol_grouped(const double *antpos, int A, const double *freqs, int nfreq, const double *crd, int64_t ld,
                          const int32_t *n_dev, int64_t nsrc, const float *coh, int64_t coh_ld, const int32_t *sidx,
                          const double *rot, const void *beam, int64_t beam_ld, int nbeam, const int32_t *beam_idx,
                          int mode, float zscale, void *z, size_t z_stride, int64_t Mpad, int64_t Kcap,
                          void *stream);

/* ---- Redundant-baseline pair selection (host memory, no device work) ------- */
/* bls: (nant, nant, 2) float64 baselines, bls[i, j] = pos[j, :2] - pos[i, :2].
 * Writes the pairs (i, j), i < j, that get_redundancies (cli.py:273-290) keeps:
 * baselines rounded to ndecimals decimals as numpy's round does, visited with i
 * slow, kept when neither (u, v) nor (-u, -v) was kept before.  pairs_out is
 * int32 [cap][2]; *n_out receives the count (MVB_ERR_OVERFLOW when it exceeds
 * cap, after counting all of them).  Feeds mvb_vecdot's pair list. */
int mvb_redundant_pairs(const double *bls, int64_t nant, int ndecimals, int32_t *pairs_out, int64_t cap,
                        int64_t *n_out);

#ifdef __cplusplus
}
#endif

#endif /* MATVIS_B200_H */

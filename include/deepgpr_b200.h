/*
 * deepgpr_b200.h -- C ABI of libdeepgpr_b200.so (CUDA, sm_100a).
 *
 * Part 1 is ABI 6 of the reference native library, unchanged in names,
 * parameter order and meaning, so the reference's ctypes bridge
 * (src/DeepGPR/native/abi.py:90-158, loader.py:138-171) can load this file in
 * place of deepgpr.so.  All pointers are device (or UVA-visible) addresses of
 * caller-owned buffers; state arrays are advanced in place; functions return
 * void and report failures through deepgpr_last_error() (per thread).
 *
 * Part 2 are extensions of this library (prefix dgb_).
 */
#ifndef DEEPGPR_B200_H
#define DEEPGPR_B200_H

#define DEEPGPR_ABI_VERSION 6

#ifdef __cplusplus
extern "C" {
#endif

/* ---- Part 1: ABI 6 (src/DeepGPR/lib/deepgpr.h) -------------------------- */

/* src/DeepGPR/lib/deepgpr.h:48-50 -- per-thread error message ("" = success). */
int deepgpr_supports_error_reporting(void);
const char* deepgpr_last_error(void);
void deepgpr_clear_last_error(void);
/* deepgpr.h:53 -- kept for ABI compatibility; this library holds no
 * cross-call resource cache, so it only clears the error message. */
void deepgpr_clear_cuda_resource_cache(void);
/* deepgpr.h:56 -- 1: the adjoint is a deterministic gather (no atomics). */
int deepgpr_deterministic_adjoint(void);
/* deepgpr.h:58 -- returns 6. */
int deepgpr_abi_version(void);
/* deepgpr.h:59-63 -- capability probes.  INT8 histories and the selectable
 * FP16/BF16 conversion / INT8 reduction backends are not provided (0); FP8
 * E4M3 histories replace the INT8 format (see dgb_supports_fp8_history). */
int deepgpr_supports_external_pml(void);
int deepgpr_supports_pml_material_gradients(void);
int deepgpr_supports_int8_wavefield(void);
int deepgpr_supports_conversion_backends(void);
int deepgpr_supports_int8_reduction_backends(void);
/* deepgpr.h:64-70 -- E-only history (storage_type bit 4). */
int deepgpr_supports_rhs_reconstruction(void);
/* deepgpr.h:71-76 -- physical-region history (storage_type bit 5). */
int deepgpr_supports_physical_history(void);
/* deepgpr.h:77-83 -- 2D Ez-TM path (storage_type bit 6). */
int deepgpr_supports_tm2d_fast_path(void);
/* deepgpr.h:87 -- process-global FDTD order (2, 4 or 8; anything else = 2).
 * dgb_set_options() sets a per-thread order that takes precedence. */
void set_fdtd_order(int order);

/* deepgpr.h:89-119 -- forward time loop (src/DeepGPR/lib/deepgpr_cpu.c:1782-1934).
 * storage_type: bits 0-3 history kind (0 FP32, 1 FP16, 2 BF16, 4 FP8 E4M3
 * with per-tile scales, 5 FP64 for dgb_forward_f64), bit 4 E-only history,
 * bit 5 physical history box, bit 6 2D TM path, bit 26 no history. */
void forward(
    const float* eps_r_pad, const float* sigma_pad, const float* mu_r_pad,
    void* E_saved, void* R_saved,
    float* Ex, float* Ey, float* Ez, float* Hx, float* Hy, float* Hz,
    float* ce_hist, float* ce_curl, float* ce_rhs, float* ch_hist, float* ch_curl, float* ch_rhs,
    float* x0_e_phi1, float* x0_e_phi2, float* x0_h_phi1, float* x0_h_phi2,
    float* xm_e_phi1, float* xm_e_phi2, float* xm_h_phi1, float* xm_h_phi2,
    float* y0_e_phi1, float* y0_e_phi2, float* y0_h_phi1, float* y0_h_phi2,
    float* ym_e_phi1, float* ym_e_phi2, float* ym_h_phi1, float* ym_h_phi2,
    float* z0_e_phi1, float* z0_e_phi2, float* z0_h_phi1, float* z0_h_phi2,
    float* zm_e_phi1, float* zm_e_phi2, float* zm_h_phi1, float* zm_h_phi2,
    int pml_x0, int pml_xm, int pml_y0, int pml_ym, int pml_z0, int pml_zm,
    const float* x0_e_coeff, const float* xm_e_coeff, const float* y0_e_coeff,
    const float* ym_e_coeff, const float* z0_e_coeff, const float* zm_e_coeff,
    const float* x0_h_coeff, const float* xm_h_coeff, const float* y0_h_coeff,
    const float* ym_h_coeff, const float* z0_h_coeff, const float* zm_h_coeff,
    float dt, int nt, int nshot, int nreceiver, float dx, float dy, float dz,
    const int* receiver_location, float* receiver_data, int receiver_component,
    int nx_fields, int ny_fields, int nz_fields, int nsource,
    const int* source_location, const float* source_waveform, int source_component,
    int sampling_interval, int fwi_mode, int storage_type, int save_model_history, int use_async_offload);

/* deepgpr.h:121-152 -- exact discrete adjoint (deepgpr_cpu.c:1975-2111);
 * lambda arrays are advanced in place, gradients accumulate (+=). */
void backward(
    const float* eps_r_pad, const float* sigma_pad, const float* mu_r_pad,
    const void* E_saved, const void* R_saved,
    float* lambda_ex, float* lambda_ey, float* lambda_ez,
    float* lambda_hx, float* lambda_hy, float* lambda_hz,
    float* ce_hist, float* ce_curl, float* ce_rhs, float* ch_hist, float* ch_curl, float* ch_rhs,
    float* lambda_x0_e_phi1, float* lambda_x0_e_phi2, float* lambda_x0_h_phi1, float* lambda_x0_h_phi2,
    float* lambda_xm_e_phi1, float* lambda_xm_e_phi2, float* lambda_xm_h_phi1, float* lambda_xm_h_phi2,
    float* lambda_y0_e_phi1, float* lambda_y0_e_phi2, float* lambda_y0_h_phi1, float* lambda_y0_h_phi2,
    float* lambda_ym_e_phi1, float* lambda_ym_e_phi2, float* lambda_ym_h_phi1, float* lambda_ym_h_phi2,
    float* lambda_z0_e_phi1, float* lambda_z0_e_phi2, float* lambda_z0_h_phi1, float* lambda_z0_h_phi2,
    float* lambda_zm_e_phi1, float* lambda_zm_e_phi2, float* lambda_zm_h_phi1, float* lambda_zm_h_phi2,
    int pml_x0, int pml_xm, int pml_y0, int pml_ym, int pml_z0, int pml_zm,
    const float* x0_e_coeff, const float* xm_e_coeff, const float* y0_e_coeff,
    const float* ym_e_coeff, const float* z0_e_coeff, const float* zm_e_coeff,
    const float* x0_h_coeff, const float* xm_h_coeff, const float* y0_h_coeff,
    const float* ym_h_coeff, const float* z0_h_coeff, const float* zm_h_coeff,
    float dt, int nt, int nshot, int nreceiver, float dx, float dy, float dz,
    int nx_fields, int ny_fields, int nz_fields,
    int ndata_source, const int* receiver_location, const float* data_grad, int receiver_component,
    int nsource, const int* source_location, int source_component,
    float* grad_source, int source_requires_grad,
    float* grad_eps_r, float* grad_sigma, int eps_r_requires_grad, int sigma_requires_grad,
    int sampling_interval, int fwi_mode, int storage_type, int use_async_offload);

/* ---- Part 2: extensions ------------------------------------------------- */

/* Version of the extension set (1). */
int dgb_version(void);
/* 1: storage kind 4 (FP8 E4M3, one FP32 scale per forward CTA tile) is accepted. */
int dgb_supports_fp8_history(void);

/* Stream of the calling thread's following forward/backward calls (a
 * cudaStream_t; 0 is the legacy default stream).  Without it, calls are
 * ordered after the legacy default stream, as the reference's are.  Work runs
 * on a private stream that is joined back to this stream with events. */
int dgb_set_stream(void* stream);
void dgb_clear_stream(void);

/* Per-thread options: acc64 = 1 sums the material gradient over shots and
 * time in FP64 (default), 0 in FP32 in the reference's order; chunk_steps =
 * time steps per launch chunk (1..4096, default 16); use_graph = 1 captures a
 * chunk into a CUDA graph and replays it; fdtd_order 2/4/8 overrides
 * set_fdtd_order for this thread (0 = use the global).  Returns 0, or -1 for
 * an invalid chunk. */
int dgb_set_options(int acc64, int chunk_steps, int use_graph, int fdtd_order);

/* Bytes of one history buffer (E_saved or R_saved) for a storage kind.
 * ncomp = 1 (mode 2) or 3 (mode 3); box_cells = cells of one frame of one
 * shot; NX, NY, NZ = field extents; tm2d = 1 when the 2D TM path is used
 * (it sets the FP8 tile geometry). */
long long dgb_history_bytes(int kind, int ncomp, int nt_saved, int nshot, long long box_cells,
                            int NX, int NY, int NZ, int tm2d);

/* FP64 instantiations of forward/backward: the same kernels in double
 * (the FP64 reference of the FP32 path).  Same parameter lists with every
 * float / float* replaced by double / double*; histories use kind 5. */
void dgb_forward_f64(/* forward's parameters, float -> double */);
void dgb_backward_f64(/* backward's parameters, float -> double */);

/* No counterpart in the reference.  forward() without device memory
 * allocation, for callers that cannot allocate during a solve: a serving
 * process whose free GPU memory belongs to its own pool (an allocation would
 * fail or make the pool trim), or code holding a fixed per-request memory
 * budget.  Same parameters, results and errors as forward().  Its device
 * scratch (control block, source / receiver tables and bitmaps, the pitched
 * 2D working copy) is a static array of DGB_NOALLOC_SCRATCH_BYTES (8 MiB) per
 * device; a solve whose scratch does not fit is rejected through
 * deepgpr_last_error() before any time step runs.  Every call looks up the
 * array's device address; the first call on a new thread also creates the
 * library's stream and events for that thread: make it before any stream
 * capture.  All calls on a device share the array, so overlapping calls (two
 * threads, or two streams) race. */
#define DGB_NOALLOC_SCRATCH_BYTES 8388608
void dgb_forward_noalloc(
    const float* eps_r_pad, const float* sigma_pad, const float* mu_r_pad,
    void* E_saved, void* R_saved,
    float* Ex, float* Ey, float* Ez, float* Hx, float* Hy, float* Hz,
    float* ce_hist, float* ce_curl, float* ce_rhs, float* ch_hist, float* ch_curl, float* ch_rhs,
    float* x0_e_phi1, float* x0_e_phi2, float* x0_h_phi1, float* x0_h_phi2,
    float* xm_e_phi1, float* xm_e_phi2, float* xm_h_phi1, float* xm_h_phi2,
    float* y0_e_phi1, float* y0_e_phi2, float* y0_h_phi1, float* y0_h_phi2,
    float* ym_e_phi1, float* ym_e_phi2, float* ym_h_phi1, float* ym_h_phi2,
    float* z0_e_phi1, float* z0_e_phi2, float* z0_h_phi1, float* z0_h_phi2,
    float* zm_e_phi1, float* zm_e_phi2, float* zm_h_phi1, float* zm_h_phi2,
    int pml_x0, int pml_xm, int pml_y0, int pml_ym, int pml_z0, int pml_zm,
    const float* x0_e_coeff, const float* xm_e_coeff, const float* y0_e_coeff,
    const float* ym_e_coeff, const float* z0_e_coeff, const float* zm_e_coeff,
    const float* x0_h_coeff, const float* xm_h_coeff, const float* y0_h_coeff,
    const float* ym_h_coeff, const float* z0_h_coeff, const float* zm_h_coeff,
    float dt, int nt, int nshot, int nreceiver, float dx, float dy, float dz,
    const int* receiver_location, float* receiver_data, int receiver_component,
    int nx_fields, int ny_fields, int nz_fields, int nsource,
    const int* source_location, const float* source_waveform, int source_component,
    int sampling_interval, int fwi_mode, int storage_type, int save_model_history, int use_async_offload);

/* Diagnostic, no counterpart in the reference.  The single-precision
 * kernels divide by a grid spacing, by dt and by per-cell coefficients
 * through an FMA path (Markstein's correction from the correctly rounded
 * reciprocal) that is meant to round exactly like the division operator.
 * This runs that path and the operator for one divisor over all 2^32 float
 * dividends on the current device and reports the number of results whose
 * bits differ and the lowest such dividend bit pattern (0xffffffff if none).
 * Synchronous; returns 0, or -1 with deepgpr_last_error() set. */
int dgb_check_fixed_division(float divisor, unsigned long long* mismatches, unsigned* first_bad);

/* No counterpart in the reference.  The solver's per-call device scratch
 * (working copies, point tables, CPML weights) comes from the current device's
 * default stream-ordered memory pool.  With the CUDA default the pool gives
 * freed memory back at every synchronisation and every call maps its scratch
 * again (on virtualised hosts such mappings stalled back-to-back solves by
 * up to 0.6 s), so on first use of a device the library keeps up to
 * min(4 GiB, 1/32 of the device memory) cached.  A caller sets the amount
 * instead: `bytes` (-1: no limit; 0: the CUDA default, and the pool is
 * trimmed now).  Affects every stream-ordered allocation of the process on
 * that device.  Returns 0, or -1 with deepgpr_last_error() set. */
int dgb_set_scratch_retention(long long bytes);

/* No counterpart in the reference.  Launch-shape choices for the calling
 * thread's next solves (set by deepgpr_b200.autotune): 2D interior row
 * chunks, 2D frame rows per warp chunk, 3D x chunks, 3D FP32 forward kernel
 * family (2 wide, 1 TMA-staged, 0 z-streamed; -1 the environment choice:
 * DEEPGPR_B200_TMA=1 staged, DEEPGPR_B200_NARROW=1 z-streamed, else wide).
 * 0 / -1 restore the built-in heuristics; results do not depend on them.
 * Returns 0, or -1 for out-of-range values. */
int dgb_set_tuning(int tm_chunks, int tm_frame_rows, int k3_xchunks, int tma);

/* No counterpart in the reference (diagnostic).  Bytes in use in the current
 * device's default stream-ordered memory pool (the pool cudaMallocAsync draws
 * on) and its high-water mark; reset_high != 0 first resets the mark to the
 * current use.  Returns 0, or -1 with deepgpr_last_error() set. */
int dgb_default_pool_usage(long long* used, long long* high, int reset_high);

/* Process-wide kernel timing (CUDA events around every time-step
 * kernel; graph replay is off while enabled).  dgb_profile(1) clears the
 * totals; dgb_profile_read fills ms[k] and launches[k] for the kinds
 * 0 forward-H, 1 forward-E, 2 adjoint-E, 3 adjoint-H, 4 imaging condition,
 * and returns the number of kinds (5). */
void dgb_profile(int enable);
int dgb_profile_read(double* ms, long long* launches, int n);
/* Time-step kernels launched by the library, all threads (graph replays included). */
long long dgb_launch_count(void);

#ifdef __cplusplus
}
#endif

#endif /* DEEPGPR_B200_H */

/*
 * gpufft-b200 — C ABI of the B200 (sm_100a) polynomial-multiplication library.
 *
 * Every function returns a gpufft_status code (0 = success). Pointers are
 * device pointers owned by the caller unless a comment says otherwise; the
 * library keeps no per-call state. Work is enqueued asynchronously on
 * `stream` (a cudaStream_t; NULL is the legacy default stream), exactly as the
 * reference's GPU_FFT / GPU_FFNT enqueue on cfg.stream and never synchronize
 * (reference src/lib/fft.cu:517-725, 1386-1515).
 *
 * Complex buffers use the reference's COMPLEX<T> layout: interleaved
 * (re, im) float2 / double2 (reference src/include/gpufft/complex.cuh:28-34,
 * 315-318).
 */
#ifndef GPUFFT_B200_H
#define GPUFFT_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* gpufft_stream_t; /* identical to cudaStream_t */

enum gpufft_status
{
    GPUFFT_SUCCESS = 0,
    /* n_power outside the supported range; the C++ drop-in maps this to
     * std::invalid_argument("Invalid n_power range!") (reference fft.cu:522-525) */
    GPUFFT_ERROR_INVALID_N_POWER = 1,
    /* a null pointer, a non-positive batch, an unknown enum value, or a size
     * whose element count does not fit the kernels' 64-bit indexing */
    GPUFFT_ERROR_INVALID_VALUE = 2,
    /* a CUDA call or kernel launch failed: gpufft_last_cuda_error() holds the
     * cudaError_t, which the C++ drop-in rethrows as gpufft::CudaException
     * (reference common_fft.cuh:19-49) */
    GPUFFT_ERROR_CUDA = 3,
    /* the caller's workspace is smaller than the *_workspace_bytes query */
    GPUFFT_ERROR_WORKSPACE = 4,
    /* a device pointer is not aligned to its element type (8/16 bytes) */
    GPUFFT_ERROR_MISALIGNED = 5
};

/* gpufft::type (reference fft.cuh:37-41) */
enum { GPUFFT_FORWARD = 0, GPUFFT_INVERSE = 1 };
/* gpufft::ReductionPolynomial (reference fft_cpu.cuh:69-73) */
enum { GPUFFT_X_N_PLUS = 0, GPUFFT_X_N_MINUS = 1 };

/* Per-kernel device-time tracing (no reference counterpart). While enabled,
 * each kernel launch of the library's entry points (outside stream capture)
 * is bracketed by two CUDA events on its stream and tagged with the kernel's
 * name and the algorithmic bytes it moves (inputs read once, outputs written
 * once). gpufft_trace_collect waits for the recorded events, returns up to
 * max_rows per-kernel totals (names NUL-terminated in slots of name_len bytes,
 * summed milliseconds, summed bytes, launch counts) and clears the records. */
int gpufft_trace_enable(int on);
int gpufft_trace_collect(int max_rows, char* names, int name_len, double* total_ms, double* alg_bytes,
                         long long* launches, int* rows);

/* Launches whose contiguous 12-stage pass covers at most max_tiles tiles of
 * 4096 points (small batches: N = 2^13..2^23 with few products) spread each
 * tile over a cluster of 8 CTAs instead of one CTA; results are bit-identical
 * either way. max_tiles = 0 disables the cluster form; a negative value only
 * queries. Returns the previous limit (default 64). Process-wide (an atomic
 * setting: calls on other threads see either the old or the new limit). */
int gpufft_set_cluster_tiles(int max_tiles);

/* The kernels of the transform and product chains are launched with CUDA's
 * programmatic stream serialization (programmatic dependent launch): a
 * kernel's CTAs may be scheduled while the previous kernel in the stream
 * runs, and each waits (griddepcontrol.wait) for that kernel to complete
 * before touching memory, which hides most of the launch gap between the
 * short kernels of small batches. Results are identical either way; on = 0
 * launches in plain stream order. A negative value only queries. Returns the
 * previous setting (default 1). Process-wide (atomic). */
int gpufft_set_programmatic_launch(int on);

/* The middle pass of the two-pass FP64 products (the last 12 forward stages of
 * both operands, their product, the first 12 inverse stages of each 4096-point
 * tile) runs on 512 threads of 8 points per operand (r8 = 1, the default) or
 * on 256 threads of 16 (r8 = 0). The values are identical. A negative value
 * only queries. Returns the previous setting. Process-wide (atomic). */
int gpufft_set_f64_middle(int r8);

/* The cudaError_t of the last GPUFFT_ERROR_CUDA raised on this host thread. */
int gpufft_last_cuda_error(void);
/* A static, human-readable string for a gpufft_status value. */
const char* gpufft_status_string(int status);
/* Library version as MAJOR*10000 + MINOR*100 + PATCH. */
int gpufft_version(void);

/* ------------------------------------------------------------------------ */
/* Drop-in transforms (the reference's GPU_FFT / GPU_FFNT, same arguments).  */
/* n_power is accepted in [1, 24] for the FFT and [2, 25] for the FFNT; the  */
/* C++ and Python drop-in layers add the reference's [12, 24] check.         */
/* ------------------------------------------------------------------------ */

/* Replaces GPU_FFT(COMPLEX<T>* device_inout, COMPLEX<T>* root_of_unity_table,
 * fft_configuration<T> cfg, int batch_size, bool multiplication)
 * — reference fft.cuh:120-124, fft.cu:517-598.
 * Forward: `batch` in-place transforms of 2^n_power complex values, natural
 * order in, +sign DFT in bit-reversed order out. Inverse: with multiplication
 * the operand is inout[i] * inout[i + batch*2^n_power]; the result (scaled by
 * mod_inverse) overwrites the first `batch` vectors. */
int gpufft_fft_c2c_f32(void* inout, const void* root_table, int n_power, int fft_type,
                       int reduction_poly, int zero_padding, float mod_inverse_re,
                       float mod_inverse_im, int batch, int multiplication, gpufft_stream_t stream);
int gpufft_fft_c2c_f64(void* inout, const void* root_table, int n_power, int fft_type,
                       int reduction_poly, int zero_padding, double mod_inverse_re,
                       double mod_inverse_im, int batch, int multiplication, gpufft_stream_t stream);

/* Replaces GPU_FFT(T* device_fix_inout, COMPLEX<T>* device_Complex64_inout,
 * COMPLEX<T>* root_of_unity_table, fft_configuration<T> cfg, int batch_size,
 * bool multiplication) — reference fft.cuh:126-132, fft.cu:600-725.
 * Forward: reals in real_inout -> complex spectra in temp. Inverse: spectra in
 * temp (product of the two halves when multiplication) -> real parts in
 * real_inout. With zero_padding the upper half of every forward input vector
 * is taken as zero and not read. */
int gpufft_fft_r2r_f32(float* real_inout, void* temp, const void* root_table, int n_power,
                       int fft_type, int reduction_poly, int zero_padding, float mod_inverse_re,
                       float mod_inverse_im, int batch, int multiplication, gpufft_stream_t stream);
int gpufft_fft_r2r_f64(double* real_inout, void* temp, const void* root_table, int n_power,
                       int fft_type, int reduction_poly, int zero_padding, double mod_inverse_re,
                       double mod_inverse_im, int batch, int multiplication, gpufft_stream_t stream);

/* Replaces GPU_FFNT(T* device_inout, COMPLEX<T>* device_temp,
 * COMPLEX<T>* twist_table, COMPLEX<T>* root_of_unity_table,
 * fft_configuration<T> cfg, int batch_size, bool multiplication)
 * — reference fft.cuh:269-273, fft.cu:1386-1515.
 * N = 2^n_power reals per polynomial, transforms of N/2 complex. Forward: fold,
 * twist, transform into temp. Inverse (twist_table = the UNTWIST table, as
 * the reference's callers pass it): product, inverse transform, scale by
 * mod_inverse, untwist, unfold into inout. */
int gpufft_ffnt_f32(float* inout, void* temp, const void* twist_table, const void* root_table,
                    int n_power, int fft_type, float mod_inverse_re, float mod_inverse_im, int batch,
                    int multiplication, gpufft_stream_t stream);
int gpufft_ffnt_f64(double* inout, void* temp, const void* twist_table, const void* root_table,
                    int n_power, int fft_type, double mod_inverse_re, double mod_inverse_im, int batch,
                    int multiplication, gpufft_stream_t stream);

/* Host-side twiddle tables of the drop-in API, written to HOST buffers:
 * FFT<T>(n).ReverseRootTable / InverseReverseRootTable (n complex each) and
 * n_inverse (one T) — reference fft_cpu.cu:93-128, 200-226; and
 * FFNT<T>(n) ReverseRootTable_ffnt / InverseReverseRootTable_ffnt /
 * twist_table_ffnt / untwist_table_ffnt (n/2 complex each) — reference
 * fft_cpu.cu:234-300, 435-473. Same values bit for bit. n is a power of two. */
int gpufft_host_fft_tables_f32(int n, void* roots, void* inv_roots, void* n_inverse);
int gpufft_host_fft_tables_f64(int n, void* roots, void* inv_roots, void* n_inverse);
int gpufft_host_ffnt_tables_f32(int n, void* roots, void* inv_roots, void* twist, void* untwist);
int gpufft_host_ffnt_tables_f64(int n, void* roots, void* inv_roots, void* twist, void* untwist);

/* ------------------------------------------------------------------------ */
/* Native fused products (no reference counterpart as single calls: each one */
/* replaces the pair GPU_FFNT(FORWARD, 2*batch) + GPU_FFNT(INVERSE, batch,  */
/* multiplication) of reference fft.cu:1386-1515 / example                  */
/* test_ffnt_gpu_R_R.cu:145-157, without writing the spectra to memory).    */
/* ------------------------------------------------------------------------ */

/* Number of complex entries of the native FFNT twiddle block for N = 2^n_power:
 * [roots N/4 | inverse roots N/4 | twist N/2 | untwist N/2 | U N/2] (0 if out of
 * range, n_power in [2, 25]). The first four hold the values of
 * FFNT<T>::ReverseRootTable_ffnt, InverseReverseRootTable_ffnt,
 * twist_table_ffnt, untwist_table_ffnt (reference fft_cpu.cu:435-473); U is
 * the transform of the all-ones polynomial (used by the split product; for
 * N > 8192 stored in that product's spectrum order, each block of 4096
 * entries permuted e -> (e >> 4) + 256 (e & 15)). All are computed on the
 * device with sincospi; each odd root is stored as exactly i times its even
 * neighbour (bit reversal makes their angles a quarter turn apart), and the
 * inverse roots as exact conjugates. */
size_t gpufft_ffnt_tables_count(int n_power);
int gpufft_ffnt_make_tables_f32(int n_power, void* tables, gpufft_stream_t stream);
int gpufft_ffnt_make_tables_f64(int n_power, void* tables, gpufft_stream_t stream);

/* ------------------------------------------------------------------------ */
/* GPU_Special_FFT (reference fft.cuh:194-197, fft.cu:929-1007): the special */
/* FFT of CKKS encoding on batch vectors of 2^n_power complex, in place.     */
/* The span-t butterfly of the pair (i, i + t) uses table[t + (i mod t)]      */
/* (the table has 2^n_power entries); FORWARD runs spans 1 .. 2^(n-1) with   */
/* Cooley-Tukey butterflies, INVERSE runs them back with Gentleman-Sande     */
/* butterflies and multiplies by mod_inverse. n_power in [1, 24] here (the   */
/* reference accepts 11..24; the C++ and Python mirrors keep that range).    */
/* ------------------------------------------------------------------------ */
int gpufft_special_fft_f32(void* inout, const void* table, int n_power, int fft_type, float mod_inverse_re,
                           float mod_inverse_im, int batch, gpufft_stream_t stream);
int gpufft_special_fft_f64(void* inout, const void* table, int n_power, int fft_type, double mod_inverse_re,
                           double mod_inverse_im, int batch, gpufft_stream_t stream);

/* Workspace for gpufft_negacyclic_mul_* (precision_bits 32 or 64); 0 when the
 * ring needs none (N <= 8192). Passing more lets larger waves run per launch. */
size_t gpufft_negacyclic_mul_workspace_bytes(int n_power, int batch, int precision_bits);

/* c[k] = a[k] * b[k] mod (X^N + 1) for k < batch, N = 2^n_power in [4, 2^22].
 * a, b, c: batch x N reals (row-major); c may alias a or b. `tables` is the
 * native twiddle block above, as gpufft_ffnt_make_tables_* writes it (the
 * kernels rely on its exact relations: roots[2j+1] = i roots[2j], inverse
 * roots the exact conjugates). The output is not rounded (as GPU_FFNT). */
int gpufft_negacyclic_mul_f32(const float* a, const float* b, float* c, int n_power, int batch,
                              const void* tables, void* workspace, size_t workspace_bytes,
                              gpufft_stream_t stream);
int gpufft_negacyclic_mul_f64(const double* a, const double* b, double* c, int n_power, int batch,
                              const void* tables, void* workspace, size_t workspace_bytes,
                              gpufft_stream_t stream);

/* The same product on HOST buffers (page-locked for overlap): the batch runs in
 * chunks of `chunk` products (0: the library's choice), each copied in, computed
 * and copied out on its own streams so that the PCIe transfers of neighbouring
 * chunks overlap the computation. Ordered after the work queued on `stream`,
 * and `stream` waits for the last copy: synchronise it before reading c. The
 * workspace holds three staging slots plus one chunk's product workspace. */
size_t gpufft_negacyclic_mul_host_workspace_bytes(int n_power, int batch, int chunk, int precision_bits);
int gpufft_negacyclic_mul_f32_host(const float* a, const float* b, float* c, int n_power, int batch, int chunk,
                                   const void* tables, void* workspace, size_t workspace_bytes,
                                   gpufft_stream_t stream);
int gpufft_negacyclic_mul_f64_host(const double* a, const double* b, double* c, int n_power, int batch, int chunk,
                                   const void* tables, void* workspace, size_t workspace_bytes,
                                   gpufft_stream_t stream);

/* Cyclic product of complex vectors, c[k] = a[k] * b[k] mod (X^M - 1),
 * M = 2^n_power (n_power in [1, 21]): the C_C product the reference forms with
 * GPU_FFT (forward of both operands, then the inverse with multiplication and
 * mod_inverse 1/M; reference fft.cu:517-598, example test_fft_gpu_C_C.cu),
 * fused into one kernel chain. a, b, c: batch x M COMPLEX<T> (row-major).
 * `tables` is the native block of the ring 2M (gpufft_ffnt_make_tables_* with
 * n_power + 1): its roots are FFT<T>(M/2)'s bit-reversed table. */
size_t gpufft_cyclic_mul_workspace_bytes(int n_power, int batch, int precision_bits);
int gpufft_cyclic_mul_f32(const void* a, const void* b, void* c, int n_power, int batch, const void* tables,
                          void* workspace, size_t workspace_bytes, gpufft_stream_t stream);
int gpufft_cyclic_mul_f64(const void* a, const void* b, void* c, int n_power, int batch, const void* tables,
                          void* workspace, size_t workspace_bytes, gpufft_stream_t stream);

/* Linear product of real polynomials, the product the reference forms with
 * GPU_FFT R_R on zero-padded inputs (reference fft.cu:600-725, example
 * test_fft_gpu_R_R.cu:153-164): c[k] = a[k] * b[k], a and b rows of
 * N = 2^n_power (n_power in [1, 21]), c rows of 2N (the last entry is 0).
 * `tables` is the native block for the ring 2N (gpufft_ffnt_make_tables_* with
 * n_power + 1). Computed as a negacyclic product of length 2N whose zero upper
 * halves make each operand a real half-length transform. Not rounded. */
size_t gpufft_linear_mul_workspace_bytes(int n_power, int batch, int precision_bits);
int gpufft_linear_mul_f32(const float* a, const float* b, float* c, int n_power, int batch, const void* tables,
                          void* workspace, size_t workspace_bytes, gpufft_stream_t stream);
int gpufft_linear_mul_f64(const double* a, const double* b, double* c, int n_power, int batch,
                          const void* tables, void* workspace, size_t workspace_bytes, gpufft_stream_t stream);

/* Vector-Jacobian product of gpufft_linear_mul_f32 (no reference counterpart):
 * for an upstream gradient g (rows of 2N), grad_a[i] = sum_k g[k] b[k-i] and
 * grad_b[j] = sum_k g[k] a[k-j] (rows of N), computed as the correlation
 * IFFT(G conj(B)), IFFT(G conj(A)) through the same fused transform chain.
 * n_power in [1, 20]; tables as for gpufft_linear_mul_f32. */
size_t gpufft_linear_mul_vjp_workspace_bytes(int n_power, int batch);
int gpufft_linear_mul_vjp_f32(const float* g, const float* a, const float* b, float* grad_a, float* grad_b,
                              int n_power, int batch, const void* tables, void* workspace, size_t workspace_bytes,
                              gpufft_stream_t stream);
/* Alias of gpufft_linear_mul_vjp_f32 (convolution naming). */
int gpufft_conv_vjp_f32(const float* g, const float* a, const float* b, float* grad_a, float* grad_b, int n_power,
                        int batch, const void* tables, void* workspace, size_t workspace_bytes,
                        gpufft_stream_t stream);

/* ------------------------------------------------------------------------ */
/* Batched products of mixed ring sizes (no reference counterpart: the      */
/* reference runs one ring size per call). One plan holds the twiddles,      */
/* workspace and work lists of a fixed list of requests; execution is one    */
/* persistent cooperative launch (capturable in a CUDA graph).               */
/* ------------------------------------------------------------------------ */
typedef struct gpufft_batch_plan_s* gpufft_batch_plan;

/* Plan for `count` negacyclic products with rings N_i = 2^n_powers[i]
 * (n_powers in [2, 17]); precision_bits 64 (double) or 32 (float). Allocates
 * the plan's device memory (tables, workspace); synchronises `stream`. */
int gpufft_batch_plan_create(gpufft_batch_plan* plan, const int* n_powers, int count, int precision_bits,
                             gpufft_stream_t stream);
/* The packed layout the plan expects for a, b and c: requests grouped by ring
 * size. order[k] is the request stored k-th, offsets[i] the coefficient offset
 * of request i in the packed arrays, *total their length. Any may be NULL. */
int gpufft_batch_plan_layout(gpufft_batch_plan plan, int* order, long long* offsets, long long* total);
/* c = a * b for every request on `stream`: one persistent launch, or (when
 * the autotuner found it faster) one fused chain per ring-size class. */
int gpufft_batch_plan_execute(gpufft_batch_plan plan, const void* a, const void* b, void* c, gpufft_stream_t stream);
/* Alias of gpufft_batch_plan_execute (create / run / destroy naming). */
int gpufft_batch_plan_run(gpufft_batch_plan plan, const void* a, const void* b, void* c, gpufft_stream_t stream);
/* Time the candidates on these buffers and keep the fastest: the persistent
 * launch with 1 or 2 CTAs per SM and 1, 2 or 4 work items per grab, and the
 * per-class fused chains (reported as 0 CTAs per SM by _info). cache_path (may
 * be NULL) is a JSON-lines file of earlier results keyed by GPU, driver,
 * precision and size histogram. The candidates run on the caller's buffers
 * about 28 times, so c must not overlap a or b (GPUFFT_ERROR_INVALID_VALUE). */
int gpufft_batch_plan_autotune(gpufft_batch_plan plan, const void* a, const void* b, void* c,
                               const char* cache_path, gpufft_stream_t stream);
/* Choose the execution mode by hand: ctas_per_sm 1 or 2 (persistent launch,
 * items_per_grab 1..8), or 0 (per-class fused chains). */
int gpufft_batch_plan_set_shape(gpufft_batch_plan plan, int ctas_per_sm, int items_per_grab);
/* Capture one execution on these buffers into a CUDA graph held by the plan
 * (stream must be a non-default stream), then launch it with _replay. */
int gpufft_batch_plan_capture(gpufft_batch_plan plan, const void* a, const void* b, void* c, gpufft_stream_t stream);
int gpufft_batch_plan_replay(gpufft_batch_plan plan, gpufft_stream_t stream);
/* Launch shape in use, grid size of the last launch, workspace size. */
int gpufft_batch_plan_info(gpufft_batch_plan plan, int* ctas_per_sm, int* items_per_grab, int* grid,
                           long long* workspace_bytes);
/* Reads and clears the plan's barrier-timeout flag (synchronous). */
int gpufft_batch_plan_status(gpufft_batch_plan plan, int* barrier_timeouts);
/* The persistent launch's grid barriers give up after max_polls polls of
 * about 64 ns each (default 2^26, several seconds) and set the timeout flag.
 * extra_arrivals (default 0, at most 1024) raises every barrier's target above
 * the grid size so that no barrier can complete: it exists only to make the
 * bounded wait run out in a test (the results of such a run are meaningless;
 * the kernel still returns and the context stays usable). */
int gpufft_batch_plan_set_barrier(gpufft_batch_plan plan, unsigned max_polls, unsigned extra_arrivals);
int gpufft_batch_plan_destroy(gpufft_batch_plan plan);

/* Allocation-free gpufft_negacyclic_mul_f64, for callers that cannot call
 * cudaMalloc (code running inside another runtime's device memory pool, plugin
 * hosts that own every device allocation, processes that must not grow their
 * device footprint after start-up). No reference counterpart. Scratch is a
 * 16 MiB library-owned device array that every GPU loading the library holds
 * until exit; every call looks up its address on the current device (the
 * first call there also loads the module), so make the first call on a device
 * before any stream capture. Rings with N > 2^20 return GPUFFT_ERROR_WORKSPACE.
 * All calls share the array: calls that overlap on the GPU race on it. */
int gpufft_negacyclic_mul_f64_noalloc(const double* a, const double* b, double* c, int n_power, int batch,
                                      const void* tables, gpufft_stream_t stream);

/* ------------------------------------------------------------------------ */
/* FP32 split-precision negacyclic product with exact int64 output (no      */
/* reference counterpart: the reference's products are plain FP32/FP64).     */
/* ------------------------------------------------------------------------ */

/* The limb plan (width, count) the library picks for rings of 2^n_power with
 * |coefficients| < 2^input_bits (non_negative: all coefficients >= 0). */
int gpufft_split_plan(int n_power, int input_bits, int non_negative, int* limb_bits, int* num_limbs);
/* Workspace for gpufft_negacyclic_mul_split_f32 with num_limbs limbs. */
size_t gpufft_negacyclic_mul_split_workspace_bytes(int n_power, int batch, int num_limbs);
/* c[k] = a[k] * b[k] mod (X^N + 1), exact in int64 (wrapping mod 2^64), from
 * int32 coefficients with |x| < 2^input_bits, N = 2^n_power in [4, 2^22].
 * Limbs: limb_bits/num_limbs, or 0/0 for the plan of gpufft_split_plan.
 * `tables` is the f32 native twiddle block (gpufft_ffnt_make_tables_f32).
 * max_error (device pointer, may be NULL; the call zeroes it first) receives
 * the largest distance of any limb-group value to its nearest integer.
 *
 * What max_error certifies. Every result coefficient is exact when the
 * floating-point error of every limb-group value is below 0.5. max_error
 * measures the distance to the NEAREST integer, so it detects errors up to
 * 0.5 but does not prove their absence: a value whose error exceeded 0.5 would
 * sit near a wrong integer and could report a small distance. A worst-case
 * (a-priori) bound for FP32 transforms of these lengths is orders of magnitude
 * above 0.5, so exactness is statistical: the limb plan (gpufft_split_plan)
 * keeps the predicted largest error at or below 0.2, from an error model
 * calibrated on measured limb products, and the measured max_error on uniform
 * 24-bit data is about 0.13 at N = 2^16 and 0.22 at N = 2^17. Group values
 * above 2^22 report 1.0 (not certified), a timed-out internal wait reports
 * +inf (see gpufft_split_wait_timeouts). */
int gpufft_negacyclic_mul_split_f32(const int32_t* a, const int32_t* b, int64_t* c, int n_power, int batch,
                                    int input_bits, int non_negative, int limb_bits, int num_limbs,
                                    const void* tables, void* workspace, size_t workspace_bytes,
                                    float* max_error, gpufft_stream_t stream);
/* Rings N = 2^14 .. 2^16 with at most five limbs (with a 16-byte aligned
 * workspace, and at least one 2048-point tile per SM per wave: 10 products at
 * N = 2^16) run the contiguous stages of every limb and limb group in one
 * persistent kernel that keeps a product
 * tile's limb spectra in shared memory (on = 1, the default), or in the chain
 * of separate pass and group-sum kernels (on = 0); the integers are the same.
 * A negative value only queries. Returns the previous setting. Process-wide. */
int gpufft_set_split_tile(int on);
/* Waits of that kernel on its bulk copies are bounded (2 s); a wait that runs
 * out makes the call report max_error = +inf and is counted here. Reads the
 * count (synchronous) and clears it when `clear` is nonzero. */
int gpufft_split_wait_timeouts(unsigned* count, int clear);
/* The same exact product with FP64 transforms, N = 2^2 .. 2^17 (no reference
 * counterpart). Its limb plan uses the FP64 error model, so it needs far fewer
 * limbs (two 12-bit limbs for 24-bit coefficients at N = 2^16). `tables` is the
 * f64 native twiddle block (gpufft_ffnt_make_tables_f64). */
int gpufft_split_plan_f64(int n_power, int input_bits, int non_negative, int* limb_bits, int* num_limbs);
size_t gpufft_negacyclic_mul_split_f64_workspace_bytes(int n_power, int batch, int num_limbs);
int gpufft_negacyclic_mul_split_f64(const int32_t* a, const int32_t* b, int64_t* c, int n_power, int batch,
                                    int input_bits, int non_negative, int limb_bits, int num_limbs,
                                    const void* tables, void* workspace, size_t workspace_bytes,
                                    float* max_error, gpufft_stream_t stream);

/* Mixed ring sizes, exact (no reference counterpart): the split product over
 * a packed batch of requests of different ring sizes (N = 4 .. 2^22). Requests
 * are grouped by size, class-major with the original order inside a class;
 * _layout gives each request's coefficient offset in the packed int32 inputs
 * and int64 output, the packed length, and each request's limb plan. Each
 * class runs the split chain with its own limbs and twiddles on one stream;
 * _capture records one execution on these buffers as a CUDA graph (non-default
 * stream) that _replay launches. max_error (device, may be NULL) covers every
 * class. The plan owns its twiddles and workspace. */
typedef struct gpufft_split_batch_plan_s* gpufft_split_batch_plan;
int gpufft_split_batch_plan_create(gpufft_split_batch_plan* plan, const int* n_powers, int count, int input_bits,
                                   int non_negative, gpufft_stream_t stream);
int gpufft_split_batch_plan_layout(gpufft_split_batch_plan plan, long long* offsets, long long* total,
                                   int* limb_bits, int* num_limbs);
int gpufft_split_batch_plan_execute(gpufft_split_batch_plan plan, const int32_t* a, const int32_t* b, int64_t* c,
                                    float* max_error, gpufft_stream_t stream);
int gpufft_split_batch_plan_capture(gpufft_split_batch_plan plan, const int32_t* a, const int32_t* b, int64_t* c,
                                    float* max_error, gpufft_stream_t stream);
int gpufft_split_batch_plan_replay(gpufft_split_batch_plan plan, gpufft_stream_t stream);
int gpufft_split_batch_plan_destroy(gpufft_split_batch_plan plan);

/* The same product on host buffers, chunked with overlapped transfers exactly
 * like gpufft_negacyclic_mul_f64_host; max_error (device) covers all chunks. */
size_t gpufft_negacyclic_mul_split_f32_host_workspace_bytes(int n_power, int batch, int chunk, int num_limbs);
int gpufft_negacyclic_mul_split_f32_host(const int32_t* a, const int32_t* b, int64_t* c, int n_power, int batch,
                                         int chunk, int input_bits, int non_negative, int limb_bits, int num_limbs,
                                         const void* tables, void* workspace, size_t workspace_bytes,
                                         float* max_error, gpufft_stream_t stream);

#ifdef __cplusplus
} /* extern "C" */
#endif

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#endif /* GPUFFT_B200_H */

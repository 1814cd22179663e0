/*
 * Thin C-ABI device layer under the phasing API (libspimage_b200.so).
 *
 * Plain pointers and sizes only.  The host C library (sp_phaser_* etc.) calls
 * these; an FFI binding may call them directly too.  Complex arrays are
 * interleaved float pairs (re, im), x fastest, zero frequency at index 0 --
 * the layout of the reference's Image data.  Return value 0 is success, a
 * negative value an error whose text spb_error_string() returns.  Calls that
 * return data to host memory synchronise the context's stream; the others
 * only enqueue work.
 *
 * Replaces the reference's CUDA engine entry points (src/phasing.cu,
 * src/support_update_cuda.cu, src/image_filter_cuda.cu, src/fft.cu) which call
 * cuFFT, Thrust and cuRAND; here every kernel is this library's own.
 */
#ifndef SPB_DEVICE_H
#define SPB_DEVICE_H 1
#ifdef __cplusplus
extern "C" {
#endif

typedef struct spb_ctx spb_ctx;

typedef struct {
  int algorithm;   /* 1 HIO, 2 RAAR, 3 difference map, 4 ER (SpPhasingAlgorithmType) */
  int constraints; /* SpPhasingConstraints bits */
  int objective;   /* 0 recover phases, 1 recover amplitudes */
  float gamma1;    /* difference map only */
  float gamma2;
} spb_alg_desc;

enum { SPB_SUPPORT_THRESHOLD = 1, SPB_SUPPORT_AREA = 2 };
enum { SPB_G0 = 0, SPB_G1 = 1, SPB_GP = 2, SPB_FMODEL = 3 };

/* Message of the last error on this thread ("" if none). */
const char *spb_error_string(void);
/* Number of usable CUDA devices (0 when there is none or the driver fails). */
int spb_device_count(void);

/* Self-check of the branch-free correctly rounded square root, reciprocal and
 * quotient that the projection and support passes use (no counterpart in the
 * reference): bit-for-bit comparisons with the IEEE intrinsics, counting
 * differences into bad[4] (expected all 0): bad[0] square root and bad[1]
 * reciprocal on every float whose bit pattern lies in [lo, hi) inside their
 * domains; bad[2] on ndiv pseudo-random quotients drawn from seed; bad[3] on
 * the quotients of pairs of significands in [1, 2): every divisor, the
 * dividends of one residue class mod a_stride chosen per divisor from seed
 * (a_stride 1: all 2^46 pairs; the calls with seed 0 .. a_stride-1 together
 * also cover every pair; 0: skip). */
int spb_check_roundings(unsigned lo, unsigned hi, unsigned long long ndiv, unsigned long long seed,
                        unsigned a_stride, unsigned long long *bad);

/* Context for one nx*ny*nz problem on the current CUDA device; replaces the
 * device buffers the reference allocates in sp_phaser_set_amplitudes and
 * sp_phaser_init_model (src/phasing.c:322-330,706-721). */
int spb_ctx_create(spb_ctx **ctx, int nx, int ny, int nz);
void spb_ctx_destroy(spb_ctx *ctx);
int spb_ctx_synchronize(spb_ctx *ctx);
/* Enqueue this context's work on `stream` (a cudaStream_t of the caller, e.g.
 * a framework's stream); NULL returns to the context's own stream.  No
 * reference counterpart (the reference uses the legacy default stream). */
int spb_ctx_set_stream(spb_ctx *ctx, void *stream);

/* Per-kernel timing with CUDA events recorded around every launch on the
 * context's stream (no reference counterpart).  Kinds are the pass kernels
 * named by spb_kernel_name(kind), 0 <= kind < SPB_KERNEL_KINDS. */
enum { SPB_KERNEL_KINDS = 20 };
int spb_ctx_profile(spb_ctx *ctx, int enable);
/* Number of kernels this context has enqueued so far (graph replays count
 * every kernel node). */
long long spb_ctx_launch_count(spb_ctx *ctx);
int spb_ctx_profile_read(spb_ctx *ctx, int kind, long long *launches, double *total_ms);
const char *spb_kernel_name(int kind);

/* Launch-shape knobs (no reference counterpart; they change no arithmetic):
 * SPB_TUNE_ROW_LINES = lines per block of the row passes (0: the built-in
 * choice, 256 threads per block); SPB_TUNE_NO_PDL = 1 launches the pass
 * kernels without programmatic dependent launch (on by default: a pass
 * kernel stages its twiddles and the previous iterate while its predecessor
 * finishes); SPB_TUNE_ROW_G0 = where the iteration's row pass stages the
 * previous iterate: 1 at the start (overlapping the inverse transform), 2
 * between the two transforms (less shared memory, more blocks per SM), 0
 * the built-in choice (2 when the grid exceeds what fits on the device at
 * once with 1); SPB_TUNE_SPLIT = how many points of a line each thread of
 * the iteration's two passes holds: 1 = 16 (the 16-point kernels), 2 = 8 (the
 * 8-point kernels, twice the threads per line, for lengths 256, 512, 1024 and
 * 4096), 0 the built-in choice (8 when the 16-point kernels would give the
 * SMs fewer than 8 warps of lines); SPB_TUNE_PERSIST = 2 runs the
 * iterations of a call of a 32x32, 64x64 or 128x128 pattern (HIO, RAAR or
 * ER; modulus projection without error margins) in one launch, one block per
 * start holding its spectrum in shared memory, 1 = the two-pass kernels,
 * 0 the built-in choice (persistent for 32x32 and 64x64 patterns with at
 * least one start per SM); SPB_TUNE_COL_WIDTH = columns per block of the
 * projection pass along the last axis, for lines of 256 (1..16 columns),
 * 512 (1..8) or 1024 (1..4) points, and of the general kernels' lengths 192
 * (1..16), 384 (1..8) and 1000 (1..4); powers of two; 0 the built-in width;
 * SPB_TUNE_TMA:
 * how the projection pass of 16-point lines of 64 points or more moves its
 * column tiles -- 0 (the built-in choice) with the tensor memory accelerator
 * (bulk tensor loads under an mbarrier and bulk tensor stores) where the
 * tile fits and no other column width is asked for (the blur column pass of
 * the support updates likewise), 2 with it wherever the
 * tile fits and, in addition, the HIO/RAAR/ER row pass with 1-D bulk copies
 * of its rows (rows of 64 points or more; measured no faster than its plain
 * coalesced loads), 1 with plain loads and stores; SPB_TUNE_PLANE: how a 3-D
 * volume with ny = nz = 64 or 128 runs the y and z parts of an iteration --
 * 2 as one plane pass (one block per x-plane: forward y, forward z,
 * projection, inverse z, inverse y; measured slower than the column passes
 * on the B200), 0 (the built-in choice) or 1 as three column passes;
 * SPB_TUNE_SELECT: how a support update selects and masks -- 2 in one
 * launch over a cluster of thread blocks per start where the start's |blur|
 * fits the cluster's shared memory (up to 327,680 pixels; measured no faster
 * on the B200), 0 (the built-in choice) or 1 with one launch per radix pass
 * and one for the mask.
 * Setting a knob drops the context's captured graphs. */
enum {
  SPB_TUNE_ROW_LINES = 0,
  SPB_TUNE_NO_PDL = 1,
  SPB_TUNE_ROW_G0 = 2,
  SPB_TUNE_SPLIT = 3,
  SPB_TUNE_PERSIST = 4,
  SPB_TUNE_COL_WIDTH = 5,
  SPB_TUNE_TMA = 6,
  SPB_TUNE_PLANE = 7,
  SPB_TUNE_SELECT = 8,
  SPB_TUNE_KNOBS = 9
};
int spb_ctx_set_tuning(spb_ctx *ctx, int knob, int value);
int spb_ctx_get_tuning(spb_ctx *ctx, int knob);
/* Autotuner (no reference counterpart): times `calls` calls of `iterations`
 * (2..64) iterations of `alg` for each candidate launch shape (row lines per
 * block, dependent launch on/off, where the row pass stages the previous
 * iterate, 16 or 8 points per thread) and keeps the fastest; the model,
 * iterates, support and parity are restored afterwards.  The choice is cached
 * per process by (shape, starts, algorithm); force = 1 measures again.
 * best_ms (optional) receives the chosen time per iteration, -1 when taken
 * from the cache. */
int spb_ctx_autotune(spb_ctx *ctx, const spb_alg_desc *alg, int iterations, int calls, int force, double *best_ms);

/* Host -> device copies of the phaser inputs (src/phasing.c:189-363). */
int spb_ctx_set_amplitudes(spb_ctx *ctx, const float *amp);
int spb_ctx_set_margins(spb_ctx *ctx, const float *amp_min, const float *amp_max);
int spb_ctx_set_phased_amplitudes(spb_ctx *ctx, const float *phased_amp);
/* pixel flags as the reference's int32 SpPhasingPixelFlags bits */
int spb_ctx_set_flags(spb_ctx *ctx, const int *flags);
/* Only the flag bits in `bits` (SpPhasingPixelFlags) from `flags`, every
 * start, the other bits kept as the device has them (no reference
 * counterpart: the host API uploads only the bits it edited, so support
 * bits a support update changed on the device need not come back first). */
int spb_ctx_set_flags_bits(spb_ctx *ctx, const int *flags, int bits);
int spb_ctx_get_flags(spb_ctx *ctx, int *flags);
/* Start 0's flag bits in `bits` into `flags`, the other bits of `flags` kept
 * (no reference counterpart; the counterpart of spb_ctx_set_flags_bits). */
int spb_ctx_get_flags_bits(spb_ctx *ctx, int *flags, int bits);

/* Model initialisation (src/phasing.c:606-724; CUDA src/phasing.cu:184-240):
 * set_model copies g1; model_from_fourier sets g1 = IFFT(F)/N; both clear g0
 * and gp when reset_others is 1.  mask_out_unmeasured replaces g1 by
 * IFFT(FFT(g1) with unmeasured pixels zeroed)/N (SpModelMaskedOutZeroed). */
int spb_ctx_set_model(spb_ctx *ctx, const float *model, int reset_others);
int spb_ctx_model_from_fourier(spb_ctx *ctx, const float *fourier, int reset_others);
int spb_ctx_mask_out_unmeasured(spb_ctx *ctx);

/* `iterations` phasing iterations of one algorithm (src/phasing.c:1111-1274;
 * CUDA src/phasing.cu:40-182); beta[i] is the schedule value of iteration i
 * (ignored for ER).  keep_gp = 1 stores the last iteration's model before
 * projection for sp_phaser_model_before_projection / sp_phaser_ereal. */
int spb_ctx_iterate(spb_ctx *ctx, const spb_alg_desc *alg, const float *beta, int iterations, int keep_gp);

/* Support update from the current model (src/support_update.c:136-179):
 * blur |g1| with `radius`, then threshold at the area quantile (type AREA,
 * value = area fraction) or at max*value (type THRESHOLD). */
int spb_ctx_support_update(spb_ctx *ctx, int type, float radius, float value);
/* SpSupportFromPatterson (src/phasing.c:744-763) */
int spb_ctx_support_patterson(spb_ctx *ctx, float value);
/* sp_support_close_update_support_cpu (src/support_update.c:225-290): `size`
 * dilations then `size` erosions of every start's support, 6-neighbourhood,
 * no wrap-around at the borders */
int spb_ctx_support_close(spb_ctx *ctx, int size);
/* support bit of every start = abs_values[i] > threshold (abs_values: one
 * start's N values on the host), as the template update's
 * support_from_absolute_threshold (src/support_update.c:193-205,392-400) */
int spb_ctx_support_from_abs(spb_ctx *ctx, const float *abs_values, float threshold);

/* Device -> host copies: SPB_G0 (old model), SPB_G1 (model), SPB_GP (model
 * before projection), SPB_FMODEL (FFT of the model, computed on the GPU). */
int spb_ctx_get_image(spb_ctx *ctx, int which, float *out);
/* Reductions in double: efourier sums {nom, den, FcFo num, FcFo den}
 * (src/phasing.c:852-891); ereal sums {nom, den} (src/phasing.c:803-832). */
int spb_ctx_efourier_sums(spb_ctx *ctx, double sums[4]);
int spb_ctx_ereal_sums(spb_ctx *ctx, double sums[2]);
int spb_ctx_support_count(spb_ctx *ctx, long long *count);
/* No reference counterpart.  Enqueues on the context's stream a check of
 * every start's current model for NaN or infinite values and a copy of the
 * result to *host_flag (page-locked host memory): 1 if such a value was
 * found by this or an earlier check since the last reset, else 0, readable
 * once the stream has passed this point.  reset = 1 clears the sticky device
 * flag first.  The reconstruction server runs it after every chunk of a job
 * to fail a job whose iterates diverged. */
int spb_ctx_nonfinite_async(spb_ctx *ctx, int reset, unsigned *host_flag);

/* Batched starts.  A batch context holds nb independent reconstructions of
 * ONE pattern (shared amplitudes, margins and measured mask; per-start model,
 * iterates and support), stacked start-major.  Every call above acts on all
 * starts at once: set_flags, set_model and model_from_fourier give every
 * start the same value, iterate advances every start, support_update
 * thresholds each start's own blurred model, and the single-start getters
 * read start 0.  This replaces the sequential loop of the reference's
 * Reconstructor.reconstruct_loop (src/_spimage_reconstructor.py:677-740),
 * which runs one SpPhaser after another; each start's result is bit-for-bit
 * the one a single-start context gives for the same start. */
int spb_ctx_create_batch(spb_ctx **ctx, int nx, int ny, int nz, int nb);
int spb_ctx_starts(spb_ctx *ctx);
/* per-start flags; the measured bit must be the same pattern in every start */
int spb_ctx_set_start_flags(spb_ctx *ctx, int start, const int *flags);
int spb_ctx_get_start_flags(spb_ctx *ctx, int start, int *flags);
int spb_ctx_set_start_model(spb_ctx *ctx, int start, const float *model, int reset_others);
/* fourier holds nb spectra, start-major: g1[b] = IFFT(fourier[b])/N */
int spb_ctx_models_from_fourier(spb_ctx *ctx, const float *fourier, int reset_others);
/* Random-phase starts from their phases (no reference counterpart; the
 * device form of sp_image_rephase followed by the inverse transform of
 * sp_phaser_init_model, src/image_util.c:1035-1067 and src/phasing.c:606-650):
 * g1[b] = IFFT(F_b)/N with F_b[i] = (cos(phase) |amp[i]|, sin(phase) |amp[i]|)
 * evaluated in double and rounded to float as the reference does, phase =
 * phases[i] (one = 1: the same phases for every start) or phases[b*N + i]
 * (one = 0).  amp is the host copy of the amplitudes the context holds.  The
 * device evaluates the trigonometry; the few elements whose float rounding
 * could depend on the last bits of cos or sin (a product within 16 ulps of
 * a float rounding midpoint) are evaluated on the host with the C library,
 * so the result is the reference's bit for bit. */
int spb_ctx_models_from_phases(spb_ctx *ctx, const float *phases, const float *amp, int one, int reset_others);
/* A page-locked host buffer of at least `bytes` owned by the context (no
 * reference counterpart): the host API draws random phases and converts pixel
 * flags into it, so their uploads run by DMA.  Valid until the next call
 * asks for more bytes or the context is destroyed; NULL on failure. */
void *spb_ctx_host_stage(spb_ctx *ctx, size_t bytes);
/* Page-lock (0 on success) / release a host range the caller keeps and
 * reuses across calls, so copies to and from it run by DMA (the host API
 * locks its amplitude array and its model image). */
int spb_host_register(void *p, size_t bytes);
void spb_host_unregister(void *p);
/* g1[b] = IFFT(amp * exp(2 pi i u))/N with u drawn on the device by
 * Philox4x32-10 keyed by seeds[b] (throughput runs; the host API's
 * SpModelRandomPhases reproduces the reference's rand() stream instead) */
int spb_ctx_random_phase_models(spb_ctx *ctx, const unsigned long long *seeds, int reset_others);
int spb_ctx_get_start_image(spb_ctx *ctx, int start, int which, float *out);
/* sums[b*4 + k]: efourier {nom, den, FcFo num, FcFo den}, ereal {nom, den, 0, 0} */
int spb_ctx_batch_efourier_sums(spb_ctx *ctx, double *sums);
int spb_ctx_batch_ereal_sums(spb_ctx *ctx, double *sums);
int spb_ctx_batch_support_counts(spb_ctx *ctx, long long *counts);

/* One-shot transforms of host buffers (sp_image_fft/ifft, src/fft.c:53-189,
 * src/fft.cu:7-43; sp_gaussian_blur, src/image_filter.c:80-90).  sign -1 is
 * forward, +1 backward (unnormalised). */
int spb_fft_host(int nx, int ny, int nz, int sign, const float *in, float *out);
int spb_blur_host(int nx, int ny, int nz, const float *in, float radius, float *out);
/* Support mask from an already blurred image (support_from_absolute_threshold,
 * src/support_update.c:392-400 with the area rule :143-144 or the threshold
 * rule :175-176): updates bit 0 of flags in place. */
int spb_support_from_blur_host(long long n, const float *blur, int type, float value, int *flags);
/* Phase-retrieval transfer function of n reconstructions (the reference's
 * Python prtf, src/_spimage_prtf.py:17-106, over sp_image_superimpose and
 * sp_image_phase_match, src/image_util.c:2974-3007,3160-3186), on the GPU.
 * images: [n][N] complex (real space, as reconstructed), supports: [n][N].
 * flags: bit 0 superimpose each image on the running sum (translation by
 * cross-correlation of the moduli, then phase matching), bit 1 also try the
 * enantiomorph.  Outputs (NULL skips): prtf[N] = |mean unit phasor of the
 * images' spectra| (zero where a spectrum vanishes), in the FFT layout
 * (the reference returns it fftshifted); super_image[N] complex = the sum of
 * the aligned images; super_mask[N] = 1 where some non-empty support left
 * the pixel out.  Translations and reflections are decided from the same
 * correlation values as the reference (bit-exact FFTs); the phase matching
 * sums in double and evaluates atan2/cos/sin on the GPU, so results agree
 * with the reference to rounding, not bit for bit. */
int spb_prtf_host(int nx, int ny, int nz, int n, const float *images, const int *supports, int flags, float *prtf,
                  float *super_image, int *super_mask);
/* sp_image_superimpose_fractional (src/image_util.c:3024-3066) on host
 * buffers: b ([N] complex) is overwritten with b superimposed on a.  flags:
 * bit 0 SpEnantiomorph, bit 1 SpCorrectPhaseShift.  The correlation peaks,
 * hence the translation and the enantiomorph choice, are the reference's
 * (bit-identical FFTs and products); the Fourier translation and the phase
 * shift evaluate cos/sin/atan2 in double on the GPU, so b agrees with the
 * reference to rounding. */
int spb_superimpose_fractional_host(int nx, int ny, int nz, const float *a, float *b, int flags, int precision);
/* sp_prtf_basic (src/prtf.c:6-34) of n images ([n][N] complex) into out
 * ([N] complex); bit for bit the reference's. */
int spb_prtf_basic_host(int nx, int ny, int nz, int n, const float *images, float *out);
/* sp_prtf_advanced (src/prtf.c:38-78) of n images ([n][N] complex, in
 * Fourier space for space = 1, real space for 2) into prtf ([N] complex);
 * write_back = 1 overwrites images with the superimposed images in their
 * own space (SpInPlace). */
int spb_prtf_advanced_host(int nx, int ny, int nz, int n, float *images, int space, int write_back, float *prtf);
/* No counterpart in the reference.  spb_support_from_blur_host without any
 * device allocation, for callers that must not allocate device memory: a
 * process whose HBM is reserved up front by another allocator (a framework's
 * caching allocator, a serving loop's job pool), where a cudaMalloc of its own
 * fails or fragments that pool, and latency-bound loops that cannot take
 * cudaFree's device-wide synchronisation.  Same arguments, results and
 * errors, except:
 *  - n is at most 65536 pixels (256 x 256); larger n returns -1 with an
 *    error naming the limit.  The device scratch is one fixed 1,122,560-byte
 *    array in the library, shared by every call.
 *  - the first call on a device looks that array's address up (once per
 *    device, with the device current); make that first call before any
 *    stream capture begins on that device.
 *  - work runs on the legacy default stream and the call returns when it is
 *    done.  Calls that overlap on the GPU (several host threads at once) race
 *    on the shared scratch: serialise them.
 * Calls no cudaMalloc, cudaFree or other allocating routine. */
int spb_support_from_blur_noalloc(long long n, const float *blur, int type, float value, int *flags);

#ifdef __cplusplus
}
#endif
#endif

/*
 * imresh_b200 -- C ABI of the B200 shrink-wrap / hybrid-input-output (HIO)
 * phase-retrieval engine (libimresh_b200.so).
 *
 * Plain C: pointers, sizes and status codes only.  Every entry point returns
 * an imr_status; none of them exits or aborts the process (the reference
 * prints and calls exit(EXIT_FAILURE) on any CUDA error,
 * src/imresh/libs/cudacommon.cu:39-56).  `stream` arguments are cudaStream_t
 * values passed as void* (NULL = the legacy default stream).
 *
 * Data convention (identical to the reference): an image is W*H float32,
 * row-major with the width contiguous.  The input is the Fourier MODULUS |F|
 * with the zero frequency at index 0 (the reference scales G' to it,
 * src/imresh/algorithms/cuda/cudaVectorElementwise.cu:168-195); pass sqrt(I)
 * for a measured intensity I.  The output is Re(g') of the last inverse
 * transform, carrying the factor W*H of the unnormalised FFTs.
 */
#ifndef IMRESH_B200_H
#define IMRESH_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum imr_status {
    IMR_SUCCESS = 0,
    IMR_ERR_INVALID_VALUE = 1,     /* NULL buffer, zero size, bad parameter   */
    IMR_ERR_UNSUPPORTED_SIZE = 2,  /* W or H outside the supported lengths   */
    IMR_ERR_OUT_OF_MEMORY = 3,     /* device or host allocation failed        */
    IMR_ERR_CUDA = 4,              /* a CUDA runtime call failed              */
    IMR_ERR_NOT_INITIALIZED = 5,   /* task queue used before imr_queue_init   */
    IMR_ERR_QUEUE = 6,             /* task queue / serving loop failure       */
    IMR_ERR_DEVICE_TIMEOUT = 7,    /* a bounded device-side wait gave up      */
    IMR_ERR_CANCELLED = 8          /* the request was cancelled (engine)      */
} imr_status;

/* Parameters of one reconstruction, same meaning as the reference's
 * cudaShrinkWrap arguments (src/imresh/algorithms/cuda/cudaShrinkWrap.hpp:114-130).
 * A value <= 0 (== 0 for the counts) selects the reference's CUDA default
 * (cudaShrinkWrap.cu:193-200): nCycles 20, targetError 1e-5, hioBeta 0.9,
 * cutOffAutoCorel 0.02, cutOff 0.2, sigma0 3.0, sigmaChange 0.01,
 * nHioCycles 20.  Pass targetError = FLT_MIN to run every cycle. */
typedef struct imr_params {
    unsigned nCycles;
    float targetError;
    float hioBeta;
    float intensityCutOffAutoCorel;
    float intensityCutOff;
    float sigma0;
    float sigmaChange;
    unsigned nHioCycles;
} imr_params;

/* Human-readable name of a status code (static string). */
const char *imr_status_string(int status);
/* Detail of the last failed CUDA call on the calling thread ("" if none). */
const char *imr_last_error(void);

/* Largest supported image side and whether a side length is supported:
 * every length from 1 to 2048 (direct mixed-radix transforms for lengths
 * whose prime factors are all in {2, 3, 5, 7}, Bluestein's chirp-z transform
 * otherwise), plus 3072 and 4096. */
unsigned imr_max_side(void);
int imr_side_supported(unsigned n);

/* ------------------------------------------------------------------------
 * Drop-in for imresh::algorithms::cuda::cudaShrinkWrap
 * (src/imresh/algorithms/cuda/cudaShrinkWrap.hpp:114-130, .cu:164-420).
 * ioData: HOST buffer of W*H floats, modulus in, Re(g') out.  Synchronous:
 * returns after the result is in ioData, like the reference (cu:403-407).
 * nBlocks / nThreads are accepted for signature compatibility and ignored:
 * the engine chooses its own launch shapes.  Returns 0 on success.
 */
int imr_cuda_shrink_wrap(float *ioData, unsigned W, unsigned H, void *stream,
                         unsigned nBlocks, unsigned nThreads, unsigned nCycles,
                         float targetError, float hioBeta,
                         float intensityCutOffAutoCorel, float intensityCutOff,
                         float sigma0, float sigmaChange, unsigned nHioCycles);

/* ------------------------------------------------------------------------
 * Reusable plan for one image size and parameter set (device buffers, FFT
 * twiddles and the captured CUDA graph of one shrink-wrap cycle).  A plan
 * serves one reconstruction at a time.
 */
typedef struct imr_plan imr_plan;

int imr_plan_create(imr_plan **plan, unsigned W, unsigned H, const imr_params *params);
/* Asynchronous on `stream`: reads W*H modulus floats from DEVICE memory
 * d_modulus, writes W*H Re(g') floats to DEVICE memory d_out. */
int imr_plan_execute(imr_plan *plan, const float *d_modulus, float *d_out, void *stream);
/* Same through HOST buffers (pinned or pageable); synchronous. */
int imr_plan_execute_host(imr_plan *plan, const float *h_modulus, float *h_out, void *stream);
/* After execution (synchronises `stream`): cycles whose HIO block ran and
 * was error-tested, and the error after each of them (errors may be NULL;
 * otherwise room for nCycles floats). */
int imr_plan_stats(imr_plan *plan, void *stream, int *cycles_done, float *errors);
/* Kernel launches one execution issues (for launch accounting). */
int imr_plan_launches(imr_plan *plan, long *launches);
/* Debug state copies to HOST memory after execution (synchronise first):
 * what = 0: mask (W*H bytes, 1 = outside the support)
 *        1: X, the iterate between passes (W*H complex64)
 *        2: g_prev (W*H complex64)
 *        3: blurred |g'| of the last cycle (W*H float32) */
int imr_plan_copy_state(imr_plan *plan, int what, void *h_dst, void *stream);
/* Times the two passes of one HIO iteration on `stream` with CUDA events,
 * on the plan's current state: the mean time of a (row pass, column pass)
 * pair from a captured graph of `iters` pairs with events only before and
 * after them (kernel after kernel, as a reconstruction runs them), split
 * between the two passes in the proportion a second replay with an event
 * after every pass measures (those events drain the GPU between kernels, so
 * they time the proportion, not the pair).  Each graph is replayed once
 * untimed first.  Returns the mean milliseconds of each pass.  Synchronous.
 * Leaves the plan's iterate changed; run it after imr_plan_execute, not
 * inside one. */
int imr_plan_profile(imr_plan *plan, int iters, void *stream, float *ms_row_pass,
                     float *ms_col_pass);
/* Algorithmic HBM bytes of one row pass and one column pass: every image
 * array touched once (row: X, g_prev in; g_prev, X out; mask in = 33 B/px;
 * column: X, modulus in; X out = 20 B/px). */
int imr_plan_pass_bytes(imr_plan *plan, double *row_bytes, double *col_bytes);
/* Limit of every bounded device-side copy wait of the plan's passes, in
 * nanoseconds (0 = the default, 0.5 s).  A wait that runs out records
 * IMR_ERR_DEVICE_TIMEOUT in the plan's state (imr_plan_stats returns it);
 * the pass waits, bounded by the default limit, for its copies still in
 * flight and returns, so the context stays usable.  Takes effect for the
 * next execution; synchronous.  The reference has no such bound: it exits
 * the process on any CUDA error (src/imresh/libs/cudacommon.cu:39-56). */
int imr_plan_set_wait_limit(imr_plan *plan, unsigned long long limit_ns);
/* Arithmetic of the plan's column pass (forward column FFT, modulus
 * projection, inverse column FFT -- the cuFFT pair around the modulus step,
 * src/imresh/algorithms/cuda/cudaShrinkWrap.cu:319,343):
 *   IMR_PREC_FP32     FP32 FFT on the CUDA cores (the default; the drop-in);
 *   IMR_PREC_BF16X3   radix-16 stages as DFT-16 matrix products on the tensor
 *                     cores, inputs and DFT matrix split into BF16 hi + lo,
 *                     three products accumulated in FP32;
 *   IMR_PREC_FP16X3   the same in FP16 hi + lo with a power-of-two scale per
 *                     tile and stage.
 * Twiddles, the last stage of radix < 16, the modulus step and every error
 * sum stay FP32 / FP64.  The split-precision passes need a height that is a
 * power of two in 256..4096 with the pipelined column pass
 * (IMR_ERR_UNSUPPORTED_SIZE otherwise).  Re-captures the plan's graphs;
 * synchronous. */
#define IMR_PREC_FP32 0
#define IMR_PREC_BF16X3 1
#define IMR_PREC_FP16X3 2
int imr_plan_set_precision(imr_plan *plan, int precision);
int imr_plan_destroy(imr_plan *plan);

/* Self-check of the bounded wait the pipelined passes rely on: one thread
 * waits, bounded by limit_ns (0 = 0.5 s), on a device barrier that nothing
 * completes.  Returns IMR_ERR_DEVICE_TIMEOUT (the expected outcome) with the
 * nanoseconds waited in *elapsed_ns, leaving the context usable; anything
 * else means the bound does not work.  Synchronous.  No counterpart in the
 * reference. */
int imr_bounded_wait_check(unsigned long long limit_ns, unsigned long long *elapsed_ns, void *stream);

/* ------------------------------------------------------------------------
 * Kernel-level entry points (device buffers, asynchronous on `stream`).
 */
/* Unnormalised 2D C2C transform in place; sign -1 forward, +1 inverse
 * (cufftExecC2C FORWARD / INVERSE as used at cudaShrinkWrap.cu:232,319,343). */
int imr_fft2d(void *d_data, unsigned W, unsigned H, int sign, void *stream);
/* The same 2D transform with the column transform on the split-precision
 * tensor-core passes (precision IMR_PREC_BF16X3 or IMR_PREC_FP16X3; rows
 * stay FP32).  H: a power of two in 256..4096; W: a multiple of the column
 * tile width (16 up to H = 512, 8 at 1024, 4 at 2048, 2 at 4096); d_data 16-byte
 * aligned.  Synchronous. */
int imr_fft2d_split(void *d_data, unsigned W, unsigned H, int sign, int precision, void *stream);
/* Separable Gaussian blur in place, clamp border, rows then columns
 * (cudaGaussianBlur, src/imresh/algorithms/cuda/cudaGaussian.cu:1044-1057);
 * axes: 1 rows only, 2 columns only, 3 both.  d_tmp: W*H floats of scratch. */
int imr_gaussian_blur(float *d_data, float *d_tmp, unsigned W, unsigned H, double sigma,
                      int axes, void *stream);
/* Gaussian weights for sigma (calcGaussianKernel,
 * src/imresh/libs/calcGaussianKernel.cpp:42-91); returns the tap count, and
 * writes the weights when it is <= cap. */
int imr_gaussian_weights(double sigma, float *h_weights, int cap);
/* Forward model |FFT2(object)| (the Fourier modulus) of a real W*H image,
 * in place in HOST memory, on the engine's FFT; synchronous
 * (diffractionIntensity, src/imresh/libs/diffractionIntensity.cpp:84-135). */
int imr_diffraction_intensity(float *h_io, unsigned W, unsigned H, void *stream);
/* Global maximum of n floats (cudaVectorMax, cudaVectorReduce.cu:229-239);
 * the result goes to HOST *h_max; synchronous. */
int imr_vector_max(const float *d_data, size_t n, float *h_max, void *stream);

/* Mask element types of imr_calculate_hio_error. */
#define IMR_MASK_F32 0
#define IMR_MASK_U8 1
/* HIO error of n complex64 values (cudaCalculateHioError<cufftComplex, float>,
 * src/imresh/algorithms/cuda/cudaVectorReduce.cu:357-403, hpp:160-170):
 * total = sum w*|z|, count = sum w, error = sqrtf(total)/count, with
 * w = (mask != 0) xor invert_mask.  Sums in double, rounded to float once.
 * Results go to HOST pointers (any may be NULL); synchronous. */
int imr_calculate_hio_error(const void *d_data, const void *d_mask, int mask_type, size_t n,
                            int invert_mask, float *h_total, float *h_count, float *h_error,
                            void *stream);

/* ------------------------------------------------------------------------
 * Fixed-support hybrid input-output with a random initial phase
 * (imresh::libs::hybridInputOutput, src/imresh/libs/hybridInputOutput.cpp:193-306,
 * hpp:81-90), on the engine's fused passes.
 *
 * io: HOST W*H floats, the Fourier modulus in, Re(g') out.  mask: HOST W*H
 * bytes, 1 = outside the support (HIO applies where mask == 1; the error
 * weighs |g'| by the mask value).  nCycles == 0 means unbounded (the
 * reference's UINT_MAX); beta <= 0 means 0.9; targetError <= 0 disables the
 * per-iteration error test.  The initial phase is the argument of the 2D FFT
 * of the C library's rand() numbers after srand(IMR_HIO_SEED), as in the
 * reference (cpp:160-167), drawn on the GPU.  Synchronous. */
#define IMR_HIO_SEED 2623091912u
int imr_hybrid_input_output(float *io, const unsigned char *mask, unsigned W, unsigned H,
                            unsigned nCycles, float targetError, float beta, void *stream);

/* The C library's numbers after srand(seed), as n DEVICE complex64 values
 * ((float)rand()/RAND_MAX, 0): the random real field of addRandomPhase
 * (hybridInputOutput.cpp:160-167), drawn in parallel by jumping glibc's
 * additive feedback generator ahead.  seed 0 acts as 1, as in glibc.
 * Asynchronous on `stream`. */
int imr_rand_field(void *d_out, size_t n, unsigned seed, void *stream);

/* The same as a reusable plan over DEVICE buffers (no allocation or graph
 * capture per call).  execute is asynchronous on `stream`; execute_host takes
 * HOST buffers and returns after the result is copied back.  seed: the
 * srand() seed of the initial phase (IMR_HIO_SEED for the reference's).
 * stats: iterations = HIO updates applied before the returned g', the last
 * tested error, and the per-iteration errors (up to cap values; iterations
 * whose error was not tested read 0). */
typedef struct imr_hio_plan imr_hio_plan;
int imr_hio_plan_create(imr_hio_plan **plan, unsigned W, unsigned H, unsigned nCycles,
                        float targetError, float beta);
int imr_hio_plan_execute(imr_hio_plan *plan, const float *d_modulus, const unsigned char *d_mask,
                         float *d_out, unsigned seed, void *stream);
int imr_hio_plan_execute_host(imr_hio_plan *plan, const float *h_modulus,
                              const unsigned char *h_mask, float *h_out, unsigned seed,
                              void *stream);
int imr_hio_plan_stats(imr_hio_plan *plan, void *stream, int *iterations, float *last_error,
                       float *errors, int cap);
int imr_hio_plan_destroy(imr_hio_plan *plan);

/* ------------------------------------------------------------------------
 * Image files (host memory) behind the task queue's read-in / write-out
 * callbacks (src/imresh/io/readInFuncs/readInFuncs.hpp:57-84,
 * src/imresh/io/writeOutFuncs/writeOutFuncs.hpp:52-106) for formats that need
 * no third-party library: NumPy .npy (float32 written; float32 or float64,
 * 1-D or 2-D, C order read), text (one image row per line) and headerless
 * float32.  W*H floats, width contiguous.  Readers allocate *data (release it
 * with imr_free_image); failures return IMR_ERR_INVALID_VALUE with a message
 * on stderr.
 */
int imr_write_npy(const char *path, const float *data, unsigned W, unsigned H);
int imr_read_npy(const char *path, float **data, unsigned *W, unsigned *H);
int imr_write_txt(const char *path, const float *data, unsigned W, unsigned H);
int imr_read_txt(const char *path, float **data, unsigned *W, unsigned *H);
int imr_write_raw(const char *path, const float *data, unsigned W, unsigned H);
void imr_free_image(float *data);

/* ------------------------------------------------------------------------
 * Reconstruction that allocates nothing -- no counterpart in the reference.
 * For callers that cannot call cudaMalloc (memory owned by a fixed arena or a
 * framework allocator, loops that must not take the driver's allocation
 * locks, processes that reserve all device memory up front).  d_modulus and
 * d_out are DEVICE buffers of W*H floats owned by the caller; they may be the
 * same buffer (the modulus is copied first, so the call can work in place
 * like the reference's cudaShrinkWrap).  All other working memory is a static
 * device array of the library (about 10 MB), so W*H is limited to 512*512
 * pixels, nCycles to 1024, and W and H to lengths of the form 2^a 3^b 5^c 7^d
 * (lengths with a larger prime factor need per-length tables that would have
 * to be allocated): IMR_ERR_UNSUPPORTED_SIZE or IMR_ERR_INVALID_VALUE beyond,
 * with a message in imr_last_error.  Asynchronous on `stream`.  The first
 * call on a device looks up the array's address and sets kernel attributes:
 * make it before any stream capture.  All calls share the one array: calls
 * whose GPU work overlaps (different streams, unordered host threads) race;
 * issue them one after another on one stream.
 */
int imr_shrink_wrap_noalloc(const float *d_modulus, float *d_out, unsigned W, unsigned H,
                            const imr_params *params, void *stream);
/* Status of the last imr_shrink_wrap_noalloc call on the current device (it
 * synchronises `stream`, which should be the call's stream): the cycles whose
 * HIO block ran and was error-tested, the error after each of them (up to cap
 * floats; errors may be NULL), and IMR_ERR_DEVICE_TIMEOUT when a bounded
 * device-side copy wait gave up during that call (its output is then not a
 * valid reconstruction).  Reads the library's static array only; allocates
 * nothing. */
int imr_shrink_wrap_noalloc_stats(void *stream, int *cycles_done, float *errors, int cap);

/* ------------------------------------------------------------------------
 * Batched, continuously-admitting engine (the served form of the path).
 * Replaces the reference's per-task std::thread + stream round robin
 * (imresh::io::taskQueue*, src/imresh/io/taskQueue.cu:91-251) with device-
 * resident state for every admitted reconstruction: one imr_engine_step runs
 * one shrink-wrap cycle of every active reconstruction, whatever their sizes,
 * as ONE CUDA graph launch (captured when the active set changes, replayed
 * otherwise), admits pending requests while the device-memory budget allows,
 * and retires finished ones (their Re(g') is copied to the caller's h_out).
 * Finishing is decided on the device; the host reads every job's state
 * asynchronously and acts on it two steps later, so a step returns without
 * waiting for the GPU (at most two steps are queued).  Results reach a
 * pageable h_out through pinned host staging that a helper thread of the
 * engine pins ahead of need (room for the resident requests' results, at
 * most 1 GiB, kept until imr_engine_destroy); a pinned h_out is written
 * directly.  Not thread safe: drive one engine from one thread.
 */
typedef struct imr_engine imr_engine;

typedef struct imr_result {
    long long tag;         /* the caller's tag from imr_engine_submit        */
    unsigned width, height;
    int cycles_done;       /* HIO blocks run and error-tested                */
    float last_error;      /* error after the last of them                   */
    double latency_ms;     /* submit -> result in h_out                      */
    int status;            /* imr_status of this reconstruction: 0, or
                              IMR_ERR_DEVICE_TIMEOUT (a device wait gave up),
                              IMR_ERR_OUT_OF_MEMORY (never admitted: its
                              memory was not available with nothing else
                              running), IMR_ERR_CANCELLED                   */
} imr_result;

typedef struct imr_engine_info {
    int pending;           /* submitted, not admitted yet                    */
    int active;            /* admitted, result not yet handed over           */
    int done;              /* results waiting for imr_engine_poll            */
    size_t device_bytes_used, device_bytes_peak, device_bytes_budget;
    long launches;         /* kernels run so far (a graph's count once per step) */
    long steps;
    long host_launches;    /* launch calls the host made (a step graph counts once) */
    long kernels_per_step; /* kernels in the current step graph              */
    long graph_builds;     /* step graphs instantiated                       */
    long graph_updates;    /* step graphs updated in place (same shape)      */
    long alloc_failures;   /* admissions whose device allocation failed      */
    int resident;          /* reconstructions holding device memory          */
    size_t resident_px;    /* their pixels                                   */
    double last_step_ms;   /* device time of the last step whose state was read */
    double ms_per_mpx;     /* step time per million resident pixels (running) */
    double device_ms;      /* device time of all steps whose state was read  */
    int schedule;          /* IMR_SCHEDULE_* in use                          */
    int grid_pct;          /* persistent grids at this % of the occupancy limit */
    long tune_explored;    /* steps the tuner ran to compare configurations  */
    long tune_cache_hits;  /* admitted sets whose configuration came from the cache */
    int cycles_per_step;   /* shrink-wrap cycles in one step's graph         */
} imr_engine_info;

/* device_bytes: admission budget (0 = 80 % of the free device memory);
 * max_jobs: reconstructions resident at once. */
int imr_engine_create(imr_engine **engine, size_t device_bytes, int max_jobs, void *stream);
/* Queue one reconstruction.  h_modulus (W*H floats) must stay valid until the
 * request is admitted, h_out (W*H floats) until its result is polled. */
int imr_engine_submit(imr_engine *engine, const float *h_modulus, float *h_out, unsigned W,
                      unsigned H, const imr_params *params, long long tag);
/* The same for a measured intensity I (W*H floats, >= 0): the engine takes
 * the modulus sqrt(I) (correctly rounded, in FP32) on the device at
 * admission, so the result equals submitting sqrtf(I).  No counterpart in
 * the reference (its callers pass the modulus). */
int imr_engine_submit_intensity(imr_engine *engine, const float *h_intensity, float *h_out, unsigned W,
                                unsigned H, const imr_params *params, long long tag);
/* Retire what had finished two steps ago, admit, launch one step (one cycle,
 * or imr_engine_set_cycles_per_step's count) of every active reconstruction.
 * Returns once the step is queued (it waits only for the step before the
 * previous one).  When every cycle of every running request has been queued
 * and nothing is pending, it waits for the last step instead and retires
 * them. */
int imr_engine_step(imr_engine *engine);
/* Step until nothing is pending, running or being copied out. */
int imr_engine_run(imr_engine *engine);
/* Finished reconstructions since the last poll (up to max_results). */
int imr_engine_poll(imr_engine *engine, imr_result *results, int max_results, int *n_results);
int imr_engine_stats(imr_engine *engine, imr_engine_info *info);
/* Cancel a pending or running request between steps: it is reported by
 * imr_engine_poll with status IMR_ERR_CANCELLED, its h_out is not written,
 * its device memory is released after the steps already queued.  Returns
 * IMR_ERR_INVALID_VALUE (with a message) when no pending or running request
 * has this tag.  No counterpart in the reference (its tasks cannot be
 * stopped). */
int imr_engine_cancel(imr_engine *engine, long long tag);
/* How a step's kernels are ordered in its graph.
 * IMR_SCHEDULE_GROUPED (default): one launch per pass and image-side class
 *   over all jobs of that class; the passes of one HIO iteration follow each
 *   other for all jobs (fewest kernels per step).
 * IMR_SCHEDULE_CHAINED: the jobs of each (row kernel, column kernel) class
 *   form an independent branch of the graph running its whole cycle, so the
 *   classes run concurrently and fill each other's pass tails (more kernels,
 *   no step-wide order between classes).  Results are bit-identical either
 *   way.  Takes effect at the next step. */
#define IMR_SCHEDULE_GROUPED 0
#define IMR_SCHEDULE_CHAINED 1
int imr_engine_set_schedule(imr_engine *engine, int schedule);
/* Online tuner of the step configuration.  For every admitted set (its
 * kernel classes and their job counts) not seen before, the next steps run
 * the candidate configurations -- the two schedules, persistent grids at 100 %
 * and 50 % of the occupancy limit -- two steps each; the times per resident
 * pixel of their second steps (device time plus the host time of the graph
 * launch) are compared and the fastest is kept for the set and
 * appended to `cache_path` (a text file, one line per set; NULL or "" keeps it
 * in memory), which later engines load here, so a known set starts with its
 * configuration.  Every candidate gives the same bits.  enable = 0 turns the
 * tuner off (the configuration in use stays). */
int imr_engine_set_autotune(imr_engine *engine, int enable, const char *cache_path);
/* Bound on the work admitted at once: a pending request is admitted only
 * while the pixels (W*H) of all resident requests, its own included, stay
 * within max_active_pixels (0 = no bound: device memory alone decides), or
 * when nothing else is running.  Each step advances every resident request
 * by one cycle, so the step time -- and with it the latency of every admitted
 * request -- grows with the admitted pixels; the bound caps it, and the
 * requests beyond it wait in arrival order. */
int imr_engine_set_admission(imr_engine *engine, size_t max_active_pixels);
/* The same bound derived from the measured step time: every step's graph is
 * timed on the device, the engine keeps a running cost per resident pixel,
 * and admits a request only while the predicted step time stays within
 * target_step_ms (0 = off) or nothing else is running.  A request's latency
 * is then about its cycle count times the target, plus its wait in the
 * queue. */
int imr_engine_set_step_target(imr_engine *engine, double target_step_ms);
/* Shrink-wrap cycles captured into one step's graph (1..256, default 1).
 * More cycles per step mean fewer host launches and state read-backs per
 * cycle, and later retirement and admission (a finished request waits for
 * the end of its step; the others skip the rest of it on the device).  The
 * step-time target then applies to a step of that many cycles.  Results are
 * bit-identical for every count.  No counterpart in the reference. */
int imr_engine_set_cycles_per_step(imr_engine *engine, int cycles);
/* Host-side fault injection for tests of the failure paths: the device
 * allocations of the next `count` admissions fail as if the device were out
 * of memory.  A request whose allocation fails waits in the queue while
 * other reconstructions run (their retirement frees memory) and is retried;
 * with nothing else running it finishes with IMR_ERR_OUT_OF_MEMORY. */
int imr_engine_inject_alloc_failures(imr_engine *engine, int count);
/* Suspend / resume of one reconstruction (for preemption and restart).  Between
 * steps, a running reconstruction (`tag` of an active request) is saved into a
 * HOST buffer of imr_engine_snapshot_size bytes: its iterate, g_prev, modulus,
 * support mask, per-cycle errors and device-side cycle state.  checkpoint
 * leaves it running; suspend also removes it from the engine and releases its
 * device memory (no result is reported for it).  resume queues the saved
 * reconstruction into this or another engine; it continues from the saved
 * cycle, bit-identical to an uninterrupted run, and its result goes to h_out
 * (W*H floats) under the saved tag.  A reconstruction that has already
 * finished on the device cannot be saved (IMR_ERR_INVALID_VALUE).
 * Synchronous.  No counterpart in the reference (its tasks cannot be
 * interrupted). */
int imr_engine_snapshot_size(imr_engine *engine, long long tag, size_t *bytes);
int imr_engine_checkpoint(imr_engine *engine, long long tag, void *h_buf, size_t capacity);
int imr_engine_suspend(imr_engine *engine, long long tag, void *h_buf, size_t capacity);
int imr_engine_resume(imr_engine *engine, const void *h_buf, size_t bytes, float *h_out);
int imr_engine_destroy(imr_engine *engine);

#ifdef __cplusplus
}
#endif
#endif

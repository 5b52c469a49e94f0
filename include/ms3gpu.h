/*
 * ms3gpu -- B200-native ms3.bandpass_filter and ms3.whiten (C ABI).
 *
 * The two processors of MountainSort 3's preprocessing front end
 * (pipelines/mountainsort3.mlp, "sort" script) as a shared library with plain
 * C entry points: caller-owned buffers, int status codes, no exceptions and
 * no torch types.  Each entry point is the in-memory form of one reference
 * processor or of one stage inside it; citations are paths inside the
 * reference project (flatironinstitute/mountainsort).
 *
 * Data layout.  A timeseries of M channels and N timepoints is the .mda
 * M x N column-major array: element (m, t) at index m + M*t (channel
 * fastest), float32 unless stated otherwise.  M x M matrices (XXt, W) are
 * column-major doubles like the reference's Mda: element (i, j) at i + M*j.
 *
 * Pointers.  Every buffer argument may be host memory (pageable or pinned)
 * or device memory of the current CUDA device; the library classifies each
 * pointer itself.  Host buffers are staged through the device.  Calls return
 * after the results are complete in the output buffers.
 *
 * Streams.  `stream` is a cudaStream_t (NULL = the legacy default stream).
 * All device work of a call is ordered on that stream.
 *
 * Threading.  Calls may come from several host threads; each call uses its
 * own scratch memory.  Errors are reported per thread by
 * ms3gpu_last_error().
 */
#ifndef MS3GPU_H
#define MS3GPU_H

#include <stdint.h>

#if defined(MS3GPU_BUILDING) && defined(__GNUC__)
#define MS3GPU_API __attribute__((visibility("default")))
#else
#define MS3GPU_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The reference's processors return bool, turned into exit
 * code 0 / -1 by main (packages/ms3/mountainsort3_main.cpp:817-820). */
#define MS3GPU_OK 0
#define MS3GPU_ERR_INVALID -1     /* bad argument (sizes, pointers, options) */
#define MS3GPU_ERR_CUDA -2        /* a CUDA runtime error */
#define MS3GPU_ERR_UNSUPPORTED -3 /* a shape the GPU path does not handle */
#define MS3GPU_ERR_NOMEM -4       /* device memory exhausted */
#define MS3GPU_ERR_IO -5          /* a read or write callback of a streaming call failed */

/* .mda data type codes (packages/ms3/mda/mdaio.h:55-62) used for outputs. */
#define MS3GPU_DTYPE_FLOAT32 -3
#define MS3GPU_DTYPE_INT16 -4

/* Bandpass_filter_opts (packages/ms3/p_bandpass_filter.h:21-31), as parsed
 * by main (packages/ms3/mountainsort3_main.cpp:547-557), plus the thread
 * count T that the reference's chunk geometry depends on
 * (p_bandpass_filter.cpp:147-155: T = omp_get_max_threads(), which
 * --_request_num_threads sets, mountainsort3_main.cpp:428-434). */
typedef struct ms3gpu_bandpass_opts {
    double samplerate;
    double freq_min;
    double freq_max;
    double freq_wid;          /* processor default 1000 */
    double quantization_unit; /* != 0: int16 output of x / quantization_unit */
    int32_t subsample_factor; /* 0 is treated as 1, like the reference */
    int32_t num_threads;      /* T of the chunk-size formula; must be >= 1 */
} ms3gpu_bandpass_opts;

/* Arithmetic of the whitening passes. */
#define MS3GPU_PRECISION_PLAIN 0 /* FP32 FMA apply: parity with the reference (<= 1e-5 rel. L2) */
#define MS3GPU_PRECISION_MIXED 1 /* tensor-core 3-term TF32 apply (tcgen05), FP32 accumulation:
                                    <= 1e-4 rel. L2 against the FP64 algorithm */

/* Whiten_opts (packages/ms3/p_whiten.h:21-26) plus the arithmetic mode. */
typedef struct ms3gpu_whiten_opts {
    double quantization_unit; /* > 0: int16 output of round(y / quantization_unit) */
    int32_t precision;        /* MS3GPU_PRECISION_PLAIN (default) or MS3GPU_PRECISION_MIXED */
} ms3gpu_whiten_opts;

/* Text of the last error on the calling thread ("" if none). */
MS3GPU_API const char* ms3gpu_last_error(void);

/* Library version string. */
MS3GPU_API const char* ms3gpu_version(void);

/* Number of CUDA kernels this library has launched in this process (for
 * throughput accounting; monotonically increasing). */
MS3GPU_API uint64_t ms3gpu_launch_count(void);

/* Device memory the library keeps for reuse between calls (its stream-ordered
 * pool on the current device holds freed buffers instead of returning them)
 * is handed back to the driver, after the work queued on the device has
 * finished.  For callers that need that memory for something else between
 * calls; the next call allocates again.  Not a replacement for any MountainSort
 * interface (the reference's processors exit after each call). */
MS3GPU_API int ms3gpu_release_cached_memory(void);

/* The reference's chunk size for M channels and T threads
 * (p_bandpass_filter.cpp:147-155); the FFT length is chunk + 120000. */
MS3GPU_API int64_t ms3gpu_bandpass_chunk_size(int64_t M, int32_t num_threads);

/* Output shape and dtype of ms3.bandpass_filter: M x (N / subsample_factor),
 * int16 when quantization_unit != 0 else float32 (p_bandpass_filter.cpp:134-142). */
MS3GPU_API int ms3gpu_bandpass_output_dims(int64_t M, int64_t N, const ms3gpu_bandpass_opts* opts,
                                int64_t* M_out, int64_t* N_out, int32_t* dtype_out);

/* "requirements" answers: the reference's peak-RAM model in MB
 * (p_bandpass_filter.cpp:157-158, p_whiten.cpp:53-57). */
MS3GPU_API int ms3gpu_bandpass_requirements(int64_t M, int64_t N, const ms3gpu_bandpass_opts* opts,
                                 double* peak_ram_mb);
MS3GPU_API int ms3gpu_whiten_requirements(int64_t M, int64_t N, double* peak_ram_mb);

/* ms3.bandpass_filter on a buffer.  Replaces p_bandpass_filter
 * (packages/ms3/p_bandpass_filter.cpp:115-229): overlap FFT filtering with
 * the reference's chunk geometry and band kernel (define_kernel, :421-447),
 * optional subsample (:480-491) and int16 quantization (:207-209).
 * timeseries_out has the shape and dtype of ms3gpu_bandpass_output_dims().
 * freq_max == 0 copies the input (:117-119). */
MS3GPU_API int ms3gpu_bandpass_filter(const float* timeseries, int64_t M, int64_t N, void* timeseries_out,
                           const ms3gpu_bandpass_opts* opts, void* stream);

/* ms3.whiten on a buffer.  Replaces p_whiten (packages/ms3/p_whiten.cpp:45-206):
 * XXt/(N-1), the power-iteration whitening matrix (pca.cpp:635-651), W^T x,
 * 1e-4 rounding and optional int16 quantization.  timeseries_out is M x N,
 * int16 when quantization_unit > 0 else float32. */
MS3GPU_API int ms3gpu_whiten(const float* timeseries, int64_t M, int64_t N, void* timeseries_out,
                  const ms3gpu_whiten_opts* opts, void* stream);

/* ms3.bandpass_filter on an int16 recording (an int16 .mda input), read
 * as the reference's reader converts it (mda/mdaio.cpp:205-230, int16 ->
 * float) -- here inside the filter's loads, so the int16 array is what
 * crosses PCIe and HBM.  Otherwise as ms3gpu_bandpass_filter; with
 * freq_max == 0 the output is an int16 copy of the input (the reference
 * copies the file). */
MS3GPU_API int ms3gpu_bandpass_filter_i16(const int16_t* timeseries, int64_t M, int64_t N, void* timeseries_out,
                                          const ms3gpu_bandpass_opts* opts, void* stream);

/* The two processors back to back as mountainsort3.mlp runs them
 * (ms3.bandpass_filter then ms3.whiten), sharing device buffers.
 * filt_out (the bandpass output, float32 M x N) may be NULL when the caller
 * does not need it.  Requires subsample_factor == 1 and
 * quantization_unit == 0 in bp (the pipeline's settings, whose filtered
 * output is float32 M x N). */
MS3GPU_API int ms3gpu_bandpass_whiten(const float* timeseries, int64_t M, int64_t N, float* filt_out,
                           void* pre_out, const ms3gpu_bandpass_opts* bp,
                           const ms3gpu_whiten_opts* wh, void* stream);

/* One recording of a batch: ms3.bandpass_filter then ms3.whiten, as
 * ms3gpu_bandpass_whiten (same buffer rules).  `status` receives the job's
 * result. */
typedef struct ms3gpu_job {
    const float* timeseries; /* M x N float32, host or device */
    int64_t M, N;
    float* filt_out;         /* optional, M x N float32 */
    void* pre_out;           /* M x N float32, int16 when wh.quantization_unit > 0 */
    ms3gpu_bandpass_opts bp; /* subsample_factor 1, quantization_unit 0 */
    ms3gpu_whiten_opts wh;
    int32_t status;          /* out: MS3GPU_OK or the job's error code */
} ms3gpu_job;

/* A batch of recordings of any sizes (no counterpart in the reference, which
 * runs one processor call per recording): the jobs run concurrently on a
 * few internal streams ordered after `stream`, so small recordings share
 * the GPU.  Outputs are those of n_jobs separate ms3gpu_bandpass_whiten
 * calls.  Returns MS3GPU_OK when every job succeeded, else the first failing
 * job's code (ms3gpu_last_error() names the job). */
MS3GPU_API int ms3gpu_bandpass_whiten_batch(ms3gpu_job* jobs, int32_t n_jobs, void* stream);

/* Stage: whiten pass 1 (p_whiten.cpp:64-118).  XXt = sum_t x_t x_t^T,
 * divided by N-1 when N > 1, M x M doubles. */
MS3GPU_API int ms3gpu_whiten_covariance(const float* timeseries, int64_t M, int64_t N, double* XXt,
                             void* stream);

/* Whiten pass 1 that allocates no memory.  No counterpart in the reference.
 *
 * Some callers cannot let the library call cudaMalloc: applications that
 * hand the whole GPU to their own memory pool before processing starts (an
 * extra allocation fails or fragments that pool), and streaming pipelines
 * whose processing loop must not stall on a device allocation, which may
 * synchronise the device.  This entry point computes the same XXt as
 * ms3gpu_whiten_covariance but keeps its partial sums in a fixed 16 MiB
 * array that is part of the library's device image (every GPU that loads the
 * library holds it until the process exits); it allocates nothing.
 *
 * timeseries and XXt must be device memory of the current device or managed
 * memory (host buffers would need staging, which allocates); other pointers
 * are rejected with MS3GPU_ERR_INVALID, and so is M above 1984 channels, the
 * most whose 64 x 64 partial tiles fit the array.  The work is queued on
 * `stream` and the call returns without waiting for it: XXt is ready once
 * the stream reaches that point (synchronise the stream, or order later work
 * after it).  The first call on a device looks the array's device address up
 * (cudaGetSymbolAddress) and keeps it for the life of the process; make that
 * first call before any stream capture, and do not keep using the entry
 * point after cudaDeviceReset on that device (the kept address would be
 * stale).  All calls share the one array, so calls that overlap on the GPU
 * (other streams, other host threads) race: serialise them.  Each call
 * overwrites every part of the array it reads. */
MS3GPU_API int ms3gpu_whiten_covariance_noalloc(const float* timeseries, int64_t M, int64_t N, double* XXt,
                                                void* stream);

/* Stage: whitening_matrix_from_XXt (packages/ms3/pca.cpp:635-651) with
 * pca_from_XXt (:172-195): M components of 10 power iterations each from
 * the start vector sin(1..M), deflation (I-cc')XXt(I-cc'), W = C D C' with
 * D = diag(1/sqrt(sigma)) (0 where sigma == 0).  FP64 on the GPU.
 * components (M x M) and sigma (M) may be NULL. */
MS3GPU_API int ms3gpu_whitening_matrix(const double* XXt, int64_t M, double* W, double* components,
                            double* sigma, void* stream);

/* Stage: whiten pass 2 (p_whiten.cpp:153-206): out(m1, t) = sum_m2
 * x(m2, t) W[m1*M + m2], rounded to multiples of 1e-4 (:31-41), then
 * int16 (int)(y/q + 0.5) when quantization_unit > 0 (:445-451).
 * precision: MS3GPU_PRECISION_PLAIN or MS3GPU_PRECISION_MIXED. */
MS3GPU_API int ms3gpu_apply_whitening_matrix(const float* timeseries, int64_t M, int64_t N, const double* W,
                                  double quantization_unit, int32_t precision, void* timeseries_out,
                                  void* stream);

/* ms3.compute_whitening_matrix (p_whiten.cpp:208-298): XXt over the
 * recordings of timeseries_list concatenated in time (n_inputs arrays of M
 * channels; recording i has N_list[i] timepoints), restricted to `channels`
 * (n_channels 1-based channel numbers, the processor's "channels" parameter;
 * NULL / 0 = all M), divided by (sum of N_list) - 1 when that is above 1,
 * then the whitening matrix of ms3gpu_whitening_matrix.  W_out: M2 x M2
 * doubles (M2 = n_channels, or M), column-major.  Channel numbers outside
 * [1, M] are MS3GPU_ERR_INVALID (the reference indexes out of range). */
MS3GPU_API int ms3gpu_compute_whitening_matrix(const float* const* timeseries_list, const int64_t* N_list,
                                               int32_t n_inputs, int64_t M, const int32_t* channels,
                                               int32_t n_channels, double* W_out, void* stream);

/* ms3.whiten per channel block (per shank): the channels are split into
 * n_blocks blocks -- block k holds block_sizes[k] 1-based channel numbers,
 * listed block after block in `channels` -- that together name every channel
 * of X exactly once.  Each block is whitened on its own (its XXt, its
 * power-iteration W, its apply with the 1e-4 rounding) and written back to
 * its channels of the M x N output: the same result as
 * ms3.compute_whitening_matrix with the block's channels followed by
 * ms3.apply_whitening_matrix on those channels. */
MS3GPU_API int ms3gpu_whiten_blocks(const float* timeseries, int64_t M, int64_t N, const int32_t* channels,
                                    const int32_t* block_sizes, int32_t n_blocks, void* timeseries_out,
                                    const ms3gpu_whiten_opts* opts, void* stream);

/* ms3.whiten_clips (p_whiten.cpp:300-345): for every timepoint of every clip
 * of an M x T x L float32 array, out(m1, t, l) = sum_m2 x(m2, t, l)
 * W[m1*M + m2] -- the apply of ms3gpu_apply_whitening_matrix without the 1e-4
 * rounding -- then int16 (int)(y/q + 0.5) when quantization_unit > 0. */
MS3GPU_API int ms3gpu_whiten_clips(const float* clips, int64_t M, int64_t T, int64_t L, const double* W,
                                   double quantization_unit, int32_t precision, void* clips_out, void* stream);

/* ms3.mask_out_artifacts (p_mask_out_artifacts.cpp:24-104): per channel the
 * norm of every whole interval of interval_size timepoints; an interval
 * whose norm exceeds the channel's mean + threshold * stdev (over its
 * intervals) is zeroed together with its two neighbours, on all channels;
 * timepoints after the last whole interval are zero.  float32 M x N in and
 * out.  threshold == 0 or interval_size <= 0 is MS3GPU_ERR_INVALID (the
 * reference refuses them).  *timepoints_kept (may be NULL) receives the
 * number of timepoints kept. */
MS3GPU_API int ms3gpu_mask_out_artifacts(const float* timeseries, int64_t M, int64_t N, double threshold,
                                         int64_t interval_size, float* timeseries_out, int64_t* timepoints_kept,
                                         void* stream);

/* Event detection of mountainsortalg on a (whitened) timeseries, the first
 * consumer of this path's output: detect_events
 * (mountainsortalg/detect_events.cpp:69-135) as NeighborhoodSorter::
 * addTimeChunk applies it (neighborhoodsorter.cpp:74-100) to every channel
 * (each channel is the centre of its own neighborhood) over the time chunks
 * of p_mountainsort3.cpp:190-215: chunks of chunk_size timepoints with 1000
 * timepoints of padding on both sides (zeros outside the recording), the
 * chunk's mean and stdev, samples whose deviation (sign > 0), negated
 * deviation (sign < 0) or absolute deviation (sign == 0) exceeds
 * detect_threshold * stdev, the greedy strongest-within-detect_interval rule,
 * times kept inside the unpadded chunk.  chunk_size <= 0 selects the
 * reference's get_time_chunk_infos length for one simultaneous batch
 * (p_mountainsort3.cpp:507-517).
 *
 * counts (M entries) receives each channel's number of events; times
 * receives all events, channel after channel, each channel's times sorted
 * (timepoint indices).  times may be NULL to ask for counts only; when the
 * events exceed `capacity` the call fails with MS3GPU_ERR_INVALID after
 * filling counts. */
MS3GPU_API int ms3gpu_detect_events(const float* timeseries, int64_t M, int64_t N, double detect_threshold,
                                    double detect_interval, int32_t detect_sign, int64_t chunk_size, int64_t* counts,
                                    int64_t* times, int64_t capacity, void* stream);

/* Streaming I/O.  The reference never holds a recording in memory: its
 * processors read chunks through DiskReadMda32::readChunk
 * (mda/diskreadmda32.cpp:615-661) and write them through
 * DiskWriteMda::writeChunk (mda/diskwritemda.cpp:255-265).  The streaming
 * entry points take the same shape of access as callbacks:
 *
 *   read(read_ctx, t0, nt, dst): fill dst with timepoints [t0, t0 + nt) of
 *     the input, M values per timepoint (channel fastest), in the input
 *     dtype; 0 <= t0 and t0 + nt <= N.
 *   write(write_ctx, t0, nt, src): take output timepoints [t0, t0 + nt),
 *     M values per timepoint, in the output dtype.
 *
 * Both return 0 on success; anything else stops the call with MS3GPU_ERR_IO.
 * They are called from the calling thread, in increasing t0, and each
 * buffer is valid only during its call.  Output timepoints that no write
 * covers (the gaps between subsampled chunks) are zero, as in the reference's
 * preallocated file.  slab_bytes bounds the rows of one read (about that
 * many bytes; 0 = 1 GiB); the call holds two slabs of input and two of
 * output in pinned host memory and as many on the device. */
typedef int (*ms3gpu_read_fn)(void* ctx, int64_t t0, int64_t nt, void* dst);
typedef int (*ms3gpu_write_fn)(void* ctx, int64_t t0, int64_t nt, const void* src);

typedef struct ms3gpu_stream_io {
    ms3gpu_read_fn read;
    void* read_ctx;
    ms3gpu_write_fn write;
    void* write_ctx;
    int64_t slab_bytes;
} ms3gpu_stream_io;

/* ms3.bandpass_filter over a recording of M x N read and written through
 * `io`: the processor's own chunk loop (p_bandpass_filter.cpp:160-220).
 * in_dtype: MS3GPU_DTYPE_FLOAT32 or MS3GPU_DTYPE_INT16 (converted on load as
 * ms3gpu_bandpass_filter_i16 does).  The output has the shape and dtype of
 * ms3gpu_bandpass_output_dims(), except that freq_max == 0 copies the input
 * rows unchanged in in_dtype.  Every output value equals the in-memory call's. */
MS3GPU_API int ms3gpu_bandpass_filter_stream(int64_t M, int64_t N, int32_t in_dtype, const ms3gpu_stream_io* io,
                                             const ms3gpu_bandpass_opts* opts, void* stream);

/* ms3.whiten over a float32 recording read and written through `io`, with
 * the reference's two passes over the input (p_whiten.cpp:64-118 reads every
 * chunk for XXt, :153-206 reads them again for the apply): the input is read
 * twice, in increasing t0 each time.  Output as ms3gpu_whiten; every value
 * equals the in-memory call's when a slab holds one slice of the covariance
 * sum (about N / 56 timepoints at M = 384; N / 1184 at M <= 64), and differs
 * otherwise only by the order of the FP64 covariance additions. */
MS3GPU_API int ms3gpu_whiten_stream(int64_t M, int64_t N, const ms3gpu_stream_io* io,
                                    const ms3gpu_whiten_opts* opts, void* stream);

/* ms3.mask_out_artifacts over a float32 recording read and written through
 * `io`: the input is read twice (the interval norms, then the masked copy),
 * in blocks of whole intervals.  Output and *timepoints_kept equal
 * ms3gpu_mask_out_artifacts'. */
MS3GPU_API int ms3gpu_mask_out_artifacts_stream(int64_t M, int64_t N, double threshold, int64_t interval_size,
                                                const ms3gpu_stream_io* io, int64_t* timepoints_kept,
                                                void* stream);

/* Time sharding.  The recording's windows (chunks of ms3gpu_bandpass_chunk_size
 * timepoints) are independent, and the covariance is a sum over time, so the
 * path splits along time across GPUs with one exchange: every GPU filters its
 * own windows, sums x x^T over its own filtered timepoints, the M x M sums are
 * added over the GPUs (a collective of the caller's choice), every GPU forms
 * W from the total divided by N - 1 (ms3gpu_whitening_matrix: deterministic,
 * so identical everywhere) and applies it to its own timepoints
 * (ms3gpu_apply_whitening_matrix).  Whitened values equal the one-GPU call's
 * up to the grouping of the FP64 covariance additions.
 *
 * ms3gpu_bandpass_filter_windows: p_bandpass_filter's chunk loop
 * (p_bandpass_filter.cpp:160-220) restricted to windows [c_begin, c_end) of
 * an M x N recording, on a slab: `timeseries` holds `rows` timepoints starting
 * at timepoint row0 (in_dtype MS3GPU_DTYPE_FLOAT32 or MS3GPU_DTYPE_INT16), and
 * must cover the windows' reads [c_begin*chunk - 60000, c_end*chunk + 60000)
 * clipped to [0, N); `timeseries_out` holds out_rows output timepoints from
 * out_row0 and must cover [c_begin*chunk, c_end*chunk) / subsample_factor
 * clipped to N / subsample_factor.  Output values equal the whole-recording
 * call's; other rows of timeseries_out are left as they are.  freq_max == 0
 * is MS3GPU_ERR_INVALID (the copy takes whole recordings). */
MS3GPU_API int ms3gpu_bandpass_filter_windows(const void* timeseries, int32_t in_dtype, int64_t M, int64_t N,
                                              int64_t row0, int64_t rows, int64_t c_begin, int64_t c_end,
                                              void* timeseries_out, int64_t out_row0, int64_t out_rows,
                                              const ms3gpu_bandpass_opts* opts, void* stream);

/* Whiten pass 1 (p_whiten.cpp:64-118) over one shard of timepoints without
 * the division: XXt_sum = sum over the N timepoints of x_t x_t^T, M x M
 * doubles. */
MS3GPU_API int ms3gpu_whiten_covariance_sum(const float* timeseries, int64_t M, int64_t N, double* XXt_sum,
                                            void* stream);

#ifdef __cplusplus
}
#endif

#endif /* MS3GPU_H */

/*
 * ccfj_b200 -- C ABI of the B200 (sm_100a) frequency-Bessel (F-J) transform.
 *
 * Every entry point takes plain pointers and sizes, returns an int status
 * (CCFJ_OK = 0) and never exits the process or resets the device; on failure
 * ccfj_last_error() returns a message for the calling thread.
 *
 * Array conventions follow the reference (src/FJcpu.cpp:247-256):
 *   u_f  float32 [nr, nf]   row ir = station pair ir (pairs sorted by r),
 *                           element index i + ir*nf
 *   r    float32 [nr]       pair distances (ascending for the F-J method;
 *                           as in the reference, unsorted input is integrated
 *                           interval by interval in the given order)
 *   f    float32 [nf]       frequencies (Hz)
 *   c    float32 [nc]       phase velocities (same length unit as r per s)
 *   out  float32 [nc, nf]   element index i + j*nf
 */
#ifndef CCFJ_B200_H
#define CCFJ_B200_H

#include <stddef.h>

#ifdef __cplusplus
#define CCFJ_API extern "C" __attribute__((visibility("default")))
#else
#define CCFJ_API __attribute__((visibility("default")))
#endif

/* ------------------------------------------------------------ status codes */
#define CCFJ_OK 0
#define CCFJ_ERR_INVALID 1     /* bad argument (size, pointer, enum)        */
#define CCFJ_ERR_CUDA 2        /* a CUDA runtime call or launch failed      */
#define CCFJ_ERR_ALLOC 3       /* device or pinned allocation failed        */
#define CCFJ_ERR_UNSUPPORTED 4 /* valid request the library cannot serve   */
#define CCFJ_ERR_TIMEOUT 5     /* a bounded device-side wait ran out        */

/* --------------------------------------------- reference-compatible entry
 * Drop-in for the reference's GPU library (include/FJgpu.hh:13-15), with the
 * semantics of its CPU library (src/FJcpu.cpp:401-419):
 *   FJ / FHr : Bessel basis J   (type 1: integral_J, type 0: trap_J)
 *   FHi      : Hankel basis Y   (type 1: integral_Y, type 0: trap_Y)
 * All pointers are HOST memory; the call is synchronous; out is overwritten.
 * The reference's GPU FJ with type 1 ran integral_c (src/FJgpu.cu:315-358),
 * a truncated odd-Bessel series that does not match its own CPU FJ; this FJ
 * follows the CPU definition.
 * Unlike the reference (which returns 0 and leaves out untouched for any
 * other type), an invalid type returns CCFJ_ERR_INVALID.
 */
CCFJ_API int FJ(float *u_f, float *r, float *f, float *out, float *c, int nc, int nr, int nf,
                int type);
CCFJ_API int FHr(float *u_f, float *r, float *f, float *out, float *c, int nc, int nr, int nf,
                 int type);
CCFJ_API int FHi(float *u_f, float *r, float *f, float *out, float *c, int nc, int nr, int nf,
                 int type);
/* The CPU library's Hankel entry (include/FJcpu.h:20); nThread is accepted
 * and ignored (all work runs on the current CUDA device). */
CCFJ_API int FH(float *u_f, float *r, float *f, float *out, float *c, int nc, int nr, int nf,
                int type, int nThread);

/* ------------------------------------------------------ general transform */
#define CCFJ_MODE_J 0      /* out = FJ(u0)                                      */
#define CCFJ_MODE_Y 1      /* out = FH(u0)  (Y basis)                           */
#define CCFJ_MODE_J_MINUS_Y 2 /* out = FJ(u0) - FH(u1)   (fj_noise func=1)       */
#define CCFJ_MODE_ABS_J 3  /* out = |FJ(u0) + i FJ(u1)|  (fj_earthquake func=0)  */
#define CCFJ_MODE_ABS_H 4  /* out = |(FJ(u0)-FH(u1)) + i(FJ(u1)+FH(u0))|  (func=1)*/

#define CCFJ_PREC_FP32 0       /* station-amortised FP32 (fast path)           */
#define CCFJ_PREC_FP64 1       /* station-amortised FP64                        */
#define CCFJ_PREC_FP64_PLAIN 2 /* reference loop structure in FP64 (comparator) */

typedef struct ccfj_fj_args {
  int struct_size;     /* sizeof(ccfj_fj_args)                                 */
  int nr, nf, nc;      /* pairs, frequencies, velocities                       */
  int itype;           /* 1: linear-interpolation integral, 0: trapezoid       */
  int mode;            /* CCFJ_MODE_*                                          */
  int precision;       /* CCFJ_PREC_*                                          */
  int normalize;       /* 1: out[:, i] /= max|out[:, i]| (reference semantics) */
  int device_ptrs;     /* 1: every pointer is device memory, call is async on  */
                       /*    `stream`; 0: host memory, call is synchronous     */
  int hilbert;         /* 1 (mode J_MINUS_Y only, u[1] = NULL): u[1] is the    */
                       /*    Hilbert transform of each full row of u[0] along  */
                       /*    frequency, as scipy.fftpack.hilbert              */
  const float *u[2];   /* input spectra; u[1] only for two-input modes         */
  long long u_ld;      /* elements between rows of u (station pairs)           */
  long long u_rows;    /* rows present in u (>= nr; >= max(perm)+1)            */
  int u_es;            /* elements between adjacent columns (1: float32 data;  */
                       /*    2: one part of interleaved complex64 data)        */
  int u_ncols;         /* columns per row; column j is u[row*u_ld + j*u_es]    */
  int fstride;         /* frequency i uses column i*fstride (needs            */
                       /*    ceil(u_ncols/fstride) == nf, as the reference)    */
  const long long *perm; /* optional [nr]: row of u for sorted pair i          */
  const float *r;      /* [nr] distances of the sorted pairs                    */
  const float *f;      /* [nf]                                                  */
  const float *c;      /* [nc]                                                  */
  float *out;          /* [nc, nf]                                              */
  float tau;           /* Hermite/closed-form switch in k*dr; <= 0: default    */
  int col_begin;       /* compute frequencies col_begin .. col_begin + nf - 1  */
  int nf_total;        /*    of the nf_total the rows hold (0: nf_total = nf); */
                       /*    f and out hold the computed frequencies only     */
} ccfj_fj_args;

CCFJ_API int ccfj_fj_v1(const ccfj_fj_args *args, void *stream);

/* -------------------------------------------------------- ragged batch
 * Many data sets (subarrays) with their own pairs, distances and spectra
 * but shared f and c grids, in one persistent launch: equivalent to calling
 * the transform once per set (fj_noise per subarray), with the sets' pairs
 * concatenated. Set b owns pairs offsets[b] .. offsets[b+1]-1 (each set
 * non-empty, distances ascending within it); perm maps pair i to its row of
 * u (global rows). out is [nsets][nc][nf]. FP32 only.
 *   use_graph = 1: the launch sequence is captured once per distinct
 *     argument set into a CUDA graph and replayed on later calls (device
 *     mode; ignored when the stream is already being captured by the
 *     caller, or when a caller allocator is installed). The library keeps
 *     the 16 most recently launched graphs and destroys older ones. With
 *     stream NULL (the legacy default stream, which cannot capture) the
 *     graph runs on a library stream that events order after the caller's
 *     earlier default-stream work and before its later default-stream
 *     work, as a launch on stream 0 would be.
 *   variant: velocities per thread, 1, 2 or 4 (0 = the choice recorded by
 *     ccfj_autotune_batch_v1 for the batch's class, else the untuned
 *     per-mode default described at ccfj_set_fj_variant).
 * No counterpart in the reference, which has no batch entry.
 */
typedef struct ccfj_batch_args {
  int struct_size;     /* sizeof(ccfj_batch_args)                              */
  int nsets;           /* data sets                                            */
  int nf, nc;          /* shared frequency / velocity grids                    */
  int itype, mode;     /* as ccfj_fj_args                                      */
  int precision;       /* CCFJ_PREC_FP32 only                                  */
  int normalize;       /* per (set, frequency) max-abs normalisation           */
  int device_ptrs;     /* as ccfj_fj_args                                      */
  int hilbert;         /* as ccfj_fj_args (mode J_MINUS_Y, u[1] = NULL)        */
  int use_graph;       /* capture and replay a CUDA graph (device mode)        */
  int variant;         /* 0, 1, 2 or 4                                         */
  const long long *offsets; /* [nsets + 1], offsets[0] = 0                     */
  long long total_pairs;    /* offsets[nsets] (required in device mode)        */
  const float *r;      /* [total_pairs], ascending within each set             */
  const float *u[2];   /* spectra rows, layout as ccfj_fj_args                 */
  long long u_ld;
  long long u_rows;
  int u_es;
  int u_ncols;
  int fstride;
  const long long *perm; /* optional [total_pairs]                            */
  const float *f;
  const float *c;
  float *out;          /* [nsets][nc][nf]                                      */
  float tau;
} ccfj_batch_args;

CCFJ_API int ccfj_fj_batch_v1(const ccfj_batch_args *args, void *stream);
/* Destroys the cached batch graphs (call before freeing buffers that a
 * cached graph refers to, if their addresses may be reused). */
CCFJ_API int ccfj_batch_graph_cache_clear(void);
/* Runs the batch (device pointers; out is overwritten) with 1, 2 and 4
 * velocities per thread, records the fastest for the batch's class (mode,
 * itype and the powers of two of total pairs, nsets, nf and nc) on this
 * device for later calls that pass variant 0 -- in this process, and in
 * later ones through the persistent table of ccfj_set_tune_cache -- and
 * returns it and its time. */
CCFJ_API int ccfj_autotune_batch_v1(const ccfj_batch_args *args, void *stream,
                                    int *best_variant, float *best_ms);

/* ------------------------------------------ allocation-free transform
 * No counterpart in the reference. The same FP32 transform as ccfj_fj_v1
 * with device pointers (device_ptrs = 1, precision CCFJ_PREC_FP32,
 * hilbert = 0), for callers that cannot allocate device memory during the
 * call: a host whose own pool allocator already holds the free device
 * memory, or code that must avoid the device-wide synchronisation that
 * cudaMalloc/cudaFree may cause. The caller still passes every input and the
 * output; the call itself allocates nothing (no cudaMalloc, cudaFree or
 * allocating library routine).
 *
 * Its scratch is one fixed 16 MiB array in the library's device image. A GPU
 * holds it from the moment the CUDA runtime loads the code module that
 * contains it onto that GPU until the process exits. Under lazy module
 * loading (CUDA_MODULE_LOADING=LAZY, the default since CUDA 12.2) that moment
 * is this entry point's first call on the device (or the first launch of a
 * kernel of the same file), so that first call itself reserves the 16 MiB.
 * It fits 24 * nr (+ 4 * nf for itype 1) plus, per input, 16 bytes (itype 1)
 * or 4 bytes (itype 0) per (pair, frequency): about nr * nf <= 1.04e6 for
 * one itype-1 input. Larger problems are rejected with CCFJ_ERR_INVALID and
 * a message giving both sizes.
 *
 * The first call on each device also looks up the array's device address
 * with that device current. Make that first call -- a warm-up call on a
 * small problem will do -- on every device before handing the free device
 * memory to your own pool allocator, and before any stream capture.
 * Every call uses the same array and leaves its contents behind (each call
 * writes all the scratch it reads, so nothing is cleared): calls whose work
 * overlaps on the GPU -- on different streams, or from different threads --
 * race on it and must be serialised by the caller. */
CCFJ_API int ccfj_fj_noalloc_v1(const ccfj_fj_args *args, void *stream);

/* ------------------------------------------ earthquake / multi-window F-J
 * fj_earthquake (src/ccfj-gpu.pyx:270-295) and MWFJ (:297-313) from
 * time-domain traces: optional taper window, real FFT on the device, F-J of
 * the real and imaginary parts, magnitude, per-frequency normalisation.
 *   func 0: out = |FJ(Re) + i FJ(Im)|
 *   func 1: out = |(FJ(Re) - FH(Im)) + i (FJ(Im) + FH(Re))|
 * Windows (nwin > 0) are the reference's `win` per (window w, trace j) given
 * by its integer sample range [n1, n2) and ramp length delta, arrays
 * [nwin][u_rows] indexed by the row of u (the caller's trace order). The
 * transform of every window shares one station geometry.
 */
typedef struct ccfj_eq_args {
  int struct_size;     /* sizeof(ccfj_eq_args)                                 */
  int ntr, npts;       /* traces (= station pairs) and samples per trace       */
  int nf, nc;          /* frequencies (bins k*fstride, k < nf), velocities     */
  int itype, func;     /* as ccfj_fj_args.itype; func 0 or 1 (see above)       */
  int precision;       /* CCFJ_PREC_*                                          */
  int normalize;       /* per-frequency max-abs normalisation of every window */
  int device_ptrs;     /* as ccfj_fj_args.device_ptrs                          */
  int fstride;         /* FFT bin of frequency k is k*fstride                  */
  int nwin;            /* 0: no window, out is [nc, nf]; else [nwin, nc, nf]   */
  const float *u;      /* traces, float32 [u_rows][u_ld], npts used            */
  long long u_ld;
  long long u_rows;
  const long long *perm; /* optional [ntr]: row of u of sorted trace i          */
  const float *r;      /* [ntr] distances of the sorted traces                  */
  const float *f;      /* [nf]                                                  */
  const float *c;      /* [nc]                                                  */
  const int *win_n1;   /* [nwin][u_rows] when nwin > 0                          */
  const int *win_n2;
  const int *win_delta;
  float *out;
  float tau;           /* as ccfj_fj_args.tau                                   */
  int out_f64;         /* 1: out points to doubles (MWFJ's result type); host
                          pointers only. The result is converted while it is
                          copied out. 0: floats                                 */
} ccfj_eq_args;

CCFJ_API int ccfj_fj_earthquake_v1(const ccfj_eq_args *args, void *stream);
/* MWFJ contraction of the windows: 0 = automatic (tensor cores, tcgen05
 * FP16x3 (hi/lo fp16 operands with exact power-of-two scales) with FP32
 * accumulation, for itype 1, func 0 and 8 <= nwin <= 128;
 * CUDA-core FMAs otherwise), 1 = always CUDA cores, 2 = tensor cores
 * wherever supported, 3 = as 2 with the A operand generated one interval at
 * a time (no paired FP32 arithmetic; for checks, the results agree with 2
 * to rounding). */
CCFJ_API int ccfj_set_mwfj_path(int path);
/* Waits for `stream` and reports CCFJ_ERR_TIMEOUT if a bounded device-side
 * wait of a tensor-core kernel ran out, in any call on this device, since
 * the previous ccfj_device_status (which clears the record). Host-memory
 * calls check their own kernels' waits through a flag of their own, so
 * calls that overlap on different streams or threads neither clear nor
 * inherit each other's timeouts. */
CCFJ_API int ccfj_device_status(void *stream);
/* Self-test of the bounded waits: runs one CTA of the tensor-core MWFJ
 * kernel whose input copy is never issued, with a ~1 ms wait limit, and
 * returns CCFJ_OK if the kernel gave up, reported the timeout and left the
 * device usable (CCFJ_ERR_CUDA otherwise). No counterpart in the reference. */
CCFJ_API int ccfj_self_test_wait_timeout(void *stream);

/* ---------------------------------------- ambient-noise cross-correlation
 * The reference's CrossCorrelation (src/CrossCorr.cpp:33-159, called by CC
 * in src/ccfj.pyx:125-147): per station, windows of fftlen samples every
 * steplen samples (one window of npts samples when fftlen >= npts), kept
 * where k*steplen >= startend[2i] and k*steplen + fftlen < startend[2i+1];
 * optional one-bit (sign) of the samples; real FFT of each kept window at
 * bins j*fstride, j < nf, optionally whitened to X/max(|X|, 1e-8); for each
 * pair (a, b) the mean over the windows both keep of conj(X_a) X_b.
 * Unlike the reference, bins past fftlen/2, steplen <= 0 with
 * fftlen < npts, and pair indices outside [0, nsta) return
 * CCFJ_ERR_INVALID. Windows of up to 16384 samples whose half length has no
 * prime factor above 5 use a shared-memory FFT; other lengths a direct
 * transform of the requested bins.
 */
typedef struct ccfj_cc_args {
  int struct_size;     /* sizeof(ccfj_cc_args)                                 */
  int nsta, npts;      /* stations and samples per station record              */
  int nf, npairs;      /* output bins and station pairs                        */
  int fstride;         /* output bin j is FFT bin j*fstride                    */
  int fftlen, steplen; /* window length and step in samples                    */
  int onebit;          /* nonzero: use sign(sample)                            */
  int whiten;          /* nonzero: whiten each window's spectrum              */
  int device_ptrs;     /* 1: data and outputs are device memory, the call is  */
                       /*    async on `stream` (pairs and startend stay host); */
                       /*    0: host memory, the call is synchronous and       */
                       /*    one-bit rewrites data in place, as the reference  */
  int accumulate;      /* 1: the sums are added to the outputs' contents       */
                       /*    before the division (the reference's +=); pairs  */
                       /*    with no common window keep their contents;        */
                       /*    0: outputs are overwritten, such pairs get 0      */
  int out_layout;      /* 0: out_re and out_im are float32 [npairs][nf];       */
                       /* 1: out_re is complex64 [npairs][nf], out_im unused   */
  const int *pairs;    /* host [2*npairs]: stations (a, b) of each pair        */
  const int *startend; /* host [2*nsta]: kept sample range [start, end)        */
  float *data;         /* [nsta][npts] float32                                 */
  float *out_re;
  float *out_im;
} ccfj_cc_args;

CCFJ_API int ccfj_cc_v1(const ccfj_cc_args *args, void *stream);

/* Drop-in for the reference's entry (include/CrossCorr.h:13-33), with its
 * struct layout: host memory, synchronous, ncfsr/ncfsi [npairs][nf]
 * accumulated into and divided as the reference does, data rewritten in
 * place by one-bit. nThreads is accepted and ignored. Returns a status
 * (the reference always returns 0). */
typedef struct ccfj_cc_data {
  int nsta;
  int npts;
  int nf;
  int npairs;
  int fstride;
  int fftlen;
  int steplen;
  int *Pairs;
  int *startend;
  float *data;
  float *ncfsr;
  float *ncfsi;
  int ifonebit;
  int ifspecwhitenning;
  int nThreads;
} ccfj_cc_data;

CCFJ_API int CrossCorrelation(ccfj_cc_data data);

/* ------------------------------------- records to dispersion spectrum
 * The reference's ambient-noise pipeline, CC then fj_noise
 * (examples/example_noise.py:6-11 over src/ccfj.pyx:125-147 and
 * src/ccfj-gpu.pyx:241-268), in one call whose cross-spectra never leave the
 * device: the cross-correlation writes them into device scratch and the
 * transform reads their real parts there.
 *   cc: as ccfj_cc_v1, with accumulate = 0; out_re, out_im and out_layout
 *       are not used. Unlike CC, one-bit never rewrites cc->data (the
 *       records are read, signed on load, and left as they were).
 *   fj: as ccfj_fj_v1 for the transform of those spectra: nr = cc->npairs,
 *       nf = cc->nf, mode CCFJ_MODE_J (fj_noise func 0) or
 *       CCFJ_MODE_J_MINUS_Y (func 1: the Hilbert transform of each pair's
 *       spectrum along frequency is taken on the device); u, u_ld, u_rows,
 *       u_es, u_ncols, fstride, hilbert, col_begin and nf_total are set by
 *       the call. perm (optional) maps sorted pair i to its row of the
 *       cross-spectra, r is the sorted distances, f the nf frequencies of the
 *       bins, c the velocities, out [nc][nf].
 *   cc->device_ptrs must equal fj->device_ptrs. Host mode: the records cross
 *   to the device once, the [nc][nf] result once back, and the call is
 *   synchronous. No counterpart entry in the reference, which returns the
 *   cross-spectra to the host between the two steps. */
CCFJ_API int ccfj_cc_fj_noise_v1(const ccfj_cc_args *cc, const ccfj_fj_args *fj, void *stream);

/* ------------------------------------------------- dispersion-curve picking
 * Per frequency column of a spectrum spec[nc][nf] (e.g. a normalised F-J
 * spectrum): the velocity of the first largest value among the velocities
 * c[j] within [cmin[i], cmax[i]] (NULL: no bound), refined between the grid
 * velocities by the vertex of the parabola through the maximum and its two
 * neighbours (when both lie in the band and the parabola opens downward;
 * the offset limited to half a grid step), into cpick[nf], and that
 * vertex's value into amp[nf] (amp may be NULL). A column with a NaN in the
 * band, or with no velocity in it, gives NaN. device_ptrs as in
 * ccfj_fj_args. No counterpart in the reference, whose users pick curves
 * from the plotted spectrum. */
CCFJ_API int ccfj_pick_v1(const float *spec, int nc, int nf, const float *c, const float *cmin,
                          const float *cmax, float *cpick, float *amp, int device_ptrs,
                          void *stream);

/* ------------------------------------------------------------- tuning
 * Tile choices of the FP32 transform: 1, 2 or 4 velocities per thread, and
 * the number of station ranges (split launch: ranges of whole 32-station
 * chunks summed in a fixed order by a second kernel, so a given choice
 * gives the same result on every run). ccfj_autotune_fj_v1 times every
 * velocities-per-thread variant with 1 range and, where the unsplit grid
 * leaves resident slots idle, with 2-8 ranges, on the given problem (device
 * pointers; out is overwritten), records the fastest for the problem's
 * class (mode, itype and the powers of two of nr, nf, nc) on this device,
 * and returns its velocities per thread and time. Untuned classes use 2
 * (itype 1) or 4 (itype 0) velocities per thread and as many ranges (at
 * most 4) as fill the SMs' resident slots without starting another wave.
 * ccfj_set_fj_variant(cpt) forces a velocities-per-thread variant (0
 * restores the tuned or default choice).
 *
 * Persistence: ccfj_set_tune_cache(path) names a text table that both
 * autotuners write every result to and that later calls (in this or any
 * later process) read per device, one line per (device name, tuner,
 * problem class); NULL returns to the default, the file named by the
 * environment variable CCFJ_TUNE_CACHE, or none. ccfj_tuned_choice_fj
 * reports the choice a call with these arguments would run. No
 * counterparts in the reference, which has no tuning. */
CCFJ_API int ccfj_autotune_fj_v1(const ccfj_fj_args *args, void *stream, int *best_cpt,
                                 float *best_ms);
CCFJ_API int ccfj_set_fj_variant(int cpt);
/* Forces the number of station ranges of FP32 transforms (1 = unsplit;
 * 0 restores the tuned or default choice). */
CCFJ_API int ccfj_set_fj_split(int nsplit);
CCFJ_API int ccfj_set_tune_cache(const char *path);
CCFJ_API int ccfj_tuned_choice_fj(const ccfj_fj_args *args, int *cpt, int *nsplit);

/* ------------------------------------------------------------------ misc */
CCFJ_API const char *ccfj_last_error(void);
CCFJ_API const char *ccfj_version(void);
/* Kernel launches issued by this library since load (all threads). */
CCFJ_API long long ccfj_launch_count(void);

/* Optional timing: after ccfj_profile_enable(1) (which also resets the
 * record), every transform records a pair of CUDA events on its stream
 * around its main F-J kernel (up to 512 pairs; no synchronisation is added).
 * ccfj_last_transform_ms() waits for the last pair and returns its duration
 * in ms (-1 if none); ccfj_profile_total_ms() waits for all of them and
 * returns the summed ms, with the number of pairs in *count. */
CCFJ_API int ccfj_profile_enable(int on);
CCFJ_API float ccfj_last_transform_ms(void);
CCFJ_API double ccfj_profile_total_ms(int *count);
/* FP32 FMA throughput of the current device in TFLOP/s (FMA = 2 flops),
 * measured with independent FMA chains on `stream`: the roofline peak of the
 * transform kernels, which are bound by the FP32 pipe. */
CCFJ_API int ccfj_fp32_peak_probe(void *stream, double *tflops);

/* Replaces the device allocator of the library's scratch memory (NULL, NULL
 * restores the default: stream-ordered allocation from a library-owned
 * memory pool per device that keeps its memory between calls). alloc returns
 * NULL on failure; both receive the cudaStream_t of the call as void*. */
typedef void *(*ccfj_alloc_fn)(size_t bytes, void *stream, void *user);
typedef void (*ccfj_free_fn)(void *ptr, void *stream, void *user);
CCFJ_API int ccfj_set_allocator(ccfj_alloc_fn alloc, ccfj_free_fn free_fn, void *user);

/* Page-locked (pinned) host memory of `bytes` bytes, usable by every device
 * (cudaHostAlloc, portable), and its release. Host arrays in pinned memory
 * cross to the device by DMA without a staging copy; ccfj.load_ncfs reads
 * stored cross-spectra straight into such a buffer. No counterpart in the
 * reference. */
CCFJ_API int ccfj_host_alloc(size_t bytes, void **ptr);
CCFJ_API int ccfj_host_free(void *ptr);

#endif /* CCFJ_B200_H */

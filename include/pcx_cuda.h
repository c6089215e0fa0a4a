/*
 * pcx_cuda.h — C ABI of the B200 (sm_100a) FFT / correlation library
 * (libpcx_cuda.so).  Plain pointers and sizes only; every call returns an
 * int status (PCX_OK = 0) and pcx_last_error() gives the message of the last
 * failing call on the calling thread.
 *
 * Data layout everywhere: packed split-complex at pack width P (a power of
 * two): per pack of P elements, P reals then P imaginaries — the layout of
 * pcxo::vector<T, P> (reference vector.hpp:26-382, element access
 * element_access.hpp:8-11).  P = 1 is interleaved complex
 * (std::vector<std::complex<T>>, reference types.hpp:119-148).
 * Pointers passed to exec calls are DEVICE pointers (or managed memory),
 * 16-byte aligned; strides count reals (T) between consecutive rows.
 *
 * The reference (Dooez/packed) is a header-only C++ template library with no
 * FFI of its own; each entry point below names the reference interface whose
 * behaviour it carries.  The headers in include/pcxo/ wrap these calls in the
 * reference's own class templates.
 */
#ifndef PCX_CUDA_H
#define PCX_CUDA_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define PCX_OK 0
#define PCX_ERR_INVALID 1      /* std::invalid_argument in the reference      */
#define PCX_ERR_CUDA 2         /* CUDA runtime failure                        */
#define PCX_ERR_UNSUPPORTED 3  /* valid in the reference, not built here      */
#define PCX_ERR_TIMEOUT 4      /* a bounded device wait gave up               */

/* element types */
#define PCX_F32 0
#define PCX_F64 1

/* output / input orders — reference fft_order, fft.hpp:540-544 */
#define PCX_ORDER_NORMAL 0
#define PCX_ORDER_BIT_REVERSED 1
#define PCX_ORDER_UNORDERED 2

/* directions */
#define PCX_FORWARD 0
#define PCX_INVERSE 1

typedef struct pcx_plan_s*   pcx_plan;
typedef struct pcx_fxcorr_s* pcx_fxcorr;

/* Message of the last failing call on this thread ("" if none). */
const char* pcx_last_error(void);

/* Library version string. */
const char* pcx_version(void);

/*
 * FFT plan.  Replaces the constructor fft_unit<T, Order>(fft_size, sub_size)
 * (reference fft.hpp:594-605; size checks check_size 1806-1812 and
 * check_sub_size 1814-1826, twiddle/sort tables get_twiddles 1969-2050).
 * n: power of two, 2 <= n <= 2^20.  sub_size: power of two >= 8 (validated as
 * the reference does; on the GPU it is a hint only).  Twiddles are generated
 * on the device in FP64 and rounded once to `dtype`.
 */
int pcx_plan_create(pcx_plan* plan, size_t n, int dtype, int order, size_t sub_size);
int pcx_plan_destroy(pcx_plan plan);
/* fft_unit::size() (fft.hpp:615-617). */
size_t pcx_plan_size(pcx_plan plan);
/*
 * PCX_ERR_TIMEOUT if a kernel of this plan gave up a bounded wait for its
 * input copy since the last call (its rows are then not written), else
 * PCX_OK.  Synchronises with the device.
 */
int pcx_plan_status(pcx_plan plan);

/*
 * Self-test of the bounded device waits (no reference counterpart).  One
 * GPU thread waits on an mbarrier phase that never completes (for at most
 * mbar_limit_ns) and on a device counter that never reaches its target (the
 * four-step kernel's cross-block wait, about one second), with the same
 * bounded waits the kernels use.  *mbar_satisfied / *counter_satisfied
 * receive 1 if a wait saw its condition, 0 if it gave up; both must be 0,
 * and the context stays usable.  Synchronises with the device.
 */
int pcx_selftest_waits(unsigned long long mbar_limit_ns, int* mbar_satisfied, int* counter_satisfied);
/*
 * Self-test of the give-up path of one plan (no reference counterpart).
 * Enqueues on `stream` one GPU thread that waits, for at most limit_ns
 * (<= 2 s), on an mbarrier phase that never completes and, when the wait
 * gives up, sets the plan's error flag exactly as a transform kernel does
 * when its input copy never lands.  The next pcx_plan_status after the
 * stream has drained returns PCX_ERR_TIMEOUT (and clears the flag), which
 * the C++ fft_unit turns into an exception.  No fault, no hang.
 */
int pcx_selftest_plan_wait(pcx_plan plan, unsigned long long limit_ns, void* stream);
/* Bytes of scratch an exec of this plan uses for `batch` rows (0 for n <= 4096). */
size_t pcx_plan_workspace_size(pcx_plan plan, size_t batch);

/* Forms of a transform larger than 4096 points (pcx_plan_tune). */
#define PCX_FORM_DEFAULT 0  /* built-in choice */
#define PCX_FORM_ONEPASS 1  /* one shared-memory pass (FP32 n = 8192) */
#define PCX_FORM_FUSED 2    /* four-step, the whole batch in one persistent launch */
#define PCX_FORM_CHUNKED 3  /* four-step, two launches per L2-sized scratch chunk */

/*
 * Autotuner (no reference counterpart: the reference picks its radix
 * schedule at compile time, fft.hpp:546-575, 1856-1958).  Times the forms
 * this plan supports on `batch` rows of scratch data (forward, natural order,
 * default pack; at most 512 MB per buffer) on `stream`: the one-pass form
 * (FP32 n = 8192), every built-in variant of the one-launch four-step for this
 * size (split N1 x N2, i.e. the radix schedule of both passes; tile shape as
 * blocks per SM; ring stages) at three dependency distances, and the chunked
 * four-step at two scratch sizes; it makes the fastest the plan's form for
 * later execs that use the plan's own scratch (pcx_fft_exec).  Allocates and
 * frees its buffers; synchronises.  *form_out (if not NULL) receives the
 * PCX_FORM_* chosen; pcx_plan_tuning gives the details.  With PCX_TUNE_CACHE
 * set, a cached result for this GPU, size, type and batch is applied without
 * timing (see the tuning cache below).  PCX_TUNE_VERBOSE=1 prints each
 * candidate's time to stderr.  A plan for n <= 4096 has one form:
 * PCX_FORM_DEFAULT, nothing is timed.
 */
int pcx_plan_tune(pcx_plan plan, size_t batch, void* stream, int* form_out);
/* The plan's current form (PCX_FORM_*), the one-launch four-step's dependency
 * distance in rounds of tiles, and the chunked form's scratch bytes per buffer. */
int pcx_plan_form(pcx_plan plan, int* form, int* rounds, size_t* chunk_bytes);

/*
 * What pcx_plan_tune chose (no reference counterpart; the reference's knobs
 * SubSize / NodeSizeRec / Strategy, fft.hpp:546-575, and its cost model
 * get_subtform_idx_strategic_, fft.hpp:1856-1958, fix its schedule at compile
 * time).  For the one-launch four-step: the split N = 2^log_n1 * 2^log_n2
 * (the radix schedule of the two sub-transforms follows from it), the tile
 * shape as resident blocks per SM (64 KB / blocks_per_sm per tile), the ring
 * stages and the dependency distance in rounds of tiles.
 */
typedef struct {
    int    form;          /* PCX_FORM_* */
    int    rounds;        /* one-launch four-step: tile distance in rounds of tiles */
    size_t chunk_bytes;   /* chunked four-step: scratch bytes per buffer */
    int    log_n1;        /* one-launch four-step: split */
    int    log_n2;
    int    blocks_per_sm; /* one-launch four-step: resident blocks per SM (tile shape) */
    int    stages;        /* one-launch four-step: ring stages */
    double ms;            /* device time of one timed transform batch when tuned (0: not timed) */
} pcx_tune_result;
int pcx_plan_tuning(pcx_plan plan, pcx_tune_result* out);
/* Make `r` the plan's form without timing (a result from pcx_plan_tuning or
 * the cache); PCX_ERR_UNSUPPORTED if it names a variant not built for the
 * plan's size.  r->ms is ignored. */
int pcx_plan_set_tuning(pcx_plan plan, const pcx_tune_result* r);

/*
 * Tuning cache (no reference counterpart): results of pcx_plan_tune keyed by
 * GPU name, size, element type and batch (rounded down to a power of two),
 * kept in memory and saved to / merged from a JSON file.  When the
 * environment variable PCX_TUNE_CACHE names a file, pcx_plan_tune loads it
 * once, uses a matching entry instead of timing, and saves new results to it.
 * Host code only: none of these calls touches the GPU.
 */
int    pcx_tune_cache_load(const char* path);
int    pcx_tune_cache_save(const char* path);
int    pcx_tune_cache_put(const char* gpu, size_t n, int dtype, size_t batch, const pcx_tune_result* r);
/* PCX_ERR_INVALID when there is no entry. */
int    pcx_tune_cache_get(const char* gpu, size_t n, int dtype, size_t batch, pcx_tune_result* r);
int    pcx_tune_cache_clear(void);
size_t pcx_tune_cache_size(void);

/*
 * Batched transform of `batch` rows.  Replaces
 *   fft_unit::fft_raw<PD,PS>(dest, src[, src_size])     fft.hpp:624-681
 *   fft_unit::ifft_raw<Norm,PD,PS>(dest, src)           fft.hpp:689-721
 *   fft_unit::operator()(vec) / operator()(dest, src)   fft.hpp:728-820
 *   fft_unit::ifft<Norm>(vec) / ifft<Norm>(dest, src)   fft.hpp:828-915
 * dst == src is the in-place form.  src_len (<= n) source elements per row
 * are read and the rest taken as zero (fft.hpp:671-681); src_len = 0 means n.
 * Forward output / inverse input follow the plan's order.  normalize scales
 * the inverse by 1/n.  The out-of-place inverse computes the mathematically
 * correct inverse for every order (the reference's differs, fft.hpp:863-915).
 * stream: a cudaStream_t (NULL = legacy default stream).
 * Pack widths: any power of two up to n for n <= 4096; up to 16 above, where
 * widths beyond the two-pass kernels' own (8 for float, 4 for double) are
 * changed in an extra pass over the rows (a wider source needs src_len = n).
 * Uses the plan's own scratch for n > 4096: concurrent execs of one plan on
 * different streams must use pcx_fft_exec_ws with separate workspaces.
 */
int pcx_fft_exec(pcx_plan plan, void* dst, const void* src, size_t src_len, int pack_dst, int pack_src,
                 int direction, int normalize, size_t batch, size_t dst_stride, size_t src_stride,
                 void* stream);

/*
 * Transform across vectors.  Replaces fft_unit_par::operator()(dest, source)
 *   (fft.hpp:2167-2572; its own test is disabled in the reference,
 *   tests/test_fft.cpp:719-754)
 * dst and src are host arrays of `count` (= plan size) device pointers, each
 * to a vector of `len` elements at pack pack_dst / pack_src.  For every
 * element position p < len, the plan's transform of src[0][p] .. src[count-1][p]
 * is written to dst[0][p] .. dst[count-1][p] (forward, or inverse scaled by
 * 1/count when normalize).  The plan keeps a gather buffer of len rows.
 */
int pcx_fft_par_exec(pcx_plan plan, void* const* dst, const void* const* src, size_t count, size_t len,
                     int pack_dst, int pack_src, int direction, int normalize, void* stream);

/*
 * Element-wise expression over packed vectors on the device.  Replaces the
 * evaluation of pcxo::vector expression templates (vector_arithm.hpp:405-1140:
 * operator+ - * / between vectors and with complex scalars, conj, and
 * vector::operator=(expression), vector.hpp:177-182) for data the GPU holds.
 * `ops` is a postfix program of n_ops nodes: PCX_OP_VEC pushes element e of
 * vecs[arg] (pack vec_packs[arg]), PCX_OP_SCALAR pushes re + i*im, the binary
 * nodes pop two values and push the result, PCX_OP_CONJ conjugates the top.
 * The program must leave one value (nesting depth <= 8); element e of dst
 * (pack pack_dst) receives it, for e < n.  dst may be one of the operands when
 * their pack widths agree.
 */
#define PCX_EXPR_MAX_OPS 32
#define PCX_EXPR_MAX_VECS 8
#define PCX_OP_VEC 0
#define PCX_OP_SCALAR 1
#define PCX_OP_ADD 2
#define PCX_OP_SUB 3
#define PCX_OP_MUL 4
#define PCX_OP_DIV 5
#define PCX_OP_CONJ 6
typedef struct {
    int    code;
    int    arg;
    double re;
    double im;
} pcx_expr_op;
int pcx_vec_eval(int dtype, void* dst, int pack_dst, size_t n, const pcx_expr_op* ops, int n_ops,
                 const void* const* vecs, const int* vec_packs, int n_vecs, void* stream);

/* As pcx_fft_exec with caller-provided scratch (>= pcx_plan_workspace_size). */
int pcx_fft_exec_ws(pcx_plan plan, void* dst, const void* src, size_t src_len, int pack_dst, int pack_src,
                    int direction, int normalize, size_t batch, size_t dst_stride, size_t src_stride,
                    void* workspace, size_t workspace_bytes, void* stream);

/*
 * Size of the device scratch array that pcx_fft_exec_noalloc uses (8 MiB,
 * held by every GPU that loads the library until the process exits).
 */
#define PCX_NOALLOC_SCRATCH_BYTES (8u << 20)

/*
 * No counterpart in the reference (which has no GPU and no scratch).
 * As pcx_fft_exec, but allocates nothing, for callers that cannot allocate
 * device memory while running (a fixed memory budget set at start-up, device
 * memory handed out only by the caller's own pool, rules that forbid device
 * allocation after initialisation).  The four-step path (n > 4096) uses a
 * file-scope device array of PCX_NOALLOC_SCRATCH_BYTES instead of allocated
 * scratch, processing the batch in chunks that fit it; sizes whose single
 * transform does not fit (n * element bytes > 8 MiB: only fp64 at n = 2^20)
 * are rejected with
 * PCX_ERR_UNSUPPORTED.  The first call on each device is its set-up: it
 * looks up the array's device address (cudaGetSymbolAddress), which also
 * makes the CUDA runtime load the module that holds the array (under lazy
 * module loading, the default, the 8 MiB are committed then, by the
 * loader); make that call during initialisation, before any stream capture.
 * All calls share the array: calls whose GPU work overlaps race.
 * The plan itself must already exist (pcx_plan_create allocates).
 */
int pcx_fft_exec_noalloc(pcx_plan plan, void* dst, const void* src, size_t src_len, int pack_dst, int pack_src,
                         int direction, int normalize, size_t batch, size_t dst_stride, size_t src_stride,
                         void* stream);

/*
 * Adjoint (vector-Jacobian product) of pcx_fft_exec with the same arguments:
 * given the cotangent g_out of the transform's output, writes the cotangent
 * of its input.  The forward DFT's adjoint is the unnormalised inverse read
 * in the plan's order; the inverse's adjoint is the forward scaled as the
 * inverse was.  No reference counterpart (the reference has no derivatives).
 */
int pcx_fft_vjp(pcx_plan plan, void* g_in, const void* g_out, int pack, int direction, int normalize,
                size_t batch, size_t stride, void* stream);

/*
 * Overlap-save cross-correlation.  Replaces fxcorr_unit<T>(g, fft_size)
 * (reference fxcorr.hpp:62-92): g is a DEVICE pointer to k elements at pack
 * width pack_g; kernel spectrum K = FFT(g zero-padded to n_fft) / n_fft is
 * computed on the device.  Requires k <= n_fft - pack + 1 so that step > 0.
 */
int pcx_fxcorr_create(pcx_fxcorr* h, const void* g, size_t k, int pack_g, size_t n_fft, int dtype);
int pcx_fxcorr_destroy(pcx_fxcorr h);

/*
 * y[n] = sum_{j<k} x[n+j] * conj(g[j]) (x zero past its end) for `channels`
 * rows of `len` elements at pack width `pack`.  Replaces
 * fxcorr_unit::operator()(vec) (fxcorr.hpp:102-136, block loop with the
 * block offset taken as a packed element index) and the empty out-of-place
 * operator()(dest, src) (fxcorr.hpp:138-140).  dst == src is in place.
 */
int pcx_fxcorr_exec(pcx_fxcorr h, void* dst, const void* src, size_t len, int pack, size_t channels,
                    size_t dst_stride, size_t src_stride, void* stream);

/*
 * PCX_ERR_TIMEOUT if a correlation or adjoint of this handle since the last
 * call had a block give up a bounded device wait (for its input copy, or, in
 * place, for its predecessor's read; the affected outputs are not written),
 * else PCX_OK.  Synchronises the device.
 */
int pcx_fxcorr_status(pcx_fxcorr h);

/*
 * Adjoint of pcx_fxcorr_exec: given gy (cotangent of y), writes gx
 * (cotangent of x: convolution of gy with g) and, if gg != NULL, accumulates
 * the cotangent of g over all channels into gg (k elements at pack width
 * pack_g, overwritten): correlation of gy with x.  x is the forward input.
 * Cotangents of complex values follow d/dRe + i d/dIm.
 */
int pcx_fxcorr_vjp(pcx_fxcorr h, void* gx, void* gg, const void* gy, const void* x, size_t len, int pack,
                   size_t channels, size_t stride, void* stream);

/*
 * Tensor-core form of the batched FFT (no reference counterpart): radix-16
 * stages as dense 32x32 real DFT-matrix products on the tensor cores
 * (tcgen05.mma, FP32 accumulation in tensor memory) with split operands,
 * precision 0: bfloat16 hi + lo, three products (kind::f16);
 * precision 1: tf32 hi + lo, three products (kind::tf32);
 * precision 2: bfloat16 hi + mid + lo, the six products up to second order
 *              (kind::f16), FP32-level accuracy from bfloat16 operands.
 * `batch` contiguous rows of a complex64 plan in natural order, pack 8,
 * 2^8 <= n <= 2^16.  Up to 2^12 one launch transforms whole rows; 2^13..2^16
 * run as two passes of 2^6..2^8-point tensor-core transforms (columns, with
 * the four-step twiddle, into the plan's scratch, then rows out in natural
 * order), one L2-sized chunk of rows at a time; like pcx_fft_exec with the
 * plan's scratch, such calls on one plan must not overlap on the GPU.
 * Errors against an FP64 oracle are reported per size by the test suite and
 * the benchmark.
 */
int pcx_tc_fft_exec(pcx_plan plan, void* dst, const void* src, int direction, int normalize, size_t batch,
                    int precision, void* stream);

/*
 * Ragged persistent batch.  No counterpart in the reference (which runs one
 * transform per call): n_fft complex64 FFTs of power-of-two sizes 2^5..2^18
 * (one transform each, device pointers, pack 8, natural order; all forward,
 * or all inverse of one size when normalised) and n_xc out-of-place
 * correlations (signal xc_len[j] samples, kernel of xc_k[j] taps at xc_g[j],
 * FFT size xc_nfft[j] in 2^7..2^14), executed by ONE persistent launch that
 * takes work items from a device queue (four-step transforms as column and
 * row tiles with device-side dependencies), captured once as a CUDA graph.
 * Pointers are fixed at creation; each exec replays the graph.  Every buffer
 * (transforms and correlation signals, pack 8) must be 16-byte aligned: the
 * data arrive by bulk copies (PCX_ERR_INVALID otherwise).
 */
typedef struct pcx_ragged_s* pcx_ragged;
int pcx_ragged_create(pcx_ragged* h, int dtype, size_t n_fft, const size_t* sizes, void* const* dst,
                      const void* const* src, int direction, int normalize, size_t n_xc, const size_t* xc_len,
                      const size_t* xc_k, const void* const* xc_g, const size_t* xc_nfft, void* const* xc_dst,
                      const void* const* xc_src);
/*
 * As pcx_ragged_create, with the transforms of 2^8..2^12 points run by the
 * tensor-core form (a second persistent launch in the same graph, items of
 * 4096 points; the precision as pcx_tc_fft_exec: 0 bf16 x3, 1 tf32 x3,
 * 2 bf16 x6); tensor_core = -1 is pcx_ragged_create.
 */
int pcx_ragged_create_tc(pcx_ragged* h, int dtype, size_t n_fft, const size_t* sizes, void* const* dst,
                         const void* const* src, int direction, int normalize, size_t n_xc, const size_t* xc_len,
                         const size_t* xc_k, const void* const* xc_g, const size_t* xc_nfft, void* const* xc_dst,
                         const void* const* xc_src, int tensor_core);
int pcx_ragged_exec(pcx_ragged h, void* stream);
/* PCX_ERR_TIMEOUT if a work item gave up waiting for a dependency (synchronises). */
int pcx_ragged_status(pcx_ragged h);
/* Work items in the queue. */
size_t pcx_ragged_items(pcx_ragged h);
int    pcx_ragged_destroy(pcx_ragged h);

#ifdef __cplusplus
}
#endif

#endif /* PCX_CUDA_H */

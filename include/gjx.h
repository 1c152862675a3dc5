/*
 * gjx.h -- C ABI of gpujachx_b200, the B200 (sm_100a) implementation of the
 * hierarchically blocked one-sided Jacobi SVD / hyperbolic SVD of GPUJACHx.
 *
 * The first two entry points are drop-in replacements of the reference's
 * own, with the same names, arguments, return codes and side effects.  The
 * rest is additive.  Plain pointers and sizes only; no C++ or torch types.
 * Library: gpujachx_b200/lib/libgjx.so.
 */
#ifndef GJX_H
#define GJX_H

#ifdef __cplusplus
extern "C" {
#endif

/* ALG / routine bits (reference share/HypJacL.hpp:88-110). */
#define GJX_CDSORT_1 1u   /* innermost (32x32 block) sorting of the eigenvalues */
#define GJX_FULL_SVD 2u   /* also accumulate V */
#define GJX_ACCUMV_2 4u   /* unused by hypJacL2, as in the reference */
#define GJX_BLK_ORI 8u    /* block-oriented: one inner sweep per block pair */

/* Positive return codes (errors that are not argument errors). */
#define GJX_ERR_CUDA 1        /* a CUDA runtime call failed: gjx_last_error() */
#define GJX_ERR_NO_STRAT 2    /* init_strats has not loaded strategy tables */
#define GJX_ERR_STRAT_ORDER 3 /* ncol / 16 differs from the loaded outer table order */
#define GJX_ERR_DEVICE 4      /* a kernel reported a bounded wait that timed out */
#define GJX_ERR_ALIGN 5       /* device pointer or leading dimension misaligned */
#define GJX_ERR_SCRATCH 6     /* the tables do not fit the static scratch (gjx_hypJacL2_noalloc) */

/*
 * Replaces hypJacL2 of 1/HypJacL2.hpp:6-27 (definition 1/HypJacL2.cu:13-202).
 * Host memory in and out, all device memory allocated and freed per call.
 *   routine  ALG, < 16 (bits above)
 *   nrow     rows of G, > 0, multiple of 64
 *   ncol     columns of G, 0 < ncol <= nrow, multiple of 32 (= 16 * n1)
 *   nplus    number of +1 signs in J = diag(I_nplus, -I_{ncol-nplus})
 *   hG       INOUT ldhG x ncol, column major: G in, U (unit columns) out
 *   hV       OUT ldhV x ncol (only the first ncol rows written); routine & 2
 *   hD       OUT ncol: D = +-||g_j||^2, the eigenvalues of G^T J G
 *   glbSwp   OUT outer sweeps; glb_s / glb_b OUT rotations / "big" rotations
 *   timing   OUT optional double[4]: wall, setup + H2D, compute, D2H + cleanup (s)
 * Returns 0; -1..-12 for the reference's argument errors (same checks, same
 * order); > 0 for the errors above.  Prints one line per outer sweep to
 * stdout like the reference, unless gjx_set_verbose(0).
 */
int hypJacL2(const unsigned routine, const unsigned nrow, const unsigned ncol, const unsigned nplus,
             double *const hG, const unsigned ldhG, double *const hV, const unsigned ldhV, double *const hD,
             unsigned *const glbSwp, unsigned long long *const glb_s, unsigned long long *const glb_b,
             double *const timing);

/*
 * Replaces init_strats of share/HypJacL.hpp:206 (definition
 * share/HypJacL.cu:11-121): loads the inner (snp0, n0 = 32 columns) and outer
 * (snp1, n1 = ncol / 16 blocks) strategy tables "<name>%05u" from the shared
 * library sdy (strat.so), bytes for n <= 256, uint16 above.  Names: mmstep,
 * BrentL, colcyc, cycloc, rowcyc, cycwor.  On failure it prints "[ERROR] ..."
 * and exits the process, as the reference does; gjx_init_strats reports the
 * same failures as a return code instead.
 */
void init_strats(const char *const sdy, const char *const snp0, const unsigned n0, const char *const snp1,
                 const unsigned n1);

/* As init_strats, returning 0 or a negative code instead of exiting:
 * -1 empty sdy, -2 empty snp0, -3 n0 not positive even, -4 empty snp1,
 * -5 n1 not positive even, -6 unknown snp0, -7 unknown snp1, -8 dlopen
 * failed, -9 no table for snp0 & n0, -10 no table for snp1 & n1,
 * -11 n0 != 32 (the inner level is 32 columns), -12 n1 > 1024. */
int gjx_init_strats(const char *const sdy, const char *const snp0, const unsigned n0, const char *const snp1,
                    const unsigned n1);

/* Loaded strategy state: ids (share/HypJacL.hpp:118-158), steps, pairs. */
int gjx_strat_info(unsigned *strat0, unsigned *steps0, unsigned *pairs0, unsigned *strat1, unsigned *steps1,
                   unsigned *pairs1);
/* Copy of the loaded outer table, [steps1][pairs1][2] uint16; returns the
 * number of entries copied (<= cap), or < 0. */
int gjx_get_strat1(unsigned short *out, unsigned cap);

/*
 * Batched form (no counterpart in the reference): nmat independent
 * decompositions of device-resident matrices, each given exactly as
 * gjx_hypJacL2_dev would give it alone (same bits, sweeps and counts), run
 * together -- one launch per outer step index for the whole batch, a sweep's
 * launches replayed from a CUDA graph, converged matrices skipped.  Per
 * matrix b: nrow[b], ncol[b], nplus[b], dG[b] (lddG[b]), dV[b] (lddV[b];
 * ALG & 2), dD[b]; outputs sweeps[b], glb_s[b], glb_b[b] and info[b] (0, or
 * the argument code of gjx_hypJacL2_dev: that matrix is left untouched).
 * The outer table of each matrix is the loaded family's (init_strats) for
 * n1 = ncol[b] / 16, read from the same strategy library.  Returns 0, -1
 * (bad batch arguments), GJX_ERR_NO_STRAT, GJX_ERR_CUDA or GJX_ERR_DEVICE.
 */
int gjx_hypJacL2_batched(unsigned routine, unsigned nmat, const unsigned *nrow, const unsigned *ncol,
                         const unsigned *nplus, double *const *dG, const unsigned *lddG, double *const *dV,
                         const unsigned *lddV, double *const *dD, void *stream, unsigned *sweeps,
                         unsigned long long *glb_s, unsigned long long *glb_b, int *info);

/* How a sweep is launched: -1 (default) the tuned choice (gjx_autotune), else
 * per step; 0 one launch per outer step, as the reference; 1 one cooperative
 * launch per sweep, in which the block pairs of
 * consecutive outer steps start as soon as their two blocks are written
 * (used when all clusters of a step fit on the GPU at once, else per step;
 * measured no faster on a B200, kept for the autotuner).  The results are
 * the same bits either way. */
void gjx_set_sweep_mode(int mode);

/* CTAs per block pair (a thread-block cluster): 1, 2 or 4, or 0 (default)
 * for the automatic choice.  The results are the same bits for any value. */
void gjx_set_split(unsigned n);

/* Block pairs that a CTA takes at a time: 2 (the Cholesky factorisations
 * and inner sweeps of the two run concurrently on two groups of 4 warps), 1,
 * 3 (batched form only: one block pair per CTA of 4 warps, two such CTAs per
 * SM, so that one CTA's serial phases overlap the other's Gram and update),
 * 4 (batched form only: two block pairs per CTA of 4 warps, two such CTAs
 * per SM; the two pairs' serial phases run concurrently on 2 warps each), or
 * 0 (default): automatic -- the batched autotuner's
 * choice, else 2 in the batched form (gjx_hypJacL2_batched), and in the
 * per-step launches of a single matrix with one CTA per block pair when a
 * step has more block pairs than the GPU has SMs (one wave of CTAs instead of
 * two); else 1.  The results are the same bits for every value. */
void gjx_set_pairs_per_cta(unsigned w);

/* The pivot-block factor of the reference's alternative builds, for
 * hypJacL2, gjx_hypJacL2_dev and gjx_hypJacL2_noalloc: 0 (default) the Gram
 * matrix and its Cholesky factor (share/device_code_common_Cholesky.hpp);
 * 1 as the -DUSE_QR build: Householder QR of the pair's 32-row chunks merged
 * by Givens rotations (share/device_code_common_QR.hpp:4-94,
 * share/device_code_common_Kepler.hpp:326-371); 2 as the -DUSE_DRMAC build:
 * the QR factor and Drmac's scaled-norm sweep in the definite sorting case
 * (share/device_code_cdsort_Drmac.hpp:4-316).  Each gives the bits of that
 * build.  Values above 2 select 0.  The batched form refuses 1 and 2. */
void gjx_set_variant(unsigned v);

/*
 * Autotuner: time every launch configuration of this shape -- 1, 2 or 4
 * CTAs per block pair (where the pairs fit), one launch per outer step or
 * per sweep -- on a seeded random nrow x ncol matrix in scratch device
 * memory, `sweeps` outer sweeps each (0: 1), and use the fastest in later
 * calls with the same (routine, nrow, ncol, nplus) unless gjx_set_split /
 * gjx_set_sweep_mode fix them.  out[2] = {CTAs per pair, sweep mode}.  The
 * loaded strategy tables must match ncol.  0 or an error code.
 */
int gjx_autotune(unsigned routine, unsigned nrow, unsigned ncol, unsigned nplus, unsigned sweeps, unsigned *out);
void gjx_autotune_clear(void);

/* The batched form's launches: -1 (default) the tuned choice
 * (gjx_autotune_batched), else one launch per outer step index; 0 one launch
 * per outer step index for the whole batch (every active matrix advances one
 * step), replayed from a CUDA graph; 1 one launch per sweep of the whole
 * batch, in which a CTA takes (matrix, step, pair) items in step order and
 * starts one as soon as its two blocks have been written by its matrix's
 * previous step.  The results are the same bits either way. */
void gjx_set_batch_mode(int mode);

/* Autotuner of the batched form: times block pairs per CTA (4, 3, 2, 1) x launch
 * mode (per step, per sweep) on seeded random matrices of the batch's shapes
 * (nrow[b] x ncol[b], the signature kind of nplus[b]), `sweeps` sweeps each
 * (0: 1; the faster of two runs after a warm-up run), and uses the fastest in
 * later gjx_hypJacL2_batched calls on a batch of the same shapes (in any
 * order) unless gjx_set_pairs_per_cta / gjx_set_batch_mode fix them.  A
 * configuration later in that order must be 3 % faster to be taken: the first
 * sweeps rank the forms closer together than whole batches do.  out[2] =
 * {pairs per CTA, mode}.  0 or an error code. */
int gjx_autotune_batched(unsigned routine, unsigned nmat, const unsigned *nrow, const unsigned *ncol,
                         const unsigned *nplus, unsigned sweeps, unsigned *out);

/* Failure-path self test of the bounded waits every kernel here uses (an
 * mbarrier or flag that never completes makes the kernel give up after a
 * cycle limit and report, instead of hanging): ctas CTAs each wait on an
 * mbarrier that nobody arrives at, limit_cycles at most.  *timed_out = CTAs
 * that gave up (all of them), *max_cycles = the longest wait.  The context
 * stays usable.  0 or an error code. */
int gjx_wait_selftest(long long limit_cycles, unsigned ctas, int *timed_out, long long *max_cycles);

/* Make dev the calling thread's current device; returns its compute
 * capability as 10 * major + minor (100 for a B200), or -1.  Stands in for
 * configureGPU (share/cuda_helper.cu:5-54) minus its process-wide device
 * flags: nothing here uses mapped host memory. */
int gjx_configure_device(int dev);

/*
 * HDF5 (own reader/writer, see gpujachx_b200/csrc/h5mini.h; no libhdf5).
 * gjx_h5_read: dataset at path ("group/name") into out as doubles
 * (as_float) or ints; dims[<= 8] and *rank receive its shape; out may be
 * NULL (shape only); cap = capacity of out in elements.  0 or < 0.
 * gjx_h5_write: nds datasets into group (one level below the root); mode 0
 * new file, 1 existing file + new group, 2 existing file, group created if
 * absent and same-shaped datasets overwritten in place.  dims: 8 entries per
 * dataset (first ranks[i] used, C order); is_float: double, else int32.
 * The text of an error is in gjx_last_error().
 */
int gjx_h5_read(const char *file, const char *path, int as_float, void *out, unsigned long long cap,
                unsigned long long *dims, int *rank);
int gjx_h5_write(const char *file, const char *group, int mode, int nds, const char *const *names, const int *ranks,
                 const unsigned long long *dims, const int *is_float, const void *const *data);

/*
 * Validate a pivot-pair table tbl[steps][n/2][2] (uint16): every entry
 * below n, p != q, each step a perfect matching of 0..n-1 (no index twice),
 * and over the table every unordered pair {p, q} at least once.  Returns 0
 * (valid), 1 (entry out of range or p == q), 2 (an index twice in a step;
 * *bad_step says which), 3 (pairs missing: *missing), -1 (bad arguments).
 * *repeats counts pairs seen more than once (mmstep tables repeat n/2).
 * No counterpart in the reference, which trusts its tables.
 */
int gjx_validate_pairs(const unsigned short *tbl, unsigned steps, unsigned n, unsigned long long *missing,
                       unsigned long long *repeats, unsigned *bad_step);
/* Both loaded tables: out[6] = {code0, missing0, repeats0, code1, missing1,
 * repeats1}; returns the first nonzero code, or -GJX_ERR_NO_STRAT. */
int gjx_validate_strats(unsigned long long *out);

/*
 * hypJacL2 on device-resident data (no host copies, no per-call allocation
 * of the matrices): dG (lddG >= nrow), dV (lddV >= ncol, routine & 2), dD
 * device pointers, 16-byte aligned, lddG and lddV even.  V is set to I here.
 * stream is a cudaStream_t (NULL = legacy default stream).  Blocks until the
 * result is ready.  Same return codes as hypJacL2.
 */
int gjx_hypJacL2_dev(const unsigned routine, const unsigned nrow, const unsigned ncol, const unsigned nplus,
                     double *const dG, const unsigned lddG, double *const dV, const unsigned lddV,
                     double *const dD, void *const stream, unsigned *const glbSwp,
                     unsigned long long *const glb_s, unsigned long long *const glb_b);

/*
 * gjx_hypJacL2_dev without any device allocation (no counterpart in the
 * reference).  For callers that cannot call cudaMalloc: a process whose device
 * memory belongs to a caching allocator or pool, a service that reserves its
 * memory at start-up, a hot path where cudaMalloc/cudaFree (which synchronise
 * the device) are not allowed.  The library's device working memory -- the
 * strategy tables and two 64-bit words -- lives in a static 520 KiB device
 * array held by every GPU that loads the library until the process exits;
 * the loaded outer table must fit it (n1 <= 512 blocks, ncol <= 8192), else
 * GJX_ERR_SCRATCH.  The first call on a device takes the array's address
 * (cudaGetSymbolAddress) with that device current; make it while no stream of
 * the device is being captured.  No call can run inside a stream capture: after
 * every sweep it reads the rotation counters back and synchronises its stream.
 * All calls share the array: each clears its counters and rewrites
 * the tables when they or the device changed (or the device's context was
 * re-created); calls that overlap on the GPU race.  The call holds the
 * library's host lock until its result is ready, so other calls into the
 * library from the same process wait for it.  Same arguments, results and
 * other codes as gjx_hypJacL2_dev.
 */
int gjx_hypJacL2_noalloc(const unsigned routine, const unsigned nrow, const unsigned ncol, const unsigned nplus,
                         double *const dG, const unsigned lddG, double *const dV, const unsigned lddV,
                         double *const dD, void *const stream, unsigned *const glbSwp,
                         unsigned long long *const glb_s, unsigned long long *const glb_b);

/*
 * Split-precision form (no counterpart in the reference, which has only the
 * FP64 form): gjx_hypJacL2_dev's arguments and outputs, the same one-sided
 * Jacobi with blocks of 32 columns and pairs of 64 (the loaded families'
 * tables for n1 = ncol / 32 outer and 64 inner columns), the Gram matrix of
 * each block pair and the update of G and V run as exact products of 8-bit
 * slices on the tensor cores (tcgen05 kind::i8, int32 accumulators),
 * recombined in FP64: 7 digits of 8 bits per entry (55 bits), scaled per
 * column by its largest entry, the slice products of weight above 2^-56 kept.  The
 * Cholesky factors, rotations, convergence test and D stay FP64.  The
 * results are not the plain form's bits; their accuracy is that of FP64
 * arithmetic (tests report it against LAPACK and the plain form).  ncol a
 * multiple of 64, nrow <= 16384; other codes as gjx_hypJacL2_dev.
 */
int gjx_hypJacL2_split(const unsigned routine, const unsigned nrow, const unsigned ncol, const unsigned nplus,
                       double *const dG, const unsigned lddG, double *const dV, const unsigned lddV,
                       double *const dD, void *const stream, unsigned *const glbSwp,
                       unsigned long long *const glb_s, unsigned long long *const glb_b);

/* Profiling of the split form: clock64 cycles from the start of block pair
 * 0's CTA in the last pair-kernel launch of the last gjx_hypJacL2_split call
 * to the end of [0] the Gram products, [1] the Gram epilogue, [2] the
 * Cholesky factor, [3] the inner sweeps, [4] the update's B operands; and
 * CTA 0 of the update kernel, summed over that call (clock64 in one thread of
 * each warp group): [5] the cutters waiting for the tensor core or the
 * epilogue (digit planes or TMEM to be freed) and issuing the products, [6]
 * cutting tiles into digits, [7] the cutters waiting for copies (tiles, B
 * operands), [8] the epilogues, [9] the tiles it took.  0 or GJX_ERR_CUDA. */
int gjx_split_phase_cycles(long long *out10);

/* Frees the device buffers that hypJacL2 keeps between calls on the current
 * device (they are reused by the next call of the same or smaller size). */
int gjx_release_cache(void);

/* 0: silent; 1 (default): per-sweep lines on stdout like the reference. */
void gjx_set_verbose(const int level);

/* Profiling.  gjx_profile(1) resets the counters and times every block-pair
 * kernel launch with CUDA events on its stream; gjx_profile(0) resets and
 * stops timing (launch counts are always kept).  gjx_profile_read returns the
 * kernel launches since the reset (all kernels of this library), the
 * block-pair launches among them, and their summed device time in ms. */
void gjx_profile(const int enable);
void gjx_profile_read(unsigned long long *launches, unsigned long long *l1_launches, double *l1_ms);

/* Message of the last GJX_ERR_CUDA / GJX_ERR_DEVICE in this thread. */
const char *gjx_last_error(void);

/* Library version string. */
const char *gjx_version(void);

/* Device check of the correctly rounded 1/sqrt: out[i] = rsqrt_rn(in[i]) for
 * device arrays; returns 0 or GJX_ERR_CUDA. */
int gjx_rsqrt_rn_dev(const double *in, double *out, const unsigned n);

#ifdef __cplusplus
}
#endif

#endif /* GJX_H */

// gjx_internal.h -- declarations shared by the host driver and the kernels.
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>
#include <cuda.h>
#include <cuda_runtime.h>

namespace gjx {

constexpr unsigned kNColB = 16u;  // columns per block (share/HypJacL.hpp:112-116)
constexpr unsigned kNSweep = 30u; // outer and full-block inner sweep cap (share/HypJacL.hpp:7-9)

// Everything one launch of the block-pair step needs.  One CTA per block pair
// (i, j) of outer step `step`; the pairs of a step are disjoint.
struct alignas(64) StepParams {
  CUtensorMap tmG;              // 3-D view (32 rows, nrow/32 pieces, ncol columns) of G
  CUtensorMap tmV;              // the same of V (ACCV only)
  CUtensorMap tmGram;           // 3-D view (64 rows, nrow/64 tiles, ncol columns) of G
  double *G;                    // nrow x ncol, column major, leading dim ldG
  double *V;                    // ncol x ncol, leading dim ldV (ACCV only)
  const uint16_t *strat1;       // [steps1][pairs][2] block pairs (outer level)
  const uint8_t *strat0;        // [32][16][2] column pairs (inner level)
  unsigned long long *cvg;      // (big << 32) | small rotation counters
  int *err;                     // device error word (bounded waits)
  unsigned ldG, ldV, nrow, ncol, nplus;
  unsigned pairs;               // block pairs per outer step (n1 / 2)
  unsigned step;                // outer step index
  unsigned s0steps;             // inner steps (31, or 32 for mmstep)
  unsigned nswp0;               // inner sweeps per block pair (1 or 30)
  int gdefinite;                // +1 J = I, -1 J = -I, 0 mixed signs
  unsigned split;               // CTAs per block pair (a cluster): 1, 2 or 4
  unsigned width;               // with split 1: block pairs per CTA, 1 or 2 (l1_step2_kernel)
  unsigned steps1;              // outer steps per sweep (persistent sweep kernel)
  unsigned *ver;                // per block: CTAs that have finished writing it this sweep
  unsigned variant;             // pivot-block factor: 0 Gram + Cholesky, 1 QR, 2 QR + Drmac's sweep
};

// one matrix of a batch: its step parameters (step unused) and D
struct alignas(64) BatchMat {
  StepParams p;
  double *D;
  unsigned steps1; // outer steps per sweep of this matrix
};

// one launch of a batch: every active matrix advances by one outer step of
// its own sweep (matrix b is at step kstep[b] mod steps1 of its sweep)
struct BatchStep {
  const BatchMat *mats;
  const uint32_t *items;   // (matrix << 16) | pair of every matrix, largest matrices first
  unsigned nitems;
  const unsigned *kstep;   // per matrix: outer steps done so far
  unsigned *queue;         // work-queue head (cleared by the step end)
  const uint32_t *done;    // converged or failed matrices (skipped)
  const int *err;          // any nonzero: stop
};

// after each launch: per matrix, count the step; at the end of its sweep fold
// the sweep's counter into its totals and test convergence
struct BatchSweep {
  const BatchMat *mats;
  unsigned *kstep;
  unsigned long long *cvg; // per matrix, (big << 32) | small of the current sweep
  uint32_t *done;
  unsigned *sweeps;
  unsigned long long *glb_s, *glb_b;
  unsigned *queue;
  unsigned *active; // matrices still sweeping (accumulated; cleared by the host between checks)
  unsigned nmat;
};

// one launch per sweep of a batch (the dataflow form): the items of every
// matrix's steps, step-major; an item waits for its blocks' previous step
struct BatchFlow {
  const BatchMat *mats;
  const uint32_t *items;  // (matrix << 16) | pair
  const uint16_t *isteps; // the item's step within the sweep
  unsigned nitems;
  unsigned *queue;        // work-queue head (cleared by the sweep end)
  const uint32_t *done;   // converged or failed matrices (skipped)
  unsigned *ver;          // per matrix at vofs[b]: per block, the writes of this sweep
  const unsigned *vofs;
  int *err;
};

cudaError_t batch_configure();
cudaError_t flow_configure();
cudaError_t launch_batch_flow(bool sort, bool accv, unsigned width, const BatchFlow &b, unsigned ctas,
                              cudaStream_t s);
cudaError_t launch_batch_flow_end(const BatchSweep &w, unsigned *ver, const unsigned *vofs, cudaStream_t s);
cudaError_t launch_fill_random(double *a, size_t n, unsigned long long seed, cudaStream_t s);
cudaError_t launch_wait_selftest(long long limit, int *timed_out, long long *cycles, unsigned ctas, cudaStream_t s);
// one launch for a whole sweep (all outer steps), when every cluster of the
// step fits on the GPU at once; false when it does not (launch per step)
bool sweep_kernel_fits(bool sort, bool accv, const StepParams &p);
cudaError_t launch_l1_sweep(bool sort, bool accv, const StepParams &p, cudaStream_t s);
// width 1: one block pair per CTA at a time; 2: two (pair_step2);
// kWidthHalf: one per CTA of 4 warps, two CTAs per SM; kWidthHalf2: two per
// CTA of 4 warps, two CTAs per SM
constexpr unsigned kWidthHalf = 3u, kWidthHalf2 = 4u;
cudaError_t launch_batch_step(bool sort, bool accv, unsigned width, const BatchStep &b, unsigned ctas,
                              cudaStream_t s);
cudaError_t launch_batch_sweep_end(const BatchSweep &w, cudaStream_t s);
cudaError_t launch_batch_initV(const BatchMat *m, unsigned nmat, cudaStream_t s);
cudaError_t launch_batch_initD(const BatchMat *m, unsigned nmat, const uint32_t *ok, cudaStream_t s);

// TMA tensor maps for the update staging (3-D view, box {34, 8, 16}); 0 or a CUDA error
cudaError_t make_update_map(CUtensorMap *tm, const double *base, unsigned nrow, unsigned ncol, unsigned ld);
// TMA tensor map for the Gram staging (3-D view, box {66, 1, 16})
cudaError_t make_gram_map(CUtensorMap *tm, const double *base, unsigned nrow, unsigned ncol, unsigned ld);

// device error codes written to *err
enum : int { kErrWaitTimeout = 1 };

size_t l1_smem_bytes();
size_t batch2_smem_bytes();
cudaError_t l1_configure();
cudaError_t launch_l1_step(bool sort, bool accv, const StepParams &p, cudaStream_t s);
// CTAs per block pair for `pairs` pairs per step on the current device
unsigned l1_split(unsigned pairs);
cudaError_t launch_initD(double *G, double *D, unsigned nrow, unsigned ncol, unsigned nplus, unsigned ldG,
                         cudaStream_t s);
cudaError_t launch_initV(double *V, unsigned ncol, unsigned ldV, cudaStream_t s);

// host driver pieces used by the allocation-free entry point (gjx_noalloc.cu)
size_t noalloc_scratch_need();
int noalloc_sweeps(unsigned routine, unsigned nrow, unsigned ncol, unsigned nplus, double *dG, unsigned lddG,
                   double *dV, unsigned lddV, double *dD, void *stream, void *scratch, size_t scratch_bytes, int dev,
                   unsigned long long ctx, unsigned *glbSwp, unsigned long long *glb_s, unsigned long long *glb_b);
int check_dev_args(unsigned routine, unsigned nrow, unsigned ncol, unsigned nplus, const double *dG, unsigned lddG,
                   const double *dV, unsigned lddV, const double *dD, const unsigned *glbSwp,
                   const unsigned long long *glb_s, const unsigned long long *glb_b);
void set_error(const char *msg);
// the profiling counters of gjx_profile: whether launches are timed, and
// launches / timed launches / their milliseconds to add
bool profiling();
void profile_add(unsigned long long launches, unsigned long long timed, double ms);
// the loaded strategy families' tables for n0 inner and n1 outer columns (the
// split form: 64 and ncol / 32), as bytes and uint16; 0 or an error code
int family_tables(unsigned n0, unsigned n1, std::vector<uint8_t> &s0, unsigned &steps0, std::vector<uint16_t> &s1,
                  unsigned &steps1, unsigned long long &version);

// exposed for the parity tests of the primitives
cudaError_t launch_rsqrt_test(const double *in, double *out, unsigned n, cudaStream_t s);

} // namespace gjx

// gjx_host.cpp -- host side of gpujachx_b200: the strategy registry and
// loader, the outer sweep driver, and the C ABI of include/gjx.h.
//
// The sweep driver follows 1/HypJacL2.cu:13-202: argument checks with the
// same codes in the same order, V = I, then outer sweeps of one launch per
// outer step until a sweep makes no "big" rotation (or 30 sweeps), then the
// column normalisation that yields U and D.  Differences by design:
//   * no host synchronisation between the steps of a sweep: the launches
//     are queued back to back on one stream and the host reads the
//     convergence counter (device memory, not mapped host memory) once per
//     sweep;
//   * errors are returned (positive codes) instead of exit();
//   * device buffers of hypJacL2 are cached between calls
//     (gjx_release_cache frees them).
#include "gjx.h"
#include "gjx_internal.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <dlfcn.h>
#include <map>
#include <mutex>
#include <tuple>
#include <string>
#include <vector>

namespace {

using clk = std::chrono::steady_clock;

// ----------------------------------------------------------------------------
// strategy registry (share/HypJacL.hpp:118-158, share/HypJacL.cu:11-121)
// ----------------------------------------------------------------------------
struct Strat {
  bool loaded = false;
  unsigned id0 = 0u, steps0 = 0u, pairs0 = 0u;
  unsigned id1 = 0u, steps1 = 0u, pairs1 = 0u;
  unsigned n0 = 0u, n1 = 0u;
  std::vector<uint8_t> s0;  // [32][16][2], steps0 rows used
  std::vector<uint16_t> s1; // [steps1][pairs1][2]
  unsigned long long version = 0ull;
  std::string sdy, snp0, snp1; // where other tables of the families come from (batched and split forms)
};

std::mutex g_mtx;
Strat g_strat;
int g_verbose = 1;
int g_sweep_mode = -1; // -1 automatic (the tuned choice, else per step), 0 per outer step, 1 one launch per sweep
unsigned g_split = 0u;  // CTAs per block pair: 0 automatic (the tuned choice, else by the SM count), else 1, 2, 4
unsigned g_pairs_per_cta = 0u; // block pairs a CTA takes at a time: 0 automatic, 1, 2, or (batched form, two
                               // CTAs of 4 warps per SM) 3: one per CTA, 4: two per CTA
unsigned g_variant = 0u; // pivot-block factor: 0 Gram + Cholesky, 1 QR (-DUSE_QR), 2 QR + Drmac (-DUSE_DRMAC)
int g_batch_mode = -1;   // batched form: -1 the tuned choice (else per step), 0 one launch per step, 1 per sweep
unsigned g_batch_cap = 0u; // nonzero: the batched form stops after this many sweeps (the autotuner's runs)
// the batched autotuner's choices, by the batch's sorted (nrow, ncol, signature) list
std::map<std::vector<unsigned>, std::pair<unsigned, int>> g_batch_tuned; // (pairs per CTA, mode)

// the autotuner's choices, by (routine, nrow, ncol, nplus)
struct TuneKey {
  unsigned routine, nrow, ncol, nplus;
  bool operator<(const TuneKey &o) const
  {
    return std::tie(routine, nrow, ncol, nplus) < std::tie(o.routine, o.nrow, o.ncol, o.nplus);
  }
};
std::map<TuneKey, std::pair<unsigned, int>> g_tuned; // (split, sweep mode)
unsigned g_sweep_cap = 0u; // nonzero: stop after this many sweeps (the autotuner's timed runs)

// profiling: launch counts always; with g_prof, CUDA events around every
// block-pair launch, read back at the end of each sweep
struct Prof {
  bool on = false;
  unsigned long long launches = 0ull, l1_launches = 0ull;
  double l1_ms = 0.0;
  std::vector<cudaEvent_t> ev;
} g_prof;
thread_local std::string g_err;

unsigned strat_id(const char *const name, const unsigned n, unsigned &steps)
{
  struct {
    const char *name;
    unsigned id;
    bool quasi; // n steps instead of n - 1
  } static const tab[] = {{"mmstep", 1u, true},  {"BrentL", 2u, false}, {"colcyc", 3u, false},
                          {"cycloc", 4u, false}, {"rowcyc", 5u, false}, {"cycwor", 6u, false}};
  for (const auto &t : tab)
    if (!std::strcmp(name, t.name)) {
      steps = t.quasi ? n : (n - 1u);
      return t.id;
    }
  return 0u;
}

// the symbol "<name>%05u" (share/my_utils.cu:50-61)
const void *strat_ptr(void *const h, const char *const snp, const unsigned n)
{
  char arrn[12] = {'\0'};
  (void)std::snprintf(arrn, sizeof(arrn), "%s%05u", snp, n);
  if (arrn[11])
    return nullptr;
  return dlsym(h, arrn);
}

// ----------------------------------------------------------------------------
// per-device context: strategy tables and counters resident on the device
// ----------------------------------------------------------------------------
struct DevCtx {
  bool ready = false;
  uint8_t *d_s0 = nullptr;
  uint16_t *d_s1 = nullptr;
  size_t s1_cap = 0u;
  unsigned long long version = ~0ull;
  unsigned long long *d_cnt = nullptr; // [0] = cvg, [1] = err (int in the low word)
  unsigned long long *h_cnt = nullptr; // pinned mirror
  unsigned *d_ver = nullptr;           // per-block write counts of the one-launch sweep (1024 blocks)
  // outer tables of the batched form, by n1, for strategy version btab_version
  bool batch_ready = false;
  cudaStream_t batch_stream = nullptr; // graphs cannot be captured on the legacy default stream
  cudaEvent_t batch_ev = nullptr;
  std::vector<std::pair<uint16_t *, unsigned>> btab; // index n1: (device table, steps)
  unsigned long long btab_version = ~0ull;
  // cached matrices of hypJacL2
  double *dG = nullptr, *dV = nullptr, *dD = nullptr;
  size_t capG = 0u, capV = 0u, capD = 0u;
};
std::vector<DevCtx> g_dev;

int set_cuda_error(const cudaError_t e, const char *const what)
{
  g_err = std::string(what) + ": " + cudaGetErrorString(e);
  return GJX_ERR_CUDA;
}

#define GJX_CUDA(call, what)                                                                                         \
  do {                                                                                                               \
    const cudaError_t e_ = (call);                                                                                   \
    if (e_ != cudaSuccess)                                                                                           \
      return set_cuda_error(e_, what);                                                                               \
  } while (0)

int dev_ctx(DevCtx *&ctx)
{
  int dev = 0;
  GJX_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
  if ((size_t)dev >= g_dev.size())
    g_dev.resize((size_t)dev + 1u);
  ctx = &g_dev[(size_t)dev];
  if (!ctx->ready) {
    GJX_CUDA(gjx::l1_configure(), "l1_configure");
    GJX_CUDA(cudaMalloc(&ctx->d_s0, 32u * 16u * 2u), "cudaMalloc(strat0)");
    GJX_CUDA(cudaMalloc(&ctx->d_cnt, 2u * sizeof(unsigned long long)), "cudaMalloc(counters)");
    GJX_CUDA(cudaMalloc(&ctx->d_ver, 1024u * sizeof(unsigned)), "cudaMalloc(block counts)");
    GJX_CUDA(cudaHostAlloc(&ctx->h_cnt, 2u * sizeof(unsigned long long), cudaHostAllocPortable),
             "cudaHostAlloc(counters)");
    ctx->ready = true;
  }
  return 0;
}

int upload_strat(DevCtx &ctx, const cudaStream_t st)
{
  if (ctx.version == g_strat.version)
    return 0;
  const size_t need = g_strat.s1.size() * sizeof(uint16_t);
  if (need > ctx.s1_cap) {
    if (ctx.d_s1)
      GJX_CUDA(cudaFree(ctx.d_s1), "cudaFree(strat1)");
    ctx.d_s1 = nullptr;
    GJX_CUDA(cudaMalloc(&ctx.d_s1, need), "cudaMalloc(strat1)");
    ctx.s1_cap = need;
  }
  GJX_CUDA(cudaMemcpyAsync(ctx.d_s1, g_strat.s1.data(), need, cudaMemcpyHostToDevice, st), "upload strat1");
  GJX_CUDA(cudaMemcpyAsync(ctx.d_s0, g_strat.s0.data(), g_strat.s0.size(), cudaMemcpyHostToDevice, st),
           "upload strat0");
  GJX_CUDA(cudaStreamSynchronize(st), "upload strategies");
  ctx.version = g_strat.version;
  return 0;
}

double secs(const clk::time_point a, const clk::time_point b)
{
  return std::chrono::duration<double>(b - a).count();
}

// The outer sweeps on device data, the sweep loop of 1/HypJacL2.cu:167-216.
// The caller holds g_mtx, has checked the arguments and the tables, has
// configured the kernels on this device and provides the device-side
// working memory: the strategy tables d_s0 / d_s1 (uploaded) and two
// 64-bit words d_cnt (counter, error word), plus a host mirror h_cnt of
// those two words.  Nothing is allocated here (profiling events aside,
// with prof).
int run_sweeps_core(const unsigned routine, const unsigned nrow, const unsigned ncol, const unsigned nplus,
                    double *const dG, const unsigned lddG, double *const dV, const unsigned lddV, double *const dD,
                    const cudaStream_t st, const uint8_t *const d_s0, const uint16_t *const d_s1,
                    unsigned long long *const d_cnt, unsigned long long *const h_cnt, unsigned *const d_ver,
                    const bool prof,
                    unsigned *const glbSwp, unsigned long long *const glb_s, unsigned long long *const glb_b)
{
  const bool cdsort = (routine & GJX_CDSORT_1) != 0u, full = (routine & GJX_FULL_SVD) != 0u,
             blk_ori = (routine & GJX_BLK_ORI) != 0u;
  if (full) {
    GJX_CUDA(gjx::launch_initV(dV, ncol, lddV, st), "initV");
    ++g_prof.launches;
  }
  if (prof && g_prof.ev.size() < 2u * g_strat.steps1) {
    const size_t have = g_prof.ev.size();
    g_prof.ev.resize(2u * g_strat.steps1);
    for (size_t i = have; i < g_prof.ev.size(); ++i)
      GJX_CUDA(cudaEventCreate(&g_prof.ev[i]), "cudaEventCreate");
  }

  gjx::StepParams p{};
  p.G = dG;
  p.V = full ? dV : nullptr;
  p.strat1 = d_s1;
  p.strat0 = d_s0;
  p.cvg = d_cnt;
  p.err = reinterpret_cast<int *>(d_cnt + 1);
  p.ldG = lddG;
  p.ldV = full ? lddV : 0u;
  p.nrow = nrow;
  p.ncol = ncol;
  p.nplus = nplus;
  p.pairs = g_strat.pairs1;
  p.s0steps = g_strat.steps0;
  p.nswp0 = blk_ori ? 1u : gjx::kNSweep;
  p.gdefinite = (nplus ? ((nplus < ncol) ? 0 : +1) : -1);
  p.split = gjx::l1_split(p.pairs);
  int mode = g_sweep_mode;
  const auto tuned = g_tuned.find(TuneKey{routine, nrow, ncol, nplus});
  if (tuned != g_tuned.end()) {
    if (!g_split)
      p.split = tuned->second.first;
    if (mode < 0)
      mode = tuned->second.second;
  }
  if (g_split && g_split * p.pairs <= 148u * 8u)
    p.split = g_split;
  // two block pairs per CTA: with 1 CTA per pair, when a step has more pairs
  // than the GPU has SMs (one wave instead of two), or when asked for
  int dev = 0, sms = 148;
  GJX_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
  GJX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
  p.width = (p.split == 1u && (g_pairs_per_cta == 2u || (!g_pairs_per_cta && p.pairs > (unsigned)sms))) ? 2u : 1u;
  p.variant = g_variant;
  if (p.variant) { // the QR factors: one CTA per block pair, one launch per outer step
    p.split = 1u;
    p.width = 1u;
    mode = 0;
  }
  GJX_CUDA(gjx::make_update_map(&p.tmG, dG, nrow, ncol, lddG), "tensor map of G");
  GJX_CUDA(gjx::make_gram_map(&p.tmGram, dG, nrow, ncol, lddG), "Gram tensor map of G");
  if (full)
    GJX_CUDA(gjx::make_update_map(&p.tmV, dV, ncol, ncol, lddV), "tensor map of V");

  GJX_CUDA(cudaMemsetAsync(d_cnt + 1, 0, sizeof(unsigned long long), st), "clear error word");
  *glb_s = 0ull;
  *glb_b = 0ull;
  unsigned blk_swp = 0u;
  clk::time_point ts = clk::now();
  p.steps1 = g_strat.steps1;
  p.ver = d_ver;
  // one launch per sweep when all clusters of a step are resident together
  bool one_launch = d_ver && mode > 0 && g_strat.n1 <= 1024u && gjx::sweep_kernel_fits(cdsort, full, p);
  const unsigned cap = g_sweep_cap ? g_sweep_cap : gjx::kNSweep;
  while (blk_swp < cap) {
    GJX_CUDA(cudaMemsetAsync(d_cnt, 0, sizeof(unsigned long long), st), "clear counter");
    if (one_launch) {
      GJX_CUDA(cudaMemsetAsync(d_ver, 0, g_strat.n1 * sizeof(unsigned), st), "clear block counts");
      if (prof)
        GJX_CUDA(cudaEventRecord(g_prof.ev[0], st), "cudaEventRecord");
      const cudaError_t le = gjx::launch_l1_sweep(cdsort, full, p, st);
      if (le != cudaSuccess && blk_swp == 0u) { // refused (a cooperative launch that does not fit): per step
        (void)cudaGetLastError();
        one_launch = false;
      }
      else
        GJX_CUDA(le, "block-pair sweep");
      if (prof)
        GJX_CUDA(cudaEventRecord(g_prof.ev[1], st), "cudaEventRecord");
      if (one_launch)
        g_prof.launches += 1u;
    }
    if (!one_launch) {
      for (unsigned stp = 0u; stp < g_strat.steps1; ++stp) {
        p.step = stp;
        if (prof)
          GJX_CUDA(cudaEventRecord(g_prof.ev[2u * stp], st), "cudaEventRecord");
        GJX_CUDA(gjx::launch_l1_step(cdsort, full, p, st), "block-pair step");
        if (prof)
          GJX_CUDA(cudaEventRecord(g_prof.ev[2u * stp + 1u], st), "cudaEventRecord");
      }
      g_prof.launches += g_strat.steps1;
    }
    g_prof.l1_launches += g_strat.steps1;
    ++blk_swp;
    GJX_CUDA(cudaMemcpyAsync(h_cnt, d_cnt, 2u * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st),
             "read counters");
    GJX_CUDA(cudaStreamSynchronize(st), "sweep");
    if (prof)
      for (unsigned stp = 0u; stp < (one_launch ? 1u : g_strat.steps1); ++stp) { // (steps: events 2 stp, 2 stp + 1)
        float ms = 0.0f;
        GJX_CUDA(cudaEventElapsedTime(&ms, g_prof.ev[2u * stp], g_prof.ev[2u * stp + 1u]), "cudaEventElapsedTime");
        g_prof.l1_ms += ms;
      }
    if ((int)h_cnt[1]) {
      g_err = "a block-pair kernel timed out waiting for its tile copies";
      return GJX_ERR_DEVICE;
    }
    const unsigned long long cvg = h_cnt[0];
    const unsigned cvg_s = (unsigned)cvg, cvg_b = (unsigned)(cvg >> 32u);
    *glb_s += cvg_s;
    *glb_b += cvg_b;
    const clk::time_point t2 = clk::now();
    if (g_verbose > 0) {
      (void)std::fprintf(stdout, "BLK_SWP(%2u), ROT_S(%10u), ROT_B(%10u), TIME(%#12.6f s)\n", blk_swp, cvg_s, cvg_b,
                         secs(ts, t2));
      (void)std::fflush(stdout);
    }
    ts = t2;
    if (!cvg_b)
      break;
  }
  *glbSwp = blk_swp;
  GJX_CUDA(gjx::launch_initD(dG, dD, nrow, ncol, nplus, lddG, st), "initD");
  ++g_prof.launches;
  GJX_CUDA(cudaStreamSynchronize(st), "initD");
  return 0;
}

// run_sweeps_core on the per-device context (allocated on first use)
int run_sweeps(const unsigned routine, const unsigned nrow, const unsigned ncol, const unsigned nplus,
               double *const dG, const unsigned lddG, double *const dV, const unsigned lddV, double *const dD,
               const cudaStream_t st, unsigned *const glbSwp, unsigned long long *const glb_s,
               unsigned long long *const glb_b)
{
  if (!g_strat.loaded)
    return GJX_ERR_NO_STRAT;
  if (ncol / gjx::kNColB != g_strat.n1)
    return GJX_ERR_STRAT_ORDER;
  DevCtx *ctx = nullptr;
  if (const int r = dev_ctx(ctx))
    return r;
  if (const int r = upload_strat(*ctx, st))
    return r;
  return run_sweeps_core(routine, nrow, ncol, nplus, dG, lddG, dV, lddV, dD, st, ctx->d_s0, ctx->d_s1, ctx->d_cnt,
                         ctx->h_cnt, ctx->d_ver, g_prof.on, glbSwp, glb_s, glb_b);
}

// argument checks of 1/HypJacL2.cu:39-77, same codes in the same order
int check_args(const unsigned routine, const unsigned nrow, const unsigned ncol, const unsigned nplus,
               const double *const G, const unsigned ldG, const double *const V, const unsigned ldV,
               const double *const D, const unsigned *const glbSwp, const unsigned long long *const glb_s,
               const unsigned long long *const glb_b)
{
  if (routine >= 16u)
    return -1;
  const bool full = (routine & GJX_FULL_SVD) != 0u;
  if (!nrow || (nrow % 64u))
    return -2;
  if (!ncol || (ncol > nrow) || (ncol % 32u))
    return -3;
  if (nplus > ncol)
    return -4;
  if (!G)
    return -5;
  if (ldG < nrow)
    return -6;
  if (full) {
    if (!V)
      return -7;
    if (ldV < ncol)
      return -8;
  }
  if (!D)
    return -9;
  if (!glbSwp)
    return -10;
  if (!glb_s)
    return -11;
  if (!glb_b)
    return -12;
  return 0;
}

// the outer table of the loaded family for n1 blocks, resident on this
// device (loaded from the strategy library on first use)
int batch_table(DevCtx &ctx, const unsigned n1, const uint16_t *&dtab, unsigned &steps)
{
  if (ctx.btab_version != g_strat.version) {
    for (auto &t : ctx.btab)
      if (t.first)
        (void)cudaFree(t.first);
    ctx.btab.clear();
    ctx.btab_version = g_strat.version;
  }
  if (ctx.btab.size() <= n1)
    ctx.btab.resize(n1 + 1u, {nullptr, 0u});
  if (!ctx.btab[n1].first) {
    unsigned st = 0u;
    if (!strat_id(g_strat.snp1.c_str(), n1, st)) {
      g_err = "no " + g_strat.snp1 + " table for n1 = " + std::to_string(n1);
      return GJX_ERR_NO_STRAT;
    }
    void *const h = dlopen(g_strat.sdy.c_str(), RTLD_LAZY);
    if (!h) {
      g_err = "cannot open " + g_strat.sdy;
      return GJX_ERR_NO_STRAT;
    }
    const void *const a = strat_ptr(h, g_strat.snp1.c_str(), n1);
    if (!a) {
      dlclose(h);
      g_err = "no " + g_strat.snp1 + " table for n1 = " + std::to_string(n1) + " in " + g_strat.sdy;
      return GJX_ERR_NO_STRAT;
    }
    const size_t e = (size_t)st * (n1 / 2u) * 2u;
    std::vector<uint16_t> t(e);
    if (n1 <= 256u)
      for (size_t i = 0u; i < e; ++i)
        t[i] = static_cast<const uint8_t *>(a)[i];
    else
      std::memcpy(t.data(), a, e * sizeof(uint16_t));
    dlclose(h);
    uint16_t *d = nullptr;
    GJX_CUDA(cudaMalloc(&d, e * sizeof(uint16_t)), "cudaMalloc(batch table)");
    GJX_CUDA(cudaMemcpy(d, t.data(), e * sizeof(uint16_t), cudaMemcpyHostToDevice), "upload batch table");
    ctx.btab[n1] = {d, st};
  }
  dtab = ctx.btab[n1].first;
  steps = ctx.btab[n1].second;
  return 0;
}

// the autotuner's key of a batch: its matrices' (nrow, ncol, signature
// kind) sorted, so that the same shapes in any order share their choice
std::vector<unsigned> batch_key(const unsigned nmat, const unsigned *const nrow, const unsigned *const ncol,
                                const unsigned *const nplus)
{
  std::vector<unsigned> k;
  k.reserve(3u * nmat);
  std::vector<std::tuple<unsigned, unsigned, unsigned>> v(nmat);
  for (unsigned b = 0u; b < nmat; ++b)
    v[b] = std::make_tuple(nrow[b], ncol[b], nplus[b] ? ((nplus[b] < ncol[b]) ? 1u : 2u) : 0u);
  std::sort(v.begin(), v.end());
  for (const auto &t : v) {
    k.push_back(std::get<0>(t));
    k.push_back(std::get<1>(t));
    k.push_back(std::get<2>(t));
  }
  return k;
}

// The batched form: nmat independent decompositions, each exactly as
// run_sweeps_core would do it alone (same steps, same per-pair code, same
// convergence test), run together: one launch per outer step index for all
// matrices, the launches of a sweep replayed from a CUDA graph.
int run_batch(const unsigned routine, const unsigned nmat, const unsigned *const nrow, const unsigned *const ncol,
              const unsigned *const nplus, double *const *const dG, const unsigned *const lddG,
              double *const *const dV, const unsigned *const lddV, double *const *const dD, cudaStream_t st,
              unsigned *const sweeps, unsigned long long *const glb_s, unsigned long long *const glb_b,
              int *const info)
{
  const bool cdsort = (routine & GJX_CDSORT_1) != 0u, full = (routine & GJX_FULL_SVD) != 0u,
             blk_ori = (routine & GJX_BLK_ORI) != 0u;
  DevCtx *ctx = nullptr;
  if (const int r = dev_ctx(ctx))
    return r;
  if (!ctx->batch_ready) {
    GJX_CUDA(gjx::batch_configure(), "batch_configure");
    GJX_CUDA(gjx::flow_configure(), "flow_configure");
    GJX_CUDA(cudaStreamCreateWithFlags(&ctx->batch_stream, cudaStreamNonBlocking), "batch stream");
    GJX_CUDA(cudaEventCreateWithFlags(&ctx->batch_ev, cudaEventDisableTiming), "batch event");
    ctx->batch_ready = true;
  }
  if (!st) { // the legacy stream: work on our own stream, after what the caller queued
    GJX_CUDA(cudaEventRecord(ctx->batch_ev, nullptr), "batch event");
    GJX_CUDA(cudaStreamWaitEvent(ctx->batch_stream, ctx->batch_ev, 0u), "batch event");
    st = ctx->batch_stream;
  }
  if (const int r = upload_strat(*ctx, st))
    return r;

  std::vector<gjx::BatchMat> mats(nmat);
  std::vector<uint32_t> ok(nmat, 0u);
  unsigned max_steps = 0u;
  for (unsigned b = 0u; b < nmat; ++b) {
    sweeps[b] = 0u;
    glb_s[b] = glb_b[b] = 0ull;
    unsigned dummy_s = 0u;
    unsigned long long dummy_l = 0ull;
    info[b] = gjx::check_dev_args(routine, nrow[b], ncol[b], nplus[b], dG[b], lddG[b], full ? dV[b] : nullptr,
                                  full ? lddV[b] : 0u, dD[b], &dummy_s, &dummy_l, &dummy_l);
    if (info[b])
      continue;
    const unsigned n1 = ncol[b] / gjx::kNColB;
    const uint16_t *tab = nullptr;
    unsigned steps = 0u;
    if (const int r = batch_table(*ctx, n1, tab, steps))
      return r;
    gjx::StepParams &p = mats[b].p;
    p.G = dG[b];
    p.V = full ? dV[b] : nullptr;
    p.strat1 = tab;
    p.strat0 = ctx->d_s0;
    p.ldG = lddG[b];
    p.ldV = full ? lddV[b] : 0u;
    p.nrow = nrow[b];
    p.ncol = ncol[b];
    p.nplus = nplus[b];
    p.pairs = n1 / 2u;
    p.s0steps = g_strat.steps0;
    p.nswp0 = blk_ori ? 1u : gjx::kNSweep;
    p.gdefinite = (nplus[b] ? ((nplus[b] < ncol[b]) ? 0 : +1) : -1);
    p.split = 1u;
    GJX_CUDA(gjx::make_update_map(&p.tmG, dG[b], nrow[b], ncol[b], lddG[b]), "tensor map of G");
    GJX_CUDA(gjx::make_gram_map(&p.tmGram, dG[b], nrow[b], ncol[b], lddG[b]), "Gram tensor map of G");
    if (full)
      GJX_CUDA(gjx::make_update_map(&p.tmV, dV[b], ncol[b], ncol[b], lddV[b]), "tensor map of V");
    mats[b].D = dD[b];
    mats[b].steps1 = steps;
    ok[b] = 1u;
    if (steps > max_steps)
      max_steps = steps;
  }
  // the work of a launch: every block pair of every matrix, the largest
  // matrices first (fewest stragglers at the end of a launch)
  std::vector<unsigned> order;
  for (unsigned b = 0u; b < nmat; ++b)
    if (ok[b])
      order.push_back(b);
  std::stable_sort(order.begin(), order.end(), [&](unsigned x, unsigned y) {
    return (unsigned long long)nrow[x] * ncol[x] > (unsigned long long)nrow[y] * ncol[y];
  });
  if (order.empty())
    return 0;
  std::vector<uint32_t> items;
  for (unsigned b : order)
    for (unsigned q = 0u; q < mats[b].p.pairs; ++q)
      items.push_back((b << 16u) | q);

  // device memory of the batch, one allocation
  auto up = [](size_t x) { return (x + 255u) & ~(size_t)255u; };
  const size_t o_mats = 0u, o_cvg = up(o_mats + nmat * sizeof(gjx::BatchMat)), o_done = up(o_cvg + nmat * 8u),
               o_ok = up(o_done + nmat * 4u), o_swp = up(o_ok + nmat * 4u), o_gs = up(o_swp + nmat * 4u),
               o_gb = up(o_gs + nmat * 8u), o_ks = up(o_gb + nmat * 8u), o_q = up(o_ks + nmat * 4u),
               o_act = up(o_q + 4u), o_err = up(o_act + 4u), o_items = up(o_err + 8u),
               total = up(o_items + items.size() * 4u);
  char *mem = nullptr;
  GJX_CUDA(cudaMalloc(&mem, total), "cudaMalloc(batch)");
  struct Free {
    char *m;
    ~Free() { (void)cudaFree(m); }
  } free_mem{mem};
  auto *d_mats = reinterpret_cast<gjx::BatchMat *>(mem + o_mats);
  auto *d_cvg = reinterpret_cast<unsigned long long *>(mem + o_cvg);
  auto *d_done = reinterpret_cast<uint32_t *>(mem + o_done);
  auto *d_ok = reinterpret_cast<uint32_t *>(mem + o_ok);
  auto *d_swp = reinterpret_cast<unsigned *>(mem + o_swp);
  auto *d_gs = reinterpret_cast<unsigned long long *>(mem + o_gs);
  auto *d_gb = reinterpret_cast<unsigned long long *>(mem + o_gb);
  auto *d_ks = reinterpret_cast<unsigned *>(mem + o_ks);
  auto *d_q = reinterpret_cast<unsigned *>(mem + o_q);
  auto *d_act = reinterpret_cast<unsigned *>(mem + o_act);
  auto *d_err = reinterpret_cast<int *>(mem + o_err);
  auto *d_items = reinterpret_cast<uint32_t *>(mem + o_items);
  for (unsigned b = 0u; b < nmat; ++b) {
    mats[b].p.cvg = d_cvg + b;
    mats[b].p.err = d_err;
  }
  std::vector<uint32_t> done(nmat);
  for (unsigned b = 0u; b < nmat; ++b)
    done[b] = ok[b] ? 0u : 1u;
  GJX_CUDA(cudaMemsetAsync(mem + o_cvg, 0, o_items - o_cvg, st), "clear batch words");
  GJX_CUDA(cudaMemcpyAsync(d_mats, mats.data(), nmat * sizeof(gjx::BatchMat), cudaMemcpyHostToDevice, st),
           "upload batch");
  GJX_CUDA(cudaMemcpyAsync(d_done, done.data(), nmat * 4u, cudaMemcpyHostToDevice, st), "upload batch");
  GJX_CUDA(cudaMemcpyAsync(d_ok, ok.data(), nmat * 4u, cudaMemcpyHostToDevice, st), "upload batch");
  GJX_CUDA(cudaMemcpyAsync(d_items, items.data(), items.size() * 4u, cudaMemcpyHostToDevice, st), "upload batch");
  if (full) {
    GJX_CUDA(gjx::launch_batch_initV(d_mats, nmat, st), "batch initV");
    ++g_prof.launches;
  }

  int dev = 0, sms = 148;
  GJX_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
  GJX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
  unsigned width = (g_pairs_per_cta == 1u || g_pairs_per_cta == gjx::kWidthHalf ||
                    g_pairs_per_cta == gjx::kWidthHalf2) ? g_pairs_per_cta : 2u;
  int mode = g_batch_mode;
  {
    const auto t = g_batch_tuned.find(batch_key(nmat, nrow, ncol, nplus));
    if (t != g_batch_tuned.end()) {
      if (!g_pairs_per_cta)
        width = t->second.first;
      if (mode < 0)
        mode = t->second.second;
    }
  }
  const unsigned cap = g_batch_cap ? g_batch_cap : gjx::kNSweep;
  if (mode == 1) { // one launch per sweep (the dataflow form)
    std::vector<uint32_t> fitems;
    std::vector<uint16_t> fsteps;
    std::vector<unsigned> vofs(nmat, 0u);
    unsigned nver = 0u;
    for (unsigned b = 0u; b < nmat; ++b)
      if (ok[b]) {
        vofs[b] = nver;
        nver += 2u * mats[b].p.pairs;
      }
    for (unsigned st1 = 0u; st1 < max_steps; ++st1)
      for (unsigned b : order)
        if (st1 < mats[b].steps1)
          for (unsigned q = 0u; q < mats[b].p.pairs; ++q) {
            fitems.push_back((b << 16u) | q);
            fsteps.push_back((uint16_t)st1);
          }
    const size_t f_items = 0u, f_steps = up(f_items + fitems.size() * 4u), f_ver = up(f_steps + fsteps.size() * 2u),
                 f_vofs = up(f_ver + (size_t)nver * 4u), ftotal = up(f_vofs + (size_t)nmat * 4u);
    char *fmem = nullptr;
    GJX_CUDA(cudaMalloc(&fmem, ftotal), "cudaMalloc(batch flow)");
    Free free_fmem{fmem};
    auto *d_fitems = reinterpret_cast<uint32_t *>(fmem + f_items);
    auto *d_fsteps = reinterpret_cast<uint16_t *>(fmem + f_steps);
    auto *d_ver = reinterpret_cast<unsigned *>(fmem + f_ver);
    auto *d_vofs = reinterpret_cast<unsigned *>(fmem + f_vofs);
    GJX_CUDA(cudaMemcpyAsync(d_fitems, fitems.data(), fitems.size() * 4u, cudaMemcpyHostToDevice, st), "upload");
    GJX_CUDA(cudaMemcpyAsync(d_fsteps, fsteps.data(), fsteps.size() * 2u, cudaMemcpyHostToDevice, st), "upload");
    GJX_CUDA(cudaMemcpyAsync(d_vofs, vofs.data(), nmat * 4u, cudaMemcpyHostToDevice, st), "upload");
    GJX_CUDA(cudaMemsetAsync(d_ver, 0, (size_t)nver * 4u, st), "clear block counts");
    constexpr unsigned kSweeps = 4u; // sweeps per graph
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    GJX_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "begin capture");
    cudaError_t ce = cudaSuccess;
    const gjx::BatchFlow bf{d_mats, d_fitems, d_fsteps, (unsigned)fitems.size(), d_q, d_done, d_ver, d_vofs, d_err};
    const gjx::BatchSweep sw{d_mats, d_ks, d_cvg, d_done, d_swp, d_gs, d_gb, d_q, d_act, nmat};
    const unsigned ctas = std::min<unsigned>((width >= gjx::kWidthHalf ? 2u : 1u) * (unsigned)sms,
                                            (unsigned)(width == gjx::kWidthHalf2 ? (fitems.size() + 1u) / 2u
                                                                                 : fitems.size()));
    for (unsigned k = 0u; k < kSweeps && ce == cudaSuccess; ++k) {
      ce = gjx::launch_batch_flow(cdsort, full, width, bf, ctas, st);
      if (ce == cudaSuccess)
        ce = cudaMemsetAsync(d_act, 0, 4u, st);
      if (ce == cudaSuccess)
        ce = gjx::launch_batch_flow_end(sw, d_ver, d_vofs, st);
    }
    const cudaError_t ee = cudaStreamEndCapture(st, &graph);
    GJX_CUDA(ce, "capture of batch sweeps");
    GJX_CUDA(ee, "end capture");
    struct Graph {
      cudaGraph_t g;
      cudaGraphExec_t *x;
      ~Graph()
      {
        if (*x)
          (void)cudaGraphExecDestroy(*x);
        if (g)
          (void)cudaGraphDestroy(g);
      }
    } guard{graph, &exec};
    GJX_CUDA(cudaGraphInstantiate(&exec, graph, 0ull), "graph instantiate");
    unsigned active = 0u;
    int err = 0;
    for (unsigned k = 0u; k * kSweeps < cap; ++k) {
      GJX_CUDA(cudaGraphLaunch(exec, st), "graph launch");
      g_prof.launches += 2u * kSweeps;
      g_prof.l1_launches += kSweeps;
      GJX_CUDA(cudaMemcpyAsync(&active, d_act, 4u, cudaMemcpyDeviceToHost, st), "read batch state");
      GJX_CUDA(cudaMemcpyAsync(&err, d_err, 4u, cudaMemcpyDeviceToHost, st), "read batch state");
      GJX_CUDA(cudaStreamSynchronize(st), "batch sweeps");
      if (err) {
        g_err = "a block-pair kernel timed out waiting for its tile copies or blocks";
        return GJX_ERR_DEVICE;
      }
      if (!active)
        break;
    }
    GJX_CUDA(gjx::launch_batch_initD(d_mats, nmat, d_ok, st), "batch initD");
    ++g_prof.launches;
    GJX_CUDA(cudaMemcpyAsync(sweeps, d_swp, nmat * 4u, cudaMemcpyDeviceToHost, st), "read sweeps");
    GJX_CUDA(cudaMemcpyAsync(glb_s, d_gs, nmat * 8u, cudaMemcpyDeviceToHost, st), "read counts");
    GJX_CUDA(cudaMemcpyAsync(glb_b, d_gb, nmat * 8u, cudaMemcpyDeviceToHost, st), "read counts");
    GJX_CUDA(cudaStreamSynchronize(st), "batch end");
    return 0;
  }

  // kLaunches launches (each followed by its step end), captured once
  constexpr unsigned kLaunches = 8u;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  GJX_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "begin capture");
  cudaError_t ce = cudaSuccess;
  const gjx::BatchStep bs{d_mats, d_items, (unsigned)items.size(), d_ks, d_q, d_done, d_err};
  const gjx::BatchSweep sw{d_mats, d_ks, d_cvg, d_done, d_swp, d_gs, d_gb, d_q, d_act, nmat};
  const unsigned ctas = std::min<unsigned>((width >= gjx::kWidthHalf ? 2u : 1u) * (unsigned)sms,
                                          (unsigned)(width == gjx::kWidthHalf2 ? (items.size() + 1u) / 2u
                                                                               : items.size()));
  for (unsigned k = 0u; k < kLaunches && ce == cudaSuccess; ++k) {
    ce = gjx::launch_batch_step(cdsort, full, width, bs, ctas, st);
    if (ce == cudaSuccess)
      ce = cudaMemsetAsync(d_act, 0, 4u, st); // the count of the last launch is the one read
    if (ce == cudaSuccess)
      ce = gjx::launch_batch_sweep_end(sw, st);
  }
  const cudaError_t ee = cudaStreamEndCapture(st, &graph);
  GJX_CUDA(ce, "capture of batch launches");
  GJX_CUDA(ee, "end capture");
  struct Graph {
    cudaGraph_t g;
    cudaGraphExec_t *x;
    ~Graph()
    {
      if (*x)
        (void)cudaGraphExecDestroy(*x);
      if (g)
        (void)cudaGraphDestroy(g);
    }
  } guard{graph, &exec};
  GJX_CUDA(cudaGraphInstantiate(&exec, graph, 0ull), "graph instantiate");

  const unsigned max_replays = (cap * max_steps + kLaunches - 1u) / kLaunches + 1u;
  unsigned active = 0u;
  int err = 0;
  for (unsigned k = 0u; k < max_replays; ++k) {
    GJX_CUDA(cudaGraphLaunch(exec, st), "graph launch");
    g_prof.launches += 2u * kLaunches;
    g_prof.l1_launches += kLaunches;
    GJX_CUDA(cudaMemcpyAsync(&active, d_act, 4u, cudaMemcpyDeviceToHost, st), "read batch state");
    GJX_CUDA(cudaMemcpyAsync(&err, d_err, 4u, cudaMemcpyDeviceToHost, st), "read batch state");
    GJX_CUDA(cudaStreamSynchronize(st), "batch launches");
    if (err) {
      g_err = "a block-pair kernel timed out waiting for its tile copies";
      return GJX_ERR_DEVICE;
    }
    if (!active)
      break;
  }
  GJX_CUDA(gjx::launch_batch_initD(d_mats, nmat, d_ok, st), "batch initD");
  ++g_prof.launches;
  GJX_CUDA(cudaMemcpyAsync(sweeps, d_swp, nmat * 4u, cudaMemcpyDeviceToHost, st), "read sweeps");
  GJX_CUDA(cudaMemcpyAsync(glb_s, d_gs, nmat * 8u, cudaMemcpyDeviceToHost, st), "read counts");
  GJX_CUDA(cudaMemcpyAsync(glb_b, d_gb, nmat * 8u, cudaMemcpyDeviceToHost, st), "read counts");
  GJX_CUDA(cudaStreamSynchronize(st), "batch end");
  return 0;
}

template <typename T> int ensure(T *&p, size_t &cap, const size_t n, const char *const what)
{
  if (n <= cap)
    return 0;
  if (p)
    GJX_CUDA(cudaFree(p), what);
  p = nullptr;
  cap = 0u;
  GJX_CUDA(cudaMalloc(&p, n * sizeof(T)), what);
  cap = n;
  return 0;
}

} // namespace

namespace gjx {

// Layout of caller-provided scratch: [0, 256) the two words, [256, 1280)
// strat0, [1280, ...) strat1.
constexpr size_t kScrCnt = 0u, kScrS0 = 256u, kScrS1 = 1280u;

size_t noalloc_scratch_need()
{
  std::lock_guard<std::mutex> lk(g_mtx);
  return g_strat.loaded ? (kScrS1 + g_strat.s1.size() * sizeof(uint16_t)) : 0u;
}

int noalloc_sweeps(const unsigned routine, const unsigned nrow, const unsigned ncol, const unsigned nplus,
                   double *const dG, const unsigned lddG, double *const dV, const unsigned lddV, double *const dD,
                   void *const stream, void *const scratch, const size_t scratch_bytes, const int dev,
                   const unsigned long long ctx, unsigned *const glbSwp, unsigned long long *const glb_s,
                   unsigned long long *const glb_b)
{
  // what the scratch of a device holds; a new context (id ctx, 0 if unknown)
  // means a new, zeroed array and unconfigured kernels: everything again
  struct Uploaded {
    const void *scratch = nullptr;
    unsigned long long version = ~0ull;
    unsigned long long ctx = 0u;
    bool configured = false;
  };
  static std::vector<Uploaded> up; // per device: what the scratch holds
  std::lock_guard<std::mutex> lk(g_mtx);
  if (!g_strat.loaded)
    return GJX_ERR_NO_STRAT;
  if (ncol / kNColB != g_strat.n1)
    return GJX_ERR_STRAT_ORDER;
  const size_t need = kScrS1 + g_strat.s1.size() * sizeof(uint16_t);
  if (need > scratch_bytes) {
    g_err = "the outer strategy table needs " + std::to_string(need) + " bytes of scratch, the static scratch holds " +
            std::to_string(scratch_bytes);
    return GJX_ERR_SCRATCH;
  }
  if ((size_t)dev >= up.size())
    up.resize((size_t)dev + 1u);
  Uploaded &u = up[(size_t)dev];
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  unsigned char *const base = static_cast<unsigned char *>(scratch);
  if (u.ctx != ctx || !ctx) {
    u.configured = false;
    u.scratch = nullptr;
    u.ctx = ctx;
  }
  if (!u.configured) {
    GJX_CUDA(l1_configure(), "l1_configure");
    u.configured = true;
  }
  if (u.scratch != scratch || u.version != g_strat.version) {
    GJX_CUDA(cudaMemcpyAsync(base + kScrS0, g_strat.s0.data(), g_strat.s0.size(), cudaMemcpyHostToDevice, st),
             "upload strat0");
    GJX_CUDA(cudaMemcpyAsync(base + kScrS1, g_strat.s1.data(), g_strat.s1.size() * sizeof(uint16_t),
                             cudaMemcpyHostToDevice, st),
             "upload strat1");
    GJX_CUDA(cudaStreamSynchronize(st), "upload strategies");
    u.scratch = scratch;
    u.version = g_strat.version;
  }
  unsigned long long h_cnt[2] = {0ull, 0ull}; // pageable host mirror of the two words
  return run_sweeps_core(routine, nrow, ncol, nplus, dG, lddG, dV, lddV, dD, st,
                         reinterpret_cast<const uint8_t *>(base + kScrS0),
                         reinterpret_cast<const uint16_t *>(base + kScrS1),
                         reinterpret_cast<unsigned long long *>(base + kScrCnt), h_cnt, nullptr, false, glbSwp, glb_s,
                         glb_b);
}

int family_tables(const unsigned n0, const unsigned n1, std::vector<uint8_t> &s0, unsigned &steps0,
                  std::vector<uint16_t> &s1, unsigned &steps1, unsigned long long &version)
{
  std::lock_guard<std::mutex> lk(g_mtx);
  if (!g_strat.loaded)
    return GJX_ERR_NO_STRAT;
  if (!strat_id(g_strat.snp0.c_str(), n0, steps0) || !strat_id(g_strat.snp1.c_str(), n1, steps1)) {
    g_err = "unknown strategy family";
    return GJX_ERR_NO_STRAT;
  }
  void *const h = dlopen(g_strat.sdy.c_str(), RTLD_LAZY);
  if (!h) {
    g_err = "cannot open " + g_strat.sdy;
    return GJX_ERR_NO_STRAT;
  }
  const void *const a0 = strat_ptr(h, g_strat.snp0.c_str(), n0);
  const void *const a1 = strat_ptr(h, g_strat.snp1.c_str(), n1);
  if (!a0 || !a1) {
    dlclose(h);
    g_err = "no " + (a0 ? g_strat.snp1 + " table for n = " + std::to_string(n1)
                        : g_strat.snp0 + " table for n = " + std::to_string(n0)) + " in " + g_strat.sdy;
    return GJX_ERR_NO_STRAT;
  }
  const size_t e0 = (size_t)steps0 * n0, e1 = (size_t)steps1 * n1; // steps x (n / 2 pairs) x 2
  s0.resize(e0);
  if (n0 <= 256u)
    std::memcpy(s0.data(), a0, e0);
  else { // the split form's inner tables are 64 columns; larger ones are refused by the caller
    dlclose(h);
    g_err = "inner table too large";
    return GJX_ERR_NO_STRAT;
  }
  s1.resize(e1);
  if (n1 <= 256u)
    for (size_t i = 0u; i < e1; ++i)
      s1[i] = static_cast<const uint8_t *>(a1)[i];
  else
    std::memcpy(s1.data(), a1, e1 * sizeof(uint16_t));
  dlclose(h);
  version = g_strat.version;
  return 0;
}

int check_dev_args(const unsigned routine, const unsigned nrow, const unsigned ncol, const unsigned nplus,
                   const double *const dG, const unsigned lddG, const double *const dV, const unsigned lddV,
                   const double *const dD, const unsigned *const glbSwp, const unsigned long long *const glb_s,
                   const unsigned long long *const glb_b)
{
  if (const int r = check_args(routine, nrow, ncol, nplus, dG, lddG, dV, lddV, dD, glbSwp, glb_s, glb_b))
    return r;
  const bool full = (routine & GJX_FULL_SVD) != 0u;
  if ((reinterpret_cast<uintptr_t>(dG) & 15u) || (lddG & 1u) || (reinterpret_cast<uintptr_t>(dD) & 7u) ||
      (full && ((reinterpret_cast<uintptr_t>(dV) & 15u) || (lddV & 1u))))
    return GJX_ERR_ALIGN;
  return 0;
}

void set_error(const char *msg) { g_err = msg; }

bool profiling()
{
  std::lock_guard<std::mutex> lk(g_mtx);
  return g_prof.on;
}

void profile_add(const unsigned long long launches, const unsigned long long timed, const double ms)
{
  std::lock_guard<std::mutex> lk(g_mtx);
  g_prof.launches += launches;
  g_prof.l1_launches += timed;
  g_prof.l1_ms += ms;
}

} // namespace gjx

extern "C" {

int gjx_init_strats(const char *const sdy, const char *const snp0, const unsigned n0, const char *const snp1,
                    const unsigned n1)
{
  if (!sdy || !*sdy)
    return -1;
  if (!snp0 || !*snp0)
    return -2;
  if (!n0 || (n0 & 1u))
    return -3;
  if (!snp1 || !*snp1)
    return -4;
  if (!n1 || (n1 & 1u))
    return -5;
  unsigned steps0 = 0u, steps1 = 0u;
  const unsigned id0 = strat_id(snp0, n0, steps0);
  if (!id0)
    return -6;
  const unsigned id1 = strat_id(snp1, n1, steps1);
  if (!id1)
    return -7;
  if (n0 != 32u)
    return -11;
  if (n1 > 1024u)
    return -12;
  void *const h = dlopen(sdy, RTLD_LAZY);
  if (!h)
    return -8;
  const uint8_t *const a0 = static_cast<const uint8_t *>(strat_ptr(h, snp0, n0));
  if (!a0) {
    dlclose(h);
    return -9;
  }
  const void *const a1 = strat_ptr(h, snp1, n1);
  if (!a1) {
    dlclose(h);
    return -10;
  }
  Strat s;
  s.id0 = id0;
  s.steps0 = steps0;
  s.pairs0 = n0 / 2u;
  s.id1 = id1;
  s.steps1 = steps1;
  s.pairs1 = n1 / 2u;
  s.n0 = n0;
  s.n1 = n1;
  s.s0.assign(32u * 16u * 2u, 0u);
  std::memcpy(s.s0.data(), a0, (size_t)steps0 * s.pairs0 * 2u);
  const size_t e1 = (size_t)steps1 * s.pairs1 * 2u;
  s.s1.resize(e1);
  if (n1 <= 256u) {
    const uint8_t *const b = static_cast<const uint8_t *>(a1);
    for (size_t i = 0u; i < e1; ++i)
      s.s1[i] = b[i];
  }
  else
    std::memcpy(s.s1.data(), a1, e1 * sizeof(uint16_t));
  dlclose(h);
  s.sdy = sdy;
  s.snp0 = snp0;
  s.snp1 = snp1;
  s.loaded = true;
  std::lock_guard<std::mutex> lk(g_mtx);
  s.version = g_strat.version + 1ull;
  g_strat = std::move(s);
  return 0;
}

void init_strats(const char *const sdy, const char *const snp0, const unsigned n0, const char *const snp1,
                 const unsigned n1)
{
  static const char *const msg[] = {"",
                                    "SDY empty",
                                    "SNP0 empty",
                                    "n0 not positive even",
                                    "SNP1 empty",
                                    "n1 not positive even",
                                    "SNP0 unknown",
                                    "SNP1 unknown",
                                    "cannot open SDY",
                                    "NO SUCH STRATEGY for SNP0 & n0",
                                    "NO SUCH STRATEGY for SNP1 & n1",
                                    "n0 must be 32",
                                    "n1 > 1024"};
  const int r = gjx_init_strats(sdy, snp0, n0, snp1, n1);
  if (r) {
    (void)std::fprintf(stderr, "[ERROR] %s(%d): %s\n", __FILE__, __LINE__, msg[-r]);
    std::exit(EXIT_FAILURE);
  }
}

int gjx_strat_info(unsigned *strat0, unsigned *steps0, unsigned *pairs0, unsigned *strat1, unsigned *steps1,
                   unsigned *pairs1)
{
  std::lock_guard<std::mutex> lk(g_mtx);
  if (!g_strat.loaded)
    return GJX_ERR_NO_STRAT;
  if (strat0)
    *strat0 = g_strat.id0;
  if (steps0)
    *steps0 = g_strat.steps0;
  if (pairs0)
    *pairs0 = g_strat.pairs0;
  if (strat1)
    *strat1 = g_strat.id1;
  if (steps1)
    *steps1 = g_strat.steps1;
  if (pairs1)
    *pairs1 = g_strat.pairs1;
  return 0;
}

int gjx_get_strat1(unsigned short *out, unsigned cap)
{
  std::lock_guard<std::mutex> lk(g_mtx);
  if (!g_strat.loaded)
    return -GJX_ERR_NO_STRAT;
  const size_t n = g_strat.s1.size() < cap ? g_strat.s1.size() : cap;
  if (out)
    std::memcpy(out, g_strat.s1.data(), n * sizeof(unsigned short));
  return (int)n;
}

int gjx_configure_device(const int dev)
{
  if (dev < 0) {
    gjx::set_error("negative device index");
    return -1;
  }
  if (cudaSetDevice(dev) != cudaSuccess) {
    gjx::set_error("cudaSetDevice failed");
    return -1;
  }
  cudaDeviceProp p;
  if (cudaGetDeviceProperties(&p, dev) != cudaSuccess) {
    gjx::set_error("cudaGetDeviceProperties failed");
    return -1;
  }
  return p.major * 10 + p.minor;
}

int gjx_validate_pairs(const unsigned short *const tbl, const unsigned steps, const unsigned n,
                       unsigned long long *const missing, unsigned long long *const repeats,
                       unsigned *const bad_step)
{
  if (missing)
    *missing = 0ull;
  if (repeats)
    *repeats = 0ull;
  if (bad_step)
    *bad_step = 0u;
  if (!tbl || !steps || !n || (n & 1u))
    return -1;
  const unsigned h = n / 2u;
  std::vector<unsigned> seen((size_t)n * n, 0u);
  std::vector<unsigned> mark(n, ~0u);
  for (unsigned st = 0u; st < steps; ++st)
    for (unsigned k = 0u; k < h; ++k) {
      const unsigned p = tbl[((size_t)st * h + k) * 2u], q = tbl[((size_t)st * h + k) * 2u + 1u];
      if (p >= n || q >= n || p == q) {
        if (bad_step)
          *bad_step = st;
        return 1;
      }
      if (mark[p] == st || mark[q] == st) { // an index twice in one step
        if (bad_step)
          *bad_step = st;
        return 2;
      }
      mark[p] = mark[q] = st;
      ++seen[(size_t)(p < q ? p : q) * n + (p < q ? q : p)];
    }
  unsigned long long miss = 0ull, rep = 0ull;
  for (unsigned p = 0u; p < n; ++p)
    for (unsigned q = p + 1u; q < n; ++q) {
      const unsigned c = seen[(size_t)p * n + q];
      if (!c)
        ++miss;
      else
        rep += c - 1u;
    }
  if (missing)
    *missing = miss;
  if (repeats)
    *repeats = rep;
  return miss ? 3 : 0;
}

int gjx_validate_strats(unsigned long long *const out)
{
  std::vector<unsigned short> t0, t1;
  unsigned steps0, n0, steps1, n1;
  {
    std::lock_guard<std::mutex> lk(g_mtx);
    if (!g_strat.loaded)
      return -GJX_ERR_NO_STRAT;
    steps0 = g_strat.steps0;
    n0 = g_strat.n0;
    steps1 = g_strat.steps1;
    n1 = g_strat.n1;
    t0.assign(g_strat.s0.begin(), g_strat.s0.begin() + (size_t)steps0 * n0);
    t1.assign(g_strat.s1.begin(), g_strat.s1.end());
  }
  unsigned long long m0, r0, m1, r1;
  unsigned b0, b1;
  const int e0 = gjx_validate_pairs(t0.data(), steps0, n0, &m0, &r0, &b0);
  const int e1 = gjx_validate_pairs(t1.data(), steps1, n1, &m1, &r1, &b1);
  if (out) {
    out[0] = (unsigned long long)e0;
    out[1] = m0;
    out[2] = r0;
    out[3] = (unsigned long long)e1;
    out[4] = m1;
    out[5] = r1;
  }
  return e0 ? e0 : e1;
}

int gjx_hypJacL2_dev(const unsigned routine, const unsigned nrow, const unsigned ncol, const unsigned nplus,
                     double *const dG, const unsigned lddG, double *const dV, const unsigned lddV,
                     double *const dD, void *const stream, unsigned *const glbSwp,
                     unsigned long long *const glb_s, unsigned long long *const glb_b)
{
  if (const int r = gjx::check_dev_args(routine, nrow, ncol, nplus, dG, lddG, dV, lddV, dD, glbSwp, glb_s, glb_b))
    return r;
  std::lock_guard<std::mutex> lk(g_mtx);
  return run_sweeps(routine, nrow, ncol, nplus, dG, lddG, dV, lddV, dD, static_cast<cudaStream_t>(stream), glbSwp,
                    glb_s, glb_b);
}

int hypJacL2(const unsigned routine, const unsigned nrow, const unsigned ncol, const unsigned nplus,
             double *const hG, const unsigned ldhG, double *const hV, const unsigned ldhV, double *const hD,
             unsigned *const glbSwp, unsigned long long *const glb_s, unsigned long long *const glb_b,
             double *const timing)
{
  const clk::time_point t0 = clk::now();
  if (const int r = check_args(routine, nrow, ncol, nplus, hG, ldhG, hV, ldhV, hD, glbSwp, glb_s, glb_b))
    return r;
  const bool full = (routine & GJX_FULL_SVD) != 0u;
  std::lock_guard<std::mutex> lk(g_mtx);
  if (!g_strat.loaded)
    return GJX_ERR_NO_STRAT;
  if (ncol / gjx::kNColB != g_strat.n1)
    return GJX_ERR_STRAT_ORDER;
  DevCtx *ctx = nullptr;
  if (const int r = dev_ctx(ctx))
    return r;

  const cudaStream_t st = nullptr;
  const size_t lddG = nrow, lddV = ncol;
  if (const int r = ensure(ctx->dG, ctx->capG, lddG * ncol, "cudaMalloc(G)"))
    return r;
  if (full)
    if (const int r = ensure(ctx->dV, ctx->capV, lddV * ncol, "cudaMalloc(V)"))
      return r;
  if (const int r = ensure(ctx->dD, ctx->capD, (size_t)ncol, "cudaMalloc(D)"))
    return r;
  GJX_CUDA(cudaMemcpy2DAsync(ctx->dG, lddG * sizeof(double), hG, (size_t)ldhG * sizeof(double),
                             (size_t)nrow * sizeof(double), ncol, cudaMemcpyHostToDevice, st),
           "copy G to the device");
  GJX_CUDA(cudaStreamSynchronize(st), "copy G to the device");
  const clk::time_point t1 = clk::now();

  const int r = run_sweeps(routine, nrow, ncol, nplus, ctx->dG, (unsigned)lddG, full ? ctx->dV : nullptr,
                           (unsigned)lddV, ctx->dD, st, glbSwp, glb_s, glb_b);
  if (r)
    return r;
  const clk::time_point t2 = clk::now();

  GJX_CUDA(cudaMemcpy2DAsync(hG, (size_t)ldhG * sizeof(double), ctx->dG, lddG * sizeof(double),
                             (size_t)nrow * sizeof(double), ncol, cudaMemcpyDeviceToHost, st),
           "copy U to the host");
  if (full)
    GJX_CUDA(cudaMemcpy2DAsync(hV, (size_t)ldhV * sizeof(double), ctx->dV, lddV * sizeof(double),
                               (size_t)ncol * sizeof(double), ncol, cudaMemcpyDeviceToHost, st),
             "copy V to the host");
  GJX_CUDA(cudaMemcpyAsync(hD, ctx->dD, (size_t)ncol * sizeof(double), cudaMemcpyDeviceToHost, st),
           "copy D to the host");
  GJX_CUDA(cudaStreamSynchronize(st), "copies to the host");
  const clk::time_point t3 = clk::now();
  if (timing) {
    timing[0] = secs(t0, t3);
    timing[1] = secs(t0, t1);
    timing[2] = secs(t1, t2);
    timing[3] = secs(t2, t3);
  }
  return 0;
}

void gjx_set_verbose(const int level) { g_verbose = level; }

void gjx_profile(const int enable)
{
  std::lock_guard<std::mutex> lk(g_mtx);
  g_prof.on = (enable != 0);
  g_prof.launches = g_prof.l1_launches = 0ull;
  g_prof.l1_ms = 0.0;
}

void gjx_profile_read(unsigned long long *launches, unsigned long long *l1_launches, double *l1_ms)
{
  std::lock_guard<std::mutex> lk(g_mtx);
  if (launches)
    *launches = g_prof.launches;
  if (l1_launches)
    *l1_launches = g_prof.l1_launches;
  if (l1_ms)
    *l1_ms = g_prof.l1_ms;
}

const char *gjx_last_error(void) { return g_err.c_str(); }

const char *gjx_version(void) { return "gpujachx_b200 0.1.0 (sm_100a)"; }

int gjx_release_cache(void)
{
  std::lock_guard<std::mutex> lk(g_mtx);
  int dev = 0;
  GJX_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
  if ((size_t)dev < g_dev.size()) {
    DevCtx &c = g_dev[(size_t)dev];
    if (c.dG)
      GJX_CUDA(cudaFree(c.dG), "cudaFree");
    if (c.dV)
      GJX_CUDA(cudaFree(c.dV), "cudaFree");
    if (c.dD)
      GJX_CUDA(cudaFree(c.dD), "cudaFree");
    c.dG = c.dV = c.dD = nullptr;
    c.capG = c.capV = c.capD = 0u;
  }
  return 0;
}

int gjx_rsqrt_rn_dev(const double *in, double *out, const unsigned n)
{
  GJX_CUDA(gjx::launch_rsqrt_test(in, out, n, nullptr), "rsqrt_rn");
  GJX_CUDA(cudaStreamSynchronize(nullptr), "rsqrt_rn");
  return 0;
}

int gjx_hypJacL2_batched(const unsigned routine, const unsigned nmat, const unsigned *const nrow,
                         const unsigned *const ncol, const unsigned *const nplus, double *const *const dG,
                         const unsigned *const lddG, double *const *const dV, const unsigned *const lddV,
                         double *const *const dD, void *const stream, unsigned *const sweeps,
                         unsigned long long *const glb_s, unsigned long long *const glb_b, int *const info)
{
  {
    std::lock_guard<std::mutex> lk(g_mtx);
    if (g_variant) {
      g_err = "the batched form takes the default pivot-block factor (gjx_set_variant(0))";
      return -1;
    }
  }
  if (!nmat || nmat > 65535u || !nrow || !ncol || !nplus || !dG || !lddG || !dD || !sweeps || !glb_s || !glb_b ||
      !info || ((routine & GJX_FULL_SVD) && (!dV || !lddV)) || routine >= 16u) {
    g_err = "gjx_hypJacL2_batched: bad arguments";
    return -1;
  }
  std::lock_guard<std::mutex> lk(g_mtx);
  if (!g_strat.loaded) {
    g_err = "init_strats has not loaded strategy tables";
    return GJX_ERR_NO_STRAT;
  }
  return run_batch(routine, nmat, nrow, ncol, nplus, dG, lddG, dV, lddV, dD, static_cast<cudaStream_t>(stream),
                   sweeps, glb_s, glb_b, info);
}

void gjx_set_sweep_mode(const int mode)
{
  std::lock_guard<std::mutex> lk(g_mtx);
  g_sweep_mode = (mode < 0) ? -1 : (mode ? 1 : 0);
}

void gjx_set_split(const unsigned n)
{
  std::lock_guard<std::mutex> lk(g_mtx);
  g_split = (n == 1u || n == 2u || n == 4u) ? n : 0u;
}

void gjx_set_variant(const unsigned v)
{
  std::lock_guard<std::mutex> lk(g_mtx);
  g_variant = (v <= 2u) ? v : 0u;
}

void gjx_set_pairs_per_cta(const unsigned w)
{
  std::lock_guard<std::mutex> lk(g_mtx);
  g_pairs_per_cta = (w >= 1u && w <= gjx::kWidthHalf2) ? w : 0u;
}

int gjx_autotune_batched(const unsigned routine, const unsigned nmat, const unsigned *const nrow,
                         const unsigned *const ncol, const unsigned *const nplus, const unsigned sweeps,
                         unsigned *const out)
{
  if (!nmat || nmat > 65535u || !nrow || !ncol || !nplus || routine >= 16u)
    return -1;
  for (unsigned b = 0u; b < nmat; ++b)
    if (const int r = check_args(routine, nrow[b], ncol[b], nplus[b], reinterpret_cast<const double *>(16), nrow[b],
                                 reinterpret_cast<const double *>(16), ncol[b], reinterpret_cast<const double *>(16),
                                 reinterpret_cast<const unsigned *>(16),
                                 reinterpret_cast<const unsigned long long *>(16),
                                 reinterpret_cast<const unsigned long long *>(16)))
      return r;
  std::lock_guard<std::mutex> lk(g_mtx);
  if (!g_strat.loaded)
    return GJX_ERR_NO_STRAT;
  if (g_variant) {
    g_err = "the batched form takes the default pivot-block factor (gjx_set_variant(0))";
    return -1;
  }
  const bool full = (routine & GJX_FULL_SVD) != 0u;
  // seeded random matrices of the batch's shapes, one allocation, kept to refill
  std::vector<size_t> oG(nmat), oV(nmat), oD(nmat);
  std::vector<unsigned> ldG(nmat), ldV(nmat);
  size_t nG = 0u, nV = 0u, nD = 0u;
  for (unsigned b = 0u; b < nmat; ++b) {
    ldG[b] = nrow[b] + (nrow[b] & 1u);
    ldV[b] = ncol[b] + (ncol[b] & 1u);
    oG[b] = nG;
    nG += (size_t)ldG[b] * ncol[b];
    oV[b] = nV;
    nV += full ? (size_t)ldV[b] * ncol[b] : 0u;
    oD[b] = nD;
    nD += ncol[b];
  }
  double *mem = nullptr;
  GJX_CUDA(cudaMalloc(&mem, (2u * nG + nV + nD) * sizeof(double)), "cudaMalloc(batch autotune)");
  struct Free {
    double *m;
    ~Free() { (void)cudaFree(m); }
  } fm{mem};
  double *const g0 = mem, *const g = mem + nG, *const v = g + nG, *const d = v + nV;
  GJX_CUDA(gjx::launch_fill_random(g0, nG, 0x5eedba7cull + nmat, nullptr), "autotune input");
  std::vector<double *> pG(nmat), pV(nmat), pD(nmat);
  for (unsigned b = 0u; b < nmat; ++b) {
    pG[b] = g + oG[b];
    pV[b] = full ? v + oV[b] : nullptr;
    pD[b] = d + oD[b];
  }
  std::vector<unsigned> swp(nmat);
  std::vector<unsigned long long> s_(nmat), b_(nmat);
  std::vector<int> info(nmat);
  cudaEvent_t e0, e1;
  GJX_CUDA(cudaEventCreate(&e0), "cudaEventCreate");
  GJX_CUDA(cudaEventCreate(&e1), "cudaEventCreate");
  const int saved_mode = g_batch_mode;
  const unsigned saved_width = g_pairs_per_cta, saved_cap = g_batch_cap;
  g_batch_cap = sweeps ? sweeps : 1u;
  float best = 3.0e38f;
  std::pair<unsigned, int> pick{gjx::kWidthHalf2, 0};
  int rc = 0;
  // The capped sweeps weigh the first sweeps, where nearly every pair rotates; over a whole batch the
  // forms that hold more pairs per CTA gain further (a batch of 4096 of n = 64...512 to convergence:
  // two pairs per CTA of 4 warps 1116 matrices/s, one 986, two per CTA of 8 warps 892, one 703), so
  // the forms are tried in that order, per-step launches first, and a later one must be 3 % faster.
  for (unsigned width : {gjx::kWidthHalf2, gjx::kWidthHalf, 2u, 1u}) {
    for (int mode : {0, 1}) {
      g_pairs_per_cta = width;
      g_batch_mode = mode;
      float ms = 3.0e38f;
      for (int rep = 0; rep < 3 && !rc; ++rep) { // the first run warms up; the faster of the other two counts
        if (cudaMemcpyAsync(g, g0, nG * sizeof(double), cudaMemcpyDeviceToDevice, nullptr) != cudaSuccess ||
            cudaEventRecord(e0, nullptr) != cudaSuccess) {
          rc = GJX_ERR_CUDA;
          break;
        }
        rc = run_batch(routine, nmat, nrow, ncol, nplus, pG.data(), ldG.data(), pV.data(), ldV.data(), pD.data(),
                       nullptr, swp.data(), s_.data(), b_.data(), info.data());
        float t = 0.0f;
        if (!rc && (cudaEventRecord(e1, nullptr) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                    cudaEventElapsedTime(&t, e0, e1) != cudaSuccess))
          rc = GJX_ERR_CUDA;
        if (!rc && rep)
          ms = std::min(ms, t);
      }
      if (rc)
        break;
      if (ms < 0.97f * best || best > 1.0e38f) {
        best = ms;
        pick = {width, mode};
      }
    }
    if (rc)
      break;
  }
  g_batch_mode = saved_mode;
  g_pairs_per_cta = saved_width;
  g_batch_cap = saved_cap;
  (void)cudaEventDestroy(e0);
  (void)cudaEventDestroy(e1);
  if (rc)
    return rc;
  g_batch_tuned[batch_key(nmat, nrow, ncol, nplus)] = pick;
  if (out) {
    out[0] = pick.first;
    out[1] = (unsigned)pick.second;
  }
  return 0;
}

void gjx_set_batch_mode(const int mode)
{
  std::lock_guard<std::mutex> lk(g_mtx);
  g_batch_mode = (mode < 0) ? -1 : (mode ? 1 : 0);
}

int gjx_autotune(const unsigned routine, const unsigned nrow, const unsigned ncol, const unsigned nplus,
                 const unsigned sweeps, unsigned *const out)
{
  if (const int r = check_args(routine, nrow, ncol, nplus, reinterpret_cast<const double *>(16), nrow,
                               reinterpret_cast<const double *>(16), ncol, reinterpret_cast<const double *>(16),
                               reinterpret_cast<const unsigned *>(16), reinterpret_cast<const unsigned long long *>(16),
                               reinterpret_cast<const unsigned long long *>(16)))
    return r;
  std::lock_guard<std::mutex> lk(g_mtx);
  if (!g_strat.loaded)
    return GJX_ERR_NO_STRAT;
  if (ncol / gjx::kNColB != g_strat.n1)
    return GJX_ERR_STRAT_ORDER;
  DevCtx *ctx = nullptr;
  if (const int r = dev_ctx(ctx))
    return r;
  if (const int r = upload_strat(*ctx, nullptr))
    return r;
  const bool full = (routine & GJX_FULL_SVD) != 0u;
  const unsigned ld = nrow + (nrow & 1u);
  double *mem = nullptr;
  const size_t nG = (size_t)ld * ncol, nV = full ? (size_t)ncol * ncol : 0u;
  GJX_CUDA(cudaMalloc(&mem, (2u * nG + nV + ncol) * sizeof(double)), "cudaMalloc(autotune)");
  struct Free {
    double *m;
    ~Free() { (void)cudaFree(m); }
  } fm{mem};
  double *const g0 = mem, *const g = mem + nG, *const v = g + nG, *const d = v + nV;
  GJX_CUDA(gjx::launch_fill_random(g0, nG, 0x5eed0000ull + ncol, nullptr), "autotune input");
  cudaEvent_t e0, e1;
  GJX_CUDA(cudaEventCreate(&e0), "cudaEventCreate");
  GJX_CUDA(cudaEventCreate(&e1), "cudaEventCreate");
  const int saved_mode = g_sweep_mode;
  const unsigned saved_split = g_split, saved_cap = g_sweep_cap, saved_verbose = (unsigned)g_verbose;
  g_verbose = 0;
  g_sweep_cap = sweeps ? sweeps : 1u;
  float best = 3.0e38f;
  std::pair<unsigned, int> pick{gjx::l1_split(g_strat.pairs1), 0};
  int rc = 0;
  for (unsigned split : {1u, 2u, 4u}) {
    if (split * g_strat.pairs1 > 148u * 8u)
      continue;
    for (int mode : {0, 1}) {
      g_split = split;
      g_sweep_mode = mode;
      unsigned swp;
      unsigned long long s_, b_;
      float ms = 0.0f;
      for (int rep = 0; rep < 2 && !rc; ++rep) { // the first run warms up
        if (cudaMemcpyAsync(g, g0, nG * sizeof(double), cudaMemcpyDeviceToDevice, nullptr) != cudaSuccess ||
            cudaEventRecord(e0, nullptr) != cudaSuccess) {
          rc = GJX_ERR_CUDA;
          break;
        }
        rc = run_sweeps_core(routine, nrow, ncol, nplus, g, ld, full ? v : nullptr, ncol, d, nullptr, ctx->d_s0,
                             ctx->d_s1, ctx->d_cnt, ctx->h_cnt, ctx->d_ver, false, &swp, &s_, &b_);
        if (!rc && (cudaEventRecord(e1, nullptr) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                    cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess))
          rc = GJX_ERR_CUDA;
      }
      if (rc)
        break;
      if (ms < best) {
        best = ms;
        pick = {split, mode};
      }
    }
    if (rc)
      break;
  }
  g_sweep_mode = saved_mode;
  g_split = saved_split;
  g_sweep_cap = saved_cap;
  g_verbose = (int)saved_verbose;
  (void)cudaEventDestroy(e0);
  (void)cudaEventDestroy(e1);
  if (rc)
    return rc;
  g_tuned[TuneKey{routine, nrow, ncol, nplus}] = pick;
  if (out) {
    out[0] = pick.first;
    out[1] = (unsigned)pick.second;
  }
  return 0;
}

void gjx_autotune_clear(void)
{
  std::lock_guard<std::mutex> lk(g_mtx);
  g_tuned.clear();
  g_batch_tuned.clear();
}

int gjx_wait_selftest(const long long limit_cycles, const unsigned ctas, int *const timed_out,
                      long long *const max_cycles)
{
  if (!ctas || ctas > 1024u || limit_cycles <= 0 || limit_cycles > (1ll << 32) || !timed_out || !max_cycles) {
    g_err = "gjx_wait_selftest: bad arguments";
    return -1;
  }
  int *d_to = nullptr;
  long long *d_cy = nullptr;
  GJX_CUDA(cudaMalloc(&d_to, sizeof(int)), "cudaMalloc(selftest)");
  struct Free {
    void *a, *b;
    ~Free()
    {
      (void)cudaFree(a);
      (void)cudaFree(b);
    }
  } fr{d_to, nullptr};
  GJX_CUDA(cudaMalloc(&d_cy, ctas * sizeof(long long)), "cudaMalloc(selftest)");
  fr.b = d_cy;
  GJX_CUDA(cudaMemset(d_to, 0, sizeof(int)), "cudaMemset(selftest)");
  GJX_CUDA(gjx::launch_wait_selftest(limit_cycles, d_to, d_cy, ctas, nullptr), "wait selftest");
  GJX_CUDA(cudaDeviceSynchronize(), "wait selftest");
  std::vector<long long> cy(ctas);
  GJX_CUDA(cudaMemcpy(timed_out, d_to, sizeof(int), cudaMemcpyDeviceToHost), "read selftest");
  GJX_CUDA(cudaMemcpy(cy.data(), d_cy, ctas * sizeof(long long), cudaMemcpyDeviceToHost), "read selftest");
  *max_cycles = *std::max_element(cy.begin(), cy.end());
  return 0;
}

} // extern "C"

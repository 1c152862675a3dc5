// gjx_noalloc.cu -- the allocation-free entry point gjx_hypJacL2_noalloc.
//
// Some callers cannot allocate device memory while they run us: a process
// whose device memory is owned by a caching allocator or pool (a framework
// such as PyTorch) that every allocation must go through, a service that
// reserves all of its device memory at start-up and admits no later
// cudaMalloc, or an embedding that forbids allocation calls on its hot path
// because cudaMalloc/cudaFree synchronise the device.  For them this entry
// point runs the same sweeps as gjx_hypJacL2_dev with every byte of device
// working memory (the strategy tables the kernels read and the two 64-bit
// words for the rotation counters and the error flag) placed in the static
// array below.  The caller passes the matrices, as always.
//
// The array is a file-scope __device__ variable: every GPU that loads this
// library holds it (kScratchBytes) until the process exits.  In host code its
// name is only a host-side stand-in, not a device address, so the address is
// taken with cudaGetSymbolAddress, once per device, with that device current,
// on the first call made on it; that first call should come before any stream
// capture.  All calls share the array and it keeps the last call's contents:
// the counters are cleared by each call, the tables are rewritten whenever
// the loaded tables or the device change.  Calls that overlap on the GPU
// (other streams, other host threads on the same device) race on it.
#include <mutex>
#include <vector>

#include "gjx.h"
#include "gjx_internal.h"

namespace {

// 256 B of words + 1 KiB inner table + up to 519 KiB outer table: enough for
// every shipped table up to n1 = 512 blocks (ncol <= 8192).
constexpr size_t kScratchBytes = 520u * 1024u;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_sym_mtx;
std::vector<void *> g_sym; // per device: the device address of g_noalloc_scratch

} // namespace

extern "C" int gjx_hypJacL2_noalloc(const unsigned routine, const unsigned nrow, const unsigned ncol,
                                    const unsigned nplus, double *const dG, const unsigned lddG, double *const dV,
                                    const unsigned lddV, double *const dD, void *const stream, unsigned *const glbSwp,
                                    unsigned long long *const glb_s, unsigned long long *const glb_b)
{
  if (const int r = gjx::check_dev_args(routine, nrow, ncol, nplus, dG, lddG, dV, lddV, dD, glbSwp, glb_s, glb_b))
    return r;
  const size_t need = gjx::noalloc_scratch_need();
  if (!need)
    return GJX_ERR_NO_STRAT;
  if (need > kScratchBytes) { // before any CUDA call
    gjx::set_error("the loaded outer strategy table does not fit the static scratch of gjx_hypJacL2_noalloc "
                   "(520 KiB: n1 <= 512 blocks, ncol <= 8192)");
    return GJX_ERR_SCRATCH;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    gjx::set_error(cudaGetErrorString(e));
    return GJX_ERR_CUDA;
  }
  void *ptr = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_sym_mtx);
    if ((size_t)dev >= g_sym.size())
      g_sym.resize((size_t)dev + 1u, nullptr);
    if (!g_sym[(size_t)dev]) { // set-up, once per device, with that device current
      e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
      if (e != cudaSuccess) {
        gjx::set_error(cudaGetErrorString(e));
        return GJX_ERR_CUDA;
      }
      g_sym[(size_t)dev] = ptr;
    }
    ptr = g_sym[(size_t)dev];
  }
  return gjx::noalloc_sweeps(routine, nrow, ncol, nplus, dG, lddG, dV, lddV, dD, stream, ptr, kScratchBytes, dev,
                             glbSwp, glb_s, glb_b);
}

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
// on the first call made on it, which must not come while a stream of the
// device is being captured.  No call can itself be captured: after every sweep
// it reads the rotation counters back and synchronises its stream.  The set-up is repeated only when the device's CUDA context is not
// the one it was made in (a caller's cudaDeviceReset destroys the context, and
// the array and its address with it): the context's id is kept beside the
// address, and the tables are uploaded again into the new array.  All calls
// share the array and it keeps the last call's contents: the counters are
// cleared by each call, the tables are rewritten whenever the loaded tables,
// the device or its context change.  Calls that overlap on the GPU (other
// streams, other host threads on the same device) race on it; calls from host
// threads are serialised by the library's lock for their whole duration.
#include <mutex>
#include <vector>

#include <cudaTypedefs.h>

#include "gjx.h"
#include "gjx_internal.h"

namespace {

// 256 B of words + 1 KiB inner table + up to 519 KiB outer table: enough for
// every shipped table up to n1 = 512 blocks (ncol <= 8192).
constexpr size_t kScratchBytes = 520u * 1024u;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_sym_mtx;
struct SymAddr {
  void *ptr = nullptr;         // device address of g_noalloc_scratch
  unsigned long long ctx = 0u; // id of the context it belongs to (0: none yet)
};
std::vector<SymAddr> g_sym; // per device

// id of the calling thread's current context (cuCtxGetId, unique for the life
// of the process), 0 if it cannot be had
unsigned long long current_ctx_id()
{
  static PFN_cuCtxGetCurrent_v4000 get_cur = nullptr;
  static PFN_cuCtxGetId_v12000 get_id = nullptr;
  if (!get_cur || !get_id) {
    void *f1 = nullptr, *f2 = nullptr;
    cudaDriverEntryPointQueryResult q1, q2;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) != cudaSuccess ||
        cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) != cudaSuccess ||
        q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess || !f1 || !f2)
      return 0u;
    get_cur = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(f1);
    get_id = reinterpret_cast<PFN_cuCtxGetId_v12000>(f2);
  }
  CUcontext c = nullptr;
  unsigned long long id = 0u;
  if (get_cur(&c) != CUDA_SUCCESS || !c || get_id(c, &id) != CUDA_SUCCESS)
    return 0u;
  return id;
}

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
  // makes the device's primary context current on this thread (no allocation)
  e = cudaSetDevice(dev);
  if (e != cudaSuccess) {
    gjx::set_error(cudaGetErrorString(e));
    return GJX_ERR_CUDA;
  }
  const unsigned long long ctx = current_ctx_id();
  void *ptr = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_sym_mtx);
    if ((size_t)dev >= g_sym.size())
      g_sym.resize((size_t)dev + 1u);
    SymAddr &a = g_sym[(size_t)dev];
    if (!a.ptr || a.ctx != ctx || !ctx) { // set-up, once per device and context, with that device current
      e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
      if (e != cudaSuccess) {
        gjx::set_error(cudaGetErrorString(e));
        return GJX_ERR_CUDA;
      }
      a.ptr = ptr;
      a.ctx = ctx;
    }
    ptr = a.ptr;
  }
  return gjx::noalloc_sweeps(routine, nrow, ncol, nplus, dG, lddG, dV, lddV, dD, stream, ptr, kScratchBytes, dev,
                             ctx, glbSwp, glb_s, glb_b);
}

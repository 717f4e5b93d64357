// y = K x for callers that cannot allocate device memory.
//
// dp_apply_K stages x and y in the lattice numbering through work vectors the
// context allocated with cudaMalloc.  Some callers cannot allocate at all:
// hosts whose device memory is owned by a pool or allocator of their own that
// the library must not bypass, and real-time loops that forbid allocation
// after start-up (cudaMalloc / cudaFree may synchronise the device and take
// unbounded time).  dp_apply_K_noalloc does the same apply with its two
// staging vectors in one static device array of this file instead, and calls
// no cudaMalloc / cudaFree / allocating library routine.
//
// Ordering: the call reads x and writes y on the context's stream and returns
// after synchronising that stream.  It does not wait for other streams, so
// the caller must have finished producing x (and consuming y) first, e.g. by
// synchronising the stream that wrote x.
//
// Limits and sharing:
//   - the array holds kNoAllocScratchDoubles doubles (32 MiB); a mesh needs
//     4 * nnod of them, so nnod <= 1,048,576 (e.g. 128 x 1024 cells);
//     larger meshes are rejected with DP_BAD_ARG;
//   - every process that loads the library holds the array on every GPU it
//     uses, until exit;
//   - all calls on a device share the one array and it keeps the last call's
//     contents; the kernels zero what must start at zero.  Two calls whose
//     work overlaps on the GPU (different streams or contexts on the same
//     device, or host threads calling concurrently) race on it.
//   - the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress, with that device current); make that first call
//     before any stream capture begins.
#include <mutex>

namespace dp {

constexpr size_t kNoAllocScratchDoubles = (size_t)4 << 20;  // 4 Mi doubles = 32 MiB

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

constexpr int kNoAllocMaxDevices = 128;
static std::mutex g_noalloc_mu;
static double* g_noalloc_addr[kNoAllocMaxDevices] = {nullptr};

// Device address of the scratch array on `device` (which must be current).
// In host code the array's name is only a stand-in for the symbol, so the
// address is looked up once per device and cached.
static double* noalloc_scratch(int device) {
  if (device < 0 || device >= kNoAllocMaxDevices) throw BadArg("device ordinal out of range for the static scratch");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[device]) {
    void* p = nullptr;
    DP_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_noalloc_addr[device] = static_cast<double*>(p);
  }
  return g_noalloc_addr[device];
}

}  // namespace dp

extern "C" int dp_apply_K_noalloc(dp_ctx* h, const double* x, double* y) {
  if (!h) return DP_BAD_ARG;
  dp::Ctx& c = h->c;
  return dp::guarded(&c, [&] {
    DP_CUDA(cudaSetDevice(c.device));
    const int64_t nn = c.fine.nnod;
    if ((size_t)(4 * nn) > dp::kNoAllocScratchDoubles)
      throw dp::BadArg("dp_apply_K_noalloc: mesh has " + std::to_string(nn) +
                       " nodes; the static scratch holds 4*nnod <= 4194304 doubles (nnod <= 1048576)");
    if (c.assembled < 0) throw dp::BadArg("dp_assemble must run first");
    if (!x || !y) throw dp::BadArg("null argument");
    double* s = dp::noalloc_scratch(c.device);
    double* xl = s;            // x in the lattice numbering
    double* yl = s + 2 * nn;   // K x in the lattice numbering (zeroed before the apply)
    dp::launch_gather_ref2lat(c, x, xl, 2);
    dp::launch_apply_K<double, double>(c.fine, c.K64, xl, yl, c.stream);
    dp::launch_scatter_lat2ref(c, yl, y, 2);
    DP_CUDA(cudaStreamSynchronize(c.stream));
    return (int)DP_OK;
  });
}

// qwsg_jinv_s_noalloc: the block-Richardson solve (jinv) without any device
// allocation by the library.
//
// Why it exists: some callers cannot let a library allocate GPU memory while
// they run.  A program that has reserved its whole device-memory budget up
// front (for example under a framework's own caching allocator, or next to
// resident gauge fields sized to the last gigabyte) gets an out-of-memory
// error from a surprise cudaMalloc; a latency-critical loop cannot afford one
// either, because cudaMalloc/cudaFree may synchronise the device and stall
// every stream.  qwsg_jinv_s (include/qwsg.h) allocates its intermediate
// Richardson iterate lazily on first use; this variant instead uses a fixed
// array compiled into the library, so the caller only provides the input b
// and the output x.
//
// The scratch array is kJinvScratchFloats floats (32 MiB).  Every GPU that
// loads the library reserves it until the process exits.  It holds one FP32
// spinor in the library's plane layout (24 * pad floats), so lattices with
// pad > kJinvScratchFloats / 24 = 349,525 sites (e.g. 16^3x32 and 24^3x24 fit;
// 32^3x64 does not) are rejected with error code 2.
//
// Host code must not take the array's address directly: on the host the
// symbol names a host-side stand-in, not device memory.  The device address
// is obtained once per device with cudaGetSymbolAddress, with that device
// current, on the first call made on that device; make that first call
// before any stream capture starts.  All calls share the one array, which
// keeps whatever the previous call left in it: calls that overlap on the GPU
// (different streams, or different lattices on one device) race on it.
// Nothing in it has to start at zero, because each call writes every scratch
// site it later reads (the Richardson steps only read sites of the colour they
// have just written).
//
// It takes handles made by qwsg_create only: a handle made by
// qwsg_create_batch reads its parent's fields through a synchronisation
// with the parent's stream and may carry a kappa per RHS, which this path
// does not follow (it returns code 1 for such handles).  It reads the 12-real
// links when an earlier FP32 call on the handle has found the links SU(3)
// and made that copy (qwsg_jinv_s does so on its first call), otherwise the
// full 18-real links; the two forms agree to a few FP32 roundoffs.  Its
// launches count in the library's launch counter and in the handle's jinv
// call count; per-kernel timing does not record them.
#include <mutex>

#include "../../include/qwsg.h"
#include "ctx.h"

namespace {

constexpr size_t kJinvScratchFloats = size_t(8) << 20;  // 32 MiB
constexpr int kMaxDevices = 64;

static __device__ __align__(256) float g_jinv_scratch[kJinvScratchFloats];

std::mutex g_mu;
float* g_scratch_dev[kMaxDevices] = {};

// device address of g_jinv_scratch on the current device (set up once)
int scratch_for_device(int dev, float** out) {
  if (dev < 0 || dev >= kMaxDevices) return 2;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_dev[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_jinv_scratch);
    if (e != cudaSuccess || !p) {
      qwsg::set_error(std::string("qwsg_jinv_s_noalloc: cudaGetSymbolAddress failed: ") +
                      cudaGetErrorString(e));
      return 3;
    }
    g_scratch_dev[dev] = static_cast<float*>(p);
  }
  *out = g_scratch_dev[dev];
  return 0;
}

}  // namespace

extern "C" int qwsg_jinv_s_noalloc(qwsg_lattice* lat, float* x, const float* b, int colour,
                                   int nm) {
  using namespace qwsg;
  if (!lat || !lat->c) {
    set_error("qwsg_jinv_s_noalloc: lattice handle is NULL");
    return 4;
  }
  Ctx& c = *lat->c;
  if (c.parent) {
    set_error("qwsg_jinv_s_noalloc: not available on a handle made by qwsg_create_batch");
    return 1;
  }
  if (c.G.nr != 1) {
    set_error("qwsg_jinv_s_noalloc: not available on a multi-RHS handle");
    return 1;
  }
  if (24 * (size_t)c.G.pad > kJinvScratchFloats) {
    set_error("qwsg_jinv_s_noalloc: lattice of " + std::to_string(c.G.V) +
              " sites exceeds the fixed scratch (at most " +
              std::to_string(kJinvScratchFloats / 24) + " sites incl. padding); use qwsg_jinv_s");
    return 2;
  }
  if (colour != 0 && colour != 1) {
    set_error("qwsg_jinv_s_noalloc: colour must be 0 or 1");
    return 1;
  }
  if (!x || !b || x == b) {
    set_error("qwsg_jinv_s_noalloc: x and b must be distinct device buffers");
    return 1;
  }
  if (!c.Us || !c.Cs) {
    set_error("qwsg_jinv_s_noalloc: gauge/clover fields not loaded");
    return 4;
  }
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev != c.device) {
    set_error("qwsg_jinv_s_noalloc: the lattice's device must be current");
    return 1;
  }
  float* scratch = nullptr;
  int rc = scratch_for_device(dev, &scratch);
  if (rc) return rc;

  // nm Richardson steps x <- b + kappa A^-1 H_blk x from x = b, ping-ponging
  // through the scratch so that the last step lands in x
  const int steps = nm < 1 ? 1 : nm;
  HopArgs<float> a{};
  a.G = c.G;
  a.U = c.Us;
  a.U12 = (c.links12_valid && c.links12_on) ? c.Us12 : nullptr;  // made earlier, if at all
  a.C = c.Cs;
  a.aux = b;
  a.coef = (float)c.kappa;
  a.site0 = colour * c.G.Vh;
  a.nsites = c.G.Vh;
  a.dom = -1;
  a.zero_col = -1;
  const float* src = b;
  for (int k = 1; k <= steps; k++) {
    float* dst = ((steps - k) % 2 == 0) ? x : scratch;
    a.src = src;
    a.out = dst;
    launch_hop<float>(HOP_INNER, EPI_JINV, a, c.st);
    src = dst;
  }
  c.n_jinv++;
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(std::string("qwsg_jinv_s_noalloc: launch failed: ") + cudaGetErrorString(e));
    return 3;
  }
  return 0;
}

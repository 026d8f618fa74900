// sj_l2.h -- L2 access-policy windows for the probe launches.
//
// The structures every probe row looks up at random -- the plain engine's
// perfect hash tables and filters, the shared scan's per-slot query-mask words --
// are a few MB to a few tens of MB, while each probe streams GBs of fact
// columns past them.  A launch carries an access-policy window over the looked-up
// region: its hits are marked persisting and stay in the L2 set-aside the engine
// reserves (sj_engine_create), so the fact stream (loads marked evict-first)
// cannot push them out.  The window is a launch attribute, so the caller's
// stream attributes are left as they were.
#ifndef SJ_L2_H
#define SJ_L2_H

#include <cuda_runtime.h>

#include <cstddef>
#include <utility>

namespace sj {

// Smallest looked-up region that gets a window.  Below it the loads' own
// evict-last hints already keep the region resident against the evict-first
// fact stream (measured: no change at 6.6 MB of hash tables and 13.6 MB of mask
// words), and the window only adds its per-launch set-up.
constexpr size_t kL2WindowMinBytes = 16ull << 20;

struct L2Window {
  const void* base = nullptr;
  size_t bytes = 0;       // 0: launch without a window
  float hit_ratio = 0.f;  // share of the window's accesses marked persisting
};

// Window over [base, base + bytes) sized against a set-aside of `persist_bytes`
// and the device's largest window `max_window` (no window when either is 0 or
// the region is under kL2WindowMinBytes).
inline L2Window l2_window(const void* base, size_t bytes, size_t persist_bytes, size_t max_window) {
  L2Window w;
  if (!base || bytes < kL2WindowMinBytes || !persist_bytes || !max_window) return w;
  w.base = base;
  w.bytes = bytes < max_window ? bytes : max_window;
  const double r = (double)persist_bytes / (double)w.bytes;
  w.hit_ratio = r >= 1.0 ? 1.f : (float)r;
  return w;
}

// Launch `kernel` with the window as a launch attribute (none when the window is
// empty).  pdl: programmatic dependent launch -- the kernel may be scheduled
// while the previous kernel of the stream runs, and waits (griddepcontrol.wait)
// for it before reading its output; only for a kernel whose predecessor in the
// stream is a kernel that calls pdl_launch_dependents.
template <typename... K, typename... A>
cudaError_t launch_windowed(void (*kernel)(K...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                            const L2Window& w, bool pdl, A&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[2];
  unsigned n = 0;
  if (w.bytes) {
    attr[n].id = cudaLaunchAttributeAccessPolicyWindow;
    attr[n].val.accessPolicyWindow.base_ptr = const_cast<void*>(w.base);
    attr[n].val.accessPolicyWindow.num_bytes = w.bytes;
    attr[n].val.accessPolicyWindow.hitRatio = w.hit_ratio;
    attr[n].val.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
    attr[n].val.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
    ++n;
  }
  if (pdl) {
    attr[n].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[n].val.programmaticStreamSerializationAllowed = 1;
    ++n;
  }
  cfg.attrs = n ? attr : nullptr;
  cfg.numAttrs = n;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...);
}

}  // namespace sj

#endif  // SJ_L2_H

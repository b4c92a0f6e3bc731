// lbl_noalloc.cu -- lbl_merge_layer_noalloc: one merge step that performs no
// memory allocation at all.
//
// Some callers cannot allocate device memory: code running where a caching
// allocator owns the device, inside a region that must not grow the memory
// footprint, or a host framework that only hands out buffers it already
// owns.  For them this entry point runs the same merge kernel as
// lbl_merge_layer (EMIN + EMINIT/RADNN) on caller-owned device buffers.  Its
// only scratch -- the per-layer plan and the table of panel origins -- lives
// in the file-scope device array below, whose size bounds the layer length.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <mutex>

#include "../../include/lblgpu.h"
#include "lbl_kernels.cuh"
#include "lbl_plan.h"

using namespace lbl;

namespace {

constexpr int kMaxPanels = LBL_NOALLOC_MAX_PANELS;
constexpr size_t kPlanBytes = (sizeof(LayerDev) + 255) & ~size_t(255);
constexpr size_t kScratchBytes = kPlanBytes + kMaxPanels * sizeof(double);

// Scratch of every call on a device; each device that loads the library
// holds it until the process exits.
static __device__ __align__(256) unsigned char g_merge_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char* g_scratch_ptr[kMaxDevices] = {nullptr};

// Device memory of GPU `device` (a buffer on another GPU would be read as a
// peer access, which faults unless peer access is enabled).
bool on_device(const void* p, int device) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (a.type == cudaMemoryTypeManaged) return true;
  return a.type == cudaMemoryTypeDevice && a.device == device;
}

// Byte ranges [a, a+na) and [b, b+nb) share memory.
bool overlap(const void* a, int64_t na, const void* b, int64_t nb) {
  if (!a || !b || na <= 0 || nb <= 0) return false;
  const uintptr_t x = reinterpret_cast<uintptr_t>(a), y = reinterpret_cast<uintptr_t>(b);
  return x < y + (uintptr_t)nb && y < x + (uintptr_t)na;
}

// Restores the caller's current device when the call returns.
struct DeviceGuard {
  int prev = -1;
  DeviceGuard() {
    if (cudaGetDevice(&prev) != cudaSuccess) {
      cudaGetLastError();
      prev = -1;
    }
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

}  // namespace

extern "C" int lbl_merge_layer_noalloc(int device, const lbl_run* run, const lbl_layer* layer,
                                       int32_t first, double dv_old, const double* rad_in,
                                       const double* tr_in, int64_t n_old, const double* od,
                                       double* rad_out, double* tr_out, int64_t n_new,
                                       void* stream) {
  if (!run || !layer || !od || !rad_out || device < 0 || device >= kMaxDevices) return LBL_E_ARG;
  if (run->iemit != 0 && run->iemit != 1) return LBL_E_ARG;
  if (run->iemit == 1 && !tr_out) return LBL_E_ARG;
  if (run->iemit == 1 && (run->ipathl != 1 || run->bndrfl != 0.)) return LBL_E_ARG;
  if (first != 0 && first != 1) return LBL_E_ARG;
  if (!first && (!rad_in || (run->iemit == 1 && !tr_in) || n_old < 1)) return LBL_E_ARG;
  if (!(layer->dv > 0.) || !(run->v2 > run->v1) || !(run->v1 > 0.) || n_new < 1)
    return LBL_E_ARG;
  if (!first && layer->dv > dv_old) return LBL_E_ITYPE;
  // the kernel reads neighbouring points of rad_in/tr_in while it writes
  // rad_out/tr_out, so an output shares memory with no other buffer, except
  // that it may be od itself (each point of od is read and then written by
  // the same thread)
  {
    const int64_t bo = 8 * n_new, bi = first ? 0 : 8 * n_old;
    const double* outs[2] = {rad_out, run->iemit == 1 ? tr_out : nullptr};
    const double* ins[2] = {first ? nullptr : rad_in,
                            (first || run->iemit != 1) ? nullptr : tr_in};
    for (const double* o : outs)
      for (const double* i : ins)
        if (overlap(o, bo, i, bi)) return LBL_E_ARG;
    if (overlap(outs[0], bo, outs[1], bo)) return LBL_E_ARG;
    for (const double* o : outs)
      if (o != od && overlap(o, bo, od, bo)) return LBL_E_ARG;
  }
  DeviceGuard guard;
  if (cudaSetDevice(device) != cudaSuccess) return LBL_E_CUDA;
  // inputs and outputs must already be memory of this device: nothing is staged
  if (!on_device(od, device) || !on_device(rad_out, device) ||
      (run->iemit == 1 && !on_device(tr_out, device)) ||
      (!first && (!on_device(rad_in, device) ||
                  (run->iemit == 1 && !on_device(tr_in, device)))))
    return LBL_E_ARG;
  // panel origins VFT_p exactly as PANEL accumulates them; the layer's
  // length is bounded by the scratch table
  double vft[kMaxPanels];
  int64_t npanel = 0, nhi_last = 0;
  {
    const double dv = layer->dv;
    double v = run->v1 - 32. * dv;
    for (;;) {
      if (npanel >= kMaxPanels) return LBL_E_RANGE;  // layer longer than the scratch
      vft[npanel++] = v;
      long nhi = 2432;
      if ((v + double(nhi - 1) * dv) > run->v2) {
        nhi = (long)((run->v2 - v) / dv + 1.);
        if (v + double(nhi - 1) * dv < run->v2) nhi = nhi + 1;
        nhi_last = nhi;
        break;
      }
      v = v + double(kNlim1 - 1) * dv;
    }
  }
  const int64_t npts = 2400 * (npanel - 1) + (nhi_last - 33 + 1);
  if (npts != n_new) return LBL_E_ARG;
  // the merge kernel reads only these plan fields
  LayerDev d;
  std::memset(&d, 0, sizeof(d));
  d.tave = layer->tave;
  d.dv = layer->dv;
  d.v1 = run->v1;
  d.v2 = run->v2;
  d.npts = npts;
  d.npanel = npanel;
  // one-time set-up on this device: the scratch array's device address
  unsigned char* scratch;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_ptr[device]) {
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, g_merge_scratch) != cudaSuccess || !p) {
        cudaGetLastError();
        return LBL_E_CUDA;
      }
      g_scratch_ptr[device] = static_cast<unsigned char*>(p);
    }
    scratch = g_scratch_ptr[device];
  }
  LayerDev* d_plan = reinterpret_cast<LayerDev*>(scratch);
  double* d_vft = reinterpret_cast<double*>(scratch + kPlanBytes);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (cudaMemcpyAsync(d_plan, &d, sizeof(d), cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(d_vft, vft, npanel * sizeof(double), cudaMemcpyHostToDevice, s) !=
          cudaSuccess)
    return LBL_E_CUDA;
  const double tbnd = (first && run->ipathl == 1) ? run->tmpbnd : 0.;
  // IEMIT=0 leaves tr_in/tr_out unused
  const double* tin = run->iemit == 1 ? tr_in : nullptr;
  double* tout = run->iemit == 1 ? tr_out : nullptr;
  if (launch_merge(d_plan, d_vft, od, npts, first, dv_old, n_old, rad_in, tin, rad_out, tout,
                   tbnd, run->bndemi, run->iemit, layer->tzu, s) != cudaSuccess)
    return LBL_E_CUDA;
  // the host-side plan buffers are on this stack frame: wait for the copies
  if (cudaStreamSynchronize(s) != cudaSuccess) return LBL_E_CUDA;
  return LBL_OK;
}

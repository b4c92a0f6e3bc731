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

bool on_device(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace

extern "C" int lbl_merge_layer_noalloc(int device, const lbl_run* run, const lbl_layer* layer,
                                       int32_t first, double dv_old, const double* rad_in,
                                       const double* tr_in, int64_t n_old, const double* od,
                                       double* rad_out, double* tr_out, int64_t n_new,
                                       void* stream) {
  if (!run || !layer || !od || !rad_out || device < 0 || device >= kMaxDevices) return LBL_E_ARG;
  if (run->iemit == 1 && !tr_out) return LBL_E_ARG;
  if (run->iemit == 1 && run->ipathl != 1) return LBL_E_ARG;
  if (!first && (!rad_in || (run->iemit == 1 && !tr_in) || n_old < 1)) return LBL_E_ARG;
  if (!(layer->dv > 0.) || !(run->v2 > run->v1)) return LBL_E_ARG;
  if (!first && layer->dv > dv_old) return LBL_E_ITYPE;
  if (cudaSetDevice(device) != cudaSuccess) return LBL_E_CUDA;
  // inputs and outputs must already be device memory: nothing is staged
  if (!on_device(od) || !on_device(rad_out) || (tr_out && !on_device(tr_out)) ||
      (!first && (!on_device(rad_in) || (tr_in && !on_device(tr_in)))))
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
  if (launch_merge(d_plan, d_vft, od, npts, first, dv_old, n_old, rad_in, tr_in, rad_out, tr_out,
                   tbnd, run->bndemi, run->iemit, layer->tzu, s) != cudaSuccess)
    return LBL_E_CUDA;
  // the host-side plan buffers are on this stack frame: wait for the copies
  if (cudaStreamSynchronize(s) != cudaSuccess) return LBL_E_CUDA;
  return LBL_OK;
}

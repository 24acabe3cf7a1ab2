// swd_pick_noalloc: the guided dispersion-curve picker of swd_pick on caller-owned device
// memory, with no device allocation anywhere on its path.
//
// swd_pick stages its spectrum and its scratch (the per-column pick differences and the pick
// status word) in cudaMalloc'd memory.  This entry point takes the spectrum, the reference curve
// and the outputs as device pointers and keeps the scratch in one static device array of this
// library (g_pick_scratch), so a caller that cannot allocate device memory can still pick.
//
// g_pick_scratch is per device: every GPU that loads libswd.so holds its 16 KiB until the process
// exits.  In host code the name g_pick_scratch is only a stand-in for the device symbol; its
// device address comes from cudaGetSymbolAddress (with the device current; return code checked)
// and is passed to the kernel as a plain pointer.  The first call on a device does that set-up,
// so it must come before any stream capture on that device.  Outside a capture every call looks
// the address up again (a cheap runtime lookup), so a cudaDeviceReset, which unloads the module
// and may place the array elsewhere when it is loaded again, never leaves a stale address
// behind; inside a capture the address found by the last uncaptured call on the device is used.
// Every call shares the array and it keeps the last call's contents: the status word is cleared
// on the stream before each launch, and the differences are written before anything reads them.
// Calls that overlap on the GPU (two streams, two host threads) race on the array.
#include <mutex>

#include "fd_host.cuh"
#include "radon.cuh"

constexpr int kMaxNpair = SWD_PICK_NOALLOC_MAX_NPAIR;
// dc[kMaxNpair] | misfit (used when the caller passes no d_res) | status word (an int)
constexpr int kScratchDoubles = kMaxNpair + 2;
static_assert((kMaxNpair + 1) * (4 * sizeof(int) + sizeof(double)) <= 48 * 1024,
              "the picker's per-column shared arrays must fit the default 48 KiB");

static __device__ __align__(256) double g_pick_scratch[kScratchDoubles];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
double* g_scratch_addr[kMaxDevices] = {};

// Device address of g_pick_scratch on the current device: looked up now unless `st` is being
// captured, else the address of the last lookup on this device.
int scratch_on_current_device(cudaStream_t st, double** out) {
  int dev = -1;
  SWD_CUDA(cudaGetDevice(&dev));
  SWD_CHECK(dev >= 0 && dev < kMaxDevices, "device %d is beyond the %d devices this entry point tracks", dev,
            kMaxDevices);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  SWD_CUDA(cudaStreamIsCapturing(st, &cap));
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (cap == cudaStreamCaptureStatusNone) {
    void* p = nullptr;
    SWD_CUDA(cudaGetSymbolAddress(&p, g_pick_scratch));
    g_scratch_addr[dev] = static_cast<double*>(p);
  }
  SWD_CHECK(g_scratch_addr[dev] != nullptr,
            "the first swd_pick_noalloc call on device %d must come before any stream capture", dev);
  *out = g_scratch_addr[dev];
  return SWD_OK;
}

}  // namespace

using namespace swd;

extern "C" int swd_pick_noalloc(const double* d_ml, int np_, int npair, double vmin, const double* d_cr_0,
                                int method, int ini, double* d_res, double* d_cr_pre, void* stream) {
  clear_error();
  SWD_CHECK(d_ml && d_cr_0 && d_cr_pre && np_ >= 1 && npair >= 1, "bad pick arguments");
  SWD_CHECK(npair <= kMaxNpair,
            "npair %d exceeds the %d columns of the allocation-free picker's static scratch (swd_pick has no "
            "such limit on the scratch)",
            npair, kMaxNpair);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  double* scratch = nullptr;
  SWD_TRY(scratch_on_current_device(st, &scratch));
  double* d_dc = scratch;
  double* d_res_scratch = scratch + kMaxNpair;
  int* d_status = reinterpret_cast<int*>(scratch + kMaxNpair + 1);
  // pick_batch clears the status word on st before it launches the picker
  SWD_TRY(pick_batch(np_, npair, 1, ini, method, vmin, nullptr, d_ml, d_cr_0, d_cr_pre, d_dc,
                     d_res ? d_res : d_res_scratch, d_status, st));
  int status = 0;
  SWD_CUDA(cudaMemcpyAsync(&status, d_status, sizeof(int), cudaMemcpyDeviceToHost, st));
  SWD_CUDA(cudaStreamSynchronize(st));
  if (status == 1) { set_error("NaN in the dispersion spectrum"); return SWD_ERR_NUMERIC; }
  if (status == 2) { set_error("interp1 needs at least two retained picks (pickFDC1.m:129)"); return SWD_ERR_NUMERIC; }
  return SWD_OK;
}

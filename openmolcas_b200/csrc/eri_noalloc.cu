// Allocation-free variant of the batched ERI entry point.
//
// mg_eri_quartets keeps its list of work items in a device workspace that it
// grows with cudaMalloc.  Some callers cannot let a library allocate device
// memory during a call: a Fortran or C++ program that reserves all device
// memory up front in its own pool, a framework whose caching allocator
// already holds the memory (cudaMalloc then fails or fragments it), or code
// that must not insert the implicit device synchronisation of cudaFree
// between its stream-ordered work.  This variant stages the work items in a
// fixed file-scope device array instead.
//
// The array is a static __device__ symbol, so every GPU that loads the
// library holds kNoAllocMaxItems * sizeof(EriItem) bytes (1.5 MiB) of it until
// the process exits.  In host code its name is only a host-side stand-in; the
// device address is obtained once per device with cudaGetSymbolAddress while
// that device is current, and that address is what the kernels receive.
#include <cuda_runtime.h>

#include <mutex>
#include <vector>

#include "../../include/molgpu.h"  // the definition below is checked against its declaration
#include "mg_internal.h"

namespace mg {

// Largest number of work items one call may use (a work item is one shell
// quartet, or a slice of one when its contracted block is large).
static const int kNoAllocMaxItems = 65536;

static __device__ __align__(256) EriItem g_noalloc_items[kNoAllocMaxItems];
// work counters of the class launches (one per class, at most 64 classes)
static __device__ int g_noalloc_counters[64];

static const int kMaxDevices = 64;
static EriItem* g_noalloc_ptr[kMaxDevices] = {nullptr};
static int* g_noalloc_cnt[kMaxDevices] = {nullptr};
static std::mutex g_noalloc_mutex;

// Device address of g_noalloc_items on `device` (set up on first use, with
// that of g_noalloc_counters; the device must be current).  Returns nullptr
// on failure.
static EriItem* noalloc_items_ptr(int device) {
  if (device < 0 || device >= kMaxDevices) return nullptr;
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[device]) {
    void* p = nullptr;
    void* c = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_items) != cudaSuccess) return nullptr;
    if (cudaGetSymbolAddress(&c, g_noalloc_counters) != cudaSuccess) return nullptr;
    g_noalloc_cnt[device] = (int*)c;
    g_noalloc_ptr[device] = (EriItem*)p;
  }
  return g_noalloc_ptr[device];
}

}  // namespace mg

struct mg_handle {
  mg::Handle h;
};

using namespace mg;

extern "C" int mg_eri_quartets_noalloc(mg_handle* H, const int32_t* q4, int64_t nq, const int64_t* offsets,
                                       double* d_out, void* stream) {
  if (!H || (!q4 && nq) || !offsets || (!d_out && nq)) return MG_ERR_ARG;
  Handle* h = &H->h;
  if (cudaSetDevice(h->device) != cudaSuccess) {
    h->err = "mg_eri_quartets_noalloc: cannot select the handle's device";
    return MG_ERR_CUDA;
  }
  std::vector<EriItem> items;
  std::vector<EriClass> classes;
  int rc = build_eri_items(h, q4, nq, offsets, items, classes);
  if (rc) return rc;
  if (items.size() > (size_t)kNoAllocMaxItems) {
    h->err = "mg_eri_quartets_noalloc: " + std::to_string(items.size()) +
             " work items exceed the fixed capacity of " + std::to_string(kNoAllocMaxItems) +
             "; split the quartet list or use mg_eri_quartets";
    return MG_ERR_ARG;
  }
  if (items.empty()) return 0;
  EriItem* d_items = noalloc_items_ptr(h->device);
  if (!d_items) {
    h->err = "mg_eri_quartets_noalloc: cudaGetSymbolAddress failed";
    return MG_ERR_CUDA;
  }
  cudaStream_t st = (cudaStream_t)stream;
  if (cudaMemcpyAsync(d_items, items.data(), sizeof(EriItem) * items.size(), cudaMemcpyHostToDevice, st) !=
      cudaSuccess) {
    h->err = "mg_eri_quartets_noalloc: work-item upload failed";
    return MG_ERR_CUDA;
  }
  int* d_cnt = g_noalloc_cnt[h->device];
  if (cudaMemsetAsync(d_cnt, 0, sizeof(int) * 64, st) != cudaSuccess) {
    h->err = "mg_eri_quartets_noalloc: counter reset failed";
    return MG_ERR_CUDA;
  }
  for (size_t ci = 0; ci < classes.size(); ++ci) {
    const EriClass& c = classes[ci];
    if (eri_launch_class(h, d_items + c.begin, c.count, c.nab, c.ncd, c.plan, d_out, d_cnt + ci, st)) {
      h->err = std::string("ERI kernel launch failed: ") + cudaGetErrorString(cudaGetLastError());
      return MG_ERR_CUDA;
    }
  }
  return 0;
}

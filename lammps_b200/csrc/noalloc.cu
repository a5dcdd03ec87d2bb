// noalloc.cu -- the kinetic-energy sum for callers that cannot allocate
// device memory.
//
// Some hosts cannot call cudaMalloc at the point where they need the sum:
// code running while a stream is being captured into a CUDA graph (an
// allocation there is not allowed), or integrations whose device memory is
// owned by another allocator.  This file gives them one entry point that
// allocates nothing: the caller passes device arrays in and a device result
// out, and the reduction's scratch (one partial sum per block and the
// completion counter) lives in a file-scope __device__ array of fixed size.
// Every GPU that loads the library holds that array until the process
// exits.  All calls share it, so calls that overlap on the GPU (on
// different streams, or from different host threads) race; serialise them.
#include <mutex>

#include "md_state.h"

namespace {

constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocBlocks = 1184;  // 8 blocks of 256 threads on each of 148 SMs
constexpr int kNoAllocMaxDevices = 64;

struct NoAllocScratch {
  double partial[kNoAllocBlocks];  // one partial sum per block, rewritten by every call
  unsigned int counter;            // blocks finished; zeroed before every call
};

// In host code this name is only a stand-in for the device array; its device
// address comes from cudaGetSymbolAddress (see scratch_address).
static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

std::mutex g_setup_mutex;
NoAllocScratch *g_scratch_addr[kNoAllocMaxDevices] = {};

// Device address of the scratch array on the current device, looked up once
// per device (with that device current) and cached.
cudaError_t scratch_address(int device, NoAllocScratch **out) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[device]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_addr[device] = static_cast<NoAllocScratch *>(p);
  }
  *out = g_scratch_addr[device];
  return cudaSuccess;
}

// sum over atoms of (vx^2 + vy^2 + vz^2) * mass[type] (the term of
// ComputeTemp::compute_scalar); grid-stride, deterministic two-level sum.
// An atom whose type lies outside 1..ntypes never indexes mass[]: it adds a
// NaN instead, so the result the caller reads is NaN.
__global__ void __launch_bounds__(kNoAllocThreads)
    k_kinetic_noalloc(int n, const double *__restrict__ v, const int *__restrict__ type,
                      const double *__restrict__ mass, int ntypes, NoAllocScratch *scratch,
                      double *__restrict__ out) {
  __shared__ double red[kNoAllocThreads / 32];
  double acc[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double vx = v[3 * i], vy = v[3 * i + 1], vz = v[3 * i + 2];
    const int t = type[i];
    acc[0] += (t >= 1 && t <= ntypes) ? (vx * vx + vy * vy + vz * vz) * mass[t]
                                      : __longlong_as_double(0x7ff8000000000000LL);
  }
  block_partials_finish<1>(acc, red, scratch->partial, &scratch->counter, out, false);
}

}  // namespace

extern "C" int b200_kinetic_sum_noalloc(int n, const double *v, const int *type,
                                        const double *mass, int ntypes, double *out,
                                        void *stream) {
  if (n < 1 || n > MD_MAX_ATOMS || !v || !type || !mass || !out || ntypes < 1 ||
      ntypes > MD_MAXTYPES)
    return B200_ERR_ARG;
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kNoAllocMaxDevices)
    return B200_ERR_CUDA;
  NoAllocScratch *scratch = nullptr;
  if (scratch_address(device, &scratch) != cudaSuccess) return B200_ERR_CUDA;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // the completion counter must start at zero; the partials need no clearing
  if (cudaMemsetAsync(&scratch->counter, 0, sizeof(unsigned int), s) != cudaSuccess)
    return B200_ERR_CUDA;
  int blocks = (n + kNoAllocThreads - 1) / kNoAllocThreads;
  if (blocks > kNoAllocBlocks) blocks = kNoAllocBlocks;
  k_kinetic_noalloc<<<blocks, kNoAllocThreads, 0, s>>>(n, v, type, mass, ntypes, scratch,
                                                        out);
  return cudaGetLastError() == cudaSuccess ? B200_OK : B200_ERR_CUDA;
}

// noalloc.cu -- dense exact permanent for callers that cannot allocate device
// memory.
//
// Some callers cannot call cudaMalloc: code that runs inside another
// framework's memory pool or allocator and must not take memory behind its
// back, plugins loaded into a host process that owns every device allocation,
// and code paths that run while allocation is forbidden (for example between
// the steps of a caller's own fixed memory plan).  perm_exact_dense_noalloc
// serves them: the caller passes a device-resident input matrix and a device
// output buffer, and every other byte the computation needs lives in
// g_noalloc_scratch below, a file-scope __device__ array that each GPU loading
// this library holds until the process exits.  The entry point calls no
// cudaMalloc, cudaFree or other allocating routine.
//
// The compute is the FP64-X dense Ryser kernel (ryser_dense.cuh), unchanged;
// only where its operand, grid partials, completion ticket and error flag live
// differs from perm_exact_dense.
//
// Rules for callers:
//  * Orders 1..64 (kNoAllocMaxOrder): the scratch holds one 64 x 64 operand
//    image and partials for at most kNoAllocMaxBlocks CTAs; larger orders are
//    rejected with PERM_EUNSUPPORTED and a message on stderr.
//  * The first call on a device performs one-time set-up for that device
//    (looks up the scratch array's device address with cudaGetSymbolAddress and
//    the kernel's occupancy).  Make that first call before any stream capture.
//  * Every call on a device shares the one scratch array, which keeps the last
//    call's contents.  Calls whose work overlaps on the GPU (different
//    streams, or host threads racing on one device) corrupt each other: order
//    them on one stream or synchronise between them.
//  * The call is asynchronous on `stream`; d_out holds (hi, lo) once the
//    stream reaches it.  A staging timeout inside the kernel turns d_out into
//    NaN instead of a wrong value.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <mutex>

#include "../../include/perman_b200.h"
#include "ryser_dense.cuh"

namespace perm {
const void* dense_kernel_0(int n);
const void* dense_kernel_1(int n);
const void* dense_kernel_2(int n);
const void* dense_kernel_3(int n);
const void* dense_kernel_4(int n);

namespace {

constexpr int kNoAllocMaxOrder = 64;
constexpr int kNoAllocMaxBlocks = 4096;
constexpr int kNoAllocMaxDevices = 64;

struct NoAllocScratch {
  double operand[kNoAllocMaxOrder * kNoAllocMaxOrder];  // column-major, even stride (32 KB)
  dd partials[kNoAllocMaxBlocks];                        // one per CTA (64 KB)
  unsigned ticket;                                       // last-CTA completion counter
  int err;                                               // staging-timeout flag
};

// The scratch: ~96 KB per GPU, allocated when the module loads.
__device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(NoAllocScratch)];

// Column-major copy of the caller's row-major matrix into the scratch, and
// the fields that must start at zero.
__global__ void noalloc_prepare(const double* mat, int n, int np) {
  NoAllocScratch* s = reinterpret_cast<NoAllocScratch*>(g_noalloc_scratch);
  for (int idx = threadIdx.x; idx < n * np; idx += blockDim.x) {
    const int k = idx / np, j = idx % np;
    s->operand[idx] = j < n ? mat[j * n + k] : 0.0;
  }
  if (threadIdx.x == 0) {
    s->ticket = 0u;
    s->err = 0;
  }
}

__global__ void noalloc_check(double* out) {
  const NoAllocScratch* s = reinterpret_cast<const NoAllocScratch*>(g_noalloc_scratch);
  if (s->err) {
    out[0] = nan("");
    out[1] = nan("");
  }
}

const void* dense_kernel_for(int n) {
  if (n >= 1 && n <= 20) return dense_kernel_0(n);
  if (n <= 32) return dense_kernel_1(n);
  if (n <= 42) return dense_kernel_2(n);
  if (n <= 52) return dense_kernel_3(n);
  if (n <= 64) return dense_kernel_4(n);
  return nullptr;
}

struct DeviceSetup {
  NoAllocScratch* scratch = nullptr;  // device address of g_noalloc_scratch
  int sms = 0;
  int occ[kNoAllocMaxOrder + 1] = {};
};

std::mutex g_setup_mu;
DeviceSetup g_setup[kNoAllocMaxDevices];

int report(int code, const char* msg, cudaError_t e = cudaSuccess) {
  if (e != cudaSuccess)
    fprintf(stderr, "perm_exact_dense_noalloc: %s: %s\n", msg, cudaGetErrorString(e));
  else
    fprintf(stderr, "perm_exact_dense_noalloc: %s\n", msg);
  return code;
}

}  // namespace
}  // namespace perm

using namespace perm;

extern "C" int perm_exact_dense_noalloc(const double* d_mat, int n, double* d_out, void* stream) {
  if (!d_mat || !d_out) return report(PERM_EINVAL, "null device pointer");
  if (n < 1 || n > kNoAllocMaxOrder) {
    char msg[128];
    snprintf(msg, sizeof msg, "order %d outside [1, %d], the scratch capacity", n, kNoAllocMaxOrder);
    return report(PERM_EUNSUPPORTED, msg);
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return report(PERM_ECUDA, "cudaGetDevice", e);
  if (dev < 0 || dev >= kNoAllocMaxDevices) return report(PERM_EUNSUPPORTED, "device index too large");
  const void* fn = dense_kernel_for(n);
  const size_t smem = dense_smem_bytes(n);
  DeviceSetup su;
  {
    std::lock_guard<std::mutex> lock(g_setup_mu);
    DeviceSetup& s = g_setup[dev];
    if (!s.scratch) {  // one-time set-up of this device, with it current
      void* ptr = nullptr;
      e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
      if (e != cudaSuccess) return report(PERM_ECUDA, "cudaGetSymbolAddress(scratch)", e);
      e = cudaDeviceGetAttribute(&s.sms, cudaDevAttrMultiProcessorCount, dev);
      if (e != cudaSuccess) return report(PERM_ECUDA, "cudaDeviceGetAttribute", e);
      s.scratch = static_cast<NoAllocScratch*>(ptr);
    }
    if (!s.occ[n]) {
      int occ = 0;
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, 128, smem);
      if (e != cudaSuccess) return report(PERM_ECUDA, "occupancy query", e);
      s.occ[n] = occ > 0 ? occ : 1;
    }
    su = s;
  }

  // Launch plan: the same range decomposition as perm_exact_dense.
  const int np = (n + 1) & ~1;
  DenseArgs args;
  args.colA = su.scratch->operand;
  args.np = np;
  args.partials = su.scratch->partials;
  args.ticket = &su.scratch->ticket;
  args.out = d_out;
  args.err = &su.scratch->err;
  args.seg_blocks = 0;
  args.inject = 0;
  int grid = 1;
  if (n < 4) {
    args.m = 0;
    args.block0 = 0;
    args.nblocks = 0;
  } else {
    const uint64_t total = 1ull << (n - 1);
    grid = su.sms * su.occ[n];
    if (grid > kNoAllocMaxBlocks) grid = kNoAllocMaxBlocks;
    const uint64_t threads = (uint64_t)grid * 128;
    int m = 3;
    while (m < 20 && m < n - 1 && (total >> (m + 1)) >= threads * 64) m++;
    const uint64_t blocks = total >> m;
    if (blocks < threads) grid = (int)((blocks + 127) / 128);
    args.m = m;
    args.block0 = 0;
    args.nblocks = blocks;
    // X re-anchored every >= 2^11 Gray steps (orders <= kAnchorMaxN), as in
    // perm_exact_dense's FP64-X launches: same rounding behaviour
    args.seg_blocks = m >= 11 ? 1 : (1ull << (11 - m));
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  noalloc_prepare<<<1, 256, 0, st>>>(d_mat, n, np);
  void* kargs[] = {&args};
  e = cudaLaunchKernel(fn, dim3(grid), dim3(128), kargs, smem, st);
  if (e != cudaSuccess) return report(PERM_ECUDA, "kernel launch", e);
  noalloc_check<<<1, 1, 0, st>>>(d_out);
  e = cudaGetLastError();
  if (e != cudaSuccess) return report(PERM_ECUDA, "launch", e);
  return PERM_OK;
}

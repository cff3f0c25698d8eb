// Allocation-free batched triangular solve.
//
// Some callers of this library cannot allocate device memory at the time
// they solve: a real-time control loop that must not enter the CUDA memory
// allocator (its latency is unbounded and it can synchronize the device),
// or a host framework whose custom-call handler may only use buffers its own
// allocator handed in and has no slot for an extra workspace.  For them,
// wmpc_solve_noalloc runs the same solve as wmpc_solve, but its per-instance
// work vectors live in one fixed array of global memory owned by this
// library (g_noalloc_scratch below), so the caller passes only inputs and
// outputs.
//
// Capacity: n * batch <= kNoAllocScratchFloats (8,388,608 floats = 32 MiB);
// larger requests are rejected before anything is launched.  Every GPU that
// loads the library holds this array until the process exits.  All calls on
// a device share it and it keeps the previous call's contents (the kernel
// overwrites every element it reads first, so nothing needs clearing); two
// calls whose kernels overlap on the GPU (different streams without
// ordering) race on it and give wrong results.
#include <mutex>

#include "common.cuh"
#include "qdldl.cuh"

namespace wmpc {

constexpr size_t kNoAllocScratchFloats = 8u * 1024u * 1024u;

// The work vectors: one [KKT row][instance] block of n * batch floats.
static __device__ __align__(256) float g_noalloc_scratch[kNoAllocScratchFloats];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
float* g_scratch_addr[kMaxDevices] = {nullptr};

// Device address of g_noalloc_scratch on the current device.  On the host the
// array's name is only a stand-in for the device symbol, so the address is
// looked up once per device (with that device current) and cached.  The
// first call on a device does this lookup, so it should come before any
// stream capture that contains the call.
int scratch_address(int device, float** out) {
  if (device < 0 || device >= kMaxDevices) return fail(WMPC_ERR_INVALID_ARGUMENT, "device %d out of range", device);
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (g_scratch_addr[device] == nullptr) {
    void* p = nullptr;
    const cudaError_t err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (err != cudaSuccess)
      return fail(WMPC_ERR_CUDA, "cudaGetSymbolAddress(g_noalloc_scratch) failed: %s", cudaGetErrorString(err));
    g_scratch_addr[device] = static_cast<float*>(p);
  }
  *out = g_scratch_addr[device];
  return WMPC_OK;
}

}  // namespace

// Same arithmetic as the per-call solve kernel with an HBM work vector:
// permute, forward L, D^-1, backward L^T, unpermute.
__global__ void __launch_bounds__(128) solve_noalloc_kernel(Pattern pat, const float* __restrict__ lx,
                                                            const float* __restrict__ dinv, int fstride, long long ldf,
                                                            const float* rhs, float* out, float* scratch, int batch) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= batch) return;
  LaneVec x{scratch + b, (long long)batch};
  const int n = pat.n;
  for (int i = 0; i < n; ++i) x(i) = rhs[(long long)__ldg(pat.p + i) * batch + b];
  const long long fo = (long long)b * fstride;
  ldl_solve_permuted(pat, lx + fo, ldf, dinv + fo, ldf, x);
  for (int i = 0; i < n; ++i) out[(long long)i * batch + b] = x(__ldg(pat.pinv + i));
}

}  // namespace wmpc

using namespace wmpc;

extern "C" int wmpc_solve_noalloc(const wmpc_plan* plan, const float* lx, const float* dinv, int32_t factor_bstride,
                                  const float* rhs, float* x, int32_t batch, wmpc_stream_t stream) {
  if (!plan || batch < 0) return fail(WMPC_ERR_INVALID_ARGUMENT, "bad plan or batch");
  if (batch == 0) return WMPC_OK;
  if ((!lx && plan->pat.nnz_l > 0) || !dinv || !rhs || !x) return fail(WMPC_ERR_INVALID_ARGUMENT, "null buffer");
  if (factor_bstride != 0 && factor_bstride != 1)
    return fail(WMPC_ERR_INVALID_ARGUMENT, "factor_bstride must be 0 or 1");
  const size_t need = (size_t)plan->pat.n * (size_t)batch;
  if (need > kNoAllocScratchFloats)
    return fail(WMPC_ERR_WORKSPACE,
                "wmpc_solve_noalloc: n * batch = %zu floats exceeds its fixed scratch of %zu floats "
                "(n = %d allows batch <= %zu); use wmpc_solve with a caller workspace",
                need, kNoAllocScratchFloats, plan->pat.n, kNoAllocScratchFloats / (size_t)plan->pat.n);
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) return fail(WMPC_ERR_CUDA, "cudaGetDevice failed");
  if (prev != plan->device && cudaSetDevice(plan->device) != cudaSuccess)
    return fail(WMPC_ERR_CUDA, "cannot select device %d", plan->device);
  float* scratch = nullptr;
  int rc = scratch_address(plan->device, &scratch);
  if (rc == WMPC_OK) {
    const long long ldf = factor_bstride ? batch : 1;
    solve_noalloc_kernel<<<ceil_div(batch, 128), 128, 0, static_cast<cudaStream_t>(stream)>>>(
        plan->pat, lx, dinv, factor_bstride, ldf, rhs, x, scratch, batch);
    count_launch();
    const cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) rc = fail(WMPC_ERR_CUDA, "kernel launch failed: %s", cudaGetErrorString(err));
  }
  if (prev != plan->device) cudaSetDevice(prev);
  return rc;
}

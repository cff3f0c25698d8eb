// Batched fixed-pattern LDL^T factorization and triangular solves (sm_100a).
//
// One lane per instance.  The factorization is QDLDL's up-looking row
// algorithm driven by the host-built row program; the solve is permute ->
// forward substitution with L (column order) -> D^-1 -> backward
// substitution with L^T (reverse column order) -> unpermute, all in one
// launch.  Per-lane work vectors (the factorization's dense accumulator y,
// the solve's x) live in shared memory laid out [row][lane] (conflict-free)
// when they fit, otherwise in an HBM workspace laid out [row][instance].
//
// Operation order follows warpmpc/jax_qdldl/warp_backend.py:41-101 (factor)
// and 176-218 (serial solve) exactly; the file is compiled with -fmad=false
// so every product and sum is rounded separately, as in the reference's
// NumPy-restated order.
#include "common.cuh"
#include "qdldl.cuh"

namespace wmpc {

// ---------------------------------------------------------------------------
// factorization
// ---------------------------------------------------------------------------

template <bool kSmem>
__global__ void __launch_bounds__(256) factor_kernel(Pattern pat, const float* __restrict__ values,
                                                     long long ldv, int bstride, float* lx, float* d,
                                                     float* dinv, float* yglob, int batch, const int* only) {
  extern __shared__ float smem[];
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= batch || (only && !only[b])) return;
  LaneVec y = kSmem ? LaneVec{smem + threadIdx.x, (long long)blockDim.x}
                    : LaneVec{yglob + b, (long long)batch};
  const float* vb = values + (long long)b * bstride;
  auto val_at = [&](int slot) -> float { return vb[(long long)__ldg(pat.perm_to_orig + slot) * ldv]; };
  factor_instance(pat, val_at, y, lx, batch, d, dinv, batch, b);
}

// ---------------------------------------------------------------------------
// triangular solve
// ---------------------------------------------------------------------------

template <bool kSmem>
__global__ void __launch_bounds__(256) solve_kernel(Pattern pat, const float* __restrict__ lx,
                                                    const float* __restrict__ dinv, int fstride,
                                                    long long ldf, const float* rhs, float* out,
                                                    float* xglob, int batch) {
  extern __shared__ float smem[];
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= batch) return;
  LaneVec x = kSmem ? LaneVec{smem + threadIdx.x, (long long)blockDim.x}
                    : LaneVec{xglob + b, (long long)batch};
  const int n = pat.n;
  for (int i = 0; i < n; ++i) x(i) = rhs[(long long)__ldg(pat.p + i) * batch + b];
  const long long fo = (long long)b * fstride;
  ldl_solve_permuted(pat, lx + fo, ldf, dinv + fo, ldf, x);
  for (int i = 0; i < n; ++i) out[(long long)i * batch + b] = x(__ldg(pat.pinv + i));
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------

size_t factor_workspace_bytes(const Pattern& pat, int batch) {
  return smem_lanes_for_rows(pat.n) >= 32 ? 0 : (size_t)4 * pat.n * (size_t)batch;
}

size_t solve_workspace_bytes(const Pattern& pat, int batch) {
  return smem_lanes_for_rows(pat.n) >= 32 ? 0 : (size_t)4 * pat.n * (size_t)batch;
}

int launch_factor(const Pattern& pat, const float* values, long long ldv, int bstride, float* lx,
                  float* d, float* dinv, int batch, void* ws, size_t ws_bytes, cudaStream_t stream, const int* only) {
  if (batch <= 0) return WMPC_OK;
  const int lanes = smem_lanes_for_rows(pat.n);
  if (lanes >= 32) {
    const int threads = lanes < 128 ? lanes : 128;
    const size_t smem = (size_t)4 * pat.n * threads;
    WMPC_CUDA_TRY(cudaFuncSetAttribute(factor_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
    profile_mark_begin(stream, kProfileFactor);
    factor_kernel<true><<<ceil_div(batch, threads), threads, smem, stream>>>(pat, values, ldv, bstride, lx,
                                                                             d, dinv, nullptr, batch, only);
    profile_mark_end(stream, kProfileFactor);
  } else {
    const size_t need = factor_workspace_bytes(pat, batch);
    if (ws == nullptr || ws_bytes < need)
      return fail(WMPC_ERR_WORKSPACE, "factor needs %zu workspace bytes, got %zu", need, ws_bytes);
    profile_mark_begin(stream, kProfileFactor);
    factor_kernel<false><<<ceil_div(batch, 128), 128, 0, stream>>>(pat, values, ldv, bstride, lx, d, dinv,
                                                                  static_cast<float*>(ws), batch, only);
    profile_mark_end(stream, kProfileFactor);
  }
  WMPC_LAUNCH_CHECK();
  return WMPC_OK;
}

int launch_solve(const Pattern& pat, const float* lx, const float* dinv, int fstride, const float* rhs,
                 float* x, int batch, void* ws, size_t ws_bytes, cudaStream_t stream) {
  if (batch <= 0) return WMPC_OK;
  const long long ldf = fstride ? batch : 1;
  const int lanes = smem_lanes_for_rows(pat.n);
  if (lanes >= 32) {
    const int threads = lanes < 128 ? lanes : 128;
    const size_t smem = (size_t)4 * pat.n * threads;
    WMPC_CUDA_TRY(cudaFuncSetAttribute(solve_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
    solve_kernel<true><<<ceil_div(batch, threads), threads, smem, stream>>>(pat, lx, dinv, fstride, ldf, rhs,
                                                                            x, nullptr, batch);
  } else {
    const size_t need = solve_workspace_bytes(pat, batch);
    if (ws == nullptr || ws_bytes < need)
      return fail(WMPC_ERR_WORKSPACE, "solve needs %zu workspace bytes, got %zu", need, ws_bytes);
    solve_kernel<false><<<ceil_div(batch, 128), 128, 0, stream>>>(pat, lx, dinv, fstride, ldf, rhs, x,
                                                                 static_cast<float*>(ws), batch);
  }
  WMPC_LAUNCH_CHECK();
  return WMPC_OK;
}

}  // namespace wmpc

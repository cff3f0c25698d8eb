// y = S x - r for a batch of symmetric matrices with one pattern, S given by
// the values of its upper triangle (symbolic-major [nnz][batch]) and a row
// table of the full symmetric pattern: row i's terms are (value position,
// column) pairs, each upper entry (i, j) appearing in row i and, off the
// diagonal, in row j.  This is the refinement residual of the reference's
// adjoint solve (_adjoint_matvec, warpmpc/jax_osqp/solver.py:1035-1044, used
// at 1133-1141), in gather form: every row's sum is one thread's, no atomics.
// Lane = instance (coalesced [.][batch] rows); each instance is split over 4
// threads taking rows p, p + 4, ... (independent rows, latency-bound loop).
#include "common.cuh"

namespace wmpc {
namespace {

constexpr int kMvParts = 4;

__global__ void __launch_bounds__(32 * kMvParts) sym_matvec_kernel(const int* __restrict__ row_ptr,
                                                                   const int* __restrict__ ent_pos,
                                                                   const int* __restrict__ ent_col, int n,
                                                                   const float* __restrict__ values, long long ld,
                                                                   const float* __restrict__ x,
                                                                   const float* __restrict__ r,
                                                                   float* __restrict__ y, int batch) {
  const int b = blockIdx.x * 32 + threadIdx.x;
  if (b >= batch) return;
  for (int i = threadIdx.y; i < n; i += kMvParts) {
    float acc = 0.0f;
    const int t0 = __ldg(row_ptr + i), t1 = __ldg(row_ptr + i + 1);
    for (int t = t0; t < t1; ++t)
      acc = acc + values[(long long)__ldg(ent_pos + t) * ld + b] * x[(long long)__ldg(ent_col + t) * batch + b];
    const long long k = (long long)i * batch + b;
    y[k] = r ? acc - r[k] : acc;
  }
}

}  // namespace
}  // namespace wmpc

using namespace wmpc;

extern "C" int wmpc_sym_matvec(const int32_t* row_ptr, const int32_t* ent_pos, const int32_t* ent_col, int32_t n,
                               const float* values, int64_t values_ld, const float* x, const float* r, float* y,
                               int32_t batch, wmpc_stream_t stream) {
  if (n < 0 || batch < 0) return fail(WMPC_ERR_INVALID_ARGUMENT, "sym matvec: negative size");
  if (n == 0 || batch == 0) return WMPC_OK;
  if (!row_ptr || !ent_pos || !ent_col || !values || !x || !y)
    return fail(WMPC_ERR_INVALID_ARGUMENT, "sym matvec: null pointer");
  if (values_ld < batch) return fail(WMPC_ERR_INVALID_ARGUMENT, "sym matvec: values_ld below the batch");
  if (y == x) return fail(WMPC_ERR_INVALID_ARGUMENT, "sym matvec: y must not alias x");
  sym_matvec_kernel<<<(batch + 31) / 32, dim3(32, kMvParts), 0, static_cast<cudaStream_t>(stream)>>>(
      row_ptr, ent_pos, ent_col, n, values, values_ld, x, r, y, batch);
  WMPC_LAUNCH_CHECK();
  return WMPC_OK;
}

// Batched SQP QP assembly (warpmpc/jax_sqp/sparse_mpc.py:855-901, the
// scatter half of _linearize_jit): from each instance's packed stage values
// (per stage: cost, g, lower, upper, grad, hess, jac) form q, the P and A
// values, l = lower - g, u = upper - g, g, lower, upper and the total cost.
// Gather form: every output entry sums its sources (stage values that the
// reference scatter-adds into it) in stage order, starting from zero, so no
// atomics and a fixed float32 operation order.  One block per instance;
// threads stride over that instance's outputs (coalesced batch-major rows;
// the gathers hit the instance's packed row in L1).  Staging the row in
// shared memory first was measured slower (2.65 ms against 1.95 ms for the
// quadrotor N=30 stages at 65536 instances): fewer blocks fit per SM.
#include "common.cuh"

namespace wmpc {
namespace {

__global__ void __launch_bounds__(256) sqp_assemble_kernel(
    wmpc_sqp_assemble_dims d, const int* __restrict__ add_ptr, const int* __restrict__ add_src,
    const int* __restrict__ row_src, const int* __restrict__ cost_src, const float* __restrict__ values,
    float* __restrict__ q, float* __restrict__ p_values, float* __restrict__ a_values, float* __restrict__ l,
    float* __restrict__ u, float* __restrict__ cost, float* __restrict__ g, float* __restrict__ lower,
    float* __restrict__ upper) {
  for (int b = blockIdx.x; b < d.batch; b += gridDim.x) {
    const float* v = values + (size_t)b * d.width;
    const int n_add = d.n + d.nnz_p + d.nnz_a;
    for (int k = threadIdx.x; k < n_add; k += blockDim.x) {
      float acc = 0.0f;
      const int t1 = __ldg(add_ptr + k + 1);
      for (int t = __ldg(add_ptr + k); t < t1; ++t) acc = acc + v[__ldg(add_src + t)];
      if (k < d.n)
        q[(size_t)b * d.n + k] = acc;
      else if (k < d.n + d.nnz_p)
        p_values[(size_t)b * d.nnz_p + (k - d.n)] = acc;
      else
        a_values[(size_t)b * d.nnz_a + (k - d.n - d.nnz_p)] = acc;
    }
    for (int r = threadIdx.x; r < d.m; r += blockDim.x) {
      // row_src[r]: row r's g column; row_src[m + r]: its stage's
      // constraint_dim, the distance to the lower and then the upper column
      const int s = __ldg(row_src + r);
      const int nc = __ldg(row_src + d.m + r);
      const float gv = v[s], lo = v[s + nc], up = v[s + 2 * nc];
      const size_t o = (size_t)b * d.m + r;
      g[o] = gv;
      lower[o] = lo;
      upper[o] = up;
      l[o] = lo - gv;
      u[o] = up - gv;
    }
    if (threadIdx.x == 0) {
      float c = 0.0f;
      for (int s = 0; s < d.n_stages; ++s) c = c + v[__ldg(cost_src + s)];
      cost[b] = c;
    }
  }
}

}  // namespace
}  // namespace wmpc

using namespace wmpc;

extern "C" int wmpc_sqp_assemble(const wmpc_sqp_assemble_dims* dims, const int32_t* add_ptr, const int32_t* add_src,
                                 const int32_t* row_src, const int32_t* cost_src, const float* values, float* q,
                                 float* p_values, float* a_values, float* l, float* u, float* cost, float* g,
                                 float* constraint_l, float* constraint_u, wmpc_stream_t stream) {
  if (!dims) return fail(WMPC_ERR_INVALID_ARGUMENT, "sqp assemble: null dims");
  const wmpc_sqp_assemble_dims d = *dims;
  if (d.batch < 0 || d.n < 0 || d.nnz_p < 0 || d.nnz_a < 0 || d.m < 0 || d.n_stages < 0 || d.width < 0)
    return fail(WMPC_ERR_INVALID_ARGUMENT, "sqp assemble: negative size");
  if (d.batch == 0) return WMPC_OK;
  if (!add_ptr || !values || !cost || !cost_src || (d.n + d.nnz_p + d.nnz_a > 0 && !add_src) ||
      (d.n > 0 && !q) || (d.nnz_p > 0 && !p_values) || (d.nnz_a > 0 && !a_values) ||
      (d.m > 0 && (!row_src || !l || !u || !g || !constraint_l || !constraint_u)))
    return fail(WMPC_ERR_INVALID_ARGUMENT, "sqp assemble: null pointer");
  const int grid = d.batch < 65536 ? d.batch : 65536;
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  profile_mark_begin(s);
  sqp_assemble_kernel<<<grid, 256, 0, s>>>(d, add_ptr, add_src, row_src, cost_src, values, q, p_values, a_values, l,
                                           u, cost, g, constraint_l, constraint_u);
  profile_mark_end(s);
  WMPC_LAUNCH_CHECK();
  return WMPC_OK;
}

// Device building blocks of the batched LDL^T path, shared by the per-call
// kernels (qdldl.cu) and the fused OSQP kernels (osqp.cu).
#pragma once

#include <vector>

#include "common.cuh"

namespace wmpc {

// Row loop of the numeric factorization for one instance.  `val_at(slot)`
// returns the permuted-KKT value in permuted slot `slot` for this instance.
template <typename ValueAt>
__device__ __forceinline__ void factor_instance(const Pattern& pat, ValueAt val_at, const LaneVec& y,
                                                float* __restrict__ lx, long long ldl,
                                                float* __restrict__ d, float* __restrict__ dinv,
                                                long long ldd, int b) {
  const int n = pat.n;
  for (int row = 0; row < n; ++row) y(row) = 0.0f;
  for (int k = 0; k < n; ++k) {
    float dk = val_at(__ldg(pat.diag_pos + k));
    const int i0 = __ldg(pat.init_ptr + k), i1 = __ldg(pat.init_ptr + k + 1);
    for (int e = i0; e < i1; ++e) {
      const int row = __ldg(pat.init_rows + e);
      y(row) = y(row) + val_at(__ldg(pat.init_pos + e));
    }
    const int p0 = __ldg(pat.proc_ptr + k), p1 = __ldg(pat.proc_ptr + k + 1);
    for (int e = p0; e < p1; ++e) {
      const int cidx = __ldg(pat.proc_cols + e);
      const int dest = __ldg(pat.proc_lidx + e);
      const int off = __ldg(pat.proc_offsets + e);
      const float val = y(cidx);
      const int base = __ldg(pat.lp + cidx);
      for (int q = 0; q < off; ++q) {
        const int r = __ldg(pat.li + base + q);
        y(r) = y(r) - lx[(long long)(base + q) * ldl + b] * val;
      }
      const float lval = val * dinv[(long long)cidx * ldd + b];
      lx[(long long)dest * ldl + b] = lval;
      dk = dk - val * lval;
    }
    d[(long long)k * ldd + b] = dk;
    dinv[(long long)k * ldd + b] = 1.0f / dk;
    for (int e = p0; e < p1; ++e) y(__ldg(pat.proc_cols + e)) = 0.0f;
  }
}

// x = L^-T (D^-1 (L^-1 x)) in the permuted space, in place on `x`.
__device__ __forceinline__ void ldl_solve_permuted(const Pattern& pat, const float* __restrict__ lx,
                                                   long long ldl, const float* __restrict__ dinv,
                                                   long long ldd, const LaneVec& x) {
  const int n = pat.n;
  for (int col = 0; col < n; ++col) {
    const int e0 = __ldg(pat.lp + col), e1 = __ldg(pat.lp + col + 1);
    if (e0 == e1) continue;
    const float val = x(col);
    for (int e = e0; e < e1; ++e) {
      const int r = __ldg(pat.li + e);
      x(r) = x(r) - lx[(long long)e * ldl] * val;
    }
  }
  for (int i = 0; i < n; ++i) x(i) = x(i) * dinv[(long long)i * ldd];
  for (int col = n - 1; col >= 0; --col) {
    const int e0 = __ldg(pat.lp + col), e1 = __ldg(pat.lp + col + 1);
    float corr = 0.0f;
    for (int e = e0; e < e1; ++e) corr = corr + lx[(long long)e * ldl] * x(__ldg(pat.li + e));
    x(col) = x(col) - corr;
  }
}

bool build_solve_tables(int n, const std::vector<int>& lp, const std::vector<int>& li, std::vector<int>* tables,
                        std::vector<int>* desc);
size_t factor_workspace_bytes(const Pattern& pat, int batch);
size_t solve_workspace_bytes(const Pattern& pat, int batch);
// only (optional, [batch]): factor just the instances marked nonzero
int launch_factor(const Pattern& pat, const float* values, long long ldv, int bstride, float* lx,
                  float* d, float* dinv, int batch, void* ws, size_t ws_bytes, cudaStream_t stream,
                  const int* only = nullptr);
// The per-call factorization of a plan: the staged kernel where the plan has
// its tables (and its shared memory fits), else the one-lane kernel (same bits).
int launch_factor_plan(const wmpc_plan& plan, const float* values, long long ldv, int bstride, float* lx, float* d,
                       float* dinv, int batch, void* ws, size_t ws_bytes, cudaStream_t stream,
                       const int* only = nullptr);
int launch_solve(const Pattern& pat, const float* lx, const float* dinv, int fstride, const float* rhs,
                 float* x, int batch, void* ws, size_t ws_bytes, cudaStream_t stream);
int launch_solve_stream(const wmpc_plan& plan, const float* lx, const float* dinv, int fstride, const float* rhs,
                        float* x, int batch, cudaStream_t s, bool* applied);
// The per-call solve of a plan: the TMA-fed kernel where it applies, else the
// one-lane-per-instance kernel (same results bit for bit).
inline int launch_solve_plan(const wmpc_plan& plan, const float* lx, const float* dinv, int fstride,
                             const float* rhs, float* x, int batch, void* ws, size_t ws_bytes, cudaStream_t stream) {
  bool applied = false;
  const int rc = launch_solve_stream(plan, lx, dinv, fstride, rhs, x, batch, stream, &applied);
  if (rc || applied) return rc;
  return launch_solve(plan.pat, lx, dinv, fstride, rhs, x, batch, ws, ws_bytes, stream);
}

}  // namespace wmpc

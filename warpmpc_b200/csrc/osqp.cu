// Batched fixed-pattern OSQP-ADMM (sm_100a): layout transposes, KKT
// assembly, the per-call ("plain") ADMM loop pieces, the fused persistent
// solve, and the residual epilogue.
//
// Arithmetic follows warpmpc/jax_osqp/solver.py operation by operation
// (assemble_kkt_values 764-776, _iterate 806-820, scaling/unscaling 842-865,
// residuals 866-871); -fmad=false keeps every product and sum separately
// rounded.
#include "common.cuh"
#include <vector>

#include "osqp.cuh"
#include "qdldl.cuh"

namespace wmpc {

// ---------------------------------------------------------------------------
// layout transposes (batch-major API <-> symbolic-major kernels)
// ---------------------------------------------------------------------------

// dst[j, b] = src[b, j] * scale[j]   (scale may be null)
__global__ void transpose_in_kernel(const float* __restrict__ src, long long lds, int rows, int cols,
                                    const float* __restrict__ scale, float* __restrict__ dst, long long ldd) {
  __shared__ float tile[32][33];
  const int j0 = blockIdx.x * 32, b0 = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int b = b0 + k, j = j0 + threadIdx.x;
    if (b < rows && j < cols) tile[k][threadIdx.x] = src[(long long)b * lds + j];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int j = j0 + k, b = b0 + threadIdx.x;
    if (b < rows && j < cols) {
      float v = tile[threadIdx.x][k];
      if (scale) v = v * scale[j];
      dst[(long long)j * ldd + b] = v;
    }
  }
}

// dst[b, j] = src[j, b]
__global__ void transpose_out_kernel(const float* __restrict__ src, long long lds, int rows, int cols,
                                     float* __restrict__ dst, long long ldd) {
  __shared__ float tile[32][33];
  const int j0 = blockIdx.y * 32, b0 = blockIdx.x * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int j = j0 + k, b = b0 + threadIdx.x;
    if (b < rows && j < cols) tile[k][threadIdx.x] = src[(long long)j * lds + b];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int b = b0 + k, j = j0 + threadIdx.x;
    if (b < rows && j < cols) dst[(long long)b * ldd + j] = tile[threadIdx.x][k];
  }
}

static int transpose_in(const float* src, long long lds, int rows, int cols, const float* scale, float* dst,
                        long long ldd, cudaStream_t s) {
  if (rows <= 0 || cols <= 0) return WMPC_OK;
  dim3 grid(ceil_div(cols, 32), ceil_div(rows, 32));
  transpose_in_kernel<<<grid, dim3(32, 8), 0, s>>>(src, lds, rows, cols, scale, dst, ldd);
  WMPC_LAUNCH_CHECK();
  return WMPC_OK;
}

static int transpose_out(const float* src, long long lds, int rows, int cols, float* dst, long long ldd,
                         cudaStream_t s) {
  if (rows <= 0 || cols <= 0) return WMPC_OK;
  dim3 grid(ceil_div(rows, 32), ceil_div(cols, 32));
  transpose_out_kernel<<<grid, dim3(32, 8), 0, s>>>(src, lds, rows, cols, dst, ldd);
  WMPC_LAUNCH_CHECK();
  return WMPC_OK;
}

// ---------------------------------------------------------------------------
// per-instance views of the problem data (symbolic-major)
// ---------------------------------------------------------------------------

struct InstanceData {
  const float* pT;  // P values of this instance: pT[j * ldp]
  long long ldp;
  const float* aT;
  long long lda;
  __device__ __forceinline__ float p(int j) const { return pT[(long long)j * ldp]; }
  __device__ __forceinline__ float a(int j) const { return aT[(long long)j * lda]; }
};

// KKT value of original KKT slot s (solver.py:764-776).
__device__ __forceinline__ float kkt_value(const Osqp& o, const InstanceData& in, int s) {
  const int src = __ldg(o.kkt_src + s);
  if (src < 0) return __ldg(o.kkt_base + s);
  if (src < o.nnz_p) return in.p(src) * __ldg(o.p_scale + src) + __ldg(o.p_diag_sigma + src);
  const int j = src - o.nnz_p;
  return in.a(j) * __ldg(o.a_scale + j);
}

__global__ void assemble_kkt_kernel(Osqp o, const float* __restrict__ pT, long long ldp, int sbp,
                                    const float* __restrict__ aT, long long lda, int sba, float* __restrict__ kkt,
                                    int batch) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= batch) return;
  InstanceData in{pT + (long long)b * sbp, ldp, aT + (long long)b * sba, lda};
  for (int s = blockIdx.y; s < o.nnz_kkt; s += gridDim.y) kkt[(long long)s * batch + b] = kkt_value(o, in, s);
}

// ---------------------------------------------------------------------------
// ADMM pieces (scaled space, symbolic-major state)
// ---------------------------------------------------------------------------

struct State {
  float* x;  // [n, batch]
  float* z;  // [m, batch]
  float* y;  // [m, batch]
  const float* qs;  // scaled q [n, batch]
  const float* ls;  // scaled l [m, batch]
  const float* us;  // scaled u [m, batch]
  long long ld;     // = batch
};

__device__ __forceinline__ float clip_nan(float v, float lo, float hi) {
  // jnp.minimum(jnp.maximum(v, lo), hi) with NaN propagation
  float t = (v < lo) ? lo : v;
  return (t > hi) ? hi : t;
}

// Per-(constraint, instance) rho and 1/rho ([m][batch]) when rho adapts per
// instance; null pointers: the plan's vector.
struct RhoRows {
  const float* rho = nullptr;
  const float* rinv = nullptr;
};

__device__ __forceinline__ float rho_at(const Osqp& o, const RhoRows& rr, int r, long long k) {
  return rr.rho ? rr.rho[k] : __ldg(o.rho + r);
}
__device__ __forceinline__ float rinv_at(const Osqp& o, const RhoRows& rr, int r, long long k) {
  return rr.rinv ? rr.rinv[k] : __ldg(o.rho_inv + r);
}

// rhs entry of KKT index `orig` (original, un-permuted numbering)
__device__ __forceinline__ float rhs_entry(const Osqp& o, const State& st, int orig, int b, const RhoRows& rr = {}) {
  if (orig < o.n) {
    const long long k = (long long)orig * st.ld + b;
    return o.sigma * st.x[k] - st.qs[k];
  }
  const int r = orig - o.n;
  const long long k = (long long)r * st.ld + b;
  return st.z[k] - rinv_at(o, rr, r, k) * st.y[k];
}

// ADMM update of KKT index `orig` given the solve output `sol`
// (solver.py:813-819); returns the next iteration's rhs entry.
__device__ __forceinline__ float admm_update(const Osqp& o, const State& st, int orig, int b, float sol,
                                             const RhoRows& rr = {}) {
  if (orig < o.n) {
    const long long k = (long long)orig * st.ld + b;
    const float x = st.x[k];
    const float xn = o.alpha * sol + o.one_minus_alpha * x;
    st.x[k] = xn;
    return o.sigma * xn - st.qs[k];
  }
  const int r = orig - o.n;
  const long long k = (long long)r * st.ld + b;
  const float rinv = rinv_at(o, rr, r, k);
  const float z = st.z[k], y = st.y[k];
  const float rz = z - rinv * y;
  const float zt = rz + rinv * sol;
  const float zr = o.alpha * zt + o.one_minus_alpha * z;
  const float zn = clip_nan(zr + rinv * y, st.ls[k], st.us[k]);
  const float yn = y + rho_at(o, rr, r, k) * (zr - zn);
  st.z[k] = zn;
  st.y[k] = yn;
  return zn - rinv * yn;
}

__global__ void admm_first_rhs_kernel(Osqp o, State st, float* __restrict__ rhs, int batch, RhoRows rr) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= batch) return;
  for (int i = blockIdx.y; i < o.nk; i += gridDim.y) rhs[(long long)i * batch + b] = rhs_entry(o, st, i, b, rr);
}

__global__ void admm_update_kernel(Osqp o, State st, float* __restrict__ rhs, int batch, RhoRows rr) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= batch) return;
  for (int i = blockIdx.y; i < o.nk; i += gridDim.y) {
    const long long k = (long long)i * batch + b;
    rhs[k] = admm_update(o, st, i, b, rhs[k], rr);
  }
}

// ---------------------------------------------------------------------------
// rho adaptation (per instance, plain mode).  No counterpart in the reference
// (solver.py:587-588 rejects adaptive_rho); the rule is OSQP's (Stellato et
// al. 2020, "OSQP: an operator splitting solver for quadratic programs",
// sec. 5.2), on the scaled iterate:
//   r_p = |A x - z|_inf / (max(|A x|_inf, |z|_inf) + 1e-10)
//   r_d = |P x + q + A^T y|_inf / (max(|P x|_inf, |A^T y|_inf, |q|_inf) + 1e-10)
//   rho' = clamp(rho sqrt(r_p / (r_d + 1e-10)), 1e-6, 1e6)
// taken when rho' > tol rho or rho' < rho / tol; the rho vector then follows
// the plan's classes (loose rows 1e-6, equality rows 1e3 rho', others rho')
// and 1/rho is one float32 division per row.  Sums run in the oracle's order
// (A x and P x by rows, A^T y by columns, entries in storage order).
// ---------------------------------------------------------------------------

__global__ void rho_init_kernel(Osqp o, float* __restrict__ rho_row, float* __restrict__ rinv_row,
                                float* __restrict__ rho_b, int* __restrict__ count, int batch) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= batch) return;
  for (int r = blockIdx.y; r < o.m; r += gridDim.y) {
    const long long k = (long long)r * batch + b;
    rho_row[k] = __ldg(o.rho + r);
    rinv_row[k] = __ldg(o.rho_inv + r);
  }
  if (blockIdx.y == 0) {
    rho_b[b] = o.rho0;
    count[b] = 0;
  }
}

__global__ void __launch_bounds__(128) rho_update_kernel(Osqp o, const float* __restrict__ pT, long long ldp, int sbp,
                                                         const float* __restrict__ aT, long long lda, int sba, State st,
                                                         float* __restrict__ rho_row, float* __restrict__ rinv_row,
                                                         float* __restrict__ rho_b, int* __restrict__ changed,
                                                         int* __restrict__ count, float tol, int batch) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= batch) return;
  InstanceData in{pT + (long long)b * sbp, ldp, aT + (long long)b * sba, lda};
  auto xs = [&](int j) { return st.x[(long long)j * st.ld + b]; };
  auto as = [&](int e) { return in.a(e) * __ldg(o.a_scale + e); };
  float prim = 0.f, axn = 0.f, zn = 0.f;
  for (int row = 0; row < o.m; ++row) {
    float ax = 0.0f;
    const int e0 = __ldg(o.a_row_ptr + row), e1 = __ldg(o.a_row_ptr + row + 1);
    for (int t = e0; t < e1; ++t) {
      const int e = __ldg(o.a_row_ent + t);
      ax = ax + as(e) * xs(__ldg(o.a_cols + e));
    }
    const float z = st.z[(long long)row * st.ld + b];
    prim = fmaxf(prim, fabsf(ax - z));
    axn = fmaxf(axn, fabsf(ax));
    zn = fmaxf(zn, fabsf(z));
  }
  float dual = 0.f, pxn = 0.f, atyn = 0.f, qn = 0.f;
  for (int j = 0; j < o.n; ++j) {
    float px = 0.0f;
    const int f0 = __ldg(o.pf_row_ptr + j), f1 = __ldg(o.pf_row_ptr + j + 1);
    for (int t = f0; t < f1; ++t) {
      const int v = __ldg(o.pf_val + t);
      px = px + (in.p(v) * __ldg(o.p_scale + v)) * xs(__ldg(o.pf_col + t));
    }
    float aty = 0.0f;
    const int c0 = __ldg(o.a_col_ptr + j), c1 = __ldg(o.a_col_ptr + j + 1);
    for (int e = c0; e < c1; ++e) aty = aty + as(e) * st.y[(long long)__ldg(o.a_rows + e) * st.ld + b];
    const float qj = st.qs[(long long)j * st.ld + b];
    dual = fmaxf(dual, fabsf(px + qj + aty));
    pxn = fmaxf(pxn, fabsf(px));
    atyn = fmaxf(atyn, fabsf(aty));
    qn = fmaxf(qn, fabsf(qj));
  }
  const float rp = prim / (fmaxf(axn, zn) + 1e-10f);
  const float rd = dual / (fmaxf(fmaxf(pxn, atyn), qn) + 1e-10f);
  const float rho = rho_b[b];
  float est = rho * sqrtf(rp / (rd + 1e-10f));
  est = fminf(fmaxf(est, 1e-6f), 1e6f);
  const bool take = est > rho * tol || est < rho / tol;
  changed[b] = take ? 1 : 0;
  if (!take) return;
  rho_b[b] = est;
  count[b] += 1;
  for (int r = 0; r < o.m; ++r) {
    const int t = __ldg(o.rho_type + r);
    const float v = t < 0 ? 1e-6f : (t > 0 ? 1e3f * est : est);
    const long long k = (long long)r * batch + b;
    rho_row[k] = v;
    rinv_row[k] = 1.0f / v;
  }
}

// The rho outputs of a plain-mode solve: each instance's final rho and rho
// changes (without adaptation: the plan's rho and 0).
__global__ void rho_report_kernel(const float* __restrict__ rho_b, const int* __restrict__ count, float rho0,
                                  float* __restrict__ rho_out, int* __restrict__ count_out, int batch) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= batch) return;
  if (rho_out) rho_out[b] = rho_b ? rho_b[b] : rho0;
  if (count_out) count_out[b] = count ? count[b] : 0;
}

// KKT values with each instance's own -1/rho entries (only the instances
// marked in `only`, when given).
__global__ void assemble_kkt_rho_kernel(Osqp o, const float* __restrict__ pT, long long ldp, int sbp,
                                        const float* __restrict__ aT, long long lda, int sba,
                                        const float* __restrict__ rinv_row, const int* __restrict__ only,
                                        float* __restrict__ kkt, int batch) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= batch || (only && !only[b])) return;
  InstanceData in{pT + (long long)b * sbp, ldp, aT + (long long)b * sba, lda};
  for (int s = blockIdx.y; s < o.nnz_kkt; s += gridDim.y) {
    const int r = __ldg(o.kkt_rho_row + s);
    kkt[(long long)s * batch + b] = r >= 0 ? -rinv_row[(long long)r * batch + b] : kkt_value(o, in, s);
  }
}

// ---------------------------------------------------------------------------
// residuals (solver.py:863-871) -- unscaled, one lane per instance
// ---------------------------------------------------------------------------

struct Residuals {
  float prim, dual, obj;
  float ax_norm, z_norm, px_norm, aty_norm, q_norm;
};

// The objective's sums run in kResParts interleaved partial sums (column j
// into part j % kResParts), added in part order: the split residual_kernel
// and this one-thread form give the same bits.
constexpr int kResParts = 8;  // threads per instance in residual_kernel

// q is the unscaled linear term: q[j * ldq]
__device__ Residuals residuals(const Osqp& o, const InstanceData& in, const State& st, int b,
                               const float* __restrict__ q, long long ldq) {
  Residuals r{0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  auto xu = [&](int j) { return st.x[(long long)j * st.ld + b] * __ldg(o.scaling_d + j); };
  for (int row = 0; row < o.m; ++row) {
    float ax = 0.0f;
    const int e0 = __ldg(o.a_row_ptr + row), e1 = __ldg(o.a_row_ptr + row + 1);
    for (int t = e0; t < e1; ++t) {
      const int e = __ldg(o.a_row_ent + t);
      ax = ax + in.a(e) * xu(__ldg(o.a_cols + e));
    }
    const float zu = st.z[(long long)row * st.ld + b] * __ldg(o.scaling_einv + row);
    r.prim = fmaxf(r.prim, fabsf(ax - zu));
    r.ax_norm = fmaxf(r.ax_norm, fabsf(ax));
    r.z_norm = fmaxf(r.z_norm, fabsf(zu));
  }
  float quad_p[kResParts], lin_p[kResParts];
#pragma unroll
  for (int p = 0; p < kResParts; ++p) quad_p[p] = lin_p[p] = 0.0f;
  for (int j0 = 0; j0 < o.n; j0 += kResParts)
#pragma unroll
   for (int p = 0; p < kResParts; ++p) {
    const int j = j0 + p;
    if (j >= o.n) break;
    float px = 0.0f;
    const int f0 = __ldg(o.pf_row_ptr + j), f1 = __ldg(o.pf_row_ptr + j + 1);
    for (int t = f0; t < f1; ++t) px = px + in.p(__ldg(o.pf_val + t)) * xu(__ldg(o.pf_col + t));
    float aty = 0.0f;
    const int c0 = __ldg(o.a_col_ptr + j), c1 = __ldg(o.a_col_ptr + j + 1);
    for (int e = c0; e < c1; ++e) {
      const int row = __ldg(o.a_rows + e);
      aty = aty + in.a(e) * (st.y[(long long)row * st.ld + b] * __ldg(o.y_unscale + row));
    }
    const float qj = q[(long long)j * ldq];
    const float xj = xu(j);
    r.dual = fmaxf(r.dual, fabsf(px + qj + aty));
    r.px_norm = fmaxf(r.px_norm, fabsf(px));
    r.aty_norm = fmaxf(r.aty_norm, fabsf(aty));
    r.q_norm = fmaxf(r.q_norm, fabsf(qj));
    quad_p[p] = quad_p[p] + xj * px;
    lin_p[p] = lin_p[p] + qj * xj;
  }
  float quad = 0.0f, lin = 0.0f;
#pragma unroll
  for (int p = 0; p < kResParts; ++p) {
    quad = quad + quad_p[p];
    lin = lin + lin_p[p];
  }
  r.obj = 0.5f * quad + lin;
  return r;
}

__device__ __forceinline__ void unscale_in_place(const Osqp& o, const State& st, int b) {
  for (int j = 0; j < o.n; ++j) {
    const long long k = (long long)j * st.ld + b;
    st.x[k] = st.x[k] * __ldg(o.scaling_d + j);
  }
  for (int r = 0; r < o.m; ++r) {
    const long long k = (long long)r * st.ld + b;
    st.z[k] = st.z[k] * __ldg(o.scaling_einv + r);
    st.y[k] = st.y[k] * __ldg(o.y_unscale + r);
  }
}

__device__ __forceinline__ bool finite_res(const Residuals& r) {
  return isfinite(r.prim) && isfinite(r.dual) && isfinite(r.obj);
}

// Exact residuals of the final iterate (residuals() above), status,
// unscaling.  eps_abs >= 0: also set SOLVED when OSQP's termination test
// holds (solves run with termination).  Each instance is split over
// kResParts threads (blockDim (32, kResParts): lane = instance, y = part):
// part p takes A's rows and the columns j = p, p + kResParts, ...; every
// row's and column's sum is still formed by one thread in the reference's
// order, so prim, dual and the norms (maxima) equal residuals()' exactly; the
// objective's two sums are added part by part.  Eight times the warps in
// flight for a latency-bound loop of dependent index and value loads.
__global__ void __launch_bounds__(32 * kResParts) residual_kernel(
    Osqp o, const float* __restrict__ pT, long long ldp, int sbp, const float* __restrict__ aT, long long lda,
    int sba, State st, const float* __restrict__ qT, float* prim, float* dual, float* obj, int* status, int batch,
    const int* status_in, const int* abort_word, float eps_abs, float eps_rel) {
  __shared__ float part_val[kResParts][9][32];
  const int lane = threadIdx.x, part = threadIdx.y;
  const int b = blockIdx.x * 32 + lane;
  const bool active = b < batch;
  if (active) {
    InstanceData in{pT + (long long)b * sbp, ldp, aT + (long long)b * sba, lda};
    auto xu = [&](int j) { return st.x[(long long)j * st.ld + b] * __ldg(o.scaling_d + j); };
    float rp = 0.f, axn = 0.f, zn = 0.f;
    for (int row = part; row < o.m; row += kResParts) {
      float ax = 0.0f;
      const int e0 = __ldg(o.a_row_ptr + row), e1 = __ldg(o.a_row_ptr + row + 1);
#pragma unroll 4
      for (int t = e0; t < e1; ++t) {
        const int e = __ldg(o.a_row_ent + t);
        ax = ax + in.a(e) * xu(__ldg(o.a_cols + e));
      }
      const float zu = st.z[(long long)row * st.ld + b] * __ldg(o.scaling_einv + row);
      rp = fmaxf(rp, fabsf(ax - zu));
      axn = fmaxf(axn, fabsf(ax));
      zn = fmaxf(zn, fabsf(zu));
    }
    float rd = 0.f, pxn = 0.f, atyn = 0.f, qn = 0.f, quad = 0.f, lin = 0.f;
    for (int j = part; j < o.n; j += kResParts) {
      float px = 0.0f;
      const int f0 = __ldg(o.pf_row_ptr + j), f1 = __ldg(o.pf_row_ptr + j + 1);
#pragma unroll 4
      for (int t = f0; t < f1; ++t) px = px + in.p(__ldg(o.pf_val + t)) * xu(__ldg(o.pf_col + t));
      float aty = 0.0f;
      const int c0 = __ldg(o.a_col_ptr + j), c1 = __ldg(o.a_col_ptr + j + 1);
#pragma unroll 4
      for (int e = c0; e < c1; ++e) {
        const int row = __ldg(o.a_rows + e);
        aty = aty + in.a(e) * (st.y[(long long)row * st.ld + b] * __ldg(o.y_unscale + row));
      }
      const float qj = qT[(long long)j * batch + b];
      const float xj = xu(j);
      rd = fmaxf(rd, fabsf(px + qj + aty));
      pxn = fmaxf(pxn, fabsf(px));
      atyn = fmaxf(atyn, fabsf(aty));
      qn = fmaxf(qn, fabsf(qj));
      quad = quad + xj * px;
      lin = lin + qj * xj;
    }
    const float v[9] = {rp, axn, zn, rd, pxn, atyn, qn, quad, lin};
#pragma unroll
    for (int k = 0; k < 9; ++k) part_val[part][k][lane] = v[k];
  }
  __syncthreads();  // every part has read the scaled iterate before any part unscales it
  if (active && part == 0) {
    Residuals r{0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    float quad = 0.f, lin = 0.f;
    for (int q = 0; q < kResParts; ++q) {
      r.prim = fmaxf(r.prim, part_val[q][0][lane]);
      r.ax_norm = fmaxf(r.ax_norm, part_val[q][1][lane]);
      r.z_norm = fmaxf(r.z_norm, part_val[q][2][lane]);
      r.dual = fmaxf(r.dual, part_val[q][3][lane]);
      r.px_norm = fmaxf(r.px_norm, part_val[q][4][lane]);
      r.aty_norm = fmaxf(r.aty_norm, part_val[q][5][lane]);
      r.q_norm = fmaxf(r.q_norm, part_val[q][6][lane]);
      quad = quad + part_val[q][7][lane];
      lin = lin + part_val[q][8][lane];
    }
    r.obj = 0.5f * quad + lin;
    prim[b] = r.prim;
    dual[b] = r.dual;
    obj[b] = r.obj;
    if (status) {
      int v = finite_res(r) ? WMPC_STATUS_MAX_ITER : WMPC_STATUS_NONFINITE;
      if (eps_abs >= 0.0f && finite_res(r)) {
        const float eps_p = eps_abs + eps_rel * fmaxf(r.ax_norm, r.z_norm);
        const float eps_d = eps_abs + eps_rel * fmaxf(fmaxf(r.px_norm, r.aty_norm), r.q_norm);
        if (r.prim <= eps_p && r.dual <= eps_d) v |= WMPC_STATUS_SOLVED;
      }
      if (status_in) v |= status_in[b];
      if (abort_word && *abort_word) v |= WMPC_STATUS_KERNEL_ABORT;
      status[b] = v;
    }
  }
  if (!active) return;
  for (int j = part; j < o.n; j += kResParts) {
    const long long k = (long long)j * st.ld + b;
    st.x[k] = st.x[k] * __ldg(o.scaling_d + j);
  }
  for (int r = part; r < o.m; r += kResParts) {
    const long long k = (long long)r * st.ld + b;
    st.z[k] = st.z[k] * __ldg(o.scaling_einv + r);
    st.y[k] = st.y[k] * __ldg(o.y_unscale + r);
  }
}

// The final iterate's unscaling alone (no residual outputs requested): x,
// z, y back to the problem's units and the status from the kernels' words.
__global__ void __launch_bounds__(32 * kResParts) unscale_state_kernel(Osqp o, State st, int* status,
                                                                     const int* status_in, const int* abort_word,
                                                                     int batch) {
  const int lane = threadIdx.x, part = threadIdx.y;
  const int b = blockIdx.x * 32 + lane;
  if (b >= batch) return;
  for (int j = part; j < o.n; j += kResParts) {
    const long long k = (long long)j * st.ld + b;
    st.x[k] = st.x[k] * __ldg(o.scaling_d + j);
  }
  for (int r = part; r < o.m; r += kResParts) {
    const long long k = (long long)r * st.ld + b;
    st.z[k] = st.z[k] * __ldg(o.scaling_einv + r);
    st.y[k] = st.y[k] * __ldg(o.y_unscale + r);
  }
  if (status && part == 0) {
    int v = WMPC_STATUS_MAX_ITER;
    if (status_in) v |= status_in[b];
    if (abort_word && *abort_word) v |= WMPC_STATUS_KERNEL_ABORT;
    status[b] = v;
  }
}

__global__ void fill_int_kernel(int* out, int value, int count) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) out[i] = value;
}

// ---------------------------------------------------------------------------
// persistent fused solve: assembly + factor + all iterations + epilogue
// ---------------------------------------------------------------------------

struct PersistentArgs {
  Pattern pat;
  Osqp o;
  const float* pT; long long ldp; int sbp;
  const float* aT; long long lda; int sba;
  const float* qT;  // unscaled q [n, batch]
  State st;
  float* lx;    // [nnz_l, fld] factor (written here when fused_factor)
  float* dinv;  // [nk, fld]
  float* d;     // [nk, fld] (fused_factor only)
  int fstride;  // 0: one factor shared by all instances, 1: per instance
  long long fld;
  int fused_factor;
  float* wglob; // [nk, batch] when the work vector does not fit in shared memory
  float* prim; float* dual; float* obj;
  int* iters; int* status;
  int batch, max_iter, check_every;
  float eps_abs, eps_rel;
};

template <bool kSmem>
__global__ void __launch_bounds__(256) persistent_kernel(PersistentArgs a) {
  extern __shared__ float smem[];
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= a.batch) return;
  const Pattern& pat = a.pat;
  const Osqp& o = a.o;
  LaneVec w = kSmem ? LaneVec{smem + threadIdx.x, (long long)blockDim.x}
                    : LaneVec{a.wglob + b, (long long)a.batch};
  InstanceData in{a.pT + (long long)b * a.sbp, a.ldp, a.aT + (long long)b * a.sba, a.lda};
  if (a.fused_factor) {
    auto val_at = [&](int slot) -> float { return kkt_value(o, in, __ldg(pat.perm_to_orig + slot)); };
    factor_instance(pat, val_at, w, a.lx, a.fld, a.d, a.dinv, a.fld, b);
  }
  const long long fo = (long long)b * a.fstride;
  const float* lx = a.lx + fo;
  const float* dinv = a.dinv + fo;

  int status = WMPC_STATUS_MAX_ITER;
  for (int k = 0; k < pat.n; ++k) {
    const float di = dinv[(long long)k * a.fld];
    if (di == 0.0f || !isfinite(di)) status |= WMPC_STATUS_ZERO_PIVOT;
  }
  int it = 0;
  for (; it < a.max_iter; ++it) {
    for (int i = 0; i < pat.n; ++i) w(i) = rhs_entry(o, a.st, __ldg(pat.p + i), b);
    ldl_solve_permuted(pat, lx, a.fld, dinv, a.fld, w);
    for (int i = 0; i < pat.n; ++i) admm_update(o, a.st, __ldg(pat.p + i), b, w(i));
    if (a.check_every > 0 && ((it + 1) % a.check_every == 0) && it + 1 < a.max_iter) {
      const Residuals r = residuals(o, in, a.st, b, a.qT + b, a.batch);
      if (!finite_res(r)) { status |= WMPC_STATUS_NONFINITE; ++it; break; }
      const float eps_p = a.eps_abs + a.eps_rel * fmaxf(r.ax_norm, r.z_norm);
      const float eps_d = a.eps_abs + a.eps_rel * fmaxf(fmaxf(r.px_norm, r.aty_norm), r.q_norm);
      if (r.prim <= eps_p && r.dual <= eps_d) { status |= WMPC_STATUS_SOLVED; ++it; break; }
    }
  }
  const Residuals r = residuals(o, in, a.st, b, a.qT + b, a.batch);
  a.prim[b] = r.prim;
  a.dual[b] = r.dual;
  a.obj[b] = r.obj;
  if (!finite_res(r)) status |= WMPC_STATUS_NONFINITE;
  if (a.iters) a.iters[b] = it;
  if (a.status) a.status[b] = status;
  unscale_in_place(o, a.st, b);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

namespace {

struct Carve {
  char* base;
  size_t used = 0;
  float* take(size_t floats) {
    size_t bytes = ((floats * 4 + 255) / 256) * 256;
    float* out = reinterpret_cast<float*>(base ? base + used : nullptr);
    used += bytes;
    return out;
  }
};

struct Layout {
  float *pT, *aT, *qs, *ls, *us, *qT, *x, *z, *y, *kkt, *lx, *d, *dinv, *rhs, *scratch;
  float *rho_row, *rinv_row, *rho_b;  // plain mode: per-instance rho vectors and scalar (rho adaptation)
  int* rho_changed;                   // [batch] 1 where the last estimate changed rho
  int* rho_count;                     // [batch] rho changes so far
  size_t scratch_bytes;
  bool factor_separately;  // factor with the per-call kernels before iterating
  bool streaming;          // persistent mode on the TMA-fed streaming kernel
  float* stream_ws;
  int* stream_status;
  int* error_word;
};

// Workspace carve-up.  `external`: the caller supplies the factorization.
Layout carve(const Osqp& o, const Pattern& pat, int batch, int pb, int ab, int mode, bool external, char* base,
             size_t* total, const wmpc_osqp* q = nullptr, bool use_stream = false, bool per_instance_factor = false) {
  Carve c{base};
  Layout L{};
  if (use_stream && q && q->has_stream && mode == WMPC_OSQP_PERSISTENT && !external) {
    L.streaming = true;
    L.pT = c.take((size_t)o.nnz_p * pb);
    L.aT = c.take((size_t)o.nnz_a * ab);
    L.qT = c.take((size_t)o.n * batch);
    L.qs = c.take((size_t)o.n * batch);
    L.ls = c.take((size_t)o.m * batch);
    L.us = c.take((size_t)o.m * batch);
    L.x = c.take((size_t)o.n * batch);
    L.z = c.take((size_t)o.m * batch);
    L.y = c.take((size_t)o.m * batch);
    // (either schedule a launch may pick)
    L.stream_ws = c.take(std::max(stream_workspace_floats(q->sp, batch),
                                  q->has_frontier ? stream_workspace_floats(q->spf, batch) : (size_t)0));
    L.stream_status = reinterpret_cast<int*>(c.take((size_t)((batch + 31) / 32) * 32));
    L.error_word = reinterpret_cast<int*>(c.take(4));
    if (o.rho_type) {  // per-instance rho (adaptation)
      L.rho_row = c.take((size_t)o.m * batch);
      L.rinv_row = c.take((size_t)o.m * batch);
      L.rho_b = c.take((size_t)batch);
      L.rho_changed = reinterpret_cast<int*>(c.take((size_t)batch));
      L.rho_count = reinterpret_cast<int*>(c.take((size_t)batch));
    }
    *total = c.used;
    return L;
  }
  // KKT (factor) batch: one factor per instance when rho adapts per instance
  const int kb = per_instance_factor ? batch : (pb > ab ? pb : ab);
  L.pT = c.take((size_t)o.nnz_p * pb);
  L.aT = c.take((size_t)o.nnz_a * ab);
  L.qT = c.take((size_t)o.n * batch);
  L.qs = c.take((size_t)o.n * batch);
  L.ls = c.take((size_t)o.m * batch);
  L.us = c.take((size_t)o.m * batch);
  L.x = c.take((size_t)o.n * batch);
  L.z = c.take((size_t)o.m * batch);
  L.y = c.take((size_t)o.m * batch);
  L.factor_separately = !external && (mode == WMPC_OSQP_PLAIN || kb == 1);
  size_t scratch = 0;
  if (!external) {
    const int fb = L.factor_separately ? kb : batch;
    if (L.factor_separately) {
      L.kkt = c.take((size_t)o.nnz_kkt * kb);
      scratch = factor_workspace_bytes(pat, kb);
    }
    L.lx = c.take((size_t)pat.nnz_l * fb);
    L.d = c.take((size_t)pat.n * fb);
    L.dinv = c.take((size_t)pat.n * fb);
  }
  if (mode == WMPC_OSQP_PLAIN) {
    L.rhs = c.take((size_t)o.nk * batch);
    L.rho_row = c.take((size_t)o.m * batch);
    L.rinv_row = c.take((size_t)o.m * batch);
    L.rho_b = c.take((size_t)batch);
    L.rho_changed = reinterpret_cast<int*>(c.take((size_t)batch));
    L.rho_count = reinterpret_cast<int*>(c.take((size_t)batch));
    size_t s2 = solve_workspace_bytes(pat, batch);
    scratch = scratch > s2 ? scratch : s2;
  } else {
    size_t s2 = smem_lanes_for_rows(pat.n) >= 32 ? 0 : (size_t)4 * pat.n * batch;
    scratch = scratch > s2 ? scratch : s2;
  }
  L.scratch_bytes = scratch;
  L.scratch = scratch ? c.take(scratch / 4 + 1) : nullptr;
  *total = c.used;
  return L;
}

int assemble_and_factor(const Osqp& o, const wmpc_plan& plan, const float* pT, int pb, const float* aT, int ab,
                        float* kkt, float* lx, float* d, float* dinv, void* scratch, size_t scratch_bytes,
                        cudaStream_t s) {
  const int kb = pb > ab ? pb : ab;
  dim3 grid(ceil_div(kb, 128), o.nnz_kkt < 4096 ? o.nnz_kkt : 4096);
  assemble_kkt_kernel<<<grid, 128, 0, s>>>(o, pT, pb, pb > 1 ? 1 : 0, aT, ab, ab > 1 ? 1 : 0, kkt, kb);
  WMPC_LAUNCH_CHECK();
  return launch_factor_plan(plan, kkt, kb, 1, lx, d, dinv, kb, scratch, scratch_bytes, s);
}

}  // namespace

int stream_begin(const Pattern& pat, const StreamPlan& sp, const Osqp& o, const float* pT, long long ldp, int sbp,
                 const float* aT, long long lda, int sba, const float* x, const float* z, const float* y,
                 const float* qs, const float* ls, const float* us, bool warm, bool track, float* work,
                 int* status, int batch, int num_sms, bool reuse_factor, StreamJobDesc* job, cudaStream_t s,
                 const float* rinv_rows = nullptr, const int* only = nullptr);
int stream_run(const StreamJobDesc* jobs, int n_jobs, int* error, int num_sms, cudaStream_t s);
int stream_end(const StreamPlan& sp, const Osqp& o, const StreamJobDesc& job, float* x, float* z, float* y,
               cudaStream_t s);

static bool stream_eligible(const wmpc_osqp& q, const wmpc_osqp_options* opt) {
  (void)opt;
  return q.has_stream && !env_disabled("WMPC_DISABLE_STREAM");
}

size_t osqp_workspace_bytes(const wmpc_osqp& q, int batch, int pb, int ab, int mode, bool external) {
  size_t total = 0, total2 = 0;
  carve(q.dev, q.kkt_plan->pat, batch, pb, ab, mode, external, nullptr, &total);
  // a workspace sized here must serve both the streaming and the fallback kernels
  carve(q.dev, q.kkt_plan->pat, batch, pb, ab, mode, external, nullptr, &total2, &q, stream_eligible(q, nullptr));
  return total > total2 ? total : total2;
}

size_t osqp_factor_workspace_bytes(const Osqp& o, const Pattern& pat, int pb, int ab) {
  const int kb = pb > ab ? pb : ab;
  Carve c{nullptr};
  c.take((size_t)o.nnz_p * pb);
  c.take((size_t)o.nnz_a * ab);
  c.take((size_t)o.nnz_kkt * kb);
  const size_t f = factor_workspace_bytes(pat, kb);
  if (f) c.take(f / 4 + 1);
  return c.used;
}

int osqp_factor(const Osqp& o, const wmpc_plan& plan, const float* p_values, int pb, const float* a_values, int ab,
                float* lx, float* d, float* dinv, void* ws, size_t ws_bytes, cudaStream_t s) {
  const Pattern& pat = plan.pat;
  const int kb = pb > ab ? pb : ab;
  const size_t need = osqp_factor_workspace_bytes(o, pat, pb, ab);
  if (ws == nullptr || ws_bytes < need)
    return fail(WMPC_ERR_WORKSPACE, "OSQP factor needs %zu workspace bytes, got %zu", need, ws_bytes);
  Carve c{static_cast<char*>(ws)};
  float* pT = c.take((size_t)o.nnz_p * pb);
  float* aT = c.take((size_t)o.nnz_a * ab);
  float* kkt = c.take((size_t)o.nnz_kkt * kb);
  const size_t f = factor_workspace_bytes(pat, kb);
  float* scratch = f ? c.take(f / 4 + 1) : nullptr;
  int rc;
  if ((rc = transpose_in(p_values, o.nnz_p, pb, o.nnz_p, nullptr, pT, pb, s))) return rc;
  if ((rc = transpose_in(a_values, o.nnz_a, ab, o.nnz_a, nullptr, aT, ab, s))) return rc;
  return assemble_and_factor(o, plan, pT, pb, aT, ab, kkt, lx, d, dinv, scratch, f, s);
}

namespace {

// Batch-major inputs -> symbolic-major, scaled where the reference scales;
// the starting iterate (warm start, or zero).
// Residual outputs requested (or termination checked): the final residuals
// need P, A and the unscaled q in the workspace.
static bool residuals_wanted(const wmpc_osqp_options& opt, const wmpc_osqp_batch& d) {
  return d.prim_res || d.dual_res || d.obj || opt.check_termination > 0;
}

// P and A are staged when the solve factors or forms residuals (a solve that
// reuses its factor without residual outputs -- the adjoint's -- skips them).
int stage_inputs(const Osqp& o, const wmpc_osqp_options& opt, const wmpc_osqp_batch& d, const Layout& L,
                 cudaStream_t s) {
  const int B = d.batch, pb = d.p_batch, ab = d.a_batch;
  const bool sums = residuals_wanted(opt, d);
  int rc;
  if (!opt.reuse_factor || sums) {
    if ((rc = transpose_in(d.p_values, o.nnz_p, pb, o.nnz_p, nullptr, L.pT, pb, s))) return rc;
    if ((rc = transpose_in(d.a_values, o.nnz_a, ab, o.nnz_a, nullptr, L.aT, ab, s))) return rc;
  }
  if (sums && (rc = transpose_in(d.q, o.n, B, o.n, nullptr, L.qT, B, s))) return rc;
  if ((rc = transpose_in(d.q, o.n, B, o.n, o.q_scale, L.qs, B, s))) return rc;
  if ((rc = transpose_in(d.l, o.m, B, o.m, o.scaling_e, L.ls, B, s))) return rc;
  if ((rc = transpose_in(d.u, o.m, B, o.m, o.scaling_e, L.us, B, s))) return rc;
  if (opt.warm_start) {
    if (!d.x0 || !d.z0 || !d.y0) return fail(WMPC_ERR_INVALID_ARGUMENT, "warm start needs x0, z0 and y0");
    if ((rc = transpose_in(d.x0, o.n, B, o.n, o.scaling_dinv, L.x, B, s))) return rc;
    if ((rc = transpose_in(d.z0, o.m, B, o.m, o.scaling_e, L.z, B, s))) return rc;
    if ((rc = transpose_in(d.y0, o.m, B, o.m, o.y_scale, L.y, B, s))) return rc;
  } else {
    WMPC_CUDA_TRY(cudaMemsetAsync(L.x, 0, sizeof(float) * (size_t)o.n * B, s));
    WMPC_CUDA_TRY(cudaMemsetAsync(L.z, 0, sizeof(float) * (size_t)o.m * B, s));
    WMPC_CUDA_TRY(cudaMemsetAsync(L.y, 0, sizeof(float) * (size_t)o.m * B, s));
  }
  return WMPC_OK;
}

// The schedule a solve of `tiles` instance tiles runs alone: the frontier form
// where this batch's launch of it would put more CTAs on an SM than the plain
// form's (both counts under the problem's CTA limit, which the launch uses
// too, and sized with the residual records of a checked solve).
static bool frontier_for(const wmpc_osqp& q, bool check, int tiles) {
  if (!q.has_frontier) return false;
  return stream_ctas_for(q.spf, q.kkt_plan->device, tiles, q.num_sms, q.ctas_limit, check) >
         stream_ctas_for(q.sp, q.kkt_plan->device, tiles, q.num_sms, q.ctas_limit, check);
}

// Streaming solve, first half: inputs staged, factor, state records; fills
// `job` (frontier: with the problem's frontier-form schedule).
int stream_solve_begin(const wmpc_osqp& q, const wmpc_osqp_options& opt, const wmpc_osqp_batch& d, const Layout& L,
                       bool frontier, StreamJobDesc* job, cudaStream_t s) {
  const Osqp& o = q.dev;
  const int B = d.batch, pb = d.p_batch, ab = d.a_batch;
  const int check = opt.check_termination > 0 ? opt.check_termination : 0;
  int rc;
  if ((rc = stage_inputs(o, opt, d, L, s))) return rc;
  WMPC_CUDA_TRY(cudaMemsetAsync(L.error_word, 0, sizeof(int), s));
  if ((rc = stream_begin(q.kkt_plan->pat, frontier ? q.spf : q.sp, o, L.pT, pb, pb > 1 ? 1 : 0, L.aT, ab, ab > 1 ? 1 : 0,
                         L.x, L.z, L.y,
                         L.qs, L.ls, L.us, opt.warm_start != 0, check > 0, L.stream_ws, L.stream_status, B,
                         q.num_sms, opt.reuse_factor != 0, job, s)))
    return rc;
  // termination: an instance stops (freezes) once both its primal residual
  // (A x - z, carried exactly through the iterations) and its largest iterate
  // change over an iteration are at most eps_abs, unscaled; the change stands
  // in for the dual residual, which needs P and A-transpose products the
  // streaming kernel does not form.  SOLVED comes from the exact residuals of
  // the final iterate.
  job->max_iter = opt.max_iter;
  job->check_every = check;
  job->ctas_limit = q.ctas_limit;
  job->chg_eps = opt.eps_abs;
  job->iters = check ? d.iters : nullptr;
  return WMPC_OK;
}

// Streaming solve with per-instance rho adaptation (fixed iterations): the
// iterations run in launches of adaptive_rho_interval; between two, the state
// comes back, each instance estimates its rho (rho_update_kernel, the plain
// path's rule and sums), the tiles holding an instance whose rho changed
// refactor with their instances' own -1/rho, and the next launch continues
// from the state with each lane's rho by row class (admm_stream_kernel's
// per-instance-rho form).  Same iterates, rho and refactor counts as the
// plain path.
int stream_solve_adaptive(const wmpc_osqp& q, const wmpc_osqp_options& opt, const wmpc_osqp_batch& d,
                          const Layout& L, StreamJobDesc* job, cudaStream_t s) {
  const Osqp& o = q.dev;
  const int B = d.batch, pb = d.p_batch, ab = d.a_batch;
  const int sbp = pb > 1 ? 1 : 0, sba = ab > 1 ? 1 : 0;
  const bool frontier = frontier_for(q, false, (B + 31) / 32);
  const StreamPlan& sp = frontier ? q.spf : q.sp;
  int rc;
  if ((rc = stage_inputs(o, opt, d, L, s))) return rc;
  WMPC_CUDA_TRY(cudaMemsetAsync(L.error_word, 0, sizeof(int), s));
  dim3 rgrid(ceil_div(B, 128), o.m > 0 ? (o.m < 2048 ? o.m : 2048) : 1);
  rho_init_kernel<<<rgrid, 128, 0, s>>>(o, L.rho_row, L.rinv_row, L.rho_b, L.rho_count, B);
  WMPC_LAUNCH_CHECK();
  State st{L.x, L.z, L.y, L.qs, L.ls, L.us, B};
  auto begin = [&](bool warm, const int* only) -> int {
    int r = stream_begin(q.kkt_plan->pat, sp, o, L.pT, pb, sbp, L.aT, ab, sba, L.x, L.z, L.y, L.qs, L.ls, L.us, warm,
                         false, L.stream_ws, L.stream_status, B, q.num_sms, false, job, s, L.rinv_row, only);
    job->check_every = 0;
    job->ctas_limit = q.ctas_limit;
    job->chg_eps = opt.eps_abs;
    job->iters = nullptr;
    job->rho_b = L.rho_b;
    job->rho_count = L.rho_count;
    return r;
  };
  if ((rc = begin(opt.warm_start != 0, nullptr))) return rc;
  const int interval = opt.adaptive_rho_interval;
  for (int it = 0; it < opt.max_iter;) {
    const int seg = opt.max_iter - it < interval ? opt.max_iter - it : interval;
    job->max_iter = seg;
    if ((rc = stream_run(job, 1, L.error_word, q.num_sms, s))) return rc;
    it += seg;
    if (it < opt.max_iter) {
      if ((rc = stream_end(sp, o, *job, L.x, L.z, L.y, s))) return rc;
      rho_update_kernel<<<ceil_div(B, 128), 128, 0, s>>>(o, L.pT, pb, sbp, L.aT, ab, sba, st, L.rho_row, L.rinv_row,
                                                         L.rho_b, L.rho_changed, L.rho_count,
                                                         opt.adaptive_rho_tolerance, B);
      WMPC_LAUNCH_CHECK();
      if ((rc = begin(true, L.rho_changed))) return rc;
    }
  }
  if (d.rho || d.rho_updates) {
    rho_report_kernel<<<ceil_div(B, 256), 256, 0, s>>>(L.rho_b, L.rho_count, o.rho0, d.rho, d.rho_updates, B);
    WMPC_LAUNCH_CHECK();
  }
  return WMPC_OK;
}

// Streaming solve, second half: state back, exact residuals and status, outputs.
int stream_solve_end(const wmpc_osqp& q, const wmpc_osqp_options& opt, const wmpc_osqp_batch& d, const Layout& L,
                     const StreamJobDesc& job, const int* error_word, cudaStream_t s) {
  const Osqp& o = q.dev;
  const int B = d.batch, pb = d.p_batch, ab = d.a_batch;
  const int check = opt.check_termination > 0 ? opt.check_termination : 0;
  int rc;
  if ((rc = stream_end(job.sp, o, job, L.x, L.z, L.y, s))) return rc;
  State st{L.x, L.z, L.y, L.qs, L.ls, L.us, B};
  if (residuals_wanted(opt, d)) {
    residual_kernel<<<ceil_div(B, 32), dim3(32, kResParts), 0, s>>>(
        o, L.pT, pb, pb > 1 ? 1 : 0, L.aT, ab, ab > 1 ? 1 : 0, st, L.qT, d.prim_res, d.dual_res, d.obj, d.status, B,
        L.stream_status, error_word, check ? opt.eps_abs : -1.0f, opt.eps_rel);
  } else {
    unscale_state_kernel<<<ceil_div(B, 32), dim3(32, kResParts), 0, s>>>(o, st, d.status, L.stream_status, error_word, B);
  }
  WMPC_LAUNCH_CHECK();
  if (d.iters && !check) {
    fill_int_kernel<<<ceil_div(B, 256), 256, 0, s>>>(d.iters, opt.max_iter, B);
    WMPC_LAUNCH_CHECK();
  }
  if ((rc = transpose_out(L.x, B, B, o.n, d.x, o.n, s))) return rc;
  if ((rc = transpose_out(L.z, B, B, o.m, d.z, o.m, s))) return rc;
  if ((rc = transpose_out(L.y, B, B, o.m, d.y, o.m, s))) return rc;
  return WMPC_OK;
}

}  // namespace

int osqp_solve(const wmpc_osqp& q, const wmpc_osqp_options& opt, const wmpc_osqp_batch& d,
               const float* lx_ext, const float* dinv_ext, int fb_ext, int mode, void* ws, size_t ws_bytes,
               cudaStream_t s) {
  const Osqp& o = q.dev;
  const Pattern& pat = q.kkt_plan->pat;
  const int B = d.batch;
  if (B <= 0) return WMPC_OK;
  const int pb = d.p_batch, ab = d.a_batch;
  const bool external = lx_ext != nullptr;
  if ((d.prim_res || d.dual_res || d.obj || opt.check_termination > 0) && !(d.prim_res && d.dual_res && d.obj))
    return fail(WMPC_ERR_INVALID_ARGUMENT, "prim_res, dual_res and obj go together (and with termination checks)");
  const bool adaptive = opt.adaptive_rho_interval > 0;
  if (adaptive) {
    if (mode != WMPC_OSQP_PLAIN && !(mode == WMPC_OSQP_PERSISTENT && stream_eligible(q, &opt)))
      return fail(WMPC_ERR_UNSUPPORTED, "rho adaptation runs in plain mode or on the streaming persistent path");
    if (mode == WMPC_OSQP_PERSISTENT && opt.check_termination > 0)
      return fail(WMPC_ERR_UNSUPPORTED, "rho adaptation on the persistent path runs fixed iterations");
    if (external || opt.reuse_factor)
      return fail(WMPC_ERR_UNSUPPORTED, "rho adaptation refactors: it cannot start from a given factorization");
    if (!o.rho_type || !o.kkt_rho_row)
      return fail(WMPC_ERR_UNSUPPORTED, "the problem was created without the rho adaptation tables");
    if (!(opt.adaptive_rho_tolerance >= 1.0f))
      return fail(WMPC_ERR_INVALID_ARGUMENT, "adaptive_rho_tolerance must be at least 1");
  }
  size_t need = 0;
  Layout L = carve(o, pat, B, pb, ab, mode, external, static_cast<char*>(ws), &need, &q, stream_eligible(q, &opt),
                   adaptive);
  if (ws == nullptr || ws_bytes < need)
    return fail(WMPC_ERR_WORKSPACE, "OSQP solve needs %zu workspace bytes, got %zu", need, ws_bytes);
  int rc;
  if (L.streaming && adaptive) {
    StreamJobDesc job;
    if ((rc = stream_solve_adaptive(q, opt, d, L, &job, s))) return rc;
    return stream_solve_end(q, opt, d, L, job, L.error_word, s);
  }
  if (L.streaming) {
    StreamJobDesc job;
    const bool frontier = frontier_for(q, opt.check_termination > 0, (B + 31) / 32);
    if ((rc = stream_solve_begin(q, opt, d, L, frontier, &job, s))) return rc;
    if ((rc = stream_run(&job, 1, L.error_word, q.num_sms, s))) return rc;
    return stream_solve_end(q, opt, d, L, job, L.error_word, s);
  }
  if ((rc = stage_inputs(o, opt, d, L, s))) return rc;
  State st{L.x, L.z, L.y, L.qs, L.ls, L.us, B};
  const int sbp = pb > 1 ? 1 : 0, sba = ab > 1 ? 1 : 0;
  const long long ldp = pb, lda = ab;
  const int kb = pb > ab ? pb : ab;

  // the factorization the iterations use
  const float* lx = lx_ext;
  const float* dinv = dinv_ext;
  int fb = fb_ext;
  dim3 rgrid(ceil_div(B, 128), o.m > 0 ? (o.m < 2048 ? o.m : 2048) : 1);
  dim3 kgrid(ceil_div(B, 128), o.nnz_kkt < 4096 ? o.nnz_kkt : 4096);
  if (adaptive) {
    // one factor per instance, each instance's rho vector starting at the plan's
    rho_init_kernel<<<rgrid, 128, 0, s>>>(o, L.rho_row, L.rinv_row, L.rho_b, L.rho_count, B);
    WMPC_LAUNCH_CHECK();
    assemble_kkt_rho_kernel<<<kgrid, 128, 0, s>>>(o, L.pT, ldp, sbp, L.aT, lda, sba, L.rinv_row, nullptr, L.kkt, B);
    WMPC_LAUNCH_CHECK();
    if ((rc = launch_factor_plan(*q.kkt_plan, L.kkt, B, 1, L.lx, L.d, L.dinv, B, L.scratch, L.scratch_bytes, s)))
      return rc;
    lx = L.lx;
    dinv = L.dinv;
    fb = B;
  } else if (!external && L.factor_separately) {
    if (!opt.reuse_factor &&
        (rc = assemble_and_factor(o, *q.kkt_plan, L.pT, pb, L.aT, ab, L.kkt, L.lx, L.d, L.dinv, L.scratch,
                                  L.scratch_bytes, s)))
      return rc;
    lx = L.lx;
    dinv = L.dinv;
    fb = kb;
  }
  if (external && fb != 1 && fb != B) return fail(WMPC_ERR_INVALID_ARGUMENT, "factor_batch must be 1 or batch");

  if (mode == WMPC_OSQP_PLAIN) {
    const int fstride = fb > 1 ? 1 : 0;
    dim3 egrid(ceil_div(B, 128), o.nk < 2048 ? o.nk : 2048);
    const RhoRows rr = adaptive ? RhoRows{L.rho_row, L.rinv_row} : RhoRows{};
    admm_first_rhs_kernel<<<egrid, 128, 0, s>>>(o, st, L.rhs, B, rr);
    WMPC_LAUNCH_CHECK();
    for (int it = 0; it < opt.max_iter; ++it) {
      profile_mark_begin(s);
      rc = launch_solve_plan(*q.kkt_plan, lx, dinv, fstride, L.rhs, L.rhs, B, L.scratch, L.scratch_bytes, s);
      profile_mark_end(s);
      if (rc) return rc;
      admm_update_kernel<<<egrid, 128, 0, s>>>(o, st, L.rhs, B, rr);
      WMPC_LAUNCH_CHECK();
      if (adaptive && (it + 1) % opt.adaptive_rho_interval == 0 && it + 1 < opt.max_iter) {
        // new rho estimates; the instances whose rho changed refactor, and
        // every instance's next right-hand side is formed with its rho
        rho_update_kernel<<<ceil_div(B, 128), 128, 0, s>>>(o, L.pT, ldp, sbp, L.aT, lda, sba, st, L.rho_row,
                                                           L.rinv_row, L.rho_b, L.rho_changed, L.rho_count,
                                                           opt.adaptive_rho_tolerance, B);
        WMPC_LAUNCH_CHECK();
        assemble_kkt_rho_kernel<<<kgrid, 128, 0, s>>>(o, L.pT, ldp, sbp, L.aT, lda, sba, L.rinv_row, L.rho_changed,
                                                      L.kkt, B);
        WMPC_LAUNCH_CHECK();
        if ((rc = launch_factor_plan(*q.kkt_plan, L.kkt, B, 1, L.lx, L.d, L.dinv, B, L.scratch, L.scratch_bytes, s,
                                L.rho_changed)))
          return rc;
        admm_first_rhs_kernel<<<egrid, 128, 0, s>>>(o, st, L.rhs, B, rr);
        WMPC_LAUNCH_CHECK();
      }
    }
    if (d.rho || d.rho_updates) {
      rho_report_kernel<<<ceil_div(B, 256), 256, 0, s>>>(adaptive ? L.rho_b : nullptr,
                                                         adaptive ? L.rho_count : nullptr, o.rho0, d.rho,
                                                         d.rho_updates, B);
      WMPC_LAUNCH_CHECK();
    }
    if (residuals_wanted(opt, d)) {
      residual_kernel<<<ceil_div(B, 32), dim3(32, kResParts), 0, s>>>(
          o, L.pT, ldp, sbp, L.aT, lda, sba, st, L.qT, d.prim_res, d.dual_res, d.obj, d.status, B, nullptr, nullptr,
          -1.0f, 0.0f);
    } else {
      unscale_state_kernel<<<ceil_div(B, 32), dim3(32, kResParts), 0, s>>>(o, st, d.status, nullptr, nullptr, B);
    }
    WMPC_LAUNCH_CHECK();
    if (d.iters) {
      fill_int_kernel<<<ceil_div(B, 256), 256, 0, s>>>(d.iters, opt.max_iter, B);
      WMPC_LAUNCH_CHECK();
    }
  } else {
    const bool fused = !external && !L.factor_separately;
    const bool refactor = fused && !opt.reuse_factor;
    PersistentArgs pa{};
    pa.pat = pat;
    pa.o = o;
    pa.pT = L.pT; pa.ldp = ldp; pa.sbp = sbp;
    pa.aT = L.aT; pa.lda = lda; pa.sba = sba;
    pa.qT = L.qT;
    pa.st = st;
    pa.lx = fused ? L.lx : const_cast<float*>(lx);
    pa.dinv = fused ? L.dinv : const_cast<float*>(dinv);
    pa.d = fused ? L.d : nullptr;
    pa.fstride = fused ? 1 : (fb > 1 ? 1 : 0);
    pa.fld = fused ? B : fb;
    pa.fused_factor = refactor ? 1 : 0;
    pa.wglob = L.scratch;
    pa.prim = d.prim_res; pa.dual = d.dual_res; pa.obj = d.obj;
    pa.iters = d.iters; pa.status = d.status;
    pa.batch = B; pa.max_iter = opt.max_iter; pa.check_every = opt.check_termination;
    pa.eps_abs = opt.eps_abs; pa.eps_rel = opt.eps_rel;
    const int lanes = smem_lanes_for_rows(pat.n);
    if (lanes >= 32) {
      const int threads = lanes < 128 ? lanes : 128;
      const size_t smem = (size_t)4 * pat.n * threads;
      WMPC_CUDA_TRY(cudaFuncSetAttribute(persistent_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem));
      profile_mark_begin(s);
      persistent_kernel<true><<<ceil_div(B, threads), threads, smem, s>>>(pa);
    } else {
      profile_mark_begin(s);
      persistent_kernel<false><<<ceil_div(B, 128), 128, 0, s>>>(pa);
    }
    profile_mark_end(s);
    WMPC_LAUNCH_CHECK();
  }
  if ((rc = transpose_out(L.x, B, B, o.n, d.x, o.n, s))) return rc;
  if ((rc = transpose_out(L.z, B, B, o.m, d.z, o.m, s))) return rc;
  if ((rc = transpose_out(L.y, B, B, o.m, d.y, o.m, s))) return rc;
  return WMPC_OK;
}

// Several OSQP classes (patterns) in one streaming launch: each class is
// staged, factored and converted on its own, then one persistent kernel walks
// every class's tiles (costliest class first), then each class's epilogue.
int osqp_solve_multi(const wmpc_osqp* const* qs, const wmpc_osqp_options* opts, const wmpc_osqp_batch* ds, int n,
                     void* const* ws, const size_t* ws_bytes, cudaStream_t s) {
  if (n < 1 || n > 6) return fail(WMPC_ERR_INVALID_ARGUMENT, "1 to 6 classes per launch, got %d", n);
  std::vector<Layout> L(n);
  std::vector<StreamJobDesc> jobs(n);
  std::vector<int> active;
  int rc;
  // one schedule form per launch: the frontier form only when every class
  // would pick it for the launch's tiles
  bool frontier = true;
  int tiles = 0;
  for (int i = 0; i < n; ++i) tiles += ds[i].batch > 0 ? (ds[i].batch + 31) / 32 : 0;
  for (int i = 0; i < n; ++i)
    if (ds[i].batch > 0) frontier = frontier && frontier_for(*qs[i], opts[i].check_termination > 0, tiles);
  for (int i = 0; i < n; ++i) {
    const wmpc_osqp& q = *qs[i];
    const wmpc_osqp_batch& d = ds[i];
    if (q.device != qs[0]->device) return fail(WMPC_ERR_INVALID_ARGUMENT, "all classes must be on one device");
    if (!stream_eligible(q, &opts[i]))
      return fail(WMPC_ERR_UNSUPPORTED, "class %d cannot use the streaming kernel: %s", i,
                  q.has_stream ? "disabled by the environment" : q.stream_why.c_str());
    if (d.batch <= 0) continue;
    size_t need = 0;
    L[i] = carve(q.dev, q.kkt_plan->pat, d.batch, d.p_batch, d.a_batch, WMPC_OSQP_PERSISTENT, false,
                 static_cast<char*>(ws[i]), &need, &q, true);
    if (ws[i] == nullptr || ws_bytes[i] < need)
      return fail(WMPC_ERR_WORKSPACE, "class %d needs %zu workspace bytes, got %zu", i, need, ws_bytes[i]);
    if ((rc = stream_solve_begin(q, opts[i], d, L[i], frontier, &jobs[i], s))) return rc;
    active.push_back(i);
  }
  if (active.empty()) return WMPC_OK;
  std::vector<StreamJobDesc> run;
  for (int i : active) run.push_back(jobs[i]);
  int* error_word = L[active[0]].error_word;
  if ((rc = stream_run(run.data(), static_cast<int>(run.size()), error_word, qs[active[0]]->num_sms, s))) return rc;
  for (int i : active)
    if ((rc = stream_solve_end(*qs[i], opts[i], ds[i], L[i], jobs[i], error_word, s))) return rc;
  return WMPC_OK;
}


// ---------------------------------------------------------------------------
// adjoint: active-set differential QP on the forward's factorization
// ---------------------------------------------------------------------------

// Per (instance, constraint): activity tau (+1 upper / -1 lower / 0 free) and
// the differential QP's bounds (t = -tau * dy on active rows, free otherwise).
__global__ void adjoint_prep_kernel(const float* __restrict__ l, const float* __restrict__ u,
                                    const float* __restrict__ z, const float* __restrict__ y,
                                    const float* __restrict__ dy, float* __restrict__ ld, float* __restrict__ ud,
                                    int* __restrict__ tau, long long count) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  const float lk = l[k], uk = u[k], zk = z[k], yk = y[k];
  int t = 0;
  if (lk == uk) t = (yk >= 0.0f) ? 1 : -1;
  else if (zk >= uk) t = 1;
  else if (zk <= lk) t = -1;
  const float dyk = dy ? dy[k] : 0.0f;
  if (t != 0) {
    const float target = -(float)t * dyk;
    ld[k] = target;
    ud[k] = target;
  } else {
    ld[k] = -1e30f;
    ud[k] = 1e30f;
  }
  tau[k] = t;
}

// dl/du from the differential QP's multipliers mu (dq = w is written by the solve)
__global__ void adjoint_bounds_kernel(const int* __restrict__ tau, const float* __restrict__ mu,
                                      float* __restrict__ dl, float* __restrict__ du, long long count) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  const int t = tau[k];
  const float g = -mu[k];
  dl[k] = t < 0 ? g : 0.0f;
  du[k] = t > 0 ? g : 0.0f;
}

// dP on P's upper pattern and dA on A's pattern, per instance (batch-major):
// dP_k = 0.5 * (w_i x_j + w_j x_i), dA_k = y_r w_c + nu_r x_c (nu = mu on
// active rows, 0 on free rows) -- solver.py:1184-1191.
__global__ void adjoint_matrix_kernel(Osqp o, const int* __restrict__ p_rows, const int* __restrict__ p_cols,
                                      const float* __restrict__ w, const float* __restrict__ x,
                                      const float* __restrict__ y, const float* __restrict__ mu,
                                      const int* __restrict__ tau, float* __restrict__ dp, float* __restrict__ da,
                                      int batch) {
  const int b = blockIdx.x;  // one instance per x block (batches beyond 65535 instances fit grid x)
  if (b >= batch) return;
  const float* wb = w + (size_t)b * o.n;
  const float* xb = x + (size_t)b * o.n;
  const float* yb = y + (size_t)b * o.m;
  const float* mb = mu + (size_t)b * o.m;
  const int* tb = tau + (size_t)b * o.m;
  for (int k = blockIdx.y * blockDim.x + threadIdx.x; k < o.nnz_p + o.nnz_a; k += gridDim.y * blockDim.x) {
    if (k < o.nnz_p) {
      const int i = __ldg(p_rows + k), j = __ldg(p_cols + k);
      dp[(size_t)b * o.nnz_p + k] = 0.5f * (wb[i] * xb[j] + wb[j] * xb[i]);
    } else {
      const int e = k - o.nnz_p;
      const int r = __ldg(o.a_rows + e), c = __ldg(o.a_cols + e);
      const float nu = tb[r] != 0 ? mb[r] : 0.0f;
      da[(size_t)b * o.nnz_a + e] = yb[r] * wb[c] + nu * xb[c];
    }
  }
}

size_t osqp_adjoint_extra_bytes(const Osqp& o, int batch) {
  Carve c{nullptr};
  c.take((size_t)o.m * batch);       // tau
  c.take((size_t)o.m * batch);       // mu
  c.take((size_t)o.m * batch);       // z of the differential QP
  c.take((size_t)o.m * batch);       // ld
  c.take((size_t)o.m * batch);       // ud
  c.take(5 * (size_t)batch);         // prim, dual, obj, iters, status
  return c.used;
}

int osqp_adjoint(const wmpc_osqp& q, const wmpc_osqp_options& opt, const wmpc_osqp_adjoint_batch& a, int mode,
                 void* ws, size_t ws_bytes, cudaStream_t s) {
  const Osqp& o = q.dev;
  const int B = a.batch;
  if (B <= 0) return WMPC_OK;
  size_t solve_bytes = 0;
  carve(o, q.kkt_plan->pat, B, a.p_batch, a.a_batch, mode, false, nullptr, &solve_bytes, &q,
        stream_eligible(q, &opt) && mode == WMPC_OSQP_PERSISTENT);
  const size_t extra = osqp_adjoint_extra_bytes(o, B);
  if (ws == nullptr || ws_bytes < solve_bytes + extra)
    return fail(WMPC_ERR_WORKSPACE, "OSQP adjoint needs %zu workspace bytes, got %zu", solve_bytes + extra, ws_bytes);
  Carve c{static_cast<char*>(ws) + solve_bytes};
  int* tau = reinterpret_cast<int*>(c.take((size_t)o.m * B));
  float* mu = c.take((size_t)o.m * B);
  float* zd = c.take((size_t)o.m * B);
  float* ld = c.take((size_t)o.m * B);
  float* ud = c.take((size_t)o.m * B);
  float* misc = c.take(5 * (size_t)B);
  const long long cm = (long long)o.m * B;
  adjoint_prep_kernel<<<ceil_div(cm, 256), 256, 0, s>>>(a.l, a.u, a.z, a.y, a.dy, ld, ud, tau, cm);
  WMPC_LAUNCH_CHECK();
  wmpc_osqp_batch d{};
  d.batch = B;
  d.p_values = a.p_values;
  d.p_batch = a.p_batch;
  d.a_values = a.a_values;
  d.a_batch = a.a_batch;
  d.q = a.dx;
  d.l = ld;
  d.u = ud;
  d.x = a.dq;  // w
  d.z = zd;
  d.y = mu;
  // residuals of the differential QP only when asked for (they need P and A staged)
  d.prim_res = a.adj_prim_res;
  d.dual_res = a.adj_prim_res ? misc + B : nullptr;
  d.obj = a.adj_prim_res ? misc + 2 * B : nullptr;
  d.iters = reinterpret_cast<int*>(misc + 3 * B);
  d.status = reinterpret_cast<int*>(misc + 4 * B);
  wmpc_osqp_options ao = opt;
  ao.warm_start = 0;
  ao.reuse_factor = 1;  // same carve as the forward: check_termination and mode must match it
  int rc = osqp_solve(q, ao, d, nullptr, nullptr, 0, mode, ws, solve_bytes, s);
  if (rc) return rc;
  adjoint_bounds_kernel<<<ceil_div(cm, 256), 256, 0, s>>>(tau, mu, a.dl, a.du, cm);
  WMPC_LAUNCH_CHECK();
  if (a.dp || a.da) {
    if (!a.dp || !a.da) return fail(WMPC_ERR_INVALID_ARGUMENT, "dp and da go together");
    dim3 grid(B, ceil_div(o.nnz_p + o.nnz_a, 256) < 64 ? ceil_div(o.nnz_p + o.nnz_a, 256) : 64);
    adjoint_matrix_kernel<<<grid, 256, 0, s>>>(o, q.p_upper_rows, q.p_upper_cols, a.dq, a.x, a.y, mu, tau, a.dp,
                                               a.da, B);
    WMPC_LAUNCH_CHECK();
  }
  return WMPC_OK;
}

}  // namespace wmpc

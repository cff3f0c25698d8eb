// Filter line search of the SQP outer loop (warpmpc/jax_sqp/line_search.py
// 62-169) and the line-search step around it (warpmpc/jax_sqp/sparse_mpc.py
// 997-1053), batched: one thread per instance for the selection, one warp
// per instance for the fused step (its row reductions and the update of z).
//
// Arithmetic is float32 with the reference's operation order per element
// (separately rounded products and sums).  The selection reads its inputs
// element by element, so it matches a float32 restatement bit for bit; the
// fused step's sums over a row (the bound violation, q . d) are warp
// reductions, whose order differs from an XLA reduction's.
#include <math.h>

#include "common.cuh"

namespace wmpc {
namespace {

struct LsParams {
  float g_max, g_min, gamma_c, one_minus_gamma_c, armijo_factor, scale;
  int trial_cost;
};

LsParams ls_params(const wmpc_line_search_settings& s) {
  LsParams p;
  p.g_max = s.g_max;
  p.g_min = s.g_min;
  p.gamma_c = s.gamma_c;
  p.one_minus_gamma_c = 1.0f - s.gamma_c;  // (1.0 - gamma_c) in the arrays' dtype
  p.armijo_factor = s.armijo_factor;
  p.scale = s.constraint_scale;
  p.trial_cost = s.cost_accept_uses_trial_cost != 0;
  return p;
}

struct LsChoice {
  float step, cost, violation;
  int reason;
  bool accepted;
};

// line_search.py:100-151 for one instance: every candidate's branch and
// acceptance, the first accepted one (else the last step of the ladder, reason
// MAX_ITER); gathers clamp their index into range as the reference's do.
__device__ LsChoice select_step(const LsParams& p, const float* __restrict__ steps, int n_steps,
                                float base_cost, float base_viol, float armijo, const float* __restrict__ cand_cost,
                                const float* __restrict__ cand_viol, int n_cand, long long ld, unsigned char* accept_out) {
  const float constraint_bound = p.one_minus_gamma_c * base_viol;
  const float armijo_bound = base_cost + p.armijo_factor * armijo;
  const float filter_cost_bound = base_cost - p.gamma_c * base_viol;
  int first = -1, first_reason = WMPC_LINE_SEARCH_MAX_ITER;
  for (int k = 0; k < n_cand; ++k) {
    const float c = cand_cost[k * ld], v = cand_viol[k * ld];
    bool acc;
    int reason;
    if (v > p.g_max) {
      acc = v < constraint_bound;
      reason = WMPC_LINE_SEARCH_CONSTRAINT;
    } else if ((v < p.g_min) & (base_viol < p.g_min) & (armijo < 0.0f)) {
      acc = (p.trial_cost ? c : base_cost) < armijo_bound;
      reason = WMPC_LINE_SEARCH_COST;
    } else {
      acc = (c < filter_cost_bound) | (v < constraint_bound);
      reason = WMPC_LINE_SEARCH_COST_OR_CONSTRAINT;
    }
    if (accept_out) accept_out[k * ld] = acc ? 1 : 0;
    if (acc && first < 0) {
      first = k;
      first_reason = reason;
    }
  }
  const int sel = first >= 0 ? first : n_steps - 1;
  const int ci = sel < n_cand ? sel : n_cand - 1;
  const int si = sel < n_steps ? sel : n_steps - 1;
  LsChoice r;
  r.step = steps[si];
  r.cost = cand_cost[ci * ld];
  r.violation = cand_viol[ci * ld];
  r.reason = first_reason;
  r.accepted = first >= 0;
  return r;
}

__global__ void filter_line_search_kernel(LsParams p, const float* __restrict__ steps, int n_steps,
                                          const float* __restrict__ base_cost, const float* __restrict__ base_viol,
                                          const float* __restrict__ armijo, const float* __restrict__ cand_cost,
                                          const float* __restrict__ cand_viol, int n_cand, int batch,
                                          float* __restrict__ step_out, float* __restrict__ cost_out,
                                          float* __restrict__ viol_out, int32_t* __restrict__ reason_out,
                                          unsigned char* __restrict__ accepted_out,
                                          unsigned char* __restrict__ acceptance_out) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= batch) return;
  const LsChoice r = select_step(p, steps, n_steps, base_cost[b], base_viol[b], armijo[b], cand_cost + b,
                                 cand_viol + b, n_cand, batch, acceptance_out ? acceptance_out + b : nullptr);
  step_out[b] = r.step;
  if (cost_out) cost_out[b] = r.cost;
  if (viol_out) viol_out[b] = r.violation;
  if (reason_out) reason_out[b] = r.reason;
  if (accepted_out) accepted_out[b] = r.accepted ? 1 : 0;
}

// Sum over a warp; every lane returns the total.
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = v + __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// sqrt(sum max(l - g, 0)^2 + sum min(u - g, 0)^2) of one batch-major row
// (line_search.py:62-69; the two sums formed separately, then added).
__device__ __forceinline__ float row_violation_sq(const float* __restrict__ lo, const float* __restrict__ g,
                                                  const float* __restrict__ up, int m, int lane) {
  float sl = 0.0f, su = 0.0f;
  for (int r = lane; r < m; r += 32) {
    const float gr = g[r];
    const float a = fmaxf(lo[r] - gr, 0.0f);
    const float c = fminf(up[r] - gr, 0.0f);
    sl = sl + a * a;
    su = su + c * c;
  }
  return warp_sum(sl) + warp_sum(su);
}

// The same with 16-byte loads (rows 16-byte aligned, m a multiple of 4):
// four independent loads per lane in flight per trip.
__device__ __forceinline__ float row_violation_sq4(const float4* __restrict__ lo, const float4* __restrict__ g,
                                                   const float4* __restrict__ up, int m4, int lane) {
  float sl = 0.0f, su = 0.0f;
#pragma unroll 4
  for (int r = lane; r < m4; r += 32) {
    const float4 gr = g[r], l = lo[r], u = up[r];
    const float a0 = fmaxf(l.x - gr.x, 0.0f), a1 = fmaxf(l.y - gr.y, 0.0f);
    const float a2 = fmaxf(l.z - gr.z, 0.0f), a3 = fmaxf(l.w - gr.w, 0.0f);
    const float c0 = fminf(u.x - gr.x, 0.0f), c1 = fminf(u.y - gr.y, 0.0f);
    const float c2 = fminf(u.z - gr.z, 0.0f), c3 = fminf(u.w - gr.w, 0.0f);
    sl = sl + a0 * a0;
    sl = sl + a1 * a1;
    sl = sl + a2 * a2;
    sl = sl + a3 * a3;
    su = su + c0 * c0;
    su = su + c1 * c1;
    su = su + c2 * c2;
    su = su + c3 * c3;
  }
  return warp_sum(sl) + warp_sum(su);
}

__global__ void constraint_violation_kernel(const float* __restrict__ lo, const float* __restrict__ g,
                                            const float* __restrict__ up, int batch, int m, float scale,
                                            float* __restrict__ out) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= batch) return;
  const size_t o = (size_t)warp * m;
  const float vsq = row_violation_sq(lo + o, g + o, up + o, m, lane);
  if (lane == 0) out[warp] = scale * sqrtf(vsq);
}

struct StepArgs {
  LsParams p;
  const float* steps;
  int n_steps;
  const float *z, *d, *q;
  int n;
  const float *cl, *g, *cu;
  int m;
  const float *base_cost, *cand_cost, *cand_viol;
  int n_cand, batch;
  float *z_next, *step_out, *cost_out, *viol_out, *base_viol_out;
  int32_t* reason_out;
  unsigned char *accepted_out, *finite_out, *acceptance_out;
};

// sparse_mpc.py:1013-1052 from the QP solve onwards, one warp per instance:
// the baseline violation of (constraint_l, g, constraint_u), the Armijo
// metric q . d, the filter selection over the candidate evaluations, then
// z_next = z + step d and whether z_next is finite.  kVec: every row is
// 16-byte aligned with n and m multiples of 4, so rows move as float4.
template <bool kVec>
__global__ void __launch_bounds__(256) sqp_line_search_step_kernel(const __grid_constant__ StepArgs a) {
  const int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (b >= a.batch) return;
  const size_t om = (size_t)b * a.m, on = (size_t)b * a.n;
  float vsq, qd = 0.0f;
  if (kVec) {
    vsq = row_violation_sq4(reinterpret_cast<const float4*>(a.cl + om), reinterpret_cast<const float4*>(a.g + om),
                            reinterpret_cast<const float4*>(a.cu + om), a.m >> 2, lane);
    const float4* q4 = reinterpret_cast<const float4*>(a.q + on);
    const float4* d4 = reinterpret_cast<const float4*>(a.d + on);
#pragma unroll 4
    for (int j = lane; j < (a.n >> 2); j += 32) {
      const float4 qv = q4[j], dv = d4[j];
      qd = qd + qv.x * dv.x;
      qd = qd + qv.y * dv.y;
      qd = qd + qv.z * dv.z;
      qd = qd + qv.w * dv.w;
    }
  } else {
    vsq = row_violation_sq(a.cl + om, a.g + om, a.cu + om, a.m, lane);
    for (int j = lane; j < a.n; j += 32) qd = qd + a.q[on + j] * a.d[on + j];
  }
  const float base_viol = a.p.scale * sqrtf(vsq);
  const float armijo = warp_sum(qd);
  // every lane selects (same inputs, same result): no broadcast needed
  const LsChoice r = select_step(a.p, a.steps, a.n_steps, a.base_cost[b], base_viol, armijo, a.cand_cost + b,
                                 a.cand_viol + b, a.n_cand, a.batch,
                                 (a.acceptance_out && lane == 0) ? a.acceptance_out + b : nullptr);
  bool finite = true;
  if (kVec) {
    const float4* z4 = reinterpret_cast<const float4*>(a.z + on);
    const float4* d4 = reinterpret_cast<const float4*>(a.d + on);
    float4* o4 = reinterpret_cast<float4*>(a.z_next + on);
#pragma unroll 4
    for (int j = lane; j < (a.n >> 2); j += 32) {
      const float4 zv = z4[j], dv = d4[j];
      const float4 v = make_float4(zv.x + r.step * dv.x, zv.y + r.step * dv.y, zv.z + r.step * dv.z,
                                   zv.w + r.step * dv.w);
      o4[j] = v;
      finite = finite && isfinite(v.x) && isfinite(v.y) && isfinite(v.z) && isfinite(v.w);
    }
  } else {
    for (int j = lane; j < a.n; j += 32) {
      const float v = a.z[on + j] + r.step * a.d[on + j];
      a.z_next[on + j] = v;
      finite = finite && isfinite(v);
    }
  }
  finite = __all_sync(0xffffffffu, finite);
  if (lane == 0) {
    a.step_out[b] = r.step;
    if (a.cost_out) a.cost_out[b] = r.cost;
    if (a.viol_out) a.viol_out[b] = r.violation;
    if (a.base_viol_out) a.base_viol_out[b] = base_viol;
    if (a.reason_out) a.reason_out[b] = r.reason;
    if (a.accepted_out) a.accepted_out[b] = r.accepted ? 1 : 0;
    if (a.finite_out) a.finite_out[b] = finite ? 1 : 0;
  }
}

bool settings_ok(const wmpc_line_search_settings* s) {
  return s && isfinite(s->g_max) && isfinite(s->g_min) && isfinite(s->gamma_c) && isfinite(s->armijo_factor) &&
         isfinite(s->constraint_scale);
}

int warps_grid(int batch) { return (batch + 7) / 8; }  // 8 warps (256 threads) per block

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

}  // namespace
}  // namespace wmpc

using namespace wmpc;

extern "C" int wmpc_constraint_violation(const float* lower, const float* g, const float* upper, int32_t batch,
                                         int32_t m, float scale, float* out, wmpc_stream_t stream) {
  if (batch < 0 || m < 0) return fail(WMPC_ERR_INVALID_ARGUMENT, "constraint violation: negative size");
  if (batch == 0) return WMPC_OK;
  if (!out || (m > 0 && (!lower || !g || !upper)))
    return fail(WMPC_ERR_INVALID_ARGUMENT, "constraint violation: null pointer");
  constraint_violation_kernel<<<warps_grid(batch), 256, 0, static_cast<cudaStream_t>(stream)>>>(lower, g, upper,
                                                                                               batch, m, scale, out);
  WMPC_LAUNCH_CHECK();
  return WMPC_OK;
}

extern "C" int wmpc_filter_line_search(const wmpc_line_search_settings* settings, const float* step_lengths,
                                       int32_t n_steps, const float* baseline_cost,
                                       const float* baseline_violation, const float* armijo_metric,
                                       const float* candidate_costs, const float* candidate_violations,
                                       int32_t n_candidates, int32_t batch, float* step_length, float* cost,
                                       float* violation, int32_t* reason, uint8_t* accepted,
                                       uint8_t* candidate_acceptance, wmpc_stream_t stream) {
  if (!settings_ok(settings)) return fail(WMPC_ERR_INVALID_ARGUMENT, "line search: bad settings");
  if (n_steps < 1 || n_candidates < 1 || batch < 0)
    return fail(WMPC_ERR_INVALID_ARGUMENT, "line search: need >= 1 step and >= 1 candidate (got %d, %d)", n_steps,
                n_candidates);
  if (batch == 0) return WMPC_OK;
  if (!step_lengths || !baseline_cost || !baseline_violation || !armijo_metric || !candidate_costs ||
      !candidate_violations || !step_length)
    return fail(WMPC_ERR_INVALID_ARGUMENT, "line search: null pointer");
  filter_line_search_kernel<<<(batch + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      ls_params(*settings), step_lengths, n_steps, baseline_cost, baseline_violation, armijo_metric, candidate_costs,
      candidate_violations, n_candidates, batch, step_length, cost, violation, reason, accepted, candidate_acceptance);
  WMPC_LAUNCH_CHECK();
  return WMPC_OK;
}

extern "C" int wmpc_sqp_line_search_step(const wmpc_line_search_settings* settings, const wmpc_sqp_step_batch* d,
                                         wmpc_stream_t stream) {
  if (!settings_ok(settings) || !d) return fail(WMPC_ERR_INVALID_ARGUMENT, "line search step: bad settings");
  if (d->n_steps < 1 || d->n_candidates < 1 || d->batch < 0 || d->n < 0 || d->m < 0)
    return fail(WMPC_ERR_INVALID_ARGUMENT, "line search step: bad sizes");
  if (d->batch == 0) return WMPC_OK;
  if (!d->step_lengths || !d->baseline_cost || !d->candidate_costs || !d->candidate_violations || !d->step_length ||
      (d->n > 0 && (!d->z || !d->direction || !d->q || !d->z_next)) ||
      (d->m > 0 && (!d->constraint_l || !d->g || !d->constraint_u)))
    return fail(WMPC_ERR_INVALID_ARGUMENT, "line search step: null pointer");
  StepArgs a;
  a.p = ls_params(*settings);
  a.steps = d->step_lengths;
  a.n_steps = d->n_steps;
  a.z = d->z;
  a.d = d->direction;
  a.q = d->q;
  a.n = d->n;
  a.cl = d->constraint_l;
  a.g = d->g;
  a.cu = d->constraint_u;
  a.m = d->m;
  a.base_cost = d->baseline_cost;
  a.cand_cost = d->candidate_costs;
  a.cand_viol = d->candidate_violations;
  a.n_cand = d->n_candidates;
  a.batch = d->batch;
  a.z_next = d->z_next;
  a.step_out = d->step_length;
  a.cost_out = d->cost;
  a.viol_out = d->violation;
  a.base_viol_out = d->baseline_violation;
  a.reason_out = d->reason;
  a.accepted_out = d->accepted;
  a.finite_out = d->is_finite;
  a.acceptance_out = d->candidate_acceptance;
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  profile_mark_begin(s);
  const bool vec = d->n % 4 == 0 && d->m % 4 == 0 && aligned16(d->z) && aligned16(d->direction) &&
                   aligned16(d->q) && aligned16(d->z_next) && aligned16(d->constraint_l) && aligned16(d->g) &&
                   aligned16(d->constraint_u);
  if (vec)
    sqp_line_search_step_kernel<true><<<warps_grid(d->batch), 256, 0, s>>>(a);
  else
    sqp_line_search_step_kernel<false><<<warps_grid(d->batch), 256, 0, s>>>(a);
  profile_mark_end(s);
  WMPC_LAUNCH_CHECK();
  return WMPC_OK;
}

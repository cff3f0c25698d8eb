// Rigid-body quadrotor stage model of the nonlinear SQP workload (sm_100a):
// one RK4 step x_next = F(x, u) per (stage, instance) and its Jacobian
// dF/d[x, u] by forward-mode differentiation (dual numbers, four tangent
// directions per pass, four passes), written in the dynamics rows' entry
// order of the SQP stage: for each row r the structurally nonzero columns c
// of dF_r/d[x, u] (ascending; negated, as they enter g = x_next - F(x, u))
// followed by the +1 of x_next,r.
//
// The reference takes its stage functions and their derivatives from CasADi
// (warpmpc/jax_sqp/casadi_stage.py:66-189), which is absent here; this is the
// hand-written model (equations in include/warpmpc_b200.h).
#include "common.cuh"

namespace wmpc {

namespace {

constexpr int kNx = 12, kNu = 4, kNz = 16, kTan = 4;

// The structural pattern of dF/d[x, u] for one RK4 step: entries reachable in
// at most four products of the continuous dynamics' pattern (plus the
// identity of x); bit c of kRowMask[r] is column c.
__host__ __device__ constexpr unsigned row_mask(int r) {
  constexpr unsigned m[kNx] = {
      0xFE79u, 0xFEBAu, 0xFF1Cu, 0xFE18u, 0xFE18u, 0xFE38u,
      0xFE78u, 0xFEB8u, 0xFF18u, 0xFE00u, 0xFE00u, 0xF800u,
  };
  return m[r];
}

__host__ __device__ constexpr int popcount16(unsigned v) {
  int c = 0;
  for (int i = 0; i < 16; ++i) c += (v >> i) & 1u;
  return c;
}

__host__ __device__ constexpr int jac_entries() {
  int e = 0;
  for (int r = 0; r < kNx; ++r) e += popcount16(row_mask(r)) + 1;
  return e;
}

// entries per (stage, instance): the 114 structural ones and the 12 x_next ones
constexpr int kJacEntries = jac_entries();
static_assert(kJacEntries == 126, "the RK4 Jacobian pattern has 114 structural entries");

// value + kTan tangents
struct Dual {
  float v, t[kTan];
};

__device__ __forceinline__ Dual dconst(float c) {
  Dual r;
  r.v = c;
#pragma unroll
  for (int i = 0; i < kTan; ++i) r.t[i] = 0.0f;
  return r;
}
__device__ __forceinline__ Dual operator+(const Dual& a, const Dual& b) {
  Dual r;
  r.v = a.v + b.v;
#pragma unroll
  for (int i = 0; i < kTan; ++i) r.t[i] = a.t[i] + b.t[i];
  return r;
}
__device__ __forceinline__ Dual operator-(const Dual& a, const Dual& b) {
  Dual r;
  r.v = a.v - b.v;
#pragma unroll
  for (int i = 0; i < kTan; ++i) r.t[i] = a.t[i] - b.t[i];
  return r;
}
__device__ __forceinline__ Dual operator*(const Dual& a, const Dual& b) {
  Dual r;
  r.v = a.v * b.v;
#pragma unroll
  for (int i = 0; i < kTan; ++i) r.t[i] = a.t[i] * b.v + a.v * b.t[i];
  return r;
}
__device__ __forceinline__ Dual operator*(float s, const Dual& a) {
  Dual r;
  r.v = s * a.v;
#pragma unroll
  for (int i = 0; i < kTan; ++i) r.t[i] = s * a.t[i];
  return r;
}
__device__ __forceinline__ Dual operator/(const Dual& a, const Dual& b) {
  Dual r;
  const float q = a.v / b.v;
  r.v = q;
#pragma unroll
  for (int i = 0; i < kTan; ++i) r.t[i] = (a.t[i] - q * b.t[i]) / b.v;
  return r;
}
__device__ __forceinline__ void dsincos(const Dual& a, Dual& s, Dual& c) {
  float sv, cv;
  sincosf(a.v, &sv, &cv);
  s.v = sv;
  c.v = cv;
#pragma unroll
  for (int i = 0; i < kTan; ++i) {
    s.t[i] = cv * a.t[i];
    c.t[i] = -sv * a.t[i];
  }
}

// x' of the model (p' = v, eta' = W(eta) w, v' = T/m R(eta) e3 - g e3,
// w' = J^-1 (tau - w x J w)).
__device__ __forceinline__ void continuous(const wmpc_quadrotor_model& md, const Dual* x, const Dual* u, Dual* dx) {
  Dual sphi, cphi, sth, cth, spsi, cpsi;
  dsincos(x[3], sphi, cphi);
  dsincos(x[4], sth, cth);
  dsincos(x[5], spsi, cpsi);
  const Dual tth = sth / cth;
  const Dual a = (1.0f / md.mass) * (((u[0] + u[1]) + u[2]) + u[3]);
  const Dual r13 = cpsi * sth * cphi + spsi * sphi;
  const Dual r23 = spsi * sth * cphi - cpsi * sphi;
  const Dual r33 = cth * cphi;
  dx[0] = x[6];
  dx[1] = x[7];
  dx[2] = x[8];
  dx[3] = x[9] + sphi * tth * x[10] + cphi * tth * x[11];
  dx[4] = cphi * x[10] - sphi * x[11];
  dx[5] = (sphi * x[10] + cphi * x[11]) / cth;
  dx[6] = a * r13;
  dx[7] = a * r23;
  dx[8] = a * r33 - dconst(md.gravity);
  const Dual tx = md.arm * (((u[2] + u[3]) - u[0]) - u[1]);
  const Dual ty = md.arm * (((u[1] + u[2]) - u[0]) - u[3]);
  const Dual tz = md.yaw_coef * (((u[1] + u[3]) - u[0]) - u[2]);
  dx[9] = (1.0f / md.jx) * (tx - (md.jz - md.jy) * (x[10] * x[11]));
  dx[10] = (1.0f / md.jy) * (ty - (md.jx - md.jz) * (x[9] * x[11]));
  dx[11] = (1.0f / md.jz) * (tz - (md.jy - md.jx) * (x[9] * x[10]));
}

// rows: (n_stages x batch) (stage, instance) pairs; thread = one pair.
__global__ void __launch_bounds__(128) quadrotor_rk4_kernel(wmpc_quadrotor_model md, const float* __restrict__ z,
                                                            long long z_stride, int batch, int n_stages, float dt,
                                                            float* __restrict__ x_next, float* __restrict__ jac) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)batch * n_stages) return;
  const int k = (int)(idx / batch), b = (int)(idx % batch);
  const float* zk = z + (long long)b * z_stride + (long long)k * kNz;
  float zv[kNz];
#pragma unroll
  for (int c = 0; c < kNz; ++c) zv[c] = zk[c];
  // jac entries of row r start at jac_off(r): sum over earlier rows of (popcount + 1)
  float* jrow = jac ? jac + idx * (long long)kJacEntries : nullptr;
  const int passes = jac ? kNz / kTan : 1;
  for (int pass = 0; pass < passes; ++pass) {
    Dual x[kNx], u[kNu];
#pragma unroll
    for (int c = 0; c < kNz; ++c) {
      Dual d = dconst(zv[c]);
#pragma unroll
      for (int i = 0; i < kTan; ++i) d.t[i] = (c == pass * kTan + i) ? 1.0f : 0.0f;
      if (c < kNx) x[c] = d; else u[c - kNx] = d;
    }
    // RK4: acc = ((k1 + 2 k2) + 2 k3) + k4, built as the stages are evaluated
    Dual acc[kNx], k[kNx], s[kNx];
    continuous(md, x, u, acc);
#pragma unroll
    for (int i = 0; i < kNx; ++i) s[i] = x[i] + (0.5f * dt) * acc[i];
    continuous(md, s, u, k);
#pragma unroll
    for (int i = 0; i < kNx; ++i) {
      acc[i] = acc[i] + 2.0f * k[i];
      s[i] = x[i] + (0.5f * dt) * k[i];
    }
    continuous(md, s, u, k);
#pragma unroll
    for (int i = 0; i < kNx; ++i) {
      acc[i] = acc[i] + 2.0f * k[i];
      s[i] = x[i] + dt * k[i];
    }
    continuous(md, s, u, k);
    const float h = dt / 6.0f;
#pragma unroll
    for (int i = 0; i < kNx; ++i) {
      const Dual f = x[i] + h * (acc[i] + k[i]);
      if (pass == 0) x_next[idx * kNx + i] = f.v;
      if (jrow) {
        int off = 0;
#pragma unroll
        for (int r = 0; r < kNx; ++r)
          if (r < i) off += __popc(row_mask(r)) + 1;
        const unsigned m = row_mask(i);
#pragma unroll
        for (int t = 0; t < kTan; ++t) {
          const int c = pass * kTan + t;
          if (m >> c & 1u) jrow[off + __popc(m & ((1u << c) - 1u))] = -f.t[t];
        }
        if (pass == passes - 1) jrow[off + __popc(m)] = 1.0f;
      }
    }
  }
}

}  // namespace

}  // namespace wmpc

using namespace wmpc;

extern "C" int wmpc_quadrotor_rk4(const wmpc_quadrotor_model* model, const float* z, int64_t z_stride, int32_t batch,
                                  int32_t n_stages, float dt, float* x_next, float* jac, wmpc_stream_t stream) {
  if (!model || batch < 0 || n_stages < 0 || z_stride < (int64_t)kNz * n_stages)
    return fail(WMPC_ERR_INVALID_ARGUMENT, "bad quadrotor model arguments");
  if ((long long)batch * n_stages == 0) return WMPC_OK;
  if (!z || !x_next) return fail(WMPC_ERR_INVALID_ARGUMENT, "null buffer");
  static_assert(kNz <= 32, "column masks are 32-bit");
  const long long rows = (long long)batch * n_stages;
  quadrotor_rk4_kernel<<<ceil_div(rows, 128), 128, 0, static_cast<cudaStream_t>(stream)>>>(
      *model, z, z_stride, batch, n_stages, dt, x_next, jac);
  WMPC_LAUNCH_CHECK();
  return WMPC_OK;
}

extern "C" int wmpc_quadrotor_jac_pattern(int32_t* cols, int32_t* row_ptr) {
  // host copy of the entry order the kernel writes
  int e = 0;
  for (int r = 0; r < kNx; ++r) {
    if (row_ptr) row_ptr[r] = e;
    for (int c = 0; c < kNz; ++c)
      if (row_mask(r) >> c & 1u) {
        if (cols) cols[e] = c;
        ++e;
      }
    if (cols) cols[e] = kNz + r;  // x_next,r
    ++e;
  }
  if (row_ptr) row_ptr[kNx] = e;
  return WMPC_OK;
}

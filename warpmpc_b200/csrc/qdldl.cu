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
#include "stream.cuh"

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

// Staged factorization: one warp per 32-instance tile, the row's reach kept
// in a compact accumulator (one shared-memory slot per reach position instead
// of a dense n-vector), and every value a row reads from memory -- its KKT
// inputs, D^-1 of its steps' columns, the L entries of those columns above
// the row -- brought into shared memory with 4-byte asynchronous copies
// before the row's arithmetic.  The copies' addresses come from index words
// read ahead (a row's ranges two rows ahead, its per-lane words -- KKT slots
// of its inputs, columns of its steps, positions of its first L re-reads --
// one row ahead, the positions of a row's next L re-read batch while the
// current one is used), and a row's KKT inputs, which depend on no factor
// value, are copied one row ahead into a second buffer: a row waits for one
// round trip per L re-read batch and no chain of table reads.  Index words
// are read by the 32 lanes in parallel and broadcast with shuffles.  Same
// operation order as factor_instance (the reference's row program), so the
// same bits.  Lanes past the batch factor a copy of the last instance; with
// `only`, lanes of unmarked instances compute and store nothing of theirs.
struct FactorTables {
  const int* init_slot;
  const int* upd_ptr;
  const int* upd_slot;
  const int* upd_lidx;
  const int4* row_info;  // [2 n] {p0, p1, i0, i1}, {first update, update end, first input, 0}
  const int* kin_slot;   // per row, per KKT input (diagonal, then initial entries): original KKT slot
  int max_row, max_kv;
};

// per-warp shared memory in 4-byte words: ys, staged D^-1 [max_row] and L
// re-reads [lbatch] and KKT inputs of this row and the next [2 max_kv] per
// lane; update slots [lbatch], step offsets, L positions and columns
// [3 max_row] shared by the warp
__host__ __device__ inline int factor_rows_words(int max_row, int max_kv, int lbatch) {
  return (2 * max_row + lbatch + 2 * max_kv) * 32 + lbatch + 3 * max_row;
}

constexpr unsigned kLanes = 0xffffffffu;
constexpr int kRowPosRegs = 4;  // L re-read positions per lane: 32 x kRowPosRegs >= lbatch (at most 128)

struct RowPos {
  int v[kRowPosRegs];
};

struct RowWords {
  int kin;  // KKT slot of input `lane`
  int col;  // column of step p0 + lane
  RowPos pos;
};

__device__ __forceinline__ void row_positions(const FactorTables& ft, int ub, int ue, int lane, RowPos& p) {
#pragma unroll
  for (int i = 0; i < kRowPosRegs; ++i) {
    const int u = ub + lane + 32 * i;
    p.v[i] = u < ue ? __ldg(ft.upd_lidx + u) : 0;
  }
}

__device__ __forceinline__ void row_words(const Pattern& pat, const FactorTables& ft, int4 a, int4 b, int lbatch,
                                          int lane, RowWords& w) {
  const int nkv = 1 + a.w - a.z;
  w.kin = lane < nkv ? __ldg(ft.kin_slot + b.z + lane) : 0;
  w.col = a.x + lane < a.y ? __ldg(pat.proc_cols + a.x + lane) : 0;
  row_positions(ft, b.x, b.x + lbatch < b.y ? b.x + lbatch : b.y, lane, w.pos);
}

__global__ void __launch_bounds__(64) factor_rows_kernel(Pattern pat, FactorTables ft, const float* __restrict__ values,
                                                         long long ldv, int bstride, float* lx, float* d, float* dinv,
                                                         int batch, int n_tiles, int lbatch, const int* only) {
  extern __shared__ float fsm[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int tile = blockIdx.x * (blockDim.x >> 5) + warp;
  if (tile >= n_tiles) return;
  const int b = tile * 32 + lane;
  const int bb = b < batch ? b : batch - 1;
  const bool keep = b < batch && (only == nullptr || only[b] != 0);
  float* wbase = fsm + (size_t)warp * factor_rows_words(ft.max_row, ft.max_kv, lbatch);
  float* ys = wbase + lane;
  float* dst = ys + ft.max_row * 32;
  float* lst = dst + ft.max_row * 32;
  float* kst = lst + lbatch * 32;
  float* kst_next = kst + ft.max_kv * 32;
  int* slot_w = reinterpret_cast<int*>(wbase + (2 * ft.max_row + lbatch + 2 * ft.max_kv) * 32);
  int* off_w = slot_w + lbatch;
  int* lid_w = off_w + ft.max_row;
  const float* vb = values + (long long)bb * bstride;
  const int n = pat.n;
  // L re-reads of updates [ub, ue) (positions of ub + lane + 32 i in p)
  auto stage_updates = [&](int ub, int ue, const RowPos& p) {
#pragma unroll
    for (int i = 0; i < kRowPosRegs; ++i) {
      const int base = ub + 32 * i;
      if (base >= ue) break;
      const int u = base + lane;
      if (u < ue) cp_async4(slot_w + (u - ub), ft.upd_slot + u);
      const int cnt = ue - base < 32 ? ue - base : 32;
      for (int j = 0; j < cnt; ++j)
        cp_async4(lst + (base + j - ub) * 32, lx + (long long)__shfl_sync(kLanes, p.v[i], j) * batch + bb);
    }
  };
  // KKT inputs [first, nkv) of a row (slot of input first + lane in slot)
  auto copy_inputs = [&](float* dstk, int first, int nkv, int slot) {
    const int cnt = nkv - first < 32 ? nkv - first : 32;
    for (int j = 0; j < cnt; ++j) cp_async4(dstk + (first + j) * 32, vb + (long long)__shfl_sync(kLanes, slot, j) * ldv);
  };
  int4 ca = __ldg(ft.row_info), cb = __ldg(ft.row_info + 1);
  int4 na = n > 1 ? __ldg(ft.row_info + 2) : ca, nb = n > 1 ? __ldg(ft.row_info + 3) : cb;
  RowWords wc;
  row_words(pat, ft, ca, cb, lbatch, lane, wc);
  copy_inputs(kst, 0, 1 + ca.w - ca.z, wc.kin);
  cp_async_commit();
  for (int k = 0; k < n; ++k) {
    const int p0 = ca.x, p1 = ca.y, i0 = ca.z, i1 = ca.w;
    const int u_end = cb.y, kbase = cb.z;
    int ub = cb.x;
    int ue = ub + lbatch < u_end ? ub + lbatch : u_end;
    const int nkv = 1 + i1 - i0;
    // reads ahead: the ranges of row k + 2, the words of row k + 1
    int4 nna = na, nnb = nb;
    if (k + 2 < n) {
      nna = __ldg(ft.row_info + 2 * (k + 2));
      nnb = __ldg(ft.row_info + 2 * (k + 2) + 1);
    }
    RowWords wn = wc;
    if (k + 1 < n) row_words(pat, ft, na, nb, lbatch, lane, wn);
    // KKT inputs past the first 32, D^-1 of the steps' columns, the step tables, the first L batch
    for (int base = 32; base < nkv; base += 32)
      copy_inputs(kst, base, nkv, base + lane < nkv ? __ldg(ft.kin_slot + kbase + base + lane) : 0);
    for (int base = p0; base < p1; base += 32) {
      const int e = base + lane;
      const int col = base == p0 ? wc.col : (e < p1 ? __ldg(pat.proc_cols + e) : 0);
      if (e < p1) {
        cp_async4(off_w + (e - p0), pat.proc_offsets + e);
        cp_async4(lid_w + (e - p0), pat.proc_lidx + e);
      }
      const int cnt = p1 - base < 32 ? p1 - base : 32;
      for (int j = 0; j < cnt; ++j)
        cp_async4(dst + (base + j - p0) * 32, dinv + (long long)__shfl_sync(kLanes, col, j) * batch + bb);
    }
    stage_updates(ub, ue, wc.pos);
    cp_async_commit();
    RowPos pnext;
    row_positions(ft, ue, ue + lbatch < u_end ? ue + lbatch : u_end, lane, pnext);
    if (k + 1 < n) copy_inputs(kst_next, 0, 1 + na.w - na.z, wn.kin);
    cp_async_commit();
    cp_async_wait_group<1>();  // everything but the next row's inputs
    __syncwarp();
    for (int s = 0; s < p1 - p0; ++s) ys[s * 32] = 0.0f;
    float dk = kst[0];
    for (int base = 0; base < nkv - 1; base += 32) {
      const int e = i0 + base + lane;
      const int slot = e < i1 ? __ldg(ft.init_slot + e) : 0;
      const int cnt = nkv - 1 - base < 32 ? nkv - 1 - base : 32;
      for (int j = 0; j < cnt; ++j) {
        const int sl = __shfl_sync(kLanes, slot, j);
        ys[sl * 32] = ys[sl * 32] + kst[(1 + base + j) * 32];
      }
    }
    int u = ub;
    for (int e = 0; e < p1 - p0; ++e) {
      const int off = off_w[e];
      const float val = ys[e * 32];
      for (int q = 0; q < off; ++q, ++u) {
        if (u == ue) {  // next batch of this row's L re-reads
          __syncwarp();
          ub = ue;
          ue = ub + lbatch < u_end ? ub + lbatch : u_end;
          stage_updates(ub, ue, pnext);
          row_positions(ft, ue, ue + lbatch < u_end ? ue + lbatch : u_end, lane, pnext);
          cp_async_wait_all();
          __syncwarp();
        }
        const int su = slot_w[u - ub];
        ys[su * 32] = ys[su * 32] - lst[(u - ub) * 32] * val;
      }
      const float lval = val * dst[e * 32];
      if (keep) lx[(long long)lid_w[e] * batch + b] = lval;
      dk = dk - val * lval;
    }
    if (keep) {
      d[(long long)k * batch + b] = dk;
      dinv[(long long)k * batch + b] = 1.0f / dk;
    }
    __syncwarp();  // the warp-shared tables are restaged by the next row
    ca = na;
    cb = nb;
    na = nna;
    nb = nnb;
    wc = wn;
    float* t = kst;
    kst = kst_next;
    kst_next = t;
  }
  cp_async_wait_all();
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

int launch_factor_plan(const wmpc_plan& plan, const float* values, long long ldv, int bstride, float* lx, float* d,
                       float* dinv, int batch, void* ws, size_t ws_bytes, cudaStream_t stream, const int* only) {
  if (batch <= 0) return WMPC_OK;
  const Pattern& pat = plan.pat;
  if (plan.fac_upd_ptr && !env_disabled("WMPC_FACTOR_STAGED_OFF")) {
    int num_sms = 0;
    if (cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, plan.device) != cudaSuccess) {
      (void)cudaGetLastError();
      num_sms = 148;
    }
    const int warps = 2;
    const int n_tiles = (batch + 31) / 32;
    // L-batch sized so that every tile's warp can be resident at once
    const int per_sm = (n_tiles + num_sms - 1) / num_sms;
    const int budget = (200 * 1024 / 4) / (per_sm > 0 ? per_sm : 1);
    int lbatch = (budget - factor_rows_words(plan.fac_max_row, plan.fac_max_kv, 0)) / 33;
    lbatch = lbatch < 8 ? 8 : (lbatch > 128 ? 128 : lbatch);
    const size_t smem = (size_t)warps * factor_rows_words(plan.fac_max_row, plan.fac_max_kv, lbatch) * sizeof(float);
    if (smem <= (size_t)kMaxSmemBytes) {
      WMPC_CUDA_TRY(cudaFuncSetAttribute(factor_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      const FactorTables ft{plan.fac_init_slot, plan.fac_upd_ptr, plan.fac_upd_slot, plan.fac_upd_lidx,
                            plan.fac_row_info, plan.fac_kin_slot, plan.fac_max_row, plan.fac_max_kv};
      profile_mark_begin(stream, kProfileFactor);
      factor_rows_kernel<<<ceil_div(n_tiles, warps), warps * 32, smem, stream>>>(pat, ft, values, ldv, bstride, lx, d,
                                                                               dinv, batch, n_tiles, lbatch, only);
      profile_mark_end(stream, kProfileFactor);
      WMPC_LAUNCH_CHECK();
      return WMPC_OK;
    }
  }
  return launch_factor(pat, values, ldv, bstride, lx, d, dinv, batch, ws, ws_bytes, stream, only);
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

// Streaming persistent OSQP-ADMM kernels (sm_100a).
//
// factor_stream_kernel: KKT assembly + LDL^T factorization, one lane per
//   instance, compact accumulator (one shared-memory slot per etree-reach
//   position instead of a dense work vector), L and D^-1 written into both
//   sweep streams (unit layout, see stream.cuh); flags zero pivots.
// admm_stream_kernel: one CTA per SM walks instance tiles; a producer warp
//   streams every chunk of the factor into a shared-memory ring with
//   cp.async.bulk (mbarrier completion), a consumer warp runs, per ADMM
//   iteration, the forward sweep (row-gather), the backward sweep (D^-1 and
//   L^T, column form, reverse order) and, as soon as the backward sweep is
//   done with a KKT index, its ADMM update, writing the next iteration's
//   right-hand side in place.  The sweeps walk 4-entry units with the next
//   unit's loads issued before the current unit's arithmetic (registers
//   forward the one value that may still be in flight).  The work vector
//   (KKT dimension + 1 zero row, x 32 lanes) stays in shared memory for all
//   iterations of a tile.
//
// Arithmetic is the reference's operation order (warp_backend.py:41-101,
// 176-218; solver.py:806-820) with separately rounded products and sums.
#include <algorithm>

#include "osqp.cuh"
#include "stream.cuh"

namespace wmpc {

struct OsqpInputs {
  const float* pT; long long ldp; int sbp;
  const float* aT; long long lda; int sba;
  // per-instance 1/rho rows [m][batch] (rho adaptation; null: the plan's -1/rho values)
  const float* rT = nullptr; long long ldr = 0;
  __device__ __forceinline__ float p(int j, int b) const { return pT[(long long)j * ldp + (long long)b * sbp]; }
  __device__ __forceinline__ float a(int j, int b) const { return aT[(long long)j * lda + (long long)b * sba]; }
};


// ---------------------------------------------------------------------------
// factorization into the stream layout
// ---------------------------------------------------------------------------

// Per-warp shared memory of the factorization, in 4-byte words: per lane
// (x 32) ys [max_row_nnz] (compact accumulator), staged D^-1 of the row's
// steps [max_row_nnz], staged L re-reads [lbatch], staged raw KKT inputs of
// this row and of the next [2 x max_row_kv]; shared by the warp: update
// slots [lbatch] and per-step update counts, backward- and forward-stream
// offsets [3 x max_row_nnz].
__host__ __device__ inline int factor_warp_words(const StreamPlan& sp, int lbatch) {
  const int r = sp.max_row_nnz > 0 ? sp.max_row_nnz : 1;
  return (2 * r + lbatch + 2 * sp.max_row_kv) * 32 + lbatch + 3 * r;
}

// Up-looking LDL^T (QDLDL row program, warp_backend.py:41-101), one lane per
// instance, one warp per tile.  Every value a row reads from memory -- its
// KKT inputs, D^-1 of the columns it eliminates with, and the L entries of
// those columns above the row (written by earlier rows) -- is independent of
// the row's own arithmetic, so each row first stages them into shared memory
// with asynchronous copies, then runs the program on shared memory.
// The copies' addresses come from index words read ahead, so that a row
// waits for one round trip (its staged values) and no chain of table reads:
// the row's ranges two rows ahead (row_info), the next row's per-lane words
// (KKT input descriptors, D^-1 offsets of its steps, positions of its first
// L re-reads) one row ahead, the next row's raw KKT inputs (they depend on
// no factor value) copied one row ahead into a second buffer, and the
// positions of a row's next L re-read batch while the current one is used.
// Index words are read by the 32 lanes in parallel (one word each, 32 at a
// time) and broadcast with shuffles.
constexpr unsigned kFullMask = 0xffffffffu;
constexpr int kPosRegs = 4;  // L re-read positions per lane: 32 x kPosRegs >= lbatch (at most 128)
constexpr int kFacStep = 8;  // updates of one step loaded before their arithmetic

struct PosBatch {
  int v[kPosRegs];
};

// positions of updates [ub, ue), lane holding update ub + lane + 32 i
__device__ __forceinline__ void load_positions(const StreamPlan& sp, int ub, int ue, int lane, PosBatch& p) {
#pragma unroll
  for (int i = 0; i < kPosRegs; ++i) {
    const int u = ub + lane + 32 * i;
    p.v[i] = u < ue ? __ldg(sp.upd_pos + u) : 0;
  }
}

// Stage the L re-reads of updates [ub, ue) (ue - ub <= 32 kPosRegs): values
// per lane (each lane its own instance's entry), slots warp-shared.
__device__ __forceinline__ void stage_updates(const StreamPlan& sp, const float* Lu, float* lst, int* slot_w, int lane,
                                              int ub, int ue, const PosBatch& p) {
#pragma unroll
  for (int i = 0; i < kPosRegs; ++i) {
    const int base = ub + 32 * i;
    if (base >= ue) break;
    const int u = base + lane;
    if (u < ue) cp_async4(slot_w + (u - ub), sp.upd_slot + u);
    const int cnt = ue - base < 32 ? ue - base : 32;
    for (int j = 0; j < cnt; ++j) cp_async4(lst + (base + j - ub) * 32, Lu + __shfl_sync(kFullMask, p.v[i], j));
  }
}

// How KKT input j of a row is formed from its staged raw input
// (solver.py:764-776), one descriptor per input in row-program order (the
// diagonal, then the row's initial entries): x the P/A entry (-1: none;
// nnz_p + nnz_a + r: constraint r's 1/rho row), y kind (0 the base value
// `add`, 1 a P entry raw * p_scale + sigma-on-the-diagonal `add`, 2 an A
// entry raw * a_scale, 3 -raw: the instance's own -1/rho), z scale bits,
// w add bits.
__device__ __forceinline__ float kkt_input_value(int kind, float scale, float add, float raw) {
  if (kind == 0) return add;
  if (kind == 1) return raw * scale + add;
  if (kind == 3) return -raw;
  return raw * scale;
}

__device__ __forceinline__ int4 kin_desc_of(const int4* kin, int base, int j, int nkv) {
  return j < nkv ? __ldg(kin + base + j) : make_int4(-1, 0, 0, 0);
}

// the raw KKT inputs [first, nkv) of a row (descriptor of input first + lane in d)
__device__ __forceinline__ void copy_kkt_inputs(const Osqp& o, const OsqpInputs& in, const float* pin,
                                                const float* ain, const float* rin, float* kst, int first, int nkv,
                                                int4 d) {
  const int cnt = nkv - first < 32 ? nkv - first : 32;
  for (int j = 0; j < cnt; ++j) {
    const int src = __shfl_sync(kFullMask, d.x, j);
    if (src >= 0)
      cp_async4(kst + (first + j) * 32,
                src < o.nnz_p ? pin + (long long)src * in.ldp
                : src < o.nnz_p + o.nnz_a ? ain + (long long)(src - o.nnz_p) * in.lda
                                          : rin + (long long)(src - o.nnz_p - o.nnz_a) * in.ldr);
  }
}

// cnt (<= W) updates of one step, to distinct slots: every load, then every store.
template <int W>
__device__ __forceinline__ void update_batch(const int* slot, const float* lv, float* ys, float val, int cnt) {
  int su[W];
  float yv[W], l[W];
#pragma unroll
  for (int i = 0; i < W; ++i)
    if (i < cnt) {
      su[i] = slot[i];
      l[i] = lv[i * 32];
      yv[i] = ys[su[i] * 32];
    }
#pragma unroll
  for (int i = 0; i < W; ++i)
    if (i < cnt) ys[su[i] * 32] = yv[i] - l[i] * val;
}

// A row's ranges: a = {p0, p1, i0, i1} (program steps, initial entries),
// b = {ub, uend, doff, kin base} (updates, D^-1 offset of the row, first
// KKT input descriptor).
struct FacRow {
  int4 a, b;
};

// the per-lane words of a row read ahead
struct FacRowWords {
  int4 kin;      // descriptor of KKT input `lane`
  int sdoff;     // D^-1 offset of step p0 + lane
  PosBatch pos;  // positions of the first L re-read batch
};

__device__ __forceinline__ FacRow load_fac_row(const StreamPlan& sp, int k) {
  FacRow r;
  r.a = __ldg(sp.row_info + 2 * k);
  r.b = __ldg(sp.row_info + 2 * k + 1);
  return r;
}

__device__ __forceinline__ void load_row_words(const int4* kin, const StreamPlan& sp, const FacRow& r, int lbatch,
                                               int lane, FacRowWords& w) {
  const int p0 = r.a.x, p1 = r.a.y, nkv = 1 + r.a.w - r.a.z;
  w.kin = kin_desc_of(kin, r.b.w, lane, nkv);
  w.sdoff = p0 + lane < p1 ? __ldg(sp.step_doff + p0 + lane) : 0;
  const int ub = r.b.x, uend = r.b.y;
  load_positions(sp, ub, ub + lbatch < uend ? ub + lbatch : uend, lane, w.pos);
}

// With per-instance 1/rho rows (in.rT) the rows' -1/rho inputs come from
// them (kin_desc_rho); with `only`, a tile none of whose instances is marked
// keeps its factorization (a marked tile's unmarked lanes recompute theirs
// from unchanged inputs: the same bits).
__global__ void __launch_bounds__(64, 1) factor_stream_kernel(Pattern pat, StreamPlan sp, Osqp o, OsqpInputs in,
                                                            float* __restrict__ bstream, float* __restrict__ fstream,
                                                            int* __restrict__ status, int n_tiles, int batch,
                                                            int lbatch, const int* __restrict__ only) {
  extern __shared__ float fsm[];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int tile = blockIdx.x * (blockDim.x >> 5) + warp;
  if (tile >= n_tiles) return;
  const int b = tile * 32 + lane;
  if (only != nullptr && !__any_sync(kFullMask, b < batch && only[b] != 0)) return;
  const int4* kin = in.rT ? o.kin_desc_rho : o.kin_desc;
  const int bb = b < batch ? b : batch - 1;  // padding lanes factor a copy of the last instance
  const int rmax = sp.max_row_nnz > 0 ? sp.max_row_nnz : 1;
  const int kvmax = sp.max_row_kv;
  float* wbase = fsm + (size_t)warp * factor_warp_words(sp, lbatch);
  float* ys = wbase + lane;
  float* dst = ys + rmax * 32;
  float* lst = dst + rmax * 32;
  float* kst = lst + lbatch * 32;        // raw KKT inputs of this row
  float* kst_next = kst + kvmax * 32;    // and of the next
  int* slot_w = reinterpret_cast<int*>(wbase + (2 * rmax + lbatch + 2 * kvmax) * 32);  // warp-shared
  int* off_w = slot_w + lbatch;
  int* boff_w = off_w + rmax;
  int* foff_w = boff_w + rmax;
  float* Lb = bstream + (size_t)tile * sp.blen;
  float* F = fstream + (size_t)tile * sp.flen + lane * 4;
  float* Lu = Lb + lane * 4;  // unit entries: lane stride 4
  float* Ld = Lb + lane;      // D^-1 rows: lane stride 1
  const float* pin = in.pT + (long long)bb * in.sbp;
  const float* ain = in.aT + (long long)bb * in.sba;
  const float* rin = in.rT ? in.rT + bb : nullptr;
  const int n = pat.n;
  bool bad = false;
  // row 0's ranges and words, row 1's ranges, row 0's raw inputs
  FacRow cur = load_fac_row(sp, 0);
  FacRow nxt = n > 1 ? load_fac_row(sp, 1) : cur;
  FacRowWords wc;
  load_row_words(kin, sp, cur, lbatch, lane, wc);
  copy_kkt_inputs(o, in, pin, ain, rin, kst, 0, 1 + cur.a.w - cur.a.z, wc.kin);
  cp_async_commit();
  for (int k = 0; k < n; ++k) {
    const int p0 = cur.a.x, p1 = cur.a.y, i0 = cur.a.z, i1 = cur.a.w;
    const int u_end = cur.b.y, doff_k = cur.b.z, kbase = cur.b.w;
    const int nkv = 1 + i1 - i0;
    int ub = cur.b.x;
    int ue = ub + lbatch < u_end ? ub + lbatch : u_end;
    // reads ahead: the ranges of row k + 2, the words of row k + 1
    FacRow nn = nxt;
    if (k + 2 < n) nn = load_fac_row(sp, k + 2);
    FacRowWords wn = wc;
    if (k + 1 < n) load_row_words(kin, sp, nxt, lbatch, lane, wn);
    // stage this row's reads: raw inputs past the first 32, D^-1 of its
    // steps, step tables, the first batch of L re-reads
    for (int base = 32; base < nkv; base += 32)
      copy_kkt_inputs(o, in, pin, ain, rin, kst, base, nkv, kin_desc_of(kin, kbase, base + lane, nkv));
    for (int base = p0; base < p1; base += 32) {
      const int e = base + lane;
      const int doff = base == p0 ? wc.sdoff : (e < p1 ? __ldg(sp.step_doff + e) : 0);
      if (e < p1) {
        cp_async4(off_w + (e - p0), pat.proc_offsets + e);
        cp_async4(boff_w + (e - p0), sp.proc_boff + e);
        cp_async4(foff_w + (e - p0), sp.proc_foff + e);
      }
      const int cnt = p1 - base < 32 ? p1 - base : 32;
      for (int j = 0; j < cnt; ++j) cp_async4(dst + (base + j - p0) * 32, Ld + __shfl_sync(kFullMask, doff, j));
    }
    stage_updates(sp, Lu, lst, slot_w, lane, ub, ue, wc.pos);
    cp_async_commit();
    // the positions of the row's next L re-read batch, if any
    PosBatch pnext;
    load_positions(sp, ue, ue + lbatch < u_end ? ue + lbatch : u_end, lane, pnext);
    // the next row's raw inputs into the other buffer (they depend on no factor value)
    if (k + 1 < n) copy_kkt_inputs(o, in, pin, ain, rin, kst_next, 0, 1 + nxt.a.w - nxt.a.z, wn.kin);
    cp_async_commit();
    cp_async_wait_group<1>();  // everything but the next row's inputs
    __syncwarp();
    // the row program (the reference's order: diagonal input, then the
    // initial entries in order, then the steps)
    for (int s = 0; s < p1 - p0; ++s) ys[s * 32] = 0.0f;
    float dk = 0.0f;
    for (int base = 0; base < nkv; base += 32) {
      const int4 kc = base == 0 ? wc.kin : kin_desc_of(kin, kbase, base + lane, nkv);
      const int jl = base + lane;
      const int islot = (jl > 0 && jl < nkv) ? __ldg(sp.init_slot + i0 + jl - 1) : 0;
      const int cnt = nkv - base < 32 ? nkv - base : 32;
      for (int jj = 0; jj < cnt; ++jj) {
        const float v = kkt_input_value(__shfl_sync(kFullMask, kc.y, jj),
                                        __int_as_float(__shfl_sync(kFullMask, kc.z, jj)),
                                        __int_as_float(__shfl_sync(kFullMask, kc.w, jj)), kst[(base + jj) * 32]);
        const int s = __shfl_sync(kFullMask, islot, jj);
        if (base + jj == 0) {
          dk = v;
        } else {
          ys[s * 32] = ys[s * 32] + v;
        }
      }
    }
    int u = ub;
    for (int e = 0; e < p1 - p0; ++e) {
      const int off = off_w[e];
      const float val = ys[e * 32];
      // a step's updates target distinct slots (the rows of one column):
      // kFacStep of them at a time, every load issued before the stores
      for (int q = 0; q < off;) {
        if (u == ue) {  // next batch of this row's L re-reads
          __syncwarp();
          ub = ue;
          ue = ub + lbatch < u_end ? ub + lbatch : u_end;
          stage_updates(sp, Lu, lst, slot_w, lane, ub, ue, pnext);
          load_positions(sp, ue, ue + lbatch < u_end ? ue + lbatch : u_end, lane, pnext);
          cp_async_wait_all();
          __syncwarp();
        }
        int cnt = off - q < ue - u ? off - q : ue - u;
        cnt = cnt < kFacStep ? cnt : kFacStep;
        // the batch width by the count (predicated-off slots still issue)
        if (cnt == 1) {
          const int su = slot_w[u - ub];
          ys[su * 32] = ys[su * 32] - lst[(u - ub) * 32] * val;
        } else if (cnt <= 4) {
          update_batch<4>(slot_w + (u - ub), lst + (u - ub) * 32, ys, val, cnt);
        } else {
          update_batch<kFacStep>(slot_w + (u - ub), lst + (u - ub) * 32, ys, val, cnt);
        }
        q += cnt;
        u += cnt;
      }
      const float lval = val * dst[e * 32];
      Lu[boff_w[e]] = lval;
      const int fo = foff_w[e];  // forward stream, or (-1 - offset) a releaser forward unit in the backward stream
      if (fo >= 0) F[fo] = lval; else Lu[-1 - fo] = lval;
      dk = dk - val * lval;
    }
    const float di = 1.0f / dk;
    bad |= !(di != 0.0f) || !isfinite(di);
    Ld[doff_k] = di;
    __syncwarp();  // the warp-shared tables are restaged by the next row
    cur = nxt;
    nxt = nn;
    wc = wn;
    float* t = kst;
    kst = kst_next;
    kst_next = t;
  }
  cp_async_wait_all();
  for (int i = 0; i < sp.n_pad_b; ++i) Lu[__ldg(sp.pad_boff + i)] = 0.0f;
  for (int i = 0; i < sp.n_pad_f; ++i) F[__ldg(sp.pad_foff + i)] = 0.0f;
  if (status) status[b] = bad ? WMPC_STATUS_ZERO_PIVOT : 0;
}

// ---------------------------------------------------------------------------
// state layout conversions: symbolic-major (KKT row, instance) <-> tile-major U order
// ---------------------------------------------------------------------------

// ADMM state per tile in release order U, per (index, lane) an iterate --
// rewritten every iteration -- and parameters -- only read --, each in
// arrays of the layout [tile][U][lane]: a primal index's x and sigma-scaled
// q as 4-byte records (state_p, param_p), a constraint's (z, y) and (l, u)
// as 8-byte records (state, param);
// and the scaled primal residual (A x - z)_r of a constraint (0 for a primal
// index), formed when `form` (a warm start whose termination is checked; a
// cold start's x = z = 0 gives 0; without checks nothing reads it).
__global__ void state_to_stream_kernel(StreamPlan sp, Osqp o, OsqpInputs in, bool form, const float* __restrict__ x,
                                       const float* __restrict__ z, const float* __restrict__ y,
                                       const float* __restrict__ qs, const float* __restrict__ ls,
                                       const float* __restrict__ us, float2* __restrict__ state,
                                       float2* __restrict__ param, float* __restrict__ state_p,
                                       float* __restrict__ param_p, float* __restrict__ pres, int batch,
                                       int n_tiles) {
  const int n_primal = o.n;
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n_tiles * 32) return;
  const int bb = b < batch ? b : batch - 1;
  const int tile = b >> 5, lane = b & 31;
  for (int u = blockIdx.y; u < sp.n; u += gridDim.y) {
    const int k = __ldg(sp.u_orig + u);
    const size_t dst = ((size_t)tile * sp.n + u) * 32 + lane;
    if (k < n_primal) {
      state_p[dst] = x[(size_t)k * batch + bb];
      param_p[dst] = qs[(size_t)k * batch + bb];
      pres[dst] = 0.0f;
    } else {
      const int r = k - n_primal;
      const float zr = z[(size_t)r * batch + bb];
      state[dst] = make_float2(zr, y[(size_t)r * batch + bb]);
      param[dst] = make_float2(ls[(size_t)r * batch + bb], us[(size_t)r * batch + bb]);
      float e = 0.0f;
      if (form) {
        float ax = 0.0f;
        const int e0 = __ldg(o.a_row_ptr + r), e1 = __ldg(o.a_row_ptr + r + 1);
        for (int t = e0; t < e1; ++t) {
          const int j = __ldg(o.a_row_ent + t);
          ax = ax + (in.a(j, bb) * __ldg(o.a_scale + j)) * x[(size_t)__ldg(o.a_cols + j) * batch + bb];
        }
        e = ax - zr;
      }
      pres[dst] = e;
    }
  }
}

__global__ void stream_to_state_kernel(StreamPlan sp, int n_primal, const float2* __restrict__ state,
                                       const float* __restrict__ state_p,
                                       float* __restrict__ x, float* __restrict__ z, float* __restrict__ y,
                                       int batch) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= batch) return;
  const int tile = b >> 5, lane = b & 31;
  for (int u = blockIdx.y; u < sp.n; u += gridDim.y) {
    const int o = __ldg(sp.u_orig + u);
    const size_t at = ((size_t)tile * sp.n + u) * 32 + lane;
    if (o < n_primal) {
      x[(size_t)o * batch + b] = state_p[at];
    } else {
      const float2 v = state[at];
      const int r = o - n_primal;
      z[(size_t)r * batch + b] = v.x;
      y[(size_t)r * batch + b] = v.y;
    }
  }
}

// ---------------------------------------------------------------------------
// streaming ADMM kernel
// ---------------------------------------------------------------------------

// One class of instances (one sparsity pattern) in a launch.
struct StreamJob {
  StreamPlan sp;
  const float* bstream;
  const float* fstream;
  float2* state;  // [tile][U][lane] constraint iterate records (z, y)
  const float2* param;  // [tile][U][lane] constraint parameter records (l, u)
  float* state_p;  // [tile][U][lane] primal iterate records x
  const float* param_p;  // [tile][U][lane] primal parameter records (sigma-scaled q)
  float* pres;    // [tile][U][lane] scaled primal residual of each constraint
  float* rhs;     // frontier form: [tile][n][lane] right-hand sides (release -> forward stage)
  float* fwd;     // frontier form: [tile][n][lane] forward results (sweep -> backward stage)
  int* iters;     // [batch] iterations run (may be null)
  int n_tiles, max_iter, batch;
  int check_every;  // > 0: stop a tile once every lane's largest unscaled iterate change <= chg_eps
  float chg_eps;
  float sigma, alpha, one_minus_alpha;
  const float* rho_b;    // per-instance rho (admm_stream_kernel<.., true>), see StreamJobDesc
  const int* rho_count;
};

constexpr int kMaxStreamJobs = 6;

// A launch: up to kMaxStreamJobs classes; CTAs walk the combined tile list
// (job 0's tiles first; jobs are ordered by cost).  The shared-memory layout
// is sized for the largest class.
struct StreamArgs {
  StreamJob job[kMaxStreamJobs];
  int tile_end[kMaxStreamJobs];  // cumulative tile counts
  int n_jobs;
  int x_rows;       // work vector rows reserved (largest KKT dimension + 2)
  int* error;       // one word: 0 ok, 1 pipeline timeout
  int lstages, sstages;
  int meta_bytes;   // per L stage, 128-byte multiple
  int lbytes;       // per L stage L area
  int sbytes;       // per S stage: max_rel x 32 lanes x (8 iterate + 8 parameter) bytes (+ 4 of residuals)
  int pres_off;     // byte offset of the residuals in an S stage (end of the records; the
                    // parameter records start at pres_off / 2)
  int rec_off;      // frontier form: byte offset in an S stage of the releases' header
                    // {nrel, u0, nprim, 0} and, after it, their 16-byte records
  unsigned long long wait_limit_ns;  // give-up time of every handshake wait (the drain keeps kWaitLimitNs)
};
static_assert(sizeof(StreamArgs) <= 4000, "launch arguments exceed the kernel parameter space");

__device__ __forceinline__ int job_of(const StreamArgs& a, int g) {
  int c = 0;
  while (c + 1 < a.n_jobs && g >= a.tile_end[c]) ++c;
  return c;
}

enum : int { kItemRel = 0, kItemFwd = 1, kItemBwd = 2 };

// 2 s: a healthy wait is microseconds.  The default give-up time of the
// warps' handshake waits (WMPC_STREAM_WAIT_LIMIT_NS overrides it per launch,
// so that a test can make them run out), and always the time the abort
// drain gives the bulk copies already issued (those always complete).
constexpr uint64_t kWaitLimitNs = 2000000000ull;

// ring position: stage index and the parity of the lap
struct Ring {
  uint32_t stage, phase;
  __device__ __forceinline__ void advance(int stages) {
    if (++stage == (uint32_t)stages) {
      stage = 0;
      phase ^= 1u;
    }
  }
};

// Visit one tile's items: backward chunks descending with releases only
// (first right-hand side), then per iteration the forward chunks ascending
// and the backward chunks descending.  Before every iteration after the first
// cont(it) decides: 1 go on, 0 the tile converged (stop here), -1 abort.
// Returns false when f or cont aborts.
template <typename F, typename C>
__device__ __forceinline__ bool traverse(int n_chunks, int n_fchunks, int max_iter, F& f, C& cont) {
  for (int ch = n_chunks - 1; ch >= 0; --ch)
    if (!f(kItemRel, ch)) return false;
  for (int it = 0; it < max_iter; ++it) {
    if (it > 0) {
      const int c = cont(it);
      if (c < 0) return false;
      if (c == 0) return true;
    }
    for (int ch = 0; ch < n_fchunks; ++ch)
      if (!f(kItemFwd, ch)) return false;
    for (int ch = n_chunks - 1; ch >= 0; --ch)
      if (!f(kItemBwd, ch)) return false;
  }
  return true;
}

// Early termination is decided before iteration `it` when checking is on and
// `it` is a multiple of the check period.
__device__ __forceinline__ bool check_point(int check_every, int it) { return check_every > 0 && it % check_every == 0; }

// Shared-memory layout: X [n + 2][32] | L ring | S ring | barriers | flags
__host__ __device__ inline size_t stream_smem_bytes(int n, int lstages, int sstages, int lstage_bytes,
                                                    int sstage_bytes) {
  return (size_t)(n + 2) * 128 + (size_t)lstages * lstage_bytes + (size_t)sstages * sstage_bytes +
         16 * (size_t)(lstages + sstages) + 32;  // barriers; abort flag, three counters, the stop item
}

// One unit's operands, loaded ahead of its arithmetic.
struct UnitOps {
  int4 src, ctl;  // meta; ctl: target byte offset, flags | D^-1 offset, L offset, store byte offset
  float4 l;
  float x0, x1, x2, x3, t, d;
};

__device__ __forceinline__ void load_meta(const int4* __restrict__ mu, int u, UnitOps& r) {
  r.src = mu[2 * u];
  r.ctl = mu[2 * u + 1];
}

// lane_l: this lane's 16 bytes of unit 0 of the stage (lst + lane * 16)
// tb: where the target offsets point (the work vector, or the stage's L area
// in the frontier form), this lane's column
template <bool kBackward>
__device__ __forceinline__ void load_data(const unsigned char* lane_l, const unsigned char* lst,
                                          const unsigned char* xb, const unsigned char* tb, int lane, UnitOps& r) {
  r.l = *reinterpret_cast<const float4*>(lane_l + r.ctl.z);
  r.x0 = *reinterpret_cast<const float*>(xb + r.src.x);
  r.x1 = *reinterpret_cast<const float*>(xb + r.src.y);
  r.x2 = *reinterpret_cast<const float*>(xb + r.src.z);
  r.x3 = *reinterpret_cast<const float*>(xb + r.src.w);
  r.t = *reinterpret_cast<const float*>(tb + r.ctl.x);
  if (kBackward) r.d = *reinterpret_cast<const float*>(lst + (r.ctl.y >> kUnitDoffShift) + lane * 4);
}

// flags & mask ? a : b, as a predicated select (no branch)
__device__ __forceinline__ float select_flag(int flags, int mask, float a, float b) {
  float r;
  asm("{\n\t.reg .pred p;\n\t.reg .b32 t;\n\tand.b32 t, %1, %2;\n\tsetp.ne.b32 p, t, 0;\n\tselp.f32 %0, %3, %4, p;\n\t}"
      : "=f"(r)
      : "r"(flags), "r"(mask), "f"(a), "f"(b));
  return r;
}

// Forward unit: acc = (first ? rhs_i : acc) - L_i,c0 x_c0 - ... (ascending c)
// kFrontier: every unit also stores acc over its row's right-hand side in the
// stage (tb + target offset: read only by this row's units, and only by the
// first), so after the chunk that block holds the rows' forward results.
// Sentinels store to offset 0 (unit 0's coefficients, no longer read).
template <bool kFrontier>
__device__ __forceinline__ void forward_unit(const UnitOps& r, unsigned char* xb, const unsigned char* tb, float& acc,
                                             float& prev) {
  const int fl = r.ctl.y;
  const float x3 = select_flag(fl, kUnitFwd, prev, r.x3);
  acc = select_flag(fl, kUnitFirst, r.t, acc);
  acc = acc - r.l.x * r.x0;
  acc = acc - r.l.y * r.x1;
  acc = acc - r.l.z * r.x2;
  acc = acc - r.l.w * x3;
  *reinterpret_cast<float*>(xb + r.ctl.w) = acc;
  if constexpr (kFrontier) *reinterpret_cast<float*>(const_cast<unsigned char*>(tb) + r.ctl.x) = acc;
  prev = acc;
}

// Backward unit: corr = (first ? 0 : corr) + L_r0,j x_r0 + ... (ascending r);
// x_j = x_j D^-1_j - corr
__device__ __forceinline__ void backward_unit(const UnitOps& r, unsigned char* xb, float& corr, float& prev) {
  const int fl = r.ctl.y;
  const float x0 = select_flag(fl, kUnitFwd, prev, r.x0);
  corr = select_flag(fl, kUnitFirst, 0.0f, corr);
  corr = corr + r.l.x * x0;
  corr = corr + r.l.y * r.x1;
  corr = corr + r.l.z * r.x2;
  corr = corr + r.l.w * r.x3;
  const float res = r.t * r.d - corr;
  *reinterpret_cast<float*>(xb + r.ctl.w) = res;
  prev = res;
}

// The plain form's sweep with 32-bit shared-window addresses (one integer add
// per operand address).  volatile with a memory clobber: the accesses keep
// their program order, which the unit pipeline relies on (a unit's operands
// are loaded after the stores of all but the previous unit).  Measured: plain
// form 89.2 -> 86.6 ms at 65,536 quadrotor instances; the frontier form is
// faster with the compiler's own scheduling of the generic accesses.
__device__ __forceinline__ int4 lds_s4(uint32_t a) {
  int4 v;
  asm volatile("ld.shared.v4.s32 {%0, %1, %2, %3}, [%4];" : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "r"(a)
               : "memory");
  return v;
}

__device__ __forceinline__ float4 lds_f4(uint32_t a) {
  float4 v;
  asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(a)
               : "memory");
  return v;
}

__device__ __forceinline__ float lds_f(uint32_t a) {
  float v;
  asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(a) : "memory");
  return v;
}

__device__ __forceinline__ void sts_f(uint32_t a, float v) {
  asm volatile("st.shared.f32 [%0], %1;" ::"r"(a), "f"(v) : "memory");
}

// A unit pass's bases: the meta list, this lane's 16 bytes of unit 0 of the
// stage, this lane's D^-1 column of the stage, this lane's column of the work
// vector (where the targets also point in the plain form).
struct UnitBase {
  uint32_t mu, lane_l, lane_d, xb;
};

__device__ __forceinline__ void load_meta_s(const UnitBase& b, int u, UnitOps& r) {
  r.src = lds_s4(b.mu + 32 * u);
  r.ctl = lds_s4(b.mu + 32 * u + 16);
}

template <bool kBackward>
__device__ __forceinline__ void load_data_s(const UnitBase& b, UnitOps& r) {
  r.l = lds_f4(b.lane_l + r.ctl.z);
  r.x0 = lds_f(b.xb + r.src.x);
  r.x1 = lds_f(b.xb + r.src.y);
  r.x2 = lds_f(b.xb + r.src.z);
  r.x3 = lds_f(b.xb + r.src.w);
  r.t = lds_f(b.xb + r.ctl.x);
  if (kBackward) r.d = lds_f(b.lane_d + (r.ctl.y >> kUnitDoffShift));
}

// forward_unit / backward_unit of the plain form on UnitBase addresses (the
// same operations)
__device__ __forceinline__ void forward_unit_s(const UnitOps& r, const UnitBase& b, float& acc, float& prev) {
  const int fl = r.ctl.y;
  const float x3 = select_flag(fl, kUnitFwd, prev, r.x3);
  acc = select_flag(fl, kUnitFirst, r.t, acc);
  acc = acc - r.l.x * r.x0;
  acc = acc - r.l.y * r.x1;
  acc = acc - r.l.z * r.x2;
  acc = acc - r.l.w * x3;
  sts_f(b.xb + r.ctl.w, acc);
  prev = acc;
}

__device__ __forceinline__ void backward_unit_s(const UnitOps& r, const UnitBase& b, float& corr, float& prev) {
  const int fl = r.ctl.y;
  const float x0 = select_flag(fl, kUnitFwd, prev, r.x0);
  corr = select_flag(fl, kUnitFirst, 0.0f, corr);
  corr = corr + r.l.x * x0;
  corr = corr + r.l.y * r.x1;
  corr = corr + r.l.z * r.x2;
  corr = corr + r.l.w * r.x3;
  const float res = r.t * r.d - corr;
  sts_f(b.xb + r.ctl.w, res);
  prev = res;
}

// Run a chunk's units as a software pipeline: while unit u is computed and
// stored, unit u+1's operands and unit u+2's meta are already loaded (three
// register sets in rotation, one exit test per three units).  The units past
// nu are sentinels: computed when nu is not a multiple of 3, harmlessly (they
// store to the trash row, and acc/prev are dead after the chunk).
template <bool kBackward, bool kFrontier = false>
__device__ __forceinline__ void run_units(const int4* __restrict__ mu, const unsigned char* lst, unsigned char* xb,
                                          const unsigned char* tb, int lane, int nu) {
  static_assert(kUnitGroup == 3 && kUnitSentinels >= 4, "loop shape and sentinel count disagree");
  if constexpr (!kFrontier) {
    // plain form (targets in the work vector: tb == xb)
    const UnitBase b{smem_u32(mu), smem_u32(lst) + lane * 16, smem_u32(lst) + lane * 4, smem_u32(xb)};
    UnitOps A, B, C;
    float acc = 0.0f, prev = 0.0f;
    load_meta_s(b, 0, A);
    load_data_s<kBackward>(b, A);
    load_meta_s(b, 1, B);
    for (int u = 0; u < nu; u += 3) {
      load_meta_s(b, u + 2, C);
      load_data_s<kBackward>(b, B);
      if (kBackward) backward_unit_s(A, b, acc, prev); else forward_unit_s(A, b, acc, prev);
      load_meta_s(b, u + 3, A);
      load_data_s<kBackward>(b, C);
      if (kBackward) backward_unit_s(B, b, acc, prev); else forward_unit_s(B, b, acc, prev);
      load_meta_s(b, u + 4, B);
      load_data_s<kBackward>(b, A);
      if (kBackward) backward_unit_s(C, b, acc, prev); else forward_unit_s(C, b, acc, prev);
    }
    return;
  }
  const unsigned char* lane_l = lst + lane * 16;
  UnitOps A, B, C;
  float acc = 0.0f, prev = 0.0f;
  load_meta(mu, 0, A);
  load_data<kBackward>(lane_l, lst, xb, tb, lane, A);
  load_meta(mu, 1, B);
  for (int u = 0; u < nu; u += 3) {
    load_meta(mu, u + 2, C);
    load_data<kBackward>(lane_l, lst, xb, tb, lane, B);
    if (kBackward) backward_unit(A, xb, acc, prev); else forward_unit<kFrontier>(A, xb, tb, acc, prev);
    load_meta(mu, u + 3, A);
    load_data<kBackward>(lane_l, lst, xb, tb, lane, C);
    if (kBackward) backward_unit(B, xb, acc, prev); else forward_unit<kFrontier>(B, xb, tb, acc, prev);
    load_meta(mu, u + 4, B);
    load_data<kBackward>(lane_l, lst, xb, tb, lane, A);
    if (kBackward) backward_unit(C, xb, acc, prev); else forward_unit<kFrontier>(C, xb, tb, acc, prev);
  }
}

// Releases of a backward chunk in groups of kRelGroup, the next group's operands
// loaded before the current group is computed and stored (every index is
// released once per pass, so groups never share a row).  A group slot past
// `end` repeats the group's first index: it loads the same operands, computes
// the same values and stores them to the same places again.
//   rel: per release (row byte offset, rho bits, rho^-1 bits, 0)
//   Recs: this lane's records of the chunk's releases in the stage (the
//         primal ones first, 4 bytes each, then the constraints', 8 bytes)
constexpr int kRelGroup = 2;  // releases per group (groups of 4 measured 3.5 % slower: register pressure)

struct RelGroup {
  int o[kRelGroup], kk[kRelGroup], ix[kRelGroup];
  float x[kRelGroup], rho[kRelGroup], rinv[kRelGroup], f[kRelGroup], e[kRelGroup];
  float4 st[kRelGroup];
};

// This lane's instance's rho by row class, when its rho adapted (on): the
// rule of the rho update (loose rows 1e-6, inequality rows rho_b, equality
// rows 1e3 rho_b; 1/rho one division each), else the records' (the plan's)
// rho vector.
struct RhoLane {
  bool on;
  float r_loose, r_ineq, r_eq, i_loose, i_ineq, i_eq;
};

__device__ __forceinline__ RhoLane rho_lane(const float* rho_b, const int* rho_count, int b) {
  RhoLane l;
  l.on = rho_count[b] > 0;
  const float est = rho_b[b];
  l.r_loose = 1e-6f;
  l.r_ineq = est;
  l.r_eq = 1e3f * est;
  l.i_loose = 1.0f / l.r_loose;
  l.i_ineq = 1.0f / l.r_ineq;
  l.i_eq = 1.0f / l.r_eq;
  return l;
}

// rho, 1/rho of a release of class cls (record values unless the lane's rho adapted)
__device__ __forceinline__ void rho_of(const RhoLane& l, int cls, int4 r, float& rho, float& rinv) {
  rho = __int_as_float(r.y);
  rinv = __int_as_float(r.z);
  if (l.on) {
    rho = cls < 0 ? l.r_loose : (cls > 0 ? l.r_eq : l.r_ineq);
    rinv = cls < 0 ? l.i_loose : (cls > 0 ? l.i_eq : l.i_ineq);
  }
}

// This lane's records of a backward chunk's releases in an S stage: release
// k < nprim (primal) at ip[32 k] (iterate x) and pp[32 k] (q), a constraint
// release k at ic[32 (k - nprim)] ((z, y)) and pc[...] ((l, u)).
struct StageRecs {
  const float* ip;
  const float* pp;
  const float2* ic;
  const float2* pc;
  int nprim;
};

// A record's last word: the released index's unscale factor (plain form) or
// the index itself (frontier form, whose unscale factors come from
// unscale_perm when termination is checked).  kRho: per-instance rho by the
// release's class (ucls: the classes of the chunk's releases).
template <bool kCons, bool kTrack, bool kFrontier, bool kRho>
__device__ __forceinline__ void load_rel_group(const int4* rel, int k, int end, const StageRecs& S, const float* SE,
                                               const unsigned char* xb, const float* unscale_perm, const int* ucls,
                                               const RhoLane& rl, RelGroup& g) {
#pragma unroll
  for (int j = 0; j < kRelGroup; ++j) {
    const int kk = (k + j < end) ? k + j : k;
    const int4 r = rel[kk];
    g.kk[j] = kk;
    g.o[j] = r.x;
    if constexpr (kRho) {
      rho_of(rl, __ldg(ucls + kk), r, g.rho[j], g.rinv[j]);
    } else {
      g.rho[j] = __int_as_float(r.y);
      g.rinv[j] = __int_as_float(r.z);
    }
    if constexpr (kFrontier) {
      g.ix[j] = r.w;
      g.f[j] = kTrack ? __ldg(unscale_perm + r.w) : 1.0f;
    } else {
      g.ix[j] = 0;
      g.f[j] = __int_as_float(r.w);
    }
    g.x[j] = *reinterpret_cast<const float*>(xb + r.x);
    if constexpr (kCons) {
      const float2 it = S.ic[(kk - S.nprim) * 32], pa = S.pc[(kk - S.nprim) * 32];
      g.st[j] = make_float4(it.x, it.y, pa.x, pa.y);
    } else {
      g.st[j] = make_float4(S.ip[kk * 32], 0.0f, S.pp[kk * 32], 0.0f);
    }
    if constexpr (kTrack) g.e[j] = SE[kk * 32];
  }
}

struct RelParams {
  float sigma, alpha, oma;
};

// primal index: x <- alpha x~ + (1 - alpha) x; next rhs sigma x - q
// constraint: z, y update and next rhs z - rho^-1 y (solver.py:806-820)
// frozen: this lane's instance has converged; its state and next right-hand
// side stay as they are (recomputed from the unchanged state).
// The scaled primal residual follows the iterates exactly (A x~ = z~ from the
// KKT solve): e_{k+1} = (z_relaxed - z_{k+1}) + (1 - alpha) e_k.  chg / pres:
// this lane's largest unscaled iterate change / primal residual so far
// (both are tracked, and lanes freeze, only when termination is checked:
// kTrack; without it the update is the plain ADMM step).
// kFrontier: the next right-hand side goes to rt (this lane's column of the
// right-hand-side vector) at the index the record carries in its last word,
// not back into the work vector.
// stu / stp: this lane's constraint / primal iterate records of the chunk's
// first release in HBM (release k at [32 k]).
template <bool kCons, bool kTrack, bool kFrontier>
__device__ __forceinline__ void update_rel_group(const RelGroup& g, const RelParams& rp, unsigned char* xb, float* rt,
                                                 float2* stu, float* stp, float* peu, float& chg, float& pres,
                                                 bool frozen_in) {
  const bool frozen = kTrack && frozen_in;
#pragma unroll
  for (int j = 0; j < kRelGroup; ++j) {
    float* xi = kFrontier ? rt + g.ix[j] * 32 : reinterpret_cast<float*>(xb + g.o[j]);
    float2* out = stu + g.kk[j] * 32;
    if (!kCons) {
      const float xa = rp.alpha * g.x[j] + rp.oma * g.st[j].x;
      const float xn = frozen ? g.st[j].x : xa;
      stp[g.kk[j] * 32] = xn;
      *xi = rp.sigma * xn - g.st[j].z;
      if constexpr (kTrack) chg = fmaxf(chg, fabsf(xn - g.st[j].x) * g.f[j]);
    } else {
      const float rinv = g.rinv[j];
      const float sv0 = g.st[j].x, yk = g.st[j].y;
      const float rz = sv0 - rinv * yk;
      const float zt = rz + rinv * g.x[j];
      const float zr = rp.alpha * zt + rp.oma * sv0;
      float za = zr + rinv * yk;
      za = (za < g.st[j].z) ? g.st[j].z : za;
      za = (za > g.st[j].w) ? g.st[j].w : za;
      const float ya = yk + g.rho[j] * (zr - za);
      const float zn = frozen ? sv0 : za, yn = frozen ? yk : ya;
      *out = make_float2(zn, yn);
      if constexpr (kTrack) {
        const float en = frozen ? g.e[j] : (zr - za) + rp.oma * g.e[j];
        peu[g.kk[j] * 32] = en;
        pres = fmaxf(pres, fabsf(en) * g.f[j]);
      }
      *xi = zn - rinv * yn;
      if constexpr (kTrack) chg = fmaxf(chg, fmaxf(fabsf(zn - sv0), fabsf(yn - yk)) * g.f[j]);
    }
  }
}

template <bool kCons, bool kTrack, bool kFrontier, bool kRho>
__device__ __forceinline__ void run_releases(const int4* rel, int begin, int end, const StageRecs& S,
                                             const float* SE, const RelParams& rp, unsigned char* xb, float* rt,
                                             float2* stu, float* stp,
                                             float* peu, float& chg, float& pres, bool frozen,
                                             const float* unscale_perm, const int* ucls, const RhoLane& rl) {
  if (begin >= end) return;
  RelGroup a, b;
  load_rel_group<kCons, kTrack, kFrontier, kRho>(rel, begin, end, S, SE, xb, unscale_perm, ucls, rl, a);
  for (int k = begin;; k += 2 * kRelGroup) {
    // a group starting at or past `end` clamps to end - 1 (loads only)
    const int kb = k + kRelGroup < end ? k + kRelGroup : end - 1;
    load_rel_group<kCons, kTrack, kFrontier, kRho>(rel, kb, end, S, SE, xb, unscale_perm, ucls, rl, b);
    update_rel_group<kCons, kTrack, kFrontier>(a, rp, xb, rt, stu, stp, peu, chg, pres, frozen);
    if (k + kRelGroup >= end) break;
    const int ka = k + 2 * kRelGroup < end ? k + 2 * kRelGroup : end - 1;
    load_rel_group<kCons, kTrack, kFrontier, kRho>(rel, ka, end, S, SE, xb, unscale_perm, ucls, rl, a);
    update_rel_group<kCons, kTrack, kFrontier>(b, rp, xb, rt, stu, stp, peu, chg, pres, frozen);
    if (k + 2 * kRelGroup >= end) break;
  }
}

// Shared-memory layout: X [n + 2][32] | L ring | S ring | barriers | flags.
// Warps: 0 sweeps (forward and backward units), 1 produces (bulk copies),
// 2 releases (first right-hand side, ADMM updates; with fixed iterations warp
// 3 releases half of each chunk's indices alongside).  Every warp walks the same
// item sequence; item t's L stage is freed by the warp that finishes with it
// last (plain form: forward sweeper, backward and first-rhs releaser; frontier
// form: forward the second releaser, backward the sweeper, first-rhs the
// releaser -- its release records travel in the S stage).  Two monotone
// counters order the consumers: sweep_done (items the sweeper finished: a
// backward item's releases need its columns solved) and rel_done (items the
// releaser finished: a forward sweep needs every right-hand side).
// kTrack: the primal residuals travel with the state (some class checks
// termination).  Without it (fixed iterations) a second releaser warp takes
// half of every chunk's releases (the releaser is on the critical path with
// the sweeper); the first releaser frees the stages and publishes rel_done
// once both halves are done.
// kFrontier: X holds slots, not rows (with termination checks too: the
// second releaser then only copies forward results and follows the first
// releaser's stop decisions, and the unscale factors come from unscale_perm,
// since the records carry indices).  The releasers
// write the right-hand sides to the per-tile vector rhs; the producer copies a
// forward chunk's rows of rhs, and a backward chunk's columns of fwd, into the
// stage behind its L data, where the units read their targets.  The sweeper
// leaves each row's forward result over its right-hand side in the stage, and
// the second releaser copies that block to fwd and frees the forward stage
// (y_done).  The copies into stages wait for the writes: a sweep's first
// forward chunk until every earlier item is released, its first backward
// chunk until every earlier forward block is in fwd.
// kRho: per-instance rho (adaptation, fixed iterations): a lane whose rho
// changed takes its constraints' rho and 1/rho from its instance's scalar
// rho by row class (RhoLane), in the first right-hand side and the updates.
template <bool kTrack, bool kFrontier, bool kRho = false>
__global__ void __launch_bounds__(128, 1) admm_stream_kernel(const __grid_constant__ StreamArgs a) {
  constexpr bool kSplit = !kTrack;  // the second releaser takes half of the releases (fixed iterations)
  extern __shared__ __align__(128) unsigned char smem[];
  const int lstage_bytes = a.meta_bytes + a.lbytes;
  const int total_tiles = a.tile_end[a.n_jobs - 1];
  float* X = reinterpret_cast<float*>(smem);
  unsigned char* lring = smem + (size_t)a.x_rows * 128;
  unsigned char* sring = lring + (size_t)a.lstages * lstage_bytes;
  uint64_t* lfull = reinterpret_cast<uint64_t*>(sring + (size_t)a.sstages * a.sbytes);
  uint64_t* lempty = lfull + a.lstages;
  uint64_t* sfull = lempty + a.lstages;
  uint64_t* sempty = sfull + a.sstages;
  volatile int* abort_flag = reinterpret_cast<volatile int*>(sempty + a.sstages);
  unsigned* sweep_done = reinterpret_cast<unsigned*>(sempty + a.sstages) + 1;
  unsigned* rel_done = sweep_done + 1;
  volatile unsigned* stop_at = rel_done + 1;  // item index where a converged tile's items end
  unsigned* rel_done1 = rel_done + 2;         // items the second releaser finished (kSplit)
  unsigned* y_done = rel_done + 3;            // frontier form: forward items whose results are in fwd
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < a.lstages; ++s) {
      mbar_init(lfull + s, 1);
      mbar_init(lempty + s, 1);
    }
    for (int s = 0; s < a.sstages; ++s) {
      mbar_init(sfull + s, 1);
      mbar_init(sempty + s, 1);
    }
    *abort_flag = 0;
    *sweep_done = 0;
    *rel_done = 0;
    *stop_at = 0xffffffffu;
    *rel_done1 = 0;
    *y_done = 0;
    fence_mbarrier_init();
  }
  __syncthreads();

  uint32_t issued_l = 0, issued_s = 0;  // producer: copies issued per ring

  if (warp == 1) {
    // ------------------------------ producer ------------------------------
    if (lane == 0) {
      Ring lr{0, 0}, sr{0, 0};
      for (int g = blockIdx.x; g < total_tiles && !*abort_flag; g += gridDim.x) {
        const int c = job_of(a, g);
        const StreamJob& J = a.job[c];
        const StreamPlan& sp = J.sp;
        const int n = sp.n;
        const int tile = g - (c ? a.tile_end[c - 1] : 0);
        const float* bt = J.bstream + (size_t)tile * sp.blen;
        const float* ft = J.fstream + (size_t)tile * sp.flen;
        const size_t soff = (size_t)tile * n * 32;
        // An item's copies: meta block, L data (first-right-hand-side pass: only
        // the releaser's forward units), frontier form: the rows' right-hand
        // sides (forward) or the columns' forward results (backward) behind
        // the L data; backward and first-rhs items also the state records.
        struct Copies {
          int moff, mwords, loff, nrel, u0, nprim;
          uint32_t lbytes, pre_at, xrow, xbytes;
        };
        auto describe = [&](int kind, int ch) {
          Copies d;
          const bool fwd = kind == kItemFwd;
          d.moff = __ldg((fwd ? sp.fmeta_off : sp.meta_off) + ch);
          d.mwords = __ldg((fwd ? sp.fmeta_words : sp.meta_words) + ch);
          d.loff = __ldg((fwd ? sp.fchunk_off : sp.chunk_off) + ch);
          d.nrel = 0;
          d.u0 = 0;
          d.nprim = 0;
          d.pre_at = 0;
          d.xrow = 0;
          d.xbytes = 0;
          if (fwd) {
            d.lbytes = (uint32_t)__ldg(sp.fchunk_units + ch) * 512u;
            if constexpr (kFrontier) {
              d.xrow = (uint32_t)__ldg(sp.frow0 + ch);
              d.xbytes = (uint32_t)__ldg(sp.frows + ch) * 128u;
            }
          } else {
            d.nrel = __ldg(sp.chunk_nrel + ch);
            d.u0 = __ldg(sp.chunk_u0 + ch);
            d.nprim = __ldg(sp.chunk_nprim + ch);
            if (kind == kItemBwd) {
              const uint32_t cols = (uint32_t)__ldg(sp.chunk_cols + ch);
              d.lbytes = (uint32_t)__ldg(sp.chunk_units + ch) * 512u + cols * 128u;
              if constexpr (kFrontier) {
                d.xrow = (uint32_t)__ldg(sp.chunk_c0 + ch);
                d.xbytes = cols * 128u;
              }
            } else {
              d.pre_at = (uint32_t)__ldg(sp.chunk_pre_u0 + ch);
              d.lbytes = (uint32_t)__ldg(sp.chunk_pre_units + ch) * 512u;
            }
          }
          return d;
        };
        // the next item's descriptors are loaded while this item waits and
        // issues (one table round trip per item would otherwise pace the ring)
        Copies ahead{};
        int ahead_kind = -1, ahead_ch = -1;
        auto produce = [&](int kind, int ch) -> bool {
          const bool fwd = kind == kItemFwd;
          const Copies d = (kind == ahead_kind && ch == ahead_ch) ? ahead : describe(kind, ch);
          if (fwd) {
            ahead_kind = ch + 1 < sp.n_fchunks ? kItemFwd : kItemBwd;
            ahead_ch = ch + 1 < sp.n_fchunks ? ch + 1 : sp.n_chunks - 1;
          } else {
            ahead_kind = ch > 0 ? kind : kItemFwd;
            ahead_ch = ch > 0 ? ch - 1 : 0;
          }
          ahead = describe(ahead_kind, ahead_ch);
          if (issued_l >= (uint32_t)a.lstages &&
              !mbar_wait_bounded(lempty + lr.stage, lr.phase ^ 1u, abort_flag, a.wait_limit_ns))
            return false;
          unsigned char* st = lring + (size_t)lr.stage * lstage_bytes;
          const float* xsrc = nullptr;
          if constexpr (kFrontier) {
            // those blocks are final once every earlier item is released
            // (forward) or swept (backward)
            if (fwd) {
              if (ch == 0 && !wait_counter_bounded(rel_done, issued_l, abort_flag, a.wait_limit_ns)) return false;
              xsrc = J.rhs + soff + (size_t)d.xrow * 32;
            } else if (kind == kItemBwd) {
              if (ch == sp.n_chunks - 1 && !wait_counter_bounded(y_done, issued_l, abort_flag, a.wait_limit_ns))
                return false;
              xsrc = J.fwd + soff + (size_t)d.xrow * 32;
            }
          }
          // (frontier form: a release item's records, the last 4 nrel words of
          // its meta block, go to its S stage)
          const uint32_t mwords_l = (uint32_t)d.mwords - (kFrontier ? 4u * (uint32_t)d.nrel : 0u);
          mbar_arrive_expect_tx(lfull + lr.stage, mwords_l * 4u + d.lbytes + d.xbytes);
          bulk_g2s(st, (fwd ? sp.fmeta : sp.meta) + d.moff, mwords_l * 4u, lfull + lr.stage);
          if (d.lbytes)
            bulk_g2s(st + a.meta_bytes + d.pre_at * 512u, (fwd ? ft : bt) + d.loff + d.pre_at * 128u, d.lbytes,
                     lfull + lr.stage);
          if (kFrontier && d.xbytes) bulk_g2s(st + a.meta_bytes + d.lbytes, xsrc, d.xbytes, lfull + lr.stage);
          lr.advance(a.lstages);
          ++issued_l;
          if (!fwd) {
            if (issued_s >= (uint32_t)a.sstages &&
                !mbar_wait_bounded(sempty + sr.stage, sr.phase ^ 1u, abort_flag, a.wait_limit_ns))
              return false;
            unsigned char* ss = sring + (size_t)sr.stage * a.sbytes;
            const uint32_t nrel = (uint32_t)d.nrel, np = (uint32_t)d.nprim, nc = nrel - np;
            // per region (iterates at 0, parameters at pres_off / 2): the primal
            // records (4 bytes), then the constraints' (8 bytes)
            if constexpr (kFrontier)  // the releases' header, then (bulk) their records
              *reinterpret_cast<int4*>(ss + a.rec_off) = make_int4(d.nrel, d.u0, d.nprim, 0);
            mbar_arrive_expect_tx(sfull + sr.stage, 2u * (np * 128u + nc * 256u) + (kTrack ? nrel * 128u : 0u) +
                                                        (kFrontier ? nrel * 16u : 0u));
            if (kFrontier && nrel)
              bulk_g2s(ss + a.rec_off + 16, sp.meta + d.moff + d.mwords - 4 * (int)nrel, nrel * 16u, sfull + sr.stage);
            const size_t u = soff + (size_t)d.u0 * 32;
            if (np) {
              bulk_g2s(ss, J.state_p + u, np * 128u, sfull + sr.stage);
              bulk_g2s(ss + a.pres_off / 2, J.param_p + u, np * 128u, sfull + sr.stage);
            }
            if (nc) {
              const size_t uc = u + (size_t)np * 32;
              bulk_g2s(ss + np * 128u, J.state + uc, nc * 256u, sfull + sr.stage);
              bulk_g2s(ss + a.pres_off / 2 + np * 128u, J.param + uc, nc * 256u, sfull + sr.stage);
            }
            if (kTrack && nrel) bulk_g2s(ss + a.pres_off, J.pres + u, nrel * 128u, sfull + sr.stage);
            sr.advance(a.sstages);
            ++issued_s;
          }
          return true;
        };
        // before a checked iteration: wait until the releaser has decided
        auto cont = [&](int it) -> int {
          if (!check_point(J.check_every, it)) return 1;
          if (!wait_counter_bounded(rel_done, issued_l, abort_flag, a.wait_limit_ns)) return -1;
          return *stop_at == issued_l ? 0 : 1;
        };
        if (!traverse(sp.n_chunks, sp.n_fchunks, J.max_iter, produce, cont)) {
          *abort_flag = 1;
          break;
        }
      }
    }
  } else if (warp == 0) {
    // ------------------------------ sweeper ------------------------------
    Ring lr{0, 0};
    unsigned t = 0;  // item index (all tiles)
    unsigned char* xb = smem + lane * 4;  // this lane's column of the work vector
    bool ok = true;
    for (int g = blockIdx.x; g < total_tiles && ok; g += gridDim.x) {
      const StreamJob& J = a.job[job_of(a, g)];
      const StreamPlan& sp = J.sp;
      auto sweep = [&](int kind, int ch) -> bool {
        if (kind != kItemRel) {
          // a forward sweep needs every right-hand side of the previous pass
          if (kind == kItemFwd && ch == 0 && !wait_counter_bounded(rel_done, t, abort_flag, a.wait_limit_ns))
            return false;
          // frontier form: the slots assume that a backward chunk's releases
          // are done before the sweep is frontier_lag chunks further (the
          // sweeper frees backward stages itself, so the ring does not pace it)
          if (kFrontier && kind == kItemBwd && t + 1 >= (unsigned)sp.frontier_lag &&
              !wait_counter_bounded(rel_done, t + 1 - (unsigned)sp.frontier_lag, abort_flag, a.wait_limit_ns))
            return false;
          if (!mbar_wait_bounded(lfull + lr.stage, lr.phase, abort_flag, a.wait_limit_ns)) return false;
          const unsigned char* stage = lring + (size_t)lr.stage * lstage_bytes;
          const int* meta = reinterpret_cast<const int*>(stage);
          const unsigned char* lst = stage + a.meta_bytes;
          const int4* mu = reinterpret_cast<const int4*>(meta + kChunkHeader);
          const int nu = meta[0];
          const unsigned char* tb = kFrontier ? lst + lane * 4 : xb;
          if (kFrontier && kind == kItemFwd) {
            // rows without entries: their right-hand side is their forward value
            const int ncopy = meta[3];
            const int2* cp = reinterpret_cast<const int2*>(meta + kChunkHeader + (nu + kUnitSentinels) * kUnitWords);
            for (int k = 0; k < ncopy; ++k) {
              const int2 e = cp[k];
              *reinterpret_cast<float*>(xb + e.y) = *reinterpret_cast<const float*>(tb + e.x);
            }
          }
          if (nu > 0) {
            if (kind == kItemFwd) {
              run_units<false, kFrontier>(mu, lst, xb, tb, lane, nu);  // forward substitution, row-gather form
            } else {
              run_units<true, kFrontier>(mu, lst, xb, tb, lane, nu);  // backward substitution, column form
            }
          }
          __syncwarp();
          if (lane == 0) {
            // (frontier form: the second releaser frees a forward stage once it
            // has copied the stage's forward results out)
            if (kFrontier ? kind == kItemBwd : kind == kItemFwd) mbar_arrive(lempty + lr.stage);
            st_release_cta(sweep_done, t + 1);
          }
          __syncwarp();
        }
        lr.advance(a.lstages);
        ++t;
        return true;
      };
      auto cont = [&](int it) -> int {
        if (!check_point(J.check_every, it)) return 1;
        if (!wait_counter_bounded(rel_done, t, abort_flag, a.wait_limit_ns)) return -1;
        return *stop_at == t ? 0 : 1;
      };
      if (!traverse(sp.n_chunks, sp.n_fchunks, J.max_iter, sweep, cont)) ok = false;
    }
    if (!ok && lane == 0) *abort_flag = 1;
  } else {
    // ------------------------------ releaser ------------------------------
    const int rw = warp - 2;  // releaser 0, or (kSplit) releaser 1
    Ring lr{0, 0}, sr{0, 0};
    unsigned t = 0;
    unsigned char* xb = smem + lane * 4;
    bool ok = true;
    for (int g = blockIdx.x; g < total_tiles && ok; g += gridDim.x) {
      const int c = job_of(a, g);
      const StreamJob& J = a.job[c];
      const StreamPlan& sp = J.sp;
      const int n = sp.n;
      const int tile = g - (c ? a.tile_end[c - 1] : 0);
      const float sigma = J.sigma, alpha = J.alpha, oma = J.one_minus_alpha;
      // this class's zero row (read by padding slots); every earlier tile is done with X
      if (rw == 0) X[(kFrontier ? sp.frontier_slots : n) * 32 + lane] = 0.0f;
      float* rt = nullptr;  // frontier form: this lane's column of the tile's right-hand sides
      float* yt = nullptr;  // and of its forward results
      if constexpr (kFrontier) {
        rt = J.rhs + (size_t)tile * n * 32 + lane;
        yt = J.fwd + (size_t)tile * n * 32 + lane;
      }
      float2* stt = J.state + (size_t)tile * n * 32 + lane;
      float* stpt = J.state_p + (size_t)tile * n * 32 + lane;
      float* pet = J.pres + (size_t)tile * n * 32 + lane;
      RhoLane rl{};
      if constexpr (kRho) {
        const int bl = tile * 32 + lane;
        rl = rho_lane(J.rho_b, J.rho_count, bl < J.batch ? bl : J.batch - 1);
      }
      float pres = 0.0f;  // this lane's largest unscaled primal residual in the current iteration
      float chg = 0.0f;  // this lane's largest unscaled iterate change in the current iteration
      int iters_run = 0, frozen_at = 0;
      bool stop = false, frozen = false;
      auto release = [&](int kind, int ch) -> bool {
        if (kFrontier && kind == kItemFwd && rw == 1) {
          // frontier form: copy the forward results the sweeper left in the
          // chunk's stage (rows [r0, r1) of its header) to fwd, then free it
          if (!wait_counter_bounded(sweep_done, t + 1, abort_flag, a.wait_limit_ns)) return false;
          const unsigned char* stage = lring + (size_t)lr.stage * lstage_bytes;
          const int* meta = reinterpret_cast<const int*>(stage);
          const int nu = meta[0], r0 = meta[1], rows = meta[2] - meta[1];
          const float* yb = reinterpret_cast<const float*>(stage + a.meta_bytes + nu * 512) + lane;
          float* yg = yt + (size_t)r0 * 32;
          for (int r = 0; r < rows; ++r) yg[r * 32] = yb[r * 32];
          // read back by the backward sweep's bulk copies once y_done covers the last chunk
          if (ch == sp.n_fchunks - 1) fence_proxy_async_global();
          __syncwarp();
          if (lane == 0) {
            mbar_arrive(lempty + lr.stage);
            st_release_cta(y_done, t + 1);
          }
          __syncwarp();
        }
        if (kind != kItemFwd) {
          if (kind == kItemBwd) {
            // the chunk's columns are solved (and its stage is full)
            if (!wait_counter_bounded(sweep_done, t + 1, abort_flag, a.wait_limit_ns)) return false;
          } else if (!mbar_wait_bounded(lfull + lr.stage, lr.phase, abort_flag, a.wait_limit_ns)) {
            return false;
          }
          // plain form: the releases' header and records are in the item's L
          // stage (with the releaser's units); frontier form: in its S stage
          // (the sweeper frees a backward L stage as soon as it is swept)
          int nrel = 0, u0 = 0, nprim = 0, nl = 0, np = 0;
          const int4* mu_pre = nullptr;
          const int4* rel = nullptr;
          const unsigned char* lst = nullptr;
          if constexpr (!kFrontier) {
            const unsigned char* stage = lring + (size_t)lr.stage * lstage_bytes;
            const int* meta = reinterpret_cast<const int*>(stage);
            lst = stage + a.meta_bytes;
            const int ns = meta[0];
            nrel = meta[2];
            u0 = meta[4];
            nprim = meta[5];
            nl = meta[6];
            np = meta[7];
            const int4* mu_leaf = reinterpret_cast<const int4*>(meta + kChunkHeader + (ns + kUnitSentinels) * kUnitWords);
            mu_pre = mu_leaf + (nl + kUnitSentinels) * (kUnitWords / 4);
            rel = reinterpret_cast<const int4*>(meta + kChunkHeader + (ns + nl + np + 3 * kUnitSentinels) * kUnitWords);
            // leaf columns (read by no other column): solved here, just before their release
            if (rw == 0 && kind == kItemBwd && nl > 0) run_units<true>(mu_leaf, lst, xb, xb, lane, nl);
          }
          if (!mbar_wait_bounded(sfull + sr.stage, sr.phase, abort_flag, a.wait_limit_ns)) return false;
          const unsigned char* sst = sring + (size_t)sr.stage * a.sbytes;
          if constexpr (kFrontier) {
            const int4 h = *reinterpret_cast<const int4*>(sst + a.rec_off);
            nrel = h.x;
            u0 = h.y;
            nprim = h.z;
            rel = reinterpret_cast<const int4*>(sst + a.rec_off + 16);
          }
          // this warp's share of the releases: halves of the primal and of the
          // constraint range (all of them, on releaser 0, when the chunk has
          // releaser units, which need every release of the chunk done first)
          const bool split = kSplit && nl == 0 && np == 0;
          auto share = [&](int b0, int e0, int& b1, int& e1) {
            const int h = split ? b0 + (e0 - b0 + 1) / 2 : e0;
            b1 = rw == 0 ? b0 : h;
            e1 = rw == 0 ? h : e0;
          };
          int pb, pe, cb, ce;
          share(0, nprim, pb, pe);
          share(nprim, nrel, cb, ce);
          const StageRecs S{reinterpret_cast<const float*>(sst) + lane,
                            reinterpret_cast<const float*>(sst + a.pres_off / 2) + lane,
                            reinterpret_cast<const float2*>(sst + nprim * 128) + lane,
                            reinterpret_cast<const float2*>(sst + a.pres_off / 2 + nprim * 128) + lane, nprim};
          const float* SE = reinterpret_cast<const float*>(sring + (size_t)sr.stage * a.sbytes + a.pres_off) + lane;
          if (kind == kItemRel) {
            // first right-hand side: sigma x - q (primal), z - rho^-1 y (constraint)
            // (frontier form: into rhs at the record's index)
            for (int k = pb; k < pe; ++k) {
              const int4 r = rel[k];
              *(kFrontier ? rt + r.w * 32 : reinterpret_cast<float*>(xb + r.x)) = sigma * S.ip[k * 32] - S.pp[k * 32];
            }
            for (int k = cb; k < ce; ++k) {
              const int4 r = rel[k];
              const float2 st = S.ic[(k - nprim) * 32];
              float rinv = __int_as_float(r.z);
              if constexpr (kRho) {
                float rho;
                rho_of(rl, __ldg(sp.u_cls + u0 + k), r, rho, rinv);
              }
              *(kFrontier ? rt + r.w * 32 : reinterpret_cast<float*>(xb + r.x)) = st.x - rinv * st.y;
            }
            // read back by bulk copies once rel_done covers the pass's last chunk
            if (kFrontier && ch == 0) fence_proxy_async_global();
          } else {
            float2* stu = stt + (size_t)u0 * 32;
            float* stp = stpt + (size_t)u0 * 32;
            float* peu = pet + (size_t)u0 * 32;
            const RelParams rp{sigma, alpha, oma};
            const int* ucls = kRho ? sp.u_cls + u0 : nullptr;
            run_releases<false, kTrack, kFrontier, false>(rel, pb, pe, S, SE, rp, xb, rt, stu, stp, peu, chg, pres, frozen,
                                                          sp.unscale_perm, ucls, rl);
            run_releases<true, kTrack, kFrontier, kRho>(rel, cb, ce, S, SE, rp, xb, rt, stu, stp, peu, chg, pres, frozen,
                                                        sp.unscale_perm, ucls, rl);
            // order these generic-proxy state writes before the bulk copies
            // that read them back in the next pass
            fence_proxy_async_global();
          }
          // forward rows whose entries all read leaf rows: their right-hand sides are now final
          if (!kFrontier && rw == 0 && np > 0) {
            __syncwarp();
            run_units<false>(mu_pre, lst, xb, xb, lane, np);
          }
          __syncwarp();
          if (rw == 1) {
            if (lane == 0) st_release_cta(rel_done1, t + 1);
          } else {
            // both halves done before the stages are freed
            if (kSplit && !wait_counter_bounded(rel_done1, t + 1, abort_flag, a.wait_limit_ns)) return false;
            if (lane == 0) {
              mbar_arrive(sempty + sr.stage);
              if (!kFrontier || kind != kItemBwd) mbar_arrive(lempty + lr.stage);
            }
          }
          sr.advance(a.sstages);
        }
        if (rw == 1) {  // the second releaser publishes nothing else and makes no decisions
          lr.advance(a.lstages);
          ++t;
          return true;
        }
        if (kind == kItemBwd && ch == 0) {
          // an iteration is complete: decide (before publishing it) whether the tile stops here
          ++iters_run;
          if (check_point(J.check_every, iters_run) && iters_run < J.max_iter) {
            if (!frozen && chg <= J.chg_eps && (!kTrack || pres <= J.chg_eps)) {
              frozen = true;
              frozen_at = iters_run;
            }
            stop = __all_sync(0xffffffffu, frozen);
            if (stop && lane == 0) *stop_at = t + 1;
          }
          chg = 0.0f;
          pres = 0.0f;
        }
        __syncwarp();
        if (lane == 0) st_release_cta(rel_done, t + 1);
        __syncwarp();
        lr.advance(a.lstages);
        ++t;
        return true;
      };
      auto cont = [&](int it) -> int {
        if (rw == 0) return stop ? 0 : 1;
        // the second releaser (frontier form) follows the first one's decision
        if (!check_point(J.check_every, it)) return 1;
        if (!wait_counter_bounded(rel_done, t, abort_flag, a.wait_limit_ns)) return -1;
        return *stop_at == t ? 0 : 1;
      };
      if (!traverse(sp.n_chunks, sp.n_fchunks, J.max_iter, release, cont)) ok = false;
      if (ok && rw == 0 && J.iters && tile * 32 + lane < J.batch)
        J.iters[tile * 32 + lane] = frozen ? frozen_at : iters_run;
    }
    if (!ok && lane == 0) *abort_flag = 1;
  }
  __syncthreads();
  if (*abort_flag) {
    if (threadIdx.x == 32) {
      // drain: wait (bounded) for the last bulk copy issued into every stage
      // (earlier ones completed before their stage was reused)
      for (uint32_t s = 0; s < (uint32_t)a.lstages && s < issued_l; ++s) {
        const uint32_t last = s + (uint32_t)a.lstages * ((issued_l - 1 - s) / (uint32_t)a.lstages);
        mbar_wait_bounded(lfull + s, (last / (uint32_t)a.lstages) & 1u, nullptr, kWaitLimitNs);
      }
      for (uint32_t s = 0; s < (uint32_t)a.sstages && s < issued_s; ++s) {
        const uint32_t last = s + (uint32_t)a.sstages * ((issued_s - 1 - s) / (uint32_t)a.sstages);
        mbar_wait_bounded(sfull + s, (last / (uint32_t)a.sstages) & 1u, nullptr, kWaitLimitNs);
      }
    }
    if (threadIdx.x == 0) atomicExch(a.error, 1);
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

namespace {

struct RingSizes {
  int meta_bytes, lbytes, sbytes, pres_off, x_rows, lmax, smax;
};

// track: the S stages also carry the primal residuals (termination checked)
RingSizes ring_sizes(const StreamPlan& sp, bool track) {
  RingSizes r;
  const bool fr = sp.frontier_slots > 0;
  // (frontier form: without a backward chunk's release records, which go to the S stage)
  const int mwb = fr ? sp.max_meta_lead : sp.max_meta_words;
  const int mw = mwb > sp.max_fmeta_words ? mwb : sp.max_fmeta_words;
  r.meta_bytes = ((mw * 4 + 127) / 128) * 128;
  // (frontier form: a backward stage also holds its columns' forward results,
  // a forward stage its rows' right-hand sides)
  const bool frontier = sp.frontier_slots > 0;
  const int bl = sp.max_units * 512 + sp.max_cols * (frontier ? 256 : 128);
  const int fl = sp.max_funits * 512 + (frontier ? sp.max_frows * 128 : 0);
  r.lbytes = ((bl > fl ? bl : fl) + 127) / 128 * 128;
  r.pres_off = (sp.max_rel > 0 ? sp.max_rel : 1) * 512;
  r.sbytes = r.pres_off + (track ? r.pres_off / 4 : 0);
  if (fr) r.sbytes += 16 + 16 * (sp.max_rel > 0 ? sp.max_rel : 1);  // releases' header and records
  r.x_rows = (frontier ? sp.frontier_slots : sp.n) + 2;
  r.lmax = sp.max_lstages >= 2 ? sp.max_lstages : 12;
  r.smax = sp.max_sstages >= 2 ? sp.max_sstages : 6;
  // the slots assume releases trail the sweep by at most frontier_lag chunks
  if (frontier) r.lmax = std::min(r.lmax, sp.frontier_lag);
  return r;
}

bool ring_config(const RingSizes& r, StreamLaunch* cfg, size_t limit = (size_t)kMaxSmemBytes) {
  // prefer deep rings: as many L stages as fit with at least 3 S stages
  for (int ls = r.lmax; ls >= 2; --ls)
    for (int ss = r.smax; ss >= 2; --ss) {
      const size_t bytes = stream_smem_bytes(r.x_rows - 2, ls, ss, r.meta_bytes + r.lbytes, r.sbytes);
      if (bytes <= limit && (ss >= 3 || ls <= 3)) {
        cfg->stages = ls;
        cfg->sstages = ss;
        cfg->meta_bytes = r.meta_bytes;
        cfg->lbytes = r.lbytes;
        cfg->sbytes = r.sbytes;
        cfg->pres_off = r.pres_off;
        cfg->smem = bytes;
        return true;
      }
    }
  return false;
}

}  // namespace

// (sized with the residuals: a pattern that fits this fits every launch)
bool stream_launch_config(const StreamPlan& sp, StreamLaunch* cfg) { return ring_config(ring_sizes(sp, true), cfg); }

namespace {

// The ring of a launch with k CTAs per SM on device `dev` (-1: the current
// device): 4-stage L and 3-stage S rings at most, 1/k of the SM's shared
// memory each (false when the device cannot be queried).
bool multi_cta_config(const RingSizes& r, int k, StreamLaunch* cfg, int dev = -1) {
  int sm_bytes = 0, reserved = 0;
  if ((dev < 0 && cudaGetDevice(&dev) != cudaSuccess) ||
      cudaDeviceGetAttribute(&sm_bytes, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  RingSizes r2 = r;
  r2.lmax = std::min(r2.lmax, 4);
  r2.smax = std::min(r2.smax, 3);
  return ring_config(r2, cfg, (size_t)(sm_bytes / k - reserved));
}

}  // namespace

// Most CTAs per SM a launch may use: 1 when WMPC_STREAM_CTAS=1, else
// WMPC_STREAM_MAX_CTAS (2 to 4; default 2).  Read when a problem is created.
int stream_ctas_limit_setting() {
  const char* one = getenv("WMPC_STREAM_CTAS");
  if (one && atoi(one) == 1) return 1;
  const char* v = getenv("WMPC_STREAM_MAX_CTAS");
  const int k = v ? atoi(v) : 2;
  return k < 1 ? 1 : (k > 4 ? 4 : k);
}

namespace {

// Whether k CTAs of `kernel` (threads each, smem bytes of dynamic shared
// memory, the SM's unified memory carved out as shared memory) are resident
// on one SM at once: shared memory alone does not decide it, registers count too.
bool ctas_resident(const void* kernel, int threads, size_t smem, int k) {
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
      cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                           (int)cudaSharedmemCarveoutMaxShared) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  int blocks = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kernel, threads, smem) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  return blocks >= k;
}

// The kernel instance of a schedule form, with or without termination checks,
// and its threads (four warps; three for the plain form's checked instance,
// which has no second releaser).
const void* stream_kernel_of(bool frontier, bool track) {
  if (track)
    return frontier ? reinterpret_cast<const void*>(admm_stream_kernel<true, true>)
                    : reinterpret_cast<const void*>(admm_stream_kernel<true, false>);
  return frontier ? reinterpret_cast<const void*>(admm_stream_kernel<false, true>)
                  : reinterpret_cast<const void*>(admm_stream_kernel<false, false>);
}
int stream_threads_of(bool frontier, bool track) { return track && !frontier ? 96 : 128; }

}  // namespace

int stream_max_ctas(const StreamPlan& sp, int device, int limit, bool track) {
  const RingSizes r = ring_sizes(sp, track);
  const bool frontier = sp.frontier_slots > 0;
  for (int k = limit; k >= 2; --k) {
    StreamLaunch cfg;
    if (multi_cta_config(r, k, &cfg, device) &&
        ctas_resident(stream_kernel_of(frontier, track), stream_threads_of(frontier, track), cfg.smem, k))
      return k;
  }
  return 1;
}

int stream_ctas_for(const StreamPlan& sp, int device, int tiles, int num_sms, int limit, bool track) {
  for (int k = stream_max_ctas(sp, device, limit, track); k >= 2; --k)
    if (tiles > (k - 1) * num_sms) return k;
  return 1;
}


// streams, state records, residuals (+ frontier form: right-hand sides and forward results)
size_t stream_workspace_floats(const StreamPlan& sp, int batch) {
  const size_t tiles = (size_t)(batch + 31) / 32;
  const size_t vectors = sp.frontier_slots > 0 ? 9 : 7;  // state 2 + 2 (+ 1 + 1 primal), pres (+ rhs, fwd)
  return tiles * ((size_t)sp.blen + (size_t)sp.flen + vectors * 32 * (size_t)sp.n) + 64;
}

// Factorization into the streams and the state into its records (one class).
int stream_begin(const Pattern& pat, const StreamPlan& sp, const Osqp& o, const float* pT, long long ldp, int sbp,
                 const float* aT, long long lda, int sba, const float* x, const float* z, const float* y,
                 const float* qs, const float* ls, const float* us, bool warm, bool track, float* work,
                 int* status, int batch, int num_sms, bool reuse_factor, StreamJobDesc* job, cudaStream_t s,
                 const float* rinv_rows, const int* only) {
  StreamLaunch cfg;
  if (!stream_launch_config(sp, &cfg)) return fail(WMPC_ERR_UNSUPPORTED, "pattern too large for the streaming kernel");
  const int n_tiles = (batch + 31) / 32;
  const size_t tl = (size_t)n_tiles * 32;
  float* bstream = work;
  float* fstream = bstream + (size_t)n_tiles * sp.blen;
  float2* state = reinterpret_cast<float2*>(fstream + (size_t)n_tiles * sp.flen);
  float2* param = state + tl * sp.n;
  float* state_p = reinterpret_cast<float*>(param + tl * sp.n);
  float* param_p = state_p + tl * sp.n;
  float* pres = param_p + tl * sp.n;
  float* rhs = sp.frontier_slots > 0 ? pres + tl * sp.n : nullptr;
  float* fwd = sp.frontier_slots > 0 ? rhs + tl * sp.n : nullptr;
  OsqpInputs in{pT, ldp, sbp, aT, lda, sba, rinv_rows, rinv_rows ? (long long)batch : 0};
  if (rinv_rows && !o.kin_desc_rho) return fail(WMPC_ERR_UNSUPPORTED, "the problem has no per-instance rho inputs");
  if (!reuse_factor) {
    // L-batch sized so that every tile's warp is resident at once (all of a
    // launch's rows then wait out their round trips together)
    const int warps = 2;
    const int per_sm = ceil_div(n_tiles, num_sms > 0 ? num_sms : 1);
    const int budget_floats = (200 * 1024 / 4) / (per_sm > 0 ? per_sm : 1);
    int lbatch = (budget_floats - factor_warp_words(sp, 0)) / 33;
    // WMPC_FACTOR_LBATCH fixes the batch instead (tuning: fewer resident
    // warps, fewer round trips per row)
    // with many tiles per SM a short batch measured faster (16: 8.98 ms against 9.23 for the budget's
    // 24 on 65,536 quadrotor instances; 32 to 128: 11.9 to 16.5 ms): the smaller shared-memory
    // request leaves more of the SM's unified memory to L1, which serves the index tables
    if (per_sm >= 8 && lbatch > 16) lbatch = 16;
    if (const char* v = getenv("WMPC_FACTOR_LBATCH")) lbatch = atoi(v);
    lbatch = lbatch < 8 ? 8 : (lbatch > 128 ? 128 : lbatch);
    const size_t smem = (size_t)warps * factor_warp_words(sp, lbatch) * sizeof(float);
    if (smem > (size_t)kMaxSmemBytes) return fail(WMPC_ERR_UNSUPPORTED, "factor rows too long for shared memory");
    WMPC_CUDA_TRY(cudaFuncSetAttribute(factor_stream_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    profile_mark_begin(s, kProfileFactor);
    factor_stream_kernel<<<ceil_div(n_tiles, warps), warps * 32, smem, s>>>(pat, sp, o, in, bstream, fstream, status,
                                                                            n_tiles, batch, lbatch, only);
    profile_mark_end(s, kProfileFactor);
    WMPC_LAUNCH_CHECK();
  }
  {
    dim3 grid(ceil_div(tl, 128), sp.n < 1024 ? sp.n : 1024);
    state_to_stream_kernel<<<grid, 128, 0, s>>>(sp, o, in, warm && track, x, z, y, qs, ls, us, state, param, state_p,
                                                 param_p, pres, batch, n_tiles);
    WMPC_LAUNCH_CHECK();
  }
  job->sp = sp;
  job->bstream = bstream;
  job->fstream = fstream;
  job->state = state;
  job->param = param;
  job->state_p = state_p;
  job->param_p = param_p;
  job->pres = pres;
  job->rhs = rhs;
  job->fwd = fwd;
  job->n_tiles = n_tiles;
  job->batch = batch;
  job->sigma = o.sigma;
  job->alpha = o.alpha;
  job->one_minus_alpha = o.one_minus_alpha;
  return WMPC_OK;
}

static int total_tiles_of(const StreamJobDesc* jobs, int n_jobs) {
  int t = 0;
  for (int i = 0; i < n_jobs; ++i) t += jobs[i].n_tiles;
  return t;
}

// One launch over every class's tiles, the costliest class first.
int stream_run(const StreamJobDesc* jobs, int n_jobs, int* error, int num_sms, cudaStream_t s) {
  if (n_jobs < 1 || n_jobs > kMaxStreamJobs) return fail(WMPC_ERR_INVALID_ARGUMENT, "1 to %d classes per launch", kMaxStreamJobs);
  RingSizes r{0, 0, 0, 0, 0, 12, 6};
  int order[kMaxStreamJobs];
  double cost[kMaxStreamJobs];
  bool track = false, rho = false;
  for (int i = 0; i < n_jobs; ++i) track = track || jobs[i].check_every > 0;
  for (int i = 0; i < n_jobs; ++i) rho = rho || jobs[i].rho_b != nullptr;
  if (rho && (track || n_jobs > 1))
    return fail(WMPC_ERR_UNSUPPORTED, "per-instance rho runs one class with fixed iterations");
  if (rho && (!jobs[0].rho_count || !jobs[0].sp.u_cls))
    return fail(WMPC_ERR_UNSUPPORTED, "per-instance rho needs the rho counts and the schedule's row classes");
  const bool frontier = jobs[0].sp.frontier_slots > 0;
  for (int i = 0; i < n_jobs; ++i)
    if ((jobs[i].sp.frontier_slots > 0) != frontier)
      return fail(WMPC_ERR_UNSUPPORTED, "frontier-form and plain classes cannot share a launch");
  for (int i = 0; i < n_jobs; ++i) {
    const RingSizes ri = ring_sizes(jobs[i].sp, track);
    r.meta_bytes = std::max(r.meta_bytes, ri.meta_bytes);
    r.lbytes = std::max(r.lbytes, ri.lbytes);
    r.sbytes = std::max(r.sbytes, ri.sbytes);
    r.pres_off = std::max(r.pres_off, ri.pres_off);
    r.x_rows = std::max(r.x_rows, ri.x_rows);
    r.lmax = std::min(r.lmax, ri.lmax);
    r.smax = std::min(r.smax, ri.smax);
    order[i] = i;
    cost[i] = (double)(jobs[i].max_iter + 1) * ((double)jobs[i].sp.blen + jobs[i].sp.flen);
  }
  std::sort(order, order + n_jobs, [&](int x, int y) { return cost[x] > cost[y]; });
  StreamLaunch cfg;
  if (!ring_config(r, &cfg)) return fail(WMPC_ERR_UNSUPPORTED, "these classes do not fit one launch's shared memory");
  // k CTAs (k sweepers) per SM when k fit with rings of at most 4 L and 3 S
  // stages (a sweeper per SM is worth more than ring depth beyond 2 stages)
  // and there are more tiles than k - 1 per SM.
  int ctas_per_sm = 1;
  {
    const int tiles = total_tiles_of(jobs, n_jobs);
    const void* kfn = stream_kernel_of(frontier, track);
    int limit = jobs[0].ctas_limit;
    for (int i = 1; i < n_jobs; ++i) limit = std::min(limit, jobs[i].ctas_limit);
    for (int k = limit; k >= 2; --k) {
      StreamLaunch cfgk;
      if (tiles > (k - 1) * num_sms && multi_cta_config(r, k, &cfgk) &&
          ctas_resident(kfn, stream_threads_of(frontier, track), cfgk.smem, k)) {
        cfg = cfgk;
        ctas_per_sm = k;
        break;
      }
    }
  }
  StreamArgs a{};
  int total = 0;
  for (int k = 0; k < n_jobs; ++k) {
    const StreamJobDesc& d = jobs[order[k]];
    StreamJob& J = a.job[k];
    J.sp = d.sp;
    J.bstream = d.bstream;
    J.fstream = d.fstream;
    J.state = d.state;
    J.param = d.param;
    J.state_p = d.state_p;
    J.param_p = d.param_p;
    J.pres = d.pres;
    J.rhs = d.rhs;
    J.fwd = d.fwd;
    J.iters = d.iters;
    J.rho_b = d.rho_b;
    J.rho_count = d.rho_count;
    J.n_tiles = d.n_tiles;
    J.max_iter = d.max_iter;
    J.batch = d.batch;
    J.check_every = d.check_every;
    J.chg_eps = d.chg_eps;
    J.sigma = d.sigma;
    J.alpha = d.alpha;
    J.one_minus_alpha = d.one_minus_alpha;
    total += d.n_tiles;
    a.tile_end[k] = total;
  }
  if (total == 0) return WMPC_OK;
  a.n_jobs = n_jobs;
  a.x_rows = r.x_rows;
  a.error = error;
  a.lstages = cfg.stages;
  a.sstages = cfg.sstages;
  a.meta_bytes = cfg.meta_bytes;
  a.lbytes = cfg.lbytes;
  a.sbytes = cfg.sbytes;
  a.pres_off = cfg.pres_off;
  a.rec_off = cfg.pres_off + (track ? cfg.pres_off / 4 : 0);
  a.wait_limit_ns = kWaitLimitNs;
  if (const char* v = getenv("WMPC_STREAM_WAIT_LIMIT_NS")) {
    const long long ns = atoll(v);
    if (ns > 0) a.wait_limit_ns = (unsigned long long)ns;
  }
  const int grid = total < ctas_per_sm * num_sms ? total : ctas_per_sm * num_sms;
  auto kernel = track ? (frontier ? admm_stream_kernel<true, true> : admm_stream_kernel<true, false>)
                : rho ? (frontier ? admm_stream_kernel<false, true, true> : admm_stream_kernel<false, false, true>)
                      : (frontier ? admm_stream_kernel<false, true> : admm_stream_kernel<false, false>);
  WMPC_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cfg.smem));
  // all of the SM's unified memory as shared memory, so that two CTAs fit
  WMPC_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     (int)cudaSharedmemCarveoutMaxShared));
  profile_mark_begin(s);
  kernel<<<grid, stream_threads_of(frontier, track), cfg.smem, s>>>(a);
  profile_mark_end(s);
  record_stream_launch(frontier ? 2 : 1, ctas_per_sm, grid, (int)cfg.smem);
  WMPC_LAUNCH_CHECK();
  return WMPC_OK;
}

// The state records back to x, z, y (one class).
int stream_end(const StreamPlan& sp, const Osqp& o, const StreamJobDesc& job, float* x, float* z, float* y,
               cudaStream_t s) {
  dim3 grid2(ceil_div(job.batch, 128), sp.n < 1024 ? sp.n : 1024);
  stream_to_state_kernel<<<grid2, 128, 0, s>>>(sp, o.n, job.state, job.state_p, x, z, y, job.batch);
  WMPC_LAUNCH_CHECK();
  return WMPC_OK;
}

}  // namespace wmpc

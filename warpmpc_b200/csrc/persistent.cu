// Streaming persistent OSQP-ADMM kernels (sm_100a).
//
// factor_stream_kernel: KKT assembly + LDL^T factorization, one lane per
//   instance, compact accumulator (one shared-memory slot per etree-reach
//   position instead of a dense work vector), L and D^-1 written in the
//   stream-major tile layout (see stream.cuh).
// admm_stream_kernel: one CTA per SM walks instance tiles; a producer warp
//   streams every chunk of the factor into a shared-memory ring with
//   cp.async.bulk (mbarrier completion), a consumer warp runs, per ADMM
//   iteration, the forward sweep (L, column order), the backward sweep
//   (D^-1 and L^T, reverse column order) and, as soon as the backward sweep
//   is done with a KKT index, its ADMM update, writing the next iteration's
//   right-hand side in place.  The work vector (KKT dimension x 32 lanes)
//   stays in shared memory for all iterations of a tile.
//
// Arithmetic is the reference's operation order (warp_backend.py:41-101,
// 176-218; solver.py:806-820) with separately rounded products and sums.
#include "osqp.cuh"
#include "stream.cuh"

namespace wmpc {

struct OsqpInputs {
  const float* pT; long long ldp; int sbp;
  const float* aT; long long lda; int sba;
  __device__ __forceinline__ float p(int j, int b) const { return pT[(long long)j * ldp + (long long)b * sbp]; }
  __device__ __forceinline__ float a(int j, int b) const { return aT[(long long)j * lda + (long long)b * sba]; }
};

__device__ __forceinline__ float kkt_value_at(const Osqp& o, const OsqpInputs& in, int s, int b) {
  const int src = __ldg(o.kkt_src + s);
  if (src < 0) return __ldg(o.kkt_base + s);
  if (src < o.nnz_p) return in.p(src, b) * __ldg(o.p_scale + src) + __ldg(o.p_diag_sigma + src);
  const int j = src - o.nnz_p;
  return in.a(j, b) * __ldg(o.a_scale + j);
}

// ---------------------------------------------------------------------------
// factorization into the stream layout
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(128) factor_stream_kernel(Pattern pat, StreamPlan sp, Osqp o, OsqpInputs in,
                                                            float* __restrict__ lstream, float* __restrict__ fstream,
                                                            int n_tiles, int batch) {
  extern __shared__ float ys_all[];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int tile = blockIdx.x * (blockDim.x >> 5) + warp;
  if (tile >= n_tiles) return;
  const int b = tile * 32 + lane;
  const int bb = b < batch ? b : batch - 1;  // padding lanes factor a copy of the last instance
  float* ys = ys_all + (size_t)warp * sp.max_row_nnz * 32 + lane;
  float* L = lstream + (size_t)tile * sp.stream_len * 32 + lane;
  float* F = fstream + (size_t)tile * sp.nnz_l * 32 + lane;
  const int n = pat.n;
  for (int k = 0; k < n; ++k) {
    const int p0 = __ldg(pat.proc_ptr + k), p1 = __ldg(pat.proc_ptr + k + 1);
    for (int s = 0; s < p1 - p0; ++s) ys[s * 32] = 0.0f;
    float dk = kkt_value_at(o, in, __ldg(pat.perm_to_orig + __ldg(pat.diag_pos + k)), bb);
    const int i0 = __ldg(pat.init_ptr + k), i1 = __ldg(pat.init_ptr + k + 1);
    for (int e = i0; e < i1; ++e) {
      const int s = __ldg(sp.init_slot + e);
      ys[s * 32] = ys[s * 32] + kkt_value_at(o, in, __ldg(pat.perm_to_orig + __ldg(pat.init_pos + e)), bb);
    }
    for (int e = p0; e < p1; ++e) {
      const int c = __ldg(pat.proc_cols + e);
      const int off = __ldg(pat.proc_offsets + e);
      const int base = __ldg(sp.col_spos + c);
      const int u0 = __ldg(sp.upd_ptr + e);
      const float val = ys[(e - p0) * 32];
      for (int q = 0; q < off; ++q) {
        const int s = __ldg(sp.upd_slot + u0 + q);
        ys[s * 32] = ys[s * 32] - L[(size_t)(base + q) * 32] * val;
      }
      const float lval = val * L[(size_t)__ldg(sp.dinv_spos + c) * 32];
      L[(size_t)__ldg(sp.proc_spos + e) * 32] = lval;
      F[(size_t)__ldg(sp.proc_fpos + e) * 32] = lval;
      dk = dk - val * lval;
    }
    L[(size_t)__ldg(sp.dinv_spos + k) * 32] = 1.0f / dk;
  }
}

// ---------------------------------------------------------------------------
// state layout conversions: symbolic-major (KKT row, instance) <-> tile-major U order
// ---------------------------------------------------------------------------

__global__ void state_to_stream_kernel(StreamPlan sp, int n_primal, const float* __restrict__ x,
                                       const float* __restrict__ z, const float* __restrict__ y,
                                       const float* __restrict__ qs, const float* __restrict__ ls,
                                       const float* __restrict__ us, float* __restrict__ s0, float* __restrict__ s1,
                                       float* __restrict__ p0, float* __restrict__ p1, int batch, int n_tiles) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n_tiles * 32) return;
  const int bb = b < batch ? b : batch - 1;
  const int tile = b >> 5, lane = b & 31;
  for (int u = blockIdx.y; u < sp.n; u += gridDim.y) {
    const int o = __ldg(sp.u_orig + u);
    const size_t dst = ((size_t)tile * sp.n + u) * 32 + lane;
    if (o < n_primal) {
      s0[dst] = x[(size_t)o * batch + bb];
      s1[dst] = 0.0f;
      p0[dst] = qs[(size_t)o * batch + bb];
      p1[dst] = 0.0f;
    } else {
      const int r = o - n_primal;
      s0[dst] = z[(size_t)r * batch + bb];
      s1[dst] = y[(size_t)r * batch + bb];
      p0[dst] = ls[(size_t)r * batch + bb];
      p1[dst] = us[(size_t)r * batch + bb];
    }
  }
}

__global__ void stream_to_state_kernel(StreamPlan sp, int n_primal, const float* __restrict__ s0,
                                       const float* __restrict__ s1, float* __restrict__ x, float* __restrict__ z,
                                       float* __restrict__ y, int batch) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= batch) return;
  const int tile = b >> 5, lane = b & 31;
  for (int u = blockIdx.y; u < sp.n; u += gridDim.y) {
    const int o = __ldg(sp.u_orig + u);
    const size_t src = ((size_t)tile * sp.n + u) * 32 + lane;
    if (o < n_primal) {
      x[(size_t)o * batch + b] = s0[src];
    } else {
      const int r = o - n_primal;
      z[(size_t)r * batch + b] = s0[src];
      y[(size_t)r * batch + b] = s1[src];
    }
  }
}

// ---------------------------------------------------------------------------
// streaming ADMM kernel
// ---------------------------------------------------------------------------

struct StreamArgs {
  StreamPlan sp;
  const float* lstream;
  const float* fstream;
  float* s0;
  float* s1;
  const float* p0;
  const float* p1;
  int* status;  // [n_tiles * 32] (ZERO_PIVOT bit), may be null
  int* error;   // one word: 0 ok, 1 pipeline timeout
  int n_tiles, max_iter;
  float sigma, alpha, one_minus_alpha;
  int lstages, sstages;
  int meta_bytes;   // per L stage, 128-byte multiple
  int lbytes;       // per L stage L area
  int sbytes;       // per S stage: 4 arrays x max_rel x 128 bytes
};

enum : int { kItemRel = 0, kItemFwd = 1, kItemBwd = 2 };

constexpr uint64_t kWaitLimitNs = 2000000000ull;  // 2 s: a healthy wait is microseconds

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
// and the backward chunks descending.  Stops (false) when f does.
template <typename F>
__device__ __forceinline__ bool traverse(int n_chunks, int n_fchunks, int max_iter, F& f) {
  for (int ch = n_chunks - 1; ch >= 0; --ch)
    if (!f(kItemRel, ch)) return false;
  for (int it = 0; it < max_iter; ++it) {
    for (int ch = 0; ch < n_fchunks; ++ch)
      if (!f(kItemFwd, ch)) return false;
    for (int ch = n_chunks - 1; ch >= 0; --ch)
      if (!f(kItemBwd, ch)) return false;
  }
  return true;
}

// per-chunk producer table kept in shared memory (8 ints per chunk)
struct ChunkInfo {
  int pos, ent, cols, meta_off, meta_words, u0, nrel, pad;
};

// Shared-memory layout: X [n][32] | chunk table | L ring | S ring | barriers
struct StreamSmem {
  float* X;
  const ChunkInfo* info;
  unsigned char* lring;
  unsigned char* sring;
  uint64_t* lfull;
  uint64_t* lempty;
  uint64_t* sfull;
  uint64_t* sempty;
  volatile int* abort_flag;
  volatile int* consumed_ctr;
};

__host__ __device__ inline size_t stream_smem_bytes(int n, int n_info, int lstages, int sstages, int lstage_bytes,
                                                    int sstage_bytes) {
  return (size_t)n * 128 + (size_t)n_info * sizeof(int) * 8 + (size_t)lstages * lstage_bytes +
         (size_t)sstages * sstage_bytes + 16 * (size_t)(lstages + sstages) + 16;
}

__global__ void __launch_bounds__(64, 1) admm_stream_kernel(StreamArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  const StreamPlan& sp = a.sp;
  const int n = sp.n;
  const int lstage_bytes = a.meta_bytes + a.lbytes;
  StreamSmem sm;
  sm.X = reinterpret_cast<float*>(smem);
  ChunkInfo* info = reinterpret_cast<ChunkInfo*>(smem + (size_t)n * 128);
  ChunkInfo* finfo = info + sp.n_chunks;
  sm.info = info;
  sm.lring = reinterpret_cast<unsigned char*>(finfo + sp.n_fchunks);
  sm.sring = sm.lring + (size_t)a.lstages * lstage_bytes;
  sm.lfull = reinterpret_cast<uint64_t*>(sm.sring + (size_t)a.sstages * a.sbytes);
  sm.lempty = sm.lfull + a.lstages;
  sm.sfull = sm.lempty + a.lstages;
  sm.sempty = sm.sfull + a.sstages;
  sm.abort_flag = reinterpret_cast<volatile int*>(sm.sempty + a.sstages);
  sm.consumed_ctr = sm.abort_flag + 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int c = threadIdx.x; c < sp.n_chunks; c += blockDim.x) {
    const int mw = __ldg(sp.meta_words + c), mo = __ldg(sp.meta_off + c);
    ChunkInfo ci;
    ci.pos = __ldg(sp.chunk_pos + c);
    ci.ent = __ldg(sp.chunk_ent + c);
    ci.cols = __ldg(sp.chunk_cols + c);
    ci.meta_off = mo;
    ci.meta_words = mw;
    ci.u0 = __ldg(sp.meta + mo + 4);
    ci.nrel = __ldg(sp.meta + mo + 2);
    ci.pad = 0;
    info[c] = ci;
  }
  for (int c = threadIdx.x; c < sp.n_fchunks; c += blockDim.x) {
    ChunkInfo ci;
    ci.pos = __ldg(sp.fchunk_pos + c);
    ci.ent = __ldg(sp.fchunk_pos + c + 1) - ci.pos;
    ci.cols = 0;
    ci.meta_off = __ldg(sp.fmeta_off + c);
    ci.meta_words = __ldg(sp.fmeta_words + c);
    ci.u0 = 0;
    ci.nrel = 0;
    ci.pad = 0;
    finfo[c] = ci;
  }
  if (threadIdx.x == 0) {
    for (int s = 0; s < a.lstages; ++s) {
      mbar_init(sm.lfull + s, 1);
      mbar_init(sm.lempty + s, 1);
    }
    for (int s = 0; s < a.sstages; ++s) {
      mbar_init(sm.sfull + s, 1);
      mbar_init(sm.sempty + s, 1);
    }
    *sm.abort_flag = 0;
    *sm.consumed_ctr = 0;
    fence_mbarrier_init();
  }
  __syncthreads();

  uint32_t issued_l = 0, issued_s = 0;

  if (warp == 1) {
    // ------------------------------ producer ------------------------------
    if (lane == 0) {
      Ring lr{0, 0}, sr{0, 0};
      uint32_t nl = 0, ns = 0;  // fills issued so far (ring reuse starts after one full lap)
      for (int tile = blockIdx.x; tile < a.n_tiles && !*sm.abort_flag; tile += gridDim.x) {
        const float* lt = a.lstream + (size_t)tile * sp.stream_len * 32;
        const float* ft = a.fstream + (size_t)tile * sp.nnz_l * 32;
        const size_t soff = (size_t)tile * n * 32;
        auto produce = [&](int kind, int ch) -> bool {
          const ChunkInfo ci = kind == kItemFwd ? finfo[ch] : info[ch];
          const int* meta_src = kind == kItemFwd ? sp.fmeta : sp.meta;
          const float* lsrc = kind == kItemFwd ? ft : lt;
          if (nl >= (uint32_t)a.lstages && !mbar_wait_bounded(sm.lempty + lr.stage, lr.phase ^ 1u, sm.abort_flag, kWaitLimitNs))
            return false;
          uint32_t lcount = 0;
          if (kind == kItemFwd) lcount = ci.ent;
          if (kind == kItemBwd) lcount = ci.ent + ci.cols;
          unsigned char* st = sm.lring + (size_t)lr.stage * lstage_bytes;
          mbar_arrive_expect_tx(sm.lfull + lr.stage, (uint32_t)ci.meta_words * 4u + lcount * 128u);
          bulk_g2s(st, meta_src + ci.meta_off, (uint32_t)ci.meta_words * 4u, sm.lfull + lr.stage);
          if (lcount) bulk_g2s(st + a.meta_bytes, lsrc + (size_t)ci.pos * 32, lcount * 128u, sm.lfull + lr.stage);
          lr.advance(a.lstages);
          ++nl;
          ++issued_l;
          if (kind != kItemFwd) {
            if (ns >= (uint32_t)a.sstages && !mbar_wait_bounded(sm.sempty + sr.stage, sr.phase ^ 1u, sm.abort_flag, kWaitLimitNs))
              return false;
            unsigned char* ss = sm.sring + (size_t)sr.stage * a.sbytes;
            const uint32_t bytes = (uint32_t)ci.nrel * 128u;
            const int quarter = a.sbytes / 4;
            mbar_arrive_expect_tx(sm.sfull + sr.stage, 4u * bytes);
            if (bytes) {
              const size_t off = soff + (size_t)ci.u0 * 32;
              bulk_g2s(ss, a.s0 + off, bytes, sm.sfull + sr.stage);
              bulk_g2s(ss + quarter, a.s1 + off, bytes, sm.sfull + sr.stage);
              bulk_g2s(ss + 2 * quarter, a.p0 + off, bytes, sm.sfull + sr.stage);
              bulk_g2s(ss + 3 * quarter, a.p1 + off, bytes, sm.sfull + sr.stage);
            }
            sr.advance(a.sstages);
            ++ns;
            ++issued_s;
          }
          return true;
        };
        if (!traverse(sp.n_chunks, sp.n_fchunks, a.max_iter, produce)) {
          *sm.abort_flag = 1;
          break;
        }
      }
    }
  } else {
    // ------------------------------ consumer ------------------------------
    Ring lr{0, 0}, sr{0, 0};
    uint32_t consumed = 0;
    const float sigma = a.sigma, alpha = a.alpha, oma = a.one_minus_alpha;
    float* xl = sm.X + lane;
    bool ok = true;
    const int quarter_f = a.sbytes / 16;  // floats per S array
    for (int tile = blockIdx.x; tile < a.n_tiles && ok; tile += gridDim.x) {
      float* s0t = a.s0 + (size_t)tile * n * 32 + lane;
      float* s1t = a.s1 + (size_t)tile * n * 32 + lane;
      int status = 0;
      auto consume = [&](int kind, int ch) -> bool {
        (void)ch;
        if (!mbar_wait_bounded(sm.lfull + lr.stage, lr.phase, sm.abort_flag, kWaitLimitNs)) return false;
        const int* meta = reinterpret_cast<const int*>(sm.lring + (size_t)lr.stage * lstage_bytes);
        const float* Ls = reinterpret_cast<const float*>(sm.lring + (size_t)lr.stage * lstage_bytes + a.meta_bytes) + lane;
        const int ncols = meta[0], nent = meta[1], nrel = meta[2], c0 = meta[3], u0 = meta[4];
        const int* col_start = meta + kMetaHeader;
        const int* rows = col_start + ncols + 1;
        const int* rel_i = rows + nent;
        const int* rel_kind = rel_i + nrel;
        const float* rel_rho = reinterpret_cast<const float*>(rel_kind + nrel);
        const float* rel_rinv = rel_rho + nrel;
        if (kind == kItemFwd) {
          // forward substitution in row-gather form: row i accumulates its
          // columns in ascending order (the reference's order for that row);
          // only a row's last entry can be the previous row, whose value is
          // forwarded in a register.
          const int nrows = meta[0], r0 = meta[2];
          const int* row_start = meta + kFMetaHeader;
          const int* coloff = row_start + nrows + 1;
          int prev_off = -1;
          float prevv = 0.0f;
          for (int i = 0; i < nrows; ++i) {
            const int e0 = row_start[i], e1 = row_start[i + 1];
            const int roff = (r0 + i) * 32;
            float acc = xl[roff];
            if (e0 < e1) {
              const int el = e1 - 1;
              int e = e0;
              for (; e + 4 <= el; e += 4) {
                const int o0 = coloff[e], o1 = coloff[e + 1], o2 = coloff[e + 2], o3 = coloff[e + 3];
                const float l0 = Ls[e * 32], l1 = Ls[(e + 1) * 32], l2 = Ls[(e + 2) * 32], l3 = Ls[(e + 3) * 32];
                const float x0 = xl[o0], x1 = xl[o1], x2 = xl[o2], x3 = xl[o3];
                acc = acc - l0 * x0;
                acc = acc - l1 * x1;
                acc = acc - l2 * x2;
                acc = acc - l3 * x3;
              }
              if (e + 2 <= el) {
                const int o0 = coloff[e], o1 = coloff[e + 1];
                const float l0 = Ls[e * 32], l1 = Ls[(e + 1) * 32];
                const float x0 = xl[o0], x1 = xl[o1];
                acc = acc - l0 * x0;
                acc = acc - l1 * x1;
                e += 2;
              }
              if (e < el) {
                acc = acc - Ls[e * 32] * xl[coloff[e]];
                ++e;
              }
              const int cl = coloff[el];
              acc = acc - Ls[el * 32] * (cl == prev_off ? prevv : xl[cl]);
              xl[roff] = acc;
            }
            prev_off = roff;
            prevv = acc;
          }
        } else {
          if (kind == kItemBwd) {
            // backward substitution, reverse column order; a column's first
            // entry may read the column just finished (forwarded)
            int prev_off = -1;
            float prevv = 0.0f;
            for (int j = ncols - 1; j >= 0; --j) {
              const int e0 = col_start[j], e1 = col_start[j + 1];
              const int coff = (c0 + j) * 32;
              const float xself = xl[coff];
              const float dinv = Ls[(nent + j) * 32];
              float corr = 0.0f;
              if (e0 < e1) {
                const int r0 = rows[e0];
                corr = corr + Ls[e0 * 32] * (r0 == prev_off ? prevv : xl[r0]);
                int e = e0 + 1;
                for (; e + 4 <= e1; e += 4) {
                  const int o0 = rows[e], o1 = rows[e + 1], o2 = rows[e + 2], o3 = rows[e + 3];
                  const float l0 = Ls[e * 32], l1 = Ls[(e + 1) * 32], l2 = Ls[(e + 2) * 32], l3 = Ls[(e + 3) * 32];
                  const float x0 = xl[o0], x1 = xl[o1], x2 = xl[o2], x3 = xl[o3];
                  corr = corr + l0 * x0;
                  corr = corr + l1 * x1;
                  corr = corr + l2 * x2;
                  corr = corr + l3 * x3;
                }
                if (e + 2 <= e1) {
                  const int o0 = rows[e], o1 = rows[e + 1];
                  const float l0 = Ls[e * 32], l1 = Ls[(e + 1) * 32];
                  const float x0 = xl[o0], x1 = xl[o1];
                  corr = corr + l0 * x0;
                  corr = corr + l1 * x1;
                  e += 2;
                }
                if (e < e1) corr = corr + Ls[e * 32] * xl[rows[e]];
              }
              if (!(dinv != 0.0f) || !isfinite(dinv)) status |= WMPC_STATUS_ZERO_PIVOT;
              const float res = xself * dinv - corr;
              xl[coff] = res;
              prev_off = coff;
              prevv = res;
            }
          }
          // releases: ADMM update (backward items) or first right-hand side
          if (!mbar_wait_bounded(sm.sfull + sr.stage, sr.phase, sm.abort_flag, kWaitLimitNs)) return false;
          const float* S = reinterpret_cast<const float*>(sm.sring + (size_t)sr.stage * a.sbytes) + lane;
          for (int k = 0; k < nrel; ++k) {
            const int ioff = rel_i[k] * 32;
            const float sv0 = S[k * 32], pv0 = S[2 * quarter_f + k * 32];
            const size_t u = (size_t)(u0 + k) * 32;
            if (kind == kItemRel) {
              xl[ioff] = rel_kind[k] == 0 ? sigma * sv0 - pv0 : sv0 - rel_rinv[k] * S[quarter_f + k * 32];
              continue;
            }
            const float sol = xl[ioff];
            if (rel_kind[k] == 0) {
              const float xn = alpha * sol + oma * sv0;
              s0t[u] = xn;
              xl[ioff] = sigma * xn - pv0;
            } else {
              const float yk = S[quarter_f + k * 32], pv1 = S[3 * quarter_f + k * 32];
              const float rinv = rel_rinv[k];
              const float rz = sv0 - rinv * yk;
              const float zt = rz + rinv * sol;
              const float zr = alpha * zt + oma * sv0;
              float zn = zr + rinv * yk;
              zn = (zn < pv0) ? pv0 : zn;
              zn = (zn > pv1) ? pv1 : zn;
              const float yn = yk + rel_rho[k] * (zr - zn);
              s0t[u] = zn;
              s1t[u] = yn;
              xl[ioff] = zn - rinv * yn;
            }
          }
          // order these generic-proxy state writes before the bulk copies
          // that read them back in the next iteration
          if (kind == kItemBwd) fence_proxy_async_global();
          __syncwarp();
          if (lane == 0) mbar_arrive(sm.sempty + sr.stage);
          sr.advance(a.sstages);
        }
        __syncwarp();
        if (lane == 0) {
          mbar_arrive(sm.lempty + lr.stage);
          *sm.consumed_ctr = (int)(consumed + 1);
        }
        lr.advance(a.lstages);
        ++consumed;
        return true;
      };
      if (!traverse(sp.n_chunks, sp.n_fchunks, a.max_iter, consume)) ok = false;
      if (ok && a.status) a.status[tile * 32 + lane] = status;
    }
    if (!ok && lane == 0) *sm.abort_flag = 1;
  }
  __syncthreads();
  if (*sm.abort_flag) {
    if (threadIdx.x == 32) {
      // drain: wait (bounded) for every bulk copy issued but not consumed
      const uint32_t consumed = (uint32_t)*sm.consumed_ctr;
      for (uint32_t t = consumed; t < issued_l; ++t)
        mbar_wait_bounded(sm.lfull + t % a.lstages, (t / a.lstages) & 1u, nullptr, kWaitLimitNs);
      const uint32_t s_lo = issued_s > (uint32_t)a.sstages ? issued_s - a.sstages : 0;
      for (uint32_t t = s_lo; t < issued_s; ++t)
        mbar_wait_bounded(sm.sfull + t % a.sstages, (t / a.sstages) & 1u, nullptr, kWaitLimitNs);
    }
    if (threadIdx.x == 0) atomicExch(a.error, 1);
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

bool stream_launch_config(const StreamPlan& sp, StreamLaunch* cfg) {
  const int mw = sp.max_meta_words > sp.max_fmeta_words ? sp.max_meta_words : sp.max_fmeta_words;
  const int meta_bytes = ((mw * 4 + 127) / 128) * 128;
  const int lent = (sp.max_ent + sp.max_cols) > sp.max_fent ? (sp.max_ent + sp.max_cols) : sp.max_fent;
  const int lbytes = lent * 128;
  const int sbytes = 4 * (sp.max_rel > 0 ? sp.max_rel : 1) * 128;
  // prefer deep rings: as many L stages as fit with at least 3 S stages
  for (int ls = 12; ls >= 2; --ls)
    for (int ss = 6; ss >= 2; --ss) {
      const size_t bytes = stream_smem_bytes(sp.n, sp.n_chunks + sp.n_fchunks, ls, ss, meta_bytes + lbytes, sbytes);
      if (bytes <= (size_t)kMaxSmemBytes && (ss >= 3 || ls <= 3)) {
        cfg->stages = ls;
        cfg->sstages = ss;
        cfg->meta_bytes = meta_bytes;
        cfg->lbytes = lbytes;
        cfg->sbytes = sbytes;
        cfg->smem = bytes;
        return true;
      }
    }
  return false;
}

size_t stream_workspace_floats(const StreamPlan& sp, int batch) {
  const size_t tiles = (size_t)(batch + 31) / 32;
  return tiles * 32 * ((size_t)sp.stream_len + (size_t)sp.nnz_l + 4 * (size_t)sp.n) + 64;
}

int launch_stream_solve(const Pattern& pat, const StreamPlan& sp, const Osqp& o, const float* pT, long long ldp,
                        int sbp, const float* aT, long long lda, int sba, float* x, float* z, float* y,
                        const float* qs, const float* ls, const float* us, float* work, int* status, int* error,
                        int batch, int max_iter, int num_sms, bool reuse_factor, cudaStream_t s) {
  StreamLaunch cfg;
  if (!stream_launch_config(sp, &cfg)) return fail(WMPC_ERR_UNSUPPORTED, "pattern too large for the streaming kernel");
  const int n_tiles = (batch + 31) / 32;
  const size_t tl = (size_t)n_tiles * 32;
  float* lstream = work;
  float* fstream = lstream + tl * sp.stream_len;
  float* s0 = fstream + tl * sp.nnz_l;
  float* s1 = s0 + tl * sp.n;
  float* p0 = s1 + tl * sp.n;
  float* p1 = p0 + tl * sp.n;
  OsqpInputs in{pT, ldp, sbp, aT, lda, sba};
  if (!reuse_factor) {
    const int warps = 4;
    const size_t smem = (size_t)warps * (sp.max_row_nnz > 0 ? sp.max_row_nnz : 1) * 32 * sizeof(float);
    WMPC_CUDA_TRY(cudaFuncSetAttribute(factor_stream_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    factor_stream_kernel<<<ceil_div(n_tiles, warps), warps * 32, smem, s>>>(pat, sp, o, in, lstream, fstream, n_tiles,
                                                                            batch);
    WMPC_LAUNCH_CHECK();
  }
  {
    dim3 grid(ceil_div(tl, 128), sp.n < 1024 ? sp.n : 1024);
    state_to_stream_kernel<<<grid, 128, 0, s>>>(sp, o.n, x, z, y, qs, ls, us, s0, s1, p0, p1, batch, n_tiles);
    WMPC_LAUNCH_CHECK();
  }
  StreamArgs a{sp, lstream, fstream, s0, s1, p0, p1, status, error, n_tiles, max_iter, o.sigma, o.alpha,
               o.one_minus_alpha, cfg.stages, cfg.sstages, cfg.meta_bytes, cfg.lbytes, cfg.sbytes};
  const int grid = n_tiles < num_sms ? n_tiles : num_sms;
  WMPC_CUDA_TRY(cudaFuncSetAttribute(admm_stream_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cfg.smem));
  profile_mark_begin(s);
  admm_stream_kernel<<<grid, 64, cfg.smem, s>>>(a);
  profile_mark_end(s);
  WMPC_LAUNCH_CHECK();
  {
    dim3 grid2(ceil_div(batch, 128), sp.n < 1024 ? sp.n : 1024);
    stream_to_state_kernel<<<grid2, 128, 0, s>>>(sp, o.n, s0, s1, x, z, y, batch);
    WMPC_LAUNCH_CHECK();
  }
  return WMPC_OK;
}

}  // namespace wmpc

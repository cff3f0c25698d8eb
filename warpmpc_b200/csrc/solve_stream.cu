// Per-call batched triangular solve fed by TMA (sm_100a): x = P^T L^-T D^-1 L^-1 P rhs
// for 32 instances per CTA (one per lane), L and D^-1 read in the caller's
// layout ([entry][instance], the reference's "symbolic-major" Warp layout).
//
// One warp (the producer) walks the tile's work items and brings each one's
// operands into a ring of shared-memory stages with 2-D tensor copies
// (cp.async.bulk.tensor, boxes of 32 rows x 32 instances = 4 KB) plus a 1-D
// bulk copy of the item's index table; an mbarrier per stage signals arrival.
// The other warp (the sweeper) works on the stage from shared memory:
//   rhs items      rows of rhs in natural order, scattered into the work
//                  vector X through pinv (X = P rhs);
//   forward chunks a run of whole L columns (ascending): for each column c
//                  with entries, x_r -= L_rc x_c for its rows r (scatter);
//   backward chunks the same runs in reverse, with D^-1 of their columns:
//                  x_c = x_c D^-1_c - sum_r L_rc x_r (gather, ascending r);
// then the tile's result rows are stored, unpermuted, to out.  X ([row][lane],
// conflict-free, plus a trash row and a zero row) stays in shared memory for
// the whole tile.  Chunks end on column boundaries, so every column's entries
// sit in one stage.  A column is worked kStep entries at a time: the step's
// index words, L values and work-vector reads are all issued before its
// arithmetic (padding slots write the trash row, or read L = 0 times the
// zero row), so one shared-memory round trip per step is on the sweep's
// critical path instead of one per entry.
//
// Operation order is the reference's serial solve (warpmpc/jax_qdldl/
// warp_backend.py:193-218: column-scatter forward substitution, D^-1, then
// row-gather backward substitution with the correction summed first); the
// D^-1 scaling of x_c is deferred to column c's backward step, where it is
// the same single rounding.  Compiled with -fmad=false: bit-identical to the
// one-lane-per-instance kernel and to the float32 oracle.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "qdldl.cuh"
#include "stream.cuh"

namespace wmpc {

namespace {

constexpr int kBox = 32;                                 // rows per tensor copy
constexpr int kChunkEntries = 64;                        // L entries per chunk, at most
constexpr int kChunkCols = 32;                           // columns per chunk, at most
constexpr int kRhsRows = 96;                             // rhs rows per item
constexpr int kTableBytes = 512;                         // index table area of a stage
constexpr int kDataBytes = (kChunkEntries + kChunkCols) * 128;  // L rows, then D^-1 rows
constexpr int kStageBytes = kTableBytes + kDataBytes;    // 12800 (a multiple of 128)
constexpr int kMaxStages = 8;
constexpr int kStep = 8;  // L entries of one column a sweeper step loads before its arithmetic
constexpr uint64_t kSolveWaitNs = 2000000000ull;          // 2 s: a healthy wait is microseconds
static_assert(kRhsRows * 128 <= kDataBytes, "an rhs item must fit the data area");
static_assert((4 + kChunkCols + kChunkEntries) * 4 <= kTableBytes, "a chunk table must fit its area");
// a step may read kStep - 1 table words and L rows past a chunk's last entry
static_assert((4 + kChunkCols + kChunkEntries + kStep - 1) * 4 <= kTableBytes, "step reads past the table area");
static_assert(kChunkEntries + kStep - 1 <= kChunkEntries + kChunkCols, "step reads past the stage's L rows");

enum : int { kSolveRhs = 0, kSolveFwd = 1, kSolveBwd = 2 };

struct __align__(64) SolveArgs {
  CUtensorMap tm_l;     // lx   [nnz_l][batch] float32, boxes 32 x 32
  CUtensorMap tm_d;     // dinv [n][batch]
  CUtensorMap tm_r;     // rhs  [n][batch]
  const int* tables;    // chunk index tables (16-byte aligned chunks)
  const int4* desc;     // per chunk: {table word offset, table words, e0, c0}, {entries, columns, 0, 0}
  const int* pinv;      // [n]
  float* out;           // [n][batch]
  int n, batch, n_tiles, n_chunks, stages;
  unsigned long long wait_limit_ns;
};

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// Items of one tile: rhs blocks, forward chunks ascending, backward chunks descending.
__device__ __forceinline__ void item_of(int i, int n_rhs, int n_chunks, int& kind, int& k) {
  if (i < n_rhs) {
    kind = kSolveRhs;
    k = i;
  } else if (i < n_rhs + n_chunks) {
    kind = kSolveFwd;
    k = i - n_rhs;
  } else {
    kind = kSolveBwd;
    k = n_chunks - 1 - (i - n_rhs - n_chunks);
  }
}

__global__ void __launch_bounds__(64, 1) solve_stream_kernel(const __grid_constant__ SolveArgs a) {
  extern __shared__ __align__(1024) unsigned char smem[];
  const int n = a.n;
  const int S = a.stages;
  float* X = reinterpret_cast<float*>(smem);  // [n + 2][32]: rows, a trash row, a zero row
  unsigned char* ring = smem + (((size_t)(n + 2) * 128 + 1023) / 1024) * 1024;  // S stages
  uint64_t* full = reinterpret_cast<uint64_t*>(ring + (size_t)S * kStageBytes);
  uint64_t* empty = full + S;
  volatile int* abort_flag = reinterpret_cast<volatile int*>(empty + S);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n_rhs = (n + kRhsRows - 1) / kRhsRows;
  const int per_tile = n_rhs + 2 * a.n_chunks;
  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(full + s, 1);
      mbar_init(empty + s, 1);
    }
    *abort_flag = 0;
    fence_mbarrier_init();
  }
  __syncthreads();
  uint32_t issued = 0;  // producer lane 0: items issued

  if (warp == 1) {
    // ------------------------------ producer ------------------------------
    if (lane == 0) {
      uint32_t stage = 0, phase = 0;
      bool ok = true;
      for (int tile = blockIdx.x; tile < a.n_tiles && ok; tile += gridDim.x) {
        const int x = tile * 32;
        for (int i = 0; i < per_tile && ok; ++i) {
          int kind, k;
          item_of(i, n_rhs, a.n_chunks, kind, k);
          if (issued >= (uint32_t)S && !mbar_wait_bounded(empty + stage, phase ^ 1u, abort_flag, a.wait_limit_ns)) {
            ok = false;
            break;
          }
          unsigned char* st = ring + (size_t)stage * kStageBytes;
          unsigned char* data = st + kTableBytes;
          if (kind == kSolveRhs) {
            const int r0 = k * kRhsRows;
            const int rows = min(kRhsRows, n - r0);
            const int boxes = (rows + kBox - 1) / kBox;
            mbar_arrive_expect_tx(full + stage, (uint32_t)boxes * kBox * 128u);
            for (int b = 0; b < boxes; ++b) tma_load_2d(data + b * kBox * 128, &a.tm_r, x, r0 + b * kBox, full + stage);
          } else {
            const int4 d0 = __ldg(a.desc + 2 * k), d1 = __ldg(a.desc + 2 * k + 1);
            const int lboxes = (d1.x + kBox - 1) / kBox;
            const int dboxes = kind == kSolveBwd ? (d1.y + kBox - 1) / kBox : 0;
            mbar_arrive_expect_tx(full + stage, (uint32_t)d0.y * 4u + (uint32_t)(lboxes + dboxes) * kBox * 128u);
            bulk_g2s(st, a.tables + d0.x, (uint32_t)d0.y * 4u, full + stage);
            for (int b = 0; b < lboxes; ++b) tma_load_2d(data + b * kBox * 128, &a.tm_l, x, d0.z + b * kBox, full + stage);
            for (int b = 0; b < dboxes; ++b)
              tma_load_2d(data + kChunkEntries * 128 + b * kBox * 128, &a.tm_d, x, d0.w + b * kBox, full + stage);
          }
          ++issued;
          if (++stage == (uint32_t)S) {
            stage = 0;
            phase ^= 1u;
          }
        }
      }
      if (!ok) *abort_flag = 1;
    }
  } else {
    // ------------------------------ sweeper ------------------------------
    uint32_t stage = 0, phase = 0;
    bool ok = true;
    unsigned char* xb = smem + lane * 4;  // this lane's column of X (row r at xb + 128 r)
    const int trash_off = n * 128, zero_off = (n + 1) * 128;
    X[(n + 1) * 32 + lane] = 0.0f;
    int tile = blockIdx.x;
    for (; tile < a.n_tiles && ok; tile += gridDim.x) {
      for (int i = 0; i < per_tile; ++i) {
        int kind, k;
        item_of(i, n_rhs, a.n_chunks, kind, k);
        if (!mbar_wait_bounded(full + stage, phase, abort_flag, a.wait_limit_ns)) {
          ok = false;
          break;
        }
        const unsigned char* st = ring + (size_t)stage * kStageBytes;
        const float* data = reinterpret_cast<const float*>(st + kTableBytes) + lane;
        if (kind == kSolveRhs) {
          const int r0 = k * kRhsRows;
          const int rows = min(kRhsRows, n - r0);
          int r = 0;
          for (; r + 4 <= rows; r += 4) {
            const int p0 = __ldg(a.pinv + r0 + r), p1 = __ldg(a.pinv + r0 + r + 1);
            const int p2 = __ldg(a.pinv + r0 + r + 2), p3 = __ldg(a.pinv + r0 + r + 3);
            const float v0 = data[r * 32], v1 = data[(r + 1) * 32], v2 = data[(r + 2) * 32], v3 = data[(r + 3) * 32];
            X[p0 * 32 + lane] = v0;
            X[p1 * 32 + lane] = v1;
            X[p2 * 32 + lane] = v2;
            X[p3 * 32 + lane] = v3;
          }
          for (; r < rows; ++r) X[__ldg(a.pinv + r0 + r) * 32 + lane] = data[r * 32];
        } else {
          const int* tb = reinterpret_cast<const int*>(st);
          const int C = tb[0], c0 = tb[2];
          const int* cend = tb + 4;
          const int* roff = tb + 4 + C;  // byte offsets (row * 128) into X
          if (kind == kSolveFwd) {
            // x_r -= L_rc x_c over column c's rows (distinct rows: independent),
            // kStep entries at a time with all their loads issued before the
            // arithmetic; slots past the column's end update the trash row
            int b = 0;
            for (int j = 0; j < C; ++j) {
              const int e = cend[j];
              if (e > b) {
                const float val = X[(c0 + j) * 32 + lane];
                for (int q = b; q < e; q += kStep) {
                  int o[kStep];
                  float l[kStep], w[kStep];
#pragma unroll
                  for (int i = 0; i < kStep; ++i) {
                    o[i] = q + i < e ? roff[q + i] : trash_off;
                    l[i] = data[(q + i) * 32];
                  }
#pragma unroll
                  for (int i = 0; i < kStep; ++i) w[i] = *reinterpret_cast<const float*>(xb + o[i]);
#pragma unroll
                  for (int i = 0; i < kStep; ++i) *reinterpret_cast<float*>(xb + o[i]) = w[i] - l[i] * val;
                }
              }
              b = e;
            }
          } else {
            // x_c = x_c D^-1_c - sum_r L_rc x_r (rows ascending), columns descending;
            // slots past the column's end add L = 0 times the zero row (+0: the
            // sum keeps its bits)
            const float* dv = data + kChunkEntries * 32;
            for (int j = C - 1; j >= 0; --j) {
              const int b = j > 0 ? cend[j - 1] : 0, e = cend[j];
              float corr = 0.0f;
              for (int q = b; q < e; q += kStep) {
                int o[kStep];
                float l[kStep], w[kStep];
#pragma unroll
                for (int i = 0; i < kStep; ++i) {
                  const bool v = q + i < e;
                  o[i] = v ? roff[q + i] : zero_off;
                  l[i] = v ? data[(q + i) * 32] : 0.0f;
                }
#pragma unroll
                for (int i = 0; i < kStep; ++i) w[i] = *reinterpret_cast<const float*>(xb + o[i]);
#pragma unroll
                for (int i = 0; i < kStep; ++i) corr = corr + l[i] * w[i];
              }
              float* xc = X + (c0 + j) * 32 + lane;
              *xc = *xc * dv[j * 32] - corr;
            }
          }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(empty + stage);
        if (++stage == (uint32_t)S) {
          stage = 0;
          phase ^= 1u;
        }
      }
      if (!ok) break;
      // the tile's solution, unpermuted: out row i is X row pinv[i]
      const int col = tile * 32 + lane;
      if (col < a.batch) {
        float* o = a.out + col;
        int r = 0;
        for (; r + 4 <= n; r += 4) {
          const int p0 = __ldg(a.pinv + r), p1 = __ldg(a.pinv + r + 1), p2 = __ldg(a.pinv + r + 2),
                    p3 = __ldg(a.pinv + r + 3);
          const float v0 = X[p0 * 32 + lane], v1 = X[p1 * 32 + lane], v2 = X[p2 * 32 + lane], v3 = X[p3 * 32 + lane];
          o[(size_t)r * a.batch] = v0;
          o[(size_t)(r + 1) * a.batch] = v1;
          o[(size_t)(r + 2) * a.batch] = v2;
          o[(size_t)(r + 3) * a.batch] = v3;
        }
        for (; r < n; ++r) o[(size_t)r * a.batch] = X[__ldg(a.pinv + r) * 32 + lane];
      }
      __syncwarp();
    }
    if (!ok) {
      *abort_flag = 1;
      // results of this CTA's unfinished tiles are invalid: make them visibly so
      const float nan = __int_as_float(0x7fc00000);
      for (; tile < a.n_tiles; tile += gridDim.x) {
        const int col = tile * 32 + lane;
        if (col < a.batch)
          for (int r = 0; r < n; ++r) a.out[(size_t)r * a.batch + col] = nan;
      }
    }
  }
  __syncthreads();
  if (*abort_flag && threadIdx.x == 32) {
    // drain: wait (bounded) for the last copy issued into every stage
    for (uint32_t s = 0; s < (uint32_t)S && s < issued; ++s) {
      const uint32_t last = s + (uint32_t)S * ((issued - 1 - s) / (uint32_t)S);
      mbar_wait_bounded(full + s, (last / (uint32_t)S) & 1u, nullptr, kSolveWaitNs);
    }
  }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    else
      (void)cudaGetLastError();
  });
  return fn;
}

// [rows][batch] float32 at `base`, boxes of 32 instances x 32 rows.
bool encode_rows(CUtensorMap* map, const float* base, int rows, int batch) {
  auto fn = encode_fn();
  if (!fn) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)batch, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)batch * 4u};
  const cuuint32_t box[2] = {32u, (cuuint32_t)kBox};
  const cuuint32_t elem[2] = {1u, 1u};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims, strides, box, elem,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

size_t solve_smem_bytes(int n, int stages) {
  return (((size_t)(n + 2) * 128 + 1023) / 1024) * 1024 + (size_t)stages * kStageBytes + 16 * (size_t)stages + 16;
}

}  // namespace

// Chunks of whole columns (at most kChunkEntries entries and kChunkCols
// columns each) and their index tables.  Returns false when a column has
// more entries than a chunk holds (the solve then uses the one-lane kernel).
bool build_solve_tables(int n, const std::vector<int>& lp, const std::vector<int>& li, std::vector<int>* tables,
                        std::vector<int>* desc) {
  tables->clear();
  desc->clear();
  int c0 = 0;
  while (c0 < n) {
    int c1 = c0;
    while (c1 < n && c1 - c0 < kChunkCols && lp[c1 + 1] - lp[c0] <= kChunkEntries) ++c1;
    if (c1 == c0) return false;  // column c0 alone exceeds a chunk
    const int C = c1 - c0, e0 = lp[c0], E = lp[c1] - e0;
    const int toff = (int)tables->size();
    tables->push_back(C);
    tables->push_back(E);
    tables->push_back(c0);
    tables->push_back(e0);
    for (int c = c0; c < c1; ++c) tables->push_back(lp[c + 1] - e0);
    for (int e = e0; e < e0 + E; ++e) tables->push_back(li[e] * 128);
    while (tables->size() % 4) tables->push_back(0);
    const int words = (int)tables->size() - toff;
    desc->insert(desc->end(), {toff, words, e0, c0, E, C, 0, 0});
    c0 = c1;
  }
  return true;
}

// The TMA-fed solve when it applies: one factor per instance (fstride 1),
// batch a multiple of 4 (16-byte row pitch), 16-byte aligned arrays, the
// plan's chunk tables built, and the work vector plus two stages in shared
// memory.  *applied is false when it did not apply (the caller then runs
// the one-lane kernel); the return value is a WMPC status.
int launch_solve_stream(const wmpc_plan& plan, const float* lx, const float* dinv, int fstride, const float* rhs,
                        float* x, int batch, cudaStream_t s, bool* applied) {
  const Pattern& pat = plan.pat;
  *applied = false;
  if (!plan.solve_tables || pat.nnz_l == 0 || fstride != 1 || batch % 4 != 0 || env_disabled("WMPC_SOLVE_STREAM_OFF"))
    return WMPC_OK;
  if ((reinterpret_cast<uintptr_t>(lx) | reinterpret_cast<uintptr_t>(dinv) | reinterpret_cast<uintptr_t>(rhs)) & 15)
    return WMPC_OK;
  int dev = plan.device, sm_bytes = 0, num_sms = 0;
  if (cudaDeviceGetAttribute(&sm_bytes, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    (void)cudaGetLastError();
    return WMPC_OK;
  }
  int stages = kMaxStages;
  while (stages >= 2 && solve_smem_bytes(pat.n, stages) > (size_t)sm_bytes) --stages;
  if (stages < 2) return WMPC_OK;
  SolveArgs a;
  if (!encode_rows(&a.tm_l, lx, pat.nnz_l, batch) || !encode_rows(&a.tm_d, dinv, pat.n, batch) ||
      !encode_rows(&a.tm_r, rhs, pat.n, batch))
    return WMPC_OK;
  a.tables = plan.solve_tables;
  a.desc = reinterpret_cast<const int4*>(plan.solve_desc);
  a.pinv = pat.pinv;
  a.out = x;
  a.n = pat.n;
  a.batch = batch;
  a.n_tiles = (batch + 31) / 32;
  a.n_chunks = plan.solve_chunks;
  a.stages = stages;
  a.wait_limit_ns = kSolveWaitNs;
  const size_t smem = solve_smem_bytes(pat.n, stages);
  if (cudaFuncSetAttribute(solve_stream_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess) {
    (void)cudaGetLastError();
    return WMPC_OK;
  }
  int per_sm = 1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, solve_stream_kernel, 64, smem) != cudaSuccess ||
      per_sm < 1) {
    (void)cudaGetLastError();
    per_sm = 1;
  }
  const int grid = std::min(a.n_tiles, per_sm * num_sms);
  *applied = true;
  solve_stream_kernel<<<grid, 64, smem, s>>>(a);
  WMPC_LAUNCH_CHECK();
  return WMPC_OK;
}

}  // namespace wmpc

// Shared definitions of the warpmpc_b200 CUDA library (sm_100a).
//
// Data layout in HBM: every per-instance array is "symbolic-major",
// element (i, b) at [i * ld + b]: one row per KKT index / L entry / value
// slot, one column per instance.  A warp owns 32 consecutive instances, so
// each of its loads and stores of row i is one contiguous 128-byte line.
// The per-pattern index tables are shared by all instances; every lane of a
// warp reads the same table entry (a broadcast).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdarg>
#include <cstdlib>
#include <cstdio>
#include <string>

#include "../../include/warpmpc_b200.h"

namespace wmpc {

// Thread-local last error message (wmpc_last_error_string).
void set_error(const char* fmt, ...);
int fail(int code, const char* fmt, ...);

// Launch accounting and per-channel kernel timing (wmpc_profile_begin/end):
// marks of the channel selected by wmpc_profile_select record event pairs,
// the others are ignored.
constexpr int kProfileDominant = 0;  // the step's dominant kernel (ADMM sweeps, per-call solves, ...)
constexpr int kProfileFactor = 1;    // factorization kernels
void count_launch();
void profile_mark_begin(cudaStream_t s, int channel = kProfileDominant);
void profile_mark_end(cudaStream_t s, int channel = kProfileDominant);
// The last streaming ADMM launch (wmpc_stream_last_launch).
void record_stream_launch(int form, int ctas_per_sm, int grid, int smem_bytes);

#define WMPC_CUDA_TRY(expr)                                                              \
  do {                                                                                   \
    cudaError_t err__ = (expr);                                                          \
    if (err__ != cudaSuccess)                                                            \
      return ::wmpc::fail(WMPC_ERR_CUDA, "%s failed: %s (%s:%d)", #expr,                   \
                          cudaGetErrorString(err__), __FILE__, __LINE__);                \
  } while (0)

#define WMPC_LAUNCH_CHECK()                                                              \
  do {                                                                                   \
    ::wmpc::count_launch();                                                              \
    cudaError_t err__ = cudaGetLastError();                                              \
    if (err__ != cudaSuccess)                                                            \
      return ::wmpc::fail(WMPC_ERR_CUDA, "kernel launch failed: %s (%s:%d)",              \
                          cudaGetErrorString(err__), __FILE__, __LINE__);                \
  } while (0)

// Device-resident pattern tables of one QDLDL plan (all int32).
struct Pattern {
  int n, nnz_a, nnz_l;
  int max_row_nnz, max_col_nnz;
  const int* perm_to_orig;  // [nnz_a]
  const int* diag_pos;      // [n]
  const int* init_ptr;      // [n+1]
  const int* init_rows;     // [.]
  const int* init_pos;      // [.]
  const int* proc_ptr;      // [n+1]
  const int* proc_cols;     // [nnz_l]
  const int* proc_lidx;     // [nnz_l]
  const int* proc_offsets;  // [nnz_l]
  const int* lp;            // [n+1]
  const int* li;            // [nnz_l]
  const int* p;             // [n]
  const int* pinv;          // [n]
};

// Largest dynamic shared memory a kernel may request (B200: 227 KB).
constexpr int kMaxSmemBytes = 227 * 1024;
// Budget for per-lane work vectors staged in shared memory.
constexpr int kWorkSmemBudget = 200 * 1024;

// Threads per block when every lane keeps `rows` floats in shared memory;
// 0 when even one warp does not fit (the work vector then lives in HBM).
inline int smem_lanes_for_rows(int rows) {
  if (rows <= 0) return 256;
  long long per_lane = 4LL * rows;
  long long lanes = kWorkSmemBudget / per_lane;
  if (lanes >= 256) return 256;
  return static_cast<int>((lanes / 32) * 32);
}

// Per-lane vector view: shared memory [row][lane] or HBM [row][instance].
struct LaneVec {
  float* base;
  long long stride;
  __device__ __forceinline__ float& operator()(int i) const { return base[i * stride]; }
};

inline unsigned ceil_div(long long a, long long b) { return static_cast<unsigned>((a + b - 1) / b); }

// Environment switch (testing/diagnostics): "1" disables a code path.
inline bool env_disabled(const char* name) {
  const char* v = getenv(name);
  return v && v[0] == '1';
}

}  // namespace wmpc

#include <vector>

struct wmpc_plan {
  int device = 0;
  wmpc::Pattern pat{};
  int* table_block = nullptr;  // single device allocation holding every table
  size_t table_ints = 0;
  // chunk index tables of the TMA-fed per-call solve (null: not applicable)
  const int* solve_tables = nullptr;
  const int* solve_desc = nullptr;  // two int4 per chunk
  int solve_chunks = 0;
  // compact-accumulator tables of the staged per-call factorization (null:
  // the one-lane kernel factors): slot of each initial entry in its row's
  // reach, per program entry its range of updates, per update its target
  // slot and the L entry it re-reads
  const int* fac_init_slot = nullptr;
  const int* fac_upd_ptr = nullptr;
  const int* fac_upd_slot = nullptr;
  const int* fac_upd_lidx = nullptr;
  const int4* fac_row_info = nullptr;  // per row {p0, p1, i0, i1}, {first update, update end, first input, 0}
  const int* fac_kin_slot = nullptr;   // per row, per KKT input: its original KKT slot
  int fac_max_row = 0, fac_max_kv = 0;
  // host copies of the ragged program (inputs of the streaming schedule)
  std::vector<int> h_init_ptr, h_init_rows, h_proc_ptr, h_proc_cols, h_proc_offsets, h_proc_lidx, h_lp, h_li, h_p;
  // host copies of the KKT-slot tables (inputs of the factorization's row descriptors)
  std::vector<int> h_perm_to_orig, h_diag_pos, h_init_pos;
};

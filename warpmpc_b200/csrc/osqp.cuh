// Device-side OSQP problem description (one FixedOSQPPlan) and launchers.
#pragma once

#include "common.cuh"
#include "stream.cuh"

namespace wmpc {

struct Osqp {
  int n, m, nk;          // variables, constraints, KKT dimension (n + m)
  int nnz_p, nnz_a, nnz_kkt, nnz_pf;
  float sigma, alpha, one_minus_alpha;
  // KKT value assembly: slot s takes kkt_base[s], or P entry / A entry j
  // scaled: kkt_src[s] = -1 (base), j (P entry j) or nnz_p + j (A entry j).
  const float* kkt_base;
  const int* kkt_src;
  // per factorization row, per KKT input in row-program order (the diagonal,
  // then the row's initial entries): {P/A entry or -1, kind (0 base value,
  // 1 P entry, 2 A entry), scale bits, add bits} -- the row's inputs of
  // kkt_base / kkt_src / p_scale / p_diag_sigma / a_scale resolved
  const int4* kin_desc;       // [n + m + initial entries]
  const int4* kin_desc_rho;   // the same with each -1/rho input taken from the instance's 1/rho row (kind 3)
  const float* p_scale;       // [nnz_p]
  const float* p_diag_sigma;  // [nnz_p]
  const float* a_scale;       // [nnz_a]
  // A by rows (entries of row r in storage order = ascending column)
  const int* a_row_ptr;       // [m+1]
  const int* a_row_ent;       // [nnz_a] A entry index
  const int* a_cols;          // [nnz_a]
  const int* a_rows;          // [nnz_a]
  const int* a_col_ptr;       // [n+1] CSC pointers of A
  // both triangles of P grouped by row, in the reference's entry order
  const int* pf_row_ptr;      // [n+1]
  const int* pf_val;          // [nnz_pf] P upper entry index
  const int* pf_col;          // [nnz_pf]
  const float* rho;           // [m]
  const float* rho_inv;       // [m]
  const float* q_scale;       // [n]
  const float* scaling_d;     // [n]
  const float* scaling_dinv;  // [n]
  const float* scaling_e;     // [m]
  const float* scaling_einv;  // [m]
  const float* y_scale;       // [m]
  const float* y_unscale;     // [m]
  // rho adaptation (null when the problem was created without its tables)
  const int* rho_type;        // [m] -1 loose, 0 inequality, 1 equality
  const int* kkt_rho_row;     // [nnz_kkt] constraint of a -1/rho slot, else -1
  float rho0;                 // the plan's scalar rho
};

}  // namespace wmpc

struct wmpc_osqp {
  int device = 0;
  int num_sms = 0;
  wmpc::Osqp dev{};
  const wmpc_plan* kkt_plan = nullptr;
  void* block = nullptr;  // single device allocation holding every table
  const int* p_upper_rows = nullptr;  // [nnz_p] row of every stored upper entry of P
  const int* p_upper_cols = nullptr;  // [nnz_p]
  int ctas_limit = 2;  // most CTAs per SM of a streaming launch (the environment's setting at creation)
  bool has_stream = false;
  wmpc::StreamPlan sp{};
  void* stream_block = nullptr;
  // optional second schedule in the frontier-slot form (fixed iterations only)
  bool has_frontier = false;
  bool frontier_pays = false;  // it fits two CTAs per SM where sp does not
  wmpc::StreamPlan spf{};
  void* stream_block_f = nullptr;
  std::string stream_why;  // why the streaming path is unavailable (diagnostics)
};

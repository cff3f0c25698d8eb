/*
 * CPU restatement (C; callers split the batch across threads) of the reference's batched
 * fixed-iteration OSQP-ADMM over QDLDL, real_t32.
 *
 * TEST INFRASTRUCTURE ONLY (oracle): the CPU baseline timed by bench.py and
 * a cross-check of oracle/osqp_ref.py.  Never linked into the product.
 *
 * Restates, per instance:
 *   - KKT value assembly            warpmpc/jax_osqp/solver.py:764-776
 *   - numeric LDL^T factorization   warpmpc/jax_qdldl/warp_backend.py:41-101
 *   - triangular solve              warpmpc/jax_qdldl/warp_backend.py:176-218
 *   - ADMM iteration                warpmpc/jax_osqp/solver.py:806-820
 *   - scaling, unscaling, residuals warpmpc/jax_osqp/solver.py:842-871
 * with every product and sum rounded separately (build with
 * -ffp-contract=off), in the reference's operation order.
 *
 * Data layout: batch-major (instance b row of width w at b*w), P/A values
 * with batch 1 broadcast.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* real_t: float (parity build) or double (truth build, -DOC_DOUBLE) */
#ifdef OC_DOUBLE
typedef double real_t;
#define OC_FN(name) name##_f64
#define OC_ABS fabs
#define OC_MAX fmax
#else
typedef float real_t;
#define OC_FN(name) name
#define OC_ABS fabsf
#define OC_MAX fmaxf
#endif

typedef struct {
  int n, nnz_a, nnz_l;
  const int32_t *perm_to_orig, *diag_pos, *init_ptr, *init_rows, *init_pos;
  const int32_t *proc_ptr, *proc_cols, *proc_lidx, *proc_offsets, *lp, *li, *p, *pinv;
} oc_pattern;

typedef struct {
  int n, m, nnz_p, nnz_a, nnz_kkt, nnz_pf;
  real_t sigma, alpha;
  const real_t* kkt_base;
  const int32_t* kkt_src; /* -1 base, j P entry, nnz_p+j A entry */
  const real_t *p_scale, *p_diag_sigma, *a_scale;
  const int32_t *a_row_ptr, *a_row_ent, *a_rows, *a_cols, *a_col_ptr;
  const int32_t *pf_row_ptr, *pf_val, *pf_col;
  const real_t *rho, *rho_inv, *q_scale, *scaling_d, *scaling_dinv, *scaling_e, *scaling_einv, *y_scale, *y_unscale;
} oc_osqp;

static void factor_one(const oc_pattern* pat, const real_t* kkt /* original order */, real_t* lx, real_t* d,
                       real_t* dinv, real_t* y) {
  const int n = pat->n;
  for (int i = 0; i < n; ++i) y[i] = (real_t)0;
  for (int k = 0; k < n; ++k) {
    real_t dk = kkt[pat->perm_to_orig[pat->diag_pos[k]]];
    for (int e = pat->init_ptr[k]; e < pat->init_ptr[k + 1]; ++e) {
      const int row = pat->init_rows[e];
      y[row] = y[row] + kkt[pat->perm_to_orig[pat->init_pos[e]]];
    }
    for (int e = pat->proc_ptr[k]; e < pat->proc_ptr[k + 1]; ++e) {
      const int cidx = pat->proc_cols[e];
      const int off = pat->proc_offsets[e];
      const int base = pat->lp[cidx];
      const real_t val = y[cidx];
      for (int q = 0; q < off; ++q) {
        const int r = pat->li[base + q];
        y[r] = y[r] - lx[base + q] * val;
      }
      const real_t lval = val * dinv[cidx];
      lx[pat->proc_lidx[e]] = lval;
      dk = dk - val * lval;
    }
    d[k] = dk;
    dinv[k] = (real_t)1 / dk;
    for (int e = pat->proc_ptr[k]; e < pat->proc_ptr[k + 1]; ++e) y[pat->proc_cols[e]] = (real_t)0;
  }
}

/* in-place solve in the permuted space */
static void solve_permuted(const oc_pattern* pat, const real_t* lx, const real_t* dinv, real_t* x) {
  const int n = pat->n;
  for (int col = 0; col < n; ++col) {
    const real_t val = x[col];
    for (int e = pat->lp[col]; e < pat->lp[col + 1]; ++e) {
      const int r = pat->li[e];
      x[r] = x[r] - lx[e] * val;
    }
  }
  for (int i = 0; i < n; ++i) x[i] = x[i] * dinv[i];
  for (int col = n - 1; col >= 0; --col) {
    real_t corr = (real_t)0;
    for (int e = pat->lp[col]; e < pat->lp[col + 1]; ++e) corr = corr + lx[e] * x[pat->li[e]];
    x[col] = x[col] - corr;
  }
}

static real_t clip_nan(real_t v, real_t lo, real_t hi) {
  real_t t = (v < lo) ? lo : v;
  return (t > hi) ? hi : t;
}

/* Solve instances [b_begin, b_end) of the batch; returns 0 (1 on allocation
 * failure).  Outputs batch-major.  Thread-safe for disjoint ranges. */
int OC_FN(oc_osqp_solve)(const oc_pattern* pat, const oc_osqp* o, int b_begin, int b_end, int max_iter, const real_t* p_values,
                  int p_batch, const real_t* a_values, int a_batch, const real_t* q, const real_t* l, const real_t* u,
                  const real_t* x0, const real_t* z0, const real_t* y0, real_t* x_out, real_t* z_out, real_t* y_out,
                  real_t* prim_out, real_t* dual_out, real_t* obj_out) {
  const int n = o->n, m = o->m, nk = n + m;
  {
    real_t* kkt = (real_t*)malloc(sizeof(real_t) * (size_t)o->nnz_kkt);
    real_t* lx = (real_t*)malloc(sizeof(real_t) * (size_t)(pat->nnz_l > 0 ? pat->nnz_l : 1));
    real_t* d = (real_t*)malloc(sizeof(real_t) * (size_t)nk);
    real_t* dinv = (real_t*)malloc(sizeof(real_t) * (size_t)nk);
    real_t* w = (real_t*)malloc(sizeof(real_t) * (size_t)nk);
    real_t* xs = (real_t*)malloc(sizeof(real_t) * (size_t)n);
    real_t* zs = (real_t*)malloc(sizeof(real_t) * (size_t)m);
    real_t* ys = (real_t*)malloc(sizeof(real_t) * (size_t)m);
    real_t* qs = (real_t*)malloc(sizeof(real_t) * (size_t)n);
    real_t* ls = (real_t*)malloc(sizeof(real_t) * (size_t)m);
    real_t* us = (real_t*)malloc(sizeof(real_t) * (size_t)m);
    const real_t one_minus = (real_t)1 - o->alpha;
    if (!kkt || !lx || !d || !dinv || !w || !xs || !zs || !ys || !qs || !ls || !us) {
      free(kkt); free(lx); free(d); free(dinv); free(w); free(xs); free(zs); free(ys); free(qs); free(ls); free(us);
      return 1;
    }
    for (int b = b_begin; b < b_end; ++b) {
      const real_t* pv = p_values + (size_t)(p_batch > 1 ? b : 0) * o->nnz_p;
      const real_t* av = a_values + (size_t)(a_batch > 1 ? b : 0) * o->nnz_a;
      for (int s = 0; s < o->nnz_kkt; ++s) {
        const int src = o->kkt_src[s];
        if (src < 0) kkt[s] = o->kkt_base[s];
        else if (src < o->nnz_p) kkt[s] = pv[src] * o->p_scale[src] + o->p_diag_sigma[src];
        else kkt[s] = av[src - o->nnz_p] * o->a_scale[src - o->nnz_p];
      }
      factor_one(pat, kkt, lx, d, dinv, w);
      const real_t* qb = q + (size_t)b * n;
      const real_t* lb = l + (size_t)b * m;
      const real_t* ub = u + (size_t)b * m;
      for (int j = 0; j < n; ++j) {
        qs[j] = qb[j] * o->q_scale[j];
        xs[j] = x0 ? x0[(size_t)b * n + j] * o->scaling_dinv[j] : (real_t)0;
      }
      for (int r = 0; r < m; ++r) {
        ls[r] = lb[r] * o->scaling_e[r];
        us[r] = ub[r] * o->scaling_e[r];
        zs[r] = z0 ? z0[(size_t)b * m + r] * o->scaling_e[r] : (real_t)0;
        ys[r] = y0 ? y0[(size_t)b * m + r] * o->y_scale[r] : (real_t)0;
      }
      for (int it = 0; it < max_iter; ++it) {
        for (int i = 0; i < nk; ++i) {
          const int orig = pat->p[i];
          if (orig < n) w[i] = o->sigma * xs[orig] - qs[orig];
          else w[i] = zs[orig - n] - o->rho_inv[orig - n] * ys[orig - n];
        }
        solve_permuted(pat, lx, dinv, w);
        for (int i = 0; i < nk; ++i) {
          const int orig = pat->p[i];
          const real_t sol = w[i];
          if (orig < n) {
            xs[orig] = o->alpha * sol + one_minus * xs[orig];
          } else {
            const int r = orig - n;
            const real_t rinv = o->rho_inv[r];
            const real_t rz = zs[r] - rinv * ys[r];
            const real_t zt = rz + rinv * sol;
            const real_t zr = o->alpha * zt + one_minus * zs[r];
            const real_t zn = clip_nan(zr + rinv * ys[r], ls[r], us[r]);
            ys[r] = ys[r] + o->rho[r] * (zr - zn);
            zs[r] = zn;
          }
        }
      }
      real_t* xb = x_out + (size_t)b * n;
      real_t* zb = z_out + (size_t)b * m;
      real_t* yb = y_out + (size_t)b * m;
      for (int j = 0; j < n; ++j) xb[j] = xs[j] * o->scaling_d[j];
      for (int r = 0; r < m; ++r) {
        zb[r] = zs[r] * o->scaling_einv[r];
        yb[r] = ys[r] * o->y_unscale[r];
      }
      real_t prim = (real_t)0, dual = (real_t)0, quad = (real_t)0, lin = (real_t)0;
      for (int r = 0; r < m; ++r) {
        real_t ax = (real_t)0;
        for (int t = o->a_row_ptr[r]; t < o->a_row_ptr[r + 1]; ++t) {
          const int e = o->a_row_ent[t];
          ax = ax + av[e] * xb[o->a_cols[e]];
        }
        prim = OC_MAX(prim, OC_ABS(ax - zb[r]));
      }
      for (int j = 0; j < n; ++j) {
        real_t px = (real_t)0;
        for (int t = o->pf_row_ptr[j]; t < o->pf_row_ptr[j + 1]; ++t) px = px + pv[o->pf_val[t]] * xb[o->pf_col[t]];
        real_t aty = (real_t)0;
        for (int e = o->a_col_ptr[j]; e < o->a_col_ptr[j + 1]; ++e) aty = aty + av[e] * yb[o->a_rows[e]];
        dual = OC_MAX(dual, OC_ABS(px + qb[j] + aty));
        quad = quad + xb[j] * px;
        lin = lin + qb[j] * xb[j];
      }
      prim_out[b] = prim;
      dual_out[b] = dual;
      obj_out[b] = (real_t)0.5 * quad + lin;
    }
    free(kkt); free(lx); free(d); free(dinv); free(w); free(xs); free(zs); free(ys); free(qs); free(ls); free(us);
  }
  return 0;
}

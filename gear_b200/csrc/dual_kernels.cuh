// Rigorous float64 weak-duality bound of batched LPs on the device: the reference's
// dual_lower_bound / certify_infeasible (complete_verifier/nlp_solver/rigorous_dual.py).
//
// For min c^T z + c0 s.t. G z <= h, l <= z <= u and y >= 0, D(y) = c0 - h^T y +
// sum_j min(r_j l_j, r_j u_j) with r = c + G^T y; the result lb <= D(y) exactly on the given
// floats: the rounding of every sum is enclosed by Higham's gamma_k terms (any summation
// order), so the block-parallel reductions here are as rigorous as the reference's. Where the
// error term is large next to the tolerance, r is recomputed in double-double (Dot2:
// TwoProduct / TwoSum in each column's entry order) and the larger bound is kept.
//
// One CTA per domain: the multipliers in shared memory, one thread per column walking the
// column's entries (CSC order, original order within a column), block reductions in a fixed
// order.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace gear {
namespace dual {

constexpr int DT = 128;                         // threads per CTA
constexpr double U = 1.1102230246251565e-16;    // 2^-53
constexpr double ETA = 4.9406564584124654e-324; // 2^-1074
constexpr double BIG = 2.5822498780869086e+120; // 2^400

__device__ __forceinline__ double gamma_k(double k) { return k * U / (1.0 - k * U); }

__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
  s = a + b;
  const double bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}
__device__ __forceinline__ void two_prod(double a, double b, double& p, double& e) {
  // Dekker / Veltkamp splitting (exact for |a|, |b| < 2^996 without underflow)
  p = a * b;
  double t = 134217729.0 * a;
  const double ah = t - (t - a), al = a - ah;
  t = 134217729.0 * b;
  const double bh = t - (t - b), bl = b - bh;
  e = ((ah * bh - p) + ah * bl + al * bh) + al * bl;
}

struct Lp {
  const int32_t* colptr;   // (n + 1)
  const int32_t* rows;     // (nnz) row of each CSC entry
  const int32_t* perm;     // (nnz) entry index of each CSC position (values are in entry order)
  const double* val;       // (Bv, nnz), Bv = B or 1
  int val_batched;
  const double* c;         // (B, n) or null (zero)
  const double* c0;        // (B) or null
  const double* h;         // (B, m)
  const double* l;         // (B, n)
  const double* u;         // (B, n)
  const double* y;         // (B, m)
  const double* tol;       // (B) or null: max(1e-5, 1e-4 |value|)
  const double* c_err;     // (B, n) or null
  const double* c0_err;    // (B) or null
  double* lb;              // (B)
  double* E;               // (B) or null
  uint8_t* dd;             // (B) or null
  int64_t B;
  int m, n, nnz;
  int infeasibility;       // 1: certify_infeasible's decision rule for the double-double step
};

// fixed-order block sum (warp butterflies, then the warps in order)
__device__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double t = 0;
  for (int i = 0; i < DT / 32; ++i) t += red[i];
  return t;
}
__device__ double block_max(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double t = red[0];
  for (int i = 1; i < DT / 32; ++i) t = fmax(t, red[i]);
  return t;
}

struct Terms {
  double t_sum, t_abs, me_sum, t_nz;
  int ok;
};

// per-column terms of _bound for reduced cost r (float or double-double)
__device__ __forceinline__ void column_terms(double r, double rho, double k, double cerr, double l, double u, bool dd,
                                             double infl, Terms& T) {
  const double kk = k > 0 ? gamma_k(k + 1.0) : 0.0;
  const double eps = (dd ? kk * kk * rho + 2 * U * fabs(r) : kk * rho) + 4 * ETA * (k + 2) + cerr;
  const double es = eps * infl;
  const bool fl = isfinite(l), fu = isfinite(u), both = fl && fu;
  const double l0 = fl ? l : 0.0, u0 = fu ? u : 0.0;
  const bool pos = (r > es) && fl, neg = (r < -es) && fu;
  const bool zero = rho == 0 && k == 0 && cerr == 0;
  T.ok &= (both || zero || pos || neg) ? 1 : 0;
  const double t = both ? fmin(r * l0, r * u0) : (pos ? r * l0 : (neg ? r * u0 : 0.0));
  const double M = both ? fmax(fabs(l0), fabs(u0)) : (pos ? fabs(l0) : (neg ? fabs(u0) : 0.0));
  T.t_sum += t;
  T.t_abs += fabs(t);
  T.me_sum += M * eps;
  T.t_nz += (t != 0) ? 1.0 : 0.0;
}

__global__ void __launch_bounds__(DT) dual_bound_kernel(Lp p) {
  extern __shared__ double ys[];          // m multipliers, clamped at 0
  __shared__ double red[DT / 32];
  const int64_t b = blockIdx.x;
  if (b >= p.B) return;
  const int m = p.m, n = p.n, tid = threadIdx.x;
  const double* vb = p.val + (p.val_batched ? b * p.nnz : 0);
  const double* cb = p.c ? p.c + b * n : nullptr;
  const double* hb = p.h + b * m;
  const double* lb_ = p.l + b * n;
  const double* ub_ = p.u + b * n;
  const double c0 = p.c0 ? p.c0[b] : 0.0;
  const double c0e = p.c0_err ? p.c0_err[b] : 0.0;
  const double infl = 1.0 + gamma_k(2.0 * (m + n) + 16);

  // multipliers, the row terms and the validity of the data
  double hy = 0, hya = 0, ypos = 0, ymax = 0;
  int valid = 1;
  for (int i = tid; i < m; i += DT) {
    double yi = p.y[b * m + i];
    yi = isnan(yi) ? yi : fmax(yi, 0.0);
    ys[i] = yi;
    valid &= isfinite(yi) ? 1 : 0;
    const double t = yi > 0 ? hb[i] * yi : 0.0;
    hy += t;
    hya += fabs(t);
    ypos += yi > 0 ? 1.0 : 0.0;
    ymax = fmax(ymax, yi);
  }
  double cmax = 0;
  for (int j = tid; j < n; j += DT) {
    const double cj = cb ? cb[j] : 0.0;
    valid &= (isfinite(cj) && !isnan(lb_[j]) && !isnan(ub_[j])) ? 1 : 0;
    cmax = fmax(cmax, fabs(cj));
  }
  double vmax = 0;
  for (int e = tid; e < p.nnz; e += DT) vmax = fmax(vmax, fabs(vb[e]));
  valid &= isfinite(c0) ? 1 : 0;
  __syncthreads();
  hy = block_sum(hy, red);
  hya = block_sum(hya, red);
  ypos = block_sum(ypos, red);
  valid = block_sum((double)valid, red) == (double)DT;
  ymax = block_max(ymax, red);
  cmax = block_max(cmax, red);
  vmax = block_max(vmax, red);

  double lbv = -INFINITY, Ev = 0;
  bool used_dd = false;
  for (int pass = 0; pass < 2; ++pass) {
    const bool dd = pass == 1;
    Terms T{0, 0, 0, 0, 1};
    for (int j = tid; j < n; j += DT) {
      const double cj = cb ? cb[j] : 0.0;
      const int e0 = p.colptr[j], e1 = p.colptr[j + 1];
      double acc = 0, rho = 0, k = 0, hi = cj, lo = 0;
      for (int e = e0; e < e1; ++e) {
        const double ya = ys[p.rows[e]];
        const double v = vb[p.perm[e]];
        const bool act = ya != 0 && v != 0;
        const double pr = act ? v * ya : 0.0;
        acc += pr;
        rho += fabs(pr);
        k += act ? 1.0 : 0.0;
        if (dd) {
          const double a = ya != 0 ? v : 0.0;
          double pp, pe, s, se;
          two_prod(a, ya, pp, pe);
          two_sum(hi, pp, s, se);
          hi = s;
          lo = lo + (se + pe);
        }
      }
      const double r = dd ? hi + lo : acc + cj;
      rho = rho + fabs(cj);
      column_terms(r, rho, k, p.c_err ? p.c_err[b * n + j] : 0.0, lb_[j], ub_[j], dd, infl, T);
    }
    const double t_sum = block_sum(T.t_sum, red);
    const double t_abs = block_sum(T.t_abs, red);
    const double me = block_sum(T.me_sum, red);
    const double tnz = block_sum(T.t_nz, red);
    const bool ok = block_sum((double)T.ok, red) == (double)DT;
    const double val = c0 - hy + t_sum;
    const double N = 1.0 + ypos + tnz;
    const double under = (double)(m + n + 3) * ETA;
    double E = gamma_k(N + 2) * (fabs(c0) + hya + t_abs) + me + under + c0e;
    E = E * infl;
    E = E + 4 * U * (fabs(val) + E);
    double lbp = val - E;
    if (!(ok && isfinite(lbp))) lbp = -INFINITY;
    if (!dd) {
      lbv = lbp;
      Ev = E;
      bool need;
      if (p.infeasibility) {
        need = (val + E > 0) && (lbp <= 0) && ypos > 0;
      } else {
        const double t = p.tol ? p.tol[b] : fmax(fabs(val) * 1e-4, 1e-5);
        need = !(E <= t / 10) || !isfinite(lbp);
      }
      const bool flag = valid && need && p.nnz > 0;
      const bool safe = vmax < BIG && ymax < BIG && cmax < BIG;
      if (!(flag && safe)) break;
      used_dd = true;
    } else if (lbp > lbv) {
      lbv = lbp;
      Ev = E;
    }
  }
  if (tid == 0) {
    p.lb[b] = lbv;
    if (p.E) p.E[b] = Ev;
    if (p.dd) p.dd[b] = used_dd ? 1 : 0;
  }
}

}  // namespace dual
}  // namespace gear

// Constrained concretisation on the device: lower bounds of objective rows c (B, H, X) over
// boxes intersected with linear rows A (B, K, X) x + b (B, K) <= 0, by the sequential dual
// sweep of the reference's constraints_solving (auto_LiRPA/concretize_func.py:415-850) and
// its preprocessing sort_out_constr_batches / drop_redundant_constraints (:312, :269).
//
//   concretize_rows_kernel   one warp per row (b, k): infeasibility / cover tests, the
//                            centred offset d rounded down, the worst-case value over the box
//                            (redundant rows never bind)
//   concretize_boxes_kernel  one thread per box: batch-wide "all covered" and the largest
//                            count of binding rows over the active boxes (the sweep length
//                            in the rounding term)
//   concretize_sweep_kernel  one warp per (box, objective row): the sweep. Per row: the
//                            breakpoints -c_i / a_i of the one-row Lagrangian with weights
//                            |a_i eps_i| are compacted and bitonic-sorted in shared memory;
//                            a warp scan of the weights finds the first breakpoint where the
//                            slope turns non-positive (the multiplier beta); c += beta a.
//                            The objective row, its magnitude and the sort buffers live in
//                            shared memory for the whole sweep.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace gear {
namespace cc {

constexpr double EPS = 2.220446049250313e-16;

__device__ __forceinline__ double fabs_fin(double v) { return isfinite(v) ? fabs(v) : 0.0; }
__device__ __forceinline__ double rerr(double mag, double n) { return mag * ((n + 16.0) * EPS * 4.0); }
__device__ __forceinline__ double widen_b(double bound, double err, double sign) {
  double out = isfinite(bound) ? bound + sign * err : bound;
  return (isinf(err) && err > 0) ? sign * INFINITY : out;
}
__device__ __forceinline__ double wsum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ unsigned long long qkey(double v) {
  // ascending total order of doubles, NaN last
  if (isnan(v)) return ~0ull;
  unsigned long long u = __double_as_longlong(v);
  return (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
}
__device__ __forceinline__ double qval(unsigned long long k) {
  unsigned long long u = (k & 0x8000000000000000ull) ? (k & 0x7fffffffffffffffull) : ~k;
  return __longlong_as_double((long long)u);
}

struct Work {
  const double* xL;   // (B, X)
  const double* xU;
  const double* obj;  // (B, H, X)
  const double* A;    // (B, K, X)
  const double* b;    // (B, K)
  double* d;          // (B, K) centred offsets, rounded down
  double* score;      // (B, K) worst-case value of a binding row, -inf for a redundant one
  int* infeasible;    // (B)
  int* uncovered;     // (B)
  int* nkeep;         // (B) binding rows per box
  int* glob;          // [0]: some box is not covered, [1]: max nkeep over uncovered boxes
  double* lb;         // (B, H)
  uint8_t* infeasible_out;   // (B) or null
  int64_t B;
  int X, H, K, max_rows;
};

// ------------------------------------------------------------------ per row
__global__ void concretize_rows_kernel(Work w) {
  const int lane = threadIdx.x & 31;
  const int64_t row = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (row >= w.B * w.K) return;
  const int64_t b = row / w.K;
  const int X = w.X;
  const double* a = w.A + row * X;
  const double* xl = w.xL + b * X;
  const double* xu = w.xU + b * X;
  double ax0 = 0, aeps = 0, mag = 0, magd = 0;
  int fin = 1;
  for (int i = lane; i < X; i += 32) {
    const double ai = a[i], l = xl[i], u = xu[i];
    const double x0 = (l + u) / 2, e = (u - l) / 2;
    fin &= isfinite(ai) ? 1 : 0;
    ax0 += ai * x0;
    aeps += fabs(ai) * e;
    const double lo_ = x0 - e, hi_ = x0 + e;
    mag += fabs_fin(ai) * fabs_fin(fmax(fabs(lo_), fabs(hi_)));
    magd += fabs_fin(ai) * fabs_fin(fabs(x0));
  }
  ax0 = wsum(ax0);
  aeps = wsum(aeps);
  mag = wsum(mag);
  magd = wsum(magd);
  fin = __all_sync(0xffffffffu, fin);
  if (lane != 0) return;
  const double bk = w.b[row];
  // _sort_out_constraints on the rows with non-finite entries replaced by 0 x - 1 <= 0
  double lo_v, hi_v;
  if (fin && isfinite(bk)) {
    const double t = ax0 + bk, err = rerr(mag + fabs_fin(bk), X);
    lo_v = widen_b(t - aeps, err, -1.0);
    hi_v = widen_b(t + aeps, err, 1.0);
  } else {
    const double err = rerr(1.0, X);
    lo_v = -1.0 - err;
    hi_v = -1.0 + err;
  }
  if (lo_v > 0) atomicOr(w.infeasible + b, 1);
  if (!(hi_v <= 0)) atomicOr(w.uncovered + b, 1);
  // centred offset, rounded down; a row that is not finite after it is inert (0 x - 1 <= 0)
  double d = widen_b(ax0 + bk, rerr(magd + fabs_fin(bk), X), -1.0);
  const bool ok = fin && isfinite(d);
  if (!ok) d = -1.0;
  const double max_val = d + (ok ? aeps : 0.0);
  const bool redundant = max_val <= 0;
  w.d[row] = d;
  w.score[row] = redundant ? -INFINITY : (isnan(max_val) ? INFINITY : max_val);
  if (!redundant) atomicAdd(w.nkeep + b, 1);
}

// ------------------------------------------------------------------ per box
__global__ void concretize_boxes_kernel(Work w) {
  const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= w.B) return;
  if (w.uncovered[b]) {
    atomicOr(w.glob, 1);
    atomicMax(w.glob + 1, w.nkeep[b]);
  }
}

// ------------------------------------------------------------------ the sweep
// shared memory per warp: c, cmag, wgt (X each), keys (XP), kidx (XP), rows (K)
__host__ __device__ inline int sweep_xp(int X) {
  int xp = 32;
  while (xp < X) xp <<= 1;
  return xp;
}
__host__ __device__ inline size_t sweep_smem_per_warp(int X, int K) {
  const int xp = sweep_xp(X);
  const size_t bytes = (size_t)3 * X * sizeof(double) + (size_t)xp * (sizeof(unsigned long long) + sizeof(int)) +
                       (size_t)K * sizeof(int);
  return (bytes + 15) / 16 * 16;   // keeps every warp's doubles 16-byte aligned
}

__global__ void concretize_sweep_kernel(Work w) {
  extern __shared__ unsigned char smraw[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int X = w.X, K = w.K, xp = sweep_xp(X);
  const size_t per = sweep_smem_per_warp(X, K);
  unsigned char* base = smraw + per * wid;
  double* c = reinterpret_cast<double*>(base);
  double* cmag = c + X;
  double* wgt = cmag + X;
  unsigned long long* keys = reinterpret_cast<unsigned long long*>(wgt + X);
  int* kidx = reinterpret_cast<int*>(keys + xp);
  int* rows = kidx + xp;

  const int64_t item = (int64_t)blockIdx.x * (blockDim.x >> 5) + wid;
  if (item >= w.B * w.H) return;
  const int64_t b = item / w.H;
  const double* xl = w.xL + b * X;
  const double* xu = w.xU + b * X;
  const double* c0 = w.obj + item * X;

  // box bound and the objective's own rounding (concretize_func.py:596-619)
  double base_t = 0, eps_t = 0, omag = 0;
  for (int i = lane; i < X; i += 32) {
    const double l = xl[i], u = xu[i], ci = c0[i];
    base_t += ci * ((u + l) / 2.0);
    eps_t += fabs(ci) * ((u - l) / 2.0);
    omag += fabs_fin(ci) * fabs_fin(fmax(fabs(l), fabs(u)));
    c[i] = ci;
    cmag[i] = fabs_fin(ci);
  }
  base_t = wsum(base_t);
  eps_t = wsum(eps_t);
  omag = wsum(omag);
  const double obj_err = rerr(omag, X);
  double naive = widen_b(base_t - eps_t, obj_err, -1.0);
  if (!isfinite(naive)) naive = -INFINITY;
  const bool infeasible = w.infeasible[b] != 0;
  if (lane == 0 && w.infeasible_out && item % w.H == 0) w.infeasible_out[b] = infeasible ? 1 : 0;
  if (!w.glob[0] || !w.uncovered[b]) {
    // every box covered (the reference drops the rows), or this box covered by every row
    if (lane == 0) w.lb[item] = naive;
    return;
  }
  const int gk = w.glob[1] > 1 ? w.glob[1] : 1;
  const bool capped = w.max_rows > 0 && gk > w.max_rows;
  const int Keff = capped ? w.max_rows : gk;

  // this box's rows in sweep order: binding rows in their original order; with the cap,
  // the max_rows largest worst-case values (ties: lower index)
  const double* sc = w.score + b * K;
  int nrows = 0;
  for (int k0 = 0; k0 < K; k0 += 32) {
    const int k = k0 + lane;
    bool keep = false;
    if (k < K && sc[k] > -INFINITY) {
      keep = true;
      if (capped && w.nkeep[b] > w.max_rows) {
        int rank = 0;
        const double s = sc[k];
        for (int j = 0; j < K; ++j) rank += (sc[j] > s || (sc[j] == s && j < k)) ? 1 : 0;
        keep = rank < w.max_rows;
      }
    }
    const unsigned m = __ballot_sync(0xffffffffu, keep);
    if (keep) rows[nrows + __popc(m & ((1u << lane) - 1))] = k;
    nrows += __popc(m);
  }
  __syncwarp();

  double dual = 0, dmag = 0;
  for (int r = 0; r < nrows; ++r) {
    const int k = rows[r];
    const double* a = w.A + (b * K + k) * X;
    const double dk = w.d[b * K + k];
    // breakpoints with positive weight, compacted
    int n = 0;
    for (int i0 = 0; i0 < X; i0 += 32) {
      const int i = i0 + lane;
      double q = 0, wt = 0;
      if (i < X) {
        const double ai = a[i], e = (xu[i] - xl[i]) / 2.0;
        q = -c[i] / ai;
        wt = fabs(ai * e);
        wgt[i] = wt;
      }
      const bool use = i < X && wt > 0;
      const unsigned m = __ballot_sync(0xffffffffu, use);
      if (use) {
        const int p = n + __popc(m & ((1u << lane) - 1));
        keys[p] = qkey(q);
        kidx[p] = i;
      }
      n += __popc(m);
    }
    int np2 = 1;
    while (np2 < n) np2 <<= 1;
    for (int p = n + lane; p < np2; p += 32) { keys[p] = ~0ull; kidx[p] = 0x7fffffff; }
    __syncwarp();
    // bitonic sort ascending by (key, index)
    for (int kk = 2; kk <= np2; kk <<= 1) {
      for (int j = kk >> 1; j > 0; j >>= 1) {
        for (int t = lane; t < (np2 >> 1); t += 32) {
          const int i = (t / j) * 2 * j + (t % j), pi = i + j;
          const bool up = (i & kk) == 0;
          const unsigned long long ka = keys[i], kb = keys[pi];
          const int ia = kidx[i], ib = kidx[pi];
          const bool gt = ka > kb || (ka == kb && ia > ib);
          if (gt == up) { keys[i] = kb; keys[pi] = ka; kidx[i] = ib; kidx[pi] = ia; }
        }
        __syncwarp();
      }
    }
    // prefix sums of the sorted weights: contiguous chunks per lane, exclusive warp scan of
    // the chunk totals; the slope is non-positive from the first j with 2 P_j - W - d >= 0
    const int ch = (n + 31) / 32;
    const int s0 = lane * ch, s1 = min(n, s0 + ch);
    double tot = 0;
    for (int p = s0; p < s1; ++p) tot += wgt[kidx[p]];
    double incl = tot;
    for (int o = 1; o < 32; o <<= 1) {
      const double v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    const double W = __shfl_sync(0xffffffffu, incl, 31);
    double P = incl - tot;
    int neg = 0;
    if (lane == 0) neg += ((0.0 - W) + 0.0 - dk) < 0 ? 1 : 0;      // j = 0 (before every breakpoint)
    for (int p = s0; p < s1; ++p) {
      P += wgt[kidx[p]];
      neg += ((P - W) + P - dk) < 0 ? 1 : 0;
    }
    for (int o = 16; o > 0; o >>= 1) neg += __shfl_xor_sync(0xffffffffu, neg, o);
    double beta;
    if (neg == 0) beta = 0.0;
    else if (neg > n) beta = INFINITY;
    else {
      const double q = qval(keys[neg - 1]);
      beta = isnan(q) ? q : fmax(q, 0.0);
    }
    // fold the row in
    for (int i = lane; i < X; i += 32) {
      const double upd = beta * a[i];
      c[i] = c[i] + upd;
      cmag[i] = cmag[i] + fabs_fin(upd);
    }
    dual += beta * dk;
    dmag = dmag + fabs_fin(beta * dk);
    __syncwarp();
  }
  double et = 0, cm = 0;
  for (int i = lane; i < X; i += 32) {
    const double e = (xu[i] - xl[i]) / 2.0;
    et += fabs(c[i]) * e;
    cm += cmag[i] * fabs_fin(e);
  }
  et = wsum(et);
  cm = wsum(cm);
  if (lane != 0) return;
  dual -= et;
  dmag = dmag + fabs_fin(et) + cm;
  double val = base_t + dual;
  const double err = obj_err + rerr(dmag + fabs_fin(base_t), (double)X + Keff);
  val = widen_b(val, err, -1.0);
  if (!isfinite(val)) val = naive;
  val = fmax(val, naive);
  w.lb[item] = infeasible ? INFINITY : val;
}

}  // namespace cc
}  // namespace gear

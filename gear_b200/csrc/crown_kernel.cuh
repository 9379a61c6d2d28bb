// CROWN bound propagation over a batch of boxes: one persistent megakernel.
// (Included by gear_capi.cu, the single translation unit of libgear_b200.so.)
//
// Each CTA takes boxes b = blockIdx.x, blockIdx.x + gridDim.x, ... and runs the whole
// compiled schedule for that box: plain IBP of every node, relaxation planes, every
// intermediate CROWN pass (lower and upper, C = I over the node width, then
// compare-with-IBP), the final pass and its box concretisation. The A coefficients of a
// pass live in shared memory as the statically-sparse entry lists the host compiler built
// (gear_b200/program.py); intervals, planes and fold vectors live in a per-CTA scratch slot
// in global memory (reused box after box, so it stays in L2).
//
// Reference semantics followed (paths relative to solver/auto_LiRPA):
//   relaxations  operators/bivariate.py:38-247 (McCormick, coefficient-aware pick),
//                operators/activations.py:186-210 (Sqr), operators/convex_concave.py:64-92
//                (Log), :569-626 (Exp), operators/s_shaped.py:325-550 and
//                operators/trigonometric.py:27-527 (Sin/Cos);
//   backward     backward_bound.py:880-1206, operators/clampmult.py:31-77;
//   IBP          interval_bound.py:156-254 and the operators' interval_propagate;
//   concretise   concretize_bounds.py:160-321, concretize_func.py:553-569,
//                fp_enclosure.py:34-98.
// Compiled with -fmad=false: the elementwise formulas round like the reference's eager
// float64 arithmetic (no contraction), which keeps the relaxation choices stable. The dot
// products of the GEMV steps, the fold vectors and the box concretisation accumulate with explicit
// fused multiply-adds (as a BLAS product does); their rounding charges bound any such order.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "gear_program.h"

namespace gear {

constexpr double PI = 3.141592653589793;
constexpr double TWO_PI = 2 * PI;
constexpr double HALF_PI = PI / 2;
constexpr double THREE_HALF_PI = 3 * PI / 2;
constexpr double EPS = 2.220446049250313e-16;   // float64 machine epsilon
constexpr double UNIT = EPS / 2;
constexpr double EPSILON = 1e-12;               // operators/base.py:32
constexpr double TIE_TOL = 1e-12;               // McCormick tie tolerance of the "exact" tie rule
constexpr double STEP_PRE = 0.01;
// The box-per-CTA kernel is instantiated for 64, 128 and 256 threads per CTA (template
// parameter NT of every function below that splits work over the CTA); the program picks one.
#ifndef GEAR_CTA_MINB
#define GEAR_CTA_MINB 768      // resident threads per SM the register budget is sized for
#endif

// sin/cos table offsets (gear_b200/tables.py SIN_TABLE_ORDER)
constexpr int T_DL = 0, T_DU = SIN_N_PRE, T_XLLD = 2 * SIN_N_PRE, T_XLLC = T_XLLD + SIN_N_TB,
              T_XLUD = T_XLLC + SIN_N_TB, T_XLUC = T_XLUD + SIN_N_TB, T_XULD = T_XLUC + SIN_N_TB,
              T_XULC = T_XULD + SIN_N_TB, T_XUUD = T_XULC + SIN_N_TB, T_XUUC = T_XUUD + SIN_N_TB;

struct Work {
  const double* xL;
  const double* xU;
  const double* C;       // (B, S, w_t) or null (identity)
  double* lb;            // (B, S)
  double* lA;            // (B, S, n) or null
  double* lbias;         // (B, S) or null
  double* lb_ibp;        // (B, S) or null: the rows' IBP bound; lb is then max(CROWN, IBP)
  double* scratch;       // per-slot scratch
  int64_t slot_doubles;
  int64_t B;
  int* status;
  // fold vectors computed before the launch by the tensor-core fold (fold_tc.cuh), (B, H_FOLDW),
  // or null; fold_fail points to its status flag (nonzero: a bounded wait expired, and every box
  // folds on the CUDA cores instead)
  const double* fold_ext;
  const int* fold_fail;
  // the final pass's product through a dense node on the input on the tensor cores (OF_SPLIT op,
  // tensor-core programs): the kernel writes that op's A rows densely, (B * S, split_k) doubles,
  // and per row the pass's bias sum, charge sum and interval fallback, (B * S, 3), and per box
  // its open flag; the GEMM and the concretisation run after it (split_tail_kernel). Null: the
  // kernel takes the product itself.
  double* split_v = nullptr;
  double* split_rows = nullptr;
  int* split_open = nullptr;
  int split_k = 0;
  // concretisation over the box intersected with cut rows (the plain form's launches only):
  // phase bit 4 of a pass writes its input A rows densely, (B, cut_h, n) with cut_h = sides * S
  // (the upper side negated: its bound is minus the lower bound of -A); the constrained sweep
  // turns them into lower bounds cut_v (B, cut_h), which the concretisation phase then takes in
  // place of the box terms A x0 -/+ |A| eps and their rounding
  double* cut_obj = nullptr;
  const double* cut_v = nullptr;
  int cut_h = 0;
};

// ------------------------------------------------------------------ small helpers
__device__ __forceinline__ double rounding_error(double mag, double n) {
  return mag * ((n + 16.0) * EPS * 4.0);
}
__device__ __forceinline__ double widen(double bound, double err, double sign) {
  double out = isfinite(bound) ? bound + sign * err : bound;
  return (isinf(err) && err > 0) ? sign * INFINITY : out;
}
__device__ __forceinline__ double finite_abs(double v) { return isfinite(v) ? fabs(v) : 0.0; }
// whether tot = fl(old + add) rounded (TwoSum's error is nonzero) or is not finite: on an
// unbounded entry only such a merge costs (_merge_charge, backward_bound.py:740-752)
__device__ __forceinline__ bool merge_rounded(double old, double add, double tot) {
  const double bv = tot - old;
  const double e = (old - (tot - bv)) + (add - bv);
  return !isfinite(tot) || e != 0.0;
}
__device__ __forceinline__ double gamma_k(double k) { return (k + 1.0) * UNIT * (1.0 + 1e-6); }
// NaN-propagating min / max (torch.minimum / np.minimum semantics)
__device__ __forceinline__ double pmax(double a, double b) { return (isnan(a) || a > b) ? a : (isnan(b) ? b : (a > b ? a : b)); }
__device__ __forceinline__ double pmin(double a, double b) { return (isnan(a) || a < b) ? a : (isnan(b) ? b : (a < b ? a : b)); }
__device__ __forceinline__ double nan_lo(double v) { return isnan(v) ? -INFINITY : v; }
__device__ __forceinline__ double nan_hi(double v) { return isnan(v) ? INFINITY : v; }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ int warp_or(int v) { return __any_sync(0xffffffffu, v); }

// ------------------------------------------------------------------ relaxations
__device__ void relax_sqr(double l, double u, double* p) {
  double uk = l + u;
  double ub = -l * uk + l * l;
  double mid = fmax(l, 0.0) - fmax(-u, 0.0);
  double lk = 2 * mid;
  double lb = -mid * lk + mid * mid;
  p[0] = lk; p[1] = lb; p[2] = uk; p[3] = ub;
}

// _stop_undefined_interval (backward_bound.py:249-292) for one element whose relaxation is
// undefined (a non-finite input interval, log of an interval reaching 0): a coefficient that
// selects an undefined side takes the node's own interval [lo_v, hi_v] as a constant plane (a
// non-finite constant still discards the row). The square is convex with a tangent below
// (require_finite_relaxation_bounds(convex_tangent_lower=True), operators/base.py:318-340): only
// its upper side is undefined, its lower tangent is built on the substitute interval (the finite
// endpoint, or 0 -/+ 1 where unbounded), unless the node's interval lies above the hull's lower
// end, where the lower side stops too (backward_bound.py:384-392).
__device__ __forceinline__ void undefined_stop(int kind, double l, double u, double lo_v, double hi_v, double* p) {
  bool stop_lower = true;
  if (kind == NK_SQR) {
    const bool fl = isfinite(l), fu = isfinite(u);
    const double lf = fl ? l : 0.0, uf = fu ? u : 0.0;
    double q[4];
    relax_sqr(fl ? l : fmin(uf, 0.0) - 1.0, fu ? u : fmax(lf, 0.0) + 1.0, q);
    const double hull = u < 0 ? u * u : (l > 0 ? l * l : 0.0);
    stop_lower = lo_v > hull;
    p[0] = q[0];
    p[1] = q[1];
  }
  if (stop_lower) {
    p[0] = 0.0;
    p[1] = lo_v;
  }
  p[2] = 0.0;
  p[3] = hi_v;
}

__device__ void relax_exp(double l, double u, double* p) {
  double du = u - l;
  double neg_expm1 = -expm1(l - u);
  double m_par = u + log(fmax(neg_expm1, EPSILON)) - log(fmax(du, EPSILON));
  double m_mid = (l + u) / 2;
  double m = du > 1e-6 ? m_par : m_mid;
  m = fmin(fmax(m, l), u);
  double exp_l = exp(l), exp_m = exp(m), exp_u = exp(u);
  double lower_k = isfinite(exp_m) ? exp_m : 0.0;
  double lower_x0 = isfinite(m) ? m : 0.0;
  double lower_b = -lower_x0 * lower_k + lower_k;
  bool lsafe = isfinite(lower_k) && isfinite(lower_b);
  p[0] = lsafe ? lower_k : 0.0;
  p[1] = lsafe ? lower_b : 0.0;
  double d = u - l;
  double k;
  if (d < 1) k = exp_l * (d > 0 ? expm1(fmin(d, 1.0)) / fmax(d, 1e-300) : 1.0);
  else k = (exp_u - exp_l) / fmax(d, 1.0);
  double upper_b = -l * k + exp_l;
  bool usafe = isfinite(k) && isfinite(upper_b);
  p[2] = usafe ? k : 0.0;
  p[3] = usafe ? upper_b : INFINITY;
}

__device__ void relax_log(double l, double u, double* p) {
  double rl = log(l), ru = log(u);
  double du = u - l;
  double ku = (ru - rl) / fmax(du, EPSILON);
  p[0] = ku;
  p[1] = -l * ku + rl;
  double dlog = fmax(ru - rl, EPSILON);
  double m_par = du / dlog;
  double m_mid = (l + u) / 2;
  double m = du > 1e-6 ? m_par : m_mid;
  m = fmin(fmax(m, l), u);
  double k = 1.0 / m;
  p[2] = k;
  p[3] = -m * k + log(m);
}

struct SinT {
  const double* T;
};

__device__ __forceinline__ long trunc_l(double v) { return (long)v; }

__device__ void sin_gen_d(const double* T, double lower, double upper, double* dl, double* du) {
  const double sp = STEP_PRE;
  double k = floor(upper / TWO_PI);
  double uc = upper - k * TWO_PI;
  double c1 = (uc >= 0 && uc <= HALF_PI) ? 1.0 : 0.0;
  double ucn = fmin(fmax(uc, 0.0), HALF_PI);
  long idx = max(0L, trunc_l(ucn / sp)) + 1;
  double d_lower = (T[T_DL + idx] + k * 2 * PI) * c1;
  double c2 = (uc >= PI && uc <= THREE_HALF_PI) ? 1.0 : 0.0;
  ucn = fmin(fmax(uc, PI), THREE_HALF_PI);
  idx = max(0L, trunc_l((PI - ucn) / -sp)) + 1;
  double d_upper = (PI - T[T_DU + idx] + k * 2 * PI) * c2;
  k = floor(lower / TWO_PI);
  double lc = lower - k * TWO_PI;
  double c3 = (lc >= THREE_HALF_PI && lc <= 2 * PI) ? 1.0 : 0.0;
  double lcn = fmin(fmax(lc, THREE_HALF_PI), 2 * PI);
  idx = max(0L, trunc_l((lcn - 2 * PI) / -sp)) + 1;
  d_upper = d_upper + (T[T_DU + idx] + (k + 1) * 2 * PI) * c3;
  double c4 = (lc >= HALF_PI && lc <= PI) ? 1.0 : 0.0;
  lcn = fmin(fmax(lc, HALF_PI), 3 * PI);
  idx = max(0L, trunc_l((PI - lcn) / sp)) + 1;
  d_lower = d_lower + (PI - T[T_DL + idx] + k * 2 * PI) * c4;
  *dl = d_lower;
  *du = d_upper;
}

__device__ double sin_pick(double mid, double lower, double upper, double lb_cyc, double ub_cyc,
                           double tl, double tr, double cl, double cr, double base) {
  double unf_l = tl + cl + lb_cyc;
  double l_ends = base + cl + lb_cyc;
  double unf_r = tr + cr + ub_cyc;
  double r_ends = base + cr + ub_cyc;
  bool leftmost = (mid < unf_l) && (unf_l <= upper);
  bool left_range = (mid >= unf_l) && (mid < l_ends);
  bool inbetween = (mid >= l_ends) && (mid < r_ends);
  bool rightmost = (mid >= unf_r) && (unf_r >= lower);
  bool right_range = (!left_range) && ((mid >= r_ends) && (mid < unf_r));
  double tp = (leftmost ? 1.0 : 0.0) * tl + (left_range ? 1.0 : 0.0) * (mid - cl - lb_cyc) +
              (inbetween ? 1.0 : 0.0) * base + (rightmost ? 1.0 : 0.0) * tr +
              (right_range ? 1.0 : 0.0) * (mid - cr - ub_cyc);
  bool any = leftmost || left_range || inbetween || rightmost || right_range;
  return any ? tp : tl;
}

__device__ void sin_bound_tb(const double* T, double lb, double ub, double* out) {
  double lower = lb, upper = ub;
  const double step = 2 * PI / (SIN_N_TB - 1);
  double lb_cyc = floor(lb / (2 * PI)) * (2 * PI);
  double lbm = fmin(fmax(lb - lb_cyc, 0.0), 2 * PI);
  double ub_cyc = floor(ub / (2 * PI)) * (2 * PI);
  double ubm = fmin(fmax(ub - ub_cyc, 0.0), 2 * PI);
  long il = trunc_l(lbm / step);
  long iu = min(trunc_l(ceil(ubm / step)), (long)(SIN_N_TB - 1));
  double tll = T[T_XLLD + il], tlu = T[T_XLUD + il], trl = T[T_XULD + iu], tru = T[T_XUUD + iu];
  double cll = T[T_XLLC + il], clu = T[T_XLUC + il], crl = T[T_XULC + iu], cru = T[T_XUUC + iu];
  double mid = (lower + upper) / 2;
  double tp_l = sin_pick(mid, lower, upper, lb_cyc, ub_cyc, tll, trl, cll, crl, 1.5 * PI);
  double tp_u = sin_pick(mid, lower, upper, lb_cyc, ub_cyc, tlu, tru, clu, cru, 2.5 * PI);
  double d_l = cos(tp_l);
  double b_l = sin(tp_l) - d_l * (tp_l + (tp_l <= 1.5 * PI ? cll + lb_cyc : crl + ub_cyc));
  double d_u = cos(tp_u);
  double b_u = sin(tp_u) - d_u * (tp_u + (tp_u <= 2.5 * PI ? clu + lb_cyc : cru + ub_cyc));
  out[0] = d_l; out[1] = b_l; out[2] = d_u; out[3] = b_u;
}

__device__ __forceinline__ double sin_n_crossing(double start, double end, double s) {
  double cycles = floor((end - start) / (2 * PI));
  double dist = floor((s - start) / (2 * PI));
  double real_s = s - dist * 2 * PI;
  double real_end = end - cycles * 2 * PI;
  return (real_s >= start ? 1.0 : 0.0) * (real_s <= real_end ? 1.0 : 0.0) + cycles;
}

__device__ void sin_branch(const double* T, double lb, double ub, double* out) {
  ub = fmax(ub, lb + 1e-8);
  double sub = sin(ub), slb = sin(lb);
  double mid = (sub + slb) / 2.;
  double smid = sin((ub + lb) / 2);
  double gap = smid - mid;
  double slope = (sub - slb) / fmax(ub - lb, 1e-10);
  double bias = slb - slope * lb;
  double c = slope;
  double cr1 = (c == -1 ? -PI / 2 : (c == 1 ? PI / 2 : asin(c))) - 0.5 * PI;
  double cr2 = PI - cr1 - 2 * (0.5 * PI);
  double crossings = sin_n_crossing(lb, ub, cr1) + sin_n_crossing(lb, ub, cr2);
  bool use_line = crossings == 1;
  double ul = (gap < 0 && use_line) ? 1.0 : 0.0;
  double ll = (gap >= 0 && use_line) ? 1.0 : 0.0;
  double tb[4];
  sin_bound_tb(T, lb, ub, tb);
  out[0] = ll * slope + (1 - ll) * tb[0];
  out[1] = ll * bias + (1 - ll) * tb[1];
  out[2] = ul * slope + (1 - ul) * tb[2];
  out[3] = ul * bias + (1 - ul) * tb[3];
}

__device__ void relax_sin(const double* T, double l, double u, double* p) {
  double twopi = 2 * PI;
  double lbc = l - floor(l / twopi) * twopi;
  double ubc = u - floor(u / twopi) * twopi;
  bool ml1 = lbc >= 0 && lbc < PI / 2, ml2 = lbc >= PI / 2 && lbc < PI, ml3 = lbc >= PI && lbc < 3 * PI / 2,
       ml4 = lbc >= 3 * PI / 2 && lbc < 2 * PI;
  bool mu1 = ubc >= 0 && ubc < PI / 2, mu2 = ubc >= PI / 2 && ubc < PI, mu3 = ubc >= PI && ubc < 3 * PI / 2,
       mu4 = ubc >= 3 * PI / 2 && ubc < 2 * PI;
  bool sig = (u - l <= PI) && (((ml2 || ml3) && (mu2 || mu3)) || ((ml1 || ml4) && (mu1 || mu4)));
  bool mneg = (ml3 || ml4) && ((mu3 || mu4) && sig);
  bool mpos = (ml1 || ml2) && ((mu1 || mu2) && sig);
  bool mboth = sig != (mneg || mpos);
  bool cc = (-sin(l)) >= 0;
  double lw = 0, lb = 0, uw = 0, ub = 0;
#define ADD_LOWER(mask, k, x0, y0) if (mask) { lw = (k); lb = -(x0) * (k) + (y0); }
#define ADD_UPPER(mask, k, x0, y0) if (mask) { uw = (k); ub = -(x0) * (k) + (y0); }
  double y_l = sin(l), y_u = sin(u);
  double width = u - l;
  double k_direct = (y_u - y_l) / fmax(width, 1e-8);
  if (width < 1e-8) k_direct = cos(l);
  ADD_UPPER(mneg, k_direct, l, y_l);
  ADD_LOWER(mpos, k_direct, l, y_l);
  double d_lower, d_upper;
  sin_gen_d(T, l, u, &d_lower, &d_upper);
  bool mdl = (cc ? (k_direct < cos(l)) : (k_direct > cos(u))) && mboth;
  bool mdu = (cc ? (k_direct < cos(u)) : (k_direct > cos(l))) && mboth;
  double m = (l + u) / 2;
  double y_m = sin(m), k_m = cos(m);
  ADD_LOWER(mneg, k_m, m, y_m);
  ADD_UPPER(mpos, k_m, m, y_m);
  ADD_LOWER(mdl, k_direct, l, y_l);
  ADD_LOWER(mboth != mdl, cos(d_lower), d_lower, sin(d_lower));
  ADD_UPPER(mdu, k_direct, l, y_l);
  ADD_UPPER(mboth != mdu, cos(d_upper), d_upper, sin(d_upper));
  ADD_LOWER(sig && (y_l < y_u) && (d_lower >= m), k_m, m, y_m);
  ADD_UPPER(sig && (y_l < y_u) && (d_upper < m), k_m, m, y_m);
  ADD_LOWER(sig && (y_l >= y_u) && (d_lower < m), k_m, m, y_m);
  ADD_UPPER(sig && (y_l >= y_u) && (d_upper >= m), k_m, m, y_m);
#undef ADD_LOWER
#undef ADD_UPPER
  if (!sig) {
    double br[4];
    sin_branch(T, l, u, br);
    lw = br[0]; lb = br[1]; uw = br[2]; ub = br[3];
  }
  double ro = 8 * EPS * (1 + fmax(fabs(l), fabs(u)));
  p[0] = lw; p[1] = lb - ro; p[2] = uw; p[3] = ub + ro;
}

__device__ void relax_cos(const double* T, double l, double u, double* p) {
  const double hp = 0.5 * PI;
  relax_sin(T, l + hp, u + hp, p);
  p[1] = p[1] + p[0] * hp;
  p[3] = p[3] + p[2] * hp;
}

// Box minimum (maximum) of the plane a x + b y + c, rounded op by op in the reference's order
// (BoundMul._affine_min_box: a * x_min + b * y_min + c, operators/bivariate.py:206-217): the
// plane choice compares two such values, so no product may be contracted into an FMA.
__device__ __forceinline__ double plane_min(double a, double b, double c, double xl, double xu, double yl,
                                            double yu) {
  return __dadd_rn(__dadd_rn(__dmul_rn(a, a >= 0 ? xl : xu), __dmul_rn(b, b >= 0 ? yl : yu)), c);
}
__device__ __forceinline__ double plane_max(double a, double b, double c, double xl, double xu, double yl,
                                            double yu) {
  return __dadd_rn(__dadd_rn(__dmul_rn(a, a >= 0 ? xu : xl), __dmul_rn(b, b >= 0 ? yu : yl)), c);
}

// McCormick planes with the coefficient-aware pick (BoundMul._compute_coeff_aware_r,
// operators/bivariate.py:219-250, and interpolated_relaxation :66-75). exact_ties = 0 is the
// reference's float comparison min_p1l >= min_p2l (max_p1u <= max_p2u); exact_ties = 1 counts a
// relative difference below TIE_TOL as a tie and picks plane 1, the exact-arithmetic outcome of
// that comparison (the planes of a tie have the same box minimum, so the choice is then
// independent of the last bits of the intermediate bounds).
__device__ void relax_mul(double xl, double xu, double yl, double yu, double* p, int exact_ties) {
  const double m1 = plane_min(yl, xl, __dmul_rn(-xl, yl), xl, xu, yl, yu);
  const double m2 = plane_min(yu, xu, __dmul_rn(-xu, yu), xl, xu, yl, yu);
  const double M1 = plane_max(yu, xl, __dmul_rn(-yu, xl), xl, xu, yl, yu);
  const double M2 = plane_max(yl, xu, __dmul_rn(-yl, xu), xl, xu, yl, yu);
  const double tl = exact_ties ? TIE_TOL * (fabs(m1) + fabs(m2)) : 0.0;
  const double tu = exact_ties ? TIE_TOL * (fabs(M1) + fabs(M2)) : 0.0;
  const double r_l = (m1 >= m2 - tl) ? 1.0 : 0.0;
  const double r_u = (M1 <= M2 + tu) ? 1.0 : 0.0;
  p[0] = __dadd_rn(__dmul_rn(__dsub_rn(yl, yu), r_l), yu);
  p[1] = __dadd_rn(__dmul_rn(__dsub_rn(xl, xu), r_l), xu);
  p[2] = __dsub_rn(__dmul_rn(__dsub_rn(__dmul_rn(yu, xu), __dmul_rn(yl, xl)), r_l), __dmul_rn(yu, xu));
  p[3] = __dadd_rn(__dmul_rn(__dsub_rn(yu, yl), r_u), yl);
  p[4] = __dadd_rn(__dmul_rn(__dsub_rn(xl, xu), r_u), xu);
  p[5] = __dsub_rn(__dmul_rn(__dsub_rn(__dmul_rn(yl, xu), __dmul_rn(yu, xl)), r_u), __dmul_rn(yl, xu));
}

// Lower bound of specification row s over the output interval [lo, hi] (width wt), as the
// reference's IBP pass applies C (BoundLinear._bound_box, operators/linear.py:621-653): center
// minus deviation (or, with an infinite endpoint, endpoints picked by sign), widened by
// rounding_error(|C| max(|lo|, |hi|), wt). Cb: this box's rows of C, or null for the identity.
template <class V>
__device__ double spec_row_lower(const double* Cb, int wt, V lo, V hi, int off, int s) {
  bool fin = true;
  for (int k = 0; k < wt; ++k) fin = fin && isfinite(lo[off + k]) && isfinite(hi[off + k]);
  double lower, mag;
  if (!Cb) {
    const double l = lo[off + s], h = hi[off + s];
    lower = fin ? (h + l) / 2 - (h - l) / 2 : l;
    mag = finite_abs(fmax(fabs(l), fabs(h)));
  } else {
    const double* c = Cb + (int64_t)s * wt;
    double center = 0, dev = 0, sl = 0;
    mag = 0;
    for (int k = 0; k < wt; ++k) {
      const double w = c[k], l = lo[off + k], h = hi[off + k];
      if (fin) {
        center += ((h + l) / 2) * w;
        dev += ((h - l) / 2) * fabs(w);
      } else {
        sl += (w > 0 ? w * l : 0.0) + (w < 0 ? w * h : 0.0);
      }
      mag += finite_abs(fmax(fabs(l), fabs(h))) * finite_abs(w);
    }
    lower = fin ? center - dev : sl;
  }
  return nan_lo(widen(lower, rounding_error(mag, wt), -1));
}

// ------------------------------------------------------------------ powers (BoundPow)
// Parameters of a pow node: dp[N_CVEC] = {exponent, class, table length}, class 0 = odd
// integer, 1 = even integer, 2 = non-integer (base restricted to x >= 0); an odd exponent's
// tangent-point tables d_lower, d_upper (grid 0.01) start at dp[N_MAP0].
enum { POW_ODD = 0, POW_EVEN = 1, POW_FRAC = 2 };

__device__ __forceinline__ double pow_table_pick(const double* t, int len, double bound, double dflt) {
  // retrieve_from_precompute: entry trunc(bound / 0.01) + 1 (at least 1), else the default
  const double v = bound / STEP_PRE;
  if (!(v < 1.0e15)) return dflt;
  const long long i = (v > 0 ? (long long)v : 0) + 1;
  return i < len ? t[i] : dflt;
}

// BoundPow.bound_relax (operators/s_shaped.py:881-1035), plain CROWN; u already raised to
// lower + 1e-8 by the caller (bound_backward). q = (lw, lb, uw, ub).
__device__ void relax_pow(const DevProgram* P, const int32_t* nd, double l, double u, double* q) {
  const double* pp = P->dp + nd[N_CVEC];
  const double p = pp[0];
  const int cls = (int)pp[1];
  if (cls == POW_ODD) {
    const int len = (int)pp[2];
    const double* dlo_t = P->dp + nd[N_MAP0];
    const double* dup_t = dlo_t + len;
    auto f = [&](double x) { return pow(x, p); };
    auto df = [&](double x) { return p * pow(x, p - 1); };
    auto d2 = [&](double x) { return p * (p - 1) * pow(x, p - 2); };
    const double yl = f(l), yu = f(u), width = u - l;
    double kd = (yu - yl) / fmax(width, 1e-8);
    if (width < 1e-8) kd = df(l);
    const bool conv = d2(l) >= 0;
    const bool mneg = d2(l) >= 0 && d2(u) >= 0, mpos = d2(l) < 0 && d2(u) < 0, mboth = !(mneg || mpos);
    double lw = 0, lb = 0, uw = 0, ub = 0;
    if (mneg) { uw = kd; ub = -l * kd + yl; }
    if (mpos) { lw = kd; lb = -l * kd + yl; }
    const double dup = pow_table_pick(dup_t, len, u, l);
    const double dlo = pow_table_pick(dlo_t, len, -l, u);
    const bool dl_dir = (conv ? kd < df(l) : kd > df(u)) && mboth;
    const bool du_dir = (conv ? kd < df(u) : kd > df(l)) && mboth;
    const double m = (l + u) / 2, ym = f(m), km = df(m);
    if (mneg) { lw = km; lb = -m * km + ym; }
    if (mpos) { uw = km; ub = -m * km + ym; }
    if (dl_dir) { lw = kd; lb = -l * kd + yl; }
    if (mboth && !dl_dir) { const double k = df(dlo); lw = k; lb = -dlo * k + f(dlo); }
    if (du_dir) { uw = kd; ub = -l * kd + yl; }
    if (mboth && !du_dir) { const double k = df(dup); uw = k; ub = -dup * k + f(dup); }
    // inverse-S smoothing: the tangent at the midpoint where the table's point is on the far side
    if (mboth && dlo < m) { lw = km; lb = -m * km + ym; }
    if (mboth && dup >= m) { uw = km; ub = -m * km + ym; }
    q[0] = lw; q[1] = lb; q[2] = uw; q[3] = ub;
    return;
  }
  if (cls == POW_EVEN) {
    const double yl = pow(l, p), yu = pow(u, p);
    const double eps = fmax(fabs(yl), fabs(yu)) * 1e-6 + 1e-12;
    const double uk = (yu - yl) / fmax(u - l, 1e-8);
    const double mid = l >= 0 ? l : (u <= 0 ? u : 0.0);
    const double lk = p * pow(mid, p - 1);
    q[0] = lk; q[1] = -mid * lk + (pow(mid, p) - eps);
    q[2] = uk; q[3] = -l * uk + (yl + eps);
    return;
  }
  // non-integer exponent, l >= 0: concave (p < 1) or convex (p > 1) tangent and secant
  const double lt = p < 1 ? fmax(l, 1e-9) : l;
  const double fl = (p < 1 && l == 0) ? 0.0 : pow(l, p);
  const double fu = pow(u, p);
  const double ks = (fu - fl) / fmax(u - l, 1e-8);
  const double m = (lt + u) / 2;
  double kt, fm;
  if (p > 1 && m == 0) { kt = 0; fm = 0; }
  else { kt = p * pow(m, p - 1); fm = pow(m, p); }
  if (p < 1) { q[0] = ks; q[1] = -l * ks + fl; q[2] = kt; q[3] = -m * kt + fm; }
  else { q[0] = kt; q[1] = -m * kt + fm; q[2] = ks; q[3] = -l * ks + fl; }
}

__device__ __forceinline__ double magnitude(double l, double h) { return l > h ? INFINITY : fmax(-l, h); }

// ------------------------------------------------------------------ per-box context
struct Box {
  const DevProgram* P;
  double* lo;      // interval arena (arena_w)
  double* hi;
  double* mag;     // magnitude arena
  double* planes;  // plane arena
  double* fold;    // fold vectors
  double* pres_lo; // pass results (maxw)
  double* pres_hi;
  const double* xL;  // this box's input box (n)
  const double* xU;
  int64_t b;
  int open;        // some coordinate has a non-finite centre or radius (box_open)
};

// The concretisation A x0 + |A| eps is a dense product over every input coordinate
// (concretize_bounds.py), so one coordinate with a non-finite centre or radius makes every
// row NaN or infinite (0 * inf included): all rows of the box are discarded.
__device__ __forceinline__ int box_open(double l, double h) {
  return !(isfinite((h + l) / 2.0) && isfinite((h - l) / 2.0));
}

__device__ __forceinline__ const int32_t* node_rec(const DevProgram* P, int v) { return P->nodes + v * NODE_REC; }

// Interval of element j of a node from its inputs' intervals (the operators'
// interval_propagate). V is the interval-arena view: a plain pointer (one box per CTA) or a
// box-interleaved view (one box per thread).
template <class V>
__device__ void ibp_element_t(const DevProgram* P, V lo, V hi, const int32_t* nd, int j, double* olo, double* ohi) {
  const int kind = nd[N_KIND];
  double l = 0, h = 0;
  switch (kind) {
    case NK_MUL: {
      const int32_t* a = node_rec(P, nd[N_IN0]);
      const int32_t* c = node_rec(P, nd[N_IN1]);
      int i0 = P->ip[nd[N_MAP0] + j], i1 = P->ip[nd[N_MAP1] + j];
      double xl = lo[a[N_CUR] + i0], xu = hi[a[N_CUR] + i0];
      double yl = lo[c[N_CUR] + i1], yu = hi[c[N_CUR] + i1];
      double r0 = xl * yl, r1 = xl * yu, r2 = xu * yl, r3 = xu * yu;
      bool nan = isnan(r0) || isnan(r1) || isnan(r2) || isnan(r3);
      l = nan ? -INFINITY : fmin(fmin(r0, r1), fmin(r2, r3));
      h = nan ? INFINITY : fmax(fmax(r0, r1), fmax(r2, r3));
      break;
    }
    case NK_MULC: {
      const int32_t* a = node_rec(P, nd[N_IN0]);
      int i0 = P->ip[nd[N_MAP0] + j];
      double xl = lo[a[N_CUR] + i0], xu = hi[a[N_CUR] + i0];
      double c = P->dp[nd[N_CVEC] + j];
      l = c > 0 ? xl * c : (c < 0 ? xu * c : 0.0);
      h = c > 0 ? xu * c : (c < 0 ? xl * c : 0.0);
      break;
    }
    case NK_ADD: case NK_SUB: case NK_ADDC: case NK_SUBC: case NK_RSUBC: {
      const int32_t* a = node_rec(P, nd[N_IN0]);
      int i0 = P->ip[nd[N_MAP0] + j];
      double xl = lo[a[N_CUR] + i0], xu = hi[a[N_CUR] + i0];
      double yl, yu;
      if (kind == NK_ADD || kind == NK_SUB) {
        const int32_t* c = node_rec(P, nd[N_IN1]);
        int i1 = P->ip[nd[N_MAP1] + j];
        yl = lo[c[N_CUR] + i1]; yu = hi[c[N_CUR] + i1];
      } else {
        yl = yu = P->dp[nd[N_CVEC] + j];
        if (kind == NK_RSUBC) { double tl = xl, tu = xu; xl = yl; xu = yu; yl = tl; yu = tu; }
      }
      if (kind == NK_ADD || kind == NK_ADDC) { l = xl + yl; h = xu + yu; }
      else { l = xl - yu; h = xu - yl; }
      l = widen(l, rounding_error(finite_abs(l), 1), -1);
      h = widen(h, rounding_error(finite_abs(h), 1), 1);
      break;
    }
    case NK_NEG: {
      const int32_t* a = node_rec(P, nd[N_IN0]);
      l = -hi[a[N_CUR] + j]; h = -lo[a[N_CUR] + j];
      break;
    }
    case NK_SQR: case NK_EXP: case NK_LOG: case NK_SIN: case NK_COS: {
      const int32_t* a = node_rec(P, nd[N_IN0]);
      double xl = lo[a[N_CUR] + j], xu = hi[a[N_CUR] + j];
      if (kind == NK_SQR) {
        l = xu < 0 ? xu * xu : (xl > 0 ? xl * xl : 0.0);
        h = pmax(xl * xl, xu * xu);
      } else if (kind == NK_EXP) {
        l = exp(xl); h = exp(xu);
      } else if (kind == NK_LOG) {
        if (xl <= 0) xl = 0.0;
        l = log(xl); h = log(xu);
      } else {
        double maxp = kind == NK_SIN ? PI / 2 : 0.0;
        double minp = kind == NK_SIN ? PI * 3 / 2 : PI;
        double fl = kind == NK_SIN ? sin(xl) : cos(xl);
        double fu = kind == NK_SIN ? sin(xu) : cos(xu);
        auto crossing = [&](double ll, double uu, double point) {
          double lc = (ll - point) / (2 * PI);
          double uc = (uu - point) / (2 * PI);
          double ro = 2 * EPS * (1 + fmax(fabs(lc), fabs(uc)));
          return (uu - ll >= 2 * PI) || (floor(uc + ro) > floor(lc - ro));
        };
        h = crossing(xl, xu, maxp) ? 1.0 : pmax(fl, fu);
        l = crossing(xl, xu, minp) ? -1.0 : pmin(fl, fu);
      }
      break;
    }
    case NK_POW: {
      // interval_propagate (s_shaped.py:1083-1121)
      const int32_t* a = node_rec(P, nd[N_IN0]);
      double xl = lo[a[N_CUR] + j], xu = hi[a[N_CUR] + j];
      const double* pp = P->dp + nd[N_CVEC];
      const double p = pp[0];
      const int cls = (int)pp[1];
      if (cls == POW_FRAC) {
        l = pow(fmax(xl, 0.0), p);
        h = pow(xu, p);
      } else {
        const double pl = pow(xl, p), pu = pow(xu, p);
        if (cls == POW_ODD) { l = pl; h = pu; }
        else {
          l = (xl < 0 && xu > 0) ? 0.0 : fmin(pl, pu);
          h = fmax(pl, pu);
        }
      }
      break;
    }
    case NK_REDUCESUM: {
      const int32_t* a = node_rec(P, nd[N_IN0]);
      const int32_t* inv = P->ip + nd[N_MAP1];
      int w = nd[N_W];
      int s0 = inv[j], s1 = inv[j + 1];
      for (int k = s0; k < s1; ++k) {
        int i = inv[w + 1 + k];
        l += lo[a[N_CUR] + i];
        h += hi[a[N_CUR] + i];
      }
      break;
    }
    case NK_MAP: {
      const int32_t* a = node_rec(P, nd[N_IN0]);
      int i = P->ip[nd[N_MAP0] + j];
      l = lo[a[N_CUR] + i]; h = hi[a[N_CUR] + i];
      break;
    }
    case NK_CONCAT: {
      int pos = P->ip[nd[N_MAP0] + j];
      const int32_t* ins = P->ip + nd[N_INS];
      for (int k = 0; k < nd[N_NIN]; ++k) {
        const int32_t* a = node_rec(P, ins[k]);
        if (pos < a[N_W]) { l = lo[a[N_CUR] + pos]; h = hi[a[N_CUR] + pos]; break; }
        pos -= a[N_W];
      }
      break;
    }
    default:
      break;
  }
  *olo = nan_lo(l);
  *ohi = nan_hi(h);
}

__device__ __forceinline__ void ibp_element(const Box& bx, const int32_t* nd, int j, double* olo, double* ohi) {
  ibp_element_t<const double*>(bx.P, bx.lo, bx.hi, nd, j, olo, ohi);
}

// Linear / MatMul interval (interval_bound + BoundLinear._bound_box): warp per output row.
template <int NT>
__device__ void ibp_linear(const Box& bx, const int32_t* nd, double* olo, double* ohi) {
  constexpr int NWARP = NT / 32;
  const DevProgram* P = bx.P;
  int w = nd[N_W], win = nd[N_WIN];
  const double* W = P->dp + nd[N_W_OFF];
  const double* bias = nd[N_B_OFF] >= 0 ? P->dp + nd[N_B_OFF] : nullptr;
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (nd[N_FOLD] >= 0) {
    const double* f = bx.fold + nd[N_FOLD];
    for (int j = threadIdx.x; j < w; j += NT) {
      double bb = bias ? bias[j] : 0.0;
      double l = f[j] - f[w + j], h = f[j] + f[w + j];
      l = l + bb; h = h + bb;
      double err = rounding_error(f[2 * w + j] + fabs(bb), win);
      olo[j] = nan_lo(widen(l, err, -1));
      ohi[j] = nan_hi(widen(h, err, 1));
    }
    return;
  }
  const int32_t* a = node_rec(P, nd[N_IN0]);
  const double* ilo = bx.lo + a[N_CUR];
  const double* ihi = bx.hi + a[N_CUR];
  for (int j = warp; j < w; j += NWARP) {
    const double* Wr = W + (int64_t)j * win;
    double center = 0, dev = 0, mag = 0, slo = 0, shi = 0;
    int nonfin = 0;
    for (int i = lane; i < win; i += 32) {
      double wv = Wr[i];
      double l = ilo[i], h = ihi[i];
      nonfin |= !(isfinite(l) && isfinite(h));
      center += ((l + h) / 2) * wv;
      dev += ((h - l) / 2) * fabs(wv);
      mag += finite_abs(fmax(fabs(l), fabs(h))) * fabs(wv);
      double pl = wv > 0 ? wv * l : (wv < 0 ? wv * h : 0.0);
      double ph = wv > 0 ? wv * h : (wv < 0 ? wv * l : 0.0);
      slo += isnan(pl) ? -INFINITY : pl;
      shi += isnan(ph) ? INFINITY : ph;
    }
    center = warp_sum(center); dev = warp_sum(dev); mag = warp_sum(mag);
    slo = warp_sum(slo); shi = warp_sum(shi);
    nonfin = warp_or(nonfin);
    if (lane == 0) {
      double l = nonfin ? slo : center - dev;
      double h = nonfin ? shi : center + dev;
      double bb = bias ? bias[j] : 0.0;
      l = l + bb; h = h + bb;
      double err = rounding_error(mag + fabs(bb), win);
      olo[j] = nan_lo(widen(l, err, -1));
      ohi[j] = nan_hi(widen(h, err, 1));
    }
  }
}

template <int NT>
__device__ void ibp_node(const Box& bx, int v, double* olo, double* ohi) {
  constexpr int NWARP = NT / 32;
  const int32_t* nd = node_rec(bx.P, v);
  int kind = nd[N_KIND];
  if (kind == NK_LINEAR || kind == NK_MATMUL) {
    ibp_linear<NT>(bx, nd, olo, ohi);
    return;
  }
  if (kind == NK_REDUCESUM) {
    // a warp per output: lanes over the summed inputs
    const DevProgram* P = bx.P;
    const int32_t* a = node_rec(P, nd[N_IN0]);
    const int32_t* inv = P->ip + nd[N_MAP1];
    const int w = nd[N_W];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int j = warp; j < w; j += NWARP) {
      double l = 0, h = 0;
      for (int k = inv[j] + lane; k < inv[j + 1]; k += 32) {
        int i = inv[w + 1 + k];
        l += bx.lo[a[N_CUR] + i];
        h += bx.hi[a[N_CUR] + i];
      }
      l = warp_sum(l);
      h = warp_sum(h);
      if (lane == 0) { olo[j] = nan_lo(l); ohi[j] = nan_hi(h); }
    }
    return;
  }
  int w = nd[N_W];
  for (int j = threadIdx.x; j < w; j += NT) ibp_element(bx, nd, j, olo + j, ohi + j);
}

// fold vectors of a linear/matmul on the input: W x0, |W| eps, |W| max(|xL|, |xU|). The box's
// centre, radius and magnitude are staged in shared memory (`stage`, 3 win doubles); each thread
// owns outputs j and reads column j of the transposed weights (coalesced across the threads).
#ifndef GEAR_FOLD_UNROLL
#define GEAR_FOLD_UNROLL 16
#endif
constexpr int FOLD_UNROLL = GEAR_FOLD_UNROLL;

template <int NT>
__device__ void fold_node(const Box& bx, int v, double* stage) {
  const DevProgram* P = bx.P;
  const int32_t* nd = node_rec(P, v);
  const int w = nd[N_W], win = nd[N_WIN];
  const double* Wt = P->dp + nd[N_WT_OFF];
  double* f = bx.fold + nd[N_FOLD];
  double* xc = stage;
  double* xr = stage + win;
  double* xm = stage + 2 * win;
  for (int i = threadIdx.x; i < win; i += NT) {
    const double l = bx.xL[i], h = bx.xU[i];
    xc[i] = (h + l) / 2.0;
    xr[i] = (h - l) / 2.0;
    xm[i] = finite_abs(fmax(fabs(l), fabs(h)));
  }
  __syncthreads();
  for (int j = threadIdx.x; j < w; j += NT) {
    const double* col = Wt + j;
    double c = 0, r = 0, t = 0;
    int i = 0;
    // FOLD_UNROLL weight loads in flight per thread (one L2 round trip per FOLD_UNROLL inputs;
    // 16 measured fastest of 4, 8, 16, 32 on dense_q_n200)
    for (; i + FOLD_UNROLL <= win; i += FOLD_UNROLL) {
      double wv[FOLD_UNROLL];
#pragma unroll
      for (int q = 0; q < FOLD_UNROLL; ++q) wv[q] = __ldg(col + (int64_t)(i + q) * w);
#pragma unroll
      for (int q = 0; q < FOLD_UNROLL; ++q) {
        const double aw = fabs(wv[q]);
        c = __fma_rn(xc[i + q], wv[q], c);
        r = __fma_rn(xr[i + q], aw, r);
        t = __fma_rn(xm[i + q], aw, t);
      }
    }
    for (; i < win; ++i) {
      const double wv = __ldg(col + (int64_t)i * w), aw = fabs(wv);
      c = __fma_rn(xc[i], wv, c);
      r = __fma_rn(xr[i], aw, r);
      t = __fma_rn(xm[i], aw, t);
    }
    f[j] = c;
    f[w + j] = r;
    f[2 * w + j] = t;
  }
}

template <int NT>
__device__ void relax_node(const Box& bx, int v) {
  const DevProgram* P = bx.P;
  const int32_t* nd = node_rec(P, v);
  int kind = nd[N_KIND], w = nd[N_W];
  double* pl = bx.planes + nd[N_PLANE];
  const double* T = P->dp + P->hdr[H_SINOFF];
  // the undefined-side stop needs the node's own interval to be NaN-free and not inverted on
  // every element (_stop_undefined_interval's precondition)
  int ivbad = 0;
  if (kind != NK_MUL)
    for (int j = threadIdx.x; j < w; j += NT) {
      const double lo_v = bx.lo[nd[N_CUR] + j], hi_v = bx.hi[nd[N_CUR] + j];
      ivbad |= isnan(lo_v) || isnan(hi_v) || lo_v > hi_v;
    }
  const bool stop_ok = !__syncthreads_or(ivbad);
  for (int j = threadIdx.x; j < w; j += NT) {
    if (kind == NK_MUL) {
      const int32_t* a = node_rec(P, nd[N_IN0]);
      const int32_t* c = node_rec(P, nd[N_IN1]);
      int i0 = P->ip[nd[N_MAP0] + j], i1 = P->ip[nd[N_MAP1] + j];
      double xl = bx.lo[a[N_CUR] + i0], xu = bx.hi[a[N_CUR] + i0];
      double yl = bx.lo[c[N_CUR] + i1], yu = bx.hi[c[N_CUR] + i1];
      double* p = pl + 6 * j;
      if (!(isfinite(xl) && isfinite(xu) && isfinite(yl) && isfinite(yu))) {
        for (int k = 0; k < 6; ++k) p[k] = NAN;
      } else {
        relax_mul(xl, xu, yl, yu, p, P->hdr[H_TIES]);
      }
    } else {
      const int32_t* a = node_rec(P, nd[N_IN0]);
      double l = bx.lo[a[N_CUR] + j], u = bx.hi[a[N_CUR] + j];
      double* p = pl + 4 * j;
      if (kind == NK_POW) {
        // bound_backward raises the input's stored upper bound to lower + 1e-8 (persistent)
        u = fmax(u, l + 1e-8);
        bx.hi[a[N_CUR] + j] = u;
        bx.mag[a[N_CUR] + j] = magnitude(l, u);
        if ((int)P->dp[nd[N_CVEC] + 1] == POW_FRAC) l = fmax(l, 0.0);   // base restricted to x >= 0
      }
      bool bad = !(isfinite(l) && isfinite(u));
      if (kind == NK_LOG) bad = bad || !(l > 0);
      const bool off = kind == NK_POW && !(u >= 0 || (int)P->dp[nd[N_CVEC] + 1] != POW_FRAC);
      if (bad || off) {
        if (stop_ok && !off) undefined_stop(kind, l, u, bx.lo[nd[N_CUR] + j], bx.hi[nd[N_CUR] + j], p);
        else p[0] = p[1] = p[2] = p[3] = NAN;
      } else if (kind == NK_SQR) relax_sqr(l, u, p);
      else if (kind == NK_EXP) relax_exp(l, u, p);
      else if (kind == NK_LOG) relax_log(l, u, p);
      else if (kind == NK_SIN) relax_sin(T, l, u, p);
      else if (kind == NK_COS) relax_cos(T, l, u, p);
      else if (kind == NK_POW) relax_pow(P, nd, l, u, p);
    }
  }
}

#ifdef GEAR_STEP_PROFILE
// cycles spent per schedule step / pass op, summed over CTAs (measurement builds only)
__device__ unsigned long long g_step_cycles[8192];
__device__ unsigned long long g_op_cycles[8192];
#endif

// ------------------------------------------------------------------ CROWN pass
// Row arrays in shared memory, per side: VAL = bias + A x0 (NaN marks an undefined row),
// ERR = every outward-rounding magnitude already scaled by its factor, plus |A| eps,
// ROOT = the input term A x0 -/+ |A| eps (for lbias).
enum { R_VAL = 0, R_ERR, R_ROOT, R_COUNT };
constexpr double RE1 = 17 * EPS * 4;   // rounding_error(x, 1) / x

struct PassCtx {
  const int32_t* pr;
  int S, sides;
  double* rows;      // [side][nrows][S]: VAL, ERR (+ ROOT in the final pass)
  int nrows;
  double* red;       // RED_SLOTS reduction slots
  double* buf;       // [side][smem]
  double* la;        // this box's lA block (S x n) when the input's A lives there
  int32_t* stage_ops;
  int smem;
  __device__ double* row(int side, int what) const { return rows + ((size_t)side * nrows + what) * S; }
  __device__ double* vals(int side, int off) const {
    return off == ROOT_IN_LA ? la : buf + (size_t)side * smem + off;
  }
};

// Work split over rows: one thread per row for short rows, one warp per row otherwise.
struct RowSplit {
  int first, step, eoff, estep;
  bool warp;
};
template <int NT>
__device__ __forceinline__ RowSplit row_split(int maxrow) {
  constexpr int NWARP = NT / 32;
  RowSplit r;
  r.warp = maxrow > ROW_THREAD_MAX;
  r.first = r.warp ? (int)(threadIdx.x >> 5) : (int)threadIdx.x;
  r.step = r.warp ? NWARP : NT;
  r.eoff = r.warp ? (int)(threadIdx.x & 31) : 0;
  r.estep = r.warp ? 32 : 1;
  return r;
}

// transformed coefficient for input `slot` of an elementwise op, and its bias term
__device__ __forceinline__ double elem_coef(int kind, int slot, int side, double a, const double* pl,
                                            double cval, double* bterm) {
  *bterm = 0.0;
  switch (kind) {
    case NK_SQR: case NK_EXP: case NK_LOG: case NK_SIN: case NK_COS: case NK_POW: {
      // lower side: positive -> (lw, lb), negative -> (uw, ub); upper side: reversed
      double wp = side == 0 ? pl[0] : pl[2], bp = side == 0 ? pl[1] : pl[3];
      double wn = side == 0 ? pl[2] : pl[0], bn = side == 0 ? pl[3] : pl[1];
      if (a > 0) { *bterm = a * bp; return wp * a; }
      if (a < 0) { *bterm = a * bn; return wn * a; }
      return 0.0;
    }
    case NK_MUL: {
      // planes: al, bl, gl, au, bu, gu (alpha multiplies x, beta y)
      const double* P_ = side == 0 ? pl : pl + 3;   // positive coefficients
      const double* N_ = side == 0 ? pl + 3 : pl;   // negative coefficients
      if (a > 0) { *bterm = a * P_[2]; return P_[slot] * a; }
      if (a < 0) { *bterm = a * N_[2]; return N_[slot] * a; }
      return 0.0;
    }
    case NK_MULC: return a * cval;
    case NK_SUB: return slot == 0 ? a : -a;
    case NK_RSUBC: return -a;
    case NK_NEG: return -a;
    default: return a;   // add, addc, subc, reducesum, map, concat
  }
}

// One row of a GEMV step: Ur[j] (+)= sum_{e0 <= e < e1} V[e] W[vcols[e], j] for this thread's
// columns j = eoff + q estep, with the charges' partial sums <|A||W|, m> (part) and
// <|A W|, m> (pmerge). JB columns per thread per sweep, EB entries per chunk: EB x JB weight
// loads in flight together.
template <int JB, int EB>
__device__ __forceinline__ void gemv_row(const double* V, const int32_t* vcols, int e0, int e1, const double* W,
                                         int win, double* Ur, const double* mu, bool zero_u, int eoff, int estep,
                                         double& part, double& pmerge) {
    // JB columns per thread per sweep of the row's entries: their weight loads are in
    // flight together instead of one dependent load chain per column
    for (int jb = eoff; jb < win; jb += JB * estep) {
      double acc[JB], ab[JB];
      bool ok[JB];
#pragma unroll
      for (int q = 0; q < JB; ++q) { acc[q] = 0.0; ab[q] = 0.0; ok[q] = jb + q * estep < win; }

      // entries in chunks of EB: their indices and coefficients first, then EB x JB weight
      // loads in flight together, then the sums (in entry order)
      for (int e = e0; e < e1; e += EB) {
        int cq[EB];
        double aq[EB];
#pragma unroll
        for (int r = 0; r < EB; ++r) {
          const bool in = e + r < e1;
          cq[r] = in ? __ldg(vcols + e + r) : 0;
          aq[r] = in ? V[e + r] : 0.0;
        }
        double wq[EB][JB];
#pragma unroll
        for (int r = 0; r < EB; ++r) {
          const double* Wr = W + (int64_t)cq[r] * win + jb;
#pragma unroll
          for (int q = 0; q < JB; ++q) wq[r][q] = (ok[q] && e + r < e1) ? __ldg(Wr + q * estep) : 0.0;
        }
#pragma unroll
        for (int r = 0; r < EB; ++r) {
          if (e + r >= e1) break;
#pragma unroll
          for (int q = 0; q < JB; ++q) {
            acc[q] = __fma_rn(aq[r], wq[r][q], acc[q]);
            ab[q] = __fma_rn(fabs(aq[r]), fabs(wq[r][q]), ab[q]);
          }
        }
      }
      double mq[JB], uq[JB];
#pragma unroll
      for (int q = 0; q < JB; ++q) {
        mq[q] = ok[q] ? mu[jb + q * estep] : 0.0;
        uq[q] = (ok[q] && !zero_u) ? Ur[jb + q * estep] : 0.0;
      }
#pragma unroll
      for (int q = 0; q < JB; ++q) {
        if (!ok[q]) continue;
        Ur[jb + q * estep] = zero_u ? acc[q] : uq[q] + acc[q];
        const double mf = isinf(mq[q]) ? 0.0 : mq[q];
        part += ab[q] * mf;
        pmerge += fabs(acc[q]) * mf;
      }
    }
}

// One CROWN pass. phase bit 1: clear the row arrays and set the initial A at the pass's target;
// ops [op_lo, op_hi) of the pass then run; phase bit 2: concretise and write the outputs. The
// fused kernels run everything in one call; the plain form calls each phase and each op in a
// launch of its own (the working set then lives in global memory).
// IDX: also skip the loads of identity source / target lists and row pointers (OpFlag). Used
// by the instances whose working set is in global memory; in the shared-memory instances the
// extra live flags cost more in register spills than the loads they save (measured).
// SPLIT: the tensor-core programs' instance, which can hand the final pass's product through a
// dense node on the input (OF_SPLIT op) to the tensor cores (Work.split_v).
template <int NT, bool WHOLE = true, bool IDX = false, bool SPLIT = false>
__device__ void run_pass(const Box& bx, int pid, double* sm, int32_t* stage_ops, const Work& wk, int op_lo_ = 0,
                         int op_hi_ = 1 << 30, int phase_ = 3) {
  // WHOLE: every phase and every op (compile-time constants for the fused kernels)
  const int op_lo = WHOLE ? 0 : op_lo_;
  const int op_hi = WHOLE ? (1 << 30) : op_hi_;
  const int phase = WHOLE ? 3 : phase_;
  constexpr int NWARP = NT / 32;
  const DevProgram* P = bx.P;
  const int32_t* pr = P->passes + pid * PASS_REC;
  PassCtx ctx;
  ctx.pr = pr;
  ctx.S = pr[P_S];
  ctx.sides = pr[P_SIDES];
  ctx.smem = pr[P_SMEM];
  ctx.rows = sm;
  ctx.nrows = pr[P_FINAL] != 0 ? R_COUNT : R_COUNT - 1;
  ctx.red = sm + (size_t)ctx.sides * ctx.nrows * ctx.S;
  ctx.buf = ctx.red + RED_SLOTS;
  const bool xdense = pr[P_XDENSE] != 0;
  ctx.la = xdense ? wk.lA + (size_t)bx.b * ctx.S * P->hdr[H_N] : nullptr;
  ctx.stage_ops = stage_ops;
  const int S = ctx.S, sides = ctx.sides;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int n = P->hdr[H_N];
  const int t = pr[P_T];
  const double fbias = ((double)max(pr[P_NVISIT], 1) + n + 16) * EPS * 4;   // bias sums
  const double fbox = ((double)n + 16) * EPS * 4;                             // box dot products
  const int32_t* tnd = node_rec(P, t);

  if (phase & 1) {
  for (int k = tid; k < sides * ctx.nrows * S; k += NT) ctx.rows[k] = 0.0;
  // initial A at t
  {
    const int32_t* trp = P->ip + pr[P_TRP];
    int nnz_t = trp[S];
    for (int side = 0; side < sides; ++side) {
      double* V = ctx.vals(side, pr[P_TBUF]);
      if (pr[P_INIT] == 0) {
        for (int k = tid; k < nnz_t; k += NT) V[k] = 1.0;     // row s -> entry (s, s)
      } else {
        int wt = tnd[N_W];
        const double* Cb = wk.C + (size_t)bx.b * S * wt;
        for (int k = tid; k < nnz_t; k += NT) V[k] = Cb[k];  // dense rows, entry order = (s, c)
      }
    }
  }
  __syncthreads();
  }

  const int op0 = pr[P_OP0], nop = pr[P_NOP];
  // this pass's op records in shared memory (decoded once per box instead of per access)
  int32_t* sops = ctx.stage_ops;
  for (int k = tid; k < nop * OP_REC; k += NT) sops[k] = __ldg(P->ops + (size_t)op0 * OP_REC + k);
  __syncthreads();
#ifdef GEAR_STEP_PROFILE
  long long t_op = clock64();
  extern __device__ unsigned long long g_op_cycles[];
#endif
  const int op_end = min(nop, op_hi);
  for (int oi = op_lo; oi < op_end; ++oi) {
    const int32_t* op = sops + oi * OP_REC;
    const int kind = op[O_KIND], v = op[O_V], slot = op[O_SLOT];
    const int32_t* vnd = node_rec(P, v);
    const int32_t* vrp = P->ip + op[O_VRP];
    const int32_t* vcols = P->ip + op[O_VCOLS];
    const double* pl = vnd[N_PLANE] >= 0 ? bx.planes + vnd[N_PLANE] : nullptr;
    const bool relax = (kind == NK_SQR || kind == NK_EXP || kind == NK_LOG || kind == NK_SIN || kind == NK_COS ||
                        kind == NK_POW);
    const int ppe = kind == NK_MUL ? 6 : 4;
    const int u = op[O_U];
    const int32_t* und = u >= 0 ? node_rec(P, u) : nullptr;
    const bool first = op[O_FIRST] != 0;
    const bool zero_u = !op[O_FOLD] && !op[O_UMERGE];
    const bool u_la = op[O_UBUF] == ROOT_IN_LA;
    const int uk = op[O_UK];
    const double gmerge = uk >= 2 ? gamma_k((double)uk) : 0.0;
    const double* mu = und ? bx.mag + und[N_CUR] : nullptr;
    const int32_t* urp = (!op[O_FOLD]) ? P->ip + op[O_URP] : nullptr;
    const int32_t* ucols = (!op[O_FOLD]) ? P->ip + op[O_UCOLS] : nullptr;
    const bool need_a = first && (relax || kind == NK_MUL || kind == NK_MULC || kind == NK_ADD || kind == NK_SUB ||
                                  kind == NK_ADDC || kind == NK_SUBC || kind == NK_RSUBC ||
                                  ((kind == NK_LINEAR) && vnd[N_B_OFF] >= 0));
    const double* cvec = vnd[N_CVEC] >= 0 ? P->dp + vnd[N_CVEC] : nullptr;
    const int32_t* map0 = vnd[N_MAP0] >= 0 ? P->ip + vnd[N_MAP0] : nullptr;
    const int32_t* map1 = vnd[N_MAP1] >= 0 ? P->ip + vnd[N_MAP1] : nullptr;
    const int32_t* inex = vnd[N_INEXACT] >= 0 ? P->ip + vnd[N_INEXACT] : nullptr;
    const double* m0 = bx.mag + node_rec(P, vnd[N_IN0])[N_CUR];
    const double* m1 = (kind == NK_ADD || kind == NK_SUB) ? bx.mag + node_rec(P, vnd[N_IN1])[N_CUR] : nullptr;
    const double* bvec = (kind == NK_LINEAR && vnd[N_B_OFF] >= 0) ? P->dp + vnd[N_B_OFF] : nullptr;
    const bool dense = op[O_DENSE] != 0 && !op[O_FOLD];
    const int oflags = op[O_SINGLE];   // OpFlag bits

    // ---- per-row work of a non-GEMV op: bias/charges over v's row, zero u's row on its first
    //      contribution, pull the row's moves (or fold it into the concretisation)
    // sum over the threads working on one row: a warp (mode 1) or the CTA (mode 2, every thread
    // takes part; two barriers). Fixed order: deterministic.
    auto row_sum = [&](double v, int mode) -> double {
      v = warp_sum(v);
      if (mode == 1) return v;
      if (lane == 0) ctx.red[warp] = v;
      __syncthreads();
      double t = 0.0;
      for (int w_ = 0; w_ < NWARP; ++w_) t += ctx.red[w_];
      __syncthreads();
      return t;
    };
    // mode 0: one thread per row, 1: a warp, 2: the whole CTA (every thread calls with the same s)
    auto row_body = [&](int s, int eoff, int estep, int mode) {
      const bool lead = mode == 0 || (mode == 1 ? lane == 0 : tid == 0);
      const bool vid = IDX && (oflags & OF_VRP_ID);
      const int e0 = vid ? s : vrp[s], e1 = vid ? s + 1 : vrp[s + 1];
      for (int side = 0; side < sides; ++side) {
        const double* V = ctx.vals(side, op[O_VBUF]);
        if (need_a && e0 < e1) {
          double sb = 0, sm_ = 0, sc = 0;
          int und_ = 0;
          for (int e = e0 + eoff; e < e1; e += estep) {
            double a = V[e];
            int c = vcols[e];
            if (relax || kind == NK_MUL) {
              const double* p = pl + ppe * c;
              double bt;
              double na = elem_coef(kind, 0, side, a, p, 0.0, &bt);
              double bt2 = 0.0, nb = 0.0;
              if (kind == NK_MUL) nb = elem_coef(kind, 1, side, a, p, 0.0, &bt2);
              if (a != 0.0 && (!isfinite(bt) || !isfinite(na) || !isfinite(nb))) und_ = 1;
              if (isfinite(bt)) { sb += bt; sm_ += fabs(bt); }
            } else if (kind == NK_MULC) {
              double cv = cvec[c];
              if (inex[c] && a != 0.0) {
                double m = m0[map0[c]];
                // on an unbounded input only a product that rounded costs (the exact error of a
                // cv, one FMA; _affine_backward_terms, backward_bound.py:611-640)
                sc += isinf(m) ? (__fma_rn(a, cv, -(a * cv)) != 0.0 ? INFINITY : 0.0) : UNIT * (fabs(a * cv) * m);
              }
            } else if (kind == NK_LINEAR) {
              // bias of a folded Linear: A_v . b
              sb += a * bvec[c];
              sm_ += fabs(a) * fabs(bvec[c]);
            } else {
              // add / sub / addc / subc / rsubc: output rounding (interval_bound.py:71-77)
              double mx = m0[map0[c]];
              double my = m1 ? m1[map1[c]] : fabs(cvec[c]);
              double e_ = rounding_error(mx + my, 2);
              double fa = finite_abs(a);
              // an unbounded output entry adds nothing (its magnitude counts as 0, as in the
              // deferred charge of _enclose_affine_backward, backward_bound.py:780-787)
              sc += fa > 0 ? (isinf(e_) ? 0.0 : fa * e_) : 0.0;
              if (kind == NK_ADDC || kind == NK_SUBC || kind == NK_RSUBC) {
                double cv = kind == NK_SUBC ? -cvec[c] : cvec[c];
                sb += a * cv;
                sm_ += fabs(a) * fabs(cv);
              }
            }
          }
          if (mode != 0) {
            // the four sums of the row: warp sums, then (whole-CTA rows) one exchange through the
            // reduction slots, each value summed over the warps in warp order as row_sum does
            sb = warp_sum(sb);
            sm_ = warp_sum(sm_);
            sc = warp_sum(sc);
            double ud = warp_sum((double)und_);
            if (mode == 2) {
              if (lane == 0) {
                ctx.red[warp] = sb;
                ctx.red[NWARP + warp] = sm_;
                ctx.red[2 * NWARP + warp] = sc;
                ctx.red[3 * NWARP + warp] = ud;
              }
              __syncthreads();
              double t0 = 0.0, t1 = 0.0, t2 = 0.0, t3 = 0.0;
              for (int w_ = 0; w_ < NWARP; ++w_) {
                t0 += ctx.red[w_];
                t1 += ctx.red[NWARP + w_];
                t2 += ctx.red[2 * NWARP + w_];
                t3 += ctx.red[3 * NWARP + w_];
              }
              __syncthreads();
              sb = t0;
              sm_ = t1;
              sc = t2;
              ud = t3;
            }
            und_ = ud != 0.0;
          }
          if (lead) {
            double* val = ctx.row(side, R_VAL);
            val[s] = und_ ? NAN : val[s] + sb;
            ctx.row(side, R_ERR)[s] += sm_ * fbias + sc;
          }
        }
        if (op[O_FOLD]) {
          // linear/matmul on the input, one entry per row: exact fold into the concretisation
          if (e0 < e1 && lead) {
            const double* f = bx.fold + vnd[N_FOLD];
            const int w = vnd[N_W];
            const double gk = gamma_k((double)op[O_WOUT]);
            double a = V[e0];
            int c = vcols[e0];
            ctx.row(side, R_VAL)[s] += a * f[c];
            ctx.row(side, R_ERR)[s] += fabs(a) * f[w + c] + (fabs(a) * f[2 * w + c]) * fbox +
                                       gk * (fabs(a) * f[2 * w + c]);
          }
          continue;
        }
        double* U = ctx.vals(side, op[O_UBUF]);
        if (zero_u) {
          if (u_la) for (int j = eoff; j < n; j += estep) U[(size_t)s * n + j] = 0.0;
          else for (int j = urp[s] + eoff; j < urp[s + 1]; j += estep) U[j] = 0.0;
          if (mode == 1) __syncwarp();
          if (mode == 2) __syncthreads();
        }
        const int32_t* tptr = P->ip + op[O_TPTR];
        const int k0 = (oflags & OF_TPTR_ID) ? s : tptr[s], k1 = (oflags & OF_TPTR_ID) ? s + 1 : tptr[s + 1];
        if (k0 == k1) continue;
        const int32_t* tgt = P->ip + op[O_TGT];
        const int32_t* sptr = P->ip + op[O_SPTR];
        const int32_t* src = P->ip + op[O_SRC];
        double pmerge = 0;
        const bool single = (oflags & OF_SINGLE) != 0;
        for (int k = k0 + eoff; k < k1; k += estep) {
          double acc = 0;
          const int q0 = single ? k : __ldg(sptr + k), q1 = single ? k + 1 : __ldg(sptr + k + 1);
          for (int q = q0; q < q1; ++q) {
            int e = (IDX && (oflags & OF_SRC_ID)) ? q : __ldg(src + q);
            double a = V[e];
            int c = __ldg(vcols + e);
            double bt;
            double na = elem_coef(kind, slot, side, a, pl ? pl + ppe * c : nullptr, cvec ? __ldg(cvec + c) : 0.0, &bt);
            if (!isfinite(na)) na = 0.0;
            acc += na;
          }
          int ti = (IDX && (oflags & OF_TGT_ID)) ? k : tgt[k];
          const double old = U[ti];
          const double tot = old + acc;
          U[ti] = tot;
          if (uk >= 2 && acc != 0.0) {
            int col = u_la ? ti - s * n : ucols[ti];
            double m = mu[col];
            pmerge += isinf(m) ? (merge_rounded(old, acc, tot) ? INFINITY : 0.0) : fabs(acc) * m;
          }
        }
        if (uk >= 2) {
          if (mode != 0) pmerge = row_sum(pmerge, mode);
          if (lead) ctx.row(side, R_ERR)[s] += gmerge * pmerge;
        }
      }
    };

    // an entry-wise op (OF_FUSED, every row short): one sweep over the row's entries takes each
    // entry's bias terms and its move (u's entry e <- v's entry e), in the order and with the
    // arithmetic of row_body's two sweeps, so the results are the same bits; u's row needs no
    // clearing (a fresh row holds exactly the moved entries)
    // OF_FUSED_T: entry e moves to u's entry tgt[e] of the same row; a fresh u row is cleared first
    auto fused_row = [&](int s) {
      const bool vid = (oflags & OF_VRP_ID) != 0;
      const bool tmap = (oflags & OF_FUSED_T) != 0;
      const int e0 = vid ? s : vrp[s], e1 = vid ? s + 1 : vrp[s + 1];
      if (e0 == e1 && !(tmap && zero_u)) return;
      const int32_t* tgt = P->ip + op[O_TGT];
      for (int side = 0; side < sides; ++side) {
        const double* V = ctx.vals(side, op[O_VBUF]);
        double* U = ctx.vals(side, op[O_UBUF]);
        // a u row the op opens is cleared even where v's row is empty (as row_body does)
        if (tmap && zero_u) for (int j = urp[s]; j < urp[s + 1]; ++j) U[j] = 0.0;
        if (e0 == e1) continue;
        double sb = 0, sm_ = 0, sc = 0, pmerge = 0;
        int und_ = 0;
        for (int e = e0; e < e1; ++e) {
          const double a = V[e];
          const int c = __ldg(vcols + e);
          double na;
          if (relax || kind == NK_MUL) {
            const double* p = pl + ppe * c;
            double bt;
            na = elem_coef(kind, slot, side, a, p, 0.0, &bt);
            if (need_a) {   // slot 0: the node's bias terms
              double bt2, nb = 0.0;
              if (kind == NK_MUL) nb = elem_coef(kind, 1, side, a, p, 0.0, &bt2);
              if (a != 0.0 && (!isfinite(bt) || !isfinite(na) || !isfinite(nb))) und_ = 1;
              if (isfinite(bt)) { sb += bt; sm_ += fabs(bt); }
            }
          } else if (kind == NK_MULC) {
            const double cv = __ldg(cvec + c);
            na = a * cv;
            if (need_a && inex[c] && a != 0.0) {
              const double m = m0[map0[c]];
              sc += isinf(m) ? (__fma_rn(a, cv, -(a * cv)) != 0.0 ? INFINITY : 0.0) : UNIT * (fabs(a * cv) * m);
            }
          } else {
            double bt;
            na = elem_coef(kind, slot, side, a, nullptr, cvec ? __ldg(cvec + c) : 0.0, &bt);
            if (need_a) {
              const double mx = m0[map0[c]];
              const double my = m1 ? m1[map1[c]] : fabs(cvec[c]);
              const double e_ = rounding_error(mx + my, 2);
              const double fa = finite_abs(a);
              sc += fa > 0 ? (isinf(e_) ? 0.0 : fa * e_) : 0.0;
              if (kind == NK_ADDC || kind == NK_SUBC || kind == NK_RSUBC) {
                const double cv = kind == NK_SUBC ? -cvec[c] : cvec[c];
                sb += a * cv;
                sm_ += fabs(a) * fabs(cv);
              }
            }
          }
          const double acc = 0.0 + (isfinite(na) ? na : 0.0);
          const int ti = tmap ? __ldg(tgt + e) : e;
          const double old = zero_u ? 0.0 : U[ti];
          const double tot = old + acc;
          U[ti] = tot;
          if (uk >= 2 && acc != 0.0) {
            const double m = mu[ucols[ti]];
            pmerge += isinf(m) ? (merge_rounded(old, acc, tot) ? INFINITY : 0.0) : fabs(acc) * m;
          }
        }
        if (need_a) {
          double* val = ctx.row(side, R_VAL);
          val[s] = und_ ? NAN : val[s] + sb;
          ctx.row(side, R_ERR)[s] += sm_ * fbias + sc;
        }
        if (uk >= 2) ctx.row(side, R_ERR)[s] += gmerge * pmerge;
      }
    };

    if (!dense) {
      const int32_t* shortr = P->ip + op[O_SHORT];
      const int32_t* longr = P->ip + op[O_LONG];
      const int nshort = op[O_NSHORT], nlong = op[O_NLONG];
      if (oflags & (OF_FUSED | OF_FUSED_T)) {
        for (int i = tid; i < nshort; i += NT) fused_row(shortr[i]);
      } else {
      for (int i = tid; i < nshort; i += NT) row_body(shortr[i], 0, 1, 0);
      if (2 * nlong <= NWARP) {
        // few long rows (single rows of a chain): the whole CTA on each, instead of idle warps
        for (int i = 0; i < nlong; ++i) row_body(longr[i], tid, NT, 2);
      } else {
        for (int i = warp; i < nlong; i += NWARP) row_body(longr[i], lane, 32, 1);
      }
      }
    } else {
      // ---- GEMV: A_u[s, :] (+)= sum_e A_v[e] W[c_e, :]; charges gamma_w <|A_v||W|, m_u> and merges
      const bool block_rows = op[O_VROWS] < NWARP;   // few rows: the whole CTA on each row
      const int s0 = block_rows ? 0 : warp, sstep = block_rows ? 1 : NWARP;
      const int eoff = block_rows ? tid : lane, estep = block_rows ? NT : 32;
      const double* W = P->dp + vnd[N_W_OFF];
      const int win = vnd[N_WIN];
      const double gk = gamma_k((double)op[O_WOUT]);
      for (int s = s0; s < S; s += sstep) {
        const int e0 = vrp[s], e1 = vrp[s + 1];
        for (int side = 0; side < sides; ++side) {
          const double* V = ctx.vals(side, op[O_VBUF]);
          double* U = ctx.vals(side, op[O_UBUF]);
          double* Ur = u_la ? U + (size_t)s * n : U + urp[s];
          const int urow = u_la ? n : urp[s + 1] - urp[s];
          if (need_a && e0 < e1) {
            // Linear bias A_v . b
            double sb = 0, sm_ = 0;
            for (int e = e0 + eoff; e < e1; e += estep) {
              double a = V[e];
              sb += a * bvec[vcols[e]];
              sm_ += fabs(a) * fabs(bvec[vcols[e]]);
            }
            sb = warp_sum(sb); sm_ = warp_sum(sm_);
            if (block_rows) {
              if (lane == 0) { ctx.red[warp] = sb; ctx.red[NWARP + warp] = sm_; }
              __syncthreads();
              if (tid == 0) {
                double tb = 0, tm = 0;
                for (int w_ = 0; w_ < NWARP; ++w_) { tb += ctx.red[w_]; tm += ctx.red[NWARP + w_]; }
                ctx.row(side, R_VAL)[s] += tb;
                ctx.row(side, R_ERR)[s] += tm * fbias;
              }
              __syncthreads();
            } else if (lane == 0) {
              ctx.row(side, R_VAL)[s] += sb;
              ctx.row(side, R_ERR)[s] += sm_ * fbias;
            }
          }
          if (SPLIT && (oflags & OF_SPLIT) && wk.split_v) {
            // the tensor cores take this row's product: its A row, dense over v's outputs
            double* dst = wk.split_v + ((size_t)bx.b * S + s) * wk.split_k;
            for (int j = eoff; j < wk.split_k; j += estep) dst[j] = 0.0;
            if (block_rows) __syncthreads();
            else __syncwarp();
            for (int e = e0 + eoff; e < e1; e += estep) dst[vcols[e]] = V[e];
            continue;
          }
          if (e0 == e1) {
            if (zero_u) for (int j = eoff; j < urow; j += estep) Ur[j] = 0.0;
            continue;
          }
          double part = 0, pmerge = 0;
          if (block_rows) gemv_row<2, 8>(V, vcols, e0, e1, W, win, Ur, mu, zero_u, eoff, estep, part, pmerge);
          else if (op[O_VMAXROW] <= 2) gemv_row<8, 1>(V, vcols, e0, e1, W, win, Ur, mu, zero_u, eoff, estep, part, pmerge);
          else gemv_row<4, 4>(V, vcols, e0, e1, W, win, Ur, mu, zero_u, eoff, estep, part, pmerge);
          double tot_ = gk * warp_sum(part) + gmerge * warp_sum(pmerge);
          if (block_rows) {
            if (lane == 0) ctx.red[warp] = tot_;
            __syncthreads();
            if (tid == 0) {
              double t_ = 0;
              for (int w_ = 0; w_ < NWARP; ++w_) t_ += ctx.red[w_];
              ctx.row(side, R_ERR)[s] += t_;
            }
            __syncthreads();
          } else if (lane == 0) {
            ctx.row(side, R_ERR)[s] += tot_;
          }
        }
      }
    }
    __syncthreads();
#ifdef GEAR_STEP_PROFILE
    if (tid == 0) {
      long long t1 = clock64();
      atomicAdd(&g_op_cycles[op0 + oi], (unsigned long long)(t1 - t_op));
      t_op = t1;
    }
#endif
  }
  if (!WHOLE && (phase & 4)) {
    // the pass's input A rows, dense and signed, for the constrained sweep (absent entries are
    // zeros of the row's sign, as in the dense product -A of the reference)
    const int H = wk.cut_h;
    double* obj = wk.cut_obj + (size_t)bx.b * H * n;
    for (int side = 0; side < sides; ++side) {
      const double z = side == 0 ? 0.0 : -0.0;
      for (int k = tid; k < S * n; k += NT) obj[(size_t)side * S * n + k] = z;
    }
    __syncthreads();
    if (pr[P_NFOLD] == 0 && pr[P_XNNZ] > 0) {
      const int32_t* xrp = P->ip + pr[P_XRP];
      const int32_t* xcols = P->ip + pr[P_XCOLS];
      for (int side = 0; side < sides; ++side) {
        const double* V = ctx.vals(side, pr[P_XBUF]);
        const double sg = side == 0 ? 1.0 : -1.0;
        for (int s = warp; s < S; s += NWARP) {
          const int e0 = xrp[s], e1 = xrp[s + 1];
          for (int e = e0 + lane; e < e1; e += 32) {
            const int c = xcols[e];
            const double a = xdense ? V[(size_t)s * n + c] : V[e];
            obj[((size_t)side * S + s) * n + c] = sg * a;
          }
        }
      }
    }
    __syncthreads();
  }
  if (!(phase & 2)) return;
#ifdef GEAR_STEP_PROFILE
  if (tid == 0) t_op = clock64();
#endif
  if (SPLIT && wk.split_v && pr[P_FINAL] != 0 && nop > 0 && (sops[(nop - 1) * OP_REC + O_SINGLE] & OF_SPLIT)) {
    // the input's A comes from the tensor cores: hand each row's bias sum, charge sum and
    // interval fallback (backward_bound.py:826) and the box's open flag to split_tail_kernel
    for (int s = tid; s < S; s += NT) {
      double fb = 0;
      if (pr[P_INIT] == 0) {
        fb = bx.lo[tnd[N_CUR] + s];
      } else {
        const int wt = tnd[N_W];
        const double* Cb = wk.C + ((size_t)bx.b * S + s) * wt;
        for (int c = 0; c < wt; ++c) {
          const double cv = Cb[c];
          fb += cv > 0 ? cv * bx.lo[tnd[N_CUR] + c] : (cv < 0 ? cv * bx.hi[tnd[N_CUR] + c] : 0.0);
        }
      }
      double* r = wk.split_rows + ((size_t)bx.b * S + s) * 3;
      r[0] = ctx.row(0, R_VAL)[s];
      r[1] = ctx.row(0, R_ERR)[s];
      r[2] = fb;
    }
    if (tid == 0) wk.split_open[bx.b] = bx.open ? 1 : 0;
    __syncthreads();
    return;
  }

  // ---- concretisation at the input and outputs
  const bool fold = pr[P_NFOLD] != 0;
  const int xnnz = pr[P_XNNZ];
  const int32_t* xrp = (!fold && xnnz > 0) ? P->ip + pr[P_XRP] : nullptr;
  const int32_t* xcols = (!fold && xnnz > 0) ? P->ip + pr[P_XCOLS] : nullptr;
  if (!WHOLE && wk.cut_v) {
    // concretisation over box ∩ cut rows: the sweep's lower bound of each signed row (its own
    // rounding included) replaces the box terms; the root term of lbias is that bound
    const double* cv = wk.cut_v + (size_t)bx.b * wk.cut_h;
    for (int side = 0; side < sides; ++side) {
      for (int s = tid; s < S; s += NT) {
        const double v = cv[side * S + s];
        const double base = side == 0 ? v : -v;
        ctx.row(side, R_VAL)[s] += base;
        if (ctx.nrows > R_ROOT) ctx.row(side, R_ROOT)[s] = base;
      }
    }
  } else if (xrp) {
    const RowSplit rs = row_split<NT>(pr[P_XMAXROW]);
    for (int side = 0; side < sides; ++side) {
      const double* V = ctx.vals(side, pr[P_XBUF]);
      const double sign = side == 0 ? -1.0 : 1.0;
      for (int s = rs.first; s < S; s += rs.step) {
        int e0 = xrp[s], e1 = xrp[s + 1];
        double bs = 0, dv = 0, be = 0;
        constexpr int XB = 8;
        // XB entries per step: index, coefficient and box loads issued before the sums
        const bool full = e1 - e0 == n;       // a full row: entry e is column e - e0
        for (int e = e0 + rs.eoff; e < e1; e += XB * rs.estep) {
          int cq[XB];
          bool ok[XB];
#pragma unroll
          for (int q = 0; q < XB; ++q) {
            ok[q] = e + q * rs.estep < e1;
            cq[q] = ok[q] ? (full ? e + q * rs.estep - e0 : __ldg(xcols + e + q * rs.estep)) : 0;
          }
          double aq[XB], lq[XB], hq[XB];
#pragma unroll
          for (int q = 0; q < XB; ++q) {
            aq[q] = ok[q] ? (xdense ? V[(size_t)s * n + cq[q]] : V[e + q * rs.estep]) : 0.0;
            lq[q] = ok[q] ? bx.xL[cq[q]] : 0.0;
            hq[q] = ok[q] ? bx.xU[cq[q]] : 0.0;
          }
#pragma unroll
          for (int q = 0; q < XB; ++q) {
            if (!ok[q]) continue;
            const double a = aq[q], l = lq[q], h = hq[q];
            bs = __fma_rn(a, (h + l) / 2.0, bs);
            dv = __fma_rn(fabs(a), (h - l) / 2.0, dv);
            be = __fma_rn(finite_abs(a), finite_abs(fmax(fabs(l), fabs(h))), be);
          }
        }
        if (rs.warp) { bs = warp_sum(bs); dv = warp_sum(dv); be = warp_sum(be); }
        if (!rs.warp || lane == 0) {
          ctx.row(side, R_VAL)[s] += bs;
          ctx.row(side, R_ERR)[s] += dv + be * fbox;
          if (ctx.nrows > R_ROOT) ctx.row(side, R_ROOT)[s] = bs + sign * dv;
        }
      }
    }
  }
  __syncthreads();
#ifdef GEAR_STEP_PROFILE
  if (tid == 0) atomicAdd(&g_op_cycles[8190], (unsigned long long)(clock64() - t_op));
#endif
  const bool final = pr[P_FINAL] != 0;
  for (int side = 0; side < sides; ++side) {
    double sign = side == 0 ? -1.0 : 1.0;
    for (int s = tid; s < S; s += NT) {
      double val = ctx.row(side, R_VAL)[s], er = ctx.row(side, R_ERR)[s];
      double tot = val + sign * (er + (fabs(val) + er) * RE1);
      const bool bad = bx.open || isnan(tot) || tot == -sign * INFINITY;
      if (bad) tot = sign * INFINITY;
      if (final) {
        double lbv = tot;
        if (bad) {
          // interval fallback for a discarded row (backward_bound.py:826)
          double fb = 0;
          if (pr[P_INIT] == 0) fb = bx.lo[tnd[N_CUR] + s];
          else {
            int wt = tnd[N_W];
            const double* Cb = wk.C + ((size_t)bx.b * S + s) * wt;
            for (int c = 0; c < wt; ++c) {
              double cv = Cb[c];
              fb += cv > 0 ? cv * bx.lo[tnd[N_CUR] + c] : (cv < 0 ? cv * bx.hi[tnd[N_CUR] + c] : 0.0);
            }
          }
          lbv = fmax(lbv, fb);
        }
        if (wk.lb_ibp) lbv = fmax(lbv, wk.lb_ibp[(size_t)bx.b * S + s]);   // IBP pass of the bounding glue
        wk.lb[(size_t)bx.b * S + s] = lbv;
        if (wk.lbias) wk.lbias[(size_t)bx.b * S + s] = bad ? -INFINITY : tot - ctx.row(side, R_ROOT)[s];
        ctx.row(side, R_VAL)[s] = bad ? NAN : tot;    // the lA rows of bad rows are cleared below
      } else {
        double* out = side == 0 ? bx.pres_lo : bx.pres_hi;
        out[s] = tot;
      }
    }
  }
  __syncthreads();
  if (final && wk.lA && xdense) {
    // the input's A was accumulated in place; rows of undefined bounds become zero
    for (int s = warp; s < S; s += NWARP) {
      if (!isnan(ctx.row(0, R_VAL)[s])) continue;
      for (int c = lane; c < n; c += 32) ctx.la[(size_t)s * n + c] = 0.0;
    }
  } else if (final && wk.lA) {
    // dense lA rows: zero, then the input's entries (rows of undefined bounds stay zero)
    double* lA = wk.lA + (size_t)bx.b * S * n;
    for (int k = tid; k < S * n; k += NT) lA[k] = 0.0;
    __syncthreads();
    if (xrp) {
      const double* V = ctx.vals(0, pr[P_XBUF]);
      for (int s = warp; s < S; s += NWARP) {
        if (isnan(ctx.row(0, R_VAL)[s])) continue;
        for (int e = xrp[s] + lane; e < xrp[s + 1]; e += 32) lA[(size_t)s * n + xcols[e]] = V[e];
      }
    }
  }
  __syncthreads();
}

template <int NT>
__device__ void compare_node(const Box& bx, int v, double* tmp_lo, double* tmp_hi, bool with_mag) {
  // IBP of v from its inputs' current intervals, intersected with the pass result
  const int32_t* nd = node_rec(bx.P, v);
  int w = nd[N_W];
  ibp_node<NT>(bx, v, tmp_lo, tmp_hi);
  __syncthreads();
  for (int j = threadIdx.x; j < w; j += NT) {
    double l = nan_lo(bx.pres_lo[j]), h = nan_hi(bx.pres_hi[j]);
    double lo_ = fmax(l, tmp_lo[j]), hi_ = fmin(h, tmp_hi[j]);
    bx.lo[nd[N_CUR] + j] = lo_;
    bx.hi[nd[N_CUR] + j] = hi_;
    if (with_mag) bx.mag[nd[N_CUR] + j] = magnitude(lo_, hi_);
  }
}


// Lay out the box's arrays in a scratch slot (and the pass working set, when the program keeps
// it in global memory).
__device__ __forceinline__ void cta_slot(Box& bx, double*& tmp_lo, double*& tmp_hi, double*& work, const int32_t* hdr,
                                         double* sm, double* slot) {
  const int arena = hdr[H_ARENA], planes_w = hdr[H_PLANES], fold_w = hdr[H_FOLDW], maxw = hdr[H_MAXW];
  bx.lo = slot;
  bx.hi = slot + arena;
  bx.mag = slot + 2 * (size_t)arena;
  bx.planes = slot + 3 * (size_t)arena;
  bx.fold = bx.planes + planes_w;
  bx.pres_lo = bx.fold + fold_w;
  bx.pres_hi = bx.pres_lo + maxw;
  tmp_lo = bx.pres_hi + maxw;
  tmp_hi = tmp_lo + maxw;
  work = hdr[H_PASS_GLOBAL] > 0 ? slot + cta_slot_fixed(hdr) : sm;
}

// Bind a program to this CTA: copy its node records into shared memory (after the pass working
// set; P.nodes then points there) and lay out the box's arrays in the CTA's scratch slot.
// Returns the shared-memory area for the running pass's op records. Every thread calls it; it
// ends with a barrier.
template <int NT>
__device__ __forceinline__ int32_t* cta_bind(DevProgram& P, Box& bx, double*& tmp_lo, double*& tmp_hi, double*& work,
                                             const DevProgram& Pg, double* sm, double* slot) {
  const int32_t* hdr = Pg.hdr;
  // shared memory: [pass working set | node table | op records of the running pass]; a working
  // set too large for shared memory sits at the end of the scratch slot instead
  const int pass_doubles = hdr[H_SMEM] - ((hdr[H_NNODES] * NODE_REC + hdr[H_MAXOPS] * OP_REC + 1) / 2 + 2);
  int32_t* snodes = reinterpret_cast<int32_t*>(sm + pass_doubles);
  __syncthreads();                                   // the previous program's last reads are done
  for (int k = threadIdx.x; k < hdr[H_NNODES] * NODE_REC; k += NT) snodes[k] = __ldg(Pg.nodes + k);
  __syncthreads();
  P = Pg;
  P.nodes = snodes;
  bx.P = &P;
  cta_slot(bx, tmp_lo, tmp_hi, work, hdr, sm, slot);
  return snodes + hdr[H_NNODES] * NODE_REC;
}

// Point the box at box b of wk; with load, copy its input box into the input node's interval.
// Every thread calls it; it ends with a barrier.
template <int NT>
__device__ __forceinline__ void cta_load(Box& bx, const int32_t* hdr, const Work& wk, int64_t b, bool load) {
  const int n = hdr[H_N];
  bx.b = b;
  bx.xL = wk.xL + (size_t)b * n;
  bx.xU = wk.xU + (size_t)b * n;
  int open = 0;
  for (int j = threadIdx.x; j < n; j += NT) {
    const double l = bx.xL[j], h = bx.xU[j];
    if (load) {
      bx.lo[j] = l;
      bx.hi[j] = h;
    }
    open |= box_open(l, h);
  }
  bx.open = __syncthreads_or(open);
}

// Schedule step si of the bound program for the current box (a CROWN pass: ops [op_lo, op_hi)
// and the phases of run_pass). FX: the fold step may read the batch's tensor-core fold vectors
// (Work::fold_ext); a separate instance, so the kernels without it keep their register budget.
template <int NT, bool WHOLE = true, bool IDX = false, bool FX = false>
__device__ __forceinline__ void cta_step(const DevProgram& P, Box& bx, double* tmp_lo, double* tmp_hi, int32_t* sops,
                                         const Work& wk, double* work, int si, int op_lo = 0, int op_hi = 1 << 30,
                                         int phase = 3) {
  const int32_t* hdr = P.hdr;
  const int64_t b = bx.b;
  const int32_t* st = P.steps + si * STEP_REC;
  const int type = st[0], a = st[1];
  switch (type) {
    case ST_FOLD:
      if (FX && wk.fold_ext && !bx.open && *wk.fold_fail == 0) {
        // tensor-core fold vectors of this box (a box with a non-finite centre or radius folds
        // here, as the reference's dense product does)
        const int32_t* nd = node_rec(&P, a);
        const int off = nd[N_FOLD], cnt = 3 * nd[N_W];
        const double* src = wk.fold_ext + (size_t)b * hdr[H_FOLDW] + off;
        for (int j = threadIdx.x; j < cnt; j += NT) bx.fold[off + j] = src[j];
      } else {
        fold_node<NT>(bx, a, work);
      }
      break;
    case ST_IBP: {
      const int32_t* nd = node_rec(&P, a);
      ibp_node<NT>(bx, a, tmp_lo, tmp_hi);
      __syncthreads();
      const bool with_mag = st[2] != 0;
      for (int j = threadIdx.x; j < nd[N_W]; j += NT) {
        bx.lo[nd[N_CUR] + j] = tmp_lo[j];
        bx.hi[nd[N_CUR] + j] = tmp_hi[j];
        if (with_mag) bx.mag[nd[N_CUR] + j] = magnitude(tmp_lo[j], tmp_hi[j]);
      }
      break;
    }
    case ST_MAG: {
      const int32_t* nd = node_rec(&P, a);
      for (int j = threadIdx.x; j < nd[N_W]; j += NT) {
        bx.mag[nd[N_CUR] + j] = magnitude(bx.lo[nd[N_CUR] + j], bx.hi[nd[N_CUR] + j]);
      }
      break;
    }
    case ST_RELAX: relax_node<NT>(bx, a); break;
    case ST_IBPOUT: {
      if (wk.lb_ibp) {
        const int32_t* nd = node_rec(&P, a);
        const int wt = nd[N_W], S = hdr[H_S];
        const double* Cb = wk.C ? wk.C + (size_t)b * S * wt : nullptr;
        for (int s = threadIdx.x; s < S; s += NT)
          wk.lb_ibp[(size_t)b * S + s] = spec_row_lower(Cb, wt, (const double*)bx.lo, (const double*)bx.hi,
                                                        nd[N_CUR], s);
      }
      break;
    }
    case ST_PASS: case ST_FINAL:
      if (WHOLE) run_pass<NT, true, IDX, FX>(bx, a, work, sops, wk);
      else run_pass<NT, false, IDX>(bx, a, work, sops, wk, op_lo, op_hi, phase);
      break;
    case ST_COMPARE: compare_node<NT>(bx, a, tmp_lo, tmp_hi, st[3] != 0); break;
    default: break;
  }
}

// The whole schedule for box b of wk on the bound program.
template <int NT, bool IDX = false, bool FX = false>
__device__ __forceinline__ void cta_box(const DevProgram& P, Box& bx, double* tmp_lo, double* tmp_hi, int32_t* sops,
                                        const Work& wk, int64_t b, double* work) {
  const int nsteps = P.hdr[H_NSTEPS];
  cta_load<NT>(bx, P.hdr, wk, b, true);
  for (int si = 0; si < nsteps; ++si) {
#ifdef GEAR_STEP_PROFILE
    long long t_step = clock64();
#endif
    cta_step<NT, true, IDX, FX>(P, bx, tmp_lo, tmp_hi, sops, wk, work, si);
    __syncthreads();
#ifdef GEAR_STEP_PROFILE
    if (threadIdx.x == 0 && si < 8192) atomicAdd(&g_step_cycles[si], (unsigned long long)(clock64() - t_step));
#endif
  }
}

// GWS: the program keeps its pass working set in global memory (H_PASS_GLOBAL > 0). A separate
// instance per address space keeps the shared-memory one on shared loads and stores. FX: the
// program's fold vectors come from the tensor-core fold (H_FOLD_TC, shared-memory programs only).
template <int NT, bool GWS, bool FX = false>
__global__ void __launch_bounds__(NT, GEAR_CTA_MINB / NT) crown_megakernel(DevProgram Pg, Work wk) {
  extern __shared__ double sm[];
  DevProgram P;
  Box bx;
  double *tmp_lo, *tmp_hi, *work;
  int32_t* sops = cta_bind<NT>(P, bx, tmp_lo, tmp_hi, work, Pg, sm, wk.scratch + (size_t)blockIdx.x * wk.slot_doubles);
  for (int64_t b = blockIdx.x; b < wk.B; b += gridDim.x)
    cta_box<NT, GWS, FX>(P, bx, tmp_lo, tmp_hi, sops, wk, b, GWS ? work : sm);
}

// ------------------------------------------------------------------ the plain (unfused) form
// One schedule step of every box per launch, and within a CROWN pass one launch for its initial
// A, one per op (one node's backward step into one input) and one for its concretisation: the
// unfused baseline the fused kernels are measured against, on the same device code. Each box has
// a scratch slot of its own (its state crosses launches through global memory; the program is
// compiled with its pass working set there). Step -1 loads the boxes.
template <int NT>
__global__ void __launch_bounds__(NT, GEAR_CTA_MINB / NT)
crown_plain_kernel(DevProgram Pg, Work wk, int si, int op_lo, int op_hi, int phase) {
  extern __shared__ double sm[];
  DevProgram P;
  Box bx;
  double *tmp_lo, *tmp_hi, *work;
  int32_t* sops = cta_bind<NT>(P, bx, tmp_lo, tmp_hi, work, Pg, sm, wk.scratch + (size_t)blockIdx.x * wk.slot_doubles);
  for (int64_t b = blockIdx.x; b < wk.B; b += gridDim.x) {
    cta_slot(bx, tmp_lo, tmp_hi, work, Pg.hdr, sm, wk.scratch + (size_t)b * wk.slot_doubles);
    cta_load<NT>(bx, Pg.hdr, wk, b, si < 0);
    if (si >= 0) cta_step<NT, false, true>(P, bx, tmp_lo, tmp_hi, sops, wk, work, si, op_lo, op_hi, phase);
    __syncthreads();
  }
}

// ------------------------------------------------------------------ several programs, one launch
// One instance of a multi-instance launch: its program and its boxes / outputs (the Work's
// scratch fields are unused: the launch's slots are sized for the largest program).
struct MultiItem {
  DevProgram P;
  Work wk;
};

// Index of the instance owning work item g: the last i with start[i] <= g (start ascending,
// start[0] = 0).
__device__ __forceinline__ int multi_owner(const int64_t* start, int count, long long g) {
  int lo = 0, hi = count - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (start[mid] <= g) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Boxes of many instances (different programs and widths) in one persistent launch; every
// program of one launch keeps its pass working set in the same address space (GWS). Work item g
// is box g - start[i] of instance i; CTAs take items from a device counter, so instances of
// uneven cost balance over the SMs (the caller orders them by cost, largest first). A CTA
// rebinds its shared-memory node table only when the instance changes.
template <int NT, bool GWS>
__global__ void __launch_bounds__(NT, GEAR_CTA_MINB / NT)
crown_multi_megakernel(const MultiItem* __restrict__ items, int count, const int64_t* __restrict__ start,
                       unsigned long long* next, double* scratch, int64_t slot_doubles) {
  extern __shared__ double sm[];
  __shared__ long long s_g;
  __shared__ int s_i;
  DevProgram P;
  Box bx;
  double *tmp_lo = nullptr, *tmp_hi = nullptr, *work = nullptr;
  int32_t* sops = nullptr;
  double* slot = scratch + (size_t)blockIdx.x * slot_doubles;
  const long long total = start[count];
  int cur = -1;
  for (;;) {
    if (threadIdx.x == 0) {
      const long long g = (long long)atomicAdd(next, 1ull);
      s_g = g;
      s_i = g < total ? multi_owner(start, count, g) : 0;
    }
    __syncthreads();
    const long long g = s_g;
    const int i = s_i;
    __syncthreads();                                 // s_g, s_i are rewritten by the next fetch
    if (g >= total) break;
    if (i != cur) {
      sops = cta_bind<NT>(P, bx, tmp_lo, tmp_hi, work, items[i].P, sm, slot);
      cur = i;
    }
    cta_box<NT, GWS>(P, bx, tmp_lo, tmp_hi, sops, items[i].wk, g - start[i], GWS ? work : sm);   // Work read in place
  }
}

}  // namespace gear

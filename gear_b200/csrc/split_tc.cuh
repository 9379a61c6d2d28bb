// The final CROWN pass's product through a dense node on the input, on the tensor cores.
//
// In a tensor-core program (H_FOLD_TC) whose final pass ends with the backward step through a
// Linear/MatMul node on the input (op flag OF_SPLIT, set by the program compiler when that op
// is the only one into the input), the product A_x = A_v W of every box is one GEMM over the
// batch, (B S x w) . (w x n): the dense work of BoundLinear.bound_backward
// (operators/linear.py:268, next_A = last_A.matmul(W)). Per box the CROWN kernel would stream
// all of W through the SM for it; here it is split off:
//
//   crown_megakernel<NT, false, true>   every step up to that op; the op writes its A rows
//                                       densely (Work.split_v) and the pass hands each row's
//                                       bias sum, charge sum and interval fallback to this file
//   row_digits_kernel + fold_tc_kernel  the rows cut into int8 digits and multiplied by the
//   (gemv mode, fold_tc.cuh)            digits of W^T on tcgen05: the product and its rigorous
//                                       enclosure radius E_c per entry
//   split_tail_kernel                   the concretisation of run_pass's final pass on the
//                                       product: lb, lbias, lA
//
// Soundness: the product P differs from the exact A_v W by at most E_c entrywise, so every bound
// built from P with the extra charge sum_j E_c,j m_j (m_j = |x_j|'s bound over the box) is a
// bound of the exact one; the plane (P, lbias) stays valid because lbias is taken from that
// widened bound. The charge replaces the float64 rounding charge of the CUDA-core product.
#pragma once
#include "crown_kernel.cuh"
#include "fold_tc.cuh"

namespace gear {

// One warp per (box, row): the tail of run_pass's final pass with A_x = prod (M = B S rows of
// 2 n: the product, then E_c). status: the GEMM's wait flag (nonzero: its product is missing and
// every row falls back to its interval bound, which stays sound).
template <int NT>
__global__ void __launch_bounds__(NT) split_tail_kernel(Work wk, int S, int n, const double* __restrict__ prod,
                                                       const foldtc::BoxStat* __restrict__ rst,
                                                       const int* __restrict__ status) {
  constexpr int NWARP = NT / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const double fbox = ((double)n + 16) * EPS * 4;   // box dot products (run_pass)
  const bool failed = *status != 0;
  const int64_t M = wk.B * S;
  for (int64_t item = (int64_t)blockIdx.x * NWARP + warp; item < M; item += (int64_t)gridDim.x * NWARP) {
    const int64_t b = item / S;
    const double* r = wk.split_rows + item * 3;
    const double* c = prod + item * 2 * n;
    const double* ec = c + n;
    const double* xl = wk.xL + b * n;
    const double* xu = wk.xU + b * n;
    const bool bad0 = failed || wk.split_open[b] != 0 || rst[item].open != 0;
    double bs = 0, dv = 0, be = 0, ech = 0;
    if (!bad0) {
      for (int j = lane; j < n; j += 32) {
        const double a = c[j], l = xl[j], h = xu[j];
        bs += a * ((h + l) / 2.0);
        dv += fabs(a) * ((h - l) / 2.0);
        be += finite_abs(a) * finite_abs(fmax(fabs(l), fabs(h)));
        const double m = magnitude(l, h);
        ech += isinf(m) ? 0.0 : ec[j] * m;
      }
      bs = warp_sum(bs);
      dv = warp_sum(dv);
      be = warp_sum(be);
      ech = warp_sum(ech);
    }
    const double val = r[0] + bs;
    const double er = r[1] + ech + dv + be * fbox;
    double tot = val - (er + (fabs(val) + er) * RE1);
    const bool bad = bad0 || isnan(tot) || tot == INFINITY;
    if (bad) tot = -INFINITY;
    double lbv = bad ? fmax(tot, r[2]) : tot;           // interval fallback (backward_bound.py:826)
    if (wk.lb_ibp) lbv = fmax(lbv, wk.lb_ibp[item]);    // IBP pass of the bounding glue
    if (lane == 0) {
      wk.lb[item] = lbv;
      if (wk.lbias) wk.lbias[item] = bad ? -INFINITY : tot - (bs - dv);
    }
    double* la = wk.lA + item * n;
    for (int j = lane; j < n; j += 32) la[j] = bad ? 0.0 : c[j];
  }
}

}  // namespace gear

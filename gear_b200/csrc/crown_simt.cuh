// CROWN over a batch of boxes, one thread per box ("box-SIMT" megakernel).
// (Included by gear_capi.cu after crown_kernel.cuh; shares its relaxations, IBP elements and
// program format.)
//
// Every thread runs the whole compiled schedule for its own box: plain IBP of every node,
// relaxation planes, every intermediate CROWN pass, compare-with-IBP, the final pass and its
// concretisation -- the same arithmetic as crown_megakernel, in the same order. Per-box state
// (interval arena, planes, fold vectors, the A entry buffers and row arrays of a pass) lives in
// global scratch laid out box-innermost: item i of the box of thread k is at tile[i * T + k], so
// each warp access is one coalesced 256-byte transaction, while every program word (patterns,
// moves, maps, weights) is the same for all 32 threads of a warp and is fetched once as a
// broadcast. There is no shared memory, no barrier and no cross-thread reduction: a warp
// executes 32 independent boxes in lockstep on a uniform control flow.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "crown_kernel.cuh"
#include "gear_program.h"

namespace gear {

constexpr int SIMT_T = 64;   // boxes (threads) per CTA tile

// box-interleaved view of one box's scratch: element i at p[i * SIMT_T]
struct SView {
  double* p;
  __device__ __forceinline__ double& operator[](int64_t i) const { return p[i * SIMT_T]; }
  __device__ __forceinline__ SView operator+(int64_t off) const { return SView{p + off * SIMT_T}; }
};

struct SBox {
  const DevProgram* P;
  SView lo, hi, mag, planes, fold, pres_lo, pres_hi, tmp_lo, tmp_hi, buf, rows;
  int64_t b;
  int open;        // some input coordinate has a non-finite centre or radius (box_open)
};

__device__ __forceinline__ int64_t simt_items(const int32_t* hdr) {
  return 3 * (int64_t)hdr[H_ARENA] + hdr[H_PLANES] + hdr[H_FOLDW] + 4 * (int64_t)hdr[H_MAXW] + hdr[H_SIMT_BUF] +
         hdr[H_SIMT_ROWS];
}

// -------------------------------------------------------------- IBP / fold / relax per box
__device__ void simt_ibp_node(const SBox& bx, int v, SView olo, SView ohi) {
  const DevProgram* P = bx.P;
  const int32_t* nd = node_rec(P, v);
  const int kind = nd[N_KIND], w = nd[N_W];
  if (kind == NK_LINEAR || kind == NK_MATMUL) {
    const int win = nd[N_WIN];
    const double* bias = nd[N_B_OFF] >= 0 ? P->dp + nd[N_B_OFF] : nullptr;
    if (nd[N_FOLD] >= 0) {
      SView f = bx.fold + nd[N_FOLD];
      for (int j = 0; j < w; ++j) {
        double bb = bias ? __ldg(bias + j) : 0.0;
        double l = f[j] - f[w + j], h = f[j] + f[w + j];
        l = l + bb;
        h = h + bb;
        double err = rounding_error(f[2 * w + j] + fabs(bb), win);
        olo[j] = nan_lo(widen(l, err, -1));
        ohi[j] = nan_hi(widen(h, err, 1));
      }
      return;
    }
    const double* W = P->dp + nd[N_W_OFF];
    const int32_t* a = node_rec(P, nd[N_IN0]);
    for (int j = 0; j < w; ++j) {
      const double* Wr = W + (int64_t)j * win;
      double center = 0, dev = 0, mag = 0, slo = 0, shi = 0;
      int nonfin = 0;
      for (int i = 0; i < win; ++i) {
        double wv = __ldg(Wr + i);
        double l = bx.lo[a[N_CUR] + i], h = bx.hi[a[N_CUR] + i];
        nonfin |= !(isfinite(l) && isfinite(h));
        center += ((l + h) / 2) * wv;
        dev += ((h - l) / 2) * fabs(wv);
        mag += finite_abs(fmax(fabs(l), fabs(h))) * fabs(wv);
        double pl_ = wv > 0 ? wv * l : (wv < 0 ? wv * h : 0.0);
        double ph_ = wv > 0 ? wv * h : (wv < 0 ? wv * l : 0.0);
        slo += isnan(pl_) ? -INFINITY : pl_;
        shi += isnan(ph_) ? INFINITY : ph_;
      }
      double l = nonfin ? slo : center - dev;
      double h = nonfin ? shi : center + dev;
      double bb = bias ? __ldg(bias + j) : 0.0;
      l = l + bb;
      h = h + bb;
      double err = rounding_error(mag + fabs(bb), win);
      olo[j] = nan_lo(widen(l, err, -1));
      ohi[j] = nan_hi(widen(h, err, 1));
    }
    return;
  }
  for (int j = 0; j < w; ++j) {
    double l, h;
    ibp_element_t<SView>(P, bx.lo, bx.hi, nd, j, &l, &h);
    olo[j] = l;
    ohi[j] = h;
  }
}

__device__ void simt_fold_node(const SBox& bx, int v) {
  // the input node's interval sits at arena offset 0: the box itself, box-interleaved. JB
  // outputs per sweep over the box, so the box is read w / JB times instead of w times.
  const DevProgram* P = bx.P;
  const int32_t* nd = node_rec(P, v);
  const int w = nd[N_W], win = nd[N_WIN];
  const double* W = P->dp + nd[N_W_OFF];
  SView f = bx.fold + nd[N_FOLD];
  constexpr int JB = 8;
  for (int j0 = 0; j0 < w; j0 += JB) {
    const int jn = min(JB, w - j0);
    double c[JB], r[JB], t[JB];
#pragma unroll
    for (int q = 0; q < JB; ++q) { c[q] = 0.0; r[q] = 0.0; t[q] = 0.0; }
    for (int i = 0; i < win; ++i) {
      const double l = bx.lo[i], h = bx.hi[i];
      const double xc = (h + l) / 2.0, xr = (h - l) / 2.0, xm = finite_abs(fmax(fabs(l), fabs(h)));
#pragma unroll
      for (int q = 0; q < JB; ++q) {
        if (q < jn) {
          const double wv = __ldg(W + (int64_t)(j0 + q) * win + i), aw = fabs(wv);
          c[q] += xc * wv;
          r[q] += xr * aw;
          t[q] += xm * aw;
        }
      }
    }
    for (int q = 0; q < jn; ++q) {
      f[j0 + q] = c[q];
      f[w + j0 + q] = r[q];
      f[2 * w + j0 + q] = t[q];
    }
  }
}

__device__ void simt_relax_node(const SBox& bx, int v) {
  const DevProgram* P = bx.P;
  const int32_t* nd = node_rec(P, v);
  const int kind = nd[N_KIND], w = nd[N_W];
  SView pl = bx.planes + nd[N_PLANE];
  const double* T = P->dp + P->hdr[H_SINOFF];
  const int32_t* a = node_rec(P, nd[N_IN0]);
  // the undefined-side stop needs the node's own interval NaN-free and not inverted everywhere
  bool stop_ok = true;
  if (kind != NK_MUL)
    for (int j = 0; j < w; ++j) {
      const double lo_v = bx.lo[nd[N_CUR] + j], hi_v = bx.hi[nd[N_CUR] + j];
      if (isnan(lo_v) || isnan(hi_v) || lo_v > hi_v) stop_ok = false;
    }
  for (int j = 0; j < w; ++j) {
    double q[6];
    if (kind == NK_MUL) {
      const int32_t* c = node_rec(P, nd[N_IN1]);
      int i0 = __ldg(P->ip + nd[N_MAP0] + j), i1 = __ldg(P->ip + nd[N_MAP1] + j);
      double xl = bx.lo[a[N_CUR] + i0], xu = bx.hi[a[N_CUR] + i0];
      double yl = bx.lo[c[N_CUR] + i1], yu = bx.hi[c[N_CUR] + i1];
      if (!(isfinite(xl) && isfinite(xu) && isfinite(yl) && isfinite(yu))) {
        for (int k = 0; k < 6; ++k) q[k] = NAN;
      } else {
        relax_mul(xl, xu, yl, yu, q, P->hdr[H_TIES]);
      }
      for (int k = 0; k < 6; ++k) pl[6 * j + k] = q[k];
    } else {
      double l = bx.lo[a[N_CUR] + j], u = bx.hi[a[N_CUR] + j];
      if (kind == NK_POW) {
        // bound_backward raises the input's stored upper bound to lower + 1e-8 (persistent)
        u = fmax(u, l + 1e-8);
        bx.hi[a[N_CUR] + j] = u;
        bx.mag[a[N_CUR] + j] = magnitude(l, u);
        if ((int)P->dp[nd[N_CVEC] + 1] == POW_FRAC) l = fmax(l, 0.0);
      }
      bool bad = !(isfinite(l) && isfinite(u));
      if (kind == NK_LOG) bad = bad || !(l > 0);
      const bool off = kind == NK_POW && !(u >= 0 || (int)P->dp[nd[N_CVEC] + 1] != POW_FRAC);
      if (bad || off) {
        if (stop_ok && !off) undefined_stop(kind, l, u, bx.lo[nd[N_CUR] + j], bx.hi[nd[N_CUR] + j], q);
        else q[0] = q[1] = q[2] = q[3] = NAN;
      } else if (kind == NK_SQR) relax_sqr(l, u, q);
      else if (kind == NK_EXP) relax_exp(l, u, q);
      else if (kind == NK_LOG) relax_log(l, u, q);
      else if (kind == NK_SIN) relax_sin(T, l, u, q);
      else if (kind == NK_COS) relax_cos(T, l, u, q);
      else relax_pow(P, nd, l, u, q);
      for (int k = 0; k < 4; ++k) pl[4 * j + k] = q[k];
    }
  }
}

// -------------------------------------------------------------- one CROWN pass per box
__device__ void simt_run_pass(const SBox& bx, int pid, const Work& wk, bool live) {
  const DevProgram* P = bx.P;
  const int32_t* pr = P->passes + pid * PASS_REC;
  const int S = pr[P_S], sides = pr[P_SIDES], smem = pr[P_SMEM];
  const int n = P->hdr[H_N];
  const int t = pr[P_T];
  const int32_t* tnd = node_rec(P, t);
  const double fbias = ((double)max(pr[P_NVISIT], 1) + n + 16) * EPS * 4;
  const double fbox = ((double)n + 16) * EPS * 4;
  auto row = [&](int side, int what) { return bx.rows + ((int64_t)side * R_COUNT + what) * S; };
  auto vals = [&](int side, int off) { return bx.buf + ((int64_t)side * smem + off); };
  for (int k = 0; k < sides * R_COUNT * S; ++k) bx.rows[k] = 0.0;
  {
    const int32_t* trp = P->ip + pr[P_TRP];
    const int nnz_t = __ldg(trp + S);
    for (int side = 0; side < sides; ++side) {
      SView V = vals(side, pr[P_TBUF]);
      if (pr[P_INIT] == 0) {
        for (int k = 0; k < nnz_t; ++k) V[k] = 1.0;
      } else {
        const double* Cb = wk.C + (size_t)bx.b * S * tnd[N_W];
        for (int k = 0; k < nnz_t; ++k) V[k] = Cb[k];
      }
    }
  }
  const int op0 = pr[P_OP0], nop = pr[P_NOP];
#ifdef GEAR_STEP_PROFILE
  long long t_op = clock64();
#endif
  for (int oi = 0; oi < nop; ++oi) {
#ifdef GEAR_STEP_PROFILE
    if (oi > 0 && threadIdx.x == 0) {
      long long t1 = clock64();
      atomicAdd(&g_op_cycles[op0 + oi - 1], (unsigned long long)(t1 - t_op));
      t_op = t1;
    }
#endif
    const int32_t* op = P->ops + (size_t)(op0 + oi) * OP_REC;
    const int kind = op[O_KIND], v = op[O_V], slot = op[O_SLOT];
    const int32_t* vnd = node_rec(P, v);
    const int32_t* vrp = P->ip + op[O_VRP];
    const int32_t* vcols = P->ip + op[O_VCOLS];
    const bool has_pl = vnd[N_PLANE] >= 0;
    SView pl = has_pl ? bx.planes + vnd[N_PLANE] : bx.planes;
    const bool relax = (kind == NK_SQR || kind == NK_EXP || kind == NK_LOG || kind == NK_SIN || kind == NK_COS ||
                        kind == NK_POW);
    const int ppe = kind == NK_MUL ? 6 : 4;
    const int u = op[O_U];
    const int32_t* und = u >= 0 ? node_rec(P, u) : nullptr;
    const bool first = op[O_FIRST] != 0;
    const bool zero_u = !op[O_FOLD] && !op[O_UMERGE];
    const int uk = op[O_UK];
    const double gmerge = uk >= 2 ? gamma_k((double)uk) : 0.0;
    const bool need_a = first && (relax || kind == NK_MUL || kind == NK_MULC || kind == NK_ADD || kind == NK_SUB ||
                                  kind == NK_ADDC || kind == NK_SUBC || kind == NK_RSUBC ||
                                  ((kind == NK_LINEAR) && vnd[N_B_OFF] >= 0));
    const double* cvec = vnd[N_CVEC] >= 0 ? P->dp + vnd[N_CVEC] : nullptr;
    const int32_t* map0 = vnd[N_MAP0] >= 0 ? P->ip + vnd[N_MAP0] : nullptr;
    const int32_t* map1 = vnd[N_MAP1] >= 0 ? P->ip + vnd[N_MAP1] : nullptr;
    const int32_t* inex = vnd[N_INEXACT] >= 0 ? P->ip + vnd[N_INEXACT] : nullptr;
    SView m0 = bx.mag + node_rec(P, vnd[N_IN0])[N_CUR];
    const bool two = (kind == NK_ADD || kind == NK_SUB);
    SView m1 = bx.mag + (two ? node_rec(P, vnd[N_IN1])[N_CUR] : 0);
    const double* bvec = (kind == NK_LINEAR && vnd[N_B_OFF] >= 0) ? P->dp + vnd[N_B_OFF] : nullptr;
    const bool dense = op[O_DENSE] != 0 && !op[O_FOLD];
    for (int side = 0; side < sides; ++side) {
      SView V = vals(side, op[O_VBUF]);
      SView rval = row(side, R_VAL), rerr = row(side, R_ERR);
      if (op[O_SINGLE] & (OF_FUSED | OF_FUSED_T)) {
        // an entry-wise op: each entry's bias terms and its move (u's entry e <- v's entry e, or
        // tgt[e] with OF_FUSED_T) in one sweep, in the order and with the arithmetic of the sweeps
        // below (same bits); with OF_FUSED u needs no clearing (its entries are the moved ones)
        SView U = vals(side, op[O_UBUF]);
        const int32_t* ucols = P->ip + op[O_UCOLS];
        const int32_t* tgt = P->ip + op[O_TGT];
        const bool tmap = (op[O_SINGLE] & OF_FUSED_T) != 0;
        SView mu = bx.mag + und[N_CUR];
        if (tmap && zero_u) {
          const int nnz_u = op[O_UNNZ];
          for (int k = 0; k < nnz_u; ++k) U[k] = 0.0;
        }
        for (int s = 0; s < S; ++s) {
          const int e0 = __ldg(vrp + s), e1 = __ldg(vrp + s + 1);
          if (e0 == e1) continue;
          double sb = 0, sm_ = 0, sc = 0, pmerge = 0;
          int und_ = 0;
          for (int e = e0; e < e1; ++e) {
            const double a = V[e];
            const int c = __ldg(vcols + e);
            double na;
            if (relax || kind == NK_MUL) {
              double p[6];
              for (int k = 0; k < ppe; ++k) p[k] = pl[ppe * c + k];
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
              if (need_a && __ldg(inex + c) && a != 0.0) {
                const double m = m0[__ldg(map0 + c)];
                sc += isinf(m) ? (__fma_rn(a, cv, -(a * cv)) != 0.0 ? INFINITY : 0.0) : UNIT * (fabs(a * cv) * m);
              }
            } else {
              double bt;
              na = elem_coef(kind, slot, side, a, nullptr, cvec ? __ldg(cvec + c) : 0.0, &bt);
              if (need_a) {
                const double mx = m0[__ldg(map0 + c)];
                const double my = two ? m1[__ldg(map1 + c)] : fabs(__ldg(cvec + c));
                const double e_ = rounding_error(mx + my, 2);
                const double fa = finite_abs(a);
                sc += fa > 0 ? (isinf(e_) ? 0.0 : fa * e_) : 0.0;
                if (kind == NK_ADDC || kind == NK_SUBC || kind == NK_RSUBC) {
                  const double cv = kind == NK_SUBC ? -__ldg(cvec + c) : __ldg(cvec + c);
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
              const double m = mu[__ldg(ucols + ti)];
              pmerge += isinf(m) ? (merge_rounded(old, acc, tot) ? INFINITY : 0.0) : fabs(acc) * m;
            }
          }
          if (need_a) {
            rval[s] = und_ ? NAN : rval[s] + sb;
            rerr[s] += sm_ * fbias + sc;
          }
          if (uk >= 2) rerr[s] += gmerge * pmerge;
        }
        continue;
      }
      // ---- bias, bias magnitude, charges and undefined flags (v's rows)
      if (need_a) {
        for (int s = 0; s < S; ++s) {
          const int e0 = __ldg(vrp + s), e1 = __ldg(vrp + s + 1);
          if (e0 == e1) continue;
          double sb = 0, sm_ = 0, sc = 0;
          int und_ = 0;
          for (int e = e0; e < e1; ++e) {
            double a = V[e];
            int c = __ldg(vcols + e);
            if (relax || kind == NK_MUL) {
              double p[6];
              for (int k = 0; k < ppe; ++k) p[k] = pl[ppe * c + k];
              double bt;
              double na = elem_coef(kind, 0, side, a, p, 0.0, &bt);
              double bt2 = 0.0, nb = 0.0;
              if (kind == NK_MUL) nb = elem_coef(kind, 1, side, a, p, 0.0, &bt2);
              if (a != 0.0 && (!isfinite(bt) || !isfinite(na) || !isfinite(nb))) und_ = 1;
              if (isfinite(bt)) { sb += bt; sm_ += fabs(bt); }
            } else if (kind == NK_MULC) {
              double cv = __ldg(cvec + c);
              if (__ldg(inex + c) && a != 0.0) {
                double m = m0[__ldg(map0 + c)];
                sc += isinf(m) ? (__fma_rn(a, cv, -(a * cv)) != 0.0 ? INFINITY : 0.0) : UNIT * (fabs(a * cv) * m);
              }
            } else if (kind == NK_LINEAR) {
              double bb = __ldg(bvec + c);
              sb += a * bb;
              sm_ += fabs(a) * fabs(bb);
            } else {
              double mx = m0[__ldg(map0 + c)];
              double my = two ? m1[__ldg(map1 + c)] : fabs(__ldg(cvec + c));
              double e_ = rounding_error(mx + my, 2);
              double fa = finite_abs(a);
              sc += fa > 0 ? (isinf(e_) ? 0.0 : fa * e_) : 0.0;
              if (kind == NK_ADDC || kind == NK_SUBC || kind == NK_RSUBC) {
                double cv = kind == NK_SUBC ? -__ldg(cvec + c) : __ldg(cvec + c);
                sb += a * cv;
                sm_ += fabs(a) * fabs(cv);
              }
            }
          }
          rval[s] = und_ ? NAN : rval[s] + sb;
          rerr[s] += sm_ * fbias + sc;
        }
      }
      if (op[O_FOLD]) {
        // linear/matmul on the input, one entry per row: exact fold into the concretisation
        SView f = bx.fold + vnd[N_FOLD];
        const int w = vnd[N_W];
        const double gk = gamma_k((double)op[O_WOUT]);
        for (int s = 0; s < S; ++s) {
          const int e0 = __ldg(vrp + s), e1 = __ldg(vrp + s + 1);
          if (e0 == e1) continue;
          double a = V[e0];
          int c = __ldg(vcols + e0);
          rval[s] += a * f[c];
          rerr[s] += fabs(a) * f[w + c] + (fabs(a) * f[2 * w + c]) * fbox + gk * (fabs(a) * f[2 * w + c]);
        }
        continue;
      }
      SView U = vals(side, op[O_UBUF]);
      const int32_t* urp = P->ip + op[O_URP];
      const int32_t* ucols = P->ip + op[O_UCOLS];
      SView mu = bx.mag + und[N_CUR];
      if (zero_u) {
        const int nnz_u = op[O_UNNZ];
        for (int k = 0; k < nnz_u; ++k) U[k] = 0.0;
      }
      if (dense) {
        // GEMV of this box's row: U[s, :] += sum_e V[e] W[c_e, :], JB output columns per sweep of
        // the row's entries (the weights are the same for every box of the warp: broadcasts)
        const double* W = P->dp + vnd[N_W_OFF];
        const int win = vnd[N_WIN];
        const double gk = gamma_k((double)op[O_WOUT]);
        constexpr int JB = 8;
        for (int s = 0; s < S; ++s) {
          const int e0 = __ldg(vrp + s), e1 = __ldg(vrp + s + 1);
          if (e0 == e1) continue;
          SView Ur = U + __ldg(urp + s);
          double part = 0, pmerge = 0;
          for (int j0 = 0; j0 < win; j0 += JB) {
            const int jn = min(JB, win - j0);
            double acc[JB], ab[JB];
#pragma unroll
            for (int q = 0; q < JB; ++q) { acc[q] = 0.0; ab[q] = 0.0; }
            for (int e = e0; e < e1; ++e) {
              const double a = V[e], fa = fabs(a);
              const double* Wr = W + (int64_t)__ldg(vcols + e) * win + j0;
              if (jn == JB) {
#pragma unroll
                for (int q = 0; q < JB; ++q) {
                  const double wv = __ldg(Wr + q);
                  acc[q] += a * wv;
                  ab[q] += fa * fabs(wv);
                }
              } else {
                for (int q = 0; q < jn; ++q) {
                  const double wv = __ldg(Wr + q);
                  acc[q] += a * wv;
                  ab[q] += fa * fabs(wv);
                }
              }
            }
            double uq[JB], mq[JB];
#pragma unroll
            for (int q = 0; q < JB; ++q) {
              uq[q] = q < jn ? Ur[j0 + q] : 0.0;
              mq[q] = q < jn ? mu[j0 + q] : 0.0;
            }
#pragma unroll
            for (int q = 0; q < JB; ++q) {
              if (q >= jn) continue;
              Ur[j0 + q] = uq[q] + acc[q];
              const double mf = isinf(mq[q]) ? 0.0 : mq[q];
              part += ab[q] * mf;
              pmerge += fabs(acc[q]) * mf;
            }
          }
          rerr[s] += gk * part + gmerge * pmerge;
        }
        continue;
      }
      // pull moves, row by row (targets of row s pull sources of row s)
      const int32_t* tptr = P->ip + op[O_TPTR];
      const int32_t* tgt = P->ip + op[O_TGT];
      const int32_t* sptr = P->ip + op[O_SPTR];
      const int32_t* src = P->ip + op[O_SRC];
      const bool single = (op[O_SINGLE] & OF_SINGLE) != 0;
      for (int s = 0; s < S; ++s) {
        const int k0 = __ldg(tptr + s), k1 = __ldg(tptr + s + 1);
        if (k0 == k1) continue;
        double pmerge = 0;
        for (int k = k0; k < k1; ++k) {
          double acc = 0;
          const int q0 = single ? k : __ldg(sptr + k), q1 = single ? k + 1 : __ldg(sptr + k + 1);
          for (int q = q0; q < q1; ++q) {
            int e = __ldg(src + q);
            double a = V[e];
            int c = __ldg(vcols + e);
            double p[6];
            if (has_pl) for (int kk = 0; kk < ppe; ++kk) p[kk] = pl[ppe * c + kk];
            double bt;
            double na = elem_coef(kind, slot, side, a, has_pl ? p : nullptr, cvec ? __ldg(cvec + c) : 0.0, &bt);
            if (!isfinite(na)) na = 0.0;
            acc += na;
          }
          int ti = __ldg(tgt + k);
          const double old = U[ti];
          const double tot = old + acc;
          U[ti] = tot;
          if (uk >= 2 && acc != 0.0) {
            double m = mu[__ldg(ucols + ti)];
            pmerge += isinf(m) ? (merge_rounded(old, acc, tot) ? INFINITY : 0.0) : fabs(acc) * m;
          }
        }
        if (uk >= 2) rerr[s] += gmerge * pmerge;
      }
    }
  }
#ifdef GEAR_STEP_PROFILE
  if (nop > 0 && threadIdx.x == 0) {
    long long t1 = clock64();
    atomicAdd(&g_op_cycles[op0 + nop - 1], (unsigned long long)(t1 - t_op));
    t_op = t1;
  }
#endif
  // ---- concretisation at the input
  const bool fold = pr[P_NFOLD] != 0;
  const int xnnz = pr[P_XNNZ];
  const int32_t* xrp = (!fold && xnnz > 0) ? P->ip + pr[P_XRP] : nullptr;
  const int32_t* xcols = (!fold && xnnz > 0) ? P->ip + pr[P_XCOLS] : nullptr;
  if (xrp) {
    for (int side = 0; side < sides; ++side) {
      SView V = vals(side, pr[P_XBUF]);
      const double sign = side == 0 ? -1.0 : 1.0;
      SView rval = row(side, R_VAL), rerr = row(side, R_ERR), rroot = row(side, R_ROOT);
      for (int s = 0; s < S; ++s) {
        const int e0 = __ldg(xrp + s), e1 = __ldg(xrp + s + 1);
        double bs = 0, dv = 0, be = 0;
        // 4 entries per step: loads issued before the sums
        for (int e = e0; e < e1; e += 4) {
          int cq[4];
          double aq[4], lq[4], hq[4];
#pragma unroll
          for (int q = 0; q < 4; ++q) cq[q] = e + q < e1 ? __ldg(xcols + e + q) : 0;
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            aq[q] = e + q < e1 ? V[e + q] : 0.0;
            lq[q] = e + q < e1 ? bx.lo[cq[q]] : 0.0;
            hq[q] = e + q < e1 ? bx.hi[cq[q]] : 0.0;
          }
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            if (e + q >= e1) continue;
            const double a = aq[q], l = lq[q], h = hq[q];
            bs += a * ((h + l) / 2.0);
            dv += fabs(a) * ((h - l) / 2.0);
            be += finite_abs(a) * finite_abs(fmax(fabs(l), fabs(h)));
          }
        }
        rval[s] += bs;
        rerr[s] += dv + be * fbox;
        rroot[s] = bs + sign * dv;
      }
    }
  }
#ifdef GEAR_STEP_PROFILE
  if (threadIdx.x == 0) atomicAdd(&g_op_cycles[8190], (unsigned long long)(clock64() - t_op));
#endif
  const bool final = pr[P_FINAL] != 0;
  const int n_ = n;
  for (int side = 0; side < sides; ++side) {
    const double sign = side == 0 ? -1.0 : 1.0;
    SView rval = row(side, R_VAL), rerr = row(side, R_ERR), rroot = row(side, R_ROOT);
    for (int s = 0; s < S; ++s) {
      double val = rval[s], er = rerr[s];
      double tot = val + sign * (er + (fabs(val) + er) * RE1);
      const bool bad = bx.open || isnan(tot) || tot == -sign * INFINITY;
      if (bad) tot = sign * INFINITY;
      if (final) {
        double lbv = tot;
        if (bad) {
          double fb = 0;
          if (pr[P_INIT] == 0) fb = bx.lo[tnd[N_CUR] + s];
          else {
            const int wt = tnd[N_W];
            const double* Cb = wk.C + ((size_t)bx.b * S + s) * wt;
            for (int c = 0; c < wt; ++c) {
              double cv = Cb[c];
              fb += cv > 0 ? cv * bx.lo[tnd[N_CUR] + c] : (cv < 0 ? cv * bx.hi[tnd[N_CUR] + c] : 0.0);
            }
          }
          lbv = fmax(lbv, fb);
        }
        if (wk.lb_ibp) lbv = fmax(lbv, wk.lb_ibp[(size_t)bx.b * S + s]);   // IBP pass of the bounding glue
        if (live && side == 0) {
          wk.lb[(size_t)bx.b * S + s] = lbv;
          if (wk.lbias) wk.lbias[(size_t)bx.b * S + s] = bad ? -INFINITY : tot - rroot[s];
          if (wk.lA) {
            // the row of lA: the input's entries, zeros elsewhere (and all zero for a bad row)
            double* la = wk.lA + ((size_t)bx.b * S + s) * n_;
            int e = xrp ? __ldg(xrp + s) : 0;
            const int e1 = xrp ? __ldg(xrp + s + 1) : 0;
            SView V = vals(0, xrp ? pr[P_XBUF] : 0);
            for (int c = 0; c < n_; ++c) {
              double a = 0.0;
              if (e < e1 && __ldg(xcols + e) == c) { a = bad ? 0.0 : V[e]; ++e; }
              la[c] = a;
            }
          }
        }
      } else {
        (side == 0 ? bx.pres_lo : bx.pres_hi)[s] = tot;
      }
    }
  }
}

// Lay out the box-interleaved views of one program in this CTA's scratch region.
__device__ __forceinline__ void simt_bind(SBox& bx, const DevProgram* Pg, double* cta_base) {
  const int32_t* hdr = Pg->hdr;
  const int arena = hdr[H_ARENA], maxw = hdr[H_MAXW];
  double* tile = cta_base + threadIdx.x;
  bx.P = Pg;
  int64_t o = 0;
  bx.lo = SView{tile + o * SIMT_T}; o += arena;
  bx.hi = SView{tile + o * SIMT_T}; o += arena;
  bx.mag = SView{tile + o * SIMT_T}; o += arena;
  bx.planes = SView{tile + o * SIMT_T}; o += hdr[H_PLANES];
  bx.fold = SView{tile + o * SIMT_T}; o += hdr[H_FOLDW];
  bx.pres_lo = SView{tile + o * SIMT_T}; o += maxw;
  bx.pres_hi = SView{tile + o * SIMT_T}; o += maxw;
  bx.tmp_lo = SView{tile + o * SIMT_T}; o += maxw;
  bx.tmp_hi = SView{tile + o * SIMT_T}; o += maxw;
  bx.buf = SView{tile + o * SIMT_T}; o += hdr[H_SIMT_BUF];
  bx.rows = SView{tile + o * SIMT_T};
}

// Tile ti (boxes ti*SIMT_T ...) of wk: the whole schedule, one box per thread.
__device__ __forceinline__ void simt_tile(SBox& bx, const Work& wk, int64_t ti, double* cta_base) {
  const DevProgram& Pg = *bx.P;
  const int32_t* hdr = Pg.hdr;
  const int arena = hdr[H_ARENA], n = hdr[H_N];
  const int nsteps = hdr[H_NSTEPS];
  const int64_t b_real = ti * SIMT_T + threadIdx.x;
  const bool live = b_real < wk.B;
  const int64_t b = live ? b_real : wk.B - 1;   // a tail thread repeats the last box, writes nothing
  bx.b = b;
  // the tile's input boxes are consecutive rows of (B, n): read them coalesced, write them
  // box-interleaved into the input node's interval slots (arena offset 0)
  __syncthreads();
  {
    const int64_t b0 = ti * SIMT_T;
    const int nb = (int)min((int64_t)SIMT_T, wk.B - b0);
    double* base = cta_base;
    for (int k = threadIdx.x; k < SIMT_T * n; k += SIMT_T) {
      const int bb = k / n, j = k - bb * n;
      const int64_t src = (b0 + min(bb, nb - 1)) * n + j;
      base[(int64_t)j * SIMT_T + bb] = wk.xL[src];
      base[((int64_t)arena + j) * SIMT_T + bb] = wk.xU[src];
    }
  }
  __syncthreads();
  bx.open = 0;
  for (int j = 0; j < n; ++j) bx.open |= box_open(bx.lo[j], bx.hi[j]);
  for (int si = 0; si < nsteps; ++si) {
#ifdef GEAR_STEP_PROFILE
    long long t_step = clock64();
#endif
    const int32_t* st = Pg.steps + si * STEP_REC;
    const int type = st[0], a = st[1];
    switch (type) {
      case ST_FOLD: simt_fold_node(bx, a); break;
      case ST_IBP: {
        const int32_t* nd = node_rec(&Pg, a);
        simt_ibp_node(bx, a, bx.tmp_lo, bx.tmp_hi);
        const bool with_mag = st[2] != 0;
        for (int j = 0; j < nd[N_W]; ++j) {
          double l = bx.tmp_lo[j], h = bx.tmp_hi[j];
          bx.lo[nd[N_CUR] + j] = l;
          bx.hi[nd[N_CUR] + j] = h;
          if (with_mag) bx.mag[nd[N_CUR] + j] = magnitude(l, h);
        }
        break;
      }
      case ST_MAG: {
        const int32_t* nd = node_rec(&Pg, a);
        for (int j = 0; j < nd[N_W]; ++j) bx.mag[nd[N_CUR] + j] = magnitude(bx.lo[nd[N_CUR] + j], bx.hi[nd[N_CUR] + j]);
        break;
      }
      case ST_RELAX: simt_relax_node(bx, a); break;
      case ST_IBPOUT: {
        if (wk.lb_ibp && live) {
          const int32_t* nd = node_rec(&Pg, a);
          const int wt = nd[N_W], S = hdr[H_S];
          const double* Cb = wk.C ? wk.C + (size_t)b * S * wt : nullptr;
          for (int s = 0; s < S; ++s)
            wk.lb_ibp[(size_t)b * S + s] = spec_row_lower(Cb, wt, bx.lo, bx.hi, nd[N_CUR], s);
        }
        break;
      }
      case ST_PASS: case ST_FINAL: simt_run_pass(bx, a, wk, live); break;
      case ST_COMPARE: {
        const int32_t* nd = node_rec(&Pg, a);
        simt_ibp_node(bx, a, bx.tmp_lo, bx.tmp_hi);
        const bool with_mag = st[3] != 0;
        for (int j = 0; j < nd[N_W]; ++j) {
          double l = nan_lo(bx.pres_lo[j]), h = nan_hi(bx.pres_hi[j]);
          double lo_ = fmax(l, bx.tmp_lo[j]), hi_ = fmin(h, bx.tmp_hi[j]);
          bx.lo[nd[N_CUR] + j] = lo_;
          bx.hi[nd[N_CUR] + j] = hi_;
          if (with_mag) bx.mag[nd[N_CUR] + j] = magnitude(lo_, hi_);
        }
        break;
      }
      default: break;
    }
#ifdef GEAR_STEP_PROFILE
    if (threadIdx.x == 0 && si < 8192) atomicAdd(&g_step_cycles[si], (unsigned long long)(clock64() - t_step));
#endif
  }
}

__global__ void __launch_bounds__(SIMT_T, 8) crown_simt_kernel(DevProgram Pg, Work wk) {
  const int64_t items = simt_items(Pg.hdr);
  const int64_t ntiles = (wk.B + SIMT_T - 1) / SIMT_T;
  double* cta_base = wk.scratch + (size_t)blockIdx.x * items * SIMT_T;
  SBox bx;
  simt_bind(bx, &Pg, cta_base);
  for (int64_t ti = blockIdx.x; ti < ntiles; ti += gridDim.x) simt_tile(bx, wk, ti, cta_base);
}

// Tiles of many instances in one persistent launch (work item g: tile g - start[i] of instance
// i, taken from a device counter; slots sized for the largest program).
__global__ void __launch_bounds__(SIMT_T, 8)
crown_multi_simt_kernel(const MultiItem* __restrict__ items, int count, const int64_t* __restrict__ start,
                        unsigned long long* next, double* scratch, int64_t slot_doubles) {
  __shared__ long long s_g;
  __shared__ int s_i;
  double* cta_base = scratch + (size_t)blockIdx.x * slot_doubles;
  const long long total = start[count];
  int cur = -1;
  SBox bx;
  for (;;) {
    if (threadIdx.x == 0) {
      const long long g = (long long)atomicAdd(next, 1ull);
      s_g = g;
      s_i = g < total ? multi_owner(start, count, g) : 0;
    }
    __syncthreads();
    const long long g = s_g;
    const int i = s_i;
    __syncthreads();
    if (g >= total) break;
    if (i != cur) {
      simt_bind(bx, &items[i].P, cta_base);          // program and Work read in place
      cur = i;
    }
    simt_tile(bx, items[i].wk, g - start[i], cta_base);
  }
}

}  // namespace gear

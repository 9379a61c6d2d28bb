// Device-resident branch-and-bound queue and one BaB iteration with device-side counts.
// (Included by gear_capi.cu, the single translation unit of libgear_b200.so.)
//
// The queue holds every open domain in slot arrays (box lo/hi, keys, insertion ids) and keeps an
// active slot list in the reference's pop order (objective key descending, insertion id
// ascending; branching_domains.py:831-962, 1171 with a stable sort), a free slot list and its
// counters in device memory. Every step of an iteration -- pop of the list's tail, prune of the
// bounded batch (get_remaining_index, branching_domains.py:412-558), SB branch
// (branching_heuristics.py:25-202), midpoint split (split.py:26-122), child keys
// (batch_branch_and_bound.py:189-225), sort of the children and merge into the active list --
// reads its sizes from these counters, so an iteration is a fixed sequence of launches with
// fixed arguments: no host read, and it can be captured once into a CUDA graph and replayed.
// A batch that finds fewer open domains than its size is padded with copies of its first box
// (their bounds are computed and ignored).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "bab_kernels.cuh"

namespace gear {
namespace bq {

using bab::BT;

// counters (int64, device)
// C_OVERFLOW: iterations whose children did not fit the free slots (nothing pushed; the caller
// keeps the capacity above 2 x batch per iteration, so this stays 0)
enum Counter { C_ACTIVE = 0, C_FREE, C_NEXT_ID, C_BOUNDED, C_POPPED, C_KEPT_TOTAL, C_ITER, C_OVERFLOW, C_COUNT = 8 };

struct QueueDev {
  int n, S;
  int64_t cap;
  double* lo;          // (cap, n)
  double* hi;          // (cap, n)
  double* key;         // (cap, S)
  double* key0;        // (cap) objective key (sort key)
  int64_t* ids;        // (cap) insertion ids
  int32_t* active;     // (cap) ordered open slots
  int32_t* merged;     // (cap) merge output
  int32_t* free_list;  // (cap)
  int64_t* counters;   // C_COUNT
  unsigned long long* disc_min;   // ordered bits of the smallest threshold of a discarded domain
  double* root_lo;     // (n) box used when the queue is empty
  double* root_hi;
};

// the popped batch: rows [0, b) are the tail of the active list (b = min(B, open)), rows
// [b, B) repeat row 0 (or the root box when nothing is open). One thread per (row, coordinate).
__global__ void pop_gather_kernel(QueueDev q, int64_t B, double* plo, double* phi, int32_t* pslot) {
  const int64_t t = (int64_t)blockIdx.x * BT + threadIdx.x;
  if (t >= B * q.n) return;
  const int64_t na = q.counters[C_ACTIVE];
  const int64_t b = na < B ? na : B;
  const int64_t r = t / q.n;
  const int j = (int)(t - r * q.n);
  if (b == 0) {
    plo[t] = q.root_lo[j];
    phi[t] = q.root_hi[j];
    if (j == 0) pslot[r] = -1;
    return;
  }
  const int32_t slot = q.active[na - b + (r < b ? r : 0)];
  plo[t] = q.lo[(int64_t)slot * q.n + j];
  phi[t] = q.hi[(int64_t)slot * q.n + j];
  if (j == 0) pslot[r] = r < b ? slot : -1;
}

// after the gather: popped slots go to the free list, the active list shrinks by b
__global__ void pop_commit_kernel(QueueDev q, int64_t B, const int32_t* pslot) {
  const int64_t na = q.counters[C_ACTIVE];
  const int64_t b = na < B ? na : B;
  const int64_t nf = q.counters[C_FREE];
  for (int64_t r = threadIdx.x; r < b; r += BT) q.free_list[nf + r] = pslot[r];
  __syncthreads();
  if (threadIdx.x == 0) {
    q.counters[C_ACTIVE] = na - b;
    q.counters[C_FREE] = nf + b;
    q.counters[C_POPPED] = b;
    q.counters[C_BOUNDED] += b;
    if (b > 0) q.counters[C_ITER] += 1;
  }
}

// thresholds of the popped rows: row 0 the incumbent (device scalar), rows 1.. the constraint
// right-hand sides
__global__ void thresholds_kernel(const double* incumbent, const double* rhs, int64_t B, int S, double* thr) {
  const int64_t t = (int64_t)blockIdx.x * BT + threadIdx.x;
  if (t >= B * S) return;
  const int s = (int)(t % S);
  thr[t] = s == 0 ? *incumbent : rhs[s - 1];
}

// keep[r] = 0 for the padding rows r >= b
__global__ void mask_padding_kernel(const int64_t* counters, int64_t B, uint8_t* keep) {
  const int64_t r = (int64_t)blockIdx.x * BT + threadIdx.x;
  if (r < B && r >= counters[C_POPPED]) keep[r] = 0;
}

// children of the K = *nk kept parents (grid sized for K = B): child k < K the upper half of
// parent kept[k], child K + k its lower half (split_kernel with a device-side count)
__global__ void split_dev_kernel(const double* lo, const double* hi, const int32_t* kept, const int32_t* nk, int n,
                                 const int32_t* split_idx, double* clo, double* chi) {
  const int64_t K = *nk;
  const int64_t t = (int64_t)blockIdx.x * BT + threadIdx.x;
  if (t >= 2 * K * n) return;
  const int64_t child = t / n;
  const int j = (int)(t - child * n);
  const int part = child < K ? 0 : 1;
  const int64_t p = kept[part == 0 ? child : child - K];
  double l = lo[p * n + j], u = hi[p * n + j];
  if (j == split_idx[p]) {
    const double nl = ((part + 1) * l + (2 - part - 1) * u) / 2;
    const double nu = (part * l + (2 - part) * u) / 2;
    l = nl;
    u = nu;
  }
  clo[child * n + j] = l;
  chi[child * n + j] = u;
}

// child keys (child_keys_kernel with a device-side count): one warp per child
__global__ void child_keys_dev_kernel(const double* lb, const double* lA, const double* lbias, const double* clo,
                                      const double* chi, const int32_t* kept, const int32_t* nk, int S, int n,
                                      double* ckey) {
  const int64_t K = *nk;
  const int64_t warp = ((int64_t)blockIdx.x * BT + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= 2 * K) return;
  const int64_t child = warp;
  const int64_t p = kept[child < K ? child : child - K];
  const double* xl = clo + child * n;
  const double* xu = chi + child * n;
  const double* a = lA + (p * S) * (int64_t)n;   // objective row 0
  double pm = 0, mg = 0;
  bool ok = true;
  for (int j = lane; j < n; j += 32) {
    const double c = (xl[j] + xu[j]) / 2, r = (xu[j] - xl[j]) / 2;
    pm += a[j] * c - fabs(a[j]) * r;
    mg += fabs(a[j]) * (fabs(c) + r);
    ok = ok && (xl[j] <= xu[j]);
  }
  for (int o = 16; o > 0; o >>= 1) {
    pm += __shfl_xor_sync(0xffffffffu, pm, o);
    mg += __shfl_xor_sync(0xffffffffu, mg, o);
  }
  ok = __all_sync(0xffffffffu, ok);
  if (lane == 0) {
    const double bb = lbias[p * S];
    const double plane = pm + bb;
    const double margin = (n + 4) * (2.220446049250313e-16 / 2) * (mg + fabs(bb));
    const double pmin = bab::next_down(plane - margin);
    const double k0 = lb[p * S];
    const bool usable = ok && isfinite(pmin);
    ckey[child * S] = usable ? fmax(k0, pmin) : k0;
  }
  for (int s = 1 + lane; s < S; s += 32) ckey[child * S + s] = lb[p * S + s];
}

// domains to push: mult x *nk (the 2K children of K kept parents, or a caller's count), or 0
// (and an overflow count) when the free slots cannot take them
__global__ void push_plan_kernel(QueueDev q, const int32_t* nk, int mult, int32_t* nchild) {
  const int64_t m = mult * (int64_t)(*nk);
  const bool fits = q.counters[C_FREE] >= m;
  *nchild = fits ? (int32_t)m : 0;
  if (!fits) q.counters[C_OVERFLOW] += 1;
}

// the m = *nchild children take the last m free slots: rows, keys, insertion ids; newslot[c] =
// slot for c < m and -1 (sorts last) for the padding up to N2 (grid covers N2 x max(n, S))
__global__ void push_scatter_kernel(QueueDev q, const int32_t* nchild, const double* clo, const double* chi,
                                    const double* ckey, int64_t N2, int32_t* newslot) {
  const int64_t m = *nchild;
  const int64_t nf = q.counters[C_FREE];
  const int64_t base = q.counters[C_NEXT_ID];
  const int w = q.n > q.S ? q.n : q.S;
  const int64_t t = (int64_t)blockIdx.x * BT + threadIdx.x;
  if (t >= N2 * w) return;
  const int64_t c = t / w;
  const int j = (int)(t - c * w);
  if (c >= m) {
    if (j == 0) newslot[c] = -1;
    return;
  }
  const int32_t slot = q.free_list[nf - m + c];
  if (j < q.n) {
    q.lo[(int64_t)slot * q.n + j] = clo[c * q.n + j];
    q.hi[(int64_t)slot * q.n + j] = chi[c * q.n + j];
  }
  if (j < q.S) q.key[(int64_t)slot * q.S + j] = ckey[c * q.S + j];
  if (j == 0) {
    q.ids[slot] = base + c;
    q.key0[slot] = ckey[c * q.S];
    newslot[c] = slot;
  }
}

// merge of the active list (na = counters[C_ACTIVE]) with the sorted children (nb = *nchild)
// into q.merged (merge_kernel with device-side lengths; grid covers the capacity)
__global__ void merge_dev_kernel(QueueDev q, const int32_t* nchild, const int32_t* b) {
  const int64_t na = q.counters[C_ACTIVE], nb = *nchild;
  const int64_t i = (int64_t)blockIdx.x * BT + threadIdx.x;
  if (i >= na + nb) return;
  const double* key = q.key0;
  const int64_t* id = q.ids;
  const int32_t* a = q.active;
  int64_t lo = i > nb ? i - nb : 0, hi = i < na ? i : na;
  while (lo < hi) {
    const int64_t j = (lo + hi) >> 1, k = i - j;
    const int32_t bk = b[k - 1], aj = a[j];
    if (bab::before(key[bk], id[bk], key[aj], id[aj])) hi = j;
    else lo = j + 1;
  }
  const int64_t j = lo, k = i - j;
  bool take_a;
  if (j >= na) take_a = false;
  else if (k >= nb) take_a = true;
  else {
    const int32_t aj = a[j], bk = b[k];
    take_a = bab::before(key[aj], id[aj], key[bk], id[bk]);
  }
  q.merged[i] = take_a ? a[j] : b[k];
}

// the merged list back into the active list
__global__ void merge_copy_kernel(QueueDev q, const int32_t* nchild) {
  const int64_t len = q.counters[C_ACTIVE] + *nchild;
  const int64_t i = (int64_t)blockIdx.x * BT + threadIdx.x;
  if (i < len) q.active[i] = q.merged[i];
}

// the counters after a push: children moved from the free list to the active list
__global__ void push_commit_kernel(QueueDev q, const int32_t* nchild) {
  const int64_t m = *nchild;
  q.counters[C_ACTIVE] += m;
  q.counters[C_FREE] -= m;
  q.counters[C_NEXT_ID] += m;
  q.counters[C_KEPT_TOTAL] += m / 2;
}

__global__ void set_count_kernel(int32_t* dst, int32_t v) { *dst = v; }

// dual bound: min(objective key of the list's tail, smallest discarded threshold)
__global__ void dual_bound_kernel(QueueDev q, double* out) {
  const int64_t na = q.counters[C_ACTIVE];
  const double open = na > 0 ? q.key0[q.active[na - 1]] : INFINITY;
  const double disc = bab::from_ordered_bits(*q.disc_min);
  out[0] = open < disc ? open : disc;
}

}  // namespace bq
}  // namespace gear

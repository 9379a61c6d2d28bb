// Branch-and-bound select / prune / branch / split on the device.
// (Included by gear_capi.cu, the single translation unit of libgear_b200.so.)
//
// Reference semantics (paths relative to solver/complete_verifier/input_split):
//   prune   branching_domains.py:412-558 get_remaining_index (solving mode, check_dm_lbs)
//   branch  branching_heuristics.py:25-56 _compute_sb_score (sb_sum), :59-101
//           input_split_branching (non-finite fallback to the longest edge), :104-125
//           input_split_heuristic_sb (top-1), :176-202 _exhaustive_guard
//   split   split.py:26-122 input_split_parallel (two partitions, no hint): children are
//           [upper halves of every box; lower halves of every box]
//   keys    batch_branch_and_bound.py:189-225 _plane_minimum_down / _raise_child_keys
//   select  branching_domains.py:831-962 pick_out_batch after the sort by lb (:1171):
//           descending lb, the batch popped from the tail; ties by insertion id (stable)
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace gear {
namespace bab {

constexpr int BT = 256;

__device__ __forceinline__ unsigned long long ordered_bits(double v) {
  // monotone map of doubles (no NaN) to unsigned integers
  unsigned long long u = __double_as_longlong(v);
  return (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
}
// the next double toward -inf (finite x), as torch.nextafter(x, -inf)
__device__ __forceinline__ double next_down(double x) {
  if (!isfinite(x)) return x;
  if (x == 0.0) return -4.9406564584124654e-324;
  long long b = __double_as_longlong(x);
  return __longlong_as_double(x > 0 ? b - 1 : b + 1);
}
__device__ __forceinline__ double from_ordered_bits(unsigned long long u) {
  u = (u & 0x8000000000000000ull) ? (u & 0x7fffffffffffffffull) : ~u;
  return __longlong_as_double(u);
}

// keep[b] = domain b is not verified; disc_min = min over verified rows of threshold[:, 0]
__global__ void prune_kernel(const double* lb, const double* thr, int64_t B, int S, uint8_t* keep,
                             unsigned long long* disc_min) {
  __shared__ unsigned long long smin[BT / 32];
  int64_t b = (int64_t)blockIdx.x * BT + threadIdx.x;
  unsigned long long mine = ordered_bits(INFINITY);
  if (b < B) {
    const double* l = lb + b * S;
    const double* t = thr + b * S;
    bool verified = false;
    for (int s = 0; s < S; ++s) {
      bool fin = isfinite(l[s]) && isfinite(t[s]);
      bool gt = fin && (l[s] > t[s]);
      if (s == 0) gt = gt || (fin && l[0] >= t[0]);
      verified = verified || gt;
    }
    if (S > 0 && isinf(l[0]) && l[0] > 0 && isfinite(t[0])) verified = true;
    keep[b] = verified ? 0 : 1;
    if (verified && S > 0 && isfinite(t[0])) mine = ordered_bits(t[0]);
  }
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long other = __shfl_xor_sync(0xffffffffu, mine, o);
    mine = other < mine ? other : mine;
  }
  if ((threadIdx.x & 31) == 0) smin[threadIdx.x >> 5] = mine;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long m = smin[0];
    for (int w = 1; w < BT / 32; ++w) m = smin[w] < m ? smin[w] : m;
    atomicMin(disc_min, m);
  }
}

// flag = 1 if any lA / lb / threshold entry of the batch is non-finite (SB falls back)
__global__ void nonfinite_kernel(const double* lA, int64_t nA, const double* lb, const double* thr, int64_t nS,
                                 int* flag) {
  int64_t i = (int64_t)blockIdx.x * BT + threadIdx.x;
  int64_t stride = (int64_t)gridDim.x * BT;
  int bad = 0;
  for (int64_t k = i; k < nA; k += stride) bad |= !isfinite(lA[k]);
  for (int64_t k = i; k < nS; k += stride) {
    double t = thr[k];
    // +inf thresholds are inactive rows: replaced by the row's lb (branching_heuristics.py:66-71)
    if (isinf(t) && t > 0) t = lb[k];
    bad |= !isfinite(lb[k]) || !isfinite(t);
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1);
}

// one warp per box: argmax of the SB score (lowest index on ties), then the width guard
__global__ void branch_kernel(const double* lA, const double* lo, const double* hi, int64_t B, int S, int n,
                              const double* root_width, double coeff_thresh, double min_width_ratio,
                              const int* nonfinite, int32_t* split_idx) {
  int warp = (blockIdx.x * BT + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (warp >= B) return;
  const int64_t b = warp;
  const double* l = lo + b * n;
  const double* u = hi + b * n;
  const bool naive = *nonfinite != 0;
  double best = -INFINITY;
  int best_i = 0x7fffffff;
  double rel_best = -INFINITY;
  int rel_i = 0x7fffffff;
  for (int j = lane; j < n; j += 32) {
    double width = u[j] - l[j];
    double score;
    if (naive) {
      score = width;
    } else {
      // raw = max(|lA|, thresh) * (u - l) / 2 summed over the specification rows
      const double* a = lA + (b * S) * (int64_t)n + j;
      score = 0;
      for (int s = 0; s < S; ++s) score += fmax(fabs(a[(int64_t)s * n]), coeff_thresh) * width / 2;
    }
    if (score > best || (score == best && j < best_i) || (isnan(best) && !isnan(score))) { best = score; best_i = j; }
    if (root_width) {
      double rw = root_width[j];
      double rel = rw > 0 ? width / fmax(rw, 1e-300) : 0.0;
      if (rel > rel_best || (rel == rel_best && j < rel_i)) { rel_best = rel; rel_i = j; }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    double ob = __shfl_xor_sync(0xffffffffu, best, o);
    int oi = __shfl_xor_sync(0xffffffffu, best_i, o);
    if (ob > best || (ob == best && oi < best_i)) { best = ob; best_i = oi; }
    double rb = __shfl_xor_sync(0xffffffffu, rel_best, o);
    int ri = __shfl_xor_sync(0xffffffffu, rel_i, o);
    if (rb > rel_best || (rb == rel_best && ri < rel_i)) { rel_best = rb; rel_i = ri; }
  }
  if (lane == 0) {
    int idx = best_i == 0x7fffffff ? 0 : best_i;
    if (!naive && root_width && min_width_ratio > 0) {
      double rw = root_width[idx];
      double chosen = rw > 0 ? (u[idx] - l[idx]) / fmax(rw, 1e-300) : 0.0;
      if (chosen < min_width_ratio * rel_best) idx = rel_i;
    }
    split_idx[b] = idx;
  }
}

// children of the kept parents: child k < K is the upper half of parent kept[k],
// child K + k the lower half (split.py:84-99, two partitions)
__global__ void split_kernel(const double* lo, const double* hi, const int32_t* kept, int64_t K, int n,
                             const int32_t* split_idx, double* clo, double* chi) {
  int64_t t = (int64_t)blockIdx.x * BT + threadIdx.x;
  if (t >= 2 * K * n) return;
  int64_t child = t / n;
  int j = (int)(t - child * n);
  int part = child < K ? 0 : 1;
  int64_t k = part == 0 ? child : child - K;
  int64_t p = kept[k];
  double l = lo[p * n + j], u = hi[p * n + j];
  if (j == split_idx[p]) {
    double nl = ((part + 1) * l + (2 - part - 1) * u) / 2;
    double nu = (part * l + (2 - part) * u) / 2;
    l = nl;
    u = nu;
  }
  clo[child * n + j] = l;
  chi[child * n + j] = u;
}

// child keys: parent's lb rows; the objective row raised to the parent's plane minimum over
// the child box (rounded toward -inf), one warp per child
__global__ void child_keys_kernel(const double* lb, const double* lA, const double* lbias, const double* clo,
                                  const double* chi, const int32_t* kept, int64_t K, int S, int n,
                                  double* ckey) {
  int warp = (blockIdx.x * BT + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (warp >= 2 * K) return;
  const int64_t child = warp;
  const int64_t p = kept[child < K ? child : child - K];
  const double* xl = clo + child * n;
  const double* xu = chi + child * n;
  const double* a = lA + (p * S) * (int64_t)n;   // objective row 0
  double pm = 0, mg = 0;
  bool ok = true;
  for (int j = lane; j < n; j += 32) {
    double c = (xl[j] + xu[j]) / 2, r = (xu[j] - xl[j]) / 2;
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
    double bb = lbias[p * S];
    double plane = pm + bb;
    double margin = (n + 4) * (2.220446049250313e-16 / 2) * (mg + fabs(bb));
    double pmin = next_down(plane - margin);
    double k0 = lb[p * S];
    bool usable = ok && isfinite(pmin);
    ckey[child * S] = usable ? fmax(k0, pmin) : k0;
  }
  for (int s = 1 + lane; s < S; s += 32) ckey[child * S + s] = lb[p * S + s];
}

// ---- queue order: bitonic sort of slot indices by (key descending, id ascending)
__device__ __forceinline__ bool before(double ka, int64_t ia, double kb, int64_t ib) {
  return ka > kb || (ka == kb && ia < ib);
}

// The whole bitonic network in one CTA for N2 <= SORT_SMEM_MAX: slots and their keys staged in
// shared memory, every (k, j) stage separated by a barrier; same comparator as bitonic_step.
constexpr int SORT_SMEM_MAX = 8192;
constexpr int SORT_THREADS = 1024;
__global__ void __launch_bounds__(SORT_THREADS) bitonic_smem(int32_t* idx, const double* key, const int64_t* id,
                                                            int N2) {
  extern __shared__ unsigned char sort_sm[];
  double* k_s = reinterpret_cast<double*>(sort_sm);
  int64_t* id_s = reinterpret_cast<int64_t*>(k_s + N2);
  int32_t* ix_s = reinterpret_cast<int32_t*>(id_s + N2);
  for (int i = threadIdx.x; i < N2; i += SORT_THREADS) {
    const int32_t a = idx[i];
    ix_s[i] = a;
    k_s[i] = a >= 0 ? key[a] : 0.0;
    id_s[i] = a >= 0 ? id[a] : 0;
  }
  __syncthreads();
  for (int k = 2; k <= N2; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int t = threadIdx.x; t < (N2 >> 1); t += SORT_THREADS) {
        const int i = (t / j) * 2 * j + (t % j), l = i + j;
        const int32_t a = ix_s[i], b = ix_s[l];
        const bool a_pad = a < 0, b_pad = b < 0;
        const bool a_first = (a_pad || b_pad) ? !a_pad : before(k_s[i], id_s[i], k_s[l], id_s[l]);
        const bool up = (i & k) == 0;
        if (up ? !a_first : a_first) {
          ix_s[i] = b; ix_s[l] = a;
          const double tk = k_s[i]; k_s[i] = k_s[l]; k_s[l] = tk;
          const int64_t ti = id_s[i]; id_s[i] = id_s[l]; id_s[l] = ti;
        }
      }
      __syncthreads();
    }
  }
  for (int i = threadIdx.x; i < N2; i += SORT_THREADS) idx[i] = ix_s[i];
}

// Merge of two slot lists, each ordered by (key descending, id ascending), into one such list:
// output position i takes its element from the co-rank split (merge path) found by binary search,
// so every position is independent. Ids are unique, so the order is total and the result is the
// one a full sort of the union gives.
__global__ void merge_kernel(const double* key, const int64_t* id, const int32_t* a, int64_t na, const int32_t* b,
                             int64_t nb, int32_t* out) {
  const int64_t i = (int64_t)blockIdx.x * BT + threadIdx.x;
  if (i >= na + nb) return;
  // smallest j (elements taken from a among the first i outputs) with b[i-j-1] before a[j]
  int64_t lo = i > nb ? i - nb : 0, hi = i < na ? i : na;
  while (lo < hi) {
    const int64_t j = (lo + hi) >> 1, k = i - j;
    const int32_t bk = b[k - 1], aj = a[j];
    if (before(key[bk], id[bk], key[aj], id[aj])) hi = j;
    else lo = j + 1;
  }
  const int64_t j = lo, k = i - j;
  bool take_a;
  if (j >= na) take_a = false;
  else if (k >= nb) take_a = true;
  else {
    const int32_t aj = a[j], bk = b[k];
    take_a = before(key[aj], id[aj], key[bk], id[bk]);
  }
  out[i] = take_a ? a[j] : b[k];
}

__global__ void bitonic_step(int32_t* idx, const double* key, const int64_t* id, int64_t N2, int64_t N, int j,
                             int k) {
  int64_t i = (int64_t)blockIdx.x * BT + threadIdx.x;
  if (i >= N2) return;
  int64_t l = i ^ j;
  if (l <= i) return;
  int32_t a = idx[i], b = idx[l];
  // padding slots (index >= N) sort last
  bool a_pad = a < 0, b_pad = b < 0;
  bool a_first;
  if (a_pad || b_pad) a_first = !a_pad;
  else a_first = before(key[a], id[a], key[b], id[b]);
  bool up = (i & k) == 0;
  if (up ? !a_first : a_first) {
    idx[i] = b;
    idx[l] = a;
  }
}

// ---- stream compaction of a keep mask into the kept indices (order preserved)
__global__ void count_kernel(const uint8_t* keep, int64_t B, int32_t* block_counts) {
  __shared__ int cnt[BT / 32];
  int64_t i = (int64_t)blockIdx.x * BT + threadIdx.x;
  int k = (i < B) ? keep[i] : 0;
  unsigned m = __ballot_sync(0xffffffffu, k);
  if ((threadIdx.x & 31) == 0) cnt[threadIdx.x >> 5] = __popc(m);
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int w = 0; w < BT / 32; ++w) t += cnt[w];
    block_counts[blockIdx.x] = t;
  }
}

// exclusive scan of the block counts by one block (nblocks <= BT * 64)
__global__ void scan_counts_kernel(int32_t* block_counts, int nblocks, int32_t* total) {
  __shared__ int32_t part[BT];
  int per = (nblocks + BT - 1) / BT;
  int start = threadIdx.x * per;
  int s = 0;
  for (int i = start; i < min(start + per, nblocks); ++i) s += block_counts[i];
  part[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    int run = 0;
    for (int t = 0; t < BT; ++t) { int v = part[t]; part[t] = run; run += v; }
    *total = run;
  }
  __syncthreads();
  int run = part[threadIdx.x];
  for (int i = start; i < min(start + per, nblocks); ++i) { int v = block_counts[i]; block_counts[i] = run; run += v; }
}

__global__ void compact_kernel(const uint8_t* keep, int64_t B, const int32_t* block_offsets, int32_t* kept) {
  __shared__ int wbase[BT / 32];
  int64_t i = (int64_t)blockIdx.x * BT + threadIdx.x;
  int k = (i < B) ? keep[i] : 0;
  unsigned m = __ballot_sync(0xffffffffu, k);
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) wbase[w] = __popc(m);
  __syncthreads();
  if (threadIdx.x == 0) {
    int run = 0;
    for (int t = 0; t < BT / 32; ++t) { int v = wbase[t]; wbase[t] = run; run += v; }
  }
  __syncthreads();
  if (k) kept[block_offsets[blockIdx.x] + wbase[w] + __popc(m & ((1u << lane) - 1))] = (int32_t)i;
}

// dst[r, :] = src[rows[r], :]   and   dst[rows[r], :] = src[r, :]
__global__ void gather_rows_kernel(const double* src, const int32_t* rows, int64_t R, int64_t w, double* dst) {
  int64_t t = (int64_t)blockIdx.x * BT + threadIdx.x;
  if (t >= R * w) return;
  int64_t r = t / w, j = t - r * w;
  dst[t] = src[(int64_t)rows[r] * w + j];
}
__global__ void scatter_rows_kernel(const double* src, const int32_t* rows, int64_t R, int64_t w, double* dst) {
  int64_t t = (int64_t)blockIdx.x * BT + threadIdx.x;
  if (t >= R * w) return;
  int64_t r = t / w, j = t - r * w;
  dst[(int64_t)rows[r] * w + j] = src[t];
}


// ------------------------------------------------------------------ domain clipping
// clip_domains / _clip_main_fn (complete_verifier/input_split/clip.py:138-486), lower planes:
// shrink each box along every coordinate to where each plane lA_s x + lbias_s can still be
// <= thr_s; a box some plane already proves done becomes empty (x_L[0] = next double above
// x_U[0]). One warp per box, lanes over coordinates; the per-row plane minima and their
// rounding bounds sit in shared memory (3 S doubles per warp).
__device__ __forceinline__ double next_up(double x) {
  if (isnan(x) || x == INFINITY) return x;
  if (x == 0.0) return 4.9406564584124654e-324;
  long long b = __double_as_longlong(x);
  return __longlong_as_double(x > 0 ? b + 1 : b - 1);
}
__device__ __forceinline__ double next_dn(double x) { return -next_up(-x); }
constexpr double CLIP_EPS = 2.220446049250313e-16;
constexpr double CLIP_TINY = 2.2250738585072014e-308;

__device__ __forceinline__ double clip_fabs_fin(double v) { return isfinite(v) ? fabs(v) : 0.0; }

__device__ void clip_planes(const double* A, const double* lbias, int S, int n, const double* xl, const double* xu,
                            double* dm, double* dm_err, double* box_err) {
  const int lane = threadIdx.x & 31;
  const double under = (n + 16) * CLIP_TINY * CLIP_EPS;
  for (int s = 0; s < S; ++s) {
    const double* a = A + (int64_t)s * n;
    double ax = 0, ae = 0, mag = 0;
    for (int i = lane; i < n; i += 32) {
      const double l = xl[i], u = xu[i], ai = a[i];
      ax += ai * ((u + l) / 2);
      ae += fabs(ai) * ((u - l) / 2);
      mag += clip_fabs_fin(ai) * clip_fabs_fin(fmax(fabs(l), fabs(u)));
    }
    for (int o = 16; o > 0; o >>= 1) {
      ax += __shfl_xor_sync(0xffffffffu, ax, o);
      ae += __shfl_xor_sync(0xffffffffu, ae, o);
      mag += __shfl_xor_sync(0xffffffffu, mag, o);
    }
    if (lane == 0) {
      const double be = (mag + clip_fabs_fin(lbias[s])) * ((n + 16) * CLIP_EPS * 4);
      dm[s] = ax - ae + lbias[s];
      box_err[s] = be;
      dm_err[s] = be * ((double)(n + 4) / (4.0 * (n + 16))) + under;
    }
  }
  __syncwarp();
}

__global__ void clip_kernel(double* x_L, double* x_U, const double* thr, const double* lA, const double* lbias,
                            const int32_t* parent, int64_t B, int S, int n, int num_iters, uint8_t* nonempty) {
  extern __shared__ double clip_sm[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int64_t b = (int64_t)blockIdx.x * (blockDim.x >> 5) + wid;
  if (b >= B) return;
  double* dm = clip_sm + (size_t)wid * 3 * S;
  double* dm_err = dm + S;
  double* box_err = dm_err + S;
  const int64_t p = parent ? parent[b] : b;
  const double* A = lA + p * S * n;
  const double* t = thr + p * S;
  const double* lb_ = lbias + p * S;
  double* xl = x_L + b * n;
  double* xu = x_U + b * n;
  // boxes with non-finite data stay as they are
  int fin = 1;
  for (int k = lane; k < S * n; k += 32) fin &= isfinite(A[k]) ? 1 : 0;
  for (int s = lane; s < S; s += 32) fin &= ((isfinite(t[s]) || t[s] == INFINITY) && isfinite(lb_[s])) ? 1 : 0;
  fin = __all_sync(0xffffffffu, fin);
  if (fin) {
    clip_planes(A, lb_, S, n, xl, xu, dm, dm_err, box_err);
    const double under = (n + 16) * CLIP_TINY * CLIP_EPS;
    int cert = 0;
    for (int s = lane; s < S; s += 32) cert |= (dm[s] - box_err[s] - under > t[s]) ? 1 : 0;
    cert = __any_sync(0xffffffffu, cert);
    if (cert) {
      if (lane == 0) xl[0] = next_up(xu[0]);
    } else {
      for (int it = 0; it < num_iters; ++it) {
        if (it > 0) clip_planes(A, lb_, S, n, xl, xu, dm, dm_err, box_err);
        for (int i = lane; i < n; i += 32) {
          const double l = xl[i], u = xu[i];
          const double xh = (u + l) / 2, e = (u - l) / 2;
          double nu = u, nl = l;
          for (int s = 0; s < S; ++s) {
            const double ai = A[(int64_t)s * n + i];
            if (!(ai > 0) && !(ai < 0)) continue;
            const double ax = ai * xh, ae = fabs(ai) * e;
            const double cmo = dm[s] - ax + ae;
            const double num = t[s] - cmo;
            const double mag = clip_fabs_fin(t[s]) + clip_fabs_fin(dm[s]) + clip_fabs_fin(ax) + clip_fabs_fin(ae);
            const double err = mag * (4 * CLIP_EPS) + under + dm_err[s];
            const bool f = isfinite(num);
            const double lo_n = f ? num - err : num, hi_n = f ? num + err : num;
            const double ql = lo_n / ai, qh = hi_n / ai;
            if (ai > 0) nu = fmin(nu, next_up(fmax(ql, qh)));
            else nl = fmax(nl, next_dn(fmin(ql, qh)));
          }
          xl[i] = nl;
          xu[i] = nu;
        }
        __syncwarp();
      }
    }
    __syncwarp();
  }
  if (nonempty) {
    int ok = 1;
    for (int i = lane; i < n; i += 32) ok &= (xl[i] <= xu[i]) ? 1 : 0;
    ok = __all_sync(0xffffffffu, ok);
    if (lane == 0) nonempty[b] = ok ? 1 : 0;
  }
}

}  // namespace bab
}  // namespace gear

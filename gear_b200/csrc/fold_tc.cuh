// Tensor-core fold products of dense linear nodes on the input (tcgen05, int8, TMEM accumulators).
//
// A Linear/MatMul node v = W x whose input is the perturbed input needs, per box b, the fold
// vectors c = W x0, r = |W| eps and t = |W| max(|x_L|, |x_U|) (x0, eps: the box's centre and
// radius). Over a batch of boxes these are two GEMMs, (B x K) . (K x w), the dense work of
// BoundLinear.bound_backward / interval_propagate on the input (operators/linear.py:268,
// interval_bound.py). They run here on the 5th-generation tensor cores with exact integer
// arithmetic, by digit slicing (the splitting method of Ozaki, Ogita and Oishi for accurate
// products on low-precision units, in its fixed-point form):
//
//   every row of W and every box row of x0 / eps is scaled by a power of two 2^e with
//   max |.| < 2^e and cut into DIGITS (6) truncated base-128 digits, d_1..d_6 in [-127, 127]
//   (|v| 2^-e = sum_i d_i 128^-i + rest, 0 <= rest < 128^-6, sign carried by every digit);
//   the digit planes are int8 matrices and every digit product d_i e_j is formed exactly by
//   tcgen05.mma.kind::i8 with int32 accumulation in TMEM. Products of equal level i + j share
//   one accumulator (one scale 128^-(i+j)); levels 2..DIGITS+1 are kept (21 of the 36 digit
//   pairs), their int32 sums are combined in float64 and scaled by 2^(e_row + e_box).
//
// Rigorous enclosure. Per input k the dropped terms are the residual products and the digit
// pairs beyond level DIGITS+1; with W^ = |W| 2^-e, X^ = |x| 2^-f (both < 1):
//   |exact - kept| < 128^-6 (W^_k + X^_k) + 128^-7 sum_{i>=2} |d_i,k|,
// and the float64 combination of the 6 level sums errs by at most 5 u sum_k X^_k. Summed over
// k, with the row and box sums taken in upward rounding, this gives E_c (centre) and E_r
// (radius) in absolute terms. The radius handed to the CROWN kernel is r^ + E_r + E_c (upward
// rounding), so the interval [c^ - r', c^ + r'] contains W x0 -/+ |W| eps: every bound built on
// it stays sound. The magnitude vector t (used only to size rounding charges) is replaced by the
// upper bound sum_k |W_k| . max_k max(|x_L|, |x_U|).
//
// Data path (sm_100a): digit planes are staged global -> shared memory with 16-byte cp.async
// into the canonical no-swizzle K-major UMMA layout (8-row x 16-byte core matrices), a 3-stage
// ring; one thread issues the MMAs (M = 128 boxes, N = 64 outputs, K = 32 per instruction) and
// commits them to an mbarrier per stage; the epilogue reads TMEM with tcgen05.ld (one TMEM lane
// per box, warp w owns lanes 32w..32w+31) and writes float64 fold vectors. Every wait is bounded;
// on expiry the CTA sets the status flag, drains its copies, frees its TMEM and returns.
#pragma once
#include <stdint.h>
#include <cuda_runtime.h>

namespace gear {
namespace foldtc {

constexpr int DIGITS = 6;                 // base-128 digits per operand (42 bits)
constexpr int LEVELS = DIGITS;            // i + j = 2 .. DIGITS + 1
constexpr int BM = 128;                   // boxes per tile (TMEM lanes)
constexpr int BN = 64;                    // outputs per tile (TMEM columns per level)
constexpr int BK = 64;                    // inputs per K block (int8: bytes)
constexpr int STAGES = 3;
constexpr int NT = 128;                   // threads per CTA (4 warps: TMEM lanes 0..127)
constexpr int PLANE_A = BM * BK;          // bytes of one box digit plane per stage
constexpr int PLANE_B = BN * BK;          // bytes of one weight digit plane per stage
constexpr int STAGE_BYTES = DIGITS * (PLANE_A + PLANE_B);
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024;   // + 1 KB for aligning the ring
constexpr uint32_t TMEM_COLS = 512;       // LEVELS * BN = 384 columns, allocated as a power of two
static_assert(LEVELS * BN <= (int)TMEM_COLS, "level accumulators exceed the TMEM allocation");
static_assert(SMEM_BYTES + 64 <= 232448, "the stage ring exceeds the opt-in shared memory of a CTA");
constexpr int CORE_SBO = (BK / 16) * 128; // bytes between 8-row groups of a plane
constexpr int CORE_LBO = 128;             // bytes between the two 16-byte K chunks of an MMA step
// instruction descriptor: D int32, A and B signed int8, both K-major, N = BN, M = BM
constexpr uint32_t IDESC = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                           ((uint32_t)(BM >> 4) << 24);
constexpr long long WAIT_LIMIT = 1ll << 25;   // mbarrier polls (~32 ns apart) before a CTA gives up

// Per-box statistics of the digit split (written by box_digits_kernel).
struct BoxStat {
  double norm_c;   // sum_k |x0_k| 2^-ec, rounded up
  double norm_r;   // sum_k eps_k 2^-er, rounded up
  double xm_max;   // max_k max(|x_L|, |x_U|) (finite part)
  int ec, er;      // scale exponents of x0 and eps
  int open;        // a non-finite centre or radius: the CROWN kernel folds this box itself
  int pad;
};

// Digit planes and row statistics of one dense node (built once per program).
struct NodeDigits {
  const int8_t* wd;      // DIGITS planes of signed digits of W, each (n_pad x k_pad), row-major
  const int8_t* wa;      // DIGITS planes of |digits| (|W|)
  int64_t plane;         // n_pad * k_pad
  const int* we;         // row exponents
  const double* wnorm;   // sum_k |W_k| 2^-e, rounded up
  const double* wdelta;  // sum_k sum_{i>=2} |d_i,k| (exact)
  int w, k_pad, n_pad, fold_off;
};

struct BatchDigits {
  const int8_t* xc;      // DIGITS planes of box centre digits, each (b_pad x k_pad)
  const int8_t* xr;      // DIGITS planes of box radius digits
  int64_t plane;         // b_pad * k_pad
  const BoxStat* st;
  double* fold;          // (B, fold_w) fold vectors out
  int64_t fold_w;
  int64_t B;
  int* status;           // set to 1 when a bounded wait expired
  // 0: the fold (two products per tile). 1: one product, the rows of xc against W^T of a dense
  // node (the final pass's A_v W, split_tc.cuh): fold[n] = the product, fold[w + n] its
  // enclosure radius E_c (0 for an all-zero row, whose product is exact)
  int gemv = 0;
};

// ------------------------------------------------------------------ digit split
// Truncated base-128 digits of |v| 2^-e (< 1), each carrying the sign of v when sgn: every step
// (scaling by 128, floor, subtraction) is exact in float64.
__device__ __forceinline__ void split_digits(double v, int e, bool sgn, int (&d)[DIGITS]) {
  double t = ldexp(fabs(v), -e);
  const bool neg = sgn && v < 0;
#pragma unroll
  for (int i = 0; i < DIGITS; ++i) {
    t = t * 128.0;
    const double f = floor(t);
    t = t - f;
    d[i] = neg ? -(int)f : (int)f;
  }
}

__device__ __forceinline__ int scale_exp(double mx) {
  int e = 0;
  if (mx > 0) frexp(mx, &e);        // mx = m 2^e, m in [0.5, 1): every |v| <= mx < 2^e
  return e;
}

template <class T, class Op>
__device__ __forceinline__ T block_reduce(T v, Op op, T* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = op(v, __shfl_xor_sync(0xffffffffu, v, o));
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  T r = red[0];
  for (int w = 1; w < (int)(blockDim.x >> 5); ++w) r = op(r, red[w]);
  return r;
}

// One row n of W (w x K, row-major) -> digit planes, exponent and row sums. Grid: n_pad rows.
__global__ void __launch_bounds__(NT) w_digits_kernel(const double* __restrict__ W, int w, int K, NodeDigits nd,
                                                      int8_t* wd, int8_t* wa, int* we, double* wnorm,
                                                      double* wdelta) {
  __shared__ double redd[NT / 32];
  __shared__ long long redl[NT / 32];
  const int n = blockIdx.x;
  const bool row = n < w;
  double mx = 0;
  if (row)
    for (int k = threadIdx.x; k < K; k += NT) mx = fmax(mx, fabs(W[(size_t)n * K + k]));
  mx = block_reduce(mx, [](double a, double b) { return fmax(a, b); }, redd);
  const int e = scale_exp(mx);
  double s = 0;
  long long dl = 0;
  for (int k = threadIdx.x; k < nd.k_pad; k += NT) {
    const double v = (row && k < K) ? W[(size_t)n * K + k] : 0.0;
    int d[DIGITS];
    split_digits(v, e, true, d);
#pragma unroll
    for (int i = 0; i < DIGITS; ++i) {
      wd[i * nd.plane + (size_t)n * nd.k_pad + k] = (int8_t)d[i];
      wa[i * nd.plane + (size_t)n * nd.k_pad + k] = (int8_t)abs(d[i]);
      if (i > 0) dl += abs(d[i]);
    }
    s = __dadd_ru(s, ldexp(fabs(v), -e));
  }
  s = block_reduce(s, [](double a, double b) { return __dadd_ru(a, b); }, redd);
  dl = block_reduce(dl, [](long long a, long long b) { return a + b; }, redl);
  if (threadIdx.x == 0) {
    we[n] = e;
    wnorm[n] = s;
    wdelta[n] = (double)dl;
  }
}

// One box b -> centre and radius digit planes and its statistics. Grid: b_pad boxes.
__global__ void __launch_bounds__(NT) box_digits_kernel(const double* __restrict__ xL, const double* __restrict__ xU,
                                                        int64_t B, int K, int k_pad, int8_t* xc, int8_t* xr,
                                                        int64_t plane, BoxStat* st) {
  __shared__ double redd[NT / 32];
  __shared__ int redi[NT / 32];
  const int64_t b = blockIdx.x;
  const bool row = b < B;
  double mc = 0, mr = 0, mm = 0;
  int bad = 0;
  if (row)
    for (int k = threadIdx.x; k < K; k += NT) {
      const double l = xL[b * K + k], h = xU[b * K + k];
      const double c = (h + l) / 2.0, r = (h - l) / 2.0;
      bad |= !(isfinite(c) && isfinite(r));
      mc = fmax(mc, fabs(c));
      mr = fmax(mr, fabs(r));
      const double m = fmax(fabs(l), fabs(h));
      mm = fmax(mm, isfinite(m) ? m : 0.0);
    }
  auto fmaxop = [](double a, double c) { return fmax(a, c); };
  mc = block_reduce(mc, fmaxop, redd);
  mr = block_reduce(mr, fmaxop, redd);
  mm = block_reduce(mm, fmaxop, redd);
  bad = block_reduce(bad, [](int a, int c) { return a | c; }, redi);
  const int ec = bad ? 0 : scale_exp(mc), er = bad ? 0 : scale_exp(mr);
  double sc = 0, sr = 0;
  for (int k = threadIdx.x; k < k_pad; k += NT) {
    double c = 0, r = 0;
    if (row && !bad && k < K) {
      const double l = xL[b * K + k], h = xU[b * K + k];
      c = (h + l) / 2.0;
      r = (h - l) / 2.0;
    }
    int dc[DIGITS], dr[DIGITS];
    split_digits(c, ec, true, dc);
    split_digits(r, er, false, dr);
#pragma unroll
    for (int i = 0; i < DIGITS; ++i) {
      xc[i * plane + b * k_pad + k] = (int8_t)dc[i];
      xr[i * plane + b * k_pad + k] = (int8_t)dr[i];
    }
    sc = __dadd_ru(sc, ldexp(fabs(c), -ec));
    sr = __dadd_ru(sr, ldexp(fabs(r), -er));
  }
  auto addru = [](double a, double c) { return __dadd_ru(a, c); };
  sc = block_reduce(sc, addru, redd);
  sr = block_reduce(sr, addru, redd);
  if (threadIdx.x == 0 && row) {
    BoxStat s;
    s.norm_c = sc;
    s.norm_r = sr;
    s.xm_max = mm;
    s.ec = ec;
    s.er = er;
    s.open = bad;
    s.pad = 0;
    st[b] = s;
  }
}

// One row m of V (M x K, row-major) -> signed digit planes and the row statistics (norm_c, ec;
// open when an entry is not finite). Grid: m_pad rows.
__global__ void __launch_bounds__(NT) row_digits_kernel(const double* __restrict__ V, int64_t M, int K, int k_pad,
                                                        int8_t* xc, int64_t plane, BoxStat* st) {
  __shared__ double redd[NT / 32];
  __shared__ int redi[NT / 32];
  const int64_t m = blockIdx.x;
  const bool row = m < M;
  double mc = 0;
  int bad = 0;
  if (row)
    for (int k = threadIdx.x; k < K; k += NT) {
      const double c = V[m * K + k];
      bad |= !isfinite(c);
      mc = fmax(mc, fabs(c));
    }
  mc = block_reduce(mc, [](double a, double c) { return fmax(a, c); }, redd);
  bad = block_reduce(bad, [](int a, int c) { return a | c; }, redi);
  const int ec = bad ? 0 : scale_exp(mc);
  double sc = 0;
  for (int k = threadIdx.x; k < k_pad; k += NT) {
    const double c = (row && !bad && k < K) ? V[m * K + k] : 0.0;
    int dc[DIGITS];
    split_digits(c, ec, true, dc);
#pragma unroll
    for (int i = 0; i < DIGITS; ++i) xc[i * plane + m * k_pad + k] = (int8_t)dc[i];
    sc = __dadd_ru(sc, ldexp(fabs(c), -ec));
  }
  sc = block_reduce(sc, [](double a, double c) { return __dadd_ru(a, c); }, redd);
  if (threadIdx.x == 0 && row) {
    BoxStat s;
    s.norm_c = sc;
    s.norm_r = 0;
    s.xm_max = 0;
    s.ec = ec;
    s.er = 0;
    s.open = bad;
    s.pad = 0;
    st[m] = s;
  }
}

// ------------------------------------------------------------------ tcgen05 helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Non-blocking polls of an mbarrier phase (test_wait: each poll returns at once, so the bound is
// a bound in time: WAIT_LIMIT polls, ~1 s).
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (long long i = 0; i < WAIT_LIMIT; ++i) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
    __nanosleep(32);
  }
  return false;
}

// shared-memory matrix descriptor: canonical K-major layout without swizzle
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
  return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)(CORE_LBO >> 4) << 16) |
         ((uint64_t)(CORE_SBO >> 4) << 32) | (1ull << 46);
}

__device__ __forceinline__ void mma_i8(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(IDESC), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, int32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// |exact - kept| of one fold product over K inputs, relative to 2^(e_row + e_box), rounded up
__device__ __forceinline__ double split_error(double wnorm, double xnorm, double wdelta) {
  constexpr double R_D = 1.0 / (double)(1ull << (7 * DIGITS));     // 128^-DIGITS, exact
  const double t1 = __dmul_ru(__dadd_ru(wnorm, xnorm), R_D);        // 128^-D (sum W^ + sum X^)
  const double t2 = __dmul_ru(wdelta, R_D / 128.0);                 // 128^-(D+1) sum |d_i>=2|
  const double t3 = __dmul_ru(xnorm, (LEVELS + 1) * 0x1p-53);       // float64 combination of the levels
  return __dadd_ru(__dadd_ru(t1, t2), t3);
}

// ------------------------------------------------------------------ the GEMM
// Grid: (n_pad / BN, b_pad / BM). Two products per tile: op 0 = signed W digits x centre digits
// (c), op 1 = |W| digits x radius digits (r, then t from the row and box statistics); with
// bt.gemv only op 0, and its enclosure radius.
__global__ void __launch_bounds__(NT, 1) fold_tc_kernel(NodeDigits nd, BatchDigits bt) {
  extern __shared__ uint8_t dyn_smem[];
  __shared__ __align__(8) uint64_t mbar[STAGES];
  __shared__ uint32_t tmem_holder;
  uint8_t* ring = (uint8_t*)(((uintptr_t)dyn_smem + 1023) & ~(uintptr_t)1023);
  const uint32_t ring_u32 = smem_u32(ring);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int n0 = blockIdx.x * BN;
  const int64_t m0 = (int64_t)blockIdx.y * BM;
  const int KB = nd.k_pad / BK;
  const int T = bt.gemv ? KB : 2 * KB;

  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&mbar[s])), "r"(1) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_holder)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_holder;

  auto load_stage = [&](int it) {
    const int op = it / KB, kb = it % KB;
    const uint32_t sb = ring_u32 + (it % STAGES) * STAGE_BYTES;
    const int8_t* X = op ? bt.xr : bt.xc;
    const int8_t* Wp = op ? nd.wa : nd.wd;
    for (int q = tid; q < DIGITS * BM * 4; q += NT) {
      const int j = q / (BM * 4), rem = q - j * (BM * 4), r = rem >> 2, c = rem & 3;
      const int8_t* src = X + j * bt.plane + (m0 + r) * nd.k_pad + kb * BK + c * 16;
      cp_async16(sb + j * PLANE_A + (r >> 3) * CORE_SBO + c * CORE_LBO + (r & 7) * 16, src);
    }
    for (int q = tid; q < DIGITS * BN * 4; q += NT) {
      const int i = q / (BN * 4), rem = q - i * (BN * 4), r = rem >> 2, c = rem & 3;
      const int8_t* src = Wp + i * nd.plane + (int64_t)(n0 + r) * nd.k_pad + kb * BK + c * 16;
      cp_async16(sb + DIGITS * PLANE_A + i * PLANE_B + (r >> 3) * CORE_SBO + c * CORE_LBO + (r & 7) * 16, src);
    }
  };

  bool ok = true;
  load_stage(0);
  cp_async_commit();
  load_stage(1);          // T >= 2
  cp_async_commit();
  for (int it = 0; it < T && ok; ++it) {
    const int st = it % STAGES, op = it / KB, kb = it % KB;
    if (it + 2 < T) {
      // the stage of it + 2 was read by the MMAs of it - 1
      if (it >= 1) ok = mbar_wait(smem_u32(&mbar[(it - 1) % STAGES]), ((it - 1) / STAGES) & 1);
      if (__syncthreads_or(!ok)) { ok = false; break; }
      load_stage(it + 2);
    }
    cp_async_commit();
    cp_async_wait<2>();
    fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      const uint32_t a0 = ring_u32 + st * STAGE_BYTES, b0 = a0 + DIGITS * PLANE_A;
#pragma unroll
      for (int ks = 0; ks < BK / 32; ++ks) {
#pragma unroll
        for (int i = 1; i <= DIGITS; ++i) {
#pragma unroll
          for (int j = 1; j <= DIGITS + 1 - i; ++j) {
            const int level = i + j - 2;
            const uint32_t acc = (kb == 0 && ks == 0 && i == 1) ? 0u : 1u;
            mma_i8(tmem + level * BN, smem_desc(a0 + (j - 1) * PLANE_A + ks * 2 * CORE_LBO),
                   smem_desc(b0 + (i - 1) * PLANE_B + ks * 2 * CORE_LBO), acc);
          }
        }
      }
      mma_commit(smem_u32(&mbar[st]));
    }
    if (kb == KB - 1) {
      // epilogue of this product: wait for its last MMAs, read the level sums from TMEM
      ok = mbar_wait(smem_u32(&mbar[st]), (it / STAGES) & 1);
      if (__syncthreads_or(!ok)) { ok = false; break; }
      tc_fence_after();
      const int64_t b = m0 + warp * 32 + lane;
      BoxStat bs;
      if (b < bt.B) bs = bt.st[b];
      else { bs.norm_c = bs.norm_r = bs.xm_max = 0; bs.ec = bs.er = 0; bs.open = 1; }
      const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
      for (int q = 0; q < BN / 16; ++q) {
        double acc[16];
#pragma unroll
        for (int c = 0; c < 16; ++c) acc[c] = 0.0;
        for (int lv = LEVELS - 1; lv >= 0; --lv) {      // smallest scale first
          int32_t v[16];
          tmem_ld16(lane_base + lv * BN + q * 16, v);
          const double sc = ldexp(1.0, -7 * (lv + 2));
#pragma unroll
          for (int c = 0; c < 16; ++c) acc[c] = acc[c] + (double)v[c] * sc;
        }
        if (b >= bt.B || bs.open) continue;
        double* out = bt.fold + b * bt.fold_w + nd.fold_off;
#pragma unroll 4
        for (int c = 0; c < 16; ++c) {
          const int n = n0 + q * 16 + c;
          if (n >= nd.w) break;
          const int en = nd.we[n];
          if (op == 0) {
            out[n] = ldexp(acc[c], en + bs.ec);
            if (bt.gemv)
              out[nd.w + n] = bs.norm_c == 0 ? 0.0 : ldexp(split_error(nd.wnorm[n], bs.norm_c, nd.wdelta[n]), en + bs.ec);
          } else {
            const double wn = nd.wnorm[n], wdl = nd.wdelta[n];
            const double e_c = ldexp(split_error(wn, bs.norm_c, wdl), en + bs.ec);
            const double e_r = ldexp(split_error(wn, bs.norm_r, wdl), en + bs.er);
            const double r = ldexp(acc[c], en + bs.er);
            out[nd.w + n] = __dadd_ru(__dadd_ru(r, e_r), e_c);
            out[2 * nd.w + n] = __dmul_ru(ldexp(wn, en), bs.xm_max);
          }
        }
      }
      tc_fence_before();
      __syncthreads();           // every TMEM read is done before the next product overwrites it
    }
  }
  if (!ok && tid == 0 && bt.status) atomicExch(bt.status, 1);
  cp_async_wait<0>();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
  }
}

}  // namespace foldtc
}  // namespace gear

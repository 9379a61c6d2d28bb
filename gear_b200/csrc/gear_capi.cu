// C ABI of libgear_b200.so: program upload, workspace sizing, megakernel launch.
// Declarations and the reference interfaces they replace: include/gear_b200.h.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/gear_b200.h"
#include "crown_kernel.cuh"
#include "crown_simt.cuh"
#include "bab_kernels.cuh"
#include "concretize_kernels.cuh"
#include "dual_kernels.cuh"
#include "fold_tc.cuh"
#include "split_tc.cuh"
#include "bab_queue.cuh"

namespace {
thread_local std::string g_err;
thread_local int g_launches = 0;

int fail(int code, const char* fmt, const char* detail = "") {
  char buf[512];
  snprintf(buf, sizeof(buf), fmt, detail);
  g_err = buf;
  return code;
}
int cuda_fail(cudaError_t e, const char* what) {
  int code = (e == cudaErrorMemoryAllocation) ? GEAR_E_NOMEM : GEAR_E_CUDA;
  std::string m = std::string(what) + ": " + cudaGetErrorString(e);
  g_err = m;
  return code;
}
}  // namespace

struct gear_dag {
  gear::DevProgram P;
  void* dev = nullptr;
  int32_t hdr[gear::HEADER_LEN];
  int64_t slot_doubles = 0;
  int smem_bytes = 0;
  int device = 0;
  int num_sms = 0;
  int blocks_per_sm = 0;
  int mode = 0;           // gear::ExecMode
  int threads = 0;        // threads per CTA
  int64_t boxes_per_slot = 1;
  std::vector<int32_t> steps;    // host copies of the step and pass records (the plain form's
  std::vector<int32_t> passes;   // launch sequence)
  // tensor-core fold (H_FOLD_TC): digit planes and row statistics of the dense nodes on the
  // input, in one device block; the box digit planes of a batch live in the caller's workspace
  void* tc_dev = nullptr;
  std::vector<gear::foldtc::NodeDigits> tc_nodes;
  int tc_k_pad = 0;
  // the final pass's product through a dense node on the input on the tensor cores (OF_SPLIT
  // op): digit planes of that node's W^T (n x w), in a device block of their own
  bool split = false;
  void* split_dev = nullptr;
  gear::foldtc::NodeDigits split_nd{};
  int split_k = 0;        // w: the node's outputs (the product's inner dimension)
};

namespace {
constexpr int64_t kAlign = 256;
inline int64_t align_up(int64_t v, int64_t a) { return (v + a - 1) / a * a; }

// Workspace of the tensor-core fold for a batch, after the CTA slots: fold vectors (B, fold_w),
// box statistics, centre and radius digit planes (b_pad x k_pad each), the status flag.
struct TcLayout {
  int64_t fold, stats, xc, xr, flag, total, b_pad, plane;
};
TcLayout tc_layout(const gear_dag* d, int64_t batch, int64_t base) {
  using namespace gear::foldtc;
  TcLayout L{};
  L.b_pad = align_up(batch, BM);
  L.plane = L.b_pad * d->tc_k_pad;
  int64_t o = align_up(base, kAlign);
  L.fold = o;  o = align_up(o + batch * d->hdr[gear::H_FOLDW] * (int64_t)sizeof(double), kAlign);
  L.stats = o; o = align_up(o + L.b_pad * (int64_t)sizeof(BoxStat), kAlign);
  L.xc = o;    o = align_up(o + DIGITS * L.plane, kAlign);
  L.xr = o;    o = align_up(o + DIGITS * L.plane, kAlign);
  L.flag = o;  o = align_up(o + (int64_t)sizeof(int), kAlign);
  L.total = o;
  return L;
}

// Workspace of the tensor-core product of the final pass (after the fold's): the dense A rows
// (M = B S rows of split_k), per row bias / charge / fallback, per box open flags, row
// statistics, digit planes (m_pad x k_pad), the product with its radius (M x 2 n), a status flag.
struct SplitLayout {
  int64_t v, rows, open, stats, xc, prod, flag, total, m_pad, plane;
};
SplitLayout split_layout(const gear_dag* d, int64_t batch, int64_t base) {
  using namespace gear::foldtc;
  SplitLayout L{};
  const int64_t M = batch * d->hdr[gear::H_S], n = d->hdr[gear::H_N];
  L.m_pad = align_up(M, BM);
  L.plane = L.m_pad * d->split_nd.k_pad;
  int64_t o = align_up(base, kAlign);
  L.v = o;     o = align_up(o + M * d->split_k * (int64_t)sizeof(double), kAlign);
  L.rows = o;  o = align_up(o + M * 3 * (int64_t)sizeof(double), kAlign);
  L.open = o;  o = align_up(o + batch * (int64_t)sizeof(int), kAlign);
  L.stats = o; o = align_up(o + L.m_pad * (int64_t)sizeof(BoxStat), kAlign);
  L.xc = o;    o = align_up(o + DIGITS * L.plane, kAlign);
  L.prod = o;  o = align_up(o + M * 2 * n * (int64_t)sizeof(double), kAlign);
  L.flag = o;  o = align_up(o + (int64_t)sizeof(int), kAlign);
  L.total = o;
  return L;
}

// The OF_SPLIT op of the final pass, if any: digit planes of its node's W^T (n rows of w).
int split_prepare(gear_dag* d, const int32_t* nodes, const int32_t* ops) {
  using namespace gear;
  using namespace gear::foldtc;
  if (!ops) return GEAR_OK;
  const int nsteps = d->hdr[H_NSTEPS];
  int fpass = -1;
  for (int si = 0; si < nsteps; ++si)
    if (d->steps[(size_t)si * STEP_REC] == ST_FINAL) fpass = d->steps[(size_t)si * STEP_REC + 1];
  if (fpass < 0 || d->passes.empty()) return GEAR_OK;
  const int32_t* pr = d->passes.data() + (size_t)fpass * PASS_REC;
  if (pr[P_NOP] < 1 || pr[P_SIDES] != 1 || pr[P_XDENSE] == 0) return GEAR_OK;
  const int32_t* op = ops + (size_t)(pr[P_OP0] + pr[P_NOP] - 1) * OP_REC;
  if (!(op[O_SINGLE] & OF_SPLIT)) return GEAR_OK;
  const int32_t* nd = nodes + (int64_t)op[O_V] * NODE_REC;
  const int w = nd[N_W], n = nd[N_WIN];
  if (nd[N_WT_OFF] < 0 || n != d->hdr[H_N] || w < 2 * BK) return GEAR_OK;
  NodeDigits dg{};
  dg.w = n;
  dg.n_pad = (int)align_up(n, BN);
  dg.k_pad = (int)align_up(w, BK);
  if ((int64_t)DIGITS * dg.k_pad * 127 * 127 >= (int64_t)1 << 31) return GEAR_OK;
  dg.plane = (int64_t)dg.n_pad * dg.k_pad;
  dg.fold_off = 0;
  const int64_t bytes = align_up(2 * DIGITS * dg.plane + (int64_t)dg.n_pad * (sizeof(int) + 2 * sizeof(double)) + 64,
                                 kAlign);
  cudaError_t e = cudaMalloc(&d->split_dev, bytes);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(final-pass product digits)");
  int8_t* wd = (int8_t*)d->split_dev;
  int8_t* wa = wd + DIGITS * dg.plane;
  double* wnorm = (double*)align_up((int64_t)(wa + DIGITS * dg.plane), 8);
  double* wdelta = wnorm + dg.n_pad;
  int* we = (int*)(wdelta + dg.n_pad);
  dg.wd = wd;
  dg.wa = wa;
  dg.we = we;
  dg.wnorm = wnorm;
  dg.wdelta = wdelta;
  // W^T is (n x w) row-major in the program (the forward products' copy): its rows are the
  // product's outputs, its columns the inner dimension
  w_digits_kernel<<<dg.n_pad, NT>>>(d->P.dp + nd[N_WT_OFF], n, w, dg, wd, wa, we, wnorm, wdelta);
  e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "final-pass product digits");
  d->split_nd = dg;
  d->split_k = w;
  d->split = true;
  return GEAR_OK;
}

// Digit planes of every dense node on the input (fold step of a box-per-CTA program), built once.
int tc_prepare(gear_dag* d, const int32_t* nodes) {
  using namespace gear;
  using namespace gear::foldtc;
  const int n_nodes = d->hdr[H_NNODES];
  struct Pending { int v, w, K, n_pad, k_pad, woff; int64_t off; };
  std::vector<Pending> todo;
  int64_t bytes = 0;
  for (int v = 0; v < n_nodes; ++v) {
    const int32_t* nd = nodes + (int64_t)v * NODE_REC;
    if (nd[N_FOLD] < 0) continue;
    Pending p;
    p.v = v;
    p.w = nd[N_W];
    p.K = nd[N_WIN];
    p.n_pad = (int)align_up(p.w, BN);
    p.k_pad = (int)align_up(p.K, BK);
    p.woff = nd[N_W_OFF];
    // int32 level sums: at most DIGITS pairs x k_pad x 127^2 must stay below 2^31
    if ((int64_t)DIGITS * p.k_pad * 127 * 127 >= (int64_t)1 << 31)
      return fail(GEAR_E_INVALID, "gear_dag_create: %s", "tensor-core fold: input width beyond the int32 accumulator bound");
    if (d->tc_k_pad && d->tc_k_pad != p.k_pad)
      return fail(GEAR_E_INVALID, "gear_dag_create: %s", "tensor-core fold: dense nodes on the input of different widths");
    d->tc_k_pad = p.k_pad;
    p.off = bytes;
    const int64_t plane = (int64_t)p.n_pad * p.k_pad;
    bytes = align_up(bytes + 2 * DIGITS * plane + (int64_t)p.n_pad * (sizeof(int) + 2 * sizeof(double)) + 64, kAlign);
    todo.push_back(p);
  }
  if (todo.empty()) return GEAR_OK;
  cudaError_t e = cudaMalloc(&d->tc_dev, bytes);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(tensor-core fold digits)");
  for (const Pending& p : todo) {
    char* base = (char*)d->tc_dev + p.off;
    NodeDigits nd;
    nd.plane = (int64_t)p.n_pad * p.k_pad;
    int8_t* wd = (int8_t*)base;
    int8_t* wa = wd + DIGITS * nd.plane;
    double* wnorm = (double*)align_up((int64_t)(wa + DIGITS * nd.plane), 8);
    double* wdelta = wnorm + p.n_pad;
    int* we = (int*)(wdelta + p.n_pad);
    nd.wd = wd;
    nd.wa = wa;
    nd.we = we;
    nd.wnorm = wnorm;
    nd.wdelta = wdelta;
    nd.w = p.w;
    nd.k_pad = p.k_pad;
    nd.n_pad = p.n_pad;
    nd.fold_off = (nodes + (int64_t)p.v * NODE_REC)[N_FOLD];
    w_digits_kernel<<<p.n_pad, NT>>>(d->P.dp + p.woff, p.w, p.K, nd, wd, wa, we, wnorm, wdelta);
    d->tc_nodes.push_back(nd);
  }
  e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "tensor-core fold digits");
  e = cudaFuncSetAttribute(fold_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
  if (e != cudaSuccess) return cuda_fail(e, "fold_tc_kernel shared memory");
  return GEAR_OK;
}

// Box digits, then one tensor-core launch per dense node: fold vectors of the batch into the
// workspace (layout L). Returns the number of kernel launches, or a negative status.
int tc_launch(const gear_dag* d, const double* x_L, const double* x_U, int64_t batch, char* ws, const TcLayout& L,
              cudaStream_t stream) {
  using namespace gear::foldtc;
  int* flag = (int*)(ws + L.flag);
  cudaError_t e = cudaMemsetAsync(flag, 0, sizeof(int), stream);
  if (e != cudaSuccess) return cuda_fail(e, "tensor-core fold status");
  BoxStat* st = (BoxStat*)(ws + L.stats);
  int8_t* xc = (int8_t*)(ws + L.xc);
  int8_t* xr = (int8_t*)(ws + L.xr);
  box_digits_kernel<<<(unsigned)L.b_pad, NT, 0, stream>>>(x_L, x_U, batch, d->hdr[gear::H_N], d->tc_k_pad, xc, xr,
                                                         L.plane, st);
  int launches = 1;
  BatchDigits bt;
  bt.xc = xc;
  bt.xr = xr;
  bt.plane = L.plane;
  bt.st = st;
  bt.fold = (double*)(ws + L.fold);
  bt.fold_w = d->hdr[gear::H_FOLDW];
  bt.B = batch;
  bt.status = flag;
  for (const NodeDigits& nd : d->tc_nodes) {
    dim3 grid((unsigned)(nd.n_pad / BN), (unsigned)(L.b_pad / BM));
    fold_tc_kernel<<<grid, NT, SMEM_BYTES, stream>>>(nd, bt);
    ++launches;
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "tensor-core fold launch");
  return launches;
}
}  // namespace

// The dynamic shared-memory limit of a kernel (a cap on what a launch may request), raised when
// a launch needs more than the value set so far on this device and never lowered: launches that
// fit make no attribute call, so the iterations of a branch-and-bound run can be captured into a
// CUDA graph after their first eager run.
static std::mutex g_smem_attr_mu;
static std::map<std::pair<const void*, int>, int> g_smem_attr;
static cudaError_t set_smem_limit(const void* func, int bytes) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(g_smem_attr_mu);
  auto key = std::make_pair(func, dev);
  auto it = g_smem_attr.find(key);
  if (it != g_smem_attr.end() && it->second >= bytes) return cudaSuccess;
  e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) g_smem_attr[key] = bytes;
  return e;
}

// box-per-CTA kernel instances: dynamic shared-memory limit and resident CTAs per SM
// (GWS: the program keeps its pass working set in global memory, a kernel instance of its own;
// FX: its fold vectors come from the tensor-core fold, shared-memory programs only)
template <int NT, bool GWS, bool FX>
cudaError_t cta_occupancy_t(int smem_bytes, int* bps) {
  cudaError_t e = set_smem_limit((const void*)gear::crown_megakernel<NT, GWS, FX>, smem_bytes);
  if (e != cudaSuccess) return e;
#ifdef GEAR_CTA_CARVEOUT
  // shared-memory share of the unified L1 (percent) for builds that fix it
  e = cudaFuncSetAttribute(gear::crown_megakernel<NT, GWS, FX>, cudaFuncAttributePreferredSharedMemoryCarveout,
                           GEAR_CTA_CARVEOUT);
  if (e != cudaSuccess) return e;
#endif

  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(bps, gear::crown_megakernel<NT, GWS, FX>, NT, smem_bytes);
}
template <int NT>
cudaError_t cta_occupancy_nt(bool gws, bool fx, int smem_bytes, int* bps) {
  if (gws) return cta_occupancy_t<NT, true, false>(smem_bytes, bps);
  return fx ? cta_occupancy_t<NT, false, true>(smem_bytes, bps) : cta_occupancy_t<NT, false, false>(smem_bytes, bps);
}
static cudaError_t cta_occupancy(int threads, bool gws, bool fx, int smem_bytes, int* bps) {
  switch (threads) {
    case 64: return cta_occupancy_nt<64>(gws, fx, smem_bytes, bps);
    case 128: return cta_occupancy_nt<128>(gws, fx, smem_bytes, bps);
    case 256: return cta_occupancy_nt<256>(gws, fx, smem_bytes, bps);
    default: return cudaErrorInvalidValue;
  }
}
template <int NT, bool GWS, bool FX>
cudaError_t cta_launch_t(const gear::DevProgram& P, const gear::Work& wk, int64_t slots, int smem_bytes, cudaStream_t st) {
  // the kernel's dynamic shared-memory limit is per function: set it for this program
  cudaError_t e = set_smem_limit((const void*)gear::crown_megakernel<NT, GWS, FX>, smem_bytes);
  if (e != cudaSuccess) return e;
  gear::crown_megakernel<NT, GWS, FX><<<(unsigned)slots, NT, smem_bytes, st>>>(P, wk);
  return cudaGetLastError();
}
template <int NT>
cudaError_t cta_launch_any(const gear::DevProgram& P, const gear::Work& wk, int64_t slots, int smem_bytes, bool gws,
                           cudaStream_t st) {
  if (gws) return cta_launch_t<NT, true, false>(P, wk, slots, smem_bytes, st);
  return wk.fold_ext ? cta_launch_t<NT, false, true>(P, wk, slots, smem_bytes, st)
                     : cta_launch_t<NT, false, false>(P, wk, slots, smem_bytes, st);
}

extern "C" const char* gear_last_error(void) { return g_err.c_str(); }
extern "C" int gear_last_launch_count(void) { return g_launches; }

extern "C" int gear_dag_create(const int32_t* header, int64_t header_len, const int32_t* nodes,
                               int64_t n_nodes_ints, const int32_t* steps, int64_t n_steps_ints,
                               const int32_t* passes, int64_t n_passes_ints, const int32_t* ops,
                               int64_t n_ops_ints, const int32_t* int_pool, int64_t n_int,
                               const double* dbl_pool, int64_t n_dbl, gear_dag** out) {
  if (!out || !header || header_len != gear::HEADER_LEN || !nodes || !steps)
    return fail(GEAR_E_INVALID, "gear_dag_create: %s", "bad arguments");
  using namespace gear;
  if (n_nodes_ints != (int64_t)header[H_NNODES] * NODE_REC || n_steps_ints != (int64_t)header[H_NSTEPS] * STEP_REC ||
      n_passes_ints != (int64_t)header[H_NPASSES] * PASS_REC || n_ops_ints != (int64_t)header[H_NOPS] * OP_REC)
    return fail(GEAR_E_INVALID, "gear_dag_create: %s", "record counts do not match the header");
  gear_dag* d = new (std::nothrow) gear_dag();
  if (!d) return fail(GEAR_E_NOMEM, "gear_dag_create: %s", "host allocation");
  memcpy(d->hdr, header, sizeof(d->hdr));
  d->steps.assign(steps, steps + n_steps_ints);
  if (passes && n_passes_ints > 0) d->passes.assign(passes, passes + n_passes_ints);
  // one device block: doubles first (8-byte aligned), then int arrays
  size_t nd = (size_t)n_dbl, ni = (size_t)(header_len + n_nodes_ints + n_steps_ints + n_passes_ints + n_ops_ints + n_int);
  size_t bytes = nd * sizeof(double) + ni * sizeof(int32_t) + 64;
  cudaError_t e = cudaGetDevice(&d->device);
  if (e != cudaSuccess) { delete d; return cuda_fail(e, "cudaGetDevice"); }
  e = cudaMalloc(&d->dev, bytes);
  if (e != cudaSuccess) { delete d; return cuda_fail(e, "cudaMalloc(program)"); }
  char* base = (char*)d->dev;
  double* dp = (double*)base;
  int32_t* ip = (int32_t*)(base + nd * sizeof(double));
  size_t o = 0;
  auto put = [&](const int32_t* src, int64_t cnt) -> const int32_t* {
    int32_t* dst = ip + o;
    if (cnt > 0) cudaMemcpy(dst, src, cnt * sizeof(int32_t), cudaMemcpyHostToDevice);
    o += (size_t)cnt;
    return dst;
  };
  d->P.hdr = put(header, header_len);
  d->P.nodes = put(nodes, n_nodes_ints);
  d->P.steps = put(steps, n_steps_ints);
  d->P.passes = put(passes, n_passes_ints);
  d->P.ops = put(ops, n_ops_ints);
  d->P.ip = put(int_pool, n_int);
  if (nd > 0) cudaMemcpy(dp, dbl_pool, nd * sizeof(double), cudaMemcpyHostToDevice);
  d->P.dp = dp;
  e = cudaGetLastError();
  if (e != cudaSuccess) { cudaFree(d->dev); delete d; return cuda_fail(e, "upload"); }
  cudaDeviceProp prop;
  e = cudaGetDeviceProperties(&prop, d->device);
  if (e != cudaSuccess) { cudaFree(d->dev); delete d; return cuda_fail(e, "cudaGetDeviceProperties"); }
  d->num_sms = prop.multiProcessorCount;
  d->mode = header[H_MODE];
  int bps = 0;
  if (d->mode == MODE_SIMT) {
    if (header[H_X_IN_LA] != 0) {
      cudaFree(d->dev);
      delete d;
      return fail(GEAR_E_INVALID, "gear_dag_create: %s", "a box-per-thread program keeps the input's A in its buffers");
    }
    // per-CTA scratch: SIMT_T boxes, every per-box item box-interleaved
    d->threads = SIMT_T;
    d->boxes_per_slot = SIMT_T;
    const int64_t items = 3 * (int64_t)header[H_ARENA] + header[H_PLANES] + header[H_FOLDW] +
                          4 * (int64_t)header[H_MAXW] + header[H_SIMT_BUF] + header[H_SIMT_ROWS];
    d->slot_doubles = items * SIMT_T;
    d->smem_bytes = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, crown_simt_kernel, SIMT_T, 0);
  } else if (d->mode == MODE_CTA) {
    // per-CTA scratch: lo, hi, mag arenas; planes; fold vectors; 4 node-wide temporaries
    d->threads = header[H_CTA_THREADS];
    d->boxes_per_slot = 1;
    d->slot_doubles = cta_slot_fixed(header) + header[H_PASS_GLOBAL];
    d->smem_bytes = header[H_SMEM] * (int)sizeof(double);
    if (d->smem_bytes > (int)prop.sharedMemPerBlockOptin) {
      cudaFree(d->dev);
      delete d;
      return fail(GEAR_E_INVALID, "gear_dag_create: %s", "pass working set exceeds shared memory");
    }
    if (header[H_PASS_GLOBAL] > 0 && header[H_FOLD_TC] != 0) {
      cudaFree(d->dev);
      delete d;
      return fail(GEAR_E_INVALID, "gear_dag_create: %s", "the tensor-core fold needs the pass working set in shared memory");
    }
    e = cta_occupancy(d->threads, header[H_PASS_GLOBAL] > 0, header[H_FOLD_TC] != 0, d->smem_bytes, &bps);
    if (e == cudaErrorInvalidValue) {
      cudaFree(d->dev);
      delete d;
      return fail(GEAR_E_INVALID, "gear_dag_create: %s", "threads per CTA must be 64, 128 or 256");
    }
  } else {
    cudaFree(d->dev);
    delete d;
    return fail(GEAR_E_INVALID, "gear_dag_create: %s", "unknown execution mode");
  }
  if (e != cudaSuccess || bps < 1) bps = 1;
  d->blocks_per_sm = bps;
  if (header[H_FOLD_TC] != 0) {
    if (d->mode != MODE_CTA) {
      cudaFree(d->dev);
      delete d;
      return fail(GEAR_E_INVALID, "gear_dag_create: %s", "the tensor-core fold is for box-per-CTA programs");
    }
    int st = tc_prepare(d, nodes);
    if (st == GEAR_OK) st = split_prepare(d, nodes, ops);
    if (st != GEAR_OK) {
      if (d->tc_dev) cudaFree(d->tc_dev);
      if (d->split_dev) cudaFree(d->split_dev);
      cudaFree(d->dev);
      delete d;
      return st;
    }
  }
  *out = d;
  return GEAR_OK;
}

extern "C" int gear_dag_destroy(gear_dag* dag) {
  if (!dag) return GEAR_OK;
  if (dag->dev) cudaFree(dag->dev);
  if (dag->tc_dev) cudaFree(dag->tc_dev);
  if (dag->split_dev) cudaFree(dag->split_dev);
  delete dag;
  return GEAR_OK;
}

// CTAs of one launch: every resident CTA, or fewer when the batch has fewer boxes (CTA mode)
// or tiles of SIMT_T boxes (SIMT mode)
static int64_t slots_for(const gear_dag* d, int64_t batch) {
  int64_t slots = (int64_t)d->num_sms * d->blocks_per_sm;
  const int64_t units = (batch + d->boxes_per_slot - 1) / d->boxes_per_slot;
  if (units < slots) slots = units;
  return slots < 1 ? 1 : slots;
}

static int launch_crown(const gear_dag* dag, const gear::Work& wk, int64_t slots, cudaStream_t stream) {
  if (dag->mode == gear::MODE_SIMT) {
    gear::crown_simt_kernel<<<(unsigned)slots, gear::SIMT_T, 0, stream>>>(dag->P, wk);
    g_launches = 1;
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? GEAR_OK : cuda_fail(e, "crown_simt_kernel launch");
  }
  cudaError_t e = cudaErrorInvalidValue;
  const bool gws = dag->hdr[gear::H_PASS_GLOBAL] > 0;
  switch (dag->threads) {
    case 64: e = cta_launch_any<64>(dag->P, wk, slots, dag->smem_bytes, gws, stream); break;
    case 128: e = cta_launch_any<128>(dag->P, wk, slots, dag->smem_bytes, gws, stream); break;
    case 256: e = cta_launch_any<256>(dag->P, wk, slots, dag->smem_bytes, gws, stream); break;
    default: break;
  }
  g_launches = 1;
  return e == cudaSuccess ? GEAR_OK : cuda_fail(e, "crown_megakernel launch");
}

extern "C" int64_t gear_crown_workspace_bytes(const gear_dag* dag, int64_t batch) {
  if (!dag || batch < 0) return -1;
  const int64_t slots = slots_for(dag, batch) * dag->slot_doubles * (int64_t)sizeof(double);
  if (dag->tc_nodes.empty() || batch == 0) return slots;
  const int64_t tc = tc_layout(dag, batch, slots).total;
  return dag->split ? split_layout(dag, batch, tc).total : tc;
}

static int crown_lower_impl(const gear_dag* dag, const double* x_L, const double* x_U, int64_t batch,
                            const double* C, double* lb, double* lA, double* lbias, double* lb_ibp, void* workspace,
                            int64_t workspace_bytes, void* stream);

extern "C" int gear_crown_lower(const gear_dag* dag, const double* x_L, const double* x_U, int64_t batch,
                                const double* C, double* lb, double* lA, double* lbias, void* workspace,
                                int64_t workspace_bytes, void* stream) {
  return crown_lower_impl(dag, x_L, x_U, batch, C, lb, lA, lbias, nullptr, workspace, workspace_bytes, stream);
}

extern "C" int gear_crown_lower_ibp(const gear_dag* dag, const double* x_L, const double* x_U, int64_t batch,
                                    const double* C, double* lb, double* lA, double* lbias, double* lb_ibp,
                                    void* workspace, int64_t workspace_bytes, void* stream) {
  if (!lb_ibp) return fail(GEAR_E_INVALID, "gear_crown_lower_ibp: %s", "lb_ibp is required");
  return crown_lower_impl(dag, x_L, x_U, batch, C, lb, lA, lbias, lb_ibp, workspace, workspace_bytes, stream);
}

static int crown_lower_impl(const gear_dag* dag, const double* x_L, const double* x_U, int64_t batch,
                            const double* C, double* lb, double* lA, double* lbias, double* lb_ibp, void* workspace,
                            int64_t workspace_bytes, void* stream) {
  g_launches = 0;
  if (!dag || batch < 0) return fail(GEAR_E_INVALID, "gear_crown_lower: %s", "bad arguments");
  if (batch == 0) return GEAR_OK;             // empty arrays may come with null pointers
  if (!x_L || !x_U || !lb) return fail(GEAR_E_INVALID, "gear_crown_lower: %s", "bad arguments");
  if (!workspace || workspace_bytes < gear_crown_workspace_bytes(dag, batch))
    return fail(GEAR_E_WORKSPACE, "gear_crown_lower: %s", "workspace too small");
  if (dag->hdr[gear::H_RETA] == 0 && lA) return fail(GEAR_E_INVALID, "gear_crown_lower: %s", "program built without A");
  if (dag->hdr[gear::H_RETA] != 0 && dag->hdr[gear::H_X_IN_LA] != 0 && !lA)
    return fail(GEAR_E_INVALID, "gear_crown_lower: %s", "this program accumulates A in the lA output: lA is required");
  gear::Work wk;
  wk.xL = x_L;
  wk.xU = x_U;
  wk.C = C;
  wk.lb = lb;
  wk.lA = lA;
  wk.lbias = lbias;
  wk.lb_ibp = lb_ibp;
  wk.scratch = (double*)workspace;
  wk.slot_doubles = dag->slot_doubles;
  wk.B = batch;
  wk.status = nullptr;
  wk.fold_ext = nullptr;
  wk.fold_fail = nullptr;
  int pre = 0;
  if (!dag->tc_nodes.empty()) {
    const int64_t slots_bytes = slots_for(dag, batch) * dag->slot_doubles * (int64_t)sizeof(double);
    const TcLayout L = tc_layout(dag, batch, slots_bytes);
    pre = tc_launch(dag, x_L, x_U, batch, (char*)workspace, L, (cudaStream_t)stream);
    if (pre < 0) return pre;
    wk.fold_ext = (const double*)((char*)workspace + L.fold);
    wk.fold_fail = (const int*)((char*)workspace + L.flag);
    if (dag->split && lA) {
      const SplitLayout SL = split_layout(dag, batch, L.total);
      char* ws = (char*)workspace;
      wk.split_v = (double*)(ws + SL.v);
      wk.split_rows = (double*)(ws + SL.rows);
      wk.split_open = (int*)(ws + SL.open);
      wk.split_k = dag->split_k;
    }
  }
  int st = launch_crown(dag, wk, slots_for(dag, batch), (cudaStream_t)stream);
  g_launches += pre;
  if (st != GEAR_OK || !wk.split_v) return st;
  // the final pass's product on the tensor cores, then its concretisation
  using namespace gear::foldtc;
  const SplitLayout SL = split_layout(dag, batch, tc_layout(dag, batch, slots_for(dag, batch) * dag->slot_doubles *
                                                                            (int64_t)sizeof(double)).total);
  char* ws = (char*)workspace;
  cudaStream_t cs = (cudaStream_t)stream;
  const int64_t M = batch * dag->hdr[gear::H_S];
  const int n = dag->hdr[gear::H_N];
  int* flag = (int*)(ws + SL.flag);
  cudaError_t e = cudaMemsetAsync(flag, 0, sizeof(int), cs);
  if (e != cudaSuccess) return cuda_fail(e, "final-pass product status");
  BoxStat* rst = (BoxStat*)(ws + SL.stats);
  int8_t* xc = (int8_t*)(ws + SL.xc);
  row_digits_kernel<<<(unsigned)SL.m_pad, NT, 0, cs>>>(wk.split_v, M, dag->split_k, dag->split_nd.k_pad, xc, SL.plane,
                                                       rst);
  BatchDigits bt;
  bt.xc = xc;
  bt.xr = xc;                 // unused: one product
  bt.plane = SL.plane;
  bt.st = rst;
  bt.fold = (double*)(ws + SL.prod);
  bt.fold_w = 2 * (int64_t)n;
  bt.B = M;
  bt.status = flag;
  bt.gemv = 1;
  dim3 grid((unsigned)(dag->split_nd.n_pad / BN), (unsigned)(SL.m_pad / BM));
  fold_tc_kernel<<<grid, NT, SMEM_BYTES, cs>>>(dag->split_nd, bt);
  int64_t tail = (M + 7) / 8;
  const int64_t tail_max = (int64_t)dag->num_sms * 8;
  if (tail > tail_max) tail = tail_max;
  gear::split_tail_kernel<256><<<(unsigned)(tail < 1 ? 1 : tail), 256, 0, cs>>>(wk, dag->hdr[gear::H_S], n,
                                                                             (const double*)(ws + SL.prod), rst, flag);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "final-pass product launch");
  g_launches += 3;
  return GEAR_OK;
}

extern "C" int gear_crown_fold_vectors(const gear_dag* dag, const double* x_L, const double* x_U, int64_t batch,
                                       double* fold_out, int* fail_out, void* workspace, int64_t workspace_bytes,
                                       void* stream) {
  g_launches = 0;
  if (!dag || batch < 0) return fail(GEAR_E_INVALID, "gear_crown_fold_vectors: %s", "bad arguments");
  if (dag->tc_nodes.empty()) return fail(GEAR_E_INVALID, "gear_crown_fold_vectors: %s", "program without the tensor-core fold");
  if (batch == 0) return GEAR_OK;
  if (!x_L || !x_U || !fold_out) return fail(GEAR_E_INVALID, "gear_crown_fold_vectors: %s", "bad arguments");
  const TcLayout L = tc_layout(dag, batch, 0);
  if (!workspace || workspace_bytes < L.total) return fail(GEAR_E_WORKSPACE, "gear_crown_fold_vectors: %s", "workspace too small");
  const int pre = tc_launch(dag, x_L, x_U, batch, (char*)workspace, L, (cudaStream_t)stream);
  if (pre < 0) return pre;
  g_launches = pre;
  cudaError_t e = cudaMemcpyAsync(fold_out, (char*)workspace + L.fold, batch * dag->hdr[gear::H_FOLDW] * sizeof(double),
                                  cudaMemcpyDeviceToDevice, (cudaStream_t)stream);
  if (e == cudaSuccess && fail_out)
    e = cudaMemcpyAsync(fail_out, (char*)workspace + L.flag, sizeof(int), cudaMemcpyDeviceToDevice, (cudaStream_t)stream);
  return e == cudaSuccess ? GEAR_OK : cuda_fail(e, "gear_crown_fold_vectors copy");
}

extern "C" int64_t gear_crown_fold_workspace_bytes(const gear_dag* dag, int64_t batch) {
  if (!dag || batch < 0 || dag->tc_nodes.empty()) return -1;
  return tc_layout(dag, batch, 0).total;
}

// ------------------------------------------------------------------ no-allocation entry point
// Scratch for callers that must not allocate device memory themselves: a solver host that
// hands this library a fixed device-memory plan (and no allocator), or a loop that cannot
// afford cudaMalloc's implicit device synchronisation or an allocation failure mid-run.
// Every GPU that loads this library holds the array until the process exits.
namespace {
constexpr int64_t kStaticScratchBytes = int64_t(64) << 20;   // 64 MiB
static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];
constexpr int kMaxDevices = 64;
void* g_static_scratch_ptr[kMaxDevices] = {nullptr};
std::mutex g_static_scratch_mu;

// The array's name is only a host-side handle; the kernel needs its device address, which
// cudaGetSymbolAddress gives per device (looked up once, with that device current).
int static_scratch(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) return fail(GEAR_E_INVALID, "gear_crown_lower_static: %s", "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_static_scratch_mu);
  if (!g_static_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess || !p) return cuda_fail(e == cudaSuccess ? cudaErrorInvalidSymbol : e, "cudaGetSymbolAddress(scratch)");
    g_static_scratch_ptr[dev] = p;
  }
  *out = g_static_scratch_ptr[dev];
  return GEAR_OK;
}
}  // namespace

extern "C" int64_t gear_crown_static_scratch_bytes(void) { return kStaticScratchBytes; }

extern "C" int gear_crown_lower_static(const gear_dag* dag, const double* x_L, const double* x_U, int64_t batch,
                                       const double* C, double* lb, double* lA, double* lbias, void* stream) {
  g_launches = 0;
  // the same argument checks, in the same order, as gear_crown_lower
  if (!dag || batch < 0) return fail(GEAR_E_INVALID, "gear_crown_lower_static: %s", "bad arguments");
  if (batch == 0) return GEAR_OK;             // empty arrays may come with null pointers
  if (!x_L || !x_U || !lb) return fail(GEAR_E_INVALID, "gear_crown_lower_static: %s", "bad arguments");
  if (dag->hdr[gear::H_RETA] == 0 && lA)
    return fail(GEAR_E_INVALID, "gear_crown_lower_static: %s", "program built without A");
  if (dag->hdr[gear::H_RETA] != 0 && dag->hdr[gear::H_X_IN_LA] != 0 && !lA)
    return fail(GEAR_E_INVALID, "gear_crown_lower_static: %s", "this program accumulates A in the lA output: lA is required");
  const int64_t slot_bytes = dag->slot_doubles * (int64_t)sizeof(double);
  const int64_t max_slots = kStaticScratchBytes / slot_bytes;
  if (max_slots < 1) {
    char msg[256];
    snprintf(msg, sizeof(msg), "gear_crown_lower_static: one CTA slot of this program needs %lld bytes of scratch, "
             "more than the static %lld bytes; use gear_crown_lower with a workspace",
             (long long)slot_bytes, (long long)kStaticScratchBytes);
    g_err = msg;
    return GEAR_E_WORKSPACE;
  }
  void* scratch = nullptr;
  int st = static_scratch(&scratch);
  if (st != GEAR_OK) return st;
  int64_t slots = slots_for(dag, batch);
  if (slots > max_slots) slots = max_slots;
  gear::Work wk;
  wk.xL = x_L;
  wk.xU = x_U;
  wk.C = C;
  wk.lb = lb;
  wk.lA = lA;
  wk.lbias = lbias;
  wk.lb_ibp = nullptr;
  wk.scratch = (double*)scratch;   // the kernel writes every scratch word before reading it: no clearing
  wk.slot_doubles = dag->slot_doubles;
  wk.B = batch;
  wk.status = nullptr;
  wk.fold_ext = nullptr;
  wk.fold_fail = nullptr;
  return launch_crown(dag, wk, slots, (cudaStream_t)stream);
}

// ------------------------------------------------------------------ the plain (unfused) form
namespace {
template <int NT>
cudaError_t plain_launch_t(const gear::DevProgram& P, const gear::Work& wk, unsigned grid, int smem, int si, int op_lo,
                           int op_hi, int phase, cudaStream_t st) {
  gear::crown_plain_kernel<NT><<<grid, NT, smem, st>>>(P, wk, si, op_lo, op_hi, phase);
  return cudaGetLastError();
}
template <int NT>
cudaError_t plain_prepare_t(int smem, int* bps) {
  cudaError_t e = cudaFuncSetAttribute(gear::crown_plain_kernel<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(bps, gear::crown_plain_kernel<NT>, NT, smem);
}
bool plain_ok(const gear_dag* d) {
  return d && d->mode == gear::MODE_CTA && d->hdr[gear::H_PASS_GLOBAL] > 0;
}
}  // namespace

extern "C" int64_t gear_crown_plain_workspace_bytes(const gear_dag* dag, int64_t batch) {
  if (!plain_ok(dag) || batch < 0) return -1;
  return batch * dag->slot_doubles * (int64_t)sizeof(double);
}

// cut rows for gear_crown_lower_cuts: the constrained sweep's state and buffers (null: plain form)
struct CutRun {
  gear::cc::Work w;     // the sweep over the boxes and their rows (obj / lb / H set per pass)
  double* obj;          // (B, sides * S, n) dense signed input rows of the running pass
  double* v;            // (B, sides * S) their lower bounds over box ∩ rows
  int warps;            // warps per CTA of the sweep
  size_t smem;          // its dynamic shared memory
};
static int plain_impl(const gear_dag* dag, const double* x_L, const double* x_U, int64_t batch, const double* C,
                      double* lb, double* lA, double* lbias, double* lb_ibp, void* workspace, int64_t workspace_bytes,
                      void* stream, CutRun* cut = nullptr);

extern "C" int gear_crown_lower_plain(const gear_dag* dag, const double* x_L, const double* x_U, int64_t batch,
                                      const double* C, double* lb, double* lA, double* lbias, void* workspace,
                                      int64_t workspace_bytes, void* stream) {
  return plain_impl(dag, x_L, x_U, batch, C, lb, lA, lbias, nullptr, workspace, workspace_bytes, stream);
}

extern "C" int gear_crown_lower_plain_ibp(const gear_dag* dag, const double* x_L, const double* x_U, int64_t batch,
                                          const double* C, double* lb, double* lA, double* lbias, double* lb_ibp,
                                          void* workspace, int64_t workspace_bytes, void* stream) {
  if (!lb_ibp) return fail(GEAR_E_INVALID, "gear_crown_lower_plain_ibp: %s", "lb_ibp is required");
  return plain_impl(dag, x_L, x_U, batch, C, lb, lA, lbias, lb_ibp, workspace, workspace_bytes, stream);
}

static int plain_impl(const gear_dag* dag, const double* x_L, const double* x_U, int64_t batch, const double* C,
                      double* lb, double* lA, double* lbias, double* lb_ibp, void* workspace, int64_t workspace_bytes,
                      void* stream, CutRun* cut) {
  if (!cut) g_launches = 0;
  if (!dag || batch < 0) return fail(GEAR_E_INVALID, "gear_crown_lower_plain: %s", "bad arguments");
  if (!plain_ok(dag))
    return fail(GEAR_E_INVALID, "gear_crown_lower_plain: %s",
                "needs a box-per-CTA program compiled with its pass working set in global memory");
  if (batch == 0) return GEAR_OK;
  if (!x_L || !x_U || !lb || !lA) return fail(GEAR_E_INVALID, "gear_crown_lower_plain: %s", "bad arguments");
  if (!cut && (!workspace || workspace_bytes < gear_crown_plain_workspace_bytes(dag, batch)))
    return fail(GEAR_E_WORKSPACE, "gear_crown_lower_plain: %s", "workspace too small");
  gear::Work wk;
  wk.xL = x_L;
  wk.xU = x_U;
  wk.C = C;
  wk.lb = lb;
  wk.lA = lA;
  wk.lbias = lbias;
  wk.lb_ibp = lb_ibp;
  wk.scratch = (double*)workspace;
  wk.slot_doubles = dag->slot_doubles;   // one slot per box
  wk.B = batch;
  wk.status = nullptr;
  wk.fold_ext = nullptr;
  wk.fold_fail = nullptr;
  cudaStream_t st = (cudaStream_t)stream;
  int bps = 0;
  cudaError_t e = cudaErrorInvalidValue;
  switch (dag->threads) {
    case 64: e = plain_prepare_t<64>(dag->smem_bytes, &bps); break;
    case 128: e = plain_prepare_t<128>(dag->smem_bytes, &bps); break;
    case 256: e = plain_prepare_t<256>(dag->smem_bytes, &bps); break;
    default: break;
  }
  if (e != cudaSuccess) return cuda_fail(e, "crown_plain_kernel setup");
  int64_t grid = (int64_t)dag->num_sms * (bps > 0 ? bps : 1);
  if (grid > batch) grid = batch;
  int launches = 0;
  auto go = [&](int si, int op_lo, int op_hi, int phase) -> cudaError_t {
    ++launches;
    switch (dag->threads) {
      case 64: return plain_launch_t<64>(dag->P, wk, (unsigned)grid, dag->smem_bytes, si, op_lo, op_hi, phase, st);
      case 128: return plain_launch_t<128>(dag->P, wk, (unsigned)grid, dag->smem_bytes, si, op_lo, op_hi, phase, st);
      default: return plain_launch_t<256>(dag->P, wk, (unsigned)grid, dag->smem_bytes, si, op_lo, op_hi, phase, st);
    }
  };
  e = go(-1, 0, 0, 0);
  const int nsteps = dag->hdr[gear::H_NSTEPS];
  for (int si = 0; si < nsteps && e == cudaSuccess; ++si) {
    const int type = dag->steps[(size_t)si * gear::STEP_REC], a = dag->steps[(size_t)si * gear::STEP_REC + 1];
    if (type == gear::ST_PASS || type == gear::ST_FINAL) {
      const int nop = dag->passes[(size_t)a * gear::PASS_REC + gear::P_NOP];
      e = go(si, 0, 0, 1);
      for (int oi = 0; oi < nop && e == cudaSuccess; ++oi) e = go(si, oi, oi + 1, 0);
      if (cut && e == cudaSuccess) {
        // dense signed input rows -> the constrained sweep -> the concretisation reads its bounds
        const int32_t* pr = dag->passes.data() + (size_t)a * gear::PASS_REC;
        const int H = pr[gear::P_SIDES] * pr[gear::P_S];
        wk.cut_obj = cut->obj;
        wk.cut_h = H;
        wk.cut_v = nullptr;
        e = go(si, 0, 0, 4);
        if (e == cudaSuccess) {
          cut->w.obj = cut->obj;
          cut->w.lb = cut->v;
          cut->w.H = H;
          const int64_t items = batch * H;
          gear::cc::concretize_sweep_kernel<<<(unsigned)((items + cut->warps - 1) / cut->warps), 32 * cut->warps,
                                              cut->smem, st>>>(cut->w);
          ++launches;
          e = cudaGetLastError();
        }
        wk.cut_v = cut->v;
      }
      if (e == cudaSuccess) e = go(si, 0, 0, 2);
      wk.cut_v = nullptr;
    } else {
      e = go(si, 0, 0, 0);
    }
  }
  g_launches += launches;
  return e == cudaSuccess ? GEAR_OK : cuda_fail(e, "crown_plain_kernel launch");
}

// ------------------------------------------------------------------ many instances, one launch
namespace {
template <int NT, bool GWS>
cudaError_t multi_cta_occupancy_t(int smem_bytes, int* bps) {
  cudaError_t e = set_smem_limit((const void*)gear::crown_multi_megakernel<NT, GWS>, smem_bytes);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(bps, gear::crown_multi_megakernel<NT, GWS>, NT, smem_bytes);
}
template <int NT>
cudaError_t multi_cta_occupancy(bool gws, int smem_bytes, int* bps) {
  return gws ? multi_cta_occupancy_t<NT, true>(smem_bytes, bps) : multi_cta_occupancy_t<NT, false>(smem_bytes, bps);
}
template <int NT>
void multi_cta_launch(bool gws, unsigned grid, int smem, cudaStream_t st, const gear::MultiItem* items, int count,
                      const int64_t* start, unsigned long long* next, double* scratch, int64_t slot_doubles) {
  if (gws) gear::crown_multi_megakernel<NT, true><<<grid, NT, smem, st>>>(items, count, start, next, scratch, slot_doubles);
  else gear::crown_multi_megakernel<NT, false><<<grid, NT, smem, st>>>(items, count, start, next, scratch, slot_doubles);
}

struct MultiPlan {
  int mode = 0, threads = 0, smem = 0, device = 0, count = 0;   // count: instances with boxes
  bool gws = false;           // box-per-CTA programs with their pass working set in global memory
  int64_t total = 0;          // work items: boxes (box per CTA) or tiles of SIMT_T boxes
  int64_t slot_doubles = 0;   // the largest program's slot
  int64_t slots = 1;          // CTAs of the launch
  int64_t items_off = 0, start_off = 0, scratch_off = 0, bytes = 0;
};

inline int64_t align256(int64_t v) { return (v + 255) / 256 * 256; }

int multi_plan(const gear_lower_args* a, int32_t count, MultiPlan& pl) {
  if (count < 0 || (count > 0 && !a)) return fail(GEAR_E_INVALID, "gear_crown_lower_multi: %s", "bad arguments");
  bool first = true;
  int num_sms = 0;
  for (int32_t i = 0; i < count; ++i) {
    const gear_dag* d = a[i].dag;
    if (!d || a[i].batch < 0) return fail(GEAR_E_INVALID, "gear_crown_lower_multi: %s", "bad instance arguments");
    if (a[i].batch > 0 && (!a[i].x_L || !a[i].x_U || !a[i].lb))
      return fail(GEAR_E_INVALID, "gear_crown_lower_multi: %s", "bad instance arguments");
    if (d->hdr[gear::H_RETA] == 0 && a[i].lA)
      return fail(GEAR_E_INVALID, "gear_crown_lower_multi: %s", "program built without A");
    if (d->hdr[gear::H_RETA] != 0 && d->hdr[gear::H_X_IN_LA] != 0 && !a[i].lA && a[i].batch > 0)
      return fail(GEAR_E_INVALID, "gear_crown_lower_multi: %s", "this program accumulates A in the lA output: lA is required");
    const bool gws = d->mode == gear::MODE_CTA && d->hdr[gear::H_PASS_GLOBAL] > 0;
    if (first) {
      pl.mode = d->mode;
      pl.threads = d->threads;
      pl.device = d->device;
      pl.gws = gws;
      num_sms = d->num_sms;
      first = false;
    } else if (d->mode != pl.mode || d->threads != pl.threads || d->device != pl.device || gws != pl.gws) {
      return fail(GEAR_E_INVALID, "gear_crown_lower_multi: %s",
                  "every program of one launch needs the same execution mode, threads per CTA, pass working-set "
                  "placement and device");
    }
    if (a[i].batch == 0) continue;
    ++pl.count;
    pl.total += (a[i].batch + d->boxes_per_slot - 1) / d->boxes_per_slot;
    if (d->slot_doubles > pl.slot_doubles) pl.slot_doubles = d->slot_doubles;
    if (d->smem_bytes > pl.smem) pl.smem = d->smem_bytes;
  }
  if (pl.count == 0) return GEAR_OK;
  int bps = 0;
  cudaError_t e = cudaSuccess;
  if (pl.mode == gear::MODE_SIMT) {
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, gear::crown_multi_simt_kernel, gear::SIMT_T, 0);
  } else {
    switch (pl.threads) {
      case 64: e = multi_cta_occupancy<64>(pl.gws, pl.smem, &bps); break;
      case 128: e = multi_cta_occupancy<128>(pl.gws, pl.smem, &bps); break;
      case 256: e = multi_cta_occupancy<256>(pl.gws, pl.smem, &bps); break;
      default: return fail(GEAR_E_INVALID, "gear_crown_lower_multi: %s", "threads per CTA must be 64, 128 or 256");
    }
  }
  if (e != cudaSuccess) return cuda_fail(e, "gear_crown_lower_multi occupancy");
  if (bps < 1) bps = 1;
  pl.slots = (int64_t)num_sms * bps;
  if (pl.total < pl.slots) pl.slots = pl.total;
  pl.items_off = 256;                                   // [0, 8): the work counter
  pl.start_off = pl.items_off + align256((int64_t)pl.count * (int64_t)sizeof(gear::MultiItem));
  pl.scratch_off = pl.start_off + align256((int64_t)(pl.count + 1) * (int64_t)sizeof(int64_t));
  pl.bytes = pl.scratch_off + pl.slots * pl.slot_doubles * (int64_t)sizeof(double);
  return GEAR_OK;
}

// Pinned staging for the per-launch instance table, one per device and host thread: the copy
// from it is asynchronous, and the buffer is reused only after the previous copy has finished.
struct Staging {
  void* host = nullptr;
  size_t cap = 0;
  cudaEvent_t done = nullptr;
};
thread_local Staging g_staging[kMaxDevices];
}  // namespace

namespace {
// The instance table and the work-item prefix of a launch, written to host memory at `host`
// (laid out as the workspace from items_off on).
void multi_table(const gear_lower_args* items, int32_t count, const MultiPlan& pl, char* host) {
  gear::MultiItem* hitems = (gear::MultiItem*)host;
  int64_t* hstart = (int64_t*)(host + (pl.start_off - pl.items_off));
  int k = 0;
  hstart[0] = 0;
  for (int32_t i = 0; i < count; ++i) {
    const gear_lower_args& a = items[i];
    if (a.batch == 0) continue;
    gear::MultiItem& it = hitems[k];
    it.P = a.dag->P;
    it.wk.xL = a.x_L;
    it.wk.xU = a.x_U;
    it.wk.C = a.C;
    it.wk.lb = a.lb;
    it.wk.lA = a.lA;
    it.wk.lbias = a.lbias;
    it.wk.lb_ibp = a.lb_ibp;
    it.wk.scratch = nullptr;
    it.wk.slot_doubles = pl.slot_doubles;
    it.wk.B = a.batch;
    it.wk.status = nullptr;
    it.wk.fold_ext = nullptr;
    it.wk.fold_fail = nullptr;
    hstart[k + 1] = hstart[k] + (a.batch + a.dag->boxes_per_slot - 1) / a.dag->boxes_per_slot;
    ++k;
  }
}

// The launch of a planned many-instance call whose table is already in the workspace.
int multi_launch(const MultiPlan& pl, char* ws, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(ws, 0, sizeof(unsigned long long), st);
  if (e != cudaSuccess) return cuda_fail(e, "crown multi-instance launch");
  const gear::MultiItem* ditems = (const gear::MultiItem*)(ws + pl.items_off);
  const int64_t* dstart = (const int64_t*)(ws + pl.start_off);
  unsigned long long* next = (unsigned long long*)ws;
  double* scratch = (double*)(ws + pl.scratch_off);
  const unsigned grid = (unsigned)pl.slots;
  if (pl.mode == gear::MODE_SIMT) {
    gear::crown_multi_simt_kernel<<<grid, gear::SIMT_T, 0, st>>>(ditems, pl.count, dstart, next, scratch,
                                                                  pl.slot_doubles);
  } else {
    switch (pl.threads) {
      case 64: multi_cta_launch<64>(pl.gws, grid, pl.smem, st, ditems, pl.count, dstart, next, scratch, pl.slot_doubles); break;
      case 128: multi_cta_launch<128>(pl.gws, grid, pl.smem, st, ditems, pl.count, dstart, next, scratch, pl.slot_doubles); break;
      default: multi_cta_launch<256>(pl.gws, grid, pl.smem, st, ditems, pl.count, dstart, next, scratch, pl.slot_doubles); break;
    }
  }
  e = cudaGetLastError();
  return e == cudaSuccess ? GEAR_OK : cuda_fail(e, "crown multi-instance launch");
}
}  // namespace

// A many-instance launch prepared once: its plan, and its instance table already in the caller's
// workspace, so that every later launch (gear_crown_multi_launch) is a counter reset and one
// kernel with fixed arguments, which a CUDA graph can capture.
struct gear_multi_plan {
  MultiPlan pl;
  char* ws = nullptr;
};

extern "C" int64_t gear_crown_multi_workspace_bytes(const gear_lower_args* items, int32_t count) {
  MultiPlan pl;
  if (multi_plan(items, count, pl) != GEAR_OK) return -1;
  return pl.count == 0 ? 0 : pl.bytes;
}

extern "C" int gear_crown_lower_multi(const gear_lower_args* items, int32_t count, void* workspace,
                                      int64_t workspace_bytes, void* stream) {
  g_launches = 0;
  MultiPlan pl;
  int rc = multi_plan(items, count, pl);
  if (rc != GEAR_OK) return rc;
  if (pl.count == 0) return GEAR_OK;
  if (!workspace || workspace_bytes < pl.bytes)
    return fail(GEAR_E_WORKSPACE, "gear_crown_lower_multi: %s", "workspace too small");
  if (pl.device < 0 || pl.device >= kMaxDevices)
    return fail(GEAR_E_INVALID, "gear_crown_lower_multi: %s", "device ordinal out of range");
  cudaStream_t st = (cudaStream_t)stream;
  char* ws = (char*)workspace;
  // the instance table and the work-item prefix, staged in pinned memory
  const size_t table_bytes = (size_t)(pl.start_off - pl.items_off) + (size_t)(pl.count + 1) * sizeof(int64_t);
  Staging& sg = g_staging[pl.device];
  cudaError_t e = cudaSuccess;
  if (sg.done) {
    e = cudaEventSynchronize(sg.done);
    if (e != cudaSuccess) return cuda_fail(e, "gear_crown_lower_multi staging");
  }
  if (sg.cap < table_bytes) {
    if (sg.host) cudaFreeHost(sg.host);
    sg.host = nullptr;
    sg.cap = 0;
    e = cudaHostAlloc(&sg.host, table_bytes, cudaHostAllocDefault);
    if (e != cudaSuccess) return cuda_fail(e, "gear_crown_lower_multi staging");
    sg.cap = table_bytes;
  }
  if (!sg.done) {
    e = cudaEventCreateWithFlags(&sg.done, cudaEventDisableTiming);
    if (e != cudaSuccess) return cuda_fail(e, "gear_crown_lower_multi staging");
  }
  multi_table(items, count, pl, (char*)sg.host);
  e = cudaMemcpyAsync(ws + pl.items_off, sg.host, table_bytes, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaEventRecord(sg.done, st);
  if (e != cudaSuccess) return cuda_fail(e, "gear_crown_lower_multi table upload");
  rc = multi_launch(pl, ws, st);
  if (rc == GEAR_OK) g_launches = 1;
  return rc;
}

extern "C" int gear_crown_multi_prepare(const gear_lower_args* items, int32_t count, void* workspace,
                                        int64_t workspace_bytes, gear_multi_plan** out) {
  g_launches = 0;
  if (!out) return fail(GEAR_E_INVALID, "gear_crown_multi_prepare: %s", "bad arguments");
  MultiPlan pl;
  int rc = multi_plan(items, count, pl);
  if (rc != GEAR_OK) return rc;
  if (pl.count > 0 && (!workspace || workspace_bytes < pl.bytes))
    return fail(GEAR_E_WORKSPACE, "gear_crown_multi_prepare: %s", "workspace too small");
  gear_multi_plan* p = new (std::nothrow) gear_multi_plan();
  if (!p) return fail(GEAR_E_NOMEM, "gear_crown_multi_prepare: %s", "host allocation");
  p->pl = pl;
  p->ws = (char*)workspace;
  if (pl.count > 0) {
    const size_t table_bytes = (size_t)(pl.start_off - pl.items_off) + (size_t)(pl.count + 1) * sizeof(int64_t);
    std::vector<char> host(table_bytes);
    multi_table(items, count, pl, host.data());
    cudaError_t e = cudaMemcpy(p->ws + pl.items_off, host.data(), table_bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) { delete p; return cuda_fail(e, "gear_crown_multi_prepare table upload"); }
  }
  *out = p;
  return GEAR_OK;
}

extern "C" int gear_crown_multi_launch(const gear_multi_plan* plan, void* stream) {
  g_launches = 0;
  if (!plan) return fail(GEAR_E_INVALID, "gear_crown_multi_launch: %s", "bad arguments");
  if (plan->pl.count == 0) return GEAR_OK;
  const int rc = multi_launch(plan->pl, plan->ws, (cudaStream_t)stream);
  if (rc == GEAR_OK) g_launches = 1;
  return rc;
}

extern "C" int gear_crown_multi_plan_destroy(gear_multi_plan* plan) {
  delete plan;
  return GEAR_OK;
}

// ------------------------------------------------------------------ branch and bound
namespace {
__global__ void u64_from_double(const double* v, unsigned long long* u) { *u = gear::bab::ordered_bits(*v); }
__global__ void double_from_u64(const unsigned long long* u, double* v) { *v = gear::bab::from_ordered_bits(*u); }
inline unsigned grid_for(int64_t work) { return (unsigned)((work + gear::bab::BT - 1) / gear::bab::BT); }
}  // namespace

extern "C" int64_t gear_bab_workspace_bytes(int64_t batch) {
  int64_t nblocks = (batch + gear::bab::BT - 1) / gear::bab::BT;
  return 64 + (nblocks + 64) * (int64_t)sizeof(int32_t);
}

extern "C" int gear_bab_prune(const double* lb, const double* thr, int64_t batch, int S, uint8_t* keep, int32_t* kept,
                              int32_t* n_kept, double* disc_min, void* workspace, int64_t ws_bytes, void* stream) {
  using namespace gear::bab;
  if (!n_kept || !disc_min || batch < 0 || S < 1 || (batch > 0 && (!lb || !thr || !keep || !kept)))
    return fail(GEAR_E_INVALID, "gear_bab_prune: %s", "bad arguments");
  if (!workspace || ws_bytes < gear_bab_workspace_bytes(batch))
    return fail(GEAR_E_WORKSPACE, "gear_bab_prune: %s", "workspace too small");
  cudaStream_t st = (cudaStream_t)stream;
  if (batch == 0) { cudaMemsetAsync(n_kept, 0, sizeof(int32_t), st); return GEAR_OK; }
  int64_t nblocks = (batch + BT - 1) / BT;
  if (nblocks > (int64_t)BT * 1024) return fail(GEAR_E_INVALID, "gear_bab_prune: %s", "batch too large");
  unsigned long long* u = (unsigned long long*)workspace;
  int32_t* counts = (int32_t*)((char*)workspace + 64);
  u64_from_double<<<1, 1, 0, st>>>(disc_min, u);
  prune_kernel<<<(unsigned)nblocks, BT, 0, st>>>(lb, thr, batch, S, keep, u);
  double_from_u64<<<1, 1, 0, st>>>(u, disc_min);
  count_kernel<<<(unsigned)nblocks, BT, 0, st>>>(keep, batch, counts);
  scan_counts_kernel<<<1, BT, 0, st>>>(counts, (int)nblocks, n_kept);
  compact_kernel<<<(unsigned)nblocks, BT, 0, st>>>(keep, batch, counts, kept);
  g_launches = 6;
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? GEAR_OK : cuda_fail(e, "gear_bab_prune");
}

extern "C" int gear_bab_branch(const double* lA, const double* lo, const double* hi, const double* lb,
                               const double* thr, int64_t batch, int S, int n, const double* root_width,
                               double coeff_thresh, double min_width_ratio, int32_t* split_idx, void* workspace,
                               int64_t ws_bytes, void* stream) {
  using namespace gear::bab;
  if (!lA || !lo || !hi || !lb || !thr || !split_idx || batch < 0 || S < 1 || n < 1)
    return fail(GEAR_E_INVALID, "gear_bab_branch: %s", "bad arguments");
  if (!workspace || ws_bytes < 64) return fail(GEAR_E_WORKSPACE, "gear_bab_branch: %s", "workspace too small");
  if (batch == 0) return GEAR_OK;
  cudaStream_t st = (cudaStream_t)stream;
  int* flag = (int*)workspace;
  cudaMemsetAsync(flag, 0, sizeof(int), st);
  int64_t nA = batch * (int64_t)S * n, nS = batch * (int64_t)S;
  unsigned g = grid_for(nA < (int64_t)1 << 26 ? nA : (int64_t)1 << 26);
  nonfinite_kernel<<<g, BT, 0, st>>>(lA, nA, lb, thr, nS, flag);
  branch_kernel<<<grid_for(batch * 32), BT, 0, st>>>(lA, lo, hi, batch, S, n, root_width, coeff_thresh,
                                                        min_width_ratio, flag, split_idx);
  g_launches = 2;
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? GEAR_OK : cuda_fail(e, "gear_bab_branch");
}

extern "C" int gear_bab_split(const double* lo, const double* hi, const int32_t* kept, int64_t n_kept, int n,
                              const int32_t* split_idx, const double* lb, const double* lA, const double* lbias,
                              int S, double* child_lo, double* child_hi, double* child_key, void* stream) {
  using namespace gear::bab;
  if (!lo || !hi || !kept || !split_idx || !child_lo || !child_hi || n_kept < 0 || n < 1)
    return fail(GEAR_E_INVALID, "gear_bab_split: %s", "bad arguments");
  if (n_kept == 0) return GEAR_OK;
  cudaStream_t st = (cudaStream_t)stream;
  split_kernel<<<grid_for(2 * n_kept * n), BT, 0, st>>>(lo, hi, kept, n_kept, n, split_idx, child_lo, child_hi);
  g_launches = 1;
  if (child_key) {
    if (!lb || !lA || !lbias || S < 1) return fail(GEAR_E_INVALID, "gear_bab_split: %s", "keys need lb, lA, lbias");
    child_keys_kernel<<<grid_for(2 * n_kept * 32), BT, 0, st>>>(lb, lA, lbias, child_lo, child_hi, kept, n_kept, S,
                                                                   n, child_key);
    g_launches = 2;
  }
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? GEAR_OK : cuda_fail(e, "gear_bab_split");
}

extern "C" int gear_queue_order(const double* key, const int64_t* id, const int32_t* slots, int64_t count,
                                int32_t* order, int64_t order_len, void* stream) {
  using namespace gear::bab;
  if (!key || !id || !slots || !order || count < 0) return fail(GEAR_E_INVALID, "gear_queue_order: %s", "bad arguments");
  int64_t n2 = 1;
  while (n2 < count) n2 <<= 1;
  if (order_len < n2) return fail(GEAR_E_WORKSPACE, "gear_queue_order: %s", "order buffer shorter than the next power of two");
  if (count == 0) return GEAR_OK;
  cudaStream_t st = (cudaStream_t)stream;
  cudaMemsetAsync(order, 0xff, n2 * sizeof(int32_t), st);             // padding = -1
  cudaMemcpyAsync(order, slots, count * sizeof(int32_t), cudaMemcpyDeviceToDevice, st);
  int launches = 0;
  if (n2 <= SORT_SMEM_MAX) {
    // the whole network in one CTA (one launch instead of log2(n2)(log2(n2)+1)/2)
    const size_t smem = (size_t)n2 * (sizeof(double) + sizeof(int64_t) + sizeof(int32_t));
    cudaError_t ea = set_smem_limit((const void*)bitonic_smem, (int)smem);
    if (ea != cudaSuccess) return cuda_fail(ea, "cudaFuncSetAttribute");
    bitonic_smem<<<1, SORT_THREADS, smem, st>>>(order, key, id, (int)n2);
    launches = 1;
  } else {
    for (int64_t k = 2; k <= n2; k <<= 1)
      for (int64_t j = k >> 1; j > 0; j >>= 1) {
        bitonic_step<<<grid_for(n2), BT, 0, st>>>(order, key, id, n2, count, (int)j, (int)k);
        ++launches;
      }
  }
  g_launches = launches;
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? GEAR_OK : cuda_fail(e, "gear_queue_order");
}

extern "C" int gear_queue_merge(const double* key, const int64_t* id, const int32_t* a, int64_t na, const int32_t* b,
                                int64_t nb, int32_t* out, void* stream) {
  using namespace gear::bab;
  if (!key || !id || !out || na < 0 || nb < 0 || (na > 0 && !a) || (nb > 0 && !b))
    return fail(GEAR_E_INVALID, "gear_queue_merge: %s", "bad arguments");
  g_launches = 0;
  if (na + nb == 0) return GEAR_OK;
  merge_kernel<<<grid_for(na + nb), BT, 0, (cudaStream_t)stream>>>(key, id, a, na, b, nb, out);
  g_launches = 1;
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? GEAR_OK : cuda_fail(e, "gear_queue_merge");
}

extern "C" int gear_gather_rows(const double* src, const int32_t* rows, int64_t count, int64_t width, double* dst,
                                void* stream) {
  if (!src || !rows || !dst || count < 0 || width < 1) return fail(GEAR_E_INVALID, "gear_gather_rows: %s", "bad arguments");
  if (count == 0) return GEAR_OK;
  gear::bab::gather_rows_kernel<<<grid_for(count * width), gear::bab::BT, 0, (cudaStream_t)stream>>>(src, rows, count,
                                                                                                    width, dst);
  g_launches = 1;
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? GEAR_OK : cuda_fail(e, "gear_gather_rows");
}

extern "C" int gear_scatter_rows(const double* src, const int32_t* rows, int64_t count, int64_t width, double* dst,
                                 void* stream) {
  if (!src || !rows || !dst || count < 0 || width < 1) return fail(GEAR_E_INVALID, "gear_scatter_rows: %s", "bad arguments");
  if (count == 0) return GEAR_OK;
  gear::bab::scatter_rows_kernel<<<grid_for(count * width), gear::bab::BT, 0, (cudaStream_t)stream>>>(src, rows, count,
                                                                                                     width, dst);
  g_launches = 1;
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? GEAR_OK : cuda_fail(e, "gear_scatter_rows");
}

extern "C" int gear_clip_domains(double* x_L, double* x_U, const double* thr, const double* lA, const double* lbias,
                                 const int32_t* parent, int64_t batch, int S, int n, int num_iters,
                                 uint8_t* nonempty, void* stream) {
  if (!x_L || !x_U || !thr || !lA || !lbias || batch < 0 || S < 1 || n < 1 || num_iters < 1)
    return fail(GEAR_E_INVALID, "gear_clip_domains: %s", "bad arguments");
  if (batch == 0) return GEAR_OK;
  const size_t per = (size_t)3 * S * sizeof(double);
  int warps = 8;
  while (warps > 1 && per * warps > (size_t)(96 << 10)) warps >>= 1;
  if (per * warps > (size_t)(200 << 10)) return fail(GEAR_E_INVALID, "gear_clip_domains: %s", "too many rows");
  cudaError_t e = cudaFuncSetAttribute(gear::bab::clip_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(per * warps));
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
  gear::bab::clip_kernel<<<(unsigned)((batch + warps - 1) / warps), 32 * warps, per * warps, (cudaStream_t)stream>>>(
      x_L, x_U, thr, lA, lbias, parent, batch, S, n, num_iters, nonempty);
  g_launches = 1;
  e = cudaGetLastError();
  return e == cudaSuccess ? GEAR_OK : cuda_fail(e, "gear_clip_domains");
}

extern "C" int gear_bab_child_keys(const double* lb, const double* lA, const double* lbias, const double* child_lo,
                                   const double* child_hi, const int32_t* kept, int64_t n_kept, int S, int n,
                                   double* child_key, void* stream) {
  using namespace gear::bab;
  if (!lb || !lA || !lbias || !child_lo || !child_hi || !kept || !child_key || n_kept < 0 || S < 1 || n < 1)
    return fail(GEAR_E_INVALID, "gear_bab_child_keys: %s", "bad arguments");
  if (n_kept == 0) return GEAR_OK;
  child_keys_kernel<<<grid_for(2 * n_kept * 32), BT, 0, (cudaStream_t)stream>>>(lb, lA, lbias, child_lo, child_hi, kept,
                                                                              n_kept, S, n, child_key);
  g_launches = 1;
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? GEAR_OK : cuda_fail(e, "gear_bab_child_keys");
}

extern "C" int gear_bab_compact(const uint8_t* keep, int64_t batch, int32_t* kept, int32_t* n_kept, void* workspace,
                                int64_t ws_bytes, void* stream) {
  using namespace gear::bab;
  if (!n_kept || batch < 0 || (batch > 0 && (!keep || !kept)))
    return fail(GEAR_E_INVALID, "gear_bab_compact: %s", "bad arguments");
  if (!workspace || ws_bytes < gear_bab_workspace_bytes(batch))
    return fail(GEAR_E_WORKSPACE, "gear_bab_compact: %s", "workspace too small");
  cudaStream_t st = (cudaStream_t)stream;
  if (batch == 0) { cudaMemsetAsync(n_kept, 0, sizeof(int32_t), st); return GEAR_OK; }
  int64_t nblocks = (batch + BT - 1) / BT;
  if (nblocks > (int64_t)BT * 1024) return fail(GEAR_E_INVALID, "gear_bab_compact: %s", "batch too large");
  int32_t* counts = (int32_t*)((char*)workspace + 64);
  count_kernel<<<(unsigned)nblocks, BT, 0, st>>>(keep, batch, counts);
  scan_counts_kernel<<<1, BT, 0, st>>>(counts, (int)nblocks, n_kept);
  compact_kernel<<<(unsigned)nblocks, BT, 0, st>>>(keep, batch, counts, kept);
  g_launches = 3;
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? GEAR_OK : cuda_fail(e, "gear_bab_compact");
}

// ------------------------------------------------------------------ device-resident BaB queue
// The queue handle of gear_queue_* / gear_bab_step (bab_queue.cuh): slot arrays, ordered active
// list, free list and counters in one device block owned by the handle, plus the buffers of one
// iteration at the handle's batch size (popped rows' thresholds, CROWN outputs, keep mask, kept
// list, split indices, children, sort buffer).
struct gear_queue {
  gear::bq::QueueDev q;
  void* dev = nullptr;
  int device = 0;
  int64_t batch = 0, N2 = 1;
  int32_t* pslot = nullptr;
  double *thr = nullptr, *lb = nullptr, *lA = nullptr, *lbias = nullptr, *lb_ibp = nullptr, *root_width = nullptr;
  uint8_t* keep = nullptr;
  int32_t *kept = nullptr, *nk = nullptr, *nchild = nullptr, *split_idx = nullptr, *newslot = nullptr;
  int32_t* block_counts = nullptr;
  int* nonfinite = nullptr;
  double *clo = nullptr, *chi = nullptr, *ckey = nullptr;
};

namespace {
// Carve the handle's arrays out of one allocation (pass dev = nullptr to size it).
int64_t queue_layout(gear_queue* h, char* dev) {
  using namespace gear::bq;
  const int n = h->q.n, S = h->q.S;
  const int64_t cap = h->q.cap, B = h->batch;
  int64_t o = 0;
  auto take = [&](int64_t bytes) -> char* {
    char* p = dev ? dev + o : nullptr;
    o = align_up(o + bytes, kAlign);
    return p;
  };
  h->q.lo = (double*)take(cap * n * 8);
  h->q.hi = (double*)take(cap * n * 8);
  h->q.key = (double*)take(cap * S * 8);
  h->q.key0 = (double*)take(cap * 8);
  h->q.ids = (int64_t*)take(cap * 8);
  h->q.active = (int32_t*)take(cap * 4);
  h->q.merged = (int32_t*)take(cap * 4);
  h->q.free_list = (int32_t*)take(cap * 4);
  h->q.counters = (int64_t*)take(C_COUNT * 8);
  h->q.disc_min = (unsigned long long*)take(8);
  h->q.root_lo = (double*)take(n * 8);
  h->q.root_hi = (double*)take(n * 8);
  h->root_width = (double*)take(n * 8);
  h->pslot = (int32_t*)take(B * 4);
  h->thr = (double*)take(B * S * 8);
  h->lb = (double*)take(B * S * 8);
  h->lA = (double*)take(B * S * n * 8);
  h->lbias = (double*)take(B * S * 8);
  h->lb_ibp = (double*)take(B * S * 8);
  h->keep = (uint8_t*)take(B);
  h->kept = (int32_t*)take(B * 4);
  h->nk = (int32_t*)take(4);
  h->nchild = (int32_t*)take(4);
  h->split_idx = (int32_t*)take(B * 4);
  h->newslot = (int32_t*)take(h->N2 * 4);
  h->block_counts = (int32_t*)take(((B + gear::bab::BT - 1) / gear::bab::BT + 64) * 4);
  h->nonfinite = (int*)take(4);
  h->clo = (double*)take(2 * B * n * 8);
  h->chi = (double*)take(2 * B * n * 8);
  h->ckey = (double*)take(2 * B * S * 8);
  return o;
}

__global__ void queue_init_kernel(gear::bq::QueueDev q, const double* root_lo, const double* root_hi,
                                  double* root_width) {
  using namespace gear::bq;
  const int64_t t = (int64_t)blockIdx.x * gear::bab::BT + threadIdx.x;
  // the root domain in slot 0 (key -inf, id 0); slots 1..cap-1 free
  if (t < q.n) {
    q.lo[t] = root_lo[t];
    q.hi[t] = root_hi[t];
    q.root_lo[t] = root_lo[t];
    q.root_hi[t] = root_hi[t];
    root_width[t] = root_hi[t] - root_lo[t];
  }
  if (t < q.S) q.key[t] = -INFINITY;
  if (t < q.cap - 1) q.free_list[t] = (int32_t)(q.cap - 1 - t);
  if (t == 0) {
    q.key0[0] = -INFINITY;
    q.ids[0] = 0;
    q.active[0] = 0;
    for (int c = 0; c < C_COUNT; ++c) q.counters[c] = 0;
    q.counters[C_ACTIVE] = 1;
    q.counters[C_FREE] = q.cap - 1;
    q.counters[C_NEXT_ID] = 1;
    *q.disc_min = gear::bab::ordered_bits(INFINITY);
  }
}

// sort the N2 new slot entries (children first, -1 padding last) by (key desc, id asc)
int queue_sort_new(gear_queue* h, cudaStream_t st) {
  using namespace gear::bab;
  if (h->N2 <= SORT_SMEM_MAX) {
    const size_t smem = (size_t)h->N2 * (sizeof(double) + sizeof(int64_t) + sizeof(int32_t));
    cudaError_t e = set_smem_limit((const void*)bitonic_smem, (int)smem);
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
    bitonic_smem<<<1, SORT_THREADS, smem, st>>>(h->newslot, h->q.key0, h->q.ids, (int)h->N2);
    return 1;
  }
  int launches = 0;
  for (int64_t k = 2; k <= h->N2; k <<= 1)
    for (int64_t j = k >> 1; j > 0; j >>= 1) {
      bitonic_step<<<grid_for(h->N2), BT, 0, st>>>(h->newslot, h->q.key0, h->q.ids, h->N2, h->N2, (int)j, (int)k);
      ++launches;
    }
  return launches;
}

// the domains in h->clo / chi / ckey (mult x *h->nk of them) into the active list
int queue_push_rows(gear_queue* h, int mult, cudaStream_t st) {
  using namespace gear::bq;
  push_plan_kernel<<<1, 1, 0, st>>>(h->q, h->nk, mult, h->nchild);
  const int w = h->q.n > h->q.S ? h->q.n : h->q.S;
  push_scatter_kernel<<<grid_for(h->N2 * w), BT, 0, st>>>(h->q, h->nchild, h->clo, h->chi, h->ckey, h->N2, h->newslot);
  int launches = 2;
  const int s = queue_sort_new(h, st);
  if (s < 0) return s;
  launches += s;
  merge_dev_kernel<<<grid_for(h->q.cap), BT, 0, st>>>(h->q, h->nchild, h->newslot);
  merge_copy_kernel<<<grid_for(h->q.cap), BT, 0, st>>>(h->q, h->nchild);
  push_commit_kernel<<<1, 1, 0, st>>>(h->q, h->nchild);
  return launches + 3;
}
}  // namespace

extern "C" int gear_queue_create(int n, int S, int64_t capacity, int64_t batch, const double* root_lo,
                                 const double* root_hi, gear_queue** out) {
  if (!out || n < 1 || S < 1 || batch < 1 || capacity < 2 * batch + 1 || capacity > ((int64_t)1 << 31) - 1 ||
      !root_lo || !root_hi)
    return fail(GEAR_E_INVALID, "gear_queue_create: %s", "bad arguments (capacity must exceed 2 x batch)");
  gear_queue* h = new (std::nothrow) gear_queue();
  if (!h) return fail(GEAR_E_NOMEM, "gear_queue_create: %s", "host allocation");
  h->q.n = n;
  h->q.S = S;
  h->q.cap = capacity;
  h->batch = batch;
  while (h->N2 < 2 * batch) h->N2 <<= 1;
  const int64_t bytes = queue_layout(h, nullptr);
  cudaError_t e = cudaGetDevice(&h->device);
  if (e == cudaSuccess) e = cudaMalloc(&h->dev, bytes);
  if (e != cudaSuccess) { delete h; return cuda_fail(e, "cudaMalloc(queue)"); }
  queue_layout(h, (char*)h->dev);
  double* root = nullptr;
  e = cudaMalloc(&root, 2 * n * sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpy(root, root_lo, n * sizeof(double), cudaMemcpyDefault);
  if (e == cudaSuccess) e = cudaMemcpy(root + n, root_hi, n * sizeof(double), cudaMemcpyDefault);
  if (e == cudaSuccess) {
    const int64_t m = capacity > n ? capacity : n;
    queue_init_kernel<<<grid_for(m > S ? m : S), gear::bab::BT>>>(h->q, root, root + n, h->root_width);
    e = cudaDeviceSynchronize();
  }
  if (root) cudaFree(root);
  if (e != cudaSuccess) { cudaFree(h->dev); delete h; return cuda_fail(e, "gear_queue_create"); }
  *out = h;
  return GEAR_OK;
}

extern "C" int gear_queue_destroy(gear_queue* q) {
  if (!q) return GEAR_OK;
  if (q->dev) cudaFree(q->dev);
  delete q;
  return GEAR_OK;
}

namespace {
__global__ void append_free_kernel(int32_t* free_list, int64_t nf, int64_t first, int64_t count) {
  const int64_t i = (int64_t)blockIdx.x * gear::bab::BT + threadIdx.x;
  if (i < count) free_list[nf + i] = (int32_t)(first + i);
}
}  // namespace

extern "C" int gear_queue_reserve(gear_queue* q, int64_t capacity, void* stream) {
  using namespace gear::bq;
  if (!q || capacity > ((int64_t)1 << 31) - 1) return fail(GEAR_E_INVALID, "gear_queue_reserve: %s", "bad arguments");
  if (capacity <= q->q.cap) return GEAR_OK;
  cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
  int64_t cnt[C_COUNT];
  if (e == cudaSuccess) e = cudaMemcpy(cnt, q->q.counters, sizeof(cnt), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "gear_queue_reserve");
  gear_queue nh = *q;
  const int64_t old = q->q.cap;
  const int n = q->q.n, S = q->q.S;
  nh.q.cap = capacity;
  const int64_t bytes = queue_layout(&nh, nullptr);
  e = cudaMalloc(&nh.dev, bytes);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(queue)");
  queue_layout(&nh, (char*)nh.dev);
  struct Copy { void* dst; const void* src; size_t bytes; };
  const Copy copies[] = {
      {nh.q.lo, q->q.lo, (size_t)old * n * 8}, {nh.q.hi, q->q.hi, (size_t)old * n * 8},
      {nh.q.key, q->q.key, (size_t)old * S * 8}, {nh.q.key0, q->q.key0, (size_t)old * 8},
      {nh.q.ids, q->q.ids, (size_t)old * 8}, {nh.q.active, q->q.active, (size_t)old * 4},
      {nh.q.free_list, q->q.free_list, (size_t)old * 4}, {nh.q.counters, q->q.counters, (size_t)C_COUNT * 8},
      {nh.q.disc_min, q->q.disc_min, 8}, {nh.q.root_lo, q->q.root_lo, (size_t)n * 8},
      {nh.q.root_hi, q->q.root_hi, (size_t)n * 8}, {nh.root_width, q->root_width, (size_t)n * 8}};
  for (const Copy& c : copies) {
    e = cudaMemcpy(c.dst, c.src, c.bytes, cudaMemcpyDeviceToDevice);
    if (e != cudaSuccess) { cudaFree(nh.dev); return cuda_fail(e, "gear_queue_reserve copy"); }
  }
  const int64_t nf = cnt[C_FREE], add = capacity - old;
  append_free_kernel<<<grid_for(add), gear::bab::BT>>>(nh.q.free_list, nf, old, add);
  cnt[C_FREE] = nf + add;
  e = cudaMemcpy(nh.q.counters, cnt, sizeof(cnt), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) { cudaFree(nh.dev); return cuda_fail(e, "gear_queue_reserve"); }
  cudaFree(q->dev);
  *q = nh;
  return GEAR_OK;
}

extern "C" int64_t gear_queue_capacity(const gear_queue* q) { return q ? q->q.cap : -1; }

extern "C" int gear_queue_counters(const gear_queue* q, int64_t* counters, double* dual, void* stream) {
  if (!q || !counters) return fail(GEAR_E_INVALID, "gear_queue_counters: %s", "bad arguments");
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaMemcpyAsync(counters, q->q.counters, gear::bq::C_COUNT * sizeof(int64_t), cudaMemcpyDefault, st);
  if (e == cudaSuccess && dual) {
    gear::bq::dual_bound_kernel<<<1, 1, 0, st>>>(q->q, dual);
    e = cudaGetLastError();
  }
  return e == cudaSuccess ? GEAR_OK : cuda_fail(e, "gear_queue_counters");
}

extern "C" int gear_queue_size(const gear_queue* q, int64_t* open, void* stream) {
  if (!q || !open) return fail(GEAR_E_INVALID, "gear_queue_size: %s", "bad arguments");
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaMemcpyAsync(open, q->q.counters + gear::bq::C_ACTIVE, sizeof(int64_t), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  return e == cudaSuccess ? GEAR_OK : cuda_fail(e, "gear_queue_size");
}

extern "C" int gear_queue_push(gear_queue* q, const double* lo, const double* hi, const double* key, int64_t count,
                               void* stream) {
  g_launches = 0;
  if (!q || count < 0 || count > 2 * q->batch || (count > 0 && (!lo || !hi || !key)))
    return fail(GEAR_E_INVALID, "gear_queue_push: %s", "bad arguments (at most 2 x batch domains per push)");
  if (count == 0) return GEAR_OK;
  cudaStream_t st = (cudaStream_t)stream;
  const int n = q->q.n, S = q->q.S;
  cudaError_t e = cudaMemcpyAsync(q->clo, lo, count * n * sizeof(double), cudaMemcpyDeviceToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(q->chi, hi, count * n * sizeof(double), cudaMemcpyDeviceToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(q->ckey, key, count * S * sizeof(double), cudaMemcpyDeviceToDevice, st);
  if (e != cudaSuccess) return cuda_fail(e, "gear_queue_push copy");
  gear::bq::set_count_kernel<<<1, 1, 0, st>>>(q->nk, (int32_t)count);
  const int l = queue_push_rows(q, 1, st);
  if (l < 0) return l;
  g_launches = l + 1;
  e = cudaGetLastError();
  return e == cudaSuccess ? GEAR_OK : cuda_fail(e, "gear_queue_push");
}

extern "C" int gear_queue_pop(gear_queue* q, double* lo_out, double* hi_out, void* stream) {
  if (!q || !lo_out || !hi_out) return fail(GEAR_E_INVALID, "gear_queue_pop: %s", "bad arguments");
  cudaStream_t st = (cudaStream_t)stream;
  gear::bq::pop_gather_kernel<<<grid_for(q->batch * q->q.n), gear::bab::BT, 0, st>>>(q->q, q->batch, lo_out, hi_out,
                                                                                     q->pslot);
  gear::bq::pop_commit_kernel<<<1, gear::bab::BT, 0, st>>>(q->q, q->batch, q->pslot);
  g_launches = 2;
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? GEAR_OK : cuda_fail(e, "gear_queue_pop");
}

extern "C" int64_t gear_bab_step_workspace_bytes(const gear_dag* dag, int64_t batch) {
  if (!dag || batch < 1) return -1;
  return align_up(gear_crown_workspace_bytes(dag, batch), kAlign) + kAlign;
}

static int bab_step_after_bound(gear_queue* q, const double* lo, const double* hi, const double* lb, const double* lA,
                                const double* lbias, const double* incumbent, const double* rhs, double sb_coeff_thresh,
                                double sb_min_width_ratio, cudaStream_t st) {
  using namespace gear;
  const int64_t B = q->batch;
  const int n = q->q.n, S = q->q.S;
  // prune against the thresholds (incumbent read on the device), drop the padding rows, compact
  bq::thresholds_kernel<<<grid_for(B * S), bab::BT, 0, st>>>(incumbent, rhs, B, S, q->thr);
  const int64_t nblocks = (B + bab::BT - 1) / bab::BT;
  bab::prune_kernel<<<(unsigned)nblocks, bab::BT, 0, st>>>(lb, q->thr, B, S, q->keep, q->q.disc_min);
  bq::mask_padding_kernel<<<(unsigned)nblocks, bab::BT, 0, st>>>(q->q.counters, B, q->keep);
  bab::count_kernel<<<(unsigned)nblocks, bab::BT, 0, st>>>(q->keep, B, q->block_counts);
  bab::scan_counts_kernel<<<1, bab::BT, 0, st>>>(q->block_counts, (int)nblocks, q->nk);
  bab::compact_kernel<<<(unsigned)nblocks, bab::BT, 0, st>>>(q->keep, B, q->block_counts, q->kept);
  // branch: SB score, top-1, width guard
  cudaError_t e = cudaMemsetAsync(q->nonfinite, 0, sizeof(int), st);
  if (e != cudaSuccess) return cuda_fail(e, "gear_bab_step");
  const int64_t nA = B * (int64_t)S * n, nS = B * (int64_t)S;
  bab::nonfinite_kernel<<<grid_for(nA < ((int64_t)1 << 26) ? nA : ((int64_t)1 << 26)), bab::BT, 0, st>>>(
      lA, nA, lb, q->thr, nS, q->nonfinite);
  bab::branch_kernel<<<grid_for(B * 32), bab::BT, 0, st>>>(lA, lo, hi, B, S, n, q->root_width, sb_coeff_thresh,
                                                           sb_min_width_ratio, q->nonfinite, q->split_idx);
  // split the kept parents, key the children, push them
  bq::split_dev_kernel<<<grid_for(2 * B * n), bab::BT, 0, st>>>(lo, hi, q->kept, q->nk, n, q->split_idx, q->clo,
                                                                  q->chi);
  bq::child_keys_dev_kernel<<<grid_for(2 * B * 32), bab::BT, 0, st>>>(lb, lA, lbias, q->clo, q->chi, q->kept, q->nk, S,
                                                                      n, q->ckey);
  const int l = queue_push_rows(q, 2, st);
  if (l < 0) return l;
  e = cudaGetLastError();
  return e == cudaSuccess ? 11 + l : cuda_fail(e, "gear_bab_step");
}

extern "C" int gear_bab_step(gear_queue* q, const gear_dag* dag, const double* lo, const double* hi,
                             const double* incumbent, const double* rhs, double sb_coeff_thresh,
                             double sb_min_width_ratio, int ibp_enhancement, void* workspace, int64_t ws_bytes,
                             void* stream) {
  using namespace gear;
  g_launches = 0;
  if (!q || !dag || !lo || !hi || !incumbent || (q->q.S > 1 && !rhs))
    return fail(GEAR_E_INVALID, "gear_bab_step: %s", "bad arguments");
  if (dag->hdr[H_N] != q->q.n || dag->hdr[H_S] != q->q.S || dag->hdr[H_RETA] == 0)
    return fail(GEAR_E_INVALID, "gear_bab_step: %s", "program and queue differ in width or rows, or the program has no A");
  const int64_t B = q->batch;
  if (!workspace || ws_bytes < gear_bab_step_workspace_bytes(dag, B))
    return fail(GEAR_E_WORKSPACE, "gear_bab_step: %s", "workspace too small");
  // bound: CROWN over the popped batch (padding rows included), with the IBP pass when asked
  int rc = crown_lower_impl(dag, lo, hi, B, nullptr, q->lb, q->lA, q->lbias, ibp_enhancement ? q->lb_ibp : nullptr,
                            workspace, ws_bytes, stream);
  if (rc != GEAR_OK) return rc;
  const int crown = g_launches;
  const int l = bab_step_after_bound(q, lo, hi, q->lb, q->lA, q->lbias, incumbent, rhs, sb_coeff_thresh,
                                     sb_min_width_ratio, (cudaStream_t)stream);
  if (l < 0) return l;
  g_launches = crown + l;
  return GEAR_OK;
}

extern "C" int gear_bab_step_bounded(gear_queue* q, const double* lo, const double* hi, const double* lb,
                                     const double* lA, const double* lbias, const double* incumbent, const double* rhs,
                                     double sb_coeff_thresh, double sb_min_width_ratio, void* stream) {
  g_launches = 0;
  if (!q || !lo || !hi || !lb || !lA || !lbias || !incumbent || (q->q.S > 1 && !rhs))
    return fail(GEAR_E_INVALID, "gear_bab_step_bounded: %s", "bad arguments");
  const int l = bab_step_after_bound(q, lo, hi, lb, lA, lbias, incumbent, rhs, sb_coeff_thresh, sb_min_width_ratio,
                                     (cudaStream_t)stream);
  if (l < 0) return l;
  g_launches = l;
  return GEAR_OK;
}

// ------------------------------------------------------------------ rigorous LP dual bound
extern "C" int gear_dual_lower_bound(const int32_t* colptr, const int32_t* rows, const int32_t* perm, const double* val,
                                     int val_batched, int64_t batch, int m, int n, int nnz, const double* c,
                                     const double* c0, const double* h, const double* l, const double* u,
                                     const double* y, const double* tol, const double* c_err, const double* c0_err,
                                     int infeasibility, double* lb, double* E, uint8_t* dd, void* stream) {
  g_launches = 0;
  if (!colptr || (nnz > 0 && (!rows || !perm || !val)) || !h || !l || !u || !y || !lb || batch < 0 || m < 0 || n < 0 ||
      nnz < 0)
    return fail(GEAR_E_INVALID, "gear_dual_lower_bound: %s", "bad arguments");
  if (batch == 0) return GEAR_OK;
  const size_t smem = (size_t)m * sizeof(double);
  if (smem > (size_t)(200 << 10)) return fail(GEAR_E_INVALID, "gear_dual_lower_bound: %s", "too many rows");
  cudaError_t e = cudaFuncSetAttribute(gear::dual::dual_bound_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
  gear::dual::Lp p;
  p.colptr = colptr; p.rows = rows; p.perm = perm; p.val = val; p.val_batched = val_batched;
  p.c = c; p.c0 = c0; p.h = h; p.l = l; p.u = u; p.y = y; p.tol = tol; p.c_err = c_err; p.c0_err = c0_err;
  p.lb = lb; p.E = E; p.dd = dd; p.B = batch; p.m = m; p.n = n; p.nnz = nnz; p.infeasibility = infeasibility;
  gear::dual::dual_bound_kernel<<<(unsigned)batch, gear::dual::DT, smem, (cudaStream_t)stream>>>(p);
  g_launches = 1;
  e = cudaGetLastError();
  return e == cudaSuccess ? GEAR_OK : cuda_fail(e, "gear_dual_lower_bound");
}

// ------------------------------------------------------------------ constrained concretisation
namespace {
struct CcLayout {
  size_t d, score, infeasible, uncovered, nkeep, glob, total;
};
CcLayout cc_layout(int64_t batch, int K) {
  CcLayout L;
  size_t o = 0;
  auto take = [&](size_t bytes) { size_t at = o; o += (bytes + 255) / 256 * 256; return at; };
  L.d = take((size_t)batch * K * sizeof(double));
  L.score = take((size_t)batch * K * sizeof(double));
  L.infeasible = take((size_t)batch * sizeof(int));
  L.uncovered = take((size_t)batch * sizeof(int));
  L.nkeep = take((size_t)batch * sizeof(int));
  L.glob = take(2 * sizeof(int));
  L.total = o;
  return L;
}
}  // namespace

extern "C" int64_t gear_constrained_workspace_bytes(int64_t batch, int K) {
  if (batch < 0 || K < 0) return -1;
  return (int64_t)cc_layout(batch, K).total;
}

extern "C" int gear_constrained_lower(const double* x_L, const double* x_U, int64_t batch, int n, const double* obj,
                                      int H, const double* A, const double* b, int K, int max_rows, double* lb,
                                      uint8_t* infeasible, void* workspace, int64_t ws_bytes, void* stream) {
  g_launches = 0;
  if (!x_L || !x_U || !obj || !lb || batch < 0 || n < 1 || H < 1 || K < 0 || max_rows < 0 || (K > 0 && (!A || !b)))
    return fail(GEAR_E_INVALID, "gear_constrained_lower: %s", "bad arguments");
  if (batch == 0) return GEAR_OK;
  const CcLayout L = cc_layout(batch, K);
  if (!workspace || ws_bytes < (int64_t)L.total)
    return fail(GEAR_E_WORKSPACE, "gear_constrained_lower: %s", "workspace smaller than gear_constrained_workspace_bytes");
  const size_t per = gear::cc::sweep_smem_per_warp(n, K);
  int warps = (int)((size_t)(160 << 10) / per);
  if (warps > 4) warps = 4;
  if (warps < 1) {
    if (per > (size_t)(227 << 10))
      return fail(GEAR_E_INVALID, "gear_constrained_lower: %s", "too many variables or rows for one warp's shared memory");
    warps = 1;
  }
  cudaStream_t st = (cudaStream_t)stream;
  char* ws = (char*)workspace;
  gear::cc::Work w;
  w.xL = x_L; w.xU = x_U; w.obj = obj; w.A = A; w.b = b;
  w.d = (double*)(ws + L.d);
  w.score = (double*)(ws + L.score);
  w.infeasible = (int*)(ws + L.infeasible);
  w.uncovered = (int*)(ws + L.uncovered);
  w.nkeep = (int*)(ws + L.nkeep);
  w.glob = (int*)(ws + L.glob);
  w.lb = lb;
  w.infeasible_out = infeasible;
  w.B = batch; w.X = n; w.H = H; w.K = K; w.max_rows = max_rows;
  // the per-box counters and flags start at zero on every call
  cudaError_t e = cudaMemsetAsync(ws + L.infeasible, 0, L.total - L.infeasible, st);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync");
  int launches = 0;
  if (K > 0) {
    const int64_t rows = batch * K;
    gear::cc::concretize_rows_kernel<<<(unsigned)((rows + 7) / 8), 256, 0, st>>>(w);
    gear::cc::concretize_boxes_kernel<<<(unsigned)((batch + 255) / 256), 256, 0, st>>>(w);
    launches += 2;
  }
  const size_t smem = per * warps;
  e = cudaFuncSetAttribute(gear::cc::concretize_sweep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
  const int64_t items = batch * H;
  gear::cc::concretize_sweep_kernel<<<(unsigned)((items + warps - 1) / warps), 32 * warps, smem, st>>>(w);
  g_launches = launches + 1;
  e = cudaGetLastError();
  return e == cudaSuccess ? GEAR_OK : cuda_fail(e, "gear_constrained_lower");
}

// ------------------------------------------------------------------ CROWN under cut rows
namespace {
struct CutsLayout {
  size_t plain, cc, obj, v, total;
  CcLayout c;
};
int cuts_rows_max(const gear_dag* d) {
  int h = 1;
  for (int p = 0; p < d->hdr[gear::H_NPASSES]; ++p) {
    const int32_t* pr = d->passes.data() + (size_t)p * gear::PASS_REC;
    h = std::max(h, pr[gear::P_SIDES] * pr[gear::P_S]);
  }
  return h;
}
bool cuts_ok(const gear_dag* d) {
  if (!plain_ok(d)) return false;
  for (int p = 0; p < d->hdr[gear::H_NPASSES]; ++p)
    if (d->passes[(size_t)p * gear::PASS_REC + gear::P_NFOLD] != 0) return false;
  return true;
}
CutsLayout cuts_layout(const gear_dag* d, int64_t batch, int K) {
  CutsLayout L;
  size_t o = 0;
  auto take = [&](size_t bytes) { size_t at = o; o += (bytes + 255) / 256 * 256; return at; };
  const int H = cuts_rows_max(d), n = d->hdr[gear::H_N];
  L.plain = take((size_t)batch * d->slot_doubles * sizeof(double));
  L.c = cc_layout(batch, K);
  L.cc = take(L.c.total);
  L.obj = take((size_t)batch * H * n * sizeof(double));
  L.v = take((size_t)batch * H * sizeof(double));
  L.total = o;
  return L;
}
}  // namespace

extern "C" int64_t gear_crown_cuts_workspace_bytes(const gear_dag* dag, int64_t batch, int K) {
  if (!cuts_ok(dag) || batch < 0 || K < 0) return -1;
  return (int64_t)cuts_layout(dag, batch, K).total;
}

extern "C" int gear_crown_lower_cuts(const gear_dag* dag, const double* x_L, const double* x_U, int64_t batch,
                                     const double* C, const double* cut_A, const double* cut_b, int K, int max_rows,
                                     double* lb, double* lA, double* lbias, double* lb_ibp, void* workspace,
                                     int64_t workspace_bytes, void* stream) {
  g_launches = 0;
  if (!dag || batch < 0 || K < 0 || max_rows < 0)
    return fail(GEAR_E_INVALID, "gear_crown_lower_cuts: %s", "bad arguments");
  if (!cuts_ok(dag))
    return fail(GEAR_E_INVALID, "gear_crown_lower_cuts: %s",
                "needs a box-per-CTA program compiled for cut rows (working set in global memory, no folded passes)");
  if (batch == 0) return GEAR_OK;
  if (!x_L || !x_U || !lb || !lA || (K > 0 && (!cut_A || !cut_b)))
    return fail(GEAR_E_INVALID, "gear_crown_lower_cuts: %s", "bad arguments");
  const int n = dag->hdr[gear::H_N];
  const CutsLayout L = cuts_layout(dag, batch, K);
  if (!workspace || workspace_bytes < (int64_t)L.total)
    return fail(GEAR_E_WORKSPACE, "gear_crown_lower_cuts: %s", "workspace smaller than gear_crown_cuts_workspace_bytes");
  const size_t per = gear::cc::sweep_smem_per_warp(n, K);
  if (per > (size_t)(227 << 10))
    return fail(GEAR_E_INVALID, "gear_crown_lower_cuts: %s", "too many variables or rows for one warp's shared memory");
  int warps = (int)((size_t)(160 << 10) / per);
  warps = std::max(1, std::min(warps, 4));
  cudaStream_t st = (cudaStream_t)stream;
  char* ws = (char*)workspace;
  char* cc = ws + L.cc;
  CutRun cut;
  cut.w.xL = x_L; cut.w.xU = x_U; cut.w.A = cut_A; cut.w.b = cut_b;
  cut.w.d = (double*)(cc + L.c.d);
  cut.w.score = (double*)(cc + L.c.score);
  cut.w.infeasible = (int*)(cc + L.c.infeasible);
  cut.w.uncovered = (int*)(cc + L.c.uncovered);
  cut.w.nkeep = (int*)(cc + L.c.nkeep);
  cut.w.glob = (int*)(cc + L.c.glob);
  cut.w.infeasible_out = nullptr;
  cut.w.B = batch; cut.w.X = n; cut.w.K = K; cut.w.max_rows = max_rows;
  cut.w.obj = nullptr; cut.w.lb = nullptr; cut.w.H = 1;
  cut.obj = (double*)(ws + L.obj);
  cut.v = (double*)(ws + L.v);
  cut.warps = warps;
  cut.smem = per * warps;
  // the per-box counters and flags start at zero on every call
  cudaError_t e = cudaMemsetAsync(cc + L.c.infeasible, 0, L.c.total - L.c.infeasible, st);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync");
  e = cudaFuncSetAttribute(gear::cc::concretize_sweep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cut.smem);
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
  if (K > 0) {
    // rows: infeasibility / cover tests, centred offsets and worst-case values, once per call
    const int64_t rows = batch * K;
    gear::cc::concretize_rows_kernel<<<(unsigned)((rows + 7) / 8), 256, 0, st>>>(cut.w);
    gear::cc::concretize_boxes_kernel<<<(unsigned)((batch + 255) / 256), 256, 0, st>>>(cut.w);
    g_launches = 2;
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "gear_crown_lower_cuts rows");
  }
  return plain_impl(dag, x_L, x_U, batch, C, lb, lA, lbias, lb_ibp, ws + L.plain, (int64_t)(L.total - L.plain),
                    stream, &cut);
}

#ifdef GEAR_STEP_PROFILE
extern "C" int gear_profile_read(unsigned long long* out, int n) {
  cudaError_t e = cudaMemcpyFromSymbol(out, gear::g_step_cycles, sizeof(unsigned long long) * n);
  return e == cudaSuccess ? 0 : -4;
}
extern "C" int gear_profile_reset(void) {
  static unsigned long long zeros[8192];
  cudaError_t e = cudaMemcpyToSymbol(gear::g_step_cycles, zeros, sizeof(zeros));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(gear::g_op_cycles, zeros, sizeof(zeros));
  return e == cudaSuccess ? 0 : -4;
}
extern "C" int gear_profile_read_ops(unsigned long long* out, int n) {
  cudaError_t e = cudaMemcpyFromSymbol(out, gear::g_op_cycles, sizeof(unsigned long long) * n);
  return e == cudaSuccess ? 0 : -4;
}
#endif

/* gear_b200: C ABI of the B200 (sm_100a) CROWN bound-propagation engine.
 *
 * Every entry point is extern "C", takes plain pointers and sizes, and returns an int
 * status: 0 on success, a negative GEAR_E* code on failure, with a message available from
 * gear_last_error() (thread-local). No exception crosses the ABI.
 *
 * Memory: the caller owns every buffer it passes (x_L, x_U, C, outputs, workspace) and
 * they must be device memory on the current device; the library never frees them.
 * A gear_dag handle owns the device copy of its compiled program and is released by
 * gear_dag_destroy. Calls on one handle from several host threads must be serialised by
 * the caller; calls on one stream run in stream order.
 *
 * Reference interfaces replaced (paths in the reference project):
 *   gear_dag_create   <- BoundedModule(model, x0, bound_opts)           solver/auto_LiRPA/bound_general.py:87
 *                        (the DAG arrives compiled by gear_b200/program.py from the same
 *                        node program; the gear_program seam is bound_general.py:817-829)
 *   gear_crown_lower  <- BoundedModule.compute_bounds(x=(BoundedTensor(x0,
 *                        PerturbationLpNorm(x_L, x_U)),), C, method='CROWN',
 *                        bound_upper=False, return_A=True, needed_A_dict)  bound_general.py:1275
 *                        as called by get_lower_bound_naive (complete_verifier/input_split/bounding.py:317)
 *   gear_bab_prune    <- get_remaining_index, solving mode        complete_verifier/input_split/branching_domains.py:412-558
 *                        + discarded-threshold minimum              batch_branch_and_bound.py:628-636
 *   gear_bab_branch   <- input_split_branching, method 'sb', sb_sum complete_verifier/input_split/branching_heuristics.py:25-202
 *   gear_bab_split    <- input_split_parallel                      complete_verifier/input_split/split.py:26-122
 *                        + child keys (_raise_child_keys)          batch_branch_and_bound.py:189-225
 *   gear_queue_order  <- UnsortedInputDomainList.sort / pick_out_batch  branching_domains.py:1171-1240, :831-962
 *   gear_gather_rows, gear_scatter_rows <- TensorStorage pop / append    complete_verifier/input_split/tensor_storage.py:351-408
 *   gear_clip_domains <- clip_domains / _clip_main_fn (lower planes)  complete_verifier/input_split/clip.py:138-486
 *   gear_bab_child_keys <- _raise_child_keys                      batch_branch_and_bound.py:189-225
 *   gear_bab_compact  <- the index compaction of filter_verified_domains  branching_domains.py:238-410
 *   gear_dual_lower_bound <- dual_lower_bound / certify_infeasible    complete_verifier/nlp_solver/rigorous_dual.py:1-238
 *   gear_constrained_lower <- sort_out_constr_batches + constraints_solving(sign=-1)
 *                        (+ drop_redundant_constraints, _solve_dual_var)  solver/auto_LiRPA/concretize_func.py:168-850
 *   gear_crown_lower_cuts <- compute_bounds with PerturbationLpNorm(x_L, x_U, constraints=(A, b))
 *                        bound_general.py:1275, perturbations.py:129-199, concretize_func.py:431-850
 */
#ifndef GEAR_B200_H
#define GEAR_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GEAR_OK 0
#define GEAR_E_INVALID (-1)     /* bad argument or malformed program */
#define GEAR_E_NOMEM (-2)       /* device allocation failed (maps to torch.OutOfMemoryError) */
#define GEAR_E_TIMEOUT (-3)     /* a bounded device wait expired */
#define GEAR_E_CUDA (-4)        /* a CUDA runtime error */
#define GEAR_E_WORKSPACE (-5)   /* workspace smaller than gear_crown_workspace_bytes */

typedef struct gear_dag gear_dag;

/* Upload a compiled program (gear_b200/program.py Program: header, node, step, pass and
 * op records, int pool, float64 pool) to the current device. */
int gear_dag_create(const int32_t* header, int64_t header_len,
                    const int32_t* nodes, int64_t n_nodes_ints,
                    const int32_t* steps, int64_t n_steps_ints,
                    const int32_t* passes, int64_t n_passes_ints,
                    const int32_t* ops, int64_t n_ops_ints,
                    const int32_t* int_pool, int64_t n_int,
                    const double* dbl_pool, int64_t n_dbl,
                    gear_dag** out);

int gear_dag_destroy(gear_dag* dag);

/* Bytes of device workspace gear_crown_lower needs for a batch of `batch` boxes
 * (bounded by the number of resident CTAs, not by the batch). */
int64_t gear_crown_workspace_bytes(const gear_dag* dag, int64_t batch);

/* CROWN lower bounds of the DAG's output over `batch` boxes.
 *   x_L, x_U  (batch, n) float64      box of every subdomain
 *   C         (batch, S, w_out) float64, or NULL for the identity specification
 *   lb        (batch, S) float64      lower bound of every specification row
 *   lA        (batch, S, n) float64   A of the bound w.r.t. the input (required for a
 *                                     box-per-CTA program, whose final pass accumulates A
 *                                     in this buffer; optional for a box-per-thread one)
 *   lbias     (batch, S) float64 or NULL      bias of that plane (lb minus the
 *                                            concretised A term)
 * `stream` is a cudaStream_t (NULL: the legacy default stream). Asynchronous. With batch 0
 * nothing is launched and the array pointers may be NULL. */
int gear_crown_lower(const gear_dag* dag, const double* x_L, const double* x_U, int64_t batch,
                     const double* C, double* lb, double* lA, double* lbias,
                     void* workspace, int64_t workspace_bytes, void* stream);

/* ---------------------------------------------------------------- branch and bound step
 * All arrays are device memory; `stream` is a cudaStream_t. Every call is asynchronous. */

/* Bytes of workspace gear_bab_prune needs for `batch` boxes. */
int64_t gear_bab_workspace_bytes(int64_t batch);

/* Prune (solving mode): keep[b] = 0 when some row proves box b done (lb_j > thr_j on a finite
 * row, lb_0 >= thr_0, or lb_0 = +inf with a finite thr_0). kept[0..n_kept) lists the kept boxes
 * in order; disc_min (one double, in/out) is lowered to the smallest finite thr_0 of the
 * discarded boxes. lb, thr (batch, S). With batch 0 only n_kept is written (0) and the
 * array pointers may be NULL. */
int gear_bab_prune(const double* lb, const double* thr, int64_t batch, int S, uint8_t* keep, int32_t* kept,
                   int32_t* n_kept, double* disc_min, void* workspace, int64_t ws_bytes, void* stream);

/* Split variable per box: argmax over i of sum_s max(|lA[b,s,i]|, coeff_thresh) (hi-lo)/2
 * (lowest index on ties); the widest variable when any lA/lb/thr is not finite, or when the
 * chosen width is below min_width_ratio of the widest relative to root_width (n). */
int gear_bab_branch(const double* lA, const double* lo, const double* hi, const double* lb, const double* thr,
                    int64_t batch, int S, int n, const double* root_width, double coeff_thresh,
                    double min_width_ratio, int32_t* split_idx, void* workspace, int64_t ws_bytes, void* stream);

/* Bisect the kept boxes at the midpoint of split_idx: children (2 n_kept, n) ordered
 * [upper halves of kept[0..n_kept); lower halves]. With child_key non-NULL also the children's
 * keys (2 n_kept, S): the parent's lb, row 0 raised to the parent plane's minimum over the child
 * box (rounded down). */
int gear_bab_split(const double* lo, const double* hi, const int32_t* kept, int64_t n_kept, int n,
                   const int32_t* split_idx, const double* lb, const double* lA, const double* lbias, int S,
                   double* child_lo, double* child_hi, double* child_key, void* stream);

/* Queue order of `count` slots: key descending, insertion id ascending on ties (bitonic sort;
 * order_len >= the next power of two of count). The batch is taken from the end. */
int gear_queue_order(const double* key, const int64_t* id, const int32_t* slots, int64_t count, int32_t* order,
                     int64_t order_len, void* stream);

/* Merge two slot lists a (na) and b (nb), each ordered by (key[slot] descending, id[slot]
 * ascending), into out (na + nb) in that order: the order gear_queue_order gives their union. A
 * queue kept in this order pops its batch from the tail with no sort (the reference re-sorts its
 * domain list, branching_domains.py:831-962); new domains are sorted (gear_queue_order) and
 * merged in. key, id: indexed by slot. */
int gear_queue_merge(const double* key, const int64_t* id, const int32_t* a, int64_t na, const int32_t* b, int64_t nb,
                     int32_t* out, void* stream);

/* dst[i, :] = src[rows[i], :] and dst[rows[i], :] = src[i, :] for float64 rows of `width`. */
int gear_gather_rows(const double* src, const int32_t* rows, int64_t count, int64_t width, double* dst,
                     void* stream);
int gear_scatter_rows(const double* src, const int32_t* rows, int64_t count, int64_t width, double* dst,
                      void* stream);

/* ---------------------------------------------------------------- device-resident queue, one BaB step
 * A gear_queue holds the open domains of one branch-and-bound run on the device: slot arrays (box,
 * keys, insertion ids), the active slot list kept in the reference's pop order (objective key
 * descending, insertion id ascending; branching_domains.py:831-962, 1171, with a stable sort), a
 * free list and the counters, all in device memory. gear_queue_pop and gear_bab_step read every
 * size from those counters: an iteration is a fixed sequence of launches with fixed arguments,
 * needs no host read, and can be captured once into a CUDA graph and replayed. They replace the
 * reference's domain list and its per-iteration loop body (UnsortedInputDomainList,
 * batch_branch_and_bound.py:275-652).
 *
 * gear_queue_create: n variables, S rows, `capacity` slots (> 2 x batch), iterations of `batch`
 * domains; the root box (n doubles each, host or device memory) is the first open domain.
 * gear_queue_pop: the next batch into lo_out / hi_out (batch, n): the tail of the active list, rows
 * beyond the open count repeat the first popped box (the root box when nothing is open).
 * gear_bab_step: bounds that batch with dag (gear_crown_lower, with the IBP pass when
 * ibp_enhancement), prunes against thresholds [*incumbent, rhs[0..S-2]] read on the device
 * (get_remaining_index, branching_domains.py:412-558), picks split variables (SB with sb_sum,
 * branching_heuristics.py:25-202), bisects the kept boxes (split.py:26-122), keys the children
 * (batch_branch_and_bound.py:189-225) and merges them into the active list. Workspace:
 * gear_bab_step_workspace_bytes. Children that would not fit the free slots are not pushed and
 * counted in counter 7: keep capacity >= open + 2 x batch per iteration run.
 * gear_queue_counters: copies the 8 counters (open, free, next id, domains bounded, last batch,
 * kept, iterations, overflows) to `counters` (host or device, asynchronous) and, when dual is
 * non-NULL, the dual bound min(open keys, smallest discarded threshold) to *dual (device).
 * gear_queue_size: the open count, synchronously. gear_queue_push: `count` <= 2 x batch domains
 * (device arrays lo, hi (count, n), key (count, S)) into the queue. */
typedef struct gear_queue gear_queue;
int gear_queue_create(int n, int S, int64_t capacity, int64_t batch, const double* root_lo, const double* root_hi,
                      gear_queue** out);
int gear_queue_destroy(gear_queue* q);
int gear_queue_push(gear_queue* q, const double* lo, const double* hi, const double* key, int64_t count, void* stream);
int gear_queue_pop(gear_queue* q, double* lo_out, double* hi_out, void* stream);
int gear_queue_size(const gear_queue* q, int64_t* open, void* stream);
int gear_queue_counters(const gear_queue* q, int64_t* counters, double* dual, void* stream);
/* Grow the queue to `capacity` slots (synchronous: waits for `stream`, copies the open domains into
 * a new block, frees the old one). The queue's device pointers change: work captured into a CUDA
 * graph that uses it must be captured again. gear_queue_capacity: the current capacity. */
int gear_queue_reserve(gear_queue* q, int64_t capacity, void* stream);
int64_t gear_queue_capacity(const gear_queue* q);
int64_t gear_bab_step_workspace_bytes(const gear_dag* dag, int64_t batch);
int gear_bab_step(gear_queue* q, const gear_dag* dag, const double* lo, const double* hi, const double* incumbent,
                  const double* rhs, double sb_coeff_thresh, double sb_min_width_ratio, int ibp_enhancement,
                  void* workspace, int64_t ws_bytes, void* stream);
/* gear_bab_step after its CROWN call: the batch's bounds lb (batch, S), lA (batch, S, n), lbias
 * (batch, S) come from the caller (a many-instance launch, gear_crown_lower_multi, bounds the
 * batches of many queues at once). Same prune, branch, split, keys and push. */
int gear_bab_step_bounded(gear_queue* q, const double* lo, const double* hi, const double* lb, const double* lA,
                          const double* lbias, const double* incumbent, const double* rhs, double sb_coeff_thresh,
                          double sb_min_width_ratio, void* stream);

/* Domain clipping, in place: shrink every box [x_L, x_U] (batch, n) along each coordinate to the
 * part where each plane lA_s x + lbias_s (s < S) can still be <= thr_s, rounding every candidate
 * outward; a box some plane already proves done becomes empty (x_L[0] = next double above x_U[0]).
 * The planes of box b are row parent[b] of lA (.., S, n), lbias and thr (.., S) (parent NULL:
 * row b). num_iters >= 1 repeats the clip with the plane minima of the clipped box. A box with a
 * non-finite plane, bias or a -inf/NaN threshold is left as it is. nonempty (batch) or NULL
 * receives 1 for a box that is not empty afterwards. */
int gear_clip_domains(double* x_L, double* x_U, const double* thr, const double* lA, const double* lbias,
                      const int32_t* parent, int64_t batch, int S, int n, int num_iters, uint8_t* nonempty,
                      void* stream);

/* Child keys of split children (child_lo, child_hi (2 n_kept, n), [upper halves; lower halves]
 * of the parents kept[0..n_kept)): the parent's lb, row 0 raised to the parent plane's minimum
 * over the child box, rounded down. */
int gear_bab_child_keys(const double* lb, const double* lA, const double* lbias, const double* child_lo,
                        const double* child_hi, const int32_t* kept, int64_t n_kept, int S, int n,
                        double* child_key, void* stream);

/* kept[0..n_kept) = the indices b with keep[b] != 0, in order. Workspace: gear_bab_workspace_bytes.
 * With batch 0 only n_kept is written (0) and keep / kept may be NULL. */
int gear_bab_compact(const uint8_t* keep, int64_t batch, int32_t* kept, int32_t* n_kept, void* workspace,
                     int64_t ws_bytes, void* stream);

/* ---------------------------------------------------------------- rigorous LP dual bound
 * For each domain b: a float64 lb <= D(y) = c0 - h^T y + sum_j min(r_j l_j, r_j u_j), r = c + G^T y,
 * the weak-duality bound of min c^T z + c0 s.t. G z <= h, l <= z <= u, exact on the given floats
 * (rounding enclosed; double-double recomputation of r where the error term exceeds tol/10, tol
 * NULL: max(1e-5, 1e-4 |value|)). G: m x n, nnz entries in CSC order: colptr (n+1), rows (nnz),
 * perm (nnz) = entry index of each CSC position into val (val_batched ? (batch, nnz) : (1, nnz)),
 * entries of a column in their original order. c, c_err (batch, n), c0, c0_err (batch) may be
 * NULL (zero). y < 0 counts as 0. -inf where nothing is certified. infeasibility = 1: the
 * double-double rule of certify_infeasible (c = c0 = 0 then; lb > 0 proves G z <= h infeasible on
 * the box). E (batch) and dd (batch, 1 = double-double used) may be NULL. */
int gear_dual_lower_bound(const int32_t* colptr, const int32_t* rows, const int32_t* perm, const double* val,
                          int val_batched, int64_t batch, int m, int n, int nnz, const double* c, const double* c0,
                          const double* h, const double* l, const double* u, const double* y, const double* tol,
                          const double* c_err, const double* c0_err, int infeasibility, double* lb, double* E,
                          uint8_t* dd, void* stream);

/* ---------------------------------------------------------------- constrained concretisation */

/* Bytes of workspace gear_constrained_lower needs. */
int64_t gear_constrained_workspace_bytes(int64_t batch, int K);

/* Lower bounds lb (batch, H) of obj (batch, H, n) . x over each box [x_L, x_U] (batch, n)
 * intersected with the rows A (batch, K, n) x + b (batch, K) <= 0, by the sequential dual sweep:
 * rows that cannot bind on the box are skipped, each remaining row k (at most max_rows of them,
 * the most binding, when max_rows > 0) gets the multiplier beta_k >= 0 that maximises the one-row
 * Lagrangian of the current objective, and the bound is widened by an outward rounding term and
 * never below the box bound. A box that some row excludes gets +inf (and infeasible[b] = 1 when
 * `infeasible` is non-NULL). Rows with a non-finite entry are ignored. n <= ~2000. */
int gear_constrained_lower(const double* x_L, const double* x_U, int64_t batch, int n, const double* obj, int H,
                           const double* A, const double* b, int K, int max_rows, double* lb, uint8_t* infeasible,
                           void* workspace, int64_t ws_bytes, void* stream);

/* gear_crown_lower with the IBP pass of the bounding glue (get_lower_bound_with_ibp_enhancement,
 * complete_verifier/input_split/bounding.py:789-948): lb_ibp (batch, S) receives every row's bound
 * over the output's plain interval (IBP from the box), and lb the larger of that and the CROWN bound.
 * lA and lbias are CROWN's. */
int gear_crown_lower_ibp(const gear_dag* dag, const double* x_L, const double* x_U, int64_t batch,
                         const double* C, double* lb, double* lA, double* lbias, double* lb_ibp,
                         void* workspace, int64_t workspace_bytes, void* stream);

/* gear_crown_lower without a workspace argument, for callers that cannot allocate device
 * memory (a solver host that owns a fixed device-memory plan and gives this library no
 * allocator, or a loop that must not pay cudaMalloc's implicit synchronisation). It has no
 * counterpart in the reference. Its scratch is a fixed array inside the library
 * (gear_crown_static_scratch_bytes(), 64 MiB) that every GPU loading the library keeps until
 * the process exits; the batch is processed by as many CTAs as fit in it, and a program whose
 * single CTA needs more scratch than that is rejected with GEAR_E_WORKSPACE. It calls no
 * cudaMalloc / cudaFree. The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress); make that first call before any stream capture. All calls share the
 * one array, so calls that overlap on the GPU (different streams, different host threads on
 * the same device) race: serialise them. The gear_dag handle itself is still created (and
 * allocated) once by gear_dag_create. A program compiled with the tensor-core fold computes its
 * fold products on the CUDA cores here (the digit planes need workspace), so its bounds differ
 * from gear_crown_lower's within the fold's stated error term (~1e-8 relative). */
int gear_crown_lower_static(const gear_dag* dag, const double* x_L, const double* x_U, int64_t batch,
                            const double* C, double* lb, double* lA, double* lbias, void* stream);

/* Size in bytes of gear_crown_lower_static's built-in scratch array. */
int64_t gear_crown_static_scratch_bytes(void);

/* ---------------------------------------------------------------- tensor-core fold
 * A program compiled with the tensor-core fold (header field H_FOLD_TC) gets, for each dense
 * Linear/MatMul node on the input, the products W x0, |W| eps and |W| max(|x_L|, |x_U|) over the
 * whole batch from int8 digit-sliced GEMMs on the tcgen05 tensor cores (exact int32 level sums in
 * TMEM, combined in float64) before the CROWN kernel runs; the radius carries the rigorous bound
 * of the slicing error, so every CROWN bound stays sound. This is the dense work of
 * BoundLinear.bound_backward / interval_propagate on the input (auto_LiRPA/operators/linear.py:268,
 * interval_bound.py:156-254). gear_crown_lower and gear_crown_lower_ibp launch it themselves
 * (their workspace then includes the digit planes: gear_crown_workspace_bytes).
 *
 * gear_crown_fold_vectors runs only that step and copies the fold vectors (batch, fold width of
 * the program: per dense node, w centres, w radii (error included), w magnitudes) to fold_out;
 * fail_out (one int, may be NULL) receives 1 when a bounded device wait expired (the vectors are
 * then invalid; gear_crown_lower falls back to the CUDA-core fold by itself). */
int gear_crown_fold_vectors(const gear_dag* dag, const double* x_L, const double* x_U, int64_t batch,
                            double* fold_out, int* fail_out, void* workspace, int64_t workspace_bytes,
                            void* stream);

/* Workspace bytes of gear_crown_fold_vectors (-1 for a program without the tensor-core fold). */
int64_t gear_crown_fold_workspace_bytes(const gear_dag* dag, int64_t batch);

/* ---------------------------------------------------------------- the plain (unfused) form
 * The same CROWN bounds as gear_crown_lower, computed the unfused way: one kernel launch per
 * schedule step, and inside every CROWN pass one launch per op (one node's backward step into
 * one input) plus one for the pass's initial A and one for its concretisation; every box's
 * state crosses launches through global memory. It is the baseline the fused launch is measured
 * against, not a production path. The DAG must be a box-per-CTA program compiled with its pass
 * working set in global memory (H_PASS_GLOBAL > 0, e.g. Program(..., smem_limit=0)); lA is
 * required. Workspace: one slot per box. */
int64_t gear_crown_plain_workspace_bytes(const gear_dag* dag, int64_t batch);
int gear_crown_lower_plain(const gear_dag* dag, const double* x_L, const double* x_U, int64_t batch,
                           const double* C, double* lb, double* lA, double* lbias, void* workspace,
                           int64_t workspace_bytes, void* stream);

/* gear_crown_lower_plain with the IBP pass of the bounding glue, as gear_crown_lower_ibp
 * (complete_verifier/input_split/bounding.py:789-948): lb_ibp (batch, S) receives the rows' bounds
 * over the output's plain interval and lb the larger of that and CROWN's. */
int gear_crown_lower_plain_ibp(const gear_dag* dag, const double* x_L, const double* x_U, int64_t batch,
                               const double* C, double* lb, double* lA, double* lbias, double* lb_ibp,
                               void* workspace, int64_t workspace_bytes, void* stream);

/* ---------------------------------------------------------------- CROWN under cut rows
 * Replaces BoundedModule.compute_bounds(x=(BoundedTensor(x0, PerturbationLpNorm(x_L, x_U,
 * constraints=(A, b))),), C, method='CROWN') (solver/auto_LiRPA/bound_general.py:1275 with
 * perturbations.py:129 carrying the rows), as the input-split BaB's constrained mode calls it
 * (complete_verifier/input_split/batch_branch_and_bound.py:422-428): EVERY concretisation of the
 * call -- each intermediate pass (both sides) and the final pass -- bounds its rows over the box
 * [x_L, x_U] intersected with the box's rows cut_A (batch, K, n) x + cut_b (batch, K) <= 0, by the
 * sequential dual sweep of gear_constrained_lower (constraints_solving, concretize_func.py:431-850;
 * an upper bound is minus the sweep's lower bound of -A), in place of the box terms. lb, lA, lbias
 * (and lb_ibp when non-NULL, as gear_crown_lower_plain_ibp) as gear_crown_lower; lA is required.
 * C (batch, S, w) or NULL (identity) as gear_crown_lower. A box its rows
 * exclude gets bounds that only say so through the concretisations (+inf lower rows are discarded
 * to the interval fallback); callers that prune on infeasibility test it with
 * gear_constrained_lower. The DAG must be compiled for cut rows (gear_b200/program.py
 * Program(..., cuts=True, smem_limit=0): box per CTA, pass working set in global memory, no
 * folded passes). Runs in the plain form's launch sequence (one launch per step / op) plus, per
 * pass, one launch writing the dense rows and one sweep. K may be 0 (the reference's box bound
 * with its rounding). n and K are bounded by one warp's shared memory (n <= ~2000). */
int64_t gear_crown_cuts_workspace_bytes(const gear_dag* dag, int64_t batch, int K);
int gear_crown_lower_cuts(const gear_dag* dag, const double* x_L, const double* x_U, int64_t batch,
                          const double* C, const double* cut_A, const double* cut_b, int K, int max_rows,
                          double* lb, double* lA, double* lbias, double* lb_ibp, void* workspace,
                          int64_t workspace_bytes, void* stream);

/* ---------------------------------------------------------------- many instances, one launch
 * One instance of a multi-instance CROWN call: the arguments gear_crown_lower takes for one
 * DAG (same shapes and meaning; batch may be 0). The reference bounds each instance with its own
 * compute_bounds call (bound_general.py:1275, from bounding.py:317); here the boxes of every
 * instance go into one persistent launch. */
typedef struct gear_lower_args {
  const gear_dag* dag;
  const double* x_L;
  const double* x_U;
  int64_t batch;
  const double* C;
  double* lb;
  double* lA;
  double* lbias;
  double* lb_ibp;   /* NULL, or (batch, S): as in gear_crown_lower_ibp (lb = max(CROWN, IBP)) */
} gear_lower_args;

/* Workspace bytes for gear_crown_lower_multi on these instances (0 when no instance has boxes,
 * -1 on invalid arguments; the text is in gear_last_error). */
int64_t gear_crown_multi_workspace_bytes(const gear_lower_args* items, int32_t count);

/* CROWN lower bounds of every instance's boxes in ONE kernel launch: the results of instance i
 * are those gear_crown_lower gives for it alone (same kernel code per box). Every DAG must have
 * the same execution mode and threads per CTA and live on the current device. CTAs take work
 * items (boxes, or tiles of 64 boxes for box-per-thread programs) from a device counter in
 * the given instance order, so list expensive instances first. The instance table is copied
 * to the device from pinned memory inside the call; `items` may be reused on return.
 * Asynchronous on `stream`. */
int gear_crown_lower_multi(const gear_lower_args* items, int32_t count, void* workspace, int64_t workspace_bytes,
                           void* stream);

/* The same launch prepared once: gear_crown_multi_prepare plans it and uploads its instance table
 * into `workspace` (gear_crown_multi_workspace_bytes; the workspace and every instance's buffers
 * must stay in place), after which each gear_crown_multi_launch is a work-counter reset and one
 * kernel with fixed arguments -- a launch a CUDA graph can capture and replay (the instances'
 * inputs change in place between replays). Synchronous prepare; the plan is host memory, freed by
 * gear_crown_multi_plan_destroy. No counterpart in the reference (its batching is per instance). */
typedef struct gear_multi_plan gear_multi_plan;
int gear_crown_multi_prepare(const gear_lower_args* items, int32_t count, void* workspace, int64_t workspace_bytes,
                             gear_multi_plan** out);
int gear_crown_multi_launch(const gear_multi_plan* plan, void* stream);
int gear_crown_multi_plan_destroy(gear_multi_plan* plan);

/* Number of kernel launches the last gear_crown_lower on this thread issued. */
int gear_last_launch_count(void);

const char* gear_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* GEAR_B200_H */

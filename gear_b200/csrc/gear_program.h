// Device-side layout of a compiled CROWN program (host side: gear_b200/program.py).
// All records are int32; offsets index the int pool (ip) or the float64 pool (dp).
#pragma once
#include <stdint.h>

namespace gear {

enum NodeKind {
  NK_INPUT = 0, NK_LINEAR = 1, NK_MATMUL = 2, NK_MUL = 3, NK_MULC = 4, NK_ADD = 5, NK_SUB = 6,
  NK_ADDC = 7, NK_SUBC = 8, NK_RSUBC = 9, NK_NEG = 10, NK_SQR = 11, NK_EXP = 12, NK_LOG = 13,
  NK_SIN = 14, NK_COS = 15, NK_POW = 16, NK_REDUCESUM = 17, NK_MAP = 18, NK_CONCAT = 19
};

// N_WT_OFF: the weights of a linear/matmul node transposed, (in, out), for the forward products
enum NodeField {
  N_KIND = 0, N_W, N_NIN, N_IN0, N_IN1, N_CUR, N_PLANE, N_CVEC, N_MAP0, N_MAP1, N_W_OFF, N_B_OFF,
  N_WIN, N_INS, N_FOLD, N_INEXACT, N_WT_OFF, NODE_REC
};

// ST_IBPOUT: the specification rows over the output's plain IBP interval, into Work.lb_ibp
enum StepType { ST_IBP = 0, ST_MAG = 1, ST_RELAX = 2, ST_PASS = 3, ST_COMPARE = 4, ST_FOLD = 5, ST_FINAL = 6,
                ST_IBPOUT = 7 };
constexpr int STEP_REC = 4;

enum PassField {
  P_T = 0, P_S, P_SIDES, P_INIT, P_OP0, P_NOP, P_TBUF, P_XNNZ, P_XBUF, P_XRP, P_XCOLS, P_NFOLD,
  P_SMEM, P_TRP, P_TCOLS, P_FINAL, P_NVISIT, P_MAXROW, P_ONEHOT, P_XMAXROW, P_XDENSE, P_TMAXROW,
  PASS_REC = 24
};

enum OpField {
  O_KIND = 0, O_V, O_SLOT, O_FIRST, O_VBUF, O_VNNZ, O_VRP, O_VCOLS, O_U, O_UBUF, O_UNNZ, O_URP,
  O_UCOLS, O_UMERGE, O_NTGT, O_TGT, O_SPTR, O_SRC, O_DENSE, O_FOLD, O_WOUT, O_VMAXROW, O_UMAXROW, O_VROWS,
  O_TPTR, O_UK, O_TMAXROW, O_SHORT, O_NSHORT, O_LONG, O_NLONG, O_SINGLE, OP_REC = 32
};
// bits of an op record's O_SINGLE field: every target pulls one source; the source list, the
// target list, the target row pointers or v's row pointers are the identity (the kernel then
// computes the index instead of loading it). OF_SPLIT: the final pass's product through a dense
// node on the input, handed to the tensor cores when the launch provides the buffers for it.
enum OpFlag {
  OF_SINGLE = 1, OF_SRC_ID = 2, OF_TGT_ID = 4, OF_TPTR_ID = 8, OF_VRP_ID = 16, OF_SPLIT = 32, OF_FUSED = 64,
  OF_FUSED_T = 128
};
// OF_FUSED: an entry-wise op (entry e of v's row s moves to entry e of u's row s, which a fresh u
// row holds exactly, all rows short): bias terms and moves in one sweep over the row's entries.
// OF_FUSED_T: the same sweep with entry e moving to u's entry tgt[e] of the same row (a fresh u row
// is cleared first).
// buffer offset marker: the input's A of a final pass accumulates in the lA output (row s at s * n)
constexpr int ROOT_IN_LA = -2;
// rows with at most this many entries are handled by one thread, longer rows by a warp
constexpr int ROW_THREAD_MAX = 16;
// shared-memory reduction slots reserved after the row arrays
constexpr int RED_SLOTS = 32;

enum HeaderField {
  H_NNODES = 0, H_NSTEPS, H_NPASSES, H_NOPS, H_N, H_S, H_T, H_ARENA, H_PLANES, H_FOLDW,
  H_SMEM, H_MAXS, H_SINOFF, H_MAXW, H_RETA, H_MAXOPS, H_SIMT_BUF, H_SIMT_ROWS, H_X_IN_LA, H_MODE,
  H_CTA_THREADS, H_PASS_GLOBAL, H_TIES, H_FOLD_TC, HEADER_LEN = 24
};
// H_TIES: McCormick tie rule, 0 = the reference's float comparison, 1 = exact-arithmetic ties.
// H_FOLD_TC: 1 = the fold vectors of the dense nodes on the input come from the tensor-core
// fold (fold_tc.cuh) launched before the CROWN kernel (box-per-CTA programs only).
// H_PASS_GLOBAL: 0, or the doubles of a box-per-CTA program's pass working set when it is too
// large for shared memory and lives at the end of the CTA's scratch slot instead (H_SMEM then
// counts only the staged node table and op records).

// Doubles of a box-per-CTA scratch slot before that global pass working set: interval and
// magnitude arenas, relaxation planes, fold vectors, 4 node-wide temporaries.
__host__ __device__ inline int64_t cta_slot_fixed(const int32_t* hdr) {
  const int64_t d = 3 * (int64_t)hdr[H_ARENA] + hdr[H_PLANES] + hdr[H_FOLDW] + 4 * (int64_t)hdr[H_MAXW] + 8;
  return (d + 31) / 32 * 32;
}

// execution model of a program: one box per CTA (pass working set in shared memory) or one box
// per thread (per-box state box-interleaved in global scratch)
enum ExecMode { MODE_CTA = 0, MODE_SIMT = 1 };

// Sin/cos table layout inside the float64 pool, from H_SINOFF (gear_b200/tables.py order).
constexpr int SIN_N_PRE = 162;   // int(pi/2 / 0.01) + 5
constexpr int SIN_N_TB = 1001;

struct DevProgram {
  const int32_t* hdr;
  const int32_t* nodes;
  const int32_t* steps;
  const int32_t* passes;
  const int32_t* ops;
  const int32_t* ip;
  const double* dp;
};

}  // namespace gear

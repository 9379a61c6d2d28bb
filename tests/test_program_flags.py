"""Program compiler: the op records' index-shape flags (OpFlag) describe their arrays exactly,
and a pass working set beyond smem_limit moves to global memory (header H_PASS_GLOBAL)."""
import numpy as np
import pytest
import torch

from gear_b200 import graph, problems
from gear_b200.program import (O_SINGLE, O_SPTR, O_SRC, O_TGT, O_TPTR, O_NTGT, O_VRP, O_DENSE, O_FOLD,
                               OF_SINGLE, OF_SRC_ID, OF_TGT_ID, OF_TPTR_ID, OF_VRP_ID, OP_REC, P_S, PASS_REC,
                               P_OP0, P_NOP, Program)


def _progs():
    for wl in ("quad_exp_n10", "dense_q_n200"):
        m = problems.make_instance(wl, 0)
        lo, hi = problems.make_boxes(wl, 2, 0)
        yield wl, Program(graph.trace(m, lo), mode="cta")
    m = problems.mixed_instance(4)
    yield "mixed4", Program(graph.trace(m, torch.zeros(2, m.n, dtype=torch.float64)), mode="cta")


@pytest.mark.parametrize("name,prog", list(_progs()))
def test_op_flags_match_arrays(name, prog):
    ops = prog.op_arr.reshape(-1, OP_REC)
    passes = prog.pass_arr.reshape(-1, PASS_REC)
    ip = prog.int_pool
    checked = 0
    for pr in passes:
        S = int(pr[P_S])
        for o in ops[int(pr[P_OP0]):int(pr[P_OP0]) + int(pr[P_NOP])]:
            f = int(o[O_SINGLE])
            if o[O_DENSE] == 1 or o[O_FOLD] == 1:
                assert f == 0
                continue
            nt = int(o[O_NTGT])
            tgt = ip[o[O_TGT]:o[O_TGT] + nt]
            tptr = ip[o[O_TPTR]:o[O_TPTR] + S + 1]
            vrp = ip[o[O_VRP]:o[O_VRP] + S + 1]
            sptr = ip[o[O_SPTR]:o[O_SPTR] + nt + 1]
            nsrc = int(sptr[-1]) if nt else 0
            src = ip[o[O_SRC]:o[O_SRC] + nsrc]
            assert bool(f & OF_SINGLE) == (nsrc == nt)
            assert bool(f & OF_SRC_ID) == (nsrc > 0 and np.array_equal(src, np.arange(nsrc)))
            assert bool(f & OF_TGT_ID) == np.array_equal(tgt, np.arange(nt))
            assert bool(f & OF_TPTR_ID) == np.array_equal(tptr, np.arange(S + 1))
            assert bool(f & OF_VRP_ID) == np.array_equal(vrp, np.arange(S + 1))
            checked += 1
    assert checked > 5


def test_pass_working_set_moves_to_global_memory():
    m = problems.make_instance("quad_exp_n10", 0)
    g = graph.trace(m, torch.zeros(2, 10, dtype=torch.float64))
    a = Program(g, mode="cta")
    b = Program(g, mode="cta", smem_limit=0)
    assert a.pass_global == 0 and b.pass_global == a.max_smem > 0
    assert b.smem_total < a.smem_total
    for f in ("node_arr", "step_arr", "pass_arr", "op_arr", "int_pool", "dbl_pool"):
        assert np.array_equal(getattr(a, f), getattr(b, f))


def test_cut_programs_fold_no_pass():
    """Program(cuts=True): the constrained sweep needs every input A row, so no pass folds its
    rows into the per-box fold vectors (dense_q_n200 folds its Linear-on-input passes otherwise);
    the fold vectors themselves stay for the IBP steps."""
    from gear_b200.program import P_NFOLD
    m = problems.make_instance("dense_q_n200", 0)
    lo, hi = problems.make_boxes("dense_q_n200", 2, 0)
    g = graph.trace(m, lo)
    plain = Program(g, mode="cta", smem_limit=0)
    cut = Program(g, mode="cta", smem_limit=0, cuts=True)
    assert any(int(r[P_NFOLD]) for r in plain.pass_arr.reshape(-1, PASS_REC))
    assert not any(int(r[P_NFOLD]) for r in cut.pass_arr.reshape(-1, PASS_REC))
    assert cut.fold_w == plain.fold_w > 0 and cut.pass_global > 0


def test_fused_flag_marks_entrywise_ops():
    """OF_FUSED (one sweep per row: bias terms and moves together, no clearing of u's row) only on
    ops whose moves are entry-wise: one identity source and target per entry, row s's moves are
    v's entries of row s, and a fresh u row holds exactly those entries; every row short. The
    elementwise chains of the mixed family get it on most ops."""
    from gear_b200.program import OF_FUSED, OF_FUSED_T, O_URP, O_UMERGE, O_NLONG, O_U, O_UBUF, ROOT_IN_LA
    m = problems.mixed_instance(70)
    prog = Program(graph.trace(m, torch.zeros(2, m.n, dtype=torch.float64)), mode="cta", cta_threads=256)
    ops = prog.op_arr.reshape(-1, OP_REC)
    passes = prog.pass_arr.reshape(-1, PASS_REC)
    ip = prog.int_pool
    fused = 0
    for pr in passes:
        S = int(pr[P_S])
        for o in ops[int(pr[P_OP0]):int(pr[P_OP0]) + int(pr[P_NOP])]:
            f = int(o[O_SINGLE])
            if not f & (OF_FUSED | OF_FUSED_T):
                continue
            fused += 1
            assert not (f & OF_FUSED and f & OF_FUSED_T)
            assert f & (OF_SINGLE | OF_SRC_ID) == (OF_SINGLE | OF_SRC_ID)
            assert o[O_DENSE] == 0 and o[O_NLONG] == 0 and o[O_UBUF] != ROOT_IN_LA
            vrp = ip[o[O_VRP]:o[O_VRP] + S + 1]
            tptr = ip[o[O_TPTR]:o[O_TPTR] + S + 1]
            urp = ip[o[O_URP]:o[O_URP] + S + 1]
            assert np.array_equal(tptr, vrp)
            if f & OF_FUSED:
                assert f & OF_TGT_ID
                assert o[O_UMERGE] == 1 or np.array_equal(urp, vrp)
            else:
                # every target of row s lies in u's row s
                tgt = ip[o[O_TGT]:o[O_TGT] + int(o[O_NTGT])]
                rows_u = np.repeat(np.arange(S), np.diff(urp))
                rows_v = np.repeat(np.arange(S), np.diff(vrp))
                assert np.array_equal(rows_u[tgt], rows_v)
    assert fused > len(ops) * 3 // 4

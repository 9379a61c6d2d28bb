"""Record node programs emitted by the reference's gear lowering (run where the reference source
is available; the committed file is what the tests read).

    python tests/golden/make_program_golden.py /path/to/reference

For the benchmark workloads and the fixture models, exports the float64 model at batch 1 with
torch.export and runs the reference's gear.lower.emit.emit_program on it; the resulting
NodeProgram (nodes_op, nodes_in, nodes_out) is stored as plain lists and tensors in
tests/golden/programs.pt. Also records gear.spec.parse_vnnlib_subset on a few property texts.
"""
import os
import sys

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))

VNNLIB = {
    "box_rows": """; two inputs, three outputs
(declare-const X_0 Real)
(declare-const X_1 Real)
(declare-const Y_0 Real)
(declare-const Y_1 Real)
(declare-const Y_2 Real)
(assert (>= X_0 -1.5))
(assert (<= X_0 2.25))
(assert (>= X_1 0.1))
(assert (<= X_1 0.3))
(assert (<= Y_1 0.0))
(assert (>= Y_2 -4e-1))
""",
    "tight": """(declare-const X_0 Real)
(declare-const Y_0 Real)
(assert (<= X_0 1))
(assert (>= X_0 0.5))
(assert (<= X_0 0.75))
(assert (<= Y_0 3.0))
""",
}


def plain(program):
    def node(n):
        return dict(name=n.name, op=n.op, inputs=list(n.inputs),
                    attr={k: v for k, v in (n.attr or {}).items()} if isinstance(n.attr, dict) else n.attr,
                    ori_name=n.ori_name, model_input_index=n.model_input_index,
                    param=None if n.param is None or isinstance(n.param, dict) else n.param.detach().clone())
    return dict(nodes_op=[node(n) for n in program.nodes_op], nodes_in=[node(n) for n in program.nodes_in],
                nodes_out=list(program.nodes_out))


def main(ref_root):
    sys.path.insert(0, HERE)
    sys.path.insert(0, REPO)
    import make_bab_golden
    sys.meta_path.insert(0, make_bab_golden._Finder())
    import make_golden
    make_golden._stub_modules()
    sys.path.insert(0, os.path.join(ref_root, "solver", "complete_verifier"))
    sys.path.insert(0, os.path.join(ref_root, "solver"))
    from gear.lower.emit import emit_program
    from gear.spec import parse_vnnlib_subset
    from gear_b200 import problems
    import models
    out = {"programs": {}, "vnnlib": {}}
    cases = {wl: (problems.make_instance(wl, 0), problems.WORKLOADS[wl]["n"]) for wl in ("quad_exp_n10", "dense_q_n200")}
    for name, (cls, n) in models.MODELS.items():
        cases[name] = (cls(), n)
    for name, (m, n) in cases.items():
        m = m.to(torch.float64).eval()
        x0 = torch.zeros(1, n, dtype=torch.float64)
        ep = torch.export.export(m, (x0,), strict=False)
        try:
            prog = emit_program(ep, state_order=list(m.state_dict().keys()))
        except Exception as exc:                    # outside the emitter's direct table
            print("emitter refused", name, exc)
            continue
        out["programs"][name] = dict(plain(prog), n=n)
    for name, text in VNNLIB.items():
        lo, hi, spec = parse_vnnlib_subset(text, name)
        out["vnnlib"][name] = dict(text=text, lo=torch.tensor(lo), hi=torch.tensor(hi), num_outputs=spec.num_outputs,
                                   indptr=torch.tensor(spec.indptr), indices=torch.tensor(spec.indices),
                                   data=torch.tensor(spec.data), rhs=torch.tensor(spec.rhs))
    torch.save(out, os.path.join(HERE, "programs.pt"))
    print("saved", list(out["programs"]), list(out["vnnlib"]))


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit(f"usage: python {os.path.basename(__file__)} REFERENCE_ROOT")
    main(sys.argv[1])

"""Run a fixed number of device-resident Stokes solves (profiling driver).

    python -m lowmachmixtures_b200.profile_solve --n 128 --method mixed --solves 1

Used under ncu to list every kernel launch of a solve, and to capture the
hot kernels on the benchmark workload (3D n^3, contrast 100, inertial
theta*alpha*dx^2 = 0.1, precon_type 2, visc_type -2).  --warm solves run
first so that a capture can skip them with ncu's -s.

    python -m lowmachmixtures_b200.profile_solve --n 128 --op net_forward --solves 5

times forward passes of the learned stage's network (random weights, one
n^3 field of 8 BF16 channels) instead.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--dm", type=int, default=3, choices=[2, 3],
                    help="2: the 2D steady workload (n^2, contrast 10, theta = 0); 3: 3D n^3, contrast 100, theta*alpha = 0.1/dx^2")
    ap.add_argument("--method", default="mixed", choices=["mixed", "plain", "reference", "learned"],
                    help="learned: mixed with the learned stage, its network trained (--train-steps, 64^3) first")
    ap.add_argument("--train-steps", type=int, default=200)
    ap.add_argument("--solves", type=int, default=1)
    ap.add_argument("--warm", type=int, default=1)
    ap.add_argument("--knob", action="append", default=[], metavar="NAME=INT",
                    help="extra lmm_knobs integer field (repeatable), e.g. --knob tail_cells=512")
    ap.add_argument("--bc", default="", help="BC code per direction, both sides, e.g. -1,100,-1 (default periodic)")
    ap.add_argument("--op", default="", choices=["", "smooth", "applyop", "apply_matrix", "vcycle", "macproject", "gram_schmidt",
                             "normalise", "net_forward"],
                    help="instead of solves: time one operation (lmm_time_op) --solves times after one warm-up; "
                         "'smooth' and 'vcycle' run in the method's precision; 'net_forward': --warm + --solves "
                         "forward passes of the learned stage's network")
    a = ap.parse_args()

    import numpy as np
    import torch

    from lowmachmixtures_b200 import abi, synth
    from lowmachmixtures_b200.gmres import StokesSolver

    if a.op == "net_forward":
        import ctypes

        from lowmachmixtures_b200 import learned
        net = learned.Net((a.n,) * 3, 1, 0)
        x = torch.randn(1, a.n, a.n, a.n, 8).to(torch.bfloat16).cuda()
        y = torch.empty(1, a.n, a.n, a.n, 4, device="cuda")
        fwd = lambda: net.lib.lmm_net_forward(net.h, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()))  # noqa: E731
        for _ in range(a.warm):
            assert fwd() == 0
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record()
        for _ in range(a.solves):
            assert fwd() == 0
        t1.record()
        torch.cuda.synchronize()
        print(json.dumps({"op": a.op, "n": a.n, "ms_per_forward": t0.elapsed_time(t1) / max(a.solves, 1)}))
        net.close()
        return

    bc = tuple(int(v) for v in a.bc.split(",")) if a.bc else None
    if a.dm == 2:
        prob = synth.make_problem(2, a.n, 10.0, 0, theta_alpha=0.0, bc=bc)
    else:
        prob = synth.config_3d_128(0, n=a.n) if bc is None else synth.make_problem(3, a.n, 100.0, 0, theta_alpha=0.1 * a.n * a.n, bc=bc)
    kn = dict(precon_type=2, visc_type=-2)
    net = None
    if a.method == "learned":
        from lowmachmixtures_b200 import learned
        net64, _, _ = learned.train(n=64, fields=20, steps=a.train_steps, batch=4, theta_alpha=0.1)
        params = net64.params()
        net64.close()
        net = learned.Net((a.n,) * 3, 1, 0)
        net.set_params(params)
        kn.update(learned_stage=1)
    if a.method in ("mixed", "learned"):
        kn.update(method=abi.LMM_METHOD_FGMRES, precision=abi.LMM_PRECISION_FP32)
    elif a.method == "plain":
        kn.update(method=abi.LMM_METHOD_FGMRES, precision=abi.LMM_PRECISION_FP64)
    for kv in a.knob:
        name, val = kv.split("=")
        kn[name] = int(val)
    dev = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()  # noqa: E731
    bu, bp = [dev(x) for x in prob.b_u], dev(prob.b_p)
    al, be, bed, ga = [dev(x) for x in prob.alpha_fc], dev(prob.beta), [dev(x) for x in prob.beta_ed], dev(prob.gamma)
    xu, xp = [torch.zeros_like(bu[0]) for _ in range(a.dm)], torch.zeros_like(bp)
    with StokesSolver(a.dm, (a.n,) * a.dm, prob.dx, knobs=abi.make_knobs(**kn), bc=bc) as s:
        if net is not None:
            assert s.lib.lmm_stokes_set_net(s._h, net.h) == 0
        if a.op:
            s.load_coeffs(al, be, bed, ga, prob.theta_alpha)
            fp32 = a.method == "mixed"
            which = {"smooth": 1 if fp32 else 0, "applyop": 2, "apply_matrix": 3, "vcycle": 5 if fp32 else 4,
                     "macproject": 6, "gram_schmidt": 7, "normalise": 8}[a.op]
            print(json.dumps({"op": a.op, "us": s.time_op(which, reps=a.solves) * 1000.0}))
            return
        out = []
        for i in range(a.warm + a.solves):
            for t in xu:
                t.zero_()
            xp.zero_()
            l0 = s.lib.lmm_kernel_launches()
            _, _, st = s.solve_device(bu, bp, xu, xp, al, be, bed, ga, prob.theta_alpha)
            out.append({"solve": i, "iters": st["total_iter"], "ms": st["solve_ms"],
                        "launches": s.lib.lmm_kernel_launches() - l0,
                        "rel_res": st["norm_resid_true"] / st["norm_b"]})
    print(json.dumps(out))


if __name__ == "__main__":
    main()

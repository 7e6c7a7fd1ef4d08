"""The full-size 3D workload: n^3 periodic (256^3 by default, 67M unknowns),
4-species mixture viscosity (synth.mixture_viscosity), right-hand side the
divergence of a stochastic stress generated on the GPU
(lmm_stochastic_rhs: kT = 1, dt = 1e-3, dV = dx^3), overdamped (theta = 0),
FGMRES with a 20-vector FP64 Krylov basis; the FP32-V-cycle method against
the plain FP64 one, both to |b - Ax| / |b| <= 1e-9.

    python -m lowmachmixtures_b200.mixture_solve --n 256
"""
from __future__ import annotations

import ctypes as C
import json
import time

import numpy as np


def run(n: int = 256, seed: int = 0, repeats: int = 2, log=print):
    import torch

    from . import _native, abi, synth
    from .gmres import StokesSolver
    lib = _native.load()
    t0 = time.time()
    prob = synth.config_3d_256_mixture(n, seed)
    gen_s = time.time() - t0
    dev = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()  # noqa: E731
    al, be, bed, ga = [dev(a) for a in prob.alpha_fc], dev(prob.beta), [dev(b) for b in prob.beta_ed], dev(prob.gamma)
    bu = [torch.zeros_like(be) for _ in range(3)]
    bp = torch.zeros_like(be)
    nn = (C.c_int * 3)(n, n, n)
    torch.cuda.synchronize()
    assert lib.lmm_stochastic_rhs(3, nn, prob.dx, 1e-3, 1.0, abi.ptr(be), abi.ptr_array(bed), seed, abi.ptr_array(bu), None) == 0
    torch.cuda.synchronize()
    out = dict(workload=f"stokes_3d_{n}^3_mixture_stochastic", n=n, unknowns=4 * n ** 3, contrast=prob.contrast,
               host_generation_s=gen_s)
    sols = {}
    for name, kw in [("plain_fp64", dict(precision=abi.LMM_PRECISION_FP64)), ("mixed", dict(precision=abi.LMM_PRECISION_FP32))]:
        kn = abi.make_knobs(precon_type=2, visc_type=-2, method=abi.LMM_METHOD_FGMRES, gmres_max_inner=20, **kw)
        with StokesSolver(3, (n, n, n), prob.dx, knobs=kn) as s:
            best = None
            for _ in range(repeats):
                xu, xp = [torch.zeros_like(be) for _ in range(3)], torch.zeros_like(be)
                _, _, st = s.solve_device(bu, bp, xu, xp, al, be, bed, ga, 0.0)
                best = st["solve_ms"] if best is None else min(best, st["solve_ms"])
            out[name] = dict(ms=best, solves_per_s=1e3 / best, iterations=st["total_iter"],
                             true_rel_residual=st["norm_resid_true"] / st["norm_b"])
            sols[name] = (xu, xp)
        log(json.dumps({name: out[name]}))
    (um, pm), (uf, pf) = sols["mixed"], sols["plain_fp64"]
    # the periodic overdamped problem fixes velocity and pressure up to constants
    num = sum(float(((a - a.mean()) - (b - b.mean())).pow(2).sum()) for a, b in zip(um, uf))
    den = sum(float((b - b.mean()).pow(2).sum()) for b in uf)
    out["mixed_vs_fp64_velocity_rel_l2"] = (num / den) ** 0.5
    out["speedup_mixed_over_plain"] = out["plain_fp64"]["ms"] / out["mixed"]["ms"]
    return out


def main():
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--seed", type=int, default=0)
    a = ap.parse_args()
    print(json.dumps(run(a.n, a.seed)), flush=True)


if __name__ == "__main__":
    main()

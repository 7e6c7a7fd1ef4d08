"""Run a fixed set of solves and operator calls with the library the
environment selects (LMM_BOUNDS_CHECK=1: the bounds-check build) and save
every result and status code to an npz file.  Used by
test_bounds_check_gpu.py, which runs it once per library and compares."""
from __future__ import annotations

import ctypes as C
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def main(out_path):
    import numpy as np
    import torch

    from lowmachmixtures_b200 import _native, abi, ensemble, learned, synth
    from lowmachmixtures_b200.gmres import StokesSolver
    lib = _native.load()
    res = {"library": np.array(os.path.basename(lib._name))}
    status = []

    def solve(tag, prob, bc=None, net=None, **kn):
        with StokesSolver(prob.dm, prob.shape[::-1], prob.dx, knobs=abi.make_knobs(**kn), bc=bc) as s:
            if net is not None:
                assert s.lib.lmm_stokes_set_net(s._h, net.h) == 0
            xu, xp = prob.zeros_like_solution()
            fin = s._fields(prob.b_u, prob.b_p, prob.alpha_fc, prob.beta, prob.beta_ed, prob.gamma, abi.LMM_LAYOUT_COMPACT, None)
            fout = abi.FieldsOut()
            fout.x_u = abi.ptr_array(xu)
            fout.x_p = abi.ptr(xp)
            th, npr, st = C.c_double(prob.theta_alpha), C.c_double(0.0), abi.Stats()
            rc = s.lib.lmm_stokes_solve(s._h, C.byref(fin), C.byref(fout), C.byref(th), C.byref(npr), C.byref(st))
        status.append(rc)
        if rc != 0:
            print(f"{tag}: status {rc}: {lib.lmm_strerror(rc).decode()}", flush=True)
        for c, a in enumerate(xu):
            res[f"{tag}_u{c}"] = a
        res[f"{tag}_p"] = xp

    p3 = synth.make_problem(3, 32, 100.0, 1, theta_alpha=0.1 * 32 * 32)
    fgmres = dict(precon_type=2, visc_type=-2, method=abi.LMM_METHOD_FGMRES)
    solve("plain64", p3, **fgmres, precision=abi.LMM_PRECISION_FP64)
    solve("mixed32", p3, **fgmres, precision=abi.LMM_PRECISION_FP32, orthogonalization=1)
    solve("reference", p3, precon_type=2, visc_type=-2)
    pw = synth.make_problem(3, 24, 100.0, 2, theta_alpha=0.1 * 24 * 24, bc=(-1, 100, -1))
    solve("walls", pw, bc=(-1, 100, -1), precon_type=2, visc_type=-2)
    p2 = synth.make_problem(2, 64, 10.0, 3)
    solve("p1_2d", p2, precon_type=1, visc_type=-1)
    # learned stage (untrained network, 16^3)
    pl = synth.make_problem(3, 16, 100.0, 4, theta_alpha=0.1 * 16 * 16)
    net = learned.Net((16, 16, 16), 1, 0)
    solve("learned", pl, net=net, **fgmres, precision=abi.LMM_PRECISION_FP32, learned_stage=1)
    net.close()

    # operator entry points on device arrays
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    with StokesSolver(3, (32, 32, 32), p3.dx, knobs=abi.make_knobs(precon_type=2, visc_type=-2)) as s:
        s.load_coeffs([dev(a) for a in p3.alpha_fc], dev(p3.beta), [dev(a) for a in p3.beta_ed], dev(p3.gamma), p3.theta_alpha)
        g = torch.Generator().manual_seed(7)
        rhs = [torch.randn(32, 32, 32, generator=g, dtype=torch.float64).cuda() for _ in range(3)]
        phi = [torch.randn(32, 32, 32, generator=g, dtype=torch.float64).cuda() for _ in range(3)]
        out = [torch.empty_like(a) for a in phi]
        coarse = [torch.zeros(16, 16, 16, dtype=torch.float64, device="cuda") for _ in range(3)]
        for color in range(7):
            s.smooth(0, rhs, phi, color)
        s.stag_applyop(phi, out, 0)
        s.residual_restrict(0, rhs, phi, coarse)
        s.prolong_add(0, coarse, phi)
        p = torch.randn(32, 32, 32, generator=g, dtype=torch.float64).cuda()
        res["ops_phi"] = np.stack([a.cpu().numpy() for a in phi])
        res["ops_applyop"] = np.stack([a.cpu().numpy() for a in out])
        res["ops_inner"] = np.array(s.inner_prod(phi, p, rhs, p))
        res["ops_sum"] = np.array(s.sum_umac_press(phi, p))
        # the entry point without a handle, on the same arrays
        o = (C.c_double * 6)()
        n3 = (C.c_int * 3)(32, 32, 32)
        rc = lib.lmm_inner_prod_noalloc(3, n3, abi.ptr_array(phi), abi.ptr(p), abi.ptr_array(rhs), abi.ptr(p), 1.0, None, o)
        status.append(rc)
        if rc != 0:
            print(f"noalloc: status {rc}: {lib.lmm_strerror(rc).decode()}", flush=True)
        res["noalloc"] = np.array(list(o))

    # a batched 2D ensemble (one batch handle per grid size)
    probs = ensemble.make_instances(6, seed=5, sizes=(32, 48), theta_alpha=0.0)
    kn = abi.make_knobs(precon_type=2, visc_type=-2, method=abi.LMM_METHOD_FGMRES, precision=1, gmres_rel_tol=1e-8)
    st, _, sols, _ = ensemble.solve(probs, kn, workers=2)
    status.extend(int(v) for v in st)
    for q, (xu, xp) in enumerate(sols):
        res[f"ens{q}_p"] = xp.cpu().numpy()
    res["status"] = np.array(status)
    np.savez(out_path, **res)


if __name__ == "__main__":
    main(sys.argv[1])

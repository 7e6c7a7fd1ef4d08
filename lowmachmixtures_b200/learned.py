"""Host driver of the learned preconditioner stage (include/lmm_learned.h).

The network is trained on the GPU by the library's own kernels on
(residual, error) pairs that the solver's own operators generate from
seeded viscosity fields (lmm_learned_make_pairs): a random error e0, r0 = A e0,
one application of the mixed-precision block preconditioner z1 = M r0, and
the pair (r1 = A (e0 - z1), e1 = e0 - z1).  The stage then corrects every
FP32 V-cycle application inside FGMRES, accepted only when it lowers the
residual.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import struct
import time

import numpy as np

from . import abi, synth


def _lib():
    from . import _native
    return _native.load()


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def field_contrast(seed: int) -> float:
    """viscosity contrast of training / evaluation field `seed`: log-uniform
    in [10, 1000]"""
    u = np.random.Generator(np.random.PCG64(90001 + seed)).uniform()
    return float(10.0 ** (1.0 + 2.0 * u))


class Net:
    """The encoder-decoder on an (nx, ny, nz) grid with `batch` samples."""

    def __init__(self, n, batch: int = 1, seed: int = 0):
        self.lib = _lib()
        self.h = C.c_void_p()
        nx, ny, nz = n
        rc = self.lib.lmm_net_create(nx, ny, nz, batch, seed, C.byref(self.h))
        if rc != 0:
            raise RuntimeError(f"lmm_net_create: {rc}")
        self.n, self.batch = tuple(n), batch

    @property
    def num_params(self) -> int:
        return int(self.lib.lmm_net_num_params(self.h))

    def params(self) -> np.ndarray:
        p = np.zeros(self.num_params, np.float32)
        assert self.lib.lmm_net_params(self.h, p.ctypes.data_as(C.c_void_p), 0) == 0
        return p

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.num_params
        assert self.lib.lmm_net_params(self.h, p.ctypes.data_as(C.c_void_p), 1) == 0

    def save(self, path: str):
        """the weight file of include/lmm_learned.h (lmm_net_save)"""
        rc = self.lib.lmm_net_save(self.h, os.fsencode(path))
        if rc != 0:
            raise RuntimeError(f"lmm_net_save: {self.lib.lmm_strerror(rc).decode()}")

    def load(self, path: str):
        """set the weights from a weight file, after its checks (lmm_net_load)"""
        rc = self.lib.lmm_net_load(self.h, os.fsencode(path))
        if rc != 0:
            raise RuntimeError(f"lmm_net_load: {self.lib.lmm_strerror(rc).decode()}")

    def close(self):
        if self.h:
            self.lib.lmm_net_destroy(self.h)
            self.h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


# ------------------------------------------------------------ weight files
# The flat file of include/lmm_learned.h, read and written without a GPU
# (lmm_net_save / lmm_net_load are the library's side of the same format).
WEIGHT_MAGIC = b"LMMNET01"
WEIGHT_VERSION = 1
LAYERS = ((8, 16), (16, 16), (16, 32), (32, 32), (32, 64), (64, 64), (64, 32), (32, 32), (32, 16), (16, 16), (16, 4))


def fnv1a64(data: bytes) -> int:
    """FNV-1a, 64-bit (the weight file's parameter checksum)"""
    h = 14695981039346656037
    for b in data:
        h = ((h ^ b) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


def num_params() -> int:
    return sum(co * 27 * ci + co for ci, co in LAYERS)


def write_weights(path: str, params: np.ndarray):
    p = np.ascontiguousarray(params, dtype="<f4")
    if p.size != num_params():
        raise ValueError(f"{p.size} parameters, the network has {num_params()}")
    payload = p.tobytes()
    head = WEIGHT_MAGIC + struct.pack("<II", WEIGHT_VERSION, len(LAYERS))
    head += b"".join(struct.pack("<II", ci, co) for ci, co in LAYERS)
    head += struct.pack("<QQ", p.size, fnv1a64(payload))
    with open(path, "wb") as f:
        f.write(head + payload)


def read_weights(path: str) -> np.ndarray:
    """the parameters of a weight file, after the checks lmm_net_load makes"""
    with open(path, "rb") as f:
        data = f.read()
    if data[:8] != WEIGHT_MAGIC:
        raise ValueError("not a weight file (magic)")
    version, nl = struct.unpack_from("<II", data, 8)
    if version != WEIGHT_VERSION:
        raise ValueError("unsupported weight-file version")
    table = [struct.unpack_from("<II", data, 16 + 8 * l) for l in range(nl)]
    if tuple(table) != LAYERS:
        raise ValueError("weight file for another architecture")
    count, h = struct.unpack_from("<QQ", data, 16 + 8 * nl)
    payload = data[32 + 8 * nl:]
    if count != num_params() or len(payload) != 4 * count:
        raise ValueError("weight file size does not match its header")
    if fnv1a64(payload) != h:
        raise ValueError("weight-file checksum mismatch")
    return np.frombuffer(payload, dtype="<f4").copy()


def mixed_knobs(**extra) -> abi.Knobs:
    kw = dict(precon_type=2, visc_type=-2, method=abi.LMM_METHOD_FGMRES, precision=abi.LMM_PRECISION_FP32,
              orthogonalization=1)
    kw.update(extra)
    return abi.make_knobs(**kw)


def _load(solver, prob):
    import torch
    dev = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()  # noqa: E731
    solver.load_coeffs([dev(a) for a in prob.alpha_fc], dev(prob.beta), [dev(b) for b in prob.beta_ed], dev(prob.gamma),
                       prob.theta_alpha)


def train(n: int = 64, fields: int = 200, steps: int = 2000, batch: int = 4, lr: float = 1e-3, seed: int = 0,
          theta_alpha: float = 0.0, field_seed0: int = 1000, log=None):
    """Train a network on pairs from `fields` seeded viscosity fields
    (steps // fields consecutive steps per field, `batch` fresh pairs per
    step, i.e. steps * batch pairs).  Returns (Net with batch 1 and the
    trained parameters, loss history, seconds)."""
    import torch

    from .gmres import StokesSolver
    lib = _lib()
    t0 = time.time()
    hist = []
    with StokesSolver(3, (n, n, n), 1.0 / n, knobs=mixed_knobs()) as s, Net((n, n, n), batch, seed) as net:
        assert lib.lmm_stokes_set_net(s._h, net.h) == 0
        x = torch.zeros(batch, n, n, n, 8, dtype=torch.bfloat16, device="cuda")
        t = torch.zeros(batch, n, n, n, 4, dtype=torch.float32, device="cuda")
        per_field = max(1, steps // fields)
        for step in range(steps):
            if step % per_field == 0:
                f = field_seed0 + step // per_field
                prob = synth.make_problem(3, n, field_contrast(f), f, theta_alpha=theta_alpha * n * n)
                _load(s, prob)
            rc = lib.lmm_learned_make_pairs(s._h, seed * 1000003 + step, batch, _ptr(x), _ptr(t))
            assert rc == 0, rc
            # cosine learning-rate decay
            lr_k = lr * 0.5 * (1.0 + math.cos(math.pi * step / steps))
            loss = C.c_float()
            rc = lib.lmm_net_train_step(net.h, _ptr(x), _ptr(t), lr_k, C.byref(loss))
            assert rc == 0, rc
            hist.append(loss.value)
            if log and (step % 100 == 0 or step == steps - 1):
                log(f"step {step} loss {loss.value:.4e}")
        params = net.params()
    out = Net((n, n, n), 1, seed)
    out.set_params(params)
    return out, hist, time.time() - t0


def residual_ratios(net: Net, prob, seeds, knobs: abi.Knobs | None = None):
    """[(|r1|/|r0|, |r1 - A c|/|r1|)] on fresh random pairs of problem `prob`"""
    from .gmres import StokesSolver
    lib = _lib()
    out = []
    with StokesSolver(3, prob.n[:3], prob.dx, knobs=knobs or mixed_knobs()) as s:
        assert lib.lmm_stokes_set_net(s._h, net.h) == 0
        _load(s, prob)
        for sd in seeds:
            r = (C.c_double * 2)()
            assert lib.lmm_learned_eval(s._h, sd, r) == 0
            out.append((r[0], r[1]))
    return out


def solve_with(prob, net: Net | None, knobs: abi.Knobs | None = None, repeats: int = 2):
    """Solve `prob` with FGMRES + FP32 V-cycles, with (net given) or without
    the learned stage.  Returns (iterations, ms of the last solve, true
    relative residual, accepted, tried)."""
    import torch

    from .gmres import StokesSolver
    lib = _lib()
    kn = knobs or mixed_knobs(learned_stage=1 if net is not None else 0)
    dev = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()  # noqa: E731
    bu, bp = [dev(a) for a in prob.b_u], dev(prob.b_p)
    al, be, bed, ga = [dev(a) for a in prob.alpha_fc], dev(prob.beta), [dev(b) for b in prob.beta_ed], dev(prob.gamma)
    with StokesSolver(3, prob.n[:3], prob.dx, knobs=kn) as s:
        if net is not None:
            assert lib.lmm_stokes_set_net(s._h, net.h) == 0
        for _ in range(repeats):
            xu, xp = [torch.zeros_like(bu[0]) for _ in range(3)], torch.zeros_like(bp)
            _, _, st = s.solve_device(bu, bp, xu, xp, al, be, bed, ga, prob.theta_alpha)
        acc, tried = C.c_int(), C.c_int()
        lib.lmm_learned_stats(s._h, C.byref(acc), C.byref(tried))
    return st["total_iter"], st["solve_ms"], st["norm_resid_true"] / st["norm_b"], acc.value, tried.value


def evaluate(net: Net, seeds, n: int = 64, log=None):
    """Held-out comparison on `seeds` (the learned-stage problems: n^3, theta = 0,
    contrast log-uniform in [10, 1000]): FGMRES + FP32 V-cycles with and
    without the learned stage, and the residual ratios of one application."""
    out = []
    for f in seeds:
        prob = synth.make_problem(3, n, field_contrast(f), f)
        rr = residual_ratios(net, prob, [f])[0]
        a = solve_with(prob, None)
        b = solve_with(prob, net)
        row = dict(seed=f, contrast=prob.contrast, mg_ratio=rr[0], net_ratio=rr[1], iters_plain=a[0], ms_plain=a[1],
                   res_plain=a[2], iters_learned=b[0], ms_learned=b[1], res_learned=b[2], accepted=b[3], tried=b[4])
        out.append(row)
        if log:
            log(row)
    return out


def main():
    import argparse
    import json
    ap = argparse.ArgumentParser(description="train the learned stage on the GPU and evaluate it on held-out seeds")
    ap.add_argument("--n", type=int, default=64)
    ap.add_argument("--fields", type=int, default=200)
    ap.add_argument("--steps", type=int, default=5000)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--eval-seeds", type=int, default=50)
    ap.add_argument("--out", default="")
    ap.add_argument("--save-weights", default="", help="write the trained weights (include/lmm_learned.h format)")
    ap.add_argument("--load-weights", default="", help="evaluate these weights instead of training")
    a = ap.parse_args()
    if a.load_weights:
        net, hist, secs = Net((a.n,) * 3, 1, 0), [float("nan")], 0.0
        net.load(a.load_weights)
    else:
        net, hist, secs = train(n=a.n, fields=a.fields, steps=a.steps, batch=a.batch, lr=a.lr,
                                log=lambda m: print(m, flush=True))
    if a.save_weights:
        net.save(a.save_weights)
    rows = evaluate(net, range(5000, 5000 + a.eval_seeds), n=a.n, log=lambda r: print(json.dumps(r), flush=True))
    summary = dict(train_seconds=secs, pairs=a.steps * a.batch, fields=a.fields, loss_first=hist[0],
                   loss_last=float(np.mean(hist[-50:])),
                   iters_plain=float(np.mean([r["iters_plain"] for r in rows])),
                   iters_learned=float(np.mean([r["iters_learned"] for r in rows])),
                   ms_plain=float(np.mean([r["ms_plain"] for r in rows])),
                   ms_learned=float(np.mean([r["ms_learned"] for r in rows])),
                   net_ratio=float(np.mean([r["net_ratio"] for r in rows])),
                   accept_rate=float(np.sum([r["accepted"] for r in rows]) / max(1, np.sum([r["tried"] for r in rows]))))
    print(json.dumps(summary), flush=True)
    if a.out:
        with open(a.out, "w") as f:
            json.dump(dict(summary=summary, rows=rows), f, indent=1)
    net.close()


if __name__ == "__main__":
    main()

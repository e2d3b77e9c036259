"""Evaluation behind the learned preconditioner's architecture: the 4-level
convolutional U-Net of configuration 3 (3x3 kernels, 16/32/48/64 channels,
BF16 weights with FP32 accumulation) against the V-cycle network the library
ships (cfdapp_b200/csrc/mg.cu), both inside FP64 flexible CG on the same 2D
p' systems, to a relative residual of 1e-8.

    python -m cfdapp_b200.unet_study [--steps 600] [--eval 512,1024,2048] > unet_study.json

The U-Net is built and trained with torch's library convolutions on the GPU;
it exists only for this comparison, not on the product path.  Training
follows the V-cycle's own recipe (cfdapp_b200/mgtrain.py): the loss
mean ||e - M A e||_A^2 / ||e||_A^2 over multi-scale random error fields e
on p' systems harvested from the library's GPU SIMPLE runs of lid-driven
cavities (Re uniform in [100, 1000], 256^2 and 512^2) plus the isolated
system.  The network sees the diagonally scaled residual and the log face
coefficients (so it can adapt to the operator); its output is scaled back by
D^-1/2 and the pinned reference cell is held at 0.

Reported per evaluation system: FCG iterations to 1e-8 (cap --cap), the
measured device time of one U-Net application (CUDA events, BF16 autocast),
the U-Net solve's total device time, and the library's learned V-cycle FCG
and FP64 Jacobi-PCG on the same system for comparison.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np


def _torch():
    import torch
    return torch


# ------------------------------------------------------------------ operator
class Op2D:
    """The 2D p' operator from face coefficients in the library's global face
    order (x-faces (ny, nx+1), then y-faces (ny+1, nx)), pinned cell 0."""

    def __init__(self, faces: np.ndarray, n: int, device, pinned=True):
        torch = _torch()
        nfx = (n + 1) * n
        fx = torch.tensor(faces[:nfx].reshape(n, n + 1), dtype=torch.float64, device=device)
        fy = torch.tensor(faces[nfx:].reshape(n + 1, n), dtype=torch.float64, device=device)
        self.n = n
        self.xl, self.xh = fx[:, :-1].clone(), fx[:, 1:].clone()
        self.yl, self.yh = fy[:-1, :].clone(), fy[1:, :].clone()
        self.diag = ((self.xl + self.xh) + self.yl) + self.yh
        self.xl[:, 0] = 0.0
        self.xh[:, -1] = 0.0
        self.yl[0, :] = 0.0
        self.yh[-1, :] = 0.0
        self.pinned = pinned
        if pinned:
            self.diag[0, 0] = 1.0
        self.isd = 1.0 / torch.sqrt(self.diag)
        # cell-centred features: log of the couplings along each axis
        self.feat = torch.stack([torch.log(0.5 * (fx[:, :-1] + fx[:, 1:]) + 1e-30),
                                 torch.log(0.5 * (fy[:-1, :] + fy[1:, :]) + 1e-30)])
        self.feat = (self.feat - self.feat.mean()) / (self.feat.std() + 1e-12)

    def apply(self, x):
        torch = _torch()
        y = self.diag * x
        y[:, 1:] -= self.xl[:, 1:] * x[:, :-1]
        y[:, :-1] -= self.xh[:, :-1] * x[:, 1:]
        y[1:, :] -= self.yl[1:, :] * x[:-1, :]
        y[:-1, :] -= self.yh[:-1, :] * x[1:, :]
        if self.pinned:
            y[0, 0] = x[0, 0]
            # the neighbours of the pinned cell keep their coupling to it
        return y


# ------------------------------------------------------------------ U-Net
def make_unet(device):
    torch = _torch()
    nn = torch.nn

    def block(cin, cout):
        return nn.Sequential(nn.Conv2d(cin, cout, 3, padding=1, bias=False), nn.ReLU(),
                             nn.Conv2d(cout, cout, 3, padding=1, bias=False), nn.ReLU())

    class UNet(nn.Module):
        def __init__(self, ch=(16, 32, 48, 64)):
            super().__init__()
            self.enc = nn.ModuleList([block(3, ch[0]), block(ch[0], ch[1]), block(ch[1], ch[2])])
            self.mid = block(ch[2], ch[3])
            self.up = nn.ModuleList([nn.ConvTranspose2d(ch[3], ch[2], 2, stride=2, bias=False),
                                     nn.ConvTranspose2d(ch[2], ch[1], 2, stride=2, bias=False),
                                     nn.ConvTranspose2d(ch[1], ch[0], 2, stride=2, bias=False)])
            self.dec = nn.ModuleList([block(2 * ch[2], ch[2]), block(2 * ch[1], ch[1]),
                                      block(2 * ch[0], ch[0])])
            self.out = nn.Conv2d(ch[0], 1, 1, bias=False)

        def forward(self, x):
            skips = []
            for e in self.enc:
                x = e(x)
                skips.append(x)
                x = nn.functional.avg_pool2d(x, 2)
            x = self.mid(x)
            for u, d, s in zip(self.up, self.dec, reversed(skips)):
                x = d(torch.cat([u(x), s], dim=1))
            return self.out(x)

    return UNet().to(device)


def precondition(net, op: Op2D, r, bf16=True):
    """z = M r: the network on the scaled residual and the coefficient
    features, scaled back by D^-1/2; the pinned cell held at 0."""
    torch = _torch()
    s = op.isd * r
    scale = torch.sqrt((s * s).mean()) + 1e-300
    inp = torch.cat([(s / scale)[None], op.feat], dim=0)[None].float()
    with torch.autocast("cuda", dtype=torch.bfloat16, enabled=bf16):
        out = net(inp)
    z = op.isd * (out[0, 0].double() * scale)
    if op.pinned:
        z[0, 0] = 0.0
    return z


def random_errors(n, count, gen, device):
    """Multi-scale random error fields (sums of bilinearly upsampled noise)."""
    torch = _torch()
    out = []
    for _ in range(count):
        e = torch.zeros(n, n, dtype=torch.float64, device=device)
        m = 4
        while m <= n:
            g = torch.randn(1, 1, m, m, generator=gen, device=device, dtype=torch.float64)
            e += torch.nn.functional.interpolate(g, size=(n, n), mode="bilinear",
                                                 align_corners=False)[0, 0] * (m / n) ** 0.5
            m *= 2
        e[0, 0] = 0.0
        out.append(e)
    return out


def train(net, ops, steps, device, log):
    torch = _torch()
    opt = torch.optim.Adam(net.parameters(), lr=1e-3)
    sched = torch.optim.lr_scheduler.CosineAnnealingLR(opt, steps)
    gen = torch.Generator(device=device)
    gen.manual_seed(20261204)
    for it in range(steps):
        op = ops[it % len(ops)]
        loss = 0.0
        for e in random_errors(op.n, 2, gen, device):
            r = op.apply(e)
            z = precondition(net, op, r, bf16=True)
            d = e - z
            loss = loss + (d * op.apply(d)).sum() / (e * op.apply(e)).sum()
        loss = loss / 2
        opt.zero_grad()
        loss.backward()
        opt.step()
        sched.step()
        if it % 100 == 0 or it == steps - 1:
            log.append({"step": it, "loss": float(loss)})
    return net


def fcg(op: Op2D, b, M, tol=1e-8, cap=2000):
    """FP64 flexible CG (truncation 1), x0 = 0; returns iterations, the true
    relative residual and the device time (ms)."""
    torch = _torch()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record()
    x = torch.zeros_like(b)
    r = b.clone()
    b0 = torch.linalg.norm(r)
    z = M(r)
    p = z.clone()
    q = op.apply(p)
    it = 0
    while it < cap:
        it += 1
        pq = (p * q).sum()
        alpha = (p * r).sum() / pq
        x += alpha * p
        r -= alpha * q
        if float(torch.linalg.norm(r) / b0) <= tol:
            break
        z = M(r)
        beta = -(z * q).sum() / pq
        p = z + beta * p
        q = op.apply(p)
    stop.record()
    torch.cuda.synchronize()
    true = float(torch.linalg.norm(b - op.apply(x)) / b0)
    return it, true, start.elapsed_time(stop)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=600)
    ap.add_argument("--eval", default="512,1024,2048")
    ap.add_argument("--cap", type=int, default=2000)
    a = ap.parse_args()
    torch = _torch()
    from . import cfdb
    device = "cuda"
    ctx = cfdb.Context(0)
    rng = np.random.default_rng(20261204)
    report = {"architecture": "U-Net, 4 levels, 3x3 convolutions, 16/32/48/64 channels, ReLU, "
                              "average-pool down, transposed-conv up, BF16 autocast (FP32 "
                              "accumulate)", "training": {}, "systems": []}

    def harvest(n, re, outer):
        case = cfdb.SimpleCase.cavity(2, n, mu=1.0 / re)
        s = cfdb.SIMPLESettings(max_iterations=outer, velocity_tolerance=0.0,
                                pressure_tolerance=0.0, continuity_tolerance=0.0)
        sim = cfdb.Simple(ctx, case, s)
        sim.set_state(None, None, None, None)
        sim.iterate(outer)
        faces, pinned, ref = sim.pprime_faces()
        sim.close()
        return faces

    def unit_faces(n):
        fx = np.ones((n, n + 1))
        fx[:, 0] = fx[:, -1] = 0.0
        fy = np.ones((n + 1, n))
        fy[0, :] = fy[-1, :] = 0.0
        return np.concatenate([fx.reshape(-1), fy.reshape(-1)])

    t0 = time.perf_counter()
    train_ops = [Op2D(unit_faces(256), 256, device)]
    for n in (256, 512):
        for _ in range(3):
            re = float(rng.uniform(100.0, 1000.0))
            train_ops.append(Op2D(harvest(n, re, int(rng.integers(20, 200))), n, device))
    net = make_unet(device)
    log = []
    train(net, train_ops, a.steps, device, log)
    report["training"] = {"systems": len(train_ops), "steps": a.steps, "loss": log,
                          "seconds": time.perf_counter() - t0,
                          "parameters": int(sum(p.numel() for p in net.parameters()))}
    net.eval()
    for n in [int(t) for t in a.eval.split(",")]:
        for kind in ("isolated", "cavity Re 700"):
            faces = unit_faces(n) if kind == "isolated" else harvest(n, 700.0, 100)
            op = Op2D(faces, n, device)
            b = torch.tensor(cfdb.synth_rhs(2, n).reshape(n, n), dtype=torch.float64,
                             device=device)
            b[0, 0] = 0.0
            with torch.no_grad():
                # one U-Net application, timed alone
                r = b.clone()
                for _ in range(3):
                    precondition(net, op, r)
                ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                ev0.record()
                for _ in range(10):
                    precondition(net, op, r)
                ev1.record()
                torch.cuda.synchronize()
                apply_ms = ev0.elapsed_time(ev1) / 10
                it, true, ms = fcg(op, b, lambda v: precondition(net, op, v), cap=a.cap)
            # the library's solves of the same system
            pop = cfdb.POperator(ctx, 2, (n, n), face_coeff=faces)
            bh = b.cpu().numpy().reshape(-1)
            lib = {}
            for pre in ("learned_mg", "jacobi"):
                s = cfdb.LinearSolverSettings(absolute_tolerance=0.0, relative_tolerance=1e-8,
                                              max_iterations=200000, preconditioner=pre)
                pop.solve(bh, s)  # warm-up (hierarchy, graph)
                res = pop.solve(bh, s)
                lib[pre] = {"iterations": res.iterations, "device_ms": res.device_ms,
                            "true_rel_residual": res.true_residual / res.initial_residual}
            pop.close()
            report["systems"].append({
                "n": n, "system": kind,
                "unet": {"iterations": it, "converged": true <= 1.01e-8, "true_rel_residual": true,
                         "apply_ms": apply_ms, "solve_ms": ms},
                "vcycle_fcg": lib["learned_mg"], "jacobi_pcg": lib["jacobi"]})
            print(json.dumps(report["systems"][-1]), flush=True)
    print(json.dumps(report), flush=True)
    ctx.close()


if __name__ == "__main__":
    main()

"""Train the learned-FSAI network on the GPU and write its weight file.

    python -m tpt_fem.train_lfsai --family elasticity --out weights/lfsai_elasticity.bin
    python -m tpt_fem.train_lfsai --family poisson    --out weights/lfsai_poisson.bin

Families (seeded synthetic inputs):
  elasticity : cantilevers on box [0,4]x[0,1]x[0,1] (x=0 clamped, traction
               (0,0,-1e-3) on x=4, nu=0.3, E = 1e-3 + (1-1e-3) rho^3 from the
               smoothed density of `workloads`), box_mesh [40,10,10],
               [56,14,14] and [80,20,20], several density seeds.
  poisson    : unit cube, u=0 on every face, f=1, k = exp(g) with g the seeded
               Gaussian random field (variance 1, correlation length 0.1) at
               tet centroids; box_mesh 32^3 and 64^3 (the training sizes of the
               heterogeneous-Poisson configuration).
Every training step runs the library's own Kaporin loss/gradient kernels and
Adam on the device on one training system.  The script keeps the parameters
with the lowest mean iteration count on held-out validation systems.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

if __package__ in (None, ""):
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import tpt_fem as F  # noqa: E402
from tpt_fem import lfsai as LF  # noqa: E402
from tpt_fem import workloads as W  # noqa: E402


def cantilever(ctx, n, seed):
    mn, mx = [0.0, 0.0, 0.0], [4.0, 1.0, 1.0]
    mesh = F.Mesh.box_mesh(mn, mx, n, ctx=ctx)
    K = F.assemble_elasticity(mesh, "3d", W.cantilever_young(n, seed=seed), 0.3, 2)
    rhs = F.apply_traction(mesh, 3, 0, 1.0, [0.0, 0.0, -1e-3], np.zeros(K.nrows))
    dof, val = W.clamp_x0_bcs(W.box_coords(mn, mx, n))
    return F.reduce_system(K, rhs, list(zip(dof, val)))


def grf_poisson(ctx, n, seed):
    return W.grf_poisson_system(ctx, n, seed)


FAMILIES = {
    "elasticity": dict(build=cantilever,
                       train=[([40, 10, 10], s) for s in range(100, 106)] + [([56, 14, 14], s) for s in range(106, 110)]
                       + [([80, 20, 20], s) for s in range(110, 112)],
                       valid=[([100, 25, 25], 900), ([120, 30, 30], 901)]),
    "poisson": dict(build=grf_poisson,
                    train=[(32, s) for s in range(0, 192)] + [(64, s) for s in range(192, 256)],
                    valid=[(96, 1000), (96, 1001)]),
}


def mean_iters(systems, model, solver):
    its = []
    for S in systems:
        if solver == F.SOLVER_LEARNED_FSAI_PCG:
            model.attach(S)
        st = S.solve(solver=solver, tol=1e-10, fresh_setup=True)
        its.append(st["iterations"] if not st["fell_back"] else 10 ** 9)
    return float(np.mean(its))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--family", choices=sorted(FAMILIES), required=True)
    ap.add_argument("--out", required=True)
    ap.add_argument("--epochs", type=int, default=6)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--max-train", type=int, default=0, help="use at most this many training systems")
    args = ap.parse_args()
    fam = FAMILIES[args.family]
    ctx = F.Context(0)
    rng = np.random.default_rng(args.seed)
    t0 = time.time()
    specs = fam["train"][: args.max_train] if args.max_train else fam["train"]
    train = []
    for spec in specs:
        train.append(fam["build"](ctx, *spec))
    valid = [fam["build"](ctx, *spec) for spec in fam["valid"]]
    print(f"built {len(train)} training / {len(valid)} validation systems in {time.time() - t0:.1f}s", flush=True)
    model = LF.LearnedFsai(ctx, seed=args.seed)
    log = {"family": args.family, "jacobi_valid_iters": mean_iters(valid, model, F.SOLVER_JACOBI_PCG),
           "fsai_valid_iters": mean_iters(valid, model, F.SOLVER_FSAI_MP_PCG), "epochs": []}
    best = (mean_iters(valid, model, F.SOLVER_LEARNED_FSAI_PCG), model.get_params())
    log["initial_valid_iters"] = best[0]
    print(json.dumps(log), flush=True)
    for ep in range(args.epochs):
        order = rng.permutation(len(train))
        losses = []
        for k in order:
            loss, _ = model.loss(train[k], grad=True)
            model.adam(args.lr)
            losses.append(loss)
        it = mean_iters(valid, model, F.SOLVER_LEARNED_FSAI_PCG)
        rec = {"epoch": ep, "mean_loss": float(np.mean(losses)), "valid_iters": it, "t": time.time() - t0}
        log["epochs"].append(rec)
        print(json.dumps(rec), flush=True)
        if it < best[0]:
            best = (it, model.get_params())
    model.set_params(best[1])
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    model.save(args.out)
    log["best_valid_iters"] = best[0]
    with open(os.path.splitext(args.out)[0] + ".json", "w") as f:
        json.dump(log, f, indent=1)
    print(json.dumps({"saved": args.out, "best_valid_iters": best[0]}), flush=True)


if __name__ == "__main__":
    main()

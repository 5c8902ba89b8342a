"""Train the learned preconditioner on the GPU and write its checkpoint.

  python -m actfemtide_b200.train_learned [--models 512] [--steps 2] [--lr 1e-3] [--base hybrid|jacobi] [--out PATH]
  python -m actfemtide_b200.train_learned --eval-only [--eval 4]     (held-out evaluation against the base
                                                                     alone, and the network's time per iteration)

Training models: seeded log-normal conductivity on the 32x32x24 mesh (air and
sea layers, M2 source); residuals from FP64 COCG with the network's base
preconditioner (the gradient-corrected SSOR, or SSOR for the Jacobi base);
the network's own forward/backward kernels and Adam on the device.  After
training, the held-out evaluation compares flexible COCG with the network
against its base alone and against the reference's SSOR-COCG on fresh models.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import learned, synth
from .forward import Forward


def evaluate(fw, params, models, freq, tol=1e-8, maxit=20000, base=0, with_ssor=True):
    """Iterations and time of flexible COCG with the network against its base and the reference's SSOR."""
    rows = []
    fw.mpnn_set_params(params)
    fw.mpnn_set_base(base == 1)
    runs = (("learned", "LEARNED"), ("hybrid", "HYBRID"), ("ssor", "SSOR")) if base == 1 else \
        (("learned", "LEARNED"), ("none", "NONE"), ("ssor", "SSOR"))
    if not with_ssor:
        runs = runs[:2]
    for m in models:
        fw.set_cond(m.sigma_air, m.sigma_ocean, 1, sigma_file=m.sigma_land)
        fw.assemble()
        rec = {}
        for name, pc in runs:
            r = fw.solve(freq, precond=pc, tol=tol, maxit=maxit)
            rec[name] = {"iterations": r.iterations, "seconds": r.seconds, "resid_true": r.resid_true,
                         "status": r.status}
        rows.append(rec)
    return rows


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--models", type=int, default=512)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--epochs", type=int, default=1)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--eval", type=int, default=4, help="held-out training-mesh models to evaluate")
    ap.add_argument("--base", choices=["jacobi", "hybrid"], default="hybrid",
                    help="jacobi: the network is the preconditioner; hybrid: it corrects the gradient-corrected SSOR")
    ap.add_argument("--out", default=None)
    ap.add_argument("--eval-only", action="store_true",
                    help="no training: evaluate the saved checkpoint, and time the network per iteration "
                         "(zero output weights leave the iterations of the base, so the time difference is the network)")
    a = ap.parse_args()
    base = 1 if a.base == "hybrid" else 0
    out = a.out or (learned.HYBRID_CKPT if base else learned.DEFAULT_CKPT)
    freq = 1.0 / synth.M2_PERIOD_S
    t0 = time.time()
    if a.eval_only:
        with Forward(0) as fw:
            held = [learned.training_model(100_000 + k) for k in range(a.eval)]
            fw.load_model(held[0])
            ev = evaluate(fw, learned.load(out), held, freq, base=base, with_ssor=False)
            ev0 = evaluate(fw, learned.init_params(a.seed), held[:1], freq, base=base, with_ssor=False)
        r0 = ev0[0]
        ref = r0["hybrid" if base else "none"]
        per_it = (r0["learned"]["seconds"] - ref["seconds"]) / max(1, r0["learned"]["iterations"])
        print(json.dumps({"checkpoint": out, "held_out": ev, "zero_output_weights": r0,
                          "network_ms_per_iteration": 1e3 * per_it, "wall_s": time.time() - t0}))
        return
    with Forward(0) as fw:
        p, rec = learned.train(fw, a.models, a.steps, a.lr, a.seed, a.epochs, base=base)
        held = [learned.training_model(100_000 + k) for k in range(a.eval)]
        ev = evaluate(fw, p, held, freq, base=base)
        ev0 = evaluate(fw, learned.init_params(a.seed), held[:1], freq, base=base)
    rec["held_out"] = ev
    rec["untrained_held_out"] = ev0
    rec["wall_s"] = time.time() - t0
    learned.save(out, p, rec)
    print(json.dumps(rec))


if __name__ == "__main__":
    main()

"""Training and checkpoints of the learned preconditioner (the network lives in csrc/afem_mpnn.cu).

Training data: plain FP64 SSOR-COCG runs on seeded conductivity models of
one mesh supply residuals r_k (the right-hand side and the true residuals
after k iterations); the network is trained on the device, by its own
forward and backward kernels, to make A P(r) close to r.  Weights are kept
as FP32 masters and used in BF16; a checkpoint is a BF16 blob plus a JSON
header (shapes, training record).
"""
from __future__ import annotations

import json
import os
import time

import numpy as np

from . import synth

H, L, FIN = 48, 6, 8
SHAPES = [("W_in", (FIN, H))] + [x for l in range(L) for x in ((f"W{l}", (3 * H, H)), (f"c{l}", (H,)))] + \
    [("W_out", (H, 2))]
NPARAM = sum(int(np.prod(s)) for _, s in SHAPES)
WEIGHTS_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights")
DEFAULT_CKPT = os.path.join(WEIGHTS_DIR, "mpnn_tidal_32x32x24")
HYBRID_CKPT = os.path.join(WEIGHTS_DIR, "mpnn_tidal_32x32x24_hybrid")  # correction over the gradient-corrected SSOR


def flatten(P: dict) -> np.ndarray:
    return np.concatenate([np.asarray(P[k], np.float32).ravel() for k, _ in SHAPES])


def unflatten(p) -> dict:
    out, o = {}, 0
    for k, s in SHAPES:
        n = int(np.prod(s))
        out[k] = np.asarray(p[o:o + n], np.float64).reshape(s)
        o += n
    return out


def init_params(seed: int = 0, scale: float = 0.5) -> np.ndarray:
    """Random initial weights; W_out starts at zero so the untrained network is the Jacobi preconditioner."""
    rng = np.random.default_rng(seed)
    P = {"W_in": rng.standard_normal((FIN, H)) * scale / np.sqrt(FIN)}
    for l in range(L):
        P[f"W{l}"] = rng.standard_normal((3 * H, H)) * scale / np.sqrt(3 * H)
        P[f"c{l}"] = np.zeros(H)
    P["W_out"] = np.zeros((H, 2))
    return flatten(P)


def to_bf16_bits(p: np.ndarray) -> np.ndarray:
    u = np.asarray(p, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return u.astype(np.uint16)


def from_bf16_bits(b: np.ndarray) -> np.ndarray:
    return (np.asarray(b, np.uint32) << 16).view(np.float32)


def save(path: str, p: np.ndarray, meta: dict):
    os.makedirs(os.path.dirname(path), exist_ok=True)
    to_bf16_bits(p).tofile(path + ".bf16")
    hdr = dict(meta)
    hdr.update({"format": "bf16 little-endian, flat", "nparam": int(len(p)), "shapes": SHAPES,
                "network": {"width": H, "layers": L, "inputs": FIN}})
    with open(path + ".json", "w") as f:
        json.dump(hdr, f, indent=1)


def load_base(path: str = DEFAULT_CKPT) -> int:
    """The base the checkpoint was trained over: 0 Jacobi, 1 the gradient-corrected SSOR."""
    with open(path + ".json") as f:
        return int(json.load(f).get("base", 0))


def load(path: str = DEFAULT_CKPT) -> np.ndarray:
    with open(path + ".json") as f:
        hdr = json.load(f)
    p = from_bf16_bits(np.fromfile(path + ".bf16", dtype=np.uint16))
    if len(p) != hdr["nparam"] or len(p) != NPARAM:
        raise ValueError("checkpoint size does not match the network")
    return p


def training_model(k: int, nx=32, ny=32, nz=24):
    """Seeded log-normal model k on the 32x32x24 training mesh (air and sea layers, M2 source)."""
    return synth.tidal_box(nx, ny, nz, seed=k, field_seed=10_000 + k, grf=True, block=False, name=f"train{k}")


def collect_residuals(fw, freq, iters=(1, 4, 16, 64), precond="SSOR"):
    """True residuals b - A x_k of FP64 COCG (SSOR, or the network's base) after k iterations on the loaded system."""
    out = []
    for k in iters:
        fw.solve(freq, precond=precond, tol=1e-30, maxit=k)
        out.append(fw.residual(0))
    return np.stack(out)


def train(fw, n_models: int = 512, steps_per_model: int = 2, lr: float = 1e-3, seed: int = 0, epochs: int = 1,
          params=None, log=print, nx=32, ny=32, nz=24, base: int = 0):
    """Train on n_models seeded models of the training mesh; returns (params, record).

    base 0: the network is the preconditioner (Jacobi term plus its output),
    trained on residuals of SSOR-COCG; base 1: it corrects the gradient-corrected
    SSOR H (z = H(r) + N(r)), trained on residuals of H-preconditioned COCG."""
    freq = 1.0 / synth.M2_PERIOD_S
    p = init_params(seed) if params is None else np.asarray(params, np.float32)
    fw.mpnn_set_params(p)
    fw.mpnn_set_base(base == 1)
    m0 = training_model(0, nx, ny, nz)
    fw.load_model(m0)
    hist = []
    t0 = time.time()
    for ep in range(epochs):
        for k in range(n_models):
            m = training_model(k, nx, ny, nz)
            fw.set_cond(m.sigma_air, m.sigma_ocean, 1, sigma_file=m.sigma_land)
            fw.assemble()
            R = collect_residuals(fw, freq, precond="HYBRID" if base == 1 else "SSOR")
            h = fw.mpnn_train(freq, R, steps_per_model, lr)
            hist.append(float(h[-1]))
            if log and (k % 64 == 0 or k == n_models - 1):
                log(f"epoch {ep} model {k}: loss {h[-1]:.4f} ({time.time() - t0:.1f} s)")
    p = fw.mpnn_get_params()
    rec = {"models": n_models, "epochs": epochs, "steps_per_model": steps_per_model, "lr": lr, "seed": seed,
           "base": base,
           "mesh": f"{nx}x{ny}x{nz}", "loss_first": hist[0] if hist else None,
           "loss_last_64": float(np.mean(hist[-64:])) if hist else None, "seconds": time.time() - t0}
    return p, rec

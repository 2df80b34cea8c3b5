"""Trains the learned warm start on (divergence, pressure) pairs from the plain MGPCG solver and
evaluates it against a zero initial guess.

  python -m slosh_b200.train_warmstart --pairs 20000 --batch 4 --out slosh_b200/warmstart_128.npz
  python -m slosh_b200.train_warmstart --eval 200 --weights slosh_b200/warmstart_128.npz

Pairs: each randomised scene (warmstart.random_scene: 1-4 fluid boxes with N(0, 0.5^2) m/s
velocities, 0-3 static solid spheres, seeds 10000+) is stepped for one frame of one substep with a
zero initial guess; the solve's right-hand side, cell types and converged pressure are packed on the
device into a training slot (slosh_unet_capture_sample). Every pair is used once (online training, no
host copies of the volumes). Held-out scenes use seeds 90000+ and are never trained on.
"""
import argparse
import json
import os
import sys
import time

import numpy as np

from . import Simulation, _abi, frame_input, settings_default, PARTICLE_DTYPE
from . import warmstart as W

TRAIN_SEED0 = 10000
EVAL_SEED0 = 90000


def _scene(seed, n):
    s, emits, colliders = W.random_scene(settings_default, seed, n)
    s.min_substeps = 1
    s.max_substeps = 1
    return s, emits, colliders


class SceneRunner:
    """One simulation context reused across scenes (a scene starts from zero particles)."""

    def __init__(self, n=128):
        self.n = n
        s, _, _ = _scene(TRAIN_SEED0, n)
        s.particle_capacity = 1 << 23
        self.sim = Simulation(s)
        self.sim.enable_phase_timing(True)
        self.empty = np.zeros(0, dtype=PARTICLE_DTYPE)

    def run(self, seed, warm_start):
        s, emits, colliders = _scene(seed, self.n)
        s.particle_capacity = max(s.particle_capacity, 1 << 23)
        s.warm_start = warm_start
        self.sim.upload_particles(self.empty)
        self.sim.step_frame(frame_input(s, emits=emits, colliders=colliders))
        r = self.sim.results()
        return {"iterations": int(r.last_solve_iterations), "rel_residual": float(r.last_solve_rel_residual),
                "pressure_ms": float(self.sim.phase_ms()["pressure"]), "fluid_cells": int(r.fluid_cells)}

    def close(self):
        self.sim.close()


def _bf16_round(x):
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    return (((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16).astype(np.uint32).view(np.float32)


def save_weights(path, params, conv_weight_mask=None):
    """Stores the parameters; entries under conv_weight_mask (the convolution weights, which the network
    runs in BF16) are stored BF16-rounded, so their zero low halves compress away."""
    p = np.asarray(params, np.float32).copy()
    if conv_weight_mask is not None:
        p[conv_weight_mask] = _bf16_round(p[conv_weight_mask])
    np.savez_compressed(path, params=p)


def conv_weight_mask(num_params):
    """Positions of the convolution weights in the parameter vector (layout of unet.cu)."""
    chans = {"in": 16, "p1": 16, "p2": 32, "p3": 64, "u2": 64, "u1": 64, "u0": 32}
    layers = [(("in",), 16, "e0a"), (("e0a",), 16, "e0"), (("p1",), 32, "e1a"), (("e1a",), 32, "e1"), (("p2",), 64, "e2a"),
              (("e2a",), 64, "e2"), (("p3",), 64, "e3a"), (("e3a",), 64, "e3"), (("u2", "e2"), 64, "d2a"), (("d2a",), 64, "d2"),
              (("u1", "e1"), 32, "d1a"), (("d1a",), 32, "d1"), (("u0", "e0"), 16, "d0a"), (("d0a",), 16, "d0")]
    m = np.zeros(num_params, bool)
    off = 0
    for ins, n, name in layers:
        cin = sum(chans[i] for i in ins)
        m[off:off + 27 * n * cin] = True
        off += 27 * n * cin + n
        chans[name] = n
    assert off + 17 == num_params
    return m


def load_weights(path):
    with np.load(path) as z:
        return np.asarray(z["params"], np.float32)


def train(pairs, batch=4, n=128, lr=1e-3, seed=TRAIN_SEED0, log_every=250, weights=None, out=None, stream=sys.stdout):
    runner = SceneRunner(n)
    net = W.WarmStartNet(dim=(n, n, n), batch=batch, seed=seed, learning_rate=lr)
    if weights is not None:
        net.set_params(weights)
    steps = max(pairs // batch, 1)
    losses = []
    t0 = time.perf_counter()
    gen_s = train_s = 0.0
    for step in range(steps):
        ta = time.perf_counter()
        for k in range(batch):
            runner.run(seed + step * batch + k, _abi.WARM_START_ZERO)
            net.capture(runner.sim, k)
        tb = time.perf_counter()
        losses.append(net.train_step())
        tc = time.perf_counter()
        gen_s += tb - ta
        train_s += tc - tb
        if log_every and (step + 1) % log_every == 0:
            m = float(np.mean(losses[-log_every:]))
            print(json.dumps({"step": step + 1, "pairs": (step + 1) * batch, "loss": m, "elapsed_s": time.perf_counter() - t0}),
                  file=stream, flush=True)
    params = net.params()
    if out:
        save_weights(out, params, conv_weight_mask(len(params)))
    info = {"pairs": steps * batch, "batch": batch, "steps": steps, "first_loss": float(np.mean(losses[:min(20, len(losses))])),
            "last_loss": float(np.mean(losses[-min(20, len(losses)):])), "generate_s": gen_s, "train_s": train_s,
            "train_ms_per_step": 1e3 * train_s / steps}
    net.close()
    runner.close()
    return params, info


def evaluate(params, scenes=200, n=128, seed=EVAL_SEED0):
    """Per held-out scene: the first frame's solve from zero and from the network's guess."""
    runner = SceneRunner(n)
    net = W.WarmStartNet(dim=(n, n, n), batch=1)
    net.set_params(params)
    rows = []
    for k in range(scenes):
        W.attach(runner.sim, None)
        z = runner.run(seed + k, _abi.WARM_START_ZERO)
        W.attach(runner.sim, net)
        l = runner.run(seed + k, _abi.WARM_START_LEARNED)
        rows.append((z, l))
    W.attach(runner.sim, None)
    # network inference alone (pack + forward + scatter are inside the learned pressure phase)
    net.forward(out=False)
    t0 = time.perf_counter()
    reps = 5
    for _ in range(reps):
        net.forward(out=False)
    infer_ms = 1e3 * (time.perf_counter() - t0) / reps
    net.close()
    runner.close()
    iz = np.array([r[0]["iterations"] for r in rows], float)
    il = np.array([r[1]["iterations"] for r in rows], float)
    mz = np.array([r[0]["pressure_ms"] for r in rows], float)
    ml = np.array([r[1]["pressure_ms"] for r in rows], float)
    res_l = max(r[1]["rel_residual"] for r in rows)
    res_z = max(r[0]["rel_residual"] for r in rows)
    return {"scenes": scenes, "iterations_zero": float(iz.mean()), "iterations_learned": float(il.mean()),
            "iterations_saved": float((iz - il).mean()), "iterations_saved_frac": float(1.0 - il.sum() / iz.sum()),
            "pressure_ms_zero": float(mz.mean()), "pressure_ms_learned": float(ml.mean()),
            "pressure_ms_saved": float((mz - ml).mean()), "inference_ms": infer_ms,
            "rel_residual_max_zero": res_z, "rel_residual_max_learned": res_l,
            "scenes_fewer_iterations": int((il < iz).sum()), "scenes_more_iterations": int((il > iz).sum())}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--pairs", type=int, default=0, help="training pairs (0: no training)")
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--weights", default=None, help="start from (or evaluate) these weights")
    ap.add_argument("--out", default=None, help="write the trained weights here")
    ap.add_argument("--eval", type=int, default=0, help="held-out scenes to evaluate")
    ap.add_argument("--log-every", type=int, default=250)
    a = ap.parse_args(argv)
    params = load_weights(a.weights) if a.weights else None
    report = {}
    if a.pairs:
        params, info = train(a.pairs, a.batch, a.n, a.lr, weights=params, out=a.out, log_every=a.log_every)
        report["training"] = info
    if a.eval:
        if params is None:
            raise SystemExit("--eval needs --weights or --pairs")
        report["evaluation"] = evaluate(params, a.eval, a.n)
    print(json.dumps(report), flush=True)


if __name__ == "__main__":
    main()

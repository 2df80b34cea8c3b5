"""Generates tests/golden/golden.json: digests of the CPU oracle's state on small seeded scenes.

The reference has no golden vectors of its own; these fixtures freeze the oracle's results so a later
change to the oracle or to the GPU kernels that alters any bit is caught. Regenerate only on purpose:
    python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oracle import oracle as O  # noqa: E402
from slosh_b200 import _abi as A, scenes  # noqa: E402
from parity import active_slots, slot_mask  # noqa: E402

CASES = {
    "tiny16_mgpcg": dict(n=16, solver=A.SOLVER_MGPCG, colliders=False, frames=4),
    "tiny16_rbgs": dict(n=16, solver=A.SOLVER_RBGS, colliders=False, frames=4),
    "tiny24_collider": dict(n=24, solver=A.SOLVER_MGPCG, colliders=True, frames=3),
}


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def state_digests(sim):
    L = sim.layout()
    slots = active_slots(sim)
    cm = slot_mask(slots, L.pool_cells)
    fm = slot_mask(slots, L.pool_cells, 3)
    out = {"particles": digest(sim.read("PARTICLES")), "brick_table": digest(sim.read("BRICK_TABLE")),
           "active_bricks": digest(sim.read("ACTIVE_BRICKS")), "stats": [int(x) for x in sim.read("STATS")]}
    for name in ("CELL_TYPE", "PRESSURE", "DIVERGENCE", "CELL_DIAG", "DENSITY_Q"):
        out[name.lower()] = digest(sim.read(name)[cm])
    for name in ("VEL", "FACE_FLAGS", "FACE_WEIGHT"):
        out[name.lower()] = digest(sim.read(name)[fm])
    return out


def run_case(make_sim, case):
    sc = scenes.tiny(O.settings_default, n=case["n"], solver=case["solver"], colliders=case["colliders"])
    sim = make_sim(sc["settings"])
    sim.set_emit_seed(sc["seed"])
    fi = A.frame_input(sc["settings"], emits=sc["emits"], colliders=sc["colliders"])
    for _ in range(case["frames"]):
        sim.step_frame(fi)
        fi = A.frame_input(sc["settings"], colliders=sc["colliders"])
    return state_digests(sim)


def sort_case():
    rng = np.random.default_rng(11)
    n = 5000
    p = np.zeros(n, dtype=A.PARTICLE_DTYPE)
    p["pos"] = rng.uniform(0.0, 1.0, size=(n, 3)).astype(np.float32)
    p["age"] = np.where(rng.uniform(size=n) < 0.2, np.float32(-1.0), np.float32(1.0))
    return p


def main():
    out = {name: run_case(O.Oracle, case) for name, case in CASES.items()}
    sc = scenes.tiny(O.settings_default, n=32)
    o = O.Oracle(sc["settings"])
    o.upload_particles(sort_case())
    o.sort_particles()
    out["sort32"] = {"perm": digest(o.read("SORT_PERM")), "offsets": digest(o.read("SORT_OFFSETS"))}
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()

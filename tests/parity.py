"""Parity helpers: compare the GPU state with the CPU oracle buffer by buffer.

Pool buffers are compared over the slots of the active bricks (stale data in free slots is not state),
plus the null slot 0, which must stay all zeros in both."""
import numpy as np

from slosh_b200 import _abi as A

POOL_CELL = ("CELL_TYPE", "CELL_COUNT", "PRESSURE", "DIVERGENCE", "CELL_DIAG", "DENSITY_Q", "DENSITY_RHS")
POOL_FACE = ("VEL", "FACE_FLAGS", "FACE_WEIGHT")
TABLES = ("BRICK_TABLE", "SLOT_BRICK", "FREE_SLOTS", "ACTIVE_BRICKS", "NEW_SLOTS", "BRICK_TOUCH")


def active_slots(sim):
    ab = sim.read("ACTIVE_BRICKS")
    bt = sim.read("BRICK_TABLE")
    n = int(ab[0])
    return np.sort(bt[ab[1:1 + n]])


def slot_mask(slots, pool_cells, planes=1):
    m = np.zeros(pool_cells, dtype=bool)
    for s in slots:
        m[int(s) * 512:(int(s) + 1) * 512] = True
    return np.tile(m, planes)


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint8) if a.dtype == np.uint8 else a.view(np.uint32 if a.itemsize == 4 else np.uint8)


class Report:
    def __init__(self):
        self.items = []

    def add(self, name, a, b, mask=None):
        if mask is not None:
            a, b = a[mask], b[mask]
        same = np.array_equal(bits(a), bits(b))
        info = dict(name=name, n=int(a.size), bit_exact=bool(same))
        if a.dtype.kind == "f":
            d = np.abs(a.astype(np.float64) - b.astype(np.float64))
            info["max_abs"] = float(d.max()) if d.size else 0.0
            den = np.sqrt(np.sum(b.astype(np.float64) ** 2))
            info["rel_l2"] = float(np.sqrt(np.sum(d ** 2)) / den) if den > 0 else float(np.sqrt(np.sum(d ** 2)))
            info["mismatch"] = int(np.count_nonzero(bits(a) != bits(b)))
        else:
            info["mismatch"] = int(np.count_nonzero(a != b))
        self.items.append(info)
        return info

    def failures(self, float_rel_l2=None):
        bad = []
        for it in self.items:
            if it["bit_exact"]:
                continue
            if float_rel_l2 is not None and "rel_l2" in it and it["rel_l2"] <= float_rel_l2:
                continue
            bad.append(it)
        return bad

    def __str__(self):
        return "\n".join(str(i) for i in self.items)


def compare_state(gpu, orc, report=None, particles=True):
    r = report or Report()
    L = gpu.layout()
    pc = int(L.pool_cells)
    slots_g = active_slots(gpu)
    slots_o = active_slots(orc)
    r.add("active_slots", slots_g, slots_o)
    for t in TABLES:
        r.add(t, gpu.read(t), orc.read(t))
    if particles:
        pg, po = gpu.read("PARTICLES"), orc.read("PARTICLES")
        r.add("particles", pg.view(np.uint32).reshape(len(pg), 12), po.view(np.uint32).reshape(len(po), 12))
    cm = slot_mask(slots_o, pc)
    fm = slot_mask(slots_o, pc, planes=3)
    for name in POOL_CELL:
        a, b = gpu.read(name), orc.read(name)
        r.add(name, a, b, cm)
        r.add(name + "[null]", a[:512], np.zeros_like(a[:512]))
    for name in POOL_FACE:
        a, b = gpu.read(name), orc.read(name)
        r.add(name, a, b, fm)
        r.add(name + "[null]", a.reshape(3, pc)[:, :512], np.zeros((3, 512), dtype=a.dtype))
    r.add("STATS", gpu.read("STATS"), orc.read("STATS"))
    r.add("COUPLING", gpu.read("COUPLING"), orc.read("COUPLING"))
    r.add("PARTICLE_COUNT", gpu.read("PARTICLE_COUNT"), orc.read("PARTICLE_COUNT"))
    return r


def pair(slosh, oracle_mod, sc):
    """A GPU context and an oracle on the same scene settings and emission seed."""
    g = slosh.Simulation(sc["settings"])
    o = oracle_mod.Oracle(sc["settings"])
    g.set_emit_seed(sc["seed"])
    o.set_emit_seed(sc["seed"])
    return g, o


def run_frames(g, o, sc, frames, check_every_substep=True, tol=1e-5, substeps=None):
    """Steps GPU and oracle frame by frame (emits on the first frame; colliders and manipulators every
    frame) and compares the whole state after every substep and the results after every frame. With
    `substeps`, runs whole frames until at least that many substeps were compared (`frames` is then a cap)."""
    extra = dict(colliders=sc.get("colliders", []), manipulators=sc.get("manipulators", []))
    fi = A.frame_input(sc["settings"], emits=sc["emits"], **extra)
    reports = []
    done = 0
    for f in range(frames):
        if substeps is not None and done >= substeps:
            break
        ng, dtg = g.begin_frame(fi)
        no, dto = o.begin_frame(fi)
        assert (ng, dtg) == (no, dto), f"frame {f}: substeps/dt differ {ng, dtg} vs {no, dto}"
        done += ng
        for s in range(ng):
            g.substep(s)
            o.substep(s)
            if check_every_substep:
                r = compare_state(g, o)
                bad = r.failures(tol)
                assert not bad, f"frame {f} substep {s}:\n{r}"
                reports.append(r)
        g.end_frame()
        o.end_frame()
        rg, ro = g.results(), o.results()
        assert rg.fluid_cells == ro.fluid_cells
        assert rg.max_particle_speed == ro.max_particle_speed
        assert rg.last_solve_iterations == ro.last_solve_iterations
        assert rg.num_colliders == ro.num_colliders
        for k in range(rg.num_colliders):
            fg, fo = rg.colliders[k], ro.colliders[k]
            for name, _ in A.ColliderFeedback._fields_:
                assert list(getattr(fg, name)) == list(getattr(fo, name)) if hasattr(getattr(fg, name), "__len__") \
                    else getattr(fg, name) == getattr(fo, name), f"frame {f} collider {k} {name}"
        fi = A.frame_input(sc["settings"], **extra)
    if substeps is not None:
        assert done >= substeps, f"only {done} substeps in {frames} frames"
    return reports

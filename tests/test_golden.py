"""The oracle (CPU) and the GPU path (gpu) against the committed golden digests."""
import json
import os

import pytest

from slosh_b200 import _abi as A, scenes

HERE = os.path.dirname(os.path.abspath(__file__))


def _golden():
    with open(os.path.join(HERE, "golden", "golden.json")) as f:
        return json.load(f)


def _mod():
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(HERE, "golden", "make_golden.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


@pytest.mark.parametrize("case", ["tiny16_mgpcg", "tiny16_rbgs", "tiny24_collider"])
def test_oracle_matches_golden(oracle_mod, case):
    m = _mod()
    assert m.run_case(oracle_mod.Oracle, m.CASES[case]) == _golden()[case]


def test_oracle_sort_matches_golden(oracle_mod):
    m = _mod()
    o = oracle_mod.Oracle(scenes.tiny(oracle_mod.settings_default, n=32)["settings"])
    o.upload_particles(m.sort_case())
    o.sort_particles()
    g = _golden()["sort32"]
    assert m.digest(o.read("SORT_PERM")) == g["perm"]
    assert m.digest(o.read("SORT_OFFSETS")) == g["offsets"]


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["tiny16_mgpcg", "tiny16_rbgs", "tiny24_collider"])
def test_gpu_matches_golden(slosh, oracle_mod, case):
    m = _mod()
    assert m.run_case(lambda s: slosh.Simulation(s, device=0), m.CASES[case]) == _golden()[case]


@pytest.mark.gpu
def test_gpu_sort_matches_golden(slosh, oracle_mod):
    m = _mod()
    g = slosh.Simulation(scenes.tiny(slosh.settings_default, n=32)["settings"], device=0)
    g.upload_particles(m.sort_case())
    g.sort_particles()
    gold = _golden()["sort32"]
    assert m.digest(g.read("SORT_PERM")) == gold["perm"]
    assert m.digest(g.read("SORT_OFFSETS")) == gold["offsets"]

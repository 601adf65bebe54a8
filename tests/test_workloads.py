"""The committed workload manifests are exactly what their seeded generator
draws (so the GPU engine, the CPU oracle and the bench read the same
instances), and every drawn parameter lies in its stated support."""
import importlib.util
import json
import math
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
WL = os.path.join(ROOT, "hosono-2dmhd_b200", "workloads")


def _gen():
    spec = importlib.util.spec_from_file_location("make_manifests", os.path.join(WL, "make_manifests.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _load(name):
    with open(os.path.join(WL, name)) as f:
        return json.load(f)


def test_blast64_manifest_is_reproducible():
    gen = _gen()
    m = _load("blast64_seed0.json")
    assert m["seed"] == 0
    assert m["instances"] == json.loads(json.dumps(gen.blast64(seed=0)))
    for e in m["instances"]:
        assert e["n"] in (128, 192, 256, 384, 512)
        assert 10.0 <= e["p_ratio"] <= 1000.0
        assert 0.0 <= e["theta"] <= math.pi / 2
        assert (e["radius"], e["ell"], e["tmax"], e["cfl"]) == (2, 6.0, 0.02, 0.8)


def test_served2000_manifest_is_reproducible():
    gen = _gen()
    m = _load("served2000_seed1.json")
    assert m["seed"] == 1 and len(m["requests"]) == 2000
    assert m["requests"] == json.loads(json.dumps(gen.served(seed=1)))
    seen = set()
    for r in m["requests"]:
        seen.add(r["problem"])
        assert 64 <= r["n"] <= 1024 and r["radius"] in (1, 2)
        assert 0.1 <= r["tmax_factor"] <= 1.0
        assert r["tmax"] == r["tmax_factor"] * gen.DEFAULT_TEND[r["problem"]]
        assert r["gap"] >= 0.0
        if r["problem"] == "explosion2d":
            assert 10.0 <= r["p_ratio"] <= 1000.0 and 0.0 <= r["theta"] <= math.pi / 2
    assert seen == {"OrszagTang2d", "sedov2d", "explosion2d"}

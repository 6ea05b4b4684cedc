"""bench.py's reference arm (the CPU port of the path: C sampler, PyTorch-CPU
hash grid, MLP, autograd and Adam) on a small sample, run as the driver runs
it: the keys of its JSON line, the same `config` as the GPU arm's, and that
it loads nothing of the product (no nect_b200 module, no libnectb.so)."""
import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]

RUNNER = """
import runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--steps", "1", "--warmup", "1", "--cpu-rays", "64",
            "--workload", "c1_static_parallel"]
runpy.run_path("bench.py", run_name="__main__")
product = sorted(m for m in sys.modules if m == "nect_b200" or m.startswith("nect_b200."))
maps = open("/proc/self/maps").read()
print("PRODUCT_MODULES", product, "LIBNECTB_MAPPED", "libnectb" in maps)
"""


def test_reference_arm_prints_one_contract_line():
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    out = subprocess.run([sys.executable, "-c", RUNNER], cwd=ROOT, env=env, capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "rays/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["e2e"]["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and "64 of the" in cb["sample"]
    for key in ("metric", "n_gpus", "steps", "warmup", "ms_per_step", "scaling", "dtype", "data", "config"):
        assert key in d
    sys.path.insert(0, str(ROOT))
    import bench

    assert d["config"] == bench.bench_config("c1_static_parallel", 65536)   # the GPU arm's config
    tail = [l for l in out.stdout.splitlines() if l.startswith("PRODUCT_MODULES")][0]
    assert tail == "PRODUCT_MODULES [] LIBNECTB_MAPPED False", tail


def test_oracle_workloads_match_the_product_geometry():
    """The CPU arm's restated workloads build the same geometry structs,
    max_distance_traveled and per-level scale as the product's classes."""
    from nect_b200.config import HashEncoderConfig
    from nect_b200.sampling import Geometry
    from oracle import workloads as owl

    sys.path.insert(0, str(ROOT))
    import bench

    for name, w in owl.WORKLOADS.items():
        spec = bench.workload_spec(name, "mixed")
        geo = Geometry(**spec["geo"])
        assert abs(geo.max_distance_traveled - w.max_distance_traveled) <= 1e-9 * w.max_distance_traveled, name
        mine, theirs = geo.get_c_geometry().c_struct, w.c_struct()
        for field, _ in theirs._fields_:
            a, b = getattr(mine, field), getattr(theirs, field)
            a = list(a) if hasattr(a, "__len__") else a
            b = list(b) if hasattr(b, "__len__") else b
            assert a == b, (name, field, a, b)
        enc: HashEncoderConfig = spec["model"].encoder
        assert abs(enc.per_level_scale - w.per_level_scale) < 1e-12, name
        assert (enc.log2_hashmap_size, enc.n_features_per_level, spec["S"], spec["rays"]) == (
            w.log2_T, w.n_features, w.S, w.rays), name
        assert spec["model"].net.n_hidden_layers == w.hidden_layers

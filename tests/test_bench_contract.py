"""The benchmark's host side, without a GPU: the command line's defaults, the
compact JSON line, and the reference arm (the oracle on the host cores) on a
small seeded case, whose line carries the keys and the workload the GPU arm's
line carries for the same case."""
import importlib.util
import os
import sys
import types

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_cli", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_defaults(monkeypatch):
    """With no flags: one GPU, a step count that finishes within minutes, at
    least three warm-up steps, the long-form record beside the line."""
    b = _bench()
    seen = {}
    monkeypatch.setattr(b, "run_reference", lambda args, rank, world: seen.update(vars(args)))
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference"])
    b.main()
    assert seen["gpus"] == 1
    assert 1 <= seen["steps"] <= 50
    assert seen["warmup"] >= 3
    assert seen["details"] == "bench_details.json"


def test_compact_line_rounds_all_but_the_headline():
    b = _bench()
    line = b.compact({"value": 1.23456789, "ms_per_step": 2.3456789, "n": 3,
                      "fp64": {"value": 7.654321e7, "x": [0.123456789]}})
    assert line["value"] == 1.23456789 and line["ms_per_step"] == 2.3456789
    assert line["n"] == 3
    assert line["fp64"] == {"value": 7.654e7, "x": [0.1235]}


def test_reference_arm_on_a_small_case(monkeypatch):
    b = _bench()
    pkg = b.load_pkg()
    from dcm_b200 import cases
    small = cases.warm_bubble(ip=12, jp=10, kp=8)
    monkeypatch.setattr(b, "make_case", lambda p, name: small)
    args = types.SimpleNamespace(case="warm_bubble", steps=2, warmup=1, ref_budget=120.0,
                                 cpu_budget=60.0)
    assert b.run_reference(args, 1, 2) is None  # ranks other than 0 do no work
    try:
        line = b.compact(b.run_reference(args, 0, 1))
    finally:
        # the timed baseline sums the oracle's dot products per thread (its
        # fast mode); the other tests compare the oracle in its fixed order
        import oracle
        oracle.set_threads(os.cpu_count() or 1, False)
    assert line["impl"] == "reference"
    assert line["unit"] == "grid-pt-steps/s" and line["value"] > 0
    assert line["steps"] == 2 and line["warmup"] == 1 and line["ms_per_step"] > 0
    assert line["higher_is_better"] is True
    assert line["config"] == b.bench_config(small, args)
    assert line["config"]["workload"].endswith("steps 1..2 from the seeded initial state")
    assert line["metric"] == b.metric_of(small)
    cpu = line["cpu_baseline"]
    assert cpu["kind"] == "port" and cpu["steps_done"] == 2 and cpu["cores"] >= 1
    # the reference arm's end-to-end figure is its own value (no device copies)
    assert line["e2e"] == {"value": float("%.4g" % line["value"]), "unit": "grid-pt-steps/s",
                           "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert pkg is sys.modules["dcm_b200"]

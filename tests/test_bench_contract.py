"""The reference arm's JSON line keeps the bench contract (CPU, no GPU).

The reference arm and the native arm must describe the same workload with the
same ``config`` object, so the two lines can be compared. The reference's own
solve is replaced here by fakes of its sampler and validation (the real ones
run the reference library for seconds); the line is built by the real
``run_reference``.
"""
import argparse
import json

import bench


class _FakeRefLib:
    @staticmethod
    def available():
        return True


def _fake_line(monkeypatch, gpus=1, steps=2, warmup=3):
    import oracle

    monkeypatch.setattr(oracle, "RefLib", _FakeRefLib)
    monkeypatch.setattr(bench, "N_POINTS", 4096)
    monkeypatch.setattr(bench, "reference_tree", lambda pts, threads: object())
    calls = []

    def sample(rt, q, seconds):
        calls.append(seconds)
        return {"value": 1.0e8 + len(calls), "est_solve_s": 900.0, "sampled_s": 5.0, "stride": 93}

    monkeypatch.setattr(bench, "reference_sample", sample)
    monkeypatch.setattr(bench, "reference_validation",
                        lambda threads: {"points": 65536, "full_solve_s": 8.0, "est_solve_s": 8.1,
                                         "validated_ratio": 8.1 / 8.0})
    monkeypatch.setattr(bench, "reference_config1", lambda threads: {"full_solve_ms": 1000.0})
    args = argparse.Namespace(gpus=gpus, steps=steps, warmup=warmup)
    return bench.run_reference(args, gpus, 0), calls


def test_reference_line_carries_the_shared_config(monkeypatch):
    line, calls = _fake_line(monkeypatch)
    assert len(calls) == 3 + 2  # warm-up and timed samples
    assert line["impl"] == "reference"
    assert line["config"] == bench.bench_config(2)
    assert line["metric"] == bench.METRIC and line["unit"] == "interactions/s" and line["higher_is_better"]
    assert line["steps"] == 2 and line["warmup"] == 3
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["e2e"]["value"] == line["value"] == line["cpu_baseline"]["value"]
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] >= 1
    assert abs(line["cpu_baseline"]["validated_ratio"] - 8.1 / 8.0) < 1e-12
    assert line["ms_per_step"] == 5000.0  # the wall time of one bounded sample
    json.dumps(line)  # one JSON line


def test_other_ranks_print_nothing(monkeypatch):
    args = argparse.Namespace(gpus=2, steps=1, warmup=3)
    assert bench.run_reference(args, 2, 1) is None


def test_config_names_the_workload_not_the_form():
    cfg = bench.bench_config(2)
    assert set(cfg) == {"workload", "tolerance_rel_l2", "value_definition"}
    assert "N=1048576" in cfg["workload"] and "n=8" in cfg["workload"] and "leaf 2000" in cfg["workload"]
    assert "FP32" not in cfg["workload"] and "FP64" not in cfg["workload"]
    assert cfg["tolerance_rel_l2"] == 1e-6

"""bench.py's reference arm on the host (it runs the FP64 oracle on the host cores, no GPU):
the one JSON line of the bench contract with its cpu_baseline and e2e keys; under a
multi-rank launch only rank 0 prints, the other ranks exit 0 without work."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench(*args, env=None):
    e = dict(os.environ)
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        e.pop(k, None)
    e.update(env or {})
    return subprocess.run([sys.executable, "bench.py", *args], cwd=ROOT, env=e, capture_output=True, text=True,
                          timeout=900)


def test_reference_arm_prints_the_contract_line():
    r = _bench("--impl", "reference", "--steps", "1", "--warmup", "0")
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    line = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference" and line["metric"] == "RK4 cell-updates/s"
    assert line["value"] > 0 and line["higher_is_better"] is True and line["steps"] == 1
    assert line["config"]["workload"].startswith("c4-1024x512x1024")
    cb = line["cpu_baseline"]
    # the reference program itself when its translated build is present, else the oracle port
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["value"] == line["value"] and cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_quietly():
    r = _bench("--impl", "reference", "--steps", "1", "--warmup", "0",
               env={"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert r.returncode == 0 and r.stdout.strip() == ""


def test_roofline_peak_is_the_measured_one_when_present(tmp_path, monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    assert bench.peaks() == (6650.0, "fallback")
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps({"hbm_gbs": 6531.5, "bf16_tflops": 1590.0}))
    assert bench.peaks() == (6531.5, "measured")


def test_clock_samples_give_median_max_and_active_reasons(tmp_path):
    sys.path.insert(0, ROOT)
    import bench

    class Proc:
        def terminate(self):
            pass

        def wait(self, timeout=None):
            return 0

    c = bench.Clocks()
    c.path = str(tmp_path / "clocks.csv")
    c.f = open(c.path, "w")
    c.f.write("0, 1770, 1965, 998.1, 0x4, Not Active, Not Active, Not Active, Active\n"
              "0, 1860, 1965, 990.0, 0x0, Not Active, Not Active, Not Active, Not Active\n"
              "garbage line\n"
              "0, 1800, 1965, 995.0, 0x4, Not Active, Not Active, Not Active, Active\n")
    c.p = Proc()
    assert c.stop() == {"sm_mhz": 1800.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 3}

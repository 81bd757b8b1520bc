"""Host-side pieces of bench.py that need no GPU: the roofline denominator
read from the per-pod measured-peaks file, with the fallback and its reason
when the file is absent or does not hold a usable `hbm_gbs`."""
import importlib.util
import json
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_load_peaks_measured_and_fallbacks(tmp_path):
    B = _bench()
    absent = B.load_peaks(str(tmp_path / "none.json"))
    assert absent == B.FALLBACK_PEAKS and absent["source"] == "fallback"

    good = tmp_path / "good.json"
    good.write_text(json.dumps({"hbm_gbs": "6557.2", "bf16_tflops": 1590.0}))
    d = B.load_peaks(str(good))
    assert d["hbm_gbs"] == 6557.2 and d["source"] == "measured" and d["bf16_tflops"] == 1590.0

    for name, text, why in (("nokey.json", json.dumps({"bf16_tflops": 1.0}), "KeyError"),
                            ("bad.json", "{not json", "JSONDecodeError"),
                            ("nan.json", json.dumps({"hbm_gbs": "fast"}), "ValueError"),
                            ("null.json", json.dumps({"hbm_gbs": None}), "TypeError")):
        f = tmp_path / name
        f.write_text(text)
        d = B.load_peaks(str(f))
        assert d["hbm_gbs"] == B.FALLBACK_PEAKS["hbm_gbs"], name
        assert d["source"].startswith("fallback") and why in d["source"], d["source"]

    zero = tmp_path / "zero.json"
    zero.write_text(json.dumps({"hbm_gbs": 0}))
    d = B.load_peaks(str(zero))
    assert d["hbm_gbs"] == B.FALLBACK_PEAKS["hbm_gbs"] and "hbm_gbs = 0" in d["source"]


def test_supplementary_section_failure_keeps_the_line():
    B = _bench()
    assert B.supplementary("ok", lambda: {"x": 1}) == {"x": 1}

    def boom():
        raise RuntimeError("out of memory at 4096^2")

    d = B.supplementary("large", boom)
    assert d["section"] == "large" and d["error"].startswith("RuntimeError: out of memory")


def test_line_leads_with_the_contract_and_target_keys():
    """The headline target numbers come right after the contract keys, so a
    reader (or a truncated log tail) of the JSON line sees them first."""
    B = _bench()
    line = {"spmv": {}, "large": {}, "roofline": {}, "metric": "m", "value": 1.0, "plain_fp32_ms": 60.0,
            "speedup_mixed_vs_plain": 1.8, "unit": "u", "batch": {}, "time_to_rtol_mg_ms": 11.0}
    keys = list(B.ordered_line(line))
    assert keys[:3] == ["metric", "value", "unit"]
    assert keys.index("speedup_mixed_vs_plain") < keys.index("roofline") < keys.index("spmv")
    assert keys.index("plain_fp32_ms") < keys.index("large") and set(keys) == set(line)


def test_reference_arm_describes_what_it_runs():
    class A:
        W, H = 1920, 1080

    c = _bench().reference_config_dict(A, 120, 16)
    assert "gaussSeidel_host" in c["workload"] and c["sweeps"] == 120 and c["threads"] == 16
    assert c["precision"].startswith("fp32") and "CG" not in c["workload"].replace("no CPU CG", "")


def test_reference_convergence_reports_the_residual_reached():
    """The reference CPU path's time-to-residual figure: the true residual
    after the sampled sweeps (on a small image here)."""
    from gpumatting_b200.synth import make_problem

    d = _bench().reference_convergence(make_problem(48, 32, 0), 5)
    assert d["sweeps"] == 5 and d["cores"] == 1 and d["seconds"] >= 0.0
    assert 0.0 < d["rel_residual_reached"] < d["rel_residual_start"]
    assert d["reached"] == (d["rel_residual_reached"] <= 1e-6)

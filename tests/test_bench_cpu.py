"""Host-side pieces of bench.py that need no GPU: the compulsory byte model,
the DRAM traffic taken from the committed ncu capture, the choice of the HBM
peak, the config object and the summary that closes the JSON line."""
import json

import bench


def test_byte_model_is_the_compulsory_one():
    # per even site: two hops of 1152 B (4 own + 4 neighbour links, input,
    # output) and f_e for the second hop's epilogue
    assert bench.BYTES_STEP == 2 * 1152 + 192


def test_traffic_comes_from_the_committed_capture():
    vh = 32 * 32 * 32 * 64 // 2
    traffic, src = bench.traffic_per_step(vh)
    assert src.startswith(bench.PROFILE_32)
    # at the compulsory level, within a few per cent (part of the output
    # stays in L2 when a launch ends)
    assert 0.95 * bench.BYTES_STEP * vh < traffic < 1.05 * bench.BYTES_STEP * vh


def test_peak_is_measured_when_the_file_exists(tmp_path, monkeypatch):
    monkeypatch.setattr(bench, "ROOT", tmp_path)
    assert bench.measured_peak() == (6650.0, "fallback")
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps({"hbm_gbs": 6547.5}))
    assert bench.measured_peak() == (6547.5, "measured")


def test_config_names_the_workload_and_no_model():
    c = bench.config_for(1)
    assert c["workload"] == bench.WORKLOAD and c["lattice"] == [32, 32, 32, 64]
    assert "model" not in c and c["parallelism"] == "replicas x1"
    assert bench.config_for(8)["parallelism"] == "replicas x8"


def _line(with_sections):
    line = {"ms_per_step": 0.45, "value": 5800.0,
            "roofline": {"frac": 0.87, "peak_kind": "fallback", "dram_frac": 0.86},
            "variants": {"wilson_fp64_24x24x24x48": {"ms": 0.15, "frac": 0.82},
                         "clover_fp64_24x24x24x48": {"ms": 0.2, "frac": 0.9}},
            "solve": {}, "batched": {}, "learned": {}, "mixed48": {}, "callers": {}}
    if with_sections:
        line["solve"] = {"double": {"ms": 49.0}, "single": {"ms": 33.0}, "half": {"ms": 25.0}}
        line["learned"] = {"gcr_network": {"ms": 170.0, "ms_min": 169.0, "iterations": 74},
                           "cg_half": {"ms": 185.0, "ms_min": 180.0, "iterations": 343},
                           "network_apply_ms": 1.3, "gcr_network_vs_best_mixed_cg": 1.09}
    return line


def test_summary_with_and_without_the_solver_sections():
    s0 = bench.summarise(_line(False), 6650.0)
    assert s0["headline_32x32x32x64_fp64"]["peak_kind"] == "fallback"
    assert s0["clover_solve_24x24x24x48_ms"] == {"double": None, "single": None, "half": None}
    assert "learned_32x32x32x64_ms" not in s0
    s1 = bench.summarise(_line(True), 6650.0)
    assert s1["clover_solve_24x24x24x48_ms"]["half"] == 25.0
    assert s1["gcr_network_vs_best_mixed_cg"] == 1.09
    assert s1["learned_iterations"] == {"gcr_network": 74, "cg_half": 343}
    # the summary is the line's last key: it has to stay short
    assert len(json.dumps(s1)) < 2000

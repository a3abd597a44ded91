"""Host-side parts of bench.py on the CPU: the term count behind every terms/s
figure, the clock-sample summary, and the reference arm's JSON line."""

import json
import sys

import numpy as np

import bench
from matvis_b200 import workloads as wl
from oracle import oracle as orc


def test_terms_per_job_counts_the_oracle_horizon():
    """Npairs x sum_t n_t x Nf, n_t the sources the oracle keeps above the horizon."""
    cfg = wl.config1()
    terms, counts = bench.terms_per_job(cfg)
    eci = orc.point_source_crd_eq(cfg["ra"], cfg["dec"])
    ref = [int((orc.rotate_fixed_order(orc.eci_to_enu_matrix(t, cfg["latitude"]), eci)[2] > 0).sum())
           for t in cfg["lsts"]]
    assert counts.tolist() == ref and 0 < min(ref)
    nant = len(cfg["antpos"])
    assert terms == nant * nant * sum(ref) * len(cfg["freqs"])
    pairs = np.array([(0, 1), (2, 3), (4, 4)])
    assert bench.terms_per_job({**cfg, "antpairs": pairs})[0] == 3 * sum(ref) * len(cfg["freqs"])


def test_clock_summary(tmp_path):
    """Median SM clock, the maximum, and only the throttle reasons that were active."""
    s = bench.ClockSampler(0)
    s.path = str(tmp_path / "clocks.csv")
    rows = [
        "0, 1590, 1965, 900.1, 0x4, Not Active, Not Active, Not Active, Active",
        "0, 1600, 1965, 910.0, 0x4, Not Active, Not Active, Not Active, Active",
        "0, 1580, 1965, 905.0, 0x0, Not Active, Not Active, Not Active, Not Active",
    ]
    (tmp_path / "clocks.csv").write_text("\n".join(rows) + "\n")
    assert s.summary() == {"sm_mhz": 1590.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 3}
    assert not (tmp_path / "clocks.csv").exists()  # the sample file is removed once read

    s.path = str(tmp_path / "hot.csv")
    (tmp_path / "hot.csv").write_text("0, 1200, 1965, 700.0, 0x48, Active, Not Active, Active, Not Active\n")
    assert s.summary()["reasons"] == ["hw_slowdown", "sw_thermal_slowdown"]
    s.path = str(tmp_path / "empty.csv")
    (tmp_path / "empty.csv").write_text("")
    assert s.summary() is None


def test_reference_arm_line(monkeypatch, capsys):
    """--impl reference prints one JSON line on the workload's metric, with its CPU
    baseline and an e2e entry that moves no bytes to or from a device."""
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0",
                                      "--nside", "8", "--nfreq", "1", "--ntimes", "1"])
    args = bench.parse()
    bench.run_reference(args, 0, 1)
    lines = [ln for ln in capsys.readouterr().out.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["metric"] == bench.METRIC and line["unit"] == bench.UNIT
    assert line["value"] > 0 and line["higher_is_better"] is True and line["steps"] == 1
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": bench.UNIT, "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert "768 sources" in line["sample"] and line["cpu_baseline"]["sample"] == line["sample"]


def test_reference_arm_loads_no_repo_library(monkeypatch, capsys):
    """The reference arm builds its workload and times the oracle without mapping
    this repository's shared library (checked in a fresh interpreter)."""
    import subprocess

    code = ("import sys, bench\n"
            "sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '0', '--nside', '4', "
            "'--nfreq', '1', '--ntimes', '1']\n"
            "bench.main()\n"
            "maps = open('/proc/self/maps').read()\n"
            "assert 'libmatvis_b200' not in maps, 'library mapped'\n"
            "assert 'matvis_b200._lib' not in sys.modules\n")
    root = str(__import__("pathlib").Path(bench.__file__).resolve().parent)
    res = subprocess.run([sys.executable, "-c", code], cwd=root, capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr[-2000:]
    assert json.loads(res.stdout.strip().splitlines()[-1])["impl"] == "reference"


def test_both_arms_share_the_config_object(monkeypatch):
    """The config object names the workload only, so the two arms print the same one."""
    monkeypatch.setattr(sys, "argv", ["bench.py", "--nside", "8", "--nfreq", "2", "--ntimes", "2"])
    args = bench.parse()
    cfg, desc = bench.load_config(args, host_only=True)
    terms, counts = bench.terms_per_job(cfg)
    c1 = bench.workload_config(args, cfg, desc, terms, counts)
    cfg2, desc2 = bench.load_config(args)
    c2 = bench.workload_config(args, cfg2, desc2, *bench.terms_per_job(cfg2))
    assert c1 == c2 and set(c1) == {"workload", "matprod", "gemm_mode", "terms_per_job", "above_horizon_per_time",
                                    "l2"}
    assert bench.accuracy_slices(cfg) == [(0, 0), (1, 1)]


def test_reference_arm_other_ranks_do_nothing(monkeypatch, capsys):
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference"])
    bench.run_reference(bench.parse(), 1, 2)
    assert capsys.readouterr().out == ""

"""CPU checks of bench.py: the reference arm imports nothing of the engine,
and its plain workload table agrees with the package's WORKLOADS."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    sys.path.insert(0, ROOT)
    import importlib
    return importlib.import_module("bench")


def test_reference_workloads_match_the_package(bh):
    bench = _bench()
    for name, wp in bench.REF_WORKLOADS.items():
        wl = bh.WORKLOADS[name]
        assert wp["n"] == wl["n"] and wp["scenario"] == wl["scenario"], name
        cfg = wl["config"]
        op = wp["oracle"]
        got = (op["G"], op["dt"], op["theta"], op["softening"], op["plummer_eps"],
               op["morton_bits"], op["morton_domain"], op["integrator"], op["walk"],
               op["multipole"], op["far_alpha"])
        want = (cfg.gravConstant, cfg.deltaTime, cfg.bhTheta, cfg.softening, cfg.plummerEps,
                cfg.mortonBits, cfg.mortonDomain, cfg.integrator, cfg.walk, cfg.multipole,
                cfg.farAlpha)
        assert got == want, name


def test_reference_arm_runs_without_the_engine(orc):
    # The reference arm on the small parity workload, in a fresh process:
    # it prints its line and never maps the engine's library.
    code = (
        "import sys, json, runpy\n"
        f"sys.argv = ['bench.py', '--impl', 'reference', '--workload', 'uniform-disk-16k',"
        " '--steps', '3', '--warmup', '3']\n"
        "try:\n"
        "    runpy.run_path('bench.py', run_name='__main__')\n"
        "except SystemExit:\n"
        "    pass\n"
        "maps = open('/proc/self/maps').read()\n"
        "print('ENGINE_MAPPED' if 'libbh_b200' in maps else 'ENGINE_NOT_MAPPED')\n"
        "print('PKG_IMPORTED' if 'webgpu-fluid-sim_b200' in sys.modules else 'PKG_NOT_IMPORTED')\n")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "ENGINE_NOT_MAPPED" in r.stdout and "PKG_NOT_IMPORTED" in r.stdout, r.stdout[-2000:]
    import json
    line = json.loads([ln for ln in r.stdout.splitlines() if ln.startswith("{")][0])
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] in ("reference", "port")
    assert line["e2e"]["h2d_bytes_per_step"] == 0
    # W untimed, then exactly K timed steps; the own arm's config
    assert line["steps"] == 3 and line["warmup"] == 3
    assert "3 untimed then 3 timed" in line["cpu_baseline"]["sample"]
    assert line["config"] == _own_config(_bench(), "uniform-disk-16k", 1, [])
    assert "uniform-disk-kepler" in line["data"]


def _own_config(bench, name, world, flags):
    """The config the own arm prints for a workload (its values from the
    package's WORKLOADS, as run_own takes them)."""
    argv, sys.argv = sys.argv, ["bench.py", "--workload", name, *flags]
    try:
        args = bench.parse()
    finally:
        sys.argv = argv
    import importlib
    wl = importlib.import_module("webgpu-fluid-sim_b200").WORKLOADS[name]
    cfg = wl["config"]
    return bench.run_config(args, wl["n"], cfg.bhTheta, cfg.plummerEps, cfg.deltaTime,
                            cfg.integrator, world)


@pytest.mark.parametrize("world,flags", [(1, []), (2, []), (2, ["--replicas"]), (1, ["--shard"])])
def test_both_arms_print_one_config(bh, world, flags):
    bench = _bench()
    for name, wp in bench.REF_WORKLOADS.items():
        own = _own_config(bench, name, world, flags)
        argv, sys.argv = sys.argv, ["bench.py", "--impl", "reference", "--workload", name, *flags]
        try:
            args = bench.parse()
        finally:
            sys.argv = argv
        op = wp["oracle"]
        ref = bench.run_config(args, wp["n"], op["theta"], op["plummer_eps"], op["dt"],
                               op["integrator"], world)
        assert own == ref, name
        assert own["workload"] == name and own["bodies"] == wp["n"]


def test_walk_roofline_flop_convention():
    bench = _bench()

    class C:
        walk, multipole = "group", 2

    r = bench.walk_roofline(C, 1.0, 1000, 100, 10, 1965.0)
    assert r["flops_per_step"] == 35 * 1000 + 16 * 100
    assert r["achieved"] == pytest.approx(r["flops_per_step"] / 1e-3 / 1e12)
    s = bench.stream_rooflines({"sort": 1.0}, 1_000_000, 8, 6000.0)
    assert s["sort"]["bytes_per_body"] == 20 + 7 * 24


def test_reference_arm_port_fallback(orc):
    # Without oracle/_ref the arm times the oracle port, with the same
    # warm-up / timed structure.
    bench = _bench()
    cb = bench.port_arm(bench.REF_WORKLOADS["uniform-disk-16k"], 2, 1)
    assert cb["kind"] == "port" and cb["value"] > 0 and cb["cores"] >= 1
    assert "1 untimed then 2 timed whole steps of the 16384-body workload" in cb["sample"]


def test_reference_arm_samples_the_walk_when_a_step_does_not_fit(orc, monkeypatch):
    # A whole step (8 s of walk) longer than its share of the run (30 s over
    # 6 steps): the walk runs on every 2nd sorted slot and its time is scaled
    # by 2; W untimed and K timed steps as asked.
    bench = _bench()
    calls = []

    def fake(mass, pos, vel, steps=1, walk_stride=1, **kw):
        calls.append((steps, walk_stride))
        return {"morton": 0.01 * steps, "sort": 0.01 * steps, "build_fill": 0.01 * steps,
                "vel_step": 8.0 * steps / walk_stride, "pos_step": 0.01 * steps}

    monkeypatch.setattr(orc, "ref_run_timed", fake)
    monkeypatch.setattr(orc, "ref_available", lambda: True)
    monkeypatch.setattr(orc, "ref_threads", lambda: 4)
    wp = bench.REF_WORKLOADS["uniform-disk-16k"]
    cb = bench.reference_arm(wp, 5, 1, seconds_total=30.0)
    assert calls == [(1, 1), (1, 2), (5, 2)]
    assert cb["walk_stride"] == 2 and cb["kind"] == "reference"
    assert cb["value"] == pytest.approx(16384 * 5 / (0.04 * 5 + 2 * 8.0 * 5 / 2))
    assert "every 2nd sorted slot and scaled by 2" in cb["sample"]
    assert [bench._ordinal(k) for k in (1, 2, 3, 4, 11, 12, 13, 21, 67, 112)] == \
        ["1st", "2nd", "3rd", "4th", "11th", "12th", "13th", "21st", "67th", "112th"]

"""bench.py's output contract, checked on the CPU arm (`--impl reference`).

The reference arm runs the oracle's FP64 restatement on the host, so it needs
no GPU; on the 2-atom cell one step takes seconds.  Its JSON line must carry
the keys the driver reads, and `config` must be the one the GPU arm prints
for the same workload and arguments (both arms build it with
`workload_config`).
"""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_reference(*extra):
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", "si2",
           "--steps", "1", "--warmup", "0", *extra]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout
    return json.loads(lines[0])


def test_reference_arm_line_has_the_contract_keys():
    d = run_reference()
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference"
    assert d["higher_is_better"] is False and d["unit"] == "ms/k-point"
    assert d["value"] > 0 and d["steps"] == 1 and d["warmup"] == 0
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    assert d["config"]["workload"].startswith("si2: 2 atoms")


def test_reference_config_is_the_gpu_arms_config():
    """The GPU arm prints workload_config(w, [ctx.npw(k) ...], args, nk, world); the
    library's basis for si2 at Gamma has the reference's 725 plane waves (pinned
    by the golden basis records), so the reference arm's line must carry exactly
    that object."""
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "deepaw-half_b200"))
    import bench
    from halfb200 import synth
    w = synth.workload("si2")
    saved = sys.argv
    try:
        sys.argv = ["bench.py", "--workload", "si2", "--steps", "1", "--warmup", "0"]
        args = bench.parse()
    finally:
        sys.argv = saved
    expected = bench.workload_config(w, [725], args, len(w.kpoints), 1)
    assert run_reference()["config"] == expected

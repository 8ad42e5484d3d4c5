"""The benchmark's reference arm on the CPU (`bench.py --impl reference`).

On the n = 1,280 system (config 1) the arm runs the reference's own code
(the compiled headers in oracle/_ref: QDLDL_etree, QDLDL_factor<float>,
GmresLDLIR::Solve) on every host core for a bounded time and prints one
JSON line of the benchmark contract, measured in full (no extrapolation).
The arm must map no code of this repository's CUDA library."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_RUN = (
    "import runpy, sys\n"
    "sys.argv = ['bench.py', '--impl', 'reference', '--config', 'small2d',"
    " '--steps', '1', '--warmup', '1']\n"
    "runpy.run_path('bench.py', run_name='__main__')\n"
    "print('LIBRARY_MAPPED', 'libmpir_b200.so' in open('/proc/self/maps').read())\n"
)


def test_reference_arm_small2d_line():
    out = subprocess.run([sys.executable, "-c", _RUN], cwd=ROOT, capture_output=True,
                         text=True, timeout=900)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert lines, out.stdout[-2000:]
    d = json.loads(lines[-1])
    assert d["impl"] == "reference"
    assert d["measured"] is True
    assert d["value"] > 0 and d["unit"] == "solves/s" and d["higher_is_better"] is True
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"]["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    # the reference's solution meets the backward-error target
    assert d["cpu_baseline"]["detail"]["backward_error"] <= 1e-14
    assert "LIBRARY_MAPPED False" in out.stdout

"""Host-side helpers of bench.py: the report parser used to time GSPARC-style
programs, and the matched-product count it divides by."""
import os
import stat
import sys

import oracle_bind as ob
from gsparc_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_run_report_parses_the_elapsed_section(tmp_path):
    prog = tmp_path / "fake_gsparc"
    prog.write_text(
        "#!/bin/sh\n"
        "cat >&2 <<'EOF'\n"
        "--------Break Down--------\n"
        "SLITOM time: 9.0\n"
        "--------Elapsed Time--------\n"
        "Result NNZ: 12345\n"
        "SLITOM time: 0.500000\n"
        "Partition time: 0.000001\n"
        "SpTC(IdxMatch + Contraction + Data Copy) time: 1.250000\n"
        "Total time: 1.750001\n"
        "EOF\n")
    prog.chmod(prog.stat().st_mode | stat.S_IEXEC)
    r = bench.run_report(str(prog), "x.tns", "y.tns", [2, 3], [0, 1], -1, iters=3)
    assert r["rc"] == 0 and "error" not in r
    assert r["Result NNZ"] == 12345
    assert r["SLITOM time"] == 0.5  # the last section wins
    assert r["SpTC(IdxMatch + Contraction + Data Copy) time"] == 1.25
    assert r["Total time"] == 1.750001


def test_run_report_records_a_failing_program(tmp_path):
    prog = tmp_path / "failing"
    prog.write_text("#!/bin/sh\necho 'CUDA error' >&2\nexit 3\n")
    prog.chmod(prog.stat().st_mode | stat.S_IEXEC)
    r = bench.run_report(str(prog), "x.tns", "y.tns", [2], [2], 0)
    assert r["rc"] == 3 and "CUDA error" in r["error"]


def test_host_products_equals_the_oracle_count():
    for X, Y, cx, cy in (synth.plain_small(scale=0.05), synth.esc_large(scale=0.003),
                         synth.dense_acc(scale=0.0005)):
        assert bench.host_products(X, Y, cx, cy) == ob.sptc(X, Y, cx, cy).ir_nnz


def test_algorithmic_bytes_of_a_contraction():
    # X, Y of order 3 and 4 with 10 and 20 nonzeros, 100 products, 30 outputs
    want = (10 * (8 * 3 + 4) + 24 * 10) + (20 * (8 * 4 + 4) + 24 * 20) + 16 * 10 + 8 * 20 + 24 * 100 + 12 * 30
    assert bench.alg_bytes_contraction(10, 3, 20, 4, 100, 30) == want


def test_reference_arm_does_not_load_the_engine_library(tmp_path):
    """The reference arm (Sparta on a sample) runs on numpy and the baseline
    binary only: neither the package nor its shared library is loaded."""
    import subprocess
    code = (
        "import sys; sys.path.insert(0, %r)\n"
        "import bench\n"
        "X, _, _, _ = bench.workload(0, 0.01)\n"
        "b = bench.CpuBaseline(X, target_seconds=0.2)\n"
        "t = b.step()\n"
        "assert t > 0, t\n"
        "maps = open('/proc/self/maps').read()\n"
        "assert 'libgsparc_b200' not in maps\n"
        "assert not any(m == 'gsparc_b200' or m.startswith('gsparc_b200.') for m in sys.modules)\n"
        "print('ok', b.kind, b.ir)\n" % ROOT)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.startswith("ok")

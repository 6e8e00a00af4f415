"""Host-side parts of bench.py's contract that need no GPU: the reference arm's other
ranks exit 0 without work or output, the defaults (one GPU, at least three warm-up steps),
and a description of the arithmetic for every mixed variant the autotuner can pick."""
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def test_reference_arm_other_ranks_exit_quietly():
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "3"],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


def test_defaults_one_gpu_and_three_warmup_steps(monkeypatch):
    import bench
    monkeypatch.setattr(sys, "argv", ["bench.py"])
    a = bench.parse_args()
    assert a.gpus == 1 and a.impl == "ours"
    assert a.warmup >= 3 and a.steps >= 1


def test_precision_text_for_every_mixed_variant():
    import bench
    from mmnorm_b200 import ops
    names = [v["name"] for v in ops.variants("mixed")]
    assert names
    for n in names:
        text = bench.precision_text(n)
        assert text.startswith("mixed: FP64 range and phase wrap")
        blk = 64 if "clen64" in n else 32
        assert "every %d samples" % blk in text, n
        if "clen64eo" in n:
            assert "even- and odd-sample chains" in text
        elif "clen" in n:
            assert "second-order" in text and "even" not in text
        else:
            assert "first-order Horner rotation recurrence" in text

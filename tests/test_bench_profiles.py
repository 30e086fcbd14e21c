"""The bench's roofline traffic comes from a committed ncu summary only when
that summary names the digest of the kernel's current source file
(bench.profiled_traffic).  These checks run on the CPU:

- every kernel summary in profiles/ that records a source digest names a
  file that exists, and its digest is the file's current one;
- the dominant kernel's summary yields its DRAM bytes;
- a summary whose digest does not match, or of another workload, yields no
  bytes;
- the step-timeline summary of the bench line takes the medians of the
  complete steps.
"""
import os
import re

import bench

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PROFILES = os.path.join(ROOT, "profiles")


def summaries():
    return sorted(f for f in os.listdir(PROFILES) if f.endswith(".md"))


def test_recorded_digests_are_current():
    seen = 0
    for name in summaries():
        text = open(os.path.join(PROFILES, name)).read()
        for m in re.finditer(r"^- source: (\S+) sha256\[:16\] ([0-9a-f]{16})$", text, re.M):
            path, digest = m.group(1), m.group(2)
            assert os.path.exists(os.path.join(ROOT, path)), (name, path)
            assert bench.source_digest(path) == digest, (name, path)
            seen += 1
    assert seen >= 3


def test_dominant_kernel_traffic_is_read():
    traffic, src = bench.profiled_traffic("k_mg_smooth_tma_mixed_1m.md", "mixed_1m")
    assert traffic is not None, src
    # 24 B per point and species on the finest level is 340 MB; the capture
    # reads the warm-up rows again, so the traffic is a little above that
    assert 340e6 < traffic < 600e6


def test_mismatched_digest_or_workload_gives_no_bytes(tmp_path, monkeypatch):
    text = open(os.path.join(PROFILES, "k_mg_smooth_tma_mixed_1m.md")).read()
    stale = re.sub(r"(^- source: \S+ sha256\[:16\] )[0-9a-f]{16}$", r"\g<1>0000000000000000", text, flags=re.M)
    (tmp_path / "profiles").mkdir()
    (tmp_path / "profiles" / "k_mg_smooth_tma_mixed_1m.md").write_text(stale)
    src_dir = tmp_path / "baccolonygrowth_b200" / "csrc"
    src_dir.mkdir(parents=True)
    src_dir.joinpath("mg_smooth.cu").write_bytes(open(os.path.join(ROOT, "baccolonygrowth_b200/csrc/mg_smooth.cu"), "rb").read())
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    traffic, src = bench.profiled_traffic("k_mg_smooth_tma_mixed_1m.md", "mixed_1m")
    assert traffic is None and "changed" in src
    monkeypatch.setattr(bench, "ROOT", ROOT)
    traffic, src = bench.profiled_traffic("k_mg_smooth_tma_mixed_1m.md", "scale_262k")
    assert traffic is None


def test_timeline_summary():
    """bench.timeline_summary: median phase ends of the steps whose seven
    marks came back, relative to each step's start, and the median period;
    a step cut short by the capacity is left out."""
    import numpy as np
    step = [0.0, 0.01, 2.28, 0.01, 0.47, 1.0, 2.29]
    tags, ms = [], []
    for k in range(3):
        tags += [1, 2, 3, 4, 5, 6, 7]
        ms += [v + 2.3 * k for v in step]
    tags += [1, 2]
    ms += [6.9, 6.91]
    out = bench.timeline_summary(np.array(tags, np.int32), np.array(ms, np.float32))
    assert out["steps"] == 3
    assert abs(out["solve_end_ms"] - 2.28) < 1e-5 and abs(out["divide_end_ms"] - 1.0) < 1e-5
    assert abs(out["period_ms"] - 2.3) < 1e-5
    assert bench.timeline_summary(np.zeros(0, np.int32), np.zeros(0, np.float32)) is None

"""Host-side helpers of bench.py: the algorithmic byte counts of the roofline
and the measurement records."""
import sys
from pathlib import Path

REPO = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(REPO))

import bench  # noqa: E402


def test_algorithmic_bytes_follow_the_fused_stage():
    kh = [(2048 * 2048, 4, 2, False, 22)]   # cells, nv, dim, Navier-Stokes, kernel class
    w = 4
    # last sweep of stages 2-3: read U^k and U^n, write U^(k+1); it also reads R
    a, m = bench.algorithmic_bytes("sweep_y", 2, kh, w)
    assert a == 2048 * 2048 * 4 * 4 * 3 and m == 2048 * 2048 * 4 * 4 * 4
    a, m = bench.algorithmic_bytes("sweep_y", 0, kh, w)   # stage 1: read U^n, write U^1
    assert a == 2048 * 2048 * 16 * 2
    a, m = bench.algorithmic_bytes("sweep_x", 1, kh, w)   # the residual round trip is not algorithmic
    assert a == 0 and m == 2048 * 2048 * 16 * 2
    # the three stages of a step add up to 8 nv w per cell
    tot = sum(bench.algorithmic_bytes(k, s, kh, w)[0] for s in range(3) for k in ("sweep_x", "sweep_y"))
    assert tot == 2048 * 2048 * 16 * 8
    one_d = [(25600, 3, 1, False, 12)]
    assert bench.algorithmic_bytes("sweep_x", 2, one_d, 8) == (25600 * 3 * 8 * 3,) * 2
    mixed = kh + [(5000, 1, 1, False, 102)]
    assert bench.algorithmic_bytes("sweep_x.c102", 2, mixed, 4)[0] == 5000 * 4 * 3


def test_records_parse(tmp_path, monkeypatch):
    f = tmp_path / "r.txt"
    f.write_text("# comment\ntraffic workload=kh2048 kernel=sweep_y stage=2 src=abc dram_read=1.5e8 "
                 "dram_write=4e7 cells=4194304 capture=\"ncu -k x\"\naccuracy n=2048 l1_ratio=1.1 src=abc\n")
    monkeypatch.setattr(bench, "RECORDS", f)
    t = bench.read_records("traffic")
    assert len(t) == 1 and t[0]["kernel"] == "sweep_y" and t[0]["dram_read"] == 1.5e8 and t[0]["capture"] == "ncu -k x"
    a = bench.read_records("accuracy")
    assert a[0]["n"] == 2048 and a[0]["l1_ratio"] == 1.1
    assert len(bench.source_hash()) == 16


def test_source_hash_ignores_comments_only():
    """The build hash drops // and /* */ comments but keeps string and
    character literals (a "//" inside a PTX string is code)."""
    src = 'asm("mov.u32 %0, 1; // not a comment");\n/* block\ncomment */ int a = \'/\'; // tail\nint b;\n'
    out = bench.strip_comments(src)
    assert '"mov.u32 %0, 1; // not a comment"' in out and "'/'" in out
    assert "block" not in out and "tail" not in out and "int b;" in out
    assert bench.strip_comments("int x = 1; // one") == bench.strip_comments("int x = 1; // two")
    assert bench.strip_comments("int x = 1;") != bench.strip_comments("int x = 2;")

"""The CLIs on a GPU: the reference's tests/validation_gpu.sh and
tests/validation.sh cases that need a device, plus the failure path."""
import os
import re
import subprocess

import pytest

pytestmark = pytest.mark.gpu
BIN = os.path.join(os.path.dirname(__file__), "..", "goldbach-gpu_b200", "bin")


def run(prog, *args, timeout=300):
    p = subprocess.run([os.path.join(BIN, prog), *map(str, args)], capture_output=True,
                       text=True, timeout=timeout)
    return p.returncode, p.stdout + p.stderr


def test_basic_run_1e9():  # validation_gpu.sh Test 1.1
    rc, out = run("goldbach", 1000000000, "--seg-size=1000000", "--p-small=100000",
                  "--batch-size=100000")
    assert rc == 0, out
    assert "satisfy Goldbach. ✓" in out and "Phase 2 fallbacks      : 0" in out
    assert re.search(r"Total computation time : [0-9.e+-]+ seconds", out)


def test_progress_flag():  # Test 1.2
    rc, out = run("goldbach", 20000000000, "--seg-size=10000000", "--p-small=1000000",
                  "--batch-size=1000000", "--progress")
    assert rc == 0 and "[Progress]" in out and "satisfy Goldbach. ✓" in out, out


def test_custom_start():  # Test 1.3
    rc, out = run("goldbach", 1000000000, "--seg-size=1000000", "--p-small=100000",
                  "--batch-size=100000", "--start=1000000")
    assert rc == 0 and "Checking range : [1000000" in out and "satisfy Goldbach. ✓" in out


def test_more_gpus_than_available():  # Test 3.6
    rc, out = run("goldbach", 100000000, "--gpus=64")
    assert "Requested" in out and "available" in out and "Using" in out
    assert rc == 0


def test_vram_guard():  # Test 3.5 (memory budget forced small)
    rc, out = run("goldbach", 100000000000, "--seg-size=100000000000", "--device-mem-mb=16")
    assert rc == 1 and "insufficient VRAM" in out


def test_failure_is_reported():
    rc, out = run("goldbach", 1000, "--seg-size=100", "--p-small=3", "--phase2-limit=3")
    assert rc == 1 and "[!] Goldbach FAILED at n = 12" in out, out


def test_json_summary():
    rc, out = run("goldbach", 10000000, "--json")
    assert rc == 0
    m = re.search(r'\{"start": 4, "limit": 10000000, "checked": (\d+)', out)
    assert m and int(m.group(1)) == 4999999


def test_single_check_1e12():  # validation.sh Test 1.2
    rc, out = run("single_check", 1000000000000)
    assert rc == 0 and "Goldbach holds. ✓" in out
    m = re.search(r"1000000000000 = (\d+) \+ (\d+)", out)
    assert m and int(m.group(1)) + int(m.group(2)) == 10**12
    assert int(m.group(1)) <= 194267


def test_journal_interrupt_and_resume(tmp_path):
    """A run stopped after 3 journal records, a torn write appended, then
    the same command resumes: same summary as one uninterrupted run, every
    segment journaled exactly once."""
    j = tmp_path / "j.txt"
    args = (2000000000, "--seg-size=67108864", "--p-small=1000000")  # 15 segments
    rc, out = run("goldbach", *args, f"--journal={j}", "--journal-segments=2",
                  "--stop-after-batches=3")
    assert rc == 3 and "rerun the same command to resume" in out, out
    assert len(j.read_text().splitlines()) == 4
    with open(j, "a") as f:
        f.write("seg 6 8 checked 1342")  # the write an interruption tore
    rc, out2 = run("goldbach", *args, f"--journal={j}", "--journal-segments=2")
    assert rc == 0 and "6 of 15 segments done, 5 batches to run" in out2, out2
    rc, ref = run("goldbach", *args)
    assert rc == 0
    for key in ("satisfy Goldbach. ✓", "Phase 2 fallbacks      :", "Max minimal p          :"):
        a = [l for l in out2.splitlines() if key in l]
        b = [l for l in ref.splitlines() if key in l]
        assert a == b and a, (key, a, b)
    segs = []
    checked = 0
    for line in j.read_text().splitlines()[1:]:
        f = line.split()
        segs += list(range(int(f[1]), int(f[2])))
        checked += int(f[4])
    assert sorted(segs) == list(range(15)) and checked == 999999999


def test_counts_mode(tmp_path):
    """goldbach --counts prints the reference's `c(n) = k` lines."""
    import json
    g = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "ref_goldbach_count.json")))
    rc, out = run("goldbach", 2000, "--counts")
    assert rc == 0, out
    lines = [l for l in out.splitlines() if l.startswith("c(")]
    want = [f"c({g['first_n'] + 2 * j}) = {v}" for j, v in enumerate(g["counts"]) if g["first_n"] + 2 * j <= 2000]
    assert lines == want and "Even numbers counted : 999" in out


def test_per_n_output_files(tmp_path, oracle):
    """--minp-out / --bitmap-out: the minimal p and verified bit of every n,
    in range order, across segment boundaries that are not byte-aligned."""
    import numpy as np
    m, b = tmp_path / "minp.u32", tmp_path / "bits.bin"
    rc, out = run("goldbach", 2000000, "--seg-size=100002", f"--minp-out={m}", f"--bitmap-out={b}")
    assert rc == 0, out
    count = 999999
    got = np.fromfile(m, np.uint32)
    np.testing.assert_array_equal(got, oracle.minp(4, count))
    bits = np.unpackbits(np.fromfile(b, np.uint8), bitorder="little")
    assert bits.size == (count + 7) // 8 * 8 and bits[:count].all() and not bits[count:].any()


def test_autotune_and_its_cache(tmp_path):
    cache = tmp_path / "tune.txt"
    args = (4000000000, "--seg-size=67108864", f"--autotune-cache={cache}")
    rc, out = run("goldbach", *args)
    assert rc == 0 and "[Autotune] chunk=" in out and "candidates)" in out, out
    line = cache.read_text().splitlines()[0]
    assert line.startswith("class 32 1000000 100000000 chunk ")
    rc, out2 = run("goldbach", *args)
    assert rc == 0 and f"(from {cache})" in out2
    ref = [l for l in out.splitlines() if "Phase 2 fallbacks" in l or "satisfy" in l]
    assert ref == [l for l in out2.splitlines() if "Phase 2 fallbacks" in l or "satisfy" in l]

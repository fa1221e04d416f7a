"""The resume journal of the goldbach CLI (--journal=FILE), on the host.

Journals are written here by hand in the CLI's format, so these cases need
no GPU: a journal that already covers the whole range, or that records a
failure, is answered from the file alone.  The interrupted-and-resumed run
on a device is in test_gpu_cli.py.
"""
import os
import subprocess

import pytest

BIN = os.path.join(os.path.dirname(__file__), "..", "goldbach-gpu_b200", "bin", "goldbach")


def fnv1a(s):
    h = 1469598103934665603
    for c in s.encode():
        h ^= c
        h = (h * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


def header(start, limit, seg, p_small, phase2=100000000):
    return (f"goldbach-journal v1 start={start} limit={limit} seg_size={seg} "
            f"p_small={p_small} phase2={phase2}")


def record(lo, hi, checked, fb=0, fail=0, first=0, maxp=0):
    body = (f"seg {lo} {hi} checked {checked} fallbacks {fb} failures {fail} "
            f"first_fail {first} max_minp {maxp}")
    return f"{body} sum {fnv1a(body):016x}"


def run(*args):
    p = subprocess.run([BIN, *map(str, args)], capture_output=True, text=True, timeout=120)
    return p.returncode, p.stdout + p.stderr


# [4, 1000] in segments of 100 even n: 499 n, 5 segments
ARGS = (1000, "--seg-size=100", "--p-small=1000000")


def write(path, lines, tail=""):
    path.write_text("\n".join(lines) + "\n" + tail)


def test_complete_journal_is_answered_without_a_device(tmp_path):
    j = tmp_path / "j.txt"
    write(j, [header(4, 1000, 100, 1000),
              record(0, 2, 200, fb=3, maxp=13), record(2, 5, 299, fb=1, maxp=19)])
    rc, out = run(*ARGS, f"--journal={j}")
    assert rc == 0, out
    assert "5 of 5 segments done" in out
    assert "All even numbers from 4 up to 1000 satisfy Goldbach. ✓" in out
    assert "Phase 2 fallbacks      : 4" in out and "Max minimal p          : 19" in out


def test_journaled_failure_is_reported(tmp_path):
    j = tmp_path / "j.txt"
    write(j, [header(4, 1000, 100, 1000), record(0, 1, 100, fail=2, first=12)])
    rc, out = run(*ARGS, f"--journal={j}")
    assert rc == 1 and "[!] Goldbach FAILED at n = 12" in out, out


def test_journal_of_another_run_is_refused(tmp_path):
    j = tmp_path / "j.txt"
    write(j, [header(4, 2000, 100, 1000)])
    rc, out = run(*ARGS, f"--journal={j}")
    assert rc == 1 and "belongs to another run" in out, out


@pytest.mark.parametrize("tail", ["seg 2 5 checked 299 fallb", "bad\n"])
def test_torn_tail_is_cut_and_its_segments_run_again(tmp_path, tail):
    j = tmp_path / "j.txt"
    good = [header(4, 1000, 100, 1000), record(0, 2, 200)]
    if tail.endswith("\n"):  # a complete line with a wrong hash
        write(j, good + [record(2, 5, 299).replace("checked 299", "checked 298")])
    else:  # a line cut short
        write(j, good, tail=tail)
    rc, out = run(*ARGS, f"--journal={j}")
    assert "2 of 5 segments done, 1 batches to run" in out, out
    # the torn record is gone; a GPU run appends the missing one after it
    lines = j.read_text().splitlines()
    assert lines[:2] == good
    if rc == 0:
        assert len(lines) == 3 and lines[2].startswith("seg 2 5 checked 299 ")
    else:
        assert "No CUDA devices found." in out and len(lines) == 2


def test_new_journal_gets_a_header(tmp_path):
    j = tmp_path / "j.txt"
    run(*ARGS, f"--journal={j}")
    assert j.read_text().splitlines()[0] == header(4, 1000, 100, 1000)


def test_outputs_and_journal_do_not_mix(tmp_path):
    rc, out = run(1000, f"--minp-out={tmp_path / 'm'}", f"--journal={tmp_path / 'j'}")
    assert rc == 1 and "cannot be combined with --journal" in out

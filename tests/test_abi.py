"""C-ABI library and CLI checks that need no GPU."""
import os
import re
import subprocess

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
PKG = os.path.join(ROOT, "goldbach-gpu_b200")
BIN = os.path.join(PKG, "bin")


def header_symbols():
    syms = set()
    for dirpath, _, files in os.walk(os.path.join(ROOT, "include")):
        for f in files:
            if f.endswith(".h"):
                txt = open(os.path.join(dirpath, f)).read()
                txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
                for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(gb_\w+)\s*\(", txt, flags=re.M):
                    syms.add(m.group(1))
    return syms


def test_library_exports_every_header_symbol(gbmod):
    L = gbmod.load()
    syms = header_symbols()
    assert len(syms) >= 12
    missing = [s for s in sorted(syms) if not hasattr(L, s)]
    assert not missing, missing


def test_library_is_in_tree_and_for_sm100a():
    so = os.path.join(PKG, "libgoldbach_b200.so")
    assert os.path.exists(so)
    out = subprocess.run(["strings", so], capture_output=True, text=True).stdout
    assert "sm_100a" in out


def run(prog, *args):
    p = subprocess.run([os.path.join(BIN, prog), *map(str, args)], capture_output=True, text=True,
                       timeout=60)
    return p.returncode, p.stdout + p.stderr


def test_goldbach_help():
    rc, out = run("goldbach", "--help")
    assert rc == 0 and "Usage:" in out and "--seg-size=N" in out
    rc, out = run("goldbach")
    assert rc == 0 and "Usage:" in out


@pytest.mark.parametrize("args,expect", [
    (["2", "--seg-size=1000000"], "Error: LIMIT must be >= 4"),            # validation_gpu.sh 3.1
    (["1000000000", "--seg-size=1000001"], "Error: SEG_SIZE must be even"),  # 3.2
    (["1000000000", "--p-small=5000000000"], "Error: P_SMALL must be <= 4000000000"),  # 3.3
    (["1000000000", "--start=1000000002"], "Error: START must be less than LIMIT"),  # 3.4
    (["abc", "--seg-size=1000000"], "Error: Invalid numeric argument"),   # 3.7
    (["1000000000", "--invalid"], "Error: Invalid"),                       # 2.2
    (["--seg-size=1000000"], "Error: "),                                   # 2.3
    (["1000000000", "--seg-size=abc"], "Error: Invalid numeric argument"),
])
def test_goldbach_argument_errors(args, expect):
    rc, out = run("goldbach", *args)
    assert rc == 1 and expect in out, out


def test_single_check_help():
    rc, out = run("single_check", "--help")
    assert rc == 0 and "Usage:" in out


@pytest.mark.parametrize("arg,expect", [
    ("100000000000000000000", "Error: Number is too large"),  # validation.sh 3.4
    ("1000000000001", "Error: n must be an even integer"),    # 3.5
    ("2", "Error: n must be >= 4"),                           # 3.6
    ("abc", "Error: Invalid numeric argument"),
])
def test_single_check_argument_errors(arg, expect):
    rc, out = run("single_check", arg)
    assert rc == 1 and expect in out, out

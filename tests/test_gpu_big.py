"""Even n beyond 2^64 (gb_check_big, big_check) against the big-n oracle:
the minimal p with n - p passing the 12-base strong test, bit for bit, and
the reference's published big_check partitions (RESULTS.md:141-149, valid
but not minimal) as upper bounds."""
import importlib.util
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
# RESULTS.md:143-147; the row labelled 10^200 gives 204 digits and p = 113,
# which is n = 10^203 (10^203 - 113 is prime, 10^200 - 113 is not; the
# minimal p of 10^200 is 7103)
PUBLISHED = {10**50: 383, 10**100: 797, 10**203: 113, 10**1000: 26981}


@pytest.fixture(scope="module")
def B():
    spec = importlib.util.spec_from_file_location("big_oracle", os.path.join(ROOT, "oracle", "big_oracle.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    mod.PR = mod.small_primes(10**6)
    return mod


def _cases():
    rng = np.random.default_rng(41)
    ns = [2**64, 2**64 + 2, 2**65 + 10, 10**20, 10**24 + 6, 3 * 10**24, 10**30, 2**127 - 1 + 1]
    for bits in (96, 128, 200, 256, 512, 1024, 2048):
        for _ in range(3):
            x = int(rng.integers(1, 2**62)) << (bits - 62)
            x |= int(rng.integers(0, 2**62))
            ns.append(x - (x & 1))
    return ns


@pytest.mark.parametrize("n", _cases(), ids=lambda n: f"{n.bit_length()}b")
def test_matches_the_oracle(ctx, B, n):
    p, q, r = ctx.check_big(n)
    assert p == B.minimal_p(n, primes=B.PR), n
    assert q == n - p and B.is_probable_prime(q)
    assert r["candidates"] >= 1


@pytest.mark.parametrize("n", list(PUBLISHED), ids=lambda n: f"1e{len(str(n)) - 1}")
def test_published_partitions_bound_minimal_p(ctx, B, n):
    p, q, _ = ctx.check_big(n)
    assert 0 < p <= PUBLISHED[n] and q == n - p
    assert p == B.minimal_p(n, primes=B.PR)


def test_below_2_64_takes_the_deterministic_path(ctx):
    ns = [4, 6, 100, 10**12, 2**64 - 2]
    for n in ns:
        p, q, _ = ctx.check_big(n)
        p1, q1, _ = ctx.check_single(np.array([n], np.uint64))
        assert (p, q) == (int(p1[0]), int(q1[0]))


def test_p_limit_and_bad_input(ctx, gbmod, B):
    n = 10**40
    want = B.minimal_p(n, primes=B.PR)
    p, _, _ = ctx.check_big(n, p_limit=want - 1)
    assert p == 0
    with pytest.raises(gbmod.GbError):
        ctx.check_big(10**40 + 1)
    with pytest.raises(gbmod.GbError):
        ctx.check_big(2**4200)


def test_big_check_cli(B):
    exe = os.path.join(ROOT, "goldbach-gpu_b200", "bin", "big_check")
    n = 10**30
    r = subprocess.run([exe, str(n)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    p = B.minimal_p(n, primes=B.PR)
    assert f"{n}\n  = {p} + {n - p}\n" in r.stdout and "Goldbach holds. ✓" in r.stdout
    r = subprocess.run([exe, "12345"], capture_output=True, text=True)
    assert r.returncode == 1 and "applies to even integers >= 4" in r.stderr
    r = subprocess.run([exe, "12a4"], capture_output=True, text=True)
    assert r.returncode == 1 and "Input must be a positive integer" in r.stderr

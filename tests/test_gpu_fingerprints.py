"""Bit-for-bit regression pin of the CUDA stepper: SHA-256 prefixes of all six fields and the
probe series after a few steps, per case (golden gain, plane-wave and PEC cases, C0, C1, the
280^3 workload), storage form (FP64, FP32, FP16, BF16 nearest and stochastic) and kernel path,
against tests/golden/fingerprints.json (written by tests/golden/make_fingerprints.py on a B200).
Launch shapes, staging and vector widths may change freely; the arithmetic may not without a
regenerated fixture."""
import json
import sys

import pytest

from conftest import GOLDEN

sys.path.insert(0, str(GOLDEN))
import make_fingerprints as mf  # noqa: E402

STORED = json.loads((GOLDEN / "fingerprints.json").read_text())


@pytest.mark.gpu
@pytest.mark.parametrize("name,steps", mf.CASES)
def test_stepper_bits_unchanged(pkg, name, steps):
    bad = []
    for n, st, prec, rnd, path in mf.keys():
        if n != name:
            continue
        k = mf.key_name(n, prec, rnd, path)
        got = mf.fingerprint(pkg, n, st, prec, rnd, path)
        if STORED.get(k) != got:
            bad.append((k, STORED.get(k), got))
    assert not bad, bad


def test_fixture_covers_every_key():
    assert set(STORED) == {mf.key_name(n, p, r, k) for n, _, p, r, k in mf.keys()}

"""Pins of the project-owned elementary functions and of the Philox stream (CPU).

exp/log/pow are shared by the CUDA path and the oracle so FP64 parity can be
bit-exact; here they are checked against glibc (through numpy) to a few ulp.
Philox4x32-10 is checked against the published Random123 known-answer vectors
(Salmon et al., SC'11, kat_vectors), and the NetStim stream layout against its
definition: uniform = (word + 1) / (2^32 + 1), negexp = -log(uniform).
"""
import math

import numpy as np
import pytest

import oracle


def ulp_error(got, want):
    want = np.asarray(want, dtype=np.float64)
    spacing = np.spacing(np.abs(want))
    return np.abs(np.asarray(got) - want) / spacing


def test_exp_within_two_ulp_of_glibc():
    xs = np.concatenate([np.linspace(-700.0, 700.0, 20001), np.linspace(-1.0, 1.0, 20001),
                         np.array([0.0, 1e-300, -1e-300, 709.0, -708.0])])
    got = np.array([oracle.exp(float(x)) for x in xs])
    assert np.max(ulp_error(got, np.exp(xs))) <= 2.0


def test_log_within_two_ulp_of_glibc():
    xs = np.concatenate([np.exp(np.linspace(-700.0, 700.0, 20001)), np.linspace(0.5, 2.0, 20001),
                         np.array([1.0, 2.0, 1e-310, 4.9e-324, 1.7e308])])
    got = np.array([oracle.log(float(x)) for x in xs])
    want = np.log(xs)
    err = ulp_error(got, want)
    err[want == 0.0] = np.abs(got[want == 0.0])
    assert np.max(err) <= 2.0


def test_special_values():
    assert oracle.exp(float("-inf")) == 0.0
    assert oracle.exp(float("inf")) == math.inf
    assert math.isnan(oracle.exp(float("nan")))
    assert oracle.log(0.0) == -math.inf
    assert math.isnan(oracle.log(-1.0))
    assert oracle.pow(3.0, 0.0) == 1.0   # hh's Q10 at celsius = 6.3
    assert abs(oracle.pow(3.0, 0.5) - math.sqrt(3.0)) < 4e-16


def test_division_free_milli_quotient_equals_ieee_division():
    """x / 0.001 without a division (the CUDA path's current and dI/dV terms) is the IEEE quotient."""
    rng = np.random.default_rng(7)
    bits = rng.integers(0, 2**63, size=2_000_000, dtype=np.uint64)
    exponent = rng.integers(1023 - 900, 1023 + 901, size=bits.size).astype(np.uint64)
    bits = (bits & np.uint64(0x800FFFFFFFFFFFFF)) | (exponent << np.uint64(52))
    xs = np.concatenate([bits.view(np.float64), np.linspace(-1.0, 1.0, 200_001), np.arange(-5000, 5001) * 1e-7,
                         np.array([0.0, -0.0, 1e-310, -1e-310, 5e-324, 1e300, np.inf, -np.inf, 2.0**-900,
                                   2.0**900, np.nextafter(2.0**-900, 0.0)])])
    got = oracle.div_milli(xs)
    want = xs / 0.001
    assert np.array_equal(got.view(np.uint64), want.view(np.uint64))
    nan = oracle.div_milli(np.array([np.nan]))
    assert np.isnan(nan[0])


@pytest.mark.parametrize("ctr,key,want", [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
])
def test_philox_known_answers(ctr, key, want):
    assert tuple(oracle.philox4x32_10(list(ctr), *key)) == want


def test_negexp_stream_matches_its_definition():
    """First block of a stream: counter words (0, id3, id1, id2) under key (seed lo, seed hi)."""
    logical, digest, seed = 4097, 0xA186833B569FF3B2, 1
    draws = oracle.negexp_stream(logical, digest, seed, 8)
    block0 = oracle.philox4x32_10([0, digest & 0xFFFFFFFF, logical & 0xFFFFFFFF, logical >> 32], seed, 0)
    block1 = oracle.philox4x32_10([1, digest & 0xFFFFFFFF, logical & 0xFFFFFFFF, logical >> 32], seed, 0)
    words = block0 + block1
    for draw, word in zip(draws, words):
        u = (word + 1.0) * (1.0 / 4294967297.0)
        assert draw == pytest.approx(-math.log(u), rel=4e-16, abs=0)


def test_negexp_mean_and_variance():
    draws = oracle.negexp_stream(123456, 0xA186833B569FF3B2, 1, 200000)
    assert abs(draws.mean() - 1.0) < 0.01
    assert abs(draws.var() - 1.0) < 0.02

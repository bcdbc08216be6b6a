"""The sampler (renderer/shaders/sample.wgsl) as the oracle restates it, pinned by the reference's own tests:
renderer/src/sample.rs:90-99 (the direction numbers), 104-125 (a (0, m, 2)-net and 1D strata), 168-179 (ids and
seeds decorrelate)."""
import json
from pathlib import Path

import numpy as np
import pytest

import oracle

GOLDEN = json.loads((Path(__file__).parent / "golden" / "sobol_directions.json").read_text())


def test_the_directions_are_the_shaders():
    d = oracle.sobol_directions()
    assert d[:, :16].tolist() == GOLDEN["first16"]
    assert d[:, 31].tolist() == GOLDEN["last"]


def test_the_gpu_table_is_the_recurrence():
    # The CUDA side fills its table from the same recurrence (pathtrace.cu sobol_directions); it is checked on the
    # GPU by test_gpu_render's camera parity. Here: the recurrence's first 16 are the literals.
    assert oracle.sobol_directions()[:, :16].tolist() == GOLDEN["first16"]


@pytest.mark.parametrize("seed,d", [(0, 0), (0x12345678, 7), (None, 0xDEAD)])
@pytest.mark.parametrize("m", [4, 6, 8])
def test_the_first_2_to_the_m_points_are_a_net(seed, d, m):
    if seed is None:
        seed = oracle.hash_hp(99)
    n = 1 << m
    pts = np.array([oracle.rng4(seed, i, d) for i in range(n)], np.float64)
    cell = lambda v, k: np.minimum((v * (1 << k)).astype(np.int64), (1 << k) - 1)
    for a in range(m + 1):
        c = (cell(pts[:, 0], a) << (m - a)) | cell(pts[:, 1], m - a)
        assert len(np.unique(c)) == n, f"interval {a}x{m - a} twice"
    for k in range(4):
        assert sorted(cell(pts[:, k], m).tolist()) == list(range(n))
    assert np.all((pts >= 0) & (pts < 1))


def test_ids_and_seeds_decorrelate():
    a = np.array([oracle.rng4(5, i, 1)[0] for i in range(64)])
    b = np.array([oracle.rng4(5, i, 2)[0] for i in range(64)])
    c = np.array([oracle.rng4(6, i, 1)[0] for i in range(64)])
    assert abs(np.corrcoef(a, b)[0, 1]) < 0.35 and abs(np.corrcoef(a, c)[0, 1]) < 0.35


def test_hash_hp_known_values():
    # sample.wgsl:77-85 on a few words, evaluated by hand-checkable 32-bit arithmetic.
    def ref(i):
        i ^= i >> 16
        i = (i * 0x21F0AAAD) & 0xFFFFFFFF
        i ^= i >> 15
        i = (i * 0xD35A2D97) & 0xFFFFFFFF
        i ^= i >> 15
        return i ^ 0xE6FE3BEB
    for x in [0, 1, 0x5EED, 0xFFFFFFFF, 123456789]:
        assert oracle.hash_hp(x) == ref(x)

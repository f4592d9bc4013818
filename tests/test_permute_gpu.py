"""Lookup permute-sort parity with permute_expression_pair_seq
(halo2_proofs/src/plonk/lookup/prover.rs:787-880; GPU-vs-seq test at
halo2_proofs/src/cuda/tests.rs:2340)."""
import numpy as np
import pytest

from conftest import assert_limbs_equal

pytestmark = pytest.mark.gpu


def make_lookup(orc, n, usable, table_size, seed, skew=False):
    rng = np.random.default_rng(seed)
    tvals = orc.chacha_fr(seed, table_size)
    table = tvals[np.arange(usable) % table_size]
    if skew:
        idx = np.minimum(rng.geometric(0.3, usable) - 1, table_size - 1)
    else:
        idx = rng.integers(0, table_size, usable)
    inp = tvals[idx]
    pad = np.zeros((n - usable, 4), np.uint64)
    return np.concatenate([inp, pad]), np.concatenate([table, pad])


def run(h2b, orc, inp, table, n, usable):
    want_a, want_s = orc.permute_pair(inp, table, n, usable)
    d_in, d_tab = h2b.to_dev(inp), h2b.to_dev(table)
    d_pa, d_ps = h2b.dev_empty(32 * n), h2b.dev_empty(32 * n)
    h2b.permute_expression_pair_device(d_in, d_tab, d_pa, d_ps, n, usable)
    assert_limbs_equal(h2b.to_host(d_pa), want_a, "A'")
    assert_limbs_equal(h2b.to_host(d_ps), want_s, "S'")


@pytest.mark.parametrize("k,table_size", [(4, 3), (8, 16), (12, 256), (13, 1024), (13, 1025), (16, 256),
                                          (16, 60000)])
def test_permute_uniform(h2b, orc, cuda, k, table_size):
    n = 1 << k
    usable = n - 7
    table_size = min(table_size, usable)
    inp, table = make_lookup(orc, n, usable, table_size, 100 + k)
    run(h2b, orc, inp, table, n, usable)


def test_permute_skewed_and_constant(h2b, orc, cuda):
    n = 1 << 14
    usable = n - 5
    inp, table = make_lookup(orc, n, usable, 256, 7, skew=True)
    run(h2b, orc, inp, table, n, usable)
    # every input row the same value
    inp2 = inp.copy()
    inp2[:usable] = table[3]
    run(h2b, orc, inp2, table, n, usable)


def test_permute_config3_size(h2b, orc, cuda):
    n = 1 << 20
    usable = n - 7
    inp, table = make_lookup(orc, n, usable, 256, 20)
    run(h2b, orc, inp, table, n, usable)


def test_permute_missing_value_is_an_error(h2b, orc, cuda):
    n = 1 << 10
    usable = n - 3
    inp, table = make_lookup(orc, n, usable, 64, 9)
    inp[5] = orc.chacha_fr(12345, 1)[0]
    d_pa, d_ps = h2b.dev_empty(32 * n), h2b.dev_empty(32 * n)
    with pytest.raises(h2b.Halo2GpuError):
        h2b.permute_expression_pair_device(h2b.to_dev(inp), h2b.to_dev(table), d_pa, d_ps, n, usable)


def test_permute_config3_table_shape(h2b, orc, cuda):
    """The config-3 lookup: a 256-entry range table in the first rows, the
    rest of the usable rows padded with its first value (zero), inputs drawn
    from the table (so the padding value is a leftover many times over)."""
    n = 1 << 16
    usable = n - 6
    rng = np.random.default_rng(3)
    tvals = orc.chacha_fr(33, 256)
    tvals[0] = 0
    table = np.zeros((n, 4), np.uint64)
    table[:256] = tvals
    inp = np.zeros((n, 4), np.uint64)
    inp[:usable] = tvals[rng.integers(0, 256, usable)]
    run(h2b, orc, inp, table, n, usable)


def test_permute_all_distinct_and_unused_values(h2b, orc, cuda):
    """Every table row distinct (the distinct-value sort carries the whole
    table), and inputs that use only a few table values (most values are
    leftovers with their full multiplicity)."""
    n = 1 << 14
    usable = n - 9
    table = np.zeros((n, 4), np.uint64)
    table[:usable] = orc.chacha_fr(44, usable)
    rng = np.random.default_rng(4)
    inp = np.zeros((n, 4), np.uint64)
    inp[:usable] = table[rng.integers(0, usable, usable)]
    run(h2b, orc, inp, table, n, usable)
    inp2 = np.zeros((n, 4), np.uint64)
    inp2[:usable] = table[rng.integers(0, 5, usable)]
    run(h2b, orc, inp2, table, n, usable)


@pytest.mark.parametrize("n,usable", [(8, 1), (16, 16), (1 << 12, (1 << 12) - 1)])
def test_permute_edge_sizes(h2b, orc, cuda, n, usable):
    inp, table = make_lookup(orc, n, usable, min(5, usable), 70 + n)
    run(h2b, orc, inp, table, n, usable)

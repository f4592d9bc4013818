"""The allocation-free batch inversion, h2b_batch_invert_noalloc.

It exists for callers that cannot allocate device memory -- code that keeps
the reference's scratch-free batch_invert call shape, code whose device
memory is wholly pre-reserved by a pool it does not own, and code that must
avoid the synchronisation an allocation implies.  It must give exactly the
result of the existing entry point, `_halo2_batch_invert`, call after call,
even though every call reuses the same fixed array inside the library.

This file is named so that pytest collects it last."""
import numpy as np
import pytest

from conftest import assert_limbs_equal

pytestmark = pytest.mark.gpu


def test_noalloc_matches_existing_entry_point_on_consecutive_calls(h2b, orc, cuda):
    L = h2b.lib()
    sh = h2b.stream_handle()
    # two calls in a row with different sizes and fields, so the second call
    # runs over the array contents the first one left behind
    for n, field_type, seed in ((1 << 20, 0, 11), (300007, 1, 12)):
        x = orc.chacha_fr(seed, n)
        x[::97] = 0
        d_existing = h2b.to_dev(x)
        d_noalloc = h2b.to_dev(x)
        h2b.check(L._halo2_batch_invert(h2b.ptr(d_existing), field_type, n, sh), "_halo2_batch_invert")
        h2b.check(L.h2b_batch_invert_noalloc(h2b.ptr(d_noalloc), field_type, n, sh), "h2b_batch_invert_noalloc")
        got = h2b.to_host(d_noalloc)
        assert_limbs_equal(got, h2b.to_host(d_existing), f"noalloc vs _halo2_batch_invert n={n}")
        sel = np.r_[0:4096, n - 4096:n]
        assert_limbs_equal(got[sel], orc.batch_invert(x[sel], field_type), "noalloc vs oracle (sampled)")


def test_noalloc_rejects_lengths_beyond_its_limit(h2b, cuda):
    L = h2b.lib()
    err = L.h2b_batch_invert_noalloc(None, 0, (1 << 26) + 1, h2b.stream_handle())
    assert err.code != 0
    with pytest.raises(h2b.Halo2GpuError):
        h2b.check(err, "h2b_batch_invert_noalloc")

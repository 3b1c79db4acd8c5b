"""The byte thresholds of the device tonemap (lrt_tonemap_table, host only) against the reference's own
to_byte (io/image_write.cpp:10-20, compiled in oracle/_ref): the committed fixture's bytes, every float
within 300 ulps of each threshold, and random radiances convert identically when a value's byte is
the number of thresholds at or below it."""
import numpy as np
import pytest

from conftest import golden

import lrt
import oracle

needs_ref = pytest.mark.skipif(not oracle.reference_available(), reason="reference oracle not built")


def bytes_from_table(table, values):
    v = np.asarray(values, dtype=np.float32)
    out = np.searchsorted(table[1:], v, side="right").astype(np.int64)
    out[np.isnan(v)] = 0
    out[(v < 0) & ~np.isinf(v)] = 0
    out[v == -np.inf] = 255
    return out.astype(np.uint8)


def test_table_is_monotonic_and_bounded():
    t = lrt.tonemap_table()
    assert t[0] == 0.0 and np.all(np.diff(t[1:]) >= 0) and np.isfinite(t).all()
    # byte 255 starts at the threshold of 255/256 (0.999 * 256 truncates to 255 as well)
    assert 0.99 < t[255] < 1.0 and 0.0 < t[1] < 1e-4


def test_table_reproduces_the_golden_bytes():
    g = golden("image_out_kat.npz")
    t = lrt.tonemap_table()
    assert np.array_equal(bytes_from_table(t, g["rgb"].ravel()), g["bytes"].ravel())


@needs_ref
def test_table_matches_reference_near_every_threshold():
    t = lrt.tonemap_table()
    bits = t[1:].view(np.int32).astype(np.int64)
    around = (bits[:, None] + np.arange(-300, 301)[None, :]).ravel()
    around = np.unique(around[around >= 0]).astype(np.int32).view(np.float32)
    vals = np.concatenate([around, np.float32([np.nan, np.inf, -np.inf, -0.0, -1.0, 1e-45, 3.4e38])])
    rng = np.random.default_rng(7)
    vals = np.concatenate([vals, np.exp(rng.normal(-1.0, 2.0, 200_000)).astype(np.float32)])
    pad = (-len(vals)) % 3
    vals = np.concatenate([vals, np.zeros(pad, np.float32)]).reshape(1, -1, 3)
    ref = oracle.to_bytes(vals).ravel()
    assert np.array_equal(bytes_from_table(t, vals.ravel()), ref)

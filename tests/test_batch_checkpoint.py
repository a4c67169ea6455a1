"""Checkpoint files of the batched OC loop (no GPU): atomic write, round trip,
version check."""
import os

import numpy as np
import pytest

from maple_b200.batch import load_checkpoint, save_checkpoint


def test_roundtrip_and_atomic_write(tmp_path):
    path = os.path.join(tmp_path, "ck.npz")
    st = dict(x=np.random.default_rng(0).random((3, 8)), iters=np.array([1, 2, 3]), it=5, stop_rule="reference")
    save_checkpoint(path, st)
    assert os.path.exists(path) and not os.path.exists(path + ".tmp.npz")
    got = load_checkpoint(path)
    np.testing.assert_array_equal(got["x"], st["x"])
    assert int(got["it"]) == 5 and str(got["stop_rule"]) == "reference" and list(got["iters"]) == [1, 2, 3]


def test_version_mismatch_is_rejected(tmp_path):
    path = os.path.join(tmp_path, "ck.npz")
    np.savez(path, version=99, x=np.zeros(2))
    with pytest.raises(ValueError):
        load_checkpoint(path)

"""Held-out sample split of the hypergradient alpha selection (host logic)."""

import numpy as np
import pytest


def test_holdout_split():
    from cs_dmri_b200.hyper import holdout_split
    from cs_dmri_b200.phantom import gradient_table
    bvals, _ = gradient_table(1)
    tr, ho = holdout_split(bvals, 0.1, seed=3)
    dwi = np.flatnonzero(bvals > 50)
    assert ho.size == round(0.1 * dwi.size) and np.all(bvals[ho] > 50)
    assert np.array_equal(np.sort(np.concatenate([tr, ho])), np.arange(bvals.size))
    assert np.all(np.isin(np.flatnonzero(bvals <= 50), tr))
    tr2, ho2 = holdout_split(bvals, 0.1, seed=3)
    assert np.array_equal(ho, ho2)
    assert not np.array_equal(ho, holdout_split(bvals, 0.1, seed=4)[1])
    with pytest.raises(ValueError, match="holdout"):
        holdout_split(bvals, 0.0)

"""FastMultipoleMethod facade: construction and argument checks that need no
GPU (the reference's constructor contract, jaccpot/solver.py:664-760)."""

from __future__ import annotations

import pytest

from jaccpot_b200 import FastMultipoleMethod


def test_defaults_mirror_the_reference():
    f = FastMultipoleMethod()
    assert f.basis == "real" and f.theta == 0.6 and f.G == 1.0 and f.softening == 1e-3


@pytest.mark.parametrize("kw", [{"basis": "cartesian"}, {"basis": "solidfmm"}, {"precision": "fp64"},
                                {"preset": "nope"}, {"theta": 1.0}, {"m2l_impl": "pallas"},
                                {"use_pallas": True}])
def test_unsupported_options_raise(kw):
    with pytest.raises(ValueError):
        FastMultipoleMethod(**kw)


def test_unknown_keywords_raise():
    with pytest.raises(TypeError):
        FastMultipoleMethod(nonsense=1)


def test_prepare_rejects_bad_shapes():
    import numpy as np

    f = FastMultipoleMethod()
    with pytest.raises(ValueError):
        f.prepare_state(np.zeros((5, 2)), np.ones(5))

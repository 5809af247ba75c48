"""Degenerate and boundary inputs through the public API on the GPU: a single
particle, a single leaf, two leaves, coincident particles with softening,
zero masses, empty target lists, the lowest and highest orders."""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

import oracle as O  # noqa: E402
from jaccpot_b200 import FastMultipoleMethod, workloads  # noqa: E402


def _direct(pos, mass, eps):
    acc, _ = O.direct_sum(pos.astype(np.float64), mass.astype(np.float64), eps2=eps * eps)
    return acc


def _oracle(fmm_state, pos, mass, p, eps):
    t = fmm_state.topology
    perm = t.permutation
    r = O.Pass(t, np.float64).run(p, pos[perm].astype(np.float64), mass[perm].astype(np.float64), 1.0, eps * eps)
    out = np.empty_like(r["acc"])
    out[perm] = r["acc"]
    return out


def test_single_particle_feels_nothing():
    fmm = FastMultipoleMethod(softening=0.0)
    acc = fmm.compute_accelerations(np.zeros((1, 3), np.float32), np.ones(1, np.float32), max_order=4)
    assert acc.shape == (1, 3) and np.all(acc == 0)


@pytest.mark.parametrize("n,leaf", [(2, 16), (10, 16), (33, 32), (200, 8)])
def test_small_systems_match_direct_sum(n, leaf):
    pos, mass = workloads.uniform_cube(n, seed=n)
    fmm = FastMultipoleMethod(theta=0.5, softening=1e-2)
    acc = fmm.compute_accelerations(pos, mass, leaf_size=leaf, max_order=8)
    ref = _direct(pos, mass, 1e-2)
    err = workloads.relative_errors(acc, ref)
    assert np.isfinite(acc).all()
    assert err.max() <= 1e-3, err.max()


def test_coincident_particles_with_softening():
    rng = np.random.default_rng(0)
    pos = np.concatenate([np.zeros((40, 3)), rng.uniform(-1, 1, (200, 3))]).astype(np.float32)
    mass = np.ones(240, np.float32)
    fmm = FastMultipoleMethod(theta=0.5, softening=0.05)
    st = fmm.prepare_state(pos, mass, leaf_size=16, max_order=6)
    acc = fmm.evaluate_prepared_state(st)
    assert np.isfinite(acc).all()
    ref = _oracle(st, pos, mass, 6, 0.05)
    err = workloads.relative_errors(acc, ref)
    assert np.percentile(err, 99) <= 1e-5


def test_zero_masses():
    pos, mass = workloads.clustered(5000, seed=4)
    mass = mass.copy()
    mass[::3] = 0.0
    mass[:200] = 0.0  # whole leaves without mass
    fmm = FastMultipoleMethod(theta=0.5, softening=0.0)
    st = fmm.prepare_state(pos, mass, leaf_size=16, max_order=6)
    acc = fmm.evaluate_prepared_state(st)
    assert np.isfinite(acc).all()
    ref = _oracle(st, pos, mass, 6, 0.0)
    err = workloads.relative_errors(acc, ref)
    assert np.percentile(err, 99) <= 1e-5


def test_empty_target_list():
    pos, mass = workloads.uniform_cube(1000, seed=1)
    fmm = FastMultipoleMethod(softening=1e-3)
    st = fmm.prepare_state(pos, mass, leaf_size=16, max_order=4)
    out = fmm.evaluate_prepared_state(st, target_indices=np.zeros(0, np.int32))
    assert out.shape == (0, 3)
    with pytest.raises(IndexError):
        fmm.evaluate_prepared_state(st, target_indices=np.array([1000], np.int32))


@pytest.mark.parametrize("p", [1, 10])
def test_extreme_orders_match_the_oracle(p):
    pos, mass = workloads.plummer(8000, seed=2)
    fmm = FastMultipoleMethod(theta=0.6, softening=0.0)
    st = fmm.prepare_state(pos, mass, leaf_size=16, max_order=p)
    acc = fmm.evaluate_prepared_state(st)
    ref = _oracle(st, pos, mass, p, 0.0)
    err = workloads.relative_errors(acc, ref)
    assert np.percentile(err, 99) <= 1e-5, np.percentile(err, [50, 99, 100])

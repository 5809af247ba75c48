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


# The reference's frozen facade surface (jaccpot tests/unit/test_public_api_surface.py:51-99):
# the keyword-only constructor arguments and the public method set.
FROZEN_INIT_KWARGS = {
    "preset", "basis", "m2l_impl", "adaptive_order", "p_gears", "use_pallas", "reuse_topology", "rebuild_every",
    "mac_force_scale_mode", "mac_force_scale_prepass_theta", "mac_force_scale_fb_inflation",
    "adaptive_error_model", "adaptive_eps", "dehnen_geometry_mode", "mac_theta_max", "theta", "G", "softening",
    "precision", "working_dtype", "advanced",
}
FROZEN_PUBLIC_METHODS = {
    "clear_prepared_state_cache", "clear_runtime_caches", "compute_accelerations", "compute_accelerations_and_jerk",
    "compute_accelerations_with_time_derivatives", "differentiable_accelerations", "differentiable_step_fn",
    "evaluate_prepared_state", "evaluate_prepared_state_with_jerk", "evaluate_prepared_state_with_time_derivatives",
    "export_m2l_autotune_cache", "get_runtime_diagnostics", "import_m2l_autotune_cache", "load_m2l_autotune_cache",
    "prepare_state", "prepare_upward_sweep", "rebuild_topology_in_place", "refresh_prepared_state",
    "save_m2l_autotune_cache", "strict_fused_prepared_eval_fn", "strict_prepare_refresh_and_evaluate",
    "strict_run_segmented", "strict_run_v2", "update_multipoles_only",
}


def test_constructor_surface_is_the_frozen_one():
    import inspect

    sig = inspect.signature(FastMultipoleMethod.__init__)
    kwargs = {n for n, p in sig.parameters.items() if n != "self" and p.kind is inspect.Parameter.KEYWORD_ONLY}
    assert kwargs == FROZEN_INIT_KWARGS


def test_public_method_set_is_the_frozen_one():
    import inspect

    methods = {n for n, _ in inspect.getmembers(FastMultipoleMethod, predicate=inspect.isfunction)
               if not n.startswith("_")}
    assert methods == FROZEN_PUBLIC_METHODS


def test_every_frozen_keyword_is_accepted_with_its_default():
    f = FastMultipoleMethod(reuse_topology=False, rebuild_every=1, mac_force_scale_mode="prev",
                            mac_force_scale_prepass_theta=None, mac_force_scale_fb_inflation=1.0,
                            adaptive_error_model="tail_proxy", adaptive_eps=None, dehnen_geometry_mode="com",
                            mac_theta_max=1.0, working_dtype=None, advanced=None)
    assert f.rebuild_every == 1 and f.mac_theta_max == 1.0 and f.adaptive_error_model == "tail_proxy"
    f = FastMultipoleMethod(reuse_topology=True, rebuild_every=4, adaptive_error_model="dehnen_paper",
                            adaptive_eps=3e-5, mac_theta_max=0.8, mac_force_scale_mode="paper",
                            mac_force_scale_prepass_theta=0.5, working_dtype="float32")
    assert f.reuse_topology and f.rebuild_every == 4 and f.adaptive_eps == 3e-5


@pytest.mark.parametrize("kw", [{"rebuild_every": 0}, {"mac_force_scale_mode": "bogus"},
                                {"mac_force_scale_mode": "paper_fb"}, {"mac_force_scale_prepass_theta": 1.5},
                                {"mac_force_scale_fb_inflation": -1.0}, {"adaptive_error_model": "bogus"},
                                {"adaptive_eps": 0.0}, {"dehnen_geometry_mode": "exact"},
                                {"dehnen_geometry_mode": "bogus"}, {"mac_theta_max": 0.0},
                                {"mac_theta_max": 1.5}, {"working_dtype": "float64"}])
def test_frozen_keywords_are_validated(kw):
    with pytest.raises(ValueError):
        FastMultipoleMethod(**kw)


def test_extension_options_through_advanced_or_keywords():
    f = FastMultipoleMethod(advanced={"nearfield_compensated": True, "device": "cuda:0"})
    assert f.p2p_mode == 1 and str(f.device) == "cuda:0"
    f = FastMultipoleMethod(nearfield_compensated=True)
    assert f.p2p_mode == 1
    with pytest.raises(TypeError):
        FastMultipoleMethod(advanced={"nonsense": 1})


def test_prepare_state_rejects_unknown_and_unsupported_keywords():
    import numpy as np

    f = FastMultipoleMethod()
    with pytest.raises(TypeError):
        f.prepare_state(np.zeros((5, 3)), np.ones(5), nonsense=1)
    with pytest.raises(ValueError):
        f.prepare_state(np.zeros((5, 3)), np.ones(5), runtime_overrides_override=object())


def test_out_of_scope_methods_say_so():
    f = FastMultipoleMethod()
    for name in ("compute_accelerations_and_jerk", "compute_accelerations_with_time_derivatives",
                 "evaluate_prepared_state_with_jerk", "evaluate_prepared_state_with_time_derivatives"):
        with pytest.raises(ValueError, match="not provided"):
            getattr(f, name)(None)


def test_autotune_cache_round_trip(tmp_path):
    f = FastMultipoleMethod()
    assert f.export_m2l_autotune_cache() == []
    path = tmp_path / "cache.json"
    assert f.save_m2l_autotune_cache(str(path)) == 0
    assert f.load_m2l_autotune_cache(str(path)) == 0
    with pytest.raises(ValueError):
        f.import_m2l_autotune_cache({"not": "a list"})
    d = f.get_runtime_diagnostics()
    assert d["prepare_state"] == 0 and not d["has_last_state"]
    f.clear_runtime_caches(clear_jax_compilation=True)


def test_strict_run_v2_requires_refresh_every_one():
    import numpy as np

    f = FastMultipoleMethod()
    with pytest.raises(ValueError, match="refresh_every=1"):
        f.strict_run_v2(state=np.zeros((4, 2, 3)), masses=np.ones(4), dt=0.1, num_steps=2, refresh_every=2,
                        leaf_size=8, max_order=4)


def test_error_monitor_options():
    assert FastMultipoleMethod().error_monitor is None
    f = FastMultipoleMethod(advanced={"error_monitor": 64})
    assert f.error_monitor == {"targets": 64, "every": 1, "bound": 1e-4, "seed": 0, "keep": 1000}
    f = FastMultipoleMethod(error_monitor={"targets": 8, "every": 5, "bound": 2e-4})
    assert (f.error_monitor["every"], f.error_monitor["bound"]) == (5, 2e-4)
    assert f.error_history == [] and "last_error_check" not in f.get_runtime_diagnostics()
    with pytest.raises(ValueError):
        FastMultipoleMethod(advanced={"error_monitor": {"targets": 0}})
    with pytest.raises(TypeError):
        FastMultipoleMethod(advanced={"error_monitor": {"sample": 3}})
    with pytest.raises(TypeError):
        FastMultipoleMethod(advanced={"error_monitor": "often"})

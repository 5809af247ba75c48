"""``FastMultipoleMethod`` facade with the reference's public signature.

Mirrors jaccpot/solver.py:540-1400 (``FastMultipoleMethod.__init__`` :664,
``compute_accelerations`` :917, ``prepare_state`` :1012,
``evaluate_prepared_state`` :1292) for the real basis.  ``prepare_state``
builds the tree and lists on the host (the yggdrax stand-in) and runs the
upward and downward sweeps on the GPU; ``evaluate_prepared_state`` runs L2P +
P2P for all particles or for ``target_indices`` -- the same split of work the
reference makes (runtime/fmm_prepare.py:3742 / runtime/fmm_evaluate.py:325).

Arrays may be numpy or torch; results come back as the same kind (torch
results stay on the GPU).  Everything runs on CUDA: there is no CPU path.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Any, Optional, Sequence

import numpy as np
import torch

from . import _lib
from .engine import DeviceTopology, Pass
from .tree import Topology, build_topology

# Preset defaults: (theta, leaf_size hint); solver.py:27-118 + config.py presets.
_PRESETS = {"fast": 0.6, "balanced": 0.6, "accurate": 0.5, "large_n_gpu": 0.6}
_M2L_IMPLS = {None: _lib.JB_M2L_FP32, "rot_scale": _lib.JB_M2L_FP32, "fp32": _lib.JB_M2L_FP32,
              "split_bf16": _lib.JB_M2L_SPLIT_BF16, "tcgen05": _lib.JB_M2L_SPLIT_BF16}


@dataclass
class FMMPreparedState:
    """What the reference's FMMPreparedState (runtime/fmm_state.py:870-897)
    carries, resident on the GPU: topology + lists, centres, multipoles and
    locals, the Morton permutation and the run parameters."""

    topology: Topology
    device_topology: DeviceTopology
    pass_: Pass
    max_order: int
    theta: float
    leaf_size: int
    num_particles: int
    input_dtype: Any
    scratch: dict = None

    def __post_init__(self):
        if self.scratch is None:
            self.scratch = {}

    @property
    def inverse_permutation(self) -> np.ndarray:
        return self.topology.inverse_permutation

    @property
    def max_leaf_size(self) -> int:
        return self.topology.max_leaf_occupancy


def _to_torch(a, device, dtype) -> torch.Tensor:
    if isinstance(a, torch.Tensor):
        return a.to(device=device, dtype=dtype)
    return torch.as_tensor(np.asarray(a), dtype=dtype, device=device)


_ADAPTIVE_MODELS = ("tail_proxy", "dehnen_degree", "dehnen_paper")
_FORCE_SCALE_MODES = ("prev", "prepass", "paper", "paper_cached", "paper_fb", "paper_fb_cached")
_GEOMETRY_MODES = ("com", "exact", "tree", "tree_approx", "runtime")
# Options of this implementation that the reference's constructor does not
# have; they are taken from ``advanced`` (a dict or an object with these
# attributes) or as extra keywords, like the reference's legacy keywords.
_EXTENSIONS = {"device": "cuda", "nearfield_compensated": False, "gear_model": None, "error_monitor": None,
               "cuda_graph": False}


def _monitor_config(cfg) -> Optional[dict]:
    """error_monitor: None (off), an int (targets per check), or a dict with
    targets (default 256), every (check every k-th whole-pass evaluation,
    default 1), bound (p99 relative error a check is judged against, default
    1e-4), seed (default 0), keep (checks kept, default 1000)."""
    if cfg is None or cfg is False:
        return None
    if isinstance(cfg, (int, np.integer)) and not isinstance(cfg, bool):
        cfg = {"targets": int(cfg)}
    if not isinstance(cfg, dict):
        raise TypeError("error_monitor must be None, an int or a dict")
    unknown = sorted(set(cfg) - {"targets", "every", "bound", "seed", "keep"})
    if unknown:
        raise TypeError(f"unknown error_monitor options: {unknown}")
    out = {"targets": int(cfg.get("targets", 256)), "every": int(cfg.get("every", 1)),
           "bound": float(cfg.get("bound", 1e-4)), "seed": int(cfg.get("seed", 0)), "keep": int(cfg.get("keep", 1000))}
    if out["targets"] < 1 or out["every"] < 1 or out["keep"] < 1 or not out["bound"] > 0.0:
        raise ValueError("error_monitor: targets, every and keep must be >= 1 and bound > 0")
    return out


def _advanced_options(advanced, legacy: dict) -> dict:
    out = dict(_EXTENSIONS)
    if advanced is not None:
        for k in _EXTENSIONS:
            if isinstance(advanced, dict):
                if k in advanced:
                    out[k] = advanced[k]
            elif hasattr(advanced, k):
                out[k] = getattr(advanced, k)
        if isinstance(advanced, dict):
            unknown = sorted(set(advanced) - set(_EXTENSIONS))
            if unknown:
                raise TypeError(f"unknown advanced options: {unknown}")
    for k in list(legacy):
        if k in _EXTENSIONS:
            out[k] = legacy.pop(k)
    if legacy:
        raise TypeError(f"unexpected keyword arguments: {sorted(legacy)}")
    return out


class FastMultipoleMethod:
    """Real-basis FMM on one B200 behind jaccpot's public API.

    The keyword-only constructor surface and the public method set are the
    reference's frozen ones (jaccpot tests/unit/test_public_api_surface.py:
    51-99).  Options outside the real-basis evaluation path raise ValueError
    with the reason; see each method."""

    def __init__(
        self,
        *,
        preset: str = "fast",
        basis: str = "real",
        m2l_impl: Optional[str] = None,
        adaptive_order: bool = False,
        p_gears: Optional[Sequence[int]] = None,
        use_pallas: Optional[bool] = None,
        reuse_topology: bool = False,
        rebuild_every: int = 1,
        mac_force_scale_mode: str = "prev",
        mac_force_scale_prepass_theta: Optional[float] = None,
        mac_force_scale_fb_inflation: float = 1.0,
        adaptive_error_model: str = "tail_proxy",
        adaptive_eps: Optional[float] = None,
        dehnen_geometry_mode: str = "com",
        mac_theta_max: float = 1.0,
        theta: float = 0.6,
        G: float = 1.0,
        softening: float = 1e-3,
        precision: Optional[str] = None,
        working_dtype: Any = None,
        advanced: Any = None,
        **legacy_kwargs: Any,
    ):
        ext = _advanced_options(advanced, dict(legacy_kwargs))
        preset = str(getattr(preset, "value", preset)).lower()
        if preset not in _PRESETS:
            raise ValueError(f"unknown preset {preset!r}")
        basis = str(basis).lower()
        if basis != "real":
            raise ValueError(f"basis {basis!r} is not provided: this implementation covers the real basis only")
        if precision not in (None, "fp32"):
            raise ValueError("only fp32 evaluation is provided on the GPU (precision='fp64' is not built)")
        if working_dtype is not None and np.dtype(str(working_dtype).replace("torch.", "")) != np.float32:
            raise ValueError("working_dtype must be float32 (the kernels compute in FP32)")
        if m2l_impl not in _M2L_IMPLS:
            raise ValueError(f"unknown m2l_impl {m2l_impl!r}")
        if use_pallas:
            raise ValueError("use_pallas is not available: the kernels are native sm_100a CUDA")
        if not (0.0 < float(theta) < 1.0):
            raise ValueError("theta must be in (0, 1)")
        if int(rebuild_every) < 1:
            raise ValueError("rebuild_every must be positive")
        fsm = str(mac_force_scale_mode).strip().lower()
        if fsm not in _FORCE_SCALE_MODES:
            raise ValueError(f"mac_force_scale_mode must be one of {_FORCE_SCALE_MODES}")
        if fsm.startswith("paper_fb"):
            raise ValueError("the eq. (16b) f_b force scale (mac_force_scale_mode='paper_fb*') is not provided; "
                             "use 'prev', 'prepass', 'paper' or 'paper_cached' (the |a| scale of eq. (16a))")
        if mac_force_scale_prepass_theta is not None and not (0.0 < float(mac_force_scale_prepass_theta) < 1.0):
            raise ValueError("mac_force_scale_prepass_theta must be in (0, 1)")
        if float(mac_force_scale_fb_inflation) < 0.0:
            raise ValueError("mac_force_scale_fb_inflation must be >= 0")
        model = str(adaptive_error_model).strip().lower()
        if model not in _ADAPTIVE_MODELS:
            raise ValueError(f"adaptive_error_model must be one of {_ADAPTIVE_MODELS}")
        geom = str(dehnen_geometry_mode).strip().lower()
        if geom not in _GEOMETRY_MODES:
            raise ValueError(f"dehnen_geometry_mode must be one of {_GEOMETRY_MODES}")
        if geom != "com":
            raise ValueError(f"dehnen_geometry_mode={geom!r} is not provided: the walk measures radii about the "
                             "expansion centres ('com')")
        if not (0.0 < float(mac_theta_max) <= 1.0):
            raise ValueError("mac_theta_max must be in (0, 1]")
        if adaptive_eps is not None and not (float(adaptive_eps) > 0.0):
            raise ValueError("adaptive_eps must be > 0 when provided")
        self.preset = preset
        self.basis = basis
        self.theta = float(theta)
        self.G = float(G)
        self.softening = float(softening)
        self.precision = precision
        self.m2l_mode = _M2L_IMPLS[m2l_impl]
        self.p2p_mode = _lib.JB_P2P_KAHAN if ext["nearfield_compensated"] else _lib.JB_P2P_FP32
        self.adaptive_order = bool(adaptive_order)
        self.p_gears = tuple(int(g) for g in p_gears) if p_gears is not None else None
        if self.p_gears is not None and (not self.p_gears or min(self.p_gears) < 1):
            raise ValueError("p_gears must hold positive orders")
        self.gear_model = ext["gear_model"]
        self.reuse_topology = bool(reuse_topology)
        self.rebuild_every = int(rebuild_every)
        self.mac_force_scale_mode = fsm
        self.mac_force_scale_prepass_theta = (None if mac_force_scale_prepass_theta is None
                                              else float(mac_force_scale_prepass_theta))
        self.mac_force_scale_fb_inflation = float(mac_force_scale_fb_inflation)
        self.adaptive_error_model = model
        self.adaptive_eps = None if adaptive_eps is None else float(adaptive_eps)
        self.dehnen_geometry_mode = geom
        self.mac_theta_max = float(mac_theta_max)
        self.device = torch.device(ext["device"])
        self._last_state: Optional[FMMPreparedState] = None
        self._reuse = None  # (state, calls since its prepare) of reuse_topology
        self._force_scale_cache = None  # per-particle |a| of the last evaluation (input order)
        self._counters = {"prepare_state": 0, "evaluate": 0, "reuse_hits": 0, "reuse_rebuilds": 0,
                          "adaptive_prepares": 0, "force_scale_prepasses": 0, "force_scale_reused": 0}
        # sampled FP64 direct-sum checks of whole-pass evaluations (off by default)
        self.error_monitor = _monitor_config(ext["error_monitor"])
        # whole re-evaluations (differentiable_accelerations without gradients)
        # replay a CUDA graph captured once per prepared state
        self.cuda_graph = bool(ext["cuda_graph"])
        self.error_history: list = []
        self._monitor_calls = 0

    # ------------------------------------------------------------------ prepare
    def _gear_orders(self, max_order: int) -> tuple:
        if self.adaptive_order and self.p_gears is not None:
            return tuple(sorted(set(self.p_gears)))
        return (int(max_order),)

    def prepare_state(self, positions, masses, *, bounds=None, leaf_size: int = 16, max_order: int = 4,
                      theta: Optional[float] = None, cache_policy: str = "auto", force_scale_nodes=None,
                      runtime_overrides_override=None, fused_device_mode: bool = False) -> FMMPreparedState:
        """Tree + lists (on the GPU), upward and downward sweeps (solver.py:1012
        there).  ``bounds`` is accepted and unused: the tree takes the particles'
        bounding cube.  ``cache_policy`` and ``fused_device_mode`` are accepted
        (the state is always device resident).  ``force_scale_nodes``: with
        ``adaptive_error_model="dehnen_paper"``, a per-particle force scale
        (shape (N,), input order) to use instead of the prepass."""
        if str(cache_policy) not in ("auto", "none", "reuse", "refresh"):
            raise ValueError(f"unknown cache_policy {cache_policy!r}")
        if runtime_overrides_override is not None:
            raise ValueError("runtime_overrides_override is not provided")
        th = self.theta if theta is None else float(theta)
        pos_np = positions.detach().cpu().numpy() if isinstance(positions, torch.Tensor) else np.asarray(positions)
        mass_np = masses.detach().cpu().numpy() if isinstance(masses, torch.Tensor) else np.asarray(masses)
        if pos_np.ndim != 2 or pos_np.shape[1] != 3 or mass_np.shape != (pos_np.shape[0],):
            raise ValueError("positions must be (N, 3) and masses (N,)")
        self._counters["prepare_state"] += 1
        if self.adaptive_error_model == "dehnen_paper":
            return self._prepare_adaptive(positions, masses, int(leaf_size), int(max_order), th, force_scale_nodes)
        if force_scale_nodes is not None:
            raise ValueError("force_scale_nodes applies to adaptive_error_model='dehnen_paper'")
        # tree + lists on the GPU when the solver runs there (the same arrays
        # as the host build, bit for bit), else on the host
        topo = build_topology(positions if isinstance(positions, torch.Tensor) else pos_np,
                              masses if isinstance(masses, torch.Tensor) else mass_np, leaf_size=int(leaf_size),
                              theta=th, device=self.device if self.device.type == "cuda" else None)
        return self._prepare_from_topology(topo, positions, masses, int(max_order), th, int(leaf_size))

    def _prepare_adaptive(self, positions, masses, leaf_size: int, max_order: int, th: float,
                          force_scale=None) -> FMMPreparedState:
        """Error-controlled walk (jaccpot_b200.adaptive): the reference's
        adaptive_error_model="dehnen_paper" lane with adaptive_eps,
        mac_theta_max and p_gears (runtime/_adaptive_policy.py:2216)."""
        from . import adaptive as _adaptive

        orders = self._gear_orders(max_order)
        if orders[-1] != int(max_order):
            raise ValueError(f"the top gear ({orders[-1]}) must equal max_order ({max_order})")
        # eps: the caller's, else the reference's theta-derived tolerance
        # theta^(p_max + 2) (_adaptive_policy.py:100-127)
        eps = self.adaptive_eps if self.adaptive_eps is not None else float(th) ** (orders[-1] + 2)
        pos = _to_torch(positions, self.device, torch.float32)
        mass = _to_torch(masses, self.device, torch.float32)
        if force_scale is None and self.mac_force_scale_mode in ("prev", "paper_cached"):
            c = self._force_scale_cache
            if c is not None and c.shape[0] == pos.shape[0]:
                force_scale = c
                self._counters["force_scale_reused"] += 1
        if force_scale is not None:
            force_scale = _to_torch(force_scale, self.device, torch.float32).reshape(-1)
            if force_scale.shape[0] != pos.shape[0]:
                raise ValueError("the force scale must be one value per particle (N,), input order")
        else:
            self._counters["force_scale_prepasses"] += 1
        prep = _adaptive.prepare(pos, mass, leaf_size=leaf_size, orders=orders, eps=eps,
                                 theta_max=self.mac_theta_max,
                                 theta_prepass=self.mac_force_scale_prepass_theta or th, G=self.G,
                                 eps2=self.softening ** 2, device=self.device, m2l_mode=self.m2l_mode,
                                 p2p_mode=self.p2p_mode, force_scale=force_scale)
        self._counters["adaptive_prepares"] += 1
        ps = prep.pass_
        ps.load_particles(pos, mass)
        ps.upward()
        ps.downward()
        ps.check_tc_status()
        st = FMMPreparedState(topology=prep.topology, device_topology=prep.device_topology, pass_=ps,
                              max_order=int(max_order), theta=th, leaf_size=int(leaf_size),
                              num_particles=int(prep.topology.num_particles),
                              input_dtype=positions.dtype if hasattr(positions, "dtype") else np.float64)
        st.scratch["adaptive"] = {"eps": eps, "orders": orders, "theta_max": self.mac_theta_max}
        self._last_state = st
        return st

    def _prepare_from_topology(self, topo: Topology, positions, masses, max_order: int, th: float,
                               leaf_size: int) -> FMMPreparedState:
        dt = DeviceTopology(topo, self.device)
        dt.validate()
        ps = Pass(dt, int(max_order), G=self.G, eps2=self.softening ** 2, m2l_mode=self.m2l_mode,
                  p2p_mode=self.p2p_mode)
        ps.load_particles(_to_torch(positions, self.device, torch.float32),
                          _to_torch(masses, self.device, torch.float32))
        if self.adaptive_order:
            # learned per-pair gears, chosen from a plain pass's force scale
            from . import gears as _gears

            model = self.gear_model if self.gear_model is not None else _gears.GearModel.load()
            if self.p_gears is not None and tuple(self.p_gears) != tuple(model.orders):
                raise ValueError(f"the gear model is trained for p_gears={model.orders}")
            _gears.apply_gears(ps, model)
        ps.upward()
        ps.downward()
        ps.check_tc_status()
        st = FMMPreparedState(topology=topo, device_topology=dt, pass_=ps, max_order=int(max_order), theta=th,
                              leaf_size=int(leaf_size), num_particles=int(topo.num_particles),
                              input_dtype=positions.dtype if hasattr(positions, "dtype") else np.float64)
        self._last_state = st
        return st

    # ------------------------------------------------------------------ refresh
    def refresh_prepared_state(self, prepared_state: FMMPreparedState, positions, masses, *, bounds=None,
                               leaf_size: Optional[int] = None, max_order: Optional[int] = None,
                               theta: Optional[float] = None, fused_device_mode: bool = False) -> FMMPreparedState:
        """Rebinds a prepared state to new particle data without a full prepare
        (solver.py:1604 / runtime/fmm_strict_run.py:54-200 there, whose fast path
        is _refresh_large_n_same_topology :1152).

        Same-topology fast path: the tree and lists of the new particles are
        built on the GPU and compared there with the state's (Morton order,
        node ranges, far and near lists).  When they are identical the state's
        work-unit schedules are reused and only the numeric payloads --
        particles, centres, multipoles, locals (and the gears, when adaptive)
        -- are recomputed, which gives exactly what ``prepare_state`` would.
        Otherwise, or when leaf_size / max_order / theta change, it is a full
        ``prepare_state``.  Returns a new state; the old one stays valid.
        ``refresh_stats`` counts attempts, hits and the reason of each miss.
        ``bounds`` and ``fused_device_mode`` are accepted for signature
        compatibility (the state is always device resident)."""
        from dataclasses import replace

        from .tree import DeviceTree

        st = prepared_state
        stats = self.__dict__.setdefault("refresh_stats", {"attempts": 0, "hits": 0, "miss_config": 0,
                                                             "miss_topology": 0})
        stats["attempts"] += 1
        leaf = st.leaf_size if leaf_size is None else int(leaf_size)
        order = st.max_order if max_order is None else int(max_order)
        th = st.theta if theta is None else float(theta)
        if (leaf, order, th) != (st.leaf_size, st.max_order, st.theta) or self.device.type != "cuda":
            stats["miss_config"] += 1
            return self.prepare_state(positions, masses, bounds=bounds, leaf_size=leaf, max_order=order, theta=th)
        if "adaptive" in st.scratch:
            # the error-controlled lists depend on the multipoles and the force
            # scale, not on the tree alone: a new walk every time
            stats["miss_adaptive"] = stats.get("miss_adaptive", 0) + 1
            return self.prepare_state(positions, masses, bounds=bounds, leaf_size=leaf, max_order=order, theta=th)
        dt = st.device_topology
        t = st.topology
        with DeviceTree(positions, masses, leaf_size=leaf, theta=th, device=self.device) as nt:
            i = nt.info
            same = (i.num_nodes, i.num_internal, i.num_far_pairs, i.num_near_pairs) == (
                t.num_nodes, t.num_internal, t.num_far_pairs, t.num_near_pairs)
            if same:
                same = (torch.equal(nt.field("permutation"), dt.perm)
                        and torch.equal(nt.field("node_ranges"), dt.node_ranges)
                        and torch.equal(nt.field("far_offsets"), dt.far_off)
                        and torch.equal(nt.field("near_offsets"), dt.near_off)
                        and (t.num_far_pairs == 0 or torch.equal(nt.field("far_sources"), dt.far_src))
                        and (t.num_near_pairs == 0 or torch.equal(nt.field("near_leaves"), dt.near_src)))
            if not same:
                stats["miss_topology"] += 1
                topo = nt.topology()
            else:
                centers = nt.field("centers_f64").reshape(-1, 3).cpu().numpy()
                radii = nt.field("radii_f64").cpu().numpy()
        if not same:
            return self._prepare_from_topology(topo, positions, masses, order, th, leaf)
        stats["hits"] += 1
        ps = st.pass_.fork()
        ps.load_particles(_to_torch(positions, self.device, torch.float32),
                          _to_torch(masses, self.device, torch.float32))
        if self.adaptive_order:
            from . import gears as _gears

            model = self.gear_model if self.gear_model is not None else _gears.GearModel.load()
            _gears.apply_gears(ps, model)
        ps.upward()
        ps.downward()
        new = FMMPreparedState(topology=replace(t, centers_f64=centers, radii_f64=radii), device_topology=dt,
                               pass_=ps, max_order=st.max_order, theta=st.theta, leaf_size=st.leaf_size,
                               num_particles=st.num_particles,
                               input_dtype=positions.dtype if hasattr(positions, "dtype") else np.float64)
        self._last_state = new
        return new

    def strict_prepare_refresh_and_evaluate(self, prepared_state: Optional[FMMPreparedState], positions, masses, *,
                                            bounds=None, leaf_size: int = 16, max_order: int = 4,
                                            theta: Optional[float] = None, jit_traversal=True):
        """Prepare when ``prepared_state`` is None, refresh it otherwise, then
        evaluate every particle (solver.py:1664 there): a time-stepping loop
        calls this unconditionally.  Returns (state, accelerations)."""
        if prepared_state is None:
            st = self.prepare_state(positions, masses, bounds=bounds, leaf_size=leaf_size, max_order=max_order,
                                    theta=theta)
        else:
            st = self.refresh_prepared_state(prepared_state, positions, masses, bounds=bounds,
                                             leaf_size=leaf_size, max_order=max_order, theta=theta)
        return st, self.evaluate_prepared_state(st, as_numpy=not isinstance(positions, torch.Tensor))

    # ----------------------------------------------------------------- evaluate
    def evaluate_prepared_state(self, state: FMMPreparedState, *, target_indices=None,
                                return_potential: bool = False, jit_traversal=None,
                                max_acc_derivative_order: int = 0, as_numpy: Optional[bool] = None):
        if max_acc_derivative_order:
            raise ValueError("acceleration derivative towers are not provided")
        ps = state.pass_
        dev = state.device_topology.device
        want_np = as_numpy if as_numpy is not None else not isinstance(target_indices, torch.Tensor)
        if target_indices is None:
            ps.evaluate(potential=return_potential)
            acc = torch.empty((state.num_particles, 3), device=dev, dtype=torch.float32)
            pot = torch.empty((state.num_particles,), device=dev, dtype=torch.float32) if return_potential else None
            ps.unsort(acc, pot)
        else:
            ti = _to_torch(target_indices, dev, torch.int64).reshape(-1)
            if ti.numel() and (int(ti.min()) < 0 or int(ti.max()) >= state.num_particles):
                raise IndexError("target_indices out of range")
            inv = torch.from_numpy(state.topology.inverse_permutation).to(dev)
            ts = inv[ti].to(torch.int32)
            out = ps.evaluate_targets(ts)
            acc = out[:, :3].contiguous()
            pot = out[:, 3].contiguous() if return_potential else None
        self._counters["evaluate"] += 1
        if target_indices is None:
            self._monitor_check(state)
        if (target_indices is None and self.adaptive_error_model == "dehnen_paper"
                and self.mac_force_scale_mode in ("prev", "paper_cached")):
            # the next error-controlled prepare takes its force scale from here
            self._force_scale_cache = torch.linalg.vector_norm(acc, dim=1)
        if want_np:
            acc = acc.cpu().numpy()
            pot = pot.cpu().numpy() if pot is not None else None
        return (acc, pot) if return_potential else acc

    def differentiable_accelerations(self, state: FMMPreparedState, positions, masses, *, target_indices=None,
                                     jit_traversal: bool = False, grad_plan=None, grad_config=None, out=None):
        """Re-evaluates the whole pass (P2M -> M2M -> M2L -> L2L -> L2P + P2P) on
        live positions/masses with the topology of `state` held fixed
        (runtime/fmm_evaluate.py:733, :542-731).  When either input is a torch
        tensor that requires grad, the result is differentiable: its backward
        runs the hand-written adjoint kernels (jaccpot_b200.autodiff).  Host inputs are copied to the
        device and the result copied back (into `out` when given, which may be
        a pinned host tensor); device inputs give a device result."""
        if target_indices is not None:
            # all particles stay sources; the result is gathered at the targets
            full = self.differentiable_accelerations(state, positions, masses, jit_traversal=jit_traversal,
                                                     grad_plan=grad_plan, grad_config=grad_config)
            ti = torch.as_tensor(np.asarray(target_indices) if not isinstance(target_indices, torch.Tensor)
                                 else target_indices).to(device=full.device, dtype=torch.int64).reshape(-1)
            if ti.numel() and (int(ti.min()) < 0 or int(ti.max()) >= state.num_particles):
                raise IndexError("target_indices out of range")
            sub = full[ti]
            if out is not None:
                out.copy_(sub)
                return out
            return sub
        ps = state.pass_
        dev = state.device_topology.device
        if (isinstance(positions, torch.Tensor) and positions.requires_grad) or (
                isinstance(masses, torch.Tensor) and masses.requires_grad):
            from .autodiff import fmm_accelerations

            pos = positions if isinstance(positions, torch.Tensor) else _to_torch(positions, dev, torch.float32)
            mass = masses if isinstance(masses, torch.Tensor) else _to_torch(masses, dev, torch.float32)
            return fmm_accelerations(pos.to(dev), mass.to(dev), ps)
        host = not (isinstance(positions, torch.Tensor) and positions.is_cuda)
        pos = _to_torch(positions, dev, torch.float32) if not isinstance(positions, torch.Tensor) else positions
        mass = _to_torch(masses, dev, torch.float32) if not isinstance(masses, torch.Tensor) else masses
        if self.cuda_graph:
            return self._replay(state, pos, mass, host, out)
        if host:
            if state.scratch.get("pos") is None:
                state.scratch["pos"] = torch.empty((state.num_particles, 3), device=dev, dtype=torch.float32)
                state.scratch["mass"] = torch.empty((state.num_particles,), device=dev, dtype=torch.float32)
                state.scratch["acc"] = torch.empty((state.num_particles, 3), device=dev, dtype=torch.float32)
            state.scratch["pos"].copy_(pos, non_blocking=True)
            state.scratch["mass"].copy_(mass, non_blocking=True)
            pos, mass = state.scratch["pos"], state.scratch["mass"]
            acc = state.scratch["acc"]
        else:
            acc = torch.empty((state.num_particles, 3), device=dev, dtype=torch.float32)
        ps.load_particles(pos, mass)
        ps.run()
        ps.unsort(acc, None)
        self._monitor_check(state)
        if not host:
            return acc
        if out is None:
            return acc.cpu()
        out.copy_(acc, non_blocking=True)
        return out

    def compute_accelerations(self, positions, masses, *, target_indices=None, bounds=None, leaf_size: int = 16,
                              max_order: int = 4, return_potential: bool = False, theta: Optional[float] = None,
                              reuse_prepared_state: bool = False, max_acc_derivative_order: int = 0):
        """Prepare + evaluate (solver.py:917 there).  With ``reuse_topology``
        (or ``reuse_prepared_state``) the tree and lists of an earlier call are
        kept for ``rebuild_every`` calls in all: the later calls re-evaluate the
        whole pass on the new particles with that topology held fixed (centres
        and expansions recomputed, lists unchanged), which trades accuracy for
        speed as the particles drift."""
        if max_acc_derivative_order:
            raise ValueError("acceleration derivative towers are not provided")
        as_np = not isinstance(positions, torch.Tensor)
        th = self.theta if theta is None else float(theta)
        key = (int(leaf_size), int(max_order), th)
        if self.reuse_topology or reuse_prepared_state:
            r = self._reuse
            n = int(positions.shape[0])
            if r is not None and r["key"] == key and r["state"].num_particles == n and r["calls"] < self.rebuild_every:
                r["calls"] += 1
                self._counters["reuse_hits"] += 1
                st = r["state"]
                pos = _to_torch(positions, self.device, torch.float32)
                mass = _to_torch(masses, self.device, torch.float32)
                st.pass_.load_particles(pos, mass)
                st.pass_.upward()
                st.pass_.downward()
                return self.evaluate_prepared_state(st, target_indices=target_indices,
                                                    return_potential=return_potential, as_numpy=as_np)
            st = self.prepare_state(positions, masses, bounds=bounds, leaf_size=leaf_size, max_order=max_order,
                                    theta=theta)
            self._reuse = {"state": st, "calls": 1, "key": key}
            self._counters["reuse_rebuilds"] += 1
        else:
            st = self.prepare_state(positions, masses, bounds=bounds, leaf_size=leaf_size, max_order=max_order,
                                    theta=theta)
        return self.evaluate_prepared_state(st, target_indices=target_indices, return_potential=return_potential,
                                            as_numpy=as_np)

    # ------------------------------------------------------- derivative towers
    _TOWERS = ("time derivatives of the acceleration (jerk and higher) are not provided: this implementation "
               "covers the acceleration pass only")

    def compute_accelerations_and_jerk(self, *args, **kwargs):
        """Not provided (solver.py:1085 there): raises ValueError."""
        raise ValueError(self._TOWERS)

    def compute_accelerations_with_time_derivatives(self, *args, **kwargs):
        """Not provided (solver.py:1182 there): raises ValueError."""
        raise ValueError(self._TOWERS)

    def evaluate_prepared_state_with_jerk(self, *args, **kwargs):
        """Not provided (solver.py:1493 there): raises ValueError."""
        raise ValueError(self._TOWERS)

    def evaluate_prepared_state_with_time_derivatives(self, *args, **kwargs):
        """Not provided (solver.py:1551 there): raises ValueError."""
        raise ValueError(self._TOWERS)

    # ----------------------------------------------------- engine-level seams
    def prepare_upward_sweep(self, tree, positions_sorted, masses_sorted, *, max_order: int = 4) -> dict:
        """P2M + M2M on a prebuilt tree (solver.py:1254 there): ``tree`` is a
        :class:`~jaccpot_b200.tree.Topology` and the particles are in its sort
        order.  Returns device tensors {"centers": (nodes, 4) COM + mass,
        "multipoles": (nodes, (p+1)^2)}."""
        if not isinstance(tree, Topology):
            raise TypeError("tree must be a jaccpot_b200.tree.Topology")
        dt = DeviceTopology(tree, self.device)
        ps = Pass(dt, int(max_order), G=self.G, eps2=self.softening ** 2)
        inv = torch.from_numpy(tree.inverse_permutation).to(self.device)
        pos = _to_torch(positions_sorted, self.device, torch.float32)[inv]
        mass = _to_torch(masses_sorted, self.device, torch.float32)[inv]
        ps.load_particles(pos, mass)
        ps.upward()
        C = (int(max_order) + 1) ** 2
        return {"centers": ps.ws.centers.clone(), "multipoles": ps.ws.mult[:, :C].clone()}

    def differentiable_step_fn(self, state: FMMPreparedState, *, target_indices=None, grad_config=None,
                               jit_traversal: bool = False, compile_now=None):
        """``f(positions, masses) -> accelerations`` on the fixed topology of
        ``state`` (solver.py:1430 there), differentiable through the
        hand-written adjoint when its inputs require grad.  There is nothing to
        compile; ``compile_now`` runs one warm-up evaluation."""
        def step(positions, masses):
            return self.differentiable_accelerations(state, positions, masses, target_indices=target_indices,
                                                     grad_config=grad_config)

        if compile_now is not None:
            step(*compile_now)
        return step

    def update_multipoles_only(self, prepared_state: FMMPreparedState, positions, masses, *,
                               leaf_size: Optional[int] = None, max_order: Optional[int] = None,
                               theta: Optional[float] = None) -> FMMPreparedState:
        """refresh_prepared_state under its own counter (solver.py:1952 there)."""
        self._counters["update_multipoles_only"] = self._counters.get("update_multipoles_only", 0) + 1
        return self.refresh_prepared_state(prepared_state, positions, masses, leaf_size=leaf_size,
                                           max_order=max_order, theta=theta)

    def rebuild_topology_in_place(self, prepared_state: FMMPreparedState, positions, masses, *, bounds=None,
                                  leaf_size: Optional[int] = None, max_order: Optional[int] = None,
                                  theta: Optional[float] = None) -> FMMPreparedState:
        """refresh_prepared_state under its own counter (solver.py:1998 there);
        returns a new state."""
        self._counters["rebuild_topology_in_place"] = self._counters.get("rebuild_topology_in_place", 0) + 1
        return self.refresh_prepared_state(prepared_state, positions, masses, bounds=bounds, leaf_size=leaf_size,
                                           max_order=max_order, theta=theta)

    def strict_fused_prepared_eval_fn(self, *, positions, masses, leaf_size: int, max_order: int,
                                      theta: Optional[float] = None):
        """``(state, eval_fn)``: eval_fn(state) evaluates the prepared state
        alone, no refresh or integration (solver.py:1908 there); the result
        stays on the device."""
        st = self.prepare_state(positions, masses, leaf_size=leaf_size, max_order=max_order, theta=theta)

        def eval_fn(state: FMMPreparedState):
            return self.evaluate_prepared_state(state, as_numpy=False)

        return st, eval_fn

    # ------------------------------------------------------------ time loops
    def strict_run_segmented(self, *, state, masses, num_steps: int, refresh_every: int, segment_runner,
                             positions_getter, prepared_state: Optional[FMMPreparedState] = None,
                             leaf_size: int = 16, max_order: int = 4, theta: Optional[float] = None,
                             jit_traversal=True, rematerialize_fn=None, collect_history: bool = False):
        """Segmented refresh cadence with a caller-provided segment kernel
        (solver.py:1720 / runtime/fmm_strict_run.py:415 there): ``num_steps``
        cut into segments of ``refresh_every`` (plus a tail); at each boundary
        the prepared state is refreshed at ``positions_getter(state)`` and the
        accelerations evaluated; ``segment_runner(state, accelerations,
        steps)`` advances the caller's state.  Returns (state, prepared_state,
        history or None)."""
        if int(num_steps) <= 0 or int(refresh_every) <= 0:
            raise ValueError("num_steps and refresh_every must be positive")
        hist = [] if collect_history else None
        done = 0
        while done < int(num_steps):
            k = min(int(refresh_every), int(num_steps) - done)
            pos = positions_getter(state)
            prepared_state, acc = self.strict_prepare_refresh_and_evaluate(
                prepared_state, pos, masses, leaf_size=leaf_size, max_order=max_order, theta=theta)
            state, out = segment_runner(state, acc, k)
            if hist is not None:
                hist.append(out)
            if rematerialize_fn is not None:
                state = rematerialize_fn(state)
            done += k
        return state, prepared_state, hist

    def strict_run_v2(self, *, state, masses, dt: float, num_steps: int, refresh_every: int, leaf_size: int,
                      max_order: int, theta: Optional[float] = None,
                      prepared_state: Optional[FMMPreparedState] = None, initial_self_acceleration=None,
                      jit_traversal=True, add_external: bool = False, external_acceleration_fn=None,
                      rematerialize_between_refresh: bool = True, return_history: bool = False,
                      return_prepared_state: bool = True, step_callback=None, step_callback_stride: int = 1):
        """Endpoint-correct velocity Verlet on the GPU (solver.py:1803 /
        runtime/fmm_strict_run.py:552 there).  ``state`` is (N, 2, 3):
        positions and velocities.  Every step: half kick, drift, refresh of the
        prepared state at the new positions (the same-topology fast path when
        the tree and lists did not change), self-gravity, half kick.  As in the
        reference ``refresh_every`` must be 1.  The state stays on the device;
        ``step_callback(step, state)`` runs every ``step_callback_stride``
        steps.  Returns (final_state, prepared_state or None, history or None)."""
        if int(num_steps) <= 0:
            raise ValueError("num_steps must be positive")
        if int(refresh_every) != 1:
            raise ValueError("strict_run_v2 requires refresh_every=1 for endpoint-correct velocity-Verlet self "
                             "gravity")
        if add_external and external_acceleration_fn is None:
            raise ValueError("add_external needs external_acceleration_fn")
        as_np = not isinstance(state, torch.Tensor)
        S = _to_torch(state, self.device, torch.float32).clone()
        if S.dim() != 3 or S.shape[1:] != (2, 3):
            raise ValueError("state must be (N, 2, 3): positions and velocities")
        m = _to_torch(masses, self.device, torch.float32)
        x, v = S[:, 0], S[:, 1]

        def accel(st):
            a = self.evaluate_prepared_state(st, as_numpy=False)
            if add_external:
                a = a + _to_torch(external_acceleration_fn(x), self.device, torch.float32)
            return a

        st = prepared_state
        if st is None:
            st = self.prepare_state(x, m, leaf_size=leaf_size, max_order=max_order, theta=theta)
        if initial_self_acceleration is not None:
            a = _to_torch(initial_self_acceleration, self.device, torch.float32)
            if add_external:
                a = a + _to_torch(external_acceleration_fn(x), self.device, torch.float32)
        else:
            st = self.refresh_prepared_state(st, x, m, leaf_size=leaf_size, max_order=max_order, theta=theta)
            a = accel(st)
        hist = [] if return_history else None
        h = float(dt)
        for i in range(int(num_steps)):
            v.add_(a, alpha=0.5 * h)
            x.add_(v, alpha=h)
            st = self.refresh_prepared_state(st, x, m, leaf_size=leaf_size, max_order=max_order, theta=theta)
            a = accel(st)
            v.add_(a, alpha=0.5 * h)
            if hist is not None:
                hist.append(S.clone())
            if step_callback is not None and (i + 1) % max(1, int(step_callback_stride)) == 0:
                step_callback(i + 1, S)
        history = torch.stack(hist) if hist is not None else None
        out = S.cpu().numpy() if as_np else S
        if history is not None and as_np:
            history = history.cpu().numpy()
        return out, (st if return_prepared_state else None), history

    def _replay(self, state: FMMPreparedState, pos, mass, host: bool, out):
        """differentiable_accelerations' whole re-evaluation through a CUDA
        graph of the step (Pass.capture), captured on the state's first call
        into fixed device buffers that later inputs are copied into."""
        sc = state.scratch
        if sc.get("graph") is None:
            dev = state.device_topology.device
            n = state.num_particles
            sc["g_pos"] = torch.empty((n, 3), device=dev, dtype=torch.float32)
            sc["g_mass"] = torch.empty((n,), device=dev, dtype=torch.float32)
            sc["g_acc"] = torch.empty((n, 3), device=dev, dtype=torch.float32)
            sc["g_pos"].copy_(pos)
            sc["g_mass"].copy_(mass)
            sc["graph"] = state.pass_.capture(sc["g_pos"], sc["g_mass"], sc["g_acc"])
            self._counters["graph_captures"] = self._counters.get("graph_captures", 0) + 1
        sc["g_pos"].copy_(pos, non_blocking=True)
        sc["g_mass"].copy_(mass, non_blocking=True)
        sc["graph"].replay()
        self._counters["graph_replays"] = self._counters.get("graph_replays", 0) + 1
        self._monitor_check(state)
        acc = sc["g_acc"]
        if not host:
            return acc.clone()
        if out is None:
            return acc.cpu()
        out.copy_(acc, non_blocking=True)
        return out

    # ------------------------------------------------------------ error monitor
    def _monitor_check(self, state: FMMPreparedState) -> None:
        """One sampled check of the whole-pass evaluation just run on
        ``state`` (its sorted results are in the pass's acc4): an FP64 direct
        sum (jb_direct_f64, the same G and softening, self pair excluded) on
        ``targets`` random particles, their relative force errors summarised
        into ``error_history``.  Synchronises the stream."""
        m = self.error_monitor
        if m is None:
            return
        self._monitor_calls += 1
        if (self._monitor_calls - 1) % m["every"]:
            return
        ps = state.pass_
        n = state.num_particles
        dev = state.device_topology.device
        k = min(m["targets"], n)
        rng = np.random.default_rng((m["seed"], self._monitor_calls))
        ts = torch.from_numpy(rng.choice(n, size=k, replace=False).astype(np.int32)).to(dev)
        ref = torch.empty((k, 4), device=dev, dtype=torch.float64)
        stream = torch.cuda.current_stream(dev).cuda_stream
        _lib.check(_lib.lib().jb_direct_f64(n, ps.ws.pos4.data_ptr(), k, ts.data_ptr(), float(ps.G), float(ps.eps2),
                                            ref.data_ptr(), stream), "jb_direct_f64")
        got = ps.ws.acc4[ts.long(), :3].double()
        r = ref[:, :3]
        e = (torch.linalg.vector_norm(got - r, dim=1) / torch.linalg.vector_norm(r, dim=1).clamp_min(1e-300)).cpu()
        q = torch.quantile(e, torch.tensor([0.5, 0.99], dtype=torch.float64)).tolist()
        rec = {"evaluation": self._monitor_calls, "targets": k, "p50": q[0], "p99": q[1], "max": float(e.max()),
               "within_bound": q[1] <= m["bound"]}
        self.error_history.append(rec)
        del self.error_history[:-m["keep"]]
        self._counters["error_checks"] = self._counters.get("error_checks", 0) + 1
        if not rec["within_bound"]:
            self._counters["error_checks_over_bound"] = self._counters.get("error_checks_over_bound", 0) + 1

    # ------------------------------------------------------ caches, counters
    def get_runtime_diagnostics(self) -> dict:
        """Counters of this solver (solver.py:2049 there): prepares,
        evaluations, reuse hits, refresh statistics, adaptive prepares and
        force-scale prepasses.  Not a stable schema."""
        d = dict(self._counters)
        if self.error_history:
            d["last_error_check"] = dict(self.error_history[-1])
        d["refresh"] = dict(getattr(self, "refresh_stats", {}))
        d["has_last_state"] = self._last_state is not None
        return d

    def clear_prepared_state_cache(self) -> None:
        """Forgets the cached prepared states (the last state and the
        reuse_topology state)."""
        self._last_state = None
        self._reuse = None

    def clear_runtime_caches(self, *, clear_jax_compilation: bool = False) -> None:
        """Clears the prepared-state caches and the cached force scale;
        ``clear_jax_compilation`` is accepted (there is no JAX here)."""
        self.clear_prepared_state_cache()
        self._force_scale_cache = None

    # The reference autotunes its M2L chunking per shape and caches the
    # choices (solver.py:2081-2163 there).  The schedules here are sized by the
    # work-unit builders at prepare time, so there is nothing to tune: the
    # cache is always empty, and imported entries are validated and ignored.
    def export_m2l_autotune_cache(self) -> list:
        """An empty list: no M2L autotuning state exists here."""
        return []

    def import_m2l_autotune_cache(self, entries, *, overwrite: bool = True) -> int:
        """Validates ``entries`` (a list of dicts) and ignores them; returns 0."""
        if not isinstance(entries, (list, tuple)) or not all(isinstance(e, dict) for e in entries):
            raise ValueError("the M2L autotune cache must be a list of dicts")
        return 0

    def save_m2l_autotune_cache(self, path: str) -> int:
        """Writes the (empty) cache as JSON; returns the number of entries (0)."""
        import json

        with open(path, "w") as f:
            json.dump(self.export_m2l_autotune_cache(), f)
        return 0

    def load_m2l_autotune_cache(self, path: str, *, overwrite: bool = True) -> int:
        """Reads a cache file written by either implementation; returns 0."""
        import json

        with open(path) as f:
            return self.import_m2l_autotune_cache(json.load(f), overwrite=overwrite)


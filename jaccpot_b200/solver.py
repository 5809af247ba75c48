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


class FastMultipoleMethod:
    """Real-basis FMM on one B200 behind jaccpot's public API."""

    def __init__(
        self,
        *,
        preset: str = "fast",
        basis: str = "real",
        m2l_impl: Optional[str] = None,
        adaptive_order: bool = False,
        p_gears: Optional[Sequence[int]] = None,
        use_pallas: Optional[bool] = None,
        theta: float = 0.6,
        G: float = 1.0,
        softening: float = 1e-3,
        precision: Optional[str] = None,
        working_dtype: Any = None,
        nearfield_compensated: bool = False,
        device: str | torch.device = "cuda",
        advanced: Any = None,
        gear_model: Any = None,
        **legacy_kwargs: Any,
    ):
        legacy_gear_model = gear_model
        preset = str(getattr(preset, "value", preset)).lower()
        if preset not in _PRESETS:
            raise ValueError(f"unknown preset {preset!r}")
        basis = str(basis).lower()
        if basis != "real":
            raise ValueError(f"basis {basis!r} is not provided: this implementation covers the real basis only")
        if precision not in (None, "fp32"):
            raise ValueError("only fp32 evaluation is provided on the GPU")
        if m2l_impl not in _M2L_IMPLS:
            raise ValueError(f"unknown m2l_impl {m2l_impl!r}")
        if use_pallas:
            raise ValueError("use_pallas is not available: the kernels are native sm_100a CUDA")
        if legacy_kwargs:
            raise TypeError(f"unexpected keyword arguments: {sorted(legacy_kwargs)}")
        if not (0.0 < float(theta) < 1.0):
            raise ValueError("theta must be in (0, 1)")
        self.preset = preset
        self.basis = basis
        self.theta = float(theta)
        self.G = float(G)
        self.softening = float(softening)
        self.m2l_mode = _M2L_IMPLS[m2l_impl]
        self.p2p_mode = _lib.JB_P2P_KAHAN if nearfield_compensated else _lib.JB_P2P_FP32
        self.adaptive_order = bool(adaptive_order)
        self.p_gears = tuple(p_gears) if p_gears is not None else None
        self.gear_model = legacy_gear_model
        if self.adaptive_order and self.p_gears is not None and max(self.p_gears) < 1:
            raise ValueError("p_gears must hold positive orders")
        self.device = torch.device(device)
        self._last_state: Optional[FMMPreparedState] = None

    # ------------------------------------------------------------------ prepare
    def prepare_state(self, positions, masses, *, bounds=None, leaf_size: int = 16, max_order: int = 4,
                      theta: Optional[float] = None, **_ignored) -> FMMPreparedState:
        th = self.theta if theta is None else float(theta)
        pos_np = positions.detach().cpu().numpy() if isinstance(positions, torch.Tensor) else np.asarray(positions)
        mass_np = masses.detach().cpu().numpy() if isinstance(masses, torch.Tensor) else np.asarray(masses)
        if pos_np.ndim != 2 or pos_np.shape[1] != 3 or mass_np.shape != (pos_np.shape[0],):
            raise ValueError("positions must be (N, 3) and masses (N,)")
        # tree + lists on the GPU when the solver runs there (the same arrays
        # as the host build, bit for bit), else on the host
        topo = build_topology(positions if isinstance(positions, torch.Tensor) else pos_np,
                              masses if isinstance(masses, torch.Tensor) else mass_np, leaf_size=int(leaf_size),
                              theta=th, device=self.device if self.device.type == "cuda" else None)
        return self._prepare_from_topology(topo, positions, masses, int(max_order), th, int(leaf_size))

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
            raise ValueError("target_indices is not provided on the fixed-topology path")
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
        if not host:
            return acc
        if out is None:
            return acc.cpu()
        out.copy_(acc, non_blocking=True)
        return out

    def compute_accelerations(self, positions, masses, *, target_indices=None, bounds=None, leaf_size: int = 16,
                              max_order: int = 4, return_potential: bool = False, theta: Optional[float] = None,
                              reuse_prepared_state: bool = False, max_acc_derivative_order: int = 0):
        st = self.prepare_state(positions, masses, bounds=bounds, leaf_size=leaf_size, max_order=max_order,
                                theta=theta)
        return self.evaluate_prepared_state(
            st, target_indices=target_indices, return_potential=return_potential,
            max_acc_derivative_order=max_acc_derivative_order,
            as_numpy=not isinstance(positions, torch.Tensor))

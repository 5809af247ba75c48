"""What the trained gear selector gains over the method without it (config
4, on a clustered system of a seed it never saw): against the plain
maximum-order pass on the same theta lists it saves M2L work while adding
little error; against the analytic selector (the Dehnen eq. (15) estimate at
the network's training budget, the per-pair order choice jaccpot itself
makes) it is compared at the same lists and budget."""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from jaccpot_b200 import engine, gears, tree, workloads  # noqa: E402


def _added(acc, plain):
    d = torch.linalg.vector_norm(acc - plain, dim=1) / torch.linalg.vector_norm(plain, dim=1).clamp_min(1e-30)
    return float(np.percentile(d.double().cpu().numpy(), 99))


def test_learned_selector_gain_on_an_unseen_seed():
    model = gears.GearModel.load()
    n = 262_144
    pos, mass = workloads.clustered(n, 300)
    topo = tree.build_topology(pos, mass, leaf_size=32, theta=0.58, device="cuda")
    ps = engine.Pass(engine.DeviceTopology(topo, "cuda"), 8)
    ps.load_particles(torch.from_numpy(pos).cuda(), torch.from_numpy(mass).cuda())
    plain = ps.run()[:, :3].clone()
    g = gears.apply_gears(ps, model)
    learned = ps.run()[:, :3].clone()
    flop_learned = gears.m2l_flop_fraction(g, model.orders)
    # the gain over the plain maximum order: at least 5% of the M2L work saved,
    # at an added p99 error a fifth of the 1e-4 budget at most
    assert flop_learned <= 0.95, flop_learned
    assert _added(learned, plain) <= 2e-5
    # the analytic estimate at the same budget on the same lists
    ps.set_gears(None, None)
    ps.run()
    ga = gears.analytic_gears(ps, model.budget, model.orders)
    ps.set_gears(ga, model.orders)
    analytic = ps.run()[:, :3].clone()
    flop_analytic = gears.m2l_flop_fraction(ga.cpu().numpy(), model.orders)
    assert _added(analytic, plain) <= 2e-5
    # measured: the two select about the same work at about the same added
    # error; the network does not lose more than 5 points against it
    assert flop_learned <= flop_analytic + 0.05, (flop_learned, flop_analytic)

"""Plans (tree built once, many evaluations) and batches of plans captured in
one CUDA graph, checked against the ordinary per-call entry points."""
import numpy as np
import pytest

import fmm2d_b200 as fmm
from conftest import rel_l2
from fmm2d_b200.plan import BatchGraph, Plan

pytestmark = pytest.mark.gpu


def _problem(rng, n, nd, kind="uniform"):
    import torch
    if kind == "uniform":
        src = rng.uniform(0, 1, (2, n))
    else:
        c = rng.uniform(0.25, 0.75, 2)
        src = c[:, None] + 10 ** rng.uniform(-3, -1) * rng.normal(size=(2, n))
    q = rng.normal(size=(nd, n)) + 1j * rng.normal(size=(nd, n))
    ts = torch.as_tensor(np.ascontiguousarray(src.T), device="cuda")
    tq = torch.as_tensor(np.ascontiguousarray(q.T), device="cuda")
    return src, q, ts, tq


@pytest.mark.parametrize("eps", [1e-6, 1e-9])
def test_plan_matches_cfmm2d_and_reevaluates(gpu, eps):
    rng = np.random.default_rng(1)
    src, q, ts, tq = _problem(rng, 30000, 2)
    plan = Plan("cfmm2d", eps=eps, sources=ts, charges=True, pg=2, nd=2)
    out = plan.eval(charges=tq)
    ref = fmm.cfmm2d(eps=eps, sources=src, charges=q, pg=2, nd=2)
    assert plan.status() == 0
    assert rel_l2(out["pot"].cpu().numpy().T, ref.pot) < 1e-12
    assert rel_l2(out["grad"].cpu().numpy().T, ref.grad) < 1e-12
    # new densities, same plan
    q2 = rng.normal(size=q.shape) + 1j * rng.normal(size=q.shape)
    import torch
    out2 = plan.eval(charges=torch.as_tensor(np.ascontiguousarray(q2.T), device="cuda"))
    ref2 = fmm.cfmm2d(eps=eps, sources=src, charges=q2, pg=2, nd=2)
    assert rel_l2(out2["pot"].cpu().numpy().T, ref2.pot) < 1e-12
    plan.close()


def test_plan_lfmm_dipoles_targets(gpu):
    import torch
    rng = np.random.default_rng(2)
    n, nt = 20000, 7000
    src = rng.uniform(0, 1, (2, n))
    trg = rng.uniform(-0.1, 1.1, (2, nt))
    q = rng.normal(size=n) + 1j * rng.normal(size=n)
    d = rng.normal(size=n) + 1j * rng.normal(size=n)
    v = rng.uniform(-1, 1, (2, n))
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")
    plan = Plan("lfmm2d", eps=1e-6, sources=dev(src.T), targets=dev(trg.T), charges=True,
                dipoles=True, pg=2, pgt=2)
    out = plan.eval(charges=dev(q.reshape(n, 1)), dipstr=dev(d.reshape(n, 1)),
                    dipvec=dev(v.T.reshape(n, 2, 1)))
    ref = fmm.lfmm2d(eps=1e-6, sources=src, charges=q, dipstr=d, dipvec=v, targets=trg, pg=2,
                     pgt=2)
    assert rel_l2(out["pot"][:, 0].cpu().numpy(), ref.pot) < 1e-12
    assert rel_l2(out["grad"][:, :, 0].cpu().numpy().T, ref.grad) < 1e-12
    assert rel_l2(out["pottarg"][:, 0].cpu().numpy(), ref.pottarg) < 1e-12
    assert rel_l2(out["gradtarg"][:, :, 0].cpu().numpy().T, ref.gradtarg) < 1e-12


def test_batch_graph_matches_individual_calls(gpu):
    """12 problems of uneven size and nd in one captured graph; a second launch
    after the densities changed in place gives the new results."""
    import torch
    rng = np.random.default_rng(3)
    probs = []
    for i in range(12):
        n = int(10 ** rng.uniform(np.log10(2000), np.log10(60000)))
        nd = [1, 2, 4][i % 3]
        probs.append(_problem(rng, n, nd, "uniform" if i % 2 else "gauss"))
    plans = [Plan("cfmm2d", eps=1e-6, sources=ts, charges=True, pg=1, nd=tq.shape[1])
             for _, _, ts, tq in probs]
    g = BatchGraph(plans, charges=[tq for _, _, _, tq in probs], nbranch=8)
    assert g.nodes > 0
    for step in range(2):
        if step == 1:
            for _, q, _, tq in probs:
                tq.mul_(-0.5)
                q *= -0.5
        g.launch()
        torch.cuda.synchronize()
        assert g.status() == 0
        for (src, q, _, tq), o in zip(probs, g.outs):
            nd = q.shape[0]
            ref = fmm.cfmm2d(eps=1e-6, sources=src, charges=q[0] if nd == 1 else q, pg=1, nd=nd)
            pot = o["pot"].cpu().numpy()
            ref_pot = ref.pot.reshape(q.shape[0], -1).T
            assert rel_l2(pot, ref_pot) < 1e-12
    g.close()
    for p in plans:
        p.close()

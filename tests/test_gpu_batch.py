"""Batching: problems of uneven size (mesh edges, source counts, density
contrasts; 19^3 is ragged, no axis a multiple of the 2x4x4 target blocks)
in one persistent launch, directly and as a replayed CUDA graph, under
every configuration the autotuner may pick.  Every problem's rates
must equal the problem run alone (march + EXACT_F32 rates) bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _workloads():
    from argot_b200 import workload as W
    rng = np.random.default_rng(12)
    out = []
    for i, (edge, nsrc) in enumerate([(16, 4), (24, 40), (32, 12), (20, 64), (40, 8), (28, 24), (19, 10)]):
        out.append(W._lognormal_ionized(f"b{i}", edge, nsrc, float(rng.uniform(0.5, 1.5)), 1e49, 1e51,
                                        100 + i))
    return out


@pytest.fixture(scope="module")
def solo(cuda_ok):
    import torch
    from argot_b200 import _lib as L
    from argot_b200.pipeline import Problem
    res = []
    for wl in _workloads():
        pb = Problem(wl)
        cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
        r = pb.run(L.PRECISION_KAHAN, L.RATE_EXACT_F32, crossings=cnt)
        torch.cuda.synchronize()
        res.append((r.view(6, -1).cpu().numpy().copy(), int(cnt.item())))
        pb.close()
    return res


@pytest.fixture(scope="module")
def batch(cuda_ok):
    from argot_b200.batch import Batch
    b = Batch(_workloads())
    yield b
    b.close()


def _check(batch, solo):
    import torch
    torch.cuda.synchronize()
    batch.check_device_error()
    for i, (want, _) in enumerate(solo):
        got = batch.rates[i].view(6, -1).cpu().numpy()
        assert np.array_equal(got, want), (i, np.abs(got - want).max())


def _clear(batch):
    for r in batch.rates:
        r.fill_(-1.0)


def test_batch_matches_solo_runs(batch, solo):
    import torch
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    _clear(batch)
    batch.run(cnt)
    _check(batch, solo)
    assert int(cnt.item()) == sum(c for _, c in solo)


_CFGS = [dict(warps_per_cta=4, ctas_per_sm=1, blocks_per_item=1, order=1, mode=0, parts=8),
         dict(warps_per_cta=8, ctas_per_sm=2, blocks_per_item=16, order=0, mode=0, parts=8),
         dict(warps_per_cta=4, ctas_per_sm=0, blocks_per_item=64, order=0, mode=0, parts=8),
         dict(warps_per_cta=8, ctas_per_sm=0, blocks_per_item=1, order=0, mode=1, parts=1),
         dict(warps_per_cta=8, ctas_per_sm=0, blocks_per_item=4, order=1, mode=1, parts=5),
         dict(warps_per_cta=8, ctas_per_sm=0, blocks_per_item=2, order=0, mode=1, parts=64)]


@pytest.mark.parametrize("cfg", _CFGS)
def test_batch_every_configuration(batch, solo, cfg):
    import torch
    batch.configure(**cfg)
    assert batch.config() == cfg
    _clear(batch)
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    batch.run(cnt)
    _check(batch, solo)
    assert int(cnt.item()) == sum(c for _, c in solo)


@pytest.mark.parametrize("mode", [0, 1])
def test_batch_graph_replay(batch, solo, mode):
    batch.configure(warps_per_cta=8, ctas_per_sm=0, blocks_per_item=4, order=0, mode=mode, parts=4)
    for _ in range(3):
        _clear(batch)
        batch.graph_launch()
        _check(batch, solo)


def test_batch_autotuner(batch, solo):
    cfg, ms = batch.tune(reps=1)
    assert ms > 0 and batch.config() == cfg
    _clear(batch)
    batch.graph_launch()
    _check(batch, solo)

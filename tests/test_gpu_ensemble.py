"""Batched ensemble (config 4): members of uneven sizes advanced together
must equal each member advanced alone by the plain kernel (same per-node
arithmetic: the results are identical), with and without the CUDA graph."""
import numpy as np
import pytest

from entropicthreadsafe_b200 import capi, ensemble, workloads
from entropicthreadsafe_b200.solver import Lattice

pytestmark = pytest.mark.gpu


def alone(dom, nsteps):
    nx, ny, nz = dom["dims"]
    with Lattice(dom["params"], nx, ny, nz) as lat:
        lat.upload_moments(dom["fields"])
        lat.step(nsteps)
        return lat.download()


def test_ensemble_equals_single_runs_with_graph_and_tuner():
    doms = ensemble.couette_droplets(n=5, seed=7)
    with ensemble.Ensemble([d["params"] for d in doms], [d["dims"] for d in doms]) as ens:
        for i, d in enumerate(doms):
            ens.upload_moments(i, d["fields"])
        zc, gr = ens.tune()
        # the persistent kernel: a resident grid
        assert zc > 0 and gr > 0
        # the tuner's table: 6 z chunks x 2 resident grids, the choice is the fastest row
        rows = ens.tune_results()
        assert len(rows) == 12 and all(r["ms"] > 0 and r["grid"] > 0 for r in rows)
        best = min(rows, key=lambda r: r["ms"])
        assert (best["zchunk"], best["grid"]) == (zc, gr)
        ens.step(3)                 # plain launches (odd count)
        ens.step_graph(4)           # graph replay
        ens.step_graph(4)
        out = [ens.download(i) for i in range(len(doms))]
    for i, d in enumerate(doms):
        ref = alone(d, 11)
        for k in capi.FIELDS:
            err = np.abs(out[i][k] - ref[k]).max() / max(np.abs(ref[k]).max(), 1e-30)
            assert err < 1e-6, (i, k, err)


@pytest.mark.parametrize("prec", [capi.PREC_BF16, capi.PREC_FP16S])
def test_16bit_ensemble_rounds_like_single_runs(prec):
    """16-bit members store with stochastic rounding seeded by the ensemble's
    device step counter, so plain launches, graph replays and a tuning pass
    (which restores the counter with the state) give the single lattices'
    results bit for bit."""
    doms = ensemble.couette_droplets(n=4, seed=11)
    for d in doms:
        d["params"].precision = prec
    with ensemble.Ensemble([d["params"] for d in doms], [d["dims"] for d in doms]) as ens:
        for i, d in enumerate(doms):
            ens.upload_moments(i, d["fields"])
        ens.tune()
        ens.step(3)
        ens.step_graph(4)
        ens.step_graph(4)
        out = [ens.download(i) for i in range(len(doms))]
    for i, d in enumerate(doms):
        ref = alone(d, 11)
        for k in capi.FIELDS:
            assert np.array_equal(out[i][k], ref[k]), (i, k, float(np.abs(out[i][k] - ref[k]).max()))


@pytest.mark.parametrize("grid", [0, 3, 296], ids=["per_item", "3_blocks", "2_per_sm"])
def test_every_launch_shape_equals_single_runs(grid):
    """A fixed z chunk and grid (set_launch): one block per work item, or
    resident blocks (3: many items each; 296: two per SM) taking the items
    from the work counter as they finish.  BF16 members, so the rounding's
    step counter must advance exactly once per launch in every shape."""
    doms = ensemble.couette_droplets(n=5, seed=13)
    for d in doms:
        d["params"].precision = capi.PREC_BF16
    with ensemble.Ensemble([d["params"] for d in doms], [d["dims"] for d in doms]) as ens:
        for i, d in enumerate(doms):
            ens.upload_moments(i, d["fields"])
        ens.set_launch(16, grid)
        ens.step(3)
        ens.step_graph(4)
        ens.step_graph(4)
        out = [ens.download(i) for i in range(len(doms))]
    for i, d in enumerate(doms):
        ref = alone(d, 11)
        for k in capi.FIELDS:
            assert np.array_equal(out[i][k], ref[k]), (i, k, float(np.abs(out[i][k] - ref[k]).max()))


def test_ensemble_mixed_shapes_phasefield_and_non_vector_width():
    params, dims, fields = [], [], []
    for n in (20, 24, 18):  # nx % 4 != 0 for 18: the ensemble falls back to scalar staging
        p = capi.make_params(mode=capi.MODE_PHASEFIELD, tau_a=0.7, sigma=0.01, sharp_c=0.9,
                             bc=[capi.BC_PERIODIC] * 4 + [capi.BC_BOUNCEBACK] * 2, bc_phi=[0.0] * 6)
        f = workloads.empty_fields(n, n + 2, n)
        z, y, x = np.meshgrid(np.arange(n), np.arange(n + 2), np.arange(n), indexing="ij")
        r = np.sqrt((x - n / 2) ** 2 + (y - n / 2) ** 2 + (z - n / 2) ** 2)
        f["phi"][:] = 0.5 * (1 + np.tanh((5 - r) / 1.5))
        params.append(p); dims.append((n, n + 2, n)); fields.append(f)
    with ensemble.Ensemble(params, dims) as ens:
        for i, f in enumerate(fields):
            ens.upload_moments(i, f)
        ens.step(6)
        out = [ens.download(i) for i in range(3)]
    for i in range(3):
        ref = alone(dict(params=params[i], dims=dims[i], fields=fields[i]), 6)
        for k in capi.FIELDS:
            err = np.abs(out[i][k] - ref[k]).max() / max(np.abs(ref[k]).max(), 1e-30)
            assert err < 1e-6, (i, k, err)


def test_deformation_of_sheared_droplet_grows():
    doms = ensemble.couette_droplets(n=1, seed=3)
    d = doms[0]
    d0 = ensemble.deformation(d["fields"]["phi"])
    out = alone(d, 1500)
    d1 = ensemble.deformation(out["phi"])
    assert d0 < 0.02 and d1 > d0 + 0.01

"""Batched form: many molecules in one persistent launch, FP32 arithmetic.

Compared with the dense FP64 path on the same molecules (which equals the
drop-in values and explicit gradients, see test_dense_adjoint.py): power
spectrum, dE/dpositions, energies and dE/dstrain of a linear model within
1e-4 of the largest magnitude, the stated error bound of the FP32 forms.
Graph replays are bit-identical, the launch configurations agree with each
other to 1e-5, and the autotuner keeps a valid configuration.
"""
import numpy as np
import pytest

import rascaline_b200 as rb
from rascaline_b200 import workloads

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

HYPERS = workloads.hypers(5.0, 7, 6)
SPECIES = [1, 6, 7, 8]


def molecules():
    mols = workloads.molecules(40, seed=4)
    # one molecule bigger than a warp of candidates and one lone atom
    mols += workloads.molecules(1, seed=9, min_atoms=70, max_atoms=70)
    mols.append(workloads.system_dict(np.array([8], dtype=np.int32), np.zeros((1, 3)), np.zeros((3, 3))))
    return mols


def flatten(mols):
    positions = np.concatenate([m["positions"] for m in mols])
    types = np.concatenate([m["types"] for m in mols]).astype(np.int32)
    sizes = np.array([len(m["types"]) for m in mols])
    return positions, types, sizes


def linear_model(n_keys, n_props, seed=12):
    rng = np.random.default_rng(seed)
    d = n_keys * n_props
    return rng.normal(0.0, 1.0 / np.sqrt(d), size=(len(SPECIES), n_keys, n_props))


def fp64_reference(calc, mols, W):
    from rascaline_b200.torch_api import dense_backward, dense_power_spectrum
    positions, types, sizes = flatten(mols)
    cells = np.zeros((len(mols), 9))
    pos = torch.as_tensor(positions, device="cuda")
    values, state = dense_power_spectrum(calc, pos, types, cells, sizes, 64, SPECIES)
    G = torch.as_tensor(W[np.searchsorted(SPECIES, types)], device="cuda")
    gpos, gstrain, _ = dense_backward(state, G, len(mols), strain=True, cell=False)
    per_atom = (values * G).sum(dim=(1, 2))
    system = torch.as_tensor(np.repeat(np.arange(len(mols)), sizes), device="cuda")
    energies = torch.zeros(len(mols), dtype=torch.float64, device="cuda").index_add_(0, system, per_atom)
    torch.cuda.synchronize()
    return {"values": values.cpu().numpy(), "gradients": gpos.cpu().numpy(), "energies": energies.cpu().numpy(),
            "strain": gstrain.cpu().numpy()}


def relative(actual, expected):
    actual = np.asarray(actual, dtype=np.float64)
    return float(np.max(np.abs(actual - expected)) / np.max(np.abs(expected)))


def host(out):
    torch.cuda.synchronize()
    return {k: v.double().cpu().numpy() for k, v in out.items()}


@pytest.fixture(scope="module")
def setup():
    from rascaline_b200.torch_api import Batch
    calc = rb.SoapPowerSpectrum(**HYPERS)
    mols = molecules()
    positions, types, sizes = flatten(mols)
    batch = Batch(calc, sizes, types, SPECIES)
    W = linear_model(batch.n_keys, batch.n_properties)
    ref = fp64_reference(calc, mols, W)
    pos = torch.as_tensor(positions, device="cuda")
    weights = torch.as_tensor(W, dtype=torch.float32, device="cuda").contiguous()
    return batch, pos, weights, ref, W, types


def test_batched_matches_fp64(setup):
    batch, pos, weights, ref, _, _ = setup
    out = batch.run(pos, batch.outputs(strain=True), weights=weights)
    assert batch.status() == 0
    got = host(out)
    for name in ("values", "gradients", "energies", "strain"):
        err = relative(got[name], ref[name])
        assert err <= 1e-4, (name, err)


def test_replays_are_deterministic_and_modes_agree(setup):
    batch, pos, weights, ref, W, types = setup
    out = batch.outputs(strain=True)
    first = host(batch.run(pos, out, weights=weights))
    second = host(batch.run(pos, out, weights=weights))
    for name in first:
        np.testing.assert_array_equal(first[name], second[name])
    # values only
    values_only = host(batch.run(pos, batch.outputs(gradients=False, energies=False)))
    np.testing.assert_array_equal(values_only["values"], first["values"])
    # the same loss given as dL/dP per atom
    G = torch.as_tensor(W[np.searchsorted(SPECIES, types)], dtype=torch.float32, device="cuda").contiguous()
    per_atom = host(batch.run(pos, batch.outputs(values=False, energies=False, strain=True), grad_values=G))
    np.testing.assert_array_equal(per_atom["gradients"], first["gradients"])
    np.testing.assert_array_equal(per_atom["strain"], first["strain"])


def test_configurations_agree_and_tuner_picks_one(setup):
    batch, pos, weights, ref, _, _ = setup
    results = []
    for config in ({"warps": 4, "chunk": 16, "layout": 0, "ctas_per_sm": 1, "pipeline": 0},
                   {"warps": 8, "chunk": 32, "layout": 1, "ctas_per_sm": 1, "pipeline": 0},
                   {"warps": 4, "chunk": 32, "layout": 1, "ctas_per_sm": 2, "pipeline": 0},
                   # the dense pipeline of the adjoint form
                   {"warps": 8, "chunk": 32, "layout": 1, "ctas_per_sm": 1, "pipeline": 1}):
        batch.config = config
        assert batch.config == config
        results.append(host(batch.run(pos, batch.outputs(), weights=weights)))
        assert batch.status() == 0
    for other in results[1:]:
        for name in ("values", "gradients", "energies"):
            assert relative(other[name], results[0][name]) <= 1e-5, name
    best = batch.tune(pos, batch.outputs(), weights=weights)
    assert np.isfinite(best) and best > 0
    config = batch.config
    assert config["warps"] in (4, 8) and config["chunk"] in (16, 32) and config["layout"] in (0, 1)
    assert config["pipeline"] in (0, 1)
    got = host(batch.run(pos, batch.outputs(), weights=weights))
    assert relative(got["gradients"], ref["gradients"]) <= 1e-4


def test_batch_rejects_unknown_species():
    from rascaline_b200.torch_api import Batch
    calc = rb.SoapPowerSpectrum(**HYPERS)
    with pytest.raises(rb.FeatomicError, match="not in the list of species"):
        Batch(calc, [2], [1, 9], species=[1, 8])

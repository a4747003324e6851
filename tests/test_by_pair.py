"""spherical_expansion_by_pair: featomic's SphericalExpansionByPair
(featomic/src/calculators/soap/spherical_expansion_pair.rs:547-822), one row
per pair and direction (plus the self pair i-i on l = 0), samples of
FullNeighborList (calculators/neighbor_list.rs:372-490).

CPU tests: registry name, parameters, and the oracle's by-pair output summing
to its spherical expansion (the reference's sums_to_spherical_expansion test,
spherical_expansion_pair.rs:983+).  GPU tests, through the C ABI: values and
positions / strain / cell gradients against the oracle at the 1e-10 relative
bound of the other parity tests, the same sum rule on the GPU output, and
finite differences of the positions gradients."""
import collections
import json

import numpy as np
import pytest

import rascaline_b200 as rb
from rascaline_b200 import workloads


def scaled_hypers(cutoff=5.0, max_radial=5, max_angular=2):
    # Willatt2018 scaling as in the reference's tests (spherical_expansion_pair.rs:870-886)
    h = workloads.hypers(cutoff, max_radial, max_angular)
    h["density"]["scaling"] = {"type": "Willatt2018", "scale": 1.5, "rate": 0.8, "exponent": 2.0}
    return h


def sum_over_pairs(by_pair):
    """{(l, first type, second type): {(system, first atom): sum of the rows}}"""
    out = {}
    for key, block in zip(by_pair["keys"], by_pair["blocks"]):
        acc = collections.defaultdict(lambda: 0.0)
        for sample, row in zip(block["samples"], block["values"]):
            acc[(int(sample[0]), int(sample[1]))] = acc[(int(sample[0]), int(sample[1]))] + row
        out[(int(key[0]), int(key[2]), int(key[3]))] = acc
    return out


def check_sums_to_expansion(by_pair, expansion):
    sums = sum_over_pairs(by_pair)
    assert len(by_pair["keys"]) == len(expansion["keys"])
    for key, block in zip(expansion["keys"], expansion["blocks"]):
        acc = sums[(int(key[0]), int(key[2]), int(key[3]))]
        scale = np.abs(block["values"]).max()
        for sample, row in zip(block["samples"], block["values"]):
            np.testing.assert_allclose(acc[(int(sample[0]), int(sample[1]))], row, rtol=1e-10, atol=1e-13 * scale)


def test_by_pair_metadata():
    calc = rb.SphericalExpansionByPair(**workloads.hypers(4.0, 3, 2))
    assert calc.name == "spherical expansion by pair"
    assert calc.cutoffs == [4.0]
    assert json.loads(calc.parameters) == workloads.hypers(4.0, 3, 2)
    # SphericalExpansionParameters has deny_unknown_fields
    h = workloads.hypers(4.0, 3, 2)
    h["comment"] = "rejected"
    with pytest.raises(rb.FeatomicError, match="unknown field `comment`"):
        rb.CalculatorBase("spherical_expansion_by_pair", h)


def test_oracle_by_pair_sums_to_spherical_expansion(oracle):
    systems = [workloads.random_box(40, density=0.1, species=(1, 8), seed=5), workloads.molecules(2, seed=3)[1]]
    h = scaled_hypers(4.5, 4, 3)
    by_pair = oracle.compute("spherical_expansion_by_pair", h, systems)
    expansion = oracle.compute("spherical_expansion", h, systems)
    check_sums_to_expansion(by_pair, expansion)


def test_oracle_by_pair_labels(oracle):
    system = workloads.random_box(30, density=0.1, species=(1, 8), seed=3)
    out = oracle.compute("spherical_expansion_by_pair", workloads.hypers(3.5, 3, 2), [system], ("positions",))
    keys = [tuple(k) for k in out["keys"]]
    types = sorted({(1, 1), (1, 8), (8, 1), (8, 8)})
    assert keys == [(l, 1, a, b) for a, b in types for l in range(3)]
    for key, block in zip(out["keys"], out["blocks"]):
        samples = block["samples"]
        is_self = (samples[:, 1] == samples[:, 2]) & (np.abs(samples[:, 3:]).sum(axis=1) == 0)
        assert is_self.any() == (key[0] == 0 and key[2] == key[3])
        grad = block["gradients"]["positions"]["samples"]
        expected = sum(0 if s else (1 if a == b else 2) for s, a, b in zip(is_self, samples[:, 1], samples[:, 2]))
        assert len(grad) == expected


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------
def _cases():
    return {
        "random_box_200": ([workloads.random_box(200, density=0.1, seed=9)], workloads.hypers(5.0, 5, 4)),
        "scaled_strained_box": ([workloads.random_box(120, strain=0.02, seed=7)], scaled_hypers(4.5, 4, 3)),
        "small_cell_images": ([workloads.system_dict([1, 8, 1], [[0.0, 0.0, 0.0], [1.1, 0.3, 0.2], [0.4, 1.6, 1.2]],
                                                     np.eye(3) * 3.2)], workloads.hypers(4.0, 3, 2)),
        "molecules": (workloads.molecules(3, seed=5, max_atoms=25), workloads.hypers(5.0, 5, 4)),
    }


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(_cases()))
def test_by_pair_matches_oracle(oracle, case):
    from test_gpu_parity import check_against_oracle
    systems, hypers = _cases()[case]
    periodic = all(np.abs(s["cell"]).sum() > 0 for s in systems)
    grads = ("positions", "strain", "cell") if periodic else ("positions",)
    product, _ = check_against_oracle(oracle, "spherical_expansion_by_pair", hypers, systems, grads)
    assert product["keys"].shape[1] == 4


@pytest.mark.gpu
def test_by_pair_sums_to_spherical_expansion_on_gpu():
    from test_gpu_parity import run_product
    systems = [workloads.random_box(80, density=0.1, seed=11), workloads.molecules(2, seed=6)[0]]
    h = scaled_hypers(5.0, 5, 3)
    check_sums_to_expansion(run_product("spherical_expansion_by_pair", h, systems),
                            run_product("spherical_expansion", h, systems))


@pytest.mark.gpu
def test_by_pair_user_neighbor_list(oracle):
    from test_gpu_parity import check_against_oracle
    # use_native_system = False: pairs come from the caller (here, the oracle's list)
    systems = [workloads.random_box(60, density=0.1, seed=13)]
    for s in systems:
        s["pairs"] = oracle.neighbors(s["positions"], s["cell"], 4.0)
    check_against_oracle(oracle, "spherical_expansion_by_pair", workloads.hypers(4.0, 3, 2), systems,
                         ("positions",), use_native_system=False)


@pytest.mark.gpu
def test_by_pair_finite_differences_positions():
    # displacement 1e-6, relative 1e-5 (spherical_expansion_pair.rs:889-900)
    from test_dense_adjoint import off_pole_box
    # no pair near the z axis, where featomic's Y_lm gradient is approximate
    calc = rb.SphericalExpansionByPair(**scaled_hypers(3.5, 3, 2))
    system = off_pole_box(3.5)
    h = 1e-6
    tm = calc.compute(rb.System.from_dict(system), gradients=["positions"])

    def values(positions):
        out = calc.compute(rb.System.from_dict(dict(system, positions=positions)))
        return {tuple(k): (b.samples.values, b.values.copy()) for k, b in zip(out.keys.values, out.blocks())}

    checked = 0
    for key, block in zip(tm.keys.values, tm.blocks()):
        g = block.gradient("positions")
        samples = block.samples.values
        for row, (sample, _, atom) in enumerate(g.samples.values[:6]):
            for x in range(3):
                plus, minus = system["positions"].copy(), system["positions"].copy()
                plus[atom, x] += h
                minus[atom, x] -= h
                sp, vp = values(plus)[tuple(key)]
                sm, vm = values(minus)[tuple(key)]
                target = tuple(samples[sample])
                ip = [tuple(s) for s in sp].index(target)
                im = [tuple(s) for s in sm].index(target)
                fd = (vp[ip] - vm[im]) / (2 * h)
                scale = max(np.abs(g.values[row, x]).max(), 1e-12)
                assert np.allclose(g.values[row, x], fd, rtol=1e-5, atol=1e-6 * scale), (tuple(key), target, x)
                checked += 1
        if checked > 40:
            break
    assert checked > 0

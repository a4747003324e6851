"""Samples / properties / keys selections (featomic/src/calculator.rs:20-158,
:287-310): the selected output equals the matching rows and columns of the
full output, gradients follow their samples, and the errors name what is
wrong.  The test recipe follows featomic's compute_partial
(featomic/src/calculators/tests_utils.rs)."""
import numpy as np
import pytest

import rascaline_b200 as rb
from rascaline_b200 import workloads

pytestmark = pytest.mark.gpu

GRADS = ["positions", "strain"]


def _system():
    return workloads.random_box(60, density=0.1, species=(1, 6, 8), seed=17, strain=0.01)


def _by_key(tm):
    return {tuple(k): b for k, b in zip(tm.keys.values, tm.blocks())}


def _check_block(full, part, rows, cols):
    np.testing.assert_array_equal(part.samples.values, full.samples.values[rows])
    np.testing.assert_array_equal(part.properties.values, full.properties.values[cols])
    np.testing.assert_array_equal(part.values, full.values[rows][..., cols])
    # positions rows of the kept samples, renumbered
    fg, pg = full.gradient("positions"), part.gradient("positions")
    expected, samples = [], []
    for new, old in enumerate(rows):
        for r in np.nonzero(fg.samples.values[:, 0] == old)[0]:
            expected.append(fg.values[r][..., cols])
            samples.append([new] + list(fg.samples.values[r, 1:]))
    np.testing.assert_array_equal(pg.samples.values.reshape(-1, 3), np.array(samples, dtype=np.int32).reshape(-1, 3))
    if expected:
        np.testing.assert_array_equal(pg.values, np.array(expected))
    sg = part.gradient("strain")
    np.testing.assert_array_equal(sg.values, full.gradient("strain").values[rows][..., cols])


@pytest.mark.parametrize("calculator", ["soap_power_spectrum", "spherical_expansion"])
def test_samples_and_properties_subsets(calculator):
    cls = {"soap_power_spectrum": rb.SoapPowerSpectrum, "spherical_expansion": rb.SphericalExpansion}[calculator]
    calc = cls(**workloads.hypers(4.5, 4, 3))
    system = rb.System.from_dict(_system())
    full = calc.compute(system, gradients=GRADS)
    samples = rb.Labels(["atom"], [[3], [0], [41], [17]])
    if calculator == "soap_power_spectrum":
        properties = rb.Labels(["l", "n_2"], [[0, 1], [2, 4], [3, 0]])
    else:
        properties = rb.Labels(["n"], [[4], [1]])
    part = calc.compute(system, gradients=GRADS, selected_samples=samples, selected_properties=properties)
    np.testing.assert_array_equal(part.keys.values, full.keys.values)
    for key, fb in _by_key(full).items():
        pb = _by_key(part)[key]
        rows = [r for r, s in enumerate(fb.samples.values) if s[1] in (3, 0, 41, 17)]
        sel = {tuple(v) for v in properties.values}
        names = properties.names
        cols = [c for c, p in enumerate(fb.properties.values)
                if tuple(p[fb.properties.names.index(n)] for n in names) in sel]
        _check_block(fb, pb, rows, cols)


def test_selected_keys():
    calc = rb.SoapPowerSpectrum(**workloads.hypers(4.5, 4, 3))
    system = rb.System.from_dict(_system())
    full = calc.compute(system, gradients=GRADS)
    # fewer names: the default keys with center_type 6
    part = calc.compute(system, gradients=GRADS, selected_keys=rb.Labels(["center_type"], [[6]]))
    assert all(k[0] == 6 for k in part.keys.values)
    assert len(part.keys) == sum(1 for k in full.keys.values if k[0] == 6)
    # all names: exactly these keys, in this order; (9, 1, 1) is not produced
    keys = rb.Labels(["center_type", "neighbor_1_type", "neighbor_2_type"], [[8, 1, 6], [9, 1, 1], [1, 1, 1]])
    part = calc.compute(system, gradients=GRADS, selected_keys=keys)
    np.testing.assert_array_equal(part.keys.values, keys.values)
    fb = _by_key(full)
    for key, pb in _by_key(part).items():
        if key == (9, 1, 1):
            assert pb.values.shape == (0, fb[(1, 1, 1)].values.shape[1])
            assert pb.gradient("positions").values.shape[0] == 0
        else:
            np.testing.assert_array_equal(pb.values, fb[key].values)


def test_missing_key_of_the_spherical_expansion_has_its_components():
    calc = rb.SphericalExpansion(**workloads.hypers(4.5, 4, 3))
    system = rb.System.from_dict(_system())
    keys = rb.Labels(["o3_lambda", "o3_sigma", "center_type", "neighbor_type"], [[2, 1, 9, 1], [1, 1, 1, 6]])
    part = calc.compute(system, gradients=GRADS, selected_keys=keys)
    block = part.block_by_id(0)
    assert block.values.shape == (0, 5, 5)
    assert block.gradient("positions").values.shape == (0, 3, 5, 5)
    with pytest.raises(rb.FeatomicError, match="max_angular"):
        calc.compute(system, selected_keys=rb.Labels(keys.names, [[7, 1, 1, 1]]))


def test_predefined_selection():
    calc = rb.SoapPowerSpectrum(**workloads.hypers(4.5, 4, 3))
    system = rb.System.from_dict(_system())
    full = calc.compute(system, gradients=GRADS)
    template = calc.compute(system, selected_samples=rb.Labels(["atom"], [[5], [2], [30]]),
                            selected_properties=rb.Labels(["l"], [[1]]))
    part = calc.compute(system, gradients=GRADS, selected_samples=template, selected_properties=template)
    for key, pb in _by_key(part).items():
        tb, fb = _by_key(template)[key], _by_key(full)[key]
        np.testing.assert_array_equal(pb.samples.values, tb.samples.values)
        np.testing.assert_array_equal(pb.properties.values, tb.properties.values)
        rows = [[tuple(s) for s in fb.samples.values].index(tuple(s)) for s in tb.samples.values]
        cols = [[tuple(p) for p in fb.properties.values].index(tuple(p)) for p in tb.properties.values]
        _check_block(fb, pb, rows, cols)


def test_selection_errors():
    calc = rb.SoapPowerSpectrum(**workloads.hypers(4.5, 4, 3))
    system = rb.System.from_dict(_system())
    with pytest.raises(rb.FeatomicError, match="'foo' in samples selection is not part of the samples"):
        calc.compute(system, selected_samples=rb.Labels(["foo"], [[0]]))
    with pytest.raises(rb.FeatomicError, match="'n' in properties selection is not part of the properties"):
        calc.compute(system, selected_properties=rb.Labels(["n"], [[0]]))
    with pytest.raises(rb.FeatomicError, match="selected keys can not be empty"):
        calc.compute(system, selected_keys=rb.Labels(["center_type"], np.zeros((0, 1))))

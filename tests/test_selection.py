"""Samples / properties / keys selections (featomic/src/calculator.rs:20-158,
:287-310) against the oracle's restatement of featomic's selection rules
(oracle/selection.py) applied to the oracle's full calculation.

Every case runs through featomic_calculator_compute (host output) and
featomic_b200_calculator_compute_device (device output, the selection applied
by a gather kernel on the device).  Labels (keys, samples, properties,
gradient samples) must be identical; values and gradients within the parity
bound |x - ref| <= 1e-10 |ref| + 1e-12 max|ref|.  Cases: subsets of samples
and properties (fewer names than the calculator's), keys with fewer names and
with all names (a key the systems do not produce gets an empty block),
predefined samples and properties, predefined samples the full calculation
does not produce (centres without neighbours of one of the key's types: zero
rows, with featomic's gradient samples), and the error messages."""
import numpy as np
import pytest

import rascaline_b200 as rb
from rascaline_b200 import workloads
from oracle import oracle
from oracle import selection as oracle_selection

pytestmark = pytest.mark.gpu

GRADS = ["positions", "strain", "cell"]
CUTOFF = 4.5


def _hypers(calculator):
    if calculator == "soap_radial_spectrum":
        return {"cutoff": {"radius": CUTOFF, "smoothing": {"type": "ShiftedCosine", "width": 0.5}},
                "density": {"type": "Gaussian", "width": 0.3},
                "basis": {"radial": {"type": "Gto", "max_radial": 4}}}
    return workloads.hypers(CUTOFF, 4, 3)


CLASSES = {"soap_power_spectrum": rb.SoapPowerSpectrum, "spherical_expansion": rb.SphericalExpansion,
           "soap_radial_spectrum": rb.SoapRadialSpectrum}


def _one_oxygen():
    # 59 H / C atoms and one O: most centres have no O neighbour, so the
    # blocks with an O neighbour type miss many centres
    box = workloads.random_box(60, density=0.1, species=(1, 6), seed=17, strain=0.01)
    box["types"] = np.array(box["types"], dtype=np.int32)
    box["types"][23] = 8
    return box


@pytest.fixture(scope="module")
def system():
    return _one_oxygen()


@pytest.fixture(scope="module")
def full_oracle(system):
    return {c: oracle.compute(c, _hypers(c), [system], GRADS, threads=4) for c in CLASSES}


def _ours(calculator, system, device, **selection):
    calc = CLASSES[calculator](**_hypers(calculator))
    if not device:
        tm = calc.compute(rb.System.from_dict(system), gradients=GRADS, **selection)
    else:
        import torch
        pos = torch.tensor(system["positions"], device="cuda")
        tm = calc.compute_device(pos, system["types"], np.asarray(system["cell"]).reshape(1, 9),
                                 [len(system["types"])], gradients=GRADS, **selection)
        torch.cuda.synchronize()
    return tm


def _close(a, b, what):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, (what, a.shape, b.shape)
    if b.size == 0:
        return
    bound = 1e-10 * np.abs(b) + 1e-12 * np.max(np.abs(b))
    assert np.all(np.abs(a - b) <= bound), (what, np.max(np.abs(a - b)))


def _compare(ours, ref):
    np.testing.assert_array_equal(ours.keys.values, ref["keys"])
    assert ours.keys.names == ref["key_names"]
    blocks = ours.blocks()
    assert len(blocks) == len(ref["blocks"])
    for block, rb_ in zip(blocks, ref["blocks"]):
        assert block.samples.names == rb_["sample_names"]
        assert block.properties.names == rb_["property_names"]
        np.testing.assert_array_equal(block.samples.values.reshape(-1, 2), rb_["samples"])
        np.testing.assert_array_equal(block.properties.values.reshape(rb_["properties"].shape), rb_["properties"])
        values = block.values
        values = values if isinstance(values, np.ndarray) else values.cpu().numpy()
        _close(values, rb_["values"], "values")
        for name in GRADS:
            g = block.gradient(name)
            gv = g.values if isinstance(g.values, np.ndarray) else g.values.cpu().numpy()
            width = rb_["gradients"][name]["samples"].shape[1]
            np.testing.assert_array_equal(g.samples.values.reshape(-1, width), rb_["gradients"][name]["samples"])
            _close(gv, rb_["gradients"][name]["values"], f"{name} gradients")


def _run(calculator, system, full_oracle, device, selection, oracle_args):
    ours = _ours(calculator, system, device, **selection)
    ref = oracle_selection.select(calculator, full_oracle[calculator], [system], CUTOFF, GRADS, **oracle_args)
    _compare(ours, ref)


DEVICE = [False, True]


@pytest.mark.parametrize("device", DEVICE, ids=["host", "device"])
@pytest.mark.parametrize("calculator", list(CLASSES))
def test_subsets(calculator, device, system, full_oracle):
    samples = (["atom"], [[3], [0], [41], [17], [23]])
    props = (["l", "n_2"], [[0, 1], [2, 4], [3, 0]]) if calculator == "soap_power_spectrum" else (["n"], [[4], [1]])
    _run(calculator, system, full_oracle, device,
         dict(selected_samples=rb.Labels(*samples), selected_properties=rb.Labels(*props)),
         dict(samples=("subset",) + samples, properties=("subset",) + props))


@pytest.mark.parametrize("device", DEVICE, ids=["host", "device"])
def test_keys(device, system, full_oracle):
    # fewer names: the default keys with center_type 6
    keys = (["center_type"], [[6]])
    _run("soap_power_spectrum", system, full_oracle, device, dict(selected_keys=rb.Labels(*keys)),
         dict(keys=keys))
    # all names: exactly these keys, in this order; (9, 1, 1) is not produced
    keys = (["center_type", "neighbor_1_type", "neighbor_2_type"], [[8, 1, 6], [9, 1, 1], [1, 1, 1]])
    _run("soap_power_spectrum", system, full_oracle, device, dict(selected_keys=rb.Labels(*keys)),
         dict(keys=keys))
    keys = (["o3_lambda", "o3_sigma", "center_type", "neighbor_type"], [[2, 1, 9, 1], [1, 1, 1, 6], [3, 1, 8, 8]])
    _run("spherical_expansion", system, full_oracle, device, dict(selected_keys=rb.Labels(*keys)),
         dict(keys=keys))


def _predefined_samples(calculator, full, key_rows, extra):
    """Per key: a few default samples in reverse order, plus `extra` samples
    (which the full calculation may not have) for the keys that accept them."""
    key_names = oracle_selection.KEY_NAMES[calculator]
    blocks = {}
    for key, block in zip(full["keys"], full["blocks"]):
        key = tuple(int(x) for x in key)
        rows = [tuple(int(x) for x in s) for s in block["samples"][::-7]]
        for s in extra.get(key, []):
            if s not in rows:
                rows.append(s)
        blocks[key] = (["system", "atom"], np.array(rows, dtype=np.int32).reshape(-1, 2))
    keys = [tuple(int(x) for x in k) for k in full["keys"]]
    tensor = rb.labels_tensormap(rb.Labels(key_names, keys), samples=[rb.Labels(*blocks[k]) for k in keys])
    return tensor, ("predefined", blocks, key_names)


def _centres_without(system, centre_type, neighbour_type):
    nl = oracle.neighbors(system["positions"], system["cell"], CUTOFF)
    types = system["types"]
    has = set()
    for i, j in zip(nl["first"], nl["second"]):
        if types[j] == neighbour_type:
            has.add(int(i))
        if types[i] == neighbour_type:
            has.add(int(j))
    return [a for a in range(len(types)) if types[a] == centre_type and a not in has]


@pytest.mark.parametrize("device", DEVICE, ids=["host", "device"])
@pytest.mark.parametrize("calculator", list(CLASSES))
def test_predefined_samples_with_absent_centres(calculator, device, system, full_oracle):
    full = full_oracle[calculator]
    lonely_h = _centres_without(system, 1, 8)[:4]
    lonely_c = _centres_without(system, 6, 8)[:3]
    assert len(lonely_h) == 4 and len(lonely_c) == 3
    extra = {}
    for key in full["keys"]:
        key = tuple(int(x) for x in key)
        if calculator == "soap_power_spectrum":
            centre, types = key[0], key[1:]
        else:
            centre, types = key[-2], key[-1:]
        if 8 in types:
            extra[key] = [(0, a) for a in (lonely_h if centre == 1 else lonely_c if centre == 6 else [])]
    assert any(extra.values())
    tensor, oracle_spec = _predefined_samples(calculator, full, None, extra)
    _run(calculator, system, full_oracle, device, dict(selected_samples=tensor), dict(samples=oracle_spec))


@pytest.mark.parametrize("device", DEVICE, ids=["host", "device"])
def test_predefined_properties(device, system, full_oracle):
    full = full_oracle["soap_power_spectrum"]
    key_names = oracle_selection.KEY_NAMES["soap_power_spectrum"]
    keys = [tuple(int(x) for x in k) for k in full["keys"]]
    blocks = {}
    for k, key in enumerate(keys):
        props = full["blocks"][k]["properties"][(k % 5)::9][::-1]
        blocks[key] = (["l", "n_1", "n_2"], props)
    tensor = rb.labels_tensormap(rb.Labels(key_names, keys), properties=[rb.Labels(*blocks[k]) for k in keys])
    _run("soap_power_spectrum", system, full_oracle, device, dict(selected_properties=tensor),
         dict(properties=("predefined", blocks, key_names)))


def test_errors(system, full_oracle):
    calc = rb.SoapPowerSpectrum(**_hypers("soap_power_spectrum"))
    s = rb.System.from_dict(system)
    with pytest.raises(rb.FeatomicError, match="'foo' in samples selection is not part of the samples"):
        calc.compute(s, selected_samples=rb.Labels(["foo"], [[0]]))
    with pytest.raises(rb.FeatomicError, match="'n' in properties selection is not part of the properties"):
        calc.compute(s, selected_properties=rb.Labels(["n"], [[0]]))
    with pytest.raises(rb.FeatomicError, match="selected keys can not be empty"):
        calc.compute(s, selected_keys=rb.Labels(["center_type"], np.zeros((0, 1))))
    # the oracle raises the same errors
    with pytest.raises(oracle_selection.SelectionError, match="'foo' in samples selection is not part of the samples"):
        oracle_selection.select("soap_power_spectrum", full_oracle["soap_power_spectrum"], [system], CUTOFF,
                                samples=("subset", ["foo"], [[0]]))
    full = full_oracle["soap_power_spectrum"]
    keys = [tuple(int(x) for x in k) for k in full["keys"]]
    key_names = oracle_selection.KEY_NAMES["soap_power_spectrum"]
    # a block missing from the predefined TensorMap
    tensor = rb.labels_tensormap(rb.Labels(key_names, keys[1:]),
                                 samples=[rb.Labels(["system", "atom"], [[0, 0]]) for _ in keys[1:]])
    printed = ", ".join(f"{n}={v}" for n, v in zip(key_names, keys[0]))
    with pytest.raises(rb.FeatomicError, match=rf"expected a block for \({printed}\) in predefined samples"):
        calc.compute(s, selected_samples=tensor)
    # wrong label names
    tensor = rb.labels_tensormap(rb.Labels(key_names, keys), samples=[rb.Labels(["atom"], [[0]]) for _ in keys])
    with pytest.raises(rb.FeatomicError, match=r"invalid predefined samples names: expected \[system, atom\]"):
        calc.compute(s, selected_samples=tensor)
    # a centre of another type than the key's center_type
    first_h = int(np.nonzero(system["types"] == 1)[0][0])
    tensor = rb.labels_tensormap(rb.Labels(key_names, keys),
                                 samples=[rb.Labels(["system", "atom"], [[0, first_h]]) for _ in keys])
    with pytest.raises(rb.FeatomicError, match="computes the atoms of the block's center_type only"):
        calc.compute(s, selected_samples=tensor)

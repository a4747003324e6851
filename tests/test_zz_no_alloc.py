"""featomic_b200_neighbor_list_noalloc against featomic_b200_neighbor_list.

The entry point without device allocation reads device positions and writes
the caller's device pair buffer.  Its pairs must equal those of the allocating
entry point on the same system field by field (tolerance: bit-exact, both run
the same arithmetic), on consecutive calls that reuse the same scratch array.
This file is collected last so that it also runs after the rest of the GPU
suite has used the device.
"""
import ctypes

import numpy as np
import pytest

import rascaline_b200 as rb
from rascaline_b200 import _c_api as C
from rascaline_b200 import workloads

pytestmark = pytest.mark.gpu

PAIR = np.dtype([("first", "<u8"), ("second", "<u8"), ("distance", "<f8"), ("vector", "<f8", (3,)),
                 ("shift", "<i4", (3,)), ("pad", "<i4")])
INVALID_PARAMETER = 1
BUFFER_SIZE_ERROR = 254


def _torch():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required")
    return torch


def call_noalloc(positions, cell, cutoff, capacity, stream):
    """Run the no-allocation neighbour list; returns (status, count, pairs as a
    structured numpy array of `capacity` entries)."""
    torch = _torch()
    pos = torch.as_tensor(np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)).cuda()
    out = torch.zeros(max(capacity, 1) * PAIR.itemsize, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    cell = np.ascontiguousarray(cell, dtype=np.float64).reshape(9)
    count = ctypes.c_size_t(12345)
    status = C.lib().featomic_b200_neighbor_list_noalloc(
        pos.data_ptr(), len(pos), cell.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), float(cutoff),
        out.data_ptr(), capacity, ctypes.byref(count), stream.cuda_stream)
    stream.synchronize()
    pairs = out.cpu().numpy().view(PAIR)[:capacity]
    return status, count.value, pairs


def systems():
    box = workloads.random_box(1000, density=0.1, min_distance=0.9, seed=2)
    lattice = workloads.sc_lattice(seed=1)
    rng = np.random.default_rng(7)
    triclinic = np.array([[3.0, 0.0, 0.0], [1.0, 3.2, 0.0], [0.5, 0.7, 3.4]])
    small = {"positions": rng.uniform(0.0, 1.0, (3, 3)) @ triclinic, "cell": triclinic}
    molecule = {"positions": rng.normal(0.0, 2.0, (40, 3)), "cell": np.zeros((3, 3))}
    return [
        ("box_1000", box["positions"], box["cell"], 5.5),
        ("triclinic_self_images", small["positions"], small["cell"], 5.0),
        ("lattice_216", lattice["positions"], lattice["cell"], 5.0),
        ("molecule_40", molecule["positions"], molecule["cell"], 4.0),
        ("box_1000_again", box["positions"], box["cell"], 5.5),
    ]


def test_matches_allocating_entry_point_on_consecutive_calls():
    torch = _torch()
    stream = torch.cuda.Stream()
    for name, positions, cell, cutoff in systems():
        expected = rb.neighbor_list(positions, cell, cutoff)
        n = len(expected["first"])
        assert n > 0, name
        status, count, pairs = call_noalloc(positions, cell, cutoff, n + 7, stream)
        assert status == 0, (name, C.lib().featomic_last_error())
        assert count == n, name
        got = pairs[:n]
        np.testing.assert_array_equal(got["first"].astype(np.int64), expected["first"], err_msg=name)
        np.testing.assert_array_equal(got["second"].astype(np.int64), expected["second"], err_msg=name)
        np.testing.assert_array_equal(got["shift"], expected["shift"], err_msg=name)
        np.testing.assert_array_equal(got["distance"], expected["distance"], err_msg=name)
        np.testing.assert_array_equal(got["vector"], expected["vector"], err_msg=name)
        # entries past the count are left untouched
        assert not pairs[n:].view(np.uint8).any(), name


def test_small_buffer_reports_the_count_and_writes_nothing():
    torch = _torch()
    stream = torch.cuda.Stream()
    box = workloads.random_box(1000, density=0.1, min_distance=0.9, seed=2)
    n = len(rb.neighbor_list(box["positions"], box["cell"], 5.5)["first"])
    status, count, pairs = call_noalloc(box["positions"], box["cell"], 5.5, 100, stream)
    assert status == BUFFER_SIZE_ERROR
    assert count == n
    assert not pairs.view(np.uint8).any()
    assert "too small" in C.lib().featomic_last_error().decode()


def test_sizes_beyond_the_limits_are_rejected():
    torch = _torch()
    stream = torch.cuda.Stream()
    rng = np.random.default_rng(11)
    # more atoms than the scratch array holds: rejected before any GPU work
    big = rng.uniform(0.0, 100.0, (65537, 3))
    status, count, _ = call_noalloc(big, np.eye(3) * 100.0, 5.0, 16, stream)
    assert status == INVALID_PARAMETER
    assert "65536 atoms" in C.lib().featomic_last_error().decode()
    # more than 2048 pairs for one atom (atom 0 keeps all its neighbours)
    dense = rng.uniform(0.0, 20.0, (8000, 3))
    status, count, pairs = call_noalloc(dense, np.eye(3) * 20.0, 8.0, 16, stream)
    assert status == INVALID_PARAMETER
    assert "2048 pairs per atom" in C.lib().featomic_last_error().decode()
    assert not pairs.view(np.uint8).any()


def test_calls_allocate_no_device_memory():
    """After the one-time set-up of the first call, calls leave the device's
    free memory (cudaMemGetInfo) unchanged, and the device's default memory
    pool records no allocation while they run, not even one freed before the
    call returns (its used-memory high watermark, reset before the calls,
    stays at the current use)."""
    torch = _torch()
    from cuda.bindings import driver
    from cuda.bindings import runtime as rt

    stream = torch.cuda.Stream()
    box = workloads.random_box(1000, density=0.1, min_distance=0.9, seed=2)
    n = len(rb.neighbor_list(box["positions"], box["cell"], 5.5)["first"])
    pos = torch.as_tensor(np.ascontiguousarray(box["positions"], dtype=np.float64)).cuda()
    out = torch.zeros(n * PAIR.itemsize, dtype=torch.uint8, device="cuda")
    cell = np.ascontiguousarray(box["cell"], dtype=np.float64).reshape(9)
    count = ctypes.c_size_t(0)

    def call():
        status = C.lib().featomic_b200_neighbor_list_noalloc(
            pos.data_ptr(), len(pos), cell.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 5.5,
            out.data_ptr(), n, ctypes.byref(count), stream.cuda_stream)
        assert status == 0, C.lib().featomic_last_error()
        assert count.value == n

    call()  # the first call on a device may do its one-time set-up
    torch.cuda.synchronize()
    err, pool = rt.cudaDeviceGetDefaultMemPool(torch.cuda.current_device())
    assert err == rt.cudaError_t.cudaSuccess
    high = rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemHigh
    current = rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent
    err, = rt.cudaMemPoolSetAttribute(pool, high, driver.cuuint64_t(0))  # resets the watermark to the current use
    assert err == rt.cudaError_t.cudaSuccess
    err, used_before = rt.cudaMemPoolGetAttribute(pool, current)
    free_before = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        call()
    stream.synchronize()
    free_after = torch.cuda.mem_get_info()[0]
    err, used_high = rt.cudaMemPoolGetAttribute(pool, high)
    assert free_after == free_before
    assert int(used_high) == int(used_before)

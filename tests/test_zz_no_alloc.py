"""tsr_samples_root_scope_noalloc through the C ABI, on the GPU.

The entry point computes the root scope of device-resident samples with a
fixed working array inside the library and no allocation.  These tests compare
it with the root scope of a tree that tsr_tree_build made from the same
samples (tolerance: none -- min/max reductions and correctly rounded
arithmetic must reproduce the build's scope bit for bit), on two calls in a
row, check that a call after set-up grows neither the device's memory use nor
its stream-ordered pool, and check the argument errors.

This file sorts last so that it also runs after every other GPU test in the
same process; it passes on its own too.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT_SCOPE_ATOL = 0.0   # bit-exact with tsr_tree_root_scope


def _torch():
    import torch
    return torch


def _random_samples(n, seed):
    from tsr_b200 import core
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-3.0, 5.0, (n, 3)) * np.array([1.0, 0.5, 2.0])
    nrm = rng.normal(size=(n, 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    scales = rng.uniform(1e-3, 2e-2, n)
    return core.Samples(pos, nrm, scales, np.ones(n), np.zeros((n, 1), np.uint32))


def _noalloc_scope(samples, params, out=None):
    """Calls the entry point on device copies of `samples`; returns the scope
    read back from the caller-owned device output."""
    from tsr_b200 import core
    torch = _torch()
    dev = torch.device("cuda", torch.cuda.current_device())
    pos = torch.from_numpy(samples.positions).to(dev)
    scales = torch.from_numpy(samples.scales).to(dev)
    if out is None:
        out = torch.full((4,), float("nan"), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream()
    rc = core.lib.tsr_samples_root_scope_noalloc(
        samples.count, ctypes.c_void_p(pos.data_ptr()), ctypes.c_void_p(scales.data_ptr()),
        ctypes.byref(params), ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
    assert rc == 0, core.lib.tsr_last_error_message().decode()
    torch.cuda.synchronize()
    return out.cpu().numpy().copy(), (pos, scales, out)


@pytest.mark.parametrize("case", ["sphere", "random_400k"])
def test_matches_tree_build_twice(case, tiny_scene):
    from tsr_b200 import core
    if case == "sphere":
        samples = core.Samples.from_scene(tiny_scene)
    else:
        # more blocks than the scratch holds partials for: the grid-stride loop runs
        samples = _random_samples(400_000, seed=7)
    params = core.params_default()
    expected = core.Tree(samples, params, reorder_samples=False).getRootScope()
    first, _ = _noalloc_scope(samples, params)
    second, _ = _noalloc_scope(samples, params)
    np.testing.assert_allclose(first, expected, rtol=0, atol=ROOT_SCOPE_ATOL)
    np.testing.assert_allclose(second, expected, rtol=0, atol=ROOT_SCOPE_ATOL)


def test_non_default_sampling_distance(tiny_scene):
    from tsr_b200 import core
    samples = core.Samples.from_scene(tiny_scene)
    params = core.make_params(h_svo=3.5)
    expected = core.Tree(samples, params, reorder_samples=False).getRootScope()
    got, _ = _noalloc_scope(samples, params)
    np.testing.assert_allclose(got, expected, rtol=0, atol=ROOT_SCOPE_ATOL)


def _root_scope_numpy(positions, scales, h_svo):
    """The build's root scope in numpy (IEEE double, correctly rounded like
    the device): the sample boxes' AABB (Samples.cpp:442-449) and the cube of
    its largest extent around its centre (Tree.cpp:70-101)."""
    r = scales * h_svo + 1e-6
    lo = (positions - r[:, None]).min(0)
    hi = (positions + r[:, None]).max(0)
    ext = hi - lo
    m = ext[1] if ext[0] < ext[1] else ext[0]
    size = ext[2] if m < ext[2] else m
    return np.concatenate([(lo + hi) * 0.5 - size * 0.5, [size]])


def test_negative_extent_follows_the_build_arithmetic():
    """Samples whose scales are negative (which only the tree build itself
    rejects) give boxes with negative extents; the entry point keeps the
    build's arithmetic for them (no clamp of the cube size at 0)."""
    from tsr_b200 import core
    rng = np.random.default_rng(11)
    n = 1000
    pos = rng.uniform(0.0, 0.1, (n, 3))
    samples = core.Samples(pos, np.tile([0.0, 0.0, 1.0], (n, 1)), np.full(n, -0.5), np.ones(n),
                           np.zeros((n, 1), np.uint32))
    params = core.params_default()
    got, _ = _noalloc_scope(samples, params)
    expected = _root_scope_numpy(samples.positions, samples.scales, 2.0)
    assert expected[3] < 0.0
    np.testing.assert_array_equal(got, expected)


def _default_pool_used_high():
    from cuda.bindings import driver as dr
    torch = _torch()
    err, dev = dr.cuDeviceGet(torch.cuda.current_device())
    assert err == dr.CUresult.CUDA_SUCCESS
    err, pool = dr.cuDeviceGetDefaultMemPool(dev)
    assert err == dr.CUresult.CUDA_SUCCESS
    return dr, pool


def test_allocates_nothing_after_setup():
    from tsr_b200 import core
    torch = _torch()
    samples = _random_samples(50_000, seed=3)
    params = core.params_default()
    _, keep = _noalloc_scope(samples, params)            # first call: per-device set-up
    pos, scales, out = keep
    stream = torch.cuda.current_stream()
    dr, pool = _default_pool_used_high()
    high = dr.CUmemPool_attribute.CU_MEMPOOL_ATTR_USED_MEM_HIGH
    cur = dr.CUmemPool_attribute.CU_MEMPOOL_ATTR_USED_MEM_CURRENT
    torch.cuda.synchronize()
    assert dr.cuMemPoolSetAttribute(pool, high, dr.cuuint64_t(0))[0] == dr.CUresult.CUDA_SUCCESS
    err, used_before = dr.cuMemPoolGetAttribute(pool, cur)
    assert err == dr.CUresult.CUDA_SUCCESS
    torch_before = torch.cuda.memory_stats().get("allocated_bytes.all.allocated", 0)
    for _ in range(2):
        rc = core.lib.tsr_samples_root_scope_noalloc(
            samples.count, ctypes.c_void_p(pos.data_ptr()), ctypes.c_void_p(scales.data_ptr()),
            ctypes.byref(params), ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, core.lib.tsr_last_error_message().decode()
    torch.cuda.synchronize()
    err, used_high = dr.cuMemPoolGetAttribute(pool, high)
    assert err == dr.CUresult.CUDA_SUCCESS
    assert int(used_high) <= int(used_before), "the call drew memory from the stream-ordered pool"
    # (the device's free memory is not compared: other threads, processes or
    # lazily loaded modules may change it between two reads)
    assert torch.cuda.memory_stats().get("allocated_bytes.all.allocated", 0) == torch_before


def test_argument_errors():
    from tsr_b200 import core
    torch = _torch()
    dev = torch.device("cuda", torch.cuda.current_device())
    params = core.params_default()
    pos = torch.zeros((8, 3), dtype=torch.float64, device=dev)
    scales = torch.full((8,), 0.01, dtype=torch.float64, device=dev)
    out = torch.zeros(4, dtype=torch.float64, device=dev)
    host_out = np.zeros(4)

    def call(n, p=pos.data_ptr(), s=scales.data_ptr(), o=out.data_ptr(), prm=params):
        return core.lib.tsr_samples_root_scope_noalloc(
            n, ctypes.c_void_p(p), ctypes.c_void_p(s), ctypes.byref(prm) if prm is not None else None,
            ctypes.c_void_p(o), None)

    assert core.STATUS[call(0)] == "TSR_ERR_INVALID_ARG"
    assert core.STATUS[call(1 << 31)] == "TSR_ERR_OVERFLOW_U32"
    assert "2^31 - 1" in core.lib.tsr_last_error_message().decode()
    assert core.STATUS[call(8, o=host_out.ctypes.data)] == "TSR_ERR_INVALID_ARG"
    assert "device" in core.lib.tsr_last_error_message().decode()
    assert core.STATUS[call(8, o=out.data_ptr() + 4)] == "TSR_ERR_INVALID_ARG"
    assert core.STATUS[call(8, prm=None)] == "TSR_ERR_INVALID_ARG"
    assert core.STATUS[call(8, prm=core.make_params(h_svo=0.0))] == "TSR_ERR_INVALID_ARG"
    assert core.STATUS[call(8, p=0)] == "TSR_ERR_INVALID_ARG"
    torch.cuda.synchronize()
    assert np.all(out.cpu().numpy() == 0.0), "a rejected call wrote the output"

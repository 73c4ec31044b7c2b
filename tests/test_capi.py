"""CPU tests of the C ABI boundary: the library loads, exports every entry
point include/tsr_core.h declares, and rejects bad input on the host with the
reference's error semantics -- all without a GPU."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from tsr_b200 import core

HEADER = Path(__file__).resolve().parents[1] / "include" / "tsr_core.h"


def declared_symbols():
    src = HEADER.read_text()
    return sorted(set(re.findall(r"^TSR_API[^(]*?\b(tsr_\w+)\s*\(", src, re.M)))


def test_header_declares_api():
    names = declared_symbols()
    assert "tsr_tree_build" in names and "tsr_dmc_extract" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    missing = [n for n in declared_symbols() if not hasattr(core.lib, n)]
    assert not missing, missing
    # the Python binding covers the whole ABI
    assert set(declared_symbols()) <= set(core.EXPORTED)


def test_params_default_are_app_cfg_values():
    p = core.params_default()
    assert (p.max_relative_sampling_distance, p.bandwidth_factor, p.confidence_threshold,
            p.relative_radius_for_priors, p.relative_sample_cone_length) == (2.0, 2.0, 100.0, 25.0, 1.0)


def test_version_string():
    assert "sm_100a" in core.version()


def _view(n=4, k=1, scale=0.01):
    pos = np.random.default_rng(0).uniform(-1, 1, (n, 3))
    nrm = np.tile([0.0, 0.0, 1.0], (n, 1))
    s = core.Samples(pos, nrm, np.full(n, scale), np.ones(n), np.zeros((n, k), np.uint32))
    return s


def test_null_arguments_rejected():
    out = ctypes.c_void_p()
    assert core.lib.tsr_tree_build(None, None, None, ctypes.byref(out)) == 1
    assert b"null" in core.lib.tsr_last_error_message()
    assert core.lib.tsr_tree_get_counts(None, None) == 1
    assert core.lib.tsr_occupancy_compute(None, None, None, 0, None, None) == 1
    assert core.lib.tsr_dmc_extract(None, None, None, None) == 1


def test_empty_sample_set_rejected():
    s = _view()
    v = s.view()
    v.count = 0
    out = ctypes.c_void_p()
    assert core.lib.tsr_tree_build(ctypes.byref(v), None, None, ctypes.byref(out)) == 1
    assert not out.value


def test_non_positive_scale_rejected():
    """Samples.cpp:280-288 throws on a non-positive scale."""
    s = _view()
    s.scales[2] = 0.0
    with pytest.raises(core.TsrError) as e:
        core.Tree(s)
    assert e.value.status == 1
    assert "scale" in str(e.value)


def test_link_count_overflow_rejected():
    """Samples::getMaxParentLinkCount (Samples.h:395-402): N * K < 2^32 - 1."""
    s = _view()
    v = s.view()
    v.count = 0x10000
    v.cams_per_sample = 0x10000
    out = ctypes.c_void_p()
    assert core.lib.tsr_tree_build(ctypes.byref(v), None, None, ctypes.byref(out)) == 2


def test_bad_params_rejected():
    s = _view()
    p = core.make_params(h_svo=0.0)
    with pytest.raises(core.TsrError) as e:
        core.Tree(s, params=p)
    assert e.value.status == 1


def test_free_null_is_harmless():
    core.lib.tsr_tree_free(None)
    core.lib.tsr_occupancy_free(None)
    core.lib.tsr_mesh_free(None)

"""Descriptor validation of sdft_request_create, which runs on the host before
any CUDA call: supported grids and topologies pass it (and, without a GPU, stop
at "no CUDA device"), unsupported ones are refused with the reason."""
import ctypes as C
import copy

import pytest

from softdft_b200 import native, workloads
from softdft_b200.api import setup_request

from tests.helpers import small_slit

pytestmark = pytest.mark.skipif(not native.library_present(), reason="libsoftdft.so not built")


def _create(ds):
    dft = setup_request(copy.deepcopy(ds))
    h = C.c_void_p()
    rc = native.lib().sdft_request_create(C.byref(dft.descriptor.desc), 0, C.byref(h))
    msg = native.lib().sdft_last_error().decode()
    if rc == native.SDFT_OK:  # a GPU is present: the request exists
        native.lib().sdft_request_destroy(h)
    return rc, msg


def _accepted(ds):
    rc, msg = _create(ds)
    assert rc == native.SDFT_OK or (rc == 4 and "no CUDA device" in msg), (rc, msg)


def _refused(ds, text):
    rc, msg = _create(ds)
    assert rc == native.SDFT_ERR_UNSUPPORTED and text in msg, (rc, msg)


def _branched(seq, **kw):
    ds = small_slit(**kw)
    ds["species"][0]["sequence"] = seq
    return ds


@pytest.mark.parametrize("np_", [128, 1000, 1001, 250, 286, 3969, 1009, 1002, 2018])
def test_supported_grids_pass_validation(np_):
    _accepted(small_slit(np_=np_, dz=0.02))


@pytest.mark.parametrize("np_,why", [(4099, "Bluestein transform of 16384 points"),
                                     (8198, "Bluestein transform of 16384 points"),
                                     (32768, "more shared memory than a CTA has")])
def test_unsupported_grids_are_refused(np_, why):
    _refused(small_slit(np_=np_, dz=0.02), why)


@pytest.mark.parametrize("seq", ["AA(AA)AA", "AAA(A)AAA(AA)A", "A(AB)A"])
def test_branched_chains_pass_validation(seq):
    _accepted(_branched(seq))


def test_branched_brush_passes_validation():
    ds = workloads.grafted_brush(256, 0.05, 6, 0.05, 4.5, 7.0, 0.01)
    ds["species"][0]["sequence"] = ds["species"][1]["sequence"] = "AA(AA)AA"
    _accepted(ds)


@pytest.mark.parametrize("seq", ["A(AA)(AA)A", "A(AB)2A"])
def test_branch_point_beyond_the_reference_arrays_is_refused(seq):
    """Three children of one segment with two states: the reference's
    other-children index (parent_propagators.jl:150) leaves its array."""
    _refused(_branched(seq), "index out of range")


def _create_mutated(mutate):
    dft = setup_request(small_slit())
    d = dft.descriptor.desc
    mutate(d)
    h = C.c_void_p()
    rc = native.lib().sdft_request_create(C.byref(d), 0, C.byref(h))
    return rc, native.lib().sdft_last_error().decode()


def _set_item(arr, i, v):
    arr[i] = v


@pytest.mark.parametrize("mutate,code,why", [
    (lambda d: setattr(d, "bin_width", float("nan")), 2, "bin_width must be positive and finite"),
    (lambda d: setattr(d, "bin_width", float("inf")), 2, "bin_width must be positive and finite"),
    (lambda d: setattr(d, "length", float("-inf")), 2, "length must be finite"),
    (lambda d: _set_item(d.diameter, 0, float("nan")), 2, "bead diameters must be finite"),
    (lambda d: _set_item(d.bond_types, 1, 99), 2, "bond_types entry out of range"),
    (lambda d: _set_item(d.bond_types, 0, -1), 2, "bond_types entry out of range"),
    (lambda d: setattr(d, "np", 2 ** 31 - 1), 3, "needs more shared memory than a CTA has"),
])
def test_descriptor_values_that_would_misindex_are_refused(mutate, code, why):
    """Values that the host tables or kernels would turn into indices (a grid
    spacing, a wall position, a diameter, a bond's bead types, NP + 1) are
    checked before anything is sized from them."""
    rc, msg = _create_mutated(mutate)
    assert rc == code and why in msg, (rc, msg)

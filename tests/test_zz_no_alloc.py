"""GPU test of the allocation-free entry point gci_eri_pairs_noalloc.

It must give the same ERI matrix as gci_eri_pairs (within the 1e-10 x max
tolerance of the ERI parity tests) on consecutive calls that reuse its one
fixed scratch, leave the device's free memory unchanged while doing so, and
reject a basis whose tables exceed that scratch.  Collected last (file name)
so that a run that stops at the first failure has run every other test
first; it passes alone in a fresh process as well as after the others.
"""
import ctypes as C

import numpy as np
import pytest

from gammcor_integrals_b200 import _capi, basis as gbasis, molecules

pytestmark = pytest.mark.gpu


def _npq(tb):
    return tb.NAO * (tb.NAO + 1) // 2


def _output(tb, ld, stream):
    """NaN-filled column-major ld x NPQ output, written on `stream` (the stream the
    library call will use), so that the fill is ordered before the call."""
    import torch
    with torch.cuda.stream(stream):
        return torch.full((_npq(tb), ld), float("nan"), dtype=torch.float64, device="cuda")


def _call(tb, ld, out, stream):
    s = tb.c_struct()
    return _capi.lib().gci_eri_pairs_noalloc(C.byref(s), 0.0, C.c_void_p(out.data_ptr()), ld,
                                             C.c_void_p(stream.cuda_stream))


def _noalloc(tb, ld, stream):
    out = _output(tb, ld, stream)
    return _call(tb, ld, out, stream), out


def _reference(tb, ld):
    out = np.full((ld, _npq(tb)), np.nan, order="F")
    s = tb.c_struct()
    _capi.check(_capi.lib().gci_eri_pairs(C.byref(s), 0.0, _capi.ptr(out), ld))
    return out


def _check(got, ref):
    got = got.cpu().numpy().T     # back to ld x NPQ
    assert np.all(np.isfinite(got)), "elements left unwritten"
    err = np.max(np.abs(got - ref))
    assert err < 1e-10 * max(1.0, np.max(np.abs(ref))), err


def test_noalloc_matches_eri_pairs_on_consecutive_calls():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test selected but no CUDA device is visible")
    # two different bases: the second call must not see the first call's scratch
    tb_a = gbasis.from_molecule(molecules.small_molecule(11, natoms=3, recipe=molecules.RECIPE_C1, nprim=(3, 4)))
    tb_b = gbasis.from_molecule(molecules.small_molecule(12, natoms=2, recipe=molecules.RECIPE_C2, nprim=(3, 4)))
    ld_a, ld_b = _npq(tb_a) + 3, _npq(tb_b)
    stream = torch.cuda.Stream()
    # one call per basis first: they load the library's device code for every
    # class involved (lazily loaded kernels take device memory on first use),
    # and the first looks up the scratch's device address
    for tb, ld in ((tb_a, ld_a), (tb_b, ld_b)):
        rc0, _ = _noalloc(tb, ld, stream)
        _capi.check(rc0)
    out_a = _output(tb_a, ld_a, stream)
    out_b = _output(tb_b, ld_b, stream)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    rc_a = _call(tb_a, ld_a, out_a, stream)
    rc_b = _call(tb_b, ld_b, out_b, stream)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    _capi.check(rc_a)
    _capi.check(rc_b)
    assert free1 == free0, f"device free memory changed by {free0 - free1} bytes across the two calls"
    _check(out_a, _reference(tb_a, ld_a))
    _check(out_b, _reference(tb_b, ld_b))


def test_noalloc_rejects_basis_beyond_scratch():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test selected but no CUDA device is visible")
    # 8 f shells of 40 primitives on one centre: 36 pairs x 1600 primitive-pair
    # records of 92 doubles = 42 MB > the 16 MiB scratch
    mol = molecules.random_molecule(77, 1, 4.0, (3,) * 8, (40, 40), (0.1, 1e3))
    tb = gbasis.from_molecule(mol)
    npq = _npq(tb)
    # an output buffer of the full size, so that nothing could be written out of bounds
    rc, out = _noalloc(tb, npq, torch.cuda.Stream())
    assert rc == _capi.GCI_ERR_BUFFER, rc
    assert "scratch" in _capi.lib().gci_last_error().decode()
    assert torch.isnan(out).all().item(), "a rejected call wrote its output"
    # the scratch is still usable afterwards
    tb_a = gbasis.from_molecule(molecules.small_molecule(11, natoms=3, recipe=molecules.RECIPE_C1, nprim=(3, 4)))
    rc, got = _noalloc(tb_a, _npq(tb_a), torch.cuda.Stream())
    _capi.check(rc)
    _check(got, _reference(tb_a, _npq(tb_a)))

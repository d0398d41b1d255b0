"""Pins the FP64 CPU oracle against outputs of the reference cuOPO3D itself
(tests/golden, produced by tests/golden/make_golden.py from the reference's own
headers on a B200).  CPU only."""
import numpy as np
import pytest

from golden_cases import Golden, fixture_names, rel_l2
from oracle import pyoracle as po

NAMES = fixture_names()


def oracle_run(g):
    """Heavy fixtures (Golden.heavy) get their scalars, grids and pump checked here; their
    output fields are checked against the FP64 CUDA path in tests/test_gpu_parity.py."""
    flags = po.OR_DISPERSION | po.OR_DIFFRACTION
    if g.asis:
        flags |= po.OR_ASIS_Q1 | po.OR_ASIS_Q2
    ph = po.make_phys(flags=flags, **g.config_kwargs())
    st = po.Setup(ph)
    s0, i0 = g.initial_fields(po.noise)
    api = st.api_complex()
    if g.heavy:
        return st, api, None
    if g.mode == "single":
        out = po.single_pass(st, api, s0, i0)
    else:
        out = po.round_trips(st, api, api, s0, i0, g.nrt)
    return st, api, out


@pytest.fixture(scope="module", params=NAMES)
def case(request):
    g = Golden(request.param)
    return g, oracle_run(g)


def test_fixture_set_present():
    assert {"g16_opo_fp64", "g16_single_fp64", "g12_opo_fp64", "c1_single_fp64",
            "g16_asis_fp32", "g16_opo_fp32"} <= set(NAMES)


def test_scalars_match_reference(case):
    """Sellmeier-derived scalars, kappa, k, steps and round-trip time (crystal, EFields
    and Cavity constructors) against the reference's own values."""
    g, (st, _, _) = case
    tol = 1e-12 if g.fp64 else 2e-6
    for k, v in st.scalars.items():
        ref = g.scalars[k]
        assert abs(v - ref) <= tol * max(abs(ref), 1e-300) or (ref == 0 and abs(v) < 1e-15), (k, v, ref)


def test_grids_match_reference(case):
    g, (st, _, _) = case
    tol = 1e-13 if g.fp64 else 1e-6
    assert rel_l2(st.t, g.t) < tol
    assert rel_l2(st.w, g.w) < tol


def test_pump_matches_reference(case):
    g, (_, api, _) = case
    tol = 1e-12 if g.fp64 else 1e-6
    assert rel_l2(api[g.tidx], g.Api) < tol


def test_fields_match_reference(case):
    """Output fields of the split-step (single pass or cavity round trips)."""
    g, (_, _, out) = case
    if out is None:
        pytest.skip("fields of this fixture are checked against the FP64 CUDA path (GPU tests)")
    ap, as_, ai = out
    if g.fp64:
        tol = 1e-10
    else:
        # FP32 reference: its own rounding; the as-shipped single pass shrinks the
        # fields by ~NT per step, leaving few significant digits.
        tol = 5e-4 if g.asis else 1e-4
    assert rel_l2(ap[g.tidx], g.Ap) < tol
    assert rel_l2(as_[g.tidx], g.As) < tol
    assert rel_l2(ai[g.tidx], g.Ai) < tol

"""The split-wave row pass with staged slice tables (bulk copies of the
transmission row and the probes' vacuum rows into shared memory) against
the plain row pass: with the default FFT radix schedule the arithmetic is
the same element for element, so every output must be bit-identical, with
and without the pipelined column pass, at every row length the staged pass
supports (256..2048) and for batch sizes that do not fill its last CTA.
The plain row pass's L1 and L2 prefetches change no arithmetic either.
The alternative radix schedule (16 elements a thread) rounds differently
and is held to the FP32 bounds against the reference's own results."""
import os

import numpy as np
import pytest

import msf
from conftest import assert_variance_close, case_argv, case_dir, load_case, rel_err

pytestmark = pytest.mark.gpu


def _run(name, golden_tmp, pipe, batch, ahead_pct=None):
    env = {"MSF_PIPE": str(pipe), "MSF_ROW_AHEAD_PCT": ahead_pct}
    old = {k: os.environ.get(k) for k in env}
    for k, v in env.items():
        if v is not None:
            os.environ[k] = v
    try:
        d = case_dir(name, golden_tmp)
        job, spec, res, ctx = msf.run_job(case_argv(name, d), precision="fp32", batch=batch)
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    return res


@pytest.mark.parametrize("name,batch", [("g512", 5), ("c2_small", 3), ("g2048", 7)])
@pytest.mark.parametrize("variant,ahead_pct", [(4, None), (16, None), (32, None), (48, None),
                                               (48, "1"), (80, None), (112, "1")])
@pytest.mark.parametrize("col", [0, 1])
def test_staged_row_pass_is_bit_identical(name, batch, col, variant, ahead_pct, golden_tmp):
    """variant 4: the staged row pass; 16: the plain one prefetching its
    tables into L1; 32: the plain one prefetching the wavefield rows of the
    CTAs one resident wave ahead into L2 (and 1 % of a wave ahead, so that
    most CTAs' prefetches land inside these small grids); 48: both
    prefetches; 64 added: each CTA's lines are one row of consecutive probes
    (the batch sizes here do not divide into them, so the last batch falls
    back to rows of one probe)."""
    plain = _run(name, golden_tmp, col, batch)
    staged = _run(name, golden_tmp, col | variant, batch, ahead_pct)
    if plain.adf_image is not None:
        assert np.array_equal(staged.adf_image, plain.adf_image)
    for m, v in plain.v.items():
        assert np.array_equal(staged.v[m], v, equal_nan=True), m


@pytest.mark.parametrize("name,batch", [("g512", 4), ("c2_small", 4), ("c2_small", 2)])
@pytest.mark.parametrize("variant", [64, 16 | 64, 16 | 32 | 64])
def test_lines_by_probe_is_bit_identical(name, batch, variant, golden_tmp):
    """Each CTA of the plain row pass transforms one row of consecutive
    probes (batches that its lines divide: 4 lines a CTA at 512 points, 2
    at 1024); the arithmetic per line is unchanged."""
    plain = _run(name, golden_tmp, 1, batch)
    got = _run(name, golden_tmp, 1 | variant, batch, "1")
    if plain.adf_image is not None:
        assert np.array_equal(got.adf_image, plain.adf_image)
    for m, v in plain.v.items():
        assert np.array_equal(got.v[m], v, equal_nan=True), m


@pytest.mark.parametrize("pipe", [1 | 8, 1 | 4 | 8])
@pytest.mark.parametrize("name,batch", [("g512", 5), ("c2_small", 3), ("g2048", 7)])
def test_alternative_schedule_matches_reference(name, batch, pipe, golden_tmp):
    """The 16-element radix schedule, in the plain and the staged row pass."""
    meta, ref = load_case(name)
    res = _run(name, golden_tmp, pipe, batch)
    if "adf_image" in ref:
        assert rel_err(res.adf_image, ref["adf_image"]).max() <= 1e-4
    for m in ("V_omega", "V_re"):
        if m in ref:
            assert_variance_close(res.v[m], ref[m][:, 1], 1e-4, 1e-7, what=m)

"""The split-wave row pass with staged slice tables (bulk copies of the
transmission row and the probes' vacuum rows into shared memory) against
the plain row pass: with the default FFT radix schedule the arithmetic is
the same element for element, so every output must be bit-identical, with
and without the pipelined column pass, at every row length the staged pass
supports (256..2048) and for batch sizes that do not fill its last CTA.
The alternative radix schedule (16 elements a thread) rounds differently
and is held to the FP32 bounds against the reference's own results."""
import os

import numpy as np
import pytest

import msf
from conftest import assert_variance_close, case_argv, case_dir, load_case, rel_err

pytestmark = pytest.mark.gpu


def _run(name, golden_tmp, pipe, batch):
    old = os.environ.get("MSF_PIPE")
    os.environ["MSF_PIPE"] = str(pipe)
    try:
        d = case_dir(name, golden_tmp)
        job, spec, res, ctx = msf.run_job(case_argv(name, d), precision="fp32", batch=batch)
    finally:
        if old is None:
            del os.environ["MSF_PIPE"]
        else:
            os.environ["MSF_PIPE"] = old
    return res


@pytest.mark.parametrize("name,batch", [("g512", 5), ("c2_small", 3), ("g2048", 7)])
@pytest.mark.parametrize("variant", [4, 16])
@pytest.mark.parametrize("col", [0, 1])
def test_staged_row_pass_is_bit_identical(name, batch, col, variant, golden_tmp):
    """variant 4: the staged row pass; 16: the plain one prefetching its
    tables into L1."""
    plain = _run(name, golden_tmp, col, batch)
    staged = _run(name, golden_tmp, col | variant, batch)
    if plain.adf_image is not None:
        assert np.array_equal(staged.adf_image, plain.adf_image)
    for m, v in plain.v.items():
        assert np.array_equal(staged.v[m], v, equal_nan=True), m


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

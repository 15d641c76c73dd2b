"""The transfer walks with their step records staged in shared memory, by
16-byte copies (k_transfer_staged, IPG_XFER_STAGE=1) and by one bulk copy
per record part (k_transfer_bulk, IPG_XFER_STAGE=2), and the default mixture
(IPG_XFER_STAGE unset: bulk copies for FP64 records except in the longest
length class, 16-byte copies otherwise; the 128x128 case is split into
length classes), against the walk that loads them from global memory
(k_transfer, IPG_XFER_STAGE=0).

All run the operations of integrate_emission's loop (src/ipolarray.c:78-244)
in the same order; the staged walks only regroup them by record (the
transfer step with record k's coefficients, then the push with record k's
transport matrices) and read the records from shared memory.  So every
image, in every step arithmetic and record layout, must be bit-identical.
"""
import os

import numpy as np
import pytest

import ipole_b200 as ip
from tests import common

pytestmark = pytest.mark.gpu

CASES = ["c1_bright_32", "c1_faraday_24", "c1_thick_24", "c1_unpol_24", "c1_refine_32", "c1_counterjet_16",
         "c1_subring1_16", "c1_full_128", "analytic_m2_32", "sphere_f223_i30_32"]
FORMS = [(ip.IPG_RECORDS_FP64, ip.IPG_STEP_FP64), (ip.IPG_RECORDS_MIXED, ip.IPG_STEP_FP64),
         (ip.IPG_RECORDS_FP64, ip.IPG_STEP_FP32), (ip.IPG_RECORDS_MIXED, ip.IPG_STEP_FP32)]


def _render(p, m, stage, rec, step):
    old = os.environ.get("IPG_XFER_STAGE")
    if stage is None:
        os.environ.pop("IPG_XFER_STAGE", None)
    else:
        os.environ["IPG_XFER_STAGE"] = str(stage)
    try:
        with ip.Context() as c:  # the setting is read when a context is created
            c.upload(m)
            c.set_record_precision(rec)
            c.set_step_precision(step)
            return c.render(p, m)
    finally:
        if old is None:
            os.environ.pop("IPG_XFER_STAGE", None)
        else:
            os.environ["IPG_XFER_STAGE"] = old


@pytest.mark.parametrize("case", CASES)
def test_staged_walk_bit_identical(case, dumps):
    meta, _ = common.load_golden(case)
    p = common.params_for(meta, dumps.get(meta))
    m = ip.Model.load(p)
    for rec, step in FORMS:
        a = _render(p, m, 0, rec, step)
        for stage in (1, 2, None):  # 16-byte copies, bulk copies, the default
            b = _render(p, m, stage, rec, step)
            assert np.array_equal(a.nstep, b.nstep)
            assert a.unpol.tobytes() == b.unpol.tobytes(), (case, rec, step, stage)
            if a.pol is not None:
                assert a.pol.tobytes() == b.pol.tobytes(), (case, rec, step, stage)

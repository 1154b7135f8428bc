"""Batches of uneven snapshots on one handle with autotuned schedule options: every job's
outputs equal a separate call's bit for bit (the options only change the schedule)."""
import numpy as np
import pytest

import distorteddustydiscanalysistoolkits_b200 as pb
from distorteddustydiscanalysistoolkits_b200 import batch

pytestmark = pytest.mark.gpu


def test_batched_jobs_match_separate_calls():
    descs = batch.c4_discs(5, seed=100, n_min=20_000, n_max=120_000, edges=(8, 12, 16))
    assert len({d["particles"] for d in descs}) == 5
    jobs = [batch.make_job(d) for d in descs]
    fresh = [batch.make_job(d) for d in descs]
    be = pb.CUDAComputeBackend(0)
    tuner = batch.Autotuner(walk_split=(8, 64), slice_queries=(1024, 1 << 22), bin_width=(1.0,), repeats=1)
    try:
        outs, ms = batch.batch_point_interpolation(be, jobs, tuner)
    finally:
        be.close()
    assert len(outs) == len(jobs) and all(m["interp_ms"] > 0 for m in ms)
    assert tuner.table
    for opts in tuner.table.values():
        assert opts["walk_split"] in (8, 64) and opts["slice_queries"] in (1024, 1 << 22)
    for job, out in zip(fresh, outs):
        ref_be = pb.CUDAComputeBackend(0)
        try:
            ref = pb.PointSamples_interpolation(ref_be, job["points"], job["input"], job["catalog"], pb.itpSymmetric,
                                                precision=pb.FP32C)
        finally:
            ref_be.close()
        a = np.stack([g.grid for g in out.grids])
        b = np.stack([g.grid for g in ref.grids])
        assert a.shape == (4, len(job["points"]))
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64))

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


def _separate(jobs, precision):
    be = pb.CUDAComputeBackend(0)
    try:
        return [np.stack([g.grid for g in pb.PointSamples_interpolation(be, j["points"], j["input"], j["catalog"],
                                                                         pb.itpSymmetric, precision=precision).grids])
                for j in jobs]
    finally:
        be.close()


@pytest.mark.parametrize("precision", [pb.FP64, pb.FP32C])
def test_device_batch_one_launch_matches_separate_calls(precision):
    """All discs built and interpolated by one batched launch: every output equals a separate
    call's bit for bit, for every schedule option (leaf-size cutoff, subtrees per disc of the
    walk, disc order, blocks per SM, slices small enough that warps straddle two discs), and the
    CUDA-graph replay equals the eager step."""
    descs = batch.c4_discs(6, seed=200, n_min=20_000, n_max=150_000, edges=(8, 12, 16))
    ref = _separate([batch.make_job(d) for d in descs], precision)
    db = batch.DeviceBatch([batch.make_job(d) for d in descs], precision=precision)
    try:
        for opts in ({"leaf_size": 1, "order": 0, "blocks_per_sm": 0, "walk_split": 16},
                     {"leaf_size": 8, "order": 1, "blocks_per_sm": 1, "walk_split": 1},
                     {"leaf_size": 32, "order": 0, "blocks_per_sm": 2, "walk_split": 64}):
            db.set_options(**opts)
            db.run()
            for a, b in zip(db.outputs(), ref):
                assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), opts
        db.backends[0].handle.set_option("slice_queries", 1040)   # slices of 32.5 warps of points
        db.set_options(walk_split=8)
        db.run()
        for a, b in zip(db.outputs(), ref):
            assert np.array_equal(a.view(np.uint64), b.view(np.uint64))
        db.backends[0].handle.set_option("slice_queries", 1 << 22)
        db.set_options(leaf_size=4, order=1)
        db.capture()
        for o in db.outs:
            for t in o:
                t.fill_(0.0)
        db.replay()
        db.replay()
        for a, b in zip(db.outputs(), ref):
            assert np.array_equal(a.view(np.uint64), b.view(np.uint64))
    finally:
        db.close()


def test_batch_autotuner_picks_an_option():
    descs = batch.c4_discs(3, seed=300, n_min=20_000, n_max=60_000, edges=(8,))
    db = batch.DeviceBatch([batch.make_job(d) for d in descs])
    try:
        tuner = batch.BatchAutotuner(leaf_size=(1, 8), order=(0,), blocks_per_sm=(0,), walk_split=(8, 32), repeats=1)
        best = tuner.tune(db)
        assert best in [t[0] for t in tuner.timings] and len(tuner.timings) == 4
        assert all(ms > 0 for _, ms in tuner.timings)
    finally:
        db.close()

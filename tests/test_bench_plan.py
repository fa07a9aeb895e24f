"""The bench's shape: what the driver's `--steps 20 --warmup 5` runs, and
that it ends well inside the driver's 1800 s limit at the measured cost of a
chunk of radial steps (bench.CHUNK_S)."""
import importlib.util
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
_spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
bench = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(bench)


def test_step_is_one_group_of_a_staggered_sweep():
    p = bench.plan("h2o_like", 32, 8, steps=20, warmup=5)
    assert p["chunks_per_sweep"] == 1501                  # 12001 points, 8 per chunk
    assert p["chunks_per_step"] == 188
    assert p["chunks_total"] == 1501 + 24 * 188
    assert p["chunks_timed"] == 20 * 188


def test_driver_run_fits_with_margin():
    for cfg in ("h2o_like", "h2_like"):
        c = bench.CONFIGS[cfg]
        t = bench.predict_seconds(cfg, c["slots"], c["groups"], steps=20, warmup=5)
        assert t <= 1500.0, (cfg, t)
    # a lock-step batch (one group) would not fit: every step a whole sweep
    assert bench.predict_seconds("h2o_like", 32, 1, steps=20, warmup=5) > 1800.0


def test_default_run_is_short():
    c = bench.CONFIGS["h2o_like"]
    assert bench.predict_seconds("h2o_like", c["slots"], c["groups"], steps=4, warmup=3) <= 600.0


def test_every_rank_streams_a_full_block():
    """Weak scaling: at N ranks the job's k grid has N times the points of
    the one-GPU workload over the same range, and every rank's cost-balanced
    block holds at least the slots it streams, so `bench.py --gpus N` runs
    the one-GPU per-rank workload at every N."""
    import numpy as np
    for cfg in ("h2o_like", "h2o_mixed", "h2_like"):
        c = bench.CONFIGS[cfg]
        one = c["ks"]()
        assert np.array_equal(bench.job_grid(cfg, 1), one)
        for world in (1, 2, 4, 8):
            ks = bench.job_grid(cfg, world)
            assert ks.size == one.size * world and ks[0] == one[0] and ks[-1] == one[-1]
            got = [bench.rank_block(cfg, world, r, 605) for r in range(world)]
            assert np.array_equal(np.concatenate([k for k, _ in got]), ks)
            for k, lc in got:
                assert k.size >= c["slots"], (cfg, world, k.size)
                assert lc.size == k.size

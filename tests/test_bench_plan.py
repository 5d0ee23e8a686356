"""bench.py's step plan (CPU): every run fuses the whole 1000-frame walk and
times --steps of its steps spread evenly after the warm-up, whatever
--steps is; the workload named in the line is that walk."""
import bench


def test_whole_walk_with_spread_timed_steps():
    a = bench.parse_args(["--steps", "20", "--warmup", "5"])
    total, timed = bench.step_plan(a)
    assert total == 100 and bench.n_frames_needed(a) == 1000
    assert len(timed) == len(set(timed)) == 20
    assert timed[0] == 5 and timed[-1] >= 95 and all(5 <= s < 100 for s in timed)
    gaps = [b - a_ for a_, b in zip(timed, timed[1:])]
    assert max(gaps) - min(gaps) <= 1


def test_default_times_every_step_after_warmup():
    a = bench.parse_args([])
    total, timed = bench.step_plan(a)
    assert total == 100 and timed == list(range(a.warmup, 100))


def test_longer_runs_extend_the_walk():
    a = bench.parse_args(["--steps", "150", "--warmup", "3"])
    total, timed = bench.step_plan(a)
    assert total == 153 and timed == list(range(3, 153))


def test_workload_names_the_whole_walk():
    a = bench.parse_args(["--steps", "20", "--warmup", "5"])
    cfg = bench.workload_config(a, bench.n_frames_needed(a))
    assert cfg["workload"].startswith("walk1000: the whole 1000 frames of the 1000-frame")
    assert cfg["timed_steps"] == bench.step_plan(a)[1]


def test_profiling_prefix():
    a = bench.parse_args(["--steps", "5", "--warmup", "3", "--walk-frames", "80"])
    total, timed = bench.step_plan(a)
    assert total == 8 and timed == [3, 4, 5, 6, 7]
    assert bench.workload_config(a, 80)["workload"].startswith("walk80: the first 80 frames")

"""Runtime tuning (ra_tuning): validation, and results that do not depend on it."""
import numpy as np
import pytest

import oracle as O
import parallel_ra_b200 as P

pytestmark = pytest.mark.gpu


def test_tuning_round_trip_and_validation():
    p = P.Program(0)
    t = p.get_tuning()
    assert set(t) == set(P.engine.Tuning.FIELDS)
    p.set_tuning(seen_load_max=0.7, join_blocks_per_sm=2)
    t2 = p.get_tuning()
    assert abs(t2["seen_load_max"] - 0.7) < 1e-12 and t2["join_blocks_per_sm"] == 2
    for bad in ({"seen_load_max": 0.95}, {"seen_load_max": 0.05}, {"seen_grow": 1.0}, {"log_growth": 5.0},
                {"join_blocks_per_sm": 0}, {"select_blocks_per_sm": 17}, {"dense_max_bytes": -1.0}):
        with pytest.raises(P.RAError):
            p.set_tuning(**bad)
    assert p.get_tuning() == t2
    p.close()


@pytest.mark.parametrize("tuning", [
    {"seen_load_max": 0.9, "seen_grow": 1.1, "log_growth": 1.1},      # many seen / log regrowths
    {"seen_load_max": 0.1, "seen_grow": 8.0, "log_growth": 4.0},
    {"join_blocks_per_sm": 1, "select_blocks_per_sm": 1},
    {"join_blocks_per_sm": 16, "select_blocks_per_sm": 16},
])
@pytest.mark.parametrize("program,rows", [
    ("tc", lambda: P.datagen.with_row_ids(P.datagen.erdos_renyi(3000, 3600, 4))),
    ("sg", lambda: P.datagen.with_row_ids(P.datagen.random_tree(1500, 8))),
])
def test_results_do_not_depend_on_tuning(tuning, program, rows):
    rows = rows()
    p = P.Program(0)
    p.set_tuning(**tuning)
    rels = P.programs.PROGRAMS[program](p, rows)
    p.execute(1)
    o = O.OracleProgram()
    orels = P.programs.PROGRAMS[program](o, rows)
    o.execute(1)
    assert p.history() == o.history()
    for name in rels:
        assert np.array_equal(p.dump_full(rels[name])[:, :-1], o.dump_full(orels[name])[:, :-1]), name


def test_release_frees_and_next_run_matches():
    rows = P.datagen.with_row_ids(P.datagen.erdos_renyi(4000, 4200, 9))
    p = P.Program(0)
    rels = P.programs.PROGRAMS["tc"](p, rows)
    p.execute(1)
    h1, d1 = p.history(), p.dump_full(rels["T"])
    held = p.stats().device_bytes
    p.release()
    assert p.stats().device_bytes < held
    with pytest.raises(P.RAError):
        p.dump_full(rels["T"])            # the run ended with the release
    p.execute(1)
    assert p.history() == h1
    assert np.array_equal(p.dump_full(rels["T"]), d1)
    p.release()
    p.set_tuning(seen_load_max=0.8)       # a release also lets the next run size under a new policy
    p.execute(1)
    assert np.array_equal(p.dump_full(rels["T"]), d1)

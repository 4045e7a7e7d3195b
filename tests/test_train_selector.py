"""The selector's training recipe on the CPU: the 200-graph set of the
benchmark configuration (R-MAT scales 16-22 with jittered a, b, c; grids of
side 1024-4096) and its determinism."""
from kites_b200.train_selector import config3_specs


def test_config3_recipe():
    specs = config3_specs(200)
    assert len(specs) == 200
    rmat = [x for x in specs if x[0] == "rmat"]
    grid = [x for x in specs if x[0] == "grid"]
    assert len(rmat) == 160 and len(grid) == 40
    assert {x[1] for x in rmat} == set(range(16, 23))
    assert all(1024 <= x[1] <= 4096 for x in grid)
    for _, _, ef, a, b, c, _ in rmat:
        assert ef == 16
        assert abs(a - 0.57) <= 0.08 and abs(b - 0.19) <= 0.05 and abs(c - 0.19) <= 0.05
        assert a + b + c <= 0.99 + 1e-12
    assert config3_specs(200) == specs
    assert len({x[6] for x in specs}) == 200  # one seed per graph

"""The per-GPU launch-parameter table (lg_tune_get / lg_tune_set /
lg_tune_reset): host logic only, no GPU needed."""
import pytest

from llama_b200 import LgError
from llama_b200.graph import TUNABLES, tune_get, tune_reset, tune_set

DEFAULTS = {"pr_ctas_per_sm": 0, "ppr_ktile": 256, "ppr_range": 2048, "sssp_range": 1024,
            "ms_heavy": 512, "pr_tile_occ": 0, "sssp_split": 0, "bfs_levels": 1,
            "sssp_levels": 0}


def test_defaults_set_and_reset():
    tune_reset(3)
    for name, v in DEFAULTS.items():
        assert tune_get(3, name) == v
    tune_set(3, "ppr_ktile", 64)
    tune_set(3, "ms_heavy", 2048)
    assert tune_get(3, "ppr_ktile") == 64 and tune_get(3, "ms_heavy") == 2048
    assert tune_get(2, "ppr_ktile") == 256          # per device
    tune_reset(3)
    assert tune_get(3, "ppr_ktile") == 256
    assert set(TUNABLES) == set(DEFAULTS)


@pytest.mark.parametrize("name,value", [("pr_ctas_per_sm", -1), ("pr_ctas_per_sm", 33),
                                        ("ppr_ktile", 16), ("ppr_range", 100),
                                        ("sssp_range", 1 << 20), ("ms_heavy", 8),
                                        ("pr_tile_occ", 9), ("sssp_split", 2),
                                        ("bfs_levels", 2), ("sssp_levels", -1)])
def test_out_of_range_values_are_rejected(name, value):
    with pytest.raises(LgError):
        tune_set(0, name, value)
    assert tune_get(0, name) == DEFAULTS[name]


def test_bad_device_is_rejected():
    with pytest.raises(LgError):
        tune_set(64, "ppr_ktile", 64)
    with pytest.raises(LgError):
        tune_get(-1, "ppr_ktile")

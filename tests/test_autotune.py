"""The tuning table of the C ABI and the autotuner's cache file (CPU: no
launch; the GPU side runs in bench.py and test_gpu_autotune)."""
import json

import pytest

from euvlitho_b200 import _lib as L
from euvlitho_b200 import autotune as A
from euvlitho_b200 import build


@pytest.fixture()
def lib():
    build.build()
    lib = L.lib()
    lib.euv_tune_clear()
    yield lib
    lib.euv_tune_clear()


def test_tune_table_set_get_clear(lib):
    assert lib.euv_tune_get(L.EUV_KNOB_ABBE_SPLIT, 24, 136) == 0
    assert lib.euv_tune_set(L.EUV_KNOB_ABBE_SPLIT, 24, 136, 6) == L.EUV_OK
    assert lib.euv_tune_set(L.EUV_KNOB_LU_CLUSTER, 961, 24, 4) == L.EUV_OK
    assert lib.euv_tune_get(L.EUV_KNOB_ABBE_SPLIT, 24, 136) == 6
    assert lib.euv_tune_get(L.EUV_KNOB_ABBE_SPLIT, 24, 137) == 0     # other shape
    assert lib.euv_tune_get(L.EUV_KNOB_LU_CLUSTER, 961, 24) == 4
    assert lib.euv_tune_set(L.EUV_KNOB_ABBE_SPLIT, 24, 136, 8) == L.EUV_OK   # overwrite
    assert lib.euv_tune_get(L.EUV_KNOB_ABBE_SPLIT, 24, 136) == 8
    assert lib.euv_tune_set(L.EUV_KNOB_ABBE_SPLIT, 24, 136, 0) == L.EUV_OK   # remove
    assert lib.euv_tune_get(L.EUV_KNOB_ABBE_SPLIT, 24, 136) == 0
    lib.euv_tune_clear()
    assert lib.euv_tune_get(L.EUV_KNOB_LU_CLUSTER, 961, 24) == 0


@pytest.mark.parametrize("knob,value", [(L.EUV_KNOB_LU_CLUSTER, 3), (L.EUV_KNOB_ABBE_SPLIT, 65),
                                        (L.EUV_KNOB_ZGEMM_ROWS, 48), (L.EUV_KNOB_LU_SUBST_COLS, 16),
                                        (99, 1)])
def test_tune_table_rejects_values_a_kernel_cannot_take(lib, knob, value):
    assert lib.euv_tune_set(knob, 1, 1, value) == L.EUV_ERR_BAD_ARG
    assert lib.euv_tune_get(knob, 1, 1) == 0


def test_cache_round_trip(lib, tmp_path, monkeypatch):
    monkeypatch.setattr(A, "gpu_name", lambda device=None: "NVIDIA B200")
    path = str(tmp_path / "tuning.json")
    A.save({("abbe_split", 24, 136): 6, ("lu_cluster", 961, 24): 0}, path)
    data = json.load(open(path))
    assert data == {"NVIDIA B200": {"abbe_split/24/136": 6, "lu_cluster/961/24": 0}}
    lib.euv_tune_set(L.EUV_KNOB_LU_CLUSTER, 961, 24, 8)
    assert A.load(path) == 2
    assert lib.euv_tune_get(L.EUV_KNOB_ABBE_SPLIT, 24, 136) == 6
    assert lib.euv_tune_get(L.EUV_KNOB_LU_CLUSTER, 961, 24) == 0   # built-in choice kept
    monkeypatch.setattr(A, "gpu_name", lambda device=None: "another GPU")
    lib.euv_tune_clear()
    assert A.load(path) == 0          # picks are per GPU model

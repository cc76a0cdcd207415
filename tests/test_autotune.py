"""The tuning table of the C ABI and the autotuner's cache file (CPU: no
launch; the GPU side runs in bench.py and test_gpu_autotune)."""
import json
import os

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


def _save_many(args):
    path, rank = args
    from euvlitho_b200 import autotune as A2
    A2.gpu_name = lambda device=None: "NVIDIA B200"  # no GPU needed to write the cache
    for i in range(200):
        A2.save({("abbe_split", 24, 100 + rank): 1 + (i % 4)}, path)
    return rank


def test_cache_save_from_concurrent_ranks(tmp_path):
    """One process per GPU may tune and save at once (torchrun): every save
    replaces the cache atomically through its own temporary file, so no rank
    fails and the file stays valid JSON."""
    import multiprocessing as mp
    path = str(tmp_path / "tuning.json")
    with mp.get_context("spawn").Pool(4) as pool:
        assert sorted(pool.map(_save_many, [(path, r) for r in range(4)])) == [0, 1, 2, 3]
    with open(path) as f:
        data = json.load(f)
    assert len(data) == 1 and all(v in (1, 2, 3, 4) for v in next(iter(data.values())).values())
    assert not [p for p in os.listdir(str(tmp_path)) if ".tmp" in p]

"""Failure detection on the host (no GPU): decoding of the device status word
and HBM-arena admission refusing an over-budget batch."""
import pytest

from euvlitho_b200 import _lib as L


def test_status_bits_decode_to_messages():
    assert L.status_message(0) is None
    assert "gave up" in L.status_message(L.EUV_STATUS_TIMEOUT)
    both = L.status_message(L.EUV_STATUS_SINGULAR | L.EUV_STATUS_STEPS_CLAMPED)
    assert "zero pivot" in both and "double-angle" in both
    assert "unknown bits 0x10" in L.status_message(16)


@pytest.mark.parametrize("bits,code", [(L.EUV_STATUS_TIMEOUT, L.EUV_ERR_TIMEOUT),
                                       (L.EUV_STATUS_SINGULAR, L.EUV_ERR_SINGULAR),
                                       (L.EUV_STATUS_STEPS_CLAMPED, L.EUV_ERR_CUDA),
                                       (L.EUV_STATUS_TIMEOUT | L.EUV_STATUS_SINGULAR,
                                        L.EUV_ERR_TIMEOUT)])
def test_check_status_raises_with_the_code(bits, code):
    L.check_status("x", 0)  # clear word: no error
    with pytest.raises(L.EuvError) as e:
        L.check_status("IntensityBatch", bits)
    assert e.value.code == code
    assert "0x%x" % bits in str(e.value)


def test_arena_refuses_over_budget_batches_and_reuses_freed_space():
    from euvlitho_b200.serving import Arena
    a = Arena(4096, "cpu")
    o1 = a.alloc(2000)           # rounded to 2048
    o2 = a.alloc(1500)           # 1536
    assert (o1, o2) == (0, 2048)
    assert a.alloc(1024) is None  # 512 left: admission refused
    a.free(o1)
    assert a.alloc(1024) == 0     # first fit in the freed region
    assert a.alloc(2048) is None
    assert a.view(o2, 1500).numel() == 1536

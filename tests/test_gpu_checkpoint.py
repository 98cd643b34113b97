"""Checkpoint / resume of a frame buffer's progressive state: a frame resumed
in a fresh context from a checkpoint continues its accumulation exactly, so
3 + 3 waves across two processes' worth of state equal 6 waves in one go
(bit-exact, plain and compensated accumulation)."""
import numpy as np
import pytest

import oracle
from tests.helpers import assert_bitexact, oracle_render, small_noise_scene

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("compensated", [False, True])
def test_resume_from_checkpoint_equals_uninterrupted_render(compensated):
    import barney_b200 as bn
    d = small_noise_scene(w=40, h=28, anisotropy=0.5, max_volume_bounces=2, compensated_accum=compensated)
    a = bn.VolumeRenderer(d)
    try:
        a.set_spp(3)
        a.render()
        first = a.read().copy()
        ck = a.checkpoint()
    finally:
        a.close()
    b = bn.VolumeRenderer(d)  # a fresh context, as after a restart
    try:
        b.set_spp(3)
        b.restore(ck)
        assert_bitexact(b.read(), first, "frame right after restore")
        b.render()
        resumed = b.read().copy()
    finally:
        b.close()
    sc = oracle.Scene(d)
    acc = np.zeros((28, 40, 4), np.float32)
    comp = np.zeros_like(acc) if compensated else None
    oracle.render(sc, 0, 6, accum=acc, comp=comp)
    assert_bitexact(resumed, oracle.resolve(acc, 6, comp=comp), "3 + 3 waves across a checkpoint")


def test_restore_rejects_a_checkpoint_of_another_size():
    import barney_b200 as bn
    a = bn.VolumeRenderer(small_noise_scene(w=16, h=16))
    b = bn.VolumeRenderer(small_noise_scene(w=17, h=16))
    try:
        a.set_spp(1)
        a.render()
        ck = a.checkpoint()
        with pytest.raises(bn.BarneyError):
            b.restore(ck)
        with pytest.raises(bn.BarneyError):
            a.restore(ck[:100])
        with pytest.raises(bn.BarneyError):
            a.restore(b"\0" * len(ck))
    finally:
        a.close()
        b.close()


def test_restore_rejects_an_accum_id_beyond_int_max():
    import struct
    import barney_b200 as bn
    a = bn.VolumeRenderer(small_noise_scene(w=16, h=16))
    try:
        bad = struct.pack("<8I", 0x43584E42, 1, 16, 16, 2 ** 31, 0, 0, 0) + bytes(16 * 16 * 16)
        with pytest.raises(bn.BarneyError):
            a.restore(bad)
        ok = struct.pack("<8I", 0x43584E42, 1, 16, 16, 2 ** 31 - 1, 0, 0, 0) + bytes(16 * 16 * 16)
        a.restore(ok)
    finally:
        a.close()


def test_failed_restore_allocation_leaves_the_frame_buffer_as_it_was():
    """A compensated checkpoint restored into an uncompensated frame buffer
    needs a compensation buffer; when that allocation fails, nothing of the
    checkpoint is applied and the frame continues as if there had been no
    restore."""
    import barney_b200 as bn
    L = bn.lib()
    dc = small_noise_scene(w=24, h=16, compensated_accum=True)
    a = bn.VolumeRenderer(dc)
    try:
        a.set_spp(2)
        a.render()
        ck = a.checkpoint()
    finally:
        a.close()
    d = small_noise_scene(w=24, h=16)
    b = bn.VolumeRenderer(d)
    try:
        b.set_spp(3)
        b.render()
        L.bnxInjectAllocationFailure(0)
        try:
            with pytest.raises(bn.BarneyError):
                b.restore(ck)
        finally:
            L.bnxInjectAllocationFailure(-1)
            L.bnClearLastError()
        b.render()
        resumed = b.read().copy()
    finally:
        b.close()
    sc = oracle.Scene(d)
    acc = np.zeros((16, 24, 4), np.float32)
    oracle.render(sc, 0, 6, accum=acc)
    assert_bitexact(resumed, oracle.resolve(acc, 6), "3 + 3 waves around a failed restore")

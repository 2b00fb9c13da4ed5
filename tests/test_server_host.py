"""Host-side pieces of the serving loop that need no GPU: the first-fit arena that serves
every wave and result from one allocation made at start-up."""

from dynamiqs_b200.server import _align, _Arena


def test_arena_first_fit_and_merge():
    a = _Arena(4096)
    x = a.alloc(100)  # rounded up to 256
    y = a.alloc(256)
    z = a.alloc(1000)  # 1024
    assert (x, y, z) == (0, 256, 512)
    assert a.used() == 256 + 256 + 1024
    assert a.alloc(4096) is None  # does not fit any more
    a.release(y, 256)
    assert a.alloc(200) == 256  # first fit reuses the hole
    a.release(256, 200)
    a.release(x, 100)
    a.release(z, 1000)
    assert a.used() == 0 and a.free == [(0, 4096)]  # neighbours merged back into one block
    assert a.alloc(4096) == 0


def test_align_is_256():
    assert [_align(v) for v in (0, 1, 255, 256, 257)] == [0, 256, 256, 256, 512]

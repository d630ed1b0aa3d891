"""GPU: CRC-32 of device memory equals zlib's crc32 (the checksum of a .sufidx
section, src/serialization.cpp:47-56), standalone and per output plane."""
import zlib

import numpy as np
import pytest

import sufkit_b200 as sg
from sufkit_b200 import synth

pytestmark = pytest.mark.gpu


def test_crc32_device_equals_zlib(ctx):
    import torch
    rng = np.random.default_rng(3)
    for nbytes in (0, 1, 15, 16384, 16385, 3 * 16384 + 7, 1 << 20, 37_000_017):
        host = rng.integers(0, 256, size=nbytes, dtype=np.uint8)
        dev = torch.from_numpy(host).cuda()
        for crc_in in (0, 0xDEADBEEF):
            got = ctx.crc32_device(dev.data_ptr() if nbytes else 0, nbytes, crc_in)
            assert got == zlib.crc32(host.tobytes(), crc_in), (nbytes, crc_in)
        if nbytes > 8:  # a start off the 16-byte grid
            got = ctx.crc32_device(dev.data_ptr() + 3, nbytes - 3, 7)
            assert got == zlib.crc32(host[3:].tobytes(), 7), nbytes


def test_plane_crcs_equal_zlib(ctx):
    t = synth.repeat_rich_100mbp(scale=0.01).logical_text()
    for sa_bits, lcp in ((32, sg.LcpEncoding.RAW32), (40, sg.LcpEncoding.BYTE32),
                         (64, sg.LcpEncoding.RAW64)):
        r = ctx.build(t, sa_bits=sa_bits, isa_bits=sa_bits, lcp=lcp, plane_crc=True)
        crc = r.stats["plane_crc"]
        assert crc["sa_low"] == zlib.crc32(r.sa_low.tobytes())
        assert crc["isa_low"] == zlib.crc32(r.isa_low.tobytes())
        assert crc["lcp"] == zlib.crc32(r.lcp.tobytes())
        if r.sa_high is not None:
            assert crc["sa_high"] == zlib.crc32(r.sa_high.tobytes())
            assert crc["isa_high"] == zlib.crc32(r.isa_high.tobytes())
    s = ctx.build(t, sa_bits=32, isa_bits=32, lcp=sg.LcpEncoding.RAW32, plane_crc=True,
                  sampling_rate=4)
    assert s.stats["plane_crc"]["sa_low"] == zlib.crc32(s.sa_low.tobytes())
    assert s.stats["plane_crc"]["lcp"] == zlib.crc32(s.lcp.tobytes())

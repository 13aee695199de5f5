"""Loading a version from its stored segments: the header and length
checks that run on the host (graph/segment/mod.rs:276-322, csr/mod.rs:90-99)
need no device and run here; the checks over every element run on the
device (tests/test_gpu_segments.py)."""

import numpy as np
import pytest

import pg_warren_b200 as W
from pg_warren_b200 import api

EXAMPLE = (np.array([0, 2, 2, 4], np.uint64), np.array([1, 2, 0, 2], np.uint32))


def segs(**over):
    rows, off, tgt, w = api.csr_segments(*EXAMPLE)
    d = {"rows": rows, "offsets": off, "targets": tgt, "weights": w}
    d.update(over)
    return d


def load(n=3, **over):
    s = segs(**over)
    return W.GraphVersion.from_segments(n, s["offsets"], s["targets"], s["weights"], s["rows"])


def test_the_encoding_is_the_references():
    # segment/mod.rs:1-16: magic, format 2, kind, width, reserved, count.
    off = api.encode_segment(1, np.array([0, 2], np.uint64))
    assert off[:8] == b"WRSG\x02\x01\x08\x00"
    assert int.from_bytes(off[8:16], "little") == 2 and len(off) == 16 + 16
    rows, off, tgt, _ = api.csr_segments(*EXAMPLE, sparse=True)
    assert np.frombuffer(rows[16:], "<u4").tolist() == [0, 2]
    assert np.frombuffer(off[16:], "<u8").tolist() == [0, 2, 4]


@pytest.mark.parametrize("bad,error", [
    (lambda s: s[:10], api.SegmentTruncated),
    (lambda s: b"XRSG" + s[4:], api.SegmentMagic),
    (lambda s: s[:4] + b"\x01" + s[5:], api.SegmentFormat),
    (lambda s: s[:5] + b"\x02" + s[6:], api.SegmentKind),
    (lambda s: s[:7] + b"\x01" + s[8:], api.SegmentReserved),
    (lambda s: s[:6] + b"\x04" + s[7:], api.SegmentWidth),
    (lambda s: s[:-8], api.SegmentLength),
])
def test_offsets_segment_header_errors(bad, error):
    with pytest.raises(error):
        load(offsets=bad(segs()["offsets"]))


def test_host_checked_csr_errors():
    with pytest.raises(api.OffsetsLength):
        load(offsets=api.encode_segment(1, np.array([0, 2, 4], np.uint64)))
    with pytest.raises(api.FirstOffsetNotZero):
        load(offsets=api.encode_segment(1, np.array([1, 2, 2, 4], np.uint64)))
    wide = np.frombuffer(segs()["targets"][16:], "<u4").astype(np.uint64)
    with pytest.raises(api.SegmentKind):
        load(targets=api.encode_segment(1, wide))
    with pytest.raises(api.SegmentWidth):
        load(targets=api.encode_segment(2, wide))

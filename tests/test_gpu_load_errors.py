"""Index load failures: corrupt or short bank files and manifests that disagree
with their banks are refused with an error (the reference's checks,
storage.rs:2208-2231, bank_io.rs:114-292), no device memory stays allocated
after a failed open, and the next open of a valid index works.
"""
import json
import shutil

import numpy as np
import pytest

from helpers import build_index, make_genomes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def framed_index(native, tmp_path_factory):
    d = tmp_path_factory.mktemp("load")
    fof = make_genomes(d / "g", 16, 1_100_000, 41)
    ix = build_index(fof, d / "index", k=31, H=4, b=16)
    bank = next(ix.glob("*.zorbank.zst"))
    assert bank.stat().st_size > (16 << 20)  # several 4 MiB frames
    return ix


def _bank(ix):
    return next(ix.glob("*.zorbank.zst"))


def _corrupt_middle(ix):
    p = _bank(ix)
    data = bytearray(p.read_bytes())
    for i in range(len(data) // 2, len(data) // 2 + 64):
        data[i] ^= 0x5A
    p.write_bytes(bytes(data))


def _truncate(ix):
    p = _bank(ix)
    data = p.read_bytes()
    p.write_bytes(data[: len(data) * 2 // 3])


def _manifest_slots(ix):
    m = json.loads((ix / "manifest.json").read_text())
    m["banks"][0]["slots"] *= 2
    (ix / "manifest.json").write_text(json.dumps(m))


@pytest.mark.parametrize("damage", [_corrupt_middle, _truncate, _manifest_slots],
                         ids=["corrupt-frame", "truncated-bank", "manifest-slots"])
def test_damaged_index_is_refused_and_releases_memory(gpu, framed_index, tmp_path, damage):
    import torch

    import zindex_b200 as zx
    from zindex_b200 import _lib

    bad = tmp_path / "bad"
    shutil.copytree(framed_index, bad)
    damage(bad)
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        with pytest.raises(zx.ZxError) as e:
            zx.Index(bad)
        assert e.value.code in (_lib.ZX_EFORMAT, _lib.ZX_EINVAL), e.value
    free_after = torch.cuda.mem_get_info()[0]
    assert free_before - free_after < (64 << 20), (free_before, free_after)
    with zx.Index(framed_index) as ix:
        seq = np.frombuffer(b"ACGT" * 100, dtype=np.uint8)
        counts, total = ix.query_records(seq, np.array([0, len(seq)], dtype=np.uint64))
        assert total == len(seq) - 31 + 1

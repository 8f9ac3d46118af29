"""The allocation-free query entry point (zx_query_device_noalloc).

It serves callers that cannot allocate device memory while they query (a host
whose HBM is fully reserved by its own allocator or by resident indexes, or a
latency-critical loop that must not enter the driver's allocator): its scratch
is one static 64 MiB device array per GPU. This file is collected last so a
run that stops at the first failure has already run every other test; it also
passes alone in a fresh process.
"""
import numpy as np
import pytest

import helpers

pytestmark = pytest.mark.gpu


def test_noalloc_query_matches_the_allocating_query_twice(gpu, tmp_path):
    import torch

    import zindex_b200 as zx

    fof = helpers.make_genomes(tmp_path / "genomes", colors=5, length=20000, seed=21)
    index = helpers.build_index(fof, tmp_path / "index", k=31, H=4, b=8)
    genomes = [helpers.dna(20000, 21 + c) for c in range(5)]
    rng = np.random.default_rng(4)
    reads = helpers.sample_reads(genomes, rng, 500, 150, n_runs=0.1)
    bases, offsets = zx.pack_records(reads)
    dev = torch.device("cuda", 0)
    d_bases = torch.from_numpy(bases).to(dev)
    d_off = torch.from_numpy(offsets.view(np.int64)).to(dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    with zx.Index(index) as ix:
        for _ in range(2):  # the shared array keeps the previous call's contents
            ref_counts = torch.zeros(ix.colors, dtype=torch.int64, device=dev)
            ref_total = torch.zeros(1, dtype=torch.int64, device=dev)
            ix.query_device(d_bases.data_ptr(), len(bases), d_off.data_ptr(), len(reads),
                            ref_counts.data_ptr(), ref_total.data_ptr(), stream=stream,
                            use_graph=False)
            counts = torch.zeros(ix.colors, dtype=torch.int64, device=dev)
            total = torch.zeros(1, dtype=torch.int64, device=dev)
            ix.query_device_noalloc(d_bases.data_ptr(), len(bases), d_off.data_ptr(), len(reads),
                                    counts.data_ptr(), total.data_ptr(), stream=stream)
            torch.cuda.synchronize(dev)
            # Integer counts: the tolerance is exact equality.
            assert int(total.item()) == int(ref_total.item()) > 0
            np.testing.assert_array_equal(counts.cpu().numpy(), ref_counts.cpu().numpy())


def test_noalloc_query_rejects_batches_beyond_its_scratch(gpu, tmp_path):
    import torch

    import zindex_b200 as zx

    fof = helpers.make_genomes(tmp_path / "genomes", colors=2, length=5000, seed=3)
    index = helpers.build_index(fof, tmp_path / "index", k=31, H=4, b=8)
    dev = torch.device("cuda", 0)
    n = 200_000_000  # needs more than the 64 MiB of scratch; never read
    d_bases = torch.zeros(16, dtype=torch.uint8, device=dev)
    d_off = torch.tensor([0, n], dtype=torch.int64, device=dev)
    counts = torch.zeros(2, dtype=torch.int64, device=dev)
    total = torch.zeros(1, dtype=torch.int64, device=dev)
    with zx.Index(index) as ix:
        with pytest.raises(zx.ZxError) as err:
            ix.query_device_noalloc(d_bases.data_ptr(), n, d_off.data_ptr(), 1, counts.data_ptr(),
                                    total.data_ptr())
        assert err.value.code == 1 and "scratch" in str(err.value)


def test_noalloc_errors_persist_until_status_and_stay_per_index(gpu, tmp_path):
    """An invalid-offsets call is still reported after later valid calls, and
    by its own index only: each index keeps its own error word in the shared
    array, and nothing but zx_query_status clears it. The decreasing offsets
    are skipped by the tile planner on the device; no kernel reads outside the
    batch."""
    import torch

    import zindex_b200 as zx

    fof = helpers.make_genomes(tmp_path / "genomes", colors=3, length=20000, seed=8)
    index = helpers.build_index(fof, tmp_path / "index", k=31, H=4, b=8)
    genomes = [helpers.dna(20000, 8 + c) for c in range(3)]
    reads = helpers.sample_reads(genomes, np.random.default_rng(2), 64, 150)
    bases, offsets = zx.pack_records(reads)
    dev = torch.device("cuda", 0)
    d_bases = torch.from_numpy(bases).to(dev)
    d_good = torch.from_numpy(offsets.view(np.int64)).to(dev)
    bad = offsets.copy()
    bad[2], bad[3] = bad[3], bad[2]  # record 2 ends before it starts
    d_bad = torch.from_numpy(bad.view(np.int64)).to(dev)
    counts = torch.zeros(3, dtype=torch.int64, device=dev)
    total = torch.zeros(1, dtype=torch.int64, device=dev)
    with zx.Index(index) as a, zx.Index(index) as b:
        a.query_device_noalloc(d_bases.data_ptr(), len(bases), d_bad.data_ptr(), len(reads),
                               counts.data_ptr(), total.data_ptr())
        a.query_device_noalloc(d_bases.data_ptr(), len(bases), d_good.data_ptr(), len(reads),
                               counts.data_ptr(), total.data_ptr())
        b.query_device_noalloc(d_bases.data_ptr(), len(bases), d_good.data_ptr(), len(reads),
                               counts.data_ptr(), total.data_ptr())
        torch.cuda.synchronize(dev)
        b.query_status()  # index b's calls were all valid
        with pytest.raises(zx.ZxError) as err:
            a.query_status()
        assert err.value.code == 1
        a.query_status()  # read and cleared

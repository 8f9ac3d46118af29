"""Parity of the wide-row form (kernels/wide_probe.cuh) with the oracle.

The wide-row probe counts fields in per-thread register planes over fixed
16-byte chunks of every row and counts a recovered origin only when the
filter missed it (a point probe of the origin's own field). These cases
cover every fingerprint width it takes (4, 8, 16, 32), hash counts whose
row loads fold by 4 and by 8 (H 2, 3, 5, 8, 13), one and two chunks per
thread, multi-member groups, hash partitions, several size classes, k-mers
(short and long), minimizers and modimizers, recovery on and off, shared and
global colour counters, seeds probed in extraction order and sorted by
their first hash, and device batches replayed from a CUDA graph.
"""
import numpy as np
import pytest

import helpers
from helpers import build_index, dna, sample_reads

pytestmark = pytest.mark.gpu

CASES = [
    dict(colors=600, H=2, b=8, k=25, groups="1,2"),
    dict(colors=1500, H=4, b=4, k=31, groups="0,1,2;7,9"),
    dict(colors=2048, H=3, b=16, k=25, groups="5,6,7,8"),
    dict(colors=4096, H=8, b=4, k=31, max_size="2MiB"),
    dict(colors=700, H=5, b=16, mode="minimizers", k=31, m=21),
    dict(colors=1000, H=3, b=32, mode="modimizers", k=31, d=4),
    dict(colors=800, H=4, b=8, k=45, groups="3,4"),
    dict(colors=300, H=13, b=4, k=21),
    dict(colors=256, H=4, b=8, k=31),     # rows of few chunks: teams of 32 threads
    dict(colors=6000, H=8, b=4, k=25),    # three chunks per thread with 8 warps
    dict(colors=4000, H=3, b=16, k=25),  # four chunks per thread with 8 warps
]


def _index(tmp_path_factory, colors, seed=83, **opts):
    d = tmp_path_factory.mktemp("wide")
    # Genomes of three lengths: several source size classes.
    lengths = [2000 if c % 3 == 0 else (4000 if c % 3 == 1 else 9000) for c in range(colors)]
    lines = []
    (d / "g").mkdir()
    for c, n in enumerate(lengths):
        p = d / "g" / f"g{c}.fa"
        helpers.write_fasta(p, [dna(n, seed + c)])
        lines.append(f"g{c}\t{p}")
    (d / "fof.tsv").write_text("\n".join(lines) + "\n")
    build_index(d / "fof.tsv", d / "index", min_docs=1, **opts)
    return d / "index", [dna(n, seed + c) for c, n in enumerate(lengths)]


@pytest.mark.parametrize("case", CASES, ids=lambda c: "c{colors}-H{H}-b{b}-k{k}".format(**c) +
                         ("-" + c["mode"] if "mode" in c else ""))
def test_wide_form_matches_oracle(gpu, oracle, tmp_path_factory, case):
    import zindex_b200 as zx

    case = dict(case)
    colors = case.pop("colors")
    ix, genomes = _index(tmp_path_factory, colors, **case)
    reads = sample_reads(genomes, np.random.default_rng(5), 700, 150, n_runs=0.1, lower=0.01)
    reads += sample_reads(genomes, np.random.default_rng(6), 20, 3000)
    bases, offsets = zx.pack_records(reads)
    with zx.Index(ix) as index:
        chunks_ok = []
        for warps in (4, 8, 9):
            try:
                index.set_launch(wide=1, warps=warps)
                chunks_ok.append(warps)
            except zx.ZxError as e:
                assert e.code == 1
        assert chunks_ok, "no block size admits the wide-row form"
        for recover in (True, False):
            want, want_total = oracle.query_records(ix, bases, offsets, recover=recover)
            for warps in chunks_ok:
                for counters, order in ((1, 1), (1, 0), (0, 1), (1, 2)):
                    index.set_launch(wide=1, warps=warps, smem_counters=counters, order=order)
                    assert index.launch()["wide"] == 1 and index.launch()["order"] == order
                    got, total = index.query_records(bases, offsets, recover=recover)
                    assert total == want_total, (warps, counters, order, recover)
                    np.testing.assert_array_equal(got, want)


def test_wide_form_device_graph_replay(gpu, oracle, tmp_path_factory):
    """The wide form's launch sequence (cursor reset, dense extraction, probe,
    reduction) captured as a CUDA graph and replayed gives the same counts."""
    import torch

    import zindex_b200 as zx

    ix, genomes = _index(tmp_path_factory, 2048, H=3, b=16, k=31)
    reads = sample_reads(genomes, np.random.default_rng(9), 3000, 150)
    bases, offsets = zx.pack_records(reads)
    want, want_total = oracle.query_records(ix, bases, offsets)
    dev = torch.device("cuda", 0)
    d_bases = torch.from_numpy(bases).to(dev)
    d_off = torch.from_numpy(offsets.view(np.int64)).to(dev)
    with zx.Index(ix) as index:
        assert index.launch()["wide"] == 1, "2,048 colours at b 16 default to the wide form"
        for _ in range(3):
            counts = torch.zeros(index.colors, dtype=torch.int64, device=dev)
            total = torch.zeros(1, dtype=torch.int64, device=dev)
            index.query_device(d_bases.data_ptr(), len(bases), d_off.data_ptr(), len(reads),
                               counts.data_ptr(), total.data_ptr(), use_graph=True)
            torch.cuda.synchronize(dev)
            index.query_status()
            assert int(total.item()) == want_total
            np.testing.assert_array_equal(counts.cpu().numpy().astype(np.uint64), want)


def test_wide_form_refuses_what_it_cannot_run(gpu, tmp_path_factory):
    import zindex_b200 as zx

    ix, _ = _index(tmp_path_factory, 40, H=4, b=2, k=25)
    with zx.Index(ix) as index:
        with pytest.raises(zx.ZxError) as err:
            index.set_launch(wide=1, warps=8)  # 2-bit fingerprints
        assert err.value.code == 1
    ix, _ = _index(tmp_path_factory, 6000, H=3, b=16, k=25)  # about 750 chunks per row
    with zx.Index(ix) as index:
        with pytest.raises(zx.ZxError):
            index.set_launch(wide=1, warps=4)  # more than 4 chunks per thread
        index.set_launch(wide=1, warps=8)
        # Back to the fused kernel: its own default fields, not the wide form's.
        index.set_launch(wide=0)
        assert index.launch() == dict(index.default_fused_launch(), blocks=0)


def test_wide_form_serves_coalesced_requests(gpu, oracle, tmp_path_factory):
    """Coalesced requests on a wide-row index (one segmented wide-form query:
    each request's seeds in its own part of the key list, probe rounds that
    never straddle requests, each block's counters added to the request it
    leaves) and the request server on it: every request's counts are the
    oracle's for that request alone, with shared and global counters and on
    rows of few chunks (teams of threads)."""
    import threading

    import torch

    import zindex_b200 as zx
    from test_gpu_serving import requests_for

    ix, genomes = _index(tmp_path_factory, 2048, H=3, b=16, k=31)
    reqs = requests_for(genomes, 90, seed=13)
    with zx.Index(ix) as index:
        assert index.launch()["wide"] == 1
        dev = torch.device("cuda", 0)
        for counters, part in ((1, reqs[:20]), (1, reqs), (0, reqs)):
            index.set_launch(wide=1, smem_counters=counters)
            flat = [r for recs in part for r in recs]
            seg = np.zeros(len(part) + 1, dtype=np.uint64)
            seg[1:] = np.cumsum([len(recs) for recs in part])
            bases, offsets = zx.pack_records(flat)
            d_bases = torch.from_numpy(bases if len(bases) else np.zeros(1, np.uint8)).to(dev)
            d_off = torch.from_numpy(offsets.view(np.int64)).to(dev)
            counts = torch.zeros((len(part), index.colors), dtype=torch.int64, device=dev)
            totals = torch.zeros(len(part), dtype=torch.int64, device=dev)
            index.query_segments(d_bases.data_ptr(), len(bases), d_off.data_ptr(), len(flat), seg,
                                 counts.data_ptr(), totals.data_ptr())
            torch.cuda.synchronize(dev)
            got, got_t = counts.cpu().numpy().astype(np.uint64), totals.cpu().numpy()
            for i in range(0, len(part), 3):
                want, want_total = oracle.query_records(ix, *zx.pack_records(part[i]))
                assert int(got_t[i]) == want_total, i
                np.testing.assert_array_equal(got[i], want, err_msg=f"request {i}")
        index.set_launch(wide=1)
        with zx.Server(index, slots=3, slot_bases=200000, slot_requests=7) as server:
            tickets = [None] * len(reqs)

            def submitter(p):
                for i in range(p, len(reqs), 3):
                    tickets[i] = server.submit(*zx.pack_records(reqs[i]))

            threads = [threading.Thread(target=submitter, args=(p,)) for p in range(3)]
            for t in threads:
                t.start()
            for t in threads:
                t.join()
            results = [server.wait(t) for t in tickets]
    for i in range(0, len(reqs), 4):
        want, want_total = oracle.query_records(ix, *zx.pack_records(reqs[i]))
        assert results[i][1] == want_total, i
        np.testing.assert_array_equal(results[i][0], want, err_msg=f"served request {i}")


@pytest.mark.parametrize("colors,opts", [(2048, dict(H=3, b=16, k=31)), (256, dict(H=4, b=8, k=31))],
                         ids=["c2048-b16", "c256-teams"])
def test_wide_segments_across_extraction_rounds(gpu, oracle, tmp_path_factory, colors, opts):
    """A segmented wide-row query of more tiles than one extraction round
    holds (two rounds on two key lists, the second extracted beside the
    first's probe): 1,000 requests of 300 short records, one of them cut by
    the round boundary. The requests' counts add up to the oracle's count of
    the whole batch, and a sample (the boundary's requests among them) equals
    the oracle's per request. The same batch unsegmented (seeds sorted per
    round, and in extraction order) gives the oracle's count."""
    import torch

    import zindex_b200 as zx

    ix, genomes = _index(tmp_path_factory, colors, **opts)
    rng = np.random.default_rng(21)
    n_req, per = 1000, 300
    reads = sample_reads(genomes, rng, n_req * per, 40, n_runs=0.05)
    bases, offsets = zx.pack_records(reads)
    seg = (np.arange(n_req + 1, dtype=np.uint64) * per).astype(np.uint64)
    dev = torch.device("cuda", 0)
    d_bases = torch.from_numpy(bases).to(dev)
    d_off = torch.from_numpy(offsets.view(np.int64)).to(dev)
    with zx.Index(ix) as index:
        index.set_launch(wide=1)
        counts = torch.zeros((n_req, index.colors), dtype=torch.int64, device=dev)
        totals = torch.zeros(n_req, dtype=torch.int64, device=dev)
        index.query_segments(d_bases.data_ptr(), len(bases), d_off.data_ptr(), len(reads), seg,
                             counts.data_ptr(), totals.data_ptr())
        torch.cuda.synchronize(dev)
        got, got_t = counts.cpu().numpy().astype(np.uint64), totals.cpu().numpy()
        # The same batch unsegmented: two ordered rounds (each block on its
        # own seeds, then interleaved seeds), and two in extraction order.
        whole = []
        for order in (1, 2, 0):
            index.set_launch(wide=1, order=order)
            c1 = torch.zeros(index.colors, dtype=torch.int64, device=dev)
            t1 = torch.zeros(1, dtype=torch.int64, device=dev)
            index.query_device(d_bases.data_ptr(), len(bases), d_off.data_ptr(), len(reads),
                               c1.data_ptr(), t1.data_ptr())
            torch.cuda.synchronize(dev)
            whole.append((c1.cpu().numpy().astype(np.uint64), int(t1.item())))
    want, want_total = oracle.query_records(ix, bases, offsets)
    assert int(got_t.sum()) == want_total
    np.testing.assert_array_equal(got.sum(axis=0, dtype=np.uint64), want)
    for c1, t1 in whole:
        assert t1 == want_total
        np.testing.assert_array_equal(c1, want)
    boundary = (1 << 18) // per  # one tile per 40-base record; 2^18 tiles per round
    for i in sorted({0, 1, boundary - 1, boundary, boundary + 1, n_req - 1, 417}):
        sub = reads[i * per:(i + 1) * per]
        w, wt = oracle.query_records(ix, *zx.pack_records(sub))
        assert int(got_t[i]) == wt, i
        np.testing.assert_array_equal(got[i], w, err_msg=f"request {i}")


def test_wide_form_per_record(gpu, oracle, tmp_path_factory):
    """Per-record queries on a wide-row index (one segment per record, most
    records one probe round, so one block writes their counters) equal the
    oracle's query of each record alone."""
    import zindex_b200 as zx

    ix, genomes = _index(tmp_path_factory, 2048, H=3, b=16, k=31)
    rng = np.random.default_rng(31)
    recs = sample_reads(genomes, rng, 150, 150, n_runs=0.1)
    recs += sample_reads(genomes, rng, 12, 2500) + [b"", b"ACGT", b"N" * 60]
    order = rng.permutation(len(recs))
    recs = [recs[i] for i in order]
    bases, offsets = zx.pack_records(recs)
    with zx.Index(ix) as index:
        assert index.launch()["wide"] == 1
        counts, totals = index.query_per_record(bases, offsets)
    for i, r in enumerate(recs):
        want, want_total = oracle.query_records(ix, *zx.pack_records([r]))
        assert int(totals[i]) == want_total, i
        np.testing.assert_array_equal(counts[i], want, err_msg=f"record {i}")

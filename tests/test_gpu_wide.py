"""Parity of the wide-row form (kernels/wide_probe.cuh) with the oracle.

The wide-row probe counts fields in per-thread register planes over fixed
16-byte chunks of every row and counts a recovered origin only when the
filter missed it (a point probe of the origin's own field). These cases
cover every fingerprint width it takes (4, 8, 16, 32), hash counts whose
row loads fold by 4 and by 8 (H 2, 3, 5, 8, 13), one and two chunks per
thread, multi-member groups, hash partitions, several size classes, k-mers
(short and long), minimizers and modimizers, recovery on and off, shared and
global colour counters, and device batches replayed from a CUDA graph.
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
                for counters in (1, 0):
                    index.set_launch(wide=1, warps=warps, smem_counters=counters)
                    assert index.launch()["wide"] == 1
                    got, total = index.query_records(bases, offsets, recover=recover)
                    assert total == want_total, (warps, counters, recover)
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
    """Coalesced requests on a wide-row index (each request its own wide-form
    launch sequence) and the request server on it: every request's counts are
    the oracle's for that request alone, and a batch of more requests than
    the per-request path takes goes through the fused segmented launch."""
    import threading

    import torch

    import zindex_b200 as zx
    from test_gpu_serving import requests_for

    ix, genomes = _index(tmp_path_factory, 2048, H=3, b=16, k=31)
    reqs = requests_for(genomes, 90, seed=13)
    with zx.Index(ix) as index:
        assert index.launch()["wide"] == 1
        dev = torch.device("cuda", 0)
        for part in (reqs[:20], reqs):  # 20 requests: per request; 90: fused segmented
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

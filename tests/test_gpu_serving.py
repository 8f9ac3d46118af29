"""Coalesced (segmented) launches and the request server, against the oracle.

A segmented launch answers several requests at once, each with its own
counters; the server admits requests into such batches as slots free up. Every
request's counts must equal the oracle's for that request alone (integer
counts: exact equality), whatever else shares its batch.
"""
import threading

import numpy as np
import pytest

from helpers import build_index, dna, make_genomes, sample_reads

pytestmark = pytest.mark.gpu

_IX = {}


def index_for(tmp_path_factory, **opts):
    key = tuple(sorted(opts.items()))
    if key not in _IX:
        d = tmp_path_factory.mktemp("srv")
        colors = opts.pop("colors", 12)
        fof = make_genomes(d / "genomes", colors, 20000, 17)
        build_index(fof, d / "index", **opts)
        _IX[key] = (d / "index", [dna(20000, 17 + c) for c in range(colors)])
    return _IX[key]


def requests_for(genomes, n, seed):
    """Mixed requests: short-read sets, long records, empty and N-only ones."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        kind = i % 5
        if kind == 0:
            recs = sample_reads(genomes, rng, int(rng.integers(1, 60)), 150, n_runs=0.1)
        elif kind == 1:
            recs = sample_reads(genomes, rng, int(rng.integers(1, 4)), int(rng.integers(2000, 9000)))
        elif kind == 2:
            recs = sample_reads(genomes, rng, int(rng.integers(1, 8)), int(rng.integers(40, 400)),
                                lower=0.05)
        elif kind == 3:
            recs = [b"", b"N" * 80] if i % 2 else []
        else:
            recs = sample_reads(genomes, rng, 1, 31)
        out.append(recs)
    return out


def oracle_counts(oracle, ix, recs, recover=True):
    import zindex_b200 as zx

    bases, offsets = zx.pack_records(recs)
    return oracle.query_records(ix, bases, offsets, recover=recover)


@pytest.mark.parametrize("launch", [dict(), dict(planes=0), dict(smem_counters=0),
                                    dict(planes=0, smem_counters=0, team=4)])
@pytest.mark.parametrize("mode", ["kmers", "findere"])
def test_segmented_launch_equals_each_request_alone(gpu, oracle, tmp_path_factory, launch, mode):
    import torch

    import zindex_b200 as zx

    opts = dict(mode=mode, k=31, H=4, b=8, groups="0,1,2;5,6")
    if mode == "findere":
        opts["z"] = 8
    ix, genomes = index_for(tmp_path_factory, **opts)
    reqs = requests_for(genomes, 25, seed=3)
    flat = [r for recs in reqs for r in recs]
    seg = np.zeros(len(reqs) + 1, dtype=np.uint64)
    seg[1:] = np.cumsum([len(recs) for recs in reqs])
    bases, offsets = zx.pack_records(flat)
    dev = torch.device("cuda", 0)
    d_bases = torch.from_numpy(bases if len(bases) else np.zeros(1, np.uint8)).to(dev)
    d_off = torch.from_numpy(offsets.view(np.int64)).to(dev)
    with zx.Index(ix) as index:
        index.set_launch(**launch)
        for _ in range(2):  # the second call reuses the staging buffers
            counts = torch.zeros((len(reqs), index.colors), dtype=torch.int64, device=dev)
            totals = torch.zeros(len(reqs), dtype=torch.int64, device=dev)
            index.query_segments(d_bases.data_ptr(), len(bases), d_off.data_ptr(), len(flat), seg,
                                 counts.data_ptr(), totals.data_ptr())
            torch.cuda.synchronize(dev)
            got, got_t = counts.cpu().numpy().astype(np.uint64), totals.cpu().numpy()
            for i, recs in enumerate(reqs):
                want, want_total = oracle_counts(oracle, ix, recs)
                assert int(got_t[i]) == want_total, i
                np.testing.assert_array_equal(got[i], want, err_msg=f"request {i}")


def test_server_results_are_the_same_alone_and_in_the_mix(gpu, oracle, tmp_path_factory):
    import zindex_b200 as zx

    ix, genomes = index_for(tmp_path_factory, mode="kmers", k=31, H=4, b=8)
    reqs = requests_for(genomes, 80, seed=7)
    recover = [i % 7 != 3 for i in range(len(reqs))]
    with zx.Index(ix) as index:
        alone = [index.query_records(*zx.pack_records(recs), recover=rc)
                 for recs, rc in zip(reqs, recover)]
        # Small slots so the mix is cut into many batches that overlap.
        with zx.Server(index, slots=3, slot_bases=60000, slot_requests=9) as server:
            tickets = [None] * len(reqs)

            def submitter(part):
                for i in range(part, len(reqs), 4):
                    tickets[i] = server.submit(*zx.pack_records(reqs[i]), recover=recover[i])

            threads = [threading.Thread(target=submitter, args=(p,)) for p in range(4)]
            for t in threads:
                t.start()
            for t in threads:
                t.join()
            results = [server.wait(t) for t in tickets]
            st = server.stats()
        assert st["completed"] == len(reqs) and st["failed"] == 0
        assert st["batches"] > 1 and 0 < st["p50_s"] <= st["p99_s"] <= st["max_s"]
    for i, ((counts, total, latency), (a_counts, a_total)) in enumerate(zip(results, alone)):
        assert total == a_total, i
        np.testing.assert_array_equal(counts, a_counts, err_msg=f"request {i}")
        assert latency > 0
    for i in range(0, len(reqs), 9):  # and the oracle, on a sample
        want, want_total = oracle_counts(oracle, ix, reqs[i], recover=recover[i])
        assert results[i][1] == want_total
        np.testing.assert_array_equal(results[i][0], want)


def test_server_admission_limits_and_timeouts(gpu, tmp_path_factory):
    import zindex_b200 as zx

    ix, genomes = index_for(tmp_path_factory, mode="kmers", k=31, H=4, b=8)
    with zx.Index(ix) as index:
        with zx.Server(index, slots=1, slot_bases=4096, slot_records=4, slot_requests=2) as server:
            with pytest.raises(zx.ZxError) as err:
                server.submit(*zx.pack_records([genomes[0][:5000]]))
            assert err.value.code == 1 and "slot" in str(err.value)
            with pytest.raises(zx.ZxError):
                server.submit(*zx.pack_records([b"ACGT"] * 5))
            t = server.submit(*zx.pack_records([genomes[1][:3000]]))
            counts, total, _ = server.wait(t)
            assert total == 3000 - 31 + 1
            with pytest.raises(zx.ZxError):
                server.wait(t)  # collected already
        with pytest.raises(zx.ZxError):
            zx.Server(index, slots=0 + 17)

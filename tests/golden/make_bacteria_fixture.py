"""Copies the reference's bundled bacteria example into tests/golden/bacteria.

The reference ships ten RefSeq assemblies with a query file of one fragment
per genome, its reverse complement and a random negative control, and the
source truth of every positive (tests/data/bacteria/ of the reference: the
inputs of utils/scripts/demo.sh:36-43). The files are copied byte for byte,
so the tests that use them run where the reference tree is not mounted. The
list of datasets is rewritten with paths relative to the fixture directory.

    python tests/golden/make_bacteria_fixture.py [reference-root]
"""
import shutil
import sys
from pathlib import Path

FILES = ["query.fa", "queries.fa", "source-truth.tsv", "README.md"]


def main():
    ref = Path(sys.argv[1] if len(sys.argv) > 1 else "/root/reference") / "tests/data/bacteria"
    out = Path(__file__).resolve().parent / "bacteria"
    (out / "genomes").mkdir(parents=True, exist_ok=True)
    for name in FILES:
        shutil.copyfile(ref / name, out / name)
    lines = []
    for line in (ref / "samples.fof").read_text().splitlines():
        name, path = line.split("\t")
        shutil.copyfile(ref / "genomes" / Path(path).name, out / "genomes" / Path(path).name)
        lines.append(f"{name}\tgenomes/{Path(path).name}")
    (out / "samples.fof").write_text("\n".join(lines) + "\n")


if __name__ == "__main__":
    main()

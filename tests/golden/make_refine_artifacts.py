#!/usr/bin/env python3
"""Write the golden fixtures' third-level refine and split-distance artifacts
with the reference's own writers (run where the reference is available; the
artifacts are committed, this script is how they were made).

For every fixture under tests/golden/ it regenerates the fixture's seeded
base vectors (the same draw tests/golden/make_golden.py made; the SHA-256 of
the raw file must equal the bundle's recorded raw_sha256) and writes
  * error4.refine -- the ERROR4 artifact of the final refine's mode 2
    (PQERR4V1 through tools/pq_refine_artifacts.py PqSource + generate_second
    for PQ bundles; SQERR4V1 through tools/generate_final_refine.py SqSource
    + generate_second for SQ bundles, with codec.json as its source manifest);
  * correction_bias.f32 -- the SQMD split-distance bias
    (tools/generate_sqmd_correction_bias.py), for the 4-bit SQ fixture only
    (split distance needs 4-bit L1 codes).
Then run tests/golden/make_cli_golden.py to record the reference CLI on them.

Usage: python tests/golden/make_refine_artifacts.py --reference REFERENCE_CHECKOUT (or $ROVER_REFERENCE)
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys
import tempfile
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from rover_b200 import bundle as B  # noqa: E402
from rover_b200 import datasets as D  # noqa: E402

GOLDEN = Path(__file__).resolve().parent
sys.path.insert(0, str(GOLDEN))
from make_golden import PQ_FIXTURES, SQ_FIXTURES  # noqa: E402


def _sha(path: Path) -> str:
    return hashlib.sha256(path.read_bytes()).hexdigest()


def _base(d: Path, n: int, dim: int, comps: int, seed: int, tmp: Path) -> Path:
    base = D.gmm(n, dim, comps, seed)
    path = tmp / "base.fvecs"
    B.write_fvecs(path, base)
    want = json.loads((d / "index.json").read_text())["raw_sha256"]
    if _sha(path) != want:
        raise SystemExit(f"{d.name}: regenerated base vectors differ from the bundle's raw_sha256")
    return path


def _fresh(path: Path) -> None:
    for p in (path, path.with_suffix(".json")):
        if p.exists():
            p.unlink()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("ROVER_REFERENCE"),
                    required="ROVER_REFERENCE" not in os.environ,
                    help="reference checkout (default: $ROVER_REFERENCE)")
    args = ap.parse_args()
    sys.path.insert(0, str(Path(args.reference) / "tools"))
    import generate_final_refine as gfr
    import generate_sqmd_correction_bias as gbias
    import pq_refine_artifacts as pra

    for name, n, dim, comps, m, code_bits, rbits, *_rest, seed in PQ_FIXTURES:
        d = GOLDEN / name
        with tempfile.TemporaryDirectory() as tmp:
            base = _base(d, n, dim, comps, seed, Path(tmp))
            out = d / "error4.refine"
            _fresh(out)
            source = pra.PqSource(d / "index", base, rbits)
            paths = [d / f"index.pqcodes", d / f"index.pqres{rbits}", d / f"index.pqres{rbits}.qparams"]
            pra.generate_second(source, out, paths, d / "index.pqbook")
        print(name, "error4.refine", out.stat().st_size, flush=True)

    for name, n, dim, comps, sq_bits, rbits, *_rest, seed in SQ_FIXTURES:
        d = GOLDEN / name
        codec = d / "codec.json"
        files = {key: {"path": f"{key}.bin", "bytes": (d / f"{key}.bin").stat().st_size,
                       "sha256": _sha(d / f"{key}.bin")} for key in ("l1", "residual", "qparams")}
        codec.write_text(json.dumps(dict(N=n, dim=dim, layout="original", order=None, **files), indent=2) + "\n")
        with tempfile.TemporaryDirectory() as tmp:
            base = _base(d, n, dim, comps, seed, Path(tmp))
            out = d / "error4.refine"
            _fresh(out)
            source = gfr.SqSource(codec, base)
            pra.generate_second(source, out, [d / "l1.bin", d / "residual.bin", d / "qparams.bin"])
        print(name, "error4.refine", out.stat().st_size, flush=True)
        if sq_bits == 4:
            bias = d / "correction_bias.f32"
            if bias.exists():
                bias.unlink()
            gbias.generate(codec, bias, 512)
            print(name, "correction_bias.f32", bias.stat().st_size, flush=True)


if __name__ == "__main__":
    main()

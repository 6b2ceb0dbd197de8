"""Generates the golden fixtures of tests/golden/ from the reference checkout.

    python tests/golden/make_golden.py [REFERENCE_DIR]

* test_dat_f32.npy - the reference's only test input (test_dat.txt, 100,000 x 2),
  parsed exactly as importNDDataset does (import_dataset.cpp:49-95, via the
  oracle's restatement) and stored as float32.
* known_answers.json - the README's known answer for that input (README.md:80-84:
  27,982,028 neighbours at eps=1.0, 2-D, float, no optimisations) next to the
  oracle's counts under each arithmetic model, and a digest of the oracle's
  sorted per-point lists.
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import pyoracle as O  # noqa: E402


def lists_digest(counts, nbrs) -> str:
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(counts, dtype=np.uint32).tobytes())
    h.update(np.ascontiguousarray(nbrs, dtype=np.uint32).tobytes())
    return h.hexdigest()


def main(ref: str) -> None:
    pts = O.import_text(os.path.join(ref, "test_dat.txt"), 2, np.float32)
    np.save(os.path.join(HERE, "test_dat_f32.npy"), pts)
    out = {"input": "test_dat_f32.npy", "eps": 1.0, "dim": 2, "readme_known_answer": 27982028}
    for name, model in (("device", O.MODEL_DEVICE), ("host", O.MODEL_HOST), ("fp64", O.MODEL_FP64)):
        c, tot, cand = O.join_counts(pts, 1.0, O.OracleConfig(k=2, model=model))
        out[f"oracle_total_{name}"] = tot
        if name == "device":
            out["candidates_full"] = cand
            counts, offs, nbrs = O.join_lists(pts, 1.0, O.OracleConfig(k=2, model=model))
            out["lists_sha256_device"] = lists_digest(counts, nbrs)
    _, tot, cand = O.join_counts(pts, 1.0, O.OracleConfig(k=2, stamp_ref=True))
    out["oracle_total_stamp_ref"] = tot
    out["candidates_stamp"] = cand
    with open(os.path.join(HERE, "known_answers.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print(json.dumps(out, indent=1, sort_keys=True))


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GSJ_REFERENCE_DIR", "")
    if not ref:
        sys.exit("usage: make_golden.py REFERENCE_DIR (or set GSJ_REFERENCE_DIR)")
    main(ref)

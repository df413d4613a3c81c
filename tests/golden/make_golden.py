"""Regenerates tests/golden/oracle_images.npz: per-iteration images of every
parity case rendered by the reference's own render loop compiled for the CPU
(oracle/_ref/libupbp_ref_cpu.so, built by `make -C oracle`).

    python tests/golden/make_golden.py [case ...]

With case names, only those cases are rendered and merged into the existing
fixtures.
"""
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, HERE)

import ref_cpu  # noqa: E402
from cases import CASES, prepare  # noqa: E402


def main():
    only = sys.argv[1:]
    out, meta = {}, {}
    if only:
        with np.load(os.path.join(HERE, "oracle_images.npz")) as old:
            out = {k: old[k] for k in old.files if k.split("/")[0] not in only}
        with open(os.path.join(HERE, "oracle_counts.json")) as f:
            meta = {k: v for k, v in json.load(f).items() if k not in only}
    with tempfile.TemporaryDirectory() as tmp:
        for name, (workload, tiny, _, iters) in CASES.items():
            if only and name not in only:
                continue
            r = ref_cpu.RefRenderer(prepare(name, tmp), threads=0)
            meta[name] = []
            for it in range(iters):
                out[f"{name}/{it}"] = r.run_iteration(it)
                st = r.stats()
                meta[name].append({k: st[k] for k in ("vertices", "surface", "medium", "beams")})
            r.close()
            print(name, meta[name], flush=True)
    np.savez_compressed(os.path.join(HERE, "oracle_images.npz"), **out)
    with open(os.path.join(HERE, "oracle_counts.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()

"""Regenerates tests/golden/cfg0_oracle.npz from the FP64 oracle.

    python tests/golden/make_golden.py

Stores, per field of config 0 (seed 0): 4096 sampled voxel values of the
oracle's tick output, the FP64 sum and L2 norm of the whole output, and the
first 16 values of the input generator streams (to pin the generator).
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (HERE, ROOT, os.path.join(ROOT, "vf-version_7_3_b200"), os.path.join(ROOT, "oracle")):
    sys.path.insert(0, p)

import numpy as np  # noqa: E402

import golden_cfg  # noqa: E402


def main():
    fields = golden_cfg.cfg0_inputs()
    V = fields[0][0].size
    sample_idx = np.random.default_rng(7).choice(V, 4096, replace=False).astype(np.int64)
    sample, sums, l2, gen_u, gen_i, gen_a = [], [], [], [], [], []
    for f, (u, idx, amt) in enumerate(fields):
        out = golden_cfg.cfg0_oracle_field(f, u, idx, amt)
        sample.append(out.ravel()[sample_idx])
        sums.append(out.sum())
        l2.append(np.sqrt((out ** 2).sum()))
        gen_u.append(u.ravel()[:16])
        gen_i.append(idx[:16])
        gen_a.append(amt[:16])
    np.savez_compressed(os.path.join(HERE, "cfg0_oracle.npz"), sample_idx=sample_idx,
                        sample=np.array(sample), sums=np.array(sums), l2=np.array(l2),
                        gen_u=np.array(gen_u), gen_idx=np.array(gen_i), gen_amt=np.array(gen_a))


if __name__ == "__main__":
    main()

"""Config-0 fixture definition shared by make_golden.py and the tests.

Config 0: 8 fields on a 64x64x32 grid (nx, ny, nz), values U[0, 1e-3],
500 sources per field, lognormal(-6, 1), Gaussian sigma per field, decay per
substep, 1 substep, zero padding, seed 0.  Inputs come from libvfd's
counter-based generator (host code, no GPU needed).
"""
import numpy as np

import oracle
from vfd import configs


def cfg0_inputs():
    c = configs.CFG0
    return configs.field_inputs(c["seed"], 0, c["grid"], c["n_sources"])


def cfg0_oracle_field(f, u, idx, amt):
    """FP64 oracle tick of field f: 1 substep, zero padding, then deposit."""
    c = configs.CFG0
    return oracle.tick(u, c["sigma"][f], c["decay"][f], c["substeps"], idx, amt)

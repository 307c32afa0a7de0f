"""Workload definitions (synthetic, seeded) of the five diffusion
configurations: field shapes, kernel widths, decay rates, source counts.

Grids are written nx x ny x nz (x fastest).  The eight fields are the
reference's cytokines in chemical_t order (src/enums.h:124-138):
TNF, TGF, FGF, MMP8, IL1, IL6, IL8, IL10.  No public dataset is involved:
all values come from the counter-based generator in libvfd
(vfd_synth_field / vfd_synth_sources).
"""
import numpy as np

FIELDS = ["TNF", "TGF", "FGF", "MMP8", "IL1", "IL6", "IL8", "IL10"]
SIGMA0 = [1.2, 0.9, 1.0, 0.8, 1.1, 1.0, 1.3, 0.9]
DECAY0 = [0.05, 0.01, 0.02, 0.03, 0.05, 0.04, 0.06, 0.02]
VALUE_RANGE = (0.0, 1e-3)
SOURCE_MU, SOURCE_SIGMA = -6.0, 1.0


def radius(sigma):
    return int(np.ceil(3.0 * sigma))


# Small world: 64x64x32, 1 substep, 500 sources per field, zero padding.
CFG0 = dict(name="plain-small-64x64x32", grid=(64, 64, 32), sigma=SIGMA0, decay=DECAY0,
            n_sources=500, substeps=1, ticks=1, seed=0)
# Human-scale world: 512x256x384, sigma x1.5, 200k sources, 10 substeps x 20 ticks.
CFG1 = dict(name="human-scale-512x256x384", grid=(512, 256, 384),
            sigma=[1.5 * s for s in SIGMA0], decay=DECAY0, n_sources=200_000,
            substeps=10, ticks=20, seed=0)
# Large-world stress: 768x384x576, sigma x2, 1M sources, 10 substeps.
CFG4 = dict(name="large-768x384x576", grid=(768, 384, 576),
            sigma=[2.0 * s for s in SIGMA0], decay=DECAY0, n_sources=1_000_000,
            substeps=10, ticks=1, seed=0)

# Batched ensemble: 32 worlds of uneven size, per-world sigma and decay
# multipliers uniform in [0.5, 2], 10 substeps, 500 sources per field.
CFG2_SIZES = [(96, 64, 64), (128, 96, 96), (192, 128, 128), (256, 128, 192)]


def cfg2_worlds(n_worlds=32, seed=0):
    rng = np.random.default_rng(seed)
    worlds = []
    for w in range(n_worlds):
        grid = CFG2_SIZES[int(rng.integers(0, len(CFG2_SIZES)))]
        sm = rng.uniform(0.5, 2.0, size=8)
        dm = rng.uniform(0.5, 2.0, size=8)
        worlds.append(dict(world=w, grid=grid, sigma=[s * m for s, m in zip(SIGMA0, sm)],
                           decay=[d * m for d, m in zip(DECAY0, dm)], n_sources=500))
    return worlds


CFG2 = dict(name="ensemble-32-worlds", n_worlds=32, substeps=10, seed=0)

# Served requests: grids with probabilities, Poisson 200 req/s, 50 ticks each,
# 1e3..2e5 sources, HBM budget 150 GB.
CFG3 = dict(name="served-requests", grids=[(64, 64, 32), (128, 96, 96), (256, 128, 192), (512, 256, 384)],
            probs=[0.4, 0.3, 0.2, 0.1], rate_hz=200.0, ticks_per_request=50,
            sources=(1_000, 200_000), hbm_budget_bytes=150 * 10**9, seed=0)


def voxels(grid):
    return grid[0] * grid[1] * grid[2]


def field_inputs(cfg_seed, world, grid, n_sources, n_fields=8):
    """Deterministic (u, idx, amt) per field for one world."""
    from . import synth_field, synth_sources
    nx, ny, nz = grid
    out = []
    for f in range(n_fields):
        u = synth_field(cfg_seed, world, f, (nz, ny, nx), *VALUE_RANGE)
        idx, amt = synth_sources(cfg_seed, world, f, n_sources, nx * ny * nz, SOURCE_MU, SOURCE_SIGMA)
        out.append((u, idx, amt))
    return out

"""Host side of a box shared by several contexts (CPU): the source shares cover every source
once and balance the luminosity, and the per-context totals add up to the box's."""
import numpy as np
import pytest

from flexrt_imaging_reion_b200 import partition as P, workloads as W


def test_source_shares_cover_and_balance():
    _, lum = W.grid_sources(W.make_inputs(W.config_M()))
    for world in (1, 2, 3, 8):
        masks = P.source_owner_masks(lum, world)
        tot = np.sum(masks, axis=0)
        assert (tot == 1).all()
        counts = [int(m.sum()) for m in masks]
        assert max(counts) - min(counts) <= 1
        share = [float(np.sum(np.asarray(lum)[m == 1])) for m in masks]
        # round robin from the brightest: no share exceeds another by more than the brightest source
        assert max(share) - min(share) <= float(np.max(lum)) * (1 + 1e-12)
    with pytest.raises(ValueError):
        P.source_owner_masks(lum, 0)


def test_sum_stats():
    a = {"rays_alive": 3, "crossings": 10, "lit_cells": 7, "photons_emitted": 1.5, "t": 2.0, "dt": 0.5,
         "error_flags": 0}
    b = {"rays_alive": 4, "crossings": 11, "lit_cells": 7, "photons_emitted": 2.5, "t": 2.0, "dt": 0.5,
         "error_flags": 2}
    s = P.sum_stats([a, b])
    assert s["rays_alive"] == 7 and s["crossings"] == 21 and s["lit_cells"] == 7
    assert s["photons_emitted"] == 4.0 and s["t"] == 2.0 and s["dt"] == 0.5 and s["error_flags"] == 2

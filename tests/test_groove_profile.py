"""get_groove_profile (reference Python/physics_engine.py:1903-1932) against a row-by-row
restatement of its definition, on a real electrode mask with random damage."""
import types

import numpy as np
import pytest

from tests.helpers import load
from thruster_cx_code_b200.physics_engine import DigitalTwinSimulator


def _by_rows(mask, depth, face):
    """Per row: depth at the first / last mask column, or the largest depth over the
    columns the mask occupies anywhere; rows without mask cells read 0."""
    ny, nx = mask.shape
    occupied = [j for j in range(nx) if mask[:, j].any()]
    out = np.zeros(ny)
    for i in range(ny):
        js = [j for j in range(nx) if mask[i, j]]
        if not js:
            continue
        if face == "upstream":
            out[i] = depth[i, js[0]]
        elif face == "downstream":
            out[i] = depth[i, js[-1]]
        else:
            out[i] = max(depth[i, j] for j in occupied)
    return out * 1000.0


@pytest.fixture(scope="module")
def state():
    d = load("domain_c1_half.npz")
    ny, nx = int(d["ny"]), int(d["nx"])
    rng = np.random.default_rng(3)
    grids = np.asarray(d["mask_grids"]) if "mask_grids" in d.files else None
    if grids is None:
        pytest.skip("domain fixture has no per-grid masks")
    eroded = rng.uniform(0.0, 0.05, (ny, nx)) * (rng.uniform(size=(ny, nx)) < 0.2)
    damage = rng.uniform(0.0, 2e3, (ny, nx))
    return types.SimpleNamespace(mask_grids=[g.astype(bool) for g in grids], eroded_depth=eroded,
                                 damage_map=damage, ny=ny, nx=nx, dy=float(d["dy"]))


@pytest.mark.parametrize("face", ["upstream", "downstream", "any"])
@pytest.mark.parametrize("thresh", [None, 5e3])
def test_profile_equals_row_definition(state, face, thresh):
    for g in range(len(state.mask_grids)):
        y, prof = DigitalTwinSimulator.get_groove_profile(state, g, thresh=thresh, face=face)
        depth = state.eroded_depth + ((state.damage_map / thresh) * state.dy if thresh else 0.0)
        assert np.array_equal(y, np.arange(state.ny) * state.dy)
        assert np.array_equal(prof, _by_rows(state.mask_grids[g], depth, face))


def test_profile_edge_cases(state):
    assert [a.size for a in DigitalTwinSimulator.get_groove_profile(state, 99)] == [0, 0]
    empty = types.SimpleNamespace(**{**vars(state), "mask_grids": [np.zeros((state.ny, state.nx), bool)]})
    assert [a.size for a in DigitalTwinSimulator.get_groove_profile(empty, 0)] == [0, 0]
    with pytest.raises(ValueError, match="face must be"):
        DigitalTwinSimulator.get_groove_profile(state, 0, face="side")

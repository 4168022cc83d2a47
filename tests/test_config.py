"""config.json front end against the reference's parser (fixtures from
tests/golden/make_config_golden.py, which ran parse_config of
Python/run_simulation_from_config.py on the same three configs)."""
import json
import os

import numpy as np
import pytest

from thruster_cx_code_b200.config import apply_config, parse_config

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _cases():
    with open(os.path.join(GOLDEN, "config_cases.json")) as f:
        return json.load(f)


@pytest.mark.parametrize("name", ["minimal", "full", "custom_material_tables"])
def test_parse_config_matches_reference(name, tmp_path, monkeypatch):
    case = _cases()[name]
    path = tmp_path / "config.json"
    path.write_text(json.dumps(case["config"]))
    monkeypatch.chdir(GOLDEN)  # table paths are relative to the fixture directory
    params, out = parse_config(str(path))
    assert out == case["output_selection"]
    ref = dict(case["params"])
    mat_name, props = params.pop("_material")
    assert [mat_name, props] == ref.pop("_material")
    store = params.pop("_cs_store")
    ref_store = ref.pop("_cs_store")
    assert sorted(store) == sorted(ref_store)
    for label, ds in store.items():
        r = ref_store[label]
        np.testing.assert_array_equal(ds["energy"], r["energy"])
        np.testing.assert_array_equal(ds["cs"], r["cs"])
        np.testing.assert_array_equal(ds["spline"].get_knots(), r["knots"])
        np.testing.assert_allclose(ds["spline"].get_coeffs(), r["coeffs"], rtol=1e-15, atol=0)
    assert params == ref


def test_parse_config_needs_grids(tmp_path):
    path = tmp_path / "c.json"
    path.write_text("{}")
    with pytest.raises(ValueError, match="No grids"):
        parse_config(str(path))
    with pytest.raises(FileNotFoundError):
        parse_config(str(tmp_path / "missing.json"))


class _SimStub:
    q = 1.602e-19

    def set_material(self, name=None, props=None):
        self.material = (name, props)


def test_apply_config_sets_species_and_material():
    params, _ = parse_config(_cases()["full"]["config"])
    s = _SimStub()
    rest = apply_config(s, params)
    assert s.Z_ion == 2 and s.q_ion == 2 * s.q
    assert s.m_ion == 83.798 * 1.6605e-27 and s.m_e == s.m_ion / 400.0
    assert s.material[1]["k"] == 21.9  # the Titanium preset
    assert "_material" not in rest and "beam_mass_amu" not in rest and rest["sim_mode"] == "Erosion"

"""Golden outputs of the reference's config parser (parse_config in
Python/run_simulation_from_config.py:30-194) for three configs written here, saved as
config_cases.json next to this file.  Run where the reference checkout is mounted, naming
its root in PYBEMCS_REFERENCE:

    PYBEMCS_REFERENCE=<checkout root> python tests/golden/make_config_golden.py

The cross-section tables in config/ are data of this test (a power law and a linear
yield), not reference files.
"""
import importlib.util
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from tests.golden.reference_loader import REFERENCE_ROOT, load_engine  # noqa: E402

CASES = {
    "minimal": {"grids": [{"V": 1000.0}]},
    "full": {
        "beam_species": {"mass_amu": 83.798, "charge_state": 2},
        "grid_material": {"preset": "Titanium"},
        "advanced_settings": {"neut_x": 12.5, "neut_r": 2.0, "V_plasma_offset": 15.0, "m_e_ratio": 400.0,
                              "Lx": 10.0, "Ly": 2.0},
        "simulation": {"n0_plasma": 2e17, "Te_up": 4.0, "Ti": 0.2, "Tn": 350.0, "n0": 3e19, "Accel": 0.2,
                       "Thresh": 5e8, "sim_mode": "Erosion", "geometry": "one_hole"},
        "rf_co_extraction": {"rf_enable": True, "rf_grid_idx": 1, "rf_freq": 2.0, "rf_amp": 150.0},
        "neutralizer": {"neut_rate": 12, "Te": 2.5},
        "grids": [{"V": 1500.0, "t": 0.4, "gap": 0.8, "r": 1.0}, {"V": -250.0, "t": 0.6, "r": 0.6, "cham": 10.0},
                  {"t": 0.5, "gap": 1.2}],
        "terminal_output": {"beam_divergence": False, "iteration_time": False},
    },
    "custom_material_tables": {
        "grid_material": {"preset": "my alloy", "k": 90.0, "Y_coeff": 2e-4},
        "cross_sections": {"cx_file": "config/cx_table.txt", "see_file": "config/see_table.csv",
                           "custom_file": "", "spline_smoothing": 0.0},
        "grids": [{"V": 1000.0, "t": 0.38, "gap": 1.0, "r": 0.95}, {"V": -200.0, "t": 1.0, "gap": 1.0, "r": 0.55}],
    },
}


def serialise(params, out):
    p = dict(params)
    name, props = p.pop("_material")
    store = p.pop("_cs_store")
    p["_material"] = [name, props]
    p["_cs_store"] = {k: {"energy": list(map(float, v["energy"])), "cs": list(map(float, v["cs"])),
                          "knots": list(map(float, v["spline"].get_knots())),
                          "coeffs": list(map(float, v["spline"].get_coeffs()))} for k, v in store.items()}
    return {"params": p, "output_selection": out}


def main():
    sys.modules["physics_engine"] = load_engine(name="physics_engine")
    spec = importlib.util.spec_from_file_location(
        "_ref_runner", os.path.join(REFERENCE_ROOT, "Python", "run_simulation_from_config.py"))
    runner = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(runner)
    results = {}
    cwd = os.getcwd()
    os.chdir(HERE)  # table paths in the configs are relative to this directory
    try:
        for name, cfg in CASES.items():
            path = os.path.join(HERE, f"_tmp_{name}.json")
            with open(path, "w") as f:
                json.dump(cfg, f)
            try:
                results[name] = {"config": cfg, **serialise(*runner.parse_config(path))}
            finally:
                os.remove(path)
    finally:
        os.chdir(cwd)
    with open(os.path.join(HERE, "config_cases.json"), "w") as f:
        json.dump(results, f, indent=1)
    print("wrote config_cases.json")


if __name__ == "__main__":
    main()

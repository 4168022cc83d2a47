"""config.json front end: the reference's run-configuration schema as the request format.

``parse_config`` reads the sections of the reference's ``config.json`` with the same keys
and defaults as ``parse_config`` in Python/run_simulation_from_config.py:30-194:
``beam_species``, ``grid_material`` (preset or custom), ``advanced_settings``,
``cross_sections`` (log-log cubic splines of two-column tables), ``simulation``,
``rf_co_extraction``, ``neutralizer``, ``grids`` and ``terminal_output``, plus a ``gpu``
section the reference does not read (``neutral_profile``: ``point_source`` or ``uniform``;
``sputter_exponent``: the power of the sputter yield, 1 for the reference's linear law).  It returns
``(params, output_selection)``.  ``apply_config`` then sets up a simulator the way the
reference runner does before ``build_domain`` (:209-231): species mass and charge,
electron mass ratio, material, cross-section store.  A config can also be given as a dict,
for the served mode.
"""
import json
import os

import numpy as np

from .physics_engine import MATERIAL_PRESETS

AMU = 1.6605e-27


def _load_table(fpath, smoothing):
    from scipy.interpolate import UnivariateSpline
    try:
        raw = np.loadtxt(fpath, delimiter=None, comments='#')
    except Exception:
        raw = np.loadtxt(fpath, delimiter=',', comments='#', skiprows=1)
    if raw.ndim != 2 or raw.shape[1] < 2:
        raise ValueError(f"{fpath} must have at least 2 columns")
    order = np.argsort(raw[:, 0])
    energy, cs = raw[order, 0], raw[order, 1]
    spline = UnivariateSpline(np.log10(np.maximum(energy, 1e-30)), np.log10(np.maximum(cs, 1e-50)), s=smoothing, k=3)
    spline._pb_smoothing = float(smoothing)  # kept with the table, so checkpoints rebuild the same spline
    return energy, cs, spline


def parse_config(config):
    """``config``: a path to a JSON file or an already-loaded dict.  Returns
    ``(params, output_selection)``.  ``params`` holds the step/build keys plus the private
    entries ``beam_mass_amu``, ``beam_charge_state``, ``_material`` and ``_cs_store`` that
    ``apply_config`` consumes."""
    if isinstance(config, (str, os.PathLike)):
        if not os.path.isfile(config):
            raise FileNotFoundError(f"Config file '{config}' not found.")
        with open(config, 'r', encoding='utf-8') as f:
            cfg = json.load(f)
    else:
        cfg = dict(config)
    params = {}
    beam = cfg.get('beam_species', {})
    params['beam_mass_amu'] = beam.get('mass_amu', 131.293)
    params['beam_charge_state'] = beam.get('charge_state', 1)

    mat = cfg.get('grid_material', {})
    name = str(mat.get('preset', 'Molybdenum')).strip()
    if name in MATERIAL_PRESETS:
        params['_material'] = (name, dict(MATERIAL_PRESETS[name]))
    else:
        defaults = MATERIAL_PRESETS['Molybdenum']
        params['_material'] = ('Custom', {k: mat.get(k, defaults[k]) for k in defaults})

    adv = cfg.get('advanced_settings', {})
    for key, default in (('neut_x', 19.9), ('neut_r', 3.0), ('V_plasma_offset', 20.0), ('m_e_ratio', 1000.0),
                         ('Lx', 20.0), ('Ly', 3.0)):
        params[key] = adv.get(key, default)

    cs_cfg = cfg.get('cross_sections', {})
    smoothing = cs_cfg.get('spline_smoothing', 0.0)
    store = {}
    for label, key in (('CX', 'cx_file'), ('SEE', 'see_file'), ('Custom', 'custom_file')):
        fpath = str(cs_cfg.get(key, '')).strip()
        if not fpath:
            continue
        if not os.path.isfile(fpath):
            print(f"Warning: cross-section file not found for {label}: {fpath}")
            continue
        try:
            energy, cs, spline = _load_table(fpath, smoothing)
        except Exception as e:
            print(f"Warning: failed to load {label} CS from {fpath}: {e}")
            continue
        store[label] = {'energy': energy, 'cs': cs, 'spline': spline, 'type': label}
    params['_cs_store'] = store

    sim = cfg.get('simulation', {})
    for key, default in (('n0_plasma', 1e17), ('Te_up', 3.0), ('Ti', 2.0), ('Tn', 300.0), ('n0', 1e20),
                         ('Accel', 0.1), ('Thresh', 10000.0), ('sim_mode', 'Both'), ('geometry', 'half_hole')):
        params[key] = sim.get(key, default)

    rf = cfg.get('rf_co_extraction', {})
    for key, default in (('rf_enable', False), ('rf_grid_idx', 0), ('rf_freq', 13.56), ('rf_amp', 500.0)):
        params[key] = rf.get(key, default)

    neut = cfg.get('neutralizer', {})
    params['neut_rate'] = neut.get('neut_rate', 0)
    params['Te'] = neut.get('Te', 5.0)

    params['grids'] = [{'V': g.get('V', 0.0), 't': g.get('t', 1.0), 'gap': g.get('gap', 1.0), 'r': g.get('r', 1.0),
                        'cham': g.get('cham', 0.0)} for g in cfg.get('grids', [])]
    if not params['grids']:
        raise ValueError("No grids found in config.json. Add at least one entry in the 'grids' list.")

    # options of this implementation that the reference ignores (a section it never reads)
    gpu = cfg.get('gpu', {})
    for key in ('neutral_profile', 'sputter_exponent'):
        if key in gpu:
            params[key] = gpu[key]

    out = cfg.get('terminal_output', {})
    output_selection = {k: out.get(k, True) for k in ('grid_temperatures', 'beam_divergence',
                                                      'saddle_point_potential', 'mean_particle_energy',
                                                      'iteration_time')}
    return params, output_selection


def apply_config(sim, params):
    """Apply the species, material and cross-section entries of ``params`` to ``sim``
    (removing them from ``params``) and return ``params`` for build_domain and step."""
    mass_amu = params.pop('beam_mass_amu', 131.293)
    charge = params.pop('beam_charge_state', 1)
    sim.m_ion = mass_amu * AMU
    sim.m_XE = sim.m_ion
    sim.Z_ion = charge
    sim.q_ion = charge * sim.q
    sim.m_e = sim.m_ion / params.get('m_e_ratio', 1000.0)
    _, props = params.pop('_material', ('Molybdenum', None))
    if props:
        sim.set_material(props=props)
    else:
        sim.set_material(name='Molybdenum')
    sim.user_cs = params.pop('_cs_store', {})
    return params

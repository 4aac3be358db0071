"""Host-side mirror of SAMoS's class-factory plugin API for the hot path.

Each ``resolve_*`` function restates one reference constructor: it takes the
conf-file parameter map (``pairs_type``: strings; flags map to ``""``),
rejects unknown keys where the reference does (``params_ok``), applies the
reference defaults, and returns the numeric vectors the C ABI expects.
Factory names are those of src/utils/register_*.cpp.

:class:`Simulation` plays the part of src/samos.cpp's command loop for the
hot-path commands (box, input, nlist, constraint, pair_potential,
pair_param, pair_align, align_param, external, timestep, integrator, run)
and forwards to a backend -- :class:`samos_b200.engine.Engine` in production.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import engine as E

DEFAULT_CUTOFF = 3.0   # src/system/defaults.hpp:34
DEFAULT_PADDING = 0.5  # src/system/defaults.hpp:35


class PluginError(RuntimeError):
    """Raised where the reference logs Messenger::ERROR and throws."""


def _known(params: dict, known: list[str], what: str) -> None:
    # PairPotential::params_ok / Integrator::params_ok
    for k in params:
        if k not in known:
            raise PluginError(f'Unknown parameter "{k}" in {what}.')


def _f(params: dict, key: str, default: float) -> float:
    return float(params[key]) if key in params else float(default)


def _value(kind: str, params: dict) -> list[float]:
    """Value object (src/system/value.hpp:59-178) -> [kind, min, max, steps]."""
    if kind not in ("constant", "linear"):
        raise PluginError(f"Unknown value type {kind}.")
    vmin = _f(params, "min_val", 0.0)
    vmax = _f(params, "max_val", 1.0)
    steps = int(params["steps"]) if "steps" in params else 1000
    if kind == "linear":
        if vmax < vmin:
            raise PluginError("Value parameters are not properly set.")
        if steps <= 0:
            raise PluginError("Value parameters. Zero steps given.")
    return [0.0 if kind == "constant" else 1.0, vmin, vmax, float(steps)]


_PAIR_BASE = ["min_val", "max_val", "ntypes", "steps"]


@dataclass
class PairSpec:
    name: str
    kind: int
    glob: np.ndarray
    table: np.ndarray
    use_radii: bool = False
    phase_in: bool = False
    shifted: bool = False
    has_pair_params: bool = False
    phase_value: list = field(default_factory=lambda: [0.0, 0.0, 1.0, 1000.0])


def resolve_pair(name: str, params: dict, ntypes: int, nlist_cut: float) -> PairSpec:
    """pair_potential <name> {...}: soft / lj / morse / gaussian."""
    g = np.zeros(E.PAIR_NPARAM)
    spec_flags = dict(use_radii="use_particle_radii" in params, phase_in="phase_in" in params,
                      shifted="shifted" in params)
    if name == "soft":  # pair_soft_potential.hpp:63-121
        _known(params, _PAIR_BASE + ["k", "a", "use_particle_radii", "phase_in"], "soft potential")
        g[0] = _f(params, "k", 1.0)
        g[1] = _f(params, "a", 2.0)
        spec_flags["shifted"] = False
    elif name == "lj":  # pair_lj_potential.hpp:61-159
        _known(params, _PAIR_BASE + ["epsilon", "sigma", "rcut", "use_particle_radii", "phase_in",
                                     "shifted", "WCA"], "Lennard-Jones potential")
        g[0] = _f(params, "epsilon", 1.0)
        g[1] = _f(params, "sigma", 1.0)
        g[2] = _f(params, "rcut", 3.0)
        if "WCA" in params:
            g[2] = 1.122462048309373 * g[1]
            spec_flags["shifted"] = True
    elif name == "morse":  # pair_morse_potential.hpp:61-160
        _known(params, _PAIR_BASE + ["D", "a", "re", "rcut", "use_particle_radii", "phase_in",
                                     "shifted"], "Morse potential")
        g[0] = _f(params, "D", 1.0)
        g[1] = _f(params, "a", 1.0)
        g[2] = _f(params, "re", 1.0)
        g[3] = _f(params, "rcut", 2.5 * g[2])
    elif name == "gaussian":  # pair_gaussian_potential.hpp:66-194 (no params_ok there)
        g[0] = _f(params, "A", 2.0)
        g[1] = _f(params, "B", -1.0)
        g[2] = _f(params, "alpha", 1.0)
        g[3] = _f(params, "beta", 3.0)
        g[4] = _f(params, "rA", 0.0)
        g[5] = _f(params, "rB", 1.5)
        g[6] = _f(params, "rcut", 3.0)
    else:
        raise PluginError(f"Unknown pair potential {name}.")
    if "ntypes" in params:
        ntypes = max(ntypes, int(params["ntypes"]))
    table = np.tile(g, ntypes * ntypes).reshape(ntypes, ntypes, E.PAIR_NPARAM).copy()
    if name == "gaussian":
        table[:, :, 1] = g[0]  # per-type default B = A (pair_gaussian_potential.hpp:174)
    phase = _value(params["phase_in"] or "constant", params) if "phase_in" in params else [0.0, 0.0, 1.0, 1000.0]
    return PairSpec(name, E.PAIR[name], g, table, phase_value=phase, **spec_flags)


_PAIR_TABLE_KEYS = {"soft": ["k", "a"], "lj": ["epsilon", "sigma", "rcut"],
                    "morse": ["D", "a", "re", "rcut"],
                    "gaussian": ["A", "B", "alpha", "beta", "rA", "rB", "rcut"]}


def apply_pair_param(spec: PairSpec, params: dict) -> None:
    """pair_param <name> {type_1; type_2; ...} -> set_pair_parameters."""
    if "type_1" not in params or "type_2" not in params:
        raise PluginError("Missing key for pair potential parameters.")
    t1, t2 = int(params["type_1"]) - 1, int(params["type_2"]) - 1
    for slot, key in enumerate(_PAIR_TABLE_KEYS[spec.name]):
        val = float(params[key]) if key in params else spec.glob[slot]
        if spec.name == "lj" and key == "rcut" and "WCA" in params:
            sigma = float(params["sigma"]) if "sigma" in params else spec.glob[1]
            val = 1.122462048309373 * sigma
            spec.shifted = True
        spec.table[t1, t2, slot] = val
        spec.table[t2, t1, slot] = val
    spec.has_pair_params = True


@dataclass
class AlignSpec:
    name: str
    kind: int
    J: float
    rcut: float
    table: np.ndarray
    has_pair_params: bool = False


def resolve_align(name: str, params: dict, ntypes: int, nlist_rcut: float) -> AlignSpec:
    """pair_align <name> {...}: polar / nematic / vicsek (pair_*_aligner.hpp)."""
    if name not in ("polar", "nematic", "vicsek"):
        raise PluginError(f"Unknown pair aligner {name}.")
    if "exclude_boundary" in params:
        raise PluginError("exclude_boundary (tissue boundaries) is not part of the GPU path.")
    J = _f(params, "J", 1.0) if name != "vicsek" else 0.0
    rcut = _f(params, "rcut", nlist_rcut)
    table = np.zeros((ntypes, ntypes, 2))
    table[:, :, 0] = J
    table[:, :, 1] = rcut
    return AlignSpec(name, E.ALIGN[name], J, rcut, table)


def apply_align_param(spec: AlignSpec, params: dict) -> None:
    """align_param <name> {type_1; type_2; J; rcut} -> set_pair_parameters."""
    if spec.name == "vicsek":
        return  # pair_vicsek_aligner.hpp:69-72 ignores per-pair parameters
    if "type_1" not in params or "type_2" not in params:
        raise PluginError("Missing key for pair alignment parameters.")
    t1, t2 = int(params["type_1"]) - 1, int(params["type_2"]) - 1
    J = float(params["J"]) if "J" in params else spec.J
    rc = float(params["rcut"]) if "rcut" in params else spec.rcut
    for a, b in ((t1, t2), (t2, t1)):
        spec.table[a, b, 0] = J
        spec.table[a, b, 1] = rc
    spec.has_pair_params = True


@dataclass
class ExternalSpec:
    name: str
    kind: int
    alpha: float
    type_alpha: np.ndarray
    has_params: bool = False


def resolve_external(name: str, params: dict, ntypes: int) -> ExternalSpec:
    """external self_propulsion {alpha} (external_self_propulsion.hpp:51-63)."""
    if name != "self_propulsion":
        raise PluginError(f"External potential {name} is not part of the GPU path.")
    alpha = _f(params, "alpha", 1.0)
    return ExternalSpec(name, E.EXTERNAL[name], alpha, np.full(ntypes, alpha))


def resolve_constraint(name: str, params: dict) -> tuple[int, list[float]]:
    """constraint <name> {...} (constraint.hpp:56-120, constraint_plane.hpp,
    constraint_sphere.hpp, constraint_cylinder.hpp, constraint_torus.hpp,
    constraint_ellipsoid.hpp, constraint_peanut.hpp, constraint_gyroid.hpp,
    constraint_hourglass.hpp, constraint_gaussian_bump.hpp, constraint_slab.hpp,
    constraint_plane_walls.hpp): returns (kind,
    [zpos|r|c|a|R|A, unlimited, maxiter, tol, rescale, rescale_steps,
    rescale_freq, second shape parameter, third shape parameter])."""
    if name not in E.CONSTRAINT:
        raise PluginError(f"Constraint {name} is not part of the GPU path.")
    if "group" in params and params["group"] != "all":
        raise PluginError("Constraint groups other than 'all' are not part of the GPU path.")
    maxiter = float(int(params["maxiter"])) if "maxiter" in params else 100.0
    tol = float(int(params["tol"])) if "tol" in params else 1e-6   # parsed as int, constraint.hpp:82
    rescale = _f(params, "rescale", 1.0)
    rescale_steps = _f(params, "rescale_steps", 1000.0)
    rescale_freq = _f(params, "rescale_freq", 10.0)
    second, third = 0.0, 0.0
    if name == "plane":
        first = _f(params, "zpos", 0.0)
        unlimited = 1.0 if "unlimited" in params else 0.0
    elif name in ("sphere", "cylinder"):  # constraint_sphere.hpp, constraint_cylinder.hpp:58-69
        first = _f(params, "r", 1.0)
        unlimited = 0.0
    elif name == "torus":  # constraint_torus.hpp: c (1), a (0.5)
        first, second, unlimited = _f(params, "c", 1.0), _f(params, "a", 0.5), 0.0
    elif name == "ellipsoid":  # constraint_ellipsoid.hpp: a, b, c (1)
        first, second, third, unlimited = _f(params, "a", 1.0), _f(params, "b", 1.0), _f(params, "c", 1.0), 0.0
    elif name == "peanut":  # constraint_peanut.hpp:62-88: a (10), b (8), b > a required
        first, second, unlimited = _f(params, "a", 10.0), _f(params, "b", 8.0), 0.0
        if second <= first:
            raise PluginError("Parameter b has to be larger than parameter a. Otherwise the surface will be "
                              "disconnected.")
    elif name == "hourglass":  # constraint_hourglass.hpp:64-102: R (10), A (1; if given, at most R), n (1)
        first, second, third, unlimited = _f(params, "R", 10.0), _f(params, "A", 1.0), _f(params, "n", 1.0), 0.0
        if "A" in params and second > first:
            raise PluginError("Hourglass constraint. Amplitude has to be smaller than the radius.")
    elif name == "gaussian_bump":  # constraint_gaussian_bump.hpp: A (1); widths a, b stored squared (1 if absent)
        first, second, third, unlimited = _f(params, "A", 1.0), _f(params, "a", 1.0), _f(params, "b", 1.0), 0.0
        second, third = second * second, third * third
    elif name == "slab":  # constraint_slab.hpp:56-78: z_lo (0), z_hi (1)
        first, second, unlimited = _f(params, "z_lo", 0.0), _f(params, "z_hi", 1.0), 0.0
    elif name == "walls":  # constraint_plane_walls.hpp:56-74: l (1; beyond the box: the box edge)
        first, unlimited = _f(params, "l", 1.0), 0.0
    elif name == "tetrahedron":  # constraint_tetrahedron.hpp:62-88: scale (10), value (1)
        first, second, unlimited = _f(params, "scale", 10.0), _f(params, "value", 1.0), 0.0
    else:
        first, unlimited = 0.0, 0.0
    return E.CONSTRAINT[name], [first, unlimited, maxiter, tol, rescale, rescale_steps, rescale_freq, second, third]


_INT_BASE = ["dt", "group", "temperature_control", "min_val", "max_val", "steps"]


def resolve_integrator(name: str, params: dict, dt_global: float) -> tuple[int, np.ndarray, list[float]]:
    """integrator <name> {...}: returns (kind, params[16], temperature value)."""
    p = np.zeros(E.INT_NPARAM)
    dt = _f(params, "dt", dt_global)
    if not dt > 0.0:
        raise PluginError("Integrator step has not been set.")
    p[0] = dt
    if name == "brownian":  # integrator_brownian.hpp:55-160
        _known(params, _INT_BASE + ["v0", "nu", "mu", "mur", "seed", "nematic", "tau", "velocity_align"],
               "brownian integrator")
        p[1] = _f(params, "v0", 1.0); p[2] = _f(params, "nu", 1.0)
        p[3] = _f(params, "mu", 1.0); p[4] = _f(params, "mur", 1.0)
        p[5] = float(int(params["seed"])) if "seed" in params else 0.0
        p[6] = 1.0 if "nematic" in params else 0.0
        p[7] = _f(params, "tau", 1.0)
        p[8] = 1.0 if "velocity_align" in params else 0.0
    elif name == "brownian_pos":  # integrator_brownian_pos.hpp:55-90
        _known(params, _INT_BASE + ["mu", "seed"], "brownian_pos integrator")
        p[3] = _f(params, "mu", 1.0)
        p[5] = float(int(params["seed"])) if "seed" in params else 0.0
    elif name == "brownian_align":  # integrator_brownian_align.hpp:55-127
        _known(params, _INT_BASE + ["nu", "mur", "seed", "nematic", "tau"], "brownian_align integrator")
        p[2] = _f(params, "nu", 1.0); p[4] = _f(params, "mur", 1.0)
        p[5] = float(int(params["seed"])) if "seed" in params else 0.0
        p[6] = 1.0 if "nematic" in params else 0.0
        p[7] = _f(params, "tau", 1.0)
    elif name == "langevin":  # integrator_langevin.hpp:64-116
        _known(params, _INT_BASE + ["gamma", "seed", "method"], "langevin integrator")
        p[5] = float(int(params["seed"])) if "seed" in params else 0.0
        p[9] = _f(params, "gamma", 1.0)
        method = params.get("method", "baoab").lower()
        if method not in ("baoab", "spv", "bbk"):
            raise PluginError("Unknown integration method")
        p[10] = {"baoab": 0, "spv": 1, "bbk": 2}[method]
    elif name == "fire":  # integrator_fire.hpp:58-154 (no params_ok there)
        p[1] = _f(params, "alpha", 0.1); p[2] = _f(params, "alpha_scale", 0.99)
        p[3] = _f(params, "f_tolerance", 1e-4); p[4] = _f(params, "e_tolerance", 1e-6)
        p[6] = _f(params, "dt_inc", 1.1); p[7] = _f(params, "dt_dec", 0.5)
        p[8] = _f(params, "dt_max", 1.0); p[9] = float(int(params["min_neg_steps"])) if "min_neg_steps" in params else 5.0
        p[11] = _f(params, "fmax_tolerance", 0.0)
    elif name == "vicsek":  # integrator_vicsek.hpp:55-105 (no params_ok there)
        p[1] = _f(params, "v0", 1.0); p[2] = _f(params, "eta", 0.1); p[3] = _f(params, "mu", 0.0)
        p[5] = float(int(params["seed"])) if "seed" in params else 0.0
    elif name == "nve":  # integrator_nve.hpp:59-75 (no params_ok there)
        if "limit" in params:
            p[12], p[13] = 1.0, float(params["limit"])
        if "angle_limit" in params:
            p[14], p[15] = 1.0, float(params["angle_limit"])
    else:
        raise PluginError(f"Integrator {name} is not part of the GPU path.")
    temp = _value(params.get("temperature_control", "constant"), params)
    return E.INTEGRATOR[name], p, temp


class Simulation:
    """The hot-path subset of the `samos` command loop over one backend.

    Pair potentials, aligners and integrators are handed to the backend in
    std::map key order at the first ``run`` (their construction has no side
    effect on the particles); constraints and the neighbour list act at once,
    as in src/samos.cpp:500-560.
    """

    def __init__(self, backend, ntypes: int = 1):
        self.b = backend
        self.ntypes = ntypes
        self.dt = 0.0
        self.nlist_rcut = None
        self.pairs: dict[str, PairSpec] = {}
        self.aligns: dict[str, AlignSpec] = {}
        self.externals: dict[str, ExternalSpec] = {}
        self.integrators: dict[str, tuple] = {}
        self.committed = False
        self.has_constraint = False
        self.groups: dict[str, int] = {}

    GROUP_CRITERIA = ("type", "not_type", "r_eq", "r_le", "r_ge", "x_le", "x_ge", "y_le", "y_ge", "z_le", "z_ge")

    def group(self, name, params=None):
        """group <name> {...} (samos.cpp:1108-1140, System::make_group,
        system.cpp:462-572): the particles meeting every given criterion, on
        the state at this command, in index order."""
        params = params or {}
        if name in ("boundary", "tissue"):
            raise PluginError('Groups "tissue" and "boundary" are reserved and cannot be used.')
        if name in self.groups:
            raise PluginError(f"Group {name} is already defined (adding to a group is not part of the GPU path).")
        if len(self.groups) >= 7:
            raise PluginError("More than 7 particle groups are not part of the GPU path.")
        unknown = [k for k in params if k not in self.GROUP_CRITERIA]
        if unknown:
            raise PluginError(f"Group criterion {unknown[0]} is not part of the GPU path.")
        tp = self.b.download("type")
        r = self.b.download("radius")
        xyz = {c: self.b.download(c) for c in "xyz"}
        add = np.ones(len(tp), bool)
        for k, v in params.items():
            if k == "type":
                add &= tp == int(v)
            elif k == "not_type":
                add &= tp != int(v)
            elif k.startswith("r_"):
                val = float(v)
                add &= {"eq": r == val, "le": r <= val, "ge": r >= val}[k[2:]]
            else:
                val, c = float(v), xyz[k[0]]
                add &= c <= val if k.endswith("_le") else c >= val
        idx = len(self.groups) + 1
        self.b.define_group(idx, add.astype(np.uint8))
        self.groups[name] = idx
    def box(self, lx, ly, lz, periodic=True):
        self.b.set_box(lx, ly, lz, periodic)

    def input(self, **arrays):
        for name, vals in arrays.items():
            self.b.upload(name, vals)

    def nlist(self, rcut=DEFAULT_CUTOFF, pad=DEFAULT_PADDING):
        self.nlist_rcut = float(rcut)
        self.b.set_nlist(float(rcut), float(pad))

    def constraint(self, name, params=None):
        kind, p = resolve_constraint(name, params or {})
        self.b.add_constraint(kind, p)
        self.has_constraint = True

    def pair_potential(self, name, params=None):
        if self.nlist_rcut is None:  # samos.cpp:347-352
            self.nlist(DEFAULT_CUTOFF, DEFAULT_PADDING)
        self.pairs[name] = resolve_pair(name, params or {}, self.ntypes, self.nlist_rcut)

    def pair_param(self, name, params):
        apply_pair_param(self.pairs[name], params)

    def pair_align(self, name, params=None):
        if self.nlist_rcut is None:
            self.nlist(DEFAULT_CUTOFF, DEFAULT_PADDING)
        self.aligns[name] = resolve_align(name, params or {}, self.ntypes, self.nlist_rcut)

    def align_param(self, name, params):
        apply_align_param(self.aligns[name], params)

    def external(self, name, params=None):
        self.externals[name] = resolve_external(name, params or {}, self.ntypes)

    def timestep(self, dt):
        self.dt = float(dt)
        self.b.set_timestep(self.dt)

    def integrator(self, name, params=None):
        params = params or {}
        group = params.get("group", "all")
        if group != "all" and group not in self.groups:
            raise PluginError(f"Group {group} is not defined.")
        key = name + "_" + group
        if key in self.integrators:
            raise PluginError(f"Integrator of type {name} (for group {group}) already exists.")
        self.integrators[key] = resolve_integrator(name, params, self.dt) + (self.groups.get(group, 0),)

    def commit(self):
        if self.committed:
            return
        for name in sorted(self.pairs):
            s = self.pairs[name]
            self.b.add_pair(s.kind, s.glob, s.table.reshape(-1), s.use_radii, s.phase_in, s.shifted,
                            s.has_pair_params, s.phase_value)
        for name in sorted(self.aligns):
            s = self.aligns[name]
            self.b.add_align(s.kind, s.J, s.rcut, s.table.reshape(-1), s.has_pair_params)
        for name in sorted(self.externals):
            s = self.externals[name]
            self.b.add_external(s.kind, s.alpha, s.type_alpha, s.has_params)
        for pos, key in enumerate(sorted(self.integrators)):
            kind, p, temp, group = self.integrators[key]
            self.b.add_integrator(kind, p, temp)
            if group:
                self.b.set_integrator_group(pos, group)
        self.committed = True

    def run(self, steps):
        if not self.has_constraint:
            raise PluginError("Constraint not defined.")
        if not self.integrators:
            raise PluginError("Integrator not defined.")
        self.commit()
        return self.b.run(int(steps))

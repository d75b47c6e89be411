"""Scene files: the reference's card-structured JSON/TOML format (config_builder.py,
params.py), restricted to the fluid and tensile-solid hot path.

``SimConfig(path).get_cfg(name)`` answers with the same flat canonical names and the
same resolved defaults as the reference's registry (params.py:256-1330) for every
parameter this package reads.  Keys the reference knows but this package does not
implement (detonation, damage models, velocity limiters, adaptive hourglass, ...) are
rejected with a SceneError rather than ignored, so a deck never runs silently without a
feature it asked for.  Unknown keys are rejected as the reference rejects them.
"""
from __future__ import annotations

import json
import math
import os
import re

try:
    import tomllib
except ImportError:  # pragma: no cover
    tomllib = None

from .materials import Material, MaterialError, derive_globals


class SceneError(ValueError):
    """A scene file that cannot be run as written (config_builder.py:56)."""


# --------------------------------------------------------------------------- comments
def strip_json_comments(text: str) -> str:
    """Remove '#' and '//' comments outside strings (the scene files carry them)."""
    out = []
    in_str = False
    esc = False
    i = 0
    n = len(text)
    while i < n:
        ch = text[i]
        if in_str:
            out.append(ch)
            if esc:
                esc = False
            elif ch == "\\":
                esc = True
            elif ch == '"':
                in_str = False
            i += 1
            continue
        if ch == '"':
            in_str = True
            out.append(ch)
            i += 1
            continue
        if ch == "#" or (ch == "/" and i + 1 < n and text[i + 1] == "/"):
            while i < n and text[i] != "\n":
                i += 1
            continue
        out.append(ch)
        i += 1
    return "".join(out)


# --------------------------------------------------------------------------- registry
# (flat name, card path, field, type, default).  Defaults are the reference's
# (params.py); a callable default is resolved after the literals.
def _colle(c):
    return str(c.get("PST_MODE") or "sun").lower() == "colle"


def _lambda_lo_default(c):
    return 0.2 if _colle(c) else 0.4


def _clamp_default(c):
    if _colle(c) and str(c.get("PST_MA_MODE") or "local").lower() != "fixed":
        return "both"
    return "displacement"


REGISTRY = [
    ("domainStart", ("Domain",), "start", "vec3", [0.0, 0.0, 0.0]),
    ("domainEnd", ("Domain",), "end", "vec3", [1.0, 1.0, 1.0]),
    ("particleRadius", ("Domain",), "particleRadius", "float", None),
    ("supportRadiusFactor", ("Domain",), "supportRadiusFactor", "float", 4.0),
    ("planeStrain", ("Domain",), "planeStrain", "bool", False),
    ("axisymmetric", ("Domain",), "axisymmetric", "bool", False),
    ("symmetryPlanes", ("Domain",), "symmetryPlanes", "str", ""),
    ("AXI_R_MIN", ("Domain",), "axisRadiusMin", "float", 0.5),
    ("AXI_CONSERVATIVE_X", ("Domain",), "conservativeAxialMomentum", "bool", True),
    ("AXI_CONSERVATIVE_R", ("Domain",), "conservativeRadialForce", "bool", False),
    ("AXI_IMAGE_RADIUS", ("Domain",), "axialImageRadius", "str", "ring"),
    ("DOMAIN_BOUNDARY", ("Domain",), "boundary", "str", "open"),
    ("DOMAIN_RESTITUTION", ("Domain",), "restitution", "float", 0.5),
    ("CFL", ("Time",), "CFL", "float", None),
    ("timeStepSize", ("Time",), "stepSize", "float", None),
    ("sim_duration", ("Time",), "duration", "float", None),
    ("maxSteps", ("Time",), "maxSteps", "int", None),
    ("numberOfStepsPerRenderUpdate", ("Time",), "stepsPerRenderUpdate", "int", None),
    ("DT_PAIR_SOUND_SPEED", ("Time",), "pairSoundSpeed", "str", "samematerial"),
    ("simulationMethod", ("Solver",), "type", "str", None),
    ("viscosity", ("Solver",), "viscosity", "float", None),
    ("stiffness", ("Solver",), "stiffness", "float", 50000.0),   # rotating-patch IC only
    ("allowNegativePressure", ("Solver",), "allowNegativePressure", "bool", False),
    ("DISPLACEMENT_POSITIONS", ("Solver",), "displacementPositions", "bool", True),
    ("COMPENSATED_VOLUME", ("Solver",), "compensatedVolume", "bool", True),
    ("BULK_VISCOSITY_Q", ("Solver", "bulkViscosity"), "quadratic", "float", 0.0),
    ("BULK_VISCOSITY_LENGTH", ("Solver", "bulkViscosity"), "lengthScale", "str", "dx0"),
    ("MONAGHAN_ALPHA", ("Solver", "artificialViscosity"), "alpha", "float", 0.0),
    ("MONAGHAN_BETA", ("Solver", "artificialViscosity"), "beta", "float", 0.0),
    ("MONAGHAN_EPS", ("Solver", "artificialViscosity"), "epsilon", "float", 0.01),
    ("dampingCoefficient", ("Solver",), "dampingCoefficient", "float", 0.0),
    ("OBJECTIVE_RATE", ("Solver",), "objectiveRate", "str", "jaumann"),
    ("KERNEL_CORRECTION", ("Solver",), "kernelCorrection", "bool", False),
    ("L_EIG_TOL", ("Solver",), "lEigTol", "float", 0.1),
    ("TRACK_VISCOUS_WORK", ("Solver",), "trackViscousWork", "bool", True),
    ("gravitation", ("Load",), "gravitation", "vec3", None),
    ("rampTime", ("Load",), "rampTime", "float", 0.0),
    ("DELTA_SPH", ("Diffusion",), "delta", "float", 0.0),
    ("DELTA_PAIRS", ("Diffusion",), "pairs", "str", "samematerial"),
    ("PST_ENABLED", ("Shifting",), "enabled", "bool", True),
    ("PST_MODE", ("Shifting",), "mode", "str", "sun"),
    ("PST_MA_MODE", ("Shifting",), "maMode", "str", "local"),
    ("PST_MA_FIXED", ("Shifting",), "maFixed", "float", 0.1),
    ("PST_R", ("Shifting",), "R", "float", 0.2),
    ("PST_N", ("Shifting",), "n", "int", 4),
    ("PST_MAX_SHIFT", ("Shifting",), "maxShift", "float", 0.05),
    ("PST_SURFACE_SHIFT", ("Shifting",), "surfaceShift", "str", "tangential"),
    ("PST_LAMBDA_LO", ("Shifting",), "lambdaLo", "float", _lambda_lo_default),
    ("PST_LAMBDA_HI", ("Shifting",), "lambdaHi", "float", 0.75),
    ("PST_NORMAL", ("Shifting",), "normal", "str", "gradlam"),
    ("PST_CLAMP", ("Shifting",), "clamp", "str", _clamp_default),
    ("PST_M_DELTA", ("Shifting",), "mDelta", "float", 0.4),
    ("PST_ALE_MOMENTUM", ("Shifting",), "aleMomentum", "bool", True),
    ("PST_ALE_HISTORY", ("Shifting",), "aleHistory", "bool", True),
    ("PST_ALE_DIFFUSION", ("Shifting",), "aleDiffusion", "float", 1.0),
    ("L_EIG_TOL_LAM", ("Shifting",), "lEigTolLam", "float", 0.02),
    ("PST_GRIP_HOLD", ("Shifting",), "gripHold", "float", 0.0),
    ("PST_RELAX_STEPS", ("Shifting",), "initialRelaxation", "int", 0),
    ("PST_RELAX_TOL", ("Shifting",), "initialRelaxationTolerance", "float", 0.03),
    ("exportRelaxationNetcdf", ("Output",), "relaxationNetcdf", "bool", False),
    ("exportRelaxationInterval", ("Output",), "relaxationInterval", "int", 1),
    ("HOURGLASS_ALPHA", ("Hourglass",), "alpha", "float", 0.0),
    ("HOURGLASS_FORM", ("Hourglass",), "form", "str", "rate"),
    ("HOURGLASS_STS_MODE", ("Hourglass", "superTimeStepping"), "mode", "str", "subcycle"),
    ("HOURGLASS_STS_STAGES", ("Hourglass", "superTimeStepping"), "stages", "int", 0),
    ("HOURGLASS_STS_REFRESH", ("Hourglass", "superTimeStepping"), "refreshGradV", "bool", True),
    ("HOURGLASS_STS_SAFETY", ("Hourglass", "superTimeStepping"), "safety", "float", 0.8),
]

# Values that select a branch this package does not implement: a SceneError names them.
UNSUPPORTED = {
    "PST_SURFACE_SHIFT": None,
    "DOMAIN_BOUNDARY": ("open", "reflect"),
    "simulationMethod": ("deltaPlusSPH", "hypoElastic"),
    "PST_MODE": ("sun", "colle"),
    "PST_MA_MODE": ("local", "global", "fixed"),
    "PST_CLAMP": ("displacement", "velocity", "both"),
    "PST_NORMAL": ("gradlam", "eigvec"),
    "DT_PAIR_SOUND_SPEED": ("all", "samematerial", "off"),
    "DELTA_PAIRS": ("samematerial", "all"),
    "OBJECTIVE_RATE": ("jaumann", "none"),
    "HOURGLASS_FORM": ("rate",),
    "HOURGLASS_STS_MODE": ("subcycle", "rkl"),
    "BULK_VISCOSITY_LENGTH": ("dx0", "h"),
    "AXI_IMAGE_RADIUS": ("ring", "signed"),
}

# Cards the format knows, and those whose content is accepted but not read here
# (output switches of the reference's driver, which this package does not replace).
KNOWN_CARDS = {"Domain", "Time", "Solver", "Materials", "Load", "Diffusion", "Shifting",
               "Hourglass", "Output", "FluidBlocks", "SolidBlocks", "Constraints", "ParticlesFile"}
OUT_OF_SCOPE_CARDS = {"Burn", "Detonators", "VelocityLimit", "Erosion"}


def _coerce(kind, value, path):
    try:
        if kind == "float":
            return None if value is None else float(value)
        if kind == "int":
            return None if value is None else int(value)
        if kind == "bool":
            if isinstance(value, bool):
                return value
            raise SceneError(f"{path}: expected true/false, got {value!r}")
        if kind == "str":
            return None if value is None else str(value)
        if kind == "vec3":
            v = [float(t) for t in value]
            if len(v) != 3:
                raise SceneError(f"{path}: expected three numbers")
            return v
    except (TypeError, ValueError) as e:
        raise SceneError(f"{path}: {e}")
    return value


class SimConfig:
    """The resolved scene (config_builder.SimConfig, config_builder.py:174-1410)."""

    def __init__(self, scene_file_path, verbose=False, overrides=None):
        self.path = scene_file_path
        if isinstance(scene_file_path, dict):
            raw = json.loads(json.dumps(scene_file_path))
        else:
            ext = os.path.splitext(scene_file_path)[1].lower()
            try:
                if ext == ".toml":
                    with open(scene_file_path, "rb") as fh:
                        raw = tomllib.load(fh)
                else:
                    with open(scene_file_path, "r", encoding="utf-8") as fh:
                        raw = json.loads(strip_json_comments(fh.read()))
            except json.JSONDecodeError as e:
                raise SceneError(f"{scene_file_path}: invalid JSON: {e}")
        if not isinstance(raw, dict):
            raise SceneError("the scene must be a JSON or TOML object")
        self.raw = raw
        errors = []
        for card in raw:
            if card in OUT_OF_SCOPE_CARDS:
                errors.append(f"{card}: not implemented by sigmasph_b200 (outside the fluid "
                              "and tensile-solid hot path)")
            elif card not in KNOWN_CARDS:
                errors.append(f"unknown card {card!r}")
        given = self._read_cards(raw, errors)
        if overrides:
            given.update(overrides)
        self.materials = self._build_materials(raw, given, errors)
        resolved = dict(given)
        for name, card, field, kind, default in REGISTRY:
            if name not in resolved and not callable(default):
                resolved[name] = default
        for name, card, field, kind, default in REGISTRY:
            if name not in resolved and callable(default):
                resolved[name] = default(resolved)
        resolved.update(derive_globals(self.materials))
        for req in ("particleRadius", "CFL", "simulationMethod", "viscosity", "gravitation"):
            if resolved.get(req) is None:
                errors.append(f"missing required parameter {req}")
        for name, allowed in UNSUPPORTED.items():
            v = resolved.get(name)
            if allowed is None:
                continue
            if isinstance(v, str):
                v = v.lower()
            if v not in [a.lower() if isinstance(a, str) else a for a in allowed]:
                errors.append(f"{name} = {resolved.get(name)!r} is not implemented by "
                              f"sigmasph_b200 (supported: {allowed})")
        if str(resolved.get("PST_SURFACE_SHIFT", "tangential")).lower() not in ("tangential", "none"):
            errors.append("Shifting.surfaceShift must be 'tangential' or 'none'")
        if float(resolved.get("PST_GRIP_HOLD") or 0.0) > 0.0:
            errors.append("Shifting.gripHold is not implemented by sigmasph_b200")
        if float(resolved.get("dampingCoefficient") or 0.0) != 0.0:
            errors.append("Solver.dampingCoefficient is not implemented by sigmasph_b200")
        if int(resolved.get("HOURGLASS_STS_STAGES") or 0) > 32:
            # the device runs at most 32 damper stages per step (the reference's automatic
            # count stops there too; only a fixed RKL count can ask for more)
            errors.append("Hourglass.superTimeStepping.stages above 32 is not implemented by "
                          "sigmasph_b200")
        if resolved.get("simulationMethod") == "deltaPlusSPH":
            if len(self.materials) > 1:
                errors.append("a deltaPlusSPH deck has exactly one material")
        self._check_blocks(raw, errors, has_particles_file="ParticlesFile" in raw)
        if errors:
            raise SceneError("%s: %d problem%s in the scene file:\n  - %s" % (
                os.path.basename(str(scene_file_path)), len(errors),
                "" if len(errors) == 1 else "s", "\n  - ".join(errors)))
        self.config = {"Configuration": resolved}
        for section in ("FluidBlocks", "SolidBlocks", "Constraints"):
            if section in raw:
                self.config[section] = raw[section]
        if "ParticlesFile" in raw:
            # a relative path is taken from the working directory, as the reference does,
            # else from the scene file's directory
            pf = str(raw["ParticlesFile"])
            if (not os.path.isabs(pf) and not os.path.exists(pf) and isinstance(scene_file_path, str)):
                alt = os.path.join(os.path.dirname(os.path.abspath(scene_file_path)), pf)
                if os.path.exists(alt):
                    pf = alt
            resolved["ParticlesFile"] = pf

    # ------------------------------------------------------------------ reading
    def _read_cards(self, raw, errors):
        by_path = {}
        for name, card, field, kind, default in REGISTRY:
            by_path.setdefault(card, {})[field] = (name, kind)
        given = {}
        ignored = {("Time",): {"maxSteps", "stepsPerRenderUpdate"}}

        def walk(node, card):
            table = by_path.get(card, {})
            for key, val in node.items():
                if isinstance(val, dict) and (card + (key,)) in by_path:
                    walk(val, card + (key,))
                    continue
                if key in table:
                    name, kind = table[key]
                    given[name] = _coerce(kind, val, ".".join(card + (key,)))
                    continue
                if key in ignored.get(card, set()):
                    continue
                # The reference knows more keys in these cards; name them precisely.
                errors.append(f"{'.'.join(card + (key,))}: not a parameter sigmasph_b200 "
                              "implements")

        for card in ("Domain", "Time", "Solver", "Load", "Diffusion", "Shifting", "Hourglass"):
            node = raw.get(card)
            if node is None:
                continue
            if not isinstance(node, dict):
                errors.append(f"{card}: expected an object")
                continue
            walk(node, (card,))
        # Output is the reference driver's card; only the relaxation dump's two switches
        # (params.py:1245-1263) are read here, the rest is accepted as written
        out = raw.get("Output") or {}
        if isinstance(out, dict):
            given["exportRelaxationNetcdf"] = bool(out.get("relaxationNetcdf", False))
            given["exportRelaxationInterval"] = int(out.get("relaxationInterval", 1) or 1)
        # the presence of Hourglass.superTimeStepping is the switch (params.py:1330)
        hg = raw.get("Hourglass") or {}
        given["HOURGLASS_STS"] = bool(isinstance(hg, dict) and "superTimeStepping" in hg)
        return given

    def _build_materials(self, raw, given, errors):
        mats = {}
        entries = raw.get("Materials") or []
        default_delta = given.get("DELTA_SPH")
        for idx, entry in enumerate(entries):
            try:
                m = Material(entry, index=idx, default_delta=0.0 if default_delta is None
                             else default_delta)
            except MaterialError as e:
                errors.append(str(e))
                continue
            if m.name in mats:
                errors.append(f"Materials: duplicate name {m.name!r}")
            mats[m.name] = m
        return mats

    def _check_blocks(self, raw, errors, has_particles_file=False):
        names = set(self.materials)
        # a ParticlesFile deck's blocks only name the objects (no extents to lay)
        required = ("objectId",) if has_particles_file else ("objectId", "start", "end")
        for section in ("FluidBlocks", "SolidBlocks"):
            for b in raw.get(section) or []:
                for req in required:
                    if req not in b:
                        errors.append(f"{section}: block without {req!r}")
                mat = b.get("material")
                if names and mat is not None and mat not in names:
                    errors.append(f"{section}: block material {mat!r} is not declared")
                b.setdefault("translation", [0.0, 0.0, 0.0])
                b.setdefault("scale", [1.0, 1.0, 1.0])
                b.setdefault("velocity", [0.0, 0.0, 0.0])
                b.setdefault("color", [0, 0, 0])
        for c in raw.get("Constraints") or []:
            if "region" not in c:
                errors.append("Constraints: entry without a region")

    # ------------------------------------------------------------------ API
    def get_cfg(self, name, enforce_exist=False):
        if enforce_exist and name not in self.config["Configuration"]:
            raise KeyError(name)
        return self.config["Configuration"].get(name)

    def get_fluid_blocks(self):
        return self.config.get("FluidBlocks", [])

    def get_solid_blocks(self):
        return self.config.get("SolidBlocks", [])

    def get_materials(self):
        return self.materials

    def get_constraints(self):
        return self.config.get("Constraints", [])

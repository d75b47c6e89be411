"""Material constants of a scene (materials.py and material_models/ of the reference).

A `Materials[]` entry is a reference density, an equation of state and, for a solid, a
strength model.  Derived constants follow the reference's derivations
(materials.py:136-330, material_models/EOS000_linear.py, EOS001_tait.py,
MAT001_linear_plasticity.py, MAT002_johnson_cook.py):

  K = E / (3 (1 - 2 nu)),  G = E / (2 (1 + nu))          elastic_constants
  c_eos = sqrt(K / rho0)  (linear),  c0 given (Tait, K = c0^2 rho0)
  c_p = sqrt((K + 4 G / 3) / rho0)                        dilatational speed
  sigma_y0, H from yieldStress | yieldStrain and hardeningModulus | tangentModulusRatio
"""
from __future__ import annotations

import copy
import math

EOS_LINEAR, EOS_TAIT = 0, 1
PLASTIC_NONE, PLASTIC_LINEAR, PLASTIC_JOHNSON_COOK = 0, 1, 2


class MaterialError(ValueError):
    """A declared material whose constants cannot be resolved as written."""


# Library presets (material_models/material_library.py), the published constants the
# shipped decks name.  Units: mm, GPa, ms, kg.
LIBRARY = {
    "stainless_steel": {
        "density0": 7.90e-06,
        "specificHeat": 500.0,
        "eos": {"type": "linear"},
        "strength": {
            "type": "hypoElastic",
            "youngsModulus": 193.0,
            "poissonRatio": 0.30,
            "plasticity": {
                "model": "johnson_cook",
                "A": 0.310, "B": 1.000, "n": 0.65, "C": 0.020, "eps0_dot": 0.001,
                "T0": 293.0, "Tm": 1720.0, "m": 1.00, "Cp": 500.0, "chi": 0.9,
                "yieldStress": 0.310, "hardeningModulus": 1.0,
            },
        },
    },
}


def _deep_merge(base, over):
    out = copy.deepcopy(base)
    for k, v in over.items():
        if isinstance(v, dict) and isinstance(out.get(k), dict):
            out[k] = _deep_merge(out[k], v)
        else:
            out[k] = copy.deepcopy(v)
    return out


def elastic_constants(E, nu):
    E, nu = float(E), float(nu)
    return E / (3.0 * (1.0 - 2.0 * nu)), E / (2.0 * (1.0 + nu))


class Material:
    """One resolved `Materials[]` entry."""

    def __init__(self, entry, index=0, default_delta=0.0):
        if not isinstance(entry, dict):
            raise MaterialError("Materials: each entry must be an object")
        name = entry.get("name")
        if not name:
            raise MaterialError("Materials: every entry needs a name")
        where = f"Materials[{name!r}]"
        lib = entry.get("library")
        if lib is not None:
            if lib not in LIBRARY:
                raise MaterialError(f"{where}: library preset {lib!r} is not available "
                                    f"(known: {sorted(LIBRARY)})")
            entry = _deep_merge(LIBRARY[lib], {k: v for k, v in entry.items() if k != "library"})
        allowed = {"name", "density0", "delta", "specificHeat", "eos", "strength", "damage"}
        for k in entry:
            if k not in allowed:
                raise MaterialError(f"{where}.{k}: not a key sigmasph_b200 implements")
        self.name = name
        self.index = index
        try:
            self.rho0 = float(entry["density0"])
        except (KeyError, TypeError, ValueError):
            raise MaterialError(f"{where}: density0 is required and must be a number")
        if not self.rho0 > 0.0:
            raise MaterialError(f"{where}: density0 must be positive")
        d = entry.get("delta")
        self.delta = float(default_delta if d is None else d)
        self.specific_heat = float(entry.get("specificHeat") or 0.0)
        dmg = entry.get("damage")
        if dmg and str(dmg.get("model", "none")).lower() != "none":
            raise MaterialError(f"{where}.damage: damage models are outside the hot path "
                                "sigmasph_b200 implements")
        eos = entry.get("eos") or {}
        kind = str(eos.get("type", "linear")).lower()
        if kind not in ("linear", "tait"):
            raise MaterialError(f"{where}.eos: type {kind!r} is not implemented by "
                                "sigmasph_b200 (linear, tait)")
        self.eos_kind = EOS_LINEAR if kind == "linear" else EOS_TAIT
        strength = entry.get("strength")
        self.has_strength = strength is not None
        self.plastic_kind = PLASTIC_NONE
        self.sigma_y0 = 0.0
        self.hardening = 0.0
        self.jc = None
        K_from_E = None
        if self.has_strength:
            E = strength.get("youngsModulus")
            nu = strength.get("poissonRatio")
            if E is None or nu is None:
                raise MaterialError(f"{where}.strength: youngsModulus and poissonRatio are "
                                    "required")
            K_from_E, self.G = elastic_constants(E, nu)
            self.E = float(E)
            plast = strength.get("plasticity")
            if plast:
                model = str(plast.get("model", "linear")).lower()
                if model == "johnson_cook":
                    for req in ("A", "B", "n"):
                        if plast.get(req) is None:
                            raise MaterialError(f"{where}.strength.plasticity: {req} is required")
                    self.jc = {
                        "A": float(plast["A"]), "B": float(plast["B"]), "n": float(plast["n"]),
                        "C": float(plast.get("C") or 0.0),
                        "eps0_dot": float(plast.get("eps0_dot", 0.001)),
                        "T0": float(plast.get("T0", 293.0)),
                        "Tm": float(plast.get("Tm", 0.0)),
                        "m": float(plast.get("m", 1.0)),
                        "chi": float(plast.get("chi", 0.9)),
                    }
                    if self.specific_heat == 0.0 and plast.get("Cp") is not None:
                        self.specific_heat = float(plast["Cp"])
                    self.plastic_kind = PLASTIC_JOHNSON_COOK
                    self.sigma_y0 = self.jc["A"]
                    self.hardening = self.jc["B"]
                elif model == "linear":
                    sy = plast.get("yieldStress")
                    ey = plast.get("yieldStrain")
                    if sy is None and ey is not None:
                        sy = float(E) * float(ey)
                    H = plast.get("hardeningModulus")
                    r = plast.get("tangentModulusRatio")
                    if H is None and r is not None:
                        r = float(r)
                        H = float(E) * r / (1.0 - r)
                    self.sigma_y0 = float(sy or 0.0)
                    self.hardening = float(H or 0.0)
                    self.plastic_kind = PLASTIC_LINEAR if self.sigma_y0 > 0.0 else PLASTIC_NONE
                else:
                    raise MaterialError(f"{where}.strength.plasticity: model {model!r} is not "
                                        "implemented by sigmasph_b200")
        else:
            self.G = 0.0
            self.E = 0.0
        if self.eos_kind == EOS_LINEAR:
            if K_from_E is not None:
                self.K = K_from_E
            else:
                K = eos.get("bulkModulus")
                if K is None:
                    raise MaterialError(f"{where}.eos: a linear EOS without a strength model "
                                        "needs bulkModulus")
                self.K = float(K)
            self.c_eos = math.sqrt(self.K / self.rho0)
            self.exponent = 1.0
            self.stiffness = self.K
        else:
            c0 = eos.get("c0")
            gam = eos.get("exponent")
            if c0 is None or gam is None:
                raise MaterialError(f"{where}.eos: a Tait equation of state needs c0 and exponent")
            c0, gam = float(c0), float(gam)
            if not (c0 > 0.0 and gam > 0.0):
                raise MaterialError(f"{where}.eos: c0 and exponent must both be positive")
            self.stiffness = c0 * c0 * self.rho0 / gam
            self.exponent = gam
            self.K = c0 * c0 * self.rho0
            self.c_eos = c0
        self.c_p = math.sqrt((self.K + 4.0 * self.G / 3.0) / self.rho0)


def derive_globals(materials):
    """Scene-wide c0, density0 and exponent from the declared materials
    (materials.py:551-604)."""
    if not materials:
        return {}
    mats = list(materials.values())
    out = {"c0": float(max(m.c_eos for m in mats)),
           "density0": float(max(m.rho0 for m in mats))}
    if len(mats) == 1 and not mats[0].has_strength:
        out["exponent"] = float(mats[0].exponent)
    else:
        out["exponent"] = 1.0
    return out

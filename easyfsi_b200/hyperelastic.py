"""Compressible neo-Hookean material card (simulation_core/hyperelastic.py:26-118).

Host-side parameter conversion only: ``lame_lambda_pa = K - 2 mu / 3`` and the
Young's-modulus constructor, as the reference defines them.
"""

from __future__ import annotations

from dataclasses import dataclass
from math import sqrt


@dataclass(frozen=True)
class NeoHookeanMaterial:
    name: str
    density_kgm3: float
    shear_modulus_pa: float
    bulk_modulus_pa: float
    youngs_modulus_pa: float
    poissons_ratio: float
    source: str = ""
    calibration_note: str = ""

    @property
    def lame_lambda_pa(self) -> float:
        return self.bulk_modulus_pa - (2.0 / 3.0) * self.shear_modulus_pa

    @property
    def sound_speed_mps(self) -> float:
        return sqrt((self.bulk_modulus_pa + (4.0 / 3.0) * self.shear_modulus_pa) / self.density_kgm3)

    def stable_explicit_dt_s(self, spacing_m: float, cfl: float = 0.35) -> float:
        if spacing_m <= 0.0:
            raise ValueError("spacing_m must be positive")
        if cfl <= 0.0:
            raise ValueError("cfl must be positive")
        return float(cfl) * float(spacing_m) / self.sound_speed_mps

    def validate(self) -> None:
        if self.density_kgm3 <= 0.0:
            raise ValueError("density_kgm3 must be positive")
        if self.shear_modulus_pa <= 0.0:
            raise ValueError("shear_modulus_pa must be positive")
        if self.bulk_modulus_pa <= 0.0:
            raise ValueError("bulk_modulus_pa must be positive")
        if not 0.0 <= self.poissons_ratio < 0.5:
            raise ValueError("poissons_ratio must be in [0, 0.5)")

    @classmethod
    def from_youngs_modulus(cls, *, name: str, density_kgm3: float, youngs_modulus_pa: float, poissons_ratio: float,
                            source: str = "", calibration_note: str = "") -> "NeoHookeanMaterial":
        e, nu = float(youngs_modulus_pa), float(poissons_ratio)
        mat = cls(
            name=name,
            density_kgm3=float(density_kgm3),
            shear_modulus_pa=e / (2.0 * (1.0 + nu)),
            bulk_modulus_pa=e / (3.0 * (1.0 - 2.0 * nu)),
            youngs_modulus_pa=e,
            poissons_ratio=nu,
            source=source,
            calibration_note=calibration_note,
        )
        mat.validate()
        return mat


def lame_parameters(youngs_modulus_pa: float, poissons_ratio: float) -> tuple[float, float]:
    """(mu, lambda) of E and nu, as the marker-MPM runner computes them
    (benchmarking/solid_mpm_fsi_runner.py:_lame_parameters)."""
    e, nu = float(youngs_modulus_pa), float(poissons_ratio)
    return e / (2.0 * (1.0 + nu)), e * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))

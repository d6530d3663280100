"""Host-side configuration types: the Python mirror of BirdFlowCore.

Mirrors (Numi2/numi-gpu-physics):
  GridSize, LatticeScaling, SimulationConfiguration  Sources/BirdFlowCore/SimulationConfiguration.swift
  WingKinematics, BirdBodyState, BirdParameters       Sources/BirdFlowCore/BirdModel.swift
  BirdFlowConfigurationError                          SimulationConfiguration.swift:3-24

Scalars are computed in float32, as the reference computes them in Swift
Float, so the relaxation rates and unit scales handed to the GPU are the same
numbers the reference would pack into GPUUniforms.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

f32 = np.float32
D3Q19_SOUND_SPEED = float(np.sqrt(f32(1.0) / f32(3.0)))


class BirdFlowConfigurationError(ValueError):
    """invalidGrid / invalidPhysicalScale / latticeMachTooHigh / relaxationTooCloseToLimit."""

    def __init__(self, kind: str, message: str):
        super().__init__(message)
        self.kind = kind


@dataclass(frozen=True)
class GridSize:
    """Lattice extent (SimulationConfiguration.swift:27-52): >= 16 per axis, <= 2^32-1 cells."""
    x: int
    y: int
    z: int

    def __post_init__(self):
        if self.x < 16 or self.y < 16 or self.z < 16:
            raise BirdFlowConfigurationError(
                "invalidGrid", "Each grid dimension must be at least 16 cells and the total cell count must fit in UInt32.")
        if self.x * self.y * self.z > 0xFFFFFFFF:
            raise BirdFlowConfigurationError(
                "invalidGrid", "Each grid dimension must be at least 16 cells and the total cell count must fit in UInt32.")

    @property
    def cell_count(self) -> int:
        return self.x * self.y * self.z


@dataclass(frozen=True)
class LatticeScaling:
    """Physical <-> lattice scales (SimulationConfiguration.swift:55-197)."""
    cell_size_meters: float
    time_step_seconds: float
    lattice_reference_speed: float
    lattice_kinematic_viscosity: float
    tau_plus: float
    tau_minus: float
    omega_plus: float
    omega_minus: float
    velocity_to_lattice: float
    velocity_to_physical: float
    pressure_scale_pascals: float
    force_to_physical: float
    torque_to_physical: float
    lattice_mach: float

    @staticmethod
    def make(characteristic_length_meters: float, characteristic_length_cells: int,
             reference_speed_meters_per_second: float, target_reynolds_number: float,
             physical_air_density: float, lattice_reference_speed: float = 0.05,
             trt_magic_parameter: float = 3.0 / 16.0, minimum_tau_plus: float = 0.50005) -> "LatticeScaling":
        L, N, U = f32(characteristic_length_meters), int(characteristic_length_cells), f32(reference_speed_meters_per_second)
        Re, rho, ul, lam = f32(target_reynolds_number), f32(physical_air_density), f32(lattice_reference_speed), f32(trt_magic_parameter)
        if not (L > 0 and N >= 8 and U > 0 and Re > 0 and rho > 0 and ul > 0 and lam > 0):
            raise BirdFlowConfigurationError("invalidPhysicalScale", "All physical and lattice scale values must be positive.")
        mach = ul / f32(D3Q19_SOUND_SPEED)
        if mach > f32(0.15):
            raise BirdFlowConfigurationError("latticeMachTooHigh", f"The estimated lattice Mach number is {mach}; keep it at or below 0.15.")
        dx = L / f32(N)
        dt = ul * dx / U
        nu = ul * f32(N) / Re
        tau_p = f32(0.5) + f32(3) * nu
        if tau_p < f32(minimum_tau_plus):
            raise BirdFlowConfigurationError("relaxationTooCloseToLimit", f"The TRT symmetric relaxation time is {tau_p}.")
        tau_m = f32(0.5) + lam / (tau_p - f32(0.5))
        force = rho * f32(float(dx) ** 4) / f32(float(dt) ** 2)
        return LatticeScaling(
            cell_size_meters=float(dx), time_step_seconds=float(dt), lattice_reference_speed=float(ul),
            lattice_kinematic_viscosity=float(nu), tau_plus=float(tau_p), tau_minus=float(tau_m),
            omega_plus=float(f32(1) / tau_p), omega_minus=float(f32(1) / tau_m),
            velocity_to_lattice=float(dt / dx), velocity_to_physical=float(dx / dt),
            pressure_scale_pascals=float(rho * f32(float(dx / dt) ** 2)),
            force_to_physical=float(force), torque_to_physical=float(force * dx), lattice_mach=float(mach))

    @staticmethod
    def lattice_only(viscosity: float, magic: float = 0.25) -> "LatticeScaling":
        """Pure lattice units (dx = dt = 1): tau+ = 0.5 + 3 nu, tau- = 0.5 + magic / (tau+ - 0.5)."""
        nu = f32(viscosity)
        tau_p = f32(0.5) + f32(3) * nu
        tau_m = f32(0.5) + f32(magic) / (tau_p - f32(0.5))
        return LatticeScaling(1.0, 1.0, 0.0, float(nu), float(tau_p), float(tau_m), float(f32(1) / tau_p),
                              float(f32(1) / tau_m), 1.0, 1.0, 1.0, 1.0, 1.0, 0.0)

    @property
    def physical_air_density(self) -> float:
        return self.pressure_scale_pascals / (self.velocity_to_physical * self.velocity_to_physical)


@dataclass
class WingKinematics:
    """Sinusoidal stroke and pitch (BirdModel.swift:4-44)."""
    frequency_hz: float
    stroke_amplitude_radians: float
    stroke_bias_radians: float = 0.0
    pitch_mean_radians: float = 0.0
    pitch_amplitude_radians: float = 0.0
    pitch_phase_radians: float = 0.0
    # bfx extension: deviation about the stroke-plane normal, amplitude * sin(2 * phase)
    deviation_amplitude_radians: float = 0.0


@dataclass
class BirdBodyState:
    """BirdModel.swift:53-68 (orientation as x, y, z, w)."""
    position_meters: tuple = (0.0, 0.0, 0.0)
    orientation_body_to_world: tuple = (0.0, 0.0, 0.0, 1.0)
    linear_velocity_meters_per_second: tuple = (0.0, 0.0, 0.0)
    angular_velocity_body_radians_per_second: tuple = (0.0, 0.0, 0.0)


@dataclass
class WingInertialProperties:
    mass_kilograms: float
    center_of_mass_from_hinge_meters: tuple
    principal_inertia_kilogram_meters_squared: tuple


@dataclass
class BirdParameters:
    """BirdModel.swift:129-213; packed as GPUBirdParameters (GPUData.swift:82-178)."""
    body_radii_meters: tuple
    mass_kilograms: float
    principal_inertia_kilogram_meters_squared: tuple
    wing_span_meters: float
    wing_root_chord_meters: float
    wing_tip_chord_meters: float
    wing_thickness_meters: float
    wing_sweep_meters: float
    wing_root_offset_meters: tuple
    tail_length_meters: float
    tail_half_width_meters: float
    tail_thickness_meters: float
    wing_kinematics: WingKinematics
    left_wing: WingInertialProperties | None = None
    right_wing: WingInertialProperties | None = None

    @staticmethod
    def demonstration() -> "BirdParameters":
        r = math.radians
        return BirdParameters(
            body_radii_meters=(0.18, 0.065, 0.075), mass_kilograms=0.42,
            principal_inertia_kilogram_meters_squared=(0.0024, 0.0068, 0.0074),
            wing_span_meters=0.34, wing_root_chord_meters=0.14, wing_tip_chord_meters=0.055,
            wing_thickness_meters=0.018, wing_sweep_meters=0.055, wing_root_offset_meters=(0.02, 0.055, 0.02),
            tail_length_meters=0.17, tail_half_width_meters=0.11, tail_thickness_meters=0.018,
            wing_kinematics=WingKinematics(4.5, float(f32(r(42))), float(f32(r(2))), float(f32(r(8))),
                                           float(f32(r(24))), float(f32(r(78)))))

    def conservative_local_half_extent(self) -> tuple:
        """BirdModel.swift:215-255 (sinusoidal branch)."""
        max_chord = max(self.wing_root_chord_meters, self.wing_tip_chord_meters)
        k = self.wing_kinematics
        max_stroke = abs(k.stroke_bias_radians) + abs(k.stroke_amplitude_radians)
        ro = self.wing_root_offset_meters
        wx = abs(ro[0]) + abs(self.wing_sweep_meters) + 0.5 * max_chord
        wy = abs(ro[1]) + self.wing_span_meters + 0.5 * self.wing_thickness_meters
        wz = abs(ro[2]) + self.wing_span_meters * min(1.0, abs(math.sin(max_stroke))) + 0.5 * max_chord + \
            0.5 * self.wing_thickness_meters
        br = self.body_radii_meters
        return (max(br[0] + self.tail_length_meters, wx),
                max(max(br[1], self.tail_half_width_meters), wy),
                max(br[2] + 0.5 * self.tail_thickness_meters, wz))

    def conservative_bounding_radius(self) -> float:
        e = self.conservative_local_half_extent()
        return math.sqrt(e[0] ** 2 + e[1] ** 2 + e[2] ** 2)

    def maximum_prescribed_wing_speed(self) -> float:
        k = self.wing_kinematics
        w = 2 * math.pi * k.frequency_hz
        return w * abs(k.stroke_amplitude_radians) * self.wing_span_meters + \
            w * abs(k.pitch_amplitude_radians) * max(self.wing_root_chord_meters, self.wing_tip_chord_meters)

    def packed(self) -> list:
        """The 13 float4 rows of GPUBirdParameters."""
        k = self.wing_kinematics
        ext = self.conservative_local_half_extent()
        rows = [
            (*self.body_radii_meters, self.mass_kilograms),
            (*self.principal_inertia_kilogram_meters_squared, 0.0),
            (self.wing_span_meters, self.wing_root_chord_meters, self.wing_tip_chord_meters, self.wing_thickness_meters),
            (self.wing_sweep_meters, *self.wing_root_offset_meters),
            (self.tail_length_meters, self.tail_half_width_meters, self.tail_thickness_meters, 0.0),
            (k.frequency_hz, k.stroke_amplitude_radians, k.stroke_bias_radians, k.pitch_mean_radians),
            (k.pitch_amplitude_radians, k.pitch_phase_radians, k.deviation_amplitude_radians, 0.0),
            (*ext, self.conservative_bounding_radius()),
            (self.maximum_prescribed_wing_speed(), 0.15, 0.0, 0.0),
        ]
        for wing in (self.left_wing, self.right_wing):
            if wing is None:
                rows += [(0.0, 0.0, 0.0, 0.0), (0.0, 0.0, 0.0, 0.0)]
            else:
                rows += [(wing.mass_kilograms, *wing.center_of_mass_from_hinge_meters),
                         (*wing.principal_inertia_kilogram_meters_squared, 1.0)]
        if self.left_wing is None or self.right_wing is None:
            rows[9] = rows[10] = rows[11] = rows[12] = (0.0, 0.0, 0.0, 0.0)
        return rows

    def validate(self, configuration: "SimulationConfiguration") -> None:
        """BirdModel.swift:278-365 (dimension checks)."""
        dx = configuration.scaling.cell_size_meters
        ok = (self.mass_kilograms > 0 and min(self.body_radii_meters) > 0 and
              min(self.principal_inertia_kilogram_meters_squared) > 0 and self.wing_span_meters > 0 and
              self.wing_root_chord_meters > 0 and self.wing_tip_chord_meters > 0 and
              self.wing_thickness_meters >= 1.5 * dx and self.tail_length_meters > 0 and
              self.tail_half_width_meters > 0 and self.tail_thickness_meters >= 1.5 * dx and
              self.wing_kinematics.frequency_hz >= 0)
        if not ok:
            raise BirdFlowConfigurationError(
                "invalidPhysicalScale",
                "Bird dimensions, mass, inertia, and wing frequency must be positive; thin surfaces must be at least 1.5 grid cells thick.")


@dataclass
class SimulationConfiguration:
    """SimulationConfiguration.swift:199-260."""
    grid: GridSize
    domain_origin_meters: tuple
    scaling: LatticeScaling
    physical_air_density: float = 1.225
    far_field_velocity_meters_per_second: tuple = (0.0, 0.0, 0.0)
    sponge_width_cells: int = 12
    sponge_strength: float = 0.08
    free_flight: bool = False
    body_substeps: int = 1
    gravity_meters_per_second_squared: tuple = (0.0, 0.0, -9.80665)
    fast_math: bool = False

    def __post_init__(self):
        g = self.grid
        if not (self.physical_air_density > 0 and
                abs(self.scaling.physical_air_density - self.physical_air_density) <= max(1e-6, self.physical_air_density * 1e-5) and
                self.sponge_width_cells >= 4 and self.sponge_width_cells * 2 < min(g.x, g.y, g.z) and
                0 <= self.sponge_strength <= 1 and 1 <= self.body_substeps <= 64):
            raise BirdFlowConfigurationError(
                "invalidPhysicalScale",
                "Air density must match the lattice scaling density, sponge settings must remain inside their valid ranges, and bodySubsteps must be in 1...64.")
        v = self.far_field_velocity_meters_per_second
        speed = math.sqrt(sum(c * c for c in v)) * self.scaling.velocity_to_lattice
        if speed / D3Q19_SOUND_SPEED > 0.15:
            raise BirdFlowConfigurationError("latticeMachTooHigh", f"far-field lattice Mach {speed / D3Q19_SOUND_SPEED}")

    @property
    def domain_size_meters(self) -> tuple:
        dx = self.scaling.cell_size_meters
        return (self.grid.x * dx, self.grid.y * dx, self.grid.z * dx)

"""Generates the golden fixtures that pin the CPU oracle to the reference.

Run in a container where the reference project is mounted (it is read, never
modified; the NumPy reference is imported from a temporary copy so that no
bytecode is written next to it):

    python tests/golden/make_golden.py /path/to/numi-gpu-physics

Outputs (committed):
  shear_wave_ref_n12_s8.npz  FP64 populations of Reference/shear_wave_reference.py
                             after 8 steps on a 12^3 periodic lattice
                             (nu=0.03, amplitude 0.01, magic 3/16), layout
                             [q, x, y, z] as the NumPy reference stores it.
  shear_wave_ref_metrics.json  run_case() results for the default 32^3 x 120
                             case and the 4-grid convergence ladder of
                             Reference/shear_wave_convergence.py.
"""
from __future__ import annotations

import importlib.util
import json
import math
import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def load_reference(root: str):
    src = os.path.join(root, "Reference", "shear_wave_reference.py")
    tmp = tempfile.mkdtemp()
    dst = os.path.join(tmp, "shear_wave_reference.py")
    shutil.copyfile(src, dst)
    sys.dont_write_bytecode = True
    spec = importlib.util.spec_from_file_location("shear_wave_reference", dst)
    mod = importlib.util.module_from_spec(spec)
    sys.modules["shear_wave_reference"] = mod
    spec.loader.exec_module(mod)
    return mod


def populations_after(ref, resolution: int, steps: int, viscosity: float, amplitude: float,
                      magic: float = 3.0 / 16.0) -> np.ndarray:
    """Replays run_case's loop (shear_wave_reference.py:122-157) keeping the field."""
    tau_plus = 0.5 + 3.0 * viscosity
    tau_minus = 0.5 + magic / (tau_plus - 0.5)
    rho = np.ones((resolution,) * 3)
    velocity = np.zeros((3,) + (resolution,) * 3)
    y = np.arange(resolution, dtype=np.float64)
    velocity[0] = amplitude * np.sin(2.0 * np.pi * y / resolution)[None, :, None]
    pops = ref.equilibrium(rho, velocity)
    for _ in range(steps):
        streamed = ref.stream(pops)
        rho, velocity = ref.moments(streamed)
        pops = ref.collide_trt(streamed, rho, velocity, 1.0 / tau_plus, 1.0 / tau_minus)
    return pops


def main() -> int:
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("BFX_REFERENCE_ROOT")
    if not root:
        print("usage: make_golden.py <reference checkout root> (or set BFX_REFERENCE_ROOT)", file=sys.stderr)
        return 2
    ref = load_reference(root)
    pops = populations_after(ref, 12, 8, 0.03, 0.01)
    np.savez_compressed(os.path.join(HERE, "shear_wave_ref_n12_s8.npz"), populations=pops,
                        resolution=12, steps=8, viscosity=0.03, amplitude=0.01, magic=3.0 / 16.0)
    default = ref.run_case().__dict__
    ladder = []
    for resolution in (12, 16, 24, 32):
        steps = max(1, round(120 * (resolution / 32) ** 2))
        ladder.append(ref.run_case(resolution=resolution, steps=steps).__dict__)
    spacing = np.asarray([1.0 / r["resolution"] for r in ladder])
    errors = np.asarray([r["relative_decay_error"] for r in ladder])
    order = float(np.polyfit(np.log(spacing), np.log(errors), 1)[0])
    with open(os.path.join(HERE, "shear_wave_ref_metrics.json"), "w") as fh:
        json.dump({"default_case": default, "ladder": ladder, "estimated_order": order,
                   "source": "Reference/shear_wave_reference.py run_case, Reference/shear_wave_convergence.py"},
                  fh, indent=2, sort_keys=True)
    print(json.dumps({"order": order, "default": default}, indent=1))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())

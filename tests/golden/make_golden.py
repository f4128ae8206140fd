"""Make the golden fixtures of this directory from the reference's own test data.

Run once in a checkout that has the reference (argument: its root; default /root/reference).
Every fixture is a compressed .npz of numbers the reference's test suite holds or produces:

- green_inf.npz      tests/data/green_inf_reference.txt  (X, Y, Ft, dFt/dX; mpmath, 30 digits)
- green_fin.npz      tests/data/green_fin_reference.txt  (mode h K R z zeta, 8 kernel values, scales)
- panel.npz          tests/data/panel_reference.txt      (R / L rows: 12 vertex coords, point, 2 values)
- dispersion.npz     tests/data/dispersion_reference.txt (H, n, root)
- cylinder_fd.npz    tests/data/cylinder_finite_depth.txt (eigenfunction-matching A, B)
- hulme.npz          tests/data/hulme1982_full.txt (hemisphere A, B, Hulme 1982)
- lo_cylinder_drift.npz  the reference solver's own outputs of that regression problem
  (tests/data/regression/lo_cylinder_drift.npz: A, B, X, FK, SC, the Haskind exciting force, the
  motions (RAO), the Kochin functions with their angular derivatives, the mean drift by momentum
  conservation and the hydrostatics of a floating cylinder with its mass and inertia, f32 / f64 as the
  reference stores them)
- lo_cylinder_field.npz  the reference solver's own field-point outputs of its regression problem
  lo_cylinder_field_body_points (the same cylinder held fixed, three points: the elevation at z = 0
  and p / (rho g) below, per radiation column and heading, complex64)
- lo_cylinder_interior.npz  the reference solver's own outputs of its regression problem
  lo_cylinder_interior (the quarter cylinder of lo_cylinder_drift held fixed, its interior free
  surface generated by the 'graded' method: A, B, X, FK, SC, the Haskind force and the field-point
  velocities at three points, float32 / complex64 as stored)
- meshes.npz         SHA-256 digests and small copies of the reference's procedural meshes
  (tests/python/meshes.py imported from the reference) for the configs' bodies
"""

from __future__ import annotations

import hashlib
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def rows(path: Path):
    out = []
    for line in path.read_text().splitlines():
        s = line.strip()
        if not s or s.startswith("#"):
            continue
        out.append(s.split())
    return out


def main(argv):
    root = Path(argv[1]) if len(argv) > 1 else Path("/root/reference")
    data = root / "tests" / "data"
    r = rows(data / "green_inf_reference.txt")
    np.savez_compressed(HERE / "green_inf.npz", xyff=np.array([[float(t) for t in x[:4]] for x in r]))
    r = rows(data / "green_fin_reference.txt")
    np.savez_compressed(HERE / "green_fin.npz", mode=np.array([int(x[0]) for x in r], np.int32),
                        vals=np.array([[float(t) for t in x[1:16]] for x in r]))
    r = rows(data / "panel_reference.txt")
    np.savez_compressed(HERE / "panel.npz", kind=np.array([x[0] for x in r]),
                        vals=np.array([[float(t) for t in x[1:18]] for x in r]))
    r = rows(data / "dispersion_reference.txt")
    np.savez_compressed(HERE / "dispersion.npz", H=np.array([float(x[0]) for x in r]),
                        n=np.array([int(x[1]) for x in r], np.int32), x=np.array([float(x[2]) for x in r]))
    r = rows(data / "cylinder_finite_depth.txt")
    np.savez_compressed(HERE / "cylinder_fd.npz", vals=np.array([[float(t) for t in x] for x in r]))
    r = rows(data / "hulme1982_full.txt")
    np.savez_compressed(HERE / "hulme.npz", vals=np.array([[float(t) for t in x] for x in r]))
    d = np.load(data / "regression" / "lo_cylinder_drift.npz")
    keep = ["omegas", "headings", "added_mass", "radiation_damping", "excitation_diffraction",
            "excitation_froude_krylov", "excitation_scattering", "excitation_haskind", "motion",
            "radiation_mode_ids", "kochin_angles", "kochin_radiation", "kochin_radiation_derivative",
            "kochin_diffraction", "kochin_diffraction_derivative", "drift_momentum_conservation",
            "drift_heading_pairs", "hydrostatics_volumes",
            "hydrostatics_volume", "hydrostatics_displaced_mass", "hydrostatics_center_of_buoyancy",
            "hydrostatics_waterplane_area", "hydrostatics_waterplane_centroid", "hydrostatics_stiffness_rho_g",
            "hydrostatics_stiffness", "hydrostatics_mass", "hydrostatics_center_of_gravity",
            "hydrostatics_metacentric_height"]
    np.savez_compressed(HERE / "lo_cylinder_drift.npz", **{k: d[k] for k in keep})
    d = np.load(data / "regression" / "lo_cylinder_field_body_points.npz")
    keep = ["omegas", "headings", "field_points", "field_points_pressure_radiation", "field_points_pressure_incident",
            "field_points_pressure_scattering", "field_points_pressure_diffraction"]
    np.savez_compressed(HERE / "lo_cylinder_field.npz", **{k: d[k] for k in keep})
    d = np.load(data / "regression" / "lo_cylinder_interior.npz")
    keep = ["omegas", "headings", "added_mass", "radiation_damping", "excitation_diffraction",
            "excitation_froude_krylov", "excitation_scattering", "excitation_haskind", "field_points",
            "field_points_velocity_radiation", "field_points_velocity_incident",
            "field_points_velocity_scattering", "field_points_velocity_diffraction"]
    np.savez_compressed(HERE / "lo_cylinder_interior.npz", **{k: d[k] for k in keep})
    sys.path.insert(0, str(root / "tests" / "python"))
    import meshes  # the reference's procedural meshes (numpy only)

    cases = {
        "c1": meshes.cylinder_panels(1.0, 0.5, n_phi=32, n_z=8, n_r=8, quarter=False),
        "c2": meshes.cylinder_panels(1.0, 0.5, n_phi=64, n_z=32, n_r=32, quarter=False),
        "drift_quarter": meshes.cylinder_panels(1.0, 0.5, n_phi=8, n_z=4, n_r=4, quarter=True),
        "hemi": meshes.hemisphere_panels(1.0, 8, 8, quarter=True),
        "box_lid": meshes.box_panels(80.0, 20.0, 10.0, n=(8, 4, 3), quarter=False, lid=True),
    }
    out = {}
    for k, v in cases.items():
        v = np.ascontiguousarray(v, dtype="<f8")
        out[k + "_sha256"] = np.array(hashlib.sha256(v.tobytes()).hexdigest())
        out[k + "_shape"] = np.array(v.shape)
        if v.size <= 4096:
            out[k] = v
    np.savez_compressed(HERE / "meshes.npz", **out)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main(sys.argv)
